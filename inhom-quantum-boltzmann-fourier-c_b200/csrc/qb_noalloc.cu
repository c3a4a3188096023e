// qb_noalloc.cu — the I3 integral without any device allocation.
//
// Some callers cannot call cudaMalloc: code that runs while a CUDA graph is
// being captured on its stream, code embedded in a host application that
// owns all device memory through its own allocator or a fixed budget, and
// real-time loops where an allocation (which may synchronise the device)
// would stall.  qb_integral_i3_noalloc serves them: it computes the same I3
// integral as qb_integral(..., which = 3, ...) but takes all of its scratch
// from one fixed array in device global memory that is part of the library
// image, so the call itself allocates nothing.
//
// The array is a file-scope static __device__ object of QB_NOALLOC_SCRATCH_BYTES
// (4 MiB).  Every GPU that loads the library holds it until the process exits.
// Host code cannot use the array's name as a device address: the first call
// on each device looks up its address there with cudaGetSymbolAddress (that
// device current), caches it per device and passes it to the kernels.  Make
// the first call on a device before any stream capture begins, because the
// lookup is not a stream operation.
//
// Every call overwrites the array.  All calls share it, so calls that can
// overlap on the GPU (different streams, different host threads, or a graph
// replayed while another call runs) race and produce garbage; serialise them.
// Each call writes every scratch byte it later reads, so nothing has to be
// cleared between calls.
#include "qb_engine.h"
#include "qb_kernels.cuh"

extern "C" {
#include "qbgpu.h"
}

#include <mutex>

#define QB_NOALLOC_SCRATCH_BYTES (4u << 20)

static __device__ __align__(256) unsigned char qb_noalloc_scratch[QB_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_addr[kMaxDevices] = {};

// device address of the scratch array on the current device (looked up once per device)
unsigned char *scratch_address() {
	int dev = 0;
	QB_CUDA(cudaGetDevice(&dev));
	if (dev < 0 || dev >= kMaxDevices) QB_FAIL("qb_integral_i3_noalloc: device ordinal out of range");
	std::lock_guard<std::mutex> lk(g_mu);
	if (g_addr[dev] == nullptr) {
		void *p = nullptr;
		const cudaError_t e = cudaGetSymbolAddress(&p, qb_noalloc_scratch);
		if (e != cudaSuccess || p == nullptr)
			QB_FAIL(std::string("qb_integral_i3_noalloc: cudaGetSymbolAddress of the static scratch failed: ") + cudaGetErrorString(e));
		g_addr[dev] = p;
	}
	return static_cast<unsigned char *>(g_addr[dev]);
}

// out = s^2 Extract(IFFT2(sum_k X[k])) over the rank-0 partials of the 2-CTA I3 kernel
template <int P>
__global__ void __launch_bounds__(qb::Geo<P>::NT) k_noalloc_finish(const double2 *__restrict__ X, int nparts, long stride, double scale,
                                                                   double2 *__restrict__ out) {
	using G = qb::Geo<P>;
	constexpr int N = G::N;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	double2 *S = reinterpret_cast<double2 *>(smem_raw), *tw = S + G::GRID;
	qb::init_twiddles<P>(tw);
	for (int i = threadIdx.x; i < P * P; i += G::NT) {
		double2 s = X[i];
		for (int k = 1; k < nparts; k++) s = qb::cadd(s, X[k * stride + i]);
		S[(i / P) * G::LDP + (i % P)] = s;
	}
	__syncthreads();
	qb::fft2_smem<P, +1>(S, tw);
	for (int q = threadIdx.x; q < N * N; q += G::NT) {
		const double2 v = S[G::pad(q / N) * G::LDP + G::pad(q % N)];
		out[q] = make_double2(scale * v.x, scale * v.y);
	}
}

template <int P>
void run(const qb::DevI3 &t, const double2 *f, const double2 *g, const double2 *h, double2 *out, cudaStream_t s) {
	using G = qb::Geo<P>;
	constexpr long NN = (long)G::N * G::N, PP = (long)P * P;
	// scratch layout: sources [h, f, g] (N x N each), g^ (P x P), partials [chunk][2][P x P]
	const size_t fixed = sizeof(double2) * (3 * NN + PP);
	const size_t per_chunk = sizeof(double2) * 2 * PP;
	if (fixed + per_chunk > QB_NOALLOC_SCRATCH_BYTES) QB_FAIL("qb_integral_i3_noalloc: grid too large for the static scratch");
	const int fit = (int)((QB_NOALLOC_SCRATCH_BYTES - fixed) / per_chunk);
	int sms = 0, dev = 0;
	QB_CUDA(cudaGetDevice(&dev));
	QB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
	const int nchunk = std::max(1, std::min(std::min(t.nterms, std::max(1, sms / 2)), fit));

	unsigned char *base = scratch_address();
	double2 *src = reinterpret_cast<double2 *>(base);
	double2 *ghat = src + 3 * NN;
	double2 *parts = ghat + PP;
	QB_CUDA(cudaMemcpyAsync(src, h, sizeof(double2) * NN, cudaMemcpyDeviceToDevice, s));
	QB_CUDA(cudaMemcpyAsync(src + NN, f, sizeof(double2) * NN, cudaMemcpyDeviceToDevice, s));
	QB_CUDA(cudaMemcpyAsync(src + 2 * NN, g, sizeof(double2) * NN, cudaMemcpyDeviceToDevice, s));

	const size_t sm1 = sizeof(double2) * (G::GRID + P), sm2 = sizeof(double2) * (2 * G::GRID + P);
	QB_CUDA(cudaFuncSetAttribute(qb::k_pad_fft<P, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1));
	qb::k_pad_fft<P, double2><<<1, G::NT, sm1, s>>>(src + 2 * NN, ghat);
	QB_CUDA(cudaGetLastError());

	qb::I3Params p{};
	p.nchunk = nchunk; p.nterms = t.nterms;
	p.src = src; p.src_cell = 0; p.src_comp[0] = 0; p.src_comp[1] = 1;
	p.Ghat = ghat; p.g_cell = 0;
	p.ncombo[0] = 1; p.ca[0][0] = 1; p.cgi[0][0] = 0; p.ccoef[0][0] = 1.0;
	p.ncombo[1] = 0;
	p.psi1 = t.psi1.as<double2>(); p.psi2T = t.psi2T.as<double>();
	p.psi2_idx = t.idx.as<int>(); p.psi2_scale = t.scale.as<double>();
	p.out = parts;
	auto kern = qb::k_i3<P, 2, double2>;
	QB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3((unsigned)(nchunk * 2));
	cfg.blockDim = dim3(G::NT);
	cfg.dynamicSmemBytes = sm2;
	cfg.stream = s;
	cudaLaunchAttribute attr;
	attr.id = cudaLaunchAttributeClusterDimension;
	attr.val.clusterDim.x = 2; attr.val.clusterDim.y = 1; attr.val.clusterDim.z = 1;
	cfg.attrs = &attr;
	cfg.numAttrs = 1;
	QB_CUDA(cudaLaunchKernelEx(&cfg, kern, p));

	QB_CUDA(cudaFuncSetAttribute(k_noalloc_finish<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1));
	const double s2 = 1.0 / (double)PP;
	k_noalloc_finish<P><<<1, G::NT, sm1, s>>>(parts, nchunk, 2 * PP, s2 * s2, out);
	QB_CUDA(cudaGetLastError());
}

}  // namespace

extern "C" int qb_integral_i3_noalloc(const qb_quad *q, const void *f, const void *g, const void *h, void *out, void *stream) {
	try {
		if (q == nullptr || q->q == nullptr) QB_FAIL("qb_integral_i3_noalloc: null quadrature handle");
		if (f == nullptr || g == nullptr || h == nullptr || out == nullptr) QB_FAIL("qb_integral_i3_noalloc: null grid pointer");
		const qb::DevI3 &t = q->q->i3;
		const cudaStream_t s = (cudaStream_t)stream;
		const double2 *F = (const double2 *)f, *G = (const double2 *)g, *H = (const double2 *)h;
		switch (q->q->N) {
		case 8: run<16>(t, F, G, H, (double2 *)out, s); break;
		case 16: run<32>(t, F, G, H, (double2 *)out, s); break;
		case 32: run<64>(t, F, G, H, (double2 *)out, s); break;
		default: QB_FAIL("qb_integral_i3_noalloc: grid size N=" + std::to_string(q->q->N) + " exceeds the supported maximum (32)");
		}
		return 0;
	} catch (const std::exception &) {
		return -1;
	}
}
