// qb_engine.cu — launch wrappers and step orchestration of the GPU engine.
#include "qb_engine.h"
#include "qb_kernels.cuh"
#include "qb_split128.cuh"
#include "qb_full128.cuh"
#include "qb_transport.cuh"

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace qb {

// ---------------------------------------------------------------------------
// errors
static std::mutex g_err_mu;
static std::string g_last_error;

void fail(const char *file, int line, const std::string &msg) {
	std::string m = std::string("qbgpu: ") + msg + " (" + file + ":" + std::to_string(line) + ")";
	{
		std::lock_guard<std::mutex> lk(g_err_mu);
		g_last_error = m;
	}
	const char *e = getenv("QB_ABORT_ON_ERROR");
	if (e == nullptr || strcmp(e, "0") != 0) {
		fprintf(stderr, "%s\n", m.c_str());
		abort();
	}
	throw std::runtime_error(m);
}

std::string last_error() {
	std::lock_guard<std::mutex> lk(g_err_mu);
	return g_last_error;
}

bool supported_n(int N) { return N == 8 || N == 16 || N == 32 || N == 64 || anyn_supported(N); }

// ---------------------------------------------------------------------------
// launch accounting
namespace {
struct ProfRec { std::string name; cudaEvent_t e0, e1; };
std::mutex g_prof_mu;
std::vector<ProfRec> g_prof;
std::atomic<bool> g_prof_on{false};
std::atomic<long> g_launches{0};
}  // namespace

void prof_enable(bool on) { g_prof_on = on; }
bool prof_enabled() { return g_prof_on.load(); }
long launch_count() { return g_launches.load(); }
void add_launches(long n) { g_launches += n; }

void prof_reset() {
	std::lock_guard<std::mutex> lk(g_prof_mu);
	for (auto &r : g_prof) { cudaEventDestroy(r.e0); cudaEventDestroy(r.e1); }
	g_prof.clear();
}

void prof_read(const char *prefix, double *ms, long *launches) {
	std::lock_guard<std::mutex> lk(g_prof_mu);
	double t = 0;
	long n = 0;
	const size_t lp = strlen(prefix);
	for (auto &r : g_prof) {
		if (r.name.compare(0, lp, prefix) != 0) continue;
		QB_CUDA(cudaEventSynchronize(r.e1));
		float e = 0;
		QB_CUDA(cudaEventElapsedTime(&e, r.e0, r.e1));
		t += e;
		n++;
	}
	*ms = t;
	*launches = n;
}

ProfScope::ProfScope(const char *n, cudaStream_t st) : name(n), s(st) {
	g_launches++;
	cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
	if (g_prof_on && cudaStreamIsCapturing(s, &cap) == cudaSuccess && cap == cudaStreamCaptureStatusNone) {
		QB_CUDA(cudaEventCreate(&e0));
		QB_CUDA(cudaEventCreate(&e1));
		QB_CUDA(cudaEventRecord(e0, s));
	}
}

ProfScope::~ProfScope() {
	if (e0 != nullptr) {
		cudaEventRecord(e1, s);
		std::lock_guard<std::mutex> lk(g_prof_mu);
		g_prof.push_back({ name, e0, e1 });
	}
}

// ---------------------------------------------------------------------------
// buffers
namespace {
std::atomic<unsigned long long> g_buffer_generation{0};
}

unsigned long long buffer_generation() { return g_buffer_generation.load(std::memory_order_acquire); }

void DevBuf::ensure(size_t n) {
	if (n <= bytes && p != nullptr) return;
	release();
	g_buffer_generation.fetch_add(1, std::memory_order_acq_rel);
	QB_CUDA(cudaGetDevice(&device));
	QB_CUDA(cudaMalloc(&p, n));
	bytes = n;
}

void DevBuf::release() {
	if (p != nullptr) {
		g_buffer_generation.fetch_add(1, std::memory_order_acq_rel);
		int cur = -1;
		cudaGetDevice(&cur);
		if (device >= 0 && cur != device) cudaSetDevice(device);
		cudaFree(p);
		if (device >= 0 && cur != device) cudaSetDevice(cur);
	}
	p = nullptr;
	bytes = 0;
}

Workspace::Workspace(int n) : N(n) {
	if (!supported_n(N)) QB_FAIL("grid size N=" + std::to_string(N) + " has no compiled kernels");
	QB_CUDA(cudaGetDevice(&device));
	QB_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
	i3stats.ensure(2 * sizeof(unsigned long long));
	QB_CUDA(cudaMemset(i3stats.p, 0, 2 * sizeof(unsigned long long)));
	kerr.ensure(sizeof(int));
	QB_CUDA(cudaMemset(kerr.p, 0, sizeof(int)));
	if (anyn_supported(N)) anyn_build_twiddles(*this);
}

Workspace::~Workspace() {
	for (auto &g : graphs)
		if (g.exec) cudaGraphExecDestroy(g.exec);
	if (ev_in) cudaEventDestroy(ev_in);
	if (ev_out) cudaEventDestroy(ev_out);
	if (ev_t) cudaEventDestroy(ev_t);
	if (ev_i) cudaEventDestroy(ev_i);
	if (stream) cudaStreamDestroy(stream);
}

// ---------------------------------------------------------------------------
// launch helpers (templated on the padded size P)
namespace {

// Kernel attributes (dynamic shared-memory limits) and occupancy results are
// per CUDA device.  These two wrappers keep one value per device, selected by
// the device current at each access, so that a process driving several GPUs
// sets every attribute on each of them.  Racing first calls from several host
// threads at worst repeat an idempotent attribute call or occupancy query.
constexpr int kMaxDevices = 64;
inline int cur_dev() {
	int d = 0;
	cudaGetDevice(&d);
	return d & (kMaxDevices - 1);
}
struct DeviceFlag {
	std::atomic<unsigned long long> bits{0};
	explicit operator bool() const { return (bits.load(std::memory_order_acquire) >> cur_dev()) & 1ull; }
	bool operator!() const { return !static_cast<bool>(*this); }
	DeviceFlag &operator=(bool v) {
		const unsigned long long b = 1ull << cur_dev();
		if (v) bits.fetch_or(b, std::memory_order_acq_rel);
		else bits.fetch_and(~b, std::memory_order_acq_rel);
		return *this;
	}
};
struct DeviceInt {
	std::atomic<int> v[kMaxDevices];
	explicit DeviceInt(int init) { for (auto &x : v) x.store(init); }
	operator int() const { return v[cur_dev()].load(std::memory_order_acquire); }
	DeviceInt &operator=(int x) { v[cur_dev()].store(x, std::memory_order_release); return *this; }
};

int num_sms() {
	static DeviceInt sms{0};
	if (sms == 0) {
		int dev = 0, n = 0;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
		sms = n > 0 ? n : 148;
	}
	return sms;
}

// before the first launch of any tensor-memory kernel on a device (defined below)
void check_tmem_coresidency();
}  // namespace
// I3 sums of the FP32 form at N = 16 as DFT-GEMMs on the tensor cores (qb_dftmma.cu)
void launch_i3_mma32(const I3ParamsT<float2> &p, long ncl, int *err, cudaStream_t s);
namespace {

template <class K> void set_smem(K kernel, size_t bytes) {
	QB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

template <int P, class C = double2> constexpr size_t smem_grids(int ngrids) { return sizeof(C) * ((size_t)ngrids * Geo<P, C>::GRID + P); }

// active clusters of the I3 kernel (occupancy query, cached per P and C)
template <int P, class C> int active_i3_clusters() {
	static DeviceInt cached{-1};
	if (cached < 0) {
		auto kern = k_i3<P, 4, C>;
		set_smem(kern, smem_grids<P, C>(2));
		cudaLaunchConfig_t cfg = {};
		cfg.gridDim = dim3(4);
		cfg.blockDim = dim3(Geo<P>::NT);
		cfg.dynamicSmemBytes = smem_grids<P, C>(2);
		cudaLaunchAttribute attr;
		attr.id = cudaLaunchAttributeClusterDimension;
		attr.val.clusterDim.x = 4; attr.val.clusterDim.y = 1; attr.val.clusterDim.z = 1;
		cfg.attrs = &attr;
		cfg.numAttrs = 1;
		int n = 0;
		if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess || n <= 0) {
			cudaGetLastError();
			n = std::max(1, num_sms() / 4);
		}
		cached = n;
	}
	return cached;
}

// number of chunks minimising (waves x terms per chunk) + penalty x chunks for
// `units` independent work units that each split their `nterms` terms into
// chunks; `penalty` is the cost of one more partial grid (written by the term
// kernel, read back by the reduction) in units of one term's time
int best_chunks(long units, int nterms, int slots, int max_chunks, double penalty = 0.02) {
	int best = 1;
	double best_cost = 1e300;
	for (int c = 1; c <= std::min(nterms, max_chunks); c++) {
		const long waves = (units * c + slots - 1) / slots;
		const double cost = (double)waves * ((nterms + c - 1) / c) + penalty * c;
		if (cost < best_cost - 1e-9) { best_cost = cost; best = c; }
	}
	return best;
}

template <int P, class C> void launch_pad_fft(int ngrids, const double2 *src, C *out, cudaStream_t s) {
	static DeviceFlag init;
	if (!init) { set_smem(k_pad_fft<P, C>, smem_grids<P, C>(1)); init = true; }
	ProfScope ps("pad_fft", s);
	k_pad_fft<P, C><<<ngrids, Geo<P>::NT, smem_grids<P, C>(1), s>>>(src, out);
	QB_CUDA(cudaGetLastError());
}

template <int P, class C> void launch_i1(const I1ParamsT<C> &p, long nblocks, cudaStream_t s) {
	static DeviceFlag init;
	if (!init) { set_smem(k_i1_terms<P, C>, smem_grids<P, C>(2)); init = true; }
	ProfScope ps("i1_terms", s);
	k_i1_terms<P, C><<<(unsigned)nblocks, Geo<P>::NT, smem_grids<P, C>(2), s>>>(p);
	QB_CUDA(cudaGetLastError());
}

template <int P, class C> void launch_i2(const I2ParamsT<C> &p, long nblocks, cudaStream_t s) {
	static DeviceFlag init;
	if (!init) { set_smem(k_i2_terms<P, C>, smem_grids<P, C>(2)); init = true; }
	ProfScope ps("i2_terms", s);
	k_i2_terms<P, C><<<(unsigned)nblocks, Geo<P>::NT, smem_grids<P, C>(2), s>>>(p);
	QB_CUDA(cudaGetLastError());
}

template <int P, int CS, class C> void launch_i3(const I3ParamsT<C> &p, long nclusters, cudaStream_t s) {
	static DeviceFlag init;
	auto kern = k_i3<P, CS, C>;
	if (!init) { set_smem(kern, smem_grids<P, C>(2)); init = true; }
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3((unsigned)(nclusters * CS));
	cfg.blockDim = dim3(Geo<P>::NT);
	cfg.dynamicSmemBytes = smem_grids<P, C>(2);
	cfg.stream = s;
	cudaLaunchAttribute attr;
	attr.id = cudaLaunchAttributeClusterDimension;
	attr.val.clusterDim.x = CS; attr.val.clusterDim.y = 1; attr.val.clusterDim.z = 1;
	cfg.attrs = &attr;
	cfg.numAttrs = 1;
	ProfScope ps("i3_cluster", s);
	QB_CUDA(cudaLaunchKernelEx(&cfg, kern, p));
}

// I3 kernels of the FP32 form at N = 32 (k_i3p) and N = 64 (k_i3_full128:
// 2-CTA clusters, a whole grid per CTA, all 512 tensor-memory columns per CTA,
// so exactly one CTA per SM, checked).  By default the cells whose Nyquist
// content is at most kRealFormBound take the real forms (k_i3pr,
// k_i3_full128r) and the others the complex kernels.  QB_I3_KERNEL selects one
// kernel for every cell instead (for comparisons): "complex" the complex
// kernels, "pair" the complex k_i3p and the pair-split k_i3_128.
inline const char *i3_kernel_env() {
	static const char *e = getenv("QB_I3_KERNEL");
	return e ? e : "";
}
inline bool use_full128() {
	static const bool on = strcmp(i3_kernel_env(), "pair") != 0;
	return on;
}
inline bool use_real_form() {
	static const bool on = use_full128() && strcmp(i3_kernel_env(), "complex") != 0;
	return on;
}
// The FP64 I3 sums at N = 32 run as one contiguous range of the (cell, term)
// work per resident cluster (QB_I3_RANGES=0: the (cell, chunk) grid instead,
// for comparisons): every cluster has the same number of terms, and a cell's
// partial sums are one per cluster that touches it instead of one per chunk.
inline bool term_ranges_enabled() {
	static const bool on = [] { const char *e = getenv("QB_I3_RANGES"); return e == nullptr || strcmp(e, "0") != 0; }();
	return on;
}
inline TermRanges term_ranges(int slots, int nterms, int ncells) {
	TermRanges g;
	g.nslots = slots;
	g.nterms = nterms;
	g.total = (long)ncells * nterms;
	g.maxc = 1;
	for (int k = 0; k < slots; k++) {
		const long a = g.start(k), b = g.start(k + 1);
		if (b > a) g.maxc = std::max(g.maxc, (int)((b - 1) / nterms - a / nterms + 1));
	}
	return g;
}

// the workspace's chunk multipliers applied to heuristic chunk counts
inline void scale_chunks(const Workspace &ws, const QuadSet &q, Chunks &ch) {
	auto sc = [](int c, float f, int nterms, int cap) {
		const int v = (int)std::lround((double)c * f);
		return std::max(1, std::min(std::min(v, std::max(1, nterms)), cap));
	};
	if (ws.chunk_scale12 != 1.0f) {
		if (q.i1) ch.i1 = sc(ch.i1, ws.chunk_scale12, q.i1->nterms, 64);
		if (q.i2) ch.i2 = sc(ch.i2, ws.chunk_scale12, q.i2->nterms, 64);
	}
	if (ws.chunk_scale3 != 1.0f && q.i3) ch.i3 = sc(ch.i3, ws.chunk_scale3, q.i3->nterms, 256);
}

constexpr double kRealFormBound = 1e-6;
// The real forms pack the combos of an output in pairs.  Both callers of the
// I3 sums (the Cd assembly and the single-integral path) set 4 combos per
// output, so this holds today; it guards the real-form launch against a
// future caller with an odd count, which then takes the complex kernel.
template <class C> bool even_combos(const I3ParamsT<C> &p) {
	for (int r = 0; r < 4; r++)
		if (p.ncombo[r] & 1) return false;
	return true;
}

void launch_nyquist_kind(int N, int ncells, const double2 *W, double bound, int *kind, unsigned long long *stats, cudaStream_t s) {
	ProfScope ps("nyquist_kind", s);
	k_nyquist_kind<<<ncells, kNyqThreads, 0, s>>>(N, W, bound, kind, stats);
	QB_CUDA(cudaGetLastError());
}

// k_i3p (P = 64): 2-CTA clusters, TMEM accumulators.  The allocation of
// I3Tmem<C>::NCOLS columns never waits as long as no more CTAs share an SM
// than its 512 columns hold; the shared-memory (FP64) or register (FP32)
// footprint keeps it at one CTA per SM, checked here before the first launch.
// three grids and the twiddles; in FP32 two more grids receive the partner's P grids
template <class C> size_t i3p_smem() {
	return sizeof(C) * ((size_t)(sizeof(C) == 8 ? 5 : 3) * Geo<64, C>::GRID + 64);
}
// the real form receives the partner's packed P grid in its second grid slot
inline size_t i3pr_smem() { return sizeof(float2) * ((size_t)3 * Geo<64, float2>::GRID + 64); }

template <class C> int active_i3p_clusters() {
	static DeviceInt cached{-1};
	if (cached < 0) {
		check_tmem_coresidency();
		auto kern = k_i3p<64, C>;
		set_smem(kern, i3p_smem<C>());
		int per_sm = 0;
		QB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Geo<64>::NT, i3p_smem<C>()));
		if (per_sm * (int)I3Tmem<C>::ALLOC > 512)
			QB_FAIL("k_i3p: " + std::to_string(per_sm) + " CTAs per SM would oversubscribe tensor memory");
		cudaLaunchConfig_t cfg = {};
		cfg.gridDim = dim3(2);
		cfg.blockDim = dim3(Geo<64>::NT);
		cfg.dynamicSmemBytes = i3p_smem<C>();
		cudaLaunchAttribute attr;
		attr.id = cudaLaunchAttributeClusterDimension;
		attr.val.clusterDim.x = 2; attr.val.clusterDim.y = 1; attr.val.clusterDim.z = 1;
		cfg.attrs = &attr;
		cfg.numAttrs = 1;
		int n = 0;
		if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess || n <= 0) {
			cudaGetLastError();
			n = std::max(1, num_sms() / 2);
		}
		cached = n;
	}
	return cached;
}

template <class C> void launch_i3p(const I3ParamsT<C> &p, long nclusters, const int *kind, cudaStream_t s) {
	active_i3p_clusters<C>();                  // attribute + occupancy check
	auto kern = k_i3p<64, C>;
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3((unsigned)(nclusters * 2));
	cfg.blockDim = dim3(Geo<64>::NT);
	cfg.dynamicSmemBytes = i3p_smem<C>();
	cfg.stream = s;
	cudaLaunchAttribute attr;
	attr.id = cudaLaunchAttributeClusterDimension;
	attr.val.clusterDim.x = 2; attr.val.clusterDim.y = 1; attr.val.clusterDim.z = 1;
	cfg.attrs = &attr;
	cfg.numAttrs = 1;
	ProfScope ps("i3_cluster", s);
	QB_CUDA(cudaLaunchKernelEx(&cfg, kern, p, kind));
}

// the real form at P = 64 (FP32): same shared memory as k_i3p, 128 tensor-memory columns
void launch_i3pr(const I3ParamsT<float2> &p, long nclusters, const int *kind, cudaStream_t s) {
	static DeviceFlag init;
	auto kern = k_i3pr<64>;
	if (!init) {
		check_tmem_coresidency();
		set_smem(kern, i3pr_smem());
		int per_sm = 0;
		QB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Geo<64>::NT, i3pr_smem()));
		if (per_sm * (int)I3TmemR::ALLOC > 512)
			QB_FAIL("k_i3pr: " + std::to_string(per_sm) + " CTAs per SM would oversubscribe tensor memory");
		init = true;
	}
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3((unsigned)(nclusters * 2));
	cfg.blockDim = dim3(Geo<64>::NT);
	cfg.dynamicSmemBytes = i3pr_smem();
	cfg.stream = s;
	cudaLaunchAttribute attr;
	attr.id = cudaLaunchAttributeClusterDimension;
	attr.val.clusterDim.x = 2; attr.val.clusterDim.y = 1; attr.val.clusterDim.z = 1;
	cfg.attrs = &attr;
	cfg.numAttrs = 1;
	ProfScope ps("i3_cluster", s);
	QB_CUDA(cudaLaunchKernelEx(&cfg, kern, p, kind));
}

template <int P, class C> void launch_fft_full(const FullParamsT<C> &p, long ngrids, cudaStream_t s) {
	static DeviceFlag init;
	if (!init) { set_smem(k_fft_full<P, C>, smem_grids<P, C>(1)); init = true; }
	ProfScope ps("fft_full", s);
	k_fft_full<P, C><<<(unsigned)ngrids, Geo<P>::NT, smem_grids<P, C>(1), s>>>(p);
	QB_CUDA(cudaGetLastError());
}

template <int P, class C> void launch_assemble(const AsmParamsT<C> &p, long ncells, cudaStream_t s) {
	static DeviceFlag init;
	if (!init) { set_smem(k_assemble<P, C>, smem_grids<P, C>(1)); init = true; }
	ProfScope ps("assemble", s);
	k_assemble<P, C><<<(unsigned)(ncells * 4), Geo<P>::NT, smem_grids<P, C>(1), s>>>(p);
	QB_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// quadrature tables in the working precision: FP64 tables as built, FP32
// copies made once, on first use, by rounding the FP64 tables
__global__ void k_round_f32(long n, const double *__restrict__ in, float *__restrict__ out) {
	const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] = (float)in[i];
}

std::mutex g_f32_mu;

void round_table(const DevBuf &d, DevBuf &f, cudaStream_t s) {
	const long n = (long)(d.bytes / sizeof(double));
	if (n == 0 || f.p != nullptr) return;
	f.ensure(sizeof(float) * n);
	k_round_f32<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, d.as<double>(), f.as<float>());
	QB_CUDA(cudaGetLastError());
}

template <class C> struct Tab;
template <> struct Tab<double2> {
	static void prepare(const QuadSet &, cudaStream_t) {}
	static const double *i1_psi2(const DevI1 &t) { return t.psi2.as<double>(); }
	static const double *i1_phi(const DevI1 &t) { return t.phi.as<double>(); }
	static const double *i2_psi1(const DevI2 &t) { return t.psi1.as<double>(); }
	static const double *i2_psi2(const DevI2 &t) { return t.psi2.as<double>(); }
	static const double2 *i3_psi1(const DevI3 &t) { return t.psi1.as<double2>(); }
	static const double *i3_psi2T(const DevI3 &t) { return t.psi2T.as<double>(); }
};
template <> struct Tab<float2> {
	// the copies are made on the caller's stream, which is then synchronised
	// so that any stream may read them afterwards; this needs a stream that is
	// not being captured, i.e. a first FP32 evaluation outside graph capture
	static void prepare(const QuadSet &q, cudaStream_t s) {
		std::lock_guard<std::mutex> lk(g_f32_mu);
		const DevI1 *i1s[2] = { q.i1, q.i4 };
		bool fresh = false;
		for (const DevI1 *t : i1s)
			if (t && t->psi2f.p == nullptr) { round_table(t->psi2, t->psi2f, s); round_table(t->phi, t->phif, s); fresh = true; }
		if (q.i2 && q.i2->psi1f.p == nullptr) { round_table(q.i2->psi1, q.i2->psi1f, s); round_table(q.i2->psi2, q.i2->psi2f, s); fresh = true; }
		if (q.i3 && q.i3->psi1f.p == nullptr) { round_table(q.i3->psi1, q.i3->psi1f, s); round_table(q.i3->psi2T, q.i3->psi2Tf, s); fresh = true; }
		if (fresh) {
			cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
			QB_CUDA(cudaStreamIsCapturing(s, &cap));
			if (cap != cudaStreamCaptureStatusNone) QB_FAIL("the first FP32 evaluation with a table set must not be captured");
			QB_CUDA(cudaStreamSynchronize(s));
		}
	}
	static const float *i1_psi2(const DevI1 &t) { return t.psi2f.as<float>(); }
	static const float *i1_phi(const DevI1 &t) { return t.phif.as<float>(); }
	static const float *i2_psi1(const DevI2 &t) { return t.psi1f.as<float>(); }
	static const float *i2_psi2(const DevI2 &t) { return t.psi2f.as<float>(); }
	static const float2 *i3_psi1(const DevI3 &t) { return t.psi1f.as<float2>(); }
	static const float *i3_psi2T(const DevI3 &t) { return t.psi2Tf.as<float>(); }
};

// ---------------------------------------------------------------------------
// the factored right-hand side for one padded size P and working complex type C
template <int P, class C> struct Rhs {
	static constexpr int N = P / 2;
	static constexpr long NN = (long)N * N, PP = (long)P * P;
	using T = Tab<C>;

	// spectra of the four components
	static void spectra(Workspace &ws, int ncells, const double2 *W, cudaStream_t s) {
		ws.What.ensure(sizeof(C) * 4 * ncells * PP);
		launch_pad_fft<P>(4 * ncells, W, ws.What.as<C>(), s);
	}

	// S sums for Cc (tasks g = W_1..W_3, F = -4 W^_0 + 2) or I4 (g = W_0..W_3, F = 2 W^_0 - 1)
	static void i1_sums(Workspace &ws, const DevI1 &t, int ncells, const double2 *W, bool cc, DevBuf &part, DevBuf &fs, int nchunk, cudaStream_t s) {
		const int ntask = cc ? 3 : 4;
		part.ensure(sizeof(C) * ncells * ntask * nchunk * PP);
		I1ParamsT<C> p{};
		p.ntask = ntask; p.nchunk = nchunk; p.nterms = t.nterms;
		p.g = W; p.g_cell = 4 * NN;
		for (int k = 0; k < 4; k++) p.g_comp[k] = cc ? std::min(k + 1, 3) : k;
		p.What = ws.What.as<C>(); p.w_cell = 4 * PP; p.f_comp = 0;
		p.fa = cc ? -4.0 : 2.0; p.fb = cc ? 2.0 : -1.0;
		p.psi2 = T::i1_psi2(t); p.phi = T::i1_phi(t);
		p.out = part.as<C>();
		launch_i1<P>(p, (long)ncells * ntask * nchunk, s);
		fs.ensure(sizeof(C) * ncells * ntask * PP);
		FullParamsT<C> f{};
		f.in = part.as<C>(); f.grid_stride = nchunk * PP; f.part_stride = PP; f.nparts = nchunk;
		f.out = fs.as<C>();
		launch_fft_full<P>(f, (long)ncells * ntask, s);
	}

	static void i2_sums(Workspace &ws, const DevI2 &t, int ncells, const double2 *W, int nchunk, cudaStream_t s) {
		ws.i2p.ensure(sizeof(C) * ncells * 4 * nchunk * PP);
		I2ParamsT<C> p{};
		p.ntask = 4; p.nchunk = nchunk; p.nterms = t.nterms;
		p.src = W; p.cell_stride = 4 * NN;
		for (int k = 0; k < 4; k++) { p.f_comp[k] = k; p.g_comp[k] = k; }
		p.psi1 = T::i2_psi1(t); p.psi2 = T::i2_psi2(t);
		p.out = ws.i2p.as<C>();
		launch_i2<P>(p, (long)ncells * 4 * nchunk, s);
	}

	static void i3_sums(Workspace &ws, const DevI3 &t, int ncells, const double2 *W, const Chunks &ch, cudaStream_t s) {
		const int nchunk = ch.i3;
		I3ParamsT<C> p{};
		p.nchunk = nchunk; p.nterms = t.nterms;
		if (ch.i3_slots > 0) {
			p.rg = term_ranges(ch.i3_slots, t.nterms, ncells);
			ws.i3p.ensure(sizeof(C) * (size_t)p.rg.nslots * p.rg.maxc * 4 * PP);
		} else {
			ws.i3p.ensure(sizeof(C) * ncells * nchunk * 4 * PP);
		}
		p.src = W; p.src_cell = 4 * NN;
		for (int r = 0; r < 4; r++) p.src_comp[r] = r;
		p.Ghat = ws.What.as<C>(); p.g_cell = 4 * PP;
		const double eta[4] = { 1, -1, -1, -1 };
		for (int r = 0; r < 4; r++) {           // CTA j: X_j = sum_i eta_i P_i . FFT2(psi2 . IFFT2(W^_i . P_j))
			p.ncombo[r] = 4;
			for (int i = 0; i < 4; i++) { p.ca[r][i] = i; p.cgi[r][i] = i; p.ccoef[r][i] = eta[i]; }
		}
		p.psi1 = T::i3_psi1(t); p.psi2T = T::i3_psi2T(t);
		p.psi2_idx = t.idx.as<int>(); p.psi2_scale = t.scale.as<double>();
		p.out = ws.i3p.as<C>();
		p.err = ws.kerr.as<int>();
		if constexpr (P == 64) {
			if constexpr (sizeof(C) == 8) {
				if (use_real_form() && even_combos(p)) {
					ws.i3kind.ensure(sizeof(int) * ncells);
					int *kind = ws.i3kind.as<int>();
					launch_nyquist_kind(P / 2, ncells, W, kRealFormBound, kind, ws.i3stats.as<unsigned long long>(), s);
					launch_i3pr(p, (long)ncells * nchunk, kind, s);
					launch_i3p<C>(p, (long)ncells * nchunk, kind, s);       // cells above the bound
					return;
				}
			}
			launch_i3p<C>(p, p.rg.nslots > 0 ? (long)p.rg.nslots : (long)ncells * nchunk, nullptr, s);
		} else {
			if constexpr (P == 32 && sizeof(C) == 8) {
				if (ws.i3_variant == 1) {
					launch_i3_mma32(p, (long)ncells * nchunk, ws.kerr.as<int>(), s);
					return;
				}
			}
			launch_i3<P, 4>(p, (long)ncells * nchunk, s);
		}
	}

	static void prepare(Workspace &ws, const QuadSet &q, int ncells, const double2 *W, int parts, Chunks &ch, cudaStream_t s) {
		T::prepare(q, s);
		ch = pick_chunks(N, ncells, q, (int)(8 * sizeof(typename CT<C>::R)));
		if (P == 32 && sizeof(C) == 8 && ws.i3_variant == 1 && q.i3) {
			check_tmem_coresidency();
			ch.i3 = best_chunks((long)ncells, std::max(1, q.i3->nterms), num_sms(), 256, 0.15);      // one CTA per SM
		}
		scale_chunks(ws, q, ch);
		// FP64 at N = 32: every resident cluster of k_i3p takes one contiguous range
		// of the (cell, term) work, one partial per cell it touches
		const bool ranges = ws.i3_ranges >= 0 ? ws.i3_ranges == 1 : term_ranges_enabled();
		if (P == 64 && sizeof(C) == 16 && q.i3 && q.i3->nterms > 0 && ranges)
			ch.i3_slots = (int)std::min<long>(active_i3p_clusters<C>(), (long)ncells * q.i3->nterms);
		spectra(ws, ncells, W, s);
		if (parts & RHS_CC) i1_sums(ws, *q.i1, ncells, W, true, ws.i1cc, ws.fs, ch.i1, s);
		if (parts & RHS_CD) {
			i1_sums(ws, *q.i4, ncells, W, false, ws.i1i4, ws.fs4, ch.i1, s);
			i2_sums(ws, *q.i2, ncells, W, ch.i2, s);
			i3_sums(ws, *q.i3, ncells, W, ch, s);
		}
	}

	static AsmParamsT<C> asm_params(Workspace &ws, int parts, const Chunks &ch, const QuadSet &q, int ncells) {
		AsmParamsT<C> a{};
		a.What = ws.What.as<C>();
		a.FS = (parts & RHS_CC) ? ws.fs.as<C>() : nullptr;
		a.FS4 = (parts & RHS_CD) ? ws.fs4.as<C>() : nullptr;
		a.Qp = (parts & RHS_CD) ? ws.i2p.as<C>() : nullptr; a.nq = ch.i2;
		a.Xp = (parts & RHS_CD) ? ws.i3p.as<C>() : nullptr; a.nx = ch.i3;
		if (ch.i3_slots > 0 && (parts & RHS_CD)) a.xrg = term_ranges(ch.i3_slots, q.i3->nterms, ncells);
		a.s2 = 1.0 / (double)PP;
		a.s1 = a.s2 * a.s2;
		return a;
	}

	static void operators(Workspace &ws, const QuadSet &q, int ncells, const double2 *W, int parts, double2 *cc, double2 *cd, cudaStream_t s) {
		Chunks ch;
		prepare(ws, q, ncells, W, parts, ch, s);
		AsmParamsT<C> a = asm_params(ws, parts, ch, q, ncells);
		a.mode = 0; a.out_cc = cc; a.out_cd = cd;
		launch_assemble<P>(a, ncells, s);
	}

	static void update(Workspace &ws, const QuadSet &q, int ncells, const double2 *base, const double2 *wcur, const double *B, double dtc, double2 *out, cudaStream_t s) {
		Chunks ch;
		prepare(ws, q, ncells, wcur, RHS_ALL, ch, s);
		AsmParamsT<C> a = asm_params(ws, RHS_ALL, ch, q, ncells);
		a.mode = 1; a.base = base; a.wcur = wcur; a.B = B; a.dtc = dtc; a.out = out;
		launch_assemble<P>(a, ncells, s);
	}
};

// ---------------------------------------------------------------------------
// N = 64: padded grids of 128 x 128 split over CTA pairs (qb_split128.cuh)

// launch with thread-block clusters of `cdim` CTAs (cdim = 1: plain launch)
template <class... KA, class... A>
void launch128(void (*kern)(KA...), const char *name, long nblocks, int cdim, size_t smem, cudaStream_t s, A... args) {
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3((unsigned)nblocks);
	cfg.blockDim = dim3(G128::NT);
	cfg.dynamicSmemBytes = smem;
	cfg.stream = s;
	cudaLaunchAttribute attr;
	attr.id = cudaLaunchAttributeClusterDimension;
	attr.val.clusterDim.x = cdim; attr.val.clusterDim.y = 1; attr.val.clusterDim.z = 1;
	cfg.attrs = &attr;
	cfg.numAttrs = cdim > 1 ? 1 : 0;
	ProfScope ps(name, s);
	QB_CUDA(cudaLaunchKernelEx(&cfg, kern, args...));
}

template <class K> void set_smem_once(K kern, size_t bytes, DeviceFlag &done) {
	if (!done) { set_smem(kern, bytes); done = true; }
}

// I3 kernel of the collision operator at N = 64: 4 components on 2 CTA pairs
constexpr int kI3Pairs128 = 2;
// its dynamic shared memory: FP64 adds the landing buffer of the bulk-copy exchange
template <class C> constexpr size_t smem_i3_128() { return smem128<C>() + (sizeof(C) == 16 ? kLbBytes : 0); }

// active clusters of the 128 I3 kernel (occupancy query, cached per C)
template <class C> int active_i3_clusters128() {
	static DeviceInt cached{-1};
	if (cached < 0) {
		auto kern = k_i3_128<4, kI3Pairs128, C>;
		set_smem(kern, smem_i3_128<C>());
		cudaLaunchConfig_t cfg = {};
		cfg.gridDim = dim3(2 * kI3Pairs128);
		cfg.blockDim = dim3(G128::NT);
		cfg.dynamicSmemBytes = smem_i3_128<C>();
		cudaLaunchAttribute attr;
		attr.id = cudaLaunchAttributeClusterDimension;
		attr.val.clusterDim.x = 2 * kI3Pairs128; attr.val.clusterDim.y = 1; attr.val.clusterDim.z = 1;
		cfg.attrs = &attr;
		cfg.numAttrs = 1;
		int n = 0;
		if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess || n <= 0) {
			cudaGetLastError();
			n = std::max(1, num_sms() / (2 * kI3Pairs128));
		}
		cached = n;
	}
	return cached;
}

template <class C> void launch_pad_fft128(int ngrids, const double2 *src, C *out, cudaStream_t s) {
	static DeviceFlag init;
	set_smem_once(k_pad_fft128<C>, smem128<C>(), init);
	launch128(k_pad_fft128<C>, "pad_fft", 2L * ngrids, 1, smem128<C>(), s, src, out);
}
template <class C> void launch_i1_128(const I1ParamsT<C> &p, long units, cudaStream_t s) {
	static DeviceFlag init;
	set_smem_once(k_i1_terms128<C>, smem128<C>(), init);
	launch128(k_i1_terms128<C>, "i1_terms", 2 * units, 2, smem128<C>(), s, p);
}
template <class C> void launch_fft_full128(const FullParamsT<C> &p, long ngrids, cudaStream_t s) {
	static DeviceFlag init;
	set_smem_once(k_fft_full128<C>, smem128<C>(), init);
	launch128(k_fft_full128<C>, "fft_full", 2 * ngrids, 1, smem128<C>(), s, p);
}
template <class C> void launch_i2_128(const I2ParamsT<C> &p, long units, C *tmp, cudaStream_t s) {
	static DeviceFlag init;
	set_smem_once(k_i2_terms128<C>, smem128<C>(), init);
	launch128(k_i2_terms128<C>, "i2_terms", 2 * units, 1, smem128<C>(), s, p, tmp);
}
// The tensor-memory allocation of k_i3_128 never waits as long as no more
// CTAs share an SM than its 512 columns hold; checked before the first launch.
template <int CS, int NPAIR, class C> void launch_i3_128(const I3ParamsT<C> &p, long nclusters, C *pscr, int *err, cudaStream_t s) {
	static DeviceFlag init;
	if (!init) {
		check_tmem_coresidency();
		set_smem(k_i3_128<CS, NPAIR, C>, smem_i3_128<C>());
		int per_sm = 0;
		QB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_i3_128<CS, NPAIR, C>, G128::NT, smem_i3_128<C>()));
		if (per_sm * (int)I3Tmem128<C, CS / NPAIR>::NCOLS > 512)
			QB_FAIL("k_i3_128: " + std::to_string(per_sm) + " CTAs per SM would oversubscribe tensor memory");
		init = true;
	}
	launch128(k_i3_128<CS, NPAIR, C>, "i3_cluster", nclusters * 2 * NPAIR, 2 * NPAIR, smem_i3_128<C>(), s, p, pscr, err);
}
constexpr size_t kFull128Smem = sizeof(float2) * ((size_t)F128::GRID + 128 + 64);

int active_i3_full128_clusters() {
	static DeviceInt cached{-1};
	if (cached < 0) {
		check_tmem_coresidency();
		auto kern = k_i3_full128<float2>;
		set_smem(kern, kFull128Smem);
		int per_sm = 0;
		QB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, F128::NT, kFull128Smem));
		if (per_sm * (int)F128Tmem::NCOLS > 512)
			QB_FAIL("k_i3_full128: " + std::to_string(per_sm) + " CTAs per SM would oversubscribe tensor memory");
		cudaLaunchConfig_t cfg = {};
		cfg.gridDim = dim3(2);
		cfg.blockDim = dim3(F128::NT);
		cfg.dynamicSmemBytes = kFull128Smem;
		cudaLaunchAttribute attr;
		attr.id = cudaLaunchAttributeClusterDimension;
		attr.val.clusterDim.x = 2; attr.val.clusterDim.y = 1; attr.val.clusterDim.z = 1;
		cfg.attrs = &attr;
		cfg.numAttrs = 1;
		int n = 0;
		if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess || n <= 0) {
			cudaGetLastError();
			n = std::max(1, num_sms() / 2);
		}
		cached = n;
	}
	return cached;
}

void launch_i3_full128(const I3ParamsT<float2> &p, long nclusters, float2 *pscr, const int *kind, cudaStream_t s) {
	active_i3_full128_clusters();              // attribute + occupancy check
	launch128(k_i3_full128<float2>, "i3_cluster", nclusters * 2, 2, kFull128Smem, s, p, pscr, kind);
}

// the real form: same shared memory, 256 tensor-memory columns
void launch_i3_full128r(const I3ParamsT<float2> &p, long nclusters, float *pscr, const int *kind, cudaStream_t s) {
	static DeviceFlag init;
	if (!init) {
		check_tmem_coresidency();
		set_smem(k_i3_full128r, kFull128Smem);
		int per_sm = 0;
		QB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_i3_full128r, F128::NT, kFull128Smem));
		if (per_sm * (int)F128TmemR::NCOLS > 512)
			QB_FAIL("k_i3_full128r: " + std::to_string(per_sm) + " CTAs per SM would oversubscribe tensor memory");
		init = true;
	}
	launch128(k_i3_full128r, "i3_cluster", nclusters * 2, 2, kFull128Smem, s, p, pscr, kind);
}


// ---- tensor memory: why no allocation ever waits -----------------------------
// tcgen05.alloc blocks while the columns it asks for are held by other CTAs
// on its SM.  With clusters that could deadlock: CTA a1 of cluster A holds
// columns on SM 1 that CTA b1 of cluster B waits for, while b2 holds columns
// on SM 2 that a2 waits for, and each cluster's CTAs wait for one another at
// a cluster barrier.  Launches from two workspaces on two streams could set
// that up.  The library excludes the wait itself, by construction: for every
// set of CTAs of its tensor-memory kernels that the SM's shared memory,
// registers, thread slots and block slots allow to be resident at the same
// time, their columns sum to at most the SM's 512.  Then every allocation is
// granted at once, whatever launches run beside it, and each kernel frees its
// columns before it exits.  This function checks that property from the
// compiled resource footprint of every tensor-memory kernel on the current
// device, by enumerating the multisets of co-resident CTAs (shared-memory
// capacity counted at its largest carve-out, which only admits more sets),
// once per device before the first launch of any of them, and fails loudly
// if a set could oversubscribe.
void check_tmem_coresidency() {
	static DeviceFlag done;
	if (done) return;
	std::vector<TmemKernel> ks = {
		{ (const void *)k_i3p<64, double2>, i3p_smem<double2>(), Geo<64>::NT, (int)I3Tmem<double2>::ALLOC, "k_i3p<f64>" },
		{ (const void *)k_i3p<64, float2>, i3p_smem<float2>(), Geo<64>::NT, (int)I3Tmem<float2>::ALLOC, "k_i3p<f32>" },
		{ (const void *)k_i3pr<64>, i3pr_smem(), Geo<64>::NT, (int)I3TmemR::ALLOC, "k_i3pr" },
		{ (const void *)k_i3_128<4, kI3Pairs128, double2>, smem_i3_128<double2>(), G128::NT,
		  (int)I3Tmem128<double2, 4 / kI3Pairs128>::NCOLS, "k_i3_128<f64>" },
		{ (const void *)k_i3_128<4, kI3Pairs128, float2>, smem_i3_128<float2>(), G128::NT,
		  (int)I3Tmem128<float2, 4 / kI3Pairs128>::NCOLS, "k_i3_128<f32>" },
		{ (const void *)k_i3_128<2, 1, double2>, smem_i3_128<double2>(), G128::NT, (int)I3Tmem128<double2, 2>::NCOLS,
		  "k_i3_128<f64, single integral>" },
		{ (const void *)k_i3_full128<float2>, kFull128Smem, F128::NT, (int)F128Tmem::NCOLS, "k_i3_full128" },
		{ (const void *)k_i3_full128r, kFull128Smem, F128::NT, (int)F128TmemR::NCOLS, "k_i3_full128r" },
	};
	for (const TmemKernel &k : dftmma_tmem_kernels()) ks.push_back(k);
	for (const TmemKernel &k : fno_tmem_kernels()) ks.push_back(k);
	const int n = (int)ks.size();
	int dev = 0, sm_smem = 0, sm_regs = 0, sm_threads = 0, sm_blocks = 0, reserved = 0;
	QB_CUDA(cudaGetDevice(&dev));
	QB_CUDA(cudaDeviceGetAttribute(&sm_smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
	QB_CUDA(cudaDeviceGetAttribute(&sm_regs, cudaDevAttrMaxRegistersPerMultiprocessor, dev));
	QB_CUDA(cudaDeviceGetAttribute(&sm_threads, cudaDevAttrMaxThreadsPerMultiProcessor, dev));
	QB_CUDA(cudaDeviceGetAttribute(&sm_blocks, cudaDevAttrMaxBlocksPerMultiprocessor, dev));
	QB_CUDA(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev));
	struct Use { long smem, regs; int threads, cols; };
	std::vector<Use> u(n);
	for (int i = 0; i < n; i++) {
		cudaFuncAttributes a;
		QB_CUDA(cudaFuncGetAttributes(&a, ks[i].fn));
		const long warps = (ks[i].threads + 31) / 32;
		const long regs_warp = (long)((a.numRegs + 7) / 8) * 8 * 32;      // registers are granted per warp, 8 per thread at a time
		u[i] = { (long)a.sharedSizeBytes + (long)ks[i].dyn_smem + reserved, warps * regs_warp, ks[i].threads, ks[i].cols };
	}
	std::vector<int> count(n, 0);
	// depth-first over multisets in non-decreasing kernel order
	struct Dfs {
		const Use *u; const TmemKernel *ks; int *count; int n, sm_smem, sm_regs, sm_threads, sm_blocks;
		void go(int from, long smem, long regs, int thr, int blocks, int cols) {
			for (int i = from; i < n; i++) {
				const long s2 = smem + u[i].smem, r2 = regs + u[i].regs;
				const int t2 = thr + u[i].threads, b2 = blocks + 1, c2 = cols + u[i].cols;
				if (s2 > sm_smem || r2 > sm_regs || t2 > sm_threads || b2 > sm_blocks) continue;
				count[i]++;
				if (c2 > 512) {
					std::string set;
					for (int k = 0; k < n; k++)
						if (count[k]) set += (set.empty() ? "" : " + ") + std::to_string(count[k]) + " x " + ks[k].name;
					QB_FAIL("tensor memory: " + set + " can share an SM and would ask for " + std::to_string(c2) + " of 512 columns");
				}
				go(i, s2, r2, t2, b2, c2);
				count[i]--;
			}
		}
	} dfs{ u.data(), ks.data(), count.data(), n, sm_smem, sm_regs, sm_threads, sm_blocks };
	dfs.go(0, 0, 0, 0, 0, 0);
	done = true;
}

}  // namespace

bool real_form_enabled() { return use_real_form(); }

int *i3_form_kinds(Workspace &ws, int ncells, const double2 *W, cudaStream_t s) {
	ws.i3kind.ensure(sizeof(int) * ncells);
	int *kind = ws.i3kind.as<int>();
	launch_nyquist_kind(ws.N, ncells, W, kRealFormBound, kind, ws.i3stats.as<unsigned long long>(), s);
	return kind;
}

void ensure_tmem_coresidency() { check_tmem_coresidency(); }
namespace {

template <class C> void launch_assemble128(const AsmParamsT<C> &p, long ncells, cudaStream_t s) {
	static DeviceFlag init;
	set_smem_once(k_assemble128<C>, smem128<C>(), init);
	launch128(k_assemble128<C>, "assemble", 2 * 4 * ncells, 2, smem128<C>(), s, p);
}

template <class C> struct Rhs<128, C> {
	static constexpr int P = 128, N = 64;
	static constexpr long NN = (long)N * N, PP = (long)P * P;
	using T = Tab<C>;

	static void spectra(Workspace &ws, int ncells, const double2 *W, cudaStream_t s) {
		ws.What.ensure(sizeof(C) * 4 * ncells * PP);
		launch_pad_fft128(4 * ncells, W, ws.What.as<C>(), s);
	}

	static void i1_sums(Workspace &ws, const DevI1 &t, int ncells, const double2 *W, bool cc, DevBuf &part, DevBuf &fs, int nchunk, cudaStream_t s) {
		const int ntask = cc ? 3 : 4;
		part.ensure(sizeof(C) * ncells * ntask * nchunk * PP);
		I1ParamsT<C> p{};
		p.ntask = ntask; p.nchunk = nchunk; p.nterms = t.nterms;
		p.g = W; p.g_cell = 4 * NN;
		for (int k = 0; k < 4; k++) p.g_comp[k] = cc ? std::min(k + 1, 3) : k;
		p.What = ws.What.as<C>(); p.w_cell = 4 * PP; p.f_comp = 0;
		p.fa = cc ? -4.0 : 2.0; p.fb = cc ? 2.0 : -1.0;
		p.psi2 = T::i1_psi2(t); p.phi = T::i1_phi(t);
		p.out = part.as<C>();
		launch_i1_128(p, (long)ncells * ntask * nchunk, s);
		fs.ensure(sizeof(C) * ncells * ntask * PP);
		FullParamsT<C> f{};
		f.in = part.as<C>(); f.grid_stride = nchunk * PP; f.part_stride = PP; f.nparts = nchunk;
		f.out = fs.as<C>();
		launch_fft_full128(f, (long)ncells * ntask, s);
	}

	static void i2_sums(Workspace &ws, const DevI2 &t, int ncells, const double2 *W, int nchunk, cudaStream_t s) {
		const long units = (long)ncells * 4 * nchunk;
		ws.i2p.ensure(sizeof(C) * units * PP);
		ws.scr128b.ensure(sizeof(C) * units * PP);
		I2ParamsT<C> p{};
		p.ntask = 4; p.nchunk = nchunk; p.nterms = t.nterms;
		p.src = W; p.cell_stride = 4 * NN;
		for (int k = 0; k < 4; k++) { p.f_comp[k] = k; p.g_comp[k] = k; }
		p.psi1 = T::i2_psi1(t); p.psi2 = T::i2_psi2(t);
		p.out = ws.i2p.as<C>();
		launch_i2_128(p, units, ws.scr128b.as<C>(), s);
	}

	static void i3_sums(Workspace &ws, const DevI3 &t, int ncells, const double2 *W, int nchunk, cudaStream_t s) {
		const long ncl = (long)ncells * nchunk;
		ws.i3p.ensure(sizeof(C) * ncl * 4 * PP);
		ws.scr128a.ensure(sizeof(C) * ncl * 4 * PP);
		I3ParamsT<C> p{};
		p.nchunk = nchunk; p.nterms = t.nterms;
		p.src = W; p.src_cell = 4 * NN;
		for (int r = 0; r < 4; r++) p.src_comp[r] = r;
		p.Ghat = ws.What.as<C>(); p.g_cell = 4 * PP;
		const double eta[4] = { 1, -1, -1, -1 };
		for (int r = 0; r < 4; r++) {
			p.ncombo[r] = 4;
			for (int i = 0; i < 4; i++) { p.ca[r][i] = i; p.cgi[r][i] = i; p.ccoef[r][i] = eta[i]; }
		}
		p.psi1 = T::i3_psi1(t); p.psi2T = T::i3_psi2T(t);
		p.psi2_idx = t.idx.as<int>(); p.psi2_scale = t.scale.as<double>();
		p.out = ws.i3p.as<C>();
		p.err = ws.kerr.as<int>();
		if constexpr (sizeof(C) == 8) {
			if (use_full128()) {
				if (use_real_form() && even_combos(p)) {
					ws.i3kind.ensure(sizeof(int) * ncells);
					int *kind = ws.i3kind.as<int>();
					launch_nyquist_kind(N, ncells, W, kRealFormBound, kind, ws.i3stats.as<unsigned long long>(), s);
					launch_i3_full128r(p, ncl, reinterpret_cast<float *>(ws.scr128a.as<C>()), kind, s);
					launch_i3_full128(p, ncl, ws.scr128a.as<C>(), kind, s);     // cells above the bound
				} else {
					launch_i3_full128(p, ncl, ws.scr128a.as<C>(), nullptr, s);
				}
				return;
			}
		}
		launch_i3_128<4, kI3Pairs128>(p, ncl, ws.scr128a.as<C>(), ws.kerr.as<int>(), s);
	}

	static void prepare(Workspace &ws, const QuadSet &q, int ncells, const double2 *W, int parts, Chunks &ch, cudaStream_t s) {
		T::prepare(q, s);
		const int pairs = std::max(1, num_sms() / 2);
		if (q.i1) ch.i1 = best_chunks((long)ncells * 7, std::max(1, q.i1->nterms), pairs, 64, 0.15);
		if (q.i2) ch.i2 = best_chunks((long)ncells * 4, std::max(1, q.i2->nterms), pairs, 64, 0.15);
		if (q.i3) {
			const int act = (sizeof(C) == 8 && use_full128()) ? active_i3_full128_clusters() : active_i3_clusters128<C>();
			ch.i3 = best_chunks((long)ncells, std::max(1, q.i3->nterms), act, 256, 0.15);
		}
		scale_chunks(ws, q, ch);
		spectra(ws, ncells, W, s);
		if (parts & RHS_CC) i1_sums(ws, *q.i1, ncells, W, true, ws.i1cc, ws.fs, ch.i1, s);
		if (parts & RHS_CD) {
			i1_sums(ws, *q.i4, ncells, W, false, ws.i1i4, ws.fs4, ch.i1, s);
			i2_sums(ws, *q.i2, ncells, W, ch.i2, s);
			i3_sums(ws, *q.i3, ncells, W, ch.i3, s);
		}
	}

	static AsmParamsT<C> asm_params(Workspace &ws, int parts, const Chunks &ch, const QuadSet &q, int ncells) {
		AsmParamsT<C> a{};
		a.What = ws.What.as<C>();
		a.FS = (parts & RHS_CC) ? ws.fs.as<C>() : nullptr;
		a.FS4 = (parts & RHS_CD) ? ws.fs4.as<C>() : nullptr;
		a.Qp = (parts & RHS_CD) ? ws.i2p.as<C>() : nullptr; a.nq = ch.i2;
		a.Xp = (parts & RHS_CD) ? ws.i3p.as<C>() : nullptr; a.nx = ch.i3;
		if (ch.i3_slots > 0 && (parts & RHS_CD)) a.xrg = term_ranges(ch.i3_slots, q.i3->nterms, ncells);
		a.s2 = 1.0 / (double)PP;
		a.s1 = a.s2 * a.s2;
		return a;
	}

	static void operators(Workspace &ws, const QuadSet &q, int ncells, const double2 *W, int parts, double2 *cc, double2 *cd, cudaStream_t s) {
		Chunks ch;
		prepare(ws, q, ncells, W, parts, ch, s);
		AsmParamsT<C> a = asm_params(ws, parts, ch, q, ncells);
		a.mode = 0; a.out_cc = cc; a.out_cd = cd;
		launch_assemble128(a, ncells, s);
	}

	static void update(Workspace &ws, const QuadSet &q, int ncells, const double2 *base, const double2 *wcur, const double *B, double dtc, double2 *out, cudaStream_t s) {
		Chunks ch;
		prepare(ws, q, ncells, wcur, RHS_ALL, ch, s);
		AsmParamsT<C> a = asm_params(ws, RHS_ALL, ch, q, ncells);
		a.mode = 1; a.base = base; a.wcur = wcur; a.B = B; a.dtc = dtc; a.out = out;
		launch_assemble128(a, ncells, s);
	}
};

template <template <int> class F, class... A> void by_n(int N, A &&...args) {
	switch (N) {
	case 8: F<16>::run(args...); break;
	case 16: F<32>::run(args...); break;
	case 32: F<64>::run(args...); break;
	case 64: F<128>::run(args...); break;
	default: QB_FAIL("grid size N=" + std::to_string(N) + " has no compiled kernels");
	}
}

template <class C> struct OpsRun {
	template <int P> struct F {
		static void run(Workspace &ws, const QuadSet &q, int n, const double2 *W, int parts, double2 *cc, double2 *cd, cudaStream_t s) {
			Rhs<P, C>::operators(ws, q, n, W, parts, cc, cd, s);
		}
	};
};
template <class C> struct UpdRun {
	template <int P> struct F {
		static void run(Workspace &ws, const QuadSet &q, int n, const double2 *base, const double2 *wcur, const double *B, double dtc, double2 *out, cudaStream_t s) {
			Rhs<P, C>::update(ws, q, n, base, wcur, B, dtc, out, s);
		}
	};
};

__global__ void k_axpy(long n, const double2 *__restrict__ base, double a, const double2 *__restrict__ k, double2 *__restrict__ out) {
	const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] = make_double2(base[i].x + a * k[i].x, base[i].y + a * k[i].y);
}

__global__ void k_rk4(long n, const double2 *__restrict__ W, double c, const double2 *k1, const double2 *k2, const double2 *k3, const double2 *k4, double2 *out) {
	const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) {
		out[i].x = W[i].x + c * (k1[i].x + 2 * k2[i].x + 2 * k3[i].x + k4[i].x);
		out[i].y = W[i].y + c * (k1[i].y + 2 * k2[i].y + 2 * k3[i].y + k4[i].y);
	}
}

}  // namespace

Chunks pick_chunks(int N, int ncells, const QuadSet &q, int prec) {
	Chunks c;
	const int sms = num_sms();
	if (q.i1) c.i1 = best_chunks((long)ncells * 7, std::max(1, q.i1->nterms), sms, 64);
	if (q.i2) c.i2 = best_chunks((long)ncells * 4, std::max(1, q.i2->nterms), sms, 64);
	if (q.i3) {
		int act = 0;
		const bool f32 = prec == 32;
		switch (N) {
		case 8: act = f32 ? active_i3_clusters<16, float2>() : active_i3_clusters<16, double2>(); break;
		case 16: act = f32 ? active_i3_clusters<32, float2>() : active_i3_clusters<32, double2>(); break;
		default: act = f32 ? active_i3p_clusters<float2>() : active_i3p_clusters<double2>(); break;
		}
		// an I3 partial is 4 padded grids per cluster (256 KB at N = 32) written
		// and read back at HBM speed; one term takes a cluster ~36 us there: 0.15
		c.i3 = best_chunks((long)ncells, std::max(1, q.i3->nterms), act, 256, 0.15);
	}
	return c;
}

void prepare_f32_tables(const QuadSet &q, cudaStream_t s) { Tab<float2>::prepare(q, s); }

void collision_operators(Workspace &ws, const QuadSet &q, int ncells, const double2 *W, int parts, double2 *out_cc, double2 *out_cd, cudaStream_t s) {
	if (anyn_route(ws.N)) { anyn_operators(ws, q, ncells, W, parts, out_cc, out_cd, s); return; }
	if (ws.prec == 32) by_n<OpsRun<float2>::F>(ws.N, ws, q, ncells, W, parts, out_cc, out_cd, s);
	else by_n<OpsRun<double2>::F>(ws.N, ws, q, ncells, W, parts, out_cc, out_cd, s);
}

void collision_update(Workspace &ws, const QuadSet &q, int ncells, const double2 *base, const double2 *wcur, const double *B, double dtc, double2 *out, cudaStream_t s) {
	if (anyn_route(ws.N)) { anyn_update(ws, q, ncells, base, wcur, B, dtc, out, s); return; }
	if (ws.prec == 32) by_n<UpdRun<float2>::F>(ws.N, ws, q, ncells, base, wcur, B, dtc, out, s);
	else by_n<UpdRun<double2>::F>(ws.N, ws, q, ncells, base, wcur, B, dtc, out, s);
}

void collision_step(Workspace &ws, const QuadSet &q, int ncells, const double2 *W, const double *B, double dt, double2 *Wnext, cudaStream_t s) {
	const size_t bytes = sizeof(double2) * 4 * (size_t)ncells * ws.N * ws.N;
	ws.wmid.ensure(bytes);
	collision_update(ws, q, ncells, W, W, B, 0.5 * dt, ws.wmid.as<double2>(), s);
	collision_update(ws, q, ncells, W, ws.wmid.as<double2>(), B, dt, Wnext, s);
}

void collision_step_rk4(Workspace &ws, const QuadSet &q, int ncells, const double2 *W, const double *B, double dt, double2 *Wnext, cudaStream_t s) {
	const long n = 4L * ncells * ws.N * ws.N;
	ws.aux.ensure(sizeof(double2) * 5 * n);
	double2 *k1 = ws.aux.as<double2>(), *k2 = k1 + n, *k3 = k2 + n, *k4 = k3 + n, *Ws = k4 + n;
	const unsigned nb = (unsigned)((n + 255) / 256);
	collision_update(ws, q, ncells, nullptr, W, B, 1.0, k1, s);
	k_axpy<<<nb, 256, 0, s>>>(n, W, 0.5 * dt, k1, Ws);
	collision_update(ws, q, ncells, nullptr, Ws, B, 1.0, k2, s);
	k_axpy<<<nb, 256, 0, s>>>(n, W, 0.5 * dt, k2, Ws);
	collision_update(ws, q, ncells, nullptr, Ws, B, 1.0, k3, s);
	k_axpy<<<nb, 256, 0, s>>>(n, W, dt, k3, Ws);
	collision_update(ws, q, ncells, nullptr, Ws, B, 1.0, k4, s);
	k_rk4<<<nb, 256, 0, s>>>(n, W, dt / 6.0, k1, k2, k3, k4, Wnext);
	QB_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// single-triple integrals (upstream I1integral / I2integral / I3integral)

// out = scale * Extract(IFFT2(Z)) for one padded grid
template <int P>
__global__ void __launch_bounds__(Geo<P>::NT) k_extract_ifft(const double2 *__restrict__ Z, double scale, double2 *__restrict__ out) {
	using G = Geo<P>;
	constexpr int N = G::N;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	double2 *S = reinterpret_cast<double2 *>(smem_raw), *tw = S + G::GRID;
	init_twiddles<P>(tw);
	for (int i = threadIdx.x; i < P * P; i += G::NT) S[(i / P) * G::LDP + (i % P)] = Z[i];
	__syncthreads();
	fft2_smem<P, +1>(S, tw);
	for (int q = threadIdx.x; q < N * N; q += G::NT) {
		const double2 v = S[G::pad(q / N) * G::LDP + G::pad(q % N)];
		out[q] = make_double2(scale * v.x, scale * v.y);
	}
}

// out[i] = a[i] * sum_k b[k*stride + i]   (a may be null: plain sum)
__global__ void k_mul_sum(long n, const double2 *__restrict__ a, const double2 *__restrict__ b, int nparts, long stride, double2 *__restrict__ out) {
	const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	double2 s = b[i];
	for (int k = 1; k < nparts; k++) s = cadd(s, b[k * stride + i]);
	out[i] = a ? cmul(a[i], s) : s;
}

namespace {
void mul_sum(long n, const double2 *a, const double2 *b, int nparts, long stride, double2 *out, cudaStream_t s) {
	k_mul_sum<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, a, b, nparts, stride, out);
	QB_CUDA(cudaGetLastError());
}

template <int P> void extract_ifft(const double2 *Z, double scale, double2 *out, cudaStream_t s) {
	static DeviceFlag init;
	if (!init) { set_smem(k_extract_ifft<P>, smem_grids<P>(1)); init = true; }
	k_extract_ifft<P><<<1, Geo<P>::NT, smem_grids<P>(1), s>>>(Z, scale, out);
	QB_CUDA(cudaGetLastError());
}

// I1 = s^2 Extract(IFFT2(h^ . FFT2(sum_t phi_t . IFFT2(f^ . FFT2(Pad(psi2_t g))))))
template <int P> struct I1S {
	static void run(Workspace &ws, const DevI1 &t, const double2 *f, const double2 *g, const double2 *h, double2 *out, cudaStream_t s) {
		constexpr long NN = (long)(P / 2) * (P / 2), PP = (long)P * P;
		ws.aux.ensure(sizeof(double2) * 2 * NN);
		double2 *fh = ws.aux.as<double2>();
		QB_CUDA(cudaMemcpyAsync(fh, f, sizeof(double2) * NN, cudaMemcpyDeviceToDevice, s));
		QB_CUDA(cudaMemcpyAsync(fh + NN, h, sizeof(double2) * NN, cudaMemcpyDeviceToDevice, s));
		ws.What.ensure(sizeof(double2) * 2 * PP);
		launch_pad_fft<P>(2, fh, ws.What.as<double2>(), s);
		const int nchunk = best_chunks(1, std::max(1, t.nterms), num_sms(), 128);
		ws.i1cc.ensure(sizeof(double2) * nchunk * PP);
		I1Params p{};
		p.ntask = 1; p.nchunk = nchunk; p.nterms = t.nterms;
		p.g = g; p.g_cell = 0; p.g_comp[0] = 0;
		p.What = ws.What.as<double2>(); p.w_cell = 0; p.f_comp = 0; p.fa = 1.0; p.fb = 0.0;
		p.psi2 = t.psi2.as<double>(); p.phi = t.phi.as<double>();
		p.out = ws.i1cc.as<double2>();
		launch_i1<P>(p, nchunk, s);
		ws.fs.ensure(sizeof(double2) * 2 * PP);
		FullParams fp{};
		fp.in = ws.i1cc.as<double2>(); fp.grid_stride = 0; fp.part_stride = PP; fp.nparts = nchunk;
		fp.out = ws.fs.as<double2>();
		launch_fft_full<P>(fp, 1, s);
		mul_sum(PP, ws.What.as<double2>() + PP, ws.fs.as<double2>(), 1, 0, ws.fs.as<double2>() + PP, s);
		const double s2 = 1.0 / (double)PP;
		extract_ifft<P>(ws.fs.as<double2>() + PP, s2 * s2, out, s);
	}
};

// I2 = s Extract(IFFT2(h^ . sum_t FFT2(Pad(psi1_t f)) . FFT2(Pad(psi2_t g))))
template <int P> struct I2S {
	static void run(Workspace &ws, const DevI2 &t, const double2 *f, const double2 *g, const double2 *h, double2 *out, cudaStream_t s) {
		constexpr long NN = (long)(P / 2) * (P / 2), PP = (long)P * P;
		ws.aux.ensure(sizeof(double2) * 3 * NN);
		double2 *fgh = ws.aux.as<double2>();
		QB_CUDA(cudaMemcpyAsync(fgh, f, sizeof(double2) * NN, cudaMemcpyDeviceToDevice, s));
		QB_CUDA(cudaMemcpyAsync(fgh + NN, g, sizeof(double2) * NN, cudaMemcpyDeviceToDevice, s));
		QB_CUDA(cudaMemcpyAsync(fgh + 2 * NN, h, sizeof(double2) * NN, cudaMemcpyDeviceToDevice, s));
		ws.What.ensure(sizeof(double2) * PP);
		launch_pad_fft<P>(1, fgh + 2 * NN, ws.What.as<double2>(), s);
		const int nchunk = best_chunks(1, std::max(1, t.nterms), num_sms(), 128);
		ws.i2p.ensure(sizeof(double2) * nchunk * PP);
		I2Params p{};
		p.ntask = 1; p.nchunk = nchunk; p.nterms = t.nterms;
		p.src = fgh; p.cell_stride = 0; p.f_comp[0] = 0; p.g_comp[0] = 1;
		p.psi1 = t.psi1.as<double>(); p.psi2 = t.psi2.as<double>();
		p.out = ws.i2p.as<double2>();
		launch_i2<P>(p, nchunk, s);
		ws.fs.ensure(sizeof(double2) * PP);
		mul_sum(PP, ws.What.as<double2>(), ws.i2p.as<double2>(), nchunk, PP, ws.fs.as<double2>(), s);
		extract_ifft<P>(ws.fs.as<double2>(), 1.0 / (double)PP, out, s);
	}
};

// I3 = s^2 Extract(IFFT2(sum_t FFT2(Pad(psi1_t f)) . FFT2(psi2_t . IFFT2(g^ . FFT2(Pad(psi1_t h))))))
// on a 2-CTA cluster: rank 0 owns h (convolved with g^), rank 1 owns f.
template <int P> struct I3S {
	static void run(Workspace &ws, const DevI3 &t, const double2 *f, const double2 *g, const double2 *h, double2 *out, cudaStream_t s) {
		constexpr long NN = (long)(P / 2) * (P / 2), PP = (long)P * P;
		ws.aux.ensure(sizeof(double2) * 3 * NN);
		double2 *src = ws.aux.as<double2>();
		QB_CUDA(cudaMemcpyAsync(src, h, sizeof(double2) * NN, cudaMemcpyDeviceToDevice, s));
		QB_CUDA(cudaMemcpyAsync(src + NN, f, sizeof(double2) * NN, cudaMemcpyDeviceToDevice, s));
		QB_CUDA(cudaMemcpyAsync(src + 2 * NN, g, sizeof(double2) * NN, cudaMemcpyDeviceToDevice, s));
		ws.What.ensure(sizeof(double2) * PP);
		launch_pad_fft<P>(1, src + 2 * NN, ws.What.as<double2>(), s);
		const int nchunk = best_chunks(1, std::max(1, t.nterms), std::max(1, num_sms() / 2), 256);
		ws.i3p.ensure(sizeof(double2) * nchunk * 2 * PP);
		I3Params p{};
		p.nchunk = nchunk; p.nterms = t.nterms;
		p.src = src; p.src_cell = 0; p.src_comp[0] = 0; p.src_comp[1] = 1;
		p.Ghat = ws.What.as<double2>(); p.g_cell = 0;
		p.ncombo[0] = 1; p.ca[0][0] = 1; p.cgi[0][0] = 0; p.ccoef[0][0] = 1.0;
		p.ncombo[1] = 0;
		p.psi1 = t.psi1.as<double2>(); p.psi2T = t.psi2T.as<double>();
		p.psi2_idx = t.idx.as<int>(); p.psi2_scale = t.scale.as<double>();
		p.out = ws.i3p.as<double2>();
		launch_i3<P, 2, double2>(p, nchunk, s);
		ws.fs.ensure(sizeof(double2) * PP);
		mul_sum(PP, nullptr, ws.i3p.as<double2>(), nchunk, 2 * PP, ws.fs.as<double2>(), s);   // rank-0 partials
		const double s2 = 1.0 / (double)PP;
		extract_ifft<P>(ws.fs.as<double2>(), s2 * s2, out, s);
	}
};

// N = 64 single integrals on the split kernels (FP64)
void extract_ifft128(const double2 *Z, double scale, double2 *out, cudaStream_t s) {
	static DeviceFlag init;
	set_smem_once(k_extract_ifft128, smem128<double2>(), init);
	launch128(k_extract_ifft128, "assemble", 2, 2, smem128<double2>(), s, Z, scale, out);
}

template <> struct I1S<128> {
	static void run(Workspace &ws, const DevI1 &t, const double2 *f, const double2 *g, const double2 *h, double2 *out, cudaStream_t s) {
		constexpr long NN = 64 * 64, PP = 128 * 128;
		ws.aux.ensure(sizeof(double2) * 2 * NN);
		double2 *fh = ws.aux.as<double2>();
		QB_CUDA(cudaMemcpyAsync(fh, f, sizeof(double2) * NN, cudaMemcpyDeviceToDevice, s));
		QB_CUDA(cudaMemcpyAsync(fh + NN, h, sizeof(double2) * NN, cudaMemcpyDeviceToDevice, s));
		ws.What.ensure(sizeof(double2) * 2 * PP);
		launch_pad_fft128(2, fh, ws.What.as<double2>(), s);
		const int nchunk = best_chunks(1, std::max(1, t.nterms), std::max(1, num_sms() / 2), 128);
		ws.i1cc.ensure(sizeof(double2) * nchunk * PP);
		I1Params p{};
		p.ntask = 1; p.nchunk = nchunk; p.nterms = t.nterms;
		p.g = g; p.g_cell = 0; p.g_comp[0] = 0;
		p.What = ws.What.as<double2>(); p.w_cell = 0; p.f_comp = 0; p.fa = 1.0; p.fb = 0.0;
		p.psi2 = t.psi2.as<double>(); p.phi = t.phi.as<double>();
		p.out = ws.i1cc.as<double2>();
		launch_i1_128(p, nchunk, s);
		ws.fs.ensure(sizeof(double2) * 2 * PP);
		FullParams fp{};
		fp.in = ws.i1cc.as<double2>(); fp.grid_stride = 0; fp.part_stride = PP; fp.nparts = nchunk;
		fp.out = ws.fs.as<double2>();
		launch_fft_full128(fp, 1, s);
		mul_sum(PP, ws.What.as<double2>() + PP, ws.fs.as<double2>(), 1, 0, ws.fs.as<double2>() + PP, s);
		const double s2 = 1.0 / (double)PP;
		extract_ifft128(ws.fs.as<double2>() + PP, s2 * s2, out, s);
	}
};

template <> struct I2S<128> {
	static void run(Workspace &ws, const DevI2 &t, const double2 *f, const double2 *g, const double2 *h, double2 *out, cudaStream_t s) {
		constexpr long NN = 64 * 64, PP = 128 * 128;
		ws.aux.ensure(sizeof(double2) * 3 * NN);
		double2 *fgh = ws.aux.as<double2>();
		QB_CUDA(cudaMemcpyAsync(fgh, f, sizeof(double2) * NN, cudaMemcpyDeviceToDevice, s));
		QB_CUDA(cudaMemcpyAsync(fgh + NN, g, sizeof(double2) * NN, cudaMemcpyDeviceToDevice, s));
		QB_CUDA(cudaMemcpyAsync(fgh + 2 * NN, h, sizeof(double2) * NN, cudaMemcpyDeviceToDevice, s));
		ws.What.ensure(sizeof(double2) * PP);
		launch_pad_fft128(1, fgh + 2 * NN, ws.What.as<double2>(), s);
		const int nchunk = best_chunks(1, std::max(1, t.nterms), std::max(1, num_sms() / 2), 128);
		ws.i2p.ensure(sizeof(double2) * nchunk * PP);
		ws.scr128b.ensure(sizeof(double2) * nchunk * PP);
		I2Params p{};
		p.ntask = 1; p.nchunk = nchunk; p.nterms = t.nterms;
		p.src = fgh; p.cell_stride = 0; p.f_comp[0] = 0; p.g_comp[0] = 1;
		p.psi1 = t.psi1.as<double>(); p.psi2 = t.psi2.as<double>();
		p.out = ws.i2p.as<double2>();
		launch_i2_128(p, nchunk, ws.scr128b.as<double2>(), s);
		ws.fs.ensure(sizeof(double2) * PP);
		mul_sum(PP, ws.What.as<double2>(), ws.i2p.as<double2>(), nchunk, PP, ws.fs.as<double2>(), s);
		extract_ifft128(ws.fs.as<double2>(), 1.0 / (double)PP, out, s);
	}
};

template <> struct I3S<128> {
	static void run(Workspace &ws, const DevI3 &t, const double2 *f, const double2 *g, const double2 *h, double2 *out, cudaStream_t s) {
		constexpr long NN = 64 * 64, PP = 128 * 128;
		ws.aux.ensure(sizeof(double2) * 3 * NN);
		double2 *src = ws.aux.as<double2>();
		QB_CUDA(cudaMemcpyAsync(src, h, sizeof(double2) * NN, cudaMemcpyDeviceToDevice, s));
		QB_CUDA(cudaMemcpyAsync(src + NN, f, sizeof(double2) * NN, cudaMemcpyDeviceToDevice, s));
		QB_CUDA(cudaMemcpyAsync(src + 2 * NN, g, sizeof(double2) * NN, cudaMemcpyDeviceToDevice, s));
		ws.What.ensure(sizeof(double2) * PP);
		launch_pad_fft128(1, src + 2 * NN, ws.What.as<double2>(), s);
		const int nchunk = best_chunks(1, std::max(1, t.nterms), std::max(1, num_sms() / 2), 256);
		ws.i3p.ensure(sizeof(double2) * nchunk * 2 * PP);
		ws.scr128a.ensure(sizeof(double2) * nchunk * 2 * PP);
		I3Params p{};
		p.nchunk = nchunk; p.nterms = t.nterms;
		p.src = src; p.src_cell = 0; p.src_comp[0] = 0; p.src_comp[1] = 1;
		p.Ghat = ws.What.as<double2>(); p.g_cell = 0;
		p.ncombo[0] = 1; p.ca[0][0] = 1; p.cgi[0][0] = 0; p.ccoef[0][0] = 1.0;
		p.ncombo[1] = 0;
		p.psi1 = t.psi1.as<double2>(); p.psi2T = t.psi2T.as<double>();
		p.psi2_idx = t.idx.as<int>(); p.psi2_scale = t.scale.as<double>();
		p.out = ws.i3p.as<double2>();
		launch_i3_128<2, 1>(p, nchunk, ws.scr128a.as<double2>(), ws.kerr.as<int>(), s);
		ws.fs.ensure(sizeof(double2) * PP);
		mul_sum(PP, nullptr, ws.i3p.as<double2>(), nchunk, 2 * PP, ws.fs.as<double2>(), s);
		const double s2 = 1.0 / (double)PP;
		extract_ifft128(ws.fs.as<double2>(), s2 * s2, out, s);
	}
};
}  // namespace

void integral_i1(Workspace &ws, const DevI1 &t, const double2 *f, const double2 *g, const double2 *h, double2 *out, cudaStream_t s) {
	by_n<I1S>(ws.N, ws, t, f, g, h, out, s);
}
void integral_i2(Workspace &ws, const DevI2 &t, const double2 *f, const double2 *g, const double2 *h, double2 *out, cudaStream_t s) {
	by_n<I2S>(ws.N, ws, t, f, g, h, out, s);
}
void integral_i3(Workspace &ws, const DevI3 &t, const double2 *f, const double2 *g, const double2 *h, double2 *out, cudaStream_t s) {
	by_n<I3S>(ws.N, ws, t, f, g, h, out, s);
}

// ---------------------------------------------------------------------------
// Fourier representation, transport, Strang step
namespace {
template <int N> void launch_to_fourier(int ngrids, const double *Wv, double2 *Wf, cudaStream_t s) {
	const size_t sm = sizeof(double2) * (N * (N + 1) + N);
	static DeviceFlag init;
	set_smem_once(k_to_fourier<N>, sm, init);
	ProfScope ps("to_fourier", s);
	k_to_fourier<N><<<ngrids, Len<N>::T * N, sm, s>>>(Wv, Wf);
	QB_CUDA(cudaGetLastError());
}
template <int N> void launch_from_fourier(int ngrids, const double2 *Wf, double *Wv, cudaStream_t s) {
	const size_t sm = sizeof(double2) * (N * (N + 1) + N);
	static DeviceFlag init;
	set_smem_once(k_from_fourier<N>, sm, init);
	ProfScope ps("from_fourier", s);
	k_from_fourier<N><<<ngrids, Len<N>::T * N, sm, s>>>(Wf, Wv);
	QB_CUDA(cudaGetLastError());
}
}  // namespace

void to_fourier(int N, int ngrids, const double *Wv, double2 *Wf, cudaStream_t s) {
	if (ngrids <= 0) return;
	switch (N) {
	case 8: launch_to_fourier<8>(ngrids, Wv, Wf, s); break;
	case 16: launch_to_fourier<16>(ngrids, Wv, Wf, s); break;
	case 32: launch_to_fourier<32>(ngrids, Wv, Wf, s); break;
	case 64: launch_to_fourier<64>(ngrids, Wv, Wf, s); break;
	default:
		if (!anyn_supported(N)) QB_FAIL("to_fourier: unsupported N");
		anyn_to_fourier(N, ngrids, Wv, Wf, s);
	}
}

void from_fourier(int N, int ngrids, const double2 *Wf, double *Wv, cudaStream_t s) {
	if (ngrids <= 0) return;
	switch (N) {
	case 8: launch_from_fourier<8>(ngrids, Wf, Wv, s); break;
	case 16: launch_from_fourier<16>(ngrids, Wf, Wv, s); break;
	case 32: launch_from_fourier<32>(ngrids, Wf, Wv, s); break;
	case 64: launch_from_fourier<64>(ngrids, Wf, Wv, s); break;
	default:
		if (!anyn_supported(N)) QB_FAIL("from_fourier: unsupported N");
		anyn_from_fourier(N, ngrids, Wf, Wv, s);
	}
}

void transport(int npts, int ncells, const double *in, double *out, const double *A_dev, double h, double dt, int bc, cudaStream_t s) {
	if (ncells <= 0 || npts <= 0) return;
	TransportParams p{};
	p.ncells = ncells; p.npts = npts; p.in = in; p.out = out; p.A = A_dev; p.h = h; p.dt = dt; p.bc = bc;
	const long n = (long)npts * ncells;
	ProfScope ps("transport", s);
	k_transport<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(p);
	QB_CUDA(cudaGetLastError());
}

void transport_maxwell_lines(int m, int ncells, const double *in, double *out, const double *A_dev, double h, double dt,
                             double lambda, const double *flux_dev, const double *UL, const double *UR, cudaStream_t s) {
	if (ncells <= 0 || m <= 0) return;
	MaxwellParams p{};
	p.ncells = ncells; p.m = m; p.remapN = 0; p.ncomp = 1;
	p.in = in; p.out = out; p.A = A_dev; p.h = h; p.dt = dt; p.lambda = lambda;
	p.flux = flux_dev; p.UL = UL; p.UR = UR;
	const long n = (long)m * ncells;
	k_transport_maxwell<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(p);
	QB_CUDA(cudaGetLastError());
}

void flux_pair(int m, const double *A_dev, const double *U_dev, double *out_dev, cudaStream_t s) {
	k_flux_pair<<<1, 32, 0, s>>>(m, 0, A_dev, U_dev, out_dev);
	QB_CUDA(cudaGetLastError());
}

namespace {
// ---------------------------------------------------------------------------
// collision invariants.  The continuous collision operator conserves the
// mass, momentum and energy of the trace component w0 (Cc_0 = 0; Cd_0 and the
// magnetic term move none of them); the discrete operator keeps them only to
// its quadrature accuracy (and the FP32 form to its rounding).  With
// conservation switched on, the velocity-space step restores them: with
// phi = (1, v_x, v_y, |v|^2) (grid-index units; the span does not depend on
// the scale) and m_a = sum_v phi_a w0, the post-collision w0 becomes
// w0 + |w0| sum_a lambda_a phi_a with lambda solving G lambda = m_before - m_after,
// G_ab = sum_v |w0| phi_a phi_b.  Every sum is a fixed-order FP64 tree.
constexpr int kInvThreads = 256;

__device__ __forceinline__ void inv_basis(int q, int N, double (&phi)[4]) {
	const int l = q / N, k = q % N;                       // l: v_x (slow index), k: v_y
	const double vx = l < N / 2 ? l : l - N, vy = k < N / 2 ? k : k - N;
	phi[0] = 1.0; phi[1] = vx; phi[2] = vy; phi[3] = vx * vx + vy * vy;
}

template <int K>
__device__ __forceinline__ void inv_block_sum(double (&v)[K], double *sh) {
	for (int k = 0; k < K; k++) sh[k * kInvThreads + threadIdx.x] = v[k];
	__syncthreads();
	for (int st = kInvThreads / 2; st > 0; st >>= 1) {
		if (threadIdx.x < st)
			for (int k = 0; k < K; k++) sh[k * kInvThreads + threadIdx.x] += sh[k * kInvThreads + threadIdx.x + st];
		__syncthreads();
	}
	for (int k = 0; k < K; k++) v[k] = sh[k * kInvThreads];
	__syncthreads();
}

__global__ void __launch_bounds__(kInvThreads) k_invariants(int N, const double *__restrict__ V, double *__restrict__ inv) {
	__shared__ double sh[4 * kInvThreads];
	const int NN = N * N;
	const double *w0 = V + (long)blockIdx.x * 4 * NN;
	double m[4] = { 0, 0, 0, 0 };
	for (int q = threadIdx.x; q < NN; q += kInvThreads) {
		double phi[4];
		inv_basis(q, N, phi);
		for (int a = 0; a < 4; a++) m[a] += phi[a] * w0[q];
	}
	inv_block_sum<4>(m, sh);
	if (threadIdx.x < 4) inv[blockIdx.x * 4 + threadIdx.x] = m[threadIdx.x];
}

__global__ void __launch_bounds__(kInvThreads) k_restore_invariants(int N, double *__restrict__ V, const double *__restrict__ inv) {
	__shared__ double sh[14 * kInvThreads];
	__shared__ double lam[4];
	const int NN = N * N;
	double *w0 = V + (long)blockIdx.x * 4 * NN;
	double a[14];                                          // m[4], then G upper triangle (10)
	for (int k = 0; k < 14; k++) a[k] = 0.0;
	for (int q = threadIdx.x; q < NN; q += kInvThreads) {
		double phi[4];
		inv_basis(q, N, phi);
		const double w = w0[q], aw = fabs(w);
		for (int i = 0; i < 4; i++) a[i] += phi[i] * w;
		int t = 4;
		for (int i = 0; i < 4; i++)
			for (int j = i; j < 4; j++) a[t++] += aw * phi[i] * phi[j];
	}
	inv_block_sum<14>(a, sh);
	if (threadIdx.x == 0) {
		double G[4][5];
		int t = 4;
		for (int i = 0; i < 4; i++)
			for (int j = i; j < 4; j++) { G[i][j] = a[t]; G[j][i] = a[t]; t++; }
		for (int i = 0; i < 4; i++) G[i][4] = inv[blockIdx.x * 4 + i] - a[i];
		// Gaussian elimination with partial pivoting (G is symmetric positive semidefinite)
		bool ok = true;
		for (int c = 0; c < 4; c++) {
			int piv = c;
			for (int r = c + 1; r < 4; r++) if (fabs(G[r][c]) > fabs(G[piv][c])) piv = r;
			if (!(fabs(G[piv][c]) > 0.0)) { ok = false; break; }
			if (piv != c) for (int k = 0; k < 5; k++) { const double x = G[c][k]; G[c][k] = G[piv][k]; G[piv][k] = x; }
			for (int r = c + 1; r < 4; r++) {
				const double f = G[r][c] / G[c][c];
				for (int k = c; k < 5; k++) G[r][k] -= f * G[c][k];
			}
		}
		if (ok)
			for (int i = 3; i >= 0; i--) {
				double x = G[i][4];
				for (int k = i + 1; k < 4; k++) x -= G[i][k] * lam[k];
				lam[i] = x / G[i][i];
			}
		else
			for (int i = 0; i < 4; i++) lam[i] = 0.0;       // degenerate cell (w0 = 0 almost everywhere): leave it
	}
	__syncthreads();
	for (int q = threadIdx.x; q < NN; q += kInvThreads) {
		double phi[4];
		inv_basis(q, N, phi);
		const double w = w0[q];
		w0[q] = w + fabs(w) * (lam[0] * phi[0] + lam[1] * phi[1] + lam[2] * phi[2] + lam[3] * phi[3]);
	}
}

}  // namespace

void fourier_collision(Workspace &ws, const QuadSet &q, int nc, double *V, const double *B, double dt, cudaStream_t s) {
	const int N = ws.N;
	const long cs = 4L * N * N;
	if (nc <= 0) return;
	const bool restore = ws.conserve != 0;
	if (restore) {
		ws.inv.ensure(sizeof(double) * 4 * nc);
		ProfScope ps("invariants", s);
		k_invariants<<<nc, kInvThreads, 0, s>>>(N, V, ws.inv.as<double>());
		QB_CUDA(cudaGetLastError());
	}
	ws.fa.ensure(sizeof(double2) * cs * nc);
	ws.fb.ensure(sizeof(double2) * cs * nc);
	to_fourier(N, 4 * nc, V, ws.fa.as<double2>(), s);
	collision_step(ws, q, nc, ws.fa.as<double2>(), B, dt, ws.fb.as<double2>(), s);
	from_fourier(N, 4 * nc, ws.fb.as<double2>(), V, s);
	if (restore) {
		ProfScope ps("invariants", s);
		k_restore_invariants<<<nc, kInvThreads, 0, s>>>(N, V, ws.inv.as<double>());
		QB_CUDA(cudaGetLastError());
	}
}

void inhom_step(Workspace &ws, const QuadSet &q, int ncells, const double *W, double *Wnext, const double *A_dev,
                double h, double dt, const double *Bext, int bc, cudaStream_t s) {
	const int N = ws.N;
	const long cs = 4L * N * N;
	ws.va.ensure(sizeof(double) * cs * ncells);
	double *Vt = ws.va.as<double>();
	transport((int)cs, ncells, W, Vt, A_dev, h, 0.5 * dt, bc, s);
	const int i0 = (bc == 1) ? 1 : 0, i1 = (bc == 1) ? ncells - 1 : ncells;
	fourier_collision(ws, q, i1 - i0, Vt + i0 * cs, Bext ? Bext + 3 * i0 : nullptr, dt, s);   // null Bext: no field
	transport((int)cs, ncells, Vt, Wnext, A_dev, h, 0.5 * dt, bc, s);
}

void inhom_step_maxwell(Workspace &ws, const QuadSet &q, int ncells, const double *W, double *Wnext, const double *vx_dev,
                        double h, double dt, double lambda, const double *WL, const double *WR, const double *Bext, cudaStream_t s) {
	const int N = ws.N, m = N * N;
	const long cs = 4L * m;
	ws.va.ensure(sizeof(double) * cs * ncells);
	ws.aux2.ensure(sizeof(double) * (8 + 8L * m));
	double *bnd = ws.aux2.as<double>(), *UL = bnd + 8, *UR = UL + 4L * m;
	double *Vt = ws.va.as<double>();
	k_maxwell_setup<<<1, 256, 0, s>>>(N, vx_dev, WL, WR, W, W + (ncells - 1) * cs, bnd, UL, UR);
	QB_CUDA(cudaGetLastError());
	MaxwellParams p{};
	p.ncells = ncells; p.m = m; p.remapN = N; p.ncomp = 4;
	p.A = vx_dev; p.h = h; p.dt = 0.5 * dt; p.lambda = lambda; p.flux = bnd + 2; p.UL = UL; p.UR = UR;
	const unsigned nb = (unsigned)((cs * ncells + 255) / 256);
	p.in = W; p.out = Vt;
	k_transport_maxwell<<<nb, 256, 0, s>>>(p);
	QB_CUDA(cudaGetLastError());
	fourier_collision(ws, q, ncells, Vt, Bext, dt, s);
	k_maxwell_flux<<<1, 32, 0, s>>>(N, vx_dev, Vt, Vt + (ncells - 1) * cs, bnd);
	p.in = Vt; p.out = Wnext;
	k_transport_maxwell<<<nb, 256, 0, s>>>(p);
	QB_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// FFTW-API plans
bool fft2_generic_supported(int n0, int n1) {
	return n0 == n1 && (n0 == 8 || n0 == 16 || n0 == 32 || n0 == 64);
}

namespace {
template <int L, int DIR> void launch_generic(bool r2c, const void *in, double2 *out, cudaStream_t s) {
	const size_t sm = sizeof(double2) * (L * (L + 1) + L);
	static DeviceFlag init;
	if (!init) { set_smem(k_fft2_generic<L, DIR>, sm); init = true; }
	k_fft2_generic<L, DIR><<<1, Len<L>::T * L, sm, s>>>(in, out, r2c ? 1 : 0);
	QB_CUDA(cudaGetLastError());
}
}  // namespace

void fft2_generic(int L, int dir, bool r2c, const void *in_dev, double2 *out_dev, cudaStream_t s) {
	if (dir < 0) {
		switch (L) {
		case 8: launch_generic<8, -1>(r2c, in_dev, out_dev, s); break;
		case 16: launch_generic<16, -1>(r2c, in_dev, out_dev, s); break;
		case 32: launch_generic<32, -1>(r2c, in_dev, out_dev, s); break;
		case 64: launch_generic<64, -1>(r2c, in_dev, out_dev, s); break;
		default: QB_FAIL("fft2: unsupported size");
		}
	} else {
		switch (L) {
		case 8: launch_generic<8, 1>(r2c, in_dev, out_dev, s); break;
		case 16: launch_generic<16, 1>(r2c, in_dev, out_dev, s); break;
		case 32: launch_generic<32, 1>(r2c, in_dev, out_dev, s); break;
		case 64: launch_generic<64, 1>(r2c, in_dev, out_dev, s); break;
		default: QB_FAIL("fft2: unsupported size");
		}
	}
}

}  // namespace qb
