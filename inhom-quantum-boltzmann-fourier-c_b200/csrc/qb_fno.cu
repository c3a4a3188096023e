// qb_fno.cu — a Fourier-neural-operator surrogate of the collision operator
// C[W] = Cc + Cd on one velocity-space cell, with hand-written forward,
// backward and Adam kernels (FP32 arithmetic, FP64 inputs and outputs; on
// request the pointwise maps and the truncated DFTs run on the tensor cores
// with BF16 operands and FP32 accumulation).
//
// Model (per cell; fields on the N x N velocity grid, point p = (l, k_v)):
//   x        = the 4 Pauli components and their 10 pairwise products (the
//              operator is cubic in W), each times a fixed input scale
//   h0       = A x + a                                  lift 14 -> w channels
//   layer l: H_i(k) = sum_p h_i(p) e^{-i theta(k,p)}     truncated DFT, modes
//            O_o(k) = sum_i R_l[i,o,k] H_i(k)            kx in [-m+1, m-1], ky in [0, m)
//            s_o(p) = Re sum_k O_o(k) e^{+i theta(k,p)} / N^2
//            u      = s + W_l h + b_l,  h' = gelu(u) (last layer: h' = u)
//   y        = Q h + q,  C~ = y * out_scale (per Pauli component)
// with theta(k, p) = 2 pi (kx l + ky k_v) / N.  The truncated transforms are
// separable matrix products (N x m then (2m-1) x N twiddle sums per field):
// only m of N frequencies per direction are kept, so this costs less than a
// full FFT and its adjoint is the same pair of sums.  Gradients use the
// complex convention dL/dRe + i dL/dIm: for O = R H, dR = dO conj(H) and
// dH = dO conj(R); for H = DFT(h) of a real field, dh = Re IDFT(dH) (no
// 1/N^2).  Every reduction (loss, weight gradients) is a fixed-order tree or
// a per-chunk partial sum reduced in order: results are deterministic.
#include "qb_engine.h"
#include "qb_kernels.cuh"
#include "qb_umma.cuh"

#include <cuda_bf16.h>

extern "C" {
#include "qbgpu.h"
}

#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

namespace {

constexpr int kFnoMaxWidth = 64;
constexpr int kFnoIn = 14;                   // input features: w_c (4) and w_i w_j, i <= j (10)

struct InScale { double s[kFnoIn]; };

struct Offsets {
	long A, a, Q, q;
	std::vector<long> Rr, Ri, W, b;
	long total;
};

Offsets offsets(int w, int K, int L) {
	Offsets o;
	long p = 0;
	o.A = p; p += (long)w * kFnoIn;
	o.a = p; p += w;
	for (int l = 0; l < L; l++) {
		o.Rr.push_back(p); p += (long)w * w * K;
		o.Ri.push_back(p); p += (long)w * w * K;
		o.W.push_back(p); p += (long)w * w;
		o.b.push_back(p); p += w;
	}
	o.Q = p; p += 4L * w;
	o.q = p; p += 4;
	o.total = p;
	return o;
}

__device__ __forceinline__ float gelu_f(float u) { return 0.5f * u * (1.0f + erff(u * 0.70710678118654752f)); }
__device__ __forceinline__ float dgelu_f(float u) {
	return 0.5f * (1.0f + erff(u * 0.70710678118654752f)) + u * expf(-0.5f * u * u) * 0.39894228040143268f;
}

// input features x[b][f][p] (FP32) of the FP64 state: f < 4: w_f; then the
// products w_i w_j (i <= j) in the order (0,0), (0,1), ..., (3,3); feature f
// is multiplied by sc.s[f]
__global__ void k_fno_in(int B, int P, const double *__restrict__ W, InScale sc, float *__restrict__ x) {
	const long n = (long)B * P;
	for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
		const long b = t / P, p = t % P;
		double w[4];
		for (int c = 0; c < 4; c++) w[c] = W[(b * 4 + c) * P + p];
		float *o = x + b * kFnoIn * P + p;
		int f = 0;
		for (int c = 0; c < 4; c++, f++) o[(long)f * P] = (float)(sc.s[f] * w[c]);
		for (int i = 0; i < 4; i++)
			for (int j = i; j < 4; j++, f++) o[(long)f * P] = (float)(sc.s[f] * w[i] * w[j]);
	}
}

// out[b][o][p] = sum_i M[o][i] in[b][i][p] + bias[o] (+ add[b][o][p]); act: store gelu in hout and u in uout
__global__ void k_fno_pointwise(int B, int P, int cin, int cout, const float *__restrict__ in, const float *__restrict__ M,
                                const float *__restrict__ bias, const float *__restrict__ add, float *__restrict__ uout,
                                float *__restrict__ hout, int act) {
	__shared__ float Ms[kFnoMaxWidth * kFnoMaxWidth + kFnoMaxWidth];
	for (int i = threadIdx.x; i < cin * cout; i += blockDim.x) Ms[i] = M[i];
	for (int i = threadIdx.x; i < cout; i += blockDim.x) Ms[cin * cout + i] = bias ? bias[i] : 0.0f;
	__syncthreads();
	const long n = (long)B * P;
	for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
		const long b = t / P, p = t % P;
		float v[kFnoMaxWidth];
		for (int i = 0; i < cin; i++) v[i] = in[(b * cin + i) * P + p];
		for (int o = 0; o < cout; o++) {
			float s = Ms[cin * cout + o];
			for (int i = 0; i < cin; i++) s = fmaf(Ms[o * cin + i], v[i], s);
			const long oi = (b * cout + o) * P + p;
			if (add) s += add[oi];
			if (uout) uout[oi] = s;
			hout[oi] = act ? gelu_f(s) : s;
		}
	}
}

// out[b][i][p] = sum_o M[o][i] in[b][o][p]  (transpose product: backward of a pointwise map)
__global__ void k_fno_pointwise_t(int B, int P, int cin, int cout, const float *__restrict__ in, const float *__restrict__ M,
                                  float *__restrict__ out) {
	__shared__ float Ms[kFnoMaxWidth * kFnoMaxWidth];
	for (int i = threadIdx.x; i < cin * cout; i += blockDim.x) Ms[i] = M[i];
	__syncthreads();
	const long n = (long)B * P;
	for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
		const long b = t / P, p = t % P;
		float v[kFnoMaxWidth];
		for (int o = 0; o < cout; o++) v[o] = in[(b * cout + o) * P + p];
		for (int i = 0; i < cin; i++) {
			float s = 0.0f;
			for (int o = 0; o < cout; o++) s = fmaf(Ms[o * cin + i], v[o], s);
			out[(b * cin + i) * P + p] = s;
		}
	}
}

// truncated forward DFT of every (b, c) field: H[b][c][k] = scale * sum_p f(p) e^{-i theta(k,p)}
__global__ void k_fno_dft(int N, int m, const float *__restrict__ f, float2 *__restrict__ H, float scale) {
	extern __shared__ float sm[];
	const int P = N * N, K = (2 * m - 1) * m;
	float *fs = sm;                                   // P
	float2 *T = reinterpret_cast<float2 *>(fs + P);  // N x m
	float2 *tw = T + N * m;                          // N: e^{-2 pi i j / N}
	const long bc = blockIdx.x;
	for (int i = threadIdx.x; i < P; i += blockDim.x) fs[i] = f[bc * P + i];
	for (int j = threadIdx.x; j < N; j += blockDim.x) {
		double s, c;
		sincospi(-2.0 * j / N, &s, &c);
		tw[j] = make_float2((float)c, (float)s);
	}
	__syncthreads();
	for (int t = threadIdx.x; t < N * m; t += blockDim.x) {
		const int l = t / m, ky = t % m;
		float re = 0.0f, im = 0.0f;
		for (int kv = 0; kv < N; kv++) {
			const float2 w = tw[(ky * kv) % N];
			const float v = fs[l * N + kv];
			re = fmaf(v, w.x, re);
			im = fmaf(v, w.y, im);
		}
		T[t] = make_float2(re, im);
	}
	__syncthreads();
	for (int t = threadIdx.x; t < K; t += blockDim.x) {
		const int kxi = t / m, ky = t % m, kx = kxi - (m - 1);
		float re = 0.0f, im = 0.0f;
		for (int l = 0; l < N; l++) {
			const float2 w = tw[(((kx * l) % N) + N) % N];
			const float2 a = T[l * m + ky];
			re += a.x * w.x - a.y * w.y;
			im += a.x * w.y + a.y * w.x;
		}
		H[bc * K + t] = make_float2(scale * re, scale * im);
	}
}

// truncated inverse: out[b][c][p] (=, or +=) scale * Re sum_k O[b][c][k] e^{+i theta(k,p)}
__global__ void k_fno_idft(int N, int m, const float2 *__restrict__ O, float *__restrict__ out, float scale, int accumulate) {
	extern __shared__ float sm[];
	const int P = N * N, K = (2 * m - 1) * m;
	float2 *Os = reinterpret_cast<float2 *>(sm);     // K
	float2 *U = Os + K;                              // N x m
	float2 *tw = U + N * m;                          // N: e^{+2 pi i j / N}
	const long bc = blockIdx.x;
	for (int i = threadIdx.x; i < K; i += blockDim.x) Os[i] = O[bc * K + i];
	for (int j = threadIdx.x; j < N; j += blockDim.x) {
		double s, c;
		sincospi(2.0 * j / N, &s, &c);
		tw[j] = make_float2((float)c, (float)s);
	}
	__syncthreads();
	for (int t = threadIdx.x; t < N * m; t += blockDim.x) {
		const int l = t / m, ky = t % m;
		float re = 0.0f, im = 0.0f;
		for (int kxi = 0; kxi < 2 * m - 1; kxi++) {
			const int kx = kxi - (m - 1);
			const float2 w = tw[(((kx * l) % N) + N) % N];
			const float2 a = Os[kxi * m + ky];
			re += a.x * w.x - a.y * w.y;
			im += a.x * w.y + a.y * w.x;
		}
		U[t] = make_float2(re, im);
	}
	__syncthreads();
	for (int t = threadIdx.x; t < P; t += blockDim.x) {
		const int l = t / N, kv = t % N;
		float s = 0.0f;
		for (int ky = 0; ky < m; ky++) {
			const float2 w = tw[(ky * kv) % N];
			const float2 a = U[l * m + ky];
			s += a.x * w.x - a.y * w.y;
		}
		if (accumulate) out[bc * P + t] += scale * s;
		else out[bc * P + t] = scale * s;
	}
}

// mode mixing: fwd (conj = 0): out[b][o][k] = sum_i R[i][o][k] in[b][i][k]
//              bwd (conj = 1): out[b][i][k] = sum_o conj(R[i][o][k]) in[b][o][k]
__global__ void k_fno_mix(int B, int w, int K, const float2 *__restrict__ in, const float *__restrict__ Rr, const float *__restrict__ Ri,
                          float2 *__restrict__ out, int conj) {
	const long n = (long)B * w * K;
	for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
		const int k = (int)(t % K);
		const int c = (int)((t / K) % w);
		const long b = t / ((long)K * w);
		float re = 0.0f, im = 0.0f;
		for (int j = 0; j < w; j++) {
			const long ri = conj ? ((long)c * w + j) * K + k : ((long)j * w + c) * K + k;
			const float rr = Rr[ri], rim = conj ? -Ri[ri] : Ri[ri];
			const float2 v = in[((long)b * w + j) * K + k];
			re += rr * v.x - rim * v.y;
			im += rr * v.y + rim * v.x;
		}
		out[t] = make_float2(re, im);
	}
}

// weight gradient of the mode mixing: dR[i][o][k] = sum_b GO[b][o][k] conj(H[b][i][k])
__global__ void k_fno_rgrad(int B, int w, int K, const float2 *__restrict__ GO, const float2 *__restrict__ H, float *__restrict__ gRr,
                            float *__restrict__ gRi) {
	const long n = (long)w * w * K;
	for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
		const int k = (int)(t % K);
		const int o = (int)((t / K) % w);
		const int i = (int)(t / ((long)K * w));
		float re = 0.0f, im = 0.0f;
		for (int b = 0; b < B; b++) {
			const float2 g = GO[((long)b * w + o) * K + k], h = H[((long)b * w + i) * K + k];
			re += g.x * h.x + g.y * h.y;
			im += g.y * h.x - g.x * h.y;
		}
		gRr[t] = re;
		gRi[t] = im;
	}
}

// partial[chunk][cx][cy] = sum over the chunk's (b, p) of X[b][cx][p] * Y[b][cy][p]
// (Y == nullptr: Y = 1, cy = 1).  Chunks of 64 points; fixed order.
constexpr int kChunk = 64;
__global__ void k_fno_outer(int B, int P, int cx, int cy, const float *__restrict__ X, const float *__restrict__ Y, float *__restrict__ partial) {
	__shared__ float xs[kFnoMaxWidth][kChunk + 1];
	__shared__ float ys[kFnoMaxWidth][kChunk + 1];
	const long n = (long)B * P;
	const long t0 = (long)blockIdx.x * kChunk;
	for (int i = threadIdx.x; i < kChunk; i += blockDim.x) {
		const long t = t0 + i;
		const bool ok = t < n;
		const long b = ok ? t / P : 0, p = ok ? t % P : 0;
		for (int c = 0; c < cx; c++) xs[c][i] = ok ? X[(b * cx + c) * P + p] : 0.0f;
		for (int c = 0; c < cy; c++) ys[c][i] = ok ? (Y ? Y[(b * cy + c) * P + p] : 1.0f) : 0.0f;
	}
	__syncthreads();
	for (int o = threadIdx.x; o < cx * cy; o += blockDim.x) {
		const int a = o / cy, c = o % cy;
		float s = 0.0f;
		for (int i = 0; i < kChunk; i++) s = fmaf(xs[a][i], ys[c][i], s);
		partial[(long)blockIdx.x * cx * cy + o] = s;
	}
}

// out[j] = sum_c partial[c][j] in chunk order
__global__ void k_fno_reduce(int nchunk, int count, const float *__restrict__ partial, float *__restrict__ out) {
	const int j = blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= count) return;
	float s = 0.0f;
	for (int c = 0; c < nchunk; c++) s += partial[(long)c * count + j];
	out[j] = s;
}

// dy = 2 (y - t / scale) / n, partial[block] = sum of squares (fixed tree)
__global__ void k_fno_loss(int B, int P, const float *__restrict__ y, const double *__restrict__ target, double s0, double s1, double s2,
                           double s3, float *__restrict__ dy, double *__restrict__ partial) {
	__shared__ double sh[256];
	const long n = (long)B * 4 * P;
	const double inv_n = 1.0 / (double)n;
	const double sc[4] = { s0, s1, s2, s3 };
	double acc = 0.0;
	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
		const int c = (int)((i / P) % 4);
		const double d = (double)y[i] - target[i] / sc[c];
		acc += d * d;
		dy[i] = (float)(2.0 * d * inv_n);
	}
	sh[threadIdx.x] = acc;
	__syncthreads();
	for (int s = 128; s > 0; s >>= 1) {
		if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
		__syncthreads();
	}
	if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

__global__ void k_fno_gelu_bwd(long n, const float *__restrict__ u, float *__restrict__ d) {
	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) d[i] *= dgelu_f(u[i]);
}

__global__ void k_fno_out(long n, int P, const float *__restrict__ y, double s0, double s1, double s2, double s3, double *__restrict__ C) {
	const double sc[4] = { s0, s1, s2, s3 };
	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
		C[i] = (double)y[i] * sc[(i / P) % 4];
}

__global__ void k_fno_adam(long n, float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v, float lr,
                           float b1, float b2, float eps, float c1, float c2) {
	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
		const float gi = g[i];
		const float mi = b1 * m[i] + (1.0f - b1) * gi;
		const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
		m[i] = mi;
		v[i] = vi;
		w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
	}
}

// ---------------------------------------------------------------------------
// The pointwise channel maps on the tensor cores (BF16 operands, FP32
// accumulation): for the points of a tile of 128 (rows of the flattened
// (b, p) index) D[row][n] = sum_k X[row][k] Wt[n][k] with one tcgen05.mma
// of M = 128, N = npad, K = 16 per step.
//   trans = 0 (forward map): X = in[b][k][p] (k < kin = cin), Wt[n][k] = M[n cin + k],
//            out = D + bias (+ add); act: uout = u, hout = gelu(u), else hout = u;
//   trans = 1 (its transpose, backward): X = in[b][k][p] (k < kin = cout),
//            Wt[n][k] = M[k cin + n] (n < nout = cin), hout = D.
// A (128 x 64 BF16) and B (npad x 64 BF16) are K-major with the 128-byte
// swizzle; D is 64 FP32 columns of tensor memory, row r in lane r, read back
// by the thread of that row.  Persistent CTAs of 128 threads stride over the
// tiles.  The MMA completion wait is bounded; a wait that runs out sets the
// error word and leaves the outputs of that tile undefined.
namespace fnomma {
constexpr int kThreads = 128, kRows = 128, kMaxK = 64, kCols = 64;
constexpr uint32_t oA = 0, oB = kRows * 128, kUsed = oB + kMaxK * 128;
// dynamic shared memory: the operands, 1024-byte alignment slack, and enough
// more that at most 7 CTAs share an SM (7 x 64 tensor-memory columns <= 512)
constexpr uint32_t kSmem = 33 * 1024;
static_assert(kUsed + 1024 <= kSmem, "operand tiles fit");
constexpr unsigned kPolls = 1u << 24;
}  // namespace fnomma

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
	__nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
	return *reinterpret_cast<uint32_t *>(&v);
}

__global__ void __launch_bounds__(fnomma::kThreads) k_fno_pointwise_mma(int B, int P, int cin, int cout, int trans,
                                                                         const float *__restrict__ in, const float *__restrict__ M,
                                                                         const float *__restrict__ bias, const float *__restrict__ add,
                                                                         float *__restrict__ uout, float *__restrict__ hout, int act,
                                                                         int *err) {
	using namespace fnomma;
	using namespace qb;
	extern __shared__ unsigned char smem_raw[];
	unsigned char *base = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
	__shared__ uint64_t mbar;
	__shared__ uint32_t tslot;
	__shared__ int abort_flag;
	const int tid = threadIdx.x, warp = tid >> 5;
	const int kin = trans ? cout : cin, nout = trans ? cin : cout;
	const int kpad = (kin + 15) & ~15, npad = (nout + 15) & ~15;
	// B: the weights as Wt[n][k], BF16, zero beyond (nout, kin)
	for (int i = tid; i < kMaxK * (kMaxK / 2); i += kThreads) {
		const int n = i / (kMaxK / 2), k = 2 * (i % (kMaxK / 2));
		float w0 = 0.0f, w1 = 0.0f;
		if (n < nout) {
			if (k < kin) w0 = trans ? M[k * cin + n] : M[n * cin + k];
			if (k + 1 < kin) w1 = trans ? M[(k + 1) * cin + n] : M[n * cin + k + 1];
		}
		*reinterpret_cast<uint32_t *>(base + oB + umma::kmajor_off16(n, k)) = pack_bf16x2(w0, w1);
	}
	if (tid == 0) {
		umma::mbar_init(&mbar, 1);
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
		abort_flag = 0;
	}
	if (warp == 0) tmem_alloc(&tslot, kCols);
	tmem_fence_before();
	__syncthreads();
	tmem_fence_after();
	const uint32_t tmem = tslot;
	const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);      // this warp's 32 lanes
	uint32_t idesc = 0;
	switch (npad) {
	case 16: idesc = umma::idesc_bf16<128, 16>(); break;
	case 32: idesc = umma::idesc_bf16<128, 32>(); break;
	case 48: idesc = umma::idesc_bf16<128, 48>(); break;
	default: idesc = umma::idesc_bf16<128, 64>(); break;
	}
	const long rows = (long)B * P, ntiles = (rows + kRows - 1) / kRows;
	unsigned phase = 0;
	for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
		const long row = tile * kRows + tid;
		const bool live = row < rows;
		const long b = live ? row / P : 0, p = live ? row % P : 0;
		// A: this thread's row (its point), BF16, zero beyond kin
		const float *x = in + b * (long)kin * P + p;
#pragma unroll 4
		for (int k = 0; k < kMaxK; k += 2) {
			const float x0 = (live && k < kin) ? x[(long)k * P] : 0.0f;
			const float x1 = (live && k + 1 < kin) ? x[(long)(k + 1) * P] : 0.0f;
			*reinterpret_cast<uint32_t *>(base + oA + umma::kmajor_off16(tid, k)) = pack_bf16x2(x0, x1);
		}
		umma::fence_async_smem();
		tmem_fence_before();
		__syncthreads();
		tmem_fence_after();
		if (tid == 0) {
			const uint32_t a0 = umma::smem_u32(base + oA), b0 = umma::smem_u32(base + oB);
			for (int k = 0; k < kpad; k += 16)
				umma::mma_f16(tmem, umma::desc_sw128(a0 + 2 * k, 16, 1024), umma::desc_sw128(b0 + 2 * k, 16, 1024), idesc, k > 0 ? 1u : 0u);
			umma::commit(&mbar);
		}
		if (!abort_flag && !umma::mbar_wait(&mbar, phase, kPolls)) {
			abort_flag = 1;
			if (err) atomicExch(err, 1);
		}
		phase ^= 1u;
		tmem_fence_after();
		// epilogue: this thread's row of D, 16 columns at a time
		for (int n0 = 0; n0 < npad; n0 += 16) {
			float d[16];
			umma::tmem_ld16(trow + (uint32_t)n0, d);
			asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
			if (!live) continue;
#pragma unroll
			for (int j = 0; j < 16; j++) {
				const int n = n0 + j;
				if (n >= nout) break;
				const long oi = (b * nout + n) * (long)P + p;
				float v = d[j];
				if (!trans) {
					if (bias) v += bias[n];
					if (add) v += add[oi];
					if (uout) uout[oi] = v;
					hout[oi] = act ? gelu_f(v) : v;
				} else {
					hout[oi] = v;
				}
			}
		}
		tmem_fence_before();
		__syncthreads();                      // D read and A free before the next tile's MMA
		tmem_fence_after();
	}
	tmem_fence_before();
	__syncthreads();
	tmem_fence_after();
	if (warp == 0) tmem_dealloc(tmem, kCols);
}

// ---------------------------------------------------------------------------
// A grouped row GEMM on the tensor cores (BF16 operands, FP32 accumulation)
// for the separable truncated DFTs and the mode mixing: for each of the
// bm.groups() groups and 128-row tiles of its bm.rows() rows,
// D[row][n] = sum_k A[row][k] Bg[n][k], k < K <= 128, n < Nn <= 128, with A
// read through the loader ld(g, row, k), Bg through bm(g, n, k) (rebuilt when a
// CTA moves to another group), and every row of D handed whole to the
// epilogue ep(g, row, d).  Operands K-major with the 128-byte swizzle in two
// 64-element atoms; D in 128 tensor-memory columns.  Persistent CTAs of 128
// threads; the MMA completion wait is bounded (a wait that runs out sets the
// error word).
namespace fnotc {
constexpr int kThreads = 128, kRows = 128, kMaxK = 128, kMaxN = 128, kCols = 128;
constexpr uint32_t oA = 0, oB = kRows * kMaxK * 2, kUsed = oB + kMaxN * kMaxK * 2;
// operands, alignment slack, and enough more that at most 3 CTAs share an SM (3 x 128 columns <= 512)
constexpr uint32_t kSmem = 72 * 1024;
static_assert(kUsed + 1024 <= kSmem, "operand tiles fit");
constexpr unsigned kPolls = 1u << 24;
__host__ __device__ constexpr uint32_t off(int R, int r, int k) {
	return (uint32_t)((k >> 6) * R * 128) + qb::umma::kmajor_off16(r, k & 63);
}
}  // namespace fnotc

template <class Ld, class Ep, class Bb>
__global__ void __launch_bounds__(fnotc::kThreads) k_fno_tc(const Ld ld, const Ep ep, const Bb bm, int K, int Nn, int *err) {
	using namespace fnotc;
	using namespace qb;
	extern __shared__ unsigned char smem_raw[];
	unsigned char *base = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
	__shared__ uint64_t mbar;
	__shared__ uint32_t tslot;
	__shared__ int abort_flag;
	const int tid = threadIdx.x, warp = tid >> 5;
	const int kpad = (K + 15) & ~15, npad = (Nn + 15) & ~15;
	if (tid == 0) {
		umma::mbar_init(&mbar, 1);
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
		abort_flag = 0;
	}
	if (warp == 0) tmem_alloc(&tslot, kCols);
	tmem_fence_before();
	__syncthreads();
	tmem_fence_after();
	const uint32_t tmem = tslot;
	const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);
	const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(npad >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
	const long rows = bm.rows(), tpg = (rows + kRows - 1) / kRows, ntiles = tpg * bm.groups();
	unsigned phase = 0;
	int cur_g = -1;
	for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
		const int g = (int)(tile / tpg);
		const long row = (tile % tpg) * kRows + tid;
		const bool live = row < rows;
		if (g != cur_g) {                     // this group's B (the previous MMA has completed)
			for (int i = tid; i < npad * (kpad / 2); i += kThreads) {
				const int n = i / (kpad / 2), k = 2 * (i % (kpad / 2));
				const float b0 = (n < Nn && k < K) ? bm(g, n, k) : 0.0f;
				const float b1 = (n < Nn && k + 1 < K) ? bm(g, n, k + 1) : 0.0f;
				*reinterpret_cast<uint32_t *>(base + oB + off(npad, n, k)) = pack_bf16x2(b0, b1);
			}
			cur_g = g;
		}
		for (int k = 0; k < kpad; k += 2) {
			const float x0 = (live && k < K) ? ld(g, row, k) : 0.0f;
			const float x1 = (live && k + 1 < K) ? ld(g, row, k + 1) : 0.0f;
			*reinterpret_cast<uint32_t *>(base + oA + off(kRows, tid, k)) = pack_bf16x2(x0, x1);
		}
		umma::fence_async_smem();
		tmem_fence_before();
		__syncthreads();
		tmem_fence_after();
		if (tid == 0) {
			const uint32_t a0 = umma::smem_u32(base + oA), b0 = umma::smem_u32(base + oB);
			for (int k = 0; k < kpad; k += 16) {
				const uint32_t ao = (uint32_t)((k >> 6) * kRows * 128 + (k & 63) * 2);
				const uint32_t bo = (uint32_t)((k >> 6) * npad * 128 + (k & 63) * 2);
				umma::mma_f16(tmem, umma::desc_sw128(a0 + ao, 16, 1024), umma::desc_sw128(b0 + bo, 16, 1024), idesc, k > 0 ? 1u : 0u);
			}
			umma::commit(&mbar);
		}
		if (!abort_flag && !umma::mbar_wait(&mbar, phase, kPolls)) {
			abort_flag = 1;
			if (err) atomicExch(err, 1);
		}
		phase ^= 1u;
		tmem_fence_after();
		float d[kMaxN];
#pragma unroll
		for (int c = 0; c < kMaxN / 16; c++) {
			if (16 * c < npad) {
				float v[16];
				umma::tmem_ld16(trow + (uint32_t)(16 * c), v);
				asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
				for (int j = 0; j < 16; j++) d[16 * c + j] = v[j];
			}
		}
		if (live) ep(g, row, d);
		tmem_fence_before();
		__syncthreads();
		tmem_fence_after();
	}
	tmem_fence_before();
	__syncthreads();
	tmem_fence_after();
	if (warp == 0) tmem_dealloc(tmem, kCols);
}

// the truncated DFT of a field f (N x N real) to H (K complex, kx in [-m+1, m-1],
// ky in [0, m)) as two row GEMMs:
//   1. along kv: T[fld][ky][l] = sum_kv f[fld][l][kv] e^{-2 pi i ky kv / N}   (rows (fld, l), K = N, Nn = 2m)
//   2. along l:  H[fld][kx][ky] = scale sum_l T[fld][ky][l] e^{-2 pi i kx l / N} (rows (fld, ky), K = 2N, Nn = 2(2m-1))
// and its inverse out[fld][l][kv] (=, +=) scale Re sum_k O[fld][k] e^{+i theta}:
//   A. along kx: U[fld][l][ky] = sum_kx O[fld][kx][ky] e^{+2 pi i kx l / N}      (rows (fld, ky), K = 2(2m-1), Nn = 2N)
//   B. along ky: out = scale Re sum_ky U[fld][l][ky] e^{+2 pi i ky kv / N}        (rows (fld, l), K = 2m, Nn = N)
// one fixed FP32 [Nn][K] matrix in global memory (the twiddles) for `nrows` rows
struct BMat {
	const float *Bm; int K; long nrows;
	__device__ long rows() const { return nrows; }
	__device__ int groups() const { return 1; }
	__device__ float operator()(int, int n, int k) const { return Bm[(long)n * K + k]; }
};
// mode mixing, one group per mode k: rows b (cells), A = [in_re | in_im] of the
// summed channels, outputs [out_re | out_im]; forward out_o = sum_i R[i][o] in_i,
// backward (conj) out_i = sum_o conj(R[i][o]) in_o (R[i][o][k] = Rr + i Ri)
struct BMix {
	const float *Rr, *Ri; int w, K, nb, conj;
	__device__ long rows() const { return nb; }
	__device__ int groups() const { return K; }
	__device__ float operator()(int g, int n, int k) const {
		const int c = n % w, j = k % w;           // output channel c, summed channel j
		const long ri = conj ? ((long)c * w + j) * K + g : ((long)j * w + c) * K + g;
		const float rr = Rr[ri], rim = conj ? -Ri[ri] : Ri[ri];
		// out_re = sum rr in_re - rim in_im, out_im = sum rim in_re + rr in_im
		if (n < w) return k < w ? rr : -rim;
		return k < w ? rim : rr;
	}
};
struct LdMix {
	const float2 *in; int w, K;
	__device__ float operator()(int g, long row, int k) const {
		const float2 v = in[(row * w + (k % w)) * (long)K + g];
		return k < w ? v.x : v.y;
	}
};
struct EpMix {
	float2 *out; int w, K;
	__device__ void operator()(int g, long row, const float (&d)[fnotc::kMaxN]) const {
		for (int c = 0; c < w; c++) out[(row * w + c) * (long)K + g] = make_float2(d[c], d[w + c]);
	}
};
struct LdDft1 { const float *f; int N; __device__ float operator()(int, long row, int k) const { return f[row * N + k]; } };
struct EpDft1 {
	float *T; int N, m;
	__device__ void operator()(int, long row, const float (&d)[fnotc::kMaxN]) const {
		const long fld = row / N;
		const int l = (int)(row % N);
		for (int ky = 0; ky < m; ky++) {
			float *t = T + (fld * m + ky) * 2L * N;
			t[l] = d[ky];
			t[N + l] = d[m + ky];
		}
	}
};
struct LdDft2 { const float *T; int N; __device__ float operator()(int, long row, int k) const { return T[row * 2L * N + k]; } };
struct EpDft2 {
	float2 *H; int m; float scale;
	__device__ void operator()(int, long row, const float (&d)[fnotc::kMaxN]) const {
		const int K = (2 * m - 1) * m, nk = 2 * m - 1;
		const long fld = row / m;
		const int ky = (int)(row % m);
		for (int kxi = 0; kxi < nk; kxi++) H[fld * K + kxi * m + ky] = make_float2(scale * d[kxi], scale * d[nk + kxi]);
	}
};
struct LdIdftA {
	const float2 *O; int m;
	__device__ float operator()(int, long row, int k) const {
		const int K = (2 * m - 1) * m, nk = 2 * m - 1;
		const long fld = row / m;
		const int ky = (int)(row % m);
		const float2 o = O[fld * K + (k % nk) * m + ky];
		return k < nk ? o.x : o.y;
	}
};
struct EpIdftA {
	float *U; int N, m;
	__device__ void operator()(int, long row, const float (&d)[fnotc::kMaxN]) const {
		const long fld = row / m;
		const int ky = (int)(row % m);
		for (int l = 0; l < N; l++) {
			float *u = U + (fld * N + l) * 2L * m;
			u[ky] = d[l];
			u[m + ky] = d[N + l];
		}
	}
};
struct LdIdftB { const float *U; int m; __device__ float operator()(int, long row, int k) const { return U[row * 2L * m + k]; } };
struct EpIdftB {
	float *out; int N; float scale; int accumulate;
	__device__ void operator()(int, long row, const float (&d)[fnotc::kMaxN]) const {
		float *o = out + row * N;           // row = fld N + l: out[fld][l][kv]
		for (int kv = 0; kv < N; kv++) o[kv] = accumulate ? o[kv] + scale * d[kv] : scale * d[kv];
	}
};

unsigned grid_for(long n) { return (unsigned)std::max<long>(1, std::min<long>((n + 255) / 256, 148L * 32)); }

}  // namespace

// the tensor-memory kernel of this file, for the engine's co-residency check
std::vector<qb::TmemKernel> qb::fno_tmem_kernels() {
	return { { (const void *)k_fno_pointwise_mma, fnomma::kSmem, fnomma::kThreads, fnomma::kCols, "k_fno_pointwise_mma" },
	         { (const void *)k_fno_tc<LdDft1, EpDft1, BMat>, fnotc::kSmem, fnotc::kThreads, fnotc::kCols, "k_fno_tc<dft 1>" },
	         { (const void *)k_fno_tc<LdDft2, EpDft2, BMat>, fnotc::kSmem, fnotc::kThreads, fnotc::kCols, "k_fno_tc<dft 2>" },
	         { (const void *)k_fno_tc<LdIdftA, EpIdftA, BMat>, fnotc::kSmem, fnotc::kThreads, fnotc::kCols, "k_fno_tc<idft A>" },
	         { (const void *)k_fno_tc<LdIdftB, EpIdftB, BMat>, fnotc::kSmem, fnotc::kThreads, fnotc::kCols, "k_fno_tc<idft B>" },
	         { (const void *)k_fno_tc<LdMix, EpMix, BMix>, fnotc::kSmem, fnotc::kThreads, fnotc::kCols, "k_fno_tc<mix>" } };
}

namespace {

// every launch is counted (and timed while profiling is on) under its kernel's name
template <class... P, class... A>
void launch(const char *name, void (*k)(P...), unsigned grid, unsigned block, size_t smem, cudaStream_t s, A... args) {
	qb::ProfScope ps(name, s);
	k<<<grid, block, smem, s>>>(args...);
	QB_CUDA(cudaGetLastError());
}

}  // namespace

struct qb_fno {
	int N = 0, w = 0, m = 0, L = 0, K = 0, P = 0;
	Offsets off;
	double scale[4] = { 1, 1, 1, 1 };
	InScale inscale = { { 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1 } };
	long adam_t = 0;
	qb::DevBuf params, grads, am, av;
	int cap = 0;                                  // batch the activation buffers hold
	qb::DevBuf x, y, dy, dh, tmp, lossp, partial;
	std::vector<qb::DevBuf> h, u, H;             // h[0..L], u[0..L-1], H[0..L-1]
	qb::DevBuf GO, GH;
	int use_tc = 0;                               // pointwise maps and truncated DFTs on the tensor cores (BF16, FP32 accumulation)
	qb::DevBuf kerr;                              // error word of the bounded MMA waits
	qb::DevBuf twm, tscr, uscr;                   // tensor-core DFTs: the 4 twiddle matrices, stage scratch
	const float *Bm1 = nullptr, *Bm2 = nullptr, *BmA = nullptr, *BmB = nullptr;

	// the twiddle matrices of the two-stage DFT and inverse (FP32 [Nn][K], from FP64)
	void build_twiddles(cudaStream_t s) {
		if (twm.p != nullptr) return;
		const int nk = 2 * m - 1;
		const long n1 = 2L * m * N, n2 = 2L * nk * 2 * N, nA = 2L * N * 2 * nk, nB = (long)N * 2 * m;
		std::vector<float> h(n1 + n2 + nA + nB);
		auto c = [&](long a) { return (float)std::cos(2.0 * M_PI * (double)a / N); };
		auto sn = [&](long a) { return (float)std::sin(2.0 * M_PI * (double)a / N); };
		float *b1 = h.data(), *b2 = b1 + n1, *bA = b2 + n2, *bB = bA + nA;
		for (int n = 0; n < m; n++)
			for (int kv = 0; kv < N; kv++) { b1[n * N + kv] = c((long)n * kv); b1[(m + n) * N + kv] = -sn((long)n * kv); }
		for (int kxi = 0; kxi < nk; kxi++) {
			const int kx = kxi - (m - 1);
			for (int l = 0; l < N; l++) {
				const long a = (long)kx * l;
				b2[kxi * 2L * N + l] = c(a);         b2[kxi * 2L * N + N + l] = sn(a);
				b2[(nk + kxi) * 2L * N + l] = -sn(a); b2[(nk + kxi) * 2L * N + N + l] = c(a);
				bA[l * 2L * nk + kxi] = c(a);        bA[l * 2L * nk + nk + kxi] = -sn(a);
				bA[(N + l) * 2L * nk + kxi] = sn(a); bA[(N + l) * 2L * nk + nk + kxi] = c(a);
			}
		}
		for (int kv = 0; kv < N; kv++)
			for (int ky = 0; ky < m; ky++) { bB[kv * 2L * m + ky] = c((long)ky * kv); bB[kv * 2L * m + m + ky] = -sn((long)ky * kv); }
		twm.ensure(sizeof(float) * h.size());
		QB_CUDA(cudaMemcpyAsync(twm.p, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice, s));
		QB_CUDA(cudaStreamSynchronize(s));
		Bm1 = twm.as<float>(); Bm2 = Bm1 + n1; BmA = Bm2 + n2; BmB = BmA + nA;
	}

	template <class Ld, class Ep, class Bb> void row_gemm(const char *name, const Ld &ld, const Ep &ep, const Bb &bm, long tiles, int K, int Nn,
	                                                      cudaStream_t s) {
		static int attr_done[64] = {};
		int dev = 0;
		QB_CUDA(cudaGetDevice(&dev));
		if (!attr_done[dev & 63]) {
			qb::ensure_tmem_coresidency();
			QB_CUDA(cudaFuncSetAttribute(k_fno_tc<Ld, Ep, Bb>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fnotc::kSmem));
			attr_done[dev & 63] = 1;
		}
		const unsigned grid = (unsigned)std::max<long>(1, std::min<long>(tiles, 148L * 3));
		launch(name, k_fno_tc<Ld, Ep, Bb>, grid, fnotc::kThreads, (size_t)fnotc::kSmem, s, ld, ep, bm, K, Nn, kerr.as<int>());
	}

	// H[fld] = scale DFT(f[fld]) for the B w fields
	void dft(int B, const float *f, float2 *Hout, float scale, cudaStream_t s) {
		if (!use_tc) {
			launch("fno_dft", k_fno_dft, (unsigned)(B * w), 256, dft_smem(), s, N, m, f, Hout, scale);
			return;
		}
		ensure_err(s);
		build_twiddles(s);
		const long nf = (long)B * w;
		row_gemm("fno_dft_tc", LdDft1{ f, N }, EpDft1{ tscr.as<float>(), N, m }, BMat{ Bm1, N, nf * N }, (nf * N + 127) / 128, N, 2 * m, s);
		row_gemm("fno_dft_tc", LdDft2{ tscr.as<float>(), N }, EpDft2{ Hout, m, scale }, BMat{ Bm2, 2 * N, nf * m }, (nf * m + 127) / 128,
		         2 * N, 2 * (2 * m - 1), s);
	}
	// out[fld] (=, +=) scale Re IDFT(O[fld])
	void idft(int B, const float2 *O, float *out, float scale, int accumulate, cudaStream_t s) {
		if (!use_tc) {
			launch("fno_idft", k_fno_idft, (unsigned)(B * w), 256, idft_smem(), s, N, m, O, out, scale, accumulate);
			return;
		}
		ensure_err(s);
		build_twiddles(s);
		const long nf = (long)B * w;
		row_gemm("fno_idft_tc", LdIdftA{ O, m }, EpIdftA{ uscr.as<float>(), N, m }, BMat{ BmA, 2 * (2 * m - 1), nf * m }, (nf * m + 127) / 128,
		         2 * (2 * m - 1), 2 * N, s);
		row_gemm("fno_idft_tc", LdIdftB{ uscr.as<float>(), m }, EpIdftB{ out, N, scale, accumulate }, BMat{ BmB, 2 * m, nf * N },
		         (nf * N + 127) / 128, 2 * m, N, s);
	}
	// mode mixing: out[b][c][k] = sum over the other channel of R (or conj R, backward) times in.
	// On the tensor cores a mode's B matrix is rebuilt per 128-cell tile, which
	// pays only when the batch fills the tiles (at 64 cells the FP32 kernel is faster)
	void mix(int B, const float2 *in, const float *Rr, const float *Ri, float2 *out, int conj, cudaStream_t s) {
		if (!use_tc || B < 128) {
			launch("fno_mix", k_fno_mix, grid_for((long)B * w * K), 256, 0, s, B, w, K, in, Rr, Ri, out, conj);
			return;
		}
		ensure_err(s);
		row_gemm("fno_mix_tc", LdMix{ in, w, K }, EpMix{ out, w, K }, BMix{ Rr, Ri, w, K, B, conj }, (long)K * ((B + 127) / 128), 2 * w,
		         2 * w, s);
	}
	void ensure_err(cudaStream_t s) {
		if (kerr.p == nullptr) {
			kerr.ensure(sizeof(int));
			QB_CUDA(cudaMemsetAsync(kerr.p, 0, sizeof(int), s));
		}
	}

	float *P_(long o) { return params.as<float>() + o; }

	// out = M in + bias (+ add), gelu when act (uout keeps the pre-activation)
	void pointwise(int B, int cin, int cout, const float *in, const float *M, const float *bias, const float *add, float *uout,
	               float *hout, int act, cudaStream_t s) {
		if (use_tc) pointwise_mma(B, cin, cout, 0, in, M, bias, add, uout, hout, act, s);
		else launch("fno_pointwise", k_fno_pointwise, grid_for((long)B * P), 256, 0, s, B, P, cin, cout, in, M, bias, add, uout, hout, act);
	}
	// out = M^T in (the backward of a pointwise map)
	void pointwise_t(int B, int cin, int cout, const float *in, const float *M, float *out, cudaStream_t s) {
		if (use_tc) pointwise_mma(B, cin, cout, 1, in, M, nullptr, nullptr, nullptr, out, 0, s);
		else launch("fno_pointwise_t", k_fno_pointwise_t, grid_for((long)B * P), 256, 0, s, B, P, cin, cout, in, M, out);
	}
	void pointwise_mma(int B, int cin, int cout, int trans, const float *in, const float *M, const float *bias, const float *add,
	                   float *uout, float *hout, int act, cudaStream_t s) {
		static int attr_done[64] = {};
		int dev = 0;
		QB_CUDA(cudaGetDevice(&dev));
		if (!attr_done[dev & 63]) {
			qb::ensure_tmem_coresidency();
			QB_CUDA(cudaFuncSetAttribute(k_fno_pointwise_mma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fnomma::kSmem));
			attr_done[dev & 63] = 1;
		}
		ensure_err(s);
		const long tiles = ((long)B * P + fnomma::kRows - 1) / fnomma::kRows;
		const unsigned grid = (unsigned)std::max<long>(1, std::min<long>(tiles, 148L * 7));
		launch("fno_pointwise_mma", k_fno_pointwise_mma, grid, fnomma::kThreads, (size_t)fnomma::kSmem, s, B, P, cin, cout, trans, in, M,
		       bias, add, uout, hout, act, kerr.as<int>());
	}
	float *G_(long o) { return grads.as<float>() + o; }

	void reserve(int B) {
		if (B <= cap) return;
		const long f = (long)B * w * P;
		x.ensure(sizeof(float) * B * (long)kFnoIn * P);
		y.ensure(sizeof(float) * B * 4L * P);
		dy.ensure(sizeof(float) * B * 4L * P);
		dh.ensure(sizeof(float) * f);
		tmp.ensure(sizeof(float) * f);
		h.resize(L + 1);
		u.resize(L);
		H.resize(L);
		for (int l = 0; l <= L; l++) h[l].ensure(sizeof(float) * f);
		for (int l = 0; l < L; l++) { u[l].ensure(sizeof(float) * f); H[l].ensure(sizeof(float2) * (long)B * w * K); }
		GO.ensure(sizeof(float2) * (long)B * w * K);
		GH.ensure(sizeof(float2) * (long)B * w * K);
		tscr.ensure(sizeof(float) * (long)B * w * m * 2 * N);
		uscr.ensure(sizeof(float) * (long)B * w * N * 2 * m);
		const long nchunk = ((long)B * P + kChunk - 1) / kChunk;
		partial.ensure(sizeof(float) * nchunk * kFnoMaxWidth * kFnoMaxWidth);
		lossp.ensure(sizeof(double) * 4096);
		cap = B;
	}

	size_t dft_smem() const { return sizeof(float) * P + sizeof(float2) * ((long)N * m + N); }
	size_t idft_smem() const { return sizeof(float2) * ((long)K + (long)N * m + N); }

	void forward(int B, const double *W, cudaStream_t s) {
		reserve(B);
		launch("fno_in", k_fno_in, grid_for((long)B * P), 256, 0, s, B, P, W, inscale, x.as<float>());
		pointwise(B, kFnoIn, w, x.as<float>(), P_(off.A), P_(off.a), nullptr, nullptr, h[0].as<float>(), 0, s);
		for (int l = 0; l < L; l++) {
			dft(B, h[l].as<float>(), H[l].as<float2>(), 1.0f, s);
			mix(B, H[l].as<float2>(), P_(off.Rr[l]), P_(off.Ri[l]), GO.as<float2>(), 0, s);
			idft(B, GO.as<float2>(), tmp.as<float>(), 1.0f / (float)P, 0, s);
			pointwise(B, w, w, h[l].as<float>(), P_(off.W[l]), P_(off.b[l]), tmp.as<float>(), u[l].as<float>(), h[l + 1].as<float>(),
			          l < L - 1 ? 1 : 0, s);
		}
		pointwise(B, w, 4, h[L].as<float>(), P_(off.Q), P_(off.q), nullptr, nullptr, y.as<float>(), 0, s);
		QB_CUDA(cudaGetLastError());
	}

	// gradient of the pointwise map `out = M in + bias`: dM = sum dout in^T, dbias = sum dout
	void pw_grads(int B, int cin, int cout, const float *in, const float *dout, long offM, long offb, cudaStream_t s) {
		const long n = (long)B * P;
		const int nchunk = (int)((n + kChunk - 1) / kChunk);
		launch("fno_outer", k_fno_outer, nchunk, 256, 0, s, B, P, cout, cin, dout, in, partial.as<float>());
		launch("fno_reduce", k_fno_reduce, (cout * cin + 255) / 256, 256, 0, s, nchunk, cout * cin, partial.as<float>(), G_(offM));
		launch("fno_outer", k_fno_outer, nchunk, 256, 0, s, B, P, cout, 1, dout, nullptr, partial.as<float>());
		launch("fno_reduce", k_fno_reduce, (cout + 255) / 256, 256, 0, s, nchunk, cout, partial.as<float>(), G_(offb));
	}

	double loss_backward(int B, const double *target, cudaStream_t s) {
		const long n4 = (long)B * 4 * P, nw = (long)B * w * P;
		const int lb = 512;
		launch("fno_loss", k_fno_loss, lb, 256, 0, s, B, P, y.as<float>(), target, scale[0], scale[1], scale[2], scale[3], dy.as<float>(), lossp.as<double>());
		// projection
		pw_grads(B, w, 4, h[L].as<float>(), dy.as<float>(), off.Q, off.q, s);
		pointwise_t(B, w, 4, dy.as<float>(), P_(off.Q), dh.as<float>(), s);
		for (int l = L - 1; l >= 0; l--) {
			if (l < L - 1) launch("fno_gelu_bwd", k_fno_gelu_bwd, grid_for(nw), 256, 0, s, nw, u[l].as<float>(), dh.as<float>());
			// dh now holds du
			pw_grads(B, w, w, h[l].as<float>(), dh.as<float>(), off.W[l], off.b[l], s);
			dft(B, dh.as<float>(), GO.as<float2>(), 1.0f / (float)P, s);
			launch("fno_rgrad", k_fno_rgrad, grid_for((long)w * w * K), 256, 0, s, B, w, K, GO.as<float2>(), H[l].as<float2>(), G_(off.Rr[l]), G_(off.Ri[l]));
			mix(B, GO.as<float2>(), P_(off.Rr[l]), P_(off.Ri[l]), GH.as<float2>(), 1, s);
			pointwise_t(B, w, w, dh.as<float>(), P_(off.W[l]), tmp.as<float>(), s);
			idft(B, GH.as<float2>(), tmp.as<float>(), 1.0f, 1, s);
			std::swap(dh, tmp);
		}
		// lift
		pw_grads(B, kFnoIn, w, x.as<float>(), dh.as<float>(), off.A, off.a, s);
		QB_CUDA(cudaGetLastError());
		std::vector<double> lp(lb);
		QB_CUDA(cudaMemcpyAsync(lp.data(), lossp.p, sizeof(double) * lb, cudaMemcpyDeviceToHost, s));
		QB_CUDA(cudaStreamSynchronize(s));
		double l2 = 0;
		for (double v : lp) l2 += v;
		return l2 / (double)n4;
	}
};

namespace {
// splitmix64 normal variates for the initial weights
struct Rng {
	unsigned long long s;
	unsigned long long next() {
		unsigned long long z = (s += 0x9E3779B97F4A7C15ULL);
		z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
		z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
		return z ^ (z >> 31);
	}
	double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
	double normal() { return std::sqrt(-2.0 * std::log(uniform())) * std::cos(6.283185307179586 * uniform()); }
};

template <class F> int fno_guard(F &&f) {
	try {
		f();
		return 0;
	} catch (const std::exception &) {
		return -1;
	}
}
}  // namespace

extern "C" {

qb_fno *qb_fno_create(int N, int width, int modes, int layers, unsigned long long seed) {
	qb_fno *net = nullptr;
	fno_guard([&] {
		if (N < 4 || N > 64 || (N & 1)) QB_FAIL("qb_fno_create: N must be even, 4..64");
		if (width < 1 || width > kFnoMaxWidth) QB_FAIL("qb_fno_create: width must be 1..64");
		if (modes < 1 || 2 * modes - 1 > N) QB_FAIL("qb_fno_create: need 1 <= modes and 2 modes - 1 <= N");
		if (layers < 1 || layers > 16) QB_FAIL("qb_fno_create: layers must be 1..16");
		auto n = std::make_unique<qb_fno>();
		n->N = N; n->w = width; n->m = modes; n->L = layers; n->K = (2 * modes - 1) * modes; n->P = N * N;
		n->off = offsets(width, n->K, layers);
		const long np = n->off.total;
		std::vector<float> p(np, 0.0f);
		Rng r{ seed };
		auto fill = [&](long o, long cnt, double sd) { for (long i = 0; i < cnt; i++) p[o + i] = (float)(sd * r.normal()); };
		fill(n->off.A, (long)kFnoIn * width, std::sqrt(1.0 / kFnoIn));
		for (int l = 0; l < layers; l++) {
			fill(n->off.Rr[l], (long)width * width * n->K, 1.0 / width);
			fill(n->off.Ri[l], (long)width * width * n->K, 1.0 / width);
			fill(n->off.W[l], (long)width * width, std::sqrt(1.0 / width));
		}
		fill(n->off.Q, 4L * width, std::sqrt(1.0 / width));
		n->params.ensure(sizeof(float) * np);
		n->grads.ensure(sizeof(float) * np);
		n->am.ensure(sizeof(float) * np);
		n->av.ensure(sizeof(float) * np);
		QB_CUDA(cudaMemcpy(n->params.p, p.data(), sizeof(float) * np, cudaMemcpyHostToDevice));
		QB_CUDA(cudaMemset(n->am.p, 0, sizeof(float) * np));
		QB_CUDA(cudaMemset(n->av.p, 0, sizeof(float) * np));
		QB_CUDA(cudaMemset(n->grads.p, 0, sizeof(float) * np));
		net = n.release();
	});
	return net;
}

void qb_fno_free(qb_fno *net) { delete net; }

long qb_fno_num_params(const qb_fno *net) { return net ? net->off.total : -1; }

int qb_fno_grid_size(const qb_fno *net) { return net ? net->N : -1; }

int qb_fno_get_params(const qb_fno *net, float *host) {
	return fno_guard([&] {
		if (net == nullptr || host == nullptr) QB_FAIL("qb_fno_get_params: null network or buffer");
		QB_CUDA(cudaMemcpy(host, net->params.p, sizeof(float) * net->off.total, cudaMemcpyDeviceToHost));
	});
}

int qb_fno_set_params(qb_fno *net, const float *host) {
	return fno_guard([&] {
		if (net == nullptr || host == nullptr) QB_FAIL("qb_fno_set_params: null network or buffer");
		QB_CUDA(cudaMemcpy(net->params.p, host, sizeof(float) * net->off.total, cudaMemcpyHostToDevice));
	});
}

int qb_fno_set_scale(qb_fno *net, const double *scale) {
	return fno_guard([&] {
		if (net == nullptr || scale == nullptr) QB_FAIL("qb_fno_set_scale: null network or scales");
		for (int c = 0; c < 4; c++) {
			if (!(scale[c] > 0)) QB_FAIL("qb_fno_set_scale: scales must be positive");
			net->scale[c] = scale[c];
		}
	});
}

int qb_fno_set_input_scale(qb_fno *net, const double *scale) {
	return fno_guard([&] {
		if (net == nullptr || scale == nullptr) QB_FAIL("qb_fno_set_input_scale: null network or scales");
		for (int f = 0; f < kFnoIn; f++) {
			if (!(scale[f] > 0)) QB_FAIL("qb_fno_set_input_scale: scales must be positive");
			net->inscale.s[f] = scale[f];
		}
	});
}

int qb_fno_set_tensor_cores(qb_fno *net, int on) {
	return fno_guard([&] {
		if (net == nullptr) QB_FAIL("qb_fno_set_tensor_cores: null network");
		net->use_tc = on ? 1 : 0;
	});
}

int qb_fno_device_errors(const qb_fno *net) {
	int h = 0;
	if (net == nullptr || net->kerr.p == nullptr) return 0;
	if (cudaMemcpy(&h, net->kerr.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
	return h;
}

int qb_fno_forward(qb_fno *net, int batch, const double *W, double *C, void *stream) {
	return fno_guard([&] {
		if (batch <= 0) return;
		if (net == nullptr || W == nullptr || C == nullptr) QB_FAIL("qb_fno_forward: null network or state");
		cudaStream_t s = (cudaStream_t)stream;
		net->forward(batch, W, s);
		const long n4 = (long)batch * 4 * net->P;
		launch("fno_out", k_fno_out, grid_for(n4), 256, 0, s, n4, net->P, net->y.as<float>(), net->scale[0], net->scale[1], net->scale[2], net->scale[3], C);
		QB_CUDA(cudaGetLastError());
	});
}

int qb_fno_gradients(qb_fno *net, int batch, const double *W, const double *target, float *grad_host, double *loss, void *stream) {
	return fno_guard([&] {
		if (batch <= 0) QB_FAIL("qb_fno_gradients: empty batch");
		if (net == nullptr || W == nullptr || target == nullptr) QB_FAIL("qb_fno_gradients: null network, state or target");
		cudaStream_t s = (cudaStream_t)stream;
		net->forward(batch, W, s);
		const double l = net->loss_backward(batch, target, s);
		if (loss) *loss = l;
		if (grad_host) {
			QB_CUDA(cudaMemcpyAsync(grad_host, net->grads.p, sizeof(float) * net->off.total, cudaMemcpyDeviceToHost, s));
			QB_CUDA(cudaStreamSynchronize(s));
		}
	});
}

int qb_fno_train_step(qb_fno *net, int batch, const double *W, const double *target, float lr, double *loss, void *stream) {
	return fno_guard([&] {
		if (batch <= 0) QB_FAIL("qb_fno_train_step: empty batch");
		if (net == nullptr || W == nullptr || target == nullptr) QB_FAIL("qb_fno_train_step: null network, state or target");
		cudaStream_t s = (cudaStream_t)stream;
		net->forward(batch, W, s);
		const double l = net->loss_backward(batch, target, s);
		if (loss) *loss = l;
		net->adam_t++;
		const float b1 = 0.9f, b2 = 0.999f;
		const float c1 = 1.0f - std::pow(b1, (float)net->adam_t), c2 = 1.0f - std::pow(b2, (float)net->adam_t);
		launch("fno_adam", k_fno_adam, grid_for(net->off.total), 256, 0, s, net->off.total, net->params.as<float>(), net->grads.as<float>(), net->am.as<float>(),
		                                                    net->av.as<float>(), lr, b1, b2, 1e-8f, c1, c2);
		QB_CUDA(cudaGetLastError());
	});
}

}  // extern "C"
