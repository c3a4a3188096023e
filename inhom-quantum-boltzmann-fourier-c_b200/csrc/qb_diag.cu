// qb_diag.cu — per-cell physics diagnostics of velocity-space Wigner states.
//
// Restates the upstream Matlab post-processing on the GPU
// (visualization/wignerMoments.m:15-37, visualization/entropy.m):
//   w_c     = sum_v W_c(v) dv^2                    (c = tr, x, y, z; dv = 2L/N)
//   u       = sum_v v W_tr(v) / sum_v W_tr(v)       (mean velocity, 2-vector)
//   e       = sum_v 1/2 |v - u|^2 W_tr(v) / sum_v W_tr(v)
//   lam_min = min_v (w_tr - |w_vec|),  lam_max = max_v (w_tr + |w_vec|)   (eigenvalues of W(v))
//   S       = sum_v sum_{lam in eig W(v), 0<lam<1} -(lam log lam + (1-lam) log(1-lam)) dv^2
// One CTA per cell; every sum is a fixed-order tree reduction in FP64, so
// results are deterministic.
#include "qb_engine.h"

extern "C" {
#include "qbgpu.h"
}

namespace {

constexpr int kThreads = 256;
constexpr int kOut = 10;   // w_tr, w_x, w_y, w_z, u_x, u_y, e, lam_min, lam_max, S

__device__ __forceinline__ double fd_entropy(double p) {
	return (p > 0.0 && p < 1.0) ? -(p * log(p) + (1.0 - p) * log1p(-p)) : 0.0;
}

template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double *sh) {
	// sh: kThreads * K doubles; result in v on thread 0
	for (int k = 0; k < K; k++) sh[k * kThreads + threadIdx.x] = v[k];
	__syncthreads();
	for (int s = kThreads / 2; s > 0; s >>= 1) {
		if (threadIdx.x < s)
			for (int k = 0; k < K; k++) sh[k * kThreads + threadIdx.x] += sh[k * kThreads + threadIdx.x + s];
		__syncthreads();
	}
	for (int k = 0; k < K; k++) v[k] = sh[k * kThreads];
	__syncthreads();
}

__global__ void __launch_bounds__(kThreads) k_diagnostics(int N, double L, const double *__restrict__ W, double *__restrict__ out) {
	__shared__ double sh[8 * kThreads];
	__shared__ double mn[kThreads], mx[kThreads];
	const long NN = (long)N * N;
	const double *w = W + blockIdx.x * 4 * NN;
	const double dv = 2.0 * L / N;
	double a[7] = { 0, 0, 0, 0, 0, 0, 0 };     // sums: tr, x, y, z, vx*tr, vy*tr, entropy
	double lo = 1e300, hi = -1e300;
	for (long q = threadIdx.x; q < NN; q += kThreads) {
		const int l = (int)(q / N), k = (int)(q % N);
		const double vx = (l < N / 2 ? l : l - N) * dv, vy = (k < N / 2 ? k : k - N) * dv;   // l: v_x (slow index)
		const double t = w[q], x = w[NN + q], y = w[2 * NN + q], z = w[3 * NN + q];
		const double r = sqrt(x * x + y * y + z * z);
		a[0] += t; a[1] += x; a[2] += y; a[3] += z;
		a[4] += vx * t; a[5] += vy * t;
		a[6] += fd_entropy(t - r) + fd_entropy(t + r);
		lo = fmin(lo, t - r);
		hi = fmax(hi, t + r);
	}
	block_sum<7>(a, sh);
	const double ux = a[4] / a[0], uy = a[5] / a[0];
	double e[1] = { 0 };
	for (long q = threadIdx.x; q < NN; q += kThreads) {
		const int l = (int)(q / N), k = (int)(q % N);
		const double vx = (l < N / 2 ? l : l - N) * dv - ux, vy = (k < N / 2 ? k : k - N) * dv - uy;
		e[0] += 0.5 * (vx * vx + vy * vy) * w[q];
	}
	block_sum<1>(e, sh);
	mn[threadIdx.x] = lo;
	mx[threadIdx.x] = hi;
	__syncthreads();
	for (int s = kThreads / 2; s > 0; s >>= 1) {
		if (threadIdx.x < s) {
			mn[threadIdx.x] = fmin(mn[threadIdx.x], mn[threadIdx.x + s]);
			mx[threadIdx.x] = fmax(mx[threadIdx.x], mx[threadIdx.x + s]);
		}
		__syncthreads();
	}
	if (threadIdx.x == 0) {
		double *o = out + blockIdx.x * kOut;
		const double d2 = dv * dv;
		o[0] = a[0] * d2; o[1] = a[1] * d2; o[2] = a[2] * d2; o[3] = a[3] * d2;
		o[4] = ux; o[5] = uy;
		o[6] = e[0] / a[0];
		o[7] = mn[0]; o[8] = mx[0];
		o[9] = a[6] * d2;
	}
}

}  // namespace

extern "C" int qb_diagnostics(int N, double L, int ncells, const double *W, double *out, void *stream) {
	try {
		if (ncells <= 0) return 0;
		if (N < 2 || (N & 1)) QB_FAIL("qb_diagnostics: N must be even and at least 2");
		qb::ProfScope ps("diagnostics", (cudaStream_t)stream);
		k_diagnostics<<<ncells, kThreads, 0, (cudaStream_t)stream>>>(N, L, W, out);
		QB_CUDA(cudaGetLastError());
		return 0;
	} catch (const std::exception &) {
		return -1;
	}
}
