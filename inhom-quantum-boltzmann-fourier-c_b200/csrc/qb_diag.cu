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

#include <cmath>
#include <cstring>
#include <vector>

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

// ---------------------------------------------------------------------------
// Fermi-Dirac equilibrium of a state's conserved moments and the quantum
// relative entropy to it (upstream visualization/asymptoticFD.m,
// calculateFDparams.m, createFD.m, relentropy.m and the loops of
// visualization/visualizeHomBoltzmann.m:116-148).
namespace {

constexpr int kFDPar = 9;     // beta, mu_1, mu_2, u_x, u_y, n_x, n_y, n_z, residual
constexpr double kPi = 3.14159265358979323846;

// dilogarithm Li_2(x) for x <= 1: power series on [0, 1/2], Euler's reflection
// Li2(x) = pi^2/6 - log(x) log(1-x) - Li2(1-x) on (1/2, 1], Landen's identity
// Li2(x) = -Li2(x/(x-1)) - log(1-x)^2 / 2 on [-1, 0) and the inversion
// Li2(x) = -pi^2/6 - log(-x)^2 / 2 - Li2(1/x) below -1.
double li2_series(double y) {          // 0 <= y <= 1/2
	double s = 0.0, p = y;
	for (int k = 1; k < 80; k++) {
		const double t = p / ((double)k * k);
		s += t;
		if (t < 1e-18 * s) break;
		p *= y;
	}
	return s;
}

double li2(double x) {
	const double pi2_6 = kPi * kPi / 6.0;
	if (x == 0.0) return 0.0;
	if (x == 1.0) return pi2_6;
	if (x > 0.0 && x <= 0.5) return li2_series(x);
	if (x > 0.5 && x < 1.0) return pi2_6 - std::log(x) * std::log1p(-x) - li2_series(1.0 - x);
	if (x >= -1.0 && x < 0.0) {
		const double l = std::log1p(-x);
		return -li2(x / (x - 1.0)) - 0.5 * l * l;
	}
	const double l = std::log(-x);      // x < -1
	return -pi2_6 - 0.5 * l * l - li2(1.0 / x);
}

// density and energy of the 2-D Fermi-Dirac distribution with fugacity z
// and inverse temperature b (calculateFDparams.m densityFD / energyFD)
double fd_rho(double z, double b) { return 2.0 * kPi / b * std::log1p(z); }
double fd_en(double z, double b) { return -2.0 * kPi / (b * b) * li2(-z); }

// moment mismatch F(z_up, z_dn, beta) and its Jacobian (calculateFDparams.m mdiff)
void fd_residual(const double x[3], const double lam[2], double en_t, double F[3], double Jm[3][3]) {
	const double zu = x[0], zd = x[1], b = x[2];
	const double ru = fd_rho(zu, b), rd = fd_rho(zd, b), eu = fd_en(zu, b), ed = fd_en(zd, b);
	F[0] = ru - lam[0];
	F[1] = rd - lam[1];
	F[2] = eu + ed - en_t;
	Jm[0][0] = 2.0 * kPi / (b * (1.0 + zu)); Jm[0][1] = 0.0; Jm[0][2] = -ru / b;
	Jm[1][0] = 0.0; Jm[1][1] = 2.0 * kPi / (b * (1.0 + zd)); Jm[1][2] = -rd / b;
	Jm[2][0] = ru / (b * zu); Jm[2][1] = rd / (b * zd); Jm[2][2] = -2.0 * eu / b - 2.0 * ed / b;
}

bool solve3(double A[3][3], double r[3], double out[3]) {
	double M[3][4];
	for (int i = 0; i < 3; i++) { for (int j = 0; j < 3; j++) M[i][j] = A[i][j]; M[i][3] = r[i]; }
	for (int c = 0; c < 3; c++) {
		int p = c;
		for (int i = c + 1; i < 3; i++) if (std::fabs(M[i][c]) > std::fabs(M[p][c])) p = i;
		if (!(std::fabs(M[p][c]) > 0.0)) return false;
		for (int k = 0; k < 4; k++) std::swap(M[c][k], M[p][k]);
		for (int i = c + 1; i < 3; i++) {
			const double f = M[i][c] / M[c][c];
			for (int k = c; k < 4; k++) M[i][k] -= f * M[c][k];
		}
	}
	for (int i = 2; i >= 0; i--) {
		double s = M[i][3];
		for (int k = i + 1; k < 3; k++) s -= M[i][k] * out[k];
		out[i] = s / M[i][i];
	}
	return true;
}

double norm3(const double F[3]) { return std::sqrt(F[0] * F[0] + F[1] * F[1] + F[2] * F[2]); }

// Newton's method with backtracking on |F| (positivity kept by the step
// halving) from (1, 1, beta0); calculateFDparams.m minimises |F|^2 by
// lsqnonlin from the same starts, which reaches the same root when one exists.
double fd_solve(const double lam[2], double en_t, double beta0, double x[3]) {
	x[0] = 1.0; x[1] = 1.0; x[2] = beta0;
	double F[3], Jm[3][3];
	fd_residual(x, lam, en_t, F, Jm);
	double nf = norm3(F);
	for (int it = 0; it < 200 && nf > 0.0; it++) {
		double d[3], mF[3] = { -F[0], -F[1], -F[2] };
		if (!solve3(Jm, mF, d)) break;
		double t = 1.0, xn[3], Fn[3], Jn[3][3], nn = nf;
		bool moved = false;
		for (int ls = 0; ls < 60; ls++, t *= 0.5) {
			for (int k = 0; k < 3; k++) xn[k] = x[k] + t * d[k];
			if (!(xn[0] > 0.0 && xn[1] > 0.0 && xn[2] > 0.0)) continue;
			fd_residual(xn, lam, en_t, Fn, Jn);
			nn = norm3(Fn);
			if (std::isfinite(nn) && nn < nf) { moved = true; break; }
		}
		if (!moved) break;
		for (int k = 0; k < 3; k++) x[k] = xn[k];
		for (int k = 0; k < 3; k++) { F[k] = Fn[k]; for (int j = 0; j < 3; j++) Jm[k][j] = Jn[k][j]; }
		const double step = std::fabs(t * d[0]) / x[0] + std::fabs(t * d[1]) / x[1] + std::fabs(t * d[2]) / x[2];
		nf = nn;
		if (step < 1e-16) break;
	}
	return nf;
}

// WFD(v) = U diag(f_1, f_2) U^H in the Pauli basis: w0 = (f1 + f2)/2,
// w = (f2 - f1)/2 n, f_i = 1/(exp(beta (|v - u|^2/2 - mu_i)) + 1)   (createFD.m)
__global__ void k_create_fd(int N, double L, const double *__restrict__ par, double *__restrict__ WFD) {
	const long NN = (long)N * N;
	const double *p = par + blockIdx.x * kFDPar;
	double *w = WFD + blockIdx.x * 4 * NN;
	const double dv = 2.0 * L / N;
	for (long q = threadIdx.x; q < NN; q += blockDim.x) {
		const int l = (int)(q / N), k = (int)(q % N);
		const double vx = (l < N / 2 ? l : l - N) * dv - p[3], vy = (k < N / 2 ? k : k - N) * dv - p[4];
		const double e = 0.5 * (vx * vx + vy * vy);
		const double f1 = 1.0 / (exp(p[0] * (e - p[1])) + 1.0), f2 = 1.0 / (exp(p[0] * (e - p[2])) + 1.0);
		w[q] = 0.5 * (f1 + f2);
		const double h = 0.5 * (f2 - f1);
		w[NN + q] = h * p[5];
		w[2 * NN + q] = h * p[6];
		w[3 * NN + q] = h * p[7];
	}
}

// eigen-decomposition of the 2x2 Hermitian w0 I + w.sigma: eigenvalues
// w0 -+ |w|, clamped to [eps, 1 - eps] as relentropy.m does; f(rho) for a
// function f of the clamped eigenvalues is a I + b n.sigma
struct Pauli2 { double lo, hi; double n[3]; bool iso; };

__device__ __forceinline__ Pauli2 pauli_eig(double w0, double x, double y, double z) {
	const double eps = 2.220446049250313e-16;
	Pauli2 r;
	const double m = sqrt(x * x + y * y + z * z);
	r.iso = !(m > 0.0);
	r.n[0] = r.iso ? 0.0 : x / m; r.n[1] = r.iso ? 0.0 : y / m; r.n[2] = r.iso ? 0.0 : z / m;
	double lo = w0 - m, hi = w0 + m;
	lo = lo <= 0.0 ? eps : (lo >= 1.0 ? 1.0 - eps : lo);
	hi = hi <= 0.0 ? eps : (hi >= 1.0 ? 1.0 - eps : hi);
	r.lo = lo; r.hi = hi;
	return r;
}

// tr(A B) for A = a0 I + a.sigma, B = b0 I + b.sigma is 2 (a0 b0 + a.b)
__device__ __forceinline__ double rel_entropy_point(const Pauli2 &r, const Pauli2 &t) {
	const double a0 = 0.5 * (r.hi + r.lo), a1 = 0.5 * (r.hi - r.lo);                 // rho (clamped)
	const double c0 = 0.5 * (log(t.hi) + log(t.lo)), c1 = 0.5 * (log(t.hi) - log(t.lo));   // log tau
	const double d0 = 0.5 * (log1p(-t.hi) + log1p(-t.lo)), d1 = 0.5 * (log1p(-t.hi) - log1p(-t.lo));   // log(1 - tau)
	const double nn = r.n[0] * t.n[0] + r.n[1] * t.n[1] + r.n[2] * t.n[2];
	const double s_rr = r.lo * log(r.lo) + r.hi * log(r.hi);                            // tr(rho log rho)
	const double s_r1 = (1.0 - r.lo) * log1p(-r.lo) + (1.0 - r.hi) * log1p(-r.hi);      // tr((1-rho) log(1-rho))
	const double x_rt = 2.0 * (a0 * c0 + a1 * c1 * nn);                                 // tr(rho log tau)
	const double x_1t = 2.0 * ((1.0 - a0) * d0 - a1 * d1 * nn);                         // tr((1-rho) log(1-tau))
	return (s_rr - x_rt) + (s_r1 - x_1t);
}

__global__ void __launch_bounds__(kThreads) k_relative_entropy(int N, double L, const double *__restrict__ W, const double *__restrict__ WFD,
                                                               double *__restrict__ out) {
	__shared__ double sh[kThreads];
	__shared__ double col[4][64];
	const long NN = (long)N * N;
	const double *w = W + blockIdx.x * 4 * NN, *f = WFD + blockIdx.x * 4 * NN;
	const double dv2 = (2.0 * L / N) * (2.0 * L / N);
	double kl[1] = { 0.0 };
	for (long q = threadIdx.x; q < NN; q += kThreads) {
		if (!(f[q] > 1e-6)) continue;
		const Pauli2 r = pauli_eig(w[q], w[NN + q], w[2 * NN + q], w[3 * NN + q]);
		const Pauli2 t = pauli_eig(f[q], f[NN + q], f[2 * NN + q], f[3 * NN + q]);
		kl[0] += rel_entropy_point(r, t);
	}
	block_sum<1>(kl, sh);
	// Matlab norm(A, 1): largest column sum, a column being a fixed v_x index l
	for (int t = threadIdx.x; t < 4 * N; t += kThreads) {
		const int j = t / N, l = t % N;
		double s = 0.0;
		for (int k = 0; k < N; k++) s += fabs(w[j * NN + (long)l * N + k] - f[j * NN + (long)l * N + k]);
		col[j][l] = s;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		double dist = 0.0;
		for (int j = 0; j < 4; j++) {
			double m = 0.0;
			for (int l = 0; l < N; l++) m = fmax(m, col[j][l]);
			dist += m;
		}
		out[blockIdx.x * 2] = kl[0] * dv2;
		out[blockIdx.x * 2 + 1] = dist * dv2;
	}
}

}  // namespace

extern "C" int qb_fermi_dirac_equilibrium(int N, double L, int ncells, const double *W, double *WFD, double *params, void *stream) {
	try {
		if (ncells <= 0) return 0;
		if (N < 2 || (N & 1) || N > 64) QB_FAIL("qb_fermi_dirac_equilibrium: N must be even, 2..64");
		cudaStream_t s = (cudaStream_t)stream;
		double *dd = nullptr, *dp = nullptr;
		QB_CUDA(cudaMallocAsync((void **)&dd, sizeof(double) * kOut * ncells, s));
		QB_CUDA(cudaMallocAsync((void **)&dp, sizeof(double) * kFDPar * ncells, s));
		{
			qb::ProfScope ps("diagnostics", s);
			k_diagnostics<<<ncells, kThreads, 0, s>>>(N, L, W, dd);
			QB_CUDA(cudaGetLastError());
		}
		std::vector<double> d((size_t)kOut * ncells), par((size_t)kFDPar * ncells);
		QB_CUDA(cudaMemcpyAsync(d.data(), dd, sizeof(double) * d.size(), cudaMemcpyDeviceToHost, s));
		QB_CUDA(cudaStreamSynchronize(s));
		for (int c = 0; c < ncells; c++) {
			const double *m = &d[(size_t)c * kOut];
			double *p = &par[(size_t)c * kFDPar];
			const double r = std::sqrt(m[1] * m[1] + m[2] * m[2] + m[3] * m[3]);
			const double lam[2] = { m[0] - r, m[0] + r };       // eigenvalues of the spin density matrix, ascending
			const double en_t = m[6] * (lam[0] + lam[1]);
			double x[3], x2[3];
			double md = fd_solve(lam, en_t, 1.0, x);
			if (!(md <= 1e-4)) {
				const double md2 = fd_solve(lam, en_t, 0.5, x2);
				if (md2 < md || !std::isfinite(md)) { md = md2; for (int k = 0; k < 3; k++) x[k] = x2[k]; }
			}
			p[0] = x[2];
			p[1] = std::log(x[0]) / x[2];
			p[2] = std::log(x[1]) / x[2];
			p[3] = m[4]; p[4] = m[5];
			if (r > 0.0) { p[5] = m[1] / r; p[6] = m[2] / r; p[7] = m[3] / r; }
			else { p[5] = 0.0; p[6] = 0.0; p[7] = -1.0; }
			p[8] = md;
		}
		QB_CUDA(cudaMemcpyAsync(dp, par.data(), sizeof(double) * par.size(), cudaMemcpyHostToDevice, s));
		{
			qb::ProfScope ps("diagnostics", s);
			k_create_fd<<<ncells, kThreads, 0, s>>>(N, L, dp, WFD);
			QB_CUDA(cudaGetLastError());
		}
		QB_CUDA(cudaFreeAsync(dd, s));
		QB_CUDA(cudaFreeAsync(dp, s));
		if (params) std::memcpy(params, par.data(), sizeof(double) * par.size());
		QB_CUDA(cudaStreamSynchronize(s));
		return 0;
	} catch (const std::exception &) {
		return -1;
	}
}

extern "C" int qb_relative_entropy(int N, double L, int ncells, const double *W, const double *WFD, double *out, void *stream) {
	try {
		if (ncells <= 0) return 0;
		if (N < 2 || (N & 1) || N > 64) QB_FAIL("qb_relative_entropy: N must be even, 2..64");
		qb::ProfScope ps("diagnostics", (cudaStream_t)stream);
		k_relative_entropy<<<ncells, kThreads, 0, (cudaStream_t)stream>>>(N, L, W, WFD, out);
		QB_CUDA(cudaGetLastError());
		return 0;
	} catch (const std::exception &) {
		return -1;
	}
}
