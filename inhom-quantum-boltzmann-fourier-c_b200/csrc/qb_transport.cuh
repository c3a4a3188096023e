// qb_transport.cuh — minmod slope-limiter transport along x (sm_100a).
//
// One thread per (cell, Pauli component, velocity point): consecutive threads
// own consecutive velocity points of one cell, so every load and store of a
// state array is coalesced; the 5-point stencil along x reads neighbouring
// cells (L2-resident).  The arithmetic follows upstream
// src/finite_volume.c:35-179 operation by operation with explicitly rounded
// double operations (__dadd_rn etc. are never contracted into FMAs), so the
// result is bit-identical to upstream's IEEE double evaluation.
#pragma once
#include <cuda_runtime.h>

namespace qb {

__device__ __forceinline__ double add_(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul_(double a, double b) { return __dmul_rn(a, b); }

// minmod, upstream finite_volume.c:35-38: 0.5*(sgn a + sgn b)*min(|a|,|b|)
__device__ __forceinline__ double minmod_(double a, double b) {
	const double fa = fabs(a), fb = fabs(b);
	const double m = (fa <= fb) ? fa : fb;
	return mul_(mul_(0.5, add_(copysign(1.0, a), copysign(1.0, b))), m);
}

// per-line coefficients (finite_volume.c:56-64)
struct LineCoef { double A, Aabs, S, Sabs, scale; };

__device__ __forceinline__ LineCoef line_coef(double h, double dt, double A) {
	LineCoef c;
	c.A = A;
	c.Aabs = fabs(A);
	const double nu = __ddiv_rn(mul_(dt, A), h);
	const double d = sub_(copysign(1.0, nu), nu);
	c.S = mul_(mul_(0.5, A), d);
	c.Sabs = mul_(mul_(0.5, c.Aabs), d);
	c.scale = __ddiv_rn(dt, mul_(2.0, h));
	return c;
}

// Un + scale*( -A(U+ - U-) + |A|(U+ - 2U + U-) - S(hb+ - hb-) + |S|(hb+ - 2hb + hb-) )
__device__ __forceinline__ double slope_update(const LineCoef &c, double um, double u, double up, double hm, double h0, double hp) {
	double s = mul_(-c.A, sub_(up, um));
	s = add_(s, mul_(c.Aabs, add_(sub_(up, mul_(2.0, u)), um)));
	s = sub_(s, mul_(c.S, sub_(hp, hm)));
	s = add_(s, mul_(c.Sabs, add_(sub_(hp, mul_(2.0, h0)), hm)));
	return add_(u, mul_(c.scale, s));
}

struct TransportParams {
	int ncells, npts;                   // cells along x, points per cell
	const double *in; double *out;      // [cell][npts]
	const double *A;                    // transport velocity of every point (npts)
	double h, dt;                       // dt is the (half) step passed to the limiter
	int bc;                             // 0 periodic, 1 Dirichlet
};

// K10: one limiter step for every x-line (upstream finite_volume.c:52-179;
// in the Strang step simulation.c:426-448 periodic, :678-700 Dirichlet)
__global__ void __launch_bounds__(256) k_transport(const TransportParams p) {
	const long cs = p.npts;
	const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= cs * p.ncells) return;
	const int i = (int)(idx / cs);
	const long off = idx % cs;
	const int n = p.ncells;
	const LineCoef c = line_coef(p.h, p.dt, p.A[off]);
	const double *U = p.in + off;
	if (p.bc == 0) {
		auto u = [&](int j) { j %= n; if (j < 0) j += n; return U[(long)j * cs]; };
		// alpha_j = U_{j+1} - U_j (periodic), hb_j = minmod(alpha_j, alpha_{j-1})
		const double um2 = u(i - 2), um1 = u(i - 1), u0 = u(i), up1 = u(i + 1), up2 = u(i + 2);
		const double a_m2 = sub_(um1, um2), a_m1 = sub_(u0, um1), a_0 = sub_(up1, u0), a_p1 = sub_(up2, up1);
		const double hbm = minmod_(a_m1, a_m2), hb0 = minmod_(a_0, a_m1), hbp = minmod_(a_p1, a_0);
		p.out[idx] = slope_update(c, um1, u0, up1, hbm, hb0, hbp);
	} else {
		// Dirichlet (finite_volume.c:118-179): alpha_{n-1} = 0, hb_0 = hb_{n-1} = 0
		auto u = [&](int j) { return U[(long)j * cs]; };
		auto alpha = [&](int j) { return (j >= n - 1) ? 0.0 : sub_(u(j + 1), u(j)); };
		auto hb = [&](int j) { return (j <= 0 || j >= n - 1) ? 0.0 : minmod_(alpha(j), alpha(j - 1)); };
		double r;
		if (i > 0 && i < n - 1) {
			r = slope_update(c, u(i - 1), u(i), u(i + 1), hb(i - 1), hb(i), hb(i + 1));
		} else if (c.A >= 0) {
			if (i == 0) r = u(0);
			else r = add_(u(n - 1), mul_(mul_(2.0, c.scale), sub_(mul_(-c.A, sub_(u(n - 1), u(n - 2))), mul_(c.S, sub_(hb(n - 1), hb(n - 2))))));
		} else {
			if (i == n - 1) r = u(n - 1);
			else r = add_(u(0), mul_(mul_(2.0, c.scale), sub_(mul_(-c.A, sub_(u(1), u(0))), mul_(c.S, sub_(hb(1), hb(0))))));
		}
		p.out[idx] = r;
	}
}

// ---------------------------------------------------------------------------
// Maxwell boundaries (upstream finite_volume.c:186-323, simulation.c:837-1165).
//
// With remapN = N the m = N*N points of a cell are the upstream "Maxwell
// velocity grid" of a component: Maxwell index mm reads standard index
// src(mm) = mm + N for mm < m/2 (the v_x = 0 row is skipped, the -L row is
// reused as +L), else mm.  With remapN = 0 the points are used as given
// (SlopeLimiterStepMaxwell on caller data).
__device__ __forceinline__ int mx_src(int remapN, int m, int mm) { return (remapN && mm < m / 2) ? mm + remapN : mm; }

// Sequential flux sums in upstream order (CalculateRightwardFlux /
// CalculateLeftwardFlux, finite_volume.c:186-216), one thread:
//   out[0] = sum_{mm<m/2} A U ;  out[1] = sum_{mm>=m/2} |A| U   of grid U (remapped)
__global__ void k_flux_pair(int m, int remapN, const double *__restrict__ A, const double *__restrict__ U, double *out) {
	if (threadIdx.x != 0 || blockIdx.x != 0) return;
	double r = 0, l = 0;
	for (int i = 0; i < m / 2; i++) r = add_(r, mul_(A[i], U[mx_src(remapN, m, i)]));
	for (int i = m / 2; i < m; i++) l = add_(l, mul_(fabs(A[i]), U[mx_src(remapN, m, i)]));
	out[0] = r;
	out[1] = l;
}

// boundary data of InhomStepMaxwell (simulation.c:887-919): normalised Maxwell
// states per component and the outgoing fluxes of the current boundary cells.
// bnd = [normL, normR, fluxL, fluxR]; UL/UR: [4][m] remapped, normalised.
__global__ void k_maxwell_setup(int N, const double *__restrict__ A, const double *__restrict__ WL, const double *__restrict__ WR,
                                const double *__restrict__ W0, const double *__restrict__ Wn, double *bnd, double *UL, double *UR) {
	const int m = N * N;
	__shared__ double sh[4];
	if (threadIdx.x == 0) {
		double r = 0, l = 0, fl = 0, fr = 0;
		for (int i = 0; i < m / 2; i++) r = add_(r, mul_(A[i], WL[mx_src(N, m, i)]));          // rightward flux of WL trace
		for (int i = m / 2; i < m; i++) l = add_(l, mul_(fabs(A[i]), WR[mx_src(N, m, i)]));    // leftward flux of WR trace
		for (int i = m / 2; i < m; i++) fl = add_(fl, mul_(fabs(A[i]), W0[mx_src(N, m, i)]));  // leftward flux at left boundary
		for (int i = 0; i < m / 2; i++) fr = add_(fr, mul_(A[i], Wn[mx_src(N, m, i)]));        // rightward flux at right boundary
		sh[0] = __ddiv_rn(1.0, r); sh[1] = __ddiv_rn(1.0, l); sh[2] = fl; sh[3] = fr;
		bnd[0] = sh[0]; bnd[1] = sh[1]; bnd[2] = fl; bnd[3] = fr;
	}
	__syncthreads();
	for (int t = threadIdx.x; t < 4 * m; t += blockDim.x) {
		const int c = t / m, mm = t % m;
		UL[t] = mul_(WL[c * m + mx_src(N, m, mm)], sh[0]);
		UR[t] = mul_(WR[c * m + mx_src(N, m, mm)], sh[1]);
	}
}

// outgoing fluxes only (second half step, simulation.c:1059-1066): bnd[2..3]
__global__ void k_maxwell_flux(int N, const double *__restrict__ A, const double *__restrict__ W0, const double *__restrict__ Wn, double *bnd) {
	if (threadIdx.x != 0 || blockIdx.x != 0) return;
	const int m = N * N;
	double fl = 0, fr = 0;
	for (int i = m / 2; i < m; i++) fl = add_(fl, mul_(fabs(A[i]), W0[mx_src(N, m, i)]));
	for (int i = 0; i < m / 2; i++) fr = add_(fr, mul_(A[i], Wn[mx_src(N, m, i)]));
	bnd[2] = fl;
	bnd[3] = fr;
}

struct MaxwellParams {
	int ncells, m, remapN, ncomp;       // ncomp grids of m points per cell
	const double *in; double *out;      // [cell][ncomp][m]
	const double *A;                    // m Maxwell-grid velocities
	double h, dt, lambda;
	const double *flux;                 // fluxL = flux[0], fluxR = flux[1]
	const double *UL, *UR;              // [ncomp][m] normalised boundary states
};

// K11: slope-limiter step with Maxwell boundary ghosts (SlopeLimiterStepMaxwell,
// finite_volume.c:241-323).  Thread per (cell, comp, output point q).  With the
// remap, q < N (v_x = 0 row) is copied from the input (CopyFromMaxwellVelocity,
// simulation.c:848-854) and q >= N maps to Maxwell index mm with src(mm) = q.
__global__ void __launch_bounds__(256) k_transport_maxwell(const MaxwellParams p) {
	const long cs = (long)p.m * p.ncomp;
	const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= cs * p.ncells) return;
	const int i = (int)(idx / cs);
	const int comp = (int)((idx % cs) / p.m), q = (int)(idx % p.m);
	const int n = p.ncells, m = p.m, N = p.remapN;
	const double *X = p.in + (long)comp * m;               // cell j, Maxwell point mm -> X[j*cs + src(mm)]
	if (N && q < N) { p.out[idx] = X[(long)i * cs + q]; return; }
	const int mm = (N && q < m / 2) ? q - N : q;
	auto x = [&](int j, int k) { return X[(long)j * cs + mx_src(N, m, k)]; };
	const double lam1 = sub_(1.0, p.lambda);
	double um1, un1;                                        // ghosts U^n_{-1}, U^n_{N+1}
	if (mm < m / 2) {
		un1 = x(n - 1, mm);
		um1 = add_(mul_(lam1, x(0, m - 1 - mm)), mul_(mul_(p.lambda, p.flux[0]), p.UL[(long)comp * m + mm]));
	} else {
		um1 = x(0, mm);
		un1 = add_(mul_(lam1, x(n - 1, m - 1 - mm)), mul_(mul_(p.lambda, p.flux[1]), p.UR[(long)comp * m + mm]));
	}
	auto V = [&](int j) { return j < 0 ? um1 : (j >= n ? un1 : x(j, mm)); };
	auto alpha = [&](int j) { return sub_(V(j + 1), V(j)); };
	auto hb = [&](int j) { return minmod_(alpha(j), alpha(j - 1)); };
	const LineCoef c = line_coef(p.h, p.dt, p.A[mm]);
	p.out[idx] = slope_update(c, V(i - 1), V(i), V(i + 1), hb(i - 1), hb(i), hb(i + 1));
}

}  // namespace qb
