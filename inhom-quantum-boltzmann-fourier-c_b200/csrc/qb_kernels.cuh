// qb_kernels.cuh — collision kernels for sm_100a, generic over the working
// complex type C (double2: the plain FP64 path; float2: the FP32 precision
// form); the Wigner state itself is always FP64.
//
// Notation: N = velocity grid size, P = 2N padded size, all Fourier-space
// grids complex, element (l, k) at index k + n*l.  A P x P grid in shared
// memory is addressed through Geo::at(row, column): row pitch P + 1 for FP64
// (row passes, column passes and the in-line exchanges free of bank
// conflicts), a wider pitch and, at P = 64, an XOR column swizzle for FP32.
// A CTA has P*T threads (T = P/8 lanes per line,
// one line = one row or one column): thread tid works on line tid / T as
// lane tau = tid % T.
//
// The collision right-hand side is evaluated in factored form (upstream
// loops: src/integrals.c:90-379, src/collision.c:74-254):
//   x^ = FFT2(Pad(x)) for the four Pauli components (k_pad_fft)
//   I1/I4-type sums  S = sum_t phi_t . IFFT2(F . FFT2(Pad(psi2_t . g)))  (k_i1_terms)
//   I2-type sums     Q = sum_t FFT2(Pad(psi1_t f)) . FFT2(Pad(psi2_t g))  (k_i2_terms)
//   I3-type sums     X_r = sum_t sum_i coef_i P_{t,a_i} . FFT2(psi2_t . IFFT2(G_i . P_{t,r}))
//                    with P_{t,c} = FFT2(Pad(psi1_t . W_c))               (k_i3)
//   then outer FFT/IFFT, Extract and the Pauli combination (k_fft_full, k_assemble).
// Moving the sums over quadrature terms inside the outer transforms is exact
// in real arithmetic; results agree with the upstream loop order to rounding.
#pragma once
#include <cooperative_groups.h>
#include "qb_fft.cuh"

namespace qb {

namespace cg = cooperative_groups;

template <int P, class C = double2> struct Geo {
	static constexpr int N = P / 2;
	static constexpr int T = Len<P>::T;
	// row pitch: P + 1 makes every 16-byte (FP64) access pattern of the row,
	// column and exchange passes conflict-free; with 8-byte (FP32) values a
	// half-warp spans two lines, and the pads below halve the excess wavefronts
	// of P + 1 (bank model of all the patterns, 1.5x of ideal instead of 2x)
	static constexpr int LDP = sizeof(C) == 16 ? P + 1 : (P == 64 ? P + 8 : (P == 32 ? P + 4 : P + 2));
	// FP32 at P = 64: pitch P + 8 with the column index XOR-ed by 2 ((row >> 1) & 3)
	// makes every pattern conflict-free (a half-warp's two lines land on
	// opposite halves of the banks, and the swizzle spreads a column's rows)
	static constexpr bool SWZ = sizeof(C) == 8 && P == 64;
	__device__ __forceinline__ static int swz(int r) { return SWZ ? 2 * ((r >> 1) & 3) : 0; }
	// slot of element (row r, column c) of a grid in shared memory
	__device__ __forceinline__ static int at(int r, int c) { return r * LDP + (c ^ swz(r)); }
	// scratch accessors of a row / a column for the transforms
	struct RowA { C *p; int m; __device__ __forceinline__ C &operator()(int pos) const { return p[pos ^ m]; } };
	struct ColA { C *S; int c; __device__ __forceinline__ C &operator()(int pos) const { return S[at(pos, c)]; } };
	__device__ __forceinline__ static RowA row(C *S, int r) { return RowA{ S + r * LDP, swz(r) }; }
	__device__ __forceinline__ static ColA col(C *S, int c) { return ColA{ S, c }; }
	static constexpr int NT = P * T;            // threads per CTA
	static constexpr int GRID = P * LDP;        // smem slots of one padded grid
	// padded index -> index in the N grid, or -1 inside the zero band
	__device__ __forceinline__ static int src(int p) { return p < N / 2 ? p : (p >= 3 * N / 2 ? p - N : -1); }
	// N-grid index -> padded index (GridZeroPad, upstream src/grid.c:171-188)
	__device__ __forceinline__ static int pad(int k) { return k < N / 2 ? k : k + N; }
};

// resident CTAs per SM the term kernels are compiled for: the FP64 kernels
// need ~128 registers a thread (one 512-thread CTA per SM at P = 64); the
// FP32 ones fit two CTAs
template <class C> struct Occ { static constexpr int CTAS = 1; };
template <> struct Occ<float2> { static constexpr int CTAS = 2; };

// ---------------------------------------------------------------------------
// multipliers applied to the FP64 N-grid state before zero padding; the
// product is formed in the working precision C
template <class C> struct MulNone {
	__device__ __forceinline__ C operator()(int, double2 v) const { return mk<C>(v.x, v.y); }
};
template <class C> struct MulReal {           // psi (real N x N) .* v   (MultiplyPointwiseRC)
	const typename CT<C>::R *psi;
	__device__ __forceinline__ C operator()(int idx, double2 v) const { return cscale(mk<C>(v.x, v.y), psi[idx]); }
};
template <class C> struct MulCplx {           // psi (complex N x N) .* v   (MultiplyPointwiseCC)
	const C *psi;
	__device__ __forceinline__ C operator()(int idx, double2 v) const { return cmul(psi[idx], mk<C>(v.x, v.y)); }
};
template <class C> struct MulCplxPair {       // psi .* (v + i b): two grids packed in one transform
	const C *psi;
	const double2 *b;
	__device__ __forceinline__ C operator()(int idx, double2 v) const {
		const double2 w = b[idx];
		return cmul(psi[idx], mk<C>(v.x - w.y, v.y + w.x));
	}
};

// lane's 8 inputs of padded row `prow` of Pad(mul . src)
template <int P, class C, class Mul>
__device__ __forceinline__ void load_pad_row(C (&x)[8], int prow, int tau, const double2 *__restrict__ src, const Mul &mul) {
	using G = Geo<P, C>;
	const int l = G::src(prow);
#pragma unroll
	for (int r = 0; r < 8; r++) {
		const int k = G::src(tau + G::T * r);
		x[r] = (l >= 0 && k >= 0) ? mul(k + G::N * l, src[k + G::N * l]) : czero<C>();
	}
}

// FFT2 (direction DIR) of Pad(mul . src) into the smem grid S (in place, two passes)
template <int P, int DIR, class C, class Mul>
__device__ __forceinline__ void fft2_pad(C *S, const C *tw, const double2 *__restrict__ src, const Mul &mul) {
	using G = Geo<P, C>;
	const int line = threadIdx.x / G::T, tau = threadIdx.x % G::T;
	C x[8];
	load_pad_row<P>(x, line, tau, src, mul);
	fft1d_acc<P, DIR>(x, tau, G::row(S, line), tw);
#pragma unroll
	for (int e = 0; e < 8; e++) S[G::at(line, Len<P>::out_pos(tau, e))] = x[e];
	__syncthreads();
#pragma unroll
	for (int r = 0; r < 8; r++) x[r] = S[G::at(tau + G::T * r, line)];
	fft1d_acc<P, DIR>(x, tau, G::col(S, line), tw);
#pragma unroll
	for (int e = 0; e < 8; e++) S[G::at(Len<P>::out_pos(tau, e), line)] = x[e];
	__syncthreads();
}

// FFT2 of a full grid already in smem S (natural layout), in place
template <int P, int DIR, class C>
__device__ __forceinline__ void fft2_smem(C *S, const C *tw) {
	using G = Geo<P, C>;
	const int line = threadIdx.x / G::T, tau = threadIdx.x % G::T;
	C x[8];
#pragma unroll
	for (int r = 0; r < 8; r++) x[r] = S[G::at(line, tau + G::T * r)];
	fft1d_acc<P, DIR>(x, tau, G::row(S, line), tw);
#pragma unroll
	for (int e = 0; e < 8; e++) S[G::at(line, Len<P>::out_pos(tau, e))] = x[e];
	__syncthreads();
#pragma unroll
	for (int r = 0; r < 8; r++) x[r] = S[G::at(tau + G::T * r, line)];
	fft1d_acc<P, DIR>(x, tau, G::col(S, line), tw);
#pragma unroll
	for (int e = 0; e < 8; e++) S[G::at(Len<P>::out_pos(tau, e), line)] = x[e];
	__syncthreads();
}

// copy smem grid (pitch LDP) to a dense global P x P grid, coalesced
template <int P, class C>
__device__ __forceinline__ void smem_to_global(C *__restrict__ out, const C *S) {
	using G = Geo<P, C>;
	for (int i = threadIdx.x; i < P * P; i += G::NT) out[i] = S[G::at(i / P, i % P)];
}

// ---------------------------------------------------------------------------
// K1: padded forward spectra  out[b] = FFT2(Pad(src[b]))   (one CTA per grid)
template <int P, class C>
__global__ void __launch_bounds__(Geo<P>::NT) k_pad_fft(const double2 *__restrict__ src, C *__restrict__ out) {
	using G = Geo<P, C>;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *S = reinterpret_cast<C *>(smem_raw), *tw = S + G::GRID;
	init_twiddles<P>(tw);
	__syncthreads();
	const long b = blockIdx.x;
	fft2_pad<P, -1>(S, tw, src + b * G::N * G::N, MulNone<C>{});
	smem_to_global<P>(out + b * P * P, S);
}

// ---------------------------------------------------------------------------
// K2: I1/I4-type term sums
//   S[cell][task][chunk] = sum_{t in chunk} phi_t . IFFT2(F . FFT2(Pad(psi2_t . g)))
//   g = gsrc[cell][g_comp[task]],  F = fa * What[cell][f_comp] + fb
template <class C> struct I1ParamsT {
	using R = typename CT<C>::R;
	int ntask, nchunk, nterms;
	const double2 *g; long g_cell;          // N x N grids (FP64 state)
	int g_comp[4];
	const C *What; long w_cell;             // P x P grids
	int f_comp; double fa, fb;
	const R *psi2;                          // nterms x N x N
	const R *phi;                           // nterms x P x P
	C *out;                                 // [cell][task][chunk][P*P]
};
using I1Params = I1ParamsT<double2>;

template <int P, class C>
__global__ void __launch_bounds__(Geo<P>::NT) k_i1_terms(const I1ParamsT<C> p) {
	using G = Geo<P, C>;
	using Lp = Len<P>;
	using R = typename CT<C>::R;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *S = reinterpret_cast<C *>(smem_raw), *F = S + G::GRID, *tw = S + 2 * G::GRID;
	const int chunk = blockIdx.x % p.nchunk;
	const int task = (blockIdx.x / p.nchunk) % p.ntask;
	const long cell = blockIdx.x / (p.nchunk * p.ntask);
	init_twiddles<P>(tw);
	const C *W = p.What + cell * p.w_cell + (long)p.f_comp * P * P;
	const R fa = (R)p.fa, fb = (R)p.fb;
	for (int i = threadIdx.x; i < P * P; i += G::NT) {
		const C w = W[i];
		C f; f.x = fa * w.x + fb; f.y = fa * w.y;
		F[G::at(i / P, i % P)] = f;
	}
	__syncthreads();
	const double2 *g = p.g + cell * p.g_cell + (long)p.g_comp[task] * G::N * G::N;
	const int t0 = (int)((long)chunk * p.nterms / p.nchunk), t1 = (int)((long)(chunk + 1) * p.nterms / p.nchunk);
	const int line = threadIdx.x / G::T, tau = threadIdx.x % G::T;
	C acc[8];
#pragma unroll
	for (int e = 0; e < 8; e++) acc[e] = czero<C>();
	for (int t = t0; t < t1; t++) {
		C x[8];
		// rows: FFT of Pad(psi2_t . g)
		load_pad_row<P>(x, line, tau, g, MulReal<C>{p.psi2 + (long)t * G::N * G::N});
		fft1d_acc<P, -1>(x, tau, G::row(S, line), tw);
#pragma unroll
		for (int e = 0; e < 8; e++) S[G::at(line, Lp::out_pos(tau, e))] = x[e];
		__syncthreads();
		// columns: FFT, multiply by F (convolution with f), inverse FFT
#pragma unroll
		for (int r = 0; r < 8; r++) x[r] = S[G::at(tau + G::T * r, line)];
		fft1d_acc<P, -1>(x, tau, G::col(S, line), tw);
#pragma unroll
		for (int e = 0; e < 8; e++) x[e] = cmul(F[G::at(Lp::out_pos(tau, e), line)], x[e]);
		out_to_in_acc<P>(x, tau, G::col(S, line));
		fft1d_acc<P, +1>(x, tau, G::col(S, line), tw);
#pragma unroll
		for (int e = 0; e < 8; e++) S[G::at(Lp::out_pos(tau, e), line)] = x[e];
		__syncthreads();
		// rows: inverse FFT, multiply by phi_t, accumulate
#pragma unroll
		for (int r = 0; r < 8; r++) x[r] = S[G::at(line, tau + G::T * r)];
		fft1d_acc<P, +1>(x, tau, G::row(S, line), tw);
		const R *phi = p.phi + (long)t * P * P + line * P;
#pragma unroll
		for (int e = 0; e < 8; e++) {
			const R f = phi[Lp::out_pos(tau, e)];
			acc[e].x += f * x[e].x;
			acc[e].y += f * x[e].y;
		}
		// no barrier: the next term's first pass writes only this group's row
	}
	C *o = p.out + ((cell * p.ntask + task) * p.nchunk + chunk) * (long)P * P + line * P;
#pragma unroll
	for (int e = 0; e < 8; e++) o[Lp::out_pos(tau, e)] = acc[e];
}

// ---------------------------------------------------------------------------
// K3: I2-type term sums
//   Q[cell][task][chunk] = sum_t FFT2(Pad(psi1_t . f)) . FFT2(Pad(psi2_t . g))
template <class C> struct I2ParamsT {
	using R = typename CT<C>::R;
	int ntask, nchunk, nterms;
	const double2 *src; long cell_stride;   // N x N grids (FP64 state)
	int f_comp[4], g_comp[4];
	const R *psi1, *psi2;                   // nterms x N x N each
	C *out;                                 // [cell][task][chunk][P*P]
};
using I2Params = I2ParamsT<double2>;

template <int P, class C>
__global__ void __launch_bounds__(Geo<P>::NT) k_i2_terms(const I2ParamsT<C> p) {
	using G = Geo<P, C>;
	using Lp = Len<P>;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *A = reinterpret_cast<C *>(smem_raw), *B = A + G::GRID, *tw = A + 2 * G::GRID;
	const int chunk = blockIdx.x % p.nchunk;
	const int task = (blockIdx.x / p.nchunk) % p.ntask;
	const long cell = blockIdx.x / (p.nchunk * p.ntask);
	init_twiddles<P>(tw);
	__syncthreads();
	const double2 *f = p.src + cell * p.cell_stride + (long)p.f_comp[task] * G::N * G::N;
	const double2 *g = p.src + cell * p.cell_stride + (long)p.g_comp[task] * G::N * G::N;
	const int t0 = (int)((long)chunk * p.nterms / p.nchunk), t1 = (int)((long)(chunk + 1) * p.nterms / p.nchunk);
	const int line = threadIdx.x / G::T, tau = threadIdx.x % G::T;
	C acc[8];
#pragma unroll
	for (int e = 0; e < 8; e++) acc[e] = czero<C>();
	for (int t = t0; t < t1; t++) {
		fft2_pad<P, -1>(A, tw, f, MulReal<C>{p.psi1 + (long)t * G::N * G::N});
		C x[8];
		load_pad_row<P>(x, line, tau, g, MulReal<C>{p.psi2 + (long)t * G::N * G::N});
		fft1d_acc<P, -1>(x, tau, G::row(B, line), tw);
#pragma unroll
		for (int e = 0; e < 8; e++) B[G::at(line, Lp::out_pos(tau, e))] = x[e];
		__syncthreads();
#pragma unroll
		for (int r = 0; r < 8; r++) x[r] = B[G::at(tau + G::T * r, line)];
		fft1d_acc<P, -1>(x, tau, G::col(B, line), tw);
#pragma unroll
		for (int e = 0; e < 8; e++) acc[e] = cfma(A[G::at(Lp::out_pos(tau, e), line)], x[e], acc[e]);
		__syncthreads();
	}
	// column-mapped accumulator -> smem -> coalesced store
#pragma unroll
	for (int e = 0; e < 8; e++) A[G::at(Lp::out_pos(tau, e), line)] = acc[e];
	__syncthreads();
	smem_to_global<P>(p.out + ((cell * p.ntask + task) * p.nchunk + chunk) * (long)P * P, A);
}

// ---------------------------------------------------------------------------
// K4: I3-type sums on a cluster of CS CTAs (one per source component).
// CTA r of the cluster for (cell, chunk) computes P_r = FFT2(Pad(psi1_t . src_r))
// into its shared memory; the other CTAs read it through distributed shared
// memory.  For each of its combos (a, g, coef) it accumulates
//   X_r += coef * P_a . FFT2(psi2_t . IFFT2(G_g . P_r)).
// Contiguous ranges of the flattened (cell, term) work of the I3 sums, one per
// cluster: cluster k takes u in [start(k), start(k + 1)) of total = ncells x
// nterms, u = cell x nterms + term, and writes one partial per cell it
// touches to slot k x maxc + (cell - first_cell(k)).  Cell c's partials are
// those of clusters cluster_of(c nterms) .. cluster_of((c + 1) nterms - 1),
// summed in that order.  nslots = 0: the (cell, chunk) grid instead.
struct TermRanges {
	int nslots = 0, nterms = 0, maxc = 0;
	long total = 0;
	__host__ __device__ long start(int k) const { return (long)k * total / nslots; }
	__host__ __device__ int cluster_of(long u) const { return (int)(((u + 1) * nslots - 1) / total); }
	__host__ __device__ long first_cell(int k) const { return start(k) / nterms; }
};

template <class C> struct I3ParamsT {
	using R = typename CT<C>::R;
	int nchunk, nterms;
	TermRanges rg;                                        // nslots > 0: one term range per cluster (k_i3p)
	const double2 *src; long src_cell; int src_comp[4];   // N x N grids (FP64 state)
	const C *Ghat; long g_cell;                           // P x P grids, G_g at Ghat + cell*g_cell + g*P*P
	int ncombo[4]; int ca[4][4], cgi[4][4]; double ccoef[4][4];
	const C *psi1;                                        // nterms x N x N (complex)
	const R *psi2T;                                       // transposed P x P tables
	const int *psi2_idx; const double *psi2_scale;        // per term
	C *out;                                               // [cell][chunk][CS][P*P]
	int *err;                                             // error word of bounded waits (may be null)
};
using I3Params = I3ParamsT<double2>;

template <int P, int CS, class C>
__global__ void __launch_bounds__(Geo<P>::NT, Occ<C>::CTAS) k_i3(const I3ParamsT<C> p) {
	using G = Geo<P, C>;
	using Lp = Len<P>;
	using R = typename CT<C>::R;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *Pr = reinterpret_cast<C *>(smem_raw), *Ug = Pr + G::GRID, *tw = Pr + 2 * G::GRID;
	cg::cluster_group cluster = cg::this_cluster();
	const int rank = (int)cluster.block_rank();
	const long cid = blockIdx.x / CS;
	const int chunk = (int)(cid % p.nchunk);
	const long cell = cid / p.nchunk;
	init_twiddles<P>(tw);
	__syncthreads();
	const double2 *src = p.src + cell * p.src_cell + (long)p.src_comp[rank] * G::N * G::N;
	const int t0 = (int)((long)chunk * p.nterms / p.nchunk), t1 = (int)((long)(chunk + 1) * p.nterms / p.nchunk);
	const int line = threadIdx.x / G::T, tau = threadIdx.x % G::T;
	C acc[8];
#pragma unroll
	for (int e = 0; e < 8; e++) acc[e] = czero<C>();
	const int nc = p.ncombo[rank];
	for (int t = t0; t < t1; t++) {
		fft2_pad<P, -1>(Pr, tw, src, MulCplx<C>{p.psi1 + (long)t * G::N * G::N});
		cluster.sync();
		const R *psi2 = p.psi2T + (long)p.psi2_idx[t] * P * P;
		const R sc = (R)p.psi2_scale[t];
		for (int c = 0; c < nc; c++) {
			const C *Gg = p.Ghat + cell * p.g_cell + (long)p.cgi[rank][c] * P * P;
			C x[8];
			// rows: IFFT of G_g . P_r
#pragma unroll
			for (int r = 0; r < 8; r++) {
				const int k = tau + G::T * r;
				x[r] = cmul(Gg[line * P + k], Pr[G::at(line, k)]);
			}
			fft1d_acc<P, +1>(x, tau, G::row(Ug, line), tw);
#pragma unroll
			for (int e = 0; e < 8; e++) Ug[G::at(line, Lp::out_pos(tau, e))] = x[e];
			__syncthreads();
			// columns: IFFT, multiply by psi2_t, FFT
#pragma unroll
			for (int r = 0; r < 8; r++) x[r] = Ug[G::at(tau + G::T * r, line)];
			fft1d_acc<P, +1>(x, tau, G::col(Ug, line), tw);
#pragma unroll
			for (int e = 0; e < 8; e++) {
				const R f = sc * psi2[line * P + Lp::out_pos(tau, e)];
				x[e].x *= f;
				x[e].y *= f;
			}
			out_to_in_acc<P>(x, tau, G::col(Ug, line));
			fft1d_acc<P, -1>(x, tau, G::col(Ug, line), tw);
#pragma unroll
			for (int e = 0; e < 8; e++) Ug[G::at(Lp::out_pos(tau, e), line)] = x[e];
			__syncthreads();
			// rows: FFT, multiply by P_a (remote), accumulate
#pragma unroll
			for (int r = 0; r < 8; r++) x[r] = Ug[G::at(line, tau + G::T * r)];
			fft1d_acc<P, -1>(x, tau, G::row(Ug, line), tw);
			const C *Pa = cluster.map_shared_rank(Pr, p.ca[rank][c]);
			const R coef = (R)p.ccoef[rank][c];
#pragma unroll
			for (int e = 0; e < 8; e++) {
				const C v = cmul(Pa[G::at(line, Lp::out_pos(tau, e))], x[e]);
				acc[e].x += coef * v.x;
				acc[e].y += coef * v.y;
			}
			__syncthreads();
		}
		cluster.sync();
	}
	C *o = p.out + ((cell * p.nchunk + chunk) * CS + rank) * (long)P * P + line * P;
#pragma unroll
	for (int e = 0; e < 8; e++) o[Lp::out_pos(tau, e)] = acc[e];
}

// ---------------------------------------------------------------------------
// Tensor memory (TMEM) as accumulator storage.  A CTA allocates `ncols`
// columns of its SM's 128-lane TMEM; warp w reaches lanes 32 (w % 4) ..
// 32 (w % 4) + 31 (thread = lane), and the four warps that share a lane
// quarter split the columns (slot w / 4).  Loads and stores are warp-wide
// (tcgen05.ld / st .32x32b) and asynchronous until tcgen05.wait.
__device__ __forceinline__ void tmem_alloc(unsigned *slot_smem, unsigned ncols) {
	const unsigned a = (unsigned)__cvta_generic_to_shared(slot_smem);
	asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(a), "r"(ncols) : "memory");
	asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols) {
	asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// one complex value per thread at column `taddr` (+ 4 columns FP64, 2 FP32)
__device__ __forceinline__ void tmem_ld(unsigned taddr, double2 &v) {
	unsigned a, b, c, d;
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];" : "=r"(a), "=r"(b), "=r"(c), "=r"(d) : "r"(taddr) : "memory");
	v.x = __hiloint2double((int)b, (int)a);
	v.y = __hiloint2double((int)d, (int)c);
}
__device__ __forceinline__ void tmem_st(unsigned taddr, double2 v) {
	const unsigned a = (unsigned)__double2loint(v.x), b = (unsigned)__double2hiint(v.x);
	const unsigned c = (unsigned)__double2loint(v.y), d = (unsigned)__double2hiint(v.y);
	asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}
__device__ __forceinline__ void tmem_ld(unsigned taddr, float2 &v) {
	unsigned a, b;
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(a), "=r"(b) : "r"(taddr) : "memory");
	v.x = __uint_as_float(a);
	v.y = __uint_as_float(b);
}
__device__ __forceinline__ void tmem_st(unsigned taddr, float2 v) {
	asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(taddr), "r"(__float_as_uint(v.x)), "r"(__float_as_uint(v.y)) : "memory");
}

// eight consecutive complex values (32 columns FP64, 16 FP32) of this
// thread's lane in one warp-wide load or store
__device__ __forceinline__ void tmem_ld8(unsigned taddr, double2 (&v)[8]) {
	unsigned r[32];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
	             : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
	             : "r"(taddr) : "memory");
#pragma unroll
	for (int e = 0; e < 8; e++) {
		v[e].x = __hiloint2double((int)r[4 * e + 1], (int)r[4 * e]);
		v[e].y = __hiloint2double((int)r[4 * e + 3], (int)r[4 * e + 2]);
	}
}
__device__ __forceinline__ void tmem_st8(unsigned taddr, const double2 (&v)[8]) {
	unsigned r[32];
#pragma unroll
	for (int e = 0; e < 8; e++) {
		r[4 * e] = (unsigned)__double2loint(v[e].x); r[4 * e + 1] = (unsigned)__double2hiint(v[e].x);
		r[4 * e + 2] = (unsigned)__double2loint(v[e].y); r[4 * e + 3] = (unsigned)__double2hiint(v[e].y);
	}
	asm volatile("tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};"
	             :: "r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]), "r"(r[16]), "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23]), "r"(r[24]), "r"(r[25]), "r"(r[26]), "r"(r[27]), "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31]) : "memory");
}
__device__ __forceinline__ void tmem_ld8(unsigned taddr, float2 (&v)[8]) {
	unsigned r[16];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
	             : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
	             : "r"(taddr) : "memory");
#pragma unroll
	for (int e = 0; e < 8; e++) { v[e].x = __uint_as_float(r[2 * e]); v[e].y = __uint_as_float(r[2 * e + 1]); }
}
__device__ __forceinline__ void tmem_st8(unsigned taddr, const float2 (&v)[8]) {
	unsigned r[16];
#pragma unroll
	for (int e = 0; e < 8; e++) { r[2 * e] = __float_as_uint(v[e].x); r[2 * e + 1] = __float_as_uint(v[e].y); }
	asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16};"
	             :: "r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]) : "memory");
}

// four consecutive FP64 complex values (16 columns) in one load or store
__device__ __forceinline__ void tmem_ld4(unsigned taddr, double2 (&v)[4]) {
	unsigned r[16];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
	             : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
	             : "r"(taddr) : "memory");
#pragma unroll
	for (int e = 0; e < 4; e++) {
		v[e].x = __hiloint2double((int)r[4 * e + 1], (int)r[4 * e]);
		v[e].y = __hiloint2double((int)r[4 * e + 3], (int)r[4 * e + 2]);
	}
}
__device__ __forceinline__ void tmem_st4(unsigned taddr, const double2 (&v)[4]) {
	unsigned r[16];
#pragma unroll
	for (int e = 0; e < 4; e++) {
		r[4 * e] = (unsigned)__double2loint(v[e].x); r[4 * e + 1] = (unsigned)__double2hiint(v[e].x);
		r[4 * e + 2] = (unsigned)__double2loint(v[e].y); r[4 * e + 3] = (unsigned)__double2hiint(v[e].y);
	}
	asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16};"
	             :: "r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]) : "memory");
}

// eight FP64 reals (16 columns) in one load or store
__device__ __forceinline__ void tmem_ld8r(unsigned taddr, double (&v)[8]) {
	unsigned r[16];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
	             : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
	             : "r"(taddr) : "memory");
#pragma unroll
	for (int e = 0; e < 8; e++) v[e] = __hiloint2double((int)r[2 * e + 1], (int)r[2 * e]);
}
__device__ __forceinline__ void tmem_st8r(unsigned taddr, const double (&v)[8]) {
	unsigned r[16];
#pragma unroll
	for (int e = 0; e < 8; e++) { r[2 * e] = (unsigned)__double2loint(v[e]); r[2 * e + 1] = (unsigned)__double2hiint(v[e]); }
	asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16};"
	             :: "r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]) : "memory");
}

// eight FP32 reals (8 columns) in one load or store
__device__ __forceinline__ void tmem_ld8r(unsigned taddr, float (&v)[8]) {
	unsigned r[8];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
	             : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
	             : "r"(taddr) : "memory");
#pragma unroll
	for (int e = 0; e < 8; e++) v[e] = __uint_as_float(r[e]);
}
__device__ __forceinline__ void tmem_st8r(unsigned taddr, const float (&v)[8]) {
	unsigned r[8];
#pragma unroll
	for (int e = 0; e < 8; e++) r[e] = __float_as_uint(v[e]);
	asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};"
	             :: "r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]) : "memory");
}

// length-L transform with the lane's twiddle powers w_L^(tau q), q = 1..4
// (forward sign), read from tensor memory at taddr (4 complex FP64 values);
// w^5..w^7 = w^4 w^1..w^3.  The load is issued before the first radix-8
// stage and waited for after it.
template <int L, int DIR, class Acc>
__device__ __forceinline__ void fft1d_acct(double2 (&x)[8], int tau, const Acc &sc, unsigned taddr) {
	double2 w[4];
	tmem_ld4(taddr, w);
	dft8<DIR>(x);
	tmem_wait_ld();
	if (DIR > 0) {
#pragma unroll
		for (int q = 0; q < 4; q++) w[q].y = -w[q].y;
	}
#pragma unroll
	for (int q = 1; q <= 4; q++) x[q] = cmul(x[q], w[q - 1]);
#pragma unroll
	for (int q = 5; q < 8; q++) x[q] = cmul(x[q], cmul(w[3], w[q - 5]));
	fft1d_tail<L, DIR>(x, tau, sc);
}

// the lane's twiddle powers computed once per kernel: FP32 in registers (wp,
// fft1d_accw), FP64 in tensor memory (registers are exhausted there; the
// loads replace the six complex multiplies of the power recurrence and add
// no shared-memory traffic)
template <int L, int DIR, class C, class Acc>
__device__ __forceinline__ void fft1d_lane(C (&x)[8], int tau, const Acc &sc, const C (&wp)[8], unsigned twaddr) {
	if constexpr (sizeof(C) == 8) fft1d_accw<L, DIR>(x, tau, sc, wp);
	else fft1d_acct<L, DIR>(x, tau, sc, twaddr);
}

// TMEM accumulators of k_i3p: 2 outputs x 8 values per thread
template <class C> struct I3Tmem {
	static constexpr unsigned WPC = sizeof(C) / 4;            // 32-bit columns per complex value
	static constexpr unsigned PER_THREAD = 2 * 8 * WPC;       // columns of one thread's slice
	static constexpr unsigned NCOLS = 4 * PER_THREAD;         // 4 warps share a lane quarter: 256 (FP64), 128 (FP32)
	// after the accumulators each thread keeps its 8 psi2 values of the current
	// term, its 8 values of the current P_j and (FP64) its twiddle powers w^1..w^4;
	// columns a slot: 16 / 32 / 16 (FP64), 8 / 16 (FP32)
	static constexpr unsigned ALLOC = sizeof(C) == 16 ? 512 : 256;
	// column address of value e of output q of this thread
	__device__ __forceinline__ static unsigned addr(unsigned base, int q, int e) {
		const unsigned w = threadIdx.x >> 5;
		return base + ((32u * (w & 3u)) << 16) + (w >> 2) * PER_THREAD + (unsigned)(q * 8 + e) * WPC;
	}
	static constexpr unsigned PSI = 8 * WPC / 2, PJ = 8 * WPC;   // columns a slot
	__device__ __forceinline__ static unsigned lanes() { return (32u * ((threadIdx.x >> 5) & 3u)) << 16; }
	__device__ __forceinline__ static unsigned slot() { return threadIdx.x >> 7; }
	__device__ __forceinline__ static unsigned psiaddr(unsigned base) { return base + lanes() + NCOLS + slot() * PSI; }
	__device__ __forceinline__ static unsigned pjaddr(unsigned base) { return base + lanes() + NCOLS + 4 * PSI + slot() * PJ; }
	__device__ __forceinline__ static unsigned twaddr(unsigned base) { return base + lanes() + NCOLS + 4 * (PSI + PJ) + slot() * 16u; }
};

// FP32 at P = 64: each CTA of the pair pushes its P grids of the term into the
// partner's shared memory by bulk copies (cp.async.bulk between the pair's
// shared memories, completing on the partner's mbarrier), so that every P_a
// of the chains is read from local shared memory.  push_issue sends `bytes`
// of the own grids at `own` to `peer_copy` in the partner, after the CTA
// barrier that follows the grid's transform (the partner has finished reading
// its copy of the previous term: a cluster barrier ends every term).
// push_wait waits for the partner's copies before the chains (bounded: a wait
// that runs out sets the error word).  push_release keeps the copies' sources
// until they have been read, before the next term overwrites them.
__device__ __forceinline__ uint32_t smem_u32a(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
// `expect` > 0: this CTA's arrival on its own mbarrier for the term, expecting
// that many bytes from the partner (the first of the term's copies)
__device__ __forceinline__ void push_issue(const void *own, void *peer_copy, uint32_t bytes, uint64_t *mbar, int prank,
                                           uint32_t expect) {
	if (threadIdx.x == 0) {
		const uint32_t mb = smem_u32a(mbar);
		uint32_t dst, mbr;
		asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(dst) : "r"(smem_u32a(peer_copy)), "r"(prank));
		asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(mbr) : "r"(mb), "r"(prank));
		if (expect > 0) asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(expect) : "memory");
		asm volatile("cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
		             "r"(smem_u32a(own)), "r"(bytes), "r"(mbr) : "memory");
		asm volatile("cp.async.bulk.commit_group;" ::: "memory");
	}
}
__device__ __forceinline__ void push_wait(uint64_t *mbar, unsigned &phase, int *err) {
	const uint32_t mb = smem_u32a(mbar);
	bool ok = false;
	for (unsigned i = 0; i < (1u << 24) && !ok; i++) {
		uint32_t done = 0;
		asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
		             : "=r"(done) : "r"(mb), "r"(phase) : "memory");
		ok = done != 0;
	}
	if (!ok && err != nullptr && (threadIdx.x & 31) == 0) atomicExch(err, 1);
	phase ^= 1u;
}
__device__ __forceinline__ void push_release() {
	if (threadIdx.x == 0) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void push_init(uint64_t *mbar) {
	if (threadIdx.x == 0) {
		asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32a(mbar)) : "memory");
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
}
__device__ __forceinline__ void fence_async_smem_a() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ---------------------------------------------------------------------------
// K4p: the I3 sums of the collision operator on a cluster of 2 CTAs, CTA r
// holding components 2r and 2r + 1: per term it computes both spectra
// P_{t,c} = FFT2(Pad(psi1_t . W_c)) into its shared memory and, after a
// cluster barrier, the 8 (pair, combo) chains of its two outputs
//   X_j += eta_i P_i . FFT2(psi2_t . IFFT2(W^_i . P_j)),  j in {2r, 2r + 1}
// with P_i of the partner's components read through distributed shared
// memory.  The two 8-value accumulators of every thread live in TMEM, which
// frees their registers and lets 2-CTA clusters use all 148 SMs (4-CTA
// clusters of k_i3 fit 33 of 37 four-SM slots).  The rest of the TMEM
// allocation caches values each thread reuses at its own positions: its psi2
// values of the current term (one L2 read for the term's 8 chains), its P_j
// values of the current output (one shared-memory read for the output's 4
// chains) and, in FP64, its twiddle powers (FP32 keeps them in registers).
// Output as k_i3 with CS = 4.
//
// kind: null (every cell) or the per-cell form of k_nyquist_kind; this kernel
// then takes the cells of kind 1 (the real form k_i3pr takes kind 0).
template <int P, class C>
__global__ void __launch_bounds__(Geo<P>::NT, 1) k_i3p(const I3ParamsT<C> p, const int *kind) {
	using G = Geo<P, C>;
	using Lp = Len<P>;
	using R = typename CT<C>::R;
	using TM = I3Tmem<C>;
	constexpr bool kPush = sizeof(C) == 8;                   // FP32: the partner's P grids copied in (Pr)
	extern __shared__ __align__(16) unsigned char smem_raw[];
	__shared__ unsigned tmem_slot;
	__shared__ __align__(8) uint64_t pmbar;
	unsigned pphase = 0;
	C *Pq = reinterpret_cast<C *>(smem_raw);                 // P of components 2r, 2r + 1 (2 grids)
	C *Ug = Pq + 2 * G::GRID, *tw = Pq + 3 * G::GRID;
	C *Pr = tw + P;                                          // FP32: the partner's 2 P grids
	cg::cluster_group cluster = cg::this_cluster();
	const int rank = (int)cluster.block_rank();
	const long cid = blockIdx.x / 2;
	// work of this cluster: terms [u, u1) of the flattened (cell, term) order
	long u, u1;
	if (p.rg.nslots > 0) {
		u = p.rg.start((int)cid);
		u1 = p.rg.start((int)cid + 1);
	} else {
		const int chunk = (int)(cid % p.nchunk);
		const long cell = cid / p.nchunk;
		if (kind != nullptr && kind[cell] != 1) return;     // both CTAs of the cluster leave before any barrier
		u = cell * p.nterms + (long)chunk * p.nterms / p.nchunk;
		u1 = cell * p.nterms + (long)(chunk + 1) * p.nterms / p.nchunk;
	}
	const int warp = threadIdx.x >> 5;
	if (warp == 0) tmem_alloc(&tmem_slot, TM::ALLOC);
	init_twiddles<P>(tw);
	tmem_fence_before();
	__syncthreads();
	tmem_fence_after();
	const unsigned tbase = tmem_slot;
	const int line = threadIdx.x / G::T, tau = threadIdx.x % G::T;
	C wp[8];
	const unsigned twaddr = TM::twaddr(tbase);
	if constexpr (sizeof(C) == 8) {
#pragma unroll
		for (int q = 0; q < 8; q++) wp[q] = tw[(tau * q) & (P - 1)];
	} else {
		double2 a[4];
#pragma unroll
		for (int q = 0; q < 4; q++) a[q] = tw[(tau * (q + 1)) & (P - 1)];
		tmem_st4(twaddr, a);
	}
	C *Ppeer = cluster.map_shared_rank(Pq, rank ^ 1);
	if constexpr (kPush) {
		push_init(&pmbar);
		cluster.sync();                                      // the partner's mbarrier is initialised
	}
	// one segment per cell of the range (the (cell, chunk) grid has one)
#pragma unroll 1
	while (u < u1) {
	const long cell = u / p.nterms;
	const int t0 = (int)(u % p.nterms);
	const int t1 = (int)min((long)p.nterms, t0 + (u1 - u));
	u += t1 - t0;
#pragma unroll
	for (int q = 0; q < 2; q++)
#pragma unroll
		for (int e = 0; e < 8; e++) tmem_st(TM::addr(tbase, q, e), czero<C>());
	tmem_wait_st();
	const C *Gcell = p.Ghat + cell * p.g_cell;
	for (int t = t0; t < t1; t++) {
#pragma unroll 1
		for (int q = 0; q < 2; q++) {
			const double2 *src = p.src + cell * p.src_cell + (long)p.src_comp[2 * rank + q] * G::N * G::N;
			fft2_pad<P, -1>(Pq + q * G::GRID, tw, src, MulCplx<C>{p.psi1 + (long)t * G::N * G::N});
			if constexpr (kPush) {
				// FP32: each grid goes to the partner as soon as it is complete, the
				// first copy overlapping the second transform
				fence_async_smem_a();
				__syncthreads();
				push_issue(Pq + q * G::GRID, Pr + q * G::GRID, (uint32_t)(G::GRID * sizeof(C)), &pmbar, rank ^ 1,
				           q == 0 ? (uint32_t)(2 * G::GRID * sizeof(C)) : 0u);
			}
		}
		if constexpr (!kPush) cluster.sync();
		const R *psi2 = p.psi2T + (long)p.psi2_idx[t] * P * P;
		const R sc = (R)p.psi2_scale[t];
		{
			// this thread's psi2 values of the term (column line, rows out_pos(tau, e)), read
			// once from L2 for the term's 8 chains; the previous term's reads of the slot
			// have completed (tcgen05.wait::ld in every chain)
			R f[8];
#pragma unroll
			for (int e = 0; e < 8; e++) f[e] = sc * psi2[line * P + Lp::out_pos(tau, e)];
			tmem_st8r(TM::psiaddr(tbase), f);
			tmem_wait_st();
		}
		if constexpr (kPush) push_wait(&pmbar, pphase, p.err);
#pragma unroll 1
		for (int q = 0; q < 2; q++) {
			const int j = 2 * rank + q;
			const C *Pj = Pq + q * G::GRID;
			{
				// this thread's 8 values of P_j (row line, columns tau + 8 r), read once from
				// shared memory for the 4 chains of output j
				C v[8];
#pragma unroll
				for (int r = 0; r < 8; r++) v[r] = Pj[G::at(line, tau + G::T * r)];
				tmem_st8(TM::pjaddr(tbase), v);
				tmem_wait_st();
			}
#pragma unroll 1
			for (int c = 0; c < p.ncombo[j]; c++) {
				const C *Gg = Gcell + (long)p.cgi[j][c] * P * P;
				C x[8];
				// rows: IFFT of G_g . P_j
				{
					C pj[8];
					tmem_ld8(TM::pjaddr(tbase), pj);
					C g[8];
#pragma unroll
					for (int r = 0; r < 8; r++) g[r] = Gg[line * P + tau + G::T * r];
					tmem_wait_ld();
#pragma unroll
					for (int r = 0; r < 8; r++) x[r] = cmul(g[r], pj[r]);
				}
				fft1d_lane<P, +1>(x, tau, G::row(Ug, line), wp, twaddr);
#pragma unroll
				for (int e = 0; e < 8; e++) Ug[G::at(line, Lp::out_pos(tau, e))] = x[e];
				__syncthreads();
				// columns: IFFT, multiply by psi2_t, FFT
#pragma unroll
				for (int r = 0; r < 8; r++) x[r] = Ug[G::at(tau + G::T * r, line)];
				fft1d_lane<P, +1>(x, tau, G::col(Ug, line), wp, twaddr);
				{
					R f[8];
					tmem_ld8r(TM::psiaddr(tbase), f);
					tmem_wait_ld();
#pragma unroll
					for (int e = 0; e < 8; e++) { x[e].x *= f[e]; x[e].y *= f[e]; }
				}
				out_to_in_acc<P>(x, tau, G::col(Ug, line));
				fft1d_lane<P, -1>(x, tau, G::col(Ug, line), wp, twaddr);
#pragma unroll
				for (int e = 0; e < 8; e++) Ug[G::at(Lp::out_pos(tau, e), line)] = x[e];
				__syncthreads();
				// rows: FFT, multiply by P_a (own or the partner's), accumulate in TMEM
#pragma unroll
				for (int r = 0; r < 8; r++) x[r] = Ug[G::at(line, tau + G::T * r)];
				fft1d_lane<P, -1>(x, tau, G::row(Ug, line), wp, twaddr);
				const int a = p.ca[j][c];
				const C *Pa = ((a >> 1) == rank ? Pq : (kPush ? Pr : Ppeer)) + (a & 1) * G::GRID;
				const R coef = (R)p.ccoef[j][c];
				C acc[8];
				if constexpr (sizeof(C) == 16) tmem_ld8(TM::addr(tbase, q, 0), acc);   // one load (FP64); FP32 per value measured faster
				else {
#pragma unroll
					for (int e = 0; e < 8; e++) tmem_ld(TM::addr(tbase, q, e), acc[e]);
				}
				tmem_wait_ld();
#pragma unroll
				for (int e = 0; e < 8; e++) {
					const C v = cmul(Pa[G::at(line, Lp::out_pos(tau, e))], x[e]);
					acc[e].x += coef * v.x;
					acc[e].y += coef * v.y;
				}
				if constexpr (sizeof(C) == 16) tmem_st8(TM::addr(tbase, q, 0), acc);
				else {
#pragma unroll
					for (int e = 0; e < 8; e++) tmem_st(TM::addr(tbase, q, e), acc[e]);
				}
				tmem_wait_st();
				// no barrier here: the row passes that end this pair and begin the
				// next touch only the rows of their own 8-lane group, and the next
				// column pass waits behind the next pair's first barrier
			}
		}
		if constexpr (kPush) push_release();              // the own P grids are read by the copy before they change
		cluster.sync();
	}
	// partial sums of this segment: slot (cluster, cell) of the ranges, or (cell, chunk)
	const long slot = p.rg.nslots > 0 ? cid * p.rg.maxc + (cell - p.rg.first_cell((int)cid))
	                                  : cell * p.nchunk + (int)(cid % p.nchunk);
#pragma unroll 1
	for (int q = 0; q < 2; q++) {
		C acc[8];
		tmem_ld8(TM::addr(tbase, q, 0), acc);
		tmem_wait_ld();
		C *o = p.out + (slot * 4 + 2 * rank + q) * (long)P * P + line * P;
#pragma unroll
		for (int e = 0; e < 8; e++) o[Lp::out_pos(tau, e)] = acc[e];
	}
	}
	tmem_fence_before();
	__syncthreads();
	tmem_fence_after();
	if (warp == 0) tmem_dealloc(tbase, TM::ALLOC);
}

// k_i3p in real arithmetic (FP32 form, cells without Nyquist content): the
// identity of k_i3_full128r at P = 64.  One transform of psi1_t . (W_2r +
// i W_2r+1) gives the real spectra P_2r (real part) and P_2r+1 (imaginary
// part) in one shared grid; the chains of combos (i0, i1) of an output share
// one complex transform of P_j . (W^_i0 + i W^_i1), and the real accumulators
// take eta_i0 P_i0 . Re + eta_i1 P_i1 . Im.  Same shared-memory layout as k_i3p
// (the second P grid unused); tensor memory: 2 x 8 real accumulators, 8 psi2
// and 8 P_j values per thread.
struct I3TmemR {
	static constexpr unsigned PER_THREAD = 16, NCOLS = 64, PSI = 8, PJ = 8, ALLOC = 128;
	__device__ __forceinline__ static unsigned lanes() { return (32u * ((threadIdx.x >> 5) & 3u)) << 16; }
	__device__ __forceinline__ static unsigned slot() { return threadIdx.x >> 7; }
	__device__ __forceinline__ static unsigned addr(unsigned base, int q) { return base + lanes() + (threadIdx.x >> 7) * PER_THREAD + (unsigned)q * 8; }
	__device__ __forceinline__ static unsigned psiaddr(unsigned base) { return base + lanes() + NCOLS + slot() * PSI; }
	__device__ __forceinline__ static unsigned pjaddr(unsigned base) { return base + lanes() + NCOLS + 4 * PSI + slot() * PJ; }
};

template <int P>
__global__ void __launch_bounds__(Geo<P>::NT, 1) k_i3pr(const I3ParamsT<float2> p, const int *kind) {
	using C = float2;
	using G = Geo<P, C>;
	using Lp = Len<P>;
	using TM = I3TmemR;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	__shared__ unsigned tmem_slot;
	C *Pq = reinterpret_cast<C *>(smem_raw);                 // P_2r + i P_2r+1
	C *Ug = Pq + 2 * G::GRID, *tw = Pq + 3 * G::GRID;
	C *Pr = Pq + G::GRID;                                    // the partner's packed P grid, copied in
	__shared__ __align__(8) uint64_t pmbar;
	unsigned pphase = 0;
	cg::cluster_group cluster = cg::this_cluster();
	const int rank = (int)cluster.block_rank();
	const long cid = blockIdx.x / 2;
	const int chunk = (int)(cid % p.nchunk);
	const long cell = cid / p.nchunk;
	if (kind[cell] != 0) return;                          // both CTAs of the cluster leave before any barrier
	const int warp = threadIdx.x >> 5;
	if (warp == 0) tmem_alloc(&tmem_slot, TM::ALLOC);
	init_twiddles<P>(tw);
	tmem_fence_before();
	__syncthreads();
	tmem_fence_after();
	const unsigned tbase = tmem_slot;
	const int line = threadIdx.x / G::T, tau = threadIdx.x % G::T;
	C wp[8];
#pragma unroll
	for (int q = 0; q < 8; q++) wp[q] = tw[(tau * q) & (P - 1)];
	{
		const float z[8] = { 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f };
		tmem_st8r(TM::addr(tbase, 0), z);
		tmem_st8r(TM::addr(tbase, 1), z);
		tmem_wait_st();
	}
	const C *Gcell = p.Ghat + cell * p.g_cell;
	const int t0 = (int)((long)chunk * p.nterms / p.nchunk), t1 = (int)((long)(chunk + 1) * p.nterms / p.nchunk);
	push_init(&pmbar);
	cluster.sync();                                          // the partner's mbarrier is initialised
	for (int t = t0; t < t1; t++) {
		{
			const double2 *sa = p.src + cell * p.src_cell + (long)p.src_comp[2 * rank] * G::N * G::N;
			const double2 *sb = p.src + cell * p.src_cell + (long)p.src_comp[2 * rank + 1] * G::N * G::N;
			fft2_pad<P, -1>(Pq, tw, sa, MulCplxPair<C>{p.psi1 + (long)t * G::N * G::N, sb});
		}
		fence_async_smem_a();
		__syncthreads();                                     // no distributed-shared-memory reads: a CTA barrier
		push_issue(Pq, Pr, (uint32_t)(G::GRID * sizeof(C)), &pmbar, rank ^ 1, (uint32_t)(G::GRID * sizeof(C)));
		const float *psi2 = p.psi2T + (long)p.psi2_idx[t] * P * P;
		const float sc = (float)p.psi2_scale[t];
		{
			float f[8];
#pragma unroll
			for (int e = 0; e < 8; e++) f[e] = sc * psi2[line * P + Lp::out_pos(tau, e)];
			tmem_st8r(TM::psiaddr(tbase), f);
			tmem_wait_st();
		}
		push_wait(&pmbar, pphase, p.err);
#pragma unroll 1
		for (int q = 0; q < 2; q++) {
			const int j = 2 * rank + q;
			{
				float v[8];
#pragma unroll
				for (int r = 0; r < 8; r++) {
					const C pv = Pq[G::at(line, tau + G::T * r)];
					v[r] = q ? pv.y : pv.x;
				}
				tmem_st8r(TM::pjaddr(tbase), v);
				tmem_wait_st();
			}
#pragma unroll 1
			for (int c = 0; c + 1 < p.ncombo[j]; c += 2) {
				const C *G0 = Gcell + (long)p.cgi[j][c] * P * P, *G1 = Gcell + (long)p.cgi[j][c + 1] * P * P;
				C x[8];
				// rows: IFFT of P_j . (W^_i0 + i W^_i1)
				{
					float pj[8];
					tmem_ld8r(TM::pjaddr(tbase), pj);
					float g0[8], g1[8];
#pragma unroll
					for (int r = 0; r < 8; r++) {
						g0[r] = G0[line * P + tau + G::T * r].x;
						g1[r] = G1[line * P + tau + G::T * r].x;
					}
					tmem_wait_ld();
#pragma unroll
					for (int r = 0; r < 8; r++) x[r] = mk<C>(pj[r] * g0[r], pj[r] * g1[r]);
				}
				fft1d_lane<P, +1>(x, tau, G::row(Ug, line), wp, 0u);
#pragma unroll
				for (int e = 0; e < 8; e++) Ug[G::at(line, Lp::out_pos(tau, e))] = x[e];
				__syncthreads();
				// columns: IFFT, multiply by psi2_t, FFT
#pragma unroll
				for (int r = 0; r < 8; r++) x[r] = Ug[G::at(tau + G::T * r, line)];
				fft1d_lane<P, +1>(x, tau, G::col(Ug, line), wp, 0u);
				{
					float f[8];
					tmem_ld8r(TM::psiaddr(tbase), f);
					tmem_wait_ld();
#pragma unroll
					for (int e = 0; e < 8; e++) { x[e].x *= f[e]; x[e].y *= f[e]; }
				}
				out_to_in_acc<P>(x, tau, G::col(Ug, line));
				fft1d_lane<P, -1>(x, tau, G::col(Ug, line), wp, 0u);
#pragma unroll
				for (int e = 0; e < 8; e++) Ug[G::at(Lp::out_pos(tau, e), line)] = x[e];
				__syncthreads();
				// rows: FFT; the real part belongs to i0, the imaginary part to i1
#pragma unroll
				for (int r = 0; r < 8; r++) x[r] = Ug[G::at(line, tau + G::T * r)];
				fft1d_lane<P, -1>(x, tau, G::row(Ug, line), wp, 0u);
				const int a0 = p.ca[j][c], a1 = p.ca[j][c + 1];
				const C *Pa0 = ((a0 >> 1) == rank ? Pq : Pr), *Pa1 = ((a1 >> 1) == rank ? Pq : Pr);
				const float c0 = (float)p.ccoef[j][c], c1 = (float)p.ccoef[j][c + 1];
				float acc[8];
				tmem_ld8r(TM::addr(tbase, q), acc);
				tmem_wait_ld();
#pragma unroll
				for (int e = 0; e < 8; e++) {
					const int n = G::at(line, Lp::out_pos(tau, e));
					const C v0 = Pa0[n], v1 = Pa1[n];
					const float p0 = (a0 & 1) ? v0.y : v0.x, p1 = (a1 & 1) ? v1.y : v1.x;
					acc[e] += c0 * (p0 * x[e].x) + c1 * (p1 * x[e].y);
				}
				tmem_st8r(TM::addr(tbase, q), acc);
				tmem_wait_st();
				// no barrier here, as in k_i3p
			}
		}
		push_release();                                      // the own P grid is read by the copy before it changes
		cluster.sync();
	}
#pragma unroll 1
	for (int q = 0; q < 2; q++) {
		float acc[8];
		tmem_ld8r(TM::addr(tbase, q), acc);
		tmem_wait_ld();
		C *o = p.out + ((cell * p.nchunk + chunk) * 4 + 2 * rank + q) * (long)P * P + line * P;
#pragma unroll
		for (int e = 0; e < 8; e++) o[Lp::out_pos(tau, e)] = mk<C>(acc[e], 0.0);
	}
	tmem_fence_before();
	__syncthreads();
	tmem_fence_after();
	if (warp == 0) tmem_dealloc(tbase, TM::ALLOC);
}

// ---------------------------------------------------------------------------
// K5: out[b] = FFT2(sum_{k<nparts} in[b*grid_stride + k*part_stride]) (full grids)
template <class C> struct FullParamsT {
	const C *in; long grid_stride, part_stride; int nparts;
	C *out;   // [b][P*P]
};
using FullParams = FullParamsT<double2>;

template <int P, class C>
__global__ void __launch_bounds__(Geo<P>::NT) k_fft_full(const FullParamsT<C> p) {
	using G = Geo<P, C>;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *S = reinterpret_cast<C *>(smem_raw), *tw = S + G::GRID;
	init_twiddles<P>(tw);
	const long b = blockIdx.x;
	const C *in = p.in + b * p.grid_stride;
	for (int i = threadIdx.x; i < P * P; i += G::NT) {
		C s = in[i];
		for (int k = 1; k < p.nparts; k++) s = cadd(s, in[k * p.part_stride + i]);
		S[G::at(i / P, i % P)] = s;
	}
	__syncthreads();
	fft2_smem<P, -1>(S, tw);
	smem_to_global<P>(p.out + b * (long)P * P, S);
}

// ---------------------------------------------------------------------------
// K6: assembly of Cc and Cd for one (cell, component j):
//   Zcc_j = Wh_h . FS_g - Wh_g . FS_h          ((g,h) = (2,3),(3,1),(1,2); upstream collision.c:232-253)
//   Zcd_j = s2 (-Wh_j + d_j0) . Q - eta2_j s1 X_j
//         + s1 (eta2_j Wh_0 . FS4_j + 2 Wh_j . FS4_0) - d_j0 2 s1 sum_c Wh_c . FS4_c   (collision.c:95-167)
//   Cc_j = s1 Extract(IFFT2(Zcc_j)), Cd_j = Extract(IFFT2(Zcd_j))
// The spectra and transforms are in the working precision C; Cc and Cd are
// widened to FP64 for the outputs.  mode 0 writes Cc and Cd; mode 1 writes
// base + dtc (Cc + Cd + CB) in FP64 with the magnetic rotation CB of `wcur`
// (upstream simulation.c:75-135).
template <class C> struct AsmParamsT {
	const C *What;                    // [cell][4][P*P]
	const C *FS;                      // [cell][3][P*P]  FFT2 of the Cc sums S_1..S_3, or null
	const C *FS4;                     // [cell][4][P*P]  FFT2 of the I4 sums, or null
	const C *Qp; int nq;              // [cell][4][nq][P*P] I2 partials, or null
	const C *Xp; int nx;              // [cell][nx][4][P*P] I3 partials, or null
	TermRanges xrg;                   // xrg.nslots > 0: Xp holds [slot][4][P*P] partials of term ranges
	double s1, s2;
	int mode;
	double2 *out_cc, *out_cd;         // mode 0: [cell][4][N*N] (either may be null)
	const double2 *base, *wcur;       // mode 1: [cell][4][N*N]; base may be null (= 0)
	const double *B; double dtc;      // B: [cell][3], or null (no magnetic field)
	double2 *out;                     // mode 1
};
using AsmParams = AsmParamsT<double2>;

template <int P, class C>
__global__ void __launch_bounds__(Geo<P>::NT) k_assemble(const AsmParamsT<C> p) {
	using G = Geo<P, C>;
	using R = typename CT<C>::R;
	constexpr int N = G::N, NN = N * N, PP = P * P;
	constexpr int PER = (NN + G::NT - 1) / G::NT;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *S = reinterpret_cast<C *>(smem_raw), *tw = S + G::GRID;
	const int j = blockIdx.x & 3;
	const long cell = blockIdx.x >> 2;
	init_twiddles<P>(tw);
	const R eta2[4] = { 2, -2, -2, -2 };
	const R s1 = (R)p.s1, s2 = (R)p.s2;
	const C *Wh = p.What + cell * 4 * PP;
	double2 cc[PER], cd[PER];
#pragma unroll
	for (int u = 0; u < PER; u++) { cc[u] = czero(); cd[u] = czero(); }

	// --- Cc ---
	if (p.FS != nullptr && j > 0) {
		const int gi = (j % 3) + 1, hi = ((j + 1) % 3) + 1;    // j=1:(2,3) j=2:(3,1) j=3:(1,2)
		const C *FS = p.FS + cell * 3 * PP;
		for (int i = threadIdx.x; i < PP; i += G::NT) {
			const C z = csub(cmul(Wh[hi * PP + i], FS[(gi - 1) * PP + i]), cmul(Wh[gi * PP + i], FS[(hi - 1) * PP + i]));
			S[G::at(i / P, i % P)] = z;
		}
		__syncthreads();
		fft2_smem<P, +1>(S, tw);
#pragma unroll
		for (int u = 0; u < PER; u++) {
			const int q = threadIdx.x + u * G::NT;
			if (q < NN) {
				const C v = S[G::at(G::pad(q / N), G::pad(q % N))];
				cc[u] = make_double2(p.s1 * (double)v.x, p.s1 * (double)v.y);
			}
		}
		__syncthreads();
	}
	// --- Cd ---
	if (p.FS4 != nullptr || p.Qp != nullptr || p.Xp != nullptr) {
		for (int i = threadIdx.x; i < PP; i += G::NT) {
			C z = czero<C>();
			if (p.Qp != nullptr) {
				C q = czero<C>();
				for (int ii = 0; ii < 4; ii++) {
					const C *Q = p.Qp + ((cell * 4 + ii) * p.nq) * (long)PP + i;
					C s = czero<C>();
					for (int k = 0; k < p.nq; k++) s = cadd(s, Q[(long)k * PP]);
					q.x += eta2[ii] * s.x; q.y += eta2[ii] * s.y;
				}
				C h; h.x = -Wh[j * PP + i].x; h.y = -Wh[j * PP + i].y;
				if (j == 0) h.x += (R)1.0;
				const C v = cmul(h, q);
				z.x += s2 * v.x; z.y += s2 * v.y;
			}
			if (p.Xp != nullptr) {
				C s = czero<C>();
				if (p.xrg.nslots > 0) {
					const TermRanges &g = p.xrg;
					const int k0 = g.cluster_of(cell * (long)g.nterms), k1 = g.cluster_of((cell + 1) * (long)g.nterms - 1);
					for (int k = k0; k <= k1; k++)
						s = cadd(s, p.Xp[(((long)k * g.maxc + (cell - g.first_cell(k))) * 4 + j) * (long)PP + i]);
				} else {
					for (int k = 0; k < p.nx; k++) s = cadd(s, p.Xp[((cell * p.nx + k) * 4 + j) * (long)PP + i]);
				}
				z.x -= eta2[j] * s1 * s.x; z.y -= eta2[j] * s1 * s.y;
			}
			if (p.FS4 != nullptr) {
				const C *F4 = p.FS4 + cell * 4 * PP;
				C v = cadd(cscale(cmul(Wh[i], F4[j * PP + i]), eta2[j]), cscale(cmul(Wh[j * PP + i], F4[i]), (R)2.0));
				if (j == 0) {
					C s = czero<C>();
					for (int c = 0; c < 4; c++) s = cadd(s, cmul(Wh[c * PP + i], F4[c * PP + i]));
					v = csub(v, cscale(s, (R)2.0));
				}
				z.x += s1 * v.x; z.y += s1 * v.y;
			}
			S[G::at(i / P, i % P)] = z;
		}
		__syncthreads();
		fft2_smem<P, +1>(S, tw);
#pragma unroll
		for (int u = 0; u < PER; u++) {
			const int q = threadIdx.x + u * G::NT;
			if (q < NN) {
				const C v = S[G::at(G::pad(q / N), G::pad(q % N))];
				cd[u] = make_double2((double)v.x, (double)v.y);
			}
		}
	}
	// --- outputs (FP64) ---
#pragma unroll
	for (int u = 0; u < PER; u++) {
		const int q = threadIdx.x + u * G::NT;
		if (q >= NN) continue;
		const long o = (cell * 4 + j) * NN + q;
		if (p.mode == 0) {
			if (p.out_cc) p.out_cc[o] = cc[u];
			if (p.out_cd) p.out_cd[o] = cd[u];
		} else {
			const double2 *w = p.wcur + cell * 4 * NN + q;
			double2 cb = czero();          // -i [B, W] = 2 (B x w) . sigma
			if (p.B != nullptr) {        // null B: no magnetic field
				const double *B = p.B + cell * 3;
				if (j == 1) cb = make_double2(2 * (B[1] * w[3 * NN].x - B[2] * w[2 * NN].x), 2 * (B[1] * w[3 * NN].y - B[2] * w[2 * NN].y));
				if (j == 2) cb = make_double2(2 * (B[2] * w[1 * NN].x - B[0] * w[3 * NN].x), 2 * (B[2] * w[1 * NN].y - B[0] * w[3 * NN].y));
				if (j == 3) cb = make_double2(2 * (B[0] * w[2 * NN].x - B[1] * w[1 * NN].x), 2 * (B[0] * w[2 * NN].y - B[1] * w[1 * NN].y));
			}
			const double2 b = p.base ? p.base[o] : czero();      // null base: the right-hand side itself
			p.out[o] = make_double2(b.x + p.dtc * ((cc[u].x + cd[u].x) + cb.x), b.y + p.dtc * ((cc[u].y + cd[u].y) + cb.y));
		}
	}
}

// ---------------------------------------------------------------------------
// K7: velocity space -> Fourier space, one CTA per real N x N component:
//   FFT2 / N^2 with the Hermitian completion of upstream simulation.c:224-261
template <int N>
__global__ void __launch_bounds__(Len<N>::T * N) k_to_fourier(const double *__restrict__ Wv, double2 *__restrict__ Wf) {
	constexpr int T = Len<N>::T, LD = N + 1;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	double2 *S = reinterpret_cast<double2 *>(smem_raw), *tw = S + N * LD;
	init_twiddles<N>(tw);
	__syncthreads();
	const long b = blockIdx.x;
	const double *in = Wv + b * N * N;
	const int line = threadIdx.x / T, tau = threadIdx.x % T;
	double2 x[8];
#pragma unroll
	for (int r = 0; r < 8; r++) x[r] = make_double2(in[line * N + tau + T * r], 0.0);
	fft1d<N, -1>(x, tau, S + line * LD, 1, tw);
#pragma unroll
	for (int e = 0; e < 8; e++) S[line * LD + Len<N>::out_pos(tau, e)] = x[e];
	__syncthreads();
#pragma unroll
	for (int r = 0; r < 8; r++) x[r] = S[(tau + T * r) * LD + line];
	fft1d<N, -1>(x, tau, S + line, LD, tw);
#pragma unroll
	for (int e = 0; e < 8; e++) S[Len<N>::out_pos(tau, e) * LD + line] = x[e];
	__syncthreads();
	const double scale = 1.0 / (N * N);
	double2 *out = Wf + b * N * N;
	for (int i = threadIdx.x; i < N * N; i += T * N) {
		const int l = i / N, k = i % N;
		if (k <= N / 2) {
			const double2 v = S[l * LD + k];
			out[i] = make_double2(v.x * scale, v.y * scale);
		} else {
			const int lc = (N - l) % N, kc = N - k;
			const double2 v = S[lc * LD + kc];
			out[i] = make_double2(v.x * scale, -(v.y * scale));
		}
	}
}

// K8: Fourier space -> velocity space: backward FFT2, real part (simulation.c:270-283)
template <int N>
__global__ void __launch_bounds__(Len<N>::T * N) k_from_fourier(const double2 *__restrict__ Wf, double *__restrict__ Wv) {
	constexpr int T = Len<N>::T, LD = N + 1;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	double2 *S = reinterpret_cast<double2 *>(smem_raw), *tw = S + N * LD;
	init_twiddles<N>(tw);
	__syncthreads();
	const long b = blockIdx.x;
	const double2 *in = Wf + b * N * N;
	const int line = threadIdx.x / T, tau = threadIdx.x % T;
	double2 x[8];
#pragma unroll
	for (int r = 0; r < 8; r++) x[r] = in[line * N + tau + T * r];
	fft1d<N, +1>(x, tau, S + line * LD, 1, tw);
#pragma unroll
	for (int e = 0; e < 8; e++) S[line * LD + Len<N>::out_pos(tau, e)] = x[e];
	__syncthreads();
#pragma unroll
	for (int r = 0; r < 8; r++) x[r] = S[(tau + T * r) * LD + line];
	fft1d<N, +1>(x, tau, S + line, LD, tw);
#pragma unroll
	for (int e = 0; e < 8; e++) S[Len<N>::out_pos(tau, e) * LD + line] = x[e];
	__syncthreads();
	double *out = Wv + b * N * N;
	for (int i = threadIdx.x; i < N * N; i += T * N) out[i] = S[(i / N) * LD + (i % N)].x;
}

// K9: generic 2-D transform of n0 x n1 = L x L complex grids (FFTW-API plans).
// mode 0: c2c (in complex), mode 1: r2c (in real, out n0 x (L/2+1))
template <int L, int DIR>
__global__ void __launch_bounds__(Len<L>::T * L) k_fft2_generic(const void *__restrict__ in, double2 *__restrict__ out, int r2c) {
	constexpr int T = Len<L>::T, LD = L + 1;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	double2 *S = reinterpret_cast<double2 *>(smem_raw), *tw = S + L * LD;
	init_twiddles<L>(tw);
	__syncthreads();
	const int line = threadIdx.x / T, tau = threadIdx.x % T;
	double2 x[8];
#pragma unroll
	for (int r = 0; r < 8; r++) {
		const int i = line * L + tau + T * r;
		x[r] = r2c ? make_double2(((const double *)in)[i], 0.0) : ((const double2 *)in)[i];
	}
	fft1d<L, DIR>(x, tau, S + line * LD, 1, tw);
#pragma unroll
	for (int e = 0; e < 8; e++) S[line * LD + Len<L>::out_pos(tau, e)] = x[e];
	__syncthreads();
#pragma unroll
	for (int r = 0; r < 8; r++) x[r] = S[(tau + T * r) * LD + line];
	fft1d<L, DIR>(x, tau, S + line, LD, tw);
#pragma unroll
	for (int e = 0; e < 8; e++) S[Len<L>::out_pos(tau, e) * LD + line] = x[e];
	__syncthreads();
	if (r2c) {
		constexpr int H = L / 2 + 1;
		for (int i = threadIdx.x; i < L * H; i += T * L) out[i] = S[(i / H) * LD + (i % H)];
	} else {
		for (int i = threadIdx.x; i < L * L; i += T * L) out[i] = S[(i / L) * LD + (i % L)];
	}
}

}  // namespace qb
