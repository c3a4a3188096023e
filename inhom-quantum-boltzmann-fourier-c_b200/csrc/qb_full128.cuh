// qb_full128.cuh — the I3 sums at N = 64 in the FP32 precision form, with
// each padded 128 x 128 grid whole in one CTA's shared memory.
//
// An FP32 complex grid of 128 x 128 is 128 KB, so unlike FP64 it fits one CTA:
// both dimensions of a transform are local, and an I3 chain
//   X_j += eta_i P_i . FFT2(psi2_t . IFFT2(W^_i . P_j))
// (upstream I3integral, src/integrals.c:283-379, summed over the quadrature
// terms inside the outer transforms) is a row pass, a column pass (inverse
// transform by decimation in frequency, psi2, forward transform by decimation
// in time, all in registers) and a row pass, with two CTA barriers and no
// exchange between CTAs.  The 4 components of a (cell, chunk) run on a
// 2-CTA cluster: CTA r computes the spectra P_{t,c} = FFT2(Pad(psi1_t . W_c))
// of its components 2r, 2r + 1 into a scratch grid in global memory (L2);
// after a cluster barrier it runs the 8 chains of its two outputs, reading
// W^_i, P_j and P_a from L2 and accumulating in tensor memory.
//
// Shared-memory grid: natural order, row pitch 129, the column index XOR-ed
// by 8 when exactly one of (row, column) is in the upper half:
//   slot(l, k) = 129 l + (k ^ 8 ((l >> 6) ^ (k >> 6)))
// With 8-byte values a half-warp spans one line (16 lanes); the pitch makes
// the column accesses conflict-free and the XOR separates the two 64-point
// halves that the in-line exchange of a 128-point transform visits together.
//
// Global layouts: W^ and the outputs are in the B layout of the N = 64 kernels
// (natural row l stored at row 64 (l & 1) + l / 2); P scratch is natural.
#pragma once
#include "qb_split128.cuh"

namespace qb {

struct F128 {
	static constexpr int P = 128, N = 64, LDP = 129, NT = 512, GRID = P * LDP;
	__device__ __forceinline__ static int at(int l, int k) { return l * LDP + (k ^ ((((l >> 6) ^ (k >> 6)) & 1) << 3)); }
	__device__ __forceinline__ static int src(int p) { return p < N / 2 ? p : (p >= 3 * N / 2 ? p - N : -1); }
	// offset of natural row l of a B-layout grid
	__device__ __forceinline__ static long brow(int l) { return (long)(64 * (l & 1) + (l >> 1)) * P; }
};

// slots of a line of the shared grid as a transform scratch: one 64-point
// half.  Within half h of row l the swizzle is one XOR of the position with
// 8 ((l >> 6) ^ h); within half h of column k it is a constant column offset.
template <class C> struct RowHalf {
	C *S; int base, m;                         // base = 129 l + 64 h, m = 8 ((l >> 6) ^ h)
	__device__ __forceinline__ RowHalf(C *S_, int row, int h) : S(S_), base(row * F128::LDP + 64 * h), m((((row >> 6) ^ h) & 1) << 3) {}
	__device__ __forceinline__ C &operator()(int pos) const { return S[base + (pos ^ m)]; }
};
template <class C> struct ColHalf {
	C *S; int base;                            // base = 129 * 64 h + (k ^ 8 (h ^ (k >> 6)))
	__device__ __forceinline__ ColHalf(C *S_, int col, int h) : S(S_), base(64 * h * F128::LDP + (col ^ ((((col >> 6) ^ h) & 1) << 3))) {}
	__device__ __forceinline__ C &operator()(int pos) const { return S[base + pos * F128::LDP]; }
};

// slots of the 8 inputs (positions tau + 16 r) and outputs (positions
// pos128(tau, e)) of lane tau on a row or column of the shared grid: the
// swizzle depends only on which half a position is in (r / 4, e / 4)
struct LineSlots {
	int in[2], out[2], step, cx[2];            // cx: a column's swizzled index in the lower / upper half (columns only)
	__device__ __forceinline__ int at_in(int r) const { return in[r >> 2] + step * r; }
	__device__ __forceinline__ int at_out(int e) const { return out[e >> 2] + step * e; }
};
__device__ __forceinline__ LineSlots row_slots(int row, int tau) {
	const int p0 = 2 * (tau & 7) + (tau >> 3), rb = row * F128::LDP, m = ((row >> 6) & 1) << 3;
	LineSlots L;
	L.in[0] = rb + (tau ^ m); L.in[1] = rb + (tau ^ m ^ 8);
	L.out[0] = rb + (p0 ^ m); L.out[1] = rb + (p0 ^ m ^ 8);
	L.step = 16;
	L.cx[0] = L.cx[1] = 0;
	return L;
}
__device__ __forceinline__ LineSlots col_slots(int col, int tau) {
	const int p0 = 2 * (tau & 7) + (tau >> 3), c0 = col ^ (((col >> 6) & 1) << 3), c1 = c0 ^ 8;
	LineSlots L;
	L.in[0] = tau * F128::LDP + c0; L.in[1] = tau * F128::LDP + c1;
	L.out[0] = p0 * F128::LDP + c0; L.out[1] = p0 * F128::LDP + c1;
	L.step = 16 * F128::LDP;
	L.cx[0] = c0; L.cx[1] = c1;
	return L;
}

// fft128 with the line given as row (ROW) or column `line` of the shared grid
template <int DIR, bool ROW, class C>
__device__ __forceinline__ void fft128_line(C (&x)[8], int tau, C *S, int line, const C *tw128, const C (&wp)[8]) {
	const int h = tau >> 3;
	C u[4], v[4];
#pragma unroll
	for (int r = 0; r < 4; r++) {
		C w = tw128[tau + 16 * r];
		if (DIR > 0) w.y = -w.y;
		u[r] = cadd(x[r], x[r + 4]);
		v[r] = cmul(csub(x[r], x[r + 4]), w);
	}
#pragma unroll
	for (int r = 0; r < 4; r++) {
		const C send = h ? u[r] : v[r];
		const C recv = shfl_xor_c(send, 8);
		x[2 * r] = h ? recv : u[r];
		x[2 * r + 1] = h ? v[r] : recv;
	}
	if constexpr (ROW) fft1d_accw<64, DIR>(x, tau & 7, RowHalf<C>(S, line, h), wp);
	else fft1d_accw<64, DIR>(x, tau & 7, ColHalf<C>(S, line, h), wp);
}

// 128-point transform by decimation in time of a column whose lane tau holds
// the samples at rows pos128(tau, e) (the output order of fft128_line):
// lanes 0-7 hold the even samples 2m, lanes 8-15 the odd ones, m = (tau & 7) +
// 8 e, which is the input order of fft1d<64> on each half.  After the two
// 64-point transforms E and O, the butterfly Z[k] = E[k] + w^k O[k],
// Z[k + 64] = E[k] - w^k O[k] is split between the lane pair: lanes 0-7 take
// k = (tau & 7) + 16 j, lanes 8-15 k = (tau & 7) + 16 j + 8, one shuffle of four
// values each way.  Output i of lane tau is Z[dpos128(tau, i)].  Applied after
// fft128_line it needs no reordering in between.
__device__ __forceinline__ int dpos128(int tau, int i) { return (tau & 7) + 16 * (i >> 1) + 8 * (tau >> 3) + 64 * (i & 1); }

template <int DIR, class C>
__device__ __forceinline__ void fft128_dit_col(C (&x)[8], int tau, C *S, int col, const C *tw128, const C (&wp)[8]) {
	const int h = tau >> 3, t = tau & 7;
	fft1d_accw<64, DIR>(x, t, ColHalf<C>(S, col, h), wp);
	C y[8];
#pragma unroll
	for (int j = 0; j < 4; j++) {
		const C send = h ? x[2 * j] : x[2 * j + 1];
		const C recv = shfl_xor_c(send, 8);
		const C E = h ? recv : x[2 * j], O = h ? x[2 * j + 1] : recv;
		C w = tw128[t + 16 * j + 8 * h];
		if (DIR > 0) w.y = -w.y;
		const C wo = cmul(w, O);
		y[2 * j] = cadd(E, wo);
		y[2 * j + 1] = csub(E, wo);
	}
#pragma unroll
	for (int i = 0; i < 8; i++) x[i] = y[i];
}

// tensor-memory accumulators: 2 outputs x 4 row iterations x 8 values per
// thread; the four warps of a lane quarter split the 512 columns
struct F128Tmem {
	static constexpr unsigned PER_THREAD = 2 * 4 * 8 * 2;     // 128 (FP32)
	static constexpr unsigned NCOLS = 4 * PER_THREAD;         // 512
	__device__ __forceinline__ static unsigned addr(unsigned base, int q, int it, int e) {
		const unsigned w = threadIdx.x >> 5;
		return base + ((32u * (w & 3u)) << 16) + (w >> 2) * PER_THREAD + (unsigned)((q * 4 + it) * 8 + e) * 2;
	}
};

// Ghat: B layout; pscr: [cluster][4][P*P] natural; out: [cell][chunk][4][P*P] B layout.
// kind: null (every cell) or the per-cell form of k_nyquist_kind; this kernel
// then takes the cells of kind 1 (the real form k_i3_full128r takes kind 0).
template <class C>
__global__ void __launch_bounds__(F128::NT, 1) k_i3_full128(const I3ParamsT<C> p, C *pscr, const int *kind) {
	static_assert(sizeof(C) == 8, "the whole-grid form is FP32 only");
	using F = F128;
	using R = typename CT<C>::R;
	using TM = F128Tmem;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	__shared__ unsigned tmem_slot;
	C *S = reinterpret_cast<C *>(smem_raw), *tw128 = S + F::GRID, *tw64 = tw128 + 128;
	cg::cluster_group cl = cg::this_cluster();
	const int rank = (int)cl.block_rank();
	const long cid = blockIdx.x / 2;
	const int chunk = (int)(cid % p.nchunk);
	const long cell = cid / p.nchunk;
	if (kind != nullptr && kind[cell] != 1) return;     // both CTAs of the cluster leave before any barrier
	const int tid = threadIdx.x, warp = tid >> 5, tau = tid & 15, sub = tid >> 4;   // line it * 32 + sub
	if (warp == 0) tmem_alloc(&tmem_slot, TM::NCOLS);
	init_tw128(tw128, tw64);
	tmem_fence_before();
	__syncthreads();
	tmem_fence_after();
	const unsigned tbase = tmem_slot;
	// the 64-point twiddle powers of this lane, w64^((tau & 7) q), for every transform of the kernel
	C wp[8];
	wp[0] = tw64[0];
#pragma unroll
	for (int q = 1; q < 8; q++) wp[q] = tw64[((tau & 7) * q) & 63];
#pragma unroll 1
	for (int q = 0; q < 2; q++)
#pragma unroll 1
		for (int it = 0; it < 4; it++)
#pragma unroll
			for (int e = 0; e < 8; e++) tmem_st(TM::addr(tbase, q, it, e), czero<C>());
	tmem_wait_st();
	C *Pall = pscr + cid * 4 * (long)F::P * F::P;
	const C *Gcell = p.Ghat + cell * p.g_cell;
	const int t0 = (int)((long)chunk * p.nterms / p.nchunk), t1 = (int)((long)(chunk + 1) * p.nterms / p.nchunk);
#pragma unroll 1
	for (int t = t0; t < t1; t++) {
		// spectra of components 2 rank + q (sign -1), natural layout, to L2
#pragma unroll 1
		for (int q = 0; q < 2; q++) {
			const int comp = 2 * rank + q;
			const double2 *src = p.src + cell * p.src_cell + (long)p.src_comp[comp] * F::N * F::N;
			const C *psi1 = p.psi1 + (long)t * F::N * F::N;
#pragma unroll 1
			for (int it = 0; it < 4; it += 3) {             // rows outside the zero band: 0..31, 96..127
				const int row = it * 32 + sub, ls = F::src(row);
				C x[8];
#pragma unroll
				for (int r = 0; r < 8; r++) {
					const int ks = F::src(tau + 16 * r);
					C v = czero<C>();
					if (ks >= 0) {
						const int idx = ks + F::N * ls;
						const double2 w = src[idx];
						v = cmul(psi1[idx], mk<C>(w.x, w.y));
					}
					x[r] = v;
				}
				fft128_line<-1, true>(x, tau, S, row, tw128, wp);
				const LineSlots ls_ = row_slots(row, tau);
#pragma unroll
				for (int e = 0; e < 8; e++) S[ls_.at_out(e)] = x[e];
			}
			__syncthreads();
#pragma unroll 1
			for (int it = 0; it < 4; it++) {
				const int col = it * 32 + sub;
				const LineSlots cs_ = col_slots(col, tau);
				C x[8];
#pragma unroll
				for (int r = 0; r < 8; r++)                     // rows tau + 16 r; 32..95 are the zero band
					x[r] = (r >= 2 && r < 6) ? czero<C>() : S[cs_.at_in(r)];
				fft128_line<-1, false>(x, tau, S, col, tw128, wp);
#pragma unroll
				for (int e = 0; e < 8; e++) S[cs_.at_out(e)] = x[e];
			}
			__syncthreads();
			C *Pq = Pall + (long)comp * F::P * F::P;
#pragma unroll 4
			for (int i = tid; i < F::P * F::P; i += F::NT) Pq[i] = S[F::at(i >> 7, i & 127)];
			__syncthreads();
		}
		cl.sync();                                          // both CTAs' spectra of term t are in L2
		const R *psi2 = p.psi2T + (long)p.psi2_idx[t] * F::P * F::P;
		const R sc = (R)p.psi2_scale[t];
#pragma unroll 1
		for (int q = 0; q < 2; q++) {
			const int j = 2 * rank + q;
			const C *Pj = Pall + (long)j * F::P * F::P;
#pragma unroll 1
			for (int cmb = 0; cmb < p.ncombo[j]; cmb++) {
				const C *Gg = Gcell + (long)p.cgi[j][cmb] * F::P * F::P;
				// rows: inverse transform along k of W^_i . P_j
#pragma unroll 1
				for (int it = 0; it < 4; it++) {
					const int row = it * 32 + sub;
					const C *g = Gg + F::brow(row), *pj = Pj + (long)row * F::P;
					C x[8];
#pragma unroll
					for (int r = 0; r < 8; r++) x[r] = cmul(g[tau + 16 * r], pj[tau + 16 * r]);
					fft128_line<+1, true>(x, tau, S, row, tw128, wp);
					const LineSlots ls_ = row_slots(row, tau);
#pragma unroll
					for (int e = 0; e < 8; e++) S[ls_.at_out(e)] = x[e];
				}
				__syncthreads();
				// columns: inverse transform along l, psi2, forward transform
#pragma unroll 1
				for (int it = 0; it < 4; it++) {
					const int col = it * 32 + sub;
					const LineSlots cs_ = col_slots(col, tau);
					C x[8];
#pragma unroll
					for (int r = 0; r < 8; r++) x[r] = S[cs_.at_in(r)];
					fft128_line<+1, false>(x, tau, S, col, tw128, wp);
					const R *ps = psi2 + (long)col * F::P;
#pragma unroll
					for (int e = 0; e < 8; e++) {
						const R f = sc * ps[pos128(tau, e)];
						x[e].x *= f;
						x[e].y *= f;
					}
					fft128_dit_col<-1>(x, tau, S, col, tw128, wp);
					const int d0 = (tau & 7) + 8 * (tau >> 3);   // rows d0 + 16 (i / 2) + 64 (i % 2)
#pragma unroll
					for (int i = 0; i < 8; i++) S[(d0 + 16 * (i >> 1) + 64 * (i & 1)) * F::LDP + cs_.cx[i & 1]] = x[i];
				}
				__syncthreads();
				// rows: forward transform along k, times P_a, accumulate
				const int a = p.ca[j][cmb];
				const C *Pa = Pall + (long)a * F::P * F::P;
				const R coef = (R)p.ccoef[j][cmb];
#pragma unroll 1
				for (int it = 0; it < 4; it++) {
					const int row = it * 32 + sub;
					const LineSlots ls_ = row_slots(row, tau);
					C x[8];
#pragma unroll
					for (int r = 0; r < 8; r++) x[r] = S[ls_.at_in(r)];
					fft128_line<-1, true>(x, tau, S, row, tw128, wp);
					const C *pa = Pa + (long)row * F::P;
					C acc[8];
					tmem_ld8(TM::addr(tbase, q, it, 0), acc);
					tmem_wait_ld();
#pragma unroll
					for (int e = 0; e < 8; e++) {
						const C v = cmul(pa[pos128(tau, e)], x[e]);
						acc[e].x += coef * v.x;
						acc[e].y += coef * v.y;
					}
					tmem_st8(TM::addr(tbase, q, it, 0), acc);
					tmem_wait_st();
				}
				// no barrier: the next chain's first row pass writes only the
				// rows this thread's 16-lane group has just read
			}
		}
		cl.sync();                                          // the partner is done with this term's spectra
	}
#pragma unroll 1
	for (int q = 0; q < 2; q++) {
		C *o = p.out + ((cell * p.nchunk + chunk) * 4 + 2 * rank + q) * (long)F::P * F::P;
#pragma unroll 1
		for (int it = 0; it < 4; it++) {
			const int row = it * 32 + sub;
			C acc[8];
			tmem_ld8(TM::addr(tbase, q, it, 0), acc);
			tmem_wait_ld();
#pragma unroll
			for (int e = 0; e < 8; e++) o[F::brow(row) + pos128(tau, e)] = acc[e];
		}
	}
	tmem_fence_before();
	__syncthreads();
	tmem_fence_after();
	if (warp == 0) tmem_dealloc(tbase, TM::NCOLS);
}


// ---------------------------------------------------------------------------
// Real form of the same sums.
//
// Let Pad(X) be Hermitian, Pad(X)(-k) = conj Pad(X)(k) on the 128 x 128
// frequency grid.  Then its forward transform is real.  Pad(W_c) and
// Pad(psi1_t . W_c) are Hermitian up to the Nyquist row and column of W_c:
// the N x N Fourier state of a real velocity-space component is Hermitian,
// psi1_t = exp(i a_t . k) is too, and padding keeps every pair (k, -k) except
// k = -N/2 (stored at 3N/2), whose partner +N/2 is not on the padded grid.
// So when the Nyquist content of W is negligible, W^_i and P_{t,c} are real
// and so is every chain input a = W^_i . P_j.  psi2_t is real and even, so
// a -> FFT2(psi2_t . IFFT2(a)) maps real grids to real grids.  Two chains
// therefore share one complex transform, one in the real part and one in
// the imaginary part, and the spectra of two components come out of one
// transform of psi1_t . (W_a + i W_b).  That halves the transforms of the
// complex kernel.
//
// What is dropped: the imaginary parts of W^ and P, which come from the
// Nyquist entries only.  The sums move by at most about the Nyquist fraction
// (sum of |W| on the Nyquist row and column over sum of |W|, all 4
// components): 0.2-0.3 of it on the extracted I3 of Gaussian-mixture states at
// N = 64, 0.5-1.1 of it on the raw sums at N = 16.  k_nyquist_kind marks each
// cell against a bound (1e-6 in the engine); cells above it go to the complex
// kernel, so the error this form adds stays at the FP32 rounding of the
// precision form.
//
// pscr: [cluster][4][P*P] real, natural order; out as k_i3_full128 (real
// parts; imaginary parts written as zero).
struct F128TmemR {
	static constexpr unsigned PER_THREAD = 2 * 4 * 8;         // 64 (real FP32)
	static constexpr unsigned NCOLS = 4 * PER_THREAD;         // 256
	__device__ __forceinline__ static unsigned addr(unsigned base, int q, int it) {
		const unsigned w = threadIdx.x >> 5;
		return base + ((32u * (w & 3u)) << 16) + (w >> 2) * PER_THREAD + (unsigned)(q * 4 + it) * 8;
	}
};

__global__ void __launch_bounds__(F128::NT, 1) k_i3_full128r(const I3ParamsT<float2> p, float *pscr, const int *kind) {
	using C = float2;
	using F = F128;
	using TM = F128TmemR;
	constexpr long PP = (long)F::P * F::P;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	__shared__ unsigned tmem_slot;
	C *S = reinterpret_cast<C *>(smem_raw), *tw128 = S + F::GRID, *tw64 = tw128 + 128;
	cg::cluster_group cl = cg::this_cluster();
	const int rank = (int)cl.block_rank();
	const long cid = blockIdx.x / 2;
	const int chunk = (int)(cid % p.nchunk);
	const long cell = cid / p.nchunk;
	if (kind[cell] != 0) return;                          // both CTAs of the cluster leave before any barrier
	const int tid = threadIdx.x, warp = tid >> 5, tau = tid & 15, sub = tid >> 4;
	if (warp == 0) tmem_alloc(&tmem_slot, TM::NCOLS);
	init_tw128(tw128, tw64);
	tmem_fence_before();
	__syncthreads();
	tmem_fence_after();
	const unsigned tbase = tmem_slot;
	C wp[8];
	wp[0] = tw64[0];
#pragma unroll
	for (int q = 1; q < 8; q++) wp[q] = tw64[((tau & 7) * q) & 63];
	{
		const float z[8] = { 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f };
#pragma unroll 1
		for (int q = 0; q < 2; q++)
#pragma unroll 1
			for (int it = 0; it < 4; it++) tmem_st8r(TM::addr(tbase, q, it), z);
	}
	tmem_wait_st();
	float *Pall = pscr + cid * 4 * PP;
	const C *Gcell = p.Ghat + cell * p.g_cell;
	const int t0 = (int)((long)chunk * p.nterms / p.nchunk), t1 = (int)((long)(chunk + 1) * p.nterms / p.nchunk);
#pragma unroll 1
	for (int t = t0; t < t1; t++) {
		// spectra of components 2 rank (real part) and 2 rank + 1 (imaginary part)
		{
			const double2 *sa = p.src + cell * p.src_cell + (long)p.src_comp[2 * rank] * F::N * F::N;
			const double2 *sb = p.src + cell * p.src_cell + (long)p.src_comp[2 * rank + 1] * F::N * F::N;
			const C *psi1 = p.psi1 + (long)t * F::N * F::N;
#pragma unroll 1
			for (int it = 0; it < 4; it += 3) {             // rows outside the zero band: 0..31, 96..127
				const int row = it * 32 + sub, ls = F::src(row);
				C x[8];
#pragma unroll
				for (int r = 0; r < 8; r++) {
					const int ks = F::src(tau + 16 * r);
					C v = czero<C>();
					if (ks >= 0) {
						const int idx = ks + F::N * ls;
						const double2 a = sa[idx], b = sb[idx];
						v = cmul(psi1[idx], mk<C>(a.x - b.y, a.y + b.x));
					}
					x[r] = v;
				}
				fft128_line<-1, true>(x, tau, S, row, tw128, wp);
				const LineSlots ls_ = row_slots(row, tau);
#pragma unroll
				for (int e = 0; e < 8; e++) S[ls_.at_out(e)] = x[e];
			}
			__syncthreads();
#pragma unroll 1
			for (int it = 0; it < 4; it++) {
				const int col = it * 32 + sub;
				const LineSlots cs_ = col_slots(col, tau);
				C x[8];
#pragma unroll
				for (int r = 0; r < 8; r++)
					x[r] = (r >= 2 && r < 6) ? czero<C>() : S[cs_.at_in(r)];
				fft128_line<-1, false>(x, tau, S, col, tw128, wp);
#pragma unroll
				for (int e = 0; e < 8; e++) S[cs_.at_out(e)] = x[e];
			}
			__syncthreads();
			float *Pa = Pall + (long)(2 * rank) * PP, *Pb = Pa + PP;
#pragma unroll 4
			for (int i = tid; i < F::P * F::P; i += F::NT) {
				const C v = S[F::at(i >> 7, i & 127)];
				Pa[i] = v.x;
				Pb[i] = v.y;
			}
		}
		cl.sync();                                          // both CTAs' spectra of term t are in L2
		const float *psi2 = p.psi2T + (long)p.psi2_idx[t] * PP;
		const float sc = (float)p.psi2_scale[t];
#pragma unroll 1
		for (int q = 0; q < 2; q++) {
			const int j = 2 * rank + q;
			const float *Pj = Pall + (long)j * PP;
#pragma unroll 1
			for (int cmb = 0; cmb + 1 < p.ncombo[j]; cmb += 2) {
				const C *G0 = Gcell + (long)p.cgi[j][cmb] * PP, *G1 = Gcell + (long)p.cgi[j][cmb + 1] * PP;
				// rows: inverse transform along k of (W^_i0 + i W^_i1) . P_j
#pragma unroll 1
				for (int it = 0; it < 4; it++) {
					const int row = it * 32 + sub;
					const C *g0 = G0 + F::brow(row), *g1 = G1 + F::brow(row);
					const float *pj = Pj + (long)row * F::P;
					C x[8];
#pragma unroll
					for (int r = 0; r < 8; r++) {
						const int n = tau + 16 * r;
						const float pv = pj[n];
						x[r] = mk<C>(pv * g0[n].x, pv * g1[n].x);
					}
					fft128_line<+1, true>(x, tau, S, row, tw128, wp);
					const LineSlots ls_ = row_slots(row, tau);
#pragma unroll
					for (int e = 0; e < 8; e++) S[ls_.at_out(e)] = x[e];
				}
				__syncthreads();
				// columns: inverse transform along l, psi2, forward transform
#pragma unroll 1
				for (int it = 0; it < 4; it++) {
					const int col = it * 32 + sub;
					const LineSlots cs_ = col_slots(col, tau);
					C x[8];
#pragma unroll
					for (int r = 0; r < 8; r++) x[r] = S[cs_.at_in(r)];
					fft128_line<+1, false>(x, tau, S, col, tw128, wp);
					const float *ps = psi2 + (long)col * F::P;
#pragma unroll
					for (int e = 0; e < 8; e++) {
						const float f = sc * ps[pos128(tau, e)];
						x[e].x *= f;
						x[e].y *= f;
					}
					fft128_dit_col<-1>(x, tau, S, col, tw128, wp);
					const int d0 = (tau & 7) + 8 * (tau >> 3);
#pragma unroll
					for (int i = 0; i < 8; i++) S[(d0 + 16 * (i >> 1) + 64 * (i & 1)) * F::LDP + cs_.cx[i & 1]] = x[i];
				}
				__syncthreads();
				// rows: forward transform along k; the real part belongs to i0,
				// the imaginary part to i1
				const float *P0 = Pall + (long)p.ca[j][cmb] * PP, *P1 = Pall + (long)p.ca[j][cmb + 1] * PP;
				const float c0 = (float)p.ccoef[j][cmb], c1 = (float)p.ccoef[j][cmb + 1];
#pragma unroll 1
				for (int it = 0; it < 4; it++) {
					const int row = it * 32 + sub;
					const LineSlots ls_ = row_slots(row, tau);
					C x[8];
#pragma unroll
					for (int r = 0; r < 8; r++) x[r] = S[ls_.at_in(r)];
					fft128_line<-1, true>(x, tau, S, row, tw128, wp);
					const float *p0 = P0 + (long)row * F::P, *p1 = P1 + (long)row * F::P;
					float acc[8];
					tmem_ld8r(TM::addr(tbase, q, it), acc);
					tmem_wait_ld();
#pragma unroll
					for (int e = 0; e < 8; e++) {
						const int n = pos128(tau, e);
						acc[e] += c0 * (p0[n] * x[e].x) + c1 * (p1[n] * x[e].y);
					}
					tmem_st8r(TM::addr(tbase, q, it), acc);
					tmem_wait_st();
				}
				// no barrier: the next chain's first row pass writes only the
				// rows this thread's 16-lane group has just read
			}
		}
		cl.sync();                                          // the partner is done with this term's spectra
	}
#pragma unroll 1
	for (int q = 0; q < 2; q++) {
		C *o = p.out + ((cell * p.nchunk + chunk) * 4 + 2 * rank + q) * PP;
#pragma unroll 1
		for (int it = 0; it < 4; it++) {
			const int row = it * 32 + sub;
			float acc[8];
			tmem_ld8r(TM::addr(tbase, q, it), acc);
			tmem_wait_ld();
#pragma unroll
			for (int e = 0; e < 8; e++) o[F::brow(row) + pos128(tau, e)] = mk<C>(acc[e], 0.0);
		}
	}
	tmem_fence_before();
	__syncthreads();
	tmem_fence_after();
	if (warp == 0) tmem_dealloc(tbase, TM::NCOLS);
}

// per cell: 0 (real form) when both
//   - the Nyquist content of the Fourier state W ([cell][4][N*N], natural
//     order k + N l; Nyquist = row l = N/2 and column k = N/2), and
//   - its anti-Hermitian part, sum of |W(k) - conj W(-k)| over the other
//     entries (nonzero when a velocity-space component is not real)
// are at most `bound` times the total (sums of |W| over the 4 components),
// else 1 (complex kernel).  stats (may be null) counts the cells of kind 0
// and all cells.
constexpr int kNyqThreads = 256;
__global__ void __launch_bounds__(kNyqThreads) k_nyquist_kind(int N, const double2 *__restrict__ W, double bound, int *__restrict__ kind,
                                                             unsigned long long *stats) {
	__shared__ double red[3][kNyqThreads / 32];
	const long NN = (long)N * N;
	const double2 *w = W + blockIdx.x * 4 * NN;
	double tot = 0.0, nyq = 0.0, anti = 0.0;
	for (long i = threadIdx.x; i < 4 * NN; i += kNyqThreads) {
		const long c = i / NN;
		const int g = (int)(i % NN), k = g % N, l = g / N;
		const double2 v = w[i];
		const double a = hypot(v.x, v.y);
		tot += a;
		if (k == N / 2 || l == N / 2) {
			nyq += a;
		} else {
			const int kc = (N - k) % N, lc = (N - l) % N;
			const double2 p = w[c * NN + kc + (long)N * lc];
			anti += hypot(v.x - p.x, v.y + p.y);
		}
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		tot += __shfl_xor_sync(0xffffffffu, tot, o);
		nyq += __shfl_xor_sync(0xffffffffu, nyq, o);
		anti += __shfl_xor_sync(0xffffffffu, anti, o);
	}
	if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = tot; red[1][threadIdx.x >> 5] = nyq; red[2][threadIdx.x >> 5] = anti; }
	__syncthreads();
	if (threadIdx.x == 0) {
		double t = 0.0, n = 0.0, h = 0.0;
		for (int i = 0; i < kNyqThreads / 32; i++) { t += red[0][i]; n += red[1][i]; h += red[2][i]; }
		const int k = (n <= bound * t && h <= bound * t) ? 0 : 1;     // NaN sums take the complex kernel
		kind[blockIdx.x] = k;
		if (stats != nullptr) {
			atomicAdd(&stats[0], (unsigned long long)(k == 0));
			atomicAdd(&stats[1], 1ull);
		}
	}
}

}  // namespace qb
