// qb_anyn.cu — the collision operator at grid sizes that have no fixed-size
// kernels: N with 2N = 2^a 3^b up to N = 128, i.e. N = 24, 48, 96 (radix-3
// transforms) and N = 128 (256 x 256 padded grids), in FP64 or the FP32 form.
//
// The sums are those of the fixed-size engine (qb_kernels.cuh), factored the
// same way:
//   spectra  W^_c  = FFT2(Pad(W_c))
//   I1 / I4  S_g   = sum_t phi_t . IFFT2(F . FFT2(Pad(psi2_t . g)))       F = fa W^_f + fb
//   I2       Q_i   = sum_t FFT2(Pad(psi1_t . W_i)) . FFT2(Pad(psi2_t . W_i))
//   I3       X_j   = sum_t sum_i eta_i P_i . FFT2(psi2_t . IFFT2(W^_i . P_j)),  P_j = FFT2(Pad(psi1_t . W_j))
//   assembly Cc_j, Cd_j = Extract(IFFT2(Z_j)) of the pointwise combinations Z_j
// (upstream src/integrals.c:90-133, :211-251, :332-379 and
// src/collision.c:74-168, :209-254).
//
// Layout and passes.  The padded P x P grids (P = 2N) live in global memory,
// dense and row-major; at these sizes a grid (18 KB to 1 MB) no longer fits a
// CTA's shared memory next to the others a term needs.  Every 2-D transform is
// a row pass and a column pass.  A pass kernel stages a tile of `nl` lines
// (rows, or columns read as row segments of nl consecutive elements) of one
// grid in shared memory, transforms them with a mixed-radix Stockham FFT
// (radices 8, 4, 3, 2 in the order of a plan, ping-ponging between two
// buffers, the twiddles from a table of the L-th roots of unity), and fuses
// the pointwise products of the sums into the load and the store of the tile.
// The quadrature terms run in waves of nt terms for all cells of the batch:
// one wave is a handful of launches over (cell, term, grid) units, and the
// sums accumulate in global memory.  Every element of a sum has one owner per
// launch (the CTA holding its line), which adds the wave's terms in order, and
// the waves follow one another on the stream, so the result is deterministic.
#include "qb_engine.h"
#include "qb_fft.cuh"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <set>
#include <tuple>

namespace qb {

namespace {

constexpr int kThreads = 256;
constexpr int kMaxStages = 8;
constexpr size_t kMaxSmem = 200 * 1024;

// radix schedule of one transform length: radices 2, 3, 4, 6, 8, 12, 16 whose product is L
struct Plan {
	int L = 0, nst = 0;
	int r[kMaxStages] = {};
	const double2 *twd = nullptr;        // the L-th roots of unity, built once per workspace (null: each CTA computes them)
	const float2 *twf = nullptr;
};

__device__ __forceinline__ int src_idx(int p, int N) {         // padded index -> N-grid index, or -1 (zero band)
	return p < N / 2 ? p : (p >= 3 * N / 2 ? p - N : -1);
}

template <int DIR, class C> __device__ __forceinline__ void dft3(C &x0, C &x1, C &x2) {
	using R = typename CT<C>::R;
	const C t1 = cadd(x1, x2);
	const C m = csub(x0, cscale(t1, (R)0.5));
	const C d = mul_i<DIR>(cscale(csub(x1, x2), (R)0.86602540378443864676));   // sin(2 pi / 3)
	x0 = cadd(x0, t1);
	x1 = cadd(m, d);
	x2 = csub(m, d);
}

// cos and sin of 2 pi m / R for R = 6, 12, 16 (the twiddles of the composite
// register DFTs; folded to constants when m is known at compile time)
__host__ __device__ constexpr double cos_r(int R, int m) {
	constexpr double h = 0.5, c3 = 0.86602540378443864676, c8 = 0.70710678118654752440;
	constexpr double a = 0.92387953251128675613, b = 0.38268343236508977173;
	if (R == 16) {
		const double t[16] = { 1, a, c8, b, 0, -b, -c8, -a, -1, -a, -c8, -b, 0, b, c8, a };
		return t[m];
	}
	if (R == 12) {
		const double t[12] = { 1, c3, h, 0, -h, -c3, -1, -c3, -h, 0, h, c3 };
		return t[m];
	}
	const double t[6] = { 1, h, -h, -1, -h, h };
	return t[m];
}
__host__ __device__ constexpr double sin_r(int R, int m) {
	if (R == 6) {
		constexpr double c3 = 0.86602540378443864676;
		const double t[6] = { 0, c3, c3, 0, -c3, -c3 };
		return t[m];
	}
	return cos_r(R, (m + 3 * R / 4) % R);     // sin x = cos(x - pi/2); R = 12, 16 are multiples of 4
}

template <int R1, int R2, int DIR, class C> __device__ __forceinline__ void dft_ct(C (&x)[R1 * R2]);

template <int RAD, int DIR, class C> __device__ __forceinline__ void dft_r(C (&v)[RAD]) {
	if constexpr (RAD == 16) dft_ct<4, 4, DIR>(v);
	else if constexpr (RAD == 12) dft_ct<4, 3, DIR>(v);
	else if constexpr (RAD == 8) dft8<DIR>(v);
	else if constexpr (RAD == 6) dft_ct<2, 3, DIR>(v);
	else if constexpr (RAD == 4) dft4<DIR>(v[0], v[1], v[2], v[3]);
	else if constexpr (RAD == 3) dft3<DIR>(v[0], v[1], v[2]);
	else dft2(v[0], v[1]);
}

// an R1 R2-point DFT in registers, in place: R2 DFTs of R1 points (stride
// R2), twiddles w_R^(n2 k1), R1 DFTs of R2 points.  Input in natural order;
// output frequency k1 + R1 k2 lands in slot k1 R2 + k2 (freq_of gives the
// frequency of a slot), so no second array of R values is live
template <int R1, int R2, int DIR, class C> __device__ __forceinline__ void dft_ct(C (&x)[R1 * R2]) {
	using R = typename CT<C>::R;
	constexpr int RR = R1 * R2;
#pragma unroll
	for (int n2 = 0; n2 < R2; n2++) {
		C v[R1];
#pragma unroll
		for (int n1 = 0; n1 < R1; n1++) v[n1] = x[n2 + R2 * n1];
		dft_r<R1, DIR>(v);
#pragma unroll
		for (int k1 = 0; k1 < R1; k1++) {
			const int m = (n2 * k1) % RR;
			if (m == 0) {
				x[n2 + R2 * k1] = v[k1];
			} else {
				C w;
				w.x = (R)cos_r(RR, m);
				w.y = (R)(DIR < 0 ? -sin_r(RR, m) : sin_r(RR, m));
				x[n2 + R2 * k1] = cmul(v[k1], w);
			}
		}
	}
#pragma unroll
	for (int k1 = 0; k1 < R1; k1++) {
		C v[R2];
#pragma unroll
		for (int n2 = 0; n2 < R2; n2++) v[n2] = x[k1 * R2 + n2];
		dft_r<R2, DIR>(v);
#pragma unroll
		for (int k2 = 0; k2 < R2; k2++) x[k1 * R2 + k2] = v[k2];
	}
}

// frequency held in slot s after dft_r<RAD> (the composite radices leave
// their output permuted; 2, 3, 4, 8 and the sub-DFTs are in natural order)
template <int RAD> __host__ __device__ constexpr int freq_of(int s) {
	if (RAD == 16) return s / 4 + 4 * (s % 4);
	if (RAD == 12) return s / 3 + 4 * (s % 3);
	if (RAD == 6) return s / 3 + 2 * (s % 3);
	return s;
}

// one Stockham stage of radix RAD over nl lines of length L (sub-transforms of
// length Ns done): butterfly j of a line reads x[j + r L/RAD], twiddles by
// w^(r (j mod Ns)) with w = exp(DIR 2 pi i / (Ns RAD)), and writes its outputs
// to (j / Ns) Ns RAD + (j mod Ns) + r Ns.  tw[m] = exp(-2 pi i m / L).
// row l of a padded P = 2N grid lies in the zero band of the padding
__device__ __forceinline__ bool in_zero_band(int l, int N) { return l >= N / 2 && l < 3 * N / 2; }

// shared-memory slot of tile element (row, col) in rows of `pitch` slots: one
// pad slot after every 16 columns of a row, and rows of L + L/16 + 3 slots
// (tile_pitch).  Among the layouts of this form, and the global pad-every-16
// and XOR forms, this one gave the fewest shared-memory wavefronts in a
// count of every access of the passes (8-byte elements, half-warps) at
// P = 48, 96, 192 and 256: 1.25-1.5 per ideal at P = 192 and 1.0 at P = 256,
// against about 1.95 and 1.75 for a global pad every 16 over rows of L + 1.
__host__ __device__ __forceinline__ int tile_pitch(int L) { return L + (L >> 4) + 3; }
__device__ __forceinline__ int tat(int row, int col, int pitch) { return row * pitch + col + (col >> 4); }

// x / d for x, d < 2^16 as a high multiply by floor(2^32 / d) + 1: the error
// x (d - 2^32 mod d) / (d 2^32) stays below 1/d, so the quotient is exact;
// d = 1 (whose multiplier does not fit 32 bits) is marked by 0
__device__ __forceinline__ unsigned magic_div(unsigned d) { return d == 1u ? 0u : 0xffffffffu / d + 1u; }
__device__ __forceinline__ int fdiv(int x, unsigned mg) { return mg ? (int)__umulhi((unsigned)x, mg) : x; }

template <int RAD, int DIR, class C>
__device__ __forceinline__ void stage(const C *in, C *out, int nl, int ls, int es, int L, int Ns, const C *tw) {
	const int m = L / RAD, tstep = L / (Ns * RAD);
	const unsigned mg_m = magic_div((unsigned)m), mg_ns = magic_div((unsigned)Ns);
	for (int b = threadIdx.x; b < nl * m; b += blockDim.x) {
		const int line = fdiv(b, mg_m), j = b - line * m;
		const int jq = fdiv(j, mg_ns), k = j - jq * Ns;
		// lines are the tile's rows (es = 1, row pitch ls) or its columns (ls = 1, row pitch es)
		auto at = [ls, es, line](int e) { return es == 1 ? tat(line, e, ls) : tat(e, line, es); };
		C v[RAD];
#pragma unroll
		for (int r = 0; r < RAD; r++) v[r] = in[at(j + r * m)];
		if (Ns > 1) {
#pragma unroll
			for (int r = 1; r < RAD; r++) {
				C w = tw[r * k * tstep];                        // r k tstep < L
				if (DIR > 0) w.y = -w.y;
				v[r] = cmul(v[r], w);
			}
		}
		dft_r<RAD, DIR>(v);
		const int ob = jq * Ns * RAD + k;
#pragma unroll
		for (int r = 0; r < RAD; r++) out[at(ob + freq_of<RAD>(r) * Ns)] = v[r];
	}
}

// transforms the nl lines at `a` (line stride ls, element stride es; rows of
// a tile: (pitch, 1), its columns: (1, pitch)) in the direction DIR, with `b`
// as the second buffer; returns the buffer that holds the result.  Starts and
// ends with the CTA synchronised.
template <int DIR, class C> __device__ C *fft_lines(C *a, C *b, int nl, int ls, int es, const Plan &pl, const C *tw) {
	int Ns = 1;
	for (int s = 0; s < pl.nst; s++) {
		const int R = pl.r[s];
		if (R == 16) stage<16, DIR>(a, b, nl, ls, es, pl.L, Ns, tw);
		else if (R == 12) stage<12, DIR>(a, b, nl, ls, es, pl.L, Ns, tw);
		else if (R == 8) stage<8, DIR>(a, b, nl, ls, es, pl.L, Ns, tw);
		else if (R == 6) stage<6, DIR>(a, b, nl, ls, es, pl.L, Ns, tw);
		else if (R == 4) stage<4, DIR>(a, b, nl, ls, es, pl.L, Ns, tw);
		else if (R == 3) stage<3, DIR>(a, b, nl, ls, es, pl.L, Ns, tw);
		else stage<2, DIR>(a, b, nl, ls, es, pl.L, Ns, tw);
		__syncthreads();
		C *t = a; a = b; b = t;
		Ns *= R;
	}
	return a;
}

// The same stages with the data path given by functors, so that a pass
// reads its first stage straight from global memory and its last stage
// stores straight to its destination (global memory, or shared memory with a
// pointwise factor applied) instead of staging whole tiles through shared
// memory.  ld(line, i) -> C and st(line, i, v) address element i of a line.
// LF (line-fastest) hands consecutive lines to consecutive threads, the
// coalesced order for the columns of a row-major grid in global memory;
// otherwise consecutive threads take consecutive butterflies of a line, the
// coalesced order for rows.  Shared-memory layouts are the caller's.
template <int RAD, int DIR, bool LF, class C, class Ld, class St>
__device__ __forceinline__ void stage_f(int nl, int L, int Ns, const C *tw, const Ld &ld, const St &st) {
	const int m = L / RAD, tstep = L / (Ns * RAD);
	const unsigned mg_m = magic_div((unsigned)m), mg_ns = magic_div((unsigned)Ns), mg_nl = magic_div((unsigned)nl);
	for (int b = threadIdx.x; b < nl * m; b += blockDim.x) {
		int line, j;
		if (LF) {
			j = fdiv(b, mg_nl);
			line = b - j * nl;
		} else {
			line = fdiv(b, mg_m);
			j = b - line * m;
		}
		const int jq = fdiv(j, mg_ns), k = j - jq * Ns;
		C v[RAD];
#pragma unroll
		for (int r = 0; r < RAD; r++) v[r] = ld(line, j + r * m);
		if (Ns > 1) {
#pragma unroll
			for (int r = 1; r < RAD; r++) {
				C w = tw[r * k * tstep];                        // r k tstep < L
				if (DIR > 0) w.y = -w.y;
				v[r] = cmul(v[r], w);
			}
		}
		dft_r<RAD, DIR>(v);
		const int ob = jq * Ns * RAD + k;
#pragma unroll
		for (int r = 0; r < RAD; r++) st(line, ob + freq_of<RAD>(r) * Ns, v[r]);
	}
}
template <int DIR, bool LF, class C, class Ld, class St>
__device__ __forceinline__ void stage_any(int R, int nl, int L, int Ns, const C *tw, const Ld &ld, const St &st) {
	if (R == 16) stage_f<16, DIR, LF>(nl, L, Ns, tw, ld, st);
	else if (R == 12) stage_f<12, DIR, LF>(nl, L, Ns, tw, ld, st);
	else if (R == 8) stage_f<8, DIR, LF>(nl, L, Ns, tw, ld, st);
	else if (R == 6) stage_f<6, DIR, LF>(nl, L, Ns, tw, ld, st);
	else if (R == 4) stage_f<4, DIR, LF>(nl, L, Ns, tw, ld, st);
	else if (R == 3) stage_f<3, DIR, LF>(nl, L, Ns, tw, ld, st);
	else stage_f<2, DIR, LF>(nl, L, Ns, tw, ld, st);
}
// An FFT of nl lines: the first stage reads through ld0 (mapping LF0), the
// middle stages ping-pong between the line-contiguous shared buffers a and b
// (element i of a line at tat(line, i, pitch)), the last stage (mapping LF1)
// stores through st1(line, i, v, free), where `free` is the buffer that the
// last stage does not read.  The first stage writes a, so ld0 must not read a.
// A barrier follows every stage but the last; returns `free`.
template <int DIR, bool LF0, bool LF1, class C, class Ld, class St>
__device__ C *fft_f(int nl, int pitch, const Plan &pl, const C *tw, C *a, C *b, const Ld &ld0, const St &st1) {
	int Ns = 1;
	C *cur = b, *nxt = a;
	for (int s = 0; s < pl.nst; s++) {
		const int R = pl.r[s];
		const bool first = s == 0, last = s == pl.nst - 1;
		C *const in = cur, *const out = nxt;
		auto sm_ld = [in, pitch](int line, int i) { return in[tat(line, i, pitch)]; };
		auto sm_st = [out, pitch](int line, int i, const C &v) { out[tat(line, i, pitch)] = v; };
		auto st_last = [&st1, out](int line, int i, const C &v) { st1(line, i, v, out); };
		if (first && last) stage_any<DIR, LF0>(R, nl, pl.L, Ns, tw, ld0, st_last);
		else if (first) stage_any<DIR, LF0>(R, nl, pl.L, Ns, tw, ld0, sm_st);
		else if (last) stage_any<DIR, LF1>(R, nl, pl.L, Ns, tw, sm_ld, st_last);
		else stage_any<DIR, false>(R, nl, pl.L, Ns, tw, sm_ld, sm_st);
		if (last) return out;
		__syncthreads();
		cur = out;
		nxt = (out == a) ? b : a;
		Ns *= R;
	}
	return nxt;
}

// fft_f for a plan of exactly two stages R1 R2 known at compile time: the
// same arithmetic with only its two stage bodies in the kernel (the run-time
// dispatch of fft_f compiles every radix at every position, and the kernels
// that hold two transforms then stall on instruction fetch).  R1 = 0: fft_f.
template <int R1, int R2, int DIR, bool LF0, bool LF1, class C, class Ld, class St>
__device__ C *fft_fx(int nl, int pitch, const Plan &pl, const C *tw, C *a, C *b, const Ld &ld0, const St &st1) {
	if constexpr (R1 == 0) {
		return fft_f<DIR, LF0, LF1>(nl, pitch, pl, tw, a, b, ld0, st1);
	} else {
		auto sm_st = [a, pitch](int line, int i, const C &v) { a[tat(line, i, pitch)] = v; };
		stage_f<R1, DIR, LF0>(nl, R1 * R2, 1, tw, ld0, sm_st);
		__syncthreads();
		auto sm_ld = [a, pitch](int line, int i) { return a[tat(line, i, pitch)]; };
		auto st_last = [&st1, b](int line, int i, const C &v) { st1(line, i, v, b); };
		stage_f<R2, DIR, LF1>(nl, R1 * R2, R1, tw, sm_ld, st_last);
		return b;
	}
}
// fft_lines with the two stages of the plan known at compile time (R1 = 0:
// fft_lines); the result is in a again
template <int R1, int R2, int DIR, class C> __device__ C *fft_lines_x(C *a, C *b, int nl, int ls, int es, const Plan &pl, const C *tw) {
	if constexpr (R1 == 0) {
		return fft_lines<DIR>(a, b, nl, ls, es, pl, tw);
	} else {
		stage<R1, DIR>(a, b, nl, ls, es, R1 * R2, 1, tw);
		__syncthreads();
		stage<R2, DIR>(b, a, nl, ls, es, R1 * R2, R1, tw);
		__syncthreads();
		return a;
	}
}
// the (R1, R2) instantiations a pass kernel has: the default plans of the
// engine's FP32 and FP64 sizes P = 48, 96, 192, 256 (16 3, 16 6, 16 12, 16 16)
inline int two_stage_key(const Plan &pl) {
	if (pl.nst != 2 || pl.r[0] != 16) return 0;
	return (pl.r[1] == 3 || pl.r[1] == 6 || pl.r[1] == 12 || pl.r[1] == 16) ? pl.r[1] : 0;
}

// the twiddle table tw[m] = exp(-2 pi i m / L), then a CTA barrier
__device__ __forceinline__ const double2 *plan_tw(const Plan &pl, double2 *) { return pl.twd; }
__device__ __forceinline__ const float2 *plan_tw(const Plan &pl, float2 *) { return pl.twf; }
// exp(-2 pi i m / L), out of line: the kernels that read the table do not
// carry its registers
__device__ __noinline__ double2 root_of_unity(int m, int L) {
	double s, c;
	sincospi(2.0 * m / L, &s, &c);
	return make_double2(c, -s);
}
// the table of the workspace (every pass of AnyRhs has one)
template <class C> __device__ void load_tw(C *tw, int L, const Plan &pl) {
	const C *g = plan_tw(pl, tw);
	for (int m = threadIdx.x; m < L; m += blockDim.x) tw[m] = g[m];
	__syncthreads();
}
// the table, or without one (the workspace-free transforms) computed per CTA
template <class C> __device__ void init_tw(C *tw, int L, const Plan &pl) {
	const C *g = plan_tw(pl, tw);
	for (int m = threadIdx.x; m < L; m += blockDim.x) {
		if (g != nullptr) {
			tw[m] = g[m];
		} else {
			const double2 w = root_of_unity(m, L);
			tw[m] = mk<C>(w.x, w.y);
		}
	}
	__syncthreads();
}
// the table of init_tw for L = P, in both precisions
__global__ void k_any_build_tw(int L, double2 *twd, float2 *twf) {
	for (int m = threadIdx.x; m < L; m += blockDim.x) {
		double s, c;
		sincospi(2.0 * m / L, &s, &c);
		twd[m] = make_double2(c, -s);
		twf[m] = mk<float2>(c, -s);
	}
}

// shared-memory layout of a pass: the twiddles, then two buffers of nl rows
// (element (row, col) of a buffer at at(row, col))
template <class C> struct Tile {
	C *tw, *a, *b;
	int pitch;
	__device__ Tile(unsigned char *sm, int L, int nl) {
		pitch = tile_pitch(L);
		tw = reinterpret_cast<C *>(sm);
		a = tw + L;
		b = a + nl * pitch;
	}
	__device__ __forceinline__ int at(int row, int col) const { return tat(row, col, pitch); }
};
// the twiddles and two buffers of nl rows of tile_pitch(L) slots
template <class C> size_t tile_bytes(int L, int nl) {
	return sizeof(C) * ((size_t)L + 2 * (size_t)nl * tile_pitch(L));
}

// ---------------------------------------------------------------------------
// passes

// element loop of a tile with kBatch global loads in flight per thread:
// v = ld(i) for i = tid + u kThreads (u < kBatch), then st(i, v)
constexpr int kBatch = 8;
template <class V, class Ld, class St> __device__ __forceinline__ void batched(int n, const Ld &ld, const St &st) {
	for (int i0 = threadIdx.x; i0 < n; i0 += kBatch * kThreads) {
		V v[kBatch];
#pragma unroll
		for (int u = 0; u < kBatch; u++) {
			const int i = i0 + u * kThreads;
			if (i < n) v[u] = ld(i);
		}
#pragma unroll
		for (int u = 0; u < kBatch; u++) {
			const int i = i0 + u * kThreads;
			if (i < n) st(i, v[u]);
		}
	}
}
template <class C> struct Two { C a, b; };

// rows of Pad(mult . W_comp) for unit u = (cell nt + tt) nsub + sub, forward
// transform: out[u] (row pass of the spectra, of P_j and of the first
// transforms of the I1 / I2 terms).  psel: 0 no factor, 1 / 2 real table A / B
// of term t0 + tt, 3 the complex table.
template <class C> struct PadRowsP {
	using R = typename CT<C>::R;
	const double2 *W; long w_cell;
	int N, nl, nt, t0, nsub;
	int comp[8], psel[8], comp2[8];      // psel 4: psiC . (W_comp + i W_comp2)
	const R *psiA, *psiB;                 // real N x N tables, one per term
	const C *psiC;                        // complex N x N tables, one per term
	C *out;
	// kind != null: the cells of kind 0 (real form) take the first nsub_rf
	// subs with comp_rf / comp2_rf / psel_rf instead
	const int *kind;
	int nsub_rf, comp_rf[4], comp2_rf[4], psel_rf[4];
	Plan pl;
};
template <class C, int R1, int R2> __global__ void __launch_bounds__(kThreads) k_any_pad_rows(const PadRowsP<C> p) {
	using R = typename CT<C>::R;
	extern __shared__ __align__(16) unsigned char sm[];
	const int N = p.N, P = 2 * N, nl = p.nl;
	const long NN = (long)N * N, PP = (long)P * P;
	Tile<C> T(sm, P, nl);
	const unsigned mgP = magic_div((unsigned)P), mgnl = magic_div((unsigned)nl);
	const int bpg = P / nl;
	const long u = blockIdx.x / bpg;
	const int l0 = (int)(blockIdx.x % bpg) * nl;
	const int sub = (int)(u % p.nsub);
	const long ct = u / p.nsub;
	const int t = p.t0 + (int)(ct % p.nt);
	const long cell = ct / p.nt;
	int ps = p.psel[sub], ca = p.comp[sub], cb = p.comp2[sub];
	if (p.kind != nullptr && p.kind[cell] == 0) {
		if (sub >= p.nsub_rf) return;
		ps = p.psel_rf[sub]; ca = p.comp_rf[sub]; cb = p.comp2_rf[sub];
	}
	// every row of the tile in the zero band: its transform is zero, and the
	// column passes that read this output (k_any_plain with zband, the I1 and
	// I2 column passes) take those rows as zero without reading them
	if (l0 >= N / 2 && l0 + nl <= 3 * N / 2) return;
	load_tw(T.tw, P, p.pl);
	const double2 *w = p.W + cell * p.w_cell + (long)ca * NN;
	const double2 *w2 = p.W + cell * p.w_cell + (long)cb * NN;
	batched<C>(nl * P, [&](int i) {
		const int li = fdiv(i, mgP), k = i - li * P;
		const int ls = src_idx(l0 + li, N), ks = src_idx(k, N);
		C v = czero<C>();
		if (ls >= 0 && ks >= 0) {
			const long q = (long)ls * N + ks;
			const double2 x = w[q];
			if (ps == 0) v = mk<C>(x.x, x.y);
			else if (ps == 3) v = cmul(p.psiC[t * NN + q], mk<C>(x.x, x.y));
			else if (ps == 4) {
				const double2 y = w2[q];
				v = cmul(p.psiC[t * NN + q], mk<C>(x.x - y.y, x.y + y.x));
			}
			else {
				const R f = (ps == 1 ? p.psiA : p.psiB)[t * NN + q];
				v.x = f * (R)x.x;
				v.y = f * (R)x.y;
			}
		}
		return v;
	}, [&](int i, const C &v) {
		const int li = fdiv(i, mgP), k = i - li * P;
		T.b[T.at(li, k)] = v;
	});
	__syncthreads();
	// staged in b; the last stage stores the rows to global memory
	C *o = p.out + u * PP + (long)l0 * P;
	const int pitch = T.pitch;
	const C *sb = T.b;
	auto ld0 = [sb, pitch](int line, int i) { return sb[tat(line, i, pitch)]; };
	auto st1 = [o, P](int line, int i, const C &v, C *) { o[(long)line * P + i] = v; };
	fft_fx<R1, R2, -1, false, false>(nl, pitch, p.pl, T.tw, T.a, T.b, ld0, st1);
}

// in-place row or column transforms of L x L grids g[u] (spectra, FS, the
// Fourier representation)
template <class C> struct PlainP {
	C *g; int L, nl;
	// kind != null: grids [cell][gpc / nsub][nsub]; a cell of kind 0 (real
	// form) skips the subs from rf_grids on
	const int *kind; long gpc; int nsub, rf_grids;
	int zband;                            // N > 0: the grids come from k_any_pad_rows, rows in its zero band read as zero (columns only)
	Plan pl;
};
template <class C, int DIR, bool COLS, int R1, int R2> __global__ void __launch_bounds__(kThreads) k_any_plain(const PlainP<C> p) {
	extern __shared__ __align__(16) unsigned char sm[];
	const int L = p.L, nl = p.nl;
	Tile<C> T(sm, L, nl);
	const unsigned mgP = magic_div((unsigned)L), mgnl = magic_div((unsigned)nl);
	const int bpg = L / nl;
	const long u = blockIdx.x / bpg;
	const int x0 = (int)(blockIdx.x % bpg) * nl;
	if (p.kind != nullptr && p.kind[u / p.gpc] == 0 && (int)(u % p.nsub) >= p.rf_grids) return;
	init_tw(T.tw, L, p.pl);
	C *g = p.g + u * (long)L * L;
	batched<C>(nl * L, [&](int i) {
		if (COLS) {
			const int l = fdiv(i, mgnl), kk = i - l * nl;
			return (p.zband > 0 && in_zero_band(l, p.zband)) ? czero<C>() : g[(long)l * L + x0 + kk];
		}
		const int li = fdiv(i, mgP), k = i - li * L;
		return g[(long)(x0 + li) * L + k];
	}, [&](int i, const C &v) {
		if (COLS) { const int l = fdiv(i, mgnl), kk = i - l * nl; T.b[T.at(kk, l)] = v; }
		else { const int li = fdiv(i, mgP), k = i - li * L; T.b[T.at(li, k)] = v; }
	});
	__syncthreads();
	// staged in b; the last stage stores to global memory in the coalesced order
	const int pitch = T.pitch;
	const C *sb = T.b;
	auto ld0 = [sb, pitch](int line, int i) { return sb[tat(line, i, pitch)]; };
	auto st1 = [g, L, x0](int line, int i, const C &v, C *) {
		if (COLS) g[(long)i * L + x0 + line] = v;
		else g[(long)(x0 + line) * L + i] = v;
	};
	fft_fx<R1, R2, DIR, false, COLS>(nl, pitch, p.pl, T.tw, T.a, T.b, ld0, st1);
}

// I1 / I4 columns of unit u = (cell nt + tt) nsub + sub: forward transform,
// times F = fa W^_f + fb, inverse transform, in place
template <class C> struct I1ColsP {
	C *g; const C *What; int N, nl, nt, nsub, fcomp;
	double fa, fb;
	Plan pl;
};
template <class C, int R1, int R2> __global__ void __launch_bounds__(kThreads) k_any_i1_cols(const I1ColsP<C> p) {
	using R = typename CT<C>::R;
	extern __shared__ __align__(16) unsigned char sm[];
	const int P = 2 * p.N, nl = p.nl;
	const long PP = (long)P * P;
	Tile<C> T(sm, P, nl);
	const unsigned mgP = magic_div((unsigned)P), mgnl = magic_div((unsigned)nl);
	load_tw(T.tw, P, p.pl);
	const int bpg = P / nl;
	const long u = blockIdx.x / bpg;
	const int k0 = (int)(blockIdx.x % bpg) * nl;
	const long cell = u / ((long)p.nsub * p.nt);
	C *g = p.g + u * PP;
	const C *F = p.What + (cell * 4 + p.fcomp) * PP;
	batched<C>(nl * P, [&](int i) {             // rows in the zero band of k_any_pad_rows read as zero
		const int l = fdiv(i, mgnl), kk = i - l * nl;
		return in_zero_band(l, p.N) ? czero<C>() : g[(long)l * P + k0 + kk];
	}, [&](int i, const C &v) {
		const int l = fdiv(i, mgnl), kk = i - l * nl;
		T.a[T.at(kk, l)] = v;
	});
	__syncthreads();
	C *r = fft_lines_x<R1, R2, -1>(T.a, T.b, nl, T.pitch, 1, p.pl, T.tw);
	const R fa = (R)p.fa, fb = (R)p.fb;
	batched<C>(nl * P, [&](int i) {
		const int l = fdiv(i, mgnl), kk = i - l * nl;
		return F[(long)l * P + k0 + kk];
	}, [&](int i, const C &w) {
		const int l = fdiv(i, mgnl), kk = i - l * nl;
		C f; f.x = fa * w.x + fb; f.y = fa * w.y;
		r[T.at(kk, l)] = cmul(f, r[T.at(kk, l)]);
	});
	__syncthreads();
	const C *r2 = fft_lines_x<R1, R2, +1>(r, r == T.a ? T.b : T.a, nl, T.pitch, 1, p.pl, T.tw);
	for (int i = threadIdx.x; i < nl * P; i += blockDim.x) {
		const int l = fdiv(i, mgnl), kk = i - l * nl;
		g[(long)l * P + k0 + kk] = r2[T.at(kk, l)];
	}
}

// I1 / I4 rows, inverse transform, S[cell][sub] += phi_t . row, for the wave's
// terms in order (one CTA per (cell, sub, row block))
template <class C> struct I1RowsP {
	using R = typename CT<C>::R;
	const C *g; C *S; const R *phi; int N, nl, nt, t0, nsub;
	Plan pl;
};
template <class C, int R1, int R2> __global__ void __launch_bounds__(kThreads) k_any_i1_rows(const I1RowsP<C> p) {
	using R = typename CT<C>::R;
	extern __shared__ __align__(16) unsigned char sm[];
	const int P = 2 * p.N, nl = p.nl;
	const long PP = (long)P * P;
	Tile<C> T(sm, P, nl);
	const unsigned mgP = magic_div((unsigned)P), mgnl = magic_div((unsigned)nl);
	load_tw(T.tw, P, p.pl);
	const int bpg = P / nl;
	const long cs = blockIdx.x / bpg;             // cell nsub + sub
	const int l0 = (int)(blockIdx.x % bpg) * nl;
	const long cell = cs / p.nsub;
	const int sub = (int)(cs % p.nsub);
	C *S = p.S + cs * PP + (long)l0 * P;
	for (int tt = 0; tt < p.nt; tt++) {
		const C *g = p.g + ((cell * p.nt + tt) * p.nsub + sub) * PP + (long)l0 * P;
		batched<C>(nl * P, [&](int i) { return g[i]; }, [&](int i, const C &v) {
			const int li = fdiv(i, mgP), k = i - li * P;
			T.a[T.at(li, k)] = v;
		});
		__syncthreads();
		const C *r = fft_lines_x<R1, R2, +1>(T.a, T.b, nl, T.pitch, 1, p.pl, T.tw);
		const R *phi = p.phi + (long)(p.t0 + tt) * PP + (long)l0 * P;
		batched<Two<C>>(nl * P, [&](int i) {
			Two<C> v;
			v.a = S[i];
			v.b.x = phi[i];
			return v;
		}, [&](int i, const Two<C> &v) {
			const int li = fdiv(i, mgP), k = i - li * P;
			const R f = v.b.x;
			const C x = r[T.at(li, k)];
			C s = v.a;
			s.x += f * x.x;
			s.y += f * x.y;
			S[i] = s;
		});
		__syncthreads();
	}
}

// I2 columns: forward transforms of A = g[(cell nt + tt) 8 + 2i] and
// B = g[... + 2i + 1], Q[cell][i] += A . B over the wave's terms in order
template <class C> struct I2ColsP {
	const C *g; C *Q; int N, nl, nt;
	Plan pl;
};
template <class C, int R1, int R2> __global__ void __launch_bounds__(kThreads) k_any_i2_cols(const I2ColsP<C> p) {
	extern __shared__ __align__(16) unsigned char sm[];
	const int P = 2 * p.N, nl = p.nl;
	const long PP = (long)P * P;
	Tile<C> T(sm, P, 2 * nl);
	const unsigned mgP = magic_div((unsigned)P), mgnl = magic_div((unsigned)nl);
	load_tw(T.tw, P, p.pl);
	const int bpg = P / nl;
	const long ci = blockIdx.x / bpg;             // cell 4 + i
	const int k0 = (int)(blockIdx.x % bpg) * nl;
	const long cell = ci / 4;
	const int ii = (int)(ci % 4);
	C *Q = p.Q + ci * PP;
	for (int tt = 0; tt < p.nt; tt++) {
		const C *ga = p.g + ((cell * p.nt + tt) * 8 + 2 * ii) * PP;
		batched<C>(2 * nl * P, [&](int i) {
			const int h = i >= nl * P ? 1 : 0, rem = i - h * nl * P, l = fdiv(rem, mgnl), kk = rem - l * nl;
			return in_zero_band(l, p.N) ? czero<C>() : ga[h * PP + (long)l * P + k0 + kk];   // zero band of k_any_pad_rows
		}, [&](int i, const C &v) {
			const int h = i >= nl * P ? 1 : 0, rem = i - h * nl * P, l = fdiv(rem, mgnl), kk = rem - l * nl;
			T.a[T.at(h * nl + kk, l)] = v;
		});
		__syncthreads();
		const C *r = fft_lines_x<R1, R2, -1>(T.a, T.b, 2 * nl, T.pitch, 1, p.pl, T.tw);
		batched<C>(nl * P, [&](int i) {
			const int l = fdiv(i, mgnl), kk = i - l * nl;
			return Q[(long)l * P + k0 + kk];
		}, [&](int i, const C &q) {
			const int l = fdiv(i, mgnl), kk = i - l * nl;
			Q[(long)l * P + k0 + kk] = cfma(r[T.at(kk, l)], r[T.at(nl + kk, l)], q);
		});
		__syncthreads();
	}
}

// resident CTAs an SM that the column pass of the chains is compiled for: two
// in FP64 (at most 128 registers); FP32 takes the compiler's choice (76
// registers, three CTAs, measured ahead of four CTAs with spills at N = 128)
template <class C> constexpr int pass_ctas() { return sizeof(C) == 16 ? 2 : 0; }

// the real form of the I3 sums exists in FP32 only
template <class C> __host__ __device__ constexpr bool has_rf() { return sizeof(typename CT<C>::R) == 4; }

// I3 chain, first rows: unit u = (cell nt + tt) 16 + c, inverse transform of
// the rows of the chain input into Y[u].  Complex form: c = 4 j + i, input
// W^_i . P_j, Pg holds P_0..P_3 per (cell, term).  Real form (kind 0: FP32
// cells without Nyquist content, where W^ and P are real): c = 2 j + pr < 8,
// one complex chain of P_j . (W^_2pr + i W^_2pr+1) for two combos, and Pg
// slots 0, 1 hold P_0 + i P_1, P_2 + i P_3; its units c >= 8 are idle.
template <class C> struct I3RowsAP {
	const C *What, *Pg; C *Y; int N, nl, nt;
	const int *kind;                      // null: every cell complex
	Plan pl;
};
template <class C, int R1, int R2> __global__ void __launch_bounds__(kThreads) k_any_i3_rows_a(const I3RowsAP<C> p) {
	extern __shared__ __align__(16) unsigned char sm[];
	const int P = 2 * p.N, nl = p.nl;
	const long PP = (long)P * P;
	Tile<C> T(sm, P, nl);
	const unsigned mgP = magic_div((unsigned)P), mgnl = magic_div((unsigned)nl);
	const int bpg = P / nl;
	const long u = blockIdx.x / bpg;
	const int l0 = (int)(blockIdx.x % bpg) * nl;
	const int c = (int)(u & 15);
	const long ct = u >> 4, cell = ct / p.nt;
	const bool rf = has_rf<C>() && p.kind != nullptr && p.kind[cell] == 0;
	if (rf && c >= 8) return;
	load_tw(T.tw, P, p.pl);
	if (rf) {
		const int pr = c & 1, j3 = c >> 1;
		const C *G0 = p.What + (cell * 4 + 2 * pr) * PP + (long)l0 * P, *G1 = G0 + PP;
		const C *Pj = p.Pg + (ct * 4 + (j3 >> 1)) * PP + (long)l0 * P;
		const bool im = j3 & 1;
		batched<Two<C>>(nl * P, [&](int i) {
			Two<C> v;
			v.a = mk<C>(G0[i].x, G1[i].x);
			v.b = Pj[i];
			return v;
		}, [&](int i, const Two<C> &v) {
			const int li = fdiv(i, mgP), k = i - li * P;
			const typename CT<C>::R pj = im ? v.b.y : v.b.x;
			T.b[T.at(li, k)] = cscale(v.a, pj);
		});
	} else {
		const C *G = p.What + (cell * 4 + (c & 3)) * PP + (long)l0 * P;
		const C *Pj = p.Pg + (ct * 4 + (c >> 2)) * PP + (long)l0 * P;
		batched<Two<C>>(nl * P, [&](int i) {
			Two<C> v;
			v.a = G[i];
			v.b = Pj[i];
			return v;
		}, [&](int i, const Two<C> &v) {
			const int li = fdiv(i, mgP), k = i - li * P;
			T.b[T.at(li, k)] = cmul(v.a, v.b);
		});
	}
	__syncthreads();
	// staged in b; the last stage stores the rows to global memory
	C *o = p.Y + u * PP + (long)l0 * P;
	const int pitch = T.pitch;
	const C *sb = T.b;
	auto ld0 = [sb, pitch](int line, int i) { return sb[tat(line, i, pitch)]; };
	auto st1 = [o, P](int line, int i, const C &v, C *) { o[(long)line * P + i] = v; };
	fft_fx<R1, R2, +1, false, false>(nl, pitch, p.pl, T.tw, T.a, T.b, ld0, st1);
}

// I3 chain, columns of Y[u]: inverse transform, times psi2_t (element (l, k)
// = scale[t] ST[idx[t]][k P + l]), forward transform, in place
template <class C> struct I3ColsP {
	using R = typename CT<C>::R;
	C *Y; const R *psi2T; const int *idx; const double *scale; int N, nl, nt, t0;
	const int *kind;                      // null: every cell complex; kind 0: units c >= 8 idle
	Plan pl;
};
template <class C, int R1, int R2> __global__ void __launch_bounds__(kThreads, pass_ctas<C>()) k_any_i3_cols(const I3ColsP<C> p) {
	using R = typename CT<C>::R;
	extern __shared__ __align__(16) unsigned char sm[];
	const int P = 2 * p.N, nl = p.nl;
	const long PP = (long)P * P;
	Tile<C> T(sm, P, nl);
	const int bpg = P / nl;
	const long u = blockIdx.x / bpg;
	const int k0 = (int)(blockIdx.x % bpg) * nl;
	const int ct = (int)(u >> 4);                                  // (cell, term) of the wave: below 2^31
	const int cell = ct / p.nt, t = p.t0 + (ct - cell * p.nt);
	if (p.kind != nullptr && p.kind[cell] == 0 && (u & 15) >= 8) return;
	load_tw(T.tw, P, p.pl);
	// columns k0 + line of the chain grid, element i = row i: the first
	// transform reads them from global memory (line-fastest, coalesced) and
	// its last stage applies psi2_t (rows k0.. of the transposed table, read
	// along a line: J-fastest, coalesced) on the way into shared memory; the
	// second transform writes them back
	C *g = p.Y + u * PP;
	const R sc = (R)p.scale[t];
	const R *ps = p.psi2T + (long)p.idx[t] * PP + (long)k0 * P;
	const int pitch = T.pitch;
	auto ld0 = [g, P, k0](int line, int i) { return g[(long)i * P + k0 + line]; };
	auto st_psi = [ps, sc, P, pitch](int line, int i, const C &v, C *out) {
		out[tat(line, i, pitch)] = cscale(v, sc * ps[line * P + i]);
	};
	C *X = fft_fx<R1, R2, +1, true, false>(nl, pitch, p.pl, T.tw, T.a, T.b, ld0, st_psi);
	__syncthreads();
	auto ld1 = [X, pitch](int line, int i) { return X[tat(line, i, pitch)]; };
	auto st_g = [g, P, k0](int line, int i, const C &v, C *) { g[(long)i * P + k0 + line] = v; };
	fft_fx<R1, R2, -1, false, true>(nl, pitch, p.pl, T.tw, X == T.a ? T.b : T.a, X, ld1, st_g);
}

// I3 chain, last rows: forward transforms of Y[(cell nt + tt) 16 + 4 j + i],
// one tile at a time, and X[cell][j] += sum_i eta_i P_i . row, over the
// wave's terms and i in order, in registers (one CTA per (cell, j, row block);
// a thread owns the tile elements tid + e kThreads, e < own_of<C>())
template <class C> __host__ __device__ constexpr int own_of() { return sizeof(C) == 16 ? 8 : 16; }   // nl P <= own_of<C>() kThreads
// the same for a compiled plan R1 R2 (P = R1 R2): FP32 tiles of 16 lines of
// 192 and 32 of 96 need 12 values a thread, 48 lines of 48 need 9; fewer
// accumulators leave the registers for three CTAs an SM
template <class C, int R1, int R2> __host__ __device__ constexpr int own_for() {
	return (sizeof(C) == 16 || R1 == 0) ? own_of<C>() : (R1 * R2 == 192 || R1 * R2 == 96) ? 12 : R1 * R2 == 48 ? 9 : 16;
}
inline int own_for_plan(const Plan &pl, bool fp64) {
	if (fp64) return 8;
	switch (two_stage_key(pl)) {
	case 12: case 6: return 12;
	case 3: return 9;
	default: return 16;
	}
}
template <class C> struct I3RowsBP {
	const C *Y, *Pg; C *X; int N, nl, nt;
	const int *kind;                      // null: every cell complex
	Plan pl;
};
// RF (kind 0): Y[(cell nt + tt) 16 + 2 j + pr] holds the two packed chains of
// (cell, term, j); X[cell][j] (real) += eta_2pr P_2pr . Re(row) + eta_2pr+1
// P_2pr+1 . Im(row)
template <class C, bool RF, int R1, int R2> __device__ __forceinline__ void i3_rows_b(const I3RowsBP<C> &p, unsigned char *sm) {
	using R = typename CT<C>::R;
	const int P = 2 * p.N, nl = p.nl, ne = nl * P;
	const long PP = (long)P * P;
	Tile<C> T(sm, P, nl);
	const unsigned mgP = magic_div((unsigned)P), mgnl = magic_div((unsigned)nl);
	const int bpg = P / nl;
	const long cj = blockIdx.x / bpg;             // cell 4 + j
	const int l0 = (int)(blockIdx.x % bpg) * nl;
	const long cell = cj / 4;
	const int j3 = (int)(cj % 4);
	load_tw(T.tw, P, p.pl);
	C *X = p.X + cj * PP + (long)l0 * P;
	constexpr int kOwn = own_for<C, R1, R2>();
	C acc[kOwn];
#pragma unroll
	for (int e = 0; e < kOwn; e++) {
		const int i = threadIdx.x + e * kThreads;
		acc[e] = i < ne ? X[i] : czero<C>();       // rows l0.. of X are contiguous: element i at X[i]
	}
	for (int tt = 0; tt < p.nt; tt++) {
		const long ct = cell * p.nt + tt;
		constexpr int kH = RF ? 2 : 4;
		for (int h = 0; h < kH; h++) {
			const C *y = p.Y + (ct * 16 + j3 * kH + h) * PP + (long)l0 * P;
			const int pitch = T.pitch;
			auto ld0 = [y, P](int line, int i) { return y[(long)line * P + i]; };
			auto st1 = [pitch](int line, int i, const C &v, C *out) { out[tat(line, i, pitch)] = v; };
			const C *r = fft_fx<R1, R2, -1, false, false>(nl, pitch, p.pl, T.tw, T.a, T.b, ld0, st1);
			__syncthreads();
			if constexpr (RF) {
				const C *Pa = p.Pg + (ct * 4 + h) * PP + (long)l0 * P;      // P_2h + i P_2h+1
				const R e0 = h == 0 ? (R)1 : (R)-1;                          // eta_2h; eta_2h+1 = -1
#pragma unroll
				for (int e = 0; e < kOwn; e++) {
					const int i = threadIdx.x + e * kThreads;
					if (i < ne) {
						const int li = fdiv(i, mgP), k = i - li * P;
						const C pa = Pa[i], y = r[T.at(li, k)];
						acc[e].x += e0 * (pa.x * y.x) - pa.y * y.y;
					}
				}
			} else {
				const C *Pa = p.Pg + (ct * 4 + h) * PP + (long)l0 * P;
				const R eta = h == 0 ? (R)1 : (R)-1;
#pragma unroll
				for (int e = 0; e < kOwn; e++) {
					const int i = threadIdx.x + e * kThreads;
					if (i < ne) {
						const int li = fdiv(i, mgP), k = i - li * P;
						const C v = cmul(Pa[i], r[T.at(li, k)]);
						acc[e].x += eta * v.x;
						acc[e].y += eta * v.y;
					}
				}
			}
			__syncthreads();
		}
	}
#pragma unroll
	for (int e = 0; e < kOwn; e++) {
		const int i = threadIdx.x + e * kThreads;
		if (i < ne) X[i] = acc[e];
	}
}
// two CTAs an SM (at most 128 registers: the accumulators live in
// registers); three (85) in FP32 where a thread holds 12 or fewer of them
// (FP64 stays at two: 1.5x slower at three)
template <class C, int R1, int R2> constexpr int rows_b_ctas() { return sizeof(C) == 8 && own_for<C, R1, R2>() <= 12 ? 3 : 2; }
template <class C, int R1, int R2> __global__ void __launch_bounds__(kThreads, rows_b_ctas<C, R1, R2>()) k_any_i3_rows_b(const I3RowsBP<C> p) {
	extern __shared__ __align__(16) unsigned char sm[];
	const long cell = blockIdx.x / (4L * (2 * p.N / p.nl));         // blocks (cell 4 + j) bpg + row block
	if constexpr (has_rf<C>()) {
		if (p.kind != nullptr && p.kind[cell] == 0) {
			i3_rows_b<C, true, R1, R2>(p, sm);
			return;
		}
	}
	i3_rows_b<C, false, R1, R2>(p, sm);
}

// The I3 chains with the whole P x P grid in shared memory (P = 48 and 96 in
// FP32, P = 48 in FP64): one CTA per (cell, j, i) runs the wave's terms in
// order, X[cell][j][i] += eta_i P_i . FFT2(psi2_t . IFFT2(W^_i . P_j)), each
// chain one load of W^_i . P_j, four in-place 2-D passes over the tile and one
// update of the partial X[cell][j][i] (in L2) instead of three global passes;
// the assembly adds the four partials of (cell, j) in the order i = 0..3.
template <class C> struct I3FusedP {
	using R = typename CT<C>::R;
	const C *What, *Pg; C *X; const R *psi2T; const int *idx; const double *scale;
	int N, nt, t0;
	const int *kind;                      // null: every cell complex
	Plan pl;
};
// RF (kind 0): the CTA (cell, j, pr), pr < 2, runs the packed chain of the
// combos 2pr, 2pr + 1 into the real partial X[cell][j][pr] (partials 2, 3 stay
// zero; the CTAs pr >= 2 are idle)
template <class C, bool RF> __device__ __forceinline__ void i3_fused(const I3FusedP<C> &p, unsigned char *sm) {
	using R = typename CT<C>::R;
	const int P = 2 * p.N, PPi = P * P;
	const long PP = (long)P * P;
	Tile<C> T(sm, P, P);
	const unsigned mgP = magic_div((unsigned)P);
	const long cji = blockIdx.x;                  // (cell 4 + j) 4 + h
	const long cell = cji / 16;
	const int j3 = (int)((cji / 4) % 4), h = (int)(cji % 4);
	load_tw(T.tw, P, p.pl);
	C *X = p.X + ((cell * 4 + j3) * 4 + h) * PP;
	const C *G = p.What + (cell * 4 + (RF ? 2 * h : h)) * PP;
	for (int tt = 0; tt < p.nt; tt++) {
		const long ct = cell * p.nt + tt;
		const int t = p.t0 + tt;
		const R sc = (R)p.scale[t];
		const R *ps = p.psi2T + (long)p.idx[t] * PP;
		const C *Pj = p.Pg + (ct * 4 + (RF ? j3 / 2 : j3)) * PP;
		{
			batched<Two<C>>(PPi, [&](int i) {
				Two<C> v;
				v.a = RF ? mk<C>(G[i].x, G[i + PP].x) : G[i];
				v.b = Pj[i];
				return v;
			}, [&](int i, const Two<C> &v) {
				const int l = fdiv(i, mgP), k = i - l * P;
				T.a[T.at(l, k)] = RF ? cscale(v.a, (j3 & 1) ? v.b.y : v.b.x) : cmul(v.a, v.b);
			});
			__syncthreads();
			C *r = fft_lines<+1>(T.a, T.b, P, T.pitch, 1, p.pl, T.tw);               // rows
			r = fft_lines<+1>(r, r == T.a ? T.b : T.a, P, 1, T.pitch, p.pl, T.tw);     // columns
			batched<R>(PPi, [&](int i) { return ps[i]; }, [&](int i, const R &f0) {
				const int k = fdiv(i, mgP), l = i - k * P;                   // transposed table: element (l, k)
				const R f = sc * f0;
				C x = r[T.at(l, k)];
				x.x *= f;
				x.y *= f;
				r[T.at(l, k)] = x;
			});
			__syncthreads();
			r = fft_lines<-1>(r, r == T.a ? T.b : T.a, P, 1, T.pitch, p.pl, T.tw);     // columns
			r = fft_lines<-1>(r, r == T.a ? T.b : T.a, P, T.pitch, 1, p.pl, T.tw);     // rows
			const C *Pa = p.Pg + (ct * 4 + h) * PP;
			const R eta = h == 0 ? (R)1 : (R)-1;
			batched<Two<C>>(PPi, [&](int i) {
				Two<C> v;
				v.a = Pa[i];
				v.b = X[i];
				return v;
			}, [&](int i, const Two<C> &v) {
				const int l = fdiv(i, mgP), k = i - l * P;
				C x = v.b;
				const C y0 = r[T.at(l, k)];
				if (RF) {                                  // eta_2h P_2h Re + eta_2h+1 P_2h+1 Im (eta_2h+1 = -1)
					x.x += eta * (v.a.x * y0.x) - v.a.y * y0.y;
				} else {
					const C y = cmul(v.a, y0);
					x.x += eta * y.x;
					x.y += eta * y.y;
				}
				X[i] = x;
			});
			__syncthreads();
		}
	}
}
template <class C> __global__ void __launch_bounds__(kThreads) k_any_i3_fused(const I3FusedP<C> p) {
	extern __shared__ __align__(16) unsigned char sm[];
	const long cell = blockIdx.x / 16;
	if constexpr (has_rf<C>()) {
		if (p.kind != nullptr && p.kind[cell] == 0) {
			if (blockIdx.x % 4 < 2) i3_fused<C, true>(p, sm);
			return;
		}
	}
	i3_fused<C, false>(p, sm);
}

// assembly rows: Zcc_j and Zcd_j (the combinations of k_assemble) for unit
// (cell, j), inverse row transforms into Z[(cell 4 + j) 2 + {0, 1}]
template <class C> struct AsmP {
	const C *What, *FS, *FS4, *Q, *X;    // FS [cell][3], FS4 / Q [cell][4], X [cell][4][nxp] (null: part absent)
	int nxp;                             // partials of X per (cell, j), added in order
	C *Z; int N, nl;
	double s1, s2;
	int mode;
	double2 *out_cc, *out_cd;
	const double2 *base, *wcur; const double *B; double dtc; double2 *out;
	Plan pl;
};
template <class C, int R1, int R2> __global__ void __launch_bounds__(kThreads) k_any_asm_rows(const AsmP<C> p) {
	using R = typename CT<C>::R;
	extern __shared__ __align__(16) unsigned char sm[];
	const int P = 2 * p.N, nl = p.nl;
	const long PP = (long)P * P;
	Tile<C> T(sm, P, 2 * nl);
	const unsigned mgP = magic_div((unsigned)P), mgnl = magic_div((unsigned)nl);
	load_tw(T.tw, P, p.pl);
	const int bpg = P / nl;
	const long cj = blockIdx.x / bpg;
	const int l0 = (int)(blockIdx.x % bpg) * nl;
	const long cell = cj / 4;
	const int j = (int)(cj % 4);
	const R eta2[4] = { 2, -2, -2, -2 };
	const R s1 = (R)p.s1, s2 = (R)p.s2;
	const C *Wh = p.What + cell * 4 * PP;
	for (int i = threadIdx.x; i < nl * P; i += blockDim.x) {
		const int li = fdiv(i, mgP), k = i - li * P;
		const long e = (long)(l0 + li) * P + k;
		C zc = czero<C>(), zd = czero<C>();
		if (p.FS != nullptr && j > 0) {
			const int gi = (j % 3) + 1, hi = ((j + 1) % 3) + 1;
			const C *FS = p.FS + cell * 3 * PP;
			zc = csub(cmul(Wh[hi * PP + e], FS[(gi - 1) * PP + e]), cmul(Wh[gi * PP + e], FS[(hi - 1) * PP + e]));
		}
		if (p.Q != nullptr) {
			C q = czero<C>();
			for (int ii = 0; ii < 4; ii++) {
				const C s = p.Q[(cell * 4 + ii) * PP + e];
				q.x += eta2[ii] * s.x;
				q.y += eta2[ii] * s.y;
			}
			C h; h.x = -Wh[j * PP + e].x; h.y = -Wh[j * PP + e].y;
			if (j == 0) h.x += (R)1.0;
			const C v = cmul(h, q);
			zd.x += s2 * v.x;
			zd.y += s2 * v.y;
		}
		if (p.X != nullptr) {
			C s = p.X[(cell * 4 + j) * p.nxp * PP + e];
			for (int k = 1; k < p.nxp; k++) s = cadd(s, p.X[((cell * 4 + j) * p.nxp + k) * PP + e]);
			zd.x -= eta2[j] * s1 * s.x;
			zd.y -= eta2[j] * s1 * s.y;
		}
		if (p.FS4 != nullptr) {
			const C *F4 = p.FS4 + cell * 4 * PP;
			C v = cadd(cscale(cmul(Wh[e], F4[j * PP + e]), eta2[j]), cscale(cmul(Wh[j * PP + e], F4[e]), (R)2.0));
			if (j == 0) {
				C s = czero<C>();
				for (int c = 0; c < 4; c++) s = cadd(s, cmul(Wh[c * PP + e], F4[c * PP + e]));
				v = csub(v, cscale(s, (R)2.0));
			}
			zd.x += s1 * v.x;
			zd.y += s1 * v.y;
		}
		T.a[T.at(li, k)] = zc;
		T.a[T.at(nl + li, k)] = zd;
	}
	__syncthreads();
	const C *r = fft_lines_x<R1, R2, +1>(T.a, T.b, 2 * nl, T.pitch, 1, p.pl, T.tw);
	C *z = p.Z + cj * 2 * PP + (long)l0 * P;
	for (int i = threadIdx.x; i < 2 * nl * P; i += blockDim.x) {
		const int h = i >= nl * P ? 1 : 0, rem = i - h * nl * P, li = fdiv(rem, mgP), k = rem - li * P;
		z[h * PP + (long)li * P + k] = r[T.at(h * nl + li, k)];
	}
}

// assembly columns: inverse column transforms of Zcc_j, Zcd_j, Extract, and
// the outputs (mode 0: Cc = s1 Zcc, Cd = Zcd; mode 1: base + dtc (Cc + Cd + CB))
template <class C, int R1, int R2> __global__ void __launch_bounds__(kThreads) k_any_asm_cols(const AsmP<C> p) {
	extern __shared__ __align__(16) unsigned char sm[];
	const int N = p.N, P = 2 * N, nl = p.nl;
	const long PP = (long)P * P, NN = (long)N * N;
	Tile<C> T(sm, P, 2 * nl);
	const unsigned mgP = magic_div((unsigned)P), mgnl = magic_div((unsigned)nl);
	load_tw(T.tw, P, p.pl);
	const int bpg = P / nl;
	const long cj = blockIdx.x / bpg;
	const int k0 = (int)(blockIdx.x % bpg) * nl;
	const long cell = cj / 4;
	const int j = (int)(cj % 4);
	const C *z = p.Z + cj * 2 * PP;
	for (int i = threadIdx.x; i < 2 * nl * P; i += blockDim.x) {
		const int h = i >= nl * P ? 1 : 0, rem = i - h * nl * P, l = fdiv(rem, mgnl), kk = rem - l * nl;
		T.a[T.at(h * nl + kk, l)] = z[h * PP + (long)l * P + k0 + kk];
	}
	__syncthreads();
	const C *r = fft_lines_x<R1, R2, +1>(T.a, T.b, 2 * nl, T.pitch, 1, p.pl, T.tw);
	for (int i = threadIdx.x; i < nl * P; i += blockDim.x) {
		const int l = fdiv(i, mgnl), kk = i - l * nl;
		const int ls = src_idx(l, N), ks = src_idx(k0 + kk, N);
		if (ls < 0 || ks < 0) continue;
		const C zc = r[T.at(kk, l)], zd = r[T.at(nl + kk, l)];
		const double2 cc = make_double2(p.s1 * (double)zc.x, p.s1 * (double)zc.y);
		const double2 cd = make_double2((double)zd.x, (double)zd.y);
		const long q = (long)ls * N + ks, o = cj * NN + q;
		if (p.mode == 0) {
			if (p.out_cc) p.out_cc[o] = cc;
			if (p.out_cd) p.out_cd[o] = cd;
		} else {
			const double2 *w = p.wcur + cell * 4 * NN + q;
			double2 cb = make_double2(0.0, 0.0);         // -i [B, W] = 2 (B x w) . sigma
			if (p.B != nullptr) {
				const double *B = p.B + cell * 3;
				if (j == 1) cb = make_double2(2 * (B[1] * w[3 * NN].x - B[2] * w[2 * NN].x), 2 * (B[1] * w[3 * NN].y - B[2] * w[2 * NN].y));
				if (j == 2) cb = make_double2(2 * (B[2] * w[1 * NN].x - B[0] * w[3 * NN].x), 2 * (B[2] * w[1 * NN].y - B[0] * w[3 * NN].y));
				if (j == 3) cb = make_double2(2 * (B[0] * w[2 * NN].x - B[1] * w[1 * NN].x), 2 * (B[0] * w[2 * NN].y - B[1] * w[1 * NN].y));
			}
			const double2 b = p.base ? p.base[o] : make_double2(0.0, 0.0);
			p.out[o] = make_double2(b.x + p.dtc * ((cc.x + cd.x) + cb.x), b.y + p.dtc * ((cc.y + cd.y) + cb.y));
		}
	}
}

// the Fourier representation (upstream simulation.c:224-283): real N x N
// components -> complex grids, and the Hermitian completion of the forward
// transform scaled by 1 / N^2
__global__ void k_any_real_to_cplx(long n, const double *__restrict__ v, double2 *__restrict__ c) {
	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) c[i] = make_double2(v[i], 0.0);
}
__global__ void k_any_hermitian(int N, long ngrids, const double2 *__restrict__ a, double2 *__restrict__ f) {
	const long NN = (long)N * N, n = ngrids * NN;
	const double sc = 1.0 / ((double)N * N);
	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
		const long g = i / NN;
		const int l = (int)((i % NN) / N), k = (int)(i % N);
		double2 z;
		if (k <= N / 2) {
			z = a[i];
		} else {
			const int lc = (N - l) % N, kc = N - k;
			z = a[g * NN + (long)lc * N + kc];
			z.y = -z.y;
		}
		f[i] = make_double2(z.x * sc, z.y * sc);
	}
}
__global__ void k_any_real_part(long n, const double2 *__restrict__ c, double *__restrict__ v) {
	for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) v[i] = c[i].x;
}

// ---------------------------------------------------------------------------
// host side

bool smooth23(int L) {
	if (L < 2) return false;
	while (L % 2 == 0) L /= 2;
	while (L % 3 == 0) L /= 3;
	return L == 1;
}

// radix plans of a length: variant 0 the fewest stages (the largest of 16,
// 12, 8, 6, 4, 3, 2 that divides what is left, first: 48 = 16 3, 96 = 16 6,
// 192 = 16 12, 256 = 16 16); variant 1 radix 8 first, then 4, 2, 3; variant 2
// the radix-3 stages first; variant 3 radix 4 instead of 8
Plan make_plan(int L, int variant) {
	Plan p;
	p.L = L;
	int a = 0, b = 0, m = L;
	while (m % 2 == 0) { m /= 2; a++; }
	while (m % 3 == 0) { m /= 3; b++; }
	if (m != 1) QB_FAIL("transform length " + std::to_string(L) + " is not of the form 2^a 3^b");
	int rad[kMaxStages], n = 0;
	auto push = [&](int r) {
		if (n >= kMaxStages) QB_FAIL("transform length " + std::to_string(L) + " needs too many stages");
		rad[n++] = r;
	};
	if (variant == 0) {
		int left = L;
		while (left > 1) {
			for (int r : { 16, 12, 8, 6, 4, 3, 2 })
				if (left % r == 0) { push(r); left /= r; break; }
		}
	} else {
		if (variant == 2) for (int i = 0; i < b; i++) push(3);
		int e = a;
		if (variant != 3) while (e >= 3) { push(8); e -= 3; }
		while (e >= 2) { push(4); e -= 2; }
		if (e == 1) push(2);
		if (variant != 2) for (int i = 0; i < b; i++) push(3);
	}
	p.nst = n;
	for (int i = 0; i < n; i++) p.r[i] = rad[i];
	return p;
}

// lines per tile: the largest of the candidates that divides L and fits
int pick_lines(int L, int want, int tiles, size_t elem) {
	for (int nl = want; nl >= 1; nl--) {
		if (L % nl) continue;
		if (elem * ((size_t)L + 2 * (size_t)tiles * nl * tile_pitch(L)) <= kMaxSmem) return nl;
	}
	return 1;
}

template <class K> void smem_attr(K kern, size_t bytes) {
	static std::mutex mu;
	static std::set<std::tuple<int, const void *>> done;
	int dev = 0;
	QB_CUDA(cudaGetDevice(&dev));
	std::lock_guard<std::mutex> lk(mu);
	if (done.insert(std::make_tuple(dev, (const void *)kern)).second) {
		QB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem));
		// occupancy is bound by shared memory, not by L1 hits (the tiles are read once)
		QB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
	}
	(void)bytes;
}

template <class K, class Prm> void launch(K kern, const char *name, long blocks, size_t smem, cudaStream_t s, const Prm &p) {
	if (blocks <= 0) return;
	smem_attr(kern, smem);
	ProfScope ps(name, s);
	kern<<<(unsigned)blocks, kThreads, smem, s>>>(p);
	QB_CUDA(cudaGetLastError());
}

template <class C> struct Tabs;
template <> struct Tabs<double2> {
	static const double *i1_psi2(const DevI1 &t) { return t.psi2.as<double>(); }
	static const double *i1_phi(const DevI1 &t) { return t.phi.as<double>(); }
	static const double *i2_psi1(const DevI2 &t) { return t.psi1.as<double>(); }
	static const double *i2_psi2(const DevI2 &t) { return t.psi2.as<double>(); }
	static const double2 *i3_psi1(const DevI3 &t) { return t.psi1.as<double2>(); }
	static const double *i3_psi2T(const DevI3 &t) { return t.psi2T.as<double>(); }
};
template <> struct Tabs<float2> {
	static const float *i1_psi2(const DevI1 &t) { return t.psi2f.as<float>(); }
	static const float *i1_phi(const DevI1 &t) { return t.phif.as<float>(); }
	static const float *i2_psi1(const DevI2 &t) { return t.psi1f.as<float>(); }
	static const float *i2_psi2(const DevI2 &t) { return t.psi2f.as<float>(); }
	static const float2 *i3_psi1(const DevI3 &t) { return t.psi1f.as<float2>(); }
	static const float *i3_psi2T(const DevI3 &t) { return t.psi2Tf.as<float>(); }
};

template <class C> struct AnyRhs {
	using R = typename CT<C>::R;
	Workspace &ws;
	const QuadSet &q;
	int N, P, ncells;
	long PP;
	Plan pl;
	int nl1;              // lines per tile of the single-tile passes
	cudaStream_t s;

	AnyRhs(Workspace &w, const QuadSet &qs, int nc, cudaStream_t st) : ws(w), q(qs), N(w.N), P(2 * w.N), ncells(nc), s(st) {
		PP = (long)P * P;
		pl = with_tw(make_plan(P, ws.anyn_plan));
		// lines per tile: the workspace's knob, else QB_ANYN_LINES (read per
		// call, for comparisons), else tiles of about 4096 (FP32) or 2048 (FP64)
		// elements.  The FP32 passes keep 4 CTAs an SM, and 16 lines of 192 or
		// 256 give their radix-16 stages 192 or 256 butterflies a CTA instead of
		// 96 or 128: 1.3x at N = 96 and 1.24x at N = 128 over 8 lines; the FP64
		// passes (2 CTAs an SM) were slower with 16.
		const int env_lines = (int)env_mb("QB_ANYN_LINES");
		const int def_lines = std::max(1, (sizeof(C) == 8 ? 4096 : 2048) / P);
		nl1 = pick_lines(P, ws.anyn_lines > 0 ? ws.anyn_lines : env_lines > 0 ? env_lines : def_lines, 1, sizeof(C));
	}
	Plan with_tw(Plan p) const {
		p.twd = ws.anyn_tw.as<double2>();
		p.twf = reinterpret_cast<const float2 *>(p.twd + P);
		return p;
	}
	size_t smem(int nl, int tiles) const { return tile_bytes<C>(P, nl * tiles); }
	// runs f on the instantiation of a pass kernel for the plan's two stages
	// (16 3, 16 6, 16 12, 16 16), else on the run-time-plan one
	template <class F, class K> void by_plan(const F &f, K k3, K k6, K k12, K k16, K kany) const {
		switch (two_stage_key(pl)) {
		case 3: f(k3); break;
		case 6: f(k6); break;
		case 12: f(k12); break;
		case 16: f(k16); break;
		default: f(kany);
		}
	}
	long blocks(long units, int nl) const { return units * (P / nl); }

	static double env_mb(const char *name) {
		const char *e = getenv(name);
		return e != nullptr ? atof(e) : 0.0;
	}
	// the wave's scratch in bytes, within L2: the workspace's knob, else
	// QB_ANYN_WAVE_MB (read per call), else 64 MB (at N = 48 in FP32, 0.82
	// against 0.90 ms per cell-evaluation with 32 MB)
	double wave_budget() const {
		const double mb = ws.anyn_wave_mb > 0 ? ws.anyn_wave_mb : env_mb("QB_ANYN_WAVE_MB");
		return (mb > 0 ? mb : 64.0) * 1048576.0;
	}
	// terms per wave: the wave's scratch of `per_term` grids per cell for nc cells within the budget
	int wave(int nterms, int per_term, int nc = -1) const {
		const double per = (double)per_term * (nc < 0 ? ncells : nc) * PP * sizeof(C);
		const int nt = (int)std::max(1.0, std::floor(wave_budget() / per));
		return std::min(nt, std::max(1, nterms));
	}
	// cells per wave: all of them, unless one term of the batch needs more
	// scratch than the cap (QB_ANYN_SLICE_MB, read per call, else 4 GB); then
	// equal slices of the batch within it.  Slices within the L2 budget were
	// measured slower (N = 96 and 128: more, smaller launches cost more than
	// the L2 misses they save), so the cap only bounds the scratch memory.
	int wave_cells(int per_term) const {
		const double mb = env_mb("QB_ANYN_SLICE_MB");
		const double cap = (mb > 0 ? mb : 4096.0) * 1048576.0;
		const double per = (double)per_term * PP * sizeof(C);
		const int fit = (int)std::max(1.0, std::floor(cap / per));
		if (fit >= ncells) return ncells;
		const int nslices = (ncells + fit - 1) / fit;
		return (ncells + nslices - 1) / nslices;
	}

	// kind != null: grids [cell][gpc / nsub][nsub], and the cells of kind 0
	// skip the subs from rf_grids on
	// zband: the grids come from k_any_pad_rows (column passes only)
	void plain(C *g, long ngrids, int dir, bool cols, const int *kind = nullptr, long gpc = 1, int nsub = 1, int rf_grids = 1,
	           bool zband = false) {
		PlainP<C> p{};
		p.g = g; p.L = P; p.nl = nl1; p.pl = pl;
		p.kind = kind; p.gpc = gpc; p.nsub = nsub; p.rf_grids = rf_grids;
		p.zband = (zband && cols) ? N : 0;
		const long nb = blocks(ngrids, nl1);
		const size_t sm = smem(nl1, 1);
		auto go = [&](const char *name) { return [&, name](auto kern) { launch(kern, name, nb, sm, s, p); }; };
		if (dir < 0) {
			if (cols) by_plan(go("any_cols"), k_any_plain<C, -1, true, 16, 3>, k_any_plain<C, -1, true, 16, 6>, k_any_plain<C, -1, true, 16, 12>,
			                  k_any_plain<C, -1, true, 16, 16>, k_any_plain<C, -1, true, 0, 0>);
			else by_plan(go("any_rows"), k_any_plain<C, -1, false, 16, 3>, k_any_plain<C, -1, false, 16, 6>, k_any_plain<C, -1, false, 16, 12>,
			             k_any_plain<C, -1, false, 16, 16>, k_any_plain<C, -1, false, 0, 0>);
		} else {
			if (cols) by_plan(go("any_cols"), k_any_plain<C, +1, true, 16, 3>, k_any_plain<C, +1, true, 16, 6>, k_any_plain<C, +1, true, 16, 12>,
			                  k_any_plain<C, +1, true, 16, 16>, k_any_plain<C, +1, true, 0, 0>);
			else by_plan(go("any_rows"), k_any_plain<C, +1, false, 16, 3>, k_any_plain<C, +1, false, 16, 6>, k_any_plain<C, +1, false, 16, 12>,
			             k_any_plain<C, +1, false, 16, 16>, k_any_plain<C, +1, false, 0, 0>);
		}
	}

	PadRowsP<C> pad_params(const double2 *W, int nt, int t0, int nsub, C *out) const {
		PadRowsP<C> p{};
		p.W = W; p.w_cell = 4L * N * N; p.N = N; p.nl = nl1; p.nt = nt; p.t0 = t0; p.nsub = nsub; p.out = out; p.pl = pl;
		return p;
	}
	void pad_rows(const PadRowsP<C> &p, int nc = -1) {
		by_plan([&](auto kern) { launch(kern, "any_pad_rows", blocks((long)(nc < 0 ? ncells : nc) * p.nt * p.nsub, nl1), smem(nl1, 1), s, p); },
		        k_any_pad_rows<C, 16, 3>, k_any_pad_rows<C, 16, 6>, k_any_pad_rows<C, 16, 12>, k_any_pad_rows<C, 16, 16>,
		        k_any_pad_rows<C, 0, 0>);
	}

	void spectra(const double2 *W) {
		ws.What.ensure(sizeof(C) * 4 * ncells * PP);
		PadRowsP<C> p = pad_params(W, 1, 0, 4, ws.What.as<C>());
		for (int c = 0; c < 4; c++) { p.comp[c] = c; p.psel[c] = 0; }
		pad_rows(p);
		plain(ws.What.as<C>(), 4L * ncells, -1, true, nullptr, 1, 1, 1, true);
	}

	// I1-type sums into S [cell][ntask] and their forward transforms into FS
	void i1_sums(const DevI1 &t, const double2 *W, bool cc, DevBuf &Sbuf, DevBuf &FSbuf) {
		const int ntask = cc ? 3 : 4;
		Sbuf.ensure(sizeof(C) * ncells * ntask * PP);
		QB_CUDA(cudaMemsetAsync(Sbuf.p, 0, sizeof(C) * ncells * ntask * PP, s));
		const int cpw = wave_cells(ntask);                  // waves of terms and, if need be, slices of cells
		const int nt = wave(t.nterms, ntask, cpw);
		ws.wave1.ensure(sizeof(C) * (size_t)cpw * nt * ntask * PP);
		C *G = ws.wave1.as<C>();
		for (int c0 = 0; c0 < ncells; c0 += cpw) {
			const int nc = std::min(cpw, ncells - c0);
			for (int t0 = 0; t0 < t.nterms; t0 += nt) {
				const int n = std::min(nt, t.nterms - t0);
				PadRowsP<C> p = pad_params(W + (long)c0 * 4 * N * N, n, t0, ntask, G);
				for (int k = 0; k < ntask; k++) { p.comp[k] = cc ? std::min(k + 1, 3) : k; p.psel[k] = 1; }
				p.psiA = Tabs<C>::i1_psi2(t);
				pad_rows(p, nc);
				I1ColsP<C> c{};
				c.g = G; c.What = ws.What.as<C>() + (long)c0 * 4 * PP; c.N = N; c.nl = nl1; c.nt = n; c.nsub = ntask; c.fcomp = 0;
				c.fa = cc ? -4.0 : 2.0; c.fb = cc ? 2.0 : -1.0; c.pl = pl;
				by_plan([&](auto kern) { launch(kern, "any_i1_cols", blocks((long)nc * n * ntask, nl1), smem(nl1, 1), s, c); },
		        k_any_i1_cols<C, 16, 3>, k_any_i1_cols<C, 16, 6>, k_any_i1_cols<C, 16, 12>, k_any_i1_cols<C, 16, 16>, k_any_i1_cols<C, 0, 0>);
				I1RowsP<C> r{};
				r.g = G; r.S = Sbuf.as<C>() + (long)c0 * ntask * PP; r.phi = Tabs<C>::i1_phi(t); r.N = N; r.nl = nl1; r.nt = n; r.t0 = t0;
				r.nsub = ntask; r.pl = pl;
				by_plan([&](auto kern) { launch(kern, "any_i1_rows", blocks((long)nc * ntask, nl1), smem(nl1, 1), s, r); },
		        k_any_i1_rows<C, 16, 3>, k_any_i1_rows<C, 16, 6>, k_any_i1_rows<C, 16, 12>, k_any_i1_rows<C, 16, 16>, k_any_i1_rows<C, 0, 0>);
			}
		}
		FSbuf.ensure(sizeof(C) * ncells * ntask * PP);
		QB_CUDA(cudaMemcpyAsync(FSbuf.p, Sbuf.p, sizeof(C) * ncells * ntask * PP, cudaMemcpyDeviceToDevice, s));
		plain(FSbuf.as<C>(), (long)ncells * ntask, -1, false);
		plain(FSbuf.as<C>(), (long)ncells * ntask, -1, true);
	}

	void i2_sums(const DevI2 &t, const double2 *W) {
		ws.i2p.ensure(sizeof(C) * ncells * 4 * PP);
		QB_CUDA(cudaMemsetAsync(ws.i2p.p, 0, sizeof(C) * ncells * 4 * PP, s));
		const int cpw = wave_cells(8);                      // waves of terms and, if need be, slices of cells
		const int nt = wave(t.nterms, 8, cpw);
		ws.wave1.ensure(sizeof(C) * (size_t)cpw * nt * 8 * PP);
		C *G = ws.wave1.as<C>();
		const int nl2 = pick_lines(P, nl1, 2, sizeof(C));
		for (int c0 = 0; c0 < ncells; c0 += cpw) {
			const int nc = std::min(cpw, ncells - c0);
			for (int t0 = 0; t0 < t.nterms; t0 += nt) {
				const int n = std::min(nt, t.nterms - t0);
				PadRowsP<C> p = pad_params(W + (long)c0 * 4 * N * N, n, t0, 8, G);
				for (int i = 0; i < 4; i++) { p.comp[2 * i] = i; p.psel[2 * i] = 1; p.comp[2 * i + 1] = i; p.psel[2 * i + 1] = 2; }
				p.psiA = Tabs<C>::i2_psi1(t); p.psiB = Tabs<C>::i2_psi2(t);
				pad_rows(p, nc);
				I2ColsP<C> c{};
				c.g = G; c.Q = ws.i2p.as<C>() + (long)c0 * 4 * PP; c.N = N; c.nl = nl2; c.nt = n; c.pl = pl;
				by_plan([&](auto kern) { launch(kern, "any_i2_cols", blocks((long)nc * 4, nl2), smem(nl2, 2), s, c); },
		        k_any_i2_cols<C, 16, 3>, k_any_i2_cols<C, 16, 6>, k_any_i2_cols<C, 16, 12>, k_any_i2_cols<C, 16, 16>, k_any_i2_cols<C, 0, 0>);
			}
		}
	}

	// whole-grid chains (k_any_i3_fused, where a grid fits a CTA) or the three
	// passes.  The workspace's knob (0 off, 1 on), else QB_ANYN_FUSED (read per
	// call), else the three passes: measured faster in FP32 at N = 24 (0.216
	// against 0.316 ms per cell-evaluation) and N = 48 (0.710 against 0.807)
	// once the passes read and store from their FFT stages, and faster still
	// with their plans compiled in
	bool fused_i3() const {
		int on = ws.anyn_fused;
		if (on < 0) {
			const char *e = getenv("QB_ANYN_FUSED");
			if (e != nullptr && (strcmp(e, "0") == 0 || strcmp(e, "1") == 0)) on = e[0] - '0';
		}
		if (on < 0) on = 0;
		return on == 1 && tile_bytes<C>(P, P) <= kMaxSmem;
	}

	// returns the partials of X per (cell, j).  FP32: the cells of kind 0 (no
	// Nyquist content, Hermitian state) take the real form, two chains packed
	// in one complex transform, the others the complex chains, in the same
	// launches (the kernels read a cell's kind; the real form leaves half of
	// its units idle)
	int i3_sums(const DevI3 &t, const double2 *W) {
		const int nxp = fused_i3() ? 4 : 1;
		ws.i3p.ensure(sizeof(C) * ncells * 4 * nxp * PP);
		QB_CUDA(cudaMemsetAsync(ws.i3p.p, 0, sizeof(C) * ncells * 4 * nxp * PP, s));
		const int *kind = nullptr;
		if constexpr (sizeof(typename CT<C>::R) == 4) {
			if (real_form_enabled()) kind = i3_form_kinds(ws, ncells, W, s);
		}
		i3_waves(t, W, nxp, kind);
		return nxp;
	}

	// the I3 chains in waves of terms and, where one term of the batch
	// overflows the scratch cap, slices of cells.  Per (cell, term): 4 grids
	// of Pg (P_0..P_3, or the packed P_0 + i P_1, P_2 + i P_3 of the real
	// form) and 16 chains (8 in the real form).  A cell's terms still run in
	// order, so the sums do not depend on the waves.
	void i3_waves(const DevI3 &t, const double2 *W, int nxp, const int *kind) {
		const bool fused = nxp == 4;
		const int per_term = fused ? 4 : 20;
		const int cpw = wave_cells(per_term);
		const int nt = wave(t.nterms, per_term, cpw);
		ws.wave1.ensure(sizeof(C) * (size_t)cpw * nt * 4 * PP);                // P_j
		if (!fused) ws.wave2.ensure(sizeof(C) * (size_t)cpw * nt * 16 * PP);   // chains
		C *Pg = ws.wave1.as<C>(), *Y = fused ? nullptr : ws.wave2.as<C>();
		int nl4 = nl1;                                      // one tile, at most kOwn elements a thread
		const int own = own_for_plan(pl, sizeof(C) == 16);
		while (nl4 > 1 && (nl4 * P > own * kThreads || P % nl4)) nl4--;
		for (int c0 = 0; c0 < ncells; c0 += cpw) {
			const int nc = std::min(cpw, ncells - c0);
			const double2 *Wc = W + (long)c0 * 4 * N * N;
			const C *What = ws.What.as<C>() + (long)c0 * 4 * PP;
			C *X = ws.i3p.as<C>() + (long)c0 * 4 * nxp * PP;
			const int *kc = kind ? kind + c0 : nullptr;
			for (int t0 = 0; t0 < t.nterms; t0 += nt) {
				const int n = std::min(nt, t.nterms - t0);
				PadRowsP<C> p = pad_params(Wc, n, t0, 4, Pg);
				for (int g = 0; g < 4; g++) { p.comp[g] = g; p.comp2[g] = g; p.psel[g] = 3; }
				p.kind = kc; p.nsub_rf = 2;
				for (int g = 0; g < 2; g++) { p.comp_rf[g] = 2 * g; p.comp2_rf[g] = 2 * g + 1; p.psel_rf[g] = 4; }
				p.psiC = Tabs<C>::i3_psi1(t);
				pad_rows(p, nc);
				plain(Pg, (long)nc * n * 4, -1, true, kc, (long)n * 4, 4, 2, true);
				if (fused) {
					I3FusedP<C> f{};
					f.What = What; f.Pg = Pg; f.X = X;
					f.psi2T = Tabs<C>::i3_psi2T(t); f.idx = t.idx.as<int>(); f.scale = t.scale.as<double>();
					f.N = N; f.nt = n; f.t0 = t0; f.kind = kc;
					// FP32 default: radix-8 stages (the radix-16 register DFTs push this
					// kernel to 173 registers, one CTA an SM); FP64 runs one CTA an SM anyway
					f.pl = (ws.anyn_plan == 0 && sizeof(C) == 8) ? with_tw(make_plan(P, 1)) : pl;
					launch(k_any_i3_fused<C>, "any_i3_fused", (long)nc * 16, tile_bytes<C>(P, P), s, f);
					continue;
				}
				I3RowsAP<C> a{};
				a.What = What; a.Pg = Pg; a.Y = Y; a.N = N; a.nl = nl1; a.nt = n; a.kind = kc; a.pl = pl;
				by_plan([&](auto kern) { launch(kern, "any_i3_rows_a", blocks((long)nc * n * 16, nl1), smem(nl1, 1), s, a); },
				        k_any_i3_rows_a<C, 16, 3>, k_any_i3_rows_a<C, 16, 6>, k_any_i3_rows_a<C, 16, 12>, k_any_i3_rows_a<C, 16, 16>,
				        k_any_i3_rows_a<C, 0, 0>);
				I3ColsP<C> c{};
				c.Y = Y; c.psi2T = Tabs<C>::i3_psi2T(t); c.idx = t.idx.as<int>(); c.scale = t.scale.as<double>();
				c.N = N; c.nl = nl1; c.nt = n; c.t0 = t0; c.kind = kc; c.pl = pl;
				by_plan([&](auto kern) { launch(kern, "any_i3_cols", blocks((long)nc * n * 16, nl1), smem(nl1, 1), s, c); },
				        k_any_i3_cols<C, 16, 3>, k_any_i3_cols<C, 16, 6>, k_any_i3_cols<C, 16, 12>, k_any_i3_cols<C, 16, 16>,
				        k_any_i3_cols<C, 0, 0>);
				I3RowsBP<C> b{};
				b.Y = Y; b.Pg = Pg; b.X = X; b.N = N; b.nl = nl4; b.nt = n; b.kind = kc; b.pl = pl;
				by_plan([&](auto kern) { launch(kern, "any_i3_rows_b", blocks((long)nc * 4, nl4), smem(nl4, 1), s, b); },
				        k_any_i3_rows_b<C, 16, 3>, k_any_i3_rows_b<C, 16, 6>, k_any_i3_rows_b<C, 16, 12>,
				        k_any_i3_rows_b<C, 16, 16>, k_any_i3_rows_b<C, 0, 0>);
			}
		}
	}

	AsmP<C> prepare(const double2 *W, int parts) {
		if (sizeof(C) == 8) prepare_f32_tables(q, s);
		spectra(W);
		AsmP<C> a{};
		a.What = ws.What.as<C>();
		if ((parts & RHS_CC) && q.i1) { i1_sums(*q.i1, W, true, ws.i1cc, ws.fs); a.FS = ws.fs.as<C>(); }
		if (parts & RHS_CD) {
			if (q.i4) { i1_sums(*q.i4, W, false, ws.i1i4, ws.fs4); a.FS4 = ws.fs4.as<C>(); }
			if (q.i2) { i2_sums(*q.i2, W); a.Q = ws.i2p.as<C>(); }
			if (q.i3) { a.nxp = i3_sums(*q.i3, W); a.X = ws.i3p.as<C>(); }
		}
		a.N = N;
		a.s2 = 1.0 / (double)PP;
		a.s1 = a.s2 * a.s2;
		a.pl = pl;
		return a;
	}

	void assemble(AsmP<C> &a) {
		const int nl2 = pick_lines(P, nl1, 2, sizeof(C));
		a.nl = nl2;
		ws.wave1.ensure(sizeof(C) * (size_t)ncells * 8 * PP);
		a.Z = ws.wave1.as<C>();
		by_plan([&](auto kern) { launch(kern, "any_asm_rows", blocks((long)ncells * 4, nl2), smem(nl2, 2), s, a); },
		        k_any_asm_rows<C, 16, 3>, k_any_asm_rows<C, 16, 6>, k_any_asm_rows<C, 16, 12>, k_any_asm_rows<C, 16, 16>, k_any_asm_rows<C, 0, 0>);
		by_plan([&](auto kern) { launch(kern, "any_asm_cols", blocks((long)ncells * 4, nl2), smem(nl2, 2), s, a); },
		        k_any_asm_cols<C, 16, 3>, k_any_asm_cols<C, 16, 6>, k_any_asm_cols<C, 16, 12>, k_any_asm_cols<C, 16, 16>, k_any_asm_cols<C, 0, 0>);
	}
};

template <class C>
void any_operators(Workspace &ws, const QuadSet &q, int ncells, const double2 *W, int parts, double2 *cc, double2 *cd, cudaStream_t s) {
	AnyRhs<C> r(ws, q, ncells, s);
	AsmP<C> a = r.prepare(W, parts);
	a.mode = 0; a.out_cc = cc; a.out_cd = cd;
	r.assemble(a);
}

template <class C>
void any_update(Workspace &ws, const QuadSet &q, int ncells, const double2 *base, const double2 *wcur, const double *B, double dtc,
                double2 *out, cudaStream_t s) {
	AnyRhs<C> r(ws, q, ncells, s);
	AsmP<C> a = r.prepare(wcur, RHS_ALL);
	a.mode = 1; a.base = base; a.wcur = wcur; a.B = B; a.dtc = dtc; a.out = out;
	r.assemble(a);
}

unsigned grid1d(long n) { return (unsigned)std::min<long>((n + 255) / 256, 148L * 16); }

}  // namespace

bool anyn_supported(int N) {
	return N >= 4 && N <= 128 && N % 2 == 0 && smooth23(N);
}

void anyn_build_twiddles(Workspace &ws) {
	const int P = 2 * ws.N;
	ws.anyn_tw.ensure(P * (sizeof(double2) + sizeof(float2)));
	double2 *twd = ws.anyn_tw.as<double2>();
	k_any_build_tw<<<1, 256, 0, ws.stream>>>(P, twd, reinterpret_cast<float2 *>(twd + P));
	QB_CUDA(cudaGetLastError());
	QB_CUDA(cudaStreamSynchronize(ws.stream));
}

bool anyn_route(int N) {
	if (N == 8 || N == 16 || N == 32 || N == 64) {
		const char *e = getenv("QB_ANYN");
		return e != nullptr && strcmp(e, "1") == 0;
	}
	return anyn_supported(N);
}

void anyn_operators(Workspace &ws, const QuadSet &q, int ncells, const double2 *W, int parts, double2 *cc, double2 *cd, cudaStream_t s) {
	if (ncells <= 0) return;
	if (ws.prec == 32) any_operators<float2>(ws, q, ncells, W, parts, cc, cd, s);
	else any_operators<double2>(ws, q, ncells, W, parts, cc, cd, s);
}

void anyn_update(Workspace &ws, const QuadSet &q, int ncells, const double2 *base, const double2 *wcur, const double *B, double dtc,
                 double2 *out, cudaStream_t s) {
	if (ncells <= 0) return;
	if (ws.prec == 32) any_update<float2>(ws, q, ncells, base, wcur, B, dtc, out, s);
	else any_update<double2>(ws, q, ncells, base, wcur, B, dtc, out, s);
}

// the Fourier representation at any supported N, through the same passes
// (length-N transforms, FP64), with a scratch grid set kept per device
namespace {
double2 *repr_scratch(long n) {
	static std::mutex mu;
	static DevBuf bufs[64];
	int dev = 0;
	QB_CUDA(cudaGetDevice(&dev));
	std::lock_guard<std::mutex> lk(mu);
	DevBuf &b = bufs[dev & 63];
	if (b.bytes < sizeof(double2) * (size_t)n) b.ensure(sizeof(double2) * (size_t)n);
	return b.as<double2>();
}
void repr_passes(int N, int ngrids, double2 *a, int dir, cudaStream_t s) {
	PlainP<double2> p{};
	p.g = a; p.L = N; p.nl = pick_lines(N, 8, 1, sizeof(double2)); p.pl = make_plan(N, 0);
	const size_t sm = tile_bytes<double2>(N, p.nl);
	const long nb = (long)ngrids * (N / p.nl);
	if (dir < 0) {
		launch(k_any_plain<double2, -1, false, 0, 0>, "any_rows", nb, sm, s, p);
		launch(k_any_plain<double2, -1, true, 0, 0>, "any_cols", nb, sm, s, p);
	} else {
		launch(k_any_plain<double2, +1, false, 0, 0>, "any_rows", nb, sm, s, p);
		launch(k_any_plain<double2, +1, true, 0, 0>, "any_cols", nb, sm, s, p);
	}
}
}  // namespace

void anyn_to_fourier(int N, int ngrids, const double *Wv, double2 *Wf, cudaStream_t s) {
	const long n = (long)ngrids * N * N;
	double2 *a = repr_scratch(n);
	{
		ProfScope ps("any_repr", s);
		k_any_real_to_cplx<<<grid1d(n), 256, 0, s>>>(n, Wv, a);
	}
	QB_CUDA(cudaGetLastError());
	repr_passes(N, ngrids, a, -1, s);
	{
		ProfScope ps("any_repr", s);
		k_any_hermitian<<<grid1d(n), 256, 0, s>>>(N, ngrids, a, Wf);
	}
	QB_CUDA(cudaGetLastError());
}

void anyn_from_fourier(int N, int ngrids, const double2 *Wf, double *Wv, cudaStream_t s) {
	const long n = (long)ngrids * N * N;
	double2 *a = repr_scratch(n);
	QB_CUDA(cudaMemcpyAsync(a, Wf, sizeof(double2) * n, cudaMemcpyDeviceToDevice, s));
	repr_passes(N, ngrids, a, +1, s);
	{
		ProfScope ps("any_repr", s);
		k_any_real_part<<<grid1d(n), 256, 0, s>>>(n, a, Wv);
	}
	QB_CUDA(cudaGetLastError());
}

}  // namespace qb
