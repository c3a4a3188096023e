// qb_dftmma.cu — DFT-as-GEMM on the tensor cores (tcgen05.mma, kind::tf32).
//
// A length-P complex DFT along the rows of a batch of grids is a real GEMM:
// with row vectors x = xr + i xi and F[k][k'] = exp(-2 pi i k k' / P),
//   [yr | yi] = [xr | xi] x [[Fr, Fi], [-Fi, Fr]]        (K = N = 2P).
// The inverse transform is conj(DFT(conj(x))), so one matrix serves both
// directions.  TF32 keeps 10 explicit mantissa bits; three products of a
// hi/lo split, A_hi B_hi + A_hi B_lo + A_lo B_hi with X_hi = tf32(X) and
// X_lo = tf32(X - X_hi), give about 2^-21 relative accuracy per GEMM, which
// the FP32 form's 1e-5 bound allows.
#include "qb_engine.h"
#include "qb_kernels.cuh"
#include "qb_umma.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <mutex>
#include <vector>

extern "C" {
#include "qbgpu.h"
}

namespace qb {
namespace {

constexpr unsigned kWaitPolls = 1u << 24;      // bounded mbarrier waits (about a second)

__device__ __forceinline__ unsigned char *align1024(unsigned char *p) {
	const uintptr_t a = (uintptr_t)p;
	return (unsigned char *)((a + 1023) & ~(uintptr_t)1023);
}

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// D (128 x 64) = A (128 x 64) x B (64 x 64) with B given transposed (Bt: 64 x 64,
// row n = column n of B), one CTA of 128 threads: a check of the K-major
// operand layouts and descriptors on the device.  err[0] is set when the MMA
// did not complete within the poll limit.
__global__ void __launch_bounds__(128, 1) k_umma_selftest(const float *__restrict__ A, const float *__restrict__ Bt,
                                                          float *__restrict__ D, int *err) {
	extern __shared__ unsigned char smem_raw[];
	unsigned char *base = align1024(smem_raw);
	unsigned char *sA = base, *sB = base + 128 * 64 * 4;
	__shared__ uint64_t mbar;
	__shared__ uint32_t tslot;
	const int t = threadIdx.x, warp = t >> 5;
	for (int k = 0; k < 64; k++) {
		const float v = umma::tf32_round(A[t * 64 + k]);
		*reinterpret_cast<float *>(sA + umma::kmajor_off(128, t, k)) = v;
	}
	if (t < 64)
		for (int k = 0; k < 64; k++) *reinterpret_cast<float *>(sB + umma::kmajor_off(64, t, k)) = umma::tf32_round(Bt[t * 64 + k]);
	if (t == 0) {
		umma::mbar_init(&mbar, 1);
		fence_mbar_init();
	}
	if (warp == 0) tmem_alloc(&tslot, 64);
	umma::fence_async_smem();
	tmem_fence_before();
	__syncthreads();
	tmem_fence_after();
	const uint32_t d = tslot;
	if (t == 0) {
		const uint32_t a0 = umma::smem_u32(sA), b0 = umma::smem_u32(sB);
		for (int kk = 0; kk < 8; kk++) {
			const uint64_t ad = umma::desc_sw128(a0 + (kk >> 2) * 16384 + (kk & 3) * 32, 16, 1024);
			const uint64_t bd = umma::desc_sw128(b0 + (kk >> 2) * 8192 + (kk & 3) * 32, 16, 1024);
			umma::mma_tf32(d, ad, bd, umma::idesc_tf32<128, 64>(), kk > 0);
		}
		umma::commit(&mbar);
	}
	__syncwarp();
	const bool ok = umma::mbar_wait(&mbar, 0, kWaitPolls);
	tmem_fence_after();
	if (!ok) {
		if ((t & 31) == 0) atomicExch(err, 1);
	} else {
		for (int c = 0; c < 64; c += 16) {
			float v[16];
			umma::tmem_ld16(d + ((uint32_t)(32 * warp) << 16) + c, v);
			tmem_wait_ld();
#pragma unroll
			for (int i = 0; i < 16; i++) D[t * 64 + c + i] = v[i];
		}
	}
	tmem_fence_before();
	__syncthreads();
	tmem_fence_after();
	if (warp == 0) tmem_dealloc(d, 64);
}

constexpr size_t kSelftestSmem = 128 * 64 * 4 + 64 * 64 * 4 + 1024;

// ---------------------------------------------------------------------------
// I3 sums of the FP32 form at N = 16 (padded grids of P = 32) as DFT-GEMMs.
//
// One CTA per (cell, chunk of terms), two warpgroups.  A tile is 4 grids of
// 32 rows (128 rows, row (q, lane) in tensor-memory lane 32 q + lane); every
// 1-D pass of a chain is one tile GEMM against the real-ified DFT matrix,
// K = N = 64, as 3 x 8 tcgen05.mma of M128 N64 K8 (TF32 hi/lo split).
// Between passes each thread reads its row of D from tensor memory and
// writes the next A tile: its own row (a pass along the same axis) or, for
// a pass along the other axis, one column of the next tile (the transpose).
// The cell's four spectra G_g (32 KB) come into shared memory once, by a
// bulk (TMA) copy.  Per term:
//   P_c = FFT2(Pad(psi1_t . W_c))   warpgroup 0, tile rows (c, k)
//   for combos c = wg, wg + 2:      tile rows (r, k) of outputs r = 0..3
//     a = G_g . P_r -> IFFT along l -> IFFT along k -> x psi2_t
//       -> FFT along k -> FFT along l -> X_r += coef P_a . (result)
// (a thread holds a column of the grid on the passes along l, a row on the
// passes along k, so every shared-memory access of a warp is conflict-free)
// with IFFT = conj . FFT . conj, so one DFT matrix serves every pass.  The
// sums X of a warpgroup live in tensor memory beside its D (row (r, l) of
// X_r: real parts in 32 columns, imaginary parts in the next 32); the two
// warpgroups' sums are added in a fixed order at the end.
namespace dm {
constexpr int P = 32, N = 16, K2 = 2 * P;
constexpr int kThreads = 256;
constexpr uint32_t kTile = 128 * K2 * 4;           // one A operand tile (32 KB)
constexpr uint32_t kBmat = K2 * K2 * 4;            // the DFT matrix (16 KB)
constexpr int kPitch = P + 1;                      // P grids in shared memory (complex pitch)
constexpr uint32_t oBhi = 0, oBlo = kBmat, oA = 2 * kBmat;
constexpr uint32_t oP = oA + 4 * kTile;            // A tiles: [warpgroup][hi, lo]
constexpr uint32_t oG = oP + 4 * P * kPitch * 8;   // the cell's spectra G (4 grids, natural order)
constexpr uint32_t kGBytes = 4 * P * P * 8;
constexpr uint32_t kSmem = oG + kGBytes + 1024;
static_assert(oG % 128 == 0 && kGBytes % 16 == 0, "the TMA tile lands 128-byte aligned");
static_assert(kSmem <= 232448, "dynamic shared memory of one CTA");
constexpr uint32_t kCols = 256;                    // tensor memory: per warpgroup a 64-column D and its 64-column sums X
}  // namespace dm

// the pointer, as a value the compiler cannot follow: per-thread addresses
// derived from it are recomputed where they are used instead of being
// hoisted out of the term and chain loops into (scarce) registers
template <class T> __device__ __forceinline__ T *opaque(T *p) {
	asm volatile("" : "+l"(p));
	return p;
}

__device__ __forceinline__ int pad_src(int p) { return p < dm::N / 2 ? p : (p >= 3 * dm::N / 2 ? p - dm::N : -1); }

__device__ __forceinline__ void wg_sync(int wg) { asm volatile("bar.sync %0, %1;" ::"r"(1 + wg), "r"(128) : "memory"); }

// 4 consecutive complex values x[0..3] at columns k0 .. k0 + 3 (real parts)
// and 32 + k0 .. (imaginary parts, conjugated when `conj`) of row r
__device__ __forceinline__ void put_row4(unsigned char *hi, unsigned char *lo, int r, int k0, const float2 (&x)[4], bool conj) {
	hi = opaque(hi);
	lo = opaque(lo);
	const float s = conj ? -1.0f : 1.0f;
	float4 h, l;
	h.x = umma::tf32_round(x[0].x); l.x = umma::tf32_round(x[0].x - h.x);
	h.y = umma::tf32_round(x[1].x); l.y = umma::tf32_round(x[1].x - h.y);
	h.z = umma::tf32_round(x[2].x); l.z = umma::tf32_round(x[2].x - h.z);
	h.w = umma::tf32_round(x[3].x); l.w = umma::tf32_round(x[3].x - h.w);
	uint32_t o = umma::kmajor_off(128, r, k0);
	*reinterpret_cast<float4 *>(hi + o) = h;
	*reinterpret_cast<float4 *>(lo + o) = l;
	h.x = umma::tf32_round(s * x[0].y); l.x = umma::tf32_round(s * x[0].y - h.x);
	h.y = umma::tf32_round(s * x[1].y); l.y = umma::tf32_round(s * x[1].y - h.y);
	h.z = umma::tf32_round(s * x[2].y); l.z = umma::tf32_round(s * x[2].y - h.z);
	h.w = umma::tf32_round(s * x[3].y); l.w = umma::tf32_round(s * x[3].y - h.w);
	o = umma::kmajor_off(128, r, 32 + k0);
	*reinterpret_cast<float4 *>(hi + o) = h;
	*reinterpret_cast<float4 *>(lo + o) = l;
}

// D = A_lo B_hi + A_hi B_lo + A_hi B_hi over K = 64 (8 steps of 8), issued by one thread
__device__ __forceinline__ void issue_pass(uint32_t d, uint32_t ahi, uint32_t alo, uint32_t bhi, uint32_t blo) {
	constexpr uint32_t id = umma::idesc_tf32<128, 64>();
	uint32_t acc = 0;
#pragma unroll 1
	for (int pass = 0; pass < 3; pass++) {
		const uint32_t a = pass == 0 ? alo : ahi, b = pass == 1 ? blo : bhi;
#pragma unroll
		for (int kk = 0; kk < 8; kk++) {
			const uint64_t ad = umma::desc_sw128(a + (kk >> 2) * (128 * 128) + (kk & 3) * 32, 16, 1024);
			const uint64_t bd = umma::desc_sw128(b + (kk >> 2) * (64 * 128) + (kk & 3) * 32, 16, 1024);
			umma::mma_tf32(d, ad, bd, id, acc);
			acc = 1;
		}
	}
}

struct MmaCtx {
	int wg;
	bool issuer;
	uint32_t dcol, trow, ahi, alo, bhi, blo;
	uint64_t *mbar;
	volatile int *abort;          // this warpgroup's flag: set on a wait that ran out
	unsigned phase;
};

// one pass: the staged A tile times the DFT matrix into D.  A wait that runs
// out marks the warpgroup aborted; later passes then issue and wait for
// nothing (every barrier still runs).  Threads then read their row of D from
// tensor memory, 16 columns at a time (real parts at columns 0..31,
// imaginary parts at 32..63).
__device__ __forceinline__ void mma_pass(MmaCtx &c) {
	umma::fence_async_smem();
	tmem_fence_before();
	wg_sync(c.wg);
	tmem_fence_after();
	const bool skip = *c.abort != 0;
	if (!skip) {
		if (c.issuer) {
			issue_pass(c.dcol, c.ahi, c.alo, c.bhi, c.blo);
			umma::commit(c.mbar);
		}
		__syncwarp();
		if (!umma::mbar_wait(c.mbar, c.phase, kWaitPolls)) *c.abort = 1;
		c.phase ^= 1u;
		tmem_fence_after();
	}
}

// values h*16 .. h*16 + 15 of this thread's row of D: re[i] = Re, im[i] = Im
__device__ __forceinline__ void d_half(const MmaCtx &c, int h, float (&re)[16], float (&im)[16]) {
	umma::tmem_ld16(c.trow + 16 * h, re);
	umma::tmem_ld16(c.trow + 32 + 16 * h, im);
	tmem_wait_ld();
}

// the transpose, streamed from tensor memory: value j of this thread's row of
// D becomes column `col` (real) and 32 + col (imaginary) of row r0 + j of the
// next A tile
__device__ __forceinline__ void put_col_d(const MmaCtx &c, unsigned char *hi, unsigned char *lo, int r0, int col) {
#pragma unroll
	for (int h = 0; h < 2; h++) {
		float re[16], im[16];
		d_half(c, h, re, im);
		hi = opaque(hi);
		lo = opaque(lo);
#pragma unroll
		for (int i = 0; i < 16; i++) {
			const int j = 16 * h + i;
			const float hr = umma::tf32_round(re[i]), hm = umma::tf32_round(im[i]);
			const uint32_t o0 = umma::kmajor_off(128, r0 + j, col), o1 = umma::kmajor_off(128, r0 + j, 32 + col);
			*reinterpret_cast<float *>(hi + o0) = hr;
			*reinterpret_cast<float *>(lo + o0) = umma::tf32_round(re[i] - hr);
			*reinterpret_cast<float *>(hi + o1) = hm;
			*reinterpret_cast<float *>(lo + o1) = umma::tf32_round(im[i] - hm);
		}
	}
}

__global__ void __launch_bounds__(dm::kThreads, 1) k_i3_mma32(const I3ParamsT<float2> p, int *err, const __grid_constant__ CUtensorMap tmG) {
	using namespace dm;
	extern __shared__ unsigned char smem_raw[];
	unsigned char *base = align1024(smem_raw);
	__shared__ uint64_t mbar[3];                                // [0], [1]: MMA completion per warpgroup; [2]: the G copy
	__shared__ uint32_t tslot;
	__shared__ int abort_flag[2];
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, wg = warp >> 2, q = warp & 3;
	const long cid = blockIdx.x;
	const int chunk = (int)(cid % p.nchunk);
	const long cell = cid / p.nchunk;
	const int t0 = (int)((long)chunk * p.nterms / p.nchunk), t1 = (int)((long)(chunk + 1) * p.nterms / p.nchunk);
	unsigned char *Ahi = base + oA + wg * 2 * kTile, *Alo = Ahi + kTile;
	float2 *Pg = reinterpret_cast<float2 *>(base + oP);       // [4][P][kPitch], P_c[l][k] natural
	const float2 *Gs = reinterpret_cast<const float2 *>(base + oG);   // the cell's 4 spectra G_g, natural [4][P][P]
	if (tid == 0) {
		umma::mbar_init(&mbar[0], 1);
		umma::mbar_init(&mbar[1], 1);
		umma::mbar_init(&mbar[2], 1);
		fence_mbar_init();
		abort_flag[0] = abort_flag[1] = 0;
		// the cell's spectra G: a 128-row tile of the spectra tensor (rows of 32
		// complex values, 4 grids a cell) into shared memory by one TMA copy
		umma::tma_load_2d(base + oG, &tmG, 0, (int)(cell * 4 * P), &mbar[2], kGBytes);
	}
	// the real-ified DFT matrix B (K x N) as its transpose, row n = column n of B, split hi / lo
	for (int i = tid; i < K2 * K2; i += kThreads) {
		const int n = i / K2, k = i % K2;
		const int e = ((k & 31) * (n & 31)) & (P - 1);
		double sn, cs;
		sincospi(2.0 * e / P, &sn, &cs);                     // F = exp(-2 pi i e / P) = cs - i sn
		const double fr = cs, fi = -sn;
		const double v = k < 32 ? (n < 32 ? fr : fi) : (n < 32 ? -fi : fr);
		const float h = umma::tf32_round((float)v);
		const float l = umma::tf32_round((float)(v - (double)h));
		const uint32_t o = umma::kmajor_off(64, n, k);
		*reinterpret_cast<float *>(base + oBhi + o) = h;
		*reinterpret_cast<float *>(base + oBlo + o) = l;
	}
	if (warp == 0) tmem_alloc(&tslot, kCols);
	umma::fence_async_smem();
	tmem_fence_before();
	__syncthreads();
	tmem_fence_after();
	MmaCtx mc;
	mc.wg = wg;
	mc.issuer = (tid & 127) == 0;
	mc.dcol = tslot + 64u * wg;
	mc.trow = mc.dcol + ((uint32_t)(32 * q) << 16);
	mc.ahi = umma::smem_u32(Ahi); mc.alo = umma::smem_u32(Alo);
	mc.bhi = umma::smem_u32(base + oBhi); mc.blo = umma::smem_u32(base + oBlo);
	mc.mbar = &mbar[wg];
	mc.abort = &abort_flag[wg];
	mc.phase = 0;
	if (!umma::mbar_wait(&mbar[2], 0, kWaitPolls)) abort_flag[wg] = 1;    // G in shared memory
	const int row = 32 * q + lane;
	const uint32_t xrow = mc.trow + 128;                       // this thread's row of X (sums)
	int ncmax = 0;
	for (int r = 0; r < 4; r++) ncmax = max(ncmax, p.ncombo[r]);
	{
		float z[16];
#pragma unroll
		for (int i = 0; i < 16; i++) z[i] = 0.0f;
#pragma unroll
		for (int c = 0; c < 64; c += 16) umma::tmem_st16(xrow + c, z);
		tmem_wait_st();
	}
#pragma unroll 1
	for (int t = t0; t < t1; t++) {
		if (wg == 0) {
			// P_q = FFT2(Pad(psi1_t . W_q)): tile row (q, k = lane) holds column k of the padded
			// grid; the pass along l, then (transposed) along k leaves row (q, l) of P_q
			const double2 *src = p.src + cell * p.src_cell + (long)p.src_comp[q] * N * N;
			const float2 *ps1 = p.psi1 + (long)t * N * N;
			const int ks = pad_src(lane);
#pragma unroll 1
			for (int l0 = 0; l0 < P; l0 += 4) {
				float2 x[4];
#pragma unroll
				for (int i = 0; i < 4; i++) {
					const int ls = pad_src(l0 + i);
					x[i] = make_float2(0.0f, 0.0f);
					if (ls >= 0 && ks >= 0) {
						const double2 w = src[ks + N * ls];
						x[i] = cmul(ps1[ks + N * ls], make_float2((float)w.x, (float)w.y));
					}
				}
				put_row4(Ahi, Alo, row, l0, x, false);
			}
			mma_pass(mc);                                       // along l: row (q, k)
			put_col_d(mc, Ahi, Alo, 32 * q, lane);
			mma_pass(mc);                                       // along k: row (q, l = lane) of P_q over k
#pragma unroll
			for (int h = 0; h < 2; h++) {
				float re[16], im[16];
				d_half(mc, h, re, im);
				float2 *pr = opaque(Pg + (q * P + lane) * kPitch + 16 * h);
#pragma unroll
				for (int i = 0; i < 16; i++) pr[i] = make_float2(re[i], im[i]);
			}
		}
		__syncthreads();                                        // P grids of the term are in place
		const float *ps2 = opaque(p.psi2T + (long)p.psi2_idx[t] * P * P + lane);   // psi2[l = lane][k] at ps2[k * P]
		const float sc = (float)p.psi2_scale[t];
#pragma unroll 1
		for (int c = wg; c < ncmax; c += 2) {
			const bool act = c < p.ncombo[q];
			// column k = lane of a = G_g . P_q, conjugated (inverse transforms as conj . FFT . conj)
			{
				const float2 *Gg = opaque(Gs + (act ? p.cgi[q][c] : 0) * P * P + lane);
				const float2 *Pq = opaque(Pg + q * P * kPitch + lane);
#pragma unroll 1
				for (int l0 = 0; l0 < P; l0 += 4) {
					float2 x[4];
#pragma unroll
					for (int i = 0; i < 4; i++) x[i] = act ? cmul(Gg[(l0 + i) * P], Pq[(l0 + i) * kPitch]) : make_float2(0.0f, 0.0f);
					put_row4(Ahi, Alo, row, l0, x, true);
				}
			}
			mma_pass(mc);                                       // along l: row (q, k)
			put_col_d(mc, Ahi, Alo, 32 * q, lane);
			mma_pass(mc);                                       // along k: row (q, l = lane), conj IFFT2(a) over k
			// IFFT2(a) . psi2_t (the conjugate of D), as the operand of the forward pass along k
#pragma unroll
			for (int h = 0; h < 2; h++) {
				float re[16], im[16];
				d_half(mc, h, re, im);
#pragma unroll
				for (int i0 = 0; i0 < 16; i0 += 4) {
					float2 x[4];
#pragma unroll
					for (int i = 0; i < 4; i++) {
						const float f = sc * ps2[(16 * h + i0 + i) * P];
						x[i] = make_float2(re[i0 + i] * f, im[i0 + i] * f);
					}
					put_row4(Ahi, Alo, row, 16 * h + i0, x, true);
				}
			}
			mma_pass(mc);                                       // FFT along k: row (q, l)
			put_col_d(mc, Ahi, Alo, 32 * q, lane);
			mma_pass(mc);                                       // FFT along l: row (q, k = lane) over l
			if (act) {
				const float2 *Pa = opaque(Pg + p.ca[q][c] * P * kPitch + lane);
				const float coef = (float)p.ccoef[q][c];
#pragma unroll
				for (int h = 0; h < 2; h++) {                    // l = 16 h .. 16 h + 15
					float xr[16], xi[16], re[16], im[16];
					d_half(mc, h, re, im);
					umma::tmem_ld16(xrow + 16 * h, xr);
					umma::tmem_ld16(xrow + 32 + 16 * h, xi);
					tmem_wait_ld();
#pragma unroll
					for (int i = 0; i < 16; i++) {
						const int l = 16 * h + i;
						const float2 y = cmul(Pa[l * kPitch], make_float2(re[i], im[i]));
						xr[i] += coef * y.x;
						xi[i] += coef * y.y;
					}
					umma::tmem_st16(xrow + 16 * h, xr);
					umma::tmem_st16(xrow + 32 + 16 * h, xi);
				}
				tmem_wait_st();
			}
		}
		__syncthreads();                                        // every chain of the term is done with Pg
	}
	// the two warpgroups' sums (column k = lane of X_q), added in a fixed order (0 + 1)
	float *red = reinterpret_cast<float *>(base + oA);          // the operand tiles are free now
	if (wg == 1) {
#pragma unroll
		for (int c = 0; c < 64; c += 16) {
			float x[16];
			umma::tmem_ld16(xrow + c, x);
			tmem_wait_ld();
#pragma unroll
			for (int i = 0; i < 16; i++) red[(c + i) * 128 + row] = x[i];
		}
	}
	__syncthreads();
	const bool failed = abort_flag[0] != 0 || abort_flag[1] != 0;
	if (wg == 0) {
		float2 *o = p.out + ((cell * p.nchunk + chunk) * 4 + q) * (long)P * P + lane;
		const float nanv = __int_as_float(0x7fc00000);
#pragma unroll
		for (int h = 0; h < 2; h++) {
			float xr[16], xi[16];
			umma::tmem_ld16(xrow + 16 * h, xr);
			umma::tmem_ld16(xrow + 32 + 16 * h, xi);
			tmem_wait_ld();
#pragma unroll
			for (int i = 0; i < 16; i++) {
				const int l = 16 * h + i;
				o[l * P] = failed ? make_float2(nanv, nanv) : make_float2(xr[i] + red[l * 128 + row], xi[i] + red[(32 + l) * 128 + row]);
			}
		}
	}
	if (failed) {
		if (tid == 0) atomicExch(err, 1);
		// an MMA may still be in flight after a wait ran out: give it one more bounded wait
		if ((tid & 127) == 0 && abort_flag[wg]) umma::mbar_wait(&mbar[wg], mc.phase, kWaitPolls);
	}
	tmem_fence_before();
	__syncthreads();
	tmem_fence_after();
	if (warp == 0) tmem_dealloc(tslot, kCols);
}

}  // namespace

// the driver's tensor-map encoder, through the runtime's entry-point query
PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
	static std::mutex mu;
	static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
	std::lock_guard<std::mutex> lk(mu);
	if (fn == nullptr) {
		void *f = nullptr;
		cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
		QB_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q));
		if (f == nullptr || q != cudaDriverEntryPointSuccess) QB_FAIL("cuTensorMapEncodeTiled is not available");
		fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
	}
	return fn;
}

// the spectra of ncells cells ([cell][4][P][P] complex FP32) as a 2-D tensor
// of FP32 values: rows of 2P floats, 4P rows a cell; the box is one cell
CUtensorMap spectra_map(const float2 *G, long ncells) {
	using namespace dm;
	CUtensorMap m;
	const cuuint64_t dims[2] = { (cuuint64_t)(2 * P), (cuuint64_t)(ncells * 4 * P) };
	const cuuint64_t strides[1] = { (cuuint64_t)(2 * P * sizeof(float)) };
	const cuuint32_t box[2] = { (cuuint32_t)(2 * P), (cuuint32_t)(4 * P) };
	const cuuint32_t estr[2] = { 1, 1 };
	const CUresult r = tmap_encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float2 *>(G), dims, strides, box, estr,
	                                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
	                                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
	if (r != CUDA_SUCCESS) QB_FAIL("cuTensorMapEncodeTiled failed for the spectra map (" + std::to_string((int)r) + ")");
	return m;
}

// launcher (engine): ncl = cells x chunks CTAs
void launch_i3_mma32(const I3ParamsT<float2> &p, long ncl, int *err, cudaStream_t s) {
	static bool attr_done[64] = {};
	int dev = 0;
	QB_CUDA(cudaGetDevice(&dev));
	if (!attr_done[dev & 63]) {
		QB_CUDA(cudaFuncSetAttribute(k_i3_mma32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dm::kSmem));
		attr_done[dev & 63] = true;
	}
	if (p.g_cell != 4L * dm::P * dm::P) QB_FAIL("k_i3_mma32: the spectra must be [cell][4][P][P]");
	const CUtensorMap tmG = spectra_map(p.Ghat, ncl / p.nchunk);
	ProfScope ps("i3_cluster", s);
	k_i3_mma32<<<(unsigned)ncl, dm::kThreads, dm::kSmem, s>>>(p, err, tmG);
	QB_CUDA(cudaGetLastError());
}

// the tensor-memory kernels of this file, for the co-residency check of the engine
std::vector<TmemKernel> dftmma_tmem_kernels() {
	return { { (const void *)k_i3_mma32, dm::kSmem, dm::kThreads, (int)dm::kCols, "k_i3_mma32" },
	         { (const void *)k_umma_selftest, kSelftestSmem, 128, 64, "k_umma_selftest" } };
}

}  // namespace qb

namespace {
template <class F> int guarded_dm(F &&f) {
	try {
		f();
		return 0;
	} catch (const std::exception &) {
		return -1;
	}
}
}  // namespace

extern "C" int qb_umma_selftest(const float *A, const float *Bt, float *D, void *stream) {
	return guarded_dm([&] {
		if (A == nullptr || Bt == nullptr || D == nullptr) QB_FAIL("qb_umma_selftest: null pointer");
		cudaStream_t s = (cudaStream_t)stream;
		int *err = nullptr;
		QB_CUDA(cudaMallocAsync(&err, sizeof(int), s));
		QB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
		QB_CUDA(cudaFuncSetAttribute(qb::k_umma_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)qb::kSelftestSmem));
		qb::k_umma_selftest<<<1, 128, qb::kSelftestSmem, s>>>(A, Bt, D, err);
		QB_CUDA(cudaGetLastError());
		int h = 0;
		QB_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s));
		QB_CUDA(cudaStreamSynchronize(s));
		cudaFreeAsync(err, s);
		if (h) QB_FAIL("qb_umma_selftest: the tensor-core MMA did not complete within the poll limit");
	});
}
