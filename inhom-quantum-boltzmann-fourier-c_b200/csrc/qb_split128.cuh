// qb_split128.cuh — collision kernels for N = 64 (padded grids of 128 x 128),
// each grid split over a pair of CTAs of a thread-block cluster.
//
// A padded FP64 grid is 256 KB, more than one CTA's shared memory, so the two
// CTAs of a pair (h = 0, 1) hold one half each (64 rows x pitch 129):
//   A layout (the padded side where Pad, psi and Extract act): CTA h holds
//     rows 64h .. 64h + 63 (row = slow index l) at local row l - 64h; A-layout
//     grids in global memory are natural (index k + 128 l).
//   B layout (the transformed side): CTA h holds rows 2m + h at local row m;
//     B-layout grids in global memory store half h contiguously,
//     index (64 h + m) * 128 + k.
// A 2-D transform is a 128-point transform along k (local: fft128), a radix-2
// butterfly along l between rows l' and l' + 64 (the only step that crosses
// the pair), and a 64-point transform along l' (local: fft1d<64> on columns):
//   forward A -> B: butterfly (decimation in frequency), column FFT64, row FFT128
//   inverse B -> A: row FFT128, column FFT64, butterfly (decimation in time)
// The forward butterfly of a padded input needs no exchange: with N = 64
// exactly one of rows l' and l' + 64 of Pad(x) is non-zero, so each CTA forms
// its half from the N-grid in global memory.  In the I3 pair chain the
// inverse butterfly, the psi2 multiply and the next forward butterfly are one
// exchange between the pair.
//
// Every kernel here runs 512 threads per CTA.  Row passes: 16 lanes per row
// (thread t: row t/16 of 32 per iteration, lane t%16), 2 iterations.  Column
// passes: 8 lanes per column (column t/8 of 64 per iteration), 2 iterations.
// Accumulators of the I1/I2 sums live in global memory (L2) as
// read-modify-write of the caller's partial-sum slot owned by the thread (a
// 16-point accumulator per thread would not fit the FP64 register budget of
// 128); those of the I3 sums live in tensor memory.
//
// Cluster barriers: every loop that contains one has a trip count that is
// uniform over the cluster (chunk bounds per cluster, combo count = the
// largest over the cluster, fixed rounds), and no CTA returns early.
#pragma once
#include "qb_kernels.cuh"

namespace qb {

struct G128 {
	static constexpr int P = 128, N = 64, H = 64, LDP = 129, NT = 512;
	static constexpr int GRID_H = H * LDP;      // shared-memory slots of a half grid
	static constexpr long PP = (long)P * P;
	// padded index -> N-grid index, or -1 inside the zero band
	__device__ __forceinline__ static int src(int p) { return p < N / 2 ? p : (p >= 3 * N / 2 ? p - N : -1); }
	// N-grid index -> padded index (GridZeroPad)
	__device__ __forceinline__ static int pad(int k) { return k < N / 2 ? k : k + N; }
	// global index of a B-layout element (half h, local row m, column k)
	__device__ __forceinline__ static long bidx(int h, int m, int k) { return (long)(h * H + m) * P + k; }
};

// dynamic shared memory of every 128 kernel: half grid + twiddles of 128 and 64
template <class C> constexpr size_t smem128() { return sizeof(C) * ((size_t)G128::GRID_H + 128 + 64); }

__device__ __forceinline__ double2 shfl_xor_c(double2 v, int m) {
	return make_double2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}
__device__ __forceinline__ float2 shfl_xor_c(float2 v, int m) {
	return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

// output position of value e of lane tau after fft128
__device__ __forceinline__ int pos128(int tau, int e) { return 2 * ((tau & 7) + 8 * e) + (tau >> 3); }

// 128-point transform (direction DIR) of x[r] = a[tau + 16 r] held by lane
// tau of a 16-lane group: radix-2 decimation in frequency in registers
// (pairs n, n + 64 are x[r], x[r + 4] of the same lane), an exchange with
// lane tau ^ 8 by shuffle (lanes 0-7 keep the even half, 8-15 the odd half),
// then fft1d<64> on each 8-lane half.  Output e is A[pos128(tau, e)].  `line`:
// the 128-slot row used as scratch (contents destroyed).  All 32 lanes of the
// warp must call it.
template <int DIR, class C>
__device__ __forceinline__ void fft128(C (&x)[8], int tau, C *line, const C *tw128, const C *tw64) {
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
	fft1d<64, DIR>(x, tau & 7, line + h * 64, 1, tw64);
}

// reorder fft128 outputs (positions pos128) into the input layout tau + 16 r
template <class C>
__device__ __forceinline__ void out_to_in128(C (&x)[8], int tau, C *line) {
	__syncwarp();
#pragma unroll
	for (int e = 0; e < 8; e++) line[pos128(tau, e)] = x[e];
	__syncwarp();
#pragma unroll
	for (int r = 0; r < 8; r++) x[r] = line[tau + 16 * r];
	__syncwarp();
}

template <class C> __device__ __forceinline__ void init_tw128(C *tw128, C *tw64) {
	init_twiddles<128>(tw128);
	init_twiddles<64>(tw64);
}

template <class C> __device__ __forceinline__ C conj_c(C a) { a.y = -a.y; return a; }

// column FFT64 (direction DIR) over the 64 local rows of every column of S, in
// place; the loader supplies the 8 inputs of a lane (rows tau + 8 r)
template <int DIR, class C, class Load>
__device__ __forceinline__ void col_pass(C *S, const C *tw64, const Load &load) {
	using G = G128;
	const int tau = threadIdx.x & 7;
#pragma unroll 1
	for (int it = 0; it < 2; it++) {
		const int col = it * 64 + (threadIdx.x >> 3);
		C x[8];
		load(x, col, tau);
		fft1d<64, DIR>(x, tau, S + col, G::LDP, tw64);
#pragma unroll
		for (int e = 0; e < 8; e++) S[(tau + 8 * e) * G::LDP + col] = x[e];
	}
}

// rows of S as the loader of a column pass
template <class C> struct ColFromS {
	const C *S;
	__device__ __forceinline__ void operator()(C (&x)[8], int col, int tau) const {
#pragma unroll
		for (int r = 0; r < 8; r++) x[r] = S[(tau + 8 * r) * G128::LDP + col];
	}
};

// Forward-transform input of half h straight from an N-grid in global memory:
// the decimation-in-frequency butterfly of rows l', l' + 64 of Pad(mul . src)
// (only one of them is non-zero: row l' of the N-grid, + for l' < 32, - else):
// h = 0 keeps a + b, h = 1 keeps (a - b) w^l'.
template <class C, class Mul> struct ColFromPad {
	const double2 *src; Mul mul; int h; const C *tw128;
	__device__ __forceinline__ void operator()(C (&x)[8], int col, int tau) const {
		const int sk = G128::src(col);
#pragma unroll
		for (int r = 0; r < 8; r++) {
			const int l = tau + 8 * r;
			C v = czero<C>();
			if (sk >= 0) v = mul(sk + G128::N * l, src[sk + G128::N * l]);
			if (h) {
				v = cmul(v, tw128[l]);
				if (l >= 32) { v.x = -v.x; v.y = -v.y; }
			}
			x[r] = v;
		}
	}
};

// Forward-transform input of half h from the sum of nparts natural (A-layout)
// P x P grids in global memory: butterfly of rows l', l' + 64.
template <class C> struct ColFromSum {
	const C *in; long part_stride; int nparts; int h; const C *tw128;
	__device__ __forceinline__ C at(int l, int k) const {
		C s = in[(long)l * G128::P + k];
		for (int q = 1; q < nparts; q++) s = cadd(s, in[q * part_stride + (long)l * G128::P + k]);
		return s;
	}
	__device__ __forceinline__ void operator()(C (&x)[8], int col, int tau) const {
#pragma unroll
		for (int r = 0; r < 8; r++) {
			const int l = tau + 8 * r;
			const C a = at(l, col), b = at(l + 64, col);
			x[r] = h ? cmul(csub(a, b), tw128[l]) : cadd(a, b);
		}
	}
};

// row pass over the 64 local rows: x[r] = S[row][tau + 16 r] (or the loader's
// values), fft128, then the epilogue gets the outputs (positions pos128)
template <int DIR, class C, class Load, class Epi>
__device__ __forceinline__ void row_pass(C *S, const C *tw128, const C *tw64, const Load &load, const Epi &epi) {
	using G = G128;
	const int tau = threadIdx.x & 15;
#pragma unroll 1
	for (int it = 0; it < 2; it++) {
		const int row = it * 32 + (threadIdx.x >> 4);
		C x[8];
		load(x, row, tau);
		fft128<DIR>(x, tau, S + row * G::LDP, tw128, tw64);
		epi(x, row, tau);
	}
}

template <class C> struct RowFromS {
	const C *S;
	__device__ __forceinline__ void operator()(C (&x)[8], int row, int tau) const {
#pragma unroll
		for (int r = 0; r < 8; r++) x[r] = S[row * G128::LDP + tau + 16 * r];
	}
};
template <class C> struct RowToS {
	C *S;
	__device__ __forceinline__ void operator()(C (&x)[8], int row, int tau) const {
#pragma unroll
		for (int e = 0; e < 8; e++) S[row * G128::LDP + pos128(tau, e)] = x[e];
	}
};
// store a B-layout half to global
template <class C> struct RowToB {
	C *out; int h;
	__device__ __forceinline__ void operator()(C (&x)[8], int row, int tau) const {
#pragma unroll
		for (int e = 0; e < 8; e++) out[G128::bidx(h, row, pos128(tau, e))] = x[e];
	}
};

// One exchange between the pair: every thread visits the (l', k) points of
// the half grid in two rounds of 8; a round reads S and the partner's S at
// the same point, the cluster barrier lets both CTAs finish reading, then
// op's results are written back.  ALONG_L: consecutive threads run along l'
// (conflict-free column access, coalesced transposed tables); else along k.
template <bool ALONG_L, class C, class Op>
__device__ __forceinline__ void pair_exchange(C *S, const C *peer, cg::cluster_group &cl, const Op &op) {
	using G = G128;
#pragma unroll 1
	for (int round = 0; round < 2; round++) {
		cl.sync();
		C res[8];
#pragma unroll
		for (int i = 0; i < 8; i++) {
			const int idx = round * 4096 + i * 512 + (int)threadIdx.x;
			const int l = ALONG_L ? (idx & 63) : (idx >> 7);
			const int k = ALONG_L ? (idx >> 6) : (idx & 127);
			res[i] = op(S[l * G::LDP + k], peer[l * G::LDP + k], l, k);
		}
		cl.sync();
#pragma unroll
		for (int i = 0; i < 8; i++) {
			const int idx = round * 4096 + i * 512 + (int)threadIdx.x;
			const int l = ALONG_L ? (idx & 63) : (idx >> 7);
			const int k = ALONG_L ? (idx >> 6) : (idx & 127);
			S[l * G::LDP + k] = res[i];
		}
	}
	__syncthreads();
}

// The same exchange for FP64 with the partner's half brought in by bulk
// copies (the tensor-memory-access engine, cp.async.bulk between the
// shared memories of the pair) instead of per-thread loads from distributed
// shared memory.  A round covers columns 64 round .. 64 round + 63 of the 64
// local rows: 64 threads each push one 1 KB row segment of their CTA's half
// into the partner's landing buffer Lb (row pitch 65 values: the column
// reads of the op are conflict-free), completing on the partner's mbarrier;
// each CTA waits for its own incoming 64 KB, computes, waits until its
// outgoing copies have read their source, then overwrites its half.  One
// cluster barrier per round keeps the landing buffers free.  A wait that runs
// out sets *abort (the kernel then stops waiting) and the error word.
constexpr int kLbPitch = 65;
constexpr size_t kLbBytes = sizeof(double2) * 64 * kLbPitch;

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint32_t map_peer(uint32_t local, int rank) {
	uint32_t r;
	asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(rank));
	return r;
}
__device__ __forceinline__ bool mbar_wait_parity(uint32_t mb, unsigned parity, unsigned limit) {
	for (unsigned i = 0; i < limit; i++) {
		uint32_t done = 0;
		asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
		             : "=r"(done) : "r"(mb), "r"(parity) : "memory");
		if (done) return true;
	}
	return false;
}

template <class Op>
__device__ __forceinline__ void pair_exchange_bulk(double2 *S, double2 *Lb, uint64_t *mbar, unsigned &phase, int prank,
                                                   cg::cluster_group &cl, volatile int *abort, int *err, const Op &op) {
	using G = G128;
	const int tid = (int)threadIdx.x;
	const uint32_t mb = smem_addr(mbar);
	const uint32_t lb_remote = map_peer(smem_addr(Lb), prank), mb_remote = map_peer(mb, prank);
#pragma unroll 1
	for (int round = 0; round < 2; round++) {
		// this thread's writes of the half (and reads of the landing buffer) are ordered before the
		// bulk copies, which go through the async proxy
		asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
		cl.sync();                                   // both halves final, the partner's landing buffer free
		const bool skip = *abort != 0;
		if (tid == 0)
			asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(64u * 64u * 16u) : "memory");
		if (tid < 64) {
			const uint32_t src = smem_addr(S + tid * G::LDP + 64 * round);
			const uint32_t dst = lb_remote + (uint32_t)(tid * kLbPitch * sizeof(double2));
			asm volatile("cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
			             ::"r"(dst), "r"(src), "r"(1024u), "r"(mb_remote) : "memory");
			asm volatile("cp.async.bulk.commit_group;" ::: "memory");
		}
		if (!skip && !mbar_wait_parity(mb, phase, 1u << 24)) {
			*abort = 1;
			atomicExch(err, 1);
		}
		phase ^= 1u;
		double2 res[8];
#pragma unroll
		for (int i = 0; i < 8; i++) {
			const int idx = i * 512 + tid;
			const int l = idx & 63, kk = idx >> 6, k = 64 * round + kk;
			res[i] = op(S[l * G::LDP + k], Lb[l * kLbPitch + kk], l, k);
		}
		if (tid < 64) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
		__syncthreads();
#pragma unroll
		for (int i = 0; i < 8; i++) {
			const int idx = i * 512 + tid;
			const int l = idx & 63, k = 64 * round + (idx >> 6);
			S[l * G::LDP + k] = res[i];
		}
	}
	__syncthreads();
}

// value of the inverse (decimation-in-time) butterfly at row l' of half h:
// CTA 0 holds E (even spectral rows), CTA 1 holds O; y[l'] = E + w'^l' O,
// y[l' + 64] = E - w'^l' O with w' = exp(+2 pi i / 128)
template <class C>
__device__ __forceinline__ C dit_value(C own, C oth, int l, int h, const C *tw128) {
	const C w = conj_c(tw128[l]);
	return h ? csub(oth, cmul(w, own)) : cadd(own, cmul(w, oth));
}

// ---------------------------------------------------------------------------
// K1 (128): padded forward spectra out[b] = FFT2(Pad(src[b])) in B layout,
// one CTA pair per grid
template <class C>
__global__ void __launch_bounds__(512, 1) k_pad_fft128(const double2 *__restrict__ src, C *__restrict__ out) {
	using G = G128;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *S = reinterpret_cast<C *>(smem_raw), *tw128 = S + G::GRID_H, *tw64 = tw128 + 128;
	const int h = (int)(blockIdx.x & 1);
	const long b = blockIdx.x >> 1;
	init_tw128(tw128, tw64);
	__syncthreads();
	col_pass<-1>(S, tw64, ColFromPad<C, MulNone<C>>{src + b * G::N * G::N, MulNone<C>{}, h, tw128});
	__syncthreads();
	row_pass<-1>(S, tw128, tw64, RowFromS<C>{S}, RowToB<C>{out + b * G::PP, h});
}

// K5 (128): out[b] = FFT2(sum of nparts natural grids) in B layout
template <class C>
__global__ void __launch_bounds__(512, 1) k_fft_full128(const FullParamsT<C> p) {
	using G = G128;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *S = reinterpret_cast<C *>(smem_raw), *tw128 = S + G::GRID_H, *tw64 = tw128 + 128;
	const int h = (int)(blockIdx.x & 1);
	const long b = blockIdx.x >> 1;
	init_tw128(tw128, tw64);
	__syncthreads();
	col_pass<-1>(S, tw64, ColFromSum<C>{p.in + b * p.grid_stride, p.part_stride, p.nparts, h, tw128});
	__syncthreads();
	row_pass<-1>(S, tw128, tw64, RowFromS<C>{S}, RowToB<C>{p.out + b * G::PP, h});
}

// ---------------------------------------------------------------------------
// K2 (128): I1/I4-type term sums, one CTA pair per (cell, task, chunk):
//   out (natural) = sum_t phi_t . IFFT2(F . FFT2(Pad(psi2_t . g)))
template <class C>
__global__ void __launch_bounds__(512, 1) k_i1_terms128(const I1ParamsT<C> p) {
	using G = G128;
	using R = typename CT<C>::R;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *S = reinterpret_cast<C *>(smem_raw), *tw128 = S + G::GRID_H, *tw64 = tw128 + 128;
	cg::cluster_group cl = cg::this_cluster();
	const int h = (int)cl.block_rank();
	const C *peer = cl.map_shared_rank(S, h ^ 1);
	const long unit = blockIdx.x >> 1;
	const int chunk = (int)(unit % p.nchunk);
	const int task = (int)((unit / p.nchunk) % p.ntask);
	const long cell = unit / ((long)p.nchunk * p.ntask);
	init_tw128(tw128, tw64);
	const C *W = p.What + cell * p.w_cell + (long)p.f_comp * G::PP;
	const R fa = (R)p.fa, fb = (R)p.fb;
	const double2 *g = p.g + cell * p.g_cell + (long)p.g_comp[task] * G::N * G::N;
	C *acc = p.out + ((cell * p.ntask + task) * p.nchunk + chunk) * G::PP;
	const int t0 = (int)((long)chunk * p.nterms / p.nchunk), t1 = (int)((long)(chunk + 1) * p.nterms / p.nchunk);
	// zero this CTA's half of the accumulator (points visited by the exchange below)
	for (int i = threadIdx.x; i < 64 * 128; i += 512) acc[(long)(h * 64 + (i >> 7)) * G::P + (i & 127)] = czero<C>();
	__syncthreads();
#pragma unroll 1
	for (int t = t0; t < t1; t++) {
		col_pass<-1>(S, tw64, ColFromPad<C, MulReal<C>>{g, MulReal<C>{p.psi2 + (long)t * G::N * G::N}, h, tw128});
		__syncthreads();
		// rows: forward FFT, multiply by F = fa W^ + fb, inverse FFT
		row_pass<-1>(S, tw128, tw64, RowFromS<C>{S}, [&](C (&x)[8], int row, int tau) {
#pragma unroll
			for (int e = 0; e < 8; e++) {
				const C w = W[G::bidx(h, row, pos128(tau, e))];
				C f; f.x = fa * w.x + fb; f.y = fa * w.y;
				x[e] = cmul(f, x[e]);
			}
			C *line = S + row * G::LDP;
			out_to_in128(x, tau, line);
			fft128<+1>(x, tau, line, tw128, tw64);
#pragma unroll
			for (int e = 0; e < 8; e++) line[pos128(tau, e)] = x[e];
		});
		__syncthreads();
		col_pass<+1>(S, tw64, ColFromS<C>{S});
		// exchange: the inverse butterfly gives A rows l' (h = 0) or l' + 64 (h = 1);
		// accumulate phi_t . y into this half of the accumulator, S unchanged
		const R *phi = p.phi + (long)t * G::PP;
		pair_exchange<false>(S, peer, cl, [&](C own, C oth, int l, int k) {
			const C y = dit_value(own, oth, l, h, tw128);
			const long o = (long)(h * 64 + l) * G::P + k;
			const R f = phi[o];
			C a = acc[o];
			a.x += f * y.x; a.y += f * y.y;
			acc[o] = a;
			return own;
		});
	}
}

// ---------------------------------------------------------------------------
// K3 (128): I2-type term sums, one CTA pair per (cell, task, chunk):
//   out (B) = sum_t FFT2(Pad(psi1_t . f)) . FFT2(Pad(psi2_t . g));
// the first spectrum goes through tmp (one P x P grid per pair)
template <class C>
__global__ void __launch_bounds__(512, 1) k_i2_terms128(const I2ParamsT<C> p, C *tmp) {
	using G = G128;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *S = reinterpret_cast<C *>(smem_raw), *tw128 = S + G::GRID_H, *tw64 = tw128 + 128;
	const int h = (int)(blockIdx.x & 1);
	const long unit = blockIdx.x >> 1;
	const int chunk = (int)(unit % p.nchunk);
	const int task = (int)((unit / p.nchunk) % p.ntask);
	const long cell = unit / ((long)p.nchunk * p.ntask);
	init_tw128(tw128, tw64);
	const double2 *f = p.src + cell * p.cell_stride + (long)p.f_comp[task] * G::N * G::N;
	const double2 *g = p.src + cell * p.cell_stride + (long)p.g_comp[task] * G::N * G::N;
	C *acc = p.out + ((cell * p.ntask + task) * p.nchunk + chunk) * G::PP;
	C *T1 = tmp + unit * G::PP;
	const int t0 = (int)((long)chunk * p.nterms / p.nchunk), t1 = (int)((long)(chunk + 1) * p.nterms / p.nchunk);
	{   // zero this CTA's half of the accumulator at the row-pass points
		const int tau = threadIdx.x & 15;
		for (int it = 0; it < 2; it++) {
			const int row = it * 32 + (threadIdx.x >> 4);
			for (int e = 0; e < 8; e++) acc[G::bidx(h, row, pos128(tau, e))] = czero<C>();
		}
	}
	__syncthreads();
#pragma unroll 1
	for (int t = t0; t < t1; t++) {
		col_pass<-1>(S, tw64, ColFromPad<C, MulReal<C>>{f, MulReal<C>{p.psi1 + (long)t * G::N * G::N}, h, tw128});
		__syncthreads();
		row_pass<-1>(S, tw128, tw64, RowFromS<C>{S}, RowToB<C>{T1, h});
		__syncthreads();
		col_pass<-1>(S, tw64, ColFromPad<C, MulReal<C>>{g, MulReal<C>{p.psi2 + (long)t * G::N * G::N}, h, tw128});
		__syncthreads();
		row_pass<-1>(S, tw128, tw64, RowFromS<C>{S}, [&](C (&x)[8], int row, int tau) {
#pragma unroll
			for (int e = 0; e < 8; e++) {
				const long o = G::bidx(h, row, pos128(tau, e));
				acc[o] = cfma(T1[o], x[e], acc[o]);
			}
		});
		__syncthreads();
	}
}

// tensor-memory accumulators of k_i3_128: CPP components x 2 row iterations
// x 8 values per thread; the four warps of a lane quarter split the columns
// (512 columns for FP64 with two components per pair, 256 for FP32)
template <class C, int CPP> struct I3Tmem128 {
	static constexpr unsigned WPC = sizeof(C) / 4;
	static constexpr unsigned PER_THREAD = CPP * 16 * WPC;
	static constexpr unsigned NCOLS = 4 * PER_THREAD;
	static_assert(NCOLS <= 512, "tensor memory holds 512 columns");
	__device__ __forceinline__ static unsigned addr(unsigned base, int q, int it, int e) {
		const unsigned w = threadIdx.x >> 5;
		return base + ((32u * (w & 3u)) << 16) + (w >> 2) * PER_THREAD + (unsigned)((q * 2 + it) * 8 + e) * WPC;
	}
};

// ---------------------------------------------------------------------------
// K4 (128): I3-type sums on a cluster of NPAIR CTA pairs; pair q holds the
// CS / NPAIR components q * CS / NPAIR ... in turn.  Per term each pair writes
// the P_r = FFT2(Pad(psi1_t . src_r)) of its components (B layout) to the
// cluster's scratch in global memory (L2); after a cluster barrier every pair
// runs the combos of its components
//   X_r += coef P_a . FFT2(psi2_t . IFFT2(G_g . P_r))
// with one pair exchange each (inverse butterfly, psi2, forward butterfly).
// Components with fewer combos than the largest count run the barriers only.
template <int CS, int NPAIR, class C>
__global__ void __launch_bounds__(512, 1) k_i3_128(const I3ParamsT<C> p, C *pscr, int *err) {
	using G = G128;
	using R = typename CT<C>::R;
	constexpr int CPP = CS / NPAIR;             // components per pair
	static_assert(CS % NPAIR == 0, "components must divide over the pairs");
	constexpr bool kBulk = sizeof(C) == 16;     // FP64: the exchange by bulk copies (landing buffer after the twiddles)
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *S = reinterpret_cast<C *>(smem_raw), *tw128 = S + G::GRID_H, *tw64 = tw128 + 128;
	double2 *Lb = reinterpret_cast<double2 *>(tw64 + 64);
	__shared__ __align__(8) uint64_t xmbar;
	__shared__ int xabort;
	unsigned xphase = 0;
	cg::cluster_group cl = cg::this_cluster();
	const int rank = (int)cl.block_rank();
	const int pair = rank >> 1, h = rank & 1;
	const C *peer = cl.map_shared_rank(S, rank ^ 1);
	if (kBulk && threadIdx.x == 0) {
		asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&xmbar)) : "memory");
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
		xabort = 0;
	}
	const long cid = blockIdx.x / (2 * NPAIR);
	const int chunk = (int)(cid % p.nchunk);
	const long cell = cid / p.nchunk;
	init_tw128(tw128, tw64);
	C *Pall = pscr + cid * CS * G::PP;
	const C *Gcell = p.Ghat + cell * p.g_cell;
	const int t0 = (int)((long)chunk * p.nterms / p.nchunk), t1 = (int)((long)(chunk + 1) * p.nterms / p.nchunk);
	int ncmax = 0;
	for (int r = 0; r < CS; r++) ncmax = max(ncmax, p.ncombo[r]);
	const int tau = threadIdx.x & 15;
	// accumulators in tensor memory: value e of row iteration `it` of component q
	using TM = I3Tmem128<C, CPP>;
	__shared__ unsigned tmem_slot;
	const int warp = threadIdx.x >> 5;
	if (warp == 0) tmem_alloc(&tmem_slot, TM::NCOLS);
	tmem_fence_before();
	__syncthreads();
	tmem_fence_after();
	const unsigned tbase = tmem_slot;
#pragma unroll 1
	for (int q = 0; q < CPP; q++)
#pragma unroll 1
		for (int it = 0; it < 2; it++)
#pragma unroll
			for (int e = 0; e < 8; e++) tmem_st(TM::addr(tbase, q, it, e), czero<C>());
	tmem_wait_st();
	__syncthreads();
#pragma unroll 1
	for (int t = t0; t < t1; t++) {
#pragma unroll 1
		for (int q = 0; q < CPP; q++) {
			const int comp = pair * CPP + q;
			const double2 *src = p.src + cell * p.src_cell + (long)p.src_comp[comp] * G::N * G::N;
			col_pass<-1>(S, tw64, ColFromPad<C, MulCplx<C>>{src, MulCplx<C>{p.psi1 + (long)t * G::N * G::N}, h, tw128});
			__syncthreads();
			row_pass<-1>(S, tw128, tw64, RowFromS<C>{S}, RowToB<C>{Pall + comp * G::PP, h});
			__syncthreads();
		}
		cl.sync();                               // every P_r of the term is in global memory
		const R *psi2 = p.psi2T + (long)p.psi2_idx[t] * G::PP;
		const R sc = (R)p.psi2_scale[t];
#pragma unroll 1
		for (int q = 0; q < CPP; q++) {
			const int comp = pair * CPP + q;
			const int nc = p.ncombo[comp];
			const C *Pown = Pall + comp * G::PP;
#pragma unroll 1
			for (int c = 0; c < ncmax; c++) {
				const bool act = c < nc;
				if (act) {
					const C *Gg = Gcell + (long)p.cgi[comp][c] * G::PP;
					// rows: inverse FFT of G_g . P_r
					row_pass<+1>(S, tw128, tw64, [&](C (&x)[8], int row, int tl) {
#pragma unroll
						for (int r = 0; r < 8; r++) {
							const long o = G::bidx(h, row, tl + 16 * r);
							x[r] = cmul(Gg[o], Pown[o]);
						}
					}, RowToS<C>{S});
					__syncthreads();
					col_pass<+1>(S, tw64, ColFromS<C>{S});
				}
				// inverse butterfly -> psi2 -> forward butterfly, one exchange
				auto xop = [&](C own, C oth, int l, int k) {
					if (!act) return own;
					const C E = h ? oth : own, O = h ? own : oth;
					const C w = tw128[l];
					const C wo = cmul(conj_c(w), O);
					const R f0 = sc * psi2[(long)k * G::P + l], f1 = sc * psi2[(long)k * G::P + l + 64];
					const C z0 = cscale(cadd(E, wo), f0), z1 = cscale(csub(E, wo), f1);
					return h ? cmul(csub(z0, z1), w) : cadd(z0, z1);
				};
				if constexpr (kBulk) pair_exchange_bulk(S, Lb, &xmbar, xphase, rank ^ 1, cl, &xabort, err, xop);
				else pair_exchange<true>(S, peer, cl, xop);
				if (act) {
					col_pass<-1>(S, tw64, ColFromS<C>{S});
					__syncthreads();
					const C *Pa = Pall + (long)p.ca[comp][c] * G::PP;
					const R coef = (R)p.ccoef[comp][c];
					row_pass<-1>(S, tw128, tw64, RowFromS<C>{S}, [&](C (&x)[8], int row, int tl) {
						const int it = row >> 5;
						C a[8];
						tmem_ld8(TM::addr(tbase, q, it, 0), a);
						tmem_wait_ld();
#pragma unroll
						for (int e = 0; e < 8; e++) {
							const C v = cmul(Pa[G::bidx(h, row, pos128(tl, e))], x[e]);
							a[e].x += coef * v.x; a[e].y += coef * v.y;
						}
						tmem_st8(TM::addr(tbase, q, it, 0), a);
						tmem_wait_st();
					});
					__syncthreads();
				}
			}
		}
		cl.sync();                               // every pair is done with this term's P grids
	}
	// accumulators -> this CTA's half of the partial-sum slots
#pragma unroll 1
	for (int q = 0; q < CPP; q++) {
		C *acc = p.out + ((cell * p.nchunk + chunk) * CS + pair * CPP + q) * G::PP;
#pragma unroll 1
		for (int it = 0; it < 2; it++) {
			const int row = it * 32 + (threadIdx.x >> 4);
			C a[8];
			tmem_ld8(TM::addr(tbase, q, it, 0), a);
			tmem_wait_ld();
#pragma unroll
			for (int e = 0; e < 8; e++) acc[G::bidx(h, row, pos128(tau, e))] = a[e];
		}
	}
	tmem_fence_before();
	__syncthreads();
	tmem_fence_after();
	if (warp == 0) tmem_dealloc(tbase, TM::NCOLS);
}

// ---------------------------------------------------------------------------
// Inverse transform of the B-layout grid in S to A layout, then the values
// at the N x N extracted points this CTA owns: half h owns N-grid rows
// q in [32 h, 32 h + 32) (padded row q for h = 0, q + 64 for h = 1, both local
// row q), 4 points per thread: point u -> (q = 32 h + (idx >> 6), kq = idx & 63),
// idx = u * 512 + tid.  Leaves S free for reuse (ends with a cluster barrier).
template <class C>
__device__ __forceinline__ void inverse_extract(C *S, const C *peer, cg::cluster_group &cl, int h, const C *tw128, const C *tw64,
                                                C (&val)[4]) {
	using G = G128;
	row_pass<+1>(S, tw128, tw64, RowFromS<C>{S}, RowToS<C>{S});
	__syncthreads();
	col_pass<+1>(S, tw64, ColFromS<C>{S});
	cl.sync();
#pragma unroll
	for (int u = 0; u < 4; u++) {
		const int idx = u * 512 + (int)threadIdx.x;
		const int l = 32 * h + (idx >> 6), k = G::pad(idx & 63);
		val[u] = dit_value(S[l * G::LDP + k], peer[l * G::LDP + k], l, h, tw128);
	}
	cl.sync();
}

// K6 (128): assembly of Cc and Cd for one (cell, component j), one CTA pair;
// same arithmetic as k_assemble (upstream collision.c:95-167, 232-253,
// simulation.c:75-135), spectra in B layout
template <class C>
__global__ void __launch_bounds__(512, 1) k_assemble128(const AsmParamsT<C> p) {
	using G = G128;
	using R = typename CT<C>::R;
	constexpr int N = G::N, NN = N * N;
	constexpr long PP = G::PP;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	C *S = reinterpret_cast<C *>(smem_raw), *tw128 = S + G::GRID_H, *tw64 = tw128 + 128;
	cg::cluster_group cl = cg::this_cluster();
	const int h = (int)cl.block_rank();
	const C *peer = cl.map_shared_rank(S, h ^ 1);
	const long unit = blockIdx.x >> 1;
	const int j = (int)(unit & 3);
	const long cell = unit >> 2;
	init_tw128(tw128, tw64);
	const R eta2[4] = { 2, -2, -2, -2 };
	const R s1 = (R)p.s1, s2 = (R)p.s2;
	const C *Wh = p.What + cell * 4 * PP;
	double2 cc[4], cd[4];
#pragma unroll
	for (int u = 0; u < 4; u++) { cc[u] = czero(); cd[u] = czero(); }
	__syncthreads();
	// this CTA's half of the B-layout spectra: global offsets (64 h + m) * 128 + k
	const long hoff = (long)h * 64 * G::P;
	if (p.FS != nullptr && j > 0) {
		const int gi = (j % 3) + 1, hi = ((j + 1) % 3) + 1;
		const C *FS = p.FS + cell * 3 * PP;
		for (int i = threadIdx.x; i < 64 * 128; i += 512) {
			const long o = hoff + i;
			S[(i >> 7) * G::LDP + (i & 127)] = csub(cmul(Wh[hi * PP + o], FS[(gi - 1) * PP + o]), cmul(Wh[gi * PP + o], FS[(hi - 1) * PP + o]));
		}
		__syncthreads();
		C v[4];
		inverse_extract(S, peer, cl, h, tw128, tw64, v);
#pragma unroll
		for (int u = 0; u < 4; u++) cc[u] = make_double2(p.s1 * (double)v[u].x, p.s1 * (double)v[u].y);
	}
	if (p.FS4 != nullptr || p.Qp != nullptr || p.Xp != nullptr) {
		for (int i = threadIdx.x; i < 64 * 128; i += 512) {
			const long o = hoff + i;
			C z = czero<C>();
			if (p.Qp != nullptr) {
				C q = czero<C>();
				for (int ii = 0; ii < 4; ii++) {
					const C *Q = p.Qp + ((cell * 4 + ii) * p.nq) * PP + o;
					C s = czero<C>();
					for (int k = 0; k < p.nq; k++) s = cadd(s, Q[(long)k * PP]);
					q.x += eta2[ii] * s.x; q.y += eta2[ii] * s.y;
				}
				C hh; hh.x = -Wh[j * PP + o].x; hh.y = -Wh[j * PP + o].y;
				if (j == 0) hh.x += (R)1.0;
				const C v = cmul(hh, q);
				z.x += s2 * v.x; z.y += s2 * v.y;
			}
			if (p.Xp != nullptr) {
				C s = czero<C>();
				for (int k = 0; k < p.nx; k++) s = cadd(s, p.Xp[((cell * p.nx + k) * 4 + j) * PP + o]);
				z.x -= eta2[j] * s1 * s.x; z.y -= eta2[j] * s1 * s.y;
			}
			if (p.FS4 != nullptr) {
				const C *F4 = p.FS4 + cell * 4 * PP;
				C v = cadd(cscale(cmul(Wh[o], F4[j * PP + o]), eta2[j]), cscale(cmul(Wh[j * PP + o], F4[o]), (R)2.0));
				if (j == 0) {
					C s = czero<C>();
					for (int c = 0; c < 4; c++) s = cadd(s, cmul(Wh[c * PP + o], F4[c * PP + o]));
					v = csub(v, cscale(s, (R)2.0));
				}
				z.x += s1 * v.x; z.y += s1 * v.y;
			}
			S[(i >> 7) * G::LDP + (i & 127)] = z;
		}
		__syncthreads();
		C v[4];
		inverse_extract(S, peer, cl, h, tw128, tw64, v);
#pragma unroll
		for (int u = 0; u < 4; u++) cd[u] = make_double2((double)v[u].x, (double)v[u].y);
	}
#pragma unroll
	for (int u = 0; u < 4; u++) {
		const int idx = u * 512 + (int)threadIdx.x;
		const int q = (32 * h + (idx >> 6)) * N + (idx & 63);   // N-grid index k + N l
		const long o = (cell * 4 + j) * NN + q;
		if (p.mode == 0) {
			if (p.out_cc) p.out_cc[o] = cc[u];
			if (p.out_cd) p.out_cd[o] = cd[u];
		} else {
			const double2 *w = p.wcur + cell * 4 * NN + q;
			double2 cb = czero();
			if (p.B != nullptr) {        // null B: no magnetic field
				const double *B = p.B + cell * 3;
				if (j == 1) cb = make_double2(2 * (B[1] * w[3 * NN].x - B[2] * w[2 * NN].x), 2 * (B[1] * w[3 * NN].y - B[2] * w[2 * NN].y));
				if (j == 2) cb = make_double2(2 * (B[2] * w[1 * NN].x - B[0] * w[3 * NN].x), 2 * (B[2] * w[1 * NN].y - B[0] * w[3 * NN].y));
				if (j == 3) cb = make_double2(2 * (B[0] * w[2 * NN].x - B[1] * w[1 * NN].x), 2 * (B[0] * w[2 * NN].y - B[1] * w[1 * NN].y));
			}
			const double2 b = p.base ? p.base[o] : czero();
			p.out[o] = make_double2(b.x + p.dtc * ((cc[u].x + cd[u].x) + cb.x), b.y + p.dtc * ((cc[u].y + cd[u].y) + cb.y));
		}
	}
}

// out = scale * Extract(IFFT2(Z)) for one B-layout padded grid (single
// integrals), one CTA pair
__global__ void __launch_bounds__(512, 1) k_extract_ifft128(const double2 *__restrict__ Z, double scale, double2 *__restrict__ out) {
	using G = G128;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	double2 *S = reinterpret_cast<double2 *>(smem_raw), *tw128 = S + G::GRID_H, *tw64 = tw128 + 128;
	cg::cluster_group cl = cg::this_cluster();
	const int h = (int)cl.block_rank();
	const double2 *peer = cl.map_shared_rank(S, h ^ 1);
	init_tw128(tw128, tw64);
	for (int i = threadIdx.x; i < 64 * 128; i += 512) S[(i >> 7) * G::LDP + (i & 127)] = Z[(long)h * 64 * G::P + i];
	__syncthreads();
	double2 v[4];
	inverse_extract(S, peer, cl, h, tw128, tw64, v);
#pragma unroll
	for (int u = 0; u < 4; u++) {
		const int idx = u * 512 + (int)threadIdx.x;
		out[(32 * h + (idx >> 6)) * G::N + (idx & 63)] = make_double2(scale * v[u].x, scale * v[u].y);
	}
}

}  // namespace qb
