// qb_fft.cuh — register/shared-memory FFT building blocks (sm_100a), generic
// over the complex type C = double2 (FP64) or float2 (FP32).
//
// A length-L transform (L = 8*T, T in {1,2,4,8}) is spread over T consecutive
// lanes of one warp; every lane holds 8 complex values in registers:
//   input : lane tau holds x[tau + T*r], r = 0..7
//   step 1: radix-8 DFT over r in registers
//   step 2: twiddle by w_L^(tau*q) (powers of the lane's base twiddle)
//   step 3: transpose among the T lanes through an L-slot scratch (the row or
//           column of the grid being transformed), XOR-swizzled so that a
//           quarter-warp touches 8 distinct 16-byte bank groups
//   step 4: R/T radix-T DFTs in registers
//   output: lane tau' holds X[out_pos(tau', e)], e = 0..7
// For T = 8 the output index set of a lane equals its input index set
// (tau + 8e), which lets an inverse transform follow a forward one (or the
// reverse) on the same column with no exchange in between.
//
// FFT sign convention as FFTW: DIR = -1 forward exp(-2 pi i jk/L),
// DIR = +1 backward exp(+2 pi i jk/L), no normalisation.
#pragma once
#include <cuda_runtime.h>

namespace qb {

// scalar type of a complex type
template <class C> struct CT;
template <> struct CT<double2> { using R = double; };
template <> struct CT<float2> { using R = float; };

template <class C> __device__ __forceinline__ C mk(double re, double im) {
	using R = typename CT<C>::R;
	C z; z.x = (R)re; z.y = (R)im; return z;
}
template <class C> __device__ __forceinline__ C czero() { return mk<C>(0.0, 0.0); }
template <class C> __device__ __forceinline__ C cadd(C a, C b) { C z; z.x = a.x + b.x; z.y = a.y + b.y; return z; }
template <class C> __device__ __forceinline__ C csub(C a, C b) { C z; z.x = a.x - b.x; z.y = a.y - b.y; return z; }
template <class C> __device__ __forceinline__ C cmul(C a, C b) { C z; z.x = a.x * b.x - a.y * b.y; z.y = a.x * b.y + a.y * b.x; return z; }
template <class C> __device__ __forceinline__ C cscale(C a, typename CT<C>::R s) { C z; z.x = a.x * s; z.y = a.y * s; return z; }
template <class C> __device__ __forceinline__ C cfma(C a, C b, C c) {   // c + a*b
	C z; z.x = c.x + (a.x * b.x - a.y * b.y); z.y = c.y + (a.x * b.y + a.y * b.x); return z;
}
// FP32: complex add and subtract as one packed two-lane instruction (sm_100
// add/sub.rn.f32x2: the same IEEE round-to-nearest result per lane as two
// scalar ones, half the issue slots)
__device__ __forceinline__ unsigned long long pack_f2(float2 a) {
	unsigned long long r;
	asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
	return r;
}
__device__ __forceinline__ float2 unpack_f2(unsigned long long r) {
	float2 a;
	asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
	return a;
}
template <> __device__ __forceinline__ float2 cadd<float2>(float2 a, float2 b) {
	unsigned long long d;
	asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pack_f2(a)), "l"(pack_f2(b)));
	return unpack_f2(d);
}
template <> __device__ __forceinline__ float2 csub<float2>(float2 a, float2 b) {
	unsigned long long d;
	asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pack_f2(a)), "l"(pack_f2(b)));
	return unpack_f2(d);
}
// FP64 shorthands used by code that is FP64 only
__device__ __forceinline__ double2 czero() { return czero<double2>(); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return cadd<double2>(a, b); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return csub<double2>(a, b); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) { return cmul<double2>(a, b); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return cscale<double2>(a, s); }
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) { return cfma<double2>(a, b, c); }

// a * (DIR * i)
template <int DIR, class C> __device__ __forceinline__ C mul_i(C a) {
	C z;
	if (DIR < 0) { z.x = a.y; z.y = -a.x; } else { z.x = -a.y; z.y = a.x; }
	return z;
}
// a * w8^1 with w8 = exp(DIR * 2 pi i / 8)
template <int DIR, class C> __device__ __forceinline__ C mul_w8(C a) {
	using R = typename CT<C>::R;
	const R s = (R)0.70710678118654752440;
	C z;
	if (DIR < 0) { z.x = s * (a.x + a.y); z.y = s * (a.y - a.x); } else { z.x = s * (a.x - a.y); z.y = s * (a.x + a.y); }
	return z;
}
// a * w8^3
template <int DIR, class C> __device__ __forceinline__ C mul_w8_3(C a) {
	using R = typename CT<C>::R;
	const R s = (R)0.70710678118654752440;
	C z;
	if (DIR < 0) { z.x = s * (a.y - a.x); z.y = -s * (a.x + a.y); } else { z.x = -s * (a.x + a.y); z.y = s * (a.x - a.y); }
	return z;
}

// in-place 8-point DFT, natural order in and out (radix-2 decimation in frequency)
template <int DIR, class C> __device__ __forceinline__ void dft8(C (&x)[8]) {
	const C a0 = cadd(x[0], x[4]), a4 = csub(x[0], x[4]);
	const C a1 = cadd(x[1], x[5]), a5 = mul_w8<DIR>(csub(x[1], x[5]));
	const C a2 = cadd(x[2], x[6]), a6 = mul_i<DIR>(csub(x[2], x[6]));
	const C a3 = cadd(x[3], x[7]), a7 = mul_w8_3<DIR>(csub(x[3], x[7]));
	const C b0 = cadd(a0, a2), b2 = csub(a0, a2), b1 = cadd(a1, a3), b3 = mul_i<DIR>(csub(a1, a3));
	const C b4 = cadd(a4, a6), b6 = csub(a4, a6), b5 = cadd(a5, a7), b7 = mul_i<DIR>(csub(a5, a7));
	x[0] = cadd(b0, b1); x[4] = csub(b0, b1);
	x[2] = cadd(b2, b3); x[6] = csub(b2, b3);
	x[1] = cadd(b4, b5); x[5] = csub(b4, b5);
	x[3] = cadd(b6, b7); x[7] = csub(b6, b7);
}

template <int DIR, class C> __device__ __forceinline__ void dft4(C &x0, C &x1, C &x2, C &x3) {
	const C a0 = cadd(x0, x2), a2 = csub(x0, x2), a1 = cadd(x1, x3), a3 = mul_i<DIR>(csub(x1, x3));
	x0 = cadd(a0, a1); x2 = csub(a0, a1); x1 = cadd(a2, a3); x3 = csub(a2, a3);
}

template <class C> __device__ __forceinline__ void dft2(C &x0, C &x1) {
	const C a = x0; x0 = cadd(a, x1); x1 = csub(a, x1);
}

// Geometry of a length-L transform spread over T = L/8 lanes.
template <int L> struct Len {
	static_assert(L == 8 || L == 16 || L == 32 || L == 64, "supported transform lengths: 8..64");
	static constexpr int T = L / 8;          // lanes per transform
	static constexpr int U = 8 / T;          // radix-T DFTs per lane in step 4
	// position of output e of lane tau
	__device__ __forceinline__ static int out_pos(int tau, int e) { return (T == 1) ? e : (tau * U + e / T) + 8 * (e % T); }
	// scratch slot of value (q, s) in the step-3 transpose
	__device__ __forceinline__ static int xpos(int q, int s) { return q * T + (s ^ (q & (T - 1))); }
};

// Scratch of a transform: sc(pos) is the slot of position pos (0 .. L-1)
// of the line being transformed (a row or a column of a grid in shared memory).
template <class C> struct Strided {
	C *p; int stride;
	__device__ __forceinline__ C &operator()(int pos) const { return p[pos * stride]; }
};

// steps 3 and 4 of a length-L transform (see file comment): the transpose
// among the T lanes through the scratch accessor sc, then the radix-T DFTs
template <int L, int DIR, class C, class Acc>
__device__ __forceinline__ void fft1d_tail(C (&x)[8], int tau, const Acc &sc) {
	using G = Len<L>;
	__syncwarp();
#pragma unroll
	for (int q = 0; q < 8; q++) sc(G::xpos(q, tau)) = x[q];
	__syncwarp();
#pragma unroll
	for (int u = 0; u < G::U; u++)
#pragma unroll
		for (int s = 0; s < G::T; s++) x[u * G::T + s] = sc(G::xpos(tau * G::U + u, s));
	__syncwarp();
#pragma unroll
	for (int u = 0; u < G::U; u++) {
		if constexpr (G::T == 2) dft2(x[2 * u], x[2 * u + 1]);
		else if constexpr (G::T == 4) dft4<DIR>(x[4 * u], x[4 * u + 1], x[4 * u + 2], x[4 * u + 3]);
		else {
			C y[8];
#pragma unroll
			for (int s = 0; s < 8; s++) y[s] = x[s];
			dft8<DIR>(y);
#pragma unroll
			for (int s = 0; s < 8; s++) x[s] = y[s];
		}
	}
}

// Length-L transform of the 8 values in x (see file comment) with the
// scratch accessor sc; its previous contents are destroyed.  `tw` is the table
// of init_twiddles (tw[e] = w_L^e); a lane reads only its base twiddle
// w_L^tau (the T lanes read T consecutive entries: one conflict-free
// wavefront) and forms w_L^(tau*q), q = 2..7, by repeated multiplication in
// registers, trading six shared-memory loads for six complex multiplies
// (relative error of the powers below 1e-15).
// Must be called by all 32 lanes of the warp (contains __syncwarp).
template <int L, int DIR, class C, class Acc>
__device__ __forceinline__ void fft1d_acc(C (&x)[8], int tau, const Acc &sc, const C *tw) {
	using G = Len<L>;
	dft8<DIR>(x);
	if constexpr (G::T > 1) {
		C w1 = tw[tau];
		if (DIR > 0) w1.y = -w1.y;
		C w = w1;
		x[1] = cmul(x[1], w);
#pragma unroll
		for (int q = 2; q < 8; q++) {
			w = cmul(w, w1);
			x[q] = cmul(x[q], w);
		}
		fft1d_tail<L, DIR>(x, tau, sc);
	}
}

// the same with the lane's twiddle powers given: wp[q] = w_L^(tau q) of the
// forward sign (conjugated here for DIR = +1), q = 1..7, e.g. computed once
// per kernel by a lane whose tau does not change
template <int L, int DIR, class C, class Acc>
__device__ __forceinline__ void fft1d_accw(C (&x)[8], int tau, const Acc &sc, const C (&wp)[8]) {
	using G = Len<L>;
	dft8<DIR>(x);
	if constexpr (G::T > 1) {
#pragma unroll
		for (int q = 1; q < 8; q++) {
			C w = wp[q];
			if (DIR > 0) w.y = -w.y;
			x[q] = cmul(x[q], w);
		}
		fft1d_tail<L, DIR>(x, tau, sc);
	}
}

// the same on an L-slot region addressed scratch[pos * sstride]
template <int L, int DIR, class C>
__device__ __forceinline__ void fft1d(C (&x)[8], int tau, C *scratch, int sstride, const C *tw) {
	fft1d_acc<L, DIR>(x, tau, Strided<C>{scratch, sstride}, tw);
}

// Reorder a lane's transform outputs (positions out_pos) into the input
// layout (positions tau + T*r) through the scratch; a no-op when T is 1 or 8.
template <int L, class C, class Acc>
__device__ __forceinline__ void out_to_in_acc(C (&x)[8], int tau, const Acc &sc) {
	using G = Len<L>;
	if constexpr (G::T != 1 && G::T != 8) {
		__syncwarp();
#pragma unroll
		for (int e = 0; e < 8; e++) sc(G::out_pos(tau, e)) = x[e];
		__syncwarp();
#pragma unroll
		for (int r = 0; r < 8; r++) x[r] = sc(tau + G::T * r);
		__syncwarp();
	}
}
template <int L, class C>
__device__ __forceinline__ void out_to_in(C (&x)[8], int tau, C *scratch, int sstride) {
	out_to_in_acc<L>(x, tau, Strided<C>{scratch, sstride});
}

// fill the twiddle table of fft1d<L>: tw[e] = exp(-2 pi i e / L), e < L,
// evaluated in FP64 and rounded to C (all threads of the block call it)
template <int L, class C>
__device__ __forceinline__ void init_twiddles(C *tw) {
	for (int e = threadIdx.x; e < L; e += blockDim.x) {
		double s, c;
		sincospi(-2.0 * (double)e / (double)L, &s, &c);
		tw[e] = mk<C>(c, s);
	}
}

}  // namespace qb
