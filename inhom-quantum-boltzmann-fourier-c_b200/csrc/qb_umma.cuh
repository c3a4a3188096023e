// qb_umma.cuh — building blocks for the 5th-generation tensor cores of
// sm_100a (tcgen05.mma with the accumulator in tensor memory).
//
// Operands live in shared memory in the 128-byte-swizzled canonical layouts
// the tensor core reads through a 64-bit matrix descriptor; the accumulator D
// (M = 128 rows x N FP32 columns) lives in tensor memory, row m in lane m.
// Only what the DFT-as-GEMM kernels need is here: kind::tf32 (FP32 operands
// read as TF32, FP32 accumulation), A and B K-major, one CTA.
//
// Layouts (byte offsets from a 1024-byte aligned base; f = 4-byte element):
//   K-major, 128B swizzle: a tile of R rows x K elements (K a multiple of 32)
//     is stored as K/32 blocks of R x 128 B; row r of a block at r * 128 B,
//     16-byte chunk c of the row at ((c ^ (r % 8)) * 16).  One MMA step reads
//     8 elements (32 B) of K: start + (k / 32) * R * 128 + (k % 32) * 4,
//     SBO = 1024 (8-row groups), LBO = 16 (unused with swizzling).
#pragma once
#include <cstdint>

namespace qb {
namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start address, leading / stride byte
// offsets (all >> 4), version 1 (sm_100), base offset 0, 128-byte swizzle (2)
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
	return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16) |
	       ((uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32) | (1ull << 46) | (2ull << 61);
}

// instruction descriptor of kind::tf32 with FP32 accumulation: D format F32
// (bits 4-5 = 1), A and B format TF32 (bits 7-9, 10-12 = 2), A and B K-major
// (bits 15, 16 = 0), N >> 3 at bits 17-22, M >> 4 at bits 24-28
template <int M, int N>
__host__ __device__ constexpr uint32_t idesc_tf32() {
	static_assert(M == 128, "one-CTA M = 128 tiles (row m of D in tensor-memory lane m)");
	static_assert(N % 16 == 0 && N >= 16 && N <= 256, "N of a kind::tf32 MMA with M = 128");
	return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// instruction descriptor of kind::f16 with BF16 operands and FP32
// accumulation: D format F32 (bits 4-5 = 1), A and B format BF16 (bits 7-9,
// 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28
template <int M, int N>
__host__ __device__ constexpr uint32_t idesc_bf16() {
	static_assert(M == 128, "one-CTA M = 128 tiles (row m of D in tensor-memory lane m)");
	static_assert(N % 16 == 0 && N >= 16 && N <= 256, "N of a kind::f16 MMA with M = 128");
	return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[desc] x B[desc], 16-bit operands (one K step: 16 elements); one thread issues
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc, uint32_t accumulate) {
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "setp.ne.b32 p, %4, 0;\n\t"
	    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
	    "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
	    : "memory");
}

// byte offset of 16-bit element (row r, k), k < 64, of a K-major 128B-swizzled
// tile: row r at (r / 8) * 1024 + (r % 8) * 128, 16-byte chunk k / 8 at
// ((k / 8) ^ (r % 8)) * 16; a K step of 16 elements starts 32 bytes further
__host__ __device__ constexpr uint32_t kmajor_off16(int r, int k) {
	return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((((k >> 3) & 7) ^ (r & 7)) << 4) + (k & 7) * 2);
}

// D[tmem] (+)= A[desc] x B[desc]; issued by one thread
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc, uint32_t accumulate) {
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "setp.ne.b32 p, %4, 0;\n\t"
	    "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
	    "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
	    : "memory");
}

// arrive on `mbar` once every MMA issued so far by this thread has completed
__device__ __forceinline__ void commit(uint64_t *mbar) {
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
	             : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, unsigned count) {
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}

// wait for phase `parity` of `mbar` to complete, at most `limit` polls; false
// when the limit ran out (the caller records an error and stops waiting)
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, unsigned parity, unsigned limit) {
	const uint32_t a = smem_u32(mbar);
	for (unsigned i = 0; i < limit; i++) {
		uint32_t done = 0;
		asm volatile(
		    "{\n\t.reg .pred p;\n\t"
		    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		    "selp.u32 %0, 1, 0, p;\n\t}\n"
		    : "=r"(done)
		    : "r"(a), "r"(parity)
		    : "memory");
		if (done) return true;
	}
	return false;
}

// bulk copy (TMA, no tensor map) of `bytes` from global to this CTA's shared
// memory, completing on `mbar` (which expects these bytes and one arrival);
// both addresses 16-byte aligned, bytes a multiple of 16; one thread issues
__device__ __forceinline__ void bulk_g2s(void *dst_smem, const void *src_global, uint32_t bytes, uint64_t *mbar) {
	const uint32_t mb = smem_u32(mbar);
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes) : "memory");
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst_smem)),
	             "l"(src_global), "r"(bytes), "r"(mb)
	             : "memory");
}

// a 2-D tile of a tensor map (TMA, no multicast) into shared memory, completing
// on `mbar` (which expects `bytes`); the map lives in kernel parameter space
// (__grid_constant__).  The innermost coordinate x times the element size is
// a multiple of 16 bytes, and the destination is 128-byte aligned.
__device__ __forceinline__ void tma_load_2d(void *dst_smem, const void *tmap, int x, int y, uint64_t *mbar, uint32_t bytes) {
	const uint32_t mb = smem_u32(mbar);
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes) : "memory");
	asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
	             ::"r"(smem_u32(dst_smem)), "l"(tmap), "r"(x), "r"(y), "r"(mb)
	             : "memory");
}

// generic-proxy shared-memory writes -> visible to the tensor core
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
	uint32_t r[16];
	asm volatile(
	    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
	    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
	      "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
	    : "r"(taddr)
	    : "memory");
#pragma unroll
	for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// 16 consecutive FP32 columns of this thread's lane, stored
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float (&v)[16]) {
	asm volatile(
	    "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16};" ::"r"(taddr),
	    "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])),
	    "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])), "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])),
	    "r"(__float_as_uint(v[8])), "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
	    "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])), "r"(__float_as_uint(v[15]))
	    : "memory");
}

// TF32 rounding (round to nearest, ties away) of an FP32 value, kept in an FP32 container
__device__ __forceinline__ float tf32_round(float x) {
	uint32_t r;
	asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
	return __uint_as_float(r);
}

// byte offset of element (row r, k) of a K-major 128B-swizzled tile of R rows
__host__ __device__ constexpr uint32_t kmajor_off(int R, int r, int k) {
	return (uint32_t)((k >> 5) * R * 128 + (r >> 3) * 1024 + (r & 7) * 128 + ((((k & 31) >> 2) ^ (r & 7)) << 4) + (k & 3) * 4);
}
}  // namespace umma
}  // namespace qb
