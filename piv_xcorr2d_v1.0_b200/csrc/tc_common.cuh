// tc_common.cuh -- sm_100a tensor-core primitives in inline PTX: tcgen05 MMA with
// operands in shared memory and the accumulator in tensor memory (TMEM), mbarrier
// completion with bounded waits, TMEM allocation and loads.
//
// Shared-memory operand layout: the no-swizzle canonical layout of 16-bit elements,
// built from 8 x 16-byte "core matrices" (8 rows of 8 elements).  Two layouts are
// used, each a function byte_offset(mn, k) of the operand's M/N index and K index:
//   K-major  : (k/8)*(R*16) + mn*16 + (k%8)*2      LBO = R*16 (next K chunk)
//                                                  SBO = 128  (next 8 rows)
//   MN-major : (mn/8)*(K*16) + k*16 + (mn%8)*2     LBO = 128  (next 8 K rows)
//                                                  SBO = K*16 (next 8 MN elements)
// with R the operand's MN extent and K its K extent.  One buffer laid out as
// buf(r, c) = (c/8)*(R*16) + r*16 + (c%8)*2 reads as the K-major operand
// (mn = r, k = c) and as the MN-major operand (mn = c, k = r), i.e. as a matrix and
// its transpose, without a second copy.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>

namespace piv {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// --- descriptors --------------------------------------------------------------
// Shared-memory matrix descriptor (tcgen05 format): start>>4 in [0,14), LBO>>4 in
// [16,30), SBO>>4 in [32,46), version 1 in [46,48), base offset 0, layout 0 = no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor for kind::f16 with BF16 A and B (a_fmt = b_fmt = 1) or F16
// (0), F32 accumulate (c_format 1), M = 128 (m_dim 8 at bit 24), N at bit 17 in units
// of 8, A/B major at bits 15/16 (1 = MN-major).
__host__ __device__ constexpr uint32_t idesc_f16(int N, bool a_mn, bool b_mn, bool bf16)
{
    return (1u << 4) | ((bf16 ? 1u : 0u) << 7) | ((bf16 ? 1u : 0u) << 10) | ((a_mn ? 1u : 0u) << 15) |
           ((b_mn ? 1u : 0u) << 16) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

// --- MMA ----------------------------------------------------------------------
// D[tmem] (+)= A * B^T over one K = 16 step; issued by one thread.
__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrive (once) on an mbarrier when every MMA issued so far by this thread is done.
__device__ __forceinline__ void mma_commit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

// --- mbarrier -----------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

// makes a fresh mbarrier's initialisation visible to the async proxy (the MMA unit)
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_inval(uint32_t mbar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(mbar) : "memory");
}

// One probe: the thread is suspended until the phase completes or kSuspendNs elapse (the
// suspend-time hint), instead of returning at once, so that waiting warps do not spend issue
// slots polling while the other warpgroups of the SM work.
constexpr uint32_t kSuspendNs = 1000000;  // 1 ms
__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(done)
        : "r"(mbar), "r"(parity), "r"(kSuspendNs)
        : "memory");
    return done != 0;
}

// Bounded wait for the phase with the given parity to complete: at most kMaxTries probes
// of at most kSuspendNs each (about 2 s in all), so the wait always ends; false means the
// phase never completed (the caller records an error and leaves without reading the
// accumulator).
constexpr int kMaxTries = 2048;
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity)
{
    for (int it = 0; it < kMaxTries; ++it)
        if (mbar_try_wait(mbar, parity)) return true;
    return false;
}

// --- TMA (bulk tensor copies, global -> shared) -------------------------------------
// Arm an mbarrier for `bytes` of incoming transactions (one arrival by the calling thread).
__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

// 2D tile load of the tensor map's box at (x, y) (x: innermost coordinate, already a multiple
// of 16 bytes) into shared memory at dst (128-byte aligned); completion counted on mbar.  No
// multicast.  Out-of-range parts of the box read zero.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const void *tmap, int x, int y, uint32_t mbar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(mbar)
        : "memory");
}

// --- named barriers (one per warpgroup; barrier 0 is __syncthreads) -------------
__device__ __forceinline__ void named_sync(uint32_t id, uint32_t nthreads)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// barrier + OR of pred over the participating threads
__device__ __forceinline__ bool named_sync_or(uint32_t id, uint32_t nthreads, bool pred)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.b32 p, %1, 0;\n\tbar.red.or.pred q, %2, %3, p;\n\t"
        "selp.b32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(id), "r"(nthreads)
        : "memory");
    return r != 0;
}

// --- fences -------------------------------------------------------------------
// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// --- TMEM ---------------------------------------------------------------------
// Whole warp: allocate `cols` columns (power of two >= 32); the base address is
// written to shared memory at `dst`.
__device__ __forceinline__ void tmem_alloc(uint32_t dst, uint32_t cols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t cols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols) : "memory");
}

// 32 lanes x 32 consecutive 32-bit columns: thread i of the warp receives lane
// (lane base + i), columns [col, col + 32).  taddr = base + (lane base << 16) + col.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]),
          "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
          "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8])
{
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr)
                 : "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// --- operand packing ------------------------------------------------------------
// Split x into bf16 hi + lo with x ~= hi + lo (hi = round(x), lo = round(x - hi));
// the pair carries about 16 significant bits.
__device__ __forceinline__ void split_bf16(float x, uint16_t &hi, uint16_t &lo)
{
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    const __nv_bfloat16 l = __float2bfloat16_rn(x - __bfloat162float(h));
    hi = __bfloat16_as_ushort(h);
    lo = __bfloat16_as_ushort(l);
}

// The same for a pair (a in the low half): two packed conversions and two subtractions.
__device__ __forceinline__ void split_bf16x2(float a, float b, uint32_t &hi, uint32_t &lo)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    const float2 hf = __bfloat1622float2(h);
    const __nv_bfloat162 l = __floats2bfloat162_rn(a - hf.x, b - hf.y);
    hi = *reinterpret_cast<const uint32_t *>(&h);
    lo = *reinterpret_cast<const uint32_t *>(&l);
}

// FP16 forms of the two splits (hi + lo carry about 22 significant bits; the caller keeps
// the values inside FP16's range).
__device__ __forceinline__ void split_f16(float x, uint16_t &hi, uint16_t &lo)
{
    const __half h = __float2half_rn(x);
    const __half l = __float2half_rn(x - __half2float(h));
    hi = __half_as_ushort(h);
    lo = __half_as_ushort(l);
}

__device__ __forceinline__ void split_f16x2(float a, float b, uint32_t &hi, uint32_t &lo)
{
    const __half2 h = __floats2half2_rn(a, b);
    const float2 hf = __half22float2(h);
    const __half2 l = __floats2half2_rn(a - hf.x, b - hf.y);
    hi = *reinterpret_cast<const uint32_t *>(&h);
    lo = *reinterpret_cast<const uint32_t *>(&l);
}

__device__ __forceinline__ uint32_t pack2(uint16_t a, uint16_t b) { return (uint32_t)a | ((uint32_t)b << 16); }

// Byte offsets of the two layouts above.
__host__ __device__ constexpr uint32_t off_kmajor(int mn, int k, int R) { return (k / 8) * (R * 16) + mn * 16 + (k % 8) * 2; }
__host__ __device__ constexpr uint32_t off_mnmajor(int mn, int k, int K) { return (mn / 8) * (K * 16) + k * 16 + (mn % 8) * 2; }

}  // namespace tc
}  // namespace piv
