// hb_common.cuh -- layouts and sm_100a primitives shared by the kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace hb {

// ---------------------------------------------------------------------------
// Layouts
//
// j-particle record (host mirror and its device copy), AoS doubles:
//   pos[3] mass vel[3] tlast acc[3] jrk[3] [snp crk] [d4a d5a]
//
// ORDER 9 is the 8th-order scheme with double-double positions (the
// reference's SRC/hermite8dd.h): the 8th-order record followed by the low
// part of the position, posL[3] -- 29 words.  Its predicted state is the
// 8th-order one (with the high part posH as the position) followed by the
// predicted low part xL[3]; its force record is the 8th-order one.
template <int ORDER> struct Rec {
    static constexpr int words = 8 + 3 * (ORDER - 2);   // 14 / 20 / 26 / 29
    static constexpr int bytes = words * 8;               // 112 / 160 / 208 / 232
};
// force record: acc jrk [snp] [crk]
template <int ORDER> struct Frc {
    static constexpr int words = 3 * (ORDER / 2);       // 6 / 9 / 12 / 12
};
// Offset of posL in an ORDER 9 record.
constexpr int kRecPosL = 26;


// Predicted j-particles: "AoSoA32" -- chunks of 32 slots, each chunk holding
// one 32-wide vector per component, so that a warp's per-component loads and
// stores are single 128/256-byte transactions and a chunk is one contiguous
// block for a bulk copy.
//   FP64 components:  x y z m vx vy vz [ax ay az] [jx jy jz]        7/10/13
//   mixed components: xh yh zh xl yl zl m vx vy vz [ax ay az] [jx jy jz]
//                                                                   10/13/16
constexpr int kChunk = 32;
template <int ORDER> struct Pred64 {
    static constexpr int ncomp = 7 + 3 * (ORDER / 2 - 2) + (ORDER == 9 ? 3 : 0);   // 7/10/13/16
    static constexpr int chunk_bytes = ncomp * kChunk * 8;
};
template <int ORDER> struct PredMx {
    static constexpr int ncomp = 10 + 3 * (ORDER / 2 - 2);
    static constexpr int chunk_bytes = ncomp * kChunk * 4;
};
// Component indices.
enum : int { P64_X = 0, P64_M = 3, P64_V = 4, P64_A = 7, P64_J = 10, P64_XL = 13 };
enum : int { PMX_XH = 0, PMX_XL = 3, PMX_M = 6, PMX_V = 7, PMX_A = 10, PMX_J = 13 };

// Slots are padded to a multiple of this (i-tiles never read past the end).
constexpr int kSlotPad = 256;

// Padding slots carry zero mass at distinct far-away positions, so that they
// contribute exactly zero to every sum and no arithmetic overflows.
__device__ __forceinline__ double pad_position(int slot, int k)
{
    return 1099511627776.0 /* 2^40 */ + (double)(slot * 3 + k);
}

// ---------------------------------------------------------------------------
// Error flag shared with the host (mapped pinned memory).
enum : int { kErrNone = 0, kErrWaitTimeout = 1 };

// Spin bound for every device-side wait: far above any legitimate wait
// (a bulk copy of a few tens of KB from L2/HBM), small enough that a lost
// completion ends in well under a second.
constexpr uint32_t kSpinLimit = 1u << 22;

// ---------------------------------------------------------------------------
// Shared-memory mbarrier + bulk async copy (TMA, non-tensor form).
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;"
                 :: "r"(smem_u32(bar)), "r"(count) : "memory");
}

// Make mbarrier initialisation visible to the async (bulk-copy) proxy.
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Bulk copy global -> this CTA's shared memory, completing on `bar`.
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes,
                                          uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return done != 0;
}

// Bounded wait for phase `parity` of `bar`.  Returns false after `limit`
// polls (each try_wait itself suspends for a hardware-chosen time).  Waits
// that drain copies still in flight always take the full kSpinLimit.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  uint32_t limit = kSpinLimit)
{
    for (uint32_t it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void raise_error(int *err, int code)
{
    if (err) atomicCAS(err, kErrNone, code);
}

}  // namespace hb
