// hb_force_table.cuh -- the compiled launch shapes of the force kernel.
#pragma once
#include "hb_force.cuh"

namespace hb {

template <int ORDER, bool MIXED, int NW, int NI, int WJ, int TCH, int MINB = 0, bool FUSED = false>
ForceVariant make_variant()
{
    using Sh = ForceShape<ORDER, MIXED, NW, NI, WJ, TCH, FUSED>;
    return ForceVariant{NW, NI, WJ, TCH, Sh::TI, Sh::smem_bytes, FUSED, 0,
                        &force_kernel<ORDER, MIXED, NW, NI, WJ, TCH, MINB, FUSED>};
}

template <int ORDER, int NW, int NI, int W32, int W64, int TCH, int Q64, int MINB = 0>
ForceVariant make_hyb_variant()
{
    using Sh = HybShape<ORDER, NW, NI, W32, W64, TCH, Q64>;
    return ForceVariant{NW, NI, W32 + W64, TCH, Sh::TI, Sh::smem_bytes, false, Q64,
                        &force_kernel_hyb<ORDER, NW, NI, W32, W64, TCH, Q64, MINB>};
}

// Shapes, by index (the tuning table refers to them by index):
//   0: 4 warps, 1 i-chunk/warp, no in-CTA j split     (128 i per CTA)
//   1: 4 warps, 2 i-chunks/warp                        (256 i per CTA)
//   2: 4 warps sharing 1 i-chunk, j tile split 4 ways  ( 32 i per CTA)
//   3: 4 warps, 2 i-groups, j tile split 2 ways        ( 64 i per CTA)
//   4: 8 warps, 1 i-chunk/warp, 8-chunk tiles          (256 i per CTA)
//   5: as 0, registers capped for 5 resident CTAs per SM
//   6: as 1, registers capped for 3 resident CTAs per SM
//   7: as 2, registers capped for 5 resident CTAs per SM
//   8: 2 warps, 1 i-chunk/warp, capped for 8 CTAs/SM    ( 64 i per CTA)
//   9: as 0 with 8-chunk tiles
//  10: as 3, registers capped for 5 resident CTAs per SM
//  11: as 8 with the j tile split 2 ways                ( 32 i per CTA)
// Fused predict + force (each CTA predicts the raw records it streams):
//  12: as 0    13: as 2    14: as 3    15: as 8    16: as 1 with 8-chunk tiles
//  17: as 5
// Two-pass, 2 i-chunks per warp (appended):
//  18: 2 warps, 2 i-chunks/warp                        (128 i per CTA)
//  19: as 1 with 8-chunk tiles
// Mixed precision on both pipes (mixed tables only; force_kernel_hyb), each
// i-group = W32 mixed-precision warps + W64 FP64 warps, Q64 of every TCH
// chunks of a j tile in FP64:
//  20: 8 warps, W32 = W64 = 1, 1 i-chunk/warp, 2 of 8 chunks FP64  (128 i)
//  21: as 20, 1 of 8 chunks FP64
//  22: as 20, 3 of 8 chunks FP64
//  23: 12 warps, W32 = 2, W64 = 1, 3 of 12 chunks FP64             (128 i)
constexpr int kBaseVariants = 20, kHybVariants = 4;
template <int ORDER, bool MIXED>
struct VariantTable {
    static constexpr int count = kBaseVariants + (MIXED ? kHybVariants : 0);
    ForceVariant v[count];
    VariantTable()
        : v{make_variant<ORDER, MIXED, 4, 1, 1, 4>(),
            make_variant<ORDER, MIXED, 4, 2, 1, 4>(),
            make_variant<ORDER, MIXED, 4, 1, 4, 4>(),
            make_variant<ORDER, MIXED, 4, 1, 2, 4>(),
            make_variant<ORDER, MIXED, 8, 1, 1, 8>(),
            make_variant<ORDER, MIXED, 4, 1, 1, 4, 5>(),
            make_variant<ORDER, MIXED, 4, 2, 1, 4, 3>(),
            make_variant<ORDER, MIXED, 4, 1, 4, 4, 5>(),
            make_variant<ORDER, MIXED, 2, 1, 1, 4, 8>(),
            make_variant<ORDER, MIXED, 4, 1, 1, 8>(),
            make_variant<ORDER, MIXED, 4, 1, 2, 4, 5>(),
            make_variant<ORDER, MIXED, 2, 1, 2, 4, 8>(),
            make_variant<ORDER, MIXED, 4, 1, 1, 4, 0, true>(),
            make_variant<ORDER, MIXED, 4, 1, 4, 4, 0, true>(),
            make_variant<ORDER, MIXED, 4, 1, 2, 4, 0, true>(),
            make_variant<ORDER, MIXED, 2, 1, 1, 4, 8, true>(),
            make_variant<ORDER, MIXED, 4, 2, 1, 8, 0, true>(),
            make_variant<ORDER, MIXED, 4, 1, 1, 4, 5, true>(),
            make_variant<ORDER, MIXED, 2, 2, 1, 4>(),
            make_variant<ORDER, MIXED, 4, 2, 1, 8>()}
    {
        if constexpr (MIXED) {
            v[20] = make_hyb_variant<ORDER, 8, 1, 1, 1, 8, 2>();
            v[21] = make_hyb_variant<ORDER, 8, 1, 1, 1, 8, 1>();
            v[22] = make_hyb_variant<ORDER, 8, 1, 1, 1, 8, 3>();
            v[23] = make_hyb_variant<ORDER, 12, 1, 2, 1, 12, 3>();
        }
    }
};

}  // namespace hb
