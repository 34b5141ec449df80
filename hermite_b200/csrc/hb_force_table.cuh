// hb_force_table.cuh -- the compiled launch shapes of the force kernel.
#pragma once
#include "hb_force.cuh"

namespace hb {

template <int ORDER, bool MIXED, int NW, int NI, int WJ, int TCH, int MINB = 0, bool FUSED = false>
ForceVariant make_variant()
{
    using Sh = ForceShape<ORDER, MIXED, NW, NI, WJ, TCH, FUSED>;
    return ForceVariant{NW, NI, WJ, TCH, Sh::TI, Sh::smem_bytes, FUSED,
                        &force_kernel<ORDER, MIXED, NW, NI, WJ, TCH, MINB, FUSED>};
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
template <int ORDER, bool MIXED>
struct VariantTable {
    static constexpr int count = 20;
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
            make_variant<ORDER, MIXED, 4, 2, 1, 8>()} {}
};

}  // namespace hb
