// hb_force_table.cuh -- the compiled launch shapes of the force kernel.
#pragma once
#include "hb_force.cuh"

namespace hb {

template <int ORDER, bool MIXED, int NW, int NI, int WJ, int TCH>
ForceVariant make_variant()
{
    using Sh = ForceShape<ORDER, MIXED, NW, NI, WJ, TCH>;
    return ForceVariant{NW, NI, WJ, TCH, Sh::TI, Sh::smem_bytes,
                        &force_kernel<ORDER, MIXED, NW, NI, WJ, TCH>};
}

// Shapes, by index (the tuning table refers to them by index):
//   0: 4 warps, 1 i-chunk/warp, no in-CTA j split     (128 i per CTA)
//   1: 4 warps, 2 i-chunks/warp                        (256 i per CTA)
//   2: 4 warps sharing 1 i-chunk, j tile split 4 ways  ( 32 i per CTA)
//   3: 4 warps, 2 i-groups, j tile split 2 ways        ( 64 i per CTA)
//   4: 8 warps, 1 i-chunk/warp, 8-chunk tiles          (256 i per CTA)
template <int ORDER, bool MIXED>
struct VariantTable {
    static constexpr int count = 5;
    ForceVariant v[count];
    VariantTable()
        : v{make_variant<ORDER, MIXED, 4, 1, 1, 4>(),
            make_variant<ORDER, MIXED, 4, 2, 1, 4>(),
            make_variant<ORDER, MIXED, 4, 1, 4, 4>(),
            make_variant<ORDER, MIXED, 4, 1, 2, 4>(),
            make_variant<ORDER, MIXED, 8, 1, 1, 8>()} {}
};

}  // namespace hb
