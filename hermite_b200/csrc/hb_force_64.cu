// hb_force_64.cu -- FP64 force kernel instantiations (orders 4, 6, 8 and the
// 8th order with double-double positions).
#include "hb_force_table.cuh"

namespace hb {

const ForceVariant *force_variant_64(int order, int v)
{
    static const VariantTable<4, false> t4;
    static const VariantTable<6, false> t6;
    static const VariantTable<8, false> t8;
    static const VariantTable<9, false> t9;   // 8th order, double-double positions
    static_assert(VariantTable<4, false>::count == 20, "keep kNumVariants in hb_capi.cu in step");
    if (v < 0 || v >= VariantTable<4, false>::count) return nullptr;
    switch (order) {
    case 4: return &t4.v[v];
    case 6: return &t6.v[v];
    case 8: return &t8.v[v];
    case 9: return &t9.v[v];
    }
    return nullptr;
}

}  // namespace hb
