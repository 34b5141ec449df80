// hb_force_mixed.cu -- mixed-precision force kernel instantiations (orders 4, 6, 8).
#include "hb_force_table.cuh"

namespace hb {

const ForceVariant *force_variant_mixed(int order, int v)
{
    static const VariantTable<4, true> t4;
    static const VariantTable<6, true> t6;
    static const VariantTable<8, true> t8;
    if (v < 0 || v >= VariantTable<4, true>::count) return nullptr;
    switch (order) {
    case 4: return &t4.v[v];
    case 6: return &t6.v[v];
    case 8: return &t8.v[v];
    }
    return nullptr;
}

}  // namespace hb
