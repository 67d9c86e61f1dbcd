// asm_variants.cu -- the table of compiled assembly kernel shapes. Each
// shape is defined in its own translation unit (generated by the build from
// asm_variant_list.h, one RBFB_DEFINE_VARIANT each) so they compile in
// parallel; this file only collects them.
#include "asm_variants.h"

namespace rbfb {

#define RBFB_VARIANT(name, ...) Variant variant_##name();
#define RBFB_BLK_VARIANT(name, ...) Variant variant_##name();
#define RBFB_BLK16_VARIANT(name, ...) Variant variant_##name();
#include "asm_variant_list.h"
#undef RBFB_VARIANT
#undef RBFB_BLK_VARIANT
#undef RBFB_BLK16_VARIANT

const std::vector<Variant>& variants() {
    static const std::vector<Variant> table = {
#define RBFB_VARIANT(name, ...) variant_##name(),
#define RBFB_BLK_VARIANT(name, ...) variant_##name(),
#define RBFB_BLK16_VARIANT(name, ...) variant_##name(),
#include "asm_variant_list.h"
#undef RBFB_VARIANT
#undef RBFB_BLK_VARIANT
#undef RBFB_BLK16_VARIANT
    };
    return table;
}

}  // namespace rbfb
