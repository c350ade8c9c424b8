// Fused passes of n = 128 and 256 in shape variant 3: radix plan 1 and half the pencils per CTA.
#include "qj_fused_run.cuh"

namespace qj {
QJ_DEFINE_SHAPE_VARIANT(3)
}  // namespace qj
