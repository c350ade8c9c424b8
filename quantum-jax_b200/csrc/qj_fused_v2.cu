// Fused passes of n = 128 and 256 in shape variant 2: default radix plan, half the pencils per CTA.
#include "qj_fused_run.cuh"

namespace qj {
QJ_DEFINE_SHAPE_VARIANT(2)
}  // namespace qj
