// Fused passes of n = 128 and 256 in shape variant 1: radix plan 1 (half the elements per thread), default tiles.
#include "qj_fused_run.cuh"

namespace qj {
QJ_DEFINE_SHAPE_VARIANT(1)
}  // namespace qj
