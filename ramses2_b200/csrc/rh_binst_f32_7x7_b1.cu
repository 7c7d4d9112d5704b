// Batch-kernel instantiations: FP32 bulk storage, 7x7-oct XY tiles,
// registers sized for 1 CTA(s) per SM; slope types 0-2 x llf/hll/hllc.
#include <type_traits>

#include "rh_batch.cuh"
namespace rh {
static BatchRegistrar<float, 7, 7, 1> breg_f32_7x7_b1;
}
