// Batch-kernel instantiations: plain FP64 storage, 8x8-oct XY tiles,
// registers sized for 1 CTA(s) per SM; slope types 0-2 x llf/hll/hllc.
#include <type_traits>

#include "rh_batch.cuh"
namespace rh {
static BatchRegistrar<double, 8, 8, 1> breg_f64_8x8_b1;
}
