// Batch-kernel instantiations: plain FP64 storage, 4x4-oct XY tiles,
// registers sized for 2 CTA(s) per SM; slope types 0-2 x llf/hll/hllc.
#include <type_traits>

#include "rh_batch.cuh"
namespace rh {
static BatchRegistrar<double, 4, 4, 2> breg_f64_4x4_b2;
}
