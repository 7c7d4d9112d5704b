// Pencil-kernel instantiations: double bulk storage, 8x8-oct XY tiles,
// registers sized for 1 CTA(s) per SM; slope types 0-2 x llf/hll/hllc.
#include "rh_launch.h"
namespace rh {
static TileRegistrar<double, 8, 8, 1> reg_f64_8x8_b1;
}
