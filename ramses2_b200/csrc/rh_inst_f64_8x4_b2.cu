// Pencil-kernel instantiations: double bulk storage, 8x4-oct XY tiles,
// registers sized for 2 CTA(s) per SM; slope types 0-2 x llf/hll/hllc.
#include "rh_launch.h"
namespace rh {
static TileRegistrar<double, 8, 4, 2> reg_f64_8x4_b2;
}
