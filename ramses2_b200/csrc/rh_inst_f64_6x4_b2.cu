// Pencil-kernel instantiations: double bulk storage, 6x4-oct XY tiles,
// registers sized for 2 CTA(s) per SM; slope types 0-2 x llf/hll/hllc.
#include "rh_launch.h"
namespace rh {
static TileRegistrar<double, 6, 4, 2> reg_f64_6x4_b2;
}
