// Pencil-kernel instantiations: double bulk storage, 7x7-oct XY tiles,
// registers sized for 1 CTA(s) per SM; slope types 0-2 x llf/hll/hllc.
#include "rh_launch.h"
namespace rh {
static TileRegistrar<double, 7, 7, 1> reg_f64_7x7_b1;
}
