// Pencil-kernel instantiations: float bulk storage, 7x7-oct XY tiles,
// registers sized for 2 CTA(s) per SM; slope types 0-2 x llf/hll/hllc.
#include "rh_launch.h"
namespace rh {
static TileRegistrar<float, 7, 7, 2> reg_f32_7x7_b2;
}
