// Pencil-kernel instantiations: float bulk storage, 8x8-oct XY tiles,
// registers sized for 1 CTA(s) per SM; slope types 0-2 x llf/hll/hllc.
#include "rh_launch.h"
namespace rh {
static TileRegistrar<float, 8, 8, 1> reg_f32_8x8_b1;
}
