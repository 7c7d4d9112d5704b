// Pencil-kernel instantiations: float bulk storage, 6x4-oct XY tiles,
// registers sized for 2 CTA(s) per SM; slope types 0-2 x llf/hll/hllc.
#include "rh_launch.h"
namespace rh {
static TileRegistrar<float, 6, 4, 2> reg_f32_6x4_b2;
}
