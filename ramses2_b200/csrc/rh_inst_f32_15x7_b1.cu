// Pencil-kernel instantiations: float bulk storage, 15x7-oct XY tiles (a
// 32-wide ring: one ring row per warp), registers sized for 1 CTA per SM;
// slope types 0-2 x llf/hll/hllc.
#include "rh_launch.h"
namespace rh {
static TileRegistrar<float, 15, 7, 1> reg_f32_15x7_b1;
}
