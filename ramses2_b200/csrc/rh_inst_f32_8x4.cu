// Pencil-kernel instantiations: float bulk arithmetic, 8x4-oct XY tiles,
// slope types 0-2 x Riemann solvers llf/hll/hllc.
#include "rh_launch.h"
namespace rh {
static TileRegistrar<float, 8, 4> reg_f32_8x4;
}
