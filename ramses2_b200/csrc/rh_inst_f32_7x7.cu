// Pencil-kernel instantiations: float bulk arithmetic, 7x7-oct XY tiles,
// slope types 0-2 x Riemann solvers llf/hll/hllc.
#include "rh_launch.h"
namespace rh {
static TileRegistrar<float, 7, 7> reg_f32_7x7;
}
