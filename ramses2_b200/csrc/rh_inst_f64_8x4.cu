// Pencil-kernel instantiations: double bulk arithmetic, 8x4-oct XY tiles,
// slope types 0-2 x Riemann solvers llf/hll/hllc.
#include "rh_launch.h"
namespace rh {
static TileRegistrar<double, 8, 4> reg_f64_8x4;
}
