// Pencil-kernel instantiations: double bulk arithmetic, 8x8-oct XY tiles,
// slope types 0-2 x Riemann solvers llf/hll/hllc.
#include "rh_launch.h"
namespace rh {
static TileRegistrar<double, 8, 8> reg_f64_8x8;
}
