// Pencil-kernel instantiations: double bulk arithmetic, 7x7-oct XY tiles,
// slope types 0-2 x Riemann solvers llf/hll/hllc.
#include "rh_launch.h"
namespace rh {
static TileRegistrar<double, 7, 7> reg_f64_7x7;
}
