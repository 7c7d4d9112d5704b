// Coarse-fine (AMR) pencil-kernel instantiations: double bulk storage,
// 8x4-oct XY tiles, registers sized for 2 CTAs per SM.
#include "rh_launch.h"
namespace rh {
static TileRegistrar<double, 8, 4, 2, true> reg_amr_f64_8x4_b2;
}
