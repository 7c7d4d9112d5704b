// Coarse-fine (AMR) pencil-kernel instantiations: float bulk storage,
// 7x7-oct XY tiles, registers sized for 2 CTAs per SM.
#include "rh_launch.h"
namespace rh {
static TileRegistrar<float, 7, 7, 2, true> reg_amr_f32_7x7_b2;
}
