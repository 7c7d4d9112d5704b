// Coarse-fine (AMR) pencil-kernel instantiations: float bulk storage,
// 4x4-oct XY tiles, registers sized for 2 CTAs per SM.
#include "rh_launch.h"
namespace rh {
static TileRegistrar<float, 4, 4, 2, true> reg_amr_f32_4x4_b2;
}
