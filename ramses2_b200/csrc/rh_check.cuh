// rh_check.cuh — per-cell test of the device state check (rh_check.cu, and
// the batch runtime's per-problem check): bit 0 NaN/Inf in a conserved
// variable, bit 1 density <= 0, bit 2 internal energy <= 0 at positive
// density (gpu/gpu_utils.cuf:90-118; hydro/godunov_utils.f90:278-287).
#pragma once
#include <cuda_runtime.h>

#include "rh_bulk.h"

namespace rh {

// Bits of one cell (the mask above); r, m1..m3 and E are its conserved values.
__device__ __forceinline__ unsigned cell_state_bits(double r, double m1, double m2, double m3, double E) {
  unsigned bad = 0;
  if (!(fabs(r) <= 1.7976931348623157e308) || !(fabs(m1) <= 1.7976931348623157e308) ||
      !(fabs(m2) <= 1.7976931348623157e308) || !(fabs(m3) <= 1.7976931348623157e308) ||
      !(fabs(E) <= 1.7976931348623157e308))
    bad |= 1u;
  if (r <= 0.0) bad |= 2u;
  else if (!(bad & 1u) && E - 0.5 * (m1 * m1 + m2 * m2 + m3 * m3) / r <= 0.0) bad |= 4u;
  return bad;
}

__device__ __forceinline__ unsigned load_cell_bits(const double* ud, const float* uf, int fp32, long long oct,
                                                   int cell) {
  double r, m1, m2, m3, E;
  if (!fp32) {
    const double* o = ud + oct * 40 + cell;
    r = o[0]; m1 = o[8]; m2 = o[16]; m3 = o[24]; E = o[32];
  } else {
    const float* o = uf + oct * kBulkF + cell;
    r = o[0]; m1 = o[8]; m2 = o[16]; m3 = o[24]; E = ud[oct * kBulkD + cell];
  }
  return cell_state_bits(r, m1, m2, m3, E);
}

}  // namespace rh
