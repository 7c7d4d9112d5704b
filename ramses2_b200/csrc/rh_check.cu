// rh_check.cu — device state check of the resident hydro state.
//
// Restates the reference's debug scan of uold after set_uold
// (check_nan_kernel, gpu/gpu_utils.cuf:90-118, run by gpu_check_nan_array,
// gpu/gpu_runner.cuf:5339-5384): one thread per cell, bad cells counted, the
// smallest bad oct index kept, and a mask of what was found:
//   bit 0 (1)  a NaN or Inf in any of the five conserved variables;
//   bit 1 (2)  density <= 0;
//   bit 2 (4)  internal energy E - |rho u|^2 / (2 rho) <= 0, i.e. a negative
//              pressure recovered from the energy (cmpdt's debug stop,
//              hydro/godunov_utils.f90:278-287), for cells of positive density.
// Where the reference prints the first bad oct and stops the run, the library
// returns the counts to the caller (RH_EBADSTATE from rh_coarse_step when the
// check is switched on); the batch marks a problem with a bad cell as stopped.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "ramses_hydro_ext.h"
#include "rh_check.cuh"
#include "rh_internal.h"

namespace rh {

// out[0] += bad cells, out[1] = min(out[1], first bad oct, 1-based), out[2] |= mask.
__global__ void check_state_kernel(const double* __restrict__ ud, const float* __restrict__ uf, int fp32,
                                   long long oct0, long long noct, unsigned* __restrict__ out) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  unsigned bad = 0;
  if (i < noct * 8) bad = load_cell_bits(ud, uf, fp32, oct0 + (i >> 3), (int)(i & 7));
  if (bad) {
    atomicAdd(&out[0], 1u);
    atomicMin(&out[1], (unsigned)(oct0 + (i >> 3) + 1));
    atomicOr(&out[2], bad);
  }
}

int check_enqueue(long long oct0, long long noct, unsigned* d_out) {
  Context& c = ctx();
  RH_CUDA(cudaMemsetAsync(d_out, 0, 3 * sizeof(unsigned), c.stream));
  RH_CUDA(cudaMemsetAsync(d_out + 1, 0xff, sizeof(unsigned), c.stream));
  if (noct <= 0) return RH_OK;
  const long long ncell = noct * 8;
  check_state_kernel<<<(unsigned)((ncell + 255) / 256), 256, 0, c.stream>>>(
      c.ud[c.cur], c.uf[c.cur], c.precision == RH_PREC_FP32_BULK ? 1 : 0, oct0, noct, d_out);
  RH_CUDA(cudaGetLastError());
  return RH_OK;
}

// Result slots of the context (3 per level), grown on demand, freed by rh_finalize.
static unsigned* check_buffer(int nlevels) {
  Context& c = ctx();
  if (c.check_cap < nlevels) {
    cudaFree(c.d_check);
    c.d_check = nullptr;
    c.check_cap = 0;
    if (cudaMalloc(&c.d_check, sizeof(unsigned) * 3 * nlevels) != cudaSuccess) return nullptr;
    c.check_cap = nlevels;
  }
  return c.d_check;
}

// The check of every level of the mesh, as rh_coarse_step runs it after
// set_uold when switched on: RH_EBADSTATE names the first bad level.
int check_all_levels() {
  Context& c = ctx();
  const int nl = c.levelmax + 1;
  unsigned* d = check_buffer(nl);
  if (!d) {
    set_error("state check: device buffer allocation failed");
    return RH_ENOMEM;
  }
  int rc;
  for (int l = c.levelmin; l <= c.levelmax; ++l)
    if (c.noct[l] > 0 && (rc = check_enqueue(c.head[l] - 1, c.noct[l], d + 3 * l))) return rc;
  std::vector<unsigned> h(3 * nl);
  RH_CUDA(cudaMemcpyAsync(h.data(), d, sizeof(unsigned) * 3 * nl, cudaMemcpyDeviceToHost, c.stream));
  RH_CUDA(cudaStreamSynchronize(c.stream));
  for (int l = c.levelmin; l <= c.levelmax; ++l) {
    if (c.noct[l] > 0 && h[3 * l] > 0) {
      set_error("state check: level %d has %u bad cells, first oct %u, mask %u (1 NaN/Inf, 2 rho<=0, "
                "4 internal energy<=0)", l, h[3 * l], h[3 * l + 1], h[3 * l + 2]);
      return RH_EBADSTATE;
    }
  }
  return RH_OK;
}

}  // namespace rh

using namespace rh;

extern "C" {

int rh_check_state(int head_idx, int num_octs, int* nbad, int* first_oct, int* mask) {
  Context& c = ctx();
  if (!c.inited || !c.have_mesh) {
    set_error("rh_check_state: no mesh (rh_init / rh_set_mesh first)");
    return RH_ESTATE;
  }
  if (head_idx < 1 || num_octs < 0 || (long long)head_idx - 1 + num_octs > c.ngridmax) {
    set_error("rh_check_state: oct range %d + %d outside 1..%d", head_idx, num_octs, c.ngridmax);
    return RH_EINVAL;
  }
  unsigned* d = check_buffer(c.levelmax + 1);
  if (!d) {
    set_error("rh_check_state: device buffer allocation failed");
    return RH_ENOMEM;
  }
  int rc = check_enqueue(head_idx - 1, num_octs, d);
  if (rc) return rc;
  unsigned h[3];
  RH_CUDA(cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
  RH_CUDA(cudaStreamSynchronize(c.stream));
  if (nbad) *nbad = (int)h[0];
  if (first_oct) *first_oct = h[0] ? (int)h[1] : 0;
  if (mask) *mask = (int)h[2];
  return RH_OK;
}

int rh_set_state_check(int on) {
  ctx().state_check = on ? 1 : 0;
  return RH_OK;
}

}  // extern "C"
