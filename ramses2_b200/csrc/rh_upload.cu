// rh_upload.cu — restriction of a fine level into its parent cells
// (hydro/upload.f90:74-271 upload_fine; the reference's GPU path is
// gpu_upload / upload_kernel, gpu/gpu_runner.cuf:1754-1784,
// gpu/gpu_hydro.cuf:6972-7066).  The averages of a fine oct's 8 cells go
// into its parent cell: one thread per (oct, variable) for the conservative
// averages, one per oct when the internal energy is averaged instead.
//
// upload_fine first zeroes every refined cell of the coarse level; in a
// single-rank mesh every refined cell has its child oct, so the averages
// overwrite all of them and that pass changes nothing — it is not repeated.
#include <cuda_runtime.h>

#include <unordered_map>
#include <vector>

#include "ramses_hydro.h"
#include "rh_internal.h"

namespace rh {

namespace {

inline uint64_t okey(long long x, long long y, long long z) {
  return ((uint64_t)x << 42) | ((uint64_t)y << 21) | (uint64_t)z;
}

// Father (0-based oct, cell) of every oct above levelmin; (-1, -1) otherwise.
int build_fathers() {
  Context& c = ctx();
  std::vector<int2> fa((size_t)c.ngridmax, make_int2(-1, -1));
  for (int l = c.levelmin + 1; l <= c.levelmax; ++l) {
    if (c.noct[l] == 0 || c.noct[l - 1] == 0) continue;
    std::unordered_map<uint64_t, int> coarse;
    coarse.reserve((size_t)c.noct[l - 1] * 2);
    for (int i = 0; i < c.noct[l - 1]; ++i) {
      const int ig = c.head[l - 1] - 1 + i;
      const rh_oct& o = c.grid[ig];
      coarse[okey(o.ckey[0], o.ckey[1], o.ckey[2])] = ig;
    }
    for (int i = 0; i < c.noct[l]; ++i) {
      const int ig = c.head[l] - 1 + i;
      const rh_oct& o = c.grid[ig];
      auto it = coarse.find(okey(o.ckey[0] >> 1, o.ckey[1] >> 1, o.ckey[2] >> 1));
      if (it == coarse.end()) {
        set_error("oct %d of level %d has no parent oct at level %d", ig + 1, l, l - 1);
        return RH_EINVAL;
      }
      fa[ig] = make_int2(it->second, (o.ckey[0] & 1) + 2 * (o.ckey[1] & 1) + 4 * (o.ckey[2] & 1));
    }
  }
  RH_CUDA(cudaMalloc(&c.d_father, sizeof(int2) * fa.size()));
  RH_CUDA(cudaMemcpy(c.d_father, fa.data(), sizeof(int2) * fa.size(), cudaMemcpyHostToDevice));
  return RH_OK;
}

// Sequential sum of the 8 cells, then / 8, as the reference's loop.
__device__ __forceinline__ double avg8(const double* v) {
  double a = 0.0;
#pragma unroll
  for (int i = 0; i < 8; ++i) a = __dadd_rn(a, v[i]);
  return __ddiv_rn(a, 8.0);
}

__device__ __forceinline__ double ekin_of(double r, double m1, double m2, double m3, double smallr) {
  const double rm = r > smallr ? r : smallr;
  double e = 0.0;
  e = __dadd_rn(e, __ddiv_rn(__dmul_rn(0.5, __dmul_rn(m1, m1)), rm));
  e = __dadd_rn(e, __ddiv_rn(__dmul_rn(0.5, __dmul_rn(m2, m2)), rm));
  e = __dadd_rn(e, __ddiv_rn(__dmul_rn(0.5, __dmul_rn(m3, m3)), rm));
  return e;
}

// One fine oct per thread.  FP64: ud = [oct][5][8].  FP32-bulk: the records
// of rh_bulk.h through their float (uf) and E (ud) views; averages in FP64.
__global__ void upload_kernel(double* __restrict__ ud, float* __restrict__ uf, int fp32,
                              const int2* __restrict__ father, long long o0, long long n, int internal_energy,
                              double smallr) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long o = o0 + i;
  const int2 fa = father[o];
  if (fa.x < 0) return;
  double u[5][8];
  if (!fp32) {
    const double* s = ud + o * 40;
#pragma unroll
    for (int v = 0; v < 5; ++v)
#pragma unroll
      for (int c = 0; c < 8; ++c) u[v][c] = s[v * 8 + c];
  } else {
    const float* s = uf + o * kBulkF;
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int c = 0; c < 8; ++c) u[v][c] = (double)s[v * 8 + c];
#pragma unroll
    for (int c = 0; c < 8; ++c) u[4][c] = ud[o * kBulkD + c];
  }
  double a[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) a[v] = avg8(u[v]);
  if (internal_energy) {
    // average = (average + E) - ekin per cell, in the reference's order
    double e = 0.0;
#pragma unroll
    for (int c = 0; c < 8; ++c)
      e = __dsub_rn(__dadd_rn(e, u[4][c]), ekin_of(u[0][c], u[1][c], u[2][c], u[3][c], smallr));
    double r[4];
    if (!fp32) {
      for (int v = 0; v < 4; ++v) r[v] = a[v];
    } else {
      for (int v = 0; v < 4; ++v) r[v] = (double)(float)a[v];  // the parent's stored values
    }
    a[4] = __dadd_rn(__ddiv_rn(e, 8.0), ekin_of(r[0], r[1], r[2], r[3], smallr));
  }
  const long long p = fa.x;
  if (!fp32) {
    double* d = ud + p * 40 + fa.y;
#pragma unroll
    for (int v = 0; v < 5; ++v) d[v * 8] = a[v];
  } else {
    float* d = uf + p * kBulkF + fa.y;
#pragma unroll
    for (int v = 0; v < 4; ++v) d[v * 8] = (float)a[v];
    ud[p * kBulkD + fa.y] = a[4];
  }
}

// Conservative averages (interpol_var = 0): one thread per (fine oct,
// variable), so that consecutive threads read consecutive runs of the oct
// records (64 bytes each in FP64, 32 bytes of floats or the 64-byte energy
// run in FP32-bulk) and a warp's loads coalesce; the per-oct thread above
// strides 320 bytes from lane to lane.  Same sums in the same order.
__global__ void upload_cons_kernel(double* __restrict__ ud, float* __restrict__ uf, int fp32,
                                   const int2* __restrict__ father, long long o0, long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n * 5) return;
  const long long o = o0 + i / 5;
  const int v = (int)(i - (i / 5) * 5);
  const int2 fa = father[o];
  if (fa.x < 0) return;
  double u[8];
  if (!fp32 || v == 4) {
    const double2* s = reinterpret_cast<const double2*>(fp32 ? ud + o * kBulkD : ud + o * 40 + v * 8);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double2 q = s[k];
      u[2 * k] = q.x;
      u[2 * k + 1] = q.y;
    }
  } else {
    const float4* s = reinterpret_cast<const float4*>(uf + o * kBulkF + v * 8);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const float4 q = s[k];
      u[4 * k] = q.x; u[4 * k + 1] = q.y; u[4 * k + 2] = q.z; u[4 * k + 3] = q.w;
    }
  }
  const double a = avg8(u);
  const long long p = fa.x;
  if (!fp32) ud[p * 40 + 8 * v + fa.y] = a;
  else if (v < 4) uf[p * kBulkF + 8 * v + fa.y] = (float)a;
  else ud[p * kBulkD + fa.y] = a;
}

}  // namespace
}  // namespace rh

namespace rh {

// rh_upload's work on a given stream (rh_coarse_step queues the restrictions
// of its concurrent levels behind the work each one depends on).
int upload_on(int head_idx, int num_octs, int internal_energy, double smallr, cudaStream_t st) {
  Context& c = ctx();
  if (num_octs == 0) return RH_OK;
  if (head_idx < 1 || num_octs < 0 || head_idx - 1 + (long long)num_octs > c.ngridmax) {
    set_error("rh_upload: range outside the mesh");
    return RH_EINVAL;
  }
  if (!(smallr >= 0)) {
    set_error("rh_upload: smallr must be >= 0");
    return RH_EINVAL;
  }
  if (!c.d_father) {
    int rc = build_fathers();
    if (rc) return rc;
  }
  const long long n = num_octs;
  const int fp32 = c.precision == RH_PREC_FP32_BULK ? 1 : 0;
  if (internal_energy) {
    const int threads = 128;
    upload_kernel<<<(unsigned)((n + threads - 1) / threads), threads, 0, st>>>(
        c.ud[c.cur], c.uf[c.cur], fp32, c.d_father, head_idx - 1, n, 1, smallr);
  } else {
    const int threads = 160;  // 32 octs x 5 variables
    upload_cons_kernel<<<(unsigned)((n * 5 + threads - 1) / threads), threads, 0, st>>>(
        c.ud[c.cur], c.uf[c.cur], fp32, c.d_father, head_idx - 1, n);
  }
  RH_CUDA(cudaGetLastError());
  return RH_OK;
}

}  // namespace rh

using namespace rh;

extern "C" int rh_upload(int head_idx, int num_octs, int internal_energy, double gamma, double smallr,
                         double smallc2) {
  Context& c = ctx();
  if (!c.inited || !c.have_mesh) {
    set_error("rh_upload: rh_init and rh_set_mesh first");
    return RH_ESTATE;
  }
  (void)gamma;
  (void)smallc2;
  return upload_on(head_idx, num_octs, internal_energy, smallr, c.stream);
}
