// rh_flag.cu — gradient refinement flags of a level (hydro_flag,
// hydro/hydro_flag.f90:7-159, with hydro_refine, hydro/godunov_utils.f90:
// 6-223; the reference's GPU path is hydro_flag_kernel, gpu/gpu_hydro.cuf:
// 6690-6902).
//
// Per level a table gives, for each oct and each of the six face directions,
// where the neighbour cells across that face live: an oct of the same level,
// the parent cell of the missing neighbour oct (one level down), or — outside
// a non-periodic box — the boundary ghost, whose density and pressure equal
// the boundary cell's (zero-gradient copy / reflexive mirror,
// amr/boundaries.f90).  One thread per cell evaluates the criteria in FP64
// with correctly rounded operations in the reference's order.
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

// Neighbour-across-face table of level l: [noct][6] int2 (direction 2d+s,
// s = 0 low / 1 high): (oct, -1) same level, (oct, cell) parent cell one level
// down, (-1, -1) boundary ghost (the cell itself).
int build_face_table(int l) {
  Context& c = ctx();
  std::unordered_map<uint64_t, int> same, coarse;
  same.reserve((size_t)c.noct[l] * 2);
  for (int i = 0; i < c.noct[l]; ++i) {
    const rh_oct& o = c.grid[c.head[l] - 1 + i];
    same[okey(o.ckey[0], o.ckey[1], o.ckey[2])] = c.head[l] - 1 + i;
  }
  if (l > c.levelmin && c.noct[l - 1] > 0) {
    coarse.reserve((size_t)c.noct[l - 1] * 2);
    for (int i = 0; i < c.noct[l - 1]; ++i) {
      const rh_oct& o = c.grid[c.head[l - 1] - 1 + i];
      coarse[okey(o.ckey[0], o.ckey[1], o.ckey[2])] = c.head[l - 1] - 1 + i;
    }
  }
  const long long nxo[3] = {(long long)c.box_nx[0] << (l - 1), (long long)c.box_nx[1] << (l - 1),
                            (long long)c.box_nx[2] << (l - 1)};
  std::vector<int2> tab((size_t)c.noct[l] * 6);
  for (int i = 0; i < c.noct[l]; ++i) {
    const rh_oct& o = c.grid[c.head[l] - 1 + i];
    for (int n = 0; n < 6; ++n) {
      const int d = n / 2;
      long long k[3] = {o.ckey[0], o.ckey[1], o.ckey[2]};
      k[d] += (n & 1) ? 1 : -1;
      int2 e = make_int2(-1, -1);
      bool outside = false;
      if (k[d] < 0 || k[d] >= nxo[d]) {
        if (c.periodic[d]) k[d] = (k[d] + nxo[d]) % nxo[d];
        else outside = true;
      }
      if (!outside) {
        auto it = same.find(okey(k[0], k[1], k[2]));
        if (it != same.end()) {
          e = make_int2(it->second, -1);
        } else {
          auto jt = coarse.find(okey(k[0] >> 1, k[1] >> 1, k[2] >> 1));
          if (jt == coarse.end()) {
            set_error("hydro flag: oct %d of level %d has neither a neighbour nor its parent cell",
                      c.head[l] + i, l);
            return RH_EINVAL;
          }
          e = make_int2(jt->second, (int)((k[0] & 1) + 2 * (k[1] & 1) + 4 * (k[2] & 1)));
        }
      }
      tab[(size_t)i * 6 + n] = e;
    }
  }
  if (c.d_face.size() < (size_t)c.levelmax + 1) c.d_face.resize(c.levelmax + 1, nullptr);
  RH_CUDA(cudaMalloc(&c.d_face[l], sizeof(int2) * std::max<size_t>(1, tab.size())));
  RH_CUDA(cudaMemcpy(c.d_face[l], tab.data(), sizeof(int2) * tab.size(), cudaMemcpyHostToDevice));
  return RH_OK;
}

struct FlagK {
  double err_d, err_p, err_u, floor_d, floor_p, floor_u, gamma, smallr;
};

__device__ __forceinline__ void load(const double* ud, const float* uf, int fp32, long long oct, int cell,
                                     double* u) {
  if (!fp32) {
    const double* s = ud + oct * 40 + cell;
#pragma unroll
    for (int v = 0; v < 5; ++v) u[v] = s[8 * v];
  } else {
    const float* s = uf + oct * kBulkF + cell;
#pragma unroll
    for (int v = 0; v < 4; ++v) u[v] = (double)s[8 * v];
    u[4] = ud[oct * kBulkD + cell];
  }
}

#define DADD __dadd_rn
#define DSUB __dsub_rn
#define DMUL __dmul_rn
#define DDIV __ddiv_rn

__device__ __forceinline__ double fmax_(double a, double b) { return a > b ? a : b; }

// hydro_refine (godunov_utils.f90:6-223) for one direction.
__device__ bool refine_1d(const double* gi, const double* mi, const double* di, const FlagK& K) {
  double g[5], m[5], d[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) { g[v] = gi[v]; m[v] = mi[v]; d[v] = di[v]; }
  g[0] = fmax_(g[0], K.smallr);
  m[0] = fmax_(m[0], K.smallr);
  d[0] = fmax_(d[0], K.smallr);
#pragma unroll
  for (int k = 1; k <= 3; ++k) { g[k] = DDIV(g[k], g[0]); m[k] = DDIV(m[k], m[0]); d[k] = DDIV(d[k], d[0]); }
  double eg = 0, em = 0, ed = 0;
#pragma unroll
  for (int k = 1; k <= 3; ++k) {
    eg = DADD(eg, DMUL(DMUL(0.5, g[0]), DMUL(g[k], g[k])));
    em = DADD(em, DMUL(DMUL(0.5, m[0]), DMUL(m[k], m[k])));
    ed = DADD(ed, DMUL(DMUL(0.5, d[0]), DMUL(d[k], d[k])));
  }
  const double gm1 = DSUB(K.gamma, 1.0);
  const double pg = DMUL(gm1, DSUB(g[4], eg)), pm = DMUL(gm1, DSUB(m[4], em)), pd = DMUL(gm1, DSUB(d[4], ed));
  bool ok = false;
  if (K.err_d >= 0.) {
    const double e = DMUL(2.0, fmax_(fabs(DDIV(DSUB(d[0], m[0]), DADD(DADD(d[0], m[0]), K.floor_d))),
                                     fabs(DDIV(DSUB(m[0], g[0]), DADD(DADD(m[0], g[0]), K.floor_d)))));
    ok = ok || e > K.err_d;
  }
  if (K.err_p >= 0.) {
    const double e = DMUL(2.0, fmax_(fabs(DDIV(DSUB(pd, pm), DADD(DADD(pd, pm), K.floor_p))),
                                     fabs(DDIV(DSUB(pm, pg), DADD(DADD(pm, pg), K.floor_p)))));
    ok = ok || e > K.err_p;
  }
  if (K.err_u >= 0.) {
    const double fu2 = DMUL(K.floor_u, K.floor_u);
    const double cg = __dsqrt_rn(fmax_(DDIV(DMUL(K.gamma, pg), g[0]), fu2));
    const double cm = __dsqrt_rn(fmax_(DDIV(DMUL(K.gamma, pm), m[0]), fu2));
    const double cd = __dsqrt_rn(fmax_(DDIV(DMUL(K.gamma, pd), d[0]), fu2));
#pragma unroll
    for (int k = 1; k <= 3; ++k) {
      const double vg = g[k], vm = m[k], vd = d[k];
      const double e = DMUL(
          2.0, fmax_(fabs(DDIV(DSUB(vd, vm), DADD(DADD(DADD(DADD(cd, cm), fabs(vd)), fabs(vm)), K.floor_u))),
                     fabs(DDIV(DSUB(vm, vg), DADD(DADD(DADD(DADD(cm, cg), fabs(vm)), fabs(vg)), K.floor_u)))));
      ok = ok || e > K.err_u;
    }
  }
  return ok;
}

__global__ void flag_kernel(const double* __restrict__ ud, const float* __restrict__ uf, int fp32,
                            const int2* __restrict__ face, long long o0, long long noct, FlagK K,
                            unsigned char* __restrict__ out) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= noct * 8) return;
  const long long li = i >> 3;
  const long long oct = o0 + li;
  const int cell = (int)(i & 7);
  double um[5];
  load(ud, uf, fp32, oct, cell, um);
  bool ok = false;
#pragma unroll 1
  for (int d = 0; d < 3; ++d) {
    double nb[2][5];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const int bit = (cell >> d) & 1;
      const int ncell = cell ^ (1 << d);
      const bool inside = s == 0 ? bit == 1 : bit == 0;  // neighbour in the same oct
      if (inside) {
        load(ud, uf, fp32, oct, ncell, nb[s]);
      } else {
        const int2 e = face[li * 6 + 2 * d + s];
        if (e.x < 0) {
#pragma unroll
          for (int v = 0; v < 5; ++v) nb[s][v] = um[v];
        } else if (e.y < 0) {
          load(ud, uf, fp32, e.x, ncell, nb[s]);
        } else {
          load(ud, uf, fp32, e.x, e.y, nb[s]);
        }
      }
    }
    ok = refine_1d(nb[0], um, nb[1], K) || ok;
  }
  out[i] = ok ? 1 : 0;
}

}  // namespace
}  // namespace rh

using namespace rh;

extern "C" int rh_hydro_flag(int ilevel, const rh_flag_params* f, double gamma, double smallr, int32_t* flag1,
                             long long* nflag) {
  Context& c = ctx();
  if (!c.inited || !c.have_mesh) {
    set_error("rh_hydro_flag: rh_init and rh_set_mesh first");
    return RH_ESTATE;
  }
  if (!f || !flag1 || ilevel < c.levelmin || ilevel > c.levelmax || !(gamma > 1) || !(smallr >= 0)) {
    set_error("rh_hydro_flag: bad level, parameters or null pointer");
    return RH_EINVAL;
  }
  if (nflag) *nflag = 0;
  const long long n = c.noct[ilevel];
  if (n == 0) return RH_OK;
  if (c.d_face.size() <= (size_t)ilevel || !c.d_face[ilevel]) {
    int rc = build_face_table(ilevel);
    if (rc) return rc;
  }
  unsigned char* d_out = nullptr;
  RH_CUDA(cudaMalloc(&d_out, (size_t)n * 8));
  const FlagK K{f->err_grad_d, f->err_grad_p, f->err_grad_u, f->floor_d, f->floor_p, f->floor_u, gamma, smallr};
  const int threads = 256;
  flag_kernel<<<(unsigned)((n * 8 + threads - 1) / threads), threads, 0, c.stream>>>(
      c.ud[c.cur], c.uf[c.cur], c.precision == RH_PREC_FP32_BULK ? 1 : 0, c.d_face[ilevel], c.head[ilevel] - 1, n, K,
      d_out);
  cudaError_t e = cudaGetLastError();
  std::vector<unsigned char> h((size_t)n * 8);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), d_out, h.size(), cudaMemcpyDeviceToHost, c.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
  cudaFree(d_out);
  if (e != cudaSuccess) return cuda_fail(e, "rh_hydro_flag");
  long long newly = 0;
  int32_t* fl = flag1 + (size_t)(c.head[ilevel] - 1) * 8;
  for (size_t i = 0; i < h.size(); ++i) {
    if (!h[i]) continue;
    if (fl[i] == 0) ++newly;
    fl[i] = 1;
  }
  if (nflag) *nflag = newly;
  return RH_OK;
}
