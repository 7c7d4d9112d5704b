// rh_amr.cu — coarse-fine levels: pencil tables over a sparse level,
// interpolated ghost octs, and their prolongation from the coarser level.
//
// A level that does not fill its box gets pencils only where it has octs:
// for every XY tile of octs, each maximal run of consecutive z layers holding
// octs (cut at lz layers) is a pencil.  Every position of a pencil's
// neighbourhood that holds no oct of the level becomes an interpolated ghost
// oct (stored after ngridmax in the state arrays), filled before each Godunov
// step from its father cell and the father's six neighbours at level l-1 by
// interpol_hydro (hydro/interpol_hydro.f90:5-109) — the role of the cache octs
// that gpu_refresh_cache / refresh_cache_octs_kernel maintain in the reference
// (gpu/gpu_runner.cuf:1295-1338, gpu/gpu_refine.cuf:2447-2538) and of the
// interpolation branch of godfine1 (hydro/godunov_fine.f90:487-556).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <unordered_map>
#include <vector>

#include "rh_internal.h"

namespace rh {

namespace {

inline uint64_t pack3(long long x, long long y, long long z) {
  const uint64_t M = (1ull << 21) - 1;
  return (((uint64_t)(x + 4) & M) << 42) | (((uint64_t)(y + 4) & M) << 21) | ((uint64_t)(z + 4) & M);
}

inline long long wrapc(long long v, long long n, int periodic) {
  if (periodic) {
    v %= n;
    if (v < 0) v += n;
    return v;
  }
  return v < 0 ? 0 : (v >= n ? n - 1 : v);
}

inline long long floordiv2(long long a) { return a >= 0 ? a / 2 : -((-a + 1) / 2); }

}  // namespace

int build_amr_tables(int l, const TileCfg& cfg, long long gbase) {
  Context& c = ctx();
  LevelTables& T = c.levels[l];
  T.cfg = cfg;
  const long long n[3] = {(long long)c.box_nx[0] << (l - 1), (long long)c.box_nx[1] << (l - 1),
                          (long long)c.box_nx[2] << (l - 1)};
  T.nxo = (int)n[0];
  T.nyo = (int)n[1];
  T.nzo = (int)n[2];
  if (l - 1 < c.levelmin || c.noct[l - 1] == 0) {
    set_error("level %d does not fill its box and has no coarser level to interpolate from", l);
    return RH_EINVAL;
  }
  // oct dictionaries of levels l and l-1
  std::unordered_map<uint64_t, int> fine, coarse;
  fine.reserve((size_t)c.noct[l] * 2);
  coarse.reserve((size_t)c.noct[l - 1] * 2);
  for (int i = 0; i < c.noct[l]; ++i) {
    const rh_oct& o = c.grid[(size_t)c.head[l] - 1 + i];
    fine[pack3(o.ckey[0], o.ckey[1], o.ckey[2])] = c.head[l] - 1 + i;
  }
  for (int i = 0; i < c.noct[l - 1]; ++i) {
    const rh_oct& o = c.grid[(size_t)c.head[l - 1] - 1 + i];
    coarse[pack3(o.ckey[0], o.ckey[1], o.ckey[2])] = c.head[l - 1] - 1 + i;
  }
  // pencils: XY tiles x runs of occupied z layers
  std::map<std::pair<long long, long long>, std::vector<long long>> tiles;
  for (int i = 0; i < c.noct[l]; ++i) {
    const rh_oct& o = c.grid[(size_t)c.head[l] - 1 + i];
    tiles[{o.ckey[1] / cfg.tyo, o.ckey[0] / cfg.txo}].push_back(o.ckey[2]);
  }
  T.phdr.clear();
  T.poff.clear();
  T.ptab.clear();
  T.gsrc_oct.clear();
  T.gsrc_cf.clear();
  T.gfather.clear();
  T.gbase = gbase;
  std::unordered_map<uint64_t, int> ghost_id;
  const int OW = cfg.txo + 2, OH = cfg.tyo + 2;
  const long long nc[3] = {n[0], n[1], n[2]};  // level l-1 cells per edge = level l octs per edge
  // Get (or create) the interpolated ghost for fine oct key k (in domain).
  auto ghost = [&](const long long* k) -> int {
    const uint64_t key = pack3(k[0], k[1], k[2]);
    auto it = ghost_id.find(key);
    if (it != ghost_id.end()) return it->second;
    // father cell = coarse cell k; its six neighbours k -+ e_d (boundary-mapped)
    int srcs[7];
    unsigned char cf[7];
    const int shift[7][3] = {{0, 0, 0}, {-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    for (int j = 0; j < 7; ++j) {
      long long q[3];
      unsigned char flip = 0;
      for (int d = 0; d < 3; ++d) {
        q[d] = k[d] + shift[j][d];
        if (q[d] < 0 || q[d] >= nc[d]) {
          if (c.periodic[d]) {
            q[d] = wrapc(q[d], nc[d], 1);
          } else {
            const int bt = c.bound_type[2 * d + (q[d] < 0 ? 0 : 1)];
            q[d] = q[d] < 0 ? 0 : nc[d] - 1;  // distance 1: mirror and clamp pick the same cell
            if (bt == RH_BOUND_REFLEXIVE) flip |= (unsigned char)(1u << d);
          }
        }
      }
      const long long oc[3] = {floordiv2(q[0]), floordiv2(q[1]), floordiv2(q[2])};
      auto ci = coarse.find(pack3(oc[0], oc[1], oc[2]));
      if (ci == coarse.end()) return -1;
      srcs[j] = ci->second;
      const int cell = (int)((q[0] - 2 * oc[0]) + 2 * (q[1] - 2 * oc[1]) + 4 * (q[2] - 2 * oc[2]));
      cf[j] = (unsigned char)(cell | (flip << 3));
    }
    const int id = (int)T.gfather.size();
    for (int j = 0; j < 7; ++j) {
      T.gsrc_oct.push_back(srcs[j]);
      T.gsrc_cf.push_back(cf[j]);
    }
    T.gfather.push_back(make_int2(srcs[0], cf[0] & 7));
    ghost_id[key] = id;
    return id;
  };
  for (auto& kv : tiles) {
    std::vector<long long>& zs = kv.second;
    std::sort(zs.begin(), zs.end());
    zs.erase(std::unique(zs.begin(), zs.end()), zs.end());
    const long long oy0 = kv.first.first * cfg.tyo, ox0 = kv.first.second * cfg.txo;
    size_t i = 0;
    while (i < zs.size()) {
      const long long z0 = zs[i];
      size_t j = i;
      while (j + 1 < zs.size() && zs[j + 1] == zs[j] + 1 && zs[j + 1] - z0 < cfg.lz) ++j;
      const int L = (int)(zs[j] - z0 + 1);
      T.phdr.push_back(make_int4((int)ox0, (int)oy0, (int)z0, L));
      T.poff.push_back((long long)T.ptab.size());
      for (int r = 0; r < L + 2; ++r)
        for (int jj = 0; jj < OH; ++jj)
          for (int ii = 0; ii < OW; ++ii) {
            const long long k[3] = {wrapc(ox0 - 1 + ii, n[0], c.periodic[0]), wrapc(oy0 - 1 + jj, n[1], c.periodic[1]),
                                    wrapc(z0 - 1 + r, n[2], c.periodic[2])};
            auto fi = fine.find(pack3(k[0], k[1], k[2]));
            int ent;
            if (fi != fine.end()) {
              ent = fi->second;
            } else {
              const int g = ghost(k);
              ent = g < 0 ? -1 : (int)(gbase + g);
            }
            T.ptab.push_back(ent);
          }
      i = j + 1;
    }
  }
  // every position within one oct of an oct this pencil updates must have a
  // source (the cell stencils and ring-cell slopes read them); farther
  // positions of the table are never read
  for (size_t p = 0; p < T.phdr.size(); ++p) {
    const int4 h = T.phdr[p];
    const int* tab = T.ptab.data() + T.poff[p];
    auto at = [&](int r, int jj, int ii) { return tab[((long long)r * OH + jj) * OW + ii]; };
    for (int r = 1; r <= h.w; ++r)
      for (int jj = 1; jj < OH - 1; ++jj)
        for (int ii = 1; ii < OW - 1; ++ii) {
          const int e = at(r, jj, ii);
          if (e < 0 || e >= c.ngridmax) continue;  // not an oct of this level
          for (int dr = -1; dr <= 1; ++dr)
            for (int dj = -1; dj <= 1; ++dj)
              for (int di = -1; di <= 1; ++di)
                if (at(r + dr, jj + dj, ii + di) < 0) {
                  set_error("level %d: the coarse neighbourhood of a missing oct next to (%d,%d,%d) does not "
                            "exist (mesh not properly nested)", l, h.x - 1 + ii + di, h.y - 1 + jj + dj,
                            h.z - 1 + r + dr);
                  return RH_EINVAL;
                }
        }
  }
  T.nghost = (int)T.gfather.size();
  T.npencil = (int)T.phdr.size();
  T.ntab = (long long)T.ptab.size();
  T.complete = false;
  return RH_OK;
}

int upload_amr_tables(int l) {
  Context& c = ctx();
  LevelTables& T = c.levels[l];
  RH_CUDA(cudaMalloc(&T.d_phdr, sizeof(int4) * std::max<size_t>(1, T.phdr.size())));
  RH_CUDA(cudaMalloc(&T.d_poff, sizeof(long long) * std::max<size_t>(1, T.poff.size())));
  RH_CUDA(cudaMalloc(&T.d_ptab, sizeof(int) * std::max<size_t>(1, T.ptab.size())));
  RH_CUDA(cudaMalloc(&T.d_cfl_partial, sizeof(double) * 5 * std::max(1, T.npencil)));
  if (!T.phdr.empty()) {
    RH_CUDA(cudaMemcpy(T.d_phdr, T.phdr.data(), sizeof(int4) * T.phdr.size(), cudaMemcpyHostToDevice));
    RH_CUDA(cudaMemcpy(T.d_poff, T.poff.data(), sizeof(long long) * T.poff.size(), cudaMemcpyHostToDevice));
    RH_CUDA(cudaMemcpy(T.d_ptab, T.ptab.data(), sizeof(int) * T.ptab.size(), cudaMemcpyHostToDevice));
  }
  if (T.nghost > 0) {
    RH_CUDA(cudaMalloc(&T.d_gsrc_oct, sizeof(int) * T.gsrc_oct.size()));
    RH_CUDA(cudaMalloc(&T.d_gsrc_cf, T.gsrc_cf.size()));
    RH_CUDA(cudaMemcpy(T.d_gsrc_oct, T.gsrc_oct.data(), sizeof(int) * T.gsrc_oct.size(), cudaMemcpyHostToDevice));
    RH_CUDA(cudaMemcpy(T.d_gsrc_cf, T.gsrc_cf.data(), T.gsrc_cf.size(), cudaMemcpyHostToDevice));
    RH_CUDA(cudaMemcpy(c.d_gfather + (T.gbase - c.ngridmax), T.gfather.data(), sizeof(int2) * T.gfather.size(),
                       cudaMemcpyHostToDevice));
  }
  T.built = true;
  return RH_OK;
}

// ---------------------------------------------------------------------------
// Prolongation of the ghost octs of a level (interpol_hydro.f90:5-109 with the
// limiters of :770-912).  One thread per ghost oct.
// ---------------------------------------------------------------------------
namespace {

__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }

__device__ void limiter_central(const double* a, double* w) {
  // Monotonized central slope, interpol_hydro.f90:798-892
  double xc[8][3];
  for (int ind = 0; ind < 8; ++ind) {
    xc[ind][0] = (double)(ind & 1) - 0.5;
    xc[ind][1] = (double)((ind >> 1) & 1) - 0.5;
    xc[ind][2] = (double)((ind >> 2) & 1) - 0.5;
  }
  for (int d = 0; d < 3; ++d) w[d] = 0.25 * (a[2 * d + 2] - a[2 * d + 1]);
  double ac[8];
  for (int ind = 0; ind < 8; ++ind) ac[ind] = a[0];
  for (int d = 0; d < 3; ++d)
    for (int ind = 0; ind < 8; ++ind) ac[ind] = ac[ind] + 2.0 * w[d] * xc[ind][d];
  double corner = ac[0];
  for (int j = 1; j < 8; ++j) corner = dmax(corner, ac[j]);
  double kernel = a[1];
  for (int j = 2; j <= 6; ++j) kernel = dmax(kernel, a[j]);
  double dk = a[0] - kernel, dc = a[0] - corner;
  double maxl = 0.0;
  if (dk * dc > 0.0) maxl = dmin(1.0, dk / dc);
  corner = ac[0];
  for (int j = 1; j < 8; ++j) corner = dmin(corner, ac[j]);
  kernel = a[1];
  for (int j = 2; j <= 6; ++j) kernel = dmin(kernel, a[j]);
  dk = a[0] - kernel;
  dc = a[0] - corner;
  double minl = 0.0;
  if (dk * dc > 0.0) minl = dmin(1.0, dk / dc);
  const double lim = dmin(minl, maxl);
  for (int d = 0; d < 3; ++d) w[d] = w[d] * lim;
}

__global__ void prolong_kernel(const int* __restrict__ src_oct, const unsigned char* __restrict__ src_cf, int ng,
                               long long gbase, double* ud, float* uf, int fp32, int ivar_mode, int itype,
                               double smallr) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ng) return;
  double u1[7][5];
  for (int j = 0; j < 7; ++j) {
    const long long o = src_oct[g * 7 + j];
    const int cf = src_cf[g * 7 + j];
    const int cell = cf & 7;
    for (int v = 0; v < 5; ++v) {
      double val;
      if (!fp32) val = ud[o * 40 + v * 8 + cell];
      else val = v < 4 ? (double)uf[o * kBulkF + v * 8 + cell] : ud[o * kBulkD + cell];
      if (v >= 1 && v <= 3 && ((cf >> (2 + v)) & 1)) val = -val;  // reflexive boundary: normal momentum
      u1[j][v] = val;
    }
  }
  if (ivar_mode == 1) {
    for (int j = 0; j < 7; ++j) {
      double ekin = 0.0;
      for (int d = 1; d <= 3; ++d) ekin = ekin + 0.5 * (u1[j][d] * u1[j][d]) / dmax(u1[j][0], smallr);
      u1[j][4] = u1[j][4] - ekin - 0.0;
    }
  }
  double u2[8][5];
  for (int v = 0; v < 5; ++v) {
    double a[7], w[3] = {0.0, 0.0, 0.0};
    for (int j = 0; j < 7; ++j) a[j] = u1[j][v];
    if (itype == 1) {  // minmod, interpol_hydro.f90:770-793
      for (int d = 0; d < 3; ++d) {
        const double dl = 0.5 * (a[2 * d + 2] - a[0]);
        const double dr = 0.5 * (a[0] - a[2 * d + 1]);
        w[d] = (dl * dr <= 0.0) ? 0.0 : dmin(fabs(dl), fabs(dr)) * dl / fabs(dl);
      }
    } else if (itype == 2) {
      limiter_central(a, w);
    } else if (itype == 3) {
      for (int d = 0; d < 3; ++d) w[d] = 0.25 * (a[2 * d + 2] - a[2 * d + 1]);
    }
    for (int ind = 0; ind < 8; ++ind) {
      double x = a[0];
      x = x + w[0] * ((double)(ind & 1) - 0.5);
      x = x + w[1] * ((double)((ind >> 1) & 1) - 0.5);
      x = x + w[2] * ((double)((ind >> 2) & 1) - 0.5);
      u2[ind][v] = x;
    }
  }
  if (ivar_mode == 1) {
    for (int ind = 0; ind < 8; ++ind) {
      double ekin = 0.0;
      for (int d = 1; d <= 3; ++d) ekin = ekin + 0.5 * (u2[ind][d] * u2[ind][d]) / dmax(u2[ind][0], smallr);
      u2[ind][4] = u2[ind][4] + ekin + 0.0;
    }
  }
  const long long o = gbase + g;
  for (int ind = 0; ind < 8; ++ind)
    for (int v = 0; v < 5; ++v) {
      if (!fp32) ud[o * 40 + v * 8 + ind] = u2[ind][v];
      else if (v < 4) uf[o * kBulkF + v * 8 + ind] = (float)u2[ind][v];
      else ud[o * kBulkD + ind] = u2[ind][v];
    }
}

}  // namespace

int prolong_ghosts(int l, double smallr, cudaStream_t st) {
  Context& c = ctx();
  LevelTables& T = c.levels[l];
  if (T.nghost == 0) return RH_OK;
  const int threads = 128;
  prolong_kernel<<<(T.nghost + threads - 1) / threads, threads, 0, st ? st : c.stream>>>(
      T.d_gsrc_oct, T.d_gsrc_cf, T.nghost, T.gbase, c.ud[c.cur], c.uf[c.cur],
      c.precision == RH_PREC_FP32_BULK ? 1 : 0, c.interpol_var, c.interpol_type, smallr);
  RH_CUDA(cudaGetLastError());
  return RH_OK;
}

}  // namespace rh
