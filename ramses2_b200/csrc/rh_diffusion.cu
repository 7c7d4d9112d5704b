// rh_diffusion.cu — artificial diffusion (difmag > 0) of a single complete
// level in FP64: the reference's cmpdivu and cmpdiff (hydro/umuscl.f90:
// 2392-2540), which unsplit calls after the Godunov fluxes when difmag > 0
// (umuscl.f90:273-283).
//
// cmpdivu takes the velocity divergence at every cell corner from the
// primitive velocities of the eight cells around it (ctoprim's velocities:
// momentum / max(rho, smallr) plus the half-step gravity term); cmpdiff adds
// to each face flux dt * difmag * min(0, the mean divergence of the face's
// four corners) times the jump of the conserved variables across the face.
// The pencil kernels have already written unew = uold + the Godunov flux
// differences; this pass adds the diffusive flux differences: one kernel
// writes the divergence of every corner of the level ((ncx+1)(ncy+1)(ncz+1)
// values, corner (i,j,k) at the low corner of cell (i,j,k), as the reference
// indexes div), a second one sums the six faces of every cell.  Per face the
// arithmetic is the reference's, operation by operation (explicitly rounded
// intrinsics, so no multiply-add contraction changes a rounding); the sum
// into unew is rounded once more than in the reference, which adds the
// diffusive flux to the Godunov flux before taking the face differences.
// Cells one step outside the box are taken as the pencils take them:
// periodic wrap, else the boundary oct (clamp) with map_coord's cell parity
// and normal-momentum sign (zero gradient or reflexive).
#include <cuda_runtime.h>

#include <algorithm>

#include "rh_godunov.cuh"
#include "rh_internal.h"

namespace rh {

namespace {

struct DiffGeo {
  int ncx, ncy, ncz;  // level extent in cells
  int nxo, nyo, nzo;  // in octs
  int periodic[3];
  int btype[6];
};

__device__ __forceinline__ double A_(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double S_(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double M_(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double min0(double a) { return 0.0 < a ? 0.0 : a; }  // Fortran min(zero, a)

// Oct and cell of level cell (gx, gy, gz), which may lie one cell outside
// the box; flip bit d: the normal momentum d of a mirrored cell is negated.
__device__ __forceinline__ long long diff_cell(const DiffGeo& G, const int* __restrict__ map, int gx, int gy, int gz,
                                               int& cell, unsigned& flip) {
  const int g3[3] = {gx, gy, gz};
  const int nc[3] = {G.ncx, G.ncy, G.ncz};
  const int no[3] = {G.nxo, G.nyo, G.nzo};
  int o[3];
  cell = 0;
  flip = 0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int g = g3[d];
    int par;
    if (G.periodic[d]) {
      g = ((g % nc[d]) + nc[d]) % nc[d];
      par = g & 1;
      o[d] = g >> 1;
    } else {
      const CellMap m = map_coord(g, nc[d], 0, G.btype[2 * d], G.btype[2 * d + 1]);
      par = m.parity;
      if (m.flip) flip |= 1u << d;
      const int od = g >= 0 ? g / 2 : (g - 1) / 2;  // floor(g / 2)
      o[d] = od < 0 ? 0 : (od >= no[d] ? no[d] - 1 : od);
    }
    cell |= par << d;
  }
  return map[((long long)o[2] * G.nyo + o[1]) * G.nxo + o[0]];
}

__device__ __forceinline__ void diff_load(const double* __restrict__ u, long long oct, int cell, unsigned flip,
                                          double* U) {
  const double* p = u + oct * 40 + cell;
#pragma unroll
  for (int n = 0; n < 5; ++n) U[n] = p[8 * n];
#pragma unroll
  for (int d = 0; d < 3; ++d)
    if ((flip >> d) & 1u) U[1 + d] = -U[1 + d];
}

// cmpdivu (umuscl.f90:2396-2440, NDIM=3): one thread per cell corner.
__global__ void corner_div_kernel(const double* __restrict__ u, const int* __restrict__ map, const DiffGeo G,
                                  double smallr, double g0, double g1, double g2, double fact,
                                  double* __restrict__ div) {
  const long long nxn = G.ncx + 1, nyn = G.ncy + 1, nzn = G.ncz + 1;
  const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (id >= nxn * nyn * nzn) return;
  const int i = (int)(id % nxn), j = (int)((id / nxn) % nyn), k = (int)(id / (nxn * nyn));
  // q velocities of cells (i-1+a, j-1+b, k-1+c) as v[c][b][a][0..2]
  double v[2][2][2][3];
#pragma unroll
  for (int c3 = 0; c3 < 2; ++c3)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int a = 0; a < 2; ++a) {
        int cell;
        unsigned fl;
        const long long o = diff_cell(G, map, i - 1 + a, j - 1 + b, k - 1 + c3, cell, fl);
        double U[5];
        diff_load(u, o, cell, fl, U);
        const double r = U[0] > smallr ? U[0] : smallr;  // max(uloc(1), smallr)
        const double oor = __ddiv_rn(1.0, r);
        v[c3][b][a][0] = A_(M_(U[1], oor), g0);
        v[c3][b][a][1] = A_(M_(U[2], oor), g1);
        v[c3][b][a][2] = A_(M_(U[3], oor), g2);
      }
  double ux = 0.0, vy = 0.0, wz = 0.0;
  ux = A_(ux, M_(fact, S_(v[1][1][1][0], v[1][1][0][0])));
  ux = A_(ux, M_(fact, S_(v[1][0][1][0], v[1][0][0][0])));
  vy = A_(vy, M_(fact, S_(A_(S_(v[1][1][1][1], v[1][0][1][1]), v[1][1][0][1]), v[1][0][0][1])));
  ux = A_(ux, M_(fact, S_(A_(S_(v[0][1][1][0], v[0][1][0][0]), v[0][0][1][0]), v[0][0][0][0])));
  vy = A_(vy, M_(fact, S_(A_(S_(v[0][1][1][1], v[0][0][1][1]), v[0][1][0][1]), v[0][0][0][1])));
  double w = S_(v[1][1][1][2], v[0][1][1][2]);
  w = A_(w, v[1][0][1][2]);
  w = S_(w, v[0][0][1][2]);
  w = A_(w, v[1][1][0][2]);
  w = S_(w, v[0][1][0][2]);
  w = A_(w, v[1][0][0][2]);
  w = S_(w, v[0][0][0][2]);
  wz = A_(wz, M_(fact, w));
  div[id] = A_(A_(ux, vy), wz);
}

// cmpdiff (umuscl.f90:2444-2540, NDIM=3, hydro): one thread per cell, its
// six faces' diffusive fluxes differenced into unew.
__global__ void diffuse_cells_kernel(const double* __restrict__ u, double* __restrict__ unew,
                                     const int* __restrict__ map, const DiffGeo G, const double* __restrict__ div,
                                     double dt, double difmag) {
  const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (id >= (long long)G.ncx * G.ncy * G.ncz) return;
  const int cx = (int)(id % G.ncx), cy = (int)((id / G.ncx) % G.ncy), cz = (int)(id / ((long long)G.ncx * G.ncy));
  const long long nxn = G.ncx + 1, nyn = G.ncy + 1;
  auto D = [&](int i, int j, int k) { return div[((long long)k * nyn + j) * nxn + i]; };
  const double fact = 0.25;  // half**(ndim-1)
  int cell;
  unsigned fl;
  const long long o = diff_cell(G, map, cx, cy, cz, cell, fl);
  double U0[5], Ul[5], Ur[5];
  diff_load(u, o, cell, fl, U0);
  double acc[5];
  // x faces: flux(i,j,k,n,1) at the left face of cell i, corners (i, j..j+1, k..k+1)
  auto dx_face = [&](int i) {
    double d1 = M_(fact, D(i, cy, cz));
    d1 = A_(d1, M_(fact, D(i, cy + 1, cz)));
    d1 = A_(d1, M_(fact, A_(D(i, cy, cz + 1), D(i, cy + 1, cz + 1))));
    return M_(dt, M_(difmag, min0(d1)));
  };
  auto dy_face = [&](int j) {
    double d1 = 0.0;
    d1 = A_(d1, M_(fact, A_(D(cx, j, cz), D(cx + 1, j, cz))));
    d1 = A_(d1, M_(fact, A_(D(cx, j, cz + 1), D(cx + 1, j, cz + 1))));
    return M_(dt, M_(difmag, min0(d1)));
  };
  auto dz_face = [&](int k) {
    const double d1 = M_(fact, A_(A_(A_(D(cx, cy, k), D(cx + 1, cy, k)), D(cx, cy + 1, k)), D(cx + 1, cy + 1, k)));
    return M_(dt, M_(difmag, min0(d1)));
  };
  int cl, cr;
  unsigned fll, flr;
  // x
  {
    diff_load(u, diff_cell(G, map, cx - 1, cy, cz, cl, fll), cl, fll, Ul);
    diff_load(u, diff_cell(G, map, cx + 1, cy, cz, cr, flr), cr, flr, Ur);
    const double tl = dx_face(cx), tr = dx_face(cx + 1);
#pragma unroll
    for (int n = 0; n < 5; ++n) acc[n] = S_(M_(tl, S_(U0[n], Ul[n])), M_(tr, S_(Ur[n], U0[n])));
  }
  // y
  {
    diff_load(u, diff_cell(G, map, cx, cy - 1, cz, cl, fll), cl, fll, Ul);
    diff_load(u, diff_cell(G, map, cx, cy + 1, cz, cr, flr), cr, flr, Ur);
    const double tl = dy_face(cy), tr = dy_face(cy + 1);
#pragma unroll
    for (int n = 0; n < 5; ++n) acc[n] = A_(acc[n], S_(M_(tl, S_(U0[n], Ul[n])), M_(tr, S_(Ur[n], U0[n]))));
  }
  // z
  {
    diff_load(u, diff_cell(G, map, cx, cy, cz - 1, cl, fll), cl, fll, Ul);
    diff_load(u, diff_cell(G, map, cx, cy, cz + 1, cr, flr), cr, flr, Ur);
    const double tl = dz_face(cz), tr = dz_face(cz + 1);
#pragma unroll
    for (int n = 0; n < 5; ++n) acc[n] = A_(acc[n], S_(M_(tl, S_(U0[n], Ul[n])), M_(tr, S_(Ur[n], U0[n]))));
  }
  double* p = unew + o * 40 + cell;
#pragma unroll
  for (int n = 0; n < 5; ++n) p[8 * n] = A_(p[8 * n], acc[n]);
}

__global__ void scatter_level_octs_kernel(const rh_oct* __restrict__ grid, long long n, int lev, int nx, int ny,
                                          int nz, long long base, int* __restrict__ map, int* __restrict__ err) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const rh_oct o = grid[i];
  const int x = o.ckey[0], y = o.ckey[1], z = o.ckey[2];
  if (o.lev != lev || x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) {
    atomicOr(err, 1);
    return;
  }
  if (atomicCAS(&map[((long long)z * ny + y) * nx + x], -1, (int)(base + i)) != -1) atomicOr(err, 2);
}

}  // namespace

bool diffusion_supported(int l) {
  const Context& c = ctx();
  int nlev = 0;
  for (int k = c.levelmin; k <= c.levelmax; ++k) nlev += c.noct[k] > 0;
  const long long nx = (long long)c.box_nx[0] << (l - 1), ny = (long long)c.box_nx[1] << (l - 1),
                  nz = (long long)c.box_nx[2] << (l - 1);
  return c.precision == RH_PREC_FP64 && nlev == 1 && (long long)c.noct[l] == nx * ny * nz;
}

int diffuse_level(int l, double dt, double dx, double difmag, double smallr, const double* gravity) {
  Context& c = ctx();
  if (!diffusion_supported(l)) {
    set_error("difmag > 0 (cmpdivu/cmpdiff) runs on a mesh of one complete level in FP64 only");
    return RH_EINVAL;
  }
  DiffGeo G;
  G.nxo = c.box_nx[0] << (l - 1);
  G.nyo = c.box_nx[1] << (l - 1);
  G.nzo = c.box_nx[2] << (l - 1);
  G.ncx = 2 * G.nxo;
  G.ncy = 2 * G.nyo;
  G.ncz = 2 * G.nzo;
  for (int d = 0; d < 3; ++d) G.periodic[d] = c.periodic[d];
  for (int i = 0; i < 6; ++i) G.btype[i] = c.bound_type[i];
  const long long nmap = (long long)G.nxo * G.nyo * G.nzo;
  if (c.difmap_level != l || !c.d_difmap) {
    // oct coordinates -> oct index, once per mesh
    cudaFree(c.d_difmap);
    c.d_difmap = nullptr;
    c.difmap_level = -1;
    rh_oct* d_grid = nullptr;
    int* d_err = nullptr;
    const long long n = c.noct[l];
    cudaError_t e = cudaMalloc(&c.d_difmap, sizeof(int) * nmap);
    if (e == cudaSuccess) e = cudaMalloc(&d_grid, sizeof(rh_oct) * n);
    if (e == cudaSuccess) e = cudaMalloc(&d_err, sizeof(int));
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_grid, c.grid.data() + (c.head[l] - 1), sizeof(rh_oct) * n, cudaMemcpyHostToDevice,
                          c.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c.d_difmap, 0xff, sizeof(int) * nmap, c.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, sizeof(int), c.stream);
    int herr = 0;
    if (e == cudaSuccess) {
      scatter_level_octs_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c.stream>>>(
          d_grid, n, l, G.nxo, G.nyo, G.nzo, c.head[l] - 1, c.d_difmap, d_err);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, c.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
    cudaFree(d_grid);
    cudaFree(d_err);
    if (e != cudaSuccess) return cuda_fail(e, "diffusion oct map");
    if (herr) {
      set_error(herr & 1 ? "level %d: an oct key lies outside the level's box" : "level %d: duplicate oct key", l);
      return RH_EINVAL;
    }
    c.difmap_level = l;
  }
  const size_t ndiv = (size_t)(G.ncx + 1) * (G.ncy + 1) * (G.ncz + 1);
  if (c.div_elems < ndiv) {
    cudaFree(c.d_div);
    c.d_div = nullptr;
    c.div_elems = 0;
    RH_CUDA(cudaMalloc(&c.d_div, sizeof(double) * ndiv));
    c.div_elems = ndiv;
  }
  const double dtxhalf = dt * 0.5;
  const double g0 = gravity[0] * dtxhalf, g1 = gravity[1] * dtxhalf, g2 = gravity[2] * dtxhalf;
  const double fact = (0.5 * 0.5) / dx;  // half**(ndim-1)/dx
  corner_div_kernel<<<(unsigned)((ndiv + 255) / 256), 256, 0, c.stream>>>(c.ud[c.cur], c.d_difmap, G, smallr, g0,
                                                                           g1, g2, fact, c.d_div);
  RH_CUDA(cudaGetLastError());
  const long long ncell = (long long)G.ncx * G.ncy * G.ncz;
  diffuse_cells_kernel<<<(unsigned)((ncell + 255) / 256), 256, 0, c.stream>>>(c.ud[c.cur], c.ud[1 - c.cur],
                                                                              c.d_difmap, G, c.d_div, dt, difmag);
  RH_CUDA(cudaGetLastError());
  return RH_OK;
}

void free_diffusion() {
  Context& c = ctx();
  cudaFree(c.d_difmap);
  c.d_difmap = nullptr;
  c.difmap_level = -1;
  cudaFree(c.d_div);
  c.d_div = nullptr;
  c.div_elems = 0;
}

}  // namespace rh
