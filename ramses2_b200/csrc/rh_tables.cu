// rh_tables.cu — pencil oct tables of a complete (uniform) level, built on the
// device.
//
// The reference builds its neighbour tables on the GPU from the oct records
// and a device hash (gpu/gpu_refine.cuf:2006-2083 nbor, gpu/gpu_hash.cuf).  A
// complete level fills its box, so a dense map from oct coordinates to oct
// index replaces the hash: the level's oct records are copied to the device as
// they are (32-byte rh_oct), one thread per oct scatters its index into the
// map (duplicates and out-of-box keys are reported), and one thread per table
// entry resolves its coordinate (periodic wrap / non-periodic clamp, as the
// boundary ghost octs of amr/boundaries.f90:150-216 take their cells from the
// adjacent interior oct) to an oct index.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "rh_internal.h"

namespace rh {

namespace {

struct TabGeo {
  long long nx, ny, nz;   // level extent in octs
  int px, py, pz;         // periodic flags
  int txo, tyo, lz;       // tile
  int ow, ns;             // oct columns per row, per layer of a pencil
  long long tx, ty;       // pencils per x, y
  long long nfull;        // pencils of full depth (all z slabs but the last)
  long long sfull, slast; // table entries of a full / last-slab pencil
  int llast;              // layers of a last-slab pencil
};

__device__ __forceinline__ long long wrapc(long long v, long long n, int periodic) {
  if (periodic) {
    v %= n;
    return v < 0 ? v + n : v;
  }
  return v < 0 ? 0 : (v >= n ? n - 1 : v);
}

__global__ void scatter_octs_kernel(const rh_oct* __restrict__ grid, long long n, int lev, long long nx, long long ny,
                                    long long nz, int base, int* __restrict__ map, int* __restrict__ err) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const rh_oct o = grid[i];
  const long long x = o.ckey[0], y = o.ckey[1], z = o.ckey[2];
  if (o.lev != lev || x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) {
    atomicOr(err, 1);
    return;
  }
  if (atomicCAS(&map[(z * ny + y) * nx + x], -1, base + (int)i) != -1) atomicOr(err, 2);
}

__global__ void fill_tables_kernel(int* __restrict__ ptab, long long total, TabGeo g, const int* __restrict__ map) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= total) return;
  long long p, off;
  if (e < g.nfull * g.sfull) {
    p = e / g.sfull;
    off = e - p * g.sfull;
  } else {
    const long long q = (e - g.nfull * g.sfull) / g.slast;
    p = g.nfull + q;
    off = e - g.nfull * g.sfull - q * g.slast;
  }
  const long long bx = p % g.tx, by = (p / g.tx) % g.ty, bz = p / (g.tx * g.ty);
  const int r = (int)(off / g.ns);
  const int rem = (int)(off - (long long)r * g.ns);
  const int j = rem / g.ow, i = rem - j * g.ow;
  const long long z = wrapc(bz * g.lz - 1 + r, g.nz, g.pz);
  const long long y = wrapc(by * g.tyo - 1 + j, g.ny, g.py);
  const long long x = wrapc(bx * g.txo - 1 + i, g.nx, g.px);
  ptab[e] = map[(z * g.ny + y) * g.nx + x];
}

}  // namespace

// Pencil tables of a complete level l for tile cfg, built on the device
// (phdr / poff computed on the host: one entry per pencil).
int build_complete_tables_device(int l, const TileCfg& cfg, LevelTables& T) {
  Context& c = ctx();
  const long long nx = (long long)c.box_nx[0] << (l - 1), ny = (long long)c.box_nx[1] << (l - 1),
                  nz = (long long)c.box_nx[2] << (l - 1);
  T.nxo = (int)nx;
  T.nyo = (int)ny;
  T.nzo = (int)nz;
  if ((long long)c.noct[l] != nx * ny * nz) {
    set_error("level %d has %d octs, its box holds %lld: coarse-fine levels need the AMR table builder", l,
              c.noct[l], nx * ny * nz);
    return RH_EINVAL;
  }
  TabGeo g;
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  g.px = c.periodic[0];
  g.py = c.periodic[1];
  g.pz = c.periodic[2];
  g.txo = cfg.txo;
  g.tyo = cfg.tyo;
  g.lz = cfg.lz;
  g.ow = cfg.txo + 2;
  g.ns = (cfg.txo + 2) * (cfg.tyo + 2);
  g.tx = (nx + cfg.txo - 1) / cfg.txo;
  g.ty = (ny + cfg.tyo - 1) / cfg.tyo;
  const long long tz = (nz + cfg.lz - 1) / cfg.lz;
  g.llast = (int)(nz - (tz - 1) * cfg.lz);
  g.nfull = (tz - 1) * g.tx * g.ty;
  g.sfull = (long long)(cfg.lz + 2) * g.ns;
  g.slast = (long long)(g.llast + 2) * g.ns;
  const long long npencil = tz * g.tx * g.ty;
  const long long total = g.nfull * g.sfull + (npencil - g.nfull) * g.slast;
  // pencil headers and table offsets (same order as the table: bz, by, bx)
  T.phdr.resize((size_t)npencil);
  T.poff.resize((size_t)npencil);
  for (long long p = 0; p < npencil; ++p) {
    const long long bx = p % g.tx, by = (p / g.tx) % g.ty, bz = p / (g.tx * g.ty);
    const int L = bz < tz - 1 ? cfg.lz : g.llast;
    T.phdr[(size_t)p] = make_int4((int)(bx * cfg.txo), (int)(by * cfg.tyo), (int)(bz * cfg.lz), L);
    T.poff[(size_t)p] = p < g.nfull ? p * g.sfull : g.nfull * g.sfull + (p - g.nfull) * g.slast;
  }
  T.ptab.clear();  // the table lives on the device only
  T.ntab = total;
  // oct records of the level -> dense coordinate map
  rh_oct* d_grid = nullptr;
  int* d_map = nullptr;
  int* d_err = nullptr;
  auto cleanup = [&]() {
    cudaFree(d_grid);
    cudaFree(d_map);
    cudaFree(d_err);
  };
  const long long n = c.noct[l];
  cudaError_t e = cudaMalloc(&d_grid, sizeof(rh_oct) * n);
  if (e == cudaSuccess) e = cudaMalloc(&d_map, sizeof(int) * nx * ny * nz);
  if (e == cudaSuccess) e = cudaMalloc(&d_err, sizeof(int));
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_grid, c.grid.data() + (c.head[l] - 1), sizeof(rh_oct) * n, cudaMemcpyHostToDevice,
                        c.stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_map, 0xff, sizeof(int) * nx * ny * nz, c.stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, sizeof(int), c.stream);
  if (e != cudaSuccess) {
    cleanup();
    return cuda_fail(e, "device table build (alloc)");
  }
  scatter_octs_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c.stream>>>(d_grid, n, l, nx, ny, nz, c.head[l] - 1,
                                                                       d_map, d_err);
  int herr = 0;
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, c.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
  if (e != cudaSuccess) {
    cleanup();
    return cuda_fail(e, "device table build (scatter)");
  }
  if (herr) {
    cleanup();
    set_error(herr & 1 ? "level %d: an oct key lies outside the level's box" : "level %d: duplicate oct key", l);
    return RH_EINVAL;
  }
  e = cudaMalloc(&T.d_ptab, sizeof(int) * std::max<long long>(1, total));
  if (e == cudaSuccess)
    fill_tables_kernel<<<(unsigned)((total + 255) / 256), 256, 0, c.stream>>>(T.d_ptab, total, g, d_map);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
  cleanup();
  if (e != cudaSuccess) return cuda_fail(e, "device table build (fill)");
  return RH_OK;
}

}  // namespace rh
