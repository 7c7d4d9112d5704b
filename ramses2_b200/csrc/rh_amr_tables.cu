// rh_amr_tables.cu — pencil tables and interpolated ghost octs of a
// coarse-fine level, built on the device.
//
// The reference rebuilds its neighbour and cache-oct tables on the GPU after
// every refinement (gpu/gpu_runner.cuf:3315-3440 gpu_build_level_cache,
// update_nbor_array, make_cache_octs; gpu/gpu_hash.cuf for the oct hash).
// This builder produces exactly the tables of the host builder
// (build_amr_tables, rh_amr.cu) from the level's oct records:
//
//   1. open-addressing hashes (64-bit packed coordinates, linear probing,
//      probes bounded by the capacity) of the octs of levels l and l-1;
//   2. pencils: per oct the key (XY tile, z), radix sort, unique -> occupied
//      (tile, z) layers; a run of consecutive layers of one tile starts where
//      the tile changes or z jumps, and a pencil every lz layers of a run
//      (scans give run starts, pencil ids and table offsets);
//   3. one block per pencil resolves each neighbourhood position
//      (periodic wrap / non-periodic clamp) to an oct of the level, or enters
//      it in a ghost hash keeping the first table entry that needs it;
//   4. one thread per ghost key finds the father cell and its six neighbours
//      at level l-1 (interpol_hydro's inputs); valid ghosts are numbered in
//      order of first use, the order the host builder creates them in, and
//      the table entries get gbase + id (or -1 where the coarse
//      neighbourhood is missing);
//   5. every position within one oct of an updated oct must have a source.
#include <cuda_runtime.h>

#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <vector>

#include "rh_internal.h"

namespace rh {

namespace {

constexpr unsigned long long kEmpty = ~0ull;

__host__ __device__ __forceinline__ unsigned long long key3(long long x, long long y, long long z) {
  const unsigned long long M = (1ull << 21) - 1;
  return (((unsigned long long)(x + 4) & M) << 42) | (((unsigned long long)(y + 4) & M) << 21) |
         ((unsigned long long)(z + 4) & M);
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ull;
  k ^= k >> 33;
  return k;
}

struct Hash {
  unsigned long long* keys;
  int* vals;
  unsigned long long mask;  // capacity - 1 (power of two)
};

__device__ __forceinline__ int hash_find(const Hash& h, unsigned long long key) {
  unsigned long long s = mix64(key) & h.mask;
  for (unsigned long long n = 0; n <= h.mask; ++n) {
    const unsigned long long k = h.keys[s];
    if (k == key) return h.vals[s];
    if (k == kEmpty) return -1;
    s = (s + 1) & h.mask;
  }
  return -1;
}

// Slot of key, inserting it if absent; -1 when the table is full.
__device__ __forceinline__ long long hash_slot(const Hash& h, unsigned long long key, bool* inserted) {
  unsigned long long s = mix64(key) & h.mask;
  for (unsigned long long n = 0; n <= h.mask; ++n) {
    const unsigned long long prev = atomicCAS(&h.keys[s], kEmpty, key);
    if (prev == kEmpty || prev == key) {
      *inserted = prev == kEmpty;
      return (long long)s;
    }
    s = (s + 1) & h.mask;
  }
  return -1;
}

__device__ __forceinline__ long long wrapd(long long v, long long n, int periodic) {
  if (periodic) {
    v %= n;
    return v < 0 ? v + n : v;
  }
  return v < 0 ? 0 : (v >= n ? n - 1 : v);
}

__device__ __forceinline__ long long floordiv2d(long long a) { return a >= 0 ? a / 2 : -((-a + 1) / 2); }

// error bits of the build
constexpr int kErrKey = 1, kErrDup = 2, kErrFull = 4, kErrNest = 8;

__global__ void hash_octs_kernel(const rh_oct* __restrict__ grid, int first, int n, Hash h, int* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const rh_oct o = grid[first + i];
  bool ins = false;
  const long long s = hash_slot(h, key3(o.ckey[0], o.ckey[1], o.ckey[2]), &ins);
  if (s < 0) {
    atomicOr(err, kErrFull);
    return;
  }
  if (!ins) atomicOr(err, kErrDup);
  h.vals[s] = first + i;
}

struct Geo {
  long long n[3];   // level extent in octs
  int periodic[3];
  int txo, tyo, lz, ow, oh;
  long long ntx;    // tiles along x
};

__global__ void layer_keys_kernel(const rh_oct* __restrict__ grid, int first, int n, Geo g,
                                  unsigned long long* __restrict__ keys, int* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const rh_oct o = grid[first + i];
  const long long x = o.ckey[0], y = o.ckey[1], z = o.ckey[2];
  if (x < 0 || y < 0 || z < 0 || x >= g.n[0] || y >= g.n[1] || z >= g.n[2]) {
    atomicOr(err, kErrKey);
    keys[i] = 0;
    return;
  }
  const unsigned long long tile = (unsigned long long)(y / g.tyo) * (unsigned long long)g.ntx + (x / g.txo);
  keys[i] = (tile << 21) | (unsigned long long)z;
}

// run starts: 1 where the tile changes or z jumps (layer i of the sorted,
// unique (tile, z) list); value i there, 0 elsewhere, for a max-scan
__global__ void run_start_kernel(const unsigned long long* __restrict__ lay, int nl, int* __restrict__ rs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nl) return;
  bool start = i == 0;
  if (!start) {
    const unsigned long long a = lay[i - 1], b = lay[i];
    start = (a >> 21) != (b >> 21) || (b & ((1ull << 21) - 1)) != (a & ((1ull << 21) - 1)) + 1;
  }
  rs[i] = start ? i : 0;
}

__global__ void pencil_flag_kernel(const unsigned long long* __restrict__ lay, const int* __restrict__ rstart, int nl,
                                   int lz, int* __restrict__ pf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nl) return;
  const long long z = (long long)(lay[i] & ((1ull << 21) - 1));
  const long long za = (long long)(lay[rstart[i]] & ((1ull << 21) - 1));
  pf[i] = ((z - za) % lz) == 0 ? 1 : 0;
}

__global__ void pencil_start_kernel(const int* __restrict__ pf, const int* __restrict__ pid, int nl,
                                    int* __restrict__ ps) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nl) return;
  if (pf[i]) ps[pid[i]] = i;
}

__global__ void pencil_hdr_kernel(const unsigned long long* __restrict__ lay, const int* __restrict__ ps, int np,
                                  int nl, Geo g, int4* __restrict__ hdr, long long* __restrict__ cnt) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const int a = ps[p], b = p + 1 < np ? ps[p + 1] : nl;
  const unsigned long long k = lay[a];
  const unsigned long long tile = k >> 21;
  const long long tx = (long long)(tile % (unsigned long long)g.ntx), ty = (long long)(tile / (unsigned long long)g.ntx);
  const int L = b - a;
  hdr[p] = make_int4((int)(tx * g.txo), (int)(ty * g.tyo), (int)(k & ((1ull << 21) - 1)), L);
  cnt[p] = (long long)(L + 2) * g.ow * g.oh;
}

// One block per pencil: every neighbourhood position -> oct of the level, or
// (ghost slot + 2) negated, entered in the ghost hash with its first use.
__global__ void fill_amr_tables_kernel(const int4* __restrict__ hdr, const long long* __restrict__ poff, Geo g,
                                       Hash fine, Hash ghost, unsigned long long* __restrict__ gfirst,
                                       int* __restrict__ ptab, int* err) {
  const int p = blockIdx.x;
  const int4 h = hdr[p];
  const long long base = poff[p];
  const int ns = g.ow * g.oh, ne = (h.w + 2) * ns;
  for (int e = threadIdx.x; e < ne; e += blockDim.x) {
    const int r = e / ns, rem = e - r * ns, jj = rem / g.ow, ii = rem - jj * g.ow;
    const long long x = wrapd((long long)h.x - 1 + ii, g.n[0], g.periodic[0]);
    const long long y = wrapd((long long)h.y - 1 + jj, g.n[1], g.periodic[1]);
    const long long z = wrapd((long long)h.z - 1 + r, g.n[2], g.periodic[2]);
    const unsigned long long key = key3(x, y, z);
    const int v = hash_find(fine, key);
    if (v >= 0) {
      ptab[base + e] = v;
      continue;
    }
    bool ins = false;
    const long long s = hash_slot(ghost, key, &ins);
    if (s < 0) {
      atomicOr(err, kErrFull);
      ptab[base + e] = -1;
      continue;
    }
    atomicMin(&gfirst[s], (unsigned long long)(base + e));
    ptab[base + e] = -(int)s - 2;
  }
}

// Sources of every ghost key: its father cell at level l-1 and the father's
// six neighbours (boundary-mapped as the host builder does: periodic wrap, or
// clamp with a normal-momentum flip for reflexive faces).
__global__ void occupied_kernel(const unsigned long long* __restrict__ keys, long long cap, int* __restrict__ occ) {
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s < cap) occ[s] = keys[s] != kEmpty;
}

__global__ void ghost_sources_kernel(const unsigned long long* __restrict__ gkeys, const int* __restrict__ occ_slots,
                                     int nocc, Hash coarse, Geo g, const int* __restrict__ bound_type,
                                     int* __restrict__ src, unsigned char* __restrict__ cf, int* __restrict__ valid) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nocc) return;
  const unsigned long long key = gkeys[occ_slots[i]];
  const unsigned long long M = (1ull << 21) - 1;
  const long long k[3] = {(long long)((key >> 42) & M) - 4, (long long)((key >> 21) & M) - 4,
                          (long long)(key & M) - 4};
  const int shift[7][3] = {{0, 0, 0}, {-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
  int ok = 1;
  for (int j = 0; j < 7; ++j) {
    long long q[3];
    unsigned char flip = 0;
    for (int d = 0; d < 3; ++d) {
      q[d] = k[d] + shift[j][d];
      if (q[d] < 0 || q[d] >= g.n[d]) {
        if (g.periodic[d]) {
          q[d] = wrapd(q[d], g.n[d], 1);
        } else {
          const int bt = bound_type[2 * d + (q[d] < 0 ? 0 : 1)];
          q[d] = q[d] < 0 ? 0 : g.n[d] - 1;
          if (bt == RH_BOUND_REFLEXIVE) flip |= (unsigned char)(1u << d);
        }
      }
    }
    const long long oc[3] = {floordiv2d(q[0]), floordiv2d(q[1]), floordiv2d(q[2])};
    const int o = hash_find(coarse, key3(oc[0], oc[1], oc[2]));
    if (o < 0) {
      ok = 0;
      break;
    }
    src[(long long)i * 7 + j] = o;
    cf[(long long)i * 7 + j] = (unsigned char)(((q[0] - 2 * oc[0]) + 2 * (q[1] - 2 * oc[1]) + 4 * (q[2] - 2 * oc[2])) | (flip << 3));
  }
  valid[i] = ok;
}

__global__ void ghost_first_kernel(const int* __restrict__ vidx, int nv, const int* __restrict__ occ_slots,
                                   const unsigned long long* __restrict__ gfirst, unsigned long long* __restrict__ first) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nv) first[k] = gfirst[occ_slots[vidx[k]]];
}

// Ghost id = rank of its first use; sources gathered in id order.
__global__ void ghost_number_kernel(const int* __restrict__ sorted_vidx, int nv, const int* __restrict__ occ_slots,
                                    const int* __restrict__ src, const unsigned char* __restrict__ cf,
                                    int* __restrict__ id_of_slot, int* __restrict__ gsrc, unsigned char* __restrict__ gcf,
                                    int2* __restrict__ gfather) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= nv) return;
  const int i = sorted_vidx[id];
  id_of_slot[occ_slots[i]] = id;
  for (int j = 0; j < 7; ++j) {
    gsrc[(long long)id * 7 + j] = src[(long long)i * 7 + j];
    gcf[(long long)id * 7 + j] = cf[(long long)i * 7 + j];
  }
  gfather[id] = make_int2(src[(long long)i * 7], cf[(long long)i * 7] & 7);
}

__global__ void finish_tables_kernel(int* __restrict__ ptab, long long ntab, const int* __restrict__ id_of_slot,
                                     long long gbase) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= ntab) return;
  const int v = ptab[e];
  if (v >= -1) return;
  const int id = id_of_slot[-v - 2];
  ptab[e] = id >= 0 ? (int)(gbase + id) : -1;
}

// Positions within one oct of an updated oct must resolve (the cell stencils
// and ring-cell slopes read them).  First failure recorded in bad[0..2].
__global__ void check_nesting_kernel(const int4* __restrict__ hdr, const long long* __restrict__ poff, Geo g,
                                     const int* __restrict__ ptab, int ngridmax, int* err, int* bad) {
  const int p = blockIdx.x;
  const int4 h = hdr[p];
  const int* tab = ptab + poff[p];
  const int ni = g.ow - 2, nj = g.oh - 2, n = h.w * nj * ni;
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const int r = 1 + t / (nj * ni), rem = t % (nj * ni), jj = 1 + rem / ni, ii = 1 + rem % ni;
    const int v = tab[((long long)r * g.oh + jj) * g.ow + ii];
    if (v < 0 || v >= ngridmax) continue;
    for (int dr = -1; dr <= 1; ++dr)
      for (int dj = -1; dj <= 1; ++dj)
        for (int di = -1; di <= 1; ++di)
          if (tab[((long long)(r + dr) * g.oh + jj + dj) * g.ow + ii + di] < 0) {
            if (atomicOr(err, kErrNest) & kErrNest) return;
            bad[0] = h.x - 1 + ii + di;
            bad[1] = h.y - 1 + jj + dj;
            bad[2] = h.z - 1 + r + dr;
            return;
          }
  }
}

unsigned long long pow2_at_least(unsigned long long n) {
  unsigned long long c = 1024;
  while (c < n) c <<= 1;
  return c;
}

unsigned nblk(long long n, int t) { return (unsigned)std::max(1LL, (n + t - 1) / t); }

// Device buffers of one build, released on every exit path.
struct Scratch {
  std::vector<void*> ptrs;
  template <typename T> cudaError_t alloc(T** p, size_t count) {
    *p = nullptr;
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(1, count));
    if (e == cudaSuccess) ptrs.push_back((void*)*p);
    return e;
  }
  ~Scratch() {
    for (void* p : ptrs) cudaFree(p);
  }
};

#define RH_TRY(call, what)                                 \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return cuda_fail(e_, what);     \
  } while (0)

}  // namespace

int build_amr_tables_device(int l, const TileCfg& cfg, long long gbase, const rh_oct* d_grid, int2** d_gfather_out) {
  Context& c = ctx();
  LevelTables& T = c.levels[l];
  cudaStream_t st = c.stream;
  T.cfg = cfg;
  Geo g;
  for (int d = 0; d < 3; ++d) {
    g.n[d] = (long long)c.box_nx[d] << (l - 1);
    g.periodic[d] = c.periodic[d];
  }
  T.nxo = (int)g.n[0];
  T.nyo = (int)g.n[1];
  T.nzo = (int)g.n[2];
  g.txo = cfg.txo;
  g.tyo = cfg.tyo;
  g.lz = cfg.lz;
  g.ow = cfg.txo + 2;
  g.oh = cfg.tyo + 2;
  g.ntx = (g.n[0] + cfg.txo - 1) / cfg.txo;
  if (l - 1 < c.levelmin || c.noct[l - 1] == 0) {
    set_error("level %d does not fill its box and has no coarser level to interpolate from", l);
    return RH_EINVAL;
  }
  const long long nty = (g.n[1] + cfg.tyo - 1) / cfg.tyo;
  if (g.n[2] >= (1LL << 21) || (double)g.ntx * (double)nty >= (double)(1ULL << 42)) {
    set_error("level %d: box of %lld^3 octs too large for the device table builder", l, g.n[0]);
    return RH_EINVAL;
  }
  const int nf = c.noct[l], nc = c.noct[l - 1];
  const int ff = c.head[l] - 1, fc = c.head[l - 1] - 1;
  Scratch S;
  int* d_err = nullptr;
  int* d_bad = nullptr;
  int* d_bt = nullptr;
  RH_TRY(S.alloc(&d_err, 1), "amr tables (alloc)");
  RH_TRY(S.alloc(&d_bad, 3), "amr tables (alloc)");
  RH_TRY(S.alloc(&d_bt, 6), "amr tables (alloc)");
  RH_TRY(cudaMemsetAsync(d_err, 0, sizeof(int), st), "amr tables (memset)");
  RH_TRY(cudaMemcpyAsync(d_bt, c.bound_type, sizeof(int) * 6, cudaMemcpyHostToDevice, st), "amr tables (copy)");
  // 1. hashes of levels l and l-1
  Hash hf, hc;
  hf.mask = pow2_at_least(2ull * nf) - 1;
  hc.mask = pow2_at_least(2ull * nc) - 1;
  RH_TRY(S.alloc(&hf.keys, hf.mask + 1), "amr tables (alloc)");
  RH_TRY(S.alloc(&hf.vals, hf.mask + 1), "amr tables (alloc)");
  RH_TRY(S.alloc(&hc.keys, hc.mask + 1), "amr tables (alloc)");
  RH_TRY(S.alloc(&hc.vals, hc.mask + 1), "amr tables (alloc)");
  RH_TRY(cudaMemsetAsync(hf.keys, 0xff, sizeof(unsigned long long) * (hf.mask + 1), st), "amr tables (memset)");
  RH_TRY(cudaMemsetAsync(hc.keys, 0xff, sizeof(unsigned long long) * (hc.mask + 1), st), "amr tables (memset)");
  hash_octs_kernel<<<nblk(nf, 256), 256, 0, st>>>(d_grid, ff, nf, hf, d_err);
  hash_octs_kernel<<<nblk(nc, 256), 256, 0, st>>>(d_grid, fc, nc, hc, d_err);
  RH_TRY(cudaGetLastError(), "amr tables (hash)");
  // 2. pencils
  unsigned long long *d_keys = nullptr, *d_sorted = nullptr, *d_lay = nullptr;
  int* d_nl = nullptr;
  RH_TRY(S.alloc(&d_keys, nf), "amr tables (alloc)");
  RH_TRY(S.alloc(&d_sorted, nf), "amr tables (alloc)");
  RH_TRY(S.alloc(&d_lay, nf), "amr tables (alloc)");
  RH_TRY(S.alloc(&d_nl, 1), "amr tables (alloc)");
  layer_keys_kernel<<<nblk(nf, 256), 256, 0, st>>>(d_grid, ff, nf, g, d_keys, d_err);
  RH_TRY(cudaGetLastError(), "amr tables (keys)");
  int end_bit = 21;
  while (end_bit < 64 && ((unsigned long long)(g.ntx * nty) >> (end_bit - 21)) != 0) ++end_bit;
  {
    size_t tb = 0;
    void* tmp = nullptr;
    RH_TRY(cub::DeviceRadixSort::SortKeys(nullptr, tb, d_keys, d_sorted, nf, 0, end_bit, st), "amr tables (sort)");
    RH_TRY(S.alloc((char**)&tmp, tb), "amr tables (alloc)");
    RH_TRY(cub::DeviceRadixSort::SortKeys(tmp, tb, d_keys, d_sorted, nf, 0, end_bit, st), "amr tables (sort)");
    tb = 0;
    RH_TRY(cub::DeviceSelect::Unique(nullptr, tb, d_sorted, d_lay, d_nl, nf, st), "amr tables (unique)");
    void* tmp2 = nullptr;
    RH_TRY(S.alloc((char**)&tmp2, tb), "amr tables (alloc)");
    RH_TRY(cub::DeviceSelect::Unique(tmp2, tb, d_sorted, d_lay, d_nl, nf, st), "amr tables (unique)");
  }
  int herr = 0, nl = 0;
  RH_TRY(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st), "amr tables (copy)");
  RH_TRY(cudaMemcpyAsync(&nl, d_nl, sizeof(int), cudaMemcpyDeviceToHost, st), "amr tables (copy)");
  RH_TRY(cudaStreamSynchronize(st), "amr tables (sync)");
  if (herr) {
    set_error(herr & kErrKey ? "level %d: an oct key lies outside the level's box"
                             : (herr & kErrDup ? "level %d: duplicate oct key" : "level %d: oct hash full"), l);
    return RH_EINVAL;
  }
  int *d_rs = nullptr, *d_rstart = nullptr, *d_pf = nullptr, *d_pid = nullptr;
  RH_TRY(S.alloc(&d_rs, nl), "amr tables (alloc)");
  RH_TRY(S.alloc(&d_rstart, nl), "amr tables (alloc)");
  RH_TRY(S.alloc(&d_pf, nl), "amr tables (alloc)");
  RH_TRY(S.alloc(&d_pid, nl), "amr tables (alloc)");
  run_start_kernel<<<nblk(nl, 256), 256, 0, st>>>(d_lay, nl, d_rs);
  {
    size_t tb = 0;
    void* tmp = nullptr;
    RH_TRY(cub::DeviceScan::InclusiveScan(nullptr, tb, d_rs, d_rstart, cub::Max(), nl, st), "amr tables (scan)");
    RH_TRY(S.alloc((char**)&tmp, tb), "amr tables (alloc)");
    RH_TRY(cub::DeviceScan::InclusiveScan(tmp, tb, d_rs, d_rstart, cub::Max(), nl, st), "amr tables (scan)");
  }
  pencil_flag_kernel<<<nblk(nl, 256), 256, 0, st>>>(d_lay, d_rstart, nl, cfg.lz, d_pf);
  {
    size_t tb = 0;
    void* tmp = nullptr;
    RH_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, d_pf, d_pid, nl, st), "amr tables (scan)");
    RH_TRY(S.alloc((char**)&tmp, tb), "amr tables (alloc)");
    RH_TRY(cub::DeviceScan::ExclusiveSum(tmp, tb, d_pf, d_pid, nl, st), "amr tables (scan)");
  }
  int last_pid = 0, last_pf = 0;
  RH_TRY(cudaMemcpyAsync(&last_pid, d_pid + nl - 1, sizeof(int), cudaMemcpyDeviceToHost, st), "amr tables (copy)");
  RH_TRY(cudaMemcpyAsync(&last_pf, d_pf + nl - 1, sizeof(int), cudaMemcpyDeviceToHost, st), "amr tables (copy)");
  RH_TRY(cudaStreamSynchronize(st), "amr tables (sync)");
  const int np = last_pid + last_pf;
  int* d_ps = nullptr;
  long long* d_cnt = nullptr;
  RH_TRY(S.alloc(&d_ps, np), "amr tables (alloc)");
  RH_TRY(S.alloc(&d_cnt, np), "amr tables (alloc)");
  RH_TRY(cudaMalloc(&T.d_phdr, sizeof(int4) * std::max(1, np)), "amr tables (alloc)");
  RH_TRY(cudaMalloc(&T.d_poff, sizeof(long long) * std::max(1, np)), "amr tables (alloc)");
  RH_TRY(cudaMalloc(&T.d_cfl_partial, sizeof(double) * 5 * std::max(1, np)), "amr tables (alloc)");
  pencil_start_kernel<<<nblk(nl, 256), 256, 0, st>>>(d_pf, d_pid, nl, d_ps);
  pencil_hdr_kernel<<<nblk(np, 256), 256, 0, st>>>(d_lay, d_ps, np, nl, g, T.d_phdr, d_cnt);
  {
    size_t tb = 0;
    void* tmp = nullptr;
    RH_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, d_cnt, T.d_poff, np, st), "amr tables (scan)");
    RH_TRY(S.alloc((char**)&tmp, tb), "amr tables (alloc)");
    RH_TRY(cub::DeviceScan::ExclusiveSum(tmp, tb, d_cnt, T.d_poff, np, st), "amr tables (scan)");
  }
  RH_TRY(cudaGetLastError(), "amr tables (pencils)");
  T.phdr.resize((size_t)np);
  T.poff.resize((size_t)np);
  RH_TRY(cudaMemcpyAsync(T.phdr.data(), T.d_phdr, sizeof(int4) * np, cudaMemcpyDeviceToHost, st), "amr tables (copy)");
  RH_TRY(cudaMemcpyAsync(T.poff.data(), T.d_poff, sizeof(long long) * np, cudaMemcpyDeviceToHost, st),
         "amr tables (copy)");
  RH_TRY(cudaStreamSynchronize(st), "amr tables (sync)");
  const long long ntab = T.poff.back() + (long long)(T.phdr.back().w + 2) * g.ow * g.oh;
  // 3. tables with provisional ghost slots
  Hash hg;
  hg.mask = pow2_at_least(2ull * (unsigned long long)ntab) - 1;  // at most one key per table entry
  if (hg.mask >= (unsigned long long)INT32_MAX) {
    set_error("level %d: %lld table entries exceed the device table builder's range", l, ntab);
    return RH_EINVAL;
  }
  unsigned long long* d_gfirst = nullptr;
  RH_TRY(S.alloc(&hg.keys, hg.mask + 1), "amr tables (alloc)");
  hg.vals = nullptr;
  RH_TRY(S.alloc(&d_gfirst, hg.mask + 1), "amr tables (alloc)");
  RH_TRY(cudaMemsetAsync(hg.keys, 0xff, sizeof(unsigned long long) * (hg.mask + 1), st), "amr tables (memset)");
  RH_TRY(cudaMemsetAsync(d_gfirst, 0xff, sizeof(unsigned long long) * (hg.mask + 1), st), "amr tables (memset)");
  RH_TRY(cudaMalloc(&T.d_ptab, sizeof(int) * std::max(1LL, ntab)), "amr tables (alloc)");
  fill_amr_tables_kernel<<<np, 128, 0, st>>>(T.d_phdr, T.d_poff, g, hf, hg, d_gfirst, T.d_ptab, d_err);
  RH_TRY(cudaGetLastError(), "amr tables (fill)");
  // 4. ghost sources, numbering in order of first use
  const long long gcap = (long long)hg.mask + 1;
  int *d_occ = nullptr, *d_occ_slots = nullptr, *d_nocc = nullptr, *d_id = nullptr;
  RH_TRY(S.alloc(&d_occ, gcap), "amr tables (alloc)");
  RH_TRY(S.alloc(&d_occ_slots, gcap), "amr tables (alloc)");
  RH_TRY(S.alloc(&d_nocc, 1), "amr tables (alloc)");
  RH_TRY(S.alloc(&d_id, gcap), "amr tables (alloc)");
  RH_TRY(cudaMemsetAsync(d_id, 0xff, sizeof(int) * gcap, st), "amr tables (memset)");
  occupied_kernel<<<nblk(gcap, 256), 256, 0, st>>>(hg.keys, gcap, d_occ);
  {
    size_t tb = 0;
    void* tmp = nullptr;
    thrust::counting_iterator<int> it(0);
    RH_TRY(cub::DeviceSelect::Flagged(nullptr, tb, it, d_occ, d_occ_slots, d_nocc, (int)gcap, st),
           "amr tables (select)");
    RH_TRY(S.alloc((char**)&tmp, tb), "amr tables (alloc)");
    RH_TRY(cub::DeviceSelect::Flagged(tmp, tb, it, d_occ, d_occ_slots, d_nocc, (int)gcap, st), "amr tables (select)");
  }
  int nocc = 0;
  RH_TRY(cudaMemcpyAsync(&nocc, d_nocc, sizeof(int), cudaMemcpyDeviceToHost, st), "amr tables (copy)");
  RH_TRY(cudaStreamSynchronize(st), "amr tables (sync)");
  int *d_src = nullptr, *d_valid = nullptr, *d_vidx = nullptr, *d_sorted_vidx = nullptr, *d_nv = nullptr;
  unsigned char* d_cf = nullptr;
  RH_TRY(S.alloc(&d_src, 7 * (size_t)nocc), "amr tables (alloc)");
  RH_TRY(S.alloc(&d_cf, 7 * (size_t)nocc), "amr tables (alloc)");
  RH_TRY(S.alloc(&d_valid, nocc), "amr tables (alloc)");
  RH_TRY(S.alloc(&d_vidx, nocc), "amr tables (alloc)");
  RH_TRY(S.alloc(&d_nv, 1), "amr tables (alloc)");
  int nv = 0;
  if (nocc > 0) {
    ghost_sources_kernel<<<nblk(nocc, 256), 256, 0, st>>>(hg.keys, d_occ_slots, nocc, hc, g, d_bt, d_src, d_cf,
                                                         d_valid);
    size_t tb = 0;
    void* tmp = nullptr;
    thrust::counting_iterator<int> it(0);
    RH_TRY(cub::DeviceSelect::Flagged(nullptr, tb, it, d_valid, d_vidx, d_nv, nocc, st), "amr tables (select)");
    RH_TRY(S.alloc((char**)&tmp, tb), "amr tables (alloc)");
    RH_TRY(cub::DeviceSelect::Flagged(tmp, tb, it, d_valid, d_vidx, d_nv, nocc, st), "amr tables (select)");
    RH_TRY(cudaMemcpyAsync(&nv, d_nv, sizeof(int), cudaMemcpyDeviceToHost, st), "amr tables (copy)");
    RH_TRY(cudaStreamSynchronize(st), "amr tables (sync)");
  }
  if (nv > 0) {
    unsigned long long *d_first = nullptr, *d_first_sorted = nullptr;
    RH_TRY(S.alloc(&d_first, nv), "amr tables (alloc)");
    RH_TRY(S.alloc(&d_first_sorted, nv), "amr tables (alloc)");
    RH_TRY(S.alloc(&d_sorted_vidx, nv), "amr tables (alloc)");
    ghost_first_kernel<<<nblk(nv, 256), 256, 0, st>>>(d_vidx, nv, d_occ_slots, d_gfirst, d_first);
    size_t tb = 0;
    void* tmp = nullptr;
    RH_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, d_first, d_first_sorted, d_vidx, d_sorted_vidx, nv, 0, 64,
                                           st), "amr tables (sort)");
    RH_TRY(S.alloc((char**)&tmp, tb), "amr tables (alloc)");
    RH_TRY(cub::DeviceRadixSort::SortPairs(tmp, tb, d_first, d_first_sorted, d_vidx, d_sorted_vidx, nv, 0, 64, st),
           "amr tables (sort)");
    RH_TRY(cudaMalloc(&T.d_gsrc_oct, sizeof(int) * 7 * (size_t)nv), "amr tables (alloc)");
    RH_TRY(cudaMalloc(&T.d_gsrc_cf, 7 * (size_t)nv), "amr tables (alloc)");
    RH_TRY(cudaMalloc(d_gfather_out, sizeof(int2) * (size_t)nv), "amr tables (alloc)");
    ghost_number_kernel<<<nblk(nv, 256), 256, 0, st>>>(d_sorted_vidx, nv, d_occ_slots, d_src, d_cf, d_id,
                                                      T.d_gsrc_oct, T.d_gsrc_cf, *d_gfather_out);
  }
  finish_tables_kernel<<<nblk(ntab, 256), 256, 0, st>>>(T.d_ptab, ntab, d_id, gbase);
  // 5. nesting check
  check_nesting_kernel<<<np, 128, 0, st>>>(T.d_phdr, T.d_poff, g, T.d_ptab, c.ngridmax, d_err, d_bad);
  RH_TRY(cudaGetLastError(), "amr tables (ghosts)");
  int bad[3] = {0, 0, 0};
  RH_TRY(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st), "amr tables (copy)");
  RH_TRY(cudaMemcpyAsync(bad, d_bad, sizeof(bad), cudaMemcpyDeviceToHost, st), "amr tables (copy)");
  RH_TRY(cudaStreamSynchronize(st), "amr tables (sync)");
  if (herr & kErrFull) {
    set_error("level %d: ghost hash full", l);
    return RH_EINVAL;
  }
  if (herr & kErrNest) {
    set_error("level %d: the coarse neighbourhood of a missing oct next to (%d,%d,%d) does not exist (mesh not "
              "properly nested)", l, bad[0], bad[1], bad[2]);
    return RH_EINVAL;
  }
  T.gbase = gbase;
  T.nghost = nv;
  T.npencil = np;
  T.ntab = ntab;
  T.complete = false;
  T.ptab.clear();
  T.built = true;
  return RH_OK;
}

}  // namespace rh
