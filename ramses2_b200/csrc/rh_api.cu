// rh_api.cu — the C ABI of include/ramses_hydro.h: device state, pencil-table
// builder, the four hydro leaf calls and their auxiliary kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "ramses_hydro_batch.h"
#include "rh_internal.h"
#include "rh_launch.h"

namespace rh {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;
void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
}
int cuda_fail(cudaError_t e, const char* what) {
  set_error("%s: %s", what, cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? RH_ENOMEM : RH_ECUDA;
}

Context& ctx() {
  static Context c;
  return c;
}

// ---------------------------------------------------------------------------
// kernel registry
// ---------------------------------------------------------------------------
struct RegEntry {
  KernelKey k;
  LaunchFn fn;
  size_t smem;
  int threads;
};
static std::vector<RegEntry>& registry() {
  static std::vector<RegEntry> r;
  return r;
}
void register_launcher(const KernelKey& k, LaunchFn fn, size_t smem, int threads) {
  registry().push_back({k, fn, smem, threads});
}
LaunchFn find_launcher(int prec, int txo, int tyo, int minb, int slope, int riemann, int amr, size_t* smem,
                       int* threads) {
  for (auto& e : registry())
    if (e.k.prec == prec && e.k.txo == txo && e.k.tyo == tyo && e.k.minb == minb && e.k.slope == slope &&
        e.k.riemann == riemann && e.k.amr == amr) {
      if (smem) *smem = e.smem;
      if (threads) *threads = e.threads;
      return e.fn;
    }
  return nullptr;
}
int list_tiles(int prec, int amr, int* txo, int* tyo, int* minb, int max) {
  int n = 0;
  for (auto& e : registry()) {
    if (e.k.prec != prec || e.k.slope != 2 || e.k.riemann != 3 || e.k.amr != amr) continue;
    if (n < max) {
      txo[n] = e.k.txo;
      tyo[n] = e.k.tyo;
      minb[n] = e.k.minb;
    }
    ++n;
  }
  return n;
}

// ---------------------------------------------------------------------------
// auxiliary kernels
// ---------------------------------------------------------------------------
// FP32-bulk packing: [oct][5][8] double -> the 192-byte records of rh_bulk.h
// (one thread per cell: its 5 values)
__global__ void pack_bulk_kernel(const double* __restrict__ src, float* __restrict__ uf, double* __restrict__ ue,
                                 long long noct) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= noct * 8) return;
  const long long oct = i >> 3;
  const int cell = (int)(i & 7);
  const double* s = src + oct * 40 + cell;
#pragma unroll
  for (int v = 0; v < 4; ++v) uf[oct * kBulkF + v * 8 + cell] = (float)s[8 * v];
  ue[oct * kBulkD + cell] = s[32];
}
__global__ void unpack_bulk_kernel(double* __restrict__ dst, const float* __restrict__ uf,
                                   const double* __restrict__ ue, long long noct) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= noct * 8) return;
  const long long oct = i >> 3;
  const int cell = (int)(i & 7);
  double* d = dst + oct * 40 + cell;
#pragma unroll
  for (int v = 0; v < 4; ++v) d[8 * v] = (double)uf[oct * kBulkF + v * 8 + cell];
  d[32] = ue[oct * kBulkD + cell];
}

// FP64 staging of FP32-bulk uploads / downloads, kept between calls (a host
// that hands its uold over every step does not pay an allocation each time).
int stage64(long long noct, double** out) {
  Context& c = ctx();
  const size_t need = sizeof(double) * 40 * (size_t)noct;
  if (c.stage64_bytes < need) {
    RH_CUDA(cudaStreamSynchronize(c.stream));
    cudaFree(c.d_stage64);
    c.d_stage64 = nullptr;
    c.stage64_bytes = 0;
    RH_CUDA(cudaMalloc(&c.d_stage64, need));
    c.stage64_bytes = need;
  }
  *out = c.d_stage64;
  return RH_OK;
}
template <typename E> __global__ void copy_kernel(E* __restrict__ dst, const E* __restrict__ src, long long n) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long stride = (long long)gridDim.x * blockDim.x;
  for (; i < n; i += stride) dst[i] = src[i];
}

// courant_fine over the leaf cells of [oct0, oct0+noct) of uold:
// per-block partial (mass, ekin, eint, emag, dt).  hydro/courant_fine.f90:57-168
__global__ void cmpdt_kernel(const double* __restrict__ ud, const float* __restrict__ uf, int fp32,
                             const uint8_t* __restrict__ refined, long long oct0, long long noct, CflConst C,
                             double vol, double* __restrict__ partial, const uint8_t* __restrict__ refbits) {
  __shared__ double red[32][4];
  long long cell_id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double m = 0, ek = 0, ei = 0, dt = 1e300;
  if (cell_id < noct * 8) {
    long long oct = oct0 + cell_id / 8;
    int cell = (int)(cell_id % 8);
    const bool ref = refined ? refined[cell_id] != 0 : (refbits ? ((refbits[oct] >> cell) & 1) != 0 : false);
    if (!ref && !fp32) {
      const double* o = ud + oct * 40 + cell;
      const double r = o[0], m1 = o[8], m2 = o[16], m3 = o[24], E = o[32];
      m = r * vol;
      ek = E * vol;
      const double rm = r > C.smallr ? r : C.smallr;
      ei = E * vol;
      ei -= 0.5 * (m1 * m1) / rm * vol;
      ei -= 0.5 * (m2 * m2) / rm * vol;
      ei -= 0.5 * (m3 * m3) / rm * vol;
      dt = cmpdt_cell(r, m1, m2, m3, E, C);
    } else if (!ref) {
      // an FP32-bulk cell in the fused epilogue's FP32-bulk form, so that a
      // level's values do not depend on which of the two computed them
      const float* o = uf + oct * kBulkF + cell;
      CflAcc a;
      a.add_bulk(o[0], o[8], o[16], o[24], ud[oct * kBulkD + cell], C);
      a.scale_bulk(vol);
      m = a.mass;
      ek = a.ekin;
      ei = a.eint;
      dt = a.dt(C);
    }
  }
  for (int off = 16; off > 0; off >>= 1) {
    m += __shfl_down_sync(0xffffffffu, m, off);
    ek += __shfl_down_sync(0xffffffffu, ek, off);
    ei += __shfl_down_sync(0xffffffffu, ei, off);
    double o = __shfl_down_sync(0xffffffffu, dt, off);
    dt = o < dt ? o : dt;
  }
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { red[w][0] = m; red[w][1] = ek; red[w][2] = ei; red[w][3] = dt; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0, c = 0, d = 1e300;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
      a += red[i][0]; b += red[i][1]; c += red[i][2];
      d = red[i][3] < d ? red[i][3] : d;
    }
    double* o = partial + blockIdx.x * 5ll;
    o[0] = a; o[1] = b; o[2] = c; o[3] = 0.0; o[4] = d;
  }
}

// Deterministic reduction of n partials (fixed order, one block).
__global__ void reduce_partials_kernel(const double* __restrict__ partial, long long n, double dt0,
                                       double* __restrict__ out) {
  __shared__ double red[1024][4];
  double a = 0, b = 0, c = 0, d = 1e300;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) {
    a += partial[i * 5 + 0]; b += partial[i * 5 + 1]; c += partial[i * 5 + 2];
    d = partial[i * 5 + 4] < d ? partial[i * 5 + 4] : d;
  }
  red[threadIdx.x][0] = a; red[threadIdx.x][1] = b; red[threadIdx.x][2] = c; red[threadIdx.x][3] = d;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      red[threadIdx.x][0] += red[threadIdx.x + s][0];
      red[threadIdx.x][1] += red[threadIdx.x + s][1];
      red[threadIdx.x][2] += red[threadIdx.x + s][2];
      double o = red[threadIdx.x + s][3];
      red[threadIdx.x][3] = o < red[threadIdx.x][3] ? o : red[threadIdx.x][3];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = red[0][0]; out[1] = red[0][1]; out[2] = red[0][2]; out[3] = 0.0;
    out[4] = red[0][3] < dt0 ? red[0][3] : dt0;
  }
}

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
static int check_ready(bool need_mesh = true) {
  Context& c = ctx();
  if (!c.inited) { set_error("rh_init has not been called"); return RH_ESTATE; }
  if (need_mesh && !c.have_mesh) { set_error("no mesh: call rh_set_mesh first"); return RH_ESTATE; }
  return RH_OK;
}

static int level_of_range(int head_idx, int num_octs) {
  Context& c = ctx();
  for (int l = c.levelmin; l <= c.levelmax; ++l)
    if (c.noct[l] > 0 && c.head[l] == head_idx && c.noct[l] == num_octs) return l;
  return -1;
}

static int level_of_subgrids(int head_sub, int num_sub) {
  Context& c = ctx();
  const int n3 = c.nsubgrid * c.nsubgrid * c.nsubgrid;
  for (int l = c.levelmin; l <= c.levelmax; ++l)
    if (c.noct[l] > 0 && (c.head[l] - 1) / n3 + 1 == head_sub && c.noct[l] / n3 == num_sub) return l;
  return -1;
}

static long long total_octs() { return ctx().ngridmax; }

static void free_tables(LevelTables& t) {
  cudaFree(t.d_phdr);
  cudaFree(t.d_poff);
  cudaFree(t.d_ptab);
  cudaFree(t.d_cfl_partial);
  cudaFree(t.d_gsrc_oct);
  cudaFree(t.d_gsrc_cf);
  t = LevelTables();
}

static void free_state() {
  Context& c = ctx();
  free_host_schedule();
  free_diffusion();
  cudaFree(c.d_gface_all);
  c.d_gface_all = nullptr;
  cudaFree(c.d_cflskip);
  c.d_cflskip = nullptr;
  cudaFree(c.d_gcfl);
  c.d_gcfl = nullptr;
  for (auto& t : c.levels) free_tables(t);
  c.levels.clear();
  for (int i = 0; i < 2; ++i) {
    cudaFree(c.uf[i] ? (void*)c.uf[i] : (void*)c.ud[i]);  // FP32-bulk: ud is a view into uf's records
    c.ud[i] = nullptr;
    c.uf[i] = nullptr;
  }
  cudaFree(c.d_cfl);
  cudaFree(c.d_scratch);
  cudaFree(c.d_refmask);
  cudaFree(c.d_gfather);
  cudaFree(c.d_father);
  for (auto* f : c.d_face) cudaFree(f);
  c.d_face.clear();
  c.d_refmask = nullptr;
  c.d_gfather = nullptr;
  c.d_father = nullptr;
  c.d_cfl = nullptr;
  c.d_scratch = nullptr;
  c.scratch_elems = 0;
  c.have_mesh = false;
  free_image_buffer();
  cudaFree(c.d_stage64);
  c.d_stage64 = nullptr;
  c.stage64_bytes = 0;
}

// Build the pencil tables of a complete (uniform) level (on the device:
// rh_tables.cu) and upload the pencil headers.
static int build_level_tables(int l, const TileCfg& cfg) {
  Context& c = ctx();
  LevelTables& T = c.levels[l];
  free_tables(T);
  T.cfg = cfg;
  int rc = build_complete_tables_device(l, cfg, T);
  if (rc) return rc;
  T.npencil = (int)T.phdr.size();
  RH_CUDA(cudaMalloc(&T.d_phdr, sizeof(int4) * T.phdr.size()));
  RH_CUDA(cudaMalloc(&T.d_poff, sizeof(long long) * T.poff.size()));
  RH_CUDA(cudaMalloc(&T.d_cfl_partial, sizeof(double) * 5 * T.npencil));
  RH_CUDA(cudaMemcpyAsync(T.d_phdr, T.phdr.data(), sizeof(int4) * T.phdr.size(), cudaMemcpyHostToDevice, c.stream));
  RH_CUDA(cudaMemcpyAsync(T.d_poff, T.poff.data(), sizeof(long long) * T.poff.size(), cudaMemcpyHostToDevice,
                          c.stream));
  RH_CUDA(cudaStreamSynchronize(c.stream));
  T.built = true;
  T.complete = true;
  return RH_OK;
}

static int upload_uold(const double* uold) {
  Context& c = ctx();
  const long long n = total_octs();
  if (c.precision == RH_PREC_FP64) {
    RH_CUDA(cudaMemcpyAsync(c.ud[c.cur], uold, sizeof(double) * 40 * n, cudaMemcpyHostToDevice, c.stream));
  } else {
    double* tmp = nullptr;
    int rc = stage64(n, &tmp);
    if (rc) return rc;
    RH_CUDA(cudaMemcpyAsync(tmp, uold, sizeof(double) * 40 * n, cudaMemcpyHostToDevice, c.stream));
    pack_bulk_kernel<<<(unsigned)((n * 8 + 255) / 256), 256, 0, c.stream>>>(tmp, c.uf[c.cur], c.ud[c.cur], n);
    RH_CUDA(cudaGetLastError());
  }
  RH_CUDA(cudaStreamSynchronize(c.stream));
  std::fill(c.cfl_on_unew.begin(), c.cfl_on_unew.end(), 0);
  std::fill(c.cfl_on_uold.begin(), c.cfl_on_uold.end(), 0);
  return RH_OK;
}

static CflConst make_cfl(double dx, double gamma, double smallr, double smallc, double courant,
                         const double* g) {
  CflConst C;
  C.gamma = gamma;
  C.gm1 = gamma - 1.0;
  C.smallr = smallr;
  C.smallp = smallc * smallc / gamma;
  C.cdx_smallc = courant * dx / smallc;
  C.two_cdx = 2.0 * courant * dx;
  C.two_c = 2.0 * courant;
  double gs = 0;
  for (int d = 0; d < 3; ++d) gs += std::fabs(g ? g[d] : 0.0);
  C.gsum_dx = gs * dx;
  C.k0 = C.two_cdx / (1.0 + std::sqrt(1.0 + C.two_c * 0.0001));
  C.ndim = 3;
  return C;
}

}  // namespace rh

using namespace rh;

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* rh_last_error(void) { return g_err.c_str(); }

int rh_init(int device_ordinal) {
  Context& c = ctx();
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    set_error("no CUDA device: %s", cudaGetErrorString(e));
    return RH_ENODEV;
  }
  if (device_ordinal < 0 || device_ordinal >= n) {
    set_error("device %d out of range (%d devices)", device_ordinal, n);
    return RH_EINVAL;
  }
  if (c.inited) {
    if (c.device == device_ordinal) return RH_OK;
    rh_finalize();
  }
  RH_CUDA(cudaSetDevice(device_ordinal));
  cudaDeviceProp prop;
  RH_CUDA(cudaGetDeviceProperties(&prop, device_ordinal));
  if (prop.major != 10) {
    set_error("device %d is sm_%d%d; this library is built for sm_100a (B200)", device_ordinal, prop.major,
              prop.minor);
    return RH_ENODEV;
  }
  c.device = device_ordinal;
  c.sm_count = prop.multiProcessorCount;
  RH_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
  RH_CUDA(cudaMalloc(&c.d_err, sizeof(int)));
  RH_CUDA(cudaMemset(c.d_err, 0, sizeof(int)));
  RH_CUDA(cudaEventCreate(&c.ev0));
  RH_CUDA(cudaEventCreate(&c.ev1));
  RH_CUDA(cudaStreamCreateWithFlags(&c.side, cudaStreamNonBlocking));
  for (auto& s : c.lev_stream) RH_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  RH_CUDA(cudaEventCreateWithFlags(&c.ev_side_start, cudaEventDisableTiming));
  RH_CUDA(cudaStreamCreateWithFlags(&c.cfl_copy, cudaStreamNonBlocking));
  RH_CUDA(cudaEventCreateWithFlags(&c.ev_cfl_copied, cudaEventDisableTiming));
  RH_CUDA(cudaEventCreateWithFlags(&c.ev_cfl_ready, cudaEventDisableTiming));
  c.inited = true;
  return RH_OK;
}

int rh_finalize(void) {
  Context& c = ctx();
  if (!c.inited) return RH_OK;
  cudaStreamSynchronize(c.stream);
  rh_batch_free();
  free_state();
  cudaFree(c.d_err);
  cudaFree(c.d_check);
  cudaFree(c.d_gface);
  cudaFreeHost(c.h_cfl);
  cudaEventDestroy(c.ev0);
  cudaEventDestroy(c.ev1);
  for (cudaEvent_t e : c.ev_prolong) cudaEventDestroy(e);
  for (cudaEvent_t e : c.ev_level) cudaEventDestroy(e);
  for (cudaEvent_t e : c.ev_gather) cudaEventDestroy(e);
  cudaEventDestroy(c.ev_side_start);
  cudaStreamDestroy(c.side);
  cudaEventDestroy(c.ev_cfl_copied);
  cudaEventDestroy(c.ev_cfl_ready);
  cudaStreamDestroy(c.cfl_copy);
  cudaFreeHost(c.h_cfl_next);
  for (auto s : c.lev_stream) cudaStreamDestroy(s);
  cudaStreamDestroy(c.stream);
  c = Context();
  return RH_OK;
}

int rh_sync(void) {
  int rc = check_ready(false);
  if (rc) return rc;
  Context& c = ctx();
  RH_CUDA(cudaStreamSynchronize(c.stream));
  int err = 0;
  RH_CUDA(cudaMemcpy(&err, c.d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    cudaMemset(c.d_err, 0, sizeof(int));
    set_error("device wait bound exceeded (error word %d)", err);
    return RH_ETIMEDOUT;
  }
  return RH_OK;
}

int rh_set_precision(int mode) {
  int rc = check_ready(false);
  if (rc) return rc;
  if (mode != RH_PREC_FP64 && mode != RH_PREC_FP32_BULK) {
    set_error("precision mode %d unknown", mode);
    return RH_EINVAL;
  }
  Context& c = ctx();
  if (c.have_mesh && mode != c.precision) {
    set_error("precision must be chosen before rh_set_mesh");
    return RH_ESTATE;
  }
  c.precision = mode;
  return RH_OK;
}

int rh_set_interpolation(int interpol_var, int interpol_type) {
  if (interpol_var < 0 || interpol_var > 1 || interpol_type < 0 || interpol_type > 3) {
    set_error("interpol_var must be 0/1 and interpol_type 0..3");
    return RH_EINVAL;
  }
  ctx().interpol_var = interpol_var;
  ctx().interpol_type = interpol_type;
  return RH_OK;
}

int rh_set_tile(int txo, int tyo, int minb, int lz) {
  int rc = check_ready(false);
  if (rc) return rc;
  Context& c = ctx();
  if (!find_launcher(c.precision, txo, tyo, minb, 2, 3, 0) || lz < 1) {
    set_error("tile %dx%d (minb=%d, lz=%d) is not compiled for this precision", txo, tyo, minb, lz);
    return RH_EINVAL;
  }
  c.cfg.txo = txo;
  c.cfg.tyo = tyo;
  c.cfg.minb = minb;
  c.cfg.lz = lz;
  if (c.have_mesh && c.nlevels_used == 1)
    for (int l = c.levelmin; l <= c.levelmax; ++l)
      if (c.levels[l].built) {
        rc = build_level_tables(l, c.cfg);
        if (rc) return rc;
      }
  return RH_OK;
}

int rh_set_amr_tile(int txo, int tyo, int minb, int lz) {
  int rc = check_ready(false);
  if (rc) return rc;
  Context& c = ctx();
  if (!find_launcher(c.precision, txo, tyo, minb, 2, 3, 1) || lz < 1) {
    set_error("coarse-fine tile %dx%d (minb=%d, lz=%d) is not compiled for this precision", txo, tyo, minb, lz);
    return RH_EINVAL;
  }
  if (c.have_mesh && c.nlevels_used > 1) {
    set_error("rh_set_amr_tile: call before rh_set_mesh (the ghost octs of a mesh follow its tiles)");
    return RH_ESTATE;
  }
  c.amr_cfg = TileCfg{txo, tyo, minb, lz};
  c.amr_cfg_set = true;
  return RH_OK;
}

int rh_set_mesh(const rh_mesh_desc* m, const double* uold, int nvar, int twotondim) {
  int rc = check_ready(false);
  if (rc) return rc;
  Context& c = ctx();
  // coarse-fine tile unless chosen: the fastest on the AMR Sedov of levels 7-10 per precision
  if (!c.amr_cfg_set) c.amr_cfg = c.precision == RH_PREC_FP32_BULK ? TileCfg{7, 7, 2, 32} : TileCfg{8, 4, 2, 32};
  if (!m || !uold || !m->grid || !m->head || !m->noct) {
    set_error("rh_set_mesh: null pointer");
    return RH_EINVAL;
  }
  if (nvar != 5 || twotondim != 8) {
    set_error("rh_set_mesh: nvar=%d twotondim=%d; this path is NDIM=3 hydro (nvar=5, twotondim=8)", nvar,
              twotondim);
    return RH_EINVAL;
  }
  if (m->levelmin < 1 || m->levelmax < m->levelmin || m->levelmax > 24 || m->ngridmax < 1 || m->nsubgrid < 1) {
    set_error("rh_set_mesh: bad levels/ngridmax/nsubgrid");
    return RH_EINVAL;
  }
  cudaStreamSynchronize(c.stream);
  free_state();
  c.nsubgrid = m->nsubgrid;
  c.levelmin = m->levelmin;
  c.levelmax = m->levelmax;
  c.ngridmax = m->ngridmax;
  for (int d = 0; d < 3; ++d) {
    c.box_nx[d] = m->box_nx[d];
    c.periodic[d] = m->periodic[d];
    c.gravity[d] = m->constant_gravity[d];
  }
  for (int i = 0; i < 6; ++i) {
    c.bound_type[i] = m->bound_type[i];
    const int d = i / 2;
    if (!c.periodic[d] && c.bound_type[i] != RH_BOUND_ZERO_GRADIENT && c.bound_type[i] != RH_BOUND_REFLEXIVE) {
      set_error("boundary %d: type %d not supported (periodic, reflexive or zero-gradient)", i, c.bound_type[i]);
      return RH_EINVAL;
    }
  }
  c.boxlen = m->boxlen;
  c.head.assign(m->head, m->head + m->levelmax + 1);
  c.noct.assign(m->noct, m->noct + m->levelmax + 1);
  long long nused = 0;
  for (int l = c.levelmin; l <= c.levelmax; ++l) {
    if (c.noct[l] < 0 || (c.noct[l] > 0 && (c.head[l] < 1 || c.head[l] - 1 + (long long)c.noct[l] > c.ngridmax))) {
      set_error("level %d range [%d, +%d) outside 1..ngridmax=%d", l, c.head[l], c.noct[l], c.ngridmax);
      return RH_EINVAL;
    }
    nused = std::max(nused, (long long)c.head[l] - 1 + c.noct[l]);
  }
  c.grid.assign(m->grid, m->grid + nused);
  c.nlevels_used = 0;
  for (int l = c.levelmin; l <= c.levelmax; ++l) c.nlevels_used += c.noct[l] > 0;
  const bool multi = c.nlevels_used > 1;
  c.levels.assign(c.levelmax + 1, LevelTables());
  // coarse-fine levels: tables first, they fix the number of ghost octs
  long long nghost = 0;
  std::vector<std::pair<int2*, long long>> dev_gfather;  // device-built ghost fathers, per level
  rh_oct* d_grid = nullptr;
  auto drop_tables = [&]() {
    for (auto& t : c.levels) free_tables(t);
    c.levels.clear();
    for (auto& f : dev_gfather) cudaFree(f.first);
    cudaFree(d_grid);
  };
  for (int l = c.levelmin; l <= c.levelmax; ++l) {
    if (c.noct[l] == 0) continue;
    const long long box = ((long long)c.box_nx[0] << (l - 1)) * ((long long)c.box_nx[1] << (l - 1)) *
                          ((long long)c.box_nx[2] << (l - 1));
    if ((long long)c.noct[l] == box) continue;
    const long long gbase = (long long)c.ngridmax + nghost;
    // A small level gets shorter pencils so that it still fills a wave of
    // CTAs (its pencils are few; each one marches lz layers one after the
    // other): halve lz, down to 2, while the level's octs make fewer pencils
    // than that.  (One wave rather than two: rh_coarse_step runs the levels
    // at once, and on the AMR Sedov of levels 7-10 that gave its level 10
    // 16 layers instead of 8, 1.9 % (FP64) / 0.5 % (FP32-bulk) faster.)
    TileCfg lcfg = c.amr_cfg;
    const long long wave = (long long)c.sm_count * std::max(1, lcfg.minb);
    while (lcfg.lz > 2 && (long long)c.noct[l] / ((long long)lcfg.txo * lcfg.tyo * lcfg.lz) < wave) lcfg.lz /= 2;
    if (c.table_builder) {
      cudaError_t e = cudaSuccess;
      if (!d_grid) {
        e = cudaMalloc(&d_grid, sizeof(rh_oct) * c.grid.size());
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(d_grid, c.grid.data(), sizeof(rh_oct) * c.grid.size(), cudaMemcpyHostToDevice,
                              c.stream);
      }
      int2* gf = nullptr;
      rc = e == cudaSuccess ? build_amr_tables_device(l, lcfg, gbase, d_grid, &gf)
                            : cuda_fail(e, "oct records to the device");
      if (gf) dev_gfather.push_back({gf, gbase});
    } else {
      rc = build_amr_tables(l, lcfg, gbase);
    }
    if (rc) {
      drop_tables();
      return rc;
    }
    nghost += c.levels[l].nghost;
  }
  cudaFree(d_grid);
  d_grid = nullptr;
  c.nstate = (long long)c.ngridmax + nghost;
  const long long n = c.nstate;
  for (int i = 0; i < 2; ++i) {
    if (c.precision == RH_PREC_FP64) {
      RH_CUDA(cudaMalloc(&c.ud[i], sizeof(double) * 40 * n));
    } else {
      RH_CUDA(cudaMalloc(&c.uf[i], (size_t)kBulkBytes * n));
      c.ud[i] = reinterpret_cast<double*>(c.uf[i]) + kBulkE;
    }
  }
  RH_CUDA(cudaMalloc(&c.d_cfl, sizeof(double) * 5 * (c.levelmax + 1)));
  c.cfl_gen++;
  cudaFreeHost(c.h_cfl_next);
  c.h_cfl_next = nullptr;
  RH_CUDA(cudaMallocHost(&c.h_cfl_next, sizeof(double) * 5 * (c.levelmax + 1)));
  {
    std::vector<uint8_t> ref((size_t)n, 0);
    for (long long i = 0; i < nused; ++i) {
      uint8_t b = 0;
      for (int k = 0; k < 8; ++k) b |= (uint8_t)((c.grid[i].refined[k] ? 1 : 0) << k);
      ref[i] = b;
    }
    RH_CUDA(cudaMalloc(&c.d_refmask, (size_t)n));
    RH_CUDA(cudaMemcpy(c.d_refmask, ref.data(), (size_t)n, cudaMemcpyHostToDevice));
    RH_CUDA(cudaMalloc(&c.d_gfather, sizeof(int2) * (size_t)std::max(1LL, nghost)));
    int nlev_ghost = 0;
    for (int l = c.levelmin; l <= c.levelmax; ++l) {
      const LevelTables& T = c.levels[l];
      if (!T.built || T.nghost == 0) continue;
      const auto& f = dev_gfather[(size_t)nlev_ghost++];
      RH_CUDA(cudaMemcpyAsync(c.d_gfather + (f.second - c.ngridmax), f.first, sizeof(int2) * T.nghost,
                              cudaMemcpyDeviceToDevice, c.stream));
    }
    RH_CUDA(cudaStreamSynchronize(c.stream));
    for (auto& f : dev_gfather) cudaFree(f.first);
    dev_gfather.clear();
  }
  c.cur = 0;
  c.unew_pending.assign(c.levelmax + 1, 0);
  c.unew_copied.assign(c.levelmax + 1, 0);
  c.unew_written.assign(c.levelmax + 1, 0);
  c.cfl_on_unew.assign(c.levelmax + 1, 0);
  c.cfl_on_uold.assign(c.levelmax + 1, 0);
  c.cfl_keys.assign(8 * (c.levelmax + 1), 0.0);
  c.have_mesh = true;
  rc = upload_uold(uold);
  if (rc) return rc;
  for (int l = c.levelmin; l <= c.levelmax; ++l) {
    if (c.noct[l] == 0) continue;
    if (c.levels[l].built) continue;  // coarse-fine level built on the device
    if (c.levels[l].nghost > 0 || (c.levels[l].npencil > 0 && !c.levels[l].complete)) {
      rc = upload_amr_tables(l);
      if (rc) return rc;
      continue;
    }
    rc = build_level_tables(l, level_cfg(l));
    if (rc) {
      // keep the mesh usable for set_unew/set_uold/cmpdt; godunov on this
      // level will report the table error
      c.levels[l].built = false;
    }
  }
  return RH_OK;
}

int rh_set_grid_device(const double* uold, int ngridmax, int nvar, int twotondim) {
  int rc = check_ready();
  if (rc) return rc;
  Context& c = ctx();
  if (!uold || ngridmax != c.ngridmax || nvar != 5 || twotondim != 8) {
    set_error("rh_set_grid_device: shape differs from the mesh (ngridmax=%d)", c.ngridmax);
    return RH_EINVAL;
  }
  return upload_uold(uold);
}

int rh_transfer_grid_host(double* uold, int ngridmax, int nvar, int twotondim) {
  int rc = check_ready();
  if (rc) return rc;
  Context& c = ctx();
  if (!uold || ngridmax != c.ngridmax || nvar != 5 || twotondim != 8) {
    set_error("rh_transfer_grid_host: shape differs from the mesh (ngridmax=%d)", c.ngridmax);
    return RH_EINVAL;
  }
  const long long n = c.ngridmax;
  if (c.precision == RH_PREC_FP64) {
    RH_CUDA(cudaMemcpyAsync(uold, c.ud[c.cur], sizeof(double) * 40 * n, cudaMemcpyDeviceToHost, c.stream));
  } else {
    double* tmp = nullptr;
    int rc2 = stage64(n, &tmp);
    if (rc2) return rc2;
    unpack_bulk_kernel<<<(unsigned)((n * 8 + 255) / 256), 256, 0, c.stream>>>(tmp, c.uf[c.cur], c.ud[c.cur], n);
    RH_CUDA(cudaGetLastError());
    RH_CUDA(cudaMemcpyAsync(uold, tmp, sizeof(double) * 40 * n, cudaMemcpyDeviceToHost, c.stream));
  }
  RH_CUDA(cudaStreamSynchronize(c.stream));
  return RH_OK;
}

// Copy a level range between the two state buffers (src -> dst).
static int copy_level(int head_idx, int num_octs, int src, int dst) {
  Context& c = ctx();
  const long long o0 = head_idx - 1, n = num_octs;
  const int threads = 256;
  const int blocks = std::max(1, std::min(c.sm_count * 8, (int)((n * 40 + threads - 1) / threads)));
  if (c.precision == RH_PREC_FP64) {
    copy_kernel<double><<<blocks, threads, 0, c.stream>>>(c.ud[dst] + o0 * 40, c.ud[src] + o0 * 40, n * 40);
  } else {
    copy_kernel<float><<<blocks, threads, 0, c.stream>>>(c.uf[dst] + o0 * kBulkF, c.uf[src] + o0 * kBulkF,
                                                       n * kBulkF);
  }
  RH_CUDA(cudaGetLastError());
  return RH_OK;
}

int rh_set_unew(int head_idx, int num_octs) {
  int rc = check_ready();
  if (rc) return rc;
  Context& c = ctx();
  if (num_octs == 0) return RH_OK;
  if (head_idx < 1 || num_octs < 0 || head_idx - 1 + (long long)num_octs > c.ngridmax) {
    set_error("rh_set_unew: range outside the mesh");
    return RH_EINVAL;
  }
  const int l = level_of_range(head_idx, num_octs);
  if (l >= 0 && c.nlevels_used == 1) {
    // unew = uold is folded into the next rh_godunov of this level, which then
    // writes unew = uold + flux differences for every oct of the level.
    c.unew_pending[l] = 1;
    c.unew_written[l] = 0;
    return RH_OK;
  }
  // several levels: finer levels add coarse corrections into this unew before
  // its own Godunov step, so the copy is made now (godunov_fine.f90:114-148)
  int rc2 = copy_level(head_idx, num_octs, c.cur, 1 - c.cur);
  if (rc2) return rc2;
  if (l >= 0) {
    c.unew_copied[l] = 1;
    c.unew_pending[l] = 0;
    c.unew_written[l] = 0;
  }
  return RH_OK;
}

int rh_set_uold(int head_idx, int num_octs) {
  int rc = check_ready();
  if (rc) return rc;
  Context& c = ctx();
  if (num_octs == 0) return RH_OK;
  if (head_idx < 1 || num_octs < 0 || head_idx - 1 + (long long)num_octs > c.ngridmax) {
    set_error("rh_set_uold: range outside the mesh");
    return RH_EINVAL;
  }
  const int l = level_of_range(head_idx, num_octs);
  if (l >= 0 && c.unew_pending[l]) {
    // set_unew without godunov: unew == uold, nothing to copy
    c.unew_pending[l] = 0;
    return RH_OK;
  }
  // single level spanning the whole state: swap the buffers
  int nlev = 0;
  for (int k = c.levelmin; k <= c.levelmax; ++k) nlev += c.noct[k] > 0;
  if (l >= 0 && nlev == 1 && c.unew_written[l]) {
    c.cur = 1 - c.cur;
    c.unew_written[l] = 0;
    if (c.cfl_on_unew[l]) {
      c.cfl_on_unew[l] = 0;
      c.cfl_on_uold[l] = 1;
    }
    return RH_OK;
  }
  rc = copy_level(head_idx, num_octs, 1 - c.cur, c.cur);
  if (rc) return rc;
  if (l >= 0) {
    c.unew_written[l] = 0;
    c.unew_copied[l] = 0;
    c.cfl_on_uold[l] = c.cfl_on_unew[l];
    c.cfl_on_unew[l] = 0;
  }
  return RH_OK;
}

}  // extern "C"

// courant_fine of one level range, queued on the library stream: the five
// reduced values land in host_out (pinned) once the stream reaches them.
// *queued is false when there is nothing to wait for (an empty range).
static int cmpdt_enqueue(int head_idx, int num_octs, double dx, double gamma, double smallr, double smallc,
                         double courant_factor, const double* constant_gravity, double* host_out, bool* queued) {
  Context& c = ctx();
  *queued = false;
  if (!(dx > 0) || !(gamma > 1) || !(smallc > 0) || !(courant_factor > 0)) {
    set_error("rh_cmpdt: need dx>0, gamma>1, smallc>0, courant_factor>0");
    return RH_EINVAL;
  }
  const double g[3] = {constant_gravity ? constant_gravity[0] : 0.0, constant_gravity ? constant_gravity[1] : 0.0,
                       constant_gravity ? constant_gravity[2] : 0.0};
  if (num_octs == 0) return RH_OK;
  if (head_idx < 1 || num_octs < 0 || head_idx - 1 + (long long)num_octs > c.ngridmax) {
    set_error("rh_cmpdt: range outside the mesh");
    return RH_EINVAL;
  }
  const int l = level_of_range(head_idx, num_octs);
  const double key[8] = {dx, gamma, smallr, smallc, courant_factor, g[0], g[1], g[2]};
  double* lkey = l >= 0 ? &c.cfl_keys[8 * l] : nullptr;
  const bool same_key = lkey && std::equal(key, key + 8, lkey);
  if (l >= 0 && c.cfl_on_uold[l] && same_key) {
    RH_CUDA(cudaMemcpyAsync(host_out, c.d_cfl + 5 * l, sizeof(double) * 5, cudaMemcpyDeviceToHost, c.stream));
  } else {
    const long long ncell = (long long)num_octs * 8;
    const int threads = 256;
    const long long nblk = (ncell + threads - 1) / threads;
    if ((size_t)nblk * 5 > c.scratch_elems) {
      cudaFree(c.d_scratch);  // synchronises: queued reductions are done with it
      c.d_scratch = nullptr;
      RH_CUDA(cudaMalloc(&c.d_scratch, sizeof(double) * 5 * nblk));
      c.scratch_elems = (size_t)nblk * 5;
    }
    // leaf mask: the refined-cell bits of the grid records, resident since rh_set_mesh
    const CflConst C = make_cfl(dx, gamma, smallr, smallc, courant_factor, g);
    const double vol = dx * dx * dx;
    const bool fp32 = c.precision == RH_PREC_FP32_BULK;
    cmpdt_kernel<<<(unsigned)nblk, threads, 0, c.stream>>>(c.ud[c.cur], c.uf[c.cur], fp32 ? 1 : 0, nullptr,
                                                           head_idx - 1, num_octs, C, vol, c.d_scratch,
                                                           c.d_refmask);
    RH_CUDA(cudaGetLastError());
    double* d_out = c.d_cfl + 5 * (l >= 0 ? l : 0);
    c.cfl_gen++;
    reduce_partials_kernel<<<1, 1024, 0, c.stream>>>(c.d_scratch, nblk, 1e300, d_out);
    RH_CUDA(cudaGetLastError());
    RH_CUDA(cudaMemcpyAsync(host_out, d_out, sizeof(double) * 5, cudaMemcpyDeviceToHost, c.stream));
    if (l >= 0) c.cfl_on_uold[l] = 0;
  }
  if (lkey) std::copy(key, key + 8, lkey);
  *queued = true;
  return RH_OK;
}

// Pinned landing area of the courant_fine values, one slot of 5 per level.
static int cfl_host(double** out) {
  Context& c = ctx();
  const size_t need = 5 * (size_t)(c.levelmax + 1);
  if (c.h_cfl_elems < need) {
    cudaFreeHost(c.h_cfl);
    c.h_cfl = nullptr;
    c.h_cfl_elems = 0;
    RH_CUDA(cudaMallocHost(&c.h_cfl, sizeof(double) * need));
    c.h_cfl_elems = need;
  }
  *out = c.h_cfl;
  return RH_OK;
}

extern "C" {

int rh_cmpdt(int head_idx, int num_octs, double dx, double gamma, double smallr, double smallc,
             double courant_factor, const double* constant_gravity, double* mass, double* ekin, double* eint,
             double* emag, double* dt) {
  int rc = check_ready();
  if (rc) return rc;
  Context& c = ctx();
  if (!mass || !ekin || !eint || !emag || !dt) {
    set_error("rh_cmpdt: null output pointer");
    return RH_EINVAL;
  }
  *mass = *ekin = *eint = *emag = 0.0;
  if (dx > 0 && smallc > 0) *dt = dx / smallc;  // courant_fine.f90:86
  double* h = nullptr;
  if ((rc = cfl_host(&h))) return rc;
  bool queued = false;
  if ((rc = cmpdt_enqueue(head_idx, num_octs, dx, gamma, smallr, smallc, courant_factor, constant_gravity, h,
                          &queued)))
    return rc;
  if (!queued) return RH_OK;
  RH_CUDA(cudaStreamSynchronize(c.stream));
  *mass = h[0];
  *ekin = h[1];
  *eint = h[2];
  *emag = 0.0;
  *dt = std::min(*dt, h[4]);
  return RH_OK;
}

}  // extern "C"

namespace rh {

// The deterministic coarse-fine update: each ghost oct of the level adds the
// 24 face slots its neighbours' pencils stored (zero where no real cell
// borders it) to its father cell, in slot order, one thread per (ghost, var):
// the sums no longer depend on which pencil ran first.  The role of the
// reference's fixed-order flush of cache octs (hydro/godunov_fine.f90:
// 1347-1459) for the father cells of a level.
__global__ void coarse_gather_kernel(const double* __restrict__ gface, int nghost, const int2* __restrict__ fathers,
                                     double* __restrict__ unew) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)nghost * 5) return;
  const int g = (int)(i / 5), v = (int)(i % 5);
  const int2 fa = fathers[g];
  if (fa.x < 0) return;
  const double* s = gface + (size_t)g * 24 * 5 + v;
  double sum = 0.0;
#pragma unroll 4
  for (int f = 0; f < 24; ++f) sum += s[5 * f];
  unew[(size_t)fa.x * 40 + 8 * v + fa.y] += sum;
}

// Tile of level l's launches: the uniform tile on a single-level mesh, the
// coarse-fine tile (kernels that handle refined cells and interpolated ghosts)
// on every level of a multi-level mesh.  A partial level takes the tile's
// layers cut down by rh_set_mesh until it fills a wave of CTAs; a
// complete level takes them all (on the AMR Sedov of levels 7-10, whose
// level 7 is complete, 32 layers there instead of 8 made the coarse step
// 4 % (FP32-bulk) and 1.4 % (FP64) faster, 64 layers 30 % / 20 % slower).
TileCfg level_cfg(int l) {
  Context& c = ctx();
  (void)l;
  return c.nlevels_used > 1 ? c.amr_cfg : c.cfg;
}

// The same for FP32-bulk records: the four float variables and the FP64
// energy of each father cell receive their slot sums (added up in FP64).
__global__ void coarse_gather_f32_kernel(const double* __restrict__ gface, int nghost,
                                         const int2* __restrict__ fathers, float* __restrict__ unew_f,
                                         double* __restrict__ unew_e) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)nghost * 5) return;
  const int g = (int)(i / 5), v = (int)(i % 5);
  const int2 fa = fathers[g];
  if (fa.x < 0) return;
  const double* s = gface + (size_t)g * 24 * 5 + v;
  double sum = 0.0;
#pragma unroll 4
  for (int f = 0; f < 24; ++f) sum += s[5 * f];
  if (v < 4) {
    float* o = unew_f + (size_t)fa.x * kBulkF + 8 * v + fa.y;
    *o = (float)((double)*o + sum);
  } else {
    unew_e[(size_t)fa.x * kBulkD + fa.y] += sum;
  }
}

// The concurrent coarse step's coarse-fine update with the courant_fine
// values of the cells it corrects.  The fused CFL epilogue of a level leaves
// out its cells that father a finer level's ghost octs (LevelArgs::cflskip):
// their state is final only once the finer level's face slots are added.
// Here one thread per (ghost, variable) adds them in slot order exactly as
// coarse_gather_kernel does, 64 ghosts per block, and one thread per ghost
// then takes its father cell's new state into the block's CFL partial (the
// cell as courant_fine sees it: the stored values, FP32 ones in FP32-bulk).
// The level's pencil partials and these together cover each of its leaf
// cells once.
constexpr int kGatherGhosts = 64;
constexpr int kGatherThreads = kGatherGhosts * 5;

__global__ void __launch_bounds__(kGatherThreads)
    coarse_gather_cfl_kernel(const double* __restrict__ gface, int nghost, const int2* __restrict__ fathers,
                             const uint8_t* __restrict__ refmask, double* __restrict__ unew, CflConst C, double vol,
                             double* __restrict__ partial) {
  __shared__ double cell[kGatherGhosts][5];
  __shared__ double red[kGatherThreads / 32 * 4];
  const int lg = threadIdx.x / 5, v = threadIdx.x - 5 * lg;
  const long long g = (long long)blockIdx.x * kGatherGhosts + lg;
  if (g < nghost) {
    const int2 fa = fathers[g];
    if (fa.x >= 0) {
      const double* s = gface + (size_t)g * 24 * 5 + v;
      double sum = 0.0;
#pragma unroll 4
      for (int f = 0; f < 24; ++f) sum += s[5 * f];
      double* o = unew + (size_t)fa.x * 40 + 8 * v + fa.y;
      const double nv = *o + sum;
      *o = nv;
      cell[lg][v] = nv;
    }
  }
  __syncthreads();
  CflAcc acc;
  if (threadIdx.x < kGatherGhosts) {
    const long long gg = (long long)blockIdx.x * kGatherGhosts + threadIdx.x;
    if (gg < nghost) {
      const int2 fa = fathers[gg];
      if (fa.x >= 0 && !((refmask[fa.x] >> fa.y) & 1u)) {
        const double* q = cell[threadIdx.x];
        acc.add(q[0], q[1], q[2], q[3], q[4], C, vol);
      }
    }
  }
  cfl_block_reduce<kGatherThreads / 32>(acc, C, red, partial + (size_t)blockIdx.x * 5);
}

__global__ void __launch_bounds__(kGatherThreads)
    coarse_gather_cfl_f32_kernel(const double* __restrict__ gface, int nghost, const int2* __restrict__ fathers,
                                 const uint8_t* __restrict__ refmask, float* __restrict__ unew_f,
                                 double* __restrict__ unew_e, CflConst C, double vol, double* __restrict__ partial) {
  __shared__ double cell[kGatherGhosts][5];
  __shared__ double red[kGatherThreads / 32 * 4];
  const int lg = threadIdx.x / 5, v = threadIdx.x - 5 * lg;
  const long long g = (long long)blockIdx.x * kGatherGhosts + lg;
  if (g < nghost) {
    const int2 fa = fathers[g];
    if (fa.x >= 0) {
      const double* s = gface + (size_t)g * 24 * 5 + v;
      double sum = 0.0;
#pragma unroll 4
      for (int f = 0; f < 24; ++f) sum += s[5 * f];
      if (v < 4) {
        float* o = unew_f + (size_t)fa.x * kBulkF + 8 * v + fa.y;
        const float nv = (float)((double)*o + sum);
        *o = nv;
        cell[lg][v] = nv;
      } else {
        double* o = unew_e + (size_t)fa.x * kBulkD + fa.y;
        const double nv = *o + sum;
        *o = nv;
        cell[lg][4] = nv;
      }
    }
  }
  __syncthreads();
  CflAcc acc;
  if (threadIdx.x < kGatherGhosts) {
    const long long gg = (long long)blockIdx.x * kGatherGhosts + threadIdx.x;
    if (gg < nghost) {
      const int2 fa = fathers[gg];
      if (fa.x >= 0 && !((refmask[fa.x] >> fa.y) & 1u)) {
        const double* q = cell[threadIdx.x];
        acc.add_bulk((float)q[0], (float)q[1], (float)q[2], (float)q[3], q[4], C);
      }
    }
  }
  acc.scale_bulk(vol);
  cfl_block_reduce<kGatherThreads / 32>(acc, C, red, partial + (size_t)blockIdx.x * 5);
}

// Bit fa.y of byte fa.x for every ghost's father cell (the byte array read
// as 32-bit words, zeroed before).
__global__ void mark_fathers_kernel(const int2* __restrict__ fathers, int nghost, unsigned* __restrict__ mask) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= nghost) return;
  const int2 fa = fathers[g];
  if (fa.x < 0) return;
  atomicOr(mask + (fa.x >> 2), 1u << (8 * (fa.x & 3) + fa.y));
}

// reduce_partials_kernel over two partial arrays taken as one (a level's
// pencil partials followed by its corrected cells' gather partials).
__global__ void reduce_partials_pair_kernel(const double* __restrict__ p1, long long n1,
                                            const double* __restrict__ p2, long long n2, double dt0,
                                            double* __restrict__ out) {
  __shared__ double red[1024][4];
  double a = 0, b = 0, c = 0, d = 1e300;
  for (long long i = threadIdx.x; i < n1 + n2; i += blockDim.x) {
    const double* q = i < n1 ? p1 + i * 5 : p2 + (i - n1) * 5;
    a += q[0]; b += q[1]; c += q[2];
    d = q[4] < d ? q[4] : d;
  }
  red[threadIdx.x][0] = a; red[threadIdx.x][1] = b; red[threadIdx.x][2] = c; red[threadIdx.x][3] = d;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      red[threadIdx.x][0] += red[threadIdx.x + s][0];
      red[threadIdx.x][1] += red[threadIdx.x + s][1];
      red[threadIdx.x][2] += red[threadIdx.x + s][2];
      double o = red[threadIdx.x + s][3];
      red[threadIdx.x][3] = o < red[threadIdx.x][3] ? o : red[threadIdx.x][3];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = red[0][0]; out[1] = red[0][1]; out[2] = red[0][2]; out[3] = 0.0;
    out[4] = red[0][3] < dt0 ? red[0][3] : dt0;
  }
}

// Pencil tables of level l for the tile the level's launches use (built, or
// rebuilt after a tile change, on demand).
int ensure_level_tables(int l) {
  Context& c = ctx();
  LevelTables& T = c.levels[l];
  const TileCfg want = level_cfg(l);
  if (T.complete || !T.built) {
    if (!T.built || T.cfg.txo != want.txo || T.cfg.tyo != want.tyo || T.cfg.lz != want.lz)
      return build_level_tables(l, want);
  }
  return RH_OK;
}

// Launch one Godunov step of level l with the given tile configuration.
// Exposed to the batch/bench layer through rh_godunov and rh_bench_*.  With
// `range` only the pencils it lists run (its headers, table offsets and CFL
// partial slots; no partial reduction): rh_coarse_step_host launches a level
// group by group that way.
int launch_level(int l, double gamma, double smallr, double smallc, double dt, double dx, double smax_cap,
                 int slope, int riemann, const double* g, bool fuse_cfl, bool accumulate, const PencilRange* range,
                 const LevelSlots* slots) {
  Context& c = ctx();
  LevelTables& T = c.levels[l];
  const bool amr = c.nlevels_used > 1;  // refined cells / coarse-fine faces exist on every level
  const TileCfg want = level_cfg(l);
  {
    int rc = ensure_level_tables(l);
    if (rc) return rc;
  }
  size_t smem = 0;
  int threads = 0;
  LaunchFn fn = find_launcher(c.precision, T.cfg.txo, T.cfg.tyo, want.minb, slope, riemann, amr ? 1 : 0, &smem,
                              &threads);
  if (!fn) {
    set_error("no kernel for precision %d tile %dx%d (minb %d) slope %d riemann %d amr %d", c.precision, T.cfg.txo,
              T.cfg.tyo, want.minb, slope, riemann, amr ? 1 : 0);
    return RH_EINVAL;
  }
  cudaStream_t st = range && range->stream ? range->stream : (slots && slots->stream ? slots->stream : c.stream);
  if (amr) {
    if (l < (int)c.prolonged.size() && c.prolonged[l]) {
      // prolonged ahead on the side stream by rh_coarse_step
      RH_CUDA(cudaStreamWaitEvent(st, c.ev_prolong[l], 0));
      c.prolonged[l] = 0;
    } else {
      int rc = prolong_ghosts(l, smallr, st);
      if (rc) return rc;
    }
  }
  if (T.npencil == 0) return RH_OK;
  if (range && range->n == 0) return RH_OK;
  LevelArgs A;
  A.phdr = range ? range->phdr : T.d_phdr;
  A.poff = range ? range->poff : T.d_poff;
  A.ptab = range ? range->ptab : T.d_ptab;
  A.npencil = range ? range->n : T.npencil;
  const int nblocks = A.npencil;
  A.ncx = 2 * T.nxo;
  A.ncy = 2 * T.nyo;
  A.ncz = 2 * T.nzo;
  for (int d = 0; d < 3; ++d) A.periodic[d] = c.periodic[d];
  for (int i = 0; i < 6; ++i) A.btype[i] = c.bound_type[i];
  A.ghost_base = c.ngridmax;
  A.err = c.d_err;
  const double* lkey = &c.cfl_keys[8 * l];
  const double courant = lkey[4] > 0 ? lkey[4] : smax_cap * dt / dx;
  A.cfl = make_cfl(dx, gamma, smallr, smallc, courant, g);
  A.vol = dx * dx * dx;
  A.cfl_partial = fuse_cfl ? (range ? range->partial : T.d_cfl_partial) : nullptr;
  A.refmask = c.d_refmask;
  A.ghost_father = c.d_gfather;
  A.accumulate = accumulate ? 1 : 0;
  A.gface = slots ? slots->gface : nullptr;
  A.gface_base = slots ? slots->base : T.gbase;
  A.cflskip = slots ? slots->cflskip : nullptr;
  const bool gather = !slots && amr && c.deterministic && T.nghost > 0;
  if (gather) {
    const size_t need = (size_t)T.nghost * 24 * 5;
    if (c.gface_elems < need) {
      RH_CUDA(cudaStreamSynchronize(c.stream));
      cudaFree(c.d_gface);
      c.d_gface = nullptr;
      c.gface_elems = 0;
      RH_CUDA(cudaMalloc(&c.d_gface, sizeof(double) * need));
      c.gface_elems = need;
    }
    RH_CUDA(cudaMemsetAsync(c.d_gface, 0, sizeof(double) * need, c.stream));
    A.gface = c.d_gface;
  }
  const int nxt = 1 - c.cur;
  A.gm1_d = gamma - 1.0;
  A.smalle_d = smallc * smallc / gamma / (gamma - 1.0);
  const double gh[3] = {(g ? g[0] : 0.0) * (dt * 0.5), (g ? g[1] : 0.0) * (dt * 0.5), (g ? g[2] : 0.0) * (dt * 0.5)};
  if (c.precision == RH_PREC_FP64) {
    StateArgs<double> S{c.ud[c.cur], nullptr, c.ud[nxt], nullptr};
    HydroK<double> H;
    H.gamma = gamma; H.entho = 1.0 / (gamma - 1.0);
    H.smallr = smallr; H.smallc2 = smallc * smallc;
    H.smallp_trace = smallr * (smallc * smallc);
    H.smallp_riem = smallc * smallc / gamma;
    H.smax_cap = smax_cap; H.dtdx = dt / dx;
    H.zero = 0.0; H.half = 0.5; H.two = 2.0;
    H.gm1 = gamma - 1.0; H.smalle = A.smalle_d;
    for (int d = 0; d < 3; ++d) H.grav[d] = gh[d];
    RH_CUDA(fn(A, &S, &H, nblocks, st));
  } else {
    StateArgs<float> S{c.ud[c.cur], c.uf[c.cur], c.ud[nxt], c.uf[nxt]};
    HydroK<float2> H;
    auto b = [](double v) { float f = (float)v; return make_float2(f, f); };
    H.gamma = b(gamma); H.entho = b(1.0 / (gamma - 1.0));
    H.smallr = b(smallr); H.smallc2 = b(smallc * smallc);
    H.smallp_trace = b(smallr * (smallc * smallc));
    H.smallp_riem = b(smallc * smallc / gamma);
    H.smax_cap = b(std::min(smax_cap, 3.0e38)); H.dtdx = b(dt / dx);
    H.zero = b(0.0); H.half = b(0.5); H.two = b(2.0);
    H.gm1 = b(gamma - 1.0); H.smalle = b(A.smalle_d);
    for (int d = 0; d < 3; ++d) H.grav[d] = b(gh[d]);
    RH_CUDA(fn(A, &S, &H, nblocks, st));
  }
  if (gather) {
    const unsigned nb = (unsigned)((T.nghost * 5ll + 255) / 256);
    if (c.precision == RH_PREC_FP64)
      coarse_gather_kernel<<<nb, 256, 0, c.stream>>>(c.d_gface, T.nghost, c.d_gfather + (T.gbase - c.ngridmax),
                                                     c.ud[nxt]);
    else
      coarse_gather_f32_kernel<<<nb, 256, 0, c.stream>>>(c.d_gface, T.nghost, c.d_gfather + (T.gbase - c.ngridmax),
                                                         c.uf[nxt], c.ud[nxt]);
    RH_CUDA(cudaGetLastError());
  }
  if (fuse_cfl && !range && !(slots && slots->defer_reduce)) {
    reduce_partials_kernel<<<1, 1024, 0, st>>>(T.d_cfl_partial, T.npencil, A.cfl.cdx_smallc, c.d_cfl + 5 * l);
    c.cfl_gen++;
    RH_CUDA(cudaGetLastError());
  }
  return RH_OK;
}

}  // namespace rh

extern "C" {

int rh_godunov(int head_idx, int num_subgrids, int ngridmax, int ilevel, int levelmin, int levelmax, double gamma,
               double smallr, double smallc2, double dt, double dx, double smax_cap, int slope, int riemann,
               const double* constant_gravity) {
  int rc = check_ready();
  if (rc) return rc;
  Context& c = ctx();
  if (num_subgrids == 0) return RH_OK;
  if (ngridmax != c.ngridmax || levelmin != c.levelmin || levelmax != c.levelmax) {
    set_error("rh_godunov: ngridmax/levelmin/levelmax differ from the mesh");
    return RH_EINVAL;
  }
  const int l = level_of_subgrids(head_idx, num_subgrids);
  if (l != ilevel) {
    set_error("rh_godunov: subgrids [%d,+%d) are not level %d of the mesh", head_idx, num_subgrids, ilevel);
    return RH_EINVAL;
  }
  if (!(dt > 0) || !(dx > 0) || !(gamma > 1) || !(smallc2 > 0)) {
    set_error("rh_godunov: need dt>0, dx>0, gamma>1, smallc2>0");
    return RH_EINVAL;
  }
  if (slope < 0 || slope > 3) {
    set_error("rh_godunov: slope_type %d not supported (0 none, 1 minmod, 2 moncen, 3 positivity)", slope);
    return RH_EINVAL;
  }
  if (riemann < 1 || riemann > 3) {
    set_error("rh_godunov: riemann %d not supported (llf=1, hll=2, hllc=3)", riemann);
    return RH_EINVAL;
  }
  if (!c.unew_pending[l] && !c.unew_copied[l]) {
    set_error("rh_godunov: call rh_set_unew for level %d first (unew must start as uold)", l);
    return RH_ESTATE;
  }
  double g[3] = {0, 0, 0};
  if (constant_gravity)
    for (int d = 0; d < 3; ++d) g[d] = constant_gravity[d];
  // The fused CFL epilogue uses the parameters of the last rh_cmpdt call.
  const double* key = &c.cfl_keys[8 * l];
  const bool fuse = key[0] == dx && key[1] == gamma && key[2] == smallr && key[5] == g[0] && key[6] == g[1] &&
                    key[7] == g[2] && key[3] * key[3] == smallc2;
  rc = launch_level(l, gamma, smallr, std::sqrt(smallc2), dt, dx, smax_cap, slope, riemann, g, fuse,
                    c.unew_copied[l] != 0);
  if (rc) return rc;
  c.unew_pending[l] = 0;
  c.unew_written[l] = 1;
  c.cfl_on_unew[l] = fuse ? 1 : 0;
  c.cfl_on_uold[l] = 0;
  return RH_OK;
}

// ---- extensions used by the Python host layer and the bench ---------------

// Device pointers of the current uold/unew buffers (for zero-copy views).
int rh_state_ptrs(void** uold_d, void** uold_f, void** unew_d, void** unew_f) {
  int rc = check_ready();
  if (rc) return rc;
  Context& c = ctx();
  if (uold_d) *uold_d = c.ud[c.cur];
  if (uold_f) *uold_f = c.uf[c.cur];
  if (unew_d) *unew_d = c.ud[1 - c.cur];
  if (unew_f) *unew_f = c.uf[1 - c.cur];
  return RH_OK;
}

// Time n back-to-back Godunov steps of a level on device (CUDA events on the
// library stream); dt fixed.  Returns the average milliseconds per launch.
int rh_bench_godunov(int ilevel, int nrep, double gamma, double smallr, double smallc, double dt, double dx,
                     double courant, int slope, int riemann, float* ms_per_step) {
  int rc = check_ready();
  if (rc) return rc;
  Context& c = ctx();
  if (ilevel < c.levelmin || ilevel > c.levelmax || nrep < 1) {
    set_error("rh_bench_godunov: bad level or nrep");
    return RH_EINVAL;
  }
  const double g[3] = {c.gravity[0], c.gravity[1], c.gravity[2]};
  RH_CUDA(cudaEventRecord(c.ev0, c.stream));
  for (int i = 0; i < nrep; ++i) {
    rc = launch_level(ilevel, gamma, smallr, smallc, dt, dx, courant * dx / dt, slope, riemann, g, true);
    if (rc) return rc;
  }
  RH_CUDA(cudaEventRecord(c.ev1, c.stream));
  RH_CUDA(cudaEventSynchronize(c.ev1));
  float ms = 0;
  RH_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
  *ms_per_step = ms / nrep;
  // the timing loop overwrote unew and the level's reduced CFL values
  c.cfl_on_unew[ilevel] = 0;
  c.cfl_on_uold[ilevel] = 0;
  c.unew_written[ilevel] = 0;
  return rh_sync();
}

// CUDA-event timer on the library stream (brackets any sequence of calls).
int rh_timer_start(void) {
  int rc = check_ready(false);
  if (rc) return rc;
  RH_CUDA(cudaEventRecord(ctx().ev0, ctx().stream));
  return RH_OK;
}
int rh_timer_stop(float* ms) {
  int rc = check_ready(false);
  if (rc) return rc;
  Context& c = ctx();
  RH_CUDA(cudaEventRecord(c.ev1, c.stream));
  RH_CUDA(cudaEventSynchronize(c.ev1));
  RH_CUDA(cudaEventElapsedTime(ms, c.ev0, c.ev1));
  return RH_OK;
}

int rh_get_tile(int* txo, int* tyo, int* minb, int* lz) {
  Context& c = ctx();
  if (txo) *txo = c.cfg.txo;
  if (tyo) *tyo = c.cfg.tyo;
  if (minb) *minb = c.cfg.minb;
  if (lz) *lz = c.cfg.lz;
  return RH_OK;
}

int rh_list_tiles(int precision, int* txo, int* tyo, int* minb, int max) {
  return list_tiles(precision, 0, txo, tyo, minb, max);
}

int rh_level_table(int ilevel, int* phdr, long long* poff, int* tab, long long max_entries) {
  int rc = check_ready();
  if (rc) return rc;
  Context& c = ctx();
  if (ilevel < 0 || ilevel > c.levelmax || !c.levels[ilevel].built) {
    set_error("rh_level_table: level %d has no tables", ilevel);
    return RH_EINVAL;
  }
  const LevelTables& T = c.levels[ilevel];
  if (max_entries < T.ntab) {
    set_error("rh_level_table: %lld entries do not fit in %lld", T.ntab, max_entries);
    return RH_EINVAL;
  }
  if (phdr) std::memcpy(phdr, T.phdr.data(), sizeof(int4) * T.phdr.size());
  if (poff) std::memcpy(poff, T.poff.data(), sizeof(long long) * T.poff.size());
  if (tab) {
    RH_CUDA(cudaMemcpyAsync(tab, T.d_ptab, sizeof(int) * T.ntab, cudaMemcpyDeviceToHost, c.stream));
    RH_CUDA(cudaStreamSynchronize(c.stream));
  }
  return RH_OK;
}

int rh_level_ghosts(int ilevel, int* gsrc_oct, unsigned char* gsrc_cf, int* gfather, long long max_ghosts) {
  int rc = check_ready();
  if (rc) return -rc;
  Context& c = ctx();
  if (ilevel < 0 || ilevel > c.levelmax || !c.levels[ilevel].built) {
    set_error("rh_level_ghosts: level %d has no tables", ilevel);
    return -RH_EINVAL;
  }
  const LevelTables& T = c.levels[ilevel];
  const long long n = T.nghost;
  if ((gsrc_oct || gsrc_cf || gfather) && max_ghosts < n) {
    set_error("rh_level_ghosts: %lld ghosts do not fit in %lld", n, max_ghosts);
    return -RH_EINVAL;
  }
  if (n > 0) {
    if (gsrc_oct) RH_CUDA(cudaMemcpy(gsrc_oct, T.d_gsrc_oct, sizeof(int) * 7 * n, cudaMemcpyDeviceToHost));
    if (gsrc_cf) RH_CUDA(cudaMemcpy(gsrc_cf, T.d_gsrc_cf, 7 * n, cudaMemcpyDeviceToHost));
    if (gfather)
      RH_CUDA(cudaMemcpy(gfather, c.d_gfather + (T.gbase - c.ngridmax), sizeof(int2) * n, cudaMemcpyDeviceToHost));
  }
  return (int)n;
}

int rh_coarse_step(const rh_hydro_params* p, double* dt, double* cfl) {
  int rc = check_ready();
  if (rc) return rc;
  Context& c = ctx();
  if (!p || !dt) {
    set_error("rh_coarse_step: null argument");
    return RH_EINVAL;
  }
  const int n3 = c.nsubgrid * c.nsubgrid * c.nsubgrid;
  std::vector<int> lev;
  for (int l = c.levelmin; l <= c.levelmax; ++l)
    if (c.noct[l] > 0) lev.push_back(l);
  auto dxl = [&](int l) { return c.boxlen / std::ldexp(1.0, l); };
  // artificial diffusion (unsplit's cmpdivu/cmpdiff when difmag > 0)
  const bool diffuse = p->difmag > 0.0;
  if (diffuse && (lev.size() != 1 || !diffusion_supported(lev[0]))) {
    set_error("rh_coarse_step: difmag > 0 (cmpdivu/cmpdiff) runs on a mesh of one complete level in FP64 only");
    return RH_EINVAL;
  }
  double step_dt = *dt;
  if (!(step_dt > 0)) {
    // courant_fine of every level queued back to back, one wait for all
    double* h = nullptr;
    if ((rc = cfl_host(&h))) return rc;
    // every level's values left by the previous step for these parameters:
    // one copy of the levels' slots instead of one per level
    bool all_cached = !lev.empty();
    for (int l : lev) {
      const double key[8] = {dxl(l), p->gamma, p->smallr, p->smallc, p->courant_factor,
                             c.gravity[0], c.gravity[1], c.gravity[2]};
      all_cached = all_cached && c.cfl_on_uold[l] && std::equal(key, key + 8, &c.cfl_keys[8 * l]);
    }
    const int l0 = lev.empty() ? 0 : lev.front(), nl = lev.empty() ? 0 : lev.back() - l0 + 1;
    if (all_cached && c.cfl_next_gen == c.cfl_gen && c.cfl_next_l0 == l0 && c.cfl_next_l1 == lev.back()) {
      // copied by the previous call as soon as they were final: no wait
      // for the rest of that step (its restrictions)
      RH_CUDA(cudaEventSynchronize(c.ev_cfl_copied));
      std::copy(c.h_cfl_next + 5 * l0, c.h_cfl_next + 5 * (l0 + nl), h + 5 * l0);
    } else {
      if (all_cached) {
        RH_CUDA(cudaMemcpyAsync(h + 5 * l0, c.d_cfl + 5 * l0, sizeof(double) * 5 * nl, cudaMemcpyDeviceToHost,
                                c.stream));
      } else {
        for (int l : lev) {
          bool queued = false;
          rc = cmpdt_enqueue(c.head[l], c.noct[l], dxl(l), p->gamma, p->smallr, p->smallc, p->courant_factor,
                             c.gravity, h + 5 * l, &queued);
          if (rc) return rc;
        }
      }
      RH_CUDA(cudaStreamSynchronize(c.stream));
    }
    step_dt = 1e300;
    for (int l : lev) {
      const double* v = h + 5 * l;
      const double ldt = std::min(dxl(l) / p->smallc, v[4]);
      if (cfl) {
        double* o = cfl + 5 * (l - c.levelmin);
        o[0] = v[0];
        o[1] = v[1];
        o[2] = v[2];
        o[3] = 0.0;
        o[4] = ldt;
      }
      step_dt = std::min(step_dt, ldt);
    }
  }
  // Every level's interpolated ghost octs, prolonged ahead on the side stream:
  // a level's ghosts come from the coarser level's uold, which no Godunov step
  // of this coarse step changes before that level's own step (set_uold and
  // the restrictions of level l-1 follow level l's step), so they overlap the
  // set_unew copy and the finer levels' steps.
  // whatever happens below, no level is left marked as prolonged ahead
  struct ClearProlonged {
    ~ClearProlonged() { std::fill(ctx().prolonged.begin(), ctx().prolonged.end(), 0); }
  } clear_prolonged;
  if (lev.size() > 1) {
    if (c.ev_prolong.size() < (size_t)(c.levelmax + 1)) {
      for (size_t k = c.ev_prolong.size(); k < (size_t)(c.levelmax + 1); ++k) {
        cudaEvent_t e;
        RH_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        c.ev_prolong.push_back(e);
      }
    }
    c.prolonged.assign(c.levelmax + 1, 0);
    RH_CUDA(cudaEventRecord(c.ev_side_start, c.stream));
    RH_CUDA(cudaStreamWaitEvent(c.side, c.ev_side_start, 0));
    for (size_t i = lev.size(); i-- > 0;) {
      const int l = lev[i];
      if (!c.levels[l].built || c.levels[l].nghost == 0) continue;
      if ((rc = prolong_ghosts(l, p->smallr, c.side))) return rc;
      RH_CUDA(cudaEventRecord(c.ev_prolong[l], c.side));
      c.prolonged[l] = 1;
    }
  }
  // Several levels that together hold every oct of the state: every level's
  // step reads only uold (its own level and, for its ghosts, the coarser
  // one) and writes its own cells of unew as uold plus its flux differences,
  // so the levels run at once on separate streams and no set_unew copy is
  // needed; the face contributions to father cells (±F/8) go to slots, added
  // to the fathers' unew afterwards in a fixed order (the deterministic
  // coarse-fine update, always on here); one swap of the state buffers then
  // stands for the per-level set_uold copies, and the restrictions follow,
  // finest first.  Otherwise level by level.
  long long covered = 0;
  for (int l : lev) covered += c.noct[l];
  const bool swap_all = lev.size() > 1 && covered == c.ngridmax;
  if (swap_all) {
    const long long nghost_all = c.nstate - c.ngridmax;
    if (nghost_all > 0 && !c.d_gface_all) {
      // zeroed once: the slots a step writes are fixed by the mesh, each
      // written in full every step, and the others stay zero
      RH_CUDA(cudaMalloc(&c.d_gface_all, sizeof(double) * 120 * nghost_all));
      RH_CUDA(cudaMemsetAsync(c.d_gface_all, 0, sizeof(double) * 120 * nghost_all, c.stream));
      // the father cells of every level's ghosts, and room for the gathers' CFL partials
      const size_t mask_bytes = ((size_t)c.ngridmax + 3) / 4 * 4;
      RH_CUDA(cudaMalloc(&c.d_cflskip, mask_bytes));
      RH_CUDA(cudaMemsetAsync(c.d_cflskip, 0, mask_bytes, c.stream));
      long long nblk = 0;
      for (int l : lev) {
        const LevelTables& T = c.levels[l];
        if (T.nghost == 0) continue;
        mark_fathers_kernel<<<(unsigned)((T.nghost + 255) / 256), 256, 0, c.stream>>>(
            c.d_gfather + (T.gbase - c.ngridmax), T.nghost, reinterpret_cast<unsigned*>(c.d_cflskip));
        RH_CUDA(cudaGetLastError());
        nblk += (T.nghost + kGatherGhosts - 1) / kGatherGhosts;
      }
      RH_CUDA(cudaMalloc(&c.d_gcfl, sizeof(double) * 5 * (size_t)std::max(1LL, nblk)));
    }
    for (auto* evs : {&c.ev_level, &c.ev_gather}) {
      for (size_t k = evs->size(); k < (size_t)(c.levelmax + 1); ++k) {
        cudaEvent_t e;
        RH_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        evs->push_back(e);
      }
    }
    RH_CUDA(cudaEventRecord(c.ev_side_start, c.stream));
    for (auto s : c.lev_stream) RH_CUDA(cudaStreamWaitEvent(s, c.ev_side_start, 0));
    std::vector<char> fused(c.levelmax + 1, 0), corrected(c.levelmax + 1, 0), gathered(c.levelmax + 3, 0);
    std::vector<cudaStream_t> lst(c.levelmax + 1, c.stream);  // each level's stream
    for (int l : lev)
      if (l > c.levelmin && c.levels[l].nghost > 0) corrected[l - 1] = 1;
    // coarsest level first: it waits for no prolongation, and the complete
    // coarse level's deep pencils are the longest kernel of the step
    for (size_t i = 0; i < lev.size(); ++i) {
      const int l = lev[i];
      const int j = (int)(lev.size() - 1 - i);  // 0: the finest level, on the library stream
      const double dx = dxl(l);
      const double* key = &c.cfl_keys[8 * l];
      fused[l] = key[0] == dx && key[1] == p->gamma && key[2] == p->smallr && key[5] == c.gravity[0] &&
                 key[6] == c.gravity[1] && key[7] == c.gravity[2] && key[3] == p->smallc;
      cudaStream_t st = j == 0 ? c.stream : c.lev_stream[(j - 1) % 3];
      lst[l] = st;
      // a level whose father cells the gathers correct leaves them to the
      // gathers' CFL and has its partials reduced together with theirs
      const bool merge = fused[l] && corrected[l] && c.d_cflskip;
      const LevelSlots S{c.d_gface_all, c.ngridmax, st, merge ? c.d_cflskip : nullptr, merge};
      rc = launch_level(l, p->gamma, p->smallr, p->smallc, step_dt, dx, p->courant_factor * dx / step_dt,
                        p->slope_type, p->riemann, c.gravity, fused[l] != 0, false, nullptr, &S);
      if (rc) return rc;
      RH_CUDA(cudaEventRecord(c.ev_level[l], st));
    }
    // The coarse-fine corrections of each level with ghost octs, into the
    // coarser level's unew: on the coarser level's stream (after its own
    // pencils) once the level's pencils have filled the slots, so that a
    // gather whose two levels are done runs while larger levels still step.
    long long goff = 0;
    for (int l : lev) {
      const LevelTables& T = c.levels[l];
      if (T.nghost == 0) continue;
      const double* slots = c.d_gface_all + (size_t)(T.gbase - c.ngridmax) * 120;
      const int2* fathers = c.d_gfather + (T.gbase - c.ngridmax);
      const int lf = l - 1;  // the fathers' level
      const cudaStream_t gs = lst[lf];
      RH_CUDA(cudaStreamWaitEvent(gs, c.ev_level[l], 0));
      if (lf >= c.levelmin && fused[lf] && corrected[lf] && c.d_cflskip) {
        // the father level's CFL constants, as launch_level formed them
        const double dxf = dxl(lf);
        const double* lkey = &c.cfl_keys[8 * lf];
        const double smax_cap = p->courant_factor * dxf / step_dt;
        const double courant = lkey[4] > 0 ? lkey[4] : smax_cap * step_dt / dxf;
        const CflConst C = make_cfl(dxf, p->gamma, p->smallr, p->smallc, courant, c.gravity);
        const double vol = dxf * dxf * dxf;
        const long long nb = (T.nghost + kGatherGhosts - 1) / kGatherGhosts;
        double* part = c.d_gcfl + 5 * goff;
        if (c.precision == RH_PREC_FP64)
          coarse_gather_cfl_kernel<<<(unsigned)nb, kGatherThreads, 0, gs>>>(
              slots, T.nghost, fathers, c.d_refmask, c.ud[1 - c.cur], C, vol, part);
        else
          coarse_gather_cfl_f32_kernel<<<(unsigned)nb, kGatherThreads, 0, gs>>>(
              slots, T.nghost, fathers, c.d_refmask, c.uf[1 - c.cur], c.ud[1 - c.cur], C, vol, part);
        RH_CUDA(cudaGetLastError());
        const LevelTables& F = c.levels[lf];
        reduce_partials_pair_kernel<<<1, 1024, 0, gs>>>(F.d_cfl_partial, F.npencil, part, nb, C.cdx_smallc,
                                                        c.d_cfl + 5 * lf);
        c.cfl_gen++;
        RH_CUDA(cudaGetLastError());
        goff += nb;
      } else {
        const unsigned nb = (unsigned)((T.nghost * 5ll + 255) / 256);
        if (c.precision == RH_PREC_FP64)
          coarse_gather_kernel<<<nb, 256, 0, gs>>>(slots, T.nghost, fathers, c.ud[1 - c.cur]);
        else
          coarse_gather_f32_kernel<<<nb, 256, 0, gs>>>(slots, T.nghost, fathers, c.uf[1 - c.cur],
                                                       c.ud[1 - c.cur]);
        RH_CUDA(cudaGetLastError());
      }
      RH_CUDA(cudaEventRecord(c.ev_gather[l], gs));
      gathered[l] = 1;
    }
    c.cur = 1 - c.cur;
    for (int l : lev) {
      c.unew_pending[l] = 0;
      c.unew_written[l] = 0;
      c.unew_copied[l] = 0;
      // every fused level's courant_fine values are complete: a corrected
      // level's own partials plus its corrected cells' from the gathers
      c.cfl_on_uold[l] = fused[l];
      c.cfl_on_unew[l] = 0;
    }
    // every level's courant_fine values of the new state are final once its
    // pencils and its gather's reduction ran: copy them to the host now, so
    // that the next call's dt need not wait for the restrictions
    bool all_fused = true;
    for (int l : lev) all_fused = all_fused && fused[l];
    if (all_fused) {
      for (int l : lev) {
        RH_CUDA(cudaStreamWaitEvent(c.cfl_copy, c.ev_level[l], 0));
        if (gathered[l + 1]) RH_CUDA(cudaStreamWaitEvent(c.cfl_copy, c.ev_gather[l + 1], 0));
      }
      const int l0 = lev.front(), nl = lev.back() - l0 + 1;
      RH_CUDA(cudaMemcpyAsync(c.h_cfl_next + 5 * l0, c.d_cfl + 5 * l0, sizeof(double) * 5 * nl,
                              cudaMemcpyDeviceToHost, c.cfl_copy));
      RH_CUDA(cudaEventRecord(c.ev_cfl_copied, c.cfl_copy));
      c.cfl_next_gen = c.cfl_gen;
      c.cfl_next_l0 = l0;
      c.cfl_next_l1 = lev.back();
    }
    // The restrictions, finest first, on the library stream (the finest
    // level's): l+1 -> l writes level l's refined cells, which level l's
    // pencils write too, and reads level l+1's cells once they are final
    // (its own step, the gather of level l+2's corrections into it and the
    // restriction l+2 -> l+1 before this one).
    for (size_t i = lev.size() - 1; i-- > 0;) {
      const int l = lev[i];
      if (l + 1 <= c.levelmax && c.noct[l + 1] > 0) {
        RH_CUDA(cudaStreamWaitEvent(c.stream, c.ev_level[l], 0));
        RH_CUDA(cudaStreamWaitEvent(c.stream, c.ev_level[l + 1], 0));
        if (gathered[l + 2]) RH_CUDA(cudaStreamWaitEvent(c.stream, c.ev_gather[l + 2], 0));
        rc = upload_on(c.head[l + 1], c.noct[l + 1], p->interpol_var == 1 ? 1 : 0, p->smallr, c.stream);
        if (rc) return rc;
      }
    }
    // the whole step ordered before the library stream's next work
    for (int l : lev) {
      RH_CUDA(cudaStreamWaitEvent(c.stream, c.ev_level[l], 0));
      if (gathered[l]) RH_CUDA(cudaStreamWaitEvent(c.stream, c.ev_gather[l], 0));
    }
    *dt = step_dt;
    if (c.state_check) return check_all_levels();
    return RH_OK;
  }
  for (int l : lev)
    if ((rc = rh_set_unew(c.head[l], c.noct[l]))) return rc;
  for (size_t i = lev.size(); i-- > 0;) {
    const int l = lev[i];
    const double dx = dxl(l);
    rc = rh_godunov((c.head[l] - 1) / n3 + 1, c.noct[l] / n3, c.ngridmax, l, c.levelmin, c.levelmax, p->gamma,
                    p->smallr, p->smallc * p->smallc, step_dt, dx, p->courant_factor * dx / step_dt, p->slope_type,
                    p->riemann, c.gravity);
    if (rc) return rc;
    if (diffuse) {
      // the diffusive face fluxes added to unew; the fused courant_fine
      // values of the pencils no longer describe it
      if ((rc = diffuse_level(l, step_dt, dx, p->difmag, p->smallr, c.gravity))) return rc;
      c.cfl_on_unew[l] = 0;
    }
    if ((rc = rh_set_uold(c.head[l], c.noct[l]))) return rc;
    if (i + 1 < lev.size() && l + 1 <= c.levelmax && c.noct[l + 1] > 0) {
      rc = rh_upload(c.head[l + 1], c.noct[l + 1], p->interpol_var == 1 ? 1 : 0, p->gamma, p->smallr,
                     p->smallc * p->smallc);
      if (rc) return rc;
    }
  }
  // every level's courant_fine values of the new state fused into its step:
  // on their way to the host before the next call asks for them
  bool all_fused = !lev.empty();
  for (int l : lev) all_fused = all_fused && c.cfl_on_uold[l];
  if (all_fused) {
    const int l0 = lev.front(), nl = lev.back() - l0 + 1;
    RH_CUDA(cudaEventRecord(c.ev_cfl_ready, c.stream));
    RH_CUDA(cudaStreamWaitEvent(c.cfl_copy, c.ev_cfl_ready, 0));
    RH_CUDA(cudaMemcpyAsync(c.h_cfl_next + 5 * l0, c.d_cfl + 5 * l0, sizeof(double) * 5 * nl,
                            cudaMemcpyDeviceToHost, c.cfl_copy));
    RH_CUDA(cudaEventRecord(c.ev_cfl_copied, c.cfl_copy));
    c.cfl_next_gen = c.cfl_gen;
    c.cfl_next_l0 = l0;
    c.cfl_next_l1 = lev.back();
  }
  *dt = step_dt;
  if (c.state_check) return check_all_levels();  // the reference's gpu_debug scan after set_uold
  return RH_OK;
}

int rh_set_deterministic(int on) {
  int rc = check_ready(false);
  if (rc) return rc;
  ctx().deterministic = on ? 1 : 0;
  return RH_OK;
}

int rh_set_table_builder(int on_device) {
  int rc = check_ready(false);
  if (rc) return rc;
  ctx().table_builder = on_device ? 1 : 0;
  return RH_OK;
}

int rh_level_info(int ilevel, int* npencil, long long* table_entries) {
  int rc = check_ready();
  if (rc) return rc;
  Context& c = ctx();
  if (ilevel < 0 || ilevel > c.levelmax) return RH_EINVAL;
  if (npencil) *npencil = c.levels[ilevel].npencil;
  if (table_entries) *table_entries = c.levels[ilevel].ntab;
  return RH_OK;
}

}  // extern "C"
