// rh_batch.cu — the batch runtime: device pool, problem admission by HBM
// footprint, device-side initial conditions, the persistent step kernel's
// work list, per-problem CFL/time reduction and CUDA-graph replay.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "ramses_hydro_batch.h"
#include "ramses_hydro_io.h"
#include "rh_batch.cuh"
#include "rh_check.cuh"
#include "rh_internal.h"

namespace rh {

struct BatchReg {
  BatchKey k;
  BatchLaunchFn fn;
  const void* func;
  size_t smem;
  int threads;
};
static std::vector<BatchReg>& batch_registry() {
  static std::vector<BatchReg> r;
  return r;
}
void register_batch_launcher(const BatchKey& k, BatchLaunchFn fn, const void* func, size_t smem, int threads) {
  batch_registry().push_back({k, fn, func, smem, threads});
}
static const BatchReg* find_batch(int prec, int txo, int tyo, int minb, int slope, int riemann) {
  for (auto& e : batch_registry())
    if (e.k.prec == prec && e.k.txo == txo && e.k.tyo == tyo && e.k.minb == minb && e.k.slope == slope &&
        e.k.riemann == riemann)
      return &e;
  return nullptr;
}

namespace {

struct HostProb {
  bool used = false;
  rh_batch_problem p;
  long long oct0 = 0, noct = 0;
};

struct Batch {
  bool inited = false;
  int precision = RH_PREC_FP64, slope = 2, riemann = 3;
  TileCfg cfg{8, 4, 2, 16};
  long long pool_octs = 0;
  int parity = 0;
  double* ud[2] = {nullptr, nullptr};
  float* uf[2] = {nullptr, nullptr};
  std::vector<std::pair<long long, long long>> free_list;  // [start, end) in octs
  std::vector<HostProb> probs;
  int cap = 0;
  // device problem tables
  BatchProb* d_prob = nullptr;
  int* d_done = nullptr;
  int* d_nstep = nullptr;
  int* d_cur = nullptr;          // pool buffer holding each problem's current state
  double* d_dt = nullptr;
  double* d_t = nullptr;
  double* d_tot = nullptr;       // [cap][5]
  int* d_order = nullptr;
  long long* d_woff = nullptr;
  double* d_partial = nullptr;
  long long partial_cap = 0;
  unsigned long long* d_counter = nullptr;
  int nslot = 0;
  long long nwork = 0;
  bool dirty = true;             // work list / graph must be rebuilt
  const void* occ_reg = nullptr; // kernel whose occupancy occ_per_sm holds
  int occ_per_sm = 0;
  int plane2d = 1;               // 2D problems on the plane tile body
  cudaGraphExec_t graph = nullptr;
  int graph_parity = 0;
  int nblocks = 0;
  double* d_tmp = nullptr;       // initial-CFL partials
  long long tmp_cap = 0;
  // state check after each step (rh_batch_set_state_check)
  int check = 0;
  int* d_bad = nullptr;          // [cap] OR of the check's bits per problem
  long long* d_coff = nullptr;   // [cap+1] first check block of each work-list slot
  long long nchunk = 0;          // check blocks (32 octs each) over the work list
};

Batch& B() {
  static Batch b;
  return b;
}

int pool_bytes_per_oct(int prec) { return prec == RH_PREC_FP64 ? 2 * 320 : 2 * 192; }

// ---- kernels ---------------------------------------------------------------

// Initial conditions of one problem (row-major octs).
__global__ void batch_ic_kernel(rh_batch_ic ic, BatchProb P, double* ud, float* uf, int fp32, const double* host) {
  const long long noct = (long long)(P.ncx >> 1) * (P.ncy >> 1) * (P.ncz >> 1);
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= noct * 8) return;
  const long long oct = i >> 3;
  const int cell = (int)(i & 7);
  const int nxo = P.ncx >> 1, nyo = P.ncy >> 1;
  const int ox = (int)(oct % nxo), oy = (int)((oct / nxo) % nyo), oz = (int)(oct / ((long long)nxo * nyo));
  const int c[3] = {2 * ox + (cell & 1), 2 * oy + ((cell >> 1) & 1), 2 * oz + ((cell >> 2) & 1)};
  const int ncell[3] = {P.ncx, P.ncy, P.ncz};
  double u[5];
  if (ic.kind == RH_IC_HOST) {
    for (int v = 0; v < 5; ++v) u[v] = host[oct * 40 + v * 8 + cell];
  } else {
    double q[5];
    if (ic.kind == RH_IC_SPLIT) {
      const bool left = c[ic.axis] < ncell[ic.axis] / 2;
      for (int v = 0; v < 5; ++v) q[v] = left ? ic.left[v] : ic.right[v];
    } else {
      double r2 = 0.0;
      for (int d = 0; d < P.ndim; ++d) {
        const double x = (c[d] + 0.5) * P.dx - ic.centre[d];
        r2 += x * x;
      }
      for (int v = 0; v < 5; ++v) q[v] = ic.ambient[v];
      if (r2 <= ic.radius * ic.radius * (1.0 + 1e-12)) q[4] = ic.p_in;
    }
    u[0] = q[0];
    u[1] = q[0] * q[1];
    u[2] = q[0] * q[2];
    u[3] = q[0] * q[3];
    u[4] = q[4] / (P.gamma - 1.0) + 0.5 * q[0] * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  }
  const long long o = P.oct0 + oct;
  if (!fp32) {
    for (int v = 0; v < 5; ++v) ud[o * 40 + v * 8 + cell] = u[v];
  } else {
    for (int v = 0; v < 4; ++v) uf[o * kBulkF + v * 8 + cell] = (float)u[v];
    ud[o * kBulkD + cell] = u[4];
  }
}

// courant_fine of one problem's state: per-block partials.
__global__ void batch_cfl_kernel(BatchProb P, const double* ud, const float* uf, int fp32, double* partial) {
  __shared__ double red[32][4];
  const long long noct = (long long)(P.ncx >> 1) * (P.ncy >> 1) * (P.ncz >> 1);
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  LevelArgs A;
  batch_level(P, 1.0, nullptr, A);
  CflAcc acc;
  if (i < noct * 8) {
    const long long o = P.oct0 + (i >> 3);
    const int cell = (int)(i & 7);
    if (!fp32) {
      const double* p = ud + o * 40 + cell;
      acc.add(p[0], p[8], p[16], p[24], p[32], A);
    } else {  // the FP32-bulk form the fused epilogue of the problem's steps uses
      const float* p = uf + o * kBulkF + cell;
      acc.add_bulk(p[0], p[8], p[16], p[24], ud[o * kBulkD + cell], A);
      acc.scale_bulk(A.vol);
    }
  }
  double v[4] = {acc.mass, acc.ekin, acc.eint, acc.dt(A.cfl)};
  for (int off = 16; off > 0; off >>= 1) {
    v[0] += __shfl_down_sync(0xffffffffu, v[0], off);
    v[1] += __shfl_down_sync(0xffffffffu, v[1], off);
    v[2] += __shfl_down_sync(0xffffffffu, v[2], off);
    const double q = __shfl_down_sync(0xffffffffu, v[3], off);
    v[3] = q < v[3] ? q : v[3];
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { red[w][0] = v[0]; red[w][1] = v[1]; red[w][2] = v[2]; red[w][3] = v[3]; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0, c = 0, d = 1e300;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      a += red[k][0]; b += red[k][1]; c += red[k][2];
      d = red[k][3] < d ? red[k][3] : d;
    }
    double* out = partial + blockIdx.x * 5ll;
    out[0] = a; out[1] = b; out[2] = c; out[3] = 0.0; out[4] = d;
  }
}

// dt of the next step from a courant_fine result: min(dx/smallc, cell dt)
// (newdt_fine.f90:71,103-108), cut so the problem lands on t_end.
__device__ __forceinline__ double next_dt(const BatchProb& P, double t, double cfl_dt) {
  double dt = P.dx / P.smallc;
  dt = cfl_dt < dt ? cfl_dt : dt;
  if (P.t_end > 0.0 && t + dt > P.t_end) dt = P.t_end - t;
  return dt;
}

// Device state check of the problems stepped this step (done == 0 before the
// reduction): block b checks 32 octs of the problem in slot s with
// coff[s] <= b < coff[s+1], in the pool buffer the step wrote; the bits of
// cell_state_bits are OR-ed into bad[id].
__global__ void batch_check_kernel(const BatchProb* __restrict__ prob, const int* __restrict__ order,
                                   const long long* __restrict__ coff, int nslot, const int* __restrict__ done,
                                   const double* ud, const float* uf, int fp32, int* __restrict__ bad) {
  const long long blk = blockIdx.x;
  int lo = 0, hi = nslot - 1;
  while (lo < hi) {  // the last slot whose first block is <= blk
    const int mid = (lo + hi + 1) >> 1;
    if (coff[mid] <= blk) lo = mid;
    else hi = mid - 1;
  }
  const int id = order[lo];
  if (done[id]) return;
  const BatchProb& P = prob[id];
  const long long noct = (long long)(P.ncx >> 1) * (P.ncy >> 1) * (P.ncz >> 1);
  const long long o = (blk - coff[lo]) * 32 + (threadIdx.x >> 3);
  if (o >= noct) return;
  const unsigned bits = load_cell_bits(ud, uf, fp32, P.oct0 + o, (int)(threadIdx.x & 7));
  if (bits) atomicOr(&bad[id], (int)bits);
}

// Reduce the partials of n blocks into totals and (optionally) advance time.
__device__ void reduce_block(const double* partial, long long n, double* out4) {
  __shared__ double red[256][4];
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
      const double o = red[threadIdx.x + s][3];
      red[threadIdx.x][3] = o < red[threadIdx.x][3] ? o : red[threadIdx.x][3];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out4[0] = red[0][0]; out4[1] = red[0][1]; out4[2] = red[0][2]; out4[3] = red[0][3];
  }
}

// Initial CFL of one problem (no time advance).
__global__ void batch_init_dt_kernel(BatchProb P, int id, const double* partial, long long n, double* dt,
                                     double* tot) {
  __shared__ double r4[4];
  reduce_block(partial, n, r4);
  if (threadIdx.x == 0) {
    dt[id] = next_dt(P, 0.0, r4[3]);
    double* o = tot + id * 5ll;
    o[0] = r4[0]; o[1] = r4[1]; o[2] = r4[2]; o[3] = 0.0; o[4] = r4[3];
  }
}

// After a batch step: per problem, reduce its pencils' partials (fixed
// order), advance t and the step count, set the next dt and the done flag.
__global__ void batch_reduce_kernel(const BatchProb* prob, const int* order, const long long* woff,
                                    const double* partial, int* done, int* nstep, int* cur, double* dt, double* t,
                                    double* tot, unsigned long long* counter, int parity, const int* bad) {
  const int slot = blockIdx.x;
  const int id = order[slot];
  if (slot == 0 && threadIdx.x == 0) *counter = 0ull;
  if (done[id]) return;
  __shared__ double r4[4];
  reduce_block(partial + woff[slot] * 5, woff[slot + 1] - woff[slot], r4);
  if (threadIdx.x == 0) {
    const BatchProb P = prob[id];
    const double tn = t[id] + dt[id];
    t[id] = tn;
    const int ns = nstep[id] + 1;
    nstep[id] = ns;
    cur[id] = 1 - parity;
    double* o = tot + id * 5ll;
    o[0] = r4[0]; o[1] = r4[1]; o[2] = r4[2]; o[3] = 0.0; o[4] = r4[3];
    const bool fin = (P.t_end > 0.0 && tn >= P.t_end * (1.0 - 1e-12)) || (P.max_steps > 0 && ns >= P.max_steps);
    done[id] = bad[id] ? 2 : (fin ? 1 : 0);  // 2: stopped by the state check
    dt[id] = next_dt(P, tn, r4[3]);
  }
}

// ---- host helpers ------------------------------------------------------------

int alloc_octs(long long n, long long* start) {
  Batch& b = B();
  for (size_t i = 0; i < b.free_list.size(); ++i) {
    auto& f = b.free_list[i];
    if (f.second - f.first >= n) {
      *start = f.first;
      f.first += n;
      if (f.first == f.second) b.free_list.erase(b.free_list.begin() + i);
      return RH_OK;
    }
  }
  return RH_ENOMEM;
}

void free_octs(long long start, long long n) {
  Batch& b = B();
  b.free_list.push_back({start, start + n});
  std::sort(b.free_list.begin(), b.free_list.end());
  std::vector<std::pair<long long, long long>> merged;
  for (auto& f : b.free_list) {
    if (!merged.empty() && merged.back().second == f.first) merged.back().second = f.second;
    else merged.push_back(f);
  }
  b.free_list.swap(merged);
}

BatchProb make_prob(const rh_batch_problem& p, long long oct0) {
  Batch& b = B();
  BatchProb P;
  P.oct0 = oct0;
  P.ncx = p.n[0];
  P.ncy = p.n[1];
  P.ncz = p.n[2];
  for (int i = 0; i < 6; ++i) P.btype[i] = p.bound_type[i];
  for (int d = 0; d < 3; ++d) P.periodic[d] = p.bound_type[2 * d] == RH_BOUND_PERIODIC ? 1 : 0;
  if (p.ndim == 2) P.periodic[2] = 1;
  P.ndim = p.ndim;
  P.tx = (p.n[0] / 2 + b.cfg.txo - 1) / b.cfg.txo;
  P.ty = (p.n[1] / 2 + b.cfg.tyo - 1) / b.cfg.tyo;
  P.tz = (p.n[2] / 2 + b.cfg.lz - 1) / b.cfg.lz;
  // 2D problems on the plane path: one work item per kPlaneGroup tile bodies
  // along y (FP32-bulk tile bodies take two tile rows, one per lane)
  if (b.plane2d && p.ndim == 2 && p.n[2] == 2 && P.periodic[2]) {
    const int bodies = b.precision == RH_PREC_FP32_BULK ? (P.ty + 1) / 2 : P.ty;
    P.ty = (bodies + kPlaneGroup - 1) / kPlaneGroup;
  }
  P.dx = p.dx;
  P.gamma = p.gamma;
  P.smallr = p.smallr;
  P.smallc = p.smallc;
  P.courant = p.courant_factor;
  P.t_end = p.t_end;
  P.max_steps = p.max_steps;
  return P;
}

// The state check of the step of the given parity (its new state is in pool
// buffer 1 - parity), when switched on.
void check_step(int parity) {
  Batch& b = B();
  if (!b.check || b.nchunk == 0) return;
  batch_check_kernel<<<(unsigned)b.nchunk, 256, 0, ctx().stream>>>(
      b.d_prob, b.d_order, b.d_coff, b.nslot, b.d_done, b.ud[1 - parity], b.uf[1 - parity],
      b.precision == RH_PREC_FP32_BULK ? 1 : 0, b.d_bad);
}

// Rebuild the work list (largest problems first) and the step graph.
int rebuild() {
  Batch& b = B();
  Context& c = ctx();
  RH_CUDA(cudaStreamSynchronize(c.stream));  // the tables below are read by steps in flight
  std::vector<int> ids;
  for (int i = 0; i < b.cap; ++i)
    if (b.probs[i].used) ids.push_back(i);
  std::sort(ids.begin(), ids.end(), [&](int x, int y) { return b.probs[x].noct > b.probs[y].noct; });
  std::vector<long long> woff(ids.size() + 1, 0);
  std::vector<BatchProb> probs(b.cap);
  for (int i = 0; i < b.cap; ++i)
    if (b.probs[i].used) probs[i] = make_prob(b.probs[i].p, b.probs[i].oct0);
  for (size_t s = 0; s < ids.size(); ++s) {
    const BatchProb& P = probs[ids[s]];
    woff[s + 1] = woff[s] + (long long)P.tx * P.ty * P.tz;
  }
  b.nslot = (int)ids.size();
  b.nwork = woff.back();
  std::vector<long long> coff(ids.size() + 1, 0);
  for (size_t s = 0; s < ids.size(); ++s) coff[s + 1] = coff[s] + (b.probs[ids[s]].noct + 31) / 32;
  b.nchunk = coff.back();
  RH_CUDA(cudaMemcpyAsync(b.d_coff, coff.data(), sizeof(long long) * coff.size(), cudaMemcpyHostToDevice,
                          c.stream));
  RH_CUDA(cudaMemcpyAsync(b.d_prob, probs.data(), sizeof(BatchProb) * b.cap, cudaMemcpyHostToDevice, c.stream));
  if (!ids.empty())
    RH_CUDA(cudaMemcpyAsync(b.d_order, ids.data(), sizeof(int) * ids.size(), cudaMemcpyHostToDevice, c.stream));
  RH_CUDA(cudaMemcpyAsync(b.d_woff, woff.data(), sizeof(long long) * woff.size(), cudaMemcpyHostToDevice, c.stream));
  RH_CUDA(cudaStreamSynchronize(c.stream));  // the host vectors above are locals
  if (b.nwork > b.partial_cap) {
    cudaFree(b.d_partial);
    b.d_partial = nullptr;
    const long long want = std::max(b.nwork, 2 * b.partial_cap);  // grow geometrically: fewer reallocations
    RH_CUDA(cudaMalloc(&b.d_partial, sizeof(double) * 5 * want));
    b.partial_cap = want;
    if (b.graph) {  // the captured steps point at the old buffer
      cudaGraphExecDestroy(b.graph);
      b.graph = nullptr;
    }
  }
  const BatchReg* reg = find_batch(b.precision, b.cfg.txo, b.cfg.tyo, b.cfg.minb, b.slope, b.riemann);
  if (!reg) {
    set_error("no batch kernel for tile %dx%d minb %d slope %d riemann %d", b.cfg.txo, b.cfg.tyo, b.cfg.minb,
              b.slope, b.riemann);
    return RH_EINVAL;
  }
  if (reg != b.occ_reg) {
    RH_CUDA(cudaFuncSetAttribute(reg->func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)reg->smem));
    RH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b.occ_per_sm, reg->func, reg->threads, reg->smem));
    b.occ_reg = reg;
  }
  b.nblocks = std::max(1, b.occ_per_sm) * c.sm_count;
  if (b.nwork > 0 && b.nwork < b.nblocks) b.nblocks = (int)b.nwork;
  // graph of two steps (parity p, then 1-p), each: persistent kernel + reduction;
  // an existing executable graph is updated in place when the topology allows
  if (b.nslot == 0 && b.graph) {
    cudaGraphExecDestroy(b.graph);
    b.graph = nullptr;
  }
  if (b.nslot > 0) {
    cudaGraph_t g;
    RH_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
    for (int h = 0; h < 2; ++h) {
      const int par = (b.parity + h) & 1;
      BatchArgs A{b.d_prob, b.d_order, b.d_woff, b.nslot, b.nwork, b.cfg.txo, b.cfg.tyo, b.cfg.lz, b.d_counter,
                  b.d_done, b.d_dt, b.d_partial, {b.ud[0], b.ud[1]}, {b.uf[0], b.uf[1]}, c.d_err,
                  b.plane2d};
      cudaError_t e = reg->fn(A, par, b.nblocks, c.stream);
      if (e != cudaSuccess) {
        cudaStreamEndCapture(c.stream, &g);
        return cuda_fail(e, "batch step capture");
      }
      check_step(par);
      batch_reduce_kernel<<<b.nslot, 256, 0, c.stream>>>(b.d_prob, b.d_order, b.d_woff, b.d_partial, b.d_done,
                                                         b.d_nstep, b.d_cur, b.d_dt, b.d_t, b.d_tot, b.d_counter,
                                                         par, b.d_bad);
    }
    RH_CUDA(cudaStreamEndCapture(c.stream, &g));
    bool updated = false;
    if (b.graph) {
      cudaGraphExecUpdateResultInfo info;
      updated = cudaGraphExecUpdate(b.graph, g, &info) == cudaSuccess;
      if (!updated) {
        cudaGetLastError();  // clear the update failure
        cudaGraphExecDestroy(b.graph);
        b.graph = nullptr;
      }
    }
    if (!updated) RH_CUDA(cudaGraphInstantiate(&b.graph, g, 0));
    cudaGraphDestroy(g);
    b.graph_parity = b.parity;
  }
  b.dirty = false;
  return RH_OK;
}

}  // namespace
}  // namespace rh

using namespace rh;

extern "C" {

int rh_batch_init(int precision, int slope, int riemann, long long pool_octs) {
  Context& c = ctx();
  if (!c.inited) {
    set_error("rh_init has not been called");
    return RH_ESTATE;
  }
  Batch& b = B();
  if (b.inited) rh_batch_free();
  if ((precision != RH_PREC_FP64 && precision != RH_PREC_FP32_BULK) || slope < 0 || slope > 2 || riemann < 1 ||
      riemann > 3 || pool_octs < 1) {
    set_error("rh_batch_init: bad precision/slope/riemann/pool size");
    return RH_EINVAL;
  }
  b.precision = precision;
  b.slope = slope;
  b.riemann = riemann;
  b.pool_octs = pool_octs;
  // default tile per precision: the fastest of the autotuner's sweep on the
  // uneven 3D ensemble and on mixed 2D/3D serving
  b.cfg = precision == RH_PREC_FP32_BULK ? TileCfg{7, 7, 2, 32} : TileCfg{8, 4, 2, 32};
  b.cap = 4096;
  for (int i = 0; i < 2; ++i) {
    if (precision == RH_PREC_FP64) {
      RH_CUDA(cudaMalloc(&b.ud[i], sizeof(double) * 40 * pool_octs));
    } else {
      RH_CUDA(cudaMalloc(&b.uf[i], (size_t)kBulkBytes * pool_octs));
      b.ud[i] = reinterpret_cast<double*>(b.uf[i]) + kBulkE;
    }
  }
  RH_CUDA(cudaMalloc(&b.d_prob, sizeof(BatchProb) * b.cap));
  RH_CUDA(cudaMalloc(&b.d_done, sizeof(int) * b.cap));
  RH_CUDA(cudaMalloc(&b.d_nstep, sizeof(int) * b.cap));
  RH_CUDA(cudaMalloc(&b.d_cur, sizeof(int) * b.cap));
  RH_CUDA(cudaMalloc(&b.d_dt, sizeof(double) * b.cap));
  RH_CUDA(cudaMalloc(&b.d_t, sizeof(double) * b.cap));
  RH_CUDA(cudaMalloc(&b.d_tot, sizeof(double) * 5 * b.cap));
  RH_CUDA(cudaMalloc(&b.d_order, sizeof(int) * b.cap));
  RH_CUDA(cudaMalloc(&b.d_woff, sizeof(long long) * (b.cap + 1)));
  RH_CUDA(cudaMalloc(&b.d_counter, sizeof(unsigned long long)));
  RH_CUDA(cudaMalloc(&b.d_bad, sizeof(int) * b.cap));
  RH_CUDA(cudaMalloc(&b.d_coff, sizeof(long long) * (b.cap + 1)));
  RH_CUDA(cudaMemset(b.d_bad, 0, sizeof(int) * b.cap));
  RH_CUDA(cudaMemset(b.d_counter, 0, sizeof(unsigned long long)));
  RH_CUDA(cudaMemset(b.d_done, 0, sizeof(int) * b.cap));
  b.probs.assign(b.cap, HostProb());
  b.free_list = {{0, pool_octs}};
  b.parity = 0;
  b.dirty = true;
  b.inited = true;
  return RH_OK;
}

int rh_batch_free(void) {
  Batch& b = B();
  if (!b.inited) return RH_OK;
  cudaStreamSynchronize(ctx().stream);
  if (b.graph) cudaGraphExecDestroy(b.graph);
  for (int i = 0; i < 2; ++i) {
    cudaFree(b.uf[i] ? (void*)b.uf[i] : (void*)b.ud[i]);  // FP32-bulk: ud is a view into uf's records
  }
  cudaFree(b.d_prob);
  cudaFree(b.d_done);
  cudaFree(b.d_nstep);
  cudaFree(b.d_cur);
  cudaFree(b.d_dt);
  cudaFree(b.d_t);
  cudaFree(b.d_tot);
  cudaFree(b.d_order);
  cudaFree(b.d_woff);
  cudaFree(b.d_partial);
  cudaFree(b.d_counter);
  cudaFree(b.d_tmp);
  cudaFree(b.d_bad);
  cudaFree(b.d_coff);
  b = Batch();
  return RH_OK;
}

long long rh_batch_footprint(const rh_batch_problem* p) {
  if (!p) return -1;
  const long long noct = (long long)(p->n[0] / 2) * (p->n[1] / 2) * (p->n[2] / 2);
  return noct * pool_bytes_per_oct(B().inited ? B().precision : RH_PREC_FP64);
}

int rh_batch_capacity(void) { return B().cap; }

int rh_batch_add(const rh_batch_problem* p, const rh_batch_ic* ic, int* id) {
  Batch& b = B();
  Context& c = ctx();
  if (!b.inited) {
    set_error("rh_batch_init has not been called");
    return RH_ESTATE;
  }
  if (!p || !ic || !id) {
    set_error("rh_batch_add: null argument");
    return RH_EINVAL;
  }
  for (int d = 0; d < 3; ++d)
    if (p->n[d] < 2 || (p->n[d] & 1)) {
      set_error("rh_batch_add: cells per edge must be even and >= 2");
      return RH_EINVAL;
    }
  if ((p->ndim != 2 && p->ndim != 3) || (p->ndim == 2 && p->n[2] != 2) || !(p->dx > 0) || !(p->gamma > 1) ||
      !(p->smallc > 0) || !(p->courant_factor > 0) || (!(p->t_end > 0) && p->max_steps <= 0)) {
    set_error("rh_batch_add: bad ndim/dx/gamma/smallc/courant or no stopping rule (t_end or max_steps)");
    return RH_EINVAL;
  }
  if (ic->kind == RH_IC_SPLIT && (ic->axis < 0 || ic->axis > 2)) {
    set_error("rh_batch_add: split axis must be 0..2");
    return RH_EINVAL;
  }
  if (ic->kind < RH_IC_SPLIT || ic->kind > RH_IC_HOST || (ic->kind == RH_IC_HOST && !ic->host_uold)) {
    set_error("rh_batch_add: unknown initial condition");
    return RH_EINVAL;
  }
  int slot = -1;
  for (int i = 0; i < b.cap; ++i)
    if (!b.probs[i].used) {
      slot = i;
      break;
    }
  if (slot < 0) {
    set_error("rh_batch_add: all %d problem slots in use", b.cap);
    return RH_EBUSY;
  }
  const long long noct = (long long)(p->n[0] / 2) * (p->n[1] / 2) * (p->n[2] / 2);
  long long oct0 = 0;
  if (alloc_octs(noct, &oct0) != RH_OK) {
    set_error("rh_batch_add: pool full (%lld octs requested)", noct);
    return RH_ENOMEM;
  }
  const BatchProb P = make_prob(*p, oct0);
  const bool fp32 = b.precision == RH_PREC_FP32_BULK;
  double* host_dev = nullptr;
  // device set-up of the problem; on any failure the pool range and the slot
  // are released again, so a failed add leaves the batch as it was
  auto setup = [&]() -> cudaError_t {
    cudaError_t e = cudaSuccess;
    if (ic->kind == RH_IC_HOST) {
      e = cudaMalloc(&host_dev, sizeof(double) * 40 * noct);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(host_dev, ic->host_uold, sizeof(double) * 40 * noct, cudaMemcpyHostToDevice, c.stream);
      if (e != cudaSuccess) return e;
    }
    const long long ncell = noct * 8;
    batch_ic_kernel<<<(unsigned)((ncell + 255) / 256), 256, 0, c.stream>>>(*ic, P, b.ud[b.parity], b.uf[b.parity],
                                                                            fp32 ? 1 : 0, host_dev);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const long long nblk = (ncell + 255) / 256;
    if (nblk > b.tmp_cap) {
      cudaStreamSynchronize(c.stream);
      cudaFree(b.d_tmp);
      b.d_tmp = nullptr;
      b.tmp_cap = 0;
      if ((e = cudaMalloc(&b.d_tmp, sizeof(double) * 5 * nblk)) != cudaSuccess) return e;
      b.tmp_cap = nblk;
    }
    batch_cfl_kernel<<<(unsigned)nblk, 256, 0, c.stream>>>(P, b.ud[b.parity], b.uf[b.parity], fp32 ? 1 : 0,
                                                           b.d_tmp);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    batch_init_dt_kernel<<<1, 256, 0, c.stream>>>(P, slot, b.d_tmp, nblk, b.d_dt, b.d_tot);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int zero = 0;
    const double dz = 0.0;
    if ((e = cudaMemcpyAsync(b.d_done + slot, &zero, sizeof(int), cudaMemcpyHostToDevice, c.stream)) ||
        (e = cudaMemcpyAsync(b.d_nstep + slot, &zero, sizeof(int), cudaMemcpyHostToDevice, c.stream)) ||
        (e = cudaMemcpyAsync(b.d_bad + slot, &zero, sizeof(int), cudaMemcpyHostToDevice, c.stream)) ||
        (e = cudaMemcpyAsync(b.d_cur + slot, &b.parity, sizeof(int), cudaMemcpyHostToDevice, c.stream)) ||
        (e = cudaMemcpyAsync(b.d_t + slot, &dz, sizeof(double), cudaMemcpyHostToDevice, c.stream)))
      return e;
    return cudaStreamSynchronize(c.stream);
  };
  const cudaError_t e = setup();
  if (host_dev) cudaFree(host_dev);
  if (e != cudaSuccess) {
    free_octs(oct0, noct);
    return cuda_fail(e, "rh_batch_add");
  }
  HostProb& hp = b.probs[slot];
  hp.used = true;
  hp.p = *p;
  hp.oct0 = oct0;
  hp.noct = noct;
  b.dirty = true;
  *id = slot;
  return RH_OK;
}

int rh_batch_remove(int id) {
  Batch& b = B();
  if (!b.inited || id < 0 || id >= b.cap || !b.probs[id].used) {
    set_error("rh_batch_remove: no problem %d", id);
    return RH_EINVAL;
  }
  RH_CUDA(cudaStreamSynchronize(ctx().stream));
  free_octs(b.probs[id].oct0, b.probs[id].noct);
  b.probs[id] = HostProb();
  const int one = 1;
  RH_CUDA(cudaMemcpy(b.d_done + id, &one, sizeof(int), cudaMemcpyHostToDevice));
  b.dirty = true;
  return RH_OK;
}

int rh_batch_set_tile(int txo, int tyo, int minb, int lz) {
  Batch& b = B();
  if (!b.inited) {
    set_error("rh_batch_init has not been called");
    return RH_ESTATE;
  }
  if (!find_batch(b.precision, txo, tyo, minb, b.slope, b.riemann) || lz < 1 || lz > kBatchMaxLz) {
    set_error("rh_batch_set_tile: %dx%d minb %d not compiled", txo, tyo, minb);
    return RH_EINVAL;
  }
  b.cfg = TileCfg{txo, tyo, minb, lz};
  b.dirty = true;
  return RH_OK;
}

int rh_batch_set_plane_path(int on) {
  Batch& b = B();
  if (!b.inited) {
    set_error("rh_batch_init has not been called");
    return RH_ESTATE;
  }
  b.plane2d = on ? 1 : 0;
  b.dirty = true;
  return RH_OK;
}

int rh_batch_step(int nsteps) {
  Batch& b = B();
  Context& c = ctx();
  if (!b.inited) {
    set_error("rh_batch_init has not been called");
    return RH_ESTATE;
  }
  if (nsteps < 0) return RH_EINVAL;
  if (b.dirty) {
    int rc = rebuild();
    if (rc) return rc;
  }
  if (b.nslot == 0) return RH_OK;
  const BatchReg* reg = find_batch(b.precision, b.cfg.txo, b.cfg.tyo, b.cfg.minb, b.slope, b.riemann);
  int done_steps = 0;
  while (done_steps < nsteps) {
    if (nsteps - done_steps >= 2 && b.parity == b.graph_parity) {
      RH_CUDA(cudaGraphLaunch(b.graph, c.stream));
      done_steps += 2;
    } else {
      BatchArgs A{b.d_prob, b.d_order, b.d_woff, b.nslot, b.nwork, b.cfg.txo, b.cfg.tyo, b.cfg.lz, b.d_counter,
                  b.d_done, b.d_dt, b.d_partial, {b.ud[0], b.ud[1]}, {b.uf[0], b.uf[1]}, c.d_err,
                  b.plane2d};
      RH_CUDA(reg->fn(A, b.parity, b.nblocks, c.stream));
      check_step(b.parity);
      batch_reduce_kernel<<<b.nslot, 256, 0, c.stream>>>(b.d_prob, b.d_order, b.d_woff, b.d_partial, b.d_done,
                                                         b.d_nstep, b.d_cur, b.d_dt, b.d_t, b.d_tot, b.d_counter,
                                                         b.parity, b.d_bad);
      RH_CUDA(cudaGetLastError());
      b.parity ^= 1;
      done_steps += 1;
      continue;
    }
  }
  return RH_OK;
}

int rh_batch_status(int id, double* t, int* nstep, int* done, double* dt, double* totals5) {
  Batch& b = B();
  Context& c = ctx();
  if (!b.inited || id < 0 || id >= b.cap || !b.probs[id].used) {
    set_error("rh_batch_status: no problem %d", id);
    return RH_EINVAL;
  }
  RH_CUDA(cudaStreamSynchronize(c.stream));
  if (t) RH_CUDA(cudaMemcpy(t, b.d_t + id, sizeof(double), cudaMemcpyDeviceToHost));
  if (nstep) RH_CUDA(cudaMemcpy(nstep, b.d_nstep + id, sizeof(int), cudaMemcpyDeviceToHost));
  if (done) RH_CUDA(cudaMemcpy(done, b.d_done + id, sizeof(int), cudaMemcpyDeviceToHost));
  if (dt) RH_CUDA(cudaMemcpy(dt, b.d_dt + id, sizeof(double), cudaMemcpyDeviceToHost));
  if (totals5) RH_CUDA(cudaMemcpy(totals5, b.d_tot + id * 5ll, 5 * sizeof(double), cudaMemcpyDeviceToHost));
  return RH_OK;
}

int rh_batch_set_state_check(int on) {
  Batch& b = B();
  if (!b.inited) {
    set_error("rh_batch_init has not been called");
    return RH_ESTATE;
  }
  b.check = on ? 1 : 0;
  b.dirty = true;  // the step graph gains or loses the check kernel
  return RH_OK;
}

int rh_batch_check_mask(int id, int* mask) {
  Batch& b = B();
  if (!b.inited || id < 0 || id >= b.cap || !b.probs[id].used || !mask) {
    set_error("rh_batch_check_mask: no problem %d", id);
    return RH_EINVAL;
  }
  RH_CUDA(cudaStreamSynchronize(ctx().stream));
  RH_CUDA(cudaMemcpy(mask, b.d_bad + id, sizeof(int), cudaMemcpyDeviceToHost));
  return RH_OK;
}

int rh_batch_poll(int* done, int* nstep, double* t) {
  Batch& b = B();
  Context& c = ctx();
  if (!b.inited) {
    set_error("rh_batch_init has not been called");
    return RH_ESTATE;
  }
  if (done) RH_CUDA(cudaMemcpyAsync(done, b.d_done, sizeof(int) * b.cap, cudaMemcpyDeviceToHost, c.stream));
  if (nstep) RH_CUDA(cudaMemcpyAsync(nstep, b.d_nstep, sizeof(int) * b.cap, cudaMemcpyDeviceToHost, c.stream));
  if (t) RH_CUDA(cudaMemcpyAsync(t, b.d_t, sizeof(double) * b.cap, cudaMemcpyDeviceToHost, c.stream));
  int err = 0;
  RH_CUDA(cudaMemcpyAsync(&err, c.d_err, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  RH_CUDA(cudaStreamSynchronize(c.stream));
  if (err) {
    cudaMemset(c.d_err, 0, sizeof(int));
    set_error("device wait bound exceeded in a batch step (error word %d)", err);
    return RH_ETIMEDOUT;
  }
  return RH_OK;
}

int rh_batch_fetch(int id, double* host_uold) {
  Batch& b = B();
  Context& c = ctx();
  if (!b.inited || id < 0 || id >= b.cap || !b.probs[id].used || !host_uold) {
    set_error("rh_batch_fetch: no problem %d", id);
    return RH_EINVAL;
  }
  const HostProb& hp = b.probs[id];
  RH_CUDA(cudaStreamSynchronize(c.stream));
  int cur = 0;
  RH_CUDA(cudaMemcpy(&cur, b.d_cur + id, sizeof(int), cudaMemcpyDeviceToHost));
  if (b.precision == RH_PREC_FP64) {
    RH_CUDA(cudaMemcpy(host_uold, b.ud[cur] + hp.oct0 * 40, sizeof(double) * 40 * hp.noct,
                       cudaMemcpyDeviceToHost));
  } else {
    std::vector<float> f((size_t)hp.noct * kBulkF);  // whole records; E read through the double view
    RH_CUDA(cudaMemcpy(f.data(), b.uf[cur] + hp.oct0 * kBulkF, (size_t)kBulkBytes * hp.noct,
                       cudaMemcpyDeviceToHost));
    const double* e = reinterpret_cast<const double*>(f.data()) + kBulkE;
    for (long long o = 0; o < hp.noct; ++o)
      for (int cell = 0; cell < 8; ++cell) {
        for (int v = 0; v < 4; ++v) host_uold[o * 40 + v * 8 + cell] = (double)f[o * kBulkF + v * 8 + cell];
        host_uold[o * 40 + 32 + cell] = e[o * kBulkD + cell];
      }
  }
  return RH_OK;
}

// A problem as a one-level mesh (level 1, n/2 octs per axis, row-major octs)
// in the restart / snapshot layouts of include/ramses_hydro_io.h.
int rh_batch_file_image(int id, int kind, void* host_buf, long long cap, long long* nbytes) {
  Batch& b = B();
  Context& c = ctx();
  if (!b.inited || id < 0 || id >= b.cap || !b.probs[id].used || !nbytes) {
    set_error("rh_batch_file_image: no problem %d", id);
    return RH_EINVAL;
  }
  const HostProb& hp = b.probs[id];
  RH_CUDA(cudaStreamSynchronize(c.stream));
  int cur = 0;
  RH_CUDA(cudaMemcpy(&cur, b.d_cur + id, sizeof(int), cudaMemcpyDeviceToHost));
  ImageSrc s;
  s.bulk = b.precision == RH_PREC_FP32_BULK;
  s.ud = b.ud[cur] + hp.oct0 * (s.bulk ? kBulkD : 40);
  s.uf = s.bulk ? b.uf[cur] + hp.oct0 * kBulkF : nullptr;
  s.levelmin = s.levelmax = 1;
  s.oct0.push_back(0);
  s.noct.push_back(hp.noct);
  s.nxo = hp.p.n[0] / 2;
  s.nyo = hp.p.n[1] / 2;
  s.nzo = hp.p.n[2] / 2;
  if (kind != RH_FILE_AMR && kind != RH_FILE_HYDRO_BACKUP && kind != RH_FILE_HYDRO_OUTPUT) {
    set_error("rh_batch_file_image: unknown kind %d", kind);
    return RH_EINVAL;
  }
  const long long need = image_bytes(kind, s);
  *nbytes = need;
  if (!host_buf || cap < need) {
    set_error("rh_batch_file_image: buffer of %lld bytes, the image needs %lld", cap, need);
    return RH_EINVAL;
  }
  const void* d = nullptr;
  long long n = 0;
  int rc = build_image(kind, s, hp.p.gamma, &d, &n);
  if (rc) return rc;
  return image_to_host(d, n, host_buf, cap);
}

int rh_batch_bench(int nsteps, float* ms_per_step) {
  Batch& b = B();
  Context& c = ctx();
  if (!b.inited || nsteps < 1 || !ms_per_step) {
    set_error("rh_batch_bench: not initialised or bad arguments");
    return RH_EINVAL;
  }
  if (b.dirty) {
    int rc = rebuild();
    if (rc) return rc;
  }
  RH_CUDA(cudaEventRecord(c.ev0, c.stream));
  int rc = rh_batch_step(nsteps);
  if (rc) return rc;
  RH_CUDA(cudaEventRecord(c.ev1, c.stream));
  RH_CUDA(cudaEventSynchronize(c.ev1));
  float ms = 0;
  RH_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
  *ms_per_step = ms / nsteps;
  return RH_OK;
}

int rh_batch_list_tiles(int precision, int* txo, int* tyo, int* minb, int max) {
  int n = 0;
  for (auto& e : batch_registry()) {
    if (e.k.prec != precision || e.k.slope != 2 || e.k.riemann != 3) continue;
    if (n < max) {
      if (txo) txo[n] = e.k.txo;
      if (tyo) tyo[n] = e.k.tyo;
      if (minb) minb[n] = e.k.minb;
    }
    ++n;
  }
  return n;
}

long long rh_batch_cells(void) {
  Batch& b = B();
  if (!b.inited) return 0;
  std::vector<int> done(b.cap, 0);
  if (cudaStreamSynchronize(ctx().stream) != cudaSuccess ||
      cudaMemcpy(done.data(), b.d_done, sizeof(int) * b.cap, cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  long long n = 0;
  for (int i = 0; i < b.cap; ++i)
    if (b.probs[i].used && !done[i]) n += b.probs[i].noct * 8;
  return n;
}

}  // extern "C"
