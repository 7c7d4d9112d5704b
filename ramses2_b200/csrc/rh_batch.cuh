// rh_batch.cuh — persistent batch kernel: one launch advances every
// unfinished problem of the batch by one Godunov step.
#pragma once
#include "rh_godunov.cuh"
#include "rh_godunov2.cuh"
#include "rh_plane2d.cuh"

namespace rh {

constexpr int kBatchMaxLz = 64;      // most oct layers of one batch pencil
constexpr int kBatchMaxSlots = 100;  // most oct columns (tile + halo) of one batch pencil
// Tile bodies per work item of a 2D problem on the plane path: a plane tile is
// one layer, so the item set-up (work counter, slot search, problem constants)
// is shared by this many tiles along y.
constexpr int kPlaneGroup = 4;

// Static description of one problem in the device pool.
struct BatchProb {
  long long oct0;           // first oct of the problem in the pool
  int ncx, ncy, ncz;        // cells per edge
  int periodic[3];
  int btype[6];
  int ndim;
  int tx, ty, tz;           // pencils per edge (tile counts)
  double dx, gamma, smallr, smallc, courant, t_end;
  int max_steps;
};

// Arguments of one batch step (parity: which pool buffer holds uold).
struct BatchArgs {
  const BatchProb* prob;
  const int* order;         // schedule slot -> problem id
  const long long* woff;    // [nslot+1] first work item of each schedule slot
  int nslot;
  long long nwork;
  int txo, tyo, lz;
  unsigned long long* counter;  // work items handed out (reset by the reduction)
  const int* done;
  const double* dt;
  double* partial;          // [nwork][5]
  double* ud[2];            // FP64 pool [oct][5][8], or the FP32-bulk records' E view
  float* uf[2];             // FP32-bulk pool: 192-byte records (rh_bulk.h)
  int* err;
  int plane2d;              // 2D problems take the plane tile body (else the pencil body)
};

// Schedule slot of work item w (woff[slot] <= w < woff[slot + 1]), searched
// by one warp: each round reads 32 evenly spaced entries of woff at once and
// keeps the interval between the last one <= w and the next, so 4096 slots
// take three dependent reads instead of twelve.  Called by all 32 lanes.
__device__ __forceinline__ int batch_slot_warp(const long long* woff, int nslot, long long w, int lane) {
  int lo = 0, hi = nslot;  // woff[lo] <= w < woff[hi]
  while (hi - lo > 1) {
    const long long span = hi - lo;
    const int q = lo + (int)(span * lane / 32);  // q(0) = lo, nondecreasing in lane, < hi
    const unsigned le = __ballot_sync(0xffffffffu, woff[q] <= w);  // a prefix of the lanes, lane 0 included
    const int k = 31 - __clz(le);
    const int nlo = lo + (int)(span * k / 32);
    hi = k < 31 ? lo + (int)(span * (k + 1) / 32) : hi;
    lo = nlo;
  }
  return lo;
}

// Per-problem LevelArgs (dense level, no tables) and the hydro constants of its dt.
__device__ __forceinline__ void batch_level(const BatchProb& P, double dt, int* err, LevelArgs& A) {
  A.phdr = nullptr;
  A.poff = nullptr;
  A.ptab = nullptr;
  A.npencil = 0;
  A.ncx = P.ncx;
  A.ncy = P.ncy;
  A.ncz = P.ncz;
  for (int d = 0; d < 3; ++d) A.periodic[d] = P.periodic[d];
  for (int i = 0; i < 6; ++i) A.btype[i] = P.btype[i];
  A.ghost_base = 0x7fffffff;
  A.cfl_partial = nullptr;
  A.err = err;
  A.cfl.gamma = P.gamma;
  A.cfl.gm1 = P.gamma - 1.0;
  A.cfl.smallr = P.smallr;
  A.cfl.smallp = P.smallc * P.smallc / P.gamma;
  A.cfl.cdx_smallc = P.courant * P.dx / P.smallc;
  A.cfl.two_cdx = 2.0 * P.courant * P.dx;
  A.cfl.two_c = 2.0 * P.courant;
  A.cfl.gsum_dx = 0.0;
  A.cfl.k0 = A.cfl.two_cdx / (1.0 + sqrt(1.0 + A.cfl.two_c * 0.0001));
  A.cfl.ndim = P.ndim;
  A.vol = P.dx * P.dx * P.dx;
  A.gm1_d = P.gamma - 1.0;
  A.smalle_d = P.smallc * P.smallc / P.gamma / (P.gamma - 1.0);
  A.refmask = nullptr;
  A.ghost_father = nullptr;
  A.accumulate = 0;
  A.gface = nullptr;
  A.gface_base = 0;
  A.cflskip = nullptr;
  (void)dt;
}

template <class V> __device__ __forceinline__ void batch_hydro(const BatchProb& P, double dt, HydroK<V>& H) {
  auto b = [](double v) { return Lane<V>::bc((typename Lane<V>::S)v); };
  H.gamma = b(P.gamma);
  H.entho = b(1.0 / (P.gamma - 1.0));
  H.smallr = b(P.smallr);
  H.smallc2 = b(P.smallc * P.smallc);
  H.smallp_trace = b(P.smallr * (P.smallc * P.smallc));
  H.smallp_riem = b(P.smallc * P.smallc / P.gamma);
  const double cap = P.courant * P.dx / dt;
  H.smax_cap = b(sizeof(typename Lane<V>::S) == 4 && cap > 3.0e38 ? 3.0e38 : cap);
  H.dtdx = b(dt / P.dx);
  H.zero = b(0.0);
  H.half = b(0.5);
  H.two = b(2.0);
  H.gm1 = b(P.gamma - 1.0);
  H.smalle = b(P.smallc * P.smallc / P.gamma / (P.gamma - 1.0));
  H.grav[0] = H.grav[1] = H.grav[2] = b(0.0);
}

// Constants of the CTA's current work item, in shared memory: the pencil
// body reads them where it uses them instead of holding them in registers.
__shared__ LevelArgs rh_bA;
__shared__ StateArgs<double> rh_bS64;
__shared__ StateArgs<float> rh_bS32;
__shared__ HydroK<double> rh_bH64;
__shared__ HydroK<float2> rh_bH32;
__shared__ double* rh_b_out;
__shared__ int4 rh_b_hdr;
__shared__ int rh_b_tab[kBatchMaxSlots + kBatchMaxLz + 2];  // dense oct offsets: xy per slot, z per row

// One pencil of the current work item.  Kept out of line so the persistent
// loop around it does not stretch the body's register live ranges.
template <typename T, int TXO, int TYO, int SLOPE, int RIEMANN>
__device__ __noinline__ void batch_pencil(int rbase) {
  const int4 hdr = rh_b_hdr;
  if constexpr (sizeof(T) == 8) {
    pencil_body_f64<T, TXO, TYO, SLOPE, RIEMANN, false, true>(rh_bA, rh_bS64, rh_bH64, hdr, rh_b_tab, rbase,
                                                              SlotCflSink{&rh_b_out});
  } else {
    pencil_body_f32<TXO, TYO, SLOPE, RIEMANN, false, true>(rh_bA, rh_bS32, rh_bH32, hdr, rh_b_tab, rbase,
                                                           SlotCflSink{&rh_b_out});
  }
}

// One XY tile of a 2D problem (rh_plane2d.cuh), out of line like batch_pencil.
template <typename T, int TXO, int TYO, int SLOPE, int RIEMANN>
__device__ __noinline__ void batch_plane(int g, CflAcc* acc) {
  constexpr int rows = sizeof(T) == 8 ? 1 : 2;  // tile rows per tile body (FP32-bulk: two, one per lane)
  const int4 h0 = rh_b_hdr;
  const int4 hdr = make_int4(h0.x, h0.y + g * rows * TYO, h0.z, h0.w);
  CflAcc a = *acc;
  if constexpr (sizeof(T) == 8) {
    plane2d_body<T, double, TXO, TYO, SLOPE, RIEMANN>(rh_bA, rh_bS64, rh_bH64, hdr, a);
  } else {
    plane2d_body<T, float2, TXO, TYO, SLOPE, RIEMANN>(rh_bA, rh_bS32, rh_bH32, hdr, a);
  }
  *acc = a;
}

template <typename T, typename V, int TXO, int TYO, int MINB, int SLOPE, int RIEMANN>
__global__ void __launch_bounds__(Geo<T, V, TXO, TYO>::NT, MINB) batch_step_kernel(const BatchArgs B, int parity) {
  using G = Geo<T, V, TXO, TYO>;
  static_assert(G::NSLOT <= kBatchMaxSlots, "tile too wide for the dense offset table");
  __shared__ long long s_w;
  __shared__ int s_skip, s_plane;
  if (threadIdx.x == 0) {
    rh_s_abort = 0;
    uint64_t* bar = reinterpret_cast<uint64_t*>(rh_smem + G::oBar);
    for (int s = 0; s < G::NSTAGE; ++s) mbar_init(&bar[s], G::NSLOT);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  int rbase = 0;
  for (;;) {
    __syncthreads();  // the previous pencil is finished with the work-item constants
    if (threadIdx.x < 32) {
      long long w = 0;
      if (threadIdx.x == 0) w = (long long)atomicAdd(B.counter, 1ull);
      w = __shfl_sync(0xffffffffu, w, 0);
      const int slot = w < B.nwork ? batch_slot_warp(B.woff, B.nslot, w, threadIdx.x) : 0;
      if (threadIdx.x == 0) {
        s_w = w;
        s_skip = 1;
        if (w < B.nwork) {
          const int pid = B.order[slot];
          if (!B.done[pid]) {
            s_skip = 0;
            rh_b_out = B.partial + w * 5;
            const BatchProb P = B.prob[pid];
            const double dt = B.dt[pid];
            const long long li = w - B.woff[slot];
            const int bx = (int)(li % P.tx), by = (int)((li / P.tx) % P.ty);
            const int bz = (int)(li / ((long long)P.tx * P.ty));
            const int nzo = P.ncz >> 1;
            s_plane = B.plane2d && P.ndim == 2 && nzo == 1 && P.periodic[2];
            // a plane item is kPlaneGroup tile bodies along y; FP32-bulk tile
            // bodies hold two tile rows, one in each lane
            const int ty0 = s_plane ? by * kPlaneGroup * (sizeof(T) == 4 ? 2 : 1) : by;
            rh_b_hdr = make_int4(bx * B.txo, ty0 * B.tyo, bz * B.lz, min(B.lz, nzo - bz * B.lz));
            batch_level(P, dt, B.err, rh_bA);
            if constexpr (sizeof(T) == 8) {
              rh_bS64.uold_d = B.ud[parity] + P.oct0 * 40;
              rh_bS64.unew_d = B.ud[1 - parity] + P.oct0 * 40;
              rh_bS64.uold_f = nullptr;
              rh_bS64.unew_f = nullptr;
              batch_hydro<double>(P, dt, rh_bH64);
            } else {
              rh_bS32.uold_d = B.ud[parity] + P.oct0 * kBulkD;
              rh_bS32.unew_d = B.ud[1 - parity] + P.oct0 * kBulkD;
              rh_bS32.uold_f = B.uf[parity] + P.oct0 * kBulkF;
              rh_bS32.unew_f = B.uf[1 - parity] + P.oct0 * kBulkF;
              batch_hydro<float2>(P, dt, rh_bH32);
            }
          }
        }
      }
    }
    __syncthreads();
    if (s_w >= B.nwork) break;
    if (s_skip) continue;
    if (s_plane) {
      const int rows = sizeof(T) == 8 ? 1 : 2;
      CflAcc acc;
      for (int g = 0; g < kPlaneGroup && rh_b_hdr.y + g * rows * TYO < (rh_bA.ncy >> 1); ++g) {
        // FP32-bulk 7x7 plane bodies need no barrier between them: the
        // previous body read its primitives before its last barrier and its
        // interface states before this body's first one
        if (g && !(sizeof(T) == 4 && 2 * TXO + 2 == 16)) __syncthreads();
        batch_plane<T, TXO, TYO, SLOPE, RIEMANN>(g, &acc);
      }
      if constexpr (sizeof(T) == 4) acc.scale_bulk(rh_bA.vol);
      cfl_block_reduce<G::NWARP>(acc, rh_bA.cfl, reinterpret_cast<double*>(rh_smem + G::oRed), rh_b_out);
      continue;
    }
    {
      // oct index of (row, slot) = tab[NSLOT + row] + tab[slot], boundary-mapped
      const int4 hdr = rh_b_hdr;
      const int nx = rh_bA.ncx >> 1, ny = rh_bA.ncy >> 1, nz = rh_bA.ncz >> 1;
      auto m = [](int v, int n, int per) { return per ? ((v % n) + n) % n : (v < 0 ? 0 : (v >= n ? n - 1 : v)); };
      for (int i = threadIdx.x; i < G::NSLOT + hdr.w + 2; i += G::NT) {
        if (i < G::NSLOT) {
          rh_b_tab[i] = m(hdr.y - 1 + i / G::OW, ny, rh_bA.periodic[1]) * nx +
                        m(hdr.x - 1 + i % G::OW, nx, rh_bA.periodic[0]);
        } else {
          rh_b_tab[i] = m(hdr.z - 1 + (i - G::NSLOT), nz, rh_bA.periodic[2]) * (nx * ny);
        }
      }
      __syncthreads();
    }
    batch_pencil<T, TXO, TYO, SLOPE, RIEMANN>(rbase);
    rbase += rh_b_hdr.w + 2;
  }
}

using BatchLaunchFn = cudaError_t (*)(const BatchArgs& B, int parity, int nblocks, cudaStream_t st);

struct BatchKey {
  int prec, txo, tyo, minb, slope, riemann;
};
void register_batch_launcher(const BatchKey& k, BatchLaunchFn fn, const void* func, size_t smem, int threads);

template <typename T, typename V, int TXO, int TYO, int MINB, int SLOPE, int RIEMANN>
cudaError_t launch_batch(const BatchArgs& B, int parity, int nblocks, cudaStream_t st) {
  using G = Geo<T, V, TXO, TYO>;
  // the dynamic shared-memory attribute is set by the runtime before any launch or capture
  batch_step_kernel<T, V, TXO, TYO, MINB, SLOPE, RIEMANN><<<nblocks, G::NT, G::kSmem, st>>>(B, parity);
  return cudaGetLastError();
}

template <typename T, int TXO, int TYO, int MINB> struct BatchRegistrar {
  BatchRegistrar() {
    using V = typename std::conditional<sizeof(T) == 8, double, float2>::type;
    using G = Geo<T, V, TXO, TYO>;
    constexpr int P = sizeof(T) == 8 ? RH_PREC_FP64 : RH_PREC_FP32_BULK;
#define RH_BREG(S, R)                                                                              \
  register_batch_launcher({P, TXO, TYO, MINB, S, R}, &launch_batch<T, V, TXO, TYO, MINB, S, R>,  \
                          (const void*)batch_step_kernel<T, V, TXO, TYO, MINB, S, R>, G::kSmem, G::NT);
    RH_BREG(0, 1) RH_BREG(0, 2) RH_BREG(0, 3)
    RH_BREG(1, 1) RH_BREG(1, 2) RH_BREG(1, 3)
    RH_BREG(2, 1) RH_BREG(2, 2) RH_BREG(2, 3)
#undef RH_BREG
  }
};

}  // namespace rh
