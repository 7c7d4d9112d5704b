// rh_batch.cuh — persistent batch kernel: one launch advances every
// unfinished problem of the batch by one Godunov step.
#pragma once
#include "rh_godunov.cuh"
#include "rh_godunov2.cuh"

namespace rh {

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
  double* ud[2];            // FP64 pool [oct][5][8], or FP32-bulk energy [oct][8]
  float* uf[2];             // FP32-bulk pool [oct][4][8]
  int* err;
};

__device__ __forceinline__ int batch_slot(const long long* woff, int nslot, long long w) {
  int lo = 0, hi = nslot;  // woff[lo] <= w < woff[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (woff[mid] <= w) lo = mid;
    else hi = mid;
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

template <typename T, typename V, int TXO, int TYO, int MINB, int SLOPE, int RIEMANN>
__global__ void __launch_bounds__(Geo<T, V, TXO, TYO>::NT, MINB) batch_step_kernel(const BatchArgs B, int parity) {
  using G = Geo<T, V, TXO, TYO>;
  __shared__ long long s_w;
  if (threadIdx.x == 0) {
    rh_s_abort = 0;
    uint64_t* bar = reinterpret_cast<uint64_t*>(rh_smem + G::oBar);
    for (int s = 0; s < G::NSTAGE; ++s) mbar_init(&bar[s], G::NSLOT);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  int rbase = 0;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_w = (long long)atomicAdd(B.counter, 1ull);
    __syncthreads();
    const long long w = s_w;
    if (w >= B.nwork) break;
    const int slot = batch_slot(B.woff, B.nslot, w);
    const int pid = B.order[slot];
    if (B.done[pid]) continue;
    const BatchProb P = B.prob[pid];
    const double dt = B.dt[pid];
    const long long li = w - B.woff[slot];
    const int bx = (int)(li % P.tx), by = (int)((li / P.tx) % P.ty), bz = (int)(li / ((long long)P.tx * P.ty));
    const int nzo = P.ncz >> 1;
    const int4 hdr = make_int4(bx * B.txo, by * B.tyo, bz * B.lz, min(B.lz, nzo - bz * B.lz));
    LevelArgs A;
    batch_level(P, dt, B.err, A);
    StateArgs<T> S;
    if (sizeof(T) == 8) {
      S.uold_d = B.ud[parity] + P.oct0 * 40;
      S.unew_d = B.ud[1 - parity] + P.oct0 * 40;
      S.uold_f = nullptr;
      S.unew_f = nullptr;
    } else {
      S.uold_d = B.ud[parity] + P.oct0 * 8;
      S.unew_d = B.ud[1 - parity] + P.oct0 * 8;
      S.uold_f = B.uf[parity] + P.oct0 * 32;
      S.unew_f = B.uf[1 - parity] + P.oct0 * 32;
    }
    HydroK<V> H;
    batch_hydro<V>(P, dt, H);
    if constexpr (sizeof(T) == 8) {
      pencil_body_f64<T, TXO, TYO, SLOPE, RIEMANN, false, true>(A, S, H, hdr, nullptr, rbase,
                                                                SlotCflSink{B.partial + w * 5});
    } else {
      pencil_body_f32<TXO, TYO, SLOPE, RIEMANN, false, true>(A, S, H, hdr, nullptr, rbase,
                                                             SlotCflSink{B.partial + w * 5});
    }
    rbase += hdr.w + 2;
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
