// rh_godunov.cuh — the fused MUSCL-Hancock Godunov kernels (sm_100a).
//
// One CTA owns a "pencil": an XY tile of TXO x TYO octs and a run of L oct
// layers along z, and marches through it along z:
//
//   * the pencil's oct table lists, for each of the L+2 layers (one halo layer
//     each side) and each of the (TXO+2)(TYO+2) oct columns, the index of the
//     oct whose cells fill that position (boundary sources already resolved);
//   * each layer's oct records are staged into shared memory by bulk async
//     copies (cp.async.bulk, one oct record per copy, completion counted on an
//     mbarrier), two layers in flight, so the gather through the oct table runs
//     ahead of the arithmetic;
//   * one thread per "ring" cell column ((2TXO+2) x (2TYO+2) columns) converts
//     its cells to primitive variables (ctoprim), keeps z-neighbours in
//     registers, takes x/y neighbours from a shared plane buffer and computes
//     slopes, the normal-velocity bound and the Hancock predictor (uslope +
//     trace3d);
//   * x/y interface states are exchanged through shared memory, z interface
//     states never leave the thread; the Riemann fluxes of the three
//     directions (cmpflxm + llf/hll/hllc) and the conservative update of the
//     oct cells (godunov_fine.f90:733-816: x, then y, then z differences)
//     follow;
//   * the epilogue evaluates the CFL time step and the conserved totals of the
//     new state (courant_fine + cmpdt) in FP64, reduced per CTA with warp
//     shuffles into a per-pencil partial, so the next step's dt costs no pass.
//
// Plain FP64 path (this file): one cell plane per iteration, lane type double.
// FP32-bulk path (rh_godunov2.cuh): one oct layer (two planes) per iteration,
// lane type float2 with packed FP32x2 arithmetic, FP64 energy/pressure/dt.
//
// This replaces the reference's per-subgrid hydro_integrator_kernel
// (gpu/gpu_hydro.cuf:8776-8964), which materialises the whole (2n+4)^3
// stencil and all interface states in shared memory.
#pragma once
#include "ramses_hydro.h"
#include "rh_device.cuh"
#include "rh_physics.cuh"

namespace rh {

// Storage policy of a precision mode (staged oct record sizes).
template <typename T> struct Store;
template <> struct Store<double> {  // plain FP64: reference layout [oct][5][8]
  static constexpr int kSlotF = 0;   // floats per staged oct
  static constexpr int kSlotD = 42;  // doubles per staged oct (40 + pad)
  static constexpr uint32_t kBytes = 320;
};
template <> struct Store<float> {  // FP32-bulk: one 192-byte record per oct (rh_bulk.h)
  static constexpr int kSlotF = 52;  // 48 + pad (floats per staged record)
  static constexpr int kSlotD = 0;
  static constexpr uint32_t kBytes = kBulkBytes;
};

// T: storage element of the bulk variables; V: lane type of the arithmetic.
// Slot of plane (or FP32-bulk layer) p >= -2 in a plane buffer of G::kNQ
// entries, written out in place (a helper call changes the register
// allocation of the pencil kernels).
#define RH_QSLOT(G, p) ((G::kNQ == 2) ? ((p) & 1) : (((p) + 3) % 3))

// NQ: primitive planes (or FP32-bulk oct layers) kept in shared memory: 2 for
// slopes along the three axes, 3 for the 27-point limiter of slope_type 3.
template <typename T, typename V, int TXO, int TYO, int NQ = 2> struct Geo {
  static constexpr int CX = 2 * TXO, CY = 2 * TYO;
  static constexpr int RW = CX + 2, RH = CY + 2;  // ring columns
  static constexpr int NRC = RW * RH;
  static constexpr int LW = CX + 4, LH = CY + 4;  // load columns
  static constexpr int NLC = LW * LH;
  static constexpr int NOC = NLC - NRC;           // outer ring columns
  static constexpr int OW = TXO + 2, OH = TYO + 2;
  static constexpr int NSLOT = OW * OH;           // oct columns per layer
  static constexpr int NWARP = (NRC + 31) / 32;
  static constexpr int NT = NWARP * 32;           // block size (full warps)
  static constexpr int NSTAGE = 2;
  static constexpr size_t kStageD = (size_t)NSTAGE * NSLOT * Store<T>::kSlotD * sizeof(double);
  static constexpr size_t kStageF = (size_t)NSTAGE * NSLOT * Store<T>::kSlotF * sizeof(float);
  static constexpr size_t kQ = (size_t)NQ * 5 * NLC * sizeof(V);
  static constexpr int kNQ = NQ;  // plane-buffer slot of plane (layer) p >= -2: RH_QSLOT(G, p)
  static constexpr size_t kFS = (size_t)10 * NRC * sizeof(V);
  static constexpr size_t kFX = (size_t)2 * 5 * NRC * sizeof(V);
  static constexpr size_t kRed = (size_t)NWARP * 4 * sizeof(double);
  static constexpr size_t kAmr = (size_t)NRC * (sizeof(int) + sizeof(uint32_t));
  static constexpr size_t a16(size_t x) { return (x + 15) & ~size_t(15); }
  static constexpr size_t oStageD = 0;
  static constexpr size_t oStageF = a16(oStageD + kStageD);
  static constexpr size_t oQ = a16(oStageF + kStageF);
  static constexpr size_t oFS = a16(oQ + kQ);
  static constexpr size_t oFX = a16(oFS + kFS);
  static constexpr size_t oRed = a16(oFX + kFX);
  static constexpr size_t oAmr = a16(oRed + kRed);
  static constexpr size_t oBar = a16(oAmr + kAmr);
  static constexpr size_t kSmem = oBar + 64;
};

// Boundary mapping of one global cell coordinate: parity of the source cell
// inside the (already resolved) source oct and the sign of the normal velocity
// (amr/boundaries.f90:150-216: reflexive mirrors, zero-gradient copies).
struct CellMap {
  int parity;
  bool flip;
};
__device__ __forceinline__ CellMap map_coord(int g, int ncell, int periodic, int blo, int bhi) {
  CellMap m{g & 1, false};
  if (periodic) return m;
  if (g < 0) {
    if (blo == RH_BOUND_REFLEXIVE) { m.parity = (-1 - g) & 1; m.flip = true; }
    else m.parity = 0;
  } else if (g >= ncell) {
    if (bhi == RH_BOUND_REFLEXIVE) { m.parity = (2 * ncell - 1 - g) & 1; m.flip = true; }
    else m.parity = (ncell - 1) & 1;
  }
  return m;
}

// Device-wide constants of one level launch.
struct LevelArgs {
  const int4* phdr;       // per pencil: ox0, oy0, oz0, L
  const long long* poff;  // per pencil: offset of its table in ptab
  const int* ptab;        // (L+2) x NSLOT oct indices (0-based; <0 absent)
  int npencil;
  int ncx, ncy, ncz;      // level extent in cells
  int periodic[3];
  int btype[6];
  int ghost_base;         // entries >= ghost_base are never updated
  double* cfl_partial;    // [npencil][5] (mass, ekin, eint, emag, dt) or null
  int* err;               // device error word (bit 0: mbarrier wait timed out)
  CflConst cfl;
  double vol;
  double gm1_d, smalle_d;  // FP64 pressure recovery constants
  // coarse-fine levels only
  const uint8_t* refmask;  // per oct (real and ghost): bit c = cell c refined
  const int2* ghost_father;  // per ghost (entry - ghost_base): father oct (0-based), father cell
  int accumulate;          // 1: unew already holds uold (+ finer-level corrections); add to it
  // deterministic coarse-fine update: per ghost oct of this level 24 face
  // slots (ghost cell x direction) of 5 values, summed later in a fixed order
  // by the coarse gather kernels; null: atomic adds into the fathers
  double* gface;
  long long gface_base;    // state entry of the level's first ghost oct
  // per real oct: bit c = cell c is the father of a finer level's ghost oct,
  // whose courant_fine values the coarse gather computes after its
  // correction (the fused epilogue leaves those cells out); null: none
  const uint8_t* cflskip;
};

// Coarse-fine status of one cell of an AMR level (hydro/godunov_fine.f90:
// 666-685 flux reset, 893-1052 coarse update): bit 0 refined, bit 1 a cell of
// this level updated by this pencil, bit 2 an interpolated ghost inside the
// domain (its father cell receives the face flux / 8), bit 3 a cell left out
// of the fused CFL epilogue (A.cflskip).  The epilogue counts a cell when
// bits 0 and 3 are clear (mask kNoCfl).
constexpr uint32_t kNoCfl = 9u;
__device__ __forceinline__ uint32_t amr_bits(const LevelArgs& A, int ent, int cell, bool upd_pos, bool in_dom) {
  uint32_t b = 0;
  if (ent >= 0) {
    b = (A.refmask[ent] >> cell) & 1u;
    if (ent < A.ghost_base) {
      b |= upd_pos ? 2u : 0u;
      if (A.cflskip) b |= ((A.cflskip[ent] >> cell) & 1u) << 3;
    } else {
      b |= in_dom ? 4u : 0u;
    }
  }
  return b;
}

// Flux through the face between a cell of this level and an interpolated
// ghost: unew(father) +- flux/8 (sign -1: ghost on the low side).  slot =
// 3 * (ghost cell in its oct) + direction names the face: a ghost cell has one
// face per direction on its oct's boundary, and only the pencil holding the
// real cell across it writes there.  Atomic adds into the father, or (A.gface
// set) a store into the face's slot for coarse_gather_kernel.
__device__ __forceinline__ void coarse_add_f64(const LevelArgs& A, double* unew, int ghost_ent, const double* f,
                                               double sign, int slot) {
  if (A.gface) {
    double* s = A.gface + ((size_t)(ghost_ent - A.gface_base) * 24 + slot) * 5;
#pragma unroll
    for (int n = 0; n < 5; ++n) s[n] = sign * (f[n] * 0.125);
    return;
  }
  const int2 fa = A.ghost_father[ghost_ent - A.ghost_base];
  if (fa.x < 0) return;
  double* o = unew + (size_t)fa.x * 40 + fa.y;
#pragma unroll
  for (int n = 0; n < 5; ++n) atomicAdd(o + 8 * n, sign * (f[n] * 0.125));
}
__device__ __forceinline__ void coarse_add_f32(const LevelArgs& A, float* unew_f, double* unew_e, int ghost_ent,
                                               const float* f, float sign, int slot) {
  if (A.gface) {  // the face's slot (as coarse_add_f64), the values the atomics would add
    double* s = A.gface + ((size_t)(ghost_ent - A.gface_base) * 24 + slot) * 5;
#pragma unroll
    for (int n = 0; n < 4; ++n) s[n] = (double)(sign * (f[n] * 0.125f));
    s[4] = (double)sign * ((double)f[4] * 0.125);
    return;
  }
  const int2 fa = A.ghost_father[ghost_ent - A.ghost_base];
  if (fa.x < 0) return;
  float* o = unew_f + (size_t)fa.x * kBulkF + fa.y;
#pragma unroll
  for (int n = 0; n < 4; ++n) atomicAdd(o + 8 * n, sign * (f[n] * 0.125f));
  atomicAdd(unew_e + (size_t)fa.x * kBulkD + fa.y, (double)sign * ((double)f[4] * 0.125));
}

template <typename T> struct StateArgs {
  const double* uold_d;  // FP64 [oct][5][8]  or the FP32-bulk records' E view (rh_bulk.h)
  const float* uold_f;   // FP32-bulk records
  double* unew_d;
  float* unew_f;
};

constexpr long long kWaitBound = 1ll << 22;  // bounded mbarrier spin (seconds at most)

// Per-thread FP64 CFL / conserved-total accumulation of one new cell
// (courant_fine.f90:317-386 + cmpdt).
// Per-thread courant_fine accumulators.  The cell time step of cmpdt
// (godunov_utils.f90:228-333) is a decreasing function of the cell's summed
// signal speed ctot (dx-scaled constant over ctot, or its gravity form), so
// the thread keeps the largest ctot and converts it once: min over cells of
// dt(ctot) = dt(max ctot), with no division or square root of the dt formula
// per cell.
struct CflAcc {
  double mass = 0, ekin = 0, eint = 0, cmax = 0;
  __device__ __forceinline__ void add(double r, double m1, double m2, double m3, double E, const LevelArgs& A) {
    add(r, m1, m2, m3, E, A.cfl, A.vol);
  }
  __device__ __forceinline__ void add(double r, double m1, double m2, double m3, double E, const CflConst& C,
                                      double vol) {
    mass += r * vol;
    ekin += E * vol;
    const double rm = r > C.smallr ? r : C.smallr;
    const double irm = vrcp(rm);
    double ei = E * vol;
    ei -= 0.5 * (m1 * m1) * irm * vol;
    ei -= 0.5 * (m2 * m2) * irm * vol;
    ei -= 0.5 * (m3 * m3) * irm * vol;
    eint += ei;
    const double u = m1 * irm, v = m2 * irm, w = m3 * irm;
    double e = E - 0.5 * rm * (u * u);
    e = e - 0.5 * rm * (v * v);
    e = e - 0.5 * rm * (w * w);
    double p = C.gm1 * e;
    const double pf = rm * C.smallp;
    p = p > pf ? p : pf;
    const double c = vsqrt(C.gamma * p * irm);
    double ctot = fabs(u) + c;
    if (C.ndim > 1) ctot += fabs(v) + c;
    if (C.ndim > 2) ctot += fabs(w) + c;
    cmax = ctot > cmax ? ctot : cmax;
  }
  // The same quantities for an FP32-bulk cell (density and momenta held in
  // FP32, E in FP64), in fewer FP64 operations: the three sums stay unscaled
  // until scale_bulk multiplies them by the cell volume once, the kinetic
  // energy is (m1^2 + m2^2 + m3^2) / (2 rho) (the squares of FP32 momenta
  // are exact in FP64) and ctot = (|m1| + |m2| + |m3|) / rho + ndim c.
  __device__ __forceinline__ void add_bulk(float rf, float m1f, float m2f, float m3f, double E,
                                           const LevelArgs& A) {
    add_bulk(rf, m1f, m2f, m3f, E, A.cfl);
  }
  __device__ __forceinline__ void add_bulk(float rf, float m1f, float m2f, float m3f, double E,
                                           const CflConst& C) {
    const double r = rf, m1 = m1f, m2 = m2f, m3 = m3f;
    mass += r;
    ekin += E;
    const double rm = r > C.smallr ? r : C.smallr;
    const double irm = vrcp(rm);
    const double e = fma(-0.5 * fma(m1, m1, fma(m2, m2, m3 * m3)), irm, E);
    eint += e;
    double p = C.gm1 * e;
    const double pf = rm * C.smallp;
    p = p > pf ? p : pf;
    const double c = vsqrt(C.gamma * p * irm);
    double a = fabs(m1);
    if (C.ndim > 1) a += fabs(m2);
    if (C.ndim > 2) a += fabs(m3);
    const double ctot = fma(a, irm, (double)C.ndim * c);
    cmax = ctot > cmax ? ctot : cmax;
  }
  __device__ __forceinline__ void scale_bulk(double vol) {
    mass *= vol;
    ekin *= vol;
    eint *= vol;
  }
  // smallest cell dt of the accumulated cells (1e300 when there were none)
  __device__ __forceinline__ double dt(const CflConst& C) const {
    if (!(cmax > 0.0)) return 1e300;
    double d;
    if (C.gsum_dx == 0.0) {
      d = C.k0 / cmax;
    } else {
      double grav = C.gsum_dx / (cmax * cmax);
      grav = grav > 0.0001 ? grav : 0.0001;
      d = C.two_cdx / (cmax * (1.0 + sqrt(1.0 + C.two_c * grav)));
    }
    return d < C.cdx_smallc ? d : C.cdx_smallc;
  }
};

// Deterministic block reduction of the CFL accumulators into the pencil partial.
template <int NWARP>
__device__ __forceinline__ void cfl_block_reduce(const CflAcc& a, const CflConst& C, double* red, double* out) {
  double v[4] = {a.mass, a.ekin, a.eint, a.dt(C)};
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    v[0] += __shfl_down_sync(0xffffffffu, v[0], off);
    v[1] += __shfl_down_sync(0xffffffffu, v[1], off);
    v[2] += __shfl_down_sync(0xffffffffu, v[2], off);
    const double o = __shfl_down_sync(0xffffffffu, v[3], off);
    v[3] = o < v[3] ? o : v[3];
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    red[warp * 4 + 0] = v[0]; red[warp * 4 + 1] = v[1]; red[warp * 4 + 2] = v[2]; red[warp * 4 + 3] = v[3];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0, s1 = 0, s2 = 0, d = 1e300;
    for (int w = 0; w < NWARP; ++w) {
      s0 += red[w * 4 + 0]; s1 += red[w * 4 + 1]; s2 += red[w * 4 + 2];
      d = red[w * 4 + 3] < d ? red[w * 4 + 3] : d;
    }
    out[0] = s0; out[1] = s1; out[2] = s2; out[3] = 0.0; out[4] = d;
  }
}

// Column geometry shared by both kernels: the thread's ring column and, for
// some threads, one outer-ring column (only converted, never traced).  Outer
// tasks are spread over all warps so no warp carries them all.
template <class G> struct Columns {
  int rx, ry, lc, slot;
  CellMap mx, my;
  bool interior, in_domain_xy, in_dom_xy, has_outer;
  int orx, ory, olc, oslot;
  CellMap omx, omy;
  static constexpr int kStride = G::NT / G::NOC > 0 ? G::NT / G::NOC : 1;
  __device__ __forceinline__ void init(int t, int ox0, int oy0, const LevelArgs& A) {
    rx = t % G::RW - 1;
    ry = t / G::RW - 1;
    lc = (rx + 2) + (ry + 2) * G::LW;
    const int gx = 2 * ox0 + rx, gy = 2 * oy0 + ry;
    mx = map_coord(gx, A.ncx, A.periodic[0], A.btype[0], A.btype[1]);
    my = map_coord(gy, A.ncy, A.periodic[1], A.btype[2], A.btype[3]);
    slot = ((rx >> 1) + 1) + G::OW * ((ry >> 1) + 1);
    interior = rx >= 0 && rx < G::CX && ry >= 0 && ry < G::CY;
    in_domain_xy = gx < A.ncx && gy < A.ncy;
    in_dom_xy = gx >= 0 && gy >= 0 && in_domain_xy;
    int o = (t % kStride == 0) ? t / kStride : -1;
    if (o >= G::NOC) o = -1;
    has_outer = o >= 0;
    orx = 0;
    ory = 0;
    if (o >= 0) {
      if (o < G::LW) { orx = o - 2; ory = -2; }
      else if (o < 2 * G::LW) { orx = o - G::LW - 2; ory = G::CY + 1; }
      else if (o < 2 * G::LW + G::RH) { orx = -2; ory = o - 2 * G::LW - 1; }
      else { orx = G::CX + 1; ory = o - 2 * G::LW - G::RH - 1; }
    }
    olc = (orx + 2) + (ory + 2) * G::LW;
    omx = map_coord(2 * ox0 + orx, A.ncx, A.periodic[0], A.btype[0], A.btype[1]);
    omy = map_coord(2 * oy0 + ory, A.ncy, A.periodic[1], A.btype[2], A.btype[3]);
    oslot = ((orx >> 1) + 1) + G::OW * ((ory >> 1) + 1);
  }
};

// Dynamic shared memory of the pencil kernels and the CTA's abort flag (set
// when an mbarrier wait gives up), referenced directly so every access is a
// shared-memory access.
extern __shared__ __align__(16) unsigned char rh_smem[];
__shared__ int rh_s_abort;

// Where a pencil's CFL partial goes.  The grid kernel derives it from the
// kernel parameters at the end (nothing held in registers through the pencil);
// the batch kernel passes the work item's slot.
struct GridCflSink {
  __device__ __forceinline__ bool on(const LevelArgs& A) const { return A.cfl_partial != nullptr; }
  __device__ __forceinline__ double* out(const LevelArgs& A) const { return A.cfl_partial + (size_t)blockIdx.x * 5; }
};
struct SlotCflSink {
  double* const* p;  // shared-memory slot holding the output address
  __device__ __forceinline__ bool on(const LevelArgs&) const { return true; }
  __device__ __forceinline__ double* out(const LevelArgs&) const { return *p; }
};

// Wait for an mbarrier phase, polling at most `bound` times.  A CTA whose
// thread gives up (or sees that another one did) stops waiting, raises the
// CTA's abort flag and sets bit 0 of the device error word, which the host
// reads as RH_ETIMEDOUT; the kernel then runs to its end instead of hanging.
__device__ __forceinline__ bool bounded_mbar_wait(uint64_t* bar, uint32_t par, int* s_abort, int* err,
                                                  long long bound) {
  long long it = 0;
  while (!mbar_try_wait(bar, par)) {
    if (*s_abort || ++it > bound) {
      if (!*s_abort) {
        *s_abort = 1;
        atomicOr(err, 1);
      }
      return false;
    }
  }
  return true;
}

// Bulk-async staging of the oct layers of a pencil.
template <typename T, class G, bool DENSE = false> struct Stager {
  double* stageD;
  float* stageF;
  uint64_t* bar;
  int* s_abort;
  const int* tab;         // pencil table; DENSE: [NSLOT] xy offsets then [L+2] z offsets
  const double* src_d;
  const float* src_f;
  int* err;
  int rbase;              // layers staged by earlier pencils of this CTA (barrier phases continue)
  __device__ __forceinline__ int rb() const { return DENSE ? rbase : 0; }
  // Oct index at table row (layer) row, oct column slot of the pencil.
  __device__ __forceinline__ int oct_at(int row, int slot) const {
    if (!DENSE) return tab[(long long)row * G::NSLOT + slot];
    return tab[G::NSLOT + row] + tab[slot];
  }
  __device__ __forceinline__ void init_barriers() {
    if (threadIdx.x == 0) {
      *s_abort = 0;
      for (int s = 0; s < G::NSTAGE; ++s) mbar_init(&bar[s], G::NSLOT);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
  }
  // The table entry this thread's copy of layer row reads (-1 for threads
  // that issue none): loaded ahead of issue(row, oct), the copy does not wait
  // for the table read.
  __device__ __forceinline__ int entry(int row) const {
    return threadIdx.x < G::NSLOT ? oct_at(row, threadIdx.x) : -1;
  }
  __device__ __forceinline__ void issue(int row) { issue(row, entry(row)); }
  __device__ __forceinline__ void issue(int row, int oct) {
    const int t = threadIdx.x;
    if (t < G::NSLOT) {
      const int st = (rb() + row) % G::NSTAGE;
      fence_proxy_async_smem();
      if (oct >= 0) {
        mbar_arrive_expect_tx(&bar[st], Store<T>::kBytes);
        if (sizeof(T) == 8) {
          bulk_g2s(stageD + ((size_t)st * G::NSLOT + t) * Store<T>::kSlotD, src_d + (size_t)oct * 40, 320, &bar[st]);
        } else {
          bulk_g2s(stageF + ((size_t)st * G::NSLOT + t) * Store<T>::kSlotF, src_f + (size_t)oct * kBulkF, kBulkBytes,
                   &bar[st]);
        }
      } else {
        mbar_arrive_expect_tx(&bar[st], 0);
      }
    }
  }
  __device__ __forceinline__ void wait(int row) {
    const int st = (rb() + row) % G::NSTAGE;
    const uint32_t par = ((rb() + row) / G::NSTAGE) & 1;
    bounded_mbar_wait(&bar[st], par, s_abort, err, kWaitBound);
  }
  __device__ __forceinline__ const double* slot_d(int row, int slot) const {
    if (sizeof(T) == 4)  // FP32-bulk: the staged record's E, after its 32 floats
      return reinterpret_cast<const double*>(slot_f(row, slot) + 32);
    return stageD + ((size_t)((rb() + row) % G::NSTAGE) * G::NSLOT + slot) * Store<T>::kSlotD;
  }
  __device__ __forceinline__ const float* slot_f(int row, int slot) const {
    return stageF + ((size_t)((rb() + row) % G::NSTAGE) * G::NSLOT + slot) * Store<T>::kSlotF;
  }
};

// FP64 ctoprim of one cell (umuscl.f90:1739-1901) from a staged oct record;
// q[5] = (rho, u, v, w, p), also returns 1/rho and the conserved values.
__device__ __forceinline__ void ctoprim_f64(const double* sd, int cell, bool fx, bool fy, bool fz,
                                            const HydroK<double>& H, double* q, double& ir, double* U) {
  double d = sd[cell], mx = sd[8 + cell], my = sd[16 + cell], mz = sd[24 + cell], E = sd[32 + cell];
  if (fx) mx = -mx;
  if (fy) my = -my;
  if (fz) mz = -mz;
  U[0] = d; U[1] = mx; U[2] = my; U[3] = mz; U[4] = E;
  const double r = d > H.smallr ? d : H.smallr;
  ir = vrcp(r);
  const double u = mx * ir, v = my * ir, w = mz * ir;
  const double ekin = (0.5 * r) * fma(u, u, fma(v, v, w * w));
  double eint = E - ekin;
  const double emin = H.smalle * r;
  eint = eint > emin ? eint : emin;
  q[0] = r;
  q[1] = u + H.grav[0];
  q[2] = v + H.grav[1];
  q[3] = w + H.grav[2];
  q[4] = H.gm1 * eint;
}

// One pencil of the plain FP64 step for a persistent CTA: the mbarriers are
// set up once per CTA and rbase counts the layers its earlier pencils staged.
template <typename T, int TXO, int TYO, int SLOPE, int RIEMANN, bool AMR, bool DENSE, class Sink>
__device__ __forceinline__ void pencil_body_f64(const LevelArgs& A, const StateArgs<T>& S, const HydroK<double>& H,
                                                const int4 hdr, const int* tab, int rbase, const Sink sink) {
  constexpr bool init_barriers = false;
#include "rh_pencil_f64.inc"
}

// One pencil per CTA (the level's pencil table gives hdr and tab).
template <typename T, int TXO, int TYO, int MINB, int SLOPE, int RIEMANN, bool AMR>
__global__ void __launch_bounds__(Geo<T, double, TXO, TYO>::NT, MINB)
godunov_pencil_kernel(const LevelArgs A, const StateArgs<T> S, const HydroK<double> H) {
  constexpr bool DENSE = false;
  constexpr bool init_barriers = true;
  constexpr int rbase = 0;
  const GridCflSink sink{};
  const int4 hdr = A.phdr[blockIdx.x];
  const int* tab = A.ptab + A.poff[blockIdx.x];
#include "rh_pencil_f64.inc"
}

}  // namespace rh
