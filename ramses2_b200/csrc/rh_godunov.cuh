// rh_godunov.cuh — the fused MUSCL-Hancock Godunov kernel (sm_100a).
//
// One CTA owns a "pencil": an XY tile of TXO x TYO octs and a run of L oct
// layers along z.  It marches through the pencil one cell plane at a time:
//
//   * the pencil's oct table lists, for each of the L+2 layers (one halo layer
//     each side) and each of the (TXO+2)(TYO+2) oct columns, the index of the
//     oct whose cells fill that position (boundary sources already resolved);
//   * each layer's oct records are staged into shared memory by bulk async
//     copies (cp.async.bulk, one 320-byte oct record per copy, completion on an
//     mbarrier), two layers in flight, so the gather through the oct table
//     runs ahead of the arithmetic;
//   * one thread per "ring" column ((2TXO+2) x (2TYO+2) cell columns) converts
//     its cell to primitive variables (ctoprim), keeps the z-neighbours in
//     registers, takes x/y neighbours from a shared plane buffer, and computes
//     slopes, the normal-velocity bound and the Hancock predictor (uslope +
//     trace3d) for its cell;
//   * x/y interface states are exchanged through shared memory, z interface
//     states never leave the thread; Riemann fluxes of the three directions
//     (cmpflxm + llf/hll/hllc) and the conservative update of the oct cells
//     (godunov_fine.f90:733-816: x, then y, then z differences) follow;
//   * the epilogue evaluates the CFL time step and the conserved totals of
//     the new state (courant_fine + cmpdt), reduced per CTA with warp
//     shuffles into a per-pencil partial, so the next step's dt costs no pass.
//
// This replaces the reference's per-subgrid hydro_integrator_kernel
// (gpu/gpu_hydro.cuf:8776-8964), which materialises the whole (2n+4)^3
// stencil and all face states in shared memory.
#pragma once
#include "rh_device.cuh"
#include "ramses_hydro.h"

namespace rh {

// Storage policy of a precision mode.
template <typename T> struct Store;
template <> struct Store<double> {  // plain FP64: reference layout [oct][5][8]
  static constexpr int kSlotF = 0;   // floats per staged oct
  static constexpr int kSlotD = 42;  // doubles per staged oct (40 + pad)
  static constexpr uint32_t kBytes = 320;
};
template <> struct Store<float> {  // FP32-bulk: [oct][4][8] float + [oct][8] double (E)
  static constexpr int kSlotF = 36;  // 32 + pad
  static constexpr int kSlotD = 10;  // 8 + pad
  static constexpr uint32_t kBytes = 128 + 64;
};

template <typename T, int TXO, int TYO> struct Geo {
  static constexpr int CX = 2 * TXO, CY = 2 * TYO;
  static constexpr int RW = CX + 2, RH = CY + 2;         // ring columns
  static constexpr int NRC = RW * RH;                     // threads per CTA
  static constexpr int LW = CX + 4, LH = CY + 4;          // load columns
  static constexpr int NLC = LW * LH;
  static constexpr int NOC = NLC - NRC;                   // outer ring columns
  static constexpr int OW = TXO + 2, OH = TYO + 2;        // oct columns per layer
  static constexpr int NSLOT = OW * OH;
  static constexpr int NWARP = (NRC + 31) / 32;
  static constexpr int NT = NWARP * 32;                   // block size (full warps)
  static constexpr int NSTAGE = 2;
  // shared memory carve-up (bytes, 16-aligned sections)
  static constexpr size_t kStageD = (size_t)NSTAGE * NSLOT * Store<T>::kSlotD * sizeof(double);
  static constexpr size_t kStageF = (size_t)NSTAGE * NSLOT * Store<T>::kSlotF * sizeof(float);
  static constexpr size_t kQ = (size_t)2 * 5 * NLC * sizeof(T);
  static constexpr size_t kFS = (size_t)10 * NRC * sizeof(T);
  static constexpr size_t kFX = (size_t)2 * 5 * NRC * sizeof(T);
  static constexpr size_t kRed = (size_t)NWARP * 4 * sizeof(double);
  static constexpr size_t a16(size_t x) { return (x + 15) & ~size_t(15); }
  static constexpr size_t oStageD = 0;
  static constexpr size_t oStageF = a16(oStageD + kStageD);
  static constexpr size_t oQ = a16(oStageF + kStageF);
  static constexpr size_t oFS = a16(oQ + kQ);
  static constexpr size_t oFX = a16(oFS + kFS);
  static constexpr size_t oRed = a16(oFX + kFX);
  static constexpr size_t oBar = a16(oRed + kRed);
  static constexpr size_t kSmem = oBar + 64;
};

// Boundary mapping of one global cell coordinate: parity of the source cell
// inside the (already resolved) source oct and the sign of the normal velocity.
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

template <typename T> struct Prim5 { T r, u, v, w, p; };

// Conserved (from the staged oct) -> primitive, ctoprim (umuscl.f90:1739-1901).
// The FP32-bulk path recovers the pressure in FP64 from the FP64 energy.
template <typename T> __device__ __forceinline__ Prim5<T> load_prim(const float* sf, const double* sd, int cell,
                                                                   bool fx, bool fy, bool fz,
                                                                   const HydroConst<T>& H, T* U5,
                                                                   double& E64);

template <> __device__ __forceinline__ Prim5<double> load_prim<double>(const float*, const double* sd, int cell,
                                                                       bool fx, bool fy, bool fz,
                                                                       const HydroConst<double>& H,
                                                                       double* U5, double& E64) {
  double d = sd[cell], mx = sd[8 + cell], my = sd[16 + cell], mz = sd[24 + cell], E = sd[32 + cell];
  if (fx) mx = -mx;
  if (fy) my = -my;
  if (fz) mz = -mz;
  U5[0] = d; U5[1] = mx; U5[2] = my; U5[3] = mz; U5[4] = E;
  E64 = E;
  Prim5<double> q;
  double r = d > H.smallr ? d : H.smallr;
  double ir = 1.0 / r;
  double u = mx * ir, v = my * ir, w = mz * ir;
  double ekin = 0.5 * r * (u * u);
  ekin = ekin + 0.5 * r * (v * v);
  ekin = ekin + 0.5 * r * (w * w);
  double eint = E - ekin;
  double emin = H.smalle * r;
  eint = eint > emin ? eint : emin;
  q.r = r;
  q.p = H.gm1 * eint;
  q.u = u + H.grav_half_dt[0];
  q.v = v + H.grav_half_dt[1];
  q.w = w + H.grav_half_dt[2];
  return q;
}

template <> __device__ __forceinline__ Prim5<float> load_prim<float>(const float* sf, const double* sd, int cell,
                                                                     bool fx, bool fy, bool fz,
                                                                     const HydroConst<float>& H, float* U5,
                                                                     double& E64) {
  float d = sf[cell], mx = sf[8 + cell], my = sf[16 + cell], mz = sf[24 + cell];
  double E = sd[cell];
  if (fx) mx = -mx;
  if (fy) my = -my;
  if (fz) mz = -mz;
  U5[0] = d; U5[1] = mx; U5[2] = my; U5[3] = mz; U5[4] = 0.f;
  E64 = E;
  Prim5<float> q;
  float r = d > H.smallr ? d : H.smallr;
  float ir = __frcp_rn(r);
  float u = mx * ir, v = my * ir, w = mz * ir;
  // pressure recovery in FP64: eint = E - ekin (high-Mach / near-vacuum cells)
  double rd = (double)r, ud = (double)u, vd = (double)v, wd = (double)w;
  double ekin = 0.5 * rd * (ud * ud + vd * vd + wd * wd);
  double eint = E - ekin;
  double emin = (double)H.smalle * rd;
  eint = eint > emin ? eint : emin;
  q.r = r;
  q.p = (float)((double)H.gm1 * eint);
  q.u = u + H.grav_half_dt[0];
  q.v = v + H.grav_half_dt[1];
  q.w = w + H.grav_half_dt[2];
  return q;
}

template <typename T, int RIEMANN> __device__ __forceinline__ void solve_face(const T* ql, const T* qr, T* f,
                                                                              const HydroConst<T>& H) {
  riemann<T, RIEMANN>(ql, qr, f, H);
#pragma unroll
  for (int n = 0; n < 5; ++n) f[n] *= H.dtdx;
}

// Device-wide constants of one level launch.
struct LevelArgs {
  const int4* phdr;            // per pencil: ox0, oy0, oz0, L
  const long long* poff;       // per pencil: offset of its table in ptab
  const int* ptab;             // (L+2) x NSLOT oct indices (0-based; <0 absent)
  int npencil;
  int ncx, ncy, ncz;           // level extent in cells
  int periodic[3];
  int btype[6];
  int ghost_base;              // entries >= ghost_base are never updated
  double* cfl_partial;         // [npencil][5] (mass, ekin, eint, emag, dt) or null
  int* err;                    // device error word (bit 0: mbarrier wait timed out)
  CflConst cfl;
  double vol;
};

template <typename T> struct StateArgs {
  const double* uold_d;  // FP64 [oct][5][8]  or FP32-bulk energy [oct][8]
  const float* uold_f;   // FP32-bulk [oct][4][8]
  double* unew_d;
  float* unew_f;
};

constexpr long long kWaitBound = 1ll << 22;  // bounded mbarrier spin (seconds at most)

template <typename T, int TXO, int TYO, int SLOPE, int RIEMANN>
__global__ void __launch_bounds__(Geo<T, TXO, TYO>::NT, 1)
godunov_pencil_kernel(const LevelArgs A, const StateArgs<T> S, const HydroConst<T> H) {
  using G = Geo<T, TXO, TYO>;
  extern __shared__ __align__(16) unsigned char smem[];
  double* stageD = reinterpret_cast<double*>(smem + G::oStageD);
  float* stageF = reinterpret_cast<float*>(smem + G::oStageF);
  T* Qb = reinterpret_cast<T*>(smem + G::oQ);    // [2][5][NLC]
  T* FS = reinterpret_cast<T*>(smem + G::oFS);   // [10][NRC]: qp_x(5), qp_y(5)
  T* FXY = reinterpret_cast<T*>(smem + G::oFX);  // [2][5][NRC]: x then y fluxes
  double* red = reinterpret_cast<double*>(smem + G::oRed);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + G::oBar);
  __shared__ int s_abort;

  const int t = threadIdx.x;
  const int pencil = blockIdx.x;
  const int4 hdr = A.phdr[pencil];
  const int ox0 = hdr.x, oy0 = hdr.y, oz0 = hdr.z, L = hdr.w;
  const int CZ = 2 * L;
  const int* tab = A.ptab + A.poff[pencil];

  // ---- per-thread column geometry ------------------------------------------------
  const int rx = t % G::RW - 1, ry = t / G::RW - 1;  // ring column
  const int lc = (rx + 2) + (ry + 2) * G::LW;        // load-column index
  const int gx = 2 * ox0 + rx, gy = 2 * oy0 + ry;
  const CellMap mx = map_coord(gx, A.ncx, A.periodic[0], A.btype[0], A.btype[1]);
  const CellMap my = map_coord(gy, A.ncy, A.periodic[1], A.btype[2], A.btype[3]);
  const int slot = ((rx >> 1) + 1) + G::OW * ((ry >> 1) + 1);
  const bool interior = rx >= 0 && rx < G::CX && ry >= 0 && ry < G::CY;
  const bool in_domain_xy = gx < A.ncx && gy < A.ncy;
  // outer-ring column handled by this thread (t < NOC)
  int orx = 0, ory = 0;
  if (t < G::NOC) {
    int o = t;
    if (o < G::LW) { orx = o - 2; ory = -2; }
    else if (o < 2 * G::LW) { orx = o - G::LW - 2; ory = G::CY + 1; }
    else if (o < 2 * G::LW + G::RH) { orx = -2; ory = o - 2 * G::LW - 1; }
    else { orx = G::CX + 1; ory = o - 2 * G::LW - G::RH - 1; }
  }
  const int olc = (orx + 2) + (ory + 2) * G::LW;
  const CellMap omx = map_coord(2 * ox0 + orx, A.ncx, A.periodic[0], A.btype[0], A.btype[1]);
  const CellMap omy = map_coord(2 * oy0 + ory, A.ncy, A.periodic[1], A.btype[2], A.btype[3]);
  const int oslot = ((orx >> 1) + 1) + G::OW * ((ory >> 1) + 1);

  // ---- TMA staging of oct layers ------------------------------------------------------
  if (t == 0) {
    s_abort = 0;
    for (int s = 0; s < G::NSTAGE; ++s) mbar_init(&bar[s], G::NSLOT);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto issue_row = [&](int row) {
    if (t < G::NSLOT) {
      const int st = row % G::NSTAGE;
      const int oct = tab[(long long)row * G::NSLOT + t];
      fence_proxy_async_smem();
      if (oct >= 0) {
        mbar_arrive_expect_tx(&bar[st], Store<T>::kBytes);
        if (sizeof(T) == 8) {
          bulk_g2s(stageD + ((size_t)st * G::NSLOT + t) * Store<T>::kSlotD, S.uold_d + (size_t)oct * 40, 320,
                   &bar[st]);
        } else {
          bulk_g2s(stageF + ((size_t)st * G::NSLOT + t) * Store<T>::kSlotF, S.uold_f + (size_t)oct * 32, 128,
                   &bar[st]);
          bulk_g2s(stageD + ((size_t)st * G::NSLOT + t) * Store<T>::kSlotD, S.uold_d + (size_t)oct * 8, 64,
                   &bar[st]);
        }
      } else {
        mbar_arrive_expect_tx(&bar[st], 0);
      }
    }
  };
  auto wait_row = [&](int row) {
    const int st = row % G::NSTAGE;
    const uint32_t par = (row / G::NSTAGE) & 1;
    long long it = 0;
    while (!mbar_try_wait(&bar[st], par)) {
      if (s_abort || ++it > kWaitBound) {
        if (!s_abort) { s_abort = 1; atomicOr(A.err, 1); }
        break;
      }
    }
  };
  issue_row(0);
  if (L + 1 >= 1) issue_row(1);

  // Convert plane p of a column to primitive; returns the primitive state,
  // the conserved values (U5, E64) and whether the column exists.
  auto plane_zmap = [&](int p) { return map_coord(2 * oz0 + p, A.ncz, A.periodic[2], A.btype[4], A.btype[5]); };
  auto stage_ptrs = [&](int p, int sl, const float*& sf, const double*& sd) {
    const int row = (p >> 1) + 1;
    const int st = row % G::NSTAGE;
    sd = stageD + ((size_t)st * G::NSLOT + sl) * Store<T>::kSlotD;
    sf = stageF + ((size_t)st * G::NSLOT + sl) * Store<T>::kSlotF;
  };

  Prim5<T> qa, qb, qc;           // own column at planes k-1, k, k+1
  T Uk[5], Uk1[5];               // uold of own cell at planes k, k+1 (bulk part)
  double Ek = 0, Ek1 = 0;        // FP64 energy at planes k, k+1
  T qmx[5], qmy[5], qmz_prev[5]; // left states kept in registers
  T fz_prev[5];
  T up[5];                       // pending update of plane k-1 (x and y differences added)
  double upE = 0;                // FP64 energy of the pending update
  double fzE_prev = 0;           // (unused for FP64; FP32-bulk keeps z energy flux in T)
  (void)fzE_prev;
  double s_mass = 0, s_ekin = 0, s_eint = 0, s_dt = 1e300;
#pragma unroll
  for (int n = 0; n < 5; ++n) { qmz_prev[n] = T(0); fz_prev[n] = T(0); up[n] = T(0); Uk[n] = T(0); Uk1[n] = T(0); }

  // ---- prologue: planes -2 and -1 ------------------------------------------------------
  wait_row(0);
  for (int p = -2; p <= -1; ++p) {
    const CellMap mz = plane_zmap(p);
    const float* sf;
    const double* sd;
    if (t < G::NRC) {
      stage_ptrs(p, slot, sf, sd);
      T U5[5];
      double E64;
      Prim5<T> q = load_prim<T>(sf, sd, mx.parity + 2 * my.parity + 4 * mz.parity, mx.flip, my.flip, mz.flip, H,
                                U5, E64);
      if (p == -2) qa = q; else qb = q;
      if (p == -1) {
        T* Qp = Qb + (size_t)(p & 1) * 5 * G::NLC;
        Qp[0 * G::NLC + lc] = q.r; Qp[1 * G::NLC + lc] = q.u; Qp[2 * G::NLC + lc] = q.v;
        Qp[3 * G::NLC + lc] = q.w; Qp[4 * G::NLC + lc] = q.p;
      }
    }
    if (t < G::NOC && p == -1) {
      stage_ptrs(p, oslot, sf, sd);
      T U5[5];
      double E64;
      Prim5<T> q = load_prim<T>(sf, sd, omx.parity + 2 * omy.parity + 4 * mz.parity, omx.flip, omy.flip,
                                mz.flip, H, U5, E64);
      T* Qp = Qb + (size_t)(p & 1) * 5 * G::NLC;
      Qp[0 * G::NLC + olc] = q.r; Qp[1 * G::NLC + olc] = q.u; Qp[2 * G::NLC + olc] = q.v;
      Qp[3 * G::NLC + olc] = q.w; Qp[4 * G::NLC + olc] = q.p;
    }
  }
  __syncthreads();
  if (L + 1 >= 2) issue_row(2);

  const bool thread_active = t < G::NRC;

  // ---- march -------------------------------------------------------------------------
  for (int k = -1; k <= CZ; ++k) {
    // (A) primitive variables of plane k+1
    {
      const int p = k + 1;
      const int row = (p >> 1) + 1;
      if ((p & 1) == 0) wait_row(row);
      const CellMap mz = plane_zmap(p);
      const float* sf;
      const double* sd;
      T* Qp = Qb + (size_t)(p & 1) * 5 * G::NLC;
      if (thread_active) {
        stage_ptrs(p, slot, sf, sd);
        double E64;
        qc = load_prim<T>(sf, sd, mx.parity + 2 * my.parity + 4 * mz.parity, mx.flip, my.flip, mz.flip, H, Uk1,
                          E64);
        Ek1 = E64;
        Qp[0 * G::NLC + lc] = qc.r; Qp[1 * G::NLC + lc] = qc.u; Qp[2 * G::NLC + lc] = qc.v;
        Qp[3 * G::NLC + lc] = qc.w; Qp[4 * G::NLC + lc] = qc.p;
      }
      if (t < G::NOC) {
        stage_ptrs(p, oslot, sf, sd);
        T U5[5];
        double E64;
        Prim5<T> q = load_prim<T>(sf, sd, omx.parity + 2 * omy.parity + 4 * mz.parity, omx.flip, omy.flip,
                                  mz.flip, H, U5, E64);
        Qp[0 * G::NLC + olc] = q.r; Qp[1 * G::NLC + olc] = q.u; Qp[2 * G::NLC + olc] = q.v;
        Qp[3 * G::NLC + olc] = q.w; Qp[4 * G::NLC + olc] = q.p;
      }
    }
    // (C) slopes, predictor and interface states of plane k (Q of plane k is
    // complete since the previous iteration's barriers)
    T fz[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) fz[n] = T(0);
    if (thread_active) {
      const T* Qk = Qb + (size_t)(k & 1) * 5 * G::NLC;
      const T q0[5] = {qb.r, qb.u, qb.v, qb.w, qb.p};
      const T qzm[5] = {qa.r, qa.u, qa.v, qa.w, qa.p};
      const T qzp[5] = {qc.r, qc.u, qc.v, qc.w, qc.p};
      T xm[5], xp[5], ym[5], yp[5];
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        xm[n] = Qk[n * G::NLC + lc - 1];
        xp[n] = Qk[n * G::NLC + lc + 1];
        ym[n] = Qk[n * G::NLC + lc - G::LW];
        yp[n] = Qk[n * G::NLC + lc + G::LW];
      }
      T dx_[5], dy_[5], dz_[5];
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        dx_[n] = limited_slope<T, SLOPE>(xm[n], q0[n], xp[n]);
        dy_[n] = limited_slope<T, SLOPE>(ym[n], q0[n], yp[n]);
        dz_[n] = limited_slope<T, SLOPE>(qzm[n], q0[n], qzp[n]);
      }
      const T ir = Num<T>::rcp(q0[0]);
      if (SLOPE > 0) {
        dx_[1] = momentum_bound(dx_[1], xm[0], xm[1], q0[1], xp[0], xp[1], ir);
        dy_[2] = momentum_bound(dy_[2], ym[0], ym[2], q0[2], yp[0], yp[2], ir);
        dz_[3] = momentum_bound(dz_[3], qzm[0], qzm[3], q0[3], qzp[0], qzp[3], ir);
      }
      // trace3d (umuscl.f90:966-1234)
#pragma unroll
      for (int n = 0; n < 5; ++n) { dx_[n] *= T(0.5); dy_[n] *= T(0.5); dz_[n] *= T(0.5); }
      const T r = q0[0], u = q0[1], v = q0[2], w = q0[3], p = q0[4];
      const T divv = dx_[1] + dy_[2] + dz_[3];
      const T sr0 = -u * dx_[0] - v * dy_[0] - w * dz_[0] - divv * r;
      const T su0 = -u * dx_[1] - v * dy_[1] - w * dz_[1] - dx_[4] * ir;
      const T sv0 = -u * dx_[2] - v * dy_[2] - w * dz_[2] - dy_[4] * ir;
      const T sw0 = -u * dx_[3] - v * dy_[3] - w * dz_[3] - dz_[4] * ir;
      const T sp0 = -u * dx_[4] - v * dy_[4] - w * dz_[4] - divv * H.gamma * p;
      const T pr[5] = {r + sr0 * H.dtdx, u + su0 * H.dtdx, v + sv0 * H.dtdx, w + sw0 * H.dtdx, p + sp0 * H.dtdx};
      T qpx[5], qpy[5], qpz[5], qmzc[5];
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        qpx[n] = pr[n] - dx_[n]; qmx[n] = pr[n] + dx_[n];
        qpy[n] = pr[n] - dy_[n]; qmy[n] = pr[n] + dy_[n];
        qpz[n] = pr[n] - dz_[n]; qmzc[n] = pr[n] + dz_[n];
      }
      // floors (umuscl.f90:1141-1232)
      if (qpx[0] < H.smallr) qpx[0] = r;
      if (qpx[4] < H.smallp_trace) qpx[4] = p;
      if (qmx[0] < H.smallr) qmx[0] = r;
      if (qmx[4] < H.smallp_trace) qmx[4] = p;
      if (qpy[0] < H.smallr) qpy[0] = r;
      if (qpy[4] < H.smallp_trace) qpy[4] = p;
      if (qmy[0] < H.smallr) qmy[0] = r;
      if (qmy[4] < H.smallp_trace) qmy[4] = p;
      if (qpz[0] < H.smallr) qpz[0] = r;
      if (qpz[4] < H.smallp_trace) qpz[4] = p;
      if (qmzc[0] < H.smallr) qmzc[0] = r;
      if (qmzc[4] < H.smallp_trace) qmzc[4] = p;
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        FS[n * G::NRC + t] = qpx[n];
        FS[(5 + n) * G::NRC + t] = qpy[n];
      }
      // z interface k-1/2: left = qm_z(k-1), right = qp_z(k); rotation (r,w,u,v,p)
      if (interior && k >= 0) {
        const T ql[5] = {qmz_prev[0], qmz_prev[3], qmz_prev[1], qmz_prev[2], qmz_prev[4]};
        const T qr[5] = {qpz[0], qpz[3], qpz[1], qpz[2], qpz[4]};
        T f[5];
        solve_face<T, RIEMANN>(ql, qr, f, H);
        fz[0] = f[0]; fz[3] = f[1]; fz[1] = f[2]; fz[2] = f[3]; fz[4] = f[4];
      }
#pragma unroll
      for (int n = 0; n < 5; ++n) qmz_prev[n] = qmzc[n];
    }
    __syncthreads();  // S2: interface states of plane k published
    if (k >= 0 && (k & 1) == 0 && k / 2 + 3 <= L + 1) issue_row(k / 2 + 3);
    // (D) x flux at the right face and y flux at the top face of the own cell
    const bool plane_ok = k >= 0 && k < CZ;
    if (thread_active && plane_ok) {
      if (rx >= -1 && rx < G::CX && ry >= 0 && ry < G::CY) {
        const T ql[5] = {qmx[0], qmx[1], qmx[2], qmx[3], qmx[4]};
        const T qr[5] = {FS[0 * G::NRC + t + 1], FS[1 * G::NRC + t + 1], FS[2 * G::NRC + t + 1],
                         FS[3 * G::NRC + t + 1], FS[4 * G::NRC + t + 1]};
        T f[5];
        solve_face<T, RIEMANN>(ql, qr, f, H);
#pragma unroll
        for (int n = 0; n < 5; ++n) FXY[n * G::NRC + t] = f[n];
      }
      if (ry >= -1 && ry < G::CY && rx >= 0 && rx < G::CX) {
        const int tn = t + G::RW;
        const T ql[5] = {qmy[0], qmy[2], qmy[1], qmy[3], qmy[4]};
        const T qr[5] = {FS[5 * G::NRC + tn], FS[7 * G::NRC + tn], FS[6 * G::NRC + tn], FS[8 * G::NRC + tn],
                         FS[9 * G::NRC + tn]};
        T f[5];
        solve_face<T, RIEMANN>(ql, qr, f, H);
        T* FY = FXY + 5 * G::NRC;
        FY[0 * G::NRC + t] = f[0];
        FY[2 * G::NRC + t] = f[1];
        FY[1 * G::NRC + t] = f[2];
        FY[3 * G::NRC + t] = f[3];
        FY[4 * G::NRC + t] = f[4];
      }
    }
    __syncthreads();  // S3: fluxes of plane k published
    // (E) updates: finish plane k-1 with its z differences, start plane k
    if (thread_active && interior) {
      const int pk = k - 1;
      if (pk >= 0 && pk < CZ) {
        const int gz = 2 * oz0 + pk;
        const int oct = tab[(long long)((pk >> 1) + 1) * G::NSLOT + slot];
        if (in_domain_xy && gz < A.ncz && oct >= 0 && oct < A.ghost_base) {
          const int cell = (rx & 1) + 2 * (ry & 1) + 4 * (pk & 1);
          T un[5];
#pragma unroll
          for (int n = 0; n < 5; ++n) un[n] = up[n] + (fz_prev[n] - fz[n]);
          double En;
          if (sizeof(T) == 8) {
            En = (double)un[4];
            double* o = S.unew_d + (size_t)oct * 40 + cell;
            o[0] = (double)un[0]; o[8] = (double)un[1]; o[16] = (double)un[2]; o[24] = (double)un[3]; o[32] = En;
          } else {
            En = upE + (double)(fz_prev[4] - fz[4]);
            float* o = S.unew_f + (size_t)oct * 32 + cell;
            o[0] = (float)un[0]; o[8] = (float)un[1]; o[16] = (float)un[2]; o[24] = (float)un[3];
            S.unew_d[(size_t)oct * 8 + cell] = En;
          }
          if (A.cfl_partial) {
            const double rr = (double)un[0], m1 = (double)un[1], m2 = (double)un[2], m3 = (double)un[3];
            s_mass += rr * A.vol;
            s_ekin += En * A.vol;
            const double rm = rr > A.cfl.smallr ? rr : A.cfl.smallr;
            double ei = En * A.vol;
            ei -= 0.5 * (m1 * m1) / rm * A.vol;
            ei -= 0.5 * (m2 * m2) / rm * A.vol;
            ei -= 0.5 * (m3 * m3) / rm * A.vol;
            s_eint += ei;
            const double dtc = cmpdt_cell(rr, m1, m2, m3, En, A.cfl);
            s_dt = dtc < s_dt ? dtc : s_dt;
          }
        }
      }
      if (plane_ok) {
        const T* FX = FXY;
        const T* FY = FXY + 5 * G::NRC;
#pragma unroll
        // uold(k) is in Uk (bulk) / Ek (energy), loaded one iteration ago
#pragma unroll
        for (int n = 0; n < 5; ++n) {
          T u0 = Uk[n];
          u0 = u0 + (FX[n * G::NRC + t - 1] - FX[n * G::NRC + t]);
          u0 = u0 + (FY[n * G::NRC + t - G::RW] - FY[n * G::NRC + t]);
          up[n] = u0;
        }
        if (sizeof(T) == 4) {
          double e0 = Ek;
          e0 = e0 + (double)(FX[4 * G::NRC + t - 1] - FX[4 * G::NRC + t]);
          e0 = e0 + (double)(FY[4 * G::NRC + t - G::RW] - FY[4 * G::NRC + t]);
          upE = e0;
        }
      }
    }
#pragma unroll
    for (int n = 0; n < 5; ++n) { fz_prev[n] = fz[n]; Uk[n] = Uk1[n]; }
    Ek = Ek1;
    qa = qb;
    qb = qc;
  }

  // ---- CFL / conservation epilogue: deterministic block reduction -----------------
  if (A.cfl_partial) {
    double v[4] = {s_mass, s_ekin, s_eint, s_dt};
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      v[0] += __shfl_down_sync(0xffffffffu, v[0], off);
      v[1] += __shfl_down_sync(0xffffffffu, v[1], off);
      v[2] += __shfl_down_sync(0xffffffffu, v[2], off);
      const double o = __shfl_down_sync(0xffffffffu, v[3], off);
      v[3] = o < v[3] ? o : v[3];
    }
    const int warp = t >> 5, lane = t & 31;
    if (lane == 0) {
      red[warp * 4 + 0] = v[0]; red[warp * 4 + 1] = v[1]; red[warp * 4 + 2] = v[2]; red[warp * 4 + 3] = v[3];
    }
    __syncthreads();
    if (t == 0) {
      double a = 0, b = 0, c = 0, d = 1e300;
      for (int w = 0; w < G::NWARP; ++w) {
        a += red[w * 4 + 0]; b += red[w * 4 + 1]; c += red[w * 4 + 2];
        d = red[w * 4 + 3] < d ? red[w * 4 + 3] : d;
      }
      double* o = A.cfl_partial + (size_t)pencil * 5;
      o[0] = a; o[1] = b; o[2] = c; o[3] = 0.0; o[4] = d;
    }
  }
}

}  // namespace rh
