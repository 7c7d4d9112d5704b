// rh_device.cuh — device-side physics of the Godunov step and PTX helpers.
//
// The physics restates RAMSES II's CPU routines (hydro/umuscl.f90,
// hydro/godunov_utils.f90) cell by cell, with the same branch structure and
// floors, templated on the bulk arithmetic type T (double: plain FP64 path;
// float: FP32-bulk path).  Divisions by the same quantity are replaced by one
// reciprocal and FMA contraction is allowed: both change results by a few
// ulps, far inside the 1e-12 relative-L1 parity bar of the FP64 path.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "rh_bulk.h"

namespace rh {

// ---------------------------------------------------------------------------
// Small helpers
// ---------------------------------------------------------------------------
template <typename T> struct Num;
template <> struct Num<double> {
  static __device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
  static __device__ __forceinline__ double rcp(double x) { return 1.0 / x; }
};
template <> struct Num<float> {
  static __device__ __forceinline__ float sqrt_(float x) { return sqrtf(x); }
  static __device__ __forceinline__ float rcp(float x) { return __frcp_rn(x); }
};

template <typename T> __device__ __forceinline__ T tmin(T a, T b) { return a < b ? a : b; }  // Fortran MIN
template <typename T> __device__ __forceinline__ T tmax(T a, T b) { return a > b ? a : b; }  // Fortran MAX

// Hydro constants handed to every kernel (one copy per launch, by value).
template <typename T> struct HydroConst {
  T gamma, gm1, entho;      // gamma, gamma-1, 1/(gamma-1)
  T smallr, smallc, smallc2;
  T smallp_trace;           // smallr*smallc**2            (umuscl.f90:931)
  T smallp_riem;            // smallc**2/gamma             (godunov_utils.f90:363,511,676)
  T smalle;                 // smallc**2/gamma/(gamma-1)   (umuscl.f90:1778)
  T dtdx, half_dtdx_unused, smax_cap;
  T grav_half_dt[3];        // constant_gravity*dt/2 (ctoprim predictor)
};

// ---------------------------------------------------------------------------
// Slope limiters, umuscl.f90:2132-2206
// ---------------------------------------------------------------------------
template <typename T, int SLOPE> __device__ __forceinline__ T limited_slope(T qm1, T q0, T qp1) {
  if (SLOPE == 0) return T(0);
  if (SLOPE == 1) {  // minmod
    T dlft = q0 - qm1, drgt = qp1 - q0;
    T r;
    if ((dlft * drgt) <= T(0)) r = T(0);
    else if (dlft > T(0)) r = tmin(dlft, drgt);
    else r = tmax(dlft, drgt);
    return r;
  }
  // moncen (slope_type = 2): dlft = 2(q0-qm1), drgt = 2(qp1-q0),
  // dcen = (dlft+drgt)/4, dq = sign(dcen)*min(dlim, |dcen|)
  T dlft = T(2) * (q0 - qm1), drgt = T(2) * (qp1 - q0);
  T dcen = T(0.25) * (dlft + drgt);
  T slop = tmin(fabs(dlft), fabs(drgt));
  T dlim = ((dlft * drgt) <= T(0)) ? T(0) : slop;
  return copysign(tmin(dlim, fabs(dcen)), dcen);
}

// Normal-velocity slope bound, umuscl.f90:2361-2385
template <typename T> __device__ __forceinline__ T momentum_bound(T dq, T rm1, T vm1, T v0, T rp1, T vp1,
                                                                  T inv_r0) {
  T dlft = rm1 * fabs(v0 - vm1);
  T drgt = rp1 * fabs(vp1 - v0);
  T dlim = T(2) * tmin(dlft, drgt) * inv_r0;
  return copysign(tmin(fabs(dq), dlim), dq);
}

// ---------------------------------------------------------------------------
// Riemann solvers, godunov_utils.f90:338-852.  Input states rotated to
// (rho, un, ut1, ut2, p); output flux (mass, normal mom, t1 mom, t2 mom, E).
// ---------------------------------------------------------------------------
template <typename T> __device__ __forceinline__ void riemann_hllc(const T* ql, const T* qr, T* f,
                                                                   const HydroConst<T>& H) {
  T rl = tmax(ql[0], H.smallr), ul = ql[1], vl = ql[2], wl = ql[3];
  T Pl = tmax(ql[4], rl * H.smallp_riem);
  T el = Pl * H.entho;
  T etotl = el + T(0.5) * rl * (ul * ul + vl * vl + wl * wl);
  T rr = tmax(qr[0], H.smallr), ur = qr[1], vr = qr[2], wr = qr[3];
  T Pr = tmax(qr[4], rr * H.smallp_riem);
  T er = Pr * H.entho;
  T etotr = er + T(0.5) * rr * (ur * ur + vr * vr + wr * wr);
  T cfl = Num<T>::sqrt_(tmax(H.gamma * Pl * Num<T>::rcp(rl), H.smallc2));
  T cfr = Num<T>::sqrt_(tmax(H.gamma * Pr * Num<T>::rcp(rr), H.smallc2));
  T cmx = tmax(cfl, cfr);
  T SL = tmin(ul, ur) - cmx;
  T SR = tmax(ul, ur) + cmx;
  T rcl = rl * (ul - SL);
  T rcr = rr * (SR - ur);
  T inv = Num<T>::rcp(rcr + rcl);
  T ustar = (rcr * ur + rcl * ul + (Pl - Pr)) * inv;
  T Pstar = (rcr * Pl + rcl * Pr + rcl * rcr * (ul - ur)) * inv;
  // Sample at x/t=0 (godunov_utils.f90:771-823): pick the side, then the
  // star state of that side unless the side's outer wave is supersonic.
  bool left = (SL > T(0)) || (ustar > T(0));
  bool star = left ? !(SL > T(0)) : (SR > T(0));
  T rs = left ? rl : rr, us = left ? ul : ur, vs = left ? vl : vr, ws = left ? wl : wr;
  T Ps = left ? Pl : Pr, es = left ? el : er, Es = left ? etotl : etotr, Ss = left ? SL : SR;
  T ro = rs, uo = us, Po = Ps, Eo = Es;
  if (star) {
    T id = Num<T>::rcp(Ss - ustar);
    T fac = (Ss - us) * id;
    ro = rs * fac;
    Eo = ((Ss - us) * Es - Ps * us + Pstar * ustar) * id;
    uo = ustar;
    Po = Pstar;
  }
  (void)es;
  T mu = ro * uo;
  f[0] = mu;
  f[1] = mu * uo + Po;
  f[2] = mu * vs;
  f[3] = mu * ws;
  f[4] = (Eo + Po) * uo;
}

template <typename T> __device__ __forceinline__ void cons_and_flux(const T* q, T entho, T* u, T* fl, bool hll) {
  u[0] = q[0];
  u[1] = q[0] * q[1];
  u[2] = q[0] * q[2];
  u[3] = q[0] * q[3];
  u[4] = q[4] * entho + T(0.5) * q[0] * (q[1] * q[1]) + T(0.5) * q[0] * (q[2] * q[2]) +
         T(0.5) * q[0] * (q[3] * q[3]);
  fl[0] = hll ? u[1] : q[1] * u[0];
  fl[1] = q[1] * u[1] + q[4];
  fl[2] = q[1] * u[2];
  fl[3] = q[1] * u[3];
  fl[4] = q[1] * (u[4] + q[4]);
}

template <typename T> __device__ __forceinline__ void riemann_llf(const T* ql, const T* qr, T* f,
                                                                  const HydroConst<T>& H) {
  T rl = tmax(ql[0], H.smallr);
  T pl = tmax(ql[4], rl * H.smallp_riem);
  T cl = Num<T>::sqrt_(H.gamma * pl * Num<T>::rcp(rl));
  T rr = tmax(qr[0], H.smallr);
  T pr = tmax(qr[4], rr * H.smallp_riem);
  T cr = Num<T>::sqrt_(H.gamma * pr * Num<T>::rcp(rr));
  T cmax = tmin(tmax(fabs(ql[1]) + cl, fabs(qr[1]) + cr), H.smax_cap);
  T ul[5], ur[5], fl[5], fr[5];
  cons_and_flux(ql, H.entho, ul, fl, false);
  cons_and_flux(qr, H.entho, ur, fr, false);
#pragma unroll
  for (int n = 0; n < 5; ++n) f[n] = T(0.5) * (fl[n] + fr[n] - cmax * (ur[n] - ul[n]));
}

template <typename T> __device__ __forceinline__ void riemann_hll(const T* ql, const T* qr, T* f,
                                                                  const HydroConst<T>& H) {
  T rl = tmax(ql[0], H.smallr);
  T pl = tmax(ql[4], rl * H.smallp_riem);
  T cl = Num<T>::sqrt_(H.gamma * pl * Num<T>::rcp(rl));
  T rr = tmax(qr[0], H.smallr);
  T pr = tmax(qr[4], rr * H.smallp_riem);
  T cr = Num<T>::sqrt_(H.gamma * pr * Num<T>::rcp(rr));
  T cm = tmax(cl, cr);
  T SL = tmax(tmin(tmin(ql[1], qr[1]) - cm, T(0)), -H.smax_cap);
  T SR = tmin(tmax(tmax(ql[1], qr[1]) + cm, T(0)), H.smax_cap);
  T ul[5], ur[5], fl[5], fr[5];
  cons_and_flux(ql, H.entho, ul, fl, true);
  cons_and_flux(qr, H.entho, ur, fr, true);
  T inv = Num<T>::rcp(SR - SL);
  T sls = SR * SL;
#pragma unroll
  for (int n = 0; n < 5; ++n) f[n] = (SR * fl[n] - SL * fr[n] + sls * (ur[n] - ul[n])) * inv;
}

template <typename T, int RIEMANN> __device__ __forceinline__ void riemann(const T* ql, const T* qr, T* f,
                                                                           const HydroConst<T>& H) {
  if (RIEMANN == 1) riemann_llf(ql, qr, f, H);
  else if (RIEMANN == 2) riemann_hll(ql, qr, f, H);
  else riemann_hllc(ql, qr, f, H);
}

// ---------------------------------------------------------------------------
// CFL time step of one cell from conserved FP64 values, cmpdt
// (godunov_utils.f90:228-333) with bb=0, induction=.false.  With zero
// magnetic field the reference's fast speed sqrt(c2+sqrt(c2**2)) equals
// sqrt(a2) exactly in IEEE arithmetic (sqrt(fl(x*x)) == x).
// ---------------------------------------------------------------------------
struct CflConst {
  double gamma, gm1, smallr, smallp;  // smallp = smallc**2/gamma
  double cdx_smallc;                  // courant*dx/smallc
  double two_cdx;                     // 2*courant*dx
  double two_c;                       // 2*courant
  double gsum_dx;                     // (|gx|+|gy|+|gz|)*dx
  double k0;                          // 2*courant*dx/(1+sqrt(1+2*courant*1e-4)): dt*ctot without gravity
  int ndim;
};

__device__ __forceinline__ double cmpdt_cell(double r, double mx, double my, double mz, double E,
                                             const CflConst& C) {
  r = r > C.smallr ? r : C.smallr;
  double ir = 1.0 / r;
  double u = mx * ir, v = my * ir, w = mz * ir;
  double e = E - 0.5 * r * (u * u);
  e = e - 0.5 * r * (v * v);
  e = e - 0.5 * r * (w * w);
  double p = C.gm1 * e;
  double pf = r * C.smallp;
  p = p > pf ? p : pf;
  double c = sqrt(C.gamma * p * ir);
  double ctot = fabs(u) + c;
  if (C.ndim > 1) ctot += fabs(v) + c;
  if (C.ndim > 2) ctot += fabs(w) + c;
  double dtcell;
  if (C.gsum_dx == 0.0) {
    // grav = max(0, 1e-4): the square root is a constant of the launch
    dtcell = C.k0 / ctot;
  } else {
    double grav = C.gsum_dx / (ctot * ctot);
    grav = grav > 0.0001 ? grav : 0.0001;
    dtcell = C.two_cdx / (ctot * (1.0 + sqrt(1.0 + C.two_c * grav)));
  }
  return dtcell < C.cdx_smallc ? dtcell : C.cdx_smallc;
}

// ---------------------------------------------------------------------------
// PTX helpers: mbarrier + bulk async copy (global -> shared, no multicast)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// Returns true once the phase with the given parity has completed.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

}  // namespace rh
