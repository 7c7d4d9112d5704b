// rh_physics.cuh — cell and interface physics of the Godunov step, generic in
// the lane type V (double: one cell; float2: two cells with packed FP32x2).
//
// Restates RAMSES II's CPU routines with the same branch structure and floors:
//   limiters            hydro/umuscl.f90:2132-2206
//   normal-velocity bound hydro/umuscl.f90:2361-2385
//   riemann_llf/hll/hllc  hydro/godunov_utils.f90:338-852
// Branches become per-lane selects; reciprocals and square roots use the
// lane's fast Newton-refined (FP64) or hardware-approximate (FP32) forms.
#pragma once
#include "rh_vec.cuh"

namespace rh {

template <class V> struct HydroK {
  V gamma, entho;
  V smallr, smallc2;
  V smallp_trace;  // smallr*smallc**2            (umuscl.f90:931)
  V smallp_riem;   // smallc**2/gamma             (godunov_utils.f90:363,511,676)
  V smax_cap;      // courant*dx/dt               (umuscl.f90:99)
  V dtdx;
  V zero, half, two;
  V gm1, smalle;   // gamma-1, smallc**2/gamma/(gamma-1) (umuscl.f90:1778)
  V grav[3];       // constant_gravity*dt/2 (ctoprim predictor)
};

// TVD slope of one variable along one direction.
template <class V, int SLOPE> __device__ __forceinline__ V limited_slope(V qm1, V q0, V qp1, const HydroK<V>& H) {
  if (SLOPE == 0) return H.zero;
  const V a = q0 - qm1, b = qp1 - q0;
  if (SLOPE == 1) {  // minmod: 0 if a*b<=0, else the smaller-magnitude one
    const V r = vsel(vgt(a, H.zero), vmin(a, b), vmax(a, b));
    return vsel(vgt(a * b, H.zero), r, H.zero);
  }
  // moncen: dlft=2a, drgt=2b, dcen=(a+b)/2, dq=sign(dcen)*min(dlim,|dcen|),
  // dlim = min(|dlft|,|drgt|) when dlft*drgt>0 else 0
  const V dcen = H.half * (a + b);
  const V slop = H.two * vmin(vabs(a), vabs(b));
  const V dlim = vsel(vgt(a * b, H.zero), slop, H.zero);
  return vcopysign(vmin(dlim, vabs(dcen)), dcen);
}

// slope_type 3, the positivity-preserving 3D unsplit slope (umuscl.f90:
// 2207-2269): the central differences of a variable, scaled by
// min(1, min(|vmin - c|, |vmax - c|) / (|dfx| + |dfy| + |dfz|)/2) with vmin,
// vmax the extremes of the 27-point neighbourhood (cell included; rounding is
// monotone, so min(v - c) = min(v) - c exactly), so that the reconstruction
// stays within the neighbourhood's range.
template <class V> __device__ __forceinline__ void slope_posdef(V c, V vmn, V vmx, V dfx, V dfy, V dfz,
                                                               const HydroK<V>& H, V& dx, V& dy, V& dz) {
  const V one = H.two * H.half;
  const V dff = H.half * (vabs(dfx) + vabs(dfy) + vabs(dfz));
  const V lim = vmin(vabs(vmn - c), vabs(vmx - c));
  const V slop = vsel(vgt(dff, H.zero), vmin(one, lim * vrcp(dff)), one);
  dx = slop * dfx;
  dy = slop * dfy;
  dz = slop * dfz;
}

// Bound on the normal-velocity slope: rho*|dq|/2 <= rho_nbor*|u_nbor-u|.
template <class V> __device__ __forceinline__ V momentum_bound(V dq, V rm1, V vm1, V v0, V rp1, V vp1, V ir0,
                                                               const HydroK<V>& H) {
  const V dlft = rm1 * vabs(v0 - vm1);
  const V drgt = rp1 * vabs(vp1 - v0);
  const V dlim = H.two * vmin(dlft, drgt) * ir0;
  return vcopysign(vmin(vabs(dq), dlim), dq);
}


// Half of limited_slope and of the momentum bound (FP64 lanes), for slope
// types 1 and 2: bitwise 0.5 * the full values (scaling by two commutes with
// rounding, so 0.5 * (2 min) = min and 0.5 * (0.5 (a + b)) = 0.25 (a + b)
// exactly).  The FP64 body takes these: two multiplications fewer per slope,
// and its registers fit without spilling (the FP32-bulk body ran 2 % slower
// with them and keeps the full slopes times one half).
template <int SLOPE> __device__ __forceinline__ double half_slope(double qm1, double q0, double qp1) {
  if (SLOPE == 0) return 0.0;
  const double a = q0 - qm1, b = qp1 - q0;
  if (SLOPE == 1) {
    const double r = vsel(vgt(a, 0.0), vmin(a, b), vmax(a, b));
    return 0.5 * vsel(vgt(a * b, 0.0), r, 0.0);
  }
  const double dcen = 0.25 * (a + b);
  const double dlim = vsel(vgt(a * b, 0.0), vmin(vabs(a), vabs(b)), 0.0);
  return vcopysign(vmin(dlim, vabs(dcen)), dcen);
}
__device__ __forceinline__ double half_momentum_bound(double dq, double rm1, double vm1, double v0, double rp1,
                                                      double vp1, double ir0) {
  const double dlft = rm1 * vabs(v0 - vm1);
  const double drgt = rp1 * vabs(vp1 - v0);
  const double dlim = vmin(dlft, drgt) * ir0;
  return vcopysign(vmin(vabs(dq), dlim), dq);
}

// HLLC (Toro), godunov_utils.f90:638-852.  q = (rho, un, ut1, ut2, p);
// f = (mass, normal momentum, t1 momentum, t2 momentum, total energy).
template <class V> __device__ __forceinline__ void riemann_hllc(const V* ql, const V* qr, V* f, const HydroK<V>& H) {
  const V rl = vmax(ql[0], H.smallr), ul = ql[1], vl = ql[2], wl = ql[3];
  const V Pl = vmax(ql[4], rl * H.smallp_riem);
  const V rr = vmax(qr[0], H.smallr), ur = qr[1], vr = qr[2], wr = qr[3];
  const V Pr = vmax(qr[4], rr * H.smallp_riem);
  const V etotl = vfma(Pl, H.entho, H.half * rl * vfma(ul, ul, vfma(vl, vl, wl * wl)));
  const V etotr = vfma(Pr, H.entho, H.half * rr * vfma(ur, ur, vfma(vr, vr, wr * wr)));
  const V cfl = vsqrt(vmax(H.gamma * Pl * vrcp(rl), H.smallc2));
  const V cfr = vsqrt(vmax(H.gamma * Pr * vrcp(rr), H.smallc2));
  const V cmx = vmax(cfl, cfr);
  const V SL = vmin(ul, ur) - cmx;
  const V SR = vmax(ul, ur) + cmx;
  const V rcl = rl * (ul - SL);
  const V rcr = rr * (SR - ur);
  const V inv = vrcp(rcr + rcl);
  const V ustar = vfma(rcr, ur, vfma(rcl, ul, Pl - Pr)) * inv;
  const V Pstar = vfma(rcr, Pl, vfma(rcl, Pr, rcl * rcr * (ul - ur))) * inv;
  // sample at x/t = 0 (godunov_utils.f90:771-823)
  const auto slpos = vgt(SL, H.zero);
  const auto left = mor(slpos, vgt(ustar, H.zero));
  const auto star = mor(mand(left, mnot(slpos)), mand(mnot(left), vgt(SR, H.zero)));
  const V rs = vsel(left, rl, rr), us = vsel(left, ul, ur), vs = vsel(left, vl, vr), ws = vsel(left, wl, wr);
  const V Ps = vsel(left, Pl, Pr), Es = vsel(left, etotl, etotr), Ss = vsel(left, SL, SR);
  const V sdu = Ss - us;
  const V id = vrcp(Ss - ustar);
  const V ro = vsel(star, rs * sdu * id, rs);
  const V uo = vsel(star, ustar, us);
  const V Po = vsel(star, Pstar, Ps);
  const V Eo = vsel(star, vfma(sdu, Es, vfma(Pstar, ustar, -(Ps * us))) * id, Es);
  const V mu = ro * uo;
  f[0] = mu;
  f[1] = vfma(mu, uo, Po);
  f[2] = mu * vs;
  f[3] = mu * ws;
  f[4] = (Eo + Po) * uo;
}

// Conservative state and physical flux of a rotated primitive state.
template <class V> __device__ __forceinline__ void cons_flux(const V* q, const HydroK<V>& H, V* u, V* fl) {
  u[0] = q[0];
  u[1] = q[0] * q[1];
  u[2] = q[0] * q[2];
  u[3] = q[0] * q[3];
  u[4] = vfma(q[4], H.entho, H.half * q[0] * vfma(q[1], q[1], vfma(q[2], q[2], q[3] * q[3])));
  fl[0] = u[1];
  fl[1] = vfma(q[1], u[1], q[4]);
  fl[2] = q[1] * u[2];
  fl[3] = q[1] * u[3];
  fl[4] = q[1] * (u[4] + q[4]);
}

// Local Lax-Friedrichs, godunov_utils.f90:338-481
template <class V> __device__ __forceinline__ void riemann_llf(const V* ql, const V* qr, V* f, const HydroK<V>& H) {
  const V rl = vmax(ql[0], H.smallr);
  const V pl = vmax(ql[4], rl * H.smallp_riem);
  const V cl = vsqrt(H.gamma * pl * vrcp(rl));
  const V rr = vmax(qr[0], H.smallr);
  const V pr = vmax(qr[4], rr * H.smallp_riem);
  const V cr = vsqrt(H.gamma * pr * vrcp(rr));
  const V cmax = vmin(vmax(vabs(ql[1]) + cl, vabs(qr[1]) + cr), H.smax_cap);
  V ul[5], ur[5], fl[5], fr[5];
  cons_flux(ql, H, ul, fl);
  cons_flux(qr, H, ur, fr);
#pragma unroll
  for (int n = 0; n < 5; ++n) f[n] = H.half * (fl[n] + fr[n] - cmax * (ur[n] - ul[n]));
}

// HLL, godunov_utils.f90:486-633
template <class V> __device__ __forceinline__ void riemann_hll(const V* ql, const V* qr, V* f, const HydroK<V>& H) {
  const V rl = vmax(ql[0], H.smallr);
  const V pl = vmax(ql[4], rl * H.smallp_riem);
  const V cl = vsqrt(H.gamma * pl * vrcp(rl));
  const V rr = vmax(qr[0], H.smallr);
  const V pr = vmax(qr[4], rr * H.smallp_riem);
  const V cr = vsqrt(H.gamma * pr * vrcp(rr));
  const V cm = vmax(cl, cr);
  const V SL = vmax(vmin(vmin(ql[1], qr[1]) - cm, H.zero), -H.smax_cap);
  const V SR = vmin(vmax(vmax(ql[1], qr[1]) + cm, H.zero), H.smax_cap);
  V ul[5], ur[5], fl[5], fr[5];
  cons_flux(ql, H, ul, fl);
  cons_flux(qr, H, ur, fr);
  const V inv = vrcp(SR - SL);
  const V sls = SR * SL;
#pragma unroll
  for (int n = 0; n < 5; ++n) f[n] = vfma(sls, ur[n] - ul[n], SR * fl[n] - SL * fr[n]) * inv;
}

template <class V, int RIEMANN> __device__ __forceinline__ void riemann_dtdx(const V* ql, const V* qr, V* f,
                                                                            const HydroK<V>& H) {
  if (RIEMANN == 1) riemann_llf(ql, qr, f, H);
  else if (RIEMANN == 2) riemann_hll(ql, qr, f, H);
  else riemann_hllc(ql, qr, f, H);
#pragma unroll
  for (int n = 0; n < 5; ++n) f[n] = f[n] * H.dtdx;
}

// Hancock predictor (trace3d, umuscl.f90:966-1234) of one cell from its
// primitive state q (with 1/rho) and half-slopes d[dir][var]; writes the six
// interface states qm[dir] (upper face of the cell) and qp[dir] (lower face),
// floored as the reference does.
template <class V> __device__ __forceinline__ void trace_cell(const V* q, V ir, V (*d)[5], V (*qm)[5], V (*qp)[5],
                                                             const HydroK<V>& H) {
  const V r = q[0], u = q[1], v = q[2], w = q[3], p = q[4];
  const V divv = d[0][1] + d[1][2] + d[2][3];
  const V sr0 = -vfma(divv, r, vfma(w, d[2][0], vfma(v, d[1][0], u * d[0][0])));
  const V su0 = -vfma(d[0][4], ir, vfma(w, d[2][1], vfma(v, d[1][1], u * d[0][1])));
  const V sv0 = -vfma(d[1][4], ir, vfma(w, d[2][2], vfma(v, d[1][2], u * d[0][2])));
  const V sw0 = -vfma(d[2][4], ir, vfma(w, d[2][3], vfma(v, d[1][3], u * d[0][3])));
  const V sp0 = -vfma(divv * H.gamma, p, vfma(w, d[2][4], vfma(v, d[1][4], u * d[0][4])));
  const V pr[5] = {vfma(sr0, H.dtdx, r), vfma(su0, H.dtdx, u), vfma(sv0, H.dtdx, v), vfma(sw0, H.dtdx, w),
                   vfma(sp0, H.dtdx, p)};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      qp[a][n] = pr[n] - d[a][n];
      qm[a][n] = pr[n] + d[a][n];
    }
    qp[a][0] = vsel(vlt(qp[a][0], H.smallr), r, qp[a][0]);
    qp[a][4] = vsel(vlt(qp[a][4], H.smallp_trace), p, qp[a][4]);
    qm[a][0] = vsel(vlt(qm[a][0], H.smallr), r, qm[a][0]);
    qm[a][4] = vsel(vlt(qm[a][4], H.smallp_trace), p, qm[a][4]);
  }
}

}  // namespace rh
