// rh_plane2d.cuh — one XY tile of a plane (2D) batch problem.
//
// A 2D problem of the batch is stored as one z oct layer with periodic z, so
// both cell planes of every oct hold the same values.  On such a problem the
// pencil body's z work is exact zeros: every z slope is +0 (the z neighbours
// equal the cell), the normal-velocity bound of a zero slope is +0, and the two
// z faces of a plane see the same Riemann problem, so their flux difference is
// +0.  This tile body does the x/y work only, with the same operations in the
// same order as the pencil body (trace_cell with zero z slopes; the update adds
// the +0 z difference as the pencil body does), and writes the result to both
// planes: it matches the pencil body on such problems bit for bit, the
// reference's 2D predictor (hydro/umuscl.f90:487-853 trace2d) being trace3d
// without its z terms.  The CFL accumulators take each cell twice (both
// planes), as the pencil body does.
//
// FP64 lanes are one cell.  FP32-bulk lanes (float2) hold two tiles of the
// problem, TYO octs apart in y: the pencil body's two lanes are the two equal
// planes, so pairing tiles instead halves the work per cell; each lane's
// arithmetic is the one its cell gets in the pencil body.
//
// No staging: the tile's (2 TXO + 4) x (2 TYO + 4) cells are read straight from
// the pool (a 2D tile is one layer, nothing to pipeline), converted to
// primitives into the plane buffer, then traced, solved and updated by the
// ring-column threads of the pencil geometry.
#pragma once
#include "rh_godunov.cuh"
#include "rh_godunov2.cuh"

namespace rh {

__device__ __forceinline__ int plane_oct(int v, int n, int periodic) {
  if (periodic) return ((v % n) + n) % n;
  return v < 0 ? 0 : (v >= n ? n - 1 : v);
}

// ctoprim_f32x2's arithmetic with each lane read from its own oct record and
// its own y flip (FP32-bulk pairs two tiles of a 2D problem in the two lanes).
__device__ __forceinline__ void ctoprim_f32_lanes(const float* sfa, const double* sda, int ca, bool fya,
                                                  const float* sfb, const double* sdb, int cb, bool fyb, bool fx,
                                                  const HydroK<float2>& H, double gm1, double smalle, float2* q,
                                                  float2& ir) {
  const float2 d = make_float2(sfa[ca], sfb[cb]);
  float2 mx = make_float2(sfa[8 + ca], sfb[8 + cb]);
  float2 my = make_float2(sfa[16 + ca], sfb[16 + cb]);
  const float2 mz = make_float2(sfa[24 + ca], sfb[24 + cb]);
  const double E0 = sda[ca], E1 = sdb[cb];
  if (fx) mx = -mx;
  if (fya) my.x = -my.x;
  if (fyb) my.y = -my.y;
  const float2 r = vmax(d, H.smallr);
  ir = vrcp(r);
  const float2 u = mx * ir, v = my * ir, w = mz * ir;
  const float2 k2 = vfma(u, u, vfma(v, v, w * w));
  double e0 = E0 - 0.5 * (double)r.x * (double)k2.x;
  double e1 = E1 - 0.5 * (double)r.y * (double)k2.y;
  const double m0 = smalle * (double)r.x, m1 = smalle * (double)r.y;
  e0 = e0 > m0 ? e0 : m0;
  e1 = e1 > m1 ? e1 : m1;
  q[0] = r;
  q[1] = u + H.grav[0];
  q[2] = v + H.grav[1];
  q[3] = w + H.grav[2];
  q[4] = make_float2((float)(gm1 * e0), (float)(gm1 * e1));
}

template <typename T, typename V, int TXO, int TYO, int SLOPE, int RIEMANN>
__device__ __forceinline__ void plane2d_body(const LevelArgs& A, const StateArgs<T>& S, const HydroK<V>& H,
                                             const int4 hdr, CflAcc& acc) {
  constexpr bool F64 = sizeof(T) == 8;
  using G = Geo<T, V, TXO, TYO>;
  V* Q = reinterpret_cast<V*>(rh_smem + G::oQ);  // [5][NLC] primitives, then [NLC] 1/rho
  V* IR = Q + 5 * G::NLC;
  V* FS = reinterpret_cast<V*>(rh_smem + G::oFS);   // [10][NRC]: qp_x(5), qp_y(5)
  V* FXY = reinterpret_cast<V*>(rh_smem + G::oFX);  // [2][5][NRC]: x then y fluxes
  const int t = threadIdx.x;
  const int ox0 = hdr.x, oy0 = hdr.y;
  const int nxo = A.ncx >> 1, nyo = A.ncy >> 1;

  // (A) primitives of every cell of the tile and its two-cell halo (plane a)
  for (int i = t; i < G::NLC; i += G::NT) {
    const int gx = 2 * ox0 - 2 + i % G::LW, gy = 2 * oy0 - 2 + i / G::LW;
    const CellMap mx = map_coord(gx, A.ncx, A.periodic[0], A.btype[0], A.btype[1]);
    const CellMap my = map_coord(gy, A.ncy, A.periodic[1], A.btype[2], A.btype[3]);
    const int oct = plane_oct(gx >> 1, nxo, A.periodic[0]) + nxo * plane_oct(gy >> 1, nyo, A.periodic[1]);
    const int c = mx.parity + 2 * my.parity;
    V q[5], ir;
    if constexpr (F64) {
      double U[5];
      ctoprim_f64(S.uold_d + (size_t)oct * 40, c, mx.flip, my.flip, false, H, q, ir, U);
    } else {
      // lane .y: the same cell of the tile TYO octs further in y
      const int gyb = gy + G::CY;
      const CellMap myb = map_coord(gyb, A.ncy, A.periodic[1], A.btype[2], A.btype[3]);
      const int octb = plane_oct(gx >> 1, nxo, A.periodic[0]) + nxo * plane_oct(gyb >> 1, nyo, A.periodic[1]);
      ctoprim_f32_lanes(S.uold_f + (size_t)oct * kBulkF, S.uold_d + (size_t)oct * kBulkD, c, my.flip,
                        S.uold_f + (size_t)octb * kBulkF, S.uold_d + (size_t)octb * kBulkD, mx.parity + 2 * myb.parity,
                        myb.flip, mx.flip, H, A.gm1_d, A.smalle_d, q, ir);
    }
#pragma unroll
    for (int n = 0; n < 5; ++n) Q[n * G::NLC + i] = q[n];
    IR[i] = ir;
  }
  __syncthreads();

  Columns<G> col;
  col.init(t, ox0, oy0, A);
  const bool active = t < G::NRC;
  // FP32-bulk 7x7 tiles (16-wide ring rows, each inside a warp): x faces by
  // warp shuffle and both y faces solved by each cell, so the flux exchange
  // needs no barrier of its own (as the pencil body); FS then holds the
  // lower and upper y states
  constexpr bool kOneBar = !F64 && G::RW == 16;
  V qmx[5], qmy[5], qpx[5], dfx[5];
#pragma unroll
  for (int n = 0; n < 5; ++n) qpx[n] = V{};
  // (C) slopes, predictor and x/y interface states of the ring cells
  if (active) {
    V cur[5], xm[5], xp[5], ym[5], yp[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      cur[n] = Q[n * G::NLC + col.lc];
      xm[n] = Q[n * G::NLC + col.lc - 1];
      xp[n] = Q[n * G::NLC + col.lc + 1];
      ym[n] = Q[n * G::NLC + col.lc - G::LW];
      yp[n] = Q[n * G::NLC + col.lc + G::LW];
    }
    const V irc = IR[col.lc];
    V d[3][5];
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      d[0][n] = limited_slope<V, SLOPE>(xm[n], cur[n], xp[n], H);
      d[1][n] = limited_slope<V, SLOPE>(ym[n], cur[n], yp[n], H);
      d[2][n] = H.zero;
    }
    if (SLOPE > 0) {
      d[0][1] = momentum_bound(d[0][1], xm[0], xm[1], cur[1], xp[0], xp[1], irc, H);
      d[1][2] = momentum_bound(d[1][2], ym[0], ym[2], cur[2], yp[0], yp[2], irc, H);
    }
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int n = 0; n < 5; ++n) d[a][n] = H.half * d[a][n];
    V qm[3][5], qp[3][5];
    trace_cell(cur, irc, d, qm, qp, H);
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      if (kOneBar) {
        FS[n * G::NRC + t] = qp[1][n];
        FS[(5 + n) * G::NRC + t] = qm[1][n];
        qpx[n] = qp[0][n];
      } else {
        FS[n * G::NRC + t] = qp[0][n];
        FS[(5 + n) * G::NRC + t] = qp[1][n];
      }
      qmx[n] = qm[0][n];
      qmy[n] = qm[1][n];
    }
  }
  if constexpr (kOneBar) {
    V qr[5], fxr[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      qr[n].x = __shfl_down_sync(0xffffffffu, qpx[n].x, 1);
      qr[n].y = __shfl_down_sync(0xffffffffu, qpx[n].y, 1);
      fxr[n] = V{};
    }
    if (active && col.rx >= -1 && col.rx < G::CX && col.ry >= 0 && col.ry < G::CY)
      riemann_dtdx<V, RIEMANN>(qmx, qr, fxr, H);
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      V fl;
      fl.x = __shfl_up_sync(0xffffffffu, fxr[n].x, 1);
      fl.y = __shfl_up_sync(0xffffffffu, fxr[n].y, 1);
      dfx[n] = vsub_nc(fl, fxr[n]);
    }
  }
  __syncthreads();
  // (D) x flux at the right face and y flux at the top face
  if (!kOneBar && active) {
    if (col.rx >= -1 && col.rx < G::CX && col.ry >= 0 && col.ry < G::CY) {
      V qr[5], f[5];
#pragma unroll
      for (int n = 0; n < 5; ++n) qr[n] = FS[n * G::NRC + t + 1];
      riemann_dtdx<V, RIEMANN>(qmx, qr, f, H);
#pragma unroll
      for (int n = 0; n < 5; ++n) FXY[n * G::NRC + t] = f[n];
    }
    if (col.ry >= -1 && col.ry < G::CY && col.rx >= 0 && col.rx < G::CX) {
      const int tn = t + G::RW;
      const V ql[5] = {qmy[0], qmy[2], qmy[1], qmy[3], qmy[4]};
      const V qr[5] = {FS[5 * G::NRC + tn], FS[7 * G::NRC + tn], FS[6 * G::NRC + tn], FS[8 * G::NRC + tn],
                       FS[9 * G::NRC + tn]};
      V f[5];
      riemann_dtdx<V, RIEMANN>(ql, qr, f, H);
      const V fy[5] = {f[0], f[2], f[1], f[3], f[4]};
      V* FY = FXY + 5 * G::NRC;
#pragma unroll
      for (int n = 0; n < 5; ++n) FY[n * G::NRC + t] = fy[n];
    }
  }
  if (!kOneBar) __syncthreads();
  // (E) conservative update of the tile's cells, written to both planes
  if constexpr (F64) {
    if (active && col.interior && col.in_domain_xy) {
      const int oct = (ox0 + (col.rx >> 1)) + nxo * (oy0 + (col.ry >> 1));
      const int c = (col.rx & 1) + 2 * (col.ry & 1);
      const double* FX = FXY;
      const double* FY = FXY + 5 * G::NRC;
      const double* o = S.uold_d + (size_t)oct * 40 + c;
      double un[5];
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        const double u0 = o[8 * n] + (FX[n * G::NRC + t - 1] - FX[n * G::NRC + t]);
        const double up = u0 + (FY[n * G::NRC + t - G::RW] - FY[n * G::NRC + t]);
        un[n] = up + 0.0;  // the z flux difference, an exact +0
      }
      double* w = S.unew_d + (size_t)oct * 40 + c;
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        w[8 * n] = un[n];
        w[8 * n + 4] = un[n];
      }
      acc.add(un[0], un[1], un[2], un[3], un[4], A);
      acc.add(un[0], un[1], un[2], un[3], un[4], A);
    }
  } else {
    const int gx = 2 * ox0 + col.rx, gya = 2 * oy0 + col.ry, gyb = gya + G::CY;
    const bool oka = active && col.interior && gx < A.ncx && gya < A.ncy;
    const bool okb = active && col.interior && gx < A.ncx && gyb < A.ncy;
    if (oka) {
      const int c = (col.rx & 1) + 2 * (col.ry & 1);
      const int octa = (gx >> 1) + nxo * (gya >> 1);
      const int octb = okb ? (gx >> 1) + nxo * (gyb >> 1) : octa;
      const float2* FX = FXY;
      const float2* FY = FXY + 5 * G::NRC;
      const float* oa = S.uold_f + (size_t)octa * kBulkF + c;
      const float* ob = S.uold_f + (size_t)octb * kBulkF + c;
      float2 dx_[5], dy_[5];
      if constexpr (kOneBar) {
        const int tn = t + G::RW, ts = t - G::RW;
        const float2 qlt[5] = {qmy[0], qmy[2], qmy[1], qmy[3], qmy[4]};
        const float2 qrt[5] = {FS[0 * G::NRC + tn], FS[2 * G::NRC + tn], FS[1 * G::NRC + tn], FS[3 * G::NRC + tn],
                               FS[4 * G::NRC + tn]};
        const float2 qlb[5] = {FS[5 * G::NRC + ts], FS[7 * G::NRC + ts], FS[6 * G::NRC + ts], FS[8 * G::NRC + ts],
                               FS[9 * G::NRC + ts]};
        const float2 qrb[5] = {FS[0 * G::NRC + t], FS[2 * G::NRC + t], FS[1 * G::NRC + t], FS[3 * G::NRC + t],
                               FS[4 * G::NRC + t]};
        float2 ft[5], fb[5];
        riemann_dtdx<float2, RIEMANN>(qlt, qrt, ft, H);
        riemann_dtdx<float2, RIEMANN>(qlb, qrb, fb, H);
        const int un[5] = {0, 2, 1, 3, 4};
#pragma unroll
        for (int n = 0; n < 5; ++n) {
          dx_[n] = dfx[n];
          dy_[n] = vsub_nc(fb[un[n]], ft[un[n]]);
        }
      } else {
#pragma unroll
        for (int n = 0; n < 5; ++n) {
          dx_[n] = FX[n * G::NRC + t - 1] - FX[n * G::NRC + t];
          dy_[n] = FY[n * G::NRC + t - G::RW] - FY[n * G::NRC + t];
        }
      }
      float2 u2[4];
#pragma unroll
      for (int n = 0; n < 4; ++n) {
        const float2 base = make_float2(oa[8 * n], ob[8 * n]);
        u2[n] = (base + dx_[n]) + dy_[n];
      }
      const double ea = (S.uold_d[(size_t)octa * kBulkD + c] + (double)dx_[4].x) + (double)dy_[4].x;
      const double eb = (S.uold_d[(size_t)octb * kBulkD + c] + (double)dx_[4].y) + (double)dy_[4].y;
      // the z flux differences, exact +0
      float ua[4], ub[4];
#pragma unroll
      for (int n = 0; n < 4; ++n) {
        ua[n] = u2[n].x + 0.f;
        ub[n] = u2[n].y + 0.f;
      }
      const double Ea = ea + (double)0.f, Eb = eb + (double)0.f;
      float* wa = S.unew_f + (size_t)octa * kBulkF + c;
#pragma unroll
      for (int n = 0; n < 4; ++n) {
        wa[8 * n] = ua[n];
        wa[8 * n + 4] = ua[n];
      }
      S.unew_d[(size_t)octa * kBulkD + c] = Ea;
      S.unew_d[(size_t)octa * kBulkD + c + 4] = Ea;
      acc.add_bulk(ua[0], ua[1], ua[2], ua[3], Ea, A);
      acc.add_bulk(ua[0], ua[1], ua[2], ua[3], Ea, A);
      if (okb) {
        float* wb = S.unew_f + (size_t)octb * kBulkF + c;
#pragma unroll
        for (int n = 0; n < 4; ++n) {
          wb[8 * n] = ub[n];
          wb[8 * n + 4] = ub[n];
        }
        S.unew_d[(size_t)octb * kBulkD + c] = Eb;
        S.unew_d[(size_t)octb * kBulkD + c + 4] = Eb;
        acc.add_bulk(ub[0], ub[1], ub[2], ub[3], Eb, A);
        acc.add_bulk(ub[0], ub[1], ub[2], ub[3], Eb, A);
      }
    }
  }
}

}  // namespace rh
