// rh_godunov2.cuh — FP32-bulk Godunov pencil kernel: one oct layer (two cell
// planes, z = 2K and 2K+1) per iteration, each thread advancing both cells of
// its column with packed FP32x2 arithmetic (lane type float2: .x = plane 2K,
// .y = plane 2K+1).
//
// Precision policy: density and momenta are stored and computed in FP32; the
// total energy is stored and updated in FP64, the pressure is recovered in
// FP64 from E minus the kinetic energy (high-Mach and near-vacuum cells), and
// the CFL dt and conserved totals are evaluated in FP64 on the new state.
//
// z interfaces of a layer, as one packed Riemann solve:
//   .x: face 2K-1/2 (left = upper state of plane 2K-1, right = lower of 2K)
//   .y: face 2K+1/2 (left = upper state of plane 2K,   right = lower of 2K+1)
// Plane 2K is finished in the same iteration; plane 2K+1 waits one iteration
// for the flux through face 2K+3/2.
#pragma once
#include "rh_godunov.cuh"

namespace rh {

// ctoprim of both cells of a column in one staged oct (umuscl.f90:1739-1901),
// pressure recovered in FP64.  ca/cb: cell indices of planes 2K and 2K+1.
__device__ __forceinline__ void ctoprim_f32x2(const float* sf, const double* sd, int ca, int cb, bool fx, bool fy,
                                              bool fz, const HydroK<float2>& H, double gm1, double smalle,
                                              float2* q, float2& ir, float2* U, double* E) {
  float2 d = make_float2(sf[ca], sf[cb]);
  float2 mx = make_float2(sf[8 + ca], sf[8 + cb]);
  float2 my = make_float2(sf[16 + ca], sf[16 + cb]);
  float2 mz = make_float2(sf[24 + ca], sf[24 + cb]);
  E[0] = sd[ca];
  E[1] = sd[cb];
  if (fx) mx = -mx;
  if (fy) my = -my;
  if (fz) mz = -mz;
  U[0] = d; U[1] = mx; U[2] = my; U[3] = mz;
  const float2 r = vmax(d, H.smallr);
  ir = vrcp(r);
  const float2 u = mx * ir, v = my * ir, w = mz * ir;
  const float2 k2 = vfma(u, u, vfma(v, v, w * w));
  // FP64 pressure recovery: eint = E - rho |v|^2 / 2
  double e0 = E[0] - 0.5 * (double)r.x * (double)k2.x;
  double e1 = E[1] - 0.5 * (double)r.y * (double)k2.y;
  const double m0 = smalle * (double)r.x, m1 = smalle * (double)r.y;
  e0 = e0 > m0 ? e0 : m0;
  e1 = e1 > m1 ? e1 : m1;
  q[0] = r;
  q[1] = u + H.grav[0];
  q[2] = v + H.grav[1];
  q[3] = w + H.grav[2];
  q[4] = make_float2((float)(gm1 * e0), (float)(gm1 * e1));
}

// Flux reset and coarse corrections of one x or y face of a layer, per plane
// (.x plane 2K, .y plane 2K+1); bl/br: status bits (a | b<<8) of the cells
// left/right of the face, el/er their oct entries.
__device__ __forceinline__ void amr_face_f32(const LevelArgs& A, const StateArgs<float>& S, float2* f, uint32_t bl,
                                             uint32_t br, int el, int er) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uint32_t l = (bl >> (8 * h)) & 0xffu, r = (br >> (8 * h)) & 0xffu;
    float c[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) c[n] = h ? f[n].y : f[n].x;
    if ((l | r) & 1u) {
#pragma unroll
      for (int n = 0; n < 5; ++n) c[n] = 0.f;
    }
    if ((l & 2u) && (r & 4u)) coarse_add_f32(A, S.unew_f, S.unew_d, er, c, 1.f);
    if ((l & 4u) && (r & 2u)) coarse_add_f32(A, S.unew_f, S.unew_d, el, c, -1.f);
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      if (h) f[n].y = c[n];
      else f[n].x = c[n];
    }
  }
}

template <int TXO, int TYO, int MINB, int SLOPE, int RIEMANN, bool AMR>
__global__ void __launch_bounds__(Geo<float, float2, TXO, TYO>::NT, MINB)
godunov_pencil2_kernel(const LevelArgs A, const StateArgs<float> S, const HydroK<float2> H) {
  using G = Geo<float, float2, TXO, TYO>;
  extern __shared__ __align__(16) unsigned char smem[];
  float2* Qb = reinterpret_cast<float2*>(smem + G::oQ);    // [2][5][NLC]
  float2* FS = reinterpret_cast<float2*>(smem + G::oFS);   // [10][NRC]
  float2* FXY = reinterpret_cast<float2*>(smem + G::oFX);  // [2][5][NRC]
  double* red = reinterpret_cast<double*>(smem + G::oRed);
  int* entb = reinterpret_cast<int*>(smem + G::oAmr);                                   // AMR: entry of layer K
  uint32_t* stb = reinterpret_cast<uint32_t*>(smem + G::oAmr + G::NRC * sizeof(int));  // AMR: bits a | b<<8
  __shared__ int s_abort;

  const int t = threadIdx.x;
  const int pencil = blockIdx.x;
  const int4 hdr = A.phdr[pencil];
  const int ox0 = hdr.x, oy0 = hdr.y, oz0 = hdr.z, L = hdr.w;
  const int* tab = A.ptab + A.poff[pencil];
  Columns<G> col;
  col.init(t, ox0, oy0, A);
  Stager<float, G> stg{reinterpret_cast<double*>(smem + G::oStageD), reinterpret_cast<float*>(smem + G::oStageF),
                       reinterpret_cast<uint64_t*>(smem + G::oBar), &s_abort, tab, S.uold_d, S.uold_f, A.err};
  stg.init_barriers();
  __syncthreads();
  stg.issue(0);
  stg.issue(1);
  const bool active = t < G::NRC;
  const int cxy = (col.rx & 1) + 2 * (col.ry & 1);
  const int ocxy = (col.orx & 1) + 2 * (col.ory & 1);

  // Convert layer K (table row K+1) of the own column (registers + plane
  // buffer) and of the owned outer column (plane buffer).
  auto convert = [&](int K, float2* q, float2& ir, float2* U, double* E) {
    const int row = K + 1;
    const CellMap ma = map_coord(2 * oz0 + 2 * K, A.ncz, A.periodic[2], A.btype[4], A.btype[5]);
    const CellMap mb = map_coord(2 * oz0 + 2 * K + 1, A.ncz, A.periodic[2], A.btype[4], A.btype[5]);
    float2* Qp = Qb + (size_t)(K & 1) * 5 * G::NLC;
    const int pa = col.mx.parity + 2 * col.my.parity;
    if (active) {
      ctoprim_f32x2(stg.slot_f(row, col.slot), stg.slot_d(row, col.slot), pa + 4 * ma.parity, pa + 4 * mb.parity,
                    col.mx.flip, col.my.flip, ma.flip, H, A.gm1_d, A.smalle_d, q, ir, U, E);
#pragma unroll
      for (int n = 0; n < 5; ++n) Qp[n * G::NLC + col.lc] = q[n];
    }
    if (col.has_outer) {
      float2 qo[5], iro, Uo[4];
      double Eo[2];
      const int po = col.omx.parity + 2 * col.omy.parity;
      ctoprim_f32x2(stg.slot_f(row, col.oslot), stg.slot_d(row, col.oslot), po + 4 * ma.parity, po + 4 * mb.parity,
                    col.omx.flip, col.omy.flip, ma.flip, H, A.gm1_d, A.smalle_d, qo, iro, Uo, Eo);
#pragma unroll
      for (int n = 0; n < 5; ++n) Qp[n * G::NLC + col.olc] = qo[n];
    }
    (void)ocxy;
  };
  // AMR: entry of layer K and status bits of its two planes (a | b << 8)
  auto status = [&](int K, int& ent) -> uint32_t {
    const int row = K + 1;
    ent = tab[(long long)row * G::NSLOT + col.slot];
    uint32_t bits = 0;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int p = 2 * K + h;
      const CellMap mz = map_coord(2 * oz0 + p, A.ncz, A.periodic[2], A.btype[4], A.btype[5]);
      const int gz = 2 * oz0 + p;
      const bool in_dom = col.in_dom_xy && gz >= 0 && gz < A.ncz;
      const bool upd = col.interior && in_dom && K >= 0 && K < L;
      bits |= amr_bits(A, ent, col.mx.parity + 2 * col.my.parity + 4 * mz.parity, upd, in_dom) << (8 * h);
    }
    return bits;
  };

  float2 cur[5], nxt[5], irc, irn;
  float prv_b[5];
  float2 Uc[4], Un[4];
  double Ec[2], En[2];
  float2 qmx[5], qmy[5];
  float qmz_b[5];                 // upper z state of plane 2K-1
  float upb[4], fzb[5];           // pending plane 2K-1: x/y-updated bulk values, flux at face 2K-1/2
  double upbE = 0;
  int pend_oct = -1;
  bool pend_ref = false;
  int ec = -1, en = -1, ep = -1;       // AMR: entries of layers K, K+1, K-1
  uint32_t sc = 0, sn = 0, sp = 0;     // AMR: status bits of layers K, K+1, K-1
  CflAcc acc;
#pragma unroll
  for (int n = 0; n < 5; ++n) { qmz_b[n] = 0.f; fzb[n] = 0.f; }
#pragma unroll
  for (int n = 0; n < 4; ++n) upb[n] = 0.f;
  Ec[0] = Ec[1] = En[0] = En[1] = 0.0;

  // prologue: layer -1 (table row 0)
  stg.wait(0);
  convert(-1, cur, irc, Uc, Ec);
  if (AMR && active) sc = status(-1, ec);
#pragma unroll
  for (int n = 0; n < 5; ++n) prv_b[n] = cur[n].x;  // plane -3 is never used
  __syncthreads();
  if (L + 1 >= 2) stg.issue(2);

  for (int K = -1; K <= L; ++K) {
    // (A) primitive variables of layer K+1
    if (K + 1 <= L) {
      stg.wait(K + 2);
      convert(K + 1, nxt, irn, Un, En);
      if (AMR && active) sn = status(K + 1, en);
    } else {
#pragma unroll
      for (int n = 0; n < 5; ++n) nxt[n] = cur[n];  // plane 2L+2 only feeds the unused plane 2L+1
      irn = irc;
    }
    // (C) slopes, predictor and interface states of layer K
    float2 fz[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) fz[n] = make_float2(0.f, 0.f);
    if (active) {
      const float2* Qk = Qb + (size_t)(K & 1) * 5 * G::NLC;
      float2 xm[5], xp[5], ym[5], yp[5], zm[5], zp[5];
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        xm[n] = Qk[n * G::NLC + col.lc - 1];
        xp[n] = Qk[n * G::NLC + col.lc + 1];
        ym[n] = Qk[n * G::NLC + col.lc - G::LW];
        yp[n] = Qk[n * G::NLC + col.lc + G::LW];
        zm[n] = make_float2(prv_b[n], cur[n].x);
        zp[n] = make_float2(cur[n].y, nxt[n].x);
      }
      float2 d[3][5];
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        d[0][n] = limited_slope<float2, SLOPE>(xm[n], cur[n], xp[n], H);
        d[1][n] = limited_slope<float2, SLOPE>(ym[n], cur[n], yp[n], H);
        d[2][n] = limited_slope<float2, SLOPE>(zm[n], cur[n], zp[n], H);
      }
      if (SLOPE > 0) {
        d[0][1] = momentum_bound(d[0][1], xm[0], xm[1], cur[1], xp[0], xp[1], irc, H);
        d[1][2] = momentum_bound(d[1][2], ym[0], ym[2], cur[2], yp[0], yp[2], irc, H);
        d[2][3] = momentum_bound(d[2][3], zm[0], zm[3], cur[3], zp[0], zp[3], irc, H);
      }
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int n = 0; n < 5; ++n) d[a][n] = H.half * d[a][n];
      float2 qm[3][5], qp[3][5];
      trace_cell(cur, irc, d, qm, qp, H);
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        FS[n * G::NRC + t] = qp[0][n];
        FS[(5 + n) * G::NRC + t] = qp[1][n];
        qmx[n] = qm[0][n];
        qmy[n] = qm[1][n];
      }
      if (col.interior && K >= 0) {
        // rotation (r, w, u, v, p)
        const int rot[5] = {0, 3, 1, 2, 4};
        float2 ql[5], qr[5], f[5];
#pragma unroll
        for (int n = 0; n < 5; ++n) {
          ql[n] = make_float2(qmz_b[rot[n]], qm[2][rot[n]].x);
          qr[n] = qp[2][rot[n]];
        }
        riemann_dtdx<float2, RIEMANN>(ql, qr, f, H);
        fz[0] = f[0]; fz[3] = f[1]; fz[1] = f[2]; fz[2] = f[3]; fz[4] = f[4];
        if (AMR) {
          // face .x: plane 2K-1 (layer K-1, plane b) / plane 2K (layer K, plane a);
          // face .y: the two planes of layer K (one oct: never coarse-fine)
          const uint32_t lo = sp >> 8, a = sc & 0xffu, b = sc >> 8;
          if ((lo | a) & 1u) {
#pragma unroll
            for (int n = 0; n < 5; ++n) fz[n].x = 0.f;
          }
          if ((a | b) & 1u) {
#pragma unroll
            for (int n = 0; n < 5; ++n) fz[n].y = 0.f;
          }
          float fx_[5];
#pragma unroll
          for (int n = 0; n < 5; ++n) fx_[n] = fz[n].x;
          if ((lo & 2u) && (a & 4u)) coarse_add_f32(A, S.unew_f, S.unew_d, ec, fx_, 1.f);
          if ((lo & 4u) && (a & 2u)) coarse_add_f32(A, S.unew_f, S.unew_d, ep, fx_, -1.f);
        }
      }
      if (AMR) {
        entb[t] = ec;
        stb[t] = sc;
      }
#pragma unroll
      for (int n = 0; n < 5; ++n) qmz_b[n] = qm[2][n].y;
    }
    __syncthreads();  // S2: interface states of layer K published
    if (K + 4 <= L + 1) stg.issue(K + 4);
    // (D) x flux at the right face and y flux at the top face, both planes
    const bool layer_ok = K >= 0 && K < L;
    if (active && layer_ok) {
      if (col.rx >= -1 && col.rx < G::CX && col.ry >= 0 && col.ry < G::CY) {
        float2 qr[5], f[5];
#pragma unroll
        for (int n = 0; n < 5; ++n) qr[n] = FS[n * G::NRC + t + 1];
        riemann_dtdx<float2, RIEMANN>(qmx, qr, f, H);
        if (AMR) amr_face_f32(A, S, f, stb[t], stb[t + 1], entb[t], entb[t + 1]);
#pragma unroll
        for (int n = 0; n < 5; ++n) FXY[n * G::NRC + t] = f[n];
      }
      if (col.ry >= -1 && col.ry < G::CY && col.rx >= 0 && col.rx < G::CX) {
        const int tn = t + G::RW;
        const float2 ql[5] = {qmy[0], qmy[2], qmy[1], qmy[3], qmy[4]};
        const float2 qr[5] = {FS[5 * G::NRC + tn], FS[7 * G::NRC + tn], FS[6 * G::NRC + tn], FS[8 * G::NRC + tn],
                              FS[9 * G::NRC + tn]};
        float2 f[5];
        riemann_dtdx<float2, RIEMANN>(ql, qr, f, H);
        float2 fy[5] = {f[0], f[2], f[1], f[3], f[4]};
        if (AMR) amr_face_f32(A, S, fy, stb[t], stb[tn], entb[t], entb[tn]);
        float2* FY = FXY + 5 * G::NRC;
#pragma unroll
        for (int n = 0; n < 5; ++n) FY[n * G::NRC + t] = fy[n];
      }
    }
    __syncthreads();  // S3: fluxes of layer K published
    // (E) finish plane 2K-1 (pending) and plane 2K; keep plane 2K+1 pending
    if (active && col.interior) {
      if (pend_oct >= 0) {
        float* o = S.unew_f + (size_t)pend_oct * 32 + cxy + 4;
        float ub[4];
#pragma unroll
        for (int n = 0; n < 4; ++n) ub[n] = upb[n] + (fzb[n] - fz[n].x);
        const double Eb = upbE + (double)(fzb[4] - fz[4].x);
        o[0] = ub[0]; o[8] = ub[1]; o[16] = ub[2]; o[24] = ub[3];
        S.unew_d[(size_t)pend_oct * 8 + cxy + 4] = Eb;
        if (A.cfl_partial && !pend_ref) acc.add(ub[0], ub[1], ub[2], ub[3], Eb, A);
        pend_oct = -1;
      }
      if (layer_ok) {
        const float2* FX = FXY;
        const float2* FY = FXY + 5 * G::NRC;
        const int gz = 2 * oz0 + 2 * K;
        const int oct = tab[(long long)(K + 1) * G::NSLOT + col.slot];
        const bool ok = col.in_domain_xy && gz < A.ncz && oct >= 0 && oct < A.ghost_base;
        float2 base[4];
        double Eba[2] = {Ec[0], Ec[1]};
#pragma unroll
        for (int n = 0; n < 4; ++n) base[n] = Uc[n];
        if (AMR && A.accumulate && ok) {
          // unew holds uold plus the finer level's coarse corrections
          const float* o = S.unew_f + (size_t)oct * 32 + cxy;
#pragma unroll
          for (int n = 0; n < 4; ++n) base[n] = make_float2(o[8 * n], o[8 * n + 4]);
          Eba[0] = S.unew_d[(size_t)oct * 8 + cxy];
          Eba[1] = S.unew_d[(size_t)oct * 8 + cxy + 4];
        }
        // reference order per cell: ((u + dFx) + dFy) + dFz
        float2 u2[4];
#pragma unroll
        for (int n = 0; n < 4; ++n)
          u2[n] = (base[n] + (FX[n * G::NRC + t - 1] - FX[n * G::NRC + t])) +
                  (FY[n * G::NRC + t - G::RW] - FY[n * G::NRC + t]);
        const double ea = (Eba[0] + (double)(FX[4 * G::NRC + t - 1].x - FX[4 * G::NRC + t].x)) +
                          (double)(FY[4 * G::NRC + t - G::RW].x - FY[4 * G::NRC + t].x);
        const double eb = (Eba[1] + (double)(FX[4 * G::NRC + t - 1].y - FX[4 * G::NRC + t].y)) +
                          (double)(FY[4 * G::NRC + t - G::RW].y - FY[4 * G::NRC + t].y);
        if (ok) {
          float ua[4];
#pragma unroll
          for (int n = 0; n < 4; ++n) ua[n] = u2[n].x + (fz[n].x - fz[n].y);
          const double Ea = ea + (double)(fz[4].x - fz[4].y);
          float* o = S.unew_f + (size_t)oct * 32 + cxy;
          o[0] = ua[0]; o[8] = ua[1]; o[16] = ua[2]; o[24] = ua[3];
          S.unew_d[(size_t)oct * 8 + cxy] = Ea;
          if (A.cfl_partial && !(AMR && (sc & 1u))) acc.add(ua[0], ua[1], ua[2], ua[3], Ea, A);
#pragma unroll
          for (int n = 0; n < 4; ++n) { upb[n] = u2[n].y; fzb[n] = fz[n].y; }
          fzb[4] = fz[4].y;
          upbE = eb;
          pend_oct = (gz + 1 < A.ncz) ? oct : -1;
          pend_ref = AMR && ((sc >> 8) & 1u);
        }
      }
    }
#pragma unroll
    for (int n = 0; n < 5; ++n) { prv_b[n] = cur[n].y; cur[n] = nxt[n]; }
#pragma unroll
    for (int n = 0; n < 4; ++n) Uc[n] = Un[n];
    Ec[0] = En[0];
    Ec[1] = En[1];
    irc = irn;
    ep = ec; ec = en;
    sp = sc; sc = sn;
  }
  if (A.cfl_partial) cfl_block_reduce<G::NWARP>(acc, red, A.cfl_partial + (size_t)pencil * 5);
}

}  // namespace rh
