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
// cr / cl: the x, y part of the ghost cell's index when the ghost is on the
// right (above) or left (below) of the face; dir: 0 x faces, 1 y faces.  The
// lanes are the two planes (z parity h) of the layer.
__device__ __forceinline__ void amr_face_f32(const LevelArgs& A, const StateArgs<float>& S, float2* f, uint32_t bl,
                                             uint32_t br, int el, int er, int cr, int cl, int dir) {
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
    if ((l & 2u) && (r & 4u)) coarse_add_f32(A, S.unew_f, S.unew_d, er, c, 1.f, 3 * (cr + 4 * h) + dir);
    if ((l & 4u) && (r & 2u)) coarse_add_f32(A, S.unew_f, S.unew_d, el, c, -1.f, 3 * (cl + 4 * h) + dir);
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      if (h) f[n].y = c[n];
      else f[n].x = c[n];
    }
  }
}

// One pencil of the FP32-bulk step for a persistent CTA (as pencil_body_f64).
template <int TXO, int TYO, int SLOPE, int RIEMANN, bool AMR, bool DENSE, class Sink>
__device__ __forceinline__ void pencil_body_f32(const LevelArgs& A, const StateArgs<float>& S,
                                                const HydroK<float2>& H, const int4 hdr, const int* tab, int rbase,
                                                const Sink sink) {
  constexpr bool init_barriers = false;
#include "rh_pencil_f32.inc"
}

// One pencil per CTA (the level's pencil table gives hdr and tab).
template <int TXO, int TYO, int MINB, int SLOPE, int RIEMANN, bool AMR>
__global__ void __launch_bounds__(Geo<float, float2, TXO, TYO>::NT, MINB)
godunov_pencil2_kernel(const LevelArgs A, const StateArgs<float> S, const HydroK<float2> H) {
  constexpr bool DENSE = false;
  constexpr bool init_barriers = true;
  constexpr int rbase = 0;
  const GridCflSink sink{};
  const int4 hdr = A.phdr[blockIdx.x];
  const int* tab = A.ptab + A.poff[blockIdx.x];
#include "rh_pencil_f32.inc"
}

}  // namespace rh
