// rh_vec.cuh — lane arithmetic shared by the precision paths.
//
// A "lane value" V is either
//   double : one cell, plain FP64 path;
//   float2 : two cells (the two z-planes of an oct layer), FP32-bulk path,
//            using sm_100's packed FP32x2 add/mul/fma (__fadd2_rn/__fmul2_rn/
//            __ffma2_rn), so one issued instruction advances both cells.
// Min/max/compare/select act per component.  Reciprocal and square root:
//   double: hardware approximation (rcp.approx.ftz.f64 / rsqrt.approx.ftz.f64)
//           refined by Newton-Raphson iterations to full double precision
//           (within 2 ulp; arguments are positive normal numbers here);
//   float : rcp.approx.ftz.f32 / sqrt.approx.ftz.f32 (about 1 ulp).
#pragma once
#include <cuda_runtime.h>

namespace rh {

// ---------------------------------------------------------------- double ---
__device__ __forceinline__ double vfma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ double vmin(double a, double b) { return a < b ? a : b; }  // Fortran MIN
__device__ __forceinline__ double vmax(double a, double b) { return a > b ? a : b; }  // Fortran MAX
__device__ __forceinline__ double vabs(double a) { return fabs(a); }
__device__ __forceinline__ double vcopysign(double a, double b) { return copysign(a, b); }
__device__ __forceinline__ double vsel(bool m, double a, double b) { return m ? a : b; }
__device__ __forceinline__ bool vlt(double a, double b) { return a < b; }
__device__ __forceinline__ bool vgt(double a, double b) { return a > b; }
__device__ __forceinline__ bool vle(double a, double b) { return a <= b; }
__device__ __forceinline__ bool mand(bool a, bool b) { return a && b; }
__device__ __forceinline__ bool mor(bool a, bool b) { return a || b; }
__device__ __forceinline__ bool mnot(bool a) { return !a; }
__device__ __forceinline__ bool many(bool a) { return a; }

// 1/x for positive normal x: y0 from the hardware estimate, then two
// Newton-Raphson steps y <- y + y(1 - x y) (quadratic convergence).
__device__ __forceinline__ double vrcp(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}
// sqrt(x) for positive normal x: reciprocal square root estimate, two
// Newton-Raphson steps y <- y + y(1 - x y^2)/2, then s = x y corrected by one
// Heron/Newton step s <- s + (x - s^2) y/2.
__device__ __forceinline__ double vsqrt(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double hy = 0.5 * y;
  double r = fma(-x * y, y, 1.0);
  y = fma(hy, r, y);
  hy = 0.5 * y;
  r = fma(-x * y, y, 1.0);
  y = fma(hy, r, y);
  double s = x * y;
  double d = fma(-s, s, x);
  return fma(0.5 * y, d, s);
}

// ---------------------------------------------------------------- float2 ---
struct M2 {
  bool x, y;
};
__device__ __forceinline__ float2 operator+(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 operator-(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 operator-(float2 a, float2 b) { return __fadd2_rn(a, -b); }
__device__ __forceinline__ float2 operator*(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 vfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// a - b rounded once per lane, never merged into a multiply-add with the
// products that formed a or b
__device__ __forceinline__ float2 vsub_nc(float2 a, float2 b) {
  float2 r;
  asm("sub.rn.f32 %0, %2, %4;\n\tsub.rn.f32 %1, %3, %5;"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
// Fortran MIN / MAX of ordered (NaN-free) operands as one FMNMX per lane;
// the results differ from a compare-and-select at most in the sign of a zero.
__device__ __forceinline__ float2 vmin(float2 a, float2 b) { return make_float2(fminf(a.x, b.x), fminf(a.y, b.y)); }
__device__ __forceinline__ float2 vmax(float2 a, float2 b) { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
__device__ __forceinline__ float2 vabs(float2 a) { return make_float2(fabsf(a.x), fabsf(a.y)); }
__device__ __forceinline__ float2 vcopysign(float2 a, float2 b) {
  return make_float2(copysignf(a.x, b.x), copysignf(a.y, b.y));
}
__device__ __forceinline__ float2 vsel(M2 m, float2 a, float2 b) {
  return make_float2(m.x ? a.x : b.x, m.y ? a.y : b.y);
}
__device__ __forceinline__ M2 vlt(float2 a, float2 b) { return {a.x < b.x, a.y < b.y}; }
__device__ __forceinline__ M2 vgt(float2 a, float2 b) { return {a.x > b.x, a.y > b.y}; }
__device__ __forceinline__ M2 vle(float2 a, float2 b) { return {a.x <= b.x, a.y <= b.y}; }
__device__ __forceinline__ M2 mand(M2 a, M2 b) { return {a.x && b.x, a.y && b.y}; }
__device__ __forceinline__ M2 mor(M2 a, M2 b) { return {a.x || b.x, a.y || b.y}; }
__device__ __forceinline__ M2 mnot(M2 a) { return {!a.x, !a.y}; }
__device__ __forceinline__ bool many(M2 a) { return a.x || a.y; }

__device__ __forceinline__ float frcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float fsqrt_approx(float x) {
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float2 vrcp(float2 x) { return make_float2(frcp_approx(x.x), frcp_approx(x.y)); }
__device__ __forceinline__ float2 vsqrt(float2 x) { return make_float2(fsqrt_approx(x.x), fsqrt_approx(x.y)); }

// broadcast of a scalar constant to a lane value
template <class V> struct Lane;
template <> struct Lane<double> {
  using S = double;
  using M = bool;
  static __device__ __forceinline__ double bc(double s) { return s; }
};
template <> struct Lane<float2> {
  using S = float;
  using M = M2;
  static __device__ __forceinline__ float2 bc(float s) { return make_float2(s, s); }
};

}  // namespace rh
