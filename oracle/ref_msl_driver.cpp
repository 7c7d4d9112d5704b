// ref_msl_driver.cpp — TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own Metal hydro shader (metal/kernels/hydro.metal,
// a float32 port of gpu/gpu_hydro.cuf) as C++ through the stand-in headers in
// msl_shim/, and exposes its per-interface Riemann solvers and its per-oct
// trace + Riemann pipeline (trace_3d, riemann_driver: one threadgroup with
// one thread) to the tests, which compare them with the FP64 oracle at FP32
// precision.  The shader source is included from the reference checkout by the
// recipe (HYDRO_METAL); nothing of it is copied here.  Built twice: as the
// shader is (float32, librh_ref_msl.so) and with RH_MSL_DOUBLE (every float of
// the shader and of the functions below is double, librh_ref_msl64.so), which
// pins the oracle to the shader's algorithm at FP64 rounding.
#include HYDRO_METAL

extern "C" {

// One interface: q = (rho, un, ut1, ut2, p); flux = (mass, mom n, t1, t2, energy).
int ref_msl_riemann(int solver, const float* ql, const float* qr, float gamma, float smallr, float smallc2,
                    float smax_cap, float* flux) {
  primitive_t L, R;
  L.density = ql[0]; L.velocity_x = ql[1]; L.velocity_y = ql[2]; L.velocity_z = ql[3]; L.pressure = ql[4];
  R.density = qr[0]; R.velocity_x = qr[1]; R.velocity_y = qr[2]; R.velocity_z = qr[3]; R.pressure = qr[4];
  conserved_t f = riemann_fluxes(L, R, gamma, smallr, smallc2, smax_cap, solver);
  flux[0] = f.density; flux[1] = f.momentum_x; flux[2] = f.momentum_y; flux[3] = f.momentum_z; flux[4] = f.energy;
  return 0;
}

// The fluxes of one oct (nsubgrid 1) from a 6^3 conserved stencil u[var][k][j][i]
// (i fastest): out[dim][var][a][b][c] with (a, b, c) the face grid of that
// direction in (k, j, i) order, 3 faces along the normal and 2 x 2 across.
int ref_msl_oct_fluxes(const float* u, float gamma, float smallr, float smallc2, float dtdx, float smax_cap,
                       int slope, int riemann, float* out) {
  static local_subgrid_t ls;
  static interfaces_x_t lx, rx;
  static interfaces_y_t ly, ry;
  static interfaces_z_t lz, rz;
  for (int k = 0; k < 6; ++k)
    for (int j = 0; j < 6; ++j)
      for (int i = 0; i < 6; ++i) {
        conserved_t c;
        const int o = (k * 6 + j) * 6 + i;
        c.density = u[0 * 216 + o];
        c.momentum_x = u[1 * 216 + o];
        c.momentum_y = u[2 * 216 + o];
        c.momentum_z = u[3 * 216 + o];
        c.energy = u[4 * 216 + o];
        primitive_t p = conserved_2_primitive(c, gamma, smallr, smallc2);
        ls.density[i][j][k] = p.density;
        ls.velocity_x[i][j][k] = p.velocity_x;
        ls.velocity_y[i][j][k] = p.velocity_y;
        ls.velocity_z[i][j][k] = p.velocity_z;
        ls.pressure[i][j][k] = p.pressure;
      }
  trace_3d(ls, 0, 1u, lx, rx, ly, ry, lz, rz, gamma, smallr, smallc2, dtdx, slope);
  riemann_driver(lx, rx, ly, ry, lz, rz, 0, 1u, gamma, smallr, smallc2, smax_cap, riemann);
  // x faces: left_x[i][j][k] i in 0..2 (faces), j, k in 0..1
  for (int v = 0; v < 5; ++v)
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int c = 0; c < 3; ++c) {
          const float* fx[5] = {&lx.density[c][b][a], &lx.velocity_x[c][b][a], &lx.velocity_y[c][b][a],
                                &lx.velocity_z[c][b][a], &lx.pressure[c][b][a]};
          out[((0 * 5 + v) * 2 + a) * 6 + b * 3 + c] = *fx[v];
        }
  for (int v = 0; v < 5; ++v)
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 3; ++b)
        for (int c = 0; c < 2; ++c) {
          const float* fy[5] = {&ly.density[c][b][a], &ly.velocity_x[c][b][a], &ly.velocity_y[c][b][a],
                                &ly.velocity_z[c][b][a], &ly.pressure[c][b][a]};
          out[60 + ((v * 2 + a) * 3 + b) * 2 + c] = *fy[v];
        }
  for (int v = 0; v < 5; ++v)
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 2; ++b)
        for (int c = 0; c < 2; ++c) {
          const float* fz[5] = {&lz.density[c][b][a], &lz.velocity_x[c][b][a], &lz.velocity_y[c][b][a],
                                &lz.velocity_z[c][b][a], &lz.pressure[c][b][a]};
          out[120 + ((v * 3 + a) * 2 + b) * 2 + c] = *fz[v];
        }
  return 0;
}

// One Godunov step of a level through the shader's hydro_integrator_kernel:
// every oct is one threadgroup run by a single thread (the shader's loops take
// the thread count as their stride, its barriers separate the phases).
// unew must hold uold on entry; nbor is the shader's [ngridmax][27] table of
// 1-based neighbour octs (x fastest).
int ref_msl_godunov(const oct_t* grid, const float* uold, float* unew, const int* nbor, int head_idx, int noct,
                    int ngridmax, int ilevel, int levelmin, int levelmax, float gamma, float smallr, float smallc2,
                    float dt, float dx, int slope, int riemann, const float* grav, float smax_cap) {
  for (int b = 0; b < noct; ++b)
    hydro_integrator_kernel(grid, uold, unew, nbor, head_idx, noct, ngridmax, ilevel, levelmin, levelmax, gamma,
                            smallr, smallc2, dt, dx, slope, riemann, grav, nullptr, nullptr, smax_cap, (uint)b, 0u,
                            1u);
  return 0;
}

// Restriction of a fine level into its parents through the shader's
// upload_kernel, one thread per fine oct; father[] holds the 1-based parent
// oct of every oct.
int ref_msl_upload(const oct_t* grid, const int* father, float* uold, int head_idx, int num_octs,
                   int internal_energy, float gamma, float smallr, float smallc2) {
  for (int t = 0; t < num_octs; ++t)
    upload_kernel(grid, father, uold, head_idx, num_octs, internal_energy, gamma, smallr, smallc2, (uint)t);
  return 0;
}

// courant_fine of a level through the shader's cmpdt_kernel, run one thread at
// a time (one-lane SIMD groups): out = (mass, ekin, eint, emag, dt).
int ref_msl_cmpdt(const oct_t* grid, const float* uold, int head_idx, int num_octs, float dx, float gamma,
                  float smallr, float smallc2, float courant, const float* grav, float* out) {
  metal::atomic_uint data[5];
  for (int i = 0; i < 4; ++i) data[i].v = 0u;
  data[4].v = metal::as_type<uint>((float)HUGE_VAL);  // +inf of the build's float (double in the FP64 build)
  const long long nthreads = (long long)num_octs * TWOTONDIM;
  for (long long t = 0; t < nthreads; ++t)
    cmpdt_kernel(grid, uold, data, head_idx, num_octs, dx, gamma, smallr, smallc2, courant, grav, nullptr,
                 (uint)(t % 1024), (uint)(t / 1024), 0u, 0u, 32u);
  for (int i = 0; i < 5; ++i) out[i] = metal::as_type<float>(data[i].v);
  return 0;
}

}  // extern "C"
