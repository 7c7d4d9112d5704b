/*
 * A plain C host of the drop-in ABI (include/ramses_hydro.h), standing in for
 * the Fortran host: it lays out uold(1:8,1:5,1:ngridmax) and the 32-byte oct
 * records exactly as RAMSES II does, and runs ten coarse steps of a 32^3
 * Sedov blast in the reference's call order (courant_fine -> set_unew ->
 * godunov_fine -> set_uold, amr/amr_step.f90).  Mass in an outflow box with
 * the ambient gas at rest is conserved to round-off while the blast is inside.
 *
 * Exit status 0: ran and conserved mass, or no CUDA device (prints
 * "no device"); nonzero: an ABI call failed or mass drifted.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ramses_hydro.h"

#define LEV 5
#define NO (1 << (LEV - 1)) /* octs per edge: 16 -> 32^3 cells */

int main(void) {
  int rc = rh_init(0);
  if (rc == RH_ENODEV) {
    printf("no device: %s\n", rh_last_error());
    return 0;
  }
  if (rc) { printf("rh_init: %s\n", rh_last_error()); return 1; }
  const int noct = NO * NO * NO;
  rh_oct* grid = (rh_oct*)calloc(noct, sizeof(rh_oct));
  double* uold = (double*)calloc((size_t)noct * 40, sizeof(double));
  int32_t head[LEV + 1], nocts[LEV + 1];
  memset(head, 0, sizeof head);
  memset(nocts, 0, sizeof nocts);
  head[LEV] = 1;
  nocts[LEV] = noct;
  const double gamma = 1.4, dx = 1.0 / (2 * NO), p0 = 1e-5;
  /* count the blast cells (centre within 2 cells of the box centre) */
  int nin = 0;
  for (int pass = 0; pass < 2; ++pass) {
    const double pin = pass ? (gamma - 1.0) / (nin * dx * dx * dx) : 0.0;
    int ig = 0;
    for (int z = 0; z < NO; ++z)
      for (int y = 0; y < NO; ++y)
        for (int x = 0; x < NO; ++x, ++ig) {
          grid[ig].ckey[0] = x;
          grid[ig].ckey[1] = y;
          grid[ig].ckey[2] = z;
          grid[ig].lev = LEV;
          for (int c = 0; c < 8; ++c) {
            const double cx = (2 * x + (c & 1) + 0.5) * dx - 0.5, cy = (2 * y + ((c >> 1) & 1) + 0.5) * dx - 0.5,
                         cz = (2 * z + (c >> 2) + 0.5) * dx - 0.5;
            const int in = sqrt(cx * cx + cy * cy + cz * cz) <= 2.0 * dx * (1 + 1e-12);
            if (!pass) { nin += in; continue; }
            double* u = uold + (size_t)ig * 40; /* uold(c, var, ig) */
            u[c] = 1.0;
            u[8 + c] = u[16 + c] = u[24 + c] = 0.0;
            u[32 + c] = (in ? pin : p0) / (gamma - 1.0);
          }
        }
  }
  rh_mesh_desc m;
  memset(&m, 0, sizeof m);
  m.nsubgrid = 1;
  m.levelmin = m.levelmax = LEV;
  m.ngridmax = noct;
  for (int d = 0; d < 3; ++d) m.box_nx[d] = 1;
  for (int i = 0; i < 6; ++i) m.bound_type[i] = RH_BOUND_ZERO_GRADIENT;
  m.boxlen = 1.0;
  m.head = head;
  m.noct = nocts;
  m.grid = grid;
  if (rh_set_mesh(&m, uold, 5, 8)) { printf("rh_set_mesh: %s\n", rh_last_error()); return 1; }
  const double g[3] = {0, 0, 0};
  double mass0 = -1, mass = 0, ekin, eint, emag, dt;
  for (int step = 0; step <= 10; ++step) {
    if (rh_cmpdt(1, noct, dx, gamma, 1e-10, 1e-10, 0.8, g, &mass, &ekin, &eint, &emag, &dt)) {
      printf("rh_cmpdt: %s\n", rh_last_error());
      return 1;
    }
    if (mass0 < 0) mass0 = mass;
    if (step == 10) break;
    if (rh_set_unew(1, noct) ||
        rh_godunov(1, noct, noct, LEV, LEV, LEV, gamma, 1e-10, 1e-20, dt, dx, 0.8 * dx / dt, 2, RH_RIEMANN_HLLC, g) ||
        rh_set_uold(1, noct)) {
      printf("step %d: %s\n", step, rh_last_error());
      return 1;
    }
  }
  if (rh_transfer_grid_host(uold, noct, 5, 8) || rh_sync()) { printf("download: %s\n", rh_last_error()); return 1; }
  rh_finalize();
  const double drift = fabs(mass - mass0) / mass0;
  printf("mass %.17g -> %.17g (relative drift %.3g), last dt %.6g, centre rho %.6g\n", mass0, mass, drift, dt,
         uold[((size_t)((NO / 2) * NO * NO + (NO / 2) * NO + NO / 2)) * 40]);
  free(grid);
  free(uold);
  return drift < 1e-12 ? 0 : 2;
}
