/*
 * rh_oracle.h — TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement (FP64, loop-faithful) of RAMSES II's unsplit MUSCL-Hancock
 * Godunov hydro step, used as the checker for the CUDA path.  Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs may
 * load this library; the product path never links or calls it.
 *
 * Parity status: the Fortran reference binary cannot be built (no Fortran
 * compiler in the image) and the reference ships no golden vectors for this
 * path.  The restatement is pinned (a) against the reference's own code: its
 * Metal port of the GPU hydro kernel (metal/kernels/hydro.metal, float32,
 * mirroring gpu/gpu_hydro.cuf) compiles as C++ (oracle/Makefile target `ref`)
 * and agrees with this oracle at FP32 rounding for the Riemann solvers, the
 * per-oct trace + Riemann pipeline of every slope type, courant_fine and a
 * whole Godunov step of a periodic level; and
 * (b) by known-answer physics (analytic Sedov solution from the reference's
 * utils/py/sedov.py, exact conservation, symmetry, rotation invariance).
 * FP64 bit-level agreement with the Fortran CPU path stays unverifiable here.
 *
 * Every function cites the reference file:line it restates.
 */
#ifndef RH_ORACLE_H
#define RH_ORACLE_H

#include <stdint.h>
#include "../include/ramses_hydro.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One HLLC/HLL/LLF interface solve: qleft/qright = (rho, un, ut1, ut2, p),
 * fgdnv[0..5] = (mass, normal mom, t1 mom, t2 mom, energy, internal-energy).
 * godunov_utils.f90:338-852 */
int rh_oracle_riemann(int solver, const double* qleft, const double* qright,
                      const rh_hydro_params* p, double smax_cap, double* fgdnv);

/* unsplit() on one gathered stencil (umuscl.f90:20-292).
 * nn = 2*nsubgrid cells per tile edge; uin is Fortran-ordered
 * uin(-1:nn+2,-1:nn+2,-1:nn+2,1:5); flux_out is flux(1:nn+1,1:nn+1,1:nn+1,1:5,1:3)
 * holding fx*dt/dx (entries outside the ranges unsplit writes are left 0). */
int rh_oracle_unsplit(int nn, const double* uin, double dx, double dt,
                      const rh_hydro_params* p, double* flux_out);

/* cmpdt() for one cell (godunov_utils.f90:228-333); uu = conserved (5). */
double rh_oracle_cmpdt(const double* uu, const double* grav, double dx,
                       const rh_hydro_params* p, int ndim);

/* Smallest cmpdt() over every cell of noct octs of uold(1:8,1:5,1:noct),
 * in ndim directions (courant_fine's cell loop, hydro/courant_fine.f90:112-168). */
double rh_oracle_cmpdt_octs(const double* uold, long long noct, const double* grav, double dx,
                            const rh_hydro_params* p, int ndim, int nthreads);

/* interpol_hydro() (interpol_hydro.f90:5-109): u1(0:6,1:5) -> u2(1:8,1:5),
 * both Fortran-ordered (first index fastest). */
int rh_oracle_interpol_hydro(const double* u1, double* u2, int interpol_var,
                             int interpol_type, double smallr);

/* godunov_fine() for one level (godunov_fine.f90:43-79 + godfine1 244-1342).
 * uold/unew are Fortran-ordered uold(1:8,1:5,1:ngrid) with oct igrid stored at
 * offset (igrid-1)*40.  unew must already hold set_unew's copy (and any
 * coarse-update contributions of finer levels).  nthreads>1 parallelises over
 * oct blocks when no coarse update is needed (ilevel==levelmin). */
int rh_oracle_godunov_fine(const rh_mesh_desc* m, const rh_hydro_params* p,
                           int ilevel, double dt, const double* uold,
                           double* unew, int nthreads);

/* courant_fine() for one level (courant_fine.f90:57-168).
 * out = (mass, ekin, eint, emag, dt). */
int rh_oracle_courant_fine(const rh_mesh_desc* m, const rh_hydro_params* p,
                           int ilevel, const double* uold, double* out);

const char* rh_oracle_last_error(void);

/* upload_fine: restriction of level ilevel+1 into the refined cells of level
 * ilevel, in place on uold (hydro/upload.f90:74-271). */
int rh_oracle_upload_fine(const rh_mesh_desc* m, const rh_hydro_params* p, int ilevel, double* uold);

/* hydro_flag's gradient branch (hydro/hydro_flag.f90:7-159 with
 * hydro_refine, hydro/godunov_utils.f90:6-223) for the cells of a level;
 * flag1 is (1:8, 1:ngridmax) int32. */
int rh_oracle_hydro_flag(const rh_mesh_desc* m, const rh_hydro_params* p, const rh_flag_params* f, int ilevel,
                         const double* uold, int* flag1, long long* nflag);

/* output_hydro's primitive variables (hydro/output_hydro.f90:86-140):
 * q(1:8,1:5,1:noct) float32 = (rho, u, v, w, p) of uold(1:8,1:5,1:noct). */
int rh_oracle_output_prims(const double* uold, long long noct, double gamma, float* q);

#ifdef __cplusplus
}
#endif
#endif
