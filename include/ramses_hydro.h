/*
 * ramses_hydro.h — C ABI of the B200-native RAMSES II Godunov hydro step.
 *
 * This is the drop-in boundary for RAMSES II's hydro leaf calls.  The Fortran
 * host reaches it through an iso_c_binding interface module; every entry
 * point takes plain pointers, sizes and scalars, returns 0 on success and a
 * nonzero RH_E* code on failure (message in rh_last_error()).  The reference
 * aborts on errors (GPU_Error_Check, gpu/gpu_utils.cuf:59-79; error stop in
 * gpu/gpu_runner.cuf:969,993); the Fortran shim turns a nonzero code into
 * mdl_abort.
 *
 * The library keeps one context per process (one device, one stream, one
 * resident mesh), as the reference drives its GPU from one host thread per
 * MPI rank; calls from several host threads at once are not supported.
 *
 * Host arrays keep the reference layout: uold(1:8,1:nvar,1:ngridmax) column
 * major (hydro/amr_commons.f90 mesh_t, amr/amr_commons.f90:811-920), i.e. oct
 * igrid occupies 8*nvar consecutive doubles at offset (igrid-1)*8*nvar, and
 * type(oct) records (amr/oct_commons.f90:5-10) are 32 bytes each.  Oct and
 * subgrid indices are 1-based as in Fortran.
 */
#ifndef RAMSES_HYDRO_H
#define RAMSES_HYDRO_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define RH_OK          0
#define RH_EINVAL      1   /* bad argument / unsupported option            */
#define RH_ENOMEM      2   /* device allocation failed or budget exceeded  */
#define RH_ECUDA       3   /* CUDA runtime error                           */
#define RH_ESTATE      4   /* call out of order (no mesh, no level table)  */
#define RH_ETIMEDOUT   5   /* bounded device wait gave up                  */
#define RH_ENODEV      6   /* no CUDA device / extension not built          */
#define RH_EBUSY       7   /* serving queue full                           */
#define RH_EBADSTATE   8   /* state check found NaN/Inf, rho<=0 or eint<=0 */

/* Riemann solver ids: hydro/hydro_parameters.f90:30-32 */
#define RH_RIEMANN_LLF  1
#define RH_RIEMANN_HLL  2
#define RH_RIEMANN_HLLC 3

/* Boundary types: amr/boundaries.f90:39-519 (init_bound_refine) */
#define RH_BOUND_PERIODIC     0
#define RH_BOUND_REFLEXIVE    1
#define RH_BOUND_ZERO_GRADIENT 2

/* Precision modes */
#define RH_PREC_FP64       0   /* plain FP64: matches the FP64 CPU path          */
#define RH_PREC_FP32_BULK  1   /* FP32 stencil/flux math; FP64 energy, pressure
                                  recovery, conserved sums and CFL dt           */

/* type(oct), amr/oct_commons.f90:5-10 with NDIM=3, nhilbert=1 (32 bytes). */
typedef struct rh_oct {
    int64_t hkey;
    int32_t ckey[3];
    uint8_t refined[8];
    int32_t lev;
} rh_oct;

/* Hydro subset of hydro_params_t, amr/amr_commons.f90:690-702, filled as
 * set_hydro_parameters does (amr/amr_commons.f90:932-952). */
typedef struct rh_hydro_params {
    double gamma;
    double smallr;
    double smallc;
    double courant_factor;
    double difmag;          /* > 0: cmpdivu/cmpdiff (umuscl.f90:2392-2540), rh_coarse_step on one FP64 level */
    int32_t slope_type;     /* 0 none, 1 minmod, 2 moncen, 3 multi-d positivity  */
    int32_t riemann;        /* RH_RIEMANN_*                                      */
    int32_t interpol_var;   /* 0: rho, rho u, E   1: rho, rho u, rho e           */
    int32_t interpol_type;  /* 0 injection, 1 minmod, 2 MC, 3 central            */
} rh_hydro_params;

/* Mesh description in the reference's flat-oct form. */
typedef struct rh_mesh_desc {
    int32_t nsubgrid;          /* octs per block edge (amr_parameters nsubgrid)   */
    int32_t levelmin, levelmax;
    int32_t ngridmax;          /* capacity of uold/grid in octs                   */
    int32_t box_nx[3];         /* domain size in level-1 octs (1,1,1: unit box)   */
    int32_t periodic[3];
    int32_t bound_type[6];     /* x-,x+,y-,y+,z-,z+: RH_BOUND_*                  */
    double  boxlen;
    double  constant_gravity[3];
    const int32_t* head;       /* head[l]: 1-based first oct of level l, l=0..levelmax */
    const int32_t* noct;       /* noct[l]: number of octs of level l                  */
    const rh_oct*  grid;       /* grid[igrid-1]                                       */
} rh_mesh_desc;

/* ---- library / device --------------------------------------------------- */

/* Select the CUDA device and create the library's stream. */
int rh_init(int device_ordinal);
/* Release every device buffer the library holds. */
int rh_finalize(void);
/* Message of the last failing call on this thread ("" if none). */
const char* rh_last_error(void);
/* Wait for all work queued by the library. */
int rh_sync(void);
/* Choose RH_PREC_FP64 (default) or RH_PREC_FP32_BULK; call before rh_set_mesh. */
int rh_set_precision(int mode);

/* ---- mesh set-up (replaces r_set_grid_device / gpu_build_level_cache) ---- */

/* Copy the mesh description (grid records, level ranges, box, boundaries)
 * and uold to the device.  Replaces r_set_grid_device
 * (gpu/gpu_manager.cuf:12-162) and mtl_set_grid_device
 * (metal/metal_interface.f90:46-55).  uold is uold(1:8,1:nvar,1:ngridmax). */
int rh_set_mesh(const rh_mesh_desc* mesh, const double* uold, int nvar, int twotondim);

/* Re-upload uold only (mesh unchanged). */
int rh_set_grid_device(const double* uold, int ngridmax, int nvar, int twotondim);

/* Copy the device uold back to the host before output.  Replaces
 * r_transfer_grid_host / mtl_transfer_grid_host (metal_interface.f90:67-74). */
int rh_transfer_grid_host(double* uold, int ngridmax, int nvar, int twotondim);

/* ---- hydro leaf calls ------------------------------------------------------ */

/* unew = uold for the octs of a level.  Replaces gpu_set_unew
 * (gpu/gpu_runner.cuf:477-498) / mtl_set_unew (metal_interface.f90:86-90).
 * head_idx is the 1-based first oct, num_octs the level's oct count. */
int rh_set_unew(int head_idx, int num_octs);

/* uold = unew for the octs of a level.  Replaces gpu_set_uold
 * (gpu/gpu_runner.cuf:447-468) / mtl_set_uold (metal_interface.f90:93-97). */
int rh_set_uold(int head_idx, int num_octs);

/* CFL time step and conserved totals over the leaf cells of a level.
 * Replaces gpu_cmpdt_2 (gpu/gpu_runner.cuf:281-438) and mtl_cmpdt
 * (metal_interface.f90:101-116); returns synchronously like both.
 * dt returns min(courant_factor*dx/smallc, min over leaf cells of cmpdt). */
int rh_cmpdt(int head_idx, int num_octs, double dx, double gamma, double smallr,
             double smallc, double courant_factor, const double* constant_gravity,
             double* mass, double* ekin, double* eint, double* emag, double* dt);

/* One MUSCL-Hancock Godunov step of a level: unew += fluxes (and, above
 * levelmin, the coarse-cell corrections into level ilevel-1).  Replaces
 * gpu_godunov (gpu/gpu_runner.cuf:862-1016) and mtl_godunov
 * (metal_interface.f90:537-558).  head_idx/num_subgrids count blocks of
 * nsubgrid^3 octs, 1-based, as gpu_godunov does.  Asynchronous. */
int rh_godunov(int head_idx, int num_subgrids, int ngridmax, int ilevel,
               int levelmin, int levelmax, double gamma, double smallr,
               double smallc2, double dt, double dx, double smax_cap,
               int slope, int riemann, const double* constant_gravity);

/* Restriction: the refined cells of level ilevel take the average of their
 * child octs, head_idx/num_octs being level ilevel+1's octs (1-based), with
 * internal energy averaged instead of total energy when internal_energy != 0
 * (interpol_var == 1).  Replaces gpu_upload (gpu/gpu_runner.cuf:1754-1784) and
 * mtl_upload (metal/metal_runner.f90:814-837), i.e. upload_fine
 * (hydro/upload.f90:74-271); called after rh_set_uold of level ilevel
 * (amr/amr_step.f90:479-483).  Asynchronous. */
int rh_upload(int head_idx, int num_octs, int internal_energy, double gamma,
              double smallr, double smallc2);

/* Gradient refinement criteria of hydro_refine (hydro/godunov_utils.f90:
 * 6-223): a criterion is off when its err_grad is negative. */
typedef struct rh_flag_params {
    double err_grad_d, err_grad_p, err_grad_u;
    double floor_d, floor_p, floor_u;
} rh_flag_params;

/* Refinement flags of the cells of level ilevel by the gradient criteria:
 * every cell is compared with its six neighbours at the same level (or, where
 * a neighbour oct does not exist, with that neighbour's parent cell); flag1 is
 * the host's (1:8, 1:ngridmax) int32 array: flagged cells get 1 (others keep
 * their value) and *nflag returns how many were newly flagged.  Replaces the
 * gradient branch of hydro_flag (hydro/hydro_flag.f90:7-159); the reference's
 * GPU flagging kernel is hydro_flag_kernel (gpu/gpu_hydro.cuf:6690).
 * Synchronous (the flags are on the host on return). */
int rh_hydro_flag(int ilevel, const rh_flag_params* f, double gamma, double smallr,
                  int32_t* flag1, long long* nflag);

/* Extra hydro parameters the reference passes through hydro_params_t but
 * mtl_godunov does not carry (interpolation scheme for coarse-fine ghosts). */
int rh_set_interpolation(int interpol_var, int interpol_type);

#ifdef __cplusplus
}
#endif
#endif /* RAMSES_HYDRO_H */
