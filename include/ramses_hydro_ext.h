/*
 * ramses_hydro_ext.h — library extensions beside the drop-in ABI.
 *
 * These entry points have no counterpart in the reference: they expose the
 * B200 kernel's tile configuration (for the autotuner), device pointers of the
 * resident state (zero-copy views for hosts that share the CUDA context), and
 * an on-device timing loop used by the benchmark.
 */
#ifndef RAMSES_HYDRO_EXT_H
#define RAMSES_HYDRO_EXT_H

#include "ramses_hydro.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Pencil tile of the Godunov kernel: txo x tyo octs in x,y, registers sized
 * for minb CTAs per SM, lz oct layers per pencil.  Only compiled shapes are
 * accepted (rh_list_tiles). */
int rh_set_tile(int txo, int tyo, int minb, int lz);
/* Tile of the coarse-fine (multi-level) kernels; before rh_set_mesh, since a
 * mesh's interpolated ghost octs follow its pencils.  Default (the fastest on
 * the AMR Sedov of levels 7-10): 7x7 octs, 2 CTAs/SM, 32 layers for FP32-bulk;
 * 8x4, 2 CTAs/SM, 32 layers for FP64.  rh_set_mesh gives a partial level
 * fewer layers (halved, down to 2) until its pencils fill a wave of CTAs. */
int rh_set_amr_tile(int txo, int tyo, int minb, int lz);
int rh_get_tile(int* txo, int* tyo, int* minb, int* lz);
/* Compiled tile shapes of a precision mode; returns their count. */
int rh_list_tiles(int precision, int* txo, int* tyo, int* minb, int max);
/* Pencil count and oct-table size of a level's current tables. */
int rh_level_info(int ilevel, int* npencil, long long* table_entries);
/* Copy a level's pencil headers (npencil x int4: ox0, oy0, oz0, layers),
 * table offsets (npencil) and oct table (entries: 0-based oct index per
 * (pencil, layer row, oct column), boundary-resolved) to the host. */
int rh_level_table(int ilevel, int* phdr, long long* poff, int* tab, long long max_entries);
/* Interpolated ghost octs of a coarse-fine level: per ghost the 7 level l-1
 * source octs (0-based; father cell first, then -x,+x,-y,+y,-z,+z) with their
 * cell | reflexive-flip bits << 3, and the father (oct, cell); returns the
 * ghost count (arrays may be null to query it), negative on error. */
int rh_level_ghosts(int ilevel, int* gsrc_oct, unsigned char* gsrc_cf, int* gfather, long long max_ghosts);
/* One coarse step of the whole mesh with one time step for every level
 * (nsubcycle = 1), making the calls amr_step.f90 makes in their order:
 * rh_cmpdt of every level, dt = min over levels of min(dx_l/smallc, cell dt)
 * (unless *dt > 0 on entry, which is then used), rh_set_unew of every level,
 * then from the finest level to the coarsest rh_godunov, rh_set_uold and,
 * below the finest level, rh_upload of the level above.  dx_l = boxlen/2^l.
 * *dt receives the time step taken; cfl (optional, 5 per level from levelmin)
 * the courant_fine values of each level.  The same results as the separate
 * calls, without a host round trip per call (the reference's host makes them
 * one by one; this is for hosts that step whole meshes).  When the levels
 * hold every oct of the state, the levels' steps run at once on separate
 * streams (each writes its own cells of unew from uold, so no set_unew copy
 * is needed), every level's ghost octs are prolonged ahead, the coarse-fine
 * corrections are added to the father cells after all steps in a fixed order
 * (results repeat bit for bit), set_uold is one swap of the two state
 * buffers and the restrictions follow, finest first: no Godunov step reads a
 * level that an earlier set_uold or restriction of the step would have
 * changed.  There the step also leaves every level's courant_fine values of
 * the new state (the pencils' fused epilogue for the cells they finish, the
 * correcting gather for the father cells), so the next call's rh_cmpdt of
 * every level reads five numbers instead of the state.
 * p->difmag > 0 adds unsplit's artificial diffusion (cmpdivu / cmpdiff,
 * hydro/umuscl.f90:2392-2540) to the step of a mesh of one complete level in
 * FP64; other meshes and FP32-bulk return RH_EINVAL with difmag > 0.  The
 * leaf call rh_godunov, like mtl_godunov, takes no difmag. */
int rh_coarse_step(const rh_hydro_params* p, double* dt, double* cfl);

/* Coarse-fine update of the father cells (unew of level l-1 += or -= the
 * flux/8 of every face between a cell of level l and an interpolated ghost,
 * hydro/godunov_fine.f90:893-1052) in the level-by-level calls (rh_godunov)
 * and in rh_coarse_step on meshes with spare octs; rh_coarse_step on a mesh
 * whose levels hold every oct always sums them in a fixed order.  0 (the
 * default): atomic adds from the pencil kernels, whose order between pencils
 * varies from run to run.
 * 1: each face's contribution goes to its own slot and one thread per father
 * cell adds its 24 slots in a fixed order after the level's kernel (the role
 * of the reference's fixed-order flush of cache octs, godunov_fine.f90:
 * 1347-1459), so AMR runs repeat bit for bit; it costs a zeroed buffer of
 * 960 bytes per ghost oct and one more small kernel per level step.  Both
 * precision modes (FP32-bulk: the slot sums are added to the float records
 * and the FP64 energy in FP64). */
int rh_set_deterministic(int on);

/* One coarse step of a mesh whose uold lives in host memory: host_in (the
 * reference layout uold(1:8,1:5,1:ngridmax)) is copied to the device, stepped
 * as rh_coarse_step steps it, and the new state is written to host_out (may
 * be host_in).  No counterpart in the reference, whose GPU runner keeps uold
 * on the device between steps; this is for hosts that hand over their state
 * every step.  On a single-level mesh the two copies and the Godunov pencils
 * overlap chunk by chunk (a pencil runs once its neighbourhood has arrived, a
 * chunk is read back once the pencils writing it are done), with the new
 * state and dt_next bitwise those of rh_set_grid_device + rh_coarse_step +
 * rh_transfer_grid_host (the cached conserved totals to rounding); other
 * meshes make those three calls.  *dt > 0 on entry is the step's dt
 * (else courant_fine of host_in, after the whole upload); *dt receives the dt
 * taken and *dt_next (optional) min(dx/smallc, courant dt) of the new state,
 * from the step's fused CFL epilogue: a host that loops passes it back as the
 * next call's dt, which lets the upload overlap the pencils.  Host buffers
 * should be pinned (cudaHostAlloc) for the copies to overlap. */
int rh_coarse_step_host(const rh_hydro_params* p, const double* host_in, double* host_out, double* dt,
                        double* dt_next);

/* Device state check of one level's current uold, the reference's debug scan
 * after set_uold (check_nan_kernel, gpu/gpu_utils.cuf:90-118, called by
 * gpu_check_nan, gpu/gpu_runner.cuf:5316-5391) extended by cmpdt's
 * negative-pressure stop (hydro/godunov_utils.f90:278-287).  Every cell of
 * octs head_idx .. head_idx+num_octs-1 (1-based) is tested; *nbad receives
 * the number of bad cells, *first_oct the smallest bad oct index (1-based,
 * 0 when none) and *mask the OR of: 1 NaN or Inf in a conserved variable,
 * 2 density <= 0, 4 internal energy E - |rho u|^2/(2 rho) <= 0 at positive
 * density.  Where the reference prints the oct and stops the run, the host
 * decides.  Synchronous. */
int rh_check_state(int head_idx, int num_octs, int* nbad, int* first_oct, int* mask);
/* on != 0: rh_coarse_step runs that check on every level after the step
 * (the reference's gpu_debug switch) and returns RH_EBADSTATE, the level,
 * count, first oct and mask in rh_last_error(), when a cell is bad.  Off by
 * default (one extra read of the state per coarse step). */
int rh_set_state_check(int on);
/* Where rh_set_mesh builds coarse-fine tables: 1 on the device (default),
 * 0 on the host (the reference builder the device one is tested against). */
int rh_set_table_builder(int on_device);
/* Device pointers of the current uold / unew buffers (FP64: *_d is
 * [oct][5][8]; FP32-bulk: one 192-byte record per oct, 32 floats (rho, rho u,
 * rho v, rho w of the 8 cells) then 8 doubles (E); *_f points at the first
 * record, *_d at the first record's E, strides 48 floats / 24 doubles). */
int rh_state_ptrs(void** uold_d, void** uold_f, void** unew_d, void** unew_f);
/* Run nrep Godunov steps of a level with a fixed dt on the device and return
 * the average time per step from CUDA events on the library's stream. */
int rh_bench_godunov(int ilevel, int nrep, double gamma, double smallr, double smallc, double dt, double dx,
                     double courant, int slope, int riemann, float* ms_per_step);

/* CUDA-event timer on the library's stream: start, then stop returns the
 * elapsed milliseconds of everything queued in between. */
int rh_timer_start(void);
int rh_timer_stop(float* ms);

/* ---- for callers that cannot allocate -------------------------------------
 * rh_cmpdt_noalloc has no counterpart in the reference (RAMSES II's
 * gpu_cmpdt_2 borrows scratch from a device array it owns).  It serves hosts
 * that must not let a library call cudaMalloc/cudaFree: solvers whose own
 * memory manager hands out all device memory under a fixed budget, and tight
 * loops that cannot afford the device-wide synchronisation an allocation
 * implies.
 *
 * courant_fine over a caller-owned FP64 state, allocating nothing:
 * d_uold    device pointer to num_octs oct records in the reference layout
 *           uold(1:8,1:5,1:num_octs) (320 bytes per oct);
 * d_refined optional device pointer to num_octs*8 bytes, nonzero = refined
 *           cell (skipped); NULL treats every cell as a leaf;
 * d_out     device pointer to 5 doubles: mass, ekin (sum of E*vol, as the
 *           reference names it), eint, emag (0), dt = min(dx/smallc, cell dt);
 * stream    cudaStream_t to run on (NULL: the legacy default stream).
 * Limit: num_octs <= 2,097,152 (one 256^3-cell level); larger sizes return
 * RH_EINVAL without touching the GPU.  The per-block partials live in one
 * file-scope device array of 2.6 MB that every GPU loading the library keeps
 * until process exit; each block overwrites its own slot, so nothing needs
 * clearing, and every call reuses the same array: calls that overlap on the
 * GPU (different streams, or host threads sharing a device) race.  The first
 * call on a device looks up the array's device address (cudaGetSymbolAddress)
 * and caches it; make that first call before any stream capture.  Every later
 * call made outside capture looks the address up again; a call on a stream
 * being captured uses the cached one, so after a device reset make one call
 * outside capture before capturing again.  Under CUDA's lazy module loading
 * (the default since CUDA 12.2) the array's 2.6 MB are reserved on the device
 * when that first call runs: a host whose memory manager reserves the whole
 * device budget makes the first call before that reservation.
 * Asynchronous: read d_out after synchronising the stream. */
int rh_cmpdt_noalloc(const double* d_uold, int num_octs, const unsigned char* d_refined, double dx,
                     double gamma, double smallr, double smallc, double courant_factor,
                     const double* constant_gravity, double* d_out, void* stream);

/* Runs the pencil kernels' bounded mbarrier wait on a barrier nothing arrives
 * on (bound polls, at most 2^20): returns RH_ETIMEDOUT through the same error
 * word rh_sync reads, with the context still usable.  For tests of the
 * failure path; faults, traps and hangs are never used. */
int rh_selftest_wait(long long bound);
/* For tests of the pencil kernels' FP64 lane arithmetic: for n device doubles
 * x, writes d_out[0:n] = the kernels' reciprocal (vrcp), d_out[n:2n] = their
 * square root (vsqrt), d_out[2n:3n] = CUDA's 1.0/x and d_out[3n:4n] = CUDA's
 * sqrt(x).  Synchronous. */
int rh_selftest_vmath(const double* d_x, long long n, double* d_out);

#ifdef __cplusplus
}
#endif
#endif /* RAMSES_HYDRO_EXT_H */
