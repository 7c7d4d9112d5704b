// rh_internal.h — host-side context of the library (not part of the ABI).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "ramses_hydro.h"
#include "rh_bulk.h"

namespace rh {

void set_error(const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);

#define RH_CUDA(call)                                         \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return ::rh::cuda_fail(e_, #call); \
  } while (0)

// Tile configuration of the pencil kernel (chosen by the autotuner).
struct TileCfg {
  int txo = 8, tyo = 8;  // XY tile in octs
  int minb = 1;          // CTAs per SM the kernel's registers are sized for
  int lz = 32;           // oct layers per pencil
};

// Pencil tables of one level (device + host copies).
struct LevelTables {
  bool built = false;
  bool complete = false;  // level covers its whole box (uniform level)
  // coarse-fine levels: interpolated ghost octs [gbase, gbase + nghost) of the
  // state arrays, prolonged from level l-1 before each Godunov step
  long long gbase = 0;
  int nghost = 0;
  std::vector<int> gsrc_oct;         // [nghost][7] level l-1 oct (0-based) of the 7 father-neighbourhood cells
  std::vector<unsigned char> gsrc_cf;  // [nghost][7] cell | flip bits (x,y,z momentum) << 3
  std::vector<int2> gfather;         // [nghost] father oct (0-based), father cell
  int* d_gsrc_oct = nullptr;
  unsigned char* d_gsrc_cf = nullptr;
  int nxo = 0, nyo = 0, nzo = 0;
  TileCfg cfg;
  int npencil = 0;
  std::vector<int4> phdr;
  std::vector<long long> poff;
  std::vector<int> ptab;             // host copy (coarse-fine levels only)
  long long ntab = 0;                // table entries on the device
  int4* d_phdr = nullptr;
  long long* d_poff = nullptr;
  int* d_ptab = nullptr;
  double* d_cfl_partial = nullptr;
};

struct Context {
  bool inited = false;
  TileCfg amr_cfg{8, 4, 2, 32};  // tiles of multi-level meshes (coarse-fine kernels)
  bool amr_cfg_set = false;     // amr_cfg chosen by rh_set_amr_tile (else by precision at rh_set_mesh)
  int table_builder = 1;        // coarse-fine tables: 1 on the device, 0 on the host
  int state_check = 0;          // rh_coarse_step checks every level after set_uold (rh_set_state_check)
  int deterministic = 0;        // FP64 coarse-fine update through face slots (rh_set_deterministic)
  double* d_gface = nullptr;    // [ghost octs of a level][24 faces][5] slots of that update
  size_t gface_elems = 0;
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  int precision = RH_PREC_FP64;
  int interpol_var = 0, interpol_type = 0;
  TileCfg cfg;
  // mesh (host copy of the description)
  bool have_mesh = false;
  int nsubgrid = 1, levelmin = 1, levelmax = 1, ngridmax = 0;
  int box_nx[3] = {1, 1, 1};
  int periodic[3] = {0, 0, 0};
  int bound_type[6] = {2, 2, 2, 2, 2, 2};
  double boxlen = 1.0;
  double gravity[3] = {0, 0, 0};
  std::vector<rh_oct> grid;
  std::vector<int> head, noct;
  std::vector<LevelTables> levels;
  // device state: FP64 -> ud[2] = [oct][5][8]; FP32-bulk -> uf[2] = records of rh_bulk.h, ud[2] their E view
  int cur = 0;
  double* ud[2] = {nullptr, nullptr};
  float* uf[2] = {nullptr, nullptr};
  long long nstate = 0;            // ngridmax + interpolated ghost octs of all levels
  uint8_t* d_refmask = nullptr;    // [nstate] refined-cell bits (ghosts: 0)
  int2* d_gfather = nullptr;       // [nstate - ngridmax] father of each ghost
  int2* d_father = nullptr;        // [ngridmax] father (oct, cell) of each oct, built by the first rh_upload
  std::vector<int2*> d_face;       // per level: [noct][6] cells across each face (rh_hydro_flag)
  int nlevels_used = 0;
  int* d_err = nullptr;
  unsigned* d_check = nullptr;    // [levelmax+1][3] state check results (rh_check.cu)
  int check_cap = 0;
  double* d_cfl = nullptr;        // [levelmax+1][5] reduced CFL values
  double* d_scratch = nullptr;    // standalone cmpdt partials
  double* h_cfl = nullptr;        // pinned: courant_fine values read back, 5 per level
  size_t h_cfl_elems = 0;
  // Every kernel that writes d_cfl bumps cfl_gen.  rh_coarse_step copies the
  // levels' values of the state it leaves to h_cfl_next on cfl_copy as soon
  // as they are final (before its restrictions end); the next call reads them
  // from there while cfl_next_gen still equals cfl_gen.
  unsigned long long cfl_gen = 0, cfl_next_gen = ~0ull;
  double* h_cfl_next = nullptr;   // pinned, 5 per level
  int cfl_next_l0 = -1, cfl_next_l1 = -1;
  cudaStream_t cfl_copy = nullptr;
  cudaEvent_t ev_cfl_copied = nullptr, ev_cfl_ready = nullptr;
  double* d_stage64 = nullptr;    // FP64 staging of FP32-bulk uploads / downloads
  size_t stage64_bytes = 0;
  size_t scratch_elems = 0;
  // lazy set_unew / fused CFL bookkeeping, per level
  std::vector<char> unew_pending;  // set_unew called, unew not yet materialised
  std::vector<char> unew_copied;   // set_unew copied uold into unew (multi-level meshes)
  std::vector<char> unew_written;  // godunov wrote unew for the whole level
  std::vector<char> cfl_on_unew;   // d_cfl[l] holds CFL values of unew
  std::vector<char> cfl_on_uold;   // d_cfl[l] holds CFL values of uold
  std::vector<double> cfl_keys;    // [levelmax+1][8]: parameters of each level's cached CFL values
  // timing of the last godunov launch (for the bench)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // rh_coarse_step prolongs every level's ghost octs ahead, on `side`; a level
  // whose flag is set waits for its event instead of prolonging in launch_level
  cudaStream_t side = nullptr;
  cudaEvent_t ev_side_start = nullptr;
  std::vector<cudaEvent_t> ev_prolong;
  std::vector<char> prolonged;
  // rh_coarse_step's levels run concurrently on the library stream and these
  cudaStream_t lev_stream[3] = {nullptr, nullptr, nullptr};
  std::vector<cudaEvent_t> ev_level;
  std::vector<cudaEvent_t> ev_gather;  // per level: its ghosts' gather into the coarser level done
  double* d_gface_all = nullptr;  // [ghost octs of the mesh][24][5], zeroed once per mesh
  uint8_t* d_cflskip = nullptr;   // [ngridmax, rounded up to 4] father cells of ghost octs (bit per cell)
  double* d_gcfl = nullptr;       // [gather blocks of all levels][5] CFL partials of the corrected cells
  // artificial diffusion (rh_diffusion.cu): oct coordinates -> oct index of
  // the level it was built for, and the corner divergences
  int* d_difmap = nullptr;
  int difmap_level = -1;
  double* d_div = nullptr;
  size_t div_elems = 0;
};

Context& ctx();

// coarse-fine levels (rh_amr.cu)
int build_amr_tables(int l, const TileCfg& cfg, long long gbase);
int upload_amr_tables(int l);
int prolong_ghosts(int l, double smallr, cudaStream_t st = nullptr);  // null: the library stream

// artificial diffusion, difmag > 0 (rh_diffusion.cu): adds cmpdiff's face
// fluxes of level l to unew after its pencils; a mesh of one complete level
// in FP64 only (diffusion_supported)
bool diffusion_supported(int l);
int diffuse_level(int l, double dt, double dx, double difmag, double smallr, const double* gravity);
void free_diffusion();
// coarse-fine levels built on the device (rh_amr_tables.cu): same tables as
// build_amr_tables; *d_gfather_out receives the level's ghost fathers (device)
int build_amr_tables_device(int l, const TileCfg& cfg, long long gbase, const rh_oct* d_grid, int2** d_gfather_out);
// complete levels (rh_tables.cu)
int build_complete_tables_device(int l, const TileCfg& cfg, LevelTables& T);

// device state check of every level (rh_check.cu): RH_EBADSTATE on a bad cell
int check_all_levels();

// A set of pencils of a level launched on its own (rh_hoststep.cu): device
// arrays of n pencil headers and table offsets into the oct table ptab (built
// for the level's tile shape, possibly another pencil depth), and n CFL
// partial slots.
struct PencilRange {
  const int4* phdr;
  const long long* poff;
  const int* ptab;
  double* partial;
  int n;
  cudaStream_t stream;  // stream of the launch (the library stream when null)
};
// A level step of rh_coarse_step's concurrent path: coarse-fine face
// contributions go to the all-level slot buffer (entry e's slots at
// (e - base) * 24), no per-level gather, launched on `stream`.
struct LevelSlots {
  double* gface;
  long long base;
  cudaStream_t stream;
  const uint8_t* cflskip;  // cells the fused CFL epilogue leaves out (null: none)
  bool defer_reduce;       // no partial reduction: the caller merges it with the gather's
};
// rh_upload.cu: rh_upload's restriction of a level into its parents, on stream st
int upload_on(int head_idx, int num_octs, int internal_energy, double smallr, cudaStream_t st);
// rh_api.cu: one Godunov step of level l (all pencils, or `range`'s), and the
// FP64 staging buffer of FP32-bulk transfers (grown on demand, kept).
int launch_level(int l, double gamma, double smallr, double smallc, double dt, double dx, double smax_cap,
                 int slope, int riemann, const double* g, bool fuse_cfl, bool accumulate = false,
                 const PencilRange* range = nullptr, const LevelSlots* slots = nullptr);
int stage64(long long noct, double** out);
int ensure_level_tables(int l);
TileCfg level_cfg(int l);  // tile of level l's launches (see rh_api.cu)
// rh_hoststep.cu: releases the overlapped host-step schedule (mesh change, finalize)
void free_host_schedule();
#ifdef __CUDACC__
__global__ void pack_bulk_kernel(const double* __restrict__ src, float* __restrict__ uf, double* __restrict__ ue,
                                 long long noct);
__global__ void unpack_bulk_kernel(double* __restrict__ dst, const float* __restrict__ uf,
                                   const double* __restrict__ ue, long long noct);
__global__ void reduce_partials_kernel(const double* __restrict__ partial, long long n, double dt0,
                                       double* __restrict__ out);
#endif

// restart / snapshot file images (rh_io.cu)
struct ImageSrc {
  const double* ud = nullptr;  // FP64: [oct][5][8]; FP32-bulk: the records' E view (rh_bulk.h)
  const float* uf = nullptr;   // FP32-bulk: the records' float view
  int bulk = 0;
  int levelmin = 1, levelmax = 1;
  std::vector<long long> oct0, noct;  // per level from levelmin: first oct (0-based) and count
  const rh_oct* grid = nullptr;       // oct records (amr file); nullptr: one row-major box level
  long long nxo = 1, nyo = 1, nzo = 1;
};
long long image_bytes(int kind, const ImageSrc& s);
int build_image(int kind, const ImageSrc& s, double gamma, const void** dimage, long long* nbytes);
int image_to_host(const void* dimage, long long nbytes, void* host_buf, long long cap);
void free_image_buffer();

}  // namespace rh
