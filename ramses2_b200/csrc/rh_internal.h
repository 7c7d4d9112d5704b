// rh_internal.h — host-side context of the library (not part of the ABI).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "ramses_hydro.h"

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
  int nxo = 0, nyo = 0, nzo = 0;
  TileCfg cfg;
  int npencil = 0;
  std::vector<int4> phdr;
  std::vector<long long> poff;
  std::vector<int> ptab;
  int4* d_phdr = nullptr;
  long long* d_poff = nullptr;
  int* d_ptab = nullptr;
  double* d_cfl_partial = nullptr;
};

struct Context {
  bool inited = false;
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
  // device state: FP64 -> ud[2] = [oct][5][8]; FP32-bulk -> uf[2] = [oct][4][8], ud[2] = [oct][8]
  int cur = 0;
  double* ud[2] = {nullptr, nullptr};
  float* uf[2] = {nullptr, nullptr};
  int* d_err = nullptr;
  double* d_cfl = nullptr;        // [levelmax+1][5] reduced CFL values
  double* d_scratch = nullptr;    // standalone cmpdt partials
  size_t scratch_elems = 0;
  // lazy set_unew / fused CFL bookkeeping, per level
  std::vector<char> unew_pending;  // set_unew called, unew not yet materialised
  std::vector<char> unew_written;  // godunov wrote unew for the whole level
  std::vector<char> cfl_on_unew;   // d_cfl[l] holds CFL values of unew
  std::vector<char> cfl_on_uold;   // d_cfl[l] holds CFL values of uold
  double cfl_key[8] = {0};         // parameters the cached CFL values were computed with
  // timing of the last godunov launch (for the bench)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

Context& ctx();

}  // namespace rh
