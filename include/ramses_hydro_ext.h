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
int rh_get_tile(int* txo, int* tyo, int* minb, int* lz);
/* Compiled tile shapes of a precision mode; returns their count. */
int rh_list_tiles(int precision, int* txo, int* tyo, int* minb, int max);
/* Pencil count and oct-table size of a level's current tables. */
int rh_level_info(int ilevel, int* npencil, long long* table_entries);
/* Device pointers of the current uold / unew buffers (FP64: *_d is
 * [oct][5][8]; FP32-bulk: *_f is [oct][4][8] float, *_d is [oct][8] energy). */
int rh_state_ptrs(void** uold_d, void** uold_f, void** unew_d, void** unew_f);
/* Run nrep Godunov steps of a level with a fixed dt on the device and return
 * the average time per step from CUDA events on the library's stream. */
int rh_bench_godunov(int ilevel, int nrep, double gamma, double smallr, double smallc, double dt, double dx,
                     double courant, int slope, int riemann, float* ms_per_step);

/* CUDA-event timer on the library's stream: start, then stop returns the
 * elapsed milliseconds of everything queued in between. */
int rh_timer_start(void);
int rh_timer_stop(float* ms);

#ifdef __cplusplus
}
#endif
#endif /* RAMSES_HYDRO_EXT_H */
