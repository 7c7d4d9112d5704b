/*
 * ramses_hydro_io.h — restart (backup) and snapshot (output) files of the
 * hydro state, byte for byte in the reference's layouts, assembled in device
 * memory from the resident state.
 *
 * All files are stream-access (no record markers), native little-endian, one
 * file per rank (this library is one rank: file number 00001).
 *
 *   RH_FILE_AMR           backup_amr (amr/output_amr.f90:666-735) and output_amr
 *                         (amr/output_amr.f90:607-660, header of
 *                         amr/ramses_commons.f90:138-158) share one layout:
 *                         int32 ndim, levelmin, nlevelmax, noct(levelmin:nlevelmax),
 *                         then per level, per oct: int32 ckey(1:ndim),
 *                         int32 refined bits (bit ind-1 = cell ind refined).
 *   RH_FILE_HYDRO_BACKUP  backup_hydro (hydro/output_hydro.f90:167-246):
 *                         int32 ndim, nvar, levelmin, nlevelmax, noct(...),
 *                         then per level, per oct: float64 uold(1:8,1:nvar).
 *   RH_FILE_HYDRO_OUTPUT  output_hydro (hydro/output_hydro.f90:40-162):
 *                         the same header, then per level, per oct:
 *                         float32 q(1:8,1:nprim), q = (rho, u, v, w, p) computed
 *                         from uold as the reference does (output_hydro.f90:86-140).
 *
 * Octs of a level are written in the mesh's order (head(l) .. tail(l)), levels
 * from levelmin to levelmax of the mesh.  The restart reader
 * (amr/init_refine_restart.f90:384-396) finds a level's first oct at
 * 13 + 4*nlevel + (4*ndim+4)*nskip (amr) and 17 + 4*nlevel + 8*8*nvar*nskip
 * (hydro), 1-based, nskip = octs of the lower levels of the file.
 */
#ifndef RAMSES_HYDRO_IO_H
#define RAMSES_HYDRO_IO_H

#include "ramses_hydro.h"

#ifdef __cplusplus
extern "C" {
#endif

#define RH_FILE_AMR           1
#define RH_FILE_HYDRO_BACKUP  2
#define RH_FILE_HYDRO_OUTPUT  3

/* Bytes of the file image of the current mesh. */
int rh_file_size(int kind, long long* nbytes);

/* Image of the current state (uold) in host_buf (cap bytes); *nbytes receives
 * its size.  gamma is used by RH_FILE_HYDRO_OUTPUT only (the pressure,
 * output_hydro.f90:128).  Replaces the per-oct loops of output_hydro /
 * backup_hydro / output_amr / backup_amr for the rank's octs; the caller
 * writes the bytes to its file. */
int rh_file_image(int kind, double gamma, void* host_buf, long long cap, long long* nbytes);

/* The same image left in library-owned device memory (*dimage), valid until
 * the next image call, rh_set_mesh or rh_finalize.  The image is complete when
 * the call returns. */
int rh_file_image_device(int kind, double gamma, const void** dimage, long long* nbytes);

/* Restart: load uold from an RH_FILE_HYDRO_BACKUP image whose header matches
 * the mesh (ndim 3, nvar 5, levelmin, levelmax and noct of every level), as
 * init_refine_restart reads the hydro file (amr/init_refine_restart.f90:389-396).
 * In FP32-bulk precision rho and momentum are rounded to float32 as rh_set_mesh does. */
int rh_restore_hydro(const void* image, long long nbytes);

/* Image of one batch problem (include/ramses_hydro_batch.h): a single level 1
 * of n[0]/2 x n[1]/2 x n[2]/2 octs in row-major order (ckey = oct coordinates,
 * no refined cells), gamma of the problem. */
int rh_batch_file_image(int id, int kind, void* host_buf, long long cap, long long* nbytes);

#ifdef __cplusplus
}
#endif
#endif /* RAMSES_HYDRO_IO_H */
