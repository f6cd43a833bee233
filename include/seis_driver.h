/*
 * seis_driver.h -- the shot driver: the reference's parameter file,
 * coordinate file and per-shot gather files driving the batched engine.
 *
 * Replaces the reference's MPI driver class Inversion (src/lsrtm/inversion.h,
 * inversion.cpp): readParamFile (:38-88), getConfig (:89-140),
 * modeling_MPI (:141-206), forward_MPI (:475-551), adjoint_MPI (:365-474) and
 * the conjugate-gradient solver it declares but never defines
 * (conope_MPI / cgsolver_MPI, inversion.h:81,87).  The MPI master/worker shot
 * farm becomes in-process batches of shots on one device; files keep the
 * reference's names and raw float32 layouts.  Status 0 / negative as in
 * seis_fd.h.
 */
#ifndef SEIS_DRIVER_H
#define SEIS_DRIVER_H
#include <stddef.h>

#include "seis_fd.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Parameter file (Inversion::readParamFile, inversion.cpp:38-88, read with
 * ParserFromFile semantics, src/util/parser.cpp:15-175): for each key, the
 * first line (after stripping from '!') containing "key " with a value token
 * after it.  Optional keys take the reference defaults (paramLSRTM,
 * src/lsrtm/datastr.h). */
typedef struct {
  int nthread, ns, ngmax, nx, nz, nt, npml, delay, delaycal, mask, maxiter, lpad, rpad, planeTag,
      sbegin, send;
  float dx, dz, dt, fr, velfx;
  int np;
  float dp, pmin;
  char precsg[256], wdir[256], v0file[256], vfile[256], coordfile[256], maskfile[256];
} seis_params;

int seis_params_read(const char *file, seis_params *out, char *err, size_t err_len);

/* Coordinate file (Coords, src/util/coord.cpp:22-175): one line per trace,
 * "source_x source_z receiver_x receiver_z"; a new shot starts where the source
 * x changes.  Counting follows the reference (a trailing newline is expected). */
int seis_coords_count(const char *file, int *ns);
/* ng[ns]; sc[ns][2] (x, z); gc[ns][2][ngmax] (x row, then z row), filled
 * with -1e10 past each shot's receivers. */
int seis_coords_read(const char *file, int ns, int ngmax, int *ng, float *sc, float *gc);

/* ------------------------------------------------------------- the driver */
typedef struct seis_driver seis_driver;

/* Reads the parameter and coordinate files; batch = shots per device batch
 * (0: all).  ctx may be NULL for the host-only steps (plane-wave preparation). */
int seis_driver_create(seis_fd_ctx *ctx, const char *param_file, int batch, seis_driver **out);
int seis_driver_destroy(seis_driver *d);
const seis_params *seis_driver_params(const seis_driver *d);

/* modeling_MPI (inversion.cpp:141-206): per shot the aperture sub-grid of
 * h_v [nx][nz] (NULL: read vfile), modeling, traces from the columns, direct
 * mute, written to precsg<is>.dat ([ng][nt] float32).  Exact-rounding
 * kernels: the files match the reference's. */
int seis_driver_modeling(seis_driver *d, const float *h_v);

/* forward_MPI (inversion.cpp:475-551): Born gathers of h_dv [nx][nz] over the
 * v0file background, written to wdir BORN<is>.dat. */
int seis_driver_born(seis_driver *d, const float *h_dv);

/* adjoint_MPI (inversion.cpp:365-474): reference RTM of shots sbegin..send
 * from precsg<is>.dat (born_data = 0) or wdir BORN<is>.dat (1) over the v0file
 * background; each shot's image goes through swapModel (and the mask file when
 * mask = 1), is written to wdir CSG_IMAGE<is>.dat and summed into h_img
 * [nx][nz]. */
int seis_driver_rtm(seis_driver *d, int born_data, float *h_img);

/* illum_MPI (inversion.cpp:207-290): source illumination of every shot over
 * the v0file background, through swapModel into the global grid, written to
 * wdir ILLUM<is>.dat and summed into h_ss [nx][nz]. */
int seis_driver_illum(seis_driver *d, float *h_ss);

/* planeWavePrepare (inversion.cpp:808-912): for each of the np wavenumbers
 * p = pmin + k dp, the phase-encoded areal source (every shot's wavelet
 * rotated by p times its x through the 201-tap Hilbert filter, harmonic,
 * InitInversion.cpp:141-150, added at its column) and the phase-encoded data
 * (every trace of every precsg<is>.dat likewise, moved to its model column and
 * summed), written to wdir PLANE_S_NEW<k>.dat ([nx][nt+delaycal]) and
 * PLANE_R_NEW<k>.dat ([nx][nt]).  Requires planeTag. */
int seis_driver_plane_prepare(seis_driver *d);

/* adjointPlane_MPI (inversion.cpp:1019-1103): for each wavenumber k < np,
 * plane-wave RTM of PLANE_S_NEW<k>.dat with PLANE_R_NEW<k>.dat (born_data = 0)
 * or BORN<k>.dat (1) over the whole v0file model, source row from shot 0's
 * depth and receiver row from its first receiver's; each image (times the mask
 * when mask = 1) written to wdir IMAGE<k>.dat and summed into h_img [nx][nz]. */
int seis_driver_rtm_plane(seis_driver *d, int born_data, float *h_img);

/* illumPlane_MPI (inversion.cpp:291-345): for each wavenumber k < np, the
 * illumination of PLANE_S_NEW<k>.dat over the whole v0file model (source row
 * from shot 0's depth), written to wdir ILLUM_PLANE<k>.dat ([nx][nz]); h_ss
 * (may be NULL) receives their sum. */
int seis_driver_illum_plane(seis_driver *d, float *h_ss);

/* Least-squares RTM by CGLS over all shots: L = Born on each aperture
 * sub-grid, L^T its exact adjoint scattered back through the transpose of the
 * sub-grid extraction; observed data from precsg<is>.dat or BORN<is>.dat
 * (born_data), direct-muted and reordered as in adjoint_MPI.  niter
 * iterations; h_img [nx][nz] = model, h_rr[0..niter] = |d|^2 then |r|^2 per
 * iteration (h_rr may be NULL). */
int seis_driver_lsrtm(seis_driver *d, int born_data, int niter, const seis_lsrtm_opts *opts,
                      float *h_img, double *h_rr);

#ifdef __cplusplus
}
#endif
#endif
