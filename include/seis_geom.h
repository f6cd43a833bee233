/*
 * seis_geom.h -- per-shot acquisition geometry of the shot driver.
 *
 * The reference keeps these as members of its MPI driver class Inversion
 * (src/lsrtm/inversion.cpp); here they are plain functions over flat arrays,
 * evaluated in the same float/double arithmetic so that every index they
 * return is the reference's.  Conventions as in seis_fd.h: models [nx][nz]
 * (z contiguous), gathers [ntrace][nt] (time contiguous), coordinates in the
 * model's length unit, status 0 / negative.  Host-only: no device is used.
 */
#ifndef SEIS_GEOM_H
#define SEIS_GEOM_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Aperture of one shot (Inversion::getVel, inversion.cpp:552-571): from the
 * smaller of the source x and the smallest receiver x, minus lpad cells, to
 * the larger plus rpad cells.  *fx_sub = first x of the sub-grid,
 * *nx_sub = its number of columns. */
int seis_geom_aperture(float sx, const float *gx, int ng, float dx, int lpad, int rpad,
                       float *fx_sub, int *nx_sub);

/* Sub-grid of a model (Inversion::getVel, inversion.cpp:572-598): column ix of
 * the sub-grid is the model column under fx_sub + ix dx, clamped to the
 * model's second and second-to-last columns.  model [nx][nz] starting at x =
 * fx, sub [nx_sub][nz].  SEIS_ERR_ARG when a column falls outside the model
 * (the reference's check). */
int seis_geom_extract(const float *model, int nz, int nx, float fx, float dx, float fx_sub,
                      int nx_sub, float *sub);

/* The model column each sub-grid column copies in seis_geom_extract:
 * cols[nx_sub], non-decreasing. */
int seis_geom_extract_columns(int nx, float fx, float dx, float fx_sub, int nx_sub, int *cols);

/* Receiver depth index per sub-grid column (Inversion::getIgz,
 * inversion.cpp:600-625): 0 where no receiver lies, else the depth sample
 * of the (last) receiver in the column.  nz = model depth samples (range
 * check). */
int seis_geom_receiver_rows(const float *gx, const float *gz, int ng, float fx_sub, int nx_sub,
                            float dx, float dz, int nz, int *igz);

/* Source sample indices in the sub-grid (inversion.cpp:428-429, :519-520). */
int seis_geom_source_index(float sx, float sz, float fx_sub, float dx, float dz, int *isx,
                           int *isz);

/* Traces <-> sub-grid columns (Inversion::swapReord, inversion.cpp:626-643).
 * to_gather = 0: rec[nx][nt] = 0, then the column under each receiver gets
 * its trace csg[ig]; to_gather = 1: csg[ng][nt] = 0, then each trace gets the
 * column under its receiver. */
int seis_geom_reorder(float *csg, int ng, int nt, const float *gx, float *rec, float fx, int nx,
                      float dx, int to_gather);

/* Sub-grid image into the global grid (Inversion::swapModel,
 * inversion.cpp:644-665), with the reference's mapping: global column ix
 * (4 <= ix < nxd - 4) takes the sub column under dfx + (ix - 1) dx, when that
 * column is 4 .. nxm - 4; rows 4 .. nzd - 5; d cleared first unless add. */
int seis_geom_swap_model(const float *m, float *d, float mfx, float dfx, int nzm, int nxm, int nzd,
                         int nxd, float dx, int add);

/* Direct-arrival mute (Inversion::removeDirect, inversion.cpp:699-752): each
 * trace is zeroed up to the horizontal travel time from the source column at
 * the receiver depth plus the delays, at least 1 and at most nt - 1 samples.
 * v [nx][nz] is the global model starting at x = velfx. */
int seis_geom_remove_direct(float *csg, int ng, int nt, const float *gx, const float *gz, float sx,
                            float sz, const float *v, int nz, int nx, float dx, float dz, float dt,
                            float fr, float velfx, int delay);

#ifdef __cplusplus
}
#endif
#endif
