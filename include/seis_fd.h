/*
 * seis_fd.h -- C ABI of the B200 2-D acoustic finite-difference engine.
 *
 * Drop-in replacement for the reference's CPU propagators (src/util/fd.h:3-16,
 * bbsun/Seis) and for its MPI shot farm (src/lsrtm/inversion.cpp:141-551,
 * :753-807), running on one NVIDIA B200 (sm_100a).
 *
 * Conventions (all from the reference):
 *  - Models and images are [nx][nz] float, z fastest (MyAlloc<float>::alc(nz,nx),
 *    src/util/memory.h:29-44).  Gathers are [nx][nt] float, t fastest.
 *  - Grid indices are unpadded; the library pads by `pml` cells on every side.
 *  - Steps simulated: NT = nt + ndel; recording starts at step ndel.
 *  - The wavelet has NT samples (rickerWavelet(dt, fr, delay, NT),
 *    src/util/wavelet.cpp:7-18).
 *  - gz[nx] holds one receiver depth index per model column.
 *
 * Differences from the reference surface, all deliberate:
 *  - Results are written into caller buffers; nothing is returned by the
 *    library that the caller must free.
 *  - Every entry point returns a status (0 = SEIS_OK, negative = error) and
 *    never calls exit(); seis_fd_last_error() gives the message.
 *  - A context owns one CUDA stream on one device; do not share a context
 *    between host threads.  Calls on one context are synchronous unless named
 *    *_async.
 *
 * Pointers named h_* are host memory; d_* are device memory of the context's
 * device.  Host pointers may be pageable or pinned.
 */
#ifndef SEIS_FD_H
#define SEIS_FD_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SEIS_FD_ABI_VERSION 1

/* status codes */
#define SEIS_OK 0
#define SEIS_ERR_ARG (-1)       /* invalid argument (size, index, null pointer) */
#define SEIS_ERR_CUDA (-2)      /* a CUDA runtime call failed */
#define SEIS_ERR_NOMEM (-3)     /* device memory exhausted */
#define SEIS_ERR_STATE (-4)     /* call not valid in the object's current state */
#define SEIS_ERR_NOTSUP (-5)    /* operation not supported for this plan */
#define SEIS_ERR_CANCELLED (-6) /* batch cancelled by the caller */

typedef struct seis_fd_ctx seis_fd_ctx;
typedef struct seis_fd_plan seis_fd_plan;

/* One shot: the argument list of modeling/forward/adjoint (src/util/fd.h:3-5)
 * minus the arrays. */
typedef struct {
  int nx, nz;     /* model (aperture) extent, cells */
  int pml;        /* absorbing pad width, cells (>= 1) */
  int nt;         /* recorded samples */
  int ndel;       /* steps simulated before recording starts */
  int sx, sz;     /* source cell, unpadded indices */
  float dt, dx, dz;
  const int *gz;  /* host pointer, gz[nx]: receiver depth index of each column */
} seis_shot_desc;

/* ---------------------------------------------------------------- context */
int seis_fd_abi_version(void);
int seis_fd_create(seis_fd_ctx **out, int device);
int seis_fd_destroy(seis_fd_ctx *ctx);
const char *seis_fd_last_error(const seis_fd_ctx *ctx);
/* Number of kernel launches this context has issued since creation
 * (graph-replayed launches included). */
int64_t seis_fd_launch_count(const seis_fd_ctx *ctx);

/* ------------------------------------------------------ host-only helpers */
/* rickerWavelet (src/util/wavelet.cpp:7-18): out[n], (1-2 tmp t^2) exp(-tmp t^2)
 * with tmp = pi^2 fr^2 formed in double, t = (i - delay) dt.  No device. */
int seis_fd_ricker(float dt, float fr, int delay, int n, float *out);
/* Argument checks of one shot without touching a device: 0 or SEIS_ERR_ARG,
 * with the reason copied into msg[msg_len] when msg is not null. */
int seis_fd_validate_shot(const seis_shot_desc *shot, char *msg, size_t msg_len);

/* ------------------------------------------------------ single-shot calls */
/* modeling (src/util/fd.cpp:15-80): h_rec[nx][nt] = shot gather. */
int seis_fd_modeling(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_wav,
                     const float *h_vel, float *h_rec);

/* forward, linearised Born modeling (src/util/fd.cpp:81-177):
 * h_rec[nx][nt] = scattered gather for velocity perturbation h_dv[nx][nz]. */
int seis_fd_born(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_wav,
                 const float *h_vel, const float *h_dv, float *h_rec);

/* adjoint, reference RTM (src/util/fd.cpp:592-719): boundary-saving source
 * reconstruction, receiver back-propagation injected as rec*vt2, imaging
 * lap*vel3*R plus the Hilbert term of FaQi (:1272-1298).
 * h_img[nx][nz] = image. */
int seis_fd_rtm(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_wav,
                const float *h_vel, const float *h_rec, float *h_img);

#ifdef __cplusplus
}
#endif
#endif
