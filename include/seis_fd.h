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

#define SEIS_FD_ABI_VERSION 2

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
/* Destroys the context and the device state of every plan created on it; the
 * plan handles stay valid for seis_fd_plan_destroy only. */
int seis_fd_destroy(seis_fd_ctx *ctx);
const char *seis_fd_last_error(const seis_fd_ctx *ctx);
/* Number of kernel launches this context has issued since creation
 * (graph-replayed launches included). */
int64_t seis_fd_launch_count(const seis_fd_ctx *ctx);
/* The cudaStream_t every call of this context is ordered on, so that callers
 * can order (or time) their own work around it. */
void *seis_fd_stream(const seis_fd_ctx *ctx);

/* ------------------------------------------------------ host-only helpers */
/* rickerWavelet (src/util/wavelet.cpp:7-18): out[n], (1-2 tmp t^2) exp(-tmp t^2)
 * with tmp = pi^2 fr^2 formed in double, t = (i - delay) dt.  No device. */
int seis_fd_ricker(float dt, float fr, int delay, int n, float *out);
/* Hilbert<float>(half).apply (src/filter/hilbert.h:22-70): out[n] = the
 * (2 half + 1)-tap Hamming-tapered Hilbert FIR of in[n], convolved in full and
 * cut to n.  Host only. */
int seis_fd_hilbert(const float *in, float *out, int n, int half);

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

/* illum (src/util/fd.cpp:275-339): h_ss[nx][nz] = sum over it > ndel of the
 * blended source field squared, accumulated step by step in FP32 (the
 * illumination of the reference's illum_MPI, inversion.cpp:207-290).
 * shot->gz may be NULL (receivers play no part). */
int seis_fd_illum(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_wav,
                  const float *h_vel, float *h_ss);
int seis_fd_illum_batch(seis_fd_ctx *ctx, int nshot, const seis_shot_desc *shots,
                        const float *const *h_wav, const float *const *h_vel,
                        float *const *h_ss);

/* forwordPlane (src/util/fd.cpp:178-274): Born modeling with the areal
 * source h_sou[nx][nt+ndel] injected at row shot->sz of every model column
 * (a plane-wave or phase-encoded source, see seis_driver_plane_prepare) and
 * receivers at rows shot->gz (the reference takes one row for all).
 * shot->sx is not used.  h_rec[nx][nt]. */
int seis_fd_born_plane(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_sou,
                       const float *h_vel, const float *h_dv, float *h_rec);

/* illumPlane (src/util/fd.cpp:720-786): seis_fd_illum with the areal source
 * h_sou[nx][nt+ndel] at row shot->sz of every model column (shot->sx and
 * shot->gz are not used).  h_ss[nx][nz]. */
int seis_fd_illum_plane(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_sou,
                        const float *h_vel, float *h_ss);

/* rtm_true (src/util/fd.cpp:924-1052): seis_fd_rtm with the receivers injected
 * as vertical dipoles (-rec vt2/dz at row gz, +rec vt2/dz at row gz + 1) and
 * the image FaQi(S vel3, R) of the reconstructed source field S itself. */
int seis_fd_rtm_true(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_wav,
                     const float *h_vel, const float *h_rec, float *h_img);

/* adjointUpDown (src/util/fd.cpp:340-590): seis_fd_rtm with a second source
 * field driven by h_wavh[nt+ndel] (the Hilbert transform of h_wav, see
 * seis_fd_hilbert) and four imaging components summed over the reverse pass,
 * H = the 61-tap Hilbert filter along depth:
 *   h_comp[0] += S R, [1] += H[S] H[R], [2] += St H[R], [3] += H[St] R
 * (S, St the two reconstructed source fields, R the receiver field);
 * h_img = comp0 - comp1 + comp3 + comp2.  h_comp [4][nx][nz] may be NULL. */
int seis_fd_rtm_updown(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_wav,
                       const float *h_wavh, const float *h_vel, const float *h_rec, float *h_img,
                       float *h_comp);

/* adjointPlane (src/util/fd.cpp:787-921): RTM of the areal source
 * h_sou[nx][nt+ndel] at row shot->sz with the gather h_rec[nx][nt] at rows
 * shot->gz; the receiver field is back-propagated first keeping its boundary
 * layers, then re-propagated beside the source field; FaQi imaging.  Gather
 * samples at negative time indices, which the reference reads outside its
 * array (fd.cpp:834, :873), are skipped.  h_img[nx][nz]. */
int seis_fd_rtm_plane(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_sou,
                      const float *h_vel, const float *h_rec, float *h_img);

/* ---------------------------------------------------------- shot batches */
/* A plan is a batch of shots resident on the device.  It replaces the
 * reference's MPI shot farm (masterRun + worker loops,
 * src/lsrtm/inversion.cpp:141-551, :753-807): every shot of the batch
 * advances in the same launches, one per time step.  All shots of a plan share
 * nt, ndel and dt; nx, nz, pml, dx, dz, sources and receivers may differ.
 * The first seis_fd_plan_run captures the time loop into a CUDA graph; later
 * runs replay it.  Inputs persist across runs until overwritten. */
#define SEIS_OP_MODELING 0 /* modeling (fd.cpp:15-80)                      */
#define SEIS_OP_BORN 1     /* forward, Born (fd.cpp:81-177)                 */
#define SEIS_OP_RTM 2      /* adjoint, reference RTM (fd.cpp:592-719)       */
#define SEIS_OP_BORN_ADJOINT 3 /* exact adjoint of SEIS_OP_BORN (no reference
                                  counterpart): gather -> image             */
#define SEIS_OP_ILLUM 4    /* illum, source illumination (fd.cpp:275-339):
                              wavelet, velocity -> image [nx][nz]           */
#define SEIS_OP_BORN_PLANE 5 /* forwordPlane, Born with an areal source
                                (fd.cpp:178-274): source, velocity, dv -> gather */
#define SEIS_OP_RTM_PLANE 6  /* adjointPlane, RTM of an areal source
                                (fd.cpp:787-921): source, velocity, gather -> image */
#define SEIS_OP_RTM_TRUE 7   /* rtm_true (fd.cpp:924-1052): the RTM with a dipole
                                receiver injection and source-field imaging */
#define SEIS_OP_RTM_UPDOWN 8 /* adjointUpDown (fd.cpp:340-590): four-component
                                RTM with a Hilbert-wavelet source field      */
#define SEIS_OP_ILLUM_PLANE 9 /* illumPlane (fd.cpp:720-786): source, velocity
                                 -> image [nx][nz]                           */

#define SEIS_IN_VEL 0      /* [nx][nz] velocity of the shot's model         */
#define SEIS_IN_DV 1       /* [nx][nz] velocity perturbation (SEIS_OP_BORN) */
#define SEIS_IN_WAVELET 2  /* [nt+ndel] source wavelet                      */
#define SEIS_IN_GATHER 3   /* [nx][nt] receiver data (SEIS_OP_RTM)          */
#define SEIS_IN_SOURCE 4   /* [nx][nt+ndel] areal source at row sz (plane-wave ops) */
#define SEIS_IN_WAVELET_H 5 /* [nt+ndel] Hilbert-transformed wavelet (SEIS_OP_RTM_UPDOWN) */
#define SEIS_OUT_GATHER 0  /* [nx][nt] recorded gather                      */
#define SEIS_OUT_IMAGE 1   /* [nx][nz] image                                */
#define SEIS_OUT_COMPONENTS 2 /* [4][nx][nz] imaging components (SEIS_OP_RTM_UPDOWN) */

/* Storage of the source-term snapshots (background second time derivative)
 * that SEIS_OP_BORN_ADJOINT images with. */
#define SEIS_SNAP_F32 1
#define SEIS_SNAP_BF16 2   /* one power-of-two scale per snapshot and kernel tile */
#define SEIS_SNAP_F16 3    /* same */

int seis_fd_plan_create(seis_fd_ctx *ctx, int op, int nshot, const seis_shot_desc *shots,
                        seis_fd_plan **out);
int seis_fd_plan_destroy(seis_fd_plan *plan);
/* Copy one input of one shot from host memory (pinned memory makes it
 * asynchronous on the context stream). */
int seis_fd_plan_set(seis_fd_plan *plan, int shot, int what, const float *h_src);
/* Same, from device memory of the context's device. */
int seis_fd_plan_set_device(seis_fd_plan *plan, int shot, int what, const float *d_src);
/* Enqueue the operator over every shot on the context stream. */
int seis_fd_plan_run(seis_fd_plan *plan);
/* Copy one output of one shot to host memory; synchronises the stream. */
int seis_fd_plan_get(seis_fd_plan *plan, int shot, int what, float *h_dst);
/* Wait for the plan's enqueued work. */
int seis_fd_plan_sync(seis_fd_plan *plan);
/* Padded cell-updates of one run (cells x steps x propagated fields). */
int64_t seis_fd_plan_cell_updates(const seis_fd_plan *plan);
/* Kernel launches of one run. */
int64_t seis_fd_plan_launches_per_run(const seis_fd_plan *plan);

/* Snapshots of SEIS_OP_BORN_ADJOINT plans: keep the source term every
 * `every` steps (1 = every step) as `dtype` (SEIS_SNAP_*).  every = 1 with
 * SEIS_SNAP_F32 makes the operator the exact transpose of SEIS_OP_BORN (up to
 * FP32 rounding); larger intervals and 16-bit storage trade accuracy for
 * memory (the imaging term of a stored step is weighted by `every`).  Default:
 * every = 1, SEIS_SNAP_F32.  Call before the first run. */
int seis_fd_plan_set_snapshots(seis_fd_plan *plan, int every, int dtype);
/* Source-field checkpoints of SEIS_OP_BORN_ADJOINT plans, for surveys whose
 * snapshots do not fit in device memory (the largest configuration, 4000 x
 * 1000 cells and 8000 steps, needs about 16 GB of BF16 snapshots per shot).
 * every = 0 (default) keeps every snapshot of the run.  every = C > 0, a
 * multiple of the snapshot interval: the source pass keeps only the two time
 * levels before every C-th step, and each run recomputes the snapshots of one
 * C-step segment at a time, just before the reverse steps that image with
 * them, into storage for C / every + 1 snapshots.  The image is bit-identical
 * to every = 0; a run advances one more field per step.  No counterpart in
 * the reference, which keeps no snapshots.  Call before the first run. */
int seis_fd_plan_set_checkpoints(seis_fd_plan *plan, int every);
/* Bytes of device memory the plan holds (fields, models, gathers, images,
 * snapshots once allocated). */
int64_t seis_fd_plan_device_bytes(const seis_fd_plan *plan);
/* Arithmetic flavour of a plan's propagation kernels.  exact = 1 (default):
 * every operation rounds on its own in the reference's order, so results equal
 * the reference's bit for bit.  exact = 0: multiply-add contraction and
 * approximate division; results agree with the reference to FP32 rounding
 * level (relative L2 well below 1e-5) and the kernels issue fewer
 * instructions. */
int seis_fd_plan_set_exact(seis_fd_plan *plan, int exact);
/* Kernel timing: run 2 x `steps` time steps of the plan's propagation kernels
 * eagerly (outside the graph) on the plan's current fields: `steps` with the
 * interior-tile kernel and the pad-tile kernel one after the other, each
 * bracketed by CUDA events on its own stream, then `steps` as a run launches
 * them (concurrently, on two streams).  ms[0] = mean interior-kernel
 * duration, ms[1] = mean pad-kernel duration (each alone), ms[2] = mean step
 * as run.  bytes[0] = algorithmic bytes one interior launch moves (16 per
 * field-update: read prev, cur, velocity; write next), bytes[1] = same for the
 * pad launch.  The plan's fields are clobbered; the next run starts from its
 * cleared state. */
int seis_fd_plan_time_kernels(seis_fd_plan *plan, int steps, double *ms, double *bytes);

/* Tile shapes of the step kernels (columns x rows of one CTA's tile; no
 * counterpart in the reference, whose OpenMP loops split x only,
 * src/util/fd.cpp:1242-1271).  Every shape gives the same results bit for bit;
 * they differ in halo overhead, threads per CTA and CTAs per SM. */
#define SEIS_TILE_32x64 0   /* 256 threads (default) */
#define SEIS_TILE_64x32 1   /* 256 threads */
#define SEIS_TILE_16x128 2  /* 256 threads */
#define SEIS_TILE_64x64 3   /* 512 threads */
#define SEIS_TILE_32x32 4   /* 128 threads */
#define SEIS_TILE_SHAPES 5
/* Set the plan's tile shape.  SEIS_ERR_STATE once an adjoint plan's snapshots
 * are allocated (their scales are tiled like the kernels). */
int seis_fd_plan_set_tile_shape(seis_fd_plan *plan, int shape);
/* The plan's tile shape, or SEIS_ERR_ARG. */
int seis_fd_plan_tile_shape(const seis_fd_plan *plan);
/* Launch form of a step (flags; results are identical in every form):
 * SEIS_LAUNCH_OVERLAP: the interior-tile and the pad-tile kernel concurrently
 * on two streams (else one after the other on the context's stream);
 * SEIS_LAUNCH_PERSISTENT: interior tiles by the persistent kernel (as many
 * CTAs as are resident at once, each taking every G-th tile through two
 * shared-memory stages); SEIS_LAUNCH_PER_TILE: one interior tile per CTA;
 * neither: the persistent kernel when each of its CTAs gets at least 4 tiles.
 * A new plan has SEIS_LAUNCH_OVERLAP. */
#define SEIS_LAUNCH_OVERLAP 1
#define SEIS_LAUNCH_PERSISTENT 2
#define SEIS_LAUNCH_PER_TILE 4
int seis_fd_plan_set_launch(seis_fd_plan *plan, int flags);
/* The plan's launch flags, or SEIS_ERR_ARG. */
int seis_fd_plan_launch(const seis_fd_plan *plan);
/* Autotuner: time `steps` steps of the plan's own kernels (as
 * seis_fd_plan_time_kernels, on its current inputs) in every tile shape and
 * launch form (one tile per CTA or persistent, one after the other or
 * overlapped), and keep the fastest.  The choice is cached in the
 * process per plan signature (operator, build flavour, every shot's padded
 * grid) and reused by later plans of the same signature unless `force` is
 * set.  h_ms[SEIS_TILE_SHAPES] (may be null) receives each shape's shortest
 * mean step time (0 where not timed), *h_best (may be null) the shape kept.
 * The plan's fields are clobbered. */
int seis_fd_plan_autotune(seis_fd_plan *plan, int steps, int force, double *h_ms, int *h_best);

/* Batched forms of the single-shot calls: h_*[i] are the arrays of shot i. */
int seis_fd_modeling_batch(seis_fd_ctx *ctx, int nshot, const seis_shot_desc *shots,
                           const float *const *h_wav, const float *const *h_vel,
                           float *const *h_rec);
int seis_fd_born_batch(seis_fd_ctx *ctx, int nshot, const seis_shot_desc *shots,
                       const float *const *h_wav, const float *const *h_vel,
                       const float *const *h_dv, float *const *h_rec);
int seis_fd_rtm_batch(seis_fd_ctx *ctx, int nshot, const seis_shot_desc *shots,
                      const float *const *h_wav, const float *const *h_vel,
                      const float *const *h_rec, float *const *h_img);

/* Exact adjoint of seis_fd_born (no reference counterpart): h_img[nx][nz] =
 * L^T h_rec for the Born operator L of the same shot, snapshots every step in
 * FP32.  <L m, d> = <m, L^T d> to FP32 rounding. */
int seis_fd_born_adjoint(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_wav,
                         const float *h_vel, const float *h_rec, float *h_img);

/* ------------------------------------------------------- vector vocabulary */
/* The CG vector operations of the reference's opern (src/util/arraymath.h),
 * on device vectors of the context's device. */
/* DOTPRODUCT (arraymath.h:230-299): *h_out = sum (double)(a[i] * b[i]). */
int seis_fd_vec_dot(seis_fd_ctx *ctx, const float *d_a, const float *d_b, size_t n,
                    double *h_out);
/* No counterpart in the reference.  The same dot product for callers that
 * cannot allocate device memory (an application that owns the whole device
 * budget, a plugin that must not bypass its host's memory pool, a loop that
 * cannot afford the synchronisation cudaMalloc/cudaFree may cause): no
 * context, no allocation.  *d_out (device memory) = sum (double)(a[i] * b[i]),
 * FP32 products and FP64 sum as above, enqueued on `stream` (a cudaStream_t;
 * null = legacy default stream) of the current device; the call returns once
 * the work is enqueued.  Its scratch, 16384 partial sums (128 KiB) in a fixed
 * array inside the library, limits n to SEIS_DOT_NOALLOC_MAX_N elements;
 * larger n returns SEIS_ERR_ARG.  Every GPU that loads the library holds the
 * array until the process exits.  The array's device address belongs to the
 * current CUDA context (each context, e.g. one made by cuCtxCreate or the
 * primary context made again after cudaDeviceReset, has its own copy): a call
 * outside stream capture looks it up in the current context; a call whose
 * stream is capturing uses the address recorded by an earlier call in the
 * same context and returns SEIS_ERR_STATE if there was none, so make one call
 * in each context before capturing.  All calls in a context share the array:
 * calls whose GPU work overlaps (e.g. on two streams without ordering between
 * them) race and give wrong sums.  A message for any error goes to err
 * (err_len bytes, may be null). */
#define SEIS_DOT_NOALLOC_MAX_N ((size_t)16384 * 4096)
int seis_fd_vec_dot_noalloc(const float *d_a, const float *d_b, size_t n, double *d_out,
                            void *stream, char *err, size_t err_len);
/* ADDSCAL (arraymath.h:338-342): y = a x + b y, formed in double. */
int seis_fd_vec_axpby(seis_fd_ctx *ctx, float *d_y, const float *d_x, double a, double b,
                      size_t n);

/* -------------------------------------------------------------- LSRTM (CG) */
/* Least-squares RTM by conjugate gradient (CGLS) on a global model grid.  The
 * reference declares this solver (Inversion::conope_MPI, cgsolver_MPI,
 * src/lsrtm/inversion.h:81,87) but never defines it.
 *   L m  = [ Born_s( m[x0_s .. x0_s + nx_s) ) ]_s      (forward, per shot)
 *   L^T d = sum_s scatter_{x0_s}( BornAdjoint_s(d_s) )
 * Shot s covers columns x0_s .. x0_s + nx_s - 1 of the nx x nz global grid and
 * has the global nz (seis_fd_lsrtm_create_mapped: any non-decreasing map).  The background velocity and wavelet are fixed: the
 * adjoint's source-term snapshots are computed once and reused by every
 * iteration.  Dot products, step lengths and residual norms are FP64. */
typedef struct seis_fd_lsrtm seis_fd_lsrtm;
typedef struct {
  int snap_every;  /* source-term snapshot interval (default 1)            */
  int snap_dtype;  /* SEIS_SNAP_* (default SEIS_SNAP_F16: with the per-tile
                      scale, 3 more mantissa bits than BF16 at the same size) */
  int exact;       /* Born kernels round like the reference (default 0)    */
  int checkpoint_every; /* source-field checkpoint interval (default 0 = keep
                           every snapshot; see seis_fd_plan_set_checkpoints) */
  int group_shots; /* 0 (default): the plans of all shots stay on the device.
                      n > 0: each operator application builds the plans of n
                      shots at a time and frees them (for surveys whose plans
                      do not fit at once); the source pass then runs in every
                      application, and the results are identical */
  int tile_shape;  /* 0 (default): the tile shape of each Born and adjoint plan
                      is picked by seis_fd_plan_autotune once its background
                      is set (cached per plan signature); k > 0: shape k - 1
                      (SEIS_TILE_*) */
} seis_lsrtm_opts;

int seis_fd_lsrtm_create(seis_fd_ctx *ctx, int nx, int nz, int nshot,
                         const seis_shot_desc *shots, const int *x0,
                         const seis_lsrtm_opts *opts, seis_fd_lsrtm **out);
/* Same with an explicit column map: colmap holds, shot after shot, the model
 * column of each of the shot's nx_s sub-grid columns (non-decreasing, as the
 * aperture extraction of the shot driver clamps at the model edges); L^T
 * scatters through the transpose of that map. */
int seis_fd_lsrtm_create_mapped(seis_fd_ctx *ctx, int nx, int nz, int nshot,
                                const seis_shot_desc *shots, const int *colmap,
                                const seis_lsrtm_opts *opts, seis_fd_lsrtm **out);
int seis_fd_lsrtm_destroy(seis_fd_lsrtm *ls);
/* background velocity [nx][nz] of the global grid and wavelet [nt+ndel] */
int seis_fd_lsrtm_set_background(seis_fd_lsrtm *ls, const float *h_v0, const float *h_wav);
/* observed data of one shot, [nx_s][nt] */
int seis_fd_lsrtm_set_data(seis_fd_lsrtm *ls, int shot, const float *h_d);
/* Start CGLS from m = 0: r = d, s = L^T r, p = s.  *h_rr = |r|^2 (may be null). */
int seis_fd_lsrtm_reset(seis_fd_lsrtm *ls, double *h_rr);
/* niter CGLS iterations (one L and one L^T each); h_rr[i] = |r|^2 after
 * iteration i (h_rr may be null).  Enqueued without host round trips; returns
 * after the last iteration completes. */
int seis_fd_lsrtm_iterate(seis_fd_lsrtm *ls, int niter, double *h_rr);
/* The three phases of one iteration, for a solver whose shots are spread
 * over several devices (one solver per rank, each with its own shots and the
 * same model grid).  Each phase is enqueued on the context's stream and leaves
 * this rank's partial sums in the caller's device buffers; the caller sums
 * them over the ranks in place (e.g. an NCCL all-reduce on that stream) before
 * the next phase reads them.  On one device nothing needs summing:
 *   reset   = phase_reset(s, rr), phase_direction(s, first = 1)
 *   iterate = phase_forward(qq), phase_update(qq, s, rr), phase_direction(s, 0)
 * d_s: [nx][nz] float; d_qq, d_rr: one double. */
int seis_fd_lsrtm_phase_reset(seis_fd_lsrtm *ls, float *d_s, double *d_rr);
int seis_fd_lsrtm_phase_forward(seis_fd_lsrtm *ls, double *d_qq);
int seis_fd_lsrtm_phase_update(seis_fd_lsrtm *ls, const double *d_qq, float *d_s, double *d_rr);
int seis_fd_lsrtm_phase_direction(seis_fd_lsrtm *ls, const float *d_s, int first);
/* current model [nx][nz] */
int seis_fd_lsrtm_model(seis_fd_lsrtm *ls, float *h_m);
/* padded cell-updates of one iteration (Born + adjoint reverse pass) */
int64_t seis_fd_lsrtm_cell_updates(const seis_fd_lsrtm *ls);
int64_t seis_fd_lsrtm_device_bytes(const seis_fd_lsrtm *ls);

#ifdef __cplusplus
}
#endif
#endif
