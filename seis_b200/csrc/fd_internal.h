// Internal structures shared by the host runtime (fd_host.cpp) and the CUDA
// kernels (fd_kernels.cu).  Not part of the public ABI.
#pragma once
#include <cuda.h>  // CUtensorMap (type only; maps are encoded through the runtime entry point)
#include <cuda_runtime.h>
#include <stdint.h>

namespace seis {

// Tiling.  The padded grid of every shot is cut into tiles of TX columns x TZ
// rows (z contiguous), one tile per CTA, each thread a 4-row x 2-column
// micro-tile (TX * TZ / 8 threads).  A plan uses one of the shapes below,
// fixed when it is built or picked by timing its own steps
// (seis_fd_plan_autotune).  Field arrays carry zero margins (ZM rows above and
// below, XM columns on either side) and are rounded up to the largest tile in
// each direction, so that every staged column segment [z0 - ZM, z0 + TZ + ZM)
// of every tile of every shape, with an HXC-column halo, lies inside the
// allocation.
enum TileShapeId : int {
  SHAPE_32x64 = 0,   // 256 threads
  SHAPE_64x32 = 1,   // 256 threads
  SHAPE_16x128 = 2,  // 256 threads
  SHAPE_64x64 = 3,   // 512 threads
  SHAPE_32x32 = 4,   // 128 threads
  NSHAPES = 5,
};
constexpr int shape_tx(int s) { return s == 1 || s == 3 ? 64 : s == 2 ? 16 : 32; }
constexpr int shape_tz(int s) { return s == 2 ? 128 : s == 0 || s == 3 ? 64 : 32; }
constexpr int TX_MAX = 64;
constexpr int TZ_MAX = 128;
constexpr int HXC = 5;      // column halo of the current field (stencil radius 4 + 1)
constexpr int ZM = 8;
constexpr int HI = 4;       // interior tiles: column and row halo of the current field
constexpr int XM = 16;
constexpr int LAYERS = 4;   // boundary layers kept for reconstruction

enum TileKind : int {
  TILE_INTERIOR = 0,  // every cell inside the model, 8th order and off the model's edge
                      // rows / columns (which the one-way update of the pad reads)
  TILE_PAD = 1,       // touches the pad, the frame, the low-order rings or the model edge
};

struct Tile {
  int shot, x0, z0, kind;
};

// 2-D TMA tensor maps of one shot (each describes one margin-padded field
// allocation, LDZ rows x ncols columns; box = staged rows x staged columns).
// Pad tiles: wide boxes (TX + 2*HXC columns, TZ + 2*ZM rows) stage a field read
// as "current"; narrow boxes (TX + 2 columns) a field read as "previous", the
// velocity or dv.  Interior tiles: the current field with an HI-cell halo on
// every side, the other arrays as the tile alone.
enum MapIndex : int {
  MAP_FA_WIDE = 0,    // + rotating buffer index 0..2
  MAP_FA_NARROW = 3,
  MAP_FB_WIDE = 6,
  MAP_FB_NARROW = 9,
  MAP_VEL = 12,
  MAP_DV = 13,
  MAP_VEL_WIDE = 14,  // velocity with the wide halo (adjoint kernels)
  MAP_FA_HALO = 15,   // interior tiles: (TX + 2 HI) x (TZ + 2 HI), + buffer index
  MAP_FB_HALO = 18,
  MAP_FA_TILE = 21,   // interior tiles: TX x TZ, + buffer index
  MAP_FB_TILE = 24,
  MAP_VEL_TILE = 27,
  MAP_DV_TILE = 28,
  MAP_VEL_HALO = 29,  // interior tiles of the adjoint: velocity with the HI-cell halo
  NMAPS = 30,
};

// Device descriptor of one shot in a batch.  Scalars derived from dt/dx/dz are
// formed on the host in the reference's operation order.
struct ShotDev {
  int nx, nz, pml, NX, NZ, LDZ;
  int sxp, szp;        // padded source cell
  int NT, ndel, nt;
  int strip_len;       // LAYERS * 2 * (nx + nz)
  float dt, dx, dz;
  float invdx2, invdz2;  // 1/(dx dx), 1/(dz dz)           fd.cpp:21-22
  float kx, kz;          // (1/dx)(1/dx) dt^2, same for z   fd.cpp:1058-1059
  float a1z, a1x;        // 1/dz/2/dt, 1/dx/2/dt            fd.cpp:1098,1124
  float hdt2;            // 1/2/dt/dt (a2 = hdt2 / v)        fd.cpp:1099
  float ax1, ax2;        // 1/dz, 1/dx                      fd.cpp:1150-1151
  float sqrt2f;          // sqrt(2.0f)                      fd.cpp:1152
  float idt2;            // 1/dt/dt                         fd.cpp:89
  double sqrt2d;         // sqrt(2) in double               fd.cpp:1176
  float *fa[3];          // field A rotating buffers, NX x LDZ
  float *fb[3];          // field B rotating buffers (Born scattered / RTM receiver)
  const float *vel;      // padded velocity, NX x LDZ
  const float *dv;       // padded perturbation (zero pad), NX x LDZ
  const int *gz;         // receiver depth index per interior column [nx]
  const float *wav;      // [NT]
  float *rec;            // gather, device layout [nt][nx]
  float *strips;         // boundary strips, [nt][strip_len]
  float *img;            // image [nx][nz]
  const CUtensorMap *maps;  // NMAPS tensor maps of this shot (device memory)
  // source-term snapshots for the adjoint imaging condition: lap of the
  // background field at every snap_every-th step, interior cells [nx][nz],
  // stored as snap_dtype with one power-of-two scale per (snapshot, tile)
  void *snap;
  float *snap_scale;     // [nsnap][ntile_x * ntile_z]
  double *grad;          // FP64 imaging accumulator [nx][nz]
  int snap_dtype;        // SNAP_NONE / SNAP_F32 / SNAP_BF16 / SNAP_F16
  int snap_every;
  int ntz;               // tiles along z of this shot (scale indexing)
  int pad_;
  float *illum;          // source illumination [nx][nz] (illumination plans)
  const float *sou;      // areal source [NT][nx] at row szp (plane-wave plans), else null
  float *comp;           // four imaging accumulators [4][nx][nz] (adjointUpDown)
  int rcv_dipole;        // receiver injection as a vertical dipole (rtm_true)
  int pad2_;
  // exact adjoint, pad and model edge cells (NX x LDZ each): the ring terms
  // of a step, in two buffers used by alternate steps (this step's read, the
  // next step's written); the prev-ring terms kept for the step after next
  float *adj_e[2], *adj_b;
  // reciprocals for the contracted build's absorbing formulas: 1/4/dx/dx,
  // 1/4/dz/dz, 1/pml
  float q4dx2, q4dz2, inv_pml;
  int pad3_;
  // exact adjoint: coefficients of the transposed frame and low-order terms
  // of the cells within 4 of the grid edge (EDGE_TAPS per cell, tap-major:
  // tap k of band cell i at edge_coef[k * edge_cells(NX, NZ) + i]; band
  // cells indexed by edge_index)
  float *edge_coef;
};
// Cells of the four edge bands of a padded grid: the 5 top and 5 bottom rows
// (column-major, 5 rows per column) and the 5 left and 5 right columns.
constexpr int EDGE_TAPS = 13;  // 7 along z (offsets -3..3), 6 along x (-3..3 but 0)
__host__ __device__ inline int edge_cells(int NX, int NZ) { return 10 * (NX + NZ); }
// Band b (0 top, 1 bottom, 2 left, 3 right) cell (cx, cz) -> its index.
__host__ __device__ inline int edge_index(int b, int NX, int NZ, int cx, int cz) {
  return b == 0 ? cx * 5 + cz
       : b == 1 ? 5 * NX + cx * 5 + (cz - (NZ - 5))
       : b == 2 ? 10 * NX + cx * NZ + cz
                : 10 * NX + 5 * NZ + (cx - (NX - 5)) * NZ + cz;
}
enum SnapType : int { SNAP_NONE = 0, SNAP_F32 = 1, SNAP_BF16 = 2, SNAP_F16 = 3 };
static_assert(sizeof(ShotDev) % sizeof(int) == 0 && sizeof(ShotDev) <= 256 * sizeof(int),
              "ShotDev is copied word by word into shared memory");

// Per-launch step arguments.  Every optional index defaults to -1 (none).
struct StepArgs {
  int rot = 0;       // buffers: prev = f[rot%3], cur = f[(rot+1)%3], next = f[(rot+2)%3]
  int rot_b = 0;     // same for field B
  int src_k = -1;    // wavelet sample injected at the source
  int rec_k = -1;    // gather sample recorded (or injected, receiver / adjoint mode)
  int strip_k = -1;  // boundary-strip sample saved
  int nshots = 0;
  int snap_k = -1;   // snapshot index written (forward) or imaged (adjoint)
  float img_w = 0.f; // adjoint: weight of the imaging term (snapshot interval)
  int illum_on = 0;  // add the square of every model cell's new value to g.illum
  // interior kernel: -1 the persistent one when each of its CTAs gets at
  // least 4 tiles, else one tile per CTA; 0 one tile per CTA; 1 persistent
  int loop = -1;
};

// Allocation geometry of one field of a shot: LDZ floats per column, and the
// element offset of cell (0,0) from the allocation start.
struct FieldGeom {
  int LDZ;
  int ncols;      // XM + NX + right margin
  size_t elems;   // ncols * LDZ
  size_t origin;  // XM * LDZ + ZM
};
inline FieldGeom field_geom(int NX, int NZ) {
  FieldGeom f;
  int nstrip = (NZ + TZ_MAX - 1) / TZ_MAX;
  f.LDZ = ((ZM + nstrip * TZ_MAX + ZM) + 31) / 32 * 32;
  int right = ((NX + TX_MAX - 1) / TX_MAX) * TX_MAX - NX + XM;
  f.ncols = XM + NX + right;
  f.elems = (size_t)f.ncols * f.LDZ;
  f.origin = (size_t)XM * f.LDZ + ZM;
  return f;
}

// Kernel launchers (fd_kernels.cu, fd_step_*.cu, fd_adjoint_fast.cu).
enum StepMode : int {
  MODE_MODEL = 0,    // field A; point source; record; optional strip save
  MODE_RCV = 1,      // field B; receiver injection rec*vt2 (reference RTM)
  MODE_BORN = 2,     // fields A (background) and B (scattered)
};

// One time step over every tile of a batch: the first n_int tiles are
// interior tiles (one CTA each, stream s_int), the next n_pad pad tiles
// (one CTA each, stream s_pad; the absorbing boundary fused in), tiles of
// shape `shape` (TileShapeId).  `exact` selects the build that rounds like the
// reference; otherwise the contracted build.
cudaError_t launch_step(int mode, bool exact, const ShotDev *d_shots, const Tile *d_tiles,
                        int n_int, int n_pad, int shape, const StepArgs &a, int *d_err,
                        cudaStream_t s_int, cudaStream_t s_pad);
namespace exact {
cudaError_t launch_step(int mode, const ShotDev *d_shots, const Tile *d_tiles, int n_int,
                        int n_pad, int shape, const StepArgs &a, int *d_err, cudaStream_t s_int,
                        cudaStream_t s_pad);
cudaError_t configure();
}  // namespace exact
namespace fast {
cudaError_t launch_step(int mode, const ShotDev *d_shots, const Tile *d_tiles, int n_int,
                        int n_pad, int shape, const StepArgs &a, int *d_err, cudaStream_t s_int,
                        cudaStream_t s_pad);
cudaError_t configure();
// one reverse step of the exact Born adjoint over the adjoint tile list
// (interior tiles on s_int, pad tiles on s_pad)
// the exact adjoint's edge-band coefficients of every shot (after its
// velocity is in place); max_cells = the largest edge_cells of the batch
cudaError_t launch_edge_coef(const ShotDev *d_shots, int nshots, int max_cells, cudaStream_t s);
cudaError_t launch_adjoint(int shape, const ShotDev *d_shots, const Tile *d_tiles, int n_int,
                           int n_pad, const StepArgs &a, int *d_err, cudaStream_t s_int,
                           cudaStream_t s_pad);
cudaError_t configure_adjoint();
}  // namespace fast
cudaError_t launch_finalize_image(const ShotDev *d_shots, int nshots, cudaStream_t s);

// Vector operations of the CG solver (fd_vec.cu).  A dot product needs a
// scratch array of DOT_PARTS doubles for its per-CTA partial sums.
constexpr int DOT_PARTS = 1184;
cudaError_t launch_dot(const float *a, const float *b, size_t n, double *partial, double *out,
                       int accumulate, cudaStream_t s);
cudaError_t launch_axpby(float *y, const float *x, double a, double b, size_t n, cudaStream_t s);
cudaError_t launch_axpby_dev(float *y, const float *x, const double *sa, double fa,
                             const double *sb, double fb, size_t n, cudaStream_t s);
cudaError_t launch_add(float *y, const float *x, size_t n, cudaStream_t s);
cudaError_t launch_gather_cols(const float *src, int nz, const int *map, int nxs, float *dst,
                               cudaStream_t s);
cudaError_t launch_scatter_cols(float *dst, int nz, const int2 *ranges, int g0, int ncols,
                                const float *img, cudaStream_t s);
cudaError_t launch_ratio(const double *num, const double *den, double *out, cudaStream_t s);
// Set kernel attributes (shared-memory limits); call once per device.
cudaError_t configure_kernels();
cudaError_t launch_pad(const float *d_src, int nx, int nz, int pml, int LDZ, int clamp,
                       float *d_dst, cudaStream_t s);
cudaError_t launch_transpose(const float *d_src, int rows, int cols, float *d_dst,
                             cudaStream_t s);
cudaError_t launch_rtm_restore(const ShotDev *d_shots, int nshots, int max_strip, int rot,
                               int it, cudaStream_t s);
cudaError_t launch_rtm_image(const ShotDev *d_shots, const int2 *d_cols, int ncols, int rot,
                             int rot_b, int max_nz, const float *d_taps, cudaStream_t s,
                             int mode = 0);
cudaError_t launch_updown_image(const ShotDev *d_shots, const ShotDev *d_shots_h,
                                const int2 *d_cols, int ncols, int rot, int rot_b, int max_nz,
                                const float *d_taps, cudaStream_t s);
cudaError_t launch_updown_finalize(const ShotDev *d_shots, int nshots, cudaStream_t s);
cudaError_t launch_plane_rcv_prep(const ShotDev *d_shots, int nshots, int max_strip, int rot_b,
                                  int strip_k, int rec_k, cudaStream_t s);

}  // namespace seis
