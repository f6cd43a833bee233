// Internal structures shared by the host runtime (fd_host.cpp) and the CUDA
// kernels (fd_kernels.cu).  Not part of the public ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace seis {

// Tile of the padded grid handled by one CTA: TZ cells along z (contiguous)
// by TX columns along x.  The shared-memory copy of the current field carries
// a halo of HX columns and HZ rows (HZ rounded up to a float4 multiple).
constexpr int TZ = 64;
constexpr int TX = 32;
constexpr int HX = 5;
constexpr int HZ = 8;
constexpr int SROWS = TZ + 2 * HZ;  // rows of the shared tile (z)
constexpr int SCOLS = TX + 2 * HX;  // columns of the shared tile (x)
constexpr int NTHREADS = 128;
constexpr int LAYERS = 4;           // boundary layers kept for reconstruction

enum TileKind : int {
  TILE_INTERIOR = 0,  // every cell interior and 8th order: no absorbing terms
  TILE_BOUNDARY = 1,  // touches the pad, the frame or the low-order rings
};

struct Tile {
  int shot, x0, z0, kind;
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
};

// Per-launch step arguments.
struct StepArgs {
  int rot;      // buffers: prev = f[rot%3], cur = f[(rot+1)%3], next = f[(rot+2)%3]
  int rot_b;    // same for field B
  int src_k;    // wavelet sample injected at the source (-1: none)
  int rec_k;    // gather sample recorded (or injected, receiver mode) (-1: none)
  int strip_k;  // boundary-strip sample saved (-1: none)
  int nshots;
};

// Kernel launchers (fd_kernels.cu).
enum StepMode : int {
  MODE_MODEL = 0,    // field A; point source; record; optional strip save
  MODE_RCV = 1,      // field B; receiver injection rec*vt2 (reference RTM)
  MODE_BORN = 2,     // fields A (background) and B (scattered)
};

cudaError_t launch_step(int mode, const ShotDev *d_shots, const Tile *d_tiles, int ntiles,
                        const StepArgs &a, cudaStream_t s);
cudaError_t launch_pad(const float *d_src, int nx, int nz, int pml, int LDZ, int clamp,
                       float *d_dst, cudaStream_t s);
cudaError_t launch_transpose(const float *d_src, int rows, int cols, float *d_dst,
                             cudaStream_t s);
cudaError_t launch_rtm_restore(const ShotDev *d_shots, int nshots, int max_strip, int rot,
                               int it, cudaStream_t s);
cudaError_t launch_rtm_image(const ShotDev *d_shots, const int2 *d_cols, int ncols, int rot,
                             int rot_b, int max_nz, const float *d_taps, cudaStream_t s);

}  // namespace seis
