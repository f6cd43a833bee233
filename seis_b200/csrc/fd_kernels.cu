// Auxiliary kernels of the FD engine (sm_100a): model padding, gather
// transposes, and the reverse-pass helpers of the reference RTM.  The time
// step itself is the tile kernel (fd_tile.cuh).
//
// Compiled with --fmad=false and IEEE division: the RTM imaging arithmetic
// rounds as the reference's does.
#include <algorithm>

#define SEIS_NS exact
#include "fd_cell.cuh"

namespace seis {
namespace {

using exact::coef;

// Pad a [nx][nz] model into a shot's field layout (cell (0,0) at dst):
// clamp-to-edge (setVel, InitInversion.cpp:92-113) or zero (setDv, :116-126).
// Only cells of the padded grid are written; the margins stay zero.
__global__ void pad_kernel(const float *__restrict__ src, int nx, int nz, int pml, int LDZ,
                           int clamp, float *__restrict__ dst) {
  const int NX = nx + 2 * pml, NZ = nz + 2 * pml;
  size_t n = (size_t)NX * NZ;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    int ix = (int)(i / NZ), iz = (int)(i - (size_t)ix * NZ);
    int jx = ix - pml, jz = iz - pml;
    float v = 0.0f;
    if (clamp) {
      jx = jx < 0 ? 0 : (jx >= nx ? nx - 1 : jx);
      jz = jz < 0 ? 0 : (jz >= nz ? nz - 1 : jz);
      v = src[(size_t)jx * nz + jz];
    } else if (jx >= 0 && jx < nx && jz >= 0 && jz < nz) {
      v = src[(size_t)jx * nz + jz];
    }
    dst[(size_t)ix * LDZ + iz] = v;
  }
}

__global__ void transpose_kernel(const float *__restrict__ src, int rows, int cols,
                                 float *__restrict__ dst) {
  __shared__ float tile[32][33];
  int c = blockIdx.x * 32 + threadIdx.x, r0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    int r = r0 + k;
    if (r < rows && c < cols) tile[k][threadIdx.x] = src[(size_t)r * cols + c];
  }
  __syncthreads();
  int r = r0 + threadIdx.x;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    int cc = blockIdx.x * 32 + k;
    if (r < rows && cc < cols) dst[(size_t)cc * rows + r] = tile[threadIdx.x][k];
  }
}

// Reverse pass of the reference RTM, before each step (fd.cpp:659-663):
// subtract the source from the older field and write the saved boundary
// strips of sample it-ndel into the current field.
__global__ void rtm_restore_kernel(const ShotDev *__restrict__ shots, int nshots, int rot,
                                   int it) {
  const int s = blockIdx.y;
  if (s >= nshots) return;
  const ShotDev &g = shots[s];
  if (it >= g.NT || it < g.ndel) return;
  float *prev = g.fa[rot % 3];
  float *cur = g.fa[(rot + 1) % 3];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0 && it - 1 > 0) {
    size_t off = (size_t)g.sxp * g.LDZ + g.szp;
    float vt2 = coef(g.vel[off], g).vt2;
    prev[off] = prev[off] - vt2 * g.wav[it - 1];
  }
  if (i >= g.strip_len) return;
  const float *src = g.strips + (size_t)(it - g.ndel) * g.strip_len;
  int rowcells = 2 * LAYERS * g.nx;
  int ix, iz;
  if (i < rowcells) {
    int l = i / g.nx, x = i - l * g.nx;
    ix = x + g.pml;
    iz = l < LAYERS ? g.pml + l : g.nz + g.pml - 1 - (l - LAYERS);
  } else {
    int j = i - rowcells;
    int l = j / g.nz, z = j - l * g.nz;
    iz = z + g.pml;
    ix = l < LAYERS ? g.pml + l : g.nx + g.pml - 1 - (l - LAYERS);
  }
  cur[(size_t)ix * g.LDZ + iz] = src[i];
}

// Before a re-propagation step of the plane-wave receiver field
// (adjointPlane, fd.cpp:870-893): the boundary layers kept for sample strip_k
// restored into the current field, and the receiver samples rec_k (times vt2)
// taken off the previous field at the receiver rows.  Either part is skipped
// when its index is negative.
__global__ void plane_rcv_prep_kernel(const ShotDev *__restrict__ shots, int nshots, int rot_b,
                                      int strip_k, int rec_k) {
  const int s = blockIdx.y;
  if (s >= nshots) return;
  const ShotDev &g = shots[s];
  float *prev = g.fb[rot_b % 3];
  float *cur = g.fb[(rot_b + 1) % 3];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (rec_k >= 0 && i < g.nx) {  // fd.cpp:870-874
    const size_t off = (size_t)(i + g.pml) * g.LDZ + (g.gz[i] + g.pml);
    const float vt2 = coef(g.vel[off], g).vt2;
    prev[off] = prev[off] - g.rec[(size_t)rec_k * g.nx + i] * vt2;
  }
  if (strip_k < 0 || i >= g.strip_len) return;
  const float *src = g.strips + (size_t)strip_k * g.strip_len;
  const int rowcells = 2 * LAYERS * g.nx;
  int ix, iz;
  if (i < rowcells) {
    int l = i / g.nx, x = i - l * g.nx;
    ix = x + g.pml;
    iz = l < LAYERS ? g.pml + l : g.nz + g.pml - 1 - (l - LAYERS);
  } else {
    int j = i - rowcells;
    int l = j / g.nz, z = j - l * g.nz;
    iz = z + g.pml;
    ix = l < LAYERS ? g.pml + l : g.nx + g.pml - 1 - (l - LAYERS);
  }
  cur[(size_t)ix * g.LDZ + iz] = src[i];  // SaveAtBoundary restore, fd.cpp:1206-1223
}

// Imaging of the reference RTM, one CTA per interior column (fd.cpp:668-669,
// :681-684, FaQi :1272-1298):
//   U = ((u2 + u0 - 2 u1)/dt^2) vel3,  img += U R,  img += 0.5 (U R - H[U] H[R])
// with H the 61-tap Hilbert FIR along z over the whole padded column.
constexpr int HILB_HALF = 30;
// imaging of adjoint (lap vel3 R + FaQi), adjointPlane (FaQi of lap vel3),
// rtm_true (FaQi of the source field times vel3)
enum ImageMode { IMG_RTM = 0, IMG_PLANE = 1, IMG_TRUE = 2 };
__global__ void rtm_image_kernel(const ShotDev *__restrict__ shots, const int2 *__restrict__ cols,
                                 int rot, int rot_b, const float *__restrict__ taps, int mode) {
  extern __shared__ float sh[];
  const int2 c = cols[blockIdx.x];
  const ShotDev &g = shots[c.x];
  const int ix = c.y + g.pml, NZ = g.NZ;
  float *sU = sh, *sR = sh + NZ;
  __shared__ float h[2 * HILB_HALF + 1];
  if (threadIdx.x < 2 * HILB_HALF + 1) h[threadIdx.x] = taps[threadIdx.x];
  // reverse-pass naming: u2 = older (prev), u1 = current, u0 = newest
  const float *u2 = g.fa[rot % 3], *u1 = g.fa[(rot + 1) % 3], *u0 = g.fa[(rot + 2) % 3];
  const float *r0 = g.fb[(rot_b + 2) % 3];
  const size_t col = (size_t)ix * g.LDZ;
  for (int iz = threadIdx.x; iz < NZ; iz += blockDim.x) {
    float v = g.vel[col + iz];
    float vel3 = 2.0f / (v * v * v);
    if (mode == IMG_TRUE) {  // rtm_true images the source field itself, fd.cpp:1014
      sU[iz] = u0[col + iz] * vel3;
    } else {
      float lap = (u2[col + iz] + u0[col + iz] - 2.0f * u1[col + iz]) * g.idt2;
      sU[iz] = lap * vel3;
    }
    sR[iz] = r0[col + iz];
  }
  __syncthreads();
  for (int iz = g.pml + threadIdx.x; iz < NZ - g.pml; iz += blockDim.x) {
    int i0 = max(iz - HILB_HALF, 0), i1 = min(iz + HILB_HALF, NZ - 1);
    float uh = 0.0f, rh = 0.0f;
    // odd offsets only: the even taps are exactly zero (hilbert.h:67)
    int start = i0 + (((iz - i0) & 1) ? 0 : 1);
    for (int i = start; i <= i1; i += 2) {
      float hk = h[iz - i + HILB_HALF];
      uh = uh + sU[i] * hk;
      rh = rh + sR[i] * hk;
    }
    float U = sU[iz], R = sR[iz];
    float *img = g.img + (size_t)c.y * g.nz + (iz - g.pml);
    float acc = mode == IMG_RTM ? *img + U * R : *img;  // the others image with FaQi alone
    acc = acc + 0.5f * (U * R - uh * rh);
    *img = acc;
  }
}

// adjointUpDown imaging (fd.cpp:501-521), one CTA per interior column: with
// S the source field of the wavelet, St that of its Hilbert transform (the
// shadow shot table) and R the receiver field, each with its 61-tap z-Hilbert
// transform over the padded column,
//   comp0 += S R, comp1 += H[S] H[R], comp2 += St H[R], comp3 += H[St] R.
__global__ void updown_image_kernel(const ShotDev *__restrict__ shots,
                                    const ShotDev *__restrict__ shots_h,
                                    const int2 *__restrict__ cols, int rot, int rot_b,
                                    const float *__restrict__ taps) {
  extern __shared__ float sh[];
  const int2 c = cols[blockIdx.x];
  const ShotDev &g = shots[c.x];
  const ShotDev &gh = shots_h[c.x];
  const int ix = c.y + g.pml, NZ = g.NZ;
  float *sS = sh, *sR = sh + NZ, *sT = sh + 2 * NZ;
  __shared__ float h[2 * HILB_HALF + 1];
  if (threadIdx.x < 2 * HILB_HALF + 1) h[threadIdx.x] = taps[threadIdx.x];
  const size_t col = (size_t)ix * g.LDZ;
  const float *S = g.fa[(rot + 2) % 3] + col, *T = gh.fa[(rot + 2) % 3] + col;
  const float *R = g.fb[(rot_b + 2) % 3] + col;
  for (int iz = threadIdx.x; iz < NZ; iz += blockDim.x) {
    sS[iz] = S[iz];
    sR[iz] = R[iz];
    sT[iz] = T[iz];
  }
  __syncthreads();
  const size_t plane = (size_t)g.nx * g.nz;
  for (int iz = g.pml + threadIdx.x; iz < NZ - g.pml; iz += blockDim.x) {
    const int i0 = max(iz - HILB_HALF, 0), i1 = min(iz + HILB_HALF, NZ - 1);
    float hs = 0.0f, hr = 0.0f, ht = 0.0f;
    const int start = i0 + (((iz - i0) & 1) ? 0 : 1);  // odd offsets: even taps are zero
    for (int i = start; i <= i1; i += 2) {
      const float hk = h[iz - i + HILB_HALF];
      hs = hs + sS[i] * hk;
      hr = hr + sR[i] * hk;
      ht = ht + sT[i] * hk;
    }
    float *cp = g.comp + (size_t)c.y * g.nz + (iz - g.pml);
    cp[0] = cp[0] + sS[iz] * sR[iz];
    cp[plane] = cp[plane] + hs * hr;
    cp[2 * plane] = cp[2 * plane] + sT[iz] * hr;
    cp[3 * plane] = cp[3 * plane] + ht * sR[iz];
  }
}

// img = comp0 - comp1 + comp3 + comp2 (fd.cpp:538-547)
__global__ void updown_finalize_kernel(const ShotDev *__restrict__ shots) {
  const ShotDev &g = shots[blockIdx.y];
  const size_t n = (size_t)g.nx * g.nz;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    g.img[i] = g.comp[i] - g.comp[n + i] + g.comp[3 * n + i] + g.comp[2 * n + i];
}

// Exact adjoint, last step: img = vt2 vel3 grad on the model interior (the
// scattering source is vt2 lap vel3 dv, fd.cpp:138-139; dv is zero-padded).
__global__ void finalize_image_kernel(const ShotDev *__restrict__ shots) {
  const ShotDev &g = shots[blockIdx.y];
  const int n = g.nx * g.nz;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int x = i / g.nz, z = i - x * g.nz;
    float v = g.vel[(size_t)(x + g.pml) * g.LDZ + (z + g.pml)];
    float vt2 = coef(v, g).vt2;
    float vel3 = 2.0f / (v * v * v);
    g.img[i] = (float)((double)(vt2 * vel3) * g.grad[i]);
  }
}

}  // namespace

cudaError_t launch_finalize_image(const ShotDev *d_shots, int nshots, cudaStream_t s) {
  dim3 grid(64, nshots);
  finalize_image_kernel<<<grid, 256, 0, s>>>(d_shots);
  return cudaGetLastError();
}

cudaError_t configure_kernels() {
  cudaError_t e = exact::configure();
  if (e == cudaSuccess) e = fast::configure();
  return e == cudaSuccess ? fast::configure_adjoint() : e;
}

cudaError_t launch_step(int mode, bool use_exact, const ShotDev *d_shots, const Tile *d_tiles,
                        int n_int, int n_pad, int shape, const StepArgs &a, int *d_err,
                        cudaStream_t s_int, cudaStream_t s_pad) {
  return use_exact ? exact::launch_step(mode, d_shots, d_tiles, n_int, n_pad, shape, a, d_err,
                                        s_int, s_pad)
                   : fast::launch_step(mode, d_shots, d_tiles, n_int, n_pad, shape, a, d_err,
                                       s_int, s_pad);
}

cudaError_t launch_pad(const float *d_src, int nx, int nz, int pml, int LDZ, int clamp,
                       float *d_dst, cudaStream_t s) {
  size_t n = (size_t)(nx + 2 * pml) * (nz + 2 * pml);
  int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  pad_kernel<<<blocks, 256, 0, s>>>(d_src, nx, nz, pml, LDZ, clamp, d_dst);
  return cudaGetLastError();
}

cudaError_t launch_transpose(const float *d_src, int rows, int cols, float *d_dst,
                             cudaStream_t s) {
  dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
  transpose_kernel<<<grid, block, 0, s>>>(d_src, rows, cols, d_dst);
  return cudaGetLastError();
}

cudaError_t launch_rtm_restore(const ShotDev *d_shots, int nshots, int max_strip, int rot,
                               int it, cudaStream_t s) {
  dim3 grid((max_strip + 255) / 256, nshots);
  rtm_restore_kernel<<<grid, 256, 0, s>>>(d_shots, nshots, rot, it);
  return cudaGetLastError();
}

cudaError_t launch_rtm_image(const ShotDev *d_shots, const int2 *d_cols, int ncols, int rot,
                             int rot_b, int max_nz, const float *d_taps, cudaStream_t s,
                             int mode) {
  size_t smem = 2 * (size_t)max_nz * sizeof(float);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(rtm_image_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  rtm_image_kernel<<<ncols, 256, smem, s>>>(d_shots, d_cols, rot, rot_b, d_taps, mode);
  return cudaGetLastError();
}

cudaError_t launch_updown_image(const ShotDev *d_shots, const ShotDev *d_shots_h,
                                const int2 *d_cols, int ncols, int rot, int rot_b, int max_nz,
                                const float *d_taps, cudaStream_t s) {
  size_t smem = 3 * (size_t)max_nz * sizeof(float);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(updown_image_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  updown_image_kernel<<<ncols, 256, smem, s>>>(d_shots, d_shots_h, d_cols, rot, rot_b, d_taps);
  return cudaGetLastError();
}

cudaError_t launch_updown_finalize(const ShotDev *d_shots, int nshots, cudaStream_t s) {
  dim3 grid(64, nshots);
  updown_finalize_kernel<<<grid, 256, 0, s>>>(d_shots);
  return cudaGetLastError();
}

cudaError_t launch_plane_rcv_prep(const ShotDev *d_shots, int nshots, int max_strip, int rot_b,
                                  int strip_k, int rec_k, cudaStream_t s) {
  dim3 grid((max_strip + 255) / 256, nshots);
  plane_rcv_prep_kernel<<<grid, 256, 0, s>>>(d_shots, nshots, rot_b, strip_k, rec_k);
  return cudaGetLastError();
}

}  // namespace seis
