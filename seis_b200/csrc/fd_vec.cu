// Vector operations of the conjugate-gradient solver (sm_100a), in the
// arithmetic of the reference's opern vocabulary (src/util/arraymath.h):
//   DOTPRODUCT  out += (double)(a[i] * b[i])  -- FP32 product, FP64 sum (:230-299)
//   ADDSCAL     y = a1 x + a2 y formed in double, stored as float (:338-342)
// The dot product is a deterministic two-pass reduction: per-CTA partial sums
// in a scratch array, then one CTA adds the partials in a fixed order.
#include <algorithm>

#include "fd_internal.h"

namespace seis {
namespace {

constexpr int VT = 256;

__device__ __forceinline__ double block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  v = 0.0;
  if (warp == 0) {
    v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  return v;
}

__global__ void dot_partial_kernel(const float *__restrict__ a, const float *__restrict__ b,
                                   size_t n, double *__restrict__ partial) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    acc += (double)(a[i] * b[i]);
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

__global__ void dot_final_kernel(const double *__restrict__ partial, int nparts,
                                 double *__restrict__ out, int accumulate) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc += partial[i];
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) *out = accumulate ? *out + acc : acc;
}

// y = a x + b y, formed in double (ADDSCAL)
__global__ void axpby_kernel(float *__restrict__ y, const float *__restrict__ x, double a,
                             double b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    y[i] = (float)(a * (double)x[i] + b * (double)y[i]);
}

// y = a x + b y with the scalars read from device memory: a = sa[0] * fa,
// b = sb[0] * fb (lets a CG step run without a host round trip)
__global__ void axpby_dev_kernel(float *__restrict__ y, const float *__restrict__ x,
                                 const double *__restrict__ sa, double fa,
                                 const double *__restrict__ sb, double fb, size_t n) {
  const double a = sa ? sa[0] * fa : fa;
  const double b = sb ? sb[0] * fb : fb;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    y[i] = (float)(a * (double)x[i] + b * (double)y[i]);
}

// y[i] += x[i]
__global__ void add_kernel(float *__restrict__ y, const float *__restrict__ x, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    y[i] = y[i] + x[i];
}

// out = num / den (FP64 scalars on the device)
__global__ void ratio_kernel(const double *num, const double *den, double *out) {
  *out = *den != 0.0 ? *num / *den : 0.0;
}

// dst[ix][iz] = src[map[ix]][iz]: the sub-grid of a model by its column map
__global__ void gather_cols_kernel(const float *__restrict__ src, int nz, const int *__restrict__ map,
                                   int nxs, float *__restrict__ dst) {
  const size_t n = (size_t)nxs * nz;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t ix = i / nz, iz = i - ix * nz;
    dst[i] = src[(size_t)map[ix] * nz + iz];
  }
}

// transpose of the gather: model column g0 + c collects the sub-grid columns
// ranges[c].x .. ranges[c].y (the map is non-decreasing, so each preimage is
// a range), summed in column order
__global__ void scatter_cols_kernel(float *__restrict__ dst, int nz, const int2 *__restrict__ ranges,
                                    int g0, int ncols, const float *__restrict__ img) {
  const size_t n = (size_t)ncols * nz;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t c = i / nz, iz = i - c * nz;
    const int2 r = ranges[c];
    if (r.y < r.x) continue;
    float acc = img[(size_t)r.x * nz + iz];
    for (int ix = r.x + 1; ix <= r.y; ix++) acc += img[(size_t)ix * nz + iz];
    const size_t o = ((size_t)g0 + c) * nz + iz;
    dst[o] = dst[o] + acc;
  }
}

int grid_for(size_t n) {
  return (int)std::min<size_t>((n + VT - 1) / VT, (size_t)DOT_PARTS);
}

}  // namespace

cudaError_t launch_dot(const float *a, const float *b, size_t n, double *partial, double *out,
                       int accumulate, cudaStream_t s) {
  int g = std::max(1, grid_for(n));
  dot_partial_kernel<<<g, VT, 0, s>>>(a, b, n, partial);
  dot_final_kernel<<<1, VT, 0, s>>>(partial, g, out, accumulate);
  return cudaGetLastError();
}

cudaError_t launch_axpby(float *y, const float *x, double a, double b, size_t n, cudaStream_t s) {
  axpby_kernel<<<std::max(1, grid_for(n)), VT, 0, s>>>(y, x, a, b, n);
  return cudaGetLastError();
}

cudaError_t launch_axpby_dev(float *y, const float *x, const double *sa, double fa,
                             const double *sb, double fb, size_t n, cudaStream_t s) {
  axpby_dev_kernel<<<std::max(1, grid_for(n)), VT, 0, s>>>(y, x, sa, fa, sb, fb, n);
  return cudaGetLastError();
}

cudaError_t launch_add(float *y, const float *x, size_t n, cudaStream_t s) {
  add_kernel<<<std::max(1, grid_for(n)), VT, 0, s>>>(y, x, n);
  return cudaGetLastError();
}

cudaError_t launch_gather_cols(const float *src, int nz, const int *map, int nxs, float *dst,
                               cudaStream_t s) {
  gather_cols_kernel<<<std::max(1, grid_for((size_t)nxs * nz)), VT, 0, s>>>(src, nz, map, nxs, dst);
  return cudaGetLastError();
}

cudaError_t launch_scatter_cols(float *dst, int nz, const int2 *ranges, int g0, int ncols,
                                const float *img, cudaStream_t s) {
  scatter_cols_kernel<<<std::max(1, grid_for((size_t)ncols * nz)), VT, 0, s>>>(dst, nz, ranges, g0,
                                                                              ncols, img);
  return cudaGetLastError();
}

cudaError_t launch_ratio(const double *num, const double *den, double *out, cudaStream_t s) {
  ratio_kernel<<<1, 1, 0, s>>>(num, den, out);
  return cudaGetLastError();
}

}  // namespace seis
