// Dot product that allocates no device memory (sm_100a).
//
// Some callers cannot call cudaMalloc: a host application that reserves its
// whole device-memory budget up front and hands out only its own buffers, a
// plugin loaded into a process whose memory pool must not be bypassed, or a
// latency-bound loop that cannot afford the device-wide synchronisation a
// cudaMalloc or cudaFree may cause.  For them this file
// gives a variant of the CG inner product (seis_fd_vec_dot) whose scratch, the
// per-CTA partial sums, lives in a fixed array compiled into the library
// instead of a buffer owned by a context.
//
// The arithmetic is that of DOTPRODUCT in the reference's opern vocabulary
// (src/util/arraymath.h:230-299): each product is formed in FP32 and the sum
// is carried in FP64.  The reduction is deterministic but chunked differently
// from seis_fd_vec_dot, so the two agree to FP64 rounding, not bit for bit.
#include <cuda_runtime.h>

#include <mutex>
#include <stdarg.h>
#include <stdio.h>

#include "fd_internal.h"
#include "seis_fd.h"

namespace seis {
namespace {

constexpr int NA_VT = 256;                   // threads per CTA
constexpr int NA_PER = 16;                   // elements per thread
constexpr int NA_CHUNK = NA_VT * NA_PER;     // elements per CTA (one partial sum)
constexpr int NA_MAX_PARTS = 16384;          // partial sums the scratch holds
static_assert((size_t)NA_MAX_PARTS * NA_CHUNK == SEIS_DOT_NOALLOC_MAX_N,
              "the header's maximum must match the scratch capacity");

// The scratch: NA_MAX_PARTS doubles (128 KiB), held by every GPU that loads
// the library until the process exits.  Every call writes each slot it later
// reads, so nothing in it has to start at zero.
static __device__ __align__(256) double g_dot_scratch[NA_MAX_PARTS];

__device__ __forceinline__ double na_block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  v = 0.0;
  if (warp == 0) {
    v = lane < NA_VT / 32 ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  return v;
}

// one partial sum per CTA over a fixed chunk of NA_CHUNK elements
__global__ void __launch_bounds__(NA_VT) na_dot_chunk_kernel(const float *__restrict__ a,
                                                             const float *__restrict__ b,
                                                             size_t n,
                                                             double *__restrict__ partial) {
  __shared__ double sh[NA_VT / 32];
  const size_t base = (size_t)blockIdx.x * NA_CHUNK + threadIdx.x;
  double acc = 0.0;
#pragma unroll
  for (int j = 0; j < NA_PER; j++) {
    const size_t i = base + (size_t)j * NA_VT;
    if (i < n) acc += (double)(a[i] * b[i]);
  }
  acc = na_block_sum(acc, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// the partial sums added in a fixed order by one CTA
__global__ void __launch_bounds__(NA_VT) na_dot_final_kernel(const double *__restrict__ partial,
                                                             int nparts, double *__restrict__ out) {
  __shared__ double sh[NA_VT / 32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < nparts; i += NA_VT) acc += partial[i];
  acc = na_block_sum(acc, sh);
  if (threadIdx.x == 0) *out = acc;
}

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_setup_mu;
double *g_scratch_ptr[NA_MAX_DEVICES] = {};  // device address of the scratch, per device

int na_error(char *err, size_t err_len, int rc, const char *fmt, ...) {
  if (err && err_len > 0) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, err_len, fmt, ap);
    va_end(ap);
  }
  return rc;
}

}  // namespace
}  // namespace seis

extern "C" int seis_fd_vec_dot_noalloc(const float *d_a, const float *d_b, size_t n,
                                       double *d_out, void *stream, char *err,
                                       size_t err_len) {
  using namespace seis;
  if (err && err_len > 0) err[0] = '\0';
  if (!d_out || (n > 0 && (!d_a || !d_b)))
    return na_error(err, err_len, SEIS_ERR_ARG, "seis_fd_vec_dot_noalloc: null pointer");
  if (n > SEIS_DOT_NOALLOC_MAX_N)
    return na_error(err, err_len, SEIS_ERR_ARG,
                    "seis_fd_vec_dot_noalloc: n = %zu exceeds the maximum of %zu elements "
                    "(the fixed scratch holds %d partial sums of %d elements each)",
                    n, (size_t)SEIS_DOT_NOALLOC_MAX_N, NA_MAX_PARTS, NA_CHUNK);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return na_error(err, err_len, SEIS_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= NA_MAX_DEVICES)
    return na_error(err, err_len, SEIS_ERR_ARG, "device %d beyond the %d supported", dev,
                    NA_MAX_DEVICES);
  double *scratch = nullptr;
  {
    // set-up, once per device, with that device current: the host-side name
    // of the array is not a device address, so look the address up
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_dot_scratch);
      if (e != cudaSuccess)
        return na_error(err, err_len, SEIS_ERR_CUDA, "cudaGetSymbolAddress: %s",
                        cudaGetErrorString(e));
      g_scratch_ptr[dev] = static_cast<double *>(p);
    }
    scratch = g_scratch_ptr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int nparts = (int)((n + NA_CHUNK - 1) / NA_CHUNK);
  if (nparts > 0) na_dot_chunk_kernel<<<nparts, NA_VT, 0, s>>>(d_a, d_b, n, scratch);
  na_dot_final_kernel<<<1, NA_VT, 0, s>>>(scratch, nparts, d_out);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return na_error(err, err_len, SEIS_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
  return SEIS_OK;
}
