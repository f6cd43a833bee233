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
#include <cuda.h>
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

// The array's device address belongs to a CUDA context: each context that
// loads the library (the device's primary context, a context the host
// application made with cuCtxCreate, or the primary context made again after
// cudaDeviceReset) holds its own copy at its own address.  A call outside
// stream capture looks the address up in the current context every time and
// records it here under that context's handle; a call made while its stream
// is capturing (where the lookup, which may load the module, must not run)
// takes the recorded address of the current context, and fails if there is
// none.
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    return cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
                   q == cudaDriverEntryPointSuccess
               ? reinterpret_cast<CtxGetCurrentFn>(p)
               : nullptr;
  }();
  return fn;
}

constexpr int NA_MAX_CONTEXTS = 64;
struct ScratchSlot {
  CUcontext ctx;
  double *ptr;
};
std::mutex g_setup_mu;
ScratchSlot g_slots[NA_MAX_CONTEXTS] = {};
int g_next_slot = 0;

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
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(s, &cap);
  if (e != cudaSuccess)
    return na_error(err, err_len, SEIS_ERR_CUDA, "cudaStreamIsCapturing: %s",
                    cudaGetErrorString(e));
  void *found = nullptr;
  if (cap == cudaStreamCaptureStatusNone) {
    // the host-side name of the array is not a device address: look the
    // address up in the current context (this also makes the device's
    // primary context current on a thread that has none yet)
    e = cudaGetSymbolAddress(&found, g_dot_scratch);
    if (e != cudaSuccess)
      return na_error(err, err_len, SEIS_ERR_CUDA, "cudaGetSymbolAddress: %s",
                      cudaGetErrorString(e));
  }
  CtxGetCurrentFn get = ctx_get_current();
  CUcontext cur = nullptr;
  if (!get || get(&cur) != CUDA_SUCCESS || !cur)
    return na_error(err, err_len, SEIS_ERR_CUDA, "no current CUDA context");
  double *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    int slot = -1;
    for (int i = 0; i < NA_MAX_CONTEXTS; i++)
      if (g_slots[i].ctx == cur) slot = i;
    if (found) {
      if (slot < 0) {
        slot = g_next_slot;
        g_next_slot = (g_next_slot + 1) % NA_MAX_CONTEXTS;
      }
      g_slots[slot] = ScratchSlot{cur, static_cast<double *>(found)};
    } else if (slot < 0) {
      return na_error(err, err_len, SEIS_ERR_STATE,
                      "seis_fd_vec_dot_noalloc: first call in this CUDA context made during "
                      "stream capture; make one call outside capture first");
    }
    scratch = g_slots[slot].ptr;
  }
  const int nparts = (int)((n + NA_CHUNK - 1) / NA_CHUNK);
  if (nparts > 0) na_dot_chunk_kernel<<<nparts, NA_VT, 0, s>>>(d_a, d_b, n, scratch);
  na_dot_final_kernel<<<1, NA_VT, 0, s>>>(scratch, nparts, d_out);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return na_error(err, err_len, SEIS_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
  return SEIS_OK;
}
