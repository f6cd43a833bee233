// Exact-adjoint kernels, built like the fast step kernels (multiply-add
// contraction, approximate division): the adjoint transposes the fast Born
// operator that the LSRTM solver applies, so it carries the same coefficient
// rounding; it has no reference rounding to reproduce.
#define SEIS_NS fast
#include "fd_adjoint.cuh"

namespace seis {
namespace fast {

constexpr size_t ADJ_TILE_SMEM = sizeof(float) * (size_t)(4 * WIDE + NARROW) + 16;
constexpr size_t ADJ_PAD_SMEM = sizeof(float) * (size_t)ADJ_PAD_FLOATS + 16;

cudaError_t configure_adjoint() {
  cudaError_t e = cudaFuncSetAttribute(adj_interior_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)ADJ_TILE_SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(adj_pad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)ADJ_PAD_SMEM);
  return e;
}

cudaError_t launch_adjoint(const ShotDev *d_shots, const Tile *d_tiles, int n_int, int n_pad,
                           const StepArgs &a, int *d_err, cudaStream_t s_int, cudaStream_t s_pad) {
  if (n_int > 0)
    adj_interior_kernel<<<n_int, A_NT_I, ADJ_TILE_SMEM, s_int>>>(d_shots, d_tiles, a, d_err);
  if (n_pad > 0)
    adj_pad_kernel<<<n_pad, A_NT_I, ADJ_PAD_SMEM, s_pad>>>(d_shots, d_tiles + n_int, a, d_err);
  return cudaGetLastError();
}

}  // namespace fast
}  // namespace seis
