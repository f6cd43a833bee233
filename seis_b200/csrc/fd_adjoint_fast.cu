// Exact-adjoint kernels, built like the fast step kernels (multiply-add
// contraction, approximate division): the adjoint transposes the fast Born
// operator that the LSRTM solver applies, so it carries the same coefficient
// rounding; it has no reference rounding to reproduce.
#define SEIS_NS fast
#define SEIS_FAST_MATH 1
#include "fd_adjoint.cuh"

namespace seis {
namespace fast {

namespace {
// CTAs of the persistent interior kernel: as many as are resident at once
template <int S>
struct AdjLoopGrid {
  static int ctas;
};
template <int S>
int AdjLoopGrid<S>::ctas = 0;

template <int S>
cudaError_t setup_adjoint() {
  cudaError_t e = cudaFuncSetAttribute(adj_interior_kernel<S>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)AGeo<S>::TILE_SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(adj_pad_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)AGeo<S>::PAD_SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(adj_interior_loop_kernel<S>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ALCfg<S>::bytes);
  int dev = 0, nsm = 0, per = 0;
  if (e == cudaSuccess) e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, adj_interior_loop_kernel<S>,
                                                      Geo<S>::NT, ALCfg<S>::bytes);
  if (e == cudaSuccess) AdjLoopGrid<S>::ctas = (per > 0 ? per : 1) * nsm;
  return e;
}

template <int S>
cudaError_t launch_adj(const ShotDev *d_shots, const Tile *d_tiles, int n_int, int n_pad,
                       const StepArgs &a, int *d_err, cudaStream_t s_int, cudaStream_t s_pad) {
  constexpr int NT = Geo<S>::NT;
  // the persistent interior kernel as a.loop says; by default when every CTA
  // gets at least 4 tiles (as the forward step)
  const int G = AdjLoopGrid<S>::ctas;
  if (n_int > 0 && (a.loop > 0 || (a.loop < 0 && n_int >= 4 * G))) {
    adj_interior_loop_kernel<S><<<G < n_int ? G : n_int, NT, ALCfg<S>::bytes, s_int>>>(
        d_shots, d_tiles, n_int, a, d_err);
  } else if (n_int > 0) {
    adj_interior_kernel<S><<<n_int, NT, AGeo<S>::TILE_SMEM, s_int>>>(d_shots, d_tiles, a, d_err);
  }
  if (n_pad > 0)
    adj_pad_kernel<S><<<n_pad, NT, AGeo<S>::PAD_SMEM, s_pad>>>(d_shots, d_tiles + n_int, a,
                                                                d_err);
  return cudaGetLastError();
}
}  // namespace

cudaError_t configure_adjoint() {
  cudaError_t e = setup_adjoint<SHAPE_32x64>();
  if (e == cudaSuccess) e = setup_adjoint<SHAPE_64x32>();
  if (e == cudaSuccess) e = setup_adjoint<SHAPE_16x128>();
  if (e == cudaSuccess) e = setup_adjoint<SHAPE_64x64>();
  if (e == cudaSuccess) e = setup_adjoint<SHAPE_32x32>();
  return e;
}

cudaError_t launch_edge_coef(const ShotDev *d_shots, int nshots, int max_cells, cudaStream_t s) {
  if (nshots <= 0 || max_cells <= 0) return cudaSuccess;
  edge_coef_kernel<<<dim3((max_cells + 255) / 256, nshots), 256, 0, s>>>(d_shots, nshots);
  return cudaGetLastError();
}

cudaError_t launch_adjoint(int shape, const ShotDev *d_shots, const Tile *d_tiles, int n_int,
                           int n_pad, const StepArgs &a, int *d_err, cudaStream_t s_int,
                           cudaStream_t s_pad) {
  switch (shape) {
    case SHAPE_32x64:
      return launch_adj<SHAPE_32x64>(d_shots, d_tiles, n_int, n_pad, a, d_err, s_int, s_pad);
    case SHAPE_64x32:
      return launch_adj<SHAPE_64x32>(d_shots, d_tiles, n_int, n_pad, a, d_err, s_int, s_pad);
    case SHAPE_16x128:
      return launch_adj<SHAPE_16x128>(d_shots, d_tiles, n_int, n_pad, a, d_err, s_int, s_pad);
    case SHAPE_64x64:
      return launch_adj<SHAPE_64x64>(d_shots, d_tiles, n_int, n_pad, a, d_err, s_int, s_pad);
    case SHAPE_32x32:
      return launch_adj<SHAPE_32x32>(d_shots, d_tiles, n_int, n_pad, a, d_err, s_int, s_pad);
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace fast
}  // namespace seis
