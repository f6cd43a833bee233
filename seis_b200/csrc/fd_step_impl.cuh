// Launchers of the tile step kernel; included once per build flavour with
// SEIS_NS set (exact / fast).
#pragma once
#include "fd_tile.cuh"

namespace seis {
namespace SEIS_NS {

namespace {
int g_ctas[3][2] = {{0, 0}, {0, 0}, {0, 0}};

template <int MODE, int KIND>
cudaError_t setup() {
  cudaError_t e = cudaFuncSetAttribute(tile_kernel<MODE, KIND>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)TCfg<MODE, KIND>::bytes);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g_ctas[MODE][KIND], tile_kernel<MODE, KIND>,
                                                      nthreads<KIND>(), TCfg<MODE, KIND>::bytes);
  return e;
}

template <int MODE>
cudaError_t launch_t(const ShotDev *d_shots, const Tile *d_tiles, int n_int, int n_pad,
                     int num_sms, const StepArgs &a, int *d_err, cudaStream_t s_int,
                     cudaStream_t s_pad) {
  if (n_int > 0)
    tile_kernel<MODE, TILE_INTERIOR>
        <<<n_int, nthreads<TILE_INTERIOR>(), TCfg<MODE, TILE_INTERIOR>::bytes, s_int>>>(
        d_shots, d_tiles, n_int, a, d_err);
  if (n_pad > 0) {
    int grid = num_sms * (g_ctas[MODE][TILE_PAD] > 0 ? g_ctas[MODE][TILE_PAD] : 1);
    grid = grid < n_pad ? grid : n_pad;
    tile_kernel<MODE, TILE_PAD><<<grid, nthreads<TILE_PAD>(), TCfg<MODE, TILE_PAD>::bytes, s_pad>>>(
        d_shots, d_tiles + n_int, n_pad, a, d_err);
  }
  return cudaGetLastError();
}
}  // namespace

cudaError_t configure() {
  cudaError_t e = setup<MODE_MODEL, TILE_INTERIOR>();
  if (e == cudaSuccess) e = setup<MODE_MODEL, TILE_PAD>();
  if (e == cudaSuccess) e = setup<MODE_RCV, TILE_INTERIOR>();
  if (e == cudaSuccess) e = setup<MODE_RCV, TILE_PAD>();
  if (e == cudaSuccess) e = setup<MODE_BORN, TILE_INTERIOR>();
  if (e == cudaSuccess) e = setup<MODE_BORN, TILE_PAD>();
  return e;
}

cudaError_t launch_step(int mode, const ShotDev *d_shots, const Tile *d_tiles, int n_int,
                        int n_pad, int num_sms, const StepArgs &a, int *d_err, cudaStream_t s_int,
                        cudaStream_t s_pad) {
  switch (mode) {
    case MODE_MODEL:
      return launch_t<MODE_MODEL>(d_shots, d_tiles, n_int, n_pad, num_sms, a, d_err, s_int, s_pad);
    case MODE_RCV:
      return launch_t<MODE_RCV>(d_shots, d_tiles, n_int, n_pad, num_sms, a, d_err, s_int, s_pad);
    case MODE_BORN:
      return launch_t<MODE_BORN>(d_shots, d_tiles, n_int, n_pad, num_sms, a, d_err, s_int, s_pad);
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace SEIS_NS
}  // namespace seis
