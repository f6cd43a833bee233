// Launchers of the tile step kernel; included once per build flavour with
// SEIS_NS set (exact / fast).
#pragma once
#include "fd_tile.cuh"

namespace seis {
namespace SEIS_NS {

namespace {
template <int MODE>
cudaError_t setup() {
  cudaError_t e = cudaFuncSetAttribute(tile_kernel<MODE, TILE_INTERIOR>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)TCfg<MODE, TILE_INTERIOR>::bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(pad_tile_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)PCfg<MODE>::bytes);
  return e;
}

// Interior tiles on s_int, pad tiles on s_pad (concurrently).
template <int MODE>
cudaError_t launch_t(const ShotDev *d_shots, const Tile *d_tiles, int n_int, int n_pad,
                     const StepArgs &a, int *d_err, cudaStream_t s_int, cudaStream_t s_pad) {
  if (n_int > 0)
    tile_kernel<MODE, TILE_INTERIOR><<<n_int, NT_T, TCfg<MODE, TILE_INTERIOR>::bytes, s_int>>>(
        d_shots, d_tiles, a, d_err);
  if (n_pad > 0)
    pad_tile_kernel<MODE><<<n_pad, NT_T, PCfg<MODE>::bytes, s_pad>>>(d_shots, d_tiles + n_int, a,
                                                                     d_err);
  return cudaGetLastError();
}
}  // namespace

cudaError_t configure() {
  cudaError_t e = setup<MODE_MODEL>();
  if (e == cudaSuccess) e = setup<MODE_RCV>();
  if (e == cudaSuccess) e = setup<MODE_BORN>();
  return e;
}

cudaError_t launch_step(int mode, const ShotDev *d_shots, const Tile *d_tiles, int n_int,
                        int n_pad, int num_sms, const StepArgs &a, int *d_err, cudaStream_t s_int,
                        cudaStream_t s_pad) {
  switch (mode) {
    case MODE_MODEL:
      return launch_t<MODE_MODEL>(d_shots, d_tiles, n_int, n_pad, a, d_err, s_int, s_pad);
    case MODE_RCV:
      return launch_t<MODE_RCV>(d_shots, d_tiles, n_int, n_pad, a, d_err, s_int, s_pad);
    case MODE_BORN:
      return launch_t<MODE_BORN>(d_shots, d_tiles, n_int, n_pad, a, d_err, s_int, s_pad);
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace SEIS_NS
}  // namespace seis
