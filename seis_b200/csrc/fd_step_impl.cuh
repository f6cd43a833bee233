// Launchers of the tile step kernel; included once per build flavour with
// SEIS_NS set (exact / fast).
#pragma once
#include "fd_tile.cuh"

namespace seis {
namespace SEIS_NS {

namespace {
// CTAs of the persistent interior kernel: as many as are resident at once
template <int S, int MODE>
struct LoopGrid {
  static int ctas;
};
template <int S, int MODE>
int LoopGrid<S, MODE>::ctas = 0;

template <int S, int MODE>
cudaError_t setup() {
  cudaError_t e = cudaFuncSetAttribute(tile_kernel<S, MODE>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)TCfg<S, MODE>::bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(pad_tile_kernel<S, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)PCfg<S, MODE>::bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(interior_loop_kernel<S, MODE>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)LCfg<S, MODE>::bytes);
  int dev = 0, nsm = 0, per = 0;
  if (e == cudaSuccess) e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, interior_loop_kernel<S, MODE>,
                                                      Geo<S>::NT, LCfg<S, MODE>::bytes);
  if (e == cudaSuccess) LoopGrid<S, MODE>::ctas = (per > 0 ? per : 1) * nsm;
  return e;
}

template <int S>
cudaError_t setup_shape() {
  cudaError_t e = setup<S, MODE_MODEL>();
  if (e == cudaSuccess) e = setup<S, MODE_RCV>();
  if (e == cudaSuccess) e = setup<S, MODE_BORN>();
  return e;
}

// Interior tiles on s_int, pad tiles (one CTA each) on s_pad.  The interior
// kernel is the persistent one as a.loop says; by default when each of its
// CTAs gets at least LOOP_MIN_TILES tiles (its double buffering pays, and the
// last round of tiles is a small part of the launch).
constexpr int LOOP_MIN_TILES = 4;
template <int S, int MODE>
cudaError_t launch_t(const ShotDev *d_shots, const Tile *d_tiles, int n_int, int n_pad,
                     const StepArgs &a, int *d_err, cudaStream_t s_int, cudaStream_t s_pad) {
  constexpr int NT = Geo<S>::NT;
  const int G = LoopGrid<S, MODE>::ctas;
  if (n_int > 0 && (a.loop > 0 || (a.loop < 0 && n_int >= LOOP_MIN_TILES * G))) {
    interior_loop_kernel<S, MODE><<<G < n_int ? G : n_int, NT, LCfg<S, MODE>::bytes, s_int>>>(
        d_shots, d_tiles, n_int, a, d_err);
  } else if (n_int > 0) {
    tile_kernel<S, MODE><<<n_int, NT, TCfg<S, MODE>::bytes, s_int>>>(d_shots, d_tiles, a, d_err);
  }
  if (n_pad > 0)
    pad_tile_kernel<S, MODE><<<n_pad, NT, PCfg<S, MODE>::bytes, s_pad>>>(d_shots, d_tiles + n_int,
                                                                       a, d_err);
  return cudaGetLastError();
}

template <int S>
cudaError_t launch_mode(int mode, const ShotDev *d_shots, const Tile *d_tiles, int n_int,
                        int n_pad, const StepArgs &a, int *d_err, cudaStream_t s_int,
                        cudaStream_t s_pad) {
  switch (mode) {
    case MODE_MODEL:
      return launch_t<S, MODE_MODEL>(d_shots, d_tiles, n_int, n_pad, a, d_err, s_int, s_pad);
    case MODE_RCV:
      return launch_t<S, MODE_RCV>(d_shots, d_tiles, n_int, n_pad, a, d_err, s_int, s_pad);
    case MODE_BORN:
      return launch_t<S, MODE_BORN>(d_shots, d_tiles, n_int, n_pad, a, d_err, s_int, s_pad);
    default:
      return cudaErrorInvalidValue;
  }
}
}  // namespace

cudaError_t configure() {
  cudaError_t e = setup_shape<SHAPE_32x64>();
  if (e == cudaSuccess) e = setup_shape<SHAPE_64x32>();
  if (e == cudaSuccess) e = setup_shape<SHAPE_16x128>();
  if (e == cudaSuccess) e = setup_shape<SHAPE_64x64>();
  if (e == cudaSuccess) e = setup_shape<SHAPE_32x32>();
  return e;
}

cudaError_t launch_step(int mode, const ShotDev *d_shots, const Tile *d_tiles, int n_int,
                        int n_pad, int shape, const StepArgs &a, int *d_err, cudaStream_t s_int,
                        cudaStream_t s_pad) {
  switch (shape) {
    case SHAPE_32x64:
      return launch_mode<SHAPE_32x64>(mode, d_shots, d_tiles, n_int, n_pad, a, d_err, s_int, s_pad);
    case SHAPE_64x32:
      return launch_mode<SHAPE_64x32>(mode, d_shots, d_tiles, n_int, n_pad, a, d_err, s_int, s_pad);
    case SHAPE_16x128:
      return launch_mode<SHAPE_16x128>(mode, d_shots, d_tiles, n_int, n_pad, a, d_err, s_int, s_pad);
    case SHAPE_64x64:
      return launch_mode<SHAPE_64x64>(mode, d_shots, d_tiles, n_int, n_pad, a, d_err, s_int, s_pad);
    case SHAPE_32x32:
      return launch_mode<SHAPE_32x32>(mode, d_shots, d_tiles, n_int, n_pad, a, d_err, s_int, s_pad);
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace SEIS_NS
}  // namespace seis
