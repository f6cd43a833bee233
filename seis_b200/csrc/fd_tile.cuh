// Time-step kernels of the 2-D acoustic FD engine (sm_100a).
//
// One step of a batch is two launches over the tile list, on two streams:
//  * interior_loop_kernel<S, MODE>: tiles whose every cell is a model cell in
//    the 8th-order region, where the absorbing blend is the identity
//    (w = 1, u31 = 0; src/util/fd.cpp:55-56); persistent CTAs, each taking
//    every G-th tile through two shared-memory stages (the tensor copies of
//    the next tile in flight while the current one is computed);
//  * pad_tile_kernel<S, MODE>: every other tile, one per CTA, in one pass:
//    the two-way update (frame and low-order cells by the per-cell formula),
//    injection, the two-way values of the tile and a one-cell halo kept in
//    shared memory, then the one-way update and blend of the pad cells
//    (processBoundary, fd.cpp:1092-1179).
// Tiles are TX x TZ cells (shape S); arrays are staged by 2-D TMA tensor
// copies into shared memory (mbarriers, bounded waits, no multicast); each
// thread owns a 4-row x 2-column micro-tile.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "fd_cell.cuh"

namespace seis {
namespace SEIS_NS {

// Geometry of tile shape S (TileShapeId).
template <int S>
struct Geo {
  static constexpr int TX = shape_tx(S), TZ = shape_tz(S);
  static constexpr int NT = TX * TZ / 8;       // threads per CTA
  static constexpr int QZ = TZ / 4;            // row quads per column
  static constexpr int SR = TZ + 2 * ZM;       // staged rows per column
  static constexpr int CW_C = TX + 2 * HXC;    // staged columns of the current fields
  static constexpr int CW_P = TX + 2;          // staged columns of the other arrays
  static constexpr int U3C = TX + 2;           // pad tiles: two-way values of tile + halo
  static constexpr int U3R = TZ + 8;
  static constexpr int U3N = U3C * U3R;
  static constexpr int NHALO = 2 * (TX + 2) + 2 * TZ;  // halo ring cells of a tile
  static_assert(NT % 32 == 0 && NT <= 1024, "whole warps");
  static_assert(NT * sizeof(int) >= sizeof(ShotDev), "one thread per word of the shot table");
};
// Local names for the geometry of shape S inside a kernel or device function.
#define SEIS_GEO(S)                                                                   \
  using G_ = Geo<S>;                                                                  \
  constexpr int TX = G_::TX, TZ = G_::TZ, NT_T = G_::NT, QZ = G_::QZ, SR = G_::SR;    \
  constexpr int CW_C = G_::CW_C, CW_P = G_::CW_P;                                     \
  (void)TX; (void)TZ; (void)NT_T; (void)QZ; (void)SR; (void)CW_C; (void)CW_P

// CTAs per SM that a kernel's shared memory allows (227 KB per SM, 1 KB
// reserved per CTA), at most `cap`.
constexpr int ctas_fit(size_t bytes, int cap) {
  return (int)((227 * 1024) / (bytes + 1024)) < cap ? (int)((227 * 1024) / (bytes + 1024)) : cap;
}

// Staged arrays of one tile (one buffer, one tile per CTA: several CTAs per SM
// hide the copy latency).
template <int S, int MODE>
struct TCfg {
  using G = Geo<S>;
  static constexpr bool BORN = MODE == MODE_BORN;
  static constexpr int NCUR = BORN ? 2 : 1;   // arrays staged with the wide halo
  static constexpr int NOTH = BORN ? 4 : 2;   // prev, vel [, prev B, dv]
  static constexpr int BUF = (NCUR * G::CW_C + NOTH * G::CW_P) * G::SR;  // floats per buffer
  static constexpr size_t bytes = sizeof(float) * (size_t)BUF + 16;
  // interior tiles: at most 1024 threads per SM for one field (64 registers
  // a thread), 768 for Born's two (85 registers)
  static constexpr int CAP = (BORN ? 768 : 1024) / G::NT;
  static constexpr int MIN_CTAS = ctas_fit(bytes, CAP) > 0 ? ctas_fit(bytes, CAP) : 1;
};

// ---- PTX helpers: mbarrier + bulk asynchronous copy global -> shared
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int c0, int c1,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, "
      "{%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, "
      "0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up after WAIT_LIMIT polls (each poll may suspend the
// thread for a short hardware-defined time).
constexpr int WAIT_LIMIT = 1 << 21;
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  for (int i = 0; i < WAIT_LIMIT; i++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ float comp(const float4 &v, int r) {
  return r == 0 ? v.x : (r == 1 ? v.y : (r == 2 ? v.z : v.w));
}
__device__ __forceinline__ void set_comp(float4 &v, int r, float x) {
  if (r == 0) v.x = x; else if (r == 1) v.y = x; else if (r == 2) v.z = x; else v.w = x;
}

// Accessor of one staged array by padded-grid coordinates (SR staged rows
// per column).
template <int SR>
struct SAT {
  const float *s;  // staged column x0h, row z0m
  int x0h, z0m;    // first staged column and row (the tile's origin less the halo)
  __device__ __forceinline__ float operator()(int ix, int iz) const {
    return s[(ix - x0h) * SR + (iz - z0m)];
  }
  __device__ __forceinline__ float4 quad(int ix, int iz) const {
    return *reinterpret_cast<const float4 *>(s + (ix - x0h) * SR + (iz - z0m));
  }
};

// Injection into the two-way value before the absorbing step: point source
// into field A (fd.cpp:49-51), or receiver data rec*vt2 in receiver mode
// (fd.cpp:673-677).  `gzc` = padded receiver row of the column (-1: none).
template <int MODE>
__device__ __forceinline__ float inject(const ShotDev &g, const StepArgs &a, int ix, int iz,
                                        int gzc, float u3, float vt2) {
  if (MODE != MODE_RCV) {
    if (a.src_k >= 0) {
      if (g.sou) {  // areal source of forwordPlane, fd.cpp:221-225
        if (iz == g.szp && ix >= g.pml && ix < g.pml + g.nx)
          u3 = u3 + vt2 * g.sou[(size_t)a.src_k * g.nx + (ix - g.pml)];
      } else if (ix == g.sxp && iz == g.szp) {
        u3 = u3 + vt2 * g.wav[a.src_k];
      }
    }
  } else if (a.rec_k >= 0 && gzc >= 0) {
    const float r = g.rec[(size_t)a.rec_k * g.nx + (ix - g.pml)];
    if (!g.rcv_dipole) {
      if (iz == gzc) u3 = u3 + r * vt2;
    } else if (iz == gzc) {  // rtm_true, fd.cpp:1003-1008
      u3 = u3 - r * vt2 / g.dz;
    } else if (iz == gzc + 1) {
      u3 = u3 + r * vt2 / g.dz;
    }
  }
  return u3;
}

// Boundary strips per sample: [top 4 x nx][bottom 4 x nx][left 4 x nz]
// [right 4 x nz] (SaveAtBoundary, fd.cpp:1183-1203); a cell can sit in several
// strips when the model is thin.
__device__ __forceinline__ void save_strips(const ShotDev &g, int strip_k, int ix, int iz,
                                            float out) {
  const int x = ix - g.pml, z = iz - g.pml;
  float *dst = g.strips + (size_t)strip_k * g.strip_len;
  if (x >= 0 && x < g.nx) {
    int lt = z, lb = g.nz - 1 - z;
    if (lt >= 0 && lt < LAYERS) dst[lt * g.nx + x] = out;
    if (lb >= 0 && lb < LAYERS) dst[(LAYERS + lb) * g.nx + x] = out;
  }
  if (z >= 0 && z < g.nz) {
    const int base = 2 * LAYERS * g.nx;
    int ll = x, lr = g.nx - 1 - x;
    if (ll >= 0 && ll < LAYERS) dst[base + ll * g.nz + z] = out;
    if (lr >= 0 && lr < LAYERS) dst[base + (LAYERS + lr) * g.nz + z] = out;
  }
}

// 8th-order two-way update of two columns x 4 rows from shared memory
// (fd.cpp:1259-1270): u3 = vvzz uzz + vvxx uxx + 2 cur - prev.
template <class SC, class SO>
__device__ __forceinline__ void pair_twoway(const SC &C, const SO &P, const SO &V, const ShotDev &g,
                                            int ix, int iz0, float4 out[2], float4 cen[2],
                                            float4 prv[2], float4 vel[2]) {
  float4 xm[10];
#pragma unroll
  for (int m = 0; m < 10; m++) xm[m] = C.quad(ix - 4 + m, iz0);
#pragma unroll
  for (int j = 0; j < 2; j++) {
    const float4 za = C.quad(ix + j, iz0 - 4), zc = C.quad(ix + j, iz0 + 4);
    const float4 zb = xm[4 + j];
    const float zz[12] = {za.x, za.y, za.z, za.w, zb.x, zb.y, zb.z, zb.w, zc.x, zc.y, zc.z, zc.w};
    prv[j] = P.quad(ix + j, iz0);
    vel[j] = V.quad(ix + j, iz0);
    cen[j] = zb;
#pragma unroll
    for (int r = 0; r < 4; r++) {
      float uzz = lap8(zz[r], zz[r + 1], zz[r + 2], zz[r + 3], zz[r + 4], zz[r + 5], zz[r + 6],
                       zz[r + 7], zz[r + 8]);
      float uxx = lap8(comp(xm[j], r), comp(xm[j + 1], r), comp(xm[j + 2], r), comp(xm[j + 3], r),
                       comp(xm[j + 4], r), comp(xm[j + 5], r), comp(xm[j + 6], r),
                       comp(xm[j + 7], r), comp(xm[j + 8], r));
      Coef k = coef(comp(vel[j], r), g);
      set_comp(out[j], r, k.vz * uzz + k.vx * uxx + 2.0f * zz[r + 4] - comp(prv[j], r));
    }
  }
}

// Same for one column x 4 rows.
template <class SA>
__device__ __forceinline__ float4 col_twoway(const SA &C, const SA &P, const SA &V, const ShotDev &g,
                                             int ix, int iz0, float4 &cen, float4 &prv,
                                             float4 &vel) {
  float4 xm[9];
#pragma unroll
  for (int m = 0; m < 9; m++) xm[m] = C.quad(ix - 4 + m, iz0);
  const float4 za = C.quad(ix, iz0 - 4), zc = C.quad(ix, iz0 + 4);
  const float4 zb = xm[4];
  const float zz[12] = {za.x, za.y, za.z, za.w, zb.x, zb.y, zb.z, zb.w, zc.x, zc.y, zc.z, zc.w};
  prv = P.quad(ix, iz0);
  vel = V.quad(ix, iz0);
  cen = zb;
  float4 out;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    float uzz = lap8(zz[r], zz[r + 1], zz[r + 2], zz[r + 3], zz[r + 4], zz[r + 5], zz[r + 6],
                     zz[r + 7], zz[r + 8]);
    float uxx = lap8(comp(xm[0], r), comp(xm[1], r), comp(xm[2], r), comp(xm[3], r),
                     comp(xm[4], r), comp(xm[5], r), comp(xm[6], r), comp(xm[7], r),
                     comp(xm[8], r));
    Coef k = coef(comp(vel, r), g);
    set_comp(out, r, k.vz * uzz + k.vx * uxx + 2.0f * zz[r + 4] - comp(prv, r));
  }
  return out;
}

// Write this thread's source-term values (lap of the background field) of
// snapshot `k`: cells (xs[i], zs[i]) where bit i of `mask` is set.  BF16 / FP16
// snapshots carry one power-of-two scale per (snapshot, tile), taken from the
// tile's largest magnitude so that the scaled values lie in [0.5, 1).  Every
// thread of the CTA calls this (it holds block barriers).
template <int NTH, int NV, int TX, int TZ>
__device__ void snap_write(const ShotDev &g, int k, int x0, int z0, const float (&v)[NV],
                           const int (&xs)[NV], const int (&zs)[NV], unsigned mask, float *red) {
  float scale = 1.0f;
  if (g.snap_dtype != SNAP_F32) {
    float m = 0.0f;
#pragma unroll
    for (int i = 0; i < NV; i++)
      if ((mask >> i) & 1u) m = fmaxf(m, fabsf(v[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = m;
    __syncthreads();
    if (warp == 0) {
      m = lane < NTH / 32 ? red[lane] : 0.0f;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
      if (lane == 0) {
        int e = 0;
        frexpf(m, &e);
        // tiny (denormal) maxima would overflow the scale: clamp to 2^126
        float sc = m > 0.0f ? ldexpf(1.0f, min(-e, 126)) : 1.0f;
        red[32] = sc;
        const int ntx = (g.NX + TX - 1) / TX;
        g.snap_scale[(size_t)k * ntx * g.ntz + (x0 / TX) * g.ntz + z0 / TZ] = sc;
      }
    }
    __syncthreads();
    scale = red[32];
  }
  const size_t base = (size_t)k * g.nx * g.nz;
#pragma unroll
  for (int i = 0; i < NV; i++) {
    if (!((mask >> i) & 1u)) continue;
    const size_t idx = base + (size_t)(xs[i] - g.pml) * g.nz + (zs[i] - g.pml);
    const float q = v[i] * scale;
    if (g.snap_dtype == SNAP_F32)
      reinterpret_cast<float *>(g.snap)[idx] = q;
    else if (g.snap_dtype == SNAP_BF16)
      reinterpret_cast<__nv_bfloat16 *>(g.snap)[idx] = __float2bfloat16_rn(q);
    else
      reinterpret_cast<__half *>(g.snap)[idx] = __float2half_rn(q);
  }
}

// Global-memory accessor of one field by padded-grid coordinates.
struct GA {
  const float *p;  // cell (0, 0)
  int ldz;
  __device__ __forceinline__ float operator()(int ix, int iz) const {
    return __ldg(p + (size_t)ix * ldz + iz);
  }
};

// The grid cells of a tile [x0, x0 + TX) x [z0, z0 + TZ) that lie outside a
// rectangle [rx0, rx1) x [rz0, rz1) (the model, or the model less its edge
// cells), enumerated column by column, z fastest, so that the threads of a
// CTA can share them evenly and consecutive threads touch consecutive rows.
// Column indices come from a float reciprocal: for i < 2^13 and column
// lengths of at most 128, (i + 0.5) / len lies at least 0.5 / len = 2^-8 from
// an integer and the rounded product within 2^-10 of it, so its floor is the
// integer quotient.
struct CellList {
  int x0, z0, xe, ze;  // tile cells inside the grid: [x0, xe) x [z0, ze)
  int ma, mb;          // tile columns crossing the rectangle: [ma, mb)
  int top, bot;        // cells of such a column above / below the rectangle
  int cp, cm, n;       // cells per other column, per crossing column, in all
  float rcp, rcm;      // 1 / cp, 1 / cm
  __device__ __forceinline__ CellList(int x0_, int z0_, int xe_, int ze_, int rx0, int rx1,
                                      int rz0, int rz1)
      : x0(x0_), z0(z0_), xe(xe_), ze(ze_) {
    ma = min(max(rx0, x0), xe);
    mb = min(max(rx1, ma), xe);
    top = max(0, min(ze, rz0) - z0);
    bot = max(0, ze - max(z0, rz1));
    if (rz1 <= rz0) top = ze - z0, bot = 0;  // empty rectangle: whole columns
    cp = ze - z0;
    cm = top + bot;
    n = (xe - x0 - (mb - ma)) * cp + (mb - ma) * cm;
    rcp = cp > 0 ? 1.0f / (float)cp : 0.0f;
    rcm = cm > 0 ? 1.0f / (float)cm : 0.0f;
  }
  static __device__ __forceinline__ int quot(int i, float r) {
    return (int)(((float)i + 0.5f) * r);
  }
  __device__ __forceinline__ void cell(int i, int &cx, int &cz) const {
    const int na = (ma - x0) * cp;
    if (i < na) {
      const int q = quot(i, rcp);
      cx = x0 + q;
      cz = z0 + (i - q * cp);
      return;
    }
    i -= na;
    const int nm = (mb - ma) * cm;
    if (i < nm) {
      const int q = quot(i, rcm);
      cx = ma + q;
      const int r = i - q * cm;
      cz = r < top ? z0 + r : ze - bot + (r - top);
      return;
    }
    i -= nm;
    const int q = quot(i, rcp);
    cx = mb + q;
    cz = z0 + (i - q * cp);
  }
};

// Two-way values of a pad tile and its one-cell halo in shared memory:
// columns x0-1 .. x0+TX, rows z0-4 .. z0+TZ+3 (U3R = TZ + 8 rows per column;
// the tile's row quads stay 16-byte aligned; only rows z0-1 .. z0+TZ are
// used).
template <int U3R>
struct UAT {
  float *s;
  int x0, z0;
  __device__ __forceinline__ float &ref(int ix, int iz) const {
    return s[(ix - x0 + 1) * U3R + (iz - z0 + 4)];
  }
  __device__ __forceinline__ float operator()(int ix, int iz) const { return ref(ix, iz); }
};
// Halo cell i of the tile at (x0, z0): the rows above and below the tile
// (TX + 2 cells each, corners included), then the columns left and right.
template <int TX, int TZ>
__device__ __forceinline__ void halo_cell(int i, int x0, int z0, int &hx, int &hz) {
  if (i < 2 * (TX + 2)) {
    hx = x0 - 1 + i % (TX + 2);
    hz = i < TX + 2 ? z0 - 1 : z0 + TZ;
  } else {
    const int j = i - 2 * (TX + 2);
    hx = j < TZ ? x0 - 1 : x0 + TX;
    hz = z0 + j % TZ;
  }
}

template <int S, int MODE>
struct PCfg {
  using G = Geo<S>;
  static constexpr int NF = MODE == MODE_BORN ? 2 : 1;  // fields with two-way arrays
  static constexpr int BUF = TCfg<S, MODE>::BUF;
  static constexpr size_t bytes = sizeof(float) * ((size_t)BUF + (size_t)NF * G::U3N) + 16;
  // Born: at most 512 threads per SM (128 registers a thread), else 1024
  // (64 registers, some spilled: the extra warps pay for them)
  static constexpr int CAP = (MODE == MODE_BORN ? 512 : 1024) / G::NT;
  static constexpr int MIN_CTAS = ctas_fit(bytes, CAP) > 0 ? ctas_fit(bytes, CAP) : 1;
};

// Stage the arrays of one tile with 2-D tensor copies: rows [z0 - ZM, z0 +
// TZ + ZM) of columns [x0 - halo, x0 + TX + halo), addressed from the
// allocation start (row + ZM, column + XM), so coordinates are never negative
// and the row coordinate is a multiple of TZ (16-byte aligned).  Thread 0
// issues the copies; every thread then waits on the mbarrier.
template <int S, int MODE>
__device__ __forceinline__ void issue_tile(const ShotDev &g, const StepArgs &a, int x0, int z0,
                                           float *bb, uint64_t *bar) {
  SEIS_GEO(S);
  using C = TCfg<S, MODE>;
  {
    const int ra = a.rot % 3, rca = (a.rot + 1) % 3, rb = a.rot_b % 3, rcb = (a.rot_b + 1) % 3;
    int maps[6];
    if (MODE == MODE_RCV) {
      maps[0] = MAP_FB_WIDE + rcb; maps[1] = MAP_FB_NARROW + rb; maps[2] = MAP_VEL;
    } else if (!C::BORN) {
      maps[0] = MAP_FA_WIDE + rca; maps[1] = MAP_FA_NARROW + ra; maps[2] = MAP_VEL;
    } else {
      maps[0] = MAP_FA_WIDE + rca; maps[1] = MAP_FB_WIDE + rcb; maps[2] = MAP_FA_NARROW + ra;
      maps[3] = MAP_VEL; maps[4] = MAP_FB_NARROW + rb; maps[5] = MAP_DV;
    }
#pragma unroll
    for (int arr = 0; arr < C::NCUR + C::NOTH; arr++) {
      const int col = x0 + XM - (arr < C::NCUR ? HXC : 1);
      const int off = arr < C::NCUR ? arr * CW_C * SR : C::NCUR * CW_C * SR + (arr - C::NCUR) * CW_P * SR;
      tma_load_2d(bb + off, g.maps + maps[arr], z0, col, bar);
    }
  }
}
template <int S, int MODE>
__device__ __forceinline__ bool stage_tile(const ShotDev &g, const StepArgs &a, int x0, int z0,
                                           float *bb, uint64_t *bar) {
  using C = TCfg<S, MODE>;
  if (threadIdx.x == 0) {
    fence_proxy_async();
    mbar_expect_tx(bar, (uint32_t)(C::BUF * sizeof(float)));
    issue_tile<S, MODE>(g, a, x0, z0, bb, bar);
  }
  return mbar_wait(bar, 0);
}

// The cells of one interior tile (every cell a model cell in the 8th-order
// region, where the absorbing blend is the identity: w = 1, u31 = 0;
// src/util/fd.cpp:55-56) from its staged arrays: the current fields CA, CB
// (with the stencil's halo), previous fields PA, PB, velocity VV and
// perturbation DV; one 4-row x 2-column micro-tile per thread, gzq the padded
// receiver rows of its two columns.  Every thread of the CTA calls this (the
// snapshot holds block barriers).
template <int S, int MODE, class SC, class SO>
__device__ __forceinline__ void interior_cells(const ShotDev &g, const StepArgs &a, int x0, int z0,
                                               const SC &CA, const SC &CB, const SO &PA,
                                               const SO &VV, const SO &PB, const SO &DV,
                                               const int (&gzq)[2], float *red) {
  SEIS_GEO(S);
  constexpr bool BORN = MODE == MODE_BORN;
  StepArgs aa = a;
  if (MODE != MODE_RCV && aa.rec_k >= g.nt) aa.rec_k = -1;
  float *na = g.fa[(a.rot + 2) % 3];
  float *nb_ = g.fb[(a.rot_b + 2) % 3];
  float *out_a = MODE == MODE_RCV ? nb_ : na;
  const int tid = threadIdx.x;
  const int qz = tid % QZ, cx = tid / QZ;  // micro-tile: rows 4qz.., columns 2cx, 2cx+1
  const int ix = x0 + 2 * cx, iz0 = z0 + 4 * qz;
  const bool record = MODE != MODE_RCV && aa.rec_k >= 0;
  const bool snap = MODE != MODE_RCV && aa.snap_k >= 0 && g.snap != nullptr;

  float lv[8];
  int lx[8], lz[8];
  unsigned mask = 0;
  float4 o[2], cen[2], prv[2], vel[2];
  pair_twoway(CA, PA, VV, g, ix, iz0, o, cen, prv, vel);
  float4 qs[2] = {make_float4(0.f, 0.f, 0.f, 0.f), make_float4(0.f, 0.f, 0.f, 0.f)};
#pragma unroll
  for (int j = 0; j < 2; j++) {
    const int cxj = ix + j;
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int iz = iz0 + r;
      lx[4 * j + r] = cxj;
      lz[4 * j + r] = iz;
      Coef kk = coef(comp(vel[j], r), g);
      const float out = inject<MODE>(g, aa, cxj, iz, gzq[j], comp(o[j], r), kk.vt2) + 0.0f;
      set_comp(o[j], r, out);
      if (!BORN && record && iz == gzq[j]) g.rec[(size_t)aa.rec_k * g.nx + (cxj - g.pml)] = out;
      if (MODE != MODE_BORN && aa.strip_k >= 0) save_strips(g, aa.strip_k, cxj, iz, out);
      if (MODE == MODE_MODEL && aa.illum_on) {  // illum, fd.cpp:317-319
        float *ss = g.illum + (size_t)(cxj - g.pml) * g.nz + (iz - g.pml);
        *ss = *ss + out * out;
      }
      lv[4 * j + r] = 0.0f;
      if (BORN || snap) {  // scattering source vt2 lap vel3 dv, fd.cpp:134-139
        float lap = (out + comp(prv[j], r) - 2.0f * comp(cen[j], r)) * g.idt2;
        lv[4 * j + r] = lap;
        mask |= 1u << (4 * j + r);
        if (BORN) {
          float vv = comp(vel[j], r);
          float vel3 = 2.0f / (vv * vv * vv);
          set_comp(qs[j], r, kk.vt2 * lap * vel3 * DV(cxj, iz));
        }
      }
    }
    *reinterpret_cast<float4 *>(out_a + (size_t)cxj * g.LDZ + iz0) = o[j];
  }
  if (BORN) {
    float4 ob[2], cb4[2], pb4[2], vb4[2];
    pair_twoway(CB, PB, VV, g, ix, iz0, ob, cb4, pb4, vb4);
#pragma unroll
    for (int j = 0; j < 2; j++) {
      const int cxj = ix + j;
#pragma unroll
      for (int r = 0; r < 4; r++) {
        const int iz = iz0 + r;
        const float out = comp(ob[j], r) + comp(qs[j], r) + 0.0f;
        set_comp(ob[j], r, out);
        if (record && iz == gzq[j]) g.rec[(size_t)aa.rec_k * g.nx + (cxj - g.pml)] = out;
      }
      *reinterpret_cast<float4 *>(nb_ + (size_t)cxj * g.LDZ + iz0) = ob[j];
    }
  }
  if (snap) snap_write<NT_T, 8, TX, TZ>(g, aa.snap_k, x0, z0, lv, lx, lz, mask, red);
}

// Interior tiles, one per CTA (the tile list's first n_int tiles).
template <int S, int MODE>
__global__ void __launch_bounds__(Geo<S>::NT, TCfg<S, MODE>::MIN_CTAS) tile_kernel(
    const ShotDev *__restrict__ shots, const Tile *__restrict__ tiles, StepArgs a,
    int *__restrict__ err) {
  SEIS_GEO(S);
  using SA = SAT<SR>;
  using C = TCfg<S, MODE>;
  constexpr bool BORN = C::BORN;
  extern __shared__ __align__(128) unsigned char smraw[];
  float *bb = reinterpret_cast<float *>(smraw);
  uint64_t *bar = reinterpret_cast<uint64_t *>(bb + C::BUF);
  __shared__ ShotDev sg;
  __shared__ float red[33];
  const int tid = threadIdx.x;
  const Tile t = tiles[blockIdx.x];
  if (tid < (int)(sizeof(ShotDev) / sizeof(int)))
    reinterpret_cast<int *>(&sg)[tid] = reinterpret_cast<const int *>(shots + t.shot)[tid];
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  const ShotDev &g = sg;
  if (!stage_tile<S, MODE>(g, a, t.x0, t.z0, bb, bar)) {
    if (tid == 0) atomicExch(err, 1);
    return;
  }
  auto arr_off = [](int arr) -> int {
    return arr < C::NCUR ? arr * CW_C * SR : C::NCUR * CW_C * SR + (arr - C::NCUR) * CW_P * SR;
  };
  const int x0 = t.x0, z0 = t.z0, zm = z0 - ZM;
  const SA CA{bb + arr_off(0), x0 - HXC, zm};
  const SA CB{bb + arr_off(BORN ? 1 : 0), x0 - HXC, zm};
  const SA PA{bb + arr_off(C::NCUR), x0 - 1, zm};
  const SA VV{bb + arr_off(C::NCUR + 1), x0 - 1, zm};
  const SA PB{bb + arr_off(BORN ? C::NCUR + 2 : C::NCUR), x0 - 1, zm};
  const SA DV{bb + arr_off(BORN ? C::NCUR + 3 : C::NCUR + 1), x0 - 1, zm};
  const int ix = x0 + 2 * (tid / QZ);
  const int gzq[2] = {g.gz[ix - g.pml] + g.pml, g.gz[ix + 1 - g.pml] + g.pml};
  interior_cells<S, MODE>(g, a, x0, z0, CA, CB, PA, VV, PB, DV, gzq, red);
}

// Persistent interior kernel: CTA b of G takes the interior tiles b, b + G,
// b + 2G, ... through two shared-memory stages, so that the tensor copies of
// its next tile are in flight while the current one is computed.  The
// current fields are staged with an HI-cell halo on every side, the other
// arrays as the tile alone (interior cells read them at the cell only).
template <int S, int MODE>
struct LCfg {
  using G = Geo<S>;
  static constexpr bool BORN = MODE == MODE_BORN;
  static constexpr int NCUR = BORN ? 2 : 1;  // current fields
  static constexpr int NOTH = BORN ? 4 : 2;  // prev, vel [, prev B, dv]
  static constexpr int CW = G::TX + 2 * HI, RW = G::TZ + 2 * HI;
  static constexpr int TILE = G::TX * G::TZ;
  static constexpr int STAGE = NCUR * CW * RW + NOTH * TILE;  // floats
  static constexpr size_t bytes = 2 * sizeof(float) * (size_t)STAGE + 2 * sizeof(uint64_t);
  // static shared memory: two shot tables and the snapshot reduction
  static constexpr size_t static_bytes = 2 * sizeof(ShotDev) + 33 * sizeof(float);
  // at most 512 threads per SM for Born's two fields (128 registers a
  // thread), 1024 for one
  static constexpr int CAP = (BORN ? 512 : 1024) / G::NT;
  static constexpr int MIN_CTAS =
      ctas_fit(bytes + static_bytes, CAP) > 0 ? ctas_fit(bytes + static_bytes, CAP) : 1;
  static_assert((NCUR * CW * RW * sizeof(float)) % 128 == 0 && (TILE * sizeof(float)) % 128 == 0 &&
                    (STAGE * sizeof(float)) % 128 == 0,
                "tensor-copy destinations stay 128-byte aligned");
};

template <int S, int MODE>
__global__ void __launch_bounds__(Geo<S>::NT, LCfg<S, MODE>::MIN_CTAS) interior_loop_kernel(
    const ShotDev *__restrict__ shots, const Tile *__restrict__ tiles, int n, StepArgs a,
    int *__restrict__ err) {
  SEIS_GEO(S);
  using L = LCfg<S, MODE>;
  constexpr bool BORN = L::BORN;
  constexpr int CW = L::CW, RW = L::RW, TILE = L::TILE;
  using SW = SAT<RW>;  // current fields, HI-cell halo
  using ST = SAT<TZ>;  // the other arrays, the tile alone
  extern __shared__ __align__(128) unsigned char smraw[];
  float *stage0 = reinterpret_cast<float *>(smraw);
  uint64_t *bar = reinterpret_cast<uint64_t *>(stage0 + 2 * L::STAGE);
  __shared__ ShotDev sg[2];
  __shared__ int2 sxz[2];  // tile origin of each stage
  __shared__ float red[33];
  __shared__ int s_fail;
  const int tid = threadIdx.x;
  int i = blockIdx.x;
  if (i >= n) return;
  auto load_shot = [&](int st, int ti) {
    const int shot = tiles[ti].shot;
    if (tid < (int)(sizeof(ShotDev) / sizeof(int)))
      reinterpret_cast<int *>(&sg[st])[tid] = reinterpret_cast<const int *>(shots + shot)[tid];
  };
  // thread 0: the tensor copies of tile ti into stage st (row coordinates
  // count from the allocation start, ZM rows above row 0; columns XM to the
  // left of column 0)
  auto issue = [&](int st, int ti) {
    const Tile t = tiles[ti];
    sxz[st] = make_int2(t.x0, t.z0);
    const CUtensorMap *maps = shots[t.shot].maps;
    float *bb = stage0 + st * L::STAGE;
    fence_proxy_async();
    mbar_expect_tx(bar + st, (uint32_t)(L::STAGE * sizeof(float)));
    const int ra = a.rot % 3, rca = (a.rot + 1) % 3, rb = a.rot_b % 3, rcb = (a.rot_b + 1) % 3;
    int cur[2], oth[4];
    if (MODE == MODE_RCV) {
      cur[0] = MAP_FB_HALO + rcb; oth[0] = MAP_FB_TILE + rb; oth[1] = MAP_VEL_TILE;
    } else if (!BORN) {
      cur[0] = MAP_FA_HALO + rca; oth[0] = MAP_FA_TILE + ra; oth[1] = MAP_VEL_TILE;
    } else {
      cur[0] = MAP_FA_HALO + rca; cur[1] = MAP_FB_HALO + rcb;
      oth[0] = MAP_FA_TILE + ra; oth[1] = MAP_VEL_TILE; oth[2] = MAP_FB_TILE + rb; oth[3] = MAP_DV_TILE;
    }
#pragma unroll
    for (int c = 0; c < L::NCUR; c++)
      tma_load_2d(bb + c * CW * RW, maps + cur[c], t.z0 + ZM - HI, t.x0 + XM - HI, bar + st);
#pragma unroll
    for (int o = 0; o < L::NOTH; o++)
      tma_load_2d(bb + L::NCUR * CW * RW + o * TILE, maps + oth[o], t.z0 + ZM, t.x0 + XM, bar + st);
  };
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_init(bar + 1, 1);
    fence_barrier_init();
    s_fail = 0;
  }
  load_shot(0, i);
  __syncthreads();
  if (tid == 0) issue(0, i);
  __syncthreads();  // the first tile's origin
  uint32_t par = 0;  // bit st: parity of the next completion of stage st
  int st = 0;
  const int cxq = 2 * (tid / QZ);
  for (;;) {
    const int next = i + (int)gridDim.x;
    const bool more = next < n;
    if (more) {  // the other stage was released at the end of the last tile
      load_shot(st ^ 1, next);
      if (tid == 0) issue(st ^ 1, next);
    }
    // this tile's receiver rows, loaded while its copies land
    const ShotDev &g = sg[st];
    const int x0 = sxz[st].x, z0 = sxz[st].y;
    const int gzq[2] = {g.gz[x0 + cxq - g.pml] + g.pml, g.gz[x0 + cxq + 1 - g.pml] + g.pml};
    // a wait that gives up leaves garbage in the stage (indices stay in
    // range); the CTA then ends after this tile
    if (!mbar_wait(bar + st, (par >> st) & 1u)) s_fail = 1;
    par ^= 1u << st;
    const float *bb = stage0 + st * L::STAGE;
    const float *ob = bb + L::NCUR * CW * RW;
    const SW CA{bb, x0 - HI, z0 - HI};
    const SW CB{bb + (BORN ? CW * RW : 0), x0 - HI, z0 - HI};
    const ST PA{ob, x0, z0};
    const ST VV{ob + TILE, x0, z0};
    const ST PB{ob + (BORN ? 2 : 0) * TILE, x0, z0};
    const ST DV{ob + (BORN ? 3 : 1) * TILE, x0, z0};
    interior_cells<S, MODE>(g, a, x0, z0, CA, CB, PA, VV, PB, DV, gzq, red);
    __syncthreads();  // stage st, its origin and shot table are free for the tile after next
    if (s_fail) {
      // the copies in flight into the other stage land before the CTA ends
      if (tid == 0) {
        atomicExch(err, 1);
        if (more) mbar_wait(bar + (st ^ 1), (par >> (st ^ 1)) & 1u);
      }
      return;
    }
    if (!more) break;
    i = next;
    st ^= 1;
  }
}

// Pad tiles: tiles with a pad cell, a cell within 3 of the grid edge (frame,
// src/util/fd.cpp:1057-1091; low-order rings, :1226-1241) or a model cell the
// interior tiles do not take.  One pass per step:
//  1. the two-way values (before injection) of the tile's and its halo's
//     cells within 3 of the grid edge, by the per-cell formula over global
//     memory (the frame's normal extrapolation reaches two cells inside),
//     into shared memory;
//  2. the tile's cells: the 8th-order two-way value from shared memory (or
//     the value of step 1), injection (fd.cpp:49-51) and, for Born, the
//     scattering source; model cells are final (w = 1) and stored, every
//     two-way value is kept in shared memory;
//  3. the same for the halo ring (one cell around the tile), which the
//     one-way update of the tile's edge cells reads;
//  4. every pad cell: the one-way update from the two-way values and the
//     blend (processBoundary fd.cpp:1092-1179, :55-56), stored.
// A halo cell's two-way value is formed by the same per-cell arithmetic as
// in the tile that owns it.
// The cells of one pad tile at (x0, z0) from its staged arrays bb (wide
// current fields, narrow previous fields, velocity, perturbation) and the
// two-way scratch u3m; the phases are listed above.  Every thread of the CTA
// calls this (it holds block barriers).
template <int S, int MODE>
__device__ __forceinline__ void pad_cells(const ShotDev &g, const StepArgs &a, int x0, int z0,
                                          const float *bb, float *u3m, float *red) {
  SEIS_GEO(S);
  using SA = SAT<SR>;
  using UA = UAT<G_::U3R>;
  constexpr int U3N = G_::U3N, NHALO = G_::NHALO;
  using C = TCfg<S, MODE>;
  constexpr bool BORN = C::BORN;
  const int tid = threadIdx.x;
  const int NX = g.NX, NZ = g.NZ;
  auto arr_off = [](int arr) -> int {
    return arr < C::NCUR ? arr * CW_C * SR : C::NCUR * CW_C * SR + (arr - C::NCUR) * CW_P * SR;
  };
  StepArgs aa = a;
  if (MODE != MODE_RCV && aa.rec_k >= g.nt) aa.rec_k = -1;
  float *na = g.fa[(a.rot + 2) % 3];
  float *nb_ = g.fb[(a.rot_b + 2) % 3];
  float *out_a = MODE == MODE_RCV ? nb_ : na;
  const int zm = z0 - ZM;
  const SA CA{bb + arr_off(0), x0 - HXC, zm};
  const SA CB{bb + arr_off(BORN ? 1 : 0), x0 - HXC, zm};
  const SA PA{bb + arr_off(C::NCUR), x0 - 1, zm};
  const SA VV{bb + arr_off(C::NCUR + 1), x0 - 1, zm};
  const SA PB{bb + arr_off(BORN ? C::NCUR + 2 : C::NCUR), x0 - 1, zm};
  const SA DV{bb + arr_off(BORN ? C::NCUR + 3 : C::NCUR + 1), x0 - 1, zm};
  const UA UA_{u3m, x0, z0};
  const UA UB_{u3m + (BORN ? U3N : 0), x0, z0};
  const bool record = MODE != MODE_RCV && aa.rec_k >= 0;
  const bool snap = MODE != MODE_RCV && aa.snap_k >= 0 && g.snap != nullptr;
  auto near_edge = [&](int cx, int cz) {
    return min(min(cx, cz), min(NX - 1 - cx, NZ - 1 - cz)) <= 3;
  };
  auto model = [&](int cx, int cz) {
    return cx >= g.pml && cx < g.pml + g.nx && cz >= g.pml && cz < g.pml + g.nz;
  };
  auto rcv_row = [&](int cx) {
    const int x = cx - g.pml;
    return (x >= 0 && x < g.nx) ? g.gz[x] + g.pml : -1;
  };

  // 1. cells of the tile and its halo within 3 of the grid edge (a cell in two
  // bands is formed twice, to the same value)
  const int xa = max(x0 - 1, 0), xb = min(x0 + TX + 1, NX);
  const int za = max(z0 - 1, 0), zb = min(z0 + TZ + 1, NZ);
  const bool edge = xa <= 3 || za <= 3 || xb - 1 >= NX - 4 || zb - 1 >= NZ - 4;
  if (edge) {
    // every read of the band's formulas lies in the staged window, except the
    // frame's normal extrapolation in a tile of at most two grid columns (it
    // reaches the velocity two columns inside, past the one-column halo):
    // such a tile reads global memory
    auto bands = [&](const auto &Ca, const auto &Pa, const auto &Vv, const auto &Cb,
                     const auto &Pb) {
#pragma unroll 1
      for (int b = 0; b < 4; b++) {  // top, bottom, left, right band
        const int bxa = b == 3 ? max(xa, NX - 4) : xa, bxb = b == 2 ? min(xb, 4) : xb;
        const int bza = b == 1 ? max(za, NZ - 4) : za, bzb = b == 0 ? min(zb, 4) : zb;
        const int nr = bzb - bza, nc = bxb - bxa;
        if (nr <= 0 || nc <= 0) continue;
        for (int i = tid; i < nr * nc; i += NT_T) {
          const int cx = bxa + i / nr, cz = bza + i % nr;
          UA_.ref(cx, cz) = twoway_cell(Ca, Pa, Vv, g, cx, cz);
          if (BORN) UB_.ref(cx, cz) = twoway_cell(Cb, Pb, Vv, g, cx, cz);
        }
      }
    };
    if (x0 <= NX - 2) {
      bands(CA, PA, VV, CB, PB);
    } else {
      const int ra = a.rot % 3, rb = a.rot_b % 3;
      float *const *FA = MODE == MODE_RCV ? g.fb : g.fa;
      const int rr = MODE == MODE_RCV ? rb : ra;
      const GA GCa{FA[(rr + 1) % 3], g.LDZ}, GPa{FA[rr], g.LDZ}, GV{g.vel, g.LDZ};
      const GA GCb{g.fb[(rb + 1) % 3], g.LDZ}, GPb{g.fb[rb], g.LDZ};
      bands(GCa, GPa, GV, GCb, GPb);
    }
    __syncthreads();
  }

  // 2. the tile's cells, one 4-row x 2-column micro-tile per thread
  const int qz = tid % QZ, cxp = tid / QZ;
  const int ix = x0 + 2 * cxp, iz0 = z0 + 4 * qz;
  float lv[8];
  int lx[8], lz[8];
  unsigned mask = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    lv[k] = 0.0f;
    lx[k] = ix + k / 4;
    lz[k] = iz0 + k % 4;
  }
  const bool vecq = !edge || (ix >= 4 && ix + 1 <= NX - 5 && iz0 >= 4 && iz0 + 3 <= NZ - 5);
  if (ix < NX && iz0 < NZ) {
    int gzq[2] = {rcv_row(ix), rcv_row(ix + 1)};
    float4 o[2], cen[2], prv[2], vel[2];
    pair_twoway(CA, PA, VV, g, ix, iz0, o, cen, prv, vel);
    if (!vecq)
#pragma unroll
      for (int j = 0; j < 2; j++)
#pragma unroll
        for (int r = 0; r < 4; r++)
          if (ix + j < NX && iz0 + r < NZ && near_edge(ix + j, iz0 + r))
            set_comp(o[j], r, UA_(ix + j, iz0 + r));
    float4 qs[2] = {make_float4(0.f, 0.f, 0.f, 0.f), make_float4(0.f, 0.f, 0.f, 0.f)};
    // the quad's rows inside the grid and inside the model's rows (bit r =
    // row iz0 + r), and per column the cells inside the grid (cin), the model
    // cells (cm) and whether a source or receiver row falls in the quad
    unsigned rin = 0u, rmod = 0u;
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int iz = iz0 + r;
      if (iz < NZ) rin |= 1u << r;
      if (iz < NZ && iz >= g.pml && iz < g.pml + g.nz) rmod |= 1u << r;
    }
    unsigned cin[2], cm[2];
    bool inj[2];
#pragma unroll
    for (int j = 0; j < 2; j++) {
      const int cxj = ix + j;
      const bool colm = cxj < NX && cxj >= g.pml && cxj < g.pml + g.nx;
      cin[j] = cxj < NX ? rin : 0u;
      cm[j] = colm ? rmod : 0u;
      if (MODE != MODE_RCV)
        inj[j] = aa.src_k >= 0 && g.szp >= iz0 && g.szp <= iz0 + 3 &&
                 (g.sou ? colm : cxj == g.sxp);
      else
        inj[j] = aa.rec_k >= 0 && gzq[j] >= iz0 - 1 && gzq[j] <= iz0 + 3;
    }
#pragma unroll
    for (int j = 0; j < 2; j++) {
      const int cxj = ix + j;
      const bool qin = cin[j] == 0xFu, qmod = cm[j] == 0xFu;
      float4 u4 = o[j];
#pragma unroll
      for (int r = 0; r < 4; r++) {
        const int iz = iz0 + r;
        if (!((cin[j] >> r) & 1u)) continue;
        float u = comp(o[j], r);
        if (inj[j]) u = inject<MODE>(g, aa, cxj, iz, gzq[j], u, coef(comp(vel[j], r), g).vt2);
        set_comp(u4, r, u);
        if (!qin) UA_.ref(cxj, iz) = u;
        if (!((cm[j] >> r) & 1u)) continue;  // pad cell: finished in part 4
        const float out = u + 0.0f;
        set_comp(o[j], r, out);
        if (!qmod) out_a[(size_t)cxj * g.LDZ + iz] = out;
        if (!BORN && record && iz == gzq[j])
          g.rec[(size_t)aa.rec_k * g.nx + (cxj - g.pml)] = out;
        if (MODE != MODE_BORN && aa.strip_k >= 0) save_strips(g, aa.strip_k, cxj, iz, out);
        if (MODE == MODE_MODEL && aa.illum_on) {  // illum, fd.cpp:317-319
          float *ss = g.illum + (size_t)(cxj - g.pml) * g.nz + (iz - g.pml);
          *ss = *ss + out * out;
        }
        if (BORN || snap) {  // scattering source vt2 lap vel3 dv, fd.cpp:134-139
          float lap = (out + comp(prv[j], r) - 2.0f * comp(cen[j], r)) * g.idt2;
          lv[4 * j + r] = lap;
          mask |= 1u << (4 * j + r);
          if (BORN) {
            float vv = comp(vel[j], r);
            float vel3 = 2.0f / (vv * vv * vv);
            const float vt2 = coef(vv, g).vt2;
            set_comp(qs[j], r, vt2 * lap * vel3 * DV(cxj, iz));
          }
        }
      }
      if (qin) *reinterpret_cast<float4 *>(&UA_.ref(cxj, iz0)) = u4;
      if (qmod) *reinterpret_cast<float4 *>(out_a + (size_t)cxj * g.LDZ + iz0) = o[j];
    }
    if (BORN) {
      float4 ob[2], cb4[2], pb4[2], vb4[2];
      pair_twoway(CB, PB, VV, g, ix, iz0, ob, cb4, pb4, vb4);
      if (!vecq)
#pragma unroll
        for (int j = 0; j < 2; j++)
#pragma unroll
          for (int r = 0; r < 4; r++)
            if (ix + j < NX && iz0 + r < NZ && near_edge(ix + j, iz0 + r))
              set_comp(ob[j], r, UB_(ix + j, iz0 + r));
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const int cxj = ix + j;
        const bool qin = cin[j] == 0xFu, qmod = cm[j] == 0xFu;
        float4 u4 = ob[j];
#pragma unroll
        for (int r = 0; r < 4; r++) {
          const int iz = iz0 + r;
          if (!((cin[j] >> r) & 1u)) continue;
          const float u = comp(ob[j], r) + comp(qs[j], r);
          set_comp(u4, r, u);
          if (!qin) UB_.ref(cxj, iz) = u;
          if (!((cm[j] >> r) & 1u)) continue;
          const float out = u + 0.0f;
          set_comp(ob[j], r, out);
          if (!qmod) nb_[(size_t)cxj * g.LDZ + iz] = out;
          if (record && iz == gzq[j]) g.rec[(size_t)aa.rec_k * g.nx + (cxj - g.pml)] = out;
        }
        if (qin) *reinterpret_cast<float4 *>(&UB_.ref(cxj, iz0)) = u4;
        if (qmod) *reinterpret_cast<float4 *>(nb_ + (size_t)cxj * g.LDZ + iz0) = ob[j];
      }
    }
  }

  // 3. the halo ring: the same two-way values, injection and scattering
  // source, for the halo cells next to a pad cell of the tile (the one-way
  // update reads its neighbours within one cell; zero elsewhere, where
  // nothing reads them)
  const int xe = min(x0 + TX, NX), ze = min(z0 + TZ, NZ);
  auto tile_pad = [&](int cx, int cz) {
    return cx >= x0 && cx < xe && cz >= z0 && cz < ze && !model(cx, cz);
  };
  for (int i = tid; i < NHALO; i += NT_T) {
    int hx, hz;
    halo_cell<TX, TZ>(i, x0, z0, hx, hz);
    bool read = false;
    if (i < 2 * (TX + 2)) {  // row above / below: the tile row next to it
      const int zz = hz < z0 ? z0 : ze - 1;
      read = tile_pad(hx - 1, zz) || tile_pad(hx, zz) || tile_pad(hx + 1, zz);
    } else {  // column left / right
      const int xx = hx < x0 ? x0 : xe - 1;
      read = tile_pad(xx, hz - 1) || tile_pad(xx, hz) || tile_pad(xx, hz + 1);
    }
    if (!read || hx < 0 || hz < 0 || hx >= NX || hz >= NZ) {
      UA_.ref(hx, hz) = 0.0f;
      if (BORN) UB_.ref(hx, hz) = 0.0f;
      continue;
    }
    const bool ne = near_edge(hx, hz);
    const float va = VV(hx, hz);
    float ua = ne ? UA_(hx, hz) : twoway_cell(CA, PA, VV, g, hx, hz);
    const Coef kk = coef(va, g);
    ua = inject<MODE>(g, aa, hx, hz, rcv_row(hx), ua, kk.vt2);
    UA_.ref(hx, hz) = ua;
    if (BORN) {
      float ub = ne ? UB_(hx, hz) : twoway_cell(CB, PB, VV, g, hx, hz);
      float q = 0.0f;
      if (model(hx, hz)) {
        const float out = ua + 0.0f;
        const float lap = (out + PA(hx, hz) - 2.0f * CA(hx, hz)) * g.idt2;
        const float vel3 = 2.0f / (va * va * va);
        q = kk.vt2 * lap * vel3 * DV(hx, hz);
      }
      UB_.ref(hx, hz) = ub + q;
    }
  }
  // snapshot of the model cells' source terms (holds block barriers), then
  // every two-way value of the tile and halo is in shared memory
  if (snap) snap_write<NT_T, 8, TX, TZ>(g, aa.snap_k, x0, z0, lv, lx, lz, mask, red);
  __syncthreads();

  // 4. pad cells: one-way update and blend, the tile's pad cells shared
  // evenly by all threads
  const CellList pads(x0, z0, min(x0 + TX, NX), min(z0 + TZ, NZ), g.pml, g.pml + g.nx, g.pml,
                      g.pml + g.nz);
  for (int i = tid; i < pads.n; i += NT_T) {
    int cxj, iz;
    pads.cell(i, cxj, iz);
    const size_t at = (size_t)cxj * g.LDZ + iz;
    const Absorb q = absorb_geom(VV, g, cxj, iz);
    out_a[at] = absorb_apply(q, UA_(cxj, iz), UA_, CA, PA, g, cxj, iz);
    if (BORN) nb_[at] = absorb_apply(q, UB_(cxj, iz), UB_, CB, PB, g, cxj, iz);
  }
}

template <int S, int MODE>
__global__ void __launch_bounds__(Geo<S>::NT, PCfg<S, MODE>::MIN_CTAS) pad_tile_kernel(
    const ShotDev *__restrict__ shots, const Tile *__restrict__ tiles, StepArgs a,
    int *__restrict__ err) {
  SEIS_GEO(S);
  using C = TCfg<S, MODE>;
  extern __shared__ __align__(128) unsigned char smraw[];
  float *bb = reinterpret_cast<float *>(smraw);
  float *u3m = bb + C::BUF;
  uint64_t *bar = reinterpret_cast<uint64_t *>(u3m + PCfg<S, MODE>::NF * G_::U3N);
  __shared__ ShotDev sg;
  __shared__ float red[33];
  const int tid = threadIdx.x;
  const Tile t = tiles[blockIdx.x];
  if (tid < (int)(sizeof(ShotDev) / sizeof(int)))
    reinterpret_cast<int *>(&sg)[tid] = reinterpret_cast<const int *>(shots + t.shot)[tid];
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (!stage_tile<S, MODE>(sg, a, t.x0, t.z0, bb, bar)) {
    if (tid == 0) atomicExch(err, 1);
    return;
  }
  pad_cells<S, MODE>(sg, a, t.x0, t.z0, bb, u3m, red);
}

}  // namespace SEIS_NS
}  // namespace seis
