// Time-step kernels of the 2-D acoustic FD engine (sm_100a).
//
// One step of a batch is two launches over the tile list plus one over the
// pad cells:
//  * tile_kernel<MODE, TILE_INTERIOR>: tiles whose every cell is a model cell
//    in the 8th-order region; the absorbing blend is the identity there
//    (w = 1, u31 = 0; src/util/fd.cpp:55-56);
//  * tile_kernel<MODE, TILE_PAD>: tiles touching the pad, the frame, the
//    low-order rings or the model edge: the same two-way update (the frame
//    and low-order cells by the per-cell formula), model cells finished as in
//    the interior, and the two-way value u3 of every cell kept in the shot's
//    scratch field;
//  * absorb_kernel<MODE>: every pad cell, the one-way update from u3 and the
//    blend (processBoundary, fd.cpp:1092-1179), elementwise from global
//    memory (no halo exchange, no barrier).
// Tile kernels: one 32 x 64 tile per CTA, 2-D TMA tensor copies of the
// current field (5-column / 8-row halo), the previous field, the velocity and,
// for Born, the perturbation (1-column / 8-row halo) into shared memory (one
// mbarrier, no multicast); each thread owns a 4-row x 2-column micro-tile.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "fd_cell.cuh"

namespace seis {
namespace SEIS_NS {

constexpr int NT_T = 256;          // threads per CTA
constexpr int QZ = TZ / 4;         // row quads per column (16)
constexpr int SR = TZ + 2 * ZM;    // staged rows per column (80)
constexpr int CW_C = TX + 2 * HXC; // staged columns of the current fields (42)
constexpr int CW_P = TX + 2;       // staged columns of the other arrays (34)

// Staged arrays of one tile (one buffer, one tile per CTA: several CTAs per SM
// hide the copy latency).
template <int MODE, int KIND>
struct TCfg {
  static constexpr bool BORN = MODE == MODE_BORN;
  static constexpr int NCUR = BORN ? 2 : 1;   // arrays staged with the wide halo
  static constexpr int NOTH = BORN ? 4 : 2;   // prev, vel [, prev B, dv]
  static constexpr int BUF = (NCUR * CW_C + NOTH * CW_P) * SR;  // floats per buffer
  static constexpr size_t bytes = sizeof(float) * (size_t)BUF + 16;
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

// Accessor of one staged array by padded-grid coordinates.
struct SA {
  const float *s;  // staged column (x0 - halo) row (z0 - ZM)
  int x0h, z0m;    // x0 - halo, z0 - ZM
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
__device__ __forceinline__ void pair_twoway(const SA &C, const SA &P, const SA &V, const ShotDev &g,
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
template <int NTH, int NV>
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

template <int MODE, int KIND>
__global__ void __launch_bounds__(NT_T, 3) tile_kernel(const ShotDev *__restrict__ shots,
                                                       const Tile *__restrict__ tiles, StepArgs a,
                                                       int *__restrict__ err) {
  using C = TCfg<MODE, KIND>;
  constexpr bool BORN = C::BORN;
  constexpr bool PAD = KIND == TILE_PAD;
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

  // staged arrays: cur A [, cur B] (wide halo), then prev A, vel [, prev B, dv]
  auto arr_off = [](int arr) -> int {
    return arr < C::NCUR ? arr * CW_C * SR : C::NCUR * CW_C * SR + (arr - C::NCUR) * CW_P * SR;
  };
  // One 2-D tensor copy per staged array: rows [z0 - ZM, z0 + TZ + ZM) of
  // columns [x0 - halo, x0 + TX + halo), addressed from the allocation start
  // (row + ZM, column + XM), so coordinates are never negative and the row
  // coordinate is a multiple of TZ (16-byte aligned).
  if (tid == 0) {
    fence_proxy_async();
    mbar_expect_tx(bar, (uint32_t)(C::BUF * sizeof(float)));
    const int ra = a.rot % 3, rca = (a.rot + 1) % 3, rb = a.rot_b % 3, rcb = (a.rot_b + 1) % 3;
    int maps[6];
    if (MODE == MODE_RCV) {
      maps[0] = MAP_FB_WIDE + rcb; maps[1] = MAP_FB_NARROW + rb; maps[2] = MAP_VEL;
    } else if (!BORN) {
      maps[0] = MAP_FA_WIDE + rca; maps[1] = MAP_FA_NARROW + ra; maps[2] = MAP_VEL;
    } else {
      maps[0] = MAP_FA_WIDE + rca; maps[1] = MAP_FB_WIDE + rcb; maps[2] = MAP_FA_NARROW + ra;
      maps[3] = MAP_VEL; maps[4] = MAP_FB_NARROW + rb; maps[5] = MAP_DV;
    }
#pragma unroll
    for (int arr = 0; arr < C::NCUR + C::NOTH; arr++) {
      const int col = t.x0 + XM - (arr < C::NCUR ? HXC : 1);
      tma_load_2d(bb + arr_off(arr), g.maps + maps[arr], t.z0, col, bar);
    }
  }
  if (!mbar_wait(bar, 0)) {
    if (tid == 0) atomicExch(err, 1);
    return;
  }

  StepArgs aa = a;
  if (MODE != MODE_RCV && aa.rec_k >= g.nt) aa.rec_k = -1;
  float *na = g.fa[(a.rot + 2) % 3];
  float *nb_ = g.fb[(a.rot_b + 2) % 3];
  float *out_a = MODE == MODE_RCV ? nb_ : na;
  const int x0 = t.x0, z0 = t.z0;
  const int zm = z0 - ZM;
  const SA CA{bb + arr_off(0), x0 - HXC, zm};
  const SA CB{bb + arr_off(BORN ? 1 : 0), x0 - HXC, zm};
  const SA PA{bb + arr_off(C::NCUR), x0 - 1, zm};
  const SA VV{bb + arr_off(C::NCUR + 1), x0 - 1, zm};
  const SA PB{bb + arr_off(BORN ? C::NCUR + 2 : C::NCUR), x0 - 1, zm};
  const SA DV{bb + arr_off(BORN ? C::NCUR + 3 : C::NCUR + 1), x0 - 1, zm};
  const int qz = tid % QZ, cx = tid / QZ;  // micro-tile: rows 4qz.., columns 2cx, 2cx+1
  const int ix = x0 + 2 * cx, iz0 = z0 + 4 * qz;
  const bool record = MODE != MODE_RCV && aa.rec_k >= 0;
  const bool snap = MODE != MODE_RCV && aa.snap_k >= 0 && g.snap != nullptr;

  // Cells within 3 of the grid edge (frame, fd.cpp:1057-1091; low-order rings,
  // :1226-1241) take the general formula.  All threads form them over the
  // tile's edge bands (a cell in two bands is formed twice, to the same
  // value) into the tile's cells of the two-way scratch field, which the
  // cell's own thread reads back after the barrier and then overwrites with
  // the injected value; every other cell takes the 8th-order vector path.  The band pass
  // reads global memory: the frame's normal extrapolation reaches the
  // velocity two columns inside the grid, past the staged one-column halo of
  // a tile that holds only the last column.
  const int xe = PAD ? min(x0 + TX, g.NX) : 0, ze = PAD ? min(z0 + TZ, g.NZ) : 0;
  const bool edge = PAD && (x0 <= 3 || z0 <= 3 || xe - 1 >= g.NX - 4 || ze - 1 >= g.NZ - 4);
  auto near_edge = [&](int cxj, int iz) {
    return min(min(cxj, iz), min(g.NX - 1 - cxj, g.NZ - 1 - iz)) <= 3;
  };
  if (edge) {
    const int ra = a.rot % 3, rb = a.rot_b % 3;
    float *const *FA = MODE == MODE_RCV ? g.fb : g.fa;
    const int rr = MODE == MODE_RCV ? rb : ra;
    const GA GCa{FA[(rr + 1) % 3], g.LDZ}, GPa{FA[rr], g.LDZ}, GV{g.vel, g.LDZ};
    const GA GCb{g.fb[(rb + 1) % 3], g.LDZ}, GPb{g.fb[rb], g.LDZ};
#pragma unroll 1
    for (int b = 0; b < 4; b++) {  // top, bottom, left, right band
      const int bxa = b == 3 ? max(x0, g.NX - 4) : x0, bxb = b == 2 ? min(xe, 4) : xe;
      const int bza = b == 1 ? max(z0, g.NZ - 4) : z0, bzb = b == 0 ? min(ze, 4) : ze;
      const int nr = bzb - bza, nc = bxb - bxa;
      if (nr <= 0 || nc <= 0) continue;
      for (int i = tid; i < nr * nc; i += NT_T) {
        const int cxj = bxa + i / nr, iz = bza + i % nr;
        const size_t at = (size_t)cxj * g.LDZ + iz;
        g.u3s[0][at] = twoway_cell(GCa, GPa, GV, g, cxj, iz);
        if (BORN) g.u3s[1][at] = twoway_cell(GCb, GPb, GV, g, cxj, iz);
      }
    }
  }
  if (PAD) __syncthreads();

  auto in_grid = [&](int cxj, int iz) { return !PAD || (cxj < g.NX && iz < g.NZ); };
  auto model = [&](int cxj, int iz) {
    return !PAD || (cxj >= g.pml && cxj < g.pml + g.nx && iz >= g.pml && iz < g.pml + g.nz);
  };

  // One micro-tile (columns qx, qx+1, rows qz0 .. qz0+3): two-way values,
  // injection, model cells finished (w = 1), every u3 of a pad tile kept.
  // `vec`: all eight cells in the 8th-order region (vector path from shared
  // memory); otherwise cell by cell with the general formula (frame,
  // low-order rings, cells past the grid skipped).  lv/mask: source-term
  // values of the model cells for the snapshot.
  auto quad = [&](int qx, int qz0, bool vec, float (&lv)[8], int (&lx)[8], int (&lz)[8],
                  unsigned &mask) {
    auto twoway = [&](const SA &Cc, const SA &Pp, int f, float4 o[2], float4 cen[2],
                      float4 prv[2], float4 vel[2]) {
      pair_twoway(Cc, Pp, VV, g, qx, qz0, o, cen, prv, vel);
      if (!vec) {  // cells within 3 of the grid edge from the band pass
#pragma unroll
        for (int j = 0; j < 2; j++)
#pragma unroll
          for (int r = 0; r < 4; r++) {
            const int cxj = qx + j, iz = qz0 + r;
            if (in_grid(cxj, iz) && near_edge(cxj, iz))
              set_comp(o[j], r, g.u3s[f][(size_t)cxj * g.LDZ + iz]);
          }
      }
    };
    // a column quad wholly in the grid (or wholly in the model) is stored as
    // one vector; the other cells of a pad tile one by one
    auto quad_in = [&](int cxj) { return !PAD || (cxj < g.NX && qz0 + 3 < g.NZ); };
    auto quad_model = [&](int cxj) {
      return !PAD || (cxj >= g.pml && cxj < g.pml + g.nx && qz0 >= g.pml && qz0 + 3 < g.pml + g.nz);
    };
    int gzq[2];
#pragma unroll
    for (int j = 0; j < 2; j++) {
      int x = qx + j - g.pml;
      gzq[j] = (x >= 0 && x < g.nx) ? g.gz[x] + g.pml : -1;
    }
    float4 o[2], cen[2], prv[2], vel[2];
    twoway(CA, PA, 0, o, cen, prv, vel);
    float4 qs[2] = {make_float4(0.f, 0.f, 0.f, 0.f), make_float4(0.f, 0.f, 0.f, 0.f)};
#pragma unroll
    for (int j = 0; j < 2; j++) {
      const int cxj = qx + j;
      float4 u4 = o[j];
#pragma unroll
      for (int r = 0; r < 4; r++) {
        const int iz = qz0 + r;
        lv[4 * j + r] = 0.0f;
        lx[4 * j + r] = cxj;
        lz[4 * j + r] = iz;
        if (!in_grid(cxj, iz)) continue;
        Coef kk = coef(comp(vel[j], r), g);
        const float u = inject<MODE>(g, aa, cxj, iz, gzq[j], comp(o[j], r), kk.vt2);
        set_comp(u4, r, u);
        if (PAD && !quad_in(cxj)) g.u3s[0][(size_t)cxj * g.LDZ + iz] = u;
        if (!model(cxj, iz)) continue;  // pad cell: finished by absorb_kernel
        const float out = u + 0.0f;
        set_comp(o[j], r, out);
        if (PAD && !quad_model(cxj)) out_a[(size_t)cxj * g.LDZ + iz] = out;
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
            set_comp(qs[j], r, kk.vt2 * lap * vel3 * DV(cxj, iz));
          }
        }
      }
      if (PAD && quad_in(cxj))
        *reinterpret_cast<float4 *>(g.u3s[0] + (size_t)cxj * g.LDZ + qz0) = u4;
      if (quad_model(cxj)) *reinterpret_cast<float4 *>(out_a + (size_t)cxj * g.LDZ + qz0) = o[j];
    }
    if (BORN) {
      float4 ob[2], cb4[2], pb4[2], vb4[2];
      twoway(CB, PB, 1, ob, cb4, pb4, vb4);
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const int cxj = qx + j;
        float4 u4 = ob[j];
#pragma unroll
        for (int r = 0; r < 4; r++) {
          const int iz = qz0 + r;
          if (!in_grid(cxj, iz)) continue;
          const float u = comp(ob[j], r) + comp(qs[j], r);
          set_comp(u4, r, u);
          if (PAD && !quad_in(cxj)) g.u3s[1][(size_t)cxj * g.LDZ + iz] = u;
          if (!model(cxj, iz)) continue;
          const float out = u + 0.0f;
          set_comp(ob[j], r, out);
          if (PAD && !quad_model(cxj)) nb_[(size_t)cxj * g.LDZ + iz] = out;
          if (record && iz == gzq[j]) g.rec[(size_t)aa.rec_k * g.nx + (cxj - g.pml)] = out;
        }
        if (PAD && quad_in(cxj))
          *reinterpret_cast<float4 *>(g.u3s[1] + (size_t)cxj * g.LDZ + qz0) = u4;
        if (quad_model(cxj)) *reinterpret_cast<float4 *>(nb_ + (size_t)cxj * g.LDZ + qz0) = ob[j];
      }
    }
  };

  float lv[8];
  int lx[8], lz[8];
  unsigned mask = 0;
  if (!PAD) {
    float (&l0)[8] = *reinterpret_cast<float(*)[8]>(lv);
    int (&x0_)[8] = *reinterpret_cast<int(*)[8]>(lx);
    int (&z0_)[8] = *reinterpret_cast<int(*)[8]>(lz);
    quad(ix, iz0, true, l0, x0_, z0_, mask);
    if (snap) snap_write<NT_T, 8>(g, aa.snap_k, x0, z0, l0, x0_, z0_, mask, red);
  } else {
    float (&l1)[8] = *reinterpret_cast<float(*)[8]>(lv);
    int (&x1)[8] = *reinterpret_cast<int(*)[8]>(lx);
    int (&z1)[8] = *reinterpret_cast<int(*)[8]>(lz);
    const bool vecq = !edge || (ix >= 4 && ix + 1 <= g.NX - 5 && iz0 >= 4 && iz0 + 3 <= g.NZ - 5);
    if (ix < g.NX && iz0 < g.NZ) quad(ix, iz0, vecq, l1, x1, z1, mask);
    else
#pragma unroll
      for (int k = 0; k < 8; k++) {
        lv[k] = 0.0f;
        lx[k] = ix;
        lz[k] = iz0;
      }
    if (snap) snap_write<NT_T, 8>(g, aa.snap_k, x0, z0, l1, x1, z1, mask, red);
  }
}

// Absorbing boundary of the pad cells: one-way update from the two-way values
// kept by the pad tiles, and the blend (fd.cpp:1092-1179, :55-56).  Each
// thread takes ABS_CPT cells of its chunk (z fastest, stride ABS_NT) and
// forms all of them before storing any, so their loads overlap; every input
// is read-only during the launch.
template <int MODE>
__global__ void __launch_bounds__(ABS_NT) absorb_kernel(const ShotDev *__restrict__ shots,
                                                        const PadChunk *__restrict__ chunks,
                                                        StepArgs a) {
  const PadChunk c = chunks[blockIdx.x];
  const ShotDev &g = shots[c.shot];
  const int ldz = g.LDZ;
  const GA V{g.vel, ldz};
  const int ra = MODE == MODE_RCV ? a.rot_b : a.rot;
  float *const *FA = MODE == MODE_RCV ? g.fb : g.fa;
  const GA UA{g.u3s[0], ldz}, CA{FA[(ra + 1) % 3], ldz}, PA{FA[ra % 3], ldz};
  float *outa = FA[(ra + 2) % 3];
  const int rb = a.rot_b;
  const GA UB{g.u3s[1], ldz}, CB{g.fb[(rb + 1) % 3], ldz}, PB{g.fb[rb % 3], ldz};
  float *outb = g.fb[(rb + 2) % 3];
  float va[ABS_CPT], vb[ABS_CPT];
  size_t off[ABS_CPT];
  bool act[ABS_CPT];
#pragma unroll
  for (int k = 0; k < ABS_CPT; k++) {
    const int flat = threadIdx.x + k * ABS_NT;
    const int col = flat / c.nrows, row = flat - col * c.nrows;
    act[k] = col < c.ncols;
    const int ix = c.x0 + (act[k] ? col : 0), iz = c.z0 + (act[k] ? row : 0);
    off[k] = (size_t)ix * ldz + iz;
    va[k] = vb[k] = 0.0f;
    if (!act[k]) continue;
    va[k] = absorb_cell(UA(ix, iz), UA, CA, PA, V, g, ix, iz);
    if (MODE == MODE_BORN) vb[k] = absorb_cell(UB(ix, iz), UB, CB, PB, V, g, ix, iz);
  }
#pragma unroll
  for (int k = 0; k < ABS_CPT; k++) {
    if (!act[k]) continue;
    outa[off[k]] = va[k];
    if (MODE == MODE_BORN) outb[off[k]] = vb[k];
  }
}

}  // namespace SEIS_NS
}  // namespace seis
