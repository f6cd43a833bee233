// Time-step kernel of the 2-D acoustic FD engine (sm_100a): persistent CTAs
// over a tile list, double-buffered bulk-copy staging.
//
// One launch advances every shot of a batch by one time step.  The padded grid
// of every shot is cut into TX x TZ tiles; each persistent CTA walks the tile
// list with stride gridDim.x.  While it computes tile i, the column segments of
// tile i+1 (current field with a 5-column / 8-row halo; previous field,
// velocity and -- for Born -- perturbation with a 1-column / 8-row halo) are in
// flight into the other shared-memory buffer as 2-D TMA tensor copies
// (cp.async.bulk.tensor, one per array, one mbarrier per buffer, no multicast).
//
// Per tile, two paths (uniform per CTA):
//  * interior tiles (every cell inside the model and in the 8th-order region):
//    vector two-way update from shared memory; the absorbing blend is the
//    identity there (w = 1, u31 = 0; src/util/fd.cpp:55-56);
//  * pad tiles: the two-way field on tile + 1 halo into shared memory (frame,
//    low-order rings and injections included), then the one-way update and
//    blend per pad cell (processBoundary, fd.cpp:1053-1180).
// Each thread owns a 4-row x 2-column micro-tile.  Cells are evaluated with
// the per-cell formulas of fd_cell.cuh.
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
constexpr int U3R = TZ + 2, U3C = TX + 2;

// KIND = TILE_INTERIOR: one interior tile per CTA, one staging buffer (many
// CTAs per SM hide the copy latency).  KIND = TILE_PAD: persistent CTAs over
// the pad tiles, two staging buffers (tile i+1 in flight while tile i computes).
template <int MODE, int KIND>
struct TCfg {
  static constexpr bool BORN = MODE == MODE_BORN;
  static constexpr int NCUR = BORN ? 2 : 1;   // arrays staged with the wide halo
  static constexpr int NOTH = BORN ? 4 : 2;   // prev, vel [, prev B, dv]
  static constexpr int BUF = (NCUR * CW_C + NOTH * CW_P) * SR;  // floats per buffer
  static constexpr int NBUF = KIND == TILE_PAD ? 2 : 1;
  static constexpr int NU3 = KIND == TILE_PAD ? (BORN ? 2 : 1) : 0;
  static constexpr size_t bytes =
      sizeof(float) * (size_t)(NBUF * BUF + NU3 * U3R * U3C) + 16 * 2;
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

struct U3Tile {  // two-way field on tile + 1 halo
  float *s;
  int x0, z0;
  __device__ __forceinline__ float &operator()(int ix, int iz) const {
    return s[(ix - x0 + 1) * U3R + (iz - z0 + 1)];
  }
};

// Injection into the two-way value before the absorbing step: point source
// into field A (fd.cpp:49-51), or receiver data rec*vt2 in receiver mode
// (fd.cpp:673-677).  `gzc` = padded receiver row of the column (-1: none).
template <int MODE>
__device__ __forceinline__ float inject(const ShotDev &g, const StepArgs &a, int ix, int iz,
                                        int gzc, float u3, float vt2) {
  if (MODE != MODE_RCV) {
    if (a.src_k >= 0 && ix == g.sxp && iz == g.szp) u3 = u3 + vt2 * g.wav[a.src_k];
  } else if (a.rec_k >= 0 && iz == gzc) {
    u3 = u3 + g.rec[(size_t)a.rec_k * g.nx + (ix - g.pml)] * vt2;
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

// Threads per CTA: interior tiles 256 (4-row x 2-column micro-tiles), pad
// tiles 512 (4-row x 1-column micro-tiles; more warps to cover the latency of
// the scalar absorbing-boundary code).
template <int KIND>
__host__ __device__ constexpr int nthreads() {
  return KIND == TILE_PAD ? 512 : NT_T;
}

template <int MODE, int KIND>
__global__ void __launch_bounds__(nthreads<KIND>(), KIND == TILE_PAD ? 1 : 2) tile_kernel(
    const ShotDev *__restrict__ shots, const Tile *__restrict__ tiles, int ntiles, StepArgs a,
    int *__restrict__ err) {
  using C = TCfg<MODE, KIND>;
  constexpr int NTH = nthreads<KIND>();
  constexpr bool BORN = C::BORN;
  extern __shared__ __align__(128) unsigned char smraw[];
  float *buf0 = reinterpret_cast<float *>(smraw);
  float *su3a = buf0 + C::NBUF * C::BUF;
  float *su3b = su3a + U3R * U3C;
  uint64_t *bar = reinterpret_cast<uint64_t *>(su3a + C::NU3 * U3R * U3C);
  const int tid = threadIdx.x;

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();

  // staged arrays within a buffer: cur A [, cur B] (wide halo), then
  // prev A, vel [, prev B, dv] (narrow halo)
  auto arr_off = [](int arr) -> int {  // float offset of array `arr` in a buffer
    return arr < C::NCUR ? arr * CW_C * SR : C::NCUR * CW_C * SR + (arr - C::NCUR) * CW_P * SR;
  };
  // One 2-D tensor copy per staged array: rows [z0 - ZM, z0 + TZ + ZM) of
  // columns [x0 - halo, x0 + TX + halo), addressed from the allocation start
  // (row + ZM, column + XM), so coordinates are never negative and the row
  // coordinate is a multiple of TZ (16-byte aligned).
  auto issue = [&](int ti, int b) {
    if (tid != 0) return;
    const Tile t = tiles[ti];
    const ShotDev &g = shots[t.shot];
    float *dst0 = buf0 + b * C::BUF;
    fence_proxy_async();
    mbar_expect_tx(&bar[b], (uint32_t)(C::BUF * sizeof(float)));
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
    const int row = t.z0;  // (z0 - ZM) + ZM
#pragma unroll
    for (int arr = 0; arr < C::NCUR + C::NOTH; arr++) {
      const int col = t.x0 + XM - (arr < C::NCUR ? HXC : 1);
      tma_load_2d(dst0 + arr_off(arr), g.maps + maps[arr], row, col, &bar[b]);
    }
  };

  const int qz = tid % QZ, cx = tid / QZ;  // micro-tile: rows 4qz.., columns 2cx, 2cx+1
  int it = 0;
  int ti = blockIdx.x;
  const int stride = C::NBUF == 2 ? (int)gridDim.x : ntiles;  // interior: one tile per CTA
  if (ti < ntiles) issue(ti, 0);
  bool ok = true;
  for (; ti < ntiles; ti += stride, it++) {
    const int b = C::NBUF == 2 ? (it & 1) : 0;
    const int tn = ti + stride;
    if (C::NBUF == 2 && tn < ntiles) issue(tn, b ^ 1);
    if (!mbar_wait(&bar[b], (uint32_t)(C::NBUF == 2 ? ((it >> 1) & 1) : (it & 1)))) {
      ok = false;
      break;
    }
    const Tile t = tiles[ti];
    // the shot descriptor in shared memory: its fields cannot alias the
    // global stores below, so they are loaded once per use site, not reloaded
    __shared__ ShotDev sg;
    __syncthreads();  // the previous tile's readers of sg are done
    if (tid < (int)(sizeof(ShotDev) / sizeof(int)))
      reinterpret_cast<int *>(&sg)[tid] = reinterpret_cast<const int *>(shots + t.shot)[tid];
    __syncthreads();
    const ShotDev &g = sg;
    StepArgs aa = a;
    if (MODE != MODE_RCV && aa.rec_k >= g.nt) aa.rec_k = -1;
    float *na = g.fa[(a.rot + 2) % 3];
    float *nb_ = g.fb[(a.rot_b + 2) % 3];
    float *out_a = MODE == MODE_RCV ? nb_ : na;
    const float *bb = buf0 + b * C::BUF;
    const int x0 = t.x0, z0 = t.z0;
    const int zm = z0 - ZM;
    const SA CA{bb + arr_off(0), x0 - HXC, zm};
    const SA CB{bb + arr_off(BORN ? 1 : 0), x0 - HXC, zm};
    const SA PA{bb + arr_off(C::NCUR), x0 - 1, zm};
    const SA VV{bb + arr_off(C::NCUR + 1), x0 - 1, zm};
    const SA PB{bb + arr_off(BORN ? C::NCUR + 2 : C::NCUR), x0 - 1, zm};
    const SA DV{bb + arr_off(BORN ? C::NCUR + 3 : C::NCUR + 1), x0 - 1, zm};
    const int ix = x0 + 2 * cx, iz0 = z0 + 4 * qz;
    // receiver rows of this thread's two columns
    int gzc[2];
#pragma unroll
    for (int j = 0; j < 2; j++) {
      int x = ix + j - g.pml;
      gzc[j] = (x >= 0 && x < g.nx) ? g.gz[x] + g.pml : -1;
    }
    const bool record = MODE != MODE_RCV && aa.rec_k >= 0;

    const bool snap = MODE != MODE_RCV && aa.snap_k >= 0 && g.snap != nullptr;
    __shared__ float red[33];
    float pout_keep[4] = {0.f, 0.f, 0.f, 0.f};  // pad tiles: this thread's new values
    if (KIND == TILE_INTERIOR) {
      // ---------------- interior tile: every cell 8th order, w = 1
      float4 o[2], cen[2], prv[2], vel[2];
      pair_twoway(CA, PA, VV, g, ix, iz0, o, cen, prv, vel);
      float4 qs[2];
      float lv[8];
      int lx[8], lz[8];
#pragma unroll
      for (int j = 0; j < 2; j++) {
#pragma unroll
        for (int r = 0; r < 4; r++) {
          const int iz = iz0 + r;
          Coef kk = coef(comp(vel[j], r), g);
          float out = inject<MODE>(g, aa, ix + j, iz, gzc[j], comp(o[j], r), kk.vt2) + 0.0f;
          set_comp(o[j], r, out);
          if (!BORN && record && iz == gzc[j])
            g.rec[(size_t)aa.rec_k * g.nx + (ix + j - g.pml)] = out;
          if (MODE == MODE_MODEL && aa.strip_k >= 0) save_strips(g, aa.strip_k, ix + j, iz, out);
          if (BORN || snap) {  // scattering source vt2 lap vel3 dv, fd.cpp:134-139
            float lap = (out + comp(prv[j], r) - 2.0f * comp(cen[j], r)) * g.idt2;
            lv[4 * j + r] = lap;
            lx[4 * j + r] = ix + j;
            lz[4 * j + r] = iz;
            if (BORN) {
              float vv = comp(vel[j], r);
              float vel3 = 2.0f / (vv * vv * vv);
              set_comp(qs[j], r, kk.vt2 * lap * vel3 * DV(ix + j, iz));
            }
          }
        }
        *reinterpret_cast<float4 *>(out_a + (size_t)(ix + j) * g.LDZ + iz0) = o[j];
      }
      if (snap) snap_write<NTH, 8>(g, aa.snap_k, x0, z0, lv, lx, lz, 0xffu, red);
      if (BORN) {
        float4 ob[2], cb4[2], pb4[2], vb4[2];
        pair_twoway(CB, PB, VV, g, ix, iz0, ob, cb4, pb4, vb4);
#pragma unroll
        for (int j = 0; j < 2; j++) {
#pragma unroll
          for (int r = 0; r < 4; r++) {
            float out = (comp(ob[j], r) + comp(qs[j], r)) + 0.0f;
            set_comp(ob[j], r, out);
            if (record && iz0 + r == gzc[j])
              g.rec[(size_t)aa.rec_k * g.nx + (ix + j - g.pml)] = out;
          }
          *reinterpret_cast<float4 *>(nb_ + (size_t)(ix + j) * g.LDZ + iz0) = ob[j];
        }
      }
    } else {
      // ---------------- pad tile: two-way field on tile + 1 halo
      // thread: column x0 + pc, rows pz .. pz+3
      const int pc = tid / QZ, pz = z0 + 4 * (tid % QZ), px = x0 + pc;
      const U3Tile Ua{su3a, x0, z0}, Ub{su3b, x0, z0};
      int gzp;
      {
        int x = px - g.pml;
        gzp = (x >= 0 && x < g.nx) ? g.gz[x] + g.pml : -1;
      }
      // items: NTH body quads (one per thread, its own), 2 x QZ halo-column
      // quads, 2 x (TX + 2) halo-row cells (the halo rows include the four
      // diagonal corners, which the one-way update of a tile-corner strip cell
      // reads)
      constexpr int NITEM = NTH + 2 * QZ + 2 * (TX + 2);
      float4 ua = make_float4(0.f, 0.f, 0.f, 0.f), ub = ua;
      bool body_vec = false;
      for (int item = tid; item < NITEM; item += NTH) {
        int c0, cz0, nrow;
        if (item < NTH) {
          c0 = px; cz0 = pz; nrow = 4;
        } else if (item < NTH + 2 * QZ) {
          int h = item - NTH;
          c0 = h < QZ ? x0 - 1 : x0 + TX;
          cz0 = z0 + 4 * (h % QZ);
          nrow = 4;
        } else {
          int h = item - NTH - 2 * QZ;
          c0 = x0 - 1 + (h % (TX + 2));
          cz0 = h < TX + 2 ? z0 - 1 : z0 + TZ;
          nrow = 1;
        }
        if (c0 < 0 || c0 >= g.NX) continue;
        const bool vec = nrow == 4 && c0 >= 4 && c0 <= g.NX - 5 && cz0 >= 4 && cz0 + 3 <= g.NZ - 5;
        float4 va, vb, cen, prv, vel;
        if (vec) {
          va = col_twoway(CA, PA, VV, g, c0, cz0, cen, prv, vel);
          if (BORN) vb = col_twoway(CB, PB, VV, g, c0, cz0, cen, prv, vel);
        }
        int x = c0 - g.pml;
        const int gz_ = (x >= 0 && x < g.nx) ? g.gz[x] + g.pml : -1;
        for (int r = 0; r < nrow; r++) {
          const int iz = cz0 + r;
          if (iz < 0 || iz >= g.NZ) continue;
          const float v = VV(c0, iz);
          Coef kk = coef(v, g);
          float u = vec ? comp(va, r) : twoway_cell(CA, PA, VV, g, c0, iz);
          u = inject<MODE>(g, aa, c0, iz, gz_, u, kk.vt2);
          Ua(c0, iz) = u;
          if (item < NTH) set_comp(ua, r, u);
          if (BORN) {
            float qv = 0.0f;
            int z = iz - g.pml;
            if (x >= 0 && x < g.nx && z >= 0 && z < g.nz) {  // dv is zero in the pad
              float lap = ((u + 0.0f) + PA(c0, iz) - 2.0f * CA(c0, iz)) * g.idt2;
              float vel3 = 2.0f / (v * v * v);
              qv = kk.vt2 * lap * vel3 * DV(c0, iz);
            }
            float ubv = (vec ? comp(vb, r) : twoway_cell(CB, PB, VV, g, c0, iz)) + qv;
            Ub(c0, iz) = ubv;
            if (item < NTH) set_comp(ub, r, ubv);
          }
        }
        if (item < NTH) body_vec = vec;
      }
      __syncthreads();
      float *pout = pout_keep;
      if (px < g.NX) {
        // a quad wholly inside the model (w = 1, u31 = 0) keeps its two-way
        // values; any other quad goes through the absorbing update per cell
        const bool inside = body_vec && px >= g.pml && px < g.pml + g.nx && pz >= g.pml &&
                            pz + 3 < g.pml + g.nz;
        const size_t off0 = (size_t)px * g.LDZ + pz;
        if (inside) {
          float4 o = ua, ob = ub;
#pragma unroll
          for (int r = 0; r < 4; r++) {
            set_comp(o, r, comp(ua, r) + 0.0f);
            if (BORN) set_comp(ob, r, comp(ub, r) + 0.0f);
          }
          *reinterpret_cast<float4 *>(out_a + off0) = o;
          if (BORN) *reinterpret_cast<float4 *>(nb_ + off0) = ob;
          pout[0] = o.x; pout[1] = o.y; pout[2] = o.z; pout[3] = o.w;
#pragma unroll
          for (int r = 0; r < 4; r++) {
            const int iz = pz + r;
            const float rv = BORN ? comp(ob, r) : comp(o, r);
            if (record && iz == gzp) g.rec[(size_t)aa.rec_k * g.nx + (px - g.pml)] = rv;
            if (MODE == MODE_MODEL && aa.strip_k >= 0) save_strips(g, aa.strip_k, px, iz, comp(o, r));
          }
        } else {
          for (int r = 0; r < 4; r++) {
            const int iz = pz + r;
            if (iz >= g.NZ) break;
            const size_t off = off0 + r;
            float out = absorb_cell(Ua(px, iz), Ua, CA, PA, VV, g, px, iz);
            out_a[off] = out;
            pout[r] = out;
            if (!BORN && record && iz == gzp) g.rec[(size_t)aa.rec_k * g.nx + (px - g.pml)] = out;
            if (MODE == MODE_MODEL && aa.strip_k >= 0) save_strips(g, aa.strip_k, px, iz, out);
            if (BORN) {
              float ob = absorb_cell(Ub(px, iz), Ub, CB, PB, VV, g, px, iz);
              nb_[off] = ob;
              if (record && iz == gzp) g.rec[(size_t)aa.rec_k * g.nx + (px - g.pml)] = ob;
            }
          }
        }
      }
    }
    if (KIND == TILE_PAD && snap) {
      // source-term snapshot of the model-interior cells of this pad tile
      const int pc = tid / QZ, pz = z0 + 4 * (tid % QZ), px = x0 + pc;
      const SA CA2{bb + arr_off(0), x0 - HXC, zm};
      const SA PA2{bb + arr_off(C::NCUR), x0 - 1, zm};
      float lv[4];
      int lx[4], lz[4];
      unsigned mask = 0;
#pragma unroll
      for (int r = 0; r < 4; r++) {
        const int iz = pz + r;
        lx[r] = px;
        lz[r] = iz;
        lv[r] = 0.0f;
        if (px >= g.pml && px < g.pml + g.nx && iz >= g.pml && iz < g.pml + g.nz) {
          lv[r] = (pout_keep[r] + PA2(px, iz) - 2.0f * CA2(px, iz)) * g.idt2;
          mask |= 1u << r;
        }
      }
      snap_write<NTH, 4>(g, aa.snap_k, x0, z0, lv, lx, lz, mask, red);
    }
    __syncthreads();  // buffer b and the u3 tiles are free again
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
    // let every copy already issued land before the CTA's shared memory goes
    // away: the current tile's buffer and, if issued, the next tile's
    if (C::NBUF == 2) {
      mbar_wait(&bar[it & 1], (uint32_t)((it >> 1) & 1));
      if (ti + stride < ntiles) mbar_wait(&bar[(it + 1) & 1], (uint32_t)(((it + 1) >> 1) & 1));
    } else {
      mbar_wait(&bar[0], (uint32_t)(it & 1));
    }
  }
}

}  // namespace SEIS_NS
}  // namespace seis
