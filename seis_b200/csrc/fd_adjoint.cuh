// Exact adjoint of the Born operator (sm_100a).  No counterpart in the
// reference: its adjoint() (src/util/fd.cpp:592-719) is a different imaging
// operator and fails the dot-product test.
//
// One forward step maps (cur, prev) to next through
//   u3  = S(cur, prev)                 two-way update + frame  fd.cpp:1057-1091, :1226-1271
//   u31 = P(u3, cur, prev)             one-way update on the pad rings  :1092-1179
//   nxt = w u3 + (1 - w) u31           blend  :55-56
// and the scattering source enters u3.  With Lk the complete adjoint of the
// field of step k, one reverse step computes
//   mu(L)  = w L + P_u3^T ((1-w) L)          (adjoint of u3: where sources enter)
//   L_k    = S_cur^T mu(L_{k+1}) + P_cur^T((1-w) L_{k+1})
//          - mu(L_{k+2}) + P_prev^T((1-w) L_{k+2}) + R^T d_{k-1-ndel}
// and images grad += w_img * lap_k * mu(L_{k+1}) on the model interior
// (lap_k = source-field second time derivative from the snapshots).
//
// The field kept between steps is M_k = mu(L_k), not L_k; with the ring
// values rho_k = (1 - w) L_k on the pad rings, one reverse step is
//   L_k = S_cur^T M_{k+1} - M_{k+2} + E_k + R^T d,
//   E_k = P_cur^T rho_{k+1} + P_prev^T rho_{k+2},
// and every term is a gather over a fixed neighbourhood summed in a fixed
// order, so the adjoint is bit-for-bit repeatable without atomics.  Two
// launches per step, on two streams:
//  * adj_interior_kernel: tiles with no pad-ring neighbour and every consumer
//    8th order: L = Lz(vz M1) + Lx(vx M1) + 2 M1 - M2 + R^T d;
//  * adj_pad_kernel: the other tiles, in one pass: L of the tile and of its
//    one-cell halo by the same gather over the 8th-order consumers, the
//    low-order and frame consumers (outer 4 cells of the grid) by a per-cell
//    transpose of the two-way formulas, plus E; rho of the ring cells with
//    their one-way coefficients in shared memory; then for the pad and model
//    edge cells M = w L + P_u3^T rho, E of the next step (the cur terms of
//    this step's rho plus the prev terms kept from the last one) and the
//    prev terms kept for the step after.  E alternates between two buffers
//    by step (a tile reads this step's E on its halo while its neighbour
//    writes the next step's).
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "fd_tile.cuh"

namespace seis {
namespace SEIS_NS {

// Adjoint geometry of tile shape S: staged window sizes, the tile + halo
// ring arrays of the pad kernel, halo cells per thread.
template <int S>
struct AGeo {
  using G = Geo<S>;
  static constexpr int WIDE = G::CW_C * G::SR, NARROW = G::CW_P * G::SR;
  static constexpr int RW = G::TZ + 2;
  static constexpr int RN = (G::TX + 2) * RW;
  static constexpr int NHALO = 2 * (G::TX + 2) + 2 * G::TZ;
  static constexpr int HPT = (NHALO + G::NT - 1) / G::NT;  // halo cells per thread
  static constexpr int PAD_FLOATS = 4 * WIDE + NARROW + RN;
  static_assert(5 * RN + G::TX * G::TZ <= 3 * WIDE + NARROW + RN,
                "ring arrays and the tile's L fit over the dead buffers");
  static constexpr size_t TILE_SMEM = sizeof(float) * (size_t)(4 * WIDE + NARROW) + 16;
  static constexpr size_t PAD_SMEM = sizeof(float) * (size_t)PAD_FLOATS + 16;
  static constexpr int MIN_I = ctas_fit(TILE_SMEM, 768 / G::NT) > 0 ? ctas_fit(TILE_SMEM, 768 / G::NT) : 1;
  // pad tiles: up to 768 threads per SM (85 registers a thread, some spilled:
  // the extra warps hide more of the kernel's latency than the spills cost)
  static constexpr int MIN_P = ctas_fit(PAD_SMEM, 768 / G::NT) > 0 ? ctas_fit(PAD_SMEM, 768 / G::NT) : 1;
};
#define SEIS_AGEO(S)                                                        \
  SEIS_GEO(S);                                                              \
  using AG_ = AGeo<S>;                                                      \
  constexpr int WIDE = AG_::WIDE, NARROW = AG_::NARROW, A_NT_I = G_::NT;    \
  (void)WIDE; (void)NARROW; (void)A_NT_I

__device__ __forceinline__ float snap_load(const ShotDev &g, int k, int x, int z) {
  size_t i = (size_t)k * g.nx * g.nz + (size_t)x * g.nz + z;
  switch (g.snap_dtype) {
    case SNAP_F32: return reinterpret_cast<const float *>(g.snap)[i];
    case SNAP_BF16: return __bfloat162float(reinterpret_cast<const __nv_bfloat16 *>(g.snap)[i]);
    case SNAP_F16: return __half2float(reinterpret_cast<const __half *>(g.snap)[i]);
    default: return 0.0f;
  }
}

template <int TX, int TZ>
__device__ __forceinline__ float snap_inv_scale(const ShotDev &g, int k, int x0, int z0) {
  if (g.snap_dtype == SNAP_F32) return 1.0f;
  const int ntx = (g.NX + TX - 1) / TX;
  return 1.0f / g.snap_scale[(size_t)k * ntx * g.ntz + (x0 / TX) * g.ntz + z0 / TZ];
}

// Imaging loads of one column quad (model column x, model rows z .. z+3, the
// rows with bit r of `ok` set): the snapshot values and the accumulator, all
// issued before the quad's arithmetic so that their latencies overlap; the
// matching stores follow in image_store.
struct ImageQuad {
  float lap[4];
  double acc[4];
};
__device__ __forceinline__ void image_load(const ShotDev &g, int k, int x, int z, unsigned ok,
                                           ImageQuad &q) {
#pragma unroll
  for (int r = 0; r < 4; r++) {
    q.lap[r] = 0.0f;
    q.acc[r] = 0.0;
    if ((ok >> r) & 1u) {
      q.lap[r] = snap_load(g, k, x, z + r);
      q.acc[r] = g.grad[(size_t)x * g.nz + z + r];
    }
  }
}
// grad += w lap M1 on the quad's cells (the product rounded to float, then
// accumulated in double)
__device__ __forceinline__ void image_store(const ShotDev &g, int x, int z, unsigned ok,
                                            const ImageQuad &q, float inv_scale, float w,
                                            const float4 &m1) {
#pragma unroll
  for (int r = 0; r < 4; r++)
    if ((ok >> r) & 1u) {
      const float lap = q.lap[r] * inv_scale;
      g.grad[(size_t)x * g.nz + z + r] = q.acc[r] + (double)(w * lap * comp(m1, r));
    }
}

// vz M, vx M of four consecutive cells (coef per cell, as the scalar form)
__device__ __forceinline__ void weigh_quad(const ShotDev &g, const float4 &v, const float4 &l,
                                           float4 &wz, float4 &wx) {
  const Coef c0 = coef(v.x, g), c1 = coef(v.y, g), c2 = coef(v.z, g), c3 = coef(v.w, g);
  wz = make_float4(c0.vz * l.x, c1.vz * l.y, c2.vz * l.z, c3.vz * l.w);
  wx = make_float4(c0.vx * l.x, c1.vx * l.y, c2.vx * l.z, c3.vx * l.w);
}

// ---------------------------------------------------------------- interior
// L_k = Lz(vz M1) + Lx(vx M1) + 2 M1 - M2 + R^T d ; grad += w lap M1.  On these
// tiles M = L (no ring cell within one cell), so the staged arrays (named L1,
// L2 below) hold M_{k+1}, M_{k+2} and the output is L_k = M_k.
template <int S>
__global__ void __launch_bounds__(Geo<S>::NT, AGeo<S>::MIN_I) adj_interior_kernel(
    const ShotDev *__restrict__ shots, const Tile *__restrict__ tiles, StepArgs a,
    int *__restrict__ err) {
  SEIS_AGEO(S);
  using SA = SAT<SR>;
  extern __shared__ __align__(128) unsigned char smraw[];
  float *sL1 = reinterpret_cast<float *>(smraw);  // wide
  float *sV = sL1 + WIDE;                          // wide
  float *sL2 = sV + WIDE;                          // narrow
  float *sWZ = sL2 + NARROW;                       // wide
  float *sWX = sWZ + WIDE;                         // wide
  uint64_t *bar = reinterpret_cast<uint64_t *>(sWX + WIDE);
  const int tid = threadIdx.x;
  const Tile t = tiles[blockIdx.x];
  __shared__ ShotDev sg;
  if (tid < (int)(sizeof(ShotDev) / sizeof(int)))
    reinterpret_cast<int *>(&sg)[tid] = reinterpret_cast<const int *>(shots + t.shot)[tid];
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  const ShotDev &g = sg;
  const int x0 = t.x0, z0 = t.z0;
  if (tid == 0) {
    fence_proxy_async();
    mbar_expect_tx(bar, (uint32_t)((2 * WIDE + NARROW) * sizeof(float)));
    tma_load_2d(sL1, g.maps + MAP_FA_WIDE + (a.rot + 1) % 3, z0, x0 + XM - HXC, bar);
    tma_load_2d(sV, g.maps + MAP_VEL_WIDE, z0, x0 + XM - HXC, bar);
    tma_load_2d(sL2, g.maps + MAP_FA_NARROW + a.rot % 3, z0, x0 + XM - 1, bar);
  }
  if (!mbar_wait(bar, 0)) {
    if (tid == 0) atomicExch(err, 2);
    return;
  }
  // weighted fields vz L1, vx L1 on the staged window, a quad at a time
  static_assert(WIDE % 4 == 0, "whole quads");
  for (int i = 4 * tid; i < WIDE; i += 4 * A_NT_I) {
    float4 wz, wx;
    weigh_quad(g, *reinterpret_cast<const float4 *>(sV + i),
               *reinterpret_cast<const float4 *>(sL1 + i), wz, wx);
    *reinterpret_cast<float4 *>(sWZ + i) = wz;
    *reinterpret_cast<float4 *>(sWX + i) = wx;
  }
  __syncthreads();
  const int zm = z0 - ZM;
  const SA L1{sL1, x0 - HXC, zm}, WZ{sWZ, x0 - HXC, zm}, WX{sWX, x0 - HXC, zm};
  const SA L2{sL2, x0 - 1, zm};
  const int qz = tid % QZ, cx = tid / QZ;
  const int ix = x0 + 2 * cx, iz0 = z0 + 4 * qz;
  float *out = g.fa[(a.rot + 2) % 3];
  float4 xm[10];
#pragma unroll
  for (int m = 0; m < 10; m++) xm[m] = WX.quad(ix - 4 + m, iz0);
  const bool img = a.snap_k >= 0 && g.snap != nullptr;
  float inv_scale = img ? snap_inv_scale<TX, TZ>(g, a.snap_k, x0, z0) : 0.0f;
#pragma unroll
  for (int j = 0; j < 2; j++) {
    const float4 za = WZ.quad(ix + j, iz0 - 4), zb = WZ.quad(ix + j, iz0), zc = WZ.quad(ix + j, iz0 + 4);
    const float zz[12] = {za.x, za.y, za.z, za.w, zb.x, zb.y, zb.z, zb.w, zc.x, zc.y, zc.z, zc.w};
    const float4 l1 = L1.quad(ix + j, iz0), l2 = L2.quad(ix + j, iz0);
    const int x = ix + j - g.pml;
    const int gzr = g.gz[x] + g.pml;
    ImageQuad iq;
    if (img) image_load(g, a.snap_k, x, iz0 - g.pml, 0xFu, iq);
    float4 o;
#pragma unroll
    for (int r = 0; r < 4; r++) {
      float sz_ = lap8(zz[r], zz[r + 1], zz[r + 2], zz[r + 3], zz[r + 4], zz[r + 5], zz[r + 6],
                       zz[r + 7], zz[r + 8]);
      float sx_ = lap8(comp(xm[j], r), comp(xm[j + 1], r), comp(xm[j + 2], r), comp(xm[j + 3], r),
                       comp(xm[j + 4], r), comp(xm[j + 5], r), comp(xm[j + 6], r),
                       comp(xm[j + 7], r), comp(xm[j + 8], r));
      float v = sz_ + sx_ + 2.0f * comp(l1, r) - comp(l2, r);
      if (a.rec_k >= 0 && iz0 + r == gzr) v += g.rec[(size_t)a.rec_k * g.nx + x];
      set_comp(o, r, v);
    }
    if (img) image_store(g, x, iz0 - g.pml, 0xFu, iq, inv_scale, a.img_w, l1);
    *reinterpret_cast<float4 *>(out + (size_t)(ix + j) * g.LDZ + iz0) = o;
  }
}

// Persistent form of the interior kernel: CTA b of G takes the interior tiles
// b, b + G, ... through a ring of NS shared-memory stages (M1 and the velocity
// with an HI-cell halo, M2 as the tile alone), the tensor copies of the next
// NS - 1 tiles in flight while the current one is computed.  vx M1 replaces
// the staged velocity in place; vz M1 has its own array.
template <int S>
struct ALCfg {
  using G = Geo<S>;
  static constexpr int CW = G::TX + 2 * HI, RW = G::TZ + 2 * HI;
  static constexpr int HALO = CW * RW, TILE = G::TX * G::TZ;
  static constexpr int STAGE = 2 * HALO + TILE;  // M1, velocity, M2
  // stages: the next tile's copies in flight (a third stage, two tiles
  // ahead, measured 2% slower)
  static constexpr int NS = 2;
  static constexpr size_t bytes =
      sizeof(float) * (NS * (size_t)STAGE + HALO) + NS * sizeof(uint64_t);
  static constexpr size_t static_bytes = NS * (sizeof(ShotDev) + sizeof(int2));
  // at most 512 threads per SM: 128 registers a thread, no spills
  static constexpr int MIN_CTAS = ctas_fit(bytes + static_bytes, 512 / G::NT) > 0
                                      ? ctas_fit(bytes + static_bytes, 512 / G::NT)
                                      : 1;
  static_assert((HALO * sizeof(float)) % 128 == 0 && (TILE * sizeof(float)) % 128 == 0,
                "tensor-copy destinations stay 128-byte aligned");
};

template <int S>
__global__ void __launch_bounds__(Geo<S>::NT, ALCfg<S>::MIN_CTAS) adj_interior_loop_kernel(
    const ShotDev *__restrict__ shots, const Tile *__restrict__ tiles, int n, StepArgs a,
    int *__restrict__ err) {
  SEIS_AGEO(S);
  using L = ALCfg<S>;
  constexpr int CW = L::CW, RW = L::RW, HALO = L::HALO;
  using SW = SAT<RW>;
  using ST = SAT<TZ>;
  constexpr int NS = L::NS;
  extern __shared__ __align__(128) unsigned char smraw[];
  float *stage0 = reinterpret_cast<float *>(smraw);
  float *sWZ = stage0 + NS * L::STAGE;
  uint64_t *bar = reinterpret_cast<uint64_t *>(sWZ + HALO);
  __shared__ ShotDev sg[NS];
  __shared__ int2 sxz[NS];  // tile origin of each stage
  __shared__ int s_fail;
  const int tid = threadIdx.x;
  const int G = (int)gridDim.x;
  int i = blockIdx.x;
  if (i >= n) return;
  auto load_shot = [&](int st, int ti) {
    const int shot = tiles[ti].shot;
    if (tid < (int)(sizeof(ShotDev) / sizeof(int)))
      reinterpret_cast<int *>(&sg[st])[tid] = reinterpret_cast<const int *>(shots + shot)[tid];
  };
  auto issue = [&](int st, int ti) {  // thread 0
    const Tile t = tiles[ti];
    sxz[st] = make_int2(t.x0, t.z0);
    const CUtensorMap *maps = shots[t.shot].maps;
    float *bb = stage0 + st * L::STAGE;
    fence_proxy_async();
    mbar_expect_tx(bar + st, (uint32_t)(L::STAGE * sizeof(float)));
    tma_load_2d(bb, maps + MAP_FA_HALO + (a.rot + 1) % 3, t.z0 + ZM - HI, t.x0 + XM - HI, bar + st);
    tma_load_2d(bb + HALO, maps + MAP_VEL_HALO, t.z0 + ZM - HI, t.x0 + XM - HI, bar + st);
    tma_load_2d(bb + 2 * HALO, maps + MAP_FA_TILE + a.rot % 3, t.z0 + ZM, t.x0 + XM, bar + st);
  };
  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < NS; k++) mbar_init(bar + k, 1);
    fence_barrier_init();
    s_fail = 0;
  }
  // the first NS - 1 tiles of this CTA into stages 0 .. NS - 2
#pragma unroll
  for (int k = 0; k < NS - 1; k++)
    if (i + k * G < n) load_shot(k, i + k * G);
  __syncthreads();
  if (tid == 0)
#pragma unroll
    for (int k = 0; k < NS - 1; k++)
      if (i + k * G < n) issue(k, i + k * G);
  __syncthreads();  // the first tiles' origins
  uint32_t par = 0;  // bit s: parity of the next completion of stage s
  int st = 0;
  const int qz = tid % QZ, cx = tid / QZ;
  for (;;) {
    const bool more = i + G < n;
    // the tile NS - 1 ahead into the stage released at the end of the last tile
    const int pf = i + (NS - 1) * G, pst = (st + NS - 1) % NS;
    if (pf < n) {
      load_shot(pst, pf);
      if (tid == 0) issue(pst, pf);
    }
    // this tile's receiver rows and snapshot scale, loaded while its copies
    // land
    const ShotDev &g = sg[st];
    const int x0 = sxz[st].x, z0 = sxz[st].y;
    const int ix = x0 + 2 * cx, iz0 = z0 + 4 * qz;
    const int gzr[2] = {g.gz[ix - g.pml] + g.pml, g.gz[ix + 1 - g.pml] + g.pml};
    const bool img = a.snap_k >= 0 && g.snap != nullptr;
    const float inv_scale = img ? snap_inv_scale<TX, TZ>(g, a.snap_k, x0, z0) : 0.0f;
    // a wait that gives up leaves garbage in the stage (indices stay in
    // range); the CTA then ends after this tile
    if (!mbar_wait(bar + st, (par >> st) & 1u)) s_fail = 1;
    par ^= 1u << st;
    float *sL1 = stage0 + st * L::STAGE, *sWX = sL1 + HALO;
    const float *sL2 = sL1 + 2 * HALO;
    static_assert(HALO % 4 == 0, "whole quads");
    for (int k = 4 * tid; k < HALO; k += 4 * A_NT_I) {  // vx M1 over the velocity, vz M1
      float4 wz, wx;
      weigh_quad(g, *reinterpret_cast<const float4 *>(sWX + k),
                 *reinterpret_cast<const float4 *>(sL1 + k), wz, wx);
      *reinterpret_cast<float4 *>(sWZ + k) = wz;
      *reinterpret_cast<float4 *>(sWX + k) = wx;
    }
    __syncthreads();
    const SW L1{sL1, x0 - HI, z0 - HI}, WZ{sWZ, x0 - HI, z0 - HI}, WX{sWX, x0 - HI, z0 - HI};
    const ST L2{sL2, x0, z0};
    float *out = g.fa[(a.rot + 2) % 3];
    float4 xm[10];
#pragma unroll
    for (int m = 0; m < 10; m++) xm[m] = WX.quad(ix - 4 + m, iz0);
#pragma unroll
    for (int j = 0; j < 2; j++) {
      const float4 za = WZ.quad(ix + j, iz0 - 4), zb = WZ.quad(ix + j, iz0),
                   zc = WZ.quad(ix + j, iz0 + 4);
      const float zz[12] = {za.x, za.y, za.z, za.w, zb.x, zb.y, zb.z, zb.w, zc.x, zc.y, zc.z, zc.w};
      const float4 l1 = L1.quad(ix + j, iz0), l2 = L2.quad(ix + j, iz0);
      const int x = ix + j - g.pml;
      ImageQuad iq;
      if (img) image_load(g, a.snap_k, x, iz0 - g.pml, 0xFu, iq);
      float4 o;
#pragma unroll
      for (int r = 0; r < 4; r++) {
        float sz_ = lap8(zz[r], zz[r + 1], zz[r + 2], zz[r + 3], zz[r + 4], zz[r + 5], zz[r + 6],
                         zz[r + 7], zz[r + 8]);
        float sx_ = lap8(comp(xm[j], r), comp(xm[j + 1], r), comp(xm[j + 2], r),
                         comp(xm[j + 3], r), comp(xm[j + 4], r), comp(xm[j + 5], r),
                         comp(xm[j + 6], r), comp(xm[j + 7], r), comp(xm[j + 8], r));
        float v = sz_ + sx_ + 2.0f * comp(l1, r) - comp(l2, r);
        if (a.rec_k >= 0 && iz0 + r == gzr[j]) v += g.rec[(size_t)a.rec_k * g.nx + x];
        set_comp(o, r, v);
      }
      if (img) image_store(g, x, iz0 - g.pml, 0xFu, iq, inv_scale, a.img_w, l1);
      *reinterpret_cast<float4 *>(out + (size_t)(ix + j) * g.LDZ + iz0) = o;
    }
    __syncthreads();  // stage st, vz M1, its origin and shot table are free
    if (s_fail) {
      if (tid == 0) {  // the copies in flight land before the CTA ends
        atomicExch(err, 2);
        for (int k = 1; k < NS; k++) {
          const int sk = (st + k) % NS;
          if (i + k * G < n) mbar_wait(bar + sk, (par >> sk) & 1u);
        }
      }
      return;
    }
    if (!more) break;
    i += G;
    st = (st + 1) % NS;
  }
}

// 8th-order weight of offset m (|m| <= 4), fd.cpp:1245-1253
__device__ __forceinline__ float tap8(int m) {
  m = m < 0 ? -m : m;
  return m == 0 ? SEIS_C4 : m == 1 ? SEIS_C3 : m == 2 ? SEIS_C2 : m == 3 ? SEIS_C1 : SEIS_C0;
}

// [t == s + 1] + [t == s - 1] - 2 [t == s]
__device__ __forceinline__ float lap3(int t, int s) {
  return t == s ? -2.0f : (t == s + 1 || t == s - 1) ? 1.0f : 0.0f;
}

// Coefficient of cur(tx, tz) in the two-way value of a consumer cell (cx, cz)
// in the frame or the low-order rings: the transpose of twoway_cell (frame
// fd.cpp:1057-1091, low order :1226-1241) without the 2 cur term that every
// branch has.
template <class VA>
__device__ float dcur(const ShotDev &g, const VA &V, int cx, int cz, int tx, int tz) {
  const int NX = g.NX, NZ = g.NZ;
  const int ox = tx - cx, oz = tz - cz;
  float k = 0.0f;
  const bool fx = (cx == 0 || cx == NX - 1), fz = (cz == 0 || cz == NZ - 1);
  if (fx || fz) {
    if (!(fx && fz)) {  // second difference along the edge
      const float v = V(cx, cz);
      if (fz) {
        const float e = v * v * g.kx;
        if (oz == 0) k += e * lap3(tx, cx);
      } else {
        const float e = v * v * (cx == 0 ? g.kz : g.kx);
        if (ox == 0) k += e * lap3(tz, cz);
      }
    }
    if (fz && ox == 0) {  // normal extrapolation along z: + 2 y1 - y2
      const int s1 = cz == 0 ? 1 : NZ - 2, s2 = cz == 0 ? 2 : NZ - 3;
      if (tz >= min(s1, s2) - 1 && tz <= max(s1, s2) + 1) {
        const float v1 = V(cx, s1), v2 = V(cx, s2);
        k += 2.0f * (v1 * v1 * g.kz) * lap3(tz, s1) - (v2 * v2 * g.kz) * lap3(tz, s2);
      }
    }
    if (fx && oz == 0) {  // along x
      const int s1 = cx == 0 ? 1 : NX - 2, s2 = cx == 0 ? 2 : NX - 3;
      if (tx >= min(s1, s2) - 1 && tx <= max(s1, s2) + 1) {
        const float v1 = V(s1, cz), v2 = V(s2, cz);
        k += 2.0f * (v1 * v1 * g.kx) * lap3(tx, s1) - (v2 * v2 * g.kx) * lap3(tx, s2);
      }
    }
    return k;
  }
  const Coef c = coef(V(cx, cz), g);
  if (ox == 0) k += c.vz * lap3(tz, cz);
  if (oz == 0) k += c.vx * lap3(tx, cx);
  return k;
}

// The part of S_cur^T M at cell (tx, tz) that comes from frame and low-order
// consumers (cells within 3 of the grid edge) on its cross is nonzero only
// within 4 of the edge.  A 2nd-order consumer reads its neighbours within one
// cell, a frame consumer (edge row or column) those within one cell along the
// edge and three cells along its normal extrapolation, so the part is
//   sum over m = -3..3 of c_z[m] M(tx, tz + m) + sum over m != 0 of c_x[m] M(tx + m, tz)
// with c = dcur of the consumer (zero for the other offsets and for
// consumers in the 8th-order region).  The coefficients depend on the
// velocity only: this kernel forms them for every cell of the four edge
// bands of every shot (band cell i of band b, see edge_index).
__global__ void edge_coef_kernel(const ShotDev *__restrict__ shots, int nshots) {
  const ShotDev &g = shots[blockIdx.y];
  const int NX = g.NX, NZ = g.NZ, n = edge_cells(NX, NZ);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int b, cx, cz;
  if (i < 5 * NX) {
    b = 0; cx = i / 5; cz = i % 5;
  } else if (i < 10 * NX) {
    b = 1; cx = (i - 5 * NX) / 5; cz = NZ - 5 + (i - 5 * NX) % 5;
  } else if (i < 10 * NX + 5 * NZ) {
    b = 2; cx = (i - 10 * NX) / NZ; cz = (i - 10 * NX) % NZ;
  } else {
    b = 3; cx = NX - 5 + (i - 10 * NX - 5 * NZ) / NZ; cz = (i - 10 * NX - 5 * NZ) % NZ;
  }
  (void)b;
  const GA V{g.vel, g.LDZ};
  auto low = [&](int x, int z) {
    return x >= 0 && x < NX && z >= 0 && z < NZ && !(x >= 4 && x <= NX - 5 && z >= 4 && z <= NZ - 5);
  };
  float *c = g.edge_coef + i;
  const bool in = cx >= 0 && cx < NX && cz >= 0 && cz < NZ;
  int k = 0;
  for (int m = -3; m <= 3; m++, k++) {
    const int z = cz + m;
    float v = 0.0f;
    if (in && ((m >= -1 && m <= 1) || z == 0 || z == NZ - 1) && low(cx, z))
      v = dcur(g, V, cx, z, cx, cz);
    c[(size_t)k * n] = v;
  }
  for (int m = -3; m <= 3; m++) {
    if (m == 0) continue;
    const int x = cx + m;
    float v = 0.0f;
    if (in && ((m >= -1 && m <= 1) || x == 0 || x == NX - 1) && low(x, cz))
      v = dcur(g, V, x, cz, cx, cz);
    c[(size_t)k * n] = v;
    k++;
  }
}

// The frame and low-order part at band cell (tx, tz) of band b from the
// precomputed coefficients (z taps, then x taps, each by increasing offset)
template <class A>
__device__ __forceinline__ float edge_terms_pre(const ShotDev &g, const A &M, int b, int tx,
                                                int tz) {
  const int n = edge_cells(g.NX, g.NZ);
  const float *c = g.edge_coef + edge_index(b, g.NX, g.NZ, tx, tz);
  float s = 0.0f;
#pragma unroll
  for (int m = -3; m <= 3; m++) s = s + __ldg(c + (size_t)(m + 3) * n) * M(tx, tz + m);
#pragma unroll
  for (int m = -3, k = 7; m <= 3; m++) {
    if (m == 0) continue;
    s = s + __ldg(c + (size_t)k * n) * M(tx + m, tz);
    k++;
  }
  return s;
}

// ---------------------------------------------------------------- pad tiles
// The one-way update of a strip cell (fd.cpp:1098-1104) is
//   u31 = al (u3_i + p) + be (u3_i+t + u3_i-t + p_+t + p_-t) + ga (c + c_i) - p_i
// with al = (a1 - a2 - 2 a3)/d, be = a3/d, ga = 2 a2/d, d = a1 + a2 (c, p =
// cur, prev at the cell; _i at the inner neighbour, +-t along the strip), and
// of a corner cell (fd.cpp:1146-1178) u31 = cz u3_z + cx u3_x + bK c.  Every
// ring cell of a tile and its halo stores rho times its coefficients and a
// 3-bit role for each of the 9 offsets of the cells it feeds; each pad or
// model edge cell then gathers from its 3 x 3 neighbours in a fixed order.
enum RingRole : int {
  ROLE_NONE = 0,
  ROLE_SELF = 1,    // strip cell itself: cur ga, prev al
  ROLE_INNER = 2,   // its inner neighbour: u3 al, cur ga, prev -1
  ROLE_TANG = 3,    // along the strip: prev be
  ROLE_DIAG = 4,    // inner +- along: u3 be
  ROLE_CZ = 5,      // corner: u3 at the z-inner neighbour
  ROLE_CX = 6,      // corner: u3 at the x-inner neighbour
  ROLE_CSELF = 7,   // corner cell itself: cur bK
};
__device__ __forceinline__ int role_slot(int ox, int oz) { return 3 * ((ox + 1) * 3 + (oz + 1)); }

// rho-weighted one-way coefficients and roles of one ring cell
__device__ __forceinline__ int ring_coefs(const ShotDev &g, const PadPos &pp, float v, float rho,
                                          float &p0, float &p1, float &p2, float &p3) {
  const int nx_ = pp.dl > 0 ? 1 : (pp.distx > 0 ? -1 : 0);
  const int nz_ = pp.du > 0 ? 1 : (pp.distz > 0 ? -1 : 0);
  if (pp.distx == pp.ring && pp.distz == pp.ring) {
    const float ax3 = g.sqrt2f / v / g.dt;
    const float re = 1.0f / (g.ax1 + g.ax2 + ax3);
    p0 = g.ax1 * re * rho;
    p1 = g.ax2 * re * rho;
    p2 = ax3 * re * rho;
    p3 = 0.0f;
    return ROLE_CSELF << role_slot(0, 0) | ROLE_CZ << role_slot(0, nz_) |
           ROLE_CX << role_slot(nx_, 0);
  }
  const bool zs = pp.distz == pp.ring;  // top / bottom strip: inner along z
  const int ix_ = zs ? 0 : nx_, iz_ = zs ? nz_ : 0, tx_ = zs, tz_ = !zs;
  const float a1 = zs ? g.a1z : g.a1x;
  const float a2 = g.hdt2 * (1.0f / v);
  const float a3 = v * 0.25f * (zs ? g.invdx2 : g.invdz2);
  const float rd = 1.0f / (a1 + a2);
  p0 = (a1 - a2 - 2.0f * a3) * rd * rho;
  p1 = a3 * rd * rho;
  p2 = 2.0f * a2 * rd * rho;
  p3 = rho;
  return ROLE_SELF << role_slot(0, 0) | ROLE_INNER << role_slot(ix_, iz_) |
         ROLE_TANG << role_slot(tx_, tz_) | ROLE_TANG << role_slot(-tx_, -tz_) |
         ROLE_DIAG << role_slot(ix_ + tx_, iz_ + tz_) |
         ROLE_DIAG << role_slot(ix_ - tx_, iz_ - tz_);
}

// Halo cell i of the tile at (x0, z0) (columns x0-1 .. x0+TX, rows z0-1 ..
// z0+TZ): the rows above and below, then the columns left and right.
template <int TX, int TZ>
__device__ __forceinline__ void adj_halo_cell(int i, int x0, int z0, int &hx, int &hz) {
  if (i < 2 * (TX + 2)) {
    hx = x0 - 1 + i % (TX + 2);
    hz = i < TX + 2 ? z0 - 1 : z0 + TZ;
  } else {
    const int j = i - 2 * (TX + 2);
    hx = j < TZ ? x0 - 1 : x0 + TX;
    hz = z0 + j % TZ;
  }
}

// L = S_cur^T M1 - M2 + E + R^T d on a tile with pad-ring cells, pad-ring
// neighbours or consumers outside the 8th-order region; grad += w lap M1 on
// its model cells; then M, E (next step) and B of its pad and model edge
// cells, L = M elsewhere.
// One pad tile at (x0, z0): thread 0 issues its tensor copies on `bar`
// (phase parity `parity`); the result is whether they landed in time (when
// not, the buffers hold garbage, every index stays in range and the caller
// reports the error).  Every thread of the CTA calls this (it holds block
// barriers).
template <int S>
__device__ __forceinline__ bool adj_pad_cells(const ShotDev &g, const StepArgs &a, int x0, int z0,
                                              unsigned char *smraw, uint64_t *bar,
                                              uint32_t parity) {
  SEIS_AGEO(S);
  using SA = SAT<SR>;
  constexpr int RW = AG_::RW, RN = AG_::RN, ADJ_NHALO = AG_::NHALO, HPT = AG_::HPT;
  float *sV = reinterpret_cast<float *>(smraw);   // wide
  float *sL1 = sV + WIDE;                          // wide
  float *sL2 = sL1 + WIDE;                         // narrow
  float *sWZ = sL2 + NARROW;                       // wide
  float *sWX = sWZ + WIDE;                         // wide
  float *sCOR = sWX + WIDE;                        // tile + halo: frame / low-order terms
  // ring arrays of tile + halo, over sL1 .. sCOR once L is formed
  float *rp0 = sL1, *rp1 = rp0 + RN, *rp2 = rp1 + RN, *rp3 = rp2 + RN;
  int *rmask = reinterpret_cast<int *>(rp3 + RN);
  const int tid = threadIdx.x;
  const int NX = g.NX, NZ = g.NZ;
  if (tid == 0) {
    fence_proxy_async();
    mbar_expect_tx(bar, (uint32_t)((2 * WIDE + NARROW) * sizeof(float)));
    tma_load_2d(sL1, g.maps + MAP_FA_WIDE + (a.rot + 1) % 3, z0, x0 + XM - HXC, bar);
    tma_load_2d(sV, g.maps + MAP_VEL_WIDE, z0, x0 + XM - HXC, bar);
    tma_load_2d(sL2, g.maps + MAP_FA_NARROW + a.rot % 3, z0, x0 + XM - 1, bar);
  }
  // this step's ring terms E of the thread's tile columns and halo cells,
  // loaded while the tensor copies are in flight
  const float *Ecur = g.adj_e[a.rot & 1];
  float *Enext = g.adj_e[(a.rot + 1) & 1];
  const int qz = tid % QZ, cxp = tid / QZ;
  const int ix = x0 + 2 * cxp, iz0 = z0 + 4 * qz;
  float4 e4[2];
#pragma unroll
  for (int j = 0; j < 2; j++) {
    e4[j] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (ix + j < NX && iz0 < NZ)
      e4[j] = *reinterpret_cast<const float4 *>(Ecur + (size_t)(ix + j) * g.LDZ + iz0);
  }
  int hx[HPT], hz[HPT];
  float eh[HPT];
  PadPos hp[HPT];
  bool hring[HPT];
#pragma unroll
  for (int h = 0; h < HPT; h++) {
    const int i = tid + h * A_NT_I;
    hx[h] = hz[h] = -1;
    eh[h] = 0.0f;
    hp[h] = PadPos{};
    hring[h] = false;
    if (i >= ADJ_NHALO) continue;
    adj_halo_cell<TX, TZ>(i, x0, z0, hx[h], hz[h]);
    const int cx = hx[h], cz = hz[h];
    if (cx >= 0 && cz >= 0 && cx < NX && cz < NZ) {
      hp[h] = pad_pos(g, cx, cz);
      hring[h] = hp[h].ring > 0;
    }
    if (hring[h]) eh[h] = Ecur[(size_t)cx * g.LDZ + cz];
  }
  const bool ok = mbar_wait(bar, parity);
  // vz M1, vx M1 of the 8th-order consumers (zero elsewhere), a quad of rows
  // at a time (SR and the window's first row are multiples of 4)
  static_assert(SR % 4 == 0 && WIDE % 4 == 0, "whole quads");
  for (int i = 4 * tid; i < WIDE; i += 4 * A_NT_I) {
    const int cx = x0 - HXC + i / SR, cz = z0 - ZM + i % SR;
    float4 wz = make_float4(0.f, 0.f, 0.f, 0.f), wx = wz;
    if (cx >= 4 && cx <= NX - 5) {
      if (cz >= 4 && cz + 3 <= NZ - 5) {
        weigh_quad(g, *reinterpret_cast<const float4 *>(sV + i),
                   *reinterpret_cast<const float4 *>(sL1 + i), wz, wx);
      } else {
#pragma unroll
        for (int r = 0; r < 4; r++)
          if (cz + r >= 4 && cz + r <= NZ - 5) {
            const Coef k = coef(sV[i + r], g);
            set_comp(wz, r, k.vz * sL1[i + r]);
            set_comp(wx, r, k.vx * sL1[i + r]);
          }
      }
    }
    *reinterpret_cast<float4 *>(sWZ + i) = wz;
    *reinterpret_cast<float4 *>(sWX + i) = wx;
  }
  const int zm = z0 - ZM;
  const SA L1{sL1, x0 - HXC, zm}, V{sV, x0 - HXC, zm}, WZ{sWZ, x0 - HXC, zm},
      WX{sWX, x0 - HXC, zm};
  const SA L2{sL2, x0 - 1, zm};
  auto ridx = [&](int cx, int cz) { return (cx - x0 + 1) * RW + (cz - z0 + 1); };
  auto near4 = [&](int cx, int cz) {
    return min(min(cx, cz), min(NX - 1 - cx, NZ - 1 - cz)) <= 4;
  };
  // cells of the tile and halo within 4 of the grid edge have low-order or
  // frame consumers: their terms are formed by all threads over the edge
  // bands (a cell in two bands is formed twice, to the same value)
  const int xa = max(x0 - 1, 0), xb = min(x0 + TX + 1, NX);
  const int za = max(z0 - 1, 0), zb = min(z0 + TZ + 1, NZ);
  const bool edge = xa <= 4 || za <= 4 || xb - 1 >= NX - 5 || zb - 1 >= NZ - 5;
  if (edge) {
#pragma unroll 1
    for (int b = 0; b < 4; b++) {  // top, bottom, left, right band
      const int bxa = b == 3 ? max(xa, NX - 5) : xa, bxb = b == 2 ? min(xb, 5) : xb;
      const int bza = b == 1 ? max(za, NZ - 5) : za, bzb = b == 0 ? min(zb, 5) : zb;
      const int nr = bzb - bza, nc = bxb - bxa;
      if (nr <= 0 || nc <= 0) continue;
      for (int i = tid; i < nr * nc; i += A_NT_I) {
        const int cx = bxa + i / nr, cz = bza + i % nr;
        sCOR[ridx(cx, cz)] = edge_terms_pre(g, L1, b, cx, cz);
      }
    }
  }
  __syncthreads();

  // L of the tile's cells (kept in registers), imaging on its model cells
  const bool img = a.snap_k >= 0 && g.snap != nullptr;
  float Lt[8];
  {
    const float inv_scale = img ? snap_inv_scale<TX, TZ>(g, a.snap_k, x0, z0) : 0.0f;
    float4 xm[10];
#pragma unroll
    for (int m = 0; m < 10; m++) xm[m] = WX.quad(ix - 4 + m, iz0);
#pragma unroll
    for (int j = 0; j < 2; j++) {
      const int cx = ix + j;
      const float4 za4 = WZ.quad(cx, iz0 - 4), zb4 = WZ.quad(cx, iz0), zc4 = WZ.quad(cx, iz0 + 4);
      const float zz[12] = {za4.x, za4.y, za4.z, za4.w, zb4.x, zb4.y,
                            zb4.z, zb4.w, zc4.x, zc4.y, zc4.z, zc4.w};
      const float4 l1 = L1.quad(cx, iz0), l2 = L2.quad(cx, iz0);
      const int x = cx - g.pml;
      const int gzr = (x >= 0 && x < g.nx && cx < NX) ? g.gz[x] + g.pml : -1;
      unsigned ok = 0;  // the quad's model cells
#pragma unroll
      for (int r = 0; r < 4; r++) {
        const int z = iz0 + r - g.pml;
        if (cx < NX && x >= 0 && x < g.nx && z >= 0 && z < g.nz) ok |= 1u << r;
      }
      ImageQuad iq;
      if (img) image_load(g, a.snap_k, x, iz0 - g.pml, ok, iq);
#pragma unroll
      for (int r = 0; r < 4; r++) {
        const int cz = iz0 + r;
        const float sz_ = lap8(zz[r], zz[r + 1], zz[r + 2], zz[r + 3], zz[r + 4], zz[r + 5],
                               zz[r + 6], zz[r + 7], zz[r + 8]);
        const float sx_ = lap8(comp(xm[j], r), comp(xm[j + 1], r), comp(xm[j + 2], r),
                               comp(xm[j + 3], r), comp(xm[j + 4], r), comp(xm[j + 5], r),
                               comp(xm[j + 6], r), comp(xm[j + 7], r), comp(xm[j + 8], r));
        float v = sz_ + sx_ + 2.0f * comp(l1, r);
        if (edge && cx < NX && cz < NZ && near4(cx, cz)) v = v + sCOR[ridx(cx, cz)];
        v = v - comp(l2, r) + comp(e4[j], r);
        if (a.rec_k >= 0 && cz == gzr) v += g.rec[(size_t)a.rec_k * g.nx + x];
        Lt[4 * j + r] = v;
      }
      if (img) image_store(g, x, iz0 - g.pml, ok, iq, inv_scale, a.img_w, l1);
    }
  }
  // L of the halo's pad cells (the only halo cells whose rho is read); halo
  // cell tid + h * A_NT_I of thread tid
  float Lh[HPT];
#pragma unroll
  for (int h = 0; h < HPT; h++) {
    Lh[h] = 0.0f;
    const int cx = hx[h], cz = hz[h];
    if (hring[h]) {
      const float sz_ = lap8(WZ(cx, cz - 4), WZ(cx, cz - 3), WZ(cx, cz - 2), WZ(cx, cz - 1),
                             WZ(cx, cz), WZ(cx, cz + 1), WZ(cx, cz + 2), WZ(cx, cz + 3),
                             WZ(cx, cz + 4));
      const float sx_ = lap8(WX(cx - 4, cz), WX(cx - 3, cz), WX(cx - 2, cz), WX(cx - 1, cz),
                             WX(cx, cz), WX(cx + 1, cz), WX(cx + 2, cz), WX(cx + 3, cz),
                             WX(cx + 4, cz));
      float v = sz_ + sx_ + 2.0f * L1(cx, cz);
      if (edge && near4(cx, cz)) v = v + sCOR[ridx(cx, cz)];
      v = v - L2(cx, cz) + eh[h];
      const int x = cx - g.pml;
      if (a.rec_k >= 0 && x >= 0 && x < g.nx && cz == g.gz[x] + g.pml)
        v += g.rec[(size_t)a.rec_k * g.nx + x];
      Lh[h] = v;
    }
  }
  __syncthreads();  // sL1, sL2, sWZ, sWX and sCOR are dead: the ring arrays go there
  float *sLt = rp0 + 5 * RN;  // L of the tile's cells, [TX][TZ]
  // rho = (1 - w) L of a ring cell, times its one-way coefficients
  auto put_ring = [&](int cx, int cz, const PadPos &pp, bool ring, float L) {
    const int i = ridx(cx, cz);
    int mask = 0;
    float p0 = 0.0f, p1 = 0.0f, p2 = 0.0f, p3 = 0.0f;
    if (ring) mask = ring_coefs(g, pp, V(cx, cz), (1.0f - pad_weight(g, pp)) * L, p0, p1, p2, p3);
    rmask[i] = mask;
    rp0[i] = p0;
    rp1[i] = p1;
    rp2[i] = p2;
    rp3[i] = p3;
  };
  // the owners keep L of the tile in shared memory and clear the roles and
  // terms of the tile cells that are no ring cells; the halo's ring cells are
  // formed by the threads that hold their L
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const int cx = ix + k / 4, cz = iz0 + k % 4;
    sLt[(cx - x0) * TZ + (cz - z0)] = Lt[k];
    // a ring cell is a pad cell (outside the model), pad_pos(...).ring > 0
    const bool pad = cx < g.pml || cx >= g.pml + g.nx || cz < g.pml || cz >= g.pml + g.nz;
    if (!(cx < NX && cz < NZ && pad)) {
      const int q = ridx(cx, cz);
      rmask[q] = 0;
      rp0[q] = rp1[q] = rp2[q] = rp3[q] = 0.0f;
    }
  }
#pragma unroll
  for (int h = 0; h < HPT; h++)
    if (tid + h * A_NT_I < ADJ_NHALO) put_ring(hx[h], hz[h], hp[h], hring[h], Lh[h]);
  __syncthreads();
  // the ring cells of the tile (its pad cells), shared evenly by all threads
  const int xe_ = min(x0 + TX, NX), ze_ = min(z0 + TZ, NZ);
  const CellList ring(x0, z0, xe_, ze_, g.pml, g.pml + g.nx, g.pml, g.pml + g.nz);
  for (int i = tid; i < ring.n; i += A_NT_I) {
    int cx, cz;
    ring.cell(i, cx, cz);
    put_ring(cx, cz, pad_pos(g, cx, cz), true, sLt[(cx - x0) * TZ + (cz - z0)]);
  }
  __syncthreads();

  // M = w L + P_u3^T rho, E of the next step and the kept prev terms on the
  // pad and model edge cells (the cells outside the model less its edge),
  // shared evenly by all threads
  float *out = g.fa[(a.rot + 2) % 3];
  const CellList aff(x0, z0, xe_, ze_, g.pml + 1, g.pml + g.nx - 1, g.pml + 1, g.pml + g.nz - 1);
  // the kept prev terms of the thread's cells, loaded before any store
  constexpr int KMAX = (TX * TZ + A_NT_I - 1) / A_NT_I;
  float bold[KMAX];
#pragma unroll
  for (int k = 0; k < KMAX; k++) {
    const int i = tid + k * A_NT_I;
    bold[k] = 0.0f;
    if (i < aff.n) {
      int cx, cz;
      aff.cell(i, cx, cz);
      bold[k] = g.adj_b[(size_t)cx * g.LDZ + cz];
    }
  }
#pragma unroll
  for (int k = 0; k < KMAX; k++) {
    const int i = tid + k * A_NT_I;
    if (i >= aff.n) continue;
    int cx, cz;
    aff.cell(i, cx, cz);
    float m = 0.0f, e = 0.0f, b = 0.0f;
    // Away from the corners every ring cell within one cell of this one lies
    // in the same strip: its roles follow from the strip's inner direction
    // (top / bottom: +-z, left / right: +-x) and the terms are summed in the
    // order of the general gather below (non-ring cells hold zero terms).
    const int fz = (cx - 1 >= g.pml && cx + 1 <= g.pml + g.nx - 1 && g.nz >= 3)
                       ? (cz <= g.pml ? 1 : (cz >= g.pml + g.nz - 1 ? -1 : 0))
                       : 0;
    const int fx = (fz == 0 && cz - 1 >= g.pml && cz + 1 <= g.pml + g.nz - 1 && g.nx >= 3)
                       ? (cx <= g.pml ? 1 : (cx >= g.pml + g.nx - 1 ? -1 : 0))
                       : 0;
    const int c0 = ridx(cx, cz);
    if (fz > 0) {  // top strip: this cell is the inner neighbour of the one above
      const int qi = ridx(cx, cz - 1);
      m += rp1[ridx(cx - 1, cz - 1)];
      b += rp1[ridx(cx - 1, cz)];
      m += rp0[qi]; e += rp2[qi]; b -= rp3[qi];
      e += rp2[c0]; b += rp0[c0];
      m += rp1[ridx(cx + 1, cz - 1)];
      b += rp1[ridx(cx + 1, cz)];
    } else if (fz < 0) {  // bottom strip
      const int qi = ridx(cx, cz + 1);
      b += rp1[ridx(cx - 1, cz)];
      m += rp1[ridx(cx - 1, cz + 1)];
      e += rp2[c0]; b += rp0[c0];
      m += rp0[qi]; e += rp2[qi]; b -= rp3[qi];
      b += rp1[ridx(cx + 1, cz)];
      m += rp1[ridx(cx + 1, cz + 1)];
    } else if (fx > 0) {  // left strip
      const int qi = ridx(cx - 1, cz);
      m += rp1[ridx(cx - 1, cz - 1)];
      m += rp0[qi]; e += rp2[qi]; b -= rp3[qi];
      m += rp1[ridx(cx - 1, cz + 1)];
      b += rp1[ridx(cx, cz - 1)];
      e += rp2[c0]; b += rp0[c0];
      b += rp1[ridx(cx, cz + 1)];
    } else if (fx < 0) {  // right strip
      const int qi = ridx(cx + 1, cz);
      b += rp1[ridx(cx, cz - 1)];
      e += rp2[c0]; b += rp0[c0];
      b += rp1[ridx(cx, cz + 1)];
      m += rp1[ridx(cx + 1, cz - 1)];
      m += rp0[qi]; e += rp2[qi]; b -= rp3[qi];
      m += rp1[ridx(cx + 1, cz + 1)];
    } else {
#pragma unroll
      for (int dx = -1; dx <= 1; dx++)
#pragma unroll
        for (int dz = -1; dz <= 1; dz++) {
          const int q = ridx(cx + dx, cz + dz);
          // this cell sits at offset (-dx, -dz) from the ring cell
          switch ((rmask[q] >> role_slot(-dx, -dz)) & 7) {
            case ROLE_SELF: e += rp2[q]; b += rp0[q]; break;
            case ROLE_INNER: m += rp0[q]; e += rp2[q]; b -= rp3[q]; break;
            case ROLE_TANG: b += rp1[q]; break;
            case ROLE_DIAG: m += rp1[q]; break;
            case ROLE_CZ: m += rp0[q]; break;
            case ROLE_CX: m += rp1[q]; break;
            case ROLE_CSELF: e += rp2[q]; break;
            default: break;
          }
        }
    }
    const PadPos pt = pad_pos(g, cx, cz);
    const float w = pt.ring == 0 ? 1.0f : pad_weight(g, pt);
    const size_t at = (size_t)cx * g.LDZ + cz;
    out[at] = w * sLt[(cx - x0) * TZ + (cz - z0)] + m;
    Enext[at] = e + bold[k];
    g.adj_b[at] = b;
  }
  // the other cells: M = L, from the owners' registers
  auto inner = [&](int cx, int cz) {
    return cx > g.pml && cx < g.pml + g.nx - 1 && cz > g.pml && cz < g.pml + g.nz - 1;
  };
#pragma unroll
  for (int j = 0; j < 2; j++) {
    const int cx = ix + j;
    if (cx >= NX || iz0 >= NZ) continue;
    const size_t col = (size_t)cx * g.LDZ;
    if (iz0 + 3 < NZ && inner(cx, iz0) && inner(cx, iz0 + 3)) {
      *reinterpret_cast<float4 *>(out + col + iz0) =
          make_float4(Lt[4 * j], Lt[4 * j + 1], Lt[4 * j + 2], Lt[4 * j + 3]);
    } else {
#pragma unroll
      for (int r = 0; r < 4; r++)
        if (iz0 + r < NZ && inner(cx, iz0 + r)) out[col + iz0 + r] = Lt[4 * j + r];
    }
  }
  return ok;
}

template <int S>
__global__ void __launch_bounds__(Geo<S>::NT, AGeo<S>::MIN_P) adj_pad_kernel(
    const ShotDev *__restrict__ shots, const Tile *__restrict__ tiles, StepArgs a,
    int *__restrict__ err) {
  SEIS_AGEO(S);
  extern __shared__ __align__(128) unsigned char smraw[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smraw + sizeof(float) * AG_::PAD_FLOATS);
  const int tid = threadIdx.x;
  const Tile t = tiles[blockIdx.x];
  __shared__ ShotDev sg;
  if (tid < (int)(sizeof(ShotDev) / sizeof(int)))
    reinterpret_cast<int *>(&sg)[tid] = reinterpret_cast<const int *>(shots + t.shot)[tid];
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (!adj_pad_cells<S>(sg, a, t.x0, t.z0, smraw, bar, 0) && tid == 0) atomicExch(err, 2);
}

}  // namespace SEIS_NS
}  // namespace seis
