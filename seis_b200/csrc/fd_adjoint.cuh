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
// Interior tiles (tile + 4-cell halo strictly inside the model, no cell read
// by the one-way update) reduce to the symmetric gather
//   L_k = Lz(vz L1) + Lx(vx L1) + 2 L1 - L2 + R^T d.
// Pad tiles: mu(L1) = w L1 + ringsT((1-w) L1) and the ring terms of cur and
// prev are scattered from every ring cell of the tile + 5-cell halo; the
// transposed two-way stencil is then a gather of vz mu, vx mu over the 8th-order
// consumers (as in the interior), plus a scatter from the low-order and frame
// consumers of the outer 4 cells.  Scatters accumulate in 64-bit fixed point
// (shared-memory integer atomics, whose sum does not depend on the order of
// the adds), so the adjoint is bit-for-bit repeatable.  The tile's scale is
// 2^(49 - e) for inputs below 2^e: every accumulator stays below 2^62 (a
// target collects at most ~2^12 times the largest input) and the resolution
// is 2^-49 of the tile's largest input.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "fd_tile.cuh"

namespace seis {
namespace SEIS_NS {

constexpr int A_NT_I = 256;  // interior adjoint kernel threads
constexpr int A_NT_P = 256;  // pad adjoint kernel threads
constexpr int WIDE = CW_C * SR, NARROW = CW_P * SR;
constexpr int MU_C = TX + 8, MU_R = TZ + 8;  // mu on tile + 4 halo

__device__ __forceinline__ float snap_load(const ShotDev &g, int k, int x, int z) {
  size_t i = (size_t)k * g.nx * g.nz + (size_t)x * g.nz + z;
  switch (g.snap_dtype) {
    case SNAP_F32: return reinterpret_cast<const float *>(g.snap)[i];
    case SNAP_BF16: return __bfloat162float(reinterpret_cast<const __nv_bfloat16 *>(g.snap)[i]);
    case SNAP_F16: return __half2float(reinterpret_cast<const __half *>(g.snap)[i]);
    default: return 0.0f;
  }
}

__device__ __forceinline__ float snap_inv_scale(const ShotDev &g, int k, int x0, int z0) {
  if (g.snap_dtype == SNAP_F32) return 1.0f;
  const int ntx = (g.NX + TX - 1) / TX;
  return 1.0f / g.snap_scale[(size_t)k * ntx * g.ntz + (x0 / TX) * g.ntz + z0 / TZ];
}

// Coefficients of the one-way update of a pad-ring cell, as the linear map
// u31 = sum coef * input (fd.cpp:1098-1104, :1146-1178).
struct RingCoef {
  int corner;         // 1: diagonal corner
  int nx_, nz_;       // unit step toward the interior (inner neighbour offset)
  int tx_, tz_;       // unit tangential step (strips)
  float au3i, au3t;   // coefficients of u3 at inner, inner +- tangential
  float bK, bi;       // of cur at the cell, at inner
  float gK, gi, gt;   // of prev at the cell, inner, cell +- tangential
  float cz, cx;       // corners: of u3 at the z-inner and x-inner neighbours
};

template <class VA>
__device__ __forceinline__ RingCoef ring_coef(const ShotDev &g, const VA &V, int ix, int iz,
                                              const PadPos &pp) {
  RingCoef r;
  float v = V(ix, iz);
  if (pp.distx == pp.ring && pp.distz == pp.ring) {
    r.corner = 1;
    r.nx_ = pp.dl > 0 ? 1 : -1;
    r.nz_ = pp.du > 0 ? 1 : -1;
    r.tx_ = r.tz_ = 0;
    float ax3;
    if (pp.dl > 0 && pp.du > 0)
      ax3 = __double2float_rn(g.sqrt2d / (double)v / (double)g.dt);
    else
      ax3 = g.sqrt2f / v / g.dt;
    float e = g.ax1 + g.ax2 + ax3;
    r.cz = g.ax1 / e;
    r.cx = g.ax2 / e;
    r.bK = ax3 / e;
    r.au3i = r.au3t = r.bi = r.gK = r.gi = r.gt = 0.0f;
    return r;
  }
  r.corner = 0;
  float a1, a3;
  if (pp.distz == pp.ring) {  // top / bottom strip
    r.nx_ = 0; r.nz_ = pp.du > 0 ? 1 : -1;
    r.tx_ = 1; r.tz_ = 0;
    a1 = g.a1z;
    a3 = v / 4.0f / g.dx / g.dx;
  } else {  // left / right strip
    r.nx_ = pp.dl > 0 ? 1 : -1; r.nz_ = 0;
    r.tx_ = 0; r.tz_ = 1;
    a1 = g.a1x;
    a3 = v / 4.0f / g.dz / g.dz;
  }
  float a2 = g.hdt2 / v;
  float d = a1 + a2;
  // u31 = -tmp / d, tmp as in fd.cpp:1101-1103
  r.au3i = (a1 - a2 - 2.0f * a3) / d;
  r.au3t = a3 / d;
  r.bK = 2.0f * a2 / d;
  r.bi = 2.0f * a2 / d;
  r.gK = (a1 - a2 - 2.0f * a3) / d;
  r.gi = -(a1 + a2) / d;
  r.gt = a3 / d;
  r.cz = r.cx = 0.0f;
  return r;
}

struct AdjTile {  // fixed-point accumulator over a rectangular window of the grid
  long long *s;
  int x0, z0, ncol, nrow;  // window origin and size
  float scale;             // value -> fixed point (a power of two)
  double inv;              // fixed point -> value
  __device__ __forceinline__ bool in(int ix, int iz) const {
    return ix >= x0 && ix < x0 + ncol && iz >= z0 && iz < z0 + nrow;
  }
  __device__ __forceinline__ void add(int ix, int iz, float v) const {
    if (in(ix, iz))
      atomicAdd(reinterpret_cast<unsigned long long *>(&s[(ix - x0) * nrow + (iz - z0)]),
                (unsigned long long)__float2ll_rn(v * scale));
  }
  __device__ __forceinline__ float get(int ix, int iz) const {
    return (float)((double)s[(ix - x0) * nrow + (iz - z0)] * inv);
  }
};

// largest |value| over n staged floats, reduced across the block
template <int NTH>
__device__ float block_amax(const float *a, int n, const float *b, int nb, float *red) {
  float m = 0.0f;
  for (int i = threadIdx.x; i < n; i += NTH) m = fmaxf(m, fabsf(a[i]));
  for (int i = threadIdx.x; i < nb; i += NTH) m = fmaxf(m, fabsf(b[i]));
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  m = 0.0f;
#pragma unroll
  for (int w = 0; w < NTH / 32; w++) m = fmaxf(m, red[w]);
  return m;
}

// Scatter of the transposed two-way update and frame of consumer cell (ix,iz)
// with adjoint mu into cb (mirrors fd.cpp:1057-1091 and :1226-1271).
template <class VA>
__device__ void stencil_T(const ShotDev &g, const VA &V, int ix, int iz, float mu,
                          const AdjTile &cb) {
  const int NX = g.NX, NZ = g.NZ;
  bool fx = (ix == 0 || ix == NX - 1), fz = (iz == 0 || iz == NZ - 1);
  auto d2T = [&](float e, float v, float k, int ax, int az, int bx, int bz, int cx_, int cz_) {
    float t = v * v * k * e;
    cb.add(ax, az, t);
    cb.add(bx, bz, t);
    cb.add(cx_, cz_, -2.0f * t);
  };
  if (fx || fz) {
    if (!(fx && fz)) {
      if (fz)
        d2T(mu, V(ix, iz), g.kx, ix + 1, iz, ix - 1, iz, ix, iz);
      else
        d2T(mu, V(ix, iz), ix == 0 ? g.kz : g.kx, ix, iz + 1, ix, iz - 1, ix, iz);
    }
    cb.add(ix, iz, 2.0f * mu);
    if (fz) {
      int s1 = iz == 0 ? 1 : NZ - 2, s2 = iz == 0 ? 2 : NZ - 3, dz = iz == 0 ? 1 : -1;
      d2T(2.0f * mu, V(ix, s1), g.kz, ix, s1 + dz, ix, s1 - dz, ix, s1);
      d2T(-mu, V(ix, s2), g.kz, ix, s2 + dz, ix, s2 - dz, ix, s2);
    }
    if (fx) {
      int s1 = ix == 0 ? 1 : NX - 2, s2 = ix == 0 ? 2 : NX - 3, dx = ix == 0 ? 1 : -1;
      d2T(2.0f * mu, V(s1, iz), g.kx, s1 + dx, iz, s1 - dx, iz, s1, iz);
      d2T(-mu, V(s2, iz), g.kx, s2 + dx, iz, s2 - dx, iz, s2, iz);
    }
    return;
  }
  Coef k = coef(V(ix, iz), g);
  float vz = k.vz * mu, vx = k.vx * mu;
  if (ix >= 4 && ix <= NX - 5 && iz >= 4 && iz <= NZ - 5) {
    const float a[9] = {SEIS_C0, SEIS_C1, SEIS_C2, SEIS_C3, SEIS_C4, SEIS_C3, SEIS_C2, SEIS_C1, SEIS_C0};
#pragma unroll
    for (int m = 0; m < 9; m++) {
      cb.add(ix, iz - 4 + m, a[m] * vz);
      cb.add(ix - 4 + m, iz, a[m] * vx);
    }
  } else {
    cb.add(ix, iz - 1, vz);
    cb.add(ix, iz + 1, vz);
    cb.add(ix + 1, iz, vx);
    cb.add(ix - 1, iz, vx);
    cb.add(ix, iz, -2.0f * vz - 2.0f * vx);
  }
  cb.add(ix, iz, 2.0f * mu);
}

// ---------------------------------------------------------------- interior
// L_k = Lz(vz L1) + Lx(vx L1) + 2 L1 - L2 + R^T d ; grad += w lap L1.
__global__ void __launch_bounds__(A_NT_I, 2) adj_interior_kernel(const ShotDev *__restrict__ shots,
                                                                 const Tile *__restrict__ tiles,
                                                                 StepArgs a, int *__restrict__ err) {
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
  // weighted fields vz L1, vx L1 on the staged window
  for (int i = tid; i < WIDE; i += A_NT_I) {
    Coef k = coef(sV[i], g);
    float l = sL1[i];
    sWZ[i] = k.vz * l;
    sWX[i] = k.vx * l;
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
  float inv_scale = img ? snap_inv_scale(g, a.snap_k, x0, z0) : 0.0f;
#pragma unroll
  for (int j = 0; j < 2; j++) {
    const float4 za = WZ.quad(ix + j, iz0 - 4), zb = WZ.quad(ix + j, iz0), zc = WZ.quad(ix + j, iz0 + 4);
    const float zz[12] = {za.x, za.y, za.z, za.w, zb.x, zb.y, zb.z, zb.w, zc.x, zc.y, zc.z, zc.w};
    const float4 l1 = L1.quad(ix + j, iz0), l2 = L2.quad(ix + j, iz0);
    const int x = ix + j - g.pml;
    const int gzr = g.gz[x] + g.pml;
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
      if (img) {
        const int z = iz0 + r - g.pml;
        float lap = snap_load(g, a.snap_k, x, z) * inv_scale;
        g.grad[(size_t)x * g.nz + z] += (double)(a.img_w * lap * comp(l1, r));
      }
    }
    *reinterpret_cast<float4 *>(out + (size_t)(ix + j) * g.LDZ + iz0) = o;
  }
}

// ---------------------------------------------------------------- pad tiles
// shared memory: staged L1, V (wide), L2 (narrow); MU1 (fixed point, tile + 4);
// ACC (fixed point, tile: ring terms of cur and prev minus mu(L2), and the
// frame-band stencil scatter); WZ, WX = vz mu, vx mu of the 8th-order
// consumers (float, tile + 4)
constexpr size_t ADJ_PAD_F32 = sizeof(float) * (size_t)(2 * WIDE + NARROW);
static_assert(ADJ_PAD_F32 % 16 == 0, "fixed-point accumulators must be 16-byte aligned");
constexpr size_t ADJ_PAD_SMEM = ADJ_PAD_F32 + sizeof(long long) * (size_t)(MU_C * MU_R + TX * TZ) +
                                sizeof(float) * (size_t)(2 * MU_C * MU_R) + 16;

struct MA {  // float array over tile + 4, column stride MU_R
  const float *s;
  int x0h, z0h;
  __device__ __forceinline__ float operator()(int ix, int iz) const {
    return s[(ix - x0h) * MU_R + (iz - z0h)];
  }
  __device__ __forceinline__ float4 quad(int ix, int iz) const {
    return *reinterpret_cast<const float4 *>(s + (ix - x0h) * MU_R + (iz - z0h));
  }
};

__global__ void __launch_bounds__(A_NT_P, 2) adj_pad_kernel(const ShotDev *__restrict__ shots,
                                                            const Tile *__restrict__ tiles,
                                                            StepArgs a, int *__restrict__ err) {
  extern __shared__ __align__(128) unsigned char smraw[];
  float *sL1 = reinterpret_cast<float *>(smraw);  // wide
  float *sV = sL1 + WIDE;                          // wide
  float *sL2 = sV + WIDE;                          // narrow
  long long *sMU1 = reinterpret_cast<long long *>(smraw + ADJ_PAD_F32);  // tile + 4
  long long *sACC = sMU1 + MU_C * MU_R;                                  // tile
  float *sWZ = reinterpret_cast<float *>(sACC + TX * TZ);                // tile + 4
  float *sWX = sWZ + MU_C * MU_R;                                        // tile + 4
  uint64_t *bar = reinterpret_cast<uint64_t *>(sWX + MU_C * MU_R);
  __shared__ float red[A_NT_P / 32];
  __shared__ ShotDev sg;
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
  const int NX = g.NX, NZ = g.NZ;
  const int zm = z0 - ZM;
  const SA L1{sL1, x0 - HXC, zm}, V{sV, x0 - HXC, zm}, L2{sL2, x0 - 1, zm};
  int e;
  frexpf(block_amax<A_NT_P>(sL1, WIDE, sL2, NARROW, red), &e);  // inputs below 2^e
  const int se = min(49 - e, 126);
  const float scale = ldexpf(1.0f, se);
  const double inv = ldexp(1.0, -se);
  const AdjTile MU1{sMU1, x0 - 4, z0 - 4, MU_C, MU_R, scale, inv};
  const AdjTile ACC{sACC, x0, z0, TX, TZ, scale, inv};
  auto fix = [&](float v) { return __float2ll_rn(v * scale); };
  auto is8 = [&](int cx, int cz) { return cx >= 4 && cx <= NX - 5 && cz >= 4 && cz <= NZ - 5; };

  // blendT of the cells themselves: MU1 = w L1 on tile + 4, ACC = -w L2 on
  // the tile (plain stores: each cell once)
  for (int i = tid; i < MU_C * MU_R; i += A_NT_P) {
    const int cx = x0 - 4 + i / MU_R, cz = z0 - 4 + i % MU_R;
    long long m = 0;
    if (cx >= 0 && cx < NX && cz >= 0 && cz < NZ) {
      PadPos pp = pad_pos(g, cx, cz);
      const float w = pp.ring == 0 ? 1.0f : pad_weight(g, pp);
      m = fix(w * L1(cx, cz));
    }
    sMU1[i] = m;
  }
  for (int i = tid; i < TX * TZ; i += A_NT_P) {
    const int cx = x0 + i / TZ, cz = z0 + i % TZ;
    long long m = 0;
    if (cx < NX && cz < NZ) {
      PadPos pp = pad_pos(g, cx, cz);
      const float w = pp.ring == 0 ? 1.0f : pad_weight(g, pp);
      m = -fix(w * L2(cx, cz));
    }
    sACC[i] = m;
  }
  __syncthreads();

  // ringsT of the pad cells of tile + 5: (1 - w) L1 through the one-way
  // update's u3, cur and prev terms, (1 - w) L2 through its prev terms and
  // (minus) its u3 terms.  Terms that land on the same cell are summed before
  // the fixed-point add; cells at least 2 inside both windows skip the
  // window test.
  constexpr int R5C = TX + 10, R5R = TZ + 10;
  auto addu = [&](long long *base, int ncol, int x0w, int z0w, int nrow, int ix, int iz, float v) {
    atomicAdd(reinterpret_cast<unsigned long long *>(&base[(ix - x0w) * nrow + (iz - z0w)]),
              (unsigned long long)fix(v));
  };
  for (int i = tid; i < R5C * R5R; i += A_NT_P) {
    const int cx = x0 - 5 + i / R5R, cz = z0 - 5 + i % R5R;
    if (cx < 0 || cx >= NX || cz < 0 || cz >= NZ) continue;
    PadPos pp = pad_pos(g, cx, cz);
    if (pp.ring == 0) continue;
    const bool near1 = cx >= x0 - 1 && cx <= x0 + TX && cz >= z0 - 1 && cz <= z0 + TZ;
    const float w = pad_weight(g, pp);
    RingCoef rc = ring_coef(g, V, cx, cz, pp);
    const float n1 = (1.0f - w) * L1(cx, cz), n2 = near1 ? (1.0f - w) * L2(cx, cz) : 0.0f;
    // deep: every target (distance <= 1) inside the tile (ACC) and tile + 4 (MU1)
    const bool deep = cx >= x0 + 1 && cx <= x0 + TX - 2 && cz >= z0 + 1 && cz <= z0 + TZ - 2;
    if (rc.corner) {
      if (deep) {
        addu(sMU1, MU_C, x0 - 4, z0 - 4, MU_R, cx, cz + rc.nz_, rc.cz * n1);
        addu(sMU1, MU_C, x0 - 4, z0 - 4, MU_R, cx + rc.nx_, cz, rc.cx * n1);
        addu(sACC, TX, x0, z0, TZ, cx, cz, rc.bK * n1);
        addu(sACC, TX, x0, z0, TZ, cx, cz + rc.nz_, -(rc.cz * n2));
        addu(sACC, TX, x0, z0, TZ, cx + rc.nx_, cz, -(rc.cx * n2));
      } else {
        MU1.add(cx, cz + rc.nz_, rc.cz * n1);
        MU1.add(cx + rc.nx_, cz, rc.cx * n1);
        ACC.add(cx, cz, rc.bK * n1);
        if (near1) {
          ACC.add(cx, cz + rc.nz_, -(rc.cz * n2));
          ACC.add(cx + rc.nx_, cz, -(rc.cx * n2));
        }
      }
    } else {
      const int ix_i = cx + rc.nx_, iz_i = cz + rc.nz_;
      const float at = rc.au3t * n1, mt = -(rc.au3t * n2), gt = rc.gt * n2;
      const float self = rc.bK * n1 + rc.gK * n2;
      const float inner = rc.bi * n1 - rc.au3i * n2 + rc.gi * n2;
      if (deep) {
        addu(sMU1, MU_C, x0 - 4, z0 - 4, MU_R, ix_i, iz_i, rc.au3i * n1);
        addu(sMU1, MU_C, x0 - 4, z0 - 4, MU_R, ix_i + rc.tx_, iz_i + rc.tz_, at);
        addu(sMU1, MU_C, x0 - 4, z0 - 4, MU_R, ix_i - rc.tx_, iz_i - rc.tz_, at);
        addu(sACC, TX, x0, z0, TZ, cx, cz, self);
        addu(sACC, TX, x0, z0, TZ, ix_i, iz_i, inner);
        addu(sACC, TX, x0, z0, TZ, ix_i + rc.tx_, iz_i + rc.tz_, mt);
        addu(sACC, TX, x0, z0, TZ, ix_i - rc.tx_, iz_i - rc.tz_, mt);
        addu(sACC, TX, x0, z0, TZ, cx + rc.tx_, cz + rc.tz_, gt);
        addu(sACC, TX, x0, z0, TZ, cx - rc.tx_, cz - rc.tz_, gt);
      } else {
        MU1.add(ix_i, iz_i, rc.au3i * n1);
        MU1.add(ix_i + rc.tx_, iz_i + rc.tz_, at);
        MU1.add(ix_i - rc.tx_, iz_i - rc.tz_, at);
        if (near1) {
          ACC.add(cx, cz, self);
          ACC.add(ix_i, iz_i, inner);
          ACC.add(ix_i + rc.tx_, iz_i + rc.tz_, mt);
          ACC.add(ix_i - rc.tx_, iz_i - rc.tz_, mt);
          ACC.add(cx + rc.tx_, cz + rc.tz_, gt);
          ACC.add(cx - rc.tx_, cz - rc.tz_, gt);
        } else {
          ACC.add(cx, cz, rc.bK * n1);
          ACC.add(ix_i, iz_i, rc.bi * n1);
        }
      }
    }
  }
  __syncthreads();

  // stencilT: vz mu, vx mu of the 8th-order consumers for the gather; the
  // low-order and frame consumers (outer 4 cells) scatter
  for (int i = tid; i < MU_C * MU_R; i += A_NT_P) {
    const int cx = x0 - 4 + i / MU_R, cz = z0 - 4 + i % MU_R;
    float wz = 0.0f, wx = 0.0f;
    if (cx >= 0 && cx < NX && cz >= 0 && cz < NZ && sMU1[i] != 0) {
      const float mu = (float)((double)sMU1[i] * inv);
      if (is8(cx, cz)) {
        Coef k = coef(V(cx, cz), g);
        wz = k.vz * mu;
        wx = k.vx * mu;
      } else {
        stencil_T(g, V, cx, cz, mu, ACC);
      }
    }
    sWZ[i] = wz;
    sWX[i] = wx;
  }
  __syncthreads();

  // L_k = gather + ACC + R^T d on the tile; grad += w lap mu(L1)
  const MA WZ{sWZ, x0 - 4, z0 - 4}, WX{sWX, x0 - 4, z0 - 4};
  const int qz = tid % QZ, cxp = tid / QZ;
  const int ix = x0 + 2 * cxp, iz0 = z0 + 4 * qz;
  float *out = g.fa[(a.rot + 2) % 3];
  const bool img = a.snap_k >= 0 && g.snap != nullptr;
  const float inv_scale = img ? snap_inv_scale(g, a.snap_k, x0, z0) : 0.0f;
  float4 xm[10];
#pragma unroll
  for (int m = 0; m < 10; m++) xm[m] = WX.quad(ix - 4 + m, iz0);
#pragma unroll
  for (int j = 0; j < 2; j++) {
    const int cx = ix + j;
    if (cx >= NX) continue;
    const float4 za = WZ.quad(cx, iz0 - 4), zb = WZ.quad(cx, iz0), zc = WZ.quad(cx, iz0 + 4);
    const float zz[12] = {za.x, za.y, za.z, za.w, zb.x, zb.y, zb.z, zb.w, zc.x, zc.y, zc.z, zc.w};
    const int x = cx - g.pml;
    const int gzr = (x >= 0 && x < g.nx) ? g.gz[x] + g.pml : -1;
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int cz = iz0 + r;
      if (cz >= NZ) break;
      const float sz_ = lap8(zz[r], zz[r + 1], zz[r + 2], zz[r + 3], zz[r + 4], zz[r + 5],
                             zz[r + 6], zz[r + 7], zz[r + 8]);
      const float sx_ = lap8(comp(xm[j], r), comp(xm[j + 1], r), comp(xm[j + 2], r),
                             comp(xm[j + 3], r), comp(xm[j + 4], r), comp(xm[j + 5], r),
                             comp(xm[j + 6], r), comp(xm[j + 7], r), comp(xm[j + 8], r));
      const float mu = MU1.get(cx, cz);
      float v = sz_ + sx_ + (is8(cx, cz) ? 2.0f * mu : 0.0f) + ACC.get(cx, cz);
      if (a.rec_k >= 0 && cz == gzr) v += g.rec[(size_t)a.rec_k * g.nx + x];
      out[(size_t)cx * g.LDZ + cz] = v;
      const int z = cz - g.pml;
      if (img && x >= 0 && x < g.nx && z >= 0 && z < g.nz) {
        float lap = snap_load(g, a.snap_k, x, z) * inv_scale;
        g.grad[(size_t)x * g.nz + z] += (double)(a.img_w * lap * mu);
      }
    }
  }
}

}  // namespace SEIS_NS
}  // namespace seis
