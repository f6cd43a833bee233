// Fused time-step kernels of the 2-D acoustic FD engine (sm_100a).
//
// One launch advances every shot of a batch by one time step.  Each CTA owns
// one TZ x TX tile of one shot's padded grid and produces the next wavefield
// there in a single pass:
//   two-way update   modeling2D_low/high      src/util/fd.cpp:1226-1271
//   source / receiver injection               fd.cpp:49-51, :673-677
//   outer frame      processBoundary (i)      fd.cpp:1057-1091
//   one-way ABC      processBoundary (ii)     fd.cpp:1092-1179
//   blend            u w + u31 (1-w)          fd.cpp:55-56, setAbs InitInversion.cpp:11-40
//   recording / boundary strips               fd.cpp:58-63, :1181-1203
// The one-way update of a pad cell reads the two-way value of its inner
// neighbours, so boundary tiles first build the two-way field on the tile plus
// a one-cell halo in shared memory.  Interior tiles (all cells inside the model
// and in the 8th-order region) skip that: their blend is the identity.
//
// This file is compiled with --fmad=false and IEEE division/sqrt, and every
// expression keeps the reference's evaluation order, so each cell rounds
// exactly as the reference's x86-64 build does.
#include "fd_internal.h"

namespace seis {
namespace {

// 8th-order second-derivative weights, fd.cpp:1245-1253.
__device__ __constant__ float kC[9] = {-1.0f / 560.0f, 8.0f / 315.0f, -1.0f / 5.0f,
                                       8.0f / 5.0f,    -205.0f / 72.0f, 8.0f / 5.0f,
                                       -1.0f / 5.0f,   8.0f / 315.0f, -1.0f / 560.0f};

__device__ __forceinline__ float4 ld4(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
__device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }
__device__ __forceinline__ float comp(const float4 &v, int r) {
  return r == 0 ? v.x : (r == 1 ? v.y : (r == 2 ? v.z : v.w));
}
__device__ __forceinline__ void set_comp(float4 &v, int r, float x) {
  if (r == 0) v.x = x; else if (r == 1) v.y = x; else if (r == 2) v.z = x; else v.w = x;
}

// Load the current field of one tile plus halo into shared memory (float4
// granularity; cells outside the padded grid read as zero).
__device__ __forceinline__ void load_tile(float *s, const float *f, const ShotDev &g, int x0,
                                          int z0) {
  constexpr int Q = SROWS / 4;
  for (int i = threadIdx.x; i < SCOLS * Q; i += NTHREADS) {
    int c = i / Q, q = i - c * Q;
    int ix = x0 - HX + c, iz = z0 - HZ + 4 * q;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (ix >= 0 && ix < g.NX && iz >= 0 && iz < g.LDZ) v = ld4(f + (size_t)ix * g.LDZ + iz);
    reinterpret_cast<float4 *>(s)[c * Q + q] = v;
  }
}

struct Coef {
  float vz, vx, vt2;
};
// vt2 = (v dt)^2, vvzz = vt2/dz^2, vvxx = vt2/dx^2 (fd.cpp:34-40).
__device__ __forceinline__ Coef coef(float v, const ShotDev &g) {
  float t = v * g.dt;
  Coef c;
  c.vt2 = t * t;
  c.vz = c.vt2 * g.invdz2;
  c.vx = c.vt2 * g.invdx2;
  return c;
}

// Accessor of the shared tile by padded-grid coordinates.
struct STile {
  const float *s;
  int x0, z0;
  __device__ __forceinline__ float operator()(int ix, int iz) const {
    return s[(ix - x0 + HX) * SROWS + (iz - z0 + HZ)];
  }
};

__device__ __forceinline__ float d2(float v, float k, float a, float b, float c) {
  return v * v * k * (a + b - 2.0f * c);
}

// Two-way value of one cell (before the absorbing blend), any region:
// frame (processBoundary part (i)), 2nd order rings 1-3, or 8th order.
__device__ float twoway_cell(const STile &cur, const float *prev, const ShotDev &g, int ix,
                             int iz) {
  const int NX = g.NX, NZ = g.NZ, L = g.LDZ;
  const float *vel = g.vel;
  auto V = [&](int x, int z) { return __ldg(vel + (size_t)x * L + z); };
  float c = cur(ix, iz);
  float p = __ldg(prev + (size_t)ix * L + iz);
  bool fx = (ix == 0 || ix == NX - 1), fz = (iz == 0 || iz == NZ - 1);
  if (fx || fz) {
    float u;
    if (fx && fz) {
      u = 2.0f * c - p;
    } else if (fz) {  // top / bottom rows, fd.cpp:1060-1063
      u = d2(V(ix, iz), g.kx, cur(ix + 1, iz), cur(ix - 1, iz), c) + 2.0f * c - p;
    } else if (ix == 0) {  // left column, fd.cpp:1065
      u = d2(V(ix, iz), g.kz, cur(ix, iz + 1), cur(ix, iz - 1), c) + 2.0f * c - p;
    } else {  // right column uses the x coefficient, fd.cpp:1066
      u = d2(V(ix, iz), g.kx, cur(ix, iz + 1), cur(ix, iz - 1), c) + 2.0f * c - p;
    }
    if (fz) {  // normal extrapolation along z, fd.cpp:1072-1081
      int s1 = iz == 0 ? 1 : NZ - 2, s2 = iz == 0 ? 2 : NZ - 3, dz = iz == 0 ? 1 : -1;
      float y1 = d2(V(ix, s1), g.kz, cur(ix, s1 + dz), cur(ix, s1 - dz), cur(ix, s1));
      float y2 = d2(V(ix, s2), g.kz, cur(ix, s2 + dz), cur(ix, s2 - dz), cur(ix, s2));
      u = u + (y1 * 2.0f - y2);
    }
    if (fx) {  // normal extrapolation along x, fd.cpp:1082-1091
      int s1 = ix == 0 ? 1 : NX - 2, s2 = ix == 0 ? 2 : NX - 3, dx = ix == 0 ? 1 : -1;
      float y1 = d2(V(s1, iz), g.kx, cur(s1 + dx, iz), cur(s1 - dx, iz), cur(s1, iz));
      float y2 = d2(V(s2, iz), g.kx, cur(s2 + dx, iz), cur(s2 - dx, iz), cur(s2, iz));
      u = u + (y1 * 2.0f - y2);
    }
    return u;
  }
  Coef k = coef(V(ix, iz), g);
  float uzz, uxx;
  if (ix >= 4 && ix <= NX - 5 && iz >= 4 && iz <= NZ - 5) {
    uzz = cur(ix, iz - 4) * kC[0];
    uxx = cur(ix - 4, iz) * kC[0];
#pragma unroll
    for (int m = 1; m < 9; m++) {
      uzz = uzz + cur(ix, iz - 4 + m) * kC[m];
      uxx = uxx + cur(ix - 4 + m, iz) * kC[m];
    }
  } else {
    uzz = cur(ix, iz - 1) + cur(ix, iz + 1) - 2.0f * c;
    uxx = cur(ix + 1, iz) + cur(ix - 1, iz) - 2.0f * c;
  }
  return k.vz * uzz + k.vx * uxx + 2.0f * c - p;
}

// One-way strip update, fd.cpp:1098-1104 (and mirrored strips).
__device__ __forceinline__ float oneway(float a1, float a2, float a3, float u3i, float u3tp,
                                        float u3tm, float cK, float ci, float pK, float pi,
                                        float ptp, float ptm) {
  float tmp = -a1 * u3i - a1 * (pK - pi) + a2 * (pK - 2.0f * cK + u3i + pi - 2.0f * ci) -
              a3 * (u3tp + u3tm - 2.0f * u3i + ptp + ptm - 2.0f * pK);
  return -tmp / (a1 + a2);
}

// Absorbing blend of one pad cell, given its two-way value u3.
// U3(x,z): two-way field (shared, tile + 1 halo); cur: shared current field.
template <class U3F>
__device__ float absorb_cell(float u3, const U3F &U3, const STile &cur, const float *prev,
                             const ShotDev &g, int ix, int iz) {
  const int pml = g.pml, L = g.LDZ;
  int dl = pml - ix, dr = ix - (pml + g.nx - 1), du = pml - iz, dd = iz - (pml + g.nz - 1);
  int distx = max(max(dl, dr), 0), distz = max(max(du, dd), 0);
  int ik = max(distx, distz);
  if (ik == 0) return u3 + 0.0f;  // interior: w = 1, u31 = 0
  auto P = [&](int x, int z) { return __ldg(prev + (size_t)x * L + z); };
  float v = __ldg(g.vel + (size_t)ix * L + iz);
  float u31;
  if (distx == ik && distz == ik) {  // diagonal corner, fd.cpp:1146-1178
    int sxn = dl > 0 ? 1 : -1, szn = du > 0 ? 1 : -1;  // toward the interior
    float ax3;
    if (dl > 0 && du > 0)  // upper-left corner forms sqrt(2)/v/dt in double, fd.cpp:1176
      ax3 = __double2float_rn(g.sqrt2d / (double)v / (double)g.dt);
    else
      ax3 = g.sqrt2f / v / g.dt;
    float tmp = -g.ax1 * U3(ix, iz + szn) - g.ax2 * U3(ix + sxn, iz) + ax3 * (-cur(ix, iz));
    u31 = -tmp / (g.ax1 + g.ax2 + ax3);
  } else if (distz == ik) {  // top / bottom strip, inner along z
    int I = du > 0 ? iz + 1 : iz - 1;
    float a2 = g.hdt2 / v;
    float a3 = v / 4.0f / g.dx / g.dx;
    u31 = oneway(g.a1z, a2, a3, U3(ix, I), U3(ix + 1, I), U3(ix - 1, I), cur(ix, iz),
                 cur(ix, I), P(ix, iz), P(ix, I), P(ix + 1, iz), P(ix - 1, iz));
  } else {  // left / right strip, inner along x
    int I = dl > 0 ? ix + 1 : ix - 1;
    float a2 = g.hdt2 / v;
    float a3 = v / 4.0f / g.dz / g.dz;
    u31 = oneway(g.a1x, a2, a3, U3(I, iz), U3(I, iz + 1), U3(I, iz - 1), cur(ix, iz),
                 cur(I, iz), P(ix, iz), P(I, iz), P(ix, iz + 1), P(ix, iz - 1));
  }
  // setAbs ramp, InitInversion.cpp:20-37: x ramp wins in the corners.
  int d = distx > 0 ? distx : distz;
  float w = 1.0f - (float)d * 1.0f / (float)pml;
  return u3 * w + u31 * (1.0f - w);
}

struct SU3 {  // two-way field on tile + 1 halo in shared memory
  const float *s;
  int x0, z0;
  __device__ __forceinline__ float operator()(int ix, int iz) const {
    return s[(ix - x0 + 1) * (TZ + 2) + (iz - z0 + 1)];
  }
};

// Record / save outputs of one final cell.  Boundary strips per sample:
// [top 4 x nx][bottom 4 x nx][left 4 x nz][right 4 x nz] (SaveAtBoundary,
// fd.cpp:1183-1203); a cell can sit in several strips when the model is thin.
__device__ __forceinline__ void emit(const ShotDev &g, const StepArgs &a, bool record, int ix,
                                     int iz, float out) {
  const int x = ix - g.pml, z = iz - g.pml;
  if (record && a.rec_k >= 0 && x >= 0 && x < g.nx && iz == g.gz[x] + g.pml)
    g.rec[(size_t)a.rec_k * g.nx + x] = out;
  if (a.strip_k >= 0) {
    float *dst = g.strips + (size_t)a.strip_k * g.strip_len;
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
}

// Injection into the two-way value before the absorbing step.
__device__ __forceinline__ float inject(const ShotDev &g, const StepArgs &a, int mode,
                                        bool field_a, int ix, int iz, float u3, float vt2) {
  if (field_a && mode != MODE_RCV) {
    if (a.src_k >= 0 && ix == g.sxp && iz == g.szp) u3 = u3 + vt2 * g.wav[a.src_k];
  } else if (mode == MODE_RCV) {
    int x = ix - g.pml;
    if (a.rec_k >= 0 && x >= 0 && x < g.nx && iz == g.gz[x] + g.pml)
      u3 = u3 + g.rec[(size_t)a.rec_k * g.nx + x] * vt2;
  }
  return u3;
}

// --------------------------------------------------------------------------
// Interior fast path: each thread owns a 4 (z) x 4 (x) micro-tile.
// --------------------------------------------------------------------------
struct Quad {
  float4 v[4];  // output per column j
};

__device__ __forceinline__ void interior_field(const float *s, const float *prev,
                                               const ShotDev &g, int x0, int z0, float4 out[4],
                                               float4 curc[4], float4 vel[4]) {
  const int qz = threadIdx.x & 15, gxx = threadIdx.x >> 4;
  const float4 *s4 = reinterpret_cast<const float4 *>(s);
  constexpr int Q = SROWS / 4;
  float4 xq[12];
#pragma unroll
  for (int k = 0; k < 12; k++) xq[k] = s4[(4 * gxx + 1 + k) * Q + qz + 2];
  const int iz0 = z0 + 4 * qz;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int col = 4 * gxx + j + HX;
    const int ix = x0 + 4 * gxx + j;
    float zz[12];
    float4 za = s4[col * Q + qz + 1], zb = xq[j + 4], zc = s4[col * Q + qz + 3];
    zz[0] = za.x; zz[1] = za.y; zz[2] = za.z; zz[3] = za.w;
    zz[4] = zb.x; zz[5] = zb.y; zz[6] = zb.z; zz[7] = zb.w;
    zz[8] = zc.x; zz[9] = zc.y; zz[10] = zc.z; zz[11] = zc.w;
    const size_t off = (size_t)ix * g.LDZ + iz0;
    float4 p = ld4(prev + off);
    float4 v = ld4(g.vel + off);
    vel[j] = v;
    curc[j] = zb;
#pragma unroll
    for (int r = 0; r < 4; r++) {
      float uzz = zz[r] * kC[0];
      float uxx = comp(xq[j], r) * kC[0];
#pragma unroll
      for (int m = 1; m < 9; m++) {
        uzz = uzz + zz[r + m] * kC[m];
        uxx = uxx + comp(xq[j + m], r) * kC[m];
      }
      Coef k = coef(comp(v, r), g);
      float u3 = k.vz * uzz + k.vx * uxx + 2.0f * zz[r + 4] - comp(p, r);
      set_comp(out[j], r, u3);
    }
  }
}

template <int MODE>
__global__ void __launch_bounds__(NTHREADS) step_kernel(const ShotDev *__restrict__ shots,
                                                        const Tile *__restrict__ tiles,
                                                        StepArgs a) {
  __shared__ __align__(16) float s_cur[SCOLS * SROWS];
  __shared__ __align__(16) float s_curb[MODE == MODE_BORN ? SCOLS * SROWS : 4];
  __shared__ __align__(16) float s_u3[(TX + 2) * (TZ + 2)];
  __shared__ __align__(16) float s_u3b[MODE == MODE_BORN ? (TX + 2) * (TZ + 2) : 4];

  const Tile t = tiles[blockIdx.x];
  const ShotDev &g = shots[t.shot];
  if (a.rec_k >= g.nt && MODE != MODE_RCV) a.rec_k = -1;
  const int x0 = t.x0, z0 = t.z0;
  const bool use_a = MODE != MODE_RCV;
  const float *pa = g.fa[a.rot % 3], *ca = g.fa[(a.rot + 1) % 3];
  float *na = g.fa[(a.rot + 2) % 3];
  const float *pb = g.fb[a.rot_b % 3], *cb = g.fb[(a.rot_b + 1) % 3];
  float *nb = g.fb[(a.rot_b + 2) % 3];

  if (use_a) load_tile(s_cur, ca, g, x0, z0);
  if (MODE == MODE_RCV) load_tile(s_cur, cb, g, x0, z0);
  if (MODE == MODE_BORN) load_tile(s_curb, cb, g, x0, z0);
  __syncthreads();

  if (t.kind == TILE_INTERIOR) {
    const int qz = threadIdx.x & 15, gxx = threadIdx.x >> 4;
    const int iz0 = z0 + 4 * qz;
    float4 outa[4], cura[4], vel[4];
    const float *p1 = MODE == MODE_RCV ? pb : pa;
    interior_field(s_cur, p1, g, x0, z0, outa, cura, vel);
    float4 lap_src[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int ix = x0 + 4 * gxx + j;
      const size_t off = (size_t)ix * g.LDZ + iz0;
      float4 o = outa[j];
#pragma unroll
      for (int r = 0; r < 4; r++) {
        float u3 = comp(o, r);
        Coef k = coef(comp(vel[j], r), g);
        u3 = inject(g, a, MODE, MODE != MODE_RCV, ix, iz0 + r, u3, k.vt2);
        float out = u3 + 0.0f;
        set_comp(o, r, out);
        if (MODE != MODE_RCV) emit(g, a, MODE == MODE_MODEL, ix, iz0 + r, out);
        if (MODE == MODE_BORN) {
          // scattering source vt2 lap vel3 dv, fd.cpp:134-139
          float prv = __ldg(pa + off + r);
          float lap = (out + prv - 2.0f * comp(cura[j], r)) * g.idt2;
          float vv = comp(vel[j], r);
          float vel3 = 2.0f / (vv * vv * vv);
          float dv = __ldg(g.dv + off + r);
          set_comp(lap_src[j], r, k.vt2 * lap * vel3 * dv);
        }
      }
      st4((MODE == MODE_RCV ? nb : na) + off, o);
    }
    if (MODE == MODE_BORN) {
      float4 outb[4], curb[4], velb[4];
      interior_field(s_curb, pb, g, x0, z0, outb, curb, velb);
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int ix = x0 + 4 * gxx + j;
        const size_t off = (size_t)ix * g.LDZ + iz0;
        float4 o = outb[j];
#pragma unroll
        for (int r = 0; r < 4; r++) {
          float out = (comp(o, r) + comp(lap_src[j], r)) + 0.0f;
          set_comp(o, r, out);
          emit(g, a, true, ix, iz0 + r, out);
        }
        st4(nb + off, o);
      }
    }
    return;
  }

  // ---------------- boundary tile: two-way field on tile + 1 halo ----------
  const STile curA{s_cur, x0, z0};
  const STile curB{s_curb, x0, z0};
  constexpr int HW = TZ + 2;
  for (int i = threadIdx.x; i < (TX + 2) * HW; i += NTHREADS) {
    int hx = i / HW, hz = i - hx * HW;
    int ix = x0 - 1 + hx, iz = z0 - 1 + hz;
    if (ix < 0 || ix >= g.NX || iz < 0 || iz >= g.NZ) continue;
    float vt2 = coef(__ldg(g.vel + (size_t)ix * g.LDZ + iz), g).vt2;
    if (MODE == MODE_RCV) {
      float u = twoway_cell(curA, pb, g, ix, iz);
      s_u3[i] = inject(g, a, MODE, false, ix, iz, u, vt2);
      continue;
    }
    float u = twoway_cell(curA, pa, g, ix, iz);
    u = inject(g, a, MODE, true, ix, iz, u, vt2);
    s_u3[i] = u;
    if (MODE == MODE_BORN) {
      float q = 0.0f;
      int x = ix - g.pml, z = iz - g.pml;
      if (x >= 0 && x < g.nx && z >= 0 && z < g.nz) {  // dv is zero in the pad
        size_t off = (size_t)ix * g.LDZ + iz;
        float out = u + 0.0f;
        float lap = (out + __ldg(pa + off) - 2.0f * curA(ix, iz)) * g.idt2;
        float vv = __ldg(g.vel + off);
        float vel3 = 2.0f / (vv * vv * vv);
        q = vt2 * lap * vel3 * __ldg(g.dv + off);
      }
      s_u3b[i] = twoway_cell(curB, pb, g, ix, iz) + q;
    }
  }
  __syncthreads();
  const SU3 U3a{s_u3, x0, z0};
  const SU3 U3b{s_u3b, x0, z0};
  for (int i = threadIdx.x; i < TX * TZ; i += NTHREADS) {
    int x = i / TZ, z = i - x * TZ;
    int ix = x0 + x, iz = z0 + z;
    if (ix >= g.NX || iz >= g.NZ) continue;
    size_t off = (size_t)ix * g.LDZ + iz;
    if (MODE == MODE_RCV) {
      float out = absorb_cell(U3a(ix, iz), U3a, curA, pb, g, ix, iz);
      nb[off] = out;
      continue;
    }
    float out = absorb_cell(U3a(ix, iz), U3a, curA, pa, g, ix, iz);
    na[off] = out;
    emit(g, a, MODE == MODE_MODEL, ix, iz, out);
    if (MODE == MODE_BORN) {
      float ob = absorb_cell(U3b(ix, iz), U3b, curB, pb, g, ix, iz);
      nb[off] = ob;
      emit(g, a, true, ix, iz, ob);
    }
  }
}

// Pad a [nx][nz] model into the NX x LDZ device layout: clamp-to-edge
// (setVel, InitInversion.cpp:92-113) or zero (setDv, :116-126).
__global__ void pad_kernel(const float *__restrict__ src, int nx, int nz, int pml, int LDZ,
                           int clamp, float *__restrict__ dst) {
  const int NX = nx + 2 * pml, NZ = nz + 2 * pml;
  size_t n = (size_t)NX * LDZ;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    int ix = (int)(i / LDZ), iz = (int)(i - (size_t)ix * LDZ);
    float v = 0.0f;
    int jx = ix - pml, jz = iz - pml;
    if (iz < NZ) {
      if (clamp) {
        jx = jx < 0 ? 0 : (jx >= nx ? nx - 1 : jx);
        jz = jz < 0 ? 0 : (jz >= nz ? nz - 1 : jz);
        v = src[(size_t)jx * nz + jz];
      } else if (jx >= 0 && jx < nx && jz >= 0 && jz < nz) {
        v = src[(size_t)jx * nz + jz];
      }
    }
    dst[i] = v;
  }
}

__global__ void transpose_kernel(const float *__restrict__ src, int rows, int cols,
                                 float *__restrict__ dst) {
  __shared__ float tile[32][33];
  int c = blockIdx.x * 32 + threadIdx.x, r0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    int r = r0 + k;
    if (r < rows && c < cols) tile[k][threadIdx.x] = src[(size_t)r * cols + c];
  }
  __syncthreads();
  int r = r0 + threadIdx.x;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    int cc = blockIdx.x * 32 + k;
    if (r < rows && cc < cols) dst[(size_t)cc * rows + r] = tile[threadIdx.x][k];
  }
}

// Reverse pass of the reference RTM, before each step (fd.cpp:659-663):
// subtract the source from the older field and write the saved boundary
// strips of sample it-ndel into the current field.
__global__ void rtm_restore_kernel(const ShotDev *__restrict__ shots, int nshots, int rot,
                                   int it) {
  const int s = blockIdx.y;
  if (s >= nshots) return;
  const ShotDev &g = shots[s];
  if (it >= g.NT || it < g.ndel) return;
  float *prev = g.fa[rot % 3];
  float *cur = g.fa[(rot + 1) % 3];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0 && it - 1 > 0) {
    size_t off = (size_t)g.sxp * g.LDZ + g.szp;
    float vt2 = coef(g.vel[off], g).vt2;
    prev[off] = prev[off] - vt2 * g.wav[it - 1];
  }
  if (i >= g.strip_len) return;
  const float *src = g.strips + (size_t)(it - g.ndel) * g.strip_len;
  int rowcells = 2 * LAYERS * g.nx;
  int ix, iz;
  if (i < rowcells) {
    int l = i / g.nx, x = i - l * g.nx;
    ix = x + g.pml;
    iz = l < LAYERS ? g.pml + l : g.nz + g.pml - 1 - (l - LAYERS);
  } else {
    int j = i - rowcells;
    int l = j / g.nz, z = j - l * g.nz;
    iz = z + g.pml;
    ix = l < LAYERS ? g.pml + l : g.nx + g.pml - 1 - (l - LAYERS);
  }
  cur[(size_t)ix * g.LDZ + iz] = src[i];
}

// Imaging of the reference RTM, one CTA per interior column (fd.cpp:668-669,
// :681-684, FaQi :1272-1298):
//   U = ((u2 + u0 - 2 u1)/dt^2) vel3,  img += U R,  img += 0.5 (U R - H[U] H[R])
// with H the 61-tap Hilbert FIR along z over the whole padded column.
constexpr int HILB_HALF = 30;
__global__ void rtm_image_kernel(const ShotDev *__restrict__ shots, const int2 *__restrict__ cols,
                                 int rot, int rot_b, const float *__restrict__ taps) {
  extern __shared__ float sh[];
  const int2 c = cols[blockIdx.x];
  const ShotDev &g = shots[c.x];
  const int ix = c.y + g.pml, NZ = g.NZ;
  float *sU = sh, *sR = sh + NZ;
  __shared__ float h[2 * HILB_HALF + 1];
  if (threadIdx.x < 2 * HILB_HALF + 1) h[threadIdx.x] = taps[threadIdx.x];
  // reverse-pass naming: u2 = older (prev), u1 = current, u0 = newest
  const float *u2 = g.fa[rot % 3], *u1 = g.fa[(rot + 1) % 3], *u0 = g.fa[(rot + 2) % 3];
  const float *r0 = g.fb[(rot_b + 2) % 3];
  const size_t col = (size_t)ix * g.LDZ;
  for (int iz = threadIdx.x; iz < NZ; iz += blockDim.x) {
    float lap = (u2[col + iz] + u0[col + iz] - 2.0f * u1[col + iz]) * g.idt2;
    float v = g.vel[col + iz];
    float vel3 = 2.0f / (v * v * v);
    sU[iz] = lap * vel3;
    sR[iz] = r0[col + iz];
  }
  __syncthreads();
  for (int iz = g.pml + threadIdx.x; iz < NZ - g.pml; iz += blockDim.x) {
    int i0 = max(iz - HILB_HALF, 0), i1 = min(iz + HILB_HALF, NZ - 1);
    float uh = 0.0f, rh = 0.0f;
    // odd offsets only: the even taps are exactly zero (hilbert.h:67)
    int start = i0 + (((iz - i0) & 1) ? 0 : 1);
    for (int i = start; i <= i1; i += 2) {
      float hk = h[iz - i + HILB_HALF];
      uh = uh + sU[i] * hk;
      rh = rh + sR[i] * hk;
    }
    float U = sU[iz], R = sR[iz];
    float *img = g.img + (size_t)c.y * g.nz + (iz - g.pml);
    float acc = *img + U * R;
    acc = acc + 0.5f * (U * R - uh * rh);
    *img = acc;
  }
}

}  // namespace

cudaError_t launch_step(int mode, const ShotDev *d_shots, const Tile *d_tiles, int ntiles,
                        const StepArgs &a, cudaStream_t s) {
  if (ntiles <= 0) return cudaSuccess;
  switch (mode) {
    case MODE_MODEL: step_kernel<MODE_MODEL><<<ntiles, NTHREADS, 0, s>>>(d_shots, d_tiles, a); break;
    case MODE_RCV: step_kernel<MODE_RCV><<<ntiles, NTHREADS, 0, s>>>(d_shots, d_tiles, a); break;
    case MODE_BORN: step_kernel<MODE_BORN><<<ntiles, NTHREADS, 0, s>>>(d_shots, d_tiles, a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_pad(const float *d_src, int nx, int nz, int pml, int LDZ, int clamp,
                       float *d_dst, cudaStream_t s) {
  size_t n = (size_t)(nx + 2 * pml) * LDZ;
  int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  pad_kernel<<<blocks, 256, 0, s>>>(d_src, nx, nz, pml, LDZ, clamp, d_dst);
  return cudaGetLastError();
}

cudaError_t launch_transpose(const float *d_src, int rows, int cols, float *d_dst,
                             cudaStream_t s) {
  dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
  transpose_kernel<<<grid, block, 0, s>>>(d_src, rows, cols, d_dst);
  return cudaGetLastError();
}

cudaError_t launch_rtm_restore(const ShotDev *d_shots, int nshots, int max_strip, int rot,
                               int it, cudaStream_t s) {
  dim3 grid((max_strip + 255) / 256, nshots);
  rtm_restore_kernel<<<grid, 256, 0, s>>>(d_shots, nshots, rot, it);
  return cudaGetLastError();
}

cudaError_t launch_rtm_image(const ShotDev *d_shots, const int2 *d_cols, int ncols, int rot,
                             int rot_b, int max_nz, const float *d_taps, cudaStream_t s) {
  size_t smem = 2 * (size_t)max_nz * sizeof(float);
  rtm_image_kernel<<<ncols, 256, smem, s>>>(d_shots, d_cols, rot, rot_b, d_taps);
  return cudaGetLastError();
}

}  // namespace seis
