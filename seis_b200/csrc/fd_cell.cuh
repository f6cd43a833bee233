// Per-cell formulas of the reference time step, written against accessor
// objects so that the same code serves any staging layout.
//
// Evaluation order follows the reference statement cited at each function.
// In the exact build (--fmad=false, IEEE division) every operation rounds on
// its own exactly as the reference's x86-64 build; the fast build of the same
// source contracts multiply-adds and uses approximate division.
#pragma once
#include "fd_internal.h"

namespace seis {
namespace SEIS_NS {

// 8th-order second-derivative weights, src/util/fd.cpp:1245-1253.
#define SEIS_C0 (-1.0f / 560.0f)
#define SEIS_C1 (8.0f / 315.0f)
#define SEIS_C2 (-1.0f / 5.0f)
#define SEIS_C3 (8.0f / 5.0f)
#define SEIS_C4 (-205.0f / 72.0f)

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

// sum_k a_k u[k] in the reference order (fd.cpp:1263-1268)
__device__ __forceinline__ float lap8(float m4, float m3, float m2, float m1, float c, float p1,
                                      float p2, float p3, float p4) {
  float s = m4 * SEIS_C0;
  s = s + m3 * SEIS_C1;
  s = s + m2 * SEIS_C2;
  s = s + m1 * SEIS_C3;
  s = s + c * SEIS_C4;
  s = s + p1 * SEIS_C3;
  s = s + p2 * SEIS_C2;
  s = s + p3 * SEIS_C1;
  s = s + p4 * SEIS_C0;
  return s;
}

__device__ __forceinline__ float d2(float v, float k, float a, float b, float c) {
  return v * v * k * (a + b - 2.0f * c);
}

// Two-way value of one cell before the absorbing blend, any region: frame
// (processBoundary part (i), fd.cpp:1057-1091), 2nd order rings 1-3
// (modeling2D_low, :1226-1241) or 8th order (modeling2D_high, :1259-1270).
template <class A>
__device__ float twoway_cell(const A &cur, const A &prev, const A &V, const ShotDev &g, int ix,
                             int iz) {
  const int NX = g.NX, NZ = g.NZ;
  float c = cur(ix, iz);
  float p = prev(ix, iz);
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
    uzz = lap8(cur(ix, iz - 4), cur(ix, iz - 3), cur(ix, iz - 2), cur(ix, iz - 1), c,
               cur(ix, iz + 1), cur(ix, iz + 2), cur(ix, iz + 3), cur(ix, iz + 4));
    uxx = lap8(cur(ix - 4, iz), cur(ix - 3, iz), cur(ix - 2, iz), cur(ix - 1, iz), c,
               cur(ix + 1, iz), cur(ix + 2, iz), cur(ix + 3, iz), cur(ix + 4, iz));
  } else {
    uzz = cur(ix, iz - 1) + cur(ix, iz + 1) - 2.0f * c;
    uxx = cur(ix + 1, iz) + cur(ix - 1, iz) - 2.0f * c;
  }
  return k.vz * uzz + k.vx * uxx + 2.0f * c - p;
}

// One-way strip update, fd.cpp:1098-1104 (and the three mirrored strips).
__device__ __forceinline__ float oneway(float a1, float a2, float a3, float u3i, float u3tp,
                                        float u3tm, float cK, float ci, float pK, float pi,
                                        float ptp, float ptm) {
  float tmp = -a1 * u3i - a1 * (pK - pi) + a2 * (pK - 2.0f * cK + u3i + pi - 2.0f * ci) -
              a3 * (u3tp + u3tm - 2.0f * u3i + ptp + ptm - 2.0f * pK);
  return -tmp / (a1 + a2);
}

// Where a cell sits relative to the absorbing pad (setAbs InitInversion.cpp:11-40
// and the ring loops of processBoundary fd.cpp:1092-1179).
struct PadPos {
  int ring;      // 0 = model interior, else the ring index IK (1..pml)
  int dl, du;    // > 0 when left of / above the interior
  int distx, distz;
};
__device__ __forceinline__ PadPos pad_pos(const ShotDev &g, int ix, int iz) {
  PadPos p;
  p.dl = g.pml - ix;
  p.du = g.pml - iz;
  int dr = ix - (g.pml + g.nx - 1), dd = iz - (g.pml + g.nz - 1);
  p.distx = max(max(p.dl, dr), 0);
  p.distz = max(max(p.du, dd), 0);
  p.ring = max(p.distx, p.distz);
  return p;
}

// Blend weight of a pad cell: the x ramp wins in the corners
// (InitInversion.cpp:20-37).  The contracted build (SEIS_FAST_MATH)
// multiplies by precomputed reciprocals where the reference divides.
__device__ __forceinline__ float pad_weight(const ShotDev &g, const PadPos &p) {
  int d = p.distx > 0 ? p.distx : p.distz;
#ifdef SEIS_FAST_MATH
  return 1.0f - (float)d * g.inv_pml;
#else
  return 1.0f - (float)d * 1.0f / (float)g.pml;
#endif
}

// What the absorbing update of one pad cell needs besides the fields
// (fd.cpp:1092-1179, blend :55-56): its kind, inner neighbour and the
// velocity-dependent coefficients, formed once per cell and applied to every
// field of the cell (Born's two fields share them).
struct Absorb {
  int kind;        // 0 model cell, 1 diagonal corner, 2 top / bottom strip, 3 left / right strip
  int I;           // strips: the inner neighbour's row (kind 2) or column (kind 3)
  int sxn, szn;    // corners: one cell toward the interior
  float a1, a2, a3;  // strips: one-way coefficients; corners: a3 = ax3
  float w;           // blend weight
};
template <class A>
__device__ __forceinline__ Absorb absorb_geom(const A &V, const ShotDev &g, int ix, int iz) {
  Absorb q;
  PadPos pp = pad_pos(g, ix, iz);
  q.kind = 0;
  q.I = 0;
  q.sxn = q.szn = 0;
  q.a1 = q.a2 = q.a3 = 0.0f;
  q.w = 1.0f;
  if (pp.ring == 0) return q;  // interior: w = 1, u31 = 0
  float v = V(ix, iz);
  if (pp.distx == pp.ring && pp.distz == pp.ring) {  // diagonal corner, fd.cpp:1146-1178
    q.kind = 1;
    q.sxn = pp.dl > 0 ? 1 : -1;  // toward the interior
    q.szn = pp.du > 0 ? 1 : -1;
    if (pp.dl > 0 && pp.du > 0)  // upper-left: sqrt(2)/v/dt formed in double, fd.cpp:1176
      q.a3 = __double2float_rn(g.sqrt2d / (double)v / (double)g.dt);
    else
      q.a3 = g.sqrt2f / v / g.dt;
  } else if (pp.distz == pp.ring) {  // top / bottom strip, inner along z
    q.kind = 2;
    q.I = pp.du > 0 ? iz + 1 : iz - 1;
    q.a1 = g.a1z;
#ifdef SEIS_FAST_MATH
    q.a2 = g.hdt2 * (1.0f / v);
    q.a3 = v * g.q4dx2;
#else
    q.a2 = g.hdt2 / v;
    q.a3 = v / 4.0f / g.dx / g.dx;
#endif
  } else {  // left / right strip, inner along x
    q.kind = 3;
    q.I = pp.dl > 0 ? ix + 1 : ix - 1;
    q.a1 = g.a1x;
#ifdef SEIS_FAST_MATH
    q.a2 = g.hdt2 * (1.0f / v);
    q.a3 = v * g.q4dz2;
#else
    q.a2 = g.hdt2 / v;
    q.a3 = v / 4.0f / g.dz / g.dz;
#endif
  }
  q.w = pad_weight(g, pp);
  return q;
}

// Absorbing blend of one field at one cell with two-way value u3.  U3 =
// two-way field (tile + 1 halo); cur/P = current and previous field.
template <class U3A, class A>
__device__ __forceinline__ float absorb_apply(const Absorb &q, float u3, const U3A &U3,
                                              const A &cur, const A &P, const ShotDev &g, int ix,
                                              int iz) {
  if (q.kind == 0) return u3 + 0.0f;
  float u31;
  if (q.kind == 1) {
    float tmp = -g.ax1 * U3(ix, iz + q.szn) - g.ax2 * U3(ix + q.sxn, iz) + q.a3 * (-cur(ix, iz));
    u31 = -tmp / (g.ax1 + g.ax2 + q.a3);
  } else if (q.kind == 2) {
    const int I = q.I;
    u31 = oneway(q.a1, q.a2, q.a3, U3(ix, I), U3(ix + 1, I), U3(ix - 1, I), cur(ix, iz),
                 cur(ix, I), P(ix, iz), P(ix, I), P(ix + 1, iz), P(ix - 1, iz));
  } else {
    const int I = q.I;
    u31 = oneway(q.a1, q.a2, q.a3, U3(I, iz), U3(I, iz + 1), U3(I, iz - 1), cur(ix, iz),
                 cur(I, iz), P(ix, iz), P(I, iz), P(ix, iz + 1), P(ix, iz - 1));
  }
  return u3 * q.w + u31 * (1.0f - q.w);
}

}  // namespace SEIS_NS
}  // namespace seis
