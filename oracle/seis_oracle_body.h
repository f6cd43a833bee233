/*
 * Body of the CPU oracle (TEST INFRASTRUCTURE ONLY), included twice by
 * seis_oracle.c with REAL = float / double.  See seis_oracle.h.
 *
 * Every arithmetic expression keeps the evaluation order of the reference
 * statement it restates (cited per function); the file is compiled with
 * -ffp-contract=off so that each + - * / is rounded on its own, as the
 * reference's x86-64 build does.
 */
#define CAT_(a, b) a##_##b
#define CAT(a, b) CAT_(a, b)
#define F(name) CAT(name, SFX)
#define KR(x) ((REAL)(x))
#define AT(a, ix, iz) (a)[(size_t)(ix) * (size_t)g->NZ + (size_t)(iz)]

typedef struct {
  int nx, nz, pml, NX, NZ;
  REAL dt, dx, dz;
} F(grid_t);

static F(grid_t) F(mkgrid)(REAL dt, REAL dx, REAL dz, int nx, int nz, int pml)
{
  F(grid_t) g;
  g.nx = nx; g.nz = nz; g.pml = pml;
  g.NX = nx + 2 * pml; g.NZ = nz + 2 * pml;
  g.dt = dt; g.dx = dx; g.dz = dz;
  return g;
}

static REAL *F(zalloc)(size_t n) { return (REAL *)calloc(n ? n : 1, sizeof(REAL)); }

/* rickerWavelet, src/util/wavelet.cpp:7-18.  tmp is formed in double from the
 * 3.1415926 literal and rounded once; exp is the single-precision overload in
 * the float build. */
void F(orc_ricker)(REAL dt, REAL fr, int delay, int n, REAL *out)
{
  REAL tmp = (REAL)(3.1415926 * 3.1415926 * (double)fr * (double)fr);
  for (int i = 0; i < n; i++) {
    REAL t = (REAL)(i - delay) * KR(1.0) * dt;
    REAL t2 = t * t;
    out[i] = (KR(1.0) - KR(2.0) * tmp * t2) * EXPR(-tmp * t2);
  }
}

/* setAbs, src/util/InitInversion.cpp:11-40: 1 inside, linear ramp to 0 at the
 * outer edge; the x ramp covers the full height, the z ramp interior x only. */
void F(orc_set_abs)(int nz, int nx, int pml, REAL *w)
{
  F(grid_t) gg = F(mkgrid)(KR(1), KR(1), KR(1), nx, nz, pml);
  const F(grid_t) *g = &gg;
  REAL *ramp = F(zalloc)((size_t)pml);
  for (int i = 0; i < pml; i++) ramp[i] = KR(1.0) - (REAL)(i + 1) * KR(1.0) / (REAL)pml;
  for (size_t i = 0; i < (size_t)g->NX * g->NZ; i++) w[i] = KR(1.0);
  for (int iz = 0; iz < g->NZ; iz++) {
    for (int ix = 0; ix < pml; ix++) AT(w, ix, iz) = ramp[pml - ix - 1];
    for (int ix = pml + nx; ix < g->NX; ix++) AT(w, ix, iz) = ramp[ix - pml - nx];
  }
  for (int ix = pml; ix < pml + nx; ix++) {
    for (int iz = 0; iz < pml; iz++) AT(w, ix, iz) = ramp[pml - iz - 1];
    for (int iz = pml + nz; iz < g->NZ; iz++) AT(w, ix, iz) = ramp[iz - pml - nz];
  }
  free(ramp);
}

/* setVel, src/util/InitInversion.cpp:92-113: the net effect of its two passes
 * is clamp-to-edge replication of the model into the pad. */
void F(orc_set_vel)(const REAL *v, int nz, int nx, int pml, REAL *out)
{
  F(grid_t) gg = F(mkgrid)(KR(1), KR(1), KR(1), nx, nz, pml);
  const F(grid_t) *g = &gg;
  for (int ix = 0; ix < g->NX; ix++) {
    int jx = ix - pml; jx = jx < 0 ? 0 : (jx >= nx ? nx - 1 : jx);
    for (int iz = 0; iz < g->NZ; iz++) {
      int jz = iz - pml; jz = jz < 0 ? 0 : (jz >= nz ? nz - 1 : jz);
      AT(out, ix, iz) = v[(size_t)jx * nz + jz];
    }
  }
}

/* setDv, src/util/InitInversion.cpp:116-126: zero pad. */
static void F(pad_zero)(const F(grid_t) *g, const REAL *dv, REAL *out)
{
  for (int ix = 0; ix < g->nx; ix++)
    for (int iz = 0; iz < g->nz; iz++)
      AT(out, ix + g->pml, iz + g->pml) = dv[(size_t)ix * g->nz + iz];
}

/* Hilbert<T>::designFilter, src/filter/hilbert.h:59-70.  The taper is formed
 * in double and rounded to REAL; the tap value is formed in double from the
 * REAL taper and rounded once. */
static void F(hilbert_taps)(int half, REAL *h)
{
  h[half] = KR(0);
  for (int i = 1; i <= half; i++) {
    REAL taper = (REAL)(0.54 + 0.46 * cos(3.1415926 * i / half));
    h[half + i] = (REAL)((double)(taper * (REAL)(i % 2)) * 2.0 / (3.1415926 * i));
    h[half - i] = -h[half + i];
  }
}

/* Hilbert<T>::apply, src/filter/hilbert.h:42-54: a full convolution cut to the
 * input length, out[k] = sum_i in[i] h[k-i+half], summed in increasing i.  Taps
 * that are exactly zero add a signed zero and are skipped. */
static void F(hilbert_apply)(const REAL *h, int half, const REAL *in, REAL *out, int n)
{
  for (int k = 0; k < n; k++) {
    int i0 = k - half < 0 ? 0 : k - half;
    int i1 = k + half > n - 1 ? n - 1 : k + half;
    REAL s = KR(0);
    for (int i = i0; i <= i1; i++) {
      REAL hk = h[k - i + half];
      if (hk != KR(0)) s += in[i] * hk;
    }
    out[k] = s;
  }
}

void F(orc_hilbert)(const REAL *in, REAL *out, int n, int half)
{
  REAL *h = F(zalloc)((size_t)(2 * half + 1));
  F(hilbert_taps)(half, h);
  F(hilbert_apply)(h, half, in, out, n);
  free(h);
}

/* Per-shot coefficient fields, src/util/fd.cpp:34-40 and :115-116:
 * vt2 = (v dt)^2, vvzz = vt2/dz^2, vvxx = vt2/dx^2, vel3 = 2/v^3. */
typedef struct {
  REAL *vel, *vt2, *vvzz, *vvxx, *vel3, *w, *u31;
} F(coefs_t);

static void F(coefs_init)(const F(grid_t) *g, const REAL *v, F(coefs_t) *c, int want_vel3)
{
  size_t n = (size_t)g->NX * g->NZ;
  c->vel = F(zalloc)(n); c->vt2 = F(zalloc)(n); c->vvzz = F(zalloc)(n);
  c->vvxx = F(zalloc)(n); c->w = F(zalloc)(n); c->u31 = F(zalloc)(n);
  c->vel3 = want_vel3 ? F(zalloc)(n) : NULL;
  F(orc_set_vel)(v, g->nz, g->nx, g->pml, c->vel);
  F(orc_set_abs)(g->nz, g->nx, g->pml, c->w);
  REAL invdx2 = KR(1.0) / (g->dx * g->dx);
  REAL invdz2 = KR(1.0) / (g->dz * g->dz);
  for (size_t i = 0; i < n; i++) {
    REAL t = c->vel[i] * g->dt;
    c->vt2[i] = t * t;
    c->vvzz[i] = c->vt2[i] * invdz2;
    c->vvxx[i] = c->vt2[i] * invdx2;
    if (want_vel3) c->vel3[i] = KR(2.0) / (c->vel[i] * c->vel[i] * c->vel[i]);
  }
}

static void F(coefs_free)(F(coefs_t) *c)
{
  free(c->vel); free(c->vt2); free(c->vvzz); free(c->vvxx); free(c->w); free(c->u31);
  free(c->vel3);
}

/* Two-way update of the non-frame cells: modeling2D_low on [1,n-2]^2
 * (src/util/fd.cpp:1226-1241), then modeling2D_high on [4,n-5]^2 (:1242-1271).
 * nxt = vvzz*uzz + vvxx*uxx + 2 cur - prv. */
static void F(twoway)(const F(grid_t) *g, const F(coefs_t) *c, const REAL *cur,
                      const REAL *prv, REAL *nxt)
{
  static const REAL a[9] = {KR(-1.0) / KR(560.0), KR(8.0) / KR(315.0), KR(-1.0) / KR(5.0),
                            KR(8.0) / KR(5.0),    KR(-205.0) / KR(72.0), KR(8.0) / KR(5.0),
                            KR(-1.0) / KR(5.0),   KR(8.0) / KR(315.0), KR(-1.0) / KR(560.0)};
  const int NX = g->NX, NZ = g->NZ;
  for (int ix = 1; ix <= NX - 2; ix++)
    for (int iz = 1; iz <= NZ - 2; iz++) {
      REAL u = AT(cur, ix, iz);
      REAL uzz, uxx;
      int high = ix >= 4 && ix <= NX - 5 && iz >= 4 && iz <= NZ - 5;
      if (high) {
        uzz = AT(cur, ix, iz - 4) * a[0];
        uxx = AT(cur, ix - 4, iz) * a[0];
        for (int k = 1; k < 9; k++) {
          uzz = uzz + AT(cur, ix, iz - 4 + k) * a[k];
          uxx = uxx + AT(cur, ix - 4 + k, iz) * a[k];
        }
      } else {
        uzz = AT(cur, ix, iz - 1) + AT(cur, ix, iz + 1) - KR(2) * u;
        uxx = AT(cur, ix + 1, iz) + AT(cur, ix - 1, iz) - KR(2) * u;
      }
      AT(nxt, ix, iz) = AT(c->vvzz, ix, iz) * uzz + AT(c->vvxx, ix, iz) * uxx + KR(2) * u -
                        AT(prv, ix, iz);
    }
}

/* 1-D second difference along an edge: (v v k)((a+b) - 2c). */
static REAL F(d2)(REAL v, REAL k, REAL a, REAL b, REAL c) { return v * v * k * (a + b - KR(2) * c); }

/* Outer frame of the two-way field, processBoundary part (i),
 * src/util/fd.cpp:1057-1091: a 1-D update along each edge (the right column
 * uses the x coefficient, :1066), the four corners as 2 cur - prv, then a
 * linearly extrapolated normal term, z first (:1072-1081) then x (:1082-1091). */
static void F(frame)(const F(grid_t) *g, const F(coefs_t) *c, const REAL *cur,
                     const REAL *prv, REAL *u3)
{
  const int NX = g->NX, NZ = g->NZ;
  const REAL *vel = c->vel;
  REAL dt2 = g->dt * g->dt;
  REAL kx = (KR(1.0) / g->dx) * (KR(1.0) / g->dx) * dt2;
  REAL kz = (KR(1.0) / g->dz) * (KR(1.0) / g->dz) * dt2;
  for (int ix = 1; ix <= NX - 2; ix++) {
    int e[2] = {0, NZ - 1};
    for (int s = 0; s < 2; s++) {
      int iz = e[s];
      AT(u3, ix, iz) = F(d2)(AT(vel, ix, iz), kx, AT(cur, ix + 1, iz), AT(cur, ix - 1, iz),
                             AT(cur, ix, iz)) + KR(2) * AT(cur, ix, iz) - AT(prv, ix, iz);
    }
  }
  for (int iz = 1; iz <= NZ - 2; iz++) {
    AT(u3, 0, iz) = F(d2)(AT(vel, 0, iz), kz, AT(cur, 0, iz + 1), AT(cur, 0, iz - 1),
                          AT(cur, 0, iz)) + KR(2) * AT(cur, 0, iz) - AT(prv, 0, iz);
    AT(u3, NX - 1, iz) = F(d2)(AT(vel, NX - 1, iz), kx, AT(cur, NX - 1, iz + 1),
                               AT(cur, NX - 1, iz - 1), AT(cur, NX - 1, iz)) +
                         KR(2) * AT(cur, NX - 1, iz) - AT(prv, NX - 1, iz);
  }
  {
    int cx[4] = {0, 0, NX - 1, NX - 1}, cz[4] = {0, NZ - 1, 0, NZ - 1};
    for (int k = 0; k < 4; k++)
      AT(u3, cx[k], cz[k]) = KR(2) * AT(cur, cx[k], cz[k]) - AT(prv, cx[k], cz[k]);
  }
  for (int ix = 0; ix < NX; ix++) {
    REAL y1 = F(d2)(AT(vel, ix, 1), kz, AT(cur, ix, 2), AT(cur, ix, 0), AT(cur, ix, 1));
    REAL y2 = F(d2)(AT(vel, ix, 2), kz, AT(cur, ix, 3), AT(cur, ix, 1), AT(cur, ix, 2));
    AT(u3, ix, 0) += y1 * KR(2) - y2;
    y1 = F(d2)(AT(vel, ix, NZ - 2), kz, AT(cur, ix, NZ - 3), AT(cur, ix, NZ - 1), AT(cur, ix, NZ - 2));
    y2 = F(d2)(AT(vel, ix, NZ - 3), kz, AT(cur, ix, NZ - 4), AT(cur, ix, NZ - 2), AT(cur, ix, NZ - 3));
    AT(u3, ix, NZ - 1) += y1 * KR(2) - y2;
  }
  for (int iz = 0; iz < NZ; iz++) {
    REAL y1 = F(d2)(AT(vel, 1, iz), kx, AT(cur, 2, iz), AT(cur, 0, iz), AT(cur, 1, iz));
    REAL y2 = F(d2)(AT(vel, 2, iz), kx, AT(cur, 3, iz), AT(cur, 1, iz), AT(cur, 2, iz));
    AT(u3, 0, iz) += y1 * KR(2) - y2;
    y1 = F(d2)(AT(vel, NX - 2, iz), kx, AT(cur, NX - 3, iz), AT(cur, NX - 1, iz), AT(cur, NX - 2, iz));
    y2 = F(d2)(AT(vel, NX - 3, iz), kx, AT(cur, NX - 4, iz), AT(cur, NX - 2, iz), AT(cur, NX - 3, iz));
    AT(u3, NX - 1, iz) += y1 * KR(2) - y2;
  }
}

/* One-way (paraxial) update of a strip cell, src/util/fd.cpp:1098-1104 and the
 * three mirrored strips.  i = inner neighbour along the normal, t+/t- = the
 * tangential neighbours of the inner cell (u3) and of the cell itself (prv);
 * a1 = 1/(2 h_n dt), a2 = 1/(2 dt^2 v), a3 = v/(4 h_t^2). */
static REAL F(oneway)(REAL a1, REAL a2, REAL a3, REAL u3i, REAL u3tp, REAL u3tm, REAL cK,
                      REAL ci, REAL pK, REAL pi, REAL ptp, REAL ptm)
{
  REAL tmp = -a1 * u3i - a1 * (pK - pi) + a2 * (pK - KR(2) * cK + u3i + pi - KR(2) * ci) -
             a3 * (u3tp + u3tm - KR(2) * u3i + ptp + ptm - KR(2) * pK);
  return -tmp / (a1 + a2);
}

/* Diagonal corner cell, src/util/fd.cpp:1146-1178.  ax3 = sqrt(2)/v/dt is
 * single precision except in the upper-left corner, where the reference writes
 * sqrt(2) with an int argument and so forms ax3 in double (:1176). */
static REAL F(corner)(REAL ax1, REAL ax2, REAL ax3, REAL u3z, REAL u3x, REAL cK)
{
  REAL tmp = -ax1 * u3z - ax2 * u3x + ax3 * (-cK);
  return -tmp / (ax1 + ax2 + ax3);
}

/* processBoundary part (ii), src/util/fd.cpp:1092-1179: one-way field u31 on
 * every ring IK = 1..pml; reads the two-way u3 (frame included), cur, prv. */
static void F(rings)(const F(grid_t) *g, const F(coefs_t) *c, const REAL *u3,
                     const REAL *cur, const REAL *prv, REAL *u31)
{
  const int nx = g->nx, nz = g->nz, pml = g->pml;
  const REAL dt = g->dt, dx = g->dx, dz = g->dz;
  const REAL *vel = c->vel;
  for (int IK = 1; IK <= pml; IK++) {
    int b1 = pml + 1 - IK, b2x = pml + nx + IK - 2, b2z = pml + nz + IK - 2;
    /* up (inner +z) and down (inner -z) */
    for (int s = 0; s < 2; s++) {
      int K = s == 0 ? pml - IK : nz + IK + pml - 1;
      int I = s == 0 ? K + 1 : K - 1;
      for (int ix = b1; ix <= b2x; ix++) {
        REAL v = AT(vel, ix, K);
        REAL a1 = KR(1.0) / dz / KR(2.0) / dt;
        REAL a2 = KR(1.0) / KR(2.0) / dt / dt / v;
        REAL a3 = v / KR(4.0) / dx / dx;
        AT(u31, ix, K) = F(oneway)(a1, a2, a3, AT(u3, ix, I), AT(u3, ix + 1, I), AT(u3, ix - 1, I),
                                   AT(cur, ix, K), AT(cur, ix, I), AT(prv, ix, K), AT(prv, ix, I),
                                   AT(prv, ix + 1, K), AT(prv, ix - 1, K));
      }
    }
    /* right (inner -x) and left (inner +x) */
    for (int s = 0; s < 2; s++) {
      int K = s == 0 ? nx + IK + pml - 1 : pml - IK;
      int I = s == 0 ? K - 1 : K + 1;
      for (int iz = b1; iz <= b2z; iz++) {
        REAL v = AT(vel, K, iz);
        REAL a1 = KR(1.0) / dx / KR(2.0) / dt;
        REAL a2 = KR(1.0) / KR(2.0) / dt / dt / v;
        REAL a3 = v / KR(4.0) / dz / dz;
        AT(u31, K, iz) = F(oneway)(a1, a2, a3, AT(u3, I, iz), AT(u3, I, iz + 1), AT(u3, I, iz - 1),
                                   AT(cur, K, iz), AT(cur, I, iz), AT(prv, K, iz), AT(prv, I, iz),
                                   AT(prv, K, iz + 1), AT(prv, K, iz - 1));
      }
    }
    /* corners: (x, z, inner dx, inner dz) */
    {
      int xr = nx + pml + IK - 1, xl = pml - IK, zd = nz + pml + IK - 1, zu = pml - IK;
      int cxs[4] = {xr, xl, xr, xl}, czs[4] = {zd, zd, zu, zu};
      int dxs[4] = {-1, +1, -1, +1}, dzs[4] = {-1, -1, +1, +1};
      REAL ax1 = KR(1.0) / dz, ax2 = KR(1.0) / dx;
      for (int k = 0; k < 4; k++) {
        int x = cxs[k], z = czs[k];
        REAL v = AT(vel, x, z);
        REAL ax3 = k == 3 ? (REAL)(sqrt(2.0) / (double)v / (double)dt)
                          : SQRTR(KR(2.0)) / v / dt;
        AT(u31, x, z) = F(corner)(ax1, ax2, ax3, AT(u3, x, z + dzs[k]), AT(u3, x + dxs[k], z),
                                  AT(cur, x, z));
      }
    }
  }
}

/* Hybrid absorbing boundary applied to a freshly stepped two-way field:
 * processBoundary (src/util/fd.cpp:1053-1180) then the blend loop
 * u = u w + u31 (1 - w) (:55-56). */
static void F(absorb)(const F(grid_t) *g, const F(coefs_t) *c, REAL *u3, const REAL *cur,
                      const REAL *prv)
{
  F(frame)(g, c, cur, prv, u3);
  F(rings)(g, c, u3, cur, prv, c->u31);
  size_t n = (size_t)g->NX * g->NZ;
  for (size_t i = 0; i < n; i++) u3[i] = u3[i] * c->w[i] + c->u31[i] * (KR(1.0) - c->w[i]);
}

/* modeling, src/util/fd.cpp:15-80.  rec [nx][nt]. */
int F(orc_modeling)(REAL dt, REAL dx, REAL dz, int nt, int ndel, int nx, int nz, int pml,
                    int sx, int sz, const int *gz, const REAL *wav, const REAL *vel, REAL *rec)
{
  F(grid_t) gg = F(mkgrid)(dt, dx, dz, nx, nz, pml);
  const F(grid_t) *g = &gg;
  F(coefs_t) c;
  F(coefs_init)(g, vel, &c, 0);
  size_t n = (size_t)g->NX * g->NZ;
  REAL *u0 = F(zalloc)(n), *u1 = F(zalloc)(n), *u2 = F(zalloc)(n);
  int sxp = sx + pml, szp = sz + pml, NT = nt + ndel;
  for (int it = 0; it < NT; it++) {
    F(twoway)(g, &c, u1, u0, u2);
    if (it >= 1) AT(u2, sxp, szp) += AT(c.vt2, sxp, szp) * wav[it - 1];
    F(absorb)(g, &c, u2, u1, u0);
    if (it >= ndel)
      for (int ix = 0; ix < nx; ix++) rec[(size_t)ix * nt + (it - ndel)] = AT(u2, ix + pml, gz[ix] + pml);
    REAL *t = u0; u0 = u1; u1 = u2; u2 = t;
  }
  free(u0); free(u1); free(u2);
  F(coefs_free)(&c);
  return 0;
}

/* illum, src/util/fd.cpp:275-339: ss[nx][nz] = sum over it > ndel of the
 * blended source field squared, accumulated in REAL step by step. */
/* illum (point source wav at (sx, sz)) and illumPlane (sou != NULL: the areal
 * source sou[ix][it] at every model column of row sz), src/util/fd.cpp:275-339,
 * :720-786: the sum of the squared blended field over steps it > ndel. */
static int F(illum_core)(REAL dt, REAL dx, REAL dz, int nt, int ndel, int nx, int nz, int pml,
                         int sx, int sz, const REAL *wav, const REAL *sou, const REAL *vel,
                         REAL *ss)
{
  F(grid_t) gg = F(mkgrid)(dt, dx, dz, nx, nz, pml);
  const F(grid_t) *g = &gg;
  F(coefs_t) c;
  F(coefs_init)(g, vel, &c, 0);
  size_t n = (size_t)g->NX * g->NZ;
  REAL *u0 = F(zalloc)(n), *u1 = F(zalloc)(n), *u2 = F(zalloc)(n);
  int sxp = sx + pml, szp = sz + pml, NT = nt + ndel;
  for (size_t i = 0; i < (size_t)nx * nz; i++) ss[i] = KR(0);
  for (int it = 0; it < NT; it++) {
    F(twoway)(g, &c, u1, u0, u2);
    if (it >= 1) {
      if (sou) {  /* fd.cpp:754-757 */
        for (int ix = 0; ix < nx; ix++)
          AT(u2, ix + pml, szp) += AT(c.vt2, ix + pml, szp) * sou[(size_t)ix * NT + it - 1];
      } else {
        AT(u2, sxp, szp) += AT(c.vt2, sxp, szp) * wav[it - 1];
      }
    }
    F(absorb)(g, &c, u2, u1, u0);
    if (it > ndel)  /* fd.cpp:318, :763 */
      for (int ix = 0; ix < nx; ix++)
        for (int iz = 0; iz < nz; iz++) {
          REAL u = AT(u2, ix + pml, iz + pml);
          ss[(size_t)ix * nz + iz] += u * u;
        }
    REAL *t = u0; u0 = u1; u1 = u2; u2 = t;
  }
  free(u0); free(u1); free(u2);
  F(coefs_free)(&c);
  return 0;
}

int F(orc_illum)(REAL dt, REAL dx, REAL dz, int nt, int ndel, int nx, int nz, int pml, int sx,
                 int sz, const REAL *wav, const REAL *vel, REAL *ss)
{
  return F(illum_core)(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, wav, NULL, vel, ss);
}

int F(orc_illum_plane)(REAL dt, REAL dx, REAL dz, int nt, int ndel, int nx, int nz, int pml,
                       int sz, const REAL *sou, const REAL *vel, REAL *ss)
{
  return F(illum_core)(dt, dx, dz, nt, ndel, nx, nz, pml, 0, sz, NULL, sou, vel, ss);
}

/* forward (Born), src/util/fd.cpp:81-177.  Scattering source
 * vt2 lap vel3 dv with lap = (u2 + u0 - 2 u1)/dt^2 of the blended background. */
/* Born core: a point source wav at (sx, sz), or (sou != NULL) the areal source
 * of forwordPlane, sou[ix][it] injected at every model column of row sz
 * (src/util/fd.cpp:221-225). */
static int F(born_core)(REAL dt, REAL dx, REAL dz, int nt, int ndel, int nx, int nz, int pml,
                        int sx, int sz, const int *gz, const REAL *wav, const REAL *sou,
                        const REAL *vel, const REAL *dv, REAL *rec)
{
  F(grid_t) gg = F(mkgrid)(dt, dx, dz, nx, nz, pml);
  const F(grid_t) *g = &gg;
  F(coefs_t) c;
  F(coefs_init)(g, vel, &c, 1);
  size_t n = (size_t)g->NX * g->NZ;
  REAL *dvp = F(zalloc)(n);
  F(pad_zero)(g, dv, dvp);
  REAL *u0 = F(zalloc)(n), *u1 = F(zalloc)(n), *u2 = F(zalloc)(n);
  REAL *b0 = F(zalloc)(n), *b1 = F(zalloc)(n), *b2 = F(zalloc)(n);
  REAL idt2 = KR(1.0) / dt / dt;
  int sxp = sx + pml, szp = sz + pml, NT = nt + ndel;
  for (int it = 0; it < NT; it++) {
    F(twoway)(g, &c, u1, u0, u2);
    if (it >= 1) {
      if (sou)
        for (int ix = 0; ix < nx; ix++)
          AT(u2, ix + pml, szp) += AT(c.vt2, ix + pml, szp) * sou[(size_t)ix * NT + (it - 1)];
      else
        AT(u2, sxp, szp) += AT(c.vt2, sxp, szp) * wav[it - 1];
    }
    F(absorb)(g, &c, u2, u1, u0);
    F(twoway)(g, &c, b1, b0, b2);
    for (size_t i = 0; i < n; i++) {
      REAL lap = (u2[i] + u0[i] - KR(2) * u1[i]) * idt2;
      b2[i] += c.vt2[i] * lap * c.vel3[i] * dvp[i];
    }
    F(absorb)(g, &c, b2, b1, b0);
    if (it >= ndel)
      for (int ix = 0; ix < nx; ix++) rec[(size_t)ix * nt + (it - ndel)] = AT(b2, ix + pml, gz[ix] + pml);
    REAL *t = u0; u0 = u1; u1 = u2; u2 = t;
    t = b0; b0 = b1; b1 = b2; b2 = t;
  }
  free(u0); free(u1); free(u2); free(b0); free(b1); free(b2); free(dvp);
  F(coefs_free)(&c);
  return 0;
}

int F(orc_born)(REAL dt, REAL dx, REAL dz, int nt, int ndel, int nx, int nz, int pml, int sx,
                int sz, const int *gz, const REAL *wav, const REAL *vel, const REAL *dv, REAL *rec)
{
  return F(born_core)(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, gz, wav, NULL, vel, dv, rec);
}

/* forwordPlane, src/util/fd.cpp:178-274: Born with the areal source
 * sou[nx][nt+ndel] at row sz and every receiver at row gz. */
int F(orc_born_plane)(REAL dt, REAL dx, REAL dz, int nt, int ndel, int nx, int nz, int pml,
                      int sz, int gz, const REAL *sou, const REAL *vel, const REAL *dv, REAL *rec)
{
  int *g = (int *)malloc(sizeof(int) * (size_t)(nx > 0 ? nx : 1));
  if (!g) return -1;
  for (int ix = 0; ix < nx; ix++) g[ix] = gz;
  int rc = F(born_core)(dt, dx, dz, nt, ndel, nx, nz, pml, 0, sz, g, NULL, sou, vel, dv, rec);
  free(g);
  return rc;
}

/* SaveAtBoundary, src/util/fd.cpp:1181-1225: the 4 outermost interior rows
 * and columns of u, kept per time sample.  Storage here is time-major
 * [it][strip] (the reference keeps time fastest; the values are the same). */
#define ORC_LAYERS 4
static size_t F(strip_len)(const F(grid_t) *g) { return (size_t)ORC_LAYERS * 2 * (g->nx + g->nz); }

static void F(strips)(const F(grid_t) *g, REAL *u, REAL *store, int save)
{
  const int nx = g->nx, nz = g->nz, pml = g->pml;
  size_t k = 0;
#define ORC_MOVE(ix, iz)                                  \
  do {                                                    \
    if (save) store[k] = AT(u, (ix), (iz));               \
    else AT(u, (ix), (iz)) = store[k];                    \
    k++;                                                  \
  } while (0)
  for (int ix = pml; ix < nx + pml; ix++)
    for (int il = 0; il < ORC_LAYERS; il++) {
      ORC_MOVE(ix, pml + il);
      ORC_MOVE(ix, nz + pml - 1 - il);
    }
  for (int il = 0; il < ORC_LAYERS; il++)
    for (int iz = pml; iz < nz + pml; iz++) {
      ORC_MOVE(pml + il, iz);
      ORC_MOVE(nx + pml - 1 - il, iz);
    }
#undef ORC_MOVE
}

/* FaQi, src/util/fd.cpp:1272-1298: out += 0.5 (U R - H[U] H[R]) on interior
 * columns, H = 61-tap Hilbert FIR along z applied to the whole padded column. */
static void F(faqi)(const F(grid_t) *g, const REAL *h, const REAL *U, const REAL *R, REAL *out,
                    REAL *uh, REAL *rh)
{
  const int pml = g->pml, NZ = g->NZ;
  REAL scal = KR(2.0) / KR(4.0);
  for (int ix = pml; ix < g->NX - pml; ix++) {
    F(hilbert_apply)(h, 30, &AT(U, ix, 0), uh, NZ);
    F(hilbert_apply)(h, 30, &AT(R, ix, 0), rh, NZ);
    for (int iz = pml; iz < NZ - pml; iz++)
      AT(out, ix, iz) += scal * (AT(U, ix, iz) * AT(R, ix, iz) - uh[iz] * rh[iz]);
  }
}

/* adjoint (RTM), src/util/fd.cpp:592-719: forward source pass saving the
 * boundary strips; reverse pass rebuilding the source field from the strips
 * (starting from zero fields, subtracting the source), back-propagating the
 * receiver data injected as rec*vt2, and imaging with lap*vel3*R plus FaQi.
 * img [nx][nz]. */
int F(orc_rtm)(REAL dt, REAL dx, REAL dz, int nt, int ndel, int nx, int nz, int pml, int sx,
               int sz, const int *gz, const REAL *wav, const REAL *vel, const REAL *rec, REAL *img)
{
  F(grid_t) gg = F(mkgrid)(dt, dx, dz, nx, nz, pml);
  const F(grid_t) *g = &gg;
  F(coefs_t) c;
  F(coefs_init)(g, vel, &c, 1);
  size_t n = (size_t)g->NX * g->NZ, sl = F(strip_len)(g);
  REAL *u0 = F(zalloc)(n), *u1 = F(zalloc)(n), *u2 = F(zalloc)(n);
  REAL *b0 = F(zalloc)(n), *b1 = F(zalloc)(n), *b2 = F(zalloc)(n);
  REAL *lap = F(zalloc)(n), *imgp = F(zalloc)(n);
  REAL *store = F(zalloc)(sl * (size_t)nt);
  REAL *h = F(zalloc)(61), *uh = F(zalloc)((size_t)g->NZ), *rh = F(zalloc)((size_t)g->NZ);
  F(hilbert_taps)(30, h);
  REAL idt2 = KR(1.0) / dt / dt;
  int sxp = sx + pml, szp = sz + pml, NT = nt + ndel;
  for (int it = 0; it < NT; it++) {
    F(twoway)(g, &c, u1, u0, u2);
    if (it >= 1) AT(u2, sxp, szp) += AT(c.vt2, sxp, szp) * wav[it - 1];
    F(absorb)(g, &c, u2, u1, u0);
    if (it >= ndel) F(strips)(g, u2, store + sl * (size_t)(it - ndel), 1);
    REAL *t = u0; u0 = u1; u1 = u2; u2 = t;
  }
  memset(u0, 0, n * sizeof(REAL)); memset(u1, 0, n * sizeof(REAL)); memset(u2, 0, n * sizeof(REAL));
  for (int it = NT - 1; it >= ndel; it--) {
    if (it - 1 > 0) AT(u2, sxp, szp) -= AT(c.vt2, sxp, szp) * wav[it - 1];
    int itp = it - ndel;
    F(strips)(g, u1, store + sl * (size_t)itp, 0);
    F(twoway)(g, &c, u1, u2, u0);
    F(absorb)(g, &c, u0, u1, u2);
    for (size_t i = 0; i < n; i++) lap[i] = (u2[i] + u0[i] - KR(2) * u1[i]) * idt2;
    F(twoway)(g, &c, b1, b2, b0);
    for (int ix = 0; ix < nx; ix++) {
      int iz = gz[ix] + pml;
      AT(b0, ix + pml, iz) += rec[(size_t)ix * nt + itp] * AT(c.vt2, ix + pml, iz);
    }
    F(absorb)(g, &c, b0, b1, b2);
    for (size_t i = 0; i < n; i++) imgp[i] += lap[i] * c.vel3[i] * b0[i];
    for (size_t i = 0; i < n; i++) lap[i] = lap[i] * c.vel3[i];
    F(faqi)(g, h, lap, b0, imgp, uh, rh);
    REAL *t = u2; u2 = u1; u1 = u0; u0 = t;
    t = b2; b2 = b1; b1 = b0; b0 = t;
  }
  for (int ix = 0; ix < nx; ix++)
    for (int iz = 0; iz < nz; iz++) img[(size_t)ix * nz + iz] = AT(imgp, ix + pml, iz + pml);
  free(u0); free(u1); free(u2); free(b0); free(b1); free(b2); free(lap); free(imgp);
  free(store); free(h); free(uh); free(rh);
  F(coefs_free)(&c);
  return 0;
}

/* rtm_true, src/util/fd.cpp:924-1052: the RTM above with a vertical-dipole
 * receiver injection (-rec vt2/dz at row gz, +rec vt2/dz at row gz + 1) and
 * imaging FaQi(S vel3, R) of the source field itself. */
int F(orc_rtm_true)(REAL dt, REAL dx, REAL dz, int nt, int ndel, int nx, int nz, int pml, int sx,
                    int sz, const int *gz, const REAL *wav, const REAL *vel, const REAL *rec,
                    REAL *img)
{
  F(grid_t) gg = F(mkgrid)(dt, dx, dz, nx, nz, pml);
  const F(grid_t) *g = &gg;
  F(coefs_t) c;
  F(coefs_init)(g, vel, &c, 1);
  size_t n = (size_t)g->NX * g->NZ, sl = F(strip_len)(g);
  REAL *u0 = F(zalloc)(n), *u1 = F(zalloc)(n), *u2 = F(zalloc)(n);
  REAL *b0 = F(zalloc)(n), *b1 = F(zalloc)(n), *b2 = F(zalloc)(n);
  REAL *lap = F(zalloc)(n), *imgp = F(zalloc)(n);
  REAL *store = F(zalloc)(sl * (size_t)nt);
  REAL *h = F(zalloc)(61), *uh = F(zalloc)((size_t)g->NZ), *rh = F(zalloc)((size_t)g->NZ);
  F(hilbert_taps)(30, h);
  int sxp = sx + pml, szp = sz + pml, NT = nt + ndel;
  for (int it = 0; it < NT; it++) {
    F(twoway)(g, &c, u1, u0, u2);
    if (it >= 1) AT(u2, sxp, szp) += AT(c.vt2, sxp, szp) * wav[it - 1];
    F(absorb)(g, &c, u2, u1, u0);
    if (it >= ndel) F(strips)(g, u2, store + sl * (size_t)(it - ndel), 1);
    REAL *t = u0; u0 = u1; u1 = u2; u2 = t;
  }
  memset(u0, 0, n * sizeof(REAL)); memset(u1, 0, n * sizeof(REAL)); memset(u2, 0, n * sizeof(REAL));
  for (int it = NT - 1; it >= ndel; it--) {
    if (it - 1 > 0) AT(u2, sxp, szp) -= AT(c.vt2, sxp, szp) * wav[it - 1];
    int itp = it - ndel;
    F(strips)(g, u1, store + sl * (size_t)itp, 0);
    F(twoway)(g, &c, u1, u2, u0);
    F(absorb)(g, &c, u0, u1, u2);
    F(twoway)(g, &c, b1, b2, b0);
    for (int ix = 0; ix < nx; ix++) {  /* fd.cpp:1003-1008 */
      int iz = gz[ix] + pml;
      AT(b0, ix + pml, iz) -= rec[(size_t)ix * nt + itp] * AT(c.vt2, ix + pml, iz) / dz;
      iz = iz + 1;
      AT(b0, ix + pml, iz) += rec[(size_t)ix * nt + itp] * AT(c.vt2, ix + pml, iz) / dz;
    }
    F(absorb)(g, &c, b0, b1, b2);
    for (size_t i = 0; i < n; i++) lap[i] = u0[i] * c.vel3[i];
    F(faqi)(g, h, lap, b0, imgp, uh, rh);
    REAL *t = u2; u2 = u1; u1 = u0; u0 = t;
    t = b2; b2 = b1; b1 = b0; b0 = t;
  }
  for (int ix = 0; ix < nx; ix++)
    for (int iz = 0; iz < nz; iz++) img[(size_t)ix * nz + iz] = AT(imgp, ix + pml, iz + pml);
  free(u0); free(u1); free(u2); free(b0); free(b1); free(b2); free(lap); free(imgp);
  free(store); free(h); free(uh); free(rh);
  F(coefs_free)(&c);
  return 0;
}

/* adjointUpDown, src/util/fd.cpp:340-591: RTM with the source field S of wav
 * and the source field St of its Hilbert transform wavh, both reconstructed
 * from their boundary layers beside the receiver field R; every reverse step
 * accumulates, with H the 61-tap z-Hilbert filter of each padded column,
 *   c00 += S R,  czz += H[S] H[R],  czt += H[St] R,  ctz += St H[R]
 * and img = c00 - czz + czt + ctz.  comp [4][nx][nz] = c00, czz, ctz, czt
 * (the reference's imagX order, :392-395) on the model grid. */
int F(orc_rtm_updown)(REAL dt, REAL dx, REAL dz, int nt, int ndel, int nx, int nz, int pml,
                      int sx, int sz, const int *gz, const REAL *wav, const REAL *wavh,
                      const REAL *vel, const REAL *rec, REAL *img, REAL *comp)
{
  F(grid_t) gg = F(mkgrid)(dt, dx, dz, nx, nz, pml);
  const F(grid_t) *g = &gg;
  F(coefs_t) c;
  F(coefs_init)(g, vel, &c, 1);
  size_t n = (size_t)g->NX * g->NZ, sl = F(strip_len)(g);
  int NZ = g->NZ;
  REAL *u[3], *t[3], *b[3];
  for (int k = 0; k < 3; k++) { u[k] = F(zalloc)(n); t[k] = F(zalloc)(n); b[k] = F(zalloc)(n); }
  REAL *store = F(zalloc)(sl * (size_t)nt), *store_t = F(zalloc)(sl * (size_t)nt);
  REAL *c4[4];
  for (int k = 0; k < 4; k++) c4[k] = F(zalloc)(n);
  REAL *h = F(zalloc)(61), *sh = F(zalloc)((size_t)NZ), *rh = F(zalloc)((size_t)NZ),
       *sth = F(zalloc)((size_t)NZ);
  F(hilbert_taps)(30, h);
  int sxp = sx + pml, szp = sz + pml, NT = nt + ndel;
  /* forward passes of S and St with their layers (:402-438) */
  for (int pass = 0; pass < 2; pass++) {
    REAL **f = pass ? t : u;
    const REAL *w = pass ? wavh : wav;
    REAL *st = pass ? store_t : store;
    REAL *f0 = f[0], *f1 = f[1], *f2 = f[2];
    for (int it = 0; it < NT; it++) {
      F(twoway)(g, &c, f1, f0, f2);
      if (it >= 1) AT(f2, sxp, szp) += AT(c.vt2, sxp, szp) * w[it - 1];
      F(absorb)(g, &c, f2, f1, f0);
      if (it >= ndel) F(strips)(g, f2, st + sl * (size_t)(it - ndel), 1);
      REAL *q = f0; f0 = f1; f1 = f2; f2 = q;
    }
    memset(f0, 0, n * sizeof(REAL)); memset(f1, 0, n * sizeof(REAL)); memset(f2, 0, n * sizeof(REAL));
    f[0] = f0; f[1] = f1; f[2] = f2;
  }
  REAL *u0 = u[0], *u1 = u[1], *u2 = u[2], *t0 = t[0], *t1 = t[1], *t2 = t[2];
  REAL *b0 = b[0], *b1 = b[1], *b2 = b[2];
  for (int it = NT - 1; it >= ndel; it--) {
    int itp = it - ndel;
    if (it - 1 > 0) AT(u2, sxp, szp) -= AT(c.vt2, sxp, szp) * wav[it - 1];
    F(strips)(g, u1, store + sl * (size_t)itp, 0);
    F(twoway)(g, &c, u1, u2, u0);
    F(absorb)(g, &c, u0, u1, u2);
    if (it - 1 > 0) AT(t2, sxp, szp) -= AT(c.vt2, sxp, szp) * wavh[it - 1];
    F(strips)(g, t1, store_t + sl * (size_t)itp, 0);
    F(twoway)(g, &c, t1, t2, t0);
    F(absorb)(g, &c, t0, t1, t2);
    F(twoway)(g, &c, b1, b2, b0);
    for (int ix = 0; ix < nx; ix++) {
      int iz = gz[ix] + pml;
      AT(b0, ix + pml, iz) += rec[(size_t)ix * nt + itp] * AT(c.vt2, ix + pml, iz);
    }
    F(absorb)(g, &c, b0, b1, b2);
    for (int ix = pml; ix < g->NX - pml; ix++) {  /* :509-521 */
      const REAL *S = u0 + (size_t)ix * NZ, *R = b0 + (size_t)ix * NZ, *St = t0 + (size_t)ix * NZ;
      F(hilbert_apply)(h, 30, S, sh, NZ);
      F(hilbert_apply)(h, 30, R, rh, NZ);
      F(hilbert_apply)(h, 30, St, sth, NZ);
      for (int iz = 0; iz < NZ; iz++) {
        size_t i = (size_t)ix * NZ + iz;
        c4[0][i] += S[iz] * R[iz];
        c4[1][i] += sh[iz] * rh[iz];
        c4[3][i] += sth[iz] * R[iz];
        c4[2][i] += St[iz] * rh[iz];
      }
    }
    REAL *q = u2; u2 = u1; u1 = u0; u0 = q;
    q = b2; b2 = b1; b1 = b0; b0 = q;
    q = t2; t2 = t1; t1 = t0; t0 = q;
  }
  for (int ix = 0; ix < nx; ix++)
    for (int iz = 0; iz < nz; iz++) {
      size_t i = (size_t)(ix + pml) * NZ + (iz + pml);
      img[(size_t)ix * nz + iz] = c4[0][i] - c4[1][i] + c4[3][i] + c4[2][i];
      for (int k = 0; k < 4; k++) comp[((size_t)k * nx + ix) * nz + iz] = c4[k][i];
    }
  free(u0); free(u1); free(u2); free(t0); free(t1); free(t2); free(b0); free(b1); free(b2);
  free(store); free(store_t); free(h); free(sh); free(rh); free(sth);
  for (int k = 0; k < 4; k++) free(c4[k]);
  F(coefs_free)(&c);
  return 0;
}

/* adjointPlane, src/util/fd.cpp:787-921: RTM of the areal source sou[nx][NT]
 * at row sz with receivers at row gz.  The receiver field is propagated back
 * first, keeping its boundary layers per step, then re-propagated forward in
 * step with the source field from those layers; imaging is FaQi alone.  The
 * reference's receiver injections run for negative sample indices too (a stray
 * ';' after the guard, fd.cpp:834, :873) and read outside rec there; this
 * restatement skips those samples, which equals the reference whenever the
 * memory it reads there holds zeros. */
int F(orc_rtm_plane)(REAL dt, REAL dx, REAL dz, int nt, int ndel, int nx, int nz, int pml, int sz,
                     int gz, const REAL *sou, const REAL *vel, const REAL *rec, REAL *img)
{
  F(grid_t) gg = F(mkgrid)(dt, dx, dz, nx, nz, pml);
  const F(grid_t) *g = &gg;
  F(coefs_t) c;
  F(coefs_init)(g, vel, &c, 1);
  int NT = nt + ndel, szp = sz + pml, gzp = gz + pml;
  size_t n = (size_t)g->NX * g->NZ, sl = F(strip_len)(g);
  REAL *u0 = F(zalloc)(n), *u1 = F(zalloc)(n), *u2 = F(zalloc)(n);
  REAL *b0 = F(zalloc)(n), *b1 = F(zalloc)(n), *b2 = F(zalloc)(n);
  REAL *lap = F(zalloc)(n), *imgp = F(zalloc)(n);
  REAL *store = F(zalloc)(sl * (size_t)NT);
  REAL *h = F(zalloc)(61), *uh = F(zalloc)((size_t)g->NZ), *rh = F(zalloc)((size_t)g->NZ);
  F(hilbert_taps)(30, h);
  REAL idt2 = KR(1.0) / dt / dt;
  /* receiver side, back in time (:829-845) */
  for (int it = NT - 1; it >= 0; it--) {
    int itp = it - ndel;
    F(twoway)(g, &c, b1, b2, b0);
    if (itp >= 0)
      for (int ix = 0; ix < nx; ix++)
        AT(b0, ix + pml, gzp) += rec[(size_t)ix * nt + itp] * AT(c.vt2, ix + pml, gzp);
    F(absorb)(g, &c, b0, b1, b2);
    F(strips)(g, b1, store + sl * (size_t)it, 1);
    REAL *t = b2; b2 = b1; b1 = b0; b0 = t;
  }
  { REAL *t = b0; b0 = b1; b1 = b2; b2 = t; }  /* :846-850 */
  memset(b2, 0, n * sizeof(REAL));
  /* source forward, receiver re-propagated from its layers (:853-893) */
  for (int it = 2; it < NT; it++) {
    F(twoway)(g, &c, u1, u0, u2);
    for (int ix = 0; ix < nx; ix++)
      AT(u2, ix + pml, szp) += AT(c.vt2, ix + pml, szp) * sou[(size_t)ix * NT + (it - 1)];
    F(absorb)(g, &c, u2, u1, u0);
    for (size_t i = 0; i < n; i++) lap[i] = (u2[i] + u0[i] - KR(2) * u1[i]) * idt2;
    int itp = it - ndel - 1;
    if (itp >= 0)
      for (int ix = 0; ix < nx; ix++)
        AT(b0, ix + pml, gzp) -= rec[(size_t)ix * nt + itp] * AT(c.vt2, ix + pml, gzp);
    F(twoway)(g, &c, b1, b0, b2);
    F(absorb)(g, &c, b2, b1, b0);
    if (it - ndel > 0) {
      for (size_t i = 0; i < n; i++) lap[i] = lap[i] * c.vel3[i];
      F(faqi)(g, h, lap, b2, imgp, uh, rh);
    }
    REAL *t = u0; u0 = u1; u1 = u2; u2 = t;
    t = b0; b0 = b1; b1 = b2; b2 = t;
    F(strips)(g, b1, store + sl * (size_t)it, 0);
  }
  for (int ix = 0; ix < nx; ix++)
    for (int iz = 0; iz < nz; iz++) img[(size_t)ix * nz + iz] = AT(imgp, ix + pml, iz + pml);
  free(u0); free(u1); free(u2); free(b0); free(b1); free(b2); free(lap); free(imgp);
  free(store); free(h); free(uh); free(rh);
  F(coefs_free)(&c);
  return 0;
}

/* ---------------------------------------------------------------------------
 * Exact adjoint of the Born operator above (no counterpart in the reference,
 * whose adjoint() is a different imaging operator).  Every stage of one
 * forward step is transposed in scatter form, in reverse order:
 *   blend^T  (fd.cpp:55-56):       u3b = w y, u31b = (1-w) y
 *   rings^T  (fd.cpp:1092-1179):   u31 = -tmp/D is linear in its 9 inputs
 *   frame^T and stencil^T (fd.cpp:1057-1091, :1226-1271)
 * The reverse time loop accumulates the adjoint fields; the gradient w.r.t.
 * dv is sum_k vt2 lap_k vel3 * u3b_k over the interior (setDv^T = crop).
 * ------------------------------------------------------------------------- */

/* transposed one-way strip update: s = u31b * (-1/D) */
static void F(oneway_T)(REAL s, REAL a1, REAL a2, REAL a3, REAL *u3i, REAL *u3tp, REAL *u3tm,
                        REAL *cK, REAL *ci, REAL *pK, REAL *pi, REAL *ptp, REAL *ptm)
{
  *u3i += s * (-a1 + a2 + KR(2) * a3);
  *u3tp += s * (-a3);
  *u3tm += s * (-a3);
  *cK += s * (KR(-2) * a2);
  *ci += s * (KR(-2) * a2);
  *pK += s * (-a1 + a2 + KR(2) * a3);
  *pi += s * (a1 + a2);
  *ptp += s * (-a3);
  *ptm += s * (-a3);
}

static void F(rings_T)(const F(grid_t) *g, const F(coefs_t) *c, const REAL *u31b, REAL *u3b,
                       REAL *cb, REAL *pb)
{
  const int nx = g->nx, nz = g->nz, pml = g->pml;
  const REAL dt = g->dt, dx = g->dx, dz = g->dz;
  const REAL *vel = c->vel;
  for (int IK = 1; IK <= pml; IK++) {
    int b1 = pml + 1 - IK, b2x = pml + nx + IK - 2, b2z = pml + nz + IK - 2;
    for (int sd = 0; sd < 2; sd++) {
      int K = sd == 0 ? pml - IK : nz + IK + pml - 1;
      int I = sd == 0 ? K + 1 : K - 1;
      for (int ix = b1; ix <= b2x; ix++) {
        REAL v = AT(vel, ix, K);
        REAL a1 = KR(1.0) / dz / KR(2.0) / dt, a2 = KR(1.0) / KR(2.0) / dt / dt / v;
        REAL a3 = v / KR(4.0) / dx / dx;
        REAL sc = AT(u31b, ix, K) * (KR(-1) / (a1 + a2));
        F(oneway_T)(sc, a1, a2, a3, &AT(u3b, ix, I), &AT(u3b, ix + 1, I), &AT(u3b, ix - 1, I),
                    &AT(cb, ix, K), &AT(cb, ix, I), &AT(pb, ix, K), &AT(pb, ix, I),
                    &AT(pb, ix + 1, K), &AT(pb, ix - 1, K));
      }
    }
    for (int sd = 0; sd < 2; sd++) {
      int K = sd == 0 ? nx + IK + pml - 1 : pml - IK;
      int I = sd == 0 ? K - 1 : K + 1;
      for (int iz = b1; iz <= b2z; iz++) {
        REAL v = AT(vel, K, iz);
        REAL a1 = KR(1.0) / dx / KR(2.0) / dt, a2 = KR(1.0) / KR(2.0) / dt / dt / v;
        REAL a3 = v / KR(4.0) / dz / dz;
        REAL sc = AT(u31b, K, iz) * (KR(-1) / (a1 + a2));
        F(oneway_T)(sc, a1, a2, a3, &AT(u3b, I, iz), &AT(u3b, I, iz + 1), &AT(u3b, I, iz - 1),
                    &AT(cb, K, iz), &AT(cb, I, iz), &AT(pb, K, iz), &AT(pb, I, iz),
                    &AT(pb, K, iz + 1), &AT(pb, K, iz - 1));
      }
    }
    {
      int xr = nx + pml + IK - 1, xl = pml - IK, zd = nz + pml + IK - 1, zu = pml - IK;
      int cxs[4] = {xr, xl, xr, xl}, czs[4] = {zd, zd, zu, zu};
      int dxs[4] = {-1, +1, -1, +1}, dzs[4] = {-1, -1, +1, +1};
      REAL ax1 = KR(1.0) / dz, ax2 = KR(1.0) / dx;
      for (int k = 0; k < 4; k++) {
        int x = cxs[k], z = czs[k];
        REAL v = AT(vel, x, z);
        REAL ax3 = k == 3 ? (REAL)(sqrt(2.0) / (double)v / (double)dt) : SQRTR(KR(2.0)) / v / dt;
        REAL sc = AT(u31b, x, z) * (KR(-1) / (ax1 + ax2 + ax3));
        AT(u3b, x, z + dzs[k]) += sc * (-ax1);
        AT(u3b, x + dxs[k], z) += sc * (-ax2);
        AT(cb, x, z) += sc * (-ax3);
      }
    }
  }
}

/* transposed 1-D second difference term (v v k)((a+b) - 2c) scaled by e */
static void F(d2_T)(REAL e, REAL v, REAL k, REAL *a, REAL *b, REAL *cc)
{
  REAL t = v * v * k * e;
  *a += t;
  *b += t;
  *cc += KR(-2) * t;
}

/* transpose of the frame (fd.cpp:1057-1091): scatter u3b of frame cells */
static void F(frame_T)(const F(grid_t) *g, const F(coefs_t) *c, const REAL *u3b, REAL *cb,
                       REAL *pb)
{
  const int NX = g->NX, NZ = g->NZ;
  const REAL *vel = c->vel;
  REAL dt2 = g->dt * g->dt;
  REAL kx = (KR(1.0) / g->dx) * (KR(1.0) / g->dx) * dt2;
  REAL kz = (KR(1.0) / g->dz) * (KR(1.0) / g->dz) * dt2;
  /* base terms */
  for (int ix = 1; ix <= NX - 2; ix++) {
    int e[2] = {0, NZ - 1};
    for (int sd = 0; sd < 2; sd++) {
      int iz = e[sd];
      REAL ub = AT(u3b, ix, iz);
      F(d2_T)(ub, AT(vel, ix, iz), kx, &AT(cb, ix + 1, iz), &AT(cb, ix - 1, iz), &AT(cb, ix, iz));
      AT(cb, ix, iz) += KR(2) * ub;
      AT(pb, ix, iz) -= ub;
    }
  }
  for (int iz = 1; iz <= NZ - 2; iz++) {
    REAL ub = AT(u3b, 0, iz);
    F(d2_T)(ub, AT(vel, 0, iz), kz, &AT(cb, 0, iz + 1), &AT(cb, 0, iz - 1), &AT(cb, 0, iz));
    AT(cb, 0, iz) += KR(2) * ub;
    AT(pb, 0, iz) -= ub;
    ub = AT(u3b, NX - 1, iz);
    F(d2_T)(ub, AT(vel, NX - 1, iz), kx, &AT(cb, NX - 1, iz + 1), &AT(cb, NX - 1, iz - 1),
            &AT(cb, NX - 1, iz));
    AT(cb, NX - 1, iz) += KR(2) * ub;
    AT(pb, NX - 1, iz) -= ub;
  }
  {
    int cxs[4] = {0, 0, NX - 1, NX - 1}, czs[4] = {0, NZ - 1, 0, NZ - 1};
    for (int k = 0; k < 4; k++) {
      REAL ub = AT(u3b, cxs[k], czs[k]);
      AT(cb, cxs[k], czs[k]) += KR(2) * ub;
      AT(pb, cxs[k], czs[k]) -= ub;
    }
  }
  /* normal extrapolation terms: u3 += 2 y1 - y2 */
  for (int ix = 0; ix < NX; ix++) {
    REAL ub = AT(u3b, ix, 0);
    F(d2_T)(KR(2) * ub, AT(vel, ix, 1), kz, &AT(cb, ix, 2), &AT(cb, ix, 0), &AT(cb, ix, 1));
    F(d2_T)(-ub, AT(vel, ix, 2), kz, &AT(cb, ix, 3), &AT(cb, ix, 1), &AT(cb, ix, 2));
    ub = AT(u3b, ix, NZ - 1);
    F(d2_T)(KR(2) * ub, AT(vel, ix, NZ - 2), kz, &AT(cb, ix, NZ - 3), &AT(cb, ix, NZ - 1),
            &AT(cb, ix, NZ - 2));
    F(d2_T)(-ub, AT(vel, ix, NZ - 3), kz, &AT(cb, ix, NZ - 4), &AT(cb, ix, NZ - 2),
            &AT(cb, ix, NZ - 3));
  }
  for (int iz = 0; iz < NZ; iz++) {
    REAL ub = AT(u3b, 0, iz);
    F(d2_T)(KR(2) * ub, AT(vel, 1, iz), kx, &AT(cb, 2, iz), &AT(cb, 0, iz), &AT(cb, 1, iz));
    F(d2_T)(-ub, AT(vel, 2, iz), kx, &AT(cb, 3, iz), &AT(cb, 1, iz), &AT(cb, 2, iz));
    ub = AT(u3b, NX - 1, iz);
    F(d2_T)(KR(2) * ub, AT(vel, NX - 2, iz), kx, &AT(cb, NX - 3, iz), &AT(cb, NX - 1, iz),
            &AT(cb, NX - 2, iz));
    F(d2_T)(-ub, AT(vel, NX - 3, iz), kx, &AT(cb, NX - 4, iz), &AT(cb, NX - 2, iz),
            &AT(cb, NX - 3, iz));
  }
}

/* transpose of the two-way stencil on [1,n-2]^2 (fd.cpp:1226-1271) */
static void F(twoway_T)(const F(grid_t) *g, const F(coefs_t) *c, const REAL *u3b, REAL *cb,
                        REAL *pb)
{
  static const REAL a[9] = {KR(-1.0) / KR(560.0), KR(8.0) / KR(315.0), KR(-1.0) / KR(5.0),
                            KR(8.0) / KR(5.0),    KR(-205.0) / KR(72.0), KR(8.0) / KR(5.0),
                            KR(-1.0) / KR(5.0),   KR(8.0) / KR(315.0), KR(-1.0) / KR(560.0)};
  const int NX = g->NX, NZ = g->NZ;
  for (int ix = 1; ix <= NX - 2; ix++)
    for (int iz = 1; iz <= NZ - 2; iz++) {
      REAL ub = AT(u3b, ix, iz);
      REAL vz = AT(c->vvzz, ix, iz) * ub, vx = AT(c->vvxx, ix, iz) * ub;
      int high = ix >= 4 && ix <= NX - 5 && iz >= 4 && iz <= NZ - 5;
      if (high) {
        for (int k = 0; k < 9; k++) {
          AT(cb, ix, iz - 4 + k) += a[k] * vz;
          AT(cb, ix - 4 + k, iz) += a[k] * vx;
        }
      } else {
        AT(cb, ix, iz - 1) += vz;
        AT(cb, ix, iz + 1) += vz;
        AT(cb, ix, iz) += KR(-2) * vz;
        AT(cb, ix + 1, iz) += vx;
        AT(cb, ix - 1, iz) += vx;
        AT(cb, ix, iz) += KR(-2) * vx;
      }
      AT(cb, ix, iz) += KR(2) * ub;
      AT(pb, ix, iz) -= ub;
    }
}

/* Transpose of one forward step: from yb (adjoint of the new field) add the
 * adjoints of the current field (cb) and of the previous one (pb); u3b gets
 * the adjoint of the two-way value before the blend (where sources enter). */
static void F(step_T)(const F(grid_t) *g, const F(coefs_t) *c, const REAL *yb, REAL *cb, REAL *pb,
                      REAL *u3b, REAL *u31b)
{
  size_t n = (size_t)g->NX * g->NZ;
  for (size_t i = 0; i < n; i++) {
    u3b[i] = yb[i] * c->w[i];
    u31b[i] = yb[i] * (KR(1.0) - c->w[i]);
  }
  /* u31 of non-ring cells never reaches the output (w = 1 there) */
  F(rings_T)(g, c, u31b, u3b, cb, pb);
  F(frame_T)(g, c, u3b, cb, pb);
  F(twoway_T)(g, c, u3b, cb, pb);
}

/* Weight of step k in the imaging sum over k = 0..K when only every m-th
 * step (and step K) of the source term is kept: trapezoid weights over the
 * kept steps, plus 1/2 at each end, summing to K + 1 (1 everywhere for m = 1).
 * This is the library's own thinning rule, restated. */
static double F(thin_weight)(int k, int K, int m)
{
  if (m == 1) return 1.0;
  if (k % m != 0 && k != K) return 0.0;
  int prev = k == 0 ? k : (k % m == 0 ? k - m : (K / m) * m);
  int next = k == K ? k : (k + m < K ? k + m : K);
  return 0.5 * (double)(next - prev + (k == 0) + (k == K));
}

/* Exact adjoint of orc_born: img[nx][nz] = L^T rec.  With every > 1 the
 * imaging sum keeps only the thinned steps (weights above): the same
 * operator with the source term sampled as the library samples it. */
int F(orc_born_adjoint_thin)(REAL dt, REAL dx, REAL dz, int nt, int ndel, int nx, int nz,
                             int pml, int sx, int sz, const int *gz, const REAL *wav,
                             const REAL *vel, const REAL *rec, int every, REAL *img)
{
  if (every < 1) return -2;
  F(grid_t) gg = F(mkgrid)(dt, dx, dz, nx, nz, pml);
  const F(grid_t) *g = &gg;
  F(coefs_t) c;
  F(coefs_init)(g, vel, &c, 1);
  size_t n = (size_t)g->NX * g->NZ;
  int sxp = sx + pml, szp = sz + pml, NT = nt + ndel;
  REAL idt2 = KR(1.0) / dt / dt;
  /* background pass, keeping lap_k of every step (small problems only) */
  REAL *laps = F(zalloc)(n * (size_t)NT);
  if (!laps) return -1;
  REAL *u0 = F(zalloc)(n), *u1 = F(zalloc)(n), *u2 = F(zalloc)(n);
  for (int it = 0; it < NT; it++) {
    F(twoway)(g, &c, u1, u0, u2);
    if (it >= 1) AT(u2, sxp, szp) += AT(c.vt2, sxp, szp) * wav[it - 1];
    F(absorb)(g, &c, u2, u1, u0);
    for (size_t i = 0; i < n; i++) laps[(size_t)it * n + i] = (u2[i] + u0[i] - KR(2) * u1[i]) * idt2;
    REAL *t = u0; u0 = u1; u1 = u2; u2 = t;
  }
  /* reverse sweep: A = adjoint of x_{k+1}, B of x_k, C of x_{k-1} */
  REAL *A = u0, *B = u1, *C = u2;
  memset(A, 0, n * sizeof(REAL)); memset(B, 0, n * sizeof(REAL)); memset(C, 0, n * sizeof(REAL));
  REAL *u3b = F(zalloc)(n), *u31b = F(zalloc)(n), *gp = F(zalloc)(n);
  for (int k = NT - 1; k >= 0; k--) {
    if (k >= ndel)
      for (int ix = 0; ix < nx; ix++) AT(A, ix + pml, gz[ix] + pml) += rec[(size_t)ix * nt + (k - ndel)];
    F(step_T)(g, &c, A, B, C, u3b, u31b);
    const REAL *lap = laps + (size_t)k * n;
    const REAL wk = (REAL)F(thin_weight)(k, NT - 1, every);
    if (wk != KR(0))
      for (size_t i = 0; i < n; i++) gp[i] += wk * lap[i] * u3b[i];
    REAL *t = A; A = B; B = C; C = t;
    memset(C, 0, n * sizeof(REAL));
  }
  for (int ix = 0; ix < nx; ix++)
    for (int iz = 0; iz < nz; iz++) {
      int jx = ix + pml, jz = iz + pml;
      img[(size_t)ix * nz + iz] = AT(c.vt2, jx, jz) * AT(c.vel3, jx, jz) * AT(gp, jx, jz);
    }
  free(laps); free(u0); free(u1); free(u2); free(u3b); free(u31b); free(gp);
  F(coefs_free)(&c);
  return 0;
}

/* The same operator as orc_born_adjoint_thin with every = 1, for grids whose
 * source terms of all steps do not fit in host memory: the background pass
 * keeps its two time levels before every ck-th step, and the reverse sweep
 * recomputes the source terms of one ck-step segment at a time from them.
 * The recomputed terms are the stored ones, so the image is the same bit for
 * bit. */
int F(orc_born_adjoint_ck)(REAL dt, REAL dx, REAL dz, int nt, int ndel, int nx, int nz,
                           int pml, int sx, int sz, const int *gz, const REAL *wav,
                           const REAL *vel, const REAL *rec, int ck, REAL *img)
{
  if (ck < 1) return -2;
  F(grid_t) gg = F(mkgrid)(dt, dx, dz, nx, nz, pml);
  const F(grid_t) *g = &gg;
  F(coefs_t) c;
  F(coefs_init)(g, vel, &c, 1);
  size_t n = (size_t)g->NX * g->NZ;
  int sxp = sx + pml, szp = sz + pml, NT = nt + ndel;
  int nseg = (NT + ck - 1) / ck;
  REAL idt2 = KR(1.0) / dt / dt;
  REAL *states = F(zalloc)(2 * n * (size_t)nseg);  /* (u0, u1) before step s*ck */
  REAL *laps = F(zalloc)(n * (size_t)ck);
  REAL *u0 = F(zalloc)(n), *u1 = F(zalloc)(n), *u2 = F(zalloc)(n);
  if (!states || !laps || !u0 || !u1 || !u2) return -1;
  for (int it = 0; it < NT; it++) {
    if (it % ck == 0) {
      memcpy(states + 2 * n * (size_t)(it / ck), u0, n * sizeof(REAL));
      memcpy(states + 2 * n * (size_t)(it / ck) + n, u1, n * sizeof(REAL));
    }
    F(twoway)(g, &c, u1, u0, u2);
    if (it >= 1) AT(u2, sxp, szp) += AT(c.vt2, sxp, szp) * wav[it - 1];
    F(absorb)(g, &c, u2, u1, u0);
    REAL *t = u0; u0 = u1; u1 = u2; u2 = t;
  }
  REAL *A = F(zalloc)(n), *B = F(zalloc)(n), *C = F(zalloc)(n);
  REAL *u3b = F(zalloc)(n), *u31b = F(zalloc)(n), *gp = F(zalloc)(n);
  int seg = -1;
  for (int k = NT - 1; k >= 0; k--) {
    if (k / ck != seg) {  /* recompute the source terms of steps s0 .. k */
      seg = k / ck;
      int s0 = seg * ck;
      memcpy(u0, states + 2 * n * (size_t)seg, n * sizeof(REAL));
      memcpy(u1, states + 2 * n * (size_t)seg + n, n * sizeof(REAL));
      for (int it = s0; it <= k; it++) {
        F(twoway)(g, &c, u1, u0, u2);
        if (it >= 1) AT(u2, sxp, szp) += AT(c.vt2, sxp, szp) * wav[it - 1];
        F(absorb)(g, &c, u2, u1, u0);
        for (size_t i = 0; i < n; i++)
          laps[(size_t)(it - s0) * n + i] = (u2[i] + u0[i] - KR(2) * u1[i]) * idt2;
        REAL *t = u0; u0 = u1; u1 = u2; u2 = t;
      }
    }
    if (k >= ndel)
      for (int ix = 0; ix < nx; ix++) AT(A, ix + pml, gz[ix] + pml) += rec[(size_t)ix * nt + (k - ndel)];
    F(step_T)(g, &c, A, B, C, u3b, u31b);
    const REAL *lap = laps + (size_t)(k - seg * ck) * n;
    for (size_t i = 0; i < n; i++) gp[i] += KR(1) * lap[i] * u3b[i];
    REAL *t = A; A = B; B = C; C = t;
    memset(C, 0, n * sizeof(REAL));
  }
  for (int ix = 0; ix < nx; ix++)
    for (int iz = 0; iz < nz; iz++) {
      int jx = ix + pml, jz = iz + pml;
      img[(size_t)ix * nz + iz] = AT(c.vt2, jx, jz) * AT(c.vel3, jx, jz) * AT(gp, jx, jz);
    }
  free(states); free(laps); free(u0); free(u1); free(u2);
  free(A); free(B); free(C); free(u3b); free(u31b); free(gp);
  F(coefs_free)(&c);
  return 0;
}

int F(orc_born_adjoint)(REAL dt, REAL dx, REAL dz, int nt, int ndel, int nx, int nz, int pml,
                        int sx, int sz, const int *gz, const REAL *wav, const REAL *vel,
                        const REAL *rec, REAL *img)
{
  return F(orc_born_adjoint_thin)(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, gz, wav, vel, rec,
                                  1, img);
}

#undef AT
#undef KR
#undef F
#undef CAT
#undef CAT_
