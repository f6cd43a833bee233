// Per-shot acquisition geometry (seis_geom.h).  Every expression keeps the
// reference's types: float arithmetic where it computes in float, double where
// a double literal promotes it (0.001*dx, 5.0, "- 0.0"), truncation toward
// zero on conversion to int.  The line cited with each function is the
// reference statement it reproduces.
#include "seis_geom.h"

#include <cmath>
#include <cstring>
#include <vector>

#include "seis_fd.h"

namespace {

inline float fmin2(float a, float b) { return a < b ? a : b; }  // arraymath.h:21-25
inline float fmax2(float a, float b) { return a > b ? a : b; }

// lower / upper x of a grid of n columns from fx, widened by a thousandth of
// a cell (inversion.cpp:604-605, :630-631, :650-651)
inline float lo_edge(float fx, float dx) { return (float)((double)fx - 0.001 * (double)dx); }
inline float hi_edge(float fx, int n, float dx) {
  const float last = fx + (float)(n - 1) * dx;
  return (float)((double)last + 0.001 * (double)dx);
}

}  // namespace

extern "C" {

int seis_geom_aperture(float sx, const float *gx, int ng, float dx, int lpad, int rpad,
                       float *fx_sub, int *nx_sub) {
  if (!gx || ng < 1 || !fx_sub || !nx_sub || !(dx > 0.0f)) return SEIS_ERR_ARG;
  float gmin = gx[0], gmax = gx[0];  // arraymath.h:57-64 (first minimum kept)
  for (int i = 1; i < ng; i++) {
    gmin = gmin > gx[i] ? gx[i] : gmin;
    gmax = gmax < gx[i] ? gx[i] : gmax;
  }
  const float x_min = fmin2(sx, gmin), x_max = fmax2(sx, gmax);  // :558-561
  const float lo = x_min - (float)lpad * dx, hi = x_max + (float)rpad * dx;  // :562-563
  *fx_sub = lo;                                                                  // :566
  *nx_sub = (int)((hi - lo) / dx + 1.0f);                                        // :568
  return *nx_sub >= 1 ? SEIS_OK : SEIS_ERR_ARG;
}

int seis_geom_extract_columns(int nx, float fx, float dx, float fx_sub, int nx_sub, int *cols) {
  if (!cols || nx < 1 || nx_sub < 1 || !(dx > 0.0f)) return SEIS_ERR_ARG;
  const float lo = fx + dx;                            // :564
  const float hi = fx + (float)(nx - 1) * dx - dx;     // :565
  for (int ix = 0; ix < nx_sub; ix++) {
    const float x = fx_sub + (float)ix * dx;           // :572-573
    if (x != x) return SEIS_ERR_ARG;                   // :594-597
    float at = x;
    if (!(x >= lo && x <= hi)) at = x < lo ? lo : hi;  // :579-593 (clamp)
    const int col = (int)((at - fx) / dx);
    if (col < 0 || col >= nx) return SEIS_ERR_ARG;
    cols[ix] = col;
  }
  return SEIS_OK;
}

int seis_geom_extract(const float *model, int nz, int nx, float fx, float dx, float fx_sub,
                      int nx_sub, float *sub) {
  if (!model || !sub || nz < 1 || nx < 1 || nx_sub < 1 || !(dx > 0.0f)) return SEIS_ERR_ARG;
  std::vector<int> cols((size_t)nx_sub);
  int rc = seis_geom_extract_columns(nx, fx, dx, fx_sub, nx_sub, cols.data());
  if (rc) return rc;
  for (int ix = 0; ix < nx_sub; ix++)
    std::memcpy(sub + (size_t)ix * nz, model + (size_t)cols[ix] * nz, sizeof(float) * nz);
  return SEIS_OK;
}

int seis_geom_receiver_rows(const float *gx, const float *gz, int ng, float fx_sub, int nx_sub,
                            float dx, float dz, int nz, int *igz) {
  if (!igz || nx_sub < 1 || ng < 0 || (ng > 0 && (!gx || !gz))) return SEIS_ERR_ARG;
  const float lo = lo_edge(fx_sub, dx), hi = hi_edge(fx_sub, nx_sub, dx);  // :604-605
  for (int ix = 0; ix < nx_sub; ix++) igz[ix] = 0;
  for (int ig = 0; ig < ng; ig++) {
    const float x = gx[ig], z = gz[ig];
    if (!(x >= lo && x <= hi)) continue;
    const int col = (int)((x - lo) / dx + 0.1f);      // :614
    const int row = (int)((z - 0.0f) / dz + 0.1f);    // :615
    if (col < 0 || col >= nx_sub || row < 0 || row >= nz) return SEIS_ERR_ARG;
    igz[col] = row;
  }
  return SEIS_OK;
}

int seis_geom_source_index(float sx, float sz, float fx_sub, float dx, float dz, int *isx,
                           int *isz) {
  if (!isx || !isz) return SEIS_ERR_ARG;
  *isx = (int)((sx - fx_sub) / dx + 0.0001f);                          // :428
  *isz = (int)(((double)sz - 0.0) / (double)dz + (double)0.0001f);     // :429
  return SEIS_OK;
}

int seis_geom_reorder(float *csg, int ng, int nt, const float *gx, float *rec, float fx, int nx,
                      float dx, int to_gather) {
  if (!csg || !rec || (ng > 0 && !gx) || nt < 1 || nx < 1) return SEIS_ERR_ARG;
  if (to_gather)
    std::memset(csg, 0, sizeof(float) * (size_t)ng * nt);   // :628
  else
    std::memset(rec, 0, sizeof(float) * (size_t)nx * nt);
  const float lo = lo_edge(fx, dx), hi = hi_edge(fx, nx, dx);  // :630-631
  for (int ig = 0; ig < ng; ig++) {
    const float x = gx[ig];
    if (!(lo <= x && x <= hi)) continue;
    const int col = (int)((x - lo) / dx + 0.1f);            // :637
    if (col < 0 || col >= nx) return SEIS_ERR_ARG;
    float *tr = csg + (size_t)ig * nt, *cl = rec + (size_t)col * nt;
    if (to_gather)
      std::memcpy(tr, cl, sizeof(float) * nt);
    else
      std::memcpy(cl, tr, sizeof(float) * nt);
  }
  return SEIS_OK;
}

int seis_geom_swap_model(const float *m, float *d, float mfx, float dfx, int nzm, int nxm, int nzd,
                         int nxd, float dx, int add) {
  const int layer = 4;
  if (!m || !d || nzm != nzd || nxm < 1 || nxd < 1) return SEIS_ERR_ARG;  // :647
  if (!add) std::memset(d, 0, sizeof(float) * (size_t)nxd * nzd);
  const float lo = lo_edge(mfx, dx), hi = hi_edge(mfx, nxm, dx);         // :651-652
  for (int ix = layer; ix < nxd - layer; ix++) {
    const float x = dfx + (float)(ix - 1) * dx;                            // :655
    if (!(x >= lo && x <= hi)) continue;
    const int col = (int)((x - lo) / dx + 0.0001f);                        // :658
    if (col < 0 || col >= nxm) return SEIS_ERR_ARG;
    if (col < 4 || col > nxm - 4) continue;                                // :660
    const float *src = m + (size_t)col * nzm;
    float *dst = d + (size_t)ix * nzd;
    for (int iz = layer; iz < nzd - layer; iz++) dst[iz] += src[iz];
  }
  return SEIS_OK;
}

int seis_geom_remove_direct(float *csg, int ng, int nt, const float *gx, const float *gz, float sx,
                            float sz, const float *v, int nz, int nx, float dx, float dz, float dt,
                            float fr, float velfx, int delay) {
  if (!csg || !v || (ng > 0 && (!gx || !gz)) || nt < 1 || nx < 1 || nz < 1) return SEIS_ERR_ARG;
  const int isx = (int)((sx - velfx) / dx + 0.0001f);                     // :712
  for (int ig = 0; ig < ng; ig++) {
    float t = 0.0f;
    const int igx = (int)((gx[ig] - velfx) / dx + 0.0001f);                // :719
    const int igz = (int)((gz[ig] - 0.0f) / dz + 0.0001f);                 // :720
    int adddelay = (int)std::fabs((gz[ig] - sz) / dz + 0.0001f);          // :721
    adddelay += 10;
    if (igz < 0 || igz >= nz) return SEIS_ERR_ARG;                         // :725
    auto slow = [&](int i) -> float {  // dx / v along the receiver row, :728-734
      if (i >= 0 && i < nx) return dx / v[(size_t)i * nz + igz];
      if (igx < 0) return dx / v[igz];
      if (igx >= nx) return dx / v[(size_t)(nx - 1) * nz + igz];
      return 0.0f;
    };
    if (igx <= isx) {
      for (int i = igx; i < isx; i++) {
        if ((i >= 0 && i < nx) || igx < 0 || igx >= nx) t += slow(i);
      }
    } else {
      for (int i = igx; i > isx; i--) {
        if ((i >= 0 && i < nx) || igx < 0 || igx >= nx) t += slow(i);
      }
    }
    // :746: float sum of the first three terms, then a double term
    const float head = t / dt + (float)delay + (float)adddelay;
    const double tail = (double)(1.0f / fr / dt * 0.5f) * 5.0;
    int it = (int)((double)head + tail + (double)0.0001f);
    it = it <= nt - 1 ? it : nt - 1;
    it = it >= 1 ? it : 1;
    std::memset(csg + (size_t)ig * nt, 0, sizeof(float) * it);
  }
  return SEIS_OK;
}

}  // extern "C"
