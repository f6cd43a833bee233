/*
 * Flat-array entry points onto the reference's own per-shot geometry members
 * (Inversion::getVel, getIgz, swapReord, swapModel, removeDirect in
 * src/lsrtm/inversion.cpp), its parameter-file parser (src/util/parser.cpp,
 * through Inversion::readParamFile) and its coordinate-file reader
 * (src/util/coord.cpp).  Test infrastructure only: the tests call these to pin
 * the library's geometry and shot driver against the reference on the same
 * inputs.  Compiled with -Dprivate=public so that the class's members and
 * fields are reachable.  A failed reference check() throws (ref_shim.cpp);
 * every entry point turns that into a -1 return.
 */
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "coord.h"
#include "inversion.h"
#include "memory.h"

namespace {

// row pointers of a flat [n2][n1] array, as MyAlloc<T>::alc(n1, n2) lays it out
template <class T>
std::vector<T *> rows(T *flat, int n1, int n2) {
  std::vector<T *> r((size_t)n2);
  for (int i = 0; i < n2; i++) r[(size_t)i] = flat + (size_t)i * n1;
  return r;
}

}  // namespace

extern "C" {

/* A reference Inversion with ns shots: ng[ns], sc[ns][2] (x, z), gc[ns][2][ngmax]
 * (x row, z row), and the scalars the geometry members read from param. */
void *ref_inv_create(int ns, int ngmax, const int *ng, const float *sc, const float *gc, float dx,
                     float dz, float dt, float fr, float velfx, int nx, int nz, int nt, int delay,
                     int lpad, int rpad) {
  Inversion *v = new Inversion(0, 1);
  v->ng = MyAlloc<int>::alc(ns);
  v->sc = MyAlloc<float>::alc(2, ns);
  v->gc = MyAlloc<float>::alc(ngmax, 2, ns);
  for (int is = 0; is < ns; is++) {
    v->ng[is] = ng[is];
    v->sc[is][0] = sc[2 * is];
    v->sc[is][1] = sc[2 * is + 1];
    for (int k = 0; k < 2; k++)
      for (int ig = 0; ig < ngmax; ig++)
        v->gc[is][k][ig] = gc[((size_t)is * 2 + k) * ngmax + ig];
  }
  v->param.dx.val = dx;
  v->param.dz.val = dz;
  v->param.dt.val = dt;
  v->param.fr.val = fr;
  v->param.velfx.val = velfx;
  v->param.nx.val = nx;
  v->param.nz.val = nz;
  v->param.nt.val = nt;
  v->param.delay.val = delay;
  v->param.lpad.val = lpad;
  v->param.rpad.val = rpad;
  v->param.ns.val = ns;
  v->param.ngmax.val = ngmax;
  return v;
}

void ref_inv_destroy(void *h) { delete static_cast<Inversion *>(h); }

/* getVel: sub-grid of vel [nx][nz]; copies it into out (cap floats) */
int ref_inv_getvel(void *h, int is, const float *vel, int nz, int nx, float velfx, float *fx_sub,
                   int *nx_sub, float *out, size_t cap) {
  try {
    Inversion *v = static_cast<Inversion *>(h);
    std::vector<float> buf(vel, vel + (size_t)nx * nz);
    std::vector<float *> r = rows(buf.data(), nz, nx);
    int nzs = 0, nxs = 0;
    float fxs = 0.0f;
    float **sub = v->getVel(fxs, nzs, nxs, r.data(), nz, nx, velfx, is);
    *fx_sub = fxs;
    *nx_sub = nxs;
    if ((size_t)nxs * nzs <= cap) std::memcpy(out, sub[0], sizeof(float) * (size_t)nxs * nzs);
    MyAlloc<float>::free(sub);
    return 0;
  } catch (...) {
    return -1;
  }
}

int ref_inv_getigz(void *h, float fx_sub, int nx_sub, int is, int *out) {
  try {
    int *igz = static_cast<Inversion *>(h)->getIgz(fx_sub, nx_sub, is);
    std::memcpy(out, igz, sizeof(int) * nx_sub);
    MyAlloc<int>::free(igz);
    return 0;
  } catch (...) {
    return -1;
  }
}

/* swapReord over csg [ng][nt] and rec [nx][nt] */
int ref_inv_swapreord(void *h, float *csg, int is, int ng, int nt, float *rec, float fx, int nx,
                      int adj) {
  try {
    std::vector<float *> c = rows(csg, nt, ng), r = rows(rec, nt, nx);
    static_cast<Inversion *>(h)->swapReord(c.data(), is, ng, nt, r.data(), fx, nx, adj != 0);
    return 0;
  } catch (...) {
    return -1;
  }
}

int ref_inv_swapmodel(void *h, float *m, float *d, float mfx, float dfx, int nzm, int nxm, int nzd,
                      int nxd, int add) {
  try {
    std::vector<float *> a = rows(m, nzm, nxm), b = rows(d, nzd, nxd);
    static_cast<Inversion *>(h)->swapModel(a.data(), b.data(), mfx, dfx, nzm, nxm, nzd, nxd,
                                           add != 0);
    return 0;
  } catch (...) {
    return -1;
  }
}

/* removeDirect over csg [ng[is]][nt] with the global model v [nx][nz] */
int ref_inv_removedirect(void *h, float *csg, float *v, int is) {
  try {
    Inversion *inv = static_cast<Inversion *>(h);
    std::vector<float *> c = rows(csg, inv->param.nt.val, inv->ng[is]);
    std::vector<float *> r = rows(v, inv->param.nz.val, inv->param.nx.val);
    inv->removeDirect(c.data(), r.data(), is);
    return 0;
  } catch (...) {
    return -1;
  }
}

/* readParamFile: the parameter values the reference reads from a file, as
 * ints[16] (nthread ns ngmax nx nz nt npml delay delaycal mask maxiter lpad
 * rpad planeTag sbegin send), floats[5] (dx dz dt fr velfx) and strings[7]
 * (precsg wdir v0file vfile coordfile maskfile, then np/dp/pmin unused) each
 * copied into a 256-byte slot of strs. */
int ref_param_read(const char *file, int *ints, float *floats, char *strs) {
  try {
    Inversion v(1, 1);  // rank 1: no parameter printout
    v.readParamFile(file);
    const paramLSRTM &p = v.param;
    const int iv[16] = {p.nthread.val, p.ns.val,   p.ngmax.val,   p.nx.val,       p.nz.val,
                        p.nt.val,      p.npml.val, p.delay.val,   p.delaycal.val, p.mask.val,
                        p.maxiter.val, p.lpad.val, p.rpad.val,    p.planeTag.val, p.sbegin.val,
                        p.send.val};
    std::memcpy(ints, iv, sizeof iv);
    const float fv[5] = {p.dx.val, p.dz.val, p.dt.val, p.fr.val, p.velfx.val};
    std::memcpy(floats, fv, sizeof fv);
    const std::string sv[6] = {p.precsg.val,  p.wdir.val,      p.v0file.val,
                               p.vfile.val,   p.coordfile.val, p.maskfile.val};
    for (int i = 0; i < 6; i++) {
      std::strncpy(strs + 256 * i, sv[i].c_str(), 255);
      strs[256 * i + 255] = '\0';
    }
    return 0;
  } catch (...) {
    return -1;
  }
}

/* planeWavePrepare (inversion.cpp:808-912) of a parameter file's survey: reads
 * its precsg<is>.dat files and writes PLANE_S_NEW / PLANE_R_NEW into its wdir. */
int ref_plane_prepare(const char *param_file) {
  std::streambuf *keep = getenv("SEIS_REF_VERBOSE") ? std::cout.rdbuf() : std::cout.rdbuf(nullptr);
  int rc = 0;
  try {
    Inversion v(0, 1);
    v.readParamFile(param_file);
    v.getConfig();
    v.planeWavePrepare();
  } catch (...) {
    rc = -1;
  }
  std::cout.rdbuf(keep);
  return rc;
}

/* Coords: number of shots, then receivers per shot, sources and receivers
 * (gc [ns][2][ngmax] with the reference's -1e10 fill). */
int ref_coords_count(const char *file, int *ns) {
  try {
    *ns = Coords::countShots(file);
    return 0;
  } catch (...) {
    return -1;
  }
}

int ref_coords_read(const char *file, int ns, int ngmax, int *ng, float *sc, float *gc) {
  try {
    int *n = 0;
    Coords::countReceivers(file, ns, n);
    std::memcpy(ng, n, sizeof(int) * ns);
    float **s = 0;
    Coords::getSources(file, ns, s);
    for (int is = 0; is < ns; is++) {
      sc[2 * is] = s[is][0];
      sc[2 * is + 1] = s[is][1];
    }
    // getConfig lets getReceivers size the array itself (max of ng)
    float ***g = 0;
    Coords::getReceivers(file, ns, n, g);
    int ngm = 0;
    for (int is = 0; is < ns; is++) ngm = n[is] > ngm ? n[is] : ngm;
    for (size_t i = 0; i < (size_t)ns * 2 * ngmax; i++) gc[i] = -1e10f;
    for (int is = 0; is < ns; is++)
      for (int k = 0; k < 2; k++)
        for (int ig = 0; ig < ngm && ig < ngmax; ig++)
          gc[((size_t)is * 2 + k) * ngmax + ig] = g[is][k][ig];
    MyAlloc<int>::free(n);
    MyAlloc<float>::free(s);
    MyAlloc<float>::free(g);
    return 0;
  } catch (...) {
    return -1;
  }
}

}  // extern "C"
