/*
 * Flat-array C entry points around the reference's FD functions, so that
 * Python tests and the CPU baseline can call the reference unmodified
 * (test infrastructure only; compiled into oracle/_ref/libseisref.so).
 *
 * Arrays follow the reference layout: model/image [nx][nz] with z fastest
 * (MyAlloc<float>::alc(nz,nx), src/util/memory.h:29-44), gathers [nx][nt] with
 * t fastest.  Every call copies into MyAlloc arrays, calls the reference, and
 * copies the result out.  Return value: 0 ok, -1 if the reference threw.
 */
#include <vector>
#include "ref_shim.h"
#include <cstring>
#include <stdexcept>
#include <streambuf>
#include "memory.h"
#include "fd.h"
#include "wavelet.h"
#include "InitInversion.h"
#include <math.h> /* hilbert.h uses cos() without including it */
#include "../filter/hilbert.h"

extern int OMP_CORE;

namespace {
struct NullBuf : std::streambuf {
  int overflow(int c) override { return c; }
};
NullBuf g_null;

/* The reference prints progress lines to std::cout (fd.cpp:46); keep stdout
 * clean for the JSON line of the benchmark unless the caller asks for them. */
struct QuietCout {
  std::streambuf *old;
  explicit QuietCout(int verbose) : old(nullptr) {
    if (!verbose) old = std::cout.rdbuf(&g_null);
  }
  ~QuietCout() { if (old) std::cout.rdbuf(old); }
};

float **to2d(const float *src, int n1, int n2) {
  float **a = MyAlloc<float>::alc(n1, n2);
  std::memcpy(a[0], src, sizeof(float) * (size_t)n1 * n2);
  return a;
}
void from2d(float *dst, float **a, int n1, int n2) {
  std::memcpy(dst, a[0], sizeof(float) * (size_t)n1 * n2);
}
int g_verbose = 0;
}  // namespace

extern "C" {

void ref_set_threads(int n) { OMP_CORE = n > 0 ? n : 1; }
void ref_set_verbose(int v) { g_verbose = v; }

/* rickerWavelet (src/util/wavelet.cpp:7-18) */
int ref_ricker(float dt, float fr, int delay, int NT, float *out) {
  float *w = rickerWavelet(dt, fr, delay, NT);
  std::memcpy(out, w, sizeof(float) * NT);
  MyAlloc<float>::free(w);
  return 0;
}

/* setAbs blend weights, padded [nxpml][nzpml] (src/util/InitInversion.cpp:11-40) */
int ref_set_abs(int nz, int nx, int pml, float *out) {
  float **w = setAbs(nz, nx, pml);
  from2d(out, w, nz + 2 * pml, nx + 2 * pml);
  MyAlloc<float>::free(w);
  return 0;
}

/* setVel edge-replicating pad (src/util/InitInversion.cpp:92-113) */
int ref_set_vel(const float *v, int nz, int nx, int pml, float *out) {
  float **a = to2d(v, nz, nx);
  float **p = setVel(a, nz, nx, pml);
  from2d(out, p, nz + 2 * pml, nx + 2 * pml);
  MyAlloc<float>::free(a);
  MyAlloc<float>::free(p);
  return 0;
}

/* Hilbert<float>::apply (src/filter/hilbert.h:42-54) */
int ref_hilbert(const float *in, float *out, int n, int half) {
  Hilbert<float> h(half);
  h.apply(const_cast<float *>(in), out, n);
  return 0;
}

/* modeling (src/util/fd.cpp:15-80): rec_out [nx][nt] */
int ref_modeling(float dt, float dx, float dz, int nt, int ndel, int nx, int nz,
                 int pml, int sx, int sz, const int *gz, const float *wav,
                 const float *vel, float *rec_out) {
  QuietCout q(g_verbose);
  try {
    float **v = to2d(vel, nz, nx);
    float **rec = modeling(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz,
                           const_cast<int *>(gz), const_cast<float *>(wav), v);
    from2d(rec_out, rec, nt, nx);
    MyAlloc<float>::free(rec);
    MyAlloc<float>::free(v);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return -1;
  }
  return 0;
}

/* forwordPlane (src/util/fd.cpp:178-274): sou [nx][nt+ndel], rec_out [nx][nt] */
int ref_born_plane(float dt, float dx, float dz, int nt, int ndel, int nx, int nz, int pml,
                   int sz, int gz, const float *sou, const float *vel, const float *dv,
                   float *rec_out) {
  QuietCout q(g_verbose);
  try {
    float **v = to2d(vel, nz, nx);
    float **d = to2d(dv, nz, nx);
    float **s = to2d(sou, nt + ndel, nx);
    float **rec = forwordPlane(dt, dx, dz, nt, ndel, nx, nz, pml, sz, gz, v, s, d);
    from2d(rec_out, rec, nt, nx);
    MyAlloc<float>::free(rec);
    MyAlloc<float>::free(v);
    MyAlloc<float>::free(d);
    MyAlloc<float>::free(s);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return -1;
  }
  return 0;
}

/* adjointPlane (src/util/fd.cpp:787-921): sou [nx][nt+ndel], rec [nx][nt],
 * img_out [nx][nz].  The reference reads rec at negative sample indices
 * (fd.cpp:834, :873); the gather is laid out after ndel + 2 zero samples so
 * that those reads stay inside this allocation. */
int ref_rtm_plane(float dt, float dx, float dz, int nt, int ndel, int nx, int nz, int pml, int sz,
                  int gz, const float *sou, const float *vel, const float *rec, float *img_out) {
  QuietCout q(g_verbose);
  try {
    float **v = to2d(vel, nz, nx);
    float **s = to2d(sou, nt + ndel, nx);
    const size_t pad = (size_t)ndel + 2;
    std::vector<float> block(pad + (size_t)nx * nt, 0.0f);
    std::copy(rec, rec + (size_t)nx * nt, block.begin() + pad);
    std::vector<float *> rows((size_t)nx);
    for (int ix = 0; ix < nx; ix++) rows[ix] = block.data() + pad + (size_t)ix * nt;
    float **img = adjointPlane(dt, dx, dz, nt, ndel, nx, nz, pml, sz, gz, v, s, rows.data());
    from2d(img_out, img, nz, nx);
    MyAlloc<float>::free(img);
    MyAlloc<float>::free(v);
    MyAlloc<float>::free(s);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return -1;
  }
  return 0;
}

/* rtm_true (src/util/fd.cpp:924-1052): rec [nx][nt], img_out [nx][nz] */
int ref_rtm_true(float dt, float dx, float dz, int nt, int ndel, int nx, int nz, int pml, int sx,
                 int sz, const int *gz, const float *wav, const float *vel, const float *rec,
                 float *img_out) {
  QuietCout q(g_verbose);
  try {
    float **v = to2d(vel, nz, nx);
    float **r = to2d(rec, nt, nx);
    float **img = rtm_true(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, const_cast<int *>(gz),
                           const_cast<float *>(wav), v, r);
    from2d(img_out, img, nz, nx);
    MyAlloc<float>::free(img);
    MyAlloc<float>::free(v);
    MyAlloc<float>::free(r);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return -1;
  }
  return 0;
}

/* adjointUpDown (src/util/fd.cpp:340-591): rec [nx][nt]; img_out [nx][nz];
 * comp_out [4][nx][nz] = the model part of its four accumulators imagX (zero
 * on entry, the caller's allocation in the reference). */
int ref_rtm_updown(float dt, float dx, float dz, int nt, int ndel, int nx, int nz, int pml, int sx,
                   int sz, const int *gz, const float *wav, const float *wavh, const float *vel,
                   const float *rec, float *img_out, float *comp_out) {
  QuietCout q(g_verbose);
  try {
    const int NX = nx + 2 * pml, NZ = nz + 2 * pml;
    float **v = to2d(vel, nz, nx);
    float **r = to2d(rec, nt, nx);
    float ***imgX = MyAlloc<float>::alc(NZ, NX, 4);
    float **img = adjointUpDown(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, const_cast<int *>(gz),
                                const_cast<float *>(wav), const_cast<float *>(wavh), v, r, r,
                                imgX);
    from2d(img_out, img, nz, nx);
    for (int k = 0; k < 4; k++)
      for (int ix = 0; ix < nx; ix++)
        for (int iz = 0; iz < nz; iz++)
          comp_out[((size_t)k * nx + ix) * nz + iz] = imgX[k][ix + pml][iz + pml];
    MyAlloc<float>::free(img);
    MyAlloc<float>::free(imgX);
    MyAlloc<float>::free(v);
    MyAlloc<float>::free(r);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return -1;
  }
  return 0;
}

/* harmonic (src/util/InitInversion.cpp:141-150): phase rotation of a trace by
 * kx x through the 201-tap Hilbert filter */
int ref_harmonic(const float *in, float *out, int nt, float kx, float x) {
  try {
    harmonic(const_cast<float *>(in), out, nt, kx, x);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return -1;
  }
  return 0;
}

/* illum (src/util/fd.cpp:275-339): ss_out [nx][nz] */
int ref_illum(float dt, float dx, float dz, int nt, int ndel, int nx, int nz, int pml, int sx,
              int sz, const float *wav, const float *vel, float *ss_out) {
  QuietCout q(g_verbose);
  try {
    float **v = to2d(vel, nz, nx);
    float **ss = illum(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, const_cast<float *>(wav), v);
    from2d(ss_out, ss, nz, nx);
    MyAlloc<float>::free(ss);
    MyAlloc<float>::free(v);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return -1;
  }
  return 0;
}

/* illumPlane (src/util/fd.cpp:720-786): sou [nx][nt+ndel] at row sz; gz is
 * not used by the reference body.  ss_out [nx][nz] */
int ref_illum_plane(float dt, float dx, float dz, int nt, int ndel, int nx, int nz, int pml,
                    int sz, const float *sou, const float *vel, float *ss_out) {
  QuietCout q(g_verbose);
  try {
    float **v = to2d(vel, nz, nx);
    float **so = to2d(sou, nt + ndel, nx);
    float **ss = illumPlane(dt, dx, dz, nt, ndel, nx, nz, pml, sz, 0, v, so);
    from2d(ss_out, ss, nz, nx);
    MyAlloc<float>::free(ss);
    MyAlloc<float>::free(so);
    MyAlloc<float>::free(v);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return -1;
  }
  return 0;
}

/* forward, Born modeling (src/util/fd.cpp:81-177): rec_out [nx][nt] */
int ref_born(float dt, float dx, float dz, int nt, int ndel, int nx, int nz,
             int pml, int sx, int sz, const int *gz, const float *wav,
             const float *vel, const float *dv, float *rec_out) {
  QuietCout q(g_verbose);
  try {
    float **v = to2d(vel, nz, nx);
    float **d = to2d(dv, nz, nx);
    float **rec = forward(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz,
                          const_cast<int *>(gz), const_cast<float *>(wav), v, d);
    from2d(rec_out, rec, nt, nx);
    MyAlloc<float>::free(rec);
    MyAlloc<float>::free(v);
    MyAlloc<float>::free(d);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return -1;
  }
  return 0;
}

/* adjoint, RTM (src/util/fd.cpp:592-719): img_out [nx][nz] */
int ref_rtm(float dt, float dx, float dz, int nt, int ndel, int nx, int nz,
            int pml, int sx, int sz, const int *gz, const float *wav,
            const float *vel, const float *rec, float *img_out) {
  QuietCout q(g_verbose);
  try {
    float **v = to2d(vel, nz, nx);
    float **r = to2d(rec, nt, nx);
    float **img = adjoint(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz,
                          const_cast<int *>(gz), const_cast<float *>(wav), v, r);
    from2d(img_out, img, nz, nx);
    MyAlloc<float>::free(img);
    MyAlloc<float>::free(v);
    MyAlloc<float>::free(r);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return -1;
  }
  return 0;
}

}  // extern "C"
