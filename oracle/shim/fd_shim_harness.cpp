/*
 * Runs the fd.h drop-in (linked into oracle/_ref/fd_shim_check
 * by build_integration.py) on one shot, through the reference's own fd.h
 * signatures and MyAlloc arrays.  Test infrastructure only.
 *
 *   fd_shim_check IN OUT
 *
 * IN (little-endian): int32 nx nz pml nt ndel sx sz; float32 dt dx dz;
 * int32 gz[nx]; float32 wav[nt+ndel]; vel[nx][nz]; dv[nx][nz]; rec[nx][nt].
 * OUT: modeling gather [nx][nt], Born gather [nx][nt], RTM image of `rec`
 * [nx][nz], illumination [nx][nz], rtm_true image of `rec` [nx][nz].
 */
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "fd.h"
#include "memory.h"

static void need(bool ok, const char *what) {
  if (!ok) {
    std::fprintf(stderr, "fd_shim_check: %s\n", what);
    std::exit(2);
  }
}

template <class T>
static void get(std::FILE *f, T *p, size_t n) {
  need(std::fread(p, sizeof(T), n, f) == n, "short input");
}

static float **grid(std::FILE *f, int n1, int n2) {  // [n2][n1], n1 contiguous
  float **a = MyAlloc<float>::alc(n1, n2);
  get(f, a[0], (size_t)n1 * n2);
  return a;
}

static void put(std::FILE *f, float **a, size_t n) {
  need(std::fwrite(a[0], sizeof(float), n, f) == n, "short output");
  MyAlloc<float>::free(a);
}

int main(int argc, char **argv) {
  need(argc == 3, "usage: fd_shim_check IN OUT");
  std::FILE *in = std::fopen(argv[1], "rb");
  need(in != nullptr, "cannot open input");
  int h[7];
  float sc[3];
  get(in, h, 7);
  get(in, sc, 3);
  const int nx = h[0], nz = h[1], pml = h[2], nt = h[3], ndel = h[4], sx = h[5], sz = h[6];
  std::vector<int> gz(nx);
  std::vector<float> wav(nt + ndel);
  get(in, gz.data(), nx);
  get(in, wav.data(), wav.size());
  float **vel = grid(in, nz, nx), **dv = grid(in, nz, nx), **rec = grid(in, nt, nx);
  std::fclose(in);
  const float dt = sc[0], dx = sc[1], dz = sc[2];
  std::FILE *out = std::fopen(argv[2], "wb");
  need(out != nullptr, "cannot open output");
  put(out, modeling(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, gz.data(), wav.data(), vel),
      (size_t)nx * nt);
  put(out, forward(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, gz.data(), wav.data(), vel, dv),
      (size_t)nx * nt);
  put(out, adjoint(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, gz.data(), wav.data(), vel, rec),
      (size_t)nx * nz);
  put(out, illum(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, wav.data(), vel), (size_t)nx * nz);
  put(out, rtm_true(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, gz.data(), wav.data(), vel, rec),
      (size_t)nx * nz);
  std::fclose(out);
  return 0;
}
