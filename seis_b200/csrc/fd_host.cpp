// Host runtime of the C ABI declared in include/seis_fd.h.
//
// A plan is a batch of shots resident on the device: per-shot padded models,
// rotating wavefield buffers, gathers and images, a device shot table and a
// tile list covering every shot's padded grid.  Each time step is one launch
// over all tiles of all shots (the reference instead runs one shot per MPI
// worker, src/lsrtm/inversion.cpp:141-551).  The single-shot entry points are
// batches of one.
//
// Host-side scalars that the kernels consume (1/dx^2, (1/dx)^2 dt^2, ...) are
// formed here in single precision in the reference's operation order; this
// file is compiled with -ffp-contract=off.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/seis_fd.h"
#include "fd_internal.h"

using namespace seis;

struct seis_fd_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  int64_t launches = 0;
};

namespace {

enum Op { OP_MODEL = 0, OP_BORN = 1, OP_RTM = 2 };

int fail(seis_fd_ctx *ctx, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (ctx) ctx->err = buf;
  return code;
}

#define CK(call)                                                                   \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess)                                                         \
      return fail(ctx, e_ == cudaErrorMemoryAllocation ? SEIS_ERR_NOMEM : SEIS_ERR_CUDA, \
                  "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

int round_up(int x, int m) { return (x + m - 1) / m * m; }

// Single-shot argument checks.  Sources and receivers must lie strictly
// inside the padded grid's outer frame: the reference overwrites the frame
// after injecting (fd.cpp:53, :678), so an injection there has no effect.
int check_shot(seis_fd_ctx *ctx, const seis_shot_desc *s, int idx) {
  if (!s) return fail(ctx, SEIS_ERR_ARG, "shot %d: null descriptor", idx);
  if (s->nx < 1 || s->nz < 1 || s->pml < 0)
    return fail(ctx, SEIS_ERR_ARG, "shot %d: nx=%d nz=%d pml=%d", idx, s->nx, s->nz, s->pml);
  int NX = s->nx + 2 * s->pml, NZ = s->nz + 2 * s->pml;
  if (NX < 5 || NZ < 5)
    return fail(ctx, SEIS_ERR_ARG, "shot %d: padded grid %dx%d smaller than 5x5", idx, NX, NZ);
  if (s->nt < 1 || s->ndel < 0)
    return fail(ctx, SEIS_ERR_ARG, "shot %d: nt=%d ndel=%d", idx, s->nt, s->ndel);
  if (!(s->dt > 0.f) || !(s->dx > 0.f) || !(s->dz > 0.f))
    return fail(ctx, SEIS_ERR_ARG, "shot %d: dt/dx/dz must be positive", idx);
  int sxp = s->sx + s->pml, szp = s->sz + s->pml;
  if (sxp < 1 || sxp > NX - 2 || szp < 1 || szp > NZ - 2)
    return fail(ctx, SEIS_ERR_ARG, "shot %d: source (%d,%d) outside the padded grid interior",
                idx, s->sx, s->sz);
  if (!s->gz) return fail(ctx, SEIS_ERR_ARG, "shot %d: gz is null", idx);
  for (int ix = 0; ix < s->nx; ix++) {
    int g = s->gz[ix] + s->pml;
    if (g < 1 || g > NZ - 2)
      return fail(ctx, SEIS_ERR_ARG, "shot %d: gz[%d]=%d outside the padded grid interior", idx,
                  ix, s->gz[ix]);
  }
  return SEIS_OK;
}

struct Plan {
  seis_fd_ctx *ctx = nullptr;
  int op = OP_MODEL;
  int nshot = 0;
  std::vector<seis_shot_desc> desc;
  std::vector<std::vector<int>> gz;
  std::vector<ShotDev> sd;
  std::vector<Tile> tiles;
  std::vector<int2> cols;
  std::vector<void *> allocs;
  ShotDev *d_sd = nullptr;
  Tile *d_tiles = nullptr;
  int2 *d_cols = nullptr;
  float *d_taps = nullptr;
  float *d_stage = nullptr;  // staging for unpadded uploads / transposes
  size_t stage_elems = 0;
  int NT = 0, nt = 0, ndel = 0, max_strip = 0, max_NZ = 0;

  ~Plan() {
    for (void *p : allocs) cudaFree(p);
  }
  template <class T>
  int alloc(T **p, size_t n) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(ctx, e == cudaErrorMemoryAllocation ? SEIS_ERR_NOMEM : SEIS_ERR_CUDA,
                  "cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
    }
    allocs.push_back(q);
    *p = static_cast<T *>(q);
    e = cudaMemsetAsync(q, 0, std::max<size_t>(n, 1) * sizeof(T), ctx->stream);
    if (e != cudaSuccess) return fail(ctx, SEIS_ERR_CUDA, "cudaMemset: %s", cudaGetErrorString(e));
    return SEIS_OK;
  }
};

// Hilbert taps of src/filter/hilbert.h:59-70 (half = 30): the taper is formed
// in double and rounded to float; the tap in double from the float taper.
void hilbert_taps(float *h, int half) {
  h[half] = 0.0f;
  for (int i = 1; i <= half; i++) {
    float taper = (float)(0.54 + 0.46 * std::cos(3.1415926 * i / half));
    h[half + i] = (float)((double)(taper * (float)(i % 2)) * 2.0 / (3.1415926 * i));
    h[half - i] = -h[half + i];
  }
}

void fill_scalars(ShotDev &g, const seis_shot_desc &s) {
  g.nx = s.nx; g.nz = s.nz; g.pml = s.pml;
  g.NX = s.nx + 2 * s.pml; g.NZ = s.nz + 2 * s.pml;
  g.LDZ = round_up(g.NZ, 32);
  g.sxp = s.sx + s.pml; g.szp = s.sz + s.pml;
  g.nt = s.nt; g.ndel = s.ndel; g.NT = s.nt + s.ndel;
  g.strip_len = LAYERS * 2 * (s.nx + s.nz);
  const float dt = s.dt, dx = s.dx, dz = s.dz;
  g.dt = dt; g.dx = dx; g.dz = dz;
  g.invdx2 = 1.0f / (dx * dx);
  g.invdz2 = 1.0f / (dz * dz);
  float dt2 = dt * dt;
  g.kx = (1.0f / dx) * (1.0f / dx) * dt2;
  g.kz = (1.0f / dz) * (1.0f / dz) * dt2;
  g.a1z = 1.0f / dz / 2.0f / dt;
  g.a1x = 1.0f / dx / 2.0f / dt;
  g.hdt2 = 1.0f / 2.0f / dt / dt;
  g.ax1 = 1.0f / dz;
  g.ax2 = 1.0f / dx;
  g.sqrt2f = std::sqrt(2.0f);
  g.sqrt2d = std::sqrt(2.0);
  g.idt2 = 1.0f / dt / dt;
}

void build_tiles(Plan &p) {
  p.tiles.clear();
  p.cols.clear();
  for (int s = 0; s < p.nshot; s++) {
    const ShotDev &g = p.sd[s];
    int lox = std::max(g.pml, 4), hix = std::min(g.pml + g.nx, g.NX - 4);
    int loz = std::max(g.pml, 4), hiz = std::min(g.pml + g.nz, g.NZ - 4);
    for (int x0 = 0; x0 < g.NX; x0 += TX)
      for (int z0 = 0; z0 < g.NZ; z0 += TZ) {
        bool in = x0 >= lox && x0 + TX <= hix && z0 >= loz && z0 + TZ <= hiz;
        p.tiles.push_back(Tile{s, x0, z0, in ? TILE_INTERIOR : TILE_BOUNDARY});
      }
    for (int x = 0; x < g.nx; x++) p.cols.push_back(make_int2(s, x));
  }
}

int plan_create(seis_fd_ctx *ctx, int op, int nshot, const seis_shot_desc *descs, Plan **out) {
  *out = nullptr;
  if (nshot < 1 || !descs) return fail(ctx, SEIS_ERR_ARG, "nshot=%d", nshot);
  for (int i = 0; i < nshot; i++) {
    int rc = check_shot(ctx, &descs[i], i);
    if (rc) return rc;
    if (descs[i].nt != descs[0].nt || descs[i].ndel != descs[0].ndel || descs[i].dt != descs[0].dt)
      return fail(ctx, SEIS_ERR_ARG, "shot %d: nt, ndel and dt must match across a batch", i);
  }
  Plan *p = new (std::nothrow) Plan();
  if (!p) return fail(ctx, SEIS_ERR_NOMEM, "host allocation failed");
  p->ctx = ctx;
  p->op = op;
  p->nshot = nshot;
  p->desc.assign(descs, descs + nshot);
  p->gz.resize(nshot);
  p->sd.resize(nshot);
  p->nt = descs[0].nt;
  p->ndel = descs[0].ndel;
  p->NT = p->nt + p->ndel;
  int rc = SEIS_OK;
  for (int s = 0; s < nshot && rc == SEIS_OK; s++) {
    const seis_shot_desc &d = descs[s];
    p->gz[s].assign(d.gz, d.gz + d.nx);
    p->desc[s].gz = p->gz[s].data();
    ShotDev &g = p->sd[s];
    std::memset(&g, 0, sizeof g);
    fill_scalars(g, d);
    size_t cells = (size_t)g.NX * g.LDZ;
    p->max_strip = std::max(p->max_strip, g.strip_len);
    p->max_NZ = std::max(p->max_NZ, g.NZ);
    p->stage_elems = std::max(p->stage_elems, std::max((size_t)d.nx * d.nz, (size_t)d.nx * d.nt));
    for (int k = 0; k < 3 && rc == SEIS_OK; k++) rc = p->alloc(&g.fa[k], cells);
    if (op != OP_MODEL)
      for (int k = 0; k < 3 && rc == SEIS_OK; k++) rc = p->alloc(&g.fb[k], cells);
    float *vel = nullptr, *dv = nullptr, *wav = nullptr, *rec = nullptr;
    int *gzd = nullptr;
    if (rc == SEIS_OK) rc = p->alloc(&vel, cells);
    if (rc == SEIS_OK && op == OP_BORN) rc = p->alloc(&dv, cells);
    if (rc == SEIS_OK) rc = p->alloc(&wav, (size_t)g.NT);
    if (rc == SEIS_OK) rc = p->alloc(&rec, (size_t)d.nt * d.nx);
    if (rc == SEIS_OK) rc = p->alloc(&gzd, (size_t)d.nx);
    if (rc == SEIS_OK && op == OP_RTM) rc = p->alloc(&g.strips, (size_t)d.nt * g.strip_len);
    if (rc == SEIS_OK && op == OP_RTM) rc = p->alloc(&g.img, (size_t)d.nx * d.nz);
    if (rc == SEIS_OK) {
      g.vel = vel; g.dv = dv; g.wav = wav; g.rec = rec; g.gz = gzd;
      cudaError_t e = cudaMemcpyAsync(gzd, d.gz, sizeof(int) * d.nx, cudaMemcpyHostToDevice,
                                      ctx->stream);
      if (e != cudaSuccess) rc = fail(ctx, SEIS_ERR_CUDA, "gz upload: %s", cudaGetErrorString(e));
    }
  }
  if (rc == SEIS_OK) rc = p->alloc(&p->d_stage, p->stage_elems);
  if (rc == SEIS_OK) {
    build_tiles(*p);
    rc = p->alloc(&p->d_sd, (size_t)nshot);
  }
  if (rc == SEIS_OK) rc = p->alloc(&p->d_tiles, p->tiles.size());
  if (rc == SEIS_OK && op == OP_RTM) rc = p->alloc(&p->d_cols, p->cols.size());
  if (rc == SEIS_OK && op == OP_RTM) rc = p->alloc(&p->d_taps, (size_t)61);
  if (rc == SEIS_OK) {
    cudaStream_t st = ctx->stream;
    cudaError_t e = cudaMemcpyAsync(p->d_sd, p->sd.data(), sizeof(ShotDev) * nshot,
                                    cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(p->d_tiles, p->tiles.data(), sizeof(Tile) * p->tiles.size(),
                          cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && op == OP_RTM) {
      e = cudaMemcpyAsync(p->d_cols, p->cols.data(), sizeof(int2) * p->cols.size(),
                          cudaMemcpyHostToDevice, st);
      float taps[61];
      hilbert_taps(taps, 30);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(p->d_taps, taps, sizeof taps, cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = fail(ctx, SEIS_ERR_CUDA, "plan upload: %s", cudaGetErrorString(e));
  }
  if (rc != SEIS_OK) {
    delete p;
    return rc;
  }
  *out = p;
  return SEIS_OK;
}

// Upload an unpadded [nx][nz] model of shot s into a padded device field.
int upload_model(Plan &p, int s, const float *h, float *d_padded, int clamp) {
  seis_fd_ctx *ctx = p.ctx;
  const seis_shot_desc &d = p.desc[s];
  const ShotDev &g = p.sd[s];
  CK(cudaMemcpyAsync(p.d_stage, h, sizeof(float) * d.nx * d.nz, cudaMemcpyHostToDevice,
                     ctx->stream));
  CK(launch_pad(p.d_stage, d.nx, d.nz, d.pml, g.LDZ, clamp, d_padded, ctx->stream));
  ctx->launches++;
  return SEIS_OK;
}

int run_forward(Plan &p, int mode) {
  seis_fd_ctx *ctx = p.ctx;
  StepArgs a{};
  a.nshots = p.nshot;
  for (int it = 0; it < p.NT; it++) {
    a.rot = it;
    a.rot_b = it;
    a.src_k = it >= 1 ? it - 1 : -1;
    int itp = it - p.ndel;
    a.rec_k = (p.op != OP_RTM && itp >= 0) ? itp : -1;
    a.strip_k = (p.op == OP_RTM && itp >= 0) ? itp : -1;
    CK(launch_step(mode, p.d_sd, p.d_tiles, (int)p.tiles.size(), a, ctx->stream));
    ctx->launches++;
  }
  return SEIS_OK;
}

// Reverse pass of the reference RTM (fd.cpp:654-693).
int run_rtm_reverse(Plan &p) {
  seis_fd_ctx *ctx = p.ctx;
  // the source fields restart from zero (fd.cpp:654-656)
  for (int s = 0; s < p.nshot; s++)
    for (int k = 0; k < 3; k++)
      CK(cudaMemsetAsync(p.sd[s].fa[k], 0, sizeof(float) * p.sd[s].NX * p.sd[s].LDZ, ctx->stream));
  StepArgs a{};
  a.nshots = p.nshot;
  a.src_k = -1;
  a.strip_k = -1;
  int k = 0;
  for (int it = p.NT - 1; it >= p.ndel; it--, k++) {
    a.rot = k;
    a.rot_b = k;
    CK(launch_rtm_restore(p.d_sd, p.nshot, p.max_strip, a.rot, it, ctx->stream));
    a.rec_k = -1;
    CK(launch_step(MODE_MODEL, p.d_sd, p.d_tiles, (int)p.tiles.size(), a, ctx->stream));
    a.rec_k = it - p.ndel;
    CK(launch_step(MODE_RCV, p.d_sd, p.d_tiles, (int)p.tiles.size(), a, ctx->stream));
    CK(launch_rtm_image(p.d_sd, p.d_cols, (int)p.cols.size(), a.rot, a.rot_b, p.max_NZ,
                        p.d_taps, ctx->stream));
    ctx->launches += 4;
  }
  return SEIS_OK;
}

int download_gather(Plan &p, int s, float *h_rec) {
  seis_fd_ctx *ctx = p.ctx;
  const seis_shot_desc &d = p.desc[s];
  CK(launch_transpose(p.sd[s].rec, d.nt, d.nx, p.d_stage, ctx->stream));
  ctx->launches++;
  CK(cudaMemcpyAsync(h_rec, p.d_stage, sizeof(float) * d.nt * d.nx, cudaMemcpyDeviceToHost,
                     ctx->stream));
  return SEIS_OK;
}

int upload_gather(Plan &p, int s, const float *h_rec) {
  seis_fd_ctx *ctx = p.ctx;
  const seis_shot_desc &d = p.desc[s];
  CK(cudaMemcpyAsync(p.d_stage, h_rec, sizeof(float) * d.nt * d.nx, cudaMemcpyHostToDevice,
                     ctx->stream));
  CK(launch_transpose(p.d_stage, d.nx, d.nt, p.sd[s].rec, ctx->stream));
  ctx->launches++;
  return SEIS_OK;
}

int upload_wavelet(Plan &p, int s, const float *h_wav) {
  seis_fd_ctx *ctx = p.ctx;
  CK(cudaMemcpyAsync(const_cast<float *>(p.sd[s].wav), h_wav, sizeof(float) * p.NT,
                     cudaMemcpyHostToDevice, ctx->stream));
  return SEIS_OK;
}

int sync(seis_fd_ctx *ctx) {
  CK(cudaStreamSynchronize(ctx->stream));
  return SEIS_OK;
}

int begin(seis_fd_ctx *ctx) {
  if (!ctx) return SEIS_ERR_ARG;
  ctx->err.clear();
  CK(cudaSetDevice(ctx->device));
  return SEIS_OK;
}

}  // namespace

extern "C" {

int seis_fd_abi_version(void) { return SEIS_FD_ABI_VERSION; }

int seis_fd_ricker(float dt, float fr, int delay, int n, float *out) {
  if (n < 0 || (n > 0 && !out)) return SEIS_ERR_ARG;
  float tmp = (float)(3.1415926 * 3.1415926 * (double)fr * (double)fr);
  for (int i = 0; i < n; i++) {
    float t = (float)(i - delay) * 1.0f * dt;
    float t2 = t * t;
    out[i] = (1.0f - 2.0f * tmp * t2) * std::exp(-tmp * t2);
  }
  return SEIS_OK;
}

int seis_fd_validate_shot(const seis_shot_desc *shot, char *msg, size_t msg_len) {
  seis_fd_ctx tmp;
  int rc = check_shot(&tmp, shot, 0);
  if (msg && msg_len) {
    std::strncpy(msg, tmp.err.c_str(), msg_len - 1);
    msg[msg_len - 1] = 0;
  }
  return rc;
}

int seis_fd_create(seis_fd_ctx **out, int device) {
  if (!out) return SEIS_ERR_ARG;
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return SEIS_ERR_CUDA;
  }
  if (device < 0 || device >= n) return SEIS_ERR_ARG;
  seis_fd_ctx *ctx = new (std::nothrow) seis_fd_ctx();
  if (!ctx) return SEIS_ERR_NOMEM;
  ctx->device = device;
  e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete ctx;
    return SEIS_ERR_CUDA;
  }
  *out = ctx;
  return SEIS_OK;
}

int seis_fd_destroy(seis_fd_ctx *ctx) {
  if (!ctx) return SEIS_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) {
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
  }
  delete ctx;
  return SEIS_OK;
}

const char *seis_fd_last_error(const seis_fd_ctx *ctx) { return ctx ? ctx->err.c_str() : ""; }

int64_t seis_fd_launch_count(const seis_fd_ctx *ctx) { return ctx ? ctx->launches : 0; }

int seis_fd_modeling(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_wav,
                     const float *h_vel, float *h_rec) {
  int rc = begin(ctx);
  if (rc) return rc;
  if (!h_wav || !h_vel || !h_rec) return fail(ctx, SEIS_ERR_ARG, "null array");
  Plan *p = nullptr;
  rc = plan_create(ctx, OP_MODEL, 1, shot, &p);
  if (rc) return rc;
  if (!rc) rc = upload_model(*p, 0, h_vel, const_cast<float *>(p->sd[0].vel), 1);
  if (!rc) rc = upload_wavelet(*p, 0, h_wav);
  if (!rc) rc = run_forward(*p, MODE_MODEL);
  if (!rc) rc = download_gather(*p, 0, h_rec);
  if (!rc) rc = sync(ctx);
  delete p;
  return rc;
}

int seis_fd_born(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_wav,
                 const float *h_vel, const float *h_dv, float *h_rec) {
  int rc = begin(ctx);
  if (rc) return rc;
  if (!h_wav || !h_vel || !h_dv || !h_rec) return fail(ctx, SEIS_ERR_ARG, "null array");
  Plan *p = nullptr;
  rc = plan_create(ctx, OP_BORN, 1, shot, &p);
  if (rc) return rc;
  if (!rc) rc = upload_model(*p, 0, h_vel, const_cast<float *>(p->sd[0].vel), 1);
  if (!rc) rc = upload_model(*p, 0, h_dv, const_cast<float *>(p->sd[0].dv), 0);
  if (!rc) rc = upload_wavelet(*p, 0, h_wav);
  if (!rc) rc = run_forward(*p, MODE_BORN);
  if (!rc) rc = download_gather(*p, 0, h_rec);
  if (!rc) rc = sync(ctx);
  delete p;
  return rc;
}

int seis_fd_rtm(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_wav,
                const float *h_vel, const float *h_rec, float *h_img) {
  int rc = begin(ctx);
  if (rc) return rc;
  if (!h_wav || !h_vel || !h_rec || !h_img) return fail(ctx, SEIS_ERR_ARG, "null array");
  Plan *p = nullptr;
  rc = plan_create(ctx, OP_RTM, 1, shot, &p);
  if (rc) return rc;
  if (!rc) rc = upload_model(*p, 0, h_vel, const_cast<float *>(p->sd[0].vel), 1);
  if (!rc) rc = upload_wavelet(*p, 0, h_wav);
  if (!rc) rc = upload_gather(*p, 0, h_rec);
  if (!rc) rc = run_forward(*p, MODE_MODEL);
  if (!rc) rc = run_rtm_reverse(*p);
  if (!rc) {
    cudaError_t e = cudaMemcpyAsync(h_img, p->sd[0].img, sizeof(float) * shot->nx * shot->nz,
                                    cudaMemcpyDeviceToHost, ctx->stream);
    if (e != cudaSuccess) rc = fail(ctx, SEIS_ERR_CUDA, "image download: %s", cudaGetErrorString(e));
  }
  if (!rc) rc = sync(ctx);
  delete p;
  return rc;
}

}  // extern "C"
