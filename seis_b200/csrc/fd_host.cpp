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
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/seis_fd.h"
#include "fd_internal.h"

using namespace seis;

struct seis_fd_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;  // all work is ordered on this stream
  cudaStream_t aux = nullptr;     // boundary tiles run here, joined every step
  cudaEvent_t fork = nullptr, join = nullptr;
  int *d_err = nullptr;  // set by kernels whose bounded waits ran out
  std::vector<seis_fd_plan *> plans;  // live plans, torn down with the context
  double *d_partial = nullptr;        // DOT_PARTS partial sums of a dot product
  double *d_scalar = nullptr;         // one FP64 result
  int num_sms = 148;
  std::string err;
  int64_t launches = 0;
};

namespace {
struct Plan;
}
struct seis_fd_plan {
  Plan *p;  // null once the owning context is destroyed
};

namespace {

enum Op {
  OP_MODEL = 0, OP_BORN = 1, OP_RTM = 2, OP_BORN_ADJ = 3, OP_ILLUM = 4, OP_BORN_PLANE = 5,
  OP_RTM_PLANE = 6, OP_RTM_TRUE = 7, OP_RTM_UPDOWN = 8, OP_ILLUM_PLANE = 9
};

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
  std::vector<Tile> tiles;  // interior tiles first (n_int), then pad tiles
  int n_int = 0, n_pad = 0;
  std::vector<Tile> adj_tiles;  // adjoint classification (stricter interior)
  int n_int_adj = 0, n_pad_adj = 0;
  Tile *d_adj_tiles = nullptr;
  int snap_every = 1, snap_dtype = SNAP_F32;
  // source-field checkpoints (adjoint plans, 0 = keep every snapshot): the
  // two time levels before every ck_every-th step; the reverse pass
  // recomputes each segment's snapshots into a buffer of one segment, on the
  // shot table sd_c (its own field A buffers)
  int ck_every = 0;
  std::vector<std::vector<float *>> ck;  // per shot: 2 fields per checkpoint j >= 1
  std::vector<ShotDev> sd_c;
  ShotDev *d_sd_c = nullptr;
  CUtensorMap *d_maps_c = nullptr;
  bool snaps_ready = false;  // storage allocated
  bool snaps_valid = false;  // storage holds the source terms of the current inputs
  int64_t device_bytes = 0;
  std::vector<int2> cols;
  std::vector<float *> field_bases;  // allocation starts of margin-padded fields
  std::vector<size_t> field_elems;
  CUtensorMap *d_maps = nullptr;
  // adjointUpDown: the shot table of the Hilbert-wavelet source field (its own
  // field A buffers, wavelet, boundary layers and tensor maps)
  std::vector<ShotDev> sd_h;
  ShotDev *d_sd_h = nullptr;
  CUtensorMap *d_maps_h = nullptr;
  bool exact = true;
  int shape = SHAPE_32x64;   // tile shape of every kernel of the plan (TileShapeId)
  // the interior and pad kernels of a step on two streams, concurrently
  // (else one after the other on the main stream)
  bool overlap = true;
  int loop = -1;  // interior kernel form (StepArgs::loop)
  std::vector<void *> allocs;
  std::vector<size_t> alloc_bytes;
  ShotDev *d_sd = nullptr;
  Tile *d_tiles = nullptr;
  int2 *d_cols = nullptr;
  float *d_taps = nullptr;
  float *d_stage = nullptr;  // staging for unpadded uploads / transposes
  size_t stage_elems = 0;
  int NT = 0, nt = 0, ndel = 0, max_strip = 0, max_NZ = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t launches_per_run = 0;
  int64_t cell_updates = 0;

  ~Plan() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (void *p : allocs) cudaFree(p);
  }
  // free one allocation made by alloc() (null: nothing)
  void release(void *q) {
    for (size_t i = 0; q && i < allocs.size(); i++)
      if (allocs[i] == q) {
        cudaFree(q);
        device_bytes -= (int64_t)alloc_bytes[i];
        allocs.erase(allocs.begin() + i);
        alloc_bytes.erase(alloc_bytes.begin() + i);
        return;
      }
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
    alloc_bytes.push_back(std::max<size_t>(n, 1) * sizeof(T));
    device_bytes += (int64_t)(std::max<size_t>(n, 1) * sizeof(T));
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
  g.LDZ = field_geom(g.NX, g.NZ).LDZ;
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
  g.q4dx2 = 1.0f / 4.0f / dx / dx;
  g.q4dz2 = 1.0f / 4.0f / dz / dz;
  g.inv_pml = s.pml > 0 ? 1.0f / (float)s.pml : 0.0f;
}

// Tiles of every shot's padded grid; interior tiles (every cell a model cell
// in the 8th-order region) take the kernel without boundary logic.  All
// interior tiles come first, then all pad tiles, each group interleaved
// across shots, so that shots are spread evenly over the SMs.
void build_tiles(Plan &p) {
  const int TX = shape_tx(p.shape), TZ = shape_tz(p.shape);
  p.tiles.clear();
  p.cols.clear();
  std::vector<std::vector<Tile>> per(p.nshot);
  size_t most = 0;
  for (int s = 0; s < p.nshot; s++) {
    const ShotDev &g = p.sd[s];
    const int lox = std::max(g.pml, 4), hix = std::min(g.pml + g.nx, g.NX - 4);
    const int loz = std::max(g.pml, 4), hiz = std::min(g.pml + g.nz, g.NZ - 4);
    for (int x0 = 0; x0 < g.NX; x0 += TX)
      for (int z0 = 0; z0 < g.NZ; z0 += TZ) {
        bool in = x0 >= lox && x0 + TX <= hix && z0 >= loz && z0 + TZ <= hiz;
        per[s].push_back(Tile{s, x0, z0, in ? TILE_INTERIOR : TILE_PAD});
      }
    most = std::max(most, per[s].size());
    for (int x = 0; x < g.nx; x++) p.cols.push_back(make_int2(s, x));
  }
  for (int kind : {TILE_INTERIOR, TILE_PAD})
    for (size_t i = 0; i < most; i++)
      for (int s = 0; s < p.nshot; s++)
        if (i < per[s].size() && per[s][i].kind == kind) p.tiles.push_back(per[s][i]);
  p.n_int = 0;
  for (const Tile &t : p.tiles) p.n_int += t.kind == TILE_INTERIOR;
  p.n_pad = (int)p.tiles.size() - p.n_int;
}

// Tiles for the exact adjoint: an interior tile holds no pad cell and no
// model edge cell (the cells whose adjoint carries the absorbing ring terms),
// and every consumer of its cells is 8th order (cells 8 or more from the grid
// edge), so that the adjoint there is the symmetric gather.
void build_adj_tiles(Plan &p) {
  const int TX = shape_tx(p.shape), TZ = shape_tz(p.shape);
  std::vector<Tile> in_t, pad_t;
  for (int s = 0; s < p.nshot; s++) {
    const ShotDev &g = p.sd[s];
    int lox = g.pml + 1, hix = g.pml + g.nx - 2;  // inclusive bounds of tile cells
    int loz = g.pml + 1, hiz = g.pml + g.nz - 2;
    lox = std::max(lox, 8); loz = std::max(loz, 8);
    hix = std::min(hix, g.NX - 9); hiz = std::min(hiz, g.NZ - 9);
    for (int x0 = 0; x0 < g.NX; x0 += TX)
      for (int z0 = 0; z0 < g.NZ; z0 += TZ) {
        bool in = x0 >= lox && x0 + TX - 1 <= hix && z0 >= loz && z0 + TZ - 1 <= hiz;
        (in ? in_t : pad_t).push_back(Tile{s, x0, z0, in ? TILE_INTERIOR : TILE_PAD});
      }
  }
  p.n_int_adj = (int)in_t.size();
  p.n_pad_adj = (int)pad_t.size();
  p.adj_tiles = in_t;
  p.adj_tiles.insert(p.adj_tiles.end(), pad_t.begin(), pad_t.end());
}

// One field of a shot in the margin-padded layout; returns the cell (0,0)
// pointer.
int alloc_field(Plan &p, const ShotDev &g, float **cell0) {
  FieldGeom fg = field_geom(g.NX, g.NZ);
  float *base = nullptr;
  int rc = p.alloc(&base, fg.elems);
  if (rc) return rc;
  p.field_bases.push_back(base);
  p.field_elems.push_back(fg.elems);
  *cell0 = base + fg.origin;
  return SEIS_OK;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on the driver library).
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// Tensor map of one field (cell (0,0) at `cell0`) with a box of `rows` staged
// rows by `width` columns.
int encode_map(seis_fd_ctx *ctx, const ShotDev &g, const float *cell0, int rows, int width,
               CUtensorMap *m) {
  auto fn = encode_fn();
  if (!fn) return fail(ctx, SEIS_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  FieldGeom fg = field_geom(g.NX, g.NZ);
  void *base = const_cast<float *>(cell0 - fg.origin);
  cuuint64_t dims[2] = {(cuuint64_t)fg.LDZ, (cuuint64_t)fg.ncols};
  cuuint64_t strides[1] = {(cuuint64_t)fg.LDZ * sizeof(float)};
  cuuint32_t box[2] = {(cuuint32_t)rows, (cuuint32_t)width};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(ctx, SEIS_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return SEIS_OK;
}

int encode_maps(Plan &p, std::vector<ShotDev> &sds, CUtensorMap **d_out) {
  std::vector<CUtensorMap> maps((size_t)p.nshot * NMAPS);
  std::memset(maps.data(), 0, maps.size() * sizeof(CUtensorMap));
  const int wide = shape_tx(p.shape) + 2 * HXC, narrow = shape_tx(p.shape) + 2;
  const int rows = shape_tz(p.shape) + 2 * ZM;
  for (int s = 0; s < p.nshot; s++) {
    const ShotDev &g = sds[s];
    CUtensorMap *m = maps.data() + (size_t)s * NMAPS;
    int rc = SEIS_OK;
    for (int k = 0; k < 3 && !rc; k++) {
      rc = encode_map(p.ctx, g, g.fa[k], rows, wide, &m[MAP_FA_WIDE + k]);
      if (!rc) rc = encode_map(p.ctx, g, g.fa[k], rows, narrow, &m[MAP_FA_NARROW + k]);
      if (!rc && g.fb[k]) rc = encode_map(p.ctx, g, g.fb[k], rows, wide, &m[MAP_FB_WIDE + k]);
      if (!rc && g.fb[k]) rc = encode_map(p.ctx, g, g.fb[k], rows, narrow, &m[MAP_FB_NARROW + k]);
    }
    if (!rc) rc = encode_map(p.ctx, g, g.vel, rows, narrow, &m[MAP_VEL]);
    if (!rc) rc = encode_map(p.ctx, g, g.vel, rows, wide, &m[MAP_VEL_WIDE]);
    if (!rc && g.dv) rc = encode_map(p.ctx, g, g.dv, rows, narrow, &m[MAP_DV]);
    // interior tiles
    const int TX = shape_tx(p.shape), TZ = shape_tz(p.shape);
    for (int k = 0; k < 3 && !rc; k++) {
      rc = encode_map(p.ctx, g, g.fa[k], TZ + 2 * HI, TX + 2 * HI, &m[MAP_FA_HALO + k]);
      if (!rc) rc = encode_map(p.ctx, g, g.fa[k], TZ, TX, &m[MAP_FA_TILE + k]);
      if (!rc && g.fb[k]) rc = encode_map(p.ctx, g, g.fb[k], TZ + 2 * HI, TX + 2 * HI, &m[MAP_FB_HALO + k]);
      if (!rc && g.fb[k]) rc = encode_map(p.ctx, g, g.fb[k], TZ, TX, &m[MAP_FB_TILE + k]);
    }
    if (!rc) rc = encode_map(p.ctx, g, g.vel, TZ, TX, &m[MAP_VEL_TILE]);
    if (!rc) rc = encode_map(p.ctx, g, g.vel, TZ + 2 * HI, TX + 2 * HI, &m[MAP_VEL_HALO]);
    if (!rc && g.dv) rc = encode_map(p.ctx, g, g.dv, TZ, TX, &m[MAP_DV_TILE]);
    if (rc) return rc;
  }
  int rc = p.alloc(d_out, maps.size());
  if (rc) return rc;
  seis_fd_ctx *ctx = p.ctx;
  CK(cudaMemcpyAsync(*d_out, maps.data(), maps.size() * sizeof(CUtensorMap),
                     cudaMemcpyHostToDevice, ctx->stream));
  for (int s = 0; s < p.nshot; s++) sds[s].maps = *d_out + (size_t)s * NMAPS;
  return SEIS_OK;
}

// adjointUpDown: the shot table of the Hilbert-wavelet source field, a copy of
// the main table with its own field A, wavelet and boundary layers
int make_hilbert_table(Plan &p) {
  p.sd_h = p.sd;
  for (int s = 0; s < p.nshot; s++) {
    ShotDev &h = p.sd_h[s];
    const seis_shot_desc &d = p.desc[s];
    for (int k = 0; k < 3; k++) {
      int rc = alloc_field(p, h, &h.fa[k]);
      if (rc) return rc;
    }
    float *wav = nullptr, *strips = nullptr;
    int rc = p.alloc(&wav, (size_t)h.NT);
    if (!rc) rc = p.alloc(&strips, (size_t)d.nt * h.strip_len);
    if (rc) return rc;
    h.wav = wav;
    h.strips = strips;
    h.img = nullptr;
    h.comp = nullptr;
  }
  int rc = encode_maps(p, p.sd_h, &p.d_maps_h);
  if (!rc) rc = p.alloc(&p.d_sd_h, (size_t)p.nshot);
  if (rc) return rc;
  seis_fd_ctx *ctx = p.ctx;
  CK(cudaMemcpyAsync(p.d_sd_h, p.sd_h.data(), sizeof(ShotDev) * p.nshot, cudaMemcpyHostToDevice,
                     ctx->stream));
  return SEIS_OK;
}

int plan_create(seis_fd_ctx *ctx, int op, int nshot, const seis_shot_desc *descs, Plan **out) {
  *out = nullptr;
  if (nshot < 1 || !descs) return fail(ctx, SEIS_ERR_ARG, "nshot=%d", nshot);
  for (int i = 0; i < nshot; i++) {
    int rc = check_shot(ctx, &descs[i], i);
    if (rc) return rc;
    // the reference keeps 4 boundary layers (fd.cpp:594, :1181-1203); they
    // must stay inside the padded grid
    if ((op == OP_RTM || op == OP_RTM_TRUE || op == OP_RTM_UPDOWN || op == OP_RTM_PLANE) &&
        descs[i].pml + std::min(descs[i].nx, descs[i].nz) < LAYERS)
      return fail(ctx, SEIS_ERR_ARG, "shot %d: RTM needs pml + min(nx, nz) >= %d", i, LAYERS);
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
    p->max_strip = std::max(p->max_strip, g.strip_len);
    p->max_NZ = std::max(p->max_NZ, g.NZ);
    p->stage_elems = std::max(p->stage_elems, std::max((size_t)d.nx * d.nz, (size_t)d.nx * d.nt));
    if (op == OP_BORN_PLANE || op == OP_RTM_PLANE || op == OP_ILLUM_PLANE)
      p->stage_elems = std::max(p->stage_elems, (size_t)d.nx * (d.nt + d.ndel));
    for (int k = 0; k < 3 && rc == SEIS_OK; k++) rc = alloc_field(*p, g, &g.fa[k]);
    if (op == OP_BORN || op == OP_RTM || op == OP_BORN_PLANE || op == OP_RTM_PLANE ||
        op == OP_RTM_TRUE || op == OP_RTM_UPDOWN)
      for (int k = 0; k < 3 && rc == SEIS_OK; k++) rc = alloc_field(*p, g, &g.fb[k]);
    float *vel = nullptr, *dv = nullptr, *wav = nullptr, *rec = nullptr;
    int *gzd = nullptr;
    if (rc == SEIS_OK) rc = alloc_field(*p, g, &vel);
    if (rc == SEIS_OK && (op == OP_BORN || op == OP_BORN_PLANE)) rc = alloc_field(*p, g, &dv);
    if (rc == SEIS_OK && (op == OP_BORN_PLANE || op == OP_RTM_PLANE || op == OP_ILLUM_PLANE)) {
      float *sou = nullptr;
      rc = p->alloc(&sou, (size_t)g.NT * d.nx);
      g.sou = sou;
    }
    if (rc == SEIS_OK) rc = p->alloc(&wav, (size_t)g.NT);
    if (rc == SEIS_OK) rc = p->alloc(&rec, (size_t)d.nt * d.nx);
    if (rc == SEIS_OK) rc = p->alloc(&gzd, (size_t)d.nx);
    if (rc == SEIS_OK && (op == OP_RTM || op == OP_RTM_TRUE || op == OP_RTM_UPDOWN))
      rc = p->alloc(&g.strips, (size_t)d.nt * g.strip_len);
    if (rc == SEIS_OK && op == OP_RTM_UPDOWN) rc = p->alloc(&g.comp, 4 * (size_t)d.nx * d.nz);
    g.rcv_dipole = op == OP_RTM_TRUE;
    if (rc == SEIS_OK && op == OP_RTM_PLANE)  // boundary layers of every step (fd.cpp:812-815)
      rc = p->alloc(&g.strips, (size_t)g.NT * g.strip_len);
    if (rc == SEIS_OK && (op == OP_RTM || op == OP_BORN_ADJ || op == OP_ILLUM || op == OP_RTM_PLANE ||
                          op == OP_RTM_TRUE || op == OP_RTM_UPDOWN || op == OP_ILLUM_PLANE))
      rc = p->alloc(&g.img, (size_t)d.nx * d.nz);
    if (op == OP_ILLUM || op == OP_ILLUM_PLANE) g.illum = g.img;
    if (rc == SEIS_OK && op == OP_BORN_ADJ) rc = p->alloc(&g.grad, (size_t)d.nx * d.nz);
    if (op == OP_BORN_ADJ) {
      if (rc == SEIS_OK) rc = alloc_field(*p, g, &g.adj_e[0]);
      if (rc == SEIS_OK) rc = alloc_field(*p, g, &g.adj_e[1]);
      if (rc == SEIS_OK) rc = alloc_field(*p, g, &g.adj_b);
      if (rc == SEIS_OK) rc = p->alloc(&g.edge_coef, (size_t)EDGE_TAPS * edge_cells(g.NX, g.NZ));
    }
    g.ntz = (g.NZ + shape_tz(p->shape) - 1) / shape_tz(p->shape);
    if (rc == SEIS_OK) {
      g.vel = vel; g.dv = dv; g.wav = wav; g.rec = rec; g.gz = gzd;
      cudaError_t e = cudaMemcpyAsync(gzd, d.gz, sizeof(int) * d.nx, cudaMemcpyHostToDevice,
                                      ctx->stream);
      if (e != cudaSuccess) rc = fail(ctx, SEIS_ERR_CUDA, "gz upload: %s", cudaGetErrorString(e));
    }
  }
  if (rc == SEIS_OK) rc = p->alloc(&p->d_stage, p->stage_elems);
  if (rc == SEIS_OK) rc = encode_maps(*p, p->sd, &p->d_maps);
  if (rc == SEIS_OK && op == OP_RTM_UPDOWN) rc = make_hilbert_table(*p);
  if (rc == SEIS_OK) {
    build_tiles(*p);
    build_adj_tiles(*p);
    // padded cell-updates of one run: modeling NT, Born 2 NT, reference RTM
    // NT + 2 nt, exact adjoint NT (source pass) + NT + 1 (reverse pass)
    for (const ShotDev &g : p->sd) {
      int64_t per = (op == OP_MODEL || op == OP_ILLUM || op == OP_ILLUM_PLANE) ? g.NT
                  : (op == OP_BORN || op == OP_BORN_PLANE) ? 2LL * g.NT
                  : (op == OP_RTM || op == OP_RTM_TRUE) ? g.NT + 2LL * g.nt
                  : op == OP_RTM_UPDOWN ? 2LL * g.NT + 3LL * g.nt
                  : op == OP_RTM_PLANE ? g.NT + 2LL * (g.NT - 2)
                                   : 2LL * g.NT + 1;
      p->cell_updates += (int64_t)g.NX * g.NZ * per;
    }
    rc = p->alloc(&p->d_sd, (size_t)nshot);
  }
  if (rc == SEIS_OK) rc = p->alloc(&p->d_tiles, p->tiles.size());
  if (rc == SEIS_OK) rc = p->alloc(&p->d_adj_tiles, p->adj_tiles.size());
  const bool imaging = op == OP_RTM || op == OP_RTM_PLANE || op == OP_RTM_TRUE || op == OP_RTM_UPDOWN;
  if (rc == SEIS_OK && imaging) rc = p->alloc(&p->d_cols, p->cols.size());
  if (rc == SEIS_OK && imaging) rc = p->alloc(&p->d_taps, (size_t)61);
  if (rc == SEIS_OK) {
    cudaStream_t st = ctx->stream;
    cudaError_t e = cudaMemcpyAsync(p->d_sd, p->sd.data(), sizeof(ShotDev) * nshot,
                                    cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(p->d_tiles, p->tiles.data(), sizeof(Tile) * p->tiles.size(),
                          cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(p->d_adj_tiles, p->adj_tiles.data(), sizeof(Tile) * p->adj_tiles.size(),
                          cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && imaging) {
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

// One time step of every shot: the interior-tile kernel on the main stream and
// the pad-tile kernel on the auxiliary stream, joined before the next step.
int step(Plan &p, int mode, const StepArgs &a0, const ShotDev *shots = nullptr) {
  seis_fd_ctx *ctx = p.ctx;
  StepArgs a = a0;
  a.loop = p.loop;
  cudaStream_t s_pad = ctx->stream;
  if (p.overlap) {
    CK(cudaEventRecord(ctx->fork, ctx->stream));
    CK(cudaStreamWaitEvent(ctx->aux, ctx->fork, 0));
    s_pad = ctx->aux;
  }
  CK(launch_step(mode, p.exact, shots ? shots : p.d_sd, p.d_tiles, p.n_int, p.n_pad, p.shape, a,
                 ctx->d_err, ctx->stream, s_pad));
  if (p.overlap) {
    CK(cudaEventRecord(ctx->join, ctx->aux));
    CK(cudaStreamWaitEvent(ctx->stream, ctx->join, 0));
  }
  ctx->launches += (p.n_int > 0) + (p.n_pad > 0);
  return SEIS_OK;
}

// Snapshot schedule of the adjoint imaging sum  sum_{k=0..K} f(k), K = NT-1,
// f(k) = lap_k * mu(L_{k+1}).  Every m-th step is stored, and step K as well;
// the stored steps t_0 = 0 < t_1 < ... < t_J = K carry trapezoid weights
//   w_j = (t_{j+1} - t_{j-1}) / 2  (+ 1/2 at each end),
// which sum to K + 1 and reduce to 1 for m = 1.  Against plain m-fold
// weights this removes the first-order end error of a wavefield that is
// still live at the last step.
int snap_slot(int k, int K, int m) {
  if (k < 0 || k > K) return -1;
  if (k % m == 0) return k / m;
  return k == K ? K / m + 1 : -1;
}

int snap_count(int K, int m) { return K / m + 1 + (K % m != 0); }

float snap_weight(int k, int K, int m) {
  if (m == 1) return 1.0f;
  const int prev = k == 0 ? k : (k % m == 0 ? k - m : (K / m) * m);
  const int next = k == K ? k : std::min(k + m, K);
  return 0.5f * (float)(next - prev + (k == 0) + (k == K));
}

// Snapshot slots held at once: every slot of the run, or with checkpoints
// those of one segment (ck_every / snap_every, and the last step's).
int snap_slots(const Plan &p, int NT) {
  return p.ck_every > 0 ? p.ck_every / p.snap_every + 1 : snap_count(NT - 1, p.snap_every);
}

// First snapshot slot of the segment that starts at step s0 (ck_every is a
// multiple of snap_every, so s0 is a stored step).
int seg_slot0(const Plan &p, int s0) { return p.ck_every > 0 ? s0 / p.snap_every : 0; }

// Checkpoint storage and the recompute shot table (after the snapshots).
int ensure_checkpoints(Plan &p) {
  seis_fd_ctx *ctx = p.ctx;
  p.sd_c = p.sd;
  p.ck.assign(p.nshot, {});
  const int nck = (p.NT - 1) / p.ck_every;  // checkpoints j = 1 .. nck
  for (int s = 0; s < p.nshot; s++) {
    ShotDev &c = p.sd_c[s];
    for (int k = 0; k < 3; k++) {
      int rc = alloc_field(p, c, &c.fa[k]);
      if (rc) return rc;
    }
    for (int j = 0; j < 2 * nck; j++) {
      float *f = nullptr;
      int rc = alloc_field(p, c, &f);
      if (rc) return rc;
      p.ck[s].push_back(f);
    }
    c.img = nullptr;
    c.grad = nullptr;
    c.illum = nullptr;
  }
  int rc = encode_maps(p, p.sd_c, &p.d_maps_c);
  if (!rc) rc = p.alloc(&p.d_sd_c, (size_t)p.nshot);
  if (rc) return rc;
  CK(cudaMemcpyAsync(p.d_sd_c, p.sd_c.data(), sizeof(ShotDev) * p.nshot, cudaMemcpyHostToDevice,
                     ctx->stream));
  return SEIS_OK;
}

// Snapshot storage of every shot (first run of an adjoint plan), then the
// shot table is uploaded again with the new pointers.
int ensure_snapshots(Plan &p) {
  if (p.snaps_ready) return SEIS_OK;
  seis_fd_ctx *ctx = p.ctx;
  const size_t esize = p.snap_dtype == SNAP_F32 ? 4 : 2;
  for (int s = 0; s < p.nshot; s++) {
    ShotDev &g = p.sd[s];
    int nsnap = snap_slots(p, g.NT);
    int ntx = (g.NX + shape_tx(p.shape) - 1) / shape_tx(p.shape);
    unsigned char *snap = nullptr;
    int rc = p.alloc(&snap, (size_t)nsnap * g.nx * g.nz * esize);
    if (!rc) rc = p.alloc(&g.snap_scale, (size_t)nsnap * ntx * g.ntz);
    if (rc) return rc;
    g.snap = snap;
    g.snap_dtype = p.snap_dtype;
    g.snap_every = p.snap_every;
  }
  CK(cudaMemcpyAsync(p.d_sd, p.sd.data(), sizeof(ShotDev) * p.nshot, cudaMemcpyHostToDevice,
                     ctx->stream));
  if (p.ck_every > 0) {
    int rc = ensure_checkpoints(p);
    if (rc) return rc;
  }
  p.snaps_ready = true;
  return SEIS_OK;
}

// One reverse step of the exact adjoint over the adjoint tile list.
int adj_step(Plan &p, const StepArgs &a0) {
  seis_fd_ctx *ctx = p.ctx;
  StepArgs a = a0;
  a.loop = p.loop;
  cudaStream_t s_pad = ctx->stream;
  if (p.overlap) {
    CK(cudaEventRecord(ctx->fork, ctx->stream));
    CK(cudaStreamWaitEvent(ctx->aux, ctx->fork, 0));
    s_pad = ctx->aux;
  }
  CK(fast::launch_adjoint(p.shape, p.d_sd, p.d_adj_tiles, p.n_int_adj, p.n_pad_adj, a,
                          ctx->d_err, ctx->stream, s_pad));
  if (p.overlap) {
    CK(cudaEventRecord(ctx->join, ctx->aux));
    CK(cudaStreamWaitEvent(ctx->stream, ctx->join, 0));
  }
  ctx->launches += (p.n_int_adj > 0) + (p.n_pad_adj > 0);
  return SEIS_OK;
}

// Zero every wavefield buffer (margins included) and the images.
int clear_fields(Plan &p) {
  seis_fd_ctx *ctx = p.ctx;
  for (const ShotDev &g : p.sd) {
    FieldGeom fg = field_geom(g.NX, g.NZ);
    for (int k = 0; k < 3; k++) {
      CK(cudaMemsetAsync(g.fa[k] - fg.origin, 0, sizeof(float) * fg.elems, ctx->stream));
      if (g.fb[k]) CK(cudaMemsetAsync(g.fb[k] - fg.origin, 0, sizeof(float) * fg.elems, ctx->stream));
    }
    if (g.img) CK(cudaMemsetAsync(g.img, 0, sizeof(float) * g.nx * g.nz, ctx->stream));
    if (g.grad) CK(cudaMemsetAsync(g.grad, 0, sizeof(double) * g.nx * g.nz, ctx->stream));
    if (g.comp) CK(cudaMemsetAsync(g.comp, 0, sizeof(float) * 4 * g.nx * g.nz, ctx->stream));
  }
  for (const ShotDev &g : p.sd_h) {
    FieldGeom fg = field_geom(g.NX, g.NZ);
    for (int k = 0; k < 3; k++)
      CK(cudaMemsetAsync(g.fa[k] - fg.origin, 0, sizeof(float) * fg.elems, ctx->stream));
  }
  return SEIS_OK;
}

int run_forward(Plan &p, int mode, const ShotDev *shots = nullptr) {
  StepArgs a{};
  a.nshots = p.nshot;
  for (int it = 0; it < p.NT; it++) {
    a.rot = it;
    a.rot_b = it;
    a.src_k = it >= 1 ? it - 1 : -1;
    int itp = it - p.ndel;
    const bool rtm = p.op == OP_RTM || p.op == OP_RTM_TRUE || p.op == OP_RTM_UPDOWN;
    const bool ill = p.op == OP_ILLUM || p.op == OP_ILLUM_PLANE;
    a.rec_k = (!rtm && p.op != OP_BORN_ADJ && !ill && itp >= 0) ? itp : -1;
    a.illum_on = ill && it > p.ndel;  // fd.cpp:318, :763
    a.strip_k = (rtm && itp >= 0) ? itp : -1;
    a.snap_k = p.op == OP_BORN_ADJ ? snap_slot(it, p.NT - 1, p.snap_every) : -1;
    int rc = step(p, mode, a, shots);
    if (rc) return rc;
  }
  return SEIS_OK;
}

// Reverse pass of the reference RTM (fd.cpp:654-693).
int run_rtm_reverse(Plan &p) {
  seis_fd_ctx *ctx = p.ctx;
  // the source fields restart from zero (fd.cpp:654-656)
  for (int s = 0; s < p.nshot; s++) {
    FieldGeom fg = field_geom(p.sd[s].NX, p.sd[s].NZ);
    for (int k = 0; k < 3; k++)
      CK(cudaMemsetAsync(p.sd[s].fa[k] - fg.origin, 0, sizeof(float) * fg.elems, ctx->stream));
  }
  StepArgs a{};
  a.nshots = p.nshot;
  a.src_k = -1;
  a.strip_k = -1;
  int k = 0;
  for (int it = p.NT - 1; it >= p.ndel; it--, k++) {
    a.rot = k;
    a.rot_b = k;
    CK(launch_rtm_restore(p.d_sd, p.nshot, p.max_strip, a.rot, it, ctx->stream));
    ctx->launches++;
    a.rec_k = -1;
    int rc = step(p, MODE_MODEL, a);
    if (rc) return rc;
    a.rec_k = it - p.ndel;
    rc = step(p, MODE_RCV, a);
    if (rc) return rc;
    CK(launch_rtm_image(p.d_sd, p.d_cols, (int)p.cols.size(), a.rot, a.rot_b, p.max_NZ,
                        p.d_taps, ctx->stream, p.op == OP_RTM_TRUE ? 2 : 0));
    ctx->launches++;
  }
  return SEIS_OK;
}

// adjointPlane (fd.cpp:787-921).  Pass 1 propagates the receiver field back
// in time from zero, injecting the gather and keeping the boundary layers of
// every step's current field; pass 2 runs the areal-source field forward from
// step 2 and, in step with it, the receiver field again from its two last
// pass-1 states, taking the gather off at the receiver rows and restoring the
// kept layers, imaging with FaQi alone.  Gather samples at negative indices
// are skipped (the reference reads outside its array there, fd.cpp:834, :873).
int run_rtm_plane(Plan &p) {
  seis_fd_ctx *ctx = p.ctx;
  for (const ShotDev &g : p.sd)
    CK(cudaMemsetAsync(g.strips, 0, sizeof(float) * (size_t)g.NT * g.strip_len, ctx->stream));
  const int NT = p.NT, ndel = p.ndel;
  StepArgs a{};
  a.nshots = p.nshot;
  a.src_k = -1;
  for (int j = 0; j < NT; j++) {  // pass 1, it = NT-1 .. 0 (fd.cpp:829-845)
    const int it = NT - 1 - j;
    a.rot_b = j;
    a.rec_k = it - ndel >= 0 ? it - ndel : -1;
    a.strip_k = it - 1 >= 0 ? it - 1 : -1;  // the new field is the next step's current
    int rc = step(p, MODE_RCV, a);
    if (rc) return rc;
  }
  // fd.cpp:846-850: (prev, cur, new) = (R0, R1, 0) for pass 2 with the buffers
  // in rotation order r0, r0+1, r0+2: R1 moves into the buffer after R0's
  const int r0 = NT + 1;
  for (const ShotDev &g : p.sd) {
    FieldGeom fg = field_geom(g.NX, g.NZ);
    float *b_r1 = g.fb[NT % 3] - fg.origin, *b_next = g.fb[(r0 + 1) % 3] - fg.origin;
    CK(cudaMemcpyAsync(b_next, b_r1, sizeof(float) * fg.elems, cudaMemcpyDeviceToDevice,
                       ctx->stream));
    CK(cudaMemsetAsync(b_r1, 0, sizeof(float) * fg.elems, ctx->stream));
  }
  for (int it = 2; it < NT; it++) {  // pass 2 (fd.cpp:853-893)
    const int k = it - 2;
    CK(launch_plane_rcv_prep(p.d_sd, p.nshot, p.max_strip, r0 + k, k > 0 ? it - 1 : -1,
                             it - ndel - 1 >= 0 ? it - ndel - 1 : -1, ctx->stream));
    ctx->launches++;
    StepArgs sa{};
    sa.nshots = p.nshot;
    sa.rot = k;
    sa.src_k = it - 1;
    int rc = step(p, MODE_MODEL, sa);
    if (rc) return rc;
    StepArgs ra{};
    ra.nshots = p.nshot;
    ra.rot_b = r0 + k;
    rc = step(p, MODE_RCV, ra);
    if (rc) return rc;
    if (it - ndel > 0) {
      CK(launch_rtm_image(p.d_sd, p.d_cols, (int)p.cols.size(), k, r0 + k, p.max_NZ, p.d_taps,
                          ctx->stream, 1));
      ctx->launches++;
    }
  }
  return SEIS_OK;
}

// Reverse pass of adjointUpDown (fd.cpp:449-537): the source fields of the
// wavelet and of its Hilbert transform reconstructed from their layers, the
// receiver field back-propagated, four-component imaging every step.
int run_updown_reverse(Plan &p) {
  seis_fd_ctx *ctx = p.ctx;
  for (const std::vector<ShotDev> *v : {&p.sd, &p.sd_h})
    for (const ShotDev &g : *v) {
      FieldGeom fg = field_geom(g.NX, g.NZ);
      for (int k = 0; k < 3; k++)
        CK(cudaMemsetAsync(g.fa[k] - fg.origin, 0, sizeof(float) * fg.elems, ctx->stream));
    }
  int k = 0;
  for (int it = p.NT - 1; it >= p.ndel; it--, k++) {
    for (const ShotDev *tab : {p.d_sd, p.d_sd_h}) {
      CK(launch_rtm_restore(tab, p.nshot, p.max_strip, k, it, ctx->stream));
      ctx->launches++;
      StepArgs a{};
      a.nshots = p.nshot;
      a.rot = k;
      int rc = step(p, MODE_MODEL, a, tab);
      if (rc) return rc;
    }
    StepArgs r{};
    r.nshots = p.nshot;
    r.rot_b = k;
    r.rec_k = it - p.ndel;
    int rc = step(p, MODE_RCV, r);
    if (rc) return rc;
    CK(launch_updown_image(p.d_sd, p.d_sd_h, p.d_cols, (int)p.cols.size(), k, k, p.max_NZ,
                           p.d_taps, ctx->stream));
    ctx->launches++;
  }
  CK(launch_updown_finalize(p.d_sd, p.nshot, ctx->stream));
  ctx->launches++;
  return SEIS_OK;
}

// Forward pass of the background field keeping the source-term snapshots
// (adjoint plans); reused by every later run until the velocity or the
// wavelet changes.
int source_pass(Plan &p) {
  int rc = SEIS_OK;
  if (p.ck_every == 0) {
    rc = run_forward(p, MODE_MODEL);
  } else {
    // the whole forward pass on the recompute table, keeping the two time
    // levels before every ck_every-th step instead of the snapshots
    seis_fd_ctx *ctx = p.ctx;
    for (const ShotDev &c : p.sd_c) {
      FieldGeom fg = field_geom(c.NX, c.NZ);
      for (int k = 0; k < 3; k++)
        CK(cudaMemsetAsync(c.fa[k] - fg.origin, 0, sizeof(float) * fg.elems, ctx->stream));
    }
    StepArgs a{};
    a.nshots = p.nshot;
    for (int it = 0; it < p.NT && !rc; it++) {
      if (it > 0 && it % p.ck_every == 0) {
        const int j = it / p.ck_every;
        for (int s = 0; s < p.nshot; s++) {
          const ShotDev &c = p.sd_c[s];
          FieldGeom fg = field_geom(c.NX, c.NZ);
          for (int l = 0; l < 2; l++)  // prev = fa[it % 3], cur = fa[(it + 1) % 3]
            CK(cudaMemcpyAsync(p.ck[s][2 * (j - 1) + l] - fg.origin, c.fa[(it + l) % 3] - fg.origin,
                               sizeof(float) * fg.elems, cudaMemcpyDeviceToDevice, ctx->stream));
        }
      }
      a.rot = it;
      a.rot_b = it;
      a.src_k = it >= 1 ? it - 1 : -1;
      rc = step(p, MODE_MODEL, a, p.d_sd_c);
    }
  }
  if (!rc) p.snaps_valid = true;
  return rc;
}

// Recompute the snapshots of forward steps s0 .. s1-1 (one checkpoint
// segment) into the segment buffer, from checkpoint s0 / ck_every.
int recompute_segment(Plan &p, int s0, int s1) {
  seis_fd_ctx *ctx = p.ctx;
  const int j = s0 / p.ck_every;
  for (int s = 0; s < p.nshot; s++) {
    const ShotDev &c = p.sd_c[s];
    FieldGeom fg = field_geom(c.NX, c.NZ);
    for (int l = 0; l < 2; l++) {
      float *dst = c.fa[(s0 + l) % 3] - fg.origin;
      if (j == 0)
        CK(cudaMemsetAsync(dst, 0, sizeof(float) * fg.elems, ctx->stream));
      else
        CK(cudaMemcpyAsync(dst, p.ck[s][2 * (j - 1) + l] - fg.origin, sizeof(float) * fg.elems,
                           cudaMemcpyDeviceToDevice, ctx->stream));
    }
  }
  StepArgs a{};
  a.nshots = p.nshot;
  const int slot0 = seg_slot0(p, s0);
  for (int it = s0; it < s1; it++) {
    a.rot = it;
    a.rot_b = it;
    a.src_k = it >= 1 ? it - 1 : -1;
    const int sl = snap_slot(it, p.NT - 1, p.snap_every);
    a.snap_k = sl >= 0 ? sl - slot0 : -1;
    int rc = step(p, MODE_MODEL, a, p.d_sd_c);
    if (rc) return rc;
  }
  return SEIS_OK;
}

// Reverse pass of the exact adjoint: L_k for k = NT .. 0 from L_{k+1}, L_{k+2};
// the step producing L_k images the source term of step k with mu(L_{k+1}).
// The exact adjoint's edge-band coefficients of every shot of the plan.
int edge_coefs(Plan &p) {
  seis_fd_ctx *ctx = p.ctx;
  int most = 0;
  for (const ShotDev &g : p.sd) most = std::max(most, edge_cells(g.NX, g.NZ));
  CK(fast::launch_edge_coef(p.d_sd, p.nshot, most, ctx->stream));
  ctx->launches++;
  return SEIS_OK;
}

int run_adjoint(Plan &p) {
  seis_fd_ctx *ctx = p.ctx;
  int rc0 = edge_coefs(p);
  if (rc0) return rc0;
  for (const ShotDev &g : p.sd) {
    FieldGeom fg = field_geom(g.NX, g.NZ);
    for (int k = 0; k < 3; k++)
      CK(cudaMemsetAsync(g.fa[k] - fg.origin, 0, sizeof(float) * fg.elems, ctx->stream));
    for (float *f : {g.adj_e[0], g.adj_e[1], g.adj_b})
      CK(cudaMemsetAsync(f - fg.origin, 0, sizeof(float) * fg.elems, ctx->stream));
  }
  StepArgs a{};
  a.nshots = p.nshot;
  a.src_k = -1;
  a.strip_k = -1;
  int r = 0;
  // with checkpoints, before the reverse steps of each segment [s0, s1) its
  // snapshots are recomputed (k = NT images nothing)
  const int C = p.ck_every > 0 ? p.ck_every : p.NT + 1;
  int slot0 = 0;
  for (int k = p.NT; k >= 0; k--, r++) {
    if (p.ck_every > 0 && k < p.NT && (k == p.NT - 1 || (k + 1) % C == 0)) {
      const int s0 = (k / C) * C;
      int rc = recompute_segment(p, s0, k + 1);
      if (rc) return rc;
      slot0 = seg_slot0(p, s0);
    }
    a.rot = r;
    a.rot_b = r;
    int kd = k - 1 - p.ndel;
    a.rec_k = (kd >= 0 && kd < p.nt) ? kd : -1;
    const int sl = snap_slot(k, p.NT - 1, p.snap_every);
    a.snap_k = sl >= 0 ? sl - slot0 : -1;
    a.img_w = sl >= 0 ? snap_weight(k, p.NT - 1, p.snap_every) : 0.0f;
    int rc = adj_step(p, a);
    if (rc) return rc;
  }
  CK(launch_finalize_image(p.d_sd, p.nshot, ctx->stream));
  ctx->launches++;
  return SEIS_OK;
}

// The whole operator as a stream of launches (captured into a graph by
// plan_run).
int enqueue_operator(Plan &p) {
  int rc = clear_fields(p);
  if (rc) return rc;
  switch (p.op) {
    case OP_MODEL: return run_forward(p, MODE_MODEL);
    case OP_BORN: return run_forward(p, MODE_BORN);
    case OP_RTM:
      rc = run_forward(p, MODE_MODEL);
      return rc ? rc : run_rtm_reverse(p);
    case OP_BORN_ADJ:
      rc = ensure_snapshots(p);
      if (!rc && !p.snaps_valid) rc = source_pass(p);
      return rc ? rc : run_adjoint(p);
    case OP_ILLUM:
    case OP_ILLUM_PLANE: return run_forward(p, MODE_MODEL);
    case OP_BORN_PLANE: return run_forward(p, MODE_BORN);
    case OP_RTM_PLANE: return run_rtm_plane(p);
    case OP_RTM_TRUE:
      rc = run_forward(p, MODE_MODEL);
      return rc ? rc : run_rtm_reverse(p);
    case OP_RTM_UPDOWN:
      rc = run_forward(p, MODE_MODEL);
      if (!rc) rc = run_forward(p, MODE_MODEL, p.d_sd_h);
      return rc ? rc : run_updown_reverse(p);
  }
  return fail(p.ctx, SEIS_ERR_NOTSUP, "unknown operator %d", p.op);
}

int plan_run(Plan &p) {
  seis_fd_ctx *ctx = p.ctx;
  if (!p.exec) {
    // everything that allocates happens before the capture
    if (p.op == OP_BORN_ADJ) {
      int rc0 = ensure_snapshots(p);
      if (rc0) return rc0;
      CK(cudaStreamSynchronize(ctx->stream));
    }
  }
  // the source pass runs outside the graph, only when its inputs changed
  if (p.op == OP_BORN_ADJ && !p.snaps_valid) {
    int rc0 = source_pass(p);
    if (rc0) return rc0;
  }
  if (!p.exec) {
    int64_t before = ctx->launches;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_operator(p);
    if (rc && p.overlap) {
      // rejoin the auxiliary stream so that it leaves the capture with the
      // main stream (an unjoined fork would keep it capturing)
      cudaEventRecord(ctx->join, ctx->aux);
      cudaStreamWaitEvent(ctx->stream, ctx->join, 0);
    }
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return rc;
    }
    CK(e);
    p.graph = g;
    CK(cudaGraphInstantiate(&p.exec, p.graph, 0));
    p.launches_per_run = ctx->launches - before;
    ctx->launches = before;
  }
  CK(cudaGraphLaunch(p.exec, ctx->stream));
  ctx->launches += p.launches_per_run;
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



int sync(seis_fd_ctx *ctx) {
  CK(cudaStreamSynchronize(ctx->stream));
  int flag = 0;
  CK(cudaMemcpy(&flag, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag) {
    CK(cudaMemset(ctx->d_err, 0, sizeof(int)));
    return fail(ctx, SEIS_ERR_CUDA, "a kernel gave up waiting for its staged input (code %d)", flag);
  }
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
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->aux, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->join, cudaEventDisableTiming);
  if (e == cudaSuccess) e = configure_kernels();
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_partial, sizeof(double) * DOT_PARTS);
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_scalar, sizeof(double));
  if (e == cudaSuccess) e = cudaMemset(ctx->d_err, 0, sizeof(int));
  if (e != cudaSuccess) {
    seis_fd_destroy(ctx);
    return SEIS_ERR_CUDA;
  }
  *out = ctx;
  return SEIS_OK;
}

int seis_fd_destroy(seis_fd_ctx *ctx) {
  if (!ctx) return SEIS_OK;
  cudaSetDevice(ctx->device);
  // plans still alive lose their device state; their handles stay valid for
  // seis_fd_plan_destroy, every other call on them returns SEIS_ERR_ARG
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (seis_fd_plan *h : ctx->plans) {
    delete h->p;
    h->p = nullptr;
  }
  ctx->plans.clear();
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->aux) cudaStreamSynchronize(ctx->aux);
  if (ctx->d_err) cudaFree(ctx->d_err);
  if (ctx->d_partial) cudaFree(ctx->d_partial);
  if (ctx->d_scalar) cudaFree(ctx->d_scalar);
  if (ctx->fork) cudaEventDestroy(ctx->fork);
  if (ctx->join) cudaEventDestroy(ctx->join);
  if (ctx->aux) cudaStreamDestroy(ctx->aux);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return SEIS_OK;
}

const char *seis_fd_last_error(const seis_fd_ctx *ctx) { return ctx ? ctx->err.c_str() : ""; }

int64_t seis_fd_launch_count(const seis_fd_ctx *ctx) { return ctx ? ctx->launches : 0; }

void *seis_fd_stream(const seis_fd_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

// ---------------------------------------------------------------- plans

int seis_fd_plan_create(seis_fd_ctx *ctx, int op, int nshot, const seis_shot_desc *shots,
                        seis_fd_plan **out) {
  int rc = begin(ctx);
  if (rc) return rc;
  if (!out) return fail(ctx, SEIS_ERR_ARG, "out is null");
  *out = nullptr;
  if (op < SEIS_OP_MODELING || op > SEIS_OP_ILLUM_PLANE) return fail(ctx, SEIS_ERR_ARG, "op=%d", op);
  Plan *p = nullptr;
  rc = plan_create(ctx, op, nshot, shots, &p);
  if (rc) return rc;
  seis_fd_plan *h = new (std::nothrow) seis_fd_plan{p};
  if (!h) {
    delete p;
    return fail(ctx, SEIS_ERR_NOMEM, "host allocation failed");
  }
  ctx->plans.push_back(h);
  *out = h;
  return SEIS_OK;
}

int seis_fd_plan_destroy(seis_fd_plan *plan) {
  if (!plan) return SEIS_OK;
  if (plan->p) {
    seis_fd_ctx *ctx = plan->p->ctx;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    auto &v = ctx->plans;
    v.erase(std::remove(v.begin(), v.end(), plan), v.end());
    delete plan->p;
  }
  delete plan;
  return SEIS_OK;
}

static int plan_input(seis_fd_plan *plan, int shot, int what, const float *src, bool device) {
  if (!plan || !plan->p) return SEIS_ERR_ARG;
  Plan &p = *plan->p;
  seis_fd_ctx *ctx = p.ctx;
  int rc = begin(ctx);
  if (rc) return rc;
  if (shot < 0 || shot >= p.nshot) return fail(ctx, SEIS_ERR_ARG, "shot=%d of %d", shot, p.nshot);
  if (!src) return fail(ctx, SEIS_ERR_ARG, "null source");
  const seis_shot_desc &d = p.desc[shot];
  ShotDev &g = p.sd[shot];
  cudaMemcpyKind kind = device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  if (what == SEIS_IN_VEL || what == SEIS_IN_WAVELET || what == SEIS_IN_WAVELET_H)
    p.snaps_valid = false;
  switch (what) {
    case SEIS_IN_VEL:
    case SEIS_IN_DV: {
      if (what == SEIS_IN_DV && !g.dv) return fail(ctx, SEIS_ERR_NOTSUP, "plan has no dv input");
      CK(cudaMemcpyAsync(p.d_stage, src, sizeof(float) * d.nx * d.nz, kind, ctx->stream));
      float *dst = const_cast<float *>(what == SEIS_IN_VEL ? g.vel : g.dv);
      CK(launch_pad(p.d_stage, d.nx, d.nz, d.pml, g.LDZ, what == SEIS_IN_VEL, dst, ctx->stream));
      ctx->launches++;
      return SEIS_OK;
    }
    case SEIS_IN_WAVELET:
      CK(cudaMemcpyAsync(const_cast<float *>(g.wav), src, sizeof(float) * g.NT, kind, ctx->stream));
      return SEIS_OK;
    case SEIS_IN_WAVELET_H:
      if (p.sd_h.empty()) return fail(ctx, SEIS_ERR_NOTSUP, "plan takes no Hilbert wavelet");
      CK(cudaMemcpyAsync(const_cast<float *>(p.sd_h[shot].wav), src, sizeof(float) * g.NT, kind,
                         ctx->stream));
      return SEIS_OK;
    case SEIS_IN_SOURCE:
      if (!g.sou) return fail(ctx, SEIS_ERR_NOTSUP, "plan takes no areal source");
      CK(cudaMemcpyAsync(p.d_stage, src, sizeof(float) * d.nx * g.NT, kind, ctx->stream));
      CK(launch_transpose(p.d_stage, d.nx, g.NT, const_cast<float *>(g.sou), ctx->stream));
      ctx->launches++;
      return SEIS_OK;
    case SEIS_IN_GATHER:
      if (p.op != OP_RTM && p.op != OP_BORN_ADJ && p.op != OP_RTM_PLANE && p.op != OP_RTM_TRUE &&
          p.op != OP_RTM_UPDOWN)
        return fail(ctx, SEIS_ERR_NOTSUP, "plan takes no gather input");
      CK(cudaMemcpyAsync(p.d_stage, src, sizeof(float) * d.nt * d.nx, kind, ctx->stream));
      CK(launch_transpose(p.d_stage, d.nx, d.nt, g.rec, ctx->stream));
      ctx->launches++;
      return SEIS_OK;
  }
  return fail(ctx, SEIS_ERR_ARG, "unknown input %d", what);
}

int seis_fd_plan_set(seis_fd_plan *plan, int shot, int what, const float *h_src) {
  return plan_input(plan, shot, what, h_src, false);
}

int seis_fd_plan_set_device(seis_fd_plan *plan, int shot, int what, const float *d_src) {
  return plan_input(plan, shot, what, d_src, true);
}

int seis_fd_plan_run(seis_fd_plan *plan) {
  if (!plan || !plan->p) return SEIS_ERR_ARG;
  int rc = begin(plan->p->ctx);
  return rc ? rc : plan_run(*plan->p);
}

int seis_fd_plan_get(seis_fd_plan *plan, int shot, int what, float *h_dst) {
  if (!plan || !plan->p) return SEIS_ERR_ARG;
  Plan &p = *plan->p;
  seis_fd_ctx *ctx = p.ctx;
  int rc = begin(ctx);
  if (rc) return rc;
  if (shot < 0 || shot >= p.nshot) return fail(ctx, SEIS_ERR_ARG, "shot=%d of %d", shot, p.nshot);
  if (!h_dst) return fail(ctx, SEIS_ERR_ARG, "null destination");
  if (what == SEIS_OUT_GATHER) {
    if (p.op == OP_RTM || p.op == OP_BORN_ADJ || p.op == OP_ILLUM || p.op == OP_RTM_PLANE ||
        p.op == OP_RTM_TRUE || p.op == OP_RTM_UPDOWN || p.op == OP_ILLUM_PLANE)
      return fail(ctx, SEIS_ERR_NOTSUP, "this plan outputs images");
    rc = download_gather(p, shot, h_dst);
  } else if (what == SEIS_OUT_IMAGE) {
    if (p.op != OP_RTM && p.op != OP_BORN_ADJ && p.op != OP_ILLUM && p.op != OP_RTM_PLANE &&
        p.op != OP_RTM_TRUE && p.op != OP_RTM_UPDOWN && p.op != OP_ILLUM_PLANE)
      return fail(ctx, SEIS_ERR_NOTSUP, "plan outputs gathers");
    const seis_shot_desc &d = p.desc[shot];
    CK(cudaMemcpyAsync(h_dst, p.sd[shot].img, sizeof(float) * d.nx * d.nz,
                       cudaMemcpyDeviceToHost, ctx->stream));
  } else if (what == SEIS_OUT_COMPONENTS) {
    if (!p.sd[shot].comp) return fail(ctx, SEIS_ERR_NOTSUP, "plan has no imaging components");
    const seis_shot_desc &d = p.desc[shot];
    CK(cudaMemcpyAsync(h_dst, p.sd[shot].comp, sizeof(float) * 4 * d.nx * d.nz,
                       cudaMemcpyDeviceToHost, ctx->stream));
  } else {
    return fail(ctx, SEIS_ERR_ARG, "unknown output %d", what);
  }
  return rc ? rc : sync(ctx);
}

int seis_fd_plan_sync(seis_fd_plan *plan) {
  if (!plan || !plan->p) return SEIS_ERR_ARG;
  int rc = begin(plan->p->ctx);
  return rc ? rc : sync(plan->p->ctx);
}

int64_t seis_fd_plan_cell_updates(const seis_fd_plan *plan) {
  return plan && plan->p ? plan->p->cell_updates : 0;
}

int64_t seis_fd_plan_launches_per_run(const seis_fd_plan *plan) {
  return plan && plan->p ? plan->p->launches_per_run : 0;
}

namespace {
// 2 x `steps` time steps of the plan's step kernels (forward plans: the
// operator's step; adjoint plans: the reverse step without imaging): first
// the interior and the pad kernel one after the other, each bracketed by CUDA
// events on its own stream, then `steps` steps as a run launches them (one
// after the other, or concurrently on two streams when the plan overlaps
// them).  ms = mean interior and pad kernel milliseconds (each
// alone) and mean step milliseconds (as run); bytes = algorithmic bytes of
// the interior and pad tiles (16 per field cell-update).  The fields are
// cleared afterwards.
int time_steps(Plan &p, int steps, double *ms, double *bytes) {
  seis_fd_ctx *ctx = p.ctx;
  const int TX = shape_tx(p.shape), TZ = shape_tz(p.shape);
  int mode = p.op == OP_BORN ? MODE_BORN : MODE_MODEL;
  int fields = p.op == OP_BORN ? 2 : 1;
  cudaEvent_t ev[5];
  for (auto &e : ev) CK(cudaEventCreate(&e));
  const bool adj = p.op == OP_BORN_ADJ;
  const std::vector<Tile> &tl = adj ? p.adj_tiles : p.tiles;
  const int n_int = adj ? p.n_int_adj : p.n_int, n_pad = adj ? p.n_pad_adj : p.n_pad;
  const Tile *d_tl = adj ? p.d_adj_tiles : p.d_tiles;
  int64_t cells_int = 0, cells_pad = 0;
  for (size_t i = 0; i < tl.size(); i++) {
    const Tile &t = tl[i];
    const ShotDev &g = p.sd[t.shot];
    int64_t c = (int64_t)std::min(TX, g.NX - t.x0) * std::min(TZ, g.NZ - t.z0);
    ((int)i < n_int ? cells_int : cells_pad) += c;
  }
  if (adj) {
    int rc0 = edge_coefs(p);
    if (rc0) return rc0;
  }
  StepArgs a{};
  a.nshots = p.nshot;
  a.strip_k = -1;
  a.loop = p.loop;
  // the interior tiles (the list's first n_int) or the pad tiles alone, on
  // the main / auxiliary stream
  auto launch = [&](bool interior) -> cudaError_t {
    const int ni = interior ? n_int : 0, np = interior ? 0 : n_pad;
    const Tile *t0 = interior ? d_tl : d_tl + n_int;
    return adj ? fast::launch_adjoint(p.shape, p.d_sd, t0, ni, np, a, ctx->d_err, ctx->stream,
                                      ctx->aux)
               : launch_step(mode, p.exact, p.d_sd, t0, ni, np, p.shape, a, ctx->d_err,
                             ctx->stream, ctx->aux);
  };
  double t_int = 0, t_pad = 0, t_step = 0;
  for (int k = 0; k < 2 * steps; k++) {
    const bool alone = k < steps;  // first each kernel alone, then the step as it runs
    a.rot = k; a.rot_b = k;
    int it = k % p.NT;
    a.src_k = it >= 1 ? it - 1 : -1;
    a.rec_k = it - p.ndel >= 0 && p.op != OP_RTM && !adj ? it - p.ndel : -1;
    CK(cudaEventRecord(ev[0], ctx->stream));
    if (alone) {
      CK(launch(true));
      CK(cudaEventRecord(ev[1], ctx->stream));
      CK(cudaEventRecord(ev[2], ctx->stream));
      CK(cudaStreamWaitEvent(ctx->aux, ev[2], 0));
      CK(launch(false));
      CK(cudaEventRecord(ev[3], ctx->aux));
      CK(cudaStreamWaitEvent(ctx->stream, ev[3], 0));
    } else if (p.overlap) {
      CK(cudaStreamWaitEvent(ctx->aux, ev[0], 0));
      CK(adj ? fast::launch_adjoint(p.shape, p.d_sd, d_tl, n_int, n_pad, a, ctx->d_err,
                                    ctx->stream, ctx->aux)
             : launch_step(mode, p.exact, p.d_sd, d_tl, n_int, n_pad, p.shape, a, ctx->d_err,
                           ctx->stream, ctx->aux));
      CK(cudaEventRecord(ev[3], ctx->aux));
      CK(cudaStreamWaitEvent(ctx->stream, ev[3], 0));
    } else {
      CK(adj ? fast::launch_adjoint(p.shape, p.d_sd, d_tl, n_int, n_pad, a, ctx->d_err,
                                    ctx->stream, ctx->stream)
             : launch_step(mode, p.exact, p.d_sd, d_tl, n_int, n_pad, p.shape, a, ctx->d_err,
                           ctx->stream, ctx->stream));
    }
    CK(cudaEventRecord(ev[4], ctx->stream));
    CK(cudaEventSynchronize(ev[4]));
    if (alone) {
      float a1 = 0, a2 = 0;
      CK(cudaEventElapsedTime(&a1, ev[0], ev[1]));
      CK(cudaEventElapsedTime(&a2, ev[2], ev[3]));
      t_int += a1; t_pad += a2;
    } else {
      float a3 = 0;
      CK(cudaEventElapsedTime(&a3, ev[0], ev[4]));
      t_step += a3;
    }
    ctx->launches += 2;
  }
  for (auto &e : ev) cudaEventDestroy(e);
  ms[0] = t_int / steps; ms[1] = t_pad / steps; ms[2] = t_step / steps;
  if (bytes) {
    bytes[0] = 16.0 * fields * (double)cells_int;
    bytes[1] = 16.0 * fields * (double)cells_pad;
  }
  return clear_fields(p) ? SEIS_ERR_CUDA : sync(ctx);
}

// Switch a plan to tile shape s: tile lists, tensor-map boxes and
// snapshot-scale tiling of every shot table, and a new graph at the next run.
// The snapshot scales are tiled like the kernels, so the shape is fixed once
// the snapshots exist.
int apply_shape(Plan &p, int s) {
  seis_fd_ctx *ctx = p.ctx;
  if (s < 0 || s >= NSHAPES) return fail(ctx, SEIS_ERR_ARG, "tile shape %d", s);
  if (s == p.shape) return SEIS_OK;
  if (p.snaps_ready)
    return fail(ctx, SEIS_ERR_STATE, "the tile shape is fixed once snapshots are allocated");
  CK(cudaStreamSynchronize(ctx->stream));
  p.shape = s;
  const int TZ = shape_tz(s);
  for (std::vector<ShotDev> *v : {&p.sd, &p.sd_c, &p.sd_h})
    for (ShotDev &g : *v) g.ntz = (g.NZ + TZ - 1) / TZ;
  build_tiles(p);
  build_adj_tiles(p);
  p.release(p.d_tiles);
  p.release(p.d_adj_tiles);
  p.d_tiles = p.d_adj_tiles = nullptr;
  int rc = p.alloc(&p.d_tiles, p.tiles.size());
  if (!rc) rc = p.alloc(&p.d_adj_tiles, p.adj_tiles.size());
  struct Table { std::vector<ShotDev> *sd; ShotDev **d; CUtensorMap **maps; };
  for (Table t : {Table{&p.sd, &p.d_sd, &p.d_maps}, Table{&p.sd_c, &p.d_sd_c, &p.d_maps_c},
                  Table{&p.sd_h, &p.d_sd_h, &p.d_maps_h}}) {
    if (rc || t.sd->empty() || !*t.d) continue;
    p.release(*t.maps);
    *t.maps = nullptr;
    rc = encode_maps(p, *t.sd, t.maps);
    if (!rc) {
      cudaError_t e = cudaMemcpyAsync(*t.d, t.sd->data(), sizeof(ShotDev) * p.nshot,
                                      cudaMemcpyHostToDevice, ctx->stream);
      if (e != cudaSuccess) rc = fail(ctx, SEIS_ERR_CUDA, "shot table: %s", cudaGetErrorString(e));
    }
  }
  if (rc) return rc;
  CK(cudaMemcpyAsync(p.d_tiles, p.tiles.data(), sizeof(Tile) * p.tiles.size(),
                     cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(p.d_adj_tiles, p.adj_tiles.data(), sizeof(Tile) * p.adj_tiles.size(),
                     cudaMemcpyHostToDevice, ctx->stream));
  if (p.exec) cudaGraphExecDestroy(p.exec);
  if (p.graph) cudaGraphDestroy(p.graph);
  p.exec = nullptr;
  p.graph = nullptr;
  return sync(ctx);
}

// Tile shape chosen for a plan signature (operator, build flavour and every
// shot's padded grid), shared by the plans of the process.
std::mutex g_tune_mu;
std::map<std::string, int> g_tune_cache;

std::string tune_key(const Plan &p) {
  std::string k = std::to_string(p.op) + (p.exact ? "e" : "f");
  for (const ShotDev &g : p.sd) k += ":" + std::to_string(g.NX) + "x" + std::to_string(g.NZ);
  return k;
}

// The launch form of a plan's steps (the captured graph follows it).
void set_launch(Plan &p, bool overlap, int loop) {
  if (p.overlap == overlap && p.loop == loop) return;
  p.overlap = overlap;
  p.loop = loop;
  if (p.exec) cudaGraphExecDestroy(p.exec);
  if (p.graph) cudaGraphDestroy(p.graph);
  p.exec = nullptr;
  p.graph = nullptr;
}

// Time `steps` steps of the plan in every tile shape and launch form (the
// interior kernel one tile per CTA or persistent, the interior and pad
// kernels one after the other or concurrently) and keep the fastest (the
// cached choice for this plan's signature unless `force`).  ms: the shortest
// mean step time of every shape (0 where not timed), may be null.
int autotune(Plan &p, int steps, bool force, double *ms, int *best) {
  const std::string key = tune_key(p);
  if (ms)
    for (int s = 0; s < NSHAPES; s++) ms[s] = 0.0;
  // choice = 4 shape + 2 persistent + overlap
  auto apply = [&](int c) {
    set_launch(p, (c & 1) != 0, (c >> 1) & 1);
    return apply_shape(p, c >> 2);
  };
  if (!force) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      if (best) *best = it->second >> 2;
      return apply(it->second);
    }
  }
  int pick = 0;
  double t_best = 0.0;
  for (int c = 0; c < 4 * NSHAPES; c++) {
    int rc = apply(c);
    double t[3];
    if (!rc) rc = time_steps(p, 3, t, nullptr);  // warm-up
    if (!rc) rc = time_steps(p, steps, t, nullptr);
    if (rc) return rc;
    const int s = c >> 2;
    if (ms && (ms[s] == 0.0 || t[2] < ms[s])) ms[s] = t[2];
    if (c == 0 || t[2] < t_best) {
      t_best = t[2];
      pick = c;
    }
  }
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_cache[key] = pick;
  }
  if (best) *best = pick >> 2;
  return apply(pick);
}
}  // namespace

int seis_fd_plan_time_kernels(seis_fd_plan *plan, int steps, double *ms, double *bytes) {
  if (!plan || !plan->p || !ms || !bytes || steps < 1) return SEIS_ERR_ARG;
  int rc = begin(plan->p->ctx);
  return rc ? rc : time_steps(*plan->p, steps, ms, bytes);
}

int seis_fd_plan_set_tile_shape(seis_fd_plan *plan, int shape) {
  if (!plan || !plan->p) return SEIS_ERR_ARG;
  int rc = begin(plan->p->ctx);
  return rc ? rc : apply_shape(*plan->p, shape);
}

int seis_fd_plan_tile_shape(const seis_fd_plan *plan) {
  return plan && plan->p ? plan->p->shape : SEIS_ERR_ARG;
}

int seis_fd_plan_set_launch(seis_fd_plan *plan, int flags) {
  if (!plan || !plan->p) return SEIS_ERR_ARG;
  if (flags & ~(SEIS_LAUNCH_OVERLAP | SEIS_LAUNCH_PERSISTENT | SEIS_LAUNCH_PER_TILE) ||
      ((flags & SEIS_LAUNCH_PERSISTENT) && (flags & SEIS_LAUNCH_PER_TILE)))
    return fail(plan->p->ctx, SEIS_ERR_ARG, "launch flags %d", flags);
  const int loop = (flags & SEIS_LAUNCH_PERSISTENT) ? 1 : (flags & SEIS_LAUNCH_PER_TILE) ? 0 : -1;
  set_launch(*plan->p, (flags & SEIS_LAUNCH_OVERLAP) != 0, loop);
  return SEIS_OK;
}

int seis_fd_plan_launch(const seis_fd_plan *plan) {
  if (!plan || !plan->p) return SEIS_ERR_ARG;
  const Plan &p = *plan->p;
  return (p.overlap ? SEIS_LAUNCH_OVERLAP : 0) | (p.loop > 0 ? SEIS_LAUNCH_PERSISTENT : 0) |
         (p.loop == 0 ? SEIS_LAUNCH_PER_TILE : 0);
}

int seis_fd_plan_autotune(seis_fd_plan *plan, int steps, int force, double *h_ms, int *h_best) {
  if (!plan || !plan->p || steps < 1) return SEIS_ERR_ARG;
  int rc = begin(plan->p->ctx);
  return rc ? rc : autotune(*plan->p, steps, force != 0, h_ms, h_best);
}

int seis_fd_plan_set_snapshots(seis_fd_plan *plan, int every, int dtype) {
  if (!plan || !plan->p) return SEIS_ERR_ARG;
  Plan &p = *plan->p;
  if (p.op != OP_BORN_ADJ) return fail(p.ctx, SEIS_ERR_NOTSUP, "plan keeps no snapshots");
  if (every < 1 || dtype < SEIS_SNAP_F32 || dtype > SEIS_SNAP_F16)
    return fail(p.ctx, SEIS_ERR_ARG, "snapshots every=%d dtype=%d", every, dtype);
  if (p.snaps_ready) return fail(p.ctx, SEIS_ERR_STATE, "snapshots already allocated");
  if (p.ck_every > 0 && p.ck_every % every != 0)
    return fail(p.ctx, SEIS_ERR_ARG, "snapshot interval %d does not divide the checkpoint interval %d",
                every, p.ck_every);
  p.snap_every = every;
  p.snap_dtype = dtype;
  return SEIS_OK;
}

int seis_fd_plan_set_checkpoints(seis_fd_plan *plan, int every) {
  if (!plan || !plan->p) return SEIS_ERR_ARG;
  Plan &p = *plan->p;
  if (p.op != OP_BORN_ADJ) return fail(p.ctx, SEIS_ERR_NOTSUP, "plan keeps no snapshots");
  if (every < 0 || (every > 0 && every % p.snap_every != 0))
    return fail(p.ctx, SEIS_ERR_ARG, "checkpoints every=%d: a multiple of the snapshot interval %d",
                every, p.snap_every);
  if (p.snaps_ready) return fail(p.ctx, SEIS_ERR_STATE, "snapshots already allocated");
  // the segment recomputation adds one forward field per step to a run
  for (const ShotDev &g : p.sd)
    p.cell_updates += (int64_t)g.NX * g.NZ * g.NT * ((every > 0) - (p.ck_every > 0));
  p.ck_every = every;
  return SEIS_OK;
}

int64_t seis_fd_plan_device_bytes(const seis_fd_plan *plan) {
  return plan && plan->p ? plan->p->device_bytes : 0;
}

int seis_fd_plan_set_exact(seis_fd_plan *plan, int exact) {
  if (!plan || !plan->p) return SEIS_ERR_ARG;
  Plan &p = *plan->p;
  if (p.exact != (exact != 0)) {
    p.exact = exact != 0;
    if (p.exec) cudaGraphExecDestroy(p.exec);
    if (p.graph) cudaGraphDestroy(p.graph);
    p.exec = nullptr;
    p.graph = nullptr;
  }
  return SEIS_OK;
}

// ------------------------------------------------------- one-call batches
static int run_batch(seis_fd_ctx *ctx, int op, int nshot, const seis_shot_desc *shots,
                     const float *const *in1, int what1, const float *const *in2, int what2,
                     const float *const *in3, int what3, float *const *out, int what_out) {
  int rc = begin(ctx);
  if (rc) return rc;
  if (!in1 || !in2 || (what3 >= 0 && !in3) || !out)
    return fail(ctx, SEIS_ERR_ARG, "null array list");
  Plan *p = nullptr;
  rc = plan_create(ctx, op, nshot, shots, &p);
  if (rc) return rc;
  seis_fd_plan h{p};
  for (int s = 0; s < nshot && !rc; s++) {
    rc = plan_input(&h, s, what1, in1[s], false);
    if (!rc) rc = plan_input(&h, s, what2, in2[s], false);
    if (!rc && what3 >= 0) rc = plan_input(&h, s, what3, in3[s], false);
  }
  if (!rc) rc = enqueue_operator(*p);  // one run: no graph
  for (int s = 0; s < nshot && !rc; s++) rc = seis_fd_plan_get(&h, s, what_out, out[s]);
  if (!rc) rc = sync(ctx);
  cudaStreamSynchronize(ctx->stream);
  delete p;
  return rc;
}

int seis_fd_modeling(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_wav,
                     const float *h_vel, float *h_rec) {
  return run_batch(ctx, OP_MODEL, 1, shot, &h_wav, SEIS_IN_WAVELET, &h_vel, SEIS_IN_VEL, nullptr,
                   -1, &h_rec, SEIS_OUT_GATHER);
}

int seis_fd_born(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_wav,
                 const float *h_vel, const float *h_dv, float *h_rec) {
  return run_batch(ctx, OP_BORN, 1, shot, &h_wav, SEIS_IN_WAVELET, &h_vel, SEIS_IN_VEL, &h_dv,
                   SEIS_IN_DV, &h_rec, SEIS_OUT_GATHER);
}

int seis_fd_hilbert(const float *in, float *out, int n, int half) {
  if (!in || !out || n < 0 || half < 1) return SEIS_ERR_ARG;
  std::vector<float> h((size_t)(2 * half + 1));
  hilbert_taps(h.data(), half);
  // a full convolution cut to the input length, summed in increasing input
  // index; a tap of exactly zero adds nothing (hilbert.h:42-54)
  for (int k = 0; k < n; k++) {
    const int i0 = std::max(0, k - half), i1 = std::min(n - 1, k + half);
    float acc = 0.0f;
    for (int i = i0; i <= i1; i++) {
      const float hk = h[(size_t)(k - i + half)];
      if (hk != 0.0f) acc += in[i] * hk;
    }
    out[k] = acc;
  }
  return SEIS_OK;
}

int seis_fd_born_plane(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_sou,
                       const float *h_vel, const float *h_dv, float *h_rec) {
  if (!shot) return begin(ctx) ? SEIS_ERR_ARG : fail(ctx, SEIS_ERR_ARG, "null shot");
  seis_shot_desc d = *shot;
  d.sx = d.nx / 2;  // the areal source has no point position
  return run_batch(ctx, OP_BORN_PLANE, 1, &d, &h_sou, SEIS_IN_SOURCE, &h_vel, SEIS_IN_VEL,
                   &h_dv, SEIS_IN_DV, &h_rec, SEIS_OUT_GATHER);
}

int seis_fd_rtm_plane(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_sou,
                      const float *h_vel, const float *h_rec, float *h_img) {
  if (!shot) return begin(ctx) ? SEIS_ERR_ARG : fail(ctx, SEIS_ERR_ARG, "null shot");
  seis_shot_desc d = *shot;
  d.sx = d.nx / 2;  // the areal source has no point position
  return run_batch(ctx, OP_RTM_PLANE, 1, &d, &h_sou, SEIS_IN_SOURCE, &h_vel, SEIS_IN_VEL,
                   &h_rec, SEIS_IN_GATHER, &h_img, SEIS_OUT_IMAGE);
}

int seis_fd_illum_plane(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_sou,
                        const float *h_vel, float *h_ss) {
  return run_batch(ctx, OP_ILLUM_PLANE, 1, shot, &h_sou, SEIS_IN_SOURCE, &h_vel, SEIS_IN_VEL,
                   nullptr, -1, &h_ss, SEIS_OUT_IMAGE);
}

int seis_fd_rtm_updown(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_wav,
                       const float *h_wavh, const float *h_vel, const float *h_rec, float *h_img,
                       float *h_comp) {
  int rc = begin(ctx);
  if (rc) return rc;
  if (!h_wav || !h_wavh || !h_vel || !h_rec || !h_img) return fail(ctx, SEIS_ERR_ARG, "null array");
  Plan *p = nullptr;
  rc = plan_create(ctx, OP_RTM_UPDOWN, 1, shot, &p);
  if (rc) return rc;
  seis_fd_plan h{p};
  rc = plan_input(&h, 0, SEIS_IN_WAVELET, h_wav, false);
  if (!rc) rc = plan_input(&h, 0, SEIS_IN_WAVELET_H, h_wavh, false);
  if (!rc) rc = plan_input(&h, 0, SEIS_IN_VEL, h_vel, false);
  if (!rc) rc = plan_input(&h, 0, SEIS_IN_GATHER, h_rec, false);
  if (!rc) rc = enqueue_operator(*p);
  if (!rc) rc = seis_fd_plan_get(&h, 0, SEIS_OUT_IMAGE, h_img);
  if (!rc && h_comp) rc = seis_fd_plan_get(&h, 0, SEIS_OUT_COMPONENTS, h_comp);
  if (!rc) rc = sync(ctx);
  cudaStreamSynchronize(ctx->stream);
  delete p;
  return rc;
}

int seis_fd_rtm_true(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_wav,
                     const float *h_vel, const float *h_rec, float *h_img) {
  return run_batch(ctx, OP_RTM_TRUE, 1, shot, &h_wav, SEIS_IN_WAVELET, &h_vel, SEIS_IN_VEL, &h_rec,
                   SEIS_IN_GATHER, &h_img, SEIS_OUT_IMAGE);
}

int seis_fd_illum(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_wav,
                  const float *h_vel, float *h_ss) {
  return seis_fd_illum_batch(ctx, 1, shot, &h_wav, &h_vel, &h_ss);
}

int seis_fd_illum_batch(seis_fd_ctx *ctx, int nshot, const seis_shot_desc *shots,
                        const float *const *h_wav, const float *const *h_vel,
                        float *const *h_ss) {
  // the receivers play no part: a shot without them gets surface rows
  if (!shots || nshot < 1) return begin(ctx) ? SEIS_ERR_ARG : fail(ctx, SEIS_ERR_ARG, "no shots");
  std::vector<seis_shot_desc> d(shots, shots + nshot);
  std::vector<std::vector<int>> zero((size_t)nshot);
  for (int s = 0; s < nshot; s++)
    if (!d[s].gz) {
      zero[s].assign((size_t)std::max(d[s].nx, 0), 0);
      d[s].gz = zero[s].data();
    }
  return run_batch(ctx, OP_ILLUM, nshot, d.data(), h_wav, SEIS_IN_WAVELET, h_vel, SEIS_IN_VEL,
                   nullptr, -1, h_ss, SEIS_OUT_IMAGE);
}

int seis_fd_rtm(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_wav,
                const float *h_vel, const float *h_rec, float *h_img) {
  return run_batch(ctx, OP_RTM, 1, shot, &h_wav, SEIS_IN_WAVELET, &h_vel, SEIS_IN_VEL, &h_rec,
                   SEIS_IN_GATHER, &h_img, SEIS_OUT_IMAGE);
}

int seis_fd_born_adjoint(seis_fd_ctx *ctx, const seis_shot_desc *shot, const float *h_wav,
                         const float *h_vel, const float *h_rec, float *h_img) {
  return run_batch(ctx, OP_BORN_ADJ, 1, shot, &h_wav, SEIS_IN_WAVELET, &h_vel, SEIS_IN_VEL, &h_rec,
                   SEIS_IN_GATHER, &h_img, SEIS_OUT_IMAGE);
}

int seis_fd_modeling_batch(seis_fd_ctx *ctx, int nshot, const seis_shot_desc *shots,
                           const float *const *h_wav, const float *const *h_vel,
                           float *const *h_rec) {
  return run_batch(ctx, OP_MODEL, nshot, shots, h_wav, SEIS_IN_WAVELET, h_vel, SEIS_IN_VEL,
                   nullptr, -1, h_rec, SEIS_OUT_GATHER);
}

int seis_fd_born_batch(seis_fd_ctx *ctx, int nshot, const seis_shot_desc *shots,
                       const float *const *h_wav, const float *const *h_vel,
                       const float *const *h_dv, float *const *h_rec) {
  return run_batch(ctx, OP_BORN, nshot, shots, h_wav, SEIS_IN_WAVELET, h_vel, SEIS_IN_VEL, h_dv,
                   SEIS_IN_DV, h_rec, SEIS_OUT_GATHER);
}

int seis_fd_rtm_batch(seis_fd_ctx *ctx, int nshot, const seis_shot_desc *shots,
                      const float *const *h_wav, const float *const *h_vel,
                      const float *const *h_rec, float *const *h_img) {
  return run_batch(ctx, OP_RTM, nshot, shots, h_wav, SEIS_IN_WAVELET, h_vel, SEIS_IN_VEL, h_rec,
                   SEIS_IN_GATHER, h_img, SEIS_OUT_IMAGE);
}

// ------------------------------------------------------------ vector ops
int seis_fd_vec_dot(seis_fd_ctx *ctx, const float *d_a, const float *d_b, size_t n,
                    double *h_out) {
  int rc = begin(ctx);
  if (rc) return rc;
  if (!d_a || !d_b || !h_out) return fail(ctx, SEIS_ERR_ARG, "null pointer");
  CK(launch_dot(d_a, d_b, n, ctx->d_partial, ctx->d_scalar, 0, ctx->stream));
  ctx->launches += 2;
  CK(cudaMemcpyAsync(h_out, ctx->d_scalar, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  return sync(ctx);
}

int seis_fd_vec_axpby(seis_fd_ctx *ctx, float *d_y, const float *d_x, double a, double b,
                      size_t n) {
  int rc = begin(ctx);
  if (rc) return rc;
  if (!d_y || !d_x) return fail(ctx, SEIS_ERR_ARG, "null pointer");
  CK(launch_axpby(d_y, d_x, a, b, n, ctx->stream));
  ctx->launches++;
  return sync(ctx);
}

}  // extern "C"

// ------------------------------------------------------------------ LSRTM
struct seis_fd_lsrtm {
  seis_fd_ctx *ctx = nullptr;
  int nx = 0, nz = 0, nshot = 0, nt = 0;
  std::vector<seis_shot_desc> shots;
  std::vector<std::vector<int>> gz;
  // model column of every sub-grid column of every shot (non-decreasing)
  std::vector<std::vector<int>> cmap;
  std::vector<size_t> cmap_off, range_off;
  std::vector<int> g0, gcount;  // model columns g0 .. g0 + gcount - 1 a shot touches
  int *d_cmap = nullptr;
  int2 *d_ranges = nullptr;
  seis_fd_plan born{nullptr}, adj{nullptr};
  std::vector<void *> allocs;
  float *m = nullptr, *p = nullptr, *s = nullptr;  // model-space vectors [nx][nz]
  float *dobs = nullptr, *r = nullptr;             // data space, per shot [nt][nx_s]
  std::vector<size_t> doff;                        // offset of shot s in data space
  size_t ndata = 0;
  double *sc = nullptr;  // FP64 scalars: 0 gamma, 1 |q|^2, 2 alpha, 3 gamma_new, 4 beta
  double *rr = nullptr;  // |r|^2 per iteration
  int rr_cap = 0;
  // shot groups (group > 0): the plans of `group` shots at a time are built
  // for each operator application and freed after it; the background and
  // wavelet stay on the device, q = L p in its own data-space buffer
  int group = 0;
  seis_lsrtm_opts opts{};
  float *d_v0 = nullptr, *d_wav = nullptr, *q = nullptr, *stage = nullptr;
  int64_t group_bytes = 0;  // largest device memory of one group's plan
  bool ready = false;    // reset done
  int64_t device_bytes = 0;
  ~seis_fd_lsrtm() {
    if (born.p) delete born.p;
    if (adj.p) delete adj.p;
    for (void *q : allocs) cudaFree(q);
  }
  template <class T>
  int alloc(T **out, size_t n) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(ctx, e == cudaErrorMemoryAllocation ? SEIS_ERR_NOMEM : SEIS_ERR_CUDA,
                  "cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
    }
    allocs.push_back(q);
    device_bytes += (int64_t)(std::max<size_t>(n, 1) * sizeof(T));
    *out = static_cast<T *>(q);
    e = cudaMemsetAsync(q, 0, std::max<size_t>(n, 1) * sizeof(T), ctx->stream);
    return e == cudaSuccess ? SEIS_OK : fail(ctx, SEIS_ERR_CUDA, "cudaMemset failed");
  }
};

namespace {

// The tile shape of a solver plan whose velocity and wavelet are loaded: the
// fixed shape of the options, or the autotuner's (10 timed steps per shape).
int lsrtm_shape(seis_fd_lsrtm &L, Plan &p) {
  if (L.opts.tile_shape > 0) return apply_shape(p, L.opts.tile_shape - 1);
  return autotune(p, 10, false, nullptr, nullptr);
}

// s = L^T r: adjoint plan over the residuals, per-shot images scattered into
// the global grid.
// The plan of shots k0 .. k1-1 of a grouped solver: velocity sub-grids and
// wavelet from the device copies; an adjoint plan reads the residual.
int lsrtm_group_plan(seis_fd_lsrtm &L, int op, int k0, int k1, Plan **out) {
  seis_fd_ctx *ctx = L.ctx;
  Plan *p = nullptr;
  int rc = plan_create(ctx, op, k1 - k0, L.shots.data() + k0, &p);
  if (rc) return rc;
  p->exact = L.opts.exact != 0;
  seis_fd_plan h{p};
  if (op == OP_BORN_ADJ) {
    rc = seis_fd_plan_set_snapshots(&h, L.opts.snap_every, L.opts.snap_dtype);
    if (!rc && L.opts.checkpoint_every > 0)
      rc = seis_fd_plan_set_checkpoints(&h, L.opts.checkpoint_every);
  }
  for (int j = 0; j < k1 - k0 && !rc; j++) {
    const int k = k0 + j;
    ShotDev &g = p->sd[j];
    cudaError_t e = launch_gather_cols(L.d_v0, L.nz, L.d_cmap + L.cmap_off[k], g.nx, p->d_stage,
                                       ctx->stream);
    if (e == cudaSuccess)
      e = launch_pad(p->d_stage, g.nx, g.nz, g.pml, g.LDZ, true, const_cast<float *>(g.vel),
                     ctx->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(const_cast<float *>(g.wav), L.d_wav, sizeof(float) * g.NT,
                          cudaMemcpyDeviceToDevice, ctx->stream);
    if (e != cudaSuccess) rc = fail(ctx, SEIS_ERR_CUDA, "group plan: %s", cudaGetErrorString(e));
    ctx->launches += 2;
    if (op == OP_BORN_ADJ) g.rec = L.r + L.doff[k];
  }
  if (!rc) rc = lsrtm_shape(L, *p);
  if (!rc && op == OP_BORN_ADJ) {
    cudaError_t e = cudaMemcpyAsync(p->d_sd, p->sd.data(), sizeof(ShotDev) * p->nshot,
                                    cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) rc = fail(ctx, SEIS_ERR_CUDA, "group plan: %s", cudaGetErrorString(e));
  }
  if (rc) {
    delete p;
    return rc;
  }
  *out = p;
  return SEIS_OK;
}

// Free a group's plan once the stream has finished with it.
int lsrtm_group_done(seis_fd_lsrtm &L, Plan *p) {
  cudaError_t e = cudaStreamSynchronize(L.ctx->stream);
  L.group_bytes = std::max(L.group_bytes, p->device_bytes);
  delete p;
  return e == cudaSuccess ? SEIS_OK : fail(L.ctx, SEIS_ERR_CUDA, "%s", cudaGetErrorString(e));
}

// s = L^T r: the adjoint plan's images scattered into the global grid, shot
// after shot.
int lsrtm_adjoint(seis_fd_lsrtm &L) {
  seis_fd_ctx *ctx = L.ctx;
  size_t nm = (size_t)L.nx * L.nz;
  if (L.group == 0) {
    int rc = plan_run(*L.adj.p);
    if (rc) return rc;
  }
  CK(cudaMemsetAsync(L.s, 0, sizeof(float) * nm, ctx->stream));
  const int G = L.group > 0 ? L.group : L.nshot;
  for (int k0 = 0; k0 < L.nshot; k0 += G) {
    const int k1 = std::min(k0 + G, L.nshot);
    Plan *pa = L.adj.p;
    if (L.group > 0) {
      int rc = lsrtm_group_plan(L, OP_BORN_ADJ, k0, k1, &pa);
      if (!rc) rc = enqueue_operator(*pa);
      if (rc) {
        if (pa) lsrtm_group_done(L, pa);
        return rc;
      }
    }
    for (int k = k0; k < k1; k++) {
      const ShotDev &g = pa->sd[k - (L.group > 0 ? k0 : 0)];
      CK(launch_scatter_cols(L.s, L.nz, L.d_ranges + L.range_off[k], L.g0[k], L.gcount[k], g.img,
                             ctx->stream));
      ctx->launches++;
    }
    if (L.group > 0) {
      int rc = lsrtm_group_done(L, pa);
      if (rc) return rc;
    }
  }
  return SEIS_OK;
}

// q = L p into the Born plan's gathers (grouped: into L.q): each shot's
// perturbation is its sub-grid of p (column map), padded into the plan.
int lsrtm_forward(seis_fd_lsrtm &L) {
  seis_fd_ctx *ctx = L.ctx;
  const int G = L.group > 0 ? L.group : L.nshot;
  for (int k0 = 0; k0 < L.nshot; k0 += G) {
    const int k1 = std::min(k0 + G, L.nshot);
    Plan *pb = L.born.p;
    if (L.group > 0) {
      int rc = lsrtm_group_plan(L, OP_BORN, k0, k1, &pb);
      if (rc) return rc;
    }
    for (int k = k0; k < k1; k++) {
      const ShotDev &g = pb->sd[k - (L.group > 0 ? k0 : 0)];
      CK(launch_gather_cols(L.p, L.nz, L.d_cmap + L.cmap_off[k], g.nx, pb->d_stage, ctx->stream));
      CK(launch_pad(pb->d_stage, g.nx, g.nz, g.pml, g.LDZ, false, const_cast<float *>(g.dv),
                    ctx->stream));
      ctx->launches += 2;
    }
    if (L.group == 0) return plan_run(*pb);
    int rc = enqueue_operator(*pb);
    for (int k = k0; k < k1 && !rc; k++) {
      const size_t n = (size_t)L.shots[k].nx * L.nt;
      cudaError_t e = cudaMemcpyAsync(L.q + L.doff[k], pb->sd[k - k0].rec, sizeof(float) * n,
                                      cudaMemcpyDeviceToDevice, ctx->stream);
      if (e != cudaSuccess) rc = fail(ctx, SEIS_ERR_CUDA, "%s", cudaGetErrorString(e));
    }
    int rc2 = lsrtm_group_done(L, pb);
    if (rc) return rc;
    if (rc2) return rc2;
  }
  return SEIS_OK;
}

// q = L p of shot k in data space ([nt][nx_s])
const float *lsrtm_q(const seis_fd_lsrtm &L, int k) {
  return L.group > 0 ? L.q + L.doff[k] : L.born.p->sd[k].rec;
}

// out = sum over shots of <a_s, b_s> in data space; a from q = L p when
// `q_left`, else the residual; b likewise.
int data_dot(seis_fd_lsrtm &L, bool q_left, bool q_right, double *out) {
  seis_fd_ctx *ctx = L.ctx;
  for (int k = 0; k < L.nshot; k++) {
    const float *q = lsrtm_q(L, k), *r = L.r + L.doff[k];
    size_t n = (size_t)L.shots[k].nx * L.nt;
    CK(launch_dot(q_left ? q : r, q_right ? q : r, n, ctx->d_partial, out, k > 0, ctx->stream));
    ctx->launches += 2;
  }
  return SEIS_OK;
}

}  // namespace

extern "C" {

int seis_fd_lsrtm_create_mapped(seis_fd_ctx *ctx, int nx, int nz, int nshot,
                                const seis_shot_desc *shots, const int *colmap,
                                const seis_lsrtm_opts *opts, seis_fd_lsrtm **out) {
  int rc = begin(ctx);
  if (rc) return rc;
  if (!out || !shots || !colmap || nshot < 1 || nx < 1 || nz < 1)
    return fail(ctx, SEIS_ERR_ARG, "lsrtm: bad arguments");
  *out = nullptr;
  size_t off = 0;
  for (int k = 0; k < nshot; k++) {
    if (shots[k].nz != nz)
      return fail(ctx, SEIS_ERR_ARG, "lsrtm: shot %d has nz %d, the model %d", k, shots[k].nz, nz);
    for (int ix = 0; ix < shots[k].nx; ix++) {
      const int c = colmap[off + ix];
      if (c < 0 || c >= nx || (ix > 0 && c < colmap[off + ix - 1]))
        return fail(ctx, SEIS_ERR_ARG,
                    "lsrtm: shot %d column map must be non-decreasing within [0, %d)", k, nx);
    }
    off += shots[k].nx;
  }
  seis_lsrtm_opts o{1, SEIS_SNAP_F16, 0, 0, 0, 0};
  if (opts) o = *opts;
  seis_fd_lsrtm *L = new (std::nothrow) seis_fd_lsrtm();
  if (!L) return fail(ctx, SEIS_ERR_NOMEM, "host allocation failed");
  L->ctx = ctx;
  L->nx = nx; L->nz = nz; L->nshot = nshot; L->nt = shots[0].nt;
  L->shots.assign(shots, shots + nshot);
  L->gz.resize(nshot);
  for (int k = 0; k < nshot; k++) {  // group plans are built after this call returns
    L->gz[k].assign(shots[k].gz, shots[k].gz + shots[k].nx);
    L->shots[k].gz = L->gz[k].data();
  }
  std::vector<int2> ranges;
  off = 0;
  for (int k = 0; k < nshot; k++) {
    const int n = shots[k].nx;
    L->cmap.emplace_back(colmap + off, colmap + off + n);
    L->cmap_off.push_back(off);
    off += n;
    const std::vector<int> &m = L->cmap.back();
    L->g0.push_back(m[0]);
    L->gcount.push_back(m[n - 1] - m[0] + 1);
    L->range_off.push_back(ranges.size());
    const size_t base = ranges.size();
    ranges.resize(base + (size_t)L->gcount.back(), make_int2(0, -1));
    for (int ix = 0; ix < n; ix++) {
      int2 &r = ranges[base + (m[ix] - m[0])];
      if (r.y < r.x) r.x = ix;
      r.y = ix;
    }
  }
  Plan *pb = nullptr, *pa = nullptr;
  L->opts = o;
  L->group = (o.group_shots > 0 && o.group_shots < nshot) ? o.group_shots : 0;
  if (o.tile_shape < 0 || o.tile_shape > NSHAPES)
    rc = fail(ctx, SEIS_ERR_ARG, "lsrtm: tile shape %d", o.tile_shape);
  if (o.snap_every < 1 || (o.checkpoint_every > 0 && o.checkpoint_every % o.snap_every != 0))
    rc = fail(ctx, SEIS_ERR_ARG, "lsrtm: snapshot interval %d, checkpoint interval %d",
              o.snap_every, o.checkpoint_every);
  if (!rc && L->group == 0) {
    rc = plan_create(ctx, OP_BORN, nshot, shots, &pb);
    if (!rc) rc = plan_create(ctx, OP_BORN_ADJ, nshot, shots, &pa);
    L->born.p = pb;
    L->adj.p = pa;
  }
  if (!rc && L->group == 0) {
    pb->exact = o.exact != 0;
    pa->exact = o.exact != 0;
    seis_fd_plan h{pa};
    rc = seis_fd_plan_set_snapshots(&h, o.snap_every, o.snap_dtype);
    if (!rc && o.checkpoint_every > 0) rc = seis_fd_plan_set_checkpoints(&h, o.checkpoint_every);
  }
  size_t nm = (size_t)nx * nz;
  if (!rc) rc = L->alloc(&L->m, nm);
  if (!rc) rc = L->alloc(&L->p, nm);
  if (!rc) rc = L->alloc(&L->s, nm);
  for (int k = 0; k < nshot; k++) {
    L->doff.push_back(L->ndata);
    L->ndata += (size_t)shots[k].nx * L->nt;
  }
  if (!rc) rc = L->alloc(&L->dobs, L->ndata);
  if (!rc) rc = L->alloc(&L->r, L->ndata);
  if (!rc) rc = L->alloc(&L->sc, 8);
  if (!rc) {
    L->rr_cap = 4096;
    rc = L->alloc(&L->rr, (size_t)L->rr_cap);
  }
  if (!rc) rc = L->alloc(&L->d_cmap, off);
  if (!rc) rc = L->alloc(&L->d_ranges, ranges.size());
  if (!rc && L->group > 0) {
    size_t st = 0;
    for (int k = 0; k < nshot; k++) st = std::max(st, (size_t)shots[k].nx * L->nt);
    rc = L->alloc(&L->d_v0, nm);
    if (!rc) rc = L->alloc(&L->d_wav, (size_t)(L->nt + shots[0].ndel));
    if (!rc) rc = L->alloc(&L->q, L->ndata);
    if (!rc) rc = L->alloc(&L->stage, st);
  }
  if (!rc) {
    // the adjoint plan reads its receiver data straight from the residual
    cudaError_t e = cudaSuccess;
    if (pa) {
      for (int k = 0; k < nshot; k++) pa->sd[k].rec = L->r + L->doff[k];
      e = cudaMemcpyAsync(pa->d_sd, pa->sd.data(), sizeof(ShotDev) * nshot,
                          cudaMemcpyHostToDevice, ctx->stream);
    }
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(L->d_cmap, colmap, sizeof(int) * off, cudaMemcpyHostToDevice,
                          ctx->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(L->d_ranges, ranges.data(), sizeof(int2) * ranges.size(),
                          cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) rc = fail(ctx, SEIS_ERR_CUDA, "lsrtm setup: %s", cudaGetErrorString(e));
  }
  if (rc) {
    delete L;
    return rc;
  }
  *out = L;
  return SEIS_OK;
}

int seis_fd_lsrtm_create(seis_fd_ctx *ctx, int nx, int nz, int nshot, const seis_shot_desc *shots,
                         const int *x0, const seis_lsrtm_opts *opts, seis_fd_lsrtm **out) {
  int rc = begin(ctx);
  if (rc) return rc;
  if (!out || !shots || !x0 || nshot < 1 || nx < 1 || nz < 1)
    return fail(ctx, SEIS_ERR_ARG, "lsrtm: bad arguments");
  std::vector<int> map;
  for (int k = 0; k < nshot; k++) {
    if (x0[k] < 0 || x0[k] + shots[k].nx > nx)
      return fail(ctx, SEIS_ERR_ARG, "lsrtm: shot %d aperture [%d, %d) outside %d columns", k,
                  x0[k], x0[k] + shots[k].nx, nx);
    for (int ix = 0; ix < shots[k].nx; ix++) map.push_back(x0[k] + ix);
  }
  return seis_fd_lsrtm_create_mapped(ctx, nx, nz, nshot, shots, map.data(), opts, out);
}

int seis_fd_lsrtm_destroy(seis_fd_lsrtm *L) {
  if (!L) return SEIS_OK;
  cudaSetDevice(L->ctx->device);
  cudaStreamSynchronize(L->ctx->stream);
  delete L;
  return SEIS_OK;
}

int seis_fd_lsrtm_set_background(seis_fd_lsrtm *L, const float *h_v0, const float *h_wav) {
  if (!L) return SEIS_ERR_ARG;
  int rc = begin(L->ctx);
  if (rc) return rc;
  if (!h_v0 || !h_wav) return fail(L->ctx, SEIS_ERR_ARG, "null array");
  if (L->group > 0) {  // group plans take their sub-grids from the device copy
    seis_fd_ctx *ctx = L->ctx;
    const int NT = L->nt + L->shots[0].ndel;
    CK(cudaMemcpyAsync(L->d_v0, h_v0, sizeof(float) * L->nx * L->nz, cudaMemcpyHostToDevice,
                       L->ctx->stream));
    CK(cudaMemcpyAsync(L->d_wav, h_wav, sizeof(float) * NT, cudaMemcpyHostToDevice,
                       L->ctx->stream));
    L->ready = false;
    return sync(L->ctx);
  }
  std::vector<float> sub;
  for (int k = 0; k < L->nshot && !rc; k++) {
    const std::vector<int> &m = L->cmap[k];
    sub.resize(m.size() * (size_t)L->nz);
    for (size_t ix = 0; ix < m.size(); ix++)
      std::memcpy(sub.data() + ix * L->nz, h_v0 + (size_t)m[ix] * L->nz, sizeof(float) * L->nz);
    rc = plan_input(&L->born, k, SEIS_IN_VEL, sub.data(), false);
    if (!rc) rc = plan_input(&L->born, k, SEIS_IN_WAVELET, h_wav, false);
    if (!rc) rc = plan_input(&L->adj, k, SEIS_IN_VEL, sub.data(), false);
    if (!rc) rc = plan_input(&L->adj, k, SEIS_IN_WAVELET, h_wav, false);
    if (!rc) rc = sync(L->ctx);  // the host sub-grid is reused by the next shot
  }
  if (!rc && !L->adj.p->snaps_ready) rc = lsrtm_shape(*L, *L->born.p);
  if (!rc && !L->adj.p->snaps_ready) rc = lsrtm_shape(*L, *L->adj.p);
  L->ready = false;
  return rc ? rc : sync(L->ctx);
}

int seis_fd_lsrtm_set_data(seis_fd_lsrtm *L, int shot, const float *h_d) {
  if (!L) return SEIS_ERR_ARG;
  seis_fd_ctx *ctx = L->ctx;
  int rc = begin(ctx);
  if (rc) return rc;
  if (shot < 0 || shot >= L->nshot || !h_d) return fail(ctx, SEIS_ERR_ARG, "shot %d", shot);
  const int nxs = L->shots[shot].nx;
  float *stage = L->group > 0 ? L->stage : L->born.p->d_stage;
  CK(cudaMemcpyAsync(stage, h_d, sizeof(float) * nxs * L->nt, cudaMemcpyHostToDevice,
                     ctx->stream));
  CK(launch_transpose(stage, nxs, L->nt, L->dobs + L->doff[shot], ctx->stream));
  ctx->launches++;
  L->ready = false;
  return sync(ctx);
}

// ---- the phases of a CGLS iteration.  Each leaves this solver's partial
// sums in the caller's device buffers; the next phase reads them summed (over
// the ranks of a solver spread across devices, or as they are on one).

// m = 0, r = d, s = L^T r, rr = |r|^2
int seis_fd_lsrtm_phase_reset(seis_fd_lsrtm *L, float *d_s, double *d_rr) {
  if (!L || !d_s || !d_rr) return SEIS_ERR_ARG;
  seis_fd_ctx *ctx = L->ctx;
  int rc = begin(ctx);
  if (rc) return rc;
  const size_t nm = (size_t)L->nx * L->nz;
  CK(cudaMemsetAsync(L->m, 0, sizeof(float) * nm, ctx->stream));
  CK(cudaMemcpyAsync(L->r, L->dobs, sizeof(float) * L->ndata, cudaMemcpyDeviceToDevice,
                     ctx->stream));
  rc = data_dot(*L, false, false, d_rr);
  if (!rc) rc = lsrtm_adjoint(*L);
  if (rc) return rc;
  if (d_s != L->s)
    CK(cudaMemcpyAsync(d_s, L->s, sizeof(float) * nm, cudaMemcpyDeviceToDevice, ctx->stream));
  L->ready = true;
  return SEIS_OK;
}

// q = L p, qq = |q|^2
int seis_fd_lsrtm_phase_forward(seis_fd_lsrtm *L, double *d_qq) {
  if (!L || !d_qq) return SEIS_ERR_ARG;
  int rc = begin(L->ctx);
  if (rc) return rc;
  if (!L->ready) return fail(L->ctx, SEIS_ERR_STATE, "lsrtm: reset first");
  rc = lsrtm_forward(*L);
  return rc ? rc : data_dot(*L, true, true, d_qq);
}

// alpha = gamma / qq, m += alpha p, r -= alpha q, rr = |r|^2, s = L^T r
int seis_fd_lsrtm_phase_update(seis_fd_lsrtm *L, const double *d_qq, float *d_s, double *d_rr) {
  if (!L || !d_qq || !d_s || !d_rr) return SEIS_ERR_ARG;
  seis_fd_ctx *ctx = L->ctx;
  int rc = begin(ctx);
  if (rc) return rc;
  if (!L->ready) return fail(ctx, SEIS_ERR_STATE, "lsrtm: reset first");
  const size_t nm = (size_t)L->nx * L->nz;
  double *gamma = L->sc + 0, *alpha = L->sc + 2;
  CK(launch_ratio(gamma, d_qq, alpha, ctx->stream));
  CK(launch_axpby_dev(L->m, L->p, alpha, 1.0, nullptr, 1.0, nm, ctx->stream));
  for (int k = 0; k < L->nshot; k++)
    CK(launch_axpby_dev(L->r + L->doff[k], lsrtm_q(*L, k), alpha, -1.0, nullptr, 1.0,
                        (size_t)L->shots[k].nx * L->nt, ctx->stream));
  ctx->launches += 2 + L->nshot;
  rc = data_dot(*L, false, false, d_rr);
  if (!rc) rc = lsrtm_adjoint(*L);
  if (rc) return rc;
  if (d_s != L->s)
    CK(cudaMemcpyAsync(d_s, L->s, sizeof(float) * nm, cudaMemcpyDeviceToDevice, ctx->stream));
  return SEIS_OK;
}

// s = the summed image, gamma' = |s|^2; first: gamma = gamma', p = s; else
// beta = gamma' / gamma, gamma = gamma', p = s + beta p
int seis_fd_lsrtm_phase_direction(seis_fd_lsrtm *L, const float *d_s, int first) {
  if (!L || !d_s) return SEIS_ERR_ARG;
  seis_fd_ctx *ctx = L->ctx;
  int rc = begin(ctx);
  if (rc) return rc;
  if (!L->ready) return fail(ctx, SEIS_ERR_STATE, "lsrtm: reset first");
  const size_t nm = (size_t)L->nx * L->nz;
  double *gamma = L->sc + 0, *gnew = L->sc + 3, *beta = L->sc + 4;
  if (d_s != L->s)
    CK(cudaMemcpyAsync(L->s, d_s, sizeof(float) * nm, cudaMemcpyDeviceToDevice, ctx->stream));
  CK(launch_dot(L->s, L->s, nm, ctx->d_partial, gnew, 0, ctx->stream));
  ctx->launches += 2;
  if (first) {
    CK(cudaMemcpyAsync(gamma, gnew, sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(L->p, L->s, sizeof(float) * nm, cudaMemcpyDeviceToDevice, ctx->stream));
    return SEIS_OK;
  }
  CK(launch_ratio(gnew, gamma, beta, ctx->stream));
  CK(cudaMemcpyAsync(gamma, gnew, sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  CK(launch_axpby_dev(L->p, L->s, nullptr, 1.0, beta, 1.0, nm, ctx->stream));
  ctx->launches += 2;
  return SEIS_OK;
}

int seis_fd_lsrtm_reset(seis_fd_lsrtm *L, double *h_rr) {
  if (!L) return SEIS_ERR_ARG;
  seis_fd_ctx *ctx = L->ctx;
  int rc = seis_fd_lsrtm_phase_reset(L, L->s, L->rr);
  if (!rc) rc = seis_fd_lsrtm_phase_direction(L, L->s, 1);
  if (rc) return rc;
  if (h_rr)
    CK(cudaMemcpyAsync(h_rr, L->rr, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  return sync(ctx);
}

int seis_fd_lsrtm_iterate(seis_fd_lsrtm *L, int niter, double *h_rr) {
  if (!L) return SEIS_ERR_ARG;
  seis_fd_ctx *ctx = L->ctx;
  int rc = begin(ctx);
  if (rc) return rc;
  if (!L->ready) return fail(ctx, SEIS_ERR_STATE, "lsrtm: call seis_fd_lsrtm_reset first");
  if (niter < 1 || niter > L->rr_cap) return fail(ctx, SEIS_ERR_ARG, "niter=%d", niter);
  double *qq = L->sc + 1;
  for (int it = 0; it < niter && !rc; it++) {
    rc = seis_fd_lsrtm_phase_forward(L, qq);
    if (!rc) rc = seis_fd_lsrtm_phase_update(L, qq, L->s, L->rr + it);
    if (!rc) rc = seis_fd_lsrtm_phase_direction(L, L->s, 0);
  }
  if (rc) return rc;
  if (h_rr)
    CK(cudaMemcpyAsync(h_rr, L->rr, sizeof(double) * niter, cudaMemcpyDeviceToHost, ctx->stream));
  return sync(ctx);
}

int seis_fd_lsrtm_model(seis_fd_lsrtm *L, float *h_m) {
  if (!L || !h_m) return SEIS_ERR_ARG;
  seis_fd_ctx *ctx = L->ctx;
  int rc = begin(ctx);
  if (rc) return rc;
  CK(cudaMemcpyAsync(h_m, L->m, sizeof(float) * L->nx * L->nz, cudaMemcpyDeviceToHost,
                     ctx->stream));
  return sync(ctx);
}

int64_t seis_fd_lsrtm_cell_updates(const seis_fd_lsrtm *L) {
  if (!L) return 0;
  int64_t c = 0;
  // Born (two fields), the adjoint's reverse pass, with checkpoints the
  // recomputed source field, with shot groups the source pass of every run
  const int64_t ck = L->opts.checkpoint_every > 0 ? 1 : 0, gr = L->group > 0 ? 1 : 0;
  for (const seis_shot_desc &d : L->shots) {
    const int64_t NX = d.nx + 2 * d.pml, NZ = d.nz + 2 * d.pml, NT = d.nt + d.ndel;
    c += NX * NZ * (2 * NT + NT + 1 + ck * NT + gr * NT);
  }
  return c;
}

int64_t seis_fd_lsrtm_device_bytes(const seis_fd_lsrtm *L) {
  if (!L) return 0;
  if (L->group > 0) return L->device_bytes + L->group_bytes;  // one group's plan at a time
  return L->device_bytes + L->born.p->device_bytes + L->adj.p->device_bytes;
}

}  // extern "C"
