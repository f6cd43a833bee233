// The shot driver (seis_driver.h): the reference's parameter file, coordinate
// file and gather files, driving batched device operators.  It replaces the
// MPI driver class Inversion (src/lsrtm/inversion.cpp): the master/worker shot
// farm (masterRun, :753-807) becomes batches of shots on one device, and each
// worker's per-shot pipeline (aperture, receiver rows, operator, trace
// reorder, direct mute, image scatter) is kept step for step.  Written against
// the public ABI only (seis_fd.h, seis_geom.h).
#include "seis_driver.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <new>
#include <string>
#include <vector>

#include "seis_geom.h"

namespace {

int put_err(char *err, size_t len, int rc, const char *fmt, ...) {
  if (err && len) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, len, fmt, ap);
    va_end(ap);
  }
  return rc;
}

// ---------------------------------------------------------- parameter file
// ParserFromFile (src/util/parser.cpp:15-175): the first line whose
// comment-stripped text contains "key " followed by a token of the value's
// character class; the token runs to the next white space.
enum Kind { K_INT, K_FLOAT, K_STRING };

bool find_value(const std::vector<std::string> &lines, const std::string &key, Kind kind,
                std::string *tok, bool *seen) {
  static const char *cls[3] = {"+-0123456789", "+-.0123456789",
                               "/qwertyuiopasdfghjklzxcvbnmQWERTYUIOPASDFGHJKLZXCVBNM"};
  const std::string k = key + " ";
  for (std::string line : lines) {
    const size_t c = line.find('!');
    if (c != std::string::npos) line.erase(c);
    const size_t at = line.find(k);
    if (at == std::string::npos) continue;
    *seen = true;
    line = line.substr(at + k.size());
    const size_t i0 = line.find_first_of(cls[kind]);
    if (i0 == std::string::npos) continue;
    size_t i = i0;
    while (i < line.size() && !std::isspace((unsigned char)line[i])) i++;
    *tok = line.substr(i0, i - i0);
    return true;
  }
  return false;
}

struct ParamReader {
  std::vector<std::string> lines;
  char *err;
  size_t err_len;
  int rc = 0;

  template <class T>
  void get(const char *key, T *val, T def, bool opt);
};

template <>
void ParamReader::get<int>(const char *key, int *val, int def, bool opt) {
  if (rc) return;
  std::string tok;
  bool seen = false;
  if (find_value(lines, key, K_INT, &tok, &seen)) {
    try {
      *val = std::stoi(tok);
    } catch (...) {
      rc = put_err(err, err_len, SEIS_ERR_ARG, "parameter %s: bad value '%s'", key, tok.c_str());
    }
  } else if (opt) {
    *val = def;
  } else {
    rc = put_err(err, err_len, SEIS_ERR_ARG, "parameter %s: %s", key,
                 seen ? "value missing" : "key not found");
  }
}

template <>
void ParamReader::get<float>(const char *key, float *val, float def, bool opt) {
  if (rc) return;
  std::string tok;
  bool seen = false;
  if (find_value(lines, key, K_FLOAT, &tok, &seen)) {
    try {
      *val = std::stof(tok);
    } catch (...) {
      rc = put_err(err, err_len, SEIS_ERR_ARG, "parameter %s: bad value '%s'", key, tok.c_str());
    }
  } else if (opt) {
    *val = def;
  } else {
    rc = put_err(err, err_len, SEIS_ERR_ARG, "parameter %s: %s", key,
                 seen ? "value missing" : "key not found");
  }
}

void get_string(ParamReader &r, const char *key, char (&val)[256], bool opt) {
  if (r.rc) return;
  std::string tok;
  bool seen = false;
  if (find_value(r.lines, key, K_STRING, &tok, &seen)) {
    if (tok.size() > 255) {
      r.rc = put_err(r.err, r.err_len, SEIS_ERR_ARG, "parameter %s: longer than 255", key);
      return;
    }
    std::snprintf(val, sizeof val, "%s", tok.c_str());
  } else if (opt) {
    val[0] = '\0';
  } else {
    r.rc = put_err(r.err, r.err_len, SEIS_ERR_ARG, "parameter %s: %s", key,
                   seen ? "value missing" : "key not found");
  }
}

// ------------------------------------------------------- coordinate file
// Coords (src/util/coord.cpp): each line read into a 256-byte buffer and
// scanned field by field, a field that does not scan keeping the previous
// line's value; reading continues until end of file, so the empty read after a
// trailing newline repeats the last trace, which the receiver count removes.
struct CoordLine {
  float hs, vs, hg, vg;
};

bool read_lines(const char *file, std::vector<std::string> *out) {
  std::ifstream in(file);
  if (!in) return false;
  std::string line;
  while (std::getline(in, line)) out->push_back(line.substr(0, 255));
  // the reference's loop runs once more after the last newline-terminated line
  in.clear();
  in.seekg(-1, std::ios::end);
  char last = 0;
  if (in.get(last) && last == '\n') out->push_back(std::string());
  return true;
}

void scan(const std::string &l, CoordLine *c) {
  const char *b = l.c_str();
  std::sscanf(b, "%f", &c->hs);
  std::sscanf(b, "%*s%f", &c->vs);
  std::sscanf(b, "%*s%*s%f", &c->hg);
  std::sscanf(b, "%*s%*s%*s%f", &c->vg);
}

}  // namespace

extern "C" {

int seis_params_read(const char *file, seis_params *out, char *err, size_t err_len) {
  if (!file || !out) return put_err(err, err_len, SEIS_ERR_ARG, "null argument");
  ParamReader r;
  r.err = err;
  r.err_len = err_len;
  {
    std::ifstream in(file);
    if (!in) return put_err(err, err_len, SEIS_ERR_ARG, "cannot open %s", file);
    std::string line;
    while (std::getline(in, line)) r.lines.push_back(line);
  }
  seis_params p;
  std::memset(&p, 0, sizeof p);
  // order and defaults of readParamFile (inversion.cpp:41-80) / paramLSRTM
  r.get<int>("nthread", &p.nthread, 1, true);
  r.get<int>("ns", &p.ns, 0, false);
  r.get<int>("ngmax", &p.ngmax, 0, false);
  r.get<int>("nx", &p.nx, 0, false);
  r.get<int>("nz", &p.nz, 0, false);
  r.get<int>("nt", &p.nt, 0, false);
  r.get<int>("npml", &p.npml, 10, true);
  r.get<int>("delay", &p.delay, 0, true);
  r.get<int>("delaycal", &p.delaycal, 0, true);
  r.get<int>("mask", &p.mask, 0, true);
  r.get<int>("maxiter", &p.maxiter, 30, true);
  r.get<int>("lpad", &p.lpad, 0, true);
  r.get<int>("rpad", &p.rpad, 0, true);
  r.get<int>("planeTag", &p.planeTag, 0, true);
  r.get<int>("sbegin", &p.sbegin, 0, false);
  r.get<int>("send", &p.send, 0, false);
  r.get<float>("dx", &p.dx, 0.0f, false);
  r.get<float>("dz", &p.dz, 0.0f, false);
  r.get<float>("dt", &p.dt, 0.0f, false);
  r.get<float>("fr", &p.fr, 0.0f, false);
  r.get<float>("velfx", &p.velfx, 0.0f, true);
  get_string(r, "precsg", p.precsg, false);
  get_string(r, "wdir", p.wdir, false);
  get_string(r, "v0file", p.v0file, false);
  get_string(r, "vfile", p.vfile, true);
  get_string(r, "coordfile", p.coordfile, false);
  if (p.mask) get_string(r, "maskfile", p.maskfile, false);
  if (p.planeTag) {
    r.get<int>("np", &p.np, 0, false);
    r.get<float>("dp", &p.dp, 0.0f, false);
    r.get<float>("pmin", &p.pmin, 0.0f, false);
  }
  if (r.rc) return r.rc;
  *out = p;
  return SEIS_OK;
}

int seis_coords_count(const char *file, int *ns) {
  std::vector<std::string> lines;
  if (!file || !ns || !read_lines(file, &lines) || lines.empty()) return SEIS_ERR_ARG;
  CoordLine c{};
  scan(lines[0], &c);
  float hs0 = c.hs;
  int n = 1;  // countShots, coord.cpp:149-175
  for (size_t i = 1; i < lines.size(); i++) {
    scan(lines[i], &c);
    if (c.hs != hs0) n++;
    hs0 = c.hs;
  }
  *ns = n;
  return SEIS_OK;
}

int seis_coords_read(const char *file, int ns, int ngmax, int *ng, float *sc, float *gc) {
  std::vector<std::string> lines;
  if (!file || ns < 1 || ngmax < 1 || !ng || !sc || !gc || !read_lines(file, &lines) ||
      lines.empty())
    return SEIS_ERR_ARG;
  const float fill = -1e10f;  // coord.cpp:60
  for (size_t i = 0; i < (size_t)ns * 2 * ngmax; i++) gc[i] = fill;
  for (int i = 0; i < ns; i++) ng[i] = 0;
  CoordLine c{};
  scan(lines[0], &c);
  float hs0 = c.hs;
  int cs = 0, ig = 0, cnt = 1;
  sc[0] = c.hs;
  sc[1] = c.vs;
  gc[0] = c.hg;
  gc[(size_t)ngmax] = c.vg;
  for (size_t i = 1; i < lines.size(); i++) {
    scan(lines[i], &c);
    if (c.hs == hs0) {
      ig++;
      cnt++;
    } else {
      cs++;
      ig = 0;
      cnt = 1;
      if (cs >= ns) return SEIS_ERR_ARG;
      sc[2 * cs] = c.hs;  // getSources, coord.cpp:40-48
      sc[2 * cs + 1] = c.vs;
    }
    if (ig < ngmax) {  // getReceivers, coord.cpp:80-93
      gc[((size_t)cs * 2) * ngmax + ig] = c.hg;
      gc[((size_t)cs * 2 + 1) * ngmax + ig] = c.vg;
    }
    ng[cs] = cnt;  // countReceivers, coord.cpp:124-141
    hs0 = c.hs;
  }
  ng[cs] = cnt - 1;  // coord.cpp:143-144: the last trace read twice
  return cs == ns - 1 ? SEIS_OK : SEIS_ERR_ARG;
}

}  // extern "C"

// ------------------------------------------------------------------ driver
struct seis_driver {
  seis_fd_ctx *ctx = nullptr;
  seis_params p{};
  int batch = 0;
  std::vector<int> ng;
  std::vector<float> sc, gc;  // sc [ns][2], gc [ns][2][ngmax]
  char err[512] = {0};

  const float *gx(int is) const { return gc.data() + (size_t)is * 2 * p.ngmax; }
  const float *gz(int is) const { return gc.data() + ((size_t)is * 2 + 1) * p.ngmax; }
  std::string csg_name(int is) const { return std::string(p.precsg) + std::to_string(is) + ".dat"; }
  std::string born_name(int is) const {
    return std::string(p.wdir) + "BORN" + std::to_string(is) + ".dat";
  }
  std::string image_name(int is) const {
    return std::string(p.wdir) + "CSG_IMAGE" + std::to_string(is) + ".dat";
  }
};

namespace {

struct ShotGeom {
  float fx = 0.0f;
  int nx = 0, isx = 0, isz = 0;
  std::vector<int> igz, cols;
  seis_shot_desc desc{};
};

// getVel / getIgz / source index of shot is (inversion.cpp:423-429)
int shot_geom(const seis_driver &d, int is, ShotGeom *s) {
  const seis_params &p = d.p;
  int rc = seis_geom_aperture(d.sc[2 * is], d.gx(is), d.ng[is], p.dx, p.lpad, p.rpad, &s->fx, &s->nx);
  if (rc) return rc;
  s->igz.assign((size_t)s->nx, 0);
  s->cols.assign((size_t)s->nx, 0);
  rc = seis_geom_extract_columns(p.nx, p.velfx, p.dx, s->fx, s->nx, s->cols.data());
  if (!rc)
    rc = seis_geom_receiver_rows(d.gx(is), d.gz(is), d.ng[is], s->fx, s->nx, p.dx, p.dz, p.nz,
                                 s->igz.data());
  if (!rc) rc = seis_geom_source_index(d.sc[2 * is], d.sc[2 * is + 1], s->fx, p.dx, p.dz, &s->isx,
                                       &s->isz);
  s->desc = seis_shot_desc{s->nx, p.nz, p.npml, p.nt, p.delaycal, s->isx, s->isz,
                           p.dt, p.dx, p.dz, s->igz.data()};
  return rc;
}

std::vector<float> sub_grid(const float *model, const seis_params &p, const ShotGeom &s) {
  std::vector<float> out((size_t)s.nx * p.nz);
  for (int ix = 0; ix < s.nx; ix++)
    std::memcpy(out.data() + (size_t)ix * p.nz, model + (size_t)s.cols[ix] * p.nz,
                sizeof(float) * p.nz);
  return out;
}

bool read_file(const std::string &name, float *dst, size_t n) {
  std::ifstream in(name, std::ios::binary);
  if (!in) return false;
  in.read(reinterpret_cast<char *>(dst), (std::streamsize)(sizeof(float) * n));
  return (size_t)in.gcount() == sizeof(float) * n;
}

bool write_file(const std::string &name, const float *src, size_t n) {
  std::ofstream out(name, std::ios::binary | std::ios::trunc);
  if (!out) return false;
  out.write(reinterpret_cast<const char *>(src), (std::streamsize)(sizeof(float) * n));
  return (bool)out;
}

int dfail(seis_driver *d, int rc, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(d->err, sizeof d->err, fmt, ap);
  va_end(ap);
  return rc;
}

// the wavelet of every shot: rickerWavelet(dt, fr, delay + delaycal, nt + delaycal)
std::vector<float> wavelet(const seis_params &p) {
  const int NT = p.nt + p.delaycal;
  std::vector<float> w((size_t)NT);
  seis_fd_ricker(p.dt, p.fr, p.delay + p.delaycal, NT, w.data());
  return w;
}

std::vector<float> load_model(seis_driver *d, const char *name, int *rc) {
  std::vector<float> m((size_t)d->p.nx * d->p.nz);
  if (!read_file(name, m.data(), m.size())) *rc = dfail(d, SEIS_ERR_ARG, "cannot read %s", name);
  return m;
}

// shots of [s0, s1) in batches; fn(first, count) for each batch
template <class F>
int in_batches(const seis_driver *d, int s0, int s1, F fn) {
  const int step = d->batch > 0 ? d->batch : std::max(1, s1 - s0);
  for (int b = s0; b < s1; b += step) {
    int rc = fn(b, std::min(step, s1 - b));
    if (rc) return rc;
  }
  return SEIS_OK;
}

// reads shot is's gather, mutes the direct arrival and moves the traces to
// the columns of its aperture (adjoint_MPI, inversion.cpp:419-422)
int observed(seis_driver *d, int is, int born_data, const float *v0, const ShotGeom &g,
             std::vector<float> *rec) {
  const seis_params &p = d->p;
  std::vector<float> csg((size_t)d->ng[is] * p.nt);
  const std::string name = born_data ? d->born_name(is) : d->csg_name(is);
  if (!read_file(name, csg.data(), csg.size()))
    return dfail(d, SEIS_ERR_ARG, "cannot read %s", name.c_str());
  int rc = seis_geom_remove_direct(csg.data(), d->ng[is], p.nt, d->gx(is), d->gz(is),
                                   d->sc[2 * is], d->sc[2 * is + 1], v0, p.nz, p.nx, p.dx, p.dz,
                                   p.dt, p.fr, p.velfx, p.delay);
  rec->assign((size_t)g.nx * p.nt, 0.0f);
  if (!rc)
    rc = seis_geom_reorder(csg.data(), d->ng[is], p.nt, d->gx(is), rec->data(), g.fx, g.nx, p.dx,
                           0);
  return rc ? dfail(d, rc, "shot %d geometry", is) : SEIS_OK;
}

}  // namespace

extern "C" {

int seis_driver_create(seis_fd_ctx *ctx, const char *param_file, int batch, seis_driver **out) {
  if (!param_file || !out) return SEIS_ERR_ARG;
  *out = nullptr;
  seis_driver *d = new (std::nothrow) seis_driver();
  if (!d) return SEIS_ERR_NOMEM;
  d->ctx = ctx;
  d->batch = batch;
  int rc = seis_params_read(param_file, &d->p, d->err, sizeof d->err);
  int ns = 0;
  if (!rc && (seis_coords_count(d->p.coordfile, &ns) || ns != d->p.ns))
    rc = dfail(d, SEIS_ERR_ARG, "coordinate file %s: %d shots, the parameter file says %d",
               d->p.coordfile, ns, d->p.ns);
  if (!rc) {
    d->ng.assign((size_t)ns, 0);
    d->sc.assign((size_t)ns * 2, 0.0f);
    d->gc.assign((size_t)ns * 2 * d->p.ngmax, 0.0f);
    if (seis_coords_read(d->p.coordfile, ns, d->p.ngmax, d->ng.data(), d->sc.data(),
                         d->gc.data()))
      rc = dfail(d, SEIS_ERR_ARG, "coordinate file %s: cannot read", d->p.coordfile);
    else if (*std::max_element(d->ng.begin(), d->ng.end()) != d->p.ngmax)
      rc = dfail(d, SEIS_ERR_ARG, "coordinate file %s: ngmax %d, the parameter file says %d",
                 d->p.coordfile, *std::max_element(d->ng.begin(), d->ng.end()), d->p.ngmax);
  }
  if (rc) {
    std::fprintf(stderr, "seis_driver_create: %s\n", d->err);
    delete d;
    return rc;
  }
  *out = d;
  return SEIS_OK;
}

int seis_driver_destroy(seis_driver *d) {
  delete d;
  return SEIS_OK;
}

const seis_params *seis_driver_params(const seis_driver *d) { return d ? &d->p : nullptr; }

int seis_driver_modeling(seis_driver *d, const float *h_v) {
  if (!d) return SEIS_ERR_ARG;
  if (!d->ctx) return dfail(d, SEIS_ERR_STATE, "driver created without a device context");
  const seis_params &p = d->p;
  int rc = SEIS_OK;
  std::vector<float> vfile;
  if (!h_v) {
    vfile = load_model(d, p.vfile, &rc);
    if (rc) return rc;
    h_v = vfile.data();
  }
  const std::vector<float> wav = wavelet(p);
  return in_batches(d, 0, p.ns, [&](int s0, int n) {
    std::vector<ShotGeom> g((size_t)n);
    std::vector<std::vector<float>> vel((size_t)n), rec((size_t)n);
    std::vector<seis_shot_desc> desc;
    std::vector<const float *> pw, pv;
    std::vector<float *> pr;
    for (int k = 0; k < n; k++) {
      int r = shot_geom(*d, s0 + k, &g[k]);
      if (r) return dfail(d, r, "shot %d geometry", s0 + k);
      vel[k] = sub_grid(h_v, p, g[k]);
      rec[k].assign((size_t)g[k].nx * p.nt, 0.0f);
    }
    for (int k = 0; k < n; k++) {
      desc.push_back(g[k].desc);
      pw.push_back(wav.data());
      pv.push_back(vel[k].data());
      pr.push_back(rec[k].data());
    }
    int r = seis_fd_modeling_batch(d->ctx, n, desc.data(), pw.data(), pv.data(), pr.data());
    if (r) return dfail(d, r, "modeling: %s", seis_fd_last_error(d->ctx));
    for (int k = 0; k < n; k++) {  // modeling_MPI, inversion.cpp:190-192
      const int is = s0 + k;
      std::vector<float> csg((size_t)d->ng[is] * p.nt);
      r = seis_geom_reorder(csg.data(), d->ng[is], p.nt, d->gx(is), rec[k].data(), g[k].fx,
                            g[k].nx, p.dx, 1);
      if (!r)
        r = seis_geom_remove_direct(csg.data(), d->ng[is], p.nt, d->gx(is), d->gz(is),
                                    d->sc[2 * is], d->sc[2 * is + 1], h_v, p.nz, p.nx, p.dx, p.dz,
                                    p.dt, p.fr, p.velfx, p.delay);
      if (r) return dfail(d, r, "shot %d geometry", is);
      if (!write_file(d->csg_name(is), csg.data(), csg.size()))
        return dfail(d, SEIS_ERR_ARG, "cannot write %s", d->csg_name(is).c_str());
    }
    return SEIS_OK;
  });
}

int seis_driver_born(seis_driver *d, const float *h_dv) {
  if (!d || !h_dv) return SEIS_ERR_ARG;
  if (!d->ctx) return dfail(d, SEIS_ERR_STATE, "driver created without a device context");
  const seis_params &p = d->p;
  int rc = SEIS_OK;
  const std::vector<float> v0 = load_model(d, p.v0file, &rc);
  if (rc) return rc;
  const std::vector<float> wav = wavelet(p);
  return in_batches(d, 0, p.ns, [&](int s0, int n) {
    std::vector<ShotGeom> g((size_t)n);
    std::vector<std::vector<float>> vel((size_t)n), dv((size_t)n), rec((size_t)n);
    std::vector<seis_shot_desc> desc;
    std::vector<const float *> pw, pv, pd;
    std::vector<float *> pr;
    for (int k = 0; k < n; k++) {
      int r = shot_geom(*d, s0 + k, &g[k]);
      if (r) return dfail(d, r, "shot %d geometry", s0 + k);
      vel[k] = sub_grid(v0.data(), p, g[k]);  // forward_MPI, inversion.cpp:515-516
      dv[k] = sub_grid(h_dv, p, g[k]);
      rec[k].assign((size_t)g[k].nx * p.nt, 0.0f);
    }
    for (int k = 0; k < n; k++) {
      desc.push_back(g[k].desc);
      pw.push_back(wav.data());
      pv.push_back(vel[k].data());
      pd.push_back(dv[k].data());
      pr.push_back(rec[k].data());
    }
    int r = seis_fd_born_batch(d->ctx, n, desc.data(), pw.data(), pv.data(), pd.data(), pr.data());
    if (r) return dfail(d, r, "born: %s", seis_fd_last_error(d->ctx));
    for (int k = 0; k < n; k++) {  // forward_MPI, inversion.cpp:526-529
      const int is = s0 + k;
      std::vector<float> csg((size_t)d->ng[is] * p.nt);
      r = seis_geom_reorder(csg.data(), d->ng[is], p.nt, d->gx(is), rec[k].data(), g[k].fx,
                            g[k].nx, p.dx, 1);
      if (!r)
        r = seis_geom_remove_direct(csg.data(), d->ng[is], p.nt, d->gx(is), d->gz(is),
                                    d->sc[2 * is], d->sc[2 * is + 1], v0.data(), p.nz, p.nx, p.dx,
                                    p.dz, p.dt, p.fr, p.velfx, p.delay);
      if (r) return dfail(d, r, "shot %d geometry", is);
      if (!write_file(d->born_name(is), csg.data(), csg.size()))
        return dfail(d, SEIS_ERR_ARG, "cannot write %s", d->born_name(is).c_str());
    }
    return SEIS_OK;
  });
}

int seis_driver_rtm(seis_driver *d, int born_data, float *h_img) {
  if (!d || !h_img) return SEIS_ERR_ARG;
  if (!d->ctx) return dfail(d, SEIS_ERR_STATE, "driver created without a device context");
  const seis_params &p = d->p;
  int rc = SEIS_OK;
  const std::vector<float> v0 = load_model(d, p.v0file, &rc);
  if (rc) return rc;
  std::vector<float> mask;
  if (p.mask) {
    mask = load_model(d, p.maskfile, &rc);
    if (rc) return rc;
  }
  const size_t nm = (size_t)p.nx * p.nz;
  std::memset(h_img, 0, sizeof(float) * nm);
  const std::vector<float> wav = wavelet(p);
  const int s0 = std::max(0, p.sbegin), s1 = std::min(p.ns, p.send + 1);
  return in_batches(d, s0, s1, [&](int b0, int n) {
    std::vector<ShotGeom> g((size_t)n);
    std::vector<std::vector<float>> vel((size_t)n), rec((size_t)n), img((size_t)n);
    std::vector<seis_shot_desc> desc;
    std::vector<const float *> pw, pv, pr;
    std::vector<float *> pi;
    for (int k = 0; k < n; k++) {
      const int is = b0 + k;
      int r = shot_geom(*d, is, &g[k]);
      if (r) return dfail(d, r, "shot %d geometry", is);
      vel[k] = sub_grid(v0.data(), p, g[k]);
      r = observed(d, is, born_data, v0.data(), g[k], &rec[k]);
      if (r) return r;
      img[k].assign((size_t)g[k].nx * p.nz, 0.0f);
    }
    for (int k = 0; k < n; k++) {
      desc.push_back(g[k].desc);
      pw.push_back(wav.data());
      pv.push_back(vel[k].data());
      pr.push_back(rec[k].data());
      pi.push_back(img[k].data());
    }
    int r = seis_fd_rtm_batch(d->ctx, n, desc.data(), pw.data(), pv.data(), pr.data(), pi.data());
    if (r) return dfail(d, r, "rtm: %s", seis_fd_last_error(d->ctx));
    std::vector<float> tmp(nm);
    for (int k = 0; k < n; k++) {  // adjoint_MPI, inversion.cpp:431-440, :459-468
      const int is = b0 + k;
      r = seis_geom_swap_model(img[k].data(), tmp.data(), g[k].fx, p.velfx, p.nz, g[k].nx, p.nz,
                               p.nx, p.dx, 0);
      if (r) return dfail(d, r, "shot %d image scatter", is);
      if (p.mask)
        for (size_t i = 0; i < nm; i++) tmp[i] = tmp[i] * mask[i];
      if (!write_file(d->image_name(is), tmp.data(), nm))
        return dfail(d, SEIS_ERR_ARG, "cannot write %s", d->image_name(is).c_str());
      for (size_t i = 0; i < nm; i++) h_img[i] = tmp[i] + h_img[i];
    }
    return SEIS_OK;
  });
}

int seis_driver_illum(seis_driver *d, float *h_ss) {
  if (!d || !h_ss) return SEIS_ERR_ARG;
  if (!d->ctx) return dfail(d, SEIS_ERR_STATE, "driver created without a device context");
  const seis_params &p = d->p;
  int rc = SEIS_OK;
  const std::vector<float> v0 = load_model(d, p.v0file, &rc);
  if (rc) return rc;
  const size_t nm = (size_t)p.nx * p.nz;
  std::memset(h_ss, 0, sizeof(float) * nm);
  const std::vector<float> wav = wavelet(p);
  return in_batches(d, 0, p.ns, [&](int s0, int n) {
    std::vector<ShotGeom> g((size_t)n);
    std::vector<std::vector<float>> vel((size_t)n), ss((size_t)n);
    std::vector<seis_shot_desc> desc;
    std::vector<const float *> pw, pv;
    std::vector<float *> po;
    for (int k = 0; k < n; k++) {
      int r = shot_geom(*d, s0 + k, &g[k]);
      if (r) return dfail(d, r, "shot %d geometry", s0 + k);
      vel[k] = sub_grid(v0.data(), p, g[k]);
      ss[k].assign((size_t)g[k].nx * p.nz, 0.0f);
    }
    for (int k = 0; k < n; k++) {
      desc.push_back(g[k].desc);
      pw.push_back(wav.data());
      pv.push_back(vel[k].data());
      po.push_back(ss[k].data());
    }
    int r = seis_fd_illum_batch(d->ctx, n, desc.data(), pw.data(), pv.data(), po.data());
    if (r) return dfail(d, r, "illum: %s", seis_fd_last_error(d->ctx));
    std::vector<float> tmp(nm);
    for (int k = 0; k < n; k++) {  // illum_MPI, inversion.cpp:257-260, :271-282
      const int is = s0 + k;
      r = seis_geom_swap_model(ss[k].data(), tmp.data(), g[k].fx, p.velfx, p.nz, g[k].nx, p.nz,
                               p.nx, p.dx, 0);
      if (r) return dfail(d, r, "shot %d illumination scatter", is);
      const std::string name = std::string(p.wdir) + "ILLUM" + std::to_string(is) + ".dat";
      if (!write_file(name, tmp.data(), nm))
        return dfail(d, SEIS_ERR_ARG, "cannot write %s", name.c_str());
      for (size_t i = 0; i < nm; i++) h_ss[i] = tmp[i] + h_ss[i];
    }
    return SEIS_OK;
  });
}

int seis_driver_plane_prepare(seis_driver *d) {
  if (!d) return SEIS_ERR_ARG;
  const seis_params &p = d->p;
  if (!p.planeTag) return dfail(d, SEIS_ERR_STATE, "planeTag is 0");
  const int NT = p.nt + p.delaycal;
  const int hb = 100;  // Hilbert<float> hl(100), InitInversion.cpp:145
  const std::vector<float> wav = wavelet(p);
  std::vector<float> hwav((size_t)NT);
  seis_fd_hilbert(wav.data(), hwav.data(), NT, hb);
  // each trace and its Hilbert transform, once for all wavenumbers
  std::vector<std::vector<float>> data((size_t)p.ns), hdata((size_t)p.ns);
  float sxmax = d->sc[0];
  for (int is = 0; is < p.ns; is++) {
    const size_t n = (size_t)d->ng[is] * p.nt;
    data[is].resize(n);
    hdata[is].resize(n);
    if (!read_file(d->csg_name(is), data[is].data(), n))
      return dfail(d, SEIS_ERR_ARG, "cannot read %s", d->csg_name(is).c_str());
    for (int ig = 0; ig < d->ng[is]; ig++)
      seis_fd_hilbert(data[is].data() + (size_t)ig * p.nt, hdata[is].data() + (size_t)ig * p.nt,
                      p.nt, hb);
    sxmax = sxmax < d->sc[2 * is] ? d->sc[2 * is] : sxmax;  // :840-843
  }
  const float xlo = (float)((double)p.velfx - 0.0001 * (double)p.dx);  // :862
  std::vector<float> sou((size_t)p.nx * NT), rec((size_t)p.nx * p.nt), tr((size_t)p.nx * p.nt);
  std::vector<float> tw((size_t)NT), csgn;
  for (int k = 0; k < p.np; k++) {
    std::fill(sou.begin(), sou.end(), 0.0f);
    std::fill(rec.begin(), rec.end(), 0.0f);
    const float kx = p.pmin + (float)k * p.dp;  // :860
    for (int is = 0; is < p.ns; is++) {
      const float sx = d->sc[2 * is];
      if (!((sx - xlo) >= 0.0f && (sxmax - sx) >= 0.0f))
        return dfail(d, SEIS_ERR_ARG, "shot %d x outside [velfx, largest source x]", is);
      // harmonic(), InitInversion.cpp:141-150: cos/sin of the float phase
      const float cn = std::cos(kx * sx), sn = std::sin(kx * sx);
      for (int it = 0; it < NT; it++) tw[it] = cn * wav[it] - sn * hwav[it];
      const int isx = (int)((sx - p.velfx) / p.dx + 0.001f);  // :879
      if (isx < 0 || isx >= p.nx) return dfail(d, SEIS_ERR_ARG, "shot %d column %d", is, isx);
      float *col = sou.data() + (size_t)isx * NT;
      for (int it = 0; it < NT; it++) col[it] = col[it] + tw[it];
      const size_t n = data[is].size();
      csgn.resize(n);
      for (size_t i = 0; i < n; i++) csgn[i] = cn * data[is][i] - sn * hdata[is][i];
      int r = seis_geom_reorder(csgn.data(), d->ng[is], p.nt, d->gx(is), tr.data(), p.velfx,
                                p.nx, p.dx, 0);
      if (r) return dfail(d, r, "shot %d traces", is);
      for (size_t i = 0; i < rec.size(); i++) rec[i] = tr[i] + rec[i];  // :897
    }
    const std::string sn_ = std::string(p.wdir) + "PLANE_S_NEW" + std::to_string(k) + ".dat";
    const std::string rn_ = std::string(p.wdir) + "PLANE_R_NEW" + std::to_string(k) + ".dat";
    if (!write_file(sn_, sou.data(), sou.size()) || !write_file(rn_, rec.data(), rec.size()))
      return dfail(d, SEIS_ERR_ARG, "cannot write %s", sn_.c_str());
  }
  return SEIS_OK;
}

int seis_driver_rtm_plane(seis_driver *d, int born_data, float *h_img) {
  if (!d || !h_img) return SEIS_ERR_ARG;
  if (!d->ctx) return dfail(d, SEIS_ERR_STATE, "driver created without a device context");
  const seis_params &p = d->p;
  int rc = SEIS_OK;
  const std::vector<float> v0 = load_model(d, p.v0file, &rc);
  if (rc) return rc;
  std::vector<float> mask;
  if (p.mask) {
    mask = load_model(d, p.maskfile, &rc);
    if (rc) return rc;
  }
  const size_t nm = (size_t)p.nx * p.nz;
  const int NT = p.nt + p.delaycal;
  std::memset(h_img, 0, sizeof(float) * nm);
  // source and receiver rows of every wavenumber (inversion.cpp:1062-1063)
  const int sz = (int)((d->sc[1] - 0.0f) / p.dz + 0.0001f);
  const int gz = (int)((d->gz(0)[0] - 0.0f) / p.dz + 0.0001f);
  std::vector<int> gzs((size_t)p.nx, gz);
  seis_shot_desc desc{p.nx, p.nz, p.npml, p.nt, p.delaycal, p.nx / 2, sz,
                      p.dt, p.dx, p.dz, gzs.data()};
  std::vector<float> sou((size_t)p.nx * NT), rec((size_t)p.nx * p.nt), img(nm);
  for (int k = 0; k < p.np; k++) {
    const std::string sn = std::string(p.wdir) + "PLANE_S_NEW" + std::to_string(k) + ".dat";
    const std::string rn = born_data ? d->born_name(k)
                                     : std::string(p.wdir) + "PLANE_R_NEW" + std::to_string(k) + ".dat";
    if (!read_file(sn, sou.data(), sou.size())) return dfail(d, SEIS_ERR_ARG, "cannot read %s", sn.c_str());
    if (!read_file(rn, rec.data(), rec.size())) return dfail(d, SEIS_ERR_ARG, "cannot read %s", rn.c_str());
    int r = seis_fd_rtm_plane(d->ctx, &desc, sou.data(), v0.data(), rec.data(), img.data());
    if (r) return dfail(d, r, "rtm_plane: %s", seis_fd_last_error(d->ctx));
    if (p.mask)
      for (size_t i = 0; i < nm; i++) img[i] = img[i] * mask[i];
    const std::string in = std::string(p.wdir) + "IMAGE" + std::to_string(k) + ".dat";
    if (!write_file(in, img.data(), nm)) return dfail(d, SEIS_ERR_ARG, "cannot write %s", in.c_str());
    for (size_t i = 0; i < nm; i++) h_img[i] = img[i] + h_img[i];
  }
  return SEIS_OK;
}

int seis_driver_illum_plane(seis_driver *d, float *h_ss) {
  if (!d) return SEIS_ERR_ARG;
  if (!d->ctx) return dfail(d, SEIS_ERR_STATE, "driver created without a device context");
  const seis_params &p = d->p;
  int rc = SEIS_OK;
  const std::vector<float> v0 = load_model(d, p.v0file, &rc);
  if (rc) return rc;
  const size_t nm = (size_t)p.nx * p.nz;
  const int NT = p.nt + p.delaycal;
  if (h_ss) std::memset(h_ss, 0, sizeof(float) * nm);
  const int sz = (int)((d->sc[1] - 0.0f) / p.dz + 0.0001f);  // inversion.cpp:331
  std::vector<int> gzs((size_t)p.nx, 0);
  seis_shot_desc desc{p.nx, p.nz, p.npml, p.nt, p.delaycal, p.nx / 2, sz,
                      p.dt, p.dx, p.dz, gzs.data()};
  std::vector<float> sou((size_t)p.nx * NT), ss(nm);
  for (int k = 0; k < p.np; k++) {
    const std::string sn = std::string(p.wdir) + "PLANE_S_NEW" + std::to_string(k) + ".dat";
    if (!read_file(sn, sou.data(), sou.size())) return dfail(d, SEIS_ERR_ARG, "cannot read %s", sn.c_str());
    int r = seis_fd_illum_plane(d->ctx, &desc, sou.data(), v0.data(), ss.data());
    if (r) return dfail(d, r, "illum_plane: %s", seis_fd_last_error(d->ctx));
    const std::string on = std::string(p.wdir) + "ILLUM_PLANE" + std::to_string(k) + ".dat";
    if (!write_file(on, ss.data(), nm)) return dfail(d, SEIS_ERR_ARG, "cannot write %s", on.c_str());
    if (h_ss)
      for (size_t i = 0; i < nm; i++) h_ss[i] = ss[i] + h_ss[i];
  }
  return SEIS_OK;
}

int seis_driver_lsrtm(seis_driver *d, int born_data, int niter, const seis_lsrtm_opts *opts,
                      float *h_img, double *h_rr) {
  if (!d || !h_img || niter < 0) return SEIS_ERR_ARG;
  if (!d->ctx) return dfail(d, SEIS_ERR_STATE, "driver created without a device context");
  const seis_params &p = d->p;
  int rc = SEIS_OK;
  const std::vector<float> v0 = load_model(d, p.v0file, &rc);
  if (rc) return rc;
  const std::vector<float> wav = wavelet(p);
  std::vector<ShotGeom> g((size_t)p.ns);
  std::vector<seis_shot_desc> desc;
  std::vector<int> cmap;
  for (int is = 0; is < p.ns; is++) {
    int r = shot_geom(*d, is, &g[is]);
    if (r) return dfail(d, r, "shot %d geometry", is);
    desc.push_back(g[is].desc);
    cmap.insert(cmap.end(), g[is].cols.begin(), g[is].cols.end());
  }
  seis_fd_lsrtm *L = nullptr;
  rc = seis_fd_lsrtm_create_mapped(d->ctx, p.nx, p.nz, p.ns, desc.data(), cmap.data(), opts, &L);
  if (rc) return dfail(d, rc, "lsrtm: %s", seis_fd_last_error(d->ctx));
  rc = seis_fd_lsrtm_set_background(L, v0.data(), wav.data());
  std::vector<float> rec, csg_t;
  for (int is = 0; is < p.ns && !rc; is++) {
    rc = observed(d, is, born_data, v0.data(), g[is], &rec);
    if (!rc) rc = seis_fd_lsrtm_set_data(L, is, rec.data());
  }
  double rr0 = 0.0;
  if (!rc) rc = seis_fd_lsrtm_reset(L, &rr0);
  if (!rc && h_rr) h_rr[0] = rr0;
  if (!rc && niter > 0) rc = seis_fd_lsrtm_iterate(L, niter, h_rr ? h_rr + 1 : nullptr);
  if (!rc) rc = seis_fd_lsrtm_model(L, h_img);
  if (rc && !d->err[0]) dfail(d, rc, "lsrtm: %s", seis_fd_last_error(d->ctx));
  seis_fd_lsrtm_destroy(L);
  return rc;
}

}  // extern "C"
