/*
 * CPU oracle for the Seis 2-D acoustic FD path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference algorithm (src/util/fd.cpp,
 * src/util/InitInversion.cpp, src/util/wavelet.cpp, src/filter/hilbert.h),
 * compiled twice from seis_oracle_body.h: REAL=float (suffix _f32, evaluated in
 * the reference's operation order so that it matches the reference bit for bit
 * on x86-64 without FMA) and REAL=double (suffix _f64, the "same code in FP64"
 * used as the accuracy yardstick).  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load it; the CUDA library never does.
 *
 * Layout: models/images [nx][nz] (z fastest), gathers [nx][nt] (t fastest),
 * padded grids [nx+2pml][nz+2pml] -- the reference's MyAlloc layout
 * (src/util/memory.h:29-44).
 */
#ifndef SEIS_ORACLE_H
#define SEIS_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

#define SEIS_ORACLE_DECL(R, S)                                                  \
  void orc_ricker_##S(R dt, R fr, int delay, int n, R *out);                    \
  void orc_set_abs_##S(int nz, int nx, int pml, R *w);                          \
  void orc_set_vel_##S(const R *v, int nz, int nx, int pml, R *out);            \
  void orc_hilbert_##S(const R *in, R *out, int n, int half);                   \
  int orc_modeling_##S(R dt, R dx, R dz, int nt, int ndel, int nx, int nz,      \
                       int pml, int sx, int sz, const int *gz, const R *wav,    \
                       const R *vel, R *rec);                                   \
  int orc_born_##S(R dt, R dx, R dz, int nt, int ndel, int nx, int nz, int pml, \
                   int sx, int sz, const int *gz, const R *wav, const R *vel,   \
                   const R *dv, R *rec);                                        \
  int orc_rtm_##S(R dt, R dx, R dz, int nt, int ndel, int nx, int nz, int pml,  \
                  int sx, int sz, const int *gz, const R *wav, const R *vel,    \
                  const R *rec, R *img);                                        \
  int orc_born_plane_##S(R dt, R dx, R dz, int nt, int ndel, int nx, int nz,     \
                         int pml, int sz, int gz, const R *sou, const R *vel,    \
                         const R *dv, R *rec);                                   \
  int orc_rtm_plane_##S(R dt, R dx, R dz, int nt, int ndel, int nx, int nz,      \
                        int pml, int sz, int gz, const R *sou, const R *vel,     \
                        const R *rec, R *img);                                   \
  int orc_rtm_true_##S(R dt, R dx, R dz, int nt, int ndel, int nx, int nz,       \
                       int pml, int sx, int sz, const int *gz, const R *wav,     \
                       const R *vel, const R *rec, R *img);                      \
  int orc_rtm_updown_##S(R dt, R dx, R dz, int nt, int ndel, int nx, int nz,     \
                         int pml, int sx, int sz, const int *gz, const R *wav,   \
                         const R *wavh, const R *vel, const R *rec, R *img,      \
                         R *comp);                                               \
  int orc_illum_##S(R dt, R dx, R dz, int nt, int ndel, int nx, int nz, int pml, \
                    int sx, int sz, const R *wav, const R *vel, R *ss);         \
  int orc_illum_plane_##S(R dt, R dx, R dz, int nt, int ndel, int nx, int nz,   \
                          int pml, int sz, const R *sou, const R *vel, R *ss);  \
  int orc_born_adjoint_##S(R dt, R dx, R dz, int nt, int ndel, int nx, int nz,  \
                           int pml, int sx, int sz, const int *gz,              \
                           const R *wav, const R *vel, const R *rec, R *img);   \
  int orc_born_adjoint_thin_##S(R dt, R dx, R dz, int nt, int ndel, int nx,     \
                                int nz, int pml, int sx, int sz, const int *gz, \
                                const R *wav, const R *vel, const R *rec,       \
                                int every, R *img);                            \
  int orc_born_adjoint_ck_##S(R dt, R dx, R dz, int nt, int ndel, int nx,       \
                              int nz, int pml, int sx, int sz, const int *gz,   \
                              const R *wav, const R *vel, const R *rec, int ck, \
                              R *img);

SEIS_ORACLE_DECL(float, f32)
SEIS_ORACLE_DECL(double, f64)

#ifdef __cplusplus
}
#endif
#endif
