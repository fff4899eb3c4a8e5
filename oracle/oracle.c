/*
 * ORACLE -- test infrastructure only (see oracle.h for the contract and the
 * "parity unpinned" statement).
 *
 * Literal CPU restatement of OpenTBL's RK3 substep with single-domain
 * semantics. Arrays keep the reference's layouts: planes (0:nz2, jee, nx)
 * complex as nz1 = 2*(nz2+1) reals fastest, pencils (nx, nz1*jee) with x
 * fastest (change.f90:563,628). Indices below are Fortran's (1-based planes
 * and rows, 0-based real index kr).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

struct orc_box {
  int nx, ny, nz, nz1, nz2, xout, xround, dt_mode;
  double dt_fixed;
  double *c;
  otbl_coef_offsets o;
  double *f[OTBL_F_COUNT]; /* u v w p rhsupa rhsvpa rhswpa */
  double *um, *u0, *v0;
  double tiempo, timeinit, dt, utauout, rthout, dout, gamma1, gamma2, timec;
  double umax, wmax, vmax;
  double ener[15]; /* module statistics, mod.F90:264 */
  int dt_frozen;
  /* planes */
  double *resu, *resv, *resw, *rhsu, *rhsv, *rhsw, *wk1, *wk2, *wk3;
  /* pencils */
  double *penu, *penv, *penw, *pen;
  orc_fft *fz;  /* complex length nz/2 */
  orc_fft *fx;  /* complex length nx-1 */
};

static int g_threads = 0;
void orc_set_threads(int n) { g_threads = n; }
int orc_get_threads(void) {
#ifdef _OPENMP
  return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
  return 1;
#endif
}
#ifdef _OPENMP
#define NTH num_threads(orc_get_threads())
#endif

#define CF(b, id) ((b)->c + (b)->o.off[OTBL_C_##id])
#define A3(a, r, i) (a)[((size_t)(i)-1) * 3 + (r)-1]
#define A2(a, r, i) (a)[((size_t)(i)-1) * 2 + (r)-1]
#define M4(a, r, cc) (a)[((cc)-1) * 4 + (r)-1]
#define M5(a, r, cc) (a)[((cc)-1) * 5 + (r)-1]
#define M2(a, r, cc) (a)[((cc)-1) * 2 + (r)-1]
#define SC(b, s) (CF(b, SCAL)[OTBL_S_##s])

static inline double rnd(const orc_box *b, double x) {
  return b->xround ? (double)(float)x : x;
}

/* pointer to row j (1-based) of plane i (1-based) of a field with jee rows */
static inline double *PL(const orc_box *b, double *a, int jee, int i, int j) {
  return a + ((size_t)(i - 1) * jee + (size_t)(j - 1)) * b->nz1;
}

/* ------------------------------------------------------------------ */
orc_box *orc_create(const otbl_config *cfg, const double *coef) {
  orc_box *b = (orc_box *)calloc(1, sizeof(orc_box));
  b->nx = cfg->nx;
  b->ny = cfg->ny;
  b->nz = cfg->nz;
  b->nz1 = 2 * (cfg->nz / 3);
  b->nz2 = b->nz1 / 2 - 1;
  b->xout = cfg->xout;
  b->xround = cfg->xpose_round;
  b->dt_mode = cfg->dt_mode;
  b->dt_fixed = cfg->dt_fixed;
  otbl_coef_layout(b->nx, b->ny, b->nz, &b->o);
  const size_t nc = b->o.off[OTBL_C_COUNT];
  b->c = (double *)malloc(sizeof(double) * nc);
  memcpy(b->c, coef, sizeof(double) * nc);
  const size_t lu = otbl_field_len(b->nx, b->ny, b->nz, 1);
  const size_t lv = otbl_field_len(b->nx, b->ny, b->nz, 0);
  for (int id = 0; id < OTBL_F_COUNT; ++id) {
    const int ut = (id == OTBL_F_U || id == OTBL_F_W || id == OTBL_F_RHSUPA ||
                    id == OTBL_F_RHSWPA);
    b->f[id] = (double *)calloc(ut ? lu : lv, sizeof(double));
  }
  double **wk[] = {&b->resu, &b->resv, &b->resw, &b->rhsu, &b->rhsv, &b->rhsw,
                   &b->wk1,  &b->wk2,  &b->wk3,  &b->penu, &b->penv, &b->penw,
                   &b->pen};
  for (size_t t = 0; t < sizeof(wk) / sizeof(wk[0]); ++t)
    *wk[t] = (double *)calloc(lu, sizeof(double));
  b->um = (double *)calloc(b->ny + 1, sizeof(double));
  b->u0 = (double *)calloc(b->ny + 1, sizeof(double));
  b->v0 = (double *)calloc(b->ny, sizeof(double));
  b->fz = orc_fft_create(b->nz / 2);
  b->fx = orc_fft_create(b->nx - 1);
  return b;
}

void orc_destroy(orc_box *b) {
  if (!b) return;
  for (int id = 0; id < OTBL_F_COUNT; ++id) free(b->f[id]);
  free(b->resu); free(b->resv); free(b->resw); free(b->rhsu); free(b->rhsv);
  free(b->rhsw); free(b->wk1); free(b->wk2); free(b->wk3); free(b->penu);
  free(b->penv); free(b->penw); free(b->pen);
  free(b->um); free(b->u0); free(b->v0); free(b->c);
  orc_fft_destroy(b->fz);
  orc_fft_destroy(b->fx);
  free(b);
}

/* read-only views for the statistics restatement (orc_stats.c) */
int orc_box_dims(const orc_box *b, int *nx, int *ny, int *nz, int *xround) {
  *nx = b->nx;
  *ny = b->ny;
  *nz = b->nz;
  *xround = b->xround;
  return 0;
}
const double *orc_box_coef(const orc_box *b, otbl_coef_offsets *o) {
  *o = b->o;
  return b->c;
}
const orc_fft *orc_box_zfft(const orc_box *b) { return b->fz; }

double *orc_field(orc_box *b, int id) {
  return (id >= 0 && id < OTBL_F_COUNT) ? b->f[id] : NULL;
}

void orc_set_inflow(orc_box *b, const double *u0, const double *v0,
                    const double *um, const otbl_inflow *st) {
  memcpy(b->u0, u0, sizeof(double) * (b->ny + 1));
  memcpy(b->v0, v0, sizeof(double) * b->ny);
  memcpy(b->um, um, sizeof(double) * (b->ny + 1));
  b->tiempo = st->tiempo;
  b->timeinit = st->timeinit;
  b->dt = st->dt;
  b->utauout = st->utauout;
  b->rthout = st->rthout;
  b->dout = st->dout;
  b->gamma1 = st->gamma1;
  b->gamma2 = st->gamma2;
  b->timec = st->timec;
  b->dt_frozen = 0; /* a restart, as otbl_set_inflow */
  memset(b->ener, 0, sizeof b->ener);
}

void orc_get_inflow(orc_box *b, double *um, otbl_inflow *st) {
  if (um) memcpy(um, b->um, sizeof(double) * (b->ny + 1));
  if (st) {
    st->tiempo = b->tiempo;
    st->timeinit = b->timeinit;
    st->dt = b->dt;
    st->utauout = b->utauout;
    st->rthout = b->rthout;
    st->dout = b->dout;
    st->gamma1 = b->gamma1;
    st->gamma2 = b->gamma2;
    st->timec = b->timec;
    st->umax = b->umax;
    st->wmax = b->wmax;
    st->vmax = b->vmax;
  }
}

/* ---------------- transposes, change.f90:224-275 + 536-690 ----------------
 * pen(i, mp) = plan(mp, i) for mp = 1..nz1*jee, rounded to REAL4 in
 * OTBL_XPOSE_FP32 mode (transpose1/3 cast to kind=4, transpose2/4 back). */
void orc_chp2x(orc_box *b, double *pen, const double *plan, int jee) {
  const int nx = b->nx;
  const size_t np = (size_t)b->nz1 * jee;
#pragma omp parallel for NTH schedule(static)
  for (long mp = 0; mp < (long)np; ++mp)
    for (int i = 0; i < nx; ++i) pen[(size_t)mp * nx + i] = rnd(b, plan[(size_t)i * np + mp]);
}

void orc_chx2p(orc_box *b, const double *pen, double *plan, int jee) {
  const int nx = b->nx;
  const size_t np = (size_t)b->nz1 * jee;
#pragma omp parallel for NTH schedule(static)
  for (int i = 0; i < nx; ++i)
    for (size_t mp = 0; mp < np; ++mp) plan[(size_t)i * np + mp] = rnd(b, pen[mp * nx + i]);
}

/* ---------------- x-line compact operators, lip.f90 ---------------- */
/* interpxx, lip.f90:248-300. which = 0: u (inxu, cofiux, chi=2, loguv=1);
 * which = 1: v,w (inxv, cofivx, chi=1, loguv=0). pencils (nx, nlin). */
void orc_interpxx(orc_box *b, const double *gen, double *geni, int which, int nlin) {
  const int nx = b->nx;
  const double *icon = which == 0 ? CF(b, INXU) : CF(b, INXV);
  const double *econ = which == 0 ? CF(b, COFIUX) : CF(b, COFIVX);
  const double *inbx = CF(b, INBX);
  const int chi = which == 0 ? 2 : 1;
  const int loguv = which == 0 ? 1 : 0;
  const int chi2 = loguv == 1 ? chi + 1 : chi + 3;
#pragma omp parallel NTH
  {
    double *bb = (double *)malloc(sizeof(double) * (nx + 1));
#pragma omp for schedule(static)
    for (int k = 1; k <= nlin; ++k) {
      const double *g = gen + (size_t)(k - 1) * nx - 1; /* g[i], i=1..nx */
      for (int i = 2; i <= nx - 1; ++i) bb[i] = A2(econ, 1, i) * g[i] + A2(econ, 2, i) * g[i + 1];
      bb[1] = M4(inbx, chi2, 1) * g[1] + M4(inbx, chi2, 2) * g[2] + M4(inbx, chi2, 3) * g[3] +
              M4(inbx, chi2, 4) * g[4];
      bb[nx] = M4(inbx, chi, 1) * g[nx] + M4(inbx, chi, 2) * g[nx - 1] +
               M4(inbx, chi, 3) * g[nx - 2] + M4(inbx, chi, 4) * g[nx - 3];
      for (int i = 2; i <= nx; ++i) bb[i] = bb[i] + A3(icon, 1, i) * bb[i - 1];
      bb[nx] = bb[nx] * A3(icon, 2, nx);
      for (int i = nx - 1; i >= 1; --i) bb[i] = (bb[i] - A3(icon, 3, i) * bb[i + 1]) * A3(icon, 2, i);
      double *o = geni + (size_t)(k - 1) * nx - 1;
      for (int i = 1; i <= nx; ++i) o[i] = bb[i];
    }
    free(bb);
  }
}

/* difvisxx, lip.f90:52-142. which = 0: u (dcxu, vixu, cofcxu, cofvxu,
 * chv=1, vel=1); which = 1: v,w (dcxv, vixv, cofcxv, cofvxv, chv=2, vel=0).
 * result may alias upen_int. */
void orc_difvisxx(orc_box *b, const double *upen_int, const double *upencil,
                  double *result, int which, int nlin) {
  const int nx = b->nx;
  const double *icon = which == 0 ? CF(b, DCXU) : CF(b, DCXV);
  const double *iconv = which == 0 ? CF(b, VIXU) : CF(b, VIXV);
  const double *econ = which == 0 ? CF(b, COFCXU) : CF(b, COFCXV);
  const double *econv = which == 0 ? CF(b, COFVXU) : CF(b, COFVXV);
  const double *dcbx = CF(b, DCBX), *cofvbx = CF(b, COFVBX);
  const int chv = which == 0 ? 1 : 2, chv1 = chv + 2;
  const int ic = which == 0 ? 3 : 1;
  const double rex = SC(b, REX), idx = SC(b, IDX), uinf = SC(b, UINF);
#pragma omp parallel NTH
  {
    double *bb = (double *)malloc(sizeof(double) * (nx + 1));
    double *cv = (double *)malloc(sizeof(double) * (nx + 1));
#pragma omp for schedule(static)
    for (int k = 1; k <= nlin; ++k) {
      const double *g = upen_int + (size_t)(k - 1) * nx - 1;
      const double *up = upencil + (size_t)(k - 1) * nx - 1;
      for (int i = 2; i <= nx - 1; ++i) bb[i] = A2(econ, 1, i) * g[i - 1] + A2(econ, 2, i) * g[i];
      bb[1] = M5(dcbx, chv, 1) * g[1] + M5(dcbx, chv, 2) * g[2] + M5(dcbx, chv, 3) * g[3] +
              M5(dcbx, chv, 4) * g[4];
      bb[nx] = M5(dcbx, chv1, 1) * g[nx] + M5(dcbx, chv1, 2) * g[nx - 1] +
               M5(dcbx, chv1, 3) * g[nx - 2] + M5(dcbx, chv1, 4) * g[nx - 3];
      for (int j = 2; j <= nx; ++j) bb[j] = bb[j] + A3(icon, 1, j) * bb[j - 1];
      bb[nx] = bb[nx] * A3(icon, 2, nx);
      for (int j = nx - 1; j >= 1; --j) bb[j] = (bb[j] - A3(icon, 3, j) * bb[j + 1]) * A3(icon, 2, j);
      bb[nx] = uinf * (up[nx] - up[nx - 1]) * idx; /* outflow BC, lip.f90:105 */
      for (int i = 2; i <= nx - 1; ++i)
        cv[i] = A3(econv, 1, i) * up[i + 1] + A3(econv, 2, i) * up[i] + A3(econv, 3, i) * up[i - 1];
      cv[1] = M4(cofvbx, ic, 1) * up[1] + M4(cofvbx, ic, 2) * up[2] + M4(cofvbx, ic, 3) * up[3] +
              M4(cofvbx, ic, 4) * up[4];
      cv[nx] = M4(cofvbx, ic + 1, 1) * up[nx] + M4(cofvbx, ic + 1, 2) * up[nx - 1] +
               M4(cofvbx, ic + 1, 3) * up[nx - 2] + M4(cofvbx, ic + 1, 4) * up[nx - 3];
      for (int i = 2; i <= nx; ++i) cv[i] = cv[i] + A3(iconv, 1, i) * cv[i - 1];
      cv[nx] = cv[nx] * A3(iconv, 2, nx);
      for (int i = nx - 1; i >= 1; --i) cv[i] = (cv[i] - A3(iconv, 3, i) * cv[i + 1]) * A3(iconv, 2, i);
      cv[nx] = 0.0; /* inviscid outflow, lip.f90:132 */
      double *o = result + (size_t)(k - 1) * nx - 1;
      for (int i = 1; i <= nx; ++i) o[i] = bb[i] + rex * cv[i];
    }
    free(bb);
    free(cv);
  }
}

/* ---------------- y-line compact operators (one plane), lip.f90 ---------- */
/* interpyy, lip.f90:359-440. which = 0: u,w (inyu, cofiuy, loguv=0,
 * jee=ny+1); which = 1: v (inyv, cofivy, loguv=1, jee=ny).
 * gen(dim, jee), geni(dim, ny+1); rows 1..ny of geni are written. */
void orc_interpyy(orc_box *b, const double *gen, double *geni, int which, int dim, int m) {
  const int ny = b->ny;
  const double *icon = which == 0 ? CF(b, INYU) : CF(b, INYV);
  const double *econ = which == 0 ? CF(b, COFIUY) : CF(b, COFIVY);
  const double *inby = CF(b, INBY);
#define G(k, j) gen[(size_t)((j)-1) * dim + (k)-1]
#define GI(k, j) geni[(size_t)((j)-1) * dim + (k)-1]
  for (int k = 1; k <= m; ++k) {
    if (which == 0) {
      GI(k, 1) = 0.0;
      const double buf = M4(inby, 1, 1) * G(k, ny + 1) + M4(inby, 1, 2) * G(k, ny) +
                         M4(inby, 1, 3) * G(k, ny - 1) + M4(inby, 1, 4) * G(k, ny - 2);
      for (int j = 2; j <= ny - 1; ++j) GI(k, j) = A2(econ, 1, j) * G(k, j) + A2(econ, 2, j) * G(k, j + 1);
      GI(k, ny) = buf;
    } else {
      const double buf = M4(inby, 3, 1) * G(k, 1) + M4(inby, 3, 2) * G(k, 2) +
                         M4(inby, 3, 3) * G(k, 3) + M4(inby, 3, 4) * G(k, 4);
      GI(k, ny) = M4(inby, 4, 1) * G(k, ny) + M4(inby, 4, 2) * G(k, ny - 1) +
                  M4(inby, 4, 3) * G(k, ny - 2) + M4(inby, 4, 4) * G(k, ny - 3);
      for (int j = ny - 1; j >= 2; --j) GI(k, j) = A2(econ, 2, j) * G(k, j) + A2(econ, 1, j) * G(k, j - 1);
      GI(k, 1) = buf;
    }
    for (int j = 2; j <= ny; ++j) GI(k, j) = GI(k, j) + A3(icon, 1, j) * GI(k, j - 1);
    GI(k, ny) = GI(k, ny) * A3(icon, 2, ny);
    for (int j = ny - 1; j >= 1; --j) GI(k, j) = (GI(k, j) - A3(icon, 3, j) * GI(k, j + 1)) * A3(icon, 2, j);
  }
#undef G
#undef GI
}

/* differzy, lip.f90:152-232 (not in place). which = 0: u-type
 * (dcyu, cofcyu, chv=3, fwb1=-1, fwb2=0, jee=ny+1); which = 1: v-type
 * (dcyv, cofcyv, chv=1, fwb1=0, fwb2=1, jee=ny). geni (nz1, >=ny rows),
 * result (nz1, ny+1); rows 1..jee of result are written. */
void orc_differzy(orc_box *b, const double *geni, double *result, int which) {
  const int ny = b->ny, nz1 = b->nz1;
  const double *icon = which == 0 ? CF(b, DCYU) : CF(b, DCYV);
  const double *econ = which == 0 ? CF(b, COFCYU) : CF(b, COFCYV);
  const double *dcby = CF(b, DCBY);
  const int chv = which == 0 ? 3 : 1, cha = chv + 1;
  const int fwb1 = which == 0 ? -1 : 0, fwb2 = which == 0 ? 0 : 1;
  const int jee = which == 0 ? ny + 1 : ny;
#define G(k, j) geni[(size_t)((j)-1) * nz1 + (k)]
#define R(k, j) result[(size_t)((j)-1) * nz1 + (k)]
  for (int k = 0; k < nz1; ++k) {
    const double bot = M4(dcby, chv, 1) * G(k, 1) + M4(dcby, chv, 2) * G(k, 2) +
                       M4(dcby, chv, 3) * G(k, 3) + M4(dcby, chv, 4) * G(k, 4);
    const double top = M4(dcby, cha, 1) * G(k, ny) + M4(dcby, cha, 2) * G(k, ny - 1) +
                       M4(dcby, cha, 3) * G(k, ny - 2) + M4(dcby, cha, 4) * G(k, ny - 3);
    for (int j = 2; j <= jee - 1; ++j)
      R(k, j) = A2(econ, 2, j) * G(k, j + fwb2) + A2(econ, 1, j) * G(k, j + fwb1);
    R(k, 1) = bot;
    R(k, jee) = top;
    for (int j = 2; j <= jee; ++j) R(k, j) = R(k, j) + A3(icon, 1, j) * R(k, j - 1);
    R(k, jee) = R(k, jee) * A3(icon, 2, jee);
    for (int j = jee - 1; j >= 1; --j) R(k, j) = (R(k, j) - A3(icon, 3, j) * R(k, j + 1)) * A3(icon, 2, j);
  }
#undef G
#undef R
}

/* vistyy, lip.f90:447-513. which = 0: u,w (viyu, cofvyu, jee=ny+1, ic=3);
 * which = 1: v (viyv, cofvyv, jee=ny, ic=1). */
void orc_vistyy(orc_box *b, const double *u, double *result, int which) {
  const int ny = b->ny, nz1 = b->nz1;
  const double *icon = which == 0 ? CF(b, VIYU) : CF(b, VIYV);
  const double *econ = which == 0 ? CF(b, COFVYU) : CF(b, COFVYV);
  const double *cofvby = CF(b, COFVBY);
  const int jee = which == 0 ? ny + 1 : ny;
  const int ic = which == 0 ? 3 : 1;
#define U(k, j) u[(size_t)((j)-1) * nz1 + (k)]
#define R(k, j) result[(size_t)((j)-1) * nz1 + (k)]
  for (int k = 0; k < nz1; ++k) {
    R(k, 1) = M4(cofvby, ic, 1) * U(k, 1) + M4(cofvby, ic, 2) * U(k, 2) + M4(cofvby, ic, 3) * U(k, 3) +
              M4(cofvby, ic, 4) * U(k, 4);
    for (int j = 2; j <= jee - 1; ++j)
      R(k, j) = A3(econ, 1, j) * U(k, j + 1) + A3(econ, 2, j) * U(k, j) + A3(econ, 3, j) * U(k, j - 1);
    R(k, jee) = M4(cofvby, ic + 1, 1) * U(k, jee) + M4(cofvby, ic + 1, 2) * U(k, jee - 1) +
                M4(cofvby, ic + 1, 3) * U(k, jee - 2) + M4(cofvby, ic + 1, 4) * U(k, jee - 3);
    for (int j = 2; j <= jee; ++j) R(k, j) = R(k, j) + A3(icon, 1, j) * R(k, j - 1);
    R(k, jee) = R(k, jee) * A3(icon, 2, jee);
    for (int j = jee - 1; j >= 1; --j) R(k, j) = (R(k, j) - A3(icon, 3, j) * R(k, j + 1)) * A3(icon, 2, j);
  }
#undef U
#undef R
}

/* implzy, lip.f90:528-597: solves (A + var1*B) u = A res for rows
 * 2..jee-1 with the boundary rows 1 and jee of u kept. which = 0: u,w
 * (vyui, cofvyu, jee=ny+1); which = 1: v (vyvi, cofvyv, jee=ny). */
void orc_implzy(orc_box *b, double *u, const double *res, int which, double var1) {
  const int ny = b->ny, nz1 = b->nz1;
  const double *icon = which == 0 ? CF(b, VYUI) : CF(b, VYVI);
  const double *econ = which == 0 ? CF(b, COFVYU) : CF(b, COFVYV);
  const int jee = which == 0 ? ny + 1 : ny;
  double a1[1024 + 2], a2[1024 + 2], a3[1024 + 2];
#define U(k, j) u[(size_t)((j)-1) * nz1 + (k)]
#define RS(k, j) res[(size_t)((j)-1) * nz1 + (k)]
  for (int j = 2; j <= jee - 1; ++j) {
    for (int k = 0; k < nz1; ++k)
      U(k, j) = A3(icon, 1, j) * RS(k, j - 1) + A3(icon, 2, j) * RS(k, j) + A3(icon, 3, j) * RS(k, j + 1);
    a1[j] = A3(icon, 1, j) + var1 * A3(econ, 3, j);
    a2[j] = A3(icon, 2, j) + var1 * A3(econ, 2, j);
    a3[j] = A3(icon, 3, j) + var1 * A3(econ, 1, j);
  }
  for (int k = 0; k < nz1; ++k) U(k, 2) = U(k, 2) - a1[2] * U(k, 1);
  for (int k = 0; k < nz1; ++k) U(k, jee - 1) = U(k, jee - 1) - a3[jee - 1] * U(k, jee);
  a1[2] = 0.0;
  a3[jee - 1] = 0.0;
  for (int j = 3; j <= jee - 1; ++j) {
    const double d = 1.0 / a2[j - 1];
    a2[j - 1] = d;
    a1[j] = -a1[j] * d;
    a2[j] = a2[j] + a1[j] * a3[j - 1];
  }
  a2[jee - 1] = 1.0 / a2[jee - 1];
  for (int k = 0; k < nz1; ++k) {
    for (int j = 3; j <= jee - 1; ++j) U(k, j) = U(k, j) + a1[j] * U(k, j - 1);
    U(k, jee - 1) = U(k, jee - 1) * a2[jee - 1];
    for (int j = jee - 2; j >= 2; --j) U(k, j) = (U(k, j) - a3[j] * U(k, j + 1)) * a2[j];
  }
#undef U
#undef RS
}

/* fourxz, ffts.f90:27-67, on nlines independent lines */
void orc_fourxz(orc_box *b, double *fou, double *phys, int iopt, int nlines) {
  const int nz = b->nz, nz2 = b->nz2, nz1 = b->nz1;
#pragma omp parallel NTH
  {
    double *work = (double *)malloc(sizeof(double) * 8 * (size_t)(nz + 2));
#pragma omp for schedule(static)
    for (int l = 0; l < nlines; ++l) {
      if (iopt < 0)
        orc_r2c_line(b->fz, nz, nz2, phys + (size_t)l * (nz + 2), fou + (size_t)l * nz1, work);
      else
        orc_c2r_line(b->fz, nz, nz2, fou + (size_t)l * nz1, phys + (size_t)l * (nz + 2), work);
    }
    free(work);
  }
}

/* cosftx, ffts.f90:147-181, on pencils c(nx, nlines): elements 2..nx */
void orc_cosftx(orc_box *b, double *c, int nlines, int iopt) {
  const int nx = b->nx;
#pragma omp parallel NTH
  {
    double *work = (double *)malloc(sizeof(double) * 4 * (size_t)(nx + 2));
#pragma omp for schedule(static)
    for (int l = 0; l < nlines; ++l) orc_dct_line(b->fx, nx - 1, c + (size_t)l * nx + 1, iopt, work);
    free(work);
  }
}

/* ---------------- boundary conditions, boun.f90:7-56 ---------------- */
void orc_boun(orc_box *b) {
  const int nx = b->nx, ny = b->ny, nz1 = b->nz1;
  const double *inby = CF(b, INBY), *ccon = CF(b, CCON), *vmagic = CF(b, VMAGIC);
  double *u = b->f[OTBL_F_U], *v = b->f[OTBL_F_V], *w = b->f[OTBL_F_W];
#pragma omp parallel for NTH schedule(static)
  for (int i = 1; i <= nx; ++i) {
    double *v1 = PL(b, v, ny, i, 1), *vn = PL(b, v, ny, i, ny);
    for (int k = 0; k < nz1; ++k) {
      v1[k] = 0.0;
      vn[k] = 0.0;
    }
    vn[0] = vmagic[i - 1];
    double *fl[2] = {u, w};
    for (int f = 0; f < 2; ++f) {
      double *r1 = PL(b, fl[f], ny + 1, i, 1), *r2 = PL(b, fl[f], ny + 1, i, 2);
      double *r3 = PL(b, fl[f], ny + 1, i, 3), *r4 = PL(b, fl[f], ny + 1, i, 4);
      double *rn = PL(b, fl[f], ny + 1, i, ny), *rn1 = PL(b, fl[f], ny + 1, i, ny - 1);
      double *rn2 = PL(b, fl[f], ny + 1, i, ny - 2), *rt = PL(b, fl[f], ny + 1, i, ny + 1);
      for (int k = 0; k < nz1; ++k) {
        r1[k] = -1.0 / M4(inby, 2, 1) * (M4(inby, 2, 2) * r2[k] + M4(inby, 2, 3) * r3[k] + M4(inby, 2, 4) * r4[k]);
        rt[k] = -1.0 / M2(ccon, 1, 1) * (M2(ccon, 1, 2) * rn[k] + M2(ccon, 1, 3) * rn1[k] + M2(ccon, 1, 4) * rn2[k]);
      }
    }
  }
}

/* ---------------- inflow recycling, genflu.F90:3-242 (NEWGENFLU) -------- */
/* dobleu, genflu.F90:173-199 */
static void dobleu(const double *eta, double *www, double *www1, int n) {
  const double ag = 4.0, bg = 0.2, w1default = (double)0.7895f;
  const double bg2 = 1.0 - 2.0 * bg, tag = 1.0 / tanh(ag);
  *www1 = w1default;
  www[1] = 0.0;
  for (int i = 2; i <= n; ++i) {
    const double xxx = 0.5 * (eta[i] + eta[i - 1]);
    double yyy;
    if (xxx >= 1.0)
      yyy = 1.0;
    else
      yyy = 0.5 * (1.0 + tag * tanh(ag * (xxx - bg) / (bg2 * xxx + bg)));
    www[i] = www[i - 1] + yyy * (eta[i] - eta[i - 1]);
    if (eta[i] >= 1.0 && eta[i - 1] < 1.0) *www1 = www[i - 1] + (1.0 - eta[i - 1]) * yyy;
  }
}

/* profile, genflu.F90:204-242; ut is plane 1 of a field with n rows */
static void profile(orc_box *b, double *ut, double *wk, int ntop, const int *kl,
                    const double *fsca, int n) {
  const int ny = b->ny, nz1 = b->nz1;
  const double ggg = 1.0 / b->gamma1;
#define UT(k, j) ut[(size_t)((j)-1) * nz1 + (k)]
#define WK(k, j) wk[(size_t)((j)-1) * nz1 + (k)]
  if (n == ny + 1) {
    for (int i = 1; i <= ntop; ++i) {
      const int kll = kl[i];
      for (int k = 2; k <= nz1 - 1; ++k) WK(k, i + 1) = UT(k, kll + 2) * fsca[i] + UT(k, kll + 1) * (1 - fsca[i]);
    }
    for (int k = 2; k <= nz1 - 1; ++k) WK(k, 1) = -WK(k, 2);
  } else {
    for (int i = 1; i <= ntop; ++i) {
      const int kll = kl[i];
      for (int k = 2; k <= nz1 - 1; ++k) WK(k, i) = UT(k, kll + 1) * fsca[i] + UT(k, kll) * (1 - fsca[i]);
    }
  }
  for (int i = ntop - 2; i <= n; ++i)
    for (int k = 2; k <= nz1 - 1; ++k) WK(k, i) = WK(k, ntop - 3);
  for (int i = 1; i <= n; ++i)
    for (int k = 2; k <= nz1 - 1; ++k) UT(k, i) = WK(k, i) * ggg;
#undef UT
#undef WK
}

void orc_genflu(orc_box *b) {
  const int ny = b->ny, nz1 = b->nz1, xout = b->xout;
  const double *y = CF(b, Y), *dy = CF(b, DY);
  const double re = SC(b, RE), din = SC(b, DIN), rthin = SC(b, RTHIN), yb = SC(b, YBLEND);
  double *u = b->f[OTBL_F_U], *v = b->f[OTBL_F_V], *w = b->f[OTBL_F_W];
  const double dt = b->dt;
  const double tloc = b->tiempo - b->timeinit;
  /* bring the reference plane xout to plane 1, genflu.F90:43-52 */
  memcpy(PL(b, u, ny + 1, 1, 1), PL(b, u, ny + 1, xout, 1), sizeof(double) * (size_t)nz1 * (ny + 1));
  memcpy(PL(b, v, ny, 1, 1), PL(b, v, ny, xout, 1), sizeof(double) * (size_t)nz1 * ny);
  memcpy(PL(b, w, ny + 1, 1, 1), PL(b, w, ny + 1, xout, 1), sizeof(double) * (size_t)nz1 * (ny + 1));
  /* blend the fluctuations above y_blend, genflu.F90:55-60 */
  for (int j = 1; j <= ny + 1; ++j) {
    const double fblend = 0.5 * (1 - tanh(y[j] - yb));
    double *uj = PL(b, u, ny + 1, 1, j), *wj = PL(b, w, ny + 1, 1, j);
    for (int k = 2; k < nz1; ++k) {
      uj[k] = uj[k] * fblend;
      wj[k] = wj[k] * fblend;
    }
  }
  /* filtered mean profile, genflu.F90:67-76 */
  double timec;
  if (tloc < 20)
    timec = 20;
  else if (tloc < 100)
    timec = 100;
  else
    timec = tloc;
  b->timec = timec;
  double *um = b->um - 1; /* um(1:ny+1) */
  for (int j = 1; j <= ny + 1; ++j) um[j] = (dt / timec) * PL(b, u, ny + 1, 1, j)[0] + um[j] * (1.0 - dt / timec);
  b->utauout = sqrt(fabs((um[2] - um[1]) / (y[2] - y[1]) / re));
  /* momentum thickness, genflu.F90:79-87 */
  double uinf = 0.0;
  for (int j = ny + 1 - 20; j <= ny + 1 - 5; ++j) uinf += um[j];
  uinf = uinf / 16.0;
  const double u99 = (double)0.99f * uinf;
  int jtop = 0;
  for (int j = 1; j <= ny - 2; ++j) {
    if (um[j] >= u99) break;
    jtop = j + 1;
  }
  b->dout = y[jtop];
  double s = 0.0;
  for (int t = 0; t < jtop + 2; ++t) s += (uinf - um[2 + t]) * um[2 + t] * dy[1 + t];
  b->rthout = s * re / uinf;
  /* scaling factors, genflu.F90:92-93 */
  b->gamma2 = rthin / b->rthout;
  b->gamma1 = pow(b->gamma2, 0.125);
  /* rescaled grids and bisection, genflu.F90:110-138 */
  int ntop[3] = {0, 0, 0};
  int *kl = (int *)calloc(2 * (size_t)(ny + 1), sizeof(int));
  double *fsca = (double *)calloc(2 * (size_t)(ny + 1), sizeof(double));
  double *ysca = (double *)calloc((size_t)ny + 1, sizeof(double));
  double *wlwa = (double *)calloc((size_t)ny + 1, sizeof(double));
  for (int kk = 1; kk <= 2; ++kk) {
    for (int j = 1; j <= ny; ++j) ysca[j] = kk == 1 ? 5e-1 * (y[j] + y[j + 1]) / din : y[j] / din;
    double www1;
    dobleu(ysca, wlwa, &www1, ny);
    for (int j = 1; j <= ny; ++j)
      wlwa[j] = ysca[j] / b->gamma1 + (1.0 / b->gamma2 - 1.0 / b->gamma1) / www1 * wlwa[j];
    int kll = 1;
    int *klk = kl + (size_t)(kk - 1) * (ny + 1);
    double *fk = fsca + (size_t)(kk - 1) * (ny + 1);
    for (int i = 1; i <= ny; ++i) {
      if (wlwa[i] <= ysca[ny]) {
        ntop[kk] = i;
        int khh = ny;
        while (khh - kll > 1) {
          const int kx = (khh + kll) / 2;
          if (ysca[kx] >= wlwa[i])
            khh = kx;
          else
            kll = kx;
        }
        klk[i] = kll;
        fk[i] = (wlwa[i] - ysca[kll]) / (ysca[khh] - ysca[kll]);
      }
    }
  }
  /* the zero mode and the rescaled fluctuations, genflu.F90:146-154 */
  for (int j = 1; j <= ny + 1; ++j) {
    double *uj = PL(b, u, ny + 1, 1, j), *wj = PL(b, w, ny + 1, 1, j);
    uj[0] = b->u0[j - 1];
    uj[1] = 0.0;
    wj[0] = 0.0;
    wj[1] = 0.0;
  }
  for (int j = 1; j <= ny; ++j) {
    double *vj = PL(b, v, ny, 1, j);
    vj[0] = b->v0[j - 1];
    vj[1] = 0.0;
  }
  double *wk = (double *)calloc((size_t)nz1 * (ny + 2), sizeof(double));
  if (ntop[1] >= 4 && ntop[2] >= 4) { /* guard: degenerate rescaled grids */
    profile(b, PL(b, u, ny + 1, 1, 1), wk, ntop[1], kl, fsca, ny + 1);
    profile(b, PL(b, w, ny + 1, 1, 1), wk, ntop[1], kl, fsca, ny + 1);
    profile(b, PL(b, v, ny, 1, 1), wk, ntop[2], kl + (ny + 1), fsca + (ny + 1), ny);
  }
  free(wk);
  free(kl);
  free(fsca);
  free(ysca);
  free(wlwa);
}

/* ---------------- rhsp, rhsp.F90:22-489 ---------------- */
static inline void cmul_kaz(double kz, const double *a, double *out_re, double *out_im) {
  /* a * kaz with kaz = (0, kz) */
  *out_re = -a[1] * kz;
  *out_im = a[0] * kz;
}

/* energies (rhsp.F90:493-509): ministats (stotf.F90:395-440) on every
 * plane in order, here the whole box in one domain, so the allreduce is the
 * identity. Plane 1 sets uner(1:3); plane nx/2 (integer division) sets
 * uner(4:15) and then overwrites uner(1:3), each row of aux adding
 * Re(u(0,1))^2 as written at stotf.F90:433-435. Sums run over j in order. */
static void orc_energies(orc_box *b) {
  const int nx = b->nx, ny = b->ny, nz1 = b->nz1, nz2 = b->nz2;
  const double *hy = CF(b, HY);
  double uner[15] = {0};
  for (int i = 1; i <= nx; ++i) {
    if (i != 1 && i != nx / 2) continue;
    for (int f = 0; f < 3; ++f) {
      const int jee = f == 1 ? ny : ny + 1;
      const double *g = b->f[f == 0 ? OTBL_F_U : (f == 1 ? OTBL_F_V : OTBL_F_W)] + (size_t)(i - 1) * jee * nz1;
      if (i == 1) { /* stotf.F90:406-414 */
        double e = 0.0;
        for (int j = 0; j < jee; ++j) {
          double a = 0.0;
          for (int k = 0; k <= nz2; ++k) a += g[(size_t)j * nz1 + 2 * k] * g[(size_t)j * nz1 + 2 * k] +
                                            g[(size_t)j * nz1 + 2 * k + 1] * g[(size_t)j * nz1 + 2 * k + 1];
          e += a * hy[j];
        }
        uner[f] = e;
      }
      if (i == nx / 2) { /* stotf.F90:417-438 */
        const double r1 = g[0];
        double e = 0.0, a01[2] = {0.0, 0.0};
        for (int j = 0; j < jee; ++j) {
          double s = 0.0;
          for (int k = 1; k <= nz2; ++k) s += g[(size_t)j * nz1 + 2 * k] * g[(size_t)j * nz1 + 2 * k] +
                                            g[(size_t)j * nz1 + 2 * k + 1] * g[(size_t)j * nz1 + 2 * k + 1];
          const double a = 2.0 * s;
          if (j < 2) a01[j] = a;
          e += (a + r1 * r1) * hy[j];
        }
        uner[3 + 4 * f] = g[0];
        uner[4 + 4 * f] = g[nz1];
        uner[5 + 4 * f] = a01[0];
        uner[6 + 4 * f] = a01[1];
        uner[f] = e;
      }
    }
  }
  memcpy(b->ener, uner, sizeof uner);
}

void orc_get_energies(orc_box *b, double *ener) { memcpy(ener, b->ener, sizeof(double) * 15); }

int orc_rhsp(orc_box *b, int m, int setstep) {
  const int nx = b->nx, ny = b->ny, nz = b->nz, nz1 = b->nz1, nz2 = b->nz2;
  const int mpu = nz1 * (ny + 1), mpv = nz1 * ny;
  double *u = b->f[OTBL_F_U], *v = b->f[OTBL_F_V], *w = b->f[OTBL_F_W], *p = b->f[OTBL_F_P];
  double *rhsupa = b->f[OTBL_F_RHSUPA], *rhsvpa = b->f[OTBL_F_RHSVPA], *rhswpa = b->f[OTBL_F_RHSWPA];
  double *rhsu = b->rhsu, *rhsv = b->rhsv, *rhsw = b->rhsw;
  double *wk1 = b->wk1, *wk2 = b->wk2, *wk3 = b->wk3;
  const double *kaz = CF(b, KAZ), *kvis = CF(b, KVIS);
  const double *idyy = CF(b, IDYY), *dymin = CF(b, DYMIN);
  const double *inby = CF(b, INBY);
  const int nth = orc_get_threads();

  if (m == 1) orc_energies(b); /* rhsp.F90:116, on the state rhsp was called on */

  /* planes -> pencils and x-interpolation, rhsp.F90:67-69,105-112 */
  orc_chp2x(b, b->penu, u, ny + 1);
  orc_chp2x(b, b->penv, v, ny);
  orc_chp2x(b, b->penw, w, ny + 1);
  orc_interpxx(b, b->penu, b->pen, 0, mpu);
  orc_chx2p(b, b->pen, wk1, ny + 1);
  orc_interpxx(b, b->penv, b->pen, 1, mpv);
  orc_chx2p(b, b->pen, wk2, ny);
  orc_interpxx(b, b->penw, b->pen, 1, mpu);
  orc_chx2p(b, b->pen, wk3, ny + 1);

  /* zy-plane loop for the terms that need d/dx, rhsp.F90:120-171 */
  double um = -1e14f, wm = -1e14f;
  double *vmt = (double *)malloc(sizeof(double) * (size_t)nth * (ny + 1));
  for (int t = 0; t < nth * (ny + 1); ++t) vmt[t] = -1e14f;
  double *umt = (double *)malloc(sizeof(double) * nth), *wmt = (double *)malloc(sizeof(double) * nth);
  for (int t = 0; t < nth; ++t) umt[t] = wmt[t] = -1e14f;
#pragma omp parallel NTH
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    const int ldp = nz + 2;
    double *wkp = (double *)malloc(sizeof(double) * (size_t)ldp * (ny + 2));
    double *wkpo = (double *)malloc(sizeof(double) * (size_t)ldp * (ny + 2));
    double *wkf = (double *)malloc(sizeof(double) * (size_t)nz1 * (ny + 2));
    double *t = (double *)malloc(sizeof(double) * (size_t)ldp);
    double *work = (double *)malloc(sizeof(double) * 8 * (size_t)ldp);
    double *vml = vmt + (size_t)tid * (ny + 1);
#pragma omp for schedule(static)
    for (int i = 1; i <= nx; ++i) {
      for (int j = 1; j <= ny + 1; ++j)
        orc_c2r_line(b->fz, nz, nz2, PL(b, u, ny + 1, i, j), wkp + (size_t)(j - 1) * ldp, work);
      if (setstep)
        for (int j = 1; j <= ny + 1; ++j)
          for (int k = 0; k < nz; ++k) umt[tid] = fmax(umt[tid], fabs(wkp[(size_t)(j - 1) * ldp + k]));
      for (int j = 1; j <= ny + 1; ++j) {
        double *a1 = PL(b, wk1, ny + 1, i, j), *a3 = PL(b, wk3, ny + 1, i, j);
        orc_c2r_line(b->fz, nz, nz2, a1, t, work);
        for (int k = 0; k < nz; ++k) t[k] = t[k] * t[k];
        orc_r2c_line(b->fz, nz, nz2, t, a1, work);
        orc_c2r_line(b->fz, nz, nz2, a3, t, work);
        if (setstep)
          for (int k = 0; k < nz; ++k) wmt[tid] = fmax(wmt[tid], fabs(t[k]));
        for (int k = 0; k < nz; ++k) t[k] = t[k] * wkp[(size_t)(j - 1) * ldp + k];
        orc_r2c_line(b->fz, nz, nz2, t, a3, work);
      }
      orc_interpyy(b, wkp, wkpo, 0, ldp, nz);
      for (int j = 1; j <= ny; ++j) {
        double *a2 = PL(b, wk2, ny, i, j);
        orc_c2r_line(b->fz, nz, nz2, a2, t, work);
        if (setstep)
          for (int k = 0; k < nz; ++k) vml[j] = fmax(vml[j], fabs(t[k]));
        for (int k = 0; k < nz; ++k) t[k] = t[k] * wkpo[(size_t)(j - 1) * ldp + k];
        orc_r2c_line(b->fz, nz, nz2, t, a2, work);
      }
      orc_differzy(b, PL(b, wk2, ny, i, 1), wkf, 0);
      for (int j = 1; j <= ny + 1; ++j) {
        double *r = PL(b, rhsu, ny + 1, i, j);
        const double *a3 = PL(b, wk3, ny + 1, i, j), *f = wkf + (size_t)(j - 1) * nz1;
        for (int k = 0; k <= nz2; ++k) {
          double re, im;
          cmul_kaz(kaz[k], a3 + 2 * k, &re, &im);
          r[2 * k] = f[2 * k] + re;
          r[2 * k + 1] = f[2 * k + 1] + im;
        }
      }
    }
    free(wkp); free(wkpo); free(wkf); free(t); free(work);
  }
  double *vm = (double *)malloc(sizeof(double) * (ny + 1));
  for (int j = 1; j <= ny; ++j) {
    vm[j] = -1e14f;
    for (int t = 0; t < nth; ++t) vm[j] = fmax(vm[j], vmt[(size_t)t * (ny + 1) + j]);
  }
  for (int t = 0; t < nth; ++t) {
    um = fmax(um, umt[t]);
    wm = fmax(wm, wmt[t]);
  }
  free(vmt); free(umt); free(wmt);

  /* x-derivatives of the products + x-viscous terms, rhsp.F90:181-193 */
  orc_chp2x(b, b->pen, wk1, ny + 1);
  orc_difvisxx(b, b->pen, b->penu, b->pen, 0, mpu);
  orc_chx2p(b, b->pen, wk1, ny + 1);
  orc_chp2x(b, b->pen, wk2, ny);
  orc_difvisxx(b, b->pen, b->penv, b->pen, 1, mpv);
  orc_chx2p(b, b->pen, wk2, ny);
  orc_chp2x(b, b->pen, wk3, ny + 1);
  orc_difvisxx(b, b->pen, b->penw, b->pen, 1, mpu);
  orc_chx2p(b, b->pen, wk3, ny + 1);

  /* complete the RHS, rhsp.F90:199-204 */
  {
    const size_t lu = (size_t)nx * mpu, lv = (size_t)nx * mpv;
    for (size_t t = 0; t < lu; ++t) rhsu[t] = rhsu[t] + wk1[t];
    memcpy(rhsv, wk2, sizeof(double) * lv);
    memcpy(rhsw, wk3, sizeof(double) * lu);
    memcpy(PL(b, rhsu, ny + 1, nx, 1), PL(b, wk1, ny + 1, nx, 1), sizeof(double) * (size_t)mpu);
  }

  /* time step, rhsp.F90:214-262 */
  if (setstep) {
    const double poco = 1e-7;
    const double dt1 = SC(b, DXMIN) / fmax(poco, um);
    const double dt2 = SC(b, DXMIN) / fmax(poco, wm);
    double dt3 = 1e300;
    double vmax = -1e300;
    for (int j = 1; j <= ny; ++j) {
      dt3 = fmin(dt3, dymin[j - 1] / fmax(poco, vm[j]));
      vmax = fmax(vmax, vm[j]);
    }
    const double dtloc = fmin(fmin(dt1, dt2), fmin(dt3, SC(b, DTRET)));
    b->umax = um;
    b->wmax = wm;
    b->vmax = vmax;
    if (b->dt_mode == OTBL_DT_ADAPTIVE) {
      b->dt = dtloc;
    } else if (!b->dt_frozen) {
      b->dt = b->dt_fixed > 0.0 ? b->dt_fixed : dtloc;
      b->dt_frozen = 1;
    }
  }
  free(vm);
  if (!(b->dt > 0.0) || !isfinite(b->dt)) return OTBL_ERR_NAN;
  const double dt = b->dt;
  const double var1 = dt * (SC(b, RKCV + m - 1) + SC(b, RKDV + m - 1));
  double var2 = dt * SC(b, REX) * SC(b, RKCV + m - 1);
  const double var3 = dt * SC(b, RKC + m - 1);
  const double var4 = dt * SC(b, RKD + m - 1);

  /* save the velocities, rhsp.F90:281-285 */
  memcpy(b->resu, u, sizeof(double) * (size_t)nx * mpu);
  memcpy(b->resv, v, sizeof(double) * (size_t)nx * mpv);
  memcpy(b->resw, w, sizeof(double) * (size_t)nx * mpu);

  orc_genflu(b);

  /* pressure gradient, rhsp.F90:291-339 */
  const double idxx = SC(b, IDXX);
#pragma omp parallel for NTH schedule(static)
  for (int i = 2; i <= nx; ++i) {
    if (i <= nx - 1)
      for (int j = 2; j <= ny; ++j) {
        double *uj = PL(b, u, ny + 1, i, j);
        const double *p1 = PL(b, p, ny, i + 1, j), *p0 = PL(b, p, ny, i, j);
        for (int k = 0; k < nz1; ++k) uj[k] = uj[k] - var1 * idxx * (p1[k] - p0[k]);
      }
    for (int j = 2; j <= ny; ++j) {
      double *wj = PL(b, w, ny + 1, i, j);
      const double *pj = PL(b, p, ny, i, j);
      if (j <= ny - 1) {
        double *vj = PL(b, v, ny, i, j);
        const double *pj1 = PL(b, p, ny, i, j + 1);
        for (int k = 0; k < nz1; ++k) vj[k] = vj[k] - var1 * idyy[j - 1] * (pj1[k] - pj[k]);
      }
      for (int k = 0; k <= nz2; ++k) {
        const double a = var1 * kaz[k];
        const double re = -a * pj[2 * k + 1], im = a * pj[2 * k];
        wj[2 * k] = wj[2 * k] - re;
        wj[2 * k + 1] = wj[2 * k + 1] - im;
      }
    }
  }

  /* rest of the RHS (z viscous terms and the vw, vv, ww products),
   * rhsp.F90:351-418, planes 2..nx-1 */
#pragma omp parallel NTH
  {
    const int ldp = nz + 2;
    double *wkpo = (double *)malloc(sizeof(double) * (size_t)ldp * (ny + 2));
    double *wkp = (double *)malloc(sizeof(double) * (size_t)ldp * (ny + 2));
    double *wkf = (double *)malloc(sizeof(double) * (size_t)nz1 * (ny + 2));
    double *wkfo = (double *)malloc(sizeof(double) * (size_t)nz1 * (ny + 2));
    double *t = (double *)malloc(sizeof(double) * (size_t)ldp);
    double *work = (double *)malloc(sizeof(double) * 8 * (size_t)ldp);
#pragma omp for schedule(static)
    for (int i = 2; i <= nx - 1; ++i) {
      for (int j = 2; j <= ny; ++j) {
        double *ru = PL(b, rhsu, ny + 1, i, j), *rw = PL(b, rhsw, ny + 1, i, j);
        const double *su = PL(b, b->resu, ny + 1, i, j), *sw = PL(b, b->resw, ny + 1, i, j);
        for (int k = 0; k <= nz2; ++k)
          for (int c = 0; c < 2; ++c) {
            ru[2 * k + c] = ru[2 * k + c] - su[2 * k + c] * kvis[k];
            rw[2 * k + c] = rw[2 * k + c] - sw[2 * k + c] * kvis[k];
          }
        if (j <= ny - 1) {
          double *rv = PL(b, rhsv, ny, i, j);
          const double *sv = PL(b, b->resv, ny, i, j);
          for (int k = 0; k <= nz2; ++k)
            for (int c = 0; c < 2; ++c) rv[2 * k + c] = rv[2 * k + c] - sv[2 * k + c] * kvis[k];
        }
      }
      /* w interpolated in y, vw at v points */
      orc_interpyy(b, PL(b, b->resw, ny + 1, i, 1), wkf, 0, nz1, nz1);
      for (int j = 1; j <= ny; ++j) orc_c2r_line(b->fz, nz, nz2, wkf + (size_t)(j - 1) * nz1, wkpo + (size_t)(j - 1) * ldp, work);
      for (int j = 1; j <= ny; ++j) {
        orc_c2r_line(b->fz, nz, nz2, PL(b, b->resv, ny, i, j), t, work);
        for (int k = 0; k < nz; ++k) wkp[(size_t)(j - 1) * ldp + k] = t[k] * wkpo[(size_t)(j - 1) * ldp + k];
      }
      for (int j = 1; j <= ny; ++j) orc_r2c_line(b->fz, nz, nz2, wkp + (size_t)(j - 1) * ldp, wkfo + (size_t)(j - 1) * nz1, work);
      for (int j = 1; j <= ny; ++j) {
        double *rv = PL(b, rhsv, ny, i, j);
        const double *f = wkfo + (size_t)(j - 1) * nz1;
        for (int k = 0; k <= nz2; ++k) {
          double re, im;
          cmul_kaz(kaz[k], f + 2 * k, &re, &im);
          rv[2 * k] = rv[2 * k] + re;
          rv[2 * k + 1] = rv[2 * k + 1] + im;
        }
      }
      orc_differzy(b, wkfo, wkf, 0);
      for (int j = 1; j <= ny + 1; ++j) {
        double *rw = PL(b, rhsw, ny + 1, i, j);
        const double *f = wkf + (size_t)(j - 1) * nz1;
        for (int k = 0; k < nz1; ++k) rw[k] = rw[k] + f[k];
      }
      /* vv */
      orc_interpyy(b, PL(b, b->resv, ny, i, 1), wkf, 1, nz1, nz1);
      for (int j = 1; j <= ny; ++j) orc_c2r_line(b->fz, nz, nz2, wkf + (size_t)(j - 1) * nz1, wkpo + (size_t)(j - 1) * ldp, work);
      for (int j = 1; j <= ny; ++j)
        for (int k = 0; k < nz; ++k) {
          const double q = wkpo[(size_t)(j - 1) * ldp + k];
          wkp[(size_t)(j - 1) * ldp + k] = q * q;
        }
      for (int j = 1; j <= ny; ++j) orc_r2c_line(b->fz, nz, nz2, wkp + (size_t)(j - 1) * ldp, wkfo + (size_t)(j - 1) * nz1, work);
      orc_differzy(b, wkfo, wkf, 1);
      for (int j = 1; j <= ny; ++j) {
        double *rv = PL(b, rhsv, ny, i, j);
        const double *f = wkf + (size_t)(j - 1) * nz1;
        for (int k = 0; k < nz1; ++k) rv[k] = rv[k] + f[k];
        /* ww */
        orc_c2r_line(b->fz, nz, nz2, PL(b, b->resw, ny + 1, i, j), t, work);
        for (int k = 0; k < nz; ++k) t[k] = t[k] * t[k];
        double *g = wkf + (size_t)(j - 1) * nz1;
        orc_r2c_line(b->fz, nz, nz2, t, g, work);
        double *rw = PL(b, rhsw, ny + 1, i, j);
        for (int k = 0; k <= nz2; ++k) {
          double re, im;
          cmul_kaz(kaz[k], g + 2 * k, &re, &im);
          rw[2 * k] = rw[2 * k] + re;
          rw[2 * k + 1] = rw[2 * k + 1] + im;
        }
      }
    }
    free(wkpo); free(wkp); free(wkf); free(wkfo); free(t); free(work);
  }

  orc_boun(b);

  /* RHS boundary rows, rhsp.F90:423-445 */
  memset(PL(b, rhsu, ny + 1, 1, 1), 0, sizeof(double) * (size_t)mpu);
  memset(PL(b, rhsv, ny, 1, 1), 0, sizeof(double) * (size_t)mpv);
  memset(PL(b, rhsw, ny + 1, 1, 1), 0, sizeof(double) * (size_t)mpu);
#pragma omp parallel for NTH schedule(static)
  for (int i = 1; i <= nx; ++i) {
    memset(PL(b, rhsv, ny, i, 1), 0, sizeof(double) * nz1);
    memset(PL(b, rhsv, ny, i, ny), 0, sizeof(double) * nz1);
    double *fl[2] = {rhsu, rhsw};
    for (int f = 0; f < 2; ++f) {
      double *r1 = PL(b, fl[f], ny + 1, i, 1), *r2 = PL(b, fl[f], ny + 1, i, 2);
      double *r3 = PL(b, fl[f], ny + 1, i, 3), *r4 = PL(b, fl[f], ny + 1, i, 4);
      double *rt = PL(b, fl[f], ny + 1, i, ny + 1);
      for (int k = 0; k < nz1; ++k) {
        r1[k] = -1.0 / M4(inby, 2, 1) * (M4(inby, 2, 2) * r2[k] + M4(inby, 2, 3) * r3[k] + M4(inby, 2, 4) * r4[k]);
        rt[k] = 0.0;
      }
    }
  }

  /* explicit y-viscous terms and the RK combination, rhsp.F90:448-470 */
  const double var2_in = var2;
#pragma omp parallel NTH
  {
    double *wkf = (double *)malloc(sizeof(double) * (size_t)nz1 * (ny + 2));
#pragma omp for schedule(static)
    for (int i = 2; i <= nx; ++i) {
      const double v2 = (i == nx) ? 0.0 : var2_in;
      orc_vistyy(b, PL(b, b->resv, ny, i, 1), wkf, 1);
      for (int j = 1; j <= ny; ++j) {
        double *o = PL(b, wk2, ny, i, j);
        const double *a = PL(b, v, ny, i, j), *r = PL(b, rhsv, ny, i, j), *q = PL(b, rhsvpa, ny, i, j);
        const double *f = wkf + (size_t)(j - 1) * nz1;
        for (int k = 0; k < nz1; ++k) o[k] = a[k] - (var3 * r[k] + v2 * f[k] + var4 * q[k]);
      }
      orc_vistyy(b, PL(b, b->resu, ny + 1, i, 1), wkf, 0);
      for (int j = 1; j <= ny + 1; ++j) {
        double *o = PL(b, wk1, ny + 1, i, j);
        const double *a = PL(b, u, ny + 1, i, j), *r = PL(b, rhsu, ny + 1, i, j), *q = PL(b, rhsupa, ny + 1, i, j);
        const double *f = wkf + (size_t)(j - 1) * nz1;
        for (int k = 0; k < nz1; ++k) o[k] = a[k] - (var3 * r[k] + v2 * f[k] + var4 * q[k]);
      }
      orc_vistyy(b, PL(b, b->resw, ny + 1, i, 1), wkf, 0);
      for (int j = 1; j <= ny + 1; ++j) {
        double *o = PL(b, wk3, ny + 1, i, j);
        const double *a = PL(b, w, ny + 1, i, j), *r = PL(b, rhsw, ny + 1, i, j), *q = PL(b, rhswpa, ny + 1, i, j);
        const double *f = wkf + (size_t)(j - 1) * nz1;
        for (int k = 0; k < nz1; ++k) o[k] = a[k] - (var3 * r[k] + v2 * f[k] + var4 * q[k]);
      }
    }
    free(wkf);
  }
  (void)var2;
  memcpy(rhsupa, rhsu, sizeof(double) * (size_t)nx * mpu);
  memcpy(rhsvpa, rhsv, sizeof(double) * (size_t)nx * mpv);
  memcpy(rhswpa, rhsw, sizeof(double) * (size_t)nx * mpu);

  /* implicit y-viscous step, rhsp.F90:479-484 */
  const double rkk = SC(b, REX) * dt * SC(b, RKDV + m - 1);
#pragma omp parallel for NTH schedule(static)
  for (int i = 2; i <= nx; ++i) {
    orc_implzy(b, PL(b, u, ny + 1, i, 1), PL(b, wk1, ny + 1, i, 1), 0, rkk);
    orc_implzy(b, PL(b, v, ny, i, 1), PL(b, wk2, ny, i, 1), 1, rkk);
    orc_implzy(b, PL(b, w, ny + 1, i, 1), PL(b, wk3, ny + 1, i, 1), 0, rkk);
  }
  b->ener[12] = b->ener[13] = b->ener[14] = 0.0; /* rhsp.F90:487 */
  return OTBL_OK;
}

/* ---------------- outflow mass correction, boun.f90:63-93 ---------------- */
void orc_outflow_correction(orc_box *b) {
  const int nx = b->nx, ny = b->ny;
  const double *dy = CF(b, DY), *y = CF(b, Y);
  double *u = b->f[OTBL_F_U], *v = b->f[OTBL_F_V], *rp = b->f[OTBL_F_RHSUPA];
  double sv = 0.0;
  for (int i = 2; i <= nx; ++i) sv += PL(b, v, ny, i, ny)[0];
  double sumax = sv * SC(b, DX1);
  double s1 = 0.0, s2 = 0.0;
  for (int j = 2; j <= ny; ++j) s1 += PL(b, u, ny + 1, 1, j)[0] * dy[j - 1];
  sumax = sumax - s1;
  for (int j = 2; j <= ny; ++j) s2 += PL(b, u, ny + 1, nx, j)[0] * dy[j - 1];
  sumax = sumax + s2;
  const double alpha = -sumax / (y[ny] - y[1]);
  for (int j = 2; j <= ny; ++j) {
    PL(b, u, ny + 1, nx, j)[0] = PL(b, u, ny + 1, nx, j)[0] + alpha;
    PL(b, rp, ny + 1, nx, j)[0] = PL(b, rp, ny + 1, nx, j)[0] + alpha * SC(b, IDX);
  }
}

/* ---------------- divergence, pois.f90:41-54 ---------------- */
void orc_divergence(orc_box *b, double *rest) {
  const int nx = b->nx, ny = b->ny, nz1 = b->nz1, nz2 = b->nz2;
  const double *kaz = CF(b, KAZ), *idy = CF(b, IDY);
  const double idx = SC(b, IDX);
  double *u = b->f[OTBL_F_U], *v = b->f[OTBL_F_V], *w = b->f[OTBL_F_W];
  memset(rest, 0, sizeof(double) * otbl_field_len(nx, ny, b->nz, 0));
#pragma omp parallel for NTH schedule(static)
  for (int i = 2; i <= nx; ++i)
    for (int j = 1; j <= ny - 1; ++j) {
      double *r = PL(b, rest, ny, i, j);
      const double *w1 = PL(b, w, ny + 1, i, j + 1), *v1 = PL(b, v, ny, i, j + 1), *v0 = PL(b, v, ny, i, j);
      const double *ua = PL(b, u, ny + 1, i, j + 1), *ub = PL(b, u, ny + 1, i - 1, j + 1);
      for (int k = 0; k <= nz2; ++k) {
        double re, im;
        cmul_kaz(kaz[k], w1 + 2 * k, &re, &im);
        r[2 * k] = re + (v1[2 * k] - v0[2 * k]) * idy[j];
        r[2 * k + 1] = im + (v1[2 * k + 1] - v0[2 * k + 1]) * idy[j];
      }
      for (int k = 0; k < nz1; ++k) r[k] = r[k] + idx * (ua[k] - ub[k]);
    }
}

/* ---------------- pressure Poisson + projection, pois.f90:11-239 -------- */
void orc_pois(orc_box *b, int m) {
  const int nx = b->nx, ny = b->ny, nz1 = b->nz1, nz2 = b->nz2;
  const int mpv = nz1 * ny;
  double *u = b->f[OTBL_F_U], *v = b->f[OTBL_F_V], *w = b->f[OTBL_F_W], *p = b->f[OTBL_F_P];
  const double *kaz = CF(b, KAZ), *kaz2 = CF(b, KAZ2), *kmod = CF(b, KMOD);
  const double *ayp = CF(b, AYP), *idyy = CF(b, IDYY);
  const double idxx = SC(b, IDXX);
  const double varstep = 5e-1 / b->dt / SC(b, RKDV + m - 1); /* bl_1.F90:117 */
  double *rest = b->resu; /* any plane-sized scratch */

  orc_divergence(b, rest);
  orc_chp2x(b, b->pen, rest, ny);
  orc_cosftx(b, b->pen, mpv, -1);
  orc_chx2p(b, b->pen, rest, ny);
  /* mode 0 forced real, pois.f90:102 */
  for (int i = 1; i <= nx; ++i)
    for (int j = 1; j <= ny; ++j) PL(b, rest, ny, i, j)[1] = 0.0;

  /* tridiagonal in y per (x-mode, kz), pois.f90:106-117 + soltriy 211-239 */
  const int ny1 = ny - 1;
#pragma omp parallel NTH
  {
    double *a = (double *)malloc(sizeof(double) * 3 * (size_t)(ny + 1));
#pragma omp for schedule(static)
    for (int i = 2; i <= nx; ++i) {
      for (int k = 0; k <= nz2; ++k) {
        for (int j = 1; j <= ny1; ++j) {
          A3(a, 1, j) = A3(ayp, 1, j);
          A3(a, 2, j) = A3(ayp, 2, j) - kaz2[k] - kmod[i - 2];
          A3(a, 3, j) = A3(ayp, 3, j);
        }
        if (i == 2 && k == 0) {
          A3(a, 2, ny1) = 2.0 * A3(ayp, 2, ny1);
          PL(b, rest, ny, 2, ny1)[0] = 0.0;
          PL(b, rest, ny, 2, ny1)[1] = 0.0;
        }
        for (int j = 2; j <= ny1; ++j) {
          const double d = 1.0 / A3(a, 2, j - 1);
          A3(a, 2, j - 1) = d;
          A3(a, 1, j) = -A3(a, 1, j) * d;
          A3(a, 2, j) = A3(a, 2, j) + A3(a, 1, j) * A3(a, 3, j - 1);
        }
        A3(a, 2, ny1) = 1.0 / A3(a, 2, ny1);
        for (int c = 0; c < 2; ++c) {
#define US(j) PL(b, rest, ny, i, j)[2 * k + c]
          for (int j = 2; j <= ny1; ++j) US(j) = US(j) + A3(a, 1, j) * US(j - 1);
          US(ny1) = US(ny1) * A3(a, 2, ny1);
          for (int j = ny1 - 1; j >= 1; --j) US(j) = (US(j) - A3(a, 3, j) * US(j + 1)) * A3(a, 2, j);
#undef US
        }
      }
    }
    free(a);
  }

  orc_chp2x(b, b->pen, rest, ny);
  orc_cosftx(b, b->pen, mpv, 1);
  orc_chx2p(b, b->pen, rest, ny);

  /* projection, pois.f90:144-162 */
#pragma omp parallel for NTH schedule(static)
  for (int i = 2; i <= nx; ++i) {
    for (int j = 2; j <= ny; ++j) {
      double *pj = PL(b, p, ny, i, j), *wj = PL(b, w, ny + 1, i, j);
      const double *r = PL(b, rest, ny, i, j - 1);
      for (int k = 0; k < nz1; ++k) pj[k] = varstep * r[k] + pj[k];
      for (int k = 0; k <= nz2; ++k) {
        double re, im;
        cmul_kaz(kaz[k], r + 2 * k, &re, &im);
        wj[2 * k] = wj[2 * k] - re;
        wj[2 * k + 1] = wj[2 * k + 1] - im;
      }
    }
    for (int j = 2; j <= ny - 1; ++j) {
      double *vj = PL(b, v, ny, i, j);
      const double *r1 = PL(b, rest, ny, i, j), *r0 = PL(b, rest, ny, i, j - 1);
      for (int k = 0; k < nz1; ++k) vj[k] = vj[k] - idyy[j - 1] * (r1[k] - r0[k]);
    }
  }
#pragma omp parallel for NTH schedule(static)
  for (int i = 2; i <= nx - 1; ++i)
    for (int j = 1; j <= ny - 1; ++j) {
      double *uj = PL(b, u, ny + 1, i, j + 1);
      const double *r1 = PL(b, rest, ny, i + 1, j), *r0 = PL(b, rest, ny, i, j);
      for (int k = 0; k < nz1; ++k) uj[k] = uj[k] - idxx * (r1[k] - r0[k]);
    }
}

int orc_substep(orc_box *b, int m, int setstep) {
  const int st = orc_rhsp(b, m, setstep);
  if (st != OTBL_OK) return st;
  orc_outflow_correction(b);
  orc_pois(b, m);
  return OTBL_OK;
}

/* bl_1.F90:85-128 without I/O */
int orc_advance(orc_box *b, int nsteps) {
  for (int s = 0; s < nsteps; ++s) {
    for (int m = 1; m <= 3; ++m) {
      const int st = orc_substep(b, m, m == 1);
      if (st != OTBL_OK) return st;
    }
    b->tiempo = b->tiempo + b->dt;
  }
  return OTBL_OK;
}
