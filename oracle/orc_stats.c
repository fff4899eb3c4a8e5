/*
 * ORACLE -- test infrastructure, never part of the product path.
 *
 * The one-point statistics of the reference as rhsp computes them when
 * dostat is set (rhsp.F90:70-101) and statsp accumulates them
 * (stotf.F90:51-291): the x pre-pass (interpx_new of u shifted by one plane,
 * diffx_inplace of u_x, v, w; lip.f90:703-765), then per streamwise plane
 * the y interpolations onto the wall positions (interpy_new, lip.f90:767-809)
 * and derivatives (diffy_inplace, lip.f90:666-699), the mean and gradient
 * accumulations, the Reynolds stresses, the pressure correlations, the
 * vorticity and dissipation terms, and the triple products in physical space
 * (fourxz). The spectra, the two-point correlations and the instantaneous
 * enstrophy field ens(:,j,i) (stotf.F90:147-149,218-262) are not
 * accumulation statistics of this set and are not restated.
 *
 * Accumulators: OTBL_NSTATS arrays of the reference's shape (ny, nx), column
 * major, in the order of OTBL_ST_* (include/otbl.h); each call adds one
 * sample, as one statsp call does. Serial per (i, j) row with the k loop in
 * the reference's order.
 */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#ifdef _OPENMP
#include <omp.h>
#endif

/* the orc_box internals this file needs (oracle.c owns the struct) */
int orc_box_dims(const orc_box *b, int *nx, int *ny, int *nz, int *xround);
const double *orc_box_coef(const orc_box *b, otbl_coef_offsets *o);
const orc_fft *orc_box_zfft(const orc_box *b);

#define C8(c, r, j) (c)[((size_t)(j)-1) * 8 + (r)-1]

/* interpx_new, lip.f90:736-765: u_in, u_out (nx) strided by `st` */
static void interpx_new(const double *c, int nx, const double *in, double *out, size_t st) {
#define I(i) in[((size_t)(i)-1) * st]
#define O(i) out[((size_t)(i)-1) * st]
  double s = 0.0;
  for (int m = 1; m <= 4; ++m) s += C8(c, m, 1) * I(m);
  O(1) = s;
  s = 0.0;
  for (int m = 1; m <= 4; ++m) s += C8(c, m, nx - 1) * I(nx - 4 + m);
  O(nx - 1) = s;
  s = 0.0;
  for (int m = 1; m <= 4; ++m) s += C8(c, m, nx) * I(nx - 4 + m);
  O(nx) = s;
  for (int i = 2; i <= nx - 2; ++i) {
    s = 0.0;
    for (int m = 1; m <= 4; ++m) s += C8(c, m, 3) * I(i - 2 + m);
    O(i) = s;
  }
  for (int j = 2; j <= nx; ++j) O(j) = O(j) - C8(c, 6, j) * O(j - 1);
  O(nx) = O(nx) * C8(c, 7, nx);
  for (int j = nx - 1; j >= 1; --j) O(j) = (O(j) - C8(c, 8, j) * O(j + 1)) * C8(c, 7, j);
#undef I
#undef O
}

/* diffx_inplace, lip.f90:703-731 */
static void diffx(const double *c, int nx, const double *in, double *out, size_t st) {
#define I(i) in[((size_t)(i)-1) * st]
#define O(i) out[((size_t)(i)-1) * st]
  double s;
  s = 0.0;
  for (int m = 1; m <= 5; ++m) s += C8(c, m, 1) * I(m);
  O(1) = s;
  s = 0.0;
  for (int m = 1; m <= 5; ++m) s += C8(c, m, 2) * I(m);
  O(2) = s;
  s = 0.0;
  for (int m = 1; m <= 5; ++m) s += C8(c, m, nx - 1) * I(nx - 5 + m);
  O(nx - 1) = s;
  s = 0.0;
  for (int m = 1; m <= 5; ++m) s += C8(c, m, nx) * I(nx - 5 + m);
  O(nx) = s;
  for (int i = 3; i <= nx - 2; ++i) {
    s = 0.0;
    for (int m = 1; m <= 5; ++m) s += C8(c, m, 3) * I(i - 3 + m);
    O(i) = s;
  }
  for (int j = 2; j <= nx; ++j) O(j) = O(j) - C8(c, 6, j) * O(j - 1);
  O(nx) = O(nx) * C8(c, 7, nx);
  for (int j = nx - 1; j >= 1; --j) O(j) = (O(j) - C8(c, 8, j) * O(j + 1)) * C8(c, 7, j);
#undef I
#undef O
}

/* interpy_new, lip.f90:767-809, one column: in has ny+1-tipo rows, out ny,
 * both strided by `st` */
static void interpy_new(const double *c, int ny, const double *in, double *out, size_t st, int tipo) {
#define I(j) in[((size_t)(j)-1) * st]
#define O(j) out[((size_t)(j)-1) * st]
  const int ch = tipo == 1 ? 0 : 1;
  double s;
  s = 0.0;
  for (int m = 1; m <= 4; ++m) s += C8(c, m, 1) * I(m + 1);
  O(1) = s;
  s = 0.0;
  for (int m = 1; m <= 5; ++m) s += C8(c, m, 2) * I(m + 1);
  O(2) = s;
  for (int j = 3; j <= ny - 2; ++j) {
    s = 0.0;
    for (int m = 1; m <= 4; ++m) s += C8(c, m, j) * I(j - 2 + m);
    O(j) = s;
  }
  if (tipo == 0) O(1) = 0.0;
  s = 0.0;
  for (int m = 1; m <= 3 + ch; ++m) s += C8(c, m, ny - 1) * I(ny - 3 + m);
  O(ny - 1) = s;
  s = 0.0;
  for (int m = 1; m <= 3 + ch; ++m) s += C8(c, m, ny) * I(ny - 3 + m);
  O(ny) = s;
  for (int j = 3; j <= ny; ++j) O(j) = O(j) - C8(c, 6, j) * O(j - 1);
  O(ny) = O(ny) * C8(c, 7, ny);
  for (int j = ny - 1; j >= 2; --j) O(j) = (O(j) - C8(c, 8, j) * O(j + 1)) * C8(c, 7, j);
#undef I
#undef O
}

/* diffy_inplace, lip.f90:666-699, one column of ny rows */
static void diffy(const double *c, int ny, const double *in, double *out, size_t st) {
#define I(j) in[((size_t)(j)-1) * st]
#define O(j) out[((size_t)(j)-1) * st]
  double s;
  s = 0.0;
  for (int m = 1; m <= 4; ++m) s += C8(c, m, 1) * I(m);
  O(1) = s;
  s = 0.0;
  for (int m = 1; m <= 4; ++m) s += C8(c, m, 2) * I(m);
  O(2) = s;
  s = 0.0;
  for (int m = 1; m <= 4; ++m) s += C8(c, m, ny - 1) * I(ny - 4 + m);
  O(ny - 1) = s;
  s = 0.0;
  for (int m = 1; m <= 4; ++m) s += C8(c, m, ny) * I(ny - 4 + m);
  O(ny) = s;
  for (int j = 3; j <= ny - 2; ++j) {
    s = 0.0;
    for (int m = 1; m <= 5; ++m) s += C8(c, m, j) * I(j - 3 + m);
    O(j) = s;
  }
  for (int j = 2; j <= ny; ++j) O(j) = O(j) - C8(c, 6, j) * O(j - 1);
  O(ny) = O(ny) * C8(c, 7, ny);
  for (int j = ny - 1; j >= 1; --j) O(j) = (O(j) - C8(c, 8, j) * O(j + 1)) * C8(c, 7, j);
#undef I
#undef O
}

/* the operators on their own, for the known-answer tests: op 0 interpx_new,
 * 1 diffx (lines of nx, stride 1), 2 interpy_new tipo 0 (ny+1 rows in, ny
 * out), 3 interpy_new tipo 1 with fd_iyp (ny in, ny out), 4 diffy (ny, ny);
 * one line/column */
void orc_stats_operator(orc_box *b, int op, const double *in, double *out) {
  int nx, ny, nz, xr;
  orc_box_dims(b, &nx, &ny, &nz, &xr);
  otbl_coef_offsets o;
  const double *cf = orc_box_coef(b, &o);
  switch (op) {
    case 0: interpx_new(cf + o.off[OTBL_C_FD_IX], nx, in, out, 1); break;
    case 1: diffx(cf + o.off[OTBL_C_FD_DX], nx, in, out, 1); break;
    case 2: interpy_new(cf + o.off[OTBL_C_FD_IY], ny, in, out, 1, 0); break;
    case 3: interpy_new(cf + o.off[OTBL_C_FD_IYP], ny, in, out, 1, 1); break;
    case 4: diffy(cf + o.off[OTBL_C_FD_DVDY], ny, in, out, 1); break;
    default: break;
  }
}

static inline double rr(int xr, double x) { return xr ? (double)(float)x : x; }

void orc_statsp(orc_box *b, double *acc) {
  int nx, ny, nz, xr;
  orc_box_dims(b, &nx, &ny, &nz, &xr);
  const int nz1 = 2 * (nz / 3), nz2 = nz1 / 2 - 1;
  otbl_coef_offsets o;
  const double *cf = orc_box_coef(b, &o);
  const double *fix = cf + o.off[OTBL_C_FD_IX], *fdx = cf + o.off[OTBL_C_FD_DX];
  const double *fiy = cf + o.off[OTBL_C_FD_IY], *fiyp = cf + o.off[OTBL_C_FD_IYP];
  const double *fdv = cf + o.off[OTBL_C_FD_DVDY], *kaz = cf + o.off[OTBL_C_KAZ];
  const double *u = orc_field(b, OTBL_F_U), *v = orc_field(b, OTBL_F_V), *w = orc_field(b, OTBL_F_W);
  const double *p = orc_field(b, OTBL_F_P);
  const size_t PU = (size_t)(ny + 1) * nz1, PV = (size_t)ny * nz1;
  const size_t lu = (size_t)nx * PU, lv = (size_t)nx * PV;
  /* the x pre-pass, rhsp.F90:65-92, on x-lines addressed in the plane
   * layout (stride PU or PV); in REAL4 mode the transposes' roundings:
   * u, v, w into pencils (chp2x) and u_x, dudx, dvdx, dwdx back (chx2p) */
  double *ux = (double *)malloc(sizeof(double) * lu), *dudx = (double *)malloc(sizeof(double) * lu);
  double *dwdx = (double *)malloc(sizeof(double) * lu), *dvdx = (double *)malloc(sizeof(double) * lv);
#pragma omp parallel num_threads(orc_get_threads())
  {
  double *lin = (double *)malloc(sizeof(double) * 4 * (size_t)nx);
  double *a = lin, *t = lin + nx, *q = lin + 2 * nx, *r = lin + 3 * nx;
#pragma omp for schedule(static)
  for (long line = 0; line < (long)PU; ++line) {
    for (int i = 0; i < nx; ++i) a[i] = rr(xr, u[(size_t)i * PU + line]);
    interpx_new(fix, nx, a, t, 1);
    for (int i = nx - 1; i >= 1; --i) t[i] = t[i - 1]; /* wki1(i+1) = wki1(i), rhsp.F90:75-79 */
    diffx(fdx, nx, t, q, 1);
    for (int i = 0; i < nx; ++i) a[i] = rr(xr, w[(size_t)i * PU + line]);
    diffx(fdx, nx, a, r, 1);
    for (int i = 0; i < nx; ++i) {
      ux[(size_t)i * PU + line] = rr(xr, t[i]);
      dudx[(size_t)i * PU + line] = rr(xr, q[i]);
      dwdx[(size_t)i * PU + line] = rr(xr, r[i]);
    }
    if (line < (long)PV) {
      for (int i = 0; i < nx; ++i) a[i] = rr(xr, v[(size_t)i * PV + line]);
      diffx(fdx, nx, a, t, 1);
      for (int i = 0; i < nx; ++i) dvdx[(size_t)i * PV + line] = rr(xr, t[i]);
    }
  }
  free(lin);
  }
  const size_t NS = (size_t)nx * ny;
#define ACC(s, i, j) acc[(size_t)(s)*NS + ((size_t)(i)-1) * ny + (j)-1]
#pragma omp parallel num_threads(orc_get_threads())
  {
    /* buf1..buf8 of statsp for one plane, each (nz1, ny) */
    double *buf = (double *)malloc(sizeof(double) * 8 * PV);
    double *work = (double *)malloc(sizeof(double) * 8 * (size_t)(nz + 2));
    double *ph = (double *)malloc(sizeof(double) * 3 * (size_t)(nz + 2));
#pragma omp for schedule(static)
    for (int i = 1; i <= nx; ++i) {
      double *b1 = buf, *b2 = buf + PV, *b3 = buf + 2 * PV, *b4 = buf + 3 * PV;
      double *b5 = buf + 4 * PV, *b6 = buf + 5 * PV, *b7 = buf + 6 * PV, *b8 = buf + 7 * PV;
      const size_t iu = (size_t)(i - 1) * PU, iv = (size_t)(i - 1) * PV;
      for (int kr = 0; kr < nz1; ++kr) { /* stotf.F90:101-110 */
        interpy_new(fiy, ny, ux + iu + kr, b1 + kr, nz1, 0);
        interpy_new(fiy, ny, w + iu + kr, b2 + kr, nz1, 0);
        interpy_new(fiy, ny, dwdx + iu + kr, b3 + kr, nz1, 0);
        interpy_new(fiy, ny, dudx + iu + kr, b4 + kr, nz1, 0);
        interpy_new(fiyp, ny, p + iv + kr, b5 + kr, nz1, 1);
        diffy(fdv, ny, b1 + kr, b6 + kr, nz1);
        diffy(fdv, ny, b2 + kr, b7 + kr, nz1);
        diffy(fdv, ny, v + iv + kr, b8 + kr, nz1);
      }
      const double *vv = v + iv, *dv = dvdx + iv;
      for (int j = 1; j <= ny; ++j) {
        const size_t r0 = (size_t)(j - 1) * nz1;
#define RE(a, k) (a)[r0 + 2 * (k)]
#define IM(a, k) (a)[r0 + 2 * (k) + 1]
        /* k = 0: means, gradient means, mean vorticity, stotf.F90:118-134 */
        ACC(OTBL_ST_UA, i, j) += RE(b1, 0);
        ACC(OTBL_ST_WA, i, j) += RE(b2, 0);
        ACC(OTBL_ST_VA, i, j) += RE(vv, 0);
        ACC(OTBL_ST_PM, i, j) += RE(b5, 0);
        ACC(OTBL_ST_DUDX0, i, j) += RE(b4, 0);
        ACC(OTBL_ST_DVDX0, i, j) += RE(dv, 0);
        ACC(OTBL_ST_DWDX0, i, j) += RE(b3, 0);
        ACC(OTBL_ST_DUDY0, i, j) += RE(b6, 0);
        ACC(OTBL_ST_DVDY0, i, j) += RE(b8, 0);
        ACC(OTBL_ST_DWDY0, i, j) += RE(b7, 0);
        ACC(OTBL_ST_VORTYA, i, j) -= RE(b3, 0);
        ACC(OTBL_ST_VORTXA, i, j) += RE(b7, 0);
        ACC(OTBL_ST_VORTZA, i, j) += RE(dv, 0) - RE(b6, 0);
        /* the k sums, stotf.F90:165-217 */
        for (int k = 0; k <= nz2; ++k) {
          const double cte = k == 0 ? 1.0 : 2.0, kz = kaz[k];
          const double u1r = RE(b1, k), u1i = IM(b1, k), w2r = RE(b2, k), w2i = IM(b2, k);
          const double vr = RE(vv, k), vi = IM(vv, k), pr = RE(b5, k), pi_ = IM(b5, k);
          const double x3r = RE(b3, k), x3i = IM(b3, k), x4r = RE(b4, k), x4i = IM(b4, k);
          const double x6r = RE(b6, k), x6i = IM(b6, k), x7r = RE(b7, k), x7i = IM(b7, k);
          const double x8r = RE(b8, k), x8i = IM(b8, k), dvr = RE(dv, k), dvi = IM(dv, k);
          /* i kz times a mode: (-kz Im, kz Re) */
          const double wzr = -w2i * kz, wzi = w2r * kz, uzr = -u1i * kz, uzi = u1r * kz;
          const double vzr = -vi * kz, vzi = vr * kz;
          ACC(OTBL_ST_US, i, j) += cte * (u1r * u1r + u1i * u1i);
          ACC(OTBL_ST_WS, i, j) += cte * (w2r * w2r + w2i * w2i);
          ACC(OTBL_ST_VS, i, j) += cte * (vr * vr + vi * vi);
          ACC(OTBL_ST_UV, i, j) += cte * (u1r * vr + u1i * vi);
          ACC(OTBL_ST_UW, i, j) += cte * (u1r * w2r + u1i * w2i);
          ACC(OTBL_ST_VW, i, j) += cte * (vr * w2r + vi * w2i);
          ACC(OTBL_ST_PUP, i, j) += cte * (pr * u1r + pi_ * u1i);
          ACC(OTBL_ST_PVP, i, j) += cte * (pr * vr + pi_ * vi);
          ACC(OTBL_ST_PP, i, j) += cte * (pr * pr + pi_ * pi_);
          ACC(OTBL_ST_PDWDZ, i, j) += cte * (pr * wzr + pi_ * wzi);
          ACC(OTBL_ST_PDUDX, i, j) += cte * (pr * x4r + pi_ * x4i);
          ACC(OTBL_ST_PDVDX, i, j) += cte * (pr * dvr + pi_ * dvi);
          ACC(OTBL_ST_PDVDY, i, j) += cte * (pr * x8r + pi_ * x8i);
          ACC(OTBL_ST_PDUDY, i, j) += cte * (pr * x6r + pi_ * x6i);
          double ar = x7r - vzr, ai = x7i - vzi; /* o_x = dwdy - dvdz */
          ACC(OTBL_ST_VORTX, i, j) += cte * (ar * ar + ai * ai);
          ar = uzr - x3r, ai = uzi - x3i; /* o_y = dudz - dwdx */
          ACC(OTBL_ST_VORTY, i, j) += cte * (ar * ar + ai * ai);
          ar = dvr - x6r, ai = dvi - x6i; /* o_z = dvdx - dudy */
          ACC(OTBL_ST_VORTZ, i, j) += cte * (ar * ar + ai * ai);
          ACC(OTBL_ST_DISPU, i, j) += cte * ((x4r * x4r + x4i * x4i) + (uzr * uzr + uzi * uzi) + (x6r * x6r + x6i * x6i));
          ACC(OTBL_ST_DISPV, i, j) += cte * ((dvr * dvr + dvi * dvi) + (vzr * vzr + vzi * vzi) + (x8r * x8r + x8i * x8i));
          ACC(OTBL_ST_DISPW, i, j) += cte * ((wzr * wzr + wzi * wzi) + (x3r * x3r + x3i * x3i) + (x7r * x7r + x7i * x7i));
          ACC(OTBL_ST_DISPUV, i, j) += cte * ((uzr * vzr + uzi * vzi) + (x4r * dvr + x4i * dvi) + (x6r * x8r + x6i * x8i));
        }
        /* triple products in physical space, stotf.F90:264-285 */
        double *pu = ph, *pw = ph + (nz + 2), *pv = ph + 2 * (nz + 2);
        orc_c2r_line(orc_box_zfft(b), nz, nz2, b1 + r0, pu, work);
        orc_c2r_line(orc_box_zfft(b), nz, nz2, b2 + r0, pw, work);
        orc_c2r_line(orc_box_zfft(b), nz, nz2, vv + r0, pv, work);
        for (int k = 0; k < nz; ++k) {
          const double uu = pu[k], ww = pw[k], vp = pv[k];
          ACC(OTBL_ST_U3, i, j) += (uu * uu) * uu;
          ACC(OTBL_ST_W2U, i, j) += uu * (ww * ww);
          ACC(OTBL_ST_V3, i, j) += (vp * vp) * vp;
          ACC(OTBL_ST_W2V, i, j) += vp * (ww * ww);
          ACC(OTBL_ST_V2U, i, j) += uu * (vp * vp);
          ACC(OTBL_ST_U2V, i, j) += vp * (uu * uu);
        }
#undef RE
#undef IM
      }
    }
    free(buf);
    free(work);
    free(ph);
  }
#undef ACC
  free(ux);
  free(dudx);
  free(dwdx);
  free(dvdx);
}
