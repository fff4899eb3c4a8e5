/*
 * ORACLE -- test infrastructure, never part of the product path.
 *
 * orc_coef_compute: the set-up that fills the reference's coefficient module
 * alloc_dns (mod.F90:96-184) before its time loop, restated in plain C from
 * the Fortran:
 *   iniciap_1 wavenumbers   bl_1.F90:357-366
 *   coef                    coeft.f90:10-1234 (the statistics-only arrays
 *                           fd_*, l_weight, ldyy, axphi/ayphi are skipped:
 *                           the substep reads none of them)
 *   mtr                     coeft.f90:1244-1332
 *   coefinv                 coeft.f90:1338-1353
 *   coefb                   coeft.f90:1360-1789
 *   ludcmp, lubksb          coeft.f90:1818-1922
 *   inlet_retheta           bl_1.F90:372-396
 *   magicnumber             boun.f90:102-143
 * into the packed buffer of include/otbl_layout.h. It is separate code from
 * the product's otbl_coef_compute (written from the Fortran, not from the
 * product), so the oracle runs on coefficients of its own and the parity
 * tests check the product's set-up too; a test compares the two buffers
 * element by element.
 *
 * Fortran semantics kept literally (the reference's build uses no
 * -r8/-autodouble/-qrealsize flag, makefile-OMP-vul:10, makefile-OMP-bg:15):
 *  - x**2, x**3, x**4 as gfortran expands integer powers: x*x, (x*x)*x,
 *    (x*x)*(x*x); expressions in Fortran precedence order, left to right
 *    (cfl*dxmin**2 is cfl*(dxmin*dxmin));
 *  - cmplx(0d0, k/az) has no KIND argument, so it is a default (REAL*4)
 *    complex: kaz(k) is k/az rounded to single precision (bl_1.F90:360) and
 *    kaz2(k) = -kaz(k)**2 its square (bl_1.F90:365);
 *  - the literal 0.99 of inlet_retheta is REAL*4 (bl_1.F90:382).
 */
#include <math.h>
#include <string.h>

#include "oracle.h"

/* gfortran's expansion of integer powers */
static double ipow2(double x) { return x * x; }
static double ipow3(double x) { return (x * x) * x; }
static double ipow4(double x) {
  const double s = x * x;
  return s * s;
}

/* ---- ludcmp / lubksb, coeft.f90:1818-1922: a(np,np) column-major, 1-based */
#define LA(i, j) a[((j)-1) * np + (i)-1]

static int f_ludcmp(double *a, int n, int np, int *indx) {
  const double tiny = 1.0e-20;
  double vv[101];
  int imax = 1;
  for (int i = 1; i <= n; ++i) {
    double aamax = 0.0;
    for (int j = 1; j <= n; ++j)
      if (fabs(LA(i, j)) > aamax) aamax = fabs(LA(i, j));
    if (aamax == 0.0) return -1; /* pause 'singular matrix.' */
    vv[i] = 1.0 / aamax;
  }
  for (int j = 1; j <= n; ++j) {
    if (j > 1) {
      for (int i = 1; i <= j - 1; ++i) {
        double sum = LA(i, j);
        if (i > 1) {
          for (int k = 1; k <= i - 1; ++k) sum = sum - LA(i, k) * LA(k, j);
          LA(i, j) = sum;
        }
      }
    }
    double aamax = 0.0;
    for (int i = j; i <= n; ++i) {
      double sum = LA(i, j);
      if (j > 1) {
        for (int k = 1; k <= j - 1; ++k) sum = sum - LA(i, k) * LA(k, j);
        LA(i, j) = sum;
      }
      const double dum = vv[i] * fabs(sum);
      if (dum >= aamax) {
        imax = i;
        aamax = dum;
      }
    }
    if (j != imax) {
      for (int k = 1; k <= n; ++k) {
        const double dum = LA(imax, k);
        LA(imax, k) = LA(j, k);
        LA(j, k) = dum;
      }
      vv[imax] = vv[j];
    }
    indx[j] = imax;
    if (j != n) {
      if (LA(j, j) == 0.0) LA(j, j) = tiny;
      const double dum = 1.0 / LA(j, j);
      for (int i = j + 1; i <= n; ++i) LA(i, j) = LA(i, j) * dum;
    }
  }
  if (LA(n, n) == 0.0) LA(n, n) = tiny;
  return 0;
}

static void f_lubksb(const double *a, int n, int np, const int *indx, double *b /* b(1:n) */) {
  int ii = 0;
  for (int i = 1; i <= n; ++i) {
    const int ll = indx[i];
    double sum = b[ll];
    b[ll] = b[i];
    if (ii != 0) {
      for (int j = ii; j <= i - 1; ++j) sum = sum - LA(i, j) * b[j];
    } else if (sum != 0.0) {
      ii = i;
    }
    b[i] = sum;
  }
  for (int i = n; i >= 1; --i) {
    double sum = b[i];
    if (i < n)
      for (int j = i + 1; j <= n; ++j) sum = sum - LA(i, j) * b[j];
    b[i] = sum / LA(i, i);
  }
}
#undef LA

/* ---- coefb, coeft.f90:1360-1789: moment conditions of one boundary
 * closure, solved by ludcmp/lubksb. bcc is 1-based, bcc[1..n]. */
static int f_coefb(int n, double a, double b, double c, double d, double *bcc, int flagv) {
  enum { np = 5 };
  double bc[np * np];
  int indx[np + 1];
#define BC(i, j) bc[((j)-1) * np + (i)-1]
  for (int i = 1; i <= n; ++i) {
    bcc[i] = 0.0;
    indx[i] = 0;
    for (int j = 1; j <= n; ++j) BC(i, j) = 0.0;
  }
  const double h = 1 / 2.0, e8 = 1 / 8.0, s6 = 1 / 6.0, f24 = 1 / 24.0, f48 = 1 / 48.0;
  if (flagv == 1) { /* coeft.f90:1369-1411 */
    bcc[1] = 1.0;
    BC(1, 1) = -1.0;       BC(1, 2) = 0.0; BC(1, 3) = h * ipow2(a);
    BC(1, 4) = h * ipow2(a + b);           BC(1, 5) = h * ipow2(a + b + c);
    BC(2, 1) = 0.0;        BC(2, 2) = 1.0; BC(2, 3) = 1.0; BC(2, 4) = 1.0; BC(2, 5) = 1.0;
    BC(3, 1) = 0.0;        BC(3, 2) = 0.0; BC(3, 3) = a; BC(3, 4) = a + b; BC(3, 5) = a + b + c;
    BC(4, 1) = -a;         BC(4, 2) = 0.0; BC(4, 3) = s6 * ipow3(a);
    BC(4, 4) = s6 * ipow3(a + b);          BC(4, 5) = s6 * ipow3(a + b + c);
    BC(5, 1) = -(h * ipow2(a));            BC(5, 2) = 0.0; BC(5, 3) = f24 * ipow4(a);
    BC(5, 4) = f24 * ipow4(a + b);         BC(5, 5) = f24 * ipow4(a + b + c);
  } else if (flagv == 0) { /* coeft.f90:1413-1437 */
    bcc[1] = 1.0;
    BC(1, 1) = 1.0; BC(1, 2) = 1.0; BC(1, 3) = 1.0;
    BC(2, 1) = -(h * a);
    BC(2, 2) = -(h * a + b);
    BC(2, 3) = -(h * a + b + c);
    BC(3, 1) = e8 * ipow2(a);
    BC(3, 2) = h * ipow2(-(h * a + b));
    BC(3, 3) = h * ipow2(-(h * a + b + c));
  } else if (flagv == 3) { /* coeft.f90:1487-1523 */
    bcc[1] = 1.0;
    BC(1, 1) = h * a;  BC(1, 2) = h * a + b;  BC(1, 3) = h * a + b + c;  BC(1, 4) = h * a + b + c + d;
    BC(2, 1) = 1.0;    BC(2, 2) = 1.0;        BC(2, 3) = 1.0;            BC(2, 4) = 1.0;
    BC(3, 1) = e8 * ipow2(a);
    BC(3, 2) = h * ipow2(h * a + b);
    BC(3, 3) = h * ipow2(h * a + b + c);
    BC(3, 4) = h * ipow2(h * a + b + c + d);
    BC(4, 1) = f48 * ipow3(a);
    BC(4, 2) = s6 * ipow3(h * a + b);
    BC(4, 3) = s6 * ipow3(h * a + b + c);
    BC(4, 4) = s6 * ipow3(h * a + b + c + d);
  } else if (flagv == 4) { /* coeft.f90:1525-1557 */
    bcc[1] = 1.0;
    BC(1, 1) = 1.0; BC(1, 2) = 1.0; BC(1, 3) = 1.0; BC(1, 4) = 1.0;
    BC(2, 1) = -(h * a);
    BC(2, 2) = h * b;
    BC(2, 3) = h * b + c;
    BC(2, 4) = h * b + c + d;
    BC(3, 1) = e8 * ipow2(a);
    BC(3, 2) = e8 * ipow2(b);
    BC(3, 3) = h * ipow2(h * b + c);
    BC(3, 4) = h * ipow2(h * b + c + d);
    BC(4, 1) = -(f48 * ipow3(a));
    BC(4, 2) = f48 * ipow3(b);
    BC(4, 3) = s6 * ipow3(h * b + c);
    BC(4, 4) = s6 * ipow3(h * b + c + d);
  } else if (flagv == 5) { /* coeft.f90:1559-1595 */
    bcc[1] = 1.0;
    BC(1, 1) = h * a;
    BC(1, 2) = -(h * b);
    BC(1, 3) = -(h * b + c);
    BC(1, 4) = -(h * b + c + d);
    BC(2, 1) = 1.0; BC(2, 2) = 1.0; BC(2, 3) = 1.0; BC(2, 4) = 1.0;
    BC(3, 1) = e8 * ipow2(a);
    BC(3, 2) = e8 * ipow2(b);
    BC(3, 3) = h * ipow2(-(h * b + c));
    BC(3, 4) = h * ipow2(-(h * b + c + d));
    BC(4, 1) = f48 * ipow3(a);
    BC(4, 2) = -(f48 * ipow3(b));
    BC(4, 3) = s6 * ipow3(-(h * b + c));
    BC(4, 4) = s6 * ipow3(-(h * b + c + d));
  } else if (flagv == 6) { /* coeft.f90:1597-1633 */
    bcc[2] = 1.0;
    BC(1, 1) = 1.0; BC(1, 2) = 1.0; BC(1, 3) = 1.0; BC(1, 4) = 1.0;
    BC(2, 1) = 0.0;
    BC(2, 2) = -(h * a);
    BC(2, 3) = -(h * a + b);
    BC(2, 4) = -(h * a + b + c);
    BC(3, 1) = 0.0;
    BC(3, 2) = e8 * ipow2(a);
    BC(3, 3) = h * ipow2(-(h * a + b));
    BC(3, 4) = h * ipow2(-(h * a + b + c));
    BC(4, 1) = 0.0;
    BC(4, 2) = -(f48 * ipow3(a));
    BC(4, 3) = s6 * ipow3(-(h * a + b));
    BC(4, 4) = s6 * ipow3(-(h * a + b + c));
  } else if (flagv == 7) { /* coeft.f90:1635-1672 */
    bcc[2] = 1.0;
    BC(1, 1) = 1.0; BC(1, 2) = 1.0; BC(1, 3) = 1.0; BC(1, 4) = 1.0;
    BC(2, 1) = h * a;
    BC(2, 2) = -(h * b);
    BC(2, 3) = -(h * b + c);
    BC(2, 4) = -(h * b + c + d);
    BC(3, 1) = e8 * ipow2(a);
    BC(3, 2) = e8 * ipow2(b);
    BC(3, 3) = ipow2(h * b + c); /* no 1/2 factor in the reference */
    BC(3, 4) = ipow2(h * b + c + d);
    BC(4, 1) = f48 * ipow3(a);
    BC(4, 2) = -(f48 * ipow3(b));
    BC(4, 3) = -(s6 * ipow3(h * b + c));
    BC(4, 4) = -(s6 * ipow3(h * b + c + d));
  } else {
    return -2; /* flags 2 and 8 are not used by coef */
  }
#undef BC
  if (f_ludcmp(bc, n, np, indx) != 0) return -1;
  f_lubksb(bc, n, np, indx, bcc);
  return 0;
}

/* ---- coefinv, coeft.f90:1338-1353, on a(3, npter1:neq) ---- */
static void f_coefinv(double *a, int neq, int npter1) {
#define CA(r, j) a[((j)-npter1) * 3 + (r)-1]
  for (int j = npter1 + 1; j <= neq; ++j) {
    const double d = 1.0 / CA(2, j - 1);
    CA(2, j - 1) = d;
    CA(1, j) = -CA(1, j) * d;
    CA(2, j) = CA(2, j) + CA(1, j) * CA(3, j - 1);
  }
  CA(2, neq) = 1.0 / CA(2, neq);
#undef CA
}

/* column accessors of the packed (3,n), (2,n) arrays and small matrices */
#define T3(p, r, i) (p)[((i)-1) * 3 + (r)-1]
#define T2(p, r, i) (p)[((i)-1) * 2 + (r)-1]
#define MAT(p, nr, r, c) (p)[((c)-1) * (nr) + (r)-1]

/* x**5 as gfortran expands an integer power: x**3 * x**2 */
static double ipow5(double x) {
  const double s = x * x;
  return ((s * x) * s);
}

/* LU reorganisation of an (8, n) compact operator, coeft.f90:146-150 and
 * its copies: from row j0 on, c6 /= c7(j-1), c7 -= c6 c8(j-1); then c7 is
 * inverted on rows inv0..n */
static void fd_lu(double *c, int n, int j0, int inv0) {
#define C8(r, j) c[((j)-1) * 8 + (r)-1]
  for (int j = j0; j <= n; ++j) {
    C8(6, j) = C8(6, j) / C8(7, j - 1);
    C8(7, j) = C8(7, j) - C8(6, j) * C8(8, j - 1);
  }
  for (int j = inv0; j <= n; ++j) C8(7, j) = 1.0 / C8(7, j);
#undef C8
}

/* The compact operators of the one-point statistics, coeft.f90:56-318
 * (Gamet et al.'s compact schemes on non-uniform meshes): fd_dvdy (d/dy at
 * the v rows), fd_dx (d/dx), fd_ix (mid-point interpolation in x), fd_iy and
 * fd_iyp (mid-point interpolation in y onto the wall positions, for u, w and
 * for p). Each is (8, n): stencil weights in rows 1..5, the tridiagonal's
 * sub-diagonal, diagonal and super-diagonal in rows 6..8, then LU-reorganised.
 * Every expression keeps the Fortran's order of operations. */
static void f_fd_operators(int nx, int ny, double ax, double pi, const double *y, double *fdvdy,
                           double *fdx, double *fix, double *fiy, double *fiyp) {
#define DV(r, j) fdvdy[((j)-1) * 8 + (r)-1]
#define FX(r, i) fdx[((i)-1) * 8 + (r)-1]
#define IX(r, i) fix[((i)-1) * 8 + (r)-1]
#define IY(r, j) fiy[((j)-1) * 8 + (r)-1]
#define IP(r, j) fiyp[((j)-1) * 8 + (r)-1]
  double h[ny + 2], hi[ny + 2], yp[ny + 2]; /* h(1:ny+1), hi(1:ny+1), yp(1:ny+1) */
  double a, b, c, d, e, f, g;

  /* ---- d/dy, coeft.f90:56-150 ---- */
  for (int j = 1; j <= ny + 1; ++j) h[j] = y[j] - y[j - 1];
  a = h[2];
  b = h[2] + h[3];
  c = h[2] + h[3] + h[4];
  DV(1, 1) = -(a * b + a * c + 2 * b * c) / b / a / c;
  DV(3, 1) = -(ipow2(a) * c / (b - c) / b / ipow2(a - b));
  DV(4, 1) = ipow2(a) * b / c / ipow2(a - c) / (b - c);
  DV(2, 1) = -(DV(1, 1) + DV(3, 1) + DV(4, 1));
  DV(7, 1) = 1.0;
  DV(8, 1) = b * c / (a - c) / (a - b);
  DV(1, 2) = ipow2(a - b) * (a - c) * (a * b + 2 * a * c + 2 * b * c) / a / ipow3(b) / ipow2(c);
  DV(2, 2) = 1 / a * (-3 * a * b + 2 * b * c + 5 * ipow2(a) - 4 * a * c) / (a - c) / (a - b);
  DV(3, 2) = ipow2(a) * (a - c) * (-2 * a * c + 3 * a * b + 4 * b * c - 5 * ipow2(b)) / ipow3(b) /
             ipow2(b - c) / (a - b);
  DV(4, 2) = -(DV(1, 2) + DV(2, 2) + DV(3, 2));
  DV(6, 2) = -(ipow2(a - b) * (a - c) / c / ipow2(b));
  DV(7, 2) = 1.0;
  DV(8, 2) = ipow2(a) * (a - c) / (b - c) / ipow2(b);
  for (int i = 3; i <= ny - 2; ++i) {
    a = h[i - 1];
    b = h[i];
    c = h[i + 1];
    d = h[i + 2];
    f = c + d;
    e = a + b;
    DV(1, i) = -(ipow2(c) * ipow2(b) * f / (f + e) / e / (ipow2(c) + 2 * c * e + ipow2(e)) /
                 (ipow2(e) - 2 * e * b + ipow2(b)));
    DV(2, i) = f / b * e * ipow2(c) *
               (3 * c * b * f - 2 * c * f * e + 4 * ipow2(b) * c - 3 * b * e * c + 5 * ipow2(b) * f -
                4 * b * e * f + 6 * ipow3(b) - 5 * e * ipow2(b)) /
               (ipow2(f) + 2 * b * f + ipow2(b)) /
               (ipow3(b) + 3 * b * ipow2(c) + ipow3(c) + 3 * ipow2(b) * c) / (ipow2(e) - 2 * e * b + ipow2(b));
    DV(3, i) = (c * b * f - b * e * c - 2 * b * e * f + 2 * c * f * e) / f / b / e / c;
    DV(4, i) = -((-3 * c * b * f - 2 * b * e * f + 3 * b * e * c + 4 * b * ipow2(c) - 5 * ipow2(c) * f -
                  4 * c * f * e + 6 * ipow3(c) + 5 * ipow2(c) * e) *
                 ipow2(b) / c * e * f / (ipow2(f) - 2 * f * c + ipow2(c)) /
                 (3 * ipow2(e) * b * ipow2(c) + 6 * e * ipow2(b) * ipow2(c) + 6 * e * b * ipow3(c) +
                  ipow2(e) * ipow3(b) + ipow5(c) + 2 * ipow4(c) * e + ipow3(c) * ipow2(e) +
                  3 * ipow2(b) * ipow3(c) + ipow3(b) * ipow2(c) + 3 * b * ipow4(c) + 2 * e * ipow3(b) * c +
                  3 * ipow2(e) * ipow2(b) * c));
    DV(5, i) = -(DV(1, i) + DV(2, i) + DV(3, i) + DV(4, i));
    DV(6, i) = -(e * ipow2(c) * f / (f + b) / (ipow2(b) + 2 * b * c + ipow2(c)) / (b - e));
    DV(7, i) = 1.0;
    DV(8, i) = -(e * ipow2(b) * f / (c - f) / (ipow2(b) + 2 * b * c + ipow2(c)) / (c + e));
  }
  a = h[ny - 2];
  b = h[ny - 1];
  c = h[ny];
  f = a + b + c;
  e = b + c;
  DV(1, ny - 1) = ipow2(c) * ipow2(c - e) / ipow2(f) / ipow2(f - e) / (c - f);
  DV(3, ny - 1) = -((5 * ipow2(c) - 4 * f * c - 3 * c * e + 2 * f * e) / c / (c - f) / (c - e));
  DV(4, ny - 1) = -(ipow2(c - e) * (c - f) * (2 * f * c + c * e + 2 * f * e) / c / ipow2(f) / ipow3(e));
  DV(2, ny - 1) = -(DV(1, ny - 1) + DV(3, ny - 1) + DV(4, ny - 1));
  DV(6, ny - 1) = -((c - f) * ipow2(c) / ipow2(e) / (f - e));
  DV(7, ny - 1) = 1.0;
  DV(8, ny - 1) = -(ipow2(c - e) * (c - f) / f / ipow2(e));
  DV(1, ny) = ipow2(c) * e / ipow2(c - f) / (f - e) / f;
  DV(2, ny) = -(ipow2(c) * f / e / ipow2(c - e) / (f - e));
  DV(4, ny) = (f * c + c * e + 2 * f * e) / c / f / e;
  DV(3, ny) = -(DV(1, ny) + DV(2, ny) + DV(4, ny));
  DV(6, ny) = f * e / (c - f) / (c - e);
  DV(7, ny) = 1.0;
  fd_lu(fdvdy, ny, 2, 1);

  /* ---- d/dx on the uniform x grid, coeft.f90:153-194 ---- */
  FX(1, 1) = -37.0 / 12.0; FX(1, 2) = -43.0 / 96.0;
  FX(2, 1) = 2.0 / 3.0;    FX(2, 2) = -5.0 / 6.0;
  FX(3, 1) = 3.0;          FX(3, 2) = 9.0 / 8.0;
  FX(4, 1) = -2.0 / 3.0;   FX(4, 2) = 1.0 / 6.0;
  FX(5, 1) = 1.0 / 12.0;   FX(5, 2) = -1.0 / 96.0;
  FX(7, 1) = 1.0;          FX(6, 2) = 1.0 / 8.0;
  FX(8, 1) = 4.0;          FX(7, 2) = 1.0;
  FX(8, 2) = 3.0 / 4.0;
  for (int i = 3; i <= nx - 2; ++i) {
    FX(1, i) = -1.0 / 36.0;
    FX(2, i) = -7.0 / 9.0;
    FX(3, i) = 0.0;
    FX(4, i) = 7.0 / 9.0;
    FX(5, i) = 1.0 / 36.0;
    FX(6, i) = 1.0 / 3.0;
    FX(7, i) = 1.0;
    FX(8, i) = 1.0 / 3.0;
  }
  FX(1, nx - 1) = 1.0 / 96.0;  FX(1, nx) = -1.0 / 12.0;
  FX(2, nx - 1) = -1.0 / 6.0;  FX(2, nx) = 2.0 / 3.0;
  FX(3, nx - 1) = -9.0 / 8.0;  FX(3, nx) = -3.0;
  FX(4, nx - 1) = 5.0 / 6.0;   FX(4, nx) = -2.0 / 3.0;
  FX(5, nx - 1) = 43.0 / 96.0; FX(5, nx) = 37.0 / 12.0;
  FX(6, nx - 1) = 3.0 / 4.0;   FX(6, nx) = 4.0;
  FX(7, nx - 1) = 1.0;         FX(7, nx) = 1.0;
  FX(8, nx - 1) = 1.0 / 8.0;
  const double point0 = ax * pi / (nx + 1);
  for (int i = 1; i <= nx; ++i)
    for (int r = 1; r <= 5; ++r) FX(r, i) = FX(r, i) / point0;
  fd_lu(fdx, nx, 2, 1);

  /* ---- mid-point interpolation in x, coeft.f90:196-228 ---- */
  IX(1, 1) = 5.0 / 24.0;   IX(1, nx - 1) = -1.0 / 84.0;
  IX(2, 1) = 15.0 / 8.0;   IX(2, nx - 1) = 1.0 / 4.0;
  IX(3, 1) = 5.0 / 8.0;    IX(3, nx - 1) = 5.0 / 4.0;
  IX(4, 1) = -1.0 / 24.0;  IX(4, nx - 1) = 5.0 / 12.0;
  IX(7, 1) = 1.0;          IX(6, nx - 1) = 5.0 / 6.0;
  IX(8, 1) = 5.0 / 3.0;    IX(7, nx - 1) = 1.0;
  IX(8, nx - 1) = 1.0 / 14.0;
  for (int i = 2; i <= nx - 2; ++i) {
    IX(1, i) = 1.0 / 20.0;
    IX(2, i) = 3.0 / 4.0;
    IX(3, i) = 3.0 / 4.0;
    IX(4, i) = 1.0 / 20.0;
    IX(6, i) = 3.0 / 10.0;
    IX(7, i) = 1.0;
    IX(8, i) = 3.0 / 10.0;
  }
  IX(1, nx) = 1.0 / 8.0;
  IX(2, nx) = -7.0 / 8.0;
  IX(3, nx) = 35.0 / 8.0;
  IX(4, nx) = 35.0 / 8.0;
  IX(6, nx) = 7.0;
  IX(7, nx) = 1.0;
  fd_lu(fix, nx, 2, 1);

  /* ---- mid-point interpolation in y onto the wall positions, for u, w
   * (fd_iy) and p (fd_iyp), coeft.f90:231-318 ---- */
  for (int j = 1; j <= ny + 1; ++j) yp[j] = (y[j - 1] + y[j]) * 0.5;
  for (int j = 1; j <= ny + 1; ++j) hi[j] = y[j] - y[j - 1];
  for (int j = 2; j <= ny + 1; ++j) h[j] = yp[j] - yp[j - 1];
  a = hi[2] / 2;
  b = a + h[3];
  c = b + h[4];
  d = c + h[5];
  IY(1, 1) = -(c * b * d / (a - d) / (a - c) / (a - b));
  IY(2, 1) = c * a * d / (b - d) / (b - c) / (a - b);
  IY(3, 1) = -(b * a * d / (c - d) / (ipow2(c) - a * c - b * c + b * a));
  IY(4, 1) = 1.0 - (IY(1, 1) + IY(2, 1) + IY(3, 1));
  a = hi[3] / 2;
  b = a + h[4];
  c = b + h[5];
  d = c + h[6];
  e = hi[2] / 2;
  IY(1, 2) = 2 * c * b * ipow2(a) * d / (e + d) / (e + c) / (b + e) / (2 * ipow2(a) + ipow2(e) + 3 * e * a);
  IY(2, 2) = -(2 * c * b * e * d / (a - d) / (a - c) / (a - b) / (a + e));
  IY(3, 2) = 2 * c * e * ipow2(a) * d / (b - d) / (b - c) /
             (2 * ipow2(a) * e + 2 * ipow2(a) * b - 3 * a * ipow2(b) - 3 * a * e * b + ipow3(b) + e * ipow2(b));
  IY(4, 2) = -(2 * ipow2(a) * b * e * d / (c - d) /
               (3 * e * a * ipow2(c) - 2 * e * ipow2(a) * c - 3 * b * e * a * c - 2 * ipow2(a) * ipow2(c) +
                2 * ipow2(a) * e * b + 3 * a * ipow3(c) + b * ipow3(c) - e * ipow3(c) + 2 * b * ipow2(a) * c -
                3 * b * a * ipow2(c) + b * e * ipow2(c) - ipow4(c)));
  IY(7, 2) = 1.0;
  IY(8, 2) = -(c * b * e * d / (2 * a + e) / (2 * a - d) / (2 * a - c) / (2 * a - b));
  IY(5, 2) = (IY(7, 2) + IY(8, 2)) - (IY(1, 2) + IY(2, 2) + IY(3, 2) + IY(4, 2));
  for (int j = 3; j <= ny - 1; ++j) {
    a = hi[j + 1] / 2;
    b = a + h[j + 2];
    e = hi[j] / 2;
    f = e + h[j];
    IY(1, j) = 4 * ipow2(e) * ipow2(a) * b / (b + f) /
               (2 * ipow2(a) * ipow2(f) + ipow4(f) + 4 * ipow2(e) * ipow2(a) - 6 * ipow2(a) * e * f -
                9 * e * a * ipow2(f) + 6 * ipow2(e) * a * f + 2 * ipow2(e) * ipow2(f) + 3 * a * ipow3(f) -
                3 * e * ipow3(f));
    IY(2, j) = -(4 * f * ipow2(a) * b / (b + e) / (a + e) / (e - f) / (2 * a + e));
    IY(3, j) = -(4 * f * ipow2(e) * b / (a - b) / (a + f) / (2 * ipow2(e) + ipow2(a) + 3 * e * a));
    IY(6, j) = -(f * b * ipow2(a) / (a + e) / (2 * e - f) / (b + 2 * e) / (a + 2 * e));
    IY(7, j) = 1.0;
    IY(8, j) = -(f * ipow2(e) * b / (2 * a - b) / (2 * a + f) / (2 * ipow2(a) + ipow2(e) + 3 * e * a));
    IY(4, j) = (IY(6, j) + IY(7, j) + IY(8, j)) - (IY(1, j) + IY(2, j) + IY(3, j));
  }
  a = hi[ny + 1] / 2;
  e = hi[ny] / 2;
  f = e + h[ny];
  g = f + h[ny - 1];
  {
    const double n3 = 8 * ipow3(e) - 4 * g * ipow2(e) - 2 * f * a * e - 2 * g * e * a - 4 * f * ipow2(e) +
                      g * a * f + 4 * a * ipow2(e) + 2 * f * g * e;
    IY(1, ny) = 2 * (4 * ipow2(e) + 2 * e * a - a * f - 2 * f * e) * ipow2(e) / (e - g) / (f - g) / g / (g + a);
    IY(2, ny) = -(2 * (2 * e * a + 4 * ipow2(e) - a * g - 2 * g * e) * ipow2(e) / (e - f) / f /
                  (ipow2(f) + a * f - g * f - a * g));
    IY(3, ny) = 2 * n3 /
                (ipow3(e) + a * ipow2(e) - f * ipow2(e) - g * ipow2(e) + g * a * f - g * e * a + f * g * e - f * a * e);
    IY(4, ny) = 2 * (-2 * f * e - 2 * g * e + g * f + 4 * ipow2(e)) * ipow2(e) / (g + a) / (a + f) / (a + e) / a;
    IY(6, ny) = 1.0;
    IY(7, ny) = n3 / g / a / f;
  }
  memcpy(fiyp, fiy, sizeof(double) * 8 * (size_t)ny);
  a = hi[ny] / 2;
  e = hi[ny - 1] / 2;
  f = e + h[ny - 1];
  IP(1, ny - 1) = 4 * ipow2(e) * ipow2(a) / (2 * a + f) / (a + f) / (2 * ipow2(e) + ipow2(f) - 3 * e * f);
  IP(2, ny - 1) = -(4 * f * ipow2(a) / (3 * e * a + ipow2(e) + 2 * ipow2(a)) / (e - f));
  IP(3, ny - 1) = 4 * ipow2(e) * f /
                  (ipow3(a) + 2 * ipow2(e) * a + 3 * e * ipow2(a) + 2 * ipow2(e) * f + f * ipow2(a) + 3 * f * e * a);
  IP(6, ny - 1) = -(f * ipow2(a) / (a + e) / (2 * e - f) / (2 * e + a));
  IP(7, ny - 1) = 1.0;
  IP(8, ny - 1) = ipow2(e) * f /
                  (4 * ipow3(a) + 2 * ipow2(e) * a + 6 * e * ipow2(a) + 3 * f * e * a + ipow2(e) * f + 2 * f * ipow2(a));
  e = hi[ny] / 2;
  f = e + h[ny];
  g = f + h[ny - 1];
  IP(1, ny) = 2 * ipow2(e) * (2 * e - f) / (e - g) / (f - g) / g;
  IP(2, ny) = -(2 * (2 * e - g) * ipow2(e) / (e - f) / f / (f - g));
  IP(3, ny) = 2 * (4 * ipow2(e) + g * f - 2 * e * f - 2 * g * e) / (ipow2(e) - e * f + g * f - g * e);
  IP(6, ny) = 1.0;
  IP(7, ny) = (4 * ipow2(e) + g * f - 2 * e * f - 2 * g * e) / g / f;
  fd_lu(fiyp, ny, 3, 2);
  fd_lu(fiy, ny, 3, 2);
#undef DV
#undef FX
#undef IX
#undef IY
#undef IP
}

int orc_coef_compute(const otbl_config *cfg, const double *yin, const double *u0in,
                     double *out) {
  if (!cfg || !yin || !u0in || !out) return OTBL_ERR_ARG;
  const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz;
  if (nx < 9 || ny < 9 || nz < 6 || nz % 2) return OTBL_ERR_CONFIG;
  const int nz2 = (2 * (nz / 3)) / 2 - 1;
  if (nz2 < 1) return OTBL_ERR_CONFIG;
  const double re = cfg->re, ax = cfg->ax, az = cfg->az, cfl = cfg->cfl;

  otbl_coef_offsets lay;
  otbl_coef_layout(nx, ny, nz, &lay);
  memset(out, 0, sizeof(double) * lay.off[OTBL_C_COUNT]);
#define ARR(id) (out + lay.off[OTBL_C_##id])
  double *S = ARR(SCAL);
  double *y = ARR(Y), *dy = ARR(DY), *idy = ARR(IDY), *idyy = ARR(IDYY), *dymin = ARR(DYMIN);
  double *hy = ARR(HY), *x = ARR(XG), *dx = ARR(DX);
  double *kaz = ARR(KAZ), *kaz2 = ARR(KAZ2), *kvis = ARR(KVIS), *kmod = ARR(KMOD);
  double *ayp = ARR(AYP), *vmagic = ARR(VMAGIC);
  double *inxu = ARR(INXU), *inxv = ARR(INXV), *inyu = ARR(INYU), *inyv = ARR(INYV);
  double *cofiux = ARR(COFIUX), *cofivx = ARR(COFIVX), *cofiuy = ARR(COFIUY), *cofivy = ARR(COFIVY);
  double *inbx = ARR(INBX), *inby = ARR(INBY);
  double *dcxu = ARR(DCXU), *dcxv = ARR(DCXV), *dcyu = ARR(DCYU), *dcyv = ARR(DCYV);
  double *cofcxu = ARR(COFCXU), *cofcxv = ARR(COFCXV), *cofcyu = ARR(COFCYU), *cofcyv = ARR(COFCYV);
  double *dcbx = ARR(DCBX), *dcby = ARR(DCBY), *ccon = ARR(CCON);
  double *vixu = ARR(VIXU), *vixv = ARR(VIXV), *viyu = ARR(VIYU), *viyv = ARR(VIYV);
  double *vyui = ARR(VYUI), *vyvi = ARR(VYVI);
  double *cofvxu = ARR(COFVXU), *cofvxv = ARR(COFVXV), *cofvyu = ARR(COFVYU), *cofvyv = ARR(COFVYV);
  double *cofvbx = ARR(COFVBX), *cofvby = ARR(COFVBY);
#undef ARR
  /* idyy(1:ny), dymin(1:ny), kmod(1:nx-1), vmagic(1:nx) are stored from
   * index 0; the others with lower bound 0 (y, dy, idy, hy, x, dx, kaz...) */
#define IDYY(j) idyy[(j)-1]
#define DYMIN(j) dymin[(j)-1]
#define KMOD(i) kmod[(i)-1]
#define VMAGIC(i) vmagic[(i)-1]

  /* iniciap_1 wavenumbers, bl_1.F90:357-366 (before coef in bl_1.F90:40,56) */
  for (int k = 0; k <= nz2; ++k) {
    /* cmplx(0d0, k/az): default complex, imaginary part REAL*4 */
    kaz[k] = (double)(float)((double)k / az);
    /* kaz2 = -kaz**2 = -((0 + i s)*(0 + i s)) = -(0*0 - s*s) */
    kaz2[k] = -(0.0 * 0.0 - kaz[k] * kaz[k]);
  }

  const double pi = 4.0 * atan(1.0); /* coeft.f90:27 */
  for (int j = 0; j <= ny + 1; ++j) y[j] = yin[j];

  /* hy, coeft.f90:32-37 */
  for (int j = 1; j <= ny - 1; ++j) hy[j] = (y[j + 1] - y[j - 1]) / 2.5 / 2.0;
  hy[0] = (y[1] - y[0]) / 2.5;
  hy[ny] = (y[ny] - y[ny - 1]) / 2.5;

  /* distances, coeft.f90:397-424 */
  double dyi[ny + 1];  /* dyi(1:ny) */
  double dxi[nx + 1];  /* dxi(0:nx), dxi(0) unused */
  for (int j = 0; j <= ny; ++j) dy[j] = y[j + 1] - y[j];
  for (int j = 1; j <= ny; ++j) dyi[j] = 0.5 * (dy[j] + dy[j - 1]);
  const double point0 = ax * pi / (double)(nx + 1);
  for (int i = 0; i <= nx + 1; ++i) x[i] = (double)i * point0;
  double daux = 1000.0;
  for (int i = 0; i <= nx; ++i) {
    dx[i] = x[i + 1] - x[i];
    daux = daux < dx[i] ? daux : dx[i];
  }
  double dxmin = daux;
  dxi[0] = 0.0;
  for (int i = 1; i <= nx; ++i) dxi[i] = 0.5 * (dx[i] + dx[i - 1]);
  const double idx = 1.0 / dx[1];
  for (int j = 0; j <= ny; ++j) idy[j] = 1.0 / dy[j];
  const double idxx = 1.0 / dx[1];
  for (int j = 1; j <= ny; ++j) IDYY(j) = 2.0 / (dy[j - 1] + dy[j]);

  /* time-step limits, coeft.f90:432-454 */
  daux = 1000.0;
  for (int i = 1; i <= ny; ++i) {
    DYMIN(i) = dy[i] * cfl / sqrt(3.0);
    daux = daux < dy[i] ? daux : dy[i];
  }
  double dzmin = az * 2 * pi / nz;
  const double dtrex = re * (cfl * ipow2(dxmin)) / 6.0;
  const double dtrez = re * (cfl * ipow2(dzmin)) / ipow2(pi);
  const double dtret = dtrex < dtrez ? dtrex : dtrez;
  for (int i = 1; i <= ny; ++i) DYMIN(i) = dy[i] * cfl / sqrt(3.0);
  dxmin = dxmin * cfl / sqrt(3.0);
  dzmin = dzmin * cfl / pi;
  const double rex = -1.0 / re; /* coeft.f90:480 */
  for (int k = 0; k <= nz2; ++k) kvis[k] = rex * kaz2[k];

  /* RK3, coeft.f90:494-508 */
  S[OTBL_S_RKC + 0] = 8.0 / 15.0;  S[OTBL_S_RKC + 1] = 5.0 / 12.0;   S[OTBL_S_RKC + 2] = 3.0 / 4.0;
  S[OTBL_S_RKD + 0] = 0.0;         S[OTBL_S_RKD + 1] = -17.0 / 60.0; S[OTBL_S_RKD + 2] = -5.0 / 12.0;
  S[OTBL_S_RKCV + 0] = 4.0 / 15.0; S[OTBL_S_RKCV + 1] = 1.0 / 15.0;  S[OTBL_S_RKCV + 2] = 1.0 / 6.0;
  S[OTBL_S_RKDV + 0] = 4.0 / 15.0; S[OTBL_S_RKDV + 1] = 1.0 / 15.0;  S[OTBL_S_RKDV + 2] = 1.0 / 6.0;

  double a, b, c, d, aux;
  int i, bad = 0;
  double bcc[6]; /* bcc(1:5) */

  /* interpolation, implicit part, coeft.f90:514-580 */
  for (i = 2; i <= nx - 1; ++i) {
    c = dxi[i + 1]; a = dxi[i]; b = dx[i];
    T3(inxu, 1, i) = c * ipow2(b) / ((2 * a + b) * (-b + 2 * a) * (c + a));
    T3(inxu, 2, i) = 1.0;
    T3(inxu, 3, i) = -(a * ipow2(b) / ((b - 2 * c) * (b + 2 * c) * (c + a)));
  }
  for (i = 2; i <= ny - 1; ++i) {
    a = dy[i]; b = dy[i - 1];
    T3(inyu, 1, i) = ipow2(a) / ((a + b) * (a + 2 * b));
    T3(inyu, 2, i) = 1.0;
    T3(inyu, 3, i) = ipow2(b) / (ipow2(b) + 2 * ipow2(a) + 3 * a * b);
  }
  for (i = 2; i <= nx - 1; ++i) {
    a = dx[i]; b = dx[i - 1];
    T3(inxv, 1, i) = ipow2(a) / ((b + a) * (a + 2.0 * b));
    T3(inxv, 2, i) = 1.0;
    T3(inxv, 3, i) = ipow2(b) / (2.0 * ipow2(a) + ipow2(b) + 3.0 * a * b);
  }
  for (i = 2; i <= ny - 1; ++i) {
    a = dyi[i]; b = dy[i - 1]; c = dyi[i - 1];
    T3(inyv, 1, i) = c * ipow2(b) / ((2 * a + b) * (-b + 2 * a) * (c + a));
    T3(inyv, 2, i) = 1.0;
    T3(inyv, 3, i) = -(a * ipow2(b) / ((b - 2 * c) * (b + 2 * c) * (c + a)));
  }
  T3(inxu, 3, 1) = 0.0;  T3(inxu, 2, 1) = 1.0;  T3(inxu, 1, 1) = 0.0;
  T3(inxu, 1, nx) = 0.0; T3(inxu, 2, nx) = 1.0; T3(inxu, 3, nx) = 0.0;
  T3(inxv, 1, 1) = 0.0;  T3(inxv, 2, 1) = 1.0;  T3(inxv, 3, 1) = 0.0;
  T3(inxv, 1, nx) = 0.0; T3(inxv, 2, nx) = 1.0; T3(inxv, 3, nx) = 0.0;
  T3(inyu, 1, 1) = 0.0;  T3(inyu, 2, 1) = 1.0;  T3(inyu, 3, 1) = 0.0;
  T3(inyu, 1, ny) = 0.0; T3(inyu, 2, ny) = 1.0; T3(inyu, 3, ny) = 0.0;
  T3(inyv, 1, 1) = 0.0;  T3(inyv, 2, 1) = 1.0;  T3(inyv, 3, 1) = 0.0;
  T3(inyv, 1, ny) = 0.0; T3(inyv, 2, ny) = 1.0; T3(inyv, 3, ny) = 0.0;

  /* x closures of the interpolations, coeft.f90:583-624 */
#define PUT_ROW(m, nr, row, ncol)                                        \
  do {                                                                   \
    for (int cc = 1; cc <= (ncol); ++cc) MAT(m, nr, row, cc) = bcc[cc]; \
  } while (0)
  a = dx[nx - 1]; b = dxi[nx - 1]; c = dxi[nx - 2]; d = dxi[nx - 3];
  bad |= f_coefb(3, a, b, c, d, bcc, 0);
  PUT_ROW(inbx, 4, 1, 3); MAT(inbx, 4, 1, 4) = 0.0;
  a = dx[nx]; b = dx[nx - 1]; c = dx[nx - 2]; d = dx[nx - 3];
  bad |= f_coefb(3, a, b, c, d, bcc, 0);
  PUT_ROW(inbx, 4, 2, 3); MAT(inbx, 4, 2, 4) = 0.0;
  a = dx[1]; b = dx[1]; c = dx[2]; d = dx[3];
  bad |= f_coefb(4, a, b, c, d, bcc, 4);
  PUT_ROW(inbx, 4, 3, 4);
  a = dx[0]; b = dx[1]; c = dxi[2]; d = dxi[3];
  bad |= f_coefb(4, a, b, c, d, bcc, 4);
  PUT_ROW(inbx, 4, 4, 4);

  /* y closures of the interpolations, coeft.f90:631-675 */
  a = dy[ny]; b = dy[ny - 1]; c = dyi[ny - 1]; d = dyi[ny - 2];
  bad |= f_coefb(4, a, b, c, d, bcc, 4);
  PUT_ROW(inby, 4, 1, 4);
  a = -dy[0]; b = -dy[1]; c = -dy[2]; d = dy[4];
  bad |= f_coefb(3, a, b, c, d, bcc, 0);
  PUT_ROW(inby, 4, 3, 3); MAT(inby, 4, 3, 4) = 0.0;
  a = dy[0]; b = dy[1]; c = dyi[2]; d = dyi[3];
  bad |= f_coefb(4, a, b, c, d, bcc, 4);
  PUT_ROW(inby, 4, 2, 4);
  a = -dy[ny - 1]; b = -dy[ny - 1]; c = -dy[ny - 2]; d = -dy[ny - 3];
  bad |= f_coefb(4, a, b, c, d, bcc, 4);
  PUT_ROW(inby, 4, 4, 4);

  f_coefinv(inxu, nx, 1);
  f_coefinv(inxv, nx, 1);
  f_coefinv(inyu, ny, 1);
  f_coefinv(inyv, ny, 1);

  /* interpolation, explicit part, coeft.f90:685-713 */
  for (i = 2; i <= ny - 1; ++i) {
    a = dyi[i]; b = dy[i - 1]; c = dyi[i - 1];
    T2(cofivy, 2, i) = (-(2.0 * c * a)) / (2 * a * b + ipow2(b) - 4 * c * a - 2 * c * b);
    T2(cofivy, 1, i) = (2.0 * c * a) / (-ipow2(b) + 2 * a * b - 2 * c * b + 4 * c * a);
    a = dy[i]; b = dy[i - 1];
    T2(cofiuy, 2, i) = 4 * ipow2(b) / (2 * ipow2(b) + ipow2(a) + 3 * a * b);
    T2(cofiuy, 1, i) = 4 * ipow2(a) / ((a + b) * (2 * a + b));
  }
  for (i = 2; i <= nx - 1; ++i) {
    a = dx[i]; b = dx[i - 1];
    T2(cofivx, 2, i) = (4.0 * ipow2(b)) / (2.0 * ipow2(b) + pow(a, 2.0) + 3.0 * a * b);
    T2(cofivx, 1, i) = (4.0 * ipow2(a)) / ((b + a) * (2.0 * a + b));
    c = dxi[i + 1]; a = dxi[i]; b = dx[i];
    T2(cofiux, 2, i) = (-(2.0 * c * a)) / (2 * a * b + ipow2(b) - 4 * c * a - 2 * c * b);
    T2(cofiux, 1, i) = (2.0 * c * a) / (-ipow2(b) + 2 * a * b - 2 * c * b + 4 * c * a);
  }

  /* first derivative, implicit part, coeft.f90:722-784 */
  for (i = 2; i <= nx - 1; ++i) {
    a = dx[i]; b = dx[i - 1];
    aux = 2.0 * ipow3(b) + 2.0 * ipow3(a) + 9.0 * ipow2(b) * a + 9.0 * b * ipow2(a);
    T3(dcxu, 1, i) = -(a * (-(2.0 * a * b) - ipow2(b) + 2.0 * ipow2(a)) / aux);
    T3(dcxu, 2, i) = 1.0;
    T3(dcxu, 3, i) = ((ipow2(a) + 2.0 * a * b - 2.0 * ipow2(b)) * b) / aux;
  }
  T3(dcxu, 2, 1) = 1.0;  T3(dcxu, 1, 1) = 0.0;  T3(dcxu, 3, 1) = 0.0;
  T3(dcxu, 2, nx) = 1.0; T3(dcxu, 1, nx) = 0.0; T3(dcxu, 3, nx) = 0.0;
  for (i = 2; i <= ny; ++i) {
    a = dyi[i]; b = dyi[i - 1]; c = dy[i - 1];
    aux = -(ipow2(c) * a) - ipow2(c) * b + 12.0 * ipow2(b) * a + 12.0 * b * ipow2(a);
    T3(dcyu, 1, i) = (b * ipow2(c)) / aux;
    T3(dcyu, 2, i) = 1.0;
    T3(dcyu, 3, i) = (ipow2(c) * a) / aux;
  }
  T3(dcyu, 2, 1) = 1.0;      T3(dcyu, 3, 1) = 0.0;      T3(dcyu, 1, 1) = 0.0;
  T3(dcyu, 2, ny + 1) = 1.0; T3(dcyu, 3, ny + 1) = 0.0; T3(dcyu, 1, ny + 1) = 0.0;
  for (i = 2; i <= nx - 1; ++i) {
    a = dxi[i]; b = dxi[i - 1]; c = dx[i - 1];
    aux = -(ipow2(c) * a) - ipow2(c) * b + 12.0 * ipow2(b) * a + 12.0 * b * ipow2(a);
    T3(dcxv, 1, i) = (b * ipow2(c)) / aux;
    T3(dcxv, 2, i) = 1.0;
    T3(dcxv, 3, i) = (ipow2(c) * a) / aux;
  }
  T3(dcxv, 2, 1) = 1.0;  T3(dcxv, 3, 1) = 0.0;  T3(dcxv, 1, 1) = 0.0;
  T3(dcxv, 2, nx) = 1.0; T3(dcxv, 3, nx) = 0.0; T3(dcxv, 1, nx) = 0.0;
  for (i = 2; i <= ny - 1; ++i) {
    a = dy[i]; b = dy[i - 1];
    aux = 2.0 * ipow3(b) + 2.0 * ipow3(a) + 9.0 * ipow2(b) * a + 9.0 * b * ipow2(a);
    T3(dcyv, 1, i) = -(a * (-(2.0 * a * b) - ipow2(b) + 2.0 * ipow2(a)) / aux);
    T3(dcyv, 2, i) = 1.0;
    T3(dcyv, 3, i) = ((ipow2(a) + 2.0 * a * b - 2.0 * ipow2(b)) * b) / aux;
  }
  T3(dcyv, 2, 1) = 1.0;  T3(dcyv, 3, 1) = 0.0;  T3(dcyv, 1, 1) = 0.0;
  T3(dcyv, 2, ny) = 1.0; T3(dcyv, 3, ny) = 0.0; T3(dcyv, 1, ny) = 0.0;

  /* first-derivative closures, coeft.f90:787-924 */
  a = dx[1]; b = dxi[2]; c = dxi[3]; d = dxi[4];
  bad |= f_coefb(4, a, b, c, d, bcc, 3);
  PUT_ROW(dcbx, 5, 1, 4);
  a = dx[0]; b = dx[1]; c = dx[2]; d = dx[3];
  bad |= f_coefb(4, a, b, c, d, bcc, 3);
  PUT_ROW(dcbx, 5, 2, 4);
  a = dx[nx]; b = dx[nx - 1]; c = dxi[nx - 1]; d = dxi[nx - 2];
  bad |= f_coefb(4, a, b, c, d, bcc, 5);
  PUT_ROW(dcbx, 5, 3, 4);
  a = dx[nx - 1]; b = dx[nx - 1]; c = dx[nx - 2]; d = dx[nx - 3];
  bad |= f_coefb(4, a, b, c, d, bcc, 5);
  PUT_ROW(dcbx, 5, 4, 4);
  a = -dx[nx - 1]; b = -dxi[nx - 1]; c = -dxi[nx - 2]; d = -dxi[nx - 3];
  bad |= f_coefb(4, a, b, c, d, bcc, 5);
  PUT_ROW(dcbx, 5, 5, 4);

  a = -dy[0]; b = -dy[1]; c = -dyi[2]; d = -dyi[3];
  bad |= f_coefb(4, a, b, c, d, bcc, 5);
  PUT_ROW(dcby, 4, 1, 4);
  a = -dy[ny - 1]; b = -dyi[ny - 1]; c = -dyi[ny - 2]; d = -dyi[ny - 3];
  bad |= f_coefb(4, a, b, c, d, bcc, 3);
  PUT_ROW(dcby, 4, 2, 4);
  a = dy[0]; b = dy[1]; c = dy[2]; d = dy[3];
  bad |= f_coefb(4, a, b, c, d, bcc, 3);
  PUT_ROW(dcby, 4, 3, 4);
  a = -dy[ny]; b = -dy[ny - 1]; c = -dy[ny - 2]; d = -dy[ny - 3];
  bad |= f_coefb(4, a, b, c, d, bcc, 3);
  PUT_ROW(dcby, 4, 4, 4);
  a = -dy[ny - 1]; b = -dyi[ny - 1]; c = -dyi[ny - 2]; d = -dyi[ny - 3];
  bad |= f_coefb(4, a, b, c, d, bcc, 3); /* row 2 again, coeft.f90:889-898 */
  PUT_ROW(dcby, 4, 2, 4);

  /* zero-vorticity closures, coeft.f90:901-924 */
  a = dy[ny]; b = dy[ny - 1]; c = dyi[ny - 1]; d = dyi[ny - 2];
  bad |= f_coefb(4, a, b, c, d, bcc, 7);
  PUT_ROW(ccon, 2, 1, 4);
  a = -dy[0]; b = -dyi[1]; c = -dyi[2]; d = 0.0;
  bad |= f_coefb(4, a, b, c, d, bcc, 6);
  PUT_ROW(ccon, 2, 2, 4);

  f_coefinv(dcxu, nx, 1);
  f_coefinv(dcxv, nx, 1);
  f_coefinv(dcyu, ny + 1, 1);
  f_coefinv(dcyv, ny, 1);

  /* first derivative, explicit part, coeft.f90:933-965 */
  for (i = 2; i <= ny - 1; ++i) {
    a = dy[i]; b = dy[i - 1];
    aux = 2.0 * ipow3(b) + 2.0 * ipow3(a) + 9.0 * ipow2(b) * a + 9.0 * b * ipow2(a);
    T2(cofcyv, 1, i) = -(24 * a * b / aux);
    T2(cofcyv, 2, i) = 24 * a * b / aux;
    a = dyi[i]; b = dyi[i - 1]; c = dy[i - 1];
    T2(cofcyu, 1, i) = -(12.0 * a * b / ((12.0 * a * b - ipow2(c)) * c));
    T2(cofcyu, 2, i) = 12.0 * a * b / ((12.0 * a * b - ipow2(c)) * c);
  }
  /* the loop leaves i = ny: zeroed, then recomputed at i = ny */
  T2(cofcyu, 1, i) = 0.0;
  T2(cofcyu, 2, i) = 0.0;
  i = ny;
  a = dyi[i]; b = dyi[i - 1]; c = dy[i - 1];
  T2(cofcyu, 1, i) = -(12.0 * a * b / ((12.0 * a * b - ipow2(c)) * c));
  T2(cofcyu, 2, i) = 12.0 * a * b / ((12.0 * a * b - ipow2(c)) * c);
  for (i = 2; i <= nx - 1; ++i) {
    a = dxi[i]; b = dxi[i - 1]; c = dx[i - 1];
    T2(cofcxv, 1, i) = -(12.0 * a * b / ((12.0 * a * b - ipow2(c)) * c));
    T2(cofcxv, 2, i) = 12.0 * a * b / ((12.0 * a * b - ipow2(c)) * c);
    a = dx[i]; b = dx[i - 1];
    aux = 2.0 * ipow3(b) + 2.0 * ipow3(a) + 9.0 * ipow2(b) * a + 9.0 * b * ipow2(a);
    T2(cofcxu, 1, i) = -(24 * a * b / aux);
    T2(cofcxu, 2, i) = 24 * a * b / aux;
  }

  /* second derivative, implicit part, coeft.f90:971-1018 */
#define VISL(A, B) ((B) * (ipow2(A) + (A) * (B) - ipow2(B)) / \
                    (ipow3(B) + ipow3(A) + 4 * ipow2(A) * (B) + 4 * (A) * ipow2(B)))
#define VISU(A, B) (-((ipow2(A) - (A) * (B) - ipow2(B)) * (A) / \
                      (ipow3(B) + ipow3(A) + 4 * ipow2(A) * (B) + 4 * (A) * ipow2(B))))
  for (i = 2; i <= nx - 1; ++i) {
    a = dx[i]; b = dx[i - 1];
    T3(vixu, 1, i) = VISL(a, b); T3(vixu, 2, i) = 1.0; T3(vixu, 3, i) = VISU(a, b);
  }
  T3(vixu, 1, 1) = 0.0; T3(vixu, 2, 1) = 1.0; T3(vixu, 3, nx) = 0.0; T3(vixu, 2, nx) = 1.0;
  for (i = 2; i <= ny; ++i) {
    a = dyi[i]; b = dyi[i - 1];
    T3(viyu, 1, i) = VISL(a, b); T3(viyu, 2, i) = 1.0; T3(viyu, 3, i) = VISU(a, b);
  }
  T3(viyu, 1, 1) = 0.0; T3(viyu, 2, 1) = 1.0; T3(viyu, 3, ny + 1) = 0.0; T3(viyu, 2, ny + 1) = 1.0;
  for (i = 2; i <= nx - 1; ++i) {
    a = dxi[i]; b = dxi[i - 1];
    T3(vixv, 1, i) = VISL(a, b); T3(vixv, 2, i) = 1.0; T3(vixv, 3, i) = VISU(a, b);
  }
  T3(vixv, 1, 1) = 0.0; T3(vixv, 2, 1) = 1.0; T3(vixv, 3, nx) = 0.0; T3(vixv, 2, nx) = 1.0;
  for (i = 2; i <= ny - 1; ++i) {
    a = dy[i]; b = dy[i - 1];
    T3(viyv, 1, i) = VISL(a, b); T3(viyv, 2, i) = 1.0; T3(viyv, 3, i) = VISU(a, b);
  }
  T3(viyv, 1, 1) = 0.0; T3(viyv, 2, 1) = 1.0; T3(viyv, 3, ny) = 0.0; T3(viyv, 2, ny) = 1.0;
#undef VISL
#undef VISU

  /* second-derivative closures, coeft.f90:1023-1113 (flag 1 ignores d) */
  a = dxi[1]; b = dxi[2]; c = dxi[3];
  bad |= f_coefb(5, a, b, c, d, bcc, 1);
  T3(vixv, 3, 1) = bcc[1];
  for (int cc = 1; cc <= 4; ++cc) MAT(cofvbx, 4, 1, cc) = bcc[cc + 1];
  a = dxi[nx - 1]; b = dxi[nx - 2]; c = dxi[nx - 3];
  bad |= f_coefb(5, a, b, c, d, bcc, 1);
  T3(vixv, 1, nx) = bcc[1];
  for (int cc = 1; cc <= 4; ++cc) MAT(cofvbx, 4, 2, cc) = bcc[cc + 1];
  a = dx[1]; b = dx[2]; c = dx[3];
  bad |= f_coefb(5, a, b, c, d, bcc, 1);
  T3(vixu, 3, 1) = bcc[1];
  for (int cc = 1; cc <= 4; ++cc) MAT(cofvbx, 4, 3, cc) = bcc[cc + 1];
  a = dx[nx - 1]; b = dx[nx - 2]; c = dx[nx - 3];
  bad |= f_coefb(5, a, b, c, d, bcc, 1);
  T3(vixu, 1, nx) = bcc[1];
  for (int cc = 1; cc <= 4; ++cc) MAT(cofvbx, 4, 4, cc) = bcc[cc + 1];
  a = dy[1]; b = dy[2]; c = dy[3];
  bad |= f_coefb(5, a, b, c, d, bcc, 1);
  T3(viyv, 3, 1) = bcc[1];
  for (int cc = 1; cc <= 4; ++cc) MAT(cofvby, 4, 1, cc) = bcc[cc + 1];
  a = dy[ny - 1]; b = dy[ny - 2]; c = dy[ny - 3];
  bad |= f_coefb(5, a, b, c, d, bcc, 1);
  T3(viyv, 1, ny) = bcc[1];
  for (int cc = 1; cc <= 4; ++cc) MAT(cofvby, 4, 2, cc) = bcc[cc + 1];
  a = dyi[1]; b = dyi[2]; c = dyi[3];
  bad |= f_coefb(5, a, b, c, d, bcc, 1);
  T3(viyu, 3, 1) = bcc[1];
  for (int cc = 1; cc <= 4; ++cc) MAT(cofvby, 4, 3, cc) = bcc[cc + 1];
  a = dyi[ny]; b = dyi[ny - 1]; c = dyi[ny - 2];
  bad |= f_coefb(5, a, b, c, d, bcc, 1);
  T3(viyu, 1, ny + 1) = bcc[1];
  for (int cc = 1; cc <= 4; ++cc) MAT(cofvby, 4, 4, cc) = bcc[cc + 1];

  /* unfactored copies for implzy, coeft.f90:1116-1127 */
  for (i = 1; i <= ny; ++i)
    for (int r = 1; r <= 3; ++r) {
      T3(vyui, r, i) = T3(viyu, r, i);
      T3(vyvi, r, i) = T3(viyv, r, i);
    }
  for (int r = 1; r <= 3; ++r) T3(vyui, r, ny + 1) = T3(viyu, r, ny + 1);

  f_coefinv(vixu, nx, 1);
  f_coefinv(vixv, nx, 1);
  f_coefinv(viyu, ny + 1, 1);
  f_coefinv(viyv, ny, 1);

  /* second derivative, explicit part, coeft.f90:1136-1168 */
#define VISE(M, I, A, B)                                                                   \
  do {                                                                                     \
    const double den_ = ipow3(B) + ipow3(A) + 4 * ipow2(A) * (B) + 4 * (A) * ipow2(B);   \
    T3(M, 1, I) = 12 * (B) / den_;                                                         \
    T3(M, 2, I) = -(12 / (ipow2(A) + 3 * (A) * (B) + ipow2(B)));                           \
    T3(M, 3, I) = 12 * (A) / den_;                                                         \
  } while (0)
  for (i = 2; i <= ny - 1; ++i) VISE(cofvyv, i, dy[i], dy[i - 1]);
  for (i = 2; i <= ny; ++i) VISE(cofvyu, i, dyi[i], dyi[i - 1]);
  for (i = 2; i <= nx - 1; ++i) {
    VISE(cofvxv, i, dxi[i], dxi[i - 1]);
    VISE(cofvxu, i, dx[i], dx[i - 1]);
  }
#undef VISE

  /* DCT eigenvalues, coeft.f90:1181-1183 */
  for (i = 1; i <= nx - 1; ++i)
    KMOD(i) = 2.0 / ipow2(dx[1]) * (1 - cos((pi * (i - 1)) / (double)(nx - 1)));

  /* mtr, coeft.f90:1244-1332; pois uses the finest level ngy2(1) = ny-1 */
  {
    double ac2 = 0.0, bc2 = 0.0, ac1, bc1, dy1, dy2, a3, b2;
    ac1 = ac2; bc1 = bc2;
    dy1 = y[2] - y[1];
    dy2 = y[3] - y[2];
    a3 = 1.0 / dy1; b2 = -1.0 / dy1;
    ac2 = 2.0 / (dy1 + dy2); bc2 = -2.0 / (dy1 + dy2);
    T3(ayp, 1, 1) = b2 * bc1;
    T3(ayp, 3, 1) = a3 * ac2;
    T3(ayp, 2, 1) = a3 * bc2 + b2 * ac1;
    const int ngy = ny - 1;
    for (int iy = 2; iy <= ngy - 1; ++iy) {
      ac1 = ac2; bc1 = bc2;
      dy1 = y[iy + 1] - y[iy];
      dy2 = y[iy + 2] - y[iy + 1];
      a3 = 1.0 / dy1; b2 = -1.0 / dy1;
      ac2 = 2.0 / (dy1 + dy2); bc2 = -2.0 / (dy1 + dy2);
      T3(ayp, 1, iy) = b2 * bc1;
      T3(ayp, 3, iy) = a3 * ac2;
      T3(ayp, 2, iy) = a3 * bc2 + b2 * ac1;
    }
    const int lt = ngy;
    b2 = -1.0 / dy2;
    ac1 = ac2; bc1 = bc2;
    T3(ayp, 1, lt) = b2 * bc1;
    T3(ayp, 3, lt) = 0.0;
    T3(ayp, 2, lt) = b2 * ac1;
  }

  /* inlet_retheta, bl_1.F90:380-388 */
  double rthin, din;
  {
#define U0(j) u0in[(j)-1] /* u0(1:ny+1) */
    double uinf = 0.0;
    for (int j = ny + 1 - 20; j <= ny + 1 - 5; ++j) uinf += U0(j);
    uinf = uinf / 16.0;
    const double u99 = (double)0.99f * uinf;
    int jtop = 1; /* unset in the reference if u0(1) >= u99 already */
    for (int j = 1; j <= ny - 2; ++j) {
      if (U0(j) >= u99) break;
      jtop = j + 1;
    }
    din = y[jtop];
    double s = 0.0;
    for (int t = 1; t <= jtop + 2; ++t) s += (uinf - U0(t + 1)) * U0(t + 1) * dy[t];
    rthin = s * re / uinf;
#undef U0
  }

  /* magicnumber, boun.f90:114-140 */
  {
    const double e1 = 0.8659, c1 = 0.01277, ei1 = 1 / e1;
    const double kap = 0.384, ckap = 4.127, cprim = 7.135;
    const double dxm = ax * pi / (nx - 1);
    double xm[nx + 1], hm[nx + 1];
    for (i = 1; i <= nx; ++i) {
      xm[i] = dxm * (i - 1);
      const double reth = pow(pow(rthin, ei1) + pow(c1, ei1) * re * xm[i], e1);
      const double uep = log(reth) / kap + ckap;
      hm[i] = reth / ((1 - cprim / uep) * re);
    }
    VMAGIC(1) = (hm[2] - hm[1]) / (xm[2] - xm[1]);
    for (i = 2; i <= nx - 1; ++i) VMAGIC(i) = (hm[i + 1] - hm[i - 1]) / (xm[i + 1] - xm[i - 1]);
    VMAGIC(nx) = (hm[nx] - hm[nx - 1]) / (xm[nx] - xm[nx - 1]);
  }

  f_fd_operators(nx, ny, ax, pi, y, out + lay.off[OTBL_C_FD_DVDY], out + lay.off[OTBL_C_FD_DX],
                 out + lay.off[OTBL_C_FD_IX], out + lay.off[OTBL_C_FD_IY], out + lay.off[OTBL_C_FD_IYP]);

  S[OTBL_S_RE] = re;
  S[OTBL_S_REX] = rex;
  S[OTBL_S_AX] = ax;
  S[OTBL_S_AY] = cfg->ay;
  S[OTBL_S_AZ] = az;
  S[OTBL_S_CFL] = cfl;
  S[OTBL_S_DX1] = dx[1];
  S[OTBL_S_IDX] = idx;
  S[OTBL_S_IDXX] = idxx;
  S[OTBL_S_DXMIN] = dxmin;
  S[OTBL_S_DZMIN] = dzmin;
  S[OTBL_S_DTRET] = dtret;
  S[OTBL_S_PI] = pi;
  S[OTBL_S_UINF] = 1.0; /* Uinfinity, mod.F90:47 */
  S[OTBL_S_RTHIN] = rthin;
  S[OTBL_S_DIN] = din;
  S[OTBL_S_YBLEND] = cfg->y_blend;
  S[OTBL_S_NX] = nx;
  S[OTBL_S_NY] = ny;
  S[OTBL_S_NZ] = nz;
  S[OTBL_S_XOUT] = cfg->xout;
#undef IDYY
#undef DYMIN
#undef KMOD
#undef VMAGIC
#undef PUT_ROW
  return bad ? OTBL_ERR_CONFIG : OTBL_OK;
}
