// Host-side setup of every coefficient the RK3 substep reads.
//
// Restates, in C++, the reference's setup routines that fill module alloc_dns
// once per run (bl_1.F90:56-58):
//   coef        coeft.f90:10-1234   grid metrics, compact-scheme coefficients,
//                                   RK3 constants, DCT eigenvalues, y-Poisson
//   coefb       coeft.f90:1360-1789 boundary closures (small dense solves)
//   ludcmp      coeft.f90:1818-1883 Crout LU with implicit pivoting
//   lubksb      coeft.f90:1890-1922 LU back substitution
//   coefinv     coeft.f90:1338-1353 Thomas pre-factorisation
//   mtr         coeft.f90:1244-1332 y-Poisson operator ayp
//   inlet_retheta bl_1.F90:372-396  inlet Re_theta and delta99
//   magicnumber boun.f90:102-143    top transpiration vmagic(x)
//   wavenumbers bl_1.F90:357-366    kaz = i*k/az, kaz2 = -kaz**2
//   fd_*        coeft.f90:56-318    the compact operators of the one-point
//                                   statistics (statsp), which the substep
//                                   itself does not read
// The pressure-extrapolation weights of coef (l_weight, ldyy) are not built:
// nothing here reads them.
//
// Output is the packed buffer described in include/otbl_layout.h, uploaded
// to the device by otbl_ctx_create. Fortran semantics are kept where they
// change bits: integer powers as gfortran expands them, Fortran precedence,
// and the single-precision kaz of cmplx() without KIND (bl_1.F90:360).

#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/otbl.h"
#include "../../include/otbl_layout.h"

namespace {

// Fortran-style accessors. A3(a,r,i): a(r,i) of an a(3,lb:ub) array whose
// first stored column is `lb`.
struct Arr3 {
  double *p;
  int lb;
  double &operator()(int r, int i) const { return p[(size_t)(i - lb) * 3 + (r - 1)]; }
};
struct Arr2 {
  double *p;
  int lb;
  double &operator()(int r, int i) const { return p[(size_t)(i - lb) * 2 + (r - 1)]; }
};
// small fixed (nr, 4 or 5) matrices, column-major: m(r,c) at (c-1)*nr + r-1
struct Mat {
  double *p;
  int nr;
  double &operator()(int r, int c) const { return p[(size_t)(c - 1) * nr + (r - 1)]; }
};

inline double sq(double a) { return a * a; }
inline double cu(double a) { return a * a * a; }
// x**4 as gfortran expands an integer power: (x*x)*(x*x)
inline double p4(double a) {
  const double s = a * a;
  return s * s;
}

// x**5 as gfortran expands an integer power: x**3 * x**2
inline double p5(double a) {
  const double s = a * a;
  return (s * a) * s;
}

// An (8, n) compact operator of the statistics: weights of the explicit
// stencil in rows 1..5, the tridiagonal's sub-, main and super-diagonal in
// rows 6..8 (coeft.f90:56-318).
struct Op8 {
  double *p;
  double &operator()(int r, int j) const { return p[(size_t)(j - 1) * 8 + (r - 1)]; }
  // the LU reorganisation done after each operator (coeft.f90:146-150,
  // 188-192, 222-226, 304-316): eliminate from row j0 on, then invert the
  // pivots of rows inv0..n
  void factor(int n, int j0, int inv0) const {
    const Op8 &c = *this;
    for (int j = j0; j <= n; ++j) {
      c(6, j) = c(6, j) / c(7, j - 1);
      c(7, j) = c(7, j) - c(6, j) * c(8, j - 1);
    }
    for (int j = inv0; j <= n; ++j) c(7, j) = 1.0 / c(7, j);
  }
};

// fd_dvdy, fd_dx, fd_ix, fd_iy, fd_iyp of coeft.f90:56-318, in the
// Fortran's order of operations (negation, commuted sums b - c for -c+b and
// the like change no bits)
void fd_operators(int nx, int ny, double ax, double pi, const double *y, Op8 dv, Op8 dx, Op8 ix, Op8 iy,
                  Op8 ip) {
  std::vector<double> hv(ny + 2), hiv(ny + 2), ypv(ny + 2);
  double *h = hv.data(), *hi = hiv.data(), *yp = ypv.data();  // (1:ny+1)
  double a, b, c, d, e, f, g;

  // d/dy at the v rows (non-uniform mesh), coeft.f90:56-150
  for (int j = 1; j <= ny + 1; ++j) h[j] = y[j] - y[j - 1];
  a = h[2], b = h[2] + h[3], c = h[2] + h[3] + h[4];
  dv(1, 1) = -(a * b + a * c + 2 * b * c) / b / a / c;
  dv(3, 1) = -(sq(a) * c / (b - c) / b / sq(a - b));
  dv(4, 1) = sq(a) * b / c / sq(a - c) / (b - c);
  dv(2, 1) = -(dv(1, 1) + dv(3, 1) + dv(4, 1));
  dv(7, 1) = 1.0;
  dv(8, 1) = b * c / (a - c) / (a - b);
  dv(1, 2) = sq(a - b) * (a - c) * (a * b + 2 * a * c + 2 * b * c) / a / cu(b) / sq(c);
  dv(2, 2) = 1 / a * (-3 * a * b + 2 * b * c + 5 * sq(a) - 4 * a * c) / (a - c) / (a - b);
  dv(3, 2) = sq(a) * (a - c) * (-2 * a * c + 3 * a * b + 4 * b * c - 5 * sq(b)) / cu(b) / sq(b - c) / (a - b);
  dv(4, 2) = -(dv(1, 2) + dv(2, 2) + dv(3, 2));
  dv(6, 2) = -(sq(a - b) * (a - c) / c / sq(b));
  dv(7, 2) = 1.0;
  dv(8, 2) = sq(a) * (a - c) / (b - c) / sq(b);
  for (int i = 3; i <= ny - 2; ++i) {
    a = h[i - 1], b = h[i], c = h[i + 1], d = h[i + 2];
    f = c + d, e = a + b;
    const double qb = sq(b) + 2 * b * c + sq(c), qe = sq(e) - 2 * e * b + sq(b);
    dv(1, i) = -(sq(c) * sq(b) * f / (f + e) / e / (sq(c) + 2 * c * e + sq(e)) / qe);
    dv(2, i) = f / b * e * sq(c) *
               (3 * c * b * f - 2 * c * f * e + 4 * sq(b) * c - 3 * b * e * c + 5 * sq(b) * f - 4 * b * e * f +
                6 * cu(b) - 5 * e * sq(b)) /
               (sq(f) + 2 * b * f + sq(b)) / (cu(b) + 3 * b * sq(c) + cu(c) + 3 * sq(b) * c) / qe;
    dv(3, i) = (c * b * f - b * e * c - 2 * b * e * f + 2 * c * f * e) / f / b / e / c;
    dv(4, i) = -((-3 * c * b * f - 2 * b * e * f + 3 * b * e * c + 4 * b * sq(c) - 5 * sq(c) * f - 4 * c * f * e +
                  6 * cu(c) + 5 * sq(c) * e) *
                 sq(b) / c * e * f / (sq(f) - 2 * f * c + sq(c)) /
                 (3 * sq(e) * b * sq(c) + 6 * e * sq(b) * sq(c) + 6 * e * b * cu(c) + sq(e) * cu(b) + p5(c) +
                  2 * p4(c) * e + cu(c) * sq(e) + 3 * sq(b) * cu(c) + cu(b) * sq(c) + 3 * b * p4(c) +
                  2 * e * cu(b) * c + 3 * sq(e) * sq(b) * c));
    dv(5, i) = -(dv(1, i) + dv(2, i) + dv(3, i) + dv(4, i));
    dv(6, i) = -(e * sq(c) * f / (f + b) / qb / (b - e));
    dv(7, i) = 1.0;
    dv(8, i) = -(e * sq(b) * f / (c - f) / qb / (c + e));
  }
  a = h[ny - 2], b = h[ny - 1], c = h[ny];
  f = a + b + c, e = b + c;
  dv(1, ny - 1) = sq(c) * sq(c - e) / sq(f) / sq(f - e) / (c - f);
  dv(3, ny - 1) = -((5 * sq(c) - 4 * f * c - 3 * c * e + 2 * f * e) / c / (c - f) / (c - e));
  dv(4, ny - 1) = -(sq(c - e) * (c - f) * (2 * f * c + c * e + 2 * f * e) / c / sq(f) / cu(e));
  dv(2, ny - 1) = -(dv(1, ny - 1) + dv(3, ny - 1) + dv(4, ny - 1));
  dv(6, ny - 1) = -((c - f) * sq(c) / sq(e) / (f - e));
  dv(7, ny - 1) = 1.0;
  dv(8, ny - 1) = -(sq(c - e) * (c - f) / f / sq(e));
  dv(1, ny) = sq(c) * e / sq(c - f) / (f - e) / f;
  dv(2, ny) = -(sq(c) * f / e / sq(c - e) / (f - e));
  dv(4, ny) = (f * c + c * e + 2 * f * e) / c / f / e;
  dv(3, ny) = -(dv(1, ny) + dv(2, ny) + dv(4, ny));
  dv(6, ny) = f * e / (c - f) / (c - e);
  dv(7, ny) = 1.0;
  dv.factor(ny, 2, 1);

  // d/dx on the uniform x grid, coeft.f90:153-194: boundary rows 1, 2,
  // nx-1, nx, the sixth-order interior scheme, weights divided by dx
  {
    const double r1[8] = {-37.0 / 12.0, 2.0 / 3.0, 3.0, -2.0 / 3.0, 1.0 / 12.0, 0.0, 1.0, 4.0};
    const double r2[8] = {-43.0 / 96.0, -5.0 / 6.0, 9.0 / 8.0, 1.0 / 6.0, -1.0 / 96.0, 1.0 / 8.0, 1.0, 3.0 / 4.0};
    const double rm[8] = {-1.0 / 36.0, -7.0 / 9.0, 0.0, 7.0 / 9.0, 1.0 / 36.0, 1.0 / 3.0, 1.0, 1.0 / 3.0};
    const double rn1[8] = {1.0 / 96.0, -1.0 / 6.0, -9.0 / 8.0, 5.0 / 6.0, 43.0 / 96.0, 3.0 / 4.0, 1.0, 1.0 / 8.0};
    const double rn[8] = {-1.0 / 12.0, 2.0 / 3.0, -3.0, -2.0 / 3.0, 37.0 / 12.0, 4.0, 1.0, 0.0};
    for (int i = 1; i <= nx; ++i) {
      const double *r = i == 1 ? r1 : (i == 2 ? r2 : (i == nx - 1 ? rn1 : (i == nx ? rn : rm)));
      for (int k = 1; k <= 8; ++k) dx(k, i) = r[k - 1];
    }
    const double point0 = ax * pi / (nx + 1);
    for (int i = 1; i <= nx; ++i)
      for (int k = 1; k <= 5; ++k) dx(k, i) = dx(k, i) / point0;
    dx.factor(nx, 2, 1);
  }

  // mid-point interpolation in x, coeft.f90:196-228
  {
    const double r1[8] = {5.0 / 24.0, 15.0 / 8.0, 5.0 / 8.0, -1.0 / 24.0, 0.0, 0.0, 1.0, 5.0 / 3.0};
    const double rm[8] = {1.0 / 20.0, 3.0 / 4.0, 3.0 / 4.0, 1.0 / 20.0, 0.0, 3.0 / 10.0, 1.0, 3.0 / 10.0};
    const double rn1[8] = {-1.0 / 84.0, 1.0 / 4.0, 5.0 / 4.0, 5.0 / 12.0, 0.0, 5.0 / 6.0, 1.0, 1.0 / 14.0};
    const double rn[8] = {1.0 / 8.0, -7.0 / 8.0, 35.0 / 8.0, 35.0 / 8.0, 0.0, 7.0, 1.0, 0.0};
    for (int i = 1; i <= nx; ++i) {
      const double *r = i == 1 ? r1 : (i == nx - 1 ? rn1 : (i == nx ? rn : rm));
      for (int k = 1; k <= 8; ++k) ix(k, i) = r[k - 1];
    }
    ix.factor(nx, 2, 1);
  }

  // mid-point interpolation in y onto the wall positions y(j): fd_iy for
  // u and w (u-type rows at yp), fd_iyp for p, coeft.f90:231-318
  for (int j = 1; j <= ny + 1; ++j) yp[j] = (y[j - 1] + y[j]) * 0.5;
  for (int j = 1; j <= ny + 1; ++j) hi[j] = y[j] - y[j - 1];
  for (int j = 2; j <= ny + 1; ++j) h[j] = yp[j] - yp[j - 1];
  a = hi[2] / 2, b = a + h[3], c = b + h[4], d = c + h[5];
  iy(1, 1) = -(c * b * d / (a - d) / (a - c) / (a - b));
  iy(2, 1) = c * a * d / (b - d) / (b - c) / (a - b);
  iy(3, 1) = -(b * a * d / (c - d) / (sq(c) - a * c - b * c + b * a));
  iy(4, 1) = 1.0 - (iy(1, 1) + iy(2, 1) + iy(3, 1));
  a = hi[3] / 2, b = a + h[4], c = b + h[5], d = c + h[6], e = hi[2] / 2;
  iy(1, 2) = 2 * c * b * sq(a) * d / (e + d) / (e + c) / (b + e) / (2 * sq(a) + sq(e) + 3 * e * a);
  iy(2, 2) = -(2 * c * b * e * d / (a - d) / (a - c) / (a - b) / (a + e));
  iy(3, 2) = 2 * c * e * sq(a) * d / (b - d) / (b - c) /
             (2 * sq(a) * e + 2 * sq(a) * b - 3 * a * sq(b) - 3 * a * e * b + cu(b) + e * sq(b));
  iy(4, 2) = -(2 * sq(a) * b * e * d / (c - d) /
               (3 * e * a * sq(c) - 2 * e * sq(a) * c - 3 * b * e * a * c - 2 * sq(a) * sq(c) + 2 * sq(a) * e * b +
                3 * a * cu(c) + b * cu(c) - e * cu(c) + 2 * b * sq(a) * c - 3 * b * a * sq(c) + b * e * sq(c) -
                p4(c)));
  iy(7, 2) = 1.0;
  iy(8, 2) = -(c * b * e * d / (2 * a + e) / (2 * a - d) / (2 * a - c) / (2 * a - b));
  iy(5, 2) = (iy(7, 2) + iy(8, 2)) - (iy(1, 2) + iy(2, 2) + iy(3, 2) + iy(4, 2));
  for (int j = 3; j <= ny - 1; ++j) {
    a = hi[j + 1] / 2, b = a + h[j + 2], e = hi[j] / 2, f = e + h[j];
    iy(1, j) = 4 * sq(e) * sq(a) * b / (b + f) /
               (2 * sq(a) * sq(f) + p4(f) + 4 * sq(e) * sq(a) - 6 * sq(a) * e * f - 9 * e * a * sq(f) +
                6 * sq(e) * a * f + 2 * sq(e) * sq(f) + 3 * a * cu(f) - 3 * e * cu(f));
    iy(2, j) = -(4 * f * sq(a) * b / (b + e) / (a + e) / (e - f) / (2 * a + e));
    iy(3, j) = -(4 * f * sq(e) * b / (a - b) / (a + f) / (2 * sq(e) + sq(a) + 3 * e * a));
    iy(6, j) = -(f * b * sq(a) / (a + e) / (2 * e - f) / (b + 2 * e) / (a + 2 * e));
    iy(7, j) = 1.0;
    iy(8, j) = -(f * sq(e) * b / (2 * a - b) / (2 * a + f) / (2 * sq(a) + sq(e) + 3 * e * a));
    iy(4, j) = (iy(6, j) + iy(7, j) + iy(8, j)) - (iy(1, j) + iy(2, j) + iy(3, j));
  }
  a = hi[ny + 1] / 2, e = hi[ny] / 2, f = e + h[ny], g = f + h[ny - 1];
  const double top = 8 * cu(e) - 4 * g * sq(e) - 2 * f * a * e - 2 * g * e * a - 4 * f * sq(e) + g * a * f +
                     4 * a * sq(e) + 2 * f * g * e;
  iy(1, ny) = 2 * (4 * sq(e) + 2 * e * a - a * f - 2 * f * e) * sq(e) / (e - g) / (f - g) / g / (g + a);
  iy(2, ny) = -(2 * (2 * e * a + 4 * sq(e) - a * g - 2 * g * e) * sq(e) / (e - f) / f /
                (sq(f) + a * f - g * f - a * g));
  iy(3, ny) = 2 * top / (cu(e) + a * sq(e) - f * sq(e) - g * sq(e) + g * a * f - g * e * a + f * g * e - f * a * e);
  iy(4, ny) = 2 * (-2 * f * e - 2 * g * e + g * f + 4 * sq(e)) * sq(e) / (g + a) / (a + f) / (a + e) / a;
  iy(6, ny) = 1.0;
  iy(7, ny) = top / g / a / f;
  for (size_t k = 0; k < 8 * (size_t)ny; ++k) ip.p[k] = iy.p[k];  // fd_iyp = fd_iy, then its top rows
  a = hi[ny] / 2, e = hi[ny - 1] / 2, f = e + h[ny - 1];
  ip(1, ny - 1) = 4 * sq(e) * sq(a) / (2 * a + f) / (a + f) / (2 * sq(e) + sq(f) - 3 * e * f);
  ip(2, ny - 1) = -(4 * f * sq(a) / (3 * e * a + sq(e) + 2 * sq(a)) / (e - f));
  ip(3, ny - 1) = 4 * sq(e) * f / (cu(a) + 2 * sq(e) * a + 3 * e * sq(a) + 2 * sq(e) * f + f * sq(a) + 3 * f * e * a);
  ip(6, ny - 1) = -(f * sq(a) / (a + e) / (2 * e - f) / (2 * e + a));
  ip(7, ny - 1) = 1.0;
  ip(8, ny - 1) = sq(e) * f / (4 * cu(a) + 2 * sq(e) * a + 6 * e * sq(a) + 3 * f * e * a + sq(e) * f + 2 * f * sq(a));
  e = hi[ny] / 2, f = e + h[ny], g = f + h[ny - 1];
  ip(1, ny) = 2 * sq(e) * (2 * e - f) / (e - g) / (f - g) / g;
  ip(2, ny) = -(2 * (2 * e - g) * sq(e) / (e - f) / f / (f - g));
  ip(3, ny) = 2 * (4 * sq(e) + g * f - 2 * e * f - 2 * g * e) / (sq(e) - e * f + g * f - g * e);
  ip(6, ny) = 1.0;
  ip(7, ny) = (4 * sq(e) + g * f - 2 * e * f - 2 * g * e) / g / f;
  ip.factor(ny, 3, 2);
  iy.factor(ny, 3, 2);
}

// ludcmp, coeft.f90:1818-1883 (Numerical Recipes, implicit pivoting).
// bc is the (np x np) column-major work matrix, n <= np.
int ludcmp(double bc[5][5] /* [col][row] */, int n, int indx[5]) {
  const double tiny = 1.0e-20;
  double vv[5];
  for (int i = 0; i < n; ++i) {
    double aamax = 0.0;
    for (int j = 0; j < n; ++j)
      if (std::fabs(bc[j][i]) > aamax) aamax = std::fabs(bc[j][i]);
    if (aamax == 0.0) return -1;  // the reference pauses: 'singular matrix.'
    vv[i] = 1.0 / aamax;
  }
  int imax = 0;
  for (int j = 0; j < n; ++j) {
    for (int i = 0; i < j; ++i) {
      double sum = bc[j][i];
      if (i > 0) {
        for (int k = 0; k < i; ++k) sum = sum - bc[k][i] * bc[j][k];
        bc[j][i] = sum;
      }
    }
    double aamax = 0.0;
    for (int i = j; i < n; ++i) {
      double sum = bc[j][i];
      if (j > 0) {
        for (int k = 0; k < j; ++k) sum = sum - bc[k][i] * bc[j][k];
        bc[j][i] = sum;
      }
      const double dum = vv[i] * std::fabs(sum);
      if (dum >= aamax) {
        imax = i;
        aamax = dum;
      }
    }
    if (j != imax) {
      for (int k = 0; k < n; ++k) {
        const double dum = bc[k][imax];
        bc[k][imax] = bc[k][j];
        bc[k][j] = dum;
      }
      vv[imax] = vv[j];
    }
    indx[j] = imax;
    if (j != n - 1) {
      if (bc[j][j] == 0.0) bc[j][j] = tiny;
      const double dum = 1.0 / bc[j][j];
      for (int i = j + 1; i < n; ++i) bc[j][i] = bc[j][i] * dum;
    }
  }
  if (bc[n - 1][n - 1] == 0.0) bc[n - 1][n - 1] = tiny;
  return 0;
}

// lubksb, coeft.f90:1890-1922
void lubksb(double bc[5][5], int n, const int indx[5], double b[5]) {
  int ii = -1;
  for (int i = 0; i < n; ++i) {
    const int ll = indx[i];
    double sum = b[ll];
    b[ll] = b[i];
    if (ii != -1) {
      for (int j = ii; j < i; ++j) sum = sum - bc[j][i] * b[j];
    } else if (sum != 0.0) {
      ii = i;
    }
    b[i] = sum;
  }
  for (int i = n - 1; i >= 0; --i) {
    double sum = b[i];
    for (int j = i + 1; j < n; ++j) sum = sum - bc[j][i] * b[j];
    b[i] = sum / bc[i][i];
  }
}

// coefb, coeft.f90:1360-1789. Builds the small moment-matching system for a
// boundary closure and solves it; bcc(1:n) is the result.
int coefb(int n, double a, double b, double c, double d, double bcc[5], int flagv) {
  double bc[5][5];  // bc[col][row], i.e. bc(row+1, col+1)
  int indx[5] = {0, 0, 0, 0, 0};
  for (int i = 0; i < 5; ++i) {
    bcc[i] = 0.0;
    for (int j = 0; j < 5; ++j) bc[j][i] = 0.0;
  }
#define BC(r, c) bc[(c)-1][(r)-1]
  const double h = 1.0 / 2.0;
  switch (flagv) {
    case 1:  // coeft.f90:1369-1411
      bcc[0] = 1.0;
      BC(1, 1) = -1.0; BC(1, 2) = 0.0; BC(1, 3) = h * sq(a);
      BC(1, 4) = h * sq(a + b); BC(1, 5) = h * sq(a + b + c);
      BC(2, 1) = 0.0; BC(2, 2) = 1.0; BC(2, 3) = 1.0; BC(2, 4) = 1.0; BC(2, 5) = 1.0;
      BC(3, 1) = 0.0; BC(3, 2) = 0.0; BC(3, 3) = a; BC(3, 4) = a + b; BC(3, 5) = a + b + c;
      BC(4, 1) = -a; BC(4, 2) = 0.0; BC(4, 3) = 1.0 / 6.0 * cu(a);
      BC(4, 4) = 1.0 / 6.0 * cu(a + b); BC(4, 5) = 1.0 / 6.0 * cu(a + b + c);
      BC(5, 1) = -h * sq(a); BC(5, 2) = 0.0; BC(5, 3) = 1.0 / 24.0 * p4(a);
      BC(5, 4) = 1.0 / 24.0 * p4(a + b); BC(5, 5) = 1.0 / 24.0 * p4(a + b + c);
      break;
    case 0:  // coeft.f90:1413-1437
      bcc[0] = 1.0;
      BC(1, 1) = 1.0; BC(1, 2) = 1.0; BC(1, 3) = 1.0;
      BC(2, 1) = -h * a; BC(2, 2) = -(h * a + b); BC(2, 3) = -(h * a + b + c);
      BC(3, 1) = 1.0 / 8.0 * sq(a); BC(3, 2) = h * sq(-(h * a + b));
      BC(3, 3) = h * sq(-(h * a + b + c));
      break;
    case 3:  // coeft.f90:1487-1523
      bcc[0] = 1.0;
      BC(1, 1) = h * a; BC(1, 2) = (h * a + b); BC(1, 3) = (h * a + b + c);
      BC(1, 4) = (h * a + b + c + d);
      BC(2, 1) = 1.0; BC(2, 2) = 1.0; BC(2, 3) = 1.0; BC(2, 4) = 1.0;
      BC(3, 1) = 1.0 / 8.0 * sq(a); BC(3, 2) = h * sq(h * a + b);
      BC(3, 3) = h * sq(h * a + b + c); BC(3, 4) = h * sq(h * a + b + c + d);
      BC(4, 1) = 1.0 / 48.0 * cu(a); BC(4, 2) = 1.0 / 6.0 * cu(h * a + b);
      BC(4, 3) = 1.0 / 6.0 * cu(h * a + b + c); BC(4, 4) = 1.0 / 6.0 * cu(h * a + b + c + d);
      break;
    case 4:  // coeft.f90:1525-1557
      bcc[0] = 1.0;
      BC(1, 1) = 1.0; BC(1, 2) = 1.0; BC(1, 3) = 1.0; BC(1, 4) = 1.0;
      BC(2, 1) = -h * a; BC(2, 2) = h * b; BC(2, 3) = h * b + c; BC(2, 4) = h * b + c + d;
      BC(3, 1) = 1.0 / 8.0 * sq(a); BC(3, 2) = 1.0 / 8.0 * sq(b);
      BC(3, 3) = h * sq(h * b + c); BC(3, 4) = h * sq(h * b + c + d);
      BC(4, 1) = -1.0 / 48.0 * cu(a); BC(4, 2) = 1.0 / 48.0 * cu(b);
      BC(4, 3) = 1.0 / 6.0 * cu(h * b + c); BC(4, 4) = 1.0 / 6.0 * cu(h * b + c + d);
      break;
    case 5:  // coeft.f90:1559-1595
      bcc[0] = 1.0;
      BC(1, 1) = h * a; BC(1, 2) = -h * b; BC(1, 3) = -(h * b + c); BC(1, 4) = -(h * b + c + d);
      BC(2, 1) = 1.0; BC(2, 2) = 1.0; BC(2, 3) = 1.0; BC(2, 4) = 1.0;
      BC(3, 1) = 1.0 / 8.0 * sq(a); BC(3, 2) = 1.0 / 8.0 * sq(b);
      BC(3, 3) = h * sq(-(h * b + c)); BC(3, 4) = h * sq(-(h * b + c + d));
      BC(4, 1) = 1.0 / 48.0 * cu(a); BC(4, 2) = -1.0 / 48.0 * cu(b);
      BC(4, 3) = 1.0 / 6.0 * cu(-(h * b + c)); BC(4, 4) = 1.0 / 6.0 * cu(-(h * b + c + d));
      break;
    case 6:  // coeft.f90:1597-1633
      bcc[1] = 1.0;
      BC(1, 1) = 1.0; BC(1, 2) = 1.0; BC(1, 3) = 1.0; BC(1, 4) = 1.0;
      BC(2, 1) = 0.0; BC(2, 2) = -h * a; BC(2, 3) = -(h * a + b); BC(2, 4) = -(h * a + b + c);
      BC(3, 1) = 0.0; BC(3, 2) = 1.0 / 8.0 * sq(a); BC(3, 3) = h * sq(-(h * a + b));
      BC(3, 4) = h * sq(-(h * a + b + c));
      BC(4, 1) = 0.0; BC(4, 2) = -1.0 / 48.0 * cu(a); BC(4, 3) = 1.0 / 6.0 * cu(-(h * a + b));
      BC(4, 4) = 1.0 / 6.0 * cu(-(h * a + b + c));
      break;
    case 7:  // coeft.f90:1635-1672
      bcc[1] = 1.0;
      BC(1, 1) = 1.0; BC(1, 2) = 1.0; BC(1, 3) = 1.0; BC(1, 4) = 1.0;
      BC(2, 1) = h * a; BC(2, 2) = -h * b; BC(2, 3) = -(h * b + c); BC(2, 4) = -(h * b + c + d);
      BC(3, 1) = 1.0 / 8.0 * sq(a); BC(3, 2) = 1.0 / 8.0 * sq(b);
      BC(3, 3) = sq(h * b + c); BC(3, 4) = sq(h * b + c + d);
      BC(4, 1) = 1.0 / 48.0 * cu(a); BC(4, 2) = -1.0 / 48.0 * cu(b);
      BC(4, 3) = -1.0 / 6.0 * cu(h * b + c); BC(4, 4) = -1.0 / 6.0 * cu(h * b + c + d);
      break;
    default:
      return -2;
  }
#undef BC
  if (ludcmp(bc, n, indx) != 0) return -1;
  lubksb(bc, n, indx, bcc);
  return 0;
}

// coefinv, coeft.f90:1338-1353 (pre-factorisation for Thomas back-substitution)
void coefinv(Arr3 a, int neq, int npter1) {
  for (int j = npter1 + 1; j <= neq; ++j) {
    const double d = 1.0 / a(2, j - 1);
    a(2, j - 1) = d;
    a(1, j) = -a(1, j) * d;
    a(2, j) = a(2, j) + a(1, j) * a(3, j - 1);
  }
  a(2, neq) = 1.0 / a(2, neq);
}

}  // namespace

extern "C" size_t otbl_coef_count(int nx, int ny, int nz) {
  otbl_coef_offsets o;
  otbl_coef_layout(nx, ny, nz, &o);
  return o.off[OTBL_C_COUNT];
}

extern "C" int otbl_coef_offset(int nx, int ny, int nz, int id, size_t *off) {
  if (id < 0 || id > OTBL_C_COUNT || !off) return OTBL_ERR_ARG;
  otbl_coef_offsets o;
  otbl_coef_layout(nx, ny, nz, &o);
  *off = o.off[id];
  return OTBL_OK;
}

extern "C" int otbl_config_check(const otbl_config *cfg) {
  if (!cfg) return OTBL_ERR_ARG;
  if (cfg->nx < 9 || cfg->ny < 9 || cfg->nz < 6) return OTBL_ERR_CONFIG;
  if ((2 * (cfg->nz / 3)) / 2 - 1 < 1) return OTBL_ERR_CONFIG;
  if (cfg->nz % 2 != 0) return OTBL_ERR_CONFIG;
  if (cfg->xout < 2 || cfg->xout > cfg->nx) return OTBL_ERR_CONFIG;
  if (!(cfg->re > 0.0) || !(cfg->ax > 0.0) || !(cfg->az > 0.0) || !(cfg->cfl > 0.0))
    return OTBL_ERR_CONFIG;
  if (cfg->xpose_round != 0 && cfg->xpose_round != 1) return OTBL_ERR_CONFIG;
  if (cfg->dt_mode != 0 && cfg->dt_mode != 1) return OTBL_ERR_CONFIG;
  if (cfg->precision != OTBL_PREC_FP64 && cfg->precision != OTBL_PREC_MIXED) return OTBL_ERR_CONFIG;
  if (cfg->precision == OTBL_PREC_MIXED && cfg->xpose_round != 0) return OTBL_ERR_CONFIG;
  if (cfg->options & ~OTBL_OPT_YDENSE) return OTBL_ERR_CONFIG;
  if ((cfg->options & OTBL_OPT_YDENSE) && (cfg->precision != OTBL_PREC_MIXED || cfg->ny > 256))
    return OTBL_ERR_CONFIG;
  return OTBL_OK;
}

// coef (coeft.f90:10-1234) + wavenumbers (bl_1.F90:357-366) +
// inlet_retheta (bl_1.F90:372-396) + magicnumber (boun.f90:102-143).
extern "C" int otbl_coef_compute(const otbl_config *cfg, const double *yin,
                                 const double *u0, double *out) {
  int st = otbl_config_check(cfg);
  if (st != OTBL_OK) return st;
  if (!yin || !u0 || !out) return OTBL_ERR_ARG;
  const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz;
  const int nz1 = 2 * (nz / 3), nz2 = nz1 / 2 - 1;
  (void)nz1;
  otbl_coef_offsets o;
  otbl_coef_layout(nx, ny, nz, &o);
  std::memset(out, 0, sizeof(double) * o.off[OTBL_C_COUNT]);
  auto P = [&](int id) { return out + o.off[id]; };

  double *S = P(OTBL_C_SCAL);
  const double re = cfg->re, ax = cfg->ax, az = cfg->az, cfl = cfg->cfl;
  const double pi = 4.0 * std::atan(1.0);

  // y(0:ny+1) as read from the restart header (getstartzy-bg.F90:571)
  double *y = P(OTBL_C_Y);
  for (int j = 0; j <= ny + 1; ++j) y[j] = yin[j];
#define Y(j) y[(j)]

  // hy, coeft.f90:32-37
  double *hy = P(OTBL_C_HY);
  for (int j = 1; j <= ny - 1; ++j) hy[j] = (Y(j + 1) - Y(j - 1)) / 2.5 / 2.0;
  hy[0] = (Y(1) - Y(0)) / 2.5;
  hy[ny] = (Y(ny) - Y(ny - 1)) / 2.5;

  // distances between nodes and faces, coeft.f90:397-424
  double *dy = P(OTBL_C_DY);  // dy(0:ny)
  for (int j = 0; j <= ny; ++j) dy[j] = Y(j + 1) - Y(j);
  std::vector<double> dyiv(ny + 1);  // dyi(1:ny)
  double *dyi = dyiv.data();
  for (int j = 1; j <= ny; ++j) dyi[j] = 0.5 * (dy[j] + dy[j - 1]);
  const double point0 = ax * pi / (nx + 1);
  double *x = P(OTBL_C_XG);  // x(0:nx+1)
  for (int i = 0; i <= nx + 1; ++i) x[i] = (double)i * point0;
  double *dx = P(OTBL_C_DX);  // dx(0:nx)
  double daux = 1000.0;
  for (int i = 0; i <= nx; ++i) {
    dx[i] = x[i + 1] - x[i];
    daux = std::fmin(daux, dx[i]);
  }
  double dxmin = daux;
  std::vector<double> dxiv(nx + 1);  // dxi(1:nx)
  double *dxi = dxiv.data();
  for (int i = 1; i <= nx; ++i) dxi[i] = 0.5 * (dx[i] + dx[i - 1]);
  const double idx = 1.0 / dx[1];
  double *idy = P(OTBL_C_IDY);
  for (int j = 0; j <= ny; ++j) idy[j] = 1.0 / dy[j];
  const double idxx = 1.0 / dx[1];
  double *idyy = P(OTBL_C_IDYY);  // idyy(1:ny) stored at [j-1]
  for (int j = 1; j <= ny; ++j) idyy[j - 1] = 2.0 / (dy[j - 1] + dy[j]);

  // time-step limits, coeft.f90:432-454
  double *dymin = P(OTBL_C_DYMIN);  // dymin(1:ny) at [j-1]
  daux = 1000.0;
  for (int i = 1; i <= ny; ++i) {
    dymin[i - 1] = dy[i] * cfl / std::sqrt(3.0);
    daux = std::fmin(daux, dy[i]);
  }
  double dzmin = az * 2 * pi / nz;
  // re*(cfl*dxmin**2)/(6.0d0): the power binds first
  const double dtrex = re * (cfl * (dxmin * dxmin)) / 6.0;
  const double dtrez = re * (cfl * (dzmin * dzmin)) / (pi * pi);
  const double dtret = std::fmin(dtrex, dtrez);
  dxmin = dxmin * cfl / std::sqrt(3.0);
  dzmin = dzmin * cfl / pi;
  const double rex = -1.0 / re;

  // wavenumbers, bl_1.F90:357-366, and kvis, coeft.f90:484-486
  double *kaz = P(OTBL_C_KAZ), *kaz2 = P(OTBL_C_KAZ2), *kvis = P(OTBL_C_KVIS);
  // kaz(k) = cmplx(0d0, k/az): CMPLX without KIND is a default-kind
  // (REAL*4) complex, so the imaginary part is k/az rounded to single
  // precision before it is stored in the complex*16 kaz (the reference's
  // builds use no default-real promotion flag)
  for (int k = 0; k <= nz2; ++k) {
    kaz[k] = (double)(float)((double)k / az);
    kaz2[k] = -(-(kaz[k] * kaz[k]));  // -kaz**2 = +k**2/az**2 (real)
    kvis[k] = rex * kaz2[k];
  }

  // RK3 constants, coeft.f90:494-508
  S[OTBL_S_RKC + 0] = 8.0 / 15.0; S[OTBL_S_RKC + 1] = 5.0 / 12.0; S[OTBL_S_RKC + 2] = 3.0 / 4.0;
  S[OTBL_S_RKD + 0] = 0.0; S[OTBL_S_RKD + 1] = -17.0 / 60.0; S[OTBL_S_RKD + 2] = -5.0 / 12.0;
  S[OTBL_S_RKCV + 0] = 4.0 / 15.0; S[OTBL_S_RKCV + 1] = 1.0 / 15.0; S[OTBL_S_RKCV + 2] = 1.0 / 6.0;
  S[OTBL_S_RKDV + 0] = 4.0 / 15.0; S[OTBL_S_RKDV + 1] = 1.0 / 15.0; S[OTBL_S_RKDV + 2] = 1.0 / 6.0;

  // ---- interpolation coefficients, implicit part, coeft.f90:514-580 ----
  Arr3 inxu{P(OTBL_C_INXU), 1}, inxv{P(OTBL_C_INXV), 1};
  Arr3 inyu{P(OTBL_C_INYU), 1}, inyv{P(OTBL_C_INYV), 1};
  for (int i = 2; i <= nx - 1; ++i) {
    const double c = dxi[i + 1], a = dxi[i], b = dx[i];
    inxu(1, i) = c * sq(b) / ((2 * a + b) * (-b + 2 * a) * (c + a));
    inxu(2, i) = 1.0;
    inxu(3, i) = -a * sq(b) / ((b - 2 * c) * (b + 2 * c) * (c + a));
  }
  for (int i = 2; i <= ny - 1; ++i) {
    const double a = dy[i], b = dy[i - 1];
    inyu(1, i) = sq(a) / ((a + b) * (a + 2 * b));
    inyu(2, i) = 1.0;
    inyu(3, i) = sq(b) / (sq(b) + 2 * sq(a) + 3 * a * b);
  }
  for (int i = 2; i <= nx - 1; ++i) {
    const double a = dx[i], b = dx[i - 1];
    inxv(1, i) = sq(a) / ((b + a) * (a + 2.0 * b));
    inxv(2, i) = 1.0;
    inxv(3, i) = sq(b) / (2.0 * sq(a) + sq(b) + 3.0 * a * b);
  }
  for (int i = 2; i <= ny - 1; ++i) {
    const double a = dyi[i], b = dy[i - 1], c = dyi[i - 1];
    inyv(1, i) = c * sq(b) / ((2 * a + b) * (-b + 2 * a) * (c + a));
    inyv(2, i) = 1.0;
    inyv(3, i) = -a * sq(b) / ((b - 2 * c) * (b + 2 * c) * (c + a));
  }
  inxu(3, 1) = 0.0; inxu(2, 1) = 1.0; inxu(1, 1) = 0.0;
  inxu(1, nx) = 0.0; inxu(2, nx) = 1.0; inxu(3, nx) = 0.0;
  inxv(1, 1) = 0.0; inxv(2, 1) = 1.0; inxv(3, 1) = 0.0;
  inxv(1, nx) = 0.0; inxv(2, nx) = 1.0; inxv(3, nx) = 0.0;
  inyu(1, 1) = 0.0; inyu(2, 1) = 1.0; inyu(3, 1) = 0.0;
  inyu(1, ny) = 0.0; inyu(2, ny) = 1.0; inyu(3, ny) = 0.0;
  inyv(1, 1) = 0.0; inyv(2, 1) = 1.0; inyv(3, 1) = 0.0;
  inyv(1, ny) = 0.0; inyv(2, ny) = 1.0; inyv(3, ny) = 0.0;

  double bcc[5];
  int bad = 0;
  // boundary closures in x for the interpolations, coeft.f90:583-624
  Mat inbx{P(OTBL_C_INBX), 4};
  bad |= coefb(3, dx[nx - 1], dxi[nx - 1], dxi[nx - 2], dxi[nx - 3], bcc, 0);
  inbx(1, 1) = bcc[0]; inbx(1, 2) = bcc[1]; inbx(1, 3) = bcc[2]; inbx(1, 4) = 0.0;
  bad |= coefb(3, dx[nx], dx[nx - 1], dx[nx - 2], dx[nx - 3], bcc, 0);
  inbx(2, 1) = bcc[0]; inbx(2, 2) = bcc[1]; inbx(2, 3) = bcc[2]; inbx(2, 4) = 0.0;
  bad |= coefb(4, dx[1], dx[1], dx[2], dx[3], bcc, 4);
  inbx(3, 1) = bcc[0]; inbx(3, 2) = bcc[1]; inbx(3, 3) = bcc[2]; inbx(3, 4) = bcc[3];
  bad |= coefb(4, dx[0], dx[1], dxi[2], dxi[3], bcc, 4);
  inbx(4, 1) = bcc[0]; inbx(4, 2) = bcc[1]; inbx(4, 3) = bcc[2]; inbx(4, 4) = bcc[3];

  // boundary closures in y for the interpolations, coeft.f90:631-675
  Mat inby{P(OTBL_C_INBY), 4};
  bad |= coefb(4, dy[ny], dy[ny - 1], dyi[ny - 1], dyi[ny - 2], bcc, 4);
  inby(1, 1) = bcc[0]; inby(1, 2) = bcc[1]; inby(1, 3) = bcc[2]; inby(1, 4) = bcc[3];
  bad |= coefb(3, -dy[0], -dy[1], -dy[2], dy[4], bcc, 0);
  inby(3, 1) = bcc[0]; inby(3, 2) = bcc[1]; inby(3, 3) = bcc[2]; inby(3, 4) = 0.0;
  bad |= coefb(4, dy[0], dy[1], dyi[2], dyi[3], bcc, 4);
  inby(2, 1) = bcc[0]; inby(2, 2) = bcc[1]; inby(2, 3) = bcc[2]; inby(2, 4) = bcc[3];
  bad |= coefb(4, -dy[ny - 1], -dy[ny - 1], -dy[ny - 2], -dy[ny - 3], bcc, 4);
  inby(4, 1) = bcc[0]; inby(4, 2) = bcc[1]; inby(4, 3) = bcc[2]; inby(4, 4) = bcc[3];

  coefinv(inxu, nx, 1);
  coefinv(inxv, nx, 1);
  coefinv(inyu, ny, 1);
  coefinv(inyv, ny, 1);

  // explicit part of the interpolations, coeft.f90:685-713
  Arr2 cofivy{P(OTBL_C_COFIVY), 1}, cofiuy{P(OTBL_C_COFIUY), 1};
  Arr2 cofivx{P(OTBL_C_COFIVX), 1}, cofiux{P(OTBL_C_COFIUX), 1};
  for (int i = 2; i <= ny - 1; ++i) {
    double a = dyi[i], b = dy[i - 1];
    const double c = dyi[i - 1];
    cofivy(2, i) = (-2.0 * c * a) / (2 * a * b + sq(b) - 4 * c * a - 2 * c * b);
    cofivy(1, i) = (2.0 * c * a) / (-sq(b) + 2 * a * b - 2 * c * b + 4 * c * a);
    a = dy[i];
    b = dy[i - 1];
    cofiuy(2, i) = 4 * sq(b) / (2 * sq(b) + sq(a) + 3 * a * b);
    cofiuy(1, i) = 4 * sq(a) / ((a + b) * (2 * a + b));
  }
  for (int i = 2; i <= nx - 1; ++i) {
    double a = dx[i], b = dx[i - 1];
    cofivx(2, i) = (4.0 * sq(b)) / (2.0 * sq(b) + std::pow(a, 2.0) + 3.0 * a * b);
    cofivx(1, i) = (4.0 * sq(a)) / ((b + a) * (2.0 * a + b));
    const double c = dxi[i + 1];
    a = dxi[i];
    b = dx[i];
    cofiux(2, i) = (-2.0 * c * a) / (2 * a * b + sq(b) - 4 * c * a - 2 * c * b);
    cofiux(1, i) = (2.0 * c * a) / (-sq(b) + 2 * a * b - 2 * c * b + 4 * c * a);
  }

  // ---- first-derivative (convective) coefficients, coeft.f90:722-784 ----
  Arr3 dcxu{P(OTBL_C_DCXU), 1}, dcxv{P(OTBL_C_DCXV), 1};
  Arr3 dcyu{P(OTBL_C_DCYU), 1}, dcyv{P(OTBL_C_DCYV), 1};
  for (int i = 2; i <= nx - 1; ++i) {
    const double a = dx[i], b = dx[i - 1];
    const double den = (2.0 * cu(b) + 2.0 * cu(a) + 9.0 * sq(b) * a + 9.0 * b * sq(a));
    dcxu(1, i) = -a * (-2.0 * a * b - sq(b) + 2.0 * sq(a)) / den;
    dcxu(2, i) = 1.0;
    dcxu(3, i) = ((sq(a) + 2.0 * a * b - 2.0 * sq(b)) * b) / den;
  }
  dcxu(2, 1) = 1.0; dcxu(1, 1) = 0.0; dcxu(3, 1) = 0.0;
  dcxu(2, nx) = 1.0; dcxu(1, nx) = 0.0; dcxu(3, nx) = 0.0;
  for (int i = 2; i <= ny; ++i) {
    const double a = dyi[i], b = dyi[i - 1], c = dy[i - 1];
    const double den = (-sq(c) * a - sq(c) * b + 12.0 * sq(b) * a + 12.0 * b * sq(a));
    dcyu(1, i) = (b * sq(c)) / den;
    dcyu(2, i) = 1.0;
    dcyu(3, i) = (sq(c) * a) / den;
  }
  dcyu(2, 1) = 1.0; dcyu(3, 1) = 0.0; dcyu(1, 1) = 0.0;
  dcyu(2, ny + 1) = 1.0; dcyu(3, ny + 1) = 0.0; dcyu(1, ny + 1) = 0.0;
  for (int i = 2; i <= nx - 1; ++i) {
    const double a = dxi[i], b = dxi[i - 1], c = dx[i - 1];
    const double den = (-sq(c) * a - sq(c) * b + 12.0 * sq(b) * a + 12.0 * b * sq(a));
    dcxv(1, i) = (b * sq(c)) / den;
    dcxv(2, i) = 1.0;
    dcxv(3, i) = (sq(c) * a) / den;
  }
  dcxv(2, 1) = 1.0; dcxv(3, 1) = 0.0; dcxv(1, 1) = 0.0;
  dcxv(2, nx) = 1.0; dcxv(3, nx) = 0.0; dcxv(1, nx) = 0.0;
  for (int i = 2; i <= ny - 1; ++i) {
    const double a = dy[i], b = dy[i - 1];
    const double aux = (2.0 * cu(b) + 2.0 * cu(a) + 9.0 * sq(b) * a + 9.0 * b * sq(a));
    dcyv(1, i) = -a * (-2.0 * a * b - sq(b) + 2.0 * sq(a)) / aux;
    dcyv(2, i) = 1.0;
    dcyv(3, i) = ((sq(a) + 2.0 * a * b - 2.0 * sq(b)) * b) / aux;
  }
  dcyv(2, 1) = 1.0; dcyv(3, 1) = 0.0; dcyv(1, 1) = 0.0;
  dcyv(2, ny) = 1.0; dcyv(3, ny) = 0.0; dcyv(1, ny) = 0.0;

  // boundary closures of the first derivatives, coeft.f90:787-924
  Mat dcbx{P(OTBL_C_DCBX), 5};
  bad |= coefb(4, dx[1], dxi[2], dxi[3], dxi[4], bcc, 3);
  for (int c = 1; c <= 4; ++c) dcbx(1, c) = bcc[c - 1];
  bad |= coefb(4, dx[0], dx[1], dx[2], dx[3], bcc, 3);
  for (int c = 1; c <= 4; ++c) dcbx(2, c) = bcc[c - 1];
  bad |= coefb(4, dx[nx], dx[nx - 1], dxi[nx - 1], dxi[nx - 2], bcc, 5);
  for (int c = 1; c <= 4; ++c) dcbx(3, c) = bcc[c - 1];
  bad |= coefb(4, dx[nx - 1], dx[nx - 1], dx[nx - 2], dx[nx - 3], bcc, 5);
  for (int c = 1; c <= 4; ++c) dcbx(4, c) = bcc[c - 1];
  bad |= coefb(4, -dx[nx - 1], -dxi[nx - 1], -dxi[nx - 2], -dxi[nx - 3], bcc, 5);
  for (int c = 1; c <= 4; ++c) dcbx(5, c) = bcc[c - 1];

  Mat dcby{P(OTBL_C_DCBY), 4};
  bad |= coefb(4, -dy[0], -dy[1], -dyi[2], -dyi[3], bcc, 5);
  for (int c = 1; c <= 4; ++c) dcby(1, c) = bcc[c - 1];
  bad |= coefb(4, -dy[ny - 1], -dyi[ny - 1], -dyi[ny - 2], -dyi[ny - 3], bcc, 3);
  for (int c = 1; c <= 4; ++c) dcby(2, c) = bcc[c - 1];
  bad |= coefb(4, dy[0], dy[1], dy[2], dy[3], bcc, 3);
  for (int c = 1; c <= 4; ++c) dcby(3, c) = bcc[c - 1];
  bad |= coefb(4, -dy[ny], -dy[ny - 1], -dy[ny - 2], -dy[ny - 3], bcc, 3);
  for (int c = 1; c <= 4; ++c) dcby(4, c) = bcc[c - 1];
  // coeft.f90:889-898 recomputes row 2 with the same arguments
  bad |= coefb(4, -dy[ny - 1], -dyi[ny - 1], -dyi[ny - 2], -dyi[ny - 3], bcc, 3);
  for (int c = 1; c <= 4; ++c) dcby(2, c) = bcc[c - 1];

  Mat ccon{P(OTBL_C_CCON), 2};
  bad |= coefb(4, dy[ny], dy[ny - 1], dyi[ny - 1], dyi[ny - 2], bcc, 7);
  for (int c = 1; c <= 4; ++c) ccon(1, c) = bcc[c - 1];
  bad |= coefb(4, -dy[0], -dyi[1], -dyi[2], 0.0, bcc, 6);
  for (int c = 1; c <= 4; ++c) ccon(2, c) = bcc[c - 1];

  coefinv(dcxu, nx, 1);
  coefinv(dcxv, nx, 1);
  coefinv(dcyu, ny + 1, 1);
  coefinv(dcyv, ny, 1);

  // explicit part of the first derivatives, coeft.f90:933-965
  Arr2 cofcyv{P(OTBL_C_COFCYV), 1}, cofcyu{P(OTBL_C_COFCYU), 1};
  Arr2 cofcxv{P(OTBL_C_COFCXV), 1}, cofcxu{P(OTBL_C_COFCXU), 1};
  for (int i = 2; i <= ny - 1; ++i) {
    double a = dy[i], b = dy[i - 1];
    const double den = (2.0 * cu(b) + 2.0 * cu(a) + 9.0 * sq(b) * a + 9.0 * b * sq(a));
    cofcyv(1, i) = -24 * a * b / den;
    cofcyv(2, i) = 24 * a * b / den;
    a = dyi[i];
    b = dyi[i - 1];
    const double c = dy[i - 1];
    cofcyu(1, i) = -12.0 * a * b / ((12.0 * a * b - sq(c)) * c);
    cofcyu(2, i) = 12.0 * a * b / ((12.0 * a * b - sq(c)) * c);
  }
  {  // coeft.f90:945-952: the loop index has run to ny
    const int i = ny;
    const double a = dyi[i], b = dyi[i - 1], c = dy[i - 1];
    cofcyu(1, i) = -12.0 * a * b / ((12.0 * a * b - sq(c)) * c);
    cofcyu(2, i) = 12.0 * a * b / ((12.0 * a * b - sq(c)) * c);
  }
  for (int i = 2; i <= nx - 1; ++i) {
    double a = dxi[i], b = dxi[i - 1];
    const double c = dx[i - 1];
    cofcxv(1, i) = -12.0 * a * b / ((12.0 * a * b - sq(c)) * c);
    cofcxv(2, i) = 12.0 * a * b / ((12.0 * a * b - sq(c)) * c);
    a = dx[i];
    b = dx[i - 1];
    const double den = (2.0 * cu(b) + 2.0 * cu(a) + 9.0 * sq(b) * a + 9.0 * b * sq(a));
    cofcxu(1, i) = -24 * a * b / den;
    cofcxu(2, i) = 24 * a * b / den;
  }

  // ---- second-derivative (viscous) coefficients, coeft.f90:971-1168 ----
  Arr3 vixu{P(OTBL_C_VIXU), 1}, vixv{P(OTBL_C_VIXV), 1};
  Arr3 viyu{P(OTBL_C_VIYU), 1}, viyv{P(OTBL_C_VIYV), 1};
  auto vis_l = [](double a, double b) {
    return b * (sq(a) + a * b - sq(b)) / (cu(b) + cu(a) + 4 * sq(a) * b + 4 * a * sq(b));
  };
  auto vis_u = [](double a, double b) {
    return -(sq(a) - a * b - sq(b)) * a / (cu(b) + cu(a) + 4 * sq(a) * b + 4 * a * sq(b));
  };
  for (int i = 2; i <= nx - 1; ++i) {
    const double a = dx[i], b = dx[i - 1];
    vixu(1, i) = vis_l(a, b); vixu(2, i) = 1.0; vixu(3, i) = vis_u(a, b);
  }
  vixu(1, 1) = 0.0; vixu(2, 1) = 1.0; vixu(3, nx) = 0.0; vixu(2, nx) = 1.0;
  for (int i = 2; i <= ny; ++i) {
    const double a = dyi[i], b = dyi[i - 1];
    viyu(1, i) = vis_l(a, b); viyu(2, i) = 1.0; viyu(3, i) = vis_u(a, b);
  }
  viyu(1, 1) = 0.0; viyu(2, 1) = 1.0; viyu(3, ny + 1) = 0.0; viyu(2, ny + 1) = 1.0;
  for (int i = 2; i <= nx - 1; ++i) {
    const double a = dxi[i], b = dxi[i - 1];
    vixv(1, i) = vis_l(a, b); vixv(2, i) = 1.0; vixv(3, i) = vis_u(a, b);
  }
  vixv(1, 1) = 0.0; vixv(2, 1) = 1.0; vixv(3, nx) = 0.0; vixv(2, nx) = 1.0;
  for (int i = 2; i <= ny - 1; ++i) {
    const double a = dy[i], b = dy[i - 1];
    viyv(1, i) = vis_l(a, b); viyv(2, i) = 1.0; viyv(3, i) = vis_u(a, b);
  }
  viyv(1, 1) = 0.0; viyv(2, 1) = 1.0; viyv(3, ny) = 0.0; viyv(2, ny) = 1.0;

  // boundary closures of the second derivatives, coeft.f90:1023-1113
  // (flagv = 1 ignores its fourth length argument)
  Mat cofvbx{P(OTBL_C_COFVBX), 4}, cofvby{P(OTBL_C_COFVBY), 4};
  bad |= coefb(5, dxi[1], dxi[2], dxi[3], 0.0, bcc, 1);
  vixv(3, 1) = bcc[0];
  for (int c = 1; c <= 4; ++c) cofvbx(1, c) = bcc[c];
  bad |= coefb(5, dxi[nx - 1], dxi[nx - 2], dxi[nx - 3], 0.0, bcc, 1);
  vixv(1, nx) = bcc[0];
  for (int c = 1; c <= 4; ++c) cofvbx(2, c) = bcc[c];
  bad |= coefb(5, dx[1], dx[2], dx[3], 0.0, bcc, 1);
  vixu(3, 1) = bcc[0];
  for (int c = 1; c <= 4; ++c) cofvbx(3, c) = bcc[c];
  bad |= coefb(5, dx[nx - 1], dx[nx - 2], dx[nx - 3], 0.0, bcc, 1);
  vixu(1, nx) = bcc[0];
  for (int c = 1; c <= 4; ++c) cofvbx(4, c) = bcc[c];
  bad |= coefb(5, dy[1], dy[2], dy[3], 0.0, bcc, 1);
  viyv(3, 1) = bcc[0];
  for (int c = 1; c <= 4; ++c) cofvby(1, c) = bcc[c];
  bad |= coefb(5, dy[ny - 1], dy[ny - 2], dy[ny - 3], 0.0, bcc, 1);
  viyv(1, ny) = bcc[0];
  for (int c = 1; c <= 4; ++c) cofvby(2, c) = bcc[c];
  bad |= coefb(5, dyi[1], dyi[2], dyi[3], 0.0, bcc, 1);
  viyu(3, 1) = bcc[0];
  for (int c = 1; c <= 4; ++c) cofvby(3, c) = bcc[c];
  bad |= coefb(5, dyi[ny], dyi[ny - 1], dyi[ny - 2], 0.0, bcc, 1);
  viyu(1, ny + 1) = bcc[0];
  for (int c = 1; c <= 4; ++c) cofvby(4, c) = bcc[c];

  // un-factorised copies for the implicit solve, coeft.f90:1116-1127
  Arr3 vyui{P(OTBL_C_VYUI), 1}, vyvi{P(OTBL_C_VYVI), 1};
  for (int i = 1; i <= ny; ++i)
    for (int r = 1; r <= 3; ++r) {
      vyui(r, i) = viyu(r, i);
      vyvi(r, i) = viyv(r, i);
    }
  for (int r = 1; r <= 3; ++r) vyui(r, ny + 1) = viyu(r, ny + 1);

  coefinv(vixu, nx, 1);
  coefinv(vixv, nx, 1);
  coefinv(viyu, ny + 1, 1);
  coefinv(viyv, ny, 1);

  // explicit part of the second derivatives, coeft.f90:1136-1168
  Arr3 cofvyv{P(OTBL_C_COFVYV), 1}, cofvyu{P(OTBL_C_COFVYU), 1};
  Arr3 cofvxv{P(OTBL_C_COFVXV), 1}, cofvxu{P(OTBL_C_COFVXU), 1};
  auto vis_e = [](Arr3 &e, int i, double a, double b) {
    e(1, i) = 12 * b / (cu(b) + cu(a) + 4 * sq(a) * b + 4 * a * sq(b));
    e(2, i) = -12 / (sq(a) + 3 * a * b + sq(b));
    e(3, i) = 12 * a / (cu(b) + cu(a) + 4 * sq(a) * b + 4 * a * sq(b));
  };
  for (int i = 2; i <= ny - 1; ++i) vis_e(cofvyv, i, dy[i], dy[i - 1]);
  for (int i = 2; i <= ny; ++i) vis_e(cofvyu, i, dyi[i], dyi[i - 1]);
  for (int i = 2; i <= nx - 1; ++i) {
    vis_e(cofvxv, i, dxi[i], dxi[i - 1]);
    vis_e(cofvxu, i, dx[i], dx[i - 1]);
  }

  // DCT eigenvalues of the second difference, coeft.f90:1181-1183
  double *kmod = P(OTBL_C_KMOD);  // kmod(1:nx-1) at [i-1]
  for (int i = 1; i <= nx - 1; ++i)
    kmod[i - 1] = 2.0 / (dx[1] * dx[1]) * (1 - std::cos((pi * (i - 1)) / (double)(nx - 1)));

  // y-Poisson operator, mtr (coeft.f90:1244-1332), only the finest level
  // ngy2(1) = ny-1 is used by pois.
  {
    Arr3 ayp{P(OTBL_C_AYP), 1};
    double ac2 = 0.0, bc2 = 0.0, ac1, bc1, dy1, dy2, a3, b2;
    ac1 = ac2;
    bc1 = bc2;
    dy1 = Y(2) - Y(1);
    dy2 = Y(3) - Y(2);
    a3 = 1.0 / dy1;
    b2 = -1.0 / dy1;
    ac2 = 2.0 / (dy1 + dy2);
    bc2 = -2.0 / (dy1 + dy2);
    ayp(1, 1) = b2 * bc1;
    ayp(3, 1) = a3 * ac2;
    ayp(2, 1) = a3 * bc2 + b2 * ac1;
    const int ngy = ny - 1;
    for (int j = 2; j <= ngy - 1; ++j) {
      ac1 = ac2;
      bc1 = bc2;
      dy1 = Y(j + 1) - Y(j);
      dy2 = Y(j + 2) - Y(j + 1);
      a3 = 1.0 / dy1;
      b2 = -1.0 / dy1;
      ac2 = 2.0 / (dy1 + dy2);
      bc2 = -2.0 / (dy1 + dy2);
      ayp(1, j) = b2 * bc1;
      ayp(3, j) = a3 * ac2;
      ayp(2, j) = a3 * bc2 + b2 * ac1;
    }
    const int lt = ngy;
    b2 = -1.0 / dy2;
    ac1 = ac2;
    bc1 = bc2;
    ayp(1, lt) = b2 * bc1;
    ayp(3, lt) = 0.0;
    ayp(2, lt) = b2 * ac1;
  }

  // inlet Re_theta and delta99, bl_1.F90:380-388. `0.99` is a default-real
  // (single precision) literal in the reference.
  double rthin, din;
  {
    double uinf = 0.0;
    for (int j = ny + 1 - 20; j <= ny + 1 - 5; ++j) uinf += u0[j - 1];
    uinf = uinf / 16.0;
    const double u99 = (double)0.99f * uinf;
    int jtop = 0;
    for (int j = 1; j <= ny - 2; ++j) {
      if (u0[j - 1] >= u99) break;
      jtop = j + 1;
    }
    din = Y(jtop);
    double s = 0.0;
    for (int t = 0; t < jtop + 2; ++t) {  // u0(2:jtop+3), dy(1:jtop+2)
      const double uu = u0[(2 + t) - 1];
      s += (uinf - uu) * uu * dy[1 + t];
    }
    rthin = s * re / uinf;
  }

  // vmagic, boun.f90:114-140
  {
    double *vm = P(OTBL_C_VMAGIC);
    const double e1 = 0.8659, c1 = 0.01277, ei1 = 1 / e1;
    const double kap = 0.384, ckap = 4.127, cprim = 7.135;
    const double dxm = ax * pi / (nx - 1);
    std::vector<double> xm(nx + 1), hm(nx + 1);
    for (int i = 1; i <= nx; ++i) {
      xm[i] = dxm * (i - 1);
      const double reth = std::pow(std::pow(rthin, ei1) + std::pow(c1, ei1) * re * xm[i], e1);
      const double uep = std::log(reth) / kap + ckap;
      hm[i] = reth / ((1 - cprim / uep) * re);
    }
    vm[0] = (hm[2] - hm[1]) / (xm[2] - xm[1]);
    for (int i = 2; i <= nx - 1; ++i) vm[i - 1] = (hm[i + 1] - hm[i - 1]) / (xm[i + 1] - xm[i - 1]);
    vm[nx - 1] = (hm[nx] - hm[nx - 1]) / (xm[nx] - xm[nx - 1]);
  }

  fd_operators(nx, ny, ax, pi, y, Op8{P(OTBL_C_FD_DVDY)}, Op8{P(OTBL_C_FD_DX)}, Op8{P(OTBL_C_FD_IX)},
               Op8{P(OTBL_C_FD_IY)}, Op8{P(OTBL_C_FD_IYP)});

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
  S[OTBL_S_UINF] = 1.0;
  S[OTBL_S_RTHIN] = rthin;
  S[OTBL_S_DIN] = din;
  S[OTBL_S_YBLEND] = cfg->y_blend;
  S[OTBL_S_NX] = nx;
  S[OTBL_S_NY] = ny;
  S[OTBL_S_NZ] = nz;
  S[OTBL_S_XOUT] = cfg->xout;
#undef Y
  return bad ? OTBL_ERR_CONFIG : OTBL_OK;
}
