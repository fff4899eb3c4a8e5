/*
 * ORACLE (test infrastructure only): transforms used by the CPU restatement.
 *
 * The reference calls FFTW 3.3.2 (makefile:141), which is not vendored and is
 * not installed here. This file restates the published transform
 * definitions that the reference relies on, with the reference's scalings:
 *   fourxz  ffts.f90:27-67   r2c (FFTW_FORWARD, x dnf = 1/nz, ffts.f90:51,91)
 *                            c2r (FFTW_BACKWARD, unscaled, modes > nz2
 *                            zeroed first, ffts.f90:55-57,92)
 *   cosftx  ffts.f90:147-181 REDFT10 (DCT-II, x dnf = 1/n, ffts.f90:132,166)
 *                            REDFT01 (DCT-III, x dnb = 0.5, ffts.f90:133,171)
 * FFTW definitions (FFTW 3 manual, "What FFTW Really Computes"):
 *   r2c   X[k] = sum_j x[j] e^{-2 pi i jk/N},  k = 0..N/2
 *   c2r   x[j] = sum_{k=0}^{N-1} X[k] e^{+2 pi i jk/N} (Hermitian X; the
 *         imaginary parts of X[0] and X[N/2] are not used)
 *   REDFT10  Y[k] = 2 sum_j x[j] cos(pi k (2j+1) / (2n))
 *   REDFT01  Y[k] = x[0] + 2 sum_{j>=1} x[j] cos(pi j (2k+1) / (2n))
 * The complex FFT is a plain recursive mixed-radix Cooley-Tukey (radices
 * 2, 3, 4, 5 and a generic odd radix). Parity against FFTW itself is
 * unpinned (no reference test stores FFTW outputs); the definitions are
 * pinned against numpy.fft / scipy.fft in tests/test_oracle_transforms.py.
 */
#include "oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

struct orc_fft {
  int n;
  int nf;
  int fac[64];
  cplx *tw; /* tw[t] = exp(-2 pi i t / n), t = 0..n-1 */
};

static int factorize(int n, int *fac) {
  int nf = 0;
  while (n % 4 == 0) { fac[nf++] = 4; n /= 4; }
  while (n % 2 == 0) { fac[nf++] = 2; n /= 2; }
  for (int p = 3; n > 1; p += 2) {
    while (n % p == 0) { fac[nf++] = p; n /= p; }
  }
  return nf;
}

orc_fft *orc_fft_create(int n) {
  orc_fft *p = (orc_fft *)calloc(1, sizeof(orc_fft));
  p->n = n;
  p->nf = factorize(n, p->fac);
  p->tw = (cplx *)malloc(sizeof(cplx) * (size_t)n);
  const double pi = 4.0 * atan(1.0);
  for (int t = 0; t < n; ++t) {
    const double a = -2.0 * pi * (double)t / (double)n;
    p->tw[t] = cos(a) + I * sin(a);
  }
  return p;
}

void orc_fft_destroy(orc_fft *p) {
  if (!p) return;
  free(p->tw);
  free(p);
}

/* recursive decimation in time; sign = -1 forward, +1 backward (unscaled) */
static void fft_rec(const orc_fft *P, int n, int f, const cplx *in, int stride,
                    cplx *out, int sign) {
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  const int p = P->fac[f];
  const int m = n / p;
  for (int r = 0; r < p; ++r)
    fft_rec(P, m, f + 1, in + (size_t)r * stride, stride * p, out + (size_t)r * m, sign);
  const int N = P->n;
  const int step = N / n; /* W_n^t = tw[t*step] */
  cplx t[64];
  cplx wp[64];
  for (int q = 0; q < p; ++q) {
    const int idx = (int)(((long)q * (N / p)) % N);
    wp[q] = sign < 0 ? P->tw[idx] : conj(P->tw[idx]);
  }
  for (int k = 0; k < m; ++k) {
    for (int r = 0; r < p; ++r) {
      const int idx = (int)(((long)r * k * step) % N);
      const cplx w = sign < 0 ? P->tw[idx] : conj(P->tw[idx]);
      t[r] = out[(size_t)r * m + k] * w;
    }
    if (p == 2) {
      out[k] = t[0] + t[1];
      out[k + m] = t[0] - t[1];
    } else if (p == 4) {
      const cplx a0 = t[0] + t[2], a1 = t[0] - t[2];
      const cplx b0 = t[1] + t[3];
      const cplx b1 = (sign < 0 ? -I : I) * (t[1] - t[3]);
      out[k] = a0 + b0;
      out[k + m] = a1 + b1;
      out[k + 2 * m] = a0 - b0;
      out[k + 3 * m] = a1 - b1;
    } else {
      for (int q = 0; q < p; ++q) {
        cplx s = 0.0;
        for (int r = 0; r < p; ++r) s += t[r] * wp[(r * q) % p];
        out[k + (size_t)q * m] = s;
      }
    }
  }
}

void orc_fft_exec(const orc_fft *P, const double *in, double *out, int sign) {
  fft_rec(P, P->n, 0, (const cplx *)in, 1, (cplx *)out, sign);
}

/* --- fourxz line transforms (ffts.f90:27-67) ---
 * c2r: fou[0..2*nz2+1] (complex modes 0..nz2) -> phys[0..nz-1]
 * r2c: phys[0..nz-1] -> fou (modes 0..nz2) x 1/nz
 * h is the complex FFT of length nz/2; work has room for 3*(nz/2)+1
 * complex (c2r) or nz complex (r2c). */
void orc_c2r_line(const orc_fft *h, int nz, int nz2, const double *fou,
                  double *phys, double *work) {
  const int M = nz / 2;
  cplx *X = (cplx *)work;           /* X[0..M] */
  cplx *Z = X + (M + 1);            /* Z[0..M-1] */
  cplx *zo = Z + M;                 /* z[0..M-1] */
  for (int k = 0; k <= M; ++k) X[k] = 0.0;
  for (int k = 0; k <= nz2 && k <= M; ++k) X[k] = fou[2 * k] + I * fou[2 * k + 1];
  X[0] = creal(X[0]);
  X[M] = creal(X[M]);
  const int N = nz;
  const double pi = 4.0 * atan(1.0);
  for (int k = 0; k < M; ++k) {
    const cplx a = X[k], b = conj(X[M - k]);
    const double ang = 2.0 * pi * (double)k / (double)N; /* W^{-k} */
    const cplx w = cos(ang) + I * sin(ang);
    Z[k] = (a + b) + I * ((a - b) * w);
  }
  orc_fft_exec(h, (const double *)Z, (double *)zo, +1);
  for (int j = 0; j < M; ++j) {
    phys[2 * j] = creal(zo[j]);
    phys[2 * j + 1] = cimag(zo[j]);
  }
}

void orc_r2c_line(const orc_fft *h, int nz, int nz2, const double *phys,
                  double *fou, double *work) {
  const int M = nz / 2;
  cplx *z = (cplx *)work;
  cplx *Z = z + M;
  for (int j = 0; j < M; ++j) z[j] = phys[2 * j] + I * phys[2 * j + 1];
  orc_fft_exec(h, (const double *)z, (double *)Z, -1);
  const double pi = 4.0 * atan(1.0);
  const double dnf = 1.0 / (double)nz;
  for (int k = 0; k <= nz2; ++k) {
    const cplx zk = Z[k % M], zc = conj(Z[(M - k) % M]);
    const cplx E = 0.5 * (zk + zc);
    const cplx O = -0.5 * I * (zk - zc);
    const double ang = -2.0 * pi * (double)k / (double)nz;
    const cplx w = cos(ang) + I * sin(ang);
    const cplx Xk = E + w * O;
    fou[2 * k] = dnf * creal(Xk);
    fou[2 * k + 1] = dnf * cimag(Xk);
  }
}

/* --- cosftx line transforms on n = nx-1 reals (ffts.f90:147-181) ---
 * iopt < 0: REDFT10 x 1/n ; iopt >= 0: REDFT01 x 0.5. In place on c[0..n-1].
 * P is the complex FFT of length n; work holds 2n complex. */
void orc_dct_line(const orc_fft *P, int n, double *c, int iopt, double *work) {
  cplx *v = (cplx *)work;
  cplx *V = v + n;
  const double pi = 4.0 * atan(1.0);
  if (iopt < 0) {
    for (int m = 0; 2 * m < n; ++m) v[m] = c[2 * m];
    for (int m = 0; 2 * m + 1 < n; ++m) v[n - 1 - m] = c[2 * m + 1];
    orc_fft_exec(P, (const double *)v, (double *)V, -1);
    const double dnf = 1.0 / (double)n;
    for (int k = 0; k < n; ++k) {
      const double ang = -pi * (double)k / (2.0 * n);
      const cplx w = cos(ang) + I * sin(ang);
      c[k] = dnf * (2.0 * creal(w * V[k]));
    }
  } else {
    for (int k = 0; k < n; ++k) {
      const double ang = pi * (double)k / (2.0 * n);
      const cplx w = cos(ang) + I * sin(ang);
      const double ynk = (k == 0) ? 0.0 : c[n - k];
      v[k] = w * (c[k] - I * ynk);
    }
    orc_fft_exec(P, (const double *)v, (double *)V, +1);
    for (int m = 0; 2 * m < n; ++m) c[2 * m] = 0.5 * creal(V[m]);
    for (int m = 0; 2 * m + 1 < n; ++m) c[2 * m + 1] = 0.5 * creal(V[n - 1 - m]);
  }
}
