/*
 * otbl_driver -- a C program that drives the B200 substep through
 * include/otbl.h alone, the way the reference's time loop (bl_1.F90:85-128)
 * drives rhsp -> outflow_correction -> pois.
 *
 *   otbl_driver [nx ny nz nsteps]      (default 33 41 32 3)
 *
 * It builds a small boundary-layer box by itself (tanh-stretched y grid, a
 * tanh mean profile with a few seeded spanwise modes), computes the
 * coefficients (otbl_coef_compute), and advances the box twice:
 *   A  through the context API (otbl_substep),
 *   B  through the reference's array surface (otbl_rhsp_arrays,
 *      otbl_outflow_correction_arrays, otbl_pois_arrays) on device arrays
 *      the caller owns: here those of a third context, obtained with
 *      otbl_field_device_ptr, so that the program needs no CUDA runtime of
 *      its own.
 * It prints dt, u_tau, Re_theta and the energies after each step and checks
 * that A and B agree bit for bit.
 *
 * Exit status: 0 ok, 3 no usable CUDA device (the library has no CPU
 * fallback: OTBL_ERR_NODEV), 1 any other error or a mismatch.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/otbl.h"
#include "../../include/otbl_layout.h"

#define CHECK(call)                                                          \
  do {                                                                       \
    int st_ = (call);                                                        \
    if (st_ != OTBL_OK) {                                                    \
      fprintf(stderr, "otbl_driver: %s failed with %d (%s)\n", #call, st_,   \
              ctx_for_msg ? otbl_last_error(ctx_for_msg) : "");              \
      return st_ == OTBL_ERR_NODEV ? 3 : 1;                                  \
    }                                                                        \
  } while (0)

static otbl_ctx *ctx_for_msg = NULL;

/* deterministic pseudo-random numbers in [-1, 1) (splitmix64) */
static double rnd(unsigned long long *s) {
  unsigned long long z = (*s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z ^= z >> 31;
  return (double)(z >> 11) / 9007199254740992.0 * 2.0 - 1.0;
}

int main(int argc, char **argv) {
  const int nx = argc > 1 ? atoi(argv[1]) : 33, ny = argc > 2 ? atoi(argv[2]) : 41;
  const int nz = argc > 3 ? atoi(argv[3]) : 32, nsteps = argc > 4 ? atoi(argv[4]) : 3;
  const int nz1 = 2 * (nz / 3), nz2 = nz1 / 2 - 1;
  const double pi = 4.0 * atan(1.0);
  otbl_config cfg;
  memset(&cfg, 0, sizeof cfg);
  cfg.nx = nx; cfg.ny = ny; cfg.nz = nz;
  cfg.xout = nx / 3 > 2 ? nx / 3 : 2;
  cfg.xpose_round = OTBL_XPOSE_NONE;
  cfg.dt_mode = OTBL_DT_ADAPTIVE;
  cfg.re = 600.0;
  cfg.ax = 12.0 / pi;            /* Lx ~ ax*pi = 12 delta0 */
  cfg.az = 4.0 / (2.0 * pi);     /* Lz = 2*pi*az = 4 delta0 */
  cfg.cfl = 0.5;
  cfg.y_blend = 1.5;
  cfg.precision = OTBL_PREC_FP64;
  CHECK(otbl_config_check(&cfg));

  /* y(0:ny+1): wall at y(1) = 0, top at y(ny) = 6, tanh stretching */
  double *y = malloc(sizeof(double) * (ny + 2));
  for (int j = 1; j <= ny; ++j) {
    const double s = (double)(j - 1) / (ny - 1);
    y[j] = 6.0 * (1.0 - tanh(2.0 * (1.0 - s)) / tanh(2.0));
  }
  y[0] = -(y[2] - y[1]);
  y[ny + 1] = y[ny] + (y[ny] - y[ny - 1]);
  /* inlet mean profile u0(1:ny+1) at the cell centres, v0 = 0 */
  double *u0 = malloc(sizeof(double) * (ny + 1)), *v0 = calloc(ny + 1, sizeof(double));
  double *um = malloc(sizeof(double) * (ny + 1));
  for (int j = 1; j <= ny + 1; ++j) {
    const double yc = j <= ny ? 0.5 * (y[j] + y[j - 1]) : y[ny] + 0.5 * (y[ny + 1] - y[ny]);
    u0[j - 1] = tanh(2.5 * (yc > 0 ? yc : 0.0));
    um[j - 1] = u0[j - 1];
  }
  const size_t ncoef = otbl_coef_count(nx, ny, nz);
  double *coef = malloc(sizeof(double) * ncoef);
  CHECK(otbl_coef_compute(&cfg, y, u0, coef));

  /* the state: the mean profile in mode 0 of every plane, seeded
   * perturbations in spanwise modes 1..min(3, nz2) below y = 1.2 */
  const size_t lu = otbl_field_len(nx, ny, nz, 1), lv = otbl_field_len(nx, ny, nz, 0);
  const size_t len[OTBL_F_COUNT] = {lu, lv, lu, lv, lu, lv, lu};
  double *state[OTBL_F_COUNT];
  for (int id = 0; id < OTBL_F_COUNT; ++id) state[id] = calloc(len[id], sizeof(double));
  unsigned long long seed = 1234;
  for (int i = 1; i <= nx; ++i)
    for (int j = 1; j <= ny + 1; ++j) {
      double *uu = state[OTBL_F_U] + ((size_t)(i - 1) * (ny + 1) + (j - 1)) * nz1;
      double *ww = state[OTBL_F_W] + ((size_t)(i - 1) * (ny + 1) + (j - 1)) * nz1;
      uu[0] = u0[j - 1];
      const double yc = j <= ny ? 0.5 * (y[j] + y[j - 1]) : y[ny];
      const double env = yc < 1.2 ? sin(pi * yc / 1.2) : 0.0;
      for (int k = 1; k <= (nz2 < 3 ? nz2 : 3); ++k) {
        uu[2 * k] = 0.01 * env * rnd(&seed);
        uu[2 * k + 1] = 0.01 * env * rnd(&seed);
        ww[2 * k] = 0.01 * env * rnd(&seed);
        ww[2 * k + 1] = 0.01 * env * rnd(&seed);
      }
    }

  otbl_ctx *a = NULL, *b = NULL, *own = NULL;
  int st = otbl_ctx_create(&cfg, coef, 0, &a);
  if (st == OTBL_ERR_NODEV) {
    printf("otbl_driver: coefficients computed (%zu values); no usable CUDA device: "
           "OTBL_ERR_NODEV, the library has no CPU fallback\n", ncoef);
    return 3;
  }
  ctx_for_msg = a;
  CHECK(st);
  CHECK(otbl_ctx_create(&cfg, coef, 0, &b));
  CHECK(otbl_ctx_create(&cfg, coef, 0, &own));
  otbl_inflow inf;
  memset(&inf, 0, sizeof inf);
  double *dev[OTBL_F_COUNT];
  for (int id = 0; id < OTBL_F_COUNT; ++id) {
    CHECK(otbl_set_field(a, id, state[id]));
    CHECK(otbl_set_field(own, id, state[id]));  /* the caller's device arrays */
    CHECK(otbl_field_device_ptr(own, id, &dev[id]));
  }
  CHECK(otbl_set_inflow(a, u0, v0, um, &inf));
  CHECK(otbl_set_inflow(b, u0, v0, um, &inf));

  double ener_a[15], ener_b[15];
  for (int step = 1; step <= nsteps; ++step) {
    for (int m = 1; m <= 3; ++m) {
      ctx_for_msg = a;
      CHECK(otbl_substep(a, m, m == 1));
      ctx_for_msg = b;
      CHECK(otbl_rhsp_arrays(b, dev[0], dev[1], dev[2], dev[3], dev[4], dev[5], dev[6], m, m == 1));
      CHECK(otbl_outflow_correction_arrays(b, dev[0], dev[1], dev[4]));
      CHECK(otbl_pois_arrays(b, dev[0], dev[1], dev[2], dev[3], m));
    }
    otbl_inflow sa, sb;
    ctx_for_msg = a;
    CHECK(otbl_get_inflow(a, um, &sa));
    CHECK(otbl_get_energies(a, ener_a));
    ctx_for_msg = b;
    CHECK(otbl_get_inflow(b, um, &sb));
    CHECK(otbl_get_energies(b, ener_b));
    printf("step %d: tiempo %.6e dt %.6e u_tau %.6e Re_theta %.6f ener(1:3) %.6e %.6e %.6e\n", step,
           sa.tiempo, sa.dt, sa.utauout, sa.rthout, ener_a[0], ener_a[1], ener_a[2]);
    if (sa.dt != sb.dt || sa.tiempo != sb.tiempo || sa.rthout != sb.rthout ||
        memcmp(ener_a, ener_b, sizeof ener_a) != 0) {
      fprintf(stderr, "otbl_driver: the array surface's scalars differ from the context API's\n");
      return 1;
    }
  }
  /* the fields: context A against the caller's arrays that B advanced */
  int same = 1;
  for (int id = 0; id < OTBL_F_COUNT; ++id) {
    double *fa = malloc(sizeof(double) * len[id]), *fb = malloc(sizeof(double) * len[id]);
    ctx_for_msg = a;
    CHECK(otbl_get_field(a, id, fa));
    ctx_for_msg = own;
    CHECK(otbl_get_field(own, id, fb));
    if (memcmp(fa, fb, sizeof(double) * len[id]) != 0) {
      fprintf(stderr, "otbl_driver: field %d differs between the two surfaces\n", id);
      same = 0;
    }
    free(fa);
    free(fb);
  }
  otbl_ctx_destroy(b);  /* B never owned the arrays it advanced */
  otbl_ctx_destroy(own);
  otbl_ctx_destroy(a);
  if (!same) return 1;
  printf("otbl_driver: OK, %d RK3 steps of %dx%dx%d, context API and array surface bit-identical\n",
         nsteps, nx, ny, nz);
  for (int id = 0; id < OTBL_F_COUNT; ++id) free(state[id]);
  free(y); free(u0); free(v0); free(um); free(coef);
  return 0;
}
