// Internal declarations of the B200 substep: device view of the coefficient
// buffer, device scalar state, the context, and launch helpers.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/otbl.h"
#include "../../include/otbl_layout.h"

namespace otbl {

// Device view of the packed coefficient buffer (include/otbl_layout.h).
// Passed by value to kernels; every pointer is into one device allocation.
// Device pointers into a packed coefficient buffer (otbl_layout.h): FP64 for
// the FP64 path, and an FP32 copy (the same layout, every value rounded) for
// the FP32 operators of the mixed-precision path.
template <typename T>
struct DCoefT {
  int nx, ny, nz, nz1, nz2, xout;
  int xround;  // OTBL_XPOSE_FP32: round x-line inputs/outputs to REAL4
  const T *S;
  const T *y, *dy, *idy, *idyy, *dymin, *kaz, *kaz2, *kvis, *kmod, *ayp, *vmagic, *hy;
  const T *inxu, *inxv, *cofiux, *cofivx, *inbx;
  const T *dcxu, *dcxv, *cofcxu, *cofcxv, *dcbx;
  const T *vixu, *vixv, *cofvxu, *cofvxv, *cofvbx;
  const T *inyu, *inyv, *cofiuy, *cofivy, *inby;
  const T *dcyu, *dcyv, *cofcyu, *cofcyv, *dcby;
  const T *viyu, *viyv, *vyui, *vyvi, *cofvyu, *cofvyv, *cofvby, *ccon;
};
using DCoef = DCoefT<double>;

// Scalars that live on the device so that no host synchronisation is needed
// inside a step (dt is produced by a reduction on the device).
struct DState {
  double dt, tiempo, timeinit, timec;
  double utauout, rthout, dout, gamma1, gamma2;
  double var1, var2, var3, var4, rkk, varstep;  // RK3 factors of the substep
  double umax, wmax, vmax;
  double ener[15];  // energies of rhsp.F90:116 (module statistics, mod.F90:264)
  unsigned long long umax_bits, wmax_bits;      // atomicMax targets (>= 0)
  int err;        // OTBL_ERR_NAN when the dt reduction saw a non-finite value
  int dt_frozen;  // fixed-dt mode: dt taken
  int pad[2];
};

// Device work buffers. Field-sized arrays use the plane layout. The fifteen
// intermediate fields hold doubles on the FP64 path and floats on the mixed
// path (OTBL_PREC_MIXED); the kernels cast them to their element type.
struct Work {
  void *ux, *vx, *wx;          // interpxx outputs (u-type, v-type, u-type)
  void *uy, *wy, *vy;          // interpyy outputs (ny rows each)
  void *uu, *uw, *uv, *vw, *vv, *ww;  // products (uu, uw u-type; others ny rows)
  void *cu, *cv, *cw;          // difvisxx outputs
  double *s1, *s2, *s3;        // line-solve scratch and pois' phi (u-type size)
  double *t1, *t2, *t3;        // the w tail's scratch (beside the v tail), as s1..s3
  double *twz, *twz2;          // z-FFT twiddles exp(-2 pi i t/M), exp(-2 pi i t/nz)
  float *twzf, *twz2f;         // the same rounded to FP32 (mixed path)
  double *twx;                 // x-DCT twiddles for the length nx-1 FFT
  double *twx2;                // exp(-i pi k/(2n)), k = 0..n-1
  float *twxf, *twx2f;         // the same rounded to FP32 (mixed path)
  unsigned long long *vm_bits; // vm(j) maxima, j = 1..ny
  double *fac_u, *fac_v;       // implzy LU factors for the current dt (3*(ny+1))
  double *rowc;                // k_final_tb's per-row coefficients, [2][ny+2][16]
  void *xrowc;                 // k_xline_t's per-plane coefficients, [2][2][nx][16] (T)
  void *yrowc;                 // k_interpy_t's per-row coefficients, [2][ny][8] (T)
  double *gf;                  // genflu tables (genflu_tab_doubles)
  double *pois_dinv;           // pivots of the (x-mode, kz) y-systems, [i][j][k]
  float *pois_dinvf;           // the same rounded to FP32 (mixed path, modes >= kPoisLow)
};

// TMA descriptors (opaque 128-byte CUtensorMap objects) of the fields the
// rhsp tail's descending pass reads, for one velocity component (k_final_tb)
struct FinalMaps {
  CUtensorMap prod, kp, vel, cx, hp, p;
  CUtensorMap prod_a, vel_a;  // pass A: boxes of 8 + 2 rows
  CUtensorMap rc, rc_a;       // per-row coefficients (Work::rowc), KF / 8 rows
};

// TMA descriptors of interpyy's inputs (u, w, v), boxes of 128 kr x rows,
// and the per-row coefficient rows of each field's operator (Work::yrowc)
struct YMaps {
  CUtensorMap g[3], r[3];
};

// TMA descriptors of the x-line kernels' inputs, per field (u, v, w): 2D
// tensors [plane][line] with boxes of 32 lines, and the per-plane
// coefficient rows of the field's operator (Work::xrowc)
struct XMaps {
  CUtensorMap g[3], u[3], r[3];
};

// TMA descriptors of the dense interpyy's inputs (u, w, v): [nx][rows][nz1]
// FP64, boxes of nt spanwise columns x 16 rows x 1 plane
struct YDenseMaps {
  CUtensorMap g[3];
};

// TMA descriptors of pois' x-DCT kernels (k_pois_fwd_t, k_pois_bwd_t):
// the velocity [nx][rows][nz1] FP64 in boxes of 2 MB kr x rows x planes (u:
// 1 row x CP + 1 planes, v: 2 rows x CP, w: 1 row x CP) and phi-hat [nx][ny]
// [nz1] in FP64 and FP32, boxes of 2 MB kr x 1 row x min(256, nx - 1) planes
struct PoisMaps {
  CUtensorMap u, v, w, phi64, phi32;
};

}  // namespace otbl

struct otbl_ctx {
  otbl_config cfg;
  int device;
  cudaStream_t stream;
  // side streams of the substep (fork/join by events, so a graph capture
  // records the overlap): `side`, at the context stream's priority, runs
  // interpyy beside interpxx, k_dt and genflu; `side_lo`, at the lowest
  // priority, runs the second half of the products beside difvisxx and the
  // u tail, taking the SM slots those leave free
  cudaStream_t side = nullptr, side_lo = nullptr;
  cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  otbl::DCoef dc;
  otbl::DCoefT<float> dcf;  // FP32 coefficients (mixed path)
  // threads per CTA of the line kernels that otbl_autotune times:
  // [0] k_interpx, [1] k_difvisx, [2] k_interpy (one thread per line, so the
  // choice changes the schedule, never the arithmetic)
  int tune_bs[3] = {128, 128, 128};
  int pois_klo = 0;  // mixed path: spanwise modes k < pois_klo solve in FP64 (kPoisCond)
  // interpyy of the mixed path as a dense operator on the tensor cores
  // (OTBL_OPT_YDENSE, k_ydense.cu): the operators' TF32 chunks on the device,
  // per input type and M-tile the K-chunks [kb, ke) of their band, the
  // tiles' column count and the inputs' TMA descriptors
  bool ydense = false;
  uint32_t *yd_op = nullptr;
  size_t yd_words_per_op = 0;
  int yd_kb[2][2] = {{0, 0}, {0, 0}}, yd_ke[2][2] = {{0, 0}, {0, 0}};
  int yd_nt = 0, yd_nb = 0;
  otbl::YDenseMaps yd_maps;
  bool yd_maps_ok = false;
  // one-point statistics (k_stats.cu): OTBL_NSTATS accumulators (ny, nx),
  // allocated by the first otbl_statsp, and the number of samples in them
  double *stats = nullptr;
  int stats_samples = 0;
  // TMA descriptors of the rhsp tail's inputs, per velocity component
  otbl::FinalMaps fmaps[3];
  bool fmaps_ok = false;
  otbl::XMaps xmi, xmd;  // k_interpx_t (state), k_difvisx_t (products, state)
  bool xmaps_ok = false;
  otbl::YMaps ymi;       // k_interpy_t
  bool ymaps_ok = false;
  otbl::PoisMaps pmaps;  // k_pois_fwd_t / k_pois_bwd_t
  bool pmaps_vel = false, pmaps_phi64 = false, pmaps_phi32 = false;
  int mixed;                // cfg.precision == OTBL_PREC_MIXED
  double *coef_dev;
  float *coef_dev_f;
  std::vector<double> coef_host;
  // state fields; on the mixed path p and the RHS history are stored as
  // float (f32[id]) behind the same pointer, u, v, w always as double
  double *f[OTBL_F_COUNT];      // the state the kernels use: own arrays or bound ones
  double *f_own[OTBL_F_COUNT];  // the context's own state arrays (freed with it)
  bool f32[OTBL_F_COUNT] = {false, false, false, false, false, false, false};
  double *u0, *v0, *um;
  otbl::DState *st;
  otbl::Work w;
  std::vector<void *> allocs;
  size_t bytes;
  long long launches;
  std::string err;
  // optional per-kernel timing: a CUDA event pair around every launch
  bool prof_on = false;
  struct ProfRec {
    int kind;
    cudaEvent_t a, b;
  };
  std::vector<ProfRec> prof;
  std::vector<cudaEvent_t> prof_pool;
  int prof_open = -1;
};

namespace otbl {
enum ProfKind {
  PK_INTERPX = 0, PK_INTERPY, PK_PRODUCTS, PK_DIFVISX, PK_DT, PK_GENFLU, PK_FINAL,
  PK_OUTFLOW, PK_POIS_FWD, PK_POIS_SOLVE, PK_POIS_BWD, PK_PROJECT, PK_MISC, PK_COUNT
};
extern const char *const kProfNames[PK_COUNT];
void prof_begin(otbl_ctx *c, int kind);
void prof_end(otbl_ctx *c);
}  // namespace otbl

// Mixed path: the Poisson solve (x-DCTs, y-systems, phi) of a spanwise mode
// k runs in FP32 only when its shifted y-system is well conditioned: kz^2 >=
// max|ayp(2,j)| / kPoisCond, so that FP32 rounding of phi, amplified by the
// y second difference (up to ~4/dy_wall^2 on the stretched grid), stays
// below kPoisCond x 6e-8 of the mode's divergence. Lower modes run in FP64.
// (FP32 from k = 4 up, tried first, left max|div u| ~1e-6 after the
// projection at 1025x193x512: kappa(k = 4) ~ 1.6e5. Measured there after 100
// RK3 steps, against the 1e-10 gate: bound 1024, FP32 from k = 35, 7e-13;
// 4096, from k = 18, 2.3e-10; 16384, from k = 9, 1.0e-7. The two looser
// bounds saved 0.1-0.2 ms per mixed step.)
constexpr double kPoisCond = 1024.0;

// Device error code written into the context's flag by genflu when the
// rescaled inflow grid cannot be profiled; reported to callers as
// OTBL_ERR_NAN with its own message (never returned as is).
#define OTBL_DEVERR_GENFLU_GRID 0x105

#define OTBL_CUDA_TRY(ctx, call)                                        \
  do {                                                                  \
    cudaError_t e__ = (call);                                           \
    if (e__ != cudaSuccess) {                                           \
      (ctx)->err = std::string(#call) + ": " + cudaGetErrorString(e__); \
      return OTBL_ERR_CUDA;                                             \
    }                                                                   \
  } while (0)

namespace otbl {
// kernel launch wrappers (kernels.cu); each returns cudaGetLastError()
cudaError_t launch_interpx(otbl_ctx *c);
cudaError_t launch_interpy(otbl_ctx *c);
// interpyy's checkpoint region in a line scratch when it can run beside
// interpxx, else nullptr
double *interpy_ck_tail(otbl_ctx *c, double *s);
// part 0: uu, uw and the u, w CFL maxima; part 2: uv and the v maxima;
// part 1: vw, vv, ww
cudaError_t launch_products(otbl_ctx *c, int setstep, int part);
cudaError_t launch_difvisx(otbl_ctx *c);
cudaError_t launch_dt(otbl_ctx *c, int m, int setstep);
cudaError_t launch_genflu(otbl_ctx *c, int tail);
// the rhsp tail of the velocity components in the bit mask comps (1 u, 2 v,
// 4 w), in that order, on line scratch s1..s3 (second_scratch: t1..t3); the
// first kernel that writes a velocity component waits for before_vel when
// it is not null
cudaError_t launch_final(otbl_ctx *c, unsigned comps, cudaEvent_t before_vel = nullptr,
                         bool second_scratch = false);
cudaError_t launch_outflow(otbl_ctx *c);
cudaError_t launch_pois(otbl_ctx *c, int m);
cudaError_t launch_reset_max(otbl_ctx *c);
cudaError_t launch_boun_all(otbl_ctx *c);
cudaError_t launch_tiempo(otbl_ctx *c);
cudaError_t launch_energies(otbl_ctx *c);
// builds c->fmaps (false if TMA cannot address the fields, e.g. an FP32 row
// pitch that is not a multiple of 16 bytes)
bool build_final_maps(otbl_ctx *c);
// fills Work::rowc from the coefficients and this substep's implzy factors
// (after k_dt, on the same stream); a no-op without the TMA-fed tail
cudaError_t launch_tail_rows(otbl_ctx *c);
// the driver's cuTensorMapEncodeTiled (as void *), nullptr if unavailable
void *tensor_map_encoder();
bool build_x_maps(otbl_ctx *c);
// fill Work::xrowc and Work::yrowc from the coefficients (at creation and on
// new coefficients)
cudaError_t launch_x_rows(otbl_ctx *c);
cudaError_t launch_y_rows(otbl_ctx *c);
bool build_y_maps(otbl_ctx *c);
cudaError_t launch_twiddles(otbl_ctx *c);
cudaError_t launch_pois_lu(otbl_ctx *c);
// columns kr < kr_split solve in FP64 on phi64, the others in FP32 on phi32
cudaError_t launch_pois_solve(otbl_ctx *c, double *phi64, float *phi32, int kr_split);
cudaError_t launch_round_f32(otbl_ctx *c, const double *in, float *out, size_t n);
// interpyy on the tensor cores (k_ydense.cu)
cudaError_t ydense_prepare(otbl_ctx *c);
cudaError_t launch_interpy_dense(otbl_ctx *c);
bool build_ydense_maps(otbl_ctx *c);
bool build_pois_maps(otbl_ctx *c);
bool ydense_ready(const otbl_ctx *c);
// one-point statistics, statsp (k_stats.cu)
cudaError_t launch_statsp(otbl_ctx *c);
size_t stats_bytes(int nx, int ny);
size_t ydense_bytes(int ny);
// standalone pieces
cudaError_t launch_chp2x(otbl_ctx *c, const double *plan, double *pen, int jee, int to_pen);
cudaError_t launch_fourxz(otbl_ctx *c, double *fou, double *phys, int iopt, int nlines);
cudaError_t launch_cosftx(otbl_ctx *c, double *cpen, int nlines, int iopt);
// genflu table scratch: fsca[2][ny+1] | kl[2][ny+1] (int) | ggg | ntop[2] (int)
constexpr size_t genflu_tab_doubles(int ny) { return 3 * (size_t)(ny + 1) + 2; }
// dynamic shared memory of k_genflu_tab: ysca, www, yyy [2][ny+1], um(0..ny+1)
// in doubles, kf, kh [2][ny+1] in ints, and slack
constexpr size_t genflu_smem_bytes(int ny) {
  return sizeof(double) * (6 * (size_t)(ny + 1) + (ny + 2)) + sizeof(int) * 4 * (size_t)(ny + 1) + 64;
}
// genflu on caller-owned buffers with the static table scratch (no
// allocation). Its one limit: ny <= 680, where both the tables fit the
// static array and k_genflu_tab's shared memory fits the 48 KB a launch gets
// without opting in (at ny = 681 the tables still fit, the shared memory no
// longer does).
constexpr int kGenfluNoallocMaxNy = 680;
static_assert(genflu_tab_doubles(kGenfluNoallocMaxNy) <= (size_t)OTBL_GENFLU_SCRATCH_MAX,
              "genflu tables of the largest admitted ny exceed the static scratch");
static_assert(genflu_smem_bytes(kGenfluNoallocMaxNy) <= 48 * 1024,
              "genflu shared memory of the largest admitted ny exceeds 48 KB");
cudaError_t genflu_scratch_addr(int device, double **p);
cudaError_t launch_genflu_noalloc(otbl_ctx *c, double *wk, double *u, double *v, double *w, const double *u0,
                                  const double *v0, double *um, double *scal, int *err);
}  // namespace otbl
