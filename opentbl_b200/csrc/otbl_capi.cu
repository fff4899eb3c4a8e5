// C ABI of the B200 substep (include/otbl.h): context lifetime, state
// transfer and the stream-ordered orchestration of the kernels in
// kernels.cu, following the call order of bl_1.F90:94-125.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>

#include "otbl_internal.cuh"

using namespace otbl;

namespace {

bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
bool factors_235(int n) {
  if (n <= 0) return false;
  for (int p : {2, 3, 5})
    while (n % p == 0) n /= p;
  return n == 1;
}

int fail(otbl_ctx *c, int code, const char *msg) {
  if (c) c->err = msg;
  return code;
}

template <typename T>
int dalloc(otbl_ctx *c, T **p, size_t count) {
  void *q = nullptr;
  const size_t bytes = count * sizeof(T);
  if (cudaMalloc(&q, bytes) != cudaSuccess) {
    cudaGetLastError();
    c->err = "cudaMalloc failed (" + std::to_string(bytes) + " bytes)";
    return OTBL_ERR_OOM;
  }
  // on the context stream: the streams are non-blocking, so work on the
  // legacy default stream would not be ordered before their kernels
  cudaMemsetAsync(q, 0, bytes, c->stream);
  c->allocs.push_back(q);
  c->bytes += bytes;
  *p = static_cast<T *>(q);
  return OTBL_OK;
}

size_t field_len(const otbl_ctx *c, int id) {
  const int ut = (id == OTBL_F_U || id == OTBL_F_W || id == OTBL_F_RHSUPA || id == OTBL_F_RHSWPA);
  return otbl_field_len(c->cfg.nx, c->cfg.ny, c->cfg.nz, ut);
}

// Device coefficient pointers into a packed buffer of element type T
// (base == nullptr gives null pointers).
template <typename T>
DCoefT<T> make_dcoef(const T *base, const otbl_coef_offsets &o, const otbl_config &cfg) {
  DCoefT<T> d{};
  d.nx = cfg.nx;
  d.ny = cfg.ny;
  d.nz = cfg.nz;
  d.nz1 = 2 * (cfg.nz / 3);
  d.nz2 = d.nz1 / 2 - 1;
  d.xout = cfg.xout;
  d.xround = cfg.xpose_round;
  auto P = [&](int id) { return base ? base + o.off[id] : (const T *)nullptr; };
  d.S = P(OTBL_C_SCAL);
  d.y = P(OTBL_C_Y);
  d.dy = P(OTBL_C_DY);
  d.idy = P(OTBL_C_IDY);
  d.idyy = P(OTBL_C_IDYY);
  d.dymin = P(OTBL_C_DYMIN);
  d.kaz = P(OTBL_C_KAZ);
  d.kaz2 = P(OTBL_C_KAZ2);
  d.kvis = P(OTBL_C_KVIS);
  d.kmod = P(OTBL_C_KMOD);
  d.ayp = P(OTBL_C_AYP);
  d.vmagic = P(OTBL_C_VMAGIC);
  d.hy = P(OTBL_C_HY);
  d.inxu = P(OTBL_C_INXU);
  d.inxv = P(OTBL_C_INXV);
  d.cofiux = P(OTBL_C_COFIUX);
  d.cofivx = P(OTBL_C_COFIVX);
  d.inbx = P(OTBL_C_INBX);
  d.dcxu = P(OTBL_C_DCXU);
  d.dcxv = P(OTBL_C_DCXV);
  d.cofcxu = P(OTBL_C_COFCXU);
  d.cofcxv = P(OTBL_C_COFCXV);
  d.dcbx = P(OTBL_C_DCBX);
  d.vixu = P(OTBL_C_VIXU);
  d.vixv = P(OTBL_C_VIXV);
  d.cofvxu = P(OTBL_C_COFVXU);
  d.cofvxv = P(OTBL_C_COFVXV);
  d.cofvbx = P(OTBL_C_COFVBX);
  d.inyu = P(OTBL_C_INYU);
  d.inyv = P(OTBL_C_INYV);
  d.cofiuy = P(OTBL_C_COFIUY);
  d.cofivy = P(OTBL_C_COFIVY);
  d.inby = P(OTBL_C_INBY);
  d.dcyu = P(OTBL_C_DCYU);
  d.dcyv = P(OTBL_C_DCYV);
  d.cofcyu = P(OTBL_C_COFCYU);
  d.cofcyv = P(OTBL_C_COFCYV);
  d.dcby = P(OTBL_C_DCBY);
  d.viyu = P(OTBL_C_VIYU);
  d.viyv = P(OTBL_C_VIYV);
  d.vyui = P(OTBL_C_VYUI);
  d.vyvi = P(OTBL_C_VYVI);
  d.cofvyu = P(OTBL_C_COFVYU);
  d.cofvyv = P(OTBL_C_COFVYV);
  d.cofvby = P(OTBL_C_COFVBY);
  d.ccon = P(OTBL_C_CCON);
  return d;
}

int check(otbl_ctx *c, cudaError_t e, const char *where) {
  if (e != cudaSuccess) {
    c->err = std::string(where) + ": " + cudaGetErrorString(e);
    return OTBL_ERR_CUDA;
  }
  return OTBL_OK;
}

}  // namespace

// Mixed path: the first spanwise mode whose shifted Poisson y-system is
// well enough conditioned for FP32 (kz^2 >= max|ayp(2,j)| / kPoisCond).
static int pois_split(const otbl_config *cfg, const double *coef) {
  otbl_coef_offsets o;
  otbl_coef_layout(cfg->nx, cfg->ny, cfg->nz, &o);
  const double *ayp = coef + o.off[OTBL_C_AYP], *kaz2 = coef + o.off[OTBL_C_KAZ2];
  double amax = 0.0;
  for (int j = 1; j <= cfg->ny - 1; ++j) amax = std::max(amax, std::fabs(ayp[(j - 1) * 3 + 1]));
  const int nz2 = (2 * (cfg->nz / 3)) / 2 - 1;
  int k = 0;
  while (k <= nz2 && kaz2[k] < amax / kPoisCond) ++k;
  return k;
}

extern "C" int otbl_ctx_create(const otbl_config *cfg, const double *coef, int device, otbl_ctx **out) {
  if (!cfg || !coef || !out) return OTBL_ERR_ARG;
  *out = nullptr;
  int st = otbl_config_check(cfg);
  if (st != OTBL_OK) return st;
  if (!is_pow2(cfg->nz / 2) || cfg->nz / 2 > 512 || cfg->nz / 2 < 8) return OTBL_ERR_CONFIG;
  if (!factors_235(cfg->nx - 1) || cfg->nx - 1 > 4096) return OTBL_ERR_CONFIG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0) {
    cudaGetLastError();
    return OTBL_ERR_NODEV;
  }
  otbl_ctx *c = new otbl_ctx();
  c->cfg = *cfg;
  c->device = device;
  c->bytes = 0;
  c->launches = 0;
  c->stream = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) {
    delete c;
    return OTBL_ERR_NODEV;
  }
  // The context stream and `side` at the greatest priority, `side_lo` at the
  // least: on B200 at 1025x193x512 the products' second half beside
  // difvisxx took 52.3 ms per RK3 step this way, 52.9 at equal priorities
  // and 53.3 with the side stream first.
  int prio_lo = 0, prio_hi = 0;
  cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
  if (cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
      cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
      cudaStreamCreateWithPriority(&c->side_lo, cudaStreamNonBlocking, prio_lo) != cudaSuccess) {
    if (c->side) cudaStreamDestroy(c->side);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return OTBL_ERR_CUDA;
  }
  for (cudaEvent_t &e : c->ev)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      otbl_ctx_destroy(c);
      return OTBL_ERR_CUDA;
    }
  const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz;
  const int nz1 = 2 * (nz / 3);
  otbl_coef_offsets o;
  otbl_coef_layout(nx, ny, nz, &o);
  const size_t ncoef = o.off[OTBL_C_COUNT];
  c->coef_host.assign(coef, coef + ncoef);
#define TRY(x)                \
  do {                        \
    int s__ = (x);            \
    if (s__ != OTBL_OK) {     \
      *out = c;               \
      return s__;             \
    }                         \
  } while (0)
  TRY(dalloc(c, &c->coef_dev, ncoef));
  if (cudaMemcpyAsync(c->coef_dev, coef, ncoef * sizeof(double), cudaMemcpyHostToDevice, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess) {
    *out = c;
    return fail(c, OTBL_ERR_CUDA, "coefficient upload failed");
  }
  c->mixed = cfg->precision == OTBL_PREC_MIXED;
  c->pois_klo = pois_split(cfg, coef);
  c->dc = make_dcoef<double>(c->coef_dev, o, *cfg);
  c->dcf = make_dcoef<float>(nullptr, o, *cfg);
  if (c->mixed) {
    // FP32 copy of the packed coefficients for the FP32 operators
    std::vector<float> cf(coef, coef + ncoef);
    TRY(dalloc(c, &c->coef_dev_f, ncoef));
    if (cudaMemcpyAsync(c->coef_dev_f, cf.data(), ncoef * sizeof(float), cudaMemcpyHostToDevice, c->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess) {
      *out = c;
      return fail(c, OTBL_ERR_CUDA, "coefficient upload failed");
    }
    c->dcf = make_dcoef<float>(c->coef_dev_f, o, *cfg);
  }

  const size_t lu = otbl_field_len(nx, ny, nz, 1);
  for (int id = 0; id < OTBL_F_COUNT; ++id) {
    c->f32[id] = c->mixed && (id == OTBL_F_P || id == OTBL_F_RHSUPA || id == OTBL_F_RHSVPA || id == OTBL_F_RHSWPA);
    if (c->f32[id]) {
      float *q = nullptr;
      TRY(dalloc(c, &q, field_len(c, id)));
      c->f[id] = reinterpret_cast<double *>(q);
    } else {
      TRY(dalloc(c, &c->f[id], field_len(c, id)));
    }
  }
  for (int id = 0; id < OTBL_F_COUNT; ++id) c->f_own[id] = c->f[id];
  TRY(dalloc(c, &c->u0, (size_t)ny + 1));
  TRY(dalloc(c, &c->v0, (size_t)ny + 1));
  TRY(dalloc(c, &c->um, (size_t)ny + 1));
  TRY(dalloc(c, &c->st, 1));
  Work &w = c->w;
  void **inter[] = {&w.ux, &w.vx, &w.wx, &w.uy, &w.wy, &w.vy, &w.uu, &w.uw,
                    &w.uv, &w.vw, &w.vv, &w.ww, &w.cu, &w.cv, &w.cw};
  for (void **b : inter) {
    if (c->mixed) {
      float *q = nullptr;
      TRY(dalloc(c, &q, lu));
      *b = q;
    } else {
      double *q = nullptr;
      TRY(dalloc(c, &q, lu));
      *b = q;
    }
  }
  // s1 holds the line kernels' checkpoints; the rhsp tail's, at segments of
  // 2 rows, take 2*ceil((ny+1)/2) <= ny+2 rows of (nx-1)*nz1 columns
  TRY(dalloc(c, &w.s1, std::max(lu, (size_t)(ny + 2) * (nx - 1) * nz1)));
  TRY(dalloc(c, &w.s2, lu));
  TRY(dalloc(c, &w.s3, lu));
  TRY(dalloc(c, &w.t1, std::max(lu, (size_t)(ny + 2) * (nx - 1) * nz1)));
  TRY(dalloc(c, &w.t2, lu));
  TRY(dalloc(c, &w.t3, lu));
  const int M = nz / 2, n = nx - 1;
  TRY(dalloc(c, &w.twz, 2 * (size_t)M));
  TRY(dalloc(c, &w.twz2, 2 * (size_t)M));
  if (c->mixed) {
    TRY(dalloc(c, &w.twzf, 2 * (size_t)M));
    TRY(dalloc(c, &w.twz2f, 2 * (size_t)M));
  }
  TRY(dalloc(c, &w.twx, 2 * (size_t)n));
  TRY(dalloc(c, &w.twx2, 2 * (size_t)n));
  if (c->mixed) {
    TRY(dalloc(c, &w.twxf, 2 * (size_t)n));
    TRY(dalloc(c, &w.twx2f, 2 * (size_t)n));
  }
  TRY(dalloc(c, &w.vm_bits, (size_t)ny + 1));
  TRY(dalloc(c, &w.fac_u, 3 * (size_t)(ny + 4)));
  TRY(dalloc(c, &w.fac_v, 3 * (size_t)(ny + 4)));
  TRY(dalloc(c, &w.rowc, 2 * 16 * (size_t)(ny + 2)));
  {
    double *q = nullptr;
    TRY(dalloc(c, &q, 4 * 16 * (size_t)nx));
    w.xrowc = q;
    TRY(dalloc(c, &q, 2 * 8 * (size_t)ny));
    w.yrowc = q;
  }
  TRY(dalloc(c, &w.gf, genflu_tab_doubles(ny)));
  TRY(dalloc(c, &w.pois_dinv, (size_t)nx * ny * (nz1 / 2)));
  if (c->mixed) TRY(dalloc(c, &w.pois_dinvf, (size_t)nx * ny * (nz1 / 2)));
#undef TRY
  if (!getenv("OTBL_NO_TMA")) {
    build_final_maps(c);
    build_x_maps(c);
    build_y_maps(c);
    build_pois_maps(c);
  }
  c->ydense = (cfg->options & OTBL_OPT_YDENSE) != 0;
  if (c->ydense && check(c, ydense_prepare(c), "dense interpyy operator") != OTBL_OK) {
    *out = c;
    return OTBL_ERR_CUDA;
  }
  if (c->ydense && !getenv("OTBL_NO_TMA")) build_ydense_maps(c);
  if (check(c, launch_twiddles(c), "twiddles") != OTBL_OK || check(c, launch_pois_lu(c), "pois_lu") != OTBL_OK ||
      check(c, launch_x_rows(c), "x rows") != OTBL_OK || check(c, launch_y_rows(c), "y rows") != OTBL_OK ||
      check(c, cudaStreamSynchronize(c->stream), "init")) {
    *out = c;
    return OTBL_ERR_CUDA;
  }
  *out = c;
  return OTBL_OK;
}

extern "C" size_t otbl_ctx_bytes(const otbl_config *cfg) {
  if (!cfg || otbl_config_check(cfg) != OTBL_OK) return 0;
  const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz, nz1 = 2 * (nz / 3), M = nz / 2, n = nx - 1;
  const bool mixed = cfg->precision == OTBL_PREC_MIXED;
  otbl_coef_offsets o;
  otbl_coef_layout(nx, ny, nz, &o);
  const size_t ncoef = o.off[OTBL_C_COUNT], lu = otbl_field_len(nx, ny, nz, 1), lv = otbl_field_len(nx, ny, nz, 0);
  size_t b = ncoef * sizeof(double) + (mixed ? ncoef * sizeof(float) : 0);
  b += (2 * lu + lv) * sizeof(double) + (2 * lu + 2 * lv) * (mixed ? sizeof(float) : sizeof(double));  // state
  b += 3 * (size_t)(ny + 1) * sizeof(double) + sizeof(DState);   // u0, v0, um, scalars
  b += 15 * lu * (mixed ? sizeof(float) : sizeof(double));       // intermediates
  b += 2 * (std::max(lu, (size_t)(ny + 2) * (nx - 1) * nz1) + 2 * lu) * sizeof(double);  // s1..s3, t1..t3
  b += (4 * (size_t)M + 4 * (size_t)n) * sizeof(double) + (mixed ? (4 * (size_t)M + 4 * (size_t)n) * sizeof(float) : 0);
  b += (size_t)(ny + 1) * 8 + 6 * (size_t)(ny + 4) * sizeof(double) + genflu_tab_doubles(ny) * sizeof(double);
  b += (size_t)nx * ny * (nz1 / 2) * (sizeof(double) + (mixed ? sizeof(float) : 0));  // Poisson pivots
  if (cfg->options & OTBL_OPT_YDENSE) b += ydense_bytes(ny);     // dense interpyy operators
  b += (2 * 16 * (size_t)(ny + 2) + 4 * 16 * (size_t)nx + 2 * 8 * (size_t)ny) * sizeof(double);  // coefficient rows
  return b;
}

extern "C" int otbl_ctx_rebind(otbl_ctx *c, const otbl_config *cfg, const double *coef) {
  if (!c || !cfg || !coef) return OTBL_ERR_ARG;
  int st = otbl_config_check(cfg);
  if (st != OTBL_OK) return st;
  if (cfg->nx != c->cfg.nx || cfg->ny != c->cfg.ny || cfg->nz != c->cfg.nz || cfg->precision != c->cfg.precision ||
      cfg->options != c->cfg.options)
    return OTBL_ERR_CONFIG;
  cudaSetDevice(c->device);
  OTBL_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  otbl_coef_offsets o;
  otbl_coef_layout(cfg->nx, cfg->ny, cfg->nz, &o);
  const size_t ncoef = o.off[OTBL_C_COUNT];
  c->cfg = *cfg;
  c->coef_host.assign(coef, coef + ncoef);
  c->pois_klo = pois_split(cfg, coef);
  OTBL_CUDA_TRY(c, cudaMemcpyAsync(c->coef_dev, coef, ncoef * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  OTBL_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  c->dc = make_dcoef<double>(c->coef_dev, o, *cfg);
  if (c->mixed) {
    std::vector<float> cf(coef, coef + ncoef);
    OTBL_CUDA_TRY(c, cudaMemcpyAsync(c->coef_dev_f, cf.data(), ncoef * sizeof(float), cudaMemcpyHostToDevice,
                                     c->stream));
    OTBL_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->dcf = make_dcoef<float>(c->coef_dev_f, o, *cfg);
  }
  if (check(c, launch_pois_lu(c), "pois_lu") != OTBL_OK) return OTBL_ERR_CUDA;
  if (c->ydense && check(c, ydense_prepare(c), "dense interpyy operator") != OTBL_OK) return OTBL_ERR_CUDA;
  if (check(c, launch_x_rows(c), "x rows") != OTBL_OK) return OTBL_ERR_CUDA;
  if (check(c, launch_y_rows(c), "y rows") != OTBL_OK) return OTBL_ERR_CUDA;
  OTBL_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return OTBL_OK;
}

extern "C" void otbl_ctx_destroy(otbl_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto &r : c->prof) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (cudaEvent_t e : c->prof_pool) cudaEventDestroy(e);
  if (c->side) cudaStreamSynchronize(c->side);
  if (c->side_lo) cudaStreamSynchronize(c->side_lo);
  for (void *p : c->allocs) cudaFree(p);
  for (cudaEvent_t e : c->ev)
    if (e) cudaEventDestroy(e);
  if (c->side_lo) cudaStreamDestroy(c->side_lo);
  if (c->side) cudaStreamDestroy(c->side);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

extern "C" const char *otbl_last_error(const otbl_ctx *c) { return c ? c->err.c_str() : "null context"; }

extern "C" size_t otbl_device_bytes(const otbl_ctx *c) { return c ? c->bytes : 0; }

extern "C" long long otbl_launch_count(const otbl_ctx *c) { return c ? c->launches : 0; }

extern "C" int otbl_set_field(otbl_ctx *c, int id, const double *host) {
  if (!c || !host || id < 0 || id >= OTBL_F_COUNT) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  const size_t n = field_len(c, id);
  if (c->f32[id]) {  // FP32 storage on the mixed path: round on the host
    std::vector<float> tmp(host, host + n);
    OTBL_CUDA_TRY(c, cudaMemcpyAsync(c->f[id], tmp.data(), n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    OTBL_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return OTBL_OK;
  }
  OTBL_CUDA_TRY(c, cudaMemcpyAsync(c->f[id], host, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  OTBL_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return OTBL_OK;
}

extern "C" int otbl_get_field(otbl_ctx *c, int id, double *host) {
  if (!c || !host || id < 0 || id >= OTBL_F_COUNT) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  const size_t n = field_len(c, id);
  if (c->f32[id]) {
    std::vector<float> tmp(n);
    OTBL_CUDA_TRY(c, cudaMemcpyAsync(tmp.data(), c->f[id], n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    OTBL_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    std::copy(tmp.begin(), tmp.end(), host);
    return OTBL_OK;
  }
  OTBL_CUDA_TRY(c, cudaMemcpyAsync(host, c->f[id], n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  OTBL_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return OTBL_OK;
}

extern "C" int otbl_field_device_ptr(otbl_ctx *c, int id, double **dptr) {
  if (!c || !dptr || id < 0 || id >= OTBL_F_COUNT) return OTBL_ERR_ARG;
  if (c->f32[id]) {
    c->err = "field is stored in FP32 on the mixed-precision path";
    return OTBL_ERR_CONFIG;
  }
  *dptr = c->f[id];
  return OTBL_OK;
}

extern "C" int otbl_set_inflow(otbl_ctx *c, const double *u0, const double *v0, const double *um,
                               const otbl_inflow *s) {
  if (!c || !u0 || !v0 || !um || !s) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  const int ny = c->cfg.ny;
  DState h;
  OTBL_CUDA_TRY(c, cudaMemcpyAsync(&h, c->st, sizeof(DState), cudaMemcpyDeviceToHost, c->stream));
  OTBL_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  h.tiempo = s->tiempo;
  h.timeinit = s->timeinit;
  h.dt = s->dt;
  h.utauout = s->utauout;
  h.rthout = s->rthout;
  h.dout = s->dout;
  h.gamma1 = s->gamma1;
  h.gamma2 = s->gamma2;
  h.timec = s->timec;
  h.err = 0;
  h.dt_frozen = 0;  // a restart: the fixed-dt mode takes its dt again
  for (double &e : h.ener) e = 0.0;
  OTBL_CUDA_TRY(c, cudaMemcpyAsync(c->st, &h, sizeof(DState), cudaMemcpyHostToDevice, c->stream));
  OTBL_CUDA_TRY(c, cudaMemcpyAsync(c->u0, u0, sizeof(double) * (ny + 1), cudaMemcpyHostToDevice, c->stream));
  OTBL_CUDA_TRY(c, cudaMemcpyAsync(c->v0, v0, sizeof(double) * ny, cudaMemcpyHostToDevice, c->stream));
  OTBL_CUDA_TRY(c, cudaMemcpyAsync(c->um, um, sizeof(double) * (ny + 1), cudaMemcpyHostToDevice, c->stream));
  OTBL_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return OTBL_OK;
}

// Maps the context's device error flag (first error wins) to a status and
// its message.
static int device_error(otbl_ctx *c, int code) {
  switch (code) {
    case OTBL_ERR_TIMEOUT:
      c->err = "a device-side wait of a kernel timed out";
      return OTBL_ERR_TIMEOUT;
    case OTBL_DEVERR_GENFLU_GRID:
      c->err = "genflu: the rescaled inflow grid could not be profiled (degenerate rescaling); "
               "plane 1 holds the blended copy of plane xout";
      return OTBL_ERR_NAN;
    default:
      c->err = "non-finite value in the CFL reduction (u, v, w maxima or dt)";
      return OTBL_ERR_NAN;
  }
}

extern "C" int otbl_get_inflow(otbl_ctx *c, double *um, otbl_inflow *s) {
  if (!c) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  DState h;
  OTBL_CUDA_TRY(c, cudaMemcpyAsync(&h, c->st, sizeof(DState), cudaMemcpyDeviceToHost, c->stream));
  if (um)
    OTBL_CUDA_TRY(c, cudaMemcpyAsync(um, c->um, sizeof(double) * (c->cfg.ny + 1), cudaMemcpyDeviceToHost,
                                     c->stream));
  OTBL_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (s) {
    s->tiempo = h.tiempo;
    s->timeinit = h.timeinit;
    s->dt = h.dt;
    s->utauout = h.utauout;
    s->rthout = h.rthout;
    s->dout = h.dout;
    s->gamma1 = h.gamma1;
    s->gamma2 = h.gamma2;
    s->timec = h.timec;
    s->umax = h.umax;
    s->wmax = h.wmax;
    s->vmax = h.vmax;
  }
  if (h.err) return device_error(c, h.err);
  return OTBL_OK;
}

extern "C" int otbl_get_energies(otbl_ctx *c, double *ener) {
  if (!c || !ener) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  OTBL_CUDA_TRY(c, cudaMemcpyAsync(ener, c->st->ener, sizeof(double) * 15, cudaMemcpyDeviceToHost, c->stream));
  OTBL_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return OTBL_OK;
}

#define LAUNCH(c, x)                                       \
  do {                                                     \
    int s__ = check((c), (x), #x);                         \
    if (s__ != OTBL_OK) return s__;                        \
  } while (0)

static int rhsp_issue(otbl_ctx *c, int m, int setstep);

extern "C" int otbl_rhsp(otbl_ctx *c, int m, int setstep) {
  if (!c || m < 1 || m > 3) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  cudaStream_t main_s = c->stream;
  const int st = rhsp_issue(c, m, setstep);
  if (st != OTBL_OK) {
    // leave no side-stream work unordered behind an error
    c->stream = main_s;
    cudaEventRecord(c->ev[3], c->side);
    cudaStreamWaitEvent(main_s, c->ev[3], 0);
    cudaEventRecord(c->ev[4], c->side_lo);
    cudaStreamWaitEvent(main_s, c->ev[4], 0);
  }
  return st;
}

static int rhsp_issue(otbl_ctx *c, int m, int setstep) {
  if (m == 1) LAUNCH(c, launch_energies(c));
  if (setstep) LAUNCH(c, launch_reset_max(c));
  cudaStream_t main_s = c->stream;
  // with per-kernel timing on, everything runs on the context stream, so
  // that each event pair brackets its own kernels only
  cudaStream_t side = c->prof_on ? main_s : c->side, side_lo = c->prof_on ? main_s : c->side_lo;
  cudaError_t e = cudaSuccess;
  // Streams (all forks and joins by events, so a graph capture records them):
  //   main:    interpxx, products 0 (uu, uw), [interpyy] products 2 (uv),
  //            difvisxx, [k_dt] u tail ([genflu] before its velocity write),
  //            [products 1] v tail, [w tail]
  //   side:    interpyy, [products 0, 2] k_dt, [difvisxx] genflu,
  //            [products 1] w tail on its own line scratch
  //   side_lo: [products 2] products 1 (vw, vv, ww)
  // interpyy and interpxx only read the state (their checkpoints take the
  // head and the tail of the line scratch); each products part reads and
  // writes fields no kernel beside it touches; difvisxx reads parts 0 and
  // 2; k_dt needs the CFL maxima of parts 0 and 2; genflu needs dt, writes
  // plane 1 of u, v, w after difvisxx has read it and reads plane xout
  // before a tail rewrites it.
  const bool ypar = interpy_ck_tail(c, c->w.s2) != nullptr;
  if (ypar) {
    OTBL_CUDA_TRY(c, cudaEventRecord(c->ev[0], main_s));
    OTBL_CUDA_TRY(c, cudaStreamWaitEvent(side, c->ev[0], 0));
    c->stream = side;
    e = launch_interpy(c);
    if (e == cudaSuccess) e = cudaEventRecord(c->ev[1], side);
    c->stream = main_s;
    if (check(c, e, "launch_interpy") != OTBL_OK) return OTBL_ERR_CUDA;
    LAUNCH(c, launch_interpx(c));
  } else {
    LAUNCH(c, launch_interpx(c));
    LAUNCH(c, launch_interpy(c));
    OTBL_CUDA_TRY(c, cudaEventRecord(c->ev[1], main_s));
  }
  LAUNCH(c, launch_products(c, setstep, 0));
  OTBL_CUDA_TRY(c, cudaStreamWaitEvent(main_s, c->ev[1], 0));
  LAUNCH(c, launch_products(c, setstep, 2));
  OTBL_CUDA_TRY(c, cudaEventRecord(c->ev[0], main_s));
  // part 1 needs only interpyy, but started beside parts 0 and 2 it measured
  // no faster (42.8 against 42.7 ms per FP64 RK3 step), so it follows them
  OTBL_CUDA_TRY(c, cudaStreamWaitEvent(side_lo, c->ev[0], 0));
  c->stream = side_lo;
  e = launch_products(c, setstep, 1);
  if (e == cudaSuccess) e = cudaEventRecord(c->ev[4], side_lo);
  c->stream = main_s;
  if (check(c, e, "products part 1") != OTBL_OK) return OTBL_ERR_CUDA;
  OTBL_CUDA_TRY(c, cudaStreamWaitEvent(side, c->ev[0], 0));
  c->stream = side;
  e = launch_dt(c, m, setstep);
  if (e == cudaSuccess) e = cudaEventRecord(c->ev[1], side);
  c->stream = main_s;
  if (check(c, e, "k_dt") != OTBL_OK) return OTBL_ERR_CUDA;
  LAUNCH(c, launch_difvisx(c));
  OTBL_CUDA_TRY(c, cudaEventRecord(c->ev[2], main_s));
  OTBL_CUDA_TRY(c, cudaStreamWaitEvent(side, c->ev[2], 0));
  c->stream = side;
  e = launch_genflu(c, 1);
  if (e == cudaSuccess) e = cudaEventRecord(c->ev[3], side);
  c->stream = main_s;
  if (check(c, e, "launch_genflu") != OTBL_OK) return OTBL_ERR_CUDA;
  OTBL_CUDA_TRY(c, cudaStreamWaitEvent(main_s, c->ev[1], 0));
  LAUNCH(c, launch_final(c, 1, c->ev[3]));
  OTBL_CUDA_TRY(c, cudaStreamWaitEvent(side, c->ev[4], 0));
  c->stream = side;
  e = launch_final(c, 4, nullptr, true);
  if (e == cudaSuccess) e = cudaEventRecord(c->ev[5], side);
  c->stream = main_s;
  if (check(c, e, "w tail") != OTBL_OK) return OTBL_ERR_CUDA;
  OTBL_CUDA_TRY(c, cudaStreamWaitEvent(main_s, c->ev[4], 0));
  LAUNCH(c, launch_final(c, 2));
  OTBL_CUDA_TRY(c, cudaStreamWaitEvent(main_s, c->ev[5], 0));
  return OTBL_OK;
}

extern "C" int otbl_outflow_correction(otbl_ctx *c) {
  if (!c) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  LAUNCH(c, launch_outflow(c));
  return OTBL_OK;
}

extern "C" int otbl_pois(otbl_ctx *c, int m) {
  if (!c || m < 1 || m > 3) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  LAUNCH(c, launch_pois(c, m));
  return OTBL_OK;
}

extern "C" int otbl_substep(otbl_ctx *c, int m, int setstep) {
  int s = otbl_rhsp(c, m, setstep);
  if (s != OTBL_OK) return s;
  s = otbl_outflow_correction(c);
  if (s != OTBL_OK) return s;
  return otbl_pois(c, m);
}

extern "C" int otbl_advance(otbl_ctx *c, int nsteps) {
  if (!c || nsteps < 0) return OTBL_ERR_ARG;
  for (int s = 0; s < nsteps; ++s) {
    for (int m = 1; m <= 3; ++m) {
      const int r = otbl_substep(c, m, m == 1);
      if (r != OTBL_OK) return r;
    }
    LAUNCH(c, launch_tiempo(c));
  }
  return OTBL_OK;
}

extern "C" int otbl_sync(otbl_ctx *c) {
  if (!c) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  int err = 0;
  OTBL_CUDA_TRY(c, cudaMemcpyAsync(&err, &c->st->err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  OTBL_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (err) return device_error(c, err);
  return OTBL_OK;
}

// ---------------------------------------------------------------------------
// The reference's array surface: the state in the caller's device arrays.
// Binding stores the pointers and re-encodes the TMA descriptors that name
// state fields (host work only, no device synchronisation: launches already
// issued keep the descriptors they were given).
// ---------------------------------------------------------------------------
static int bind_fields(otbl_ctx *c, double *const *ptr, const bool *use) {
  bool changed = false;
  for (int id = 0; id < OTBL_F_COUNT; ++id) {
    if (!use[id]) continue;
    double *q = ptr[id] ? ptr[id] : c->f_own[id];
    if (q == c->f[id]) continue;
    if (c->mixed) return fail(c, OTBL_ERR_CONFIG, "caller-owned state arrays need the FP64 path");
    if (reinterpret_cast<uintptr_t>(q) % 16 != 0)
      return fail(c, OTBL_ERR_ARG, "state arrays must be 16-byte aligned");
    changed = true;
  }
  if (!changed) return OTBL_OK;
  for (int id = 0; id < OTBL_F_COUNT; ++id)
    if (use[id]) c->f[id] = ptr[id] ? ptr[id] : c->f_own[id];
  if (!getenv("OTBL_NO_TMA")) {
    build_final_maps(c);
    build_x_maps(c);
    build_y_maps(c);
    build_ydense_maps(c);
    build_pois_maps(c);
  }
  return OTBL_OK;
}

extern "C" int otbl_bind_state(otbl_ctx *c, double *u, double *v, double *w, double *p, double *rhsupa,
                               double *rhsvpa, double *rhswpa) {
  if (!c) return OTBL_ERR_ARG;
  double *ptr[OTBL_F_COUNT] = {u, v, w, p, rhsupa, rhsvpa, rhswpa};
  const bool use[OTBL_F_COUNT] = {true, true, true, true, true, true, true};
  cudaSetDevice(c->device);
  return bind_fields(c, ptr, use);
}

extern "C" int otbl_rhsp_arrays(otbl_ctx *c, double *u, double *v, double *w, double *p, double *rhsupa,
                                double *rhsvpa, double *rhswpa, int m, int setstep) {
  if (!c || !u || !v || !w || !p || !rhsupa || !rhsvpa || !rhswpa) return OTBL_ERR_ARG;
  const int st = otbl_bind_state(c, u, v, w, p, rhsupa, rhsvpa, rhswpa);
  return st != OTBL_OK ? st : otbl_rhsp(c, m, setstep);
}

extern "C" int otbl_outflow_correction_arrays(otbl_ctx *c, double *u, double *v, double *rhsupa) {
  if (!c || !u || !v || !rhsupa) return OTBL_ERR_ARG;
  double *ptr[OTBL_F_COUNT] = {u, v, nullptr, nullptr, rhsupa, nullptr, nullptr};
  const bool use[OTBL_F_COUNT] = {true, true, false, false, true, false, false};
  cudaSetDevice(c->device);
  const int st = bind_fields(c, ptr, use);
  return st != OTBL_OK ? st : otbl_outflow_correction(c);
}

extern "C" int otbl_pois_arrays(otbl_ctx *c, double *u, double *v, double *w, double *p, int m) {
  if (!c || !u || !v || !w || !p) return OTBL_ERR_ARG;
  double *ptr[OTBL_F_COUNT] = {u, v, w, p, nullptr, nullptr, nullptr};
  const bool use[OTBL_F_COUNT] = {true, true, true, true, false, false, false};
  cudaSetDevice(c->device);
  const int st = bind_fields(c, ptr, use);
  return st != OTBL_OK ? st : otbl_pois(c, m);
}

extern "C" int otbl_boun_arrays(otbl_ctx *c, double *u, double *v, double *w) {
  if (!c || !u || !v || !w) return OTBL_ERR_ARG;
  double *ptr[OTBL_F_COUNT] = {u, v, w, nullptr, nullptr, nullptr, nullptr};
  const bool use[OTBL_F_COUNT] = {true, true, true, false, false, false, false};
  cudaSetDevice(c->device);
  const int st = bind_fields(c, ptr, use);
  return st != OTBL_OK ? st : otbl_boun(c);
}

extern "C" int otbl_genflu_arrays(otbl_ctx *c, double *u, double *v, double *w) {
  if (!c || !u || !v || !w) return OTBL_ERR_ARG;
  double *ptr[OTBL_F_COUNT] = {u, v, w, nullptr, nullptr, nullptr, nullptr};
  const bool use[OTBL_F_COUNT] = {true, true, true, false, false, false, false};
  cudaSetDevice(c->device);
  const int st = bind_fields(c, ptr, use);
  return st != OTBL_OK ? st : otbl_genflu(c);
}

extern "C" int otbl_chp2x(otbl_ctx *c, double *pen, const double *plan, int jee) {
  if (!c || !plan || !pen || (jee != c->cfg.ny && jee != c->cfg.ny + 1)) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  LAUNCH(c, launch_chp2x(c, plan, pen, jee, 1));
  return OTBL_OK;
}

extern "C" int otbl_chx2p(otbl_ctx *c, const double *pen, double *plan, int jee) {
  if (!c || !plan || !pen || (jee != c->cfg.ny && jee != c->cfg.ny + 1)) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  LAUNCH(c, launch_chp2x(c, pen, plan, jee, 0));
  return OTBL_OK;
}

extern "C" int otbl_fourxz(otbl_ctx *c, double *fou, double *phys, int iopt, int nlines) {
  if (!c || !fou || !phys || nlines < 0) return OTBL_ERR_ARG;
  if (nlines == 0) return OTBL_OK;
  cudaSetDevice(c->device);
  LAUNCH(c, launch_fourxz(c, fou, phys, iopt, nlines));
  return OTBL_OK;
}

extern "C" int otbl_cosftx(otbl_ctx *c, double *cp, int nlines, int iopt) {
  if (!c || !cp || nlines < 0) return OTBL_ERR_ARG;
  if (nlines == 0) return OTBL_OK;
  cudaSetDevice(c->device);
  LAUNCH(c, launch_cosftx(c, cp, nlines, iopt));
  return OTBL_OK;
}

extern "C" int otbl_interpyy(otbl_ctx *c, double *uy, double *wy, double *vy) {
  if (!c || !uy || !wy || !vy) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  LAUNCH(c, launch_interpy(c));
  const size_t n = otbl_field_len(c->cfg.nx, c->cfg.ny, c->cfg.nz, 0);
  void *src[3] = {c->w.uy, c->w.wy, c->w.vy};
  double *dst[3] = {uy, wy, vy};
  for (int f = 0; f < 3; ++f) {
    if (c->mixed) {
      std::vector<float> tmp(n);
      OTBL_CUDA_TRY(c, cudaMemcpyAsync(tmp.data(), src[f], n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
      OTBL_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
      std::copy(tmp.begin(), tmp.end(), dst[f]);
    } else {
      OTBL_CUDA_TRY(c, cudaMemcpyAsync(dst[f], src[f], n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
  }
  OTBL_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  int err = 0;
  OTBL_CUDA_TRY(c, cudaMemcpy(&err, &c->st->err, sizeof(int), cudaMemcpyDeviceToHost));
  return err ? device_error(c, err) : OTBL_OK;
}

extern "C" int otbl_statsp(otbl_ctx *c) {
  if (!c) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  LAUNCH(c, launch_statsp(c));
  return OTBL_OK;
}

extern "C" int otbl_get_stats(otbl_ctx *c, double *host, int *samples) {
  if (!c || !host) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  const size_t n = (size_t)OTBL_NSTATS * c->cfg.nx * c->cfg.ny;
  if (!c->stats) {
    std::fill(host, host + n, 0.0);
  } else {
    OTBL_CUDA_TRY(c, cudaMemcpyAsync(host, c->stats, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    OTBL_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  }
  if (samples) *samples = c->stats_samples;
  return OTBL_OK;
}

extern "C" int otbl_reset_stats(otbl_ctx *c) {
  if (!c) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  if (c->stats)
    OTBL_CUDA_TRY(c, cudaMemsetAsync(c->stats, 0, stats_bytes(c->cfg.nx, c->cfg.ny), c->stream));
  c->stats_samples = 0;
  return OTBL_OK;
}

extern "C" int otbl_boun(otbl_ctx *c) {
  if (!c) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  LAUNCH(c, launch_boun_all(c));
  return OTBL_OK;
}

extern "C" int otbl_genflu(otbl_ctx *c) {
  if (!c) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  LAUNCH(c, launch_genflu(c, 0));
  return OTBL_OK;
}

// The success path allocates nothing: the table scratch is the static array
// of kernels.cu, found once per device (only an error path stores a message
// string in the context).
extern "C" int otbl_genflu_noalloc(otbl_ctx *c, double *u, double *v, double *w, const double *u0, const double *v0,
                                   double *um, double *scal, int *err) {
  if (!c) return OTBL_ERR_ARG;
  if (!u || !v || !w || !u0 || !v0 || !um || !scal)
    return fail(c, OTBL_ERR_ARG, "otbl_genflu_noalloc: null device pointer");
  if (c->cfg.ny > kGenfluNoallocMaxNy)
    return fail(c, OTBL_ERR_CONFIG,
                "otbl_genflu_noalloc: ny > 680 (its tables would exceed OTBL_GENFLU_SCRATCH_MAX or its "
                "shared memory 48 KB)");
  OTBL_CUDA_TRY(c, cudaSetDevice(c->device));
  double *wk = nullptr;
  OTBL_CUDA_TRY(c, genflu_scratch_addr(c->device, &wk));
  LAUNCH(c, launch_genflu_noalloc(c, wk, u, v, w, u0, v0, um, scal, err));
  return OTBL_OK;
}

extern "C" int otbl_get_stream(otbl_ctx *c, void **stream) {
  if (!c || !stream) return OTBL_ERR_ARG;
  *stream = (void *)c->stream;
  return OTBL_OK;
}

extern "C" int otbl_profile_enable(otbl_ctx *c, int on) {
  if (!c) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  OTBL_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  for (auto &r : c->prof) {
    c->prof_pool.push_back(r.a);
    c->prof_pool.push_back(r.b);
  }
  c->prof.clear();
  c->prof_open = -1;
  c->prof_on = on != 0;
  return OTBL_OK;
}

extern "C" int otbl_profile_read(otbl_ctx *c, int kind, const char **name, double *total_ms, int *count) {
  if (!c || kind < 0 || kind >= PK_COUNT) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  OTBL_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  double tot = 0.0;
  int n = 0;
  for (auto &r : c->prof) {
    if (r.kind != kind) continue;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
      tot += ms;
      ++n;
    }
  }
  if (name) *name = kProfNames[kind];
  if (total_ms) *total_ms = tot;
  if (count) *count = n;
  return OTBL_OK;
}
