// Streamwise (x) line operators of lip.f90 (interpxx, difvisxx), one thread
// per line. A line is a fixed (j, kr) of the plane layout; its nx values are
// read with the plane stride, so the reference's chp2x transpose is replaced
// by these strided, warp-coalesced loads (its REAL4 rounding is applied at
// the same points when OTBL_XPOSE_FP32 is set).
#include <cudaTypedefs.h>

#include <type_traits>

#include "devcommon.cuh"
#include "otbl_internal.cuh"
#include "tma.cuh"

namespace otbl {

// ---------------------------------------------------------------------------
// x-lines streamed through registers: one thread per line (pencil), the
// threads of a warp on consecutive (j, kr), so every row access is a
// coalesced 256-byte request and every coefficient a broadcast. The forward
// sweep y_i = b_i + l_i y_{i-1} (b the explicit stencil) leaves a checkpoint
// of y every K rows in scratch; the backward sweep x_i = (y_i - u_i x_{i+1})
// d_i walks the segments from the last one, recomputing each segment's y in
// registers from its checkpoint. This is the serial Thomas of lip.f90 in the
// reference's order; the traffic is about 1.5x the minimum (inputs read
// twice) with no shared memory and no scan.
//
// T is the arithmetic and output type: double, or float on the mixed path
// (the FP64 state is read and rounded on load, the FP32 coefficient copy is
// used). Element types of the buffers: interpx reads the state (double),
// difvisx reads the products (T) and the state; outputs and checkpoints T.
// ---------------------------------------------------------------------------
struct XStream {
  const void *in[3];
  const double *in2[3];  // in2: the second input of difvisxx (velocity)
  void *out[3];
  double *ck[3];         // checkpoint scratch of each line set
  int which[3], np[3];
};

// Segment lengths and occupancy per arithmetic type, measured on B200 at
// 1025x193x512 over segments of 8-32 rows and 4-8 CTAs of 128 threads per
// SM: interpxx 16 rows (FP64) / 8 rows (FP32) at >= 8 CTAs per SM; difvisxx
// 8 rows at >= 6 CTAs per SM (3.16 ms per substep in FP64 against 3.46 for
// 16 rows at 4 CTAs; 1.78 against 2.50 in FP32). FP32 interpxx runs
// unbounded (56 registers).
template <typename T>
struct XTune;
// tma: the TMA-fed kernels (k_xline_t) instead of the register streams,
// with segments of kti (interpxx) and ktd (difvisxx) planes; at 1025x193x512
// with the coefficient rows staged in the ring, FP64 RK3 step: 42.2 ms at
// kti 8, 42.5 at 4; ktd 6 against 4 and 8: 42.5, 42.7, 42.7 (FP32 ktd 8
// against 12: 30.8, 30.9). Before the staging: FP64 interpxx 1.17 ms (4
// planes; 1.49 register-streamed), difvisxx 3.02 (6 planes; 3.18); FP32
// interpxx 0.87, difvisxx 1.70.
#ifndef OTBL_XT_DI
#define OTBL_XT_DI 8
#endif
#ifndef OTBL_XT_DD
#define OTBL_XT_DD 6
#endif
#ifndef OTBL_XT_FI
#define OTBL_XT_FI 8
#endif
#ifndef OTBL_XT_FD
#define OTBL_XT_FD 8
#endif
template <>
struct XTune<double> {
  static constexpr int kxi = 16, kxd = 8, minb_i = 8, kti = OTBL_XT_DI, ktd = OTBL_XT_DD;
  static constexpr bool tma = true;
};
template <>
struct XTune<float> {
  // minb_i: 0.88 ms unbounded, 1.19 at >= 8
  static constexpr int kxi = 8, kxd = 8, minb_i = 1, kti = OTBL_XT_FI, ktd = OTBL_XT_FD;
  static constexpr bool tma = true;
};


template <typename T>
__global__ void __launch_bounds__(128, XTune<T>::minb_i) k_interpx(DCoefT<T> c, XStream a) {
  constexpr int KXI = XTune<T>::kxi;
  const int f = blockIdx.y, np = pick3(a.np, f);
  const int mp = blockIdx.x * blockDim.x + threadIdx.x;
  if (mp >= np) return;
  const int nx = c.nx, xr = c.xround, which = pick3(a.which, f);
  const double *in = static_cast<const double *>(pick3(a.in, f)) + mp;
  T *out = static_cast<T *>(pick3(a.out, f)) + mp;
  T *ck = reinterpret_cast<T *>(pick3(a.ck, f)) + mp;
  const T *icon = which == 0 ? c.inxu : c.inxv;
  const T *econ = which == 0 ? c.cofiux : c.cofivx;
  const int chi = which == 0 ? 2 : 1, chi2 = which == 0 ? 3 : 4;
  const T *ib = c.inbx;
  auto G = [&](int i) { return (T)rnd(__ldg(in + (size_t)i * np), xr); };
  const T b0 = M4(ib, chi2, 1) * G(0) + M4(ib, chi2, 2) * G(1) + M4(ib, chi2, 3) * G(2) + M4(ib, chi2, 4) * G(3);
  const T bN = M4(ib, chi, 1) * G(nx - 1) + M4(ib, chi, 2) * G(nx - 2) + M4(ib, chi, 3) * G(nx - 3) +
               M4(ib, chi, 4) * G(nx - 4);
  // right-hand side of row i from g_i, g_{i+1} (interior: lip.f90 stencil)
  auto rhs = [&](int i, T gi, T gi1) {
    return i == 0 ? b0 : (i == nx - 1 ? bN : __ldg(econ + 2 * i) * gi + __ldg(econ + 2 * i + 1) * gi1);
  };
  const int nseg = (nx + KXI - 1) / KXI;
  T y = T(0);
  for (int sg = 0; sg < nseg; ++sg) {
    const int s = sg * KXI;
    ck[(size_t)sg * np] = y;  // y of row s-1
    T gv[KXI + 1];
#pragma unroll
    for (int b = 0; b <= KXI; ++b) gv[b] = G(min(s + b, nx - 1));
#pragma unroll
    for (int b = 0; b < KXI; ++b) {
      const int i = s + b;
      if (i < nx) y = rhs(i, gv[b], gv[b + 1]) + (i > 0 ? __ldg(icon + 3 * i) : T(0)) * y;
    }
  }
  T xn = T(0);
  for (int sg = nseg - 1; sg >= 0; --sg) {
    const int s = sg * KXI;
    T gv[KXI + 1], yv[KXI];
#pragma unroll
    for (int b = 0; b <= KXI; ++b) gv[b] = G(min(s + b, nx - 1));
    T yy = ck[(size_t)sg * np];
#pragma unroll
    for (int b = 0; b < KXI; ++b) {
      const int i = s + b;
      if (i < nx) yy = rhs(i, gv[b], gv[b + 1]) + (i > 0 ? __ldg(icon + 3 * i) : T(0)) * yy;
      yv[b] = yy;
    }
#pragma unroll
    for (int b = KXI - 1; b >= 0; --b) {
      const int i = s + b;
      if (i < nx) {
        xn = (yv[b] - __ldg(icon + 3 * i + 2) * xn) * __ldg(icon + 3 * i + 1);
        out[(size_t)i * np] = (T)rnd(xn, xr);
      }
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(128, 6) k_difvisx(DCoefT<T> c, XStream a) {
  constexpr int KXD = XTune<T>::kxd;
  const int f = blockIdx.y, np = pick3(a.np, f);
  const int mp = blockIdx.x * blockDim.x + threadIdx.x;
  if (mp >= np) return;
  const int nx = c.nx, xr = c.xround, which = pick3(a.which, f);
  const T *gin = static_cast<const T *>(pick3(a.in, f)) + mp;
  const double *uin = pick3(a.in2, f) + mp;
  T *out = static_cast<T *>(pick3(a.out, f)) + mp;
  T *ck = reinterpret_cast<T *>(pick3(a.ck, f)) + mp;
  const T *icon = which == 0 ? c.dcxu : c.dcxv;
  const T *iconv = which == 0 ? c.vixu : c.vixv;
  const T *econ = which == 0 ? c.cofcxu : c.cofcxv;
  const T *econv = which == 0 ? c.cofvxu : c.cofvxv;
  const int chv = which == 0 ? 1 : 2, chv1 = chv + 2, ic = which == 0 ? 3 : 1;
  const T *db = c.dcbx, *vb = c.cofvbx;
  const T rex = c.S[OTBL_S_REX], idx = c.S[OTBL_S_IDX], uinf = c.S[OTBL_S_UINF];
  auto G = [&](int i) { return (T)rnd(__ldg(gin + (size_t)i * np), xr); };
  auto U = [&](int i) { return (T)rnd(__ldg(uin + (size_t)i * np), xr); };
  const T gb0 = M5(db, chv, 1) * G(0) + M5(db, chv, 2) * G(1) + M5(db, chv, 3) * G(2) + M5(db, chv, 4) * G(3);
  const T ub0 = M4(vb, ic, 1) * U(0) + M4(vb, ic, 2) * U(1) + M4(vb, ic, 3) * U(2) + M4(vb, ic, 4) * U(3);
  const T gbN = M5(db, chv1, 1) * G(nx - 1) + M5(db, chv1, 2) * G(nx - 2) + M5(db, chv1, 3) * G(nx - 3) +
                M5(db, chv1, 4) * G(nx - 4);
  const T uN = U(nx - 1), uN1 = U(nx - 2);
  const T ubN = M4(vb, ic + 1, 1) * uN + M4(vb, ic + 1, 2) * uN1 + M4(vb, ic + 1, 3) * U(nx - 3) +
                M4(vb, ic + 1, 4) * U(nx - 4);
  // right-hand sides of row i: convective e1 g_{i-1} + e2 g_i, viscous
  // f1 u_{i+1} + f2 u_i + f3 u_{i-1} (lip.f90:52-142)
  auto rg = [&](int i, T gm, T g0) {
    return i == 0 ? gb0 : (i == nx - 1 ? gbN : __ldg(econ + 2 * i) * gm + __ldg(econ + 2 * i + 1) * g0);
  };
  auto ru = [&](int i, T um, T u0, T up) {
    return i == 0 ? ub0
                  : (i == nx - 1 ? ubN
                                 : __ldg(econv + 3 * i) * up + __ldg(econv + 3 * i + 1) * u0 +
                                       __ldg(econv + 3 * i + 2) * um);
  };
  const int nseg = (nx + KXD - 1) / KXD;
  T yg = T(0), yu = T(0);
  for (int sg = 0; sg < nseg; ++sg) {
    const int s = sg * KXD;
    ck[(size_t)(2 * sg) * np] = yg;
    ck[(size_t)(2 * sg + 1) * np] = yu;
    T gv[KXD + 1], uv[KXD + 2];  // rows s-1 .. s+K-1 (g), s-1 .. s+K (u)
#pragma unroll
    for (int b = 0; b <= KXD; ++b) gv[b] = G(min(max(s + b - 1, 0), nx - 1));
#pragma unroll
    for (int b = 0; b <= KXD + 1; ++b) uv[b] = U(min(max(s + b - 1, 0), nx - 1));
#pragma unroll
    for (int b = 0; b < KXD; ++b) {
      const int i = s + b;
      if (i < nx) {
        yg = rg(i, gv[b], gv[b + 1]) + (i > 0 ? __ldg(icon + 3 * i) : T(0)) * yg;
        yu = ru(i, uv[b], uv[b + 1], uv[b + 2]) + (i > 0 ? __ldg(iconv + 3 * i) : T(0)) * yu;
      }
    }
  }
  T xg = T(0), xu = T(0);
  for (int sg = nseg - 1; sg >= 0; --sg) {
    const int s = sg * KXD;
    T gv[KXD + 1], uv[KXD + 2], ygv[KXD], yuv[KXD];
#pragma unroll
    for (int b = 0; b <= KXD; ++b) gv[b] = G(min(max(s + b - 1, 0), nx - 1));
#pragma unroll
    for (int b = 0; b <= KXD + 1; ++b) uv[b] = U(min(max(s + b - 1, 0), nx - 1));
    T a1 = ck[(size_t)(2 * sg) * np], a2 = ck[(size_t)(2 * sg + 1) * np];
#pragma unroll
    for (int b = 0; b < KXD; ++b) {
      const int i = s + b;
      if (i < nx) {
        a1 = rg(i, gv[b], gv[b + 1]) + (i > 0 ? __ldg(icon + 3 * i) : T(0)) * a1;
        a2 = ru(i, uv[b], uv[b + 1], uv[b + 2]) + (i > 0 ? __ldg(iconv + 3 * i) : T(0)) * a2;
      }
      ygv[b] = a1;
      yuv[b] = a2;
    }
#pragma unroll
    for (int b = KXD - 1; b >= 0; --b) {
      const int i = s + b;
      if (i < nx) {
        xg = (ygv[b] - __ldg(icon + 3 * i + 2) * xg) * __ldg(icon + 3 * i + 1);
        xu = (yuv[b] - __ldg(iconv + 3 * i + 2) * xu) * __ldg(iconv + 3 * i + 1);
        const T v = i == nx - 1 ? uinf * (uN - uN1) * idx + rex * T(0) : xg + rex * xu;
        out[(size_t)i * np] = (T)rnd(v, xr);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// The same x-line operators fed by TMA: a CTA owns TB consecutive lines of
// one field; thread 0 loads, for the next segment of K planes, boxes of 32
// lines x K+1 (K+2) planes of each input into a two-stage shared-memory ring
// counted on mbarriers (bounded waits), while every thread runs its line's
// serial sweeps from shared memory. The sequence of segments is the forward
// sweep (0..nseg-1) then the backward one (nseg-1..0). DV: difvisxx (inputs:
// the product, FP32 on the mixed path, and the FP64 velocity) or interpxx
// (input: the FP64 velocity). The arithmetic is k_interpx / k_difvisx's,
// with segments of K planes (XTune kti, ktd).
// ---------------------------------------------------------------------------
template <typename T, bool DV>
constexpr int xseg() {
  return DV ? XTune<T>::ktd : XTune<T>::kti;
}

template <typename T, bool DV, int TB>
__global__ void __launch_bounds__(TB) k_xline_t(DCoefT<T> c, XStream a, int *err, const __grid_constant__ XMaps maps) {
  constexpr int K = xseg<T, DV>(), NB = TB / 32;
  using TG = typename std::conditional<DV, T, double>::type;
  constexpr int GR = K + 1, UR = K + 2;
  constexpr int GBYTES = NB * GR * 32 * (int)sizeof(TG);
  constexpr int GB = (GBYTES + 127) / 128 * 128;
  constexpr int UBYTES = DV ? NB * UR * 32 * 8 : 0;
  constexpr int RCB = K * 16 * (int)sizeof(T);  // the segment's coefficient rows
  constexpr int STG = GB + UBYTES + RCB;
  constexpr unsigned TX = (unsigned)(GBYTES + UBYTES + RCB);
  extern __shared__ __align__(128) unsigned char smraw[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smraw + 2 * STG);
  const int f = blockIdx.y, np = pick3(a.np, f);
  const int t = threadIdx.x, mp0 = blockIdx.x * TB;
  if (mp0 >= np) return;  // the whole CTA lies past this field's lines
  const int mp = mp0 + t;
  const bool active = mp < np;
  const int mpc = active ? mp : np - 1;
  const CUtensorMap *mg = f == 0 ? &maps.g[0] : (f == 1 ? &maps.g[1] : &maps.g[2]);
  const CUtensorMap *mu = f == 0 ? &maps.u[0] : (f == 1 ? &maps.u[1] : &maps.u[2]);
  const CUtensorMap *mr = f == 0 ? &maps.r[0] : (f == 1 ? &maps.r[1] : &maps.r[2]);
  const int nx = c.nx, xr = c.xround, which = pick3(a.which, f);
  const int nseg = (nx + K - 1) / K;
  auto seg_of = [&](int it) { return it < nseg ? it : 2 * nseg - 1 - it; };
  auto issue = [&](int stg, int sg) {
    unsigned char *b = smraw + stg * STG;
    const int s0 = sg * K;
    mbar_arrive_expect_tx(&bar[stg], TX);
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      tma_load_2d(b + j * GR * 32 * (int)sizeof(TG), mg, mp0 + 32 * j, DV ? s0 - 1 : s0, &bar[stg]);
      if (DV) tma_load_2d(b + GB + j * UR * 32 * 8, mu, mp0 + 32 * j, s0 - 1, &bar[stg]);
    }
    tma_load_2d(b + GB + UBYTES, mr, 0, s0, &bar[stg]);
  };
  if (t == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (t == 0) issue(0, 0);
  T *out = static_cast<T *>(pick3(a.out, f)) + mpc;
  T *ck = reinterpret_cast<T *>(pick3(a.ck, f)) + mpc;
  const int gofs = ((t >> 5) * GR) * 32 + (t & 31), uofs = ((t >> 5) * UR) * 32 + (t & 31);
  // ---- operator setup (boundary stencils from global memory)
  T gb0, gbN, ub0 = T(0), ubN = T(0), uN = T(0), uN1 = T(0);
  const T rex = c.S[OTBL_S_REX], idx = c.S[OTBL_S_IDX], uinf = c.S[OTBL_S_UINF];
  if constexpr (DV) {
    const TG *gin = static_cast<const TG *>(pick3(a.in, f)) + mpc;
    const double *uin = pick3(a.in2, f) + mpc;
    const int chv = which == 0 ? 1 : 2, chv1 = chv + 2, ic = which == 0 ? 3 : 1;
    const T *db = c.dcbx, *vb = c.cofvbx;
    auto G = [&](int i) { return (T)rnd(__ldg(gin + (size_t)i * np), xr); };
    auto U = [&](int i) { return (T)rnd(__ldg(uin + (size_t)i * np), xr); };
    gb0 = M5(db, chv, 1) * G(0) + M5(db, chv, 2) * G(1) + M5(db, chv, 3) * G(2) + M5(db, chv, 4) * G(3);
    ub0 = M4(vb, ic, 1) * U(0) + M4(vb, ic, 2) * U(1) + M4(vb, ic, 3) * U(2) + M4(vb, ic, 4) * U(3);
    gbN = M5(db, chv1, 1) * G(nx - 1) + M5(db, chv1, 2) * G(nx - 2) + M5(db, chv1, 3) * G(nx - 3) +
          M5(db, chv1, 4) * G(nx - 4);
    uN = U(nx - 1);
    uN1 = U(nx - 2);
    ubN = M4(vb, ic + 1, 1) * uN + M4(vb, ic + 1, 2) * uN1 + M4(vb, ic + 1, 3) * U(nx - 3) +
          M4(vb, ic + 1, 4) * U(nx - 4);
  } else {
    const double *gin = static_cast<const double *>(pick3(a.in, f)) + mpc;
    const int chi = which == 0 ? 2 : 1, chi2 = which == 0 ? 3 : 4;
    const T *ib = c.inbx;
    auto G = [&](int i) { return (T)rnd(__ldg(gin + (size_t)i * np), xr); };
    gb0 = M4(ib, chi2, 1) * G(0) + M4(ib, chi2, 2) * G(1) + M4(ib, chi2, 3) * G(2) + M4(ib, chi2, 4) * G(3);
    gbN = M4(ib, chi, 1) * G(nx - 1) + M4(ib, chi, 2) * G(nx - 2) + M4(ib, chi, 3) * G(nx - 3) +
          M4(ib, chi, 4) * G(nx - 4);
  }
  // right-hand sides: interpxx e1 g_i + e2 g_{i+1}; difvisxx convective
  // e1 g_{i-1} + e2 g_i and viscous f1 u_{i+1} + f2 u_i + f3 u_{i-1}; q is
  // the plane's coefficient row in shared memory (k_x_rows' layout)
  auto rg = [&](int i, const T *q, T ga, T gb) { return i == 0 ? gb0 : (i == nx - 1 ? gbN : q[0] * ga + q[1] * gb); };
  auto ru = [&](int i, const T *q, T um, T u0, T up) {
    return i == 0 ? ub0 : (i == nx - 1 ? ubN : q[5] * up + q[6] * u0 + q[7] * um);
  };
  T yg = T(0), yu = T(0), xg = T(0), xu = T(0);
  for (int it = 0; it < 2 * nseg; ++it) {
    const int stg = it & 1;
    const bool ok = mbar_wait_bounded(&bar[stg], (it >> 1) & 1, 2000000000ull);
    if (__syncthreads_or(!ok)) {
      if (t == 0) atomicExch(err, OTBL_ERR_TIMEOUT);
      return;
    }
    if (t == 0 && it + 1 < 2 * nseg) issue(stg ^ 1, seg_of(it + 1));
    if (!active) continue;
    const int sg = seg_of(it), s0 = sg * K;
    const unsigned char *bs = smraw + stg * STG;
    const TG *gs = reinterpret_cast<const TG *>(bs) + gofs;
    const double *us = reinterpret_cast<const double *>(bs + GB) + uofs;
    const T *rcs = reinterpret_cast<const T *>(bs + GB + UBYTES);
    auto g = [&](int b) { return (T)rnd(gs[b * 32], xr); };
    auto u = [&](int b) { return (T)rnd(us[b * 32], xr); };
    if (it < nseg) {  // forward sweep, checkpoint at the segment start
      ck[(size_t)((DV ? 2 : 1) * sg) * np] = yg;
      if (DV) ck[(size_t)(2 * sg + 1) * np] = yu;
#pragma unroll
      for (int b = 0; b < K; ++b) {
        const int i = s0 + b;
        const T *q = rcs + 16 * b;
        if (i < nx) {
          yg = rg(i, q, g(b), g(b + 1)) + (i > 0 ? q[2] : T(0)) * yg;
          if (DV) yu = ru(i, q, u(b), u(b + 1), u(b + 2)) + (i > 0 ? q[8] : T(0)) * yu;
        }
      }
    } else {  // backward sweep: recompute the segment, then substitute
      T a1 = ck[(size_t)((DV ? 2 : 1) * sg) * np], a2 = DV ? ck[(size_t)(2 * sg + 1) * np] : T(0);
      T y1[K], y2[K];
#pragma unroll
      for (int b = 0; b < K; ++b) {
        const int i = s0 + b;
        const T *q = rcs + 16 * b;
        if (i < nx) {
          a1 = rg(i, q, g(b), g(b + 1)) + (i > 0 ? q[2] : T(0)) * a1;
          if (DV) a2 = ru(i, q, u(b), u(b + 1), u(b + 2)) + (i > 0 ? q[8] : T(0)) * a2;
        }
        y1[b] = a1;
        y2[b] = a2;
      }
#pragma unroll
      for (int b = K - 1; b >= 0; --b) {
        const int i = s0 + b;
        const T *q = rcs + 16 * b;
        if (i < nx) {
          xg = (y1[b] - q[4] * xg) * q[3];
          T v = xg;
          if (DV) {
            xu = (y2[b] - q[10] * xu) * q[9];
            v = i == nx - 1 ? uinf * (uN - uN1) * idx + rex * T(0) : xg + rex * xu;
          }
          out[(size_t)i * np] = (T)rnd(v, xr);
        }
      }
    }
  }
}

template <typename T, bool DV>
static void xline_t_launch(otbl_ctx *c, const DCoefT<T> &dc, const XStream &a, const XMaps &m, int npmax) {
  constexpr int K = xseg<T, DV>();
  using TG = typename std::conditional<DV, T, double>::type;
  auto smem = [&](int tb) {
    const int nb = tb / 32;
    const int gb = (nb * (K + 1) * 32 * (int)sizeof(TG) + 127) / 128 * 128;
    return 2 * (gb + (DV ? nb * (K + 2) * 32 * 8 : 0) + K * 16 * (int)sizeof(T)) + 128;
  };
  const int bs = c->tune_bs[DV ? 1 : 0];
  int *err = &c->st->err;
  if (bs <= 32) {
    cudaFuncSetAttribute(k_xline_t<T, DV, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem(32));
    k_xline_t<T, DV, 32><<<dim3((npmax + 31) / 32, 3), 32, smem(32), c->stream>>>(dc, a, err, m);
  } else if (bs <= 64) {
    cudaFuncSetAttribute(k_xline_t<T, DV, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem(64));
    k_xline_t<T, DV, 64><<<dim3((npmax + 63) / 64, 3), 64, smem(64), c->stream>>>(dc, a, err, m);
  } else {
    cudaFuncSetAttribute(k_xline_t<T, DV, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem(128));
    k_xline_t<T, DV, 128><<<dim3((npmax + 127) / 128, 3), 128, smem(128), c->stream>>>(dc, a, err, m);
  }
}

// One row of 16 T per plane i of each table (dv, which), dv 0 interpxx and
// 1 difvisxx, which 0 u-type and 1 v-type coefficients: the right-hand-side
// weights econ[2i], econ[2i+1] and the LU coefficients icon[3i..3i+2], then
// for difvisxx the viscous operator's econv[3i..3i+2] and iconv[3i..3i+2].
// k_xline_t's ring stages a segment's rows with its line boxes. Entries a
// plane does not use are 0.
template <typename T>
__global__ void __launch_bounds__(128) k_x_rows(DCoefT<T> c, T *tab) {
  const int nx = c.nx;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 4 * nx) return;
  const int dv = e / (2 * nx), which = (e / nx) & 1, i = e % nx;
  T *q = tab + (size_t)e * 16;
  for (int k = 0; k < 16; ++k) q[k] = T(0);
  const T *icon = dv ? (which == 0 ? c.dcxu : c.dcxv) : (which == 0 ? c.inxu : c.inxv);
  const T *econ = dv ? (which == 0 ? c.cofcxu : c.cofcxv) : (which == 0 ? c.cofiux : c.cofivx);
  const bool inner = i > 0 && i < nx - 1;
  if (inner) {
    q[0] = econ[2 * i];
    q[1] = econ[2 * i + 1];
  }
  for (int k = 0; k < 3; ++k) q[2 + k] = icon[3 * i + k];
  if (dv) {
    const T *iconv = which == 0 ? c.vixu : c.vixv, *econv = which == 0 ? c.cofvxu : c.cofvxv;
    for (int k = 0; k < 3; ++k) {
      if (inner) q[5 + k] = econv[3 * i + k];
      q[8 + k] = iconv[3 * i + k];
    }
  }
}

cudaError_t launch_x_rows(otbl_ctx *c) {
  const int n = 4 * c->cfg.nx;
  if (c->mixed)
    k_x_rows<float><<<(n + 127) / 128, 128, 0, c->stream>>>(c->dcf, static_cast<float *>(c->w.xrowc));
  else
    k_x_rows<double><<<(n + 127) / 128, 128, 0, c->stream>>>(c->dc, static_cast<double *>(c->w.xrowc));
  c->launches += 1;
  return cudaGetLastError();
}

// 2D map of one table of Work::xrowc: [nx planes][16 T], boxes of K planes
static bool encode_xrows(CUtensorMap *m, const void *base, size_t esz, int nx, int k) {
  auto fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
  if (!fn || ((uintptr_t)base) % 16 != 0) return false;
  const cuuint64_t dims[2] = {16, (cuuint64_t)nx};
  const cuuint64_t strides[1] = {16 * esz};
  const cuuint32_t box[2] = {16, (cuuint32_t)k};
  const cuuint32_t es[2] = {1, 1};
  const CUtensorMapDataType dt = esz == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  return fn(m, dt, 2, const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// ---- TMA descriptors (host): field [nx][np], boxes of 32 lines x rows
static bool encode_lines(CUtensorMap *m, const void *base, size_t esz, int nx, int np, int rows) {
  auto fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
  if (!fn || (np * esz) % 16 != 0 || ((uintptr_t)base) % 16 != 0) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)np, (cuuint64_t)nx};
  const cuuint64_t strides[1] = {(cuuint64_t)np * esz};
  const cuuint32_t box[2] = {32, (cuuint32_t)rows};
  const cuuint32_t es[2] = {1, 1};
  const CUtensorMapDataType dt = esz == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  return fn(m, dt, 2, const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool build_x_maps(otbl_ctx *c) {
  const int KI = c->mixed ? xseg<float, false>() : xseg<double, false>();
  const int KD = c->mixed ? xseg<float, true>() : xseg<double, true>();
  const int nx = c->cfg.nx, nz1 = c->dc.nz1, ny = c->cfg.ny;
  const int np[3] = {nz1 * (ny + 1), nz1 * ny, nz1 * (ny + 1)};
  const double *st[3] = {c->f[OTBL_F_U], c->f[OTBL_F_V], c->f[OTBL_F_W]};
  const void *pr[3] = {c->w.uu, c->w.uv, c->w.uw};
  const size_t ew = c->mixed ? sizeof(float) : sizeof(double);
  bool ok = true;
  const int which[3] = {0, 1, 1};  // u-type or v-type operator of each field
  const char *tab = static_cast<const char *>(c->w.xrowc);
  auto table = [&](int dv, int wh) { return tab + (size_t)(2 * dv + wh) * nx * 16 * ew; };
  for (int f = 0; f < 3 && ok; ++f) {
    ok = ok && encode_lines(&c->xmi.g[f], st[f], 8, nx, np[f], KI + 1);
    c->xmi.u[f] = c->xmi.g[f];  // unused by interpxx
    ok = ok && encode_xrows(&c->xmi.r[f], table(0, which[f]), ew, nx, KI);
    ok = ok && encode_lines(&c->xmd.g[f], pr[f], ew, nx, np[f], KD + 1);
    ok = ok && encode_lines(&c->xmd.u[f], st[f], 8, nx, np[f], KD + 2);
    ok = ok && encode_xrows(&c->xmd.r[f], table(1, which[f]), ew, nx, KD);
  }
  c->xmaps_ok = ok;
  return ok;
}

cudaError_t launch_interpx(otbl_ctx *c) {
  const int nz1 = c->dc.nz1, ny = c->cfg.ny;
  const int npu = nz1 * (ny + 1), npv = nz1 * ny;
  XStream a;
  const double *ins[3] = {c->f[OTBL_F_U], c->f[OTBL_F_V], c->f[OTBL_F_W]};
  void *outs[3] = {c->w.ux, c->w.vx, c->w.wx};
  double *cks[3] = {c->w.s1, c->w.s2, c->w.s3};
  const int which[3] = {0, 1, 1}, np[3] = {npu, npv, npu};
  for (int f = 0; f < 3; ++f) {
    a.in[f] = ins[f];
    a.in2[f] = nullptr;
    a.out[f] = outs[f];
    a.ck[f] = cks[f];
    a.which[f] = which[f];
    a.np[f] = np[f];
  }
  const int bs = c->tune_bs[0];
  prof_begin(c, PK_INTERPX);
  if (c->xmaps_ok && (c->mixed ? XTune<float>::tma : XTune<double>::tma)) {
    if (c->mixed)
      xline_t_launch<float, false>(c, c->dcf, a, c->xmi, npu);
    else
      xline_t_launch<double, false>(c, c->dc, a, c->xmi, npu);
  } else if (c->mixed)
    k_interpx<float><<<dim3((npu + bs - 1) / bs, 3), bs, 0, c->stream>>>(c->dcf, a);
  else
    k_interpx<double><<<dim3((npu + bs - 1) / bs, 3), bs, 0, c->stream>>>(c->dc, a);
  prof_end(c);
  c->launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_difvisx(otbl_ctx *c) {
  const int nz1 = c->dc.nz1, ny = c->cfg.ny;
  const int npu = nz1 * (ny + 1), npv = nz1 * ny;
  XStream a;
  const void *gins[3] = {c->w.uu, c->w.uv, c->w.uw};
  const double *uins[3] = {c->f[OTBL_F_U], c->f[OTBL_F_V], c->f[OTBL_F_W]};
  void *outs[3] = {c->w.cu, c->w.cv, c->w.cw};
  double *cks[3] = {c->w.s1, c->w.s2, c->w.s3};
  const int which[3] = {0, 1, 1}, np[3] = {npu, npv, npu};
  for (int f = 0; f < 3; ++f) {
    a.in[f] = gins[f];
    a.in2[f] = uins[f];
    a.out[f] = outs[f];
    a.ck[f] = cks[f];
    a.which[f] = which[f];
    a.np[f] = np[f];
  }
  const int bs = c->tune_bs[1];
  prof_begin(c, PK_DIFVISX);
  if (c->xmaps_ok && (c->mixed ? XTune<float>::tma : XTune<double>::tma)) {
    if (c->mixed)
      xline_t_launch<float, true>(c, c->dcf, a, c->xmd, npu);
    else
      xline_t_launch<double, true>(c, c->dc, a, c->xmd, npu);
  } else if (c->mixed)
    k_difvisx<float><<<dim3((npu + bs - 1) / bs, 3), bs, 0, c->stream>>>(c->dcf, a);
  else
    k_difvisx<double><<<dim3((npu + bs - 1) / bs, 3), bs, 0, c->stream>>>(c->dc, a);
  prof_end(c);
  c->launches += 1;
  return cudaGetLastError();
}

}  // namespace otbl
