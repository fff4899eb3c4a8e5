// Wall-normal (y) line operators of the substep, one thread per column
// (i, kr) of the plane layout: consecutive threads take consecutive kr, so
// every row access is a coalesced request and every per-row coefficient a
// broadcast, and there are far more columns (nx*nz1) than resident threads.
// A column's compact operators are the serial Thomas sweeps of lip.f90 in
// the reference's order: the forward sweep keeps a checkpoint every KY rows
// in scratch, the backward sweep recomputes each KY-row segment from its
// checkpoint in registers.
//   k_interpy    interpyy (lip.f90:359-440) of u, w and v in Fourier space
//   k_final_s1/2 the tail of rhsp (rhsp.F90:291-484)
//   k_pois_lu    pivots of the (x-mode, kz) y-systems of pois (once)
//   k_pois_solve their solution every substep (pois.f90:106-117, soltriy)
#include <cudaTypedefs.h>

#include <type_traits>

#include "devcommon.cuh"
#include "otbl_internal.cuh"
#include "tma.cuh"

namespace otbl {

constexpr int KY = 8;  // rows per checkpointed segment
// Segment length and occupancy of the rhsp tail (k_final_s1), per
// element type of its FP32-capable inputs; measured on B200 at
// 1025x193x512 over KF in {4, 6, 8} x CTAs/SM in {3..6}: FP64 4 rows at 4
// CTAs of 128 threads per SM (7.2 ms per substep, 7.8 at 8 rows), mixed 6
// rows at 5 CTAs (7.0 ms, 8.4 at 8 rows at 4).
template <typename W>
struct FinalTune;
#ifndef OTBL_FT_DK
#define OTBL_FT_DK 4
#define OTBL_FT_DM 4
#endif
#ifndef OTBL_FT_FK
#define OTBL_FT_FK 6
#define OTBL_FT_FM 5
#endif
// split: pass A in a kernel of its own (FP32 inputs: 6.69 against 7.09 ms;
// FP64: 7.18 against 6.84 ms fused)
// kf_tma: segment of the TMA-fed pass (k_final_tb) and its pass A. With the
// coefficient rows staged in the ring, 4 rows: rhsp tail 3.47 ms per FP64
// substep against 3.73 at 3, 3.90 at 2, 3.71 at 5 and 3.82 at 6 (mixed 2.62,
// 2.77, 2.87, 2.74, 2.72), and 3.99 with a three-stage ring; before the
// staging 2 rows were best (6.38 against 6.49 at 4).
#ifndef OTBL_FT_TK
#define OTBL_FT_TK 4
#endif
#ifndef OTBL_FT_NS
#define OTBL_FT_NS 2
#endif
// tma_a: pass A fed by TMA too (k_final_ta). With the per-row coefficients
// staged in its ring: FP64 4.00 against 4.76 ms per substep for the
// register-streamed pass A (before the staging, 6.50 against 5.94); FP32
// inputs 2.97 ms.
template <>
struct FinalTune<double> {
  static constexpr int kf = OTBL_FT_DK, minb = OTBL_FT_DM, kf_tma = OTBL_FT_TK, ns_tma = OTBL_FT_NS;
  static constexpr bool split = false, tma_a = true;
};
template <>
struct FinalTune<float> {
  static constexpr int kf = OTBL_FT_FK, minb = OTBL_FT_FM, kf_tma = OTBL_FT_TK, ns_tma = OTBL_FT_NS;
  static constexpr bool split = true, tma_a = true;
};

// interpyy, which 0: u, w (in rows ny+1), which 1: v (in rows ny); out rows
// 1..ny. blockIdx.y = field (u, w, v). T: arithmetic and output type (float
// on the mixed path, with the FP32 coefficient copy); the state is FP64.
struct InterpyArgs {
  const double *in[3];
  void *out[3];
  double *ck[3];
  int which[3];
};

template <typename T>
__global__ void __launch_bounds__(128) k_interpy(DCoefT<T> c, InterpyArgs a) {
  const int f = blockIdx.y;
  const int ny = c.ny, nz1 = c.nz1, ncol = c.nx * nz1;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  const int which = pick3(a.which, f), jin = which == 0 ? ny + 1 : ny;
  const int i = col / nz1 + 1, kr = col - (i - 1) * nz1;
  const size_t S = nz1;
  const double *g = pick3(a.in, f) + (size_t)(i - 1) * jin * nz1 + kr;
  T *o = static_cast<T *>(pick3(a.out, f)) + (size_t)(i - 1) * ny * nz1 + kr;
  T *ck = reinterpret_cast<T *>(pick3(a.ck, f)) + col;
  const T *iny = which == 0 ? c.inyu : c.inyv;
  const T *econ = which == 0 ? c.cofiuy : c.cofivy;
  const T *ib = c.inby;
  auto G = [&](int r) { return (T)__ldg(g + (size_t)min(max(r, 0), jin - 1) * S); };
  T b0 = T(0), bN;
  if (which == 0) {
    bN = M4(ib, 1, 1) * G(ny) + M4(ib, 1, 2) * G(ny - 1) + M4(ib, 1, 3) * G(ny - 2) + M4(ib, 1, 4) * G(ny - 3);
  } else {
    b0 = M4(ib, 3, 1) * G(0) + M4(ib, 3, 2) * G(1) + M4(ib, 3, 3) * G(2) + M4(ib, 3, 4) * G(3);
    bN = M4(ib, 4, 1) * G(ny - 1) + M4(ib, 4, 2) * G(ny - 2) + M4(ib, 4, 3) * G(ny - 3) + M4(ib, 4, 4) * G(ny - 4);
  }
  // right-hand side of output row r from input rows r-1, r, r+1:
  // u,w: e1 g(r) + e2 g(r+1), wall row 0; v: e2 g(r) + e1 g(r-1)
  auto rhs = [&](int r, T gm, T g0, T gp) {
    const T e1 = __ldg(econ + 2 * r), e2 = __ldg(econ + 2 * r + 1);
    const T in = which == 0 ? e1 * g0 + e2 * gp : e2 * g0 + e1 * gm;
    return r == 0 ? b0 : (r == ny - 1 ? bN : in);
  };
  const int nseg = (ny + KY - 1) / KY;
  T y = T(0);
  for (int sg = 0; sg < nseg; ++sg) {
    const int s0 = sg * KY;
    ck[(size_t)sg * ncol] = y;
    T gv[KY + 2];
#pragma unroll
    for (int b = 0; b < KY + 2; ++b) gv[b] = G(s0 + b - 1);
#pragma unroll
    for (int b = 0; b < KY; ++b) {
      const int r = s0 + b;
      if (r < ny) y = rhs(r, gv[b], gv[b + 1], gv[b + 2]) + (r > 0 ? __ldg(iny + 3 * r) : T(0)) * y;
    }
  }
  T x = T(0);
  for (int sg = nseg - 1; sg >= 0; --sg) {
    const int s0 = sg * KY;
    T gv[KY + 2], yv[KY];
#pragma unroll
    for (int b = 0; b < KY + 2; ++b) gv[b] = G(s0 + b - 1);
    T yy = ck[(size_t)sg * ncol];
#pragma unroll
    for (int b = 0; b < KY; ++b) {
      const int r = s0 + b;
      if (r < ny) yy = rhs(r, gv[b], gv[b + 1], gv[b + 2]) + (r > 0 ? __ldg(iny + 3 * r) : T(0)) * yy;
      yv[b] = yy;
    }
#pragma unroll
    for (int b = KY - 1; b >= 0; --b) {
      const int r = s0 + b;
      if (r < ny) {
        x = (yv[b] - __ldg(iny + 3 * r + 2) * x) * __ldg(iny + 3 * r + 1);
        o[(size_t)r * S] = x;
      }
    }
  }
}

// interpyy fed by TMA: a CTA owns 128 consecutive kr of one plane of one
// field; thread 0 loads, for the next segment of KYT rows, a box of 128 kr x
// KYT+2 rows of the input into a two-stage shared-memory ring on mbarriers
// (bounded waits); the segments run forward (0..nseg-1), then backward. The
// arithmetic is k_interpy's with segments of KYT rows.
template <typename T>
struct YTune;
#ifndef OTBL_YT
#define OTBL_YT 8
#endif
template <>
struct YTune<double> {
  static constexpr int kt = OTBL_YT;
};
template <>
struct YTune<float> {
  static constexpr int kt = OTBL_YT;
};

template <typename T>
__global__ void __launch_bounds__(128) k_interpy_t(DCoefT<T> c, InterpyArgs a, int *err,
                                                   const __grid_constant__ YMaps maps) {
  constexpr int K = YTune<T>::kt, TB = 128, R = K + 2;
  constexpr int RC = K * 8 * (int)sizeof(T);  // the segment's coefficient rows
  constexpr int STG = R * TB * 8 + RC;
  constexpr unsigned TX = (unsigned)STG;
  extern __shared__ __align__(128) unsigned char smraw[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smraw + 2 * STG);
  const int f = blockIdx.z;
  const int ny = c.ny, nz1 = c.nz1, ncol = c.nx * nz1;
  const int t = threadIdx.x, kr0 = blockIdx.x * TB, kr = kr0 + t, i = blockIdx.y + 1;
  const bool active = kr < nz1;
  const int krc = active ? kr : 0;
  const int which = pick3(a.which, f), jin = which == 0 ? ny + 1 : ny;
  const CUtensorMap *mg = f == 0 ? &maps.g[0] : (f == 1 ? &maps.g[1] : &maps.g[2]);
  const CUtensorMap *mr = f == 0 ? &maps.r[0] : (f == 1 ? &maps.r[1] : &maps.r[2]);
  const int nseg = (ny + K - 1) / K;
  auto seg_of = [&](int it) { return it < nseg ? it : 2 * nseg - 1 - it; };
  auto issue = [&](int stg, int sg) {
    mbar_arrive_expect_tx(&bar[stg], TX);
    tma_load_3d(smraw + stg * STG, mg, kr0, sg * K - 1, i - 1, &bar[stg]);
    tma_load_2d(smraw + stg * STG + R * TB * 8, mr, 0, sg * K, &bar[stg]);
  };
  if (t == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (t == 0) issue(0, 0);
  const size_t S = nz1;
  const int col = (i - 1) * nz1 + krc;
  const double *g = pick3(a.in, f) + (size_t)(i - 1) * jin * nz1 + krc;
  T *o = static_cast<T *>(pick3(a.out, f)) + (size_t)(i - 1) * ny * nz1 + krc;
  T *ck = reinterpret_cast<T *>(pick3(a.ck, f)) + col;
  const T *ib = c.inby;
  auto G = [&](int r) { return (T)__ldg(g + (size_t)min(max(r, 0), jin - 1) * S); };
  T b0 = T(0), bN;
  if (which == 0) {
    bN = M4(ib, 1, 1) * G(ny) + M4(ib, 1, 2) * G(ny - 1) + M4(ib, 1, 3) * G(ny - 2) + M4(ib, 1, 4) * G(ny - 3);
  } else {
    b0 = M4(ib, 3, 1) * G(0) + M4(ib, 3, 2) * G(1) + M4(ib, 3, 3) * G(2) + M4(ib, 3, 4) * G(3);
    bN = M4(ib, 4, 1) * G(ny - 1) + M4(ib, 4, 2) * G(ny - 2) + M4(ib, 4, 3) * G(ny - 3) + M4(ib, 4, 4) * G(ny - 4);
  }
  // q: the row's coefficients in shared memory (k_y_rows' layout)
  auto rhs = [&](int r, const T *q, T gm, T g0, T gp) {
    const T e1 = q[0], e2 = q[1];
    const T in = which == 0 ? e1 * g0 + e2 * gp : e2 * g0 + e1 * gm;
    return r == 0 ? b0 : (r == ny - 1 ? bN : in);
  };
  T y = T(0), x = T(0);
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
    const double *gs = reinterpret_cast<const double *>(smraw + stg * STG) + t;
    const T *rcs = reinterpret_cast<const T *>(smraw + stg * STG + R * TB * 8);
    auto gv = [&](int b) { return (T)gs[b * TB]; };  // row s0 - 1 + b
    if (it < nseg) {
      ck[(size_t)sg * ncol] = y;
#pragma unroll
      for (int b = 0; b < K; ++b) {
        const int r = s0 + b;
        const T *q = rcs + 8 * b;
        if (r < ny) y = rhs(r, q, gv(b), gv(b + 1), gv(b + 2)) + (r > 0 ? q[2] : T(0)) * y;
      }
    } else {
      T yy = ck[(size_t)sg * ncol], yv[K];
#pragma unroll
      for (int b = 0; b < K; ++b) {
        const int r = s0 + b;
        const T *q = rcs + 8 * b;
        if (r < ny) yy = rhs(r, q, gv(b), gv(b + 1), gv(b + 2)) + (r > 0 ? q[2] : T(0)) * yy;
        yv[b] = yy;
      }
#pragma unroll
      for (int b = K - 1; b >= 0; --b) {
        const int r = s0 + b;
        const T *q = rcs + 8 * b;
        if (r < ny) {
          x = (yv[b] - q[4] * x) * q[3];
          o[(size_t)r * S] = x;
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// tail of rhsp (rhsp.F90:291-484) for planes 2..nx, one velocity component
// per launch pair: RHS assembly, pressure gradient, boun, vistyy, RK3
// combination, rhs history, implzy.
// ---------------------------------------------------------------------------
// W: element type of the difvisxx outputs, the products, the pressure and
// the RHS history (float on the mixed path); the arithmetic is FP64
// throughout.
template <typename W>
struct FinalArgs {
  double *u, *v, *w;                 // state: old on entry, new on exit
  const W *p;                        // p and the RHS history: W as well
  W *rhsupa, *rhsvpa, *rhswpa;       // old on entry, new on exit
  const W *cu, *cv, *cw;             // difvisxx outputs
  const W *uv, *uw, *vw, *vv, *ww;
  const double *fac_u, *fac_v;
  const DState *st;
};

// ---------------------------------------------------------------------------
// The rhsp tail streamed through registers, one thread per column (i, kr),
// consecutive threads on consecutive kr: every row access is a coalesced
// request, every coefficient a broadcast, and there are far more columns
// (nx*nz1) than a GPU has threads, so latency is hidden by occupancy.
//   k_final_s1<.., 1>, pass A (rows ascending): the forward sweeps of
//     differzy (of the product) and vistyy (of the old velocity), with a
//     checkpoint every KF rows (FinalTune); a light kernel of its own, at
//     high occupancy.
//   k_final_s1<.., 2>, pass B (segments descending): both forward sweeps recomputed
//     from the checkpoints into registers, both back-substitutions, the RHS
//     assembly, the RK3 combination, the new RHS history, the right-hand
//     side of implzy (rows q..q+2 of the combination) and, in the same
//     descending order, its elimination with the top-down factors of k_dt
//     (implzy_factor), written to scratch.
//   k_final_s2 (rows ascending): implzy's substitution and the new
//     velocity, with the boundary values ub1, ubt; a light kernel, so that
//     this serial sweep runs at high occupancy.
// differzy and vistyy are the serial Thomas sweeps of lip.f90 in the
// reference's order; implzy is eliminated from the top row down.
// ---------------------------------------------------------------------------
template <typename W>
struct FinalStream {
  FinalArgs<W> a;
  double *ck;   // checkpoints: [2*seg + op][column]
  double *yq;   // implzy right-hand side after the descending elimination: [q][column]
  double *ub;   // ub1, ubt: [2][column]
};

// PASSES: 1 pass A only (k_final_sA, a light kernel at high occupancy),
// 2 pass B only, 3 both
template <int COMP, typename W, int PASSES, int KF = FinalTune<W>::kf>
__global__ void __launch_bounds__(128, PASSES == 1 ? 6 : FinalTune<W>::minb)
    k_final_s1(DCoef c, FinalStream<W> fs) {
  const FinalArgs<W> &a = fs.a;
  const int nx = c.nx, ny = c.ny, nz1 = c.nz1;
  const int ncol = (nx - 1) * nz1;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  const int i = col / nz1 + 2, kr = col - (i - 2) * nz1;
  const int k = kr >> 1, odd = kr & 1, pof = odd ? -1 : 1;
  const bool last = i == nx;
  const int jee = COMP == 1 ? ny : ny + 1, n = jee - 2;
  const int krows = COMP == 0 ? ny + 1 : ny;
  const size_t PU = (size_t)(ny + 1) * nz1, PV = (size_t)ny * nz1;
  const size_t pl = (size_t)(i - 1) * (COMP == 1 ? PV : PU), plv = (size_t)(i - 1) * PV;
  const size_t S = nz1;  // row stride
  const W *prod = (COMP == 0 ? a.uv : (COMP == 1 ? a.vv : a.vw)) + plv + kr;
  const W *kp = (COMP == 0 ? a.uw : (COMP == 1 ? a.vw : a.ww)) + (COMP == 0 ? pl : plv) + kr + pof;
  double *vel = (COMP == 0 ? a.u : (COMP == 1 ? a.v : a.w)) + pl + kr;
  const W *cX = (COMP == 0 ? a.cu : (COMP == 1 ? a.cv : a.cw)) + pl + kr;
  W *hp = (COMP == 0 ? a.rhsupa : (COMP == 1 ? a.rhsvpa : a.rhswpa)) + pl + kr;
  const W *pc = a.p + plv + kr;
  const double kz = c.kaz[k], kv = c.kvis[k];
  const double var1 = a.st->var1, var3 = a.st->var3, var4 = a.st->var4;
  const double v2 = last ? 0.0 : a.st->var2;
  const double idxx = c.S[OTBL_S_IDXX];
  const double *ib = c.inby, *cc = c.ccon;
  const double sgn = odd ? 1.0 : -1.0;
  const int which = COMP == 1 ? 1 : 0;
  const double *dcy = which == 0 ? c.dcyu : c.dcyv, *ecd = which == 0 ? c.cofcyu : c.cofcyv;
  const double *viy = which == 0 ? c.viyu : c.viyv, *ecv = which == 0 ? c.cofvyu : c.cofvyv;
  const double *vyi = which == 0 ? c.vyui : c.vyvi;
  const double *fac = COMP == 1 ? a.fac_v : a.fac_u;
  auto Pg = [&](int r) { return (double)__ldg(prod + (size_t)min(max(r, 0), ny - 1) * S); };
  auto Vg = [&](int r) { return __ldg(vel + (size_t)min(max(r, 0), jee - 1) * S); };
  // velocity after the pressure gradient (rhsp.F90:291-339) at row r
  auto star = [&](int r, double o) -> double {
    const int rp = min(r, ny - 1);
    if (COMP == 0)
      return last ? o
                  : o - var1 * idxx * ((double)__ldg(pc + PV + (size_t)rp * S) - (double)__ldg(pc + (size_t)rp * S));
    if (COMP == 1)
      return o - var1 * c.idyy[r] *
                     ((double)__ldg(pc + (size_t)min(r + 1, ny - 1) * S) - (double)__ldg(pc + (size_t)rp * S));
    const double pp = (double)__ldg(pc + (size_t)rp * S + pof);
    const double av = var1 * kz;
    return o - (odd ? av * pp : -av * pp);
  };
  // boundary stencils of differzy (prod) and vistyy (velocity), boun values
  const int chv = which == 0 ? 3 : 1, cha = chv + 1, ic = which == 0 ? 3 : 1;
  const double *db = c.dcby, *vb = c.cofvby;
  double bot = 0.0, top = 0.0;
  if (!last) {
    bot = M4(db, chv, 1) * Pg(0) + M4(db, chv, 2) * Pg(1) + M4(db, chv, 3) * Pg(2) + M4(db, chv, 4) * Pg(3);
    top = M4(db, cha, 1) * Pg(ny - 1) + M4(db, cha, 2) * Pg(ny - 2) + M4(db, cha, 3) * Pg(ny - 3) +
          M4(db, cha, 4) * Pg(ny - 4);
  }
  const double b0 = M4(vb, ic, 1) * Vg(0) + M4(vb, ic, 2) * Vg(1) + M4(vb, ic, 3) * Vg(2) + M4(vb, ic, 4) * Vg(3);
  const double bN = M4(vb, ic + 1, 1) * Vg(jee - 1) + M4(vb, ic + 1, 2) * Vg(jee - 2) +
                    M4(vb, ic + 1, 3) * Vg(jee - 3) + M4(vb, ic + 1, 4) * Vg(jee - 4);
  double ub1 = 0.0, ubt = 0.0;
  if (COMP == 1) {
    ubt = kr == 0 ? c.vmagic[i - 1] : 0.0;
  } else {
    const double s2 = star(1, Vg(1)), s3 = star(2, Vg(2)), s4 = star(3, Vg(3));
    const double sn = star(ny - 1, Vg(ny - 1)), sn1 = star(ny - 2, Vg(ny - 2)), sn2 = star(ny - 3, Vg(ny - 3));
    ub1 = -1.0 / M4(ib, 2, 1) * (M4(ib, 2, 2) * s2 + M4(ib, 2, 3) * s3 + M4(ib, 2, 4) * s4);
    ubt = -1.0 / M2(cc, 1, 1) * (M2(cc, 1, 2) * sn + M2(cc, 1, 3) * sn1 + M2(cc, 1, 4) * sn2);
  }
  // right-hand sides of row r from rows r-1, r, r+1 of the product (g) and
  // the old velocity (u)
  auto rd = [&](int r, double gm, double g0, double gp) {
    const double in = which == 0 ? __ldg(ecd + 2 * r + 1) * g0 + __ldg(ecd + 2 * r) * gm
                                 : __ldg(ecd + 2 * r + 1) * gp + __ldg(ecd + 2 * r) * g0;
    return r == 0 ? bot : (r == jee - 1 ? top : in);
  };
  auto rv = [&](int r, double um, double u0, double up) {
    const double in = __ldg(ecv + 3 * r) * up + __ldg(ecv + 3 * r + 1) * u0 + __ldg(ecv + 3 * r + 2) * um;
    return r == 0 ? b0 : (r == jee - 1 ? bN : in);
  };
  const int nseg = (jee + KF - 1) / KF;
  double *ck = fs.ck + col;
  // ---- pass A: forward sweeps, checkpoints every KF rows; the loads go in
  // batches of KA >= KF rows (a multiple of KF), so that short checkpoint
  // segments still keep many loads in flight
  if constexpr ((PASSES & 1) != 0) {
  constexpr int KA = KF >= 8 ? KF : (8 / KF) * KF;
  double yd = 0.0, yv = 0.0;
  for (int s0 = 0; s0 < jee; s0 += KA) {
    double gv[KA + 2], uv[KA + 2];  // rows s0-1 .. s0+KA
#pragma unroll
    for (int b = 0; b < KA + 2; ++b) {
      gv[b] = last ? 0.0 : Pg(s0 + b - 1);
      uv[b] = Vg(s0 + b - 1);
    }
#pragma unroll
    for (int b = 0; b < KA; ++b) {
      const int r = s0 + b;
      if (r % KF == 0 && r < jee) {  // y of row r-1 at the start of segment r/KF
        ck[(size_t)(2 * (r / KF)) * ncol] = yd;
        ck[(size_t)(2 * (r / KF) + 1) * ncol] = yv;
      }
      if (r < jee) {
        if (!last) yd = rd(r, gv[b], gv[b + 1], gv[b + 2]) + (r > 0 ? __ldg(dcy + 3 * r) : 0.0) * yd;
        yv = rv(r, uv[b], uv[b + 1], uv[b + 2]) + (r > 0 ? __ldg(viy + 3 * r) : 0.0) * yv;
      }
    }
  }
  }
  if constexpr ((PASSES & 2) == 0) return;
  // ---- pass B: back-substitutions and everything row-local, rows descending
  const double a1raw = fac[3 * (jee + 1)], a3raw = fac[3 * (jee + 1) + 1];
  double xd = 0.0, xv = 0.0;
  double R1 = 0.0, R2 = 0.0, R3 = 0.0;       // RHS rows 1..3 (wall row of u,w)
  double res1 = 0.0, res2 = 0.0;             // combination of rows r+1, r+2
  double *yq = fs.yq + col;
  double yel = 0.0;  // implzy right-hand side of row q+1 after elimination
  for (int sg = nseg - 1; sg >= 0; --sg) {
    const int s0 = sg * KF;
    double gv[KF + 2], uv[KF + 2], ydv[KF], yvv[KF];
#pragma unroll
    for (int b = 0; b < KF + 2; ++b) {
      gv[b] = last ? 0.0 : Pg(s0 + b - 1);
      uv[b] = Vg(s0 + b - 1);
    }
    double ad = ck[(size_t)(2 * sg) * ncol], av = ck[(size_t)(2 * sg + 1) * ncol];
#pragma unroll
    for (int b = 0; b < KF; ++b) {
      const int r = s0 + b;
      if (r < jee) {
        if (!last) ad = rd(r, gv[b], gv[b + 1], gv[b + 2]) + (r > 0 ? __ldg(dcy + 3 * r) : 0.0) * ad;
        av = rv(r, uv[b], uv[b + 1], uv[b + 2]) + (r > 0 ? __ldg(viy + 3 * r) : 0.0) * av;
      }
      ydv[b] = ad;
      yvv[b] = av;
    }
    double cxv[KF], kpv[KF], hv[KF];
#pragma unroll
    for (int b = 0; b < KF; ++b) {
      const int rr = min(s0 + b, jee - 1);
      cxv[b] = (double)__ldg(cX + (size_t)rr * S);
      kpv[b] = last ? 0.0 : (double)__ldg(kp + (size_t)min(rr, krows - 1) * S);
      hv[b] = (double)__ldg(hp + (size_t)rr * S);
    }
#pragma unroll
    for (int b = KF - 1; b >= 0; --b) {
      const int r = s0 + b, j = r + 1;
      if (r >= jee) continue;
      if (!last) xd = (ydv[b] - __ldg(dcy + 3 * r + 2) * xd) * __ldg(dcy + 3 * r + 1);
      xv = (yvv[b] - __ldg(viy + 3 * r + 2) * xv) * __ldg(viy + 3 * r + 1);
      // RHS assembly (rhsp.F90:164-169, 181-204, 351-418, 423-445)
      const double d1 = last ? 0.0 : xd;
      const double u0 = uv[b + 1];
      double R = cxv[b];
      const double kzt = sgn * kz * ((!last && (COMP != 2 || r < ny)) ? kpv[b] : 0.0);
      if (COMP == 0) {
        if (!last) {
          R = (d1 + kzt) + R;
          if (j >= 2 && j <= ny) R = R - u0 * kv;
        }
      } else if (COMP == 1) {
        if (!last) {
          if (j >= 2 && j <= ny - 1) R = R - u0 * kv;
          R = R + kzt;
          R = R + d1;
        }
        if (j == 1 || j == ny) R = 0.0;
      } else {
        if (!last) {
          if (j >= 2 && j <= ny) R = R - u0 * kv;
          R = R + d1;
          if (j <= ny) R = R + kzt;
        }
      }
      if (COMP != 1) {  // wall and top rows of the u,w RHS (rhsp.F90:438-442)
        if (r == jee - 1) R = 0.0;
        if (r == 0) R = -1.0 / M4(ib, 2, 1) * (M4(ib, 2, 2) * R1 + M4(ib, 2, 3) * R2 + M4(ib, 2, 4) * R3);
        if (r == 3) R3 = R;
        if (r == 2) R2 = R;
        if (r == 1) R1 = R;
      }
      // RK3 combination and the new RHS history (rhsp.F90:448-475)
      const double st = r == 0 ? ub1 : (r == jee - 1 ? ubt : star(r, u0));
      const double res = st - (var3 * R + v2 * xv + var4 * hv[b]);
      hp[(size_t)r * S] = (W)R;
      // implzy right-hand side of row q = r from rows r..r+2 (lip.f90:528-597)
      if (r < n) {
        double v = __ldg(vyi + 3 * (r + 1)) * res + __ldg(vyi + 3 * (r + 1) + 1) * res1 +
                   __ldg(vyi + 3 * (r + 1) + 2) * res2;
        if (r == 0) v = v - a1raw * ub1;
        if (r == n - 1) v = v - a3raw * ubt;
        yel = v + fac[3 * (r + 2) + 2] * yel;
        yq[(size_t)r * ncol] = yel;
      }
      res2 = res1;
      res1 = res;
    }
  }
  fs.ub[col] = ub1;
  fs.ub[(size_t)ncol + col] = ubt;
}

// implzy substitution x_q = (y_q - A_q x_{q-1}) / B'_q on the eliminated
// right-hand side of k_final_s1 (rows q = 0..n-1 are velocity rows q+1),
// then the boundary rows ub1, ubt
template <int COMP>
__global__ void __launch_bounds__(128) k_final_s2(DCoef c, double *u, double *v, double *w, const double *fac_u,
                                                  const double *fac_v, const double *__restrict__ yqb,
                                                  const double *__restrict__ ub) {
  const int nx = c.nx, ny = c.ny, nz1 = c.nz1;
  const int ncol = (nx - 1) * nz1;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  const int i = col / nz1 + 2, kr = col - (i - 2) * nz1;
  const int jee = COMP == 1 ? ny : ny + 1, n = jee - 2;
  const size_t PU = (size_t)(ny + 1) * nz1, PV = (size_t)ny * nz1;
  double *vel = (COMP == 0 ? u : (COMP == 1 ? v : w)) + (size_t)(i - 1) * (COMP == 1 ? PV : PU) + kr;
  const double *fac = COMP == 1 ? fac_v : fac_u;
  const double *yq = yqb + col;
  constexpr int K = 8;
  double x = 0.0;
  for (int q0 = 0; q0 < n; q0 += K) {
    double yv[K];
#pragma unroll
    for (int b = 0; b < K; ++b) yv[b] = yq[(size_t)min(q0 + b, n - 1) * ncol];
#pragma unroll
    for (int b = 0; b < K; ++b) {
      const int q = q0 + b;
      if (q < n) {
        x = (yv[b] - __ldg(fac + 3 * (q + 2)) * x) * __ldg(fac + 3 * (q + 2) + 1);
        vel[(size_t)(q + 1) * nz1] = x;
      }
    }
  }
  vel[0] = ub[col];
  vel[(size_t)(jee - 1) * nz1] = ub[(size_t)ncol + col];
}

// ---------------------------------------------------------------------------
// Pass B of the rhsp tail fed by TMA. A CTA owns 128 consecutive kr of one
// plane i (one column per thread); thread 0 loads, for the next segment of
// KF rows (descending), one box per field (the product and the velocity on
// rows s0-1..s0+KF, the difvisxx output, the kz product and the RHS history
// on rows s0..s0+KF-1, the pressure rows that component's pressure
// gradient needs)
// into a two-stage shared-memory ring, counted on one mbarrier per stage,
// while all threads work on the current segment from shared memory. Element
// (row b, column t) of a box is at b*128 + t, so each thread's reads are
// conflict-free. Rows outside the field read as 0 and are not used. The
// arithmetic is k_final_s1's pass B, operation for operation.
// ---------------------------------------------------------------------------
template <typename W, int COMP>
struct FinalBox {
  static constexpr int KF = FinalTune<W>::kf_tma, T = 128, E = (int)sizeof(W);
  // pressure box: u needs planes i, i+1 on rows s0..s0+KF-1, v rows
  // s0..s0+KF of plane i, w rows s0..s0+KF-1 of plane i
  static constexpr int PR = COMP == 1 ? KF + 1 : KF, PP = COMP == 0 ? 2 : 1;
  static constexpr int r128(int b) { return (b + 127) / 128 * 128; }
  static constexpr int prod = 0;                              // W (KF+2) rows
  static constexpr int vel = prod + r128((KF + 2) * T * E);   // double (KF+2) rows
  static constexpr int cx = vel + (KF + 2) * T * 8;           // W KF rows
  static constexpr int kp = cx + r128(KF * T * E);            // W KF rows
  static constexpr int hp = kp + r128(KF * T * E);            // W KF rows
  static constexpr int p = hp + r128(KF * T * E);             // W PR x PP
  static constexpr int rc = p + r128(PR * PP * T * E);         // KF coefficient rows
  static constexpr int stage = rc + KF * 128;
  static constexpr unsigned tx =
      (unsigned)((KF + 2) * T * E + (KF + 2) * T * 8 + 3 * KF * T * E + PR * PP * T * E + KF * 128);
  static constexpr int NS = FinalTune<W>::ns_tma;  // ring stages
  static constexpr int smem = NS * stage + 128;    // the stages and the barriers
};

template <int COMP, typename W>
__global__ void __launch_bounds__(128) k_final_tb(DCoef c, DCoefT<W> cw, FinalStream<W> fs, int *err,
                                                  const __grid_constant__ FinalMaps maps) {
  using B = FinalBox<W, COMP>;
  constexpr int KF = B::KF, TB = B::T;
  extern __shared__ __align__(128) unsigned char smraw[];
  constexpr int NS = B::NS;
  uint64_t *full = reinterpret_cast<uint64_t *>(smraw + NS * B::stage);
  const FinalArgs<W> &a = fs.a;
  const int nx = c.nx, ny = c.ny, nz1 = c.nz1;
  const int ncol = (nx - 1) * nz1;
  const int t = threadIdx.x;
  const int i = blockIdx.y + 2, kr0 = blockIdx.x * TB, kr = kr0 + t;
  const bool active = kr < nz1;
  const int col = (i - 2) * nz1 + kr;
  const int k = kr >> 1, odd = kr & 1;
  const bool last = i == nx;
  const int jee = COMP == 1 ? ny : ny + 1, n = jee - 2;
  const int nseg = (jee + KF - 1) / KF;
  // ---- the ring: thread 0 initialises the barriers and loads segment nseg-1
  auto issue = [&](int stg, int sg) {
    unsigned char *b = smraw + stg * B::stage;
    const int s0 = sg * KF;
    mbar_arrive_expect_tx(&full[stg], B::tx);
    tma_load_3d(b + B::prod, &maps.prod, kr0, s0 - 1, i - 1, &full[stg]);
    tma_load_3d(b + B::vel, &maps.vel, kr0, s0 - 1, i - 1, &full[stg]);
    tma_load_3d(b + B::cx, &maps.cx, kr0, s0, i - 1, &full[stg]);
    tma_load_3d(b + B::kp, &maps.kp, kr0, s0, i - 1, &full[stg]);
    tma_load_3d(b + B::hp, &maps.hp, kr0, s0, i - 1, &full[stg]);
    tma_load_3d(b + B::p, &maps.p, kr0, s0, i - 1, &full[stg]);
    tma_load_2d(b + B::rc, &maps.rc, 0, s0, &full[stg]);
  };
  if (t == 0) {
    for (int q = 0; q < NS; ++q) mbar_init(&full[q], 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (t == 0)  // the first NS-1 segments (descending)
    for (int q = 0; q < NS - 1 && q < nseg; ++q) issue(q, nseg - 1 - q);
  // ---- per-column setup (as k_final_s1)
  const int pof = odd ? -1 : 1;
  const size_t PU = (size_t)(ny + 1) * nz1, PV = (size_t)ny * nz1;
  const size_t pl = (size_t)(i - 1) * (COMP == 1 ? PV : PU), plv = (size_t)(i - 1) * PV;
  const size_t S = nz1;
  const int krc = active ? kr : 0;  // inactive threads read a valid column and write nothing
  const W *prod = (COMP == 0 ? a.uv : (COMP == 1 ? a.vv : a.vw)) + plv + krc;
  const double *vel = (COMP == 0 ? a.u : (COMP == 1 ? a.v : a.w)) + pl + krc;
  W *hp = (COMP == 0 ? a.rhsupa : (COMP == 1 ? a.rhsvpa : a.rhswpa)) + pl + krc;
  const W *pc = a.p + plv + krc;
  const double kz = c.kaz[k], kv = c.kvis[k];
  const double var1 = a.st->var1, var3 = a.st->var3, var4 = a.st->var4;
  const double v2 = last ? 0.0 : a.st->var2;
  const double idxx = c.S[OTBL_S_IDXX];
  const double *ib = c.inby, *cc = c.ccon;
  const double sgn = odd ? 1.0 : -1.0;
  const int which = COMP == 1 ? 1 : 0;
  // differzy and vistyy run in W on the coefficient copy cw (FP32 on the
  // mixed path); the RHS assembly, RK3 combination and implzy in FP64
  // (per-row coefficients: k_tail_rows' rows, staged with each segment)
  const double *fac = COMP == 1 ? a.fac_v : a.fac_u;
  auto Pg = [&](int r) { return (double)__ldg(prod + (size_t)min(max(r, 0), ny - 1) * S); };
  auto Vg = [&](int r) { return __ldg(vel + (size_t)min(max(r, 0), jee - 1) * S); };
  // velocity after the pressure gradient (rhsp.F90:291-339), from global
  // memory (boundary rows) ...
  auto star_g = [&](int r, double o) -> double {
    const int rp = min(r, ny - 1);
    if (COMP == 0)
      return last ? o
                  : o - var1 * idxx * ((double)__ldg(pc + PV + (size_t)rp * S) - (double)__ldg(pc + (size_t)rp * S));
    if (COMP == 1)
      return o - var1 * c.idyy[r] *
                     ((double)__ldg(pc + (size_t)min(r + 1, ny - 1) * S) - (double)__ldg(pc + (size_t)rp * S));
    const double pp = (double)__ldg(pc + (size_t)rp * S + pof);
    const double av = var1 * kz;
    return o - (odd ? av * pp : -av * pp);
  };
  const int chv = which == 0 ? 3 : 1, cha = chv + 1, ic = which == 0 ? 3 : 1;
  const W *db = cw.dcby, *vb = cw.cofvby;
  W bot = W(0), top = W(0);
  if (!last) {
    bot = M4(db, chv, 1) * (W)Pg(0) + M4(db, chv, 2) * (W)Pg(1) + M4(db, chv, 3) * (W)Pg(2) + M4(db, chv, 4) * (W)Pg(3);
    top = M4(db, cha, 1) * (W)Pg(ny - 1) + M4(db, cha, 2) * (W)Pg(ny - 2) + M4(db, cha, 3) * (W)Pg(ny - 3) +
          M4(db, cha, 4) * (W)Pg(ny - 4);
  }
  const W b0 = M4(vb, ic, 1) * (W)Vg(0) + M4(vb, ic, 2) * (W)Vg(1) + M4(vb, ic, 3) * (W)Vg(2) + M4(vb, ic, 4) * (W)Vg(3);
  const W bN = M4(vb, ic + 1, 1) * (W)Vg(jee - 1) + M4(vb, ic + 1, 2) * (W)Vg(jee - 2) +
               M4(vb, ic + 1, 3) * (W)Vg(jee - 3) + M4(vb, ic + 1, 4) * (W)Vg(jee - 4);
  double ub1 = 0.0, ubt = 0.0;
  if (COMP == 1) {
    ubt = kr == 0 ? c.vmagic[i - 1] : 0.0;
  } else {
    const double s2 = star_g(1, Vg(1)), s3 = star_g(2, Vg(2)), s4 = star_g(3, Vg(3));
    const double sn = star_g(ny - 1, Vg(ny - 1)), sn1 = star_g(ny - 2, Vg(ny - 2)), sn2 = star_g(ny - 3, Vg(ny - 3));
    ub1 = -1.0 / M4(ib, 2, 1) * (M4(ib, 2, 2) * s2 + M4(ib, 2, 3) * s3 + M4(ib, 2, 4) * s4);
    ubt = -1.0 / M2(cc, 1, 1) * (M2(cc, 1, 2) * sn + M2(cc, 1, 3) * sn1 + M2(cc, 1, 4) * sn2);
  }
  // q: the row's W coefficients in shared memory (k_tail_rows' layout)
  auto rd = [&](int r, const W *q, W gm, W g0, W gp) {
    const W in = which == 0 ? q[1] * g0 + q[0] * gm : q[1] * gp + q[0] * g0;
    return r == 0 ? bot : (r == jee - 1 ? top : in);
  };
  auto rv = [&](int r, const W *q, W um, W u0, W up) {
    const W in = q[5] * up + q[6] * u0 + q[7] * um;
    return r == 0 ? b0 : (r == jee - 1 ? bN : in);
  };
  const W *ck = reinterpret_cast<const W *>(fs.ck) + (active ? col : 0);
  double *yq = fs.yq + (active ? col : 0);
  const double a1raw = fac[3 * (jee + 1)], a3raw = fac[3 * (jee + 1) + 1];
  W xd = W(0), xv = W(0);
  double R1 = 0.0, R2 = 0.0, R3 = 0.0;
  double res1 = 0.0, res2 = 0.0;
  double yel = 0.0;
  W ckd = ck[(size_t)(2 * (nseg - 1)) * ncol], ckv = ck[(size_t)(2 * (nseg - 1) + 1) * ncol];
  const int tk = t ^ 1;  // kr+1 for even kr, kr-1 for odd kr (the chunk starts even)
  for (int sg = nseg - 1, it = 0; sg >= 0; --sg, ++it) {
    const int stg = it % NS;
    const bool ok = mbar_wait_bounded(&full[stg], (it / NS) & 1, 2000000000ull);
    if (__syncthreads_or(!ok)) {  // the stage of iteration it-1 is free from here on
      if (t == 0) atomicExch(err, OTBL_ERR_TIMEOUT);
      return;
    }
    if (t == 0 && sg >= NS - 1) issue((it + NS - 1) % NS, sg - (NS - 1));
    const int s0 = sg * KF;
    const unsigned char *bs = smraw + stg * B::stage;
    const W *sp = reinterpret_cast<const W *>(bs + B::prod);
    const double *sv = reinterpret_cast<const double *>(bs + B::vel);
    const W *sc = reinterpret_cast<const W *>(bs + B::cx);
    const W *sk = reinterpret_cast<const W *>(bs + B::kp);
    const W *sh = reinterpret_cast<const W *>(bs + B::hp);
    const W *spp = reinterpret_cast<const W *>(bs + B::p);
    const double *rcs = reinterpret_cast<const double *>(bs + B::rc);
    W ad = ckd, av = ckv;
    if (sg >= 1) {  // next segment's checkpoints, ahead of use
      ckd = ck[(size_t)(2 * (sg - 1)) * ncol];
      ckv = ck[(size_t)(2 * (sg - 1) + 1) * ncol];
    }
    if (!active) continue;
    W ydv[KF], yvv[KF];
#pragma unroll
    for (int b = 0; b < KF; ++b) {
      const int r = s0 + b;
      const W *q = reinterpret_cast<const W *>(rcs + 16 * b + 5);
      if (r < jee) {
        if (!last)
          ad = rd(r, q, sp[b * TB + t], sp[(b + 1) * TB + t], sp[(b + 2) * TB + t]) + (r > 0 ? q[2] : W(0)) * ad;
        av = rv(r, q, (W)sv[b * TB + t], (W)sv[(b + 1) * TB + t], (W)sv[(b + 2) * TB + t]) +
             (r > 0 ? q[8] : W(0)) * av;
      }
      ydv[b] = ad;
      yvv[b] = av;
    }
#pragma unroll
    for (int b = KF - 1; b >= 0; --b) {
      const int r = s0 + b, j = r + 1;
      if (r >= jee) continue;
      const double *rq = rcs + 16 * b;
      const W *q = reinterpret_cast<const W *>(rq + 5);
      if (!last) xd = (ydv[b] - q[4] * xd) * q[3];
      xv = (yvv[b] - q[10] * xv) * q[9];
      // RHS assembly (rhsp.F90:164-169, 181-204, 351-418, 423-445)
      const double d1 = last ? 0.0 : (double)xd;
      const double u0 = sv[(b + 1) * TB + t];
      double R = (double)sc[b * TB + t];
      const double kzt = sgn * kz * ((!last && (COMP != 2 || r < ny)) ? (double)sk[b * TB + tk] : 0.0);
      if (COMP == 0) {
        if (!last) {
          R = (d1 + kzt) + R;
          if (j >= 2 && j <= ny) R = R - u0 * kv;
        }
      } else if (COMP == 1) {
        if (!last) {
          if (j >= 2 && j <= ny - 1) R = R - u0 * kv;
          R = R + kzt;
          R = R + d1;
        }
        if (j == 1 || j == ny) R = 0.0;
      } else {
        if (!last) {
          if (j >= 2 && j <= ny) R = R - u0 * kv;
          R = R + d1;
          if (j <= ny) R = R + kzt;
        }
      }
      if (COMP != 1) {  // wall and top rows of the u,w RHS (rhsp.F90:438-442)
        if (r == jee - 1) R = 0.0;
        if (r == 0) R = -1.0 / M4(ib, 2, 1) * (M4(ib, 2, 2) * R1 + M4(ib, 2, 3) * R2 + M4(ib, 2, 4) * R3);
        if (r == 3) R3 = R;
        if (r == 2) R2 = R;
        if (r == 1) R1 = R;
      }
      // RK3 combination and the new RHS history (rhsp.F90:448-475); rows
      // 1..jee-2 of the pressure box (no clamp needed there)
      double st;
      if (r == 0) {
        st = ub1;
      } else if (r == jee - 1) {
        st = ubt;
      } else if (COMP == 0) {
        st = last ? u0 : u0 - var1 * idxx * ((double)spp[(B::PR + b) * TB + t] - (double)spp[b * TB + t]);
      } else if (COMP == 1) {
        st = u0 - var1 * rq[4] * ((double)spp[(b + 1) * TB + t] - (double)spp[b * TB + t]);
      } else {
        const double pp = (double)spp[b * TB + tk];
        const double avz = var1 * kz;
        st = u0 - (odd ? avz * pp : -avz * pp);
      }
      const double res = st - (var3 * R + v2 * (double)xv + var4 * (double)sh[b * TB + t]);
      hp[(size_t)r * S] = (W)R;
      if (r < n) {
        double v = rq[1] * res + rq[2] * res1 + rq[3] * res2;
        if (r == 0) v = v - a1raw * ub1;
        if (r == n - 1) v = v - a3raw * ubt;
        yel = v + rq[0] * yel;
        yq[(size_t)r * ncol] = yel;
      }
      res2 = res1;
      res1 = res;
    }
  }
  if (active) {
    fs.ub[col] = ub1;
    fs.ub[(size_t)ncol + col] = ubt;
  }
}

// Pass A of the rhsp tail fed by TMA: the same ring as k_final_tb, ascending,
// with boxes of 128 columns x KA+2 rows of the product and the velocity
// (KA = 8 rows per stage); the checkpoints are still written every KF rows
// of k_final_tb's segments. The arithmetic is k_final_s1's pass A.
template <int COMP, typename W>
__global__ void __launch_bounds__(128) k_final_ta(DCoef c, DCoefT<W> cw, FinalStream<W> fs, int *err,
                                                  const __grid_constant__ FinalMaps maps) {
  constexpr int KF = FinalTune<W>::kf_tma, KA = 8, TB = 128, R = KA + 2;
  constexpr int PB = (R * TB * (int)sizeof(W) + 127) / 128 * 128;
  constexpr int STG = PB + R * TB * 8 + KA * 128;  // + the KA coefficient rows
  constexpr unsigned TX = (unsigned)(R * TB * sizeof(W) + R * TB * 8 + KA * 128);
  extern __shared__ __align__(128) unsigned char smraw[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smraw + 2 * STG);
  const FinalArgs<W> &a = fs.a;
  const int nx = c.nx, ny = c.ny, nz1 = c.nz1;
  const int ncol = (nx - 1) * nz1;
  const int t = threadIdx.x;
  const int i = blockIdx.y + 2, kr0 = blockIdx.x * TB, kr = kr0 + t;
  const bool active = kr < nz1;
  const int krc = active ? kr : 0;
  const int col = (i - 2) * nz1 + krc;
  const bool last = i == nx;
  const int jee = COMP == 1 ? ny : ny + 1;
  const int nst = (jee + KA - 1) / KA;
  auto issue = [&](int stg, int sa) {
    unsigned char *b = smraw + stg * STG;
    mbar_arrive_expect_tx(&bar[stg], TX);
    tma_load_3d(b, &maps.prod_a, kr0, sa * KA - 1, i - 1, &bar[stg]);
    tma_load_3d(b + PB, &maps.vel_a, kr0, sa * KA - 1, i - 1, &bar[stg]);
    tma_load_2d(b + PB + R * TB * 8, &maps.rc_a, 0, sa * KA, &bar[stg]);
  };
  if (t == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (t == 0) issue(0, 0);
  const size_t PU = (size_t)(ny + 1) * nz1, PV = (size_t)ny * nz1;
  const size_t pl = (size_t)(i - 1) * (COMP == 1 ? PV : PU), plv = (size_t)(i - 1) * PV;
  const size_t S = nz1;
  const W *prod = (COMP == 0 ? a.uv : (COMP == 1 ? a.vv : a.vw)) + plv + krc;
  const double *vel = (COMP == 0 ? a.u : (COMP == 1 ? a.v : a.w)) + pl + krc;
  const int which = COMP == 1 ? 1 : 0;
  // the sweeps run in W on the coefficient copy cw (FP32 on the mixed path);
  // the per-row coefficients come staged with the boxes (k_tail_rows' rows)
  auto Pg = [&](int r) { return (W)__ldg(prod + (size_t)min(max(r, 0), ny - 1) * S); };
  auto Vg = [&](int r) { return (W)__ldg(vel + (size_t)min(max(r, 0), jee - 1) * S); };
  const int chv = which == 0 ? 3 : 1, cha = chv + 1, ic = which == 0 ? 3 : 1;
  const W *db = cw.dcby, *vb = cw.cofvby;
  W bot = W(0), top = W(0);
  if (!last) {
    bot = M4(db, chv, 1) * Pg(0) + M4(db, chv, 2) * Pg(1) + M4(db, chv, 3) * Pg(2) + M4(db, chv, 4) * Pg(3);
    top = M4(db, cha, 1) * Pg(ny - 1) + M4(db, cha, 2) * Pg(ny - 2) + M4(db, cha, 3) * Pg(ny - 3) +
          M4(db, cha, 4) * Pg(ny - 4);
  }
  const W b0 = M4(vb, ic, 1) * Vg(0) + M4(vb, ic, 2) * Vg(1) + M4(vb, ic, 3) * Vg(2) + M4(vb, ic, 4) * Vg(3);
  const W bN = M4(vb, ic + 1, 1) * Vg(jee - 1) + M4(vb, ic + 1, 2) * Vg(jee - 2) +
               M4(vb, ic + 1, 3) * Vg(jee - 3) + M4(vb, ic + 1, 4) * Vg(jee - 4);
  auto rd = [&](int r, const W *q, W gm, W g0, W gp) {
    const W in = which == 0 ? q[1] * g0 + q[0] * gm : q[1] * gp + q[0] * g0;
    return r == 0 ? bot : (r == jee - 1 ? top : in);
  };
  auto rv = [&](int r, const W *q, W um, W u0, W up) {
    const W in = q[5] * up + q[6] * u0 + q[7] * um;
    return r == 0 ? b0 : (r == jee - 1 ? bN : in);
  };
  W *ck = reinterpret_cast<W *>(fs.ck) + col;  // checkpoints in W, read back by k_final_tb
  W yd = W(0), yv = W(0);
  for (int sa = 0; sa < nst; ++sa) {
    const int stg = sa & 1;
    const bool ok = mbar_wait_bounded(&bar[stg], (sa >> 1) & 1, 2000000000ull);
    if (__syncthreads_or(!ok)) {
      if (t == 0) atomicExch(err, OTBL_ERR_TIMEOUT);
      return;
    }
    if (t == 0 && sa + 1 < nst) issue(stg ^ 1, sa + 1);
    if (!active) continue;
    const W *sp = reinterpret_cast<const W *>(smraw + stg * STG) + t;
    const double *sv = reinterpret_cast<const double *>(smraw + stg * STG + PB) + t;
    const double *rcs = reinterpret_cast<const double *>(smraw + stg * STG + PB + R * TB * 8);
    const int s0 = sa * KA;
#pragma unroll
    for (int b = 0; b < KA; ++b) {
      const int r = s0 + b;
      const W *q = reinterpret_cast<const W *>(rcs + 16 * b + 5);
      if (r % KF == 0 && r < jee) {  // y of row r-1 at the start of segment r/KF
        ck[(size_t)(2 * (r / KF)) * ncol] = yd;
        ck[(size_t)(2 * (r / KF) + 1) * ncol] = yv;
      }
      if (r < jee) {
        if (!last) yd = rd(r, q, sp[b * TB], sp[(b + 1) * TB], sp[(b + 2) * TB]) + (r > 0 ? q[2] : W(0)) * yd;
        yv = rv(r, q, (W)sv[b * TB], (W)sv[(b + 1) * TB], (W)sv[(b + 2) * TB]) + (r > 0 ? q[8] : W(0)) * yv;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// pois.f90:106-117 + soltriy: tridiagonal in y per (x-mode, kz). The LU of
// each (i, k) system depends only on the grid, so its pivots are computed
// once (k_pois_lu) and every substep runs the pre-factored solve.
// ---------------------------------------------------------------------------
// dinv[(i-1)][j-1][k] = 1/pivot_j of the system (i, k), planes i = 2..nx
__global__ void k_pois_lu(DCoef c, double *dinv) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k > c.nz2) return;
  const int i = blockIdx.y + 2, ny = c.ny, ny1 = ny - 1, nm = c.nz2 + 1;
  const double *ayp = c.ayp;
  const bool sing = (i == 2 && k == 0);
  auto a2 = [&](int j) {
    if (sing && j == ny1) return 2.0 * A3(ayp, 2, ny1);
    return A3(ayp, 2, j) - c.kaz2[k] - c.kmod[i - 2];
  };
  double *dv = dinv + (size_t)(i - 1) * ny * nm + k;
  double a2p = a2(1);
  for (int j = 2; j <= ny1; ++j) {
    const double d = 1.0 / a2p;
    dv[(size_t)(j - 2) * nm] = d;
    const double l = -A3(ayp, 1, j) * d;
    a2p = a2(j) + l * A3(ayp, 3, j - 1);
  }
  dv[(size_t)(ny1 - 1) * nm] = 1.0 / a2p;
}

// The solve in place on phi rows 0..ny-2 of planes 2..nx, one thread per
// column: y_r = rhs_r + l_r y_{r-1}, l_r = -ayp(1,r+1) dinv(r-1); then
// x_r = (y_r - ayp(3,r+1) x_{r+1}) dinv(r). The singular (i = 2, k = 0)
// system has its last row zeroed first (pois.f90:111-114). The launch takes
// the columns kr0 <= kr < kr0 + nkr of every plane, in T (FP64, or FP32 for
// the higher spanwise modes of the mixed path, with FP32 coefficients and
// pivots); phi and the checkpoints hold T.
template <typename T>
__global__ void __launch_bounds__(128) k_pois_solve(DCoefT<T> c, T *phi, const T *__restrict__ dinv, T *ckbuf,
                                                    int kr0, int nkr) {
  const int ny = c.ny, ny1 = ny - 1, nz1 = c.nz1, nm = c.nz2 + 1;
  const int ncol = (c.nx - 1) * nkr;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  const int i = col / nkr + 2, kr = kr0 + (col - (i - 2) * nkr), k = kr >> 1;
  const size_t S = nz1;
  T *x = phi + (size_t)(i - 1) * ny * nz1 + kr;
  const T *dv = dinv + (size_t)(i - 1) * ny * nm + k;
  T *ck = ckbuf + col;
  const T *ayp = c.ayp;
  const bool sing = i == 2 && k == 0;
  auto X = [&](int r) { return (sing && r == ny1 - 1) ? (T)0 : x[(size_t)min(r, ny1 - 1) * S]; };
  auto D = [&](int r) { return __ldg(dv + (size_t)min(max(r, 0), ny1 - 1) * nm); };
  const int nseg = (ny1 + KY - 1) / KY;
  T y = 0;
  for (int sg = 0; sg < nseg; ++sg) {
    const int s0 = sg * KY;
    ck[(size_t)sg * ncol] = y;
    T bv[KY], dp[KY + 1];
#pragma unroll
    for (int b = 0; b < KY; ++b) bv[b] = X(s0 + b);
#pragma unroll
    for (int b = 0; b <= KY; ++b) dp[b] = D(s0 + b - 1);
#pragma unroll
    for (int b = 0; b < KY; ++b) {
      const int r = s0 + b;
      if (r < ny1) y = bv[b] + (r > 0 ? -A3(ayp, 1, r + 1) * dp[b] : (T)0) * y;
    }
  }
  T xn = 0;
  for (int sg = nseg - 1; sg >= 0; --sg) {
    const int s0 = sg * KY;
    T bv[KY], dp[KY + 1], yv[KY];
#pragma unroll
    for (int b = 0; b < KY; ++b) bv[b] = X(s0 + b);
#pragma unroll
    for (int b = 0; b <= KY; ++b) dp[b] = D(s0 + b - 1);
    T yy = ck[(size_t)sg * ncol];
#pragma unroll
    for (int b = 0; b < KY; ++b) {
      const int r = s0 + b;
      if (r < ny1) yy = bv[b] + (r > 0 ? -A3(ayp, 1, r + 1) * dp[b] : (T)0) * yy;
      yv[b] = yy;
    }
#pragma unroll
    for (int b = KY - 1; b >= 0; --b) {
      const int r = s0 + b;
      if (r < ny1) {
        xn = (yv[b] - (r < ny1 - 1 ? A3(ayp, 3, r + 1) : (T)0) * xn) * dp[b + 1];
        x[(size_t)r * S] = xn;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// launch wrappers
// ---------------------------------------------------------------------------
// Checkpoints of interpyy at the tail of each line scratch, so that
// interpyy can run beside interpxx (whose checkpoints start at the head);
// nullptr when the two would overlap.
double *interpy_ck_tail(otbl_ctx *c, double *s) {
  const int nx = c->cfg.nx, ny = c->cfg.ny, nz = c->cfg.nz, nz1 = c->dc.nz1;
  const size_t lu = otbl_field_len(nx, ny, nz, 1);  // doubles in s2, s3 (s1 may be larger)
  const size_t ncol = (size_t)nx * nz1;
  // the shorter of the register-streamed and the TMA-fed segments
  const int ky = KY < YTune<double>::kt ? KY : YTune<double>::kt;
  const size_t y_need = (size_t)((ny + ky - 1) / ky) * ncol;  // doubles (floats need less)
  // interpxx: at most one checkpoint per 4 planes per line (4 is its shortest segment)
  const size_t x_need = (size_t)((nx + 3) / 4) * (size_t)(ny + 1) * nz1;
  if (x_need + y_need + 64 > lu) return nullptr;
  return s + ((lu - y_need) & ~(size_t)31);
}

cudaError_t launch_interpy(otbl_ctx *c) {
  InterpyArgs a;
  const double *ins[3] = {c->f[OTBL_F_U], c->f[OTBL_F_W], c->f[OTBL_F_V]};
  void *outs[3] = {c->w.uy, c->w.wy, c->w.vy};
  double *tail[3] = {interpy_ck_tail(c, c->w.s1), interpy_ck_tail(c, c->w.s2), interpy_ck_tail(c, c->w.s3)};
  double *cks[3] = {tail[0] ? tail[0] : c->w.s1, tail[1] ? tail[1] : c->w.s2, tail[2] ? tail[2] : c->w.s3};
  const int which[3] = {0, 0, 1};
  for (int f = 0; f < 3; ++f) {
    a.in[f] = ins[f];
    a.out[f] = outs[f];
    a.ck[f] = cks[f];
    a.which[f] = which[f];
  }
  const int ncol = c->cfg.nx * c->dc.nz1;
  prof_begin(c, PK_INTERPY);
  if (ydense_ready(c)) {
    const cudaError_t e = launch_interpy_dense(c);
    prof_end(c);
    return e;
  }
  const int bs = c->tune_bs[2];
  if (c->ymaps_ok) {
    const dim3 gt((c->dc.nz1 + 127) / 128, c->cfg.nx, 3);
    if (c->mixed) {
      const int sm = 2 * ((YTune<float>::kt + 2) * 128 * 8 + YTune<float>::kt * 8 * 4) + 128;
      cudaFuncSetAttribute(k_interpy_t<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
      k_interpy_t<float><<<gt, 128, sm, c->stream>>>(c->dcf, a, &c->st->err, c->ymi);
    } else {
      const int sm = 2 * ((YTune<double>::kt + 2) * 128 * 8 + YTune<double>::kt * 8 * 8) + 128;
      cudaFuncSetAttribute(k_interpy_t<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
      k_interpy_t<double><<<gt, 128, sm, c->stream>>>(c->dc, a, &c->st->err, c->ymi);
    }
  } else if (c->mixed)
    k_interpy<float><<<dim3((ncol + bs - 1) / bs, 3), bs, 0, c->stream>>>(c->dcf, a);
  else
    k_interpy<double><<<dim3((ncol + bs - 1) / bs, 3), bs, 0, c->stream>>>(c->dc, a);
  prof_end(c);
  c->launches += 1;
  return cudaGetLastError();
}

// One row of 8 T per y row r of each table (which 0: u-type input, u and w;
// 1: v-type input, v): interpyy's right-hand-side weights econ[2r],
// econ[2r+1] and LU coefficients iny[3r..3r+2]; the rest 0. k_interpy_t's
// ring stages a segment's rows with its field box.
template <typename T>
__global__ void __launch_bounds__(128) k_y_rows(DCoefT<T> c, T *tab) {
  const int ny = c.ny;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 2 * ny) return;
  const int which = e / ny, r = e - which * ny;
  const T *iny = which == 0 ? c.inyu : c.inyv, *econ = which == 0 ? c.cofiuy : c.cofivy;
  T *q = tab + (size_t)e * 8;
  q[0] = econ[2 * r];
  q[1] = econ[2 * r + 1];
  for (int k = 0; k < 3; ++k) q[2 + k] = iny[3 * r + k];
  for (int k = 5; k < 8; ++k) q[k] = T(0);
}

cudaError_t launch_y_rows(otbl_ctx *c) {
  const int n = 2 * c->cfg.ny;
  if (c->mixed)
    k_y_rows<float><<<(n + 127) / 128, 128, 0, c->stream>>>(c->dcf, static_cast<float *>(c->w.yrowc));
  else
    k_y_rows<double><<<(n + 127) / 128, 128, 0, c->stream>>>(c->dc, static_cast<double *>(c->w.yrowc));
  c->launches += 1;
  return cudaGetLastError();
}

// ---- TMA descriptors (host) ----
// cuTensorMapEncodeTiled from the driver, looked up once (thread-safe
// initialisation of a function-local static); nullptr if unavailable
void *tensor_map_encoder() {
  static void *const fn = []() -> void * {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    cudaGetLastError();
    return p;
  }();
  return fn;
}

// a field [planes][rows][nz1] of element size esz, boxes of 128 x brows x bplanes
static bool encode_field(CUtensorMap *m, const void *base, size_t esz, int planes, int rows, int nz1, int brows,
                         int bplanes) {
  auto fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
  if (!fn || (nz1 * esz) % 16 != 0 || ((uintptr_t)base) % 16 != 0) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)nz1, (cuuint64_t)rows, (cuuint64_t)planes};
  const cuuint64_t strides[2] = {(cuuint64_t)nz1 * esz, (cuuint64_t)rows * nz1 * esz};
  const cuuint32_t box[3] = {128, (cuuint32_t)brows, (cuuint32_t)bplanes};
  const cuuint32_t es[3] = {1, 1, 1};
  const CUtensorMapDataType dt = esz == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  return fn(m, dt, 3, const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

static bool encode_rows(CUtensorMap *m, const double *base, int rows, int brows);

// 2D map of a coefficient table [rows][width elements of esz bytes], boxes
// of brows full rows
static bool encode_table(CUtensorMap *m, const void *base, size_t esz, int width, int rows, int brows) {
  auto fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
  if (!fn || ((uintptr_t)base) % 16 != 0 || (width * esz) % 16 != 0) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)width, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {width * esz};
  const cuuint32_t box[2] = {(cuuint32_t)width, (cuuint32_t)brows};
  const cuuint32_t es[2] = {1, 1};
  const CUtensorMapDataType dt = esz == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  return fn(m, dt, 2, const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename W>
static bool build_maps_t(otbl_ctx *c) {
  constexpr int KF = FinalTune<W>::kf_tma;
  const int nx = c->cfg.nx, ny = c->cfg.ny, nz1 = c->dc.nz1;
  const size_t ew = sizeof(W);
  bool ok = nz1 >= 2;
  for (int comp = 0; comp < 3 && ok; ++comp) {
    FinalMaps &m = c->fmaps[comp];
    const int jee = comp == 1 ? ny : ny + 1;
    const void *prod = comp == 0 ? c->w.uv : (comp == 1 ? c->w.vv : c->w.vw);
    const void *kp = comp == 0 ? c->w.uw : (comp == 1 ? c->w.vw : c->w.ww);
    const int kprows = comp == 0 ? ny + 1 : ny;
    const double *vel = c->f[comp == 0 ? OTBL_F_U : (comp == 1 ? OTBL_F_V : OTBL_F_W)];
    const void *cx = comp == 0 ? c->w.cu : (comp == 1 ? c->w.cv : c->w.cw);
    const void *hp = c->f[comp == 0 ? OTBL_F_RHSUPA : (comp == 1 ? OTBL_F_RHSVPA : OTBL_F_RHSWPA)];
    ok = ok && encode_field(&m.prod, prod, ew, nx, ny, nz1, KF + 2, 1);
    ok = ok && encode_field(&m.prod_a, prod, ew, nx, ny, nz1, 8 + 2, 1);
    ok = ok && encode_field(&m.vel_a, vel, 8, nx, jee, nz1, 8 + 2, 1);
    ok = ok && encode_field(&m.kp, kp, ew, nx, kprows, nz1, KF, 1);
    ok = ok && encode_field(&m.vel, vel, 8, nx, jee, nz1, KF + 2, 1);
    ok = ok && encode_field(&m.cx, cx, ew, nx, jee, nz1, KF, 1);
    ok = ok && encode_field(&m.hp, hp, ew, nx, jee, nz1, KF, 1);
    ok = ok && encode_field(&m.p, c->f[OTBL_F_P], ew, nx, ny, nz1, comp == 1 ? KF + 1 : KF, comp == 0 ? 2 : 1);
    ok = ok && encode_rows(&m.rc, c->w.rowc + (comp == 1 ? (size_t)16 * (ny + 2) : 0), ny + 2, KF);
    ok = ok && encode_rows(&m.rc_a, c->w.rowc + (comp == 1 ? (size_t)16 * (ny + 2) : 0), ny + 2, 8);
  }
  return ok;
}

bool build_y_maps(otbl_ctx *c) {
  const int K = c->mixed ? YTune<float>::kt : YTune<double>::kt;
  const int nx = c->cfg.nx, ny = c->cfg.ny, nz1 = c->dc.nz1;
  const double *in[3] = {c->f[OTBL_F_U], c->f[OTBL_F_W], c->f[OTBL_F_V]};
  const int rows[3] = {ny + 1, ny + 1, ny};
  bool ok = true;
  const size_t ew = c->mixed ? sizeof(float) : sizeof(double);
  const int which[3] = {0, 0, 1};
  for (int f = 0; f < 3 && ok; ++f) {
    ok = encode_field(&c->ymi.g[f], in[f], 8, nx, rows[f], nz1, K + 2, 1);
    const char *tab = static_cast<const char *>(c->w.yrowc) + (size_t)which[f] * ny * 8 * ew;
    ok = ok && encode_table(&c->ymi.r[f], tab, ew, 8, ny, K);
  }
  c->ymaps_ok = ok;
  return ok;
}

// One 128-byte row per y row r and tail kind (table 0: the u and w tails,
// u-type coefficients; table 1: the v tail): the FP64 values fac[3(r+2)+2]
// (the implzy factor of the descending elimination), vyi[3(r+1)+0..2] and
// idyy[r], then in W ecd[2r+0..1], dcy[3r+0..2], ecv[3r+0..2],
// viy[3r+0..2] (differzy's and vistyy's right-hand-side and LU
// coefficients). k_final_tb's ring stages a segment's rows with its field
// boxes, so its sweeps read them from shared memory as broadcasts. Entries
// that a row does not use are 0.
template <typename W>
__global__ void __launch_bounds__(128) k_tail_rows(DCoef c, DCoefT<W> cw, const double *fac_u, const double *fac_v,
                                                   double *rowc) {
  const int ny = c.ny, R = ny + 2;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 2 * R) return;
  const int which = e / R, r = e - which * R;
  const int jee = which == 1 ? ny : ny + 1, n = jee - 2;
  double *row = rowc + (size_t)e * 16;
  const double *fac = which == 1 ? fac_v : fac_u;
  const double *vyi = which == 0 ? c.vyui : c.vyvi;
  row[0] = r < n ? fac[3 * (r + 2) + 2] : 0.0;
  for (int q = 0; q < 3; ++q) row[1 + q] = r < n ? vyi[3 * (r + 1) + q] : 0.0;
  row[4] = (which == 1 && r < ny) ? c.idyy[r] : 0.0;
  W *q = reinterpret_cast<W *>(row + 5);
  constexpr int NW = (int)((128 - 5 * sizeof(double)) / sizeof(W));
  for (int k = 0; k < NW; ++k) q[k] = W(0);
  if (r < jee) {
    const W *dcy = which == 0 ? cw.dcyu : cw.dcyv, *ecd = which == 0 ? cw.cofcyu : cw.cofcyv;
    const W *viy = which == 0 ? cw.viyu : cw.viyv, *ecv = which == 0 ? cw.cofvyu : cw.cofvyv;
    q[0] = ecd[2 * r];
    q[1] = ecd[2 * r + 1];
    for (int k = 0; k < 3; ++k) {
      q[2 + k] = dcy[3 * r + k];
      q[5 + k] = ecv[3 * r + k];
      q[8 + k] = viy[3 * r + k];
    }
  }
}

cudaError_t launch_tail_rows(otbl_ctx *c) {
  if (!c->fmaps_ok) return cudaSuccess;
  const int n = 2 * (c->cfg.ny + 2);
  if (c->mixed)
    k_tail_rows<float><<<(n + 127) / 128, 128, 0, c->stream>>>(c->dc, c->dcf, c->w.fac_u, c->w.fac_v, c->w.rowc);
  else
    k_tail_rows<double><<<(n + 127) / 128, 128, 0, c->stream>>>(c->dc, c->dc, c->w.fac_u, c->w.fac_v, c->w.rowc);
  c->launches += 1;
  return cudaGetLastError();
}

// 2D map of one table of Work::rowc: [ny+2 rows][16 doubles], boxes of KF rows
static bool encode_rows(CUtensorMap *m, const double *base, int rows, int brows) {
  auto fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
  if (!fn || ((uintptr_t)base) % 16 != 0) return false;
  const cuuint64_t dims[2] = {16, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {16 * sizeof(double)};
  const cuuint32_t box[2] = {16, (cuuint32_t)brows};
  const cuuint32_t es[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double *>(base), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool build_final_maps(otbl_ctx *c) {
  c->fmaps_ok = c->mixed ? build_maps_t<float>(c) : build_maps_t<double>(c);
  return c->fmaps_ok;
}

template <typename W>
static int final_t(otbl_ctx *c, unsigned comps, cudaEvent_t before_vel, bool second_scratch) {
  FinalStream<W> fs;
  FinalArgs<W> &a = fs.a;
  a.u = c->f[OTBL_F_U];
  a.v = c->f[OTBL_F_V];
  a.w = c->f[OTBL_F_W];
  a.p = reinterpret_cast<const W *>(c->f[OTBL_F_P]);
  a.rhsupa = reinterpret_cast<W *>(c->f[OTBL_F_RHSUPA]);
  a.rhsvpa = reinterpret_cast<W *>(c->f[OTBL_F_RHSVPA]);
  a.rhswpa = reinterpret_cast<W *>(c->f[OTBL_F_RHSWPA]);
  a.cu = static_cast<const W *>(c->w.cu);
  a.cv = static_cast<const W *>(c->w.cv);
  a.cw = static_cast<const W *>(c->w.cw);
  a.uv = static_cast<const W *>(c->w.uv);
  a.uw = static_cast<const W *>(c->w.uw);
  a.vw = static_cast<const W *>(c->w.vw);
  a.vv = static_cast<const W *>(c->w.vv);
  a.ww = static_cast<const W *>(c->w.ww);
  a.fac_u = c->w.fac_u;
  a.fac_v = c->w.fac_v;
  a.st = c->st;
  const int ncol = (c->cfg.nx - 1) * c->dc.nz1;
  fs.ck = second_scratch ? c->w.t1 : c->w.s1;
  fs.yq = second_scratch ? c->w.t2 : c->w.s2;
  fs.ub = second_scratch ? c->w.t3 : c->w.s3;
  const dim3 g((ncol + 127) / 128);
  double *U = c->f[OTBL_F_U], *V = c->f[OTBL_F_V], *Wv = c->f[OTBL_F_W];
  const bool tma = c->fmaps_ok;
  DCoefT<W> cw;  // the sweeps' coefficients in W
  if constexpr (std::is_same<W, float>::value)
    cw = c->dcf;
  else
    cw = c->dc;
  const dim3 gt((c->dc.nz1 + 127) / 128, c->cfg.nx - 1);
  auto comp = [&](auto C) {
    constexpr int K = decltype(C)::value;
    const int smem_t = FinalBox<W, K>::smem;
    if (tma) {
      // pass A (register-streamed or TMA-fed), then the TMA-fed pass B
      if constexpr (FinalTune<W>::tma_a) {
        constexpr int sma = 2 * ((10 * 128 * (int)sizeof(W) + 127) / 128 * 128 + 10 * 128 * 8 + 8 * 128) + 128;
        cudaFuncSetAttribute(k_final_ta<K, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, sma);
        k_final_ta<K, W><<<gt, 128, sma, c->stream>>>(c->dc, cw, fs, &c->st->err, c->fmaps[K]);
      } else {
        k_final_s1<K, W, 1, FinalTune<W>::kf_tma><<<g, 128, 0, c->stream>>>(c->dc, fs);
      }
      cudaFuncSetAttribute(k_final_tb<K, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_t);
      k_final_tb<K, W><<<gt, 128, smem_t, c->stream>>>(c->dc, cw, fs, &c->st->err, c->fmaps[K]);
    } else if constexpr (FinalTune<W>::split) {
      k_final_s1<K, W, 1><<<g, 128, 0, c->stream>>>(c->dc, fs);
      k_final_s1<K, W, 2><<<g, 128, 0, c->stream>>>(c->dc, fs);
    } else {
      k_final_s1<K, W, 3><<<g, 128, 0, c->stream>>>(c->dc, fs);
    }
    if (before_vel) {  // the first velocity write waits for this event
      cudaStreamWaitEvent(c->stream, before_vel, 0);
      before_vel = nullptr;
    }
    k_final_s2<K><<<g, 128, 0, c->stream>>>(c->dc, U, V, Wv, c->w.fac_u, c->w.fac_v, fs.yq, fs.ub);
  };
  int n = 0;
  if (comps & 1) comp(std::integral_constant<int, 0>{}), ++n;
  if (comps & 2) comp(std::integral_constant<int, 1>{}), ++n;
  if (comps & 4) comp(std::integral_constant<int, 2>{}), ++n;
  return n * ((tma || FinalTune<W>::split) ? 3 : 2);
}

cudaError_t launch_final(otbl_ctx *c, unsigned comps, cudaEvent_t before_vel, bool second_scratch) {
  prof_begin(c, PK_FINAL);
  const int nl = c->mixed ? final_t<float>(c, comps, before_vel, second_scratch)
                          : final_t<double>(c, comps, before_vel, second_scratch);
  prof_end(c);
  c->launches += nl;
  return cudaGetLastError();
}

cudaError_t launch_pois_lu(otbl_ctx *c) {
  dim3 g((c->dc.nz2 + 1 + 127) / 128, c->cfg.nx - 1);
  k_pois_lu<<<g, 128, 0, c->stream>>>(c->dc, c->w.pois_dinv);
  c->launches += 1;
  if (c->mixed) {
    const size_t n = (size_t)c->cfg.nx * c->cfg.ny * (c->dc.nz1 / 2);
    const cudaError_t e = launch_round_f32(c, c->w.pois_dinv, c->w.pois_dinvf, n);
    if (e != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

// columns kr0 <= kr < kr0 + nkr of every plane; phi holds T
template <typename T>
static void pois_solve_t(otbl_ctx *c, const DCoefT<T> &dc, T *phi, const T *dinv, int kr0, int nkr) {
  const int ncol = (c->cfg.nx - 1) * nkr;
  k_pois_solve<T><<<(ncol + 127) / 128, 128, 0, c->stream>>>(dc, phi, dinv, reinterpret_cast<T *>(c->w.s1), kr0,
                                                            nkr);
  c->launches += 1;
}

cudaError_t launch_pois_solve(otbl_ctx *c, double *phi64, float *phi32, int kr_split) {
  const int nz1 = c->dc.nz1;
  prof_begin(c, PK_POIS_SOLVE);
  if (kr_split > 0) pois_solve_t<double>(c, c->dc, phi64, c->w.pois_dinv, 0, kr_split);
  if (kr_split < nz1) pois_solve_t<float>(c, c->dcf, phi32, c->w.pois_dinvf, kr_split, nz1 - kr_split);
  prof_end(c);
  return cudaGetLastError();
}

}  // namespace otbl
