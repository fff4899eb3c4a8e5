// Wall-normal (y) line operators and the tail of rhsp on shared-memory tiles.
//
// A CTA owns one streamwise plane i and YT consecutive real indices kr
// (16 spanwise modes, re/im interleaved), all rows j. Eight lanes of a warp
// share one column (chunked Thomas sweeps, lines.cuh); a warp holds four
// columns. Tiles are filled with cp.async (every copy of a thread in flight
// at once); global reads that feed element-wise steps are issued four rows
// at a time.
#include "devcommon.cuh"
#include <type_traits>

#include "lines.cuh"
#include "otbl_internal.cuh"

namespace otbl {

#ifndef OTBL_YT
#define OTBL_YT 32
#endif
constexpr int YT = OTBL_YT;  // columns per CTA (a multiple of 4)
constexpr int YNCH = 8;      // lanes per column
constexpr int YTHREADS = YT * YNCH;
constexpr int YB = 4;       // rows per batch of global reads

// a chunk-interleaved coefficient (lines.cuh CCo) addressed by the chunk
// offset t of lane h: entry t*YNCH + h
struct RCo8 {
  const double *p;
  __device__ __forceinline__ RCo8(const double *a, int h) : p(a + h) {}
  __device__ __forceinline__ double operator()(int t) const { return __ldg(p + t * YNCH); }
};

struct YIdx {
  int col, h, kr, k, odd, pof;
  bool valid;
};

__device__ __forceinline__ YIdx yidx(int nz1) {
  YIdx q;
  const int lane = threadIdx.x & 31;
  q.col = (threadIdx.x >> 5) * (32 / YNCH) + lane / YNCH;
  q.h = lane % YNCH;
  q.kr = blockIdx.x * YT + q.col;
  q.valid = q.kr < nz1;
  q.k = q.valid ? q.kr >> 1 : 0;
  q.odd = q.kr & 1;
  q.pof = q.odd ? -1 : 1;
  return q;
}

// rows [0, rows) of the YT columns starting at kr0 of a plane whose rows are
// nz1 apart -> tile (column-major, pitch Lp); asynchronous
__device__ __forceinline__ void ytile_load(double *t, const double *__restrict__ g, int rows, int nz1, int kr0,
                                           int Lp) {
  for (int e = threadIdx.x; e < rows * YT; e += YTHREADS) {
    const int j0 = e / YT, col = e - j0 * YT, kr = kr0 + col;
    const bool ok = kr < nz1;
    cp_async8(t + col * Lp + j0, ok ? g + (size_t)j0 * nz1 + kr : g, ok);
  }
}

// ---------------------------------------------------------------------------
// In-place explicit stencils (each followed by a tile solve). Every lane
// first reads the halo rows and boundary stencils it needs, then the warp
// synchronises, then rows are rewritten in an order that never reads an
// overwritten row.
// ---------------------------------------------------------------------------

// differzy (lip.f90:152-232): which 0 u-type (out rows 0..ny, reads 0..ny-1),
// which 1 v-type (rows 0..ny-1). Then the solve with dcyu/dcyv.
__device__ __forceinline__ void y_differzy(const DCoef &c, const YSet &ys, double *x, int h, int which) {
  const int ny = c.ny, jee = which == 0 ? ny + 1 : ny;
  const int CL = ys.CL;
  const CCo<YNCH> E1(ys.k[YD_E1], h, CL), E2(ys.k[YD_E2], h, CL);
  const double *db = c.dcby;
  const int chv = which == 0 ? 3 : 1, cha = chv + 1;
  int s, e;
  chunk_range(jee, h, ys.CL, s, e);
  double bot = 0.0, top = 0.0;
  if (s == 0 && e > s)
    bot = M4(db, chv, 1) * x[0] + M4(db, chv, 2) * x[1] + M4(db, chv, 3) * x[2] + M4(db, chv, 4) * x[3];
  if (e == jee && e > s)
    top = M4(db, cha, 1) * x[ny - 1] + M4(db, cha, 2) * x[ny - 2] + M4(db, cha, 3) * x[ny - 3] +
          M4(db, cha, 4) * x[ny - 4];
  if (which == 0) {  // result(j) = e2(j) g(j) + e1(j) g(j-1), descending
    const double gprev = s > 0 ? x[s - 1] : 0.0;
    __syncwarp();
    for (int r1 = e - 1; r1 >= s; r1 -= LB) {
      double gv[LB + 1], e1[LB], e2[LB];
#pragma unroll
      for (int b = 0; b <= LB; ++b) gv[b] = r1 - b >= s ? x[r1 - b] : gprev;
#pragma unroll
      for (int b = 0; b < LB; ++b) {
        const bool ok = r1 - b >= s;
        e1[b] = ok ? E1(r1 - b) : 0.0;
        e2[b] = ok ? E2(r1 - b) : 0.0;
      }
#pragma unroll
      for (int b = 0; b < LB; ++b) {
        const int r = r1 - b;
        if (r < s) break;
        x[r] = r == 0 ? bot : (r == jee - 1 ? top : e2[b] * gv[b] + e1[b] * gv[b + 1]);
      }
    }
  } else {  // result(j) = e2(j) g(j+1) + e1(j) g(j), ascending
    const double gnext = e < jee ? x[e] : 0.0;
    __syncwarp();
    for (int r0 = s; r0 < e; r0 += LB) {
      double gv[LB + 1], e1[LB], e2[LB];
#pragma unroll
      for (int b = 0; b <= LB; ++b) gv[b] = r0 + b < e ? x[r0 + b] : gnext;
#pragma unroll
      for (int b = 0; b < LB; ++b) {
        const bool ok = r0 + b < e;
        e1[b] = ok ? E1(r0 + b) : 0.0;
        e2[b] = ok ? E2(r0 + b) : 0.0;
      }
#pragma unroll
      for (int b = 0; b < LB; ++b) {
        const int r = r0 + b;
        if (r >= e) break;
        x[r] = r == 0 ? bot : (r == jee - 1 ? top : e2[b] * gv[b + 1] + e1[b] * gv[b]);
      }
    }
  }
  __syncwarp();
  solve_cco<YNCH>(x, jee, h, ys.CL, CCo<YNCH>(ys.k[YD_L], h, CL), CCo<YNCH>(ys.k[YD_D], h, CL),
                        CCo<YNCH>(ys.k[YD_U], h, CL));
}

// vistyy (lip.f90:447-513): which 0 u,w (jee = ny+1, ic = 3), which 1 v.
__device__ __forceinline__ void y_vistyy(const DCoef &c, const YSet &ys, double *x, int h, int which) {
  const int ny = c.ny, jee = which == 0 ? ny + 1 : ny, ic = which == 0 ? 3 : 1;
  const int CL = ys.CL;
  const CCo<YNCH> F1(ys.k[YV_F1], h, CL), F2(ys.k[YV_F2], h, CL), F3(ys.k[YV_F3], h, CL);
  const double *vb = c.cofvby;
  int s, e;
  chunk_range(jee, h, ys.CL, s, e);
  double uprev = s > 0 ? x[s - 1] : 0.0;
  const double unext = e < jee ? x[e] : 0.0;
  double b0 = 0.0, bN = 0.0;
  if (s == 0 && e > s) b0 = M4(vb, ic, 1) * x[0] + M4(vb, ic, 2) * x[1] + M4(vb, ic, 3) * x[2] + M4(vb, ic, 4) * x[3];
  if (e == jee && e > s)
    bN = M4(vb, ic + 1, 1) * x[jee - 1] + M4(vb, ic + 1, 2) * x[jee - 2] + M4(vb, ic + 1, 3) * x[jee - 3] +
         M4(vb, ic + 1, 4) * x[jee - 4];
  __syncwarp();
  for (int r0 = s; r0 < e; r0 += LB) {  // ascending; uv[0] = original row r0-1
    double uv[LB + 2], f1[LB], f2[LB], f3[LB];
    uv[0] = uprev;
#pragma unroll
    for (int b = 0; b <= LB; ++b) uv[b + 1] = r0 + b < e ? x[r0 + b] : unext;
#pragma unroll
    for (int b = 0; b < LB; ++b) {
      const bool ok = r0 + b < e;
      f1[b] = ok ? F1(r0 + b) : 0.0;
      f2[b] = ok ? F2(r0 + b) : 0.0;
      f3[b] = ok ? F3(r0 + b) : 0.0;
    }
#pragma unroll
    for (int b = 0; b < LB; ++b) {
      const int r = r0 + b;
      if (r >= e) break;
      x[r] = r == 0 ? b0 : (r == jee - 1 ? bN : f1[b] * uv[b + 2] + f2[b] * uv[b + 1] + f3[b] * uv[b]);
    }
    uprev = uv[LB];
  }
  __syncwarp();
  solve_cco<YNCH>(x, jee, h, ys.CL, CCo<YNCH>(ys.k[YV_L], h, CL), CCo<YNCH>(ys.k[YV_D], h, CL),
                        CCo<YNCH>(ys.k[YV_U], h, CL));
}

// implzy (lip.f90:528-597): right-hand side A*res for rows 2..jee-1 from the
// column `res` (rows 0..jee-1) into `out` rows 0..jee-3, boundary values
// ub1 / ubj moved to the right-hand side, then the pre-factored solve of
// (A + var1*B) (factors from k_dt, interleaved YM_L/YM_D/YM_U; fac holds the
// boundary couplings a1raw, a3raw).
__device__ __forceinline__ void y_implzy(const DCoef &c, const YSet &ys, const double *res, double *out, int h,
                                         int which, double ub1, double ubj, const double *__restrict__ fac) {
  const int ny = c.ny, jee = which == 0 ? ny + 1 : ny, n = jee - 2;
  const int CL = ys.CL;
  const CCo<YNCH> F1(ys.k[YM_F1], h, CL), F2(ys.k[YM_F2], h, CL), F3(ys.k[YM_F3], h, CL);
  const double a1raw = fac[3 * (jee + 1)], a3raw = fac[3 * (jee + 1) + 1];
  int s, e;
  chunk_range(n, h, ys.CL, s, e);
  for (int q0 = s; q0 < e; q0 += LB) {
    double rv[LB + 2], f1[LB], f2[LB], f3[LB];
#pragma unroll
    for (int b = 0; b < LB + 2; ++b) rv[b] = q0 + b < e + 2 ? res[q0 + b] : 0.0;
#pragma unroll
    for (int b = 0; b < LB; ++b) {
      const bool ok = q0 + b < e;
      f1[b] = ok ? F1(q0 + b) : 0.0;
      f2[b] = ok ? F2(q0 + b) : 0.0;
      f3[b] = ok ? F3(q0 + b) : 0.0;
    }
#pragma unroll
    for (int b = 0; b < LB; ++b) {
      const int q = q0 + b;
      if (q >= e) break;
      const int j = q + 2;
      double t = f1[b] * rv[b] + f2[b] * rv[b + 1] + f3[b] * rv[b + 2];
      if (j == 2) t = t - a1raw * ub1;
      if (j == jee - 1) t = t - a3raw * ubj;
      out[q] = t;
    }
  }
  __syncwarp();
  solve_cco<YNCH>(out, n, h, ys.CL, CCo<YNCH>(ys.k[YM_L], h, CL), CCo<YNCH>(ys.k[YM_D], h, CL),
                        CCo<YNCH>(ys.k[YM_U], h, CL));
}

// interpyy (lip.f90:359-440) in Fourier space: which 0 u,w (in rows ny+1),
// which 1 v (in rows ny); out rows 1..ny.
__global__ void __launch_bounds__(YTHREADS) k_interpy(DCoef c, YSet ys, const double *__restrict__ in,
                                                      double *__restrict__ out, int which, int Lp) {
  extern __shared__ double sm[];
  const int ny = c.ny, nz1 = c.nz1, jin = which == 0 ? ny + 1 : ny;
  const int i = blockIdx.y + 1, kr0 = blockIdx.x * YT;
  ytile_load(sm, in + (size_t)(i - 1) * jin * nz1, jin, nz1, kr0, Lp);
  cp_async_wait_all();
  __syncthreads();
  const YIdx q = yidx(nz1);
  double *x = sm + q.col * Lp;
  const int CL = ys.CL;
  const CCo<YNCH> E1(ys.k[YI_E1], q.h, CL), E2(ys.k[YI_E2], q.h, CL);
  const double *ib = c.inby;
  int s, e;
  chunk_range(ny, q.h, ys.CL, s, e);
  if (which == 0) {  // result(j) = e1(j) g(j) + e2(j) g(j+1), ascending
    const double gnext = x[e];  // e <= ny < jin
    double bN = 0.0;
    if (e == ny && e > s)
      bN = M4(ib, 1, 1) * x[ny] + M4(ib, 1, 2) * x[ny - 1] + M4(ib, 1, 3) * x[ny - 2] + M4(ib, 1, 4) * x[ny - 3];
    __syncwarp();
    for (int r0 = s; r0 < e; r0 += LB) {
      double gv[LB + 1], e1[LB], e2[LB];
#pragma unroll
      for (int b = 0; b <= LB; ++b) gv[b] = r0 + b < e ? x[r0 + b] : gnext;
#pragma unroll
      for (int b = 0; b < LB; ++b) {
        const bool ok = r0 + b < e;
        e1[b] = ok ? E1(r0 + b) : 0.0;
        e2[b] = ok ? E2(r0 + b) : 0.0;
      }
#pragma unroll
      for (int b = 0; b < LB; ++b) {
        const int r = r0 + b;
        if (r >= e) break;
        x[r] = r == 0 ? 0.0 : (r == ny - 1 ? bN : e1[b] * gv[b] + e2[b] * gv[b + 1]);
      }
    }
  } else {  // result(j) = e2(j) g(j) + e1(j) g(j-1), descending
    const double gprev = s > 0 ? x[s - 1] : 0.0;
    double b0 = 0.0, bN = 0.0;
    if (s == 0 && e > s) b0 = M4(ib, 3, 1) * x[0] + M4(ib, 3, 2) * x[1] + M4(ib, 3, 3) * x[2] + M4(ib, 3, 4) * x[3];
    if (e == ny && e > s)
      bN = M4(ib, 4, 1) * x[ny - 1] + M4(ib, 4, 2) * x[ny - 2] + M4(ib, 4, 3) * x[ny - 3] + M4(ib, 4, 4) * x[ny - 4];
    __syncwarp();
    for (int r1 = e - 1; r1 >= s; r1 -= LB) {
      double gv[LB + 1], e1[LB], e2[LB];
#pragma unroll
      for (int b = 0; b <= LB; ++b) gv[b] = r1 - b >= s ? x[r1 - b] : gprev;
#pragma unroll
      for (int b = 0; b < LB; ++b) {
        const bool ok = r1 - b >= s;
        e1[b] = ok ? E1(r1 - b) : 0.0;
        e2[b] = ok ? E2(r1 - b) : 0.0;
      }
#pragma unroll
      for (int b = 0; b < LB; ++b) {
        const int r = r1 - b;
        if (r < s) break;
        x[r] = r == 0 ? b0 : (r == ny - 1 ? bN : e2[b] * gv[b] + e1[b] * gv[b + 1]);
      }
    }
  }
  __syncwarp();
  solve_cco<YNCH>(x, ny, q.h, ys.CL, CCo<YNCH>(ys.k[YI_L], q.h, CL), CCo<YNCH>(ys.k[YI_D], q.h, CL),
                        CCo<YNCH>(ys.k[YI_U], q.h, CL));
  __syncthreads();
  double *o = out + (size_t)(i - 1) * ny * nz1;
  for (int t = threadIdx.x; t < ny * YT; t += YTHREADS) {
    const int j0 = t / YT, col = t - j0 * YT, kr = kr0 + col;
    if (kr < nz1) o[(size_t)j0 * nz1 + kr] = sm[col * Lp + j0];
  }
}

// ---------------------------------------------------------------------------
// tail of rhsp (rhsp.F90:291-484) for planes 2..nx, one velocity component
// per kernel: RHS assembly, pressure gradient, boun, vistyy, RK3
// combination, rhs history, implzy.
// ---------------------------------------------------------------------------
struct FinalArgs {
  double *u, *v, *w;                 // state: old on entry, new on exit
  const double *p;
  double *rhsupa, *rhsvpa, *rhswpa;  // old on entry, new on exit
  const double *cu, *cv, *cw;        // difvisxx outputs
  const double *uv, *uw, *vw, *vv, *ww;
  const double *fac_u, *fac_v;
  const DState *st;
};

template <int COMP>  // 0: u, 1: v, 2: w
__global__ void __launch_bounds__(YTHREADS) k_final(DCoef c, YSet ys, FinalArgs a, int Lp) {
  extern __shared__ double sm[];
  __shared__ double ub1s[YT], ubts[YT];
  const int nx = c.nx, ny = c.ny, nz1 = c.nz1;
  const int i = blockIdx.y + 2, kr0 = blockIdx.x * YT;
  const bool last = i == nx;
  const YIdx q = yidx(nz1);
  const int jee = COMP == 1 ? ny : ny + 1;
  const size_t PU = (size_t)(ny + 1) * nz1, PV = (size_t)ny * nz1;
  const size_t pl = (size_t)(i - 1) * (COMP == 1 ? PV : PU);  // this plane of the component
  const size_t plv = (size_t)(i - 1) * PV;
  double *T1 = sm, *T2 = sm + YT * Lp;
  const double *prod = COMP == 0 ? a.uv : (COMP == 1 ? a.vv : a.vw);     // y-derivative term
  const double *kprod = COMP == 0 ? a.uw : (COMP == 1 ? a.vw : a.ww);    // z-derivative term
  double *vel = COMP == 0 ? a.u : (COMP == 1 ? a.v : a.w);
  if (!last) ytile_load(T1, prod + plv, ny, nz1, kr0, Lp);
  ytile_load(T2, vel + pl, jee, nz1, kr0, Lp);
  cp_async_wait_all();
  __syncthreads();
  double *x1 = T1 + q.col * Lp, *x2 = T2 + q.col * Lp;
  const double kz = c.kaz[q.k], kv = c.kvis[q.k];
  const double var1 = a.st->var1, var3 = a.st->var3, var4 = a.st->var4;
  const double v2 = last ? 0.0 : a.st->var2;
  const double idxx = c.S[OTBL_S_IDXX];
  const double *ib = c.inby, *cc = c.ccon;
  // column pointers (row r at + r*nz1); invalid columns point at column 0
  const int kc = q.valid ? q.kr : 0;
  const double *cX = (COMP == 0 ? a.cu : (COMP == 1 ? a.cv : a.cw)) + pl + kc;
  const double *kp = kprod + (COMP == 0 ? pl : plv) + kc + (q.valid ? q.pof : 1);  // partner component
  double *hp = (COMP == 0 ? a.rhsupa : (COMP == 1 ? a.rhsvpa : a.rhswpa)) + pl + kc;
  const double *velg = vel + pl + kc;
  const double *pc = a.p + plv + kc;
  const double sgn = q.odd ? 1.0 : -1.0;  // (x * kaz) component = sgn * kz * x[partner]

  int s, e;
  chunk_range(jee, q.h, ys.CL, s, e);
  // ---- RHS into tile 1 (rhsp.F90:164-169, 181-204, 351-418, 423-445)
  if (!last) y_differzy(c, ys, x1, q.h, COMP == 1 ? 1 : 0);
  const CCo<YNCH> IDYY(ys.k[Y_IDYY], q.h, ys.CL);
  for (int r0 = s; r0 < e; r0 += YB) {
    double cxv[YB], kpv[YB];
#pragma unroll
    for (int b = 0; b < YB; ++b) {
      const int r = r0 + b;
      const bool ok = r < e;
      cxv[b] = ok ? __ldg(cX + (size_t)r * nz1) : 0.0;
      kpv[b] = (ok && !last && (COMP != 2 || r < ny)) ? __ldg(kp + (size_t)r * nz1) : 0.0;
    }
#pragma unroll
    for (int b = 0; b < YB; ++b) {
      const int r = r0 + b;
      if (r >= e) break;
      const int j = r + 1;
      double R = cxv[b];
      const double kzt = sgn * kz * kpv[b];
      if (COMP == 0) {
        if (!last) {
          R = (x1[r] + kzt) + R;
          if (j >= 2 && j <= ny) R = R - x2[r] * kv;
        }
      } else if (COMP == 1) {
        if (!last) {
          if (j >= 2 && j <= ny - 1) R = R - x2[r] * kv;
          R = R + kzt;
          R = R + x1[r];
        }
        if (j == 1 || j == ny) R = 0.0;
      } else {
        if (!last) {
          if (j >= 2 && j <= ny) R = R - x2[r] * kv;
          R = R + x1[r];
          if (j <= ny) R = R + kzt;
        }
      }
      x1[r] = q.valid ? R : 0.0;
    }
  }
  __syncwarp();
  if (COMP != 1) {  // wall and top rows of the u,w RHS (rhsp.F90:438-442)
    if (s == 0 && e > s)
      x1[0] = -1.0 / M4(ib, 2, 1) * (M4(ib, 2, 2) * x1[1] + M4(ib, 2, 3) * x1[2] + M4(ib, 2, 4) * x1[3]);
    if (e == jee && e > s) x1[jee - 1] = 0.0;
  }
  // ---- velocity after the pressure gradient (rhsp.F90:291-339); interior rows
  auto star = [&](int r, double o) -> double {  // r = j - 1, o = old velocity
    if (COMP == 0) {
      if (last) return o;
      return o - var1 * idxx * (__ldg(pc + PV + (size_t)r * nz1) - __ldg(pc + (size_t)r * nz1));
    } else if (COMP == 1) {
      return o - var1 * IDYY(r) * (__ldg(pc + (size_t)(r + 1) * nz1) - __ldg(pc + (size_t)r * nz1));
    } else {
      const double pp = __ldg(pc + (size_t)r * nz1 + (q.valid ? q.pof : 1));
      const double av = var1 * kz;
      return o - (q.odd ? av * pp : -av * pp);
    }
  };
  // boun rows 1 and jee of the updated velocity (boun.f90:37-52)
  if (q.h == 0) {
    double ub1 = 0.0, ubt = 0.0;
    if (COMP == 1) {
      ubt = q.kr == 0 ? c.vmagic[i - 1] : 0.0;
    } else if (q.valid) {
      const double s2 = star(1, x2[1]), s3 = star(2, x2[2]), s4 = star(3, x2[3]);
      const double sn = star(ny - 1, x2[ny - 1]), sn1 = star(ny - 2, x2[ny - 2]), sn2 = star(ny - 3, x2[ny - 3]);
      ub1 = -1.0 / M4(ib, 2, 1) * (M4(ib, 2, 2) * s2 + M4(ib, 2, 3) * s3 + M4(ib, 2, 4) * s4);
      ubt = -1.0 / M2(cc, 1, 1) * (M2(cc, 1, 2) * sn + M2(cc, 1, 3) * sn1 + M2(cc, 1, 4) * sn2);
    }
    ub1s[q.col] = ub1;
    ubts[q.col] = ubt;
  }
  // vistyy below overwrites tile 2; the RK3 combination after it reads the
  // old velocity from global memory, which this kernel only overwrites in
  // its final store.
  __syncthreads();
  // ---- explicit y-viscous term of the old velocity into tile 2
  y_vistyy(c, ys, x2, q.h, COMP == 1 ? 1 : 0);
  // ---- RK3 combination into tile 2 and the new RHS history (rhsp.F90:448-475)
  const double ub1 = ub1s[q.col], ubt = ubts[q.col];
  for (int r0 = s; r0 < e; r0 += YB) {
    double ov[YB], hv[YB];
#pragma unroll
    for (int b = 0; b < YB; ++b) {
      const int r = r0 + b;
      const bool ok = r < e && q.valid;
      ov[b] = ok ? __ldg(velg + (size_t)r * nz1) : 0.0;
      hv[b] = ok ? hp[(size_t)r * nz1] : 0.0;
    }
#pragma unroll
    for (int b = 0; b < YB; ++b) {
      const int r = r0 + b;
      if (r >= e || !q.valid) break;
      const double st = r == 0 ? ub1 : (r == jee - 1 ? ubt : star(r, ov[b]));
      x2[r] = st - (var3 * x1[r] + v2 * x2[r] + var4 * hv[b]);
      hp[(size_t)r * nz1] = x1[r];
    }
  }
  __syncwarp();
  // ---- implicit y-viscous step (rhsp.F90:479-484) into tile 1 rows 0..jee-3
  y_implzy(c, ys, x2, x1, q.h, COMP == 1 ? 1 : 0, ub1, ubt, COMP == 1 ? a.fac_v : a.fac_u);
  __syncthreads();
  for (int t = threadIdx.x; t < jee * YT; t += YTHREADS) {
    const int j0 = t / YT, col = t - j0 * YT, kr = kr0 + col;
    if (kr >= nz1) continue;
    const double v = j0 == 0 ? ub1s[col] : (j0 == jee - 1 ? ubts[col] : T1[col * Lp + j0 - 1]);
    vel[pl + (size_t)j0 * nz1 + kr] = v;
  }
}

// ---------------------------------------------------------------------------
// Fixed-length chunks (CL a compile-time constant, one of kYFixCL). Columns
// are padded to YNCH*CL rows; rows past an operator's n hold zeros and have
// zero coefficients (A of row 0 and U of row n-1 are stored as 0 too), so
// every lane runs exactly CL unrolled steps with constant shared-memory
// offsets and no per-row predicate. Each operator's right-hand side is formed
// inside its forward sweep, the forward fix-up is applied inside the
// backward sweep (prefix products g[] in registers), and the backward fix-up
// inside the pass that consumes the result (suffix products hh[]), so a
// stencil + solve is three passes over the column instead of five. The
// arithmetic is chunk_tri's, step for step.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void scan_up8(double &z, double &G, int h) {
#pragma unroll
  for (int d = 1; d < YNCH; d <<= 1) {
    const double zp = __shfl_up_sync(0xffffffffu, z, d, YNCH);
    const double Gp = __shfl_up_sync(0xffffffffu, G, d, YNCH);
    if (h >= d) {
      z = z + G * zp;
      G = G * Gp;
    }
  }
}
__device__ __forceinline__ void scan_down8(double &w, double &H, int h) {
#pragma unroll
  for (int d = 1; d < YNCH; d <<= 1) {
    const double wn = __shfl_down_sync(0xffffffffu, w, d, YNCH);
    const double Hn = __shfl_down_sync(0xffffffffu, H, d, YNCH);
    if (h + d < YNCH) {
      w = w + H * wn;
      H = H * Hn;
    }
  }
}

// rows [0, YNCH*CL) of the YT columns at kr0; rows past `rows` (and columns
// past nz1) are zero-filled
template <int CL>
__device__ __forceinline__ void ytile_load_pad(double *t, const double *__restrict__ g, int rows, int nz1, int kr0,
                                               int Lp) {
  for (int e = threadIdx.x; e < YNCH * CL * YT; e += YTHREADS) {
    const int j0 = e / YT, col = e - j0 * YT, kr = kr0 + col;
    const bool ok = kr < nz1 && j0 < rows;
    cp_async8(t + col * Lp + j0, ok ? g + (size_t)j0 * nz1 + kr : g, ok);
  }
}

// Forward sweep of the chunk at x (rows s..s+CL-1) with the right-hand side
// rhs(t, x[t-1], x[t], x[t+1]) of the original values; z_t = rhs + A(t)
// z_{t-1}. Leaves the local z in x, the prefix products in g and the carried
// value Yp of the preceding chunks.
template <int CL, class FS, class FA>
__device__ __forceinline__ void fx_forward(double *x, int h, FS rhs, FA A, double (&g)[CL], double &Yp) {
  const double xm = h > 0 ? x[-1] : 0.0;
  const double xp = h < YNCH - 1 ? x[CL] : 0.0;
  __syncwarp();
  double prv = xm, z = 0.0, G = h == 0 ? 0.0 : 1.0;
#pragma unroll
  for (int t = 0; t < CL; ++t) {
    const double cur = x[t];
    const double nxt = t + 1 < CL ? x[t + 1 < CL ? t + 1 : t] : xp;
    const double b = rhs(t, prv, cur, nxt);
    const double a = A(t);
    z = b + a * z;
    G = G * a;
    g[t] = G;
    x[t] = z;
    prv = cur;
  }
  scan_up8(z, G, h);
  Yp = __shfl_up_sync(0xffffffffu, z, 1, YNCH);
  if (h == 0) Yp = 0.0;
}

// Backward sweep with the forward fix-up y = z + g Yp folded in; leaves the
// local w in x, the suffix products in hh and the carried Xn: the solution
// of row t is x[t] + hh[t] * Xn.
template <int CL, class FC, class FU>
__device__ __forceinline__ void fx_backward(double *x, int h, const double (&g)[CL], double Yp, FC C, FU U,
                                            double (&hh)[CL], double &Xn) {
  double w = 0.0, H = 1.0;
#pragma unroll
  for (int t = CL - 1; t >= 0; --t) {
    const double y = x[t] + g[t] * Yp;
    const double cv = C(t);
    const double m = cv * (-U(t));
    w = cv * y + m * w;
    H = H * m;
    hh[t] = H;
    x[t] = w;
  }
  scan_down8(w, H, h);
  Xn = __shfl_down_sync(0xffffffffu, w, 1, YNCH);
  if (h == YNCH - 1) Xn = 0.0;
}

template <int COMP, int CL>  // 0: u, 1: v, 2: w
__global__ void __launch_bounds__(YTHREADS, 2) k_final_f(DCoef c, YSet ys, FinalArgs a, int Lp) {
  extern __shared__ double sm[];
  const int nx = c.nx, ny = c.ny, nz1 = c.nz1;
  const int i = blockIdx.y + 2, kr0 = blockIdx.x * YT;
  const bool last = i == nx;
  const YIdx q = yidx(nz1);
  const int h = q.h, s = h * CL;
  const int jee = COMP == 1 ? ny : ny + 1;
  const size_t PU = (size_t)(ny + 1) * nz1, PV = (size_t)ny * nz1;
  const size_t pl = (size_t)(i - 1) * (COMP == 1 ? PV : PU);
  const size_t plv = (size_t)(i - 1) * PV;
  double *T1 = sm, *T2 = sm + YT * Lp;
  const double *prod = COMP == 0 ? a.uv : (COMP == 1 ? a.vv : a.vw);
  const double *kprod = COMP == 0 ? a.uw : (COMP == 1 ? a.vw : a.ww);
  const int krows = COMP == 0 ? ny + 1 : ny;
  double *vel = COMP == 0 ? a.u : (COMP == 1 ? a.v : a.w);
  if (!last) ytile_load_pad<CL>(T1, prod + plv, ny, nz1, kr0, Lp);
  ytile_load_pad<CL>(T2, vel + pl, jee, nz1, kr0, Lp);
  cp_async_wait_all();
  __syncthreads();
  double *c1 = T1 + q.col * Lp, *c2 = T2 + q.col * Lp;
  double *x1 = c1 + s, *x2 = c2 + s;
  const int kc = q.valid ? q.kr : 0;
  const double *cX = (COMP == 0 ? a.cu : (COMP == 1 ? a.cv : a.cw)) + pl + kc;
  const double *kp = kprod + (COMP == 0 ? pl : plv) + kc + (q.valid ? q.pof : 1);
  double *hp = (COMP == 0 ? a.rhsupa : (COMP == 1 ? a.rhsvpa : a.rhswpa)) + pl + kc;
  const double *velg = vel + pl + kc;
  const double *pc = a.p + plv + kc;
  const double kz = c.kaz[q.k], kv = c.kvis[q.k];
  const double var1 = a.st->var1, var3 = a.st->var3, var4 = a.st->var4;
  const double v2 = last ? 0.0 : a.st->var2;
  const double idxx = c.S[OTBL_S_IDXX];
  const double *ib = c.inby, *cc = c.ccon;
  const double sgn = q.odd ? 1.0 : -1.0;  // (x * kaz) component = sgn * kz * x[partner]
  const int ppof = q.valid ? q.pof : 1;
  const size_t pnext = last ? 0 : PV;
  double g[CL], hh[CL];
  double Yp = 0.0, Xn = 0.0;
  // ---- differzy of the product (lip.f90:152-232) into x1
  if (!last) {
    const int which = COMP == 1 ? 1 : 0;
    const double *db = c.dcby;
    const int chv = which == 0 ? 3 : 1, cha = chv + 1;
    const double bot = M4(db, chv, 1) * c1[0] + M4(db, chv, 2) * c1[1] + M4(db, chv, 3) * c1[2] + M4(db, chv, 4) * c1[3];
    const double top = M4(db, cha, 1) * c1[ny - 1] + M4(db, cha, 2) * c1[ny - 2] + M4(db, cha, 3) * c1[ny - 3] +
                       M4(db, cha, 4) * c1[ny - 4];
    const RCo8 E1(ys.k[YD_E1], h), E2(ys.k[YD_E2], h);
    fx_forward<CL>(
        x1, h,
        [&](int t, double pv, double cu, double nx_) {
          const int r = s + t;
          const double in = which == 0 ? E2(t) * cu + E1(t) * pv : E2(t) * nx_ + E1(t) * cu;
          return r == 0 ? bot : (r == jee - 1 ? top : (r < jee ? in : 0.0));
        },
        RCo8(ys.k[YD_L], h), g, Yp);
    fx_backward<CL>(x1, h, g, Yp, RCo8(ys.k[YD_D], h), RCo8(ys.k[YD_U], h), hh, Xn);
  }
  // ---- RHS assembly (rhsp.F90:164-169, 181-204, 351-418, 423-445). The
  // differzy fix-up is applied first (freeing its products), so that the
  // global loads of each batch of rows are all in flight before the
  // arithmetic that uses them.
  if (!last) {
#pragma unroll
    for (int t = 0; t < CL; ++t) x1[t] = x1[t] + hh[t] * Xn;
  }
#pragma unroll
  for (int t0 = 0; t0 < CL; t0 += 8) {
    double cxv[8], kpv[8];
#pragma unroll
    for (int b = 0; b < 8; ++b)
      if (t0 + b < CL) {
        const int rr = min(s + t0 + b, jee - 1);
        cxv[b] = __ldg(cX + (size_t)rr * nz1);
        kpv[b] = last ? 0.0 : __ldg(kp + (size_t)min(rr, krows - 1) * nz1);
      }
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const int t = t0 + b;
      if (t >= CL) break;
      const int r = s + t, j = r + 1;
      const double d1 = last ? 0.0 : x1[t];
      double R = cxv[b];
      const double kzt = sgn * kz * ((COMP != 2 || r < ny) ? kpv[b] : 0.0);
      if (COMP == 0) {
        if (!last) {
          R = (d1 + kzt) + R;
          if (j >= 2 && j <= ny) R = R - x2[t] * kv;
        }
      } else if (COMP == 1) {
        if (!last) {
          if (j >= 2 && j <= ny - 1) R = R - x2[t] * kv;
          R = R + kzt;
          R = R + d1;
        }
        if (j == 1 || j == ny) R = 0.0;
      } else {
        if (!last) {
          if (j >= 2 && j <= ny) R = R - x2[t] * kv;
          R = R + d1;
          if (j <= ny) R = R + kzt;
        }
      }
      if (COMP != 1 && r == jee - 1) R = 0.0;  // top row of the u,w RHS (rhsp.F90:441-442)
      x1[t] = (q.valid && r < jee) ? R : 0.0;
    }
  }
  if (COMP != 1 && h == 0)  // wall row of the u,w RHS (rhsp.F90:438-440)
    x1[0] = -1.0 / M4(ib, 2, 1) * (M4(ib, 2, 2) * x1[1] + M4(ib, 2, 3) * x1[2] + M4(ib, 2, 4) * x1[3]);
  // ---- velocity after the pressure gradient (rhsp.F90:291-339). P0(r),
  // P1(r) are the pressure values row r needs (p has ny rows; rows past
  // them are padding and read row ny-1)
  auto P0 = [&](int r) {  // p(r) for u and v, the partner component for w
    return __ldg(pc + (size_t)min(r, ny - 1) * nz1 + (COMP == 2 ? ppof : 0));
  };
  auto P1 = [&](int r) {  // p of plane i+1 (u) or of row r+1 (v)
    if (COMP == 0) return last ? 0.0 : __ldg(pc + pnext + (size_t)min(r, ny - 1) * nz1);
    return __ldg(pc + (size_t)min(r + 1, ny - 1) * nz1);
  };
  auto star_v = [&](double o, double p0, double p1, double idyy) -> double {
    if (COMP == 0) return last ? o : o - var1 * idxx * (p1 - p0);
    if (COMP == 1) return o - var1 * idyy * (p1 - p0);
    const double av = var1 * kz;
    return o - (q.odd ? av * p0 : -av * p0);
  };
  auto star = [&](int r, double o, double idyy) -> double {
    return star_v(o, P0(r), COMP == 2 ? 0.0 : P1(r), idyy);
  };
  // boun rows 1 and jee of the updated velocity (boun.f90:37-52), from the
  // old velocity still in the tile
  double ub1 = 0.0, ubt = 0.0;
  if (COMP == 1) {
    ubt = q.kr == 0 ? c.vmagic[i - 1] : 0.0;
  } else {
    if (h == 0 && q.valid) {
      const double s2 = star(1, c2[1], 0.0), s3 = star(2, c2[2], 0.0), s4 = star(3, c2[3], 0.0);
      const double sn = star(ny - 1, c2[ny - 1], 0.0), sn1 = star(ny - 2, c2[ny - 2], 0.0);
      const double sn2 = star(ny - 3, c2[ny - 3], 0.0);
      ub1 = -1.0 / M4(ib, 2, 1) * (M4(ib, 2, 2) * s2 + M4(ib, 2, 3) * s3 + M4(ib, 2, 4) * s4);
      ubt = -1.0 / M2(cc, 1, 1) * (M2(cc, 1, 2) * sn + M2(cc, 1, 3) * sn1 + M2(cc, 1, 4) * sn2);
    }
    ub1 = __shfl_sync(0xffffffffu, ub1, 0, YNCH);
    ubt = __shfl_sync(0xffffffffu, ubt, 0, YNCH);
  }
  // ---- vistyy of the old velocity (lip.f90:447-513) in x2
  {
    const int which = COMP == 1 ? 1 : 0, ic = which == 0 ? 3 : 1;
    const double *vb = c.cofvby;
    const double b0 = M4(vb, ic, 1) * c2[0] + M4(vb, ic, 2) * c2[1] + M4(vb, ic, 3) * c2[2] + M4(vb, ic, 4) * c2[3];
    const double bN = M4(vb, ic + 1, 1) * c2[jee - 1] + M4(vb, ic + 1, 2) * c2[jee - 2] +
                      M4(vb, ic + 1, 3) * c2[jee - 3] + M4(vb, ic + 1, 4) * c2[jee - 4];
    const RCo8 F1(ys.k[YV_F1], h), F2(ys.k[YV_F2], h), F3(ys.k[YV_F3], h);
    fx_forward<CL>(
        x2, h,
        [&](int t, double pv, double cu, double nx_) {
          const int r = s + t;
          const double in = F1(t) * nx_ + F2(t) * cu + F3(t) * pv;
          return r == 0 ? b0 : (r == jee - 1 ? bN : (r < jee ? in : 0.0));
        },
        RCo8(ys.k[YV_L], h), g, Yp);
    fx_backward<CL>(x2, h, g, Yp, RCo8(ys.k[YV_D], h), RCo8(ys.k[YV_U], h), hh, Xn);
  }
  // ---- RK3 combination and the new RHS history (rhsp.F90:448-475): the
  // vistyy fix-up first, then batches of rows with their loads in flight
#pragma unroll
  for (int t = 0; t < CL; ++t) x2[t] = x2[t] + hh[t] * Xn;
  {
    const RCo8 IDYY(ys.k[Y_IDYY], h);
#pragma unroll
    for (int t0 = 0; t0 < CL; t0 += 4) {
      double ov[4], hv[4], p0[4], p1[4], iy[4];
#pragma unroll
      for (int b = 0; b < 4; ++b)
        if (t0 + b < CL) {
          const int rr = min(s + t0 + b, jee - 1);
          ov[b] = __ldg(velg + (size_t)rr * nz1);
          hv[b] = __ldg(hp + (size_t)rr * nz1);
          p0[b] = P0(rr);
          p1[b] = COMP == 2 ? 0.0 : P1(rr);
          iy[b] = COMP == 1 ? IDYY(t0 + b) : 0.0;
        }
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int t = t0 + b;
        if (t >= CL) break;
        const int r = s + t;
        const double st = r == 0 ? ub1 : (r == jee - 1 ? ubt : star_v(ov[b], p0[b], p1[b], iy[b]));
        const double nv = st - (var3 * x1[t] + v2 * x2[t] + var4 * hv[b]);
        x2[t] = (q.valid && r < jee) ? nv : 0.0;
        if (q.valid && r < jee) hp[(size_t)r * nz1] = x1[t];
      }
    }
  }
  // ---- implzy (lip.f90:528-597): rows qq = 0..jee-3 from rows qq..qq+2 of
  // x2, into x1; the fix-up is folded into the store
  {
    const int n = jee - 2;
    const double *fac = COMP == 1 ? a.fac_v : a.fac_u;
    const double a1raw = fac[3 * (jee + 1)], a3raw = fac[3 * (jee + 1) + 1];
    const RCo8 F1(ys.k[YM_F1], h), F2(ys.k[YM_F2], h), F3(ys.k[YM_F3], h);
    fx_forward<CL>(
        x1, h,
        [&](int t, double, double, double) {
          const int qq = s + t;
          double v = F1(t) * x2[t] + F2(t) * x2[t + 1] + F3(t) * x2[t + 2];
          if (qq == 0) v = v - a1raw * ub1;
          if (qq == n - 1) v = v - a3raw * ubt;
          return qq < n ? v : 0.0;
        },
        RCo8(ys.k[YM_L], h), g, Yp);
    fx_backward<CL>(x1, h, g, Yp, RCo8(ys.k[YM_D], h), RCo8(ys.k[YM_U], h), hh, Xn);
    if (q.valid) {
      double *o = vel + pl + q.kr;
#pragma unroll
      for (int t = 0; t < CL; ++t) {
        const int qq = s + t;
        if (qq < n) o[(size_t)(qq + 1) * nz1] = x1[t] + hh[t] * Xn;
      }
      if (h == 0) {
        o[0] = ub1;
        o[(size_t)(jee - 1) * nz1] = ubt;
      }
    }
  }
}

// Runs f(std::integral_constant<int, CL>) when the fixed-length kernels are
// compiled for CL.
template <class F>
bool with_yfix(int CL, F f) {
  switch (CL) {
    case 6: f(std::integral_constant<int, 6>{}); return true;
    case 10: f(std::integral_constant<int, 10>{}); return true;
    case 14: f(std::integral_constant<int, 14>{}); return true;
    case 18: f(std::integral_constant<int, 18>{}); return true;
    case 22: f(std::integral_constant<int, 22>{}); return true;
    case 26: f(std::integral_constant<int, 26>{}); return true;
    case 30: f(std::integral_constant<int, 30>{}); return true;
    case 34: f(std::integral_constant<int, 34>{}); return true;
    default: return false;
  }
}

// ---------------------------------------------------------------------------
// pois.f90:106-117 + soltriy: tridiagonal in y per (x-mode, kz). The LU of
// each (i, k) system depends only on the grid, so its pivots are computed
// once (k_pois_lu) and every substep runs the pre-factored tile solve.
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

// The pivots of the CTA's 16 modes are staged in shared memory next to the
// right-hand-side tile (column c uses pivot column c/2).
__global__ void __launch_bounds__(YTHREADS) k_pois_solve(DCoef c, YSet ys, double *phi,
                                                         const double *__restrict__ dinv, int Lp) {
  extern __shared__ double sm[];
  const int ny = c.ny, ny1 = ny - 1, nz1 = c.nz1, nm = c.nz2 + 1;
  const int i = blockIdx.y + 2, kr0 = blockIdx.x * YT, k0 = kr0 / 2;
  double *col0 = phi + (size_t)(i - 1) * ny * nz1;
  double *D = sm + YT * Lp;  // YT/2 pivot columns, pitch Lp
  ytile_load(sm, col0, ny1, nz1, kr0, Lp);
  const double *dv0 = dinv + (size_t)(i - 1) * ny * nm;
  for (int e = threadIdx.x; e < ny1 * (YT / 2); e += YTHREADS) {
    const int j0 = e / (YT / 2), m = e - j0 * (YT / 2), k = k0 + m;
    const bool ok = k < nm;
    cp_async8(D + m * Lp + j0, ok ? dv0 + (size_t)j0 * nm + k : dv0, ok);
  }
  cp_async_wait_all();
  __syncthreads();
  const YIdx q = yidx(nz1);
  double *x = sm + q.col * Lp;
  const double *dcol = D + (q.col >> 1) * Lp;
  if (i == 2 && q.k == 0 && q.valid && q.h == 0) x[ny1 - 1] = 0.0;  // pois.f90:113
  __syncwarp();
  const int CL = ys.CL;
  const CCo<YNCH> A1(ys.k[YP_A1], q.h, CL), A3c(ys.k[YP_A3], q.h, CL);
  chunk_tri<YNCH>(
      x, ny1, q.h, CL, [&](int r) { return -A1(r) * dcol[r - 1]; }, [&](int r) { return dcol[r]; },
      [&](int r) { return A3c(r); });
  __syncthreads();
  for (int t = threadIdx.x; t < ny1 * YT; t += YTHREADS) {
    const int j0 = t / YT, col = t - j0 * YT, kr = kr0 + col;
    if (kr < nz1) col0[(size_t)j0 * nz1 + kr] = sm[col * Lp + j0];
  }
}

// ---------------------------------------------------------------------------
// launch wrappers
// ---------------------------------------------------------------------------
// Column pitch: odd, so 16 consecutive columns of one row fall in distinct
// 8-byte banks (tile loads/stores), and, with chunk lengths = 2 mod 4
// (chunk_len(.., true)), the 2-column x 8-chunk half-warp pattern of the
// sweeps is conflict-free as well.
static int ypitch(int rows) { return rows | 1; }

cudaError_t launch_interpy(otbl_ctx *c) {
  const int nz1 = c->dc.nz1, ny = c->cfg.ny;
  const int Lp = ypitch(ny + 1);
  const size_t smem = sizeof(double) * YT * Lp;
  cudaFuncSetAttribute(k_interpy, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dim3 g((nz1 + YT - 1) / YT, c->cfg.nx);
  prof_begin(c, PK_INTERPY);
  k_interpy<<<g, YTHREADS, smem, c->stream>>>(c->dc, yset(c->yco, 0), c->f[OTBL_F_U], c->w.uy, 0, Lp);
  k_interpy<<<g, YTHREADS, smem, c->stream>>>(c->dc, yset(c->yco, 0), c->f[OTBL_F_W], c->w.wy, 0, Lp);
  k_interpy<<<g, YTHREADS, smem, c->stream>>>(c->dc, yset(c->yco, 1), c->f[OTBL_F_V], c->w.vy, 1, Lp);
  prof_end(c);
  c->launches += 3;
  return cudaGetLastError();
}

cudaError_t launch_final(otbl_ctx *c) {
  FinalArgs a;
  a.u = c->f[OTBL_F_U];
  a.v = c->f[OTBL_F_V];
  a.w = c->f[OTBL_F_W];
  a.p = c->f[OTBL_F_P];
  a.rhsupa = c->f[OTBL_F_RHSUPA];
  a.rhsvpa = c->f[OTBL_F_RHSVPA];
  a.rhswpa = c->f[OTBL_F_RHSWPA];
  a.cu = c->w.cu;
  a.cv = c->w.cv;
  a.cw = c->w.cw;
  a.uv = c->w.uv;
  a.uw = c->w.uw;
  a.vw = c->w.vw;
  a.vv = c->w.vv;
  a.ww = c->w.ww;
  a.fac_u = c->w.fac_u;
  a.fac_v = c->w.fac_v;
  a.st = c->st;
  const int ny = c->cfg.ny;
  const int Lp = ypitch(ny + 1);
  const size_t smem = sizeof(double) * 2 * YT * Lp;
  cudaFuncSetAttribute(k_final<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaFuncSetAttribute(k_final<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaFuncSetAttribute(k_final<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dim3 g((c->dc.nz1 + YT - 1) / YT, c->cfg.nx - 1);
  prof_begin(c, PK_FINAL);
  const int CL = c->yco.CL;
  const bool fixed = with_yfix(CL, [&](auto cl) {
    constexpr int C = decltype(cl)::value;
    // padded column plus two rows read by the implzy stencil past the last
    // chunk (they feed only padded output rows); odd pitch
    const int Lpf = YNCH * C + 3;
    const size_t smf = sizeof(double) * 2 * YT * Lpf;
    cudaFuncSetAttribute(k_final_f<0, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf);
    cudaFuncSetAttribute(k_final_f<1, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf);
    cudaFuncSetAttribute(k_final_f<2, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf);
    k_final_f<1, C><<<g, YTHREADS, smf, c->stream>>>(c->dc, yset(c->yco, 1), a, Lpf);
    k_final_f<0, C><<<g, YTHREADS, smf, c->stream>>>(c->dc, yset(c->yco, 0), a, Lpf);
    k_final_f<2, C><<<g, YTHREADS, smf, c->stream>>>(c->dc, yset(c->yco, 0), a, Lpf);
  });
  if (!fixed) {
    k_final<1><<<g, YTHREADS, smem, c->stream>>>(c->dc, yset(c->yco, 1), a, Lp);
    k_final<0><<<g, YTHREADS, smem, c->stream>>>(c->dc, yset(c->yco, 0), a, Lp);
    k_final<2><<<g, YTHREADS, smem, c->stream>>>(c->dc, yset(c->yco, 0), a, Lp);
  }
  prof_end(c);
  c->launches += 3;
  return cudaGetLastError();
}

cudaError_t launch_pois_lu(otbl_ctx *c) {
  dim3 g((c->dc.nz2 + 1 + 127) / 128, c->cfg.nx - 1);
  k_pois_lu<<<g, 128, 0, c->stream>>>(c->dc, c->w.pois_dinv);
  c->launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_pois_solve(otbl_ctx *c, double *phi) {
  const int ny = c->cfg.ny;
  const int Lp = ypitch(ny - 1);
  const size_t smem = sizeof(double) * (YT + YT / 2) * Lp;
  cudaFuncSetAttribute(k_pois_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dim3 g((c->dc.nz1 + YT - 1) / YT, c->cfg.nx - 1);
  prof_begin(c, PK_POIS_SOLVE);
  k_pois_solve<<<g, YTHREADS, smem, c->stream>>>(c->dc, yset(c->yco, 0), phi, c->w.pois_dinv, Lp);
  prof_end(c);
  c->launches += 1;
  return cudaGetLastError();
}

}  // namespace otbl
