// Streamwise (x) line operators of lip.f90 on shared-memory tiles.
//
// A CTA owns XT consecutive pencils (contiguous (j, kr) indices of the plane
// layout) over all nx planes. Loads read XT consecutive doubles per plane
// (the reference's chp2x transpose is replaced by this gather; its REAL4
// rounding is applied at the same points when OTBL_XPOSE_FP32 is set). One
// warp solves one pencil: 32 lanes own contiguous chunks of planes.
#include "devcommon.cuh"
#include "lines.cuh"
#include "otbl_internal.cuh"

namespace otbl {

#ifndef OTBL_XT_INTERP
#define OTBL_XT_INTERP 8
#endif
#ifndef OTBL_XT_DIFVIS
#define OTBL_XT_DIFVIS 4
#endif
constexpr int XT_INTERP = OTBL_XT_INTERP;  // pencils per CTA for interpxx (1 tile)
constexpr int XT_DIFVIS = OTBL_XT_DIFVIS;  // pencils per CTA for difvisxx (2 tiles)

// Issues the asynchronous copies of a tile (nx planes x XT pencils); the
// caller waits with xtile_wait.
template <int XT>
__device__ __forceinline__ void xtile_load(double *sm, const double *__restrict__ in, int nx, int np, int mp0,
                                           int Lp) {
  for (int e = threadIdx.x; e < nx * XT; e += XT * 32) {
    const int i0 = e / XT, col = e - i0 * XT, mp = mp0 + col;
    const bool ok = mp < np;
    cp_async8(sm + col * Lp + i0, ok ? in + (size_t)i0 * np + mp : in, ok);
  }
}

// Completes the copies; with REAL4 transposes, rounds the tile in place.
template <int XT>
__device__ __forceinline__ void xtile_wait(double *sm, int ntiles, int nx, int Lp, int xr) {
  cp_async_wait_all();
  __syncthreads();
  if (xr) {
    for (int e = threadIdx.x; e < ntiles * XT * Lp; e += XT * 32) sm[e] = rnd(sm[e], 1);
    __syncthreads();
  }
}

template <int XT>
__device__ __forceinline__ void xtile_store(const double *sm, double *__restrict__ out, int nx, int np, int mp0,
                                            int Lp, int xr) {
  for (int e = threadIdx.x; e < nx * XT; e += XT * 32) {
    const int i0 = e / XT, col = e - i0 * XT, mp = mp0 + col;
    if (mp < np) out[(size_t)i0 * np + mp] = rnd(sm[col * Lp + i0], xr);
  }
}

// interpxx, lip.f90:248-300. which 0: u (inxu, cofiux, chi=2, chi2=3);
// which 1: v,w (inxv, cofivx, chi=1, chi2=4). Coefficients of the stencil
// and the solve come chunk-interleaved (XSet).
__global__ void __launch_bounds__(XT_INTERP * 32) k_interpx(DCoef c, XSet xs, const double *__restrict__ in,
                                                            double *__restrict__ out, int which, int np, int Lp) {
  extern __shared__ double sm[];
  const int nx = c.nx, xr = c.xround;
  const int mp0 = blockIdx.x * XT_INTERP;
  xtile_load<XT_INTERP>(sm, in, nx, np, mp0, Lp);
  xtile_wait<XT_INTERP>(sm, 1, nx, Lp, xr);
  const int h = threadIdx.x & 31;
  double *x = sm + (threadIdx.x >> 5) * Lp;
  const int chi = which == 0 ? 2 : 1, chi2 = which == 0 ? 3 : 4;
  const double *ib = c.inbx;
  const CCo<32> E1(xs.k[XI_E1], h, xs.CL), E2(xs.k[XI_E2], h, xs.CL);
  int s, e;
  chunk_range(nx, h, xs.CL, s, e);
  const double gnext = e < nx ? x[e] : 0.0;
  double b0 = 0.0, bN = 0.0;
  if (s == 0 && e > s)
    b0 = M4(ib, chi2, 1) * x[0] + M4(ib, chi2, 2) * x[1] + M4(ib, chi2, 3) * x[2] + M4(ib, chi2, 4) * x[3];
  if (e == nx && e > s)
    bN = M4(ib, chi, 1) * x[nx - 1] + M4(ib, chi, 2) * x[nx - 2] + M4(ib, chi, 3) * x[nx - 3] +
         M4(ib, chi, 4) * x[nx - 4];
  __syncwarp();
  for (int r0 = s; r0 < e; r0 += LB) {  // ascending; a batch reads rows r0..r0+LB first
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
      x[r] = r == 0 ? b0 : (r == nx - 1 ? bN : e1[b] * gv[b] + e2[b] * gv[b + 1]);
    }
  }
  __syncwarp();
  solve_cco<32>(x, nx, h, xs.CL, CCo<32>(xs.k[XI_L], h, xs.CL), CCo<32>(xs.k[XI_D], h, xs.CL),
                       CCo<32>(xs.k[XI_U], h, xs.CL));
  __syncthreads();
  xtile_store<XT_INTERP>(sm, out, nx, np, mp0, Lp, xr);
}

// difvisxx, lip.f90:52-142: Pade d/dx(gin) + rex * Pade d2/dx2(upin), with
// the outflow rows of lip.f90:105,132. which 0: u; which 1: v,w.
__global__ void __launch_bounds__(XT_DIFVIS * 32) k_difvisx(DCoef c, XSet xs, const double *__restrict__ gin,
                                                            const double *__restrict__ upin,
                                                            double *__restrict__ out, int which, int np, int Lp) {
  extern __shared__ double sm[];
  const int nx = c.nx, xr = c.xround;
  const int mp0 = blockIdx.x * XT_DIFVIS;
  double *smg = sm, *smu = sm + XT_DIFVIS * Lp;
  xtile_load<XT_DIFVIS>(smg, gin, nx, np, mp0, Lp);
  xtile_load<XT_DIFVIS>(smu, upin, nx, np, mp0, Lp);
  xtile_wait<XT_DIFVIS>(sm, 2, nx, Lp, xr);
  const int h = threadIdx.x & 31, wv = threadIdx.x >> 5;
  double *x = smg + wv * Lp, *u = smu + wv * Lp;
  const int CL = xs.CL;
  const CCo<32> E1(xs.k[XD_E1], h, CL), E2(xs.k[XD_E2], h, CL);
  const CCo<32> F1(xs.k[XV_F1], h, CL), F2(xs.k[XV_F2], h, CL), F3(xs.k[XV_F3], h, CL);
  const int chv = which == 0 ? 1 : 2, chv1 = chv + 2, ic = which == 0 ? 3 : 1;
  const double *db = c.dcbx, *vb = c.cofvbx;
  const double rex = c.S[OTBL_S_REX], idx = c.S[OTBL_S_IDX], uinf = c.S[OTBL_S_UINF];
  int s, e;
  chunk_range(nx, h, xs.CL, s, e);
  // halos and boundary stencils, read before anything is overwritten
  const double gprev = s > 0 ? x[s - 1] : 0.0;
  double uprev = s > 0 ? u[s - 1] : 0.0;
  const double unext = e < nx ? u[e] : 0.0;
  double gb0 = 0.0, gbN = 0.0, ub0 = 0.0, ubN = 0.0, uN = 0.0, uN1 = 0.0;
  if (s == 0 && e > s) {
    gb0 = M5(db, chv, 1) * x[0] + M5(db, chv, 2) * x[1] + M5(db, chv, 3) * x[2] + M5(db, chv, 4) * x[3];
    ub0 = M4(vb, ic, 1) * u[0] + M4(vb, ic, 2) * u[1] + M4(vb, ic, 3) * u[2] + M4(vb, ic, 4) * u[3];
  }
  if (e == nx && e > s) {
    gbN = M5(db, chv1, 1) * x[nx - 1] + M5(db, chv1, 2) * x[nx - 2] + M5(db, chv1, 3) * x[nx - 3] +
          M5(db, chv1, 4) * x[nx - 4];
    ubN = M4(vb, ic + 1, 1) * u[nx - 1] + M4(vb, ic + 1, 2) * u[nx - 2] + M4(vb, ic + 1, 3) * u[nx - 3] +
          M4(vb, ic + 1, 4) * u[nx - 4];
    uN = u[nx - 1];
    uN1 = u[nx - 2];
  }
  __syncwarp();
  // convective right-hand side, descending in place; a batch reads rows
  // r1-LB..r1 before writing r1-LB+1..r1
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
      x[r] = r == 0 ? gb0 : (r == nx - 1 ? gbN : e1[b] * gv[b + 1] + e2[b] * gv[b]);
    }
  }
  // viscous right-hand side, ascending in place
  for (int r0 = s; r0 < e; r0 += LB) {
    double uv[LB + 2], f1[LB], f2[LB], f3[LB];
    uv[0] = uprev;  // original value of row r0-1
#pragma unroll
    for (int b = 0; b <= LB; ++b) uv[b + 1] = r0 + b < e ? u[r0 + b] : unext;
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
      u[r] = r == 0 ? ub0 : (r == nx - 1 ? ubN : f1[b] * uv[b + 2] + f2[b] * uv[b + 1] + f3[b] * uv[b]);
    }
    uprev = uv[LB];  // original value of the last row of this batch
  }
  __syncwarp();
  solve_cco<32>(x, nx, h, xs.CL, CCo<32>(xs.k[XD_L], h, CL), CCo<32>(xs.k[XD_D], h, CL),
                       CCo<32>(xs.k[XD_U], h, CL));
  solve_cco<32>(u, nx, h, xs.CL, CCo<32>(xs.k[XV_L], h, CL), CCo<32>(xs.k[XV_D], h, CL),
                       CCo<32>(xs.k[XV_U], h, CL));
  for (int r = s; r < e; ++r) x[r] = r == nx - 1 ? uinf * (uN - uN1) * idx + rex * 0.0 : x[r] + rex * u[r];
  __syncthreads();
  xtile_store<XT_DIFVIS>(smg, out, nx, np, mp0, Lp, xr);
}

cudaError_t launch_interpx(otbl_ctx *c) {
  const int nz1 = c->dc.nz1, ny = c->cfg.ny, nx = c->cfg.nx;
  const int npu = nz1 * (ny + 1), npv = nz1 * ny;
  const int Lp = nx | 1;
  const size_t smem = sizeof(double) * XT_INTERP * Lp;
  const dim3 gu((npu + XT_INTERP - 1) / XT_INTERP), gv((npv + XT_INTERP - 1) / XT_INTERP);
  const XSet x0 = xset(c->xco, 0), x1 = xset(c->xco, 1);
  prof_begin(c, PK_INTERPX);
  cudaFuncSetAttribute(k_interpx, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_interpx<<<gu, XT_INTERP * 32, smem, c->stream>>>(c->dc, x0, c->f[OTBL_F_U], c->w.ux, 0, npu, Lp);
  k_interpx<<<gv, XT_INTERP * 32, smem, c->stream>>>(c->dc, x1, c->f[OTBL_F_V], c->w.vx, 1, npv, Lp);
  k_interpx<<<gu, XT_INTERP * 32, smem, c->stream>>>(c->dc, x1, c->f[OTBL_F_W], c->w.wx, 1, npu, Lp);
  prof_end(c);
  c->launches += 3;
  return cudaGetLastError();
}

cudaError_t launch_difvisx(otbl_ctx *c) {
  const int nz1 = c->dc.nz1, ny = c->cfg.ny, nx = c->cfg.nx;
  const int npu = nz1 * (ny + 1), npv = nz1 * ny;
  const int Lp = nx | 1;
  const size_t smem = sizeof(double) * 2 * XT_DIFVIS * Lp;
  const int T = XT_DIFVIS * 32;
  const dim3 gu((npu + XT_DIFVIS - 1) / XT_DIFVIS), gv((npv + XT_DIFVIS - 1) / XT_DIFVIS);
  const XSet x0 = xset(c->xco, 0), x1 = xset(c->xco, 1);
  prof_begin(c, PK_DIFVISX);
  cudaFuncSetAttribute(k_difvisx, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_difvisx<<<gu, T, smem, c->stream>>>(c->dc, x0, c->w.uu, c->f[OTBL_F_U], c->w.cu, 0, npu, Lp);
  k_difvisx<<<gv, T, smem, c->stream>>>(c->dc, x1, c->w.uv, c->f[OTBL_F_V], c->w.cv, 1, npv, Lp);
  k_difvisx<<<gu, T, smem, c->stream>>>(c->dc, x1, c->w.uw, c->f[OTBL_F_W], c->w.cw, 1, npu, Lp);
  prof_end(c);
  c->launches += 3;
  return cudaGetLastError();
}

}  // namespace otbl
