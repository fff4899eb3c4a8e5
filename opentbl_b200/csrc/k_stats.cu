// One-point statistics, statsp (stotf.F90:51-291), with the x pre-pass rhsp
// does when dostat is set (rhsp.F90:70-92). Not on the substep path: the
// reference computes them every avcrt steps (bl_1.F90:92).
//
//   k_stats_x    one thread per x-line (j, kr), coalesced across kr:
//                u_x = interpx_new(u) shifted by one plane (rhsp.F90:71-79),
//                dudx = diffx(u_x), dwdx = diffx(w), dvdx = diffx(v)
//                (lip.f90:703-765, fd_ix and fd_dx), into the line scratch
//                s1, s2, s3, t1
//   k_stats_y    one thread per y-column (i, kr) of a group of planes:
//                buf1..buf5 = interpy_new of u_x, w, dwdx, dudx (fd_iy) and
//                p (fd_iyp) onto the wall positions, buf6..buf8 = diffy of
//                buf1, buf2, v (fd_dvdy) (stotf.F90:101-110,
//                lip.f90:666-699,767-809), into t2 and t3
//   k_stats_acc  one warp per row (i, j): the k = 0 terms, the sums over the
//                spanwise modes (cte = 1 for k = 0, 2 otherwise,
//                stotf.F90:118-217) reduced across the warp, and the triple
//                products over the physical points after three c2r
//                transforms (stotf.F90:264-285), added to the accumulators
//
// The groups of planes are sized so that the eight buffers fit in t2 and
// t3. Every compact solve is the reference's serial recurrence in its order;
// the sums over k and over the physical points are reduced in a different
// order than the reference's serial loops (rounding-level differences).
#include <algorithm>

#include "devcommon.cuh"
#include "otbl_internal.cuh"
#include "zline.cuh"

namespace otbl {

namespace {

#define C8(c, r, j) (c)[((size_t)(j)-1) * 8 + (r)-1]

__device__ __forceinline__ double rd(double x, int xr) { return xr ? (double)(float)x : x; }

// interpx_new (lip.f90:736-765) of a line of nx values at stride st, the
// input rounded to REAL4 when xr (the chp2x transpose), the result written
// shifted by one plane as rhsp.F90:75-79 does: out(i+1) = interp(i), out(1)
// = interp(1). The backward sweep writes x_j into row j+1, whose forward
// value it has already consumed.
__device__ void interpx_shift(const double *c, int nx, const double *in, double *out, size_t st, int xr) {
  auto I = [&](int i) { return rd(in[(size_t)(i - 1) * st], xr); };
  auto O = [&](int i) -> double & { return out[(size_t)(i - 1) * st]; };
  double s = 0.0;
  for (int m = 1; m <= 4; ++m) s += C8(c, m, 1) * I(m);
  O(1) = s;
  for (int i = 2; i <= nx - 2; ++i) {
    s = 0.0;
    for (int m = 1; m <= 4; ++m) s += C8(c, m, 3) * I(i - 2 + m);
    O(i) = s;
  }
  s = 0.0;
  for (int m = 1; m <= 4; ++m) s += C8(c, m, nx - 1) * I(nx - 4 + m);
  O(nx - 1) = s;
  s = 0.0;
  for (int m = 1; m <= 4; ++m) s += C8(c, m, nx) * I(nx - 4 + m);
  O(nx) = s;
  double prev = O(1);
  for (int j = 2; j <= nx; ++j) {
    prev = O(j) - C8(c, 6, j) * prev;
    O(j) = prev;
  }
  double xn = prev * C8(c, 7, nx);  // interp(nx): dropped by the shift
  for (int j = nx - 1; j >= 1; --j) {
    xn = (O(j) - C8(c, 8, j) * xn) * C8(c, 7, j);
    O(j + 1) = xn;
  }
  O(1) = xn;
}

// diffx_inplace (lip.f90:703-731) of a line at stride st
__device__ void diffx_line(const double *c, int nx, const double *in, double *out, size_t st, int xr) {
  auto I = [&](int i) { return rd(in[(size_t)(i - 1) * st], xr); };
  auto O = [&](int i) -> double & { return out[(size_t)(i - 1) * st]; };
  double s = 0.0;
  for (int m = 1; m <= 5; ++m) s += C8(c, m, 1) * I(m);
  O(1) = s;
  s = 0.0;
  for (int m = 1; m <= 5; ++m) s += C8(c, m, 2) * I(m);
  O(2) = s;
  for (int i = 3; i <= nx - 2; ++i) {
    s = 0.0;
    for (int m = 1; m <= 5; ++m) s += C8(c, m, 3) * I(i - 3 + m);
    O(i) = s;
  }
  s = 0.0;
  for (int m = 1; m <= 5; ++m) s += C8(c, m, nx - 1) * I(nx - 5 + m);
  O(nx - 1) = s;
  s = 0.0;
  for (int m = 1; m <= 5; ++m) s += C8(c, m, nx) * I(nx - 5 + m);
  O(nx) = s;
  double prev = O(1);
  for (int j = 2; j <= nx; ++j) {
    prev = O(j) - C8(c, 6, j) * prev;
    O(j) = prev;
  }
  double xn = prev * C8(c, 7, nx);
  O(nx) = xn;
  for (int j = nx - 1; j >= 1; --j) {
    xn = (O(j) - C8(c, 8, j) * xn) * C8(c, 7, j);
    O(j) = xn;
  }
}

// interpy_new (lip.f90:767-809) of a column at stride st: ny+1-tipo input
// rows of element type TI, ny output rows
template <typename TI>
__device__ void interpy_col(const double *c, int ny, const TI *in, double *out, size_t st, int tipo) {
  auto I = [&](int j) { return (double)in[(size_t)(j - 1) * st]; };
  auto O = [&](int j) -> double & { return out[(size_t)(j - 1) * st]; };
  const int ch = tipo == 1 ? 0 : 1;
  double s = 0.0;
  for (int m = 1; m <= 4; ++m) s += C8(c, m, 1) * I(m + 1);
  O(1) = tipo == 0 ? 0.0 : s;  // u and w vanish at the wall
  s = 0.0;
  for (int m = 1; m <= 5; ++m) s += C8(c, m, 2) * I(m + 1);
  O(2) = s;
  for (int j = 3; j <= ny - 2; ++j) {
    s = 0.0;
    for (int m = 1; m <= 4; ++m) s += C8(c, m, j) * I(j - 2 + m);
    O(j) = s;
  }
  s = 0.0;
  for (int m = 1; m <= 3 + ch; ++m) s += C8(c, m, ny - 1) * I(ny - 3 + m);
  O(ny - 1) = s;
  s = 0.0;
  for (int m = 1; m <= 3 + ch; ++m) s += C8(c, m, ny) * I(ny - 3 + m);
  O(ny) = s;
  double prev = O(2);
  for (int j = 3; j <= ny; ++j) {
    prev = O(j) - C8(c, 6, j) * prev;
    O(j) = prev;
  }
  double xn = prev * C8(c, 7, ny);
  O(ny) = xn;
  for (int j = ny - 1; j >= 2; --j) {
    xn = (O(j) - C8(c, 8, j) * xn) * C8(c, 7, j);
    O(j) = xn;
  }
}

// diffy_inplace (lip.f90:666-699) of a column of ny rows at stride st
__device__ void diffy_col(const double *c, int ny, const double *in, double *out, size_t st) {
  auto I = [&](int j) { return in[(size_t)(j - 1) * st]; };
  auto O = [&](int j) -> double & { return out[(size_t)(j - 1) * st]; };
  double s = 0.0;
  for (int m = 1; m <= 4; ++m) s += C8(c, m, 1) * I(m);
  O(1) = s;
  s = 0.0;
  for (int m = 1; m <= 4; ++m) s += C8(c, m, 2) * I(m);
  O(2) = s;
  for (int j = 3; j <= ny - 2; ++j) {
    s = 0.0;
    for (int m = 1; m <= 5; ++m) s += C8(c, m, j) * I(j - 3 + m);
    O(j) = s;
  }
  s = 0.0;
  for (int m = 1; m <= 4; ++m) s += C8(c, m, ny - 1) * I(ny - 4 + m);
  O(ny - 1) = s;
  s = 0.0;
  for (int m = 1; m <= 4; ++m) s += C8(c, m, ny) * I(ny - 4 + m);
  O(ny) = s;
  double prev = O(1);
  for (int j = 2; j <= ny; ++j) {
    prev = O(j) - C8(c, 6, j) * prev;
    O(j) = prev;
  }
  double xn = prev * C8(c, 7, ny);
  O(ny) = xn;
  for (int j = ny - 1; j >= 1; --j) {
    xn = (O(j) - C8(c, 8, j) * xn) * C8(c, 7, j);
    O(j) = xn;
  }
}

struct StatsOps {
  const double *fdvdy, *fdx, *fix, *fiy, *fiyp;
};

// the eight buffers of a group of G planes: buffer b at base[b] + (il*ny +
// j-1)*nz1 + kr
struct StatsBufs {
  double *b[8];
};

__global__ void __launch_bounds__(128) k_stats_x(DCoef c, StatsOps op, const double *__restrict__ u,
                                                 const double *__restrict__ v, const double *__restrict__ w,
                                                 double *ux, double *dudx, double *dwdx, double *dvdx) {
  const int nx = c.nx, ny = c.ny, nz1 = c.nz1, xr = c.xround;
  const size_t PU = (size_t)(ny + 1) * nz1, PV = (size_t)ny * nz1;
  const size_t line = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (line >= PU) return;
  interpx_shift(op.fix, nx, u + line, ux + line, PU, xr);
  diffx_line(op.fdx, nx, ux + line, dudx + line, PU, 0);  // of the unrounded u_x
  diffx_line(op.fdx, nx, w + line, dwdx + line, PU, xr);
  if (line < PV) diffx_line(op.fdx, nx, v + line, dvdx + line, PV, xr);
  if (xr) {  // the chx2p transposes back to planes round to REAL4
    for (int i = 0; i < nx; ++i) {
      ux[(size_t)i * PU + line] = rd(ux[(size_t)i * PU + line], 1);
      dudx[(size_t)i * PU + line] = rd(dudx[(size_t)i * PU + line], 1);
      dwdx[(size_t)i * PU + line] = rd(dwdx[(size_t)i * PU + line], 1);
      if (line < PV) dvdx[(size_t)i * PV + line] = rd(dvdx[(size_t)i * PV + line], 1);
    }
  }
}

template <typename TP>
__global__ void __launch_bounds__(128) k_stats_y(DCoef c, StatsOps op, const double *__restrict__ ux,
                                                 const double *__restrict__ w, const double *__restrict__ dwdx,
                                                 const double *__restrict__ dudx, const TP *__restrict__ p,
                                                 const double *__restrict__ v, StatsBufs bf, int i0, int G) {
  const int ny = c.ny, nz1 = c.nz1;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= G * nz1) return;
  const int il = col / nz1, kr = col - il * nz1, i = i0 + il;
  const size_t PU = (size_t)(ny + 1) * nz1, PV = (size_t)ny * nz1;
  const size_t cu = (size_t)(i - 1) * PU + kr, cv = (size_t)(i - 1) * PV + kr;
  const size_t cb = (size_t)il * PV + kr;
  interpy_col(op.fiy, ny, ux + cu, bf.b[0] + cb, nz1, 0);
  interpy_col(op.fiy, ny, w + cu, bf.b[1] + cb, nz1, 0);
  interpy_col(op.fiy, ny, dwdx + cu, bf.b[2] + cb, nz1, 0);
  interpy_col(op.fiy, ny, dudx + cu, bf.b[3] + cb, nz1, 0);
  interpy_col(op.fiyp, ny, p + cv, bf.b[4] + cb, nz1, 1);
  diffy_col(op.fdvdy, ny, bf.b[0] + cb, bf.b[5] + cb, nz1);
  diffy_col(op.fdvdy, ny, bf.b[1] + cb, bf.b[6] + cb, nz1);
  diffy_col(op.fdvdy, ny, v + cv, bf.b[7] + cb, nz1);
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// the 27 sums over k, in the order of their OTBL_ST_* slots from OTBL_ST_US
enum { KS_US = 0, KS_VS, KS_WS, KS_UV, KS_UW, KS_VW, KS_PUP, KS_PVP, KS_PP, KS_PDUDX, KS_PDUDY, KS_PDVDX, KS_PDVDY,
       KS_PDWDZ, KS_VORTX, KS_VORTY, KS_VORTZ, KS_DISPU, KS_DISPV, KS_DISPW, KS_DISPUV, KS_N };

__global__ void __launch_bounds__(128) k_stats_acc(DCoef c, ZTab z, StatsBufs bf, const double *__restrict__ v,
                                                   const double *__restrict__ dvdx, double *acc, int i0, int G) {
  extern __shared__ __align__(16) unsigned char stsm[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int row = blockIdx.x * 4 + wid;
  const int nx = c.nx, ny = c.ny, nz1 = c.nz1, nz2 = c.nz2, M = z.M;
  if (row >= G * ny) return;
  const int il = row / ny, j = row - il * ny + 1, i = i0 + il;
  const size_t PV = (size_t)ny * nz1;
  const size_t rb = (size_t)il * PV + (size_t)(j - 1) * nz1, rv = (size_t)(i - 1) * PV + (size_t)(j - 1) * nz1;
  const double *b1 = bf.b[0] + rb, *b2 = bf.b[1] + rb, *b3 = bf.b[2] + rb, *b4 = bf.b[3] + rb;
  const double *b5 = bf.b[4] + rb, *b6 = bf.b[5] + rb, *b7 = bf.b[6] + rb, *b8 = bf.b[7] + rb;
  const double *vv = v + rv, *dv = dvdx + rv;
  double ks[KS_N];
#pragma unroll
  for (int q = 0; q < KS_N; ++q) ks[q] = 0.0;
  for (int k = lane; k <= nz2; k += 32) {
    const double cte = k == 0 ? 1.0 : 2.0, kz = c.kaz[k];
    const double u1r = b1[2 * k], u1i = b1[2 * k + 1], w2r = b2[2 * k], w2i = b2[2 * k + 1];
    const double vr = vv[2 * k], vi = vv[2 * k + 1], pr = b5[2 * k], pi = b5[2 * k + 1];
    const double x3r = b3[2 * k], x3i = b3[2 * k + 1], x4r = b4[2 * k], x4i = b4[2 * k + 1];
    const double x6r = b6[2 * k], x6i = b6[2 * k + 1], x7r = b7[2 * k], x7i = b7[2 * k + 1];
    const double x8r = b8[2 * k], x8i = b8[2 * k + 1], dvr = dv[2 * k], dvi = dv[2 * k + 1];
    // i kz times a mode: (-kz Im, kz Re)
    const double wzr = -w2i * kz, wzi = w2r * kz, uzr = -u1i * kz, uzi = u1r * kz;
    const double vzr = -vi * kz, vzi = vr * kz;
    ks[KS_US] += cte * (u1r * u1r + u1i * u1i);
    ks[KS_VS] += cte * (vr * vr + vi * vi);
    ks[KS_WS] += cte * (w2r * w2r + w2i * w2i);
    ks[KS_UV] += cte * (u1r * vr + u1i * vi);
    ks[KS_UW] += cte * (u1r * w2r + u1i * w2i);
    ks[KS_VW] += cte * (vr * w2r + vi * w2i);
    ks[KS_PUP] += cte * (pr * u1r + pi * u1i);
    ks[KS_PVP] += cte * (pr * vr + pi * vi);
    ks[KS_PP] += cte * (pr * pr + pi * pi);
    ks[KS_PDUDX] += cte * (pr * x4r + pi * x4i);
    ks[KS_PDUDY] += cte * (pr * x6r + pi * x6i);
    ks[KS_PDVDX] += cte * (pr * dvr + pi * dvi);
    ks[KS_PDVDY] += cte * (pr * x8r + pi * x8i);
    ks[KS_PDWDZ] += cte * (pr * wzr + pi * wzi);
    double ar = x7r - vzr, ai = x7i - vzi;  // o_x = dwdy - dvdz
    ks[KS_VORTX] += cte * (ar * ar + ai * ai);
    ar = uzr - x3r, ai = uzi - x3i;  // o_y = dudz - dwdx
    ks[KS_VORTY] += cte * (ar * ar + ai * ai);
    ar = dvr - x6r, ai = dvi - x6i;  // o_z = dvdx - dudy
    ks[KS_VORTZ] += cte * (ar * ar + ai * ai);
    ks[KS_DISPU] += cte * ((x4r * x4r + x4i * x4i) + (uzr * uzr + uzi * uzi) + (x6r * x6r + x6i * x6i));
    ks[KS_DISPV] += cte * ((dvr * dvr + dvi * dvi) + (vzr * vzr + vzi * vzi) + (x8r * x8r + x8i * x8i));
    ks[KS_DISPW] += cte * ((wzr * wzr + wzi * wzi) + (x3r * x3r + x3i * x3i) + (x7r * x7r + x7i * x7i));
    ks[KS_DISPUV] += cte * ((uzr * vzr + uzi * vzi) + (x4r * dvr + x4i * dvi) + (x6r * x8r + x6i * x8i));
  }
#pragma unroll
  for (int q = 0; q < KS_N; ++q) ks[q] = warp_sum(ks[q]);
  // triple products of u, w, v in physical space (three c2r transforms)
  double2 *bu = reinterpret_cast<double2 *>(stsm) + (size_t)wid * 3 * M, *bw = bu + M, *bv = bw + M;
  line_c2r(z, b1, bu, lane);
  line_c2r(z, b2, bw, lane);
  line_c2r(z, vv, bv, lane);
  double t3[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // u3, v3, u2v, v2u, w2v, w2u
  for (int t = lane; t < M; t += 32) {
    const double2 a = bu[t], b = bw[t], d = bv[t];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const double uu = h ? a.y : a.x, ww = h ? b.y : b.x, vp = h ? d.y : d.x;
      t3[0] += (uu * uu) * uu;
      t3[1] += (vp * vp) * vp;
      t3[2] += vp * (uu * uu);
      t3[3] += uu * (vp * vp);
      t3[4] += vp * (ww * ww);
      t3[5] += uu * (ww * ww);
    }
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) t3[q] = warp_sum(t3[q]);
  if (lane == 0) {
    const size_t NS = (size_t)nx * ny, at = (size_t)(i - 1) * ny + (j - 1);
    double *A = acc + at;
    // k = 0: means, gradient means, mean vorticity (stotf.F90:118-134)
    A[OTBL_ST_UA * NS] += b1[0];
    A[OTBL_ST_VA * NS] += vv[0];
    A[OTBL_ST_WA * NS] += b2[0];
    A[OTBL_ST_PM * NS] += b5[0];
    A[OTBL_ST_DUDX0 * NS] += b4[0];
    A[OTBL_ST_DVDX0 * NS] += dv[0];
    A[OTBL_ST_DWDX0 * NS] += b3[0];
    A[OTBL_ST_DUDY0 * NS] += b6[0];
    A[OTBL_ST_DVDY0 * NS] += b8[0];
    A[OTBL_ST_DWDY0 * NS] += b7[0];
    A[OTBL_ST_VORTXA * NS] += b7[0];
    A[OTBL_ST_VORTYA * NS] -= b3[0];
    A[OTBL_ST_VORTZA * NS] += dv[0] - b6[0];
#pragma unroll
    for (int q = 0; q < KS_N; ++q) A[(OTBL_ST_US + q) * NS] += ks[q];
#pragma unroll
    for (int q = 0; q < 6; ++q) A[(OTBL_ST_U3 + q) * NS] += t3[q];
  }
}

static_assert(OTBL_ST_US + KS_N == OTBL_ST_U3, "the k sums fill the slots from OTBL_ST_US to OTBL_ST_U3");
static_assert(OTBL_ST_U3 + 6 == OTBL_NSTATS, "six triple products");
static_assert(OTBL_ST_US + KS_PDUDX == OTBL_ST_PDUDX && OTBL_ST_US + KS_DISPUV == OTBL_ST_DISPUV &&
                  OTBL_ST_US + KS_VORTX == OTBL_ST_VORTX,
              "k-sum slots in the order of OTBL_ST_*");

}  // namespace

size_t stats_bytes(int nx, int ny) { return (size_t)OTBL_NSTATS * nx * ny * sizeof(double); }

cudaError_t launch_statsp(otbl_ctx *c) {
  const int nx = c->cfg.nx, ny = c->cfg.ny, nz = c->cfg.nz, nz1 = c->dc.nz1;
  cudaStream_t s = c->stream;
  if (!c->stats) {
    void *p = nullptr;
    const size_t b = stats_bytes(nx, ny);
    cudaError_t e = cudaMalloc(&p, b);
    if (e != cudaSuccess) return e;
    c->allocs.push_back(p);
    c->bytes += b;
    c->stats = static_cast<double *>(p);
    e = cudaMemsetAsync(c->stats, 0, b, s);
    if (e != cudaSuccess) return e;
    c->stats_samples = 0;
  }
  otbl_coef_offsets o;
  otbl_coef_layout(nx, ny, nz, &o);
  StatsOps op;
  op.fdvdy = c->coef_dev + o.off[OTBL_C_FD_DVDY];
  op.fdx = c->coef_dev + o.off[OTBL_C_FD_DX];
  op.fix = c->coef_dev + o.off[OTBL_C_FD_IX];
  op.fiy = c->coef_dev + o.off[OTBL_C_FD_IY];
  op.fiyp = c->coef_dev + o.off[OTBL_C_FD_IYP];
  const size_t PU = (size_t)(ny + 1) * nz1, PV = (size_t)ny * nz1;
  double *ux = c->w.s1, *dudx = c->w.s2, *dwdx = c->w.s3, *dvdx = c->w.t1;
  k_stats_x<<<(unsigned)((PU + 127) / 128), 128, 0, s>>>(c->dc, op, c->f[OTBL_F_U], c->f[OTBL_F_V],
                                                          c->f[OTBL_F_W], ux, dudx, dwdx, dvdx);
  c->launches += 1;
  // groups of G planes: four buffers of G planes in each of t2 and t3
  const size_t lu = otbl_field_len(nx, ny, nz, 1);
  const int G = (int)std::max<size_t>(1, std::min<size_t>(nx, lu / (4 * PV)));
  ZTab z;
  z.tw = reinterpret_cast<const double2 *>(c->w.twz);
  z.tw2 = reinterpret_cast<const double2 *>(c->w.twz2);
  z.M = nz / 2;
  z.nz = nz;
  z.nz2 = c->dc.nz2;
  const size_t smem = (size_t)4 * 3 * z.M * sizeof(double2);
  cudaFuncSetAttribute(k_stats_acc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  for (int i0 = 1; i0 <= nx; i0 += G) {
    const int g = std::min(G, nx - i0 + 1);
    StatsBufs bf;
    for (int b = 0; b < 8; ++b) bf.b[b] = (b < 4 ? c->w.t2 : c->w.t3) + (size_t)(b % 4) * G * PV;
    const int ncol = g * nz1;
    if (c->f32[OTBL_F_P])
      k_stats_y<float><<<(ncol + 127) / 128, 128, 0, s>>>(c->dc, op, ux, c->f[OTBL_F_W], dwdx, dudx,
                                                         reinterpret_cast<const float *>(c->f[OTBL_F_P]),
                                                         c->f[OTBL_F_V], bf, i0, g);
    else
      k_stats_y<double><<<(ncol + 127) / 128, 128, 0, s>>>(c->dc, op, ux, c->f[OTBL_F_W], dwdx, dudx,
                                                          c->f[OTBL_F_P], c->f[OTBL_F_V], bf, i0, g);
    k_stats_acc<<<(g * ny + 3) / 4, 128, smem, s>>>(c->dc, z, bf, c->f[OTBL_F_V], dvdx, c->stats, i0, g);
    c->launches += 2;
  }
  c->stats_samples += 1;
  return cudaGetLastError();
}

}  // namespace otbl
