// Streamwise (x) line operators of lip.f90 (interpxx, difvisxx), one thread
// per line. A line is a fixed (j, kr) of the plane layout; its nx values are
// read with the plane stride, so the reference's chp2x transpose is replaced
// by these strided, warp-coalesced loads (its REAL4 rounding is applied at
// the same points when OTBL_XPOSE_FP32 is set).
#include "devcommon.cuh"
#include "otbl_internal.cuh"

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
template <>
struct XTune<double> {
  static constexpr int kxi = 16, kxd = 8, minb_i = 8;
};
template <>
struct XTune<float> {
  static constexpr int kxi = 8, kxd = 8, minb_i = 1;  // 0.88 ms unbounded, 1.19 at >= 8 CTAs
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
  if (c->mixed)
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
  if (c->mixed)
    k_difvisx<float><<<dim3((npu + bs - 1) / bs, 3), bs, 0, c->stream>>>(c->dcf, a);
  else
    k_difvisx<double><<<dim3((npu + bs - 1) / bs, 3), bs, 0, c->stream>>>(c->dc, a);
  prof_end(c);
  c->launches += 1;
  return cudaGetLastError();
}

}  // namespace otbl
