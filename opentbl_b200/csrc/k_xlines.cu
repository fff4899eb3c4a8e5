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
// ---------------------------------------------------------------------------
struct XStream {
  const double *in[3], *in2[3];  // in2: the second input of difvisxx (velocity)
  double *out[3], *ck[3];        // ck: checkpoint scratch of each line set
  int which[3], np[3];
};

constexpr int KXI = 16;  // interpxx segment
constexpr int KXD = 16;  // difvisxx segment (two recurrences)

__global__ void __launch_bounds__(128) k_interpx(DCoef c, XStream a) {
  const int f = blockIdx.y, np = a.np[f];
  const int mp = blockIdx.x * blockDim.x + threadIdx.x;
  if (mp >= np) return;
  const int nx = c.nx, xr = c.xround, which = a.which[f];
  const double *in = a.in[f] + mp;
  double *out = a.out[f] + mp, *ck = a.ck[f] + mp;
  const double *icon = which == 0 ? c.inxu : c.inxv;
  const double *econ = which == 0 ? c.cofiux : c.cofivx;
  const int chi = which == 0 ? 2 : 1, chi2 = which == 0 ? 3 : 4;
  const double *ib = c.inbx;
  auto G = [&](int i) { return rnd(__ldg(in + (size_t)i * np), xr); };
  const double b0 = M4(ib, chi2, 1) * G(0) + M4(ib, chi2, 2) * G(1) + M4(ib, chi2, 3) * G(2) + M4(ib, chi2, 4) * G(3);
  const double bN = M4(ib, chi, 1) * G(nx - 1) + M4(ib, chi, 2) * G(nx - 2) + M4(ib, chi, 3) * G(nx - 3) +
                    M4(ib, chi, 4) * G(nx - 4);
  // right-hand side of row i from g_i, g_{i+1} (interior: lip.f90 stencil)
  auto rhs = [&](int i, double gi, double gi1) {
    return i == 0 ? b0 : (i == nx - 1 ? bN : __ldg(econ + 2 * i) * gi + __ldg(econ + 2 * i + 1) * gi1);
  };
  const int nseg = (nx + KXI - 1) / KXI;
  double y = 0.0;
  for (int sg = 0; sg < nseg; ++sg) {
    const int s = sg * KXI;
    ck[(size_t)sg * np] = y;  // y of row s-1
    double gv[KXI + 1];
#pragma unroll
    for (int b = 0; b <= KXI; ++b) gv[b] = G(min(s + b, nx - 1));
#pragma unroll
    for (int b = 0; b < KXI; ++b) {
      const int i = s + b;
      if (i < nx) y = rhs(i, gv[b], gv[b + 1]) + (i > 0 ? __ldg(icon + 3 * i) : 0.0) * y;
    }
  }
  double xn = 0.0;
  for (int sg = nseg - 1; sg >= 0; --sg) {
    const int s = sg * KXI;
    double gv[KXI + 1], yv[KXI];
#pragma unroll
    for (int b = 0; b <= KXI; ++b) gv[b] = G(min(s + b, nx - 1));
    double yy = ck[(size_t)sg * np];
#pragma unroll
    for (int b = 0; b < KXI; ++b) {
      const int i = s + b;
      if (i < nx) yy = rhs(i, gv[b], gv[b + 1]) + (i > 0 ? __ldg(icon + 3 * i) : 0.0) * yy;
      yv[b] = yy;
    }
#pragma unroll
    for (int b = KXI - 1; b >= 0; --b) {
      const int i = s + b;
      if (i < nx) {
        xn = (yv[b] - __ldg(icon + 3 * i + 2) * xn) * __ldg(icon + 3 * i + 1);
        out[(size_t)i * np] = rnd(xn, xr);
      }
    }
  }
}

__global__ void __launch_bounds__(128) k_difvisx(DCoef c, XStream a) {
  const int f = blockIdx.y, np = a.np[f];
  const int mp = blockIdx.x * blockDim.x + threadIdx.x;
  if (mp >= np) return;
  const int nx = c.nx, xr = c.xround, which = a.which[f];
  const double *gin = a.in[f] + mp, *uin = a.in2[f] + mp;
  double *out = a.out[f] + mp, *ck = a.ck[f] + mp;
  const double *icon = which == 0 ? c.dcxu : c.dcxv;
  const double *iconv = which == 0 ? c.vixu : c.vixv;
  const double *econ = which == 0 ? c.cofcxu : c.cofcxv;
  const double *econv = which == 0 ? c.cofvxu : c.cofvxv;
  const int chv = which == 0 ? 1 : 2, chv1 = chv + 2, ic = which == 0 ? 3 : 1;
  const double *db = c.dcbx, *vb = c.cofvbx;
  const double rex = c.S[OTBL_S_REX], idx = c.S[OTBL_S_IDX], uinf = c.S[OTBL_S_UINF];
  auto G = [&](int i) { return rnd(__ldg(gin + (size_t)i * np), xr); };
  auto U = [&](int i) { return rnd(__ldg(uin + (size_t)i * np), xr); };
  const double gb0 = M5(db, chv, 1) * G(0) + M5(db, chv, 2) * G(1) + M5(db, chv, 3) * G(2) + M5(db, chv, 4) * G(3);
  const double ub0 = M4(vb, ic, 1) * U(0) + M4(vb, ic, 2) * U(1) + M4(vb, ic, 3) * U(2) + M4(vb, ic, 4) * U(3);
  const double gbN = M5(db, chv1, 1) * G(nx - 1) + M5(db, chv1, 2) * G(nx - 2) + M5(db, chv1, 3) * G(nx - 3) +
                     M5(db, chv1, 4) * G(nx - 4);
  const double uN = U(nx - 1), uN1 = U(nx - 2);
  const double ubN = M4(vb, ic + 1, 1) * uN + M4(vb, ic + 1, 2) * uN1 + M4(vb, ic + 1, 3) * U(nx - 3) +
                     M4(vb, ic + 1, 4) * U(nx - 4);
  // right-hand sides of row i: convective e1 g_{i-1} + e2 g_i, viscous
  // f1 u_{i+1} + f2 u_i + f3 u_{i-1} (lip.f90:52-142)
  auto rg = [&](int i, double gm, double g0) {
    return i == 0 ? gb0 : (i == nx - 1 ? gbN : __ldg(econ + 2 * i) * gm + __ldg(econ + 2 * i + 1) * g0);
  };
  auto ru = [&](int i, double um, double u0, double up) {
    return i == 0 ? ub0
                  : (i == nx - 1 ? ubN
                                 : __ldg(econv + 3 * i) * up + __ldg(econv + 3 * i + 1) * u0 +
                                       __ldg(econv + 3 * i + 2) * um);
  };
  const int nseg = (nx + KXD - 1) / KXD;
  double yg = 0.0, yu = 0.0;
  for (int sg = 0; sg < nseg; ++sg) {
    const int s = sg * KXD;
    ck[(size_t)(2 * sg) * np] = yg;
    ck[(size_t)(2 * sg + 1) * np] = yu;
    double gv[KXD + 1], uv[KXD + 2];  // rows s-1 .. s+K-1 (g), s-1 .. s+K (u)
#pragma unroll
    for (int b = 0; b <= KXD; ++b) gv[b] = G(min(max(s + b - 1, 0), nx - 1));
#pragma unroll
    for (int b = 0; b <= KXD + 1; ++b) uv[b] = U(min(max(s + b - 1, 0), nx - 1));
#pragma unroll
    for (int b = 0; b < KXD; ++b) {
      const int i = s + b;
      if (i < nx) {
        yg = rg(i, gv[b], gv[b + 1]) + (i > 0 ? __ldg(icon + 3 * i) : 0.0) * yg;
        yu = ru(i, uv[b], uv[b + 1], uv[b + 2]) + (i > 0 ? __ldg(iconv + 3 * i) : 0.0) * yu;
      }
    }
  }
  double xg = 0.0, xu = 0.0;
  for (int sg = nseg - 1; sg >= 0; --sg) {
    const int s = sg * KXD;
    double gv[KXD + 1], uv[KXD + 2], ygv[KXD], yuv[KXD];
#pragma unroll
    for (int b = 0; b <= KXD; ++b) gv[b] = G(min(max(s + b - 1, 0), nx - 1));
#pragma unroll
    for (int b = 0; b <= KXD + 1; ++b) uv[b] = U(min(max(s + b - 1, 0), nx - 1));
    double a1 = ck[(size_t)(2 * sg) * np], a2 = ck[(size_t)(2 * sg + 1) * np];
#pragma unroll
    for (int b = 0; b < KXD; ++b) {
      const int i = s + b;
      if (i < nx) {
        a1 = rg(i, gv[b], gv[b + 1]) + (i > 0 ? __ldg(icon + 3 * i) : 0.0) * a1;
        a2 = ru(i, uv[b], uv[b + 1], uv[b + 2]) + (i > 0 ? __ldg(iconv + 3 * i) : 0.0) * a2;
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
        const double v = i == nx - 1 ? uinf * (uN - uN1) * idx + rex * 0.0 : xg + rex * xu;
        out[(size_t)i * np] = rnd(v, xr);
      }
    }
  }
}

cudaError_t launch_interpx(otbl_ctx *c) {
  const int nz1 = c->dc.nz1, ny = c->cfg.ny;
  const int npu = nz1 * (ny + 1), npv = nz1 * ny;
  XStream a;
  const double *ins[3] = {c->f[OTBL_F_U], c->f[OTBL_F_V], c->f[OTBL_F_W]};
  double *outs[3] = {c->w.ux, c->w.vx, c->w.wx};
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
  prof_begin(c, PK_INTERPX);
  k_interpx<<<dim3((npu + 127) / 128, 3), 128, 0, c->stream>>>(c->dc, a);
  prof_end(c);
  c->launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_difvisx(otbl_ctx *c) {
  const int nz1 = c->dc.nz1, ny = c->cfg.ny;
  const int npu = nz1 * (ny + 1), npv = nz1 * ny;
  XStream a;
  const double *gins[3] = {c->w.uu, c->w.uv, c->w.uw};
  const double *uins[3] = {c->f[OTBL_F_U], c->f[OTBL_F_V], c->f[OTBL_F_W]};
  double *outs[3] = {c->w.cu, c->w.cv, c->w.cw};
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
  prof_begin(c, PK_DIFVISX);
  k_difvisx<<<dim3((npu + 127) / 128, 3), 128, 0, c->stream>>>(c->dc, a);
  prof_end(c);
  c->launches += 1;
  return cudaGetLastError();
}

}  // namespace otbl
