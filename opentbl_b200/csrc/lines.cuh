// Shared-memory line solvers for the compact (Pade) operators of lip.f90.
//
// Every operator of the path is "explicit stencil, then a tridiagonal solve
// with coefficients pre-factored once" (coeft.f90 coefinv: icon(1,j) = -l_j,
// icon(2,j) = 1/pivot_j, icon(3,j) = upper), applied to many independent
// lines. A CTA stages a tile of whole lines in shared memory, column-major
// (line c at tile + c*Lp), and NCH lanes of one warp share a line: each lane
// owns a contiguous chunk of rows, runs the first-order recurrences of the
// Thomas sweeps locally, and the chunks are stitched by a shuffle scan of the
// affine maps y -> z + G*y (Hillis-Steele, log2(NCH) steps), followed by a
// fix-up pass. The result is the Thomas solution up to rounding order.
//
// Every pass reads its rows B at a time (loads first, then the dependent
// arithmetic) so that several shared-memory and coefficient loads are in
// flight per lane.
#pragma once
#include <cuda_runtime.h>

namespace otbl {

constexpr int LB = 4;  // rows per batch in the sequential passes

// Chunk length for n rows over nch lanes. With `even` it is rounded up to
// 2 mod 4: eight chunk starts then fall in eight distinct even banks, and
// with an odd column pitch the neighbouring column takes the odd banks (a
// conflict-free half-warp of 2 columns x 8 chunks).
__host__ __device__ inline int chunk_len(int n, int nch, bool even) {
  int CL = (n + nch - 1) / nch;
  if (even) CL += (6 - (CL & 3)) & 3;
  return CL;
}

// Rows [s, e) of an n-row line owned by rank h when chunks are CL rows long
// (one CL serves every operator of a kernel, so that all of them share the
// chunk-interleaved coefficient layout).
__device__ __forceinline__ void chunk_range(int n, int h, int CL, int &s, int &e) {
  s = min(n, h * CL);
  e = min(n, s + CL);
}

// In-place solve on rows [0, n) of x:
//   forward  y_0 = b_0,  y_r = b_r + A(r) y_{r-1}
//   backward x_{n-1} = C(n-1) y_{n-1},  x_r = C(r) (y_r - U(r) x_{r+1})
// All 32 lanes of the warp must call this (shuffles use the full mask).
template <int NCH, class FA, class FC, class FU>
__device__ __forceinline__ void chunk_tri(double *x, int n, int h, int CL, FA A, FC C, FU U) {
  int s, e;
  chunk_range(n, h, CL, s, e);
  // ---- forward, local (y_{s-1} = 0)
  double z = 0.0, G = (h == 0) ? 0.0 : 1.0;
  for (int r0 = s; r0 < e; r0 += LB) {
    double xv[LB], av[LB];
#pragma unroll
    for (int b = 0; b < LB; ++b) {
      const int r = r0 + b;
      xv[b] = r < e ? x[r] : 0.0;
      av[b] = (r < e && r > 0) ? A(r) : 0.0;
    }
#pragma unroll
    for (int b = 0; b < LB; ++b) {
      if (r0 + b < e) {
        z = xv[b] + av[b] * z;
        G = G * av[b];
        x[r0 + b] = z;
      }
    }
  }
#pragma unroll
  for (int d = 1; d < NCH; d <<= 1) {
    const double zp = __shfl_up_sync(0xffffffffu, z, d, NCH);
    const double Gp = __shfl_up_sync(0xffffffffu, G, d, NCH);
    if (h >= d) {
      z = z + G * zp;
      G = G * Gp;
    }
  }
  const double Yp = __shfl_up_sync(0xffffffffu, z, 1, NCH);
  if (h > 0) {
    double g = 1.0;
    for (int r0 = s; r0 < e; r0 += LB) {
      double xv[LB], av[LB];
#pragma unroll
      for (int b = 0; b < LB; ++b) {
        const int r = r0 + b;
        xv[b] = r < e ? x[r] : 0.0;
        av[b] = r < e ? A(r) : 0.0;
      }
#pragma unroll
      for (int b = 0; b < LB; ++b) {
        if (r0 + b < e) {
          g = g * av[b];
          x[r0 + b] = xv[b] + g * Yp;
        }
      }
    }
  }
  // ---- backward, local (x_e = 0)
  double w = 0.0, H = 1.0;
  for (int r1 = e - 1; r1 >= s; r1 -= LB) {
    double xv[LB], cv[LB], mv[LB];
#pragma unroll
    for (int b = 0; b < LB; ++b) {
      const int r = r1 - b;
      const bool ok = r >= s;
      xv[b] = ok ? x[r] : 0.0;
      cv[b] = ok ? C(r) : 0.0;
      mv[b] = (ok && r < n - 1) ? -U(r) : 0.0;
    }
#pragma unroll
    for (int b = 0; b < LB; ++b) {
      if (r1 - b >= s) {
        const double m = cv[b] * mv[b];
        w = cv[b] * xv[b] + m * w;
        H = H * m;
        x[r1 - b] = w;
      }
    }
  }
#pragma unroll
  for (int d = 1; d < NCH; d <<= 1) {
    const double wn = __shfl_down_sync(0xffffffffu, w, d, NCH);
    const double Hn = __shfl_down_sync(0xffffffffu, H, d, NCH);
    if (h + d < NCH) {
      w = w + H * wn;
      H = H * Hn;
    }
  }
  double Xn = __shfl_down_sync(0xffffffffu, w, 1, NCH);
  if (h == NCH - 1) Xn = 0.0;
  double g = 1.0;
  for (int r1 = e - 1; r1 >= s; r1 -= LB) {
    double xv[LB], mv[LB];
#pragma unroll
    for (int b = 0; b < LB; ++b) {
      const int r = r1 - b;
      const bool ok = r >= s;
      xv[b] = ok ? x[r] : 0.0;
      mv[b] = (ok && r < n - 1) ? -C(r) * U(r) : 0.0;
    }
#pragma unroll
    for (int b = 0; b < LB; ++b) {
      if (r1 - b >= s) {
        g = g * mv[b];
        x[r1 - b] = xv[b] + g * Xn;
      }
    }
  }
}

// A per-row coefficient in chunk-interleaved order: the value for row r of
// chunk h (rows [h*CL, (h+1)*CL)) sits at (r - h*CL)*NCH + h. The lanes of a
// warp step through their chunks in lockstep, so one warp request reads NCH
// consecutive doubles instead of NCH rows spread over as many cache lines.
// The host builds these copies with the kernel's CL.
template <int NCH>
struct CCo {
  const double *a;
  int base;
  __device__ __forceinline__ CCo(const double *p, int h, int CL) : a(p), base(h - h * CL * NCH) {}
  __device__ __forceinline__ double operator()(int r) const { return __ldg(a + r * NCH + base); }
};

template <int NCH>
__device__ __forceinline__ void solve_cco(double *x, int n, int h, int CL, CCo<NCH> L, CCo<NCH> D, CCo<NCH> U) {
  chunk_tri<NCH>(x, n, h, CL, L, D, U);
}

}  // namespace otbl
