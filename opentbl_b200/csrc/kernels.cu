// CUDA kernels of the RK3 substep (sm_100a, FP64).
//
// Stage map (reference routine -> kernel):
//   interpxx  lip.f90:248   k_interpx     x-lines (one thread per line), mid-point interp.
//   interpyy  lip.f90:359   k_interpy     y-lines in Fourier space
//   fourxz    ffts.f90:27   k_products    z-lines: 9 c2r + 6 r2c per (i,j)
//                                          line, the six nonlinear products
//                                          and the CFL maxima (rhsp.F90:120-171,
//                                          367-415)
//   difvisxx  lip.f90:52    k_difvisx     x-lines (one thread per line), d/dx + d2/dx2
//   dt        rhsp.F90:214  k_dt          dt, RK3 factors, implzy LU factors
//   genflu    genflu.F90:3  k_genflu_tab  integral quantities, rescaling tables
//                           k_genflu_cols inflow plane + boun of plane 1
//   rhsp tail rhsp.F90:291-484 k_final_s1 y-lines: pressure gradient, RHS
//                                          assembly (differzy), boun, vistyy,
//                                          RK3 combination, implzy
//   outflow_correction boun.f90:63  k_outflow
//   pois      pois.f90:11   k_pois_fwd    divergence + DCT-II along x
//                           k_pois_solve  tridiagonal in y per (x-mode, kz)
//                           k_pois_bwd    DCT-III along x
//                           k_project     pressure/velocity update
// The reference's transposes (change.f90) are not executed on the substep:
// x-lines are read straight from the plane layout (threads over the
// contiguous (j, kr) index, a walk over i with the plane stride), and the
// REAL4 rounding of the transposed payload (OTBL_XPOSE_FP32) is applied at
// exactly the loads/stores where the reference transposes.
#include <cfloat>
#include <cudaTypedefs.h>
#include <mutex>
#include <algorithm>
#include <type_traits>

#include "devcommon.cuh"
#include "fft.cuh"
#include "otbl_internal.cuh"
#include "tma.cuh"
#include "zline.cuh"

namespace otbl {
__device__ __forceinline__ double warp_nmax(double m) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = nmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  return m;
}

template <typename V>
__device__ __forceinline__ void buf_mul(V *a, const V *b, int M, int lane) {
  for (int t = lane; t < M; t += 32) {
    const V x = a[t], y = b[t];
    a[t] = cmake<V>(x.x * y.x, x.y * y.y);
  }
  __syncwarp();
}
template <typename V>
__device__ __forceinline__ void buf_sq(V *a, int M, int lane) {
  for (int t = lane; t < M; t += 32) {
    const V x = a[t];
    a[t] = cmake<V>(x.x * x.x, x.y * x.y);
  }
  __syncwarp();
}
template <typename V>
__device__ __forceinline__ double buf_absmax(const V *a, int M, int lane) {
  double m = 0.0;
  for (int t = lane; t < M; t += 32) m = nmax(nmax(m, fabs((double)a[t].x)), fabs((double)a[t].y));
  return m;
}

// products inputs: the FP64 state u, v, w and the interpolants, outputs the
// six products (W: element type of the intermediate fields)
template <typename W>
struct ProdArgs {
  const double *u, *v, *w;
  const W *ux, *vx, *wx, *uy, *wy, *vy;
  W *uu, *uw, *uv, *vw, *vv, *ww;
  unsigned long long *vm_bits;
  DState *st;
  int setstep;
};

// rhsp.F90:120-171 and 367-415, one warp per (i, j) line, in three parts
// with disjoint inputs and outputs: PART 0 uu, uw and the u, w CFL maxima
// (all planes, rows 1..ny+1; interpxx's outputs only, so it runs beside
// interpyy), PART 2 uv and the v maxima (all planes, rows 1..ny), PART 1
// vw, vv, ww (planes 2..nx-1, rows 1..ny; interpyy's outputs only, so it
// runs beside difvisxx, which reads parts 0 and 2).
template <int PART>
struct ProdPart {
  static constexpr int i0 = PART == 1 ? 2 : 1;      // first plane
  static constexpr int extra = PART == 0 ? 1 : 0;   // rows ny + extra
};
template <typename T, int PART>
__global__ void __launch_bounds__(128) k_products(DCoef c, ZTabT<T> z, ProdArgs<T> a) {
  using V = V2<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  V *sm = reinterpret_cast<V *>(smraw);
  const int M = z.M, lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int j = blockIdx.x * 4 + wid + 1;
  const int i = blockIdx.y + ProdPart<PART>::i0;
  const int ny = c.ny, nz1 = c.nz1;
  if (j > ny + ProdPart<PART>::extra) return;
  V *A = sm + (size_t)wid * 3 * M, *B = A + M, *P = B + M;
  const size_t offu = ((size_t)(i - 1) * (ny + 1) + (j - 1)) * nz1;
  const size_t offv = ((size_t)(i - 1) * ny + (j - 1)) * nz1;
  if (PART == 1) {
    line_c2r(z, a.v + offv, A, lane);
    line_c2r(z, a.wy + offv, B, lane);
    buf_mul(A, B, M, lane);
    line_r2c(z, A, a.vw + offv, lane);
    line_c2r(z, a.vy + offv, A, lane);
    buf_sq(A, M, lane);
    line_r2c(z, A, a.vv + offv, lane);
    line_c2r(z, a.w + offu, A, lane);
    buf_sq(A, M, lane);
    line_r2c(z, A, a.ww + offv, lane);
    return;
  }
  if (PART == 2) {
    double mv = 0.0;
    line_c2r(z, a.vx + offv, A, lane);
    if (a.setstep) mv = buf_absmax(A, M, lane);
    line_c2r(z, a.uy + offv, B, lane);
    buf_mul(A, B, M, lane);
    line_r2c(z, A, a.uv + offv, lane);
    if (a.setstep) {
      mv = warp_nmax(mv);
      if (lane == 0) atomicMax(&a.vm_bits[j], (unsigned long long)__double_as_longlong(mv));
    }
    return;
  }
  double mu = 0.0, mw = 0.0;
  line_c2r(z, a.u + offu, P, lane);
  if (a.setstep) mu = buf_absmax(P, M, lane);
  line_c2r(z, a.ux + offu, A, lane);
  buf_sq(A, M, lane);
  line_r2c(z, A, a.uu + offu, lane);
  line_c2r(z, a.wx + offu, A, lane);
  if (a.setstep) mw = buf_absmax(A, M, lane);
  buf_mul(A, P, M, lane);
  line_r2c(z, A, a.uw + offu, lane);
  if (a.setstep) {
    mu = warp_nmax(mu);
    mw = warp_nmax(mw);
    if (lane == 0) {
      atomicMax(&a.st->umax_bits, (unsigned long long)__double_as_longlong(mu));
      atomicMax(&a.st->wmax_bits, (unsigned long long)__double_as_longlong(mw));
    }
  }
}

// ---------------------------------------------------------------------------
// k_products for M = nz/2 = 32..256 (nz = 64..512): the transforms and
// products of k_products with each line kept in registers between the
// inverse transform's last Stockham pass and the forward transform's first
// one. Register layout L: lane t holds complex element n = t + 32 m in v[m],
// m < E = M/32. Passes: radix E (Ns = 1; its butterflies' inputs j + 32 r are
// one lane's registers; a copy for E = 1), radix 8 (Ns = E), radix 4 (Ns =
// 8 E = M/4); the first reads L, the last writes L (for M < 128 through the
// buffer, its outputs not being in layout L), the two in between go through
// a per-warp shared buffer. M = 256: radices 8, 8, 4, warp_fft's order;
// M = 128: 4, 8, 4, M = 64: 2, 8, 4, M = 32: 8, 4 (warp_fft's order would
// need eight register inputs per butterfly). The buffer's element i is
// stored at i + i/8 for 16-byte (FP64) elements and at i ^ ((i/8) mod 16)
// for 8-byte (FP32) ones, which at M = 256 makes every exchange of the three
// passes conflict-free for its element size (a bank model of the access
// patterns: the FP32 buffer at i + i/8 needed 160 wavefronts per transform
// where 96 is the minimum, and ncu showed 15 M of its 42 M shared wavefronts
// as conflicts at 257x193x512; 0.4 M with the swizzle). The real-to-complex post-step takes the mirrored element
// Z[M-k] from the lane that holds it by warp shuffles instead of a round
// trip through the buffer. For M = 256 the arithmetic is warp_fft's,
// operation for operation.
// ---------------------------------------------------------------------------
template <int M>
struct ZPlan {
  static_assert(M == 256 || M == 128 || M == 64 || M == 32, "register transforms for M = 32..256");
  static constexpr int E = M / 32;
  static constexpr int R3 = 4;  // M = E x 8 x 4
};
template <typename V>
__device__ __forceinline__ int zpad(int i) {
  if constexpr (sizeof(V) == 16)
    return i + (i >> 3);
  else
    return i ^ ((i >> 3) & 15);
}
template <typename V>
__device__ __forceinline__ V shfl_cx(V v, int src) {
  V r;
  r.x = __shfl_sync(0xffffffffu, v.x, src);
  r.y = __shfl_sync(0xffffffffu, v.y, src);
  return r;
}

// inverse (SIGN = +1) or forward (SIGN = -1) FFT of a line in layout L
template <int M, int SIGN, typename V>
__device__ __forceinline__ void zfft_regs(V (&L)[M / 32], V *buf, const V *__restrict__ tw, int t) {
  constexpr int E = M / 32, R3 = ZPlan<M>::R3;
  // pass A: radix E, Ns = 1, input from registers (inputs t + 32 r; a copy
  // for E = 1)
  {
    V v[E];
#pragma unroll
    for (int r = 0; r < E; ++r) v[r] = L[r];
    if constexpr (E > 1) dft_small<E, SIGN>(v);
#pragma unroll
    for (int r = 0; r < E; ++r) buf[zpad<V>(t * E + r)] = v[r];
  }
  __syncwarp();
  // pass B: radix 8, Ns = E (M / 8 butterflies: IB per lane, or the first
  // M / 8 lanes)
  {
    constexpr int NB = M / 8, IB = (NB + 31) / 32;
    V v[IB][8];
#pragma unroll
    for (int it = 0; it < IB; ++it) {
      const int j = t + 32 * it;
      if (j < NB) {
#pragma unroll
        for (int r = 0; r < 8; ++r) v[it][r] = buf[zpad<V>(j + r * NB)];
      }
    }
    __syncwarp();
#pragma unroll
    for (int it = 0; it < IB; ++it) {
      const int j = t + 32 * it, k = j % E;
      if (j < NB) {
        if constexpr (E > 1) {  // Ns = 1 has no twiddles
#pragma unroll
          for (int r = 1; r < 8; ++r) {
            V w = __ldg(&tw[r * k * (M / (8 * E))]);
            if (SIGN > 0) w.y = -w.y;
            v[it][r] = cmul(v[it][r], w);
          }
        }
        dft_small<8, SIGN>(v[it]);
        const int base = (j / E) * (8 * E) + k;
#pragma unroll
        for (int r = 0; r < 8; ++r) buf[zpad<V>(base + r * E)] = v[it][r];
      }
    }
  }
  __syncwarp();
  // pass C: radix R3, Ns = M / R3, output to registers (for M < 128, whose
  // outputs j + r M/R3 are not in layout L, through the buffer)
  {
    constexpr int NC = M / R3, IC = (NC + 31) / 32;
    V v[IC][R3];
#pragma unroll
    for (int it = 0; it < IC; ++it) {
      const int j = t + 32 * it;
      if (j < NC) {
#pragma unroll
        for (int r = 0; r < R3; ++r) v[it][r] = buf[zpad<V>(j + r * NC)];
      }
    }
    __syncwarp();
#pragma unroll
    for (int it = 0; it < IC; ++it) {
      const int j = t + 32 * it;  // k = j mod (M / R3) = j, twiddle stride M/(Ns R3) = 1
      if (j < NC) {
#pragma unroll
        for (int r = 1; r < R3; ++r) {
          V w = __ldg(&tw[r * j]);
          if (SIGN > 0) w.y = -w.y;
          v[it][r] = cmul(v[it][r], w);
        }
        dft_small<R3, SIGN>(v[it]);
#pragma unroll
        for (int r = 0; r < R3; ++r) {
          if constexpr (NC >= 32)
            L[it + r * IC] = v[it][r];
          else
            buf[zpad<V>(j + r * NC)] = v[it][r];
        }
      }
    }
    if constexpr (NC < 32) {
      __syncwarp();
#pragma unroll
      for (int m = 0; m < E; ++m) L[m] = buf[zpad<V>(t + 32 * m)];
      __syncwarp();
    }
  }
}

// c2r of fou (modes 0..nz2, global) into layout L (physical values packed
// as complex), the line_c2r pre-step followed by the inverse FFT
template <int M, typename T, typename TI>
__device__ __forceinline__ void zc2r_regs(const ZTabT<T> &z, const TI *__restrict__ fou, V2<T> (&L)[M / 32],
                                          V2<T> *buf, int t) {
  using V = V2<T>;
  constexpr int E = M / 32;
  const int nz2 = z.nz2;
  V a[E], b[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {  // modes above nz2 are not read (they are 0)
    const int k = t + 32 * m, km = M - k;
    a[m] = k <= nz2 ? ldcx<T>(fou, k) : cmake<V>(T(0), T(0));
    b[m] = km <= nz2 ? ldcx<T>(fou, km) : cmake<V>(T(0), T(0));
  }
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int k = t + 32 * m, km = M - k;
    V aa = k <= nz2 ? a[m] : cmake<V>(T(0), T(0));
    if (k == 0) aa.y = T(0);  // c2r ignores Im X[0]
    V bb = km <= nz2 ? b[m] : cmake<V>(T(0), T(0));
    bb.y = -bb.y;
    const V s = cadd(aa, bb), d = csub(aa, bb);
    const V tt = cmul(cconj(__ldg(z.tw2 + k)), d);  // W^{-k} d
    L[m] = cmake<V>(s.x - tt.y, s.y + tt.x);       // s + i t
  }
  zfft_regs<M, 1>(L, buf, z.tw, t);
}

// r2c of layout L (physical values packed as complex) into fou (modes
// 0..nz2) x 1/nz: forward FFT, then the line_r2c post-step
template <int M, typename T, typename TO>
__device__ __forceinline__ void zr2c_regs(const ZTabT<T> &z, V2<T> (&L)[M / 32], TO *__restrict__ fou, V2<T> *buf,
                                          int t) {
  using V = V2<T>;
  constexpr int E = M / 32;
  zfft_regs<M, -1>(L, buf, z.tw, t);
  const int nz2 = z.nz2;
  const T dnf = T(1) / (T)z.nz;
#pragma unroll
  for (int m = 0; m < E; ++m) {
    // Z[(M - k) mod M], k = t + 32 m: element (32 - t) + 32 (E - 1 - m), held
    // by lane 32 - t in L[E - 1 - m] for t >= 1; element 32 ((E - m) mod E),
    // this lane's own L[(E - m) mod E], for t = 0
    const V other = shfl_cx(L[E - 1 - m], (32 - t) & 31);
    const V zm = t == 0 ? L[(E - m) % E] : other;
    const int k = t + 32 * m;
    if (k <= nz2) {
      const V zk = L[m];
      const V zc = cconj(zm);
      const V e = cmake<V>(T(0.5) * (zk.x + zc.x), T(0.5) * (zk.y + zc.y));
      const V d = csub(zk, zc);
      const V o = cmake<V>(T(0.5) * d.y, T(-0.5) * d.x);  // -i d / 2
      const V xk = cadd(e, cmul(__ldg(z.tw2 + k), o));
      stcx(fou, k, cmake<V>(dnf * xk.x, dnf * xk.y));
    }
  }
  __syncwarp();
}

template <int E, typename V>
__device__ __forceinline__ void regs_mul(V (&a)[E], const V (&b)[E]) {
#pragma unroll
  for (int m = 0; m < E; ++m) a[m] = cmake<V>(a[m].x * b[m].x, a[m].y * b[m].y);
}
template <int E, typename V>
__device__ __forceinline__ void regs_sq(V (&a)[E]) {
#pragma unroll
  for (int m = 0; m < E; ++m) a[m] = cmake<V>(a[m].x * a[m].x, a[m].y * a[m].y);
}
template <int E, typename V>
__device__ __forceinline__ double regs_absmax(const V (&a)[E]) {
  double mx = 0.0;
#pragma unroll
  for (int m = 0; m < E; ++m) mx = nmax(nmax(mx, fabs((double)a[m].x)), fabs((double)a[m].y));
  return mx;
}

// CTAs per SM bound: FP64 unbounded (252 registers, 4.49 ms per substep at
// 1025x193x512; 5.02 at >= 3 CTAs with spills), FP32 >= 4 CTAs (126-128
// registers, 36 bytes of spills in part 0; 2.29-2.30 ms per substep against
// 2.34-2.43 at >= 3 CTAs and 162-168 registers, after the exchange buffer's
// swizzle; 3.16 unbounded before it). M < 256: FP32 >= 5 CTAs (M = 128: 96
// registers, 0.69 against 0.72 ms per substep at 513x193x256 at 111); FP64
// unbounded (M = 128: 152-168 registers, three CTAs; four at 128 registers
// took 1.10-1.11 against 1.08-1.10 ms). A variant with two warps per line (4
// elements per thread, radix-4 passes, named barriers) measured slower in
// both precisions (4.92 and 3.61 ms) and was dropped.
#ifndef OTBL_PR_MB_D
#define OTBL_PR_MB_D 1
#endif
#ifndef OTBL_PR_MB_F
#define OTBL_PR_MB_F 4
#endif
template <int M, typename T, int PART>
__global__ void __launch_bounds__(128, std::is_same<T, double>::value ? OTBL_PR_MB_D : (M < 256 ? 5 : OTBL_PR_MB_F))
    k_products_r(DCoef c, ZTabT<T> z, ProdArgs<T> a) {
  using V = V2<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  V *sm = reinterpret_cast<V *>(smraw);
  constexpr int E = M / 32;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int j = blockIdx.x * 4 + wid + 1;
  const int i = blockIdx.y + ProdPart<PART>::i0;
  const int ny = c.ny, nz1 = c.nz1;
  if (j > ny + ProdPart<PART>::extra) return;
  V *buf = sm + (size_t)wid * (M + M / 8);
  const size_t offu = ((size_t)(i - 1) * (ny + 1) + (j - 1)) * nz1;
  const size_t offv = ((size_t)(i - 1) * ny + (j - 1)) * nz1;
  V A[E], B[E];
  if (PART == 1) {  // planes 2..nx-1, rows 1..ny
    zc2r_regs<M>(z, a.v + offv, A, buf, lane);  // vw = v wy
    zc2r_regs<M>(z, a.wy + offv, B, buf, lane);
    regs_mul<E>(A, B);
    zr2c_regs<M>(z, A, a.vw + offv, buf, lane);
    zc2r_regs<M>(z, a.vy + offv, A, buf, lane);  // vv = vy^2
    regs_sq<E>(A);
    zr2c_regs<M>(z, A, a.vv + offv, buf, lane);
    zc2r_regs<M>(z, a.w + offu, A, buf, lane);  // ww = w^2
    regs_sq<E>(A);
    zr2c_regs<M>(z, A, a.ww + offv, buf, lane);
    return;
  }
  if (PART == 2) {  // all planes, rows 1..ny
    double mv = 0.0;
    zc2r_regs<M>(z, a.vx + offv, A, buf, lane);  // uv = vx uy
    if (a.setstep) mv = regs_absmax<E>(A);
    zc2r_regs<M>(z, a.uy + offv, B, buf, lane);
    regs_mul<E>(A, B);
    zr2c_regs<M>(z, A, a.uv + offv, buf, lane);
    if (a.setstep) {
      mv = warp_nmax(mv);
      if (lane == 0) atomicMax(&a.vm_bits[j], (unsigned long long)__double_as_longlong(mv));
    }
    return;
  }
  double mu = 0.0, mw = 0.0;
  zc2r_regs<M>(z, a.ux + offu, A, buf, lane);  // uu = ux^2
  regs_sq<E>(A);
  zr2c_regs<M>(z, A, a.uu + offu, buf, lane);
  zc2r_regs<M>(z, a.u + offu, B, buf, lane);  // uw = wx u
  if (a.setstep) mu = regs_absmax<E>(B);
  zc2r_regs<M>(z, a.wx + offu, A, buf, lane);
  if (a.setstep) mw = regs_absmax<E>(A);
  regs_mul<E>(A, B);
  zr2c_regs<M>(z, A, a.uw + offu, buf, lane);
  if (a.setstep) {
    mu = warp_nmax(mu);
    mw = warp_nmax(mw);
    if (lane == 0) {
      atomicMax(&a.st->umax_bits, (unsigned long long)__double_as_longlong(mu));
      atomicMax(&a.st->wmax_bits, (unsigned long long)__double_as_longlong(mw));
    }
  }
}

// ---------------------------------------------------------------------------
// dt (rhsp.F90:214-267), RK3 factors, implzy LU (lip.f90:545-568)
// ---------------------------------------------------------------------------
// Factors of (A + var1*B) for implzy (lip.f90:545-568, rows j = 2..jee-1),
// eliminated from the top row down (a UL factorisation; the reference's LU
// eliminates from the bottom, and both solve the same diagonally dominant
// system to rounding), so that the rhsp tail, which forms the right-hand
// side from the top row down, eliminates as it goes. With A_j, B_j, C_j the
// sub-, main and super-diagonal of row j:
//   B'_{jee-1} = B_{jee-1},  m_j = C_j / B'_{j+1},  B'_j = B_j - m_j A_{j+1}
//   fac[3j] = A_j (0 for j = 2), fac[3j+1] = 1/B'_j, fac[3j+2] = -m_j (0 for
//   j = jee-1); descending y_j = r_j + fac[3j+2] y_{j+1}, ascending
//   x_j = (y_j - fac[3j] x_{j-1}) fac[3j+1].
// The two boundary couplings that implzy moves to the right-hand side:
// fac[3*(jee+1)] = A_2, fac[3*(jee+1)+1] = C_{jee-1}.
__device__ void implzy_factor(const DCoef &c, double *fac, int which, double var1) {
  const int ny = c.ny, jee = which == 0 ? ny + 1 : ny;
  const double *icon = which == 0 ? c.vyui : c.vyvi;
  const double *econ = which == 0 ? c.cofvyu : c.cofvyv;
  auto Aj = [&](int j) { return A3(icon, 1, j) + var1 * A3(econ, 3, j); };
  auto Bj = [&](int j) { return A3(icon, 2, j) + var1 * A3(econ, 2, j); };
  auto Cj = [&](int j) { return A3(icon, 3, j) + var1 * A3(econ, 1, j); };
  fac[3 * (jee + 1)] = Aj(2);
  fac[3 * (jee + 1) + 1] = Cj(jee - 1);
  double bp = Bj(jee - 1);
  fac[3 * (jee - 1) + 2] = 0.0;
  for (int j = jee - 1;; --j) {
    const double ib = 1.0 / bp;
    fac[3 * j + 1] = ib;
    fac[3 * j] = j == 2 ? 0.0 : Aj(j);
    if (j == 2) break;
    const double m = Cj(j - 1) * ib;  // m_{j-1} = C_{j-1} / B'_j
    fac[3 * (j - 1) + 2] = -m;
    bp = Bj(j - 1) - m * Aj(j);
  }
}

// One CTA of 64 threads: the CFL reduction over the rows, then dt, the RK3
// factors and the two implzy factorisations (one warp each).
__global__ void __launch_bounds__(64) k_dt(DCoef c, DState *st, const unsigned long long *vm_bits, double *fac_u,
                                           double *fac_v, int m, int setstep, int dt_mode, double dt_fixed) {
  __shared__ double s_dt3[2], s_vmax[2];
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const double *S = c.S;
  const double poco = 1e-7;
  if (setstep) {
    double dt3 = DBL_MAX, vmax = 0.0;
    for (int j = t + 1; j <= c.ny; j += 64) {
      const double vm = __longlong_as_double((long long)vm_bits[j]);
      dt3 = fmin(dt3, c.dymin[j - 1] / fmax(poco, vm));
      vmax = nmax(vmax, vm);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      dt3 = fmin(dt3, __shfl_xor_sync(0xffffffffu, dt3, o));
      vmax = nmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
    }
    if (lane == 0) {
      s_dt3[wid] = dt3;
      s_vmax[wid] = vmax;
    }
  }
  __syncthreads();
  if (t == 0) {
    if (setstep) {
      const double um = __longlong_as_double((long long)st->umax_bits);
      const double wm = __longlong_as_double((long long)st->wmax_bits);
      const double dt1 = S[OTBL_S_DXMIN] / fmax(poco, um);
      const double dt2 = S[OTBL_S_DXMIN] / fmax(poco, wm);
      const double dt3 = fmin(s_dt3[0], s_dt3[1]);
      const double vmax = nmax(s_vmax[0], s_vmax[1]);
      const double dtloc = fmin(fmin(dt1, dt2), fmin(dt3, S[OTBL_S_DTRET]));
      st->umax = um;
      st->wmax = wm;
      st->vmax = vmax;
      if (!isfinite(um) || !isfinite(wm) || !isfinite(vmax)) atomicCAS(&st->err, 0, OTBL_ERR_NAN);
      if (dt_mode == OTBL_DT_ADAPTIVE) {
        st->dt = dtloc;
      } else if (!st->dt_frozen) {
        st->dt = dt_fixed > 0.0 ? dt_fixed : dtloc;
        st->dt_frozen = 1;
      }
    }
    const double dt = st->dt;
    if (!(dt > 0.0) || !isfinite(dt)) atomicCAS(&st->err, 0, OTBL_ERR_NAN);
    const int q = m - 1;
    st->var1 = dt * (S[OTBL_S_RKCV + q] + S[OTBL_S_RKDV + q]);
    st->var2 = dt * S[OTBL_S_REX] * S[OTBL_S_RKCV + q];
    st->var3 = dt * S[OTBL_S_RKC + q];
    st->var4 = dt * S[OTBL_S_RKD + q];
    st->rkk = S[OTBL_S_REX] * dt * S[OTBL_S_RKDV + q];
    st->varstep = 5e-1 / dt / S[OTBL_S_RKDV + q];
  }
  __syncthreads();
  if (lane == 0) {
    const double rkk = *(volatile double *)&st->rkk;
    if (wid == 0)
      implzy_factor(c, fac_u, 0, rkk);
    else
      implzy_factor(c, fac_v, 1, rkk);
  }
}

__global__ void k_reset_max(DState *st, unsigned long long *vm_bits, int ny) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) {
    st->umax_bits = 0ull;
    st->wmax_bits = 0ull;
  }
  if (t <= ny) vm_bits[t] = 0ull;
}

// energies + ministats (rhsp.F90:493-509, stotf.F90:395-440) when one
// context holds every plane: ministats' plane-1 branch sets uner(1:3) and its
// plane-nx/2 branch, later in the same loop over planes, overwrites them, so
// the result is that of plane nx/2 alone, including the reference's addition
// of Re u(k=0, j=1)^2 to every row of aux (stotf.F90:433-435). rhsp zeroes
// ener(13:15) before it returns (rhsp.F90:487); so does this kernel.
// One CTA; warp w takes rows j = w, w+32, ..., lanes the modes k = 1..nz2;
// the per-warp partial integrals are added in warp order.
__global__ void __launch_bounds__(1024) k_energies(DCoef c, DState *st, const double *u, const double *v,
                                                  const double *w) {
  __shared__ double part[3][32], row2[3][2];
  const int ny = c.ny, nz1 = c.nz1, i = c.nx / 2;
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  for (int f = 0; f < 3; ++f) {
    const int jee = f == 1 ? ny : ny + 1;
    const double *g = (f == 0 ? u : (f == 1 ? v : w)) + (size_t)(i - 1) * jee * nz1;
    const double r1 = g[0];
    double acc = 0.0;
    for (int j = wp; j < jee; j += 32) {
      double s = 0.0;
      for (int kr = 2 + lane; kr < nz1; kr += 32) {
        const double x = g[(size_t)j * nz1 + kr];
        s += x * x;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      const double a = 2.0 * s;
      if (j < 2 && lane == 0) row2[f][j] = a;
      acc += (a + r1 * r1) * c.hy[j];
    }
    if (lane == 0) part[f][wp] = acc;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    const int f = threadIdx.x, jee = f == 1 ? ny : ny + 1;
    const double *g = (f == 0 ? u : (f == 1 ? v : w)) + (size_t)(i - 1) * jee * nz1;
    double e = 0.0;
    for (int q = 0; q < 32; ++q) e += part[f][q];
    st->ener[f] = e;
    const double q4[4] = {g[0], g[nz1], row2[f][0], row2[f][1]};
    for (int q = 0; q < 4; ++q) {
      const int n = 3 + 4 * f + q;
      st->ener[n] = n >= 12 ? 0.0 : q4[q];
    }
  }
}

__global__ void k_tiempo(DState *st) {
  if (threadIdx.x == 0 && blockIdx.x == 0) st->tiempo = st->tiempo + st->dt;
}

// ---------------------------------------------------------------------------
// genflu (genflu.F90:3-242, NEWGENFLU) in two launches:
//   k_genflu_tab  one CTA: the filtered mean um, u_tau, delta99, Re_theta and
//                 gamma (genflu.F90:67-93), and for the u and the v grid the
//                 rescaled-grid interpolation tables kl, fsca, ntop of
//                 genflu.F90:95-140, into the table scratch `tab`;
//   k_genflu_cols one thread per (component, kr): plane 1 from plane xout,
//                 i.e. the blending of genflu.F90:55-60, the zero modes of
//                 :146-150 and profile (:204-242) in closed form (every output
//                 row is a blend of two rows of the blended input plane).
// Inside the substep (tail = 1) the column threads then apply boun on plane 1
// (boun.f90:33-55) and rhs*pa(plane 1) = 0 (rhsp.F90:424-426,441-442); plane
// 1 is not touched by the rest of rhsp. Sums whose order sets the rounding
// are taken sequentially in the reference's order; everything else is
// element-wise with the reference's expressions, so the result is the one
// of a single sequential pass.
// ---------------------------------------------------------------------------
struct GenArgs {
  double *u, *v, *w;
  void *rhsupa, *rhsvpa, *rhswpa;  // double, or float when rhs32 (mixed path)
  int rhs32;
  const double *u0, *v0;
  double *um;
  double *tab;  // genflu_tab_doubles(ny) doubles of table scratch
  // scalars: inputs dt, tiempo, timeinit; outputs of genflu.F90:67-93
  const double *dt, *tiempo, *timeinit;
  double *timec, *utauout, *rthout, *dout, *gamma1, *gamma2;
  int *err;       // set to err_code for a degenerate rescaled grid; may be null
  int err_code;   // OTBL_DEVERR_GENFLU_GRID (context flag) or OTBL_ERR_NAN
  int tail;
};

__global__ void __launch_bounds__(256) k_genflu_tab(DCoef c, GenArgs a) {
  extern __shared__ double gsm[];
  const int ny = c.ny, nz1 = c.nz1, t = threadIdx.x, T = blockDim.x;
  const size_t PU = (size_t)(ny + 1) * nz1;
  const double *y = c.y, *dy = c.dy;
  const int N1 = ny + 1;
  double *ysca = gsm;             // [2][ny+1]
  double *www = ysca + 2 * N1;    // [2][ny+1]: dobleu output, then wlwa
  double *yyy = www + 2 * N1;     // [2][ny+1]
  double *um = yyy + 2 * N1;      // um(1..ny+1) at um[1..]
  int *kf = reinterpret_cast<int *>(um + ny + 2);  // [2][ny+1] fresh bisection, -1 = outside
  int *kh = kf + 2 * N1;                            // [2][ny+1] its khh
  __shared__ double s_timec, s_g1, s_g2, s_www1[2];
  __shared__ int s_jfirst;
  const double re = c.S[OTBL_S_RE], din = c.S[OTBL_S_DIN], rthin = c.S[OTBL_S_RTHIN];
  const double dt = *a.dt;
  if (t == 0) {
    const double tloc = *a.tiempo - *a.timeinit;
    s_timec = tloc < 20 ? 20.0 : (tloc < 100 ? 100.0 : tloc);
    s_jfirst = ny - 1;
  }
  __syncthreads();
  const double timec = s_timec;
  // um(j) <- (dt/timec) u(k=0, j, plane 1) + um(j)(1 - dt/timec); plane 1's
  // mode 0 is plane xout's (the blending leaves modes 0 alone)
  const double *ux = a.u + (size_t)(c.xout - 1) * PU;
  for (int j = t + 1; j <= ny + 1; j += T) {
    const double v = (dt / timec) * ux[(size_t)(j - 1) * nz1] + a.um[j - 1] * (1.0 - dt / timec);
    um[j] = v;
    a.um[j - 1] = v;
  }
  __syncthreads();
  double uinf = 0.0;  // every thread, same order
  for (int j = ny + 1 - 20; j <= ny + 1 - 5; ++j) uinf += um[j];
  uinf = uinf / 16.0;
  const double u99 = (double)0.99f * uinf;
  // jtop: the loop of genflu.F90:80-84 stops at the first um(j) >= u99
  for (int j = t + 1; j <= ny - 2; j += T)
    if (um[j] >= u99) atomicMin(&s_jfirst, j);
  __syncthreads();
  if (t == 0) {
    const int jf = s_jfirst;
    const int jtop = jf == 1 ? 0 : jf;
    *a.timec = timec;
    *a.utauout = sqrt(fabs((um[2] - um[1]) / (y[2] - y[1]) / re));
    *a.dout = y[jtop];
    double s = 0.0;
    for (int q = 0; q < jtop + 2; ++q) s += (uinf - um[2 + q]) * um[2 + q] * dy[1 + q];
    const double rthout = s * re / uinf;
    *a.rthout = rthout;
    const double gamma2 = rthin / rthout;
    const double gamma1 = pow(gamma2, 0.125);
    *a.gamma2 = gamma2;
    *a.gamma1 = gamma1;
    s_g1 = gamma1;
    s_g2 = gamma2;
    a.tab[3 * N1] = 1.0 / gamma1;  // ggg
  }
  // rescaled grids: kk = 0 (u rows, cell centres) and kk = 1 (v rows)
  for (int e = t; e < 2 * N1; e += T) {
    const int kk = e / N1, j = e - kk * N1;
    if (j >= 1) ysca[e] = kk == 0 ? 5e-1 * (y[j] + y[j + 1]) / din : y[j] / din;
  }
  __syncthreads();
  // dobleu (genflu.F90:250-298): the tanh weights element-wise, the running
  // integral sequentially
  {
    const double ag = 4.0, bg = 0.2;
    const double bg2 = 1.0 - 2.0 * bg, tag = 1.0 / tanh(ag);
    for (int e = t; e < 2 * N1; e += T) {
      const int kk = e / N1, i = e - kk * N1;
      if (i < 2 || i > ny) continue;
      const double *eta = ysca + kk * N1;
      const double xxx = 0.5 * (eta[i] + eta[i - 1]);
      yyy[e] = xxx >= 1.0 ? 1.0 : 0.5 * (1.0 + tag * tanh(ag * (xxx - bg) / (bg2 * xxx + bg)));
    }
  }
  __syncthreads();
  if (t == 0 || t == 32) {
    const int kk = t / 32;
    const double *eta = ysca + kk * N1, *yy = yyy + kk * N1;
    double *ww = www + kk * N1;
    double www1 = (double)0.7895f;
    ww[1] = 0.0;
    for (int i = 2; i <= ny; ++i) {
      ww[i] = ww[i - 1] + yy[i] * (eta[i] - eta[i - 1]);
      if (eta[i] >= 1.0 && eta[i - 1] < 1.0) www1 = ww[i - 1] + (1.0 - eta[i - 1]) * yy[i];
    }
    s_www1[kk] = www1;
  }
  __syncthreads();
  const double gamma1 = s_g1, gamma2 = s_g2;
  double *fsca = a.tab;
  int *kl = reinterpret_cast<int *>(a.tab + 2 * N1);
  int *ntop = reinterpret_cast<int *>(a.tab + 3 * N1 + 1);
  for (int e = t; e < 2 * N1; e += T) {
    const int kk = e / N1, j = e - kk * N1;
    if (j >= 1) www[e] = ysca[e] / gamma1 + (1.0 / gamma2 - 1.0 / gamma1) / s_www1[kk] * www[e];
  }
  __syncthreads();
  // bisection of genflu.F90:120-135 for every row from kll = 1, khh = ny
  for (int e = t; e < 2 * N1; e += T) {
    const int kk = e / N1, i = e - kk * N1;
    const double *ys = ysca + kk * N1;
    const double wl = www[e];
    kf[e] = -1;
    if (i >= 1 && wl <= ys[ny]) {
      int kll = 1, khh = ny;
      while (khh - kll > 1) {
        const int kx = (khh + kll) / 2;
        if (ys[kx] >= wl)
          khh = kx;
        else
          kll = kx;
      }
      kf[e] = kll;
      kh[e] = khh;
    }
  }
  __syncthreads();
  // the reference carries kll from one row to the next; a bisection started
  // at the carried kll = lo ends where the fresh one does unless the target
  // lies at or below ys[lo], where it stays at lo (redone sequentially)
  if (t == 0 || t == 32) {
    const int kk = t / 32;
    const double *ys = ysca + kk * N1, *wl = www + kk * N1;
    int *kfk = kf + kk * N1, *khk = kh + kk * N1;
    int lo = 1, nt = 0;
    for (int i = 1; i <= ny; ++i) {
      if (kfk[i] < 0) continue;
      nt = i;
      if (!(ys[lo] < wl[i])) {
        int kll = lo, khh = ny;
        while (khh - kll > 1) {
          const int kx = (khh + kll) / 2;
          if (ys[kx] >= wl[i])
            khh = kx;
          else
            kll = kx;
        }
        kfk[i] = kll;
        khk[i] = khh;
      }
      lo = kfk[i];
    }
    ntop[kk] = nt;
  }
  __syncthreads();
  for (int e = t; e < 2 * N1; e += T) {
    const int kk = e / N1, i = e - kk * N1;
    const double *ys = ysca + kk * N1;
    if (kf[e] < 0 || i == 0) {
      kl[e] = 0;
      fsca[e] = 0.0;
    } else {
      const int kll = kf[e], khh = kh[e];
      kl[e] = kll;
      fsca[e] = (www[e] - ys[kll]) / (ys[khh] - ys[kll]);
    }
  }
}

// One thread per (kr, component); blockIdx.y = 0 u, 1 w, 2 v.
__global__ void __launch_bounds__(128) k_genflu_cols(DCoef c, GenArgs a) {
  const int ny = c.ny, nz1 = c.nz1, xout = c.xout;
  const int kr = blockIdx.x * blockDim.x + threadIdx.x;
  const int comp = blockIdx.y, r = blockIdx.z;  // one thread per (kr, component, row)
  if (kr >= nz1) return;
  const bool vt = comp == 2;
  const int rows = vt ? ny : ny + 1;
  if (r >= rows) return;
  const size_t P = (size_t)rows * nz1;
  double *f = comp == 0 ? a.u : (comp == 1 ? a.w : a.v);
  const double *in = f + (size_t)(xout - 1) * P + kr;
  double *out = f + kr;
  const int N1 = ny + 1;
  const double *fsca = a.tab + (vt ? N1 : 0);
  const int *kl = reinterpret_cast<const int *>(a.tab + 2 * N1) + (vt ? N1 : 0);
  const int *ntp = reinterpret_cast<const int *>(a.tab + 3 * N1 + 1);
  const int nt = vt ? ntp[1] : ntp[0];
  const bool prof = ntp[0] >= 4 && ntp[1] >= 4;
  const double ggg = a.tab[3 * N1];
  const double yb = c.S[OTBL_S_YBLEND];
  // input row q (0-based) of the blended plane: genflu.F90:55-60 (modes >= 1)
  auto inp = [&](int q) -> double {
    const double v = in[(size_t)q * nz1];
    if (vt || kr < 2) return v;
    const double fb = 0.5 * (1 - tanh(c.y[q + 1] - yb));
    return v * fb;
  };
  // the new plane-1 value of row q before boun
  auto val = [&](int q) -> double {
    if (kr < 2) {  // zero mode, genflu.F90:146-150
      if (kr == 0 && comp == 0) return a.u0[q];
      if (kr == 0 && comp == 2) return a.v0[q];
      return 0.0;
    }
    if (!prof) return inp(q);  // degenerate rescaled grid: blended copy, flagged
    if (!vt) {                 // profile, u-type rows 0..ny
      auto W = [&](int i) {
        const int kll = max(kl[i], 1);
        return inp(kll + 1) * fsca[i] + inp(kll) * (1 - fsca[i]);
      };
      const int rr = q >= nt - 3 ? nt - 4 : q;
      const double wv = rr == 0 ? -W(1) : W(rr);
      return wv * ggg;
    }
    const int i = (q >= nt - 3 ? nt - 4 : q) + 1;  // profile, v-type rows 0..ny-1
    const int kll = max(kl[i], 1);
    return (inp(kll) * fsca[i] + inp(kll - 1) * (1 - fsca[i])) * ggg;
  };
  if (kr == 2 && comp == 0 && r == 0 && !prof && a.err) atomicCAS(a.err, 0, a.err_code);
  double v;
  if (!a.tail) {
    v = val(r);
  } else if (vt) {  // boun on plane 1 (boun.f90:33-55) and the plane-1 RHS history
    v = r == 0 ? 0.0 : (r == ny - 1 ? (kr == 0 ? c.vmagic[0] : 0.0) : val(r));
    if (a.rhs32)
      static_cast<float *>(a.rhsvpa)[(size_t)r * nz1 + kr] = 0.0f;
    else
      static_cast<double *>(a.rhsvpa)[(size_t)r * nz1 + kr] = 0.0;
  } else {
    const double *ib = c.inby, *cc = c.ccon;
    if (r == 0)
      v = -1.0 / M4(ib, 2, 1) * (M4(ib, 2, 2) * val(1) + M4(ib, 2, 3) * val(2) + M4(ib, 2, 4) * val(3));
    else if (r == ny)
      v = -1.0 / M2(cc, 1, 1) * (M2(cc, 1, 2) * val(ny - 1) + M2(cc, 1, 3) * val(ny - 2) + M2(cc, 1, 4) * val(ny - 3));
    else
      v = val(r);
    void *h = comp == 0 ? a.rhsupa : a.rhswpa;
    if (a.rhs32)
      static_cast<float *>(h)[(size_t)r * nz1 + kr] = 0.0f;
    else
      static_cast<double *>(h)[(size_t)r * nz1 + kr] = 0.0;
  }
  out[(size_t)r * nz1] = v;
}

cudaError_t genflu_launch(otbl_ctx *c, const GenArgs &a) {
  const size_t smem = genflu_smem_bytes(c->cfg.ny);
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_genflu_tab, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_genflu_tab<<<1, 256, smem, c->stream>>>(c->dc, a);
  dim3 g((c->dc.nz1 + 127) / 128, 3, c->cfg.ny + 1);
  k_genflu_cols<<<g, 128, 0, c->stream>>>(c->dc, a);
  c->launches += 2;
  return cudaGetLastError();
}

// boun (boun.f90:7-56) on every plane, for the standalone entry point
__global__ void k_boun(DCoef c, double *u, double *v, double *w) {
  const int kr = blockIdx.x * blockDim.x + threadIdx.x;
  if (kr >= c.nz1) return;
  const int i = blockIdx.y + 1, ny = c.ny, nz1 = c.nz1;
  const double *ib = c.inby, *cc = c.ccon;
  double *vc = v + (size_t)(i - 1) * ny * nz1 + kr;
  vc[0] = 0.0;
  vc[(size_t)(ny - 1) * nz1] = kr == 0 ? c.vmagic[i - 1] : 0.0;
  double *fl[2] = {u + (size_t)(i - 1) * (ny + 1) * nz1 + kr, w + (size_t)(i - 1) * (ny + 1) * nz1 + kr};
  for (int f = 0; f < 2; ++f) {
    double *q = fl[f];
    q[0] = -1.0 / M4(ib, 2, 1) * (M4(ib, 2, 2) * q[nz1] + M4(ib, 2, 3) * q[2 * nz1] + M4(ib, 2, 4) * q[3 * nz1]);
    q[(size_t)ny * nz1] = -1.0 / M2(cc, 1, 1) *
                          (M2(cc, 1, 2) * q[(size_t)(ny - 1) * nz1] + M2(cc, 1, 3) * q[(size_t)(ny - 2) * nz1] +
                           M2(cc, 1, 4) * q[(size_t)(ny - 3) * nz1]);
  }
}

// ---------------------------------------------------------------------------
// outflow_correction, boun.f90:63-93: one CTA, fixed-order reductions.
// ---------------------------------------------------------------------------
__device__ double block_sum(double v, double *red) {
  const int t = threadIdx.x;
  red[t] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (t < s) red[t] = red[t] + red[t + s];
    __syncthreads();
  }
  const double r = red[0];
  __syncthreads();
  return r;
}

template <typename TR>
__global__ void __launch_bounds__(256) k_outflow(DCoef c, double *u, const double *v, TR *rhsupa) {
  __shared__ double red[256];
  const int t = threadIdx.x, nx = c.nx, ny = c.ny, nz1 = c.nz1;
  const size_t PU = (size_t)(ny + 1) * nz1, PV = (size_t)ny * nz1;
  double a = 0.0, b = 0.0, d = 0.0;
  for (int i = 2 + t; i <= nx; i += 256) a += v[(size_t)(i - 1) * PV + (size_t)(ny - 1) * nz1];
  for (int j = 2 + t; j <= ny; j += 256) {
    b += u[(size_t)(j - 1) * nz1] * c.dy[j - 1];
    d += u[(size_t)(nx - 1) * PU + (size_t)(j - 1) * nz1] * c.dy[j - 1];
  }
  const double sv = block_sum(a, red), s1 = block_sum(b, red), s2 = block_sum(d, red);
  double sumax = sv * c.S[OTBL_S_DX1];
  sumax = sumax - s1;
  sumax = sumax + s2;
  const double alpha = -sumax / (c.y[ny] - c.y[1]);
  for (int j = 2 + t; j <= ny; j += 256) {
    double *q = u + (size_t)(nx - 1) * PU + (size_t)(j - 1) * nz1;
    q[0] = q[0] + alpha;
    TR *h = rhsupa + (size_t)(nx - 1) * PU + (size_t)(j - 1) * nz1;
    h[0] = (TR)((double)h[0] + alpha * c.S[OTBL_S_IDX]);
  }
}

// ---------------------------------------------------------------------------
// pois (pois.f90:11-189)
// ---------------------------------------------------------------------------
template <typename T>
struct XTabT {
  const V2<T> *tw;   // exp(-2 pi i t/n), t < n
  const V2<T> *tw2;  // exp(-i pi t/(2n)), t < n
  int n;
};
using XTab = XTabT<double>;

// The x-line transforms of pois: MB spanwise modes of one row j per CTA of
// 256 threads. The loads and stores walk the planes with the MB modes of a
// plane on consecutive threads (MB x 16 contiguous bytes per plane row); the
// MB complex lines of length n = nx-1 sit in shared memory in the layout of
// xpad (line stride xline_ld, which puts the MB lines of one plane on
// different banks) and are transformed together, NT/MB threads per line.
// MB is chosen per n so that n * MB <= 4096 (n = 1024: 4 modes, 74 KB in
// FP64, 33 KB in FP32).

// divergence (pois.f90:41-54) + DCT-II along x (cosftx iopt=-1); output
// phi-hat in plane layout (v-type, plane i = x-mode index + 2). Mode 0 made
// real (pois.f90:102). The launch covers spanwise modes kbeg..kend, MB per
// CTA; T is the transform's arithmetic and phi's element type (FP64, or FP32
// for the higher modes of the mixed path). The divergence itself is formed
// in FP64 from the FP64 velocity.
// With 512 threads both x-DCT kernels are bounded to 64 registers (two CTAs
// per SM): at 66 registers the FP64 forward kernel of n = 1024 fits one CTA
// per SM instead of two and took 1.18 instead of 0.83 ms per substep at
// 1025x193x512. The 256-thread variants are not bounded (at 64 registers
// they spill).
template <typename T, int MB, int NT>
__global__ void __launch_bounds__(NT, NT >= 512 ? 2 : 1) k_pois_fwd(DCoef c, XTabT<T> x, const double *__restrict__ u,
                                                 const double *__restrict__ v, const double *__restrict__ w,
                                                 T *__restrict__ phi, int kbeg, int kend) {
  using V = V2<T>;
  extern __shared__ __align__(16) unsigned char xsm_raw[];
  V *xsm = reinterpret_cast<V *>(xsm_raw);
  const int n = x.n, ld = xline_ld<V>(n, MB), ny = c.ny, nz1 = c.nz1, xr = c.xround;
  const int j = blockIdx.y + 1;
  const int k0 = kbeg + blockIdx.x * MB;
  const size_t PU = (size_t)(ny + 1) * nz1, PV = (size_t)ny * nz1;
  const double idx = c.S[OTBL_S_IDX], idy = c.idy[j];
  for (int e = threadIdx.x; e < n * MB; e += NT) {
    const int l = e % MB, tt = e / MB;
    const int k = k0 + l;
    V val;
    val.x = 0;
    val.y = 0;
    if (k <= kend) {
      const int i = tt + 2;
      const double kz = c.kaz[k];
      const double2 wv = *reinterpret_cast<const double2 *>(w + (size_t)(i - 1) * PU + (size_t)j * nz1 + 2 * k);
      const double2 v1 = *reinterpret_cast<const double2 *>(v + (size_t)(i - 1) * PV + (size_t)j * nz1 + 2 * k);
      const double2 v0 = *reinterpret_cast<const double2 *>(v + (size_t)(i - 1) * PV + (size_t)(j - 1) * nz1 + 2 * k);
      const double2 ua = *reinterpret_cast<const double2 *>(u + (size_t)(i - 1) * PU + (size_t)j * nz1 + 2 * k);
      const double2 ub = *reinterpret_cast<const double2 *>(u + (size_t)(i - 2) * PU + (size_t)j * nz1 + 2 * k);
      double re = -kz * wv.y + (v1.x - v0.x) * idy;
      double im = kz * wv.x + (v1.y - v0.y) * idy;
      re = re + idx * (ua.x - ub.x);
      im = im + idx * (ua.y - ub.y);
      val.x = (T)rnd(re, xr);
      val.y = (T)rnd(im, xr);
    }
    const int dst = (tt & 1) ? n - 1 - (tt >> 1) : (tt >> 1);
    xsm[l * ld + xpad<V>(dst)] = val;
  }
  __syncthreads();
  {
    const int G = NT / MB, l = threadIdx.x / G;
    block_fft_lines<-1, NT>(xsm + l * ld, n, x.tw, threadIdx.x % G, G);
  }
  const T dnf = (T)(1.0 / (double)n);
  for (int e = threadIdx.x; e < n * MB; e += NT) {
    const int l = e % MB, kk = e / MB;
    const int k = k0 + l;
    if (k > kend) continue;
    const V Vv = xsm[l * ld + xpad<V>(kk)], Vm = xsm[l * ld + xpad<V>(kk == 0 ? 0 : n - kk)];
    const V wq = __ldg(x.tw2 + kk);
    const V y = cadd(cmul(wq, Vv), cmul(cconj(wq), Vm));
    V out;
    out.x = (T)rnd((double)(dnf * y.x), xr);
    out.y = k == 0 ? (T)0 : (T)rnd((double)(dnf * y.y), xr);
    *reinterpret_cast<V *>(phi + (size_t)(kk + 1) * PV + (size_t)(j - 1) * nz1 + 2 * k) = out;
  }
}

// DCT-III along x (cosftx iopt=+1), in place on phi-hat, modes kbeg..kend
template <typename T, int MB, int NT>
__global__ void __launch_bounds__(NT, NT >= 512 ? 2 : 1) k_pois_bwd(DCoef c, XTabT<T> x, T *__restrict__ phi, int kbeg, int kend) {
  using V = V2<T>;
  extern __shared__ __align__(16) unsigned char xsm_raw[];
  V *xsm = reinterpret_cast<V *>(xsm_raw);
  const int n = x.n, ld = xline_ld<V>(n, MB), ny = c.ny, nz1 = c.nz1, xr = c.xround;
  const int j = blockIdx.y + 1;
  const int k0 = kbeg + blockIdx.x * MB;
  const size_t PV = (size_t)ny * nz1;
  for (int e = threadIdx.x; e < n * MB; e += NT) {
    const int l = e % MB, kk = e / MB;
    const int k = k0 + l;
    V val;
    val.x = 0;
    val.y = 0;
    if (k <= kend) {
      const V q = *reinterpret_cast<const V *>(phi + (size_t)(kk + 1) * PV + (size_t)(j - 1) * nz1 + 2 * k);
      V Y, Ym;
      Y.x = (T)rnd((double)q.x, xr);
      Y.y = (T)rnd((double)q.y, xr);
      Ym.x = 0;
      Ym.y = 0;
      if (kk > 0) {
        const V qm = *reinterpret_cast<const V *>(phi + (size_t)(n - kk + 1) * PV + (size_t)(j - 1) * nz1 + 2 * k);
        Ym.x = (T)rnd((double)qm.x, xr);
        Ym.y = (T)rnd((double)qm.y, xr);
      }
      V d;  // Y - i Ym
      d.x = Y.x + Ym.y;
      d.y = Y.y - Ym.x;
      val = cmul(cconj(__ldg(x.tw2 + kk)), d);
    }
    xsm[l * ld + xpad<V>(kk)] = val;
  }
  __syncthreads();
  {
    const int G = NT / MB, l = threadIdx.x / G;
    block_fft_lines<1, NT>(xsm + l * ld, n, x.tw, threadIdx.x % G, G);
  }
  for (int e = threadIdx.x; e < n * MB; e += NT) {
    const int l = e % MB, tt = e / MB;
    const int k = k0 + l;
    if (k > kend) continue;
    const V Vv = xsm[l * ld + xpad<V>((tt & 1) ? n - 1 - (tt >> 1) : (tt >> 1))];
    // mode 0 is real (pois.f90:102): its imaginary pencil is identically zero
    // in the reference's real transforms, while the complex line transform
    // used here leaves rounding-level values there
    V out;
    out.x = (T)rnd((double)((T)0.5 * Vv.x), xr);
    out.y = k == 0 ? (T)0 : (T)rnd((double)((T)0.5 * Vv.y), xr);
    *reinterpret_cast<V *>(phi + (size_t)(tt + 1) * PV + (size_t)(j - 1) * nz1 + 2 * k) = out;
  }
}

// TMA-fed persistent forms of the two x-DCT kernels, for the power-of-two
// line lengths N = 256..2048. One CTA per SM (two for the FP32 backward
// transform) walks the tiles q = blockIdx.x + m gridDim.x, a tile being row j
// and MB spanwise modes (k-group fastest, so the CTAs at work share rows and
// the v row pair of a tile meets its neighbour's in L2). The loads are TMA
// boxes issued by thread 0 and counted on mbarriers, the waits bounded
// (OTBL_ERR_TIMEOUT, after draining the copies in flight); the next tile's
// data arrive while this tile's FFT runs, which the one-shot kernels above
// leave to other CTAs' warps (measured there: long-scoreboard stalls 15 per
// issue in the forward, 7 in the backward transform, DRAM at 30% and 9% of
// its peak on a 1025x49x512 box). Arithmetic: k_pois_fwd's and k_pois_bwd's,
// operation for operation.

// spanwise modes per x-DCT CTA: n * MB <= 4096 and at most 8
__host__ __device__ constexpr int pois_mb(int n) { return n <= 512 ? 8 : (n <= 1024 ? 4 : (n <= 2048 ? 2 : 1)); }

template <int MB>
struct PoisChunk {
  static constexpr int CP = MB >= 8 ? 64 : 128;  // planes per chunk
  static constexpr int RW = 2 * MB;              // kr of a row segment
  static constexpr int UB = ((CP + 1) * RW * 8 + 127) / 128 * 128;
  static constexpr int VB = CP * 2 * RW * 8, WB = CP * RW * 8;
  static constexpr int CH = UB + VB + WB;  // chunk stride in the ring (bytes)
  static constexpr unsigned TX = (unsigned)((CP + 1) * RW * 8 + VB + WB);
};

// forward: the tile's velocity rows stream through a ring of S chunks of CP
// planes (u row j over CP + 1 planes, v rows j - 1 and j, w row j); thread 0
// refills a slot at the first CTA barrier after its chunk was read, so S
// chunks are in flight through the FFT
template <typename T, int N>
__global__ void __launch_bounds__(512, 1) k_pois_fwd_t(DCoef c, XTabT<T> x, const __grid_constant__ PoisMaps maps,
                                                      T *__restrict__ phi, int kbeg, int kend, int S, int *err) {
  using V = V2<T>;
  constexpr int MB = pois_mb(N), NT = 512, n = N;
  using P = PoisChunk<MB>;
  extern __shared__ __align__(128) unsigned char pxraw[];
  const int ld = xline_ld<V>(n, MB), ny = c.ny, nz1 = c.nz1, xr = c.xround;
  V *xsm = reinterpret_cast<V *>(pxraw + (size_t)S * P::CH);
  uint64_t *bar = reinterpret_cast<uint64_t *>(pxraw + (size_t)S * P::CH +
                                               ((size_t)MB * ld * sizeof(V) + 15) / 16 * 16);
  const int t = threadIdx.x;
  // tiles start at an even mode (a 16-byte box origin for FP32 kr); modes
  // below kbeg are computed as zeros and not stored
  const int kb0 = kbeg & ~1, nkg = (kend - kb0) / MB + 1, ntile = nkg * (ny - 1);
  const int mine = (int)blockIdx.x < ntile ? (ntile - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int NC = (n + P::CP - 1) / P::CP, G = mine * NC;
  const size_t PV = (size_t)ny * nz1;
  int issued = 0;  // thread 0's count of chunks issued
  auto issue_upto = [&](int h_end) {
    for (; issued < h_end && issued < G; ++issued) {
      const int h = issued, sl = h % S, q = (int)blockIdx.x + (h / NC) * (int)gridDim.x;
      const int j = q / nkg + 1, k0 = kb0 + (q % nkg) * MB, tt0 = (h % NC) * P::CP;
      unsigned char *b = pxraw + (size_t)sl * P::CH;
      mbar_arrive_expect_tx(&bar[sl], P::TX);
      tma_load_3d(b, &maps.u, 2 * k0, j, tt0, &bar[sl]);
      tma_load_3d(b + P::UB, &maps.v, 2 * k0, j - 1, tt0 + 1, &bar[sl]);
      tma_load_3d(b + P::UB + P::VB, &maps.w, 2 * k0, j, tt0 + 1, &bar[sl]);
    }
  };
  if (t == 0) {
    for (int sl = 0; sl < S; ++sl) mbar_init(&bar[sl], 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (t == 0) issue_upto(S);
  const double idx = c.S[OTBL_S_IDX];
  int g = 0;
  for (int m = 0; m < mine; ++m) {
    const int q = (int)blockIdx.x + m * (int)gridDim.x;
    const int j = q / nkg + 1, k0 = kb0 + (q % nkg) * MB;
    const double idy = c.idy[j];
    for (int cc = 0; cc < NC; ++cc, ++g) {
      const int sl = g % S;
      const bool ok = mbar_wait_bounded(&bar[sl], (unsigned)((g / S) & 1), 2000000000ull);
      if (__syncthreads_or(!ok)) {
        if (t == 0) {
          atomicExch(err, OTBL_ERR_TIMEOUT);
          for (int h = g; h < issued; ++h) mbar_wait_bounded(&bar[h % S], (unsigned)((h / S) & 1), 200000000ull);
        }
        return;
      }
      if (t == 0) issue_upto(g + S);  // chunks before g are consumed
      const unsigned char *b = pxraw + (size_t)sl * P::CH;
      const double *us = reinterpret_cast<const double *>(b);
      const double *vs = reinterpret_cast<const double *>(b + P::UB);
      const double *ws = reinterpret_cast<const double *>(b + P::UB + P::VB);
      const int tt0 = cc * P::CP;
      for (int e = t; e < P::CP * MB; e += NT) {
        const int l = e % MB, pl = e / MB, tt = tt0 + pl;
        if (tt >= n) continue;
        const int k = k0 + l;
        V val;
        val.x = 0;
        val.y = 0;
        if (k >= kbeg && k <= kend) {
          const double kz = c.kaz[k];
          const double2 wv = *reinterpret_cast<const double2 *>(ws + pl * P::RW + 2 * l);
          const double2 v1 = *reinterpret_cast<const double2 *>(vs + (2 * pl + 1) * P::RW + 2 * l);
          const double2 v0 = *reinterpret_cast<const double2 *>(vs + (2 * pl) * P::RW + 2 * l);
          const double2 ua = *reinterpret_cast<const double2 *>(us + (pl + 1) * P::RW + 2 * l);
          const double2 ub = *reinterpret_cast<const double2 *>(us + pl * P::RW + 2 * l);
          double re = -kz * wv.y + (v1.x - v0.x) * idy;
          double im = kz * wv.x + (v1.y - v0.y) * idy;
          re = re + idx * (ua.x - ub.x);
          im = im + idx * (ua.y - ub.y);
          val.x = (T)rnd(re, xr);
          val.y = (T)rnd(im, xr);
        }
        const int dst = (tt & 1) ? n - 1 - (tt >> 1) : (tt >> 1);
        xsm[l * ld + xpad<V>(dst)] = val;
      }
    }
    __syncthreads();  // the tile's lines are complete and its chunks read
    if (t == 0) issue_upto(g + S);
    {
      constexpr int GL = NT / MB;
      block_fft_lines_n<-1, NT, N>(xsm + (t / GL) * ld, x.tw, t % GL, GL);
    }
    const T dnf = (T)(1.0 / (double)n);
    for (int e = t; e < n * MB; e += NT) {
      const int l = e % MB, kk = e / MB;
      const int k = k0 + l;
      if (k < kbeg || k > kend) continue;
      const V Vv = xsm[l * ld + xpad<V>(kk)], Vm = xsm[l * ld + xpad<V>(kk == 0 ? 0 : n - kk)];
      const V wq = __ldg(x.tw2 + kk);
      const V y = cadd(cmul(wq, Vv), cmul(cconj(wq), Vm));
      V out;
      out.x = (T)rnd((double)(dnf * y.x), xr);
      out.y = k == 0 ? (T)0 : (T)rnd((double)(dnf * y.y), xr);
      *reinterpret_cast<V *>(phi + (size_t)(kk + 1) * PV + (size_t)(j - 1) * nz1 + 2 * k) = out;
    }
  }
}

// backward: the tile's phi-hat row (planes 1..n, min(256, n) per box) lands
// in one of two line buffers while the other tile's FFT runs
template <typename T, int N, int MINB>
__global__ void __launch_bounds__(512, MINB) k_pois_bwd_t(DCoef c, XTabT<T> x, const __grid_constant__ PoisMaps maps,
                                                         T *__restrict__ phi, int kbeg, int kend, int *err) {
  using V = V2<T>;
  constexpr int MB = pois_mb(N), NT = 512, RW = 2 * MB, n = N;
  constexpr int BZ = n < 256 ? n : 256, NBX = (n + BZ - 1) / BZ;
  extern __shared__ __align__(128) unsigned char pxraw[];
  const int ld = xline_ld<V>(n, MB), ny = c.ny, nz1 = c.nz1, xr = c.xround;
  const unsigned TX = (unsigned)(NBX * BZ * RW * sizeof(T));
  const size_t RB = ((size_t)TX + 127) / 128 * 128;
  V *xsm = reinterpret_cast<V *>(pxraw + 2 * RB);
  uint64_t *bar = reinterpret_cast<uint64_t *>(pxraw + 2 * RB + ((size_t)MB * ld * sizeof(V) + 15) / 16 * 16);
  const CUtensorMap *mp = sizeof(T) == 8 ? &maps.phi64 : &maps.phi32;
  const int t = threadIdx.x;
  // tiles start at an even mode (a 16-byte box origin for FP32 kr); modes
  // below kbeg are computed as zeros and not stored
  const int kb0 = kbeg & ~1, nkg = (kend - kb0) / MB + 1, ntile = nkg * (ny - 1);
  const int mine = (int)blockIdx.x < ntile ? (ntile - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const size_t PV = (size_t)ny * nz1;
  auto issue = [&](int m) {
    const int q = (int)blockIdx.x + m * (int)gridDim.x;
    const int j = q / nkg + 1, k0 = kb0 + (q % nkg) * MB;
    unsigned char *b = pxraw + (size_t)(m & 1) * RB;
    mbar_arrive_expect_tx(&bar[m & 1], TX);
    for (int z = 0; z < NBX; ++z)
      tma_load_3d(b + (size_t)z * BZ * RW * sizeof(T), mp, 2 * k0, j - 1, 1 + z * BZ, &bar[m & 1]);
  };
  if (t == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (t == 0 && mine > 0) issue(0);
  for (int m = 0; m < mine; ++m) {
    const int q = (int)blockIdx.x + m * (int)gridDim.x;
    const int j = q / nkg + 1, k0 = kb0 + (q % nkg) * MB;
    // the other buffer was read by the previous tile's pre-step, before its FFT
    if (t == 0 && m + 1 < mine) issue(m + 1);
    const bool ok = mbar_wait_bounded(&bar[m & 1], (unsigned)((m >> 1) & 1), 2000000000ull);
    if (__syncthreads_or(!ok)) {
      if (t == 0) {
        atomicExch(err, OTBL_ERR_TIMEOUT);
        mbar_wait_bounded(&bar[m & 1], (unsigned)((m >> 1) & 1), 200000000ull);
        if (m + 1 < mine) mbar_wait_bounded(&bar[(m + 1) & 1], (unsigned)(((m + 1) >> 1) & 1), 200000000ull);
      }
      return;
    }
    const T *raw = reinterpret_cast<const T *>(pxraw + (size_t)(m & 1) * RB);
    for (int e = t; e < n * MB; e += NT) {
      const int l = e % MB, kk = e / MB;
      const int k = k0 + l;
      V val;
      val.x = 0;
      val.y = 0;
      if (k >= kbeg && k <= kend) {
        const V qv = *reinterpret_cast<const V *>(raw + kk * RW + 2 * l);
        V Y, Ym;
        Y.x = (T)rnd((double)qv.x, xr);
        Y.y = (T)rnd((double)qv.y, xr);
        Ym.x = 0;
        Ym.y = 0;
        if (kk > 0) {
          const V qm = *reinterpret_cast<const V *>(raw + (n - kk) * RW + 2 * l);
          Ym.x = (T)rnd((double)qm.x, xr);
          Ym.y = (T)rnd((double)qm.y, xr);
        }
        V d;  // Y - i Ym
        d.x = Y.x + Ym.y;
        d.y = Y.y - Ym.x;
        val = cmul(cconj(__ldg(x.tw2 + kk)), d);
      }
      xsm[l * ld + xpad<V>(kk)] = val;
    }
    __syncthreads();
    {
      constexpr int GL = NT / MB;
      block_fft_lines_n<1, NT, N>(xsm + (t / GL) * ld, x.tw, t % GL, GL);
    }
    for (int e = t; e < n * MB; e += NT) {
      const int l = e % MB, tt = e / MB;
      const int k = k0 + l;
      if (k < kbeg || k > kend) continue;
      const V Vv = xsm[l * ld + xpad<V>((tt & 1) ? n - 1 - (tt >> 1) : (tt >> 1))];
      V out;
      out.x = (T)rnd((double)((T)0.5 * Vv.x), xr);
      out.y = k == 0 ? (T)0 : (T)rnd((double)((T)0.5 * Vv.y), xr);
      *reinterpret_cast<V *>(phi + (size_t)(tt + 1) * PV + (size_t)(j - 1) * nz1 + 2 * k) = out;
    }
  }
}

// projection, pois.f90:144-162; one thread per (i >= 2, j, spanwise mode k),
// the mode's two components kr = 2k, 2k+1 together (16-byte velocity and
// 8- or 16-byte phi and p accesses; the w update of one component takes the
// other component's phi, pof = +-1 in the reference). phi holds the modes
// 2k < kr_split in FP64 (phi64) and the others in FP32 (phi32, the mixed
// path's higher spanwise modes); the update is FP64, operation for operation
// the reference's per-component statements.
template <typename TP>
__global__ void __launch_bounds__(256) k_project(DCoef c, const DState *st, const double *__restrict__ phi64,
                                                 const float *__restrict__ phi32, int kr_split, double *u,
                                                 double *v, double *w, TP *p) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = c.nx, ny = c.ny, nz1 = c.nz1;
  if (2 * k >= nz1) return;
  const int j = blockIdx.y + 1, i = blockIdx.z + 2;
  const size_t PU = (size_t)(ny + 1) * nz1, PV = (size_t)ny * nz1;
  const double kz = c.kaz[k];
  const size_t base = (size_t)(i - 1) * PV + 2 * k;  // phi(j, i) at base + (j-1)*nz1
  const bool lo = 2 * k < kr_split;
  auto F = [&](size_t off) -> double2 {
    if (lo) return *reinterpret_cast<const double2 *>(phi64 + base + off);
    const float2 f = *reinterpret_cast<const float2 *>(phi32 + base + off);
    return make_double2((double)f.x, (double)f.y);
  };
  using VP = V2<TP>;
  double2 f1 = make_double2(0.0, 0.0);
  if (j <= ny - 1) f1 = F((size_t)(j - 1) * nz1);
  if (j >= 2) {
    const double2 fm = F((size_t)(j - 2) * nz1);
    VP *pq = reinterpret_cast<VP *>(p + (size_t)(i - 1) * PV + (size_t)(j - 1) * nz1 + 2 * k);
    const VP p0 = *pq;
    VP p1;
    p1.x = (TP)(st->varstep * fm.x + (double)p0.x);
    p1.y = (TP)(st->varstep * fm.y + (double)p0.y);
    *pq = p1;
    double2 *wq = reinterpret_cast<double2 *>(w + (size_t)(i - 1) * PU + (size_t)(j - 1) * nz1 + 2 * k);
    double2 wv = *wq;
    wv.x = wv.x - -kz * fm.y;
    wv.y = wv.y - kz * fm.x;
    *wq = wv;
    if (j <= ny - 1) {
      const double dy = c.idyy[j - 1];
      double2 *vq = reinterpret_cast<double2 *>(v + (size_t)(i - 1) * PV + (size_t)(j - 1) * nz1 + 2 * k);
      double2 vv = *vq;
      vv.x = vv.x - dy * (f1.x - fm.x);
      vv.y = vv.y - dy * (f1.y - fm.y);
      *vq = vv;
    }
  }
  if (j <= ny - 1 && i <= nx - 1) {
    const double2 f2 = F(PV + (size_t)(j - 1) * nz1);
    const double idxx = c.S[OTBL_S_IDXX];
    double2 *uq = reinterpret_cast<double2 *>(u + (size_t)(i - 1) * PU + (size_t)j * nz1 + 2 * k);
    double2 uv = *uq;
    uv.x = uv.x - idxx * (f2.x - f1.x);
    uv.y = uv.y - idxx * (f2.y - f1.y);
    *uq = uv;
  }
}

// ---------------------------------------------------------------------------
// standalone pieces of the path
// ---------------------------------------------------------------------------
// planes [nx][np] <-> pencils [np][nx] (change.f90 chp2x / chx2p), rounded
__global__ void k_transpose(const double *__restrict__ in, double *__restrict__ out, int rows, int cols, int xr) {
  __shared__ double tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int row = by + r, col = bx + threadIdx.x;
    if (row < rows && col < cols) tile[r][threadIdx.x] = in[(size_t)row * cols + col];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int orow = bx + r, ocol = by + threadIdx.x;
    if (orow < cols && ocol < rows) out[(size_t)orow * rows + ocol] = rnd(tile[threadIdx.x][r], xr);
  }
}

__global__ void __launch_bounds__(128) k_fourxz(DCoef c, ZTab z, double *fou, double *phys, int iopt,
                                                int nlines) {
  extern __shared__ double2 sm[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int l = blockIdx.x * 4 + wid;
  if (l >= nlines) return;
  const int M = z.M;
  double2 *A = sm + (size_t)wid * M;
  double *ph = phys + (size_t)l * (z.nz + 2);
  double *fo = fou + (size_t)l * c.nz1;
  if (iopt < 0) {
    for (int t = lane; t < M; t += 32) A[t] = make_double2(ph[2 * t], ph[2 * t + 1]);
    __syncwarp();
    line_r2c(z, A, fo, lane);
  } else {
    line_c2r(z, fo, A, lane);
    for (int t = lane; t < M; t += 32) {
      ph[2 * t] = A[t].x;
      ph[2 * t + 1] = A[t].y;
    }
    for (int t = lane; t < 2; t += 32) ph[z.nz + t] = 0.0;
  }
}

// cosftx on pencils c(nx, nlines), elements 2..nx; two real lines per CTA
__global__ void __launch_bounds__(256) k_cosftx(XTab x, double *cp, int nx, int nlines, int iopt) {
  extern __shared__ double2 xsm[];
  const int n = x.n;
  const int l0 = blockIdx.x * 2;
  double *la = cp + (size_t)l0 * nx + 1;
  double *lb = (l0 + 1 < nlines) ? cp + (size_t)(l0 + 1) * nx + 1 : nullptr;
  if (iopt < 0) {
    for (int tt = threadIdx.x; tt < n; tt += 256) {
      const int dst = (tt & 1) ? n - 1 - (tt >> 1) : (tt >> 1);
      xsm[dst] = make_double2(la[tt], lb ? lb[tt] : 0.0);
    }
    __syncthreads();
    block_fft<-1, 1>(xsm, n, x.tw);
    const double dnf = 1.0 / (double)n;
    for (int kk = threadIdx.x; kk < n; kk += 256) {
      const double2 V = xsm[kk], Vm = xsm[kk == 0 ? 0 : n - kk];
      const double2 wq = __ldg(x.tw2 + kk);
      const double2 y = cadd(cmul(wq, V), cmul(cconj(wq), Vm));
      la[kk] = dnf * y.x;
      if (lb) lb[kk] = dnf * y.y;
    }
  } else {
    for (int kk = threadIdx.x; kk < n; kk += 256) {
      const double2 Y = make_double2(la[kk], lb ? lb[kk] : 0.0);
      const double2 Ym = kk > 0 ? make_double2(la[n - kk], lb ? lb[n - kk] : 0.0) : make_double2(0.0, 0.0);
      const double2 d = make_double2(Y.x + Ym.y, Y.y - Ym.x);
      xsm[kk] = cmul(cconj(__ldg(x.tw2 + kk)), d);
    }
    __syncthreads();
    block_fft<1, 1>(xsm, n, x.tw);
    for (int tt = threadIdx.x; tt < n; tt += 256) {
      const double2 V = xsm[(tt & 1) ? n - 1 - (tt >> 1) : (tt >> 1)];
      la[tt] = 0.5 * V.x;
      if (lb) lb[tt] = 0.5 * V.y;
    }
  }
}

__global__ void k_twiddles(double2 *tw, int n, double2 *tw2, int n2, int mode2) {
  // tw[t] = exp(-2 pi i t/n); tw2[t] = exp(-2 pi i t/n2) (mode2 = 0) or
  // exp(-i pi t/(2 n2)) (mode2 = 1), t < count
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) {
    double s, co;
    sincospi(-2.0 * (double)t / (double)n, &s, &co);
    tw[t] = make_double2(co, s);
  }
  if (tw2 && t < n2) {
    double s, co;
    if (mode2 == 0)
      sincospi(-2.0 * (double)t / (double)(2 * n2), &s, &co);
    else
      sincospi(-(double)t / (2.0 * (double)n2), &s, &co);
    tw2[t] = make_double2(co, s);
  }
}

#ifndef OTBL_POIS_NT
#define OTBL_POIS_NT 512
#endif
constexpr int POIS_NT_BIG = OTBL_POIS_NT;

// FP32 copy of an FP64 table (mixed path)
__global__ void k_round_f32(const double *in, float *out, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[t] = (float)in[t];
}

cudaError_t launch_round_f32(otbl_ctx *c, const double *in, float *out, size_t n) {
  k_round_f32<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(in, out, (int)n);
  c->launches += 1;
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// launch wrappers
// ---------------------------------------------------------------------------
const char *const kProfNames[PK_COUNT] = {"interpx", "interpy", "products", "difvisx", "dt",
                                          "genflu", "final", "outflow", "pois_fwd", "pois_solve",
                                          "pois_bwd", "project", "misc"};

static cudaEvent_t prof_event(otbl_ctx *c) {
  if (!c->prof_pool.empty()) {
    cudaEvent_t e = c->prof_pool.back();
    c->prof_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

void prof_begin(otbl_ctx *c, int kind) {
  if (!c->prof_on) return;
  otbl_ctx::ProfRec r;
  r.kind = kind;
  r.a = prof_event(c);
  r.b = prof_event(c);
  cudaEventRecord(r.a, c->stream);
  c->prof.push_back(r);
  c->prof_open = (int)c->prof.size() - 1;
}

void prof_end(otbl_ctx *c) {
  if (!c->prof_on || c->prof_open < 0) return;
  cudaEventRecord(c->prof[c->prof_open].b, c->stream);
  c->prof_open = -1;
}
static inline ZTab ztab(otbl_ctx *c) {
  ZTab z;
  z.tw = reinterpret_cast<const double2 *>(c->w.twz);
  z.tw2 = reinterpret_cast<const double2 *>(c->w.twz2);
  z.M = c->cfg.nz / 2;
  z.nz = c->cfg.nz;
  z.nz2 = c->dc.nz2;
  return z;
}
static inline XTab xtab(otbl_ctx *c) {
  XTab x;
  x.tw = reinterpret_cast<const double2 *>(c->w.twx);
  x.tw2 = reinterpret_cast<const double2 *>(c->w.twx2);
  x.n = c->cfg.nx - 1;
  return x;
}
static inline XTabT<float> xtabf(otbl_ctx *c) {
  XTabT<float> x;
  x.tw = reinterpret_cast<const float2 *>(c->w.twxf);
  x.tw2 = reinterpret_cast<const float2 *>(c->w.twx2f);
  x.n = c->cfg.nx - 1;
  return x;
}

cudaError_t launch_twiddles(otbl_ctx *c) {
  const int M = c->cfg.nz / 2, n = c->cfg.nx - 1;
  k_twiddles<<<(M + 255) / 256, 256, 0, c->stream>>>(reinterpret_cast<double2 *>(c->w.twz), M,
                                                     reinterpret_cast<double2 *>(c->w.twz2), M, 0);
  k_twiddles<<<(n + 255) / 256, 256, 0, c->stream>>>(reinterpret_cast<double2 *>(c->w.twx), n,
                                                     reinterpret_cast<double2 *>(c->w.twx2), n, 1);
  c->launches += 2;
  if (c->mixed) {
    k_round_f32<<<(2 * M + 255) / 256, 256, 0, c->stream>>>(c->w.twz, c->w.twzf, 2 * M);
    k_round_f32<<<(2 * M + 255) / 256, 256, 0, c->stream>>>(c->w.twz2, c->w.twz2f, 2 * M);
    k_round_f32<<<(2 * n + 255) / 256, 256, 0, c->stream>>>(c->w.twx, c->w.twxf, 2 * n);
    k_round_f32<<<(2 * n + 255) / 256, 256, 0, c->stream>>>(c->w.twx2, c->w.twx2f, 2 * n);
    c->launches += 4;
  }
  return cudaGetLastError();
}

cudaError_t launch_reset_max(otbl_ctx *c) {
  k_reset_max<<<(c->cfg.ny + 1 + 255) / 256, 256, 0, c->stream>>>(c->st, c->w.vm_bits, c->cfg.ny);
  c->launches += 1;
  return cudaGetLastError();
}

template <typename T>
static cudaError_t products_t(otbl_ctx *c, int setstep, int part, const ZTabT<T> &z) {
  ProdArgs<T> a;
  a.u = c->f[OTBL_F_U];
  a.v = c->f[OTBL_F_V];
  a.w = c->f[OTBL_F_W];
  a.ux = static_cast<const T *>(c->w.ux);
  a.vx = static_cast<const T *>(c->w.vx);
  a.wx = static_cast<const T *>(c->w.wx);
  a.uy = static_cast<const T *>(c->w.uy);
  a.wy = static_cast<const T *>(c->w.wy);
  a.vy = static_cast<const T *>(c->w.vy);
  a.uu = static_cast<T *>(c->w.uu);
  a.uw = static_cast<T *>(c->w.uw);
  a.uv = static_cast<T *>(c->w.uv);
  a.vw = static_cast<T *>(c->w.vw);
  a.vv = static_cast<T *>(c->w.vv);
  a.ww = static_cast<T *>(c->w.ww);
  a.vm_bits = c->w.vm_bits;
  a.st = c->st;
  a.setstep = setstep;
  const int M = c->cfg.nz / 2;
  // part 0: all planes, rows 1..ny+1; part 2: all planes, rows 1..ny;
  // part 1: planes 2..nx-1, rows 1..ny
  const dim3 g((c->cfg.ny + (part == 0 ? 1 : 0) + 3) / 4, c->cfg.nx - (part == 1 ? 2 : 0));
  // the register-pipelined transforms for M = 32..256; other M (and
  // OTBL_PRODUCTS_SMEM=1) the shared-memory kernel
  if ((M == 32 || M == 64 || M == 128 || M == 256) && !getenv("OTBL_PRODUCTS_SMEM")) {
    const size_t smem = (size_t)4 * (M + M / 8) * sizeof(V2<T>);
    auto go = [&](auto k0, auto k1, auto k2) {
      if (part == 0)
        k0<<<g, 128, smem, c->stream>>>(c->dc, z, a);
      else if (part == 1)
        k1<<<g, 128, smem, c->stream>>>(c->dc, z, a);
      else
        k2<<<g, 128, smem, c->stream>>>(c->dc, z, a);
    };
    if (M == 256)
      go(k_products_r<256, T, 0>, k_products_r<256, T, 1>, k_products_r<256, T, 2>);
    else if (M == 128)
      go(k_products_r<128, T, 0>, k_products_r<128, T, 1>, k_products_r<128, T, 2>);
    else if (M == 64)
      go(k_products_r<64, T, 0>, k_products_r<64, T, 1>, k_products_r<64, T, 2>);
    else
      go(k_products_r<32, T, 0>, k_products_r<32, T, 1>, k_products_r<32, T, 2>);
  } else {
    const size_t smem = (size_t)4 * 3 * M * sizeof(V2<T>);
    auto k = part == 0 ? k_products<T, 0> : (part == 1 ? k_products<T, 1> : k_products<T, 2>);
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k<<<g, 128, smem, c->stream>>>(c->dc, z, a);
  }
  return cudaGetLastError();
}

cudaError_t launch_products(otbl_ctx *c, int setstep, int part) {
  if (part == 1 && c->cfg.nx <= 2) return cudaSuccess;  // no interior planes
  prof_begin(c, PK_PRODUCTS);
  cudaError_t e;
  if (c->mixed) {
    ZTabT<float> z;
    z.tw = reinterpret_cast<const float2 *>(c->w.twzf);
    z.tw2 = reinterpret_cast<const float2 *>(c->w.twz2f);
    z.M = c->cfg.nz / 2;
    z.nz = c->cfg.nz;
    z.nz2 = c->dc.nz2;
    e = products_t<float>(c, setstep, part, z);
  } else {
    e = products_t<double>(c, setstep, part, ztab(c));
  }
  prof_end(c);
  c->launches += 1;
  return e;
}

cudaError_t launch_dt(otbl_ctx *c, int m, int setstep) {
  prof_begin(c, PK_DT);
  k_dt<<<1, 64, 0, c->stream>>>(c->dc, c->st, c->w.vm_bits, c->w.fac_u, c->w.fac_v, m, setstep,
                                c->cfg.dt_mode, c->cfg.dt_fixed);
  c->launches += 1;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = launch_tail_rows(c);
  prof_end(c);
  return e;
}

cudaError_t launch_genflu(otbl_ctx *c, int tail) {
  GenArgs a;
  a.u = c->f[OTBL_F_U];
  a.v = c->f[OTBL_F_V];
  a.w = c->f[OTBL_F_W];
  a.rhsupa = c->f[OTBL_F_RHSUPA];
  a.rhsvpa = c->f[OTBL_F_RHSVPA];
  a.rhswpa = c->f[OTBL_F_RHSWPA];
  a.rhs32 = c->f32[OTBL_F_RHSUPA];
  a.u0 = c->u0;
  a.v0 = c->v0;
  a.um = c->um;
  a.tab = c->w.gf;
  DState *st = c->st;
  a.dt = &st->dt;
  a.tiempo = &st->tiempo;
  a.timeinit = &st->timeinit;
  a.timec = &st->timec;
  a.utauout = &st->utauout;
  a.rthout = &st->rthout;
  a.dout = &st->dout;
  a.gamma1 = &st->gamma1;
  a.gamma2 = &st->gamma2;
  a.err = &st->err;
  a.err_code = OTBL_DEVERR_GENFLU_GRID;
  a.tail = tail;
  prof_begin(c, PK_GENFLU);
  const cudaError_t e = genflu_launch(c, a);
  prof_end(c);
  return e;
}

// ---------------------------------------------------------------------------
// genflu on caller-owned buffers, with its table scratch in a static device
// array instead of a context allocation. Callers that cannot allocate
// device memory at call time use it: a host that owns the fields in its own
// device allocations and has handed the rest of HBM to its own pool has no
// room for a scratch buffer mid-run, and a cudaMalloc/cudaFree pair would
// also synchronise the device inside its stream-ordered time loop.
//
// The array is part of this module's data, so it comes into existence when
// the module is loaded on a device; the first call on each device looks its
// address up (cudaGetSymbolAddress, which may load the module) and caches
// it. Nothing in it needs to start at zero: k_genflu_tab writes every table
// entry that k_genflu_cols reads, earlier on the same stream. All calls on one device
// share the one array, so two calls whose launches overlap (different
// streams, contexts or host threads without ordering between them) race.
// ---------------------------------------------------------------------------
static __device__ __align__(256) double g_genflu_scratch[OTBL_GENFLU_SCRATCH_MAX];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
double *g_scratch_addr[kMaxDevices] = {};
}  // namespace

// The caller has made `device` current.
cudaError_t genflu_scratch_addr(int device, double **p) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_addr[device]) {
    void *q = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&q, g_genflu_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[device] = static_cast<double *>(q);
  }
  *p = g_scratch_addr[device];
  return cudaSuccess;
}

cudaError_t launch_genflu_noalloc(otbl_ctx *c, double *wk, double *u, double *v, double *w, const double *u0,
                                  const double *v0, double *um, double *scal, int *err) {
  GenArgs a;
  a.u = u;
  a.v = v;
  a.w = w;
  a.rhsupa = a.rhsvpa = a.rhswpa = nullptr;  // only touched with tail = 1
  a.rhs32 = 0;
  a.u0 = u0;
  a.v0 = v0;
  a.um = um;
  a.tab = wk;
  a.dt = scal + OTBL_GF_DT;
  a.tiempo = scal + OTBL_GF_TIEMPO;
  a.timeinit = scal + OTBL_GF_TIMEINIT;
  a.timec = scal + OTBL_GF_TIMEC;
  a.utauout = scal + OTBL_GF_UTAUOUT;
  a.rthout = scal + OTBL_GF_RTHOUT;
  a.dout = scal + OTBL_GF_DOUT;
  a.gamma1 = scal + OTBL_GF_GAMMA1;
  a.gamma2 = scal + OTBL_GF_GAMMA2;
  a.err = err;
  a.err_code = OTBL_ERR_NAN;
  a.tail = 0;
  return genflu_launch(c, a);
}

cudaError_t launch_outflow(otbl_ctx *c) {
  prof_begin(c, PK_OUTFLOW);
  if (c->f32[OTBL_F_RHSUPA])
    k_outflow<float><<<1, 256, 0, c->stream>>>(c->dc, c->f[OTBL_F_U], c->f[OTBL_F_V],
                                               reinterpret_cast<float *>(c->f[OTBL_F_RHSUPA]));
  else
    k_outflow<double><<<1, 256, 0, c->stream>>>(c->dc, c->f[OTBL_F_U], c->f[OTBL_F_V], c->f[OTBL_F_RHSUPA]);
  prof_end(c);
  c->launches += 1;
  return cudaGetLastError();
}

// 3D map [planes][rows][nz1] of esz-byte elements, boxes of bx x by x bz
static bool encode_pois(CUtensorMap *m, const void *base, size_t esz, int nz1, int rows, int planes, int bx, int by,
                        int bz) {
  auto fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
  if (!fn || !base || ((uintptr_t)base) % 16 != 0 || ((size_t)nz1 * esz) % 16 != 0 || ((size_t)bx * esz) % 16 != 0)
    return false;
  const cuuint64_t dims[3] = {(cuuint64_t)nz1, (cuuint64_t)rows, (cuuint64_t)planes};
  const cuuint64_t strides[2] = {(cuuint64_t)nz1 * esz, (cuuint64_t)rows * nz1 * esz};
  const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz};
  const cuuint32_t es[3] = {1, 1, 1};
  const CUtensorMapDataType dt = esz == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  return fn(m, dt, 3, const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool build_pois_maps(otbl_ctx *c) {
  const int nx = c->cfg.nx, ny = c->cfg.ny, nz1 = c->dc.nz1, n = nx - 1;
  const int MB = pois_mb(n), CP = MB >= 8 ? 64 : 128, BZ = std::min(256, n);
  c->pmaps_vel = encode_pois(&c->pmaps.u, c->f[OTBL_F_U], 8, nz1, ny + 1, nx, 2 * MB, 1, CP + 1) &&
                 encode_pois(&c->pmaps.v, c->f[OTBL_F_V], 8, nz1, ny, nx, 2 * MB, 2, CP) &&
                 encode_pois(&c->pmaps.w, c->f[OTBL_F_W], 8, nz1, ny + 1, nx, 2 * MB, 1, CP);
  c->pmaps_phi64 = encode_pois(&c->pmaps.phi64, c->w.s2, 8, nz1, ny, nx, 2 * MB, 1, BZ);
  c->pmaps_phi32 = c->mixed && encode_pois(&c->pmaps.phi32, c->w.s3, 4, nz1, ny, nx, 2 * MB, 1, BZ);
  return c->pmaps_vel && c->pmaps_phi64;
}

// SMs of the current device (the persistent x-DCT grids; any grid size is
// correct, the count only spreads the tiles), cached per device ordinal
static int sm_count() {
  constexpr int kDevs = 64;
  static int nsm[kDevs] = {0};  // the same value if two host threads race
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevs) return 148;
  if (nsm[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    nsm[dev] = n;
  }
  return nsm[dev];
}

// The TMA-fed x-DCT pass when its descriptors exist and n is 256, 512, 1024
// or 2048; false leaves the pass to pois_xdct's one-shot kernels
// (OTBL_POIS_ONESHOT=1 forces them).
template <typename T>
static bool pois_xdct_t(otbl_ctx *c, bool fwd, T *phi, int kbeg, int kend) {
  constexpr bool F64 = sizeof(T) == 8;
  const int ny = c->cfg.ny, n = c->cfg.nx - 1, MB = pois_mb(n);
  if (getenv("OTBL_POIS_ONESHOT")) return false;
  if (fwd && !c->pmaps_vel) return false;
  if (!fwd && !(F64 ? c->pmaps_phi64 : c->pmaps_phi32)) return false;
  if (!fwd && !F64 && MB < 2) return false;
  if ((void *)phi != (F64 ? (void *)c->w.s2 : (void *)c->w.s3)) return false;
  using V = V2<T>;
  const size_t xs = ((size_t)MB * xline_ld<V>(n, MB) * sizeof(V) + 15) / 16 * 16;
  const int ntile = ((kend - (kbeg & ~1)) / MB + 1) * (ny - 1);
  const int smax = 232448;  // dynamic shared memory per CTA (227 KB)
  XTabT<T> xt;
  if constexpr (F64)
    xt = xtab(c);
  else
    xt = xtabf(c);
  int *err = &c->st->err;
  if (fwd) {
    auto go = [&](auto kern, int ch) {
      const int S = std::min(6, (int)((smax - xs - 64) / ch));
      if (S < 2) return false;
      const size_t smem = (size_t)S * ch + xs + 8 * (size_t)S;
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      kern<<<std::min(ntile, sm_count()), 512, smem, c->stream>>>(c->dc, xt, c->pmaps, phi, kbeg, kend, S, err);
      return true;
    };
    switch (n) {
      case 256: return go(k_pois_fwd_t<T, 256>, PoisChunk<pois_mb(256)>::CH);
      case 512: return go(k_pois_fwd_t<T, 512>, PoisChunk<pois_mb(512)>::CH);
      case 1024: return go(k_pois_fwd_t<T, 1024>, PoisChunk<pois_mb(1024)>::CH);
      case 2048: return go(k_pois_fwd_t<T, 2048>, PoisChunk<pois_mb(2048)>::CH);
      default: return false;
    }
  }
  const int BZ = std::min(256, n), NBX = (n + BZ - 1) / BZ;
  const size_t rb = ((size_t)NBX * BZ * 2 * MB * sizeof(T) + 127) / 128 * 128;
  const size_t smem = 2 * rb + xs + 16;
  if (smem > (size_t)smax) return false;
  constexpr int MINB = F64 ? 1 : 2;
  auto go = [&](auto kern) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int per = smem * 2 + 2048 <= 233472 ? MINB : 1;  // CTAs per SM that fit
    kern<<<std::min(ntile, per * sm_count()), 512, smem, c->stream>>>(c->dc, xt, c->pmaps, phi, kbeg, kend, err);
    return true;
  };
  switch (n) {
    case 256: return go(k_pois_bwd_t<T, 256, MINB>);
    case 512: return go(k_pois_bwd_t<T, 512, MINB>);
    case 1024: return go(k_pois_bwd_t<T, 1024, MINB>);
    case 2048: return go(k_pois_bwd_t<T, 2048, MINB>);
    default: return false;
  }
}

// One x-DCT pass (forward: divergence + DCT-II; backward: DCT-III) over the
// spanwise modes kbeg..kend in T, MB modes per CTA.
template <typename T>
static void pois_xdct(otbl_ctx *c, bool fwd, T *phi, int kbeg, int kend) {
  if (kend < kbeg) return;
  if (pois_xdct_t<T>(c, fwd, phi, kbeg, kend)) {
    c->launches += 1;
    return;
  }
  const int ny = c->cfg.ny, n = c->cfg.nx - 1;
  const int MB = pois_mb(n);
  const size_t smem = (size_t)MB * xline_ld<V2<T>>(n, MB) * sizeof(V2<T>);
  const dim3 gx((kend - kbeg + 1 + MB - 1) / MB, ny - 1);
  // threads per CTA: 512 when the CTA holds 2048-4096 points (fewer items
  // and registers per thread, the same barriers), else 256
  const int NT = n * MB >= 2048 ? POIS_NT_BIG : 256;
  XTabT<T> xt;
  if constexpr (std::is_same<T, double>::value)
    xt = xtab(c);
  else
    xt = xtabf(c);
  auto go = [&](auto kf, auto kb) {
    if (fwd) {
      cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      kf<<<gx, NT, smem, c->stream>>>(c->dc, xt, c->f[OTBL_F_U], c->f[OTBL_F_V], c->f[OTBL_F_W], phi, kbeg, kend);
    } else {
      cudaFuncSetAttribute(kb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      kb<<<gx, NT, smem, c->stream>>>(c->dc, xt, phi, kbeg, kend);
    }
  };
#define OTBL_POIS_GO(MBV, NTV) go(k_pois_fwd<T, MBV, NTV>, k_pois_bwd<T, MBV, NTV>)
  if (MB == 8)
    NT == 512 ? OTBL_POIS_GO(8, 512) : OTBL_POIS_GO(8, 256);
  else if (MB == 4)
    NT == 512 ? OTBL_POIS_GO(4, 512) : OTBL_POIS_GO(4, 256);
  else if (MB == 2)
    NT == 512 ? OTBL_POIS_GO(2, 512) : OTBL_POIS_GO(2, 256);
  else
    NT == 512 ? OTBL_POIS_GO(1, 512) : OTBL_POIS_GO(1, 256);
#undef OTBL_POIS_GO
  c->launches += 1;
}

// pois.f90:11-189. FP64 path: every spanwise mode in FP64 on phi = s2. Mixed
// path: modes k < pois_klo in FP64 (phi64 = s2), the others in FP32 (phi32 =
// s3, free between the rhsp tails); the projection is FP64 on both.
cudaError_t launch_pois(otbl_ctx *c, int m) {
  (void)m;  // varstep for substep m was set by k_dt
  const int nz2 = c->dc.nz2, ny = c->cfg.ny, nx = c->cfg.nx, nz1 = c->dc.nz1;
  double *phi64 = c->w.s2;
  float *phi32 = c->mixed ? reinterpret_cast<float *>(c->w.s3) : nullptr;
  const int klo = c->mixed ? std::min(c->pois_klo, nz2 + 1) : nz2 + 1;  // modes 0..klo-1 in FP64
  const int kr_split = 2 * klo;
  prof_begin(c, PK_POIS_FWD);
  pois_xdct<double>(c, true, phi64, 0, klo - 1);
  if (klo <= nz2) pois_xdct<float>(c, true, phi32, klo, nz2);
  prof_end(c);
  cudaError_t e = launch_pois_solve(c, phi64, phi32, kr_split);
  if (e != cudaSuccess) return e;
  prof_begin(c, PK_POIS_BWD);
  pois_xdct<double>(c, false, phi64, 0, klo - 1);
  if (klo <= nz2) pois_xdct<float>(c, false, phi32, klo, nz2);
  prof_end(c);
  // one thread per complex mode: 170 modes of nz = 512 in one CTA of 192
  const int nmodes = nz1 / 2, pt = std::min(256, (nmodes + 31) / 32 * 32);
  dim3 gp((nmodes + pt - 1) / pt, ny, nx - 1);
  prof_begin(c, PK_PROJECT);
  if (c->f32[OTBL_F_P])
    k_project<float><<<gp, pt, 0, c->stream>>>(c->dc, c->st, phi64, phi32, kr_split, c->f[OTBL_F_U],
                                                c->f[OTBL_F_V], c->f[OTBL_F_W],
                                                reinterpret_cast<float *>(c->f[OTBL_F_P]));
  else
    k_project<double><<<gp, pt, 0, c->stream>>>(c->dc, c->st, phi64, phi32, kr_split, c->f[OTBL_F_U],
                                                 c->f[OTBL_F_V], c->f[OTBL_F_W], c->f[OTBL_F_P]);
  prof_end(c);
  c->launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_boun_all(otbl_ctx *c) {
  dim3 g((c->dc.nz1 + 127) / 128, c->cfg.nx);
  k_boun<<<g, 128, 0, c->stream>>>(c->dc, c->f[OTBL_F_U], c->f[OTBL_F_V], c->f[OTBL_F_W]);
  c->launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_energies(otbl_ctx *c) {
  k_energies<<<1, 1024, 0, c->stream>>>(c->dc, c->st, c->f[OTBL_F_U], c->f[OTBL_F_V], c->f[OTBL_F_W]);
  c->launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_tiempo(otbl_ctx *c) {
  k_tiempo<<<1, 32, 0, c->stream>>>(c->st);
  c->launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_chp2x(otbl_ctx *c, const double *in, double *out, int jee, int to_pen) {
  const int np = c->dc.nz1 * jee, nx = c->cfg.nx;
  const int rows = to_pen ? nx : np, cols = to_pen ? np : nx;
  dim3 g((cols + 31) / 32, (rows + 31) / 32), b(32, 8);
  k_transpose<<<g, b, 0, c->stream>>>(in, out, rows, cols, c->dc.xround);
  c->launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_fourxz(otbl_ctx *c, double *fou, double *phys, int iopt, int nlines) {
  const int M = c->cfg.nz / 2;
  const size_t smem = (size_t)4 * M * sizeof(double2);
  k_fourxz<<<(nlines + 3) / 4, 128, smem, c->stream>>>(c->dc, ztab(c), fou, phys, iopt, nlines);
  c->launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_cosftx(otbl_ctx *c, double *cp, int nlines, int iopt) {
  const int n = c->cfg.nx - 1;
  const size_t smem = (size_t)n * sizeof(double2);
  k_cosftx<<<(nlines + 1) / 2, 256, smem, c->stream>>>(xtab(c), cp, c->cfg.nx, nlines, iopt);
  c->launches += 1;
  return cudaGetLastError();
}

}  // namespace otbl
