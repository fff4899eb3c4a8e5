// Hand-written FFT building blocks for the substep (sm_100a), in FP64
// (double2) or, on the mixed-precision path, FP32 (float2).
//
// Spanwise transforms (ffts.f90:27-67 fourxz): a real line of nz points is
// handled as a complex line of M = nz/2 points (even/odd packing) and
// transformed by one warp with a Stockham autosort FFT in shared memory
// (radix 8/4/2 passes, each pass: registers <- smem, small DFT, smem <-
// registers). Streamwise cosine transforms (ffts.f90:147-181 cosftx) use the
// same Stockham passes with a whole CTA over a length nx-1 complex line
// (radices 8/4/2/3/5), with Makhoul's permutation turning a DCT-II/III of
// length n into one complex FFT of length n.
//
// Twiddles come from tables tw[t] = exp(-2 pi i t / N) built on the device by
// sincospi at context creation.
#pragma once
#include <cuda_runtime.h>

#include <type_traits>

namespace otbl {

// complex type of a real type: V2<double> = double2, V2<float> = float2
template <typename T>
struct Vec2;
template <>
struct Vec2<double> {
  using type = double2;
};
template <>
struct Vec2<float> {
  using type = float2;
};
template <typename T>
using V2 = typename Vec2<T>::type;

// complex arithmetic on double2 (FP64 path) and float2 (mixed path)
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// multiply by i*s (s = +1 or -1)
template <typename V>
__device__ __forceinline__ V cmul_i(V a, int s) {
  V r;
  r.x = s > 0 ? -a.y : a.y;
  r.y = s > 0 ? a.x : -a.x;
  return r;
}
// a*(x, y) for a real scalar
template <typename V, typename S>
__device__ __forceinline__ V cscale(S a, V v) {
  V r;
  r.x = a * v.x;
  r.y = a * v.y;
  return r;
}
template <typename V>
__device__ __forceinline__ V cmake(decltype(V{}.x) x, decltype(V{}.x) y) {
  V r;
  r.x = x;
  r.y = y;
  return r;
}

template <int SIGN, typename V>
__device__ __forceinline__ void dft4(V &t0, V &t1, V &t2, V &t3) {
  const V a0 = cadd(t0, t2), a1 = csub(t0, t2);
  const V b0 = cadd(t1, t3), b1 = cmul_i(csub(t1, t3), SIGN);
  t0 = cadd(a0, b0);
  t1 = cadd(a1, b1);
  t2 = csub(a0, b0);
  t3 = csub(a1, b1);
}

template <int SIGN, typename V>
__device__ __forceinline__ void dft8(V *v) {
  using S = decltype(V{}.x);
  const S c = S(0.70710678118654752440);  // cos(pi/4)
  V e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  V o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<SIGN>(e0, e1, e2, e3);
  dft4<SIGN>(o0, o1, o2, o3);
  // W8^q = exp(SIGN*2*pi*i*q/8)
  const V w1 = cmake<V>(c, SIGN * c);
  const V w3 = cmake<V>(-c, SIGN * c);
  o1 = cmul(o1, w1);
  o2 = cmul_i(o2, SIGN);
  o3 = cmul(o3, w3);
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1);
  v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2);
  v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3);
  v[7] = csub(e3, o3);
}

template <int SIGN, typename V>
__device__ __forceinline__ void dft3(V *v) {
  using S = decltype(V{}.x);
  const S s3 = S(0.86602540378443864676);  // sin(2 pi/3)
  const V a = v[0], b = v[1], cc = v[2];
  const V t1 = cadd(b, cc);
  const V t2 = cmake<V>(a.x - S(0.5) * t1.x, a.y - S(0.5) * t1.y);
  const V t3 = cmul_i(csub(b, cc), SIGN);  // i*SIGN*(b-c)
  v[0] = cadd(a, t1);
  v[1] = cmake<V>(t2.x + s3 * t3.x, t2.y + s3 * t3.y);
  v[2] = cmake<V>(t2.x - s3 * t3.x, t2.y - s3 * t3.y);
}

template <int SIGN, typename V>
__device__ __forceinline__ void dft5(V *v) {
  using S = decltype(V{}.x);
  // cos/sin of 2 pi/5 and 4 pi/5
  const S c1 = S(0.30901699437494742410), c2 = S(-0.80901699437494742410);
  const S s1 = S(0.95105651629515357212), s2 = S(0.58778525229247312917);
  const V a = v[0];
  const V b1 = cadd(v[1], v[4]), b2 = cadd(v[2], v[3]);
  const V d1 = csub(v[1], v[4]), d2 = csub(v[2], v[3]);
  const V r1 = cmake<V>(a.x + c1 * b1.x + c2 * b2.x, a.y + c1 * b1.y + c2 * b2.y);
  const V r2 = cmake<V>(a.x + c2 * b1.x + c1 * b2.x, a.y + c2 * b1.y + c1 * b2.y);
  const V i1 = cmul_i(cmake<V>(s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y), SIGN);
  const V i2 = cmul_i(cmake<V>(s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y), SIGN);
  v[0] = cadd(a, cadd(b1, b2));
  v[1] = cadd(r1, i1);
  v[4] = csub(r1, i1);
  v[2] = cadd(r2, i2);
  v[3] = csub(r2, i2);
}

// In-register DFT of size R; SIGN = -1 forward (e^{-}), +1 backward (e^{+}).
template <int R, int SIGN, typename V>
__device__ __forceinline__ void dft_small(V *v) {
  if constexpr (R == 2) {
    const V a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (R == 3) {
    dft3<SIGN>(v);
  } else if constexpr (R == 4) {
    dft4<SIGN>(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 5) {
    dft5<SIGN>(v);
  } else {
    static_assert(R == 8, "radix 2, 3, 4, 5 or 8");
    dft8<SIGN>(v);
  }
}

// One Stockham pass of radix R over a length-M complex line in shared memory,
// in place, by a group of G threads (rank t in the group). Pass with span Ns:
//   item j (0 <= j < M/R), k = j mod Ns:
//   v[r] = buf[j + r*M/R] * W_{Ns*R}^{r*k};  v = DFT_R(v);
//   buf[(j/Ns)*Ns*R + k + r*Ns] = v[r]
// MAXIT bounds the items per thread. SYNC is __syncwarp or __syncthreads.
template <int R, int SIGN, int MAXIT, bool BLOCK, typename V>
__device__ __forceinline__ void stockham_pass(V *buf, int M, int Ns, const V *__restrict__ tw, int t, int G) {
  const int nit = M / R;
  const int stride_tw = M / (Ns * R);
  V v[MAXIT][R];
#pragma unroll
  for (int it = 0; it < MAXIT; ++it) {
    const int j = t + it * G;
    if (j < nit) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[it][r] = buf[j + r * nit];
    }
  }
  if (BLOCK)
    __syncthreads();
  else
    __syncwarp();
#pragma unroll
  for (int it = 0; it < MAXIT; ++it) {
    const int j = t + it * G;
    if (j < nit) {
      const int k = j % Ns;
      if (Ns > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          V w = __ldg(&tw[r * k * stride_tw]);
          if (SIGN > 0) w.y = -w.y;
          v[it][r] = cmul(v[it][r], w);
        }
      }
      dft_small<R, SIGN>(v[it]);
      const int base = (j / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) buf[base + r * Ns] = v[it][r];
    }
  }
  if (BLOCK)
    __syncthreads();
  else
    __syncwarp();
}

// Warp FFT of a power-of-two length M <= 512 in shared memory (in place).
template <int SIGN, typename V>
__device__ __forceinline__ void warp_fft(V *buf, int M, const V *__restrict__ tw, int lane) {
  int Ns = 1;
  while (Ns * 8 <= M) {
    stockham_pass<8, SIGN, 2, false>(buf, M, Ns, tw, lane, 32);
    Ns *= 8;
  }
  if (Ns * 4 <= M) {
    stockham_pass<4, SIGN, 4, false>(buf, M, Ns, tw, lane, 32);
    Ns *= 4;
  }
  if (Ns * 2 <= M) {
    stockham_pass<2, SIGN, 8, false>(buf, M, Ns, tw, lane, 32);
    Ns *= 2;
  }
}

// CTA FFT of length n = 2^a 3^b 5^c (n <= 4096) in shared memory; NB lines
// stored back to back (line l at buf + l*n) are transformed in turn by the
// 256 threads of the CTA. The twiddle table has n entries.
template <int R, int SIGN, int NB, typename V>
__device__ __forceinline__ void block_pass(V *buf, int n, int Ns, const V *__restrict__ tw) {
  constexpr int MAXIT = (4096 / R + 255) / 256;
#pragma unroll 1
  for (int l = 0; l < NB; ++l)
    stockham_pass<R, SIGN, MAXIT, true>(buf + l * n, n, Ns, tw, threadIdx.x, 256);
}

template <int SIGN, int NB, typename V>
__device__ __forceinline__ void block_fft(V *buf, int n, const V *__restrict__ tw) {
  int Ns = 1, rem = n;
  while (rem % 8 == 0) { block_pass<8, SIGN, NB>(buf, n, Ns, tw); Ns *= 8; rem /= 8; }
  while (rem % 4 == 0) { block_pass<4, SIGN, NB>(buf, n, Ns, tw); Ns *= 4; rem /= 4; }
  while (rem % 2 == 0) { block_pass<2, SIGN, NB>(buf, n, Ns, tw); Ns *= 2; rem /= 2; }
  while (rem % 3 == 0) { block_pass<3, SIGN, NB>(buf, n, Ns, tw); Ns *= 3; rem /= 3; }
  while (rem % 5 == 0) { block_pass<5, SIGN, NB>(buf, n, Ns, tw); Ns *= 5; rem /= 5; }
}

// Shared-memory index of element i of a line for the line FFTs below.
// 16-byte (FP64) elements: one element of padding every 8, which turns the
// radix-8, Ns = 1 write stride of 8 elements (128 bytes, a 32-way bank
// conflict) into 9. 8-byte (FP32) elements: i ^ ((i / 8) mod 16), a
// permutation inside each block of 128 elements that keeps every run of 16
// consecutive elements on distinct banks and sends the stride-8 writes to 16
// distinct bank pairs (the padding of the FP64 layout leaves two of every 16
// consecutive FP32 elements on one bank pair).
template <typename V>
__host__ __device__ __forceinline__ int xpad(int i) {
  if constexpr (sizeof(V) == 16)
    return i + (i >> 3);
  else
    return i ^ ((i >> 3) & 15);
}

// Line stride (elements) of MB lines of n elements in the layout of xpad:
// the first index past a line, rounded up so that the MB lines start P / MB
// elements apart modulo the P elements of a 128-byte bank row (P = 8 for
// FP64, 16 for FP32), which spreads the MB lines of one plane row, loaded and
// stored by consecutive threads, over distinct banks. For n = 1024, MB = 4 a
// bank model of the x-DCT kernels' accesses gives 3200 wavefronts per CTA
// for FP32 (6208 with the FP64 layout and an odd stride; 2816 minimum) and
// 6272 for FP64 (7040 with an odd stride; 5632 minimum).
template <typename V>
__host__ __device__ __forceinline__ int xline_ld(int n, int MB) {
  if constexpr (sizeof(V) == 16) {
    const int b = xpad<V>(n - 1) + 1;
    return b + (((8 / MB - b) % 8) + 8) % 8;
  } else {
    return ((n + 15) / 16) * 16 + 16 / MB;
  }
}

// Stockham pass as stockham_pass, on a padded line, by the G threads (rank t)
// that own this line; every thread of the CTA runs the same passes on its own
// line, so the barriers are CTA-wide.
template <int R, int SIGN, int MAXIT, typename V>
__device__ __forceinline__ void stockham_pass_pad(V *buf, int M, int Ns, const V *__restrict__ tw, int t, int G) {
  const int nit = M / R;
  const int stride_tw = M / (Ns * R);
  V v[MAXIT][R];
#pragma unroll
  for (int it = 0; it < MAXIT; ++it) {
    const int j = t + it * G;
    if (j < nit) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[it][r] = buf[xpad<V>(j + r * nit)];
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < MAXIT; ++it) {
    const int j = t + it * G;
    if (j < nit) {
      const int k = j % Ns;
      if (Ns > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          V w = __ldg(&tw[r * k * stride_tw]);
          if (SIGN > 0) w.y = -w.y;
          v[it][r] = cmul(v[it][r], w);
        }
      }
      dft_small<R, SIGN>(v[it]);
      const int base = (j / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) buf[xpad<V>(base + r * Ns)] = v[it][r];
    }
  }
  __syncthreads();
}

// FFT of length n = 2^a 3^b 5^c of this thread's padded line (n * lines per
// CTA <= 4096), the radix order of block_fft (8s, 4s, 2s, 3s, 5s), so the
// arithmetic is block_fft's operation for operation.
// NT: threads of the CTA (n * lines <= 4096, so a thread has at most
// 4096 / (NT R) items of a radix-R pass)
template <int SIGN, int NT = 256, typename V>
__device__ __forceinline__ void block_fft_lines(V *buf, int n, const V *__restrict__ tw, int t, int G) {
  constexpr int I8 = (4096 / 8 + NT - 1) / NT, I4 = (4096 / 4 + NT - 1) / NT, I2 = (4096 / 2 + NT - 1) / NT;
  constexpr int I3 = (4096 / 3 + NT - 1) / NT, I5 = (4096 / 5 + NT - 1) / NT;
  int Ns = 1, rem = n;
  while (rem % 8 == 0) { stockham_pass_pad<8, SIGN, I8>(buf, n, Ns, tw, t, G); Ns *= 8; rem /= 8; }
  while (rem % 4 == 0) { stockham_pass_pad<4, SIGN, I4>(buf, n, Ns, tw, t, G); Ns *= 4; rem /= 4; }
  while (rem % 2 == 0) { stockham_pass_pad<2, SIGN, I2>(buf, n, Ns, tw, t, G); Ns *= 2; rem /= 2; }
  while (rem % 3 == 0) { stockham_pass_pad<3, SIGN, I3>(buf, n, Ns, tw, t, G); Ns *= 3; rem /= 3; }
  while (rem % 5 == 0) { stockham_pass_pad<5, SIGN, I5>(buf, n, Ns, tw, t, G); Ns *= 5; rem /= 5; }
}

// block_fft_lines for a length N = 2^a known at compile time: the same
// passes in the same order (8s, 4s, 2s), each with its constant stride. Inside
// the persistent x-DCT kernels' tile loop the run-time form needs more than
// the 128 registers a 512-thread CTA may hold (ptxas: 0.1-2 KB of spills per
// thread with the run-time length, none with this one).
template <int SIGN, int NT, int N, int NS = 1, typename V>
__device__ __forceinline__ void block_fft_lines_n(V *buf, const V *__restrict__ tw, int t, int G) {
  constexpr int rem = N / NS;
  if constexpr (rem > 1) {
    static_assert(rem % 2 == 0, "power-of-two lengths only");
    constexpr int R = rem % 8 == 0 ? 8 : (rem % 4 == 0 ? 4 : 2);
    constexpr int MAXIT = (4096 / R + NT - 1) / NT;
    stockham_pass_pad<R, SIGN, MAXIT>(buf, N, NS, tw, t, G);
    block_fft_lines_n<SIGN, NT, N, NS * R>(buf, tw, t, G);
  }
}

}  // namespace otbl
