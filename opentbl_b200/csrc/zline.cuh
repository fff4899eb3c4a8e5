// z-line transforms (fourxz, ffts.f90:27-67), one warp per line, shared by
// the products (kernels.cu) and the statistics (k_stats.cu).
#pragma once
#include <cuda_runtime.h>

#include "fft.cuh"

namespace otbl {

// z-line transforms (fourxz, ffts.f90:27-67), one warp per line, in the
// arithmetic type T (double, or float on the mixed path). Fields of element
// type TI/TO are read and written with conversion to and from T.
// ---------------------------------------------------------------------------
template <typename T>
struct ZTabT {
  const V2<T> *tw;   // exp(-2 pi i t/M), t < M
  const V2<T> *tw2;  // exp(-2 pi i t/nz), t < M
  int M, nz, nz2;
};
using ZTab = ZTabT<double>;

// complex element k of a field of element type TI, as V2<T>
template <typename T, typename TI>
__device__ __forceinline__ V2<T> ldcx(const TI *__restrict__ f, int k) {
  const V2<TI> a = __ldg(reinterpret_cast<const V2<TI> *>(f) + k);
  return cmake<V2<T>>((T)a.x, (T)a.y);
}
template <typename TO, typename V>
__device__ __forceinline__ void stcx(TO *__restrict__ f, int k, V v) {
  reinterpret_cast<V2<TO> *>(f)[k] = cmake<V2<TO>>((TO)v.x, (TO)v.y);
}

// c2r of fou (nz2+1 complex modes, global) into buf (M complex = nz reals)
template <typename T, typename TI>
__device__ __forceinline__ void line_c2r(const ZTabT<T> &z, const TI *__restrict__ fou, V2<T> *buf, int lane) {
  using V = V2<T>;
  const int M = z.M, nz2 = z.nz2;
  for (int k = lane; k < M; k += 32) {
    V a = k <= nz2 ? ldcx<T>(fou, k) : cmake<V>(T(0), T(0));
    if (k == 0) a.y = T(0);  // c2r ignores Im X[0]
    const int km = M - k;
    V b = km <= nz2 ? ldcx<T>(fou, km) : cmake<V>(T(0), T(0));
    b.y = -b.y;
    const V s = cadd(a, b), d = csub(a, b);
    const V t = cmul(cconj(__ldg(z.tw2 + k)), d);  // W^{-k} d
    buf[k] = cmake<V>(s.x - t.y, s.y + t.x);      // s + i t
  }
  __syncwarp();
  warp_fft<1>(buf, M, z.tw, lane);
}

// r2c of buf (nz reals packed as M complex) into fou (modes 0..nz2) x 1/nz
template <typename T, typename TO>
__device__ __forceinline__ void line_r2c(const ZTabT<T> &z, V2<T> *buf, TO *__restrict__ fou, int lane) {
  using V = V2<T>;
  const int M = z.M, nz2 = z.nz2;
  warp_fft<-1>(buf, M, z.tw, lane);
  const T dnf = T(1) / (T)z.nz;
  for (int k = lane; k <= nz2; k += 32) {
    const V zk = buf[k];
    const V zc = cconj(buf[(M - k) & (M - 1)]);
    const V e = cmake<V>(T(0.5) * (zk.x + zc.x), T(0.5) * (zk.y + zc.y));
    const V d = csub(zk, zc);
    const V o = cmake<V>(T(0.5) * d.y, T(-0.5) * d.x);  // -i d / 2
    const V xk = cadd(e, cmul(__ldg(z.tw2 + k), o));
    stcx(fou, k, cmake<V>(dnf * xk.x, dnf * xk.y));
  }
  __syncwarp();
}

}  // namespace otbl
