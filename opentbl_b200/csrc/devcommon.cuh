// Small device helpers shared by the kernel files.
#pragma once
#include <cuda_runtime.h>

// Fortran-shaped accessors into the packed coefficient buffer
#define A3(a, r, i) (a)[((i)-1) * 3 + (r)-1]
#define A2(a, r, i) (a)[((i)-1) * 2 + (r)-1]
#define M4(a, r, cc) (a)[((cc)-1) * 4 + (r)-1]
#define M5(a, r, cc) (a)[((cc)-1) * 5 + (r)-1]
#define M2(a, r, cc) (a)[((cc)-1) * 2 + (r)-1]

namespace otbl {

// REAL4 rounding of the reference's transposes (change.f90:579,608,...)
__device__ __forceinline__ double rnd(double x, int xr) { return xr ? (double)(float)x : x; }
__device__ __forceinline__ float rnd(float x, int) { return x; }

// NaN-propagating maximum of non-negative values
__device__ __forceinline__ double nmax(double m, double v) {
  return (m != m) ? m : ((v != v) ? v : fmax(m, v));
}

// Asynchronous 8-byte global -> shared copy (cp.async, zero-filled when
// !valid: the source size operand is 0 and nothing is read from `g`).
__device__ __forceinline__ void cp_async8(double *s, const double *g, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  const int sz = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(g), "r"(sz) : "memory");
}
// Waits for every cp.async this thread issued (the caller then syncs the CTA).
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// a[f] of a kernel-parameter array with f uniform across the grid's y index,
// selected without indexing the parameter block (which would copy it to
// local memory)
template <typename P>
__device__ __forceinline__ P pick3(const P (&a)[3], int f) {
  return f == 0 ? a[0] : (f == 1 ? a[1] : a[2]);
}

}  // namespace otbl
