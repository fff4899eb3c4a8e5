// interpyy (lip.f90:359-440) of the mixed-precision path as a dense
// operator on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// interpyy maps every y-column (plane i, real spanwise index kr) of a field
// linearly: out(1:ny) = Mop * in(1:K), K = ny+1 for u and w (u-type input),
// ny for v, with one operator Mop = A^-1 B for all columns (A the
// pre-factored tridiagonal, B the explicit stencil with its boundary rows).
// So each field is one GEMM
//   Out[ny x C] = Mop[ny x K] * In[K x C],   C = nx * nz1 columns,
// whose columns are the plane layout's (i, kr) pairs in storage order.
//
// Mop is built once per context on the host in FP64 by running the
// interpyy recurrence on unit vectors, and split into two TF32 parts
// (hi = tf32(Mop), lo = tf32(Mop - hi)); each FP64 field value is split the
// same way on the device. The products hi*hi + hi*lo + lo*hi (three
// tcgen05.mma of kind::tf32) accumulate in FP32 in tensor memory, which gives
// the FP32 accuracy of the mixed path's other operators.
//
// Kernel: persistent, one CTA of 128 threads per SM, tiles of N = 256
// columns, both M-tiles of 128 output rows (TMEM columns 0..255 and
// 256..511). K runs in chunks of 16 input rows through two shared-memory
// stages: the operator chunk (both M-tiles, both parts, 32 KB, stored in
// global memory in the canonical K-major layout) arrives by one bulk copy
// (cp.async.bulk, no tensor map, no multicast), the field chunk (16 rows x
// 256 columns, FP64) is loaded, split and written by the threads in the
// canonical K-major layout too, i.e. transposed on the way into shared
// memory. (The field's natural order would be the MN-major operand form, but
// kind::tf32 with B MN-major, no swizzle, left the accumulators at zero on
// B200 in a one-MMA probe, while the K-major form was exact.) Thread 0 issues
// the MMAs and commits each stage to
// an mbarrier that releases it. Chunks in which an M-tile's rows of Mop are
// below 2^-40 of its largest entry (the inverse of the diagonally dominant
// tridiagonal decays geometrically away from the diagonal) are skipped for
// that M-tile. The epilogue reads the accumulators (tcgen05.ld) and stores
// FP32. Every wait is bounded: on a timeout the CTA records
// OTBL_ERR_TIMEOUT, stops, frees its tensor memory and returns.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "devcommon.cuh"
#include "otbl_internal.cuh"
#include "tma.cuh"

namespace otbl {

namespace {

constexpr int YD_N = 256;                      // columns per tile
constexpr int YD_KC = 16;                      // input rows per K-chunk
constexpr int YD_THREADS = 128;
constexpr int YD_A_PART = 128 * YD_KC * 4;     // one M-tile, one part: 8 KB
constexpr int YD_A_CHUNK = 4 * YD_A_PART;      // 2 M-tiles x 2 parts: 32 KB
constexpr int YD_B_PART = YD_N * YD_KC * 4;    // 16 KB
constexpr int YD_B_CHUNK = 2 * YD_B_PART;      // hi, lo: 32 KB
constexpr int YD_STAGE = YD_A_CHUNK + YD_B_CHUNK;
constexpr int YD_SMEM = 2 * YD_STAGE + 2048;   // two stages, barriers, alignment slack
constexpr uint32_t YD_TMEM_COLS = 512;
constexpr uint64_t YD_WAIT_NS = 2000000000ull;  // 2 s

// canonical K-major, no swizzle: element (m, k) of one M-tile part, k < 16
__host__ __device__ constexpr int yd_a_off(int m, int k) {
  return (m & 7) * 16 + (m >> 3) * (YD_KC / 4 * 128) + (k >> 2) * 128 + (k & 3) * 4;
}
// the field chunk in the same K-major form: element (n, k) of one part, k < 16
__host__ __device__ constexpr int yd_b_off(int n, int k) {
  return (n & 7) * 16 + (n >> 3) * (YD_KC / 4 * 128) + (k >> 2) * 128 + (k & 3) * 4;
}
static_assert(yd_a_off(127, 15) + 4 == YD_A_PART, "A part layout");
static_assert(yd_b_off(255, 15) + 4 == YD_B_PART, "B part layout");

// shared-memory matrix descriptor (sm_100): start, LBO, SBO in 16-byte
// units, version 1, no swizzle
__device__ __forceinline__ uint64_t yd_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
// instruction descriptor, kind::tf32: F32 accumulator, A and B K-major
constexpr uint32_t yd_idesc(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | (0u << 15) | (0u << 16) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void yd_mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void yd_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void yd_bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ uint32_t yd_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return r;
}
// 16 consecutive accumulator columns of this warp's 32 lanes
__device__ __forceinline__ void yd_tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

}  // namespace

struct YDenseField {
  const double *in;  // K rows per plane
  float *out;        // ny rows per plane
  const uint32_t *op;  // operator chunks: [chunk][mt][part][YD_A_PART bytes]
  int K;             // input rows per plane
  int kb[2], ke[2];  // per M-tile, the chunks [kb, ke) that carry its band
};
struct YDenseArgs {
  YDenseField f[3];
  int nchunk;        // K-chunks (ceil(max K / 16))
  int tiles;         // tiles per field
};

__global__ void __launch_bounds__(YD_THREADS, 1) k_ydense(int nx, int ny, int nz1, YDenseArgs a, int *err) {
  extern __shared__ __align__(1024) unsigned char ydsm[];
  unsigned char *base = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(ydsm) + 1023) & ~(uintptr_t)1023);
  uint64_t *bar_full = reinterpret_cast<uint64_t *>(base + 2 * YD_STAGE);  // [2]
  uint64_t *bar_done = bar_full + 2;                                       // [2]
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar_done + 2);
  int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const long C = (long)nx * nz1;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(YD_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (t == 0) {
    for (int s = 0; s < 2; ++s) {
      mbar_init(&bar_full[s], 1);
      mbar_init(&bar_done[s], 1);
    }
    *abort_flag = 0;
    mbar_init_fence();
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  constexpr uint32_t IDESC = yd_idesc(128, YD_N);

  unsigned fills[2] = {0u, 0u};  // completed uses of each stage
  int stage = 0;
  const int total = 3 * a.tiles;
  for (int tile = blockIdx.x; tile < total && !*abort_flag; tile += gridDim.x) {
    const int fi = tile / a.tiles;
    const YDenseField F = a.f[fi];
    const long c0 = (long)(tile - fi * a.tiles) * YD_N;
    const int nchunk = (F.K + YD_KC - 1) / YD_KC;
    for (int kc = 0; kc < nchunk; ++kc) {
      const int s = stage;
      unsigned char *sa = base + s * YD_STAGE, *sb = sa + YD_A_CHUNK;
      // the stage's previous MMAs must have read it before it is refilled
      if (fills[s] > 0 && !mbar_wait_bounded(&bar_done[s], (fills[s] - 1) & 1, YD_WAIT_NS)) {
        if (t == 0) {
          atomicExch(err, OTBL_ERR_TIMEOUT);
          *abort_flag = 1;
        }
      }
      __syncthreads();
      if (*abort_flag) break;
      if (t == 0) {
        mbar_arrive_expect_tx(&bar_full[s], YD_A_CHUNK);
        yd_bulk_g2s(sa, reinterpret_cast<const unsigned char *>(F.op) + (size_t)kc * YD_A_CHUNK, YD_A_CHUNK,
                    &bar_full[s]);
      }
      // the field chunk: rows k0..k0+15 x 256 columns, split into hi/lo.
      // Item e = (column n = e % 256, rows k0+4g..k0+4g+3, g = e / 256): four
      // loads of one column (a warp reads 32 consecutive columns of a row),
      // one 16-byte store per part (8 consecutive lanes fill the 8 rows of a
      // core matrix: conflict-free).
      const int k0 = kc * YD_KC;
      for (int e = t; e < YD_N * (YD_KC / 4); e += YD_THREADS) {
        const int n = e & (YD_N - 1), g = e / YD_N;
        const long cidx = c0 + n;
        const bool col_ok = cidx < C;
        const long i = col_ok ? cidx / nz1 : 0, kr = col_ok ? cidx - i * nz1 : 0;
        uint32_t hi[4], lo[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int j = k0 + 4 * g + q;
          const double x = (col_ok && j < F.K) ? F.in[((size_t)i * F.K + j) * nz1 + kr] : 0.0;
          hi[q] = yd_tf32((float)x);
          lo[q] = yd_tf32((float)(x - (double)__uint_as_float(hi[q])));
        }
        const int off = yd_b_off(n, 4 * g);
        *reinterpret_cast<uint4 *>(sb + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<uint4 *>(sb + YD_B_PART + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
      }
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      __syncthreads();
      if (t == 0) {
        if (!mbar_wait_bounded(&bar_full[s], fills[s] & 1, YD_WAIT_NS)) {
          atomicExch(err, OTBL_ERR_TIMEOUT);
          *abort_flag = 1;
        } else {
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          const uint32_t sa_u = smem_u32(sa), sb_u = smem_u32(sb);
#pragma unroll
          for (int mt = 0; mt < 2; ++mt) {
            if (kc < F.kb[mt] || kc >= F.ke[mt]) continue;
            const uint32_t d = tmem + (uint32_t)(mt * YD_N);
#pragma unroll
            for (int ks = 0; ks < YD_KC / 8; ++ks) {
              const uint32_t ah = sa_u + (uint32_t)((mt * 2 + 0) * YD_A_PART + ks * 256);
              const uint32_t al = sa_u + (uint32_t)((mt * 2 + 1) * YD_A_PART + ks * 256);
              const uint32_t bh = sb_u + (uint32_t)(ks * 256);
              const uint32_t bl = bh + YD_B_PART;
              const uint64_t dah = yd_desc(ah, 128, YD_KC / 4 * 128), dal = yd_desc(al, 128, YD_KC / 4 * 128);
              const uint64_t dbh = yd_desc(bh, 128, YD_KC / 4 * 128), dbl = yd_desc(bl, 128, YD_KC / 4 * 128);
              const uint32_t first = (kc == F.kb[mt] && ks == 0) ? 0u : 1u;
              yd_mma(d, dah, dbh, IDESC, first);
              yd_mma(d, dah, dbl, IDESC, 1u);
              yd_mma(d, dal, dbh, IDESC, 1u);
            }
          }
          yd_commit(&bar_done[s]);
        }
      }
      fills[s] += 1;
      stage ^= 1;
    }
    __syncthreads();
    if (*abort_flag) break;
    // the last stage's commit covers every MMA of the tile
    const int sl = stage ^ 1;
    if (!mbar_wait_bounded(&bar_done[sl], (fills[sl] - 1) & 1, YD_WAIT_NS)) {
      if (lane == 0) {
        atomicExch(err, OTBL_ERR_TIMEOUT);
        *abort_flag = 1;
      }
    }
    __syncthreads();
    if (*abort_flag) break;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    // epilogue: warp w owns TMEM lanes 32w..32w+31 = output rows
    for (int mt = 0; mt < 2; ++mt) {
      const int r = mt * 128 + warp * 32 + lane;  // output row, 0-based
      for (int cb = 0; cb < YD_N; cb += 16) {
        uint32_t v[16];
        yd_tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(mt * YD_N + cb), v);
        if (r < ny && F.ke[mt] > F.kb[mt]) {
#pragma unroll
          for (int p = 0; p < 16; p += 2) {
            const long cidx = c0 + cb + p;
            if (cidx < C) {
              const long i = cidx / nz1, kr = cidx - i * nz1;
              *reinterpret_cast<float2 *>(F.out + ((size_t)i * ny + r) * nz1 + kr) =
                  make_float2(__uint_as_float(v[p]), __uint_as_float(v[p + 1]));
            }
          }
        } else if (r < ny) {  // an M-tile without any band: zero rows
#pragma unroll
          for (int p = 0; p < 16; p += 2) {
            const long cidx = c0 + cb + p;
            if (cidx < C) {
              const long i = cidx / nz1, kr = cidx - i * nz1;
              *reinterpret_cast<float2 *>(F.out + ((size_t)i * ny + r) * nz1 + kr) = make_float2(0.f, 0.f);
            }
          }
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
  }
  // drain: MMAs that may still be in flight before the memory is freed
  __syncthreads();
  for (int s = 0; s < 2; ++s)
    if (fills[s] > 0 && !*abort_flag) mbar_wait_bounded(&bar_done[s], (fills[s] - 1) & 1, YD_WAIT_NS);
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(YD_TMEM_COLS) : "memory");
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

// cvt.rna.tf32.f32 on the host: round the magnitude to 10 mantissa bits,
// ties away from zero
uint32_t host_tf32(float x) {
  uint32_t b;
  std::memcpy(&b, &x, 4);
  if ((b & 0x7F800000u) == 0x7F800000u) return b;  // inf/nan unchanged
  b += 0x1000u;
  return b & 0xFFFFE000u;
}
float bits_f(uint32_t b) {
  float f;
  std::memcpy(&f, &b, 4);
  return f;
}

// The interpyy operator of lip.f90:359-440 for input type `which` (0: u-type,
// K = ny+1; 1: v-type, K = ny), column jj = the response to the unit vector
// at input row jj: op[(r-1)*K + (jj-1)], r = 1..ny.
std::vector<double> interpyy_operator(const otbl_ctx *c, int which) {
  const int nx = c->cfg.nx, ny = c->cfg.ny, nz = c->cfg.nz;
  otbl_coef_offsets o;
  otbl_coef_layout(nx, ny, nz, &o);
  const double *cf = c->coef_host.data();
  const double *icon = cf + o.off[which == 0 ? OTBL_C_INYU : OTBL_C_INYV];
  const double *econ = cf + o.off[which == 0 ? OTBL_C_COFIUY : OTBL_C_COFIVY];
  const double *inby = cf + o.off[OTBL_C_INBY];
  auto IC = [&](int r, int j) { return icon[(j - 1) * 3 + (r - 1)]; };
  auto EC = [&](int r, int j) { return econ[(j - 1) * 2 + (r - 1)]; };
  auto IB = [&](int r, int col) { return inby[(col - 1) * 4 + (r - 1)]; };
  const int K = which == 0 ? ny + 1 : ny;
  std::vector<double> op((size_t)ny * K, 0.0), g(K + 2), gi(ny + 2);
  for (int jj = 1; jj <= K; ++jj) {
    std::fill(g.begin(), g.end(), 0.0);
    g[jj] = 1.0;
    auto G = [&](int j) { return g[j]; };
    if (which == 0) {
      gi[1] = 0.0;
      const double buf = IB(1, 1) * G(ny + 1) + IB(1, 2) * G(ny) + IB(1, 3) * G(ny - 1) + IB(1, 4) * G(ny - 2);
      for (int j = 2; j <= ny - 1; ++j) gi[j] = EC(1, j) * G(j) + EC(2, j) * G(j + 1);
      gi[ny] = buf;
    } else {
      const double buf = IB(3, 1) * G(1) + IB(3, 2) * G(2) + IB(3, 3) * G(3) + IB(3, 4) * G(4);
      gi[ny] = IB(4, 1) * G(ny) + IB(4, 2) * G(ny - 1) + IB(4, 3) * G(ny - 2) + IB(4, 4) * G(ny - 3);
      for (int j = ny - 1; j >= 2; --j) gi[j] = EC(2, j) * G(j) + EC(1, j) * G(j - 1);
      gi[1] = buf;
    }
    for (int j = 2; j <= ny; ++j) gi[j] = gi[j] + IC(1, j) * gi[j - 1];
    gi[ny] = gi[ny] * IC(2, ny);
    for (int j = ny - 1; j >= 1; --j) gi[j] = (gi[j] - IC(3, j) * gi[j + 1]) * IC(2, j);
    for (int r = 1; r <= ny; ++r) op[(size_t)(r - 1) * K + (jj - 1)] = gi[r];
  }
  return op;
}

}  // namespace

// Builds the two operators' TF32 chunks and band ranges on the device
// (once per context; again after new coefficients).
cudaError_t ydense_prepare(otbl_ctx *c) {
  const int ny = c->cfg.ny;
  if (ny > 256) return cudaErrorInvalidValue;  // two M-tiles of 128 rows
  const int nchunk = (ny + 1 + YD_KC - 1) / YD_KC;
  const size_t words_per_op = (size_t)nchunk * YD_A_CHUNK / 4;
  std::vector<uint32_t> host(2 * words_per_op, 0u);
  for (int which = 0; which < 2; ++which) {
    const int K = which == 0 ? ny + 1 : ny;
    const std::vector<double> op = interpyy_operator(c, which);
    double amax = 0.0;
    for (double v : op) amax = std::max(amax, std::fabs(v));
    const double thr = amax * 9.094947017729282e-13;  // 2^-40
    int kb[2] = {nchunk, nchunk}, ke[2] = {0, 0};
    uint32_t *dst = host.data() + which * words_per_op;
    for (int kc = 0; kc < nchunk; ++kc)
      for (int mt = 0; mt < 2; ++mt)
        for (int m = 0; m < 128; ++m) {
          const int r = mt * 128 + m;  // 0-based output row
          for (int k = 0; k < YD_KC; ++k) {
            const int jj = kc * YD_KC + k;  // 0-based input row
            const double v = (r < ny && jj < K) ? op[(size_t)r * K + jj] : 0.0;
            if (std::fabs(v) > thr) {
              kb[mt] = std::min(kb[mt], kc);
              ke[mt] = std::max(ke[mt], kc + 1);
            }
            const uint32_t hi = host_tf32((float)v);
            const uint32_t lo = host_tf32((float)(v - (double)bits_f(hi)));
            const size_t chunk_w = (size_t)kc * (YD_A_CHUNK / 4);
            dst[chunk_w + ((size_t)(mt * 2 + 0) * YD_A_PART + yd_a_off(m, k)) / 4] = hi;
            dst[chunk_w + ((size_t)(mt * 2 + 1) * YD_A_PART + yd_a_off(m, k)) / 4] = lo;
          }
        }
    for (int mt = 0; mt < 2; ++mt) {
      if (ke[mt] <= kb[mt]) kb[mt] = ke[mt] = 0;  // no band: the rows are zero
      c->yd_kb[which][mt] = kb[mt];
      c->yd_ke[which][mt] = ke[mt];
    }
  }
  if (!c->yd_op) {
    void *p = nullptr;
    if (cudaMalloc(&p, host.size() * 4) != cudaSuccess) return cudaErrorMemoryAllocation;
    c->allocs.push_back(p);
    c->bytes += host.size() * 4;
    c->yd_op = static_cast<uint32_t *>(p);
  }
  c->yd_words_per_op = words_per_op;
  cudaError_t e = cudaMemcpyAsync(c->yd_op, host.data(), host.size() * 4, cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(c->stream);
}

size_t ydense_bytes(int ny) {
  const int nchunk = (ny + 1 + YD_KC - 1) / YD_KC;
  return 2 * (size_t)nchunk * YD_A_CHUNK;
}

cudaError_t launch_interpy_dense(otbl_ctx *c) {
  cudaStream_t s = c->stream;
  const int nx = c->cfg.nx, ny = c->cfg.ny, nz1 = c->dc.nz1;
  YDenseArgs a;
  const double *ins[3] = {c->f[OTBL_F_U], c->f[OTBL_F_W], c->f[OTBL_F_V]};
  void *outs[3] = {c->w.uy, c->w.wy, c->w.vy};
  const int which[3] = {0, 0, 1};
  for (int f = 0; f < 3; ++f) {
    YDenseField &F = a.f[f];
    F.in = ins[f];
    F.out = static_cast<float *>(outs[f]);
    F.op = c->yd_op + which[f] * c->yd_words_per_op;
    F.K = which[f] == 0 ? ny + 1 : ny;
    for (int mt = 0; mt < 2; ++mt) {
      F.kb[mt] = c->yd_kb[which[f]][mt];
      F.ke[mt] = c->yd_ke[which[f]][mt];
    }
  }
  a.nchunk = (ny + 1 + YD_KC - 1) / YD_KC;
  const long C = (long)nx * nz1;
  a.tiles = (int)((C + YD_N - 1) / YD_N);
  static int nsm = 0;
  if (nsm == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (nsm <= 0) nsm = 148;
  }
  const int grid = std::min(3 * a.tiles, nsm);
  cudaFuncSetAttribute(k_ydense, cudaFuncAttributeMaxDynamicSharedMemorySize, YD_SMEM);
  k_ydense<<<grid, YD_THREADS, YD_SMEM, s>>>(nx, ny, nz1, a, &c->st->err);
  c->launches += 1;
  return cudaGetLastError();
}

}  // namespace otbl
