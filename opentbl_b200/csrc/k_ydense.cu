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
// Kernel: persistent, one CTA per SM, warp-specialised. A tile is one
// plane i and NT consecutive spanwise columns kr (NT a multiple of 16, at
// most 128, chosen so that nb = ceil(nz1/NT) tiles cover a plane); both
// M-tiles of 128 output rows accumulate in tensor memory, in one of two
// accumulator sets of 256 columns (set a: columns 256a + mt*NT ...), so that
// the epilogue of one tile overlaps the MMAs of the next. K runs in chunks of
// 16 input rows:
//   warp 0, one lane: the field producer. Per chunk, a 3D TMA box of the
//     FP64 field (NT columns x 16 rows x 1 plane; columns past nz1 and rows
//     past K read as zero) into a ring of SF slots, which the converters
//     release as soon as they have read it, so that many boxes are in flight.
//   warp 10, one lane: the operator producer. Per chunk, the operator chunk
//     (stored in global memory in the canonical K-major layout, 16 KB per
//     M-tile for both parts; an M-tile's part only in the chunks of its band)
//     by bulk copies (no tensor map) into a ring of SA slots, which the MMA
//     completion releases. No multicast anywhere.
//   warps 1-4: converters. Each FP64 value is split into hi/lo TF32 and
//     written to one of NB operand buffers in the canonical K-major layout,
//     i.e. transposed on the way. (The field's natural order would be the
//     MN-major operand form, but kind::tf32 with B MN-major, no swizzle, left
//     the accumulators at zero on B200 in a one-MMA probe, while the K-major
//     form was exact.)
//   warp 5, one lane: issues the MMAs and commits each chunk to the
//     mbarriers that release its operator slot and operand buffer, and each
//     tile to the one the epilogue waits on.
//   warps 6-9: the epilogue, one TMEM lane quadrant each: tcgen05.ld of the
//     accumulators, FP32 stores, then the tile's accumulator set is released.
// Chunks in which an M-tile's rows of Mop are below 2^-40 of its largest
// entry (the inverse of the diagonally dominant tridiagonal decays
// geometrically away from the diagonal) are skipped for that M-tile. Every
// wait is bounded: on a timeout the CTA records OTBL_ERR_TIMEOUT, every role
// stops, the MMAs and copies in flight are waited for (bounded again), the
// tensor memory is freed and the CTA returns.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "devcommon.cuh"
#include "otbl_internal.cuh"
#include "tma.cuh"

namespace otbl {

namespace {

constexpr int YD_KC = 16;                      // input rows per K-chunk
constexpr int YD_WARPS = 11;                   // 2 producers, 4 converters, MMA, 4 epilogue
constexpr int YD_THREADS = 32 * YD_WARPS;
constexpr int YD_A_PART = 128 * YD_KC * 4;     // one M-tile, one part: 8 KB
constexpr int YD_A_CHUNK = 4 * YD_A_PART;      // 2 M-tiles x 2 parts: 32 KB
constexpr int YD_SMEM_MAX = 227 * 1024;
constexpr int YD_SA = 2;                       // operator ring slots
constexpr int YD_NBUF = 4;                     // operand buffers (hi and lo parts)
constexpr int YD_MAX_SF = 8;                   // field ring slots, at most
constexpr uint32_t YD_TMEM_COLS = 512;
constexpr uint64_t YD_WAIT_NS = 2000000000ull;  // 2 s

// bytes of one field box and of one operand buffer (hi and lo parts) for
// tiles of nt columns
__host__ __device__ constexpr int yd_fp_bytes(int nt) { return nt * YD_KC * 8; }
__host__ __device__ constexpr int yd_bbuf_bytes(int nt) { return 2 * nt * YD_KC * 4; }
constexpr int YD_BAR_BYTES = 1024;

// canonical K-major, no swizzle: element (m, k) of one M-tile part, k < 16
__host__ __device__ constexpr int yd_a_off(int m, int k) {
  return (m & 7) * 16 + (m >> 3) * (YD_KC / 4 * 128) + (k >> 2) * 128 + (k & 3) * 4;
}
// the field chunk in the same K-major form: element (n, k) of one part, k < 16
__host__ __device__ constexpr int yd_b_off(int n, int k) {
  return (n & 7) * 16 + (n >> 3) * (YD_KC / 4 * 128) + (k >> 2) * 128 + (k & 3) * 4;
}
static_assert(yd_a_off(127, 15) + 4 == YD_A_PART, "A part layout");
static_assert(yd_b_off(255, 15) + 4 == 256 * YD_KC * 4, "B part layout");

// shared-memory matrix descriptor (sm_100): start, LBO, SBO in 16-byte
// units, version 1, no swizzle
__device__ __forceinline__ uint64_t yd_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
// instruction descriptor, kind::tf32: F32 accumulator, A and B K-major
__host__ __device__ constexpr uint32_t yd_idesc(int M, int N) {
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

struct YDenseArgs {
  float *out[3];          // u, w, v interpolants, ny rows per plane
  const uint32_t *op[3];  // each field's operator chunks: [chunk][mt][part][YD_A_PART bytes]
  int kb[3][2], ke[3][2];  // per field and M-tile, the chunks [kb, ke) that carry its band
  int c0[3], c1[3];       // per field, the chunks a tile runs through
  int nt, nb, sf;         // tile columns, tiles per plane, field ring slots
  int tiles;              // tiles per field: nx * nb
};

namespace {
// the smem of the CTA, from a 1024-byte aligned base: SA operator slots, SF
// field slots, YD_NBUF operand buffers (hi part, lo part), the barriers
struct YdSmem {
  unsigned char *base;
  int nt, sf;
  __device__ unsigned char *op(int s) const { return base + (size_t)s * YD_A_CHUNK; }
  __device__ unsigned char *fp(int s) const { return op(YD_SA) + (size_t)s * yd_fp_bytes(nt); }
  __device__ unsigned char *bb(int b) const { return fp(sf) + (size_t)b * yd_bbuf_bytes(nt); }
  __device__ uint64_t *bars() const { return reinterpret_cast<uint64_t *>(bb(YD_NBUF)); }
};
// barrier slots
enum {
  YB_FPFULL = 0,                       // [YD_MAX_SF] field box landed (TMA bytes)
  YB_FPEMPTY = YB_FPFULL + YD_MAX_SF,  // [YD_MAX_SF] converters read it (128 arrivals)
  YB_OPFULL = YB_FPEMPTY + YD_MAX_SF,  // [YD_SA] operator chunk landed
  YB_OPEMPTY = YB_OPFULL + YD_SA,      // [YD_SA] its MMAs completed
  YB_BFULL = YB_OPEMPTY + YD_SA,       // [YD_NBUF] operand written (128 arrivals)
  YB_BEMPTY = YB_BFULL + YD_NBUF,      // [YD_NBUF] its MMAs completed
  YB_TFULL = YB_BEMPTY + YD_NBUF,      // [2] accumulator set complete
  YB_TEMPTY = YB_TFULL + 2,            // [2] accumulator set read (128 arrivals)
  YB_DRAIN = YB_TEMPTY + 2,
  YB_COUNT
};

__device__ __forceinline__ bool yd_wait(uint64_t *bar, unsigned parity, volatile int *abort_flag, int *err) {
  if (*abort_flag) return false;
  if (mbar_wait_bounded(bar, parity, YD_WAIT_NS)) return true;
  atomicExch(err, OTBL_ERR_TIMEOUT);
  *abort_flag = 1;
  return false;
}
__device__ __forceinline__ void yd_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
// after a timeout: the copies this thread issued into a ring of n slots
// (issued = how many) land before the CTA leaves
__device__ void yd_drain_ring(uint64_t *full, int n, unsigned issued) {
  for (int s = 0; s < n; ++s) {
    if (issued <= (unsigned)s) continue;
    const unsigned last = issued - 1 - (unsigned)(((int)((issued - 1) % n) - s + n) % n);  // last q, q % n == s
    mbar_wait_bounded(&full[s], (last / n) & 1, YD_WAIT_NS);
  }
}
}  // namespace

__global__ void __launch_bounds__(YD_THREADS, 1)
    k_ydense(int nx, int ny, int nz1, YDenseArgs a, int *err, const __grid_constant__ YDenseMaps maps) {
  extern __shared__ __align__(1024) unsigned char ydsm[];
  YdSmem sm;
  sm.base = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(ydsm) + 1023) & ~(uintptr_t)1023);
  sm.nt = a.nt;
  sm.sf = a.sf;
  uint64_t *bar = sm.bars();
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar + YB_COUNT);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int NT = a.nt, SF = a.sf, total = 3 * a.tiles;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(YD_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (t == 32) {
    for (int s = 0; s < YD_MAX_SF; ++s) {
      mbar_init(&bar[YB_FPFULL + s], 1);
      mbar_init(&bar[YB_FPEMPTY + s], 128);
    }
    for (int s = 0; s < YD_SA; ++s) {
      mbar_init(&bar[YB_OPFULL + s], 1);
      mbar_init(&bar[YB_OPEMPTY + s], 1);
    }
    for (int b = 0; b < YD_NBUF; ++b) {
      mbar_init(&bar[YB_BFULL + b], 128);
      mbar_init(&bar[YB_BEMPTY + b], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&bar[YB_TFULL + b], 1);
      mbar_init(&bar[YB_TEMPTY + b], 128);
    }
    mbar_init(&bar[YB_DRAIN], 1);
    *abort_flag = 0;
    mbar_init_fence();
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    // ---- field producer ----
    if (lane == 0) {
      unsigned q = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < total && ok && !*abort_flag; tile += gridDim.x) {
        const int fi = tile / a.tiles, rem = tile - fi * a.tiles, i = rem / a.nb, b = rem - i * a.nb;
        for (int kc = a.c0[fi]; kc < a.c1[fi]; ++kc, ++q) {
          const int s = (int)(q % SF);
          if (q >= (unsigned)SF && !yd_wait(&bar[YB_FPEMPTY + s], ((q / SF) - 1) & 1, abort_flag, err)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&bar[YB_FPFULL + s], yd_fp_bytes(NT));
          tma_load_3d(sm.fp(s), &maps.g[fi], b * NT, kc * YD_KC, i, &bar[YB_FPFULL + s]);
        }
      }
      yd_drain_ring(&bar[YB_FPFULL], SF, q);
    }
  } else if (warp == 10) {
    // ---- operator producer ----
    if (lane == 0) {
      unsigned q = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < total && ok && !*abort_flag; tile += gridDim.x) {
        const int fi = tile / a.tiles;
        for (int kc = a.c0[fi]; kc < a.c1[fi]; ++kc, ++q) {
          const int s = (int)(q % YD_SA);
          if (q >= (unsigned)YD_SA && !yd_wait(&bar[YB_OPEMPTY + s], ((q / YD_SA) - 1) & 1, abort_flag, err)) {
            ok = false;
            break;
          }
          const bool m0 = kc >= a.kb[fi][0] && kc < a.ke[fi][0], m1 = kc >= a.kb[fi][1] && kc < a.ke[fi][1];
          const unsigned char *opc = reinterpret_cast<const unsigned char *>(a.op[fi]) + (size_t)kc * YD_A_CHUNK;
          if (m0 || m1) {
            mbar_arrive_expect_tx(&bar[YB_OPFULL + s], (m0 + m1) * (YD_A_CHUNK / 2));
            if (m0) yd_bulk_g2s(sm.op(s), opc, YD_A_CHUNK / 2, &bar[YB_OPFULL + s]);
            if (m1) yd_bulk_g2s(sm.op(s) + YD_A_CHUNK / 2, opc + YD_A_CHUNK / 2, YD_A_CHUNK / 2, &bar[YB_OPFULL + s]);
          } else {
            yd_arrive(&bar[YB_OPFULL + s]);  // no part of this chunk is used
          }
        }
      }
      yd_drain_ring(&bar[YB_OPFULL], YD_SA, q);
    }
  } else if (warp <= 4) {
    // ---- converters: FP64 box -> hi/lo TF32, K-major ----
    const int ct = t - 32;
    unsigned q = 0;
    bool ok = true;
    for (int tile = blockIdx.x; tile < total && ok && !*abort_flag; tile += gridDim.x) {
      const int fi = tile / a.tiles;
      for (int kc = a.c0[fi]; kc < a.c1[fi]; ++kc, ++q) {
        const int s = (int)(q % SF), bs = (int)(q % YD_NBUF);
        if (!yd_wait(&bar[YB_FPFULL + s], (q / SF) & 1, abort_flag, err) ||
            (q >= YD_NBUF && !yd_wait(&bar[YB_BEMPTY + bs], ((q / YD_NBUF) - 1) & 1, abort_flag, err))) {
          ok = false;
          break;
        }
        const double *fp = reinterpret_cast<const double *>(sm.fp(s));
        unsigned char *hi = sm.bb(bs), *lo = hi + NT * YD_KC * 4;
#pragma unroll
        for (int g = 0; g < YD_KC / 4; ++g)
          for (int n = ct; n < NT; n += 128) {
            uint32_t h[4], l[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
              const double x = fp[(size_t)(4 * g + r) * NT + n];
              h[r] = yd_tf32((float)x);
              l[r] = yd_tf32((float)(x - (double)__uint_as_float(h[r])));
            }
            const int off = yd_b_off(n, 4 * g);
            *reinterpret_cast<uint4 *>(hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
            *reinterpret_cast<uint4 *>(lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
          }
        yd_arrive(&bar[YB_FPEMPTY + s]);  // the box has been read
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        yd_arrive(&bar[YB_BFULL + bs]);
      }
    }
  } else if (warp == 5) {
    // ---- MMA issue ----
    if (lane == 0) {
      const uint32_t idesc = yd_idesc(128, NT);
      unsigned q = 0, tl = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < total && ok && !*abort_flag; tile += gridDim.x, ++tl) {
        const int fi = tile / a.tiles, ab = (int)(tl & 1);
        if (tl >= 2 && !yd_wait(&bar[YB_TEMPTY + ab], ((tl >> 1) - 1) & 1, abort_flag, err)) break;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        for (int kc = a.c0[fi]; kc < a.c1[fi]; ++kc, ++q) {
          const int so = (int)(q % YD_SA), bs = (int)(q % YD_NBUF);
          if (!yd_wait(&bar[YB_OPFULL + so], (q / YD_SA) & 1, abort_flag, err) ||
              !yd_wait(&bar[YB_BFULL + bs], (q / YD_NBUF) & 1, abort_flag, err)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          const uint32_t sa_u = smem_u32(sm.op(so)), sb_u = smem_u32(sm.bb(bs));
#pragma unroll
          for (int mt = 0; mt < 2; ++mt) {
            if (kc < a.kb[fi][mt] || kc >= a.ke[fi][mt]) continue;
            const uint32_t d = tmem + (uint32_t)(ab * 256 + mt * NT);
#pragma unroll
            for (int ks = 0; ks < YD_KC / 8; ++ks) {
              const uint32_t ah = sa_u + (uint32_t)((mt * 2 + 0) * YD_A_PART + ks * 256);
              const uint32_t al = sa_u + (uint32_t)((mt * 2 + 1) * YD_A_PART + ks * 256);
              const uint32_t bh = sb_u + (uint32_t)(ks * 256), bl = bh + (uint32_t)(NT * YD_KC * 4);
              const uint64_t dah = yd_desc(ah, 128, YD_KC / 4 * 128), dal = yd_desc(al, 128, YD_KC / 4 * 128);
              const uint64_t dbh = yd_desc(bh, 128, YD_KC / 4 * 128), dbl = yd_desc(bl, 128, YD_KC / 4 * 128);
              const uint32_t first = (kc == a.kb[fi][mt] && ks == 0) ? 0u : 1u;
              yd_mma(d, dah, dbh, idesc, first);
              yd_mma(d, dah, dbl, idesc, 1u);
              yd_mma(d, dal, dbh, idesc, 1u);
            }
          }
          yd_commit(&bar[YB_OPEMPTY + so]);
          yd_commit(&bar[YB_BEMPTY + bs]);
        }
        if (!ok) break;
        yd_commit(&bar[YB_TFULL + ab]);
      }
      // every MMA issued has completed before the tensor memory is freed
      yd_commit(&bar[YB_DRAIN]);
      mbar_wait_bounded(&bar[YB_DRAIN], 0, YD_WAIT_NS);
    }
  } else {
    // ---- epilogue: TMEM lane quadrant (warp % 4) ----
    const int qd = warp & 3;
    const bool vec4 = (nz1 & 3) == 0;
    unsigned tl = 0;
    for (int tile = blockIdx.x; tile < total && !*abort_flag; tile += gridDim.x, ++tl) {
      const int fi = tile / a.tiles, rem = tile - fi * a.tiles, i = rem / a.nb, b = rem - i * a.nb;
      const int ab = (int)(tl & 1);
      if (!yd_wait(&bar[YB_TFULL + ab], (tl >> 1) & 1, abort_flag, err)) break;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      float *out = a.out[fi];
#pragma unroll 1
      for (int mt = 0; mt < 2; ++mt) {
        const int r = mt * 128 + qd * 32 + lane;  // output row, 0-based
        const bool band = a.ke[fi][mt] > a.kb[fi][mt];
        float *orow = out + ((size_t)i * ny + (r < ny ? r : 0)) * nz1;
        const uint32_t tbase = tmem + ((uint32_t)(qd * 32) << 16) + (uint32_t)(ab * 256 + mt * NT);
#pragma unroll 1
        for (int cb = 0; cb < NT; cb += 16) {
          uint32_t v[16];
          yd_tmem_ld16(tbase + (uint32_t)cb, v);
          const int kr0 = b * NT + cb;
          if (r < ny && kr0 < nz1) {
            if (vec4) {
#pragma unroll
              for (int p = 0; p < 16; p += 4)
                if (kr0 + p < nz1)
                  *reinterpret_cast<float4 *>(orow + kr0 + p) =
                      band ? make_float4(__uint_as_float(v[p]), __uint_as_float(v[p + 1]), __uint_as_float(v[p + 2]),
                                         __uint_as_float(v[p + 3]))
                           : make_float4(0.f, 0.f, 0.f, 0.f);
            } else {
#pragma unroll
              for (int p = 0; p < 16; p += 2)
                if (kr0 + p < nz1)
                  *reinterpret_cast<float2 *>(orow + kr0 + p) =
                      band ? make_float2(__uint_as_float(v[p]), __uint_as_float(v[p + 1])) : make_float2(0.f, 0.f);
            }
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      yd_arrive(&bar[YB_TEMPTY + ab]);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
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

// tile columns: nb = ceil(nz1/128) tiles per plane of nt = nz1/nb columns
// rounded up to 16 (the MMA's N); two M-tiles of nt columns make one of the
// two 256-column accumulator sets
static void ydense_tiling(int nz1, int *nt, int *nb) {
  *nb = (nz1 + 127) / 128;
  *nt = ((nz1 + *nb - 1) / *nb + 15) / 16 * 16;
}

// field ring slots that fit beside the operator ring and the operand buffers
static int ydense_field_slots(int nt) {
  const int room = YD_SMEM_MAX - 1024 - YD_SA * YD_A_CHUNK - YD_NBUF * yd_bbuf_bytes(nt) - YD_BAR_BYTES;
  return std::min(YD_MAX_SF, room / yd_fp_bytes(nt));
}

static size_t ydense_smem(int nt, int sf) {
  return 1024 + (size_t)YD_SA * YD_A_CHUNK + (size_t)sf * yd_fp_bytes(nt) + YD_NBUF * (size_t)yd_bbuf_bytes(nt) +
         YD_BAR_BYTES;
}

void *tensor_map_encoder();

bool build_ydense_maps(otbl_ctx *c) {
  c->yd_maps_ok = false;
  if (!c->ydense) return false;
  const int nx = c->cfg.nx, ny = c->cfg.ny, nz1 = c->dc.nz1;
  ydense_tiling(nz1, &c->yd_nt, &c->yd_nb);
  auto fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
  if (!fn || (nz1 * 8) % 16 != 0) return false;
  const double *in[3] = {c->f[OTBL_F_U], c->f[OTBL_F_W], c->f[OTBL_F_V]};
  const int rows[3] = {ny + 1, ny + 1, ny};
  for (int f = 0; f < 3; ++f) {
    if (reinterpret_cast<uintptr_t>(in[f]) % 16 != 0) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)nz1, (cuuint64_t)rows[f], (cuuint64_t)nx};
    const cuuint64_t strides[2] = {(cuuint64_t)nz1 * 8, (cuuint64_t)rows[f] * nz1 * 8};
    const cuuint32_t box[3] = {(cuuint32_t)c->yd_nt, (cuuint32_t)YD_KC, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    if (fn(&c->yd_maps.g[f], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double *>(in[f]), dims, strides, box, es,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
  }
  c->yd_maps_ok = true;
  return true;
}

// false when the dense path cannot run on this context (its TMA descriptors
// could not be made); the caller then runs the banded interpyy
bool ydense_ready(const otbl_ctx *c) { return c->ydense && c->yd_maps_ok && c->yd_op; }

cudaError_t launch_interpy_dense(otbl_ctx *c) {
  cudaStream_t s = c->stream;
  const int nx = c->cfg.nx, ny = c->cfg.ny, nz1 = c->dc.nz1;
  YDenseArgs a;
  void *outs[3] = {c->w.uy, c->w.wy, c->w.vy};
  const int which[3] = {0, 0, 1};
  for (int f = 0; f < 3; ++f) {
    a.out[f] = static_cast<float *>(outs[f]);
    a.op[f] = c->yd_op + which[f] * c->yd_words_per_op;
    int c0 = 1 << 30, c1 = 0;
    for (int mt = 0; mt < 2; ++mt) {
      a.kb[f][mt] = c->yd_kb[which[f]][mt];
      a.ke[f][mt] = c->yd_ke[which[f]][mt];
      if (a.ke[f][mt] > a.kb[f][mt]) {
        c0 = std::min(c0, a.kb[f][mt]);
        c1 = std::max(c1, a.ke[f][mt]);
      }
    }
    if (c1 == 0) c0 = 0;
    a.c0[f] = c0;
    a.c1[f] = c1;
  }
  a.nt = c->yd_nt;
  a.nb = c->yd_nb;
  a.sf = ydense_field_slots(a.nt);
  a.tiles = nx * a.nb;
  static int nsm = 0;
  if (nsm == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (nsm <= 0) nsm = 148;
  }
  const int grid = std::min(3 * a.tiles, nsm);
  const size_t smem = ydense_smem(a.nt, a.sf);
  cudaFuncSetAttribute(k_ydense, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_ydense<<<grid, YD_THREADS, smem, s>>>(nx, ny, nz1, a, &c->st->err, c->yd_maps);
  c->launches += 1;
  return cudaGetLastError();
}

}  // namespace otbl
