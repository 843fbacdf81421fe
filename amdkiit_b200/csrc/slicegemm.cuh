// Integer-slice GEMMs on the tcgen05 tensor cores (sm_100a) for the Gram and
// rotation products of the mixed-precision path: the overlap S = C0^T C0 and
// Lambda = C2^T C0 (OVLAP_D, wfn_initialize.f90:234-263; ortho_gs :481), and
// the rotations C2 -= C0 Lambda (gradient.f90:31) and C0 U^{-1} (ortho_gs
// DTRMM, wfn_initialize.f90:485).
//
// Method (the split-integer scheme of Ozaki et al., Numer. Algorithms 59, 95
// (2012), with Ootomo-Ozaki-Yokota's int8 tensor-core variant, IJHPCA 2024):
// every row r of an operand (a band) is scaled by a power of two sigma_r so
// that |x| / sigma_r < 1/2, rounded to the fixed-point integer
// v = rint(x / sigma_r 2^{7S}) (|v| <= 2^{7S-1}) and cut into S balanced
// base-128 digits,
//   x / sigma_r = sum_t d_t 2^{-7(t+1)} + O(2^{-7S}),  d_t in [-64, 64].
// A product of two rows is
//   sum_k x_k y_k = sigma_x sigma_y sum_{t,u} 2^{-7(t+u+2)} sum_k dx_t dy_u,
// whose inner sums are exact int8 x int8 -> int32 tensor-core products; the
// terms with t + u >= S are dropped (relative truncation ~2^{-7S}), and the
// pairs with equal t + u share one int32 accumulator in tensor memory (S
// accumulators of 128 x 128 = all 512 TMEM columns).  With S = 4 each operand
// keeps 28 bits and the accumulation is exact; the dropped pairs leave a
// product error of about 2^-21 |x||y|, that of an FP32 GEMM of the same rows.
//
// Planes: int8 [S][128 rows][kpad], row r = band r (zero rows above the band
// count), kpad = the real length 2*ngpw rounded up to 128 with zeros.  TMA
// loads 64-byte (TN) or 128-byte (NN) swizzled tiles straight into the
// canonical UMMA shared-memory layouts.
//
// TN (C = A B^T over the long real index, A and B K-major): one CTA per
// chunk of 64-wide k tiles, 3-stage TMA -> MMA pipeline on mbarriers, one
// thread issues the MMAs, four warps read the accumulators back and write an
// FP64 partial; k_sgemm_reduce sums the partials and applies the scales.
// NN (C[m][n] = sum_k A[m][k] B[k][n], A = the band planes read MN-major,
// B a 128 x 128 matrix sliced per column after scaling its rows by the A
// bands' sigma): persistent CTAs over 128-row tiles of the long index, the
// epilogue writes (or subtracts from) FP64 output.
//
// Every wait is bounded: on expiry the kernel records a code in *err, writes
// NaN where its result would go, waits for its own copies and MMAs in flight,
// frees its tensor memory and returns.  The pipeline waits (a stage's data,
// a free stage, the accumulators of a tile) give up after plim polls (a
// kernel argument, SG_SPIN normally, smaller to test the expiry path); the
// drains of a block's own copies and MMAs always allow SG_SPIN polls.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace amdk {

constexpr int SG_S = 4;          // digit planes per operand
constexpr int SG_M = 128;        // rows per plane (bands, padded)
constexpr int SG_TN_KT = 64;     // k bytes per TN stage (64-byte swizzle)
constexpr int SG_TN_ST = 3;      // TN pipeline stages
constexpr int SG_NN_ST = 2;      // NN pipeline stages
constexpr int SG_TMEM_COLS = 512;
constexpr long SG_SPIN = 1L << 22;

// ------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t sg_smem(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void sg_bar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void sg_bar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void sg_bar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void sg_bar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool sg_bar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait for the phase of the given parity; false (and *err = code)
// after limit polls (limit <= 0: at once, without polling)
__device__ __forceinline__ bool sg_bar_wait(uint32_t bar, uint32_t parity, int *err, int code, long limit = SG_SPIN) {
  for (long it = 0; it < limit; ++it) {
    if (sg_bar_try(bar, parity)) return true;
    if (it > 32) __nanosleep(64);
  }
  atomicExch(err, code);
  return false;
}
__device__ __forceinline__ void sg_tma_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void sg_tmem_alloc(uint32_t slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void sg_tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void sg_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void sg_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// D[tmem] (+)= A[smem] B[smem]^T, 128 x 128 x 32 int8 -> int32
__device__ __forceinline__ void sg_mma_i8(uint32_t dtm, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtm),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
      : "memory");
}
// arrive on the mbarrier once every MMA issued so far by this thread is done
__device__ __forceinline__ void sg_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
// 16 consecutive 32-bit columns of this thread's TMEM lane; the registers
// are valid after sg_tmem_wait_ld (several loads may share one wait)
__device__ __forceinline__ void sg_tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void sg_tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}
__device__ __forceinline__ void sg_tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor (tcgen05): start address, leading and
// stride byte offsets (16-byte units), version 1, layout (2 = 128-byte
// swizzle, 4 = 64-byte swizzle).
__device__ __forceinline__ uint64_t sg_desc(uint32_t addr, uint32_t lbo, uint32_t sbo, uint32_t layout) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | ((uint64_t)layout << 61);
}
// Instruction descriptor, kind::i8: D s32 (bits 4-5 = 2), A and B signed
// (bits 7-9, 10-12 = 1), A MN-major (bit 15) when a_mn, B K-major, N = 128
// (bits 17-22 = N/8), M = 128 (bits 24-28 = M/16).
__host__ __device__ constexpr uint32_t sg_idesc(bool a_mn) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((128u >> 3) << 17) | ((128u >> 4) << 24);
}

// ---------------------------------------------------------------- slicing
// S balanced base-128 digits of y = x 2^{7S} / sigma (|y| < 2^{7S-1}), most
// significant first: rint(y) = sum_t d_t 128^{S-1-t}, d_t in [-64, 63]
// except d_0 in [-64, 64].
template <int S> __device__ __forceinline__ void sg_digits(double y, int (&d)[S]) {
  static_assert(S >= 1 && S <= 4, "the fixed-point value must fit 32 bits");
  int v = __double2int_rn(y);
#pragma unroll
  for (int t = S - 1; t > 0; --t) {
    const int q = ((v + 64) & 127) - 64;
    d[t] = q;
    v = (v - q) >> 7;
  }
  d[0] = v;
}
// Per-row max |x| of the bands (len reals at x + r*ldx) and the row's sum of
// squares by segment: grid (SG_SEG, nrows), block 256; bmax (as the bit
// patterns of non-negative doubles, which order like the values) must be
// cleared first; nsq[r * SG_SEG + segment].  The sums of squares give the
// exact diagonal of a Gram matrix A A^T: there the dropped digit products
// d_t d_u with t + u >= S include squares (t = u), which would bias it.
constexpr int SG_SEG = 8;  // blocks per band in the slicing passes
__global__ void __launch_bounds__(256) k_band_absmax(const double *__restrict__ x, long ldx, long len, int nrows,
                                                     unsigned long long *__restrict__ bmax, double *__restrict__ nsq) {
  const int r = blockIdx.y;
  if (r >= nrows) return;
  const long seg = (len / 2 + SG_SEG - 1) / SG_SEG * 2;  // even
  const long k0 = blockIdx.x * seg, k1 = min(len, k0 + seg);
  const double *xr = x + (long)r * ldx;
  double m = 0.0, q = 0.0;
  for (long k = k0 + 2L * threadIdx.x; k < k1; k += 2L * blockDim.x) {
    const double2 v = *reinterpret_cast<const double2 *>(xr + k);
    m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
    q = fma(v.x, v.x, fma(v.y, v.y, q));
  }
  for (int o = 16; o > 0; o >>= 1) {
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    q += __shfl_xor_sync(0xffffffffu, q, o);
  }
  __shared__ double red[8], rq[8];
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5] = m;
    rq[threadIdx.x >> 5] = q;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) {
      m = fmax(m, red[i]);
      q += rq[i];
    }
    atomicMax(bmax + r, (unsigned long long)__double_as_longlong(m));
    nsq[r * SG_SEG + blockIdx.x] = q;
  }
}
// Row r -> sigma_r = 2^e (max / 2^e < 1/2) and S digit planes; grid
// (SG_SEG, SG_M) over kpad (rows >= nrows are zero), block 256.
template <int S>
__global__ void __launch_bounds__(256) k_slice_rows(const double *__restrict__ x, long ldx, long len, int nrows,
                                                    const unsigned long long *__restrict__ bmax,
                                                    int8_t *__restrict__ planes, long kpad, double *__restrict__ scale) {
  const int r = blockIdx.y;
  const long pstride = (long)SG_M * kpad;
  const long seg = (kpad / 8 + SG_SEG - 1) / SG_SEG * 8;
  const long k0 = blockIdx.x * seg, k1 = min(kpad, k0 + seg);
  int8_t *dst = planes + (long)r * kpad;
  if (r >= nrows) {
    for (long k = k0 + 8L * threadIdx.x; k < k1; k += 8L * blockDim.x)
#pragma unroll
      for (int t = 0; t < S; ++t) *reinterpret_cast<uint2 *>(dst + t * pstride + k) = make_uint2(0u, 0u);
    if (blockIdx.x == 0 && threadIdx.x == 0) scale[r] = 1.0;
    return;
  }
  const double w = __longlong_as_double((long long)bmax[r]);
  int E = 0;
  if (w > 0.0) frexp(w, &E);  // w = f 2^E, f in [1/2, 1): w / 2^(E+1) < 1/2
  const int e = w > 0.0 ? E + 1 : 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) scale[r] = ldexp(1.0, e);
  const double sc = ldexp(1.0, 7 * S - e);  // x -> fixed point with 7S fraction bits
  const double *xr = x + (long)r * ldx;
  for (long k = k0 + 8L * threadIdx.x; k < k1; k += 8L * blockDim.x) {
    double v[8];
#pragma unroll
    for (int i = 0; i < 8; i += 2) {
      if (k + i < len) {
        const double2 q = *reinterpret_cast<const double2 *>(xr + k + i);
        v[i] = q.x;
        v[i + 1] = q.y;
      } else {
        v[i] = v[i + 1] = 0.0;
      }
    }
    uint32_t lo[S], hi[S];
#pragma unroll
    for (int t = 0; t < S; ++t) lo[t] = hi[t] = 0u;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      int d[S];
      sg_digits<S>(v[i] * sc, d);
#pragma unroll
      for (int t = 0; t < S; ++t) {
        const uint32_t b = (uint32_t)(uint8_t)(int8_t)d[t];
        if (i < 4) lo[t] |= b << (8 * i);
        else hi[t] |= b << (8 * (i - 4));
      }
    }
#pragma unroll
    for (int t = 0; t < S; ++t) *reinterpret_cast<uint2 *>(dst + t * pstride + k) = make_uint2(lo[t], hi[t]);
  }
}

// A small matrix B (nk x nn, column-major, ldb) for the NN product: column n
// of diag(rowscale) B -> tau_n and S digit planes [t][n][k] (K-major rows n).
// grid SG_M, block SG_M.
template <int S>
__global__ void __launch_bounds__(SG_M) k_slice_small(const double *__restrict__ B, int ldb, int nk, int nn,
                                                      const double *__restrict__ rowscale, int8_t *__restrict__ planes,
                                                      double *__restrict__ colscale) {
  const int n = blockIdx.x, k = threadIdx.x;
  const double v = (n < nn && k < nk) ? B[k + (long)ldb * n] * rowscale[k] : 0.0;
  double m = fabs(v);
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double red[SG_M / 32];
  if ((k & 31) == 0) red[k >> 5] = m;
  __syncthreads();
  double w = 0.0;
#pragma unroll
  for (int i = 0; i < SG_M / 32; ++i) w = fmax(w, red[i]);
  int E = 0;
  if (w > 0.0) frexp(w, &E);
  const int e = w > 0.0 ? E + 1 : 0;
  if (k == 0) colscale[n] = ldexp(1.0, e);
  int d[S];
  sg_digits<S>(v * ldexp(1.0, 7 * S - e), d);
#pragma unroll
  for (int t = 0; t < S; ++t) planes[(long)t * SG_M * SG_M + n * SG_M + k] = (int8_t)d[t];
}

__global__ void k_sg_fill(double *__restrict__ s, int n, double v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) s[i] = v;
}

// ------------------------------------------------------------------ TN GEMM
template <int S> struct SgTn {
  static constexpr int PLANE = SG_M * SG_TN_KT;  // 8 KB: 128 rows x 64 bytes
  static constexpr int STAGE = 2 * S * PLANE;
  static constexpr int SMEM = SG_TN_ST * STAGE + 1024 + 256;
};
// partial[chunk][n][m] = sum over the chunk's k of
//   sum_{t+u<S} 2^{-7(t+u+2)} dA_t[m][k] dB_u[n][k]
// (same != 0: B = A, loaded once).  grid = chunks, block SG_TN_THREADS:
// thread 0 loads, thread 32 issues the MMAs, all eight warps read the
// accumulators back (TMEM lanes 32 (w % 4) ..., columns 64 (w / 4) ...) and
// combine them exactly in 64-bit integers.
constexpr int SG_TN_THREADS = 256;
template <int S>
__global__ void __launch_bounds__(SG_TN_THREADS, 1) k_sgemm_tn(const __grid_constant__ CUtensorMap ta,
                                                     const __grid_constant__ CUtensorMap tb, int same, int ktiles,
                                                     int per_cta, double *__restrict__ partial, int *err,
                                                     long plim) {
  using G = SgTn<S>;
  __shared__ int aborted;  // a pipeline wait of this block expired
  extern __shared__ unsigned char sg_raw[];
  unsigned char *base = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(sg_raw) + 1023) & ~uintptr_t(1023));
  // a Gram product (same) stages A alone, so twice as many stages fit
  const int nst = same ? 2 * SG_TN_ST : SG_TN_ST;
  const int sbytes = (same ? 1 : 2) * S * G::PLANE;
  uint64_t *bars = reinterpret_cast<uint64_t *>(base + SG_TN_ST * G::STAGE);  // full[2 ST], empty[2 ST], done
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 4 * SG_TN_ST + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int kt0 = blockIdx.x * per_cta;
  const int nt = max(0, min(per_cta, ktiles - kt0));
  const uint32_t full0 = sg_smem(bars), empty0 = sg_smem(bars + 2 * SG_TN_ST), done = sg_smem(bars + 4 * SG_TN_ST);
  if (threadIdx.x == 0) {
    aborted = 0;
    for (int i = 0; i < 2 * SG_TN_ST; ++i) {
      sg_bar_init(full0 + 8 * i, 1);
      sg_bar_init(empty0 + 8 * i, 1);
    }
    sg_bar_init(done, 1);
    sg_bar_fence_init();
  }
  if (warp == 0) sg_tmem_alloc(sg_smem(tslot), SG_TMEM_COLS);
  sg_fence_before();
  __syncthreads();
  sg_fence_after();
  const uint32_t tbase = *tslot;
  const uint32_t bytes = (uint32_t)sbytes;
  if (threadIdx.x == 0 && nt > 0) {
    // producer: TMA of the S planes of A (and B) for each k tile
    int issued = 0;
    for (int i = 0; i < nt; ++i) {
      const int s = i % nst;
      if (i >= nst && !sg_bar_wait(empty0 + 8 * s, ((i / nst) - 1) & 1, err, 1, plim)) {
        aborted = 1;
        break;
      }
      const uint32_t fb = full0 + 8 * s;
      sg_bar_expect_tx(fb, bytes);
      const uint32_t dA = sg_smem(base + s * sbytes), dB = dA + S * G::PLANE;
      const int kx = (kt0 + i) * SG_TN_KT;
#pragma unroll
      for (int t = 0; t < S; ++t) sg_tma_2d(dA + t * G::PLANE, &ta, kx, t * SG_M, fb);
      if (!same)
#pragma unroll
        for (int t = 0; t < S; ++t) sg_tma_2d(dB + t * G::PLANE, &tb, kx, t * SG_M, fb);
      issued = i + 1;
    }
    // the copies in flight land before the block can leave
    for (int i = max(0, issued - nst); i < issued; ++i) sg_bar_wait(full0 + 8 * (i % nst), (i / nst) & 1, err, 4);
  } else if (threadIdx.x == 32 && nt > 0) {
    // MMA issuer
    constexpr uint32_t idesc = sg_idesc(false);
    for (int i = 0; i < nt; ++i) {
      const int s = i % nst;
      if (!sg_bar_wait(full0 + 8 * s, (i / nst) & 1, err, 2, plim)) {
        aborted = 1;
        break;
      }
      sg_fence_after();
      const uint32_t aA = sg_smem(base + s * sbytes), aB = same ? aA : aA + S * G::PLANE;
#pragma unroll
      for (int t = 0; t < S; ++t)
#pragma unroll
        for (int u = 0; u < S - t; ++u)
#pragma unroll
          for (int kk = 0; kk < SG_TN_KT / 32; ++kk) {
            const uint64_t ad = sg_desc(aA + t * G::PLANE + 32 * kk, 16, 512, 4);
            const uint64_t bd = sg_desc(aB + u * G::PLANE + 32 * kk, 16, 512, 4);
            sg_mma_i8(tbase + (uint32_t)((t + u) * SG_M), ad, bd, idesc, (i > 0 || t > 0 || kk > 0) ? 1u : 0u);
          }
      sg_commit(empty0 + 8 * s);
    }
    sg_commit(done);
    sg_bar_wait(done, 0, err, 5);  // every MMA of this block has finished
  }
  __syncthreads();  // the producer's copies and the issuer's MMAs have drained; `aborted` is final
  // epilogue: lane m of warp w holds row m = 32 (w % 4) + lane of every accumulator
  const bool ok = __all_sync(0xffffffffu, nt > 0 && !aborted && sg_bar_wait(done, 0, err, 3));
  sg_fence_after();
  const int ew = warp & 3, half = warp >> 2;
  const int m = 32 * ew + lane;
  const double w0 = ldexp(1.0, -7 * (S + 1));
  double *out = partial + (long)blockIdx.x * SG_M * SG_M;
  for (int cb = 4 * half; cb < 4 * half + 4; ++cb) {
    double v[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = 0.0;
    if (ok) {
      uint32_t r[S][16];
#pragma unroll
      for (int d = 0; d < S; ++d) sg_tmem_ld16(tbase + ((uint32_t)(32 * ew) << 16) + (uint32_t)(d * SG_M + 16 * cb), r[d]);
      sg_tmem_wait_ld();
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        long long t = (int)r[0][j];
#pragma unroll
        for (int d = 1; d < S; ++d) t = t * 128 + (int)r[d][j];
        v[j] = (double)t * w0;
      }
    } else if (nt > 0) {
#pragma unroll
      for (int j = 0; j < 16; ++j) v[j] = __longlong_as_double(0x7ff8000000000000LL);
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) out[(cb * 16 + j) * SG_M + m] = v[j];
  }
  sg_fence_before();
  __syncthreads();
  if (warp == 0) {
    sg_fence_after();
    sg_tmem_dealloc(tbase, SG_TMEM_COLS);
  }
}

// out[m + ldo n] = alpha sa[m] sb[n] sum_c partial[c][n][m], m < nm, n < nn;
// with nsq (a Gram matrix) the diagonal is alpha sum_seg nsq[m][seg] instead.
// grid nn, block SG_RG SG_M: SG_RG interleaved partial sums per row, fixed order.
constexpr int SG_RG = 8;
__global__ void __launch_bounds__(SG_RG * SG_M) k_sgemm_reduce(int nchunk, const double *__restrict__ partial, int nm,
                                                               const double *__restrict__ sa,
                                                               const double *__restrict__ sb,
                                                               const double *__restrict__ nsq, double alpha,
                                                               double *__restrict__ out, int ldo) {
  const int m = threadIdx.x % SG_M, g = threadIdx.x / SG_M, n = blockIdx.x;
  __shared__ double red[SG_RG][SG_M];
  double s = 0.0;
#pragma unroll 8
  for (int c = g; c < nchunk; c += SG_RG) s += partial[(long)c * SG_M * SG_M + n * SG_M + m];
  red[g][m] = s;
  __syncthreads();
  if (g == 0 && m < nm) {
    double t = 0.0;
#pragma unroll
    for (int i = 0; i < SG_RG; ++i) t += red[i][m];
    double v = alpha * sa[m] * sb[n] * t;
    if (nsq && m == n) {
      double q = 0.0;
      for (int i = 0; i < SG_SEG; ++i) q += nsq[m * SG_SEG + i];
      v = alpha * q;
    }
    out[m + (long)ldo * n] = v;
  }
}

// ------------------------------------------------------------------ NN GEMM
template <int S> struct SgNn {
  static constexpr int PLANE = SG_M * SG_M;  // 16 KB: 128 x 128 bytes
  static constexpr int SMEM = S * PLANE + SG_NN_ST * S * PLANE + 1024 + 256;
};
// out[m + ldo n] (=, or -= for MODE 1) colscale[n] sum_{t+u<S} 2^{-7(t+u+2)}
//   sum_k dA_t[k][m] dB_u[n][k]   for m < mreal, n < nn,
// A planes [t][k][m] (MN-major tiles of 128 m x 128 k), B planes [t][n][k].
// Persistent: CTA b takes the 128-row tiles b, b + grid, ...  block 576:
// warp 0 loads, warp 1 issues the MMAs (and owns the tensor memory), warps
// 2-17 read the accumulators back (TMEM lanes 32 (w % 4) ..., columns
// 32 ((w - 2) / 4) ...), 8 columns at a time with one TMEM wait for the S
// accumulators, which are combined exactly in 64-bit integers
// (sum_d acc_d 128^{S-1-d}, below 2^45) and converted once; the old values of
// a subtraction are loaded before the accumulators are read.  MODE 0 stores,
// 1 subtracts, 2 stores and also cuts the result into the S digit planes
// dig[t][n][m] with the fixed scale sigma = 2 (an orthonormalisation: its
// output bands satisfy |x| <= 1), ready as the next product's operand,
// setting its real index 1 (Im c(G=0)) to zero as ZCLEAN does.
constexpr int SG_NN_THREADS = 576;
template <int S, int MODE>
__global__ void __launch_bounds__(SG_NN_THREADS, 1) k_sgemm_nn(const __grid_constant__ CUtensorMap ta,
                                                     const __grid_constant__ CUtensorMap tb, int mtiles, long mreal,
                                                     double *__restrict__ out, long ldo, int nn,
                                                     const double *__restrict__ colscale,
                                                     int8_t *__restrict__ dig, long kpad, int *err, long plim) {
  using G = SgNn<S>;
  extern __shared__ unsigned char sg_raw[];
  unsigned char *base = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(sg_raw) + 1023) & ~uintptr_t(1023));
  unsigned char *sB = base;
  unsigned char *sA = base + S * G::PLANE;
  // bfull, full[ST], empty[ST], tfull, tfree, fin
  uint64_t *bars = reinterpret_cast<uint64_t *>(sA + SG_NN_ST * S * G::PLANE);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 4 + 2 * SG_NN_ST);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t bfull = sg_smem(bars), full0 = sg_smem(bars + 1), empty0 = sg_smem(bars + 1 + SG_NN_ST);
  const uint32_t tfull = sg_smem(bars + 1 + 2 * SG_NN_ST), tfree = sg_smem(bars + 2 + 2 * SG_NN_ST);
  const uint32_t fin = sg_smem(bars + 3 + 2 * SG_NN_ST);
  const int nq = blockIdx.x < mtiles ? (mtiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  __shared__ double cs[SG_M];  // colscale 2^{-7(S+1)}
  for (int i = threadIdx.x; i < SG_M; i += blockDim.x) cs[i] = i < nn ? ldexp(colscale[i], -7 * (S + 1)) : 0.0;
  if (threadIdx.x == 0) {
    sg_bar_init(bfull, 1);
    for (int i = 0; i < SG_NN_ST; ++i) {
      sg_bar_init(full0 + 8 * i, 1);
      sg_bar_init(empty0 + 8 * i, 1);
    }
    sg_bar_init(tfull, 1);
    sg_bar_init(tfree, (SG_NN_THREADS - 64) / 32);
    sg_bar_init(fin, 1);
    sg_bar_fence_init();
  }
  if (warp == 1) sg_tmem_alloc(sg_smem(tslot), SG_TMEM_COLS);
  sg_fence_before();
  __syncthreads();
  sg_fence_after();
  const uint32_t tbase = *tslot;
  if (threadIdx.x == 0 && nq > 0) {
    sg_bar_expect_tx(bfull, S * G::PLANE);
#pragma unroll
    for (int t = 0; t < S; ++t) sg_tma_2d(sg_smem(sB + t * G::PLANE), &tb, 0, t * SG_M, bfull);
    int issued = 0;
    for (int q = 0; q < nq; ++q) {
      const int s = q % SG_NN_ST;
      if (q >= SG_NN_ST && !sg_bar_wait(empty0 + 8 * s, ((q / SG_NN_ST) - 1) & 1, err, 11, plim)) break;
      const uint32_t fb = full0 + 8 * s;
      sg_bar_expect_tx(fb, S * G::PLANE);
      const int m0 = (blockIdx.x + q * gridDim.x) * SG_M;
#pragma unroll
      for (int t = 0; t < S; ++t) sg_tma_2d(sg_smem(sA + (s * S + t) * G::PLANE), &ta, m0, t * SG_M, fb);
      issued = q + 1;
    }
    sg_bar_wait(bfull, 0, err, 14);
    for (int q = max(0, issued - SG_NN_ST); q < issued; ++q)
      sg_bar_wait(full0 + 8 * (q % SG_NN_ST), (q / SG_NN_ST) & 1, err, 14);
  } else if (threadIdx.x == 32 && nq > 0) {
    constexpr uint32_t idesc = sg_idesc(true);
    bool ok = sg_bar_wait(bfull, 0, err, 12, plim);
    for (int q = 0; q < nq && ok; ++q) {
      const int s = q % SG_NN_ST;
      if (!sg_bar_wait(full0 + 8 * s, (q / SG_NN_ST) & 1, err, 12, plim)) break;
      if (q > 0 && !sg_bar_wait(tfree, (q - 1) & 1, err, 13, plim)) break;
      sg_fence_after();
      const uint32_t aA = sg_smem(sA + s * S * G::PLANE), aB = sg_smem(sB);
#pragma unroll
      for (int t = 0; t < S; ++t)
#pragma unroll
        for (int u = 0; u < S - t; ++u)
#pragma unroll
          for (int kk = 0; kk < SG_M / 32; ++kk) {
            // A: 32 k rows of 128 bytes per MMA (four 8-row swizzle atoms)
            const uint64_t ad = sg_desc(aA + t * G::PLANE + 4096 * kk, G::PLANE, 1024, 2);
            const uint64_t bd = sg_desc(aB + u * G::PLANE + 32 * kk, 16, 1024, 2);
            sg_mma_i8(tbase + (uint32_t)((t + u) * SG_M), ad, bd, idesc, (t > 0 || kk > 0) ? 1u : 0u);
          }
      sg_commit(empty0 + 8 * s);
      sg_commit(tfull);
    }
    sg_commit(fin);
    sg_bar_wait(fin, 0, err, 16);  // every MMA of this block has finished
  } else if (warp >= 2) {
    const int ew = warp & 3, cg = (warp - 2) >> 2;
    const int m = 32 * ew + lane;
    for (int q = 0; q < nq; ++q) {
      const bool ok = __all_sync(0xffffffffu, sg_bar_wait(tfull, q & 1, err, 15, plim));
      sg_fence_after();
      const long gm = (long)(blockIdx.x + q * gridDim.x) * SG_M + m;
      const bool row_ok = gm < mreal;
#pragma unroll 1
      for (int cb = 4 * cg; cb < 4 * cg + 4; ++cb) {
        double old[8];
        if (MODE == 1 && row_ok) {
#pragma unroll
          for (int j = 0; j < 8; ++j) old[j] = (8 * cb + j < nn) ? out[(long)(8 * cb + j) * ldo + gm] : 0.0;
        }
        double v[8];
        if (ok) {
          uint32_t r[S][8];
#pragma unroll
          for (int d = 0; d < S; ++d) sg_tmem_ld8(tbase + ((uint32_t)(32 * ew) << 16) + (uint32_t)(d * SG_M + 8 * cb), r[d]);
          sg_tmem_wait_ld();
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            long long t = (int)r[0][j];
#pragma unroll
            for (int d = 1; d < S; ++d) t = t * 128 + (int)r[d][j];
            v[j] = (double)t * cs[8 * cb + j];
          }
        } else {
#pragma unroll
          for (int j = 0; j < 8; ++j) v[j] = __longlong_as_double(0x7ff8000000000000LL);
        }
        if (row_ok) {
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int n = 8 * cb + j;
            double val = v[j];
            if (MODE == 1) val = old[j] - val;
            if (MODE == 2) {
              val = (gm == 1) ? 0.0 : val;
              int dd[S];
              sg_digits<S>(val * (double)(1 << (7 * S - 1)), dd);
              if (n < nn) {
#pragma unroll
                for (int t = 0; t < S; ++t) dig[((long)t * SG_M + n) * kpad + gm] = (int8_t)dd[t];
              }
            }
            if (n < nn) out[(long)n * ldo + gm] = val;
          }
        }
      }
      sg_fence_before();
      __syncwarp();
      if (lane == 0) sg_bar_arrive(tfree);
      if (!ok) break;
    }
  }
  sg_fence_before();
  __syncthreads();
  if (warp == 1) {
    sg_fence_after();
    sg_tmem_dealloc(tbase, SG_TMEM_COLS);
  }
}

}  // namespace amdk
