// FP64 products of the band space on the FP64 tensor cores (DMMA,
// mma.sync.m8n8k4.f64), fed by TMA: the FP64 path's overlap S = 2 C0^T C0
// (ortho_gs DSYRK, wfn_initialize.f90:481), Lambda = 2 C2^T C0 (OVLAP_D,
// wfn_initialize.f90:234-263), the projections nl = 2 P^T C0
// (pseudopotential.f90:211-213) and dfnl = 2 tpiba Q^T C0
// (nuclear_grad.f90:135,359), and the rotations C2 -= C0 Lambda
// (gradient.f90:31) and C0 U^{-1} (ortho_gs DTRMM, wfn_initialize.f90:485).
// tcgen05 has no FP64 kind, so these are warp-level MMAs; every product is
// exact FP64 arithmetic (a fused multiply-add chain per output in a fixed
// order), like the DGEMM calls of the reference.
//
// TN (out = alpha A^T B over the long real index K; A is K x m and B is
// K x n, both column-major with leading dimension K): output tiles of 64 x 64,
// the K range split over enough blocks to fill the GPU; one copy warp streams
// 16-wide k tiles of A and B (128-byte swizzled TMA boxes of 16 x 64) through a
// 4-stage mbarrier pipeline, four MMA warps each own a 32 x 32 quarter of the
// tile.  The partial tiles go to a buffer that k_dgemm_tn_sum adds up in
// split order (deterministic).  With sym only the tiles on and above the
// diagonal are formed and the sum mirrors them (S is symmetric).
//
// NN (out = alpha A G + beta out; A is K x n1 column-major, G is n1 x n
// column-major): persistent blocks over work items of 64 rows of the long
// index x 128 output columns, eight warps each owning 32 rows x 32
// columns; per 64-band half chunk, A arrives in four TMA boxes of 16 rows x
// 64 bands through a 2-stage pipeline and the 64 x 128 slice of G by cp.async
// into one of two buffers (kept for the whole kernel when G is at most
// 128 x 128).  With upper, G is
// upper triangular (U^{-1}): band blocks below a column block are skipped and
// the lower part of G is read as zero.
//
// Fragment layouts (PTX ISA, mma.m8n8k4 with .f64): A (8 x 4, row) one value
// per thread at row lane/4, column lane%4; B (4 x 8, col) row lane%4, column
// lane/4; C (8 x 8) two values at row lane/4, columns 2 (lane%4) + {0, 1}.
// Each thread reads 16 bytes of shared memory at a time: in TN the two values
// are consecutive k and serve two MMA steps (step s of half kb takes
// k = 4 t + 2 kb + s, the same set for A and B, so that the eight lanes of a
// quarter warp read eight different 16-byte bank groups of the swizzled
// rows); in NN they are consecutive rows of the long index and serve two row
// tiles (rows 2 g and 2 g + 1), from 128-byte-swizzled boxes as well.
//
// Waits are bounded as in the integer-slice kernels: a pipeline wait gives up
// after plim polls, sets *err and the shared abort flag; the block then runs
// its loops to the end without waiting (so every warp reaches the same
// barriers), the copy warp waits (SG_SPIN polls) for its own copies in
// flight, and the results are written as NaN.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "slicegemm.cuh"

namespace amdk {

constexpr int DG_T = 64;    // TN output tile
constexpr int DG_KT = 16;   // doubles per TN k tile (one 128-byte row)
constexpr int DG_ST = 4;    // TN stages
constexpr int DG_THREADS = 160;  // TN: 4 MMA warps + 1 copy warp
constexpr int DG_TN_STAGE = 2 * DG_T * DG_KT * 8;  // A and B boxes, 16 KB
constexpr int DG_TN_SMEM = DG_ST * DG_TN_STAGE + 1024 + 2 * DG_ST * 8;
constexpr int DG_NN_R = 64;    // rows of the long index per work item
constexpr int DG_NN_B = 128;   // bands per staged G chunk
constexpr int DG_NN_BS = 64;   // bands per A stage
constexpr int DG_NN_J = 128;   // output columns per work item
constexpr int DG_NN_GLD = DG_NN_BS + 8;  // padded row of a staged G slice (doubles): rows
                                         // g and g + 1 half a bank line apart
constexpr int DG_NN_ST = 2;
constexpr int DG_NN_THREADS = 256;  // 8 MMA warps (thread 0 also issues the copies)
constexpr int DG_NN_BOX = 16 * DG_NN_BS * 8;   // one TMA box, 16 rows x 64 bands, 8 KB
constexpr int DG_NN_STAGE = 4 * DG_NN_BOX;     // 64 rows, 32 KB
constexpr int DG_NN_SMEM = DG_NN_ST * DG_NN_STAGE + 2 * DG_NN_J * DG_NN_GLD * 8 + 1024 + 2 * DG_NN_ST * 8;

__device__ __forceinline__ void dg_mma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}
// 16 bytes (16-byte chunk `chunk` of row `row`) of a 128-byte-swizzled tile
// of 128-byte rows (the tile 1024-byte aligned)
__device__ __forceinline__ double2 dg_ld_sw(const unsigned char *tile, int row, int chunk) {
  return *reinterpret_cast<const double2 *>(tile + row * 128 + ((chunk ^ (row & 7)) << 4));
}
__device__ __forceinline__ unsigned char *dg_align1k(unsigned char *p) {
  return reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(p) + 1023) & ~(uintptr_t)1023);
}
// tile index -> (it, jt): column-major over mt x nt, or the upper triangle
// (it <= jt) enumerated column by column when sym
__host__ __device__ inline void dg_tile(int tile, int mt, int sym, int &it, int &jt) {
  if (sym) {
    jt = 0;
    while (tile > jt) {
      tile -= jt + 1;
      ++jt;
    }
    it = tile;
  } else {
    it = tile % mt;
    jt = tile / mt;
  }
}

// partial tiles: part[(split * ntile + tile) * 4096 + i + 64 j] =
// sum over the split's k tiles of A[k][64 it + i] B[k][64 jt + j]
__global__ void __launch_bounds__(DG_THREADS) k_dgemm_tn(const __grid_constant__ CUtensorMap ta,
                                                         const __grid_constant__ CUtensorMap tb, int m, int n, int mt,
                                                         int sym, int ktiles, int per, double *part, int *err,
                                                         long plim) {
  extern __shared__ unsigned char dg_raw[];
  unsigned char *sm = dg_align1k(dg_raw);
  uint64_t *full = reinterpret_cast<uint64_t *>(sm + DG_ST * DG_TN_STAGE);
  uint64_t *empty = full + DG_ST;
  __shared__ int aborted;
  volatile int *ab = &aborted;
  int it, jt;
  dg_tile(blockIdx.x, mt, sym, it, jt);
  const int k0 = blockIdx.y * per, nk = max(0, min(ktiles, k0 + per) - k0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    aborted = 0;
    for (int s = 0; s < DG_ST; ++s) {
      sg_bar_init(sg_smem(full + s), 1);
      sg_bar_init(sg_smem(empty + s), 4);
    }
    sg_bar_fence_init();
  }
  __syncthreads();
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  if (warp == 4) {
    if (lane == 0) {
      int issued = 0;
      for (int q = 0; q < nk; ++q) {
        const int s = q % DG_ST;
        if (q >= DG_ST && !*ab && !sg_bar_wait(sg_smem(empty + s), ((q / DG_ST) - 1) & 1, err, 31, plim)) *ab = 1;
        if (*ab) break;
        unsigned char *st = sm + s * DG_TN_STAGE;
        sg_bar_expect_tx(sg_smem(full + s), DG_TN_STAGE);
        sg_tma_2d(sg_smem(st), &ta, (k0 + q) * DG_KT, it * DG_T, sg_smem(full + s));
        sg_tma_2d(sg_smem(st + DG_TN_STAGE / 2), &tb, (k0 + q) * DG_KT, jt * DG_T, sg_smem(full + s));
        issued = q + 1;
      }
      // no copy of this block may land after it exits
      for (int q = max(0, issued - DG_ST); q < issued; ++q)
        sg_bar_wait(sg_smem(full + q % DG_ST), (q / DG_ST) & 1, err, 32);
    }
  } else {
    const int wr = warp & 1, wc = warp >> 1, g = lane >> 2, t = lane & 3;
    // a 32 x 32 quarter entirely outside m x n (few bands or projectors) has nothing to form
    const bool live = it * DG_T + wr * 32 < m && jt * DG_T + wc * 32 < n;
    for (int q = 0; q < nk; ++q) {
      const int s = q % DG_ST;
      if (!*ab && !sg_bar_wait(sg_smem(full + s), (q / DG_ST) & 1, err, 33, plim)) *ab = 1;
      if (!*ab && live) {
        const unsigned char *A = sm + s * DG_TN_STAGE, *B = A + DG_TN_STAGE / 2;
#pragma unroll
        for (int kb = 0; kb < 2; ++kb) {
          double2 a[4], b[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) a[i] = dg_ld_sw(A, wr * 32 + i * 8 + g, 2 * t + kb);
#pragma unroll
          for (int j = 0; j < 4; ++j) b[j] = dg_ld_sw(B, wc * 32 + j * 8 + g, 2 * t + kb);
          // the two steps one after the other: 16 independent MMAs between
          // the two that update one accumulator
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) dg_mma(acc[i][j], a[i].x, b[j].x);
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) dg_mma(acc[i][j], a[i].y, b[j].y);
        }
      }
      __syncwarp();
      if (lane == 0) sg_bar_arrive(sg_smem(empty + s));
    }
  }
  __syncthreads();
  if (warp < 4) {
    const bool bad = *ab != 0;
    const int wr = warp & 1, wc = warp >> 1, g = lane >> 2, t = lane & 3;
    double *p = part + ((long)blockIdx.y * gridDim.x + blockIdx.x) * (DG_T * DG_T);
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int r = wr * 32 + i * 8 + g, col = wc * 32 + j * 8 + 2 * t;
        p[r + DG_T * col] = bad ? __longlong_as_double(0x7ff8000000000000LL) : acc[i][j][0];
        p[r + DG_T * (col + 1)] = bad ? __longlong_as_double(0x7ff8000000000000LL) : acc[i][j][1];
      }
  }
}

// out[i + ldo j] = alpha sum_split part (i < m, j < n).  A block takes 32
// consecutive elements of the partial tiles; each of its 8 warps sums a
// contiguous range of the splits in order, and warp 0 adds the 8 results in
// order (deterministic).  With sym, an element of a tile above the diagonal
// is written at (i, j) and (j, i).
__global__ void __launch_bounds__(256) k_dgemm_tn_sum(const double *part, int nsplit, int ntile, int mt, int sym, int m,
                                                      int n, double alpha, double *out, int ldo) {
  __shared__ double red[8][32];
  const int lane = threadIdx.x & 31, grp = threadIdx.x >> 5;
  const long tot = (long)ntile * (DG_T * DG_T);
  const int qn = (nsplit + 7) / 8, q0 = grp * qn, q1 = min(nsplit, q0 + qn);
  for (long base = (long)blockIdx.x * 32; base < tot; base += (long)gridDim.x * 32) {
    const long e = base + lane;
    double s0 = 0.0, s1 = 0.0;
    int i = m, j = n, it = 0, jt = 0;
    if (e < tot) {
      const int tile = (int)(e / (DG_T * DG_T)), loc = (int)(e % (DG_T * DG_T));
      dg_tile(tile, mt, sym, it, jt);
      i = it * DG_T + loc % DG_T;
      j = jt * DG_T + loc / DG_T;
    }
    if (i < m && j < n) {
      const double *p = part + e;
      int q = q0;
      for (; q + 1 < q1; q += 2) {
        s0 += p[(long)q * tot];
        s1 += p[(long)(q + 1) * tot];
      }
      if (q < q1) s0 += p[(long)q * tot];
    }
    red[grp][lane] = s0 + s1;
    __syncthreads();
    if (grp == 0 && i < m && j < n) {
      double v = red[0][lane];
#pragma unroll
      for (int k = 1; k < 8; ++k) v += red[k][lane];
      out[i + (long)ldo * j] = alpha * v;
      if (sym && it != jt) out[j + (long)ldo * i] = alpha * v;
    }
    __syncthreads();
  }
}

// the MMAs of one band block for the column tiles C0 <= c < C1 of a warp; the
// two steps one after the other, so that up to 16 independent MMAs separate
// the two that update one accumulator
template <int C0, int C1>
__device__ __forceinline__ void dg_nn_cols(double (&acc)[2][2][4][2], const double2 (&a)[2][2], const double2 (&b)[4]) {
#pragma unroll
  for (int c = C0; c < C1; ++c)
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      dg_mma(acc[p][0][c], a[p][0].x, b[c].x);
      dg_mma(acc[p][1][c], a[p][0].y, b[c].x);
    }
#pragma unroll
  for (int c = C0; c < C1; ++c)
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      dg_mma(acc[p][0][c], a[p][1].x, b[c].y);
      dg_mma(acc[p][1][c], a[p][1].y, b[c].y);
    }
}

__device__ __forceinline__ void dg_cp8(uint32_t dst, const double *src, int bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void dg_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void dg_cp_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// out (K x n, leading dimension ldo) = alpha A G + beta out (beta 0: out is
// only written).  ta maps A (K x n1, boxes of 16 rows x 64 bands); G is
// n1 x n with leading dimension ldg; the boxes are 128-byte swizzled (the
// 16-byte chunk of rows 2g, 2g + 1 of band b sits at chunk g ^ (b & 7)).
// The work of a block is a sequence of units (work item, 64-band half chunk);
// the A half chunk of a unit comes by TMA (thread 0 issues each load as soon
// as every warp has released the stage it goes to), the matching 64 x 128
// slice of G by cp.async into one of two buffers, the next unit's slice
// copied while this unit multiplies.  When G has at most 128 rows and columns
// both of its halves stay in the two buffers for the whole kernel.
__global__ void __launch_bounds__(DG_NN_THREADS, 1) k_dgemm_nn(const __grid_constant__ CUtensorMap ta, const double *G,
                                                               int ldg, long K, int n1, int n, double alpha,
                                                               double beta, int upper, double *out, long ldo, int *err,
                                                               long plim) {
  extern __shared__ unsigned char dg_raw[];
  unsigned char *sm = dg_align1k(dg_raw);
  double *Gb = reinterpret_cast<double *>(sm + DG_NN_ST * DG_NN_STAGE);  // [2][128 columns][DG_NN_GLD]
  uint64_t *full = reinterpret_cast<uint64_t *>(sm + DG_NN_ST * DG_NN_STAGE + 2 * DG_NN_J * DG_NN_GLD * 8);
  uint64_t *empty = full + DG_NN_ST;
  __shared__ int aborted;
  volatile int *ab = &aborted;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nrt = (int)((K + DG_NN_R - 1) / DG_NN_R), njt = (n + DG_NN_J - 1) / DG_NN_J;
  const int nbc = (n1 + DG_NN_B - 1) / DG_NN_B;
  const long items = (long)nrt * njt;
  const bool resident = njt == 1 && nbc == 1;
  // G chunks of work item column tile jt (with upper only those at or above
  // its column block), and the 64-band halves of chunk bc
  auto chunks = [&](int jt) { return upper ? min(nbc, jt + 1) : nbc; };
  auto halves = [&](int bc) { return min(2, (n1 - bc * DG_NN_B + DG_NN_BS - 1) / DG_NN_BS); };
  // a cursor over the block's units
  struct Cur {
    long w;
    int bc, hf;
  };
  auto next = [&](Cur &u) {
    if (++u.hf >= halves(u.bc)) {
      u.hf = 0;
      if (++u.bc >= chunks((int)(u.w % njt))) {
        u.bc = 0;
        u.w += gridDim.x;
      }
    }
  };
  // G slice of unit u into buffer buf (zero outside n1 x n and, with upper,
  // below the diagonal); only whole 8-blocks that the products read
  auto stage_g = [&](const Cur &u, int buf) {
    const int jt = (int)(u.w % njt), b0 = u.bc * DG_NN_B + u.hf * DG_NN_BS;
    const int jv = min(DG_NN_J, (n - jt * DG_NN_J + 7) / 8 * 8), bv = min(DG_NN_BS, (n1 - b0 + 7) / 8 * 8);
    double *dst = Gb + (size_t)buf * DG_NN_J * DG_NN_GLD;
    for (int e = threadIdx.x; e < jv * bv; e += DG_NN_THREADS) {
      const int jl = e / bv, bl = e % bv;
      const int b = b0 + bl, j = jt * DG_NN_J + jl;
      const bool on = b < n1 && j < n && !(upper && b > j);
      dg_cp8(sg_smem(dst + jl * DG_NN_GLD + bl), on ? G + b + (long)ldg * j : G, on ? 8 : 0);
    }
    dg_cp_commit();
  };
  // copy cursor (thread 0): the unit of the next A load
  Cur cp{(long)blockIdx.x, 0, 0};
  int issued = 0;
  auto issue = [&]() {
    const int s = issued % DG_NN_ST;
    unsigned char *st = sm + s * DG_NN_STAGE;
    const int rt = (int)(cp.w / njt);
    sg_bar_expect_tx(sg_smem(full + s), DG_NN_STAGE);
#pragma unroll
    for (int b4 = 0; b4 < 4; ++b4)
      sg_tma_2d(sg_smem(st + b4 * DG_NN_BOX), &ta, rt * DG_NN_R + 16 * b4, cp.bc * DG_NN_B + cp.hf * DG_NN_BS,
                sg_smem(full + s));
    ++issued;
    next(cp);
  };
  if (threadIdx.x == 0) {
    aborted = 0;
    for (int s = 0; s < DG_NN_ST; ++s) {
      sg_bar_init(sg_smem(full + s), 1);
      sg_bar_init(sg_smem(empty + s), DG_NN_THREADS / 32);
    }
    sg_bar_fence_init();
    for (int k = 0; k < DG_NN_ST && cp.w < items; ++k) issue();
  }
  // G for the first unit (resident: both halves, for good)
  Cur gu{(long)blockIdx.x, 0, 0};
  if (gu.w < items) {
    if (resident) {
      for (int h = 0; h < halves(0); ++h) stage_g(Cur{gu.w, 0, h}, h);
    } else {
      stage_g(gu, 0);
    }
  }
  const int wr = warp >> 2, wc = warp & 3, g = lane >> 2, t = lane & 3;
  int q = 0;
  Cur gn = gu;  // the unit whose G slice is copied next (streaming)
  if (!resident) next(gn);
  for (long w = blockIdx.x; w < items; w += gridDim.x) {
    const int rt = (int)(w / njt), jt = (int)(w % njt);
    // column tiles of this warp with a column below n
    const int clive = min(4, max(0, (n - jt * DG_NN_J - 8 * wc + 31) / 32));
    double acc[2][2][4][2];
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[p][h][c][0] = acc[p][h][c][1] = 0.0;
    // beta != 0: the output's old values, loaded now so that the item's
    // products hide their latency
    double2 old[2][4][2];
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
      for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const long r = (long)rt * DG_NN_R + 32 * wr + 16 * p + 2 * g;
          const int j = jt * DG_NN_J + 8 * (wc + 4 * c) + 2 * t + e;
          old[p][c][e] = (beta != 0.0 && r < K && j < n) ? *reinterpret_cast<const double2 *>(out + r + ldo * j)
                                                         : make_double2(0.0, 0.0);
        }
    for (int bc = 0; bc < chunks(jt); ++bc) {
      for (int hf = 0; hf < halves(bc); ++hf, ++q) {
        // this unit's G slice has landed (every thread's copies), and every
        // warp is done with the previous unit, whose buffer the next copy reuses
        dg_cp_wait_all();
        __syncthreads();
        if (!resident && gn.w < items) {
          stage_g(gn, (q + 1) & 1);
          next(gn);
        }
        const double *Gs = Gb + (size_t)(resident ? hf : (q & 1)) * DG_NN_J * DG_NN_GLD;
        const int s = q % DG_NN_ST;
        if (!*ab && !sg_bar_wait(sg_smem(full + s), (q / DG_NN_ST) & 1, err, 36, plim)) *ab = 1;
        if (!*ab) {
          const unsigned char *A = sm + s * DG_NN_STAGE + 2 * wr * DG_NN_BOX;
          const int nkb = min(DG_NN_BS / 8, (n1 - bc * DG_NN_B - hf * DG_NN_BS + 7) / 8);
#pragma unroll 2
          for (int kb = 0; kb < nkb; ++kb) {
            // band block of 8 (global index) against the column blocks of this warp
            const int gkb = bc * (DG_NN_B / 8) + hf * (DG_NN_BS / 8) + kb;
            double2 a[2][2], b[4];
#pragma unroll
            for (int p = 0; p < 2; ++p)
#pragma unroll
              for (int s2 = 0; s2 < 2; ++s2) {
                const int band = 8 * kb + 2 * t + s2;
                a[p][s2] = *reinterpret_cast<const double2 *>(A + p * DG_NN_BOX + band * 128 + ((g ^ (band & 7)) << 4));
              }
#pragma unroll
            for (int c = 0; c < 4; ++c)
              b[c] = *reinterpret_cast<const double2 *>(Gs + (8 * (wc + 4 * c) + g) * DG_NN_GLD + 8 * kb + 2 * t);
            // with upper, column tile c takes this band block when its column
            // block jt*16 + wc + 4c is not below it: the tiles c >= cmin;
            // and the tiles c >= clive hold no column below n
            int cmin = 0;
            if (upper) cmin = min(4, max(0, (gkb - jt * (DG_NN_J / 8) - wc + 3) / 4));
            switch (cmin * 5 + clive) {
              case 1: dg_nn_cols<0, 1>(acc, a, b); break;
              case 2: dg_nn_cols<0, 2>(acc, a, b); break;
              case 3: dg_nn_cols<0, 3>(acc, a, b); break;
              case 4: dg_nn_cols<0, 4>(acc, a, b); break;
              case 7: dg_nn_cols<1, 2>(acc, a, b); break;
              case 8: dg_nn_cols<1, 3>(acc, a, b); break;
              case 9: dg_nn_cols<1, 4>(acc, a, b); break;
              case 13: dg_nn_cols<2, 3>(acc, a, b); break;
              case 14: dg_nn_cols<2, 4>(acc, a, b); break;
              case 19: dg_nn_cols<3, 4>(acc, a, b); break;
              default: break;  // no tile of this warp takes the block
            }
          }
        }
        __syncwarp();
        if (lane == 0) sg_bar_arrive(sg_smem(empty + s));
        if (threadIdx.x == 0 && cp.w < items && !*ab) {
          // the next load goes to this stage once every warp has released
          // it and this load has landed (no stage ever holds two copies)
          if (!sg_bar_wait(sg_smem(empty + s), (q / DG_NN_ST) & 1, err, 34, plim) ||
              !sg_bar_wait(sg_smem(full + s), (q / DG_NN_ST) & 1, err, 37))
            *ab = 1;
          else
            issue();
        }
      }
    }
    // epilogue: rows r, r + 1 of column j as one 16-byte access
    const bool bad = *ab != 0;
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      const long r = (long)rt * DG_NN_R + 32 * wr + 16 * p + 2 * g;
      if (r >= K) continue;
#pragma unroll
      for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int j = jt * DG_NN_J + 8 * (wc + 4 * c) + 2 * t + e;
          if (j >= n) continue;
          double2 v = make_double2(alpha * acc[p][0][c][e], alpha * acc[p][1][c][e]);
          if (beta != 0.0) {
            v.x += beta * old[p][c][e].x;
            v.y += beta * old[p][c][e].y;
          }
          if (bad) v.x = v.y = __longlong_as_double(0x7ff8000000000000LL);
          *reinterpret_cast<double2 *>(out + r + ldo * j) = v;
        }
    }
  }
  dg_cp_wait_all();
  // no copy of this block may land after it exits
  if (threadIdx.x == 0)
    for (int p = max(0, issued - DG_NN_ST); p < issued; ++p)
      sg_bar_wait(sg_smem(full + p % DG_NN_ST), (p / DG_NN_ST) & 1, err, 35);
  __syncthreads();
}

}  // namespace amdk
