// "Pencil" path for the band-pair transforms of vpsi and eval_density
// (wfn_initialize.f90:283-362, density.f90:19-90) on cubic grids.
//
// The x pass writes the ray buffer transposed, RT[t][kx][ray], so that one
// block can take one x-plane of one band pair: it scatters the plane's rays
// into a shared-memory slab plane P[zi][ky] (only the z planes that carry
// rays), runs the y transforms of those rows, then per tile of columns the
// z transform, V(r)*psi and the inverse z transform (or the |psi|^2
// accumulation), the inverse y transforms, and gathers the rays back.  Every
// line transform is the two-level register FFT of fft.cuh; the backward y
// transform leaves its output in the permuted order the forward one takes,
// so no pass reorders data.  No slab or grid buffer goes through HBM: the
// only HBM traffic is the ray buffer (read and written once per pass), V
// (L2 resident) and the coefficients.
#pragma once
#include "fft.cuh"

namespace amdk {

constexpr int PG_MAXSEG = 16;  // source ranks of a slab-decomposed plane buffer
struct PencilGeom {
  int n1, n2, n3, nray, nz;  // n1: x planes of the buffers the plane kernels read
  const int *rpos;   // [nray] zi*(n2+1) + ky of the ray in the padded plane
  const int *zinv;   // [n3] slab index of kz, -1 outside the slab
  const int *zlist;  // [nz] kz of slab plane
  const int *gmapt;  // [n1][nray] G code of (ray, kx): +(ig+1) at +G, -(ig+1) at -G, 0 empty
  // x passes: element kx of the line (pair t, ray r) at t*xt_t + kx*xt_x + r
  long xt_t, xt_x;
  // plane kernels: the rays of plane kx of pair t form row pr = t*pr_t +
  // kx*pr_x of nseg segments; segment s holds rays seg_r0[s] .. seg_r0[s+1]-1
  // (in rpos order), its row pr at seg_mul*seg_r0[s] + pr*(its ray count).
  // One GPU: one segment, row pr = t*n1 + kx of nray rays.  Slab
  // decomposition: one segment per source rank, as the all-to-all leaves them.
  int pr_t, pr_x, nseg;
  long seg_mul;
  int seg_r0[PG_MAXSEG + 1];
};
// the one-GPU layout RT[t][kx][ray]
inline PencilGeom pencil_geom_1gpu(int n1, int n2, int n3, int nray, int nz, const int *rpos, const int *zinv,
                                   const int *zlist, const int *gmapt) {
  PencilGeom g{};
  g.n1 = n1;
  g.n2 = n2;
  g.n3 = n3;
  g.nray = nray;
  g.nz = nz;
  g.rpos = rpos;
  g.zinv = zinv;
  g.zlist = zlist;
  g.gmapt = gmapt;
  g.xt_t = (long)n1 * nray;
  g.xt_x = nray;
  g.pr_t = n1;
  g.pr_x = 1;
  g.nseg = 1;
  g.seg_mul = 0;
  g.seg_r0[0] = 0;
  g.seg_r0[1] = nray;
  return g;
}
// position of ray r of row pr in the plane kernels' buffer
// (the segment tables are read with compile-time indices only, so they stay
// in the kernel's parameter space)
__device__ __forceinline__ long ray_at(const PencilGeom &pg, long pr, int r) {
  int r0 = 0, r1 = pg.seg_r0[1];
#pragma unroll
  for (int s = 1; s < PG_MAXSEG; ++s)
    if (s < pg.nseg && r >= pg.seg_r0[s]) {
      r0 = pg.seg_r0[s];
      r1 = pg.seg_r0[s + 1];
    }
  return pg.seg_mul * r0 + pr * (r1 - r0) + (r - r0);
}

constexpr int PNT = 512;  // threads per pencil block
// Shared-memory rows (slab plane P, column tile S, density accumulator) have
// stride N+1 so that threads taking consecutive rows hit distinct banks.

constexpr int XL = 32;  // lines per x-pass block
// Backward x pass with the band-pair pack (psi_a + i psi_b, the pack of
// vpsi and eval_density), output transposed: RT[t][kx][r] on one GPU, the
// slab decomposition's send layout [kx][t][r] (strides xt_t, xt_x).  Block = XL lines
// (consecutive rays) x N2 threads; thread (l, j2) gathers the N1 elements
// kx = j2 + N2*j1 of its ray straight from the coefficients, the second
// phase writes kx = k1 + N1*k2 back with consecutive threads on consecutive
// rays.
template <typename C, int N>
__global__ void __launch_bounds__(512) k_xt_bwd_pair(const double2 *__restrict__ c0, int ngpw, int nstate, int band0,
                                                     int T, PencilGeom pg, Plan<C> p, C *__restrict__ rt) {
  typedef decltype(C().x) Rl;
  constexpr int N1 = fft_n1(N), N2 = N / N1, NP = N + 1;
  extern __shared__ unsigned char smraw[];
  C *S = reinterpret_cast<C *>(smraw);
  C *tw = S + XL * NP;
  load_tw<C, N>(tw, p);
  __syncthreads();
  const int R = pg.nray;
  const long line0 = (long)blockIdx.x * XL;
  const long nlines = (long)T * R;
  {
    const int l = threadIdx.x % XL, j2 = threadIdx.x / XL;
    const long line = line0 + l;
    C v[N1];
#pragma unroll
    for (int j1 = 0; j1 < N1; ++j1) v[j1] = czero<C>();
    if (line < nlines) {
      const int t = (int)(line / R), r = (int)(line % R);
      const int ba = band0 + 2 * t, bb = ba + 1;
      const double2 *ca = c0 + (long)ba * ngpw;
      const double2 *cb = c0 + (long)bb * ngpw;
      const bool hb = bb < nstate;
#pragma unroll
      for (int j1 = 0; j1 < N1; ++j1) {
        const int code = pg.gmapt[(long)(j2 + N2 * j1) * R + r];
        const int ig = (code > 0 ? code : -code) - 1;
        if (code != 0 && ig < ngpw) {
          const double2 a = ca[ig];
          const double2 b = hb ? cb[ig] : make_double2(0.0, 0.0);
          if (code > 0) v[j1] = mk((Rl)(a.x - b.y), (Rl)(a.y + b.x));
          else v[j1] = mk((Rl)(a.x + b.y), (Rl)(-a.y + b.x));
        }
      }
    }
    Dft<C, N1, 1>::run(v);
    twiddle_tab<C, N, N1, 1, 0>(v, j2, tw);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) S[l * NP + k1 * N2 + j2] = v[k1];
  }
  __syncthreads();
  if (threadIdx.x < XL * N1) {
    const int l = threadIdx.x % XL, k1 = threadIdx.x / XL;
    const long line = line0 + l;
    C u[N2];
#pragma unroll
    for (int j2 = 0; j2 < N2; ++j2) u[j2] = S[l * NP + k1 * N2 + j2];
    Dft<C, N2, 1>::run(u);
    if (line < nlines) {
      const int t = (int)(line / R), r = (int)(line % R);
      C *o = rt + t * pg.xt_t + r;
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) o[(long)(k1 + N1 * k2) * pg.xt_x] = u[k2];
    }
  }
}

// Forward x pass in place on the transposed ray buffer (same blocking)
template <typename C, int N>
__global__ void __launch_bounds__(512) k_xt_fwd(int T, PencilGeom pg, Plan<C> p, C *__restrict__ rt) {
  constexpr int N1 = fft_n1(N), N2 = N / N1, NP = N + 1;
  extern __shared__ unsigned char smraw[];
  C *S = reinterpret_cast<C *>(smraw);
  C *tw = S + XL * NP;
  load_tw<C, N>(tw, p);
  __syncthreads();
  const int R = pg.nray;
  const long line0 = (long)blockIdx.x * XL;
  const long nlines = (long)T * R;
  {
    const int l = threadIdx.x % XL, j2 = threadIdx.x / XL;
    const long line = line0 + l;
    C v[N1];
    if (line < nlines) {
      const int t = (int)(line / R), r = (int)(line % R);
      const C *in = rt + t * pg.xt_t + r;
#pragma unroll
      for (int j1 = 0; j1 < N1; ++j1) v[j1] = in[(long)(j2 + N2 * j1) * pg.xt_x];
    } else {
#pragma unroll
      for (int j1 = 0; j1 < N1; ++j1) v[j1] = czero<C>();
    }
    Dft<C, N1, -1>::run(v);
    twiddle_tab<C, N, N1, -1, 0>(v, j2, tw);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) S[l * NP + k1 * N2 + j2] = v[k1];
  }
  __syncthreads();
  if (threadIdx.x < XL * N1) {
    const int l = threadIdx.x % XL, k1 = threadIdx.x / XL;
    const long line = line0 + l;
    C u[N2];
#pragma unroll
    for (int j2 = 0; j2 < N2; ++j2) u[j2] = S[l * NP + k1 * N2 + j2];
    Dft<C, N2, -1>::run(u);
    if (line < nlines) {
      const int t = (int)(line / R), r = (int)(line % R);
      C *o = rt + t * pg.xt_t + r;
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) o[(long)(k1 + N1 * k2) * pg.xt_x] = u[k2];
    }
  }
}

// x = q d + r for task indices: q = (x m) >> 20 with m = 2^20/d + 1 is exact
// while x d < 2^20 (here x < 16 d and d <= 256), three integer instructions
// instead of a division by a run-time value
struct DivMod {
  unsigned d, m;
  __device__ __forceinline__ explicit DivMod(int dd) : d((unsigned)dd), m((1u << 20) / (unsigned)dd + 1u) {}
  __device__ __forceinline__ void operator()(int x, int &q, int &r) const {
    const unsigned qq = ((unsigned)x * m) >> 20;
    q = (int)qq;
    r = x - (int)(qq * d);
  }
};

// Length-N transforms of the nz rows of the slab plane P (row stride N+1), in
// place.  nat_to_perm: natural order in, X[k1 + N1*k2] left at position
// k1*N2 + k2.  perm_to_nat: that permuted order in, natural order out.  Each
// phase's sub-transform reads and writes the same positions, so a phase needs
// no barrier inside; the two phases are separated by one.
template <typename C, int N, int SG>
__device__ __forceinline__ void rows_nat_to_perm(C *P, int nrow, const DivMod &dr, const C *tw) {
  constexpr int N1 = fft_n1(N), N2 = N / N1, NP = N + 1;
  for (int idx = threadIdx.x; idx < nrow * N2; idx += blockDim.x) {
    int j2, r;
    dr(idx, j2, r);
    C *row = P + r * NP;
    C v[N1];
#pragma unroll
    for (int j1 = 0; j1 < N1; ++j1) v[j1] = row[j2 + N2 * j1];
    Dft<C, N1, SG>::run(v);
    twiddle_tab<C, N, N1, SG, 0, true>(v, j2, tw);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) row[k1 * N2 + j2] = v[k1];
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < nrow * N1; idx += blockDim.x) {
    int k1, r;
    dr(idx, k1, r);
    C *row = P + r * NP + k1 * N2;
    C u[N2];
#pragma unroll
    for (int j2 = 0; j2 < N2; ++j2) u[j2] = row[j2];
    Dft<C, N2, SG>::run(u);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) row[k2] = u[k2];
  }
  __syncthreads();
}
template <typename C, int N, int SG>
__device__ __forceinline__ void rows_perm_to_nat(C *P, int nrow, const DivMod &dr, const C *tw) {
  constexpr int N1 = fft_n1(N), N2 = N / N1, NP = N + 1;
  for (int idx = threadIdx.x; idx < nrow * N1; idx += blockDim.x) {
    int k1, r;
    dr(idx, k1, r);
    C *row = P + r * NP + k1 * N2;
    C u[N2];
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) u[k2] = row[k2];
    Dft<C, N2, SG>::run(u);
    twiddle_tab<C, N, N2, SG, 1, true>(u, k1, tw);
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) row[n2] = u[n2];
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < nrow * N2; idx += blockDim.x) {
    int n2, r;
    dr(idx, n2, r);
    C *row = P + r * NP;
    C w[N1];
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) w[k1] = row[k1 * N2 + n2];
    Dft<C, N1, SG>::run(w);
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) row[n2 + N2 * n1] = w[n1];
  }
  __syncthreads();
}

// scatter the rays of row pr (one x-plane of one pair) into P (zero elsewhere)
template <typename C, int N>
__device__ __forceinline__ void pencil_scatter(C *P, const C *__restrict__ rt, long pr, const PencilGeom &pg) {
  for (int idx = threadIdx.x; idx < pg.nz * (N + 1); idx += blockDim.x) P[idx] = czero<C>();
  __syncthreads();
#pragma unroll
  for (int s = 0; s < PG_MAXSEG; ++s) {
    if (s >= pg.nseg) break;
    const int r0 = pg.seg_r0[s], nr = pg.seg_r0[s + 1] - r0;
    const C *src = rt + pg.seg_mul * r0 + pr * nr;
    for (int j = threadIdx.x; j < nr; j += blockDim.x) P[pg.rpos[r0 + j]] = src[j];
  }
  __syncthreads();
}

// slab plane of kz = j2 + N2*j1 from the packed table zp (one 16-byte entry
// per j2, byte j1; 0xFF where the slab has no plane)
__device__ __forceinline__ int zp_plane(const uint4 &e, int j1) {
  const unsigned w = (j1 < 4) ? e.x : (j1 < 8) ? e.y : (j1 < 12) ? e.z : e.w;
  const int b = (int)((w >> (8 * (j1 & 3))) & 0xFFu);
  return b == 0xFF ? -1 : b;
}
// Backward z transform of the column tile q0 .. q0+ct-1 of P, first phase:
// thread (column, j2) takes the slab planes at kz = j2 + N2*j1 (zero where
// the slab has no plane) and leaves W_N^(j2 k1) DFT_N1 in S[col][k1*N2 + j2].
template <typename C, int N>
__device__ __forceinline__ void zcols_phase_a(const C *P, C *S, const uint4 *zp, int q0, int ct, const DivMod &dq,
                                              const C *tw) {
  constexpr int N1 = fft_n1(N), N2 = N / N1, NP = N + 1;
  for (int idx = threadIdx.x; idx < ct * N2; idx += blockDim.x) {
    int j2, qq;
    dq(idx, j2, qq);
    const uint4 e = zp[j2];
    C v[N1];
#pragma unroll
    for (int j1 = 0; j1 < N1; ++j1) {
      const int zi = zp_plane(e, j1);
      v[j1] = (zi >= 0) ? P[zi * NP + q0 + qq] : czero<C>();
    }
    Dft<C, N1, 1>::run(v);
    twiddle_tab<C, N, N1, 1, 0, true>(v, j2, tw);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) S[qq * NP + k1 * N2 + j2] = v[k1];
  }
}

// shared memory of a pencil block: P[nz][N+1], S[CTs][N+1], the twiddle
// tables (2N, from a 16-byte boundary) and the packed slab-plane table zp
// (one 16-byte entry per j2 < N2: the slab plane of kz = j2 + N2*j1 in byte
// j1, 0xFF for none; the slab has fewer than 255 planes)
template <typename C, int N> struct PencilSmem {
  C *P, *S, *tw;
  uint4 *zp;
  __device__ __forceinline__ PencilSmem(unsigned char *raw, int nz, int CTs) {
    constexpr int NP = N + 1;
    P = reinterpret_cast<C *>(raw);
    S = P + nz * NP;
    const size_t off = ((size_t)(nz + CTs) * NP * sizeof(C) + 15) & ~(size_t)15;
    tw = reinterpret_cast<C *>(raw + off);
    zp = reinterpret_cast<uint4 *>(tw + 2 * N);
  }
  // twiddles, and zp from the kz -> slab plane table zinv (global)
  __device__ __forceinline__ void load(const Plan<C> &p, const int *zinv) {
    constexpr int N1 = fft_n1(N), N2 = N / N1;
    load_tw<C, N>(tw, p);
    for (int j2 = threadIdx.x; j2 < N2; j2 += blockDim.x) {
      unsigned w[4] = {~0u, ~0u, ~0u, ~0u};
      for (int j1 = 0; j1 < N1; ++j1) {
        const int zi = zinv[j2 + N2 * j1];
        const unsigned b = zi >= 0 ? (unsigned)zi : 0xFFu;
        w[j1 >> 2] = (w[j1 >> 2] & ~(0xFFu << (8 * (j1 & 3)))) | (b << (8 * (j1 & 3)));
      }
      zp[j2] = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
};

// One x-plane of one band pair through y, z, V(r), z, y (vpsi,
// wfn_initialize.f90:311-340).  grid (n1, T).  P[zi][q] holds the slab
// plane (row stride N+1); after the backward y transform column q carries
// ky = q/N2 + N1*(q%N2).  vp[kx][q][k'] is V at that ky and at
// kz = k'/N2 + N1*(k'%N2), the order in which the z transform leaves psi.
// The column tiles are CTs wide (the last may be narrower); the V values of a
// thread's first task of a tile are loaded before the tile's first phase.
// LSD (open shell): pair gp0 + blockIdx.y takes the spin-2 potential vp2 from
// pair psplit on, and the pair pstraddle (whose first band is the last of
// spin 1) multiplies its real part by V_1 and its imaginary part by V_2
// (wfn_initialize.f90:313-326).
template <typename C, int N, bool LSD = false>
__global__ void __launch_bounds__(PNT) k_pencil_vpsi(PencilGeom pg, Plan<C> p, C *__restrict__ rt,
                                                     const decltype(C().x) *__restrict__ vp, int CTs,
                                                     const decltype(C().x) *__restrict__ vp2, int gp0, int psplit,
                                                     int pstraddle) {
  typedef decltype(C().x) Rl;
  constexpr int N1 = fft_n1(N), N2 = N / N1, NP = N + 1;
  extern __shared__ unsigned char smraw[];
  const int nz = pg.nz;
  PencilSmem<C, N> sm(smraw, nz, CTs);
  C *P = sm.P, *S = sm.S, *tw = sm.tw;
  const uint4 *zp = sm.zp;
  sm.load(p, pg.zinv);
  const int kx = blockIdx.x, t = blockIdx.y;
  const long pr = (long)t * pg.pr_t + (long)kx * pg.pr_x;
  pencil_scatter<C, N>(P, rt, pr, pg);
  const DivMod dz(nz);
  rows_nat_to_perm<C, N, 1>(P, nz, dz, tw);
  const Rl *V = vp + (long)kx * N * N;
  const Rl *V2 = nullptr;
  bool straddle = false;
  if constexpr (LSD) {
    const int gp = gp0 + t;
    if (gp == pstraddle) {
      straddle = true;
      V2 = vp2 + (long)kx * N * N;
    } else if (gp >= psplit) {
      V = vp2 + (long)kx * N * N;
    }
  }
  for (int q0 = 0; q0 < N; q0 += CTs) {
    const int ct = min(CTs, N - q0);
    const DivMod dq(ct);
    // V of this thread's first middle task, in flight during phase A
    int k1_0 = 0, qq_0 = 0;
    dq(threadIdx.x, k1_0, qq_0);
    const bool has0 = threadIdx.x < ct * N1;
    Rl v0[N2];
    {
      const Rl *vv = V + (long)(q0 + qq_0) * N + k1_0 * N2;
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) v0[k2] = has0 ? vv[k2] : (Rl)0;
    }
    zcols_phase_a<C, N>(P, S, zp, q0, ct, dq, tw);
    __syncthreads();
    // DFT_N2 -> psi(kz = k1 + N1*k2), times V, then the first phase of the
    // forward z transform, in registers
    for (int idx = threadIdx.x; idx < ct * N1; idx += blockDim.x) {
      int k1, qq;
      dq(idx, k1, qq);
      C *row = S + qq * NP + k1 * N2;
      Rl vv[N2];
      if (idx == threadIdx.x) {
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) vv[k2] = v0[k2];
      } else {
        const Rl *vg = V + (long)(q0 + qq) * N + k1 * N2;
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) vv[k2] = vg[k2];
      }
      C u[N2];
#pragma unroll
      for (int j2 = 0; j2 < N2; ++j2) u[j2] = row[j2];
      Dft<C, N2, 1>::run(u);
      if (LSD && straddle) {
        const Rl *vg2 = V2 + (long)(q0 + qq) * N + k1 * N2;
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) {
          u[k2].x = u[k2].x * vv[k2];
          u[k2].y = u[k2].y * vg2[k2];
        }
      } else {
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) u[k2] = cscale(u[k2], vv[k2]);
      }
      Dft<C, N2, -1>::run(u);
      twiddle_tab<C, N, N2, -1, 1, true>(u, k1, tw);
#pragma unroll
      for (int n2 = 0; n2 < N2; ++n2) row[n2] = u[n2];
    }
    __syncthreads();
    // second phase: x(kz = n2 + N2*n1), stored back for the slab planes only
    for (int idx = threadIdx.x; idx < ct * N2; idx += blockDim.x) {
      int n2, qq;
      dq(idx, n2, qq);
      const uint4 e = zp[n2];
      C w[N1];
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) w[k1] = S[qq * NP + k1 * N2 + n2];
      Dft<C, N1, -1>::run(w);
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) {
        const int zi = zp_plane(e, n1);
        if (zi >= 0) P[zi * NP + q0 + qq] = w[n1];
      }
    }
    __syncthreads();
  }
  rows_perm_to_nat<C, N, -1>(P, nz, dz, tw);
#pragma unroll
  for (int sg = 0; sg < PG_MAXSEG; ++sg) {
    if (sg >= pg.nseg) break;
    const int r0 = pg.seg_r0[sg], nr = pg.seg_r0[sg + 1] - r0;
    C *dst = rt + pg.seg_mul * r0 + pr * nr;
    for (int j = threadIdx.x; j < nr; j += blockDim.x) dst[j] = P[pg.rpos[r0 + j]];
  }
}

// Density: one x-plane for a group of band pairs (density.f90:49-86);
// rho_part[grp][kx][q][k'] += wa_t Re^2 + wb_t Im^2 in the permuted (ky, kz)
// order of the vpsi kernel.  grid (n1, ngroups).  A thread takes the same
// (column, k1) tasks for every pair, so its group sums stay in registers
// (NS slots of N2 values: column tiles x task rounds, NS = ntiles * reps with
// reps = ceil(CTs N1 / PNT)), in the data's precision (FP32 for float2: the
// mixed path ends on FP64).  At the end the sums go through shared memory
// (over P and S) and are stored to (add = 0: the first batch of pairs) or
// added to (add = 1) the FP64 partial grid.
template <typename C, int N, int NS>
__global__ void __launch_bounds__(PNT, sizeof(C) == 8 ? 2 : 1) k_pencil_density(PencilGeom pg, Plan<C> p, const C *__restrict__ rt, int T,
                                                        int per_group, const double *__restrict__ wa,
                                                        const double *__restrict__ wb, double *__restrict__ rho_part,
                                                        int CTs, int add) {
  typedef decltype(C().x) Rl;
  constexpr int N1 = fft_n1(N), N2 = N / N1, NP = N + 1;
  extern __shared__ unsigned char smraw[];
  const int nz = pg.nz;
  PencilSmem<C, N> sm(smraw, nz, CTs);
  C *P = sm.P, *S = sm.S, *tw = sm.tw;
  const uint4 *zp = sm.zp;
  sm.load(p, pg.zinv);
  const int kx = blockIdx.x, grp = blockIdx.y;
  const int t0 = grp * per_group, t1 = min(T, t0 + per_group);
  const int ntiles = (N + CTs - 1) / CTs;
  const int reps = NS / ntiles;  // the launch guarantees ntiles * reps == NS and CTs N1 <= reps PNT
  Rl acc[NS][N2];
#pragma unroll
  for (int s = 0; s < NS; ++s)
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) acc[s][k2] = (Rl)0;
  // the next pair's rays are loaded into registers while this pair is
  // transformed (planes of up to PREF * blockDim rays; else loaded in turn)
  constexpr int PREF = 4;
  const bool pre = pg.nray <= PREF * (int)blockDim.x;
  C nxt[PREF];
  auto fetch = [&](int t) {
    const long pr = (long)t * pg.pr_t + (long)kx * pg.pr_x;
    if (pg.nseg == 1) {
      const C *pl = rt + pr * pg.nray;
#pragma unroll
      for (int i = 0; i < PREF; ++i) {
        const int r = threadIdx.x + i * blockDim.x;
        nxt[i] = r < pg.nray ? pl[r] : czero<C>();
      }
    } else {
#pragma unroll
      for (int i = 0; i < PREF; ++i) {
        const int r = threadIdx.x + i * blockDim.x;
        nxt[i] = r < pg.nray ? rt[ray_at(pg, pr, r)] : czero<C>();
      }
    }
  };
  const DivMod dz(nz);
  if (pre && t0 < t1) fetch(t0);
  for (int t = t0; t < t1; ++t) {
    if (pre) {
      for (int idx = threadIdx.x; idx < nz * NP; idx += blockDim.x) P[idx] = czero<C>();
      __syncthreads();
#pragma unroll
      for (int i = 0; i < PREF; ++i) {
        const int r = threadIdx.x + i * blockDim.x;
        if (r < pg.nray) P[pg.rpos[r]] = nxt[i];
      }
      __syncthreads();
      if (t + 1 < t1) fetch(t + 1);
    } else {
      pencil_scatter<C, N>(P, rt, (long)t * pg.pr_t + (long)kx * pg.pr_x, pg);
    }
    rows_nat_to_perm<C, N, 1>(P, nz, dz, tw);
    const Rl fa = (Rl)wa[t], fb = (Rl)wb[t];
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const int ti = s / reps, rr = s - ti * reps;
      const int q0 = ti * CTs, ct = min(CTs, N - q0);
      const DivMod dq(ct);
      if (rr == 0) {
        zcols_phase_a<C, N>(P, S, zp, q0, ct, dq, tw);
        __syncthreads();
      }
      const int idx = threadIdx.x + rr * PNT;
      if (idx < ct * N1) {
        int k1, qq;
        dq(idx, k1, qq);
        const C *row = S + qq * NP + k1 * N2;
        C u[N2];
#pragma unroll
        for (int j2 = 0; j2 < N2; ++j2) u[j2] = row[j2];
        Dft<C, N2, 1>::run(u);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) {
          const Rl re = u[k2].x, im = u[k2].y;
          acc[s][k2] += fa * re * re + fb * im * im;
        }
      }
      if (rr == reps - 1) __syncthreads();
    }
  }
  __syncthreads();  // a group without pairs has seen no barrier since the tables
  // group sums -> shared memory [q][k'] (row stride N+1) -> the partial grid
  Rl *stage = reinterpret_cast<Rl *>(smraw);
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const int ti = s / reps, rr = s - ti * reps;
    const int q0 = ti * CTs, ct = min(CTs, N - q0);
    const int idx = threadIdx.x + rr * PNT;
    if (idx < ct * N1) {
      int k1, qq;
      const DivMod dq(ct);
      dq(idx, k1, qq);
      Rl *ar = stage + (q0 + qq) * NP + k1 * N2;
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) ar[k2] = acc[s][k2];
    }
  }
  __syncthreads();
  double *out = rho_part + ((long)grp * pg.n1 + kx) * N * N;
  for (int idx = threadIdx.x; idx < N * N; idx += blockDim.x) {
    const int q = idx / N, k = idx % N;
    const double v = (double)stage[q * NP + k];
    out[idx] = add ? out[idx] + v : v;
  }
}

// Balanced schedule of the density sums over one batch of T pairs: the
// n1 T (x-plane, pair) units, plane-major (unit u = plane u / T, pair u % T),
// in nblk contiguous ranges, block b taking [b U / nblk, (b+1) U / nblk),
// U = n1 T; one wave of blocks then has equal work to within one pair, where
// (plane, pair-group) blocks leave a partial last wave.  A plane is shared by
// the consecutive blocks bal_block(plane T) .. bal_block(plane T + T - 1); the
// k-th of them stores its sums of that plane in partial grid k.
__host__ __device__ __forceinline__ int bal_block(long u, long U, int nblk) {
  return (int)(((u + 1) * nblk - 1) / U);  // the largest b with floor(b U / nblk) <= u
}
__host__ __device__ __forceinline__ int bal_slots(int kx, int T, long U, int nblk) {
  return bal_block((long)kx * T + T - 1, U, nblk) - bal_block((long)kx * T, U, nblk) + 1;
}
template <typename C, int N, int NS>
__global__ void __launch_bounds__(PNT, sizeof(C) == 8 ? 2 : 1)
    k_pencil_density_bal(PencilGeom pg, Plan<C> p, const C *__restrict__ rt, int T, const double *__restrict__ wa,
                         const double *__restrict__ wb, double *__restrict__ rho_part, int CTs) {
  typedef decltype(C().x) Rl;
  constexpr int N1 = fft_n1(N), N2 = N / N1, NP = N + 1;
  extern __shared__ unsigned char smraw[];
  const int nz = pg.nz;
  PencilSmem<C, N> sm(smraw, nz, CTs);
  C *P = sm.P, *S = sm.S, *tw = sm.tw;
  const uint4 *zp = sm.zp;
  sm.load(p, pg.zinv);
  const long U = (long)pg.n1 * T;
  const int nb = gridDim.x, b = blockIdx.x;
  const long u0 = (long)b * U / nb, u1 = (long)(b + 1) * U / nb;
  const int ntiles = (N + CTs - 1) / CTs;
  const int reps = NS / ntiles;  // the launch guarantees ntiles * reps == NS and CTs N1 <= reps PNT
  Rl acc[NS][N2];
  constexpr int PREF = 4;
  const bool pre = pg.nray <= PREF * (int)blockDim.x;
  C nxt[PREF];
  auto row_of = [&](long u) {
    const long kx = u / T;
    return (u - kx * T) * pg.pr_t + kx * pg.pr_x;
  };
  auto fetch = [&](long u) {
    const C *pl = rt + row_of(u) * pg.nray;  // one ray segment (the one-GPU layout)
#pragma unroll
    for (int i = 0; i < PREF; ++i) {
      const int r = threadIdx.x + i * blockDim.x;
      nxt[i] = r < pg.nray ? pl[r] : czero<C>();
    }
  };
  const DivMod dz(nz);
  if (pre && u0 < u1) fetch(u0);
  __syncthreads();  // the tables
  for (long u = u0; u < u1;) {
    const int kx = (int)(u / T);
    const long ue = min(u1, (long)(kx + 1) * T);
#pragma unroll
    for (int s = 0; s < NS; ++s)
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) acc[s][k2] = (Rl)0;
    for (; u < ue; ++u) {
      const int t = (int)(u - (long)kx * T);
      if (pre) {
        for (int idx = threadIdx.x; idx < nz * NP; idx += blockDim.x) P[idx] = czero<C>();
        __syncthreads();
#pragma unroll
        for (int i = 0; i < PREF; ++i) {
          const int r = threadIdx.x + i * blockDim.x;
          if (r < pg.nray) P[pg.rpos[r]] = nxt[i];
        }
        __syncthreads();
        if (u + 1 < u1) fetch(u + 1);
      } else {
        pencil_scatter<C, N>(P, rt, row_of(u), pg);
      }
      rows_nat_to_perm<C, N, 1>(P, nz, dz, tw);
      const Rl fa = (Rl)wa[t], fb = (Rl)wb[t];
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const int ti = s / reps, rr = s - ti * reps;
        const int q0 = ti * CTs, ct = min(CTs, N - q0);
        const DivMod dq(ct);
        if (rr == 0) {
          zcols_phase_a<C, N>(P, S, zp, q0, ct, dq, tw);
          __syncthreads();
        }
        const int idx = threadIdx.x + rr * PNT;
        if (idx < ct * N1) {
          int k1, qq;
          dq(idx, k1, qq);
          const C *row = S + qq * NP + k1 * N2;
          C w[N2];
#pragma unroll
          for (int j2 = 0; j2 < N2; ++j2) w[j2] = row[j2];
          Dft<C, N2, 1>::run(w);
#pragma unroll
          for (int k2 = 0; k2 < N2; ++k2) {
            const Rl re = w[k2].x, im = w[k2].y;
            acc[s][k2] += fa * re * re + fb * im * im;
          }
        }
        if (rr == reps - 1) __syncthreads();
      }
    }
    // this plane's sums -> shared memory [q][k'] (row stride N+1) -> its partial grid
    Rl *stage = reinterpret_cast<Rl *>(smraw);
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const int ti = s / reps, rr = s - ti * reps;
      const int q0 = ti * CTs, ct = min(CTs, N - q0);
      const int idx = threadIdx.x + rr * PNT;
      if (idx < ct * N1) {
        int k1, qq;
        const DivMod dq(ct);
        dq(idx, k1, qq);
        Rl *ar = stage + (q0 + qq) * NP + k1 * N2;
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) ar[k2] = acc[s][k2];
      }
    }
    __syncthreads();
    const int slot = b - bal_block((long)kx * T, U, nb);
    double *out = rho_part + ((long)slot * pg.n1 + kx) * N * N;
    for (int idx = threadIdx.x; idx < N * N; idx += blockDim.x) {
      const int q = idx / N, k = idx % N;
      out[idx] = (double)stage[q * NP + k];
    }
    __syncthreads();  // the stage overlaps P, which the next plane's first pair fills
  }
}

// position <-> index of the permuted (ky, kz) order: position a*N2 + b holds
// index a + N1*b
__device__ __forceinline__ int perm_index(int pos, int n1f, int n2f) { return pos / n2f + n1f * (pos % n2f); }

// rho[kz][ky][kx] (=, or += with add) sum over groups of rho_part[g][kx][q][k'],
// for nx x planes (n on one GPU, a rank's planes in the slab decomposition);
// ngroups grids per plane, or with bal_nblk > 0 the balanced schedule's
// bal_slots grids of each plane.
// grid ((n+31)/32, (nx+31)/32, n), block (32, 8): a 32 (k') x 32 (kx) tile of
// plane q; a thread adds the groups of its four rows together (four loads
// per group in flight; each element's sum keeps the group order), the tile
// is transposed through shared memory.
__global__ void k_rho_reduce_p(int n, int nx, int n1f, int n2f, int ngroups, const double *__restrict__ part,
                               double *__restrict__ rho, int add, int bal_T, int bal_nblk) {
  __shared__ double tile[32][33];
  const int q = blockIdx.z;
  const int k0 = blockIdx.x * 32, kx0 = blockIdx.y * 32;
  const long gstride = (long)nx * n * n;
  const int k = k0 + threadIdx.x;
  long off[4];
  int ng[4];
  double s[4];
  int gmax = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int kx = kx0 + threadIdx.y + 8 * i;
    const bool ok = kx < nx && k < n;
    ng[i] = !ok ? 0 : (bal_nblk > 0 ? bal_slots(kx, bal_T, (long)nx * bal_T, bal_nblk) : ngroups);
    gmax = max(gmax, ng[i]);
    off[i] = ok ? ((long)kx * n + q) * n + k : 0;
    s[i] = 0.0;
  }
#pragma unroll 2
  for (int g = 0; g < gmax; ++g) {
    const double *pg = part + g * gstride;
    double v[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = g < ng[i] ? pg[off[i]] : 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) s[i] += v[i];
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) tile[threadIdx.y + 8 * i][threadIdx.x] = s[i];
  __syncthreads();
  const int ky = perm_index(q, n1f, n2f);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int kk = k0 + threadIdx.y + 8 * i, kx = kx0 + threadIdx.x;
    if (kx < nx && kk < n) {
      double *o = rho + ((long)perm_index(kk, n1f, n2f) * n + ky) * nx + kx;
      const double t = tile[threadIdx.x][threadIdx.y + 8 * i];
      *o = add ? *o + t : t;
    }
  }
}

// vp[kx][q][k'] (working precision) from V[kz][ky][kx] (FP64), permuted
// order, for nx x planes
template <typename Rl>
__global__ void k_v_permute(int n, int nx, int n1f, int n2f, const double *__restrict__ v, Rl *__restrict__ vp) {
  __shared__ double tile[32][33];
  const int q = blockIdx.z;
  const int ky = perm_index(q, n1f, n2f);
  const int kx0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int k = k0 + j, kx = kx0 + threadIdx.x;
    tile[j][threadIdx.x] = (kx < nx && k < n) ? v[((long)perm_index(k, n1f, n2f) * n + ky) * nx + kx] : 0.0;
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int kx = kx0 + j, k = k0 + threadIdx.x;
    if (kx < nx && k < n) vp[((long)kx * n + q) * n + k] = (Rl)tile[threadIdx.x][j];
  }
}

// Slab decomposition: the +G / -G positions of a rank's G vectors in its
// send/return buffer [kx][t][local ray] for T pairs (row = T * local rays),
// from the planes and local rays of the two positions
__global__ void k_slab_pos(int ng, const int *__restrict__ kxp, const int *__restrict__ rlp,
                           const int *__restrict__ kxm, const int *__restrict__ rlm, long row, int *__restrict__ pp,
                           int *__restrict__ pm) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < ng) {
    pp[g] = (int)(kxp[g] * row + rlp[g]);
    pm[g] = (int)(kxm[g] * row + rlm[g]);
  }
}

}  // namespace amdk
