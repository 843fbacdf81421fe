// "Pencil" path for the band-pair transforms of vpsi and eval_density
// (wfn_initialize.f90:283-362, density.f90:19-90) on cubic grids.
//
// The x pass writes the ray buffer transposed, RT[t][kx][ray], so that one
// block can take one x-plane of one band pair: it scatters the plane's rays
// into a shared-memory slab plane P[zi][ky] (only the z planes that carry
// rays), runs the y FFTs, then per chunk of ky columns the z FFT, V(r)*psi
// and the inverse z FFT (or the |psi|^2 accumulation), the inverse y FFTs,
// and gathers the rays back.  No slab or grid buffer goes through HBM; the
// only HBM traffic is the ray buffer (read and written once per pass), V
// (L2 resident) and the coefficients.
#pragma once
#include "fft.cuh"

namespace amdk {

struct PencilGeom {
  int n1, n2, n3, nray, nz;
  const int *rpos;   // [nray] zi*(n2+1) + ky of the ray in the padded plane
  const int *zinv;   // [n3] slab index of kz, -1 outside the slab
  const int *zlist;  // [nz] kz of slab plane
};

constexpr int PL = 16;    // lines per scratch tile in the pencil kernel
constexpr int PNT = 512;  // maximum threads per pencil block
// The plane P[zi][ky] is stored with row stride N+1 so that the y-tile
// gathers (stride one row per line) hit distinct shared-memory banks.

// Backward x pass with the pair pack, output transposed: RT[t][kx][r]
template <typename C, int N>
__global__ void __launch_bounds__(256) k_xt_bwd_pair(const double2 *__restrict__ c0, int ngpw, int nstate, int band0,
                                                     int T, Geom g, Plan<C> p, C *__restrict__ rt) {
  extern __shared__ unsigned char smraw[];
  constexpr int L = 16, ES = L + 1;
  C *sa = reinterpret_cast<C *>(smraw);
  const int n1 = g.n1, R = g.nray[0];
  C *sb = sa + n1 * ES;
  C *tw = sb + n1 * ES;
  load_tw<C, N>(tw, p);
  const long line0 = (long)blockIdx.x * L;
  const long nlines = (long)T * R;
  for (int idx = threadIdx.x; idx < L * n1; idx += blockDim.x) {
    const int l = idx / n1, k = idx % n1;
    const long line = line0 + l;
    C v = czero<C>();
    if (line < nlines) {
      const int t = (int)(line / R), r = (int)(line % R);
      const int code = g.gmap[(long)r * n1 + k];
      const int ig = (code > 0 ? code : -code) - 1;
      if (code != 0 && ig < ngpw) {
        const int ba = band0 + 2 * t, bb = ba + 1;
        double2 a = c0[(long)ba * ngpw + ig];
        double2 b = (bb < nstate) ? c0[(long)bb * ngpw + ig] : make_double2(0.0, 0.0);
        if (code > 0) v = mk((decltype(v.x))(a.x - b.y), (decltype(v.x))(a.y + b.x));
        else v = mk((decltype(v.x))(a.x + b.y), (decltype(v.x))(-a.y + b.x));
      }
    }
    sa[k * ES + l] = v;
  }
  __syncthreads();
  C *res = fft_tile<C, N, L, ES>(sa, sb, p, tw, +1);
  // transposed store: consecutive threads take consecutive rays of one kx
  for (int idx = threadIdx.x; idx < L * n1; idx += blockDim.x) {
    const int k = idx / L, l = idx % L;
    const long line = line0 + l;
    if (line < nlines) {
      const int t = (int)(line / R), r = (int)(line % R);
      rt[((long)t * n1 + k) * R + r] = res[k * ES + l];
    }
  }
}

// Forward x pass in place on the transposed ray buffer
template <typename C, int N>
__global__ void __launch_bounds__(256) k_xt_fwd(int T, Geom g, Plan<C> p, C *__restrict__ rt) {
  extern __shared__ unsigned char smraw[];
  constexpr int L = 16, ES = L + 1;
  C *sa = reinterpret_cast<C *>(smraw);
  const int n1 = g.n1, R = g.nray[0];
  C *sb = sa + n1 * ES;
  C *tw = sb + n1 * ES;
  load_tw<C, N>(tw, p);
  const long line0 = (long)blockIdx.x * L;
  const long nlines = (long)T * R;
  for (int idx = threadIdx.x; idx < L * n1; idx += blockDim.x) {
    const int k = idx / L, l = idx % L;
    const long line = line0 + l;
    C v = czero<C>();
    if (line < nlines) {
      const int t = (int)(line / R), r = (int)(line % R);
      v = rt[((long)t * n1 + k) * R + r];
    }
    sa[k * ES + l] = v;
  }
  __syncthreads();
  C *res = fft_tile<C, N, L, ES>(sa, sb, p, tw, -1);
  for (int idx = threadIdx.x; idx < L * n1; idx += blockDim.x) {
    const int k = idx / L, l = idx % L;
    const long line = line0 + l;
    if (line < nlines) {
      const int t = (int)(line / R), r = (int)(line % R);
      rt[((long)t * n1 + k) * R + r] = res[k * ES + l];
    }
  }
}

// y FFTs of the nz slab lines of the plane P[zi][ky] in tiles of PL lines
template <typename C, int N>
__device__ __forceinline__ void pencil_y(C *P, C *s0, C *s1, const Plan<C> &p, const C *tw, int nz, int sg) {
  for (int z0 = 0; z0 < nz; z0 += PL) {
    for (int idx = threadIdx.x; idx < PL * N; idx += blockDim.x) {
      const int ky = idx / PL, l = idx % PL;
      s0[idx] = (z0 + l < nz) ? P[(z0 + l) * (N + 1) + ky] : czero<C>();
    }
    __syncthreads();
    C *res = fft_tile<C, N, PL, PL>(s0, s1, p, tw, sg);
    for (int idx = threadIdx.x; idx < PL * N; idx += blockDim.x) {
      const int ky = idx / PL, l = idx % PL;
      if (z0 + l < nz) P[(z0 + l) * (N + 1) + ky] = res[idx];
    }
    __syncthreads();
  }
}

// scatter the rays of plane kx of transform t into P (zero elsewhere)
template <typename C, int N>
__device__ __forceinline__ void pencil_scatter(C *P, const C *__restrict__ rt_plane, const PencilGeom &pg) {
  for (int idx = threadIdx.x; idx < pg.nz * (N + 1); idx += blockDim.x) P[idx] = czero<C>();
  __syncthreads();
  for (int r = threadIdx.x; r < pg.nray; r += blockDim.x) P[pg.rpos[r]] = rt_plane[r];
  __syncthreads();
}

// One x-plane of one band pair through y, z, V(r), z, y (vpsi :311-340).
// grid (n1, T); V_T[kx][ky][kz] in the working precision.
template <typename C, int N>
__global__ void __launch_bounds__(PNT) k_pencil_vpsi(PencilGeom pg, Plan<C> p, C *__restrict__ rt,
                                                     const decltype(C().x) *__restrict__ vt) {
  typedef decltype(C().x) Rl;
  extern __shared__ unsigned char smraw[];
  const int nz = pg.nz;
  C *P = reinterpret_cast<C *>(smraw);
  C *s0 = P + nz * (N + 1);
  C *s1 = s0 + PL * N;
  C *tw = s1 + PL * N;
  load_tw<C, N>(tw, p);
  const int kx = blockIdx.x, t = blockIdx.y;
  C *plane = rt + ((long)t * pg.n1 + kx) * pg.nray;
  pencil_scatter<C, N>(P, plane, pg);
  pencil_y<C, N>(P, s0, s1, p, tw, nz, +1);
  const Rl *V = vt + (long)kx * N * N;
  for (int y0 = 0; y0 < N; y0 += PL) {
    // column tile: element kz of column l (= ky - y0) at s0[kz*PL + l]
    for (int idx = threadIdx.x; idx < PL * N; idx += blockDim.x) {
      const int kz = idx / PL, l = idx % PL;
      const int zi = pg.zinv[kz];
      s0[idx] = (zi >= 0 && y0 + l < N) ? P[zi * (N + 1) + y0 + l] : czero<C>();
    }
    __syncthreads();
    C *res = fft_tile<C, N, PL, PL>(s0, s1, p, tw, +1);
    C *other = (res == s0) ? s1 : s0;
    // V tile staged through the free buffer: coalesced along kz, row stride N+1
    Rl *vs = reinterpret_cast<Rl *>(other);
    for (int idx = threadIdx.x; idx < PL * N; idx += blockDim.x) {
      const int l = idx / N, kz = idx % N;
      vs[l * (N + 1) + kz] = (y0 + l < N) ? V[(long)(y0 + l) * N + kz] : (Rl)0;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < PL * N; idx += blockDim.x) {
      const int kz = idx / PL, l = idx % PL;
      res[idx] = cscale(res[idx], vs[l * (N + 1) + kz]);
    }
    __syncthreads();
    C *out = fft_tile<C, N, PL, PL>(res, other, p, tw, -1);
    for (int idx = threadIdx.x; idx < PL * nz; idx += blockDim.x) {
      const int zi = idx / PL, l = idx % PL;
      if (y0 + l < N) P[zi * (N + 1) + y0 + l] = out[pg.zlist[zi] * PL + l];
    }
    __syncthreads();
  }
  pencil_y<C, N>(P, s0, s1, p, tw, nz, -1);
  for (int r = threadIdx.x; r < pg.nray; r += blockDim.x) plane[r] = P[pg.rpos[r]];
}

// Density: one x-plane for a group of band pairs; rho_part[grp][kx][ky][kz]
// += sum_t wa_t Re^2 + wb_t Im^2 (density.f90:49-86).  grid (n1, ngroups).
template <typename C, int N>
__global__ void __launch_bounds__(PNT) k_pencil_density(PencilGeom pg, Plan<C> p, const C *__restrict__ rt, int T,
                                                        int per_group, const double *__restrict__ wa,
                                                        const double *__restrict__ wb, double *__restrict__ rho_part) {
  extern __shared__ unsigned char smraw[];
  const int nz = pg.nz;
  double *acc = reinterpret_cast<double *>(smraw);        // [ky][kz], row stride N+1
  C *P = reinterpret_cast<C *>(acc + N * (N + 1));
  C *s0 = P + nz * (N + 1);
  C *s1 = s0 + PL * N;
  C *tw = s1 + PL * N;
  load_tw<C, N>(tw, p);
  for (int idx = threadIdx.x; idx < N * (N + 1); idx += blockDim.x) acc[idx] = 0.0;
  const int kx = blockIdx.x, grp = blockIdx.y;
  const int t0 = grp * per_group, t1 = min(T, t0 + per_group);
  for (int t = t0; t < t1; ++t) {
    const C *plane = rt + ((long)t * pg.n1 + kx) * pg.nray;
    pencil_scatter<C, N>(P, plane, pg);
    pencil_y<C, N>(P, s0, s1, p, tw, nz, +1);
    const double fa = wa[t], fb = wb[t];
    for (int y0 = 0; y0 < N; y0 += PL) {
      for (int idx = threadIdx.x; idx < PL * N; idx += blockDim.x) {
        const int kz = idx / PL, l = idx % PL;
        const int zi = pg.zinv[kz];
        s0[idx] = (zi >= 0 && y0 + l < N) ? P[zi * (N + 1) + y0 + l] : czero<C>();
      }
      __syncthreads();
      C *res = fft_tile<C, N, PL, PL>(s0, s1, p, tw, +1);
      for (int idx = threadIdx.x; idx < PL * N; idx += blockDim.x) {
        const int kz = idx / PL, l = idx % PL;
        if (y0 + l < N) {
          const C v = res[idx];
          const double re = (double)v.x, im = (double)v.y;
          acc[(y0 + l) * (N + 1) + kz] += fa * re * re + fb * im * im;
        }
      }
      __syncthreads();
    }
  }
  double *out = rho_part + ((long)grp * pg.n1 + kx) * N * N;
  for (int idx = threadIdx.x; idx < N * N; idx += blockDim.x) {
    const int ky = idx / N, kz = idx % N;
    out[idx] += acc[ky * (N + 1) + kz];
  }
}

// rho[kz][ky][kx] = sum over groups of rho_part[g][kx][ky][kz]
__global__ void k_rho_reduce_t(int n1, int n2, int n3, int ngroups, const double *__restrict__ part, double *__restrict__ rho) {
  __shared__ double tile[32][33];
  // tile over (kx, kz) at fixed ky: read along kz, write along kx
  const int ky = blockIdx.z;
  const int kz0 = blockIdx.x * 32, kx0 = blockIdx.y * 32;
  const long gstride = (long)n1 * n2 * n3;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int kx = kx0 + j, kz = kz0 + threadIdx.x;
    double s = 0.0;
    if (kx < n1 && kz < n3)
      for (int g = 0; g < ngroups; ++g) s += part[g * gstride + ((long)kx * n2 + ky) * n3 + kz];
    tile[j][threadIdx.x] = s;
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int kz = kz0 + j, kx = kx0 + threadIdx.x;
    if (kx < n1 && kz < n3) rho[((long)kz * n2 + ky) * n1 + kx] = tile[threadIdx.x][j];
  }
}

// V_T[kx][ky][kz] (working precision) from V[kz][ky][kx] (FP64)
template <typename Rl>
__global__ void k_v_transpose(int n1, int n2, int n3, const double *__restrict__ v, Rl *__restrict__ vt) {
  __shared__ double tile[32][33];
  const int ky = blockIdx.z;
  const int kx0 = blockIdx.x * 32, kz0 = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int kz = kz0 + j, kx = kx0 + threadIdx.x;
    tile[j][threadIdx.x] = (kx < n1 && kz < n3) ? v[((long)kz * n2 + ky) * n1 + kx] : 0.0;
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int kx = kx0 + j, kz = kz0 + threadIdx.x;
    if (kx < n1 && kz < n3) vt[((long)kx * n2 + ky) * n3 + kz] = (Rl)tile[threadIdx.x][j];
  }
}

}  // namespace amdk
