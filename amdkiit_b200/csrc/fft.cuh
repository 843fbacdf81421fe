// Pruned, batched 3D FFT engine for the G-sphere (sm_100a).
//
// Replaces do_fft (fft_interface.f90:33-148), which runs three FFTW passes
// with two full-grid work arrays per transform.  Here a transform is split in
// three passes whose extents follow the sphere:
//   X pass : the x-rays that carry G vectors (ngrays of the wavefunction
//            sphere, nhrays of the density sphere; PW rays are a prefix of
//            the density rays, in the reference's numbering), layout
//            R[t][ray][kx]
//   Y pass : the z planes that contain rays (the slab), layout S[t][zi][ky][kx]
//   Z pass : every (kx,ky) column of the full grid
// Each pass loads a tile of lines into shared memory (x-fastest global tiles,
// coalesced), transforms it (the two-level register FFT for the specialised
// lengths, a shared-memory Stockham mixed-radix (4,2,3,5) FFT otherwise) and
// stores the tile.  The Z pass carries the fused consumers: |psi|^2 density
// accumulation, and V(r)*psi between the backward and forward z transforms
// (the full grid is never written for H|psi>).  The band-pair transforms of
// cubic grids take the pencil path of pencil.cuh instead; these kernels
// serve the density-sphere fields and the other grids.
//
// Index convention: grid index k = (Miller index) mod N, x fastest.  The
// backward transform is sum_G c(G) exp(+iG.r) (FFTW_BACKWARD, unscaled); the
// forward one is exp(-iG.r), and the 1/N of fft_interface.f90:121 is applied
// by the gather kernels.  The reference's centred layout and its (-1)^(i+j+k)
// phasen (fft_interface.f90:515-532) are the same transform in a shifted index
// and are not needed here.
#pragma once
#include <cuda_runtime.h>

namespace amdk {

// ---------------------------------------------------------------- complex
template <typename R> struct CT;
template <> struct CT<double> { typedef double2 T; };
template <> struct CT<float> { typedef float2 T; };

__host__ __device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }
__host__ __device__ __forceinline__ float2 mk(float x, float y) { return make_float2(x, y); }
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { a.x += b.x; a.y += b.y; return a; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename C> __device__ __forceinline__ C cconjmul(C a, C b) {  // a * conj(b)
  C r;
  r.x = a.x * b.x + a.y * b.y;
  r.y = a.y * b.x - a.x * b.y;
  return r;
}
template <typename C, typename R> __device__ __forceinline__ C cscale(C a, R s) { a.x *= s; a.y *= s; return a; }
// i*sg*a
template <typename C> __device__ __forceinline__ C cimul(C a, int sg) {
  C r;
  if (sg > 0) { r.x = -a.y; r.y = a.x; }
  else { r.x = a.y; r.y = -a.x; }
  return r;
}
template <typename C> __device__ __forceinline__ C czero() { C r; r.x = 0; r.y = 0; return r; }
// a*s + b, s real
template <typename C, typename R> __device__ __forceinline__ C cfmas(C a, R s, C b) {
  b.x += a.x * s;
  b.y += a.y * s;
  return b;
}

// float2 arithmetic on the packed FP32x2 instructions of sm_100 (one
// instruction for both components)
__device__ __forceinline__ unsigned long long f2pack(float2 v) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(v.x), "f"(v.y));
  return r;
}
__device__ __forceinline__ float2 f2unpack(unsigned long long u) {
  float2 v;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(u));
  return v;
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2pack(a)), "l"(f2pack(b)));
  return f2unpack(r);
}
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2pack(a)), "l"(f2pack(b)));
  return f2unpack(r);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2pack(a)), "l"(f2pack(make_float2(s, s))));
  return f2unpack(r);
}
__device__ __forceinline__ float2 cfmas(float2 a, float s, float2 b) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(f2pack(a)), "l"(f2pack(make_float2(s, s))), "l"(f2pack(b)));
  return f2unpack(r);
}

// ---------------------------------------------------------------- plans
constexpr int MAXF = 8;
template <typename C> struct Plan {
  int n, nf;
  int f[MAXF];
  const C *w;   // w[k] = exp(-2 pi i k/n), k < n (device)
};

// Radix-r DFT with exponent sign sg: y_p = sum_q a_q exp(sg 2 pi i p q / r)
template <typename C> __device__ __forceinline__ void dft_r(C *a, int r, int sg) {
  typedef decltype(a[0].x) R;
  if (r == 2) {
    C t = a[0];
    a[0] = cadd(t, a[1]);
    a[1] = csub(t, a[1]);
  } else if (r == 4) {
    C t0 = cadd(a[0], a[2]), t1 = csub(a[0], a[2]);
    C t2 = cadd(a[1], a[3]), t3 = cimul(csub(a[1], a[3]), sg);
    a[0] = cadd(t0, t2);
    a[2] = csub(t0, t2);
    a[1] = cadd(t1, t3);
    a[3] = csub(t1, t3);
  } else if (r == 3) {
    const R c3 = (R)-0.5, s3 = (R)0.86602540378443864676;
    C t1 = cadd(a[1], a[2]), t2 = cimul(cscale(csub(a[1], a[2]), s3), sg);
    C m = cfmas(t1, c3, a[0]);
    a[0] = cadd(a[0], t1);
    a[1] = cadd(m, t2);
    a[2] = csub(m, t2);
  } else {  // r == 5
    const R c1 = (R)0.30901699437494742410, c2 = (R)-0.80901699437494742410;
    const R s1 = (R)0.95105651629515357212, s2 = (R)0.58778525229247312917;
    C t1 = cadd(a[1], a[4]), t2 = cadd(a[2], a[3]);
    C t3 = csub(a[1], a[4]), t4 = csub(a[2], a[3]);
    C m1 = cfmas(t2, c2, cfmas(t1, c1, a[0]));
    C m2 = cfmas(t2, c1, cfmas(t1, c2, a[0]));
    C n1 = cimul(cfmas(t4, s2, cscale(t3, s1)), sg);
    C n2 = cimul(cfmas(t4, -s1, cscale(t3, s2)), sg);
    a[0] = cadd(a[0], cadd(t1, t2));
    a[1] = cadd(m1, n1);
    a[4] = csub(m1, n1);
    a[2] = cadd(m2, n2);
    a[3] = csub(m2, n2);
  }
}

// Stockham FFT of L lines held in shared memory, element k of line l at
// buf[k*es + l].  Ping-pong between a and b; returns the buffer holding the
// result.  Must be called by all threads of the block.
template <typename C>
__device__ C *smem_fft(C *a, C *b, int L, int es, const Plan<C> &p, int sg) {
  const int n = p.n;
  int s = 1;
  for (int st = 0; st < p.nf; ++st) {
    const int r = p.f[st];
    const int m = n / (s * r);
    const int nbf = L * (n / r);
    for (int idx = threadIdx.x; idx < nbf; idx += blockDim.x) {
      const int l = idx % L;
      const int bf = idx / L;
      const int k = bf % s;
      const int j = bf / s;
      C v[5];
#pragma unroll 5
      for (int q = 0; q < 5; ++q)
        if (q < r) v[q] = a[(k + s * j + s * m * q) * es + l];
      dft_r(v, r, sg);
#pragma unroll 5
      for (int q = 0; q < 5; ++q)
        if (q < r) {
          int e = (s * j * q) % n;
          C w = p.w[e];
          if (sg > 0) w.y = -w.y;
          b[(k + s * q + s * r * j) * es + l] = (q == 0) ? v[q] : cmul(v[q], w);
        }
    }
    __syncthreads();
    C *t = a;
    a = b;
    b = t;
    s *= r;
  }
  return a;
}


// ---------------------------------------------------------------- register FFT
// Small DFTs held in registers (R <= 16 with factors 2, 3, 4, 5) and the
// two-level line transform N = N1*N2 built on them: each thread loads the N1
// (or N2) elements of one sub-transform, works in registers and writes back,
// so a length-N line costs two shared-memory round trips.  Twiddles
// W_R^m = exp(-2 pi i m/R) of the small DFTs (R = 2..16) sit in constant
// memory at ctw_off(R) + m and are filled by the host.
__host__ __device__ constexpr int ctw_off(int R) { return R * (R - 1) / 2 - 1; }
constexpr int CTW_LEN = ctw_off(17);
__constant__ double2 c_twd[CTW_LEN];
__constant__ float2 c_twf[CTW_LEN];
template <typename C> __device__ __forceinline__ C ctw(int i);
template <> __device__ __forceinline__ double2 ctw<double2>(int i) { return c_twd[i]; }
template <> __device__ __forceinline__ float2 ctw<float2>(int i) { return c_twf[i]; }

__host__ __device__ constexpr int reg_radix(int r) { return (r % 4 == 0) ? 4 : (r % 2 == 0) ? 2 : (r % 3 == 0) ? 3 : 5; }
// N = N1 * N2 with N1 <= N2 <= 16 and N1 as large as possible (0: none)
__host__ __device__ constexpr int fft_n1(int n) {
  int best = 0;
  for (int d = 2; d <= 16; ++d)
    if (n % d == 0 && n / d <= 16 && d <= n / d) best = d;
  return best;
}

// y_k = sum_j v_j exp(SG 2 pi i jk/R), natural order in and out
template <typename C, int R, int SG> struct Dft {
  static __device__ __forceinline__ void run(C (&v)[R]) {
    if constexpr (R == 2 || R == 3 || R == 4 || R == 5) {
      dft_r(v, R, SG);
    } else if constexpr (R > 5) {
      constexpr int A = reg_radix(R), B = R / A;
      // j = j2 + B*j1: DFT_A over j1, twiddle W_R^(j2 k1), DFT_B over j2
#pragma unroll
      for (int j2 = 0; j2 < B; ++j2) {
        C a[A];
#pragma unroll
        for (int j1 = 0; j1 < A; ++j1) a[j1] = v[j2 + B * j1];
        Dft<C, A, SG>::run(a);
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) {
          if ((j2 * k1) % R == 0) {
            v[j2 + B * k1] = a[k1];
          } else {
            C w = ctw<C>(ctw_off(R) + (j2 * k1) % R);
            if (SG > 0) w.y = -w.y;
            v[j2 + B * k1] = cmul(a[k1], w);
          }
        }
      }
      C o[R];
#pragma unroll
      for (int k1 = 0; k1 < A; ++k1) {
        C b[B];
#pragma unroll
        for (int j2 = 0; j2 < B; ++j2) b[j2] = v[j2 + B * k1];
        Dft<C, B, SG>::run(b);
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2) o[k1 + A * k2] = b[k2];
      }
#pragma unroll
      for (int k = 0; k < R; ++k) v[k] = o[k];
    }
  }
};

// Twiddles of the two-level transform of a specialised length N = N1*N2,
// built per block in shared memory (2N entries) from the plan's
// w[e] = exp(-2 pi i e/N): tw[j2*N1 + k1] = W_N^(j2 k1) (table 0, the
// twiddles of a natural-order-in transform's first phase) and
// tw[N + k1*N2 + k2] = W_N^(k1 k2) (table 1, those of a permuted-order-in
// transform's first phase).  A thread reads its row with constant offsets,
// so no exponent arithmetic is left in the butterflies.
template <typename C, int N> __device__ __forceinline__ void load_tw(C *tw, const Plan<C> &p) {
  if constexpr (N > 0) {
    constexpr int N1 = fft_n1(N), N2 = N / N1;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
      tw[i] = p.w[(i / N1) * (i % N1) % N];
      tw[N + i] = p.w[(i / N2) * (i % N2) % N];
    }
  }
}
// v[k] *= W_N^(SG j k), k = 1..R-1, from row j of twiddle table TAB (table 0
// for R = N1, j = j2; table 1 for R = N2, j = k1).  VEC: the table starts on a
// 16-byte boundary (the caller guarantees it), so FP32 rows of even length are
// read two twiddles per load.
template <typename C, int N, int R, int SG, int TAB, bool VEC = false>
__device__ __forceinline__ void twiddle_tab(C (&v)[R], int j, const C *tw) {
  const C *row = tw + TAB * N + j * R;
  if constexpr (VEC && sizeof(C) == 8 && R % 2 == 0 && N % 2 == 0) {
    const float4 *r4 = reinterpret_cast<const float4 *>(row);
#pragma unroll
    for (int k2 = 0; k2 < R / 2; ++k2) {
      const float4 q = r4[k2];
      C wa, wb;
      wa.x = q.x;
      wa.y = SG > 0 ? -q.y : q.y;
      wb.x = q.z;
      wb.y = SG > 0 ? -q.w : q.w;
      if (k2 > 0) v[2 * k2] = cmul(v[2 * k2], wa);
      v[2 * k2 + 1] = cmul(v[2 * k2 + 1], wb);
    }
  } else {
#pragma unroll
    for (int k = 1; k < R; ++k) {
      C w = row[k];
      if (SG > 0) w.y = -w.y;
      v[k] = cmul(v[k], w);
    }
  }
}

// Two-level register FFT of a tile of L lines (element k of line l at
// a[k*ES + l]), natural order in a, natural order out in b: phase A in place
// in a (thread (l, j2): DFT_N1 of elements j2 + N2*j1, twiddle, back to
// k1*N2 + j2), phase B from a to b (thread (l, k1): DFT_N2 of the N2
// contiguous elements, out to k1 + N1*k2).
template <typename C, int N, int L, int ES, int SG>
__device__ __forceinline__ void tile_reg_fft(C *a, C *b, const C *tw) {
  constexpr int N1 = fft_n1(N), N2 = N / N1;
  for (int idx = threadIdx.x; idx < L * N2; idx += blockDim.x) {
    const int l = idx % L, j2 = idx / L;
    C v[N1];
#pragma unroll
    for (int j1 = 0; j1 < N1; ++j1) v[j1] = a[(j2 + N2 * j1) * ES + l];
    Dft<C, N1, SG>::run(v);
    twiddle_tab<C, N, N1, SG, 0>(v, j2, tw);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) a[(k1 * N2 + j2) * ES + l] = v[k1];
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < L * N1; idx += blockDim.x) {
    const int l = idx % L, k1 = idx / L;
    C u[N2];
#pragma unroll
    for (int j2 = 0; j2 < N2; ++j2) u[j2] = a[(k1 * N2 + j2) * ES + l];
    Dft<C, N2, SG>::run(u);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) b[(k1 + N1 * k2) * ES + l] = u[k2];
  }
  __syncthreads();
}

// FFT of a tile of L lines (element k of line l at buf[k*ES + l]); returns
// the buffer that holds the result.  N = 0 is the run-time-length Stockham
// path; a specialised N uses the register FFT (tw: shared copy of p.w).
template <typename C, int N, int L, int ES>
__device__ __forceinline__ C *fft_tile(C *a, C *b, const Plan<C> &p, const C *tw, int sg) {
  if constexpr (N == 0) {
    return smem_fft(a, b, L, ES, p, sg);
  } else {
    if (sg > 0) tile_reg_fft<C, N, L, ES, 1>(a, b, tw);
    else tile_reg_fft<C, N, L, ES, -1>(a, b, tw);
    return b;
  }
}

// ---------------------------------------------------------------- geometry
struct Geom {
  int n1, n2, n3;
  int ngpw, ngrho;
  int nray[2];            // rays of the PW (0) / density (1) sphere
  const int *gmap;        // [nhrays*n1]: +(ig+1) at +G, -(ig+1) at -G, 0 empty
  const int *pos_p;       // [ngrho] ray*n1 + kx of +G
  const int *pos_m;       // [ngrho] ray*n1 + kx of -G
  int nz[2];              // slab planes per sphere
  const int *zlist[2];    // [nz] kz of each slab plane
  const int *rayidx[2];   // [nz*n2] ray of (zi, ky) or -1
};

constexpr int TX = 16;    // x-extent of a Y/Z tile (16 complex = 256 B in FP64)
constexpr int LX = 8;     // lines per X-pass block

// ---------------------------------------------------------------- X pass
// Backward X pass with the band-pair pack fused (vpsi/eval_density pack,
// wfn_initialize.f90:286-308, density.f90:26-47): psi_a + i psi_b.
template <typename C, int N = 0>
__global__ void __launch_bounds__(256) k_x_bwd_pair(const double2 *__restrict__ c0, int ngpw, int nstate, int band0, int T,
                                                    Geom g, Plan<C> p, C *__restrict__ rb) {
  extern __shared__ unsigned char smraw[];
  C *sa = reinterpret_cast<C *>(smraw);
  const int n1 = g.n1, R = g.nray[0];
  const int es = LX + 1;
  C *sb = sa + n1 * es;
  C *tw = sb + n1 * es;
  load_tw<C, N>(tw, p);
  const long line0 = (long)blockIdx.x * LX;
  const long nlines = (long)T * R;
  for (int idx = threadIdx.x; idx < LX * n1; idx += blockDim.x) {
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
    sa[k * es + l] = v;
  }
  __syncthreads();
  C *res = fft_tile<C, N, LX, LX + 1>(sa, sb, p, tw, +1);
  for (int idx = threadIdx.x; idx < LX * n1; idx += blockDim.x) {
    const int l = idx / n1, k = idx % n1;
    const long line = line0 + l;
    if (line < nlines) rb[line * n1 + k] = res[k * es + l];
  }
}

// Backward X pass from a G field given at +G (fp) and -G (fm), t-th field at
// fp + t*ngrho (eval_pot / rhog2r / GRAD_CAL packs).
template <typename C, int N = 0>
__global__ void __launch_bounds__(256) k_x_bwd_field(const double2 *__restrict__ fp, const double2 *__restrict__ fm, int ngmax,
                                                     int sphere, int T, Geom g, Plan<C> p, C *__restrict__ rb) {
  extern __shared__ unsigned char smraw[];
  C *sa = reinterpret_cast<C *>(smraw);
  const int n1 = g.n1, R = sphere ? g.nray[1] : g.nray[0];
  const int es = LX + 1;
  C *sb = sa + n1 * es;
  C *tw = sb + n1 * es;
  load_tw<C, N>(tw, p);
  const long line0 = (long)blockIdx.x * LX;
  const long nlines = (long)T * R;
  auto gather = [&](int idx) {
    const int l = idx / n1, k = idx % n1;
    const long line = line0 + l;
    C v = czero<C>();
    if (line < nlines) {
      const int t = (int)(line / R), r = (int)(line % R);
      const int code = g.gmap[(long)r * n1 + k];
      const int ig = (code > 0 ? code : -code) - 1;
      if (code != 0 && ig < ngmax) {
        double2 a = (code > 0) ? fp[(long)t * ngmax + ig] : fm[(long)t * ngmax + ig];
        v = mk((decltype(v.x))a.x, (decltype(v.x))a.y);
      }
    }
    return v;
  };
  if constexpr (N > 0) {
    // all of a thread's gathers in flight at once (256 threads per block)
    constexpr int CNT = (LX * N + 255) / 256;
    C v[CNT];
#pragma unroll
    for (int i = 0; i < CNT; ++i) {
      const int idx = threadIdx.x + 256 * i;
      v[i] = idx < LX * N ? gather(idx) : czero<C>();
    }
#pragma unroll
    for (int i = 0; i < CNT; ++i) {
      const int idx = threadIdx.x + 256 * i;
      if (idx < LX * N) sa[(idx % N) * es + idx / N] = v[i];
    }
  } else {
    for (int idx = threadIdx.x; idx < LX * n1; idx += blockDim.x) sa[(idx % n1) * es + idx / n1] = gather(idx);
  }
  __syncthreads();
  C *res = fft_tile<C, N, LX, LX + 1>(sa, sb, p, tw, +1);
  for (int idx = threadIdx.x; idx < LX * n1; idx += blockDim.x) {
    const int l = idx / n1, k = idx % n1;
    const long line = line0 + l;
    if (line < nlines) rb[line * n1 + k] = res[k * es + l];
  }
}

// Forward X pass in place on the ray buffer.
template <typename C, int N = 0>
__global__ void __launch_bounds__(256) k_x_fwd(int sphere, int T, Geom g, Plan<C> p, C *__restrict__ rb) {
  extern __shared__ unsigned char smraw[];
  C *sa = reinterpret_cast<C *>(smraw);
  const int n1 = g.n1, R = sphere ? g.nray[1] : g.nray[0];
  const int es = LX + 1;
  C *sb = sa + n1 * es;
  C *tw = sb + n1 * es;
  load_tw<C, N>(tw, p);
  const long line0 = (long)blockIdx.x * LX;
  const long nlines = (long)T * R;
  for (int idx = threadIdx.x; idx < LX * n1; idx += blockDim.x) {
    const int l = idx / n1, k = idx % n1;
    const long line = line0 + l;
    sa[k * es + l] = (line < nlines) ? rb[line * n1 + k] : czero<C>();
  }
  __syncthreads();
  C *res = fft_tile<C, N, LX, LX + 1>(sa, sb, p, tw, -1);
  for (int idx = threadIdx.x; idx < LX * n1; idx += blockDim.x) {
    const int l = idx / n1, k = idx % n1;
    const long line = line0 + l;
    if (line < nlines) rb[line * n1 + k] = res[k * es + l];
  }
}

// ---------------------------------------------------------------- Y pass
// grid: (ceil(n1/TX), nz[sphere], T).  dir=+1 backward (rays -> slab),
// dir=-1 forward (slab -> rays).
template <typename C, int N = 0>
__global__ void __launch_bounds__(256) k_y(int sphere, int dir, Geom g, Plan<C> p, C *__restrict__ rb, C *__restrict__ sbuf,
                                           long rstride, long sstride) {
  extern __shared__ unsigned char smraw[];
  C *sa = reinterpret_cast<C *>(smraw);
  const int n1 = g.n1, n2 = g.n2, nz = sphere ? g.nz[1] : g.nz[0];
  C *sb = sa + n2 * TX;
  C *tw = sb + n2 * TX;
  load_tw<C, N>(tw, p);
  const int kx0 = blockIdx.x * TX, zi = blockIdx.y, t = blockIdx.z;
  const int *ri = (sphere ? g.rayidx[1] : g.rayidx[0]) + (long)zi * n2;
  C *R = rb + (long)t * rstride;
  C *S = sbuf + (long)t * sstride + (long)zi * n2 * n1;
  auto fetch = [&](int idx) {
    const int ky = idx / TX, tx = idx % TX, kx = kx0 + tx;
    C v = czero<C>();
    if (kx < n1) {
      if (dir > 0) {
        const int r = ri[ky];
        if (r >= 0) v = R[(long)r * n1 + kx];
      } else {
        v = S[(long)ky * n1 + kx];
      }
    }
    return v;
  };
  if constexpr (N > 0) {
    // all of a thread's loads in flight at once (256 threads per block)
    constexpr int CNT = (TX * N + 255) / 256;
    C v[CNT];
#pragma unroll
    for (int i = 0; i < CNT; ++i) {
      const int idx = threadIdx.x + 256 * i;
      v[i] = idx < TX * N ? fetch(idx) : czero<C>();
    }
#pragma unroll
    for (int i = 0; i < CNT; ++i) {
      const int idx = threadIdx.x + 256 * i;
      if (idx < TX * N) sa[idx] = v[i];
    }
  } else {
    for (int idx = threadIdx.x; idx < TX * n2; idx += blockDim.x) sa[idx] = fetch(idx);
  }
  __syncthreads();
  C *res = fft_tile<C, N, TX, TX>(sa, sb, p, tw, dir);
  for (int idx = threadIdx.x; idx < TX * n2; idx += blockDim.x) {
    const int ky = idx / TX, tx = idx % TX, kx = kx0 + tx;
    if (kx >= n1) continue;
    if (dir > 0) {
      S[(long)ky * n1 + kx] = res[ky * TX + tx];
    } else {
      const int r = ri[ky];
      if (r >= 0) R[(long)r * n1 + kx] = res[ky * TX + tx];
    }
  }
  (void)nz;
}

// ---------------------------------------------------------------- Z pass
enum { Z_TO_GRID = 0, Z_FROM_GRID_REAL = 1, Z_FROM_GRID_CPLX = 2, Z_VPSI = 3, Z_DENSITY = 4 };

// grid: (ceil(n1/TX), n2, T) for TO_GRID/FROM_GRID/VPSI; (ceil(n1/TX), n2, 1)
// for DENSITY, which loops over the T transforms of the batch.
//   TO_GRID          slab -> complex grid (double2)                    backward
//   FROM_GRID_REAL   real grid (double) -> slab                        forward
//   FROM_GRID_CPLX   complex grid (double2) -> slab                    forward
//   VPSI             slab -> (bwd) * V(r) -> (fwd) -> slab  (vpsi, wfn_initialize.f90:311-340)
//   DENSITY          slab -> (bwd) -> rho += f_a/Omega Re^2 + f_b/Omega Im^2 (density.f90:49-86)
template <typename C, int MODE, int N = 0>
__global__ void __launch_bounds__(256) k_z(int sphere, int T, Geom g, Plan<C> p, C *__restrict__ sbuf, long sstride,
                                           double2 *__restrict__ cgrid, const double *__restrict__ rgrid, long gstride,
                                           const double *__restrict__ vpot, double *__restrict__ rho,
                                           const double *__restrict__ wa, const double *__restrict__ wb) {
  typedef decltype(C().x) R;
  extern __shared__ unsigned char smraw[];
  C *sa = reinterpret_cast<C *>(smraw);
  const int n1 = g.n1, n2 = g.n2, n3 = g.n3, nz = sphere ? g.nz[1] : g.nz[0];
  C *sb = sa + n3 * TX;
  C *tw = sb + n3 * TX;
  load_tw<C, N>(tw, p);
  const int kx0 = blockIdx.x * TX, ky = blockIdx.y;
  const int *zl = sphere ? g.zlist[1] : g.zlist[0];
  const long plane = (long)n2 * n1;
  double acc[16];  // TX*n3 <= 16*blockDim (checked at setup)
  if (MODE == Z_DENSITY)
    for (int i = 0; i < 16; ++i) acc[i] = 0.0;
  const int tb = (MODE == Z_DENSITY) ? 0 : blockIdx.z;
  const int te = (MODE == Z_DENSITY) ? T : blockIdx.z + 1;
  for (int t = tb; t < te; ++t) {
    C *S = sbuf + (long)t * sstride;
    if (MODE == Z_TO_GRID || MODE == Z_VPSI || MODE == Z_DENSITY) {
      if constexpr (N > 0) {
        // the slab loads are issued before the clearing barrier (256 threads per block)
        constexpr int CNT = (TX * N + 255) / 256;
        C v[CNT];
        int dst[CNT];
#pragma unroll
        for (int i = 0; i < CNT; ++i) {
          const int idx = threadIdx.x + 256 * i;
          dst[i] = -1;
          if (idx < TX * nz) {
            const int zi = idx / TX, tx = idx % TX, kx = kx0 + tx;
            if (kx < n1) {
              v[i] = S[(long)zi * plane + (long)ky * n1 + kx];
              dst[i] = zl[zi] * TX + tx;
            }
          }
        }
        for (int idx = threadIdx.x; idx < TX * n3; idx += blockDim.x) sa[idx] = czero<C>();
        __syncthreads();
#pragma unroll
        for (int i = 0; i < CNT; ++i)
          if (dst[i] >= 0) sa[dst[i]] = v[i];
      } else {
        for (int idx = threadIdx.x; idx < TX * n3; idx += blockDim.x) sa[idx] = czero<C>();
        __syncthreads();
        for (int idx = threadIdx.x; idx < TX * nz; idx += blockDim.x) {
          const int zi = idx / TX, tx = idx % TX, kx = kx0 + tx;
          if (kx < n1) sa[zl[zi] * TX + tx] = S[(long)zi * plane + (long)ky * n1 + kx];
        }
      }
      __syncthreads();
      C *res = fft_tile<C, N, TX, TX>(sa, sb, p, tw, +1);
      if (MODE == Z_TO_GRID) {
        double2 *G = cgrid + (long)t * gstride;
        for (int idx = threadIdx.x; idx < TX * n3; idx += blockDim.x) {
          const int kz = idx / TX, tx = idx % TX, kx = kx0 + tx;
          if (kx < n1) {
            C v = res[idx];
            G[(long)kz * plane + (long)ky * n1 + kx] = make_double2((double)v.x, (double)v.y);
          }
        }
        __syncthreads();
      } else if (MODE == Z_DENSITY) {
        const double fa = wa[t], fb = wb[t];
        int i = 0;
        for (int idx = threadIdx.x; idx < TX * n3; idx += blockDim.x, ++i) {
          C v = res[idx];
          double re = (double)v.x, im = (double)v.y;
          acc[i] += fa * re * re + fb * im * im;
        }
        __syncthreads();
      } else {  // VPSI
        C *other = (res == sa) ? sb : sa;
        for (int idx = threadIdx.x; idx < TX * n3; idx += blockDim.x) {
          const int kz = idx / TX, tx = idx % TX, kx = kx0 + tx;
          R v = (kx < n1) ? (R)vpot[(long)kz * plane + (long)ky * n1 + kx] : (R)0;
          res[idx] = cscale(res[idx], v);
        }
        __syncthreads();
        C *out = fft_tile<C, N, TX, TX>(res, other, p, tw, -1);
        for (int idx = threadIdx.x; idx < TX * nz; idx += blockDim.x) {
          const int zi = idx / TX, tx = idx % TX, kx = kx0 + tx;
          if (kx < n1) S[(long)zi * plane + (long)ky * n1 + kx] = out[zl[zi] * TX + tx];
        }
        __syncthreads();
      }
    } else {  // FROM_GRID
      auto fetch = [&](int idx) {
        const int kz = idx / TX, tx = idx % TX, kx = kx0 + tx;
        C v = czero<C>();
        if (kx < n1) {
          const long o = (long)t * gstride + (long)kz * plane + (long)ky * n1 + kx;
          if (MODE == Z_FROM_GRID_REAL) v.x = (R)rgrid[o];
          else { double2 c = cgrid[o]; v.x = (R)c.x; v.y = (R)c.y; }
        }
        return v;
      };
      if constexpr (N > 0) {
        constexpr int CNT = (TX * N + 255) / 256;
        C v[CNT];
#pragma unroll
        for (int i = 0; i < CNT; ++i) {
          const int idx = threadIdx.x + 256 * i;
          v[i] = idx < TX * N ? fetch(idx) : czero<C>();
        }
#pragma unroll
        for (int i = 0; i < CNT; ++i) {
          const int idx = threadIdx.x + 256 * i;
          if (idx < TX * N) sa[idx] = v[i];
        }
      } else {
        for (int idx = threadIdx.x; idx < TX * n3; idx += blockDim.x) sa[idx] = fetch(idx);
      }
      __syncthreads();
      C *res = fft_tile<C, N, TX, TX>(sa, sb, p, tw, -1);
      for (int idx = threadIdx.x; idx < TX * nz; idx += blockDim.x) {
        const int zi = idx / TX, tx = idx % TX, kx = kx0 + tx;
        if (kx < n1) S[(long)zi * plane + (long)ky * n1 + kx] = res[zl[zi] * TX + tx];
      }
      __syncthreads();
    }
  }
  if (MODE == Z_DENSITY) {
    int i = 0;
    for (int idx = threadIdx.x; idx < TX * n3; idx += blockDim.x, ++i) {
      const int kz = idx / TX, tx = idx % TX, kx = kx0 + tx;
      if (kx < n1) rho[(long)kz * plane + (long)ky * n1 + kx] += acc[i];
    }
  }
}

}  // namespace amdk
