// Non-FFT kernels of libamdk (FP64 unless stated).  Each kernel names the
// reference routine it implements (paths relative to the AMDKIIT project root).
#pragma once
#include <cuda_runtime.h>

#include "fft.cuh"

namespace amdk {

constexpr int RED_BLOCKS = 1184;  // 8 x 148 SMs: enough loads in flight for the streaming reductions
constexpr int NTHR = 256;

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// block sum in fixed order (deterministic for a fixed launch shape)
__device__ double block_sum(double v, double *sh) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r += sh[i];
  return r;  // valid in thread 0
}
__device__ double block_max(double v, double *sh) {
  v = warp_max(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = -1.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r = fmax(r, sh[i]);
  return r;
}
// sum partials[k*nb .. k*nb+nb) -> out[k], for k < nk (one block per k)
__global__ void k_finish_sum(const double *part, int nb, double *out, int nk) {
  __shared__ double sh[32];
  const int k = blockIdx.x;
  double v = 0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) v += part[(long)k * nb + i];
  double r = block_sum(v, sh);
  if (threadIdx.x == 0 && k < nk) out[k] = r;
}

// Reductions finished by the kernel that produces them: each block reduces
// its threads' v[k] (a sum, or a max for the bits of MAXMASK), writes its
// partials part[k*gridDim + block], and the last block to arrive (an atomic
// ticket taken after a fence) reduces the partials in block order into out[k]
// and re-arms the ticket.  Deterministic for a fixed launch shape; one launch
// instead of a partials kernel and a finishing kernel.  Every thread of every
// block must call it; a ticket serves one kernel at a time.
template <int NK, unsigned MAXMASK = 0u>
__device__ void reduce_and_finish(const double (&v)[NK], double *part, double *out, unsigned *ticket) {
  __shared__ double sh[32];
  __shared__ unsigned last;
  double r[NK];
#pragma unroll
  for (int k = 0; k < NK; ++k) r[k] = ((MAXMASK >> k) & 1u) ? block_max(v[k], sh) : block_sum(v[k], sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NK; ++k) part[(long)k * gridDim.x + blockIdx.x] = r[k];
    __threadfence();
    last = (atomicAdd(ticket, 1u) == gridDim.x - 1) ? 1u : 0u;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
#pragma unroll
  for (int k = 0; k < NK; ++k) {
    const bool mx = (MAXMASK >> k) & 1u;
    double a = mx ? -1.0 : 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
      const double x = __ldcg(part + (long)k * gridDim.x + i);
      a = mx ? fmax(a, x) : a + x;
    }
    const double t = mx ? block_max(a, sh) : block_sum(a, sh);
    if (threadIdx.x == 0) out[k] = t;
  }
  if (threadIdx.x == 0) *ticket = 0u;
}
// slots of the device scalar array: CG norms, energy sums, GEMAX, CG step
enum { S_GGPREV = 1, S_EH = 2, S_ELOC, S_EXC, S_EKIN, S_ENL, S_ISTEP = 8, S_GMAX = 9, S_GG = 10, S_NSCAL = 16 };
// tickets of the self-finishing reductions (one per kernel)
enum { TK_VLOC = 0, TK_XC, TK_ENL, TK_EKIN, TK_GRAD, TK_N = 8 };

// ---------------------------------------------------------------- tables
// spline_inter (spline_inter.f90:1-36) evaluated at one point; the hunt is
// spline_hunt's linear search done by bisection (same interval).  Points
// beyond the last abscissa return 0, as the reference leaves them unset.
__device__ double spline_at(const double *xp, const double *yp, const double *h, const double *sdd, int n, double x) {
  if (x > xp[n - 1]) return 0.0;
  int ig;
  if (!(x < xp[n - 1])) ig = 1;
  else {
    int lo = 2, hi = n;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (x < xp[mid - 1]) hi = mid;
      else lo = mid + 1;
    }
    ig = lo - 1;
  }
  const double *X = xp - 1, *Y = yp - 1;
  double d1 = x - X[ig], d2 = X[ig + 1] - x;
  double t1 = sdd[ig + 1] / 6.0 / h[ig] * (d1 * d1 * d1);
  double t2 = sdd[ig] / 6.0 / h[ig] * (d2 * d2 * d2);
  double t3 = (Y[ig + 1] / h[ig] - sdd[ig + 1] / 6.0 * h[ig]) * d1;
  double t4 = (Y[ig] / h[ig] - h[ig] / 6.0 * sdd[ig]) * d2;
  return t1 + t2 + t3 + t4;
}

// compute_yL (spherical_func.f90:158-206), real harmonics S,PX,PZ,PY,D...
__device__ double ylm_dev(int L, double hg, const double *g) {
  const double fp = 16.0 * atan(1.0);
  if (fabs(hg) >= 1e-6) {
    switch (L) {
      case 1: return sqrt(1.0 / fp);
      case 2: return sqrt(3.0 / fp) * g[0] / sqrt(hg);
      case 3: return sqrt(3.0 / fp) * g[2] / sqrt(hg);
      case 4: return sqrt(3.0 / fp) * g[1] / sqrt(hg);
      case 5: return sqrt(15.0 / fp) * g[0] * g[1] / hg;
      case 6: return sqrt(15.0 / fp) * g[0] * g[2] / hg;
      case 7: return sqrt(5.0 / fp / 4.0) * (3.0 * (g[2] * g[2]) / hg - 1.0);
      case 8: return sqrt(15.0 / fp) * g[1] * g[2] / hg;
      case 9: return sqrt(15.0 / fp / 4.0) * (g[0] * g[0] - g[1] * g[1]) / hg;
      default: return 0.0;
    }
  }
  return L == 1 ? sqrt(1.0 / fp) : 0.0;
}

// vps (form_factor*, exp_igr.f90:190-206,273-285) and rhos per species and G
__global__ void k_vps_rhos(int ngrho, const double *hg, const double *xp, const double *voo, const double *h,
                           const double *sdd, int n, double zv, double omega, double tpiba2, double *vps, double *rhos) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngrho) return;
  double x = hg[g];
  vps[g] = (1.0 / omega) * spline_at(xp, voo, h, sdd, n, x);
  if (g == 0) rhos[g] = -zv * (1.0 / omega);
  else rhos[g] = -zv * exp(-(0.25 * (1.2 * 1.2) * x * tpiba2)) * (1.0 / omega);
}

// twnl (nlpro, pseudopotential.f90:108-162 / upf_nlpro :293-354)
__global__ void k_twnl(int ngpw, const double *hg, const double *gvec, const double *xp, const double *wns,
                       const double *h, const double *sdd, int n, int lp, double vol, double *tw) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngpw) return;
  double x = hg[g];
  tw[g] = ylm_dev(lp, x, gvec + 3L * g) * vol * spline_at(xp, wns, h, sdd, n, x);
}

// ---------------------------------------------------------------- geometry
// exp_igrxfactor (exp_igr.f90:4-140): S_I(G) = exp(-i G.R_I).  The phase is
// evaluated directly as sum_d n_d * arg_d (arg_d = tpiba b_d.R_I) instead of
// the reference's recursive products of 1D phases.
struct AtomArgs {
  const double *arg;   // [nat*3]
  const int *is;       // [nat]
};
__device__ __forceinline__ double2 eig_at(const int *inyh, int g, int nh1, int nh2, int nh3, const double *arg3) {
  double ph = (double)(inyh[3 * g] - nh1) * arg3[0] + (double)(inyh[3 * g + 1] - nh2) * arg3[1] +
              (double)(inyh[3 * g + 2] - nh3) * arg3[2];
  double s, c;
  sincos(ph, &s, &c);
  return make_double2(c, -s);
}
// eigrxvps(G) = sum_I S_I vps, eigrxrhos(G) = sum_I S_I rhos  (exp_igr.f90:130-136)
__global__ void k_sfac_sums(int ngrho, int nat, const int *inyh, int nh1, int nh2, int nh3, AtomArgs aa,
                            const double *vps, const double *rhos, double2 *evps, double2 *erhos) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngrho) return;
  double2 v = make_double2(0, 0), r = make_double2(0, 0);
  for (int a = 0; a < nat; ++a) {
    double2 e = eig_at(inyh, g, nh1, nh2, nh3, aa.arg + 3 * a);
    int is = aa.is[a];
    double pv = vps[(long)is * ngrho + g], pr = rhos[(long)is * ngrho + g];
    v.x += e.x * pv; v.y += e.y * pv;
    r.x += pr * e.x; r.y += pr * e.y;
  }
  evps[g] = v;
  erhos[g] = r;
}
// Projector matrix P_j(G) = (-i)^l twnl(G) S_I(G), G=0 entry halved
// (the scr arrays of fnl, pseudopotential.f90:179-209).
struct ProjArgs {
  const int *isa, *is, *iv, *l;   // [nproj]
  int nghmax;
};
__global__ void k_projectors(int ngpw, int nproj, const int *inyh, int nh1, int nh2, int nh3, AtomArgs aa, ProjArgs pa,
                             const double *twnl, double2 *P) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y;
  if (g >= ngpw || j >= nproj) return;
  int isa = pa.isa[j];
  double2 e = eig_at(inyh, g, nh1, nh2, nh3, aa.arg + 3 * isa);
  double t = twnl[((long)pa.is[j] * pa.nghmax + pa.iv[j]) * ngpw + g];
  if (g == 0) t *= 0.5;
  double2 v;
  switch (pa.l[j] & 3) {
    case 0: v = make_double2(t * e.x, t * e.y); break;
    case 1: v = make_double2(t * e.y, -t * e.x); break;   // -i
    case 2: v = make_double2(-t * e.x, -t * e.y); break;
    default: v = make_double2(-t * e.y, t * e.x); break;  // +i
  }
  P[(long)j * ngpw + g] = v;
}
// hess (cg.f90:3-61): K(G) = 1/max(1/2 |G|^2 + V_loc(0) + sum n_s w twnl^2, 0.5)
__global__ void k_hess(int ngpw, const double *hg, double tpiba2, const double2 *evps, const double *twnl, int nsp,
                       int nghmax, const int *na, const int *ngh, const double *wsg, double *vpp) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngpw) return;
  double v = evps[0].x;
  for (int is = 0; is < nsp; ++is)
    for (int iv = 0; iv < ngh[is]; ++iv) {
      double t = twnl[((long)is * nghmax + iv) * ngpw + g];
      v = v + na[is] * wsg[is * 120 + iv] * t * t;
    }
  v = 0.5 * tpiba2 * hg[g] + v;
  if (v < 0.5) v = 0.5;
  vpp[g] = 1.0 / v;
}

// ---------------------------------------------------------------- G-space
// ray buffer (forward X done) -> F(+G)/N   (rhor2g, density.f90:143-145)
template <typename C>
__global__ void k_gather_p(int ng, const int *pos_p, const C *rb, double scale, double2 *out) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ng) return;
  C v = rb[pos_p[g]];
  out[g] = make_double2((double)v.x * scale, (double)v.y * scale);
}

// eval_pot (potential.f90:4-46) in G space + e_hartree / pp_energy E_loc
// partial sums: part[0*nb+b] = Re sum 4pi/G^2 |rho+rho_ion|^2,
// part[1*nb+b] = Re sum eigrxvps conj(rho) (G=0 weighted 1/2).
__global__ void k_vloc_g(int ngrho, const double *hg, double tpiba2, const double2 *rhog, const double2 *erhos,
                         const double2 *evps, double2 *vg, double *part, double *out, unsigned *ticket) {
  const double fp = 16.0 * atan(1.0);
  double eh = 0, el = 0;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ngrho; g += gridDim.x * blockDim.x) {
    double2 rg = rhog[g], e = evps[g];
    if (g == 0) {
      vg[0] = make_double2(0.0, 0.0);
      el += 0.5 * (e.x * rg.x + e.y * rg.y);
    } else {
      double f = fp / (tpiba2 * hg[g]);
      double2 r = make_double2(rg.x + erhos[g].x, rg.y + erhos[g].y);
      vg[g] = make_double2(f * r.x + e.x, f * r.y + e.y);
      eh += f * (r.x * r.x + r.y * r.y);
      el += e.x * rg.x + e.y * rg.y;
    }
  }
  const double v[2] = {eh, el};
  reduce_and_finish<2>(v, part, out, ticket);  // out[0] = E_H sum, out[1] = E_loc sum
}

// GRAD_CAL fields (xc.f90:471-487): t=0: rho + i d_x rho, t=1: d_y rho + i d_z rho
__global__ void k_grad_fields(int ngrho, const double *gvec, double tpiba, const double2 *rhog, double2 *fp, double2 *fm) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngrho) return;
  double2 r = rhog[g];
  double gx = tpiba * gvec[3 * g], gy = gvec[3 * g + 1], gz = gvec[3 * g + 2];
  fp[g] = make_double2(r.x - gx * r.x, r.y - gx * r.y);
  fm[g] = make_double2(r.x + gx * r.x, -(r.y + gx * r.y));
  // tpiba (i gy - gz) r  and tpiba (-i gy + gz) conj(r)
  double ax = -tpiba * gz, ay = tpiba * gy;
  fp[ngrho + g] = make_double2(ax * r.x - ay * r.y, ax * r.y + ay * r.x);
  double bx = tpiba * gz, by = -tpiba * gy;
  fm[ngrho + g] = make_double2(bx * r.x + by * r.y, by * r.x - bx * r.y);
}
__global__ void k_conj_field(int ng, const double2 *fp, double2 *fm) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ng) return;
  fm[g] = make_double2(fp[g].x, -fp[g].y);
}

// ---------------------------------------------------------------- XC
// The functionals in the arithmetic type R: double on the FP64 path, float on
// the mixed path (whose last iterations run this in FP64 again).
template <typename R> __device__ void xc_teter93(R rho, R &e, R &v) {
  const R a0 = (R)0.4581652932831429, a1 = (R)2.217058676663745, a2 = (R)0.7405551735357053,
          a3 = (R)0.01968227878617998;
  const R b1 = (R)1.0, b2 = (R)4.504130959426697, b3 = (R)1.110667363742916, b4 = (R)0.02359291751427506;
  const R fp = (R)12.566370614359172954;  // 4 pi
  R rs = cbrt((R)3 / (fp * rho));
  R num = a0 + rs * (a1 + rs * (a2 + rs * a3));
  R den = rs * (b1 + rs * (b2 + rs * (b3 + rs * b4)));
  R dnum = a1 + rs * ((R)2 * a2 + rs * (R)3 * a3);
  R dden = b1 + rs * ((R)2 * b2 + rs * ((R)3 * b3 + rs * (R)4 * b4));
  R eps = -num / den;
  R deps = -(dnum * den - num * dden) / (den * den);
  e = rho * eps;
  v = eps - rs / (R)3 * deps;
}
template <typename R> __device__ void xc_pz(R rho, R &e, R &v) {
  const R pi = (R)3.14159265358979323846, fp = (R)12.566370614359172954;
  R ex = (R)-0.75 * cbrt((R)3 / pi) * cbrt(rho);
  R rs = cbrt((R)3 / (fp * rho)), eps, deps;
  if (rs >= (R)1) {
    const R gg = (R)-0.1423, b1 = (R)1.0529, b2 = (R)0.3334;
    R sq = sqrt(rs), den = (R)1 + b1 * sq + b2 * rs;
    eps = gg / den;
    deps = -gg * ((R)0.5 * b1 / sq + b2) / (den * den);
  } else {
    const R A = (R)0.0311, B = (R)-0.048, Cc = (R)0.0020, D = (R)-0.0116;
    R lr = log(rs);
    eps = A * lr + B + Cc * rs * lr + D * rs;
    deps = A / rs + Cc * lr + Cc + D;
  }
  e = rho * ex + rho * eps;
  v = (R)4 / (R)3 * ex + (eps - rs / (R)3 * deps);
}
template <typename R> __device__ void xc_pbe(R rho, R sigma, R &e, R &v, R &vs) {
  // PBE exchange and correlation (PW92 correlation, unpolarised); the
  // reciprocals of rho and k_F are formed once and r_s = (9 pi/4)^(1/3) / k_F
  const R pi = (R)3.14159265358979323846, fp = (R)12.566370614359172954;
  const R kappa = (R)0.804, mu = (R)0.2195149727645171, beta = (R)0.06672455060314922;
  const R gamma = ((R)1 - log((R)2)) / (pi * pi);
  const R ir = (R)1 / rho;
  R kf = cbrt((R)3 * pi * pi * rho);
  const R ikf = (R)1 / kf;
  R exu = (R)-3 / fp * kf * rho;
  const R q4 = (R)0.25 * ikf * ikf * ir * ir;  // 1 / (4 kf^2 rho^2)
  R s2 = sigma * q4;
  const R iden = (R)1 / ((R)1 + mu * s2 / kappa);
  R Fx = (R)1 + kappa - kappa * iden, dF = mu * iden * iden;
  R ex = exu * Fx;
  R vx = (R)4 / (R)3 * exu * ir * Fx + exu * dF * ((R)-8 / (R)3 * s2 * ir);
  R vsx = exu * dF * q4;
  R rs = (R)1.9191582926775128 * ikf;  // (9 pi / 4)^(1/3) / k_F
  const R A = (R)0.0310907, a1 = (R)0.21370, b1 = (R)7.5957, b2 = (R)3.5876, b3 = (R)1.6382, b4 = (R)0.49294;
  R sq = sqrt(rs);
  R q = (R)2 * A * (b1 * sq + b2 * rs + b3 * rs * sq + b4 * rs * rs);
  R dq = (R)2 * A * ((R)0.5 * b1 / sq + b2 + (R)1.5 * b3 * sq + (R)2 * b4 * rs);
  R L = log((R)1 + (R)1 / q), dL = -dq / (q * q + q);
  R ec = (R)-2 * A * ((R)1 + a1 * rs) * L;
  R dec = (R)-2 * A * a1 * L - (R)2 * A * ((R)1 + a1 * rs) * dL;
  R t2 = pi * sigma * (R)0.25 * q4 * kf;  // pi sigma / (16 kf rho^2)
  R bg = beta / gamma, E = exp(-ec / gamma), iE1 = (R)1 / (E - (R)1), AA = bg * iE1;
  R At2 = AA * t2, num = (R)1 + At2, idd = (R)1 / ((R)1 + At2 + At2 * At2);
  R Q = t2 * num * idd;
  const R ibq = (R)1 / ((R)1 + bg * Q);
  R H = gamma * log((R)1 + bg * Q);
  R dHdQ = beta * ibq;
  R dQdt2 = (num + t2 * AA) * idd - t2 * num * (AA + (R)2 * AA * AA * t2) * idd * idd;
  R dQdA = (t2 * t2) * idd - t2 * num * (t2 + (R)2 * AA * t2 * t2) * idd * idd;
  R dAdec = bg * E * iE1 * iE1 / gamma;
  R decdrho = dec * (-rs * ir / (R)3);
  R dt2drho = (R)-7 / (R)3 * t2 * ir;
  R vc = ec + H + rho * (decdrho + dHdQ * dQdA * dAdec * decdrho + dHdQ * dQdt2 * dt2drho);
  R vsc = rho * dHdQ * dQdt2 * pi * (R)0.25 * q4 * kf;
  e = ex + rho * (ec + H);
  v = vx + vc;
  vs = vsx + vsc;
}

// cal_vpot_ex pointwise part (xc.f90:66-131): smoothing below 4e-8, etxc
// sums, and the two complex fields for the G-space assembly:
// g0 <- v1 + i v2 d_x rho, g1 <- v2 d_y rho + i v2 d_z rho  (xc.f90:262-279).
// The functional runs in R; the E_xc sums and the fields are FP64.
template <typename R>
__global__ void k_xc(long npt, int xc, const double *rho, double2 *g0, double2 *g1, double *part, double *out,
                     unsigned *ticket) {
  const double gc = 1.0e-8;
  double sm = 0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < npt; i += (long)gridDim.x * blockDim.x) {
    double r = rho[i];
    double sigma = 0, dx = 0, dy = 0, dz = 0;
    if (xc == 2) {
      double2 a = g0[i], b = g1[i];
      dx = a.y; dy = b.x; dz = b.y;
      sigma = dx * dx + (dy * dy + dz * dz);
    }
    R e = 0, v = 0, vs = 0;
    if (r > 1e-30) {
      if (xc == 0) xc_teter93<R>((R)r, e, v);
      else if (xc == 1) xc_pz<R>((R)r, e, v);
      else xc_pbe<R>((R)r, (R)sigma, e, v, vs);
    }
    double rt = r > 0.0 ? r : 0.0, v1 = 0, v2 = 0;
    if (rt > 0.1 * gc) {
      double smoo, dsmoo;
      if (rt > 4.0 * gc) { smoo = 1.0; dsmoo = 0.0; }
      else {
        double texp = exp(3.0 * (1.0 - rt / gc));
        smoo = 1.0 / (1.0 + texp);
        dsmoo = 3.0 / gc * texp * smoo * smoo;
      }
      sm += smoo * (double)e;
      v1 = dsmoo * (double)e + smoo * (double)v;
      v2 = smoo * (2.0 * (double)vs);
    }
    g0[i] = make_double2(v1, v2 * dx);
    if (xc == 2) g1[i] = make_double2(v2 * dy, v2 * dz);
  }
  const double vv[1] = {sm};
  reduce_and_finish<1>(vv, part, out, ticket);
}

// Teter93 spin polarized (libxc XC_LDA_XC_TETER93 with two spin densities;
// Goedecker, Teter and Hutter, Phys. Rev. B 54, 1703 (1996)): every Pade
// coefficient c = c(unpolarized) + f(zeta) dc with
// f(zeta) = ((1+zeta)^(4/3) + (1-zeta)^(4/3) - 2) / (2^(4/3) - 2);
// e = rho eps, va / vb = d(rho eps) / d rho_a / rho_b.
template <typename R> __device__ void xc_teter93_pol(R ra, R rb, R &e, R &va, R &vb) {
  const R a0 = (R)0.4581652932831429, a1 = (R)2.217058676663745, a2 = (R)0.7405551735357053,
          a3 = (R)0.01968227878617998;
  const R b1 = (R)1.0, b2 = (R)4.504130959426697, b3 = (R)1.110667363742916, b4 = (R)0.02359291751427506;
  const R da0 = (R)0.119086804055547, da1 = (R)0.6157402568883345, da2 = (R)0.1574201515892867,
          da3 = (R)0.003532336663397157;
  const R db1 = (R)0.0, db2 = (R)0.2673612973836267, db3 = (R)0.2052004607777787, db4 = (R)0.004200005045691381;
  const R fp = (R)12.566370614359172954;  // 4 pi
  const R rho = ra + rb;
  R z = (ra - rb) / rho;
  z = z > (R)1 ? (R)1 : (z < (R)-1 ? (R)-1 : z);
  const R fden = cbrt((R)16) - (R)2;  // 2^(4/3) - 2
  const R cp = cbrt((R)1 + z), cm = cbrt((R)1 - z);
  const R f = (((R)1 + z) * cp + ((R)1 - z) * cm - (R)2) / fden;
  const R dfz = (R)4 / (R)3 * (cp - cm) / fden;
  const R A0 = a0 + f * da0, A1 = a1 + f * da1, A2 = a2 + f * da2, A3 = a3 + f * da3;
  const R B1 = b1 + f * db1, B2 = b2 + f * db2, B3 = b3 + f * db3, B4 = b4 + f * db4;
  const R rs = cbrt((R)3 / (fp * rho));
  const R num = A0 + rs * (A1 + rs * (A2 + rs * A3));
  const R den = rs * (B1 + rs * (B2 + rs * (B3 + rs * B4)));
  const R dnum = A1 + rs * ((R)2 * A2 + rs * (R)3 * A3);
  const R dden = B1 + rs * ((R)2 * B2 + rs * ((R)3 * B3 + rs * (R)4 * B4));
  const R nf = da0 + rs * (da1 + rs * (da2 + rs * da3));
  const R dfden = rs * (db1 + rs * (db2 + rs * (db3 + rs * db4)));
  const R eps = -num / den;
  const R deps_drs = -(dnum * den - num * dden) / (den * den);
  const R deps_dz = -(nf * den - num * dfden) / (den * den) * dfz;
  e = rho * eps;
  va = eps - rs / (R)3 * deps_drs + deps_dz * ((R)1 - z);
  vb = eps - rs / (R)3 * deps_drs - deps_dz * ((R)1 + z);
}

// Open-shell XC (xc.f90:135-246, LDA): rho_a = rho - rho2, rho_b = rho2 (the
// reference subtracts the spin-2 density from the total, :46-50), the
// polarized functional with the smoothing of the total (:196-236);
// g0 = (v1a, 0), g1 = (v1b, 0); E_xc partial sums finished into out.
template <typename R>
__global__ void k_xc_lsd(long npt, const double *rho, const double *rho2, double2 *g0, double2 *g1, double *part,
                         double *out, unsigned *ticket) {
  const double gc = 1.0e-8;
  double sm = 0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < npt; i += (long)gridDim.x * blockDim.x) {
    const double ra = rho[i] - rho2[i], rb = rho2[i];
    const double pa = ra > 0.0 ? ra : 0.0, pb = rb > 0.0 ? rb : 0.0;
    R e = 0, va = 0, vb = 0;
    if (pa + pb > 1e-30) xc_teter93_pol<R>((R)pa, (R)pb, e, va, vb);
    const double rt = pa + pb;
    double v1a = 0, v1b = 0;
    if (rt > 0.1 * gc) {
      double smoo, dsmoo;
      if (rt > 4.0 * gc) { smoo = 1.0; dsmoo = 0.0; }
      else {
        double texp = exp(3.0 * (1.0 - rt / gc));
        smoo = 1.0 / (1.0 + texp);
        dsmoo = 3.0 / gc * texp * smoo * smoo;
      }
      sm += smoo * (double)e;
      v1a = dsmoo * (double)e + smoo * (double)va;
      v1b = dsmoo * (double)e + smoo * (double)vb;
    }
    g0[i] = make_double2(v1a, 0.0);
    g1[i] = make_double2(v1b, 0.0);
  }
  const double vv[1] = {sm};
  reduce_and_finish<1>(vv, part, out, ticket);
}

// Open shell: band-space matrices are block diagonal by spin (OVLAP_D and
// ortho_gs take the spin-1 and spin-2 blocks separately,
// wfn_initialize.f90:245-253,458-477): entries coupling the two spins are zeroed
__global__ void k_spin_mask(int n, int nel_up, double *A) {
  const long tot = (long)n * n;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < tot; e += (long)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), j = (int)(e / n);
    if ((i < nel_up) != (j < nel_up)) A[e] = 0.0;
  }
}

// G-space assembly of the XC potential (xc.f90:257-297): from the forward
// transforms of g0 (and g1 for GGA) in the ray buffer (t stride) build
// vpotg = V_H+V_loc + v1(G) - i G.(v2 grad rho)(G)
template <typename C>
__global__ void k_xc_combine(int ngrho, int gga, const int *pos_p, const int *pos_m, const C *rb, long rstride, double scale,
                             const double *gvec, double tpiba, const double2 *vg, double2 *vout) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngrho) return;
  double2 acc = vg[g];
  for (int t = 0; t < (gga ? 2 : 1); ++t) {
    C p = rb[t * rstride + pos_p[g]], m = rb[t * rstride + pos_m[g]];
    double fax = ((double)p.x + (double)m.x) * scale, fay = ((double)p.y + (double)m.y) * scale;
    double fbx = ((double)p.x - (double)m.x) * scale, fby = ((double)p.y - (double)m.y) * scale;
    double2 vg1 = make_double2(0.5 * fax, 0.5 * fby), vg2 = make_double2(0.5 * fay, -0.5 * fbx);
    if (t == 0) {
      double vf = tpiba * gvec[3 * g];
      acc.x = acc.x + vg1.x + vf * vg2.y;
      acc.y = acc.y + vg1.y - vf * vg2.x;
    } else {
      double v2 = tpiba * gvec[3 * g + 1], v3 = tpiba * gvec[3 * g + 2];
      acc.x = acc.x + v2 * vg1.y + v3 * vg2.y;
      acc.y = acc.y - v2 * vg1.x - v3 * vg2.x;
    }
  }
  vout[g] = acc;
}

// ---------------------------------------------------------------- vpsi unpack
// vpsi unpack (wfn_initialize.f90:342-361) fused with fnonloc / upf_fnonloc
// (wfn_initialize.f90:560-695) for the projectors j < npj:
//   C2_a = -f_a/2 (tpiba2 hg c_a + (Re FP, Im FM)) + sum_j P_j(G) D(j, a)
//   C2_b = -f_b/2 (tpiba2 hg c_b + (Im FP, -Re FM)) + sum_j P_j(G) D(j, b)
// with FP = F(G)+F(-G), FM = F(G)-F(-G) of the pair's forward transform in the
// ray buffer.  grid (ngpw/128, ceil(T/PAIRS)): a thread takes one G and the
// PAIRS pairs of its block's chunk (8 on FP32 data, 4 in FP64, whose sums
// take twice the registers); it first sums the projector
// terms of the chunk's bands (P_j(G) read once per chunk, coalesced over G and
// L2-resident; the chunk's rows of D in shared memory), then unpacks, so C2
// is written once.  P holds P_j(0)/2 at G = 0 (the convention of fnl's real
// dot products); the full value is used here.  The projector sums run in the
// transform's precision (FP32 with packed FMAs on the mixed path).  With bmax
// (the int8 slice products of the mixed path) the kernel also records each
// band's max |Re|, |Im| of C2 (atomic max of the FP64 bits, non-negative
// values), which the slicing of C2 needs, so C2 is not read once more for it.
// gzero: index of G = 0 among the ngpw G vectors (0; -1 for a rank of the
// slab decomposition that does not own it).
constexpr int UNPACK_NPJ = 32;
template <typename C> __host__ __device__ constexpr int unpack_pairs() { return sizeof(C) == sizeof(float2) ? 8 : 4; }
template <typename C>
__global__ void __launch_bounds__(128) k_unpack_fnonloc(int ngpw, int nstate, int band0, int T, int npj,
                                                        const int *__restrict__ pos_p, const int *__restrict__ pos_m,
                                                        const C *__restrict__ rb, long rstride, double scale,
                                                        const double *__restrict__ hg, double tpiba2,
                                                        const double *__restrict__ occ, const double2 *__restrict__ P,
                                                        const double *__restrict__ D, int nproj,
                                                        const double2 *__restrict__ c0, double2 *__restrict__ c2,
                                                        unsigned long long *__restrict__ bmax, int gzero) {
  typedef decltype(C().x) Rl;
  constexpr int PAIRS = unpack_pairs<C>(), NB = 2 * PAIRS;
  __shared__ double red[4][NB];  // per-warp band maxima (128 threads)
  extern __shared__ unsigned char smraw[];
  Rl *Ds = reinterpret_cast<Rl *>(smraw);  // [j][band - b0]
  const int t0 = blockIdx.y * PAIRS, t1 = min(T, t0 + PAIRS);
  const int b0 = band0 + 2 * t0;
  const int nb = min(2 * (t1 - t0), nstate - b0);
  for (int i = threadIdx.x; i < NB * npj; i += blockDim.x) {
    const int j = i / NB, b = i - j * NB;
    Ds[i] = b < nb ? (Rl)D[j + (long)nproj * (b0 + b)] : (Rl)0;
  }
  __syncthreads();
  const int g0 = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = g0 < ngpw;
  const int g = valid ? g0 : 0;  // lanes past the sphere follow along for the reductions
  C acc[NB];
#pragma unroll
  for (int b = 0; b < NB; ++b) acc[b] = czero<C>();
  const double gw = (g == gzero) ? 2.0 : 1.0;
#pragma unroll 4
  for (int j = 0; j < npj; ++j) {
    const double2 v = P[(long)j * ngpw + g];
    const C pj = mk((Rl)(gw * v.x), (Rl)(gw * v.y));
    const Rl *dj = Ds + j * NB;
#pragma unroll
    for (int b = 0; b < NB; ++b) acc[b] = cfmas(pj, dj[b], acc[b]);
  }
  const int pp = pos_p[g], pm = pos_m[g];
  const double kin = tpiba2 * hg[g];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int tt = 0; tt < PAIRS; ++tt) {
    const int t = t0 + tt;
    if (t >= t1) break;
    const C *R = rb + (long)t * rstride;
    const C vp = R[pp], vm = R[pm];
    const double fpx = ((double)vp.x + (double)vm.x) * scale, fpy = ((double)vp.y + (double)vm.y) * scale;
    const double fmx = ((double)vp.x - (double)vm.x) * scale, fmy = ((double)vp.y - (double)vm.y) * scale;
    const int ba = band0 + 2 * t, bb = ba + 1;
    double fi = occ[ba] * 0.5;
    if (fi == 0.0) fi = 1.0;
    const double2 ca = c0[(long)ba * ngpw + g];
    const C na = acc[2 * tt];
    const double2 xa = make_double2(-fi * (kin * ca.x + fpx) + (double)na.x, -fi * (kin * ca.y + fmy) + (double)na.y);
    if (valid) c2[(long)ba * ngpw + g] = xa;
    double ma = valid ? fmax(fabs(xa.x), fabs(xa.y)) : 0.0, mb = 0.0;
    if (bb < nstate) {
      const C nbv = acc[2 * tt + 1];
      double fb = occ[bb] * 0.5;
      if (fb == 0.0) fb = 1.0;
      const double2 cb = c0[(long)bb * ngpw + g];
      const double2 xb =
          make_double2(-fb * (kin * cb.x + fpy) + (double)nbv.x, -fb * (kin * cb.y - fmx) + (double)nbv.y);
      if (valid) c2[(long)bb * ngpw + g] = xb;
      mb = valid ? fmax(fabs(xb.x), fabs(xb.y)) : 0.0;
    }
    if (bmax) {
      for (int o = 16; o > 0; o >>= 1) {
        ma = fmax(ma, __shfl_xor_sync(0xffffffffu, ma, o));
        mb = fmax(mb, __shfl_xor_sync(0xffffffffu, mb, o));
      }
      if (lane == 0) {
        red[warp][2 * tt] = ma;
        red[warp][2 * tt + 1] = mb;
      }
    }
  }
  if (bmax) {
    __syncthreads();
    if (threadIdx.x < nb) {
      double m = 0.0;
#pragma unroll
      for (int w = 0; w < 4; ++w) m = fmax(m, red[w][threadIdx.x]);
      atomicMax(bmax + b0 - band0 + threadIdx.x, (unsigned long long)__double_as_longlong(m));
    }
  }
}
// fnonloc for projectors j0 .. j0+npj-1 beyond the first UNPACK_NPJ, FP64:
// C2(b, G) += sum_j P_j(G) D(j, b) for bands band0 .. band0+nball-1; grid
// (ngpw/128, ceil(nball/FNL_BANDS)), FNL_BANDS bands per block
constexpr int FNL_BANDS = 16;
template <int NPJ>
__global__ void __launch_bounds__(128) k_fnonloc_add(int ngpw, int band0, int nball, int j0, int npj,
                                                     const double2 *__restrict__ P, const double *__restrict__ D,
                                                     int nproj, double2 *__restrict__ c2) {
  extern __shared__ double Dsd[];  // [b][j]
  band0 += blockIdx.y * FNL_BANDS;
  const int nb = min(FNL_BANDS, nball - (int)blockIdx.y * FNL_BANDS);
  for (int i = threadIdx.x; i < nb * npj; i += blockDim.x) {
    const int b = i / npj, j = i - b * npj;
    Dsd[i] = D[j0 + j + (long)nproj * (band0 + b)];
  }
  __syncthreads();
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngpw) return;
  double2 pj[NPJ];
#pragma unroll
  for (int j = 0; j < NPJ; ++j) {
    pj[j] = make_double2(0.0, 0.0);
    if (j < npj) {
      double2 v = P[(long)(j0 + j) * ngpw + g];
      if (g == 0) v = make_double2(2.0 * v.x, 2.0 * v.y);
      pj[j] = v;
    }
  }
  for (int b = 0; b < nb; ++b) {
    const double *d = Dsd + b * npj;
    double2 a = make_double2(0.0, 0.0);
#pragma unroll
    for (int j = 0; j < NPJ; ++j)
      if (j < npj) a = cfmas(pj[j], d[j], a);
    double2 &o = c2[(long)(band0 + b) * ngpw + g];
    o = make_double2(o.x + a.x, o.y + a.y);
  }
}

// ---------------------------------------------------------------- bands
// E_kin partial sums (total_energy.f90:38-61)
// Band-major [nstate][ngpw] arrays in fixed contiguous chunks per block
// (deterministic partials): thread t walks k = k0 + t, k0 + t + blockDim...,
// tracking (band, g) incrementally (blockDim < ngpw), four loads in flight.
struct BandWalk {
  long k, k1;
  int b, g;
  __device__ BandWalk(long tot, int ngpw) {
    const long per = (tot + gridDim.x - 1) / gridDim.x;
    const long chunk = (per + blockDim.x - 1) / blockDim.x * blockDim.x;
    const long k0 = blockIdx.x * chunk;
    k1 = min(tot, k0 + chunk);
    k = k0 + threadIdx.x;
    b = (int)(k / ngpw);
    g = (int)(k % ngpw);
  }
  __device__ __forceinline__ void next(int ngpw) {
    k += blockDim.x;
    g += blockDim.x;
    if (g >= ngpw) {
      g -= ngpw;
      ++b;
    }
  }
};

// A block's contiguous chunk of the (band, G) index space (as BandWalk), read
// STREAM_U elements per thread per round with every load of the round (the
// coefficients and the per-G and per-band factors) issued first, so that
// enough of them are in flight to stream at the copy rate; the (band, G)
// position advances by additions, not a division per element.  The kernels
// are launched with one wave of blocks (the resident count, not RED_BLOCKS).
constexpr int STREAM_U = 4;
__device__ __forceinline__ void stream_chunk(long tot, long &k0, long &k1) {
  const long per = (tot + gridDim.x - 1) / gridDim.x;
  const long chunk = (per + blockDim.x - 1) / blockDim.x * blockDim.x;
  k0 = blockIdx.x * chunk;
  k1 = min(tot, k0 + chunk);
}
// (band, G) of element k + d from that of k (band-major, ngpw per band)
__device__ __forceinline__ void band_step(int &b, int &g, int d, int ngpw) {
  g += d;
  while (g >= ngpw) {
    g -= ngpw;
    ++b;
  }
}
__global__ void k_ekin(int ngpw, int nstate, const double2 *c0, const double *hg, const double *occ, double *part,
                       double *out, unsigned *ticket) {
  double s = 0;
  long k0, k1;
  stream_chunk((long)ngpw * nstate, k0, k1);
  long k = k0 + threadIdx.x;
  int b = (int)(k / ngpw), g = (int)(k - (long)b * ngpw);
  const int step = blockDim.x;
  while (k < k1) {
    double2 c[STREAM_U];
    double h[STREAM_U], o[STREAM_U];
#pragma unroll
    for (int u = 0; u < STREAM_U; ++u) {
      const bool v = k < k1;
      c[u] = v ? c0[k] : make_double2(0.0, 0.0);
      h[u] = v ? hg[g] : 0.0;
      o[u] = v ? occ[b] : 0.0;
      k += step;
      band_step(b, g, step, ngpw);
    }
#pragma unroll
    for (int u = 0; u < STREAM_U; ++u) s += o[u] * h[u] * (c[u].x * c[u].x + c[u].y * c[u].y);
  }
  const double v[1] = {s};
  reduce_and_finish<1>(v, part, out, ticket);
}
// c = 2 a - c (wavefunction predictor)
// c = w a + c (the current step's term of the wavefunction predictor)
__global__ void k_axpy_c(long n, double w, const double2 *__restrict__ a, double2 *__restrict__ c) {
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
    const double2 x = a[k], y = c[k];
    c[k] = make_double2(fma(w, x.x, y.x), fma(w, x.y, y.y));
  }
}

// Weights of Kolafa's always-stable predictor (J. Comput. Chem. 25, 335
// (2004)) with npoints = K + 2 points, most recent first:
// B_j = (-1)^(j+1) j binom(2K+4, K+2-j) / binom(2K+2, K+1), j = 1..K+2.
// npoints = 2 gives (2, -1), linear extrapolation; npoints = 1 gives (1).
inline void aspc_coefficients(int npoints, double *w) {
  if (npoints <= 1) {
    w[0] = 1.0;
    return;
  }
  auto binom = [](int n, int k) {
    double r = 1.0;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
  };
  const int K = npoints - 2;
  const double den = binom(2 * K + 2, K + 1);
  for (int j = 1; j <= npoints; ++j) w[j - 1] = ((j & 1) ? 1.0 : -1.0) * j * binom(2 * K + 4, K + 2 - j) / den;
}
// rank-1 G=0 correction and occupation mask of OVLAP_D / ortho_gs DGER
// (wfn_initialize.f90:257,482): A(i,j) -= Re a_i(0) Re b_j(0); mask fsc
__global__ void k_g0_correct(int n, int ngpw, const double2 *a, const double2 *b, double *A, const double *occ, int mask,
                             int upper_only) {
  int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i >= n || j >= n) return;
  if (upper_only && i > j) return;
  double v = A[i + (long)n * j] - a[(long)i * ngpw].x * b[(long)j * ngpw].x;
  if (mask) v *= (occ[i] == 0.0 ? 0.0 : 1.0) * (occ[j] == 0.0 ? 0.0 : 1.0);
  A[i + (long)n * j] = v;
}
// ZCLEAN (wfn_initialize.f90:531-558)
__global__ void k_zclean(int n, int ngpw, double2 *c) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) c[(long)i * ngpw].y = 0.0;
}
// eval_GMAX (gradient.f90:36-61) and the preconditioned-gradient norm of
// PRECON + GGNORM (cg.f90:102-107, 281-311) in one pass over the occupied
// bands of C2: out[0] = GEMAX = max |C2|, out[1] = sum_i DOTP(cp_i, cp_i)
// with cp = f_i^-1 K(G) C2 (f_i^-1 = 1 for f_i <= 0.01); cp itself is not
// stored, the PCG update forms it again from C2.
__global__ void k_gmax_precon(int ngpw, int nocc, const double *vpp, const double *occ, const double2 *c2,
                              double *part, double *out, unsigned *ticket) {
  double m = 0.0, s = 0.0;
  long k0, k1;
  stream_chunk((long)ngpw * nocc, k0, k1);
  long k = k0 + threadIdx.x;
  int b = (int)(k / ngpw), g = (int)(k - (long)b * ngpw);
  const int step = blockDim.x;
  while (k < k1) {
    double2 c[STREAM_U];
    double kv[STREAM_U], o[STREAM_U];
    bool g0[STREAM_U];
#pragma unroll
    for (int u = 0; u < STREAM_U; ++u) {
      const bool v = k < k1;
      c[u] = v ? c2[k] : make_double2(0.0, 0.0);
      kv[u] = v ? vpp[g] : 0.0;
      o[u] = v ? occ[b] : 1.0;
      g0[u] = g == 0;
      k += step;
      band_step(b, g, step, ngpw);
    }
#pragma unroll
    for (int u = 0; u < STREAM_U; ++u) {
      const double fi = o[u] > 0.01 ? 1.0 / o[u] : 1.0;  // 1/f_i
      m = fmax(m, c[u].x * c[u].x + c[u].y * c[u].y);
      const double f = fi * kv[u];
      const double2 v = make_double2(f * c[u].x, f * c[u].y);
      s += g0[u] ? v.x * v.x : 2.0 * (v.x * v.x + v.y * v.y);
    }
  }
  const double vals[2] = {sqrt(m), s};  // sqrt is monotonic: the max of the roots is the root of the max
  reduce_and_finish<2, 1u>(vals, part, out, ticket);
}
// PCG direction and step (cg.f90:109-143) with cp = f_i^-1 K(G) C2 (PRECON,
// cg.f90:281-311); gamma = forget * ggnorm(new) / ggnorm(previous)
__global__ void k_pcg_update(int ngpw, int nstate, const double *scal, const double *vpp, const double *occ,
                             const double2 *__restrict__ c2, double2 *__restrict__ hnm1, double2 *__restrict__ c0) {
  const int istep = (int)scal[S_ISTEP];
  const double forget = istep <= 10 ? 0.60 : (istep <= 20 ? 0.91 : 0.95);
  const double gamma = (istep == 1) ? 0.0 : forget * (scal[S_GG] / scal[S_GGPREV]);
  const double dt = 5.0 * 5.0 / 400.0;
  BandWalk w((long)ngpw * nstate, ngpw);
  int bf = -1;
  double fi = 1.0;
#pragma unroll 4
  for (; w.k < w.k1; w.next(ngpw)) {
    if (w.b != bf) {
      bf = w.b;
      fi = occ[bf] > 0.01 ? 1.0 / occ[bf] : 1.0;
    }
    const double f = fi * vpp[w.g];
    const double2 c = c2[w.k];
    double2 d = make_double2(f * c.x, f * c.y);
    if (istep > 1) {
      const double2 h = hnm1[w.k];
      d.x += gamma * h.x;
      d.y += gamma * h.y;
    }
    hnm1[w.k] = d;
    double2 x = c0[w.k];
    x.x += dt * d.x;
    x.y += dt * d.y;
    c0[w.k] = x;
  }
}
__global__ void k_copy_scalar(const double *src, double *dst) { *dst = *src; }

// Shared-memory blocked Cholesky + inverse for n <= CHOL_NMAX, one block of
// CHOL_NT threads (DPOTRF + DTRTRI of UINV, wfn_initialize.f90:504-530).
// The matrix is padded to np = 16*ceil(n/16) with the identity and held in
// shared memory with leading dimension np+1.  Per 16-column block k
// (right-looking), with U_kk and X_kk = U_kk^{-1} already in the diagonal
// block:
//   phase 2 (all warps): the panel U_k,c = X_kk^T S_k,c (c beyond block k)
//     and T = U_0:k,k X_kk (the rows above block k, stored aside);
//   phase 3: warp 0 applies this step's update to the next diagonal block
//     and factors and inverts it in registers (lookahead), while the other
//     warps update the trailing upper triangle S_c,d -= U_k,c^T U_k,d and
//     form the inverse's block column X_0:k,k = -X_0:k,0:k T.
// X overwrites U block column by block column once T has consumed it, so the
// inverse needs no separate back substitution: two barriers per block.  A
// non-positive pivot sets *info to its 1-based index; Ui gets U^{-1} (upper,
// zero below).
constexpr int CHOL_NMAX = 144;
constexpr int CHOL_NT = 512;
constexpr int CHOL_B = 16;
__device__ __forceinline__ void warp_chol_inv16(double *D, int ld, int base, int *bad) {
  const int l = threadIdx.x & 31;
  const bool own = l < CHOL_B;
  double col[CHOL_B], invd[CHOL_B];  // invd[j] = 1 / U_jj, the same in every lane
  int badj = 0;
#pragma unroll
  for (int r = 0; r < CHOL_B; ++r) col[r] = own ? D[r + ld * l] : 0.0;
#pragma unroll
  for (int j = 0; j < CHOL_B; ++j) {
    const double d = __shfl_sync(0xffffffffu, col[j], j);
    if (!(d > 0.0) && badj == 0) badj = base + j + 1;
    const double inv = rsqrt(d);
    invd[j] = inv;
    if (l == j) col[j] = d * inv;
    else if (l > j) col[j] *= inv;
    // constant bounds: the loop unrolls and col[] stays in registers (a bound
    // that depends on j left it in local memory, doubling the kernel's time)
#pragma unroll
    for (int a = 0; a < CHOL_B; ++a) {
      if (a > j) {
        const double uja = __shfl_sync(0xffffffffu, col[j], a);
        if (l >= a) col[a] -= uja * col[j];
      }
    }
  }
  if (l == 0 && badj && *bad == 0) *bad = badj;
  if (own) {
#pragma unroll
    for (int r = 0; r < CHOL_B; ++r)
      if (r <= l) D[r + ld * l] = col[r];
  }
  __syncwarp();
  double x[CHOL_B];
#pragma unroll
  for (int i = CHOL_B - 1; i >= 0; --i) {
    double t = 0.0;
#pragma unroll
    for (int k = 0; k < CHOL_B; ++k)
      if (k > i) t += D[i + ld * k] * x[k];
    const double di = invd[i];
    x[i] = (i == l) ? di : ((i < l) ? -t * di : 0.0);
  }
  __syncwarp();
  if (own) {
#pragma unroll
    for (int r = 0; r < CHOL_B; ++r)
      if (r <= l) D[r + ld * l] = x[r];
  }
}

// A (leading dimension lda) in, U^-1 into Ui (leading dimension ldu); a
// non-positive pivot j sets *info = base + j + 1 (first: the status is also
// cleared on success; otherwise an earlier failure is kept)
__global__ void __launch_bounds__(CHOL_NT) k_chol_inv_s(int n, const double *A, int lda, double *Ui, int ldu, int *info,
                                                        int base, int first) {
  extern __shared__ double M[];
  __shared__ int bad;
  const int np = (n + CHOL_B - 1) / CHOL_B * CHOL_B, ld = np + 1, nb = np / CHOL_B;
  double *Tb = M + (size_t)np * ld;  // [np][CHOL_B]: T(i, s) at Tb[i*CHOL_B + s]
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, nw = blockDim.x >> 5;
  const int hr = lane & 15, hc = 2 * w + (lane >> 4);  // half-warp: row hr of column hc (+32p)
  if (tid == 0) bad = 0;
  for (int b = w; b < np; b += nw)
    for (int a = lane; a < np; a += 32)
      M[a + ld * b] = (a < n && b < n) ? A[a + (long)lda * b] : (a == b ? 1.0 : 0.0);
  __syncthreads();
  if (w == 0) warp_chol_inv16(M, ld, 0, &bad);
  __syncthreads();
  for (int kb = 0; kb < nb; ++kb) {
    if (bad) break;
    const int k0 = CHOL_B * kb, c0 = k0 + CHOL_B;
    // phase 2a: panel, U(k0+r, c) = sum_{s<=r} X(s,r) S(k0+s, c); column c lives in one half-warp
    for (int p = 0; c0 + 32 * p < np; ++p) {
      const int c = c0 + hc + 32 * p;
      double t = 0.0;
      if (c < np) {
#pragma unroll
        for (int s = 0; s < CHOL_B; ++s)  // constant bounds: the loads issue together
          if (s <= hr) t += M[(k0 + s) + ld * (k0 + hr)] * M[(k0 + s) + ld * c];
      }
      __syncwarp();
      if (c < np) M[(k0 + hr) + ld * c] = t;
      __syncwarp();
    }
    // phase 2b: T(i, s) = sum_{s' <= s} U(i, k0+s') X(s', s), rows i < k0
    for (int idx = tid; idx < k0 * CHOL_B; idx += blockDim.x) {
      const int i = idx / CHOL_B, s = idx - i * CHOL_B;
      double t0 = 0.0, t1 = 0.0;
#pragma unroll
      for (int q = 0; q < CHOL_B; q += 2) {
        if (q <= s) t0 = fma(M[i + ld * (k0 + q)], M[(k0 + q) + ld * (k0 + s)], t0);
        if (q + 1 <= s) t1 = fma(M[i + ld * (k0 + q + 1)], M[(k0 + q + 1) + ld * (k0 + s)], t1);
      }
      Tb[i * CHOL_B + s] = t0 + t1;
    }
    __syncthreads();
    if (w == 0) {
      // lookahead: this step's update of the next diagonal block, then its
      // factor and inverse
      if (c0 < np) {
        for (int e = lane; e < CHOL_B * CHOL_B; e += 32) {
          const int r = c0 + (e & 15), c = c0 + (e >> 4);
          if (r <= c) {
            double t0 = 0.0, t1 = 0.0;
#pragma unroll
            for (int s = 0; s < CHOL_B; s += 2) {
              t0 = fma(M[(k0 + s) + ld * r], M[(k0 + s) + ld * c], t0);
              t1 = fma(M[(k0 + s + 1) + ld * r], M[(k0 + s + 1) + ld * c], t1);
            }
            M[r + ld * c] -= t0 + t1;
          }
        }
        __syncwarp();
        warp_chol_inv16(M + c0 + ld * c0, ld, c0, &bad);
      }
    } else {
      // warps 1..nw-1: the inverse's block column k, one lane per (row i < k0,
      // four columns s0..s0+3: four independent sums); the lanes of a warp
      // step through m together (from the warp's smallest row, masked below
      // their own), so T(m, .) is a broadcast and X(i, m) a contiguous row
      for (int base = tid - 32 - lane; base < 4 * k0; base += blockDim.x - 32) {
        const int idx = base + lane;
        const bool act = idx < 4 * k0;
        const int grp = act ? idx / k0 : 0, i = act ? idx - grp * k0 : k0, s0 = 4 * grp;
        const int m0 = __reduce_min_sync(0xffffffffu, i);
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        for (int m = m0; m < k0; ++m) {
          const double x = (m >= i) ? M[i + ld * m] : 0.0;
          const double2 ta = *reinterpret_cast<const double2 *>(Tb + m * CHOL_B + s0);
          const double2 tb = *reinterpret_cast<const double2 *>(Tb + m * CHOL_B + s0 + 2);
          a0 = fma(x, ta.x, a0);
          a1 = fma(x, ta.y, a1);
          a2 = fma(x, tb.x, a2);
          a3 = fma(x, tb.y, a3);
        }
        if (act) {
          M[i + ld * (k0 + s0)] = -a0;
          M[i + ld * (k0 + s0 + 1)] = -a1;
          M[i + ld * (k0 + s0 + 2)] = -a2;
          M[i + ld * (k0 + s0 + 3)] = -a3;
        }
      }
      const int ntask = max(0, np - c0 - CHOL_B);
      for (int task = w - 1; task < ntask; task += nw - 1) {
        const int c = c0 + CHOL_B + task;
        double uc[CHOL_B];
#pragma unroll
        for (int s = 0; s < CHOL_B; ++s) uc[s] = M[(k0 + s) + ld * c];
        for (int r = c0 + lane; r <= c; r += 32) {
          double t0 = 0.0, t1 = 0.0;  // two chains of eight
#pragma unroll
          for (int s = 0; s < CHOL_B; s += 2) {
            t0 = fma(M[(k0 + s) + ld * r], uc[s], t0);
            t1 = fma(M[(k0 + s + 1) + ld * r], uc[s + 1], t1);
          }
          M[r + ld * c] -= t0 + t1;
        }
      }
    }
    __syncthreads();
  }
  if (bad) {
    if (tid == 0 && (first || *info == 0)) *info = base + bad;
    return;
  }
  for (int b = w; b < n; b += nw)
    for (int a = lane; a < n; a += 32) Ui[a + (long)ldu * b] = (a <= b) ? M[a + ld * b] : 0.0;
  if (tid == 0 && first) *info = 0;
}

// Small dense FP64 product for the blocked Cholesky above 144 bands:
// C (m x n, ldc) = alpha op(A) op(B) + beta C, column-major operands, op = the
// matrix (0) or its transpose (1); 64 x 64 tiles, 256 threads of 4 x 4
// outputs, k in steps of 16 through shared memory
__global__ void __launch_bounds__(256) k_small_dgemm(int ta, int tb, int m, int n, int k, double alpha, const double *A,
                                                    int lda, const double *B, int ldb, double beta, double *C,
                                                    int ldc) {
  __shared__ double As[16][64 + 1], Bs[16][64 + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int i0 = blockIdx.x * 64, j0 = blockIdx.y * 64;
  double acc[4][4] = {};
  for (int k0 = 0; k0 < k; k0 += 16) {
    for (int e = threadIdx.x; e < 16 * 64; e += 256) {
      const int kk = e / 64, r = e % 64;
      const int i = i0 + r, j = j0 + r, q = k0 + kk;
      As[kk][r] = (i < m && q < k) ? (ta ? A[q + (long)lda * i] : A[i + (long)lda * q]) : 0.0;
      Bs[kk][r] = (j < n && q < k) ? (tb ? B[j + (long)ldb * q] : B[q + (long)ldb * j]) : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        a[u] = As[kk][tx + 16 * u];
        b[u] = Bs[kk][ty + 16 * u];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = fma(a[u], b[v], acc[u][v]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int i = i0 + tx + 16 * u, j = j0 + ty + 16 * v;
      if (i < m && j < n) {
        double *c = C + i + (long)ldc * j;
        *c = alpha * acc[u][v] + (beta != 0.0 ? beta * *c : 0.0);
      }
    }
}

// e_sr (total_energy.f90:133-239) with minimum image: one thread per atom
// sums its pair forces over every other atom (deterministic order) and the
// pair energies with the atoms after it.  Pair terms are those of the
// reference loop; esr -> out[0], forces F(3,na_max,nsp).
__device__ void pbc_min_image(int sym, double alat, double x1, double y1, double z1, double &X, double &Y, double &Z) {
  if (sym == 1) {
    double A = alat, h = A / 2.0;
    X = fmod(x1, A); Y = fmod(y1, A); Z = fmod(z1, A);
    X = X - A * trunc(X / h); Y = Y - A * trunc(Y / h); Z = Z - A * trunc(Z / h);
  } else {
    double ma = alat * sqrt(2.0) / 4.0, s2 = sqrt(2.0);
    X = (x1 + y1) / s2; Y = (-x1 + y1) / s2;
    X = fmod(X, 2.0 * ma); Y = fmod(Y, 2.0 * ma);
    Z = fmod(z1, 2.0 * ma * s2);
    X = X - 2.0 * ma * trunc(X / ma); Y = Y - 2.0 * ma * trunc(Y / ma);
    Z = Z - 2.0 * ma * s2 * trunc(Z / (s2 * ma));
    if (!(fabs(X) + fabs(Y) + s2 * fabs(Z) < 2.0 * ma)) {
      X = X - copysign(ma, X); Y = Y - copysign(ma, Y); Z = Z - copysign(s2 * ma, Z);
    }
    double xt = (X - Y) / s2;
    Y = (X + Y) / s2;
    X = xt;
  }
}
__global__ void k_esr_par(int nat, const int *isa_is, const int *isa_ia, int na_max, const int *zv, const double *atco,
                          double alat, int sym, double *F, double *out) {
  __shared__ double sh[32];
  const double pi = 4.0 * atan(1.0), rckj = sqrt(1.2 * 1.2 + 1.2 * 1.2);
  double esr = 0;
  for (int l = threadIdx.x; l < nat; l += blockDim.x) {
    const int kl = isa_is[l];
    const double *xl = atco + 3 * (isa_ia[l] + (long)na_max * kl);
    double fx = 0, fy = 0, fz = 0;
    for (int m = 0; m < nat; ++m) {
      if (m == l) continue;
      const int km = isa_is[m];
      const double zv2 = (double)(zv[kl] * zv[km]);
      if (fabs(zv2) < 1e-10) continue;
      const double *xm = atco + 3 * (isa_ia[m] + (long)na_max * km);
      double X, Y, Z;
      pbc_min_image(sym, alat, xl[0] - xm[0], xl[1] - xm[1], xl[2] - xm[2], X, Y, Z);
      const double e2 = X * X + Y * Y + Z * Z, r = sqrt(e2), arg = r / rckj;
      if (arg <= 20.0) {
        const double add = zv2 * erfc(arg) / r;
        if (m > l) esr += add;
        const double pre = (2.0 * zv2 / sqrt(pi)) * exp(-arg * arg) / rckj;
        const double rep = (add + pre) / e2;
        fx += rep * X; fy += rep * Y; fz += rep * Z;
      }
    }
    double *f = F + 3 * (isa_ia[l] + (long)na_max * kl);
    f[0] = fx; f[1] = fy; f[2] = fz;
  }
  const double e = block_sum(esr, sh);
  if (threadIdx.x == 0) out[0] = e;
}

// D = -f' (H nl), f' = occ (1 when < 1e-5)   (FNONLOC T = -FFI*WSG, UPF DDIA)
// and E_nl partial: sum_b occ_b sum_j nl(j,b) (H nl)(j,b)
// with (H nl)(j, b) = sum_j' H(j, j') nl(j', b) formed here (H couples the
// projectors of one atom: wsg on the diagonal, or hlsg between projectors of
// equal l and m) and stored for the forces
__global__ void k_nl_energy_d(int nproj, int nstate, const double *H, const double *nl, double *hn, const double *occ,
                              double *D, double *part, double *out, unsigned *ticket) {
  double s = 0;
  long tot = (long)nproj * nstate;
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < tot; k += (long)gridDim.x * blockDim.x) {
    const int b = (int)(k / nproj), j = (int)(k - (long)b * nproj);
    const double *nb = nl + (long)nproj * b;
    double h = 0.0;
    for (int jp = 0; jp < nproj; ++jp) h += H[j + (long)nproj * jp] * nb[jp];
    hn[k] = h;
    double f = occ[b] < 1e-5 ? 1.0 : occ[b];
    D[k] = -f * h;
    s += occ[b] * nl[k] * h;
  }
  const double v[1] = {s};
  reduce_and_finish<1>(v, part, out, ticket);
}

// ---------------------------------------------------------------- forces
// e_sr (total_energy.f90:133-239) with minimum image (nlp = 0); one block.
// F(3,na_max,nsp) zeroed first as in the reference; esr -> out[0].
__global__ void k_esr(int nsp, const int *na, int na_max, const int *zv, const double *atco, double alat, int sym,
                      int tfor, double *F, double *out) {
  const double pi = 4.0 * atan(1.0);
  const double rckj = sqrt(1.2 * 1.2 + 1.2 * 1.2);
  double esr = 0;
  if (threadIdx.x == 0)
    for (int k = 0; k < 3 * na_max * nsp; ++k) F[k] = 0.0;
  __syncthreads();
  // serial over pairs in thread 0 for the force accumulation order; the
  // pair count is O(atoms^2) and small
  if (threadIdx.x == 0) {
    for (int k = 0; k < nsp; ++k)
      for (int j = k; j < nsp; ++j) {
        double zv2 = (double)(zv[k] * zv[j]);
        if (fabs(zv2) < 1e-10) continue;
        for (int l = 0; l < na[k]; ++l)
          for (int m = (k == j) ? l + 1 : 0; m < na[j]; ++m) {
            const double *xl = atco + 3 * (l + (long)na_max * k), *xm = atco + 3 * (m + (long)na_max * j);
            double x1 = xl[0] - xm[0], y1 = xl[1] - xm[1], z1 = xl[2] - xm[2], X, Y, Z;
            if (sym == 1) {
              double A = alat, h = A / 2.0;
              X = fmod(x1, A); Y = fmod(y1, A); Z = fmod(z1, A);
              X = X - A * trunc(X / h); Y = Y - A * trunc(Y / h); Z = Z - A * trunc(Z / h);
            } else {
              double ma = alat * sqrt(2.0) / 4.0, s2 = sqrt(2.0);
              X = (x1 + y1) / s2; Y = (-x1 + y1) / s2;
              X = fmod(X, 2.0 * ma); Y = fmod(Y, 2.0 * ma);
              Z = fmod(z1, 2.0 * ma * s2);
              X = X - 2.0 * ma * trunc(X / ma); Y = Y - 2.0 * ma * trunc(Y / ma);
              Z = Z - 2.0 * ma * s2 * trunc(Z / (s2 * ma));
              if (!(fabs(X) + fabs(Y) + s2 * fabs(Z) < 2.0 * ma)) {
                X = X - copysign(ma, X); Y = Y - copysign(ma, Y); Z = Z - copysign(s2 * ma, Z);
              }
              double xt = (X - Y) / s2;
              Y = (X + Y) / s2;
              X = xt;
            }
            double e2 = X * X + Y * Y + Z * Z, r = sqrt(e2), arg = r / rckj;
            if (arg <= 20.0) {
              double add = zv2 * erfc(arg) / r;
              esr += add;
              if (tfor) {
                double pre = (2.0 * zv2 / sqrt(pi)) * exp(-arg * arg) / rckj;
                double rep = (add + pre) / e2;
                double *fl = F + 3 * (l + (long)na_max * k), *fm = F + 3 * (m + (long)na_max * j);
                fl[0] += rep * X; fl[1] += rep * Y; fl[2] += rep * Z;
                fm[0] -= rep * X; fm[1] -= rep * Y; fm[2] -= rep * Z;
              }
            }
          }
      }
    out[0] = esr;
  }
}

// POTFOR (nuclear_grad.f90:4-50): per atom and block partial sums of
// Re[S_I(G) (rhos V_H(G)* + vps rho_e(G)*) i G] 2 Omega tpiba over G != 0
__global__ void k_potfor(int ngrho, const int *inyh, int nh1, int nh2, int nh3, AtomArgs aa, const double *hg,
                         const double *gvec, double tpiba2, const double2 *rhog, const double2 *erhos, const double *vps,
                         const double *rhos, double omtp, double *part) {
  __shared__ double sh[32];
  const double fp = 16.0 * atan(1.0);
  int a = blockIdx.y, is = aa.is[a];
  double fx = 0, fy = 0, fz = 0;
  for (int g = 1 + blockIdx.x * blockDim.x + threadIdx.x; g < ngrho; g += gridDim.x * blockDim.x) {
    double2 rh = rhog[g], rp = erhos[g];
    double rgx = rh.x + rp.x, rgy = rh.y + rp.y;
    double f = fp / (tpiba2 * hg[g]);
    double rs = rhos[(long)is * ngrho + g], vs = vps[(long)is * ngrho + g];
    // base = rhos f conj(rho+rho_ion) + vps conj(rho)
    double bx = rs * f * rgx + vs * rh.x, by = -(rs * f * rgy) - vs * rh.y;
    double2 e = eig_at(inyh, g, nh1, nh2, nh3, aa.arg + 3 * a);
    double im = e.x * by + e.y * bx;  // Im(e * base)
    fx += -im * gvec[3 * g] * omtp;
    fy += -im * gvec[3 * g + 1] * omtp;
    fz += -im * gvec[3 * g + 2] * omtp;
  }
  double sx = block_sum(fx, sh), sy = block_sum(fy, sh), sz = block_sum(fz, sh);
  if (threadIdx.x == 0) {
    long o = ((long)a * 3) * gridDim.x + blockIdx.x;
    part[o] = sx;
    part[o + gridDim.x] = sy;
    part[o + 2 * gridDim.x] = sz;
  }
}
// Q_{k,j}(G) = -i G_k P_j(G) for the projector derivatives (D_FNL,
// nuclear_grad.f90:330-357): rows ordered k*nproj + j
__global__ void k_dproj(int ngpw, int nproj, const double *gvec, const double2 *P, double2 *Q) {
  int g = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (g >= ngpw) return;
  double2 p = P[(long)j * ngpw + g];
  double gk = gvec[3L * g + k];
  Q[((long)k * nproj + j) * ngpw + g] = make_double2(gk * p.y, -gk * p.x);
}
// NLFOR / UPF_NLFOR (nuclear_grad.f90:51-89,153-199) plus POTFOR/e_sr sums:
// F(isa) += potfor - sum_{j of isa} sum_b 2 occ_b (H nl)(j,b) dfnl_k(j,b)
__global__ void k_force_total(int nat, int nproj, int nstate, const int *proj_isa, const double *hn, const double *dfnl,
                              const double *occ, const double *potpart, int pnb, const int *isa_is, const int *isa_ia,
                              int na_max, double *F) {
  __shared__ double sh[32];
  int a = blockIdx.x;
  for (int k = 0; k < 3; ++k) {
    double s = 0;
    for (long q = threadIdx.x; q < (long)nproj * nstate; q += blockDim.x) {
      int j = (int)(q % nproj), b = (int)(q / nproj);
      if (proj_isa[j] != a) continue;
      double w = occ[b];
      if (!(fabs(w) > 1e-12)) continue;
      s += 2.0 * w * hn[j + (long)nproj * b] * dfnl[(long)k * nproj + j + (long)3 * nproj * b];
    }
    double nlf = block_sum(s, sh);
    double pf = 0;
    for (int i = threadIdx.x; i < pnb; i += blockDim.x) pf += potpart[((long)a * 3 + k) * pnb + i];
    double pfs = block_sum(pf, sh);
    if (threadIdx.x == 0) F[3 * (isa_ia[a] + (long)na_max * isa_is[a]) + k] += pfs - nlf;
    __syncthreads();
  }
}

}  // namespace amdk
