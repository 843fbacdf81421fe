/*
 * oracle.c -- CPU FP64 restatement of AMDKIIT's wavefunction hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker for amdkiit_b200/; never linked by
 * the product).  Every function names the reference routine it restates
 * (file:line relative to the AMDKIIT project root).  Array layouts follow
 * the reference: Fortran column-major, 1-based integer maps, real-space
 * grids with odd leading dimensions nrlead (gvectors.f90:492-497).
 *
 * Compile with -ffp-contract=off: the integer G-vector order depends on the
 * exact bits of |G|^2 (gvectors.f90:229-248).
 */
#include "oracle.h"
#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double _Complex zc;

static double PI_, TWOPI_, FOURPI_;
/* constants.f90:3-5, set when the library is loaded */
__attribute__((constructor)) static void init_constants(void) {
  PI_ = 4.0 * atan(1.0);
  TWOPI_ = 8.0 * atan(1.0);
  FOURPI_ = 16.0 * atan(1.0);
}
static const double RAGGIO = 1.2;      /* system_data_types.f90:72 */
static const double EPSGX = 1.0e-12;   /* gvectors.f90:125 */
static const double HCUT = 0.5;        /* constants.f90:15 */
static const double GC_CUTOFF = 1.0e-8;/* constants.f90:11 */

#define MAXNGH 120
#define MPRO 4
#define LMAXX 5

/* ------------------------------------------------------------------ */
/* 1D mixed-radix FFT (replaces FFTW in fft_interface.f90:366-498)     */
/* ------------------------------------------------------------------ */
typedef struct {
  int n, nf, f[40];
  zc *w; /* w[k] = exp(-2 pi i k / n) */
} fftplan;

static void plan_init(fftplan *p, int n) {
  int m = n;
  p->n = n;
  p->nf = 0;
  while (m % 4 == 0) { p->f[p->nf++] = 4; m /= 4; }
  while (m % 2 == 0) { p->f[p->nf++] = 2; m /= 2; }
  while (m % 3 == 0) { p->f[p->nf++] = 3; m /= 3; }
  while (m % 5 == 0) { p->f[p->nf++] = 5; m /= 5; }
  if (m != 1) { fprintf(stderr, "oracle: FFT length %d is not 2,3,5-smooth\n", n); abort(); }
  p->w = (zc *)malloc(sizeof(zc) * n);
  for (int k = 0; k < n; k++) {
    double a = -TWOPI_ * (double)k / (double)n;
    p->w[k] = cos(a) + I * sin(a);
  }
}

/* Stockham autosort: stage with s = product of previous radices, radix r,
 * m = n/(s r):  y[k + s p + s r j] = w_{n/s}^{j p} sum_q x[k + s j + s m q] w_r^{p q}.
 * sign = -1 -> exp(-i...) (FFTW_FORWARD), +1 -> exp(+i...) (FFTW_BACKWARD). */
static void fft1d(const fftplan *p, zc *x, zc *tmp, int sign) {
  int n = p->n, s = 1;
  zc *a = x, *b = tmp;
  for (int st = 0; st < p->nf; st++) {
    int r = p->f[st];
    int m = n / (s * r);
    for (int j = 0; j < m; j++) {
      for (int k = 0; k < s; k++) {
        zc in[5], out[5];
        for (int q = 0; q < r; q++) in[q] = a[k + s * j + s * m * q];
        if (r == 2) {
          out[0] = in[0] + in[1];
          out[1] = in[0] - in[1];
        } else if (r == 4) {
          zc t0 = in[0] + in[2], t1 = in[0] - in[2];
          zc t2 = in[1] + in[3], t3 = in[1] - in[3];
          zc it3 = (sign > 0) ? (I * t3) : (-I * t3);
          out[0] = t0 + t2;
          out[2] = t0 - t2;
          out[1] = t1 + it3;
          out[3] = t1 - it3;
        } else {
          for (int pp = 0; pp < r; pp++) {
            zc acc = 0;
            for (int q = 0; q < r; q++) {
              int e = (pp * q) % r;
              zc wq = p->w[(e * (n / r)) % n];
              if (sign > 0) wq = conj(wq);
              acc += in[q] * wq;
            }
            out[pp] = acc;
          }
        }
        for (int pp = 0; pp < r; pp++) {
          int e = (int)(((long)s * j * pp) % n);
          zc tw = p->w[e];
          if (sign > 0) tw = conj(tw);
          b[k + s * pp + s * r * j] = out[pp] * tw;
        }
      }
    }
    zc *t = a; a = b; b = t;
    s *= r;
  }
  if (a != x) memcpy(x, a, sizeof(zc) * n);
}

/* batched strided 1D FFT: line l element k at in[l*idist + k*istride] */
static void fft_many(const fftplan *p, int howmany, const zc *in, long istride, long idist,
                     zc *out, long ostride, long odist, int sign, double scale) {
  int n = p->n;
#pragma omp parallel
  {
    zc *buf = (zc *)malloc(sizeof(zc) * 2 * n);
#pragma omp for schedule(static)
    for (int l = 0; l < howmany; l++) {
      for (int k = 0; k < n; k++) buf[k] = in[(long)l * idist + (long)k * istride];
      fft1d(p, buf, buf + n, sign);
      if (scale != 1.0)
        for (int k = 0; k < n; k++) out[(long)l * odist + (long)k * ostride] = scale * buf[k];
      else
        for (int k = 0; k < n; k++) out[(long)l * odist + (long)k * ostride] = buf[k];
    }
    free(buf);
  }
}

/* ------------------------------------------------------------------ */
/* system state                                                        */
/* ------------------------------------------------------------------ */
struct orc_sys {
  int nthreads;
  int nsp, na[ORC_MAXSP], na_max, nat, xc, symmetry;
  int zv[ORC_MAXSP];          /* INTEGER in the reference (system_data_types.f90:151) */
  orc_species sp[ORC_MAXSP];
  double *rr[ORC_MAXSP], *rw[ORC_MAXSP], *vr[ORC_MAXSP], *rps[ORC_MAXSP];
  double *rab[ORC_MAXSP], *vloc[ORC_MAXSP], *beta[ORC_MAXSP];
  double ecut, ecut_rho;
  double a_cell[9], b_cell[9], alat, omega, tpiba, tpiba2, gcut_pw, gcut_rho;
  int nr[3], nrl[3];
  long nnr1, max_fft;
  /* G vectors (gvectors.f90) */
  int ngpw, ngrho, ngpw_le, ngrays, nhrays;
  int *inyh;      /* inyh(3,ngrho) */
  double *hg, *gvec, *hg_pert;
  int *mapp, *mapm, *msp;
  int *xrays;     /* xrays_pw(nrl2,nrl3) after prepare_fft */
  /* atoms */
  int *isa_is, *isa_ia;
  double *atco;   /* atco(3,na_max,nsp) */
  /* pseudopotential tables */
  int upf;
  int ngh[ORC_MAXSP], nghmax, nghtol[ORC_MAXSP][MAXNGH], nghcom[ORC_MAXSP][MAXNGH];
  int lpval[ORC_MAXSP][MAXNGH], lfval[ORC_MAXSP][MAXNGH];
  double wsg[ORC_MAXSP][MAXNGH];
  double hlsg[ORC_MAXSP][LMAXX][MPRO][MPRO];
  double *wns[ORC_MAXSP];       /* wns(nspln, MAXNGH) per species */
  double *voo[ORC_MAXSP];       /* local form factor on ggnh */
  double *vps, *rhos;           /* vps(is,ig) -> [is*ngrho+ig] */
  double *twnl;                 /* twnl(ngpw,nghmax,nsp) */
  zc *eigr, *eigrxvps, *eigrxrhos;
  /* electronic state */
  int nstate;
  double *occ;
  /* open shell (LSD): bands 1..nel_up are spin 1, the rest spin 2 (init_module.f90:122-131);
     rho = total density, rho2 = spin-2 density, v_pot / v_pot2 the potentials of spins 1 / 2 */
  int lsd, nel_up;
  double *rho2, *v_pot2;
  zc *c0, *c2, *hnm1, *c2p;
  double *rho, *v_pot;
  zc *rho_g;
  double *nl, *dfnl;            /* nl(atom_t,nghmax,nstate), dfnl(atom_t,nghmax,3,nstate) */
  double *force;                /* force(3,na_max,nsp) */
  double *grad;                 /* grad(nnr1,4) */
  /* energies (total_energy.f90) */
  double eke, enl, eloc, exc, etxc, esr, eself, estat, etotal, eh_re;
  double gemax, cnorm;
  int convwf, tfor;
  double ghist[10], fhist[10];
  /* FFT */
  fftplan pl[3];
  zc *w1, *w2, *wk;
};

static void *xcalloc(size_t n, size_t sz) {
  void *p = calloc(n ? n : 1, sz);
  if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
  return p;
}

/* ------------------------------------------------------------------ */
/* set_cell.f90 / fft_support.f90                                      */
/* ------------------------------------------------------------------ */
#define A3(m, i, j) (m)[((i)-1) + 3 * ((j)-1)]

/* math.f90:4-64 inverse_matrix (Gauss-Jordan with pivoting) */
static void inverse_matrix3(const double *ain, double *b) {
  double a[9], d[9];
  int ip[4];
  memcpy(a, ain, sizeof a);
  for (int i = 0; i < 9; i++) b[i] = 0.0;
  for (int i = 1; i <= 3; i++) A3(b, i, i) = 1.0;
  for (int k = 1; k <= 3; k++) ip[k] = k;
  for (int k = 1; k <= 3; k++) {
    double dmax = fabs(A3(a, ip[k], ip[k]));
    int imax = k;
    for (int l = k; l <= 3; l++)
      if (fabs(A3(a, ip[l], ip[k])) > dmax) { dmax = fabs(A3(a, ip[l], ip[k])); imax = l; }
    int t = ip[imax]; ip[imax] = ip[k]; ip[k] = t;
    for (int i = 1; i <= 3; i++) {
      if (i != k) {
        double s = A3(a, ip[i], k) / A3(a, ip[k], k);
        double rowk[4];
        for (int c = k; c <= 3; c++) rowk[c] = A3(a, ip[k], c) * s;
        for (int c = k; c <= 3; c++) A3(a, ip[i], c) = A3(a, ip[i], c) - rowk[c];
        for (int c = 1; c <= 3; c++) rowk[c] = A3(b, ip[k], c) * s;
        for (int c = 1; c <= 3; c++) A3(b, ip[i], c) = A3(b, ip[i], c) - rowk[c];
      }
    }
  }
  for (int i = 1; i <= 3; i++)
    for (int c = 1; c <= 3; c++) A3(d, i, c) = A3(b, ip[i], c) / A3(a, ip[i], i);
  memcpy(b, d, sizeof d);
}

/* fft_support.f90:50-83 permitted */
static int permitted(int n) {
  int m = n;
  int f[5] = {2, 3, 5, 7, 11}, pw[5] = {0, 0, 0, 0, 0};
  for (int i = 0; i < 5; i++)
    while (m % f[i] == 0 && m > 1) { m /= f[i]; pw[i]++; }
  if (m != 1) return 0;
  return pw[3] == 0 && pw[4] == 0;
}

/* fft_support.f90:85-118 optimal_fft_order(n,2) */
static int optimal_fft_order(int n_old, int n_order) {
  int n = n_old;
  while ((!permitted(n) || n % n_order != 0) && n <= 2049) n++;
  return n;
}

/* set_cell.f90:177-211 set_r_grids */
static void set_r_grids(const double *a, double ecut_rho, int *nr) {
  for (int j = 1; j <= 3; j++) {
    double d = A3(a, 1, j) * A3(a, 1, j) + A3(a, 2, j) * A3(a, 2, j);
    d = d + A3(a, 3, j) * A3(a, 3, j);
    double ax = sqrt(d);
    double x = ax / PI_;
    x = x * sqrt(ecut_rho);
    x = x + 0.5;
    int n = (int)lround(x);
    nr[j - 1] = optimal_fft_order(n, 2);
  }
}

/* gvectors.f90:500-511 Gsquare */
static double gsquare(int ix, int iy, int iz, const double *b) {
  double t1 = (double)ix * A3(b, 1, 1);
  t1 = t1 + (double)iy * A3(b, 1, 2);
  t1 = t1 + (double)iz * A3(b, 1, 3);
  double t2 = (double)ix * A3(b, 2, 1);
  t2 = t2 + (double)iy * A3(b, 2, 2);
  t2 = t2 + (double)iz * A3(b, 2, 3);
  double t3 = (double)ix * A3(b, 3, 1);
  t3 = t3 + (double)iy * A3(b, 3, 2);
  t3 = t3 + (double)iz * A3(b, 3, 3);
  double g = t1 * t1;
  g = g + t2 * t2;
  g = g + t3 * t3;
  return g;
}

/* math.f90:200-305 sort_array2 (quicksort + insertion, 1-based) */
static void sort_array2(int n, double *arr1, int *index1) {
  double *arr = arr1 - 1;
  int *index = index1 - 1;
  enum { M = 7, NSTACK = 50 };
  int istack[NSTACK + 1];
  int i, l, ib, ir, jstack, k, itemp, j;
  double a, temp;
  for (i = 1; i <= n; i++) index[i] = i;
  jstack = 0;
  l = 1;
  ir = n;
  for (;;) {
    if (ir - l < M) {
      for (j = l + 1; j <= ir; j++) {
        a = arr[j];
        ib = index[j];
        for (i = j - 1; i >= 1; i--) {
          if (arr[i] <= a) goto l2;
          arr[i + 1] = arr[i];
          index[i + 1] = index[i];
        }
        i = 0;
      l2:
        arr[i + 1] = a;
        index[i + 1] = ib;
      }
      if (jstack == 0) return;
      ir = istack[jstack];
      l = istack[jstack - 1];
      jstack -= 2;
    } else {
      k = (l + ir) / 2;
      temp = arr[k]; arr[k] = arr[l + 1]; arr[l + 1] = temp;
      itemp = index[k]; index[k] = index[l + 1]; index[l + 1] = itemp;
      if (arr[l + 1] > arr[ir]) {
        temp = arr[l + 1]; arr[l + 1] = arr[ir]; arr[ir] = temp;
        itemp = index[l + 1]; index[l + 1] = index[ir]; index[ir] = itemp;
      }
      if (arr[l] > arr[ir]) {
        temp = arr[l]; arr[l] = arr[ir]; arr[ir] = temp;
        itemp = index[l]; index[l] = index[ir]; index[ir] = itemp;
      }
      if (arr[l + 1] > arr[l]) {
        temp = arr[l + 1]; arr[l + 1] = arr[l]; arr[l] = temp;
        itemp = index[l + 1]; index[l + 1] = index[l]; index[l] = itemp;
      }
      i = l + 1;
      j = ir;
      a = arr[l];
      ib = index[l];
      for (;;) {
        do { i++; } while (arr[i] < a);
        do { j--; } while (arr[j] > a);
        if (j < i) break;
        temp = arr[i]; arr[i] = arr[j]; arr[j] = temp;
        itemp = index[i]; index[i] = index[j]; index[j] = itemp;
      }
      arr[l] = arr[j];
      arr[j] = a;
      index[l] = index[j];
      index[j] = ib;
      jstack += 2;
      if (jstack > NSTACK) { fprintf(stderr, "oracle: SORT2 Nstack too small\n"); abort(); }
      if (ir - i + 1 >= j - l) {
        istack[jstack] = ir;
        istack[jstack - 1] = i;
        ir = j - 1;
      } else {
        istack[jstack] = j - 1;
        istack[jstack - 1] = l;
        l = i;
      }
    }
  }
}

/* gvectors.f90:111-341 distribute_gvectors (ncpu = 1), sort_gvectors
 * (:514-564), compute_gvec_gvec2 (:742-776); fft_interface.f90:151-363
 * prepare_fft (ray numbering and the compressed maps). */
static void setup_gvectors(orc_sys *s) {
  int nr1 = s->nr[0], nr2 = s->nr[1], nr3 = s->nr[2];
  int nh1 = nr1 / 2 + 1, nh2 = nr2 / 2 + 1, nh3 = nr3 / 2 + 1;
  const double *b = s->b_cell;
  /* count */
  long cnt = 0;
  for (int ix = 0; ix <= nr1 - 1; ix++) {
    int ymin = (ix == 0) ? 0 : -nr2 + 1;
    for (int iy = ymin; iy <= nr2 - 1; iy++) {
      int zmin = (ix == 0 && iy == 0) ? 0 : -nr3 + 1;
      for (int iz = zmin; iz <= nr3 - 1; iz++)
        if (gsquare(ix, iy, iz, b) < s->gcut_rho) cnt++;
    }
  }
  s->ngrho = (int)cnt;
  s->inyh = (int *)xcalloc(3 * cnt, sizeof(int));
  s->hg = (double *)xcalloc(cnt, sizeof(double));
  s->hg_pert = (double *)xcalloc(cnt, sizeof(double));
  s->gvec = (double *)xcalloc(3 * cnt, sizeof(double));
  int ig = 0, ngpw = 0;
  for (int ix = 0; ix <= nr1 - 1; ix++) {
    int ymin = (ix == 0) ? 0 : -nr2 + 1;
    for (int iy = ymin; iy <= nr2 - 1; iy++) {
      int zmin = (ix == 0 && iy == 0) ? 0 : -nr3 + 1;
      for (int iz = zmin; iz <= nr3 - 1; iz++) {
        double gsq = gsquare(ix, iy, iz, b);
        if (gsq < s->gcut_rho) {
          ig++;
          double sign;
          if (gsq < s->gcut_pw) { ngpw++; sign = -1.0; } else sign = 1.0;
          double t = sqrt((double)(ig - 1));
          t = t * EPSGX;
          t = t * sign;
          t = 1.0 + t;
          s->hg[ig - 1] = gsq * t;
          s->inyh[3 * (ig - 1) + 0] = nh1 + ix;
          s->inyh[3 * (ig - 1) + 1] = nh2 + iy;
          s->inyh[3 * (ig - 1) + 2] = nh3 + iz;
        }
      }
    }
  }
  s->ngpw = ngpw;
  /* sort_gvectors */
  int n = s->ngrho;
  int *gi = (int *)xcalloc(n, sizeof(int));
  sort_array2(n, s->hg, gi);
  memcpy(s->hg_pert, s->hg, sizeof(double) * n);
  int *g_index = gi - 1;
  for (int g = 1; g <= n - 1; g++) {
    for (;;) {
      if (g_index[g] != g) {
        int jg = g_index[g];
        g_index[g] = g_index[jg];
        g_index[jg] = jg;
        int ind[3];
        int a = g_index[g];
        for (int c = 0; c < 3; c++) ind[c] = s->inyh[3 * (a - 1) + c];
        for (int c = 0; c < 3; c++) s->inyh[3 * (a - 1) + c] = s->inyh[3 * (g_index[jg] - 1) + c];
        for (int c = 0; c < 3; c++) s->inyh[3 * (jg - 1) + c] = ind[c];
      } else
        break;
    }
  }
  free(gi);
  /* compute_gvec_gvec2 */
  for (int g = 0; g < n; g++) {
    int ix = s->inyh[3 * g] - nh1, iy = s->inyh[3 * g + 1] - nh2, iz = s->inyh[3 * g + 2] - nh3;
    for (int r = 1; r <= 3; r++) {
      double t = (double)ix * A3(b, r, 1);
      t = t + (double)iy * A3(b, r, 2);
      t = t + (double)iz * A3(b, r, 3);
      s->gvec[3 * g + r - 1] = t;
    }
    double h = s->gvec[3 * g] * s->gvec[3 * g];
    h = h + s->gvec[3 * g + 1] * s->gvec[3 * g + 1];
    h = h + s->gvec[3 * g + 2] * s->gvec[3 * g + 2];
    s->hg[g] = h;
  }
  /* prepare_fft: ray numbering (PW rays first, then density-only rays) */
  int k2 = s->nrl[1], k3 = s->nrl[2];
  int *xr = (int *)xcalloc((long)k2 * k3, sizeof(int));
#define XR(i, j) xr[((i)-1) + (long)k2 * ((j)-1)]
  for (int g = 0; g < s->ngpw; g++) {
    int i2 = s->inyh[3 * g + 1], i3 = s->inyh[3 * g + 2];
    int j2 = -i2 + 2 * nh2, j3 = -i3 + 2 * nh3;
    if (j2 > k2 || j3 > k3 || j2 < 1 || j3 < 1) { fprintf(stderr, "oracle: mirror ray outside the grid\n"); abort(); }
    XR(i2, i3) += 1;
    XR(j2, j3) += 1;
  }
  int ii = 0;
  for (int j = 1; j <= k3; j++)
    for (int i = 1; i <= k2; i++)
      if (XR(i, j) != 0) XR(i, j) = ++ii;
  s->ngrays = ii;
  for (int g = s->ngpw; g < s->ngrho; g++) {
    int i2 = s->inyh[3 * g + 1], i3 = s->inyh[3 * g + 2];
    int j2 = -i2 + 2 * nh2, j3 = -i3 + 2 * nh3;
    if (j2 > k2 || j3 > k3 || j2 < 1 || j3 < 1) { fprintf(stderr, "oracle: mirror ray outside the grid\n"); abort(); }
    if (XR(i2, i3) == 0) XR(i2, i3) = -1;
    if (XR(j2, j3) == 0) XR(j2, j3) = -1;
  }
  for (int j = 1; j <= k3; j++)
    for (int i = 1; i <= k2; i++)
      if (XR(i, j) < 0) XR(i, j) = ++ii;
  s->nhrays = ii;
  s->msp = (int *)xcalloc(s->nhrays, sizeof(int));
  for (int i = 1; i <= k2; i++)
    for (int j = 1; j <= k3; j++) {
      int r = XR(i, j);
      if (r > 0) s->msp[r - 1] = i + (j - 1) * k2;
    }
  s->mapp = (int *)xcalloc(n, sizeof(int));
  s->mapm = (int *)xcalloc(n, sizeof(int));
  for (int g = 0; g < n; g++) {
    int i1 = s->inyh[3 * g], i2 = s->inyh[3 * g + 1], i3 = s->inyh[3 * g + 2];
    int j1 = -i1 + 2 * nh1, j2 = -i2 + 2 * nh2, j3 = -i3 + 2 * nh3;
    s->mapp[g] = i1 + (XR(i2, i3) - 1) * s->nrl[0];
    s->mapm[g] = j1 + (XR(j2, j3) - 1) * s->nrl[0];
  }
#undef XR
  s->xrays = xr;
  long a1 = (long)s->nrl[0] * s->nrl[1] * s->nrl[2];
  long a2 = (long)s->nr[0] * s->nhrays;
  s->max_fft = a1 > a2 ? a1 : a2;
}

/* ------------------------------------------------------------------ */
/* math helpers: spline (spline.f90, spline_inter.f90), simpsn          */
/* (math.f90:319-343), sph_bes (bessel_func.f90:210-260)                */
/* ------------------------------------------------------------------ */
typedef struct { int n; const double *xp; const double *yp; double *h, *sdd; } spl;

static void spline_setup(spl *sp, int n, const double *xp, const double *yp) {
  sp->n = n; sp->xp = xp; sp->yp = yp;
  sp->h = (double *)xcalloc(n + 1, sizeof(double));
  sp->sdd = (double *)xcalloc(n + 1, sizeof(double));
  double *h = sp->h, *v = (double *)xcalloc(n + 1, sizeof(double)), *u = (double *)xcalloc(n + 1, sizeof(double));
  double *bb = (double *)xcalloc(n + 1, sizeof(double));
  /* 1-based: h[i], i=1..n-1 */
  for (int i = 1; i <= n - 1; i++) {
    h[i] = xp[i] - xp[i - 1];
    bb[i] = (yp[i] - yp[i - 1]) / h[i];
  }
  v[1] = 0; u[1] = 0;
  for (int i = 2; i <= n - 1; i++) {
    v[i] = 2.0 * (h[i - 1] + h[i]);
    u[i] = 6.0 * (bb[i] - bb[i - 1]);
  }
  int m = n - 2;
  double *d = (double *)xcalloc(m + 1, sizeof(double)), *a = (double *)xcalloc(m + 1, sizeof(double));
  double *b = (double *)xcalloc(m + 1, sizeof(double)), *c = (double *)xcalloc(m + 1, sizeof(double));
  double *x = (double *)xcalloc(m + 1, sizeof(double));
  for (int i = 1; i <= m; i++) { d[i] = v[i + 1]; a[i] = h[i + 1]; c[i] = h[i + 1]; b[i] = u[i + 1]; }
  for (int i = 2; i <= m; i++) {
    double s = a[i - 1] / d[i - 1];
    d[i] = d[i] - s * c[i - 1];
    b[i] = b[i] - s * b[i - 1];
  }
  x[m] = b[m] / d[m];
  for (int i = m - 1; i >= 1; i--) x[i] = (b[i] - c[i] * x[i + 1]) / d[i];
  sp->sdd[1] = 0; sp->sdd[n] = 0;
  for (int i = 2; i <= n - 1; i++) sp->sdd[i] = x[i - 1];
  free(v); free(u); free(bb); free(d); free(a); free(b); free(c); free(x);
}
static void spline_free(spl *sp) { free(sp->h); free(sp->sdd); }

/* spline_hunt: ig = first i in 2..n with x < xp(i), minus 1; else 1 */
static int spline_hunt(const spl *sp, double x) {
  const double *xp = sp->xp;
  int n = sp->n;
  if (!(x < xp[n - 1])) return 1;
  int lo = 2, hi = n; /* 1-based: find smallest i in [lo,hi] with x < xp(i) */
  while (lo < hi) {
    int mid = (lo + hi) / 2;
    if (x < xp[mid - 1]) hi = mid; else lo = mid + 1;
  }
  return lo - 1;
}
static double spline_eval(const spl *sp, int ig, double x) {
  const double *xp = sp->xp - 1, *yp = sp->yp - 1, *h = sp->h, *sdd = sp->sdd;
  double d1 = x - xp[ig], d2 = xp[ig + 1] - x;
  double t1 = sdd[ig + 1] / 6.0 / h[ig] * (d1 * d1 * d1);
  double t2 = sdd[ig] / 6.0 / h[ig] * (d2 * d2 * d2);
  double t3 = (yp[ig + 1] / h[ig] - sdd[ig + 1] / 6.0 * h[ig]) * d1;
  double t4 = (yp[ig] / h[ig] - h[ig] / 6.0 * sdd[ig]) * d2;
  return t1 + t2 + t3 + t4;
}
/* spline_inter(n,xpp,ypp,intp_x,intp_y,intp_n): values beyond xp(n) keep
 * their previous content (the loop EXITs) */
static void spline_inter(int n, const double *xp, const double *yp, const double *x, double *y, int nx) {
  spl sp;
  spline_setup(&sp, n, xp, yp);
  for (int i = 0; i < nx; i++) {
    if (x[i] > xp[n - 1]) break;
    y[i] = spline_eval(&sp, spline_hunt(&sp, x[i]), x[i]);
  }
  spline_free(&sp);
}

static double simpsn(int n, double *f1) {
  const double C1 = 109.0 / 48.0, C2 = -5.0 / 48.0, C3 = 63.0 / 48.0, C4 = 49.0 / 48.0;
  double *f = f1 - 1;
  f[1] *= C1; f[2] *= C2; f[3] *= C3; f[4] *= C4;
  f[n - 1] *= C1; f[n - 2] *= C2; f[n - 3] *= C3; f[n - 4] *= C4;
  double sum = 0;
  for (int i = 1; i <= n - 1; i++) sum = sum + f[i];
  return sum;
}

static double sph_bes(int n, double xx) {
  const int kmax = 40;
  const double toler = 1e-15;
  if (fabs(xx) < toler) return n == 0 ? 1.0 : 0.0;
  double jl, jlp = 0, jr, fact;
  if (xx < 1) {
    fact = 1;
    for (int id = 1; id <= n; id++) fact = fact * xx / (double)(2 * id + 1);
    jl = 1; jr = 1;
    int k = 0;
    while (fabs(jr) >= toler && k < kmax) {
      k++;
      jr = -jr * (0.5 * xx * xx) / (double)(k * (2 * (n + k) + 1));
      jl = jl + jr;
    }
    return jl * fact;
  }
  jl = sin(xx) / xx;
  jlp = (-cos(xx) + jl) / xx;
  for (int id = 2; id <= n + 1; id++) {
    jr = -jl + (double)(2 * id - 1) * jlp / xx;
    jl = jlp;
    jlp = jr;
  }
  return jl;
}

/* spherical_func.f90:158-206 compute_yL for one G */
static double ylm_one(int L, double hg, const double *g) {
  if (fabs(hg) >= 1e-6) {
    switch (L) {
      case 1: return sqrt(1.0 / FOURPI_);
      case 2: return sqrt(3.0 / FOURPI_) * g[0] / sqrt(hg);
      case 3: return sqrt(3.0 / FOURPI_) * g[2] / sqrt(hg);
      case 4: return sqrt(3.0 / FOURPI_) * g[1] / sqrt(hg);
      case 5: return sqrt(15.0 / FOURPI_) * g[0] * g[1] / hg;
      case 6: return sqrt(15.0 / FOURPI_) * g[0] * g[2] / hg;
      case 7: return sqrt(5.0 / FOURPI_ / 4.0) * (3.0 * (g[2] * g[2]) / hg - 1.0);
      case 8: return sqrt(15.0 / FOURPI_) * g[1] * g[2] / hg;
      case 9: return sqrt(15.0 / FOURPI_ / 4.0) * (g[0] * g[0] - g[1] * g[1]) / hg;
      default: return 0.0;
    }
  }
  return L == 1 ? sqrt(1.0 / FOURPI_) : 0.0;
}

/* ------------------------------------------------------------------ */
/* pseudopotential tables                                              */
/* ------------------------------------------------------------------ */
/* interpolgrid.f90:146-168 INTRP_GRID: cc keeps its value when rw > rp(mp) */
static void intrp_grid(const double *rp, int mp, const double *rw, int mw, double *f) {
  double *fc = (double *)xcalloc(mp, sizeof(double));
  memcpy(fc, f, sizeof(double) * mp);
  spl sp;
  spline_setup(&sp, mp, rp, fc);
  double cc = 0.0;
  for (int i = 0; i < mw; i++) {
    if (!(rw[i] > rp[mp - 1])) cc = spline_eval(&sp, spline_hunt(&sp, rw[i]), rw[i]);
    f[i] = cc;
  }
  spline_free(&sp);
  free(fc);
}

/* exp_igr.f90:211-288 form_factor (psp) and :142-209 form_factor_upf */
static void form_factors(orc_sys *s) {
  int ngrho = s->ngrho;
  s->vps = (double *)xcalloc((long)s->nsp * ngrho, sizeof(double));
  s->rhos = (double *)xcalloc((long)s->nsp * ngrho, sizeof(double));
  double *ggnh = (double *)xcalloc(ORC_NSPLN, sizeof(double));
  double *vo = (double *)xcalloc(ngrho, sizeof(double));
  for (int is = 0; is < s->nsp; is++) {
    int mesh = s->sp[is].mesh;
    double *rr = s->rr[is], *rw = s->rw[is];
    double *fint = (double *)xcalloc(mesh, sizeof(double)), *dfint = (double *)xcalloc(mesh, sizeof(double));
    s->voo[is] = (double *)xcalloc(ORC_NSPLN, sizeof(double));
    double zvd = (double)s->zv[is];
    if (!s->upf) {
      rw[0] = rr[0];
      for (int ir = 1; ir < mesh; ir++) rw[ir] = rw[ir - 1] * exp(log(rr[mesh - 1] / rr[0]) / (double)(mesh - 1));
      for (int il = 0; il < s->sp[is].lmax; il++) intrp_grid(rr, mesh, rw, mesh, s->vr[is] + (long)il * mesh);
      const double *vl = s->vr[is] + (long)(s->sp[is].l_local - 1) * mesh;
      for (int ir = 0; ir < mesh; ir++) {
        double e = erf(rw[ir] / RAGGIO);
        fint[ir] = rw[ir] * rw[ir] * rw[ir] * vl[ir] + zvd * e * rw[ir] * rw[ir];
        double check;
        if (!(fabs(rw[ir]) < 1e-8)) check = vl[ir] + zvd * e / rw[ir];
        else check = vl[ir] + 2.0 * zvd / (sqrt(PI_) * RAGGIO);
        if (fabs(check) < 1e-8) fint[ir] = 0.0;
      }
      double dlog = log(rr[mesh - 1] / rr[0]) / (double)(mesh - 1);
      for (int il = 1; il <= ORC_NSPLN; il++) {
        ggnh[il - 1] = (double)(il - 1) * s->gcut_rho / (double)(ORC_NSPLN - 1);
        double xg = sqrt(ggnh[il - 1]) * s->tpiba;
        if (xg > 1e-6) {
          for (int ir = 0; ir < mesh; ir++) {
            double xrg = rw[ir] * xg;
            dfint[ir] = fint[ir] * sin(xrg) / xrg;
          }
        } else
          memcpy(dfint, fint, sizeof(double) * mesh);
        double flx = simpsn(mesh, dfint);
        s->voo[is][il - 1] = dlog * FOURPI_ * flx;
      }
    } else {
      const double *vl = s->vr[is];
      for (int ir = 0; ir < mesh; ir++) fint[ir] = rr[ir] * rr[ir] * vl[ir] + zvd * erf(rr[ir] / RAGGIO) * rr[ir];
      for (int il = 1; il <= ORC_NSPLN; il++) {
        ggnh[il - 1] = (double)(il - 1) * (s->gcut_rho / (double)(ORC_NSPLN - 1));
        double sq = sqrt(ggnh[il - 1]);
        if (sq * s->tpiba > 1e-6) {
          for (int ir = 0; ir < mesh; ir++) {
            double xrg = rr[ir] * sq * s->tpiba;
            dfint[ir] = fint[ir] * sin(xrg) / xrg * rw[ir];
          }
        } else
          for (int ir = 0; ir < mesh; ir++) dfint[ir] = fint[ir] * rw[ir];
        double flx = simpsn(mesh, dfint);
        s->voo[is][il - 1] = FOURPI_ * flx;
      }
    }
    spline_inter(ORC_NSPLN, ggnh, s->voo[is], s->hg, vo, ngrho);
    for (int g = 0; g < ngrho; g++) s->vps[(long)is * ngrho + g] = (1.0 / s->omega) * vo[g];
    for (int g = 0; g < ngrho; g++)
      s->rhos[(long)is * ngrho + g] = -zvd * exp(-(0.25 * (RAGGIO * RAGGIO) * s->hg[g] * s->tpiba2)) * (1.0 / s->omega);
    s->rhos[(long)is * ngrho + 0] = -zvd * (1.0 / s->omega);
    free(fint); free(dfint);
  }
  free(ggnh); free(vo);
}

/* atomic_basis.f90:91-121 (ngh, nghtol, nghcom) for the psp path and
 * readupf.f90:251-352 (NPRO, LPVAL, LFVAL, hlsg) for the UPF path */
static void projector_layout(orc_sys *s) {
  s->nghmax = 1;
  for (int is = 0; is < s->nsp; is++) {
    s->ngh[is] = 0;
    if (!s->upf) {
      orc_species *p = &s->sp[is];
      int iv = 0;
      for (int il = 1; il <= p->lmax; il++) {
        if (il != p->l_local && il != p->skip) {
          int l = il - 1;
          s->ngh[is] += 2 * l + 1;
          if (s->ngh[is] > s->nghmax) s->nghmax = s->ngh[is];
          int ic = (l == 0) ? 0 : l * l;
          for (int j = 1; j <= 2 * l + 1; j++) {
            s->nghtol[is][iv] = l;
            s->nghcom[is][iv] = ic + j;
            iv++;
          }
        }
      }
    } else {
      orc_species *p = &s->sp[is];
      int npro[LMAXX + 1] = {0}, pl1[64], pl2[64];
      for (int nb = 0; nb < p->nbeta; nb++) {
        int l = p->beta_l[nb];
        pl1[nb] = l;
        npro[l + 1]++;
        pl2[nb] = npro[l + 1];
      }
      int iv = 0, lp = 0;
      for (int L = 1; L <= p->upf_lmax; L++)
        for (int M = 1; M <= 2 * L - 1; M++) {
          lp++;
          for (int K = 1; K <= npro[L]; K++) {
            s->nghtol[is][iv] = L - 1;
            s->lpval[is][iv] = lp;
            s->lfval[is][iv] = K;
            s->nghcom[is][iv] = lp;
            iv++;
          }
        }
      s->ngh[is] = iv;
      if (iv > s->nghmax) s->nghmax = iv;
      memset(s->hlsg[is], 0, sizeof(s->hlsg[is]));
      int nb = p->nbeta;
      for (int i = 0; i < nb; i++)
        for (int j = 0; j < nb; j++) {
          if (i != j) continue;
          int l = pl1[i] + 1, a = pl2[i], b2 = pl2[j];
          s->hlsg[is][l - 1][a - 1][b2 - 1] = 0.5 * p->dij[i * nb + j];
          s->hlsg[is][l - 1][b2 - 1][a - 1] = 0.5 * p->dij[i * nb + j];
        }
    }
  }
}

/* pseudopotential.f90:434-529 nlppgrid (psp) and :234-291 upf_nlppgrid */
static void nlppgrid(orc_sys *s) {
  double *ggng = (double *)xcalloc(ORC_NSPLN, sizeof(double));
  for (int is = 0; is < s->nsp; is++) {
    orc_species *p = &s->sp[is];
    int mesh = p->mesh;
    double *rr = s->rr[is], *rw = s->rw[is];
    s->wns[is] = (double *)xcalloc((long)ORC_NSPLN * (s->ngh[is] + 1), sizeof(double));
    double *fnt = (double *)xcalloc(mesh, sizeof(double));
    if (!s->upf) {
      if (!p->tkb) continue;
      /* rps(:,is,1) re-interpolated with the first species' radial grid */
      intrp_grid(s->rr[0], mesh, rw, mesh, s->rps[is]);
      const double *gmax = s->vr[is] + (long)(p->l_local - 1) * mesh;
      double *gnl = (double *)xcalloc((long)(p->lmax + 1) * mesh, sizeof(double));
      double wsgtmp[LMAXX + 2] = {0};
      double loggrid = log(rr[mesh - 1] / rr[0]) / (double)(mesh - 1);
      double wsgl[LMAXX + 2] = {0};
      for (int l = 1; l <= p->lmax; l++) {
        if (l == p->skip || l == p->l_local) { wsgtmp[l] = 0.0; continue; }
        double *g = gnl + (long)l * mesh;
        const double *vl = s->vr[is] + (long)(l - 1) * mesh;
        for (int ir = 0; ir < mesh; ir++) {
          g[ir] = vl[ir] - gmax[ir];
          if (fabs(g[ir]) < 1e-10) g[ir] = 0.0;
        }
        const double *ps = s->rps[is] + (long)(l - 1) * mesh;
        for (int ir = 0; ir < mesh; ir++) fnt[ir] = ps[ir] * ps[ir] * g[ir] * rw[ir];
        wsgl[l] = simpsn(mesh, fnt);
        wsgtmp[l] = 1.0 / (loggrid * wsgl[l]);
      }
      int k = 0;
      for (int l = 1; l <= p->lmax; l++)
        if (l != p->l_local && l != p->skip)
          for (int lm = 1; lm <= 2 * l - 1; lm++) s->wsg[is][k++] = wsgtmp[l];
      for (int il = 1; il <= ORC_NSPLN; il++) ggng[il - 1] = (double)(il - 1) * s->gcut_pw / (double)(ORC_NSPLN - 1);
      int lold = -1;
      for (int iv = 0; iv < s->ngh[is]; iv++) {
        int l = s->nghtol[is][iv] + 1;
        double *w = s->wns[is] + (long)iv * ORC_NSPLN;
        if (l == lold) {
          memcpy(w, w - ORC_NSPLN, sizeof(double) * ORC_NSPLN);
        } else if (l != p->skip) {
          const double *ps = s->rps[is] + (long)(l - 1) * mesh;
          const double *g = gnl + (long)l * mesh;
          for (int il = 0; il < ORC_NSPLN; il++) {
            double xg = sqrt(ggng[il]) * TWOPI_ / s->alat;
            for (int ir = 0; ir < mesh; ir++) {
              double jl = sph_bes(l - 1, xg * rw[ir]);
              fnt[ir] = rw[ir] * rw[ir] * ps[ir] * g[ir] * jl;
            }
            double tmp = simpsn(mesh, fnt);
            w[il] = loggrid * FOURPI_ * tmp;
          }
        }
        lold = l;
      }
      free(gnl);
    } else {
      for (int il = 1; il <= ORC_NSPLN; il++) ggng[il - 1] = (double)(il - 1) * s->gcut_pw / (double)(ORC_NSPLN - 1);
      int lold = -1;
      for (int iv = 0; iv < s->ngh[is]; iv++) {
        int l = s->nghtol[is][iv] + 1;
        double *w = s->wns[is] + (long)iv * ORC_NSPLN;
        if (l == lold) {
          memcpy(w, w - ORC_NSPLN, sizeof(double) * ORC_NSPLN);
        } else {
          /* upf_gnl(:,is,l): the beta indexed by the angular momentum slot */
          const double *bt = s->beta[is] + (long)(l - 1) * mesh;
          for (int il = 0; il < ORC_NSPLN; il++) {
            double xg = sqrt(ggng[il]) * TWOPI_ / s->alat;
            for (int ir = 0; ir < mesh; ir++) {
              double jl = sph_bes(l - 1, xg * rr[ir]);
              fnt[ir] = rw[ir] * rr[ir] * bt[ir] * jl;
            }
            double tmp = simpsn(mesh, fnt);
            w[il] = FOURPI_ * tmp;
          }
        }
        lold = l;
      }
    }
    free(fnt);
  }
  free(ggng);
}

/* pseudopotential.f90:108-162 nlpro and :293-354 upf_nlpro */
static void nlpro(orc_sys *s) {
  int ngpw = s->ngpw;
  s->twnl = (double *)xcalloc((long)ngpw * s->nghmax * s->nsp, sizeof(double));
  double *ggng = (double *)xcalloc(ORC_NSPLN, sizeof(double));
  double *mw = (double *)xcalloc(ngpw, sizeof(double));
  for (int il = 1; il <= ORC_NSPLN; il++) ggng[il - 1] = (double)(il - 1) * s->gcut_pw / (double)(ORC_NSPLN - 1);
  double vol = 1.0 / sqrt(s->omega);
  for (int is = 0; is < s->nsp; is++) {
    if (!s->upf && !s->sp[is].tkb) continue;
    for (int iv = 0; iv < s->ngh[is]; iv++) {
      int lp = s->nghcom[is][iv];
      double *w = s->wns[is] + (long)iv * ORC_NSPLN;
      double xx = 0;
      for (int il = 0; il < ORC_NSPLN; il++) xx += fabs(w[il]);
      memset(mw, 0, sizeof(double) * ngpw);
      spline_inter(ORC_NSPLN, ggng, w, s->hg, mw, ngpw);
      if (xx > 1e-12)
        for (int g = 0; g < ngpw; g++)
          s->twnl[g + (long)ngpw * (iv + (long)s->nghmax * is)] = ylm_one(lp, s->hg[g], s->gvec + 3 * g) * vol * mw[g];
    }
  }
  free(ggng); free(mw);
}

/* exp_igr.f90:4-140 exp_igrxfactor */
static zc cmul(zc a, zc b) {
  double ar = creal(a), ai = cimag(a), br = creal(b), bi = cimag(b);
  return (ar * br - ai * bi) + I * (ar * bi + ai * br);
}
static zc cdiv_smith(zc a, zc b) {
  double ar = creal(a), ai = cimag(a), c = creal(b), d = cimag(b);
  if (fabs(c) >= fabs(d)) {
    double r = d / c, den = c + d * r;
    return ((ar + ai * r) / den) + I * ((ai - ar * r) / den);
  }
  double r = c / d, den = c * r + d;
  return ((ar * r + ai) / den) + I * ((ai * r - ar) / den);
}
static void exp_igrxfactor(orc_sys *s) {
  int ngrho = s->ngrho, nat = s->nat;
  int nr[3] = {s->nr[0], s->nr[1], s->nr[2]}, nh[3];
  for (int d = 0; d < 3; d++) nh[d] = nr[d] / 2 + 1;
  if (!s->eigr) {
    s->eigr = (zc *)xcalloc((long)ngrho * nat, sizeof(zc));
    s->eigrxvps = (zc *)xcalloc(ngrho, sizeof(zc));
    s->eigrxrhos = (zc *)xcalloc(ngrho, sizeof(zc));
  }
  zc *ei[3];
  for (int d = 0; d < 3; d++) ei[d] = (zc *)xcalloc(2 * nr[d], sizeof(zc));
  for (int isa = 0; isa < nat; isa++) {
    int ia = s->isa_ia[isa], is = s->isa_is[isa];
    const double *x = s->atco + 3 * (ia + (long)s->na_max * is);
    for (int d = 1; d <= 3; d++) {
      double sm = A3(s->b_cell, 1, d) * x[0];
      sm = sm + A3(s->b_cell, 2, d) * x[1];
      sm = sm + A3(s->b_cell, 3, d) * x[2];
      double arg = s->tpiba * sm;
      zc *e = ei[d - 1];
      int n = nr[d - 1];
      e[0] = 1.0;
      zc dp = cos(arg) - I * sin(arg), dm = conj(dp);
      zc tp = dp, tm = dm;
      for (int i = 2; i <= n; i++) {
        e[i - 1] = tp;
        tp = cmul(tp, dp);
        e[n + i - 2] = tm;
        tm = cmul(tm, dm);
      }
      zc e0 = cdiv_smith(1.0, e[nh[d - 1] - 1]);
      for (int i = 0; i < 2 * n - 1; i++) e[i] = cmul(e[i], e0);
    }
    for (int g = 0; g < ngrho; g++) {
      zc v = cmul(ei[0][s->inyh[3 * g] - 1], ei[1][s->inyh[3 * g + 1] - 1]);
      s->eigr[g + (long)ngrho * isa] = cmul(v, ei[2][s->inyh[3 * g + 2] - 1]);
    }
  }
  for (int g = 0; g < ngrho; g++) {
    zc vp = 0, rp = 0;
    for (int isa = 0; isa < nat; isa++) {
      int is = s->isa_is[isa];
      zc e = s->eigr[g + (long)ngrho * isa];
      double v = s->vps[(long)is * ngrho + g];
      vp = vp + (creal(e) * v + I * (cimag(e) * v));
      rp = rp + s->rhos[(long)is * ngrho + g] * e;
    }
    s->eigrxvps[g] = vp;
    s->eigrxrhos[g] = rp;
  }
  for (int d = 0; d < 3; d++) free(ei[d]);
}

/* ------------------------------------------------------------------ */
/* fft_interface.f90:33-148 do_fft (ncpu = 1)                          */
/* ------------------------------------------------------------------ */
/* phasen (fft_interface.f90:515-532): multiply by (-1)^(i+j+k+1) on x in
 * 1..nr1, all padded y and z */
static void phasen(orc_sys *s, zc *f) {
  int q1 = s->nrl[0], q2 = s->nrl[1], q3 = s->nrl[2];
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= q3; k++)
    for (int j = 1; j <= q2; j++)
      for (int i = 1; i <= s->nr[0]; i++) {
        long idx = (i - 1) + (long)q1 * ((j - 1) + (long)q2 * (k - 1));
        if ((k + j + i + 1) % 2 != 0) f[idx] = -f[idx];
      }
}

/* sign = -1: backward (G -> r, unscaled); sign = +1: forward (r -> G, 1/N) */
static void do_fft(orc_sys *s, int sign, zc *fz) {
  int q1 = s->nrl[0], q2 = s->nrl[1], q3 = s->nrl[2];
  int l1 = s->nr[0], l2 = s->nr[1], l3 = s->nr[2];
  int nh = s->nhrays;
  zc *w1 = s->w1, *w2 = s->w2;
  long mf = s->max_fft;
  if (sign == -1) {
    /* MLTFFT('N','T',fz,qr1s,m,work1,m,qr1s,lr1s,m): x lines of the rays */
    memset(w1, 0, sizeof(zc) * mf);
    fft_many(&s->pl[0], nh, fz, 1, q1, w1, nh, 1, +1, 1.0);
    /* pack_x2y / all-to-all (identity) / unpack_x2y: scatter rays to (y,z) */
    long mm = (long)q2 * q3;
    memset(w2, 0, sizeof(zc) * mf);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < l1; i++)
      for (int r = 0; r < nh; r++) w2[(long)i * mm + s->msp[r] - 1] = w1[(long)i * nh + r];
    /* MLTFFT('N','T',work2,QR2S,M,work1,M,QR2S,LR2S,M): y lines */
    long M = (long)q1 * q3;
    memset(w1, 0, sizeof(zc) * mf);
    fft_many(&s->pl[1], (int)M, w2, 1, q2, w1, M, 1, +1, 1.0);
    /* MLTFFT('N','T',work1,QR3S,M,fz,M,QR3S,LR3S,M): z lines */
    M = (long)q1 * q2;
    memset(fz, 0, sizeof(zc) * mf);
    fft_many(&s->pl[2], (int)M, w1, 1, q3, fz, M, 1, +1, 1.0);
    phasen(s, fz);
  } else {
    phasen(s, fz);
    long M = (long)q1 * q2;
    memset(w1, 0, sizeof(zc) * mf);
    fft_many(&s->pl[2], (int)M, fz, M, 1, w1, 1, q3, -1, 1.0);
    M = (long)q1 * q3;
    memset(w2, 0, sizeof(zc) * mf);
    fft_many(&s->pl[1], (int)M, w1, M, 1, w2, 1, q2, -1, 1.0);
    long mm = (long)q2 * q3;
    memset(w1, 0, sizeof(zc) * mf);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < l1; i++)
      for (int r = 0; r < nh; r++) w1[(long)i * nh + r] = w2[(long)i * mm + s->msp[r] - 1];
    double scale = 1.0 / (double)(l1 * l2 * l3);
    memset(fz, 0, sizeof(zc) * mf);
    fft_many(&s->pl[0], nh, w1, nh, 1, fz, 1, q1, -1, scale);
  }
}

void orc_fft(orc_sys *s, int sign, double *fz) { do_fft(s, sign, (zc *)fz); }

/* ------------------------------------------------------------------ */
/* density.f90:5-98 eval_density, :128-150 rhor2g                       */
/* ------------------------------------------------------------------ */
void orc_eval_density(orc_sys *s) {
  zc *work = s->wk;
  long nnr1 = s->nnr1;
  int n = s->nstate, ngpw = s->ngpw;
  memset(s->rho, 0, sizeof(double) * nnr1);
  if (s->lsd) memset(s->rho2, 0, sizeof(double) * nnr1);
  for (int id = 1; id <= n; id += 2) {
    int tfcal = 0;
    int ilast = id + 1 <= n ? id + 1 : n;
    for (int i = id; i <= ilast; i++) tfcal = (s->occ[i - 1] != 0.0);
    if (!tfcal) continue;
    memset(work, 0, sizeof(zc) * s->max_fft);
    int is1 = id, is2 = id + 1;
    const zc *c1 = s->c0 + (long)(is1 - 1) * ngpw;
    if (is2 > n) {
      for (int g = 0; g < ngpw; g++) {
        work[s->mapp[g] - 1] = c1[g];
        work[s->mapm[g] - 1] = conj(c1[g]);
      }
      work[s->mapp[0] - 1] = c1[0];
    } else {
      const zc *c2 = s->c0 + (long)(is2 - 1) * ngpw;
      for (int g = 0; g < ngpw; g++) {
        work[s->mapp[g] - 1] = c1[g] + I * c2[g];
        work[s->mapm[g] - 1] = conj(c1[g]) + I * conj(c2[g]);
      }
      work[s->mapp[0] - 1] = c1[0] + I * c2[0];
    }
    do_fft(s, -1, work);
    double coef3 = s->occ[is1 - 1] / s->omega;
    double coef4 = (is2 > n) ? 0.0 : s->occ[is2 - 1] / s->omega;
    /* open shell: each band also adds to the spin-2 density when it is a
       spin-2 band (density.f90:64-76; the total is rho1 + rho2, :94-98) */
    const double w3 = (s->lsd && is1 > s->nel_up) ? 1.0 : 0.0, w4 = (s->lsd && is2 > s->nel_up) ? 1.0 : 0.0;
#pragma omp parallel for schedule(static)
    for (long l = 0; l < nnr1; l++) {
      double r1 = creal(work[l]), r2 = cimag(work[l]);
      double tt = coef3 * r1 * r1 + coef4 * r2 * r2;
      s->rho[l] = s->rho[l] + tt;
      if (s->lsd) s->rho2[l] = s->rho2[l] + (w3 * (coef3 * r1 * r1) + w4 * (coef4 * r2 * r2));
    }
  }
}

void orc_rhor2g(orc_sys *s) {
  zc *work = s->wk;
  memset(work, 0, sizeof(zc) * s->max_fft);
  for (long l = 0; l < s->nnr1; l++) work[l] = s->rho[l];
  do_fft(s, +1, work);
  for (int g = 0; g < s->ngrho; g++) s->rho_g[g] = work[s->mapp[g] - 1];
}

/* potential.f90:4-46 eval_pot */
void orc_eval_pot(orc_sys *s) {
  zc *work = s->wk;
  int ngrho = s->ngrho;
  zc *vt = (zc *)xcalloc(ngrho, sizeof(zc));
  vt[0] = 0.0;
  for (int g = 1; g < ngrho; g++) {
    double f = FOURPI_ / (s->tpiba2 * s->hg[g]);
    zc r = s->rho_g[g] + s->eigrxrhos[g];
    vt[g] = (f * creal(r) + I * (f * cimag(r))) + s->eigrxvps[g];
  }
  memset(work, 0, sizeof(zc) * s->max_fft);
  for (int g = 0; g < ngrho; g++) {
    work[s->mapm[g] - 1] = conj(vt[g]);
    work[s->mapp[g] - 1] = vt[g];
  }
  work[s->mapp[0] - 1] = vt[0];
  do_fft(s, -1, work);
  for (long l = 0; l < s->nnr1; l++) s->v_pot[l] = creal(work[l]);
  /* open shell: both spins start from the same Hartree + local potential (potential.f90:43) */
  if (s->lsd) memcpy(s->v_pot2, s->v_pot, sizeof(double) * s->nnr1);
  free(vt);
}

/* ------------------------------------------------------------------ */
/* exchange-correlation (the libxc functionals named in xc.f90:75-94)   */
/* ------------------------------------------------------------------ */
static void lda_teter93(double rho, double *e, double *v) {
  const double a0 = 0.4581652932831429, a1 = 2.217058676663745, a2 = 0.7405551735357053, a3 = 0.01968227878617998;
  const double b1 = 1.0, b2 = 4.504130959426697, b3 = 1.110667363742916, b4 = 0.02359291751427506;
  double rs = cbrt(3.0 / (FOURPI_ * rho));
  double num = a0 + rs * (a1 + rs * (a2 + rs * a3));
  double den = rs * (b1 + rs * (b2 + rs * (b3 + rs * b4)));
  double dnum = a1 + rs * (2.0 * a2 + rs * 3.0 * a3);
  double dden = b1 + rs * (2.0 * b2 + rs * (3.0 * b3 + rs * 4.0 * b4));
  double eps = -num / den;
  double deps = -(dnum * den - num * dden) / (den * den);
  *e = rho * eps;
  *v = eps - rs / 3.0 * deps;
}
/* libxc XC_LDA_XC_TETER93 spin polarized (Goedecker, Teter and Hutter,
   Phys. Rev. B 54, 1703 (1996)): the Pade form above with every coefficient
   c = c(unpolarized) + f(zeta) dc, f(zeta) = ((1+zeta)^(4/3) + (1-zeta)^(4/3)
   - 2) / (2^(4/3) - 2).  e = rho eps, va = d(rho eps)/d rho_a,
   vb = d(rho eps)/d rho_b (d zeta/d rho_a = (1 - zeta)/rho, d zeta/d rho_b =
   -(1 + zeta)/rho). */
static void lda_teter93_pol(double ra, double rb, double *e, double *va, double *vb) {
  const double a[4] = {0.4581652932831429, 2.217058676663745, 0.7405551735357053, 0.01968227878617998};
  const double b[4] = {1.0, 4.504130959426697, 1.110667363742916, 0.02359291751427506};
  const double da[4] = {0.119086804055547, 0.6157402568883345, 0.1574201515892867, 0.003532336663397157};
  const double db[4] = {0.0, 0.2673612973836267, 0.2052004607777787, 0.004200005045691381};
  double rho = ra + rb;
  double z = (ra - rb) / rho;
  if (z > 1.0) z = 1.0;
  if (z < -1.0) z = -1.0;
  const double fden = cbrt(16.0) - 2.0; /* 2^(4/3) - 2 */
  double cp = cbrt(1.0 + z), cm = cbrt(1.0 - z);
  double f = ((1.0 + z) * cp + (1.0 - z) * cm - 2.0) / fden;
  double df = 4.0 / 3.0 * (cp - cm) / fden;
  double A[4], B[4];
  for (int i = 0; i < 4; i++) { A[i] = a[i] + f * da[i]; B[i] = b[i] + f * db[i]; }
  double rs = cbrt(3.0 / (FOURPI_ * rho));
  double num = A[0] + rs * (A[1] + rs * (A[2] + rs * A[3]));
  double den = rs * (B[0] + rs * (B[1] + rs * (B[2] + rs * B[3])));
  double dnum = A[1] + rs * (2.0 * A[2] + rs * 3.0 * A[3]);
  double dden = B[0] + rs * (2.0 * B[1] + rs * (3.0 * B[2] + rs * 4.0 * B[3]));
  double nf = da[0] + rs * (da[1] + rs * (da[2] + rs * da[3]));
  double df_den = rs * (db[0] + rs * (db[1] + rs * (db[2] + rs * db[3])));
  double eps = -num / den;
  double deps_drs = -(dnum * den - num * dden) / (den * den);
  double deps_dz = -(nf * den - num * df_den) / (den * den) * df;
  *e = rho * eps;
  *va = eps - rs / 3.0 * deps_drs + deps_dz * (1.0 - z);
  *vb = eps - rs / 3.0 * deps_drs - deps_dz * (1.0 + z);
}
static void lda_slater(double rho, double *e, double *v) {
  double ex = -0.75 * cbrt(3.0 / PI_) * cbrt(rho);
  *e = rho * ex;
  *v = 4.0 / 3.0 * ex;
}
static void lda_pz81(double rho, double *e, double *v) {
  double rs = cbrt(3.0 / (FOURPI_ * rho)), eps, deps;
  if (rs >= 1.0) {
    const double g = -0.1423, b1 = 1.0529, b2 = 0.3334;
    double sq = sqrt(rs), den = 1.0 + b1 * sq + b2 * rs;
    eps = g / den;
    deps = -g * (0.5 * b1 / sq + b2) / (den * den);
  } else {
    const double A = 0.0311, B = -0.048, C = 0.0020, D = -0.0116;
    double lr = log(rs);
    eps = A * lr + B + C * rs * lr + D * rs;
    deps = A / rs + C * lr + C + D;
  }
  *e = rho * eps;
  *v = eps - rs / 3.0 * deps;
}
static void pw92_unpol(double rs, double *ec, double *dec) {
  const double A = 0.0310907, a1 = 0.21370, b1 = 7.5957, b2 = 3.5876, b3 = 1.6382, b4 = 0.49294;
  double sq = sqrt(rs);
  double q = 2.0 * A * (b1 * sq + b2 * rs + b3 * rs * sq + b4 * rs * rs);
  double dq = 2.0 * A * (0.5 * b1 / sq + b2 + 1.5 * b3 * sq + 2.0 * b4 * rs);
  double L = log(1.0 + 1.0 / q);
  double dL = -dq / (q * q + q);
  *ec = -2.0 * A * (1.0 + a1 * rs) * L;
  *dec = -2.0 * A * a1 * L - 2.0 * A * (1.0 + a1 * rs) * dL;
}
static void gga_pbe(double rho, double sigma, double *e, double *v, double *vs) {
  const double kappa = 0.804, mu = 0.2195149727645171;
  const double beta = 0.06672455060314922;
  const double gamma = (1.0 - log(2.0)) / (PI_ * PI_);
  double kf = cbrt(3.0 * PI_ * PI_ * rho);
  /* exchange */
  double exu = -3.0 / (FOURPI_)*kf * rho;
  double s2 = sigma / (4.0 * kf * kf * rho * rho);
  double den = 1.0 + mu * s2 / kappa;
  double Fx = 1.0 + kappa - kappa / den;
  double dF = mu / (den * den);
  double ex = exu * Fx;
  double vx = 4.0 / 3.0 * exu / rho * Fx + exu * dF * (-8.0 / 3.0 * s2 / rho);
  double vsx = exu * dF / (4.0 * kf * kf * rho * rho);
  /* correlation */
  double rs = cbrt(3.0 / (FOURPI_ * rho));
  double ec, dec;
  pw92_unpol(rs, &ec, &dec);
  double t2 = PI_ * sigma / (16.0 * kf * rho * rho);
  double bg = beta / gamma;
  double E = exp(-ec / gamma);
  double A = bg / (E - 1.0);
  double At2 = A * t2;
  double num = 1.0 + At2, dd = 1.0 + At2 + At2 * At2;
  double Q = t2 * num / dd;
  double H = gamma * log(1.0 + bg * Q);
  double dHdQ = beta / (1.0 + bg * Q);
  double dQdt2 = (num + t2 * A) / dd - t2 * num * (A + 2.0 * A * A * t2) / (dd * dd);
  double dQdA = (t2 * t2) / dd - t2 * num * (t2 + 2.0 * A * t2 * t2) / (dd * dd);
  double dAdec = bg * E / (gamma * (E - 1.0) * (E - 1.0));
  double decdrho = dec * (-rs / (3.0 * rho));
  double dt2drho = -7.0 / 3.0 * t2 / rho;
  double vc = ec + H + rho * (decdrho + dHdQ * dQdA * dAdec * decdrho + dHdQ * dQdt2 * dt2drho);
  double vsc = rho * dHdQ * dQdt2 * PI_ / (16.0 * kf * rho * rho);
  *e = ex + rho * (ec + H);
  *v = vx + vc;
  *vs = vsx + vsc;
}

void orc_xc_point(int xc, double rho, double sigma, double *e, double *v, double *vs) {
  *e = 0; *v = 0; *vs = 0;
  if (!(rho > 1e-30)) return;
  if (xc == ORC_XC_TETER93) {
    lda_teter93(rho, e, v);
  } else if (xc == ORC_XC_PZ) {
    double e1, v1, e2, v2;
    lda_slater(rho, &e1, &v1);
    lda_pz81(rho, &e2, &v2);
    *e = e1 + e2;
    *v = v1 + v2;
  } else {
    gga_pbe(rho, sigma, e, v, vs);
  }
}

/* xc.f90:436-497 GRAD_CAL */
static void grad_cal(orc_sys *s, const double *ro, double *grad) {
  long nnr1 = s->nnr1;
  int ngrho = s->ngrho;
  zc *work = s->wk;
  zc *tmp = (zc *)xcalloc(ngrho, sizeof(zc));
  memset(work, 0, sizeof(zc) * s->max_fft);
  for (long l = 0; l < nnr1; l++) work[l] = ro[l];
  do_fft(s, +1, work);
  for (int g = 0; g < ngrho; g++) tmp[g] = work[s->mapp[g] - 1];
  memset(work, 0, sizeof(zc) * s->max_fft);
  for (int g = 0; g < ngrho; g++) {
    double gx = s->tpiba * s->gvec[3 * g];
    work[s->mapp[g] - 1] = tmp[g] - gx * tmp[g];
    work[s->mapm[g] - 1] = conj(tmp[g] + gx * tmp[g]);
  }
  do_fft(s, -1, work);
  for (long l = 0; l < nnr1; l++) {
    grad[l] = cimag(work[l]) * cimag(work[l]);
    grad[l + nnr1] = cimag(work[l]);
  }
  memset(work, 0, sizeof(zc) * s->max_fft);
  for (int g = 0; g < ngrho; g++) {
    double gy = s->gvec[3 * g + 1], gz = s->gvec[3 * g + 2];
    zc f1 = s->tpiba * (I * gy - gz);
    zc f2 = s->tpiba * (-I * gy + gz);
    work[s->mapp[g] - 1] = f1 * tmp[g];
    work[s->mapm[g] - 1] = f2 * conj(tmp[g]);
  }
  do_fft(s, -1, work);
  for (long l = 0; l < nnr1; l++) {
    grad[l] = grad[l] + creal(work[l] * conj(work[l]));
    grad[l + 2 * nnr1] = creal(work[l]);
    grad[l + 3 * nnr1] = cimag(work[l]);
  }
  free(tmp);
}

/* the G-space assembly of one potential (xc.f90:252-301 closed shell,
   :302-425 per spin): vp = band limit of [vp + v1 - i G.(v2 grad rho)] */
static void assemble_v(orc_sys *s, double *vp, const double *v1, const double *v2, const double *grad) {
  long nnr1 = s->nnr1;
  int ngrho = s->ngrho;
  int gga = v2 != NULL;
  zc *work = s->wk;
  zc *vpotg = (zc *)xcalloc(ngrho, sizeof(zc));
  memset(work, 0, sizeof(zc) * s->max_fft);
  for (long l = 0; l < nnr1; l++) work[l] = vp[l];
  do_fft(s, +1, work);
  for (int g = 0; g < ngrho; g++) vpotg[g] = work[s->mapp[g] - 1];
  memset(work, 0, sizeof(zc) * s->max_fft);
  for (long l = 0; l < nnr1; l++) work[l] = v1[l] + I * (gga ? v2[l] * grad[l + nnr1] : 0.0);
  do_fft(s, +1, work);
  for (int g = 0; g < ngrho; g++) {
    double vfac = s->tpiba * s->gvec[3 * g];
    zc fp = work[s->mapp[g] - 1], fm = work[s->mapm[g] - 1];
    zc fa = fp + fm, fb = fp - fm;
    zc vg1 = 0.5 * (creal(fa) + I * cimag(fb));
    zc vg2 = 0.5 * (cimag(fa) - I * creal(fb));
    vpotg[g] = vpotg[g] + vg1 - (-vfac * cimag(vg2) + I * (vfac * creal(vg2)));
  }
  if (gga) {
    memset(work, 0, sizeof(zc) * s->max_fft);
    for (long l = 0; l < nnr1; l++) work[l] = v2[l] * grad[l + 2 * nnr1] + I * (v2[l] * grad[l + 3 * nnr1]);
    do_fft(s, +1, work);
    for (int g = 0; g < ngrho; g++) {
      double vf2 = s->tpiba * s->gvec[3 * g + 1], vf3 = s->tpiba * s->gvec[3 * g + 2];
      zc fp = work[s->mapp[g] - 1], fm = work[s->mapm[g] - 1];
      zc fa = fp + fm, fb = fp - fm;
      zc vg1 = 0.5 * (creal(fa) + I * cimag(fb));
      zc vg2 = 0.5 * (cimag(fa) - I * creal(fb));
      vpotg[g] = vpotg[g] - (-vf2 * cimag(vg1) + I * (vf2 * creal(vg1))) - (-vf3 * cimag(vg2) + I * (vf3 * creal(vg2)));
    }
  }
  memset(work, 0, sizeof(zc) * s->max_fft);
  for (int g = 0; g < ngrho; g++) {
    work[s->mapp[g] - 1] = vpotg[g];
    work[s->mapm[g] - 1] = conj(vpotg[g]);
  }
  do_fft(s, -1, work);
  for (long l = 0; l < nnr1; l++) vp[l] = creal(work[l]);
  free(vpotg);
}

/* smoothing of the functional near zero density (xc.f90:100-130, :196-236) */
static void smoothing(double rt, double *smoo, double *dsmoo) {
  if (rt > 4.0 * GC_CUTOFF) { *smoo = 1.0; *dsmoo = 0.0; return; }
  double texp = exp(3.0 * (1.0 - rt / GC_CUTOFF));
  *smoo = 1.0 / (1.0 + texp);
  *dsmoo = 3.0 / GC_CUTOFF * texp * (*smoo) * (*smoo);
}

/* xc.f90:4-434 cal_vpot_ex: closed shell (:64-131) or, open shell, the
   polarized LDA branch (:135-246) with rho_a = rho - rho2, rho_b = rho2 */
void orc_cal_vpot_ex(orc_sys *s) {
  long nnr1 = s->nnr1;
  int gga = (s->xc == ORC_XC_PBE) && !s->lsd;
  double *grad = s->grad;
  if (gga) grad_cal(s, s->rho, grad);
  double *v1 = (double *)xcalloc(nnr1, sizeof(double)), *v2 = (double *)xcalloc(nnr1, sizeof(double));
  double *v1b = s->lsd ? (double *)xcalloc(nnr1, sizeof(double)) : NULL;
  double *sxa = (double *)xcalloc(nnr1, sizeof(double));
#pragma omp parallel for schedule(static)
  for (long i = 0; i < nnr1; i++) {
    if (s->lsd) {
      double ra = s->rho[i] - s->rho2[i], rb = s->rho2[i];
      double pa = ra > 0.0 ? ra : 0.0, pb = rb > 0.0 ? rb : 0.0;
      double e = 0, va = 0, vb = 0;
      if (pa + pb > 1e-30) lda_teter93_pol(pa, pb, &e, &va, &vb);
      double rt = pa + pb, sm = 0, a = 0, b = 0;
      if (rt > 0.1 * GC_CUTOFF) {
        double smoo, dsmoo;
        smoothing(rt, &smoo, &dsmoo);
        sm = smoo * e;
        a = dsmoo * e + smoo * va;
        b = dsmoo * e + smoo * vb;
      }
      sxa[i] = sm;
      v1[i] = a;
      v1b[i] = b;
      continue;
    }
    double e, v, vs;
    orc_xc_point(s->xc, s->rho[i], gga ? grad[i] : 0.0, &e, &v, &vs);
    double rt = s->rho[i] > 0.0 ? s->rho[i] : 0.0;
    double v1_ = 0, v2_ = 0, sm = 0;
    if (rt > 0.1 * GC_CUTOFF) {
      double smoo, dsmoo;
      smoothing(rt, &smoo, &dsmoo);
      sm = smoo * e;
      v1_ = dsmoo * e + smoo * v;
      v2_ = smoo * (2.0 * vs);
    }
    sxa[i] = sm;
    v1[i] = v1_;
    v2[i] = v2_;
  }
  double sgcx = 0.0;
  for (long i = 0; i < nnr1; i++) sgcx = sgcx + sxa[i];
  s->etxc = sgcx;
  assemble_v(s, s->v_pot, v1, gga ? v2 : NULL, grad);
  if (s->lsd) assemble_v(s, s->v_pot2, v1b, NULL, grad);
  free(v1); free(v2); free(v1b); free(sxa);
}

/* ------------------------------------------------------------------ */
/* pseudopotential.f90:3-103 pp_energy, :164-226 fnl, :356-433 upf_fnl  */
/* ------------------------------------------------------------------ */
static zc mi_pow(int l) { /* (0,-1)**l */
  switch (((l % 4) + 4) % 4) { case 0: return 1.0; case 1: return -I; case 2: return -1.0; default: return I; }
}

static void fnl(orc_sys *s) {
  int ngpw = s->ngpw, n = s->nstate, nat = s->nat, ngrho = s->ngrho;
  memset(s->nl, 0, sizeof(double) * (long)nat * s->nghmax * n);
  int isa0 = 0;
  double *scr = (double *)xcalloc(2L * ngpw, sizeof(double));
  for (int is = 0; is < s->nsp; is++) {
    for (int iv = 0; iv < s->ngh[is]; iv++) {
      zc ci = mi_pow(s->nghtol[is][iv]);
      const double *tw = s->twnl + (long)ngpw * (iv + (long)s->nghmax * is);
      for (int ia = 0; ia < s->na[is]; ia++) {
        int isa = isa0 + ia;
        const zc *e = s->eigr + (long)ngrho * isa;
        for (int g = 0; g < ngpw; g++) {
          double er = creal(e[g]), ei = cimag(e[g]);
          if (fabs(creal(ci)) > 0.5) {
            double t = tw[g] * creal(ci);
            scr[2 * g] = t * er; scr[2 * g + 1] = t * ei;
          } else {
            double t = tw[g] * cimag(ci);
            scr[2 * g] = -t * ei; scr[2 * g + 1] = t * er;
          }
        }
        scr[0] *= 0.5; scr[1] *= 0.5;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) {
          const double *c = (const double *)(s->c0 + (long)i * ngpw);
          double acc = 0;
          for (long k = 0; k < 2L * ngpw; k++) acc += scr[k] * c[k];
          s->nl[isa + (long)nat * (iv + (long)s->nghmax * i)] = 2.0 * acc;
        }
      }
    }
    isa0 += s->na[is];
  }
  free(scr);
}

void orc_pp_energy(orc_sys *s) {
  zc el = 0.5 * s->eigrxvps[0] * conj(s->rho_g[0]);
  for (int g = 1; g < s->ngrho; g++) el = el + s->eigrxvps[g] * conj(s->rho_g[g]);
  s->eloc = 2.0 * creal(el) * s->omega;
  fnl(s);
  int nat = s->nat, n = s->nstate;
  double enl = 0.0;
  int isa0 = 0;
  for (int is = 0; is < s->nsp; is++) {
    if (!s->upf) {
      for (int iv = 0; iv < s->ngh[is]; iv++) {
        double sum = 0.0;
        for (int i = 0; i < n; i++)
          for (int ia = 0; ia < s->na[is]; ia++) {
            double x = s->nl[isa0 + ia + (long)nat * (iv + (long)s->nghmax * i)];
            sum = sum + s->occ[i] * 1 * x * x;
          }
        enl = enl + s->wsg[is][iv] * sum;
      }
    } else {
      for (int iv = 0; iv < s->ngh[is]; iv++) {
        int l = s->nghtol[is][iv] + 1, ki = s->lfval[is][iv], li = s->lpval[is][iv];
        for (int jv = iv; jv < s->ngh[is]; jv++) {
          int l2 = s->nghtol[is][jv] + 1, lj = s->lpval[is][jv];
          if (l2 == l && li == lj) {
            int kj = s->lfval[is][jv];
            double sum = 0.0;
            for (int i = 0; i < n; i++) {
              if (s->occ[i] == 0.0) continue;
              for (int ia = 0; ia < s->na[is]; ia++) {
                int isa = isa0 + ia;
                sum = sum + s->occ[i] * s->nl[isa + (long)nat * (iv + (long)s->nghmax * i)] *
                                s->nl[isa + (long)nat * (jv + (long)s->nghmax * i)];
              }
            }
            if (iv != jv) sum = 2.0 * sum;
            enl = enl + sum * s->hlsg[is][l - 1][ki - 1][kj - 1];
          }
        }
      }
    }
    isa0 += s->na[is];
  }
  s->enl = enl;
}

/* ------------------------------------------------------------------ */
/* total_energy.f90                                                     */
/* ------------------------------------------------------------------ */
/* apply_pbc.f90:1-40 (cubic, fcc) with M = 1 */
static void apply_pbc(orc_sys *s, double x1, double y1, double z1, double *x2, double *y2, double *z2) {
  double A = s->alat;
  if (s->symmetry == 1) {
    double aby2 = A / 2.0;
    double X = fmod(x1, A), Y = fmod(y1, A), Z = fmod(z1, A);
    X = X - A * trunc(X / aby2);
    Y = Y - A * trunc(Y / aby2);
    Z = Z - A * trunc(Z / aby2);
    *x2 = X; *y2 = Y; *z2 = Z;
  } else if (s->symmetry == 2) {
    double m_a = 1 * A * sqrt(2.0) / 4.0, s2 = sqrt(2.0);
    double x2t = (x1 + y1) / s2, y2t = (-x1 + y1) / s2;
    double X = x2t, Y = y2t;
    X = fmod(X, 2.0 * m_a);
    Y = fmod(Y, 2.0 * m_a);
    double Z = fmod(z1, 2.0 * m_a * s2);
    X = X - 2.0 * m_a * trunc(X / m_a);
    Y = Y - 2.0 * m_a * trunc(Y / m_a);
    Z = Z - 2.0 * m_a * s2 * trunc(Z / (s2 * m_a));
    if (!(fabs(X) + fabs(Y) + s2 * fabs(Z) < 2.0 * m_a)) {
      X = X - copysign(m_a, X);
      Y = Y - copysign(m_a, Y);
      Z = Z - copysign(s2 * m_a, Z);
    }
    double xt = (X - Y) / s2;
    Y = (X + Y) / s2;
    X = xt;
    *x2 = X; *y2 = Y; *z2 = Z;
  } else {
    fprintf(stderr, "oracle: apply_pbc for symmetry %d is not restated\n", s->symmetry);
    abort();
  }
}

/* total_energy.f90:133-239 e_sr (nlp = 0) */
void orc_e_sr(orc_sys *s, int tfor) {
  double *F = s->force;
  memset(F, 0, sizeof(double) * 3 * s->na_max * s->nsp);
  double esr = 0.0;
  for (int k = 0; k < s->nsp; k++)
    for (int j = k; j < s->nsp; j++) {
      double zv2 = (double)(s->zv[k] * s->zv[j]);
      if (fabs(zv2) < 1e-10) continue;
      double rckj = sqrt(RAGGIO * RAGGIO + RAGGIO * RAGGIO);
      for (int l = 0; l < s->na[k]; l++) {
        int inf = (k == j) ? l : 0;
        for (int m = inf; m < s->na[j]; m++) {
          if (l == m && k == j) continue; /* tzero with nlp = 0: no image */
          const double *xl = s->atco + 3 * (l + (long)s->na_max * k);
          const double *xm = s->atco + 3 * (m + (long)s->na_max * j);
          double xlm, ylm, zlm;
          apply_pbc(s, xl[0] - xm[0], xl[1] - xm[1], xl[2] - xm[2], &xlm, &ylm, &zlm);
          double erre2 = xlm * xlm + ylm * ylm + zlm * zlm;
          double rlm = sqrt(erre2);
          double arg = rlm / rckj;
          if (arg <= 20.0) {
            double addesr = zv2 * erfc(arg) / rlm;
            esr = esr + addesr * 1.0;
            if (tfor) {
              double addpre = (2.0 * zv2 / sqrt(PI_)) * exp(-arg * arg) / rckj;
              double repand = 1.0 * (addesr + addpre) / erre2;
              double *fl = F + 3 * (l + (long)s->na_max * k), *fm = F + 3 * (m + (long)s->na_max * j);
              fl[0] += repand * xlm; fl[1] += repand * ylm; fl[2] += repand * zlm;
              fm[0] -= repand * xlm; fm[1] -= repand * ylm; fm[2] -= repand * zlm;
            }
          }
        }
      }
    }
  s->esr = esr;
}

void orc_e_total(orc_sys *s) {
  /* e_hartree */
  zc eh = 0.0;
  for (int g = 1; g < s->ngrho; g++) {
    zc r = s->rho_g[g] + s->eigrxrhos[g];
    double f = FOURPI_ / (s->tpiba2 * s->hg[g]);
    eh = eh + (f * r) * conj(r);
  }
  s->eh_re = creal(eh);
  double es = 0.0;
  for (int is = 0; is < s->nsp; is++) es = es + (double)s->na[is] * s->zv[is] * s->zv[is] / RAGGIO;
  es = es / sqrt(2.0 * PI_);
  s->eself = es;
  orc_e_sr(s, s->tfor);
  s->estat = (creal(eh) * s->omega) + s->esr - s->eself;
  /* e_ke */
  double eke = 0.0;
  for (int i = 0; i < s->nstate; i++) {
    double ek = 0.0;
    const zc *c = s->c0 + (long)i * s->ngpw;
    for (int g = 0; g < s->ngpw; g++) ek = ek + s->hg[g] * (creal(c[g]) * creal(c[g]) + cimag(c[g]) * cimag(c[g]));
    eke = eke + ek * s->occ[i];
  }
  s->eke = eke * s->tpiba2;
  /* e_xc */
  s->exc = s->omega / (double)(s->nr[0] * s->nr[1] * s->nr[2]) * s->etxc;
  s->etotal = s->enl + s->eloc + s->eke + s->exc + s->estat;
}

/* ------------------------------------------------------------------ */
/* wfn_initialize.f90:268-365 vpsi                                      */
/* ------------------------------------------------------------------ */
void orc_vpsi(orc_sys *s) {
  int n = s->nstate, ngpw = s->ngpw;
  long nnr1 = s->nnr1;
  zc *psy = s->wk;
  for (int ia = 1; ia <= n; ia += 2) {
    memset(psy, 0, sizeof(zc) * s->max_fft);
    int is1 = ia, is2 = ia + 1;
    const zc *ca = s->c0 + (long)(is1 - 1) * ngpw;
    const zc *cb = (is2 <= n) ? s->c0 + (long)(is2 - 1) * ngpw : NULL;
    if (is2 > n) {
      for (int g = 0; g < ngpw; g++) {
        psy[s->mapp[g] - 1] = ca[g];
        psy[s->mapm[g] - 1] = conj(ca[g]);
      }
      psy[s->mapp[0] - 1] = ca[0];
    } else {
      for (int g = 0; g < ngpw; g++) {
        psy[s->mapp[g] - 1] = ca[g] + I * cb[g];
        psy[s->mapm[g] - 1] = conj(ca[g]) + I * conj(cb[g]);
      }
      psy[s->mapp[0] - 1] = ca[0] + I * cb[0];
    }
    do_fft(s, -1, psy);
    if (s->lsd) {
      /* open shell (wfn_initialize.f90:313-326): each band of the pair with
         its own spin's potential (V_1 on Re, V_2 on Im for the pair that
         straddles the spins) */
      const double *va = is1 > s->nel_up ? s->v_pot2 : s->v_pot;
      const double *vb = is2 > s->nel_up ? s->v_pot2 : s->v_pot;
#pragma omp parallel for schedule(static)
      for (long l = 0; l < nnr1; l++) psy[l] = va[l] * creal(psy[l]) + I * (vb[l] * cimag(psy[l]));
    } else {
#pragma omp parallel for schedule(static)
      for (long l = 0; l < nnr1; l++) psy[l] = s->v_pot[l] * psy[l];
    }
    do_fft(s, +1, psy);
    double fi = s->occ[is1 - 1] * 0.5;
    if (fi == 0.0) fi = 1.0;
    double fip1 = 0.0;
    if (is2 <= n) fip1 = s->occ[is2 - 1] * 0.5;
    if (fip1 == 0.0) fip1 = 1.0;
    zc *c2a = s->c2 + (long)(is1 - 1) * ngpw;
    zc *c2b = (is2 <= n) ? s->c2 + (long)(is2 - 1) * ngpw : NULL;
    for (int g = 0; g < ngpw; g++) {
      zc pp = psy[s->mapp[g] - 1], pm = psy[s->mapm[g] - 1];
      zc fp = pp + pm, fm = pp - pm;
      double kin = s->tpiba2 * s->hg[g];
      c2a[g] = -fi * (kin * ca[g] + (creal(fp) + I * cimag(fm)));
      if (is2 <= n) c2b[g] = -fip1 * (kin * cb[g] + (cimag(fp) - I * creal(fm)));
    }
  }
}

/* wfn_initialize.f90:560-612 FNONLOC and :614-695 UPF_FNONLOC */
void orc_fnonloc(orc_sys *s) {
  int ngpw = s->ngpw, n = s->nstate, nat = s->nat, ngrho = s->ngrho;
  zc *c2l = (zc *)xcalloc((long)ngpw * n, sizeof(zc));
  int isa0 = 0;
  for (int is = 0; is < s->nsp; is++) {
    for (int iv = 0; iv < s->ngh[is]; iv++) {
      double *ddia = (double *)xcalloc((long)s->na[is] * n, sizeof(double));
      if (!s->upf) {
        for (int i = 0; i < n; i++)
          for (int ia = 0; ia < s->na[is]; ia++)
            ddia[ia + (long)s->na[is] * i] = s->nl[isa0 + ia + (long)nat * (iv + (long)s->nghmax * i)];
      } else {
        int l = s->nghtol[is][iv] + 1, ki = s->lfval[is][iv], li = s->lpval[is][iv];
        for (int jv = 0; jv < s->ngh[is]; jv++) {
          int l2 = s->nghtol[is][jv] + 1, lj = s->lpval[is][jv];
          if (l == l2 && li == lj) {
            int kj = s->lfval[is][jv];
            for (int i = 0; i < n; i++)
              for (int ia = 0; ia < s->na[is]; ia++)
                ddia[ia + (long)s->na[is] * i] += s->nl[isa0 + ia + (long)nat * (jv + (long)s->nghmax * i)] *
                                                   s->hlsg[is][l - 1][ki - 1][kj - 1];
          }
        }
      }
      const double *tw = s->twnl + (long)ngpw * (iv + (long)s->nghmax * is);
      zc ci = mi_pow(s->nghtol[is][iv]);
#pragma omp parallel for schedule(static)
      for (int i = 0; i < n; i++) {
        double ffi = s->occ[i];
        if (ffi < 1e-5) ffi = 1.0;
        zc ctm;
        if (!s->upf) ctm = ci * (-ffi * s->wsg[is][iv]);
        else ctm = ci * (-ffi);
        for (int g = 0; g < ngpw; g++) {
          zc au = 0;
          for (int ia = 0; ia < s->na[is]; ia++) au += s->eigr[g + (long)ngrho * (isa0 + ia)] * ddia[ia + (long)s->na[is] * i];
          if (!s->upf) {
            au = ctm * au;
            c2l[g + (long)ngpw * i] += tw[g] * au;
          } else if (fabs(creal(ctm)) > 0.01) {
            double t1 = tw[g] * creal(ctm);
            c2l[g + (long)ngpw * i] += t1 * creal(au) + I * (t1 * cimag(au));
          } else {
            double t1 = tw[g] * cimag(ctm);
            c2l[g + (long)ngpw * i] += -t1 * cimag(au) + I * (t1 * creal(au));
          }
        }
      }
      free(ddia);
    }
    isa0 += s->na[is];
  }
  for (long k = 0; k < (long)ngpw * n; k++) s->c2[k] += c2l[k];
  free(c2l);
}

/* ------------------------------------------------------------------ */
/* gradient.f90:5-61 forces, eval_GMAX                                 */
/* ------------------------------------------------------------------ */
/* A(i,j) = 2 Re<a_i|b_j> - Re a_i(G0) Re b_j(G0)   (OVLAP_D) */
static void ovlap_d(orc_sys *s, const zc *ca, const zc *cb, double *A) {
  int n = s->nstate, ngpw = s->ngpw;
#pragma omp parallel for schedule(static) collapse(2)
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) {
      const double *a = (const double *)(ca + (long)i * ngpw), *b = (const double *)(cb + (long)j * ngpw);
      double acc = 0;
      for (long k = 0; k < 2L * ngpw; k++) acc += a[k] * b[k];
      A[i + (long)n * j] = 2.0 * acc - a[0] * b[0];
    }
}

/* open shell: the overlap matrices are block diagonal by spin (OVLAP_D and
   ortho_gs each take the spin-1 and spin-2 blocks separately,
   wfn_initialize.f90:245-253,458-477) */
static void spin_mask(orc_sys *s, double *A) {
  if (!s->lsd) return;
  int n = s->nstate;
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++)
      if ((i < s->nel_up) != (j < s->nel_up)) A[i + (long)n * j] = 0.0;
}

static void eval_gmax(orc_sys *s, double gcut) {
  int nocc = 0;
  for (int i = 0; i < s->nstate; i++) if (s->occ[i] > 1e-5) nocc++;
  double xmax = -1.0;
  for (long k = 0; k < (long)nocc * s->ngpw; k++) {
    double y = cabs(s->c2[k]);
    if (y > xmax) xmax = y;
  }
  s->gemax = xmax;
  s->convwf = s->gemax < gcut;
}

void orc_forces(orc_sys *s) {
  int n = s->nstate, ngpw = s->ngpw;
  double *gam = (double *)xcalloc((long)n * n, sizeof(double));
  ovlap_d(s, s->c2, s->c0, gam);
  spin_mask(s, gam);
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) {
      double fi = s->occ[i] == 0.0 ? 0.0 : 1.0, fj = s->occ[j] == 0.0 ? 0.0 : 1.0;
      gam[i + (long)n * j] = fi * fj * gam[i + (long)n * j];
    }
#pragma omp parallel for schedule(static)
  for (int j = 0; j < n; j++) {
    double *c2 = (double *)(s->c2 + (long)j * ngpw);
    for (int i = 0; i < n; i++) {
      const double *c0 = (const double *)(s->c0 + (long)i * ngpw);
      double g = gam[i + (long)n * j];
      for (long k = 0; k < 2L * ngpw; k++) c2[k] -= c0[k] * g;
    }
  }
  for (int i = 0; i < n; i++) s->c2[(long)i * ngpw] = creal(s->c2[(long)i * ngpw]);
  free(gam);
}

/* ------------------------------------------------------------------ */
/* nuclear_grad.f90:4-50 POTFOR, :51-89 NLFOR, :314-372 D_FNL,          */
/* :153-199 UPF_NLFOR                                                   */
/* ------------------------------------------------------------------ */
void orc_potfor(orc_sys *s) {
  int ngrho = s->ngrho;
  double omtp = 2.0 * s->omega * s->tpiba;
  for (int isa = 0; isa < s->nat; isa++) {
    int is = s->isa_is[isa], ia = s->isa_ia[isa];
    double fx = 0, fy = 0, fz = 0;
    for (int g = 1; g < ngrho; g++) {
      zc rp = s->eigrxrhos[g], rhet = s->rho_g[g];
      zc rhog = rhet + rp;
      double f = FOURPI_ / (s->tpiba2 * s->hg[g]);
      zc vcgs = f * conj(rhog);
      zc base = s->rhos[(long)is * ngrho + g] * vcgs + s->vps[(long)is * ngrho + g] * conj(rhet);
      zc e = s->eigr[g + (long)ngrho * isa];
      zc eb = e * base;
      /* Re(eigr * base * i g) = -Im(eigr*base) * g */
      fx += -cimag(eb) * s->gvec[3 * g] * omtp;
      fy += -cimag(eb) * s->gvec[3 * g + 1] * omtp;
      fz += -cimag(eb) * s->gvec[3 * g + 2] * omtp;
    }
    double *F = s->force + 3 * (ia + (long)s->na_max * is);
    F[0] += fx; F[1] += fy; F[2] += fz;
  }
}

static void d_fnl(orc_sys *s) {
  int ngpw = s->ngpw, n = s->nstate, nat = s->nat, ngrho = s->ngrho;
  double tfac = 2.0 * s->tpiba;
  double *scr = (double *)xcalloc(2L * ngpw, sizeof(double));
  for (int k = 0; k < 3; k++) {
    int isa0 = 0;
    for (int is = 0; is < s->nsp; is++) {
      for (int iv = 0; iv < s->ngh[is]; iv++) {
        zc ci = mi_pow(s->nghtol[is][iv] + 1);
        const double *tw = s->twnl + (long)ngpw * (iv + (long)s->nghmax * is);
        for (int ia = 0; ia < s->na[is]; ia++) {
          int isa = isa0 + ia;
          const zc *e = s->eigr + (long)ngrho * isa;
          for (int g = 0; g < ngpw; g++) {
            double er = creal(e[g]), ei = cimag(e[g]);
            if (fabs(creal(ci)) > 0.5) {
              double arg = s->gvec[3 * g + k] * tw[g] * creal(ci);
              scr[2 * g] = arg * er; scr[2 * g + 1] = arg * ei;
            } else {
              double arg = s->gvec[3 * g + k] * tw[g] * cimag(ci);
              scr[2 * g] = -arg * ei; scr[2 * g + 1] = arg * er;
            }
          }
          scr[0] *= 0.5; scr[1] *= 0.5;
#pragma omp parallel for schedule(static)
          for (int i = 0; i < n; i++) {
            const double *c = (const double *)(s->c0 + (long)i * ngpw);
            double acc = 0;
            for (long q = 0; q < 2L * ngpw; q++) acc += scr[q] * c[q];
            s->dfnl[isa + (long)nat * (iv + (long)s->nghmax * (k + 3L * i))] = tfac * acc;
          }
        }
      }
      isa0 += s->na[is];
    }
  }
  free(scr);
}

void orc_nlfor(orc_sys *s) {
  d_fnl(s);
  int nat = s->nat, n = s->nstate;
  int isa0 = 0;
  for (int is = 0; is < s->nsp; is++) {
    for (int iv = 0; iv < s->ngh[is]; iv++) {
      if (!s->upf) {
        double temp = 2.0 * s->wsg[is][iv];
        for (int i = 0; i < n; i++) {
          double w = s->occ[i];
          if (!(fabs(w) > 1e-12)) continue;
          for (int ia = 0; ia < s->na[is]; ia++) {
            int isa = isa0 + ia;
            double nlv = s->nl[isa + (long)nat * (iv + (long)s->nghmax * i)];
            double *F = s->force + 3 * (ia + (long)s->na_max * is);
            for (int k = 0; k < 3; k++)
              F[k] = F[k] - temp * w * (s->dfnl[isa + (long)nat * (iv + (long)s->nghmax * (k + 3L * i))] * nlv);
          }
        }
      } else {
        int l = s->nghtol[is][iv] + 1, ki = s->lfval[is][iv], li = s->lpval[is][iv];
        for (int jv = 0; jv < s->ngh[is]; jv++) {
          int l2 = s->nghtol[is][jv] + 1, lj = s->lpval[is][jv];
          if (!(l2 == l && li == lj)) continue;
          int kj = s->lfval[is][jv];
          for (int i = 0; i < n; i++) {
            double w = s->occ[i];
            if (!(fabs(w) > 1e-12)) continue;
            double tt = 2.0 * w * s->hlsg[is][l - 1][ki - 1][kj - 1];
            for (int ia = 0; ia < s->na[is]; ia++) {
              int isa = isa0 + ia;
              double nlv = s->nl[isa + (long)nat * (jv + (long)s->nghmax * i)];
              double *F = s->force + 3 * (ia + (long)s->na_max * is);
              for (int k = 0; k < 3; k++)
                F[k] = F[k] - tt * nlv * s->dfnl[isa + (long)nat * (iv + (long)s->nghmax * (k + 3L * i))];
            }
          }
        }
      }
    }
    isa0 += s->na[is];
  }
}

/* ------------------------------------------------------------------ */
/* cg.f90:3-61 hess, :63-145 PCG, :281-311 PRECON                       */
/* ------------------------------------------------------------------ */
static double dotp(const zc *a, const zc *b, int n) { /* wfn_initialize.f90:382-426 with g0_stat */
  const double *A = (const double *)a, *B = (const double *)b;
  double d = A[0] * B[0];
  double acc = 0;
  for (long k = 2; k < 2L * n; k++) acc += A[k] * B[k];
  return d + 2.0 * acc;
}

void orc_pcg(orc_sys *s, int istep) {
  int ngpw = s->ngpw, n = s->nstate;
  double *vpp = (double *)xcalloc(ngpw, sizeof(double));
  double vloc = creal(s->eigrxvps[0]);
  for (int g = 0; g < ngpw; g++) {
    double v = vloc;
    for (int is = 0; is < s->nsp; is++)
      for (int iv = 0; iv < s->ngh[is]; iv++) {
        double t = s->twnl[g + (long)ngpw * (iv + (long)s->nghmax * is)];
        double w = s->upf ? 0.0 : s->wsg[is][iv];
        v = v + s->na[is] * w * t * t;
      }
    vpp[g] = v;
  }
  for (int g = 0; g < ngpw; g++) {
    vpp[g] = 0.5 * s->tpiba2 * s->hg[g] + vpp[g];
    if (vpp[g] < HCUT) vpp[g] = HCUT;
  }
  for (int g = 0; g < ngpw; g++) vpp[g] = 1.0 / vpp[g];
  int nocc = 0;
  for (int i = 0; i < n; i++) if (s->occ[i] > 1e-5) nocc++;
  zc *cp = s->c2p;
  for (int i = 0; i < n; i++) {
    double fi = s->occ[i] > 0.01 ? 1.0 / s->occ[i] : 1.0;
    for (int g = 0; g < ngpw; g++) cp[g + (long)ngpw * i] = fi * vpp[g] * s->c2[g + (long)ngpw * i];
  }
  double ggnorm = 0.0;
  for (int i = 0; i < nocc; i++) ggnorm = ggnorm + dotp(cp + (long)ngpw * i, cp + (long)ngpw * i, ngpw);
  long tot = (long)ngpw * n;
  if (istep == 1) {
    s->fhist[0] = 5.0 * 5.0 / 400.0;
    s->ghist[0] = ggnorm;
    memcpy(s->hnm1, cp, sizeof(zc) * tot);
    for (long k = 0; k < tot; k++) s->c0[k] += s->fhist[0] * cp[k];
  } else {
    double forget = istep <= 10 ? 0.60 : (istep <= 20 ? 0.91 : 0.95);
    int ih;
    if (istep > 10) {
      ih = 10;
      for (int i = 0; i < 9; i++) { s->fhist[i] = s->fhist[i + 1]; s->ghist[i] = s->ghist[i + 1]; }
    } else
      ih = istep;
    s->ghist[ih - 1] = ggnorm;
    s->fhist[ih - 1] = s->fhist[ih - 2];
    double gamma = s->ghist[ih - 1] / s->ghist[ih - 2];
    gamma = forget * gamma;
    for (long k = 0; k < tot; k++) cp[k] += gamma * s->hnm1[k];
    memcpy(s->hnm1, cp, sizeof(zc) * tot);
    for (long k = 0; k < tot; k++) s->c0[k] += s->fhist[ih - 1] * s->hnm1[k];
  }
  free(vpp);
}

/* ------------------------------------------------------------------ */
/* wfn_initialize.f90:448-558 ortho_gs, UINV, ZCLEAN                    */
/* ------------------------------------------------------------------ */
int orc_ortho(orc_sys *s) {
  int n = s->nstate, ngpw = s->ngpw;
  double *S = (double *)xcalloc((long)n * n, sizeof(double));
  ovlap_d(s, s->c0, s->c0, S);
  spin_mask(s, S);
  /* DPOTRF('U'): S = U^T U, U stored in the upper triangle; block diagonal
     by spin when open shell, so the blocks factor separately */
  for (int j = 0; j < n; j++) {
    double d = S[j + (long)n * j];
    for (int k = 0; k < j; k++) d -= S[k + (long)n * j] * S[k + (long)n * j];
    if (!(d > 0.0)) { free(S); return 1; }
    d = sqrt(d);
    S[j + (long)n * j] = d;
    for (int i = j + 1; i < n; i++) {
      double t = S[j + (long)n * i];
      for (int k = 0; k < j; k++) t -= S[k + (long)n * j] * S[k + (long)n * i];
      S[j + (long)n * i] = t / d;
    }
  }
  /* DTRTRI('U','N'): U <- U^{-1} */
  double *Ui = (double *)xcalloc((long)n * n, sizeof(double));
  for (int j = 0; j < n; j++) {
    Ui[j + (long)n * j] = 1.0 / S[j + (long)n * j];
    for (int i = j - 1; i >= 0; i--) {
      double t = 0;
      for (int k = i + 1; k <= j; k++) t += S[i + (long)n * k] * Ui[k + (long)n * j];
      Ui[i + (long)n * j] = -t / S[i + (long)n * i];
    }
  }
  /* DTRMM('R','U','N','N'): C <- C U^{-1} */
  zc *tmp = (zc *)xcalloc((long)ngpw * n, sizeof(zc));
#pragma omp parallel for schedule(static)
  for (int j = 0; j < n; j++) {
    double *t = (double *)(tmp + (long)ngpw * j);
    for (int k = 0; k <= j; k++) {
      const double *c = (const double *)(s->c0 + (long)ngpw * k);
      double u = Ui[k + (long)n * j];
      for (long q = 0; q < 2L * ngpw; q++) t[q] += c[q] * u;
    }
  }
  memcpy(s->c0, tmp, sizeof(zc) * (long)ngpw * n);
  for (int i = 0; i < n; i++) s->c0[(long)ngpw * i] = creal(s->c0[(long)ngpw * i]);
  free(tmp); free(S); free(Ui);
  return 0;
}

/* ------------------------------------------------------------------ */
/* do_opt.f90:51-138 wfn_opt, gradient.f90:113-136 CHK_TFOR             */
/* ------------------------------------------------------------------ */
int orc_scf_iteration(orc_sys *s, int istep, double gcut) {
  orc_eval_density(s);
  orc_rhor2g(s);
  orc_eval_pot(s);
  orc_cal_vpot_ex(s);
  orc_pp_energy(s);
  orc_e_total(s);
  memset(s->c2, 0, sizeof(zc) * (long)s->ngpw * s->nstate);
  orc_vpsi(s);
  orc_fnonloc(s);
  orc_forces(s);
  eval_gmax(s, gcut);
  if (istep == 1) s->tfor = 0;
  else if (s->gemax < 3 * gcut) s->tfor = 1;
  if (s->tfor) {
    orc_e_sr(s, 1);
    orc_potfor(s);
    orc_nlfor(s);
  }
  orc_pcg(s, istep);
  if (orc_ortho(s)) return -1;
  return s->convwf;
}

int orc_wfn_opt(orc_sys *s, int max_step, double gcut) {
  for (int i = 1; i <= max_step; i++) {
    int r = orc_scf_iteration(s, i, gcut);
    if (r < 0) return -i;
    if (r) return i;
  }
  return max_step;
}

/* ------------------------------------------------------------------ */
/* construction (init_module.f90:3-162 order)                          */
/* ------------------------------------------------------------------ */
static double *dupd(const double *p, long n) {
  double *q = (double *)xcalloc(n, sizeof(double));
  if (p) memcpy(q, p, sizeof(double) * n);
  return q;
}

orc_sys *orc_create(const orc_input *in, int nthreads) {
  PI_ = 4.0 * atan(1.0);
  TWOPI_ = 8.0 * atan(1.0);
  FOURPI_ = 16.0 * atan(1.0);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  orc_sys *s = (orc_sys *)xcalloc(1, sizeof(orc_sys));
  s->nthreads = nthreads;
  s->nsp = in->nsp;
  s->na_max = in->na_max;
  s->xc = in->xc;
  s->symmetry = in->symmetry;
  s->upf = in->sp[0].type == ORC_PP_UPF;
  s->nat = 0;
  for (int is = 0; is < s->nsp; is++) {
    s->na[is] = in->na[is];
    s->nat += in->na[is];
    s->sp[is] = in->sp[is];
    s->zv[is] = (int)in->sp[is].zv;
    int mesh = in->sp[is].mesh;
    s->rr[is] = dupd(in->sp[is].rr, mesh);
    s->rw[is] = (double *)xcalloc(mesh, sizeof(double));
    if (!s->upf) {
      s->vr[is] = dupd(in->sp[is].vr, (long)in->sp[is].lmax * mesh);
      s->rps[is] = dupd(in->sp[is].rps, (long)in->sp[is].lmax * mesh);
    } else {
      /* convert_upf_to_psp (readupf.f90:412-425): rw = rab, vr(:,1) = vloc/2 */
      memcpy(s->rw[is], in->sp[is].rab, sizeof(double) * mesh);
      s->vr[is] = dupd(in->sp[is].vloc, mesh);
      long nb = in->sp[is].nbeta > 0 ? in->sp[is].nbeta : 1;
      s->beta[is] = dupd(in->sp[is].beta, nb * mesh);
    }
  }
  memcpy(s->a_cell, in->a_cell, sizeof s->a_cell);
  s->alat = in->alat;
  s->ecut = in->ecut;
  s->ecut_rho = in->ecut * 4.0;
  {
    const double *a = s->a_cell;
    double vol = A3(a, 1, 1) * (A3(a, 2, 2) * A3(a, 3, 3) - A3(a, 2, 3) * A3(a, 3, 2)) +
                 A3(a, 1, 2) * (A3(a, 2, 3) * A3(a, 3, 1) - A3(a, 2, 1) * A3(a, 3, 3)) +
                 A3(a, 1, 3) * (A3(a, 2, 1) * A3(a, 3, 2) - A3(a, 2, 2) * A3(a, 3, 1));
    s->omega = fabs(vol);
  }
  s->tpiba = 2.0 * PI_ / s->alat;
  s->tpiba2 = s->tpiba * s->tpiba;
  s->gcut_pw = s->ecut / s->tpiba2;
  s->gcut_rho = s->ecut_rho / s->tpiba2;
  {
    double at[9];
    for (int i = 1; i <= 3; i++)
      for (int j = 1; j <= 3; j++) A3(at, i, j) = A3(s->a_cell, j, i);
    inverse_matrix3(at, s->b_cell);
    for (int k = 0; k < 9; k++) s->b_cell[k] = s->b_cell[k] * s->alat;
  }
  set_r_grids(s->a_cell, s->ecut_rho, s->nr);
  for (int d = 0; d < 3; d++) s->nrl[d] = s->nr[d] + (s->nr[d] + 1) % 2;
  s->nnr1 = (long)s->nrl[0] * s->nrl[1] * s->nrl[2];
  setup_gvectors(s);
  for (int d = 0; d < 3; d++) plan_init(&s->pl[d], s->nr[d]);
  /* atoms */
  s->atco = dupd(in->atco, 3L * s->na_max * s->nsp);
  s->isa_is = (int *)xcalloc(s->nat, sizeof(int));
  s->isa_ia = (int *)xcalloc(s->nat, sizeof(int));
  {
    int k = 0;
    for (int is = 0; is < s->nsp; is++)
      for (int ia = 0; ia < s->na[is]; ia++) { s->isa_is[k] = is; s->isa_ia[k] = ia; k++; }
  }
  form_factors(s);
  projector_layout(s);
  nlppgrid(s);
  nlpro(s);
  exp_igrxfactor(s);
  /* occupations (atomic_basis.f90:49-79): closed shell two electrons per
     orbital; open shell one orbital per valence electron, occupation 1 */
  s->lsd = in->multiplicity > 0;
  int nst = in->nstate;
  if (nst <= 0) {
    nst = 0;
    for (int is = 0; is < s->nsp; is++) {
      if (s->lsd) {
        nst = nst + s->na[is] * s->zv[is];
      } else {
        nst = nst + (int)((double)(s->na[is] * s->zv[is]) / 2.0);
        if (2.0 * (double)nst < (double)(s->na[is] * s->zv[is])) { nst++; break; }
      }
    }
  }
  s->nstate = nst;
  s->occ = (double *)xcalloc(nst, sizeof(double));
  for (int i = 0; i < nst; i++) s->occ[i] = s->lsd ? 1.0 : 2.0;
  if (s->lsd) {
    /* NSPIN unpaired electrons; NEL_UP = INT((NSTATE-NSPIN)/2) bands of spin 1,
       NEL_DOWN = INT((NSTATE+NSPIN)/2) of spin 2 (init_module.f90:122-131) */
    int nspin = in->multiplicity - 1;
    int up = (int)((double)(nst - nspin) / 2.0), down = (int)((double)(nst + nspin) / 2.0);
    if (up + down != nst || up < 0 || down < 0) {
      fprintf(stderr, "oracle: incorrect multiplicity\n");
      abort();
    }
    if (in->xc != ORC_XC_TETER93) {
      fprintf(stderr, "oracle: the open-shell branch is restated for Teter93 only\n");
      abort();
    }
    s->nel_up = up;
  }
  long tot = (long)s->ngpw * nst;
  s->c0 = (zc *)xcalloc(tot, sizeof(zc));
  s->c2 = (zc *)xcalloc(tot, sizeof(zc));
  s->c2p = (zc *)xcalloc(tot, sizeof(zc));
  s->hnm1 = (zc *)xcalloc(tot, sizeof(zc));
  s->rho = (double *)xcalloc(s->nnr1, sizeof(double));
  s->v_pot = (double *)xcalloc(s->nnr1, sizeof(double));
  s->rho2 = (double *)xcalloc(s->nnr1, sizeof(double));
  s->v_pot2 = (double *)xcalloc(s->nnr1, sizeof(double));
  s->grad = (double *)xcalloc(4 * s->nnr1, sizeof(double));
  s->rho_g = (zc *)xcalloc(s->ngrho, sizeof(zc));
  s->nl = (double *)xcalloc((long)s->nat * s->nghmax * nst, sizeof(double));
  s->dfnl = (double *)xcalloc((long)s->nat * s->nghmax * 3 * nst, sizeof(double));
  s->force = (double *)xcalloc(3L * s->na_max * s->nsp, sizeof(double));
  s->w1 = (zc *)xcalloc(s->max_fft, sizeof(zc));
  s->w2 = (zc *)xcalloc(s->max_fft, sizeof(zc));
  s->wk = (zc *)xcalloc(s->max_fft, sizeof(zc));
  return s;
}

void orc_destroy(orc_sys *s) {
  if (!s) return;
  for (int is = 0; is < s->nsp; is++) {
    free(s->rr[is]); free(s->rw[is]); free(s->vr[is]); free(s->rps[is]); free(s->beta[is]);
    free(s->wns[is]); free(s->voo[is]);
  }
  for (int d = 0; d < 3; d++) free(s->pl[d].w);
  free(s->inyh); free(s->hg); free(s->hg_pert); free(s->gvec); free(s->mapp); free(s->mapm); free(s->msp); free(s->xrays);
  free(s->isa_is); free(s->isa_ia); free(s->atco);
  free(s->vps); free(s->rhos); free(s->twnl); free(s->eigr); free(s->eigrxvps); free(s->eigrxrhos);
  free(s->occ); free(s->c0); free(s->c2); free(s->c2p); free(s->hnm1);
  free(s->rho); free(s->v_pot); free(s->rho2); free(s->v_pot2); free(s->grad); free(s->rho_g); free(s->nl); free(s->dfnl); free(s->force);
  free(s->w1); free(s->w2); free(s->wk);
  free(s);
}

void orc_set_positions(orc_sys *s, const double *atco) {
  memcpy(s->atco, atco, sizeof(double) * 3L * s->na_max * s->nsp);
  exp_igrxfactor(s);
}

void orc_set_wfn(orc_sys *s, const double *c) {
  memcpy(s->c0, c, sizeof(zc) * (long)s->ngpw * s->nstate);
}

long orc_get_int(orc_sys *s, const char *k) {
  if (!strcmp(k, "ngpw")) return s->ngpw;
  if (!strcmp(k, "ngrho")) return s->ngrho;
  if (!strcmp(k, "ngrays")) return s->ngrays;
  if (!strcmp(k, "nhrays")) return s->nhrays;
  if (!strcmp(k, "nr1")) return s->nr[0];
  if (!strcmp(k, "nr2")) return s->nr[1];
  if (!strcmp(k, "nr3")) return s->nr[2];
  if (!strcmp(k, "nrl1")) return s->nrl[0];
  if (!strcmp(k, "nrl2")) return s->nrl[1];
  if (!strcmp(k, "nrl3")) return s->nrl[2];
  if (!strcmp(k, "nnr1")) return s->nnr1;
  if (!strcmp(k, "max_fft")) return s->max_fft;
  if (!strcmp(k, "nstate")) return s->nstate;
  if (!strcmp(k, "nat")) return s->nat;
  if (!strcmp(k, "nghmax")) return s->nghmax;
  if (!strcmp(k, "convwf")) return s->convwf;
  if (!strcmp(k, "tfor")) return s->tfor;
  if (!strncmp(k, "ngh", 3)) return s->ngh[atoi(k + 3)];
  return -1;
}

double orc_get_dbl(orc_sys *s, const char *k) {
  if (!strcmp(k, "etotal")) return s->etotal;
  if (!strcmp(k, "eke")) return s->eke;
  if (!strcmp(k, "estat")) return s->estat;
  if (!strcmp(k, "eself")) return s->eself;
  if (!strcmp(k, "esr")) return s->esr;
  if (!strcmp(k, "eloc")) return s->eloc;
  if (!strcmp(k, "enl")) return s->enl;
  if (!strcmp(k, "exc")) return s->exc;
  if (!strcmp(k, "etxc")) return s->etxc;
  if (!strcmp(k, "eh")) return s->eh_re;
  if (!strcmp(k, "gemax")) return s->gemax;
  if (!strcmp(k, "omega")) return s->omega;
  if (!strcmp(k, "tpiba")) return s->tpiba;
  if (!strcmp(k, "gcut_pw")) return s->gcut_pw;
  if (!strcmp(k, "gcut_rho")) return s->gcut_rho;
  return NAN;
}

void *orc_get_ptr(orc_sys *s, const char *k) {
  if (!strcmp(k, "inyh")) return s->inyh;
  if (!strcmp(k, "hg")) return s->hg;
  if (!strcmp(k, "hg_pert")) return s->hg_pert;
  if (!strcmp(k, "gvec")) return s->gvec;
  if (!strcmp(k, "mapp")) return s->mapp;
  if (!strcmp(k, "mapm")) return s->mapm;
  if (!strcmp(k, "msp")) return s->msp;
  if (!strcmp(k, "b_cell")) return s->b_cell;
  if (!strcmp(k, "vps")) return s->vps;
  if (!strcmp(k, "rhos")) return s->rhos;
  if (!strcmp(k, "twnl")) return s->twnl;
  if (!strcmp(k, "eigr")) return s->eigr;
  if (!strcmp(k, "eigrxvps")) return s->eigrxvps;
  if (!strcmp(k, "eigrxrhos")) return s->eigrxrhos;
  if (!strcmp(k, "occ")) return s->occ;
  if (!strcmp(k, "c0")) return s->c0;
  if (!strcmp(k, "c2")) return s->c2;
  if (!strcmp(k, "rho")) return s->rho;
  if (!strcmp(k, "v_pot")) return s->v_pot;
  if (!strcmp(k, "rho2")) return s->rho2;
  if (!strcmp(k, "v_pot2")) return s->v_pot2;
  if (!strcmp(k, "rho_g")) return s->rho_g;
  if (!strcmp(k, "nl")) return s->nl;
  if (!strcmp(k, "dfnl")) return s->dfnl;
  if (!strcmp(k, "force")) return s->force;
  if (!strcmp(k, "wsg")) return s->wsg;
  if (!strcmp(k, "atco")) return s->atco;
  return NULL;
}
