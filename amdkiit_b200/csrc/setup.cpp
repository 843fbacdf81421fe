// Host-side setup of libamdk: what AMDKIIT's driver computes once per run
// before the first SCF iteration (init_module.f90:3-162).  FP64 on the host:
// cell and FFT grid (set_cell.f90, fft_support.f90), the G half-sphere with
// its EPSGX-perturbed sort (gvectors.f90:111-341, math.f90:200-305), the
// x-ray numbering and compressed maps (fft_interface.f90:151-363), and the
// radial pseudopotential tables (exp_igr.f90:142-288 form factors,
// pseudopotential.f90:234-291,434-529 projector transforms).  Everything
// evaluated per G vector (spline lookups, structure factors) runs on the GPU.
//
// Built with -ffp-contract=off: the G-vector order depends on the exact bits
// of |G|^2 and of the perturbed keys.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "amdk_internal.h"

namespace amdk {

static const double PI_ = 4.0 * std::atan(1.0);
static const double TWOPI_ = 8.0 * std::atan(1.0);
static const double FOURPI_ = 16.0 * std::atan(1.0);

#define A3(m, i, j) (m)[((i)-1) + 3 * ((j)-1)]

// math.f90:4-64 (Gauss-Jordan with row pivoting)
static void inverse3(const double *ain, double *b) {
  double a[9], d[9];
  int ip[4];
  std::memcpy(a, ain, sizeof a);
  for (int i = 0; i < 9; i++) b[i] = 0.0;
  for (int i = 1; i <= 3; i++) A3(b, i, i) = 1.0;
  for (int k = 1; k <= 3; k++) ip[k] = k;
  for (int k = 1; k <= 3; k++) {
    double dmax = std::fabs(A3(a, ip[k], ip[k]));
    int imax = k;
    for (int l = k; l <= 3; l++)
      if (std::fabs(A3(a, ip[l], ip[k])) > dmax) {
        dmax = std::fabs(A3(a, ip[l], ip[k]));
        imax = l;
      }
    std::swap(ip[imax], ip[k]);
    for (int i = 1; i <= 3; i++) {
      if (i == k) continue;
      double s = A3(a, ip[i], k) / A3(a, ip[k], k);
      double row[4];
      for (int c = k; c <= 3; c++) row[c] = A3(a, ip[k], c) * s;
      for (int c = k; c <= 3; c++) A3(a, ip[i], c) = A3(a, ip[i], c) - row[c];
      for (int c = 1; c <= 3; c++) row[c] = A3(b, ip[k], c) * s;
      for (int c = 1; c <= 3; c++) A3(b, ip[i], c) = A3(b, ip[i], c) - row[c];
    }
  }
  for (int i = 1; i <= 3; i++)
    for (int c = 1; c <= 3; c++) A3(d, i, c) = A3(b, ip[i], c) / A3(a, ip[i], i);
  std::memcpy(b, d, sizeof d);
}

// fft_support.f90:50-118: even and 2,3,5-smooth
static bool permitted(int n) {
  int m = n;
  const int f[3] = {2, 3, 5};
  for (int i = 0; i < 3; i++)
    while (m % f[i] == 0 && m > 1) m /= f[i];
  return m == 1;
}
static int optimal_fft_order(int n, int order) {
  while ((!permitted(n) || n % order != 0) && n <= 2049) n++;
  return n;
}

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

// math.f90:200-305 sort_array2: the reference's quicksort, kept so that the
// G order is the reference's even if two perturbed keys ever tie.
static void sort_array2(int n, double *arr1, int *index1) {
  double *arr = arr1 - 1;
  int *index = index1 - 1;
  const int M = 7, NSTACK = 64;
  int istack[NSTACK + 1];
  int i, l = 1, ib, ir = n, jstack = 0, k, j;
  double a;
  for (i = 1; i <= n; i++) index[i] = i;
  for (;;) {
    if (ir - l < M) {
      for (j = l + 1; j <= ir; j++) {
        a = arr[j];
        ib = index[j];
        for (i = j - 1; i >= 1; i--) {
          if (arr[i] <= a) break;
          arr[i + 1] = arr[i];
          index[i + 1] = index[i];
        }
        if (i < 1) i = 0;
        arr[i + 1] = a;
        index[i + 1] = ib;
      }
      if (jstack == 0) return;
      ir = istack[jstack];
      l = istack[jstack - 1];
      jstack -= 2;
    } else {
      k = (l + ir) / 2;
      std::swap(arr[k], arr[l + 1]);
      std::swap(index[k], index[l + 1]);
      if (arr[l + 1] > arr[ir]) { std::swap(arr[l + 1], arr[ir]); std::swap(index[l + 1], index[ir]); }
      if (arr[l] > arr[ir]) { std::swap(arr[l], arr[ir]); std::swap(index[l], index[ir]); }
      if (arr[l + 1] > arr[l]) { std::swap(arr[l + 1], arr[l]); std::swap(index[l + 1], index[l]); }
      i = l + 1;
      j = ir;
      a = arr[l];
      ib = index[l];
      for (;;) {
        do i++; while (arr[i] < a);
        do j--; while (arr[j] > a);
        if (j < i) break;
        std::swap(arr[i], arr[j]);
        std::swap(index[i], index[j]);
      }
      arr[l] = arr[j];
      arr[j] = a;
      index[l] = index[j];
      index[j] = ib;
      jstack += 2;
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

static int setup_gvectors(HostSetup &s) {
  int nr1 = s.nr[0], nr2 = s.nr[1], nr3 = s.nr[2];
  int nh1 = nr1 / 2 + 1, nh2 = nr2 / 2 + 1, nh3 = nr3 / 2 + 1;
  const double *b = s.b_cell;
  std::vector<double> key;
  std::vector<int> iy3;
  int ig = 0, ngpw = 0;
  for (int ix = 0; ix <= nr1 - 1; ix++) {
    int ymin = (ix == 0) ? 0 : -nr2 + 1;
    for (int iy = ymin; iy <= nr2 - 1; iy++) {
      int zmin = (ix == 0 && iy == 0) ? 0 : -nr3 + 1;
      for (int iz = zmin; iz <= nr3 - 1; iz++) {
        double gsq = gsquare(ix, iy, iz, b);
        if (!(gsq < s.gcut_rho)) continue;
        ig++;
        double sign = (gsq < s.gcut_pw) ? -1.0 : 1.0;
        if (sign < 0) ngpw++;
        double t = std::sqrt((double)(ig - 1));
        t = t * 1.0e-12;
        t = t * sign;
        t = 1.0 + t;
        key.push_back(gsq * t);
        iy3.push_back(nh1 + ix);
        iy3.push_back(nh2 + iy);
        iy3.push_back(nh3 + iz);
      }
    }
  }
  s.ngrho = ig;
  s.ngpw = ngpw;
  std::vector<int> idx(ig);
  sort_array2(ig, key.data(), idx.data());
  s.inyh.resize(3L * ig);
  for (int g = 0; g < ig; g++)
    for (int c = 0; c < 3; c++) s.inyh[3L * g + c] = iy3[3L * (idx[g] - 1) + c];
  s.gvec.resize(3L * ig);
  s.hg.resize(ig);
  for (int g = 0; g < ig; g++) {
    int ix = s.inyh[3L * g] - nh1, iy = s.inyh[3L * g + 1] - nh2, iz = s.inyh[3L * g + 2] - nh3;
    for (int r = 1; r <= 3; r++) {
      double t = (double)ix * A3(b, r, 1);
      t = t + (double)iy * A3(b, r, 2);
      t = t + (double)iz * A3(b, r, 3);
      s.gvec[3L * g + r - 1] = t;
    }
    double h = s.gvec[3L * g] * s.gvec[3L * g];
    h = h + s.gvec[3L * g + 1] * s.gvec[3L * g + 1];
    h = h + s.gvec[3L * g + 2] * s.gvec[3L * g + 2];
    s.hg[g] = h;
  }
  // fft_interface.f90:194-343 ray numbering and maps
  int k2 = s.nrl[1], k3 = s.nrl[2];
  s.xrays.assign((size_t)k2 * k3, 0);
  auto XR = [&](int i, int j) -> int & { return s.xrays[(i - 1) + (size_t)k2 * (j - 1)]; };
  for (int g = 0; g < ig; g++) {
    int i2 = s.inyh[3L * g + 1], i3 = s.inyh[3L * g + 2];
    int j2 = -i2 + 2 * nh2, j3 = -i3 + 2 * nh3;
    if (j2 < 1 || j2 > k2 || j3 < 1 || j3 > k3) {
      set_error("G sphere reaches the grid edge: mirror ray outside the grid");
      return AMDK_ERR_UNSUPPORTED;
    }
  }
  for (int g = 0; g < ngpw; g++) {
    int i2 = s.inyh[3L * g + 1], i3 = s.inyh[3L * g + 2];
    XR(i2, i3) += 1;
    XR(-i2 + 2 * nh2, -i3 + 2 * nh3) += 1;
  }
  int ii = 0;
  for (int j = 1; j <= k3; j++)
    for (int i = 1; i <= k2; i++)
      if (XR(i, j) != 0) XR(i, j) = ++ii;
  s.ngrays = ii;
  for (int g = ngpw; g < ig; g++) {
    int i2 = s.inyh[3L * g + 1], i3 = s.inyh[3L * g + 2];
    int j2 = -i2 + 2 * nh2, j3 = -i3 + 2 * nh3;
    if (XR(i2, i3) == 0) XR(i2, i3) = -1;
    if (XR(j2, j3) == 0) XR(j2, j3) = -1;
  }
  for (int j = 1; j <= k3; j++)
    for (int i = 1; i <= k2; i++)
      if (XR(i, j) < 0) XR(i, j) = ++ii;
  s.nhrays = ii;
  s.msp.assign(s.nhrays, 0);
  for (int i = 1; i <= k2; i++)
    for (int j = 1; j <= k3; j++)
      if (XR(i, j) > 0) s.msp[XR(i, j) - 1] = i + (j - 1) * k2;
  s.mapp.resize(ig);
  s.mapm.resize(ig);
  for (int g = 0; g < ig; g++) {
    int i1 = s.inyh[3L * g], i2 = s.inyh[3L * g + 1], i3 = s.inyh[3L * g + 2];
    s.mapp[g] = i1 + (XR(i2, i3) - 1) * s.nrl[0];
    s.mapm[g] = (-i1 + 2 * nh1) + (XR(-i2 + 2 * nh2, -i3 + 2 * nh3) - 1) * s.nrl[0];
  }
  return 0;
}

// spline.f90 spline_params + spline_thomas (natural cubic spline)
void spline_coeffs(int n, const double *xp, const double *yp, std::vector<double> &h, std::vector<double> &sdd) {
  h.assign(n + 1, 0.0);
  sdd.assign(n + 1, 0.0);
  std::vector<double> v(n + 1), u(n + 1), bb(n + 1);
  for (int i = 1; i <= n - 1; i++) {
    h[i] = xp[i] - xp[i - 1];
    bb[i] = (yp[i] - yp[i - 1]) / h[i];
  }
  for (int i = 2; i <= n - 1; i++) {
    v[i] = 2.0 * (h[i - 1] + h[i]);
    u[i] = 6.0 * (bb[i] - bb[i - 1]);
  }
  int m = n - 2;
  std::vector<double> d(m + 1), a(m + 1), b(m + 1), c(m + 1), x(m + 1);
  for (int i = 1; i <= m; i++) {
    d[i] = v[i + 1];
    a[i] = h[i + 1];
    c[i] = h[i + 1];
    b[i] = u[i + 1];
  }
  for (int i = 2; i <= m; i++) {
    double t = a[i - 1] / d[i - 1];
    d[i] = d[i] - t * c[i - 1];
    b[i] = b[i] - t * b[i - 1];
  }
  x[m] = b[m] / d[m];
  for (int i = m - 1; i >= 1; i--) x[i] = (b[i] - c[i] * x[i + 1]) / d[i];
  for (int i = 2; i <= n - 1; i++) sdd[i] = x[i - 1];
}

static int spline_hunt(int n, const double *xp, double x) {
  if (!(x < xp[n - 1])) return 1;
  int lo = 2, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) / 2;
    if (x < xp[mid - 1]) hi = mid;
    else lo = mid + 1;
  }
  return lo - 1;
}
static double spline_eval(const double *xp0, const double *yp0, const std::vector<double> &h, const std::vector<double> &sdd,
                          int ig, double x) {
  const double *xp = xp0 - 1, *yp = yp0 - 1;
  double d1 = x - xp[ig], d2 = xp[ig + 1] - x;
  double t1 = sdd[ig + 1] / 6.0 / h[ig] * (d1 * d1 * d1);
  double t2 = sdd[ig] / 6.0 / h[ig] * (d2 * d2 * d2);
  double t3 = (yp[ig + 1] / h[ig] - sdd[ig + 1] / 6.0 * h[ig]) * d1;
  double t4 = (yp[ig] / h[ig] - h[ig] / 6.0 * sdd[ig]) * d2;
  return t1 + t2 + t3 + t4;
}

// interpolgrid.f90:146-168 (the value is held when rw exceeds the last rp)
static void intrp_grid(const double *rp, int mp, const double *rw, int mw, double *f) {
  std::vector<double> fc(f, f + mp), h, sdd;
  spline_coeffs(mp, rp, fc.data(), h, sdd);
  double cc = 0.0;
  for (int i = 0; i < mw; i++) {
    if (!(rw[i] > rp[mp - 1])) cc = spline_eval(rp, fc.data(), h, sdd, spline_hunt(mp, rp, rw[i]), rw[i]);
    f[i] = cc;
  }
}

// math.f90:319-343
static double simpsn(int n, double *f1) {
  double *f = f1 - 1;
  f[1] *= 109.0 / 48.0;
  f[2] *= -5.0 / 48.0;
  f[3] *= 63.0 / 48.0;
  f[4] *= 49.0 / 48.0;
  f[n - 1] *= 109.0 / 48.0;
  f[n - 2] *= -5.0 / 48.0;
  f[n - 3] *= 63.0 / 48.0;
  f[n - 4] *= 49.0 / 48.0;
  double sum = 0;
  for (int i = 1; i <= n - 1; i++) sum = sum + f[i];
  return sum;
}

// bessel_func.f90:210-260
static double sph_bes(int n, double xx) {
  if (std::fabs(xx) < 1e-15) return n == 0 ? 1.0 : 0.0;
  if (xx < 1) {
    double fact = 1;
    for (int id = 1; id <= n; id++) fact = fact * xx / (double)(2 * id + 1);
    double jl = 1, jr = 1;
    int k = 0;
    while (std::fabs(jr) >= 1e-15 && k < 40) {
      k++;
      jr = -jr * (0.5 * xx * xx) / (double)(k * (2 * (n + k) + 1));
      jl = jl + jr;
    }
    return jl * fact;
  }
  double jl = std::sin(xx) / xx, jlp = (-std::cos(xx) + jl) / xx, jr;
  for (int id = 2; id <= n + 1; id++) {
    jr = -jl + (double)(2 * id - 1) * jlp / xx;
    jl = jlp;
    jlp = jr;
  }
  return jl;
}

int host_setup(const amdk_system *in, HostSetup &s, bool gvectors_only) {
  if (!in || in->nsp < 1 || in->nsp > AMDK_MAXSP) {
    set_error("amdk_create: nsp must be 1..4");
    return AMDK_ERR_BADARG;
  }
  if (in->symmetry != 1 && in->symmetry != 2) {
    set_error("amdk_create: only cubic (1) and fcc (2) cells are supported");
    return AMDK_ERR_UNSUPPORTED;
  }
  s.nsp = in->nsp;
  s.na_max = in->na_max;
  s.xc = in->xc;
  s.symmetry = in->symmetry;
  s.upf = in->sp[0].type == AMDK_PP_UPF;
  s.nat = 0;
  for (int is = 0; is < s.nsp; is++) {
    if ((in->sp[is].type == AMDK_PP_UPF) != s.upf) {
      set_error("amdk_create: psp and UPF species cannot be mixed (read_pp_file.f90:136-139)");
      return AMDK_ERR_BADARG;
    }
    s.na[is] = in->na[is];
    s.nat += in->na[is];
    s.zv[is] = (int)in->sp[is].zv;
  }
  std::memcpy(s.a_cell, in->a_cell, sizeof s.a_cell);
  s.alat = in->alat;
  s.ecut = in->ecut;
  double ecut_rho = in->ecut * 4.0;
  const double *a = s.a_cell;
  double vol = A3(a, 1, 1) * (A3(a, 2, 2) * A3(a, 3, 3) - A3(a, 2, 3) * A3(a, 3, 2)) +
               A3(a, 1, 2) * (A3(a, 2, 3) * A3(a, 3, 1) - A3(a, 2, 1) * A3(a, 3, 3)) +
               A3(a, 1, 3) * (A3(a, 2, 1) * A3(a, 3, 2) - A3(a, 2, 2) * A3(a, 3, 1));
  s.omega = std::fabs(vol);
  s.tpiba = 2.0 * PI_ / s.alat;
  s.tpiba2 = s.tpiba * s.tpiba;
  s.gcut_pw = s.ecut / s.tpiba2;
  s.gcut_rho = ecut_rho / s.tpiba2;
  double at[9];
  for (int i = 1; i <= 3; i++)
    for (int j = 1; j <= 3; j++) A3(at, i, j) = A3(s.a_cell, j, i);
  inverse3(at, s.b_cell);
  for (int k = 0; k < 9; k++) s.b_cell[k] = s.b_cell[k] * s.alat;
  for (int j = 1; j <= 3; j++) {
    double d = A3(a, 1, j) * A3(a, 1, j) + A3(a, 2, j) * A3(a, 2, j);
    d = d + A3(a, 3, j) * A3(a, 3, j);
    double x = std::sqrt(d) / PI_;
    x = x * std::sqrt(ecut_rho);
    x = x + 0.5;
    s.nr[j - 1] = optimal_fft_order((int)std::lround(x), 2);
    s.nrl[j - 1] = s.nr[j - 1] + (s.nr[j - 1] + 1) % 2;
  }
  int rc = setup_gvectors(s);
  if (rc) return rc;
  if (gvectors_only) return 0;
  s.atco.assign(in->atco, in->atco + 3L * s.na_max * s.nsp);
  for (int is = 0; is < s.nsp; is++)
    for (int ia = 0; ia < s.na[is]; ia++) {
      s.isa_is.push_back(is);
      s.isa_ia.push_back(ia);
    }
  // ---- projector layout (atomic_basis.f90:91-121, readupf.f90:251-352)
  s.nghmax = 1;
  std::memset(s.hlsg, 0, sizeof s.hlsg);
  std::memset(s.wsg, 0, sizeof s.wsg);
  for (int is = 0; is < s.nsp; is++) {
    const amdk_species &p = in->sp[is];
    int iv = 0;
    if (!s.upf) {
      for (int il = 1; il <= p.lmax; il++) {
        if (il == p.l_local || il == p.skip) continue;
        int l = il - 1, ic = (l == 0) ? 0 : l * l;
        for (int j = 1; j <= 2 * l + 1; j++) {
          s.nghtol[is][iv] = l;
          s.lpval[is][iv] = ic + j;
          s.lfval[is][iv] = 1;
          iv++;
        }
      }
    } else {
      int npro[LMAXX + 2] = {0}, pl1[64], pl2[64];
      for (int nb = 0; nb < p.nbeta; nb++) {
        int l = p.beta_l[nb];
        pl1[nb] = l;
        npro[l + 1]++;
        pl2[nb] = npro[l + 1];
      }
      int lp = 0;
      for (int L = 1; L <= p.upf_lmax; L++)
        for (int M = 1; M <= 2 * L - 1; M++) {
          lp++;
          for (int K = 1; K <= npro[L]; K++) {
            s.nghtol[is][iv] = L - 1;
            s.lpval[is][iv] = lp;
            s.lfval[is][iv] = K;
            iv++;
          }
        }
      for (int i = 0; i < p.nbeta; i++) {
        int l = pl1[i] + 1, k = pl2[i];
        s.hlsg[is][l - 1][k - 1][k - 1] = 0.5 * p.dij[i * p.nbeta + i];
      }
    }
    s.ngh[is] = iv;
    s.nghmax = std::max(s.nghmax, iv);
  }
  // ---- form factors (exp_igr.f90:142-288) and projector tables
  s.ggnh.resize(NSPLN);
  s.ggng.resize(NSPLN);
  for (int il = 1; il <= NSPLN; il++) s.ggng[il - 1] = (double)(il - 1) * s.gcut_pw / (double)(NSPLN - 1);
  std::vector<std::vector<double>> rw(s.nsp), vr(s.nsp), rps(s.nsp);
  for (int is = 0; is < s.nsp; is++) {
    const amdk_species &p = in->sp[is];
    int mesh = p.mesh;
    const double *rr = p.rr;
    double zvd = (double)s.zv[is];
    std::vector<double> fint(mesh), dfint(mesh);
    s.voo[is].assign(NSPLN, 0.0);
    rw[is].assign(mesh, 0.0);
    if (!s.upf) {
      rw[is][0] = rr[0];
      for (int ir = 1; ir < mesh; ir++) rw[is][ir] = rw[is][ir - 1] * std::exp(std::log(rr[mesh - 1] / rr[0]) / (double)(mesh - 1));
      vr[is].assign(p.vr, p.vr + (size_t)p.lmax * mesh);
      rps[is].assign(p.rps, p.rps + (size_t)p.lmax * mesh);
      for (int il = 0; il < p.lmax; il++) intrp_grid(rr, mesh, rw[is].data(), mesh, vr[is].data() + (size_t)il * mesh);
      const double *vl = vr[is].data() + (size_t)(p.l_local - 1) * mesh;
      const double *w = rw[is].data();
      for (int ir = 0; ir < mesh; ir++) {
        double e = std::erf(w[ir] / RAGGIO);
        fint[ir] = w[ir] * w[ir] * w[ir] * vl[ir] + zvd * e * w[ir] * w[ir];
        double check = !(std::fabs(w[ir]) < 1e-8) ? vl[ir] + zvd * e / w[ir] : vl[ir] + 2.0 * zvd / (std::sqrt(PI_) * RAGGIO);
        if (std::fabs(check) < 1e-8) fint[ir] = 0.0;
      }
      double dlog = std::log(rr[mesh - 1] / rr[0]) / (double)(mesh - 1);
      for (int il = 1; il <= NSPLN; il++) {
        s.ggnh[il - 1] = (double)(il - 1) * s.gcut_rho / (double)(NSPLN - 1);
        double xg = std::sqrt(s.ggnh[il - 1]) * s.tpiba;
        if (xg > 1e-6) {
          for (int ir = 0; ir < mesh; ir++) {
            double xrg = w[ir] * xg;
            dfint[ir] = fint[ir] * std::sin(xrg) / xrg;
          }
        } else
          dfint = fint;
        s.voo[is][il - 1] = dlog * FOURPI_ * simpsn(mesh, dfint.data());
      }
    } else {
      rw[is].assign(p.rab, p.rab + mesh);
      vr[is].assign(p.vloc, p.vloc + mesh);
      for (int ir = 0; ir < mesh; ir++) fint[ir] = rr[ir] * rr[ir] * vr[is][ir] + zvd * std::erf(rr[ir] / RAGGIO) * rr[ir];
      for (int il = 1; il <= NSPLN; il++) {
        s.ggnh[il - 1] = (double)(il - 1) * (s.gcut_rho / (double)(NSPLN - 1));
        double sq = std::sqrt(s.ggnh[il - 1]);
        if (sq * s.tpiba > 1e-6) {
          for (int ir = 0; ir < mesh; ir++) {
            double xrg = rr[ir] * sq * s.tpiba;
            dfint[ir] = fint[ir] * std::sin(xrg) / xrg * rw[is][ir];
          }
        } else
          for (int ir = 0; ir < mesh; ir++) dfint[ir] = fint[ir] * rw[is][ir];
        s.voo[is][il - 1] = FOURPI_ * simpsn(mesh, dfint.data());
      }
    }
  }
  // ---- projector tables (pseudopotential.f90:434-529, :234-291)
  for (int is = 0; is < s.nsp; is++) {
    const amdk_species &p = in->sp[is];
    int mesh = p.mesh;
    const double *rr = p.rr;
    const double *w = rw[is].data();
    s.wns[is].assign((size_t)NSPLN * (s.ngh[is] + 1), 0.0);
    std::vector<double> fnt(mesh);
    if (!s.upf) {
      if (!p.tkb) continue;
      intrp_grid(in->sp[0].rr, mesh, w, mesh, rps[is].data());
      const double *gmax = vr[is].data() + (size_t)(p.l_local - 1) * mesh;
      std::vector<double> gnl((size_t)(p.lmax + 1) * mesh, 0.0);
      double loggrid = std::log(rr[mesh - 1] / rr[0]) / (double)(mesh - 1);
      double wsgtmp[LMAXX + 2] = {0};
      for (int l = 1; l <= p.lmax; l++) {
        if (l == p.skip || l == p.l_local) continue;
        double *g = gnl.data() + (size_t)l * mesh;
        const double *vl = vr[is].data() + (size_t)(l - 1) * mesh;
        for (int ir = 0; ir < mesh; ir++) {
          g[ir] = vl[ir] - gmax[ir];
          if (std::fabs(g[ir]) < 1e-10) g[ir] = 0.0;
        }
        const double *ps = rps[is].data() + (size_t)(l - 1) * mesh;
        for (int ir = 0; ir < mesh; ir++) fnt[ir] = ps[ir] * ps[ir] * g[ir] * w[ir];
        double wl = simpsn(mesh, fnt.data());
        wsgtmp[l] = 1.0 / (loggrid * wl);
      }
      int k = 0;
      for (int l = 1; l <= p.lmax; l++)
        if (l != p.l_local && l != p.skip)
          for (int lm = 1; lm <= 2 * l - 1; lm++) s.wsg[is][k++] = wsgtmp[l];
      int lold = -1;
      for (int iv = 0; iv < s.ngh[is]; iv++) {
        int l = s.nghtol[is][iv] + 1;
        double *wn = s.wns[is].data() + (size_t)iv * NSPLN;
        if (l == lold) {
          std::memcpy(wn, wn - NSPLN, sizeof(double) * NSPLN);
        } else if (l != p.skip) {
          const double *ps = rps[is].data() + (size_t)(l - 1) * mesh;
          const double *g = gnl.data() + (size_t)l * mesh;
          for (int il = 0; il < NSPLN; il++) {
            double xg = std::sqrt(s.ggng[il]) * TWOPI_ / s.alat;
            for (int ir = 0; ir < mesh; ir++) fnt[ir] = w[ir] * w[ir] * ps[ir] * g[ir] * sph_bes(l - 1, xg * w[ir]);
            wn[il] = loggrid * FOURPI_ * simpsn(mesh, fnt.data());
          }
        }
        lold = l;
      }
    } else {
      int lold = -1;
      for (int iv = 0; iv < s.ngh[is]; iv++) {
        int l = s.nghtol[is][iv] + 1;
        double *wn = s.wns[is].data() + (size_t)iv * NSPLN;
        if (l == lold) {
          std::memcpy(wn, wn - NSPLN, sizeof(double) * NSPLN);
        } else {
          if (l - 1 >= p.nbeta) {
            set_error("UPF: projector slot indexed by angular momentum exceeds number_of_proj");
            return AMDK_ERR_UNSUPPORTED;
          }
          const double *bt = p.beta + (size_t)(l - 1) * mesh;   // upf_gnl(:,is,l)
          for (int il = 0; il < NSPLN; il++) {
            double xg = std::sqrt(s.ggng[il]) * TWOPI_ / s.alat;
            for (int ir = 0; ir < mesh; ir++) fnt[ir] = w[ir] * rr[ir] * bt[ir] * sph_bes(l - 1, xg * rr[ir]);
            wn[il] = FOURPI_ * simpsn(mesh, fnt.data());
          }
        }
        lold = l;
      }
    }
  }
  // ---- occupations (atomic_basis.f90:49-79): closed shell two electrons per
  // orbital; open shell one orbital per valence electron, occupation 1
  s.lsd = in->multiplicity > 0;
  int nst = in->nstate;
  if (nst <= 0) {
    nst = 0;
    for (int is = 0; is < s.nsp; is++) {
      if (s.lsd) {
        nst = nst + s.na[is] * s.zv[is];
      } else {
        nst = nst + (int)((double)(s.na[is] * s.zv[is]) / 2.0);
        if (2.0 * (double)nst < (double)(s.na[is] * s.zv[is])) {
          nst++;
          break;
        }
      }
    }
  }
  s.nstate = nst;
  s.occ.assign(nst, s.lsd ? 1.0 : 2.0);
  if (s.lsd) {
    // NSPIN unpaired electrons; NEL_UP = INT((NSTATE-NSPIN)/2) bands of spin 1,
    // NEL_DOWN = INT((NSTATE+NSPIN)/2) of spin 2 (init_module.f90:122-131)
    const int nspin = in->multiplicity - 1;
    const int up = (int)((double)(nst - nspin) / 2.0), down = (int)((double)(nst + nspin) / 2.0);
    if (up + down != nst || up < 0 || down < 0) {
      set_error("incorrect multiplicity for the number of bands");
      return AMDK_ERR_BADARG;
    }
    if (in->xc != AMDK_XC_TETER93) {
      set_error("the open-shell branch supports Teter93 only");
      return AMDK_ERR_UNSUPPORTED;
    }
    s.nel_up = up;
  }
  return 0;
}

}  // namespace amdk
