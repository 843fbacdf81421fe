/*
 * oracle.h -- CPU FP64 restatement of AMDKIIT's wavefunction hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the sm_100a
 * implementation in amdkiit_b200/: only tests/, __graft_entry__.smoke() and
 * the cpu_baseline leg of bench.py load it.  The product never links it.
 *
 * It restates, routine by routine, the reference Fortran sources (paths are
 * relative to the AMDKIIT project root):
 *   source/set_cell.f90, source/fft_support.f90      cell, b_cell, FFT grid
 *   source/gvectors.f90, source/math.f90             G half-sphere, EPSGX sort
 *   source/fft_interface.f90                         ray maps, do_fft
 *   source/exp_igr.f90                               structure/form factors
 *   source/pseudopotential.f90, source/readupf.f90   KB projectors (psp, UPF)
 *   source/density.f90, source/potential.f90         rho(r), rho(G), V_H+V_loc
 *   source/xc.f90                                    LDA/GGA potential
 *   source/total_energy.f90                          energies, Ewald (e_sr)
 *   source/wfn_initialize.f90                        vpsi, fnonloc, ortho_gs
 *   source/gradient.f90, source/cg.f90               Lambda, GEMAX, PCG
 *   source/nuclear_grad.f90                          POTFOR, NLFOR
 *   source/do_opt.f90                                wfn_opt loop
 * libxc (XC_LDA_XC_TETER93, XC_LDA_X+XC_LDA_C_PZ, XC_GGA_X_PBE+XC_GGA_C_PBE)
 * is not vendored by the reference; the functionals are restated from the
 * publications (Goedecker-Teter-Hutter PRB 54, 1703 (1996); Perdew-Zunger
 * PRB 23, 5048 (1981); Perdew-Burke-Ernzerhof PRL 77, 3865 (1996); PW92
 * correlation with the libxc "PW_MOD" A = 0.0310907).  FFTW, BLAS and LAPACK
 * are replaced by the plain loops and the mixed-radix FFT in oracle.c.
 */
#ifndef AMDK_ORACLE_H
#define AMDK_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAXSP 4
#define ORC_NSPLN 5000

enum { ORC_PP_PSP = 0, ORC_PP_UPF = 1 };
enum { ORC_XC_TETER93 = 0, ORC_XC_PZ = 1, ORC_XC_PBE = 2 };

/* One species as the reference holds it after read_psp / read_upf.
 * PSP: rr[mesh], vr[l*mesh+ir] (Ha) and rps[l*mesh+ir] for l < lmax,
 *      lmax/l_local/skip 1-based as after reading_input (yamlread.f90:300-314).
 * UPF: rr = PP_R, rab = PP_RAB, vloc = PP_LOCAL already halved (Ha),
 *      beta[nb*mesh+ir] = PP_BETA.nb (r*beta), beta_l[nb], dij[nb*nbeta+nb2]
 *      as in the file (Ry; the reader halves it, readupf.f90:347). */
typedef struct {
  int type;
  int z;
  double zv;
  int mesh;
  const double *rr;
  const double *vr;
  const double *rps;
  int lmax, l_local, skip, tkb;
  const double *rab;
  const double *vloc;
  int nbeta;
  const int *beta_l;
  const double *beta;
  const double *dij;
  int upf_lmax;            /* l_max + 1 from the header */
} orc_species;

typedef struct {
  double a_cell[9];        /* a_cell(3,3) column-major, bohr (set_vec) */
  double alat;             /* a_lattice, bohr */
  int symmetry;            /* 1 cubic, 2 fcc (set_cell.f90:17-40) */
  double ecut;             /* wavefunction cutoff, Ry */
  int nsp;
  int na[ORC_MAXSP];
  int na_max;
  const double *atco;      /* atco(3,na_max,nsp) column-major, bohr */
  int xc;
  int nstate;              /* 0: derived as in setbasis (atomic_basis.f90:49-71) */
  orc_species sp[ORC_MAXSP];
  int multiplicity;        /* 0: closed shell; m >= 1: OPEN_SHELL with MULTIPLICITY m (LSD,
                              init_module.f90:122-160; Teter93 only) */
} orc_input;

typedef struct orc_sys orc_sys;

orc_sys *orc_create(const orc_input *in, int nthreads);
void orc_destroy(orc_sys *s);

/* integer / pointer accessors by name (see orc_get_* in oracle.c) */
long orc_get_int(orc_sys *s, const char *name);
double orc_get_dbl(orc_sys *s, const char *name);
void *orc_get_ptr(orc_sys *s, const char *name);

/* geometry: new positions -> exp_igrxfactor (atco layout as orc_input) */
void orc_set_positions(orc_sys *s, const double *atco);

/* the seeded initial guess used by every configuration of the library:
 * complex Gaussian N(0,1) per real and imaginary part, damped by
 * 1/(1+|G|^2) with |G|^2 in bohr^-2, Im c(G=0)=0, then ortho_gs.
 * The random numbers come from the caller (so the product and the oracle
 * start from the same bits). */
void orc_set_wfn(orc_sys *s, const double *c0_interleaved);

/* hot-path routines (one call = one reference subroutine) */
void orc_fft(orc_sys *s, int sign, double *fz_interleaved);
void orc_eval_density(orc_sys *s);
void orc_rhor2g(orc_sys *s);
void orc_eval_pot(orc_sys *s);
void orc_cal_vpot_ex(orc_sys *s);
void orc_pp_energy(orc_sys *s);
void orc_e_total(orc_sys *s);
void orc_vpsi(orc_sys *s);
void orc_fnonloc(orc_sys *s);
void orc_forces(orc_sys *s);
void orc_e_sr(orc_sys *s, int tfor);
void orc_potfor(orc_sys *s);
void orc_nlfor(orc_sys *s);
void orc_pcg(orc_sys *s, int istep);
int  orc_ortho(orc_sys *s);
/* one CG iteration of wfn_opt (do_opt.f90:80-128); returns 1 when CONVWF */
int  orc_scf_iteration(orc_sys *s, int istep, double gcut);
/* full wfn_opt loop; returns the number of iterations done */
int  orc_wfn_opt(orc_sys *s, int max_step, double gcut);

/* pointwise XC restatement (exposed for finite-difference self tests):
 * e = rho*eps_xc, v = de/drho, vs = de/dsigma */
void orc_xc_point(int xc, double rho, double sigma, double *e, double *v, double *vs);

#ifdef __cplusplus
}
#endif
#endif
