/*
 * amdk.h -- C-ABI of libamdk, the sm_100a implementation of AMDKIIT's
 * wavefunction hot path (one GPU).
 *
 * The reference (AMDKIIT, Fortran) has no plugin API: its hot path is a set
 * of argument-less subroutines that read and write module globals
 * (source/system_data_types.f90:63-234).  Each entry point below replaces one
 * of those subroutines (cited per function, paths relative to the AMDKIIT
 * project root) and is callable from Fortran through iso_c_binding in the
 * way the reference already binds C (source/yaml.f90:35-42 <-> yaml.cpp:168).
 *
 * Conventions
 *  - every function returns 0 on success or a negative AMDK_ERR_* code;
 *    amdk_last_error() returns a message for the calling thread;
 *  - host arrays are caller-owned; Fortran column-major layouts are kept
 *    (C0(ngpw,nstate) complex, atco(3,na_max,nsp), force(3,na_max,nsp));
 *  - device state is owned by the context; one CUDA stream per context;
 *    calls on one context are not re-entrant, separate contexts may be used
 *    from separate host threads;
 *  - there is no CPU fallback: if the CUDA kernels cannot run, calls fail.
 */
#ifndef AMDK_H
#define AMDK_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

#define AMDK_MAXSP 4

enum {
  AMDK_OK = 0,
  AMDK_ERR_BADARG = -1,
  AMDK_ERR_CUDA = -2,
  AMDK_ERR_ALLOC = -3,
  AMDK_ERR_NOT_SPD = -4,     /* overlap not positive definite (UINV STOP, wfn_initialize.f90:514-528) */
  AMDK_ERR_NONFINITE = -5,   /* NaN/Inf in energy or gradient */
  AMDK_ERR_TIMEOUT = -6,
  AMDK_ERR_UNSUPPORTED = -7
};

enum { AMDK_PP_PSP = 0, AMDK_PP_UPF = 1 };
enum { AMDK_XC_TETER93 = 0, AMDK_XC_PZ = 1, AMDK_XC_PBE = 2 };
enum { AMDK_FP64 = 0, AMDK_MIXED = 1 };

/* One species as held after read_psp (source/readpsp.f90:11-67) or
 * read_upf (source/readupf.f90:19-85). Same meaning as orc_species. */
typedef struct {
  int type;               /* AMDK_PP_PSP or AMDK_PP_UPF */
  int z;
  double zv;
  int mesh;
  const double *rr;       /* radial mesh (PSP rr, UPF PP_R) */
  const double *vr;       /* PSP: vr[l*mesh+ir], l < lmax, Hartree */
  const double *rps;      /* PSP: rps[l*mesh+ir] */
  int lmax, l_local, skip, tkb;   /* PSP, 1-based (yamlread.f90:300-314) */
  const double *rab;      /* UPF PP_RAB */
  const double *vloc;     /* UPF PP_LOCAL / 2 (Hartree) */
  int nbeta;
  const int *beta_l;
  const double *beta;     /* beta[nb*mesh+ir] = r*beta_nb(r) */
  const double *dij;      /* PP_DIJ as in the file (Ry) */
  int upf_lmax;           /* header l_max + 1 */
} amdk_species;

/* The system after the reference's input stage (init_module.f90:3-113). */
typedef struct {
  double a_cell[9];       /* a_cell(3,3) column-major, bohr */
  double alat;            /* a_lattice, bohr */
  int symmetry;           /* 1 cubic, 2 fcc */
  double ecut;            /* wavefunction cutoff, Ry (density cutoff = 4 ecut) */
  int nsp;
  int na[AMDK_MAXSP];
  int na_max;
  const double *atco;     /* atco(3,na_max,nsp), bohr */
  int xc;                 /* AMDK_XC_* */
  int nstate;             /* 0: from the valence charge (atomic_basis.f90:49-71) */
  amdk_species sp[AMDK_MAXSP];
  int multiplicity;       /* 0: closed shell; m >= 1: OPEN_SHELL with MULTIPLICITY m, the LSD
                             branch (init_module.f90:122-160): one orbital per valence electron,
                             occupation 1, bands 1..NEL_UP = INT((NSTATE-m+1)/2) of spin 1,
                             the rest of spin 2; Teter93 only, pencil transforms only */
} amdk_system;

typedef struct {
  int device;             /* CUDA device ordinal */
  int precision;          /* AMDK_FP64 or AMDK_MIXED */
  int pair_batch;         /* band pairs per FFT batch (0: automatic) */
  int reserved[8];        /* zero; tests of the failure path only: reserved[0] != 0, the
                             pipeline waits of the int8 tensor-core kernels (mixed path)
                             give up after max(reserved[0], 0) polls; reserved[1] != 0, the
                             same for the FP64 tensor-core kernels; the call then returns
                             AMDK_ERR_TIMEOUT */
} amdk_options;

typedef struct {
  int nr[3];              /* FFT grid (set_cell.f90:177-211) */
  int ngpw, ngrho;        /* wavefunction / density half-sphere sizes */
  int ngrays, nhrays;     /* x-rays of the two spheres (fft_interface.f90:262-293) */
  int nstate, nat, nghmax;
  double omega;
} amdk_info;

typedef struct {
  double etotal, eke, estat, eself, esr, eloc, enl, exc, eh;  /* total_energy.f90:4-36 */
} amdk_energies;

typedef struct amdk_ctx amdk_ctx;

const char *amdk_last_error(void);

/* Setup: init_module.f90:3-162 from the input stage on (grids, G vectors,
 * ray maps, form factors, projector tables, structure factors), then
 * uploads every immutable table to the device. */
int amdk_create(const amdk_system *sys, const amdk_options *opt, amdk_ctx **out);
int amdk_destroy(amdk_ctx *ctx);
int amdk_info_get(amdk_ctx *ctx, amdk_info *info);

/* G half-sphere in the reference's layout (gvectors.f90:111-341 and
 * fft_interface.f90:151-363 with one rank): inyh(3,ngrho) 1-based grid
 * indices, hg(ngrho), gvec(3,ngrho), map_grid1d_p/m(ngrho) 1-based into the
 * ray-compressed x-line buffer of leading dimension nrlead(1).  Any pointer
 * may be NULL. */
int amdk_get_gvectors(amdk_ctx *ctx, int *inyh, double *hg, double *gvec, int *map_p, int *map_m);

/* The same G half-sphere and maps from the host setup alone, without a GPU
 * context (gvectors.f90 + prepare_fft for callers that only need the
 * integer maps).  Call first with NULL arrays to get the sizes in *info. */
int amdk_host_gvectors(const amdk_system *sys, amdk_info *info, int *inyh, double *hg, double *gvec, int *map_p,
                       int *map_m);

/* exp_igr.f90:4-140 exp_igrxfactor for new positions atco(3,na_max,nsp) */
int amdk_set_positions(amdk_ctx *ctx, const double *atco);

/* Precision of the band-pair transforms (vpsi, eval_density) from the next
 * call on: AMDK_FP64 or AMDK_MIXED (FP32 FFT data, FP64 everything else).
 * Lets a driver converge in mixed precision and refine the last iterations
 * in FP64 (no reference counterpart: the reference is FP64 only). */
int amdk_set_precision(amdk_ctx *ctx, int precision);

/* C_0(ngpw,nstate) complex as interleaved doubles (host memory) */
int amdk_set_wfn(amdk_ctx *ctx, const double *c0);
int amdk_get_wfn(amdk_ctx *ctx, double *c0);

/* rho(r) given instead of computed from C0 (nr3*nr2*nr1 FP64, host memory, x
 * fastest), with rhor2g (density.f90:128-150) applied, so that amdk_potential
 * and amdk_energy use it: the density of a system whose bands are spread over
 * several processes, gathered from their slabs (amdk_slab_planes_density).
 * Closed shell only. */
int amdk_set_density(amdk_ctx *ctx, const double *rho);

/* wfn_initialize.f90:448-499 ortho_gs (Cholesky of the overlap) */
int amdk_ortho(amdk_ctx *ctx);
/* density.f90:5-98 eval_density + density.f90:128-150 rhor2g */
int amdk_density(amdk_ctx *ctx);
/* potential.f90:4-46 eval_pot + xc.f90:4-434 cal_vpot_ex */
int amdk_potential(amdk_ctx *ctx);
/* pseudopotential.f90:3-103 pp_energy (fnl) + total_energy.f90:4-36 e_total */
int amdk_energy(amdk_ctx *ctx, amdk_energies *out);
/* wfn_initialize.f90:268-365 vpsi + :560-695 fnonloc/upf_fnonloc: C2 = -f H C0 */
int amdk_apply_h(amdk_ctx *ctx);
/* gradient.f90:5-61 forces (Lambda, C2 -= C0 Lambda, ZCLEAN) + eval_GMAX */
int amdk_gradient(amdk_ctx *ctx, double *gemax);
/* cg.f90:63-145 PCG (hess, precon, direction, C0 += 0.0625 d) */
int amdk_pcg(amdk_ctx *ctx, int istep);
/* One CG iteration of do_opt.f90:80-128 (density ... ortho_gs), ionic
 * forces included once GEMAX < 3*gcut as in CHK_TFOR (gradient.f90:113-136). */
int amdk_scf_iteration(amdk_ctx *ctx, int istep, double gcut, amdk_energies *e, double *gemax, int *converged);
/* total_energy.f90:133-239 e_sr + nuclear_grad.f90:4-89 POTFOR, NLFOR
 * (UPF_NLFOR :153-199) for the current C0 and density: force(3,na_max,nsp) */
int amdk_ionic_forces(amdk_ctx *ctx, double *force);

/* Backward (adjoint) entry for the current C0 and positions:
 * dE_dR(3,na_max,nsp) = dE_total/dR_I = -(e_sr + POTFOR + NLFOR forces), the
 * derivative of the local-pseudopotential/structure-factor term, of the
 * nonlocal projectors (D_FNL, nuclear_grad.f90:314-372) and of the Ewald sum;
 * dE_dpsi(ngpw,nstate) complex = f_i (H c_i)(G), the unconstrained gradient
 * of E with respect to the coefficients as vpsi + fnonloc build it (the
 * reference's C2 negated).  Either pointer may be NULL. */
int amdk_backward(amdk_ctx *ctx, double *dE_dR, double *dE_dpsi);

/* Wavefunction predictor for BOMD (no reference counterpart: the reference
 * restarts each step from the previous C0, molecular_dynamics.f90:106-109).
 * amdk_wfn_extrapolate predicts
 *   C0 <- sum_j w_j C0(t-j dt) M_j,  M_j = C0(t-j dt)^T C0(t)
 * (M_0 = 1; the overlap in the Gamma convention aligns step j's occupied
 * subspace with the current one, a density-matrix extrapolation applied to
 * C0(t)) and then stores C0(t).  The caller orthonormalises afterwards
 * (amdk_ortho), as after a geometry update.  amdk_wfn_set_predictor sets
 * the number of points (C0(t) included, 1..8; default 2) and their weights,
 * most recent first; coef = NULL selects Kolafa's always-stable predictor
 * weights for that many points ((2,-1) for 2: linear extrapolation).  Until
 * enough steps are stored the always-stable weights of the points there are
 * used.  amdk_wfn_history_clear forgets the stored steps. */
int amdk_wfn_set_predictor(amdk_ctx *ctx, int npoints, const double *coef);
int amdk_wfn_extrapolate(amdk_ctx *ctx);
int amdk_wfn_history_clear(amdk_ctx *ctx);

/* Copy a named device array to host memory (parity tests and drivers).
 * Names: "rho","v_pot" (nr3*nr2*nr1 real, x fastest), "rho_g" (ngrho complex),
 * "c2" (ngpw*nstate complex), "nl" (nat*nghmax*nstate), "vps","rhos"
 * (nsp*ngrho), "twnl" (ngpw*nghmax*nsp), "eigrxvps","eigrxrhos" (ngrho complex),
 * "overlap" (nstate*nstate: the last Gram matrix, S of ortho_gs or Lambda). */
int amdk_get_array(amdk_ctx *ctx, const char *name, void *dst, size_t bytes);

/* Raw pruned 3D FFT on the density sphere (fft_interface.f90:6-29):
 * sign=-1: coef(ngrho) complex (the +G half; -G taken as conj) -> grid
 *          (nr3*nr2*nr1 complex); sign=+1: grid -> coef = F(+G)/N. */
int amdk_fft_sphere(amdk_ctx *ctx, int sign, double *coef, double *grid);

/* Live kernel timing with CUDA events on the context stream (no
 * counterpart in the reference, whose only tracing is cpu_time per CG
 * iteration, do_opt.f90:81,118).  kind: 0 fused z pass of H|psi>, 1 fused
 * z pass of the density, 2 y passes, 3 forward x passes.  bytes = the
 * algorithmic bytes of the timed launches. */
int amdk_profile(amdk_ctx *ctx, int enable);
int amdk_profile_get(amdk_ctx *ctx, int kind, long *launches, double *total_ms, double *bytes);

/* Number of this library's kernels launched so far on the context (cuBLAS
 * kernels are not counted). */
int amdk_launch_count(amdk_ctx *ctx, long *n);

/* amdk_fft_sphere for callers that cannot allocate device memory (an
 * application that hands every device allocation to its own pool, or a
 * Fortran code whose device memory is managed by OpenACC/OpenMP runtimes):
 * no counterpart in the reference.  coef (ngrho complex) and grid
 * (nr3*nr2*nr1 complex) are DEVICE pointers owned by the caller; the call
 * allocates nothing.  Its scratch is one fixed 24 MiB device array inside the
 * library (held by every GPU that loads it), which limits it to grids whose
 * density-sphere transform fits (about 90^3: the 90^3 H2 cell needs 22.3 MB);
 * larger grids return AMDK_ERR_UNSUPPORTED.  Each call looks up the array's
 * device address on the current device, so make the first call before any
 * stream capture.  The call starts with a device-wide synchronisation, so
 * inputs written on any stream of the caller's are complete before it reads
 * them, and returns after the transform has finished.  All calls share the
 * array: calls that overlap on the GPU (several contexts or threads at once)
 * race. */
int amdk_fft_sphere_noalloc(amdk_ctx *ctx, int sign, double *coef, double *grid);

/* Elapsed device time of the last amdk_scf_iteration, milliseconds. */
int amdk_last_iteration_ms(amdk_ctx *ctx, double *ms);

/* Several systems on one GPU advanced together, e.g. an ensemble of small
 * clusters (no reference counterpart: the reference runs one system per
 * process).  The contexts stay owned by the caller and must outlive the
 * ensemble.  amdk_ensemble_iteration runs one CG iteration, as
 * amdk_scf_iteration does, of every member (istep[i]: member i's CG step
 * number): from every member's second iteration on, segment A of all members
 * (density, potential, energies, H|psi>, gradient) is one CUDA graph launch
 * whose children are the members' own segment graphs, then one host read of
 * all the GEMAX values decides CHK_TFOR per member, then segment B (forces,
 * PCG, ortho) is a second launch.  Results equal per-context
 * amdk_scf_iteration calls.  e, gemax, converged: arrays of n entries (any may
 * be NULL).  amdk_ensemble_last_ms: device time of the last iteration of all
 * members together. */
typedef struct amdk_ensemble amdk_ensemble;
int amdk_ensemble_create(amdk_ctx **ctx, int n, amdk_ensemble **out);
int amdk_ensemble_iteration(amdk_ensemble *ens, const int *istep, double gcut, amdk_energies *e, double *gemax,
                            int *converged);
int amdk_ensemble_last_ms(amdk_ensemble *ens, double *ms);
int amdk_ensemble_destroy(amdk_ensemble *ens);

/* Slab decomposition of the band-pair transforms over nranks processes, as
 * the reference distributes its FFTs (do_fft, fft_interface.f90:109-137):
 * G space by x-rays, real space by contiguous x planes
 * (distribute_YZplanes, gvectors.f90:80-108), an all-to-all in between
 * (FFT_COMM -> MPI_trans, fft_interface.f90:500-511).  The library does the
 * compute on each side of the exchange and writes/reads the exchange
 * buffers in place; the caller moves them (one all-to-all, e.g. NCCL's, per
 * direction), so no collective library is linked here.
 *
 * Ownership: rays go to ranks in mirror pairs {(ky,kz), (-ky,-kz)} (the rank
 * holds +G and -G of every G it owns), largest first onto the rank with the
 * fewest G vectors; rank r holds x planes [plane0[r], plane0[r+1]) with
 * plane0[r] = floor(r n1 / nranks).  A rank's coefficients are C0/C2 arrays
 * [nstate][ngpw_local] (complex FP64, its G vectors in increasing global
 * order, amdk_slab_local_g); its real-space arrays are [nr3][nr2][nplane]
 * FP64 (x fastest, over its planes).
 *
 * Exchange buffers (complex, elem_bytes each: the context's precision at
 * amdk_slab_create): for npairs pairs the send buffer holds npairs *
 * send_elems[r] elements for each rank r, in rank order; the receive buffer
 * npairs * recv_elems[s] elements from each source s, in rank order (what an
 * all-to-all with those counts produces).  The reverse exchange uses the
 * same counts swapped and returns the blocks to where they came from.
 *
 * Per pass over pairs [band0/2, band0/2 + npairs) (band0 even):
 *   amdk_slab_pairs_out      pack + backward x pass of the rank's rays -> send
 *   (all-to-all send -> recv)
 *   amdk_slab_planes_vpsi    y/z passes, V(r) psi, inverse (recv in place);
 *                            v: this rank's slab of V(r), FP64
 *   amdk_slab_planes_density rho(r) (=, or += with accumulate) sum of f/Omega
 *                            |psi|^2 over the pairs' bands on this rank's slab
 *   (all-to-all recv -> back, after planes_vpsi)
 *   amdk_slab_pairs_in       forward x pass + unpack: C2 = -f (|G|^2/2 C0 +
 *                            FFT(V psi)) on the rank's G vectors (vpsi,
 *                            wfn_initialize.f90:283-362, without fnonloc)
 * Pointers are device pointers; stream: a cudaStream_t to launch on
 * (asynchronous), or NULL for the context's stream with the call waited for.
 * A slab object serves one call at a time.  Closed-shell systems on grids
 * with the pencil transforms only; nranks <= 16. */
#define AMDK_SLAB_MAXRANKS 16
typedef struct amdk_slab amdk_slab;
typedef struct {
  int nranks, rank;
  int ngpw_local;         /* plane-wave G vectors of this rank */
  int nray_local;         /* wavefunction x-rays of this rank */
  int plane0, nplane;     /* x planes [plane0, plane0 + nplane) */
  int gzero_local;        /* local index of G = 0, -1 on the other ranks */
  int elem_bytes;         /* bytes per complex element of the exchange buffers */
  long send_elems[AMDK_SLAB_MAXRANKS];  /* per pair, to each rank */
  long recv_elems[AMDK_SLAB_MAXRANKS];  /* per pair, from each rank */
} amdk_slab_info;
/* Host only (no GPU): the owner of every plane-wave G vector (g_owner[ngpw])
 * and the plane ranges (plane0[nranks+1]); either may be NULL. */
int amdk_slab_layout(const amdk_system *sys, int nranks, int *g_owner, int *plane0);
int amdk_slab_create(amdk_ctx *ctx, int nranks, int rank, amdk_slab **out);
int amdk_slab_info_get(amdk_slab *slab, amdk_slab_info *info);
int amdk_slab_local_g(amdk_slab *slab, int *ig);
int amdk_slab_pairs_out(amdk_slab *slab, const double *c0, int band0, int npairs, void *send, void *stream);
int amdk_slab_planes_vpsi(amdk_slab *slab, void *recv, int npairs, const double *v, void *stream);
int amdk_slab_planes_density(amdk_slab *slab, const void *recv, int band0, int npairs, double *rho, int accumulate,
                             void *stream);
int amdk_slab_pairs_in(amdk_slab *slab, void *back, const double *c0, int band0, int npairs, double *c2,
                       void *stream);
/* The rank's share of a band-space Gram matrix (the overlap S of ortho_gs,
 * wfn_initialize.f90:481-482, or Lambda of OVLAP_D): out (n x n, column-major,
 * device) = 2 Re sum over the rank's G of conj(a_i) b_j, less Re a_i(0) Re b_j(0)
 * on the rank that holds G = 0, for bands 0..n-1 of the rank's arrays a and b
 * ([nstate][ngpw_local] complex, device); the sum over ranks (an all-reduce) is
 * the whole matrix.  FP64 tensor-core product; waits for its stream; uses the
 * context's split buffer, so it does not run concurrently with the context's
 * own calls.  AMDK_ERR_TIMEOUT if a pipeline wait gave up. */
int amdk_slab_gram(amdk_slab *slab, const double *a, const double *b, int n, double *out, void *stream);
int amdk_slab_destroy(amdk_slab *slab);

#ifdef __cplusplus
}
#endif
#endif
