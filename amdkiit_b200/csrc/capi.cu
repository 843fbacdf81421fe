// libamdk: device context and the extern "C" entry points of include/amdk.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <queue>
#include <type_traits>
#include <string>
#include <vector>

#include "amdk_internal.h"
#include "fft.cuh"
#include "kernels.cuh"
#include "pencil.cuh"
#include "slicegemm.cuh"
#include "dgemm.cuh"

#include <cudaTypedefs.h>

namespace amdk {

static thread_local std::string g_err;
void set_error(const std::string &m) { g_err = m; }

#define CK(x)                                                                                     \
  do {                                                                                            \
    cudaError_t e_ = (x);                                                                         \
    if (e_ != cudaSuccess) {                                                                      \
      set_error(std::string("CUDA: ") + cudaGetErrorString(e_) + " at " + __FILE__ + ":" +        \
                std::to_string(__LINE__));                                                        \
      return AMDK_ERR_CUDA;                                                                       \
    }                                                                                             \
  } while (0)
#define RC(x)                    \
  do {                           \
    int r_ = (x);                \
    if (r_) return r_;           \
  } while (0)

template <typename T> static int dalloc(T **p, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
  if (e != cudaSuccess) {
    set_error(std::string("cudaMalloc failed: ") + cudaGetErrorString(e) + " (" + std::to_string(n * sizeof(T)) + " bytes)");
    return AMDK_ERR_ALLOC;
  }
  return 0;
}
// setup upload; a pageable-source cudaMemcpy may return before its DMA has
// landed, and the context's streams do not wait for the legacy stream, so the
// copy is waited for here
template <typename T> static int upload(T **p, const std::vector<T> &v) {
  RC(dalloc(p, v.size()));
  if (!v.empty()) {
    CK(cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    CK(cudaStreamSynchronize(0));
  }
  return 0;
}

}  // namespace amdk

using namespace amdk;

// one profiled interval: kernel class, algorithmic bytes, events around it
struct ProfRec {
  int kind;
  double bytes;
  cudaEvent_t a, b;
};

struct amdk_ctx {
  HostSetup hs;
  int device = 0, precision = AMDK_FP64, batch = 4;
  cudaStream_t st = nullptr;
  // the blocked Cholesky of overlaps too large for one SM: work copy, block row
  double *d_cholw = nullptr, *d_cholt = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms = 0;
  // geometry / FFT
  Geom geom;
  Plan<double2> pd[3];
  Plan<float2> pf[3];
  std::vector<void *> allocs;
  int *d_gmap = nullptr, *d_posp = nullptr, *d_posm = nullptr, *d_zlist[2] = {}, *d_rayidx[2] = {};
  int *d_inyh = nullptr;
  double *d_hg = nullptr, *d_gvec = nullptr;
  long rb_elems_pw = 0, sb_elems_pw = 0, rb_elems_rho = 0, sb_elems_rho = 0;
  void *d_rb = nullptr, *d_sb = nullptr;
  void *d_rbf = nullptr;  // ray buffer of the density-sphere fields
  // side stream for the work that needs only C0 (projections, E_kin, C2
  // clearing), overlapped with the density and the potential
  cudaStream_t st2 = nullptr;
  double *d_part2 = nullptr;
  // FP64 tensor-core GEMMs: split-K partial tiles (one buffer per stream)
  // and the poll limit of their pipeline waits (options.reserved[1])
  double *d_dgpart = nullptr, *d_dgpart2 = nullptr;
  long dg_plim = SG_SPIN;
  cudaEvent_t ev_fork = nullptr, ev_side_done = nullptr;
  size_t fftbuf_bytes = 0;
  // tables
  double *d_vps = nullptr, *d_rhos = nullptr, *d_twnl = nullptr, *d_vpp = nullptr, *d_wsg = nullptr;
  int *d_na = nullptr, *d_ngh = nullptr, *d_zv = nullptr;
  double2 *d_evps = nullptr, *d_erhos = nullptr;
  double *d_atarg = nullptr, *d_atco = nullptr;
  int *d_isa_is = nullptr, *d_isa_ia = nullptr;
  // projectors (compact list)
  int nproj = 0;
  std::vector<int> p_isa, p_is, p_iv, p_l;
  int *d_pisa = nullptr, *d_pis = nullptr, *d_piv = nullptr, *d_pl = nullptr;
  double2 *d_P = nullptr, *d_Q = nullptr;
  double *d_H = nullptr, *d_nl = nullptr, *d_hn = nullptr, *d_D = nullptr, *d_dfnl = nullptr;
  // electronic state
  int nstate = 0, npairs = 0;
  double *d_occ = nullptr, *d_wa = nullptr, *d_wb = nullptr;
  // open shell (LSD): the spin-2 pair weights, density and potentials
  double *d_wa2 = nullptr, *d_wb2 = nullptr, *d_rho2 = nullptr, *d_vpot2 = nullptr;
  void *d_vt2 = nullptr;
  double2 *d_c0 = nullptr, *d_c2 = nullptr, *d_cp = nullptr, *d_hnm1 = nullptr;
  double *d_rho = nullptr, *d_vpot = nullptr;
  double2 *d_rhog = nullptr, *d_vg = nullptr, *d_vxg = nullptr, *d_fp = nullptr, *d_fm = nullptr, *d_cgrid = nullptr;
  double *d_gam = nullptr, *d_uinv = nullptr;
  int *d_info = nullptr;
  double *d_part = nullptr, *d_scal = nullptr, *d_force = nullptr, *d_esr = nullptr, *d_fsr = nullptr;
  unsigned *d_ticket = nullptr;  // tickets of the self-finishing reductions (TK_*)
  // pencil path (cubic grids with a specialised length): tables and buffers
  bool pencil_vpsi = false, pencil_density = false;
  double *h_pin = nullptr;  // pinned: scalar slots [S_NSCAL], GEMAX, CG step
  // CUDA graphs of the CG iteration's two segments (before and after the
  // GEMAX read), keyed by segment, precision/forces flag, which buffer holds
  // C0, and profiling
  struct SegGraph {
    cudaGraph_t graph = nullptr;  // kept: an ensemble launches it as a child graph
    cudaGraphExec_t exec = nullptr;
    std::vector<ProfRec> recs;
    size_t nevents = 0;
    long nlaunch = 0;
  };
  std::map<std::array<int, 4>, SegGraph> graphs;
  bool use_graphs = true;
  bool tune = true;  // measure launch shapes at first use (AMDK_NO_TUNE=1: model only)
  bool overlap = true;  // C0-only work on the side stream (AMDK_NO_OVERLAP=1: one stream)
  // integer-slice tensor-core GEMMs of the mixed path (<= 128 bands;
  // AMDK_NO_SLICE=1: DGEMM/DTRMM as the FP64 path)
  bool slice_gemm = true, sg_ready = false;
  int8_t *d_plA = nullptr, *d_plB = nullptr, *d_plS = nullptr;  // C0, C2, small-matrix digit planes
  double *d_sgA = nullptr, *d_sgB = nullptr, *d_sgS = nullptr;  // their row (column) scales
  double *d_sgpart = nullptr;
  unsigned long long *d_sgmax = nullptr;  // per-band max |x| of the slicing pass
  unsigned long long *d_c2max = nullptr;  // per-band max |x| of C2, recorded by the H|psi> unpack
  bool c2max_ok = false;                  // d_c2max belongs to the current C2
  double *d_sgnsq = nullptr;               // per-band sums of squares (by segment) of the slicing pass
  int *d_sgerr = nullptr;
  long sg_kpad = 0;
  long sg_plim = SG_SPIN;  // poll limit of the slice kernels' pipeline waits (options.reserved[0])
  int sg_ktiles = 0, sg_per = 0, sg_chunks = 0, sg_mtiles = 0;
  void *sg_c0_buf = nullptr;  // the C0 buffer whose digit planes are in d_plA (written by the ortho)
  // projector planes (mixed path, nproj <= 128; 3 nproj <= 128 for the dbeta rows):
  // P and Q = -i G_k P sliced once per geometry, for fnl and D_FNL on the tensor cores
  bool sg_proj = false, sg_dproj = false;
  int8_t *d_plP = nullptr, *d_plQ = nullptr;
  double *d_sgP = nullptr, *d_sgQ = nullptr;
  CUtensorMap tm_p_tn, tm_q_tn;
  CUtensorMap tm_a_tn, tm_b_tn, tm_a_nn, tm_s_nn;
  bool warm[2] = {false, false};  // an eager iteration has run at this pair precision
  void *c0_first = nullptr;       // the buffer that held C0 at creation
  // BOMD predictor: converged C0 of earlier steps, most recent first
  static constexpr int MAX_PRED = 8;
  double2 *d_hist[MAX_PRED] = {};
  int nhist = 0;                                  // steps stored
  int pred_npts = 2;                              // points per prediction, C0(t) included
  double pred_coef[MAX_PRED] = {2.0, -1.0};       // weights of C0(t), C0(t-dt), ...
  bool pred_user = false;                         // coefficients given by the caller
  int *h_info = nullptr;    // pinned: Cholesky status
  int pencil_groups = 1;  // upper bound on the density pair groups
  int ct_vpsi = 0, ct_dens = 0;  // column tiles of the pencil kernels (current precision)
  int ns_dens = 1;               // register slots of the density kernel's sums (tiles x task rounds)
  int nsd_p[2] = {1, 1};
  bool pv_p[2] = {false, false}, pd_p[2] = {false, false};  // per pair precision: FP64, mixed
  int ctv_p[2] = {0, 0}, ctd_p[2] = {0, 0};
  int pn1 = 0, pn2 = 0;          // two-level split n = pn1 * pn2
  int nsm = 148;
  // one resident wave of the streaming reductions (blocks per SM x SMs)
  int red_ekin = RED_BLOCKS, red_gmax = RED_BLOCKS;
  std::map<int, int> pencil_grp_cache;
  int vpsi_tuned[2] = {0, 0};  // batch size the V(r)psi column tile was measured for, per precision
  PencilGeom pg{};
  int *d_rpos = nullptr, *d_gmapt = nullptr, *d_zinv = nullptr, *d_postp = nullptr, *d_postm = nullptr;
  double *d_rhopart = nullptr;
  void *d_vt = nullptr;
  // live per-kernel timing (CUDA events on the context stream)
  long nlaunch = 0;  // kernels of this library launched on the context stream
  bool prof = false;
  typedef ProfRec Rec;
  std::vector<Rec> recs;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> evpool;
  size_t evused = 0;
  long kt_count[8] = {0};
  double kt_ms[8] = {0}, kt_bytes[8] = {0};
  // host copies of scalars
  double esr = 0, eself = 0;
  bool tfor = false;
  bool have_prev_g = false;

  template <typename T> int alloc(T **p, size_t n) {
    RC(dalloc(p, n));
    allocs.push_back((void *)*p);
    return 0;
  }
  template <typename T> int up(T **p, const std::vector<T> &v) {
    RC(amdk::upload(p, v));
    allocs.push_back((void *)*p);
    return 0;
  }
};

// kernel classes timed in profiling mode
enum { KT_ZVPSI = 0, KT_ZDENS, KT_Y, KT_X, KT_UNPACK, KT_DGEMM, KT_OTHER, KT_N };

// an event record that is also a node of a graph being captured (a plain
// record inside a capture is only a dependency marker)
static void prof_record(amdk_ctx *c, cudaEvent_t ev) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(c->st, &st);
  if (st == cudaStreamCaptureStatusActive) cudaEventRecordWithFlags(ev, c->st, cudaEventRecordExternal);
  else cudaEventRecord(ev, c->st);
}
static void prof_begin(amdk_ctx *c, int kind, double bytes) {
  if (!c->prof) return;
  if (c->evused == c->evpool.size()) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    c->evpool.push_back({a, b});
  }
  auto &e = c->evpool[c->evused++];
  prof_record(c, e.first);
  c->recs.push_back({kind, bytes, e.first, e.second});
}
static void prof_end(amdk_ctx *c) {
  if (!c->prof) return;
  prof_record(c, c->recs.back().b);
}
// after a stream synchronisation: fold the recorded intervals into the totals
static void prof_harvest(amdk_ctx *c) {
  if (!c->prof) return;
  for (auto &r : c->recs) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, r.a, r.b) != cudaSuccess) {
      cudaGetLastError();  // a failed interval is dropped, not left as a sticky error
      continue;
    }
    c->kt_count[r.kind]++;
    c->kt_ms[r.kind] += ms;
    c->kt_bytes[r.kind] += r.bytes;
  }
  c->recs.clear();
  c->evused = 0;
}


static int nblk(long n, int t = NTHR) { return (int)std::min<long>((n + t - 1) / t, 1L << 30); }

template <typename C> static int make_plan(amdk_ctx *c, int n, Plan<C> &p) {
  int m = n, nf = 0;
  int f[MAXF];
  while (m % 4 == 0) { f[nf++] = 4; m /= 4; }
  while (m % 2 == 0) { f[nf++] = 2; m /= 2; }
  while (m % 3 == 0) { f[nf++] = 3; m /= 3; }
  while (m % 5 == 0) { f[nf++] = 5; m /= 5; }
  if (m != 1 || nf > MAXF) {
    set_error("FFT length " + std::to_string(n) + " is not 2,3,5-smooth");
    return AMDK_ERR_UNSUPPORTED;
  }
  p.n = n;
  p.nf = nf;
  for (int i = 0; i < nf; i++) p.f[i] = f[i];
  std::vector<C> w(n);
  const double tp = 8.0 * std::atan(1.0);
  for (int k = 0; k < n; k++) {
    double a = -tp * (double)k / (double)n;
    w[k].x = (decltype(w[k].x))std::cos(a);
    w[k].y = (decltype(w[k].x))std::sin(a);
  }
  C *d;
  RC(c->up(&d, w));
  p.w = d;
  return 0;
}

// ------------------------------------------------------------------ FFT driver
// FFT lengths with compile-time specialised kernels (the grid sizes of the
// reference's set_r_grids for the configurations of interest); any other
// 2,3,5-smooth length runs the run-time-length kernels.
template <typename F> static void with_n(int n, F &&f) {
  switch (n) {
#define AMDK_NCASE(v) \
  case v: f(std::integral_constant<int, v>{}); break;
    AMDK_NCASE(36) AMDK_NCASE(48) AMDK_NCASE(60) AMDK_NCASE(64) AMDK_NCASE(72) AMDK_NCASE(80) AMDK_NCASE(90) AMDK_NCASE(96)
    AMDK_NCASE(100) AMDK_NCASE(108) AMDK_NCASE(120) AMDK_NCASE(128) AMDK_NCASE(144) AMDK_NCASE(160)
#undef AMDK_NCASE
    default: f(std::integral_constant<int, 0>{}); break;
  }
}
// opt every kernel instantiation into the large dynamic shared memory once
// (one flag per kernel: the kernel itself is the template argument)
template <auto K> static void smem_opt_in() {
  static bool done = []() {
    cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    return true;
  }();
  (void)done;
}

// shared memory of the slab-path kernels: two tiles and the twiddle tables (2n)
template <typename C> static size_t x_smem(int n1) { return 2 * (size_t)n1 * (LX + 1) * sizeof(C) + 2 * n1 * sizeof(C); }
template <typename C> static size_t yz_smem(int n) { return 2 * (size_t)n * TX * sizeof(C) + 2 * n * sizeof(C); }

template <typename C> static void set_smem_attrs() {
  int mx = 227 * 1024;
  cudaFuncSetAttribute(k_x_bwd_pair<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_x_bwd_field<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_x_fwd<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_y<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_z<C, Z_TO_GRID>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_z<C, Z_FROM_GRID_REAL>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_z<C, Z_FROM_GRID_CPLX>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_z<C, Z_VPSI>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_z<C, Z_DENSITY>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
}

template <typename C> static const Plan<C> &plan(amdk_ctx *c, int d);
template <> const Plan<double2> &plan<double2>(amdk_ctx *c, int d) { return c->pd[d]; }
template <> const Plan<float2> &plan<float2>(amdk_ctx *c, int d) { return c->pf[d]; }

// ray buffer of a sphere: band pairs (0) or density-sphere fields (1)
static void *rays(amdk_ctx *c, int sphere) { return sphere ? c->d_rbf : c->d_rb; }

// strides of the FFT buffers for transforms of a sphere
static long rstride(amdk_ctx *c, int sphere) { return (long)c->geom.nray[sphere] * c->geom.n1; }
static long sstride(amdk_ctx *c, int sphere) { return (long)c->geom.nz[sphere] * c->geom.n2 * c->geom.n1; }

// Ray and slab buffers of a slab-path transform; null members select the
// context's own (the allocation-free entry passes its fixed scratch instead).
struct XBufs {
  void *rays = nullptr;
  void *slab = nullptr;
};
static void *rays_of(amdk_ctx *c, int sphere, const XBufs &b) { return b.rays ? b.rays : rays(c, sphere); }
static void *slab_of(amdk_ctx *c, const XBufs &b) { return b.slab ? b.slab : c->d_sb; }

template <typename C> static void y_pass(amdk_ctx *c, int sphere, int dir, int T, const XBufs &b = XBufs{}) {
  const Geom &g = c->geom;
  dim3 grid((g.n1 + TX - 1) / TX, g.nz[sphere], T);
  prof_begin(c, KT_Y, (double)T * (rstride(c, sphere) + sstride(c, sphere)) * sizeof(C));
  ++c->nlaunch;
  with_n(g.n2, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    smem_opt_in<k_y<C, N>>();
    k_y<C, N><<<grid, NTHR, yz_smem<C>(g.n2), c->st>>>(sphere, dir, g, plan<C>(c, 1), (C *)rays_of(c, sphere, b),
                                                      (C *)slab_of(c, b), rstride(c, sphere), sstride(c, sphere));
  });
  prof_end(c);
}
template <typename C, int MODE>
static void z_pass(amdk_ctx *c, int sphere, int T, double2 *cg, const double *rg, int pair0 = 0,
                   const XBufs &b = XBufs{}) {
  const Geom &g = c->geom;
  dim3 grid((g.n1 + TX - 1) / TX, g.n2, MODE == Z_DENSITY ? 1 : T);
  long gs = (long)g.n1 * g.n2 * g.n3;
  // algorithmic bytes: slab planes in (and out for VPSI), V once, rho read+write once
  double slab = (double)T * sstride(c, sphere) * sizeof(C);
  if (MODE == Z_VPSI) prof_begin(c, KT_ZVPSI, 2.0 * slab + gs * 8.0);
  else if (MODE == Z_DENSITY) prof_begin(c, KT_ZDENS, slab + 2.0 * gs * 8.0);
  else prof_begin(c, KT_OTHER, 0.0);
  ++c->nlaunch;
  with_n(g.n3, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    smem_opt_in<k_z<C, MODE, N>>();
    k_z<C, MODE, N><<<grid, NTHR, yz_smem<C>(g.n3), c->st>>>(sphere, T, g, plan<C>(c, 2), (C *)slab_of(c, b),
                                                             sstride(c, sphere), cg, rg, gs, c->d_vpot, c->d_rho,
                                                             c->d_wa + pair0, c->d_wb + pair0);
  });
  prof_end(c);
}
template <typename C> static void x_fwd(amdk_ctx *c, int sphere, int T, const XBufs &b = XBufs{}) {
  const Geom &g = c->geom;
  long lines = (long)T * g.nray[sphere];
  prof_begin(c, KT_X, 2.0 * lines * g.n1 * sizeof(C));
  ++c->nlaunch;
  with_n(g.n1, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    smem_opt_in<k_x_fwd<C, N>>();
    k_x_fwd<C, N><<<nblk(lines, LX), NTHR, x_smem<C>(g.n1), c->st>>>(sphere, T, g, plan<C>(c, 0),
                                                                     (C *)rays_of(c, sphere, b));
  });
  prof_end(c);
}

// T fields on the density sphere (fp at +G, fm at -G) -> real or complex
// grids (FP64 in and out; C is the precision of the transform itself)
template <typename C = double2>
static int field_to_grid(amdk_ctx *c, int T, const double2 *fp, const double2 *fm, double2 *cgrid,
                         const XBufs &b = XBufs{}) {
  const Geom &g = c->geom;
  long lines = (long)T * g.nray[1];
  ++c->nlaunch;
  with_n(g.n1, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    smem_opt_in<k_x_bwd_field<C, N>>();
    k_x_bwd_field<C, N><<<nblk(lines, LX), NTHR, x_smem<C>(g.n1), c->st>>>(fp, fm, g.ngrho, 1, T, g, plan<C>(c, 0),
                                                                         (C *)rays_of(c, 1, b));
  });
  y_pass<C>(c, 1, +1, T, b);
  z_pass<C, Z_TO_GRID>(c, 1, T, cgrid, nullptr, 0, b);
  return 0;
}
// T complex grids (or one real grid) -> forward transform left in the ray buffer
template <typename C = double2>
static int grid_to_rays(amdk_ctx *c, int T, const double2 *cgrid, const double *rgrid, const XBufs &b = XBufs{}) {
  if (rgrid) z_pass<C, Z_FROM_GRID_REAL>(c, 1, 1, nullptr, rgrid, 0, b);
  else z_pass<C, Z_FROM_GRID_CPLX>(c, 1, T, (double2 *)cgrid, nullptr, 0, b);
  y_pass<C>(c, 1, -1, T, b);
  x_fwd<C>(c, 1, T, b);
  return 0;
}

// ------------------------------------------------------------------ pencil path
// shared memory of a pencil block: slab plane, column tile of ct columns,
// the twiddle tables (2n, from a 16-byte boundary) and the packed slab-plane
// table (16 bytes for each of at most 16 j2)
template <typename C> static size_t pencil_smem(int n, int nz, int ct) {
  return (((size_t)(nz + ct) * (n + 1) * sizeof(C) + 15) & ~(size_t)15) + 2 * (size_t)n * sizeof(C) + 16 * 16;
}
// widest column tile with the block within `budget` bytes (0: none fits)
template <typename C> static int pencil_tile(int n, int nz, size_t extra, size_t budget) {
  const size_t base = pencil_smem<C>(n, nz, 0) + extra;
  if (base >= budget) return 0;
  const int widest = (int)std::min<size_t>(n, (budget - base) / ((n + 1) * sizeof(C)));
  if (widest <= 0) return 0;
  const int tiles = (n + widest - 1) / widest;  // equal tiles
  return (n + tiles - 1) / tiles;
}
// Column tiles of the density pencil kernel: the fewest equal tiles (1, 2 or
// 4) whose block fits the shared memory of two blocks per SM (else of one),
// whose group sums fit 1, 2 or 4 register slots (tiles x rounds of PNT
// tasks) and whose final staging of the sums (n x (n+1) reals) fits over the
// plane and the tile.  ct = 0 when none does.
static void density_tiles(int n, int nz, size_t csize, size_t lim, int *ct, int *ns) {
  *ct = 0;
  *ns = 1;
  const int n1f = fft_n1(n);
  for (size_t budget : {lim / 2, lim})
    for (int tiles : {1, 2, 4}) {
      const int w = (n + tiles - 1) / tiles;
      const size_t smem = (((size_t)(nz + w) * (n + 1) * csize + 15) & ~(size_t)15) + 2 * (size_t)n * csize + 16 * 16;
      const int reps = (w * n1f + PNT - 1) / PNT;
      const int slots = tiles * reps;
      const bool stage_ok = (size_t)n * (n + 1) * (csize / 2) <= (size_t)(nz + w) * (n + 1) * csize;
      if (smem <= budget && stage_ok && (slots == 1 || slots == 2 || slots == 4) && (n + w - 1) / w == tiles) {
        *ct = w;
        *ns = slots;
        return;
      }
    }
}
template <typename C> static size_t xt_smem(int n1) { return ((size_t)XL * (n1 + 1) + 2 * n1) * sizeof(C); }
// Pair groups of the density pencil kernel: each (x-plane, group) block sums
// its group's pairs into its own partial grid.  Pick the group count whose
// block list, scheduled greedily on the SMs, ends first; each group also
// costs one partial grid written and read back.
static int pencil_density_groups(int n1, int T, int nsm, int bps, int maxg) {
  int best = 1;
  double best_cost = 1e300;
  for (int grp = 1; grp <= std::min(maxg, T); ++grp) {
    const int per = (T + grp - 1) / grp;
    if ((grp - 1) * per >= T) continue;  // an empty group
    std::priority_queue<double, std::vector<double>, std::greater<double>> slots;
    for (int i = 0; i < nsm * bps; ++i) slots.push(0.0);
    double end = 0.0;
    for (int gi = 0; gi < grp; ++gi) {
      const int np = std::min(T, (gi + 1) * per) - gi * per;
      for (int kx = 0; kx < n1; ++kx) {
        double t0 = slots.top();
        slots.pop();
        double t1 = t0 + (np + 0.5) / bps;
        end = std::max(end, t1);
        slots.push(t1);
      }
    }
    const double cost = end + 0.3 * grp;
    if (cost < best_cost) {
      best_cost = cost;
      best = grp;
    }
  }
  return best;
}

template <typename C> static void xt_bwd_pair(amdk_ctx *c, int p0, int T) {
  const Geom &g = c->geom;
  long lines = (long)T * g.nray[0];
  with_n(g.n1, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    if constexpr (N > 0) {
      smem_opt_in<k_xt_bwd_pair<C, N>>();
      ++c->nlaunch;
      constexpr int N2 = N / fft_n1(N);
      k_xt_bwd_pair<C, N><<<nblk(lines, XL), XL * N2, xt_smem<C>(N), c->st>>>(c->d_c0, c->hs.ngpw, c->nstate, 2 * p0, T,
                                                                             c->pg, plan<C>(c, 0), (C *)c->d_rb);
    }
  });
}
template <typename C> static void xt_fwd(amdk_ctx *c, int T) {
  const Geom &g = c->geom;
  long lines = (long)T * g.nray[0];
  prof_begin(c, KT_X, 2.0 * lines * g.n1 * sizeof(C));
  with_n(g.n1, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    if constexpr (N > 0) {
      smem_opt_in<k_xt_fwd<C, N>>();
      ++c->nlaunch;
      constexpr int N2 = N / fft_n1(N);
      k_xt_fwd<C, N><<<nblk(lines, XL), XL * N2, xt_smem<C>(N), c->st>>>(T, c->pg, plan<C>(c, 0), (C *)c->d_rb);
    }
  });
  prof_end(c);
}
// ------------------------------------------------------------------ tuning
// Launch shapes measured at first use (AMDK_NO_TUNE=1: the model's choice
// instead) are kept per context and, when AMDK_TUNE_CACHE names a file, in
// that JSON object of "key": value pairs (keys name the kernel, precision,
// grid, slab planes and batch), so that later contexts and processes reuse
// them without measuring.
static std::mutex g_tune_mu;
static std::map<std::string, int> g_tune;
static bool g_tune_loaded = false;
static const char *tune_path() {
  const char *p = getenv("AMDK_TUNE_CACHE");
  return (p && *p) ? p : nullptr;
}
static void tune_load_locked() {
  if (g_tune_loaded) return;
  g_tune_loaded = true;
  const char *path = tune_path();
  if (!path) return;
  FILE *f = std::fopen(path, "r");
  if (!f) return;
  std::string txt;
  char buf[4096];
  size_t nr;
  while ((nr = std::fread(buf, 1, sizeof(buf), f)) > 0) txt.append(buf, nr);
  std::fclose(f);
  size_t i = 0;
  while ((i = txt.find('"', i)) != std::string::npos) {
    const size_t j = txt.find('"', i + 1);
    if (j == std::string::npos) break;
    const size_t k = txt.find(':', j);
    if (k == std::string::npos) break;
    g_tune[txt.substr(i + 1, j - i - 1)] = (int)std::strtol(txt.c_str() + k + 1, nullptr, 10);
    i = txt.find_first_of(",}", k);
    if (i == std::string::npos) break;
  }
}
static bool tune_get(const std::string &key, int *v) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  tune_load_locked();
  auto it = g_tune.find(key);
  if (it == g_tune.end()) return false;
  *v = it->second;
  return true;
}
static void tune_put(const std::string &key, int v) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  tune_load_locked();
  g_tune[key] = v;
  const char *path = tune_path();
  if (!path) return;
  const std::string tmp = std::string(path) + ".tmp";
  FILE *f = std::fopen(tmp.c_str(), "w");
  if (!f) return;
  std::fprintf(f, "{\n");
  size_t n = 0;
  for (auto &kv : g_tune) std::fprintf(f, "  \"%s\": %d%s\n", kv.first.c_str(), kv.second, ++n < g_tune.size() ? "," : "");
  std::fprintf(f, "}\n");
  std::fclose(f);
  std::rename(tmp.c_str(), path);
}
// key of a tuned pencil launch shape
static std::string pencil_key(const amdk_ctx *c, const char *what, int T) {
  const Geom &g = c->geom;
  return std::string(what) + "/" + (c->precision == AMDK_MIXED ? "mixed" : "fp64") + "/" + std::to_string(g.n1) + "x" +
         std::to_string(g.n2) + "x" + std::to_string(g.n3) + "/nz" + std::to_string(c->pg.nz) + "/T" + std::to_string(T);
}

// pairs [p0, p0 + T) of the ray buffer rb; open shell: each pair with its
// spin's potential (the pair straddling the spins with both)
template <typename C, int N> static void launch_pencil_vpsi(amdk_ctx *c, int T, int ct, C *rb, int p0 = 0) {
  typedef decltype(C().x) Rl;
  const size_t sm = pencil_smem<C>(N, c->pg.nz, ct);
  ++c->nlaunch;
  if (c->hs.lsd) {
    const int nu = c->hs.nel_up, psplit = (nu + 1) / 2, pstr = (nu & 1) ? nu / 2 : -1;
    smem_opt_in<k_pencil_vpsi<C, N, true>>();
    k_pencil_vpsi<C, N, true><<<dim3(c->geom.n1, T), PNT, sm, c->st>>>(
        c->pg, plan<C>(c, 1), rb, (const Rl *)c->d_vt, ct, (const Rl *)c->d_vt2, p0, psplit, pstr);
  } else {
    smem_opt_in<k_pencil_vpsi<C, N>>();
    k_pencil_vpsi<C, N><<<dim3(c->geom.n1, T), PNT, sm, c->st>>>(c->pg, plan<C>(c, 1), rb, (const Rl *)c->d_vt, ct,
                                                                nullptr, 0, 0, -1);
  }
}
// Column-tile width of the V(r)psi pencil kernel for T pairs: measured once
// per shape (every width ceil(N/t), t = 1..6, whose block fits, launched on a
// scratch copy of the ray buffer, which the kernel transforms in place),
// from the tuning cache, or the model's choice (capture, AMDK_NO_TUNE=1).
template <typename C, int N> static int vpsi_tile(amdk_ctx *c, int T) {
  const std::string key = pencil_key(c, "pencil_vpsi_tile", T);
  const int q = (c->precision == AMDK_MIXED) ? 1 : 0;
  int best = c->ctv_p[q];
  if (c->vpsi_tuned[q] == T) return best;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(c->st, &cap);
  if (cap != cudaStreamCaptureStatusNone || !c->tune) return best;
  int cached = 0;
  if (tune_get(key, &cached) && cached >= 8 && pencil_smem<C>(N, c->pg.nz, cached) <= 227 * 1024) {
    best = cached;
  } else {
    const size_t bytes = (size_t)T * rstride(c, 0) * sizeof(C);
    C *scratch = nullptr;
    if (cudaMalloc(&scratch, bytes) == cudaSuccess) {
      cudaMemcpyAsync(scratch, c->d_rb, bytes, cudaMemcpyDeviceToDevice, c->st);
      cudaEvent_t e0, e1;
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      const long nl = c->nlaunch;
      float best_ms = 1e30f;
      int prev = 0;
      for (int t = 1; t <= 6; ++t) {
        const int w = (N + t - 1) / t;
        if (w == prev || w < 8 || pencil_smem<C>(N, c->pg.nz, w) > 227 * 1024) continue;
        prev = w;
        launch_pencil_vpsi<C, N>(c, T, w, scratch);  // warm
        cudaEventRecord(e0, c->st);
        launch_pencil_vpsi<C, N>(c, T, w, scratch);
        launch_pencil_vpsi<C, N>(c, T, w, scratch);
        cudaEventRecord(e1, c->st);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) {
          best_ms = ms;
          best = w;
        }
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      cudaStreamSynchronize(c->st);
      cudaFree(scratch);
      c->nlaunch = nl;  // tuning launches are not part of the work
      tune_put(key, best);
    }
    cudaGetLastError();
  }
  c->ctv_p[q] = best;
  c->ct_vpsi = best;
  c->vpsi_tuned[q] = T;
  return best;
}
template <typename C> static void pencil_vpsi(amdk_ctx *c, int T, int p0 = 0) {
  const Geom &g = c->geom;
  typedef decltype(C().x) Rl;
  const double npt = (double)g.n1 * g.n2 * g.n3;
  with_n(g.n2, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    if constexpr (N > 0) {
      const int ct = vpsi_tile<C, N>(c, T);
      prof_begin(c, KT_ZVPSI, 2.0 * T * rstride(c, 0) * sizeof(C) + npt * sizeof(Rl));
      launch_pencil_vpsi<C, N>(c, T, ct, (C *)c->d_rb, p0);
      prof_end(c);
    }
  });
}
template <typename C, int N, int NS> static void launch_pencil_density_ns(amdk_ctx *c, int p0, int T, int grp, int add) {
  const Geom &g = c->geom;
  const size_t sm = pencil_smem<C>(N, c->pg.nz, c->ct_dens);
  ++c->nlaunch;
  if (grp < 0) {  // balanced schedule, -grp blocks (one batch of pairs)
    smem_opt_in<k_pencil_density_bal<C, N, NS>>();
    k_pencil_density_bal<C, N, NS><<<-grp, PNT, sm, c->st>>>(c->pg, plan<C>(c, 1), (const C *)c->d_rb, T, c->d_wa + p0,
                                                             c->d_wb + p0, c->d_rhopart, c->ct_dens);
    return;
  }
  const int per = (T + grp - 1) / grp;
  smem_opt_in<k_pencil_density<C, N, NS>>();
  k_pencil_density<C, N, NS><<<dim3(g.n1, grp), PNT, sm, c->st>>>(c->pg, plan<C>(c, 1), (const C *)c->d_rb, T, per,
                                                                  c->d_wa + p0, c->d_wb + p0, c->d_rhopart, c->ct_dens,
                                                                  add);
}
template <typename C> static void launch_pencil_density(amdk_ctx *c, int p0, int T, int grp, int add) {
  with_n(c->geom.n2, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    if constexpr (N > 0) {
      if (c->ns_dens == 1) launch_pencil_density_ns<C, N, 1>(c, p0, T, grp, add);
      else if (c->ns_dens == 2) launch_pencil_density_ns<C, N, 2>(c, p0, T, grp, add);
      else launch_pencil_density_ns<C, N, 4>(c, p0, T, grp, add);
    }
  });
}
// rho (FP64 grid) from the partial grids of a density schedule (grp > 0
// groups per plane, grp < 0 the balanced schedule of -grp blocks over T pairs)
static void reduce_density(amdk_ctx *c, int grp, int T, double *rho) {
  const Geom &g = c->geom;
  ++c->nlaunch;
  k_rho_reduce_p<<<dim3((g.n1 + 31) / 32, (g.n1 + 31) / 32, g.n1), dim3(32, 8), 0, c->st>>>(
      g.n1, g.n1, c->pn1, c->pn2, grp > 0 ? grp : 0, c->d_rhopart, rho, 0, grp < 0 ? T : 0, grp < 0 ? -grp : 0);
}
// most partial grids a plane takes under the balanced schedule of nblk blocks
static int bal_max_slots(int n1, int T, int nblk) {
  int m = 0;
  for (int kx = 0; kx < n1; ++kx) m = std::max(m, bal_slots(kx, T, (long)n1 * T, nblk));
  return m;
}
// Pair groups of the density pencil kernel for T pairs at the current
// precision: measured once (every candidate launched on the current buffers,
// whose contents do not matter for the timing; the partial grids are cleared
// before use), then cached.  Inside a graph capture the schedule model's
// choice is used instead.
template <typename C> static int density_groups(amdk_ctx *c, int T) {
  const Geom &g = c->geom;
  const size_t sm = pencil_smem<C>(g.n2, c->pg.nz, c->ct_dens);
  const int key = 2 * T + (c->precision == AMDK_MIXED ? 1 : 0);
  auto it = c->pencil_grp_cache.find(key);
  if (it != c->pencil_grp_cache.end()) return it->second;
  int best = pencil_density_groups(g.n1, T, c->nsm, (int)std::max<size_t>(1, (228 * 1024) / (sm + 1024)),
                                   c->pencil_groups);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(c->st, &cap);
  const std::string tkey = pencil_key(c, "pencil_density_groups_with_reduce", T) + "/ct" +
                           std::to_string(c->ct_dens) + "/ns" + std::to_string(c->ns_dens);
  // the balanced schedule (negative values: -blocks) for a batch that holds
  // every pair, with at most pencil_groups partial grids per plane
  auto bal_ok = [&](int nblk) {
    return T == c->npairs && nblk >= 1 && (long)nblk <= (long)g.n1 * T &&
           bal_max_slots(g.n1, T, nblk) <= c->pencil_groups;
  };
  int cached = 0;
  if (cap == cudaStreamCaptureStatusNone && c->tune && tune_get(tkey, &cached) &&
      ((cached >= 1 && cached <= std::min(c->pencil_groups, T)) || (cached < 0 && bal_ok(-cached)))) {
    best = cached;
  } else if (cap == cudaStreamCaptureStatusNone && c->tune) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const long nl = c->nlaunch;
    float best_ms = 1e30f;
    // each candidate timed with the reduction of its partial grids: more
    // groups spread the blocks better but leave more grids to add
    auto run = [&](int grp) {
      launch_pencil_density<C>(c, 0, T, grp, 0);
      reduce_density(c, grp, T, c->d_rho);
    };
    // (plane, pair group) blocks, then the balanced schedule with one, two or
    // three waves of resident blocks
    std::vector<int> cands = {1, 2, 3, 4, 5, 6, 8, 10, 12, 16};
    const int bps = (int)std::min<size_t>(sizeof(C) == sizeof(float2) ? 2 : 1,
                                          std::max<size_t>(1, (228 * 1024) / (sm + 1024)));
    for (int w = 1; w <= 3; ++w)
      if (bal_ok(w * bps * c->nsm)) cands.push_back(-w * bps * c->nsm);
    for (int grp : cands) {
      if (grp > 0 && (grp > c->pencil_groups || grp > T || (grp - 1) * ((T + grp - 1) / grp) >= T))
        continue;  // no empty group
      run(grp);  // warm
      float ms = 1e30f;
      for (int rep = 0; rep < 3; ++rep) {  // the fastest of three (another context may share the GPU)
        cudaEventRecord(e0, c->st);
        run(grp);
        cudaEventRecord(e1, c->st);
        cudaEventSynchronize(e1);
        float m1 = 0;
        cudaEventElapsedTime(&m1, e0, e1);
        ms = std::min(ms, m1);
      }
      if (ms < best_ms) {
        best_ms = ms;
        best = grp;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->nlaunch = nl;  // tuning launches are not part of the work
    tune_put(tkey, best);
  }
  c->pencil_grp_cache.emplace(key, best);
  return best;
}
template <typename C> static void pencil_density(amdk_ctx *c, int p0, int T) {
  const Geom &g = c->geom;
  const int grp = density_groups<C>(c, T);
  const double npt = (double)g.n1 * g.n2 * g.n3;
  const int add = p0 > 0;
  // partial grids written: groups per plane, or about one per block and plane boundary
  const double grids = grp > 0 ? (double)grp : 1.0 + (double)(-grp) / g.n1;
  prof_begin(c, KT_ZDENS, (double)T * rstride(c, 0) * sizeof(C) + (1.0 + add) * grids * npt * 8.0);
  launch_pencil_density<C>(c, p0, T, grp, add);
  prof_end(c);
}

// ------------------------------------------------------------------ routines

template <typename C> static int density_pairs_t(amdk_ctx *c) {
  const HostSetup &h = c->hs;
  const Geom &g = c->geom;
  if (c->pencil_density) {
    // pencil path: transposed x pass, then one block per (x-plane, pair group)
    // the first batch stores its groups' partial grids, later batches add;
    // groups that only later batches use are cleared first
    const int ng_full = density_groups<C>(c, c->batch);
    const int ng_rem = (c->npairs % c->batch) ? density_groups<C>(c, c->npairs % c->batch) : 0;
    // the balanced schedule (ng_full < 0) runs only when one batch holds
    // every pair: each plane's partial grids are all written, none cleared
    const int ng = ng_full < 0 ? ng_full : std::max(ng_full, ng_rem);
    const int ng_first = c->npairs < c->batch ? ng_rem : ng_full;
    const size_t npt = (size_t)g.n1 * g.n2 * g.n3;
    if (ng > ng_first)
      CK(cudaMemsetAsync(c->d_rhopart + (size_t)ng_first * npt, 0, sizeof(double) * (ng - ng_first) * npt, c->st));
    for (int p0 = 0; p0 < c->npairs; p0 += c->batch) {
      int T = std::min(c->batch, c->npairs - p0);
      xt_bwd_pair<C>(c, p0, T);
      pencil_density<C>(c, p0, T);
    }
    reduce_density(c, ng, c->npairs, c->d_rho);
    if (h.lsd) {
      // open shell: the spin-2 density from the same pair transforms, weighted
      // by the spin-2 bands only (density.f90:64-76); with all pairs in one
      // batch the ray buffer still holds them
      if (ng > ng_first)
        CK(cudaMemsetAsync(c->d_rhopart + (size_t)ng_first * npt, 0, sizeof(double) * (ng - ng_first) * npt, c->st));
      std::swap(c->d_wa, c->d_wa2);
      std::swap(c->d_wb, c->d_wb2);
      for (int p0 = 0; p0 < c->npairs; p0 += c->batch) {
        int T = std::min(c->batch, c->npairs - p0);
        if (c->batch < c->npairs) xt_bwd_pair<C>(c, p0, T);
        pencil_density<C>(c, p0, T);
      }
      std::swap(c->d_wa, c->d_wa2);
      std::swap(c->d_wb, c->d_wb2);
      reduce_density(c, ng, c->npairs, c->d_rho2);
    }
  } else {
  CK(cudaMemsetAsync(c->d_rho, 0, sizeof(double) * (size_t)g.n1 * g.n2 * g.n3, c->st));
  for (int p0 = 0; p0 < c->npairs; p0 += c->batch) {
    int T = std::min(c->batch, c->npairs - p0);
    long lines = (long)T * g.nray[0];
    ++c->nlaunch;
    with_n(g.n1, [&](auto NC) {
      constexpr int N = decltype(NC)::value;
      smem_opt_in<k_x_bwd_pair<C, N>>();
      k_x_bwd_pair<C, N><<<nblk(lines, LX), NTHR, x_smem<C>(g.n1), c->st>>>(c->d_c0, h.ngpw, c->nstate, 2 * p0, T, g,
                                                                           plan<C>(c, 0), (C *)c->d_rb);
    });
    y_pass<C>(c, 0, +1, T);
    z_pass<C, Z_DENSITY>(c, 0, T, nullptr, nullptr, p0);
  }
  }
  CK(cudaGetLastError());
  return 0;
}
// rhor2g (density.f90:128-150), in the pair transforms' precision
template <typename C> static int rhor2g_t(amdk_ctx *c) {
  const HostSetup &h = c->hs;
  const Geom &g = c->geom;
  RC(grid_to_rays<C>(c, 1, nullptr, c->d_rho));
  double scale = 1.0 / ((double)g.n1 * g.n2 * g.n3);
  ++c->nlaunch;
  k_gather_p<C><<<nblk(h.ngrho), NTHR, 0, c->st>>>(h.ngrho, c->d_posp, (C *)c->d_rbf, scale, c->d_rhog);
  CK(cudaGetLastError());
  return 0;
}

template <typename C> static int density_t(amdk_ctx *c) {
  RC(density_pairs_t<C>(c));
  return rhor2g_t<C>(c);
}
static int do_density(amdk_ctx *c) {
  if (c->precision == AMDK_MIXED) return density_t<float2>(c);
  return density_t<double2>(c);
}

// V(r) (real part of a complex grid) into vpot and, on the pencil path, its
// permuted copy vt for the V(r)psi kernel
static int store_potential(amdk_ctx *c, const double2 *grid, double *vpot, void *vt) {
  const Geom &g = c->geom;
  const long npt = (long)g.n1 * g.n2 * g.n3;
  CK(cudaMemcpy2DAsync(vpot, sizeof(double), grid, sizeof(double2), sizeof(double), npt, cudaMemcpyDeviceToDevice,
                       c->st));
  if (c->pencil_vpsi) {
    dim3 gt((g.n1 + 31) / 32, (g.n1 + 31) / 32, g.n1);
    ++c->nlaunch;
    if (c->precision == AMDK_MIXED)
      k_v_permute<float><<<gt, dim3(32, 8), 0, c->st>>>(g.n1, g.n1, c->pn1, c->pn2, vpot, (float *)vt);
    else
      k_v_permute<double><<<gt, dim3(32, 8), 0, c->st>>>(g.n1, g.n1, c->pn1, c->pn2, vpot, (double *)vt);
  }
  return 0;
}

// Open shell (LDA): both spins start from V_H + V_loc of the total density
// (potential.f90:43); the polarized XC of rho_a = rho - rho2, rho_b = rho2
// (xc.f90:135-246) gives v1a, v1b, and each spin's potential is band limited
// through the density sphere as the closed-shell one (xc.f90:302-425).
template <typename C> static int potential_lsd_t(amdk_ctx *c) {
  const HostSetup &h = c->hs;
  const Geom &g = c->geom;
  const long npt = (long)g.n1 * g.n2 * g.n3;
  double2 *g0 = c->d_cgrid, *g1 = c->d_cgrid + npt;
  ++c->nlaunch;
  if (sizeof(C) == sizeof(float2))
    k_xc_lsd<float><<<RED_BLOCKS, NTHR, 0, c->st>>>(npt, c->d_rho, c->d_rho2, g0, g1, c->d_part, c->d_scal + S_EXC,
                                                   c->d_ticket + TK_XC);
  else
    k_xc_lsd<double><<<RED_BLOCKS, NTHR, 0, c->st>>>(npt, c->d_rho, c->d_rho2, g0, g1, c->d_part,
                                                    c->d_scal + S_EXC, c->d_ticket + TK_XC);
  RC(grid_to_rays<C>(c, 2, c->d_cgrid, nullptr));
  const double scale = 1.0 / (double)npt;
  // both spins' G-space potentials first (the ray buffer holds both fields)
  double2 *vx[2] = {c->d_vxg, c->d_fp + h.ngrho}, *vm[2] = {c->d_fm, c->d_fm + h.ngrho};
  for (int sp = 0; sp < 2; ++sp) {
    ++c->nlaunch;
    k_xc_combine<C><<<nblk(h.ngrho), NTHR, 0, c->st>>>(h.ngrho, 0, c->d_posp, c->d_posm,
                                                       (const C *)c->d_rbf + (size_t)sp * rstride(c, 1), rstride(c, 1),
                                                       scale, c->d_gvec, h.tpiba, c->d_vg, vx[sp]);
    ++c->nlaunch;
    k_conj_field<<<nblk(h.ngrho), NTHR, 0, c->st>>>(h.ngrho, vx[sp], vm[sp]);
  }
  for (int sp = 0; sp < 2; ++sp) {
    RC(field_to_grid<C>(c, 1, vx[sp], vm[sp], c->d_cgrid));
    RC(store_potential(c, c->d_cgrid, sp ? c->d_vpot2 : c->d_vpot, sp ? c->d_vt2 : c->d_vt));
  }
  CK(cudaGetLastError());
  return 0;
}

// eval_pot + cal_vpot_ex; the density-sphere transforms run in the pair
// transforms' precision (FP32 on the mixed path, which ends on FP64)
template <typename C> static int potential_t(amdk_ctx *c) {
  const HostSetup &h = c->hs;
  const Geom &g = c->geom;
  long npt = (long)g.n1 * g.n2 * g.n3;
  // eval_pot in G space and E_H, E_loc sums
  ++c->nlaunch;
  k_vloc_g<<<RED_BLOCKS, NTHR, 0, c->st>>>(h.ngrho, c->d_hg, h.tpiba2, c->d_rhog, c->d_erhos, c->d_evps, c->d_vg,
                                           c->d_part, c->d_scal + S_EH, c->d_ticket + TK_VLOC);
  int gga = (h.xc == AMDK_XC_PBE);
  double2 *g0 = c->d_cgrid, *g1 = c->d_cgrid + npt;
  if (h.lsd) return potential_lsd_t<C>(c);
  if (gga) {
    ++c->nlaunch;
    k_grad_fields<<<nblk(h.ngrho), NTHR, 0, c->st>>>(h.ngrho, c->d_gvec, h.tpiba, c->d_rhog, c->d_fp, c->d_fm);
    RC(field_to_grid<C>(c, 2, c->d_fp, c->d_fm, c->d_cgrid));
  }
  ++c->nlaunch;
  // the functional in the transforms' precision (FP32 on the mixed path)
  if (sizeof(C) == sizeof(float2))
    k_xc<float><<<RED_BLOCKS, NTHR, 0, c->st>>>(npt, h.xc, c->d_rho, g0, g1, c->d_part, c->d_scal + S_EXC,
                                               c->d_ticket + TK_XC);
  else
    k_xc<double><<<RED_BLOCKS, NTHR, 0, c->st>>>(npt, h.xc, c->d_rho, g0, g1, c->d_part, c->d_scal + S_EXC,
                                                c->d_ticket + TK_XC);
  RC(grid_to_rays<C>(c, gga ? 2 : 1, c->d_cgrid, nullptr));
  double scale = 1.0 / (double)npt;
  ++c->nlaunch;
  k_xc_combine<C><<<nblk(h.ngrho), NTHR, 0, c->st>>>(h.ngrho, gga, c->d_posp, c->d_posm, (C *)c->d_rbf, rstride(c, 1),
                                                     scale, c->d_gvec, h.tpiba, c->d_vg, c->d_vxg);
  ++c->nlaunch;
  k_conj_field<<<nblk(h.ngrho), NTHR, 0, c->st>>>(h.ngrho, c->d_vxg, c->d_fm);
  RC(field_to_grid<C>(c, 1, c->d_vxg, c->d_fm, c->d_cgrid));
  // V(r) = Re of the backward transform (xc.f90:299-301), and V in the
  // x-plane-major layout the pencil kernel reads
  RC(store_potential(c, c->d_cgrid, c->d_vpot, c->d_vt));
  CK(cudaGetLastError());
  return 0;
}
static int do_potential(amdk_ctx *c) {
  if (c->precision == AMDK_MIXED) return potential_t<float2>(c);
  return potential_t<double2>(c);
}

static bool use_slice(const amdk_ctx *c);
// The unpack of pairs [p0, p0+T) (kinetic term, occupation scaling) fused
// with fnonloc for the first UNPACK_NPJ projectors; further projectors are
// added in chunks (k_fnonloc_add).  pp/pm: +G/-G positions in the ray buffer.
template <typename C> static void unpack_h(amdk_ctx *c, int p0, int T, const int *pp, const int *pm) {
  typedef decltype(C().x) Rl;
  const HostSetup &h = c->hs;
  const Geom &g = c->geom;
  const double scale = 1.0 / ((double)g.n1 * g.n2 * g.n3);
  const int npj0 = std::min(c->nproj, UNPACK_NPJ);
  const int nb = std::min(2 * T, c->nstate - 2 * p0);
  // per-band maxima of C2 for its slicing (int8 products of the mixed path)
  unsigned long long *bmax = use_slice(c) ? c->d_c2max + 2 * p0 : nullptr;
  if (bmax && p0 == 0) cudaMemsetAsync(c->d_c2max, 0, sizeof(unsigned long long) * SG_M, c->st);
  ++c->nlaunch;
  constexpr int PAIRS = unpack_pairs<C>();
  const dim3 gu(nblk(h.ngpw, 128), (T + PAIRS - 1) / PAIRS);
  k_unpack_fnonloc<C><<<gu, 128, (size_t)2 * PAIRS * npj0 * sizeof(Rl), c->st>>>(
      h.ngpw, c->nstate, 2 * p0, T, npj0, pp, pm, (const C *)c->d_rb, rstride(c, 0), scale, c->d_hg, h.tpiba2,
      c->d_occ, c->d_P, c->d_D, c->nproj, c->d_c0, c->d_c2, c->nproj > npj0 ? nullptr : bmax, 0);
  // with projector chunks still to add, C2 is sliced from scratch
  c->c2max_ok = bmax != nullptr && c->nproj <= npj0;
  for (int j0 = npj0; j0 < c->nproj; j0 += UNPACK_NPJ) {
    const int npj = std::min(UNPACK_NPJ, c->nproj - j0);
    smem_opt_in<k_fnonloc_add<UNPACK_NPJ>>();
    ++c->nlaunch;
    const dim3 ga(nblk(h.ngpw, 128), (nb + FNL_BANDS - 1) / FNL_BANDS);
    k_fnonloc_add<UNPACK_NPJ><<<ga, 128, (size_t)FNL_BANDS * npj * sizeof(double), c->st>>>(
        h.ngpw, 2 * p0, nb, j0, npj, c->d_P, c->d_D, c->nproj, c->d_c2);
  }
}

// vpsi + fnonloc: C2 = -f H C0 (C2 is written, not accumulated)
template <typename C> static int apply_h_t(amdk_ctx *c) {
  const HostSetup &h = c->hs;
  const Geom &g = c->geom;
  if (c->pencil_vpsi) {
    for (int p0 = 0; p0 < c->npairs; p0 += c->batch) {
      int T = std::min(c->batch, c->npairs - p0);
      xt_bwd_pair<C>(c, p0, T);
      pencil_vpsi<C>(c, T, p0);
      xt_fwd<C>(c, T);
      unpack_h<C>(c, p0, T, c->d_postp, c->d_postm);
    }
    CK(cudaGetLastError());
    return 0;
  }
  for (int p0 = 0; p0 < c->npairs; p0 += c->batch) {
    int T = std::min(c->batch, c->npairs - p0);
    long lines = (long)T * g.nray[0];
    ++c->nlaunch;
    with_n(g.n1, [&](auto NC) {
      constexpr int N = decltype(NC)::value;
      smem_opt_in<k_x_bwd_pair<C, N>>();
      k_x_bwd_pair<C, N><<<nblk(lines, LX), NTHR, x_smem<C>(g.n1), c->st>>>(c->d_c0, h.ngpw, c->nstate, 2 * p0, T, g,
                                                                           plan<C>(c, 0), (C *)c->d_rb);
    });
    y_pass<C>(c, 0, +1, T);
    z_pass<C, Z_VPSI>(c, 0, T, nullptr, nullptr);
    y_pass<C>(c, 0, -1, T);
    x_fwd<C>(c, 0, T);
    unpack_h<C>(c, p0, T, c->d_posp, c->d_posm);
  }
  CK(cudaGetLastError());
  return 0;
}

// fnl (pseudopotential.f90:164-226): nl = 2 P^T C0; hn = H nl
// ------------------------------------------------- integer-slice GEMMs
// Mixed path with at most 128 bands: Lambda, S, C2 -= C0 Lambda and C0 U^{-1}
// on the int8 tensor cores (slicegemm.cuh) instead of DGEMM/DTRMM.
static bool use_slice(const amdk_ctx *c) { return c->sg_ready && c->slice_gemm && c->precision == AMDK_MIXED; }
// the driver's tensor-map encoder (nullptr, with the error set, if absent)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
  if (!enc) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
      set_error("cuTensorMapEncodeTiled not available");
      return nullptr;
    }
    enc = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  }
  return enc;
}
// 2D map of S digit planes (kdim bytes per row, S*128 rows): box box_x x 128
static int sg_encode(CUtensorMap *m, void *base, long kdim, int box_x, CUtensorMapSwizzle sw) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return AMDK_ERR_CUDA;
  cuuint64_t dims[2] = {(cuuint64_t)kdim, (cuuint64_t)SG_S * SG_M};
  cuuint64_t strides[1] = {(cuuint64_t)kdim};
  cuuint32_t box[2] = {(cuuint32_t)box_x, (cuuint32_t)SG_M};
  cuuint32_t es[2] = {1, 1};
  if (enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed");
    return AMDK_ERR_CUDA;
  }
  return 0;
}
static int sg_setup(amdk_ctx *c) {
  const HostSetup &h = c->hs;
  const char *ns = getenv("AMDK_NO_SLICE");
  c->slice_gemm = !(ns && ns[0] == '1');
  // below 64 bands the products are small and the slicing launches cost more
  // than they save (water1: 4 bands, 3250 vs 3800 SCF iter/s)
  if (h.nstate > SG_M || h.nstate < 64) return 0;
  const long K = 2L * h.ngpw;
  c->sg_kpad = (K + SG_M - 1) / SG_M * SG_M;
  c->sg_ktiles = (int)(c->sg_kpad / SG_TN_KT);
  c->sg_per = (c->sg_ktiles + c->nsm - 1) / c->nsm;
  c->sg_chunks = (c->sg_ktiles + c->sg_per - 1) / c->sg_per;
  c->sg_mtiles = (int)(c->sg_kpad / SG_M);
  const size_t pl = (size_t)SG_S * SG_M * c->sg_kpad;
  RC(c->alloc(&c->d_plA, pl));
  RC(c->alloc(&c->d_plB, pl));
  RC(c->alloc(&c->d_plS, (size_t)SG_S * SG_M * SG_M));
  RC(c->alloc(&c->d_sgA, SG_M));
  RC(c->alloc(&c->d_sgB, SG_M));
  RC(c->alloc(&c->d_sgS, SG_M));
  RC(c->alloc(&c->d_sgpart, (size_t)c->sg_chunks * SG_M * SG_M));
  RC(c->alloc(&c->d_sgmax, SG_M));
  RC(c->alloc(&c->d_c2max, SG_M));
  RC(c->alloc(&c->d_sgnsq, (size_t)SG_M * SG_SEG));
  c->d_sgerr = c->d_info + 1;
  RC(sg_encode(&c->tm_a_tn, c->d_plA, c->sg_kpad, SG_TN_KT, CU_TENSOR_MAP_SWIZZLE_64B));
  RC(sg_encode(&c->tm_b_tn, c->d_plB, c->sg_kpad, SG_TN_KT, CU_TENSOR_MAP_SWIZZLE_64B));
  RC(sg_encode(&c->tm_a_nn, c->d_plA, c->sg_kpad, SG_M, CU_TENSOR_MAP_SWIZZLE_128B));
  RC(sg_encode(&c->tm_s_nn, c->d_plS, SG_M, SG_M, CU_TENSOR_MAP_SWIZZLE_128B));
  CK(cudaFuncSetAttribute(k_sgemm_tn<SG_S>, cudaFuncAttributeMaxDynamicSharedMemorySize, SgTn<SG_S>::SMEM));
  CK(cudaFuncSetAttribute(k_sgemm_nn<SG_S, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, SgNn<SG_S>::SMEM));
  CK(cudaFuncSetAttribute(k_sgemm_nn<SG_S, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, SgNn<SG_S>::SMEM));
  CK(cudaFuncSetAttribute(k_sgemm_nn<SG_S, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, SgNn<SG_S>::SMEM));
  c->sg_ready = true;
  return 0;
}
// digit planes and row scales of the first nrows rows of x (C0, C2 or a
// projector matrix; rows up to 128 are planes of zeros)
static void sg_slice(amdk_ctx *c, const double2 *x, int8_t *planes, double *scale, int nrows = -1) {
  const long K = 2L * c->hs.ngpw;
  if (nrows < 0) nrows = c->nstate;
  c->nlaunch += 2;
  cudaMemsetAsync(c->d_sgmax, 0, sizeof(unsigned long long) * SG_M, c->st);
  k_band_absmax<<<dim3(SG_SEG, nrows), 256, 0, c->st>>>((const double *)x, K, K, nrows, c->d_sgmax, c->d_sgnsq);
  k_slice_rows<SG_S><<<dim3(SG_SEG, SG_M), 256, 0, c->st>>>((const double *)x, K, K, nrows, c->d_sgmax, planes,
                                                            c->sg_kpad, scale);
}
// out (nm x n, leading dimension ldo) = alpha diag(sa) A B^T diag(sb), the
// product over the real index; n = nstate columns (B = C0 or C2 planes)
static void sg_tn(amdk_ctx *c, const CUtensorMap &ta, const CUtensorMap &tb, int same, const double *sa,
                  const double *sb, double alpha, double *out, int nm = -1, int ldo = -1) {
  const int n = c->nstate;
  if (nm < 0) nm = n;
  if (ldo < 0) ldo = n;
  c->nlaunch += 2;
  k_sgemm_tn<SG_S><<<c->sg_chunks, SG_TN_THREADS, SgTn<SG_S>::SMEM, c->st>>>(ta, tb, same, c->sg_ktiles, c->sg_per, c->d_sgpart,
                                                                     c->d_sgerr, c->sg_plim);
  k_sgemm_reduce<<<n, SG_RG * SG_M, 0, c->st>>>(c->sg_chunks, c->d_sgpart, nm, sa, sb, same ? c->d_sgnsq : nullptr,
                                            alpha, out, ldo);
}
// projector planes: set up once the projector count is known (mixed-capable
// contexts with slice products)
static int sg_proj_setup(amdk_ctx *c) {
  if (!c->sg_ready || c->nproj == 0 || c->nproj > SG_M) return 0;
  const size_t pl = (size_t)SG_S * SG_M * c->sg_kpad;
  RC(c->alloc(&c->d_plP, pl));
  RC(c->alloc(&c->d_sgP, SG_M));
  RC(sg_encode(&c->tm_p_tn, c->d_plP, c->sg_kpad, SG_TN_KT, CU_TENSOR_MAP_SWIZZLE_64B));
  c->sg_proj = true;
  if (3 * c->nproj <= SG_M) {
    RC(c->alloc(&c->d_plQ, pl));
    RC(c->alloc(&c->d_sgQ, SG_M));
    RC(sg_encode(&c->tm_q_tn, c->d_plQ, c->sg_kpad, SG_TN_KT, CU_TENSOR_MAP_SWIZZLE_64B));
    c->sg_dproj = true;
  }
  return 0;
}
// C0's digit planes are those of the current C0 (written by the last ortho)
static bool c0_planes_current(const amdk_ctx *c) { return c->sg_c0_buf == (const void *)c->d_c0; }
// out (the real view, 2 ngpw x n) = (or -=, sub) C0 B for B n x n, with C0's
// planes and scales in d_plA / d_sgA.  With digits (an orthonormalisation)
// the result's own planes replace C0's in d_plA, scale 2 (|x| <= 1).
static void sg_nn(amdk_ctx *c, const double *B, double2 *out, int sub, bool digits) {
  const int n = c->nstate;
  const long K = 2L * c->hs.ngpw;
  c->nlaunch += 2;
  k_slice_small<SG_S><<<SG_M, SG_M, 0, c->st>>>(B, n, n, n, c->d_sgA, c->d_plS, c->d_sgS);
  const dim3 grid(std::min(c->sg_mtiles, c->nsm));
  if (sub)
    k_sgemm_nn<SG_S, 1><<<grid, SG_NN_THREADS, SgNn<SG_S>::SMEM, c->st>>>(
        c->tm_a_nn, c->tm_s_nn, c->sg_mtiles, K, (double *)out, K, n, c->d_sgS, nullptr, c->sg_kpad, c->d_sgerr, c->sg_plim);
  else if (digits)
    k_sgemm_nn<SG_S, 2><<<grid, SG_NN_THREADS, SgNn<SG_S>::SMEM, c->st>>>(
        c->tm_a_nn, c->tm_s_nn, c->sg_mtiles, K, (double *)out, K, n, c->d_sgS, c->d_plA, c->sg_kpad, c->d_sgerr, c->sg_plim);
  else
    k_sgemm_nn<SG_S, 0><<<grid, SG_NN_THREADS, SgNn<SG_S>::SMEM, c->st>>>(
        c->tm_a_nn, c->tm_s_nn, c->sg_mtiles, K, (double *)out, K, n, c->d_sgS, nullptr, c->sg_kpad, c->d_sgerr, c->sg_plim);
  if (digits) {
    ++c->nlaunch;
    k_sg_fill<<<1, SG_M, 0, c->st>>>(c->d_sgA, n, 2.0);
  }
}

// ------------------------------------------------- FP64 tensor-core GEMMs
// 2D map of a column-major FP64 matrix, dim0 x dim1 (dim0 contiguous, the
// leading dimension), box box0 x box1
static int dg_encode(CUtensorMap *m, const void *base, long dim0, long dim1, int box0, int box1, CUtensorMapSwizzle sw) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return AMDK_ERR_CUDA;
  cuuint64_t dims[2] = {(cuuint64_t)dim0, (cuuint64_t)dim1};
  cuuint64_t strides[1] = {(cuuint64_t)dim0 * sizeof(double)};
  cuuint32_t box[2] = {(cuuint32_t)box0, (cuuint32_t)box1};
  cuuint32_t es[2] = {1, 1};
  if (enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void *>(base), dims, strides, box, es,
          CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled (FP64) failed");
    return AMDK_ERR_CUDA;
  }
  return 0;
}
// split-K partial tiles a TN product of m x n needs at most (buffer size)
static size_t dg_part_doubles(const amdk_ctx *c, int m, int n) {
  const size_t ntile = (size_t)((m + DG_T - 1) / DG_T) * ((n + DG_T - 1) / DG_T);
  return (2 * (size_t)c->nsm + ntile) * DG_T * DG_T;
}
// out (m x n, leading dimension ldo) = alpha A^T B over the real index
// K = 2 ngpw; A (K x m) and B (K x n) are the real views of complex band or
// projector arrays.  sym: B = A, only the upper tiles are formed and the
// result is mirrored.
static int dg_tn(amdk_ctx *c, const void *A, int m, const void *B, int n, double alpha, double *out, int ldo,
                 bool sym = false, long Kin = 0, cudaStream_t sin = nullptr) {
  // K: 2 ngpw unless given (a slab rank's 2 ngpw_local); stream: the context's unless given
  const long K = Kin > 0 ? Kin : 2L * c->hs.ngpw;
  cudaStream_t st = sin ? sin : c->st;
  CUtensorMap ta, tb;
  RC(dg_encode(&ta, A, K, m, DG_KT, DG_T, CU_TENSOR_MAP_SWIZZLE_128B));
  if (sym)
    tb = ta;
  else
    RC(dg_encode(&tb, B, K, n, DG_KT, DG_T, CU_TENSOR_MAP_SWIZZLE_128B));
  const int mt = (m + DG_T - 1) / DG_T, nt = (n + DG_T - 1) / DG_T;
  const int ntile = sym ? mt * (mt + 1) / 2 : mt * nt;
  const int ktiles = (int)((K + DG_KT - 1) / DG_KT);
  // enough blocks to fill the GPU twice, but at least 8 k tiles each (a short
  // block costs its pipeline fill, and every split is a partial tile to add)
  int nsplit = std::max(1, std::min((ktiles + 7) / 8, (2 * c->nsm + ntile - 1) / ntile));
  const int per = (ktiles + nsplit - 1) / nsplit;
  nsplit = (ktiles + per - 1) / per;
  c->nlaunch += 2;
  k_dgemm_tn<<<dim3(ntile, nsplit), DG_THREADS, DG_TN_SMEM, st>>>(ta, tb, m, n, mt, sym ? 1 : 0, ktiles, per, c->d_dgpart,
                                                                 c->d_info + 1, c->dg_plim);
  k_dgemm_tn_sum<<<(int)std::min<long>((long)ntile * (DG_T * DG_T / 32), 8L * c->nsm), 256, 0, st>>>(
      c->d_dgpart, nsplit, ntile, mt, sym ? 1 : 0, m, n, alpha, out, ldo);
  CK(cudaGetLastError());
  return 0;
}
// out (K x n, the real view of a complex band array) = alpha A G + beta out,
// A the real view of n1 bands, G n1 x n (leading dimension n1); upper: G is
// upper triangular (its lower part is not read)
static int dg_nn(amdk_ctx *c, const void *A, int n1, const double *G, int n, double alpha, double beta, bool upper,
                 void *out) {
  const long K = 2L * c->hs.ngpw;
  CUtensorMap ta;
  RC(dg_encode(&ta, A, K, n1, 16, DG_NN_BS, CU_TENSOR_MAP_SWIZZLE_128B));
  const long items = ((K + DG_NN_R - 1) / DG_NN_R) * ((n + DG_NN_J - 1) / DG_NN_J);
  ++c->nlaunch;
  k_dgemm_nn<<<(int)std::min<long>(items, c->nsm), DG_NN_THREADS, DG_NN_SMEM, c->st>>>(
      ta, G, n1, K, n1, n, alpha, beta, upper ? 1 : 0, (double *)out, K, c->d_info + 1, c->dg_plim);
  CK(cudaGetLastError());
  return 0;
}

// On the mixed path with the projector planes and C0's current planes: the
// int8 tensor-core slice product (nl = 2 P^T C0, FP32-level accuracy);
// otherwise the FP64 tensor-core product.
static int do_fnl(amdk_ctx *c) {
  if (c->nproj == 0) return 0;
  if (use_slice(c) && c->sg_proj && c0_planes_current(c)) {
    sg_tn(c, c->tm_p_tn, c->tm_a_tn, 0, c->d_sgP, c->d_sgA, 2.0, c->d_nl, c->nproj, c->nproj);
    return 0;
  }
  return dg_tn(c, c->d_P, c->nproj, c->d_c0, c->nstate, 2.0, c->d_nl, c->nproj);
}

// energies from the device scalar slots (copied to the host)
static int fill_energies(amdk_ctx *c, const double *sc, amdk_energies *e) {
  const HostSetup &h = c->hs;
  e->eh = sc[S_EH];
  e->eloc = 2.0 * sc[S_ELOC] * h.omega;
  e->eself = c->eself;
  e->esr = c->esr;
  e->estat = (sc[S_EH] * h.omega) + c->esr - c->eself;
  e->eke = sc[S_EKIN] * h.tpiba2;
  e->exc = h.omega / (double)(h.nr[0] * h.nr[1] * h.nr[2]) * sc[S_EXC];
  e->enl = sc[S_ENL];
  e->etotal = e->enl + e->eloc + e->eke + e->exc + e->estat;
  if (!std::isfinite(e->etotal)) {
    set_error("non-finite total energy");
    return AMDK_ERR_NONFINITE;
  }
  return 0;
}

// pp_energy + e_total.  With e the energies are read back now (one stream
// synchronisation); without, the scalar slots are copied to the pinned host
// buffer in stream order for fill_energies after the caller's own sync.
// the C0-only part of pp_energy/e_total: projections, E_nl, E_kin
static int energy_c0_terms(amdk_ctx *c) {
  const HostSetup &h = c->hs;
  RC(do_fnl(c));
  if (c->nproj) {
    ++c->nlaunch;
    k_nl_energy_d<<<nblk((long)c->nproj * c->nstate), NTHR, 0, c->st>>>(c->nproj, c->nstate, c->d_H, c->d_nl, c->d_hn,
                                                                          c->d_occ, c->d_D, c->d_part,
                                                  c->d_scal + S_ENL, c->d_ticket + TK_ENL);
  } else {
    CK(cudaMemsetAsync(c->d_scal + S_ENL, 0, sizeof(double), c->st));
  }
  ++c->nlaunch;
  k_ekin<<<c->red_ekin, NTHR, 0, c->st>>>(h.ngpw, c->nstate, c->d_c0, c->d_hg, c->d_occ, c->d_part,
                                         c->d_scal + S_EKIN, c->d_ticket + TK_EKIN);
  return 0;
}
static int do_energy(amdk_ctx *c, amdk_energies *e) {
  RC(energy_c0_terms(c));
  CK(cudaMemcpyAsync(c->h_pin, c->d_scal, sizeof(double) * S_NSCAL, cudaMemcpyDeviceToHost, c->st));
  if (e) {
    CK(cudaStreamSynchronize(c->st));
    RC(fill_energies(c, c->h_pin, e));
  }
  return 0;
}

static int do_apply_h(amdk_ctx *c) {
  if (c->precision == AMDK_MIXED) return apply_h_t<float2>(c);
  return apply_h_t<double2>(c);
}

// forces (gradient.f90:5-34) and eval_GMAX
// occupied bands (occupation above 1e-5, as eval_GMAX and PCG count them)
static int n_occupied(const amdk_ctx *c) {
  int nocc = 0;
  for (int i = 0; i < c->nstate; i++)
    if (c->hs.occ[i] > 1e-5) nocc++;
  return nocc;
}
// GEMAX and the preconditioned-gradient norm of PCG from the current C2, in
// one pass: S_GMAX and S_GG
static void gmax_precon(amdk_ctx *c) {
  ++c->nlaunch;
  k_gmax_precon<<<c->red_gmax, NTHR, 0, c->st>>>(c->hs.ngpw, n_occupied(c), c->d_vpp, c->d_occ, c->d_c2, c->d_part,
                                                c->d_scal + S_GMAX, c->d_ticket + TK_GRAD);
}

// open shell: zero the entries of an nstate x nstate band matrix that couple
// the two spins (the reference forms the spin blocks separately)
static void spin_mask(amdk_ctx *c, double *A) {
  if (!c->hs.lsd) return;
  const int n = c->nstate;
  ++c->nlaunch;
  k_spin_mask<<<nblk((long)n * n), NTHR, 0, c->st>>>(n, c->hs.nel_up, A);
}

static int do_gradient(amdk_ctx *c) {
  const HostSetup &h = c->hs;
  const int n = c->nstate;
  const bool sl = use_slice(c);
  if (sl) {
    if (c->c2max_ok) {
      // the unpack recorded C2's band maxima: only the digit pass
      const long K = 2L * c->hs.ngpw;
      ++c->nlaunch;
      k_slice_rows<SG_S><<<dim3(SG_SEG, SG_M), 256, 0, c->st>>>((const double *)c->d_c2, K, K, c->nstate, c->d_c2max,
                                                                c->d_plB, c->sg_kpad, c->d_sgB);
    } else {
      sg_slice(c, c->d_c2, c->d_plB, c->d_sgB);
    }
    // C0's planes are those the last orthonormalisation wrote, if C0 has not changed since
    if (c->sg_c0_buf != (void *)c->d_c0) sg_slice(c, c->d_c0, c->d_plA, c->d_sgA);
    sg_tn(c, c->tm_b_tn, c->tm_a_tn, 0, c->d_sgB, c->d_sgA, 2.0, c->d_gam);
  } else {
    RC(dg_tn(c, c->d_c2, n, c->d_c0, n, 2.0, c->d_gam, n));
  }
  ++c->nlaunch;
  k_g0_correct<<<dim3(nblk(n), n), NTHR, 0, c->st>>>(n, h.ngpw, c->d_c2, c->d_c0, c->d_gam, c->d_occ, 1, 0);
  spin_mask(c, c->d_gam);
  if (sl)
    sg_nn(c, c->d_gam, c->d_c2, 1, false);
  else
    RC(dg_nn(c, c->d_c0, n, c->d_gam, n, -1.0, 1.0, false, c->d_c2));
  ++c->nlaunch;
  k_zclean<<<nblk(n), NTHR, 0, c->st>>>(n, h.ngpw, c->d_c2);
  c->c2max_ok = false;  // C2 is the projected gradient now
  gmax_precon(c);
  CK(cudaGetLastError());
  return 0;
}

// PCG; the step number goes through pinned host memory and the S_ISTEP slot
// so that a captured graph of this step reads the current one.  The
// gradient norm S_GG is the one do_gradient left for the current C2
// (recompute: form it here, for a caller that changed C2 since).
static int do_pcg(amdk_ctx *c, int istep, bool recompute = false) {
  const HostSetup &h = c->hs;
  c->sg_c0_buf = nullptr;  // C0 changes in place
  c->h_pin[S_NSCAL + 1] = (double)istep;
  CK(cudaMemcpyAsync(c->d_scal + S_ISTEP, c->h_pin + S_NSCAL + 1, sizeof(double), cudaMemcpyHostToDevice, c->st));
  if (recompute) gmax_precon(c);
  ++c->nlaunch;
  k_pcg_update<<<RED_BLOCKS * 4, NTHR, 0, c->st>>>(h.ngpw, c->nstate, c->d_scal, c->d_vpp, c->d_occ, c->d_c2, c->d_hnm1,
                                                   c->d_c0);
  ++c->nlaunch;
  k_copy_scalar<<<1, 1, 0, c->st>>>(c->d_scal + S_GG, c->d_scal + S_GGPREV);
  CK(cudaGetLastError());
  return 0;
}

// ortho_gs.  With check the Cholesky status is read back now; without, it is
// copied to the pinned host buffer in stream order (checked by the caller
// after its own sync with check_ortho).
static int check_ortho(amdk_ctx *c) {
  // an expired wait comes first: its NaN results reach the overlap, whose
  // Cholesky then fails too; the recorded code is cleared once reported
  if (c->h_info[1]) {
    set_error("tensor-core GEMM: a pipeline wait expired (code " + std::to_string(c->h_info[1]) + ")");
    c->h_info[1] = 0;
    CK(cudaMemset(c->d_info + 1, 0, sizeof(int)));
    return AMDK_ERR_TIMEOUT;
  }
  const int info = c->h_info[0];
  if (info) {
    set_error("overlap matrix not positive definite at leading minor " + std::to_string(info));
    return AMDK_ERR_NOT_SPD;
  }
  return 0;
}
// C (m x n, ldc) = alpha op(A) op(B) + beta C for the blocked factorisation
static void small_dgemm(amdk_ctx *c, int ta, int tb, int m, int n, int k, double alpha, const double *A, int lda,
                        const double *B, int ldb, double beta, double *Cm, int ldc) {
  if (m <= 0 || n <= 0) return;
  ++c->nlaunch;
  k_small_dgemm<<<dim3((m + 63) / 64, (n + 63) / 64), 256, 0, c->st>>>(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, Cm,
                                                                      ldc);
}
// Cholesky factor and inverse of the overlap above CHOL_NMAX bands (UINV,
// DPOTRF + DTRTRI, wfn_initialize.f90:504-530), blocked by 128:
// right-looking over a work copy W of S, each diagonal block factored and
// inverted by k_chol_inv_s (X_kk = U_kk^-1 into U^-1's diagonal block), the
// block row U_k,j = X_kk^T S_k,j (j > k) and the trailing update
// S_j,l -= U_k,j^T U_k,l as small products; then the inverse's off-diagonal
// blocks column by column from the bottom, X_i,j = -X_i,i sum_{k=i+1..j}
// U_i,k X_k,j.  All on the context stream (capturable).
static int chol_inv_blocked(amdk_ctx *c, int n) {
  constexpr int BK = 128;
  double *W = c->d_cholw, *T = c->d_cholt, *X = c->d_uinv;
  CK(cudaMemcpyAsync(W, c->d_gam, sizeof(double) * (size_t)n * n, cudaMemcpyDeviceToDevice, c->st));
  CK(cudaMemsetAsync(X, 0, sizeof(double) * (size_t)n * n, c->st));
  const int nb = (n + BK - 1) / BK;
  const size_t sm = ((size_t)BK * (BK + 1) + (size_t)CHOL_B * BK) * sizeof(double);
  for (int kb = 0; kb < nb; ++kb) {
    const int k0 = kb * BK, kn = std::min(BK, n - k0), k1 = k0 + kn, rest = n - k1;
    ++c->nlaunch;
    k_chol_inv_s<<<1, CHOL_NT, sm, c->st>>>(kn, W + k0 + (size_t)n * k0, n, X + k0 + (size_t)n * k0, n, c->d_info, k0,
                                            kb == 0);
    if (rest <= 0) break;
    // block row: T = X_kk^T W[k0:k1, k1:n], then back into W
    small_dgemm(c, 1, 0, kn, rest, kn, 1.0, X + k0 + (size_t)n * k0, n, W + k0 + (size_t)n * k1, n, 0.0, T, kn);
    CK(cudaMemcpy2DAsync(W + k0 + (size_t)n * k1, sizeof(double) * n, T, sizeof(double) * kn, sizeof(double) * kn,
                         rest, cudaMemcpyDeviceToDevice, c->st));
    // trailing matrix (the whole square; only its upper triangle is read later)
    small_dgemm(c, 1, 0, rest, rest, kn, -1.0, W + k0 + (size_t)n * k1, n, W + k0 + (size_t)n * k1, n, 1.0,
                W + k1 + (size_t)n * k1, n);
  }
  for (int jb = 1; jb < nb; ++jb) {
    const int j0 = jb * BK, jn = std::min(BK, n - j0), j1 = j0 + jn;
    for (int ib = jb - 1; ib >= 0; --ib) {
      const int i0 = ib * BK, in = BK, i1 = i0 + in;
      // T = U[i0:i1, i1:j1] X[i1:j1, j0:j1], then X[i0:i1, j0:j1] = -X_ii T
      small_dgemm(c, 0, 0, in, jn, j1 - i1, 1.0, W + i0 + (size_t)n * i1, n, X + i1 + (size_t)n * j0, n, 0.0, T, in);
      small_dgemm(c, 0, 0, in, jn, in, -1.0, X + i0 + (size_t)n * i0, n, T, in, 0.0, X + i0 + (size_t)n * j0, n);
    }
  }
  CK(cudaGetLastError());
  return 0;
}

static int do_ortho(amdk_ctx *c, bool check = true, bool swap = true) {
  const HostSetup &h = c->hs;
  const int n = c->nstate;
  // S = 2 Re C0^T C0 - Re c0(0) Re c0(0)^T  (DSYRK + DGER, wfn_initialize.f90:481-482)
  const bool sl = use_slice(c);
  if (sl) {
    sg_slice(c, c->d_c0, c->d_plA, c->d_sgA);
    sg_tn(c, c->tm_a_tn, c->tm_a_tn, 1, c->d_sgA, c->d_sgA, 2.0, c->d_gam);
  } else {
    RC(dg_tn(c, c->d_c0, n, c->d_c0, n, 2.0, c->d_gam, n, true));
  }
  ++c->nlaunch;
  k_g0_correct<<<dim3(nblk(n), n), NTHR, 0, c->st>>>(n, h.ngpw, c->d_c0, c->d_c0, c->d_gam, c->d_occ, 0, 1);
  spin_mask(c, c->d_gam);
  if (n <= CHOL_NMAX) {
    const int np = (n + CHOL_B - 1) / CHOL_B * CHOL_B;
    const size_t sm = ((size_t)np * (np + 1) + (size_t)CHOL_B * np) * sizeof(double);
    ++c->nlaunch;
    k_chol_inv_s<<<1, CHOL_NT, sm, c->st>>>(n, c->d_gam, n, c->d_uinv, n, c->d_info, 0, 1);
  } else {
    RC(chol_inv_blocked(c, n));
  }
  CK(cudaMemcpyAsync(c->h_info, c->d_info, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->st));
  if (check) {
    CK(cudaStreamSynchronize(c->st));
    RC(check_ortho(c));
  }
  // C0 <- C0 U^{-1} (DTRMM, wfn_initialize.f90:485) out of place into the
  // spare buffer (ZCLEAN there), then the buffers swap roles
  if (sl)
    sg_nn(c, c->d_uinv, c->d_cp, 0, true);
  else
    RC(dg_nn(c, c->d_c0, n, c->d_uinv, n, 1.0, 0.0, true, c->d_cp));
  ++c->nlaunch;
  k_zclean<<<nblk(n), NTHR, 0, c->st>>>(n, h.ngpw, c->d_cp);
  if (swap) std::swap(c->d_c0, c->d_cp);
  // the buffer whose digit planes d_plA holds (set again after a replayed graph)
  c->sg_c0_buf = sl ? (void *)(swap ? c->d_c0 : c->d_cp) : nullptr;
  CK(cudaGetLastError());
  return 0;
}

// exp_igrxfactor and everything that depends on the positions: structure
// factor sums, projector matrix, preconditioner, e_sr energy and forces.
static int do_positions(amdk_ctx *c, const double *atco) {
  HostSetup &h = c->hs;
  h.atco.assign(atco, atco + 3L * h.na_max * h.nsp);
  std::vector<double> arg(3L * h.nat);
  for (int a = 0; a < h.nat; a++) {
    const double *x = atco + 3 * (h.isa_ia[a] + (long)h.na_max * h.isa_is[a]);
    for (int d = 1; d <= 3; d++) {
      double sm = h.b_cell[0 + 3 * (d - 1)] * x[0];
      sm = sm + h.b_cell[1 + 3 * (d - 1)] * x[1];
      sm = sm + h.b_cell[2 + 3 * (d - 1)] * x[2];
      arg[3 * a + d - 1] = h.tpiba * sm;
    }
  }
  CK(cudaMemcpyAsync(c->d_atarg, arg.data(), sizeof(double) * arg.size(), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_atco, h.atco.data(), sizeof(double) * h.atco.size(), cudaMemcpyHostToDevice, c->st));
  AtomArgs aa{c->d_atarg, c->d_isa_is};
  int nh1 = h.nr[0] / 2 + 1, nh2 = h.nr[1] / 2 + 1, nh3 = h.nr[2] / 2 + 1;
  ++c->nlaunch;
  k_sfac_sums<<<nblk(h.ngrho), NTHR, 0, c->st>>>(h.ngrho, h.nat, c->d_inyh, nh1, nh2, nh3, aa, c->d_vps, c->d_rhos,
                                                 c->d_evps, c->d_erhos);
  if (c->nproj) {
    ProjArgs pa{c->d_pisa, c->d_pis, c->d_piv, c->d_pl, h.nghmax};
    ++c->nlaunch;
    k_projectors<<<dim3(nblk(h.ngpw), c->nproj), NTHR, 0, c->st>>>(h.ngpw, c->nproj, c->d_inyh, nh1, nh2, nh3, aa, pa,
                                                                   c->d_twnl, c->d_P);
    // the G_k-weighted projectors of D_FNL (nuclear_grad.f90:314-372)
    ++c->nlaunch;
    k_dproj<<<dim3(nblk(h.ngpw), c->nproj, 3), NTHR, 0, c->st>>>(h.ngpw, c->nproj, c->d_gvec, c->d_P, c->d_Q);
    if (c->sg_proj) sg_slice(c, c->d_P, c->d_plP, c->d_sgP, c->nproj);
    if (c->sg_dproj) sg_slice(c, c->d_Q, c->d_plQ, c->d_sgQ, 3 * c->nproj);
  }
  ++c->nlaunch;
  k_hess<<<nblk(h.ngpw), NTHR, 0, c->st>>>(h.ngpw, c->d_hg, h.tpiba2, c->d_evps, c->d_twnl, h.nsp, h.nghmax, c->d_na,
                                           c->d_ngh, c->d_wsg, c->d_vpp);
  ++c->nlaunch;
  k_esr_par<<<1, NTHR, 0, c->st>>>(h.nat, c->d_isa_is, c->d_isa_ia, h.na_max, c->d_zv, c->d_atco, h.alat, h.symmetry,
                                   c->d_fsr, c->d_esr);
  CK(cudaMemcpyAsync(&c->esr, c->d_esr, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  CK(cudaGetLastError());
  return 0;
}

// e_sr + POTFOR + NLFOR (wfn_opt when tfor, do_opt.f90:98-106)
static int do_ionic_forces(amdk_ctx *c) {
  const HostSetup &h = c->hs;
  size_t fb = sizeof(double) * 3 * h.na_max * h.nsp;
  CK(cudaMemcpyAsync(c->d_force, c->d_fsr, fb, cudaMemcpyDeviceToDevice, c->st));
  const int pnb = 64;
  AtomArgs aa{c->d_atarg, c->d_isa_is};
  int nh1 = h.nr[0] / 2 + 1, nh2 = h.nr[1] / 2 + 1, nh3 = h.nr[2] / 2 + 1;
  double omtp = 2.0 * h.omega * h.tpiba;
  ++c->nlaunch;
  k_potfor<<<dim3(pnb, h.nat), NTHR, 0, c->st>>>(h.ngrho, c->d_inyh, nh1, nh2, nh3, aa, c->d_hg, c->d_gvec, h.tpiba2,
                                                 c->d_rhog, c->d_erhos, c->d_vps, c->d_rhos, omtp, c->d_part);
  if (c->nproj) {
    // dfnl = 2 tpiba Q^T C0: the int8 slice product on the mixed path (C0's
    // planes current), the FP64 tensor-core product otherwise
    const double tfac = 2.0 * h.tpiba;
    if (use_slice(c) && c->sg_dproj && c0_planes_current(c)) {
      sg_tn(c, c->tm_q_tn, c->tm_a_tn, 0, c->d_sgQ, c->d_sgA, tfac, c->d_dfnl, 3 * c->nproj, 3 * c->nproj);
    } else {
      RC(dg_tn(c, c->d_Q, 3 * c->nproj, c->d_c0, c->nstate, tfac, c->d_dfnl, 3 * c->nproj));
    }
  }
  ++c->nlaunch;
  k_force_total<<<h.nat, NTHR, 0, c->st>>>(h.nat, c->nproj, c->nstate, c->d_pisa, c->d_hn, c->d_dfnl, c->d_occ, c->d_part,
                                           pnb, c->d_isa_is, c->d_isa_ia, h.na_max, c->d_force);
  CK(cudaGetLastError());
  return 0;
}

// ------------------------------------------------------------------ setup
// pair-transform precision in use (FP32 band-pair FFTs for AMDK_MIXED)
static void set_pair_precision(amdk_ctx *c, int prec) {
  const int q = (prec == AMDK_MIXED) ? 1 : 0;
  c->precision = prec;
  c->pencil_vpsi = c->pv_p[q];
  c->pencil_density = c->pd_p[q];
  c->ct_vpsi = c->ctv_p[q];
  c->ct_dens = c->ctd_p[q];
  c->ns_dens = c->nsd_p[q];
}

// Ray coordinates (ky, kz) of the density-sphere x-rays in the reference's
// ray numbering (the wavefunction sphere's rays first), and per G vector of
// the density half sphere the position ray*n1 + kx of +G and of -G
// (prepare_fft, fft_interface.f90:262-293).
static void ray_tables(const HostSetup &h, std::vector<int> &ray_ky, std::vector<int> &ray_kz, std::vector<int> &posp,
                       std::vector<int> &posm) {
  const int n1 = h.nr[0], n2 = h.nr[1], n3 = h.nr[2];
  const int nh1 = n1 / 2 + 1, nh2 = n2 / 2 + 1, nh3 = n3 / 2 + 1;
  ray_ky.assign(h.nhrays, 0);
  ray_kz.assign(h.nhrays, 0);
  for (int r = 0; r < h.nhrays; r++) {
    int m = h.msp[r] - 1;
    int i = m % h.nrl[1] + 1, j = m / h.nrl[1] + 1;
    int iy = i - nh2, iz = j - nh3;
    ray_ky[r] = ((iy % n2) + n2) % n2;
    ray_kz[r] = ((iz % n3) + n3) % n3;
  }
  posp.assign(h.ngrho, 0);
  posm.assign(h.ngrho, 0);
  for (int ig = 0; ig < h.ngrho; ig++) {
    int i1 = h.inyh[3L * ig], i2 = h.inyh[3L * ig + 1], i3 = h.inyh[3L * ig + 2];
    int ix = i1 - nh1;
    int rp = h.xrays[(i2 - 1) + (size_t)h.nrl[1] * (i3 - 1)] - 1;
    int rm = h.xrays[(-i2 + 2 * nh2 - 1) + (size_t)h.nrl[1] * (-i3 + 2 * nh3 - 1)] - 1;
    int kxp = ((ix % n1) + n1) % n1, kxm = ((-ix % n1) + n1) % n1;
    posp[ig] = rp * n1 + kxp;
    posm[ig] = rm * n1 + kxm;
  }
}

static int build_device(amdk_ctx *c) {
  HostSetup &h = c->hs;
  Geom &g = c->geom;
  g.n1 = h.nr[0];
  g.n2 = h.nr[1];
  g.n3 = h.nr[2];
  g.ngpw = h.ngpw;
  g.ngrho = h.ngrho;
  g.nray[0] = h.ngrays;
  g.nray[1] = h.nhrays;
  int n1 = g.n1, n2 = g.n2, n3 = g.n3;
  std::vector<int> ray_ky, ray_kz, posp, posm;
  ray_tables(h, ray_ky, ray_kz, posp, posm);
  std::vector<int> gmap((size_t)h.nhrays * n1, 0);
  for (int ig = 0; ig < h.ngrho; ig++) {
    if (ig != 0) gmap[(size_t)posm[ig]] = -(ig + 1);
    gmap[(size_t)posp[ig]] = ig + 1;
  }
  RC(c->up(&c->d_gmap, gmap));
  RC(c->up(&c->d_posp, posp));
  RC(c->up(&c->d_posm, posm));
  for (int S = 0; S < 2; S++) {
    int R = g.nray[S];
    std::vector<int> zi_of(n3, -1), zl;
    for (int r = 0; r < R; r++) zi_of[ray_kz[r]] = 1;
    for (int kz = 0; kz < n3; kz++)
      if (zi_of[kz] > 0) {
        zi_of[kz] = (int)zl.size();
        zl.push_back(kz);
      }
    std::vector<int> ri(zl.size() * (size_t)n2, -1);
    for (int r = 0; r < R; r++) ri[(size_t)zi_of[ray_kz[r]] * n2 + ray_ky[r]] = r;
    g.nz[S] = (int)zl.size();
    RC(c->up(&c->d_zlist[S], zl));
    RC(c->up(&c->d_rayidx[S], ri));
    g.zlist[S] = c->d_zlist[S];
    g.rayidx[S] = c->d_rayidx[S];
  }
  g.gmap = c->d_gmap;
  g.pos_p = c->d_posp;
  g.pos_m = c->d_posm;
  for (int d = 0; d < 3; d++) {
    RC(make_plan<double2>(c, h.nr[d], c->pd[d]));
    RC(make_plan<float2>(c, h.nr[d], c->pf[d]));
  }
  if (n3 * TX > 16 * NTHR) {
    set_error("grid dimension above 256 is not supported");
    return AMDK_ERR_UNSUPPORTED;
  }
  set_smem_attrs<double2>();
  set_smem_attrs<float2>();
  {
    // constant twiddles of the register DFTs: W_R^m = exp(-2 pi i m/R), R = 2..16
    std::vector<double2> twd(CTW_LEN);
    std::vector<float2> twf(CTW_LEN);
    for (int R = 2; R <= 16; ++R)
      for (int m = 0; m < R; ++m) {
        const double ang = 8.0 * std::atan(1.0) * m / R;
        twd[ctw_off(R) + m] = make_double2(std::cos(ang), -std::sin(ang));
        twf[ctw_off(R) + m] = make_float2((float)std::cos(ang), (float)-std::sin(ang));
      }
    CK(cudaMemcpyToSymbol(c_twd, twd.data(), sizeof(double2) * CTW_LEN));
    CK(cudaMemcpyToSymbol(c_twf, twf.data(), sizeof(float2) * CTW_LEN));
  }
  CK(cudaFuncSetAttribute(k_chol_inv_s, cudaFuncAttributeMaxDynamicSharedMemorySize, 216 * 1024));
  // G vectors
  RC(c->up(&c->d_inyh, h.inyh));
  RC(c->up(&c->d_hg, h.hg));
  RC(c->up(&c->d_gvec, h.gvec));
  // electronic state
  c->nstate = h.nstate;
  c->npairs = (h.nstate + 1) / 2;
  size_t cw = (size_t)h.ngpw * h.nstate;
  RC(c->alloc(&c->d_c0, cw));
  RC(c->alloc(&c->d_c2, cw));
  RC(c->alloc(&c->d_cp, cw));
  RC(c->alloc(&c->d_hnm1, cw));
  CK(cudaMemset(c->d_c0, 0, cw * sizeof(double2)));
  c->c0_first = c->d_c0;
  {
    RC(c->alloc(&c->d_part2, (size_t)RED_BLOCKS * 4));
    const char *env = getenv("AMDK_NO_GRAPHS");
    c->use_graphs = !(env && env[0] == '1');
    const char *nt = getenv("AMDK_NO_TUNE");
    c->tune = !(nt && nt[0] == '1');
    const char *no = getenv("AMDK_NO_OVERLAP");
    c->overlap = !(no && no[0] == '1');
  }
  if (h.nstate > CHOL_NMAX) {
    // large overlaps: the blocked factorisation's work copy and block row
    RC(c->alloc(&c->d_cholw, (size_t)h.nstate * h.nstate));
    RC(c->alloc(&c->d_cholt, (size_t)128 * h.nstate));
  }
  RC(c->up(&c->d_occ, h.occ));
  {
    // density weights per band pair (density.f90:51-62)
    std::vector<double> wa(c->npairs), wb(c->npairs);
    for (int p = 0; p < c->npairs; p++) {
      wa[p] = h.occ[2 * p] / h.omega;
      wb[p] = (2 * p + 1 < h.nstate) ? h.occ[2 * p + 1] / h.omega : 0.0;
    }
    RC(c->up(&c->d_wa, wa));
    RC(c->up(&c->d_wb, wb));
    if (h.lsd) {
      // the spin-2 bands' weights (bands nel_up.. are spin 2)
      for (int p = 0; p < c->npairs; p++) {
        if (2 * p < h.nel_up) wa[p] = 0.0;
        if (2 * p + 1 < h.nel_up) wb[p] = 0.0;
      }
      RC(c->up(&c->d_wa2, wa));
      RC(c->up(&c->d_wb2, wb));
    }
  }
  long npt = (long)n1 * n2 * n3;
  RC(c->alloc(&c->d_rho, npt));
  RC(c->alloc(&c->d_vpot, npt));
  if (h.lsd) {
    RC(c->alloc(&c->d_rho2, npt));
    RC(c->alloc(&c->d_vpot2, npt));
  }
  RC(c->alloc(&c->d_cgrid, 2 * npt));
  RC(c->alloc(&c->d_rhog, h.ngrho));
  RC(c->alloc(&c->d_vg, h.ngrho));
  RC(c->alloc(&c->d_vxg, h.ngrho));
  RC(c->alloc(&c->d_fp, 2L * h.ngrho));
  RC(c->alloc(&c->d_fm, 2L * h.ngrho));
  RC(c->alloc(&c->d_gam, (size_t)h.nstate * h.nstate));
  RC(c->alloc(&c->d_uinv, (size_t)h.nstate * h.nstate));
  RC(c->alloc(&c->d_info, 2));  // [0] Cholesky status, [1] slice-GEMM wait status
  CK(cudaMemset(c->d_info, 0, 2 * sizeof(int)));
  RC(c->alloc(&c->d_part, (size_t)RED_BLOCKS * 4 + 3L * 64 * h.nat + 64));
  RC(c->alloc(&c->d_scal, S_NSCAL));
  RC(c->alloc(&c->d_ticket, TK_N));
  CK(cudaMemset(c->d_ticket, 0, TK_N * sizeof(unsigned)));
  CK(cudaMallocHost(&c->h_pin, sizeof(double) * (S_NSCAL + 8)));
  CK(cudaMallocHost(&c->h_info, sizeof(int) * 4));
  c->h_info[0] = c->h_info[1] = 0;
  CK(cudaMemset(c->d_scal, 0, S_NSCAL * sizeof(double)));
  // Pencil path for the pair transforms (cubic grids with a specialised
  // length whose slab plane fits in shared memory): V(r)psi and the density
  // go plane by plane through shared memory with no slab buffer in HBM.
  // Decided for both pair precisions (index 0 FP64, 1 mixed) so that
  // amdk_set_precision can switch between them; buffers are sized for FP64.
  {
    bool known = false;
    with_n(n1, [&](auto NC) { known = decltype(NC)::value > 0; });
    const bool ok = (n1 == n2 && n2 == n3) && known && g.nz[0] < 255;  // slab planes fit the packed table
    const size_t lim = 227 * 1024;
    const int nz0 = g.nz[0];
    const char *env = getenv("AMDK_NO_PENCIL");
    const bool off = env && env[0] == '1';
    if (ok) {
      c->pn1 = fft_n1(n1);
      c->pn2 = n1 / c->pn1;
      // V(r)psi: two blocks per SM when the tile can stay at least half the
      // plane wide, else one
      int ct2 = pencil_tile<double2>(n1, nz0, 0, lim / 2), ct1 = pencil_tile<double2>(n1, nz0, 0, lim);
      c->ctv_p[0] = (2 * ct2 >= n1) ? ct2 : ct1;
      ct2 = pencil_tile<float2>(n1, nz0, 0, lim / 2);
      ct1 = pencil_tile<float2>(n1, nz0, 0, lim);
      c->ctv_p[1] = (2 * ct2 >= n1) ? ct2 : ct1;
      // density: equal column tiles (1, 2 or 4) whose sums fit 1, 2 or 4
      // register slots; two blocks per SM when possible
      density_tiles(n1, nz0, sizeof(double2), lim, &c->ctd_p[0], &c->nsd_p[0]);
      density_tiles(n1, nz0, sizeof(float2), lim, &c->ctd_p[1], &c->nsd_p[1]);
    }
    for (int q = 0; q < 2; ++q) {
      c->pv_p[q] = ok && !off && c->ctv_p[q] >= 8;
      c->pd_p[q] = ok && !off && c->ctd_p[q] >= 8;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, dev);
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_ekin, NTHR, 0) == cudaSuccess && nb > 0)
      c->red_ekin = std::min(RED_BLOCKS, nb * c->nsm);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_gmax_precon, NTHR, 0) == cudaSuccess && nb > 0)
      c->red_gmax = std::min(RED_BLOCKS, nb * c->nsm);
    cudaGetLastError();
  }
  if (h.lsd && !(c->pv_p[0] && c->pd_p[0] && c->pv_p[1] && c->pd_p[1])) {
    set_error("the open-shell branch needs the pencil transforms in both precisions (this grid has none)");
    return AMDK_ERR_UNSUPPORTED;
  }
  RC(sg_setup(c));
  const int q0 = (c->precision == AMDK_MIXED) ? 1 : 0;
  const bool pencil_all = c->pv_p[q0] && c->pd_p[q0];
  // pair batch: all pairs at once on the pencil path, else 8
  if (c->batch <= 0) c->batch = pencil_all ? c->npairs : 8;
  c->batch = std::max(1, std::min(c->batch, c->npairs));
  size_t rb = (size_t)c->batch * rstride(c, 0) * sizeof(double2);
  const size_t rbf = 2 * (size_t)rstride(c, 1) * sizeof(double2);
  size_t sb = 2 * (size_t)sstride(c, 1) * sizeof(double2);
  if (!(c->pv_p[0] && c->pd_p[0] && c->pv_p[1] && c->pd_p[1]))
    sb = std::max(sb, (size_t)c->batch * sstride(c, 0) * sizeof(double2));
  RC(c->alloc((char **)&c->d_rb, rb));
  RC(c->alloc((char **)&c->d_rbf, rbf));
  RC(c->alloc((char **)&c->d_sb, sb));
  c->fftbuf_bytes = rb + rbf + sb;
  set_pair_precision(c, c->precision);
  if (c->pv_p[0] || c->pv_p[1] || c->pd_p[0] || c->pd_p[1]) {
    std::vector<int> rpos(h.ngrays), zinv(n3, -1), zl0(g.nz[0]), postp(h.ngpw), postm(h.ngpw);
    CK(cudaMemcpy(zl0.data(), c->d_zlist[0], sizeof(int) * g.nz[0], cudaMemcpyDeviceToHost));
    for (int zi = 0; zi < g.nz[0]; zi++) zinv[zl0[zi]] = zi;
    for (int r = 0; r < h.ngrays; r++) rpos[r] = zinv[ray_kz[r]] * (n2 + 1) + ray_ky[r];
    // G -> transposed ray buffer position kx*R + ray
    for (int ig = 0; ig < h.ngpw; ig++) {
      postp[ig] = (posp[ig] % n1) * h.ngrays + posp[ig] / n1;
      postm[ig] = (posm[ig] % n1) * h.ngrays + posm[ig] / n1;
    }
    RC(c->up(&c->d_rpos, rpos));
    RC(c->up(&c->d_zinv, zinv));
    RC(c->up(&c->d_postp, postp));
    RC(c->up(&c->d_postm, postm));
    std::vector<int> gmapt((size_t)n1 * h.ngrays);
    for (int r = 0; r < h.ngrays; r++)
      for (int k = 0; k < n1; k++) gmapt[(size_t)k * h.ngrays + r] = gmap[(size_t)r * n1 + k];
    RC(c->up(&c->d_gmapt, gmapt));
    c->pg = pencil_geom_1gpu(n1, n2, n3, h.ngrays, g.nz[0], c->d_rpos, c->d_zinv, c->d_zlist[0], c->d_gmapt);
    c->pencil_groups = std::max(1, std::min(c->batch, 16));
    if (c->pd_p[0] || c->pd_p[1]) RC(c->alloc(&c->d_rhopart, (size_t)c->pencil_groups * npt));
    if (c->pv_p[0] || c->pv_p[1]) {
      char *vt;
      RC(c->alloc(&vt, (size_t)npt * sizeof(double)));
      c->d_vt = vt;
      if (h.lsd) {
        RC(c->alloc(&vt, (size_t)npt * sizeof(double)));
        c->d_vt2 = vt;
      }
    }
  }
  // pseudopotential tables on the device
  RC(c->alloc(&c->d_vps, (size_t)h.nsp * h.ngrho));
  RC(c->alloc(&c->d_rhos, (size_t)h.nsp * h.ngrho));
  RC(c->alloc(&c->d_twnl, (size_t)h.nsp * h.nghmax * h.ngpw));
  CK(cudaMemset(c->d_twnl, 0, sizeof(double) * (size_t)h.nsp * h.nghmax * h.ngpw));
  {
    double *xp, *yp, *hh, *sd;
    std::vector<double> hv, sdd;
    RC(c->alloc(&xp, NSPLN));
    RC(c->alloc(&yp, NSPLN));
    RC(c->alloc(&hh, NSPLN + 1));
    RC(c->alloc(&sd, NSPLN + 1));
    double vol = 1.0 / std::sqrt(h.omega);
    for (int is = 0; is < h.nsp; is++) {
      spline_coeffs(NSPLN, h.ggnh.data(), h.voo[is].data(), hv, sdd);
      CK(cudaMemcpy(xp, h.ggnh.data(), sizeof(double) * NSPLN, cudaMemcpyHostToDevice));
      CK(cudaMemcpy(yp, h.voo[is].data(), sizeof(double) * NSPLN, cudaMemcpyHostToDevice));
      CK(cudaMemcpy(hh, hv.data(), sizeof(double) * (NSPLN + 1), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(sd, sdd.data(), sizeof(double) * (NSPLN + 1), cudaMemcpyHostToDevice));
      ++c->nlaunch;
      k_vps_rhos<<<nblk(h.ngrho), NTHR>>>(h.ngrho, c->d_hg, xp, yp, hh, sd, NSPLN, (double)h.zv[is], h.omega, h.tpiba2,
                                           c->d_vps + (size_t)is * h.ngrho, c->d_rhos + (size_t)is * h.ngrho);
      CK(cudaDeviceSynchronize());
      for (int iv = 0; iv < h.ngh[is]; iv++) {
        const double *w = h.wns[is].data() + (size_t)iv * NSPLN;
        double xx = 0;
        for (int k = 0; k < NSPLN; k++) xx += std::fabs(w[k]);
        if (!(xx > 1e-12)) continue;
        spline_coeffs(NSPLN, h.ggng.data(), w, hv, sdd);
        CK(cudaMemcpy(xp, h.ggng.data(), sizeof(double) * NSPLN, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(yp, w, sizeof(double) * NSPLN, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(hh, hv.data(), sizeof(double) * (NSPLN + 1), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(sd, sdd.data(), sizeof(double) * (NSPLN + 1), cudaMemcpyHostToDevice));
        ++c->nlaunch;
        k_twnl<<<nblk(h.ngpw), NTHR>>>(h.ngpw, c->d_hg, c->d_gvec, xp, yp, hh, sd, NSPLN, h.lpval[is][iv], vol,
                                        c->d_twnl + ((size_t)is * h.nghmax + iv) * h.ngpw);
        CK(cudaDeviceSynchronize());
      }
    }
  }
  RC(c->alloc(&c->d_evps, h.ngrho));
  RC(c->alloc(&c->d_erhos, h.ngrho));
  RC(c->alloc(&c->d_vpp, h.ngpw));
  RC(c->alloc(&c->d_atarg, 3L * h.nat));
  RC(c->alloc(&c->d_atco, 3L * h.na_max * h.nsp));
  RC(c->up(&c->d_isa_is, h.isa_is));
  RC(c->up(&c->d_isa_ia, h.isa_ia));
  std::vector<int> na(h.na, h.na + h.nsp), ngh(h.ngh, h.ngh + h.nsp), zv(h.zv, h.zv + h.nsp);
  RC(c->up(&c->d_na, na));
  RC(c->up(&c->d_ngh, ngh));
  RC(c->up(&c->d_zv, zv));
  std::vector<double> wsg((size_t)h.nsp * 120, 0.0);
  for (int is = 0; is < h.nsp; is++)
    for (int iv = 0; iv < MAXNGH; iv++) wsg[is * 120 + iv] = h.wsg[is][iv];
  RC(c->up(&c->d_wsg, wsg));
  RC(c->alloc(&c->d_force, 3L * h.na_max * h.nsp));
  RC(c->alloc(&c->d_fsr, 3L * h.na_max * h.nsp));
  CK(cudaMemset(c->d_fsr, 0, sizeof(double) * 3L * h.na_max * h.nsp));
  RC(c->alloc(&c->d_esr, 1));
  // projector list (isa-major within a species, as nl(isa,iv) of fnl)
  int isa0 = 0;
  for (int is = 0; is < h.nsp; is++) {
    for (int iv = 0; iv < h.ngh[is]; iv++)
      for (int ia = 0; ia < h.na[is]; ia++) {
        c->p_isa.push_back(isa0 + ia);
        c->p_is.push_back(is);
        c->p_iv.push_back(iv);
        c->p_l.push_back(h.nghtol[is][iv]);
      }
    isa0 += h.na[is];
  }
  c->nproj = (int)c->p_isa.size();
  if (c->nproj) {
    RC(c->up(&c->d_pisa, c->p_isa));
    RC(c->up(&c->d_pis, c->p_is));
    RC(c->up(&c->d_piv, c->p_iv));
    RC(c->up(&c->d_pl, c->p_l));
    RC(c->alloc(&c->d_P, (size_t)c->nproj * h.ngpw));
    RC(c->alloc(&c->d_Q, 3 * (size_t)c->nproj * h.ngpw));
    size_t pn = (size_t)c->nproj * h.nstate;
    RC(c->alloc(&c->d_nl, pn));
    RC(c->alloc(&c->d_hn, pn));
    RC(c->alloc(&c->d_D, pn));
    RC(c->alloc(&c->d_dfnl, 3 * pn));
    // H: wsg on the diagonal (psp) or hlsg between projectors of equal l
    // and m on the same atom (UPF): pseudopotential.f90:56-99
    std::vector<double> H((size_t)c->nproj * c->nproj, 0.0);
    for (int a = 0; a < c->nproj; a++)
      for (int b = 0; b < c->nproj; b++) {
        if (c->p_isa[a] != c->p_isa[b]) continue;
        int is = c->p_is[a], iv = c->p_iv[a], jv = c->p_iv[b];
        if (!h.upf) {
          if (iv == jv) H[a + (size_t)c->nproj * b] = h.wsg[is][iv];
        } else if (h.nghtol[is][iv] == h.nghtol[is][jv] && h.lpval[is][iv] == h.lpval[is][jv]) {
          H[a + (size_t)c->nproj * b] = h.hlsg[is][h.nghtol[is][iv]][h.lfval[is][iv] - 1][h.lfval[is][jv] - 1];
        }
      }
    RC(c->up(&c->d_H, H));
    RC(sg_proj_setup(c));
  }
  {
    // FP64 tensor-core GEMM partials: the largest TN product is the overlap,
    // nl (nproj rows) or dfnl (3 nproj rows) against the bands
    const int rows = std::max(h.nstate, 3 * c->nproj);
    const size_t np = dg_part_doubles(c, rows, h.nstate);
    RC(c->alloc(&c->d_dgpart, np));
    RC(c->alloc(&c->d_dgpart2, np));
    CK(cudaFuncSetAttribute(k_dgemm_tn, cudaFuncAttributeMaxDynamicSharedMemorySize, DG_TN_SMEM));
    CK(cudaFuncSetAttribute(k_dgemm_nn, cudaFuncAttributeMaxDynamicSharedMemorySize, DG_NN_SMEM));
  }
  double es = 0.0;
  for (int is = 0; is < h.nsp; is++) es = es + (double)h.na[is] * h.zv[is] * h.zv[is] / RAGGIO;
  c->eself = es / std::sqrt(2.0 * (4.0 * std::atan(1.0)));
  CK(cudaDeviceSynchronize());
  return 0;
}

// ------------------------------------------------------------------ C ABI
// Launches inside its scope go to the side stream, with the side stream's
// reduction and GEMM partials.
struct OnSideStream {
  amdk_ctx *c;
  cudaStream_t s;
  double *p, *q;
  explicit OnSideStream(amdk_ctx *cc) : c(cc), s(cc->st), p(cc->d_part), q(cc->d_dgpart) {
    c->st = c->st2;
    c->d_part = c->d_part2;
    c->d_dgpart = c->d_dgpart2;
  }
  ~OnSideStream() {
    c->st = s;
    c->d_part = p;
    c->d_dgpart = q;
  }
};

// Segment A of the CG iteration with the C0-only work (projections, E_nl,
// E_kin) on the side stream; the context stream runs the density, rho(G),
// the potential, then (after the join) V(r)psi with fnonloc and the
// gradient.  The x pass of H|psi> is the density's: the density
// kernel only reads the transposed ray buffer, and the field transforms have
// their own, so V(r)psi starts from it as it is.  Same results as the
// sequential order; used on the pencil path with all pairs in one batch.
template <typename C> static int seg_a_overlap(amdk_ctx *c) {
  const int T = c->npairs;
  CK(cudaEventRecord(c->ev_fork, c->st));
  CK(cudaStreamWaitEvent(c->st2, c->ev_fork, 0));
  {
    OnSideStream side(c);
    RC(energy_c0_terms(c));
    CK(cudaEventRecord(c->ev_side_done, c->st));
  }
  RC(density_pairs_t<C>(c));
  RC(rhor2g_t<C>(c));
  RC(potential_t<C>(c));
  CK(cudaStreamWaitEvent(c->st, c->ev_side_done, 0));
  CK(cudaMemcpyAsync(c->h_pin, c->d_scal, sizeof(double) * S_NSCAL, cudaMemcpyDeviceToHost, c->st));
  pencil_vpsi<C>(c, T);
  xt_fwd<C>(c, T);
  unpack_h<C>(c, 0, T, c->d_postp, c->d_postm);
  RC(do_gradient(c));
  CK(cudaMemcpyAsync(c->h_pin + S_NSCAL, c->d_scal + S_GMAX, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  return 0;
}

// One segment of the CG iteration as a CUDA graph: captured the first time
// its key is seen, then kept.  body() only enqueues work on the context
// stream (no host synchronisation, no host-side state change a replay would
// miss).  A capture that fails turns graphs off for the context (nullptr: the
// caller runs body() eagerly).
template <typename F> static amdk_ctx::SegGraph *ensure_segment(amdk_ctx *c, const std::array<int, 4> &key, F &&body) {
  auto it = c->graphs.find(key);
  if (it != c->graphs.end()) return &it->second;
  const size_t rec0 = c->recs.size(), ev0 = c->evused;
  const long nl0 = c->nlaunch;
  if (cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    c->use_graphs = false;
    return nullptr;
  }
  const int rc = body();
  cudaGraph_t g = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(c->st, &g);
  amdk_ctx::SegGraph sg;
  const bool ok = rc == 0 && ce == cudaSuccess && g && cudaGraphInstantiate(&sg.exec, g, 0) == cudaSuccess;
  sg.graph = g;
  sg.recs.assign(c->recs.begin() + rec0, c->recs.end());
  sg.nevents = c->evused - ev0;
  sg.nlaunch = c->nlaunch - nl0;
  c->recs.resize(rec0);
  c->evused = ev0;
  c->nlaunch = nl0;
  if (!ok) {
    cudaGetLastError();
    if (sg.exec) cudaGraphExecDestroy(sg.exec);
    if (g) cudaGraphDestroy(g);
    c->use_graphs = false;
    return nullptr;
  }
  return &c->graphs.emplace(key, std::move(sg)).first->second;
}
// the bookkeeping of a segment launched (alone or inside an ensemble graph)
static void account_segment(amdk_ctx *c, const amdk_ctx::SegGraph &sg) {
  c->recs.insert(c->recs.end(), sg.recs.begin(), sg.recs.end());
  c->evused += sg.nevents;
  c->nlaunch += sg.nlaunch;
}
template <typename F> static int run_segment(amdk_ctx *c, const std::array<int, 4> &key, F &&body) {
  amdk_ctx::SegGraph *sg = ensure_segment(c, key, body);
  if (!sg) return body();
  CK(cudaGraphLaunch(sg->exec, c->st));
  account_segment(c, *sg);
  return 0;
}

// The pieces of one CG iteration (do_opt.f90:80-128), shared by
// amdk_scf_iteration and amdk_ensemble_iteration: segment A (density ...
// H|psi>, gradient, GEMAX copied to pinned memory), the host's CHK_TFOR
// decision on GEMAX, segment B (forces, PCG, ortho) and the bookkeeping after.
static bool iter_overlap(const amdk_ctx *c) {
  return c->overlap && c->pencil_vpsi && c->pencil_density && c->batch == c->npairs;
}
static int seg_a_body(amdk_ctx *c) {
  const int q = (c->precision == AMDK_MIXED) ? 1 : 0;
  if (iter_overlap(c)) return q ? seg_a_overlap<float2>(c) : seg_a_overlap<double2>(c);
  RC(do_density(c));
  RC(do_potential(c));
  RC(do_energy(c, nullptr));  // energies read after the end-of-iteration sync
  RC(do_apply_h(c));
  RC(do_gradient(c));
  CK(cudaMemcpyAsync(c->h_pin + S_NSCAL, c->d_scal + S_GMAX, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  return 0;
}
static std::array<int, 4> seg_a_key(const amdk_ctx *c) {
  const int q = (c->precision == AMDK_MIXED) ? 1 : 0;
  const int parity = (c->d_c0 == c->c0_first) ? 0 : 1;
  const int c0_digits = (use_slice(c) && c->sg_c0_buf == (void *)c->d_c0) ? 1 : 0;
  return {0, q + 2 * c0_digits, parity, c->prof ? 1 : 0};
}
// after segment A has finished: GEMAX, CHK_TFOR (gradient.f90:113-136)
static int chk_tfor(amdk_ctx *c, int istep, double gcut, double *gm) {
  *gm = c->h_pin[S_NSCAL];
  if (!std::isfinite(*gm)) {
    set_error("non-finite wavefunction gradient");
    return AMDK_ERR_NONFINITE;
  }
  if (istep == 1) c->tfor = false;
  else if (*gm < 3 * gcut) c->tfor = true;
  c->h_pin[S_NSCAL + 1] = (double)istep;  // read by the PCG step through a captured copy
  return 0;
}
static int seg_b_body(amdk_ctx *c, int istep) {
  if (c->tfor) RC(do_ionic_forces(c));
  RC(do_pcg(c, istep));
  RC(do_ortho(c, false, false));
  return 0;
}
static std::array<int, 4> seg_b_key(const amdk_ctx *c) {
  const int parity = (c->d_c0 == c->c0_first) ? 0 : 1;
  return {1, c->tfor ? 1 : 0, parity, c->prof ? 1 : 0};
}
// after segment B has finished: the ortho's output buffer holds C0, status
// and energies
static int iter_end(amdk_ctx *c, double gm, double gcut, amdk_energies *e, double *gemax, int *converged) {
  c->sg_c0_buf = use_slice(c) ? (void *)c->d_cp : nullptr;  // the ortho's output (digits written)
  std::swap(c->d_c0, c->d_cp);
  prof_harvest(c);
  c->warm[(c->precision == AMDK_MIXED) ? 1 : 0] = true;
  RC(check_ortho(c));
  amdk_energies en;
  RC(fill_energies(c, c->h_pin, &en));
  if (e) *e = en;
  if (gemax) *gemax = gm;
  if (converged) *converged = gm < gcut;
  return 0;
}

// Several contexts (independent systems on one GPU) advanced together: each
// segment of every member's CG iteration is one CUDA graph launch, the
// members' segment graphs being child graphs of one parent (cached by the
// members' segment keys), which run concurrently.
struct amdk_ensemble {
  std::vector<amdk_ctx *> m;
  int device = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms = 0;
  std::map<std::vector<std::array<int, 4>>, cudaGraphExec_t> parents;
};
// the parent graph of the members' segment graphs for these keys
static int ensemble_parent(amdk_ensemble *E, const std::vector<std::array<int, 4>> &keys,
                           const std::vector<amdk_ctx::SegGraph *> &sgs, cudaGraphExec_t *out) {
  auto it = E->parents.find(keys);
  if (it != E->parents.end()) {
    *out = it->second;
    return 0;
  }
  cudaGraph_t parent = nullptr;
  CK(cudaGraphCreate(&parent, 0));
  for (amdk_ctx::SegGraph *sg : sgs) {
    cudaGraphNode_t node;
    const cudaError_t e = cudaGraphAddChildGraphNode(&node, parent, nullptr, 0, sg->graph);
    if (e != cudaSuccess) {
      cudaGraphDestroy(parent);
      CK(e);
    }
  }
  cudaGraphExec_t exec = nullptr;
  const cudaError_t e = cudaGraphInstantiate(&exec, parent, 0);
  cudaGraphDestroy(parent);
  CK(e);
  E->parents.emplace(keys, exec);
  *out = exec;
  return 0;
}

// ------------------------------------------------------------------ slab decomposition
// The band-pair transforms distributed over nranks processes as the
// reference distributes its FFTs (fft_interface.f90:109-137: x-rays in G
// space per rank, an all-to-all, contiguous x planes per rank in real space).
// G vectors go to ranks with their x-ray, the rays in mirror pairs
// {(ky, kz), (-ky, -kz)} so that +G and -G of every owned G lie on the rank's
// rays (the pair pack and unpack then need no remote coefficient); pairs are
// placed largest first on the rank with the fewest G vectors so far (ties:
// fewer rays, then the lower rank).  The x planes are split into contiguous
// ranges of n1/nranks (rounded down at each boundary).
static int slab_partition(const HostSetup &h, int nranks, const std::vector<int> &ray_ky,
                          const std::vector<int> &ray_kz, const std::vector<int> &posp, std::vector<int> &ray_owner,
                          std::vector<int> &plane0) {
  const int n1 = h.nr[0], n2 = h.nr[1], n3 = h.nr[2], R = h.ngrays;
  if (nranks < 1 || nranks > PG_MAXSEG || nranks > n1) {
    set_error("slab decomposition: nranks must be 1.." + std::to_string(std::min(PG_MAXSEG, n1)));
    return AMDK_ERR_BADARG;
  }
  std::vector<long> ng(R, 0);
  for (int ig = 0; ig < h.ngpw; ig++) ng[posp[ig] / n1]++;
  std::vector<int> at((size_t)n2 * n3, -1);
  for (int r = 0; r < R; r++) at[(size_t)ray_kz[r] * n2 + ray_ky[r]] = r;
  struct Cls {
    int r, m;
    long g;
  };
  std::vector<Cls> cls;
  for (int r = 0; r < R; r++) {
    const int m = at[(size_t)((n3 - ray_kz[r]) % n3) * n2 + (n2 - ray_ky[r]) % n2];
    if (m < 0) {
      set_error("slab decomposition: the wavefunction rays are not closed under G -> -G");
      return AMDK_ERR_UNSUPPORTED;
    }
    if (r <= m) cls.push_back({r, m, ng[r] + (m != r ? ng[m] : 0)});
  }
  if ((int)cls.size() < nranks) {
    set_error("slab decomposition: fewer ray pairs than ranks");
    return AMDK_ERR_BADARG;
  }
  std::stable_sort(cls.begin(), cls.end(), [](const Cls &a, const Cls &b) { return a.g > b.g; });
  std::vector<long> gl(nranks, 0), rl(nranks, 0);
  ray_owner.assign(R, -1);
  for (const Cls &k : cls) {
    int best = 0;
    for (int q = 1; q < nranks; q++)
      if (gl[q] < gl[best] || (gl[q] == gl[best] && rl[q] < rl[best])) best = q;
    ray_owner[k.r] = best;
    ray_owner[k.m] = best;
    gl[best] += k.g;
    rl[best] += (k.m != k.r) ? 2 : 1;
  }
  plane0.assign(nranks + 1, 0);
  for (int q = 0; q <= nranks; q++) plane0[q] = (int)((long)q * n1 / nranks);
  return 0;
}

struct amdk_slab {
  amdk_ctx *c = nullptr;
  int nranks = 1, rank = 0, precision = AMDK_FP64;
  int ng = 0, nray_loc = 0, gzero = -1, nplane = 0, nray = 0;
  std::vector<int> plane0, seg_r0, local_g;
  // sender side: local G code of (kx, local ray), planes and local rays of
  // each local G's +G / -G position, |G|^2; receiver side: rpos of every ray
  // in owner order
  int *d_gmapt = nullptr, *d_kxp = nullptr, *d_rlp = nullptr, *d_kxm = nullptr, *d_rlm = nullptr;
  int *d_pp = nullptr, *d_pm = nullptr, *d_rpos = nullptr;
  double *d_hg = nullptr, *d_rhopart = nullptr;
  void *d_vp = nullptr;
  int pos_T = -1, groups_max = 8;
  std::vector<void *> allocs;
  template <typename T> int alloc(T **p, size_t n) {
    RC(dalloc(p, n));
    allocs.push_back((void *)*p);
    return 0;
  }
  template <typename T> int up(T **p, const std::vector<T> &v) {
    RC(amdk::upload(p, v));
    allocs.push_back((void *)*p);
    return 0;
  }
  ~amdk_slab() {
    for (void *p : allocs) cudaFree(p);
  }
};

static int slab_create(amdk_ctx *c, int nranks, int rank, amdk_slab *s) {
  const HostSetup &h = c->hs;
  const int q = (c->precision == AMDK_MIXED) ? 1 : 0;
  if (h.lsd) {
    set_error("slab decomposition: the open-shell branch is not distributed");
    return AMDK_ERR_UNSUPPORTED;
  }
  if (!(c->pv_p[q] && c->pd_p[q])) {
    set_error("slab decomposition: needs the pencil transforms of this grid at the context's precision");
    return AMDK_ERR_UNSUPPORTED;
  }
  if (rank < 0 || rank >= nranks) {
    set_error("slab decomposition: rank out of range");
    return AMDK_ERR_BADARG;
  }
  const int n1 = h.nr[0], n2 = h.nr[1];
  std::vector<int> ray_ky, ray_kz, posp, posm, owner;
  ray_tables(h, ray_ky, ray_kz, posp, posm);
  RC(slab_partition(h, nranks, ray_ky, ray_kz, posp, owner, s->plane0));
  s->c = c;
  s->nranks = nranks;
  s->rank = rank;
  s->precision = c->precision;
  s->nray = h.ngrays;
  s->nplane = s->plane0[rank + 1] - s->plane0[rank];
  // rays in owner order (increasing ray number within an owner): the
  // receiver's segments, and the sender's local ray numbering
  std::vector<int> order, rloc(h.ngrays, -1);
  s->seg_r0.assign(nranks + 1, 0);
  for (int o = 0; o < nranks; o++) {
    s->seg_r0[o] = (int)order.size();
    int k = 0;
    for (int r = 0; r < h.ngrays; r++)
      if (owner[r] == o) {
        order.push_back(r);
        rloc[r] = k++;
      }
  }
  s->seg_r0[nranks] = (int)order.size();
  s->nray_loc = s->seg_r0[rank + 1] - s->seg_r0[rank];
  // the ray's plane position, as in the one-GPU pencil tables
  std::vector<int> zl0(c->geom.nz[0]), zinv(h.nr[2], -1), rpos(h.ngrays);
  CK(cudaMemcpy(zl0.data(), c->d_zlist[0], sizeof(int) * zl0.size(), cudaMemcpyDeviceToHost));
  for (int zi = 0; zi < (int)zl0.size(); zi++) zinv[zl0[zi]] = zi;
  for (int j = 0; j < h.ngrays; j++) rpos[j] = zinv[ray_kz[order[j]]] * (n2 + 1) + ray_ky[order[j]];
  RC(s->up(&s->d_rpos, rpos));
  // local G vectors (increasing global index) and their tables
  const int R = s->nray_loc;
  std::vector<int> gmapt((size_t)n1 * std::max(R, 1), 0), kxp, rlp, kxm, rlm;
  std::vector<double> hg;
  for (int ig = 0; ig < h.ngpw; ig++) {
    const int rp = posp[ig] / n1;
    if (owner[rp] != rank) continue;
    const int il = (int)s->local_g.size(), rm = posm[ig] / n1;
    s->local_g.push_back(ig);
    kxp.push_back(posp[ig] % n1);
    rlp.push_back(rloc[rp]);
    kxm.push_back(posm[ig] % n1);
    rlm.push_back(rloc[rm]);
    hg.push_back(h.hg[ig]);
    if (ig == 0) s->gzero = il;
    if (ig != 0) gmapt[(size_t)(posm[ig] % n1) * R + rloc[rm]] = -(il + 1);
    gmapt[(size_t)(posp[ig] % n1) * R + rloc[rp]] = il + 1;
  }
  s->ng = (int)s->local_g.size();
  RC(s->up(&s->d_gmapt, gmapt));
  RC(s->up(&s->d_kxp, kxp));
  RC(s->up(&s->d_rlp, rlp));
  RC(s->up(&s->d_kxm, kxm));
  RC(s->up(&s->d_rlm, rlm));
  RC(s->up(&s->d_hg, hg));
  RC(s->alloc(&s->d_pp, std::max(s->ng, 1)));
  RC(s->alloc(&s->d_pm, std::max(s->ng, 1)));
  const size_t pl = (size_t)s->nplane * n1 * n1;  // cubic grid (pencil path)
  RC(s->alloc(&s->d_rhopart, (size_t)s->groups_max * pl));
  char *vp;
  RC(s->alloc(&vp, pl * sizeof(double)));
  s->d_vp = vp;
  return 0;
}

static cudaStream_t slab_stream(const amdk_slab *s, void *stream) {
  return stream ? (cudaStream_t)stream : s->c->st;
}
static int slab_check_pairs(const amdk_slab *s, int band0, int npairs) {
  const int nst = s->c->nstate;
  if (band0 < 0 || (band0 & 1) || npairs < 1 || band0 + 2 * (npairs - 1) >= nst) {
    set_error("slab transform: band0 must be even and the pairs within the bands");
    return AMDK_ERR_BADARG;
  }
  if (npairs > 65535 || (long)npairs * s->nray * s->c->hs.nr[0] > (long)INT32_MAX) {
    set_error("slab transform: too many pairs in one call for 32-bit positions");
    return AMDK_ERR_BADARG;
  }
  return 0;
}
// sender side: local rays, layout [kx][t][ray] (rank-major send order)
static PencilGeom slab_xgeom(const amdk_slab *s, int T) {
  const HostSetup &h = s->c->hs;
  PencilGeom g = pencil_geom_1gpu(h.nr[0], h.nr[1], h.nr[2], s->nray_loc, s->c->geom.nz[0], nullptr, nullptr, nullptr,
                                  s->d_gmapt);
  g.xt_t = s->nray_loc;
  g.xt_x = (long)T * s->nray_loc;
  return g;
}
// receiver side: this rank's planes, every ray, one segment per source rank
static PencilGeom slab_pgeom(const amdk_slab *s, int T) {
  const HostSetup &h = s->c->hs;
  PencilGeom g = pencil_geom_1gpu(s->nplane, h.nr[1], h.nr[2], s->nray, s->c->geom.nz[0], s->d_rpos, s->c->d_zinv,
                                  s->c->d_zlist[0], nullptr);
  g.pr_t = 1;
  g.pr_x = T;
  g.nseg = s->nranks;
  g.seg_mul = (long)s->nplane * T;
  for (int o = 0; o <= s->nranks; o++) g.seg_r0[o] = s->seg_r0[o];
  return g;
}

template <typename C>
static int slab_pairs_out_t(amdk_slab *s, const double2 *c0, int band0, int T, C *send, cudaStream_t st) {
  amdk_ctx *c = s->c;
  const PencilGeom gx = slab_xgeom(s, T);
  const long lines = (long)T * s->nray_loc;
  if (lines == 0) return 0;
  with_n(c->hs.nr[0], [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    if constexpr (N > 0) {
      smem_opt_in<k_xt_bwd_pair<C, N>>();
      ++c->nlaunch;
      constexpr int N2 = N / fft_n1(N);
      k_xt_bwd_pair<C, N><<<nblk(lines, XL), XL * N2, xt_smem<C>(N), st>>>(c0, s->ng, c->nstate, band0, T, gx,
                                                                          plan<C>(c, 0), send);
    }
  });
  CK(cudaGetLastError());
  return 0;
}
template <typename C> static int slab_vpsi_t(amdk_slab *s, C *recv, int T, const double *v, cudaStream_t st) {
  typedef decltype(C().x) Rl;
  amdk_ctx *c = s->c;
  const int n = c->hs.nr[1], q = (s->precision == AMDK_MIXED) ? 1 : 0;
  ++c->nlaunch;
  k_v_permute<Rl><<<dim3((s->nplane + 31) / 32, (n + 31) / 32, n), dim3(32, 8), 0, st>>>(n, s->nplane, c->pn1, c->pn2,
                                                                                      v, (Rl *)s->d_vp);
  const PencilGeom gp = slab_pgeom(s, T);
  const int ct = c->ctv_p[q];
  with_n(n, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    if constexpr (N > 0) {
      smem_opt_in<k_pencil_vpsi<C, N>>();
      ++c->nlaunch;
      k_pencil_vpsi<C, N><<<dim3(s->nplane, T), PNT, pencil_smem<C>(N, gp.nz, ct), st>>>(
          gp, plan<C>(c, 1), recv, (const Rl *)s->d_vp, ct, nullptr, 0, 0, -1);
    }
  });
  CK(cudaGetLastError());
  return 0;
}
template <typename C, int N, int NS>
static void slab_density_launch(amdk_slab *s, const C *recv, int band0, int T, int grp, int ct, cudaStream_t st) {
  amdk_ctx *c = s->c;
  const PencilGeom gp = slab_pgeom(s, T);
  const int per = (T + grp - 1) / grp;
  smem_opt_in<k_pencil_density<C, N, NS>>();
  ++c->nlaunch;
  k_pencil_density<C, N, NS><<<dim3(s->nplane, grp), PNT, pencil_smem<C>(N, gp.nz, ct), st>>>(
      gp, plan<C>(c, 1), recv, T, per, c->d_wa + band0 / 2, c->d_wb + band0 / 2, s->d_rhopart, ct, 0);
}
template <typename C>
static int slab_density_t(amdk_slab *s, const C *recv, int band0, int T, double *rho, int add, cudaStream_t st) {
  amdk_ctx *c = s->c;
  const int n = c->hs.nr[1], q = (s->precision == AMDK_MIXED) ? 1 : 0;
  const int ct = c->ctd_p[q], ns = c->nsd_p[q];
  // pair groups: enough blocks for two waves, at most groups_max grids
  int grp = std::max(1, std::min({T, s->groups_max, (2 * c->nsm + s->nplane - 1) / s->nplane}));
  const int per = (T + grp - 1) / grp;
  grp = (T + per - 1) / per;  // no empty group
  with_n(n, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    if constexpr (N > 0) {
      if (ns == 1) slab_density_launch<C, N, 1>(s, recv, band0, T, grp, ct, st);
      else if (ns == 2) slab_density_launch<C, N, 2>(s, recv, band0, T, grp, ct, st);
      else slab_density_launch<C, N, 4>(s, recv, band0, T, grp, ct, st);
    }
  });
  ++c->nlaunch;
  k_rho_reduce_p<<<dim3((n + 31) / 32, (s->nplane + 31) / 32, n), dim3(32, 8), 0, st>>>(
      n, s->nplane, c->pn1, c->pn2, grp, s->d_rhopart, rho, add, 0, 0);
  CK(cudaGetLastError());
  return 0;
}
template <typename C>
static int slab_pairs_in_t(amdk_slab *s, C *back, const double2 *c0, int band0, int T, double2 *c2, cudaStream_t st) {
  amdk_ctx *c = s->c;
  const HostSetup &h = c->hs;
  const long lines = (long)T * s->nray_loc;
  if (lines == 0 || s->ng == 0) return 0;
  if (s->pos_T != T) {
    ++c->nlaunch;
    k_slab_pos<<<nblk(s->ng), NTHR, 0, st>>>(s->ng, s->d_kxp, s->d_rlp, s->d_kxm, s->d_rlm, (long)T * s->nray_loc,
                                             s->d_pp, s->d_pm);
    s->pos_T = T;
  }
  const PencilGeom gx = slab_xgeom(s, T);
  with_n(h.nr[0], [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    if constexpr (N > 0) {
      smem_opt_in<k_xt_fwd<C, N>>();
      ++c->nlaunch;
      constexpr int N2 = N / fft_n1(N);
      k_xt_fwd<C, N><<<nblk(lines, XL), XL * N2, xt_smem<C>(N), st>>>(T, gx, plan<C>(c, 0), back);
    }
  });
  const double scale = 1.0 / ((double)h.nr[0] * h.nr[1] * h.nr[2]);
  constexpr int PAIRS = unpack_pairs<C>();
  ++c->nlaunch;
  k_unpack_fnonloc<C><<<dim3(nblk(s->ng, 128), (T + PAIRS - 1) / PAIRS), 128, 0, st>>>(
      s->ng, c->nstate, band0, T, 0, s->d_pp, s->d_pm, back, s->nray_loc, scale, s->d_hg, h.tpiba2, c->d_occ, nullptr,
      nullptr, 0, c0, c2, nullptr, s->gzero);
  CK(cudaGetLastError());
  return 0;
}

extern "C" {

const char *amdk_last_error(void) { return g_err.c_str(); }

int amdk_create(const amdk_system *sys, const amdk_options *opt, amdk_ctx **out) {
  if (!sys || !out) {
    set_error("amdk_create: null argument");
    return AMDK_ERR_BADARG;
  }
  *out = nullptr;
  amdk_ctx *c = new amdk_ctx();
  if (opt) {
    c->device = opt->device;
    c->precision = opt->precision;
    c->batch = opt->pair_batch;
    if (opt->reserved[0] != 0) c->sg_plim = std::max(opt->reserved[0], 0);
    if (opt->reserved[1] != 0) c->dg_plim = std::max(opt->reserved[1], 0);
  }
  int rc = host_setup(sys, c->hs);
  if (rc) {
    delete c;
    return rc;
  }
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) {
    set_error(std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    delete c;
    return AMDK_ERR_CUDA;
  }
  if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) {
    set_error("stream creation failed");
    amdk_destroy(c);
    return AMDK_ERR_CUDA;
  }
  cudaEventCreate(&c->ev0);
  cudaEventCreate(&c->ev1);
  if (cudaStreamCreateWithFlags(&c->st2, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_side_done, cudaEventDisableTiming) != cudaSuccess) {
    set_error("side stream creation failed");
    amdk_destroy(c);
    return AMDK_ERR_CUDA;
  }
  rc = build_device(c);
  if (!rc) rc = do_positions(c, sys->atco);
  if (rc) {
    amdk_destroy(c);
    return rc;
  }
  *out = c;
  return 0;
}

int amdk_destroy(amdk_ctx *c) {
  if (!c) return 0;
  cudaSetDevice(c->device);
  if (c->st) cudaStreamSynchronize(c->st);
  for (void *p : c->allocs) cudaFree(p);
  for (auto &kv : c->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
  }
  if (c->h_pin) cudaFreeHost(c->h_pin);
  if (c->h_info) cudaFreeHost(c->h_info);
  for (auto &e : c->evpool) {
    cudaEventDestroy(e.first);
    cudaEventDestroy(e.second);
  }
  if (c->st2) {
    cudaStreamSynchronize(c->st2);
    cudaStreamDestroy(c->st2);
  }
  for (cudaEvent_t e : {c->ev_fork, c->ev_side_done})
    if (e) cudaEventDestroy(e);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
  return 0;
}

int amdk_info_get(amdk_ctx *c, amdk_info *info) {
  if (!c || !info) return AMDK_ERR_BADARG;
  const HostSetup &h = c->hs;
  for (int d = 0; d < 3; d++) info->nr[d] = h.nr[d];
  info->ngpw = h.ngpw;
  info->ngrho = h.ngrho;
  info->ngrays = h.ngrays;
  info->nhrays = h.nhrays;
  info->nstate = h.nstate;
  info->nat = h.nat;
  info->nghmax = h.nghmax;
  info->omega = h.omega;
  return 0;
}

int amdk_get_gvectors(amdk_ctx *c, int *inyh, double *hg, double *gvec, int *map_p, int *map_m) {
  if (!c) return AMDK_ERR_BADARG;
  const HostSetup &h = c->hs;
  if (inyh) std::memcpy(inyh, h.inyh.data(), sizeof(int) * h.inyh.size());
  if (hg) std::memcpy(hg, h.hg.data(), sizeof(double) * h.hg.size());
  if (gvec) std::memcpy(gvec, h.gvec.data(), sizeof(double) * h.gvec.size());
  if (map_p) std::memcpy(map_p, h.mapp.data(), sizeof(int) * h.mapp.size());
  if (map_m) std::memcpy(map_m, h.mapm.data(), sizeof(int) * h.mapm.size());
  return 0;
}

int amdk_host_gvectors(const amdk_system *sys, amdk_info *info, int *inyh, double *hg, double *gvec, int *map_p,
                       int *map_m) {
  if (!sys || !info) {
    set_error("amdk_host_gvectors: null argument");
    return AMDK_ERR_BADARG;
  }
  HostSetup h;
  int rc = host_setup(sys, h, true);
  if (rc) return rc;
  std::memset(info, 0, sizeof(*info));
  for (int d = 0; d < 3; d++) info->nr[d] = h.nr[d];
  info->ngpw = h.ngpw;
  info->ngrho = h.ngrho;
  info->ngrays = h.ngrays;
  info->nhrays = h.nhrays;
  info->nat = h.nat;
  info->omega = h.omega;
  if (inyh) std::memcpy(inyh, h.inyh.data(), sizeof(int) * h.inyh.size());
  if (hg) std::memcpy(hg, h.hg.data(), sizeof(double) * h.hg.size());
  if (gvec) std::memcpy(gvec, h.gvec.data(), sizeof(double) * h.gvec.size());
  if (map_p) std::memcpy(map_p, h.mapp.data(), sizeof(int) * h.mapp.size());
  if (map_m) std::memcpy(map_m, h.mapm.data(), sizeof(int) * h.mapm.size());
  return 0;
}

int amdk_set_precision(amdk_ctx *c, int precision) {
  if (!c || (precision != AMDK_FP64 && precision != AMDK_MIXED)) return AMDK_ERR_BADARG;
  set_pair_precision(c, precision);
  return 0;
}

int amdk_set_positions(amdk_ctx *c, const double *atco) {
  if (!c || !atco) return AMDK_ERR_BADARG;
  cudaSetDevice(c->device);
  return do_positions(c, atco);
}

int amdk_set_wfn(amdk_ctx *c, const double *c0) {
  if (!c || !c0) return AMDK_ERR_BADARG;
  cudaSetDevice(c->device);
  // on the context stream (after any kernel still reading or writing C0, e.g.
  // the rotation of an ortho that returned), and complete before returning
  CK(cudaMemcpyAsync(c->d_c0, c0, sizeof(double2) * (size_t)c->hs.ngpw * c->nstate, cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->sg_c0_buf = nullptr;
  return 0;
}

int amdk_set_density(amdk_ctx *c, const double *rho) {
  if (!c || !rho) return AMDK_ERR_BADARG;
  if (c->hs.lsd) {
    set_error("amdk_set_density: the open-shell branch keeps a density per spin; not supported");
    return AMDK_ERR_UNSUPPORTED;
  }
  cudaSetDevice(c->device);
  const size_t npt = (size_t)c->hs.nr[0] * c->hs.nr[1] * c->hs.nr[2];
  CK(cudaMemcpyAsync(c->d_rho, rho, sizeof(double) * npt, cudaMemcpyHostToDevice, c->st));
  if (c->precision == AMDK_MIXED) RC(rhor2g_t<float2>(c));
  else RC(rhor2g_t<double2>(c));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int amdk_get_wfn(amdk_ctx *c, double *c0) {
  if (!c || !c0) return AMDK_ERR_BADARG;
  cudaSetDevice(c->device);
  CK(cudaStreamSynchronize(c->st));
  CK(cudaMemcpy(c0, c->d_c0, sizeof(double2) * (size_t)c->hs.ngpw * c->nstate, cudaMemcpyDeviceToHost));
  return 0;
}

int amdk_ortho(amdk_ctx *c) {
  if (!c) return AMDK_ERR_BADARG;
  cudaSetDevice(c->device);
  return do_ortho(c);
}
int amdk_density(amdk_ctx *c) {
  if (!c) return AMDK_ERR_BADARG;
  cudaSetDevice(c->device);
  return do_density(c);
}
int amdk_potential(amdk_ctx *c) {
  if (!c) return AMDK_ERR_BADARG;
  cudaSetDevice(c->device);
  return do_potential(c);
}
int amdk_energy(amdk_ctx *c, amdk_energies *e) {
  if (!c) return AMDK_ERR_BADARG;
  cudaSetDevice(c->device);
  return do_energy(c, e);
}
int amdk_apply_h(amdk_ctx *c) {
  if (!c) return AMDK_ERR_BADARG;
  cudaSetDevice(c->device);
  return do_apply_h(c);
}
int amdk_gradient(amdk_ctx *c, double *gemax) {
  if (!c) return AMDK_ERR_BADARG;
  cudaSetDevice(c->device);
  RC(do_gradient(c));
  if (gemax) {
    CK(cudaMemcpyAsync(gemax, c->d_scal + S_GMAX, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  return 0;
}
int amdk_pcg(amdk_ctx *c, int istep) {
  if (!c || istep < 1) return AMDK_ERR_BADARG;
  cudaSetDevice(c->device);
  return do_pcg(c, istep, true);
}

int amdk_scf_iteration(amdk_ctx *c, int istep, double gcut, amdk_energies *e, double *gemax, int *converged) {
  if (!c || istep < 1) return AMDK_ERR_BADARG;
  cudaSetDevice(c->device);
  const int q = (c->precision == AMDK_MIXED) ? 1 : 0;
  // graphs from the second iteration on, once this precision has run eagerly
  // (first-call setup of kernels and cuBLAS stays out of the capture)
  const bool graph = c->use_graphs && istep > 1 && c->warm[q];
  cudaEventRecord(c->ev0, c->st);
  auto seg_a = [&]() -> int { return seg_a_body(c); };
  if (graph) RC(run_segment(c, seg_a_key(c), seg_a));
  else RC(seg_a());
  // GEMAX decides CHK_TFOR (forces or not) before PCG: the one host sync
  // inside the iteration
  CK(cudaStreamSynchronize(c->st));
  double gm = 0;
  RC(chk_tfor(c, istep, gcut, &gm));
  auto seg_b = [&]() -> int { return seg_b_body(c, istep); };
  if (graph) RC(run_segment(c, seg_b_key(c), seg_b));
  else RC(seg_b());
  cudaEventRecord(c->ev1, c->st);
  CK(cudaEventSynchronize(c->ev1));
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  c->last_ms = ms;
  return iter_end(c, gm, gcut, e, gemax, converged);
}

int amdk_ensemble_create(amdk_ctx **ctx, int n, amdk_ensemble **out) {
  if (!ctx || n < 1 || !out) return AMDK_ERR_BADARG;
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    if (!ctx[i] || ctx[i]->device != ctx[0]->device) {
      set_error("amdk_ensemble_create: null context or members on different devices");
      return AMDK_ERR_BADARG;
    }
    for (int j = 0; j < i; ++j)
      if (ctx[j] == ctx[i]) {
        set_error("amdk_ensemble_create: a context appears twice");
        return AMDK_ERR_BADARG;
      }
  }
  amdk_ensemble *E = new amdk_ensemble();
  E->m.assign(ctx, ctx + n);
  E->device = ctx[0]->device;
  cudaSetDevice(E->device);
  if (cudaStreamCreateWithFlags(&E->st, cudaStreamNonBlocking) != cudaSuccess || cudaEventCreate(&E->ev0) != cudaSuccess ||
      cudaEventCreate(&E->ev1) != cudaSuccess) {
    set_error("amdk_ensemble_create: stream or event creation failed");
    amdk_ensemble_destroy(E);
    return AMDK_ERR_CUDA;
  }
  *out = E;
  return 0;
}

int amdk_ensemble_destroy(amdk_ensemble *E) {
  if (!E) return 0;
  cudaSetDevice(E->device);
  if (E->st) cudaStreamSynchronize(E->st);
  for (auto &kv : E->parents) cudaGraphExecDestroy(kv.second);
  if (E->ev0) cudaEventDestroy(E->ev0);
  if (E->ev1) cudaEventDestroy(E->ev1);
  if (E->st) cudaStreamDestroy(E->st);
  delete E;
  return 0;
}

int amdk_ensemble_iteration(amdk_ensemble *E, const int *istep, double gcut, amdk_energies *e, double *gemax,
                            int *converged) {
  if (!E || !istep) return AMDK_ERR_BADARG;
  const int n = (int)E->m.size();
  cudaSetDevice(E->device);
  for (int i = 0; i < n; ++i)
    if (istep[i] < 1) {
      set_error("amdk_ensemble_iteration: CG step below 1");
      return AMDK_ERR_BADARG;
    }
  // members that cannot replay graphs yet (first iteration, first at this
  // precision, graphs off, profiling on) iterate on their own
  bool together = true;
  for (amdk_ctx *c : E->m) {
    const int q = (c->precision == AMDK_MIXED) ? 1 : 0;
    together = together && c->use_graphs && c->warm[q] && !c->prof;
  }
  for (int i = 0; i < n; ++i) together = together && istep[i] > 1;
  if (!together) {
    for (int i = 0; i < n; ++i)
      RC(amdk_scf_iteration(E->m[i], istep[i], gcut, e ? e + i : nullptr, gemax ? gemax + i : nullptr,
                            converged ? converged + i : nullptr));
    return 0;
  }
  std::vector<std::array<int, 4>> keys(n);
  std::vector<amdk_ctx::SegGraph *> sgs(n);
  auto run_all = [&](bool b, const std::vector<int> &steps) -> int {
    for (int i = 0; i < n; ++i) {
      amdk_ctx *c = E->m[i];
      keys[i] = b ? seg_b_key(c) : seg_a_key(c);
      const int st = steps[i];
      sgs[i] = b ? ensure_segment(c, keys[i], [&]() -> int { return seg_b_body(c, st); })
                 : ensure_segment(c, keys[i], [&]() -> int { return seg_a_body(c); });
      if (!sgs[i]) {
        set_error("amdk_ensemble_iteration: a member's segment could not be captured");
        return AMDK_ERR_CUDA;
      }
    }
    cudaGraphExec_t exec = nullptr;
    RC(ensemble_parent(E, keys, sgs, &exec));
    CK(cudaGraphLaunch(exec, E->st));
    for (int i = 0; i < n; ++i) account_segment(E->m[i], *sgs[i]);
    return 0;
  };
  const std::vector<int> steps(istep, istep + n);
  CK(cudaEventRecord(E->ev0, E->st));
  RC(run_all(false, steps));
  CK(cudaStreamSynchronize(E->st));
  std::vector<double> gm(n);
  for (int i = 0; i < n; ++i) RC(chk_tfor(E->m[i], istep[i], gcut, &gm[i]));
  RC(run_all(true, steps));
  CK(cudaEventRecord(E->ev1, E->st));
  CK(cudaEventSynchronize(E->ev1));
  float ms = 0;
  cudaEventElapsedTime(&ms, E->ev0, E->ev1);
  E->last_ms = ms;
  for (int i = 0; i < n; ++i) {
    E->m[i]->last_ms = ms;
    RC(iter_end(E->m[i], gm[i], gcut, e ? e + i : nullptr, gemax ? gemax + i : nullptr, converged ? converged + i : nullptr));
  }
  return 0;
}

int amdk_ensemble_last_ms(amdk_ensemble *E, double *ms) {
  if (!E || !ms) return AMDK_ERR_BADARG;
  *ms = E->last_ms;
  return 0;
}

int amdk_ionic_forces(amdk_ctx *c, double *force) {
  if (!c || !force) return AMDK_ERR_BADARG;
  cudaSetDevice(c->device);
  // forces of the current C0: density (for POTFOR) and projections with
  // H nl (NLFOR)
  RC(do_density(c));
  RC(energy_c0_terms(c));
  RC(do_ionic_forces(c));
  CK(cudaMemcpyAsync(force, c->d_force, sizeof(double) * 3 * c->hs.na_max * c->hs.nsp, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int amdk_wfn_set_predictor(amdk_ctx *c, int npoints, const double *coef) {
  if (!c || npoints < 1 || npoints > amdk_ctx::MAX_PRED) return AMDK_ERR_BADARG;
  c->pred_npts = npoints;
  c->pred_user = coef != nullptr;
  if (coef)
    for (int j = 0; j < npoints; ++j) c->pred_coef[j] = coef[j];
  else
    amdk::aspc_coefficients(npoints, c->pred_coef);
  if (c->nhist > npoints - 1) c->nhist = npoints - 1;
  return 0;
}

int amdk_wfn_extrapolate(amdk_ctx *c) {
  if (!c) return AMDK_ERR_BADARG;
  cudaSetDevice(c->device);
  const HostSetup &h = c->hs;
  const size_t cw = (size_t)h.ngpw * c->nstate;
  const int keep = c->pred_npts - 1;  // earlier steps the predictor uses
  // points of this prediction: all configured ones once enough steps are
  // stored, else the always-stable weights of the points there are
  const int np = std::min(c->pred_npts, c->nhist + 1);
  double w[amdk_ctx::MAX_PRED];
  if (np == c->pred_npts)
    for (int j = 0; j < np; ++j) w[j] = c->pred_coef[j];
  else
    amdk::aspc_coefficients(np, w);
  if (np > 1) {
    const int n = c->nstate;
    for (int j = 1; j < np; ++j) {
      const double2 *hj = c->d_hist[j - 1];
      // M = 2 Re C_j^T C0 - Re c_j(0) Re c0(0)^T aligns step j's occupied
      // subspace with the current one; cp (+)= w_j C_j M
      RC(dg_tn(c, hj, n, c->d_c0, n, 2.0, c->d_gam, n));
      ++c->nlaunch;
      k_g0_correct<<<dim3(nblk(n), n), NTHR, 0, c->st>>>(n, h.ngpw, hj, c->d_c0, c->d_gam, c->d_occ, 0, 0);
      spin_mask(c, c->d_gam);
      RC(dg_nn(c, hj, n, c->d_gam, n, w[j], j == 1 ? 0.0 : 1.0, false, c->d_cp));
    }
    ++c->nlaunch;
    k_axpy_c<<<RED_BLOCKS * 4, NTHR, 0, c->st>>>((long)cw, w[0], c->d_c0, c->d_cp);
  }
  if (keep > 0) {
    // store C0(t) as the most recent step: it takes the oldest slot
    const int slots = std::min(c->nhist + 1, keep);
    if (!c->d_hist[slots - 1]) RC(c->alloc(&c->d_hist[slots - 1], cw));
    double2 *t = c->d_hist[slots - 1];
    for (int j = slots - 1; j > 0; --j) c->d_hist[j] = c->d_hist[j - 1];
    c->d_hist[0] = t;
    CK(cudaMemcpyAsync(t, c->d_c0, sizeof(double2) * cw, cudaMemcpyDeviceToDevice, c->st));
    c->nhist = slots;
  }
  if (np > 1) std::swap(c->d_c0, c->d_cp);
  c->sg_c0_buf = nullptr;
  CK(cudaStreamSynchronize(c->st));
  return 0;
}
int amdk_wfn_history_clear(amdk_ctx *c) {
  if (!c) return AMDK_ERR_BADARG;
  c->nhist = 0;
  return 0;
}

int amdk_backward(amdk_ctx *c, double *dE_dR, double *dE_dpsi) {
  if (!c || (!dE_dR && !dE_dpsi)) return AMDK_ERR_BADARG;
  cudaSetDevice(c->device);
  const HostSetup &h = c->hs;
  RC(do_density(c));
  if (dE_dpsi) RC(do_potential(c));
  RC(do_energy(c, nullptr));
  if (dE_dR) {
    RC(do_ionic_forces(c));
    const size_t nf = 3 * (size_t)h.na_max * h.nsp;
    std::vector<double> f(nf);
    CK(cudaMemcpyAsync(f.data(), c->d_force, sizeof(double) * nf, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (size_t k = 0; k < nf; k++) dE_dR[k] = -f[k];
  }
  if (dE_dpsi) {
    RC(do_apply_h(c));
    const size_t nc = 2 * (size_t)h.ngpw * c->nstate;
    CK(cudaMemcpyAsync(dE_dpsi, c->d_c2, sizeof(double) * nc, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (size_t k = 0; k < nc; k++) dE_dpsi[k] = -dE_dpsi[k];
  }
  return 0;
}

int amdk_get_array(amdk_ctx *c, const char *name, void *dst, size_t bytes) {
  if (!c || !name || !dst) return AMDK_ERR_BADARG;
  cudaSetDevice(c->device);
  const HostSetup &h = c->hs;
  long npt = (long)h.nr[0] * h.nr[1] * h.nr[2];
  const void *src = nullptr;
  size_t n = 0;
  std::string k(name);
  if (k == "rho") { src = c->d_rho; n = npt * sizeof(double); }
  else if (k == "v_pot") { src = c->d_vpot; n = npt * sizeof(double); }
  else if (k == "rho2" && c->d_rho2) { src = c->d_rho2; n = npt * sizeof(double); }
  else if (k == "v_pot2" && c->d_vpot2) { src = c->d_vpot2; n = npt * sizeof(double); }
  else if (k == "rho_g") { src = c->d_rhog; n = h.ngrho * sizeof(double2); }
  else if (k == "c2") { src = c->d_c2; n = (size_t)h.ngpw * c->nstate * sizeof(double2); }
  else if (k == "c0") { src = c->d_c0; n = (size_t)h.ngpw * c->nstate * sizeof(double2); }
  else if (k == "nl") { src = c->d_nl; n = (size_t)c->nproj * c->nstate * sizeof(double); }
  else if (k == "vps") { src = c->d_vps; n = (size_t)h.nsp * h.ngrho * sizeof(double); }
  else if (k == "rhos") { src = c->d_rhos; n = (size_t)h.nsp * h.ngrho * sizeof(double); }
  else if (k == "twnl") { src = c->d_twnl; n = (size_t)h.nsp * h.nghmax * h.ngpw * sizeof(double); }
  else if (k == "eigrxvps") { src = c->d_evps; n = h.ngrho * sizeof(double2); }
  else if (k == "eigrxrhos") { src = c->d_erhos; n = h.ngrho * sizeof(double2); }
  else if (k == "vpp") { src = c->d_vpp; n = h.ngpw * sizeof(double); }
  else if (k == "force") { src = c->d_force; n = 3 * h.na_max * h.nsp * sizeof(double); }
  else if (k == "overlap") { src = c->d_gam; n = (size_t)c->nstate * c->nstate * sizeof(double); }
  else {
    set_error("amdk_get_array: unknown array " + k);
    return AMDK_ERR_BADARG;
  }
  if (bytes < n) {
    set_error("amdk_get_array: destination too small for " + k);
    return AMDK_ERR_BADARG;
  }
  CK(cudaStreamSynchronize(c->st));
  if (n && src) CK(cudaMemcpy(dst, src, n, cudaMemcpyDeviceToHost));
  return 0;
}

int amdk_fft_sphere(amdk_ctx *c, int sign, double *coef, double *grid) {
  if (!c || !coef || !grid || (sign != 1 && sign != -1)) return AMDK_ERR_BADARG;
  cudaSetDevice(c->device);
  const HostSetup &h = c->hs;
  long npt = (long)h.nr[0] * h.nr[1] * h.nr[2];
  if (sign == -1) {
    CK(cudaMemcpyAsync(c->d_vxg, coef, sizeof(double2) * h.ngrho, cudaMemcpyHostToDevice, c->st));
    ++c->nlaunch;
    k_conj_field<<<nblk(h.ngrho), NTHR, 0, c->st>>>(h.ngrho, c->d_vxg, c->d_fm);
    RC(field_to_grid(c, 1, c->d_vxg, c->d_fm, c->d_cgrid));
    CK(cudaMemcpyAsync(grid, c->d_cgrid, sizeof(double2) * npt, cudaMemcpyDeviceToHost, c->st));
  } else {
    CK(cudaMemcpyAsync(c->d_cgrid, grid, sizeof(double2) * npt, cudaMemcpyHostToDevice, c->st));
    RC(grid_to_rays(c, 1, c->d_cgrid, nullptr));
    ++c->nlaunch;
    k_gather_p<double2><<<nblk(h.ngrho), NTHR, 0, c->st>>>(h.ngrho, c->d_posp, (double2 *)c->d_rbf, 1.0 / (double)npt,
                                                           c->d_vxg);
    CK(cudaMemcpyAsync(coef, c->d_vxg, sizeof(double2) * h.ngrho, cudaMemcpyDeviceToHost, c->st));
  }
  CK(cudaStreamSynchronize(c->st));
  CK(cudaGetLastError());
  return 0;
}

int amdk_profile(amdk_ctx *c, int enable) {
  if (!c) return AMDK_ERR_BADARG;
  cudaSetDevice(c->device);
  CK(cudaStreamSynchronize(c->st));
  prof_harvest(c);
  c->prof = enable != 0;
  for (int k = 0; k < KT_N; k++) {
    c->kt_count[k] = 0;
    c->kt_ms[k] = 0;
    c->kt_bytes[k] = 0;
  }
  return 0;
}

int amdk_profile_get(amdk_ctx *c, int kind, long *launches, double *total_ms, double *bytes) {
  if (!c || kind < 0 || kind >= KT_N) return AMDK_ERR_BADARG;
  cudaSetDevice(c->device);
  CK(cudaStreamSynchronize(c->st));
  prof_harvest(c);
  if (launches) *launches = c->kt_count[kind];
  if (total_ms) *total_ms = c->kt_ms[kind];
  if (bytes) *bytes = c->kt_bytes[kind];
  return 0;
}

// ---------------------------------------------------------------------------
// amdk_fft_sphere_noalloc: the density-sphere FFT for callers that cannot
// allocate device memory.  Its scratch (the ray buffer, the slab buffer and
// the -G field of one FP64 transform) lives in this file-scope array, which
// every GPU that loads the library holds until the process exits.  Host code
// must not pass the array's name to a kernel: on the host that name is only a
// stand-in, so each call looks the device address up with
// cudaGetSymbolAddress on the current device (a cached address would go stale
// if the caller reset the device and a new context took its place).
// ---------------------------------------------------------------------------
constexpr size_t kNoAllocScratchBytes = (size_t)24 << 20;  // 24 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of the scratch array on the current device.
static int noalloc_scratch(unsigned char **out) {
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    set_error(std::string("amdk_fft_sphere_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
    return AMDK_ERR_CUDA;
  }
  *out = (unsigned char *)p;
  return 0;
}

// Scratch bytes one transform of this context's density sphere needs.
static size_t noalloc_bytes(amdk_ctx *c, size_t *rbytes, size_t *sbytes) {
  auto round256 = [](size_t b) { return (b + 255) & ~(size_t)255; };
  *rbytes = round256((size_t)rstride(c, 1) * sizeof(double2));
  *sbytes = round256((size_t)sstride(c, 1) * sizeof(double2));
  return *rbytes + *sbytes + round256((size_t)c->hs.ngrho * sizeof(double2));
}

int amdk_fft_sphere_noalloc(amdk_ctx *c, int sign, double *coef, double *grid) {
  if (!c || !coef || !grid || (sign != 1 && sign != -1)) {
    set_error("amdk_fft_sphere_noalloc: null pointer or sign not +-1");
    return AMDK_ERR_BADARG;
  }
  CK(cudaSetDevice(c->device));
  const HostSetup &h = c->hs;
  size_t rbytes = 0, sbytes = 0;
  const size_t need = noalloc_bytes(c, &rbytes, &sbytes);
  if (need > kNoAllocScratchBytes) {
    set_error("amdk_fft_sphere_noalloc: this grid needs " + std::to_string(need) +
              " bytes of scratch; the fixed maximum is " + std::to_string(kNoAllocScratchBytes) +
              " bytes (use amdk_fft_sphere)");
    return AMDK_ERR_UNSUPPORTED;
  }
  unsigned char *base = nullptr;
  RC(noalloc_scratch(&base));
  // the inputs may have been written on any stream of the caller's (an
  // OpenACC async queue, a torch stream, the legacy default stream): wait
  // for all work on the device before reading them
  CK(cudaDeviceSynchronize());
  const XBufs b{base, base + rbytes};
  double2 *FM = (double2 *)(base + rbytes + sbytes);
  const long npt = (long)h.nr[0] * h.nr[1] * h.nr[2];
  if (sign == -1) {
    // coef (+G half) -> complex grid; the -G values are conj(coef)
    ++c->nlaunch;
    k_conj_field<<<nblk(h.ngrho), NTHR, 0, c->st>>>(h.ngrho, (const double2 *)coef, FM);
    RC(field_to_grid<double2>(c, 1, (const double2 *)coef, FM, (double2 *)grid, b));
  } else {
    // complex grid -> coef = F(+G)/N
    RC(grid_to_rays<double2>(c, 1, (const double2 *)grid, nullptr, b));
    ++c->nlaunch;
    k_gather_p<double2><<<nblk(h.ngrho), NTHR, 0, c->st>>>(h.ngrho, c->d_posp, (double2 *)b.rays, 1.0 / (double)npt,
                                                           (double2 *)coef);
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int amdk_launch_count(amdk_ctx *c, long *n) {
  if (!c || !n) return AMDK_ERR_BADARG;
  *n = c->nlaunch;
  return 0;
}

int amdk_last_iteration_ms(amdk_ctx *c, double *ms) {
  if (!c || !ms) return AMDK_ERR_BADARG;
  *ms = c->last_ms;
  return 0;
}

// ------------------------------------------------------------------ slab decomposition entries
int amdk_slab_layout(const amdk_system *sys, int nranks, int *g_owner, int *plane0) {
  if (!sys) {
    set_error("amdk_slab_layout: null system");
    return AMDK_ERR_BADARG;
  }
  HostSetup h;
  RC(host_setup(sys, h, true));
  std::vector<int> ray_ky, ray_kz, posp, posm, owner, p0;
  ray_tables(h, ray_ky, ray_kz, posp, posm);
  RC(slab_partition(h, nranks, ray_ky, ray_kz, posp, owner, p0));
  if (g_owner)
    for (int ig = 0; ig < h.ngpw; ig++) g_owner[ig] = owner[posp[ig] / h.nr[0]];
  if (plane0) std::memcpy(plane0, p0.data(), sizeof(int) * p0.size());
  return 0;
}

int amdk_slab_create(amdk_ctx *c, int nranks, int rank, amdk_slab **out) {
  if (!c || !out) {
    set_error("amdk_slab_create: null argument");
    return AMDK_ERR_BADARG;
  }
  *out = nullptr;
  CK(cudaSetDevice(c->device));
  amdk_slab *s = new (std::nothrow) amdk_slab();
  if (!s) return AMDK_ERR_ALLOC;
  const int rc = slab_create(c, nranks, rank, s);
  if (rc) {
    delete s;
    return rc;
  }
  *out = s;
  return 0;
}

int amdk_slab_info_get(amdk_slab *s, amdk_slab_info *info) {
  if (!s || !info) return AMDK_ERR_BADARG;
  std::memset(info, 0, sizeof(*info));
  info->nranks = s->nranks;
  info->rank = s->rank;
  info->ngpw_local = s->ng;
  info->nray_local = s->nray_loc;
  info->plane0 = s->plane0[s->rank];
  info->nplane = s->nplane;
  info->gzero_local = s->gzero;
  info->elem_bytes = (s->precision == AMDK_MIXED) ? (int)sizeof(float2) : (int)sizeof(double2);
  for (int o = 0; o < s->nranks; o++) {
    info->send_elems[o] = (long)(s->plane0[o + 1] - s->plane0[o]) * s->nray_loc;
    info->recv_elems[o] = (long)s->nplane * (s->seg_r0[o + 1] - s->seg_r0[o]);
  }
  return 0;
}

int amdk_slab_local_g(amdk_slab *s, int *ig) {
  if (!s || !ig) return AMDK_ERR_BADARG;
  if (s->ng) std::memcpy(ig, s->local_g.data(), sizeof(int) * s->ng);
  return 0;
}

// the call's stream, or the context's stream with the call waited for
static int slab_finish(amdk_slab *s, void *stream) {
  if (!stream) CK(cudaStreamSynchronize(s->c->st));
  return 0;
}

int amdk_slab_pairs_out(amdk_slab *s, const double *c0, int band0, int npairs, void *send, void *stream) {
  if (!s || !c0 || !send) return AMDK_ERR_BADARG;
  RC(slab_check_pairs(s, band0, npairs));
  CK(cudaSetDevice(s->c->device));
  const cudaStream_t st = slab_stream(s, stream);
  if (s->precision == AMDK_MIXED) RC(slab_pairs_out_t<float2>(s, (const double2 *)c0, band0, npairs, (float2 *)send, st));
  else RC(slab_pairs_out_t<double2>(s, (const double2 *)c0, band0, npairs, (double2 *)send, st));
  return slab_finish(s, stream);
}

int amdk_slab_planes_vpsi(amdk_slab *s, void *recv, int npairs, const double *v, void *stream) {
  if (!s || !recv || !v) return AMDK_ERR_BADARG;
  RC(slab_check_pairs(s, 0, npairs));
  CK(cudaSetDevice(s->c->device));
  const cudaStream_t st = slab_stream(s, stream);
  if (s->precision == AMDK_MIXED) RC(slab_vpsi_t<float2>(s, (float2 *)recv, npairs, v, st));
  else RC(slab_vpsi_t<double2>(s, (double2 *)recv, npairs, v, st));
  return slab_finish(s, stream);
}

int amdk_slab_planes_density(amdk_slab *s, const void *recv, int band0, int npairs, double *rho, int accumulate,
                             void *stream) {
  if (!s || !recv || !rho) return AMDK_ERR_BADARG;
  RC(slab_check_pairs(s, band0, npairs));
  CK(cudaSetDevice(s->c->device));
  const cudaStream_t st = slab_stream(s, stream);
  if (s->precision == AMDK_MIXED) RC(slab_density_t<float2>(s, (const float2 *)recv, band0, npairs, rho, accumulate, st));
  else RC(slab_density_t<double2>(s, (const double2 *)recv, band0, npairs, rho, accumulate, st));
  return slab_finish(s, stream);
}

int amdk_slab_pairs_in(amdk_slab *s, void *back, const double *c0, int band0, int npairs, double *c2, void *stream) {
  if (!s || !back || !c0 || !c2) return AMDK_ERR_BADARG;
  RC(slab_check_pairs(s, band0, npairs));
  CK(cudaSetDevice(s->c->device));
  const cudaStream_t st = slab_stream(s, stream);
  if (s->precision == AMDK_MIXED)
    RC(slab_pairs_in_t<float2>(s, (float2 *)back, (const double2 *)c0, band0, npairs, (double2 *)c2, st));
  else RC(slab_pairs_in_t<double2>(s, (double2 *)back, (const double2 *)c0, band0, npairs, (double2 *)c2, st));
  return slab_finish(s, stream);
}

int amdk_slab_gram(amdk_slab *s, const double *a, const double *b, int n, double *out, void *stream) {
  if (!s || !a || !b || !out || n < 1 || n > s->c->nstate) {
    set_error("amdk_slab_gram: null pointer or band count outside 1..nstate");
    return AMDK_ERR_BADARG;
  }
  amdk_ctx *c = s->c;
  CK(cudaSetDevice(c->device));
  const cudaStream_t st = slab_stream(s, stream);
  if (s->ng == 0) {
    CK(cudaMemsetAsync(out, 0, sizeof(double) * n * n, st));
    CK(cudaStreamSynchronize(st));
    return 0;
  }
  // the FP64 tensor-core product over the rank's 2 ngpw_local real components
  RC(dg_tn(c, a, n, b, n, 2.0, out, n, a == b, 2L * s->ng, st));
  if (s->gzero == 0) {  // the rank holding G = 0 (local index 0) removes its doubled term
    ++c->nlaunch;
    k_g0_correct<<<dim3(nblk(n), n), NTHR, 0, st>>>(n, s->ng, (const double2 *)a, (const double2 *)b, out, c->d_occ, 0,
                                                    0);
  }
  CK(cudaGetLastError());
  int expired = 0;
  CK(cudaMemcpyAsync(&expired, c->d_info + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (expired) {
    CK(cudaMemset(c->d_info + 1, 0, sizeof(int)));
    set_error("amdk_slab_gram: a pipeline wait of the FP64 tensor-core product gave up");
    return AMDK_ERR_TIMEOUT;
  }
  return 0;
}

int amdk_slab_destroy(amdk_slab *s) {
  if (!s) return 0;
  cudaSetDevice(s->c->device);
  cudaDeviceSynchronize();
  delete s;
  return 0;
}

}  // extern "C"
