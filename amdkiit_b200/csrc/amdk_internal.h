// Internal declarations of libamdk (host setup, device context, kernels).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/amdk.h"

namespace amdk {

constexpr int NSPLN = 5000;     // max_parameter_pp.f90:3
constexpr int MAXNGH = 120;     // max_parameter_pp.f90:8
constexpr int MPRO = 4;
constexpr int LMAXX = 5;
constexpr double RAGGIO = 1.2;  // system_data_types.f90:72

void set_error(const std::string &msg);

// Result of the host-side setup that the reference performs in
// init_module.f90:3-162 (all FP64, once per run).
struct HostSetup {
  double a_cell[9], b_cell[9], alat, omega, tpiba, tpiba2, gcut_pw, gcut_rho, ecut;
  int nr[3], nrl[3];
  int nsp, na[AMDK_MAXSP], na_max, nat, zv[AMDK_MAXSP], xc, symmetry;
  bool upf;
  std::vector<int> isa_is, isa_ia;
  std::vector<double> atco;
  // G vectors (gvectors.f90, sorted with the EPSGX tie-break)
  int ngpw, ngrho, ngrays, nhrays;
  std::vector<int> inyh;       // 3*ngrho, 1-based centred grid indices
  std::vector<double> hg, gvec;
  std::vector<int> mapp, mapm; // reference maps (1-based, nrlead(1) leading dim)
  std::vector<int> xrays;      // nrl2*nrl3 ray numbers (1-based, 0 = none)
  std::vector<int> msp;        // ray -> i + (j-1)*nrl2
  // pseudopotential tables
  int ngh[AMDK_MAXSP], nghmax;
  int nghtol[AMDK_MAXSP][MAXNGH], lpval[AMDK_MAXSP][MAXNGH], lfval[AMDK_MAXSP][MAXNGH];
  double wsg[AMDK_MAXSP][MAXNGH];
  double hlsg[AMDK_MAXSP][LMAXX][MPRO][MPRO];
  std::vector<double> ggng, ggnh;                 // spline abscissae
  std::vector<double> voo[AMDK_MAXSP];            // local form factor on ggnh
  std::vector<double> wns[AMDK_MAXSP];            // projector tables on ggng (ngh*NSPLN)
  int nstate;
  std::vector<double> occ;
  // open shell (LSD): bands [0, nel_up) spin 1, [nel_up, nstate) spin 2
  bool lsd = false;
  int nel_up = 0;
};

// Host setup entry: returns 0 or an AMDK_ERR code (message via set_error).
int host_setup(const amdk_system *sys, HostSetup &hs, bool gvectors_only = false);

// Natural cubic spline (spline.f90): h and second derivatives for a table.
void spline_coeffs(int n, const double *xp, const double *yp, std::vector<double> &h, std::vector<double> &sdd);

}  // namespace amdk
