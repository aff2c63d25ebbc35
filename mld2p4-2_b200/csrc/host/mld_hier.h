// mld_hier.h -- host-side producers of the level hierarchy (C++).
//
// These restate, for the GPU drop-in's own callers, what the reference builds
// on the host before any apply: the pdegen problem (tests/pdegen), decoupled
// aggregation, the smoothed prolongator and Galerkin product, and the ILU(0)
// / diagonal smoother data.  The integer structure (aggregates, patterns) is
// the reference's exactly; values use the reference's operation order.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace mld {

struct CSR {
  int nr = 0, nc = 0;
  std::vector<int> irp, ja;
  std::vector<double> val;
  int64_t nnz() const { return irp.empty() ? 0 : irp[nr]; }
  bool present() const { return !irp.empty(); }
};

enum SmootherKind { SM_JACOBI = 1, SM_BJAC = 2, SM_FBGS = 3 };

struct Parms {
  // global (mld_dprec_type, mlprec/mld_d_prec_type.f90:84-110)
  int min_coarse_size = -1;   // < 0: 40 * n^(1/3)
  int max_levs = 20;
  double min_cr_ratio = 1.5;
  int outer_sweeps = 1;
  // per-level aggregation (mld_dml_parms defaults, mld_d_onelev_mod.f90:433-445)
  double aggr_thresh = 0.01;
  // smoother for levels < nlev
  int smoother = SM_BJAC;
  int sweeps_pre = 1, sweeps_post = 1;
  double damping = 1.0;  // extension (not in the reference)
  // coarsest level
  int coarse_solver = SM_BJAC;
  int coarse_sweeps = 1;
  // extension: >= 0 runs the sparse products of the smoothed prolongator and
  // the Galerkin product (mldg_spgemm) and the ILU(0) factorisations
  // (mldg_ilu0_factor) on this CUDA device, bit for bit the host's; < 0 on the host
  int setup_device = -1;
};

struct Level {
  CSR A;         // level matrix
  CSR P, R;      // maps to the previous level (level >= 1)
  std::vector<int> ilaggr;
  int naggr = 0;
  double omega = 0;
  int kind = SM_BJAC, sweeps_pre = 1, sweeps_post = 1;
  double damping = 1.0;
  CSR L, U, ND;  // ILU(0) factors, FBGS strict triangles / off-diagonal part
  std::vector<double> d;  // ILU 1/pivot, diag-solver inverse diagonal or FBGS diagonal a_ii
};

// tests/pdegen/mld_d_pde3d.f90:98-412 with constant coefficients
// coef = {a1,a2,a3,b1,b2,b3,c}, h = 1/(idim+hden)
void gen_pde3d(int idim, int hden, const double *coef, CSR &a);

// -div(kappa grad u) with a cell-centred kappa (idim^3 cells = unknowns),
// harmonic-mean face coefficients, zero Dirichlet boundaries, h = 1/(idim+1).
// The boundary face uses kappa of the cell itself.
void gen_kappa3d(int idim, const double *kappa, CSR &a);

// Hierarchy (mld_d_hierarchy_bld.f90:187-413) and smoothers
// (mld_d_smoothers_bld.f90:156-169).  Return 0 or an error code; msg set.
int hierarchy_build(const CSR &a, const Parms &p, std::vector<Level> &lv, std::string &msg);
int smoothers_build(std::vector<Level> &lv, const Parms &p, std::string &msg);

// building blocks (exposed for tests)
int dec_aggregate(const CSR &a, double theta, std::vector<int> &ilaggr, int &naggr);
// device >= 0: the three sparse products on that CUDA device (mldg_spgemm)
void smoothed_aggr_asb(const CSR &a, const std::vector<int> &ilaggr, int naggr, double &omega, int device,
                       CSR &P, CSR &R, CSR &Ac);
int ilu0_factor(const CSR &a, CSR &L, CSR &U, std::vector<double> &d);
int ilu0_factor_gpu(const CSR &a, CSR &L, CSR &U, std::vector<double> &d, int device, std::string &msg);
CSR transpose(const CSR &a);
CSR spgemm(const CSR &a, const CSR &b);

}  // namespace mld
