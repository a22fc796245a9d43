// LNV / McWeeny solver state (see chain.cpp).
#pragma once
#include <chrono>
#include <initializer_list>
#include <utility>
#include <vector>

#include "cq_internal.hpp"

namespace cqb {

class LNVSolver;

// a device block matrix of one named range; temporaries return to their pool on destruction
struct DMat {
  int rng = -1;
  double* p = nullptr;
  int64_t n = 0;
  LNVSolver* owner = nullptr;
  DMat() = default;
  DMat(int r, double* ptr, int64_t len, LNVSolver* o) : rng(r), p(ptr), n(len), owner(o) {}
  DMat(const DMat&) = delete;
  DMat& operator=(const DMat&) = delete;
  DMat(DMat&& o) noexcept : rng(o.rng), p(o.p), n(o.n), owner(o.owner) { o.p = nullptr; o.owner = nullptr; }
  DMat& operator=(DMat&& o) noexcept {
    if (this != &o) {
      this->~DMat();
      rng = o.rng; p = o.p; n = o.n; owner = o.owner;
      o.p = nullptr; o.owner = nullptr;
    }
    return *this;
  }
  ~DMat();
};

bool sym_inverse_bk(double* A, int n);

struct LNVStats {
  int64_t n_products = 0, flops = 0, n_reductions = 0, n_lnv = 0, n_products_mixed = 0, flops_mixed = 0;
  int mcw_sweeps = 0, early_iters = 0, late_iters = 0, ne_corrections = 0, inflexions = 0, converged = 0;
  int outer_iters = 0;
  int split_restarts = 0;         // mixed form: FP64 phases started again from the McWeeny start
  int64_t graph_launches = 0;     // LNV calls run as CUDA graph launches
  double energy = 0, electrons = 0, last_energy = 0, last_residual = 0, invs_omega = 0;
  double mubar = 0, lambda = 0, hmin = 0, hmax = 0;
};

class LNVSolver {
 public:
  // named ranges of the chain, in the order of cq_lnv_create's range list
  enum Rng { RS = 0, RH, RL, RT, RLS, RLH, RLSL, RSLS, RTS, RTH, RTL, NR };
  enum MultId { L_S_LS = 0, L_H_LH, T_S_TS, SL_S_SLS, LS_L_LSL, HL_S_LSL, HLS_LS_L, SLS_LS_L, LSL_SL_H, TS_T_T,
                TH_T_L, T_H_TH, T_L_TL, TL_T_L, LH_L_SLS, LHL_SL_S };
  struct Mult { int type, a, b, c; };
  static const Mult kMults[];

  LNVSolver(System& sys, const int ranges[NR], double ne_spin, const cq_lnv_params& p);
  ~LNVSolver();

  System& S;
  cq_lnv_params prm;
  int R[NR];
  double ne, n_o;
  int ni_in_cell;
  double delta_e = 0.0;  // `save` variable of FindMinDM
  LNVStats stats;
  std::vector<double> rlog;   // every trace / product-trace value in call order, when rlog_on
  bool rlog_on = false;
  // per earlyDM / lateDM iteration: residual, band energy, products run so far, 1 if the iteration's
  // products were split-precision, host seconds since the solve started (the residual has just been
  // read from the device, so the time includes the iteration's device work) -- the reference's
  // PulayR / PulayE record, DMMinModule.f90:289-294
  static constexpr int kLogFields = 5;
  std::vector<double> glog;
  std::chrono::steady_clock::time_point t_solve = std::chrono::steady_clock::now();
  void log_iteration(double g, double energy) {
    if (glog.size() < (size_t)kLogFields << 16)
      glog.insert(glog.end(), {g, energy, (double)stats.n_products, use_mixed ? 1.0 : 0.0,
                               std::chrono::duration<double>(std::chrono::steady_clock::now() - t_solve).count()});
  }
  DMat Smat, Hmat, L, T, Ttran, LS, SL, K, phi;

  DMat temp(int rng);
  void release(DMat& m);

  double invert_S();
  void find_min_dm(bool resetL);
  // complete solve: T = S^-1, FindMinDM from the McWeeny start; with prm.mixed the products run in
  // split precision until the residual reaches prm.mixed_tolerance, then FindMinDM continues in FP64
  void solve();
  void purify(int sweeps);
  // M12 (S range) and M4 (H range) of the current L: the doM1 + doM2 and doM4 branches of
  // LNV_matrix_multiply, the density-matrix terms of the forces
  void force_matrices(DMat& M12, DMat& M4);
  bool use_mixed = false;   // current product arithmetic of mult_dispatch
  static void do_pulay(int iPulay, const double* Aij, int n, int max_n, double* al);
  static double solve_cubic(double a, double b, double c, double guess);
  void lnv(bool doK, bool doM3, bool dophi, bool doE, DMat* M3, DMat* phim, double* electrons, double* energy);

 private:
  // workspace of lnv(): fixed addresses so a call can be captured in a CUDA graph
  DMat wLH, wHL, wHLS, wSLH, wA, wBm, wCm, wSLS, wSLSLS, wLSLSL;
  bool ws_ready = false;
  void ensure_workspace();
  int lnv_body(bool doK, bool doM3, bool dophi, bool doE, DMat* M3, DMat* phim);
  struct LnvGraph {
    cudaGraphExec_t exec = nullptr;
    int64_t launches = 0, products = 0, flops = 0, products_mixed = 0, flops_mixed = 0;
    int nsum = 0;
  };
  std::map<std::vector<uintptr_t>, LnvGraph> graphs_;
  std::map<std::vector<uintptr_t>, int> seen_;
  std::vector<DevBuf<double>> owned_;
  std::vector<DevBuf<double>> pool_;
  std::map<int, std::vector<double*>> free_;
  DMat own(int rng);

  void product(const DMat& A, const DMat& B, DMat& C, MultId id);
  void mult_dispatch(ProductPlan& P, double* a, const double* b, double* c);
  void msum(double alpha, DMat& A, double beta, const DMat& B);
  void scale(double alpha, DMat& A);
  void transpose(const DMat& A, DMat& AT);
  double ptrace(const DMat& A, const DMat& B);
  void ptraces(std::initializer_list<std::pair<const DMat*, const DMat*>> ops, double* out);
  double trace(const DMat& A);
  void copy(DMat& dst, const DMat& src);
  void set_identity_onsite(DMat& A);
  void symmetrise_L();
  void tmt(const DMat& M, DMat& out, DMat& tl, const DMat& Tright);
  double gnorm(const DMat& A, const DMat& B);
  void init_mcw();
  void mcw_mm_nonds(DMat& RhoNew, double& energy, double& c);
  double mcw_min(int n_L_iterations);
  void correct_electron_number();
  bool line_min_L(DMat& M3, DMat& D, DMat& mtemp, DMat& SM3, double energy_in, double& energy_out, double& zeta);
  void project_search(DMat& search, DMat& SM3, DMat& Sphi, DMat& mtemp);
  void project_gradient(DMat& M3, DMat& SM3, DMat& Sphi, DMat& mtemp);
  int early_dm(int ndone, bool& inflex);
  int late_dm(int ndone, bool& done, double& deltaE);
 public:
  // minE.MixedLSelfConsistent: the caller's density and H rebuild from K, run by lateDM
  cq_h_rebuild_fn h_rebuild = nullptr;
  void* h_rebuild_user = nullptr;
 private:
  void rebuild_H();
};

}  // namespace cqb
