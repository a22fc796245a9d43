// C ABI of the LNV / McWeeny solver (declarations in include/cq_b200.h).
#include <algorithm>
#include <cstring>
#include <functional>
#include <string>

#include "chain.hpp"

using namespace cqb;

struct cq_system;  // defined in capi.cpp: its first member is the cqb::System
namespace cqb { System& system_of(cq_system* s); int guarded_call(const std::function<void()>& f); }

struct cq_lnv {
  std::unique_ptr<LNVSolver> solver;
};

static void fill_result(const LNVStats& st, cq_lnv_result* r) {
  if (!r) return;
  r->energy = st.energy;
  r->electrons = st.electrons;
  r->residual = st.last_residual;
  r->invs_omega = st.invs_omega;
  r->mcw_sweeps = st.mcw_sweeps;
  r->early_iters = st.early_iters;
  r->late_iters = st.late_iters;
  r->ne_corrections = st.ne_corrections;
  r->inflexions = st.inflexions;
  r->converged = st.converged;
  r->outer_iters = st.outer_iters;
  r->graph_launches = st.graph_launches;
  r->n_products = st.n_products;
  r->flops = st.flops;
  r->n_products_mixed = st.n_products_mixed;
  r->flops_mixed = st.flops_mixed;
  r->split_restarts = st.split_restarts;
}

static DMat* matrix_by_name(LNVSolver& L, const char* name) {
  std::string n(name ? name : "");
  if (n == "L") return &L.L;
  if (n == "K") return &L.K;
  if (n == "T") return &L.T;
  if (n == "S") return &L.Smat;
  if (n == "H") return &L.Hmat;
  if (n == "phi") return &L.phi;
  throw Error(CQ_ERR_ARG, "unknown LNV matrix " + n);
}

extern "C" {

int cq_lnv_params_default(cq_lnv_params* p) {
  if (!p) return CQ_ERR_ARG;
  p->n_L_iterations = 50;
  p->tolerance = 1.0e-7;
  p->maxpulay = 5;
  p->minpulaystep = 1.0e-3;
  p->maxpulaystep = 0.1;
  p->lintol = 0.1;
  p->global_tolerance = 0;
  p->vary_mu = 1;
  p->invs_max_steps = 100;
  p->invs_delta_tol = 1.0e-4;
  p->invs_tol = 1.0e-2;
  p->exact = 1;
  p->max_outer = 40;
  p->mixed = 0;
  p->mixed_tolerance = 0.0;
  p->fp64_mcw_sweeps = 0;
  p->graphs = 1;
  p->mixed_mcw = 0;
  p->fp64_continue = 1;
  p->split_parts = 3;
  p->mixed_max_outer = 0;
  p->fp64_tensor = 1;
  return CQ_OK;
}

int cq_lnv_create(cq_system* sys, const int* ranges, double ne_spin, const cq_lnv_params* p, cq_lnv** out) {
  return guarded_call([&] {
    CQ_CHECK(sys && ranges && out, CQ_ERR_ARG, "null argument");
    cq_lnv_params prm;
    cq_lnv_params_default(&prm);
    if (p) prm = *p;
    CQ_CHECK(prm.maxpulay >= 1 && prm.maxpulay <= 16, CQ_ERR_ARG, "maxpulay must be 1..16");
    CQ_CHECK(ne_spin > 0, CQ_ERR_ARG, "ne_spin must be positive");
    CQ_CHECK(prm.split_parts == 0 || prm.split_parts == 2 || prm.split_parts == 3, CQ_ERR_ARG,
             "split_parts must be 0, 2 or 3");
    CQ_CHECK(prm.mixed_max_outer >= 0, CQ_ERR_ARG, "mixed_max_outer must be >= 0");
    auto s = std::make_unique<cq_lnv>();
    s->solver = std::make_unique<LNVSolver>(system_of(sys), ranges, ne_spin, prm);
    *out = s.release();
  });
}

int cq_lnv_destroy(cq_lnv* s) {
  return guarded_call([&] {
    if (s) {
      cudaStreamSynchronize(s->solver->S.stream);
      delete s;
    }
  });
}

int cq_lnv_set_SH(cq_lnv* s, const double* S, const double* H, int on_device) {
  return guarded_call([&] {
    CQ_CHECK(s && S && H, CQ_ERR_ARG, "null argument");
    LNVSolver& L = *s->solver;
    auto kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    CQ_CUDA(cudaMemcpyAsync(L.Smat.p, S, sizeof(double) * L.Smat.n, kind, L.S.stream));
    CQ_CUDA(cudaMemcpyAsync(L.Hmat.p, H, sizeof(double) * L.Hmat.n, kind, L.S.stream));
    if (!on_device) CQ_CUDA(cudaStreamSynchronize(L.S.stream));
  });
}

int cq_lnv_invert_S(cq_lnv* s, double* omega) {
  return guarded_call([&] {
    CQ_CHECK(s, CQ_ERR_ARG, "null argument");
    double w = s->solver->invert_S();
    if (omega) *omega = w;
  });
}

int cq_lnv_find_min_dm(cq_lnv* s, int resetL, cq_lnv_result* res) {
  return guarded_call([&] {
    CQ_CHECK(s, CQ_ERR_ARG, "null argument");
    LNVSolver& L = *s->solver;
    L.stats = LNVStats();
    L.find_min_dm(resetL != 0);
    fill_result(L.stats, res);
  });
}

int cq_lnv_get(cq_lnv* s, const char* name, double* out, int64_t cap, int on_device) {
  return guarded_call([&] {
    CQ_CHECK(s && out, CQ_ERR_ARG, "null argument");
    LNVSolver& L = *s->solver;
    DMat* m = matrix_by_name(L, name);
    CQ_CHECK(cap >= m->n, CQ_ERR_ARG, "output buffer too small");
    CQ_CUDA(cudaMemcpyAsync(out, m->p, sizeof(double) * m->n, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                            L.S.stream));
    CQ_CUDA(cudaStreamSynchronize(L.S.stream));
  });
}

int cq_lnv_put(cq_lnv* s, const char* name, const double* in, int on_device) {
  return guarded_call([&] {
    CQ_CHECK(s && in, CQ_ERR_ARG, "null argument");
    LNVSolver& L = *s->solver;
    std::string n(name ? name : "");
    CQ_CHECK(n == "L" || n == "T", CQ_ERR_ARG, "only L and T can be loaded");
    DMat* m = matrix_by_name(L, name);
    CQ_CUDA(cudaMemcpyAsync(m->p, in, sizeof(double) * m->n, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                            L.S.stream));
    CQ_CUDA(cudaStreamSynchronize(L.S.stream));
  });
}

int cq_pulay_alphas(int ipulay, const double* Aij, int n, int max_n, double* alphas) {
  return guarded_call([&] {
    CQ_CHECK(Aij && alphas && n >= 1 && n <= max_n && ipulay >= 1 && ipulay <= max_n, CQ_ERR_ARG, "bad Pulay arguments");
    LNVSolver::do_pulay(ipulay, Aij, n, max_n, alphas);
  });
}

int cq_solve_cubic(double a, double b, double c, double guess, double* x) {
  return guarded_call([&] {
    CQ_CHECK(x != nullptr, CQ_ERR_ARG, "null argument");
    *x = LNVSolver::solve_cubic(a, b, c, guess);
  });
}

int cq_lnv_solve(cq_lnv* s, cq_lnv_result* res) {
  return guarded_call([&] {
    CQ_CHECK(s, CQ_ERR_ARG, "null argument");
    LNVSolver& L = *s->solver;
    L.solve();
    fill_result(L.stats, res);
  });
}

int cq_lnv_solve_host(cq_lnv* s, const double* S, const double* H, double* L_out, double* K_out, cq_lnv_result* res) {
  return guarded_call([&] {
    CQ_CHECK(s && S && H, CQ_ERR_ARG, "null argument");
    LNVSolver& L = *s->solver;
    CQ_CUDA(cudaMemcpyAsync(L.Smat.p, S, sizeof(double) * L.Smat.n, cudaMemcpyHostToDevice, L.S.stream));
    CQ_CUDA(cudaMemcpyAsync(L.Hmat.p, H, sizeof(double) * L.Hmat.n, cudaMemcpyHostToDevice, L.S.stream));
    L.solve();
    if (L_out) CQ_CUDA(cudaMemcpyAsync(L_out, L.L.p, sizeof(double) * L.L.n, cudaMemcpyDeviceToHost, L.S.stream));
    if (K_out) CQ_CUDA(cudaMemcpyAsync(K_out, L.K.p, sizeof(double) * L.K.n, cudaMemcpyDeviceToHost, L.S.stream));
    CQ_CUDA(cudaStreamSynchronize(L.S.stream));
    fill_result(L.stats, res);
  });
}

int cq_lnv_force_matrices(cq_lnv* s, double* M12, double* M4, int on_device) {
  return guarded_call([&] {
    CQ_CHECK(s, CQ_ERR_ARG, "null argument");
    LNVSolver& L = *s->solver;
    DMat m12 = L.temp(LNVSolver::RS), m4 = L.temp(LNVSolver::RH);
    L.force_matrices(m12, m4);
    const auto kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (M12) CQ_CUDA(cudaMemcpyAsync(M12, m12.p, sizeof(double) * m12.n, kind, L.S.stream));
    if (M4) CQ_CUDA(cudaMemcpyAsync(M4, m4.p, sizeof(double) * m4.n, kind, L.S.stream));
    CQ_CUDA(cudaStreamSynchronize(L.S.stream));
  });
}

int cq_lnv_reduction_log(cq_lnv* s, int enable, double* out, int64_t cap, int64_t* n) {
  return guarded_call([&] {
    CQ_CHECK(s, CQ_ERR_ARG, "null argument");
    LNVSolver& L = *s->solver;
    if (n) *n = (int64_t)L.rlog.size();
    if (out) std::memcpy(out, L.rlog.data(), sizeof(double) * std::min<int64_t>(cap, (int64_t)L.rlog.size()));
    L.rlog_on = enable != 0;
    L.rlog.clear();
  });
}

int cq_lnv_residual_history(cq_lnv* s, double* out, int64_t cap, int64_t* n) {
  return guarded_call([&] {
    CQ_CHECK(s && s->solver && n, CQ_ERR_ARG, "null argument");
    const std::vector<double>& g = s->solver->glog;
    const int f = LNVSolver::kLogFields;
    *n = (int64_t)g.size() / f;
    if (out) std::memcpy(out, g.data(), sizeof(double) * f * std::min<int64_t>(cap, *n));
  });
}

int cq_lnv_set_h_rebuild(cq_lnv* s, cq_h_rebuild_fn fn, void* user) {
  return guarded_call([&] {
    CQ_CHECK(s && s->solver, CQ_ERR_ARG, "null solver");
    s->solver->h_rebuild = fn;
    s->solver->h_rebuild_user = fn ? user : nullptr;
  });
}

}  // extern "C"
