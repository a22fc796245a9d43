// LNV / McWeeny density-matrix minimisation on device-resident block matrices.
//
// Host control flow follows the reference routine by routine (one spin channel,
// nspin = 1, spin_factor = 2); every matrix operation is a device kernel and the
// host only reads the scalars the control flow branches on (traces, energies,
// electron counts) and solves the <=5x5 Pulay system.
//   mult_module.f90      LNV_matrix_multiply 1478-1823, symmetrise_L 1856-1893
//   DMMinModule.f90      FindMinDM 172-312, earlyDM 366-723, lateDM 809-1339,
//                        lineMinL 1395-1614, correct_electron_number_fixspin 1676-1817,
//                        SolveCubic 2072-2143
//   McWeeny.f90          McWMin 107-272, InitMcW 340-570, McW_matrix_multiply_nonds 620-740,
//                        McWXHX 908-946, McWRho0 961-987, GetHLimits 1020-1109
//   Pulay.f90            DoPulay2D_nospin 188-262 (Bunch-Kaufman inverse, restated below)
//   S_matrix_module.f90  Iter_Hott_InvS 746-963, HotInvS_mm 994-1032
#include <cmath>
#include <cstring>
#include <functional>

#include "chain.hpp"

namespace cqb {

// ---------------------------------------------------------------------------
// temporary matrices: per-range free lists, zeroed on hand-out (allocate_temp_matrix)
// ---------------------------------------------------------------------------
DMat LNVSolver::temp(int rng) {
  int r = R[rng];
  auto& fl = free_[r];
  double* p;
  if (!fl.empty()) { p = fl.back(); fl.pop_back(); }
  else {
    pool_.emplace_back();
    pool_.back().alloc(std::max<int64_t>(S.ranges[r]->length, 1), S.stream);
    p = pool_.back().p;
  }
  CQ_CUDA(cudaMemsetAsync(p, 0, sizeof(double) * std::max<int64_t>(S.ranges[r]->length, 1), S.stream));
  return DMat{rng, p, S.ranges[r]->length, this};
}
void LNVSolver::release(DMat& m) {
  if (m.owner && m.p) free_[R[m.rng]].push_back(m.p);
  m.p = nullptr;
  m.owner = nullptr;
}
DMat::~DMat() { if (owner) owner->release(*this); }

// ---------------------------------------------------------------------------
// matrix layer
// ---------------------------------------------------------------------------
// product table in mat_mult roles (type, a, b, c) -- mult_module.f90:571-...
const LNVSolver::Mult LNVSolver::kMults[] = {
    {1, RL, RS, RLS},     // L_S_LS
    {1, RL, RH, RLH},     // L_H_LH
    {1, RT, RS, RTS},     // T_S_TS
    {1, RLS, RS, RSLS},   // SL_S_SLS
    {1, RLS, RL, RLSL},   // LS_L_LSL
    {1, RLH, RS, RLSL},   // HL_S_LSL
    {2, RL, RLS, RLSL},   // HLS_LS_L == LSL_SL_L
    {2, RL, RLS, RSLS},   // SLS_LS_L
    {2, RH, RLS, RLSL},   // LSL_SL_H
    {2, RT, RT, RTS},     // TS_T_T
    {2, RL, RT, RTH},     // TH_T_L (type 2: rcut(TH) > rcut(L))
    {1, RT, RH, RTH},     // T_H_TH
    {1, RT, RL, RTL},     // T_L_TL
    {2, RL, RT, RTL},     // TL_T_L
    {1, RLH, RL, RSLS},   // LH_L_SLS (type 1 while rcut(SLS) >= rcut(LH), mult_module.f90:660-680)
    {2, RS, RLS, RSLS},   // LHL_SL_S (mult_module.f90:753-760)
};

void LNVSolver::product(const DMat& A, const DMat& B, DMat& C, MultId id) {
  const Mult& m = kMults[id];
  stats.n_products++;
  if (m.type == 1) {
    CQ_CHECK(A.rng == m.a && B.rng == m.b && C.rng == m.c, CQ_ERR_STATE, "product: operand ranges do not match the table");
    ProductPlan& P = get_plan(S, 1, R[m.a], R[m.b], R[m.c]);
    stats.flops += P.flops;
    mult_dispatch(P, A.p, B.p, C.p);
  } else {
    CQ_CHECK(C.rng == m.a && B.rng == m.b && A.rng == m.c, CQ_ERR_STATE, "product: operand ranges do not match the table");
    ProductPlan& P = get_plan(S, 2, R[m.a], R[m.b], R[m.c]);
    stats.flops += P.flops;
    mult_dispatch(P, C.p, B.p, const_cast<double*>(A.p));
  }
}

void LNVSolver::mult_dispatch(ProductPlan& P, double* a, const double* b, double* c) {
  // Split precision only where it pays: a 16 x 16 tensor-core tile holds one padded block, so
  // blocks of 8 x 8 or less (SZ, 4 x 4) run faster as FP64 products, which the phase keeps.
  if (use_mixed && S.max_nsf > 8) {
    stats.n_products_mixed++;
    stats.flops_mixed += P.flops;
    mat_mult_mixed(S, P.mult_type, P.ra, P.rb, P.rc, a, b, c, prm.split_parts);
  } else if (prm.mixed && prm.fp64_tensor && S.max_nsf > 8) {
    // the mixed form's FP64 products on the FP64 tensor cores (padded 16 x 16 blocks)
    launch_mat_mult(S, P, a, b, c, kPrecFp64Tensor);
  } else if (S.batch_submit) {
    S.batch_submit(P, a, b, c, prm.exact);
  } else {
    launch_mat_mult(S, P, a, b, c, prm.exact);
  }
}

void LNVSolver::solve() {
  stats = LNVStats();
  glog.clear();
  t_solve = std::chrono::steady_clock::now();
  delta_e = 0.0;
  // every solve starts from the state of a new solver: the matrices the chain carries from one
  // call to the next (L, phi, K, T and the products of L) are cleared
  for (DMat* m : {&L, &T, &Ttran, &LS, &SL, &K, &phi})
    CQ_CUDA(cudaMemsetAsync(m->p, 0, sizeof(double) * std::max<int64_t>(m->n, 1), S.stream));
  use_mixed = false;
  invert_S();                       // T = S^-1 in FP64 in both forms
  // no product of this system would run in split precision (mult_dispatch keeps blocks of 8 x 8
  // or less in FP64): the mixed form is the FP64 solve, in one phase
  if (!prm.mixed || S.max_nsf <= 8 || prm.split_parts == 0) {
    find_min_dm(true);
    return;
  }
  // split-precision phase to the hand-over residual, optional FP64 McWeeny purification sweeps,
  // then FP64 FindMinDM from that L to the final tolerance
  const double tol = prm.tolerance;
  const int max_outer_all = prm.max_outer;
  use_mixed = true;
  // hand-over residual: the three-part split carries the solve to the final tolerance (its products'
  // rounding, about 1e-7 of sum |a||b|, stalls the residual near 1e-8 on DZP Si), the two-part split
  // to 1e-6
  const double handover = prm.mixed_tolerance > 0 ? prm.mixed_tolerance
                                                 : (prm.split_parts == 3 ? std::max(tol, 1e-8) : 1e-6);
  prm.tolerance = handover;
  // the split phase gets a bounded number of passes and leaves at least one to the FP64 continuation:
  // where the split products' rounding keeps the residual above the hand-over (small dense clusters
  // with the two-part split), a stalled split phase must not use up the passes the FP64 phase needs
  const int split_passes = prm.mixed_max_outer > 0 ? prm.mixed_max_outer : (prm.split_parts == 3 ? 4 : 2);
  prm.max_outer = std::max(1, std::min(max_outer_all - 1, split_passes));
  try {
    find_min_dm(true);
  } catch (...) {
    prm.tolerance = tol;
    prm.max_outer = max_outer_all;
    use_mixed = false;
    throw;
  }
  prm.tolerance = tol;
  prm.max_outer = max_outer_all;
  use_mixed = false;
  if (prm.fp64_mcw_sweeps > 0) purify(prm.fp64_mcw_sweeps);
  if (!prm.fp64_continue) {
    // finish without further minimisation: the purified L, with K, the band energy and the
    // electron count evaluated in FP64 (errors in L enter the energy at second order)
    double el = 0, en = 0;
    lnv(true, false, true, true, nullptr, &phi, &el, &en);
    stats.energy = 2.0 * en;
    stats.electrons = 2.0 * el;
    return;
  }
  stats.converged = 0;
  // A split phase that ended far above its hand-over residual (more than 100 times) has stalled, and
  // on small dense DZP systems its L can lie where FP64 FindMinDM no longer reaches the tolerance
  // within the passes left (measured: 1e-3 Ha/atom from the FP64 solve): the FP64 phase then starts
  // again from the McWeeny start with the whole pass limit.  Otherwise both phases share the pass
  // limit of the FP64 solve (at least one FP64 pass) and FP64 continues from the split phase's L.
  const bool restart = stats.last_residual > 100.0 * handover;
  if (restart) {
    // the FP64 solve from the beginning: the chain's matrices cleared and T = S^-1 again, as at the
    // start of solve() (measured: a FindMinDM restart that kept the split phase's T and chain
    // matrices did not converge where the FP64 solve from the beginning does)
    stats.split_restarts++;
    for (DMat* m : {&L, &T, &Ttran, &LS, &SL, &K, &phi})
      CQ_CUDA(cudaMemsetAsync(m->p, 0, sizeof(double) * std::max<int64_t>(m->n, 1), S.stream));
    delta_e = 0.0;
    invert_S();
  }
  const int max_outer = prm.max_outer;
  prm.max_outer = restart ? max_outer : std::max(1, max_outer - stats.outer_iters);
  try {
    find_min_dm(restart);
  } catch (...) {
    prm.max_outer = max_outer;
    throw;
  }
  prm.max_outer = max_outer;
}

// McWeeny purification sweeps of L (McW_matrix_multiply_nonds, McWeeny.f90:620-740), kept while
// the purification parameter c stays in [0, 1].
void LNVSolver::purify(int sweeps) {
  DMat RhoNew = temp(RL);
  for (int n = 0; n < sweeps; ++n) {
    double omega, cn;
    mcw_mm_nonds(RhoNew, omega, cn);
    if (cn > 1.0 || cn < 0.0) break;
    msum(0.0, L, 1.0, RhoNew);
    symmetrise_L();
    stats.mcw_sweeps++;
  }
}

void LNVSolver::msum(double alpha, DMat& A, double beta, const DMat& B) {
  if (A.rng == B.rng) {
    dev_axpby(S, A.p, A.n, alpha, beta, B.p);
  } else {
    dev_matrix_add(S, R[A.rng], A.p, alpha, R[B.rng], B.p, beta);
  }
}
void LNVSolver::scale(double alpha, DMat& A) { dev_scale(S, A.p, A.n, alpha); }
void LNVSolver::transpose(const DMat& A, DMat& AT) { dev_transpose(S, R[A.rng], A.p, AT.p); }
double LNVSolver::ptrace(const DMat& A, const DMat& B) {
  CQ_CHECK(A.rng == B.rng, CQ_ERR_STATE, "matrix_product_trace needs equal ranges");
  stats.n_reductions++;
  double v = dev_dot(S, A.p, B.p, A.n);
  if (rlog_on) rlog.push_back(v);
  return v;
}
// Several matrix_product_trace values computed back to back and read with one host wait; the
// values (and the reduction log) are those of the same ptrace calls in this order.
void LNVSolver::ptraces(std::initializer_list<std::pair<const DMat*, const DMat*>> ops, double* out) {
  const double* xs[32] = {};
  const double* ys[32] = {};
  int64_t ns[32] = {};
  int k = 0;
  CQ_CHECK(ops.size() <= 32, CQ_ERR_ARG, "at most 32 traces per batch");
  for (auto& o : ops) {
    CQ_CHECK(o.first->rng == o.second->rng, CQ_ERR_STATE, "matrix_product_trace needs equal ranges");
    xs[k] = o.first->p; ys[k] = o.second->p; ns[k] = o.first->n;
    ++k;
  }
  stats.n_reductions += k;
  dev_dots(S, k, xs, ys, ns, out);
  if (rlog_on) rlog.insert(rlog.end(), out, out + k);
}
double LNVSolver::trace(const DMat& A) {
  stats.n_reductions++;
  double v = dev_trace(S, R[A.rng], A.p);
  if (rlog_on) rlog.push_back(v);
  return v;
}
void LNVSolver::copy(DMat& dst, const DMat& src) { dev_copy(S, dst.p, src.p, src.n); }

void LNVSolver::set_identity_onsite(DMat& A) {
  // store_matrix_value(..., j, j, one) on every onsite block
  dev_set_onsite_diag(S, R[A.rng], A.p, 1.0);
}

// ---------------------------------------------------------------------------
LNVSolver::LNVSolver(System& sys, const int ranges[NR], double ne_spin, const cq_lnv_params& p)
    : S(sys), prm(p), ne(ne_spin) {
  for (int i = 0; i < NR; ++i) {
    CQ_CHECK(ranges[i] >= 0 && ranges[i] < (int)S.ranges.size(), CQ_ERR_ARG, "LNV range index out of bounds");
    R[i] = ranges[i];
  }
  n_o = 0.0;
  for (int v : S.geo.nsf) n_o += (double)v;
  ni_in_cell = S.geo.n_atoms;
  Smat = own(RS); Hmat = own(RH); L = own(RL); T = own(RT); Ttran = own(RT);
  LS = own(RLS); SL = own(RLS); K = own(RH); phi = own(RL);
  ++S.n_solvers;                  // last: a constructor that throws leaves the count unchanged
}

DMat LNVSolver::own(int rng) {
  owned_.emplace_back();
  int64_t n = S.ranges[R[rng]]->length;
  owned_.back().alloc(std::max<int64_t>(n, 1), S.stream);
  CQ_CUDA(cudaMemsetAsync(owned_.back().p, 0, sizeof(double) * std::max<int64_t>(n, 1), S.stream));
  return DMat{rng, owned_.back().p, n, nullptr};
}

// ---- LNV_matrix_multiply (doK, doM3, dophi, doE) ---------------------------
// The temporaries of one call live in a workspace owned by the solver (allocate_temp_matrix
// hands out zeroed matrices; every one of them except A is fully overwritten by a product or a
// transpose before it is read, so only A is cleared), which keeps the device addresses of a call
// fixed: the call can then be captured once in a CUDA graph and replayed.
void LNVSolver::ensure_workspace() {
  if (ws_ready) return;
  wLH = own(RLH); wHL = own(RLH); wHLS = own(RLSL); wSLH = own(RLSL); wA = own(RLSL);
  wBm = own(RL); wCm = own(RL); wSLS = own(RSLS); wSLSLS = own(RL); wLSLSL = own(RH);
  ws_ready = true;
}

// Everything of one call up to the traces, enqueued on S.stream with no host synchronisation;
// returns the number of traces enqueued (their values: dev_dots_fetch).
int LNVSolver::lnv_body(bool doK, bool doM3, bool dophi, bool doE, DMat* M3, DMat* phim) {
  product(L, Smat, LS, L_S_LS);
  transpose(LS, SL);
  if (doM3) {
    product(L, Hmat, wLH, L_H_LH);
    transpose(wLH, wHL);
    CQ_CUDA(cudaMemsetAsync(wA.p, 0, sizeof(double) * std::max<int64_t>(wA.n, 1), S.stream));
    product(wHL, Smat, wHLS, HL_S_LSL);
    product(wHL, Smat, wHLS, HL_S_LSL);   // computed twice in the reference (mult_module.f90:1609, 1615)
    transpose(wHLS, wSLH);
    msum(0.0, wA, 2.0, wHLS);
    msum(1.0, wA, 1.0, wSLH);
    product(wA, SL, wBm, HLS_LS_L);
    transpose(wBm, wCm);
  }
  if (dophi) {
    product(SL, Smat, wSLS, SL_S_SLS);
    product(wSLS, SL, wSLSLS, SLS_LS_L);
  }
  if (doK || doE) {
    DMat& LSL = wA;                      // A is dead here; LSL takes its matrix
    product(LS, L, LSL, LS_L_LSL);
    product(LSL, LS, wLSLSL, LSL_SL_H);
    msum(0.0, K, 3.0, LSL);
    msum(1.0, K, -2.0, wLSLSL);
  }
  if (doM3) {
    msum(0.0, *M3, 3.0, wHLS);
    msum(1.0, *M3, 3.0, wSLH);
    msum(1.0, *M3, -1.0, wBm);
    msum(1.0, *M3, -1.0, wCm);
  }
  if (dophi) msum(0.0, *phim, 1.0, wSLS);
  // Tr(HK), Tr(L SLS), Tr(L SLSLS), enqueued before phi is overwritten, in the reference's order
  // (mult_module.f90:1700-1800)
  const double* xs[3];
  const double* ys[3];
  int64_t ns[3];
  int k = 0;
  if (doE) { xs[k] = Hmat.p; ys[k] = K.p; ns[k] = Hmat.n; ++k; }
  if (dophi) {
    xs[k] = L.p; ys[k] = phim->p; ns[k] = L.n; ++k;
    xs[k] = L.p; ys[k] = wSLSLS.p; ns[k] = L.n; ++k;
  }
  dev_dots_enqueue(S, k, xs, ys, ns);
  if (dophi) msum(6.0, *phim, -6.0, wSLSLS);
  return k;
}

LNVSolver::~LNVSolver() {
  for (auto& g : graphs_) if (g.second.exec) cudaGraphExecDestroy(g.second.exec);
  --S.n_solvers;
}

// One LNV_matrix_multiply call.  With prm.graphs, the first call with a given set of operands runs
// directly (it builds and tunes the products' plans and allocates their buffers), the second is
// captured into a CUDA graph, and later ones replay that graph: one launch instead of ~60.
void LNVSolver::lnv(bool doK, bool doM3, bool dophi, bool doE, DMat* M3, DMat* phim, double* electrons, double* energy) {
  ensure_workspace();
  int nsum = 0;
  auto body = [&] { nsum = lnv_body(doK, doM3, dophi, doE, M3, phim); };
  if (!prm.graphs || S.prof.on) {
    body();
  } else {
    const std::vector<uintptr_t> key = {(uintptr_t)(doK | doM3 << 1 | dophi << 2 | doE << 3 | use_mixed << 4),
                                        (uintptr_t)(M3 ? M3->p : nullptr), (uintptr_t)(phim ? phim->p : nullptr)};
    auto it = graphs_.find(key);
    if (it != graphs_.end()) {
      LnvGraph& g = it->second;
      CQ_CUDA(cudaGraphLaunch(g.exec, S.stream));
      S.launches += g.launches;
      stats.n_products += g.products; stats.flops += g.flops;
      stats.n_products_mixed += g.products_mixed; stats.flops_mixed += g.flops_mixed;
      nsum = g.nsum;
      stats.graph_launches++;
    } else if (seen_[key]++ == 0) {
      body();
    } else {
      if (graphs_.size() >= 32) {        // bound the cache
        for (auto& g : graphs_) if (g.second.exec) cudaGraphExecDestroy(g.second.exec);
        graphs_.clear();
      }
      const int64_t l0 = S.launches, p0 = stats.n_products, f0 = stats.flops, pm0 = stats.n_products_mixed,
                    fm0 = stats.flops_mixed;
      CQ_CUDA(cudaStreamBeginCapture(S.stream, cudaStreamCaptureModeThreadLocal));
      cudaGraph_t graph = nullptr;
      try {
        body();
      } catch (...) {
        cudaStreamEndCapture(S.stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
      }
      CQ_CUDA(cudaStreamEndCapture(S.stream, &graph));
      LnvGraph g;
      cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
      cudaGraphDestroy(graph);
      CQ_CUDA(e);
      g.launches = S.launches - l0; g.products = stats.n_products - p0; g.flops = stats.flops - f0;
      g.products_mixed = stats.n_products_mixed - pm0; g.flops_mixed = stats.flops_mixed - fm0;
      g.nsum = nsum;
      CQ_CUDA(cudaGraphLaunch(g.exec, S.stream));
      graphs_[key] = g;
      stats.graph_launches++;
    }
  }
  double t[3] = {0, 0, 0};
  dev_dots_fetch(S, nsum, t);
  stats.n_reductions += nsum;
  if (rlog_on) rlog.insert(rlog.end(), t, t + nsum);
  if (doE) *energy = t[0];
  if (dophi) *electrons = 3.0 * t[doE ? 1 : 0] - 2.0 * t[doE ? 2 : 1];
  stats.n_lnv++;
}

void LNVSolver::force_matrices(DMat& M12, DMat& M4) {
  CQ_CHECK(M12.rng == RS && M4.rng == RH, CQ_ERR_STATE, "force matrices: M12 has the S range, M4 the H range");
  CQ_CHECK(S.ranges[R[RSLS]]->rcut >= S.ranges[R[RLH]]->rcut, CQ_ERR_STATE,
           "LH.L -> SLS is a type-1 product only while rcut(SLS) >= rcut(LH)");
  const bool um = use_mixed;
  use_mixed = false;
  product(L, Smat, LS, L_S_LS);
  transpose(LS, SL);
  DMat LH = temp(RLH), LHL = temp(RSLS);
  product(L, Hmat, LH, L_H_LH);
  product(LH, L, LHL, LH_L_SLS);
  DMat LHLSL = temp(RS), LSLHL = temp(RS);
  product(LHL, LS, LHLSL, LHL_SL_S);
  transpose(LHLSL, LSLHL);
  ensure_workspace();
  DMat& LSL = wA;
  product(LS, L, LSL, LS_L_LSL);
  product(LSL, LS, wLSLSL, LSL_SL_H);
  msum(0.0, M4, 12.0, LSL);
  msum(1.0, M4, -12.0, wLSLSL);
  msum(0.0, M12, 3.0, LHL);
  msum(1.0, M12, -2.0, LHLSL);
  msum(1.0, M12, -2.0, LSLHL);
  use_mixed = um;
}

void LNVSolver::symmetrise_L() {
  DMat tmp = temp(RL);
  transpose(L, tmp);
  msum(0.5, L, 0.5, tmp);
}

void LNVSolver::tmt(const DMat& M, DMat& out, DMat& tl, const DMat& Tright) {
  product(T, M, tl, T_L_TL);
  product(tl, Tright, out, TL_T_L);
}

double LNVSolver::gnorm(const DMat& A, const DMat& B) {
  double g = 2.0 * ptrace(A, B);
  if (!prm.global_tolerance) g /= (double)ni_in_cell;
  return g;
}

// ---- Iter_Hott_InvS / HotInvS_mm --------------------------------------------
double LNVSolver::invert_S() {
  DMat I = temp(RTS), T1 = temp(RT), Told = temp(RT), TM = temp(RTS);
  set_identity_onsite(I);
  scale(0.0, T);
  set_identity_onsite(T);
  // sum of squares of S in the reference's visiting order (row orbital, then column orbital)
  double tot = 0.0;
  {
    std::vector<double> hS(Smat.n);
    CQ_CUDA(cudaMemcpyAsync(hS.data(), Smat.p, sizeof(double) * Smat.n, cudaMemcpyDeviceToHost, S.stream));
    host_wait(S);
    RangeIndex& RI = *S.ranges[R[RS]];
    std::vector<int> cov = RI.nb_cover.download(S.stream);
    std::vector<int64_t> el = RI.nb_elem.download(S.stream);
    for (int p = 0; p < S.geo.n_prim; ++p) {
      int ndi = S.geo.nsf[S.geo.prim_global[p]];
      for (int e = RI.h_row_ptr[p]; e < RI.h_row_ptr[p + 1]; ++e) {
        int ndj = S.geo.cover_nsf[cov[e]];
        for (int n1 = 0; n1 < ndi; ++n1)
          for (int n2 = 0; n2 < ndj; ++n2) { double x = hS[el[e] + n1 + (int64_t)ndi * n2]; tot += x * x; }
      }
    }
  }
  double eps = 1.0 / tot;
  scale(0.0, T);
  msum(0.0, T, eps, Smat);
  double deltaomega = 0.0, oldomega = 0.0, omega = 0.0;
  for (int n = 1; n <= prm.invs_max_steps; ++n) {
    deltaomega *= 0.5;
    if (n < 3 || std::fabs(deltaomega) > prm.invs_delta_tol) {
      // HotInvS_mm
      DMat T0S = temp(RTS), Grad = temp(RT);
      product(T, Smat, T0S, T_S_TS);
      msum(0.0, TM, 1.0, I);
      msum(1.0, TM, -1.0, T0S);
      product(T0S, T, Grad, TS_T_T);
      msum(0.0, T1, 2.0, T);
      msum(1.0, T1, -1.0, Grad);
      omega = ptrace(TM, TM);
      deltaomega = omega - oldomega;
      if (omega > oldomega && oldomega != 0.0) {
        msum(0.0, T, 1.0, Told);
        omega = oldomega;
        break;
      }
      oldomega = omega;
      msum(0.0, Told, 1.0, T);
      msum(0.0, T, 1.0, T1);
    } else {
      break;
    }
  }
  if (omega / n_o > prm.invs_tol) {
    scale(0.0, T);
    set_identity_onsite(T);
  }
  stats.invs_omega = omega;
  return omega;
}

// ---- McWeeny -----------------------------------------------------------------
void LNVSolver::init_mcw() {
  DMat TS = temp(RTS);
  product(T, Smat, TS, T_S_TS);
  double SX = trace(TS);
  DMat XHX = temp(RL), mtemp = temp(RS);
  {
    DMat BA = temp(RTH);
    product(T, Hmat, BA, T_H_TH);
    product(BA, T, XHX, TH_T_L);
    msum(0.0, mtemp, 1.0, XHX);
  }
  double SXHX = ptrace(Smat, mtemp);
  double hmin, hmax;
  dev_h_limits(S, R[RH], Hmat.p, &hmin, &hmax);
  double A = 1.0 - SX / n_o;
  double mubar, lambda;
  if (n_o == ne) {
    mubar = 0.0; lambda = 0.0;
  } else {
    double mu1 = SXHX / n_o + hmax * A;
    double mu2 = (hmin * A * ne / (n_o - ne) - SXHX / n_o) / (n_o * A / (n_o - ne) - 1.0);
    if ((ne / (hmax - mu1)) < ((n_o - ne) / (mu1 - hmin))) { mubar = mu1; lambda = ne / (hmax - mu1); }
    else if ((ne / (hmax - mu2)) > ((n_o - ne) / (mu2 - hmin))) { mubar = mu2; lambda = (n_o - ne) / (mu2 - hmin); }
    else throw Error(CQ_ERR_NOT_CONVERGED, "InitMcW: Cannot find mubar.");
  }
  stats.mubar = mubar; stats.lambda = lambda; stats.hmin = hmin; stats.hmax = hmax;
  // McWRho0
  msum(0.0, L, (lambda * mubar + ne) / n_o, T);
  msum(1.0, L, -lambda / n_o, XHX);
}

void LNVSolver::mcw_mm_nonds(DMat& RhoNew, double& energy, double& c) {
  product(L, Smat, LS, L_S_LS);
  ensure_workspace();
  DMat& LSL = wA;                        // the LNV workspace's LSL-range matrix, free outside lnv()
  DMat LSLSL = temp(RL), top = temp(RS), bottom = temp(RS);
  product(LS, L, LSL, LS_L_LSL);
  product(LSL, LS, LSLSL, HLS_LS_L);
  msum(0.0, top, 1.0, LSL);
  msum(1.0, top, -1.0, LSLSL);
  msum(0.0, bottom, 1.0, L);
  msum(1.0, bottom, -1.0, LSL);
  double cc[2];
  ptraces({{&Smat, &top}, {&Smat, &bottom}}, cc);
  const double c1 = cc[0], c2 = cc[1];
  CQ_CHECK(std::fabs(c2) > 1e-15, CQ_ERR_NOT_CONVERGED, "McW_matrix_multiply: c2 is near zero");
  double cn = c1 / c2;
  c = cn;
  scale(0.0, RhoNew);
  msum(0.0, RhoNew, -1.0, LSLSL);
  msum(1.0, RhoNew, 1.0 + cn, LSL);
  if (cn < 0.5) {
    msum(1.0, RhoNew, 1.0 - 2.0 * cn, L);
    scale(1.0 / (1.0 - cn), RhoNew);
  } else {
    scale(1.0 / cn, RhoNew);
  }
  DMat bottomH = temp(RH);
  msum(0.0, bottomH, 1.0, RhoNew);
  energy = ptrace(bottomH, Hmat);
  if (std::fabs(c2) < 1.0e-6) c = -0.01;
}

double LNVSolver::mcw_min(int n_L_iterations) {
  double oldE = 1.0e30;
  DMat oldL = temp(RL), RhoNew = temp(RL);
  copy(oldL, L);
  double deltaE = delta_e;   // left unchanged when the first sweep is rejected
  int n_it = n_L_iterations + 1;
  for (int n = 1; n <= n_L_iterations; ++n) {
    double omega1, cn;
    mcw_mm_nonds(RhoNew, omega1, cn);
    if (omega1 > oldE || std::fabs(omega1 - oldE) < 1.0e-8 || cn > 1.0 || cn < 0.0) { n_it = n; break; }
    deltaE = 2.0 * (omega1 - oldE);
    msum(0.0, L, 1.0, RhoNew);
    oldE = omega1;
    symmetrise_L();
  }
  if (n_it < 3) msum(0.0, L, 1.0, oldL);
  stats.mcw_sweeps += n_it - 1;
  return deltaE;
}

// ---- DMMin -----------------------------------------------------------------
double LNVSolver::solve_cubic(double a, double b, double c, double guess) {
  const double twopi = 2.0 * M_PI;
  double Q = (a * a - 3.0 * b) / 9.0;
  double Rr = (2.0 * a * a * a - 9.0 * a * b + 27.0 * c) / 54.0;
  if (Rr * Rr < Q * Q * Q) {
    double theta = std::acos(Rr / (std::sqrt(Q * Q * Q)));
    double Tt = -2.0 * std::sqrt(Q);
    double z1 = Tt * std::cos(theta / 3.0) - (a / 3.0);
    double z2 = Tt * std::cos((theta + twopi) / 3.0) - (a / 3.0);
    double z3 = Tt * std::cos((theta - twopi) / 3.0) - (a / 3.0);
    if (std::fabs(z1) <= std::fabs(z2) && std::fabs(z1) <= std::fabs(z3)) return z1;
    if (std::fabs(z2) <= std::fabs(z3)) return z2;
    return z3;
  }
  Q = -Q;
  Rr = -Rr;
  double Ss = Rr + std::sqrt(Q * Q * Q + Rr * Rr);
  double Tt = Rr - std::sqrt(Q * Q * Q + Rr * Rr);
  Ss = Ss >= 0.0 ? std::pow(Ss, 1.0 / 3.0) : -std::pow(std::fabs(Ss), 1.0 / 3.0);
  Tt = Tt >= 0.0 ? std::pow(Tt, 1.0 / 3.0) : -std::pow(std::fabs(Tt), 1.0 / 3.0);
  double x = Ss + Tt - a / 3.0;
  if (std::fabs(x) > 10.0 * std::fabs(guess)) x = guess;
  return x;
}

void LNVSolver::correct_electron_number() {
  transpose(T, Ttran);
  DMat TL = temp(RTL), phi2 = temp(RL), Sphi = temp(RL), Sphi2 = temp(RL);
  const double ne0 = ne;
  bool done = false;
  int it = 0;
  while (!done && it < 20) {
    double electrons = 0, e2 = 0;
    lnv(false, false, true, false, nullptr, &phi, &electrons, nullptr);
    tmt(phi, Sphi, TL, Ttran);
    double g0 = ptrace(Sphi, phi);
    double step1 = (ne0 - electrons) / g0;
    double step = 0.1;
    if (std::fabs(ne0 - electrons) < 1.0e-9) {
      msum(1.0, L, step1, Sphi);
      done = true;
    } else {
      step = step1;
      msum(1.0, L, step1, Sphi);
      lnv(false, false, true, false, nullptr, &phi2, &e2, nullptr);
      tmt(phi2, Sphi2, TL, Ttran);
      double g1 = ptrace(phi, Sphi2);
      double D = electrons - ne0;
      double C = g0;
      double B = 3.0 * (e2 - electrons) / (step * step) - (g1 + 2.0 * g0) / step;
      double recA = (step * step * step) / (2.0 * (electrons - e2) + (g0 + g1) * step);
      B *= recA; C *= recA; D *= recA;
      double truestep = solve_cubic(B, C, D, step);
      msum(1.0, L, truestep - step, Sphi);
      if (truestep == step) {
        lnv(false, false, true, false, nullptr, &phi, &e2, nullptr);
        if (std::fabs(e2 - ne0) < 1e-4) done = true;
        it++;
      } else {
        done = true;
        lnv(false, false, true, false, nullptr, &phi, &e2, nullptr);
      }
    }
    stats.ne_corrections++;
  }
}

bool LNVSolver::line_min_L(DMat& M3, DMat& D, DMat& mtemp, DMat& SM3, double energy_in, double& energy_out,
                           double& zeta) {
  DMat M3old = temp(RL);
  copy(M3old, M3);
  double g0 = 2.0 * ptrace(D, M3);
  double ig0 = g0;
  double step = delta_e / g0;
  if (std::fabs(step) < 1.0e-2) step = 0.01;
  if (std::fabs(step) > 0.1) step = 0.1;
  msum(1.0, L, step, D);
  double el, e1;
  lnv(true, true, false, true, &M3, nullptr, &el, &e1);
  double energy_1 = 2.0 * e1;
  double gg[2];
  ptraces({{&D, &M3}, {&SM3, &M3}}, gg);
  double g1 = 2.0 * gg[0];
  double igcross = 2.0 * gg[1];
  tmt(M3, SM3, mtemp, T);
  double ig1 = 2.0 * ptrace(SM3, M3);
  double ig1_step = ig1;
  double Dq = energy_in, C = g0;
  double B = 3.0 * (energy_1 - Dq) / (step * step) - (g1 - 2.0 * C) / step;
  double A = (g1 - 2.0 * B * step - C) / (3.0 * step * step);
  double SQ = 4.0 * B * B - 12.0 * A * C;
  if (SQ < 0) return true;   // inflexion
  double truestep = std::fabs(A) > 1.0e-8 ? (-2.0 * B + std::sqrt(SQ)) / (6.0 * A) : -C / (2.0 * B);
  if (truestep < 1.e-04) truestep = 1.e-04;
  msum(1.0, L, truestep - step, D);
  symmetrise_L();
  double e2;
  lnv(true, true, false, true, &M3, nullptr, &el, &e2);
  energy_out = 2.0 * e2;
  delta_e = energy_out - energy_in;
  double lamG, interpG;
  if (truestep < step) {
    lamG = truestep / step;
    interpG = ig0 * (1 - lamG) * (1 - lamG) + ig1 * lamG * lamG + 2.0 * igcross * lamG * (1 - lamG);
    zeta = (interpG - ig1) / (ig0 - ig1);
  } else {
    tmt(M3, SM3, mtemp, T);
    double ii[2];
    ptraces({{&SM3, &M3}, {&SM3, &M3old}}, ii);
    ig1 = 2.0 * ii[0];
    igcross = 2.0 * ii[1];
    lamG = step / truestep;
    interpG = ig0 * (1 - lamG) * (1 - lamG) + ig1 * lamG * lamG + 2.0 * igcross * lamG * (1 - lamG);
    zeta = (interpG - ig1_step) / (ig0 - ig1_step);
  }
  return false;
}

void LNVSolver::project_search(DMat& search, DMat& SM3, DMat& Sphi, DMat& mtemp) {
  tmt(phi, Sphi, mtemp, T);
  double d[2];
  ptraces({{&SM3, &phi}, {&Sphi, &phi}}, d);
  const double e_dot_n = d[0], n_dot_n = d[1];
  if (std::fabs(n_dot_n) > 1.0e-8) msum(1.0, search, e_dot_n / n_dot_n, Sphi);
}

void LNVSolver::project_gradient(DMat& M3, DMat& SM3, DMat& Sphi, DMat& mtemp) {
  tmt(phi, Sphi, mtemp, T);
  double d[2];
  ptraces({{&SM3, &phi}, {&Sphi, &phi}}, d);
  double et = 2.0 * d[0], nt = 2.0 * d[1];
  if (std::fabs(nt) > 1.0e-8) {
    double f = et / nt;
    msum(1.0, SM3, -f, Sphi);
    msum(1.0, M3, -f, phi);
  }
}

// returns ndone; sets inflex
int LNVSolver::early_dm(int ndone, bool& inflex) {
  inflex = false;
  DMat M3 = temp(RL), SM3 = temp(RL), Sphi = temp(RL), mtemp = temp(RTL), search = temp(RL);
  if (prm.vary_mu) correct_electron_number();
  double el, e0;
  lnv(false, true, true, true, &M3, &phi, &el, &e0);
  double energy0 = 2.0 * e0;
  tmt(M3, SM3, mtemp, T);
  msum(0.0, search, -1.0, SM3);
  if (prm.vary_mu) project_search(search, SM3, Sphi, mtemp);
  delta_e = 0.0;
  for (int n_iter = 1; n_iter <= prm.n_L_iterations; ++n_iter) {
    double energy1, zeta;
    if (line_min_L(M3, search, mtemp, SM3, energy0, energy1, zeta)) { inflex = true; stats.inflexions++; return n_iter; }
    tmt(M3, SM3, mtemp, T);
    if (prm.vary_mu) correct_electron_number();
    double e1;
    lnv(false, true, true, true, &M3, &phi, &el, &e1);
    energy1 = 2.0 * e1;
    tmt(M3, SM3, mtemp, T);
    energy0 = energy1;
    msum(0.0, search, -1.0, SM3);
    if (prm.vary_mu) project_search(search, SM3, Sphi, mtemp);
    double g0 = gnorm(M3, SM3);
    CQ_CHECK(std::isfinite(g0) && std::isfinite(energy0), CQ_ERR_NOT_CONVERGED,
             "earlyDM: the residual or the energy is not finite");
    stats.early_iters++;
    stats.last_energy = energy0;
    stats.last_residual = g0;
    log_iteration(g0, energy0);
    if (std::fabs(zeta) < prm.lintol) return n_iter;
  }
  return ndone;
}

// Pulay.f90 DoPulay2D_nospin: alphas from the inverse of the <=5x5 residual overlap.
void LNVSolver::do_pulay(int iPulay, const double* Aij /* col-major max_n x max_n */, int n, int max_n, double* al) {
  std::vector<double> A(n * n);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) A[i + n * j] = Aij[i + max_n * j];
  bool invertible = true;
  if (n == 1) A[0] = 1.0 / A[0];
  else invertible = sym_inverse_bk(A.data(), n);
  for (int i = 0; i < max_n; ++i) al[i] = 0.0;
  if (invertible) {
    double s = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) { al[i] += A[j + n * i]; s += A[j + n * i]; }
    for (int i = 0; i < n; ++i) al[i] /= s;
  } else {
    al[iPulay - 1] = 1.0;
  }
}

int LNVSolver::late_dm(int ndone, bool& done, double& deltaE) {
  const int npul = prm.maxpulay;
  std::vector<DMat> Lst, Gst, SGst;
  for (int i = 0; i < npul; ++i) { Lst.push_back(temp(RL)); Gst.push_back(temp(RL)); SGst.push_back(temp(RL)); }
  DMat M3 = temp(RL), SM3 = temp(RL), Sphi = temp(RL), mtemp = temp(RTL);
  int iter_stuck = 0;
  double el, e0;
  if (h_rebuild) rebuild_H();
  lnv(false, true, true, true, &M3, &phi, &el, &e0);
  double energy0 = 2.0 * e0;
  tmt(M3, SM3, mtemp, T);
  if (prm.vary_mu) {
    tmt(phi, Sphi, mtemp, T);
    double d[2];
    ptraces({{&SM3, &phi}, {&Sphi, &phi}}, d);
    const double e_dot_n = d[0], n_dot_n = d[1];
    if (std::fabs(n_dot_n) > 1.0e-8) {
      double f = e_dot_n / n_dot_n;
      msum(1.0, SM3, -f, Sphi);
      msum(1.0, M3, -f, phi);
    }
  }
  msum(0.0, SGst[0], -1.0, SM3);
  msum(0.0, Gst[0], -1.0, M3);
  msum(0.0, Lst[0], 1.0, L);
  double g0 = gnorm(M3, SM3);
  if (prm.n_L_iterations == 0) done = true;
  std::vector<double> Aij(npul * npul), alph(npul);
  for (int n_iter = 1; n_iter <= prm.n_L_iterations; ++n_iter) {
    int npmod = (n_iter % npul) + 1;
    int pul_mx = std::min(n_iter + 1, npul);
    double step = prm.global_tolerance ? deltaE / (g0 + 1.0e-8) : deltaE / ((double)ni_in_cell * g0 + 1.0e-8);
    step = std::fabs(step);
    if (std::fabs(step) < prm.minpulaystep) step = prm.minpulaystep;
    if (std::fabs(step) > prm.maxpulaystep) step = prm.maxpulaystep;
    int src = npmod > 1 ? npmod - 1 : pul_mx;
    msum(0.0, L, 1.0, Lst[src - 1]);
    msum(1.0, L, step, SGst[src - 1]);
    if (prm.vary_mu) correct_electron_number();
    double e1;
    lnv(false, true, true, true, &M3, &phi, &el, &e1);
    tmt(M3, SM3, mtemp, T);
    if (prm.vary_mu) project_gradient(M3, SM3, Sphi, mtemp);
    msum(0.0, SGst[npmod - 1], -1.0, SM3);
    msum(0.0, Gst[npmod - 1], -1.0, M3);
    msum(0.0, Lst[npmod - 1], 1.0, L);
    std::fill(Aij.begin(), Aij.end(), 0.0);
    {
      // the pul_mx^2 traces Tr(G_j SG_i), in the reference's loop order, read with one wait
      const int nt = pul_mx * pul_mx;
      std::vector<const double*> xs(nt), ys(nt);
      std::vector<int64_t> ns(nt);
      std::vector<double> v(nt);
      int k = 0;
      for (int i = 0; i < pul_mx; ++i)
        for (int j = 0; j < pul_mx; ++j) { xs[k] = Gst[j].p; ys[k] = SGst[i].p; ns[k] = Gst[j].n; ++k; }
      stats.n_reductions += k;
      for (int k0 = 0; k0 < nt; k0 += 32)     // dev_dots reads at most 32 sums per wait
        dev_dots(S, std::min(32, nt - k0), xs.data() + k0, ys.data() + k0, ns.data() + k0, v.data() + k0);
      if (rlog_on) rlog.insert(rlog.end(), v.begin(), v.end());
      k = 0;
      for (int i = 0; i < pul_mx; ++i)
        for (int j = 0; j < pul_mx; ++j) Aij[j + npul * i] = 2.0 * v[k++];
    }
    do_pulay(npmod, Aij.data(), pul_mx, npul, alph.data());
    scale(0.0, L);
    for (int i = 0; i < pul_mx; ++i) msum(1.0, L, alph[i], Lst[i]);
    if (prm.vary_mu) correct_electron_number();
    if (h_rebuild) rebuild_H();
    lnv(false, true, true, true, &M3, &phi, &el, &e1);
    double energy1 = 2.0 * e1;
    tmt(M3, SM3, mtemp, T);
    if (prm.vary_mu) project_gradient(M3, SM3, Sphi, mtemp);
    deltaE = energy1 - energy0;
    double g1 = gnorm(M3, SM3);
    CQ_CHECK(std::isfinite(g1) && std::isfinite(energy1), CQ_ERR_NOT_CONVERGED,
             "lateDM: the residual or the energy is not finite");
    stats.late_iters++;
    stats.last_energy = energy1;
    stats.last_residual = g1;
    log_iteration(g1, energy1);
    if (g1 < prm.tolerance) { done = true; return n_iter; }
    else if (!h_rebuild && g1 > 2.0 * g0) return n_iter;   // no residual-rise exit with the H coupling
    else if (g1 > 0.99 * g0) {
      if (++iter_stuck > 5) return n_iter;
    }
    msum(0.0, SGst[npmod - 1], -1.0, SM3);
    msum(0.0, Gst[npmod - 1], -1.0, M3);
    msum(0.0, Lst[npmod - 1], 1.0, L);
    g0 = g1;
    energy0 = energy1;
  }
  return ndone;
}

// Mixed-L self-consistency step of lateDM (DMMinModule.f90:894-907, 1138-1149): K and Tr(KH) of
// the current L, then the caller rebuilds H from the density of K (get_electronic_density and
// get_H_matrix in the reference).  H keeps its address, so captured LNV graphs stay valid.
void LNVSolver::rebuild_H() {
  double el = 0.0, e = 0.0;
  lnv(true, false, false, true, nullptr, nullptr, &el, &e);
  const int rc = h_rebuild(h_rebuild_user, K.p, Hmat.p, Hmat.n, (void*)S.stream);
  CQ_CHECK(rc == 0, CQ_ERR_CALLBACK, "the H rebuild callback returned " + std::to_string(rc));
}

void LNVSolver::find_min_dm(bool resetL) {
  bool problem = false, inflex = false, done = false, early = true;
  transpose(T, Ttran);
  int ndone = 0, niter = 0, outer = 0;
  while (!done) {
    // the reference loops until done; a problem whose residual stalls above the tolerance stops
    // here after max_outer passes, reported as not converged
    if (++outer > prm.max_outer) break;
    stats.outer_iters++;
    if (resetL || inflex) {
      // the McWeeny start runs in FP64 unless mixed_mcw: split-precision noise in its stopping
      // test (energy rise, |dE| < 1e-8) changes the start, and a truncated functional can then
      // descend into another minimum than the FP64 solve
      const bool um = use_mixed;
      if (!prm.mixed_mcw) use_mixed = false;
      init_mcw();
      delta_e = mcw_min(prm.n_L_iterations);
      use_mixed = um;
      early = true;
      resetL = false;
    }
    if (early || problem) {
      inflex = false;
      ndone = early_dm(ndone, inflex);
    }
    if (!done && !inflex) ndone = late_dm(ndone, done, delta_e);
    niter++;
    if (problem) resetL = true;
    if (niter > 10) { problem = true; niter = 0; }
  }
  double el = 0, en = 0;
  lnv(true, false, true, true, nullptr, &phi, &el, &en);
  stats.energy = 2.0 * en;
  stats.electrons = 2.0 * el;
  stats.converged = done ? 1 : 0;
}

// ---------------------------------------------------------------------------
// symmetric indefinite inverse for the Pulay system: Bunch-Kaufman diagonal
// pivoting (alpha = (1 + sqrt 17)/8, upper triangle, as LAPACK dsytf2) followed
// by the inverse of the block-diagonal factor and back substitution (dsytri).
// Returns false when a pivot block is singular.  A is n x n column major.
// ---------------------------------------------------------------------------
bool sym_inverse_bk(double* A, int n) {
  const double alpha = (1.0 + std::sqrt(17.0)) / 8.0;
  auto a = [&](int i, int j) -> double& { return A[i + n * j]; };
  std::vector<int> ipiv(n, 0);
  // ---- factorisation U D U^T, processing columns from the last one upwards
  int k = n - 1;
  while (k >= 0) {
    int kstep = 1;
    double absakk = std::fabs(a(k, k));
    int imax = 0;
    double colmax = 0.0;
    for (int i = 0; i < k; ++i) if (std::fabs(a(i, k)) > colmax) { colmax = std::fabs(a(i, k)); imax = i; }
    int kp;
    // a zero or NaN pivot column: singular (dsytf2 sets INFO and leaves the column)
    if (std::max(absakk, colmax) == 0.0 || std::isnan(absakk)) return false;
    if (absakk >= alpha * colmax) kp = k;
    else {
      double rowmax = 0.0;
      for (int j = imax + 1; j <= k; ++j) rowmax = std::max(rowmax, std::fabs(a(imax, j)));
      for (int j = 0; j < imax; ++j) rowmax = std::max(rowmax, std::fabs(a(j, imax)));
      if (absakk >= alpha * colmax * (colmax / rowmax)) kp = k;
      else if (std::fabs(a(imax, imax)) >= alpha * rowmax) kp = imax;
      else { kp = imax; kstep = 2; }
    }
    int kk = k - kstep + 1;
    if (kp != kk) {
      for (int i = 0; i < kp; ++i) std::swap(a(i, kk), a(i, kp));
      for (int j = kp + 1; j < kk; ++j) std::swap(a(j, kk), a(kp, j));
      std::swap(a(kk, kk), a(kp, kp));
      if (kstep == 2) std::swap(a(k - 1, k), a(kp, k));
    }
    if (kstep == 1) {
      double r1 = 1.0 / a(k, k);
      for (int j = k - 1; j >= 0; --j) {
        double f = -r1 * a(j, k);
        for (int i = 0; i <= j; ++i) a(i, j) += a(i, k) * f;
      }
      for (int i = 0; i < k; ++i) a(i, k) *= r1;
    } else if (k > 1) {
      double d12 = a(k - 1, k);
      double d22 = a(k - 1, k - 1) / d12;
      double d11 = a(k, k) / d12;
      double t = 1.0 / (d11 * d22 - 1.0);
      d12 = t / d12;
      for (int j = k - 2; j >= 0; --j) {
        double wkm1 = d12 * (d11 * a(j, k - 1) - a(j, k));
        double wk = d12 * (d22 * a(j, k) - a(j, k - 1));
        for (int i = j; i >= 0; --i) a(i, j) = a(i, j) - a(i, k) * wk - a(i, k - 1) * wkm1;
        a(j, k) = wk;
        a(j, k - 1) = wkm1;
      }
    }
    if (kstep == 1) ipiv[k] = kp + 1;
    else { ipiv[k] = -(kp + 1); ipiv[k - 1] = -(kp + 1); }
    k -= kstep;
  }
  // ---- inverse (dsytri, upper)
  for (int i = n - 1; i >= 0; --i)
    if (ipiv[i] > 0 && a(i, i) == 0.0) return false;
  std::vector<double> work(n), y(n);
  auto dot = [&](int m, const double* x, const double* z) { double s = 0.0; for (int i = 0; i < m; ++i) s += x[i] * z[i]; return s; };
  // column kc of the leading k x k block: work = old column, column = -A11 work; returns work . column
  auto inv_col = [&](int kc, int m) {
    for (int i = 0; i < m; ++i) work[i] = a(i, kc);
    for (int i = 0; i < m; ++i) {
      double s = 0.0;
      for (int j = 0; j < m; ++j) s += (i <= j ? a(i, j) : a(j, i)) * work[j];
      y[i] = s;
    }
    for (int i = 0; i < m; ++i) a(i, kc) = -y[i];
    return dot(m, work.data(), &A[(size_t)n * kc]);
  };
  k = 0;
  while (k < n) {
    int kstep;
    if (ipiv[k] > 0) {
      a(k, k) = 1.0 / a(k, k);
      if (k > 0) a(k, k) -= inv_col(k, k);
      kstep = 1;
    } else {
      double t = std::fabs(a(k, k + 1));
      double ak = a(k, k) / t;
      double akp1 = a(k + 1, k + 1) / t;
      double akkp1 = a(k, k + 1) / t;
      double d = t * (ak * akp1 - 1.0);
      a(k, k) = akp1 / d;
      a(k + 1, k + 1) = ak / d;
      a(k, k + 1) = -akkp1 / d;
      if (k > 0) {
        a(k, k) -= inv_col(k, k);
        a(k, k + 1) -= dot(k, &A[(size_t)n * k], &A[(size_t)n * (k + 1)]);
        a(k + 1, k + 1) -= inv_col(k + 1, k);
      }
      kstep = 2;
    }
    int kp = std::abs(ipiv[k]) - 1;
    if (kp != k) {
      for (int i = 0; i < kp; ++i) std::swap(a(i, k), a(i, kp));
      for (int j = kp + 1; j < k; ++j) std::swap(a(j, k), a(kp, j));
      std::swap(a(k, k), a(kp, kp));
      if (kstep == 2) std::swap(a(k, k + 1), a(kp, k + 1));
    }
    k += kstep;
  }
  // complete the lower triangle
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) a(j, i) = a(i, j);
  return true;
}

}  // namespace cqb
