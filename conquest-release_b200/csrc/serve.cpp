// Serving loop for independent density-matrix solves (declarations in include/cq_b200.h).
//
// Continuous batching: n_slots worker threads, each with its own CUDA stream, take requests
// from one arrival-ordered queue as soon as a slot is free and the request's memory estimate
// fits into the HBM budget left by the requests already admitted.  A request keeps all of its
// state (geometry, indices, pair lists, S, H, L and the chain's temporaries) on the device from
// admission to result, and the kernels of different slots overlap on the GPU.  Nothing is shared
// between slots but the device's memory pool, so a solve gives the same bits alone and in a mix.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <mutex>
#include <thread>

#include "chain.hpp"

namespace cqb {

int guarded_call(const std::function<void()>& f);

namespace {

// Gathers the FP64 products of the slots' solves and runs each gathering as one persistent launch
// over the concatenated output-block lists (launch_mat_mult_batch) on the batcher's own stream.  A
// product's system stream records an event the launch waits for, and waits for the launch's completion
// event itself, so stream order is kept without host synchronisation.  A gathering is launched as soon
// as every solving slot has a product waiting, or when the oldest waiting product has waited the
// window; each product is computed exactly as alone, so the results do not change.
class ProductBatcher {
 public:
  ProductBatcher(int device, double window_us) : window_(window_us > 0 ? window_us : 50.0) {
    CQ_CUDA(cudaSetDevice(device));
    CQ_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
  }
  ~ProductBatcher() {
    if (st_) { cudaStreamSynchronize(st_); cudaStreamDestroy(st_); }
  }
  void enter() { std::lock_guard<std::mutex> lk(mu_); ++active_; }
  void leave() {
    std::lock_guard<std::mutex> lk(mu_);
    --active_;
    if (!pending_.empty() && (int)pending_.size() >= active_) flush_locked();
  }

  void submit(System& S, ProductPlan& P, double* a, const double* b, double* c, int exact) {
    ensure_product_order(S, P);
    cudaEvent_t ready;
    CQ_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    CQ_CUDA(cudaEventRecord(ready, S.stream));
    auto ticket = std::make_shared<Ticket>();
    std::unique_lock<std::mutex> lk(mu_);
    pending_.push_back({BatchItem{&S, &P, a, b, c, exact}, ready, ticket});
    const uint64_t gen = gen_;
    if ((int)pending_.size() >= active_) {
      flush_locked();
    } else {
      cv_.wait_for(lk, std::chrono::duration<double, std::micro>(window_), [&] { return gen_ != gen; });
      if (gen_ == gen) flush_locked();
    }
    lk.unlock();
    if (!ticket->error.empty()) throw Error(ticket->code, ticket->error);
    CQ_CUDA(cudaStreamWaitEvent(S.stream, ticket->done->e, 0));
  }

 private:
  struct Event {
    cudaEvent_t e = nullptr;
    ~Event() { if (e) cudaEventDestroy(e); }
  };
  struct Ticket {
    std::shared_ptr<Event> done;
    std::string error;
    int code = 0;
  };
  struct Pending {
    BatchItem item;
    cudaEvent_t ready;
    std::shared_ptr<Ticket> ticket;
  };
  void flush_locked() {
    std::vector<BatchItem> items;
    auto done = std::make_shared<Event>();
    try {
      for (auto& p : pending_) {
        CQ_CUDA(cudaStreamWaitEvent(st_, p.ready, 0));
        items.push_back(p.item);
      }
      launch_mat_mult_batch(items, st_);
      CQ_CUDA(cudaEventCreateWithFlags(&done->e, cudaEventDisableTiming));
      CQ_CUDA(cudaEventRecord(done->e, st_));
      for (auto& p : pending_) p.ticket->done = done;
    } catch (const Error& e) {
      for (auto& p : pending_) { p.ticket->error = e.what(); p.ticket->code = e.code; }
    }
    for (auto& p : pending_) cudaEventDestroy(p.ready);
    pending_.clear();
    ++gen_;
    cv_.notify_all();
  }
  double window_;
  cudaStream_t st_ = nullptr;
  std::mutex mu_;
  std::condition_variable cv_;
  std::vector<Pending> pending_;
  int active_ = 0;
  uint64_t gen_ = 0;
};

struct Request {
  int64_t id = 0;
  int n = 0;
  std::vector<double> coords, cell;
  std::vector<int> nsf;
  double rcut[LNVSolver::NR];
  double ne_spin = 0;
  uint64_t seed = 0;
  int mixed = 0;
  double t_arrival = 0;
  int64_t est = 0;
  int bypassed = 0;
};

// The chain's ranges from the S, H, L and T ranges (dimens_module.f90:302-355), in the order of
// LNVSolver::Rng.
void chain_ranges(double rs, double rh, double rl, double rt, double* r) {
  r[LNVSolver::RS] = rs; r[LNVSolver::RH] = rh; r[LNVSolver::RL] = rl; r[LNVSolver::RT] = rt;
  r[LNVSolver::RLS] = rl + rs; r[LNVSolver::RLH] = rl + rh; r[LNVSolver::RLSL] = 2 * rl + rs;
  r[LNVSolver::RSLS] = 2 * rs + rl; r[LNVSolver::RTS] = rt + rs; r[LNVSolver::RTH] = rt + rh;
  r[LNVSolver::RTL] = rt + rl;
}

// Memory estimate of one solve.  Neighbour counts and block sizes per range come from up to 24
// atoms sampled at a fixed stride (every periodic image within the largest range counted with
// the strict test of get_naba); the device footprint is then
//   matrices:   range length x 8 bytes x the number of live matrices of that range in the chain
//               (owned matrices, the LNV temporaries, the Pulay history),
//   indices:    64 bytes per stored block,
//   pair lists: 8 bytes per (i,k,j) triple of each product of the chain, twice for the
//               split-precision lists, plus 2 KiB per block for the bf16 fragments,
// times 1.25, plus 64 MiB.
int64_t estimate_bytes(int n, const double* x, const double* cell, const int* nsf, const double* rc, int mixed) {
  if (n <= 0) return 0;
  double rmax = 0;
  for (int r = 0; r < LNVSolver::NR; ++r) rmax = std::max(rmax, rc[r]);
  const int ns = std::min(n, 24);
  int img[3];
  for (int d = 0; d < 3; ++d) img[d] = cell[d] > 0 ? (int)std::ceil(rmax / cell[d]) : 0;
  double cnt[LNVSolver::NR] = {0}, elem[LNVSolver::NR] = {0};
  for (int q = 0; q < ns; ++q) {
    const int i = (int)((int64_t)q * n / ns);
    for (int j = 0; j < n; ++j)
      for (int a = -img[0]; a <= img[0]; ++a)
        for (int b = -img[1]; b <= img[1]; ++b)
          for (int c = -img[2]; c <= img[2]; ++c) {
            const double dx = x[3 * j] + a * cell[0] - x[3 * i], dy = x[3 * j + 1] + b * cell[1] - x[3 * i + 1],
                         dz = x[3 * j + 2] + c * cell[2] - x[3 * i + 2];
            const double d2 = dx * dx + dy * dy + dz * dz;
            if (d2 >= rmax * rmax) continue;
            for (int r = 0; r < LNVSolver::NR; ++r)
              if (d2 < rc[r] * rc[r] - 1e-8) { cnt[r] += 1; elem[r] += (double)nsf[i] * nsf[j]; }
          }
  }
  double nb[LNVSolver::NR], len[LNVSolver::NR];
  for (int r = 0; r < LNVSolver::NR; ++r) {
    nb[r] = cnt[r] / ns;               // neighbours per atom
    len[r] = elem[r] / ns * n;         // stored elements
  }
  // live matrices per range: owned (S, H+K, L+phi, T+Ttran, LS+SL) plus the pool's high-water
  static const int kLive[LNVSolver::NR] = {/*S*/ 1, /*H*/ 3, /*L*/ 24, /*T*/ 5, /*LS*/ 4, /*LH*/ 2,
                                           /*LSL*/ 4, /*SLS*/ 1, /*TS*/ 3, /*TH*/ 2, /*TL*/ 2};
  double bytes = 0;
  for (int r = 0; r < LNVSolver::NR; ++r) bytes += 8.0 * len[r] * kLive[r] + 64.0 * n * nb[r];
  for (int m = 0; m <= LNVSolver::TL_T_L; ++m) {
    const LNVSolver::Mult& M = LNVSolver::kMults[m];
    const double triples = (double)n * nb[M.a] * nb[M.b];
    bytes += 8.0 * triples * (mixed ? 2.0 : 1.0);
  }
  if (mixed)
    for (int r = 0; r < LNVSolver::NR; ++r) bytes += 2.0 * 1024.0 * n * nb[r];
  return (int64_t)(1.25 * bytes) + (64ll << 20);
}

}  // namespace

class Server {
 public:
  explicit Server(const cq_server_config& c) : cfg_(c), t0_(std::chrono::steady_clock::now()) {
    CQ_CHECK(c.n_slots >= 1 && c.n_slots <= 64, CQ_ERR_ARG, "n_slots must be 1..64");
    CQ_CHECK(c.hbm_budget > 0, CQ_ERR_ARG, "hbm_budget must be positive");
    if (!c.dry_run) {
      CQ_CUDA(cudaGetDevice(&device_));
      init_device_pool();
      if (c.batch_products) batcher_ = std::make_unique<ProductBatcher>(device_, c.batch_window_us);
    }
    for (int s = 0; s < c.n_slots; ++s) workers_.emplace_back([this, s] { worker(s); });
  }
  ~Server() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_work_.notify_all();
    for (auto& t : workers_) t.join();
  }
  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
  }
  int64_t submit(const cq_request& r) {
    CQ_CHECK(r.n_atoms > 0 && r.coords && r.cell && r.nsf, CQ_ERR_ARG, "bad request");
    CQ_CHECK(r.ne_spin > 0 && r.rs > 0 && r.rh > 0 && r.rl > 0 && r.rt > 0, CQ_ERR_ARG, "bad request ranges");
    for (int i = 0; i < r.n_atoms; ++i) CQ_CHECK(r.nsf[i] >= 1 && r.nsf[i] <= 16, CQ_ERR_ARG, "block sizes must be 1..16");
    auto q = std::make_unique<Request>();
    q->n = r.n_atoms;
    q->coords.assign(r.coords, r.coords + 3 * (size_t)r.n_atoms);
    q->cell.assign(r.cell, r.cell + 3);
    q->nsf.assign(r.nsf, r.nsf + r.n_atoms);
    chain_ranges(r.rs, r.rh, r.rl, r.rt, q->rcut);
    q->ne_spin = r.ne_spin;
    q->seed = r.seed;
    q->mixed = r.mixed;
    q->t_arrival = r.t_arrival >= 0 ? r.t_arrival : now();
    q->est = estimate_bytes(q->n, q->coords.data(), q->cell.data(), q->nsf.data(), q->rcut, q->mixed);
    std::lock_guard<std::mutex> lk(mu_);
    CQ_CHECK(!stop_, CQ_ERR_STATE, "server is stopping");
    q->id = next_id_++;
    int64_t id = q->id;
    queue_.push_back(std::move(q));
    cv_work_.notify_all();
    return id;
  }
  bool wait(int64_t id, double timeout_s, cq_request_result* out) {
    std::unique_lock<std::mutex> lk(mu_);
    auto ready = [&] { return done_.count(id) != 0; };
    if (timeout_s < 0) cv_done_.wait(lk, ready);
    else if (!cv_done_.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) return false;
    *out = done_[id];
    done_.erase(id);
    return true;
  }

 private:
  // First queued request that fits; a request overtaken max_bypass times blocks the rest.
  std::unique_ptr<Request> take_admissible() {
    for (size_t k = 0; k < queue_.size(); ++k) {
      Request& q = *queue_[k];
      const bool fits = in_use_ + q.est <= cfg_.hbm_budget || running_ == 0;
      if (fits) {
        for (size_t m = 0; m < k; ++m) queue_[m]->bypassed++;
        std::unique_ptr<Request> r = std::move(queue_[k]);
        queue_.erase(queue_.begin() + k);
        return r;
      }
      if (q.bypassed >= cfg_.max_bypass) break;
    }
    return nullptr;
  }

  void worker(int slot) {
    cudaStream_t st = nullptr;
    cudaError_t setup = cudaSuccess;
    if (!cfg_.dry_run) {
      setup = cudaSetDevice(device_);
      if (setup == cudaSuccess) setup = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    }
    for (;;) {
      std::unique_ptr<Request> q;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_work_.wait(lk, [&] {
          if (stop_ && queue_.empty()) return true;
          q = take_admissible();
          return q != nullptr;
        });
        if (!q) break;
        in_use_ += q->est;
        running_++;
      }
      cq_request_result res;
      std::memset(&res, 0, sizeof(res));
      res.id = q->id;
      res.n_atoms = q->n;
      res.mixed = q->mixed;
      res.slot = slot;
      res.t_arrival = q->t_arrival;
      res.t_admit = now();
      res.bytes_estimate = q->est;
      if (cfg_.dry_run) {
        std::this_thread::sleep_for(std::chrono::duration<double>(cfg_.dry_run_seconds));
        res.status = CQ_OK;
      } else if (setup != cudaSuccess) {
        // this slot has no device stream: its requests fail with the CUDA error
        res.status = CQ_ERR_CUDA;
        std::snprintf(res.message, sizeof(res.message), "slot set-up failed: %s", cudaGetErrorString(setup));
      } else {
        solve(*q, st, res);
      }
      res.t_done = now();
      {
        std::lock_guard<std::mutex> lk(mu_);
        in_use_ -= q->est;
        running_--;
        done_[res.id] = res;
      }
      cv_done_.notify_all();
      cv_work_.notify_all();
    }
    if (st) cudaStreamDestroy(st);
  }

  void solve(const Request& q, cudaStream_t st, cq_request_result& res) {
    DevAccount& acct = dev_account();
    const int64_t base = acct.live;
    acct.peak = acct.live;
    res.status = guarded_call([&] {
      System S;
      S.stream = st;
      S.blocking_sync = cfg_.blocking_sync != 0;
      double rmax = 0;
      for (int r = 0; r < LNVSolver::NR; ++r) rmax = std::max(rmax, q.rcut[r]);
      build_geometry(S.geo, q.n, q.coords.data(), q.cell.data(), q.nsf.data(), rmax, GeometryParams());
      upload_geometry(S);
      for (int r = 0; r < LNVSolver::NR; ++r) {
        S.ranges.emplace_back(new RangeIndex());
        S.ranges.back()->rcut = q.rcut[r];
        build_range_index(S, *S.ranges.back());
      }
      int idx[LNVSolver::NR];
      for (int r = 0; r < LNVSolver::NR; ++r) idx[r] = r;
      cq_lnv_params prm = cfg_.lnv;
      prm.mixed = q.mixed;
      if (batcher_) {
        prm.graphs = 0;             // products leave the system's stream: no graph capture
        S.batch_submit = [this, &S](ProductPlan& P, double* a, const double* b, double* c, int exact) {
          batcher_->submit(S, P, a, b, c, exact);
        };
      }
      LNVSolver L(S, idx, q.ne_spin, prm);
      generate_SH(S, LNVSolver::RS, 0, q.seed, L.Smat.p);
      generate_SH(S, LNVSolver::RH, 1, q.seed, L.Hmat.p);
      struct Active {              // this slot counts as solving while its chain runs
        ProductBatcher* b;
        explicit Active(ProductBatcher* x) : b(x) { if (b) b->enter(); }
        ~Active() { if (b) b->leave(); }
      } active(batcher_.get());
      L.solve();
      host_wait(S);
      const LNVStats& s = L.stats;
      res.energy = s.energy;
      res.electrons = s.electrons;
      res.residual = s.last_residual;
      res.converged = s.converged;
      res.n_products = s.n_products;
      res.flops = s.flops;
      res.n_products_mixed = s.n_products_mixed;
      res.flops_mixed = s.flops_mixed;
      res.split_restarts = s.split_restarts;
    });
    if (res.status != CQ_OK) {
      std::strncpy(res.message, cq_last_error(), sizeof(res.message) - 1);
      cudaStreamSynchronize(st);
    }
    res.bytes_peak = acct.peak - base;
  }

  cq_server_config cfg_;
  std::chrono::steady_clock::time_point t0_;
  int device_ = 0;
  std::mutex mu_;
  std::condition_variable cv_work_, cv_done_;
  std::deque<std::unique_ptr<Request>> queue_;
  std::map<int64_t, cq_request_result> done_;
  int64_t in_use_ = 0, next_id_ = 1;
  int running_ = 0;
  bool stop_ = false;
  std::vector<std::thread> workers_;
  std::unique_ptr<ProductBatcher> batcher_;   // declared last: destroyed after the workers are joined
};

}  // namespace cqb

using namespace cqb;

struct cq_server {
  std::unique_ptr<Server> srv;
};

extern "C" {

int cq_server_config_default(cq_server_config* c) {
  if (!c) return CQ_ERR_ARG;
  std::memset(c, 0, sizeof(*c));
  c->n_slots = 8;
  c->hbm_budget = 64ll << 30;
  c->max_bypass = 4;
  c->blocking_sync = 1;
  c->dry_run = 0;
  c->dry_run_seconds = 0.01;
  cq_lnv_params_default(&c->lnv);
  c->batch_products = 0;
  c->batch_window_us = 50.0;
  return CQ_OK;
}

int cq_server_create(const cq_server_config* c, cq_server** out) {
  return guarded_call([&] {
    CQ_CHECK(c && out, CQ_ERR_ARG, "null argument");
    *out = nullptr;
    auto s = std::make_unique<cq_server>();
    s->srv = std::make_unique<Server>(*c);
    *out = s.release();
  });
}

int cq_server_submit(cq_server* s, const cq_request* r, int64_t* id) {
  return guarded_call([&] {
    CQ_CHECK(s && r && id, CQ_ERR_ARG, "null argument");
    *id = s->srv->submit(*r);
  });
}

int cq_server_wait(cq_server* s, int64_t id, double timeout_s, cq_request_result* out) {
  return guarded_call([&] {
    CQ_CHECK(s && out, CQ_ERR_ARG, "null argument");
    CQ_CHECK(s->srv->wait(id, timeout_s, out), CQ_ERR_TIMEOUT, "request not finished");
  });
}

int cq_server_now(cq_server* s, double* t) {
  return guarded_call([&] {
    CQ_CHECK(s && t, CQ_ERR_ARG, "null argument");
    *t = s->srv->now();
  });
}

int cq_request_estimate(const cq_request* r, int64_t* bytes) {
  return guarded_call([&] {
    CQ_CHECK(r && bytes && r->n_atoms > 0 && r->coords && r->cell && r->nsf, CQ_ERR_ARG, "bad request");
    double rc[LNVSolver::NR];
    chain_ranges(r->rs, r->rh, r->rl, r->rt, rc);
    *bytes = estimate_bytes(r->n_atoms, r->coords, r->cell, r->nsf, rc, r->mixed);
  });
}

int cq_server_destroy(cq_server* s) {
  return guarded_call([&] { delete s; });
}

}  // extern "C"
