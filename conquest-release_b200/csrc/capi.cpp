// C ABI of libcqb200.so (declarations and reference citations in include/cq_b200.h).
#include <algorithm>
#include <cstring>
#include <functional>
#include <mutex>
#include <numeric>
#include <string>

#include "cq_internal.hpp"

namespace cqb {

static thread_local std::string g_last_error = "";
void set_last_error(const std::string& m) { g_last_error = m; }

static thread_local DevAccount t_account;
DevAccount& dev_account() { return t_account; }
void dev_account_add(int64_t bytes) {
  t_account.live += bytes;
  if (t_account.live > t_account.peak) t_account.peak = t_account.live;
}

// Keep freed blocks of the device's default pool cached in the process (release threshold =
// unlimited) so stream-ordered reallocation does not go back to the driver at every
// synchronisation.  A property of this process's pool only; it ends with the process.
void init_device_pool() {
  int dev = 0;
  CQ_CUDA(cudaGetDevice(&dev));
  static std::mutex mu;
  static std::vector<int> done;
  std::lock_guard<std::mutex> lk(mu);
  if (std::find(done.begin(), done.end(), dev) != done.end()) return;
  cudaMemPool_t pool;
  CQ_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
  uint64_t thr = UINT64_MAX;
  CQ_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
  done.push_back(dev);
}

System::~System() {
  // buffers may have been used on a stream given with cq_system_set_stream: finish that work
  // before they are released (on the stream recorded at their allocation)
  if (stream) cudaStreamSynchronize(stream);
  if (sync_ev) cudaEventDestroy(sync_ev);
  if (host_res) pinned_put(host_res);
  if (umma_err_host) cudaFreeHost(umma_err_host);
}

// Small pinned host buffers (exact-sum results) are kept in a process-wide free list: freeing
// pinned memory can synchronise the device, which would stall the solves of other systems.
static std::mutex g_pinned_mu;
static std::vector<uint64_t*> g_pinned_free;
uint64_t* pinned_get() {
  {
    std::lock_guard<std::mutex> lk(g_pinned_mu);
    if (!g_pinned_free.empty()) { uint64_t* p = g_pinned_free.back(); g_pinned_free.pop_back(); return p; }
  }
  uint64_t* p = nullptr;
  CQ_CUDA(cudaMallocHost((void**)&p, kPinnedWords * sizeof(uint64_t)));
  return p;
}
void pinned_put(uint64_t* p) {
  std::lock_guard<std::mutex> lk(g_pinned_mu);
  g_pinned_free.push_back(p);
}

void host_wait(System& S) {
  if (!S.blocking_sync) {
    CQ_CUDA(cudaStreamSynchronize(S.stream));
  } else {
    if (!S.sync_ev) CQ_CUDA(cudaEventCreateWithFlags(&S.sync_ev, cudaEventBlockingSync | cudaEventDisableTiming));
    CQ_CUDA(cudaEventRecord(S.sync_ev, S.stream));
    CQ_CUDA(cudaEventSynchronize(S.sync_ev));
  }
  umma_check(S);
}

// drop-in kernels (one m_kern_max / m_kern_min call): explicit offsets prepared on the host
void launch_dropin(int type, const int64_t* d_out, const int* d_dims, const int64_t* d_ptr, const int64_t* d_pairs,
                   int n_out, const double* x, const double* b, double* out, cudaStream_t st);

}  // namespace cqb

using namespace cqb;

// A matrix bound to an id (cq_matrix_bind): the system-owned device copy in the layout of its
// range, and the caller's host array it is copied from and to on demand.
struct BoundMatrix {
  int r = -1;
  double* host = nullptr;
  DevBuf<double> dev;
};

struct cq_system {
  cqb::System S;
  // staging buffers of the host-memory entry points
  DevBuf<double> ha, hb, hc;
  // matrices by id; destroyed before S, whose stream their memory is released on
  std::map<int, std::unique_ptr<BoundMatrix>> store;
};

template <class F>
static int guarded(F&& f) {
  try {
    f();
    return CQ_OK;
  } catch (const cqb::Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return CQ_ERR_OOM;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return CQ_ERR_STATE;
  }
}

namespace cqb {
System& system_of(cq_system* s) {
  CQ_CHECK(s != nullptr, CQ_ERR_ARG, "null system");
  return s->S;
}
int guarded_call(const std::function<void()>& f) { return guarded(f); }
}  // namespace cqb

static void check_sys(cq_system* s) { CQ_CHECK(s != nullptr, CQ_ERR_ARG, "null system"); }
static void check_range(cq_system* s, int r) {
  CQ_CHECK(r >= 0 && r < (int)s->S.ranges.size(), CQ_ERR_ARG, "range index out of bounds");
}

extern "C" {

const char* cq_last_error(void) { return g_last_error.c_str(); }
const char* cq_version(void) { return "cqb200 0.1 (sm_100a)"; }

int cq_system_create(int n_atoms, const double* coords, const double* cell, const int* nsf, int n_ranges,
                     const double* rcuts, int max_atoms_part, double gap_threshold, double avg_atomic_diameter,
                     cq_system** out) {
  return guarded([&] {
    CQ_CHECK(out && coords && cell && nsf && rcuts && n_ranges > 0, CQ_ERR_ARG, "null argument");
    *out = nullptr;
    for (int r = 0; r < n_ranges; ++r) CQ_CHECK(rcuts[r] > 0, CQ_ERR_ARG, "ranges must be positive");
    for (int i = 0; i < n_atoms; ++i) CQ_CHECK(nsf[i] >= 1 && nsf[i] <= 16, CQ_ERR_ARG, "block sizes must be 1..16");
    auto sys = std::make_unique<cq_system>();
    System& S = sys->S;
    init_device_pool();
    CQ_CUDA(cudaStreamCreateWithFlags(&S.own.s, cudaStreamNonBlocking));
    S.stream = S.own.s;
    GeometryParams prm;
    prm.max_atoms_part = max_atoms_part > 0 ? max_atoms_part : 34;
    prm.gap_threshold = gap_threshold;
    prm.avg_atomic_diameter = avg_atomic_diameter > 0 ? avg_atomic_diameter : 5.0;
    double rmax = *std::max_element(rcuts, rcuts + n_ranges);
    build_geometry(S.geo, n_atoms, coords, cell, nsf, rmax, prm);
    upload_geometry(S);
    for (int r = 0; r < n_ranges; ++r) {
      S.ranges.emplace_back(new RangeIndex());
      S.ranges.back()->rcut = rcuts[r];
      build_range_index(S, *S.ranges.back());
    }
    CQ_CUDA(cudaStreamSynchronize(S.stream));
    *out = sys.release();
  });
}

int cq_system_destroy(cq_system* sys) {
  return guarded([&] {
    if (sys) {
      CQ_CHECK(sys->S.n_solvers == 0, CQ_ERR_STATE,
               "the system still has LNV solvers: destroy them (cq_lnv_destroy) before the system");
      cudaStreamSynchronize(sys->S.stream);
      delete sys;
    }
  });
}

int cq_range_length(cq_system* sys, int r, int64_t* length, int64_t* n_blocks) {
  return guarded([&] {
    check_sys(sys); check_range(sys, r);
    if (length) *length = sys->S.ranges[r]->length;
    if (n_blocks) *n_blocks = sys->S.ranges[r]->nnz;
  });
}

int cq_export_index(cq_system* sys, int r, const char* name, int64_t* out, int64_t cap, int64_t* n) {
  return guarded([&] {
    check_sys(sys);
    CQ_CHECK(name && n, CQ_ERR_ARG, "null argument");
    std::vector<int64_t> v;
    export_range_array(sys->S, r, name, v);
    *n = (int64_t)v.size();
    if (out) std::memcpy(out, v.data(), sizeof(int64_t) * std::min<int64_t>(cap, (int64_t)v.size()));
  });
}

int cq_export_radius(cq_system* sys, int r, double* out, int64_t cap, int64_t* n) {
  return guarded([&] {
    check_sys(sys); check_range(sys, r);
    CQ_CHECK(n, CQ_ERR_ARG, "null argument");
    RangeIndex& R = *sys->S.ranges[r];
    *n = R.nnz;
    if (out) {
      std::vector<double> v = R.nb_radius.download(sys->S.stream);
      std::memcpy(out, v.data(), sizeof(double) * std::min<int64_t>(cap, R.nnz));
    }
  });
}

int cq_mat_mult(cq_system* sys, int mult_type, int ra, int rb, int rc, double* a_dev, const double* b_dev, double* c_dev,
                int exact) {
  return guarded([&] {
    check_sys(sys); check_range(sys, ra); check_range(sys, rb); check_range(sys, rc);
    CQ_CHECK(a_dev && b_dev && c_dev, CQ_ERR_ARG, "null operand");
    ProductPlan& P = get_plan(sys->S, mult_type, ra, rb, rc);
    CQ_CHECK(exact >= CQ_PREC_FP64_FMA && exact <= CQ_PREC_FP64_TC, CQ_ERR_ARG, "unknown precision");
    if (exact == CQ_PREC_BF16X3 || exact == CQ_PREC_BF16X6)
      mat_mult_mixed(sys->S, mult_type, ra, rb, rc, a_dev, b_dev, c_dev, exact == CQ_PREC_BF16X6 ? 3 : 2);
    else launch_mat_mult(sys->S, P, a_dev, b_dev, c_dev, exact);
  });
}

int cq_mat_mult_batch(int n, cq_system* const* systems, const int* mult_type, const int* ra, const int* rb,
                      const int* rc, double* const* a_dev, const double* const* b_dev, double* const* c_dev,
                      const int* precision) {
  return guarded([&] {
    CQ_CHECK(n >= 1 && systems && mult_type && ra && rb && rc && a_dev && b_dev && c_dev && precision, CQ_ERR_ARG,
             "null argument");
    std::vector<BatchItem> items;
    std::vector<cudaStream_t> streams;
    for (int k = 0; k < n; ++k) {
      cq_system* sys = systems[k];
      check_sys(sys); check_range(sys, ra[k]); check_range(sys, rb[k]); check_range(sys, rc[k]);
      CQ_CHECK(mult_type[k] == 1 || mult_type[k] == 2, CQ_ERR_ARG, "mult_type must be 1 or 2");
      CQ_CHECK(precision[k] == CQ_PREC_FP64 || precision[k] == CQ_PREC_FP64_FMA, CQ_ERR_ARG,
               "batched products are FP64 (CQ_PREC_FP64 or CQ_PREC_FP64_FMA)");
      CQ_CHECK(a_dev[k] && b_dev[k] && c_dev[k], CQ_ERR_ARG, "null operand");
      ProductPlan& P = get_plan(sys->S, mult_type[k], ra[k], rb[k], rc[k]);
      items.push_back({&sys->S, &P, a_dev[k], b_dev[k], c_dev[k], precision[k] == CQ_PREC_FP64 ? 1 : 0});
      if (std::find(streams.begin(), streams.end(), sys->S.stream) == streams.end()) streams.push_back(sys->S.stream);
    }
    // one launch on the first system's stream, after the work already on every system's stream;
    // every system's later work waits for it
    cudaStream_t st = streams[0];
    std::vector<cudaEvent_t> evs;
    auto make_event = [&] {
      cudaEvent_t e;
      CQ_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      evs.push_back(e);
      return e;
    };
    try {
      for (size_t k = 1; k < streams.size(); ++k) {
        cudaEvent_t e = make_event();
        CQ_CUDA(cudaEventRecord(e, streams[k]));
        CQ_CUDA(cudaStreamWaitEvent(st, e, 0));
      }
      launch_mat_mult_batch(items, st);
      if (streams.size() > 1) {
        cudaEvent_t done = make_event();
        CQ_CUDA(cudaEventRecord(done, st));
        for (size_t k = 1; k < streams.size(); ++k) CQ_CUDA(cudaStreamWaitEvent(streams[k], done, 0));
      }
    } catch (...) {
      for (cudaEvent_t e : evs) cudaEventDestroy(e);
      throw;
    }
    for (cudaEvent_t e : evs) cudaEventDestroy(e);
  });
}

int cq_mat_mult_host(cq_system* sys, int mult_type, int ra, int rb, int rc, double* a, const double* b, double* c,
                     int exact) {
  return guarded([&] {
    check_sys(sys); check_range(sys, ra); check_range(sys, rb); check_range(sys, rc);
    CQ_CHECK(a && b && c, CQ_ERR_ARG, "null operand");
    CQ_CHECK(exact >= CQ_PREC_FP64_FMA && exact <= CQ_PREC_FP64_TC, CQ_ERR_ARG, "unknown precision");
    System& S = sys->S;
    int64_t la = S.ranges[ra]->length, lb = S.ranges[rb]->length, lc = S.ranges[rc]->length;
    if (sys->ha.n < (size_t)std::max<int64_t>(la, 1)) sys->ha.alloc(std::max<int64_t>(la, 1), sys->S.stream);
    if (sys->hb.n < (size_t)std::max<int64_t>(lb, 1)) sys->hb.alloc(std::max<int64_t>(lb, 1), sys->S.stream);
    if (sys->hc.n < (size_t)std::max<int64_t>(lc, 1)) sys->hc.alloc(std::max<int64_t>(lc, 1), sys->S.stream);
    ProductPlan& P = get_plan(S, mult_type, ra, rb, rc);
    if (mult_type == 1) CQ_CUDA(cudaMemcpyAsync(sys->ha.p, a, la * sizeof(double), cudaMemcpyHostToDevice, S.stream));
    CQ_CUDA(cudaMemcpyAsync(sys->hb.p, b, lb * sizeof(double), cudaMemcpyHostToDevice, S.stream));
    if (mult_type == 2) CQ_CUDA(cudaMemcpyAsync(sys->hc.p, c, lc * sizeof(double), cudaMemcpyHostToDevice, S.stream));
    if (exact == CQ_PREC_BF16X3 || exact == CQ_PREC_BF16X6)
      mat_mult_mixed(S, mult_type, ra, rb, rc, sys->ha.p, sys->hb.p, sys->hc.p, exact == CQ_PREC_BF16X6 ? 3 : 2);
    else launch_mat_mult(S, P, sys->ha.p, sys->hb.p, sys->hc.p, exact);
    if (mult_type == 1) CQ_CUDA(cudaMemcpyAsync(c, sys->hc.p, lc * sizeof(double), cudaMemcpyDeviceToHost, S.stream));
    else CQ_CUDA(cudaMemcpyAsync(a, sys->ha.p, la * sizeof(double), cudaMemcpyDeviceToHost, S.stream));
    CQ_CUDA(cudaStreamSynchronize(S.stream));
    umma_check(S);
  });
}

int cq_product_work(cq_system* sys, int mult_type, int ra, int rb, int rc, int64_t* triples, int64_t* flops) {
  return guarded([&] {
    check_sys(sys); check_range(sys, ra); check_range(sys, rb); check_range(sys, rc);
    ProductPlan& P = get_plan(sys->S, mult_type, ra, rb, rc);
    if (triples) *triples = P.n_pairs;
    if (flops) *flops = P.flops;
  });
}

int cq_product_tuning(cq_system* sys, int mult_type, int ra, int rb, int rc, int* variant, float* ms, int* group,
                      float* group_ms) {
  return guarded([&] {
    check_sys(sys); check_range(sys, ra); check_range(sys, rb); check_range(sys, rc);
    ProductPlan& P = get_plan(sys->S, mult_type, ra, rb, rc);
    if (variant) *variant = P.tuned;
    if (ms) for (int v = 0; v < 7; ++v) ms[v] = P.tune_ms[v];
    auto it = sys->S.mplans.find(std::make_tuple(mult_type, ra, rb, rc));
    const MixedPlan* M = it == sys->S.mplans.end() ? nullptr : it->second.get();
    static const int kGs[4] = {1, 2, 4, 8};
    if (group) *group = (M && M->tuned_g >= 0) ? kGs[M->tuned_g] : -1;
    if (group_ms) for (int g = 0; g < 4; ++g) group_ms[g] = M ? M->tune_ms[g] : 0.f;
  });
}

int cq_product_tensor_work(cq_system* sys, int mult_type, int ra, int rb, int rc, int64_t* tiles,
                           int64_t* issued_flops, int* usable) {
  return guarded([&] {
    check_sys(sys); check_range(sys, ra); check_range(sys, rb); check_range(sys, rc);
    CQ_CHECK(mult_type == 1 || mult_type == 2, CQ_ERR_ARG, "mult_type must be 1 or 2");
    UmmaPlan& U = get_umma_plan(sys->S, mult_type, ra, rb, rc);
    if (tiles) *tiles = U.n_tiles;
    if (issued_flops) *issued_flops = U.issued_flops;
    if (usable) *usable = U.usable ? 1 : 0;
  });
}

int cq_matrix_sum(cq_system* sys, int ra, double* a_dev, double alpha, int rb, const double* b_dev, double beta) {
  return guarded([&] {
    check_sys(sys); check_range(sys, ra); check_range(sys, rb);
    System& S = sys->S;
    if (ra == rb) {
      dev_scale(S, a_dev, S.ranges[ra]->length, alpha);
      dev_axpy(S, a_dev, S.ranges[ra]->length, beta, b_dev);
    } else {
      dev_matrix_add(S, ra, a_dev, alpha, rb, b_dev, beta);
    }
  });
}

int cq_matrix_transpose(cq_system* sys, int r, const double* a_dev, double* at_dev) {
  return guarded([&] { check_sys(sys); check_range(sys, r); dev_transpose(sys->S, r, a_dev, at_dev); });
}

int cq_matrix_trace(cq_system* sys, int r, const double* a_dev, double* result) {
  return guarded([&] { check_sys(sys); check_range(sys, r); *result = dev_trace(sys->S, r, a_dev); });
}

int cq_matrix_product_trace(cq_system* sys, int r, const double* a_dev, const double* b_dev, double* result) {
  return guarded([&] {
    check_sys(sys); check_range(sys, r);
    *result = dev_dot(sys->S, a_dev, b_dev, sys->S.ranges[r]->length);
  });
}

int cq_synchronize(cq_system* sys) {
  return guarded([&] {
    check_sys(sys);
    CQ_CUDA(cudaStreamSynchronize(sys->S.stream));
    umma_check(sys->S);
  });
}

int cq_system_set_stream(cq_system* sys, void* stream) {
  return guarded([&] {
    check_sys(sys);
    CQ_CUDA(cudaStreamSynchronize(sys->S.stream));
    sys->S.stream = stream ? (cudaStream_t)stream : sys->S.own.s;
  });
}

int cq_profile_enable(cq_system* sys, int on) {
  return guarded([&] {
    check_sys(sys);
    sys->S.prof.on = on != 0;
    sys->S.prof.clear();
  });
}

int cq_profile_read(cq_system* sys, int64_t* launches, double* ms, double* bytes, double* flops) {
  return guarded([&] {
    check_sys(sys);
    CQ_CUDA(cudaStreamSynchronize(sys->S.stream));
    double t = 0, by = 0, fl = 0;
    for (auto& r : sys->S.prof.recs) {
      float e = 0.f;
      CQ_CUDA(cudaEventElapsedTime(&e, r.a, r.b));
      t += e; by += r.bytes; fl += r.flops;
    }
    if (launches) *launches = (int64_t)sys->S.prof.recs.size();
    if (ms) *ms = t;
    if (bytes) *bytes = by;
    if (flops) *flops = fl;
    sys->S.prof.clear();
  });
}

int cq_system_set_option(cq_system* sys, int option, int value) {
  return guarded([&] {
    check_sys(sys);
    if (option == CQ_OPT_MULT_VARIANT) {
      CQ_CHECK(value >= -1 && value <= 6, CQ_ERR_ARG, "mult variant must be -1 (autotuned) or 0..6");
      sys->S.mult_variant = value;
    } else if (option == CQ_OPT_BLOCKING_SYNC) {
      sys->S.blocking_sync = value != 0;
    } else if (option == CQ_OPT_TEST_STALL) {
      sys->S.umma_test_stall = value != 0;
    } else if (option == CQ_OPT_MIXED_KERNEL) {
      CQ_CHECK(value >= -1 && value <= 1, CQ_ERR_ARG,
               "mixed kernel must be -1 (timed choice), 0 (tcgen05 tiles) or 1 (mma.sync blocks)");
      sys->S.mixed_kernel = value;
    } else if (option == CQ_OPT_SPLIT_GROUP) {
      CQ_CHECK(value == -1 || value == 1 || value == 2 || value == 4 || value == 8, CQ_ERR_ARG,
               "split group must be -1 (autotuned), 1, 2, 4 or 8");
      sys->S.split_group = value;
    } else {
      throw Error(CQ_ERR_ARG, "unknown option");
    }
  });
}

int cq_generate_SH(cq_system* sys, int r, int which, uint64_t seed, double* out) {
  return guarded([&] {
    check_sys(sys); check_range(sys, r);
    CQ_CHECK(out && (which == 0 || which == 1), CQ_ERR_ARG, "bad generator arguments");
    generate_SH(sys->S, r, which, seed, out);
  });
}

int cq_launch_count(cq_system* sys, int64_t* count) {
  return guarded([&] { check_sys(sys); CQ_CHECK(count, CQ_ERR_ARG, "null argument"); *count = sys->S.launches; });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Deferred drop-in calls (cq_m_kern_defer): the device copies of a and c live across the partition
// loop of one mat_mult, each call copies only its partition's b and block lists (through pinned,
// double-buffered staging) and enqueues its arithmetic on the drop-in stream, and the call of the
// last partition copies the result back and synchronises.  Buffers grow and are reused: after the
// first loop no call allocates.  Per calling thread.
// ---------------------------------------------------------------------------
struct PinnedBuf {
  unsigned char* p = nullptr;
  size_t n = 0;
  cudaEvent_t used = nullptr;      // recorded after the copy that last read this buffer
  void reserve(size_t bytes) {
    if (bytes <= n) return;
    if (p) cudaFreeHost(p);
    p = nullptr; n = 0;
    CQ_CUDA(cudaMallocHost((void**)&p, bytes));
    n = bytes;
  }
  ~PinnedBuf() {
    if (used) cudaEventDestroy(used);
    if (p) cudaFreeHost(p);
  }
};

struct DropinState {
  int np = 0;                      // A-halo partitions of the current loop (0: complete every call)
  int type = 0;
  bool open = false;               // a loop's device copies hold pending work
  double* host_out = nullptr;      // result array of the open loop (c for max, a for min)
  int64_t len_out = 0;
  cudaStream_t st = nullptr;
  DevBuf<double> da, db, dc;
  DevBuf<unsigned char> didx;
  PinnedBuf stage[2];
  int turn = 0;
  ~DropinState() {
    if (st) { cudaStreamSynchronize(st); }
  }
};
static thread_local DropinState t_dropin;

template <class T>
static void grow(DevBuf<T>& b, size_t n, cudaStream_t st) {
  if (b.n < n) b.alloc(n, st);
}

static void dropin_flush(DropinState& D) {
  if (!D.open) return;
  D.open = false;
  const double* src = D.type == 1 ? D.dc.p : D.da.p;
  if (D.len_out) CQ_CUDA(cudaMemcpyAsync(D.host_out, src, sizeof(double) * D.len_out, cudaMemcpyDeviceToHost, D.st));
  CQ_CUDA(cudaStreamSynchronize(D.st));
}

static void dropin_deferred(DropinState& D, int type, int kpart, const std::vector<int64_t>& out_off,
                            const std::vector<int>& dims, const std::vector<int64_t>& ptr,
                            const std::vector<int64_t>& pairs, double* a, const double* b, double* c, int lena,
                            int lenb, int lenc) {
  if (!D.st) CQ_CUDA(cudaStreamCreateWithFlags(&D.st, cudaStreamNonBlocking));
  if (kpart == 1 || !D.open) {
    dropin_flush(D);                 // a loop left without its last partition completes here
    D.type = type;
    D.host_out = type == 1 ? c : a;
    D.len_out = type == 1 ? lenc : lena;
    grow(D.da, (size_t)std::max(lena, 1), D.st);
    grow(D.dc, (size_t)std::max(lenc, 1), D.st);
    CQ_CUDA(cudaMemcpyAsync(D.da.p, a, sizeof(double) * lena, cudaMemcpyHostToDevice, D.st));
    CQ_CUDA(cudaMemcpyAsync(D.dc.p, c, sizeof(double) * lenc, cudaMemcpyHostToDevice, D.st));
    CQ_CUDA(cudaStreamSynchronize(D.st));   // the caller may reuse a and c only after their copies
    D.open = true;
  }
  CQ_CHECK(type == D.type, CQ_ERR_STATE, "m_kern: mult type changed inside a deferred partition loop");
  const int n_out = (int)out_off.size();
  if (n_out > 0) {
    // staging: b of this partition, then the block lists (8-byte aligned sections)
    const size_t sb = sizeof(double) * lenb, so = sizeof(int64_t) * out_off.size(), sp = sizeof(int64_t) * ptr.size(),
                 sq = sizeof(int64_t) * pairs.size(), sd = ((sizeof(int) * dims.size() + 7) / 8) * 8;
    const size_t total = sb + so + sp + sq + sd;
    PinnedBuf& P = D.stage[D.turn];
    D.turn ^= 1;
    if (P.used) CQ_CUDA(cudaEventSynchronize(P.used));   // the copy that last read this buffer is done
    P.reserve(total);
    unsigned char* h = P.p;
    std::memcpy(h, b, sb);
    std::memcpy(h + sb, out_off.data(), so);
    std::memcpy(h + sb + so, ptr.data(), sp);
    std::memcpy(h + sb + so + sp, pairs.data(), sq);
    std::memcpy(h + sb + so + sp + sq, dims.data(), sizeof(int) * dims.size());
    grow(D.didx, total - sb + 8, D.st);
    grow(D.db, (size_t)std::max(lenb, 1), D.st);
    CQ_CUDA(cudaMemcpyAsync(D.db.p, h, sb, cudaMemcpyHostToDevice, D.st));
    CQ_CUDA(cudaMemcpyAsync(D.didx.p, h + sb, total - sb, cudaMemcpyHostToDevice, D.st));
    if (!P.used) CQ_CUDA(cudaEventCreateWithFlags(&P.used, cudaEventDisableTiming));
    CQ_CUDA(cudaEventRecord(P.used, D.st));
    const int64_t* d_out = reinterpret_cast<const int64_t*>(D.didx.p);
    const int64_t* d_ptr = d_out + out_off.size();
    const int64_t* d_pairs = d_ptr + ptr.size();
    const int* d_dims = reinterpret_cast<const int*>(d_pairs + pairs.size());
    if (type == 1) launch_dropin(1, d_out, d_dims, d_ptr, d_pairs, n_out, D.da.p, D.db.p, D.dc.p, D.st);
    else launch_dropin(2, d_out, d_dims, d_ptr, d_pairs, n_out, D.dc.p, D.db.p, D.da.p, D.st);
  }
  if (kpart == D.np) dropin_flush(D);
}

extern "C" {

// ---------------------------------------------------------------------------
// drop-in m_kern_max / m_kern_min: the loop nest of the default kernel walked
// on the host to list the block triples of this partition (in order), the
// arithmetic done on the GPU with the same per-element operation sequence.
// ---------------------------------------------------------------------------
static int dropin(int type, int k_off, int kpart, const int* ib_nd_acc, const int* ibaddr, const int* nbnab,
                  const int* ibpart, const int* ibseq, const int* bndim2, double* a, const double* b, double* c,
                  const int* nh_part, const int* j_beg, const int* j_seq, const int* ndimi, const int* ndimj,
                  const int* i_halo, const int* i_hbeg, const int* i_h2d, int ni_in_halo, const int* i_prim,
                  const int* i_beg, const int* i_nd_beg, const int* n_hnab, int lena, int lenb, int lenc) {
  return guarded([&] {
    CQ_CHECK(ib_nd_acc && ibaddr && nbnab && ibpart && ibseq && bndim2 && a && b && c && nh_part && j_beg && j_seq &&
                 ndimi && ndimj && i_halo && i_hbeg && i_h2d && i_prim && i_beg && i_nd_beg && n_hnab,
             CQ_ERR_ARG, "null argument");
    CQ_CHECK(kpart >= 1, CQ_ERR_ARG, "kpart must be >= 1");
    // Fortran 1-based views
    auto F = [](const int* p) { return p - 1; };
    const int *ib_nd_acc1 = F(ib_nd_acc), *ibaddr1 = F(ibaddr), *nbnab1 = F(nbnab), *ibpart1 = F(ibpart),
              *ibseq1 = F(ibseq), *bndim21 = F(bndim2), *nh_part1 = F(nh_part), *j_beg1 = F(j_beg), *j_seq1 = F(j_seq),
              *ndimi1 = F(ndimi), *ndimj1 = F(ndimj), *i_halo1 = F(i_halo), *i_hbeg1 = F(i_hbeg), *i_h2d1 = F(i_h2d),
              *i_prim1 = F(i_prim), *i_beg1 = F(i_beg), *i_nd_beg1 = F(i_nd_beg), *n_hnab1 = F(n_hnab);
    // triples (out_off, x_off, b_off, nd_out_rows, nd_out_cols, ndk) in kernel order, 0-based element offsets
    struct Tri { int64_t out, x, b; int r, cols, kd; };
    std::vector<Tri> tri;
    std::vector<int> jb2ch;
    for (int k = 1; k <= nh_part1[kpart]; ++k) {
      int k_in_halo = j_beg1[kpart] + k - 1;
      int k_in_part = j_seq1[k_in_halo];
      int nbkbeg = ibaddr1[k_in_part];
      int nb_nd_kbeg = ib_nd_acc1[k_in_part];
      int nd3 = ndimj1[k_in_halo];
      int nbn = nbnab1[k_in_part];
      jb2ch.assign(nbn + 1, 0);
      for (int j = 1; j <= nbn; ++j)
        jb2ch[j] = i_halo1[i_hbeg1[ibpart1[nbkbeg + j - 1] + k_off] + ibseq1[nbkbeg + j - 1] - 1];
      int nabeg = i_nd_beg1[k_in_halo];
      for (int i = 1; i <= n_hnab1[k_in_halo]; ++i) {
        int ip = i_prim1[i_beg1[k_in_halo] + i - 1];
        int nd1 = ndimi1[ip];
        int64_t icad = (int64_t)(ip - 1) * ni_in_halo;
        int nbbeg = nb_nd_kbeg;
        for (int j = 1; j <= nbn; ++j) {
          int nd2 = bndim21[nbkbeg + j - 1];
          if (jb2ch[j] != 0) {
            int ncbeg = i_h2d1[icad + jb2ch[j]];
            if (ncbeg != 0) {
              CQ_CHECK(nabeg + nd1 * nd3 - 1 <= lena && nbbeg + nd3 * nd2 - 1 <= lenb && ncbeg + nd1 * nd2 - 1 <= lenc,
                       CQ_ERR_BOUNDS, "m_kern: block outside the passed arrays");
              if (type == 1) tri.push_back({ncbeg - 1, nabeg - 1, nbbeg - 1, nd1, nd2, nd3});
              else tri.push_back({nabeg - 1, ncbeg - 1, nbbeg - 1, nd1, nd3, nd2});
            }
          }
          nbbeg += nd3 * nd2;
        }
        nabeg += nd1 * nd3;
      }
    }
    if (tri.empty()) {
      DropinState& D = t_dropin;
      if (D.np > 0) dropin_deferred(D, type, kpart, {}, {}, {0}, {}, a, b, c, lena, lenb, lenc);
      return;
    }
    // group by output block, preserving order
    std::vector<int> order(tri.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int p, int q) { return tri[p].out < tri[q].out; });
    std::vector<int64_t> out_off, ptr, pairs;
    std::vector<int> dims;
    for (size_t t = 0; t < order.size(); ++t) {
      const Tri& T = tri[order[t]];
      if (t == 0 || T.out != tri[order[t - 1]].out) {
        out_off.push_back(T.out);
        dims.push_back(T.r); dims.push_back(T.cols);
        ptr.push_back((int64_t)t);
      }
      pairs.push_back(T.x); pairs.push_back(T.b); pairs.push_back(T.kd);
    }
    ptr.push_back((int64_t)order.size());
    DropinState& D = t_dropin;
    if (D.np > 0) {
      dropin_deferred(D, type, kpart, out_off, dims, ptr, pairs, a, b, c, lena, lenb, lenc);
      return;
    }
    cudaStream_t st = 0;
    DevBuf<int64_t> d_out, d_ptr, d_pairs;
    DevBuf<int> d_dims;
    DevBuf<double> da, db, dc;
    d_out.upload(out_off, st); d_ptr.upload(ptr, st); d_pairs.upload(pairs, st); d_dims.upload(dims, st);
    da.upload(a, lena, st); db.upload(b, lenb, st); dc.upload(c, lenc, st);
    if (type == 1) launch_dropin(1, d_out.p, d_dims.p, d_ptr.p, d_pairs.p, (int)out_off.size(), da.p, db.p, dc.p, st);
    else launch_dropin(2, d_out.p, d_dims.p, d_ptr.p, d_pairs.p, (int)out_off.size(), dc.p, db.p, da.p, st);
    if (type == 1) CQ_CUDA(cudaMemcpyAsync(c, dc.p, sizeof(double) * lenc, cudaMemcpyDeviceToHost, st));
    else CQ_CUDA(cudaMemcpyAsync(a, da.p, sizeof(double) * lena, cudaMemcpyDeviceToHost, st));
    CQ_CUDA(cudaStreamSynchronize(st));
  });
}

int cq_m_kern_defer(int np_in_halo) {
  return guarded([&] {
    CQ_CHECK(np_in_halo >= 0, CQ_ERR_ARG, "np_in_halo must be >= 0");
    DropinState& D = t_dropin;
    if (np_in_halo == 0) dropin_flush(D);
    D.np = np_in_halo;
  });
}

int cq_m_kern_flush(void) {
  return guarded([&] { dropin_flush(t_dropin); });
}

int cq_m_kern_max(int k_off, int kpart, const int* ib_nd_acc, const int* ibaddr, const int* nbnab, const int* ibpart,
                  const int* ibseq, const int* bndim2, const double* a, const double* b, double* c,
                  const int* ahalo_nh_part, const int* ahalo_j_beg, const int* ahalo_j_seq, const int* ahalo_ndimi,
                  const int* ahalo_ndimj, const int* chalo_i_halo, const int* chalo_i_hbeg, const int* chalo_i_h2d,
                  int chalo_ni_in_halo, const int* at_i_prim, const int* at_i_beg, const int* at_i_nd_beg,
                  const int* at_n_hnab, int mx_absb, int mx_part, int mx_iprim, int lena, int lenb, int lenc) {
  (void)mx_absb; (void)mx_part; (void)mx_iprim;
  return dropin(1, k_off, kpart, ib_nd_acc, ibaddr, nbnab, ibpart, ibseq, bndim2, const_cast<double*>(a), b, c,
                ahalo_nh_part, ahalo_j_beg, ahalo_j_seq, ahalo_ndimi, ahalo_ndimj, chalo_i_halo, chalo_i_hbeg,
                chalo_i_h2d, chalo_ni_in_halo, at_i_prim, at_i_beg, at_i_nd_beg, at_n_hnab, lena, lenb, lenc);
}

int cq_m_kern_min(int k_off, int kpart, const int* ib_nd_acc, const int* ibaddr, const int* nbnab, const int* ibpart,
                  const int* ibseq, const int* bndim2, double* a, const double* b, const double* c,
                  const int* ahalo_nh_part, const int* ahalo_j_beg, const int* ahalo_j_seq, const int* ahalo_ndimi,
                  const int* ahalo_ndimj, const int* chalo_i_halo, const int* chalo_i_hbeg, const int* chalo_i_h2d,
                  int chalo_ni_in_halo, const int* at_i_prim, const int* at_i_beg, const int* at_i_nd_beg,
                  const int* at_n_hnab, int mx_absb, int mx_part, int mx_iprim, int lena, int lenb, int lenc) {
  (void)mx_absb; (void)mx_part; (void)mx_iprim;
  return dropin(2, k_off, kpart, ib_nd_acc, ibaddr, nbnab, ibpart, ibseq, bndim2, a, b, const_cast<double*>(c),
                ahalo_nh_part, ahalo_j_beg, ahalo_j_seq, ahalo_ndimi, ahalo_ndimj, chalo_i_halo, chalo_i_hbeg,
                chalo_i_h2d, chalo_ni_in_halo, at_i_prim, at_i_beg, at_i_nd_beg, at_n_hnab, lena, lenb, lenc);
}

// ---- matrices by id (the device side of mat_p(id)%matrix) ----------------------------------
static BoundMatrix& bound(cq_system* sys, int id) {
  auto it = sys->store.find(id);
  CQ_CHECK(it != sys->store.end(), CQ_ERR_ARG, "matrix id " + std::to_string(id) + " is not bound");
  return *it->second;
}

int cq_matrix_bind(cq_system* sys, int id, int r, double* host) {
  return guarded([&] {
    check_sys(sys); check_range(sys, r);
    CQ_CHECK(sys->store.find(id) == sys->store.end(), CQ_ERR_STATE,
             "matrix id " + std::to_string(id) + " is already bound");
    auto m = std::make_unique<BoundMatrix>();
    const int64_t n = std::max<int64_t>(sys->S.ranges[r]->length, 1);
    m->r = r;
    m->host = host;
    m->dev.alloc((size_t)n, sys->S.stream);
    CQ_CUDA(cudaMemsetAsync(m->dev.p, 0, sizeof(double) * n, sys->S.stream));
    sys->store[id] = std::move(m);
  });
}

int cq_matrix_unbind(cq_system* sys, int id) {
  return guarded([&] {
    check_sys(sys);
    BoundMatrix& m = bound(sys, id);
    // release on the stream the system uses now: the buffer may have been allocated on a stream
    // replaced since by cq_system_set_stream (whose earlier work that call waited for), while
    // work enqueued on the current stream may still read or write it
    m.dev.st = sys->S.stream;
    sys->store.erase(id);
  });
}

int cq_matrix_device(cq_system* sys, int id, double** dev, int64_t* length) {
  return guarded([&] {
    check_sys(sys);
    BoundMatrix& m = bound(sys, id);
    if (dev) *dev = m.dev.p;
    if (length) *length = sys->S.ranges[m.r]->length;
  });
}

int cq_matrix_upload(cq_system* sys, int id) {
  return guarded([&] {
    check_sys(sys);
    BoundMatrix& m = bound(sys, id);
    CQ_CHECK(m.host != nullptr, CQ_ERR_STATE, "matrix id " + std::to_string(id) + " has no host array");
    const int64_t n = sys->S.ranges[m.r]->length;
    if (n) CQ_CUDA(cudaMemcpyAsync(m.dev.p, m.host, sizeof(double) * n, cudaMemcpyHostToDevice, sys->S.stream));
  });
}

int cq_matrix_download(cq_system* sys, int id) {
  return guarded([&] {
    check_sys(sys);
    BoundMatrix& m = bound(sys, id);
    CQ_CHECK(m.host != nullptr, CQ_ERR_STATE, "matrix id " + std::to_string(id) + " has no host array");
    const int64_t n = sys->S.ranges[m.r]->length;
    if (n) CQ_CUDA(cudaMemcpyAsync(m.host, m.dev.p, sizeof(double) * n, cudaMemcpyDeviceToHost, sys->S.stream));
    CQ_CUDA(cudaStreamSynchronize(sys->S.stream));
  });
}

int cq_matrix_product_id(cq_system* sys, int mult_type, int ida, int idb, int idc, int precision) {
  return guarded([&] {
    check_sys(sys);
    CQ_CHECK(mult_type == 1 || mult_type == 2, CQ_ERR_ARG, "mult_type must be 1 or 2");
    CQ_CHECK(precision >= CQ_PREC_FP64_FMA && precision <= CQ_PREC_FP64_TC, CQ_ERR_ARG, "unknown precision");
    const int out = mult_type == 1 ? idc : ida;
    CQ_CHECK(out != (mult_type == 1 ? ida : idc) && out != idb, CQ_ERR_ARG, "the product's output must not be an input");
    BoundMatrix &A = bound(sys, ida), &B = bound(sys, idb), &C = bound(sys, idc);
    ProductPlan& P = get_plan(sys->S, mult_type, A.r, B.r, C.r);
    if (precision == CQ_PREC_BF16X3 || precision == CQ_PREC_BF16X6)
      mat_mult_mixed(sys->S, mult_type, A.r, B.r, C.r, A.dev.p, B.dev.p, C.dev.p, precision == CQ_PREC_BF16X6 ? 3 : 2);
    else launch_mat_mult(sys->S, P, A.dev.p, B.dev.p, C.dev.p, precision);
  });
}

int cq_matrix_sum_id(cq_system* sys, int ida, double alpha, int idb, double beta) {
  return guarded([&] {
    check_sys(sys);
    BoundMatrix &A = bound(sys, ida), &B = bound(sys, idb);
    System& S = sys->S;
    if (A.r == B.r) {
      dev_scale(S, A.dev.p, S.ranges[A.r]->length, alpha);
      dev_axpy(S, A.dev.p, S.ranges[A.r]->length, beta, B.dev.p);
    } else {
      dev_matrix_add(S, A.r, A.dev.p, alpha, B.r, B.dev.p, beta);
    }
  });
}

int cq_matrix_transpose_id(cq_system* sys, int ida, int idat) {
  return guarded([&] {
    check_sys(sys);
    BoundMatrix &A = bound(sys, ida), &AT = bound(sys, idat);
    CQ_CHECK(A.r == AT.r && ida != idat, CQ_ERR_ARG, "transpose: two different matrices of one range");
    dev_transpose(sys->S, A.r, A.dev.p, AT.dev.p);
  });
}

int cq_matrix_product_trace_id(cq_system* sys, int ida, int idb, double* result) {
  return guarded([&] {
    check_sys(sys);
    CQ_CHECK(result != nullptr, CQ_ERR_ARG, "null result");
    BoundMatrix &A = bound(sys, ida), &B = bound(sys, idb);
    CQ_CHECK(A.r == B.r, CQ_ERR_ARG, "product trace: both matrices of one range");
    *result = dev_dot(sys->S, A.dev.p, B.dev.p, sys->S.ranges[A.r]->length);
  });
}

}  // extern "C"
