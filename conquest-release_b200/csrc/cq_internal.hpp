// Internal declarations of the B200 block-sparse multiply / LNV library.
// Everything here is device-resident state plus the host-side geometry that
// feeds the GPU index builders.  See include/cq_b200.h for the public C ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/cq_b200.h"

namespace cqb {

// ---------------------------------------------------------------------------
// errors: every failure becomes a status code at the C ABI
// ---------------------------------------------------------------------------
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
void set_last_error(const std::string& m);

#define CQ_CUDA(call)                                                                              \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      throw ::cqb::Error(CQ_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));         \
  } while (0)
#define CQ_CHECK(cond, code, msg)                 \
  do {                                            \
    if (!(cond)) throw ::cqb::Error(code, (msg)); \
  } while (0)

// ---------------------------------------------------------------------------
// device buffer (RAII, stream-ordered allocator)
// Memory comes from the device's default pool with cudaMallocAsync on the stream
// given to alloc() and goes back with cudaFreeAsync on that stream, so neither
// allocation nor release synchronises the device: solves of independent systems
// on their own streams keep running while another one sets up or tears down.
// A buffer is released on the stream it was (last) allocated on; every buffer is
// used on that stream or on a later stream of the same system, which is
// synchronised before the system (or solver) holding it is destroyed.
// ---------------------------------------------------------------------------
struct DevAccount {               // device bytes held through DevBuf by the calling thread
  int64_t live = 0, peak = 0;
};
DevAccount& dev_account();        // thread-local
void dev_account_add(int64_t bytes);

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t st = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), st(o.st) { o.p = nullptr; o.n = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; st = o.st; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DevBuf() { release(); }
  // (re)allocate on stream s; old memory is released on s, the stream any pending use is on
  void alloc(size_t count, cudaStream_t s) {
    st = s;
    release();
    if (count) {
      cudaError_t e = cudaMallocAsync((void**)&p, count * sizeof(T), s);
      if (e != cudaSuccess) {
        p = nullptr;
        throw Error(CQ_ERR_OOM, "cudaMallocAsync failed: " + std::string(cudaGetErrorString(e)));
      }
      n = count;
      dev_account_add((int64_t)(count * sizeof(T)));
    }
  }
  void release() {
    if (p) {
      cudaFreeAsync(p, st);
      dev_account_add(-(int64_t)(n * sizeof(T)));
    }
    p = nullptr; n = 0;
  }
  void upload(const T* h, size_t count, cudaStream_t s) {
    alloc(count, s);
    if (count) CQ_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void upload(const std::vector<T>& v, cudaStream_t s) { upload(v.data(), v.size(), s); }
  std::vector<T> download(cudaStream_t s) const {
    std::vector<T> v(n);
    if (n) {
      CQ_CUDA(cudaMemcpyAsync(v.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost, s));
      CQ_CUDA(cudaStreamSynchronize(s));
    }
    return v;
  }
};

// ---------------------------------------------------------------------------
// host geometry: partitions, primary set, covering set (one process)
// All indices 0-based; partition/cover labels keep the reference's 1-based
// CC numbering where they enter index arithmetic.
// ---------------------------------------------------------------------------
struct Geometry {
  int n_atoms = 0;
  double cell[3] = {0, 0, 0};
  std::vector<double> coord;          // wrapped, input order, 3*n
  std::vector<int> nsf;               // block size per input atom
  int n_parts[3] = {1, 1, 1};
  int np_in_cell = 0;
  std::vector<int> hilbert_to_cc;     // [hilbert pos] -> 1-based CC label
  std::vector<int> cc_to_seq;         // [cc label] -> 0-based primary-partition position
  std::vector<int> part_natoms;       // [cc label]
  std::vector<int> part_first_cell;   // [cc label] first cell-order atom (0-based)
  std::vector<int> cell_to_global;    // cell-order -> input atom
  // primary set (primary order == cell order on one process)
  int n_prim = 0;
  std::vector<int> prim_global;       // [p] input atom
  std::vector<int> prim_part;         // [p] primary partition position
  std::vector<int> prim_seq;          // [p] 1-based sequence in partition
  std::vector<int> part_first_prim;   // [partition position] first primary atom
  std::vector<int> part_disp;         // [partition position*3] idisp_prim
  std::vector<int> prim_cover_label;  // [p] lab_cover of its partition (1-based)
  std::vector<double> prim_x;         // [3p]
  // covering set
  int ncover[3] = {0, 0, 0};
  int nspan[3] = {0, 0, 0};
  int ng_cover = 0, n_cover_atoms = 0;
  std::vector<int> cover_label;       // [np] 1-based lab_cover
  std::vector<int> cover_cell;        // [np] 1-based lab_cell (CC of the home partition)
  std::vector<int> cover_first;       // [np] first cover atom (0-based)
  std::vector<int> cover_count;       // [np]
  std::vector<int> label_to_cover;    // [label] -> np (0-based), -1 if none
  std::vector<int> cover_shift;       // [3*np] periodic image of the partition, in cell vectors
  std::vector<double> cover_x;        // [3c]
  std::vector<int> cover_global;      // [c] input atom
  std::vector<int> cover_part;        // [c] cover partition np
  std::vector<int> cover_seq;         // [c] 1-based seq in partition
  std::vector<int> cover_nsf;         // [c]
  std::vector<int> cover_home_prim;   // [c] primary atom of the same input atom
  std::vector<int> global_to_prim;    // [input atom] -> primary index
};

struct GeometryParams {
  int max_atoms_part = 34;
  double gap_threshold = 14.0;
  double avg_atomic_diameter = 5.0;
};

void build_geometry(Geometry& g, int n, const double* coords, const double* cell, const int* nsf, double cover_rcut,
                    const GeometryParams& prm);

// ---------------------------------------------------------------------------
// device geometry + one index per range
// ---------------------------------------------------------------------------
struct DevGeometry {
  DevBuf<double> prim_x, cover_x;
  DevBuf<int> prim_nsf, prim_cover_label, prim_seq, prim_part, part_disp, cover_nsf, cover_part, cover_seq,
      cover_label_of_part, label_to_cover, cover_first, cover_home_prim, part_first_prim;
  DevBuf<int> prim_global, cover_global, cover_shift;   // uploaded on first use (input generators)
};

struct RangeIndex {
  double rcut = 0;
  int nnz = 0;                  // stored blocks
  int64_t length = 0;           // stored elements
  int ni_in_halo = 0, np_in_halo = 0;
  int max_row = 0;              // largest neighbour count of a row
  DevBuf<int> row_ptr;          // [n_prim+1]
  DevBuf<int64_t> row_elem;     // [n_prim+1]
  DevBuf<int> nb_cover;         // [nnz] cover atom (row-sorted ascending)
  DevBuf<int> nb_halo;          // [nnz] halo index
  DevBuf<int64_t> nb_elem;      // [nnz] first element of the block
  DevBuf<int> nb_row;           // [nnz] owning primary atom
  DevBuf<int> nb_ibpart;        // [nnz] partition displacement code (end_part_comms)
  DevBuf<double> nb_radius;     // [nnz]
  DevBuf<int64_t> onsite;       // [n_prim] element offset of the self block
  DevBuf<int> cover_to_halo;    // [n_cover_atoms] -> halo index or -1
  DevBuf<int> halo_cover;       // [ni_in_halo]
  DevBuf<int> col_ptr;          // [ni_in_halo+1] retro lists (primary atoms of each halo atom)
  DevBuf<int> col_row;          // [nnz]
  DevBuf<int> col_blk;          // [nnz]
  DevBuf<int> trans_dest;       // [nnz] block of the global transpose
  std::vector<int> h_row_ptr;   // host copy (small)
};

// Per-product pair lists: for each output block, the ordered list of
// (first operand block, B block) pairs in the reference's summation order.
constexpr int kVariantAuto = -1;

struct ProductPlan {
  int mult_type = 1;
  int ra = -1, rb = -1, rc = -1;  // mat_mult roles: a (A or type-2 output), b, c (C or type-2 input)
  int out_range = -1;             // range of the block list owner (C for type 1, a for type 2)
  int64_t n_pairs = 0;            // total (x, b) pairs = block triples with a stored result
  int64_t flops = 0;              // 2 * sum nd_i nd_j nd_k over the triples
  DevBuf<int64_t> ptr;            // [n_out_blocks+1]
  DevBuf<int2> pairs;             // [n_pairs] (x block, b block)
  int n_tiles = 0;                // row tiles of the staged 4x4 kernel: (q0, q1, x row first, x row end)
  DevBuf<int4> tiles;
  DevBuf<int> order;              // output blocks by descending pair count (warp-staged 4x4 kernel)
  int tuned = -1;                 // FP64 kernel variant chosen by the autotuner (-1: not tuned yet)
  float tune_ms[7] = {0, 0, 0, 0, 0, 0, 0};
};

// Split-precision tensor-core product: pair lists sorted by the first operand block,
// and groups of consecutive output blocks of one row (one warp each).
struct MixedPlan {
  int mult_type = 1, ra = -1, rb = -1, rc = -1, out_range = -1;
  int n_groups[4] = {-1, -1, -1, -1};   // groups of 1, 2, 4 and 8 output blocks (-1: not built yet)
  int tuned_g = -1;                 // group size chosen by the autotuner (index into 1, 2, 4, 8)
  int kernel = -1;                  // 0 = tcgen05 tiles, 1 = per-block mma.sync (-1: not chosen yet)
  float tune_ms[4] = {0, 0, 0, 0};
  int tuned_g6 = -1;                // three-part split: group size chosen (index into 1, 2, 4)
  float tune_ms6[3] = {0, 0, 0};
  int64_t n_pairs = 0, flops = 0;
  DevBuf<int64_t> own_ptr;        // type 2 only (type 1 uses the FP64 plan's lists, already sorted)
  DevBuf<int2> own_pairs;
  const int64_t* ptr = nullptr;
  const int2* pairs = nullptr;
  DevBuf<int2> groups[4];
};

struct FragBuf { DevBuf<uint4> hi, lo, mid; };   // mid: three-part split only

// Dense tensor-core tile of a split-precision product (umma.cu): up to 128 output rows (a run of
// primary atoms) x one column chunk (a run of up to 128 orbitals of cover atoms), contracted over the
// units (runs of cover atoms of up to 16 orbitals) that its pair lists use.
struct UmmaTile {
  int row_first, n_rows;          // primary atoms [row_first, row_first + n_rows)
  int n_cols;                     // atoms of the column chunk
  int row_tab, col_tab;           // offsets of the 128-entry row tables of the row group and the chunk
  int om_off;                     // outmap[om_off + ii * n_cols + jj]: output block or -1
  int u_off, n_u;                 // unit entries units[u_off, u_off + n_u): (X slab, B slab)
};

struct UmmaPlan {
  bool usable = false;            // every block size in 4..16
  int n_tiles = 0;
  int64_t flops = 0, n_pairs = 0; // useful work (the FP64 plan's)
  int64_t issued_flops = 0;       // tensor work issued: 3 MMAs x 2 x 128 x 128 x 16 per unit of every tile
  int64_t n_xslabs = 0, n_bslabs = 0;
  DevBuf<UmmaTile> tiles;
  DevBuf<int2> units;
  DevBuf<unsigned int> rtabs, ktabs;   // row tables (row groups, column chunks); K tables of the units
  DevBuf<int> outmap, xtab, btab, xs_rtab, xs_unit, bs_rtab, bs_unit;
  DevBuf<uint4> xslabs, bslabs;   // packed bf16 operands, 8 KB per slab, rewritten by every product call
  DevBuf<int> tile_counter;       // the persistent kernel's next tile
  // host side of the plan, kept to build the slab tables and buffers on the product's first
  // tensor-core call (a product that runs on the per-block kernel never allocates them)
  bool materialised = false;
  int mult_type = 1, ra = -1, rb = -1, rc = -1, n_groups = 0, n_chunks = 0;
  std::vector<int2> h_q_tile;
  std::vector<int> h_xh, h_xcov, h_unit_of, h_unit_pos, h_chunk_of, h_chunk_pos, h_u_cand, h_bpre;
  std::vector<unsigned int> h_bmark;
  std::vector<int64_t> h_u_off, h_xs_tile;
};

struct AddMap {                   // partner of each block of range A in range B (-1 = none)
  DevBuf<int> partner;
};

// CUDA-event timing of the block-product launches (enabled on request)
struct ProductProfile {
  bool on = false;
  struct Rec { cudaEvent_t a, b; double bytes, flops; };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> spare;
  cudaEvent_t get();
  void clear();
  ~ProductProfile();
};

struct OwnedStream {              // destroyed after every buffer of the system has been released on it
  cudaStream_t s = nullptr;
  ~OwnedStream() {
    if (s) { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
  }
};

struct System {
  OwnedStream own;                // the stream created with the system (first member: destroyed last)
  Geometry geo;
  DevGeometry dg;
  std::vector<std::unique_ptr<RangeIndex>> ranges;
  std::map<std::tuple<int, int, int, int>, std::unique_ptr<ProductPlan>> plans;
  std::map<std::pair<int, int>, std::unique_ptr<AddMap>> addmaps;
  std::map<std::tuple<int, int, int, int>, std::unique_ptr<MixedPlan>> mplans;
  std::map<std::pair<int, int>, FragBuf> frags;   // (range, slot) fragment buffers of the mixed products
  std::map<std::tuple<int, int, int, int>, std::unique_ptr<UmmaPlan>> uplans;   // tensor-core tile plans
  int mixed_kernel = -1;          // split-precision products: 0 = tcgen05 tiles (umma.cu), 1 = mma.sync per block,
                                  // -1 = chosen per product by the tile plan's useful fraction
  int* umma_err_host = nullptr;   // mapped host word set by a tensor-core product whose bounded wait ran out
  int split_group = -1;           // CQ_OPT_SPLIT_GROUP: forced output blocks per mma.sync split warp (-1 tuned)
  int umma_test_stall = 0;        // test hook (CQ_OPT_TEST_STALL): the next tensor-core product stalls
  int* umma_err_dev = nullptr;
  cudaStream_t stream = nullptr;  // the stream all work of the system is enqueued on
  int uniform_nsf = 0;            // block size when every atom has the same one, else 0
  int n_solvers = 0;              // live LNV solvers built on this system (destroyed before it)
  int max_nsf = 0;                // largest block size
  DevBuf<double> red_scratch;     // scratch of the min/max reductions
  DevBuf<uint64_t> acc_part;      // 192-bit partials of the exact sums
  DevBuf<int> acc_flags;          // largest exponent, non-finite flag
  DevBuf<int> diag_off;           // first onsite-diagonal slot of each primary atom
  DevBuf<double> diag_buf;        // gathered onsite diagonal (exact trace)
  uint64_t* host_res = nullptr;   // pinned host copy of the exact-sum results (4 words per sum)
  int64_t launches = 0;           // kernels launched by this system (all kinds)
  int mult_variant = -1;          // 4x4 FP64 product kernel: -1 = chosen per product by the autotuner,
                                  // 0 = one lane per element, 1 = one thread per block,
                                  // 2 = one thread per block with the operand row staged in shared memory,
                                  // 3 = one thread per block with warp-cooperative staging of the operand blocks,
                                  // 5 = four lanes per block, 6 = one thread per block with bulk-copy staging;
                                  // other block sizes: 0 = generic warp per block, 4 = warp per block with
                                  // 4 x 2 register tiles per lane
  bool blocking_sync = false;     // host waits sleep on a blocking-sync event instead of spinning
  // when set (batched serving), the chain's FP64 products go through this call instead of their own
  // launch: it joins them to the products of other systems in one persistent launch
  std::function<void(ProductPlan&, double*, const double*, double*, int)> batch_submit;
  cudaEvent_t sync_ev = nullptr;
  ProductProfile prof;
  ~System();
};

void init_device_pool();          // once per device: cache freed pool memory in the process
void host_wait(System& S);        // wait for all work enqueued on S.stream
constexpr int kPinnedWords = 4 * 32;
uint64_t* pinned_get();           // kPinnedWords of pinned host memory from a process-wide free list
void pinned_put(uint64_t* p);

// index.cu
void upload_geometry(System& S);
void build_range_index(System& S, RangeIndex& R);
ProductPlan& get_plan(System& S, int mult_type, int ra, int rb, int rc);
AddMap& get_addmap(System& S, int ra, int rb);
void export_range_array(System& S, int r, const std::string& name, std::vector<int64_t>& out);

MixedPlan& get_mixed_plan(System& S, int mult_type, int ra, int rb, int rc);

// mult.cu
void launch_mat_mult(System& S, ProductPlan& P, double* a, const double* b, double* c, int exact);
struct BatchItem {                 // one FP64 product of a batched launch (roles of launch_mat_mult)
  System* S;
  ProductPlan* P;
  double* a;
  const double* b;
  double* c;
  int exact;
};
void launch_mat_mult_batch(const std::vector<BatchItem>& items, cudaStream_t st);
void ensure_product_order(System& S, ProductPlan& P);   // the 4 x 4 kernels' output order (built once)

// gen.cu: synthetic S (which = 0) or H (which = 1) of range r into out
void generate_SH(System& S, int r, int which, uint64_t seed, double* out);

// mixed.cu
void to_fragments(System& S, int r, const double* src, int role_b, int trans, uint4* hi, uint4* lo, uint4* mid);
void launch_mult_tc(System& S, MixedPlan& MP, const uint4* xa_hi, const uint4* xa_lo, const uint4* bb_hi,
                    const uint4* bb_lo, double* out);
// split-precision mat_mult with the roles of launch_mat_mult: tcgen05 tiles where every block size is
// 4..128 (unless the system selects the per-block kernel), else the per-block mma.sync kernel
// `exact` argument of launch_mat_mult: 1 = the reference kernel's separate multiply and add, 0 = fused
// multiply-add, kPrecFp64Tensor = FP64 on the tensor cores (DMMA); the values of CQ_PREC_* in the C ABI
constexpr int kPrecFp64Tensor = 4;
// parts = 2: BF16x3 (tcgen05 tiles or mma.sync blocks by the fill rule); parts = 3: BF16x6 (mma.sync)
void mat_mult_mixed(System& S, int mult_type, int ra, int rb, int rc, double* a, const double* b, double* c,
                    int parts = 2);

// umma.cu
UmmaPlan& get_umma_plan(System& S, int mult_type, int ra, int rb, int rc);
bool umma_usable(System& S, int mult_type, int ra, int rb, int rc);
void mat_mult_umma(System& S, int mult_type, int ra, int rb, int rc, double* a, const double* b, double* c);
void umma_check(System& S);       // throws CQ_ERR_TIMEOUT if a kernel's bounded wait ran out
int* device_timeout_word(System& S);   // mapped host word the bounded waits of the system's kernels set
size_t umma_smem_bytes();

// algebra.cu
void dev_scale(System& S, double* a, int64_t n, double alpha);
void dev_axpy(System& S, double* a, int64_t n, double beta, const double* b);
// a = fl(alpha*a) + fl(beta*b) elementwise: dev_scale then dev_axpy in one pass, same bits
void dev_axpby(System& S, double* a, int64_t n, double alpha, double beta, const double* b);
void dev_copy(System& S, double* dst, const double* src, int64_t n);
void dev_matrix_add(System& S, int ra, double* a, double alpha, int rb, const double* b, double beta);
void dev_transpose(System& S, int r, const double* a, double* at);
double dev_dot(System& S, const double* x, const double* y, int64_t n);
// up to 32 exact dot products (y[k] may be null: plain sums), computed back to back and read
// with one host synchronisation
void dev_dots(System& S, int count, const double* const* x, const double* const* y, const int64_t* n, double* out);
// the same in two halves: enqueue the sums and the copy of their results to pinned host memory
// (no host synchronisation: can be captured in a CUDA graph), then wait and decode
void dev_dots_enqueue(System& S, int count, const double* const* x, const double* const* y, const int64_t* n);
void dev_dots_fetch(System& S, int count, double* out);
double dev_trace(System& S, int r, const double* a);
void dev_h_limits(System& S, int r, const double* h, double* hmin, double* hmax);
void dev_set_onsite_diag(System& S, int r, double* a, double value);   // diagonal of every self block

}  // namespace cqb
