// Matrix algebra of the LNV chain on device-resident block matrices:
//   matrix_scale / matrix_sum (same range: scal + axpy, src/mult_module.f90:2677-2738)
//   matrix_add / addscan       (different ranges, src/multiply_module.f90:807-943):
//                               a = alpha*a + beta*b on the blocks both ranges store
//   matrix_transpose           (src/mult_module.f90:2609-2673 via the retro/transposed addresses)
//   matrix_trace / matrix_product_trace (src/mult_module.f90:2773-2916)
//   GetHLimits                 (src/McWeeny.f90:1020-1109)
// Elementwise kernels are HBM-bound grid-stride loops with 16-byte accesses;
// the reductions are two-level with a fixed grid, so results are identical
// from run to run.
#include <climits>
#include <functional>
#include <cmath>
#include <limits>

#include "cq_internal.hpp"

namespace cqb {
namespace {

constexpr int kT = 256;
constexpr int kRedBlocks = 1184;   // 148 SMs x 8: the largest grid of the exact sums

int grid_for(int64_t n) {
  int64_t b = (n + kT - 1) / kT;
  return (int)std::min<int64_t>(std::max<int64_t>(b, 1), 148 * 16);
}

__global__ void k_scale(double* __restrict__ a, int64_t n, double alpha) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    a[i] = __dmul_rn(a[i], alpha);
}
// a = a + fl(beta*b)  (daxpy with separate rounding of the product)
__global__ void k_axpy(double* __restrict__ a, int64_t n, double beta, const double* __restrict__ b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    a[i] = __dadd_rn(a[i], __dmul_rn(beta, b[i]));
}
// a = fl(fl(alpha*a) + fl(beta*b)): k_scale followed by k_axpy in one pass (same roundings);
// 16-byte accesses when both arrays are 16-byte aligned
__global__ void k_axpby(double* __restrict__ a, int64_t n, double alpha, double beta, const double* __restrict__ b,
                        int vec) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (vec) {
    double2* a2 = reinterpret_cast<double2*>(a);
    const double2* b2 = reinterpret_cast<const double2*>(b);
    for (int64_t i = i0; i < n / 2; i += stride) {
      double2 x = a2[i], y = b2[i];
      x.x = __dadd_rn(__dmul_rn(x.x, alpha), __dmul_rn(beta, y.x));
      x.y = __dadd_rn(__dmul_rn(x.y, alpha), __dmul_rn(beta, y.y));
      a2[i] = x;
    }
    if (i0 == 0 && (n & 1)) a[n - 1] = __dadd_rn(__dmul_rn(a[n - 1], alpha), __dmul_rn(beta, b[n - 1]));
  } else {
    for (int64_t i = i0; i < n; i += stride) a[i] = __dadd_rn(__dmul_rn(a[i], alpha), __dmul_rn(beta, b[i]));
  }
}
// matched blocks: a = fl(alpha*a) + fl(beta*b); unmatched blocks of a are left as they are
__global__ void k_masked_add(int nnz, const int* __restrict__ partner, const int64_t* __restrict__ a_elem,
                             const int64_t* __restrict__ b_elem, const int* __restrict__ row, const int* __restrict__ cover,
                             const int* __restrict__ prim_nsf, const int* __restrict__ cover_nsf, double* __restrict__ a,
                             double alpha, const double* __restrict__ b, double beta) {
  int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (e >= nnz) return;
  int pb = partner[e];
  if (pb < 0) return;
  int ne = prim_nsf[row[e]] * cover_nsf[cover[e]];
  double* A = a + a_elem[e];
  const double* B = b + b_elem[pb];
  for (int t = lane; t < ne; t += 32) A[t] = __dadd_rn(__dmul_rn(alpha, A[t]), __dmul_rn(beta, B[t]));
}
// AT(dest) = A(e)^T
__global__ void k_transpose(int nnz, const int* __restrict__ dest, const int64_t* __restrict__ elem,
                            const int* __restrict__ row, const int* __restrict__ cover, const int* __restrict__ prim_nsf,
                            const int* __restrict__ cover_nsf, const double* __restrict__ a, double* __restrict__ at) {
  int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (e >= nnz) return;
  int ndi = prim_nsf[row[e]], ndj = cover_nsf[cover[e]];
  const double* A = a + elem[e];
  double* T = at + elem[dest[e]];
  for (int t = lane; t < ndi * ndj; t += 32) {
    int n1 = t % ndi, n2 = t / ndi;
    T[n2 + ndj * n1] = A[t];
  }
}
// ---------------------------------------------------------------------------
// Exact, order-independent sums (matrix_product_trace / matrix_trace).
// Every term (a rounded product x*y, or an element) is converted exactly to a
// 192-bit two's-complement fixed-point integer whose least significant bit is
// 2^(emax-150), emax being the largest binary exponent among the terms (pass 1).
// Integer addition is associative, so the sum does not depend on the grid or on
// the order of the terms; the host rounds it once to the nearest double.
// Terms below 2^(emax-150) are truncated toward zero (relative effect < n 2^-150).
// ---------------------------------------------------------------------------
constexpr int kAccFrac = 150;   // fraction bits kept below the largest term's exponent
constexpr int kSumSlots = 32;   // exact sums fetched together by dev_dots
constexpr int kEBias = 2048;    // exponent bias of the pass-1 maximum (frexp exponents lie in [-1073, 1024])

struct Acc192 { uint64_t w[3]; };

__device__ __forceinline__ void acc_add(Acc192& a, const Acc192& b) {
  uint64_t s0 = a.w[0] + b.w[0];
  uint64_t c0 = s0 < a.w[0];
  uint64_t s1 = a.w[1] + b.w[1];
  uint64_t c1 = s1 < a.w[1];
  uint64_t s1c = s1 + c0;
  c1 += s1c < s1;
  a.w[0] = s0; a.w[1] = s1c; a.w[2] = a.w[2] + b.w[2] + c1;
}
// term v -> fixed point with lsb 2^lsb_exp (exact for every bit at or above the lsb)
__device__ __forceinline__ void acc_term(Acc192& a, double v, int lsb_exp) {
  if (v == 0.0) return;
  int e;
  double f = frexp(v, &e);                              // v = f 2^e, 0.5 <= |f| < 1
  long long m = (long long)ldexp(f, 53);                // exact, |m| < 2^53
  bool neg = m < 0;
  uint64_t mag = (uint64_t)(neg ? -m : m);
  int s = e - 53 - lsb_exp;                             // bit position of m's lsb
  Acc192 t = {{0, 0, 0}};
  if (s >= 0) {
    int idx = s >> 6, off = s & 63;
    if (idx < 3) t.w[idx] = mag << off;
    if (off && idx + 1 < 3) t.w[idx + 1] = mag >> (64 - off);
  } else if (-s < 64) {
    t.w[0] = mag >> (-s);
  }
  if (neg) {                                            // two's complement negation
    t.w[0] = ~t.w[0]; t.w[1] = ~t.w[1]; t.w[2] = ~t.w[2];
    Acc192 one = {{1, 0, 0}};
    acc_add(t, one);
  }
  acc_add(a, t);
}
__device__ __forceinline__ double dterm(const double* x, const double* y, int64_t i) {
  return y ? __dmul_rn(x[i], y[i]) : x[i];
}
// pass 1: largest exponent of the nonzero terms, stored biased by kEBias (0 = every term is zero);
// a non-finite term sets the flag.  Both words start at zero (cudaMemsetAsync).
__global__ void k_acc_emax(const double* __restrict__ x, const double* __restrict__ y, int64_t n, int* __restrict__ emax,
                           int* __restrict__ nonfinite) {
  int best = 0;
  bool bad = false;
  for (int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x; i < n; i += (int64_t)gridDim.x * kT) {
    double v = dterm(x, y, i);
    if (!isfinite(v)) { bad = true; continue; }
    if (v != 0.0) { int e; frexp(v, &e); best = max(best, e + kEBias); }
  }
  for (int o = 16; o; o >>= 1) best = max(best, __shfl_down_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0 && best != 0) atomicMax(emax, best);
  if (bad) atomicExch(nonfinite, 1);
}
__device__ void block_acc_reduce(Acc192 a, uint64_t* __restrict__ out) {
  __shared__ uint64_t s[3][kT];
  for (int k = 0; k < 3; ++k) s[k][threadIdx.x] = a.w[k];
  __syncthreads();
  for (int w = kT / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      Acc192 x = {{s[0][threadIdx.x], s[1][threadIdx.x], s[2][threadIdx.x]}};
      Acc192 z = {{s[0][threadIdx.x + w], s[1][threadIdx.x + w], s[2][threadIdx.x + w]}};
      acc_add(x, z);
      for (int k = 0; k < 3; ++k) s[k][threadIdx.x] = x.w[k];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) for (int k = 0; k < 3; ++k) out[k] = s[k][0];
}
// pass 2: fixed-point accumulation, one 192-bit partial per block (zero when pass 1 found no
// nonzero term or a non-finite one: the host reports 0 or NaN from the flags)
__global__ void __launch_bounds__(kT) k_acc_sum(const double* __restrict__ x, const double* __restrict__ y, int64_t n,
                                                const int* __restrict__ flags, uint64_t* __restrict__ part) {
  Acc192 a = {{0, 0, 0}};
  const int eb = flags[0];
  if (eb != 0 && flags[1] == 0) {
    const int lsb = eb - kEBias - kAccFrac;
    for (int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x; i < n; i += (int64_t)gridDim.x * kT)
      acc_term(a, dterm(x, y, i), lsb);
  }
  block_acc_reduce(a, part + 3 * blockIdx.x);
}
// pass 3: sum of the block partials into out[0..2]; out[3] carries the flags of pass 1
__global__ void __launch_bounds__(kT) k_acc_final(const uint64_t* __restrict__ part, int nb, const int* __restrict__ flags,
                                                  uint64_t* __restrict__ out) {
  Acc192 a = {{0, 0, 0}};
  for (int b = threadIdx.x; b < nb; b += kT) {
    Acc192 t = {{part[3 * b], part[3 * b + 1], part[3 * b + 2]}};
    acc_add(a, t);
  }
  block_acc_reduce(a, out);
  if (threadIdx.x == 0) out[3] = (uint64_t)(uint32_t)flags[0] | ((uint64_t)(uint32_t)flags[1] << 32);
}
// store_matrix_value(..., j, j, one) on every onsite block: the diagonal of each atom's self block
__global__ void k_set_onsite_diag(int n_prim, const int64_t* __restrict__ onsite, const int* __restrict__ prim_nsf,
                                  double value, double* __restrict__ a) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n_prim) return;
  const int nd = prim_nsf[p];
  for (int j = 0; j < nd; ++j) a[onsite[p] + j * nd + j] = value;
}
// onsite diagonal elements gathered for the exact trace
__global__ void k_gather_diag(int n_prim, const int64_t* __restrict__ onsite, const int* __restrict__ prim_nsf,
                              const int* __restrict__ diag_off, const double* __restrict__ a, double* __restrict__ out) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n_prim) return;
  int nd = prim_nsf[p];
  for (int j = 0; j < nd; ++j) out[diag_off[p] + j] = a[onsite[p] + j * nd + j];
}
// GetHLimits: per primary atom and column orbital i, HMin_i = sum(+-|H|), HMax_i = sum |H|
// (onsite block adds |H| to both); min/max over atoms are order independent.
__global__ void k_hlimits(int n_prim, const int* __restrict__ row_ptr, const int64_t* __restrict__ nb_elem,
                          const int* __restrict__ nb_cover, const int64_t* __restrict__ onsite,
                          const int* __restrict__ prim_nsf, const int* __restrict__ cover_nsf, const double* __restrict__ h,
                          double* __restrict__ hmin_atom, double* __restrict__ hmax_atom) {
  int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (p >= n_prim) return;
  const int nsfi = prim_nsf[p];
  double mn = 0.0, mx = 0.0;
  for (int e = row_ptr[p]; e < row_ptr[p + 1]; ++e) {
    int nsfj = cover_nsf[nb_cover[e]];
    const double* H = h + nb_elem[e];
    bool on = nb_elem[e] == onsite[p];
    if (lane < nsfj) {
      for (int j = 0; j < nsfi; ++j) {
        double v = fabs(H[j + nsfi * lane]);
        mn = on ? mn + v : mn - v;
        mx = mx + v;
      }
    }
  }
  double amn = 1.0e30, amx = -1.0e30;
  if (lane < nsfi) { amn = mn; amx = mx; }
  for (int o = 16; o; o >>= 1) {
    amn = fmin(amn, __shfl_down_sync(0xffffffffu, amn, o));
    amx = fmax(amx, __shfl_down_sync(0xffffffffu, amx, o));
  }
  if (lane == 0) { hmin_atom[p] = amn; hmax_atom[p] = amx; }
}
__global__ void k_minmax(const double* __restrict__ mn, const double* __restrict__ mx, int n, double* __restrict__ out) {
  __shared__ double smn[kT], smx[kT];
  double a = 1.0e30, b = -1.0e30;
  for (int i = threadIdx.x; i < n; i += kT) { a = fmin(a, mn[i]); b = fmax(b, mx[i]); }
  smn[threadIdx.x] = a; smx[threadIdx.x] = b;
  __syncthreads();
  for (int w = kT / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) { smn[threadIdx.x] = fmin(smn[threadIdx.x], smn[threadIdx.x + w]); smx[threadIdx.x] = fmax(smx[threadIdx.x], smx[threadIdx.x + w]); }
    __syncthreads();
  }
  if (threadIdx.x == 0) { out[0] = smn[0]; out[1] = smx[0]; }
}

}  // namespace

void dev_scale(System& S, double* a, int64_t n, double alpha) {
  if (n <= 0) return;
  k_scale<<<grid_for(n), kT, 0, S.stream>>>(a, n, alpha);
  S.launches++;
  CQ_CUDA(cudaGetLastError());
}
void dev_axpy(System& S, double* a, int64_t n, double beta, const double* b) {
  if (n <= 0) return;
  k_axpy<<<grid_for(n), kT, 0, S.stream>>>(a, n, beta, b);
  S.launches++;
  CQ_CUDA(cudaGetLastError());
}
void dev_axpby(System& S, double* a, int64_t n, double alpha, double beta, const double* b) {
  if (n <= 0) return;
  const int vec = ((uintptr_t)a % 16 == 0) && ((uintptr_t)b % 16 == 0);
  k_axpby<<<grid_for(vec ? (n + 1) / 2 : n), kT, 0, S.stream>>>(a, n, alpha, beta, b, vec);
  S.launches++;
  CQ_CUDA(cudaGetLastError());
}
void dev_copy(System& S, double* dst, const double* src, int64_t n) {
  if (n <= 0 || dst == src) return;
  CQ_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToDevice, S.stream));
}
void dev_matrix_add(System& S, int ra, double* a, double alpha, int rb, const double* b, double beta) {
  RangeIndex &A = *S.ranges[ra], &B = *S.ranges[rb];
  AddMap& m = get_addmap(S, ra, rb);
  if (A.nnz == 0) return;
  k_masked_add<<<(int)(((int64_t)A.nnz * 32 + kT - 1) / kT), kT, 0, S.stream>>>(
      A.nnz, m.partner.p, A.nb_elem.p, B.nb_elem.p, A.nb_row.p, A.nb_cover.p, S.dg.prim_nsf.p, S.dg.cover_nsf.p, a, alpha,
      b, beta);
  S.launches++;
  CQ_CUDA(cudaGetLastError());
}
void dev_transpose(System& S, int r, const double* a, double* at) {
  RangeIndex& R = *S.ranges[r];
  CQ_CHECK(a != at, CQ_ERR_ARG, "transpose cannot run in place");
  if (R.nnz == 0) return;
  k_transpose<<<(int)(((int64_t)R.nnz * 32 + kT - 1) / kT), kT, 0, S.stream>>>(
      R.nnz, R.trans_dest.p, R.nb_elem.p, R.nb_row.p, R.nb_cover.p, S.dg.prim_nsf.p, S.dg.cover_nsf.p, a, at);
  S.launches++;
  CQ_CUDA(cudaGetLastError());
}
// Round a 192-bit two's-complement fixed-point value (lsb = 2^lsb_exp) to the nearest double, ties to even.
double acc192_to_double(const uint64_t in[3], int lsb_exp) {
  uint64_t w[3] = {in[0], in[1], in[2]};
  bool neg = (w[2] >> 63) != 0;
  if (neg) {
    w[0] = ~w[0]; w[1] = ~w[1]; w[2] = ~w[2];
    if (++w[0] == 0 && ++w[1] == 0) ++w[2];
  }
  int h = -1;
  for (int k = 2; k >= 0 && h < 0; --k)
    if (w[k]) h = 64 * k + 63 - __builtin_clzll(w[k]);
  if (h < 0) return 0.0;
  auto bit = [&](int b) -> uint64_t { return b < 0 ? 0 : (w[b >> 6] >> (b & 63)) & 1u; };
  uint64_t m = 0;
  int sh = h > 52 ? h - 52 : 0;                  // bits dropped below the 53-bit mantissa
  for (int b = h; b >= sh; --b) m = (m << 1) | bit(b);
  if (sh > 0) {
    uint64_t half = bit(sh - 1), sticky = 0;
    for (int b = sh - 2; b >= 0 && !sticky; --b) sticky |= bit(b);
    if (half && (sticky || (m & 1))) ++m;         // may carry to 2^53, still exact in a double
  }
  double v = std::ldexp((double)m, lsb_exp + sh);
  return neg ? -v : v;
}

// Grid of the exact sums: integer accumulation is associative, so the grid only sets the
// parallelism (about four elements per thread, at most 148 SMs x 8 blocks).
static int acc_grid(int64_t n) {
  int64_t g = (n + 4 * kT - 1) / (4 * kT);
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, kRedBlocks));
}

// Enqueue the three passes; the 4-word result (3 fixed-point words, flags) lands in res.
static void exact_sum_enqueue(System& S, const double* x, const double* y, int64_t n, int* flags, uint64_t* part,
                              uint64_t* res) {
  const int g = acc_grid(n);
  CQ_CUDA(cudaMemsetAsync(flags, 0, 2 * sizeof(int), S.stream));
  k_acc_emax<<<g, kT, 0, S.stream>>>(x, y, n, flags, flags + 1);
  k_acc_sum<<<g, kT, 0, S.stream>>>(x, y, n, flags, part);
  k_acc_final<<<1, kT, 0, S.stream>>>(part, g, flags, res);
  S.launches += 3;
  CQ_CUDA(cudaGetLastError());
}

// Value of a 4-word exact-sum result (k_acc_final layout).
static double exact_sum_value(const uint64_t r[4]) {
  const int eb = (int)(uint32_t)(r[3] & 0xffffffffu);
  if ((r[3] >> 32) != 0) return std::numeric_limits<double>::quiet_NaN();
  if (eb == 0) return 0.0;
  return acc192_to_double(r, eb - kEBias - kAccFrac);
}

// Scratch of the exact sums: the block partials of the sum being computed (the three passes of
// one sum run back to back on the stream, so consecutive sums share them), then one 4-word
// result per slot; two flag words per slot.
static void acc_scratch(System& S) {
  if (S.acc_part.n < (size_t)(3 * kRedBlocks + 4 * kSumSlots)) S.acc_part.alloc(3 * kRedBlocks + 4 * kSumSlots, S.stream);
  if (S.acc_flags.n < (size_t)(2 * kSumSlots)) S.acc_flags.alloc(2 * kSumSlots, S.stream);
}

static double exact_sum(System& S, const double* x, const double* y, int64_t n) {
  acc_scratch(S);
  exact_sum_enqueue(S, x, y, n, S.acc_flags.p, S.acc_part.p, S.acc_part.p + 3 * kRedBlocks);
  uint64_t w[4];
  CQ_CUDA(cudaMemcpyAsync(w, S.acc_part.p + 3 * kRedBlocks, sizeof(w), cudaMemcpyDeviceToHost, S.stream));
  host_wait(S);
  return exact_sum_value(w);
}

void dev_dots_enqueue(System& S, int count, const double* const* x, const double* const* y, const int64_t* n) {
  CQ_CHECK(count >= 0 && count <= kSumSlots, CQ_ERR_ARG, "too many sums in one batch");
  if (count == 0) return;
  acc_scratch(S);
  static_assert(4 * kSumSlots <= kPinnedWords, "pinned result buffer too small");
  if (!S.host_res) S.host_res = pinned_get();
  uint64_t* res = S.acc_part.p + 3 * kRedBlocks;
  for (int k = 0; k < count; ++k) exact_sum_enqueue(S, x[k], y[k], n[k], S.acc_flags.p + 2 * k, S.acc_part.p, res + 4 * k);
  CQ_CUDA(cudaMemcpyAsync(S.host_res, res, sizeof(uint64_t) * 4 * count, cudaMemcpyDeviceToHost, S.stream));
}

void dev_dots_fetch(System& S, int count, double* out) {
  if (count == 0) return;
  host_wait(S);
  for (int k = 0; k < count; ++k) out[k] = exact_sum_value(&S.host_res[4 * k]);
}

void dev_dots(System& S, int count, const double* const* x, const double* const* y, const int64_t* n, double* out) {
  dev_dots_enqueue(S, count, x, y, n);
  dev_dots_fetch(S, count, out);
}

double dev_dot(System& S, const double* x, const double* y, int64_t n) { return exact_sum(S, x, y, n); }

double dev_trace(System& S, int r, const double* a) {
  RangeIndex& R = *S.ranges[r];
  const int N = S.geo.n_prim;
  if (S.diag_off.n == 0) {
    std::vector<int> off(N + 1, 0);
    for (int p = 0; p < N; ++p) off[p + 1] = off[p] + S.geo.nsf[S.geo.prim_global[p]];
    S.diag_off.upload(off, S.stream);
    S.diag_buf.alloc(std::max(off[N], 1), S.stream);
  }
  k_gather_diag<<<(N + kT - 1) / kT, kT, 0, S.stream>>>(N, R.onsite.p, S.dg.prim_nsf.p, S.diag_off.p, a, S.diag_buf.p);
  S.launches++;
  CQ_CUDA(cudaGetLastError());
  return exact_sum(S, S.diag_buf.p, nullptr, (int64_t)S.diag_buf.n);
}
void dev_set_onsite_diag(System& S, int r, double* a, double value) {
  RangeIndex& R = *S.ranges[r];
  const int N = S.geo.n_prim;
  if (N == 0) return;
  k_set_onsite_diag<<<(N + kT - 1) / kT, kT, 0, S.stream>>>(N, R.onsite.p, S.dg.prim_nsf.p, value, a);
  S.launches++;
  CQ_CUDA(cudaGetLastError());
}
void dev_h_limits(System& S, int r, const double* h, double* hmin, double* hmax) {
  RangeIndex& R = *S.ranges[r];
  int N = S.geo.n_prim;
  DevBuf<double> mn, mx, out;
  mn.alloc(N, S.stream); mx.alloc(N, S.stream); out.alloc(2, S.stream);
  k_hlimits<<<(N * 32 + kT - 1) / kT, kT, 0, S.stream>>>(N, R.row_ptr.p, R.nb_elem.p, R.nb_cover.p, R.onsite.p,
                                                       S.dg.prim_nsf.p, S.dg.cover_nsf.p, h, mn.p, mx.p);
  k_minmax<<<1, kT, 0, S.stream>>>(mn.p, mx.p, N, out.p);
  S.launches += 2;
  CQ_CUDA(cudaGetLastError());
  double o[2];
  CQ_CUDA(cudaMemcpyAsync(o, out.p, sizeof(o), cudaMemcpyDeviceToHost, S.stream));
  host_wait(S);
  *hmin = o[0];
  *hmax = o[1];
}

// ---------------------------------------------------------------------------
// Exact dot products without any device allocation (cq_exact_dots_noalloc).
//
// Some callers cannot allocate device memory at the moment they need a trace: a Fortran/MPI
// host that has given the whole device to its own memory pool, or a latency-critical loop that
// must not take the device-wide synchronisation cudaMalloc and cudaFree can imply.  This entry
// point runs the same three kernels as the library's traces, with their scratch (block
// partials, results and flags) in one static device array instead of library-allocated memory.
// Every call uses that same array, so calls that overlap on the GPU (from two streams or two
// threads) race on it.
// ---------------------------------------------------------------------------
namespace {
constexpr int kNoAllocSums = CQ_NOALLOC_MAX_SUMS;
// words: block partials of one sum | 4-word result per sum | 2 int flags per sum (one word)
constexpr int kNoAllocWords = 3 * kRedBlocks + 4 * kNoAllocSums + kNoAllocSums;
static __device__ __align__(256) uint64_t g_noalloc_scratch[kNoAllocWords];   // 28.7 KiB per device

// Device address of the static scratch on the current device.  The host-side name of the array
// is not a device address, so it is looked up with cudaGetSymbolAddress on every call (cheap, and
// it allocates nothing): a cached address would go stale if the host tore the context down
// (cudaDeviceReset) between calls.
uint64_t* noalloc_scratch() {
  void* p = nullptr;
  CQ_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
  return static_cast<uint64_t*>(p);
}
}  // namespace

int guarded_call(const std::function<void()>& f);   // capi.cpp: exceptions to status codes

}  // namespace cqb

extern "C" int cq_exact_dots_noalloc(int count, const double* const* x_dev, const double* const* y_dev,
                                     const int64_t* n, void* stream, double* out) {
  using namespace cqb;
  return guarded_call([&] {
    CQ_CHECK(x_dev && n && out, CQ_ERR_ARG, "null argument");
    CQ_CHECK(count >= 1 && count <= kNoAllocSums, CQ_ERR_ARG,
             "cq_exact_dots_noalloc: count must be 1..CQ_NOALLOC_MAX_SUMS (8) sums per call");
    for (int k = 0; k < count; ++k) CQ_CHECK(n[k] >= 0 && (x_dev[k] || n[k] == 0), CQ_ERR_ARG, "bad operand");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint64_t* base = noalloc_scratch();
    uint64_t* part = base;
    uint64_t* res = base + 3 * kRedBlocks;
    int* flags = reinterpret_cast<int*>(base + 3 * kRedBlocks + 4 * kNoAllocSums);
    // the pass-1 flags (largest exponent, non-finite) start at zero; the partials and results
    // are overwritten by every call
    CQ_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * 2 * count, st));
    for (int k = 0; k < count; ++k) {
      const double* x = x_dev[k];
      const double* y = y_dev ? y_dev[k] : nullptr;
      const int g = acc_grid(n[k]);
      k_acc_emax<<<g, kT, 0, st>>>(x, y, n[k], flags + 2 * k, flags + 2 * k + 1);
      k_acc_sum<<<g, kT, 0, st>>>(x, y, n[k], flags + 2 * k, part);
      k_acc_final<<<1, kT, 0, st>>>(part, g, flags + 2 * k, res + 4 * k);
    }
    CQ_CUDA(cudaGetLastError());
    uint64_t w[4 * kNoAllocSums];
    CQ_CUDA(cudaMemcpyAsync(w, res, sizeof(uint64_t) * 4 * count, cudaMemcpyDeviceToHost, st));
    CQ_CUDA(cudaStreamSynchronize(st));
    for (int k = 0; k < count; ++k) out[k] = exact_sum_value(&w[4 * k]);
  });
}

