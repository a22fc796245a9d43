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
#include "cq_internal.hpp"

namespace cqb {
namespace {

constexpr int kT = 256;
constexpr int kRedBlocks = 1184;   // 148 SMs x 8: fixed so the reduction order never changes

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
// deterministic dot product: fixed-grid partials, then one block sums them in order
__global__ void k_dot_partial(const double* __restrict__ x, const double* __restrict__ y, int64_t n, double* __restrict__ part) {
  __shared__ double s[kT];
  double acc = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x; i < n; i += (int64_t)gridDim.x * kT)
    acc = fma(x[i], y[i], acc);
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = kT / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}
__global__ void k_sum_final(const double* __restrict__ part, int n, double* __restrict__ out) {
  __shared__ double s[kT];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += kT) acc += part[i];
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = kT / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = s[0];
}
// onsite diagonal sum: sequential over primary atoms inside one block (n_prim is small)
__global__ void k_trace(int n_prim, const int64_t* __restrict__ onsite, const int* __restrict__ prim_nsf,
                        const double* __restrict__ a, double* __restrict__ out) {
  __shared__ double s[kT];
  double acc = 0.0;
  for (int p = threadIdx.x; p < n_prim; p += kT) {
    int nd = prim_nsf[p];
    const double* A = a + onsite[p];
    double t = 0.0;
    for (int j = 0; j < nd; ++j) t += A[j * nd + j];
    acc += t;
  }
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = kT / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = s[0];
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

double fetch_scalar(System& S, const double* d) {
  double h = 0.0;
  CQ_CUDA(cudaMemcpyAsync(&h, d, sizeof(double), cudaMemcpyDeviceToHost, S.stream));
  CQ_CUDA(cudaStreamSynchronize(S.stream));
  return h;
}

void ensure_scratch(System& S) {
  if (S.red_scratch.n < (size_t)kRedBlocks + 8) S.red_scratch.alloc(kRedBlocks + 8);
}

}  // namespace

void dev_scale(System& S, double* a, int64_t n, double alpha) {
  if (n <= 0) return;
  k_scale<<<grid_for(n), kT, 0, S.stream>>>(a, n, alpha);
  CQ_CUDA(cudaGetLastError());
}
void dev_axpy(System& S, double* a, int64_t n, double beta, const double* b) {
  if (n <= 0) return;
  k_axpy<<<grid_for(n), kT, 0, S.stream>>>(a, n, beta, b);
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
  CQ_CUDA(cudaGetLastError());
}
void dev_transpose(System& S, int r, const double* a, double* at) {
  RangeIndex& R = *S.ranges[r];
  CQ_CHECK(a != at, CQ_ERR_ARG, "transpose cannot run in place");
  if (R.nnz == 0) return;
  k_transpose<<<(int)(((int64_t)R.nnz * 32 + kT - 1) / kT), kT, 0, S.stream>>>(
      R.nnz, R.trans_dest.p, R.nb_elem.p, R.nb_row.p, R.nb_cover.p, S.dg.prim_nsf.p, S.dg.cover_nsf.p, a, at);
  CQ_CUDA(cudaGetLastError());
}
double dev_dot(System& S, const double* x, const double* y, int64_t n) {
  ensure_scratch(S);
  k_dot_partial<<<kRedBlocks, kT, 0, S.stream>>>(x, y, n, S.red_scratch.p);
  k_sum_final<<<1, kT, 0, S.stream>>>(S.red_scratch.p, kRedBlocks, S.red_scratch.p + kRedBlocks);
  CQ_CUDA(cudaGetLastError());
  return fetch_scalar(S, S.red_scratch.p + kRedBlocks);
}
double dev_trace(System& S, int r, const double* a) {
  ensure_scratch(S);
  RangeIndex& R = *S.ranges[r];
  k_trace<<<1, kT, 0, S.stream>>>(S.geo.n_prim, R.onsite.p, S.dg.prim_nsf.p, a, S.red_scratch.p + kRedBlocks);
  CQ_CUDA(cudaGetLastError());
  return fetch_scalar(S, S.red_scratch.p + kRedBlocks);
}
void dev_h_limits(System& S, int r, const double* h, double* hmin, double* hmax) {
  RangeIndex& R = *S.ranges[r];
  int N = S.geo.n_prim;
  DevBuf<double> mn, mx, out;
  mn.alloc(N); mx.alloc(N); out.alloc(2);
  k_hlimits<<<(N * 32 + kT - 1) / kT, kT, 0, S.stream>>>(N, R.row_ptr.p, R.nb_elem.p, R.nb_cover.p, R.onsite.p,
                                                       S.dg.prim_nsf.p, S.dg.cover_nsf.p, h, mn.p, mx.p);
  k_minmax<<<1, kT, 0, S.stream>>>(mn.p, mx.p, N, out.p);
  CQ_CUDA(cudaGetLastError());
  double o[2];
  CQ_CUDA(cudaMemcpyAsync(o, out.p, sizeof(o), cudaMemcpyDeviceToHost, S.stream));
  CQ_CUDA(cudaStreamSynchronize(S.stream));
  *hmin = o[0];
  *hmax = o[1];
}

}  // namespace cqb
