// GPU construction of the matrix index of every range and of the per-product
// pair lists.  Integer and comparison work only: warps scan the covering set
// in 32-atom chunks, vote with __ballot_sync and compact with population
// counts, so every list comes out in the reference's order:
//   get_naba      src/matrix_elements_module.f90:257-384  (neighbours, covering-set order)
//   make_npxyz    src/matrix_elements_module.f90:836-903  (partition displacement code)
//   make_halo     src/matrix_elements_module.f90:593-716  (halo numbering, i_h2d)
//   get_retr      src/matrix_elements_module.f90:517-557  (primary atoms of each halo atom)
//   a_and_b / index_transpose  src/trans_module.f90:72-330 (global transpose addresses)
//   m_kern_max / m_kern_min loop nests, src/multiply_kernel_default.f90:169-221, 361-410
//     (the (k, i, j) triples of a product, grouped per output block in summation order)
#include <cub/block/block_scan.cuh>

#include <algorithm>
#include <numeric>

#include "cq_internal.hpp"

namespace cqb {

namespace {

constexpr double kRdErr = 1.0e-8;  // RD_ERR (numbers_module.f90:96)
constexpr int kWarp = 32;

// distance test of get_naba with the reference's operation order and rounding
__device__ __forceinline__ bool within(const double* xc, const double* xp, double thr, double* d2out) {
  double dx = __dsub_rn(xc[0], xp[0]);
  double dy = __dsub_rn(xc[1], xp[1]);
  double dz = __dsub_rn(xc[2], xp[2]);
  double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  if (d2out) *d2out = d2;
  return d2 < thr;
}

// ---------------------------------------------------------------------------
// neighbour lists: one warp per primary atom, covering set scanned in order
// ---------------------------------------------------------------------------
__global__ void k_naba_count(int n_prim, int n_cover, const double* __restrict__ prim_x, const double* __restrict__ cover_x,
                             const int* __restrict__ prim_nsf, const int* __restrict__ cover_nsf, double thr,
                             int* __restrict__ row_cnt, int64_t* __restrict__ row_len) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) / kWarp, lane = threadIdx.x % kWarp;
  if (warp >= n_prim) return;
  const double* xp = prim_x + 3 * (size_t)warp;
  int cnt = 0;
  int64_t len = 0;
  for (int base = 0; base < n_cover; base += kWarp) {
    int c = base + lane;
    bool in = c < n_cover && within(cover_x + 3 * (size_t)c, xp, thr, nullptr);
    unsigned m = __ballot_sync(0xffffffffu, in);
    cnt += __popc(m);
    if (in) len += cover_nsf[c];
  }
  for (int o = 16; o; o >>= 1) len += __shfl_down_sync(0xffffffffu, len, o);
  if (lane == 0) { row_cnt[warp] = cnt; row_len[warp] = len * prim_nsf[warp]; }
}

__global__ void k_naba_fill(int n_prim, int n_cover, const double* __restrict__ prim_x, const double* __restrict__ cover_x,
                            const int* __restrict__ prim_nsf, const int* __restrict__ cover_nsf,
                            const int* __restrict__ cover_part, const int* __restrict__ cover_seq,
                            const int* __restrict__ cover_label_of_part, const int* __restrict__ prim_cover_label,
                            const int* __restrict__ prim_seq, const int* __restrict__ prim_part,
                            const int* __restrict__ part_disp, int ncy, int ncz, int spx, int spy, int spz, double thr,
                            const int* __restrict__ row_ptr, const int64_t* __restrict__ row_elem,
                            int* __restrict__ nb_cover, int64_t* __restrict__ nb_elem, int* __restrict__ nb_row,
                            int* __restrict__ nb_ibpart, double* __restrict__ nb_radius, int64_t* __restrict__ onsite) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) / kWarp, lane = threadIdx.x % kWarp;
  if (warp >= n_prim) return;
  const int p = warp;
  const double* xp = prim_x + 3 * (size_t)p;
  const int ndi = prim_nsf[p];
  const int* dsp = part_disp + 3 * prim_part[p];
  int pos = row_ptr[p];
  int64_t elem = row_elem[p];
  const unsigned lt = (1u << lane) - 1u;
  for (int base = 0; base < n_cover; base += kWarp) {
    int c = base + lane;
    double d2 = 0.0;
    bool in = c < n_cover && within(cover_x + 3 * (size_t)c, xp, thr, &d2);
    unsigned m = __ballot_sync(0xffffffffu, in);
    if (!m) continue;
    int sz = in ? ndi * cover_nsf[c] : 0;
    int incl = sz;  // inclusive warp scan of block sizes
    for (int o = 1; o < kWarp; o <<= 1) {
      int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    int total = __shfl_sync(0xffffffffu, incl, kWarp - 1);
    if (in) {
      int e = pos + __popc(m & lt);
      int64_t off = elem + (incl - sz);
      nb_cover[e] = c;
      nb_elem[e] = off;
      nb_row[e] = p;
      nb_radius[e] = __dsqrt_rn(d2);
      int lab = cover_label_of_part[cover_part[c]];
      if (lab == prim_cover_label[p] && cover_seq[c] == prim_seq[p]) onsite[p] = off;
      // make_npxyz: displacement of the neighbour's partition from the row's partition
      int l0 = lab - 1;
      int nx = l0 / (ncy * ncz), ny = (l0 - nx * ncy * ncz) / ncz, nz = l0 - nx * ncy * ncz - ny * ncz;
      int npx = nx - spx - dsp[0], npy = ny - spy - dsp[1], npz = nz - spz - dsp[2];
      nb_ibpart[e] = npx * ncy * ncz + npy * ncz + npz;
    }
    pos += __popc(m);
    elem += total;
  }
}

// ---------------------------------------------------------------------------
// halo numbering and retro lists
// ---------------------------------------------------------------------------
__global__ void k_flag(int nnz, const int* __restrict__ nb_cover, int* __restrict__ flag) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < nnz) flag[nb_cover[e]] = 1;
}
__global__ void k_halo_number(int n_cover, const int* __restrict__ flag, const int* __restrict__ excl,
                              int* __restrict__ cover_to_halo, int* __restrict__ halo_cover) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cover) return;
  if (flag[c]) { cover_to_halo[c] = excl[c]; halo_cover[excl[c]] = c; }
  else cover_to_halo[c] = -1;
}
__global__ void k_gather_int(int n, const int* __restrict__ idx, const int* __restrict__ table, int* __restrict__ out) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) out[e] = table[idx[e]];
}

// first entry of row p whose cover atom equals c (rows are sorted by cover atom), or -1
__device__ __forceinline__ int find_in_row(const int* __restrict__ row_ptr, const int* __restrict__ nb_cover, int p, int c) {
  int lo = row_ptr[p], hi = row_ptr[p + 1] - 1;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    int v = nb_cover[mid];
    if (v == c) return mid;
    if (v < c) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

// retro lists: one warp per halo atom, primary atoms scanned in order with the get_naba test
__global__ void k_retr_count(int nh, int n_prim, const int* __restrict__ halo_cover, const double* __restrict__ cover_x,
                             const double* __restrict__ prim_x, double thr, int* __restrict__ col_cnt) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) / kWarp, lane = threadIdx.x % kWarp;
  if (warp >= nh) return;
  const double* xc = cover_x + 3 * (size_t)halo_cover[warp];
  int cnt = 0;
  for (int base = 0; base < n_prim; base += kWarp) {
    int p = base + lane;
    bool in = p < n_prim && within(xc, prim_x + 3 * (size_t)p, thr, nullptr);
    cnt += __popc(__ballot_sync(0xffffffffu, in));
  }
  if (lane == 0) col_cnt[warp] = cnt;
}
__global__ void k_retr_fill(int nh, int n_prim, const int* __restrict__ halo_cover, const double* __restrict__ cover_x,
                            const double* __restrict__ prim_x, double thr, const int* __restrict__ col_ptr,
                            const int* __restrict__ row_ptr, const int* __restrict__ nb_cover, int* __restrict__ col_row,
                            int* __restrict__ col_blk, int* __restrict__ err) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) / kWarp, lane = threadIdx.x % kWarp;
  if (warp >= nh) return;
  int c = halo_cover[warp];
  const double* xc = cover_x + 3 * (size_t)c;
  int pos = col_ptr[warp];
  const unsigned lt = (1u << lane) - 1u;
  for (int base = 0; base < n_prim; base += kWarp) {
    int p = base + lane;
    bool in = p < n_prim && within(xc, prim_x + 3 * (size_t)p, thr, nullptr);
    unsigned m = __ballot_sync(0xffffffffu, in);
    if (in) {
      int e = pos + __popc(m & lt);
      int b = find_in_row(row_ptr, nb_cover, p, c);
      if (b < 0) atomicExch(err, 1);
      col_row[e] = p;
      col_blk[e] = b;
    }
    pos += __popc(m);
  }
}

// global transpose: block (p, c) -> block (home(c), image of p seen from home(c))
__global__ void k_trans_dest(int nnz, const int* __restrict__ nb_row, const int* __restrict__ nb_cover,
                             const int* __restrict__ cover_part, const int* __restrict__ cover_label_of_part,
                             const int* __restrict__ cover_home_prim, const int* __restrict__ prim_cover_label,
                             const int* __restrict__ prim_seq, const int* __restrict__ label_to_cover,
                             const int* __restrict__ cover_first, const int* __restrict__ row_ptr, int ncy, int ncz,
                             int ng_cover, int* __restrict__ dest, int* __restrict__ err) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nnz) return;
  int p = nb_row[e], c = nb_cover[e];
  int yz = ncy * ncz;
  auto xyz = [&](int lab, int& x, int& y, int& z) { int l = lab - 1; x = l / yz; y = (l - x * yz) / ncz; z = l - x * yz - y * ncz; };
  int ax, ay, az, bx, by, bz, hx, hy, hz;
  xyz(cover_label_of_part[cover_part[c]], ax, ay, az);   // partition of the neighbour image
  xyz(prim_cover_label[p], bx, by, bz);                   // partition of the row atom
  int jh = cover_home_prim[c];
  xyz(prim_cover_label[jh], hx, hy, hz);                  // home partition of the neighbour
  int lab = (hx + bx - ax) * yz + (hy + by - ay) * ncz + (hz + bz - az) + 1;
  int d = -1;
  if (lab >= 1 && lab <= ng_cover) {
    int np_ = label_to_cover[lab];
    if (np_ >= 0) d = find_in_row(row_ptr, nb_cover, jh, cover_first[np_] + prim_seq[p] - 1);
  }
  if (d < 0) atomicExch(err, 1);
  dest[e] = d;
}

// ---------------------------------------------------------------------------
// per-product pair lists
// ---------------------------------------------------------------------------
struct PlanArgs {
  // ranges: a (A or type-2 output), b, c (C or type-2 input)
  const int *a_row_ptr, *a_cover, *a_row;
  const int *b_row_ptr, *b_cover, *b_ibpart;
  const int *c_row_ptr, *c_cover;
  const int *cover_part, *cover_label_of_part, *cover_home_prim, *label_to_cover, *cover_first, *cover_seq, *cover_nsf,
      *prim_nsf;
  int ng_cover;
};

// cover atom of the j-th B neighbour of halo atom k, translated into the frame of k's image
__device__ __forceinline__ int translate_j(const PlanArgs& A, int k_label, int eb, int* err) {
  int lab = k_label + A.b_ibpart[eb];
  if (lab < 1 || lab > A.ng_cover) { atomicExch(err, 1); return -1; }
  int np_ = A.label_to_cover[lab];
  if (np_ < 0) { atomicExch(err, 1); return -1; }
  return A.cover_first[np_] + A.cover_seq[A.b_cover[eb]] - 1;
}

// type 1: one warp per C row p; A neighbours k of p in order, B neighbours j of k across lanes.
// pass 0 counts pairs per C block, pass 1 writes them at ptr[c] + cursor[c].
__global__ void k_plan1(PlanArgs A, int n_prim, int pass, int* __restrict__ cnt, const int64_t* __restrict__ ptr,
                        int* __restrict__ cursor, int2* __restrict__ pairs, unsigned long long* __restrict__ flops,
                        int* __restrict__ err) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) / kWarp, lane = threadIdx.x % kWarp;
  if (warp >= n_prim) return;
  const int p = warp;
  const int ndi = A.prim_nsf[p];
  unsigned long long fl = 0;
  for (int ea = A.a_row_ptr[p]; ea < A.a_row_ptr[p + 1]; ++ea) {
    int k = A.a_cover[ea];
    int kh = A.cover_home_prim[k];
    int klab = A.cover_label_of_part[A.cover_part[k]];
    int ndk = A.cover_nsf[k];
    for (int eb0 = A.b_row_ptr[kh]; eb0 < A.b_row_ptr[kh + 1]; eb0 += kWarp) {
      int eb = eb0 + lane;
      if (eb < A.b_row_ptr[kh + 1]) {
        int cj = translate_j(A, klab, eb, err);
        int cb = cj >= 0 ? find_in_row(A.c_row_ptr, A.c_cover, p, cj) : -1;
        if (cb >= 0) {
          if (pass == 0) {
            cnt[cb] += 1;  // distinct C blocks within one k step; steps are ordered by __syncwarp
            fl += 2ull * ndi * ndk * A.cover_nsf[cj];
          } else {
            int s = cursor[cb];
            cursor[cb] = s + 1;
            pairs[ptr[cb] + s] = make_int2(ea, eb);
          }
        }
      }
    }
    __syncwarp();
  }
  if (pass == 0) {
    for (int o = 16; o; o >>= 1) fl += __shfl_down_sync(0xffffffffu, fl, o);
    if (lane == 0 && fl) atomicAdd(flops, fl);
  }
}

// type 2: one warp per output block (p, k); B neighbours j of k in order, looked up in row p of the input.
__global__ void k_plan2(PlanArgs A, int nnz_out, int pass, int* __restrict__ cnt, const int64_t* __restrict__ ptr,
                        int2* __restrict__ pairs, unsigned long long* __restrict__ flops, int* __restrict__ err) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) / kWarp, lane = threadIdx.x % kWarp;
  if (warp >= nnz_out) return;
  const int eo = warp;
  const int p = A.a_row[eo];
  const int k = A.a_cover[eo];
  const int kh = A.cover_home_prim[k];
  const int klab = A.cover_label_of_part[A.cover_part[k]];
  const int ndi = A.prim_nsf[p], ndk = A.cover_nsf[k];
  const unsigned lt = (1u << lane) - 1u;
  int n = 0;
  unsigned long long fl = 0;
  int64_t base_out = pass ? ptr[eo] : 0;
  for (int eb0 = A.b_row_ptr[kh]; eb0 < A.b_row_ptr[kh + 1]; eb0 += kWarp) {
    int eb = eb0 + lane;
    int xb = -1, cj = -1;
    if (eb < A.b_row_ptr[kh + 1]) {
      cj = translate_j(A, klab, eb, err);
      xb = cj >= 0 ? find_in_row(A.c_row_ptr, A.c_cover, p, cj) : -1;
    }
    unsigned m = __ballot_sync(0xffffffffu, xb >= 0);
    if (xb >= 0) {
      if (pass == 1) pairs[base_out + n + __popc(m & lt)] = make_int2(xb, eb);
      else fl += 2ull * ndi * ndk * A.cover_nsf[cj];
    }
    n += __popc(m);
  }
  if (pass == 0) {
    for (int o = 16; o; o >>= 1) fl += __shfl_down_sync(0xffffffffu, fl, o);
    if (lane == 0) { cnt[eo] = n; if (fl) atomicAdd(flops, fl); }
  }
}

// type 2, lists ordered by the input block: one warp per output block (p, k); lanes walk row p of
// the input c, map each neighbour j back into the frame of k's home atom and look it up in B's row.
// Label of j in kh's frame = label(j in p's frame) - label(k's partition) + label(kh's home partition).
__global__ void k_plan2x(PlanArgs A, int nnz_out, int pass, const int* __restrict__ prim_cover_label, int ncx, int ncy,
                         int ncz, int* __restrict__ cnt, const int64_t* __restrict__ ptr, int2* __restrict__ pairs) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) / kWarp, lane = threadIdx.x % kWarp;
  if (warp >= nnz_out) return;
  const int eo = warp;
  const int p = A.a_row[eo];
  const int k = A.a_cover[eo];
  const int kh = A.cover_home_prim[k];
  const int yz = ncy * ncz;
  auto xyz = [&](int lab, int& x, int& y, int& z) { int l = lab - 1; x = l / yz; y = (l - x * yz) / ncz; z = l - x * yz - y * ncz; };
  int kx, ky, kz, hx, hy, hz;
  xyz(A.cover_label_of_part[A.cover_part[k]], kx, ky, kz);
  xyz(prim_cover_label[kh], hx, hy, hz);
  const unsigned lt = (1u << lane) - 1u;
  int n = 0;
  int64_t base = pass ? ptr[eo] : 0;
  for (int ex0 = A.c_row_ptr[p]; ex0 < A.c_row_ptr[p + 1]; ex0 += kWarp) {
    int ex = ex0 + lane, eb = -1;
    if (ex < A.c_row_ptr[p + 1]) {
      int c = A.c_cover[ex];
      int cx, cy, cz;
      xyz(A.cover_label_of_part[A.cover_part[c]], cx, cy, cz);
      int tx = cx - kx + hx, ty = cy - ky + hy, tz = cz - kz + hz;
      if (tx >= 0 && tx < ncx && ty >= 0 && ty < ncy && tz >= 0 && tz < ncz) {
        int np_ = A.label_to_cover[tx * yz + ty * ncz + tz + 1];
        if (np_ >= 0) eb = find_in_row(A.b_row_ptr, A.b_cover, kh, A.cover_first[np_] + A.cover_seq[c] - 1);
      }
    }
    unsigned m = __ballot_sync(0xffffffffu, eb >= 0);
    if (pass == 1 && eb >= 0) pairs[base + n + __popc(m & lt)] = make_int2(ex, eb);
    n += __popc(m);
  }
  if (pass == 0 && lane == 0) cnt[eo] = n;
}

// partner block of each block of range A in range B (same row, same cover atom), or -1
__global__ void k_addmap(int nnz, const int* __restrict__ a_row, const int* __restrict__ a_cover,
                         const int* __restrict__ b_row_ptr, const int* __restrict__ b_cover, int* __restrict__ partner) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < nnz) partner[e] = find_in_row(b_row_ptr, b_cover, a_row[e], a_cover[e]);
}

// ---------------------------------------------------------------------------
// exclusive scan (three phases, deterministic), int -> int64
// ---------------------------------------------------------------------------
template <class Tin>
__global__ void __launch_bounds__(256) k_scan_blocks(const Tin* __restrict__ in, int64_t n, int64_t* __restrict__ out, int64_t* __restrict__ block_sums) {
  typedef cub::BlockScan<int64_t, 256> Scan;
  __shared__ typename Scan::TempStorage tmp;
  int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
  int64_t v = i < n ? (int64_t)in[i] : 0, excl, agg;
  Scan(tmp).ExclusiveSum(v, excl, agg);
  if (i < n) out[i] = excl;
  if (threadIdx.x == 0) block_sums[blockIdx.x] = agg;
}
__global__ void __launch_bounds__(1024) k_scan_sums(int64_t* __restrict__ s, int nb, int64_t* __restrict__ total) {
  typedef cub::BlockScan<int64_t, 1024> Scan;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ int64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += 1024) {
    int i = base + threadIdx.x;
    int64_t v = i < nb ? s[i] : 0, excl, agg;
    Scan(tmp).ExclusiveSum(v, excl, agg);
    if (i < nb) s[i] = excl + carry;
    __syncthreads();
    if (threadIdx.x == 0) carry += agg;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}
__global__ void k_scan_add(int64_t* __restrict__ out, int64_t n, const int64_t* __restrict__ s) {
  int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (i < n) out[i] += s[blockIdx.x];
}

// exclusive scan of n values into out[0..n]; out[n] = total.  Returns the total (synchronises).
template <class Tin>
int64_t exclusive_scan(const Tin* in, int64_t n, int64_t* out, cudaStream_t st) {
  int nb = (int)std::max<int64_t>(1, (n + 255) / 256);
  DevBuf<int64_t> sums;
  sums.alloc(nb + 1, st);
  if (n > 0) k_scan_blocks<Tin><<<nb, 256, 0, st>>>(in, n, out, sums.p);
  else CQ_CUDA(cudaMemsetAsync(sums.p, 0, sizeof(int64_t), st));
  k_scan_sums<<<1, 1024, 0, st>>>(sums.p, n > 0 ? nb : 0, out + n);
  if (n > 0) k_scan_add<<<nb, 256, 0, st>>>(out, n, sums.p);
  CQ_CUDA(cudaGetLastError());
  int64_t total = 0;
  CQ_CUDA(cudaMemcpyAsync(&total, out + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  CQ_CUDA(cudaStreamSynchronize(st));
  return total;
}

__global__ void k_i64_to_i32(const int64_t* __restrict__ in, int n, int* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (int)in[i];
}

inline int nblk(int64_t n, int t) { return (int)((n + t - 1) / t); }

int read_flag(int* d, cudaStream_t st) {
  int h = 0;
  CQ_CUDA(cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, st));
  CQ_CUDA(cudaStreamSynchronize(st));
  return h;
}

}  // namespace

void upload_geometry(System& S) {
  Geometry& g = S.geo;
  DevGeometry& d = S.dg;
  cudaStream_t st = S.stream;
  std::vector<int> prim_nsf(g.n_prim);
  for (int p = 0; p < g.n_prim; ++p) prim_nsf[p] = g.nsf[g.prim_global[p]];
  d.prim_x.upload(g.prim_x, st);
  d.cover_x.upload(g.cover_x, st);
  d.prim_nsf.upload(prim_nsf, st);
  d.prim_cover_label.upload(g.prim_cover_label, st);
  d.prim_seq.upload(g.prim_seq, st);
  d.prim_part.upload(g.prim_part, st);
  d.part_disp.upload(g.part_disp, st);
  d.cover_nsf.upload(g.cover_nsf, st);
  d.cover_part.upload(g.cover_part, st);
  d.cover_seq.upload(g.cover_seq, st);
  d.cover_label_of_part.upload(g.cover_label, st);
  d.label_to_cover.upload(g.label_to_cover, st);
  d.cover_first.upload(g.cover_first, st);
  d.cover_home_prim.upload(g.cover_home_prim, st);
  d.part_first_prim.upload(g.part_first_prim, st);
  int u = g.nsf.empty() ? 0 : g.nsf[0];
  for (int v : g.nsf) if (v != u) { u = 0; break; }
  S.uniform_nsf = u;
  S.max_nsf = 0;
  for (int v : g.nsf) S.max_nsf = std::max(S.max_nsf, v);
}

void build_range_index(System& S, RangeIndex& R) {
  Geometry& g = S.geo;
  DevGeometry& d = S.dg;
  cudaStream_t st = S.stream;
  const int N = g.n_prim, NC = g.n_cover_atoms;
  volatile double rcutsq = R.rcut * R.rcut;       // rounded product, then the difference, as in the reference
  const double thr = rcutsq - kRdErr;
  const int T = 256, WPB = T / kWarp;
  // ---- neighbour counts and offsets
  DevBuf<int> row_cnt;
  row_cnt.alloc(N, st);
  DevBuf<int64_t> row_len, ptr64;
  row_len.alloc(N, st);
  ptr64.alloc(N + 1, st);
  k_naba_count<<<nblk(N, WPB), T, 0, st>>>(N, NC, d.prim_x.p, d.cover_x.p, d.prim_nsf.p, d.cover_nsf.p, thr, row_cnt.p,
                                          row_len.p);
  CQ_CUDA(cudaGetLastError());
  int64_t nnz = exclusive_scan(row_cnt.p, N, ptr64.p, st);
  CQ_CHECK(nnz < (int64_t)INT32_MAX, CQ_ERR_ARG, "too many blocks for 32-bit block ids");
  R.nnz = (int)nnz;
  R.row_ptr.alloc(N + 1, st);
  k_i64_to_i32<<<nblk(N + 1, T), T, 0, st>>>(ptr64.p, N + 1, R.row_ptr.p);
  R.row_elem.alloc(N + 1, st);
  R.length = exclusive_scan(row_len.p, N, R.row_elem.p, st);
  // ---- fill
  R.nb_cover.alloc(std::max(R.nnz, 1), st);
  R.nb_elem.alloc(std::max(R.nnz, 1), st);
  R.nb_row.alloc(std::max(R.nnz, 1), st);
  R.nb_ibpart.alloc(std::max(R.nnz, 1), st);
  R.nb_radius.alloc(std::max(R.nnz, 1), st);
  R.onsite.alloc(N, st);
  CQ_CUDA(cudaMemsetAsync(R.onsite.p, 0xff, sizeof(int64_t) * N, st));
  k_naba_fill<<<nblk(N, WPB), T, 0, st>>>(N, NC, d.prim_x.p, d.cover_x.p, d.prim_nsf.p, d.cover_nsf.p, d.cover_part.p,
                                         d.cover_seq.p, d.cover_label_of_part.p, d.prim_cover_label.p, d.prim_seq.p,
                                         d.prim_part.p, d.part_disp.p, g.ncover[1], g.ncover[2], g.nspan[0], g.nspan[1],
                                         g.nspan[2], thr, R.row_ptr.p, R.row_elem.p, R.nb_cover.p, R.nb_elem.p, R.nb_row.p,
                                         R.nb_ibpart.p, R.nb_radius.p, R.onsite.p);
  CQ_CUDA(cudaGetLastError());
  // ---- halo
  DevBuf<int> flag;
  flag.alloc(NC, st);
  CQ_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int) * NC, st));
  if (R.nnz) k_flag<<<nblk(R.nnz, T), T, 0, st>>>(R.nnz, R.nb_cover.p, flag.p);
  DevBuf<int64_t> hex;
  hex.alloc(NC + 1, st);
  int64_t nh = exclusive_scan(flag.p, NC, hex.p, st);
  R.ni_in_halo = (int)nh;
  DevBuf<int> hex32;
  hex32.alloc(NC + 1, st);
  k_i64_to_i32<<<nblk(NC + 1, T), T, 0, st>>>(hex.p, NC + 1, hex32.p);
  R.cover_to_halo.alloc(NC, st);
  R.halo_cover.alloc(std::max<int64_t>(nh, 1), st);
  k_halo_number<<<nblk(NC, T), T, 0, st>>>(NC, flag.p, hex32.p, R.cover_to_halo.p, R.halo_cover.p);
  R.nb_halo.alloc(std::max(R.nnz, 1), st);
  if (R.nnz) k_gather_int<<<nblk(R.nnz, T), T, 0, st>>>(R.nnz, R.nb_cover.p, R.cover_to_halo.p, R.nb_halo.p);
  CQ_CUDA(cudaGetLastError());
  // halo partitions (host bookkeeping of np_in_halo from the flags)
  {
    std::vector<int> hf = flag.download(st);
    int np_h = 0;
    for (int np_ = 0; np_ < g.ng_cover; ++np_) {
      bool any = false;
      for (int c = g.cover_first[np_]; c < g.cover_first[np_ + 1]; ++c) any |= hf[c] != 0;
      np_h += any;
    }
    R.np_in_halo = np_h;
  }
  // ---- retro lists
  DevBuf<int> err;
  err.alloc(1, st);
  CQ_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), st));
  DevBuf<int> col_cnt;
  col_cnt.alloc(std::max<int64_t>(nh, 1), st);
  DevBuf<int64_t> col64;
  col64.alloc(nh + 1, st);
  if (nh) k_retr_count<<<nblk(nh, WPB), T, 0, st>>>((int)nh, N, R.halo_cover.p, d.cover_x.p, d.prim_x.p, thr, col_cnt.p);
  int64_t ncol = exclusive_scan(col_cnt.p, nh, col64.p, st);
  CQ_CHECK(ncol == nnz, CQ_ERR_STATE, "retro lists disagree with the neighbour lists");
  R.col_ptr.alloc(nh + 1, st);
  k_i64_to_i32<<<nblk(nh + 1, T), T, 0, st>>>(col64.p, (int)nh + 1, R.col_ptr.p);
  R.col_row.alloc(std::max(R.nnz, 1), st);
  R.col_blk.alloc(std::max(R.nnz, 1), st);
  if (nh)
    k_retr_fill<<<nblk(nh, WPB), T, 0, st>>>((int)nh, N, R.halo_cover.p, d.cover_x.p, d.prim_x.p, thr, R.col_ptr.p,
                                             R.row_ptr.p, R.nb_cover.p, R.col_row.p, R.col_blk.p, err.p);
  // ---- transpose destinations
  R.trans_dest.alloc(std::max(R.nnz, 1), st);
  if (R.nnz)
    k_trans_dest<<<nblk(R.nnz, T), T, 0, st>>>(R.nnz, R.nb_row.p, R.nb_cover.p, d.cover_part.p, d.cover_label_of_part.p,
                                               d.cover_home_prim.p, d.prim_cover_label.p, d.prim_seq.p, d.label_to_cover.p,
                                               d.cover_first.p, R.row_ptr.p, g.ncover[1], g.ncover[2], g.ng_cover,
                                               R.trans_dest.p, err.p);
  CQ_CUDA(cudaGetLastError());
  CQ_CHECK(read_flag(err.p, st) == 0, CQ_ERR_BOUNDS, "index build: retro or transpose lookup failed");
  R.h_row_ptr = R.row_ptr.download(st);
  R.max_row = 0;
  for (int p = 0; p < N; ++p) R.max_row = std::max(R.max_row, R.h_row_ptr[p + 1] - R.h_row_ptr[p]);
}

ProductPlan& get_plan(System& S, int mult_type, int ra, int rb, int rc) {
  auto key = std::make_tuple(mult_type, ra, rb, rc);
  auto it = S.plans.find(key);
  if (it != S.plans.end()) return *it->second;
  CQ_CHECK(mult_type == 1 || mult_type == 2, CQ_ERR_ARG, "mult_type must be 1 or 2");
  int nr = (int)S.ranges.size();
  CQ_CHECK(ra >= 0 && ra < nr && rb >= 0 && rb < nr && rc >= 0 && rc < nr, CQ_ERR_ARG, "range out of bounds");
  auto plan = std::make_unique<ProductPlan>();
  ProductPlan& P = *plan;
  P.mult_type = mult_type; P.ra = ra; P.rb = rb; P.rc = rc;
  RangeIndex &A = *S.ranges[ra], &B = *S.ranges[rb], &C = *S.ranges[rc];
  DevGeometry& d = S.dg;
  cudaStream_t st = S.stream;
  PlanArgs pa;
  pa.a_row_ptr = A.row_ptr.p; pa.a_cover = A.nb_cover.p; pa.a_row = A.nb_row.p;
  pa.b_row_ptr = B.row_ptr.p; pa.b_cover = B.nb_cover.p; pa.b_ibpart = B.nb_ibpart.p;
  pa.c_row_ptr = C.row_ptr.p; pa.c_cover = C.nb_cover.p;
  pa.cover_part = d.cover_part.p; pa.cover_label_of_part = d.cover_label_of_part.p; pa.cover_home_prim = d.cover_home_prim.p;
  pa.label_to_cover = d.label_to_cover.p; pa.cover_first = d.cover_first.p; pa.cover_seq = d.cover_seq.p;
  pa.cover_nsf = d.cover_nsf.p; pa.prim_nsf = d.prim_nsf.p; pa.ng_cover = S.geo.ng_cover;
  const int N = S.geo.n_prim;
  const int T = 256, WPB = T / kWarp;
  RangeIndex& out = mult_type == 1 ? C : A;
  P.out_range = mult_type == 1 ? rc : ra;
  int nout = out.nnz;
  DevBuf<int> cnt, err;
  cnt.alloc(std::max(nout, 1), st);
  err.alloc(1, st);
  DevBuf<unsigned long long> fl;
  fl.alloc(1, st);
  CQ_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * std::max(nout, 1), st));
  CQ_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), st));
  CQ_CUDA(cudaMemsetAsync(fl.p, 0, sizeof(unsigned long long), st));
  if (mult_type == 1) k_plan1<<<nblk(N, WPB), T, 0, st>>>(pa, N, 0, cnt.p, nullptr, nullptr, nullptr, fl.p, err.p);
  else if (nout) k_plan2<<<nblk(nout, WPB), T, 0, st>>>(pa, nout, 0, cnt.p, nullptr, nullptr, fl.p, err.p);
  CQ_CUDA(cudaGetLastError());
  P.ptr.alloc(nout + 1, st);
  P.n_pairs = exclusive_scan(cnt.p, nout, P.ptr.p, st);
  CQ_CHECK(read_flag(err.p, st) == 0, CQ_ERR_BOUNDS, "pair list: neighbour partition outside the covering set");
  unsigned long long hfl = 0;
  CQ_CUDA(cudaMemcpyAsync(&hfl, fl.p, sizeof(hfl), cudaMemcpyDeviceToHost, st));
  CQ_CUDA(cudaStreamSynchronize(st));
  P.flops = (int64_t)hfl;
  P.pairs.alloc(std::max<int64_t>(P.n_pairs, 1), st);
  if (mult_type == 1) {
    CQ_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * std::max(nout, 1), st));
    k_plan1<<<nblk(N, WPB), T, 0, st>>>(pa, N, 1, nullptr, P.ptr.p, cnt.p, P.pairs.p, nullptr, err.p);
  } else if (nout) {
    k_plan2<<<nblk(nout, WPB), T, 0, st>>>(pa, nout, 1, nullptr, P.ptr.p, P.pairs.p, nullptr, err.p);
  }
  CQ_CUDA(cudaGetLastError());
  CQ_CHECK(read_flag(err.p, st) == 0, CQ_ERR_BOUNDS, "pair list: lookup failed");
  auto res = S.plans.emplace(key, std::move(plan));
  return *res.first->second;
}

MixedPlan& get_mixed_plan(System& S, int mult_type, int ra, int rb, int rc) {
  auto key = std::make_tuple(mult_type, ra, rb, rc);
  auto it = S.mplans.find(key);
  if (it != S.mplans.end()) return *it->second;
  ProductPlan& P = get_plan(S, mult_type, ra, rb, rc);
  auto mp = std::make_unique<MixedPlan>();
  MixedPlan& M = *mp;
  M.mult_type = mult_type; M.ra = ra; M.rb = rb; M.rc = rc;
  M.out_range = P.out_range;
  M.flops = P.flops;
  M.n_pairs = P.n_pairs;
  cudaStream_t st = S.stream;
  if (mult_type == 1) {
    // type-1 lists follow row i of A in order: already sorted by the first operand
    M.ptr = P.ptr.p;
    M.pairs = P.pairs.p;
  } else {
    RangeIndex &A = *S.ranges[ra], &B = *S.ranges[rb], &C = *S.ranges[rc];
    DevGeometry& d = S.dg;
    PlanArgs pa;
    pa.a_row_ptr = A.row_ptr.p; pa.a_cover = A.nb_cover.p; pa.a_row = A.nb_row.p;
    pa.b_row_ptr = B.row_ptr.p; pa.b_cover = B.nb_cover.p; pa.b_ibpart = B.nb_ibpart.p;
    pa.c_row_ptr = C.row_ptr.p; pa.c_cover = C.nb_cover.p;
    pa.cover_part = d.cover_part.p; pa.cover_label_of_part = d.cover_label_of_part.p;
    pa.cover_home_prim = d.cover_home_prim.p; pa.label_to_cover = d.label_to_cover.p; pa.cover_first = d.cover_first.p;
    pa.cover_seq = d.cover_seq.p; pa.cover_nsf = d.cover_nsf.p; pa.prim_nsf = d.prim_nsf.p;
    pa.ng_cover = S.geo.ng_cover;
    const int nout = A.nnz, T = 256, WPB = T / kWarp;
    DevBuf<int> cnt;
    cnt.alloc(std::max(nout, 1), st);
    const int* g = S.geo.ncover;
    if (nout) k_plan2x<<<nblk(nout, WPB), T, 0, st>>>(pa, nout, 0, d.prim_cover_label.p, g[0], g[1], g[2], cnt.p, nullptr, nullptr);
    CQ_CUDA(cudaGetLastError());
    M.own_ptr.alloc(nout + 1, st);
    int64_t np2 = exclusive_scan(cnt.p, nout, M.own_ptr.p, st);
    CQ_CHECK(np2 == P.n_pairs, CQ_ERR_STATE, "type-2 lists by input block disagree with the default-order lists");
    M.own_pairs.alloc(std::max<int64_t>(np2, 1), st);
    if (nout) k_plan2x<<<nblk(nout, WPB), T, 0, st>>>(pa, nout, 1, d.prim_cover_label.p, g[0], g[1], g[2], nullptr, M.own_ptr.p, M.own_pairs.p);
    CQ_CUDA(cudaGetLastError());
    M.ptr = M.own_ptr.p;
    M.pairs = M.own_pairs.p;
  }
  CQ_CUDA(cudaStreamSynchronize(st));
  auto res = S.mplans.emplace(key, std::move(mp));
  return *res.first->second;
}

AddMap& get_addmap(System& S, int ra, int rb) {
  auto key = std::make_pair(ra, rb);
  auto it = S.addmaps.find(key);
  if (it != S.addmaps.end()) return *it->second;
  RangeIndex &A = *S.ranges[ra], &B = *S.ranges[rb];
  auto m = std::make_unique<AddMap>();
  m->partner.alloc(std::max(A.nnz, 1), S.stream);
  if (A.nnz) k_addmap<<<nblk(A.nnz, 256), 256, 0, S.stream>>>(A.nnz, A.nb_row.p, A.nb_cover.p, B.row_ptr.p, B.nb_cover.p, m->partner.p);
  CQ_CUDA(cudaGetLastError());
  auto res = S.addmaps.emplace(key, std::move(m));
  return *res.first->second;
}

// ---------------------------------------------------------------------------
// exports in the reference's 1-based conventions (parity checks)
// ---------------------------------------------------------------------------
void export_range_array(System& S, int r, const std::string& nm, std::vector<int64_t>& v) {
  Geometry& g = S.geo;
  cudaStream_t st = S.stream;
  v.clear();
  if (r < 0) {
    if (nm == "n_parts") { for (int q = 0; q < 3; ++q) v.push_back(g.n_parts[q]); }
    else if (nm == "cover_dims") {
      v = {g.ncover[0], g.ncover[1], g.ncover[2], g.nspan[0], g.nspan[1], g.nspan[2], g.ng_cover, g.n_cover_atoms};
    } else if (nm == "ngnode") { for (int x : g.hilbert_to_cc) v.push_back(x); }
    else if (nm == "nm_group") { for (int cc = 1; cc <= g.np_in_cell; ++cc) v.push_back(g.part_natoms[cc]); }
    else if (nm == "ig_prim") { for (int x : g.prim_global) v.push_back(x + 1); }
    else if (nm == "lab_cell") { for (int x : g.cover_cell) v.push_back(x); }
    else if (nm == "lab_cover") { for (int x : g.cover_label) v.push_back(x); }
    else if (nm == "n_ing_cover") { for (int x : g.cover_count) v.push_back(x); }
    else if (nm == "icover_ibeg") { for (int q = 0; q < g.ng_cover; ++q) v.push_back(g.cover_first[q] + 1); }
    else if (nm == "ig_cover") { for (int x : g.cover_global) v.push_back(x + 1); }
    else if (nm == "iprim_group") { for (int x : g.prim_cover_label) v.push_back(x); }
    else throw Error(CQ_ERR_ARG, "unknown geometry array " + nm);
    return;
  }
  CQ_CHECK(r < (int)S.ranges.size(), CQ_ERR_ARG, "range out of bounds");
  RangeIndex& R = *S.ranges[r];
  const int N = g.n_prim;
  std::vector<int> rp = R.h_row_ptr;
  std::vector<int> cov = R.nb_cover.download(st);
  std::vector<int64_t> el = R.nb_elem.download(st);
  std::vector<int> ibp = R.nb_ibpart.download(st);
  std::vector<int> c2h = R.cover_to_halo.download(st);
  std::vector<int64_t> ons = R.onsite.download(st);
  cov.resize(R.nnz); el.resize(R.nnz); ibp.resize(R.nnz);
  auto prim_nsf = [&](int p) { return g.nsf[g.prim_global[p]]; };
  // per-partition relative offsets (i_acc, i_nd_acc are relative to the partition start)
  std::vector<int> part_of_row(N), first_row_of_part(g.np_in_cell + 1);
  for (int q = 0; q <= g.np_in_cell; ++q) first_row_of_part[q] = g.part_first_prim[q];
  for (int p = 0; p < N; ++p) part_of_row[p] = g.prim_part[p];
  if (nm == "shift") {  // image of each stored neighbour, in cell vectors (3 per block)
    for (int e = 0; e < R.nnz; ++e) for (int d = 0; d < 3; ++d) v.push_back(g.cover_shift[3 * g.cover_part[cov[e]] + d]);
  } else if (nm == "ig_j") { for (int e = 0; e < R.nnz; ++e) v.push_back(g.cover_global[cov[e]] + 1); }
  else if (nm == "elem") { for (int e = 0; e < R.nnz; ++e) v.push_back(el[e]); }
  else if (nm == "n_nab") { for (int p = 0; p < N; ++p) v.push_back(rp[p + 1] - rp[p]); }
  else if (nm == "i_acc") { for (int p = 0; p < N; ++p) v.push_back(rp[p] + 1); }
  else if (nm == "i_nd_acc") {
    for (int p = 0; p < N; ++p) v.push_back(rp[p + 1] > rp[p] ? el[rp[p]] + 1 : 0);
  } else if (nm == "ndimi") { for (int p = 0; p < N; ++p) v.push_back(prim_nsf(p)); }
  else if (nm == "onsite") { for (int p = 0; p < N; ++p) v.push_back(ons[p] + 1); }
  else if (nm == "i_part") { for (int e = 0; e < R.nnz; ++e) v.push_back(g.cover_part[cov[e]] + 1); }
  else if (nm == "i_seq") { for (int e = 0; e < R.nnz; ++e) v.push_back(g.cover_seq[cov[e]]); }
  else if (nm == "ndimj") { for (int e = 0; e < R.nnz; ++e) v.push_back(g.cover_nsf[cov[e]]); }
  else if (nm == "npxyz") {
    int yz = g.ncover[1] * g.ncover[2];
    int p = 0;
    for (int e = 0; e < R.nnz; ++e) {
      int lab = g.cover_label[g.cover_part[cov[e]]] - 1;
      int nx = lab / yz, ny = (lab - nx * yz) / g.ncover[2], nz = lab - nx * yz - ny * g.ncover[2];
      while (p + 1 <= N && rp[p + 1] <= e) ++p;
      const int* dsp = &g.part_disp[3 * g.prim_part[p]];
      v.push_back(nx - g.nspan[0] - dsp[0]);
      v.push_back(ny - g.nspan[1] - dsp[1]);
      v.push_back(nz - g.nspan[2] - dsp[2]);
    }
  } else if (nm == "bind") {
    // set_matrix_pointers2 layout: per partition n_nab, i_acc, i_nd_acc, i_seq, npxyz, ndimj (partition-relative)
    std::vector<int64_t> npx;
    export_range_array(S, r, "npxyz", npx);
    for (int q = 0; q < g.np_in_cell; ++q) {
      int p0 = first_row_of_part[q], p1 = first_row_of_part[q + 1];
      int e0 = rp[p0], e1 = rp[p1];
      int na = p1 - p0, nabs = e1 - e0;
      int64_t el0 = (e1 > e0) ? el[e0] : 0;
      if (na == 0) { v.push_back(0); v.push_back(1); v.push_back(1); }
      else {
        for (int p = p0; p < p1; ++p) v.push_back(rp[p + 1] - rp[p]);
        for (int p = p0; p < p1; ++p) v.push_back(rp[p] - e0 + 1);
        for (int p = p0; p < p1; ++p) {
          int64_t first = (rp[p + 1] > rp[p]) ? el[rp[p]] : (p + 1 < p1 && rp[p + 1] < e1 ? el[rp[p + 1]] : el0);
          v.push_back(first - el0 + 1);
        }
      }
      if (nabs == 0) { v.push_back(0); v.push_back(0); v.push_back(0); v.push_back(0); v.push_back(0); }
      else {
        for (int e = e0; e < e1; ++e) v.push_back(g.cover_seq[cov[e]]);
        for (int e = e0; e < e1; ++e) for (int t = 0; t < 3; ++t) v.push_back(npx[3 * (size_t)e + t]);
        for (int e = e0; e < e1; ++e) v.push_back(g.cover_nsf[cov[e]]);
      }
    }
  } else if (nm == "halo_sizes") { v = {R.np_in_halo, R.ni_in_halo}; }
  else if (nm == "nh_part" || nm == "j_beg" || nm == "lab_hcell" || nm == "lab_hcover") {
    int jb = 1;
    for (int np_ = 0; np_ < g.ng_cover; ++np_) {
      int k = 0;
      for (int c = g.cover_first[np_]; c < g.cover_first[np_ + 1]; ++c) k += c2h[c] >= 0;
      if (!k) continue;
      if (nm == "nh_part") v.push_back(k);
      else if (nm == "j_beg") v.push_back(jb);
      else if (nm == "lab_hcell") v.push_back(g.cover_cell[np_]);
      else v.push_back(g.cover_label[np_]);
      jb += k;
    }
  } else if (nm == "j_seq" || nm == "halo_ndimj") {
    std::vector<int> hc = R.halo_cover.download(st);
    for (int h = 0; h < R.ni_in_halo; ++h) v.push_back(nm == "j_seq" ? g.cover_seq[hc[h]] : g.cover_nsf[hc[h]]);
  } else if (nm == "i_halo") { for (int c = 0; c < g.n_cover_atoms; ++c) v.push_back(c2h[c] + 1); }
  else if (nm == "i_h2d") {
    size_t nh = R.ni_in_halo;
    v.assign((size_t)N * nh, 0);
    for (int p = 0; p < N; ++p)
      for (int e = rp[p]; e < rp[p + 1]; ++e) v[(size_t)p * nh + c2h[cov[e]]] = el[e] + 1;
  } else if (nm == "t_i_prim" || nm == "t_i_beg" || nm == "t_i_nd_beg" || nm == "t_n_hnab" || nm == "itran_addr") {
    std::vector<int> cp = R.col_ptr.download(st), cr = R.col_row.download(st), cb = R.col_blk.download(st);
    std::vector<int> td = R.trans_dest.download(st);
    int64_t nd_beg = 1;
    for (int h = 0; h < R.ni_in_halo; ++h) {
      if (nm == "t_n_hnab") v.push_back(cp[h + 1] - cp[h]);
      else if (nm == "t_i_beg") v.push_back(cp[h] + 1);
      else if (nm == "t_i_nd_beg") v.push_back(nd_beg);
      for (int t = cp[h]; t < cp[h + 1]; ++t) {
        int p = cr[t];
        if (nm == "t_i_prim") v.push_back(p + 1);
        if (nm == "itran_addr") v.push_back(el[td[cb[t]]] + 1);
        nd_beg += (int64_t)prim_nsf(p) * g.cover_nsf[cov[cb[t]]];
      }
    }
  } else {
    throw Error(CQ_ERR_ARG, "unknown range array " + nm);
  }
}

}  // namespace cqb
