// Split-precision block products on the tensor cores (blocks of up to 16 x 16).
//
// Each FP64 operand block is padded to 16 x 16 and split into two bf16 parts,
// v = hi + lo (hi = bf16(v), lo = bf16(v - hi)); a block product is the sum of
// hi.hi + hi.lo + lo.hi (three bf16 MMAs, FP32 accumulation), which carries
// about 16 significant bits per term.  The three-part split (v = hi + mid + lo,
// six MMAs per term, FP64 accumulation across terms) carries about 22.  The result is written back as FP64 into
// the block storage of the output range, so the matrices of the chain stay FP64.
//
// Work decomposition (output stationary, same pair lists as the FP64 path):
// one warp owns G consecutive output blocks of one output row i (G = 1, 2, 4 or 8, chosen per
// product by the autotuner: larger groups reuse each first-operand fragment more, smaller ones
// need fewer registers and give more warps; the results do not depend on G, since each output
// block accumulates its own pairs in its own order).  Their pair
// lists are sorted by the first operand block (A_ik for type 1, C_ij for type 2,
// both in row i), so the warp walks the union of those blocks in order, loads each
// first-operand fragment once and multiplies it into every output block whose list
// contains it.  Operands are pre-converted into the per-lane fragment order of
// mma.m16n8k16, so every fragment is one coalesced 16-byte load per lane.
#include <cuda_bf16.h>

#include <algorithm>
#include <climits>

#include "cq_internal.hpp"

namespace cqb {
namespace {


__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 lo_k, __nv_bfloat16 hi_k) {
  return (uint32_t)__bfloat16_as_ushort(lo_k) | ((uint32_t)__bfloat16_as_ushort(hi_k) << 16);
}

// element (r, c) of a padded 16 x 16 view of a column-major nd_r x nd_c FP64 block
__device__ __forceinline__ double blk_at(const double* B, int nd_r, int nd_c, int r, int c) {
  return (r < nd_r && c < nd_c) ? B[r + nd_r * c] : 0.0;
}

__device__ __forceinline__ void split2(double v, __nv_bfloat16& h, __nv_bfloat16& l) {
  h = __double2bfloat16(v);
  l = __double2bfloat16(v - (double)__bfloat162float(h));
}

// v = hi + mid + lo + r with |r| <= 2^-24 |v| (about 2^-25 for round-to-nearest parts): both
// differences are exact in FP64
__device__ __forceinline__ void split3(double v, __nv_bfloat16& h, __nv_bfloat16& m, __nv_bfloat16& l) {
  h = __double2bfloat16(v);
  const double r1 = v - (double)__bfloat162float(h);
  m = __double2bfloat16(r1);
  l = __double2bfloat16(r1 - (double)__bfloat162float(m));
}

// A-role fragments (M = block rows, K = block columns):
//   reg0 (row g,   k 2t..2t+1), reg1 (row g+8, k 2t..2t+1), reg2 (row g, k 2t+8..), reg3 (row g+8, k 2t+8..)
// B-role fragments (K = block rows, N = block columns; `trans` uses the transposed block),
//   two n8 tiles: {tile0 (k 2t.., n g), tile0 (k 2t+8.., n g), tile1 (k 2t.., n g+8), tile1 (k 2t+8.., n g+8)}
__global__ void k_to_frag(int nnz, const int64_t* __restrict__ elem, const int* __restrict__ row,
                          const int* __restrict__ cover, const int* __restrict__ prim_nsf,
                          const int* __restrict__ cover_nsf, const double* __restrict__ src, int role_b, int trans,
                          uint4* __restrict__ hi, uint4* __restrict__ lo, uint4* __restrict__ mid) {
  int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int e = (int)(tid >> 5), lane = (int)(tid & 31);
  if (e >= nnz) return;
  const int ndr = prim_nsf[row[e]], ndc = cover_nsf[cover[e]];
  const double* B = src + elem[e];
  const int g = lane >> 2, t = lane & 3;
  int rr[8], cc[8];
  if (!role_b) {
    const int r0[4] = {g, g + 8, g, g + 8}, c0[4] = {2 * t, 2 * t, 2 * t + 8, 2 * t + 8};
    for (int q = 0; q < 4; ++q) { rr[2 * q] = r0[q]; cc[2 * q] = c0[q]; rr[2 * q + 1] = r0[q]; cc[2 * q + 1] = c0[q] + 1; }
  } else {
    // (K, N) pairs; element (K=k, N=n) is block (k, n), or block (n, k) when transposed
    const int k0[4] = {2 * t, 2 * t + 8, 2 * t, 2 * t + 8}, n0[4] = {g, g, g + 8, g + 8};
    for (int q = 0; q < 4; ++q) {
      for (int h = 0; h < 2; ++h) {
        int k = k0[q] + h, n = n0[q];
        rr[2 * q + h] = trans ? n : k;
        cc[2 * q + h] = trans ? k : n;
      }
    }
  }
  uint32_t wh[4], wm[4], wl[4];
  for (int q = 0; q < 4; ++q) {
    __nv_bfloat16 h0, m0, l0, h1, m1, l1;
    const double v0 = blk_at(B, ndr, ndc, rr[2 * q], cc[2 * q]), v1 = blk_at(B, ndr, ndc, rr[2 * q + 1], cc[2 * q + 1]);
    if (mid) {
      split3(v0, h0, m0, l0);
      split3(v1, h1, m1, l1);
      wm[q] = pack_bf16(m0, m1);
    } else {
      split2(v0, h0, l0);
      split2(v1, h1, l1);
    }
    wh[q] = pack_bf16(h0, h1);
    wl[q] = pack_bf16(l0, l1);
  }
  hi[(int64_t)e * 32 + lane] = make_uint4(wh[0], wh[1], wh[2], wh[3]);
  lo[(int64_t)e * 32 + lane] = make_uint4(wl[0], wl[1], wl[2], wl[3]);
  if (mid) mid[(int64_t)e * 32 + lane] = make_uint4(wm[0], wm[1], wm[2], wm[3]);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint4& a, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a.x), "r"(a.y), "r"(a.z), "r"(a.w), "r"(b0), "r"(b1));
}

struct TCArgs {
  const int2* __restrict__ groups;     // (first output block, count) per warp, never crossing a row
  int n_groups;
  const int64_t* __restrict__ ptr;     // pair list offsets per output block
  const int2* __restrict__ pairs;      // (first-operand block, B block), first operand ascending
  const uint4* __restrict__ xa_hi;     // first operand, A-role fragments
  const uint4* __restrict__ xa_lo;
  const uint4* __restrict__ bb_hi;     // B operand, B-role fragments
  const uint4* __restrict__ bb_lo;
  const uint4* __restrict__ xa_mid;    // middle parts (three-part split only)
  const uint4* __restrict__ bb_mid;
  const int* __restrict__ o_row;
  const int* __restrict__ o_cover;
  const int64_t* __restrict__ o_elem;
  const int* __restrict__ prim_nsf;
  const int* __restrict__ cover_nsf;
  double* __restrict__ out;
};

template <int kG>   // output blocks per warp
__global__ void __launch_bounds__(128) k_mult_tc(TCArgs M) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= M.n_groups) return;
  const int2 grp = M.groups[w];
  int64_t p[kG], pe[kG];
  int nx[kG];
  float acc[kG][2][4];
#pragma unroll
  for (int b = 0; b < kG; ++b) {
    if (b < grp.y) { p[b] = M.ptr[grp.x + b]; pe[b] = M.ptr[grp.x + b + 1]; }
    else { p[b] = 0; pe[b] = 0; }
    nx[b] = p[b] < pe[b] ? M.pairs[p[b]].x : INT_MAX;
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[b][h][r] = 0.f;
  }
  while (true) {
    int kc = INT_MAX;
#pragma unroll
    for (int b = 0; b < kG; ++b) kc = min(kc, nx[b]);
    if (kc == INT_MAX) break;
    const uint4 ah = __ldg(M.xa_hi + (int64_t)kc * 32 + lane);
    const uint4 al = __ldg(M.xa_lo + (int64_t)kc * 32 + lane);
#pragma unroll
    for (int b = 0; b < kG; ++b) {
      if (nx[b] == kc) {
        const int y = M.pairs[p[b]].y;
        const uint4 bh = __ldg(M.bb_hi + (int64_t)y * 32 + lane);
        const uint4 bl = __ldg(M.bb_lo + (int64_t)y * 32 + lane);
        mma_bf16(acc[b][0], al, bh.x, bh.y);
        mma_bf16(acc[b][0], ah, bl.x, bl.y);
        mma_bf16(acc[b][0], ah, bh.x, bh.y);
        mma_bf16(acc[b][1], al, bh.z, bh.w);
        mma_bf16(acc[b][1], ah, bl.z, bl.w);
        mma_bf16(acc[b][1], ah, bh.z, bh.w);
        ++p[b];
        nx[b] = p[b] < pe[b] ? M.pairs[p[b]].x : INT_MAX;
      }
    }
  }
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int b = 0; b < kG; ++b) {
    if (b < grp.y) {
      const int q = grp.x + b;
      const int ndr = M.prim_nsf[M.o_row[q]], ndc = M.cover_nsf[M.o_cover[q]];
      double* O = M.out + M.o_elem[q];
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          int row = g + ((r & 2) ? 8 : 0), col = 8 * h + 2 * t + (r & 1);
          if (row < ndr && col < ndc) O[row + ndr * col] = (double)acc[b][h][r];
        }
    }
  }
}

// One output block per warp with the next term's four fragments loaded while the current term's
// six MMAs run (the group-of-one case of k_mult_tc, same terms in the same order, so the same
// result): the fragment loads of consecutive terms overlap instead of stalling each term.
__global__ void __launch_bounds__(128) k_mult_tc1(TCArgs M) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= M.n_groups) return;
  const int q = M.groups[w].x;
  int64_t p = M.ptr[q];
  const int64_t pe = M.ptr[q + 1];
  float acc[2][4];
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int r = 0; r < 4; ++r) acc[h][r] = 0.f;
  uint4 ah = {0, 0, 0, 0}, al = ah, bh = ah, bl = ah;
  if (p < pe) {
    const int2 pr = M.pairs[p];
    ah = __ldg(M.xa_hi + (int64_t)pr.x * 32 + lane);
    al = __ldg(M.xa_lo + (int64_t)pr.x * 32 + lane);
    bh = __ldg(M.bb_hi + (int64_t)pr.y * 32 + lane);
    bl = __ldg(M.bb_lo + (int64_t)pr.y * 32 + lane);
  }
  for (; p < pe; ++p) {
    uint4 nah = ah, nal = al, nbh = bh, nbl = bl;
    if (p + 1 < pe) {
      const int2 pn = M.pairs[p + 1];
      nah = __ldg(M.xa_hi + (int64_t)pn.x * 32 + lane);
      nal = __ldg(M.xa_lo + (int64_t)pn.x * 32 + lane);
      nbh = __ldg(M.bb_hi + (int64_t)pn.y * 32 + lane);
      nbl = __ldg(M.bb_lo + (int64_t)pn.y * 32 + lane);
    }
    mma_bf16(acc[0], al, bh.x, bh.y);
    mma_bf16(acc[0], ah, bl.x, bl.y);
    mma_bf16(acc[0], ah, bh.x, bh.y);
    mma_bf16(acc[1], al, bh.z, bh.w);
    mma_bf16(acc[1], ah, bl.z, bl.w);
    mma_bf16(acc[1], ah, bh.z, bh.w);
    ah = nah; al = nal; bh = nbh; bl = nbl;
  }
  const int g = lane >> 2, t = lane & 3;
  const int ndr = M.prim_nsf[M.o_row[q]], ndc = M.cover_nsf[M.o_cover[q]];
  double* O = M.out + M.o_elem[q];
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      int row = g + ((r & 2) ? 8 : 0), col = 8 * h + 2 * t + (r & 1);
      if (row < ndr && col < ndc) O[row + ndr * col] = (double)acc[h][r];
    }
}

// Three-part split (BF16x6): v = hi + mid + lo, one output block per warp.  Per term and n8 half the
// six products that carry terms down to 2^-16 of hi.hi run into a zeroed FP32 accumulator, smallest
// first (hi.lo, lo.hi, mid.mid, hi.mid, mid.hi, hi.hi), and the term's 16 x 8 result is added to FP64
// accumulators, so the FP32 rounding spans one 16-wide contraction rather than the whole sum.  The
// omitted products (mid.lo, lo.mid, lo.lo) and the split remainders are below 2^-23 of |a||b| per
// element product.  The next term's six fragments load while the current term's MMAs run.
__global__ void __launch_bounds__(128) k_mult_tc6(TCArgs M) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= M.n_groups) return;
  const int q = M.groups[w].x;
  int64_t p = M.ptr[q];
  const int64_t pe = M.ptr[q + 1];
  double acc[2][4];
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int r = 0; r < 4; ++r) acc[h][r] = 0.0;
  uint4 ah = {0, 0, 0, 0}, am = ah, al = ah, bh = ah, bm = ah, bl = ah;
  if (p < pe) {
    const int2 pr = M.pairs[p];
    ah = __ldg(M.xa_hi + (int64_t)pr.x * 32 + lane);
    am = __ldg(M.xa_mid + (int64_t)pr.x * 32 + lane);
    al = __ldg(M.xa_lo + (int64_t)pr.x * 32 + lane);
    bh = __ldg(M.bb_hi + (int64_t)pr.y * 32 + lane);
    bm = __ldg(M.bb_mid + (int64_t)pr.y * 32 + lane);
    bl = __ldg(M.bb_lo + (int64_t)pr.y * 32 + lane);
  }
  for (; p < pe; ++p) {
    uint4 nah = ah, nam = am, nal = al, nbh = bh, nbm = bm, nbl = bl;
    if (p + 1 < pe) {
      const int2 pn = M.pairs[p + 1];
      nah = __ldg(M.xa_hi + (int64_t)pn.x * 32 + lane);
      nam = __ldg(M.xa_mid + (int64_t)pn.x * 32 + lane);
      nal = __ldg(M.xa_lo + (int64_t)pn.x * 32 + lane);
      nbh = __ldg(M.bb_hi + (int64_t)pn.y * 32 + lane);
      nbm = __ldg(M.bb_mid + (int64_t)pn.y * 32 + lane);
      nbl = __ldg(M.bb_lo + (int64_t)pn.y * 32 + lane);
    }
    float t[2][4];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int r = 0; r < 4; ++r) t[h][r] = 0.f;
    mma_bf16(t[0], ah, bl.x, bl.y);
    mma_bf16(t[0], al, bh.x, bh.y);
    mma_bf16(t[0], am, bm.x, bm.y);
    mma_bf16(t[0], ah, bm.x, bm.y);
    mma_bf16(t[0], am, bh.x, bh.y);
    mma_bf16(t[0], ah, bh.x, bh.y);
    mma_bf16(t[1], ah, bl.z, bl.w);
    mma_bf16(t[1], al, bh.z, bh.w);
    mma_bf16(t[1], am, bm.z, bm.w);
    mma_bf16(t[1], ah, bm.z, bm.w);
    mma_bf16(t[1], am, bh.z, bh.w);
    mma_bf16(t[1], ah, bh.z, bh.w);
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[h][r] += (double)t[h][r];
    ah = nah; am = nam; al = nal; bh = nbh; bm = nbm; bl = nbl;
  }
  const int g = lane >> 2, t4 = lane & 3;
  const int ndr = M.prim_nsf[M.o_row[q]], ndc = M.cover_nsf[M.o_cover[q]];
  double* O = M.out + M.o_elem[q];
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      int row = g + ((r & 2) ? 8 : 0), col = 8 * h + 2 * t4 + (r & 1);
      if (row < ndr && col < ndc) O[row + ndr * col] = acc[h][r];
    }
}

// Three-part split, G output blocks of one row per warp (G = 2 or 4): each first-operand fragment is
// loaded once for the blocks whose lists contain it.  Every output block takes its terms in its own
// list order, each term rounded to FP32 once as in k_mult_tc6, so the result is the same bits for
// every G.
template <int kG>
__global__ void __launch_bounds__(128) k_mult_tc6g(TCArgs M) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= M.n_groups) return;
  const int2 grp = M.groups[w];
  int64_t p[kG], pe[kG];
  int nx[kG];
  double acc[kG][2][4];
#pragma unroll
  for (int b = 0; b < kG; ++b) {
    if (b < grp.y) { p[b] = M.ptr[grp.x + b]; pe[b] = M.ptr[grp.x + b + 1]; }
    else { p[b] = 0; pe[b] = 0; }
    nx[b] = p[b] < pe[b] ? M.pairs[p[b]].x : INT_MAX;
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[b][h][r] = 0.0;
  }
  while (true) {
    int kc = INT_MAX;
#pragma unroll
    for (int b = 0; b < kG; ++b) kc = min(kc, nx[b]);
    if (kc == INT_MAX) break;
    const uint4 ah = __ldg(M.xa_hi + (int64_t)kc * 32 + lane);
    const uint4 am = __ldg(M.xa_mid + (int64_t)kc * 32 + lane);
    const uint4 al = __ldg(M.xa_lo + (int64_t)kc * 32 + lane);
#pragma unroll
    for (int b = 0; b < kG; ++b) {
      if (nx[b] == kc) {
        const int y = M.pairs[p[b]].y;
        const uint4 bh = __ldg(M.bb_hi + (int64_t)y * 32 + lane);
        const uint4 bm = __ldg(M.bb_mid + (int64_t)y * 32 + lane);
        const uint4 bl = __ldg(M.bb_lo + (int64_t)y * 32 + lane);
        float t[2][4];
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
          for (int r = 0; r < 4; ++r) t[h][r] = 0.f;
        mma_bf16(t[0], ah, bl.x, bl.y);
        mma_bf16(t[0], al, bh.x, bh.y);
        mma_bf16(t[0], am, bm.x, bm.y);
        mma_bf16(t[0], ah, bm.x, bm.y);
        mma_bf16(t[0], am, bh.x, bh.y);
        mma_bf16(t[0], ah, bh.x, bh.y);
        mma_bf16(t[1], ah, bl.z, bl.w);
        mma_bf16(t[1], al, bh.z, bh.w);
        mma_bf16(t[1], am, bm.z, bm.w);
        mma_bf16(t[1], ah, bm.z, bm.w);
        mma_bf16(t[1], am, bh.z, bh.w);
        mma_bf16(t[1], ah, bh.z, bh.w);
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
          for (int r = 0; r < 4; ++r) acc[b][h][r] += (double)t[h][r];
        ++p[b];
        nx[b] = p[b] < pe[b] ? M.pairs[p[b]].x : INT_MAX;
      }
    }
  }
  const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
  for (int b = 0; b < kG; ++b) {
    if (b < grp.y) {
      const int q = grp.x + b;
      const int ndr = M.prim_nsf[M.o_row[q]], ndc = M.cover_nsf[M.o_cover[q]];
      double* O = M.out + M.o_elem[q];
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          int row = g + ((r & 2) ? 8 : 0), col = 8 * h + 2 * t4 + (r & 1);
          if (row < ndr && col < ndc) O[row + ndr * col] = acc[b][h][r];
        }
    }
  }
}

}  // namespace

// A-role (first operand) or B-role fragments of a whole range, hi and lo parts (1 KB per block)
// (and the middle parts of the three-part split when `mid` is given)
void to_fragments(System& S, int r, const double* src, int role_b, int trans, uint4* hi, uint4* lo, uint4* mid) {
  RangeIndex& R = *S.ranges[r];
  if (R.nnz == 0) return;
  int64_t threads = (int64_t)R.nnz * 32;
  k_to_frag<<<(int)((threads + 255) / 256), 256, 0, S.stream>>>(R.nnz, R.nb_elem.p, R.nb_row.p, R.nb_cover.p,
                                                                S.dg.prim_nsf.p, S.dg.cover_nsf.p, src, role_b, trans,
                                                                hi, lo, mid);
  S.launches++;
  CQ_CUDA(cudaGetLastError());
}

static FragBuf& frag_buffer(System& S, int r, int slot, bool three = false) {
  FragBuf& f = S.frags[std::make_pair(r, slot)];
  size_t need = (size_t)std::max(S.ranges[r]->nnz, 1) * 32;
  if (f.hi.n < need) { f.hi.alloc(need, S.stream); f.lo.alloc(need, S.stream); }
  if (three && f.mid.n < need) f.mid.alloc(need, S.stream);
  return f;
}

static void mat_mult_mma_sync(System& S, MixedPlan& MP, int mult_type, int ra, int rb, int rc, double* a,
                              const double* b, double* c) {
  int rx = mult_type == 1 ? ra : rc;
  const double* x = mult_type == 1 ? a : c;
  double* out = mult_type == 1 ? c : a;
  FragBuf& fx = frag_buffer(S, rx, 0);
  FragBuf& fb = frag_buffer(S, rb, 1);
  to_fragments(S, rx, x, 0, 0, fx.hi.p, fx.lo.p, nullptr);
  to_fragments(S, rb, b, 1, mult_type == 2 ? 1 : 0, fb.hi.p, fb.lo.p, nullptr);
  launch_mult_tc(S, MP, fx.hi.p, fx.lo.p, fb.hi.p, fb.lo.p, out);
}

static void ensure_groups(System& S, MixedPlan& MP, int gi);
static void launch_tc6_g(System& S, MixedPlan& MP, TCArgs M, int gi);

// three-part split products (one output block per warp)
static void mat_mult_split6(System& S, MixedPlan& MP, int mult_type, int ra, int rb, int rc, double* a,
                            const double* b, double* c) {
  int rx = mult_type == 1 ? ra : rc;
  const double* x = mult_type == 1 ? a : c;
  double* out = mult_type == 1 ? c : a;
  FragBuf& fx = frag_buffer(S, rx, 0, true);
  FragBuf& fb = frag_buffer(S, rb, 1, true);
  to_fragments(S, rx, x, 0, 0, fx.hi.p, fx.lo.p, fx.mid.p);
  to_fragments(S, rb, b, 1, mult_type == 2 ? 1 : 0, fb.hi.p, fb.lo.p, fb.mid.p);
  RangeIndex& O = *S.ranges[MP.out_range];
  if (O.nnz == 0) return;
  ensure_groups(S, MP, 0);
  TCArgs M;
  M.ptr = MP.ptr;
  M.pairs = MP.pairs;
  M.xa_hi = fx.hi.p; M.xa_lo = fx.lo.p; M.xa_mid = fx.mid.p;
  M.bb_hi = fb.hi.p; M.bb_lo = fb.lo.p; M.bb_mid = fb.mid.p;
  M.o_row = O.nb_row.p; M.o_cover = O.nb_cover.p; M.o_elem = O.nb_elem.p;
  M.prim_nsf = S.dg.prim_nsf.p; M.cover_nsf = S.dg.cover_nsf.p;
  M.out = out;
  if (MP.tuned_g6 < 0) {
    // autotuner: groups of 1, 2 and 4 output blocks (the same bits), as for the two-part kernel
    cudaEvent_t e0, e1;
    CQ_CUDA(cudaEventCreate(&e0));
    CQ_CUDA(cudaEventCreate(&e1));
    float best[3] = {1e30f, 1e30f, 1e30f};
    for (int gi = 0; gi < 3; ++gi) launch_tc6_g(S, MP, M, gi);
    for (int round = 0; round < 3; ++round)
      for (int gi = 0; gi < 3; ++gi) {
        CQ_CUDA(cudaEventRecord(e0, S.stream));
        launch_tc6_g(S, MP, M, gi);
        CQ_CUDA(cudaEventRecord(e1, S.stream));
        CQ_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        CQ_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        best[gi] = std::min(best[gi], ms);
      }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int pick = 0;
    for (int gi = 1; gi < 3; ++gi)
      if (best[gi] < 0.95f * best[pick]) pick = gi;
    for (int gi = 0; gi < 3; ++gi) MP.tune_ms6[gi] = best[gi];
    MP.tuned_g6 = pick;
  }
  const int forced = S.split_group == 1 ? 0 : S.split_group == 2 ? 1 : S.split_group == 4 ? 2 : -1;
  launch_tc6_g(S, MP, M, forced >= 0 ? forced : MP.tuned_g6);
}

// gi = 0: one output block per warp with prefetch; 1, 2: groups of 2 and 4 blocks of one row
static void launch_tc6_g(System& S, MixedPlan& MP, TCArgs M, int gi) {
  static const int kGi[3] = {0, 1, 2};   // index into the group sizes 1, 2, 4, 8
  ensure_groups(S, MP, kGi[gi]);
  M.groups = MP.groups[kGi[gi]].p;
  M.n_groups = MP.n_groups[kGi[gi]];
  if (M.n_groups == 0) return;
  const int grid = (M.n_groups * 32 + 127) / 128;
  if (gi == 0) k_mult_tc6<<<grid, 128, 0, S.stream>>>(M);
  else if (gi == 1) k_mult_tc6g<2><<<grid, 128, 0, S.stream>>>(M);
  else k_mult_tc6g<4><<<grid, 128, 0, S.stream>>>(M);
  S.launches++;
  CQ_CUDA(cudaGetLastError());
}

// Kernel choice of a split-precision product: the system's setting, or (setting -1) a fixed rule on
// the product's tile plan, so that a product always runs the same kernel (and gives the same bits)
// whatever else runs on the device: the tcgen05 tiles where at least kTileMinFill of their issued
// tensor work is useful (3 x the product's flops / issued flops), else the per-block mma.sync kernel.
// Measured on B200 (4096-atom DZP cell, the nine products of an LNV call): the tiles issue 330-850
// TFLOP/s at useful fractions of 0.056-0.114 and the per-block kernel reaches 25-31 TFLOP/s useful;
// the tiles were faster for the product with fraction 0.114 (31.1 against 29.3) and slower below.
constexpr double kTileMinFill = 0.11;

void mat_mult_mixed(System& S, int mult_type, int ra, int rb, int rc, double* a, const double* b, double* c,
                    int parts) {
  MixedPlan& MP = get_mixed_plan(S, mult_type, ra, rb, rc);
  if (parts == 3) {
    mat_mult_split6(S, MP, mult_type, ra, rb, rc, a, b, c);
    return;
  }
  const bool tiles_ok = umma_usable(S, mult_type, ra, rb, rc);
  int k = S.mixed_kernel;
  if (k == 0 && !tiles_ok) k = 1;
  if (k < 0) {
    if (MP.kernel < 0) {
      MP.kernel = 1;
      if (tiles_ok) {
        const UmmaPlan& U = get_umma_plan(S, mult_type, ra, rb, rc);
        if (U.issued_flops > 0 && 3.0 * (double)U.flops / (double)U.issued_flops >= kTileMinFill) MP.kernel = 0;
      }
    }
    k = MP.kernel;
  }
  if (k == 0) mat_mult_umma(S, mult_type, ra, rb, rc, a, b, c);
  else mat_mult_mma_sync(S, MP, mult_type, ra, rb, rc, a, b, c);
}

static void ensure_groups(System& S, MixedPlan& MP, int gi) {
  static const int kGs[4] = {1, 2, 4, 8};
  if (MP.n_groups[gi] < 0) {
    // groups of up to G consecutive output blocks of one row
    RangeIndex& O = *S.ranges[MP.out_range];
    const int G = kGs[gi];
    std::vector<int2> grp;
    for (int p = 0; p < S.geo.n_prim; ++p)
      for (int s0 = O.h_row_ptr[p]; s0 < O.h_row_ptr[p + 1]; s0 += G)
        grp.push_back(make_int2(s0, std::min(G, O.h_row_ptr[p + 1] - s0)));
    MP.n_groups[gi] = (int)grp.size();
    MP.groups[gi].upload(grp, S.stream);
  }
}

static void launch_tc_g(System& S, MixedPlan& MP, TCArgs M, int gi) {
  ensure_groups(S, MP, gi);
  M.groups = MP.groups[gi].p;
  M.n_groups = MP.n_groups[gi];
  if (M.n_groups == 0) return;
  const int grid = (M.n_groups * 32 + 127) / 128;
  if (gi == 0) k_mult_tc1<<<grid, 128, 0, S.stream>>>(M);
  else if (gi == 1) k_mult_tc<2><<<grid, 128, 0, S.stream>>>(M);
  else if (gi == 2) k_mult_tc<4><<<grid, 128, 0, S.stream>>>(M);
  else k_mult_tc<8><<<grid, 128, 0, S.stream>>>(M);
  S.launches++;
  CQ_CUDA(cudaGetLastError());
}

void launch_mult_tc(System& S, MixedPlan& MP, const uint4* xa_hi, const uint4* xa_lo, const uint4* bb_hi,
                    const uint4* bb_lo, double* out) {
  RangeIndex& O = *S.ranges[MP.out_range];
  TCArgs M;
  M.ptr = MP.ptr;
  M.pairs = MP.pairs;
  M.xa_hi = xa_hi; M.xa_lo = xa_lo; M.bb_hi = bb_hi; M.bb_lo = bb_lo;
  M.xa_mid = nullptr; M.bb_mid = nullptr;
  M.o_row = O.nb_row.p; M.o_cover = O.nb_cover.p; M.o_elem = O.nb_elem.p;
  M.prim_nsf = S.dg.prim_nsf.p; M.cover_nsf = S.dg.cover_nsf.p;
  M.out = out;
  if (O.nnz == 0) return;
  if (MP.tuned_g < 0) {
    // autotuner: each group size once warm, then three interleaved timed rounds; the fastest
    // round counts, and a smaller group replaces a larger one only when it is 5 % faster.  Every launch overwrites
    // the whole output with the same values.
    cudaEvent_t e0, e1;
    CQ_CUDA(cudaEventCreate(&e0));
    CQ_CUDA(cudaEventCreate(&e1));
    float best[4] = {1e30f, 1e30f, 1e30f, 1e30f};
    for (int gi = 0; gi < 4; ++gi) launch_tc_g(S, MP, M, gi);
    for (int round = 0; round < 3; ++round)
      for (int gi = 0; gi < 4; ++gi) {
        CQ_CUDA(cudaEventRecord(e0, S.stream));
        launch_tc_g(S, MP, M, gi);
        CQ_CUDA(cudaEventRecord(e1, S.stream));
        CQ_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        CQ_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        best[gi] = std::min(best[gi], ms);
      }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int pick = 3;
    for (int gi = 0; gi < 3; ++gi)
      if (best[gi] < 0.95f * best[pick]) pick = gi;
    for (int gi = 0; gi < 4; ++gi) MP.tune_ms[gi] = best[gi];
    MP.tuned_g = pick;
  }
  const int forced = S.split_group == 1 ? 0 : S.split_group == 2 ? 1 : S.split_group == 4 ? 2 : S.split_group == 8 ? 3 : -1;
  launch_tc_g(S, MP, M, forced >= 0 ? forced : MP.tuned_g);
}

}  // namespace cqb
