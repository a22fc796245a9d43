// FP64 block-sparse products on the pair lists built in index.cu.
//
// Output stationary: each output block is owned by one group of lanes (one
// lane per element) that walks the block's (operand, B) pair list in the
// reference's order, so every element sees exactly the operation sequence of
// the default kernel (src/multiply_kernel_default.f90:204-214 for type 1,
// 390-402 for type 2):
//   type 1  c(n1,n2) = sum over k (A-halo order) of sum_n3 a(n1,n3) * b(n3,n2)
//   type 2  a(n1,n3) = sum over j (B-neighbour order) of sum_n2 c(n1,n2) * b(n3,n2)
// With `exact` the multiply and the add of every term round separately, which
// reproduces the default kernel built without FMA contraction bit for bit.
// No atomics, no reduction trees: results are deterministic and independent of
// the launch shape.
//
// The bound is the L2/HBM traffic of the operand blocks (an nd x nd FP64 block
// pair per triple, 2 nd^3 flops): for nd = 4 this is 256 B per 128 flops.  The 4 x 4 kernels write
// their output blocks with streaming (evict-first) stores, and every kernel reads its pair list (8
// bytes per triple, each read once) with streaming loads: an output range and a pair list are often
// larger than L2 (the 42-bohr range of the 512-atom cell: 152 MB; the pair list of LS.L -> LSL: 272 MB)
// and would otherwise push the operand blocks, which every output block re-reads, out of L2.
#include <algorithm>
#include <memory>
#include <numeric>

#include "cq_internal.hpp"

namespace cqb {
namespace {

template <bool EXACT>
__device__ __forceinline__ double madd(double acc, double x, double y) {
  if (EXACT) return __dadd_rn(acc, __dmul_rn(x, y));
  return fma(x, y, acc);
}

struct MultArgs {
  const int64_t* __restrict__ ptr;   // [n_out+1]
  const int2* __restrict__ pairs;    // (x block, b block)
  int n_out;
  // output blocks
  const int* __restrict__ o_row;
  const int* __restrict__ o_cover;
  const int64_t* __restrict__ o_elem;
  // first operand blocks (type 1: A; type 2: the input c)
  const int* __restrict__ x_cover;
  const int64_t* __restrict__ x_elem;
  // B blocks
  const int64_t* __restrict__ b_elem;
  const int* __restrict__ b_cover;
  const int* __restrict__ prim_nsf;
  const int* __restrict__ cover_nsf;
  const double* __restrict__ x;
  const double* __restrict__ b;
  double* __restrict__ out;
};

// Generic block sizes (nd <= 16): one warp per output block, up to 8 elements per lane.
template <int TYPE, bool EXACT>
__global__ void __launch_bounds__(256) k_mult_generic(MultArgs M) {
  int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (q >= M.n_out) return;
  const int ndi = M.prim_nsf[M.o_row[q]];
  const int ndo = M.cover_nsf[M.o_cover[q]];    // type 1: nd_j ; type 2: nd_k
  const int ne = ndi * ndo;
  double acc[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) acc[r] = 0.0;
  const int64_t p0 = M.ptr[q], p1 = M.ptr[q + 1];
  for (int64_t t = p0; t < p1; ++t) {
    int2 pr = __ldcs(M.pairs + t);
    const double* X = M.x + M.x_elem[pr.x];
    const double* B = M.b + M.b_elem[pr.y];
    if (TYPE == 1) {
      const int ndk = M.cover_nsf[M.x_cover[pr.x]];
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        int e = lane + 32 * r;
        if (e < ne) {
          int n1 = e % ndi, n2 = e / ndi;
          double a = acc[r];
          for (int n3 = 0; n3 < ndk; ++n3) a = madd<EXACT>(a, X[n1 + ndi * n3], B[n3 + ndk * n2]);
          acc[r] = a;
        }
      }
    } else {
      const int ndj = M.cover_nsf[M.b_cover[pr.y]];
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        int e = lane + 32 * r;
        if (e < ne) {
          int n1 = e % ndi, n3 = e / ndi;
          double a = acc[r];
          for (int n2 = 0; n2 < ndj; ++n2) a = madd<EXACT>(a, X[n1 + ndi * n2], B[n3 + ndo * n2]);
          acc[r] = a;
        }
      }
    }
  }
  double* O = M.out + M.o_elem[q];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    int e = lane + 32 * r;
    if (e < ne) O[e] = acc[r];
  }
}

// 4 x 4 blocks (SZ basis): 16 lanes per output block, one element per lane.  Each lane
// loads its operand row/column as two 16-byte vectors per block; blocks are 128 B aligned.
template <int TYPE, bool EXACT>
__global__ void __launch_bounds__(256) k_mult_nd4(MultArgs M) {
  int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 4, l = threadIdx.x & 15;
  if (g >= M.n_out) return;
  const int n1 = l & 3, m = l >> 2;   // element (n1, m) of the output block
  double acc = 0.0;
  const int64_t p0 = M.ptr[g], p1 = M.ptr[g + 1];
  for (int64_t t = p0; t < p1; ++t) {
    int2 pr = __ldcs(M.pairs + t);
    const double* X = M.x + M.x_elem[pr.x];
    const double* B = M.b + M.b_elem[pr.y];
    if (TYPE == 1) {
      // c(n1,m) += sum_n3 a(n1,n3) b(n3,m): a row is strided, b column contiguous
      double2 b01 = __ldg(reinterpret_cast<const double2*>(B + 4 * m));
      double2 b23 = __ldg(reinterpret_cast<const double2*>(B + 4 * m + 2));
      acc = madd<EXACT>(acc, __ldg(X + n1), b01.x);
      acc = madd<EXACT>(acc, __ldg(X + n1 + 4), b01.y);
      acc = madd<EXACT>(acc, __ldg(X + n1 + 8), b23.x);
      acc = madd<EXACT>(acc, __ldg(X + n1 + 12), b23.y);
    } else {
      // a(n1,m) += sum_n2 c(n1,n2) b(m,n2)
      acc = madd<EXACT>(acc, __ldg(X + n1), __ldg(B + m));
      acc = madd<EXACT>(acc, __ldg(X + n1 + 4), __ldg(B + m + 4));
      acc = madd<EXACT>(acc, __ldg(X + n1 + 8), __ldg(B + m + 8));
      acc = madd<EXACT>(acc, __ldg(X + n1 + 12), __ldg(B + m + 12));
    }
  }
  M.out[M.o_elem[g] + l] = acc;
}

// 4 x 4 blocks, one thread per output block with the whole block in registers: per triple
// the thread streams both operand blocks (8 + 8 16-byte loads) and does 64 multiply-adds,
// so the load/arithmetic ratio is 8x lower than with one lane per element.  Block b of a
// uniform 4 x 4 range starts at element 16 b.
template <int TYPE, bool EXACT>
__global__ void __launch_bounds__(128) k_mult_nd4_tpb(MultArgs M) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= M.n_out) return;
  double acc[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) acc[e] = 0.0;
  const int64_t p0 = M.ptr[q], p1 = M.ptr[q + 1];
  for (int64_t t = p0; t < p1; ++t) {
    int2 pr = __ldcs(M.pairs + t);
    const double2* X2 = reinterpret_cast<const double2*>(M.x + 16 * (int64_t)pr.x);
    const double2* B2 = reinterpret_cast<const double2*>(M.b + 16 * (int64_t)pr.y);
    double x[16], b[16];
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      double2 xv = __ldg(X2 + v), bv = __ldg(B2 + v);
      x[2 * v] = xv.x; x[2 * v + 1] = xv.y;
      b[2 * v] = bv.x; b[2 * v + 1] = bv.y;
    }
    if (TYPE == 1) {
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int n1 = 0; n1 < 4; ++n1) {
          double a = acc[n1 + 4 * m];
#pragma unroll
          for (int n3 = 0; n3 < 4; ++n3) a = madd<EXACT>(a, x[n1 + 4 * n3], b[n3 + 4 * m]);
          acc[n1 + 4 * m] = a;
        }
    } else {
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int n1 = 0; n1 < 4; ++n1) {
          double a = acc[n1 + 4 * m];
#pragma unroll
          for (int n2 = 0; n2 < 4; ++n2) a = madd<EXACT>(a, x[n1 + 4 * n2], b[m + 4 * n2]);
          acc[n1 + 4 * m] = a;
        }
    }
  }
  double2* O2 = reinterpret_cast<double2*>(M.out + 16 * (int64_t)q);
#pragma unroll
  for (int v = 0; v < 8; ++v) __stcs(O2 + v, make_double2(acc[2 * v], acc[2 * v + 1]));
}

// 4 x 4 blocks, one thread per output block, the first operand's row staged in shared memory.
// A CTA owns up to 128 consecutive output blocks of one row i; every pair of those blocks reads
// its first operand from row i of that operand (A_ik for type 1, c_ij for type 2), so the row
// is copied into shared memory in chunks of CHUNK blocks with coalesced 16-byte loads, and each
// thread walks its pair list in order, taking the pairs whose operand lies in the current chunk
// (a pair list that goes back to an earlier chunk reads that block from global memory, so the
// order of the terms is never changed).  Only the B blocks come from L2 per pair.
template <int TYPE, bool EXACT, int CHUNK>
__global__ void __launch_bounds__(128) k_mult_nd4_rows(MultArgs M, const int4* __restrict__ tiles) {
  __shared__ double2 xs[CHUNK * 8];
  const int4 d = tiles[blockIdx.x];           // output blocks [d.x, d.y), operand row blocks [d.z, d.w)
  const int q = d.x + (int)threadIdx.x;
  int64_t t = 0, tend = 0;
  if (q < d.y) { t = M.ptr[q]; tend = M.ptr[q + 1]; }
  double acc[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) acc[e] = 0.0;
  const double2* X2g = reinterpret_cast<const double2*>(M.x);
  const double2* B2g = reinterpret_cast<const double2*>(M.b);
  for (int c0 = d.z; c0 < d.w; c0 += CHUNK) {
    const int c1 = min(c0 + CHUNK, d.w);
    __syncthreads();
    for (int v = threadIdx.x; v < (c1 - c0) * 8; v += blockDim.x) xs[v] = __ldg(X2g + (int64_t)c0 * 8 + v);
    __syncthreads();
    while (t < tend) {
      const int2 pr = __ldcs(M.pairs + t);
      if (pr.x >= c1) break;
      double x[16], b[16];
      const double2* B2 = B2g + (int64_t)pr.y * 8;
      if (pr.x >= c0) {
        const double2* X2 = xs + (pr.x - c0) * 8;
#pragma unroll
        for (int v = 0; v < 8; ++v) { double2 xv = X2[v]; x[2 * v] = xv.x; x[2 * v + 1] = xv.y; }
      } else {
        const double2* X2 = X2g + (int64_t)pr.x * 8;
#pragma unroll
        for (int v = 0; v < 8; ++v) { double2 xv = __ldg(X2 + v); x[2 * v] = xv.x; x[2 * v + 1] = xv.y; }
      }
#pragma unroll
      for (int v = 0; v < 8; ++v) { double2 bv = __ldg(B2 + v); b[2 * v] = bv.x; b[2 * v + 1] = bv.y; }
      if (TYPE == 1) {
#pragma unroll
        for (int m = 0; m < 4; ++m)
#pragma unroll
          for (int n1 = 0; n1 < 4; ++n1) {
            double a = acc[n1 + 4 * m];
#pragma unroll
            for (int n3 = 0; n3 < 4; ++n3) a = madd<EXACT>(a, x[n1 + 4 * n3], b[n3 + 4 * m]);
            acc[n1 + 4 * m] = a;
          }
      } else {
#pragma unroll
        for (int m = 0; m < 4; ++m)
#pragma unroll
          for (int n1 = 0; n1 < 4; ++n1) {
            double a = acc[n1 + 4 * m];
#pragma unroll
            for (int n2 = 0; n2 < 4; ++n2) a = madd<EXACT>(a, x[n1 + 4 * n2], b[m + 4 * n2]);
            acc[n1 + 4 * m] = a;
          }
      }
      ++t;
    }
  }
  if (q < d.y) {
    double2* O2 = reinterpret_cast<double2*>(M.out + 16 * (int64_t)q);
#pragma unroll
    for (int v = 0; v < 8; ++v) __stcs(O2 + v, make_double2(acc[2 * v], acc[2 * v + 1]));
  }
}

// 4 x 4 blocks, one thread per output block, operand blocks staged through shared memory by
// the whole warp.  A thread-per-block kernel that reads its own operand blocks issues 16-byte
// loads that touch 32 different blocks per warp instruction, which saturates the L1 on
// wavefronts long before the FP64 pipe is busy.  Here, per step, the warp first copies the 32
// (x, b) block pairs its lanes need with loads in which 8 consecutive lanes read one whole
// 128-byte block (4 blocks per instruction), stores them in padded shared memory (9 x 16 bytes
// per block: conflict-free 16-byte reads per quarter warp), then every lane does its own 4 x 4
// product in the reference order.  Output blocks are taken in `order` (descending pair count)
// so the lanes of a warp have pair lists of similar length.
constexpr int kStageStride = 9;   // double2 per staged 4 x 4 block (8 + 1 padding)

// One warp of the warp-staged 4 x 4 kernel: output slots [base, base + 32) of `order`, operand blocks
// staged through X and B (32 x kStageStride double2 each, this warp's own shared memory).
template <int TYPE, bool EXACT>
__device__ __forceinline__ void warp_nd4_staged(const MultArgs& M, const int* __restrict__ order, int base, double2* X,
                                                double2* B) {
  constexpr int kStride = kStageStride;
  const unsigned kFull = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int slot = base + lane;
  const bool has = slot < M.n_out;
  const int q = has ? order[slot] : 0;
  int64_t t = has ? M.ptr[q] : 0, tend = has ? M.ptr[q + 1] : 0;
  double acc[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) acc[e] = 0.0;
  const double2* Xg = reinterpret_cast<const double2*>(M.x);
  const double2* Bg = reinterpret_cast<const double2*>(M.b);
  const int chunk = lane & 7;
  int2 pr_next = t < tend ? __ldcs(M.pairs + t) : make_int2(-1, -1);   // pair of the next step, loaded a step ahead
  while (__any_sync(kFull, t < tend)) {
    const bool act = t < tend;
    const int2 pr = pr_next;
    pr_next = t + 1 < tend ? __ldcs(M.pairs + t + 1) : make_int2(-1, -1);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int src = 4 * j + (lane >> 3);
      const int xb = __shfl_sync(kFull, pr.x, src);
      const int bb = __shfl_sync(kFull, pr.y, src);
      if (xb >= 0) {
        X[src * kStride + chunk] = __ldg(Xg + (int64_t)xb * 8 + chunk);
        B[src * kStride + chunk] = __ldg(Bg + (int64_t)bb * 8 + chunk);
      }
    }
    __syncwarp();
    if (act) {
      double x[16], b[16];
#pragma unroll
      for (int v = 0; v < 8; ++v) {
        const double2 xv = X[lane * kStride + v], bv = B[lane * kStride + v];
        x[2 * v] = xv.x; x[2 * v + 1] = xv.y;
        b[2 * v] = bv.x; b[2 * v + 1] = bv.y;
      }
      if (TYPE == 1) {
#pragma unroll
        for (int m = 0; m < 4; ++m)
#pragma unroll
          for (int n1 = 0; n1 < 4; ++n1) {
            double a = acc[n1 + 4 * m];
#pragma unroll
            for (int n3 = 0; n3 < 4; ++n3) a = madd<EXACT>(a, x[n1 + 4 * n3], b[n3 + 4 * m]);
            acc[n1 + 4 * m] = a;
          }
      } else {
#pragma unroll
        for (int m = 0; m < 4; ++m)
#pragma unroll
          for (int n1 = 0; n1 < 4; ++n1) {
            double a = acc[n1 + 4 * m];
#pragma unroll
            for (int n2 = 0; n2 < 4; ++n2) a = madd<EXACT>(a, x[n1 + 4 * n2], b[m + 4 * n2]);
            acc[n1 + 4 * m] = a;
          }
      }
      ++t;
    }
    __syncwarp();
  }
  if (has) {
    double2* O2 = reinterpret_cast<double2*>(M.out + 16 * (int64_t)q);
#pragma unroll
    for (int v = 0; v < 8; ++v) __stcs(O2 + v, make_double2(acc[2 * v], acc[2 * v + 1]));
  }
}

template <int TYPE, bool EXACT>
__global__ void __launch_bounds__(128, 5) k_mult_nd4_warp(MultArgs M, const int* __restrict__ order) {
  __shared__ double2 sx[4][32 * kStageStride];
  __shared__ double2 sb[4][32 * kStageStride];
  const int warp = threadIdx.x >> 5;
  const int base = (blockIdx.x * 4 + warp) * 32;
  if (base >= M.n_out) return;                  // whole warp
  warp_nd4_staged<TYPE, EXACT>(M, order, base, sx[warp], sb[warp]);
}

// Uniform 4 x 4 blocks, one thread per output block, operand blocks staged by the bulk-copy (TMA)
// engine.  The warp-staged kernel spends per triple about two L1 wavefronts on its coalesced global
// loads, two on the shared-memory stores and two on each lane's shared-memory reads; here every lane
// issues two 128-byte cp.async.bulk copies (its X and B blocks) into its slot of the warp's stage,
// whose mbarrier counts the bytes, so only the reads of the staged blocks go through the load/store
// pipe.  Three stages per warp keep the copies of the next two steps in flight.  Every wait is bounded
// (about a second; the error word is set and the warp stops).  The arithmetic is the warp-staged
// kernel's, in the same order: the same bits.  Measured on the nine products of the 512-atom SZ LNV
// call it runs at 1.48 TFLOP/s against 3.65 for the warp-staged kernel: 68 M copies of 128 B in
// 2.59 ms on LS.L -> LSL is one copy per about 11 SM cycles, so the copy engine, not L1, bounds it.
constexpr int kBulkStages = 3;
constexpr int kBulkSlot = 144;            // bytes per staged block (128 + 16: conflict-free 16-byte reads)

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool warp_bar_wait(unsigned long long* bar, uint32_t parity, int* err) {
  const uint32_t a = smem_addr(bar);
  uint64_t t0 = 0;
  for (uint32_t it = 0;; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
    if ((it & 63) == 0) {
      uint64_t t;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
      if (it == 0) t0 = t;
      else if (t - t0 > 1000000000ull) { *(volatile int*)err = 1; return false; }
    }
  }
}

template <int TYPE, bool EXACT>
__global__ void __launch_bounds__(128, 2) k_mult_nd4_bulk(MultArgs M, const int* __restrict__ order, int* err) {
  extern __shared__ __align__(128) unsigned char bulk_smem[];
  __shared__ unsigned long long bars[4][kBulkStages];
  const unsigned kFull = 0xffffffffu;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int base = (blockIdx.x * 4 + warp) * 32;
  unsigned char* W = bulk_smem + (size_t)warp * kBulkStages * 64 * kBulkSlot;   // this warp's stages
  if (lane < kBulkStages)
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bars[warp][lane])) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncwarp();
  if (base >= M.n_out) return;                  // whole warp (nothing waits on its barriers)
  const int slot = base + lane;
  const bool has = slot < M.n_out;
  const int q = has ? order[slot] : 0;
  const int64_t t = has ? M.ptr[q] : 0;
  const int64_t tend = has ? M.ptr[q + 1] : 0;
  double acc[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) acc[e] = 0.0;
  const unsigned char* Xg = reinterpret_cast<const unsigned char*>(M.x);
  const unsigned char* Bg = reinterpret_cast<const unsigned char*>(M.b);
  // the copies of step s (the lane's pair t + s) into stage s % kBulkStages; lane 0 states the bytes
  // on the stage's barrier before any lane copies
  auto issue = [&](int s) {
    const int st = s % kBulkStages;
    const bool act = t + s < tend;
    const unsigned m = __ballot_sync(kFull, act);
    unsigned long long* bar = &bars[warp][st];
    if (lane == 0)
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(__popc(m) * 256u)
                   : "memory");
    __syncwarp();
    if (act) {
      const int2 pr = __ldcs(M.pairs + t + s);
      unsigned char* dst = W + ((size_t)st * 64 + 2 * lane) * kBulkSlot;
      asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], 128, [%2];" ::"r"(
                       smem_addr(dst)),
                   "l"(Xg + (int64_t)pr.x * 128), "r"(smem_addr(bar))
                   : "memory");
      asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], 128, [%2];" ::"r"(
                       smem_addr(dst + kBulkSlot)),
                   "l"(Bg + (int64_t)pr.y * 128), "r"(smem_addr(bar))
                   : "memory");
    }
  };
  int issued = 0, done = 0;                     // steps whose copies were issued / which were consumed
  for (; issued < kBulkStages - 1; ++issued) issue(issued);
  for (int s = 0; __any_sync(kFull, t + s < tend); ++s) {
    issue(issued++);
    const int st = s % kBulkStages;
    const bool ok = __all_sync(kFull, warp_bar_wait(&bars[warp][st], (s / kBulkStages) & 1, err));
    if (!ok) break;
    if (t + s < tend) {
      const double2* X2 = reinterpret_cast<const double2*>(W + ((size_t)st * 64 + 2 * lane) * kBulkSlot);
      const double2* B2 = reinterpret_cast<const double2*>(W + ((size_t)st * 64 + 2 * lane + 1) * kBulkSlot);
      double x[16], b[16];
#pragma unroll
      for (int v = 0; v < 8; ++v) {
        const double2 xv = X2[v], bv = B2[v];
        x[2 * v] = xv.x; x[2 * v + 1] = xv.y;
        b[2 * v] = bv.x; b[2 * v + 1] = bv.y;
      }
      if (TYPE == 1) {
#pragma unroll
        for (int m = 0; m < 4; ++m)
#pragma unroll
          for (int n1 = 0; n1 < 4; ++n1) {
            double a = acc[n1 + 4 * m];
#pragma unroll
            for (int n3 = 0; n3 < 4; ++n3) a = madd<EXACT>(a, x[n1 + 4 * n3], b[n3 + 4 * m]);
            acc[n1 + 4 * m] = a;
          }
      } else {
#pragma unroll
        for (int m = 0; m < 4; ++m)
#pragma unroll
          for (int n1 = 0; n1 < 4; ++n1) {
            double a = acc[n1 + 4 * m];
#pragma unroll
            for (int n2 = 0; n2 < 4; ++n2) a = madd<EXACT>(a, x[n1 + 4 * n2], b[m + 4 * n2]);
            acc[n1 + 4 * m] = a;
          }
      }
    }
    done = s + 1;
    __syncwarp();                               // the stage is read before step s + kBulkStages refills it
  }
  // steps issued but not consumed (the empty steps after the last pair, or the copies in flight when a
  // wait ran out): wait for them (bounded) before the CTA's shared memory is released
  for (int s = done; s < issued; ++s) warp_bar_wait(&bars[warp][s % kBulkStages], (s / kBulkStages) & 1, err);
  if (has) {
    double2* O2 = reinterpret_cast<double2*>(M.out + 16 * (int64_t)q);
#pragma unroll
    for (int v = 0; v < 8; ++v) __stcs(O2 + v, make_double2(acc[2 * v], acc[2 * v + 1]));
  }
}

// Uniform 4 x 4 blocks, four lanes per output block: lane m of a quad owns column m of the block
// (elements n1 + 4m, n1 = 0..3).  At each step the quad takes the next pair of its list: its lanes
// load the first-operand block with two coalesced 16-byte loads each into shared memory, all four
// read the whole block back (broadcast), and each lane loads the four B values of its column
// straight into registers.  Four times the lanes of k_mult_nd4_warp, for products with few output
// blocks and long pair lists (type 2 into the H and L ranges).  Every element keeps the order of
// its terms, so the results are the same bits.
template <int TYPE, bool EXACT>
__global__ void __launch_bounds__(128, 8) k_mult_nd4_quad(MultArgs M, const int* __restrict__ order) {
  constexpr int kStride = 9;                     // double2 per staged block (8 + 1 padding)
  __shared__ double2 sx[4][8 * kStride];
  const unsigned kFull = 0xffffffffu;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int qd = lane >> 2, m = lane & 3;
  const int base = (blockIdx.x * 4 + warp) * 8;  // first output slot of this warp
  if (base >= M.n_out) return;                   // whole warp
  const int slot = base + qd;
  const bool has = slot < M.n_out;
  const int q = has ? order[slot] : 0;
  int64_t t = has ? M.ptr[q] : 0;
  const int64_t tend = has ? M.ptr[q + 1] : 0;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  double2* X = sx[warp] + qd * kStride;          // this quad's staged block
  const double2* Xg = reinterpret_cast<const double2*>(M.x);
  const double2* Bg = reinterpret_cast<const double2*>(M.b);
  int2 pr_next = t < tend ? __ldcs(M.pairs + t) : make_int2(-1, -1);   // pair of the next step, loaded a step ahead
  while (__any_sync(kFull, t < tend)) {
    const bool act = t < tend;                   // uniform over the quad
    const int2 pr = pr_next;
    pr_next = t + 1 < tend ? __ldcs(M.pairs + t + 1) : make_int2(-1, -1);
    double bc[4];
    if (act) {
      X[m] = __ldg(Xg + (int64_t)pr.x * 8 + m);
      X[m + 4] = __ldg(Xg + (int64_t)pr.x * 8 + m + 4);
      if (TYPE == 1) {
        // B[n3 + 4m], n3 = 0..3: the four contiguous values of column m
        const double2 u = __ldg(Bg + (int64_t)pr.y * 8 + 2 * m), v = __ldg(Bg + (int64_t)pr.y * 8 + 2 * m + 1);
        bc[0] = u.x; bc[1] = u.y; bc[2] = v.x; bc[3] = v.y;
      } else {
        // B[m + 4 n2], n2 = 0..3: for each n2 the quad reads one 32-byte sector
        const double* Bb = M.b + (int64_t)pr.y * 16 + m;
#pragma unroll
        for (int n2 = 0; n2 < 4; ++n2) bc[n2] = __ldg(Bb + 4 * n2);
      }
    }
    __syncwarp();
    if (act) {
      double x[16];
#pragma unroll
      for (int v = 0; v < 8; ++v) {
        const double2 xv = X[v];
        x[2 * v] = xv.x; x[2 * v + 1] = xv.y;
      }
      // type 1: acc[n1] += sum_n3 x[n1 + 4 n3] B[n3 + 4m]; type 2: acc[n1] += sum_n2 x[n1 + 4 n2] B[m + 4 n2]
#pragma unroll
      for (int n1 = 0; n1 < 4; ++n1) {
        double a = acc[n1];
#pragma unroll
        for (int n = 0; n < 4; ++n) a = madd<EXACT>(a, x[n1 + 4 * n], bc[n]);
        acc[n1] = a;
      }
      ++t;
    }
    __syncwarp();
  }
  if (has) {
    double2* O2 = reinterpret_cast<double2*>(M.out + 16 * (int64_t)q) + 2 * m;
    __stcs(O2, make_double2(acc[0], acc[1]));
    __stcs(O2 + 1, make_double2(acc[2], acc[3]));
  }
}

// Any block sizes up to 16 (DZP 13 x 13, mixed SZ/DZP): one warp per output block, each lane a
// 4 x 2 register tile of the output block (rows 4rt..4rt+3, columns 2ct..2ct+1, lane = rt * nct + ct),
// so per term of the inner sum a lane loads 4 + 2 operand values for 8 multiply-adds instead of
// 2 per multiply-add.  The order of the terms of every element is unchanged.
template <int TYPE, bool EXACT>
__device__ __forceinline__ void warp_tile(const MultArgs& M, int q) {
  const int lane = threadIdx.x & 31;
  const int ndi = M.prim_nsf[M.o_row[q]];
  const int ndo = M.cover_nsf[M.o_cover[q]];     // type 1: nd_j ; type 2: nd_k
  const int nct = (ndo + 1) >> 1, nrt = (ndi + 3) >> 2;
  const int rt = lane / nct, ct = lane - rt * nct;
  const bool live = rt < nrt;                       // lanes beyond the tiles only keep the warp together
  int r[4], c[2];
#pragma unroll
  for (int i = 0; i < 4; ++i) r[i] = min(4 * rt + i, ndi - 1);     // clamped: in-bounds reads
#pragma unroll
  for (int j = 0; j < 2; ++j) c[j] = min(2 * ct + j, ndo - 1);
  double acc[4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i) { acc[i][0] = 0.0; acc[i][1] = 0.0; }
  const int64_t p0 = M.ptr[q], p1 = M.ptr[q + 1];
  if (live) {
    for (int64_t t = p0; t < p1; ++t) {
      const int2 pr = __ldcs(M.pairs + t);
      const double* X = M.x + M.x_elem[pr.x];
      const double* B = M.b + M.b_elem[pr.y];
      if (TYPE == 1) {
        const int ndk = M.cover_nsf[M.x_cover[pr.x]];
        for (int n3 = 0; n3 < ndk; ++n3) {
          double xv[4], bv[2];
#pragma unroll
          for (int i = 0; i < 4; ++i) xv[i] = __ldg(X + r[i] + ndi * n3);
#pragma unroll
          for (int j = 0; j < 2; ++j) bv[j] = __ldg(B + n3 + ndk * c[j]);
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) acc[i][j] = madd<EXACT>(acc[i][j], xv[i], bv[j]);
        }
      } else {
        const int ndj = M.cover_nsf[M.b_cover[pr.y]];
        for (int n2 = 0; n2 < ndj; ++n2) {
          double xv[4], bv[2];
#pragma unroll
          for (int i = 0; i < 4; ++i) xv[i] = __ldg(X + r[i] + ndi * n2);
#pragma unroll
          for (int j = 0; j < 2; ++j) bv[j] = __ldg(B + c[j] + ndo * n2);
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) acc[i][j] = madd<EXACT>(acc[i][j], xv[i], bv[j]);
        }
      }
    }
    double* O = M.out + M.o_elem[q];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int n1 = 4 * rt + i, n2 = 2 * ct + j;
        if (n1 < ndi && n2 < ndo) O[n1 + ndi * n2] = acc[i][j];
      }
  }
}

// FP64 on the tensor cores (DMMA, mma.sync.m8n8k4.f64): one warp per output block, the block padded to
// 16 x 16 as 2 x 2 tiles of 8 x 8, the contraction in steps of 4.  Per step a lane loads one element of
// each first-operand row tile (row g = lane / 4, column t = lane % 4 of the step) and one of each B column
// tile (row t, column g) straight from the block storage (zeros outside the blocks), and the warp issues
// four MMAs; C/D hold rows g, columns 2t and 2t + 1 of each tile.  The terms of an element are summed in
// FP64 by the tensor cores in the blocks' order, four at a time, so the result differs from the reference
// kernel's separate multiply and add in rounding only (about 1e-16 of sum |a||b|).
__device__ __forceinline__ void dmma_8x8x4(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

// One term's operands in DMMA fragment order: for k-step ks (contraction columns 4 ks .. 4 ks + 3) a
// lane holds element (row 8 i + g, column 4 ks + t) of the first operand for row tile i and element
// (row 4 ks + t, column 8 j + g) of the B operand for column tile j; zeros outside the blocks.
template <int TYPE>
__device__ __forceinline__ void dmma_load_term(const MultArgs& M, int2 pr, int ndi, int ndo, int g, int t,
                                               double (&av)[4][2], double (&bv)[4][2], int& nks) {
  const double* X = M.x + M.x_elem[pr.x];
  const double* B = M.b + M.b_elem[pr.y];
  const int ndk = TYPE == 1 ? M.cover_nsf[M.x_cover[pr.x]] : M.cover_nsf[M.b_cover[pr.y]];
  nks = (ndk + 3) >> 2;
#pragma unroll
  for (int ks = 0; ks < 4; ++ks) {
    const int kk = 4 * ks + t;
    const bool kin = kk < ndk;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int r = 8 * i + g;
      av[ks][i] = (kin && r < ndi) ? __ldg(X + r + ndi * kk) : 0.0;
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int c = 8 * j + g;
      // type 1: B(kk, c) of the nd_k x nd_j block; type 2: B(c, kk) of the nd_k x nd_j block (B^T)
      bv[ks][j] = (kin && c < ndo) ? __ldg(TYPE == 1 ? B + kk + ndk * c : B + c + ndo * kk) : 0.0;
    }
  }
}

// The next term's operands are loaded while the current term's MMAs run.
template <int TYPE>
__global__ void __launch_bounds__(128) k_mult_dmma(MultArgs M) {
  const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (q >= M.n_out) return;
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int ndi = M.prim_nsf[M.o_row[q]];
  const int ndo = M.cover_nsf[M.o_cover[q]];     // type 1: nd_j ; type 2: nd_k
  const int nrt = ndi > 8 ? 2 : 1, nct = ndo > 8 ? 2 : 1;
  double acc[2][2][2];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) { acc[i][j][0] = 0.0; acc[i][j][1] = 0.0; }
  const int64_t p0 = M.ptr[q], p1 = M.ptr[q + 1];
  double av[4][2], bv[4][2];
  int nks = 0;
  if (p0 < p1) dmma_load_term<TYPE>(M, __ldcs(M.pairs + p0), ndi, ndo, g, t, av, bv, nks);
  for (int64_t p = p0; p < p1; ++p) {
    double nav[4][2], nbv[4][2];
    int nnks = 0;
    if (p + 1 < p1) dmma_load_term<TYPE>(M, __ldcs(M.pairs + p + 1), ndi, ndo, g, t, nav, nbv, nnks);
#pragma unroll
    for (int ks = 0; ks < 4; ++ks)
      if (ks < nks) {
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
          for (int j = 0; j < 2; ++j)
            if (i < nrt && j < nct) dmma_8x8x4(acc[i][j], av[ks][i], bv[ks][j]);
      }
#pragma unroll
    for (int ks = 0; ks < 4; ++ks)
#pragma unroll
      for (int i = 0; i < 2; ++i) { av[ks][i] = nav[ks][i]; bv[ks][i] = nbv[ks][i]; }
    nks = nnks;
  }
  double* O = M.out + M.o_elem[q];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int r = 8 * i + g, c = 8 * j + 2 * t + e;
        if (r < ndi && c < ndo) O[r + ndi * c] = acc[i][j][e];
      }
}

template <int TYPE, bool EXACT>
__global__ void __launch_bounds__(256) k_mult_tile(MultArgs M) {
  const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (q >= M.n_out) return;
  warp_tile<TYPE, EXACT>(M, q);
}

// Many independent products in one persistent launch (the concatenation of their output-block
// lists): every warp takes work units u = warp id, warp id + warps in the grid, ...; a unit is 32
// output slots of a uniform 4 x 4 product (the warp-staged kernel) or one output block of any other
// product (the register-tiled kernel).  Each output block is computed by exactly the operations of the
// single-product kernels, so the results are the same bits as separate launches.  The product table
// travels in the kernel's parameters (no host-to-device copy before the launch).
struct BatchProduct {
  MultArgs M;
  const int* order;                // 4 x 4 products: output blocks by descending pair count
  int kind;                        // bit 0: type 2, bit 1: exact rounding, bit 2: uniform 4 x 4 blocks
};
constexpr int kBatchMax = 96;      // products per launch (the table stays within the 32 KB parameter space)
struct BatchParams {
  int n_prod;
  int unit_off[kBatchMax + 1];     // first work unit of each product; unit_off[n_prod] = all units
  BatchProduct prods[kBatchMax];
};
static_assert(sizeof(BatchParams) < 32000, "batched product table exceeds the kernel parameter space");

__global__ void __launch_bounds__(128, 5) k_mult_batch(const __grid_constant__ BatchParams B) {
  __shared__ double2 sx[4][32 * kStageStride];
  __shared__ double2 sb[4][32 * kStageStride];
  const int warp = threadIdx.x >> 5;
  const int n_units = B.unit_off[B.n_prod];
  for (int u = blockIdx.x * 4 + warp; u < n_units; u += gridDim.x * 4) {
    int lo = 0, hi = B.n_prod - 1;               // product of unit u: last p with unit_off[p] <= u
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (B.unit_off[mid] <= u) lo = mid; else hi = mid - 1;
    }
    const BatchProduct& P = B.prods[lo];
    const int kind = P.kind;
    const int first = (u - B.unit_off[lo]) * ((kind & 4) ? 32 : 1);
    switch (kind) {
      case 0: warp_tile<1, false>(P.M, first); break;
      case 1: warp_tile<2, false>(P.M, first); break;
      case 2: warp_tile<1, true>(P.M, first); break;
      case 3: warp_tile<2, true>(P.M, first); break;
      case 4: warp_nd4_staged<1, false>(P.M, P.order, first, sx[warp], sb[warp]); break;
      case 5: warp_nd4_staged<2, false>(P.M, P.order, first, sx[warp], sb[warp]); break;
      case 6: warp_nd4_staged<1, true>(P.M, P.order, first, sx[warp], sb[warp]); break;
      default: warp_nd4_staged<2, true>(P.M, P.order, first, sx[warp], sb[warp]); break;
    }
  }
}

// One drop-in m_kern_max (type 1) / m_kern_min (type 2) call: output blocks with explicit
// offsets, accumulated in place in the layouts mat_mult passes (type 1 reads the local
// transpose a(n3 + nd3*n1); type 2 accumulates into it).  One warp per output block.
__global__ void __launch_bounds__(256) k_dropin(int type, const int64_t* __restrict__ out_off, const int* __restrict__ dims,
                                                const int64_t* __restrict__ ptr, const int64_t* __restrict__ pairs, int n_out,
                                                const double* __restrict__ x, const double* __restrict__ b,
                                                double* __restrict__ out) {
  int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (q >= n_out) return;
  const int r = dims[2 * q], cols = dims[2 * q + 1], ne = r * cols;
  double* O = out + out_off[q];
  for (int e = lane; e < ne; e += 32) {
    double acc = O[e];
    if (type == 1) {
      int n1 = e % r, n2 = e / r;
      for (int64_t t = ptr[q]; t < ptr[q + 1]; ++t) {
        const double* X = x + pairs[3 * t];
        const double* B = b + pairs[3 * t + 1];
        int nd3 = (int)pairs[3 * t + 2];
        for (int n3 = 0; n3 < nd3; ++n3) acc = madd<true>(acc, X[n3 + nd3 * n1], B[n3 + nd3 * n2]);
      }
    } else {
      int n3 = e % cols, n1 = e / cols;   // atrans block: nd3 x nd1, n3 fastest
      for (int64_t t = ptr[q]; t < ptr[q + 1]; ++t) {
        const double* X = x + pairs[3 * t];
        const double* B = b + pairs[3 * t + 1];
        int nd2 = (int)pairs[3 * t + 2];
        for (int n2 = 0; n2 < nd2; ++n2) acc = madd<true>(acc, X[n1 + r * n2], B[n3 + cols * n2]);
      }
    }
    O[e] = acc;
  }
}

}  // namespace

void launch_dropin(int type, const int64_t* d_out, const int* d_dims, const int64_t* d_ptr, const int64_t* d_pairs,
                   int n_out, const double* x, const double* b, double* out, cudaStream_t st) {
  if (n_out <= 0) return;
  int grid = (int)(((int64_t)n_out * 32 + 255) / 256);
  k_dropin<<<grid, 256, 0, st>>>(type, d_out, d_dims, d_ptr, d_pairs, n_out, x, b, out);
  CQ_CUDA(cudaGetLastError());
}

// output blocks by descending pair count (stable): lanes of a warp get similar list lengths
static void ensure_order(System& S, ProductPlan& P) {
  if (P.order.n != 0) return;
  std::vector<int64_t> ptr = P.ptr.download(S.stream);
  const int n_out = (int)ptr.size() - 1;
  std::vector<int> ord(std::max(n_out, 0));
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int u, int v) { return ptr[u + 1] - ptr[u] > ptr[v + 1] - ptr[v]; });
  P.order.upload(ord, S.stream);
}

// One launch of the FP64 product with kernel `variant` (0..3 and 5 for uniform 4 x 4 blocks with
// 16-byte aligned operands; anything else runs the generic kernel).  All variants give the same
// bits: they differ only in how the work is mapped onto the GPU.
static void launch_variant(System& S, ProductPlan& P, const MultArgs& M, int variant, int exact, bool nd4) {
  cudaStream_t st = S.stream;
  const int T = 256;
  RangeIndex& O = P.mult_type == 1 ? *S.ranges[P.rc] : *S.ranges[P.ra];
  RangeIndex& X = P.mult_type == 1 ? *S.ranges[P.ra] : *S.ranges[P.rc];
  if (nd4 && (variant == 3 || variant == 5 || variant == 6)) ensure_order(S, P);
  if (nd4 && variant == 6) {
    const int grid = (M.n_out + 127) / 128;
    const size_t smem = (size_t)4 * kBulkStages * 64 * kBulkSlot;
    int* err = device_timeout_word(S);
    auto launch = [&](auto kern) {
      CQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      kern<<<grid, 128, smem, st>>>(M, P.order.p, err);
    };
    if (P.mult_type == 1) {
      if (exact) launch(k_mult_nd4_bulk<1, true>); else launch(k_mult_nd4_bulk<1, false>);
    } else {
      if (exact) launch(k_mult_nd4_bulk<2, true>); else launch(k_mult_nd4_bulk<2, false>);
    }
  } else if (nd4 && variant == 5) {
    const int grid = (M.n_out + 31) / 32;        // 8 output blocks per warp, 4 warps per CTA
    if (P.mult_type == 1) {
      if (exact) k_mult_nd4_quad<1, true><<<grid, 128, 0, st>>>(M, P.order.p);
      else k_mult_nd4_quad<1, false><<<grid, 128, 0, st>>>(M, P.order.p);
    } else {
      if (exact) k_mult_nd4_quad<2, true><<<grid, 128, 0, st>>>(M, P.order.p);
      else k_mult_nd4_quad<2, false><<<grid, 128, 0, st>>>(M, P.order.p);
    }
  } else if (nd4 && variant == 3) {
    const int grid = (M.n_out + 127) / 128;
    if (P.mult_type == 1) {
      if (exact) k_mult_nd4_warp<1, true><<<grid, 128, 0, st>>>(M, P.order.p);
      else k_mult_nd4_warp<1, false><<<grid, 128, 0, st>>>(M, P.order.p);
    } else {
      if (exact) k_mult_nd4_warp<2, true><<<grid, 128, 0, st>>>(M, P.order.p);
      else k_mult_nd4_warp<2, false><<<grid, 128, 0, st>>>(M, P.order.p);
    }
  } else if (nd4 && variant == 2) {
    constexpr int kChunk = 256;                 // 32 KiB of operand blocks per chunk
    if (P.n_tiles == 0) {
      // tiles: up to 128 output blocks of one row, with that row's range of operand blocks
      std::vector<int4> tl;
      for (int i = 0; i < S.geo.n_prim; ++i)
        for (int q0 = O.h_row_ptr[i]; q0 < O.h_row_ptr[i + 1]; q0 += 128)
          tl.push_back(make_int4(q0, std::min(q0 + 128, O.h_row_ptr[i + 1]), X.h_row_ptr[i], X.h_row_ptr[i + 1]));
      P.tiles.upload(tl, st);
      P.n_tiles = (int)tl.size();
    }
    if (P.mult_type == 1) {
      if (exact) k_mult_nd4_rows<1, true, kChunk><<<P.n_tiles, 128, 0, st>>>(M, P.tiles.p);
      else k_mult_nd4_rows<1, false, kChunk><<<P.n_tiles, 128, 0, st>>>(M, P.tiles.p);
    } else {
      if (exact) k_mult_nd4_rows<2, true, kChunk><<<P.n_tiles, 128, 0, st>>>(M, P.tiles.p);
      else k_mult_nd4_rows<2, false, kChunk><<<P.n_tiles, 128, 0, st>>>(M, P.tiles.p);
    }
  } else if (nd4 && variant == 1) {
    const int T1 = 128;
    int grid = (M.n_out + T1 - 1) / T1;
    if (P.mult_type == 1) {
      if (exact) k_mult_nd4_tpb<1, true><<<grid, T1, 0, st>>>(M); else k_mult_nd4_tpb<1, false><<<grid, T1, 0, st>>>(M);
    } else {
      if (exact) k_mult_nd4_tpb<2, true><<<grid, T1, 0, st>>>(M); else k_mult_nd4_tpb<2, false><<<grid, T1, 0, st>>>(M);
    }
  } else if (nd4) {
    int grid = (int)(((int64_t)M.n_out * 16 + T - 1) / T);
    if (P.mult_type == 1) {
      if (exact) k_mult_nd4<1, true><<<grid, T, 0, st>>>(M); else k_mult_nd4<1, false><<<grid, T, 0, st>>>(M);
    } else {
      if (exact) k_mult_nd4<2, true><<<grid, T, 0, st>>>(M); else k_mult_nd4<2, false><<<grid, T, 0, st>>>(M);
    }
  } else if (variant == 4) {
    int grid = (int)(((int64_t)M.n_out * 32 + T - 1) / T);
    if (P.mult_type == 1) {
      if (exact) k_mult_tile<1, true><<<grid, T, 0, st>>>(M); else k_mult_tile<1, false><<<grid, T, 0, st>>>(M);
    } else {
      if (exact) k_mult_tile<2, true><<<grid, T, 0, st>>>(M); else k_mult_tile<2, false><<<grid, T, 0, st>>>(M);
    }
  } else {
    int grid = (int)(((int64_t)M.n_out * 32 + T - 1) / T);
    if (P.mult_type == 1) {
      if (exact) k_mult_generic<1, true><<<grid, T, 0, st>>>(M); else k_mult_generic<1, false><<<grid, T, 0, st>>>(M);
    } else {
      if (exact) k_mult_generic<2, true><<<grid, T, 0, st>>>(M); else k_mult_generic<2, false><<<grid, T, 0, st>>>(M);
    }
  }
  S.launches++;
  CQ_CUDA(cudaGetLastError());
}

// Autotuner: on the first call of a product, time the candidate kernels (one warm launch each,
// then three rounds in which every candidate runs once between CUDA events on the system's
// stream; a candidate's time is its fastest round) and keep the fastest for the plan; a later
// candidate replaces the preferred one only when it is at least 5 % faster.  The candidates give identical
// bits and each fully overwrites the output, so tuning changes speed only; the last timed launch
// leaves the correct result.
static int tuned_variant(System& S, ProductPlan& P, const MultArgs& M, int exact, bool nd4) {
  if (P.tuned >= 0) return P.tuned;
  // candidates, the preferred kernel first: uniform 4x4 blocks: warp-staged, four lanes per
  // block, thread per block, 16 lanes per block (the last two the most parallel, for products with
  // few output blocks); other sizes: register-tiled, generic
  // (variant 6, the bulk-copy-staged kernel, is not a candidate: 2.4x slower than variant 3 on every
  // product of the 512-atom SZ chain, since one 128-byte bulk copy takes about 11 SM cycles)
  int cands[4];
  int nc = 0;
  if (nd4) { cands[0] = 3; cands[1] = 5; cands[2] = 1; cands[3] = 0; nc = 4; }
  else { cands[0] = 4; cands[1] = 0; nc = 2; }
  cudaEvent_t e0, e1;
  CQ_CUDA(cudaEventCreate(&e0));
  CQ_CUDA(cudaEventCreate(&e1));
  float best[4] = {1e30f, 1e30f, 1e30f, 1e30f};
  for (int c = 0; c < nc; ++c) launch_variant(S, P, M, cands[c], exact, nd4);
  for (int round = 0; round < 3; ++round)
    for (int c = 0; c < nc; ++c) {
      CQ_CUDA(cudaEventRecord(e0, S.stream));
      launch_variant(S, P, M, cands[c], exact, nd4);
      CQ_CUDA(cudaEventRecord(e1, S.stream));
      CQ_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      CQ_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      best[c] = std::min(best[c], ms);
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int pick = 0;
  for (int c = 1; c < nc; ++c)
    if (best[c] < 0.95f * best[pick]) pick = c;
  for (int c = 0; c < nc; ++c) P.tune_ms[cands[c]] = best[c];
  P.tuned = cands[pick];
  return P.tuned;
}

// kernel arguments of one product (roles of mat_mult: type 1 writes c from a, b; type 2 writes a from c, b);
// nd4: uniform 4 x 4 blocks with 16-byte aligned operands (the 4 x 4 kernels read 16-byte vectors)
static MultArgs product_args(System& S, ProductPlan& P, double* a, const double* b, double* c, bool* nd4) {
  RangeIndex &A = *S.ranges[P.ra], &B = *S.ranges[P.rb], &C = *S.ranges[P.rc];
  MultArgs M;
  M.ptr = P.ptr.p;
  M.pairs = P.pairs.p;
  M.b_elem = B.nb_elem.p;
  M.b_cover = B.nb_cover.p;
  M.prim_nsf = S.dg.prim_nsf.p;
  M.cover_nsf = S.dg.cover_nsf.p;
  M.b = b;
  RangeIndex& O = P.mult_type == 1 ? C : A;
  RangeIndex& X = P.mult_type == 1 ? A : C;
  M.n_out = O.nnz;
  M.o_row = O.nb_row.p; M.o_cover = O.nb_cover.p; M.o_elem = O.nb_elem.p;
  M.x_cover = X.nb_cover.p; M.x_elem = X.nb_elem.p;
  M.x = P.mult_type == 1 ? a : c;
  M.out = P.mult_type == 1 ? c : a;
  const bool aligned = ((uintptr_t)b % 16 == 0) && ((uintptr_t)M.x % 16 == 0) && ((uintptr_t)M.out % 16 == 0);
  *nd4 = S.uniform_nsf == 4 && aligned;
  return M;
}

void launch_mat_mult(System& S, ProductPlan& P, double* a, const double* b, double* c, int exact) {
  RangeIndex &A = *S.ranges[P.ra], &B = *S.ranges[P.rb], &C = *S.ranges[P.rc];
  bool nd4 = false;
  MultArgs M = product_args(S, P, a, b, c, &nd4);
  if (M.n_out == 0) return;
  cudaStream_t st = S.stream;
  cudaEvent_t ev0 = nullptr;
  if (S.prof.on) { ev0 = S.prof.get(); CQ_CUDA(cudaEventRecord(ev0, st)); }
  // fused multiply-add products of blocks larger than 8 x 8 run on the FP64 tensor cores: an m8n8k4 MMA
  // chains its four products into the accumulator as fused multiply-adds in k order, so the bits are
  // those of the CUDA-core kernels (checked on B200), about three times faster on 13 x 13 blocks
  // (unless a CUDA-core variant is forced with CQ_OPT_MULT_VARIANT)
  if (exact == kPrecFp64Tensor || (exact == 0 && S.max_nsf > 8 && S.mult_variant == kVariantAuto)) {
    const int grid = (M.n_out * 32 + 127) / 128;
    if (P.mult_type == 1) k_mult_dmma<1><<<grid, 128, 0, st>>>(M);
    else k_mult_dmma<2><<<grid, 128, 0, st>>>(M);
    S.launches++;
    CQ_CUDA(cudaGetLastError());
  } else {
    int variant = S.mult_variant;
    if (variant == kVariantAuto) variant = tuned_variant(S, P, M, exact, nd4);
    launch_variant(S, P, M, variant, exact, nd4);
  }
  if (S.prof.on) {
    cudaEvent_t ev1 = S.prof.get();
    CQ_CUDA(cudaEventRecord(ev1, st));
    // algorithmic bytes: read both operands once, write the result once (8 bytes per element)
    double bytes = 8.0 * (double)(A.length + B.length + C.length);
    S.prof.recs.push_back({ev0, ev1, bytes, (double)P.flops});
  }
}

void ensure_product_order(System& S, ProductPlan& P) {
  if (S.uniform_nsf == 4) ensure_order(S, P);
}

// Products of independent systems (or of one system) in persistent launches on `st` (up to kBatchMax
// products each).  The caller orders `st` after the work the operands depend on and the systems' later
// work after it.
void launch_mat_mult_batch(const std::vector<BatchItem>& items, cudaStream_t st) {
  int dev_id = 0, sms = 0, occ = 0;
  CQ_CUDA(cudaGetDevice(&dev_id));
  CQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_id));
  CQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_mult_batch, 128, 0));
  auto params = std::make_unique<BatchParams>();
  BatchParams& B = *params;
  auto flush = [&] {
    if (B.n_prod == 0) return;
    const int n_units = B.unit_off[B.n_prod];
    const int grid = std::max(1, std::min(sms * std::max(occ, 1), (n_units + 3) / 4));
    k_mult_batch<<<grid, 128, 0, st>>>(B);
    CQ_CUDA(cudaGetLastError());
    B.n_prod = 0;
  };
  B.n_prod = 0;
  B.unit_off[0] = 0;
  for (const BatchItem& it : items) {
    System& S = *it.S;
    ProductPlan& P = *it.P;
    bool nd4 = false;
    BatchProduct bp;
    bp.M = product_args(S, P, it.a, it.b, it.c, &nd4);
    if (bp.M.n_out == 0) continue;
    if (nd4) ensure_order(S, P);
    bp.order = nd4 ? P.order.p : nullptr;
    bp.kind = (P.mult_type == 2 ? 1 : 0) | (it.exact ? 2 : 0) | (nd4 ? 4 : 0);
    if (B.n_prod == kBatchMax) { flush(); B.unit_off[0] = 0; }
    B.prods[B.n_prod] = bp;
    B.unit_off[B.n_prod + 1] = B.unit_off[B.n_prod] + (nd4 ? (bp.M.n_out + 31) / 32 : bp.M.n_out);
    ++B.n_prod;
    S.launches++;
  }
  flush();
}

cudaEvent_t ProductProfile::get() {
  if (!spare.empty()) { cudaEvent_t e = spare.back(); spare.pop_back(); return e; }
  cudaEvent_t e;
  CQ_CUDA(cudaEventCreate(&e));
  return e;
}
void ProductProfile::clear() {
  for (auto& r : recs) { spare.push_back(r.a); spare.push_back(r.b); }
  recs.clear();
}
ProductProfile::~ProductProfile() {
  clear();
  for (cudaEvent_t e : spare) cudaEventDestroy(e);
}

}  // namespace cqb
