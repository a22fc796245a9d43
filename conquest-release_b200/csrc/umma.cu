// Split-precision block products on the 5th-generation tensor cores (tcgen05.mma, TMEM accumulators).
//
// The atom-block product C(i,j) = sum_k A(i,k) B(k,j) (type 1, src/multiply_kernel_default.f90:204-214;
// type 2 a(i,k) = sum_j c(i,j) b(k,j)^T, :390-402) is regrouped into dense tiles:
//   rows        a run of consecutive primary atoms whose block sizes add up to at most 128 (M = 128),
//   columns     a run of output column atoms (the output range's cover atoms of those rows, in cover
//               order) adding up to at most kNT orbitals (N = kNT),
//   contraction the cover atoms k (type 1) or j (type 2) that occur in the tile's pair lists, packed
//               back to back along K (no padding between atoms).
// Each tile is one CTA.  Eight producer warps gather the FP64 blocks of a K chunk (kKC orbitals)
// from HBM/L2, split every value v = hi + lo into two bf16 parts (hi = bf16(v), lo = bf16(v - hi),
// about 16 significant bits) and store them in shared memory in the tensor core's K-major canonical
// layout (8-row x 16-byte core matrices, no swizzle); absent blocks are stored as zeros.  One thread
// issues per 16-wide K step the three MMAs lo.hi + hi.lo + hi.hi (kind::f16, bf16 inputs, FP32
// accumulation) into a 128 x kNT FP32 accumulator in tensor memory; a tcgen05.commit per chunk
// frees its shared-memory stage.  Four warps then read the accumulator back with tcgen05.ld and
// write every stored output block of the tile as FP64 (the whole block is overwritten, as the FP64
// kernels do).  Pairs absent from the pair lists contribute zero blocks, so the tile computes exactly
// the sum over the (i, k, j) triples of the reference kernel, in a different order and precision.
//
// Every wait on an mbarrier is bounded (about one second of GPU time); a wait that runs out sets an
// error word in mapped host memory, the kernel still drains the MMAs it issued before releasing
// the tensor memory, and the host reports CQ_ERR_TIMEOUT.
#include <cuda_bf16.h>

#include <algorithm>
#include <numeric>

#include "cq_internal.hpp"

namespace cqb {

namespace {

constexpr int kM = 128;             // accumulator rows (TMEM lanes)
constexpr int kNT = 128;            // accumulator columns
constexpr int kKC = 32;             // K orbitals per pipeline stage (two 16-wide MMA steps)
constexpr int kStages = 3;
constexpr int kProducerWarps = 8;
constexpr int kProducers = 32 * kProducerWarps;
constexpr int kThreads = kProducers + 32;   // + one warp: TMEM allocation and MMA issue
constexpr int kMaxRowAtoms = 32;    // block sizes >= 4: at most 32 atoms per 128 rows / columns
constexpr int kMinNd = 4;
constexpr int kMaxChunkAtoms = kKC / kMinNd + 2;
constexpr uint32_t kTmemCols = kNT;

// operand tiles of one stage: A (rows x K) and B (columns x K), bf16 hi and lo parts, K-major core matrices
constexpr int kTileBytesA = kM * kKC * 2;
constexpr int kTileBytesB = kNT * kKC * 2;
constexpr int kStageBytes = 2 * kTileBytesA + 2 * kTileBytesB;

struct ChunkMeta {
  long long xo[kMaxChunkAtoms][kMaxRowAtoms];   // first element of X(i, c) for the chunk's atoms c (-1: absent)
  long long bo[kMaxChunkAtoms][kMaxRowAtoms];   // first element of the B block of (c, column atom)
  int cnd[kMaxChunkAtoms];                      // block size of each chunk atom
  unsigned short kmap[kKC];                     // K position -> (chunk atom, orbital), 0xffff = padding
};

struct Smem {
  alignas(1024) unsigned char stage[kStages][kStageBytes];
  ChunkMeta meta[2];
  unsigned int rowtab[kM];          // row m -> ii | n1 << 8 | nd << 16 (0xffffffff: unused row)
  unsigned int coltab[kNT];         // column -> jj | nn << 8 | nd << 16
  unsigned long long full[kStages], empty[kStages], accfull;
  unsigned int tmem_base;
  int abort;
};

// two CTAs per SM (228 KB of shared memory, 1 KB reserved per CTA), so that one CTA's epilogue and
// set-up overlap the other's MMAs; two 128-column accumulators fit the 512 TMEM columns with room
static_assert(sizeof(Smem) + 1024 <= 113 * 1024, "shared memory of the tensor-core product exceeds half an SM");

__device__ const double g_umma_zero = 0.0;   // load target of absent blocks (the loads stay unconditional)

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Wait for the phase with the given parity to complete; false once the CTA has aborted, or after
// `limit_ns` of GPU time (then the error word is set and the CTA aborts).
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, uint32_t parity, int* err, int* abort,
                                          uint64_t limit_ns = 1000000000ull) {
  const uint32_t a = smem_u32(bar);
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
    if (*(volatile int*)abort) return false;
    if ((it & 63) == 0) {
      const uint64_t t = global_ns();
      if (it == 0) t0 = t;
      else if (t - t0 > limit_ns) {
        *(volatile int*)err = 1;                  // plain store: the word is mapped host memory
        *(volatile int*)abort = 1;
        return false;
      }
    }
  }
}

// named barrier of the producer warps that also ORs a flag over them (a uniform decision)
__device__ __forceinline__ bool producers_any(bool flag) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.b32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)flag), "n"(kProducers)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// shared-memory matrix descriptor: K-major, no swizzle; lbo = byte distance of core matrices along K,
// sbo = byte distance of 8-row groups along M / N; bits 46-47 = 1 (tcgen05 descriptor version)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3fff) | ((uint64_t)((lbo >> 4) & 0x3fff) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3fff) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: FP32 accumulator, bf16 A and B, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// byte offset of the 16-byte K group g of row r in a K-major operand tile of kKC columns
__device__ __forceinline__ uint32_t core_off(int r, int g) { return ((r >> 3) * (kKC / 8) + g) * 128 + (r & 7) * 16; }

// v = hi + lo for 8 values: two 16-byte rows of bf16 (element e at bytes 2e, 2e+1)
__device__ __forceinline__ void split8(const float (&v)[8], uint4& hi, uint4& lo) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    __nv_bfloat162 hb = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
    const float2 hf = __bfloat1622float2(hb);
    __nv_bfloat162 lb = __floats2bfloat162_rn(v[2 * q] - hf.x, v[2 * q + 1] - hf.y);
    h[q] = *reinterpret_cast<uint32_t*>(&hb);
    l[q] = *reinterpret_cast<uint32_t*>(&lb);
  }
  hi = make_uint4(h[0], h[1], h[2], h[3]);
  lo = make_uint4(l[0], l[1], l[2], l[3]);
}

}  // namespace

struct UmmaArgs {
  const UmmaTile* __restrict__ tiles;
  const int* __restrict__ col_atoms;
  const int* __restrict__ c_atoms;
  const int* __restrict__ c_koff;
  const long long* __restrict__ xpanel;   // first element of X(i, c) per (contraction atom, row atom), -1: absent
  const long long* __restrict__ bpanel;   // first element of the B block per (contraction atom, column atom)
  const int* __restrict__ outmap;
  const int* __restrict__ prim_nsf;
  const int* __restrict__ cover_nsf;
  const int64_t* __restrict__ o_elem;
  const double* __restrict__ x;
  const double* __restrict__ b;
  double* __restrict__ out;
  int type;
  int* err;                        // mapped host word: a bounded wait ran out
};

__global__ void __launch_bounds__(kThreads, 2) k_mult_umma(UmmaArgs P) {
  extern __shared__ unsigned char smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const UmmaTile T = P.tiles[blockIdx.x];
  const int nchunk = (T.k_total + kKC - 1) / kKC;

  // ---- set-up: barriers, TMEM, row / column / output tables of the tile
  if (tid == kProducers) {
    for (int s = 0; s < kStages; ++s) { mbar_init(&sm.full[s], kProducers); mbar_init(&sm.empty[s], 1); }
    mbar_init(&sm.accfull, 1);
    sm.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kProducerWarps) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  for (int m = tid; m < kM; m += kThreads) {
    unsigned int v = 0xffffffffu;
    int off = 0;
    for (int ii = 0; ii < T.n_rows; ++ii) {
      const int nd = P.prim_nsf[T.row_first + ii];
      if (m < off + nd) { v = (unsigned)ii | ((unsigned)(m - off) << 8) | ((unsigned)nd << 16); break; }
      off += nd;
    }
    sm.rowtab[m] = v;
  }
  for (int n = tid; n < kNT; n += kThreads) {
    unsigned int v = 0xffffffffu;
    int off = 0;
    for (int jj = 0; jj < T.n_cols; ++jj) {
      const int nd = P.cover_nsf[P.col_atoms[T.col_off + jj]];
      if (n < off + nd) { v = (unsigned)jj | ((unsigned)(n - off) << 8) | ((unsigned)nd << 16); break; }
      off += nd;
    }
    sm.coltab[n] = v;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm.tmem_base;

  if (warp < kProducerWarps) {
    // ---- producers: gather, split and store one K chunk per stage.  The metadata of chunk c + 1
    // (element offsets of its blocks, K map) is loaded while chunk c's values are in flight, and
    // every thread issues all its value loads of a chunk before it uses any of them.
    int cur = 0;                                     // first contraction atom overlapping the next chunk
    auto load_meta = [&](int c, ChunkMeta& M) {
      const int k0 = c * kKC;
      while (cur + 1 < T.n_c && __ldg(P.c_koff + T.c_off + cur + 1) <= k0) ++cur;
      int nca = 0;                                   // atoms overlapping [k0, k0 + kKC)
      while (cur + nca < T.n_c && nca < kMaxChunkAtoms && __ldg(P.c_koff + T.c_off + cur + nca) < k0 + kKC) ++nca;
      const int nrc = T.n_rows + T.n_cols;
      for (int e = tid; e < nca * nrc; e += kProducers) {
        const int la = e / nrc, r = e - la * nrc;
        const int64_t cc = cur + la;
        if (r < T.n_rows) M.xo[la][r] = __ldg(P.xpanel + T.xp_off + cc * T.n_rows + r);
        else M.bo[la][r - T.n_rows] = __ldg(P.bpanel + T.bp_off + cc * T.n_cols + (r - T.n_rows));
      }
      if (tid < nca) M.cnd[tid] = P.cover_nsf[P.c_atoms[T.c_off + cur + tid]];
      if (tid < kKC) {
        const int kk = k0 + tid;
        unsigned short v = 0xffff;
        if (kk < T.k_total) {
          for (int la = nca - 1; la >= 0; --la) {
            const int ko = __ldg(P.c_koff + T.c_off + cur + la);
            if (ko <= kk) { v = (unsigned short)(la | ((kk - ko) << 8)); break; }
          }
        }
        M.kmap[tid] = v;
      }
    };
    constexpr int kItems = (kM + kNT) * (kKC / 8) / kProducers;   // items per thread per chunk
    static_assert((kM + kNT) * (kKC / 8) % kProducers == 0, "items must divide evenly over the producers");
    if (nchunk > 0) load_meta(0, sm.meta[0]);
    producers_any(false);
    for (int c = 0; c < nchunk; ++c) {
      const int s = c % kStages;
      const ChunkMeta& M = sm.meta[c & 1];
      // the stage is free once the MMAs that read it (chunk c - kStages) have completed
      const bool ok = c < kStages || mbar_wait(&sm.empty[s], ((c / kStages) - 1) & 1, P.err, &sm.abort);
      // items: A rows x 4 K groups, then B columns x 4 K groups; consecutive threads take consecutive rows
      double v[kItems][8];
#pragma unroll
      for (int q = 0; q < kItems; ++q) {
        const int it = tid + q * kProducers;
        const bool isA = it < kM * (kKC / 8);
        const int j = isA ? it : it - kM * (kKC / 8);
        const int rows = isA ? kM : kNT;
        const int r = j % rows, g = j / rows;
        const unsigned int info = isA ? sm.rowtab[r] : sm.coltab[r];
        const int idx = info & 0xff, pos = (info >> 8) & 0xff, nd = info >> 16;
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const unsigned short km = M.kmap[g * 8 + e];
          const double* p = &g_umma_zero;
          if (info != 0xffffffffu && km != 0xffff) {
            const int la = km & 0xff, n = km >> 8;
            if (isA) {
              const long long o = M.xo[la][idx];
              if (o >= 0) p = P.x + o + pos + (int64_t)nd * n;
            } else {
              const long long o = M.bo[la][idx];
              if (o >= 0) p = P.b + o + (P.type == 1 ? n + (int64_t)M.cnd[la] * pos : pos + (int64_t)nd * n);
            }
          }
          v[q][e] = __ldg(p);
        }
      }
      if (c + 1 < nchunk) load_meta(c + 1, sm.meta[(c + 1) & 1]);
      unsigned char* st = sm.stage[s];
#pragma unroll
      for (int q = 0; q < kItems; ++q) {
        const int it = tid + q * kProducers;
        const bool isA = it < kM * (kKC / 8);
        const int j = isA ? it : it - kM * (kKC / 8);
        const int rows = isA ? kM : kNT;
        const int r = j % rows, g = j / rows;
        float f[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) f[e] = (float)v[q][e];
        uint4 hi, lo;
        split8(f, hi, lo);
        unsigned char* base = st + (isA ? 0 : 2 * kTileBytesA);
        const int tb = isA ? kTileBytesA : kTileBytesB;
        *reinterpret_cast<uint4*>(base + core_off(r, g)) = hi;
        *reinterpret_cast<uint4*>(base + tb + core_off(r, g)) = lo;
      }
      fence_async_smem();
      mbar_arrive(&sm.full[s]);
      // publishes chunk c + 1's metadata; stops every producer together once a wait has failed
      if (producers_any(!ok)) break;
    }
  } else if (lane == 0) {
    // ---- MMA issue (one thread)
    constexpr uint32_t idesc = idesc_bf16(kM, kNT);
    int c = 0;
    for (; c < nchunk; ++c) {
      const int s = c % kStages;
      if (!mbar_wait(&sm.full[s], (c / kStages) & 1, P.err, &sm.abort)) break;
      tc_fence_after();
      const uint32_t a_hi = smem_u32(sm.stage[s]), a_lo = a_hi + kTileBytesA;
      const uint32_t b_hi = a_hi + 2 * kTileBytesA, b_lo = b_hi + kTileBytesB;
#pragma unroll
      for (int ks = 0; ks < kKC / 16; ++ks) {
        const uint32_t ko = ks * 256;            // two 16-byte K groups per 16-wide step
        const uint32_t sbo = (kKC / 8) * 128;
        const uint64_t dah = smem_desc(a_hi + ko, 128, sbo), dal = smem_desc(a_lo + ko, 128, sbo);
        const uint64_t dbh = smem_desc(b_hi + ko, 128, sbo), dbl = smem_desc(b_lo + ko, 128, sbo);
        umma_bf16(tmem, dal, dbh, idesc, (c > 0 || ks > 0) ? 1u : 0u);
        umma_bf16(tmem, dah, dbl, idesc, 1u);
        umma_bf16(tmem, dah, dbh, idesc, 1u);
      }
      umma_commit(&sm.empty[s]);
    }
    // completion of every MMA issued above (also on the error path, before TMEM is released)
    umma_commit(&sm.accfull);
  }

  // ---- epilogue (warps 0-3: TMEM lane quarter = warp): accumulator -> FP64 output blocks
  if (warp < 4) {
    bool have = nchunk > 0 && mbar_wait(&sm.accfull, 0, P.err, &sm.abort, 2000000000ull);
    have = __all_sync(0xffffffffu, have && !*(volatile int*)&sm.abort);   // tcgen05.ld is warp-wide
    tc_fence_after();
    const int m = warp * 32 + lane;
    const unsigned int ri = sm.rowtab[m];
    for (int cb = 0; cb < kNT / 16; ++cb) {
      uint32_t r[16];
      if (have) tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + cb * 16, r);
      else {
#pragma unroll
        for (int e = 0; e < 16; ++e) r[e] = 0u;
      }
      if (ri == 0xffffffffu) continue;
      const int ii = ri & 0xff, n1 = (ri >> 8) & 0xff, ndi = ri >> 16;
      int jj_prev = -1;
      long long base = -1;
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const unsigned int ci = sm.coltab[cb * 16 + e];
        if (ci == 0xffffffffu) continue;
        const int jj = ci & 0xff, nn = (ci >> 8) & 0xff;
        if (jj != jj_prev) {
          const int q = __ldg(P.outmap + T.om_off + ii * T.n_cols + jj);
          base = q >= 0 ? (long long)P.o_elem[q] : -1ll;
          jj_prev = jj;
        }
        if (base >= 0) P.out[base + n1 + (int64_t)ndi * nn] = (double)__uint_as_float(r[e]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kProducerWarps) {
    tc_fence_after();
    // after an aborted pipeline the epilogue may not have seen the MMAs complete: wait for them (bounded)
    // before the tensor memory is released
    if (nchunk > 0 && *(volatile int*)&sm.abort) {
      int dummy = 0;
      mbar_wait(&sm.accfull, 0, P.err, &dummy, 2000000000ull);
      __syncwarp();
    }
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// ---------------------------------------------------------------------------
// tile plan (built once per product from its FP64 pair lists)
// ---------------------------------------------------------------------------
namespace {

// one warp per output block: mark the contraction atoms its pairs use in the tile's bit set
__global__ void k_umma_mark(int n_out, const int64_t* __restrict__ ptr, const int2* __restrict__ pairs,
                            const int2* __restrict__ q_tile, const int* __restrict__ xh,
                            const int64_t* __restrict__ mark_off, unsigned int* __restrict__ mark) {
  const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (q >= n_out) return;
  const int t = q_tile[q].x;
  const int64_t mo = mark_off[t];
  for (int64_t p = ptr[q] + lane; p < ptr[q + 1]; p += 32) {
    const int64_t bit = mo + xh[pairs[p].x];
    atomicOr(mark + (bit >> 5), 1u << (bit & 31));
  }
}

// one thread per tile: contraction atom list, their K offsets and the tile's K extent; per-word prefix counts
__global__ void k_umma_clist(int n_tiles, UmmaTile* __restrict__ tiles, const int64_t* __restrict__ mark_off,
                             const int* __restrict__ mark_bits, const unsigned int* __restrict__ mark,
                             const int* __restrict__ u_atoms, const int64_t* __restrict__ u_off,
                             const int* __restrict__ tile_group, const int* __restrict__ cover_nsf,
                             int* __restrict__ wpre, int* __restrict__ c_atoms, int* __restrict__ c_koff) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_tiles) return;
  UmmaTile& T = tiles[t];
  const int64_t w0 = mark_off[t] >> 5;
  const int nw = (mark_bits[t] + 31) >> 5;
  const int* U = u_atoms + u_off[tile_group[t]];
  int cnt = 0, k = 0;
  for (int w = 0; w < nw; ++w) {
    wpre[w0 + w] = cnt;
    unsigned int m = mark[w0 + w];
    while (m) {
      const int b = __ffs(m) - 1;
      m &= m - 1;
      if (c_atoms) {
        const int atom = U[32 * w + b];
        c_atoms[T.c_off + cnt] = atom;
        c_koff[T.c_off + cnt] = k;
        k += cover_nsf[atom];
      }
      ++cnt;
    }
  }
  if (c_atoms) T.k_total = k;
  else T.n_c = cnt;
}

// one warp per output block: panel entries of its pairs
__global__ void k_umma_scatter(int n_out, const int64_t* __restrict__ ptr, const int2* __restrict__ pairs,
                               const int2* __restrict__ q_tile, const int* __restrict__ xh,
                               const int64_t* __restrict__ mark_off, const unsigned int* __restrict__ mark,
                               const int* __restrict__ wpre, const UmmaTile* __restrict__ tiles,
                               const int64_t* __restrict__ x_elem, const int64_t* __restrict__ b_elem,
                               long long* __restrict__ xpanel, long long* __restrict__ bpanel) {
  const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (q >= n_out) return;
  const int2 tq = q_tile[q];
  const int t = tq.x, ii = tq.y & 0xffff, jj = tq.y >> 16;
  const UmmaTile& T = tiles[t];
  const int64_t mo = mark_off[t];
  for (int64_t p = ptr[q] + lane; p < ptr[q + 1]; p += 32) {
    const int2 pr = pairs[p];
    const int64_t bit = mo + xh[pr.x];
    const int64_t w = bit >> 5;
    const int pos = wpre[w] + __popc(mark[w] & ((1u << (bit & 31)) - 1u));
    xpanel[T.xp_off + (int64_t)pos * T.n_rows + ii] = x_elem[pr.x];
    bpanel[T.bp_off + (int64_t)pos * T.n_cols + jj] = b_elem[pr.y];
  }
}

}  // namespace

UmmaPlan& get_umma_plan(System& S, int mult_type, int ra, int rb, int rc) {
  auto key = std::make_tuple(mult_type, ra, rb, rc);
  auto it = S.uplans.find(key);
  if (it != S.uplans.end()) return *it->second;
  ProductPlan& P = get_plan(S, mult_type, ra, rb, rc);
  auto up = std::make_unique<UmmaPlan>();
  UmmaPlan& U = *up;
  U.flops = P.flops;
  U.n_pairs = P.n_pairs;
  cudaStream_t st = S.stream;
  RangeIndex& O = mult_type == 1 ? *S.ranges[rc] : *S.ranges[ra];
  RangeIndex& X = mult_type == 1 ? *S.ranges[ra] : *S.ranges[rc];
  const Geometry& g = S.geo;
  const int np = g.n_prim;
  std::vector<int> nd_prim(np);
  for (int p = 0; p < np; ++p) nd_prim[p] = g.nsf[g.prim_global[p]];
  U.usable = true;
  for (int p = 0; p < np; ++p) U.usable = U.usable && nd_prim[p] >= kMinNd && nd_prim[p] <= kM;
  for (int c = 0; c < g.n_cover_atoms; ++c) U.usable = U.usable && g.cover_nsf[c] >= kMinNd && g.cover_nsf[c] <= kNT;
  if (!U.usable || O.nnz == 0) {
    auto res = S.uplans.emplace(key, std::move(up));
    return *res.first->second;
  }
  // host copies of the output and first-operand neighbour lists
  std::vector<int> ocov(O.nnz), xcov(std::max(X.nnz, 1));
  CQ_CUDA(cudaMemcpyAsync(ocov.data(), O.nb_cover.p, sizeof(int) * O.nnz, cudaMemcpyDeviceToHost, st));
  if (X.nnz) CQ_CUDA(cudaMemcpyAsync(xcov.data(), X.nb_cover.p, sizeof(int) * X.nnz, cudaMemcpyDeviceToHost, st));
  CQ_CUDA(cudaStreamSynchronize(st));
  // row groups: consecutive primary atoms, at most kM rows
  std::vector<int> grp_first;
  for (int p = 0, rows = kM + 1; p < np; ++p) {
    if (rows + nd_prim[p] > kM) { grp_first.push_back(p); rows = 0; }
    rows += nd_prim[p];
  }
  grp_first.push_back(np);
  const int ng = (int)grp_first.size() - 1;
  std::vector<UmmaTile> tiles;
  std::vector<int> col_atoms, outmap, tile_group, mark_bits;
  std::vector<int2> q_tile(O.nnz);
  std::vector<int> xh(std::max(X.nnz, 1), 0);
  std::vector<int> u_atoms;
  std::vector<int64_t> u_off(ng + 1, 0), mark_off;
  int64_t mark_total = 0;
  for (int gi = 0; gi < ng; ++gi) {
    const int r0 = grp_first[gi], r1 = grp_first[gi + 1];
    // output columns of the group: sorted cover atoms of its rows, cut into runs of <= kNT orbitals
    std::vector<int> cols(ocov.begin() + O.h_row_ptr[r0], ocov.begin() + O.h_row_ptr[r1]);
    std::sort(cols.begin(), cols.end());
    cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
    std::vector<int> chunk_of(cols.size()), pos_in(cols.size());
    std::vector<int> chunk_first;
    for (size_t c = 0, w = kNT + 1, cnt = kMaxRowAtoms; c < cols.size(); ++c) {
      const int nd = g.cover_nsf[cols[c]];
      if (w + nd > (size_t)kNT || cnt == (size_t)kMaxRowAtoms) { chunk_first.push_back((int)c); w = 0; cnt = 0; }
      chunk_of[c] = (int)chunk_first.size() - 1;
      pos_in[c] = (int)(c - chunk_first.back());
      w += nd; ++cnt;
    }
    chunk_first.push_back((int)cols.size());
    // contraction candidates of the group: sorted cover atoms of the first operand's rows
    std::vector<int> cand(xcov.begin() + X.h_row_ptr[r0], xcov.begin() + X.h_row_ptr[r1]);
    std::sort(cand.begin(), cand.end());
    cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
    for (int e = X.h_row_ptr[r0]; e < X.h_row_ptr[r1]; ++e)
      xh[e] = (int)(std::lower_bound(cand.begin(), cand.end(), xcov[e]) - cand.begin());
    u_off[gi] = (int64_t)u_atoms.size();
    u_atoms.insert(u_atoms.end(), cand.begin(), cand.end());
    const int t0 = (int)tiles.size();
    for (size_t ch = 0; ch + 1 < chunk_first.size(); ++ch) {
      UmmaTile T{};
      T.row_first = r0;
      T.n_rows = r1 - r0;
      T.col_off = (int)col_atoms.size();
      T.n_cols = chunk_first[ch + 1] - chunk_first[ch];
      T.om_off = (int)outmap.size();
      for (int c = chunk_first[ch]; c < chunk_first[ch + 1]; ++c) col_atoms.push_back(cols[c]);
      outmap.resize(outmap.size() + (size_t)T.n_rows * T.n_cols, -1);
      tiles.push_back(T);
      tile_group.push_back(gi);
      mark_off.push_back(mark_total);
      mark_bits.push_back((int)cand.size());
      mark_total += ((int64_t)cand.size() + 31) / 32 * 32;
    }
    for (int p = r0; p < r1; ++p)
      for (int q = O.h_row_ptr[p]; q < O.h_row_ptr[p + 1]; ++q) {
        const int c = (int)(std::lower_bound(cols.begin(), cols.end(), ocov[q]) - cols.begin());
        const int t = t0 + chunk_of[c];
        const int ii = p - r0, jj = pos_in[c];
        q_tile[q] = make_int2(t, ii | (jj << 16));
        outmap[tiles[t].om_off + ii * tiles[t].n_cols + jj] = q;
      }
  }
  u_off[ng] = (int64_t)u_atoms.size();
  const int nt = (int)tiles.size();
  U.n_tiles = nt;
  DevBuf<int2> d_qt; d_qt.upload(q_tile, st);
  DevBuf<int> d_xh; d_xh.upload(xh, st);
  DevBuf<int64_t> d_moff; d_moff.upload(mark_off, st);
  DevBuf<int> d_mbits; d_mbits.upload(mark_bits, st);
  DevBuf<int> d_tg; d_tg.upload(tile_group, st);
  DevBuf<int> d_u; d_u.upload(u_atoms.empty() ? std::vector<int>{0} : u_atoms, st);
  DevBuf<int64_t> d_uoff; d_uoff.upload(u_off, st);
  DevBuf<unsigned int> d_mark; d_mark.alloc(std::max<int64_t>(mark_total / 32, 1), st);
  CQ_CUDA(cudaMemsetAsync(d_mark.p, 0, sizeof(unsigned int) * d_mark.n, st));
  DevBuf<int> d_wpre; d_wpre.alloc(d_mark.n, st);
  U.tiles.upload(tiles, st);
  U.col_atoms.upload(col_atoms.empty() ? std::vector<int>{0} : col_atoms, st);
  U.outmap.upload(outmap.empty() ? std::vector<int>{-1} : outmap, st);
  const int T256 = 256;
  const int n_out = O.nnz;
  k_umma_mark<<<(int)(((int64_t)n_out * 32 + T256 - 1) / T256), T256, 0, st>>>(n_out, P.ptr.p, P.pairs.p, d_qt.p, d_xh.p,
                                                                               d_moff.p, d_mark.p);
  k_umma_clist<<<(nt + 127) / 128, 128, 0, st>>>(nt, U.tiles.p, d_moff.p, d_mbits.p, d_mark.p, d_u.p, d_uoff.p, d_tg.p,
                                                 S.dg.cover_nsf.p, d_wpre.p, nullptr, nullptr);
  CQ_CUDA(cudaGetLastError());
  // sizes of the contraction lists and panels
  CQ_CUDA(cudaMemcpyAsync(tiles.data(), U.tiles.p, sizeof(UmmaTile) * nt, cudaMemcpyDeviceToHost, st));
  CQ_CUDA(cudaStreamSynchronize(st));
  int64_t coff = 0, xoff = 0, boff = 0;
  for (auto& T : tiles) {
    T.c_off = (int)coff;
    T.xp_off = xoff;
    T.bp_off = boff;
    coff += T.n_c;
    xoff += (int64_t)T.n_c * T.n_rows;
    boff += (int64_t)T.n_c * T.n_cols;
  }
  CQ_CHECK(coff < (int64_t)1 << 31, CQ_ERR_BOUNDS, "tensor-core tile plan: contraction list too long");
  U.tiles.upload(tiles, st);
  U.c_atoms.alloc(std::max<int64_t>(coff, 1), st);
  U.c_koff.alloc(std::max<int64_t>(coff, 1), st);
  U.xpanel.alloc(std::max<int64_t>(xoff, 1), st);
  U.bpanel.alloc(std::max<int64_t>(boff, 1), st);
  CQ_CUDA(cudaMemsetAsync(U.xpanel.p, 0xff, sizeof(long long) * U.xpanel.n, st));
  CQ_CUDA(cudaMemsetAsync(U.bpanel.p, 0xff, sizeof(long long) * U.bpanel.n, st));
  k_umma_clist<<<(nt + 127) / 128, 128, 0, st>>>(nt, U.tiles.p, d_moff.p, d_mbits.p, d_mark.p, d_u.p, d_uoff.p, d_tg.p,
                                                 S.dg.cover_nsf.p, d_wpre.p, U.c_atoms.p, U.c_koff.p);
  k_umma_scatter<<<(int)(((int64_t)n_out * 32 + T256 - 1) / T256), T256, 0, st>>>(
      n_out, P.ptr.p, P.pairs.p, d_qt.p, d_xh.p, d_moff.p, d_mark.p, d_wpre.p, U.tiles.p, X.nb_elem.p,
      S.ranges[rb]->nb_elem.p, U.xpanel.p, U.bpanel.p);
  CQ_CUDA(cudaGetLastError());
  CQ_CUDA(cudaMemcpyAsync(tiles.data(), U.tiles.p, sizeof(UmmaTile) * nt, cudaMemcpyDeviceToHost, st));
  CQ_CUDA(cudaStreamSynchronize(st));
  U.issued_flops = 0;
  for (auto& T : tiles) U.issued_flops += 3ll * 2 * kM * kNT * (((int64_t)T.k_total + kKC - 1) / kKC * kKC);
  S.launches += 3;
  auto res = S.uplans.emplace(key, std::move(up));
  return *res.first->second;
}

static int* umma_err_word(System& S) {
  if (!S.umma_err_host) {
    CQ_CUDA(cudaHostAlloc((void**)&S.umma_err_host, sizeof(int), cudaHostAllocMapped));
    *S.umma_err_host = 0;
    CQ_CUDA(cudaHostGetDevicePointer((void**)&S.umma_err_dev, S.umma_err_host, 0));
  }
  return S.umma_err_dev;
}

bool umma_usable(System& S, int mult_type, int ra, int rb, int rc) {
  return get_umma_plan(S, mult_type, ra, rb, rc).usable;
}

void mat_mult_umma(System& S, int mult_type, int ra, int rb, int rc, double* a, const double* b, double* c) {
  UmmaPlan& U = get_umma_plan(S, mult_type, ra, rb, rc);
  CQ_CHECK(U.usable, CQ_ERR_ARG, "tensor-core tiles need block sizes of 4 to 128");
  if (U.n_tiles == 0) return;
  RangeIndex &A = *S.ranges[ra], &B = *S.ranges[rb], &C = *S.ranges[rc];
  RangeIndex& O = mult_type == 1 ? C : A;
  UmmaArgs M;
  M.tiles = U.tiles.p; M.col_atoms = U.col_atoms.p; M.c_atoms = U.c_atoms.p; M.c_koff = U.c_koff.p;
  M.xpanel = U.xpanel.p; M.bpanel = U.bpanel.p; M.outmap = U.outmap.p;
  M.prim_nsf = S.dg.prim_nsf.p; M.cover_nsf = S.dg.cover_nsf.p;
  M.o_elem = O.nb_elem.p;
  M.x = mult_type == 1 ? a : c;
  M.b = b;
  M.out = mult_type == 1 ? c : a;
  M.type = mult_type;
  M.err = umma_err_word(S);
  const size_t smem = sizeof(Smem) + 1024;
  CQ_CUDA(cudaFuncSetAttribute(k_mult_umma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  cudaEvent_t ev0 = nullptr;
  if (S.prof.on) { ev0 = S.prof.get(); CQ_CUDA(cudaEventRecord(ev0, S.stream)); }
  k_mult_umma<<<U.n_tiles, kThreads, smem, S.stream>>>(M);
  CQ_CUDA(cudaGetLastError());
  S.launches++;
  if (S.prof.on) {
    cudaEvent_t ev1 = S.prof.get();
    CQ_CUDA(cudaEventRecord(ev1, S.stream));
    S.prof.recs.push_back({ev0, ev1, 8.0 * (double)(A.length + B.length + C.length), (double)U.flops});
  }
}

void umma_check(System& S) {
  if (S.umma_err_host && *(volatile int*)S.umma_err_host) {
    *S.umma_err_host = 0;
    throw Error(CQ_ERR_TIMEOUT, "tensor-core product: a bounded pipeline wait ran out");
  }
}

size_t umma_smem_bytes() { return sizeof(Smem) + 1024; }

}  // namespace cqb
