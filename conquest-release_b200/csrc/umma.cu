// Split-precision block products on the 5th-generation tensor cores (tcgen05.mma, TMEM accumulators,
// operand tiles staged by the bulk-copy (TMA) engine).
//
// The atom-block product C(i,j) = sum_k A(i,k) B(k,j) (type 1, src/multiply_kernel_default.f90:204-214;
// type 2 a(i,k) = sum_j c(i,j) b(k,j)^T, :390-402) is regrouped into dense tiles:
//   rows        a run of consecutive primary atoms whose block sizes add up to at most 128 (M = 128);
//   columns     a column chunk: a run of consecutive cover atoms adding up to at most 128 orbitals
//               (N = 128), the same chunks for every row group;
//   contraction units: runs of consecutive cover atoms adding up to at most 16 orbitals (one
//               16-wide MMA step each: four 4x4 atoms, or one 13x13 atom padded to 16); a tile
//               contracts over the units that hold a contraction atom (k for type 1, j for type 2)
//               of its pair lists.
// Before each product, two packing kernels write the operands once as bf16 "slabs" in the tensor
// core's K-major shared-memory layout (8-row x 16-byte core matrices, no swizzle): an X slab per
// (row group, unit) holds the first operand's 128 rows x 16 K, a B slab per (unit, column chunk)
// the second operand's 128 columns x 16 K, each as a hi part (bf16(v)) and a lo part (bf16(v - hi)),
// about 16 significant bits; absent blocks are zeros.
// The product kernel is persistent, two CTAs per SM each walking its share of the tiles.  One thread moves
// the slabs of each pipeline stage into shared memory with cp.async.bulk (no multicast; 16 KB per unit,
// completion counted on an mbarrier), in one ring of three stages across the CTA's tiles; one thread
// issues per unit the three MMAs lo.hi + hi.lo + hi.hi (kind::f16, bf16 inputs, FP32 accumulation)
// into a 128 x 128 FP32 accumulator in tensor memory, a tcgen05.commit per stage frees it; the tiles
// alternate between two accumulators, so that while the MMAs of one tile run, four warps read the
// previous tile's accumulator back with tcgen05.ld and write every stored output block of it as FP64
// (the whole block is overwritten, as the FP64 kernels do).  Pairs absent from the
// pair lists contribute zero blocks, so a tile computes exactly the sums over the (i, k, j) triples of
// the reference kernel, in a different order and precision.
//
// Every wait on an mbarrier is bounded (about one second of GPU time); a wait that runs out sets an
// error word in mapped host memory, the kernel drains the copies and MMAs it issued before it releases
// the tensor memory, and the host reports CQ_ERR_TIMEOUT.
#include <cuda_bf16.h>

#include <algorithm>
#include <numeric>

#include "cq_internal.hpp"

namespace cqb {

namespace {

constexpr int kM = 128;             // accumulator rows (TMEM lanes)
constexpr int kNT = 128;            // accumulator columns
constexpr int kUK = 16;             // K orbitals of one contraction unit (one MMA step)
constexpr int kUnitsPerStage = 2;
constexpr int kStages = 3;
constexpr int kMaxAtoms = 32;       // atoms per row group / column chunk (block sizes >= 4)
constexpr int kMaxUnitAtoms = 4;
constexpr int kMinNd = 4;
constexpr uint32_t kTmemCols = 2 * kNT;   // two accumulators: one tile's epilogue overlaps the next one's MMAs
constexpr int kThreads = 192;       // warps 0-3 epilogue, warp 4 bulk copies, warp 5 TMEM + MMA

// one slab: hi part then lo part, each [K group (2)][row group (16)][8 rows x 16 bytes]
constexpr int kSlabHalf = kM * kUK * 2;          // 4 KB
constexpr int kSlabBytes = 2 * kSlabHalf;        // 8 KB
static_assert(kNT == kM, "B slabs use the X slab layout");
// stage: A hi, A lo, B hi, B lo regions of kUnitsPerStage slab halves each
constexpr int kRegion = kUnitsPerStage * kSlabHalf;
constexpr int kStageBytes = 4 * kRegion;

struct Smem {
  alignas(1024) unsigned char stage[kStages][kStageBytes];
  unsigned int coltab[kNT];         // column -> jj | nn << 8 | nd << 16 of the epilogue's current tile
  unsigned long long full[kStages], empty[kStages];
  unsigned long long acc_full[2], acc_empty[2], drain;
  unsigned long long tile_full[4], tile_empty[4];   // ring of the CTA's next tiles (fetched dynamically)
  int tile_ring[4];
  unsigned int tmem_base;
  int abort;
};
// two persistent CTAs per SM (228 KB of shared memory, 1 KB reserved per CTA; 2 x 256 TMEM columns)
static_assert(sizeof(Smem) + 1024 <= 113 * 1024, "shared memory of the tensor-core product exceeds half an SM");

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
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
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

// bulk copy global -> shared memory (no multicast), completion counted in bytes on `bar`
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// named barrier of the four epilogue warps that also ORs a flag over them
__device__ __forceinline__ bool epilogue_any(bool flag) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.b32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 2, 128, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)flag)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

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

// byte offset of (row r, K group g) within a slab half
__host__ __device__ __forceinline__ uint32_t slab_off(int r, int g) { return g * 2048 + (r >> 3) * 128 + (r & 7) * 16; }

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

// ---------------------------------------------------------------------------
// packing: one CTA of 256 threads per slab, one thread per (row, K group of 8)
//   rtabs: row r of the slab -> atom position | orbital << 8 | block size << 16 (0xffffffff: empty)
//   ktabs: K position of the slab's unit -> atom position | orbital << 8 | block size << 16
//   btab:  [slab][atom of the unit (4)][row atom (32)] -> block index or -1
// The value at (row r, K k) is the block (row atom, unit atom) at element (orbital_r, orbital_k),
// column-major: k_fastest = 1 puts the K orbital fastest (leading dimension = the K atom's block
// size), k_fastest = 0 the row orbital (leading dimension = the row atom's block size).
// ---------------------------------------------------------------------------
struct PackArgs {
  const int* __restrict__ slab_rtab;  // per slab: offset of its 128-entry row table
  const int* __restrict__ slab_unit;  // per slab: its unit
  const unsigned int* __restrict__ rtabs;
  const unsigned int* __restrict__ ktabs;   // [unit][16]
  const int* __restrict__ btab;
  const int64_t* __restrict__ elem;
  const double* __restrict__ src;
  uint4* __restrict__ out;            // [slab][512] (8 KB)
  int k_fastest;
};

__global__ void __launch_bounds__(256) k_umma_pack(PackArgs A) {
  const int s = blockIdx.x, t = threadIdx.x;
  const int r = t & 127, g = t >> 7;
  const unsigned int ri = A.rtabs[A.slab_rtab[s] + r];
  const unsigned int* kt = A.ktabs + (size_t)A.slab_unit[s] * kUK + g * 8;
  float v[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    double val = 0.0;
    const unsigned int ki = kt[e];
    if (ri != 0xffffffffu && ki != 0xffffffffu) {
      const int ra = ri & 0xff, ro = (ri >> 8) & 0xff, rnd = ri >> 16;
      const int ka = ki & 0xff, ko = (ki >> 8) & 0xff, knd = ki >> 16;
      const int blk = A.btab[(size_t)s * (kMaxUnitAtoms * kMaxAtoms) + ka * kMaxAtoms + ra];
      if (blk >= 0) val = __ldg(A.src + A.elem[blk] + (A.k_fastest ? ko + (int64_t)knd * ro : ro + (int64_t)rnd * ko));
    }
    v[e] = (float)val;
  }
  uint4 hi, lo;
  split8(v, hi, lo);
  unsigned char* base = reinterpret_cast<unsigned char*>(A.out + (size_t)s * (kSlabBytes / 16));
  *reinterpret_cast<uint4*>(base + slab_off(r, g)) = hi;
  *reinterpret_cast<uint4*>(base + kSlabHalf + slab_off(r, g)) = lo;
}

// ---------------------------------------------------------------------------
// the product kernel: one CTA per tile
// ---------------------------------------------------------------------------
struct UmmaArgs {
  const UmmaTile* __restrict__ tiles;
  const int2* __restrict__ units;     // per tile unit entry: (X slab, B slab)
  const unsigned int* __restrict__ rtabs;   // row tables of the row groups and of the column chunks
  const int* __restrict__ outmap;
  const uint4* __restrict__ xslabs;
  const uint4* __restrict__ bslabs;
  const int64_t* __restrict__ o_elem;
  double* __restrict__ out;
  int* err;                           // mapped host word: a bounded wait ran out
  int* tile_counter;                  // next tile to take (zeroed before the launch)
  int test_stall;                     // test hook: the copy thread stops after publishing its first tile
};

// Persistent: the bulk-copy thread of each CTA takes the next tile from a device-wide counter when it
// is ready for one (long and short tiles balance over the CTAs) and passes its number to the MMA
// thread and the epilogue warps through a four-entry ring in shared memory.  The bulk-copy thread and
// the MMA thread walk one continuous ring of stages across the CTA's tiles; tile number c of the CTA
// accumulates in TMEM buffer c % 2, which the epilogue warps read back (and release) while the MMAs
// of tile c + 1 run in the other buffer.
__global__ void __launch_bounds__(kThreads, 2) k_mult_umma(UmmaArgs P, int n_tiles) {
  extern __shared__ unsigned char smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // ---- set-up: barriers and TMEM
  if (tid == 128) {
    for (int s = 0; s < kStages; ++s) { mbar_init(&sm.full[s], 1); mbar_init(&sm.empty[s], 1); }
    for (int b = 0; b < 2; ++b) { mbar_init(&sm.acc_full[b], 1); mbar_init(&sm.acc_empty[b], 128); }
    // a ring entry is read by the MMA thread and by the four epilogue warps before it is reused
    for (int q = 0; q < 4; ++q) { mbar_init(&sm.tile_full[q], 1); mbar_init(&sm.tile_empty[q], 5); }
    mbar_init(&sm.drain, 1);
    sm.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm.tmem_base;

  if (warp == 4) {
    if (lane == 0) {
      // ---- bulk copies: the X and B slabs of each stage's units, tile after tile
      uint32_t it = 0;                 // stages issued by this CTA
      bool ok = true;
      for (uint32_t q = 0; ok; ++q) {
        // the next tile of the product: taken from a device-wide counter, published in the ring
        const int slot = q & 3;
        if (q >= 4 && !mbar_wait(&sm.tile_empty[slot], ((q >> 2) - 1) & 1, P.err, &sm.abort)) { ok = false; break; }
        const int t = atomicAdd(P.tile_counter, 1);
        sm.tile_ring[slot] = t < n_tiles ? t : -1;
        mbar_arrive(&sm.tile_full[slot]);
        if (t >= n_tiles) break;
        if (P.test_stall) break;       // no stage of the tile will arrive: the MMA thread's wait runs out
        const UmmaTile T = P.tiles[t];
        for (int u0 = 0; u0 < T.n_u; u0 += kUnitsPerStage, ++it) {
          const int s = it % kStages;
          if (it >= kStages && !mbar_wait(&sm.empty[s], ((it / kStages) - 1) & 1, P.err, &sm.abort)) { ok = false; break; }
          const int nu = min(kUnitsPerStage, T.n_u - u0);
          mbar_expect_tx(&sm.full[s], (uint32_t)(nu * 2 * kSlabBytes));
          unsigned char* st = sm.stage[s];
          for (int u = 0; u < nu; ++u) {
            const int2 e = P.units[T.u_off + u0 + u];
            const unsigned char* xs = reinterpret_cast<const unsigned char*>(P.xslabs) + (size_t)e.x * kSlabBytes;
            const unsigned char* bs = reinterpret_cast<const unsigned char*>(P.bslabs) + (size_t)e.y * kSlabBytes;
            bulk_g2s(st + 0 * kRegion + u * kSlabHalf, xs, kSlabHalf, &sm.full[s]);
            bulk_g2s(st + 1 * kRegion + u * kSlabHalf, xs + kSlabHalf, kSlabHalf, &sm.full[s]);
            bulk_g2s(st + 2 * kRegion + u * kSlabHalf, bs, kSlabHalf, &sm.full[s]);
            bulk_g2s(st + 3 * kRegion + u * kSlabHalf, bs + kSlabHalf, kSlabHalf, &sm.full[s]);
          }
        }
      }
      if (!ok) {
        // copies still in flight land in shared memory: wait for the stages issued last (bounded)
        int dummy = 0;
        for (uint32_t k = it > kStages ? it - kStages : 0; k < it; ++k)
          mbar_wait(&sm.full[k % kStages], (k / kStages) & 1, P.err, &dummy);
      }
    }
  } else if (warp == 5) {
    if (lane == 0) {
      // ---- MMA issue (one thread)
      constexpr uint32_t idesc = idesc_bf16(kM, kNT);
      uint32_t it = 0, tc = 0;         // stages consumed, tiles accumulated by this CTA
      bool ok = true;
      for (uint32_t q = 0; ok; ++q, ++tc) {
        const int slot = q & 3;
        if (!mbar_wait(&sm.tile_full[slot], (q >> 2) & 1, P.err, &sm.abort)) { ok = false; break; }
        const int t = *(volatile int*)&sm.tile_ring[slot];
        mbar_arrive(&sm.tile_empty[slot]);
        if (t < 0) break;
        const int n_u = P.tiles[t].n_u;
        const int b = tc & 1;
        if (tc >= 2 && !mbar_wait(&sm.acc_empty[b], ((tc >> 1) - 1) & 1, P.err, &sm.abort)) { ok = false; break; }
        tc_fence_after();
        const uint32_t acc = tmem + b * kNT;
        for (int u0 = 0; u0 < n_u; u0 += kUnitsPerStage, ++it) {
          const int s = it % kStages;
          if (!mbar_wait(&sm.full[s], (it / kStages) & 1, P.err, &sm.abort)) { ok = false; break; }
          tc_fence_after();
          const uint32_t base = smem_u32(sm.stage[s]);
          const int nu = min(kUnitsPerStage, n_u - u0);
          for (int u = 0; u < nu; ++u) {
            const uint32_t o = u * kSlabHalf;
            const uint64_t dah = smem_desc(base + 0 * kRegion + o, 2048, 128);
            const uint64_t dal = smem_desc(base + 1 * kRegion + o, 2048, 128);
            const uint64_t dbh = smem_desc(base + 2 * kRegion + o, 2048, 128);
            const uint64_t dbl = smem_desc(base + 3 * kRegion + o, 2048, 128);
            umma_bf16(acc, dal, dbh, idesc, (u0 > 0 || u > 0) ? 1u : 0u);
            umma_bf16(acc, dah, dbl, idesc, 1u);
            umma_bf16(acc, dah, dbh, idesc, 1u);
          }
          umma_commit(&sm.empty[s]);
        }
        if (ok) umma_commit(&sm.acc_full[b]);   // the tile's accumulator is complete (empty tiles too)
      }
      // every MMA issued above has completed before the tensor memory can be released
      umma_commit(&sm.drain);
      int dummy = 0;
      mbar_wait(&sm.drain, 0, P.err, &dummy, 2000000000ull);
    }
  } else {
    // ---- epilogue (warps 0-3, TMEM lane quarter = warp): accumulators -> FP64 output blocks
    const int m = warp * 32 + lane;
    uint32_t tc = 0;
    for (uint32_t q = 0;; ++q, ++tc) {
      const int slot = q & 3;
      const bool got = mbar_wait(&sm.tile_full[slot], (q >> 2) & 1, P.err, &sm.abort);
      const int t = got ? *(volatile int*)&sm.tile_ring[slot] : -1;
      __syncwarp();
      if (lane == 0 && got) mbar_arrive(&sm.tile_empty[slot]);
      if (epilogue_any(!got)) break;   // uniform over the epilogue warps (a wait ran out: aborted)
      if (t < 0) break;                // the same ring entry for every epilogue thread: uniform
      const UmmaTile T = P.tiles[t];
      const int b = tc & 1;
      const bool ok = mbar_wait(&sm.acc_full[b], (tc >> 1) & 1, P.err, &sm.abort, 2000000000ull);
      // the column table of this tile (the previous tile's users have passed the barrier at the end)
      sm.coltab[m] = P.rtabs[T.col_tab + m];
      if (epilogue_any(!ok)) break;    // a barrier of the four epilogue warps: the decision is uniform
      tc_fence_after();
      const unsigned int ri = P.rtabs[T.row_tab + m];
      const int ii = ri & 0xff, n1 = (ri >> 8) & 0xff, ndi = ri >> 16;
      // two halves of 64 columns; the buffer is released once the second half has been read
#pragma unroll 1
      for (int half = 0; half < 2; ++half) {
        uint32_t r[4][16];
#pragma unroll
        for (int cb = 0; cb < 4; ++cb) {
          if (T.n_u > 0) tmem_ld16(tmem + b * kNT + ((uint32_t)(warp * 32) << 16) + (half * 4 + cb) * 16, r[cb]);
          else {
#pragma unroll
            for (int e = 0; e < 16; ++e) r[cb][e] = 0u;
          }
        }
        if (half == 1) {
          tc_fence_before();
          mbar_arrive(&sm.acc_empty[b]);   // the MMAs of tile c + 2 may overwrite this buffer now
        }
        if (ri == 0xffffffffu) continue;
        int jj_prev = -1;
        long long base = -1;
#pragma unroll
        for (int e = 0; e < 64; ++e) {
          const unsigned int ci = sm.coltab[half * 64 + e];
          if (ci == 0xffffffffu) continue;
          const int jj = ci & 0xff, nn = (ci >> 8) & 0xff;
          if (jj != jj_prev) {
            const int q = __ldg(P.outmap + T.om_off + ii * T.n_cols + jj);
            base = q >= 0 ? (long long)P.o_elem[q] : -1ll;
            jj_prev = jj;
          }
          if (base >= 0) P.out[base + n1 + (int64_t)ndi * nn] = (double)__uint_as_float(r[e >> 4][e & 15]);
        }
      }
      asm volatile("bar.sync 2, 128;" ::: "memory");
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 5) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// ---------------------------------------------------------------------------
// tile plan (built once per product from its FP64 pair lists)
// ---------------------------------------------------------------------------
namespace {

struct PlanDev {                     // per output block / pair lookups of the plan kernels
  const int64_t* ptr;
  const int2* pairs;
  const int2* q_tile;                // output block -> (tile, ii | jj << 16)
  const int* xh;                     // X block -> candidate position of its unit in the row group
  const int* xcov;                   // X block -> contraction atom (cover)
  const int* ocov;                   // output block -> column atom (cover)
  const int* unit_of;                // cover atom -> unit
  const int* unit_pos;               // cover atom -> position in its unit
  const int* chunk_of;               // cover atom -> column chunk
  const int* chunk_pos;              // cover atom -> position in its chunk
  const int64_t* mark_off;           // tile -> first bit of its candidate bit set
  int n_chunks;
};

// one warp per output block: mark the units its pairs contract over (tile bit sets) and the
// (unit, column chunk) B slabs they need
__global__ void k_umma_mark(int n_out, PlanDev D, unsigned int* __restrict__ mark, unsigned int* __restrict__ bmark) {
  const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (q >= n_out) return;
  const int t = D.q_tile[q].x;
  const int64_t mo = D.mark_off[t];
  const int ch = D.chunk_of[D.ocov[q]];
  for (int64_t p = D.ptr[q] + lane; p < D.ptr[q + 1]; p += 32) {
    const int x = D.pairs[p].x;
    const int64_t bit = mo + D.xh[x];
    atomicOr(mark + (bit >> 5), 1u << (bit & 31));
    const int64_t bk = (int64_t)D.unit_of[D.xcov[x]] * D.n_chunks + ch;
    atomicOr(bmark + (bk >> 5), 1u << (bk & 31));
  }
}

// per-word population counts of a bit set (scanned on the host afterwards)
__global__ void k_word_count(int64_t n_words, const unsigned int* __restrict__ bits, int* __restrict__ cnt) {
  const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (w < n_words) cnt[w] = __popc(bits[w]);
}

__device__ __forceinline__ int rank_of(const unsigned int* bits, const int* pre, int64_t bit) {
  const int64_t w = bit >> 5;
  return pre[w] + __popc(bits[w] & ((1u << (bit & 31)) - 1u));
}

// one thread per tile: without `units` its unit count, with it the unit entries (X slab, B slab)
__global__ void k_umma_units(int n_tiles, UmmaTile* __restrict__ tiles, const int64_t* __restrict__ mark_off,
                             const int* __restrict__ mark_bits, const unsigned int* __restrict__ mark,
                             const int* __restrict__ u_cand, const int64_t* __restrict__ u_off,
                             const int* __restrict__ tile_group, const int* __restrict__ tile_chunk, int n_chunks,
                             const unsigned int* __restrict__ bmark, const int* __restrict__ bpre,
                             int2* __restrict__ units) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_tiles) return;
  UmmaTile& T = tiles[t];
  const int64_t w0 = mark_off[t] >> 5;
  const int nw = (mark_bits[t] + 31) >> 5;
  const int g = tile_group[t];
  const int* U = u_cand + u_off[g];
  int cnt = 0;
  for (int w = 0; w < nw; ++w) {
    unsigned int m = mark[w0 + w];
    while (m) {
      const int b = __ffs(m) - 1;
      m &= m - 1;
      if (units) {
        const int h = 32 * w + b;
        const int64_t bk = (int64_t)U[h] * n_chunks + tile_chunk[t];
        units[T.u_off + cnt] = make_int2((int)(u_off[g] + h), rank_of(bmark, bpre, bk));
      }
      ++cnt;
    }
  }
  if (!units) T.n_u = cnt;
}

// one warp per output block: block tables of the X and B slabs from the pairs
__global__ void k_umma_btab(int n_out, PlanDev D, const unsigned int* __restrict__ bmark, const int* __restrict__ bpre,
                            const int64_t* __restrict__ xs_of_tile, int* __restrict__ xtab, int* __restrict__ btab) {
  const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (q >= n_out) return;
  const int2 tq = D.q_tile[q];
  const int ii = tq.y & 0xffff;
  const int oc = D.ocov[q];
  const int ch = D.chunk_of[oc], jpos = D.chunk_pos[oc];
  const int64_t uo = xs_of_tile[tq.x];
  for (int64_t p = D.ptr[q] + lane; p < D.ptr[q + 1]; p += 32) {
    const int2 pr = D.pairs[p];
    const int c = D.xcov[pr.x];
    const int cpos = D.unit_pos[c];
    const int64_t xs = uo + D.xh[pr.x];
    xtab[xs * (kMaxUnitAtoms * kMaxAtoms) + cpos * kMaxAtoms + ii] = pr.x;
    const int bs = rank_of(bmark, bpre, (int64_t)D.unit_of[c] * D.n_chunks + ch);
    btab[(int64_t)bs * (kMaxUnitAtoms * kMaxAtoms) + cpos * kMaxAtoms + jpos] = pr.y;
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
  const int np = g.n_prim, ncov = g.n_cover_atoms;
  std::vector<int> nd_prim(np);
  for (int p = 0; p < np; ++p) nd_prim[p] = g.nsf[g.prim_global[p]];
  U.usable = true;
  for (int p = 0; p < np; ++p) U.usable = U.usable && nd_prim[p] >= kMinNd && nd_prim[p] <= kUK;
  for (int c = 0; c < ncov; ++c) U.usable = U.usable && g.cover_nsf[c] >= kMinNd && g.cover_nsf[c] <= kUK;
  if (!U.usable || O.nnz == 0) {
    auto res = S.uplans.emplace(key, std::move(up));
    return *res.first->second;
  }
  // contraction units and column chunks over the cover atoms (cover order, the same for every row group)
  std::vector<int> unit_of(ncov), unit_pos(ncov), chunk_of(ncov), chunk_pos(ncov), chunk_first;
  std::vector<unsigned int> ktab;                   // [unit][16]
  {
    int u = -1, uw = kUK + 1, ua = kMaxUnitAtoms;
    for (int c = 0; c < ncov; ++c) {
      const int nd = g.cover_nsf[c];
      if (uw + nd > kUK || ua == kMaxUnitAtoms) { ++u; uw = 0; ua = 0; ktab.resize((size_t)(u + 1) * kUK, 0xffffffffu); }
      for (int o = 0; o < nd; ++o) ktab[(size_t)u * kUK + uw + o] = (unsigned)ua | ((unsigned)o << 8) | ((unsigned)nd << 16);
      unit_of[c] = u; unit_pos[c] = ua;
      uw += nd; ++ua;
    }
    int w = kNT + 1, cnt = kMaxAtoms;
    for (int c = 0; c < ncov; ++c) {
      const int nd = g.cover_nsf[c];
      if (w + nd > kNT || cnt == kMaxAtoms) { chunk_first.push_back(c); w = 0; cnt = 0; }
      chunk_of[c] = (int)chunk_first.size() - 1;
      chunk_pos[c] = cnt;
      w += nd; ++cnt;
    }
    chunk_first.push_back(ncov);
  }
  const int n_units = (int)(ktab.size() / kUK), n_chunks = (int)chunk_first.size() - 1;
  // host copies of the output and first-operand neighbour lists
  std::vector<int> ocov(O.nnz), xcov(std::max(X.nnz, 1));
  CQ_CUDA(cudaMemcpyAsync(ocov.data(), O.nb_cover.p, sizeof(int) * O.nnz, cudaMemcpyDeviceToHost, st));
  if (X.nnz) CQ_CUDA(cudaMemcpyAsync(xcov.data(), X.nb_cover.p, sizeof(int) * X.nnz, cudaMemcpyDeviceToHost, st));
  CQ_CUDA(cudaStreamSynchronize(st));
  // row groups: consecutive primary atoms, at most kM rows and kMaxAtoms atoms
  std::vector<int> grp_first;
  for (int p = 0, rows = kM + 1, cnt = 0; p < np; ++p) {
    if (rows + nd_prim[p] > kM || cnt == kMaxAtoms) { grp_first.push_back(p); rows = 0; cnt = 0; }
    rows += nd_prim[p]; ++cnt;
  }
  grp_first.push_back(np);
  const int ng = (int)grp_first.size() - 1;
  // row tables of the row groups (offset 128 g) and of the column chunks (offset 128 (ng + chunk))
  std::vector<unsigned int> rtabs((size_t)(ng + n_chunks) * kM, 0xffffffffu);
  for (int gi = 0; gi < ng; ++gi)
    for (int p = grp_first[gi], off = 0; p < grp_first[gi + 1]; off += nd_prim[p], ++p)
      for (int o = 0; o < nd_prim[p]; ++o)
        rtabs[(size_t)gi * kM + off + o] = (unsigned)(p - grp_first[gi]) | ((unsigned)o << 8) | ((unsigned)nd_prim[p] << 16);
  for (int ch = 0; ch < n_chunks; ++ch)
    for (int c = chunk_first[ch], off = 0; c < chunk_first[ch + 1]; off += g.cover_nsf[c], ++c)
      for (int o = 0; o < g.cover_nsf[c]; ++o)
        rtabs[(size_t)(ng + ch) * kM + off + o] = (unsigned)(c - chunk_first[ch]) | ((unsigned)o << 8) |
                                                  ((unsigned)g.cover_nsf[c] << 16);
  // tiles: (row group, column chunk) pairs holding output blocks; candidate units of each row group
  std::vector<UmmaTile> tiles;
  std::vector<int> outmap, tile_group, tile_chunk, mark_bits, u_cand, xh(std::max(X.nnz, 1), 0);
  std::vector<int2> q_tile(O.nnz);
  std::vector<int64_t> u_off(ng + 1, 0), mark_off;
  int64_t mark_total = 0;
  for (int gi = 0; gi < ng; ++gi) {
    const int r0 = grp_first[gi], r1 = grp_first[gi + 1];
    std::vector<int> chs;
    for (int q = O.h_row_ptr[r0]; q < O.h_row_ptr[r1]; ++q) chs.push_back(chunk_of[ocov[q]]);
    std::sort(chs.begin(), chs.end());
    chs.erase(std::unique(chs.begin(), chs.end()), chs.end());
    std::vector<int> cand;
    for (int e = X.h_row_ptr[r0]; e < X.h_row_ptr[r1]; ++e) cand.push_back(unit_of[xcov[e]]);
    std::sort(cand.begin(), cand.end());
    cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
    for (int e = X.h_row_ptr[r0]; e < X.h_row_ptr[r1]; ++e)
      xh[e] = (int)(std::lower_bound(cand.begin(), cand.end(), unit_of[xcov[e]]) - cand.begin());
    u_off[gi] = (int64_t)u_cand.size();
    u_cand.insert(u_cand.end(), cand.begin(), cand.end());
    const int t0 = (int)tiles.size();
    for (int ch : chs) {
      UmmaTile T{};
      T.row_first = r0;
      T.n_rows = r1 - r0;
      T.n_cols = chunk_first[ch + 1] - chunk_first[ch];
      T.row_tab = gi * kM;
      T.col_tab = (ng + ch) * kM;
      T.om_off = (int)outmap.size();
      outmap.resize(outmap.size() + (size_t)T.n_rows * T.n_cols, -1);
      tiles.push_back(T);
      tile_group.push_back(gi);
      tile_chunk.push_back(ch);
      mark_off.push_back(mark_total);
      mark_bits.push_back((int)cand.size());
      mark_total += ((int64_t)cand.size() + 31) / 32 * 32;
    }
    for (int p = r0; p < r1; ++p)
      for (int q = O.h_row_ptr[p]; q < O.h_row_ptr[p + 1]; ++q) {
        const int ch = chunk_of[ocov[q]];
        const int t = t0 + (int)(std::lower_bound(chs.begin(), chs.end(), ch) - chs.begin());
        const int ii = p - r0, jj = chunk_pos[ocov[q]];
        q_tile[q] = make_int2(t, ii | (jj << 16));
        outmap[tiles[t].om_off + ii * tiles[t].n_cols + jj] = q;
      }
  }
  u_off[ng] = (int64_t)u_cand.size();
  const int nt = (int)tiles.size();
  U.n_tiles = nt;
  U.n_xslabs = u_off[ng];
  std::vector<int64_t> xs_tile(nt);
  for (int t = 0; t < nt; ++t) xs_tile[t] = u_off[tile_group[t]];
  // device copies of the plan inputs
  DevBuf<int2> d_qt; d_qt.upload(q_tile, st);
  DevBuf<int> d_xh; d_xh.upload(xh, st);
  DevBuf<int> d_xcov; d_xcov.upload(xcov, st);
  DevBuf<int> d_uof; d_uof.upload(unit_of, st);
  DevBuf<int> d_upos; d_upos.upload(unit_pos, st);
  DevBuf<int> d_chof; d_chof.upload(chunk_of, st);
  DevBuf<int> d_chpos; d_chpos.upload(chunk_pos, st);
  DevBuf<int64_t> d_moff; d_moff.upload(mark_off, st);
  DevBuf<int> d_mbits; d_mbits.upload(mark_bits, st);
  DevBuf<int> d_tg; d_tg.upload(tile_group, st);
  DevBuf<int> d_tc; d_tc.upload(tile_chunk, st);
  DevBuf<int> d_uc; d_uc.upload(u_cand.empty() ? std::vector<int>{0} : u_cand, st);
  DevBuf<int64_t> d_uoff; d_uoff.upload(u_off, st);
  const int64_t mark_words = std::max<int64_t>(mark_total / 32, 1);
  const int64_t bkeys = (int64_t)n_units * n_chunks;
  const int64_t bwords = std::max<int64_t>((bkeys + 31) / 32, 1);
  DevBuf<unsigned int> d_mark; d_mark.alloc(mark_words, st);
  DevBuf<unsigned int> d_bmark; d_bmark.alloc(bwords, st);
  CQ_CUDA(cudaMemsetAsync(d_mark.p, 0, sizeof(unsigned int) * mark_words, st));
  CQ_CUDA(cudaMemsetAsync(d_bmark.p, 0, sizeof(unsigned int) * bwords, st));
  U.tiles.upload(tiles, st);
  U.outmap.upload(outmap.empty() ? std::vector<int>{-1} : outmap, st);
  U.rtabs.upload(rtabs, st);
  U.ktabs.upload(ktab, st);
  PlanDev D;
  D.ptr = P.ptr.p; D.pairs = P.pairs.p; D.q_tile = d_qt.p; D.xh = d_xh.p; D.xcov = d_xcov.p; D.ocov = O.nb_cover.p;
  D.unit_of = d_uof.p; D.unit_pos = d_upos.p; D.chunk_of = d_chof.p; D.chunk_pos = d_chpos.p; D.mark_off = d_moff.p;
  D.n_chunks = n_chunks;
  const int n_out = O.nnz;
  const int T256 = 256;
  const int gw = (int)(((int64_t)n_out * 32 + T256 - 1) / T256);
  k_umma_mark<<<gw, T256, 0, st>>>(n_out, D, d_mark.p, d_bmark.p);
  k_umma_units<<<(nt + 127) / 128, 128, 0, st>>>(nt, U.tiles.p, d_moff.p, d_mbits.p, d_mark.p, d_uc.p, d_uoff.p, d_tg.p,
                                                 d_tc.p, n_chunks, d_bmark.p, nullptr, nullptr);
  // ranks of the B slab keys: per-word counts, scanned on the host
  DevBuf<int> d_bpre; d_bpre.alloc(bwords, st);
  k_word_count<<<(int)((bwords + 255) / 256), 256, 0, st>>>(bwords, d_bmark.p, d_bpre.p);
  CQ_CUDA(cudaGetLastError());
  std::vector<int> bpre(bwords);
  std::vector<unsigned int> bm(bwords);
  CQ_CUDA(cudaMemcpyAsync(bpre.data(), d_bpre.p, sizeof(int) * bwords, cudaMemcpyDeviceToHost, st));
  CQ_CUDA(cudaMemcpyAsync(bm.data(), d_bmark.p, sizeof(unsigned int) * bwords, cudaMemcpyDeviceToHost, st));
  CQ_CUDA(cudaMemcpyAsync(tiles.data(), U.tiles.p, sizeof(UmmaTile) * nt, cudaMemcpyDeviceToHost, st));
  CQ_CUDA(cudaStreamSynchronize(st));
  int64_t n_bslabs = 0;
  for (auto& x : bpre) { const int c = x; x = (int)n_bslabs; n_bslabs += c; }
  d_bpre.upload(bpre, st);
  U.n_bslabs = n_bslabs;
  int64_t uoff = 0;
  U.issued_flops = 0;
  for (auto& T : tiles) {
    T.u_off = (int)uoff;
    uoff += T.n_u;
    U.issued_flops += 3ll * 2 * kM * kNT * kUK * T.n_u;
  }
  CQ_CHECK(uoff < ((int64_t)1 << 31) && n_bslabs < ((int64_t)1 << 31) && U.n_xslabs < ((int64_t)1 << 31), CQ_ERR_BOUNDS,
           "tensor-core tile plan too large");
  U.tiles.upload(tiles, st);
  U.units.alloc(std::max<int64_t>(uoff, 1), st);
  k_umma_units<<<(nt + 127) / 128, 128, 0, st>>>(nt, U.tiles.p, d_moff.p, d_mbits.p, d_mark.p, d_uc.p, d_uoff.p, d_tg.p,
                                                 d_tc.p, n_chunks, d_bmark.p, d_bpre.p, U.units.p);
  CQ_CUDA(cudaStreamSynchronize(st));
  // what the slab tables need later (host copies; the device temporaries above are released now)
  U.mult_type = mult_type; U.ra = ra; U.rb = rb; U.rc = rc;
  U.n_groups = ng; U.n_chunks = n_chunks;
  U.h_q_tile = std::move(q_tile); U.h_xh = std::move(xh); U.h_xcov = std::move(xcov);
  U.h_unit_of = std::move(unit_of); U.h_unit_pos = std::move(unit_pos);
  U.h_chunk_of = std::move(chunk_of); U.h_chunk_pos = std::move(chunk_pos);
  U.h_u_cand = std::move(u_cand); U.h_u_off = std::move(u_off); U.h_xs_tile = std::move(xs_tile);
  U.h_bmark = std::move(bm); U.h_bpre = std::move(bpre);
  S.launches += 4;
  auto res = S.uplans.emplace(key, std::move(up));
  return *res.first->second;
}

// Slab tables and buffers of a tile plan, built on the product's first tensor-core call: the block of
// every slab position (from the pair lists), the row tables and units of the packing kernels, and the
// slab buffers themselves.
static void umma_materialise(System& S, UmmaPlan& U) {
  if (U.materialised) return;
  cudaStream_t st = S.stream;
  ProductPlan& P = get_plan(S, U.mult_type, U.ra, U.rb, U.rc);
  RangeIndex& O = U.mult_type == 1 ? *S.ranges[U.rc] : *S.ranges[U.ra];
  DevBuf<int2> d_qt; d_qt.upload(U.h_q_tile, st);
  DevBuf<int> d_xh; d_xh.upload(U.h_xh, st);
  DevBuf<int> d_xcov; d_xcov.upload(U.h_xcov, st);
  DevBuf<int> d_uof; d_uof.upload(U.h_unit_of, st);
  DevBuf<int> d_upos; d_upos.upload(U.h_unit_pos, st);
  DevBuf<int> d_chof; d_chof.upload(U.h_chunk_of, st);
  DevBuf<int> d_chpos; d_chpos.upload(U.h_chunk_pos, st);
  DevBuf<unsigned int> d_bmark; d_bmark.upload(U.h_bmark, st);
  DevBuf<int> d_bpre; d_bpre.upload(U.h_bpre, st);
  DevBuf<int64_t> d_xst; d_xst.upload(U.h_xs_tile, st);
  PlanDev D;
  D.ptr = P.ptr.p; D.pairs = P.pairs.p; D.q_tile = d_qt.p; D.xh = d_xh.p; D.xcov = d_xcov.p; D.ocov = O.nb_cover.p;
  D.unit_of = d_uof.p; D.unit_pos = d_upos.p; D.chunk_of = d_chof.p; D.chunk_pos = d_chpos.p; D.mark_off = nullptr;
  D.n_chunks = U.n_chunks;
  const int64_t tabw = kMaxUnitAtoms * kMaxAtoms;
  U.xtab.alloc(std::max<int64_t>(U.n_xslabs, 1) * tabw, st);
  U.btab.alloc(std::max<int64_t>(U.n_bslabs, 1) * tabw, st);
  CQ_CUDA(cudaMemsetAsync(U.xtab.p, 0xff, sizeof(int) * U.xtab.n, st));
  CQ_CUDA(cudaMemsetAsync(U.btab.p, 0xff, sizeof(int) * U.btab.n, st));
  const int n_out = O.nnz;
  const int gw = (int)(((int64_t)n_out * 32 + 255) / 256);
  k_umma_btab<<<gw, 256, 0, st>>>(n_out, D, d_bmark.p, d_bpre.p, d_xst.p, U.xtab.p, U.btab.p);
  CQ_CUDA(cudaGetLastError());
  std::vector<int> xs_rtab(std::max<int64_t>(U.n_xslabs, 1), 0), xs_unit(std::max<int64_t>(U.n_xslabs, 1), 0);
  for (int gi = 0; gi < U.n_groups; ++gi)
    for (int64_t h = U.h_u_off[gi]; h < U.h_u_off[gi + 1]; ++h) { xs_rtab[h] = gi * kM; xs_unit[h] = U.h_u_cand[h]; }
  U.xs_rtab.upload(xs_rtab, st);
  U.xs_unit.upload(xs_unit, st);
  // B slabs in key order (key = unit * n_chunks + chunk), as ranked by the plan
  std::vector<int> bs_rtab, bs_unit;
  bs_rtab.reserve(std::max<int64_t>(U.n_bslabs, 1)); bs_unit.reserve(std::max<int64_t>(U.n_bslabs, 1));
  for (size_t w = 0; w < U.h_bmark.size(); ++w)
    for (unsigned int m = U.h_bmark[w]; m; m &= m - 1) {
      const int64_t k = 32 * (int64_t)w + __builtin_ctz(m);
      bs_unit.push_back((int)(k / U.n_chunks));
      bs_rtab.push_back((int)((U.n_groups + k % U.n_chunks) * kM));
    }
  if (bs_rtab.empty()) { bs_rtab.push_back(0); bs_unit.push_back(0); }
  U.bs_rtab.upload(bs_rtab, st);
  U.bs_unit.upload(bs_unit, st);
  U.xslabs.alloc((size_t)std::max<int64_t>(U.n_xslabs, 1) * (kSlabBytes / 16), st);
  U.bslabs.alloc((size_t)std::max<int64_t>(U.n_bslabs, 1) * (kSlabBytes / 16), st);
  CQ_CUDA(cudaStreamSynchronize(st));
  S.launches += 1;
  U.materialised = true;
}

int* device_timeout_word(System& S) {
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
  CQ_CHECK(U.usable, CQ_ERR_ARG, "tensor-core tiles need block sizes of 4 to 16");
  if (U.n_tiles == 0) return;
  umma_materialise(S, U);
  RangeIndex &A = *S.ranges[ra], &B = *S.ranges[rb], &C = *S.ranges[rc];
  RangeIndex& O = mult_type == 1 ? C : A;
  RangeIndex& X = mult_type == 1 ? A : C;
  cudaStream_t st = S.stream;
  cudaEvent_t ev0 = nullptr;
  if (S.prof.on) { ev0 = S.prof.get(); CQ_CUDA(cudaEventRecord(ev0, st)); }
  // pack the operands: X slabs (first operand, row orbital fastest), B slabs (type 1: B(k, j) with the
  // K orbital fastest; type 2: B(k, j) with the column orbital fastest)
  PackArgs pk;
  pk.ktabs = U.ktabs.p;
  pk.rtabs = U.rtabs.p;
  if (U.n_xslabs > 0) {
    pk.slab_rtab = U.xs_rtab.p; pk.slab_unit = U.xs_unit.p; pk.btab = U.xtab.p;
    pk.elem = X.nb_elem.p; pk.src = mult_type == 1 ? a : c; pk.out = U.xslabs.p; pk.k_fastest = 0;
    k_umma_pack<<<(int)U.n_xslabs, 256, 0, st>>>(pk);
  }
  if (U.n_bslabs > 0) {
    pk.slab_rtab = U.bs_rtab.p; pk.slab_unit = U.bs_unit.p; pk.btab = U.btab.p;
    pk.elem = B.nb_elem.p; pk.src = b; pk.out = U.bslabs.p; pk.k_fastest = mult_type == 1 ? 1 : 0;
    k_umma_pack<<<(int)U.n_bslabs, 256, 0, st>>>(pk);
  }
  UmmaArgs M;
  M.tiles = U.tiles.p; M.units = U.units.p; M.rtabs = U.rtabs.p; M.outmap = U.outmap.p;
  M.xslabs = U.xslabs.p; M.bslabs = U.bslabs.p;
  M.o_elem = O.nb_elem.p;
  M.out = mult_type == 1 ? c : a;
  M.err = device_timeout_word(S);
  if (!U.tile_counter.n) U.tile_counter.alloc(1, st);
  CQ_CUDA(cudaMemsetAsync(U.tile_counter.p, 0, sizeof(int), st));
  M.tile_counter = U.tile_counter.p;
  M.test_stall = S.umma_test_stall;
  S.umma_test_stall = 0;              // one product only
  const size_t smem = sizeof(Smem) + 1024;
  CQ_CUDA(cudaFuncSetAttribute(k_mult_umma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev_id = 0, sms = 0;
  CQ_CUDA(cudaGetDevice(&dev_id));
  CQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_id));
  k_mult_umma<<<std::min(U.n_tiles, 2 * sms), kThreads, smem, st>>>(M, U.n_tiles);
  CQ_CUDA(cudaGetLastError());
  S.launches += 3;
  if (S.prof.on) {
    cudaEvent_t ev1 = S.prof.get();
    CQ_CUDA(cudaEventRecord(ev1, st));
    S.prof.recs.push_back({ev0, ev1, 8.0 * (double)(A.length + B.length + C.length), (double)U.flops});
  }
}

void umma_check(System& S) {
  if (S.umma_err_host && *(volatile int*)S.umma_err_host) {
    *S.umma_err_host = 0;
    throw Error(CQ_ERR_TIMEOUT, "block product: a bounded wait of the kernel ran out (bulk copy or pipeline stage never completed)");
  }
}

size_t umma_smem_bytes() { return sizeof(Smem) + 1024; }

}  // namespace cqb
