// Device-side synthetic S and H (the generators of cq_b200/inputs.py, evaluated on the GPU so a
// request never round-trips its matrices through the host):
//   S: onsite block 1.0 * I, offsite 0.3 exp(-r/2) w on every entry
//   H: onsite block diagonal with -0.5 u (u uniform [0,1) from the counter hash of
//      (seed, tag 21, atom, atom, 0, 0, 0, orbital)), offsite -0.2 exp(-r/2) w on every entry
// with the block weight w = min(1, 4 / sqrt(nd_i nd_j)) (1 for SZ blocks; it keeps the overlap of
// larger blocks diagonally dominant).
// The hash is integer arithmetic identical to inputs.hash_uniform; exp() may differ from the
// host's libm in the last bit.
#include "cq_internal.hpp"

namespace cqb {
namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

__device__ double hash_uniform(uint64_t seed, uint64_t tag, int64_t a, int64_t b, int64_t sx, int64_t sy, int64_t sz,
                               int64_t e) {
  uint64_t k = mix64(seed * 0x9E3779B97F4A7C15ull + tag);
  k = mix64(k ^ ((uint64_t)a * 0xD1B54A32D192ED03ull));
  k = mix64(k ^ ((uint64_t)b * 0xABC98388FB8FAC03ull));
  k = mix64(k ^ ((uint64_t)sx * 0x8CB92BA72F3D8DD7ull));
  k = mix64(k ^ ((uint64_t)sy * 0xC2B2AE3D27D4EB4Full));
  k = mix64(k ^ ((uint64_t)sz * 0x165667B19E3779F9ull));
  k = mix64(k ^ ((uint64_t)e * 0x27D4EB2F165667C5ull));
  return (double)(k >> 11) * (1.0 / 9007199254740992.0);
}

// one warp per stored block
__global__ void k_gen_SH(int nnz, int which, uint64_t seed, const int* __restrict__ nb_row,
                         const int* __restrict__ nb_cover, const int64_t* __restrict__ nb_elem,
                         const double* __restrict__ nb_radius, const int* __restrict__ prim_global,
                         const int* __restrict__ cover_global, const int* __restrict__ cover_part,
                         const int* __restrict__ cover_shift, const int* __restrict__ prim_nsf,
                         const int* __restrict__ cover_nsf, double* __restrict__ out) {
  int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (e >= nnz) return;
  const int p = nb_row[e], c = nb_cover[e];
  const int ndi = prim_nsf[p], ndj = cover_nsf[c];
  const int gi = prim_global[p], gj = cover_global[c];
  const int* sh = cover_shift + 3 * cover_part[c];
  const bool onsite = gi == gj && sh[0] == 0 && sh[1] == 0 && sh[2] == 0;
  const double w = fmin(1.0, 4.0 / sqrt((double)ndi * (double)ndj));
  const double off = (which == 0 ? 0.3 : -0.2) * w * exp(-nb_radius[e] / 2.0);
  double* O = out + nb_elem[e];
  for (int t = lane; t < ndi * ndj; t += 32) {
    const int r = t % ndi, col = t / ndi;
    double v;
    if (!onsite) v = off;
    else if (which == 0) v = (r == col) ? 1.0 : 0.0;
    else v = (r == col) ? -0.5 * hash_uniform(seed, 21, gi, gi, 0, 0, 0, r) : 0.0;
    O[t] = v;
  }
}

}  // namespace

void generate_SH(System& S, int r, int which, uint64_t seed, double* out) {
  RangeIndex& R = *S.ranges[r];
  if (S.dg.prim_global.n == 0) {
    S.dg.prim_global.upload(S.geo.prim_global, S.stream);
    S.dg.cover_global.upload(S.geo.cover_global, S.stream);
    S.dg.cover_shift.upload(S.geo.cover_shift, S.stream);
  }
  if (R.nnz == 0) return;
  k_gen_SH<<<(int)(((int64_t)R.nnz * 32 + 255) / 256), 256, 0, S.stream>>>(
      R.nnz, which, seed, R.nb_row.p, R.nb_cover.p, R.nb_elem.p, R.nb_radius.p, S.dg.prim_global.p, S.dg.cover_global.p,
      S.dg.cover_part.p, S.dg.cover_shift.p, S.dg.prim_nsf.p, S.dg.cover_nsf.p, out);
  S.launches++;
  CQ_CUDA(cudaGetLastError());
}

}  // namespace cqb
