// Host geometry for one process: Hilbert-ordered partitions, the primary set
// and the covering set with periodic images.  This is O(N) bookkeeping that
// feeds the GPU index builders; the neighbour lists themselves are built on
// the device (index.cu).
//
// Algorithm sources (the partition and cover-set order fixes the storage
// layout and the summation order, so it follows the reference step by step):
//   src/Hilbert3D.f90                      curve index <-> partition coordinates
//   src/sfc_partitions_module.f90:475-724  partition grid choice and refinement
//   src/sfc_partitions_module.f90:843-1150 get_cell_info / get_extent / check_gap
//   src/sfc_partitions_module.f90:389-447  construct_cq_partitions
//   src/primary_module.f90:97-301          make_prim, calliper
//   src/cover_module.f90:133-429, 430-700  make_cs, make_iprim, convert_primary
#include <algorithm>
#include <array>
#include <cmath>
#include <numeric>

#include "cq_internal.hpp"

namespace cqb {
namespace {

constexpr double kShift = 1.0e-6;     // shift_in_bohr (global_module.f90:376)
constexpr double kVerySmall = 1.0e-8; // very_small (numbers_module.f90:93)

int rnd(double x) { return (int)std::lround(x); }
int modf_(int a, int n) { return a % n; }

// ---------------------------------------------------------------------------
// Hilbert curve on a 2^a x 2^b x 2^c grid, decomposed into a line of squares
// of cubes (Hilbert3D.f90).  Indices 0-based internally.
// ---------------------------------------------------------------------------
class HilbertCurve {
 public:
  explicit HilbertCurve(std::array<int, 3> divs) {
    std::array<int, 3> alpha = divs, axis = {0, 1, 2};
    // stable descending bubble sort of the exponents, carrying the axis map
    for (int n = 3; n > 1;) {
      int last = 1;
      for (int i = 1; i < n; ++i)
        if (alpha[i - 1] < alpha[i]) { std::swap(alpha[i], alpha[i - 1]); std::swap(axis[i], axis[i - 1]); last = i + 1; }
      n = last;
    }
    axis_ = axis;
    line_ = 1 << (alpha[0] - alpha[1]);
    square_ = 1 << (alpha[1] - alpha[2]);
    cube_ = 1 << alpha[2];
  }
  int index_of(const int c[3]) const {  // 0-based coords -> 0-based curve index
    int l = (c[axis_[0]] / cube_) / square_;
    int p[2] = {(c[axis_[0]] / cube_) % square_, (c[axis_[1]] / cube_) % square_};
    int q[3] = {c[axis_[0]] % cube_, c[axis_[1]] % cube_, c[axis_[2]] % cube_};
    std::vector<int> dl = bits_by_level(&l, 1, levels(line_ - 1, 2));
    std::vector<int> dp = bits_by_level(p, 2, levels(square_ - 1, 2));
    std::vector<int> dc = bits_by_level(q, 3, levels(cube_ - 1, 2));
    int start = 0, end = 1;
    std::vector<int> il(dl.size(), 0), ip(dp.size(), 0), ic(dc.size(), 0);
    if (line_ > 1) walk_decode(dl, il, 1, start, end);
    start *= 2; end *= 2;
    if (square_ > 1) walk_decode(dp, ip, 2, start, end);
    start *= 2; end *= 2;
    if (cube_ > 1) walk_decode(dc, ic, 3, start, end);
    int lv = pack(il, 2), pv = pack(ip, 4), cv = pack(ic, 8);
    return (lv * square_ * square_ + pv) * cube_ * cube_ * cube_ + cv;
  }
  void coords_of(int index, int c[3]) const {  // 0-based curve index -> 0-based coords
    int pts = cube_ * cube_ * cube_, sq = square_ * square_;
    int ic = index / pts, cc = index % pts, lv = ic / sq, pv = ic % sq;
    std::vector<int> il = digits(lv, 2, levels(line_ - 1, 2));
    std::vector<int> ip = digits(pv, 4, levels(sq - 1, 4));
    std::vector<int> icc = digits(cc, 8, levels(pts - 1, 8));
    std::vector<int> ol(il.size(), 0), op(ip.size(), 0), oc(icc.size(), 0);
    int start = 0, end = 1;
    if (line_ > 1) walk_encode(il, ol, 1, start, end);
    start *= 2; end *= 2;
    if (square_ > 1) walk_encode(ip, op, 2, start, end);
    start *= 2; end *= 2;
    if (cube_ > 1) walk_encode(icc, oc, 3, start, end);
    std::vector<int> l1 = levels_to_bits(ol, 1), p2 = levels_to_bits(op, 2), c3 = levels_to_bits(oc, 3);
    int a0 = (l1[0] * square_ + p2[0]) * cube_ + c3[0];
    int a1 = p2[1] * cube_ + c3[1];
    int a2 = c3[2];
    c[axis_[0]] = a0; c[axis_[1]] = a1; c[axis_[2]] = a2;
  }

 private:
  std::array<int, 3> axis_;
  int line_, square_, cube_;
  static int levels(int n, int base) { int m = 1; while (n >= base) { n /= base; ++m; } return m; }
  static int gray(int i) { return i ^ (int)((unsigned)i >> 1); }
  static int ungray(int g) { int b = g; for (int s = 1; ((unsigned)g >> s) > 0; ++s) b ^= (int)((unsigned)g >> s); return b; }
  static int enc_travel(int start, int end, int nb, int i) {
    int g = gray(i) * ((start ^ end) << 1);
    return ((g | (int)((unsigned)g >> nb)) & ((1 << nb) - 1)) ^ start;
  }
  static int dec_travel(int start, int end, int nb, int g) {
    int r = ((g ^ start) << nb) / ((start ^ end) << 1);
    return ungray((r | (int)((unsigned)r >> nb)) & ((1 << nb) - 1));
  }
  static void child(int& start, int& end, int nb, int i) {
    int lo = std::max(0, (i - 1) & ~1), hi = std::min((1 << nb) - 1, (i + 1) | 1);
    int s2 = enc_travel(start, end, nb, lo), e2 = enc_travel(start, end, nb, hi);
    start = s2; end = e2;
  }
  static void walk_decode(const std::vector<int>& in, std::vector<int>& out, int nb, int& start, int& end) {
    for (size_t k = 0; k < in.size(); ++k) { out[k] = dec_travel(start, end, nb, in[k]); child(start, end, nb, out[k]); }
  }
  static void walk_encode(const std::vector<int>& in, std::vector<int>& out, int nb, int& start, int& end) {
    for (size_t k = 0; k < in.size(); ++k) { out[k] = enc_travel(start, end, nb, in[k]); child(start, end, nb, in[k]); }
  }
  // value of axis d's bits spread over levels, most significant level first (TransposeBits)
  static std::vector<int> bits_by_level(const int* v, int nv, int nlev) {
    std::vector<int> out(nlev, 0), tmp(v, v + nv);
    for (int lev = nlev - 1; lev >= 0; --lev) {
      int o = 0;
      for (int d = 0; d < nv; ++d) { o = (o << 1) + tmp[d] % 2; tmp[d] = (int)((unsigned)tmp[d] >> 1); }
      out[lev] = o;
    }
    return out;
  }
  static std::vector<int> levels_to_bits(const std::vector<int>& lev, int nv) {
    std::vector<int> out(nv, 0), tmp(lev);
    for (int d = nv - 1; d >= 0; --d) {
      int o = 0;
      for (size_t k = 0; k < tmp.size(); ++k) { o = (o << 1) + tmp[k] % 2; tmp[k] = (int)((unsigned)tmp[k] >> 1); }
      out[d] = o;
    }
    return out;
  }
  static std::vector<int> digits(int v, int base, int n) {
    std::vector<int> d(n, 0);
    for (int k = n - 1; k >= 0; --k) { d[k] = v % base; v /= base; }
    return d;
  }
  static int pack(const std::vector<int>& d, int base) {
    int v = d.empty() ? 0 : d[0];
    for (size_t k = 1; k < d.size(); ++k) v = v * base + d[k];
    return v;
  }
};

struct CellInfo {
  bool pbc[3], folded[3];
  int system_type;
  double gap_lo[3], gap_hi[3], amin[3], amax[3];
};

void extent(const Geometry& g, int d, double lo, double hi, bool limited, double& emin, double& emax) {
  emin = HUGE_VAL; emax = 0.0;
  for (int i = 0; i < g.n_atoms; ++i) {
    double v = g.coord[3 * i + d];
    if (limited) { if (v > emax && v <= hi) emax = v; if (v < emin && v >= lo) emin = v; }
    else { emax = std::max(emax, v); emin = std::min(emin, v); }
  }
  if (emin > emax) emin = emax;
}

CellInfo cell_info(const Geometry& g, const GeometryParams& prm) {
  CellInfo F;
  double rb[3], minr = HUGE_VAL;
  for (int d = 0; d < 3; ++d) { rb[d] = g.cell[d] / 10.0; minr = std::min(minr, rb[d]); }
  // reference picks the first minimum in axis order; min() is equivalent
  minr = std::max(minr, prm.avg_atomic_diameter);
  int nb[3];
  for (int d = 0; d < 3; ++d) { nb[d] = rnd(g.cell[d] / minr); rb[d] = g.cell[d] / (double)nb[d]; }
  std::vector<int> occ((size_t)nb[0] * nb[1] * nb[2], 0);
  for (int i = 0; i < g.n_atoms; ++i) {
    int b[3];
    for (int d = 0; d < 3; ++d) b[d] = (int)std::floor((g.coord[3 * i + d] + kShift) / rb[d]);
    occ[((size_t)b[0] * nb[1] + b[1]) * nb[2] + b[2]] += 1;
  }
  F.system_type = 3;
  for (int d = 0; d < 3; ++d) {
    F.pbc[d] = true; F.folded[d] = false; F.gap_lo[d] = F.gap_hi[d] = 0.0;
    extent(g, d, 0, 0, false, F.amin[d], F.amax[d]);
    // longest run of empty slabs perpendicular to d (1-based slab numbers, 0 = none)
    int t1 = (d + 1) % 3, t2 = (d + 2) % 3;
    int best = 0, gs = 0, ge = 0, run_start = 0;
    bool in_run = false;
    for (int a = 1; a <= nb[d]; ++a) {
      bool found = false;
      for (int b1 = 0; b1 < nb[t1] && !found; ++b1)
        for (int b2 = 0; b2 < nb[t2] && !found; ++b2) {
          int idx[3]; idx[d] = a - 1; idx[t1] = b1; idx[t2] = b2;
          if (occ[((size_t)idx[0] * nb[1] + idx[1]) * nb[2] + idx[2]] > 0) found = true;
        }
      if (found && in_run) { in_run = false; if (a - run_start > best) { best = a - run_start; gs = run_start; ge = a - 1; } }
      if (!in_run && !found) { run_start = a; in_run = true; }
      if (in_run && !found && a == nb[d]) { if (a - run_start + 1 > best) { best = a - run_start + 1; gs = run_start; ge = a; } }
    }
    if (gs > 0 && ge > 0) {
      double glo = (gs - 1) * rb[d], ghi = (ge - 1) * rb[d];
      if (glo >= F.amin[d] && ghi <= F.amax[d]) {
        F.folded[d] = true;
        double t;
        extent(g, d, F.amin[d], glo, true, t, F.gap_lo[d]);
        extent(g, d, ghi, F.amax[d], true, F.gap_hi[d], t);
        if ((F.gap_hi[d] - F.gap_lo[d]) / g.cell[d] > 0.5) { F.system_type -= 1; F.pbc[d] = false; }
      } else {
        // the reference tests 1 - (atom extent) against the threshold; kept as written
        if (1.0 - (F.amax[d] - F.amin[d]) > prm.gap_threshold) { F.system_type -= 1; F.pbc[d] = false; }
        if (glo >= F.amax[d]) { F.gap_lo[d] = F.amax[d]; F.gap_hi[d] = g.cell[d]; }
        else if (ghi <= F.amin[d]) { F.gap_lo[d] = 0.0; F.gap_hi[d] = F.amin[d]; }
      }
    }
  }
  return F;
}

int log2_ceil(int x) { int y = 0; while ((1 << y) < x) ++y; return y; }

void partition_cell(Geometry& g, const GeometryParams& prm) {
  CellInfo F = cell_info(g, prm);
  const int N = g.n_atoms;
  int cap = std::min(std::max(N, 1), prm.max_atoms_part);
  std::vector<int> autod, fixedd;
  std::array<int, 3> divs = {0, 0, 0};
  double rpart[3];
  for (int d = 0; d < 3; ++d) {
    if (F.pbc[d] || F.system_type == 0) autod.push_back(d);
    else { fixedd.push_back(d); divs[d] = 0; rpart[d] = g.cell[d]; }
  }
  if (!autod.empty()) {
    double occ[3];
    for (int d = 0; d < 3; ++d) occ[d] = F.folded[d] ? g.cell[d] - F.gap_hi[d] + F.gap_lo[d] : F.amax[d] - F.amin[d];
    double vol = ((double)cap / (double)N) * (occ[0] * occ[1] * occ[2]);
    if (autod.size() == 3) for (int d = 0; d < 3; ++d) rpart[d] = std::pow(vol, 1.0 / 3.0);
    else if (autod.size() == 2) {
      double area = vol / std::min(rpart[fixedd[0]], occ[fixedd[0]]);
      for (int d : autod) rpart[d] = std::sqrt(area);
    } else {
      rpart[autod[0]] = vol / (std::min(rpart[fixedd[0]], occ[fixedd[0]]) * std::min(rpart[fixedd[1]], occ[fixedd[1]]));
    }
    for (int d = 0; d < 3; ++d) {
      int np_ = rpart[d] < 1.0 ? 1 : std::max(rnd(g.cell[d] / rpart[d]), 1);
      divs[d] = log2_ceil(np_);
    }
  }
  auto part_coords = [&](int i, const double* rp, int c[3]) {
    for (int d = 0; d < 3; ++d) c[d] = (int)std::floor((g.coord[3 * i + d] + kShift) / rp[d]);
  };
  auto set_rpart = [&]() { for (int d = 0; d < 3; ++d) rpart[d] = g.cell[d] / (double)(1 << divs[d]); };
  set_rpart();
  if (!autod.empty()) {
    for (bool refine = true; refine;) {
      refine = false;
      HilbertCurve hc(divs);
      std::vector<int> cnt((size_t)1 << (divs[0] + divs[1] + divs[2]), 0);
      set_rpart();
      for (int i = 0; i < N && !refine; ++i) {
        int c[3]; part_coords(i, rpart, c);
        int h = hc.index_of(c);
        if (++cnt[h] > cap && std::min(rpart[0], std::min(rpart[1], rpart[2])) > 1.0) {
          double best = 0.0; int dir = -1;
          for (int d : autod) if (rpart[d] > best) { best = rpart[d]; dir = d; }
          divs[dir] += 1;
          refine = true;
        }
      }
    }
  }
  set_rpart();
  HilbertCurve hc(divs);
  for (int d = 0; d < 3; ++d) g.n_parts[d] = 1 << divs[d];
  int total = g.n_parts[0] * g.n_parts[1] * g.n_parts[2];
  g.np_in_cell = total;
  std::vector<std::vector<int>> members(total);
  for (int i = 0; i < N; ++i) { int c[3]; part_coords(i, rpart, c); members[hc.index_of(c)].push_back(i); }
  g.hilbert_to_cc.assign(total, 0);
  g.cc_to_seq.assign(total + 1, -1);
  g.part_natoms.assign(total + 1, 0);
  g.part_first_cell.assign(total + 1, 0);
  g.cell_to_global.clear();
  for (int h = 0; h < total; ++h) {
    int c[3]; hc.coords_of(h, c);
    int cc = (c[0] * g.n_parts[1] + c[1]) * g.n_parts[2] + c[2] + 1;
    g.hilbert_to_cc[h] = cc;
    g.cc_to_seq[cc] = h;  // one process: partition position == Hilbert position
    g.part_natoms[cc] = (int)members[h].size();
    g.part_first_cell[cc] = (int)g.cell_to_global.size();
    for (int a : members[h]) g.cell_to_global.push_back(a);
  }
}

void cc_to_xyz(const Geometry& g, int cc, int& x, int& y, int& z) {  // 1-based coords of a CC label
  int yz = g.n_parts[1] * g.n_parts[2];
  x = 1 + (cc - 1) / yz;
  y = 1 + (cc - 1 - (x - 1) * yz) / g.n_parts[2];
  z = cc - (x - 1) * yz - (y - 1) * g.n_parts[2];
}

// width of the occupied span of one axis and its left offset (calliper, primary_module.f90:268)
void calliper(int ngcell, int origin, const std::vector<char>& used, int& width, int& left) {
  int gap = 0, gap_begin = 1;
  for (int i = 1; i <= ngcell; ++i) {
    int prev = 1 + modf_(i + ngcell - 2, ngcell);
    if (used[prev] && !used[i]) {
      int n = 0;
      for (int k = i; !used[k]; k = 1 + modf_(k, ngcell)) ++n;
      if (n > gap) { gap = n; gap_begin = i; }
    }
  }
  width = ngcell - gap;
  int first = 1 + modf_(gap_begin + gap - 1, ngcell);
  left = modf_(origin - first + ngcell, ngcell);
}

}  // namespace

void build_geometry(Geometry& g, int n, const double* coords, const double* cell, const int* nsf, double cover_rcut,
                    const GeometryParams& prm) {
  CQ_CHECK(n > 0, CQ_ERR_ARG, "n_atoms must be positive");
  g.n_atoms = n;
  for (int d = 0; d < 3; ++d) { CQ_CHECK(cell[d] > 0, CQ_ERR_ARG, "cell lengths must be positive"); g.cell[d] = cell[d]; }
  g.coord.resize(3 * (size_t)n);
  g.nsf.assign(nsf, nsf + n);
  for (int i = 0; i < n; ++i) {
    CQ_CHECK(nsf[i] > 0 && nsf[i] <= 64, CQ_ERR_ARG, "block sizes must be in 1..64");
    for (int d = 0; d < 3; ++d) {
      double x = coords[3 * i + d];
      g.coord[3 * i + d] = x - std::floor((x + kShift) / cell[d]) * cell[d];
    }
  }
  partition_cell(g, prm);
  const int P = g.np_in_cell;
  // ---- primary set (make_prim): all partitions in Hilbert order
  int ox, oy, oz;
  cc_to_xyz(g, g.hilbert_to_cc[0], ox, oy, oz);
  int origin[3] = {ox, oy, oz}, width[3], left[3];
  for (int d = 0; d < 3; ++d) {
    std::vector<char> used(g.n_parts[d] + 1, 0);
    for (int q = 0; q < P; ++q) { int c[3]; cc_to_xyz(g, g.hilbert_to_cc[q], c[0], c[1], c[2]); used[c[d]] = 1; }
    calliper(g.n_parts[d], origin[d], used, width[d], left[d]);
  }
  g.part_disp.assign(3 * (size_t)P, 0);
  g.part_first_prim.assign(P + 1, 0);
  g.prim_global.clear(); g.prim_part.clear(); g.prim_seq.clear(); g.prim_x.clear();
  double dcell[3] = {g.cell[0] / g.n_parts[0], g.cell[1] / g.n_parts[1], g.cell[2] / g.n_parts[2]};
  for (int q = 0; q < P; ++q) {
    int cc = g.hilbert_to_cc[q];
    int c[3]; cc_to_xyz(g, cc, c[0], c[1], c[2]);
    for (int d = 0; d < 3; ++d) g.part_disp[3 * q + d] = modf_(c[d] + left[d] - origin[d] + g.n_parts[d], g.n_parts[d]) - left[d];
    g.part_first_prim[q] = (int)g.prim_global.size();
    for (int a = 0; a < g.part_natoms[cc]; ++a) {
      int gl = g.cell_to_global[g.part_first_cell[cc] + a];
      g.prim_global.push_back(gl);
      g.prim_part.push_back(q);
      g.prim_seq.push_back(a + 1);
      for (int d = 0; d < 3; ++d) {
        double add = (double)(origin[d] + g.part_disp[3 * q + d] - c[d]) * dcell[d];
        g.prim_x.push_back(g.coord[3 * gl + d] + add);
      }
    }
  }
  g.part_first_prim[P] = (int)g.prim_global.size();
  g.n_prim = (int)g.prim_global.size();
  g.global_to_prim.assign(n, -1);
  for (int p = 0; p < g.n_prim; ++p) g.global_to_prim[g.prim_global[p]] = p;
  // ---- covering set (convert_primary + make_cs)
  int co[3], span[3], ncov[3];
  for (int d = 0; d < 3; ++d) {
    double dx = dcell[d];
    double ro = (double)(origin[d] - 1) * dx + kVerySmall;
    co[d] = 1 + rnd(ro / dx);
    double roc = (double)(co[d] - 1) * dx;
    double lh = dx * (origin[d] - 1 - left[d]) - cover_rcut;
    double rh = dx * (origin[d] - 1 - left[d] + width[d]) + cover_rcut;
    span[d] = (int)std::ceil((roc - lh) / dx);
    ncov[d] = (int)std::ceil(rh / dx) - (co[d] - 1 - span[d]);
    double lhc = dx * (co[d] - 1 - span[d]);
    double rhc = dx * (co[d] - 1 - span[d] + ncov[d]);
    if (lh + kVerySmall < lhc) span[d] += (int)std::ceil((lhc - lh) / dx);
    if (rh > rhc + kVerySmall) ncov[d] += (int)std::ceil((rh - rhc) / dx);
    if (lh - lhc > dx) span[d] -= (int)std::floor((lh - lhc) / dx);
    if (rhc - rh > dx) ncov[d] -= (int)std::floor((rh - rhc) / dx);
    g.ncover[d] = ncov[d]; g.nspan[d] = span[d];
  }
  g.ng_cover = ncov[0] * ncov[1] * ncov[2];
  int nmod[3], minc[3];
  std::vector<int> nrep[3];
  for (int d = 0; d < 3; ++d) {
    int ng = g.n_parts[d];
    nmod[d] = ((ng + span[d] - 1) / ng) * ng;
    int occ = ncov[d] / ng, rem = ncov[d] - occ * ng;
    minc[d] = std::min(ncov[d], ng);
    nrep[d].assign(minc[d] + 1, 0);
    for (int k = 1; k <= minc[d]; ++k) nrep[d][k] = k <= rem ? occ + 1 : occ;
  }
  // home partitions of the minimal box, visited in Hilbert order of the home partition
  struct Home { int key, gx, gy, gz; };
  std::vector<Home> homes;
  for (int a = 1; a <= minc[0]; ++a)
    for (int b = 1; b <= minc[1]; ++b)
      for (int c = 1; c <= minc[2]; ++c) {
        int q[3] = {1 + modf_(co[0] + a - span[0] - 2 + nmod[0], g.n_parts[0]),
                    1 + modf_(co[1] + b - span[1] - 2 + nmod[1], g.n_parts[1]),
                    1 + modf_(co[2] + c - span[2] - 2 + nmod[2], g.n_parts[2])};
        int cc = ((q[0] - 1) * g.n_parts[1] + (q[1] - 1)) * g.n_parts[2] + q[2];
        homes.push_back({g.cc_to_seq[cc], a, b, c});
      }
  std::sort(homes.begin(), homes.end(), [](const Home& x, const Home& y) { return x.key < y.key; });
  std::vector<std::array<int, 3>> off;
  off.reserve(g.ng_cover);
  for (const Home& h : homes)
    for (int rx = 1; rx <= nrep[0][h.gx]; ++rx)
      for (int ry = 1; ry <= nrep[1][h.gy]; ++ry)
        for (int rz = 1; rz <= nrep[2][h.gz]; ++rz)
          off.push_back({h.gx - 1 - span[0] + (rx - 1) * g.n_parts[0], h.gy - 1 - span[1] + (ry - 1) * g.n_parts[1],
                         h.gz - 1 - span[2] + (rz - 1) * g.n_parts[2]});
  CQ_CHECK((int)off.size() == g.ng_cover, CQ_ERR_STATE, "covering set size mismatch");
  g.cover_label.assign(g.ng_cover, 0); g.cover_cell.assign(g.ng_cover, 0);
  g.cover_first.assign(g.ng_cover + 1, 0); g.cover_count.assign(g.ng_cover, 0);
  g.label_to_cover.assign(g.ng_cover + 1, -1);
  g.cover_x.clear(); g.cover_global.clear(); g.cover_part.clear(); g.cover_seq.clear(); g.cover_nsf.clear();
  g.cover_shift.clear();
  for (int np_ = 0; np_ < g.ng_cover; ++np_) {
    int q[3];
    double add[3];
    for (int d = 0; d < 3; ++d) {
      q[d] = 1 + modf_(co[d] + off[np_][d] + nmod[d] - 1, g.n_parts[d]);
      add[d] = (double)(co[d] + off[np_][d] - q[d]) * (g.cell[d] / (double)g.n_parts[d]);
    }
    int cc = ((q[0] - 1) * g.n_parts[1] + (q[1] - 1)) * g.n_parts[2] + q[2];
    for (int d = 0; d < 3; ++d) g.cover_shift.push_back((co[d] + off[np_][d] - q[d]) / g.n_parts[d]);
    g.cover_cell[np_] = cc;
    g.cover_label[np_] = ((off[np_][0] + span[0]) * ncov[1] + (off[np_][1] + span[1])) * ncov[2] + (off[np_][2] + span[2]) + 1;
    g.label_to_cover[g.cover_label[np_]] = np_;
    g.cover_first[np_] = (int)g.cover_global.size();
    g.cover_count[np_] = g.part_natoms[cc];
    for (int a = 0; a < g.part_natoms[cc]; ++a) {
      int gl = g.cell_to_global[g.part_first_cell[cc] + a];
      for (int d = 0; d < 3; ++d) g.cover_x.push_back(g.coord[3 * gl + d] + add[d]);
      g.cover_global.push_back(gl);
      g.cover_part.push_back(np_);
      g.cover_seq.push_back(a + 1);
      g.cover_nsf.push_back(g.nsf[gl]);
    }
  }
  g.cover_first[g.ng_cover] = (int)g.cover_global.size();
  g.n_cover_atoms = (int)g.cover_global.size();
  g.cover_home_prim.resize(g.n_cover_atoms);
  for (int c = 0; c < g.n_cover_atoms; ++c) g.cover_home_prim[c] = g.global_to_prim[g.cover_global[c]];
  // make_iprim: cover label of each primary atom's own partition
  g.prim_cover_label.resize(g.n_prim);
  for (int p = 0; p < g.n_prim; ++p) {
    const int* dsp = &g.part_disp[3 * g.prim_part[p]];
    g.prim_cover_label[p] = ((dsp[0] + span[0]) * ncov[1] + (dsp[1] + span[1])) * ncov[2] + (dsp[2] + span[2]) + 1;
  }
}

}  // namespace cqb
