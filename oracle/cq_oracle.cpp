// ============================================================================
// CONQUEST atom-block sparse multiply -- CPU ORACLE (test infrastructure only)
// ============================================================================
//
// This file is a plain, sequential C++ restatement of the reference's index
// layer and block-sparse multiply, used ONLY as the checker for the CUDA
// product (tests/, bench.py's CPU baseline leg and __graft_entry__.smoke()).
// The product never links, loads or calls anything here.
//
// Parity status: the reference is Fortran and cannot be compiled in this
// image (no Fortran compiler, no MPI), and its own tests hold no golden
// vectors at this boundary (they are end-to-end DFT runs).  The restatement
// is therefore pinned by known-answer tests written for this build (dense
// image-expanded products, brute-force neighbour enumeration, dense eigh),
// not by reference outputs: "parity unpinned" in the strict sense.
//
// Every routine follows the reference loop order so that the index arrays
// (partition order, cover-set order, halo numbering, i_h2d, retro lists) and
// the floating-point summation order of m_kern_max/m_kern_min are those of
// the reference.  Arrays are kept 1-based (index 0 unused) to mirror the
// Fortran and keep the restatement checkable line by line.
//
// Reference files restated (paths relative to the CONQUEST-release tree):
//   src/Hilbert3D.f90                       Hilbert curve ordering
//   src/sfc_partitions_module.f90           partitions (one process)
//   src/primary_module.f90  make_prim, calliper
//   src/cover_module.f90    make_cs, convert_primary, make_iprim
//   src/matrix_elements_module.f90  get_naba, make_npxyz, make_halo, get_retr
//   src/matrix_module.f90   set_matrix_pointers2 (index array layout)
//   src/matrix_comms_module.f90  Mquest_get_local, end_part_comms
//   src/multiply_module.f90 mat_mult, loc_trans, matrix_add, addscan, mat_tran
//   src/multiply_kernel_default.f90  m_kern_max / m_kern_min
//   src/multiply_kernel_ompGemm.f90  m_kern_max / m_kern_min (timed baseline)
//   src/trans_module.f90    a_and_b, index_transpose (one process)
//   src/mult_module.f90     matrix_trace, matrix_product_trace
//
// Compile with -ffp-contract=off so that `c = c + a*b` rounds like the
// reference's default kernel built without FMA contraction.
// ============================================================================
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using std::vector;
typedef vector<int> IV;   // 1-based by convention: element 0 unused
typedef vector<double> DV;

static const double RD_ERR = 1.0e-8;        // numbers_module.f90:96
static const double very_small = 1.0e-8;    // numbers_module.f90:93
static const double shift_in_bohr = 1.0e-6; // global_module.f90:376

static int f_mod(int a, int n) { return a % n; }  // Fortran MOD (sign of a)
static int f_nint(double x) { return (int)std::lround(x); }                      // NINT / ANINT
static int f_ceiling(double x) { return (int)std::ceil(x); }
static int f_floor(double x) { return (int)std::floor(x); }

// ----------------------------------------------------------------------------
// Hilbert3D (src/Hilbert3D.f90)
// ----------------------------------------------------------------------------
struct Hilbert3D {
  int Alpha[4], Direction[4], XYZ[4];
  int DimLine, DimSquare, DimCube, NSquaresInLine, NCubesInSquare, NPointsInCube;

  static int ipow2(int e) { return 1 << e; }
  // Hilbert3D.f90 Hilbert3D_Initialise
  void init(int ax, int ay, int az) {
    Alpha[1] = ax; Alpha[2] = ay; Alpha[3] = az;
    Direction[1] = 4; Direction[2] = 2; Direction[3] = 1;
    XYZ[1] = 1; XYZ[2] = 2; XYZ[3] = 3;
    int n = 3;
    while (n > 1) {
      int newn = 1;
      for (int ii = 2; ii <= n; ++ii) {
        if (Alpha[ii - 1] < Alpha[ii]) {
          std::swap(Alpha[ii], Alpha[ii - 1]);
          std::swap(Direction[ii], Direction[ii - 1]);
          std::swap(XYZ[ii], XYZ[ii - 1]);
          newn = ii;
        }
      }
      n = newn;
    }
    DimLine = ipow2(Alpha[1] - Alpha[2]);
    DimSquare = ipow2(Alpha[2] - Alpha[3]);
    DimCube = ipow2(Alpha[3]);
    NSquaresInLine = DimLine;
    NCubesInSquare = DimSquare * DimSquare;
    NPointsInCube = DimCube * DimCube * DimCube;
  }
  static int GrayEncode(int i) { return i ^ (int)((unsigned)i >> 1); }
  static int GrayDecode(int gn) {
    int bn = gn, ii = 1;
    while (((unsigned)gn >> ii) > 0) { bn ^= (int)((unsigned)gn >> ii); ii++; }
    return bn;
  }
  static int GrayEncodeTravel(int start, int end, int nBits, int ind) {
    int travel = start ^ end;
    int mask = (1 << nBits) - 1;
    int gn = GrayEncode(ind) * (travel << 1);
    int rotated = (gn | (int)((unsigned)gn >> nBits)) & mask;
    return rotated ^ start;
  }
  static int GrayDecodeTravel(int start, int end, int nBits, int gn) {
    int travel = start ^ end;
    int mask = (1 << nBits) - 1;
    int rg = ((gn ^ start) << nBits) / (travel << 1);
    int rotated = (rg | (int)((unsigned)rg >> nBits)) & mask;
    return GrayDecode(rotated);
  }
  static void ChildStartEnd(int pS, int pE, int nDims, int pInd, int& cS, int& cE) {
    int maximum = (1 << nDims) - 1;
    int start_ind = std::max(0, (pInd - 1) & ~1);
    int end_ind = std::min(maximum, (pInd + 1) | 1);
    cS = GrayEncodeTravel(pS, pE, nDims, start_ind);
    cE = GrayEncodeTravel(pS, pE, nDims, end_ind);
  }
  static int MinLen(int n, int base) {
    int num = n, ml = 1;
    while (num >= base) { num /= base; ml++; }
    return ml;
  }
  // TransposeBits(nSrc, src, nDest, dest): src/dest 1-based
  static void TransposeBits(int nSrc, const int* src, int nDest, int* dest) {
    vector<int> input(src + 1, src + 1 + nSrc);
    for (int ii = nDest; ii >= 1; --ii) {
      int out = 0;
      for (int jj = 0; jj < nSrc; ++jj) { out = (out << 1) + input[jj] % 2; input[jj] = (int)((unsigned)input[jj] >> 1); }
      dest[ii] = out;
    }
  }
  // Hilbert3D_CoordsToInt: coords 0-based partition coords (x,y,z) -> 1-based index
  int coords_to_int(const int coords[3]) const {
    int ic[3], c[4];
    int cf[4] = {0, coords[0], coords[1], coords[2]};
    for (int ii = 1; ii <= 2; ++ii) ic[ii] = cf[XYZ[ii]] / DimCube;
    for (int ii = 1; ii <= 3; ++ii) c[ii] = cf[XYZ[ii]] % DimCube;
    int ip = ic[1] / DimSquare;
    int p[3];
    for (int ii = 1; ii <= 2; ++ii) p[ii] = ic[ii] % DimSquare;
    int l[2] = {0, ip};
    int nl = MinLen(DimLine - 1, 2), np_ = MinLen(DimSquare - 1, 2), nc = MinLen(DimCube - 1, 2);
    vector<int> ul(nl + 1), up(np_ + 1), uc(nc + 1);
    TransposeBits(1, l, nl, ul.data());
    TransposeBits(2, p, np_, up.data());
    TransposeBits(3, c, nc, uc.data());
    vector<int> il(nl + 1, 0), ipv(np_ + 1, 0), icv(nc + 1, 0);
    int start = 0, end = 1, cs, ce;
    if (DimLine > 1) {
      for (int ii = 1; ii <= nl; ++ii) {
        il[ii] = GrayDecodeTravel(start, end, 1, ul[ii]);
        ChildStartEnd(start, end, 1, il[ii], cs, ce); start = cs; end = ce;
      }
    }
    start *= 2; end *= 2;
    if (DimSquare > 1) {
      for (int ii = 1; ii <= np_; ++ii) {
        ipv[ii] = GrayDecodeTravel(start, end, 2, up[ii]);
        ChildStartEnd(start, end, 2, ipv[ii], cs, ce); start = cs; end = ce;
      }
    }
    start *= 2; end *= 2;
    if (DimCube > 1) {
      for (int ii = 1; ii <= nc; ++ii) {
        icv[ii] = GrayDecodeTravel(start, end, 3, uc[ii]);
        ChildStartEnd(start, end, 3, icv[ii], cs, ce); start = cs; end = ce;
      }
    }
    // PackIndex
    int lv = il[1]; for (int ii = 2; ii <= nl; ++ii) lv = lv * 2 + il[ii];
    int pv = ipv[1]; for (int ii = 2; ii <= np_; ++ii) pv = pv * 4 + ipv[ii];
    int cv = icv[1]; for (int ii = 2; ii <= nc; ++ii) cv = cv * 8 + icv[ii];
    int index = (lv * NCubesInSquare + pv) * NPointsInCube + cv;
    return index + 1;
  }
  // Hilbert3D_IntToCoords: 1-based index -> 0-based coords
  void int_to_coords(int ind, int coords[3]) const {
    int index = std::max(0, ind - 1);
    int ic = index / NPointsInCube, c = index % NPointsInCube;
    int ip = ic / NCubesInSquare, p = ic % NCubesInSquare;
    int l = ip;
    int nl = MinLen(NSquaresInLine - 1, 2), np_ = MinLen(NCubesInSquare - 1, 4), nc = MinLen(NPointsInCube - 1, 8);
    vector<int> il(nl + 1), ipv(np_ + 1), icv(nc + 1);
    for (int ii = nl; ii >= 1; --ii) { il[ii] = l % 2; l /= 2; }
    for (int ii = np_; ii >= 1; --ii) { ipv[ii] = p % 4; p /= 4; }
    for (int ii = nc; ii >= 1; --ii) { icv[ii] = c % 8; c /= 8; }
    vector<int> cl(nl + 1, 0), cp(np_ + 1, 0), cc(nc + 1, 0);
    int start = 0, end = 1, cs, ce;
    if (DimLine > 1) {
      for (int ii = 1; ii <= nl; ++ii) {
        cl[ii] = GrayEncodeTravel(start, end, 1, il[ii]);
        ChildStartEnd(start, end, 1, il[ii], cs, ce); start = cs; end = ce;
      }
    }
    start *= 2; end *= 2;
    if (DimSquare > 1) {
      for (int ii = 1; ii <= np_; ++ii) {
        cp[ii] = GrayEncodeTravel(start, end, 2, ipv[ii]);
        ChildStartEnd(start, end, 2, ipv[ii], cs, ce); start = cs; end = ce;
      }
    }
    start *= 2; end *= 2;
    if (DimCube > 1) {
      for (int ii = 1; ii <= nc; ++ii) {
        cc[ii] = GrayEncodeTravel(start, end, 3, icv[ii]);
        ChildStartEnd(start, end, 3, icv[ii], cs, ce); start = cs; end = ce;
      }
    }
    // PackCoords
    int lo[2], po[3], co[4];
    TransposeBits(nl, cl.data(), 1, lo);
    TransposeBits(np_, cp.data(), 2, po);
    TransposeBits(nc, cc.data(), 3, co);
    int icc1 = lo[1] * DimSquare + po[1];
    int icc2 = po[2];
    int out[4];
    out[XYZ[1]] = icc1 * DimCube + co[1];
    out[XYZ[2]] = icc2 * DimCube + co[2];
    out[XYZ[3]] = co[3];
    coords[0] = out[1]; coords[1] = out[2]; coords[2] = out[3];
  }
};

// ----------------------------------------------------------------------------
// Matrix structures (src/matrix_module.f90:63-136)
// ----------------------------------------------------------------------------
struct PartMatrix {        // type(matrix), one per primary partition
  int n_atoms = 0, part_nabs = 0, part_nd_nabs = 0, offset = 0, nd_offset = 0, array_posn = 0;
  IV n_nab, i_acc, i_nd_acc, ndimi, onsite;  // 1..n_atoms
  IV i_part, i_seq, ndimj, npxyz;            // 1..part_nabs (npxyz 1..3*part_nabs)
  DV radius;
};
struct Halo {              // type(matrix_halo)
  int np_in_halo = 0, ni_in_halo = 0, mx_part = 0, mx_halo = 0;
  IV nh_part, j_beg, lab_hcell, lab_hcover, j_seq, ndimj; // halo partitions / atoms
  IV i_halo;   // 1..mx_mcover : halo index of cover atom (0 = not in halo)
  IV i_hbeg;   // 1..ng_cover (indexed by lab_cover)
  IV ndimi;    // 1..n_prim
  vector<int64_t> i_h2d; // 1..n_prim*ni_in_halo
};
struct Trans {             // type(matrix_trans)
  IV i_prim, i_beg, i_nd_beg, n_hnab;
};
struct Range {
  double rcut = 0;
  vector<PartMatrix> mat;  // 1..groups_on_node
  IV bind;                 // the flat matrix index (aind) laid out as set_matrix_pointers2
  Halo halo;
  Trans trans;
  int length = 0;
  int mx_abs = 0;
  IV itran_addr;           // transpose destination per retro pair (1-based offsets)
};

struct System {
  // input
  int ni_in_cell = 0;
  double rcell[3];
  DV atom_coord;   // 3*N, global (input) order, wrapped
  IV nsf_glob;     // 1..N
  int global_maxatomspart = 34;
  double gap_threshold = 0.0, average_atomic_diameter = 5.0;
  // partitions (group_set)
  int n_parts[3], n_divs[3];
  int ngcellx, ngcelly, ngcellz, np_in_cell;
  IV nm_group, icell_beg, ngnode, inv_ngnode, i_cc2seq;  // indexed by icc or hilbert position
  IV id_glob;                                            // cell-order index -> global id
  DV x_atom_cell, y_atom_cell, z_atom_cell;
  IV nsf_cell;
  // primary set
  int groups_on_node, n_prim;
  int nx_origin, ny_origin, nz_origin, nleftx, nlefty, nleftz, nw_primx, nw_primy, nw_primz;
  IV idisp_primx, idisp_primy, idisp_primz, nm_nodgroup, nm_nodbeg;
  IV iprim_seq, iprim_part, ig_prim, nsf_prim;
  DV xprim, yprim, zprim;
  // cover set
  double cs_rcut;
  int c_nx_origin, c_ny_origin, c_nz_origin;
  int nspanlx, nspanly, nspanlz, ncoverx, ncovery, ncoverz, ng_cover, mx_mcover;
  IV lab_cell, lab_cover, inv_lab_cover, n_ing_cover, icover_ibeg, ig_cover, iprim_group;
  DV xcover, ycover, zcover;
  vector<Range> ranges;
};

// ----------------------------------------------------------------------------
// sfc partitions on one process (src/sfc_partitions_module.f90)
// ----------------------------------------------------------------------------
static int int_log2(int x) { int y = 0; while ((1 << y) < x) y++; return y; }  // sfc_partitions_module.f90 int_log2

struct FSCInfo { double dims[4]; int system_type; bool has_pbc[4], is_folded[4]; double gap[3][4]; double r_atoms_min[4], r_atoms_max[4]; };

// sfc_partitions_module.f90 get_extent
static void get_extent(const System& s, int dir, double& emin, double& emax, const double* limits) {
  emin = HUGE_VAL; emax = 0.0;
  for (int ii = 0; ii < s.ni_in_cell; ++ii) {
    double v = s.atom_coord[3 * ii + dir - 1];
    if (limits) {
      if (v > emax && v <= limits[1]) emax = v;
      if (v < emin && v >= limits[0]) emin = v;
    } else {
      if (v > emax) emax = v;
      if (v < emin) emin = v;
    }
  }
  if (emin > emax) emin = emax;
}
// sfc_partitions_module.f90 check_gap
static void check_gap(int dir, const int n_blocks[4], const IV& n_atoms_block, int& gap_start, int& gap_end) {
  int tran_dir[3];
  for (int ii = 1; ii <= 2; ++ii) tran_dir[ii] = (dir + ii - 1) % 3 + 1;
  int ccm[4] = {0, n_blocks[2] * n_blocks[3], n_blocks[3], 1};
  int gap = 0, tmp_start = 0, tmp_gap;
  bool start_count = false;
  gap_start = 0; gap_end = 0;
  for (int ia = 1; ia <= n_blocks[dir]; ++ia) {
    bool found_atom = false;
    for (int ib = 1; ib <= n_blocks[tran_dir[1]] && !found_atom; ++ib) {
      for (int ic = 1; ic <= n_blocks[tran_dir[2]]; ++ic) {
        int icc = (ia - 1) * ccm[dir] + (ib - 1) * ccm[tran_dir[1]] + (ic - 1) * ccm[tran_dir[2]] + 1;
        if (n_atoms_block[icc] > 0) {
          found_atom = true;
          if (start_count) {
            start_count = false;
            tmp_gap = ia - tmp_start;
            if (tmp_gap > gap) { gap = tmp_gap; gap_start = tmp_start; gap_end = ia - 1; }
          }
          break;  // exit loop_b
        }
      }
    }
    if (!start_count && !found_atom) { tmp_start = ia; start_count = true; }
    if (start_count && !found_atom && ia == n_blocks[dir]) {
      tmp_gap = ia - tmp_start + 1;
      if (tmp_gap > gap) { gap = tmp_gap; gap_start = tmp_start; gap_end = ia; }
    }
  }
}
// sfc_partitions_module.f90 get_cell_info
static void get_cell_info(const System& s, FSCInfo& F) {
  const int min_n_slices = 10;
  for (int d = 1; d <= 3; ++d) F.dims[d] = s.rcell[d - 1];
  double r_block[4];
  for (int d = 1; d <= 3; ++d) r_block[d] = F.dims[d] / (double)min_n_slices;
  double min_r_block = r_block[1];
  for (int ii = 2; ii <= 3; ++ii) if (r_block[ii] < min_r_block) min_r_block = r_block[ii];
  if (min_r_block < s.average_atomic_diameter) min_r_block = s.average_atomic_diameter;
  int n_blocks[4];
  for (int d = 1; d <= 3; ++d) n_blocks[d] = f_nint(F.dims[d] / min_r_block);
  for (int d = 1; d <= 3; ++d) r_block[d] = F.dims[d] / (double)n_blocks[d];
  int nbt = n_blocks[1] * n_blocks[2] * n_blocks[3];
  IV n_atoms_block(nbt + 1, 0);
  for (int ia = 0; ia < s.ni_in_cell; ++ia) {
    int ib[4];
    for (int d = 1; d <= 3; ++d) ib[d] = f_floor((s.atom_coord[3 * ia + d - 1] + shift_in_bohr) / r_block[d]);
    int icc = ib[1] * n_blocks[2] * n_blocks[3] + ib[2] * n_blocks[3] + ib[3] + 1;
    n_atoms_block[icc] += 1;
  }
  F.system_type = 3;
  for (int d = 1; d <= 3; ++d) { F.has_pbc[d] = true; F.is_folded[d] = false; F.gap[1][d] = F.gap[2][d] = 0.0; }
  const double no_pbc = 0.5;
  for (int ii = 1; ii <= 3; ++ii) {
    get_extent(s, ii, F.r_atoms_min[ii], F.r_atoms_max[ii], nullptr);
    int gmin, gmax;
    check_gap(ii, n_blocks, n_atoms_block, gmin, gmax);
    if (gmin > 0 && gmax > 0) {
      double rgmin = (gmin - 1) * r_block[ii], rgmax = (gmax - 1) * r_block[ii];
      if (rgmin >= F.r_atoms_min[ii] && rgmax <= F.r_atoms_max[ii]) {
        F.is_folded[ii] = true;
        double lim[2] = {F.r_atoms_min[ii], rgmin}, tmp;
        get_extent(s, ii, tmp, F.gap[1][ii], lim);
        double lim2[2] = {rgmax, F.r_atoms_max[ii]};
        get_extent(s, ii, F.gap[2][ii], tmp, lim2);
        if ((F.gap[2][ii] - F.gap[1][ii]) / F.dims[ii] > no_pbc) { F.system_type -= 1; F.has_pbc[ii] = false; }
      } else {
        // reference criterion compares 1 - extent with the threshold (kept as written)
        if (1.0 - (F.r_atoms_max[ii] - F.r_atoms_min[ii]) > s.gap_threshold) { F.system_type -= 1; F.has_pbc[ii] = false; }
        if (rgmin >= F.r_atoms_max[ii]) { F.gap[1][ii] = F.r_atoms_max[ii]; F.gap[2][ii] = F.dims[ii]; }
        else if (rgmax <= F.r_atoms_min[ii]) { F.gap[1][ii] = 0.0; F.gap[2][ii] = F.r_atoms_min[ii]; }
      }
    }
  }
}

// sfc_partitions_module.f90 setup_partitions/get_initial_partitions/construct_cq_partitions (numprocs = 1)
static void make_partitions(System& s) {
  FSCInfo F;
  get_cell_info(s, F);
  const int N = s.ni_in_cell;
  int max_natoms_part = std::min(std::max(N, 1), s.global_maxatomspart);
  int n_dim_auto = 0, n_dim_fixed = 0, dim_auto[4] = {0, 0, 0, 0}, dim_fixed[4] = {0, 0, 0, 0};
  double r_part[4];
  for (int ii = 1; ii <= 3; ++ii) {
    if (F.has_pbc[ii] || F.system_type == 0) { dim_auto[++n_dim_auto] = ii; }
    else { dim_fixed[++n_dim_fixed] = ii; s.n_parts[ii - 1] = 1; s.n_divs[ii - 1] = 0; r_part[ii] = F.dims[ii]; }
  }
  if (n_dim_auto > 0) {
    double r_occ[4];
    for (int ii = 1; ii <= 3; ++ii)
      r_occ[ii] = F.is_folded[ii] ? F.dims[ii] - F.gap[2][ii] + F.gap[1][ii] : F.r_atoms_max[ii] - F.r_atoms_min[ii];
    double v_part = ((double)max_natoms_part / (double)N) * (r_occ[1] * r_occ[2] * r_occ[3]);
    if (n_dim_auto == 3) {
      for (int ii = 1; ii <= 3; ++ii) r_part[ii] = std::pow(v_part, 1.0 / 3.0);
    } else if (n_dim_auto == 2) {
      double area = v_part / std::min(r_part[dim_fixed[1]], r_occ[dim_fixed[1]]);
      for (int ii = 1; ii <= 2; ++ii) r_part[dim_auto[ii]] = std::sqrt(area);
    } else {
      r_part[dim_auto[1]] = v_part / (std::min(r_part[dim_fixed[1]], r_occ[dim_fixed[1]]) *
                                      std::min(r_part[dim_fixed[2]], r_occ[dim_fixed[2]]));
    }
    for (int ii = 1; ii <= 3; ++ii) {
      int np_;
      if (r_part[ii] < 1.0) np_ = 1; else np_ = std::max(f_nint(F.dims[ii] / r_part[ii]), 1);
      s.n_divs[ii - 1] = int_log2(np_);
      s.n_parts[ii - 1] = 1 << s.n_divs[ii - 1];
      r_part[ii] = F.dims[ii] / (double)s.n_parts[ii - 1];
    }
  }
  Hilbert3D H;
  auto part_of = [&](int ia, int* ixyz) {
    for (int d = 0; d < 3; ++d) ixyz[d] = f_floor((s.atom_coord[3 * ia + d] + shift_in_bohr) / r_part[d + 1]);
  };
  if (n_dim_auto > 0) {
    bool refine = true;
    while (refine) {
      refine = false;
      int total = s.n_parts[0] * s.n_parts[1] * s.n_parts[2];
      IV cnt(total + 1, 0);
      H.init(s.n_divs[0], s.n_divs[1], s.n_divs[2]);
      for (int d = 1; d <= 3; ++d) r_part[d] = F.dims[d] / (double)s.n_parts[d - 1];
      for (int ia = 0; ia < N; ++ia) {
        int ixyz[3]; part_of(ia, ixyz);
        int ih = H.coords_to_int(ixyz);
        cnt[ih] += 1;
        double minr = std::min(r_part[1], std::min(r_part[2], r_part[3]));
        if (cnt[ih] > max_natoms_part && minr > 1.0) {
          refine = true;
          // refine_direction: longest partition edge among refinable dims
          double max_r = 0.0; int dir = 0;
          for (int k = 1; k <= n_dim_auto; ++k) { int d = dim_auto[k]; if (r_part[d] > max_r) { max_r = r_part[d]; dir = d; } }
          s.n_divs[dir - 1] += 1;
          s.n_parts[dir - 1] = 1 << s.n_divs[dir - 1];
          r_part[dir] = F.dims[dir] / (double)s.n_parts[dir - 1];
          break;
        }
      }
    }
  }
  H.init(s.n_divs[0], s.n_divs[1], s.n_divs[2]);
  for (int d = 1; d <= 3; ++d) r_part[d] = F.dims[d] / (double)s.n_parts[d - 1];
  int total = s.n_parts[0] * s.n_parts[1] * s.n_parts[2];
  IV cnt(total + 1, 0);
  for (int ia = 0; ia < N; ++ia) {
    int ixyz[3]; part_of(ia, ixyz);
    int ih = H.coords_to_int(ixyz);
    cnt[ih] += 1;
    if (cnt[ih] > max_natoms_part) max_natoms_part = cnt[ih];
  }
  vector<IV> members(total + 1);
  for (int ia = 0; ia < N; ++ia) {
    int ixyz[3]; part_of(ia, ixyz);
    members[H.coords_to_int(ixyz)].push_back(ia + 1);
  }
  s.ngcellx = s.n_parts[0]; s.ngcelly = s.n_parts[1]; s.ngcellz = s.n_parts[2];
  s.np_in_cell = total;
  s.nm_group.assign(total + 1, 0); s.icell_beg.assign(total + 1, 0);
  s.ngnode.assign(total + 1, 0); s.inv_ngnode.assign(total + 1, 0); s.i_cc2seq.assign(total + 1, 0);
  s.id_glob.assign(N + 1, 0);
  int counter = 1;
  for (int ii = 1; ii <= total; ++ii) {
    int c[3]; H.int_to_coords(ii, c);
    int icc = c[0] * s.n_parts[1] * s.n_parts[2] + c[1] * s.n_parts[2] + c[2] + 1;
    s.ngnode[ii] = icc;
    s.nm_group[icc] = (int)members[ii].size();
    s.icell_beg[icc] = counter;
    for (size_t a = 0; a < members[ii].size(); ++a) s.id_glob[counter + (int)a] = members[ii][a];
    counter += (int)members[ii].size();
  }
  for (int np_ = 1; np_ <= total; ++np_) s.inv_ngnode[s.ngnode[np_]] = np_;   // io_module.f90:836-838
  for (int np_ = 1; np_ <= total; ++np_) s.i_cc2seq[s.ngnode[np_]] = np_;     // group_module.f90 make_cc2
  s.x_atom_cell.assign(N + 1, 0); s.y_atom_cell.assign(N + 1, 0); s.z_atom_cell.assign(N + 1, 0);
  s.nsf_cell.assign(N + 1, 0);
  for (int ni = 1; ni <= N; ++ni) {  // io_module.f90:840-846
    int ig = s.id_glob[ni];
    s.x_atom_cell[ni] = s.atom_coord[3 * (ig - 1) + 0];
    s.y_atom_cell[ni] = s.atom_coord[3 * (ig - 1) + 1];
    s.z_atom_cell[ni] = s.atom_coord[3 * (ig - 1) + 2];
    s.nsf_cell[ni] = s.nsf_glob[ig];
  }
}

// primary_module.f90 calliper
static void calliper(int ngcell, int n_origin, const IV& iproj, int& nw_prim, int& nleft) {
  int n_in_gap = 0, ngap_beg = 1;
  for (int i = 1; i <= ngcell; ++i) {
    int im = 1 + f_mod(i + ngcell - 2, ngcell);
    if (iproj[im] == 1 && iproj[i] == 0) {
      int n1 = 0, i1 = i;
      while (iproj[i1] == 0) { n1++; i1 = 1 + f_mod(i1, ngcell); }
      if (n1 > n_in_gap) { n_in_gap = n1; ngap_beg = i; }
    }
  }
  nw_prim = ngcell - n_in_gap;
  int i_left = 1 + f_mod(ngap_beg + n_in_gap - 1, ngcell);
  nleft = f_mod(n_origin - i_left + ngcell, ngcell);
}

// primary_module.f90 make_prim (one process: all partitions, Hilbert order)
static void make_prim(System& s) {
  int yz = s.ngcelly * s.ngcellz;
  s.groups_on_node = s.np_in_cell;
  int g0 = s.ngnode[1];
  s.nx_origin = 1 + (g0 - 1) / yz;
  s.ny_origin = 1 + (g0 - 1 - (s.nx_origin - 1) * yz) / s.ngcellz;
  s.nz_origin = g0 - (s.nx_origin - 1) * yz - (s.ny_origin - 1) * s.ngcellz;
  int mx_edge = std::max(s.ngcellx, std::max(s.ngcelly, s.ngcellz));
  IV px(mx_edge + 1, 0), py(mx_edge + 1, 0), pz(mx_edge + 1, 0);
  auto decode = [&](int g, int& nx, int& ny, int& nz) {
    nx = 1 + (g - 1) / yz; ny = 1 + (g - 1 - (nx - 1) * yz) / s.ngcellz; nz = g - (nx - 1) * yz - (ny - 1) * s.ngcellz;
  };
  for (int ng = 1; ng <= s.groups_on_node; ++ng) { int nx, ny, nz; decode(s.ngnode[ng], nx, ny, nz); px[nx] = 1; py[ny] = 1; pz[nz] = 1; }
  calliper(s.ngcellx, s.nx_origin, px, s.nw_primx, s.nleftx);
  calliper(s.ngcelly, s.ny_origin, py, s.nw_primy, s.nlefty);
  calliper(s.ngcellz, s.nz_origin, pz, s.nw_primz, s.nleftz);
  int G = s.groups_on_node;
  s.idisp_primx.assign(G + 1, 0); s.idisp_primy.assign(G + 1, 0); s.idisp_primz.assign(G + 1, 0);
  for (int ng = 1; ng <= G; ++ng) {
    int nx, ny, nz; decode(s.ngnode[ng], nx, ny, nz);
    s.idisp_primx[ng] = f_mod(nx + s.nleftx - s.nx_origin + s.ngcellx, s.ngcellx) - s.nleftx;
    s.idisp_primy[ng] = f_mod(ny + s.nlefty - s.ny_origin + s.ngcelly, s.ngcelly) - s.nlefty;
    s.idisp_primz[ng] = f_mod(nz + s.nleftz - s.nz_origin + s.ngcellz, s.ngcellz) - s.nleftz;
  }
  double dcx = s.rcell[0] / s.ngcellx, dcy = s.rcell[1] / s.ngcelly, dcz = s.rcell[2] / s.ngcellz;
  int N = s.ni_in_cell;
  s.iprim_seq.assign(N + 1, 0); s.iprim_part.assign(N + 1, 0); s.ig_prim.assign(N + 1, 0); s.nsf_prim.assign(N + 1, 0);
  s.xprim.assign(N + 1, 0); s.yprim.assign(N + 1, 0); s.zprim.assign(N + 1, 0);
  s.nm_nodgroup.assign(G + 1, 0); s.nm_nodbeg.assign(G + 1, 0);
  s.n_prim = 0; s.nm_nodbeg[1] = 1;
  for (int ng = 1; ng <= G; ++ng) {
    int g = s.ngnode[ng]; int nx, ny, nz; decode(g, nx, ny, nz);
    int nx1 = s.nx_origin + s.idisp_primx[ng], ny1 = s.ny_origin + s.idisp_primy[ng], nz1 = s.nz_origin + s.idisp_primz[ng];
    double xadd = (double)(nx1 - nx) * dcx, yadd = (double)(ny1 - ny) * dcy, zadd = (double)(nz1 - nz) * dcz;
    s.nm_nodgroup[ng] = s.nm_group[g];
    for (int ni = 1; ni <= s.nm_nodgroup[ng]; ++ni) {
      int p = ++s.n_prim;
      int cell = s.icell_beg[g] + ni - 1;
      s.iprim_seq[p] = ni; s.iprim_part[p] = ng; s.ig_prim[p] = s.id_glob[cell];
      s.xprim[p] = s.x_atom_cell[cell] + xadd; s.yprim[p] = s.y_atom_cell[cell] + yadd; s.zprim[p] = s.z_atom_cell[cell] + zadd;
      s.nsf_prim[p] = s.nsf_cell[cell];
    }
    if (ng < G) s.nm_nodbeg[ng + 1] = s.nm_nodbeg[ng] + s.nm_nodgroup[ng];
  }
}

// cover_module.f90 convert_primary + make_cs + make_iprim
static void make_cs(System& s, double gr_rcut) {
  s.cs_rcut = gr_rcut;
  double dx = s.rcell[0] / s.ngcellx, dy = s.rcell[1] / s.ngcelly, dz = s.rcell[2] / s.ngcellz;
  double dcx = dx, dcy = dy, dcz = dz;
  double ro_x = (double)(s.nx_origin - 1) * dx + very_small;
  double ro_y = (double)(s.ny_origin - 1) * dy + very_small;
  double ro_z = (double)(s.nz_origin - 1) * dz + very_small;
  int ncx_o = 1 + f_nint(ro_x / dcx), ncy_o = 1 + f_nint(ro_y / dcy), ncz_o = 1 + f_nint(ro_z / dcz);
  s.c_nx_origin = ncx_o; s.c_ny_origin = ncy_o; s.c_nz_origin = ncz_o;
  double ro_cx = (double)(ncx_o - 1) * dcx, ro_cy = (double)(ncy_o - 1) * dcy, ro_cz = (double)(ncz_o - 1) * dcz;
  double lhx = dx * (s.nx_origin - 1 - s.nleftx) - gr_rcut;
  double lhy = dy * (s.ny_origin - 1 - s.nlefty) - gr_rcut;
  double lhz = dz * (s.nz_origin - 1 - s.nleftz) - gr_rcut;
  double rhx = dx * (s.nx_origin - 1 - s.nleftx + s.nw_primx) + gr_rcut;
  double rhy = dy * (s.ny_origin - 1 - s.nlefty + s.nw_primy) + gr_rcut;
  double rhz = dz * (s.nz_origin - 1 - s.nleftz + s.nw_primz) + gr_rcut;
  s.nspanlx = f_ceiling((ro_cx - lhx) / dcx);
  s.nspanly = f_ceiling((ro_cy - lhy) / dcy);
  s.nspanlz = f_ceiling((ro_cz - lhz) / dcz);
  s.ncoverx = f_ceiling(rhx / dcx) - (ncx_o - 1 - s.nspanlx);
  s.ncovery = f_ceiling(rhy / dcy) - (ncy_o - 1 - s.nspanly);
  s.ncoverz = f_ceiling(rhz / dcz) - (ncz_o - 1 - s.nspanlz);
  double lhcx = dcx * (ncx_o - 1 - s.nspanlx), lhcy = dcy * (ncy_o - 1 - s.nspanly), lhcz = dcz * (ncz_o - 1 - s.nspanlz);
  double rhcx = dcx * (ncx_o - 1 - s.nspanlx + s.ncoverx), rhcy = dcy * (ncy_o - 1 - s.nspanly + s.ncovery),
         rhcz = dcz * (ncz_o - 1 - s.nspanlz + s.ncoverz);
  if (lhx + very_small < lhcx) s.nspanlx += f_ceiling((lhcx - lhx) / dcx);
  if (lhy + very_small < lhcy) s.nspanly += f_ceiling((lhcy - lhy) / dcy);
  if (lhz + very_small < lhcz) s.nspanlz += f_ceiling((lhcz - lhz) / dcz);
  if (rhx > rhcx + very_small) s.ncoverx += f_ceiling((rhx - rhcx) / dcx);
  if (rhy > rhcy + very_small) s.ncovery += f_ceiling((rhy - rhcy) / dcy);
  if (rhz > rhcz + very_small) s.ncoverz += f_ceiling((rhz - rhcz) / dcz);
  if (lhx - lhcx > dcx) s.nspanlx -= f_floor((lhx - lhcx) / dcx);
  if (lhy - lhcy > dcy) s.nspanly -= f_floor((lhy - lhcy) / dcy);
  if (lhz - lhcz > dcz) s.nspanlz -= f_floor((lhz - lhcz) / dcz);
  if (rhcx - rhx > dcx) s.ncoverx -= f_floor((rhx - rhcx) / dcx);
  if (rhcy - rhy > dcy) s.ncovery -= f_floor((rhy - rhcy) / dcy);
  if (rhcz - rhz > dcz) s.ncoverz -= f_floor((rhz - rhcz) / dcz);
  // make_cs proper
  int nx_o = ncx_o, ny_o = ncy_o, nz_o = ncz_o;
  s.ng_cover = s.ncoverx * s.ncovery * s.ncoverz;
  int ngc = s.ng_cover;
  IV nxc(ngc + 1), nyc(ngc + 1), nzc(ngc + 1);
  double dcellx = s.rcell[0] / (double)s.ngcellx, dcelly = s.rcell[1] / (double)s.ngcelly, dcellz = s.rcell[2] / (double)s.ngcellz;
  int nmodx = ((s.ngcellx + s.nspanlx - 1) / s.ngcellx) * s.ngcellx;
  int nmody = ((s.ngcelly + s.nspanly - 1) / s.ngcelly) * s.ngcelly;
  int nmodz = ((s.ngcellz + s.nspanlz - 1) / s.ngcellz) * s.ngcellz;
  int noccx = s.ncoverx / s.ngcellx, nremx = s.ncoverx - noccx * s.ngcellx, minx = std::min(s.ncoverx, s.ngcellx);
  int noccy = s.ncovery / s.ngcelly, nremy = s.ncovery - noccy * s.ngcelly, miny = std::min(s.ncovery, s.ngcelly);
  int noccz = s.ncoverz / s.ngcellz, nremz = s.ncoverz - noccz * s.ngcellz, minz = std::min(s.ncoverz, s.ngcellz);
  IV nrepx(minx + 1), nrepy(miny + 1), nrepz(minz + 1);
  for (int g = 1; g <= minx; ++g) nrepx[g] = (g <= nremx) ? noccx + 1 : noccx;
  for (int g = 1; g <= miny; ++g) nrepy[g] = (g <= nremy) ? noccy + 1 : noccy;
  for (int g = 1; g <= minz; ++g) nrepz[g] = (g <= nremz) ? noccz + 1 : noccz;
  int ng_in_cell = s.np_in_cell, ng_in_min = minx * miny * minz;
  IV ind_min(ng_in_min + 1), gx(ng_in_min + 1), gy(ng_in_min + 1), gz(ng_in_min + 1);
  int ind = 0;
  for (int a = 1; a <= minx; ++a)
    for (int b = 1; b <= miny; ++b)
      for (int c = 1; c <= minz; ++c) {
        ++ind;
        int nqx = 1 + f_mod(nx_o + a - s.nspanlx - 2 + nmodx, s.ngcellx);
        int nqy = 1 + f_mod(ny_o + b - s.nspanly - 2 + nmody, s.ngcelly);
        int nqz = 1 + f_mod(nz_o + c - s.nspanlz - 2 + nmodz, s.ngcellz);
        int iq = (nqx - 1) * s.ngcelly * s.ngcellz + (nqy - 1) * s.ngcellz + nqz;
        int ino = s.inv_ngnode[iq];
        ind_min[ind] = 1 + f_mod(ino - 1 + ng_in_cell, ng_in_cell);   // inode_beg(1) = 1
        gx[ind] = a; gy[ind] = b; gz[ind] = c;
      }
  // heapsort_integer_index: ind_min keys are distinct, so any sort gives the reference order
  IV order(ng_in_min);
  for (int i = 0; i < ng_in_min; ++i) order[i] = i + 1;
  std::sort(order.begin(), order.end(), [&](int p, int q) { return ind_min[p] < ind_min[q]; });
  int ic = 0;
  for (int t = 0; t < ng_in_min; ++t) {
    int k = order[t];
    for (int rx = 1; rx <= nrepx[gx[k]]; ++rx)
      for (int ry = 1; ry <= nrepy[gy[k]]; ++ry)
        for (int rz = 1; rz <= nrepz[gz[k]]; ++rz) {
          ++ic;
          nxc[ic] = gx[k] - 1 - s.nspanlx + (rx - 1) * s.ngcellx;
          nyc[ic] = gy[k] - 1 - s.nspanly + (ry - 1) * s.ngcelly;
          nzc[ic] = gz[k] - 1 - s.nspanlz + (rz - 1) * s.ngcellz;
        }
  }
  s.lab_cell.assign(ngc + 1, 0); s.lab_cover.assign(ngc + 1, 0); s.inv_lab_cover.assign(ngc + 1, 0);
  s.n_ing_cover.assign(ngc + 1, 0); s.icover_ibeg.assign(ngc + 1, 0);
  int nm_in_cover = 0;
  for (int c = 1; c <= ngc; ++c) {
    int nqx = 1 + f_mod(nx_o + nxc[c] + nmodx - 1, s.ngcellx);
    int nqy = 1 + f_mod(ny_o + nyc[c] + nmody - 1, s.ngcelly);
    int nqz = 1 + f_mod(nz_o + nzc[c] + nmodz - 1, s.ngcellz);
    int iq = (nqx - 1) * s.ngcelly * s.ngcellz + (nqy - 1) * s.ngcellz + nqz;
    s.lab_cell[c] = iq;
    s.lab_cover[c] = (nxc[c] + s.nspanlx) * s.ncovery * s.ncoverz + (nyc[c] + s.nspanly) * s.ncoverz + (nzc[c] + s.nspanlz) + 1;
    s.inv_lab_cover[s.lab_cover[c]] = c;
    nm_in_cover += s.nm_group[iq];
  }
  s.mx_mcover = nm_in_cover;
  s.xcover.assign(nm_in_cover + 1, 0); s.ycover.assign(nm_in_cover + 1, 0); s.zcover.assign(nm_in_cover + 1, 0);
  s.ig_cover.assign(nm_in_cover + 1, 0);
  s.icover_ibeg[1] = 1;
  for (int c = 1; c <= ngc; ++c) {
    int nqx = 1 + f_mod(nx_o + nxc[c] + nmodx - 1, s.ngcellx);
    int nqy = 1 + f_mod(ny_o + nyc[c] + nmody - 1, s.ngcelly);
    int nqz = 1 + f_mod(nz_o + nzc[c] + nmodz - 1, s.ngcellz);
    double xadd = (double)(nx_o + nxc[c] - nqx) * dcellx;
    double yadd = (double)(ny_o + nyc[c] - nqy) * dcelly;
    double zadd = (double)(nz_o + nzc[c] - nqz) * dcellz;
    int iq = s.lab_cell[c];
    if (s.nm_group[iq] > 0) {
      s.n_ing_cover[c] = s.nm_group[iq];
      for (int ni = 1; ni <= s.nm_group[iq]; ++ni) {
        int cell = s.icell_beg[iq] + ni - 1, dst = s.icover_ibeg[c] + ni - 1;
        s.xcover[dst] = s.x_atom_cell[cell] + xadd;
        s.ycover[dst] = s.y_atom_cell[cell] + yadd;
        s.zcover[dst] = s.z_atom_cell[cell] + zadd;
        s.ig_cover[dst] = s.id_glob[cell];
      }
    } else {
      s.n_ing_cover[c] = 0;
    }
    if (c < ngc) s.icover_ibeg[c + 1] = s.icover_ibeg[c] + s.nm_group[iq];
  }
  // make_iprim
  s.iprim_group.assign(s.n_prim + 1, 0);
  int pr = 0;
  for (int i = 1; i <= s.groups_on_node; ++i) {
    int lab = (s.idisp_primx[i] + s.nspanlx) * s.ncovery * s.ncoverz + (s.idisp_primy[i] + s.nspanly) * s.ncoverz +
              (s.idisp_primz[i] + s.nspanlz) + 1;
    for (int j = 1; j <= s.nm_nodgroup[i]; ++j) s.iprim_group[++pr] = lab;
  }
}

// ----------------------------------------------------------------------------
// Index for one range: get_naba, set_matrix_pointers2, make_npxyz, make_halo, get_retr
// (src/matrix_elements_module.f90:257-384, 517-716, 836-903; matrix_module.f90:330-400)
// ----------------------------------------------------------------------------
static void build_range(System& s, Range& R) {
  const int G = s.groups_on_node;
  double rcutsq = R.rcut * R.rcut;
  R.mat.assign(G + 1, PartMatrix());
  // get_naba (first pass counts are not needed: vectors grow)
  int inp = 1;
  R.mat[1].offset = 0; R.mat[1].nd_offset = 0;
  R.mx_abs = 0;
  for (int nn = 1; nn <= G; ++nn) {
    PartMatrix& m = R.mat[nn];
    m.part_nabs = 0; m.part_nd_nabs = 0;
    int na = s.nm_nodgroup[nn];
    m.n_atoms = na;
    int sz1 = std::max(na, 1);
    m.n_nab.assign(sz1 + 1, 0); m.i_acc.assign(sz1 + 1, 0); m.i_nd_acc.assign(sz1 + 1, 0);
    m.ndimi.assign(sz1 + 1, 0); m.onsite.assign(sz1 + 1, 0);
    m.i_part.assign(1, 0); m.i_seq.assign(1, 0); m.ndimj.assign(1, 0); m.radius.assign(1, 0.0);
    if (na > 0) {
      m.i_acc[1] = 1; m.i_nd_acc[1] = 1;
      for (int j = 1; j <= na; ++j) {
        m.n_nab[j] = 0;
        m.ndimi[j] = s.nsf_prim[inp];
        int cumu = 0;
        for (int np_ = 1; np_ <= s.ng_cover; ++np_) {
          if (s.n_ing_cover[np_] > 0) {
            for (int ni = 1; ni <= s.n_ing_cover[np_]; ++ni) {
              int ca = s.icover_ibeg[np_] + ni - 1;
              double dx = s.xcover[ca] - s.xprim[inp];
              double dy = s.ycover[ca] - s.yprim[inp];
              double dz = s.zcover[ca] - s.zprim[inp];
              double d2 = dx * dx + dy * dy + dz * dz;
              if (d2 < rcutsq - RD_ERR) {
                m.n_nab[j] += 1;
                int ist = m.i_acc[j] + m.n_nab[j] - 1;
                if ((int)m.i_part.size() <= ist) {
                  m.i_part.resize(ist + 1); m.i_seq.resize(ist + 1); m.radius.resize(ist + 1); m.ndimj.resize(ist + 1);
                }
                m.i_part[ist] = np_;
                m.i_seq[ist] = ni;
                m.radius[ist] = std::sqrt(d2);
                if (s.lab_cover[np_] == s.iprim_group[inp] && ni == j)
                  m.onsite[j] = m.nd_offset + m.i_nd_acc[j] + cumu;
                int cell = s.icell_beg[s.lab_cell[np_]] + ni - 1;
                cumu += m.ndimi[j] * s.nsf_cell[cell];
              }
            }
          }
        }
        R.mx_abs = std::max(R.mx_abs, m.n_nab[j]);
        if (j < na) {
          m.i_acc[j + 1] = m.i_acc[j] + m.n_nab[j];
          m.i_nd_acc[j + 1] = m.i_nd_acc[j] + cumu;
        }
        m.part_nabs += m.n_nab[j];
        m.part_nd_nabs += cumu;
        inp++;
      }
    } else {
      m.i_acc[1] = 1; m.i_nd_acc[1] = 1;
    }
    if (nn < G) {
      R.mat[nn + 1].offset = m.offset + m.part_nabs;
      R.mat[nn + 1].nd_offset = m.nd_offset + m.part_nd_nabs;
    }
  }
  R.length = 0;
  for (int nn = 1; nn <= G; ++nn) R.length += R.mat[nn].part_nd_nabs;
  // make_npxyz (ndimj and npxyz per neighbour)
  int ncoveryz = s.ncovery * s.ncoverz;
  for (int np_ = 1; np_ <= G; ++np_) {
    PartMatrix& m = R.mat[np_];
    int sz2 = std::max(m.part_nabs, 1);
    m.i_part.resize(sz2 + 1); m.i_seq.resize(sz2 + 1); m.radius.resize(sz2 + 1);
    m.ndimj.assign(sz2 + 1, 0); m.npxyz.assign(3 * sz2 + 1, 0);
    for (int i = 1; i <= m.n_atoms; ++i) {
      for (int nb = 1; nb <= m.n_nab[i]; ++nb) {
        int isu = m.i_acc[i] + nb - 1;
        int ind_cover = m.i_part[isu];
        int ibpartp = s.lab_cover[ind_cover];
        int nx = 1 + (ibpartp - 1) / ncoveryz;
        int ny = 1 + (ibpartp - 1 - (nx - 1) * ncoveryz) / s.ncoverz;
        int nz = ibpartp - (nx - 1) * ncoveryz - (ny - 1) * s.ncoverz;
        int npx = nx - 1 - s.nspanlx - s.idisp_primx[np_];
        int npy = ny - 1 - s.nspanly - s.idisp_primy[np_];
        int npz = nz - 1 - s.nspanlz - s.idisp_primz[np_];
        int cell = s.icell_beg[s.lab_cell[ind_cover]] + m.i_seq[isu] - 1;
        m.ndimj[isu] = s.nsf_cell[cell];
        m.npxyz[3 * (isu - 1) + 1] = npx;
        m.npxyz[3 * (isu - 1) + 2] = npy;
        m.npxyz[3 * (isu - 1) + 3] = npz;
      }
    }
  }
  // set_matrix_pointers2: flat index layout per partition
  R.bind.assign(1, 0);
  int offset = 0;
  for (int i = 1; i <= G; ++i) {
    PartMatrix& m = R.mat[i];
    m.array_posn = offset + 1;
    int size1 = m.n_atoms > 0 ? m.n_atoms : 1;
    int size2 = m.part_nabs > 0 ? m.part_nabs : 1;
    for (int k = 1; k <= size1; ++k) R.bind.push_back(m.n_nab[k]);
    for (int k = 1; k <= size1; ++k) R.bind.push_back(m.i_acc[k]);
    for (int k = 1; k <= size1; ++k) R.bind.push_back(m.i_nd_acc[k]);
    for (int k = 1; k <= size2; ++k) R.bind.push_back(m.i_seq[k]);
    for (int k = 1; k <= 3 * size2; ++k) R.bind.push_back(m.npxyz[k]);
    for (int k = 1; k <= size2; ++k) R.bind.push_back(m.ndimj[k]);
    offset += 3 * size1 + 5 * size2;
  }
  // make_halo
  Halo& h = R.halo;
  h.i_halo.assign(s.mx_mcover + 1, 0);
  h.i_hbeg.assign(s.ng_cover + 1, 0);
  h.ndimi.assign(s.n_prim + 1, 0);
  int pr = 1;
  for (int i = 1; i <= G; ++i)
    for (int j = 1; j <= R.mat[i].n_atoms; ++j) {
      h.ndimi[pr] = R.mat[i].ndimi[j];
      for (int nb = 1; nb <= R.mat[i].n_nab[j]; ++nb) {
        int e = R.mat[i].i_acc[j] + nb - 1;
        h.i_halo[s.icover_ibeg[R.mat[i].i_part[e]] + R.mat[i].i_seq[e] - 1] = 1;
      }
      pr++;
    }
  h.np_in_halo = 0; h.ni_in_halo = 0;
  h.nh_part.assign(1, 0); h.j_beg.assign(1, 0); h.lab_hcell.assign(1, 0); h.lab_hcover.assign(1, 0);
  h.j_seq.assign(1, 0); h.ndimj.assign(1, 0);
  for (int np_ = 1; np_ <= s.ng_cover; ++np_) {
    int in_part = 0;
    h.i_hbeg[s.lab_cover[np_]] = s.icover_ibeg[np_];
    for (int ni = 1; ni <= s.n_ing_cover[np_]; ++ni) {
      int ca = s.icover_ibeg[np_] + ni - 1;
      if (h.i_halo[ca] == 1) {
        in_part++;
        h.ni_in_halo++;
        h.j_seq.push_back(ni);
        h.ndimj.push_back(s.nsf_cell[s.icell_beg[s.lab_cell[np_]] + ni - 1]);
        h.i_halo[ca] = h.ni_in_halo;
      }
    }
    if (in_part > 0) {
      h.np_in_halo++;
      h.j_beg.push_back(h.np_in_halo == 1 ? 1 : h.j_beg[h.np_in_halo - 1] + h.nh_part[h.np_in_halo - 1]);
      h.nh_part.push_back(in_part);
      h.lab_hcell.push_back(s.lab_cell[np_]);
      h.lab_hcover.push_back(s.lab_cover[np_]);
    }
  }
  h.mx_part = h.np_in_halo; h.mx_halo = h.ni_in_halo;
  int nh = h.ni_in_halo;
  h.i_h2d.assign((size_t)s.n_prim * nh + 1, 0);
  pr = 1;
  for (int i = 1; i <= G; ++i)
    for (int j = 1; j <= R.mat[i].n_atoms; ++j) {
      PartMatrix& m = R.mat[i];
      int ist = m.nd_offset + m.i_nd_acc[j];
      int nd1 = m.ndimi[j];
      for (int nb = 1; nb <= m.n_nab[j]; ++nb) {
        int isu = m.i_acc[j] + nb - 1;
        int hh = h.i_halo[s.icover_ibeg[m.i_part[isu]] + m.i_seq[isu] - 1];
        h.i_h2d[(size_t)(pr - 1) * nh + hh] = ist;
        ist += nd1 * m.ndimj[isu];
      }
      pr++;
    }
  // get_retr
  Trans& t = R.trans;
  t.n_hnab.assign(nh + 1, 0); t.i_beg.assign(nh + 1, 0); t.i_nd_beg.assign(nh + 1, 0);
  t.i_prim.assign(1, 0);
  t.i_beg[1] = 1; t.i_nd_beg[1] = 1;
  for (int ni = 1; ni <= nh; ++ni) {
    int cumu = 0;
    for (int i = 1; i <= s.n_prim; ++i) {
      if (h.i_h2d[(size_t)(i - 1) * nh + ni] != 0) {
        t.n_hnab[ni]++;
        cumu += h.ndimi[i] * h.ndimj[ni];
        t.i_prim.push_back(i);
      }
    }
    if (ni < nh) { t.i_beg[ni + 1] = t.i_beg[ni] + t.n_hnab[ni]; t.i_nd_beg[ni + 1] = t.i_nd_beg[ni] + cumu; }
  }
  // a_and_b + index_transpose (one process, transpose within the same range):
  // itran_addr(pair) = i_h2d position in the transpose for each retro pair.
  R.itran_addr.assign(1, 0);
  int na_ = 0, ia = 0, npr = 0;
  for (int npp = 1; npp <= h.np_in_halo; ++npp) {
    na_++;
    int ind_part = h.lab_hcell[na_];
    int ind_covera = h.lab_hcover[na_] - 1;
    int nxa = ind_covera / ncoveryz, nya = (ind_covera - nxa * ncoveryz) / s.ncoverz, nza = ind_covera - nxa * ncoveryz - nya * s.ncoverz;
    for (int n = 1; n <= h.nh_part[na_]; ++n) {
      ia++;
      int ind_seq = h.j_seq[ia];
      for (int i = 1; i <= t.n_hnab[ia]; ++i) {
        npr++;
        int ip = t.i_prim[npr];
        int ind_coverb = s.iprim_group[ip] - 1;
        int nxb = ind_coverb / ncoveryz, nyb = (ind_coverb - nxb * ncoveryz) / s.ncoverz, nzb = ind_coverb - nxb * ncoveryz - nyb * s.ncoverz;
        int ipart_b = (nxb - nxa) * ncoveryz + (nyb - nya) * s.ncoverz + (nzb - nza);
        int iseq_b = s.iprim_seq[ip];
        // index_transpose
        int iiip = s.i_cc2seq[ind_part];
        int ipd = s.nm_nodbeg[iiip] + ind_seq - 1;
        int noffx = 1 + s.nspanlx + s.idisp_primx[iiip];
        int noffy = 1 + s.nspanly + s.idisp_primy[iiip];
        int noffz = 1 + s.nspanlz + s.idisp_primz[iiip];
        int jjjp = ipart_b + (noffx - 1) * ncoveryz + (noffy - 1) * s.ncoverz + noffz;
        if (jjjp < 1 || jjjp > s.ng_cover) { fprintf(stderr, "oracle: index_transpose jjjp out of range\n"); abort(); }
        int ih = h.i_halo[h.i_hbeg[jjjp] + iseq_b - 1];
        R.itran_addr.push_back((int)h.i_h2d[(size_t)(ipd - 1) * nh + ih]);
      }
    }
  }
}

// ----------------------------------------------------------------------------
// multiply (src/multiply_module.f90, src/multiply_kernel_default.f90, src/multiply_kernel_ompGemm.f90)
// ----------------------------------------------------------------------------
// loc_trans (multiply_module.f90:454-539)
static void loc_trans(const Range& R, double* a /*1-based*/, double* atrans /*1-based*/, int invdir) {
  const Halo& h = R.halo; const Trans& t = R.trans;
  int nh = h.ni_in_halo;
  for (int ni = 1; ni <= nh; ++ni) {
    int tpos = t.i_nd_beg[ni];
    int nd2 = h.ndimj[ni];
    for (int nn = 1; nn <= t.n_hnab[ni]; ++nn) {
      int i = t.i_prim[t.i_beg[ni] + nn - 1];
      int istart = (int)h.i_h2d[(size_t)(i - 1) * nh + ni];
      int nd1 = h.ndimi[i];
      for (int n1 = 1; n1 <= nd1; ++n1)
        for (int n2 = 1; n2 <= nd2; ++n2) {
          if (invdir == 0) atrans[(n1 - 1) * nd2 + n2 - 1 + tpos] = a[(n2 - 1) * nd1 + n1 - 1 + istart];
          else a[(n2 - 1) * nd1 + n1 - 1 + istart] = atrans[(n1 - 1) * nd2 + n2 - 1 + tpos];
        }
      tpos += nd2 * nd1;
    }
  }
}

struct KernArgs {
  int k_off, kpart;
  const int* ib_nd_acc; const int* ibaddr; const int* nbnab; const int* ibpart; const int* ibseq; const int* bndim2;  // 1-based views
  double* a; const double* b; double* c;   // 1-based views
  const Halo* ahalo; const Halo* chalo; const Trans* at;
};

// m_kern_max, default kernel (multiply_kernel_default.f90:132-224); FMA = true: the same terms in
// the same order, each multiply-add fused (std::fma, one rounding)
template <bool FMA = false>
static void m_kern_max_default(const KernArgs& K) {
  const Halo& ah = *K.ahalo; const Halo& ch = *K.chalo; const Trans& at = *K.at;
  vector<int> jbnab2ch(64);
  for (int k = 1; k <= ah.nh_part[K.kpart]; ++k) {
    int k_in_halo = ah.j_beg[K.kpart] + k - 1;
    int k_in_part = ah.j_seq[k_in_halo];
    int nbkbeg = K.ibaddr[k_in_part];
    int nb_nd_kbeg = K.ib_nd_acc[k_in_part];
    int nd3 = ah.ndimj[k_in_halo];
    int nbn = K.nbnab[k_in_part];
    if ((int)jbnab2ch.size() < nbn + 1) jbnab2ch.resize(nbn + 1);
    for (int j = 1; j <= nbn; ++j) {
      int jpart = K.ibpart[nbkbeg + j - 1] + K.k_off;
      int jseq = K.ibseq[nbkbeg + j - 1];
      jbnab2ch[j] = ch.i_halo[ch.i_hbeg[jpart] + jseq - 1];
    }
    int nabeg = at.i_nd_beg[k_in_halo];
    for (int i = 1; i <= at.n_hnab[k_in_halo]; ++i) {
      int i_in_prim = at.i_prim[at.i_beg[k_in_halo] + i - 1];
      int nd1 = ah.ndimi[i_in_prim];
      size_t icad = (size_t)(i_in_prim - 1) * ch.ni_in_halo;
      int nbbeg = nb_nd_kbeg;
      for (int j = 1; j <= nbn; ++j) {
        int nd2 = K.bndim2[nbkbeg + j - 1];
        int j_in_halo = jbnab2ch[j];
        if (j_in_halo != 0) {
          int ncbeg = (int)ch.i_h2d[icad + j_in_halo];
          if (ncbeg != 0) {
            for (int n2 = 1; n2 <= nd2; ++n2) {
              int nbaddr = nbbeg + nd3 * (n2 - 1);
              int ncaddr = ncbeg + nd1 * (n2 - 1);
              for (int n1 = 1; n1 <= nd1; ++n1) {
                int naaddr = nabeg + nd3 * (n1 - 1);
                for (int n3 = 1; n3 <= nd3; ++n3)
                  K.c[ncaddr + n1 - 1] = FMA ? std::fma(K.a[naaddr + n3 - 1], K.b[nbaddr + n3 - 1], K.c[ncaddr + n1 - 1])
                                             : K.c[ncaddr + n1 - 1] + K.a[naaddr + n3 - 1] * K.b[nbaddr + n3 - 1];
              }
            }
          }
        }
        nbbeg += nd3 * nd2;
      }
      nabeg += nd1 * nd3;
    }
  }
}

// m_kern_min, default kernel (multiply_kernel_default.f90:325-412); FMA as for m_kern_max_default
template <bool FMA = false>
static void m_kern_min_default(const KernArgs& K) {
  const Halo& ah = *K.ahalo; const Halo& ch = *K.chalo; const Trans& at = *K.at;
  vector<int> jbnab2ch(64);
  for (int k = 1; k <= ah.nh_part[K.kpart]; ++k) {
    int k_in_halo = ah.j_beg[K.kpart] + k - 1;
    int k_in_part = ah.j_seq[k_in_halo];
    int nbkbeg = K.ibaddr[k_in_part];
    int nb_nd_kbeg = K.ib_nd_acc[k_in_part];
    int nd3 = ah.ndimj[k_in_halo];
    int nbn = K.nbnab[k_in_part];
    if ((int)jbnab2ch.size() < nbn + 1) jbnab2ch.resize(nbn + 1);
    for (int j = 1; j <= nbn; ++j) {
      int jpart = K.ibpart[nbkbeg + j - 1] + K.k_off;
      int jseq = K.ibseq[nbkbeg + j - 1];
      jbnab2ch[j] = ch.i_halo[ch.i_hbeg[jpart] + jseq - 1];
    }
    int nabeg = at.i_nd_beg[k_in_halo];
    for (int i = 1; i <= at.n_hnab[k_in_halo]; ++i) {
      int i_in_prim = at.i_prim[at.i_beg[k_in_halo] + i - 1];
      int nd1 = ah.ndimi[i_in_prim];
      size_t icad = (size_t)(i_in_prim - 1) * ch.ni_in_halo;
      int nbbeg = nb_nd_kbeg;
      for (int j = 1; j <= nbn; ++j) {
        int nd2 = K.bndim2[nbkbeg + j - 1];
        int j_in_halo = jbnab2ch[j];
        if (j_in_halo != 0) {
          int ncbeg = (int)ch.i_h2d[icad + j_in_halo];
          if (ncbeg != 0) {
            for (int n2 = 1; n2 <= nd2; ++n2) {
              int nbaddr = nbbeg + nd3 * (n2 - 1);
              int ncaddr = ncbeg + nd1 * (n2 - 1);
              for (int n1 = 1; n1 <= nd1; ++n1) {
                int naaddr = nabeg + nd3 * (n1 - 1);
                for (int n3 = 1; n3 <= nd3; ++n3)
                  K.a[naaddr + n3 - 1] = FMA ? std::fma(K.c[ncaddr + n1 - 1], K.b[nbaddr + n3 - 1], K.a[naaddr + n3 - 1])
                                             : K.a[naaddr + n3 - 1] + K.c[ncaddr + n1 - 1] * K.b[nbaddr + n3 - 1];
              }
            }
          }
        }
        nbbeg += nd3 * nd2;
      }
      nabeg += nd1 * nd3;
    }
  }
}

// Work of one partition's kernel call without the arithmetic: the loop structure of the default
// kernel (multiply_kernel_default.f90:165-222), counting the (k, i, j) triples with a stored result
// (the ncbeg != 0 test, :198) and their flops 2 nd1 nd2 nd3.  Both mult types share the structure.
static int64_t g_cnt_triples = 0, g_cnt_flops = 0;
static void m_kern_count(const KernArgs& K) {
  const Halo& ah = *K.ahalo; const Halo& ch = *K.chalo; const Trans& at = *K.at;
  for (int k = 1; k <= ah.nh_part[K.kpart]; ++k) {
    int k_in_halo = ah.j_beg[K.kpart] + k - 1;
    int k_in_part = ah.j_seq[k_in_halo];
    int nbkbeg = K.ibaddr[k_in_part];
    int nd3 = ah.ndimj[k_in_halo];
    int nbn = K.nbnab[k_in_part];
    for (int i = 1; i <= at.n_hnab[k_in_halo]; ++i) {
      int i_in_prim = at.i_prim[at.i_beg[k_in_halo] + i - 1];
      int nd1 = ah.ndimi[i_in_prim];
      size_t icad = (size_t)(i_in_prim - 1) * ch.ni_in_halo;
      for (int j = 1; j <= nbn; ++j) {
        int jpart = K.ibpart[nbkbeg + j - 1] + K.k_off;
        int jh = ch.i_halo[ch.i_hbeg[jpart] + K.ibseq[nbkbeg + j - 1] - 1];
        if (jh == 0 || ch.i_h2d[icad + jh] == 0) continue;
        g_cnt_triples += 1;
        g_cnt_flops += 2ll * nd1 * nd3 * K.bndim2[nbkbeg + j - 1];
      }
    }
  }
}

// m_kern_max / m_kern_min, ompDoii kernel (multiply_kernel_ompDoii.f90:132-262 and its m_kern_min):
// the default kernel's arithmetic with `!$omp do` over the primary neighbours i of each k.
// Different i write different output blocks, so every element sees the default kernel's
// operation sequence: results are bit-identical to the default kernel for any thread count.
static void m_kern_doii(const KernArgs& K, int type) {
  const Halo& ah = *K.ahalo; const Halo& ch = *K.chalo; const Trans& at = *K.at;
  for (int k = 1; k <= ah.nh_part[K.kpart]; ++k) {
    int k_in_halo = ah.j_beg[K.kpart] + k - 1;
    int k_in_part = ah.j_seq[k_in_halo];
    int nbkbeg = K.ibaddr[k_in_part];
    int nb_nd_kbeg = K.ib_nd_acc[k_in_part];
    int nd3 = ah.ndimj[k_in_halo];
    int nhn = at.n_hnab[k_in_halo];
    int nbn = K.nbnab[k_in_part];
    vector<int> nd1_1st(nhn + 2, 0), nd2_1st(nbn + 2, 0), jbnab2ch(nbn + 1, 0);
    for (int i = 2; i <= nhn; ++i) nd1_1st[i] = nd1_1st[i - 1] + nd3 * ah.ndimi[at.i_prim[at.i_beg[k_in_halo] + i - 2]];
    for (int j = 2; j <= nbn; ++j) nd2_1st[j] = nd2_1st[j - 1] + nd3 * K.bndim2[nbkbeg + j - 2];
    for (int j = 1; j <= nbn; ++j) {
      int jpart = K.ibpart[nbkbeg + j - 1] + K.k_off;
      jbnab2ch[j] = ch.i_halo[ch.i_hbeg[jpart] + K.ibseq[nbkbeg + j - 1] - 1];
    }
#pragma omp for schedule(runtime)
    for (int i = 1; i <= nhn; ++i) {
      int i_in_prim = at.i_prim[at.i_beg[k_in_halo] + i - 1];
      int nd1 = ah.ndimi[i_in_prim];
      size_t icad = (size_t)(i_in_prim - 1) * ch.ni_in_halo;
      int nabeg = at.i_nd_beg[k_in_halo] + nd1_1st[i];
      for (int j = 1; j <= nbn; ++j) {
        int nd2 = K.bndim2[nbkbeg + j - 1];
        int nbbeg = nb_nd_kbeg + nd2_1st[j];
        int jh = jbnab2ch[j];
        if (jh == 0) continue;
        int ncbeg = (int)ch.i_h2d[icad + jh];
        if (ncbeg == 0) continue;
        for (int n2 = 1; n2 <= nd2; ++n2) {
          int nbaddr = nbbeg + nd3 * (n2 - 1);
          int ncaddr = ncbeg + nd1 * (n2 - 1);
          for (int n1 = 1; n1 <= nd1; ++n1) {
            int naaddr = nabeg + nd3 * (n1 - 1);
            for (int n3 = 1; n3 <= nd3; ++n3) {
              if (type == 1) K.c[ncaddr + n1 - 1] = K.c[ncaddr + n1 - 1] + K.a[naaddr + n3 - 1] * K.b[nbaddr + n3 - 1];
              else K.a[naaddr + n3 - 1] = K.a[naaddr + n3 - 1] + K.c[ncaddr + n1 - 1] * K.b[nbaddr + n3 - 1];
            }
          }
        }
      }
    }
  }
}

// scipy's bundled OpenBLAS dgemm (Fortran ABI), resolved at load time by the Python side
typedef void (*dgemm_fn)(const char*, const char*, const int*, const int*, const int*, const double*, const double*,
                         const int*, const double*, const int*, const double*, double*, const int*);
static dgemm_fn g_dgemm = nullptr;
extern "C" void orc_set_dgemm(void* fn) { g_dgemm = (dgemm_fn)fn; }

// m_kern_max, ompGemm kernel (multiply_kernel_ompGemm.f90:132-269): called by every thread of the region
static void m_kern_max_ompgemm(const KernArgs& K) {
  const Halo& ah = *K.ahalo; const Halo& ch = *K.chalo; const Trans& at = *K.at;
  for (int k = 1; k <= ah.nh_part[K.kpart]; ++k) {
    int k_in_halo = ah.j_beg[K.kpart] + k - 1;
    int k_in_part = ah.j_seq[k_in_halo];
    int nbkbeg = K.ibaddr[k_in_part];
    int nb_nd_kbeg = K.ib_nd_acc[k_in_part];
    int nd3 = ah.ndimj[k_in_halo];
    int nhn = at.n_hnab[k_in_halo];
    int nbn = K.nbnab[k_in_part];
    vector<int> nd1_1st(nhn + 2, 0), nd2_1st(nbn + 2, 0), jbnab2ch(nbn + 1, 0);
    for (int i = 2; i <= nhn; ++i) nd1_1st[i] = nd1_1st[i - 1] + nd3 * ah.ndimi[at.i_prim[at.i_beg[k_in_halo] + i - 2]];
    for (int j = 2; j <= nbn; ++j) nd2_1st[j] = nd2_1st[j - 1] + nd3 * K.bndim2[nbkbeg + j - 2];
    int maxlen = 0;
    for (int j = 1; j <= nbn; ++j) {
      int jpart = K.ibpart[nbkbeg + j - 1] + K.k_off;
      jbnab2ch[j] = ch.i_halo[ch.i_hbeg[jpart] + K.ibseq[nbkbeg + j - 1] - 1];
      maxlen += K.bndim2[nbkbeg + j - 1];
    }
    vector<double> tempb((size_t)nd3 * std::max(maxlen, 1)), tempa, tempc;
#pragma omp for schedule(runtime)
    for (int i = 1; i <= nhn; ++i) {
      int i_in_prim = at.i_prim[at.i_beg[k_in_halo] + i - 1];
      int nd1 = ah.ndimi[i_in_prim];
      int nabeg = at.i_nd_beg[k_in_halo] + nd1_1st[i];
      tempa.assign((size_t)nd1 * nd3, 0.0);
      tempc.assign((size_t)nd1 * std::max(maxlen, 1), 0.0);
      std::fill(tempb.begin(), tempb.end(), 0.0);
      for (int n1 = 1; n1 <= nd1; ++n1) {
        int naaddr = nabeg + nd3 * (n1 - 1);
        for (int n3 = 1; n3 <= nd3; ++n3) tempa[(n1 - 1) + (size_t)nd1 * (n3 - 1)] = K.a[naaddr + n3 - 1];
      }
      size_t icad = (size_t)(i_in_prim - 1) * ch.ni_in_halo;
      int sofar = 0;
      for (int j = 1; j <= nbn; ++j) {
        int nd2 = K.bndim2[nbkbeg + j - 1];
        int nbbeg = nb_nd_kbeg + nd2_1st[j];
        int jh = jbnab2ch[j];
        if (jh != 0 && ch.i_h2d[icad + jh] != 0) {
          for (int n2 = 1; n2 <= nd2; ++n2) {
            int nbaddr = nbbeg + nd3 * (n2 - 1);
            for (int n3 = 1; n3 <= nd3; ++n3) tempb[(n3 - 1) + (size_t)nd3 * (sofar + n2 - 1)] = K.b[nbaddr + n3 - 1];
          }
          sofar += nd2;
        }
      }
      if (sofar > 0) {
        double one = 1.0, zero = 0.0;
        g_dgemm("n", "n", &nd1, &sofar, &nd3, &one, tempa.data(), &nd1, tempb.data(), &nd3, &zero, tempc.data(), &nd1);
      }
      sofar = 0;
      for (int j = 1; j <= nbn; ++j) {
        int nd2 = K.bndim2[nbkbeg + j - 1];
        int jh = jbnab2ch[j];
        if (jh != 0) {
          int ncbeg = (int)ch.i_h2d[icad + jh];
          if (ncbeg != 0) {
            for (int n2 = 1; n2 <= nd2; ++n2) {
              int ncaddr = ncbeg + nd1 * (n2 - 1);
              for (int n1 = 1; n1 <= nd1; ++n1) K.c[ncaddr + n1 - 1] += tempc[(n1 - 1) + (size_t)nd1 * (sofar + n2 - 1)];
            }
            sofar += nd2;
          }
        }
      }
    }
  }
}

// m_kern_min, ompGemm kernel (multiply_kernel_ompGemm.f90:354-494)
static void m_kern_min_ompgemm(const KernArgs& K) {
  const Halo& ah = *K.ahalo; const Halo& ch = *K.chalo; const Trans& at = *K.at;
  for (int k = 1; k <= ah.nh_part[K.kpart]; ++k) {
    int k_in_halo = ah.j_beg[K.kpart] + k - 1;
    int k_in_part = ah.j_seq[k_in_halo];
    int nbkbeg = K.ibaddr[k_in_part];
    int nb_nd_kbeg = K.ib_nd_acc[k_in_part];
    int nd3 = ah.ndimj[k_in_halo];
    int nhn = at.n_hnab[k_in_halo];
    int nbn = K.nbnab[k_in_part];
    vector<int> nd1_1st(nhn + 2, 0), nd2_1st(nbn + 2, 0), jbnab2ch(nbn + 1, 0);
    for (int i = 2; i <= nhn; ++i) nd1_1st[i] = nd1_1st[i - 1] + nd3 * ah.ndimi[at.i_prim[at.i_beg[k_in_halo] + i - 2]];
    for (int j = 2; j <= nbn; ++j) nd2_1st[j] = nd2_1st[j - 1] + nd3 * K.bndim2[nbkbeg + j - 2];
    int maxlen = 0;
    for (int j = 1; j <= nbn; ++j) {
      int jpart = K.ibpart[nbkbeg + j - 1] + K.k_off;
      jbnab2ch[j] = ch.i_halo[ch.i_hbeg[jpart] + K.ibseq[nbkbeg + j - 1] - 1];
      maxlen += K.bndim2[nbkbeg + j - 1];
    }
#pragma omp for schedule(runtime)
    for (int i = 1; i <= nhn; ++i) {
      int i_in_prim = at.i_prim[at.i_beg[k_in_halo] + i - 1];
      int nd1 = ah.ndimi[i_in_prim];
      int nabeg = at.i_nd_beg[k_in_halo] + nd1_1st[i];
      size_t icad = (size_t)(i_in_prim - 1) * ch.ni_in_halo;
      int sofar = 0;
      int ml = std::max(maxlen, 1);
      vector<double> tempb((size_t)nd3 * ml, 0.0), tempc((size_t)ml * nd1, 0.0);
      for (int j = 1; j <= nbn; ++j) {
        int nd2 = K.bndim2[nbkbeg + j - 1];
        int nbbeg = nb_nd_kbeg + nd2_1st[j];
        int jh = jbnab2ch[j];
        if (jh != 0) {
          int ncbeg = (int)ch.i_h2d[icad + jh];
          if (ncbeg != 0) {
            for (int n2 = 1; n2 <= nd2; ++n2) {
              int nbaddr = nbbeg + nd3 * (n2 - 1);
              int ncaddr = ncbeg + nd1 * (n2 - 1);
              for (int n3 = 1; n3 <= nd3; ++n3) tempb[(n3 - 1) + (size_t)nd3 * (sofar + n2 - 1)] = K.b[nbaddr + n3 - 1];
              for (int n1 = 1; n1 <= nd1; ++n1) tempc[(sofar + n2 - 1) + (size_t)ml * (n1 - 1)] = K.c[ncaddr + n1 - 1];
            }
            sofar += nd2;
          }
        }
      }
      if (sofar > 0) {
        double one = 1.0;
        g_dgemm("n", "n", &nd3, &nd1, &sofar, &one, tempb.data(), &nd3, tempc.data(), &ml, &one, &K.a[nabeg], &nd3);
      }
    }
  }
}

// mat_mult (multiply_module.f90:115-359), one process: prefetch = Mquest_get_local
// kernel: 0 = default, 1 = ompGemm, 2 = ompDoii, 3 = count only, 4 = default order with fused
// multiply-add
static void mat_mult(System& s, int mult_type, int ra, int rb, int rc, double* a0, int lena, const double* b0, int lenb,
                     double* c0, int lenc, int kernel, int nthreads) {
  Range& A = s.ranges[ra]; Range& B = s.ranges[rb]; Range& C = s.ranges[rc];
  (void)lenb; (void)lenc;
  double* a = a0 - 1; const double* b = b0 - 1; double* c = c0 - 1;   // 1-based views
  vector<double> atrans_v(lena + 1, 0.0);
  double* atrans = atrans_v.data();
  // A halo / ltrans belong to range ra (type 1: amat; type 2: output), C halo to range rc
  if (mult_type == 1) {
    loc_trans(A, a, atrans, 0);
    for (int i = 1; i <= lenc; ++i) c[i] = 0.0;
  }
  int ncover_yz = s.ncovery * s.ncoverz;
  int np_in_halo = A.halo.np_in_halo;
  vector<int> part_array;
  vector<double> b_rem;
  vector<int> ibpart_rem;
  int n_cont = 0, ilen2 = 0;
#ifdef _OPENMP
  if (kernel != 0 && nthreads > 0) omp_set_num_threads(nthreads);
#endif
  int kpart_shared = 0, k_off_shared = 0;
  auto prefetch_part = [&](int kpart) {
    int ind_part = A.halo.lab_hcell[kpart];
    bool new_partition = true;
    if (kpart > 1 && ind_part == A.halo.lab_hcell[kpart - 1]) new_partition = false;
    if (new_partition) {
      int ipart = s.i_cc2seq[ind_part];
      const PartMatrix& bm = B.mat[ipart];
      n_cont = s.nm_group[ind_part];
      ilen2 = bm.part_nabs;
      // Mquest_get_local: index block copy and element copy
      int indsize = 3 * bm.n_atoms + 5 * bm.part_nabs;
      part_array.assign(indsize + 1, 0);
      for (int q = 1; q <= indsize; ++q) part_array[q] = B.bind[bm.array_posn - 1 + q];
      b_rem.assign(bm.part_nd_nabs + 1, 0.0);
      int istart2 = bm.nd_offset + bm.i_nd_acc[1] - 1;
      for (int q = 1; q <= bm.part_nd_nabs; ++q) b_rem[q] = b[istart2 + q];
      // end_part_comms
      ibpart_rem.assign(std::max(ilen2, 1) + 1, 0);
      const int* nbnab_rem = &part_array[0];
      const int* ibind_rem = &part_array[n_cont];
      const int* npxyz_rem = &part_array[3 * n_cont + ilen2];
      int noff = 0;
      for (int k = 1; k <= n_cont; ++k) {
        for (int ni = 1; ni <= nbnab_rem[k]; ++ni)
          ibpart_rem[ibind_rem[k] + ni - 1] = npxyz_rem[noff + 1 + 3 * (ni - 1)] * ncover_yz +
                                              npxyz_rem[noff + 2 + 3 * (ni - 1)] * s.ncoverz + npxyz_rem[noff + 3 + 3 * (ni - 1)];
        noff += 3 * nbnab_rem[k];
      }
    }
  };
  auto make_args = [&](int kpart, int k_off) {
    KernArgs K;
    K.k_off = k_off; K.kpart = kpart;
    K.nbnab = &part_array[0];
    K.ibaddr = &part_array[n_cont];
    K.ib_nd_acc = &part_array[2 * n_cont];
    K.ibseq = &part_array[3 * n_cont];
    K.bndim2 = &part_array[3 * n_cont + 4 * ilen2];
    K.ibpart = ibpart_rem.data();
    K.a = atrans; K.b = b_rem.data(); K.c = c;
    K.ahalo = &A.halo; K.chalo = &C.halo; K.at = &A.trans;
    return K;
  };
  if (kernel == 0 || kernel == 3 || kernel == 4) {
    for (int kpart = 1; kpart <= np_in_halo; ++kpart) {
      prefetch_part(kpart);
      KernArgs K = make_args(kpart, A.halo.lab_hcover[kpart]);
      if (kernel == 3) m_kern_count(K);
      else if (kernel == 4) { if (mult_type == 1) m_kern_max_default<true>(K); else m_kern_min_default<true>(K); }
      else if (mult_type == 1) m_kern_max_default(K);
      else m_kern_min_default(K);
    }
  } else {
#pragma omp parallel default(shared)
    {
      for (int kpart = 1; kpart <= np_in_halo; ++kpart) {
#pragma omp master
        {
          prefetch_part(kpart);
          kpart_shared = kpart;
          k_off_shared = A.halo.lab_hcover[kpart];
        }
#pragma omp barrier
        KernArgs K = make_args(kpart_shared, k_off_shared);
        if (kernel == 2) m_kern_doii(K, mult_type);
        else if (mult_type == 1) m_kern_max_ompgemm(K);
        else m_kern_min_ompgemm(K);
#pragma omp barrier
      }
    }
  }
  if (mult_type == 2) loc_trans(A, a, atrans, 1);
}

// matrix_add / addscan (multiply_module.f90:807-943): A = alpha*A + beta*B for ranges ra != rb
static void addscan(System& s, int nn, int j, Range& am, Range& bm, double* a, int lena, double* b, int lenb,
                    double alpha, double beta, int dr) {
  (void)s;
  PartMatrix& A = am.mat[nn]; PartMatrix& Bm = bm.mat[nn];
  int marker = Bm.i_acc[j];
  int aposn = A.nd_offset + A.i_nd_acc[j];
  int bposn = Bm.nd_offset + Bm.i_nd_acc[j];
  int nd1 = A.ndimi[j];
  int nbtot = (int)Bm.i_part.size() - 1;
  auto bpart = [&](int m) { return m <= nbtot ? Bm.i_part[m] : INT32_MAX; };
  auto bseq = [&](int m) { return m <= nbtot ? Bm.i_seq[m] : INT32_MAX; };
  for (int nb = 1; nb <= A.n_nab[j]; ++nb) {
    int apos_arr = A.i_acc[j] + nb - 1;
    int nd2 = A.ndimj[apos_arr];
    int bsize = nd1 * nd2;
    while (bpart(marker) < A.i_part[apos_arr]) { bposn += nd1 * Bm.ndimj[marker]; marker++; }
    if (bpart(marker) > A.i_part[apos_arr]) {
      continue;  // Fortran `cycle`: the A position is not advanced (reference behaviour)
    } else if (bpart(marker) == A.i_part[apos_arr]) {
      while (bseq(marker) < A.i_seq[apos_arr] && bpart(marker) == A.i_part[apos_arr]) { bposn += nd1 * Bm.ndimj[marker]; marker++; }
      if (bpart(marker) > A.i_part[apos_arr]) continue;
      if (bseq(marker) > A.i_seq[apos_arr]) continue;
      if (bpart(marker) == A.i_part[apos_arr] && bseq(marker) == A.i_seq[apos_arr]) {
        for (int q = 0; q < bsize; ++q) {
          if (dr == 0) a[aposn + q] = alpha * a[aposn + q] + beta * b[bposn + q];
          else b[bposn + q] = beta * b[bposn + q] + alpha * a[aposn + q];
        }
        marker++;
        bposn += bsize;
      }
    }
    aposn += bsize;
    (void)lena; (void)lenb;
  }
}
// Note on the `cycle` statements of addscan: in the reference, `cycle` skips the
// `aposn = aposn+bsize` at the loop end, so an A entry that has no partner in B
// also shifts the positions used for the later entries of that row.  With the
// nested ranges of the LNV chain the shorter list is always a subset of the
// longer one and no `cycle` is taken; the restatement keeps the reference
// behaviour for the other case as well.
static void matrix_add(System& s, double alpha, double* a0, int ra, double beta, double* b0, int rb) {
  Range& Am = s.ranges[ra]; Range& Bm = s.ranges[rb];
  double* a = a0 - 1; double* b = b0 - 1;
  for (int nn = 1; nn <= s.groups_on_node; ++nn) {
    for (int j = 1; j <= s.nm_nodgroup[nn]; ++j) {
      if (Am.mat[nn].n_nab[j] <= Bm.mat[nn].n_nab[j]) addscan(s, nn, j, Am, Bm, a, Am.length, b, Bm.length, alpha, beta, 0);
      else addscan(s, nn, j, Bm, Am, b, Bm.length, a, Am.length, beta, alpha, 1);
    }
  }
}

// ============================================================================
// C ABI for the Python side of the oracle
// ============================================================================
extern "C" {

void* orc_create(int n, const double* coords, const double* cell, const int* nsf, int n_ranges, const double* rcuts,
                 int max_atoms_part, double gap_threshold, double avg_atomic_diameter) {
  System* s = new System();
  s->ni_in_cell = n;
  for (int d = 0; d < 3; ++d) s->rcell[d] = cell[d];
  s->atom_coord.assign(3 * (size_t)n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) {  // io_module.f90:418-419 wrapping
      double x = coords[3 * i + d];
      s->atom_coord[3 * i + d] = x - std::floor((x + shift_in_bohr) / cell[d]) * cell[d];
    }
  s->nsf_glob.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) s->nsf_glob[i + 1] = nsf[i];
  s->global_maxatomspart = max_atoms_part;
  s->gap_threshold = gap_threshold;
  s->average_atomic_diameter = avg_atomic_diameter;
  make_partitions(*s);
  make_prim(*s);
  double rmax = 0;
  for (int r = 0; r < n_ranges; ++r) rmax = std::max(rmax, rcuts[r]);
  make_cs(*s, rmax);
  s->ranges.resize(n_ranges);
  for (int r = 0; r < n_ranges; ++r) { s->ranges[r].rcut = rcuts[r]; build_range(*s, s->ranges[r]); }
  return s;
}

void orc_destroy(void* h) { delete (System*)h; }

int orc_range_length(void* h, int r) { return ((System*)h)->ranges[r].length; }

// Generic array export. Returns the number of elements (0-based copy of the 1-based array body).
// range < 0 selects a system-level array.
long orc_get_int(void* h, int r, const char* name, int64_t* out, long cap) {
  System& s = *(System*)h;
  vector<int64_t> v;
  auto put = [&](const IV& x, int from = 1) { for (size_t i = from; i < x.size(); ++i) v.push_back(x[i]); };
  std::string nm(name);
  if (r < 0) {
    if (nm == "n_parts") { for (int d = 0; d < 3; ++d) v.push_back(s.n_parts[d]); }
    else if (nm == "cover_dims") { v = {s.ncoverx, s.ncovery, s.ncoverz, s.nspanlx, s.nspanly, s.nspanlz, s.ng_cover, s.mx_mcover,
                                         s.c_nx_origin, s.c_ny_origin, s.c_nz_origin}; }
    else if (nm == "prim_origin") { v = {s.nx_origin, s.ny_origin, s.nz_origin, s.nleftx, s.nlefty, s.nleftz, s.nw_primx, s.nw_primy, s.nw_primz}; }
    else if (nm == "ngnode") put(s.ngnode);
    else if (nm == "nm_group") put(s.nm_group);
    else if (nm == "icell_beg") put(s.icell_beg);
    else if (nm == "id_glob") put(s.id_glob);
    else if (nm == "ig_prim") put(s.ig_prim);
    else if (nm == "nm_nodgroup") put(s.nm_nodgroup);
    else if (nm == "idisp_prim") { for (int g = 1; g <= s.groups_on_node; ++g) { v.push_back(s.idisp_primx[g]); v.push_back(s.idisp_primy[g]); v.push_back(s.idisp_primz[g]); } }
    else if (nm == "lab_cell") put(s.lab_cell);
    else if (nm == "lab_cover") put(s.lab_cover);
    else if (nm == "n_ing_cover") put(s.n_ing_cover);
    else if (nm == "icover_ibeg") put(s.icover_ibeg);
    else if (nm == "ig_cover") put(s.ig_cover);
    else if (nm == "iprim_group") put(s.iprim_group);
    else return -1;
  } else {
    Range& R = s.ranges[r];
    if (nm == "n_nab" || nm == "i_acc" || nm == "i_nd_acc" || nm == "ndimi" || nm == "onsite") {
      for (int g = 1; g <= s.groups_on_node; ++g) {
        PartMatrix& m = R.mat[g];
        for (int j = 1; j <= m.n_atoms; ++j) {
          if (nm == "n_nab") v.push_back(m.n_nab[j]);
          else if (nm == "i_acc") v.push_back(m.offset + m.i_acc[j]);
          else if (nm == "i_nd_acc") v.push_back(m.nd_offset + m.i_nd_acc[j]);
          else if (nm == "ndimi") v.push_back(m.ndimi[j]);
          else v.push_back(m.onsite[j]);
        }
      }
    } else if (nm == "i_part" || nm == "i_seq" || nm == "ndimj" || nm == "npxyz") {
      for (int g = 1; g <= s.groups_on_node; ++g) {
        PartMatrix& m = R.mat[g];
        for (int e = 1; e <= m.part_nabs; ++e) {
          if (nm == "i_part") v.push_back(m.i_part[e]);
          else if (nm == "i_seq") v.push_back(m.i_seq[e]);
          else if (nm == "ndimj") v.push_back(m.ndimj[e]);
          else for (int q = 1; q <= 3; ++q) v.push_back(m.npxyz[3 * (e - 1) + q]);
        }
      }
    } else if (nm == "bind") put(R.bind);
    else if (nm == "array_posn") { for (int g = 1; g <= s.groups_on_node; ++g) v.push_back(R.mat[g].array_posn); }
    else if (nm == "halo_sizes") { v = {R.halo.np_in_halo, R.halo.ni_in_halo}; }
    else if (nm == "nh_part") put(R.halo.nh_part);
    else if (nm == "j_beg") put(R.halo.j_beg);
    else if (nm == "lab_hcell") put(R.halo.lab_hcell);
    else if (nm == "lab_hcover") put(R.halo.lab_hcover);
    else if (nm == "j_seq") put(R.halo.j_seq);
    else if (nm == "halo_ndimj") put(R.halo.ndimj);
    else if (nm == "i_halo") put(R.halo.i_halo);
    else if (nm == "i_hbeg") put(R.halo.i_hbeg);
    else if (nm == "i_h2d") { for (size_t q = 1; q < R.halo.i_h2d.size(); ++q) v.push_back(R.halo.i_h2d[q]); }
    else if (nm == "t_i_prim") put(R.trans.i_prim);
    else if (nm == "t_i_beg") put(R.trans.i_beg);
    else if (nm == "t_i_nd_beg") put(R.trans.i_nd_beg);
    else if (nm == "t_n_hnab") put(R.trans.n_hnab);
    else if (nm == "itran_addr") put(R.itran_addr);
    else return -1;
  }
  long n = (long)v.size();
  if (out) for (long i = 0; i < std::min(n, cap); ++i) out[i] = v[i];
  return n;
}

long orc_get_double(void* h, int r, const char* name, double* out, long cap) {
  System& s = *(System*)h;
  vector<double> v;
  std::string nm(name);
  if (r < 0) {
    if (nm == "xprim") { for (int p = 1; p <= s.n_prim; ++p) { v.push_back(s.xprim[p]); v.push_back(s.yprim[p]); v.push_back(s.zprim[p]); } }
    else if (nm == "xcover") { for (int p = 1; p <= s.mx_mcover; ++p) { v.push_back(s.xcover[p]); v.push_back(s.ycover[p]); v.push_back(s.zcover[p]); } }
    else return -1;
  } else {
    Range& R = s.ranges[r];
    if (nm == "radius") { for (int g = 1; g <= s.groups_on_node; ++g) for (int e = 1; e <= R.mat[g].part_nabs; ++e) v.push_back(R.mat[g].radius[e]); }
    else return -1;
  }
  long n = (long)v.size();
  if (out) for (long i = 0; i < std::min(n, cap); ++i) out[i] = v[i];
  return n;
}

// mat_mult with mat_mult's own argument roles (a: A or the type-2 output; c: C or the type-2 input)
int orc_mat_mult(void* h, int mult_type, int ra, int rb, int rc, double* a, int lena, const double* b, int lenb, double* c,
                 int lenc, int kernel, int nthreads) {
  System& s = *(System*)h;
  if (kernel == 1 && !g_dgemm) return 2;
  mat_mult(s, mult_type, ra, rb, rc, a, lena, b, lenb, c, lenc, kernel, nthreads);
  return 0;
}

// Triples and flops of one product (no arithmetic): the partition loop of mat_mult with the counting
// kernel; the operand arrays are scratch copies of the ranges' lengths.
int orc_product_work(void* h, int mult_type, int ra, int rb, int rc, int64_t* triples, int64_t* flops) {
  System& s = *(System*)h;
  std::vector<double> a(std::max<int64_t>(s.ranges[ra].length, 1), 0.0), b(std::max<int64_t>(s.ranges[rb].length, 1), 0.0),
      c(std::max<int64_t>(s.ranges[rc].length, 1), 0.0);
  g_cnt_triples = 0; g_cnt_flops = 0;
  mat_mult(s, mult_type, ra, rb, rc, a.data(), (int)a.size(), b.data(), (int)b.size(), c.data(), (int)c.size(), 3, 0);
  *triples = g_cnt_triples; *flops = g_cnt_flops;
  return 0;
}

void orc_matrix_add(void* h, double alpha, double* a, int ra, double beta, double* b, int rb) {
  matrix_add(*(System*)h, alpha, a, ra, beta, b, rb);
}

// matrix_transpose (mult_module.f90:2609-2673) on one process: loc_trans then mat_tran with itran_addr
void orc_matrix_transpose(void* h, int r, const double* a0, double* at0) {
  System& s = *(System*)h;
  Range& R = s.ranges[r];
  vector<double> acopy(a0, a0 + R.length);
  vector<double> tmp(R.length + 1, 0.0);
  loc_trans(R, acopy.data() - 1, tmp.data(), 0);
  double* at = at0 - 1;
  int posn = 0;
  int nh = R.halo.ni_in_halo;
  int npair = 0;
  for (int ni = 1; ni <= nh; ++ni)
    for (int nn = 1; nn <= R.trans.n_hnab[ni]; ++nn) {
      npair++;
      int ip = R.trans.i_prim[R.trans.i_beg[ni] + nn - 1];
      int count = R.halo.ndimi[ip] * R.halo.ndimj[ni];
      int dst = R.itran_addr[npair];
      for (int q = 0; q < count; ++q) at[dst + q] = tmp[posn + 1 + q];
      posn += count;
    }
}

// matrix_trace (mult_module.f90:2773-2811)
double orc_matrix_trace(void* h, int r, const double* a0) {
  System& s = *(System*)h;
  Range& R = s.ranges[r];
  const double* a = a0 - 1;
  std::vector<double> diag;
  for (int np_ = 1; np_ <= s.groups_on_node; ++np_)
    for (int i = 1; i <= s.nm_nodgroup[np_]; ++i) {
      int sf1 = R.mat[np_].ndimi[i];
      for (int j = 1; j <= sf1; ++j) diag.push_back(a[(j - 1) * sf1 + j - 1 + R.mat[np_].onsite[i]]);
    }
  // the sum over the onsite diagonal uses the order-independent exact sum (see orc_exact_sum)
  double orc_exact_sum(long n, const double* x, const double* y);
  return orc_exact_sum((long)diag.size(), diag.data(), nullptr);
}

// matrix_product_trace (mult_module.f90:2885-2916): vdot over storage, sequential sum
double orc_vdot(long n, const double* x, const double* y) {
  double s = 0.0;
  for (long i = 0; i < n; ++i) s += x[i] * y[i];
  return s;
}

// The reference's vdot/gsum order depends on the BLAS build, so the sum itself
// is not pinned by the reference.  This is the sum used by the oracle's LNV chain:
// each term (the rounded product x_i*y_i, or x_i when y is null) is added exactly
// in fixed point with 150 fraction bits below the largest term's binary
// exponent (smaller bits truncated toward zero), and the total is rounded once to
// the nearest double (ties to even).  The result does not depend on term order.
double orc_exact_sum(long n, const double* x, const double* y) {
  int emax = INT32_MIN;
  for (long i = 0; i < n; ++i) {
    double v = y ? x[i] * y[i] : x[i];
    if (!std::isfinite(v)) return NAN;
    if (v != 0.0) { int e; std::frexp(v, &e); if (e > emax) emax = e; }
  }
  if (emax == INT32_MIN) return 0.0;
  const int lsb = emax - 150;
  // 192-bit two's complement accumulator, limb 0 least significant
  uint64_t acc[3] = {0, 0, 0};
  auto add = [&](const uint64_t t[3]) {
    unsigned __int128 s = (unsigned __int128)acc[0] + t[0];
    acc[0] = (uint64_t)s;
    s = (unsigned __int128)acc[1] + t[1] + (uint64_t)(s >> 64);
    acc[1] = (uint64_t)s;
    acc[2] = acc[2] + t[2] + (uint64_t)(s >> 64);
  };
  for (long i = 0; i < n; ++i) {
    double v = y ? x[i] * y[i] : x[i];
    if (v == 0.0) continue;
    int e;
    double f = std::frexp(v, &e);
    long long m = (long long)std::ldexp(f, 53);
    bool neg = m < 0;
    unsigned __int128 mag = (unsigned __int128)(neg ? -m : m);
    int s = e - 53 - lsb;
    uint64_t t[3] = {0, 0, 0};
    if (s >= 0) {
      // place mag << s into the 192-bit word
      for (int k = 0; k < 3; ++k) {
        int lo = 64 * k;  // bit range [lo, lo+64) of the word
        int sh = lo - s;  // word bit b holds mag bit (b - s)
        uint64_t w = 0;
        if (sh >= 0) { if (sh < 128) w = (uint64_t)(mag >> sh); }
        else if (-sh < 64) w = (uint64_t)(mag << (-sh));
        t[k] = w;
      }
    } else if (-s < 64) {
      t[0] = (uint64_t)(mag >> (-s));
    }
    if (neg) {
      t[0] = ~t[0]; t[1] = ~t[1]; t[2] = ~t[2];
      uint64_t one[3] = {1, 0, 0};
      uint64_t tmp[3] = {acc[0], acc[1], acc[2]};
      acc[0] = t[0]; acc[1] = t[1]; acc[2] = t[2];
      add(one);
      t[0] = acc[0]; t[1] = acc[1]; t[2] = acc[2];
      acc[0] = tmp[0]; acc[1] = tmp[1]; acc[2] = tmp[2];
    }
    add(t);
  }
  // round to double
  bool neg = (acc[2] >> 63) != 0;
  uint64_t w[3] = {acc[0], acc[1], acc[2]};
  if (neg) {
    w[0] = ~w[0]; w[1] = ~w[1]; w[2] = ~w[2];
    if (++w[0] == 0 && ++w[1] == 0) ++w[2];
  }
  int h = -1;
  for (int b = 191; b >= 0; --b)
    if ((w[b / 64] >> (b % 64)) & 1u) { h = b; break; }
  if (h < 0) return 0.0;
  auto bit = [&](int b) -> uint64_t { return b < 0 ? 0 : (w[b / 64] >> (b % 64)) & 1u; };
  int drop = h > 52 ? h - 52 : 0;
  uint64_t m = 0;
  for (int b = h; b >= drop; --b) m = (m << 1) | bit(b);
  if (drop > 0) {
    bool half = bit(drop - 1), sticky = false;
    for (int b = drop - 2; b >= 0; --b) if (bit(b)) { sticky = true; break; }
    if (half && (sticky || (m & 1))) ++m;
  }
  double r = std::ldexp((double)m, lsb + drop);
  return neg ? -r : r;
}

}  // extern "C"
