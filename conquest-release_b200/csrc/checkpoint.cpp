// Checkpoint of a device-resident block matrix in the reference's matrix file format
// (dump_matrix2 / grab_matrix2, src/store_matrix_module.f90:340-430 and 1199-1421, binary
// branch: Fortran unformatted sequential records, each framed by a 4-byte length before and
// after the payload).  Records of one file (one process):
//   (inode, n_prim)                           int32 x 2
//   nsf of every primary atom                 int32 x n_prim
//   neighbours j of every primary atom        int32 x n_prim
//   sum of the neighbours' nsf per atom       int32 x n_prim
//   number of matrices (spin channels)        int32
//   per primary atom i (partition order):
//     global id of i                          int32
//     nsf of every neighbour j                int32 x jmax
//     global id of every neighbour j          int32 x jmax
//     per neighbour: (x_i - x_j) / cell       float64 x 3, one record each (fractional)
//     per matrix, per element of row i         float64, one record each (storage order)
// Global ids are 1-based input order, as id_glob.  Reading matches every stored block of the
// file to a block of this system's range by (global i, global j, image vector), so a file
// written by this library or by the reference for the same geometry and range can be read.
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>

#include "chain.hpp"

namespace cqb {

int guarded_call(const std::function<void()>& f);

namespace {

struct RangeHost {
  std::vector<int> cover;
  std::vector<int64_t> elem;
};

RangeHost range_host(System& S, int r) {
  RangeIndex& R = *S.ranges[r];
  RangeHost h;
  h.cover = R.nb_cover.download(S.stream);
  h.elem = R.nb_elem.download(S.stream);
  h.cover.resize(R.nnz);
  h.elem.resize(R.nnz);
  return h;
}

class RecordWriter {
 public:
  explicit RecordWriter(const std::string& path) : f_(std::fopen(path.c_str(), "wb")) {
    CQ_CHECK(f_ != nullptr, CQ_ERR_ARG, "cannot open " + path + " for writing");
  }
  ~RecordWriter() { if (f_) std::fclose(f_); }
  void record(const void* p, size_t bytes) {
    CQ_CHECK(bytes < (1ull << 31), CQ_ERR_ARG, "record too long for 4-byte markers");
    const int32_t m = (int32_t)bytes;
    CQ_CHECK(std::fwrite(&m, 4, 1, f_) == 1 && (bytes == 0 || std::fwrite(p, bytes, 1, f_) == 1) &&
                 std::fwrite(&m, 4, 1, f_) == 1,
             CQ_ERR_STATE, "write failed");
  }
  template <class T>
  void vec(const std::vector<T>& v) { record(v.data(), v.size() * sizeof(T)); }
  template <class T>
  void one(T v) { record(&v, sizeof(T)); }

 private:
  FILE* f_;
};

class RecordReader {
 public:
  explicit RecordReader(const std::string& path) : f_(std::fopen(path.c_str(), "rb")) {
    CQ_CHECK(f_ != nullptr, CQ_ERR_ARG, "cannot open " + path);
  }
  ~RecordReader() { if (f_) std::fclose(f_); }
  std::vector<char> record() {
    int32_t m = 0, m2 = 0;
    CQ_CHECK(std::fread(&m, 4, 1, f_) == 1 && m >= 0, CQ_ERR_ARG, "matrix file truncated (record marker)");
    std::vector<char> b((size_t)m);
    CQ_CHECK(m == 0 || std::fread(b.data(), (size_t)m, 1, f_) == 1, CQ_ERR_ARG, "matrix file truncated (record)");
    CQ_CHECK(std::fread(&m2, 4, 1, f_) == 1 && m2 == m, CQ_ERR_ARG, "matrix file record markers disagree");
    return b;
  }
  template <class T>
  std::vector<T> vec(size_t n) {
    std::vector<char> b = record();
    CQ_CHECK(b.size() == n * sizeof(T), CQ_ERR_ARG, "matrix file record has the wrong length");
    std::vector<T> v(n);
    if (n) std::memcpy(v.data(), b.data(), b.size());
    return v;
  }
  template <class T>
  T one() { return vec<T>(1)[0]; }

 private:
  FILE* f_;
};

}  // namespace

void dump_matrix_file(System& S, int r, const double* dev, const std::string& path, int inode) {
  const Geometry& g = S.geo;
  RangeIndex& R = *S.ranges[r];
  RangeHost h = range_host(S, r);
  std::vector<double> data((size_t)std::max<int64_t>(R.length, 0));
  if (R.length) CQ_CUDA(cudaMemcpyAsync(data.data(), dev, sizeof(double) * R.length, cudaMemcpyDeviceToHost, S.stream));
  host_wait(S);
  const int np = g.n_prim;
  std::vector<int32_t> nsf_i(np), jmax(np), jbeta(np);
  for (int p = 0; p < np; ++p) {
    nsf_i[p] = g.nsf[g.prim_global[p]];
    jmax[p] = R.h_row_ptr[p + 1] - R.h_row_ptr[p];
    int s = 0;
    for (int e = R.h_row_ptr[p]; e < R.h_row_ptr[p + 1]; ++e) s += g.cover_nsf[h.cover[e]];
    jbeta[p] = s;
  }
  RecordWriter w(path);
  const int32_t head[2] = {inode, np};
  w.record(head, sizeof(head));
  w.vec(nsf_i);
  w.vec(jmax);
  w.vec(jbeta);
  w.one<int32_t>(1);
  for (int p = 0; p < np; ++p) {
    const int e0 = R.h_row_ptr[p], e1 = R.h_row_ptr[p + 1];
    std::vector<int32_t> beta, idj;
    for (int e = e0; e < e1; ++e) {
      beta.push_back(g.cover_nsf[h.cover[e]]);
      idj.push_back(g.cover_global[h.cover[e]] + 1);
    }
    w.one<int32_t>(g.prim_global[p] + 1);
    w.vec(beta);
    w.vec(idj);
    for (int e = e0; e < e1; ++e) {
      const int c = h.cover[e];
      double v[3];
      for (int d = 0; d < 3; ++d) v[d] = (g.prim_x[3 * p + d] - g.cover_x[3 * c + d]) / g.cell[d];
      w.record(v, sizeof(v));
    }
    const int64_t b0 = e0 < e1 ? h.elem[e0] : 0;
    const int64_t len = (int64_t)jbeta[p] * nsf_i[p];
    for (int64_t k = 0; k < len; ++k) w.one<double>(data[(size_t)(b0 + k)]);
  }
}

// Returns the number of file blocks that matched a block of the range; blocks of the range that
// the file does not hold are set to zero.
int64_t grab_matrix_file(System& S, int r, double* dev, const std::string& path) {
  const Geometry& g = S.geo;
  RangeIndex& R = *S.ranges[r];
  RangeHost h = range_host(S, r);
  std::vector<double> data((size_t)std::max<int64_t>(R.length, 0), 0.0);
  RecordReader rd(path);
  std::vector<int32_t> head = rd.vec<int32_t>(2);
  const int nfile = head[1];
  CQ_CHECK(nfile >= 0 && nfile <= g.n_atoms, CQ_ERR_ARG, "matrix file: bad atom count");
  std::vector<int32_t> nsf_i = rd.vec<int32_t>(nfile), jmax = rd.vec<int32_t>(nfile), jbeta = rd.vec<int32_t>(nfile);
  for (int q = 0; q < nfile; ++q)
    CQ_CHECK(jmax[q] >= 0 && jbeta[q] >= 0 && nsf_i[q] >= 1 && nsf_i[q] <= 16, CQ_ERR_ARG, "matrix file: bad counts");
  const int32_t nspin = rd.one<int32_t>();
  CQ_CHECK(nspin >= 1, CQ_ERR_ARG, "matrix file: bad number of matrices");
  int64_t matched = 0;
  for (int q = 0; q < nfile; ++q) {
    const int32_t idi = rd.one<int32_t>();
    CQ_CHECK(idi >= 1 && idi <= g.n_atoms, CQ_ERR_ARG, "matrix file: atom id out of range");
    std::vector<int32_t> beta = rd.vec<int32_t>((size_t)jmax[q]), idj = rd.vec<int32_t>((size_t)jmax[q]);
    std::vector<std::array<double, 3>> vec((size_t)jmax[q]);
    for (int jj = 0; jj < jmax[q]; ++jj) {
      std::vector<double> v = rd.vec<double>(3);
      vec[jj] = {v[0], v[1], v[2]};
    }
    int64_t sum_beta = 0;
    for (int jj = 0; jj < jmax[q]; ++jj) sum_beta += beta[jj];
    CQ_CHECK(sum_beta == jbeta[q] && jmax[q] >= 0, CQ_ERR_ARG, "matrix file: neighbour block sizes disagree");
    const int64_t len = (int64_t)jbeta[q] * nsf_i[q];
    std::vector<double> row((size_t)len);
    for (int64_t k = 0; k < len; ++k) row[(size_t)k] = rd.one<double>();
    for (int s = 1; s < nspin; ++s)
      for (int64_t k = 0; k < len; ++k) rd.one<double>();     // further spin channels: not used here
    const int p = g.global_to_prim[idi - 1];
    CQ_CHECK(p >= 0, CQ_ERR_ARG, "matrix file: atom is not a primary atom of this system");
    CQ_CHECK(nsf_i[q] == g.nsf[idi - 1], CQ_ERR_ARG, "matrix file: block size of an atom differs");
    int64_t off = 0;
    for (int jj = 0; jj < jmax[q]; ++jj) {
      const int64_t blen = (int64_t)beta[jj] * nsf_i[q];
      for (int e = R.h_row_ptr[p]; e < R.h_row_ptr[p + 1]; ++e) {
        const int c = h.cover[e];
        if (g.cover_global[c] != idj[jj] - 1) continue;
        bool same = true;
        for (int d = 0; d < 3 && same; ++d)
          same = std::fabs((g.prim_x[3 * p + d] - g.cover_x[3 * c + d]) / g.cell[d] - vec[jj][d]) < 1e-8;
        if (!same) continue;
        CQ_CHECK(g.cover_nsf[c] == beta[jj], CQ_ERR_ARG, "matrix file: block size of a neighbour differs");
        std::memcpy(&data[(size_t)h.elem[e]], &row[(size_t)off], sizeof(double) * blen);
        ++matched;
        break;
      }
      off += blen;
    }
  }
  if (R.length) CQ_CUDA(cudaMemcpyAsync(dev, data.data(), sizeof(double) * R.length, cudaMemcpyHostToDevice, S.stream));
  host_wait(S);
  return matched;
}

}  // namespace cqb

using namespace cqb;

struct cq_system;
namespace cqb { System& system_of(cq_system* s); }

extern "C" {

int cq_dump_matrix(cq_system* sys, int r, const double* a_dev, const char* path, int inode) {
  return guarded_call([&] {
    System& S = system_of(sys);
    CQ_CHECK(r >= 0 && r < (int)S.ranges.size() && a_dev && path, CQ_ERR_ARG, "bad argument");
    dump_matrix_file(S, r, a_dev, path, inode);
  });
}

int cq_grab_matrix(cq_system* sys, int r, double* a_dev, const char* path, int64_t* matched) {
  return guarded_call([&] {
    System& S = system_of(sys);
    CQ_CHECK(r >= 0 && r < (int)S.ranges.size() && a_dev && path, CQ_ERR_ARG, "bad argument");
    int64_t m = grab_matrix_file(S, r, a_dev, path);
    if (matched) *matched = m;
  });
}

}  // extern "C"
