// The reference's output and restart file formats (TopOpt.cpp:97-508,
// RecMesh.cpp:34-412), host side: raw native arrays, the PETSc binary
// Vec / AIJ matrix encoding, and the structured-mesh matrices MeshOut
// writes (the density filter, the max-length filter, the multigrid
// interpolations).
#include "io.h"

#include <cmath>
#include <cstdio>
#include <cstring>

namespace tpo {
namespace io {

namespace {

struct File {
  std::FILE *f = nullptr;
  ~File() {
    if (f) std::fclose(f);
  }
};

// big-endian encodings of the PETSc binary viewer
void put_be(std::vector<unsigned char> &b, uint64_t v, int bytes) {
  for (int i = bytes - 1; i >= 0; --i) b.push_back((unsigned char)(v >> (8 * i)));
}
uint64_t get_be(const unsigned char *p, int bytes) {
  uint64_t v = 0;
  for (int i = 0; i < bytes; ++i) v = (v << 8) | p[i];
  return v;
}
void put_int(std::vector<unsigned char> &b, int64_t v, int ib) { put_be(b, (uint64_t)v, ib); }
int64_t get_int(const unsigned char *p, int ib) {
  const uint64_t u = get_be(p, ib);
  return ib == 4 ? (int64_t)(int32_t)(uint32_t)u : (int64_t)u;
}
void put_double(std::vector<unsigned char> &b, double v) {
  uint64_t u;
  std::memcpy(&u, &v, 8);
  put_be(b, u, 8);
}
double get_double(const unsigned char *p) {
  const uint64_t u = get_be(p, 8);
  double v;
  std::memcpy(&v, &u, 8);
  return v;
}

bool check_ib(int ib, std::string &err) {
  if (ib == 4 || ib == 8) return true;
  err = "PetscInt size must be 4 or 8 bytes";
  return false;
}

// an index that must fit a 4-byte PetscInt
bool fits(int64_t v, int ib, std::string &err) {
  if (ib == 8 || (v >= INT32_MIN && v <= INT32_MAX)) return true;
  err = "index does not fit a 4-byte PetscInt";
  return false;
}

}  // namespace

bool write_raw(const std::string &path, const void *data, size_t bytes, std::string &err) {
  File f;
  f.f = std::fopen(path.c_str(), "wb");
  if (!f.f) {
    err = "cannot open " + path + " for writing";
    return false;
  }
  if (bytes && std::fwrite(data, 1, bytes, f.f) != bytes) {
    err = "short write to " + path;
    return false;
  }
  return true;
}

bool read_raw(const std::string &path, std::vector<char> &out, std::string &err) {
  File f;
  f.f = std::fopen(path.c_str(), "rb");
  if (!f.f) {
    err = "cannot open " + path;
    return false;
  }
  std::fseek(f.f, 0, SEEK_END);
  const long n = std::ftell(f.f);
  std::fseek(f.f, 0, SEEK_SET);
  out.resize(n > 0 ? (size_t)n : 0);
  if (n > 0 && std::fread(out.data(), 1, (size_t)n, f.f) != (size_t)n) {
    err = "short read from " + path;
    return false;
  }
  return true;
}

bool write_ints(const std::string &path, const int64_t *v, size_t n, int ib, std::string &err) {
  if (!check_ib(ib, err)) return false;
  if (ib == 8) return write_raw(path, v, n * 8, err);
  std::vector<int32_t> w(n);
  for (size_t i = 0; i < n; ++i) {
    if (!fits(v[i], ib, err)) return false;
    w[i] = (int32_t)v[i];
  }
  return write_raw(path, w.data(), n * 4, err);
}

bool read_ints(const std::string &path, std::vector<int64_t> &out, int ib, std::string &err) {
  if (!check_ib(ib, err)) return false;
  std::vector<char> raw;
  if (!read_raw(path, raw, err)) return false;
  if (raw.size() % ib) {
    err = path + ": size is not a multiple of the PetscInt size";
    return false;
  }
  out.resize(raw.size() / ib);
  for (size_t i = 0; i < out.size(); ++i) {
    if (ib == 8) {
      std::memcpy(&out[i], raw.data() + 8 * i, 8);
    } else {
      int32_t v;
      std::memcpy(&v, raw.data() + 4 * i, 4);
      out[i] = v;
    }
  }
  return true;
}

// VecView on a binary viewer (one process): classid, global size, values
bool write_vec(const std::string &path, const double *v, int64_t n, int ib, std::string &err) {
  if (!check_ib(ib, err) || !fits(n, ib, err)) return false;
  std::vector<unsigned char> b;
  b.reserve(2 * ib + 8 * (size_t)n);
  put_int(b, kVecClassId, ib);
  put_int(b, n, ib);
  for (int64_t i = 0; i < n; ++i) put_double(b, v[i]);
  return write_raw(path, b.data(), b.size(), err);
}

bool read_vec(const std::string &path, std::vector<double> &out, int ib, std::string &err) {
  if (!check_ib(ib, err)) return false;
  std::vector<char> raw;
  if (!read_raw(path, raw, err)) return false;
  const unsigned char *p = reinterpret_cast<const unsigned char *>(raw.data());
  if (raw.size() < (size_t)2 * ib || get_int(p, ib) != kVecClassId) {
    err = path + ": not a PETSc binary Vec";
    return false;
  }
  const int64_t n = get_int(p + ib, ib);
  if (n < 0 || raw.size() != (size_t)2 * ib + 8 * (size_t)n) {
    err = path + ": Vec length does not match the file size";
    return false;
  }
  out.resize(n);
  for (int64_t i = 0; i < n; ++i) out[i] = get_double(p + 2 * ib + 8 * i);
  return true;
}

// MatView of an AIJ matrix on a binary viewer (one process)
bool write_mat(const std::string &path, const Csr &A, int ib, std::string &err) {
  if (!check_ib(ib, err)) return false;
  const int64_t nnz = A.rowptr.empty() ? 0 : A.rowptr.back();
  if (!fits(A.M, ib, err) || !fits(A.N, ib, err) || !fits(nnz, ib, err)) return false;
  std::vector<unsigned char> b;
  b.reserve(4 * ib + (size_t)ib * (A.M + nnz) + 8 * (size_t)nnz);
  put_int(b, kMatClassId, ib);
  put_int(b, A.M, ib);
  put_int(b, A.N, ib);
  put_int(b, nnz, ib);
  for (int64_t r = 0; r < A.M; ++r) put_int(b, A.rowptr[r + 1] - A.rowptr[r], ib);
  for (int64_t t = 0; t < nnz; ++t) put_int(b, A.col[t], ib);
  for (int64_t t = 0; t < nnz; ++t) put_double(b, A.val[t]);
  return write_raw(path, b.data(), b.size(), err);
}

bool read_mat(const std::string &path, Csr &A, int ib, std::string &err) {
  if (!check_ib(ib, err)) return false;
  std::vector<char> raw;
  if (!read_raw(path, raw, err)) return false;
  const unsigned char *p = reinterpret_cast<const unsigned char *>(raw.data());
  if (raw.size() < (size_t)4 * ib || get_int(p, ib) != kMatClassId) {
    err = path + ": not a PETSc binary matrix";
    return false;
  }
  A.M = get_int(p + ib, ib);
  A.N = get_int(p + 2 * ib, ib);
  const int64_t nnz = get_int(p + 3 * ib, ib);
  if (A.M < 0 || A.N < 0 || nnz < 0 ||
      raw.size() != (size_t)4 * ib + (size_t)ib * (A.M + nnz) + 8 * (size_t)nnz) {
    err = path + ": matrix header does not match the file size";
    return false;
  }
  const unsigned char *q = p + 4 * ib;
  A.rowptr.assign(A.M + 1, 0);
  for (int64_t r = 0; r < A.M; ++r) A.rowptr[r + 1] = A.rowptr[r] + get_int(q + ib * r, ib);
  if (A.rowptr.back() != nnz) {
    err = path + ": row lengths do not add up to the nonzero count";
    return false;
  }
  q += (size_t)ib * A.M;
  A.col.resize(nnz);
  A.val.resize(nnz);
  for (int64_t t = 0; t < nnz; ++t) A.col[t] = get_int(q + ib * t, ib);
  q += (size_t)ib * nnz;
  for (int64_t t = 0; t < nnz; ++t) A.val[t] = get_double(q + 8 * t);
  return true;
}

Csr filter_matrix(const int nel[3], const double dx[3], double R, bool scale) {
  // the cone template of RecFilter: N = (short)(R/dx) cells per side,
  // weight 1 - d/R where d < R (strict), in (k, j, i) order, which is
  // ascending column order
  short N[3];
  for (int d = 0; d < 3; ++d) N[d] = (short)(R / dx[d]);
  struct Tap {
    int i, j, k;
    double w;
  };
  std::vector<Tap> taps;
  for (int k = -N[2]; k <= N[2]; ++k)
    for (int j = -N[1]; j <= N[1]; ++j)
      for (int i = -N[0]; i <= N[0]; ++i) {
        const double dist = std::sqrt(std::pow(i * dx[0], 2) + std::pow(j * dx[1], 2) +
                                      std::pow(k * dx[2], 2));
        if (dist < R) taps.push_back({i, j, k, 1 - dist / R});
      }
  Csr A;
  A.M = A.N = (int64_t)nel[0] * nel[1] * nel[2];
  A.rowptr.assign(A.M + 1, 0);
  A.col.reserve(A.M * taps.size());
  A.val.reserve(A.M * taps.size());
  for (int64_t e = 0; e < A.M; ++e) {
    const int ei = (int)(e % nel[0]), ej = (int)((e / nel[0]) % nel[1]),
              ek = (int)(e / ((int64_t)nel[0] * nel[1]));
    const size_t start = A.col.size();
    double rs = 0;
    for (const Tap &t : taps) {
      const int i = ei + t.i, j = ej + t.j, k = ek + t.k;
      if (i < 0 || i >= nel[0] || j < 0 || j >= nel[1] || k < 0 || k >= nel[2]) continue;
      A.col.push_back(i + (int64_t)j * nel[0] + (int64_t)k * nel[0] * nel[1]);
      A.val.push_back(t.w);
      rs += t.w;
    }
    if (scale) {
      // MatGetRowSum, VecPointwiseDivide(Ones, rowSum), MatDiagonalScale
      const double inv = 1.0 / rs;
      for (size_t t = start; t < A.col.size(); ++t) A.val[t] *= inv;
    }
    A.rowptr[e + 1] = (int64_t)A.col.size();
  }
  return A;
}

Csr prolongation_matrix(const int fine[3], const int coarse[3]) {
  // coarse node c sits on fine index 2c; the 1-D weight of c for fine f is
  // 1 (f = 2c) or 1/2 (|f - 2c| = 1), and 1 for the last fine index when
  // it has a single coarse neighbour, i.e. the row-normalised weights
  // (the normalisation factorises over the dimensions); a 3x3 identity
  // block per (fine, coarse) node pair, dof = 3 * node + component
  const int64_t nf = (int64_t)fine[0] * fine[1] * fine[2];
  Csr A;
  A.M = 3 * nf;
  A.N = 3 * (int64_t)coarse[0] * coarse[1] * coarse[2];
  A.rowptr.assign(A.M + 1, 0);
  for (int64_t n = 0; n < nf; ++n) {
    const int f[3] = {(int)(n % fine[0]), (int)((n / fine[0]) % fine[1]),
                      (int)(n / ((int64_t)fine[0] * fine[1]))};
    int cs[3][2], nc[3];
    double ws[3][2];
    for (int d = 0; d < 3; ++d) {
      if (f[d] % 2 == 0) {
        nc[d] = 1;
        cs[d][0] = f[d] / 2;
        ws[d][0] = 1.0;
      } else if (f[d] + 1 <= fine[d] - 1) {
        nc[d] = 2;
        cs[d][0] = (f[d] - 1) / 2;
        cs[d][1] = (f[d] + 1) / 2;
        ws[d][0] = ws[d][1] = 0.5;
      } else {
        nc[d] = 1;
        cs[d][0] = (f[d] - 1) / 2;
        ws[d][0] = 1.0;
      }
    }
    std::vector<std::pair<int64_t, double>> row;
    for (int c = 0; c < nc[2]; ++c)
      for (int b = 0; b < nc[1]; ++b)
        for (int a = 0; a < nc[0]; ++a)
          row.push_back({cs[0][a] + (int64_t)cs[1][b] * coarse[0] +
                             (int64_t)cs[2][c] * coarse[0] * coarse[1],
                         ws[0][a] * ws[1][b] * ws[2][c]});
    for (int comp = 0; comp < 3; ++comp) {
      for (const auto &cw : row) {
        A.col.push_back(3 * cw.first + comp);
        A.val.push_back(cw.second);
      }
      A.rowptr[3 * n + comp + 1] = (int64_t)A.col.size();
    }
  }
  return A;
}

void element_nodes(const int nel[3], int64_t e, int64_t nodes[8]) {
  const int64_t Nx = nel[0] + 1, Ny = nel[1] + 1;
  const int64_t i = e % nel[0], j = (e / nel[0]) % nel[1], k = e / ((int64_t)nel[0] * nel[1]);
  const int64_t n0 = i + j * Nx + k * Nx * Ny;
  nodes[0] = n0;
  nodes[1] = n0 + 1;
  nodes[2] = n0 + 1 + Nx;
  nodes[3] = n0 + Nx;
  for (int a = 0; a < 4; ++a) nodes[4 + a] = nodes[a] + Nx * Ny;
}

}  // namespace io
}  // namespace tpo
