// The reference's output and restart files, host side (io.cpp).
//
// Two encodings occur (TopOpt.cpp:97-508, RecMesh.cpp:34-412):
//  * raw native arrays written with ofstream / MPI-IO: PetscInt (4 or 8
//    bytes, `ib`), double and bool (1 byte), little-endian on x86;
//  * the PETSc binary viewer format (VecView / MatView of an AIJ matrix),
//    big-endian: a Vec is [1211214, n] as PetscInt then n doubles; a
//    matrix is [1211216, M, N, nnz] then the M row lengths, the nnz column
//    indices (PetscInt) and the nnz values (double), columns ascending in
//    each row.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace tpo {
namespace io {

constexpr int32_t kVecClassId = 1211214;
constexpr int32_t kMatClassId = 1211216;

struct Csr {
  int64_t M = 0, N = 0;
  std::vector<int64_t> rowptr, col;   // rowptr has M + 1 entries
  std::vector<double> val;
};

bool write_raw(const std::string &path, const void *data, size_t bytes, std::string &err);
bool read_raw(const std::string &path, std::vector<char> &out, std::string &err);
bool write_ints(const std::string &path, const int64_t *v, size_t n, int ib, std::string &err);
bool read_ints(const std::string &path, std::vector<int64_t> &out, int ib, std::string &err);

bool write_vec(const std::string &path, const double *v, int64_t n, int ib, std::string &err);
bool read_vec(const std::string &path, std::vector<double> &out, int ib, std::string &err);
bool write_mat(const std::string &path, const Csr &A, int ib, std::string &err);
bool read_mat(const std::string &path, Csr &A, int ib, std::string &err);

// RecFilter (Filter.cpp:21-94) over the structured mesh, with the row
// scaling of Assemble_Filter (:136-147) when `scale`
Csr filter_matrix(const int nel[3], const double dx[3], double R, bool scale);
// the dof-level interpolation matrix PR[i] (Interpolation.cpp:200-347)
// from the fine level's node dims to the next coarser level's
Csr prolongation_matrix(const int fine[3], const int coarse[3]);
// the 8 nodes of element e in the reference's order (RecMesh.cpp:486-512)
void element_nodes(const int nel[3], int64_t e, int64_t nodes[8]);

}  // namespace io
}  // namespace tpo
