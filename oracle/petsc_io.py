"""Test infrastructure: an independent numpy restatement of the files the
reference's MeshOut / PrintVals / LoadMesh read and write (TopOpt.cpp:97-508,
RecMesh.cpp:34-412), used only by tests to check the library's writers and
readers.

Two encodings:
  * raw native arrays (ofstream / MPI-IO): PetscInt (4 or 8 bytes), double,
    bool (1 byte), little-endian;
  * the PETSc binary viewer format, big-endian: a Vec is [1211214, n] as
    PetscInt then n doubles (VecView); an AIJ matrix is [1211216, M, N, nnz]
    then M row lengths, nnz column indices (PetscInt) and nnz values
    (MatView), columns ascending within a row.

Parity is unpinned against PETSc itself: neither PETSc nor petsc4py is in
this image and the reference ships no sample output files, so the layout is
restated from PETSc's published binary format (PetscBinaryWrite writes
big-endian; VecView_Seq_Binary and MatView_SeqAIJ_Binary write the headers
above).  The structured-mesh matrices are restated here from the reference's
RecFilter / Assemble_Filter (Filter.cpp:21-147) and its level layout
(Interpolation.cpp:200-347) through the C oracle's filter and prolongation
weights.
"""
from __future__ import annotations

import numpy as np

VEC_CLASSID = 1211214
MAT_CLASSID = 1211216


def _idt(ib, be=True):
    return np.dtype((">" if be else "<") + ("i4" if ib == 4 else "i8"))


def write_vec(path, v, ib=4):
    v = np.asarray(v, np.float64)
    with open(path, "wb") as f:
        f.write(np.array([VEC_CLASSID, v.size], _idt(ib)).tobytes())
        f.write(v.astype(">f8").tobytes())


def read_vec(path, ib=4):
    b = open(path, "rb").read()
    h = np.frombuffer(b[:2 * ib], _idt(ib))
    assert h[0] == VEC_CLASSID, "not a PETSc binary Vec"
    n = int(h[1])
    assert len(b) == 2 * ib + 8 * n, "Vec length does not match the file size"
    return np.frombuffer(b[2 * ib:], ">f8").astype(np.float64)


def write_mat(path, rowptr, col, val, shape, ib=4):
    rowptr = np.asarray(rowptr, np.int64)
    with open(path, "wb") as f:
        f.write(np.array([MAT_CLASSID, shape[0], shape[1], rowptr[-1]], _idt(ib)).tobytes())
        f.write(np.diff(rowptr).astype(_idt(ib)).tobytes())
        f.write(np.asarray(col).astype(_idt(ib)).tobytes())
        f.write(np.asarray(val, np.float64).astype(">f8").tobytes())


def read_mat(path, ib=4):
    """-> (rowptr, col, val, (M, N))"""
    b = open(path, "rb").read()
    h = np.frombuffer(b[:4 * ib], _idt(ib))
    assert h[0] == MAT_CLASSID, "not a PETSc binary matrix"
    M, N, nnz = (int(t) for t in h[1:])
    o = 4 * ib
    lens = np.frombuffer(b[o:o + ib * M], _idt(ib)).astype(np.int64)
    o += ib * M
    col = np.frombuffer(b[o:o + ib * nnz], _idt(ib)).astype(np.int64)
    o += ib * nnz
    val = np.frombuffer(b[o:o + 8 * nnz], ">f8").astype(np.float64)
    assert o + 8 * nnz == len(b), "matrix header does not match the file size"
    rowptr = np.concatenate([[0], np.cumsum(lens)])
    return rowptr, col, val, (M, N)


def read_ints(path, ib=4):
    return np.fromfile(path, _idt(ib, be=False)).astype(np.int64)


def read_doubles(path):
    return np.fromfile(path, "<f8")


def read_bools(path):
    return np.fromfile(path, np.uint8).astype(bool)


def max_filter(nel, dx, R):
    """RecFilter without the row scaling (Assemble_Filter with scale =
    false, RecMesh.cpp:706): weights 1 - d/R for d < R, in CSR, and
    REdge = max(rowsum) - rowsum (RecMesh.cpp:710-718)."""
    N = [int(R / d) for d in dx]
    taps = []
    for k in range(-N[2], N[2] + 1):
        for j in range(-N[1], N[1] + 1):
            for i in range(-N[0], N[0] + 1):
                dist = np.sqrt((i * dx[0]) ** 2 + (j * dx[1]) ** 2 + (k * dx[2]) ** 2)
                if dist < R:
                    taps.append((i, j, k, 1 - dist / R))
    rp, col, val = [0], [], []
    for e in range(int(np.prod(nel))):
        ei, ej, ek = e % nel[0], (e // nel[0]) % nel[1], e // (nel[0] * nel[1])
        for i, j, k, w in taps:
            a, b, c = ei + i, ej + j, ek + k
            if 0 <= a < nel[0] and 0 <= b < nel[1] and 0 <= c < nel[2]:
                col.append(a + b * nel[0] + c * nel[0] * nel[1])
                val.append(w)
        rp.append(len(col))
    rp, val = np.array(rp), np.array(val)
    rs = np.array([val[rp[r]:rp[r + 1]].sum() for r in range(len(rp) - 1)])
    return rp, np.array(col), val, rs.max() - rs


def prolongation_dense(pb, level, fine_dims, coarse_dims):
    """The dof-level interpolation PR[level] as a dense array from the C
    oracle's weights (3x3 identity blocks, dof = 3 * node + component)."""
    nf, nc = int(np.prod(fine_dims)), int(np.prod(coarse_dims))
    W = np.zeros((nf, nc))
    for f in range(nf):
        fx, fy, fz = f % fine_dims[0], (f // fine_dims[0]) % fine_dims[1], \
            f // (fine_dims[0] * fine_dims[1])
        for cz in {fz // 2, (fz + 1) // 2}:
            for cy in {fy // 2, (fy + 1) // 2}:
                for cx in {fx // 2, (fx + 1) // 2}:
                    if cx < coarse_dims[0] and cy < coarse_dims[1] and cz < coarse_dims[2]:
                        c = cx + cy * coarse_dims[0] + cz * coarse_dims[0] * coarse_dims[1]
                        W[f, c] = pb.prolong_weight(level, f, c)
    return np.kron(W, np.eye(3))
