"""The benchmark problem definitions: structured meshes, boundary
conditions in the reference's Set_BC form and seeded synthetic densities.

A boundary condition is (kind, center, radius, limits, values) exactly as a
[BC] block of the reference input file (Inputs.cpp:785-871): the node set
is every node with sum_d ((x_d - c_d)/r_d)^2 <= 1 inside the limits.
Densities are drawn with numpy.random.default_rng(seed) in reference
element order (e = i + j*nx + k*nx*ny).
"""
from __future__ import annotations

import numpy as np

BIG = 1e10
TINY = 1e-10
OPEN = (-1e30, 1e30, -1e30, 1e30, -1e30, 1e30)


def cantilever_bcs(nel, dx=(1.0, 1.0, 1.0)):
    """x = 0 face clamped; total load -1 in z split evenly over the nodes of
    the (x = max, z = 0) edge.  Coordinates are physical: element edges dx."""
    nx, ny, nz = nel
    return [
        ("support", (0.0, 0.0, 0.0), (TINY, BIG, BIG), OPEN, (1.0, 1.0, 1.0)),
        ("load", (float(nx) * dx[0], 0.0, 0.0), (TINY, BIG, TINY), OPEN,
         (0.0, 0.0, -1.0 / (ny + 1))),
    ]


def column_bcs(nel):
    """z = 0 face clamped; z = max face loaded uniformly, total -1 in z."""
    nx, ny, nz = nel
    nface = (nx + 1) * (ny + 1)
    return [
        ("support", (0.0, 0.0, 0.0), (BIG, BIG, TINY), OPEN, (1.0, 1.0, 1.0)),
        ("load", (0.0, 0.0, float(nz)), (BIG, BIG, TINY), OPEN,
         (0.0, 0.0, -1.0 / nface)),
    ]


CONFIGS = {
    # name: nel, density law, seed, rmin, GMG levels, boundary conditions
    "cfg0": dict(nel=(48, 24, 24), x=("const", 0.3), seed=0, rmin=1.5,
                 levels=3, bcs="cantilever"),
    "cfg1": dict(nel=(192, 96, 96), x=("uniform", 0.0, 1.0), seed=1, rmin=1.5,
                 levels=5, bcs="cantilever"),
    "cfg2": dict(nel=(128, 64, 64), x=("uniform", 0.05, 1.0), seed=2, rmin=1.5,
                 levels=5, bcs="multiload"),
    "cfg3": dict(nel=(64, 32, 32), x=("uniform", 0.1, 0.9), seed=3, rmin=2.0,
                 levels=4, bcs="cantilever"),
    "cfg4": dict(nel=(96, 48, 48), x=("uniform", 0.2, 1.0), seed=4, rmin=1.5,
                 levels=4, bcs="column"),
}


def design(cfg, nel=None):
    c = CONFIGS[cfg] if isinstance(cfg, str) else cfg
    nel = nel or c["nel"]
    ne = int(np.prod(nel))
    law = c["x"]
    if law[0] == "const":
        return np.full(ne, float(law[1]))
    rng = np.random.default_rng(c["seed"])
    return rng.uniform(law[1], law[2], ne)


def bcs(cfg, nel=None):
    c = CONFIGS[cfg] if isinstance(cfg, str) else cfg
    nel = nel or c["nel"]
    kind = c["bcs"]
    if kind == "column":
        return column_bcs(nel)
    # the multi-load problem shares the cantilever support
    b = cantilever_bcs(nel)
    return b if kind == "cantilever" else b[:1]


def point_loads(nel, nrhs, seed):
    """nrhs unit point loads on seeded random nodes of the x = max face with
    seeded random unit directions (normalised Gaussian 3-vectors); returns
    the column-major load matrix (3*nNode, nrhs)."""
    nx, ny, nz = nel
    Nx, Ny = nx + 1, ny + 1
    nn = Nx * Ny * (nz + 1)
    rng = np.random.default_rng(seed)
    F = np.zeros((nrhs, 3 * nn))
    for j in range(nrhs):
        jy, kz = rng.integers(0, ny + 1), rng.integers(0, nz + 1)
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        n = nx + jy * Nx + kz * Nx * Ny
        F[j, 3 * n:3 * n + 3] = d
    return F


def apply_bcs(target, spec):
    """Apply a BC list to a product TopOpt (Set_BC) or an oracle Problem
    (add_bc)."""
    for kind, center, radius, limits, values in spec:
        if hasattr(target, "Set_BC"):
            t = target.SUPPORT if kind == "support" else target.LOAD
            target.Set_BC(center, radius, limits, values, t)
        else:
            target.add_bc(kind, center, radius, limits, values)
