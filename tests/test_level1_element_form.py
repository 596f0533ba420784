"""The identity the tensor-core level-1 operator rests on, checked on the
oracle alone (no GPU): with even element counts, the Galerkin level-1
operator of the clamped fine operator (FEAnalysis.cpp:410-416) equals
P^T (sum_e E_e K0) P -- the element sum without boundary conditions, which
the kernel forms as sum_E sum_i E_{E,i} G_i u_E -- in every row except those
of the level-1 nodes next to a coarse element that holds a fixed fine dof.
Those rows are the ones the library stores correction rows for."""
import numpy as np

from topopt3d_b200 import problems as P


def trilinear(nel):
    """P (3 nf x 3 nc): coarse node C sits on fine index 2C; weight 1 on it
    and 1/2 one fine node away in each direction (even element counts)."""
    fx, fy, fz = (n + 1 for n in nel)
    cx, cy, cz = (n // 2 + 1 for n in nel)
    Pm = np.zeros((3 * fx * fy * fz, 3 * cx * cy * cz))
    w1 = lambda f, c: 1.0 if f == 2 * c else (0.5 if abs(f - 2 * c) == 1 else 0.0)
    for gz in range(fz):
        for gy in range(fy):
            for gx in range(fx):
                f = (gz * fy + gy) * fx + gx
                for kz in range(cz):
                    for ky in range(cy):
                        for kx in range(cx):
                            w = w1(gx, kx) * w1(gy, ky) * w1(gz, kz)
                            if w:
                                c = (kz * cy + ky) * cx + kx
                                for d in range(3):
                                    Pm[3 * f + d, 3 * c + d] = w
    return Pm, (cx, cy, cz)


def test_level1_is_the_element_sum_away_from_fixed_dofs(oracle):
    nel = (6, 4, 4)
    ref = oracle.Problem(nel, rmin=1.5, mg_levels=3)
    P.apply_bcs(ref, P.cantilever_bcs(nel))
    ne = int(np.prod(nel))
    ref.set_design(np.random.default_rng(3).uniform(0.05, 1.0, ne), 3.0, 1e-10)
    ref.assemble(oracle.default_opts())
    _, E, _ = ref.material()
    K0 = oracle.element_stiffness()
    nf = int(np.prod([n + 1 for n in nel]))
    K = np.zeros((3 * nf, 3 * nf))
    for e in range(ne):
        nodes = oracle.element_nodes(nel, e)
        dofs = np.ravel([[3 * n, 3 * n + 1, 3 * n + 2] for n in nodes])
        K[np.ix_(dofs, dofs)] += E[e] * K0
    Pm, (cx, cy, cz) = trilinear(nel)
    A_elem = Pm.T @ K @ Pm
    nc, dims = ref.level_nodes(1)
    assert dims == (cx, cy, cz) and nc == cx * cy * cz
    A1 = np.zeros((3 * nc, 3 * nc))
    for i in range(nc):
        for j in range(nc):
            A1[3 * i:3 * i + 3, 3 * j:3 * j + 3] = ref.level_block(1, i, j)
    D = A1 - A_elem
    scale = np.abs(A1).max()
    # the clamped face is x = 0: coarse elements with EI = 0 follow the
    # general path, so the nodes X = 0 and X = 1 carry the difference
    for n in range(nc):
        X = n % cx
        row = np.abs(D[3 * n:3 * n + 3]).max() / scale
        if X >= 2:
            assert row < 1e-13, (n, row)
    assert max(np.abs(D[3 * n:3 * n + 3]).max() for n in range(nc) if n % cx == 0) > 1e-6 * scale
