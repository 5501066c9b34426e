"""The per-node ghost elimination of assemble_poisson_2d / assemble_poisson_3d
against PSuM's formulation (ghost_element_manager.hpp, Poisson_solver_2d.hpp:
246-300, Poisson_solver_3d.hpp:240-300): every mixed (node, direction) gets a
ghost unknown that replaces the node's neighbour across the boundary in the
node's row, and the ghost's own row is the boundary condition with the
central difference, a phi + b (ghost - opposite) dr / 2 = value.  Solving
that augmented system directly gives the same node values as the eliminated
system (CPU only)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

import psum_b200 as P
from psum_b200.field_solver import DIRECTIONS, _merge_fixed, _merge_mixed

OPPOSITE = {"N": "S", "S": "N", "E": "W", "W": "E", "Xpos": "Xneg", "Xneg": "Xpos", "Ypos": "Yneg",
            "Yneg": "Ypos", "Zpos": "Zneg", "Zneg": "Zpos"}


def neighbour(grid, node, direction):
    dims = [c + 1 for c in grid.cells]
    idx = list(np.unravel_index(node, dims))
    axis, side = DIRECTIONS[grid.dim][direction]
    idx[axis] = (idx[axis] + side) % dims[axis]
    return int(np.ravel_multi_index(idx, dims))


def augmented_solve(grid, assemble, fixed, mixed, rho):
    ridx, rval = _merge_fixed(fixed)
    (r, c, v), _ = assemble(ridx, [])
    n = grid.n_nodes
    A = sp.lil_matrix(sp.csr_matrix((v, (r.astype(np.int64), c.astype(np.int64))), shape=(n, n)))
    entries = _merge_mixed(list(mixed), ridx)
    m = len(entries)
    Aug = sp.lil_matrix((n + m, n + m))
    Aug[:n, :n] = A
    b = np.zeros(n + m)
    b[:n] = rho
    b[ridx.astype(np.int64)] = rval
    coefs = {k: mb.coefficient_pairs() for k, mb in enumerate(mixed)}
    values = {k: mb.values() for k, mb in enumerate(mixed)}
    for t, (nd, d, bi, k) in enumerate(entries):
        g = n + t
        across = neighbour(grid, nd, d)
        Aug[nd, g] = Aug[nd, across]      # the ghost takes the neighbour's place in the node's row
        Aug[nd, across] = 0.0
        axis = DIRECTIONS[grid.dim][d][0]
        dr = 1.0 / grid.delta[axis]
        a_val, b_grad = coefs[bi][0][k], coefs[bi][1][k]
        opp = neighbour(grid, nd, OPPOSITE[d])
        Aug[g, g] = b_grad * dr / 2
        Aug[g, opp] = -b_grad * dr / 2
        Aug[g, nd] = a_val
        b[g] = values[bi][k]
    return spl.spsolve(Aug.tocsc(), b)[:n]


def eliminated_solve(grid, assemble, fixed, mixed, rho):
    ridx, rval = _merge_fixed(fixed)
    (r, c, v), M = assemble(ridx, mixed)
    n = grid.n_nodes
    A = sp.csr_matrix((v, (r.astype(np.int64), c.astype(np.int64))), shape=(n, n)).tocsc()
    ps = P.Poisson_solver_2d() if grid.dim == 2 else P.Poisson_solver_3d()
    ps.mixed, ps.mixed_M = list(mixed), M
    idx, val = ps.addback()
    b = np.asarray(rho, np.float64).copy()
    b[idx.astype(np.int64)] += val
    b[ridx.astype(np.int64)] = rval
    return spl.spsolve(A, b)


@pytest.mark.parametrize("domain", ["Cartesian", "Cylindrical"])
def test_2d_elimination_equals_augmented_system(domain):
    g = P.simple_grid((0.0, 0.0), (1.0, 1.5), (12, 10))
    rng = np.random.default_rng(3)
    rho = rng.normal(size=g.n_nodes)
    mixed = [P.Neumann_line(g, "E", lambda x, y: 0.3 * y), P.Robin_Line(g, "N", (2.0, 0.5), 0.7),
             P.Neumann_line(g, "S", 0.1)]
    fixed = [P.Dirichlet_line(g, "W", 1.0)]
    eps = lambda x, y: 1.0 + 0.4 * x

    def assemble(ridx, mb):
        return P.assemble_poisson_2d(g, domain, ridx, mb, eps)

    aug = augmented_solve(g, assemble, fixed, mixed, rho)
    eli = eliminated_solve(g, assemble, fixed, mixed, rho)
    assert np.abs(aug - eli).max() <= 1e-10 * np.abs(aug).max()


def test_3d_elimination_equals_augmented_system():
    g = P.simple_grid((0.0, 0.0, 0.0), (1.0, 1.2, 0.8), (6, 5, 4))
    rng = np.random.default_rng(4)
    rho = rng.normal(size=g.n_nodes)
    mixed = [P.Neumann_plane(g, "Xpos", 0.2), P.Robin_plane(g, "Ypos", (1.0, 0.5), lambda x, y, z: x - z),
             P.Neumann_plane(g, "Zneg", 0.0), P.Robin_plane(g, "Zpos", lambda x, y, z: (0.5, 1.0 + y), 0.4)]
    fixed = [P.Dirichlet_plane(g, "Xneg", 0.0)]
    eps = lambda x, y, z: 1.0 + 0.3 * y * z

    def assemble(ridx, mb):
        return P.assemble_poisson_3d(g, ridx, mb, eps)

    aug = augmented_solve(g, assemble, fixed, mixed, rho)
    eli = eliminated_solve(g, assemble, fixed, mixed, rho)
    assert np.abs(aug - eli).max() <= 1e-10 * np.abs(aug).max()
