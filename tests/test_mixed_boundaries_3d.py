"""3-D Poisson frontend with mixed (Neumann / Robin) boundary planes and a
position-dependent epsilon (Poisson_solver_3d.hpp:178-349, Neumann.hpp:96-133,
Robin.hpp:116-163): the assembled operator against the compiled assembly and
against manufactured solutions, solved directly on the host."""
import math

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

import psum_b200 as P
from psum_b200.field_solver import _merge_fixed


def direct_solve(grid, fixed, mixed, rho, eps=1.0):
    """b = rho + M * boundary values, fixed values replaced, then A' phi = b."""
    ps = P.Poisson_solver_3d()
    ridx, rval = _merge_fixed(fixed)
    (r, c, v), M = P.assemble_poisson_3d(grid, ridx, mixed, eps)
    n = grid.n_nodes
    A = sp.csr_matrix((v, (r.astype(np.int64), c.astype(np.int64))), shape=(n, n)).tocsc()
    ps.mixed, ps.mixed_M = mixed, M
    idx, val = ps.addback()
    b = np.asarray(rho, np.float64).copy()
    b[idx.astype(np.int64)] += val
    b[ridx.astype(np.int64)] = rval
    return spl.spsolve(A, b)


def node_xyz(g):
    axes = [g.lower[a] + np.arange(g.cells[a] + 1) * g.delta[a] for a in range(3)]
    return [c.reshape(-1) for c in np.meshgrid(*axes, indexing="ij")]


def test_plain_operator_matches_compiled_assembly():
    # no mixed boundary, uniform epsilon: the general assembly gives the
    # compiled assembly's operator bit for bit
    g = P.simple_grid((0.0, -1.0, 0.5), (2.0, 1.5, 1.7), (7, 6, 5))
    fixed = np.unique(np.concatenate([P.Dirichlet_plane(g, d, 0)[0] for d in ("Xneg", "Ypos", "Zneg")]))
    r1, c1, v1 = P.assemble_poisson(g, fixed, 2.5)
    (r2, c2, v2), M = P.assemble_poisson_3d(g, fixed, [], 2.5)
    n = g.n_nodes
    A1 = sp.csr_matrix((v1, (r1.astype(np.int64), c1.astype(np.int64))), shape=(n, n))
    A2 = sp.csr_matrix((v2, (r2.astype(np.int64), c2.astype(np.int64))), shape=(n, n))
    assert (A1 != A2).nnz == 0
    assert len(M[0]) == 0


def exact(x, y, z):
    return np.cos(x) * (1 + 0.3 * y * y) * (1 + 0.2 * z)


def grad(x, y, z):
    return (-np.sin(x) * (1 + 0.3 * y * y) * (1 + 0.2 * z),
            np.cos(x) * 0.6 * y * (1 + 0.2 * z),
            np.cos(x) * (1 + 0.3 * y * y) * 0.2)


def laplacian(x, y, z):
    return (-np.cos(x) * (1 + 0.3 * y * y) * (1 + 0.2 * z) + np.cos(x) * 0.6 * (1 + 0.2 * z))


def test_neumann_and_robin_planes_second_order():
    # Dirichlet on x = 0, Neumann on x = 1 and both y planes, Robin
    # a phi + b dphi/dn = g on z = 1, Neumann on z = 0: edges and corners
    # carry one ghost per direction; the error falls as h^2
    a, b = 1.5, 0.75
    errs = []
    for N in (6, 12, 24):
        g = P.simple_grid((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (N, N, N))
        x, y, z = node_xyz(g)
        mixed = [P.Neumann_plane(g, "Xpos", lambda x, y, z: grad(x, y, z)[0]),
                 P.Neumann_plane(g, "Yneg", lambda x, y, z: -grad(x, y, z)[1]),
                 P.Neumann_plane(g, "Ypos", lambda x, y, z: grad(x, y, z)[1]),
                 P.Neumann_plane(g, "Zneg", lambda x, y, z: -grad(x, y, z)[2]),
                 P.Robin_plane(g, "Zpos", (a, b), lambda x, y, z: a * exact(x, y, z) + b * grad(x, y, z)[2])]
        fx = P.Dirichlet_plane(g, "Xneg", 0.0)[0]
        fixed = [(fx, exact(x[fx.astype(np.int64)], y[fx.astype(np.int64)], z[fx.astype(np.int64)]))]
        phi = direct_solve(g, fixed, mixed, -laplacian(x, y, z))
        errs.append(np.abs(phi - exact(x, y, z)).max())
    order = math.log(errs[0] / errs[-1]) / math.log(4)
    assert 1.7 < order < 2.3, (errs, order)
    assert errs[-1] < 2e-4


def test_epsilon_function_second_order():
    # -div(eps grad phi) = rho with eps(x, y, z) = 1 + 0.5 x + 0.25 y z taken
    # at the face midpoints; Dirichlet on the x planes, Neumann elsewhere
    def eps(x, y, z):
        return 1 + 0.5 * x + 0.25 * y * z

    def rho(x, y, z):
        gx, gy, gz = grad(x, y, z)
        return -(eps(x, y, z) * laplacian(x, y, z) + 0.5 * gx + 0.25 * z * gy + 0.25 * y * gz)

    errs = []
    for N in (6, 12, 24):
        g = P.simple_grid((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (N, N, N))
        x, y, z = node_xyz(g)
        mixed = [P.Neumann_plane(g, "Yneg", lambda x, y, z: -grad(x, y, z)[1]),
                 P.Neumann_plane(g, "Ypos", lambda x, y, z: grad(x, y, z)[1]),
                 P.Neumann_plane(g, "Zneg", lambda x, y, z: -grad(x, y, z)[2]),
                 P.Neumann_plane(g, "Zpos", lambda x, y, z: grad(x, y, z)[2])]
        fixed = []
        for d in ("Xneg", "Xpos"):
            fx = P.Dirichlet_plane(g, d, 0.0)[0].astype(np.int64)
            fixed.append((fx.astype(np.uint64), exact(x[fx], y[fx], z[fx])))
        phi = direct_solve(g, fixed, mixed, rho(x, y, z), eps=eps)
        errs.append(np.abs(phi - exact(x, y, z)).max())
    order = math.log(errs[0] / errs[-1]) / math.log(4)
    assert 1.7 < order < 2.3, (errs, order)


def test_plane_creators_merge_rules_and_errors():
    g = P.simple_grid((0.0, 0.0, 0.0), (1.0, 2.0, 3.0), (4, 5, 6))
    # plane nodes and the min_max filter (x for Y / Z planes, y for X planes)
    zp = P.Neumann_plane(g, "Zpos")
    assert len(zp.nodes) == 5 * 6 and all(n % 7 == 6 for n in zp.nodes)
    xn = P.Neumann_plane(g, "Xneg", min_max=(0.5, 1.25))
    _, yy, _ = node_xyz(g)
    assert sorted(set(np.round(yy[xn.nodes], 12))) == [0.8, 1.2]
    yq = P.Robin_plane(g, "Ypos", (1.0, 2.0), 0.0, min_max=(0.25, 0.5))
    xx, _, _ = node_xyz(g)
    assert sorted(set(np.round(xx[yq.nodes], 12))) == [0.25, 0.5]
    with pytest.raises(ValueError):
        P.Neumann_plane(g, "N")
    with pytest.raises(ValueError):
        P.Neumann_line(g, "N")
    # a later boundary on the same (node, direction) covers an earlier one;
    # fixed nodes cover mixed ones; an edge node keeps one condition per direction
    fixed = P.Dirichlet_plane(g, "Xneg", 0.0)[0]
    mixed = [P.Neumann_plane(g, "Zpos", 1.0), P.Neumann_plane(g, "Zpos", 2.0), P.Neumann_plane(g, "Ypos", 3.0),
             P.Neumann_plane(g, "Xneg", 4.0)]
    _, (rows, mvals, entries) = P.assemble_poisson_3d(g, fixed, mixed, 1.0)
    fx = set(fixed.tolist())
    assert all(b != 0 for (_, _, b, _) in entries)          # the later Zpos wins
    assert not any(nd in fx for (nd, _, _, _) in entries)    # Xneg nodes are fixed
    edge = g.n2i(2, 5, 6)
    assert sorted(dn for (nd, dn, _, _) in entries if nd == edge) == ["Ypos", "Zpos"]
    ps = P.Poisson_solver_3d()
    ps.mixed, ps.mixed_M = mixed, (rows, mvals, entries)
    idx, val = ps.addback()
    # Neumann value v on a plane: M = -2 c / (b dr) with b = 1 ->  -2 c v / dr per ghost
    assert idx.size == len(set(rows.tolist()))
    # mixed conditions on opposite sides of one node (their ghosts would be coupled)
    node = g.n2i(2, 2, 2)
    with pytest.raises(ValueError):
        P.assemble_poisson_3d(g, [], [P.MixedBoundary(g, [node], "Xneg", (0.0, 1.0), 0.0),
                                      P.MixedBoundary(g, [node], "Xpos", (0.0, 1.0), 0.0)], 1.0)
    with pytest.raises(ValueError):
        P.assemble_poisson_3d(g, [], [P.MixedBoundary(g, [0], "Zneg", (1.0, 0.0), 0.0)], 1.0)
    # the cylindrical domain is 2-D only
    with pytest.raises(ValueError):
        P.Poisson_solver_3d().init("cuda_multigrid64_gpu", g, "Cylindrical", [])
