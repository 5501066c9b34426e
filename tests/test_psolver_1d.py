"""PSuM's 1-D Poisson frontend (Poisson_solver_1d.hpp) and its tests
(test/field_solver/test_psolver_1d.cpp) restated on the host: the operator
of assemble_poisson_1d solved directly, with the right-hand side PSuM's
make_righthand_item builds (source plus mixed values, fixed values
replaced), and the multigrid algorithm of the backends (the oracle's
FP32-in-FP64 restatement) on the same operator."""
import math

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

import psum_b200 as P
from oracle import oracle as O
from psum_b200.field_solver import _merge_fixed

EPS0 = 8.854e-12


def system(g, fixed, mixed, rho, eps=EPS0):
    ps = P.Poisson_solver_1d()
    ridx, rval = _merge_fixed(fixed)
    (r, c, v), M = P.assemble_poisson_1d(g, ridx, mixed, eps)
    n = g.n_nodes
    A = sp.csr_matrix((v, (r.astype(np.int64), c.astype(np.int64))), shape=(n, n))
    ps.mixed, ps.mixed_M = list(mixed), M
    idx, val = ps.addback()
    b = np.asarray(rho, np.float64).copy()
    b[idx.astype(np.int64)] += val
    b[ridx.astype(np.int64)] = rval
    return A, b, (r, c, v)


def solve(g, fixed, mixed, rho, eps=EPS0):
    A, b, _ = system(g, fixed, mixed, rho, eps)
    return spl.spsolve(A.tocsc(), b)


def xs(g):
    return g.lower[0] + np.arange(g.cells[0] + 1) * g.delta[0]


def test_manufactured_solution():
    # test_psolver_1d.cpp:16-73: phi = sin(pi x), grounded ends; order 2
    errs = []
    for k in range(1, 7):
        g = P.simple_grid((0.0,), (1.0,), (40 * k,))
        x = xs(g)
        phi = solve(g, [P.Dirichlet_point(g, "L", 0.0), P.Dirichlet_point(g, "R", 0.0)], [],
                    -EPS0 * (-np.pi ** 2 * np.sin(np.pi * x)))
        errs.append(np.sqrt(np.mean((phi - np.sin(np.pi * x)) ** 2)))
    order = math.log(errs[0] / errs[-1]) / math.log(6)
    assert 1.95 < order < 2.05, (errs, order)


def test_simple_case():
    # :75-116: phi(0) = 0, phi(1) = 1, no charge -> phi = x to 1e-10
    g = P.simple_grid((0.0,), (1.0,), (100,))
    phi = solve(g, [P.Dirichlet_point(g, "L", 0.0), P.Dirichlet_point(g, "R", 1.0)], [], np.zeros(101))
    assert np.abs(phi - xs(g)).max() < 1e-10


def test_neumann_boundary():
    # :118-164: phi = x^2, phi'(0) = 0, phi(1) = 1, rho = -2 eps0 everywhere
    # (the mixed row's right-hand side is rho + value, as in PSuM) -> 1e-8
    g = P.simple_grid((0.0,), (1.0,), (100,))
    phi = solve(g, [P.Dirichlet_point(g, "R", 1.0)], [P.Neumann_point(g, "L", 0.0)], np.full(101, -2 * EPS0))
    assert np.abs(phi - xs(g) ** 2).max() < 1e-8


@pytest.mark.parametrize("coef_R,value_R", [((1.0, 1.0), 3.0), (lambda x: (1.0, 2.0), 5.0)])
def test_robin_boundary(coef_R, value_R):
    # :166-265: phi = x^2 with Robin ends a phi + b dphi/dn = value, fixed
    # (A) and function (B) coefficients -> 1e-8
    g = P.simple_grid((0.0,), (1.0,), (100,))
    mixed = [P.Robin_point(g, "L", (1.0, 1.0), 0.0), P.Robin_point(g, "R", coef_R, value_R)]
    phi = solve(g, [], mixed, np.full(101, -2 * EPS0))
    assert np.abs(phi - xs(g) ** 2).max() < 1e-8


def test_variable_epsilon():
    # :267-326: eps = eps0 (1 + x), phi = x^2, rho = -eps0 (2 + 4x) -> 1e-8
    g = P.simple_grid((0.0,), (1.0,), (100,))
    x = xs(g)
    phi = solve(g, [P.Dirichlet_point(g, "L", 0.0), P.Dirichlet_point(g, "R", 1.0)], [],
                -EPS0 * (2.0 + 4.0 * x), eps=lambda v: EPS0 * (1.0 + v))
    assert np.abs(phi - x * x).max() < 1e-8


def test_multigrid_algorithm_on_the_1d_operator():
    # the backends' FP32-in-FP64 V-cycles (I = cells + 1, J = K = 1) reach the
    # direct solution of the grounded manufactured problem
    g = P.simple_grid((0.0,), (1.0,), (256,))
    x = xs(g)
    rho = -EPS0 * (-np.pi ** 2 * np.sin(np.pi * x))
    fixed = [P.Dirichlet_point(g, "L", 0.0), P.Dirichlet_point(g, "R", 0.0)]
    A, b, (r, c, v) = system(g, fixed, [], rho)
    direct = spl.spsolve(A.tocsc(), b)
    mg = O.Multigrid(r, c, v, g.n_nodes, g.n_nodes, 1, 1, 4)
    phi, hist = mg.solve_mixed(b, np.zeros(g.n_nodes), max_cycles=200, correction_interval=4, pre=2, post=2)
    assert hist[-1] < 1e-9, hist[-5:]
    assert np.abs(phi - direct).max() < 1e-7 * np.abs(direct).max()


def test_creators_and_errors():
    g = P.simple_grid((-1.0,), (3.0,), (8,))
    assert P.Dirichlet_point(g, "R", 2.0)[0].tolist() == [8]
    idx, val = P.Dirichlet_range(g, 0.0, 1.0, 4.0)
    assert idx.tolist() == [2, 3, 4] and (val == 4.0).all()
    with pytest.raises(ValueError):
        P.Neumann_point(g, "N")
    with pytest.raises(ValueError):
        P.Dirichlet_point(P.simple_grid((0.0, 0.0), (1.0, 1.0), (2, 2)), "L", 0.0)
    # a fixed node covers a mixed condition on it
    _, (rows, _, entries) = P.assemble_poisson_1d(g, [0], [P.Neumann_point(g, "L", 1.0)], 1.0)
    assert len(entries) == 0 and len(rows) == 0


def test_frontends_host_path_gives_the_same_system():
    # assemble + coeff_matrix + make_righthand_item(rho) (the (rho, b)
    # overload of PSuM's frontends) reproduce the systems built by hand
    import scipy.sparse as sp
    g1 = P.simple_grid((0.0,), (1.0,), (50,))
    rho1 = np.linspace(-1.0, 1.0, 51)
    fixed1, mixed1 = [P.Dirichlet_point(g1, "R", 1.0)], [P.Robin_point(g1, "L", (1.0, 2.0), 0.5)]
    ps1 = P.Poisson_solver_1d()
    ps1.assemble(g1, fixed1, 2.0, mixed1)
    A_ref, b_ref, _ = system(g1, fixed1, mixed1, rho1, 2.0)
    r, c, v = ps1.coeff_matrix()
    A = sp.csr_matrix((v, (r.astype(np.int64), c.astype(np.int64))), shape=A_ref.shape)
    assert abs(A - A_ref).max() == 0.0
    assert (ps1.make_righthand_item(rho1) == b_ref).all()

    g3 = P.simple_grid((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (5, 4, 3))
    rho3 = np.random.default_rng(8).normal(size=g3.n_nodes)
    fixed3 = [P.Dirichlet_plane(g3, "Zneg", 0.5)]
    mixed3 = [P.Neumann_plane(g3, "Zpos", 0.25), P.Robin_plane(g3, "Xneg", (1.0, 1.0), 0.1)]
    ps3 = P.Poisson_solver_3d()
    ps3.assemble(g3, "Cartesian", fixed3, 1.5, mixed3)
    ridx, rval = P.field_solver._merge_fixed(fixed3)
    (r3, c3, v3), M = P.assemble_poisson_3d(g3, ridx, mixed3, 1.5)
    assert all((x == y).all() for x, y in zip(ps3.coeff_matrix(), (r3, c3, v3)))
    ps_ref = P.Poisson_solver_3d()
    ps_ref.mixed, ps_ref.mixed_M = mixed3, M
    idx, val = ps_ref.addback()
    b = rho3.copy()
    b[idx.astype(np.int64)] += val
    b[ridx.astype(np.int64)] = rval
    assert (ps3.make_righthand_item(rho3) == b).all()
    # the plain Cartesian case goes through the compiled assembly
    ps2 = P.Poisson_solver_2d()
    g2 = P.simple_grid((0.0, 0.0), (1.0, 1.0), (6, 6))
    ps2.assemble(g2, "Cartesian", [P.Dirichlet_line(g2, "N", 0.0)], 3.0)
    r2, c2, v2 = P.assemble_poisson(g2, P.Dirichlet_line(g2, "N", 0.0)[0], 3.0)
    assert all((x == y).all() for x, y in zip(ps2.coeff_matrix(), (r2, c2, v2)))
    with pytest.raises(ValueError):
        ps3.assemble(g3, "Cylindrical", fixed3)
