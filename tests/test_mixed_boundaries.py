"""2-D Poisson frontend with mixed (Neumann / Robin) boundaries, the
cylindrical domain and position-dependent epsilon: the assembled operator
against PSuM's own known answers (test/field_solver/test_psolver_2d.cpp),
solved directly on the host."""
import math

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

import psum_b200 as P
from psum_b200.field_solver import _merge_fixed


def direct_solve(grid, domain, fixed, mixed, rho, eps=8.854e-12):
    """PSuM's solve on the host: b = rho + M * boundary values, fixed values
    replaced, then A' phi = b."""
    ps = P.Poisson_solver_2d()
    ridx, rval = _merge_fixed(fixed)
    (r, c, v), M = P.assemble_poisson_2d(grid, domain, ridx, mixed, eps)
    n = grid.n_nodes
    A = sp.csr_matrix((v, (r.astype(np.int64), c.astype(np.int64))), shape=(n, n)).tocsc()
    ps.mixed, ps.mixed_M = mixed, M
    idx, val = ps.addback()
    b = np.asarray(rho, np.float64).copy()
    b[idx.astype(np.int64)] += val
    b[ridx.astype(np.int64)] = rval
    return spl.spsolve(A, b)


def node_xy(g):
    i = np.arange(g.cells[0] + 1)
    j = np.arange(g.cells[1] + 1)
    x, y = np.meshgrid(g.lower[0] + i * g.delta[0], g.lower[1] + j * g.delta[1], indexing="ij")
    return x.reshape(-1), y.reshape(-1)


def test_plain_operator_matches_compiled_assembly():
    # no mixed boundary, Cartesian, uniform epsilon: the general assembly
    # gives the compiled assembly's operator bit for bit
    g = P.simple_grid((0.0, -1.0), (2.0, 1.5), (12, 9))
    fixed = np.unique(np.concatenate([P.Dirichlet_line(g, d, 0)[0] for d in "NSW"]))
    r1, c1, v1 = P.assemble_poisson(g, fixed, 2.5)
    (r2, c2, v2), _ = P.assemble_poisson_2d(g, "Cartesian", fixed, [], 2.5)
    n = g.n_nodes
    A1 = sp.csr_matrix((v1, (r1.astype(np.int64), c1.astype(np.int64))), shape=(n, n))
    A2 = sp.csr_matrix((v2, (r2.astype(np.int64), c2.astype(np.int64))), shape=(n, n))
    assert (A1 != A2).nnz == 0


def test_cylindrical_known_answer_second_order():
    # test_psolver_2d.cpp:16-66 (test_c_rate_simple): z-r domain, Neumann on
    # E, W and the axis, grounded at r = R, charge c1 r^c2; phi on the axis
    # at z = 1 against maxR^(c2+2) c1 / (eps0 (c2+2)^2), order ~2
    c1, c2, R = 0.01, 0.5, 1.67
    theory = R ** (c2 + 2) * c1 / (8.854e-12 * (c2 + 2) ** 2)
    errs = []
    for k in (1, 2, 4):
        g = P.simple_grid((0.0, 0.0), (1.0, R), (60 * k, 40 * k))
        _, r = node_xy(g)
        mixed = [P.Neumann_line(g, "E", 0.0), P.Neumann_line(g, "W", 0.0), P.Neumann_line(g, "S", 0.0)]
        phi = direct_solve(g, "Cylindrical", [P.Dirichlet_line(g, "N", 0.0)], mixed, c1 * np.power(r, c2))
        errs.append(abs(phi[g.n2i(g.cells[0], 0)] - theory) / theory)
    order = math.log(errs[0] / errs[-1]) / math.log(4)
    assert 1.7 < order < 2.3, (errs, order)
    assert errs[-1] < 1e-4


def test_robin_manufactured_second_order():
    # phi = cos x on [0,1]^2: Dirichlet phi = 1 at x = 0, Robin
    # a phi + b dphi/dn = a cos 1 - b sin 1 at x = 1, zero flux on y = 0, 1
    a, b = 2.0, 0.5
    errs = []
    for N in (16, 32, 64):
        g = P.simple_grid((0.0, 0.0), (1.0, 1.0), (N, N))
        x, _ = node_xy(g)
        mixed = [P.Neumann_line(g, "N", 0.0), P.Neumann_line(g, "S", 0.0),
                 P.Robin_Line(g, "E", (a, b), a * math.cos(1) - b * math.sin(1))]
        phi = direct_solve(g, "Cartesian", [P.Dirichlet_line(g, "W", 1.0)], mixed, np.cos(x), eps=1.0)
        errs.append(np.abs(phi - np.cos(x)).max())
    order = math.log(errs[0] / errs[-1]) / math.log(4)
    assert 1.9 < order < 2.1, (errs, order)


def test_epsilon_function_and_value_function():
    # layered epsilon(y) and a position-dependent Neumann flux: phi = y^2 / 2
    # with eps = 1 + y solves -(eps phi')' = -(1 + 2y) = rho, flux phi'(1) = 1
    N = 64
    g = P.simple_grid((0.0, 0.0), (1.0, 1.0), (8, N))
    _, y = node_xy(g)
    mixed = [P.Neumann_line(g, "N", lambda x_, y_: 1.0), P.Neumann_line(g, "E", 0.0), P.Neumann_line(g, "W", 0.0)]
    phi = direct_solve(g, "Cartesian", [P.Dirichlet_line(g, "S", 0.0)], mixed, -(1 + 2 * y),
                       eps=lambda x_, y_: 1.0 + y_)
    assert np.abs(phi - y * y / 2).max() < 2e-4


def test_sphere_in_cylindrical_coordinates():
    # test_psolver_2d.cpp:124-150 (test_fixedZone_func): a grounded sphere
    # of radius 0.5 with uniform charge; centre potential 0.25 q / (6 eps0)
    g = P.simple_grid((0.0, 0.0), (2.0, 2.0), (100, 200))
    fixed = [P.Dirichlet_func(g, lambda z, r: ((z - 1) ** 2 + r * r) > 0.25, 0.0)]
    phi = direct_solve(g, "Cylindrical", fixed, [], np.full(g.n_nodes, 0.01))
    theory = 0.25 * 0.01 / (6 * 8.854e-12)
    assert abs(phi[g.n2i(50, 0)] - theory) / theory < 0.03


def test_overlap_rules_and_creators():
    g = P.simple_grid((0.0, 0.0), (4.0, 3.0), (4, 3))
    # a later boundary covers the nodes it shares with an earlier one; fixed covers mixed
    early = P.Neumann_line(g, "E", 1.0)
    late = P.Robin_Line(g, "E", (1.0, 2.0), 5.0, min_max=(1.0, 2.0))
    corner = g.n2i(4, 0)
    (_, _, _), (rows, mvals, entries) = P.assemble_poisson_2d(
        g, "Cartesian", np.array([corner]), [early, late], 1.0)
    by_node = {e[0]: e[2] for e in entries}
    assert corner not in by_node
    assert by_node[g.n2i(4, 1)] == 1 and by_node[g.n2i(4, 2)] == 1 and by_node[g.n2i(4, 3)] == 0
    # keyed by (node, direction): a corner keeps one condition per side
    (_, _, _), (_, _, entries) = P.assemble_poisson_2d(
        g, "Cartesian", [], [P.Neumann_line(g, "N", 0.0), P.Neumann_line(g, "E", 0.0)], 1.0)
    assert sorted(e[1] for e in entries if e[0] == g.n2i(4, 3)) == ["E", "N"]
    # creators: box with tolerance, predicate, line with min_max
    idx, val = P.Dirichlet_box(g, 1.0, 1.0, 2.0, 2.0, 3.0)
    assert sorted(idx.tolist()) == sorted(g.n2i(i, j) for i in (1, 2) for j in (1, 2)) and (val == 3.0).all()
    idx, _ = P.Dirichlet_func(g, lambda x, y: x + y < 1.5, 0.0)
    assert sorted(idx.tolist()) == sorted([g.n2i(0, 0), g.n2i(0, 1), g.n2i(1, 0)])
    assert late.nodes.tolist() == [g.n2i(4, 1), g.n2i(4, 2)]
    with pytest.raises(ValueError):
        P.assemble_poisson_2d(g, "Cartesian", [], [P.Robin_Line(g, "W", (1.0, 0.0), 0.0)], 1.0)


def collisionless_flow_field(N=48):
    """The field set-up of PSuM's collision-less-flow application
    (application/collision-less-flow/field_ops.hpp:92-124): (z, r) domain,
    Robin lines on E and N with coefficients (1, (z^2 + r^2) / z) and
    (1, (z^2 + r^2) / r), zero flux on the axis, grounded W for r <= r_length."""
    g = P.simple_grid((0.0, 0.0), (2.0, 1.0), (2 * N, N))
    mixed = [P.Robin_Line(g, "E", lambda z, r: (1.0, (z * z + r * r) / z), lambda z, r: 0.5 * r),
             P.Robin_Line(g, "N", lambda z, r: (1.0, (z * z + r * r) / r), lambda z, r: 0.2 * z),
             P.Neumann_line(g, "S", 0.0)]
    fixed = [P.Dirichlet_line(g, "W", 0.0, (0.0, 0.6))]
    z, r = node_xy(g)
    rho = 1e-9 * np.exp(-((z - 0.5) ** 2 + r ** 2) / 0.05)
    return g, fixed, mixed, rho


def test_collisionless_flow_field_setup():
    g, fixed, mixed, rho = collisionless_flow_field()
    # the partial Dirichlet line: W nodes with r in [0, 0.6] only
    idx, _ = fixed[0]
    assert len(idx) == sum(1 for j in range(g.cells[1] + 1) if j * g.delta[1] <= 0.6 + 1e-12)
    phi = direct_solve(g, "Cylindrical", fixed, mixed, rho)
    assert np.isfinite(phi).all()
    # the Robin condition holds at the E boundary to O(h): phi + b dphi/dz = 0.5 r
    I = g.cells[0]
    dz = g.delta[0]
    for j in (g.cells[1] // 4, g.cells[1] // 2):
        z, r = g.lower[0] + I * dz, j * g.delta[1]
        b = (z * z + r * r) / z
        dphi = (3 * phi[g.n2i(I, j)] - 4 * phi[g.n2i(I - 1, j)] + phi[g.n2i(I - 2, j)]) / (2 * dz)
        lhs = phi[g.n2i(I, j)] + b * dphi
        assert abs(lhs - 0.5 * r) < 0.05 * max(abs(0.5 * r), np.abs(phi).max() * 1e-3) + 1e-3
