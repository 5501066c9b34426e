"""PSuM's 3-D Poisson frontend tests restated on the host
(test/field_solver/test_psolver_3d.cpp and test_psolver_3d_multigrid.cpp):
the manufactured sin-sin-sin solution with grounded planes, the grounded
sphere around a uniform charge (Dirichlet_func), and the same manufactured
problem through the multigrid algorithm the backends run (the oracle's
FP32-in-FP64 restatement of the V-cycle schedule)."""
import math

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

import psum_b200 as P
from oracle import oracle as O
from psum_b200.field_solver import _merge_fixed

EPS0 = 8.854e-12


def node_xyz(g):
    axes = [g.lower[a] + np.arange(g.cells[a] + 1) * g.delta[a] for a in range(3)]
    return [c.reshape(-1) for c in np.meshgrid(*axes, indexing="ij")]


def solve_fixed(g, fixed, rho, eps=EPS0):
    """A phi = rho with the fixed rows replaced, solved on the free nodes
    (conjugate gradients to a relative residual of 1e-13)."""
    ridx, rval = _merge_fixed(fixed)
    r, c, v = P.assemble_poisson(g, ridx, eps)
    n = g.n_nodes
    A = sp.csr_matrix((v, (r.astype(np.int64), c.astype(np.int64))), shape=(n, n))
    fixed_mask = np.zeros(n, bool)
    fixed_mask[ridx.astype(np.int64)] = True
    free = np.nonzero(~fixed_mask)[0]
    fx = np.nonzero(fixed_mask)[0]
    phi = np.zeros(n)
    phi[ridx.astype(np.int64)] = rval
    b = np.asarray(rho, np.float64)[free] - A[free][:, fx] @ phi[fx]
    # the free-node block of a uniform-epsilon operator is symmetric positive definite
    sol, info = spl.cg(A[free][:, free].tocsr(), b, rtol=1e-13, atol=0.0, maxiter=20000)
    assert info == 0
    phi[free] = sol
    return phi, (r, c, v), ridx, rval


def grounded_planes(g):
    return [P.Dirichlet_plane(g, d, 0.0) for d in ("Ypos", "Yneg", "Xpos", "Xneg", "Zpos", "Zneg")]


def test_manufactured_solution_grounded_planes():
    # test_psolver_3d.cpp:13-77: phi = sin(pi x) sin(pi y) sin(pi z) on the
    # unit cube, rho = -eps0 lap(phi), all six planes grounded; L2 error of
    # order 2
    errs, Ns = [], (10, 20, 40)
    for N in Ns:
        g = P.simple_grid((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (N, N, N))
        x, y, z = node_xyz(g)
        exact = np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)
        rho = -EPS0 * (-3 * np.pi ** 2 * exact)
        phi, _, _, _ = solve_fixed(g, grounded_planes(g), rho)
        errs.append(np.sqrt(np.mean((phi - exact) ** 2)))
    order = math.log(errs[0] / errs[-1]) / math.log(Ns[-1] / Ns[0])
    assert 1.9 < order < 2.1, (errs, order)
    assert errs[-1] < 5e-4


def test_grounded_sphere_around_uniform_charge():
    # test_psolver_3d.cpp:79-119: nodes outside a sphere of radius 0.5 in
    # [0, 2]^3 are grounded (Dirichlet_func), the charge density is q0
    # everywhere; phi at the centre against r^2 q0 / (6 eps0).  The staircase
    # sphere makes the error first order in the cell size.
    radius, q0 = 0.5, 0.01
    theory = radius * radius * q0 / (6 * EPS0)
    errs = []
    for N in (40, 80):
        g = P.simple_grid((0.0, 0.0, 0.0), (2.0, 2.0, 2.0), (N, N, N))
        fixed = [P.Dirichlet_func(g, lambda x, y, z: (x - 1) ** 2 + (y - 1) ** 2 + (z - 1) ** 2 > radius ** 2, 0.0)]
        phi, _, _, _ = solve_fixed(g, fixed, np.full(g.n_nodes, q0))
        errs.append(abs(phi[g.n2i(N // 2, N // 2, N // 2)] - theory) / theory)
    assert errs[1] < 0.6 * errs[0] and errs[1] < 0.035, errs   # 5.8 % and 2.9 %


def test_multigrid_algorithm_matches_direct_solution():
    # test_psolver_3d_multigrid.cpp:13-92: the manufactured problem with the
    # multigrid backend; depth = ceil(log2(max nodes)) capped at 4.  Here the
    # backends' algorithm (FP32 V-cycles inside FP64 refinement) runs in the
    # oracle and must reach the direct solution
    for N in (16, 24):
        g = P.simple_grid((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (N, N, N))
        x, y, z = node_xyz(g)
        exact = np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)
        rho = -EPS0 * (-3 * np.pi ** 2 * exact)
        phi_direct, (r, c, v), ridx, rval = solve_fixed(g, grounded_planes(g), rho)
        nodes = N + 1
        depth = min(4, max(d for d in range(8) if (1 << d) < nodes) + 1)
        mg = O.Multigrid(r, c, v, g.n_nodes, nodes, nodes, nodes, depth)
        b = rho.copy()
        b[ridx.astype(np.int64)] = rval
        phi_mg, hist = mg.solve_mixed(b, np.zeros(g.n_nodes), max_cycles=60, correction_interval=4, pre=2, post=2)
        assert hist[-1] < 1e-9, hist
        assert np.abs(phi_mg - phi_direct).max() < 1e-8 * np.abs(phi_direct).max()
        l2_mg = np.sqrt(np.mean((phi_mg - exact) ** 2))
        l2_direct = np.sqrt(np.mean((phi_direct - exact) ** 2))
        assert l2_mg == pytest.approx(l2_direct, rel=1e-6)


def test_dirichlet_creators_3d():
    g = P.simple_grid((-1.0, -1.0, 0.0), (1.0, 1.0, 2.0), (8, 8, 8))
    x, y, z = node_xyz(g)
    idx, val = P.Dirichlet_box(g, -0.5, -0.5, 0.5, 0.5, 0.5, 1.5, 2.0)
    sel = (np.abs(x) <= 0.5 + 1e-9) & (np.abs(y) <= 0.5 + 1e-9) & (z >= 0.5 - 1e-9) & (z <= 1.5 + 1e-9)
    assert idx.tolist() == np.nonzero(sel)[0].tolist() and (val == 2.0).all()
    idx, _ = P.Dirichlet_box_rz(g, 0.0, 0.25, 1.0, 0.75, 1.0)
    r = np.sqrt(x * x + y * y)
    sel = (z <= 1.0 + 1e-9) & (r >= 0.25 - 1e-9) & (r <= 0.75 + 1e-9)
    assert idx.tolist() == np.nonzero(sel)[0].tolist()
    idx, _ = P.Dirichlet_func(g, lambda x, y, z: x + y + z > 2.0, 0.0)
    assert idx.tolist() == np.nonzero(x + y + z > 2.0)[0].tolist()
    # shape filter on a plane: in-plane coordinates (x, y) of a Z plane
    idx, _ = P.Dirichlet_plane(g, "Zpos", 0.0, shape=lambda u, v: u * u + v * v < 0.3)
    sel = (z == 2.0) & (x * x + y * y < 0.3)
    assert idx.tolist() == np.nonzero(sel)[0].tolist()
    with pytest.raises(TypeError):
        P.Dirichlet_box(g, 0.0, 0.0, 1.0, 1.0, 0.0)


# ---- test_native_vs_multigrid_3d.cpp:14-159: the Hall thruster case ----
HALL_Z, HALL_R = 0.080, 0.070
HALL_BODY_LEN, HALL_UP_TH, HALL_DOWN_TH, HALL_CERAMIC, HALL_METAL = 0.025, 0.016, 0.031, 0.004, 0.003


def hall_thruster_system(nx, ny, nz):
    """The reference case's frontend set-up: Robin planes a = 1, b = |p|^2 / p_n
    with value -10 on five sides, zero flux on z = 0, the anode annulus at
    300 on z = 0, two grounded-at--10 electrodes (Dirichlet_box_rz), ceramic
    rings at 4 eps0 and a charged annulus.  Returns (frontend, A, b)."""
    g = P.simple_grid((-HALL_R, -HALL_R, 0.0), (HALL_R, HALL_R, HALL_Z), (nx, ny, nz))

    def robin(normal):
        return lambda x, y, z: (1.0, (x * x + y * y + z * z) / normal(x, y, z))

    mixed = [P.Robin_plane(g, "Xpos", robin(lambda x, y, z: x), -10.0),
             P.Robin_plane(g, "Xneg", robin(lambda x, y, z: -x), -10.0),
             P.Robin_plane(g, "Ypos", robin(lambda x, y, z: y), -10.0),
             P.Robin_plane(g, "Yneg", robin(lambda x, y, z: -y), -10.0),
             P.Robin_plane(g, "Zpos", robin(lambda x, y, z: z), -10.0),
             P.Neumann_plane(g, "Zneg", 0.0)]
    fixed = [P.Dirichlet_plane(g, "Zneg", 300.0,
                               shape=lambda x, y: HALL_DOWN_TH < math.hypot(x, y) < HALL_R - HALL_UP_TH),
             P.Dirichlet_box_rz(g, HALL_BODY_LEN - HALL_METAL, 0.0, HALL_BODY_LEN, HALL_DOWN_TH, -10.0),
             P.Dirichlet_box_rz(g, HALL_BODY_LEN - HALL_METAL, HALL_R - HALL_UP_TH, HALL_BODY_LEN, HALL_R, -10.0)]

    def eps(x, y, z):
        r = math.hypot(x, y)
        ceramic = (0 < z < HALL_BODY_LEN and HALL_DOWN_TH < r < HALL_DOWN_TH + HALL_CERAMIC) or \
                  (0 < z < HALL_BODY_LEN and HALL_R - HALL_UP_TH - HALL_CERAMIC < r < HALL_R - HALL_UP_TH)
        return (4.0 if ceramic else 1.0) * EPS0

    ps = P.Poisson_solver_3d()
    ps.assemble(g, "Cartesian", fixed, eps, mixed)
    x, y, z = node_xyz(g)
    r = np.hypot(x, y)
    q = np.where((z > 0.005) & (z < 0.02) & (r > 0.037) & (r < 0.048), 1e-5, 0.0)
    rows, cols, vals = ps.coeff_matrix()
    A = sp.csr_matrix((vals, (rows.astype(np.int64), cols.astype(np.int64))), shape=(g.n_nodes, g.n_nodes))
    return ps, A, ps.make_righthand_item(q)


def test_hall_thruster_multigrid_approaches_direct_solution():
    # FP64 V(2,1) cycles at depth 2 (the reference's eigen_multigrid_cpu
    # settings) against the direct solution: the relative L2 difference
    # falls with the cycle count (1, 5, 15, 20 as the reference prints)
    nx, ny, nz = 32, 32, 20
    ps, A, b = hall_thruster_system(nx, ny, nz)
    direct = spl.spsolve(A.tocsc(), b)
    assert direct.max() == pytest.approx(300.0) and direct.min() >= -10.0 - 1e-6
    rows, cols, vals = ps.coeff_matrix()
    mg = O.Multigrid(rows, cols, vals, A.shape[0], nx + 1, ny + 1, nz + 1, 2)
    errs = [np.linalg.norm(mg.vcycles(b, np.zeros(A.shape[0]), c, 2, 1) - direct) / np.linalg.norm(direct)
            for c in (1, 5, 15, 20)]
    assert all(e1 < e0 for e0, e1 in zip(errs, errs[1:])), errs
    assert errs[-1] < 1e-7, errs        # 0.21, 1.5e-3, 4.7e-7, 1.1e-8
