"""The FP64 CPU oracle pinned against the golden known answers and against the
properties PSuM's own tests assert for this path (CPU only)."""
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

from oracle import oracle as O

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "known_answers.npz"))


def csr(rows, cols, vals, n):
    return sp.csr_matrix((vals, (rows.astype(np.int64), cols.astype(np.int64))), shape=(n, n))


# ---------------------------------------------------------------- CIC -----
def test_cic_golden():
    g = O.make_grid((8, 8), (0, 0), (1, 1), (0, 0))
    for p, idx, w in zip(GOLD["cic2_points"], GOLD["cic2_idx"], GOLD["cic2_w"]):
        i, c = O.interp(g, p)
        assert (i == idx).all()
        np.testing.assert_allclose(c, w, rtol=0, atol=1e-15)


@pytest.mark.parametrize("dim", [2, 3])
def test_cic_partition_of_unity_and_linear(dim):
    # test/field/test_simpleinterp.cpp:51-218: partition of unity, one-hot at
    # nodes, exact reproduction of linear functions, all at 1e-12.
    rng = np.random.default_rng(1)
    cells = (7, 5, 6)[:dim]
    lo = (-1.0, 0.5, 2.0)[:dim]
    hi = (2.5, 3.0, 4.0)[:dim]
    g = O.make_grid(cells, lo, hi, (0,) * dim)
    dx = [(h - l) / c for l, h, c in zip(lo, hi, cells)]
    nodes = [np.arange(c + 1) * d + l for c, d, l in zip(cells, dx, lo)]
    coords = np.stack(np.meshgrid(*nodes, indexing="ij"), 0).reshape(dim, -1)
    a = rng.normal(size=dim)
    lin = a @ coords + 0.7
    for _ in range(200):
        p = np.array([rng.uniform(l, h) for l, h in zip(lo, hi)])
        idx, c = O.interp(g, p)
        assert abs(c.sum() - 1) < 1e-12
        assert abs((lin[idx] * c).sum() - (a @ p + 0.7)) < 1e-12
        _, dc = O.interp_diff(g, p)
        np.testing.assert_allclose([(lin[idx] * dc[d]).sum() for d in range(dim)], a, atol=1e-10)
    # one-hot at interior nodes
    node = [2] * dim
    p = np.array([lo[d] + node[d] * dx[d] for d in range(dim)])
    idx, c = O.interp(g, p)
    assert abs(c.max() - 1.0) < 1e-12 and np.sort(np.abs(c))[-2] < 1e-12


@pytest.mark.parametrize("dim", [2, 3])
def test_interp_diff_vs_central_differences(dim):
    # test/field/test_field_interpDiff.cpp:47-143: h = 1e-7, mean abs error < 1e-6
    rng = np.random.default_rng(2)
    cells = (9, 8, 7)[:dim]
    g = O.make_grid(cells, (0,) * dim, (1,) * dim, (0,) * dim)
    nn = int(np.prod([c + 1 for c in cells]))
    phi = rng.normal(size=nn)
    pts = rng.uniform(0.05, 0.95, size=(dim, 300))
    grad = O.gather_grad(g, pts, phi)
    h = 1e-7
    errs = []
    for i in range(pts.shape[1]):
        for d in range(dim):
            pp, pm = pts[:, i].copy(), pts[:, i].copy()
            pp[d] += h
            pm[d] -= h
            ip, cp = O.interp(g, pp)
            im, cm = O.interp(g, pm)
            fd = ((phi[ip] * cp).sum() - (phi[im] * cm).sum()) / (2 * h)
            errs.append(abs(fd - grad[d, i]))
    errs = np.array(errs)
    # points whose FD stencil crosses a cell face see the kink; the mean stays small
    assert errs.mean() < 1e-3 and np.median(errs) < 1e-6


def test_interp_wraps_periodic_support():
    # TSI idiom: lo = dx/2, 63 cells, nodes wrap at 64 (simple_grid.hpp:338-343)
    g = O.make_grid((63,), (0.5,), (63.5,), (1,))
    idx, c = O.interp(g, [0.25])
    assert list(idx) == [63, 0]
    np.testing.assert_allclose(c, [0.25, 0.75])


# ----------------------------------------------------------- push/deposit --
def test_push_golden_uniform_field():
    g = O.make_grid((16, 16), (0, 0), (16, 16), (0, 0))
    qm, dt = GOLD["push_qm_dt"]
    pos, vel, loss = O.push(g, GOLD["push_pos0"], GOLD["push_vel0"], GOLD["push_phi"], qm, dt)
    np.testing.assert_allclose(pos, GOLD["push_pos1"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(vel, GOLD["push_vel1"], rtol=0, atol=1e-13)
    assert loss.sum() == 0


def test_deposit_golden():
    g = O.make_grid((8, 8), (0, 0), (1, 1), (0, 0))
    rho = O.deposit(g, GOLD["dep_points"].T, 1.0, 81)
    np.testing.assert_allclose(rho, GOLD["dep_rho"], atol=1e-15)


def test_push_absorb_and_wrap_counts():
    g = O.make_grid((4, 4), (0, 0), (4, 4), (0, 1))
    pos = np.array([[0.05, 3.95, 2.0, 1.0], [1.0, 1.0, 0.02, 3.99]])
    vel = np.array([[-1.0, 1.0, 0.0, 0.0], [0.0, 0.0, -1.0, 1.0], [0, 0, 0, 0.0]])
    phi = np.zeros(25)
    p, v, loss = O.push(g, pos, vel, phi, 1.0, 0.1)
    assert np.isnan(p[0, 0]) and np.isnan(p[0, 1])
    assert loss.tolist() == [[1, 1], [0, 0]]
    # y is periodic with period 5 (wrapping node lattice): 0.02-0.1 -> 4.92
    assert abs(p[1, 2] - 4.92) < 1e-12 and abs(p[1, 3] - 4.09) < 1e-12


def test_binning_golden():
    g = O.make_grid((4, 3), (0, 0), (4, 3), (0, 0))
    keys, counts, offsets, perm = O.bin_particles(g, GOLD["bin_pos"])
    assert (keys == GOLD["bin_keys"]).all()
    assert (counts == GOLD["bin_counts"]).all()
    assert (offsets == GOLD["bin_offsets"]).all()
    assert (perm == GOLD["bin_perm"]).all()


def test_binning_clamps_truncation_to_the_last_cell():
    """inGrid admits p = nextafter(hi, lo), but (p - lo) * dr can truncate to `cells` when dr = 1/dx rounds
    up; the oracle bins such a position into the last cell (the reference's nC would index past the counts)."""
    cells, lo, hi = (199, 7), (0.0, 0.0), (3.3, 7.0)
    dr = 1.0 / ((hi[0] - lo[0]) / cells[0])
    edge = np.nextafter(hi[0], lo[0])
    assert int((edge - lo[0]) * dr) == cells[0]                    # the case is reached on this grid
    # how common the case is: (cells, hi) pairs on [0, hi) where the position below hi truncates to cells
    hits = sum(int(np.nextafter(h, 0.0) * (1.0 / (h / c))) == c for c in range(1, 200) for h in (1.1, 3.3, 0.7))
    assert hits > 0
    pos = np.array([[edge, edge, 1.0, edge], [0.5, 6.999999999999999, 3.2, np.nextafter(7.0, 0.0)]])
    keys, counts, offsets, perm = O.bin_particles(O.make_grid(cells, lo, hi, (0, 0)), pos)
    last_row = (cells[0] - 1) * cells[1]
    assert list(keys) == [last_row + 0, last_row + 6, int(1.0 * dr) * 7 + 3, last_row + 6]
    assert counts.sum() == 4 and counts.size == cells[0] * cells[1]
    assert list(perm) == [2, 0, 1, 3]


# ------------------------------------------------------------- multigrid ---
def dirichlet_box_2d(N, eps=1.0, lo=0.0, hi=1.0):
    fixed = [i * (N + 1) + j for i in range(N + 1) for j in range(N + 1) if i in (0, N) or j in (0, N)]
    r, c, v = O.poisson_assemble((N, N), (lo, lo), (hi, hi), eps, fixed)
    return r, c, v, np.array(fixed, np.int64)


def test_mg_vs_direct_manufactured_2d():
    # test_native_vs_mg_2d_manufactured.cpp:22-129: 64^2, depth 3, V(2,2),
    # within 1e-4 of the direct solution in <= 5 cycles.
    N = 64
    eps = 8.854e-12
    r, c, v, fixed = dirichlet_box_2d(N, eps)
    n = (N + 1) ** 2
    x = np.linspace(0, 1, N + 1)
    X, Y = np.meshgrid(x, x, indexing="ij")
    b = (-eps * (-2 * np.pi ** 2 * np.sin(np.pi * X) * np.sin(np.pi * Y))).ravel()
    b[fixed] = 0.0
    direct = spl.spsolve(csr(r, c, v, n).tocsc(), b)
    mg = O.Multigrid(r, c, v, n, N + 1, N + 1, 1, 3)
    ok = False
    for cyc in (1, 2, 5):
        xm = mg.vcycles(b, np.zeros(n), cyc, 2, 2)
        if np.linalg.norm(xm - direct) / np.linalg.norm(direct) < 1e-4:
            ok = True
            break
    assert ok


def test_mg_residual_reduction_5pt():
    # test_multigrid_core.cpp:142-207: 5-point, b = 1, x0 = 0, depth 4, V(2,1),
    # residual monotone (<= 1.1x previous), total reduction < 1e-5 in 10 cycles.
    N = 128   # node box 129^2 (the reference uses 256^2; same coarsening ratios)
    r, c, v, fixed = dirichlet_box_2d(N)
    n = (N + 1) ** 2
    b = np.ones(n)
    b[fixed] = 0.0
    mg = O.Multigrid(r, c, v, n, N + 1, N + 1, 1, 4)
    x = np.zeros(n)
    res = [mg.rel_residual(b, x)]
    for _ in range(10):
        x = mg.vcycles(b, x, 1, 2, 1)
        res.append(mg.rel_residual(b, x))
    for a, bb in zip(res, res[1:]):
        assert bb <= 1.1 * a
    assert res[-1] / res[0] < 1e-5


def test_open_interval_transfers_diverge_on_wrapping_lattice():
    # PSuM's transfers (multigrid_utilities.hpp:55-104) on a periodic 64^2
    # lattice pinned at node 0 (TSI idiom, main.cpp:106-113): depth 3 V(2,2)
    # cycles diverge -- the reason the periodic transfer option exists.
    n1 = 64
    r, c, v = O.poisson_assemble((n1 - 1,) * 2, (0.5,) * 2, (n1 - 0.5,) * 2, 1.0, [0])
    n = n1 ** 2
    rng = np.random.default_rng(3)
    b = rng.normal(size=n)
    b -= b.mean()
    b[0] = 0.0
    direct = spl.spsolve(csr(r, c, v, n).tocsc(), b)
    err = {}
    for per in (0, 1):
        mg = O.Multigrid(r, c, v, n, n1, n1, 1, 3, periodic=(per, per, 0))
        x = mg.vcycles(b, np.zeros(n), 30, 2, 2)
        err[per] = np.linalg.norm(x - direct) / np.linalg.norm(direct)
    assert err[0] > 1.0
    assert err[1] < 1e-8


def test_mg_7pt_periodic_pinned_3d():
    # 7-point periodic operator with one pinned node, periodic transfers
    n1 = 16
    r, c, v = O.poisson_assemble((n1 - 1,) * 3, (0.5,) * 3, (n1 - 0.5,) * 3, 1.0, [0])
    n = n1 ** 3
    rng = np.random.default_rng(3)
    b = rng.normal(size=n)
    b -= b.mean()
    b[0] = 0.0
    A = csr(r, c, v, n)
    direct = spl.spsolve(A.tocsc(), b)
    mg = O.Multigrid(r, c, v, n, n1, n1, n1, 3, periodic=(1, 1, 1))
    assert [mg.level_rows(l) for l in range(mg.levels)] == [4096, 512, 64, 8]
    x = mg.vcycles(b, np.zeros(n), 25, 2, 1)
    assert np.linalg.norm(x - direct) / np.linalg.norm(direct) < 1e-6


def test_mg_mixed_refinement_reaches_fp64():
    N = 64
    r, c, v, fixed = dirichlet_box_2d(N)
    n = (N + 1) ** 2
    rng = np.random.default_rng(4)
    b = rng.normal(size=n)
    b[fixed] = 0.0
    mg = O.Multigrid(r, c, v, n, N + 1, N + 1, 1, 4)
    x, hist = mg.solve_mixed(b, np.zeros(n), 24, 4, 2, 1)
    assert hist[-1] < 1e-10
    assert all(h2 < h1 for h1, h2 in zip(hist, hist[1:]))


def test_mg_mixed_refinement_stops_at_tol():
    """The tol-stopped mixed solve of the CPU arm stops after the first batch of cycles whose relative
    residual reaches tol (the GPU backends' rule), with the same iterate as the fixed-count solve run for as
    many batches."""
    N = 64
    r, c, v, fixed = dirichlet_box_2d(N)
    n = (N + 1) ** 2
    rng = np.random.default_rng(5)
    b = rng.normal(size=n)
    b[fixed] = 0.0
    mg = O.Multigrid(r, c, v, n, N + 1, N + 1, 1, 4)
    x, hist = mg.solve_mixed_tol(b, np.zeros(n), 24, 2, 2, 2, 1e-8)
    assert hist[-1] <= 1e-8 < hist[-2]
    assert all(h > 1e-8 for h in hist[:-1])
    assert mg.rel_residual(b, x) <= 1.01e-8
    x_fixed, _ = mg.solve_mixed(b, np.zeros(n), 2 * len(hist), 2, 2, 2)
    assert np.array_equal(x, x_fixed)


def test_fd_order_manufactured():
    # test_manufactured_solution_2d.cpp:87-91: L2 < 1e-3 and order in (1.5, 2.5)
    errs = []
    for N in (16, 32, 64):
        r, c, v, fixed = dirichlet_box_2d(N)
        n = (N + 1) ** 2
        x = np.linspace(0, 1, N + 1)
        X, Y = np.meshgrid(x, x, indexing="ij")
        exact = (np.sin(np.pi * X) * np.sin(np.pi * Y)).ravel()
        b = (2 * np.pi ** 2 * exact).copy()
        b[fixed] = 0
        phi = spl.spsolve(csr(r, c, v, n).tocsc(), b)
        errs.append(np.sqrt(np.mean((phi - exact) ** 2)))
    orders = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert errs[-1] < 1e-3
    assert ((orders > 1.5) & (orders < 2.5)).all()


def test_five_point_check_solvers_residual():
    # check_solvers.cpp:56-107: n^2 interior 5-point stencil, b = 1; residual < 1e-8
    n = 63
    h = 1.0 / (n + 1)
    rows, cols, vals = [], [], []
    for j in range(n):
        for i in range(n):
            idx = j * n + i
            rows.append(idx); cols.append(idx); vals.append(4.0 / h / h)
            for di, ok in ((-1, i > 0), (1, i < n - 1), (-n, j > 0), (n, j < n - 1)):
                if ok:
                    rows.append(idx); cols.append(idx + di); vals.append(-1.0 / h / h)
    rows, cols, vals = np.array(rows, np.uint64), np.array(cols, np.uint64), np.array(vals)
    N = n * n
    b = np.ones(N)
    mg = O.Multigrid(rows, cols, vals, N, n, n, 1, 4)
    x = mg.vcycles(b, np.zeros(N), 40, 4, 2)
    res = np.abs(csr(rows, cols, vals, N) @ x - b).max()
    assert res < 1e-8


def test_transfer_structure_keeps_endpoints():
    # multigrid_utilities.hpp:28-33: coarse axis = every 2nd node + last node
    N1 = 9   # 2-D box 9x9 nodes: axes 0..8 -> 0,2,4,6,8
    r, c, v, fixed = dirichlet_box_2d(N1 - 1)
    mg = O.Multigrid(r, c, v, N1 * N1, N1, N1, 1, 2)
    assert [mg.level_rows(l) for l in range(mg.levels)] == [81, 25, 9]
    N2 = 8   # 8 nodes per axis: 0,2,4,6,7 -> 0,4,7? (every 2nd of 5 coarse + last)
    r, c, v = O.poisson_assemble((7, 7), (0.5, 0.5), (7.5, 7.5), 1.0, [0])
    mg = O.Multigrid(r, c, v, 64, 8, 8, 1, 2)
    assert [mg.level_rows(l) for l in range(mg.levels)] == [64, 25, 9]
