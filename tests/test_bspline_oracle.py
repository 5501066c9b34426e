"""The oracle's B-spline restatement (orders 1-4; src/field/higher_order_interp.hpp,
src/field/simple_interpolation.hpp:105-184, simple_grid.hpp:316-397) pinned
against the properties PSuM's own tests assert for it (CPU only):

  test/field/test_higher_order_interp.cpp      order p = cell average of order p-1
  test/field/test_higher_order_interpDiff.cpp  derivative weights = central differences
  test/field/test_higher_order_addback.cpp     deposit = k^2 sub-cell deposits of order p-1
plus partition of unity and linear reproduction (test_simpleinterp.cpp's
criteria carried to the higher orders).
"""
import numpy as np
import pytest

from oracle import oracle as O


def adversarial_grid(rng, dim):
    """Per-axis cell counts and extents drawn as the reference tests draw them."""
    lower = rng.random(dim) - 0.5
    size = (20 * rng.random(dim)).astype(int) + 6 + np.arange(dim)
    upper = lower + (1.0 + 0.7 * np.arange(dim) + 0.5 * rng.random(dim)) * size * 0.1
    return lower, upper, size


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("order", [1, 2, 3, 4])
def test_partition_of_unity_and_linear_reproduction(order, dim):
    rng = np.random.default_rng(10 * order + dim)
    lower, upper, size = adversarial_grid(rng, dim)
    g = O.make_grid(size, lower, upper, (0,) * dim)
    dx = (upper - lower) / size
    a = rng.normal(size=dim)
    S = order + 1
    for _ in range(200):
        # interior points: the support must not wrap for linear reproduction
        p = lower + dx * (S / 2 + 1 + rng.random(dim) * (size - S - 2))
        idx, w, dw = O.bspline_support(g, order, p)
        assert len(idx) == S ** dim
        assert abs(w.sum() - 1.0) < 1e-12
        assert np.abs(dw.sum(axis=1)).max() < 1e-10 * np.abs(1 / dx).max()
        assert (w >= -1e-15).all()
        node = np.stack(np.unravel_index(idx, tuple(size + 1)), 0)
        xn = lower[:, None] + node * dx[:, None]
        f = a @ xn
        assert abs(f @ w - a @ p) < 1e-12 * (1 + np.abs(f).max())
        np.testing.assert_allclose(dw @ f, a, rtol=0, atol=1e-10 * (1 + np.abs(a).max()))


def _ghost_extended(rng, dim, lower, upper, size):
    """f1 on the grid and f2 on the grid grown by two ghost layers per side,
    mapped periodically like the stencil wrap (test_higher_order_interp.cpp:46-66)."""
    dx = (upper - lower) / size
    N = size + 1
    f1 = rng.random(int(np.prod(N)))
    size2 = size + 4
    N2 = size2 + 1
    grid_idx = np.stack(np.unravel_index(np.arange(int(np.prod(N2))), tuple(N2)), 0)
    src = np.mod(grid_idx - 2, N[:, None])
    f2 = f1[np.ravel_multi_index(tuple(src), tuple(N))]
    g1 = O.make_grid(size, lower, upper, (0,) * dim)
    g2 = O.make_grid(size2, lower - 2 * dx, upper + 2 * dx, (0,) * dim)
    return g1, g2, f1, f2, dx


@pytest.mark.parametrize("dim,m", [(1, 100), (2, 100), (3, 8)])
@pytest.mark.parametrize("order", [2, 3, 4])
def test_integral_regression(order, dim, m):
    # sum_j b_p(u - j) f_j = lim_k (1/k^d) sum over the k^d sub-cell centres of
    # the one-cell window around u of sum_j b_{p-1}(x - j) f_j; the midpoint
    # rule converges as 1/k^2, so each 4x refinement must cut the mean error
    # by at least 4x, ending below 1e-4 (worst 5e-4).  Raw weighted sums, no
    # weight skip, as the reference test sums them.
    rng = np.random.default_rng(100 + 10 * order + dim)
    lower, upper, size = adversarial_grid(rng, dim)
    g1, g2, f1, f2, dx = _ghost_extended(rng, dim, lower, upper, size)
    u = lower[:, None] + (upper - lower)[:, None] * rng.random((dim, m))
    vp = O.bspline_gather(g1, order, u, f1, tol=0.0)
    means, worsts = [], []
    for k in (4, 16, 64):
        sub = (np.arange(k) + 0.5) / k - 0.5
        offs = np.stack(np.meshgrid(*([sub] * dim), indexing="ij"), 0).reshape(dim, -1) * dx[:, None]
        x = (u[:, :, None] + offs[:, None, :]).reshape(dim, -1)
        vm = O.bspline_gather(g2, order - 1, x, f2, tol=0.0).reshape(m, -1).mean(axis=1)
        err = np.abs(vp - vm)
        means.append(err.mean())
        worsts.append(err.max())
    for a, b in zip(means, means[1:]):
        assert b < 0.25 * a
    assert means[-1] < 1e-4 and worsts[-1] < 5e-4


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("order", [1, 2, 3, 4])
def test_diff_vs_central_difference(order, dim):
    # test_higher_order_interpDiff.cpp:21-80: white-noise node field, h = 1e-4
    # cells, every coordinate at least 4h from a node plane; mean error below
    # 1e-6 and worst below 1e-4.
    rng = np.random.default_rng(200 + 10 * order + dim)
    lower, upper, size = adversarial_grid(rng, dim)
    g = O.make_grid(size, lower, upper, (0,) * dim)
    dx = (upper - lower) / size
    f = rng.random(int(np.prod(size + 1)))
    h = 1e-4
    m = 200
    u = np.empty((dim, m))
    for a in range(dim):
        vals = []
        while len(vals) < m:
            c = lower[a] + (upper[a] - lower[a]) * rng.random()
            v = (c - lower[a]) / dx[a]
            frac = v - np.floor(v)
            if 4 * h <= frac <= 1 - 4 * h:
                vals.append(c)
        u[a] = vals
    direct = O.bspline_gather(g, order, u, f, grad=True, tol=0.0)
    errs = []
    for d in range(dim):
        e = np.zeros((dim, 1))
        e[d] = h * dx[d]
        fd = (O.bspline_gather(g, order, u + e, f, tol=0.0) - O.bspline_gather(g, order, u - e, f, tol=0.0)) \
            / (2 * h * dx[d])
        errs.append(np.abs(direct[d] - fd))
    errs = np.concatenate(errs)
    assert errs.mean() < 1e-6 and errs.max() < 1e-4


@pytest.mark.parametrize("hi", [2, 3, 4])
def test_addback_matches_subcell_deposits(hi):
    # test_higher_order_addback.cpp: one order-p deposit at p against k^2
    # order-(p-1) deposits of weight w/k^2 at the sub-cell centres of the
    # one-cell window around p; the charge is kept (up to the 1e-10 weight
    # skip) and the difference falls as the window is refined.
    N = 32
    g = O.make_grid((N, N), (0.0, 0.0), (1.0, 1.0), (0, 0))
    nn = (N + 1) ** 2
    delta = 1.0 / N
    p = np.array([[0.50625], [0.50625]])
    f_hi, skipped = O.bspline_deposit(g, hi, p, 1.0, nn)
    assert skipped == 0
    assert abs(f_hi.sum() - 1.0) < 1e-9
    l2 = []
    for k in (1, 8, 32):
        sub = (np.arange(k) + 0.5) / k * delta - 0.5 * delta
        xs = np.stack(np.meshgrid(sub, sub, indexing="ij"), 0).reshape(2, -1) + p
        f_lo, _ = O.bspline_deposit(g, hi - 1, xs, 1.0 / k ** 2, nn)
        assert abs(f_lo.sum() - 1.0) < 1e-9
        l2.append(np.sqrt(((f_hi - f_lo) ** 2).sum()) * delta)
    assert l2[2] < 0.25 * l2[1] < l2[0]


def test_no_support_far_outside_and_nonfinite():
    g = O.make_grid((8, 8), (0.0, 0.0), (1.0, 1.0), (0, 0))
    for p in ([np.nan, 0.5], [0.5, np.inf], [5.0, 0.5], [-3.0, 0.5]):
        idx, w, _ = O.bspline_support(g, 3, np.array(p))
        assert len(idx) == 0
    # near the upper edge the stencil wraps once and keeps its support (the reference's stencil wrap)
    idx, w, _ = O.bspline_support(g, 2, np.array([0.999, 0.5]))
    assert len(idx) == 9 and abs(w.sum() - 1) < 1e-12
    pos = np.array([[0.3, np.nan, 7.0], [0.4, 0.5, 0.5]])
    out = O.bspline_gather(g, 2, pos, np.ones(81))
    assert out[0] == pytest.approx(1.0) and np.isnan(out[1]) and np.isnan(out[2])
    field, skipped = O.bspline_deposit(g, 2, pos, 1.0, 81)
    assert skipped == 2 and field.sum() == pytest.approx(1.0)
