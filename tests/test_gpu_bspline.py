"""GPU parity of the B-spline gathers and deposit (include/psum_interp.h)
against the oracle's restatement of interp_B_spline / interp_diff_B_spline /
add_back_B_spline (src/field/higher_order_interp.hpp:196-247).

Tolerances: the gathers evaluate the full tensor-product sum, factor by
factor, so they are compared with the oracle's full sum (no weight skip) at
1e-12 of the field scale (times dr for gradients), and with the reference's
skipped sum at the skip bound 1e-10 * sum|field| over the support.  The
deposit keeps the skip and rounds each weight to 2^-F (F from
psum_bspline_deposit_bits), so each node may differ from the oracle by at
most (contributions to the node) * 2^-(F+1) * weight, plus FP64 rounding.
"""
import numpy as np
import pytest

import psum_b200 as P
from psum_b200 import interp as I
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def case(dim, seed, n=6000):
    rng = np.random.default_rng(seed)
    cells = (23, 17, 11)[:dim]
    lower = np.array((-0.5, 0.25, 1.0)[:dim])
    upper = lower + np.array((2.3, 1.7, 1.1)[:dim])
    grid = P.simple_grid(lower, upper, cells)
    g = O.make_grid(cells, lower, upper, (0,) * dim)
    # the whole domain and half a cell beyond it (stencils wrap), a few
    # non-finite and far-away positions without support
    dx = (upper - lower) / np.array(cells)
    pos = lower[:, None] - 0.5 * dx[:, None] + (upper - lower + dx)[:, None] * rng.random((dim, n))
    pos[0, 7] = np.nan
    pos[-1, 11] = np.inf
    pos[0, 13] = upper[0] + 10 * (upper[0] - lower[0])
    field = rng.normal(size=int(np.prod([c + 1 for c in cells])))
    return grid, g, pos, field, dx


def dev(a):
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("order", [1, 2, 3, 4])
def test_gathers_match_oracle(order, dim):
    grid, g, pos, field, dx = case(dim, 300 + 10 * order + dim)
    skipped = torch.zeros(1, dtype=torch.int64, device="cuda")
    val = P.interp_B_spline(order, grid, dev(pos), dev(field), skipped).cpu().numpy()
    grad = P.interp_diff_B_spline(order, grid, dev(pos), dev(field), skipped).cpu().numpy()
    assert int(skipped.item()) == 2 * 3
    ref_v = O.bspline_gather(g, order, pos, field, tol=0.0)
    ref_g = O.bspline_gather(g, order, pos, field, grad=True, tol=0.0)
    assert (np.isnan(val) == np.isnan(ref_v)).all()
    assert (np.isnan(grad) == np.isnan(ref_g)).all()
    ok = ~np.isnan(ref_v)
    scale = np.abs(field).max()
    dr = (1 / dx).max()
    np.testing.assert_allclose(val[ok], ref_v[ok], rtol=0, atol=1e-12 * scale)
    np.testing.assert_allclose(grad[:, ok], ref_g[:, ok], rtol=0, atol=1e-12 * scale * dr)
    # against the reference's own sum with the 1e-10 weight skip
    S = (order + 1) ** dim
    skip_v = O.bspline_gather(g, order, pos, field, tol=1e-10)
    skip_g = O.bspline_gather(g, order, pos, field, grad=True, tol=1e-10)
    assert np.abs(val[ok] - skip_v[ok]).max() <= 1e-10 * S * scale + 1e-12 * scale
    assert np.abs(grad[:, ok] - skip_g[:, ok]).max() <= 1e-10 * S * scale + 1e-12 * scale * dr


def _contributions(g, order, pos, nn):
    c = np.zeros(nn)
    for i in range(pos.shape[1]):
        idx, w, _ = O.bspline_support(g, order, pos[:, i])
        c[idx[np.abs(w) > 1e-10]] += 1
    return c


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("order", [1, 2, 3, 4])
def test_deposit_matches_oracle_and_is_order_independent(order, dim):
    grid, g, pos, field, dx = case(dim, 400 + 10 * order + dim, n=3000)
    nn = field.size
    w = 0.37
    base = np.random.default_rng(5).normal(size=nn)
    out = dev(base)
    skipped = torch.zeros(1, dtype=torch.int64, device="cuda")
    P.add_back_B_spline(order, grid, dev(pos), w, out, skipped=skipped)
    got = out.cpu().numpy()
    assert int(skipped.item()) == 3
    ref, ref_skipped = O.bspline_deposit(g, order, pos, w, nn)
    assert ref_skipped == 3
    F = I.deposit_bits(pos.shape[1])
    bound = _contributions(g, order, pos, nn) * 2.0 ** -(F + 1) * w + 1e-13 * (1 + np.abs(ref) + np.abs(base))
    assert (np.abs(got - base - ref) <= bound).all()
    # charge: w per supported position, less the skipped weights (< 1e-10 each)
    assert abs((got - base).sum() - w * (pos.shape[1] - 3)) < 1e-9 * pos.shape[1]
    # the result does not depend on the order of the positions, and a caller
    # scratch gives the same bits as the pool allocation
    perm = np.random.default_rng(6).permutation(pos.shape[1])
    out2 = dev(base)
    scratch = torch.empty(nn, dtype=torch.int64, device="cuda")
    P.add_back_B_spline(order, grid, dev(pos[:, perm]), w, out2, scratch=scratch)
    assert (out2.cpu().numpy().view(np.int64) == got.view(np.int64)).all()


def test_argument_errors():
    grid, g, pos, field, dx = case(2, 1, n=20)
    with pytest.raises(ValueError):
        P.interp_B_spline(5, grid, dev(pos), dev(field))
    bad = P.simple_grid((0.0, 0.0), (1.0, 1.0), (4, 4))
    gd = I.grid_desc(bad)
    gd.cells[1] = 0
    code = P.lib().psum_interp_bspline(gd, 2, 20, dev(pos).data_ptr(), dev(field).data_ptr(),
                                       dev(np.zeros(20)).data_ptr(), None, None)
    assert code == 1
    code = P.lib().psum_add_back_bspline(I.grid_desc(grid), 2, 20, dev(pos).data_ptr(), float("nan"),
                                         dev(field).data_ptr(), None, None, None)
    assert code == 7
