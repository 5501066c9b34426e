"""Host-side pieces of the differentiable run (no GPU): the loss and its
gradient on the node lattice."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
from psum_b200.adjoint import field_energy_loss  # noqa: E402


def test_field_energy_loss_gradient_matches_autograd_reference():
    rng = np.random.default_rng(3)
    phi = torch.tensor(rng.normal(size=(5 * 7)), dtype=torch.float64, requires_grad=True)
    L = field_energy_loss(phi, (5, 7), (0.5, 2.0), (1, 0))
    g = torch.autograd.grad(L, phi)[0].numpy()
    p = phi.detach().numpy().reshape(5, 7)
    ref = np.zeros_like(p)
    d0 = (np.roll(p, -1, 0) - p) / 0.5
    ref += -2 * d0 / 0.5 + np.roll(2 * d0 / 0.5, 1, 0)
    d1 = (p[:, 1:] - p[:, :-1]) / 2.0
    ref[:, 1:] += 2 * d1 / 2.0
    ref[:, :-1] -= 2 * d1 / 2.0
    assert np.allclose(g, ref.ravel())


def test_poisson_solve_is_self_adjoint_on_free_nodes():
    # S = A^-1 P (P zeroes the fixed rows' sources) is symmetric for PSuM's
    # Cartesian operator, so the adjoint solve is the forward solve
    import scipy.sparse as sp

    import psum_b200 as P
    from psum_b200.adjoint import check_free_block_symmetric
    cases = []
    g = P.simple_grid((0.5, 0.5), (7.5, 7.5), (7, 7))               # periodic wrapping nodes, pinned node
    cases.append((g, P.Dirichlet_nodes(g, [(0, 0)], 0.0)[0]))
    g2 = P.simple_grid((0.0, 0.0), (1.0, 2.0), (6, 5))              # Dirichlet box
    cases.append((g2, np.unique(np.concatenate([P.Dirichlet_line(g2, d, 0.0)[0] for d in "NSEW"]))))
    for grid, fixed in cases:
        r, c, v = P.assemble_poisson(grid, fixed, 1.0)
        n = grid.n_nodes
        check_free_block_symmetric(r, c, v, fixed, n)
        A = sp.csr_matrix((v, (r.astype(np.int64), c.astype(np.int64))), shape=(n, n)).toarray()
        Pm = np.eye(n)
        Pm[fixed.astype(np.int64), fixed.astype(np.int64)] = 0.0
        S = np.linalg.solve(A, Pm)
        assert np.allclose(S, S.T, atol=1e-12 * np.abs(S).max())


def test_asymmetric_free_block_is_refused():
    from psum_b200.adjoint import check_free_block_symmetric
    rows = np.array([0, 0, 1, 1, 2], np.uint64)
    cols = np.array([0, 1, 0, 1, 2], np.uint64)
    vals = np.array([2.0, -1.0, -0.5, 2.0, 1.0])
    with pytest.raises(NotImplementedError):
        check_free_block_symmetric(rows, cols, vals, np.array([2], np.uint64), 3)
