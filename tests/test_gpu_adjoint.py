"""Adjoint of the electrostatic step (differentiable runs) on the GPU.

A small Landau-damping run (2-D periodic wrapping-node grid pinned at one
node, electrons over a uniform ion background, leapfrog, checkpoints every
K steps) differentiated with respect to the electrons' initial velocities
and an external potential.  The FP64 adjoint is checked against central
finite differences of the FP64 forward (eps = 1e-3); the mixed-precision
adjoint (FP32 adjoint arrays) against the FP64 adjoint."""
import numpy as np
import pytest

import psum_b200 as P
from psum_b200.adjoint import ElectrostaticLoss, ElectrostaticRun

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

CELLS = 31            # 32 wrapping nodes per axis, period 32
PPC = 16
STEPS, K, DT = 20, 5, 0.1
MG = ("I 32 J 32 K 1 depth 4 pre_relax 2 post_relax 2 max_cycles 60 correction_interval 4 tol 1e-12 "
      "periodic_I 1 periodic_J 1")


def landau_setup(seed=41):
    rng = np.random.default_rng(seed)
    L = CELLS + 1.0
    n = int(L * L * PPC)
    # 5% mode-1 density perturbation in x by inverse-CDF displacement of uniform positions
    u = rng.uniform(0.0, L, n)
    x = u.copy()
    k = 2 * np.pi / L
    for _ in range(20):   # Newton on x + (0.05/k) sin(k x) = u
        x -= (x + 0.05 / k * np.sin(k * x) - u) / (1 + 0.05 * np.cos(k * x))
    # TSI idiom: lower corner at dx/2, period L
    pos = np.stack([np.mod(x, L) + 0.5, rng.uniform(0.0, L, n) + 0.5])
    vel = rng.normal(0.0, 1.0, (3, n))
    phi_ext = rng.normal(0.0, 0.02, (CELLS + 1) ** 2)
    return pos, vel, phi_ext, n


def make_run(precision, pos):
    grid = P.simple_grid((0.5, 0.5), (CELLS + 0.5, CELLS + 0.5), (CELLS, CELLS))
    n = pos.shape[1]
    w = (CELLS + 1.0) ** 2 / n            # electron density 1 per unit area
    posd = torch.tensor(pos, device="cuda", dtype=torch.float64)
    return ElectrostaticRun(grid, (1, 1), [(-1.0, 1.0, w, posd)], [P.Dirichlet_nodes(grid, [(0, 0)], 0.0)], MG, DT,
                            STEPS, checkpoint_every=K, precision=precision, background=1.0)


def grads(run, vel, phi_ext, dtype):
    v = torch.tensor(vel, device="cuda", dtype=dtype, requires_grad=True)
    pe = torch.tensor(phi_ext, device="cuda", dtype=torch.float64, requires_grad=True)
    loss = ElectrostaticLoss.apply(run, pe, v)
    loss.backward()
    torch.cuda.synchronize()
    return float(loss.detach()), v.grad.double().cpu().numpy(), pe.grad.cpu().numpy()


def loss_and_cells(run, vel, phi_ext):
    """Forward loss and the cell key of every particle at every step."""
    v = torch.tensor(vel, device="cuda", dtype=torch.float64)
    pe = torch.tensor(phi_ext, device="cuda", dtype=torch.float64)
    n = vel.shape[1]
    keys = []
    with torch.cuda.stream(run.stream):
        run._load([v])
        for _ in range(run.steps):
            k = torch.empty(n, dtype=torch.int32, device="cuda")
            run.ctx.get_keys(0, k)
            keys.append(k)
            run.ctx.push(run._field(pe), run.dt)
        k = torch.empty(n, dtype=torch.int32, device="cuda")
        run.ctx.get_keys(0, k)
        keys.append(k)
        loss = run._loss(run._field(pe))
    torch.cuda.synchronize()
    return float(loss), torch.stack(keys)


def fd_probe(run, vel, phi_ext, which, idx, eps):
    """Central difference of the loss in one input component, and whether
    the two perturbed runs visit the same cells (the loss is smooth between
    them only then: the gathered field jumps across cell faces)."""
    a, b = (vel.copy(), vel.copy()) if which == "v" else (phi_ext.copy(), phi_ext.copy())
    a[idx] += eps
    b[idx] -= eps
    if which == "v":
        (lp, kp), (lm, km) = loss_and_cells(run, a, phi_ext), loss_and_cells(run, b, phi_ext)
    else:
        (lp, kp), (lm, km) = loss_and_cells(run, vel, a), loss_and_cells(run, vel, b)
    return (lp - lm) / (2 * eps), bool(torch.equal(kp, km))


def test_fp64_adjoint_matches_central_differences():
    pos, vel, phi_ext, n = landau_setup()
    run = make_run(P.FP64, pos)
    L0, gv, gp = grads(run, vel, phi_ext, torch.float64)
    assert np.isfinite(L0) and L0 > 0
    rng = np.random.default_rng(5)
    eps = 1e-3
    # the largest-gradient components plus random ones
    flat = np.abs(gv[:2]).ravel()
    probes = [("v", divmod(int(i), n)) for i in list(np.argsort(flat)[-4:]) + list(rng.integers(0, flat.size, 6))]
    probes += [("p", int(i)) for i in list(np.argsort(np.abs(gp))[-4:]) + list(rng.integers(0, gp.size, 6))]
    smooth = crossing = 0
    worst, worst_rich = 0.0, 0.0
    for which, idx in probes:
        g = gv[idx] if which == "v" else gp[idx]
        gmax = np.abs(gv).max() if which == "v" else np.abs(gp).max()
        scale = max(abs(g), 1e-2 * gmax)
        fd1, same1 = fd_probe(run, vel, phi_ext, which, idx, eps)
        fd2, same2 = fd_probe(run, vel, phi_ext, which, idx, eps / 2)
        if not (same1 and same2):
            crossing += 1   # reported, not compared
            continue
        smooth += 1
        rich = (4 * fd2 - fd1) / 3            # Richardson: removes the eps^2 term
        worst = max(worst, abs(fd1 - g) / scale)
        worst_rich = max(worst_rich, abs(rich - g) / scale)
        assert abs(fd1 - g) <= 1e-4 * scale, (which, idx, fd1, g)
        assert abs(rich - g) <= 1e-5 * scale, (which, idx, rich, g)
    print(f"finite-difference probes: {smooth} smooth (compared), {crossing} crossing a cell face; "
          f"max error {worst:.2e} (eps=1e-3), {worst_rich:.2e} (Richardson)")
    assert smooth >= len(probes) // 2


def test_mixed_adjoint_matches_fp64_adjoint():
    pos, vel, phi_ext, n = landau_setup()
    L64, gv64, gp64 = grads(make_run(P.FP64, pos), vel, phi_ext, torch.float64)
    L32, gv32, gp32 = grads(make_run(P.MIXED, pos), vel, phi_ext, torch.float32)
    assert abs(L32 - L64) <= 1e-5 * abs(L64)
    assert np.linalg.norm(gv32 - gv64) <= 1e-3 * np.linalg.norm(gv64)
    assert np.linalg.norm(gp32 - gp64) <= 1e-3 * np.linalg.norm(gp64)


def test_adjoint_repeats_bitwise():
    pos, vel, phi_ext, n = landau_setup(seed=43)
    run = make_run(P.MIXED, pos)
    a = grads(run, vel, phi_ext, torch.float32)
    b = grads(run, vel, phi_ext, torch.float32)
    assert a[0] == b[0]
    assert (a[1] == b[1]).all() and (a[2] == b[2]).all()

