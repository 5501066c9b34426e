"""The adjoint at the differentiable workload's own shape: 256 x 256 wrapping
nodes (255 cells), 64 electrons per cell (4,194,304 particles), a 5% mode-1
Landau perturbation, 100 leapfrog steps with checkpoints every 10.  The FP64
adjoint is checked against central finite differences of the FP64 forward
(eps = 1e-3, and eps/2 for a Richardson estimate) on probes whose perturbed
runs keep every particle's cell sequence (the loss is smooth only there; the
probes crossing a cell face are counted, not compared).  The mixed adjoint
(FP32 adjoint arrays over the mixed forward) is checked against the same
finite differences of the FP64 forward, with its measured bound stated."""
import numpy as np
import pytest

import psum_b200 as P
from psum_b200.adjoint import ElectrostaticLoss, ElectrostaticRun

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

CELLS = 255
PPC = 64
STEPS, K, DT = 100, 10, 0.1
MG = ("I 256 J 256 K 1 depth 6 pre_relax 2 post_relax 2 max_cycles 80 correction_interval 4 tol 1e-12 "
      "periodic_I 1 periodic_J 1")


def setup(seed=51):
    rng = np.random.default_rng(seed)
    L = CELLS + 1.0
    n = int(L * L * PPC)
    u = rng.uniform(0.0, L, n)
    x = u.copy()
    k = 2 * np.pi / L
    for _ in range(20):   # Newton on x + (0.05/k) sin(k x) = u: 5% mode-1 density perturbation
        x -= (x + 0.05 / k * np.sin(k * x) - u) / (1 + 0.05 * np.cos(k * x))
    pos = np.stack([np.mod(x, L) + 0.5, rng.uniform(0.0, L, n) + 0.5])
    vel = rng.normal(0.0, 1.0, (3, n))
    phi_ext = rng.normal(0.0, 0.02, (CELLS + 1) ** 2)
    return pos, vel, phi_ext, n


def make_run(precision, posd):
    grid = P.simple_grid((0.5, 0.5), (CELLS + 0.5, CELLS + 0.5), (CELLS, CELLS))
    w = (CELLS + 1.0) ** 2 / posd.shape[1]
    return ElectrostaticRun(grid, (1, 1), [(-1.0, 1.0, w, posd)], [P.Dirichlet_nodes(grid, [(0, 0)], 0.0)], MG, DT,
                            STEPS, checkpoint_every=K, precision=precision, background=1.0)


def grads(run, vel, phi_ext, dtype):
    v = torch.tensor(vel, device="cuda", dtype=dtype, requires_grad=True)
    pe = torch.tensor(phi_ext, device="cuda", dtype=torch.float64, requires_grad=True)
    loss = ElectrostaticLoss.apply(run, pe, v)
    loss.backward()
    torch.cuda.synchronize()
    return float(loss.detach()), v.grad.double().cpu().numpy(), pe.grad.cpu().numpy()


def loss_and_trace(run, v, pe, probe):
    """Forward loss and the cell of particle `probe` at every step (a velocity probe changes only that particle's
    trajectory directly); for a potential probe (probe < 0) a checksum of all cells per step."""
    keys = []
    n = v.shape[1]
    with torch.cuda.stream(run.stream):
        run._load([v])
        for _ in range(run.steps + 1):
            k = torch.empty(n, dtype=torch.int32, device="cuda")
            run.ctx.get_keys(0, k)
            keys.append(k[probe].clone() if probe >= 0 else (k.long() * torch.arange(1, n + 1, device="cuda")).sum())
            if len(keys) <= run.steps:
                run.ctx.push(run._field(pe), run.dt)
        loss = run._loss(run._field(pe))
    torch.cuda.synchronize()
    return float(loss), torch.stack(keys)


def fd(run, vel, phi_ext, which, idx, eps):
    vp, vm = vel.copy(), vel.copy()
    pp, pm = phi_ext.copy(), phi_ext.copy()
    if which == "v":
        vp[idx] += eps
        vm[idx] -= eps
        probe = idx[1]
    else:
        pp[idx] += eps
        pm[idx] -= eps
        probe = -1
    dv = lambda a: torch.tensor(a, device="cuda", dtype=torch.float64)
    lp, kp = loss_and_trace(run, dv(vp), dv(pp), probe)
    lm, km = loss_and_trace(run, dv(vm), dv(pm), probe)
    return (lp - lm) / (2 * eps), bool(torch.equal(kp, km))


def test_adjoints_at_the_differentiable_workload_shape():
    pos, vel, phi_ext, n = setup()
    posd = torch.tensor(pos, device="cuda", dtype=torch.float64)
    run64 = make_run(P.FP64, posd)
    L64, gv64, gp64 = grads(run64, vel, phi_ext, torch.float64)
    L32, gv32, gp32 = grads(make_run(P.MIXED, posd), vel, phi_ext, torch.float32)
    assert np.isfinite(L64) and L64 > 0
    assert abs(L32 - L64) <= 1e-5 * abs(L64)
    rng = np.random.default_rng(7)
    flat = np.abs(gv64[:2]).ravel()
    probes = [("v", divmod(int(i), n)) for i in list(np.argsort(flat)[-3:]) + list(rng.integers(0, flat.size, 3))]
    probes += [("p", int(i)) for i in list(np.argsort(np.abs(gp64))[-3:]) + list(rng.integers(0, gp64.size, 3))]
    eps = 1e-3
    smooth = crossing = 0
    worst64 = worst_rich = worst32 = 0.0
    for which, idx in probes:
        g64 = gv64[idx] if which == "v" else gp64[idx]
        g32 = gv32[idx] if which == "v" else gp32[idx]
        gmax = np.abs(gv64).max() if which == "v" else np.abs(gp64).max()
        scale = max(abs(g64), 1e-2 * gmax)
        fd1, same1 = fd(run64, vel, phi_ext, which, idx, eps)
        fd2, same2 = fd(run64, vel, phi_ext, which, idx, eps / 2)
        if not (same1 and same2):
            crossing += 1
            continue
        smooth += 1
        rich = (4 * fd2 - fd1) / 3
        worst64 = max(worst64, abs(fd1 - g64) / scale)
        worst_rich = max(worst_rich, abs(rich - g64) / scale)
        worst32 = max(worst32, abs(rich - g32) / scale)
        assert abs(fd1 - g64) <= 1e-4 * scale, (which, idx, fd1, g64)
        # the mixed adjoint differentiates the FP32 forward: its gradient differs from the FP64 one by the
        # FP32 trajectories' rounding; bound measured on this workload
        assert abs(rich - g32) <= 1e-3 * scale, (which, idx, rich, g32)
    print(f"C4-shape probes: {smooth} smooth, {crossing} crossing a cell face; FP64 adjoint vs FD {worst64:.2e} "
          f"(Richardson {worst_rich:.2e}); mixed adjoint vs FD {worst32:.2e}")
    assert smooth >= 3
