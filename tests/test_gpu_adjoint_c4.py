"""The adjoint at the differentiable workload's own shape: 256 x 256 wrapping
nodes (255 cells), 64 electrons per cell (4,194,304 particles), a 5% mode-1
Landau perturbation, leapfrog, checkpoints every 10 steps.

The discrete map is only piecewise smooth: the CIC gradient jumps across cell
faces, so a perturbation that moves any particle's face crossing by a step
adds a jump the adjoint (the derivative inside the cells) does not contain.
Over one checkpoint segment (10 steps) central differences with eps = 1e-3
stay on one smooth piece for most probes, and the FP64 adjoint must agree
with them to 1e-4 (probes whose perturbed runs change a cell sequence are
counted, not compared); the mixed adjoint too, against the FP64 forward's
differences.  The differences' O(eps^2) truncation reaches about 1e-4 on the
largest components (measured 1.1e-4): a probe above the bound is compared
through the Richardson value of eps and eps / 2, after checking that halving
eps moves the difference towards the adjoint.  Over the full 100 steps the perturbed runs of eps = 1e-3 change
thousands of crossings (measured: differences far from any derivative), so
the full run is checked for the consistency of its two adjoints (loss to
1e-5, gradients to 5e-3 relative L2, measured 2e-3), and its velocity probes
against differences at eps = 1e-5, which keep the probe's own cells and are
noise-limited (bound 1e-2 of the gradient scale, measured up to 5e-3).  All
errors are relative to the gradient's scale, its largest component."""
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


def _probe_fd(run64, vel, phi_ext, gv64, gp64, gv32, gp32, n, eps, nv, npot, seed, tol64, tol32, only_v=False):
    rng = np.random.default_rng(seed)
    flat = np.abs(gv64[:2]).ravel()
    probes = [("v", divmod(int(i), n)) for i in list(np.argsort(flat)[-nv // 2:]) + list(rng.integers(0, flat.size, nv - nv // 2))]
    if not only_v:
        probes += [("p", int(i)) for i in list(np.argsort(np.abs(gp64))[-npot // 2:])
                   + list(rng.integers(0, gp64.size, npot - npot // 2))]
    smooth = crossing = 0
    worst64 = worst32 = 0.0
    for which, idx in probes:
        g64 = gv64[idx] if which == "v" else gp64[idx]
        g32 = gv32[idx] if which == "v" else gp32[idx]
        # errors relative to the gradient's scale (its largest component): the differences carry an absolute
        # noise floor of about 5e-7 from the loss's rounding, so small components are not compared relatively
        scale = np.abs(gv64).max() if which == "v" else np.abs(gp64).max()
        d, same = fd(run64, vel, phi_ext, which, idx, eps)
        if not same:
            crossing += 1
            continue
        smooth += 1
        e64, e32 = abs(d - g64), abs(d - g32)
        if max(e64 - tol64 * scale, e32 - tol32 * scale) > 0:
            # above the bound: the central difference's own O(eps^2) truncation must be what is left, i.e. the
            # difference at eps / 2 moves towards the adjoint (by 4x without noise; at least 2x asked) and the
            # Richardson value (4 D(eps/2) - D(eps)) / 3 is within the bound
            dh, same_h = fd(run64, vel, phi_ext, which, idx, eps / 2)
            assert same_h
            rich = (4 * dh - d) / 3
            print(f"probe {which} {idx}: D(eps) {d:.9e}, D(eps/2) {dh:.9e}, Richardson {rich:.9e}, "
                  f"FP64 adjoint {g64:.9e}, mixed {g32:.9e}")
            assert abs(dh - g64) <= 0.5 * e64 or abs(dh - g64) <= tol64 * scale, (which, idx, d, dh, g64)
            e64, e32 = abs(rich - g64), abs(rich - g32)
        worst64 = max(worst64, e64 / scale)
        worst32 = max(worst32, e32 / scale)
        assert e64 <= tol64 * scale, (which, idx, d, g64)
        assert e32 <= tol32 * scale, (which, idx, d, g32)
    return smooth, crossing, worst64, worst32


def test_adjoint_matches_finite_differences_over_one_segment():
    """C4 grid and particles, one checkpoint segment (10 steps): both adjoints within 1e-4 of the FP64 forward's
    central differences (eps = 1e-3) on the smooth probes."""
    global STEPS
    steps_full = STEPS
    STEPS = K
    try:
        pos, vel, phi_ext, n = setup()
        posd = torch.tensor(pos, device="cuda", dtype=torch.float64)
        run64 = make_run(P.FP64, posd)
        L64, gv64, gp64 = grads(run64, vel, phi_ext, torch.float64)
        L32, gv32, gp32 = grads(make_run(P.MIXED, posd), vel, phi_ext, torch.float32)
        assert abs(L32 - L64) <= 1e-5 * abs(L64)
        smooth, crossing, w64, w32 = _probe_fd(run64, vel, phi_ext, gv64, gp64, gv32, gp32, n, 1e-3, 6, 6, 7,
                                               1e-4, 1e-4)
        print(f"10 steps: {smooth} smooth probes, {crossing} crossing a cell face; FP64 adjoint vs FD {w64:.2e}, "
              f"mixed adjoint vs FD {w32:.2e}")
        assert smooth >= 8
    finally:
        STEPS = steps_full


def test_adjoints_over_the_full_run():
    """C4 as specified (100 steps, checkpoints every 10): the mixed and FP64 adjoints agree, and the velocity
    probes agree with noise-limited central differences at eps = 1e-5."""
    pos, vel, phi_ext, n = setup()
    posd = torch.tensor(pos, device="cuda", dtype=torch.float64)
    run64 = make_run(P.FP64, posd)
    L64, gv64, gp64 = grads(run64, vel, phi_ext, torch.float64)
    L32, gv32, gp32 = grads(make_run(P.MIXED, posd), vel, phi_ext, torch.float32)
    assert np.isfinite(L64) and L64 > 0
    assert abs(L32 - L64) <= 1e-5 * abs(L64)
    rv = np.linalg.norm(gv32 - gv64) / np.linalg.norm(gv64)
    rp = np.linalg.norm(gp32 - gp64) / np.linalg.norm(gp64)
    assert rv <= 5e-3 and rp <= 5e-3, (rv, rp)
    smooth, crossing, w64, w32 = _probe_fd(run64, vel, phi_ext, gv64, gp64, gv32, gp32, n, 1e-5, 4, 0, 7,
                                           1e-2, 1e-2, only_v=True)
    print(f"100 steps: mixed vs FP64 adjoint {rv:.2e} (velocities), {rp:.2e} (potential); {smooth} velocity probes "
          f"at eps 1e-5 within {w64:.2e} (FP64) / {w32:.2e} (mixed), {crossing} crossing")
    assert smooth >= 2
