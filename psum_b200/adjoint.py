"""Differentiable electrostatic PIC runs (the adjoint of the step).

``ElectrostaticRun`` holds one run: a particle context (no re-sorting, so
particles keep their order and per-particle adjoints stay aligned), the
Poisson solver for A (with PSuM's source fix-ups) and a second solver for
A^T, the fixed initial positions of every species, dt, the number of steps
and the checkpoint interval.  ``ElectrostaticLoss`` is a
``torch.autograd.Function`` mapping (external potential, initial velocities
of every species) to the loss at the final step,

    L = sum over grid edges of ((phi(n + e_a) - phi(n)) / dx_a)^2,
    phi = S rho(s) + phi_ext        (S: the Poisson solve with its fix-ups),

and its backward pass runs the hand-written adjoint kernels of the library
backwards over the steps: the adjoint of the gather is a scatter
(``adjoint_push``), the adjoint of the deposit is a gather
(``adjoint_deposit``) and the adjoint of the Poisson solve reuses the
multigrid: with the fixed-node rows of A replaced by identity rows and their
right-hand sides by the fixed values, the linear part of the solve is
S = E L0^-1 E^T (L0: the operator on the free nodes, E: their embedding), so
S^T = S whenever L0 is symmetric, which PSuM's Cartesian operator is; the
adjoint solve is then the forward solve with zero fixed values.  The forward keeps a device snapshot of the state every K steps; the
backward recomputes each segment of K steps from its snapshot.  Every solve
starts from a zero guess, so a recomputed step repeats the forward bits.

PSuM has no adjoint; this layer is new.
"""
import numpy as np
import torch

from . import field_solver as _fs
from .pic import MIXED, ParticleContext


def field_energy_loss(phi, shape, dx, periodic):
    """sum over edges ((phi(n + e_a) - phi(n)) / dx_a)^2 on the node lattice
    (wrapping edges on periodic axes)."""
    p = phi.view(*shape)
    total = phi.new_zeros(())
    for a in range(len(shape)):
        if periodic[a]:
            d = torch.roll(p, -1, dims=a) - p
        else:
            d = p.narrow(a, 1, shape[a] - 1) - p.narrow(a, 0, shape[a] - 1)
        total = total + (d / dx[a]).pow(2).sum()
    return total


def check_free_block_symmetric(rows, cols, vals, fixed, n, rtol=1e-12):
    """Raises unless the operator restricted to the free (not fixed) nodes is
    symmetric, the condition under which the adjoint solve is the forward solve."""
    import scipy.sparse as sp
    free = np.ones(n, bool)
    free[np.asarray(fixed, np.int64)] = False
    r, c = rows.astype(np.int64), cols.astype(np.int64)
    keep = free[r] & free[c]
    A = sp.csr_matrix((vals[keep], (r[keep], c[keep])), shape=(n, n))
    d = abs(A - A.T)
    scale = abs(A).max() if A.nnz else 1.0
    if d.nnz and d.max() > rtol * scale:
        raise NotImplementedError("adjoint solve: the operator on the free nodes is not symmetric")


class ElectrostaticRun:
    """One differentiable run.

    species: list of (charge, mass, weight, positions) with positions a
    (dim, n) float64 CUDA tensor (absolute coordinates, the same at every
    forward); velocities are the differentiable input."""

    def __init__(self, grid, periodic, species, fixed_boundaries, mg_options, dt, steps, checkpoint_every=10,
                 precision=MIXED, epsilon=1.0, background=0.0):
        self.grid = grid
        self.dim = grid.dim
        self.periodic = tuple(int(bool(p)) for p in periodic)
        self.precision = precision
        self.dt = float(dt)
        self.steps = int(steps)
        self.K = int(checkpoint_every)
        self.background = float(background)
        self.shape = tuple(c + 1 for c in grid.cells)
        self.dx = tuple(grid.delta)
        self.n_nodes = int(np.prod(self.shape))
        # one stream orders all work of the run: context, solves and torch ops
        self.stream = torch.cuda.Stream()
        self.ctx = ParticleContext(grid.cells, grid.lower, grid.upper, self.periodic, precision)
        self.ctx.set_options("sort_interval 0")
        self.ctx.set_stream(self.stream)
        self.species = []
        for q, m, w, pos in species:
            n = pos.shape[1]
            sid = self.ctx.add_species(q, m, w, n)
            self.species.append((sid, pos.contiguous(), n))
        backend = "cuda_multigrid32f_gpu" if precision == MIXED else "cuda_multigrid64_gpu"
        frontend = _fs.Poisson_solver_2d() if self.dim == 2 else _fs.Poisson_solver_3d()
        frontend.set_options(mg_options)
        frontend.init(backend, grid, frontend.Cartesian, fixed_boundaries, epsilon)
        frontend.make_righthand_item()
        self.solver = frontend
        rows, cols, vals = frontend.coeff_matrix()
        check_free_block_symmetric(rows, cols, vals, frontend.replace_idx, self.n_nodes)
        # the adjoint solve: the same operator, fixed values zero
        self.solver_t = _fs.solver_backend(backend)
        self.solver_t.set_options(mg_options)
        self.solver_t.set_matrix(self.n_nodes, self.n_nodes, rows.size, rows, cols, vals)
        self.solver_t.set_source_replace(frontend.replace_idx, np.zeros(frontend.replace_idx.size))
        dev = torch.device("cuda", torch.cuda.current_device())
        self.replace_idx = torch.as_tensor(frontend.replace_idx.astype(np.int64), device=dev)
        self.adj_dtype = torch.float32 if precision == MIXED else torch.float64
        self.dev = dev
        # persistent solve buffers: the solvers replay one captured graph per (b, x)
        self._b = torch.zeros(self.n_nodes, dtype=torch.float64, device=dev)
        self._x = torch.zeros(self.n_nodes, dtype=torch.float64, device=dev)
        self._bt = torch.zeros_like(self._b)
        self._xt = torch.zeros_like(self._x)
        self.state_bytes = [self.ctx.state_bytes(sid) for sid, _, _ in self.species]

    # -------------------------------------------------------------- pieces --
    def _load(self, v0s):
        for (sid, pos, n), v in zip(self.species, v0s):
            self.ctx.load(sid, pos, v.to(torch.float64).contiguous())
        self.ctx.deposit()

    def _save(self):
        snaps = []
        for (sid, _, _), nb in zip(self.species, self.state_bytes):
            buf = torch.empty(nb, dtype=torch.uint8, device=self.dev)
            self.ctx.save_state(sid, buf)
            snaps.append(buf)
        return snaps

    def _restore(self, snaps, deposit=True):
        for (sid, _, _), buf in zip(self.species, snaps):
            self.ctx.restore_state(sid, buf)
        if deposit:
            self.ctx.deposit()

    def _field(self, phi_ext):
        """phi = S rho(current state) + phi_ext (zero initial guess)."""
        self.ctx.rho(self.background, self._b)
        self._x.zero_()
        self.solver.backend.solve_async(self._b, self._x, self.stream)
        return self._x + phi_ext

    def _solve_t(self, mu):
        """nu = S^T mu = S mu: the forward solve with the fixed values zero."""
        self._bt.copy_(mu)
        self._xt.zero_()
        self.solver_t.solve_async(self._bt, self._xt, self.stream)
        return self._xt.clone()

    def _loss(self, phi):
        return field_energy_loss(phi, self.shape, self.dx, self.periodic)

    # ------------------------------------------------------------- forward --
    def forward(self, phi_ext, v0s, keep=False):
        """Runs the steps; returns the loss (and the snapshots when keep)."""
        caller = torch.cuda.current_stream()
        self.stream.wait_stream(caller)
        with torch.cuda.stream(self.stream):
            out = self._forward(phi_ext, v0s, keep)
        caller.wait_stream(self.stream)
        return out

    def _forward(self, phi_ext, v0s, keep):
        phi_ext = phi_ext.to(torch.float64).contiguous()
        self._load(v0s)
        ckpts = []
        for n in range(self.steps):
            if keep and n % self.K == 0:
                ckpts.append(self._save())
            phi = self._field(phi_ext)
            self.ctx.push(phi, self.dt)
        final = self._save() if keep else None
        loss = self._loss(self._field(phi_ext))
        return (loss, ckpts, final) if keep else loss

    # ------------------------------------------------------------ backward --
    def backward(self, phi_ext, ckpts, final, grad_loss):
        """Gradients of grad_loss * L with respect to phi_ext and the initial
        velocities of every species."""
        caller = torch.cuda.current_stream()
        self.stream.wait_stream(caller)
        with torch.cuda.stream(self.stream):
            out = self._backward(phi_ext, ckpts, final, grad_loss)
        caller.wait_stream(self.stream)
        return out

    def _backward(self, phi_ext, ckpts, final, grad_loss):
        phi_ext = phi_ext.to(torch.float64).contiguous()
        # final step: L(phi_N), phi_N = S rho(s_N) + phi_ext
        self._restore(final)
        phi_n = self._field(phi_ext).requires_grad_(True)
        with torch.enable_grad():
            g = torch.autograd.grad(self._loss(phi_n), phi_n)[0]
        g = (g * grad_loss).detach().contiguous()
        lam_phi = g.clone()
        nu = self._solve_t(g)
        lam_x, lam_v = [], []
        for sid, _, n in self.species:
            lx = torch.zeros(self.dim, n, dtype=self.adj_dtype, device=self.dev)
            lv = torch.zeros(3, n, dtype=self.adj_dtype, device=self.dev)
            self.ctx.adjoint_deposit(sid, nu, lx)
            lam_x.append(lx)
            lam_v.append(lv)
        # segments of K steps, last first, recomputed from their snapshots
        for j in reversed(range(len(ckpts))):
            start, end = j * self.K, min(j * self.K + self.K, self.steps)
            self._restore(ckpts[j])
            states, phis = [], []
            for _ in range(start, end):
                states.append(self._save())
                phi = self._field(phi_ext)
                phis.append(phi)
                self.ctx.push(phi, self.dt)
            for k in reversed(range(end - start)):
                self._restore(states[k], deposit=False)
                mu = torch.zeros(self.n_nodes, dtype=torch.float64, device=self.dev)
                for (sid, _, _), lx, lv in zip(self.species, lam_x, lam_v):
                    self.ctx.adjoint_push(sid, phis[k], self.dt, lx, lv, mu)
                lam_phi += mu
                nu = self._solve_t(mu)
                for (sid, _, _), lx in zip(self.species, lam_x):
                    self.ctx.adjoint_deposit(sid, nu, lx)
        st = self.solver_t.last_stats()   # the last adjoint solve (synchronises)
        if not np.isfinite(st["rel_residual"]) or st["rel_residual"] > 1e-6:
            raise RuntimeError(f"adjoint solve did not converge: {st}")
        return lam_phi, lam_v


class ElectrostaticLoss(torch.autograd.Function):
    """loss = ElectrostaticLoss.apply(run, phi_ext, v0_species0, v0_species1, ...)"""

    @staticmethod
    def forward(fctx, run, phi_ext, *v0s):
        loss, ckpts, final = run.forward(phi_ext.detach(), [v.detach() for v in v0s], keep=True)
        fctx.run = run
        fctx.ckpts = ckpts
        fctx.final = final
        fctx.dtypes = [v.dtype for v in v0s]
        fctx.phi_dtype = phi_ext.dtype
        fctx.save_for_backward(phi_ext.detach())
        return loss

    @staticmethod
    def backward(fctx, grad_loss):
        (phi_ext,) = fctx.saved_tensors
        lam_phi, lam_v = fctx.run.backward(phi_ext, fctx.ckpts, fctx.final, float(grad_loss))
        fctx.ckpts = None
        fctx.final = None
        return (None, lam_phi.to(fctx.phi_dtype), *[lv.to(dt) for lv, dt in zip(lam_v, fctx.dtypes)])
