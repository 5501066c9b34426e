"""ctypes binding of the FP64 CPU oracle (oracle/oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker.  The product package
(psum_b200) never imports it.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")


class GridDesc(C.Structure):
    """Same layout as psum_pic_grid_desc (include/psum_pic.h)."""
    _fields_ = [("dim", C.c_int), ("cells", C.c_int * 3), ("lower", C.c_double * 3),
                ("upper", C.c_double * 3), ("periodic", C.c_int * 3)]


def make_grid(cells, lower, upper, periodic):
    g = GridDesc()
    g.dim = len(cells)
    for a in range(3):
        g.cells[a] = int(cells[a]) if a < len(cells) else 1
        g.lower[a] = float(lower[a]) if a < len(lower) else 0.0
        g.upper[a] = float(upper[a]) if a < len(upper) else 1.0
        g.periodic[a] = int(periodic[a]) if a < len(periodic) else 0
    return g


def build():
    """Compile liboracle.so with its Makefile (no-op when up to date)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P = C.c_void_p
        d, ll, i = C.c_double, C.c_longlong, C.c_int
        L.oracle_interp.argtypes = [P, P, P, P]; L.oracle_interp.restype = i
        L.oracle_interp_diff.argtypes = [P, P, P, P]; L.oracle_interp_diff.restype = i
        L.oracle_gather_grad.argtypes = [P, ll, P, P, P]; L.oracle_gather_grad.restype = None
        L.oracle_push.argtypes = [P, ll, P, P, P, d, d, i, P, P]; L.oracle_push.restype = None
        L.oracle_deposit.argtypes = [P, ll, P, d, P]; L.oracle_deposit.restype = None
        L.oracle_bin.argtypes = [P, ll, P, P, P, P, P]; L.oracle_bin.restype = ll
        L.oracle_poisson_assemble.argtypes = [i, P, P, P, d, ll, P, P, P, P]
        L.oracle_poisson_assemble.restype = ll
        L.oracle_mg_create.argtypes = [ll, ll, P, P, P, i, i, i, i, P]; L.oracle_mg_create.restype = P
        L.oracle_mg_destroy.argtypes = [P]; L.oracle_mg_destroy.restype = None
        L.oracle_mg_levels.argtypes = [P]; L.oracle_mg_levels.restype = i
        L.oracle_mg_level_rows.argtypes = [P, i]; L.oracle_mg_level_rows.restype = ll
        L.oracle_mg_level_coo.argtypes = [P, i, P, P, P, P]; L.oracle_mg_level_coo.restype = ll
        L.oracle_mg_vcycles.argtypes = [P, P, P, i, i, i]; L.oracle_mg_vcycles.restype = None
        L.oracle_mg_solve_mixed.argtypes = [P, P, P, i, i, i, i, P]; L.oracle_mg_solve_mixed.restype = i
        L.oracle_mg_solve_mixed_tol.argtypes = [P, P, P, i, i, i, i, d, P]; L.oracle_mg_solve_mixed_tol.restype = i
        L.oracle_rel_residual.argtypes = [P, P, P]; L.oracle_rel_residual.restype = d
        L.oracle_kinetic_energy.argtypes = [ll, P, P, d]; L.oracle_kinetic_energy.restype = d
        L.oracle_field_energy.argtypes = [P, P, d]; L.oracle_field_energy.restype = d
        L.oracle_last_error.argtypes = []; L.oracle_last_error.restype = C.c_char_p
        L.oracle_bspline_support.argtypes = [P, i, P, P, P, P]; L.oracle_bspline_support.restype = i
        L.oracle_bspline_gather.argtypes = [P, i, ll, P, P, P, P, d]; L.oracle_bspline_gather.restype = None
        L.oracle_bspline_deposit.argtypes = [P, i, ll, P, d, P, d]; L.oracle_bspline_deposit.restype = ll
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def interp(grid, p):
    idx = np.zeros(8, np.int64); coef = np.zeros(8)
    n = lib().oracle_interp(C.byref(grid), _p(_f64(p)), _p(idx), _p(coef))
    return idx[:n], coef[:n]


def interp_diff(grid, p):
    idx = np.zeros(8, np.int64); dcoef = np.zeros(24)
    n = lib().oracle_interp_diff(C.byref(grid), _p(_f64(p)), _p(idx), _p(dcoef))
    return idx[:n], dcoef[:grid.dim * n].reshape(grid.dim, n)


def gather_grad(grid, pos, phi):
    pos = _f64(pos); phi = _f64(phi)
    n = pos.shape[1]
    out = np.zeros((grid.dim, n))
    lib().oracle_gather_grad(C.byref(grid), n, _p(pos), _p(phi), _p(out))
    return out


def push(grid, pos, vel, phi, q_m, dt, pusher=0, B=(0.0, 0.0, 0.0)):
    """One push; returns (new_pos, new_vel, losses[dim][2]).  pos is (dim, n), vel (3, n)."""
    pos = _f64(pos).copy(); vel = _f64(vel).copy(); phi = _f64(phi)
    n = pos.shape[1]
    Bv = _f64(B)
    losses = np.zeros(2 * grid.dim, np.uint64)
    lib().oracle_push(C.byref(grid), n, _p(pos), _p(vel), _p(phi), q_m, dt, pusher, _p(Bv), _p(losses))
    return pos, vel, losses.reshape(grid.dim, 2)


def deposit(grid, pos, w, n_nodes):
    pos = _f64(pos)
    rho = np.zeros(n_nodes)
    lib().oracle_deposit(C.byref(grid), pos.shape[1], _p(pos), w, _p(rho))
    return rho


def bspline_support(grid, order, p):
    """(node indices, weights, derivative weights (dim, S^D)) of one point at
    B-spline order 1-4; empty arrays when the point has no support."""
    m = (order + 1) ** grid.dim
    idx = np.zeros(m, np.int64); coef = np.zeros(m); dcoef = np.zeros(grid.dim * m)
    k = lib().oracle_bspline_support(C.byref(grid), order, _p(_f64(p)), _p(idx), _p(coef), _p(dcoef))
    return idx[:k], coef[:k], dcoef[:grid.dim * k].reshape(grid.dim, k)


def bspline_gather(grid, order, pos, field, grad=False, tol=1e-10):
    """interp_B_spline / interp_diff_B_spline at (dim, n) positions; tol is the
    weight skip threshold (1e-10 in the reference, 0 for the full sum)."""
    pos = _f64(pos); field = _f64(field)
    n = pos.shape[1]
    if grad:
        out = np.zeros((grid.dim, n))
        lib().oracle_bspline_gather(C.byref(grid), order, n, _p(pos), _p(field), None, _p(out), tol)
    else:
        out = np.zeros(n)
        lib().oracle_bspline_gather(C.byref(grid), order, n, _p(pos), _p(field), _p(out), None, tol)
    return out


def bspline_deposit(grid, order, pos, w, n_nodes, tol=1e-10):
    """add_back_B_spline of (dim, n) positions with weight w into a zero field."""
    pos = _f64(pos)
    field = np.zeros(n_nodes)
    skipped = lib().oracle_bspline_deposit(C.byref(grid), order, pos.shape[1], _p(pos), w, _p(field), tol)
    return field, skipped


def bin_particles(grid, pos):
    pos = _f64(pos)
    n = pos.shape[1]
    ncell = int(np.prod([grid.cells[a] for a in range(grid.dim)]))
    keys = np.zeros(n, np.int64)
    counts = np.zeros(ncell, np.uint64); offsets = np.zeros(ncell, np.uint64)
    perm = np.zeros(n, np.uint64)
    m = lib().oracle_bin(C.byref(grid), n, _p(pos), _p(keys), _p(counts), _p(offsets), _p(perm))
    return keys, counts, offsets, perm[:m]


def poisson_assemble(cells, lower, upper, eps, fixed_nodes):
    dim = len(cells)
    c = np.array(list(cells) + [1] * (3 - dim), np.int32)
    lo = _f64(list(lower) + [0.0] * (3 - dim)); hi = _f64(list(upper) + [1.0] * (3 - dim))
    fx = np.ascontiguousarray(fixed_nodes, np.uint64)
    L = lib()
    nnz = L.oracle_poisson_assemble(dim, _p(c), _p(lo), _p(hi), eps, fx.size, _p(fx), None, None, None)
    rows = np.zeros(nnz, np.uint64); cols = np.zeros(nnz, np.uint64); vals = np.zeros(nnz)
    L.oracle_poisson_assemble(dim, _p(c), _p(lo), _p(hi), eps, fx.size, _p(fx), _p(rows), _p(cols), _p(vals))
    return rows, cols, vals


class Multigrid:
    """FP64 multigrid_core restatement; dims are node counts (I, J, K)."""

    def __init__(self, rows, cols, vals, n, I, J, K, depth, periodic=(0, 0, 0)):
        self._r = np.ascontiguousarray(rows, np.uint64)
        self._c = np.ascontiguousarray(cols, np.uint64)
        self._v = _f64(vals)
        self.n = n
        per = np.ascontiguousarray(periodic, np.int32)
        self.h = lib().oracle_mg_create(n, self._r.size, _p(self._r), _p(self._c), _p(self._v), I, J, K, depth,
                                        _p(per))
        if not self.h:
            raise RuntimeError(lib().oracle_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_mg_destroy(self.h)
            self.h = None

    @property
    def levels(self):
        return lib().oracle_mg_levels(self.h)

    def level_rows(self, l):
        return lib().oracle_mg_level_rows(self.h, l)

    def level_coo(self, l):
        L = lib()
        nnz = L.oracle_mg_level_coo(self.h, l, None, None, None, None)
        rows = np.zeros(nnz, np.uint64); cols = np.zeros(nnz, np.uint64); vals = np.zeros(nnz)
        dinv = np.zeros(self.level_rows(l))
        L.oracle_mg_level_coo(self.h, l, _p(rows), _p(cols), _p(vals), _p(dinv))
        return rows, cols, vals, dinv

    def vcycles(self, b, x0, cycles, pre=2, post=1):
        x = _f64(x0).copy()
        lib().oracle_mg_vcycles(self.h, _p(_f64(b)), _p(x), cycles, pre, post)
        return x

    def solve_mixed(self, b, x0, max_cycles=10, correction_interval=4, pre=2, post=1):
        x = _f64(x0).copy()
        hist = np.zeros(max(max_cycles, 1))
        nb = lib().oracle_mg_solve_mixed(self.h, _p(_f64(b)), _p(x), max_cycles, correction_interval, pre, post,
                                         _p(hist))
        return x, hist[:nb]

    def solve_mixed_tol(self, b, x0, max_cycles, correction_interval, pre, post, tol):
        """solve_mixed stopping after the first batch with relative residual <= tol (the GPU backends' rule)."""
        x = _f64(x0).copy()
        hist = np.zeros(max(max_cycles, 1))
        nb = lib().oracle_mg_solve_mixed_tol(self.h, _p(_f64(b)), _p(x), max_cycles, correction_interval, pre, post,
                                             tol, _p(hist))
        return x, hist[:nb]

    def rel_residual(self, b, x):
        return lib().oracle_rel_residual(self.h, _p(_f64(b)), _p(_f64(x)))


def kinetic_energy(pos, vel, mass_times_weight):
    pos = _f64(pos); vel = _f64(vel)
    return lib().oracle_kinetic_energy(pos.shape[1], _p(pos), _p(vel), mass_times_weight)


def field_energy(grid, phi, eps):
    return lib().oracle_field_energy(C.byref(grid), _p(_f64(phi)), eps)
