"""Host-side mirror of PSuM's field-solver interface over the B200 backend.

* ``solver_backend`` mirrors ``psum::field_solver::solver_backend``
  (src/field_solver/backend.hpp:11-107): a move-only owner of a backend handle
  obtained by name from the plugin registry, with the same seven operations.
* ``Poisson_solver_2d`` / ``Poisson_solver_3d`` mirror the FD frontends
  (src/field_solver/Poisson_solver_2d.hpp:22-411, Poisson_solver_3d.hpp:21-...)
  for Cartesian grids with uniform epsilon and Dirichlet boundaries: ``init``
  assembles the operator (bit-identical values, psum_poisson_assemble),
  creates the backend, replays the cached options and calls ``set_matrix``;
  ``solve(phi, rho)`` sets the Dirichlet values with ``set_source_replace``
  and solves on device buffers, overwriting ``rho`` like PSuM does.
* ``Dirichlet_line`` / ``Dirichlet_plane`` / ``Dirichlet_nodes`` mirror the
  boundary creators of src/field_solver/boundary_creator/Dirichlet.hpp.

Device buffers are torch CUDA float64 tensors (or raw device addresses).
Errors raise ``PsumError`` (a RuntimeError), as PSuM's frontends rethrow.
"""
import ctypes as C

import numpy as np

from ._lib import PsumError, check, lib

__all__ = ["simple_grid", "solver_backend", "Poisson_solver_2d", "Poisson_solver_3d", "Dirichlet_line",
           "Dirichlet_plane", "Dirichlet_nodes", "assemble_poisson", "registered_table"]


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def _ready(*tensors):
    """Order torch's producer work before the library reads or writes these
    tensors: the library enqueues on its own stream, torch on its current
    stream, and CUDA orders two streams only when told to."""
    for t in tensors:
        if getattr(t, "is_cuda", False):
            import torch
            torch.cuda.current_stream(t.device).synchronize()
            return


def _stream_handle(stream):
    """cudaStream_t value for a torch stream / int; torch's default stream
    (handle 0) maps to cudaStreamLegacy (1), since NULL means 'own stream'."""
    if stream is None:
        return None
    h = stream if isinstance(stream, int) else stream.cuda_stream
    return h if h != 0 else 1


class simple_grid:
    """Node/cell indexing of ``simple_grid<D>`` (src/field/simple_grid.hpp:16-198)."""

    def __init__(self, lower, upper, cells):
        self.dim = len(cells)
        self.lower = [float(v) for v in lower]
        self.upper = [float(v) for v in upper]
        self.cells = [int(v) for v in cells]
        self.delta = [(u - l) / c for l, u, c in zip(self.lower, self.upper, self.cells)]

    def n2i(self, *node):
        ans = node[0]
        for a in range(1, self.dim):
            ans = ans * (self.cells[a] + 1) + node[a]
        return ans

    @property
    def n_nodes(self):
        return int(np.prod([c + 1 for c in self.cells]))

    def node_dims(self):
        return tuple(c + 1 for c in self.cells)


def Dirichlet_line(grid, direction, value):
    """Nodes of one boundary line of a 2-D grid (Dirichlet.hpp:58-99): S/N fix
    j = 0 / j = J, W/E fix i = 0 / i = I."""
    I, J = grid.cells
    if direction == "S":
        idx = [grid.n2i(i, 0) for i in range(I + 1)]
    elif direction == "N":
        idx = [grid.n2i(i, J) for i in range(I + 1)]
    elif direction == "W":
        idx = [grid.n2i(0, j) for j in range(J + 1)]
    elif direction == "E":
        idx = [grid.n2i(I, j) for j in range(J + 1)]
    else:
        raise ValueError("direction must be one of N, S, E, W")
    return np.asarray(idx, np.uint64), np.full(len(idx), float(value))


def Dirichlet_plane(grid, direction, value):
    """Nodes of one boundary plane of a 3-D grid (Dirichlet.hpp:139-186):
    Xneg/Xpos fix i = 0 / I, Yneg/Ypos j, Zneg/Zpos k."""
    I, J, K = grid.cells
    rng = {"X": range(I + 1), "Y": range(J + 1), "Z": range(K + 1)}
    axis, side = direction[0], direction[1:]
    fixed = {"X": I, "Y": J, "Z": K}[axis] if side == "pos" else 0
    ii = [fixed] if axis == "X" else rng["X"]
    jj = [fixed] if axis == "Y" else rng["Y"]
    kk = [fixed] if axis == "Z" else rng["Z"]
    idx = [grid.n2i(i, j, k) for i in ii for j in jj for k in kk]
    return np.asarray(idx, np.uint64), np.full(len(idx), float(value))


def Dirichlet_nodes(grid, nodes, value):
    """Fixed value on explicit node tuples (e.g. the pinned node that makes a
    periodic operator non-singular, application/benchmark/TSI/main.cpp:106-113)."""
    idx = [grid.n2i(*n) for n in nodes]
    return np.asarray(idx, np.uint64), np.full(len(idx), float(value))


def _merge_fixed(fixed_boundaries):
    """Later entries win for nodes listed twice (an unordered map keyed by node)."""
    table = {}
    for idx, val in fixed_boundaries:
        for i, v in zip(np.asarray(idx, np.uint64).tolist(), np.asarray(val, np.float64).tolist()):
            table[i] = v
    keys = np.fromiter(table.keys(), np.uint64, len(table))
    vals = np.fromiter(table.values(), np.float64, len(table))
    order = np.argsort(keys)
    return keys[order], vals[order]


def assemble_poisson(grid, fixed_nodes, epsilon):
    """COO (rows, cols, vals) of the FD operator, column-major like PSuM's frontend."""
    L = lib()
    cells = np.array(grid.cells + [1] * (3 - grid.dim), np.int32)
    lo = np.array(grid.lower + [0.0] * (3 - grid.dim))
    hi = np.array(grid.upper + [1.0] * (3 - grid.dim))
    fx = np.ascontiguousarray(fixed_nodes, np.uint64)
    nnz = C.c_ulonglong(0)
    check(L.psum_poisson_assemble(grid.dim, _ptr(cells), _ptr(lo), _ptr(hi), float(epsilon), fx.size,
                                  _ptr(fx) if fx.size else None, C.byref(nnz), None, None, None))
    rows = np.zeros(nnz.value, np.uint64)
    cols = np.zeros(nnz.value, np.uint64)
    vals = np.zeros(nnz.value)
    check(L.psum_poisson_assemble(grid.dim, _ptr(cells), _ptr(lo), _ptr(hi), float(epsilon), fx.size,
                                  _ptr(fx) if fx.size else None, C.byref(nnz), _ptr(rows), _ptr(cols), _ptr(vals)))
    return rows, cols, vals


def registered_table(name):
    """The raw ``func_table`` registered under ``name`` (init is NULL when unknown)."""
    return lib().get_solver_funcs(name.encode())


class solver_backend:
    """Owner of one backend handle (backend.hpp:11-107).  Uses the
    status-returning psum_mg_* mirrors of the func_table entries, so errors
    surface as PsumError instead of C++ exceptions."""

    def __init__(self, kind=None):
        self.handle = None
        self.kind = kind
        if kind is None:
            return
        h = C.c_void_p()
        check(lib().psum_mg_create(kind.encode(), C.byref(h)))
        self.handle = h

    def is_null(self):
        return self.handle is None

    def _h(self):
        if self.handle is None:
            raise PsumError(1, "Error: null pointer")   # backend.hpp:16-20
        return self.handle

    def set_options(self, options):
        check(lib().psum_mg_set_options(self._h(), options.encode()))

    def set_matrix(self, n_row, n_col, nnz, rows, cols, vals):
        rows = np.ascontiguousarray(rows, np.uint64)
        cols = np.ascontiguousarray(cols, np.uint64)
        vals = np.ascontiguousarray(vals, np.float64)
        check(lib().psum_mg_set_matrix(self._h(), n_row, n_col, nnz, _ptr(rows), _ptr(cols), _ptr(vals)))

    def set_source_replace(self, idxs, values):
        idxs = np.ascontiguousarray(idxs, np.uint64)
        values = np.ascontiguousarray(values, np.float64)
        check(lib().psum_mg_set_source_replace(self._h(), idxs.size, _ptr(idxs) if idxs.size else None,
                                               _ptr(values) if values.size else None))

    def set_source_addback(self, idxs, values):
        idxs = np.ascontiguousarray(idxs, np.uint64)
        values = np.ascontiguousarray(values, np.float64)
        check(lib().psum_mg_set_source_addback(self._h(), idxs.size, _ptr(idxs) if idxs.size else None,
                                               _ptr(values) if values.size else None))

    def solve(self, b, x):
        """Synchronous solve on device buffers; returns the status (0 or
        PSUM_ERR_NOT_CONVERGED = 4 when `tol` was set and not met)."""
        _ready(b, x)
        code = lib().psum_mg_solve(self._h(), _ptr(b), _ptr(x))
        if code not in (0, 4):
            check(code)
        return code

    def solve_async(self, b, x, stream=None):
        if stream is None:
            _ready(b, x)
        check(lib().psum_mg_solve_async(self._h(), _ptr(b), _ptr(x), _stream_handle(stream)))

    def last_stats(self):
        cyc, ref = C.c_int(), C.c_int()
        rel, rel0 = C.c_double(), C.c_double()
        check(lib().psum_mg_last_stats(self._h(), C.byref(cyc), C.byref(ref), C.byref(rel), C.byref(rel0)))
        return {"cycles": cyc.value, "refinements": ref.value, "rel_residual": rel.value,
                "initial_rel_residual": rel0.value}

    def hierarchy_info(self):
        lv, cr, ex = C.c_int(), C.c_ulonglong(), C.c_ulonglong()
        check(lib().psum_mg_hierarchy_info(self._h(), C.byref(lv), C.byref(cr), C.byref(ex)))
        return {"levels": lv.value, "coarse_rows": cr.value, "exception_rows_level0": ex.value}

    def free(self):
        if self.handle is not None:
            check(lib().psum_mg_destroy(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class _PoissonFrontend:
    dim = 0
    Cartesian = "Cartesian"

    def __init__(self):
        self.backend_name = "native"
        self.options = ""
        self.backend = solver_backend()
        self.replace_idx = np.zeros(0, np.uint64)
        self.replace_val = np.zeros(0)
        self.coo = None
        self.grid = None

    def set_options(self, options):
        """Cached and replayed at init, like Poisson_solver_2d::set_options (:158-165)."""
        self.options = options
        if not self.backend.is_null():
            self.backend.set_options(options)

    def init(self, backend_name, grid, domain, fixed_boundaries, epsilon=8.854e-12):
        if grid.dim != self.dim:
            raise ValueError(f"grid must be {self.dim}-D")
        if domain != self.Cartesian:
            raise ValueError("only the Cartesian operator is provided by this frontend")
        if backend_name == "native":
            raise PsumError(1, "the 'native' Eigen direct solver is not part of this backend; "
                               "use cuda_multigrid32f_gpu or cuda_multigrid64_gpu")
        self.grid = grid
        self.replace_idx, self.replace_val = _merge_fixed(fixed_boundaries)
        rows, cols, vals = assemble_poisson(grid, self.replace_idx, epsilon)
        self.coo = (rows, cols, vals)
        self.backend_name = backend_name
        self.backend = solver_backend(backend_name)
        if self.options:
            self.backend.set_options(self.options)
        n = grid.n_nodes
        self.backend.set_matrix(n, n, rows.size, rows, cols, vals)

    def coeff_matrix(self):
        return self.coo

    def make_righthand_item(self):
        """Poisson_solver_2d::make_righthand_item (:73-103) without mixed boundaries."""
        self.backend.set_source_addback(np.zeros(0, np.uint64), np.zeros(0))
        self.backend.set_source_replace(self.replace_idx, self.replace_val)

    def solve(self, phi, source):
        """Solve A phi = source on device buffers; `source` is overwritten."""
        self.make_righthand_item()
        return self.backend.solve(source, phi)


class Poisson_solver_2d(_PoissonFrontend):
    dim = 2


class Poisson_solver_3d(_PoissonFrontend):
    dim = 3
