"""Host-side mirror of PSuM's field-solver interface over the B200 backend.

* ``solver_backend`` mirrors ``psum::field_solver::solver_backend``
  (src/field_solver/backend.hpp:11-107): a move-only owner of a backend handle
  obtained by name from the plugin registry, with the same seven operations.
* ``Poisson_solver_2d`` / ``Poisson_solver_3d`` mirror the FD frontends
  (src/field_solver/Poisson_solver_2d.hpp:22-411, Poisson_solver_3d.hpp:21-...)
  (and Poisson_solver_1d.hpp): ``assemble`` builds the operator on the host
  (bit-identical values through psum_poisson_assemble for the plain Cartesian
  case), ``init`` assembles, creates the backend, replays the cached options
  and calls ``set_matrix``; ``solve(phi, rho)`` hands the backend the mixed
  add-back and the Dirichlet values and solves on device buffers,
  overwriting ``rho`` like PSuM does; ``coeff_matrix()`` and
  ``make_righthand_item(rho)`` give the discrete system on the host.
* ``Dirichlet_line`` / ``Dirichlet_plane`` / ``Dirichlet_nodes`` /
  ``Dirichlet_box`` / ``Dirichlet_box_rz`` / ``Dirichlet_func`` mirror the boundary creators of
  src/field_solver/boundary_creator/Dirichlet.hpp; ``Neumann_line`` /
  ``Robin_Line`` (2-D) and ``Neumann_plane`` / ``Robin_plane`` (3-D) those of
  Neumann.hpp / Robin.hpp.  ``init`` also takes mixed (Neumann / Robin)
  boundaries and a position-dependent epsilon (``assemble_poisson_2d``,
  ``assemble_poisson_3d``), and in 2-D the cylindrical (z, r) operator.

Device buffers are torch CUDA float64 tensors (or raw device addresses).
Errors raise ``PsumError`` (a RuntimeError), as PSuM's frontends rethrow.
"""
import ctypes as C

import numpy as np

from ._lib import PsumError, check, lib

__all__ = ["simple_grid", "solver_backend", "Poisson_solver_2d", "Poisson_solver_3d", "Dirichlet_line",
           "Dirichlet_plane", "Dirichlet_nodes", "Dirichlet_box", "Dirichlet_box_rz", "Dirichlet_func",
           "Neumann_line", "Robin_Line", "Neumann_plane", "Robin_plane", "MixedBoundary", "assemble_poisson",
           "assemble_poisson_2d", "assemble_poisson_3d", "registered_table", "Poisson_solver_1d",
           "Dirichlet_point", "Dirichlet_range", "Neumann_point", "Robin_point", "assemble_poisson_1d"]


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


def Dirichlet_line(grid, direction, value, min_max=None):
    """Nodes of one boundary line of a 2-D grid (Dirichlet.hpp:58-99): S/N fix
    j = 0 / j = J, W/E fix i = 0 / i = I; with min_max = (lo, hi) only the
    nodes whose coordinate along the line lies in [lo, hi]."""
    if direction not in ("N", "S", "E", "W"):
        raise ValueError("direction must be one of N, S, E, W")
    idx = _line_nodes(grid, direction, min_max)
    return np.asarray(idx, np.uint64), np.full(len(idx), float(value))


def Dirichlet_plane(grid, direction, value, shape=None):
    """Nodes of one boundary plane of a 3-D grid (Dirichlet.hpp:137-181):
    Xneg/Xpos fix i = 0 / I, Yneg/Ypos j, Zneg/Zpos k; with shape(u, v) only
    the nodes whose in-plane coordinates satisfy it ((y, z) on X planes,
    (x, z) on Y planes, (x, y) on Z planes)."""
    I, J, K = grid.cells
    rng = {"X": range(I + 1), "Y": range(J + 1), "Z": range(K + 1)}
    axis, side = direction[0], direction[1:]
    fixed = {"X": I, "Y": J, "Z": K}[axis] if side == "pos" else 0
    ii = [fixed] if axis == "X" else rng["X"]
    jj = [fixed] if axis == "Y" else rng["Y"]
    kk = [fixed] if axis == "Z" else rng["Z"]
    idx = []
    for i in ii:
        for j in jj:
            for k in kk:
                if shape is not None:
                    x, y, z = (grid.lower[0] + i * grid.delta[0], grid.lower[1] + j * grid.delta[1],
                               grid.lower[2] + k * grid.delta[2])
                    uv = {"X": (y, z), "Y": (x, z), "Z": (x, y)}[axis]
                    if not shape(*uv):
                        continue
                idx.append(grid.n2i(i, j, k))
    return np.asarray(idx, np.uint64), np.full(len(idx), float(value))


def Dirichlet_nodes(grid, nodes, value):
    """Fixed value on explicit node tuples (e.g. the pinned node that makes a
    periodic operator non-singular, application/benchmark/TSI/main.cpp:106-113)."""
    idx = [grid.n2i(*n) for n in nodes]
    return np.asarray(idx, np.uint64), np.full(len(idx), float(value))


def Dirichlet_box(grid, *args, geo_tolerance=1e-10):
    """Nodes inside a box, with a tolerance of geo_tolerance times the
    grid's size: Dirichlet_box(g2, x0, y0, x1, y1, value[, geo_tolerance])
    (Dirichlet.hpp:104-119) or Dirichlet_box(g3, x0, y0, z0, x1, y1, z1,
    value[, geo_tolerance]) (:184-201)."""
    D = grid.dim
    if len(args) not in (2 * D + 1, 2 * D + 2):
        raise TypeError(f"Dirichlet_box on a {D}-D grid takes {2 * D} bounds and a value")
    lo, hi, value = args[:D], args[D:2 * D], args[2 * D]
    if len(args) == 2 * D + 2:
        geo_tolerance = args[2 * D + 1]
    coords = _node_coords(grid)
    span = np.prod([grid.upper[a] - grid.lower[a] for a in range(D)])
    tol = geo_tolerance * (np.sqrt(span) if D == 2 else np.cbrt(span))
    sel = np.ones(grid.n_nodes, bool)
    for a in range(D):
        sel &= (coords[a] >= lo[a] - tol) & (coords[a] <= hi[a] + tol)
    idx = np.nonzero(sel)[0].astype(np.uint64)
    return idx, np.full(idx.size, float(value))


def Dirichlet_box_rz(grid, z0, r0, z1, r1, value, geo_tolerance=1e-10):
    """Nodes of a 3-D grid inside the annular cylinder z0 <= z <= z1,
    r0 <= sqrt(x^2 + y^2) <= r1 (Dirichlet.hpp:204-223)."""
    if grid.dim != 3:
        raise ValueError("a 3-D grid is required")
    x, y, z = _node_coords(grid)
    span = np.prod([grid.upper[a] - grid.lower[a] for a in range(3)])
    tol = geo_tolerance * span ** (1.0 / 3)
    r = np.sqrt(x * x + y * y)
    sel = (z >= z0 - tol) & (z <= z1 + tol) & (r >= r0 - tol) & (r <= r1 + tol)
    idx = np.nonzero(sel)[0].astype(np.uint64)
    return idx, np.full(idx.size, float(value))


def Dirichlet_func(grid, predicate, value):
    """Nodes where predicate(x, y) (2-D, Dirichlet.hpp:121-135) or
    predicate(x, y, z) (3-D, :226-240) holds."""
    coords = _node_coords(grid)
    sel = np.array([bool(predicate(*p)) for p in zip(*coords)], bool)
    idx = np.nonzero(sel)[0].astype(np.uint64)
    return idx, np.full(idx.size, float(value))


def _node_positions(grid):
    """(x, y) of every node of a 2-D grid, shaped (I + 1, J + 1)."""
    if grid.dim != 2:
        raise ValueError("a 2-D grid is required")
    i = np.arange(grid.cells[0] + 1)
    j = np.arange(grid.cells[1] + 1)
    return np.meshgrid(grid.lower[0] + i * grid.delta[0], grid.lower[1] + j * grid.delta[1], indexing="ij")


def _node_coords(grid):
    """Flattened node coordinates per axis (nodePosition, simple_grid.hpp:209-214)."""
    axes = [grid.lower[a] + np.arange(grid.cells[a] + 1) * grid.delta[a] for a in range(grid.dim)]
    return [c.reshape(-1) for c in np.meshgrid(*axes, indexing="ij")]


# boundary directions: (axis, side) of boundary_direction_{1,2,3}d
DIRECTIONS = {1: {"R": (0, 1), "L": (0, -1)},
              2: {"E": (0, 1), "W": (0, -1), "N": (1, 1), "S": (1, -1)},
              3: {"Xpos": (0, 1), "Xneg": (0, -1), "Ypos": (1, 1), "Yneg": (1, -1), "Zpos": (2, 1), "Zneg": (2, -1)}}


class MixedBoundary:
    """mixed_boundary<D> (src/field_solver/mixed_boundary.hpp:17-150): the
    nodes of one boundary line (2-D) or plane (3-D) with the condition

        a * phi + b * dphi/dn = value      (n: the outward normal of `direction`)

    where (a, b) = coeffs (a pair, or a function of the node coordinates
    giving one) and value is a number or a function of the node coordinates.
    Directions are L, R in 1-D, N, S, E, W in 2-D and Xneg, Xpos, Yneg, Ypos,
    Zneg, Zpos in 3-D.  ``set`` plays the role of PSuM's ``boundary = value``."""

    def __init__(self, grid, nodes, direction, coeffs, value=None):
        names = DIRECTIONS.get(grid.dim, {})
        if direction not in names:
            raise ValueError(f"direction must be one of {', '.join(names) or '(1-D, 2-D or 3-D grids only)'}")
        self.grid = grid
        self.nodes = np.asarray(nodes, np.int64)
        self.direction = direction
        self.coeffs = coeffs
        self.value = value

    def set(self, value):
        self.value = value
        return self

    def _positions(self):
        return [c[self.nodes] for c in _node_coords(self.grid)]

    def values(self):
        if self.value is None:
            raise ValueError("mixed_boundary::evaluate: no value is set")
        pos = self._positions()
        if callable(self.value):
            return np.array([float(self.value(*p)) for p in zip(*pos)])
        return np.full(self.nodes.size, float(self.value))

    def coefficient_pairs(self):
        pos = self._positions()
        if callable(self.coeffs):
            pairs = np.array([self.coeffs(*p) for p in zip(*pos)], np.float64).reshape(-1, 2)
        else:
            pairs = np.tile(np.asarray(self.coeffs, np.float64), (self.nodes.size, 1))
        return pairs[:, 0], pairs[:, 1]


def _line_nodes(grid, direction, min_max):
    """Boundary line nodes (Neumann.hpp:48-88): S / N are j = 0 / J, W / E
    i = 0 / I; with min_max only those whose coordinate along the line lies
    in [min, max]."""
    I, J = grid.cells
    if direction == "S":
        ij = [(i, 0) for i in range(I + 1)]
    elif direction == "N":
        ij = [(i, J) for i in range(I + 1)]
    elif direction == "W":
        ij = [(0, j) for j in range(J + 1)]
    elif direction == "E":
        ij = [(I, j) for j in range(J + 1)]
    else:
        raise ValueError("direction must be one of N, S, E, W")
    out = []
    for i, j in ij:
        along = grid.lower[1] + j * grid.delta[1] if direction in ("W", "E") else grid.lower[0] + i * grid.delta[0]
        if min_max is None or not (along < min_max[0] or along > min_max[1]):
            out.append(grid.n2i(i, j))
    return out


def Neumann_line(grid, direction, value=None, min_max=None):
    """dphi/dn = value on a boundary line (Neumann.hpp:48-93)."""
    return MixedBoundary(grid, _line_nodes(grid, direction, min_max), direction, (0.0, 1.0), value)


def Robin_Line(grid, direction, coef_value_and_grad, value=None, min_max=None):
    """a * phi + b * dphi/dn = value on a boundary line (Robin.hpp:55-110);
    coef_value_and_grad is (a, b) or a function of (x, y) giving it."""
    return MixedBoundary(grid, _line_nodes(grid, direction, min_max), direction, coef_value_and_grad, value)


def _plane_nodes(grid, direction, min_max):
    """Boundary plane nodes of a 3-D grid (Neumann.hpp:96-128, Robin.hpp:116-150):
    i = 0 / I for Xneg / Xpos, j = 0 / J for Yneg / Ypos, k = 0 / K for Zneg /
    Zpos; with min_max only those whose x (Y and Z planes) or y (X planes)
    lies in [min, max]."""
    if grid.dim != 3:
        raise ValueError("a 3-D grid is required")
    if direction not in DIRECTIONS[3]:
        raise ValueError("direction must be one of " + ", ".join(DIRECTIONS[3]))
    axis, side = DIRECTIONS[3][direction]
    dims = tuple(c + 1 for c in grid.cells)
    idx = np.arange(int(np.prod(dims))).reshape(dims)
    sel = [slice(None)] * 3
    sel[axis] = 0 if side < 0 else dims[axis] - 1
    nodes = np.sort(idx[tuple(sel)].reshape(-1))
    if min_max is not None:
        coords = _node_coords(grid)
        along = coords[1] if axis == 0 else coords[0]
        v = along[nodes]
        nodes = nodes[~((v < min_max[0]) | (v > min_max[1]))]
    return nodes.tolist()


def Neumann_plane(grid, direction, value=None, min_max=None):
    """dphi/dn = value on a boundary plane (Neumann.hpp:96-133)."""
    return MixedBoundary(grid, _plane_nodes(grid, direction, min_max), direction, (0.0, 1.0), value)


def Robin_plane(grid, direction, coef_value_and_grad, value=None, min_max=None):
    """a * phi + b * dphi/dn = value on a boundary plane (Robin.hpp:116-163);
    coef_value_and_grad is (a, b) or a function of (x, y, z) giving it."""
    return MixedBoundary(grid, _plane_nodes(grid, direction, min_max), direction, coef_value_and_grad, value)


def _point_node(grid, direction):
    if grid.dim != 1:
        raise ValueError("a 1-D grid is required")
    if direction not in DIRECTIONS[1]:
        raise ValueError("direction must be L or R")
    return 0 if direction == "L" else grid.cells[0]


def Dirichlet_point(grid, direction, value):
    """The end node of a 1-D grid (Dirichlet.hpp:24-41): L is node 0, R node I."""
    return np.asarray([_point_node(grid, direction)], np.uint64), np.full(1, float(value))


def Dirichlet_range(grid, x0, x1, value, geo_tolerance=1e-10):
    """Nodes of a 1-D grid with x0 <= x <= x1 up to geo_tolerance times the
    grid's span (Dirichlet.hpp:43-56)."""
    if grid.dim != 1:
        raise ValueError("a 1-D grid is required")
    x = _node_coords(grid)[0]
    tol = geo_tolerance * (grid.upper[0] - grid.lower[0])
    idx = np.nonzero((x >= x0 - tol) & (x <= x1 + tol))[0].astype(np.uint64)
    return idx, np.full(idx.size, float(value))


def Neumann_point(grid, direction, value=None):
    """dphi/dn = value at an end of a 1-D grid (Neumann.hpp:24-44)."""
    return MixedBoundary(grid, [_point_node(grid, direction)], direction, (0.0, 1.0), value)


def Robin_point(grid, direction, coef_value_and_grad, value=None):
    """a * phi + b * dphi/dn = value at an end of a 1-D grid (Robin.hpp:24-54);
    coef_value_and_grad is (a, b) or a function of x giving it."""
    return MixedBoundary(grid, [_point_node(grid, direction)], direction, coef_value_and_grad, value)


def _merge_mixed(mixed_boundaries, fixed_idx):
    """mixed_boundary_list (mixed_boundary.hpp:158-190): keyed by (node,
    direction), a later boundary covers an earlier one's (node, direction)
    pairs, so a corner node keeps one condition per direction; fixed nodes
    cover every mixed condition of theirs (Poisson_solver_2d.hpp:191-199).
    Returns (node, direction, boundary index, position in that boundary) per
    mixed condition."""
    fixed = set(int(v) for v in np.asarray(fixed_idx, np.int64).tolist())
    taken = set()
    entries = []
    for b in reversed(range(len(mixed_boundaries))):
        mb = mixed_boundaries[b]
        for k, node in enumerate(mb.nodes.tolist()):
            if (node, mb.direction) in taken or node in fixed:
                continue
            taken.add((node, mb.direction))
            entries.append((node, mb.direction, b, k))
    entries.sort()
    return entries


def assemble_poisson_2d(grid, domain, fixed_nodes, mixed_boundaries=(), epsilon=8.854e-12):
    """Operator of Poisson_solver_2d::_init_impl (Poisson_solver_2d.hpp:182-368)
    for Cartesian or cylindrical (z along axis 0, r along axis 1) domains,
    epsilon a number or a function of (x, y) taken at the face midpoints, and
    mixed boundaries by ghost nodes: a mixed node's neighbour across its
    boundary is a ghost defined by the boundary condition with a central
    difference, and eliminating it changes the node's row and adds
    M * boundary values to its right-hand side (ghost_element_manager.hpp:
    A' = A - B D^-1 C, M = -B D^-1; here each ghost has its own equation, so
    D is diagonal and the elimination is per node).

    Returns ((rows, cols, vals) of A', (addback_rows, M_vals, mixed_entries)),
    where the right-hand side of row addback_rows[t] gains M_vals[t] times the
    value of mixed node t."""
    if grid.dim != 2:
        raise ValueError("a 2-D grid is required")
    if domain not in ("Cartesian", "Cylindrical"):
        raise ValueError("domain must be Cartesian or Cylindrical")
    I, J = grid.cells
    nI, nJ = I + 1, J + 1
    n = nI * nJ
    dx, dy = grid.delta
    dxr, dyr = 1.0 / dx, 1.0 / dy
    x, y = _node_positions(grid)
    ii, jj = np.meshgrid(np.arange(nI), np.arange(nJ), indexing="ij")
    node = (ii * nJ + jj).reshape(-1)
    nbr = {   # cyclic neighbours (the :225-231 cyclic_index)
        "N": (ii * nJ + (jj + 1) % nJ).reshape(-1), "S": (ii * nJ + (jj - 1) % nJ).reshape(-1),
        "E": (((ii + 1) % nI) * nJ + jj).reshape(-1), "W": (((ii - 1) % nI) * nJ + jj).reshape(-1),
    }
    if callable(epsilon):
        eps_f = np.vectorize(lambda a, b: float(epsilon(a, b)), otypes=[np.float64])
    else:
        eps_f = lambda a, b: np.full(np.shape(a), float(epsilon))
    # face midpoints of the unwrapped neighbours, as PSuM takes them
    eps = {"N": eps_f(x, y + 0.5 * dy), "S": eps_f(x, y - 0.5 * dy),
           "E": eps_f(x + 0.5 * dx, y), "W": eps_f(x - 0.5 * dx, y)}
    eps = {k: v.reshape(-1) for k, v in eps.items()}
    xf, yf = x.reshape(-1), y.reshape(-1)
    if domain == "Cylindrical":
        r_up = (yf + (yf + dy)) / 2
        r_lo = np.maximum((yf + (yf - dy)) / 2, 0.0)
        s_n = dx * np.pi * 2 * r_up
        s_s = dx * np.pi * 2 * r_lo
        s_e = s_w = np.pi * (r_up * r_up - r_lo * r_lo)
        vol = dx * np.pi * (r_up * r_up - r_lo * r_lo)
    else:
        s_n = s_s = np.full(n, dx)
        s_e = s_w = np.full(n, dy)
        vol = np.full(n, dx * dy)
    m = -1.0 / vol
    # (grad_E S_E eps_E - grad_W S_W eps_W + grad_N S_N eps_N - grad_S S_S eps_S) * (-1 / V)
    c = {"E": ((dxr * s_e) * eps["E"]) * m, "W": ((dxr * s_w) * eps["W"]) * m,
         "N": ((dyr * s_n) * eps["N"]) * m, "S": ((dyr * s_s) * eps["S"]) * m}
    cen = ((((-dxr * s_e) * eps["E"] - (dxr * s_w) * eps["W"]) + (-dyr * s_n) * eps["N"]) - (dyr * s_s) * eps["S"]) * m
    fixed = np.zeros(n, bool)
    fixed[np.asarray(fixed_nodes, np.int64)] = True
    entries = _merge_mixed(list(mixed_boundaries), np.nonzero(fixed)[0])
    opposite = {"N": "S", "S": "N", "E": "W", "W": "E"}
    ghost = {d: np.zeros(n, bool) for d in "NSEW"}
    extra_r, extra_c, extra_v = [], [], []
    add_rows, add_vals = [], []
    coef_cache = {}
    for t, (nd, d, b, k) in enumerate(entries):
        if b not in coef_cache:
            coef_cache[b] = mixed_boundaries[b].coefficient_pairs()
        a_val, b_grad = coef_cache[b][0][k], coef_cache[b][1][k]
        if b_grad == 0.0:
            raise ValueError("a mixed boundary needs a non-zero gradient coefficient (use a fixed boundary)")
        dr = dyr if d in ("N", "S") else dxr
        if ghost[opposite[d]][nd]:
            raise ValueError("a node with mixed boundaries on opposite sides is not supported")
        ghost[d][nd] = True
        cg = c[d][nd]
        # ghost = phi_opposite + 2 (value - a phi) / (b dr)
        extra_r += [nd, nd]
        extra_c += [nbr[opposite[d]][nd], nd]
        extra_v += [cg, cg * (-2.0 * a_val / (b_grad * dr))]
        add_rows.append(nd)
        add_vals.append(-cg * 2.0 / (b_grad * dr))
    free = ~fixed
    rows, cols, vals = [np.nonzero(fixed)[0]], [np.nonzero(fixed)[0]], [np.ones(int(fixed.sum()))]
    rows.append(node[free])
    cols.append(node[free])
    vals.append(cen[free])
    for d in "NSEW":
        sel = free & ~ghost[d]
        rows.append(node[sel])
        cols.append(nbr[d][sel])
        vals.append(c[d][sel])
    if extra_r:
        rows.append(np.asarray(extra_r, np.int64))
        cols.append(np.asarray(extra_c, np.int64))
        vals.append(np.asarray(extra_v))
    r = np.concatenate(rows).astype(np.int64)
    cc = np.concatenate(cols).astype(np.int64)
    v = np.concatenate(vals)
    # coalesce duplicates (a cyclic neighbour or a ghost's partner can repeat a column)
    key = r * n + cc
    order = np.argsort(key, kind="stable")
    key, v = key[order], v[order]
    uniq, start = np.unique(key, return_index=True)
    v = np.add.reduceat(v, start)
    keep = v != 0.0
    uniq, v = uniq[keep], v[keep]
    A = ((uniq // n).astype(np.uint64), (uniq % n).astype(np.uint64), v)
    M = (np.asarray(add_rows, np.int64), np.asarray(add_vals), entries)
    return A, M


def assemble_poisson_1d(grid, fixed_nodes, mixed_boundaries=(), epsilon=8.854e-12):
    """Operator of Poisson_solver_1d::_init_impl (Poisson_solver_1d.hpp:126-222).
    Free nodes: (grad_R eps_R - grad_L eps_L) * (-1 / dx) with epsilon (a
    number or a function of x) at the mean of the two node positions and
    cyclic neighbours.  A mixed node's row is its boundary condition itself,
    a phi + b dphi/dn, with the gradient taken one-sided to second order at
    the ends (-1.5, 2, -0.5 at node 0; 0.5, -2, 1.5 at node I) and centred
    elsewhere, b negated for the L direction and the row divided by the
    number of directions at the node.  The right-hand side of a mixed row is
    the source plus the boundary value, as PSuM's add-back makes it.

    Returns ((rows, cols, vals), (addback_rows, M_vals, mixed_entries)) like
    assemble_poisson_2d, with M_vals all 1."""
    if grid.dim != 1:
        raise ValueError("a 1-D grid is required")
    I = grid.cells[0]
    n = I + 1
    dx = grid.delta[0]
    dxr = 1.0 / dx
    fixed = np.zeros(n, bool)
    fixed[np.asarray(fixed_nodes, np.int64)] = True
    entries = _merge_mixed(list(mixed_boundaries), np.nonzero(fixed)[0])
    by_node = {}
    coef_cache = {}
    for nd, dname, b, k in entries:
        if b not in coef_cache:
            coef_cache[b] = mixed_boundaries[b].coefficient_pairs()
        by_node.setdefault(nd, []).append((dname, coef_cache[b][0][k], coef_cache[b][1][k]))
    eps_f = (lambda v: float(epsilon(v))) if callable(epsilon) else (lambda v: float(epsilon))
    pos = lambda i: grid.lower[0] + i * dx
    trip = {}

    def add(r, c, v):
        trip[(r, c)] = trip.get((r, c), 0.0) + v

    for i in range(n):
        if fixed[i]:
            add(i, i, 1.0)
            continue
        iR, iL = (i + 1) % n, (i - 1) % n
        if i in by_node:
            if i == I:
                grad = [((i - 2) % n, dxr * 0.5), (iL, dxr * -2.0), (i, dxr * 1.5)]
            elif i == 0:
                grad = [(i, dxr * -1.5), (iR, dxr * 2.0), ((i + 2) % n, dxr * -0.5)]
            else:
                grad = [(iL, dxr * -0.5), (iR, dxr * 0.5)]
            conds = sorted(by_node[i], key=lambda t: 0 if t[0] == "L" else 1)   # enum order: L, R
            row = {}
            for dname, a_val, b_grad in conds:
                g = b_grad if dname == "R" else -b_grad
                for c, v in grad:
                    row[c] = row.get(c, 0.0) + v * g
                row[i] = row.get(i, 0.0) + a_val
            scale = 1.0 / len(conds)
            for c, v in row.items():
                add(i, c, v * scale)
        else:
            eps_R = eps_f((pos(i) + pos(i + 1)) / 2)
            eps_L = eps_f((pos(i) + pos(i - 1)) / 2)
            m = -1.0 / dx
            # (grad_R S eps_R - grad_L S eps_L) * (-1 / V), S = 1, V = dx
            add(i, i, (((dxr * -1) * 1.0) * eps_R - (dxr * 1.0) * eps_L) * m)
            add(i, iR, ((dxr * 1.0) * eps_R) * m)
            add(i, iL, (-((dxr * -1) * 1.0) * eps_L) * m)
    keys = sorted(trip)
    rows = np.asarray([k[0] for k in keys], np.uint64)
    cols = np.asarray([k[1] for k in keys], np.uint64)
    vals = np.asarray([trip[k] for k in keys])
    keep = vals != 0.0
    A = (rows[keep], cols[keep], vals[keep])
    M = (np.asarray([e[0] for e in entries], np.int64), np.ones(len(entries)), entries)
    return A, M


def assemble_poisson_3d(grid, fixed_nodes, mixed_boundaries=(), epsilon=8.854e-12):
    """Operator of Poisson_solver_3d::_init_impl (Poisson_solver_3d.hpp:178-349):
    the 7-point finite-volume stencil with epsilon a number or a function of
    (x, y, z) taken at the face midpoints (the mean of the two node
    positions, :311-322), cyclic neighbours (:221-227), and mixed boundaries
    by ghost nodes eliminated per node as in assemble_poisson_2d: a mixed
    node's neighbour across the boundary is the ghost
    phi_opposite + 2 (value - a phi) / (b dr).

    Returns ((rows, cols, vals) of A', (addback_rows, M_vals, mixed_entries))
    with the meaning of assemble_poisson_2d's result."""
    if grid.dim != 3:
        raise ValueError("a 3-D grid is required")
    dims = [c + 1 for c in grid.cells]
    nI, nJ, nK = dims
    n = nI * nJ * nK
    d = list(grid.delta)
    dr = [1.0 / v for v in d]
    ii, jj, kk = [a.reshape(-1) for a in np.meshgrid(np.arange(nI), np.arange(nJ), np.arange(nK), indexing="ij")]
    ijk = [ii, jj, kk]
    node = (ii * nJ + jj) * nK + kk

    def at(i, j, k):
        return ((i % nI) * nJ + (j % nJ)) * nK + (k % nK)

    names = DIRECTIONS[3]
    nbr = {}
    for name, (axis, side) in names.items():
        shifted = [v.copy() for v in ijk]
        shifted[axis] = shifted[axis] + side
        nbr[name] = at(*shifted)
    pos = [grid.lower[a] + ijk[a] * d[a] for a in range(3)]
    if callable(epsilon):
        eps_f = np.vectorize(lambda a, b, c: float(epsilon(a, b, c)), otypes=[np.float64])
    else:
        eps_f = lambda a, b, c: np.full(np.shape(a), float(epsilon))
    eps = {}
    for name, (axis, side) in names.items():
        mid = list(pos)
        mid[axis] = (pos[axis] + (grid.lower[axis] + (ijk[axis] + side) * d[axis])) / 2
        eps[name] = eps_f(*mid)
    surface = [d[1] * d[2], d[0] * d[2], d[0] * d[1]]
    m = -1.0 / (d[0] * d[1] * d[2])
    c = {name: ((dr[axis] * surface[axis]) * eps[name]) * m for name, (axis, _) in names.items()}
    # (grad_E S eps_E - grad_W S eps_W + grad_N S eps_N - grad_S S eps_S + grad_U S eps_U - grad_D S eps_D) * (-1 / V)
    cen = (-dr[0] * surface[0]) * eps["Xpos"] - (dr[0] * surface[0]) * eps["Xneg"]
    cen = cen + (-dr[1] * surface[1]) * eps["Ypos"]
    cen = cen - (dr[1] * surface[1]) * eps["Yneg"]
    cen = cen + (-dr[2] * surface[2]) * eps["Zpos"]
    cen = (cen - (dr[2] * surface[2]) * eps["Zneg"]) * m
    fixed = np.zeros(n, bool)
    fixed[np.asarray(fixed_nodes, np.int64)] = True
    entries = _merge_mixed(list(mixed_boundaries), np.nonzero(fixed)[0])
    opposite = {"Xpos": "Xneg", "Xneg": "Xpos", "Ypos": "Yneg", "Yneg": "Ypos", "Zpos": "Zneg", "Zneg": "Zpos"}
    ghost = {name: np.zeros(n, bool) for name in names}
    extra_r, extra_c, extra_v = [], [], []
    add_rows, add_vals = [], []
    coef_cache = {}
    for nd, dname, b, k in entries:
        if b not in coef_cache:
            coef_cache[b] = mixed_boundaries[b].coefficient_pairs()
        a_val, b_grad = coef_cache[b][0][k], coef_cache[b][1][k]
        if b_grad == 0.0:
            raise ValueError("a mixed boundary needs a non-zero gradient coefficient (use a fixed boundary)")
        if ghost[opposite[dname]][nd]:
            raise ValueError("a node with mixed boundaries on opposite sides is not supported")
        ghost[dname][nd] = True
        drd = dr[names[dname][0]]
        cg = c[dname][nd]
        extra_r += [nd, nd]
        extra_c += [nbr[opposite[dname]][nd], nd]
        extra_v += [cg, cg * (-2.0 * a_val / (b_grad * drd))]
        add_rows.append(nd)
        add_vals.append(-cg * 2.0 / (b_grad * drd))
    free = ~fixed
    rows, cols, vals = [np.nonzero(fixed)[0]], [np.nonzero(fixed)[0]], [np.ones(int(fixed.sum()))]
    rows.append(node[free])
    cols.append(node[free])
    vals.append(cen[free])
    for name in names:
        sel = free & ~ghost[name]
        rows.append(node[sel])
        cols.append(nbr[name][sel])
        vals.append(c[name][sel])
    if extra_r:
        rows.append(np.asarray(extra_r, np.int64))
        cols.append(np.asarray(extra_c, np.int64))
        vals.append(np.asarray(extra_v))
    r = np.concatenate(rows).astype(np.int64)
    cc = np.concatenate(cols).astype(np.int64)
    v = np.concatenate(vals)
    key = r * n + cc
    order = np.argsort(key, kind="stable")
    key, v = key[order], v[order]
    uniq, start = np.unique(key, return_index=True)
    v = np.add.reduceat(v, start)
    keep = v != 0.0
    uniq, v = uniq[keep], v[keep]
    A = ((uniq // n).astype(np.uint64), (uniq % n).astype(np.uint64), v)
    M = (np.asarray(add_rows, np.int64), np.asarray(add_vals), entries)
    return A, M


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

    def tma_sweeps(self):
        """Level vectors the TMA-staged sweep kernel has read so far (one tensor map each)."""
        lv = C.c_int()
        check(lib().psum_mg_tma_sweeps(self._h(), C.byref(lv)))
        return lv.value

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
    Cylindrical = "Cylindrical"

    def __init__(self):
        self.backend_name = "native"
        self.options = ""
        self.backend = solver_backend()
        self.replace_idx = np.zeros(0, np.uint64)
        self.replace_val = np.zeros(0)
        self.coo = None
        self.grid = None
        self.mixed = []
        self.mixed_M = None

    def set_options(self, options):
        """Cached and replayed at init, like Poisson_solver_2d::set_options (:158-165)."""
        self.options = options
        if not self.backend.is_null():
            self.backend.set_options(options)

    def assemble(self, grid, domain, fixed_boundaries, epsilon=8.854e-12, mixed_boundaries=()):
        """The host half of Poisson_solver_{2,3}d::_init_impl
        (Poisson_solver_2d.hpp:182-368, Poisson_solver_3d.hpp:178-349): merge
        the fixed boundaries and assemble the operator, with mixed (Neumann /
        Robin) boundaries, an epsilon function of the node coordinates and, in
        2-D, the cylindrical domain.  Needs no GPU; ``coeff_matrix`` and
        ``make_righthand_item(rho)`` then give the discrete system."""
        if grid.dim != self.dim:
            raise ValueError(f"grid must be {self.dim}-D")
        general = bool(mixed_boundaries) or domain != self.Cartesian or callable(epsilon)
        if domain not in (self.Cartesian, self.Cylindrical) or (domain == self.Cylindrical and self.dim != 2):
            raise ValueError("the cylindrical domain is provided in 2-D; 3-D domains are Cartesian")
        self.grid = grid
        self.replace_idx, self.replace_val = _merge_fixed(fixed_boundaries)
        if general and self.dim == 2:
            (rows, cols, vals), self.mixed_M = assemble_poisson_2d(grid, domain, self.replace_idx,
                                                                   list(mixed_boundaries), epsilon)
            self.mixed = list(mixed_boundaries)
        elif general:
            (rows, cols, vals), self.mixed_M = assemble_poisson_3d(grid, self.replace_idx, list(mixed_boundaries),
                                                                   epsilon)
            self.mixed = list(mixed_boundaries)
        else:
            rows, cols, vals = assemble_poisson(grid, self.replace_idx, epsilon)
            self.mixed, self.mixed_M = [], None
        self.coo = (rows, cols, vals)

    def init(self, backend_name, grid, domain, fixed_boundaries, epsilon=8.854e-12, mixed_boundaries=()):
        """Poisson_solver_{2,3}d::init / _init_impl (Poisson_solver_2d.hpp:182-404,
        Poisson_solver_3d.hpp:178-395): ``assemble``, then create the backend,
        replay the cached options and hand it the operator."""
        if backend_name == "native":
            raise PsumError(1, "the 'native' Eigen direct solver is not part of this backend; "
                               "use cuda_multigrid32f_gpu or cuda_multigrid64_gpu")
        self.assemble(grid, domain, fixed_boundaries, epsilon, mixed_boundaries)
        self._attach(backend_name)

    def _attach(self, backend_name):
        rows, cols, vals = self.coo
        self.backend_name = backend_name
        self.backend = solver_backend(backend_name)
        if self.options:
            self.backend.set_options(self.options)
        n = self.grid.n_nodes
        self.backend.set_matrix(n, n, rows.size, rows, cols, vals)

    def coeff_matrix(self):
        return self.coo

    def addback(self):
        """(rows, values) added to the right-hand side for the mixed
        boundaries: M times the boundary values, summed per row."""
        if not self.mixed_M or len(self.mixed_M[0]) == 0:
            return np.zeros(0, np.uint64), np.zeros(0)
        rows, mvals, entries = self.mixed_M
        vals_of = [mb.values() for mb in self.mixed]
        bv = np.array([vals_of[b][k] for (_, _, b, k) in entries])
        contrib = mvals * bv
        uniq, inv = np.unique(rows, return_inverse=True)
        return uniq.astype(np.uint64), np.bincount(inv, weights=contrib, minlength=uniq.size)

    def make_righthand_item(self, rho=None):
        """Poisson_solver_2d::make_righthand_item (:73-131).  Without an
        argument: hand the backend the mixed boundaries' add-back and the
        fixed values, which it applies to the source at solve time.  With a
        host array rho: return the right-hand side itself, rho plus the
        add-back with the fixed values replaced (the (rho, b) overload)."""
        idx, val = self.addback()
        if rho is not None:
            b = np.array(rho, np.float64, copy=True)
            np.add.at(b, idx.astype(np.int64), val)
            b[self.replace_idx.astype(np.int64)] = self.replace_val
            return b
        self.backend.set_source_addback(idx, val)
        self.backend.set_source_replace(self.replace_idx, self.replace_val)

    def solve(self, phi, source):
        """Solve A phi = source on device buffers; `source` is overwritten."""
        self.make_righthand_item()
        return self.backend.solve(source, phi)


class Poisson_solver_1d(_PoissonFrontend):
    """Poisson_solver_1d (Poisson_solver_1d.hpp): init(backend_name, grid,
    fixed_boundaries, epsilon, mixed_boundaries) with the operator of
    assemble_poisson_1d; the backend options give I = cells + 1, J = K = 1."""
    dim = 1

    def assemble(self, grid, fixed_boundaries, epsilon=8.854e-12, mixed_boundaries=()):
        """The host half of Poisson_solver_1d::_init_impl: merge the fixed
        boundaries and assemble the operator (no GPU needed)."""
        if grid.dim != 1:
            raise ValueError("grid must be 1-D")
        self.grid = grid
        self.replace_idx, self.replace_val = _merge_fixed(fixed_boundaries)
        self.coo, self.mixed_M = assemble_poisson_1d(grid, self.replace_idx, list(mixed_boundaries), epsilon)
        self.mixed = list(mixed_boundaries)

    def init(self, backend_name, grid, fixed_boundaries, epsilon=8.854e-12, mixed_boundaries=()):
        if backend_name == "native":
            raise PsumError(1, "the 'native' Eigen direct solver is not part of this backend; "
                               "use cuda_multigrid32f_gpu or cuda_multigrid64_gpu")
        self.assemble(grid, fixed_boundaries, epsilon, mixed_boundaries)
        self._attach(backend_name)


class Poisson_solver_2d(_PoissonFrontend):
    dim = 2


class Poisson_solver_3d(_PoissonFrontend):
    dim = 3
