"""Property-based checks of the Poisson frontends' host logic over random
set-ups (hypothesis; CPU only).  For random small 2-D / 3-D grids, random
Neumann / Robin boundaries on random sides (with coefficient and value
functions), a random fixed side and a random epsilon:
  * the per-node ghost elimination equals PSuM's augmented ghost system
    (ghost_element_manager.hpp), solved directly;
  * the backends' host multigrid setup (mg_host.cpp) builds the hierarchy of
    the oracle's restatement of multigrid_core::setup."""
import tempfile

import numpy as np
import pytest
from hypothesis import HealthCheck, given, settings, strategies as st

import psum_b200 as P
from test_ghost_elimination import augmented_solve, eliminated_solve
from test_mg_host import compare, program  # noqa: F401  (module-scoped fixture)

SIDES = {2: ["N", "S", "E", "W"], 3: ["Xneg", "Xpos", "Yneg", "Ypos", "Zneg", "Zpos"]}
FIXED_2D = {"N": "N", "S": "S", "E": "E", "W": "W"}


@st.composite
def setups(draw):
    dim = draw(st.sampled_from([2, 3]))
    cells = [draw(st.integers(3, 7)) for _ in range(dim)]
    lower = [draw(st.floats(-1.0, 1.0)) for _ in range(dim)]
    upper = [lo + draw(st.floats(0.5, 2.0)) for lo in lower]
    g = P.simple_grid(tuple(lower), tuple(upper), tuple(cells))
    sides = SIDES[dim]
    fixed_side = draw(st.sampled_from(sides))
    mixed = []
    for side in draw(st.lists(st.sampled_from(sides), min_size=1, max_size=len(sides), unique=True)):
        kind = draw(st.sampled_from(["neumann", "robin", "robin_fn"]))
        value = draw(st.floats(-2.0, 2.0))
        if kind == "neumann":
            coeffs = (0.0, 1.0)
        elif kind == "robin":
            coeffs = (draw(st.floats(0.0, 2.0)), draw(st.floats(0.2, 2.0)))
        else:
            a0, b0 = draw(st.floats(0.0, 1.0)), draw(st.floats(0.5, 1.5))
            coeffs = lambda *p, a0=a0, b0=b0: (a0 + 0.1 * abs(p[0]), b0 + 0.1 * abs(p[-1]))
        mixed.append(P.MixedBoundary(g, _side_nodes(g, side), side, coeffs,
                                     (lambda *p, v=value: v + 0.3 * p[0]) if draw(st.booleans()) else value))
    if draw(st.booleans()):
        e0 = draw(st.floats(0.5, 2.0))
        eps = lambda *p, e0=e0: e0 + 0.2 * abs(p[0])
    else:
        eps = draw(st.floats(0.5, 2.0))
    fixed_val = draw(st.floats(-1.0, 1.0))
    fixed = [P.Dirichlet_line(g, fixed_side, fixed_val) if dim == 2 else P.Dirichlet_plane(g, fixed_side, fixed_val)]
    return g, mixed, fixed, eps


def _side_nodes(g, side):
    if g.dim == 2:
        return P.Neumann_line(g, side).nodes
    return P.Neumann_plane(g, side).nodes


def assembler(g, eps):
    if g.dim == 2:
        return lambda ridx, mb: P.assemble_poisson_2d(g, "Cartesian", ridx, mb, eps)
    return lambda ridx, mb: P.assemble_poisson_3d(g, ridx, mb, eps)


@settings(max_examples=25, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow])
@given(setups(), st.integers(0, 2 ** 31 - 1))
def test_elimination_equals_augmented_ghost_system(setup, seed):
    g, mixed, fixed, eps = setup
    rho = np.random.default_rng(seed).normal(size=g.n_nodes)
    asm = assembler(g, eps)
    aug = augmented_solve(g, asm, fixed, mixed, rho)
    eli = eliminated_solve(g, asm, fixed, mixed, rho)
    assert np.abs(aug - eli).max() <= 1e-9 * max(1.0, np.abs(aug).max())


@settings(max_examples=15, deadline=None, derandomize=True,
          suppress_health_check=[HealthCheck.too_slow, HealthCheck.function_scoped_fixture])
@given(setup=setups())
def test_host_hierarchy_equals_oracle(program, setup):  # noqa: F811
    g, mixed, fixed, eps = setup
    ridx = np.unique(np.concatenate([f[0] for f in fixed]))
    coo, _ = assembler(g, eps)(ridx, mixed)
    dims = [c + 1 for c in g.cells] + [1] * (3 - g.dim)
    with tempfile.TemporaryDirectory() as d:
        import pathlib
        compare(program, pathlib.Path(d), coo, g.n_nodes, tuple(dims), 2)
