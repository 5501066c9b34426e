"""The library's multigrid host setup (psum_b200/csrc/mg_host.cpp) against the
oracle's restatement of PSuM's multigrid_core::setup (multigrid_core.hpp:49-150)
on operators the GPU tests do not cover: 1-D, 3-D with mixed boundary planes
and a position-dependent epsilon, and 2-D mixed boundaries.  The product's
source is compiled into tests/cpp/mg_host_check.cpp, which writes every
level's scaled operator and inverse diagonal and the dense coarse inverse
(CPU only)."""
import glob
import os
import shutil
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

import psum_b200 as P
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    exe = str(tmp_path_factory.mktemp("mgh") / "mg_host_check")
    gomp = (glob.glob("/usr/lib/gcc/x86_64-linux-gnu/*/libgomp.so") + ["-lgomp"])[0]
    cmd = ["g++", "-std=c++17", "-O2", "-fopenmp", "-Wall", "-Wextra", "-Werror",
           os.path.join(ROOT, "tests", "cpp", "mg_host_check.cpp"), os.path.join(ROOT, "psum_b200", "csrc", "mg_host.cpp"),
           "-o", exe, gomp]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def product_levels(program, tmp_path, coo, n, dims, depth):
    r, c, v = coo
    src, dst = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(src, "wb") as f:
        np.array([n, len(v), dims[0], dims[1], dims[2], depth], np.int64).tofile(f)
        np.asarray(r, np.uint64).tofile(f)
        np.asarray(c, np.uint64).tofile(f)
        np.asarray(v, np.float64).tofile(f)
    res = subprocess.run([program, str(src), str(dst)], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    raw = np.fromfile(dst, np.uint8)
    pos = 0

    def take(dtype, count):
        nonlocal pos
        a = raw[pos:pos + 8 * count].view(dtype)
        pos += 8 * count
        return a

    levels = []
    for _ in range(int(take(np.int64, 1)[0])):
        nl, m = (int(x) for x in take(np.int64, 2))
        rr, cc, vv = take(np.uint64, m), take(np.uint64, m), take(np.float64, m)
        dinv = take(np.float64, nl)
        levels.append((sp.csr_matrix((vv, (rr.astype(np.int64), cc.astype(np.int64))), shape=(nl, nl)), dinv))
    cn = int(take(np.int64, 1)[0])
    coarse_inv = take(np.float64, cn).reshape(levels[-1][0].shape)
    return levels, coarse_inv


def compare(program, tmp_path, coo, n, dims, depth):
    mine, coarse_inv = product_levels(program, tmp_path, coo, n, dims, depth)
    # the dense inverse of the coarsest scaled operator (sycl_inner_solver.hpp:51-71)
    Ac = mine[-1][0].toarray()
    assert np.abs(coarse_inv @ Ac - np.eye(Ac.shape[0])).max() < 1e-9
    mg = O.Multigrid(coo[0], coo[1], coo[2], n, dims[0], dims[1], dims[2], depth)
    assert len(mine) == mg.levels
    for level, (A, dinv) in enumerate(mine):
        r, c, v, dref = mg.level_coo(level)
        nl = mg.level_rows(level)
        R = sp.csr_matrix((v, (r.astype(np.int64), c.astype(np.int64))), shape=(nl, nl))
        scale = abs(R).max()
        assert abs(A - R).max() <= 1e-12 * scale, level
        np.testing.assert_allclose(dinv, dref, rtol=1e-12, atol=0)
    return len(mine)


def test_3d_mixed_planes_and_epsilon(program, tmp_path):
    g = P.simple_grid((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (16, 16, 16))
    fixed = P.Dirichlet_plane(g, "Xneg", 0.0)[0]
    mixed = [P.Neumann_plane(g, "Xpos", 0.0), P.Neumann_plane(g, "Yneg", 0.0), P.Neumann_plane(g, "Ypos", 0.0),
             P.Neumann_plane(g, "Zneg", 0.0), P.Robin_plane(g, "Zpos", (1.5, 0.75), 0.0)]
    coo, _ = P.assemble_poisson_3d(g, fixed, mixed, lambda x, y, z: 1.0 + 0.5 * x + 0.25 * y * z)
    assert compare(program, tmp_path, coo, g.n_nodes, (17, 17, 17), 3) >= 3


def test_1d_boundary_rows(program, tmp_path):
    g = P.simple_grid((0.0,), (1.0,), (256,))
    coo, _ = P.assemble_poisson_1d(g, P.Dirichlet_point(g, "R", 1.0)[0], [P.Neumann_point(g, "L", 0.0)], 1.0)
    assert compare(program, tmp_path, coo, g.n_nodes, (257, 1, 1), 4) >= 3


def test_2d_mixed_boundaries(program, tmp_path):
    g = P.simple_grid((0.0, 0.0), (1.0, 1.0), (64, 64))
    mixed = [P.Neumann_line(g, "N", 0.0), P.Neumann_line(g, "S", 0.0), P.Robin_Line(g, "E", (2.0, 0.5), 0.3)]
    coo, _ = P.assemble_poisson_2d(g, "Cartesian", P.Dirichlet_line(g, "W", 1.0)[0], mixed,
                                   lambda a, b: 1.0 + 0.5 * b)
    assert compare(program, tmp_path, coo, g.n_nodes, (65, 65, 1), 3) >= 3


def test_hall_thruster_operator(program, tmp_path):
    # the reference's 3-D Hall thruster set-up (Robin planes with coefficient
    # functions, electrodes, ceramic epsilon) at depth 2 as its test uses
    from test_psolver_3d import hall_thruster_system
    ps, A, _ = hall_thruster_system(24, 24, 14)
    assert compare(program, tmp_path, ps.coeff_matrix(), A.shape[0], (25, 25, 15), 2) == 3


@pytest.mark.parametrize("name", ["fixed_zone", "robin_plates", "neumann_lid"])
def test_native_vs_multigrid_2d_operators(program, tmp_path, name):
    # the three set-ups of test_native_vs_multigrid_2d.cpp at depth 3
    import test_multigrid_convergence_2d as T
    g, ps, _, _ = getattr(T, name)()
    assert compare(program, tmp_path, ps.coeff_matrix(), g.n_nodes, (g.cells[0] + 1, g.cells[1] + 1, 1), 3) == 4
