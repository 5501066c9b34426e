"""The header-only C++ particle_group adapter (include/psum_particle_group.hpp)
compiled into a small program against the library: it must compile and link
everywhere, and its checks (insert with and without validation, size,
NaN-invalid content, compress, clear, the capacity error) pass on a GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "psum_b200")


def _build(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    exe = str(tmp_path / "particle_group_check")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "particle_group_check.cpp"), "-L", LIBDIR, "-lpsum_b200",
           f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_adapter_compiles_and_links(tmp_path):
    _build(tmp_path)


@pytest.mark.gpu
def test_adapter_program_on_gpu(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("ok")
