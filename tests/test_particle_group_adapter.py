"""The header-only C++ adapters compiled into small programs against the
library: include/psum_particle_group.hpp (insert with and without
validation, size, NaN-invalid content, compress, clear, the capacity error)
and include/psum_device_field.hpp (B-spline deposit and gathers of a group at
orders 1-4).  The programs must compile and link everywhere; their checks
pass on a GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "psum_b200")


CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
PROGRAMS = ["particle_group_check", "device_field_check"]


def _build(tmp_path, name):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    exe = str(tmp_path / name)
    cuda_lib = os.path.join(CUDA, "lib64")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "cpp", name + ".cpp"),
           "-L", LIBDIR, "-lpsum_b200", "-L", cuda_lib, "-lcudart", f"-Wl,-rpath,{LIBDIR}", f"-Wl,-rpath,{cuda_lib}",
           "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


@pytest.mark.parametrize("name", PROGRAMS)
def test_adapter_compiles_and_links(tmp_path, name):
    _build(tmp_path, name)


@pytest.mark.gpu
@pytest.mark.parametrize("name", PROGRAMS)
def test_adapter_program_on_gpu(tmp_path, name):
    exe = _build(tmp_path, name)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("ok")
