"""Builds libpsum_b200.so in-tree for sm_100a (nvcc cross-compiles without a GPU)."""
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs=8):
    """Compile the CUDA/C++ sources under psum_b200/csrc into psum_b200/libpsum_b200.so."""
    subprocess.run(["make", "-s", f"-j{jobs}", "-C", os.path.join(_HERE, "csrc")], check=True)
    return os.path.join(_HERE, "libpsum_b200.so")


if __name__ == "__main__":
    print(build())
