"""Builds libdgq.so in-tree for sm_100a (nvcc cross-compiles without a GPU)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs=8, verbose=False):
    out = None if verbose else subprocess.DEVNULL
    subprocess.run(["make", "-C", HERE, f"-j{jobs}"], check=True, stdout=out)
    return os.path.join(HERE, "libdgq.so")


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
