"""Build libscattersim_b200.so (sm_100a) in-tree with nvcc through the csrc Makefile.

    python -m scattersim_b200.build [--clean]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")


def build(clean: bool = False, jobs: int = 8) -> str:
    if clean:
        subprocess.run(["make", "-C", CSRC, "clean"], check=True)
    subprocess.run(["make", "-C", CSRC, f"-j{jobs}"], check=True)
    cli = os.path.join(HERE, "cli")
    if os.path.exists(os.path.join(cli, "Makefile")):
        subprocess.run(["make", "-C", cli, f"-j{jobs}"], check=True)
    return os.path.join(HERE, "libscattersim_b200.so")


if __name__ == "__main__":
    print(build(clean="--clean" in sys.argv))
