"""Builds libpbrcm.so (and the bounds-checked libpbrcm_checks.so) in-tree with
nvcc for sm_100a, using parallelbatchrcm_b200/csrc/Makefile."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")


def build(jobs: int = 8, quiet: bool = True) -> None:
    cmd = ["make", "-C", CSRC, f"-j{jobs}"]
    if quiet:
        cmd.insert(1, "-s")
    subprocess.run(cmd, check=True)


if __name__ == "__main__":
    build(quiet=False)
