"""Build libcucosma.so (sm_100a) in-tree with nvcc via the csrc Makefile."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs=8, verbose=False):
    r = subprocess.run(["make", "-s", "-j%d" % jobs, "-C", os.path.join(HERE, "csrc")], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("libcucosma build failed:\n" + r.stdout[-6000:] + r.stderr[-6000:])
    if verbose:
        print(r.stdout)
    return os.path.join(HERE, "libcucosma.so")


if __name__ == "__main__":
    print(build(verbose=True))
