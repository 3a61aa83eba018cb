"""Build libecgb200.so in-tree (nvcc, -gencode arch=compute_100a,code=sm_100a).

Usage: python atom-mol-nonbo_b200/build.py [--force]
The library lands in atom-mol-nonbo_b200/ecg_b200/libecgb200.so next to the
ctypes binding that loads it; per-kernel register and spill counts from
ptxas -v are left in csrc/*.ptxas.log.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")


def build(force=False, jobs=4):
    if force:
        subprocess.run(["make", "-s", "-C", CSRC, "clean"], check=True)
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", CSRC], check=True)
    return os.path.join(HERE, "ecg_b200", "libecgb200.so")


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
