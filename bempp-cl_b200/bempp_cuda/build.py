"""Build libbemppcuda.so in-tree (nvcc, sm_100a): ``python -m bempp_cuda.build``."""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "csrc")


def build(jobs=4):
    subprocess.run(["make", "-s", "-j%d" % jobs, "-C", CSRC], check=True)
    lib = os.path.join(HERE, "libbemppcuda.so")
    if not os.path.exists(lib):
        raise RuntimeError("build finished but %s is missing" % lib)
    return lib


if __name__ == "__main__":
    print(build(int(sys.argv[1]) if len(sys.argv) > 1 else 4))
