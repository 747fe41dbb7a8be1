"""Build recipe for the sm_100a shared library (nvcc; no GPU needed to build)."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build_library(jobs: int = 8, extra_nvflags: str = "") -> str:
    """Compile every CUDA source under csrc/ for sm_100a into libordvec_b200.so."""
    env = dict(os.environ)
    if extra_nvflags:
        env["EXTRA_NVFLAGS"] = extra_nvflags
    subprocess.run(["make", "-s", f"-j{jobs}", "-C", os.path.join(HERE, "csrc")], check=True, env=env)
    return os.path.join(HERE, "libordvec_b200.so")


if __name__ == "__main__":
    print(build_library())
