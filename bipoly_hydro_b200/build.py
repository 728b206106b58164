"""Build step for the package: compiles libbph.so for sm_100a with nvcc."""
from __future__ import annotations

import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8) -> str:
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", os.path.join(_HERE, "csrc")], check=True)
    return os.path.join(_HERE, "libbph.so")


if __name__ == "__main__":
    print(build())
