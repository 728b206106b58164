"""Generates the golden fixtures of tests/golden/ with the CPU oracle.

The reference ships no golden vectors and cannot be run here, so these are
the oracle's own outputs on seeded inputs: they pin the oracle (and through
it the CUDA path) against regressions.  Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

# name: (numr, numz, numphi, dr, isym, mmax, seed)
CASES = {
    "g14x12x16_isym2": (14, 12, 16, 1.0 / 12.0, 2, 6, 11),
    "g14x10x32_isym1": (14, 10, 32, 1.0 / 12.0, 1, 8, 12),
    "g12x12x32_isym3": (12, 12, 32, 1.0 / 10.0, 3, 6, 13),
    "g14x10x64_isym2_m30": (14, 10, 64, 1.0 / 12.0, 2, 30, 14),
}


def density(numr, numz, numphi, dr, isym, seed):
    from tests.helpers import smooth_density

    return smooth_density(numr, numz, numphi, dr, isym, seed=seed)


def main():
    from oracle import oracle as O

    O.build()
    for name, (numr, numz, numphi, dr, isym, mmax, seed) in CASES.items():
        o = O.Oracle(numr, numz, numphi, dr, isym, mmax)
        rho = density(numr, numz, numphi, dr, isym, seed)
        cold = o.potential_solver(rho, 0)
        rho2 = np.asfortranarray(np.roll(rho, 1, axis=2))  # the warm step sees rho rotated one zone
        warm = o.potential_solver(rho2, 2)
        S = o.moments_S()
        G = o.green()
        np.savez_compressed(os.path.join(HERE, name + ".npz"), grid=np.array([numr, numz, numphi, isym, mmax]),
                            dr=dr, seed=seed, rho=rho, cold=cold, warm=warm, S_warm=S,
                            green_m0=G[0, :4], green_mlast=G[-1, :4])
        o.close()
        print(name, os.path.getsize(os.path.join(HERE, name + ".npz")), "bytes")


if __name__ == "__main__":
    main()
