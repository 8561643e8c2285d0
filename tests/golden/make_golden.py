"""Regenerate the golden fixtures of tests/golden_cases.py from the CPU oracle.

    python tests/golden/make_golden.py

Writes one compressed .npz per case next to this script.
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "tests"), os.path.join(ROOT, "oracle")]

import numpy as np  # noqa: E402

import golden_cases as G  # noqa: E402
import oracle  # noqa: E402


def main():
    oracle.build()
    for name, fn in G.CASES.items():
        out = fn(oracle)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **out)
        print(path, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
