"""Regenerate tests/golden/*.npz from the CPU oracle.

The reference (Julia) cannot be executed in this environment, so these fixtures are oracle
outputs on the `ring64` workload (single ring, 64 nodes); the oracle itself is pinned to the
reference's known-answer tests in tests/test_oracle.py.  Run: python tests/golden/make_golden.py
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE.parent))

from conftest import load_package  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    vp = load_package()
    fs, p = vp.configs.ring64()
    v, psi, st = O.compute_on_nodes(p, fs, streamfunction=True)


    np.savez_compressed(HERE / "ring64.npz", nodes=np.concatenate(fs), velocity=v, streamfunction=psi,
                        pairs_in_range=st["pairs_in_range"])


if __name__ == "__main__":
    main()
