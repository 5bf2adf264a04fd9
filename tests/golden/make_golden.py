"""Regenerate the golden residual vectors in this directory from the oracle.

Run from the repository root:  python tests/golden/make_golden.py
The vectors freeze the oracle's output (state, residual, limiters) for two
small cases so that any change to the restatement is caught by
tests/test_oracle.py::test_golden_vectors.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from freecfd_b200 import cases  # noqa: E402


def main():
    for name, case in (("wedge_12x6", cases.wedge_case(ni=12, nj=6)),
                       ("hypersonic_16x8", cases.hypersonic_case(ntheta=16, nr=8))):
        o = oracle.Oracle(case)
        out = o.residual(case.state, full=True)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), W=case.state, R=out["R"], limiter=out["limiter"],
                            grads=out["grads"], mdot=out["mdot"])
        print(name, out["R"].shape)


if __name__ == "__main__":
    main()
