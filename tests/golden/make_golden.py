"""Regenerate the golden vectors in this directory from the reference itself.

Run from the repository root:  python tests/golden/make_golden.py
It needs the compiled reference, oracle/_ref/freecfd_ref (Free CFD's own
sources built with `make -C oracle ref`; see oracle/reference.py).  Each .npz
holds a seeded state and what the reference computes from it: the residual
(the rhs Vec of NavierStokes::assemble_linear_system), limiters, gradients,
mdot, ghost states, and for the k-omega plate the RANS::terms rhs; the wedge
file also holds time_terms' P V / dt blocks for seeded time steps.
tests/test_oracle.py::test_golden_vectors holds the oracle to these doubles,
so the pin survives on machines without the reference's sources.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from freecfd_b200 import cases  # noqa: E402
from oracle import reference  # noqa: E402

CASES = {
    "wedge_12x6": lambda: cases.wedge_case(ni=12, nj=6),
    "hypersonic_16x8": lambda: cases.hypersonic_case(ntheta=16, nr=8),
    "cylinder_16x8": lambda: cases.cylinder_case(ntheta=16, nr=8),
    "box_tet_4x3x2": lambda: cases.box_case("tet", nx=4, ny=3, nz=2),
    "plate_komega_8x4x2": lambda: cases.plate_case(ni=8, nj=4, nk=2),
}


def main():
    if not reference.build():
        raise SystemExit("the compiled reference is not available")
    for name, make in CASES.items():
        case = make()
        ref = reference.Reference(case)
        out = ref.residual(case.state, case.kstate)
        arrays = dict(W=case.state, R=out["R"], limiter=out["limiter"], grads=out["grads"], mdot=out["mdot"],
                      ghost=out["ghost"])
        if case.kstate is not None:
            arrays.update(K=case.kstate, RK=out["RK"])
        if name == "wedge_12x6":
            dt = np.random.default_rng(11).uniform(0.5, 2.0, case.state.shape[0]) * 1e-5
            arrays.update(dt=dt, time_terms=ref.time_terms(case.state, dt))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
        print(name, out["R"].shape)


if __name__ == "__main__":
    main()
