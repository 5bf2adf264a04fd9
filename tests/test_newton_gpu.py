"""Device Newton-Krylov solve (pseudo-transient, block-Jacobi + GMRES).

The converged state is a steady solution of the reference discretisation: the
oracle's residual there is below the tolerance; plain FP64 (finite-difference
J.v) and tangent-kernel / FP32-Krylov runs reach the same state."""
import numpy as np
import pytest

from freecfd_b200 import cases
from tests.util import build_pair


def _setup(case, oracle_mod, fb):
    o, cs, m = build_pair(case, oracle_mod, fb)
    return o, fb.NavierStokes(m, cs, 0)


@pytest.mark.gpu
@pytest.mark.parametrize("jvp,fp32", [(False, False), (True, False), (True, True)])
def test_newton_wedge_converges(jvp, fp32, oracle_mod, fb):
    case = cases.wedge_case(ni=30, nj=15)
    o, ns = _setup(case, oracle_mod, fb)
    W, rep = ns.newton_solve(case.state, tol=1e-10, max_newton=300, jvp=jvp, fp32_krylov=fp32, cfl0=5.0,
                             cfl_max=1e5, krylov_rtol=1e-3)
    assert rep["status"] == 0, rep
    r0 = np.linalg.norm(o.residual(case.state)[:, 0])
    r = np.linalg.norm(o.residual(W)[:, 0])
    assert r <= 1e-9 * r0


@pytest.mark.gpu
def test_newton_variants_agree(oracle_mod, fb):
    case = cases.cylinder_case(ntheta=32, nr=16, limiter="none")
    o, ns = _setup(case, oracle_mod, fb)
    kw = dict(tol=1e-10, max_newton=400, cfl0=2.0, cfl_max=1e5, krylov_rtol=1e-3)
    Wa, ra = ns.newton_solve(case.state, jvp=False, **kw)
    Wb, rb = ns.newton_solve(case.state, jvp=True, fp32_krylov=True, **kw)
    scale = np.abs(Wa).max(axis=0)
    assert (np.abs(Wa - Wb).max(axis=0) / scale).max() <= 1e-8
    r0 = np.linalg.norm(o.residual(case.state)[:, 0])
    assert np.linalg.norm(o.residual(Wb)[:, 0]) <= 1e-9 * r0
