"""k-omega RANS residual (config: turbulent flat plate) against the oracle.

The device evaluates the NS residual with the eddy viscosity in the viscous
flux and the k, omega right-hand side of RANS::terms (rans_terms.cc:39-275);
the oracle restates the same code on the CPU.  Gradients of k and omega use
the fused LSQ form on the device, so the bar is the residual's: 1e-12
normwise relative per equation."""
import numpy as np
import pytest

from freecfd_b200 import cases
from tests.util import build_pair, res_err


def _plate(**kw):
    return cases.plate_case(turbulent=True, **kw)


def _krel(a, b):
    b = np.asarray(b)
    return np.abs(np.asarray(a) - b).max(axis=0) / np.abs(b).max(axis=0)


@pytest.mark.gpu
def test_rans_bc_values(oracle_mod, fb):
    case = _plate(ni=8, nj=4, nk=2)
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    got, ref = ns.rans_bcs(), o.rans_bcs()
    assert np.array_equal(got[:, [0, 3]], ref[:, [0, 3]])
    assert np.abs(got - ref).max() <= 1e-15 * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("size,limiter,flux", [((8, 4, 2), "vk", "Roe"), ((24, 12, 3), "vk", "Roe"),
                                               ((24, 12, 3), "none", "AUSM+up"), ((24, 12, 3), "minmod", "vanLeer"),
                                               ((24, 12, 3), "vk", "SD-SLAU"), ((24, 12, 3), "vk", "SW")])
def test_rans_residual_parity(size, limiter, flux, oracle_mod, fb):
    ni, nj, nk = size
    case = _plate(ni=ni, nj=nj, nk=nk, limiter=limiter, flux=flux)
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    R, RK = ns.rans_residual(case.state, case.kstate)
    Ro, RKo = o.rans_residual(case.state, case.kstate)
    # Steger-Warming: split-flux rounding grows like 1/M (test_residual_gpu.tol)
    t = 1e-11 if flux == "SW" else 1e-12
    assert res_err(R, Ro).max() <= t
    assert _krel(RK, RKo).max() <= t, _krel(RK, RKo)
    # the eddy viscosity changes the NS residual (it is really coupled)
    assert np.abs(R - ns.residual(case.state)).max() > 1e-6 * np.abs(R).max()


@pytest.mark.gpu
def test_rans_residual_full_plate(oracle_mod, fb):
    """Configuration-sized plate 384x192x4 (294,912 cells)."""
    case = _plate()
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    R, RK = ns.rans_residual(case.state, case.kstate)
    Ro, RKo = o.rans_residual(case.state, case.kstate)
    assert res_err(R, Ro).max() <= 1e-12
    assert _krel(RK, RKo).max() <= 1e-12


@pytest.mark.gpu
def test_rans_rejects_laminar_case(fb, oracle_mod):
    case = cases.cylinder_case(ntheta=16, nr=8)
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    with pytest.raises(fb.FcfdError):
        ns.rans_residual(case.state, np.ones((m.nc, 2)))
