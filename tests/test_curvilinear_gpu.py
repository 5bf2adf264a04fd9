"""Curvilinear gradient maps on the device (the reference's default for
hexahedra and prisms).

The device sums the stored map weights w . phi in key order with rounded
operations, the reference's cell_gradient over its gradMap
(variable.h:194-202), so gradients are bit-exact wherever the ghost states
are and the noise-deciding limiters (minmod, Barth-Jespersen) decide as the
oracle does.  Bars: the residual's (1e-12 normwise per equation), the
tangent's against the oracle's complex step (1e-10), the adjoint's
dot-product identity (1e-11), the k-omega residual's (1e-12), and the
Newton solve reaching the oracle's 1e-10 residual drop."""
import tempfile

import numpy as np
import pytest

from freecfd_b200 import cases
from tests.test_curvilinear import CURV
from tests.util import build_pair, rel_err, res_err


@pytest.mark.gpu
@pytest.mark.parametrize("family", sorted(CURV))
@pytest.mark.parametrize("flux,limiter", [("Roe", "vk"), ("AUSM+up", "minmod"), ("vanLeer", "bj"), ("SD-SLAU", "none")])
def test_curvilinear_residual_parity(family, flux, limiter, oracle_mod, fb):
    case = CURV[family](flux=flux, limiter=limiter)
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    R, ref = ns.residual(case.state), o.residual(case.state)
    assert res_err(R, ref).max() <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("family,limiter", [("cylinder", "vk"), ("hypersonic", "minmod"), ("box_tet", "vk")])
def test_curvilinear_jvp_matches_complex_step(family, limiter, oracle_mod, fb):
    case = CURV[family](limiter=limiter)
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    W = case.state.copy()
    rng = np.random.default_rng(5)
    W[:, 2] = 0.02 * W[:, 1] * rng.uniform(-1.0, 1.0, W.shape[0])
    scale = np.abs(W).max(axis=0)
    V = rng.standard_normal(W.shape) * scale
    jv = ns.jvp(W, V)
    ref = o.residual_cstep(W, V)
    cols = [k for k in range(5) if np.abs(ref[:, k]).max() > 1e-12 * np.abs(ref).max()]
    assert rel_err(jv[:, cols], ref[:, cols]).max() <= 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("family", ["cylinder", "hypersonic", "plate", "box_hexpyr"])
def test_curvilinear_vjp_dot_product(family, oracle_mod, fb):
    """<Rbar, J V> (oracle complex step) = <J^T Rbar, V>: the adjoint's
    transposed map uses the stored weights."""
    case = CURV[family]()
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    W = case.state.copy()
    rng = np.random.default_rng(3)
    W[:, 2] = 0.02 * W[:, 1] * rng.uniform(-1.0, 1.0, W.shape[0])
    scale = np.abs(W).max(axis=0)
    for _ in range(2):
        V = rng.standard_normal(W.shape) * scale
        Rb = rng.standard_normal(W.shape)
        jv = o.residual_cstep(W, V)
        wb = ns.vjp(W, Rb)
        lhs, rhs = float((Rb * jv).sum()), float((wb * V).sum())
        mag = float(np.abs(Rb * jv).sum())
        assert abs(lhs - rhs) <= 1e-11 * mag, (lhs, rhs, mag)


@pytest.mark.gpu
def test_curvilinear_rans_residual(oracle_mod, fb):
    """k-omega plate with curvilinear maps: the k, omega gradients use the
    stored weights too (RANS::calc_cell_grads over the same gradMap)."""
    case = cases.plate_case(ni=24, nj=12, nk=3, turbulent=True, grad="curvilinear")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    R, RK = ns.rans_residual(case.state, case.kstate)
    Ro, RKo = o.rans_residual(case.state, case.kstate)
    assert res_err(R, Ro).max() <= 1e-12
    krel = np.abs(RK - RKo).max(axis=0) / np.abs(RKo).max(axis=0)
    assert krel.max() <= 1e-12, krel


@pytest.mark.gpu
def test_curvilinear_rans_vjp_dot_product(oracle_mod, fb):
    """Adjoint of the coupled k-omega residual on curvilinear maps (the flow
    and the k, omega gradients' transposed maps use the stored weights):
    <(Rbar, RKbar), J (V, VK)> with J (V, VK) from the oracle's complex step
    equals <J^T (Rbar, RKbar), (V, VK)>."""
    case = cases.plate_case(ni=24, nj=12, nk=3, turbulent=True, grad="curvilinear")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    W = case.state.copy()
    rng = np.random.default_rng(43)
    W[:, 2] = 0.02 * W[:, 1] * rng.uniform(-1.0, 1.0, W.shape[0])
    K = case.kstate
    for _ in range(2):
        V = rng.standard_normal(W.shape) * np.abs(W).max(axis=0)
        VK = rng.standard_normal(K.shape) * np.abs(K).max(axis=0)
        dR, dRK = o.rans_residual_cstep(W, K, V, VK)
        Rb = rng.standard_normal(W.shape)
        RKb = rng.standard_normal(K.shape) * np.abs(dR).max() / np.abs(dRK).max()
        Wb, Kb = ns.rans_vjp(W, K, Rb, RKb)
        lhs = float((Rb * dR).sum() + (RKb * dRK).sum())
        rhs = float((Wb * V).sum() + (Kb * VK).sum())
        mag = float(np.abs(Rb * dR).sum() + np.abs(RKb * dRK).sum())
        assert abs(lhs - rhs) <= 1e-11 * mag, (lhs, rhs, mag)


@pytest.mark.gpu
def test_curvilinear_newton_converges(oracle_mod, fb):
    """Laminar cylinder 64x32 with the default (curvilinear) hexahedron
    gradients, unlimited: the plain FP64 and mixed Newton arms reach a 1e-10
    drop of the oracle's mass residual."""
    case = cases.cylinder_case(ntheta=64, nr=32, limiter="none", grad="curvilinear")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    r0 = np.linalg.norm(o.residual(case.state)[:, 0])
    for opts in (dict(jvp=False), dict(jvp=True, fp32_jvp=True, fp32_krylov=True)):
        W, rep = ns.newton_solve(case.state, tol=1e-10, max_newton=300, cfl0=2.0, cfl_max=1e6, krylov_rtol=1e-3,
                                 precond_sweeps=4, krylov_cycles=3, **opts)
        assert rep["status"] == 0, rep
        assert np.linalg.norm(o.residual(W)[:, 0]) <= 1e-9 * r0
