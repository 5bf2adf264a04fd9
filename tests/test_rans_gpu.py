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


def _generic(case, seed=3):
    """Seeded state with v perturbed too, so no face sits on a |V.n| = 0 or
    limiter tie (the complex step decides those by the h^2 term)."""
    W = case.state.copy()
    rng = np.random.default_rng(seed)
    W[:, 2] = 0.02 * W[:, 1] * rng.uniform(-1.0, 1.0, W.shape[0])
    return W


@pytest.mark.gpu
@pytest.mark.parametrize("size,limiter,flux", [((8, 4, 2), "vk", "Roe"), ((12, 6, 3), "none", "AUSM+up"),
                                               ((12, 6, 3), "minmod", "vanLeer"), ((12, 6, 3), "vk", "SD-SLAU")])
def test_rans_jvp_matches_complex_step(size, limiter, flux, oracle_mod, fb):
    """Tangent of the coupled NS + k-omega residual (dual numbers through the
    eddy viscosity, the k-omega fluxes and sources) against the oracle's
    complex step (h = 1e-30) along seeded directions in (W, K)."""
    ni, nj, nk = size
    case = _plate(ni=ni, nj=nj, nk=nk, limiter=limiter, flux=flux)
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    W, K = _generic(case), case.kstate
    rng = np.random.default_rng(17)
    for _ in range(2):
        V = rng.standard_normal(W.shape) * np.abs(W).max(axis=0) * 1e-3
        VK = rng.standard_normal(K.shape) * np.abs(K).max(axis=0) * 1e-3
        R, RK, JV, JVK = ns.rans_jvp(W, K, V, VK, with_residual=True)
        R0, RK0 = ns.rans_residual(W, K)
        assert res_err(R, R0).max() <= 1e-13 and _krel(RK, RK0).max() <= 1e-13
        dR, dRK = o.rans_residual_cstep(W, K, V, VK)
        cols = [k for k in range(5) if np.abs(dR[:, k]).max() > 1e-12 * np.abs(dR).max()]
        err = np.abs(JV - dR)[:, cols].max(axis=0) / np.abs(dR[:, cols]).max(axis=0)
        assert err.max() <= 1e-10, err
        assert _krel(JVK, dRK).max() <= 1e-10, _krel(JVK, dRK)


@pytest.mark.gpu
def test_rans_jvp_matches_central_difference(oracle_mod, fb):
    """The tangent against FP64 central differences (h = 1e-6) of the device's
    own coupled residual, limiter off (smooth), 8 seeded directions."""
    case = _plate(ni=16, nj=8, nk=2, limiter="none", flux="Roe")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    W, K = _generic(case), case.kstate
    rng = np.random.default_rng(23)
    worst = 0.0
    for _ in range(8):
        V = rng.standard_normal(W.shape) * np.abs(W).max(axis=0) * np.array([1, 1, 1, 0, 1]) * 1e-3
        VK = rng.standard_normal(K.shape) * np.abs(K).max(axis=0) * 1e-3
        JV, JVK = ns.rans_jvp(W, K, V, VK)
        h = 1e-6
        Rp, RKp = ns.rans_residual(W + h * V, K + h * VK)
        Rm, RKm = ns.rans_residual(W - h * V, K - h * VK)
        fd, fdk = (Rp - Rm) / (2 * h), (RKp - RKm) / (2 * h)
        cols = [0, 1, 2, 4]
        worst = max(worst, (np.abs(JV - fd)[:, cols].max(axis=0) / np.abs(fd[:, cols]).max(axis=0)).max(),
                    _krel(JVK, fdk).max())
    assert worst <= 1e-5, worst


@pytest.mark.gpu
def test_rans_jvp_fp32(oracle_mod, fb):
    """The FP32 tangent chain of the coupled residual (mixed-precision inner
    products) agrees with the FP64 tangent to single-precision accuracy:
    <= 1e-4 normwise per equation."""
    case = _plate(ni=16, nj=8, nk=2, limiter="none", flux="Roe")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    W, K = _generic(case), case.kstate
    rng = np.random.default_rng(29)
    for _ in range(2):
        V = rng.standard_normal(W.shape) * np.abs(W).max(axis=0) * np.array([1, 1, 1, 0, 1]) * 1e-3
        VK = rng.standard_normal(K.shape) * np.abs(K).max(axis=0) * 1e-3
        JV, JVK = ns.rans_jvp(W, K, V, VK)
        JV32, JVK32 = ns.rans_jvp(W, K, V, VK, fp32=True)
        cols = [0, 1, 2, 4]
        err = np.abs(JV32 - JV)[:, cols].max(axis=0) / np.abs(JV[:, cols]).max(axis=0)
        assert err.max() <= 1e-4, err
        assert _krel(JVK32, JVK).max() <= 1e-4, _krel(JVK32, JVK)


@pytest.mark.gpu
def test_coupled_komega_newton(fb):
    """The coupled flow + k-omega Newton-Krylov solve on a small plate: from
    the seeded state both arms (FP64 finite-difference J.v, FP32 tangent)
    drop the mass and energy residuals by three orders, the momentum residual
    by two and the k and omega residuals by more than half within 150 steps,
    keep k, omega positive, and give the same wall skin-friction drag to
    1e-3.  (The solve does not reach machine-level convergence: the k and
    omega residuals level off near 1e-2 of their initial values.)"""
    case = cases.plate_case(ni=48, nj=24, nk=2)
    cs = fb.Case.from_case(case)
    m = fb.Mesh(case.mesh, cs)
    drag = {}
    for label, kw in (("plain", {}), ("mixed", dict(fp32_jvp=True))):
        ns = fb.NavierStokes(m, cs, 0)
        W, K, rep = ns.rans_newton_solve(case.state, case.kstate, tol=1e-10, max_newton=150, cfl0=1.0, krylov_dim=40,
                                         krylov_rtol=1e-2, cfl_mode=2, stop_all_rows=True, raise_on_fail=False, **kw)
        r = rep["rows_final"]
        assert r[0] <= 1e-3 and r[2] <= 1e-3 and r[1] <= 1e-2, r
        assert max(rep["kw_final"]) <= 0.5, rep["kw_final"]
        assert np.isfinite(W).all() and (K > 0).all()
        drag[label] = ns.drag(W, [2], (1.0, 0.0, 0.0), gradient=False)[0][0]
    assert abs(drag["mixed"] - drag["plain"]) <= 1e-3 * abs(drag["plain"])


def _rans_jacobian_cs(o, W, K):
    """Dense d(R, RK)/d(W, K) ([7nc] x [7nc]; rows and columns ordered
    (W AoS, then K AoS)) from the oracle's complex-step columns."""
    nc = W.shape[0]
    n = 7 * nc
    J = np.empty((n, n))
    eW, eK = np.zeros((nc, 5)), np.zeros((nc, 2))
    for k in range(n):
        e = eW if k < 5 * nc else eK
        i = k if k < 5 * nc else k - 5 * nc
        e.flat[i] = 1.0
        dR, dRK = o.rans_residual_cstep(W, K, eW, eK)
        J[:, k] = np.concatenate([dR.ravel(), dRK.ravel()])
        e.flat[i] = 0.0
    return J


@pytest.mark.gpu
@pytest.mark.parametrize("limiter,flux", [("vk", "Roe"), ("none", "AUSM+up"), ("minmod", "vanLeer"), ("bj", "SD-SLAU")])
def test_rans_vjp_matches_jacobian_transpose(limiter, flux, oracle_mod, fb):
    """Adjoint of the coupled residual entry by entry against the transpose of
    the Jacobian assembled from the oracle's complex step (8x4x2 plate: inlet
    with fixed k, omega and mu_t, no-slip wall with mu_t = 0, outlet,
    symmetry)."""
    case = _plate(ni=8, nj=4, nk=2, limiter=limiter, flux=flux)
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    W, K = _generic(case), case.kstate
    J = _rans_jacobian_cs(o, W, K)
    nc = m.nc
    rng = np.random.default_rng(31)
    for _ in range(2):
        Rb, RKb = rng.standard_normal((nc, 5)), rng.standard_normal((nc, 2))
        ref = J.T @ np.concatenate([Rb.ravel(), RKb.ravel()])
        rW, rK = ref[:5 * nc].reshape(nc, 5), ref[5 * nc:].reshape(nc, 2)
        Wb, Kb = ns.rans_vjp(W, K, Rb, RKb)
        cols = [k for k in range(5) if np.abs(rW[:, k]).max() > 1e-9 * np.abs(rW).max()]
        errW = (np.abs(Wb - rW).max(axis=0) / np.maximum(np.abs(rW).max(axis=0), 1e-300))[cols]
        errK = np.abs(Kb - rK).max(axis=0) / np.abs(rK).max(axis=0)
        assert errW.max() <= 1e-9 and errK.max() <= 1e-9, (errW, errK)


@pytest.mark.gpu
@pytest.mark.parametrize("size,limiter,flux", [((24, 12, 3), "vk", "Roe"), ((24, 12, 3), "minmod", "AUSM+up"),
                                               ((24, 12, 3), "vk", "SW")])
def test_rans_vjp_dot_product(size, limiter, flux, oracle_mod, fb):
    """<(Rbar, RKbar), J (V, VK)> with J (V, VK) from the oracle's complex
    step equals <J^T (Rbar, RKbar), (V, VK)> from the device adjoint."""
    ni, nj, nk = size
    case = _plate(ni=ni, nj=nj, nk=nk, limiter=limiter, flux=flux)
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    W, K = _generic(case), case.kstate
    rng = np.random.default_rng(37)
    for _ in range(3):
        V = rng.standard_normal(W.shape) * np.abs(W).max(axis=0)
        VK = rng.standard_normal(K.shape) * np.abs(K).max(axis=0)
        Rb, RKb = rng.standard_normal(W.shape), rng.standard_normal(K.shape)
        # scale the k-omega seed so both halves weigh alike in the sums
        dR, dRK = o.rans_residual_cstep(W, K, V, VK)
        RKb *= np.abs(dR).max() / np.abs(dRK).max()
        Wb, Kb = ns.rans_vjp(W, K, Rb, RKb)
        lhs = float((Rb * dR).sum() + (RKb * dRK).sum())
        rhs = float((Wb * V).sum() + (Kb * VK).sum())
        mag = float(np.abs(Rb * dR).sum() + np.abs(RKb * dRK).sum())
        assert abs(lhs - rhs) <= 1e-11 * mag, (lhs, rhs, mag)


@pytest.mark.gpu
def test_rans_vjp_deterministic_and_pairs_with_jvp(oracle_mod, fb):
    """Repeated adjoints are the same bits (fixed-order accumulations), and
    the device pair (fcfd_rans_jvp, fcfd_rans_vjp) satisfies the dot-product
    identity on its own; the flow-only seed reaches K through the eddy
    viscosity."""
    case = _plate(ni=24, nj=12, nk=3)
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    W, K = _generic(case), case.kstate
    rng = np.random.default_rng(41)
    Rb, RKb = rng.standard_normal(W.shape), rng.standard_normal(K.shape)
    Wb, Kb = ns.rans_vjp(W, K, Rb, RKb)
    for _ in range(3):
        W2, K2 = ns.rans_vjp(W, K, Rb, RKb)
        assert np.array_equal(W2, Wb) and np.array_equal(K2, Kb)
    V = rng.standard_normal(W.shape) * np.abs(W).max(axis=0)
    VK = rng.standard_normal(K.shape) * np.abs(K).max(axis=0)
    JV, JVK = ns.rans_jvp(W, K, V, VK)
    lhs = float((Rb * JV).sum() + (RKb * JVK).sum())
    rhs = float((Wb * V).sum() + (Kb * VK).sum())
    assert abs(lhs - rhs) <= 1e-11 * float(np.abs(Rb * JV).sum() + np.abs(RKb * JVK).sum())
    _, Kf = ns.rans_vjp(W, K, Rb, np.zeros_like(RKb))
    assert np.abs(Kf).max() > 0.0


@pytest.mark.gpu
def test_rans_vjp_full_plate(fb):
    """At the full 384x192x4 plate the adjoint and the FP64 tangent of the
    coupled residual satisfy the dot-product identity along seeded
    directions, and repeated adjoints are the same bits."""
    case = cases.plate_case()
    cs = fb.Case.from_case(case)
    m = fb.Mesh(case.mesh, cs)
    ns = fb.NavierStokes(m, cs, 0)
    W, K = _generic(case), case.kstate
    rng = np.random.default_rng(47)
    Rb, RKb = rng.standard_normal(W.shape), rng.standard_normal(K.shape)
    Wb, Kb = ns.rans_vjp(W, K, Rb, RKb)
    W2, K2 = ns.rans_vjp(W, K, Rb, RKb)
    assert np.array_equal(W2, Wb) and np.array_equal(K2, Kb)
    for _ in range(2):
        V = rng.standard_normal(W.shape) * np.abs(W).max(axis=0)
        VK = rng.standard_normal(K.shape) * np.abs(K).max(axis=0)
        JV, JVK = ns.rans_jvp(W, K, V, VK)
        lhs = float((Rb * JV).sum() + (RKb * JVK).sum())
        rhs = float((Wb * V).sum() + (Kb * VK).sum())
        assert abs(lhs - rhs) <= 1e-11 * float(np.abs(Rb * JV).sum() + np.abs(RKb * JVK).sum())
