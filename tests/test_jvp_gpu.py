"""Forward-tangent (JVP) kernels against the oracle's complex-step derivative
(h = 1e-30, exact to rounding) and against FP64 central differences (h = 1e-7,
the check of the adjoint/JVP benchmark case).

Both the JVP and complex step differentiate the same discrete residual, branch
for branch, so they agree to rounding; central differences only agree where
the residual is smooth along the direction (no limiter switch inside +-h)."""
import numpy as np
import pytest

from tests.util import ELEMENTS, SMALL, build_pair, rel_err, res_err


def _dirs(shape, seed, n):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        v = rng.standard_normal(shape)
        out.append(v / np.linalg.norm(v))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("family", sorted(SMALL))
@pytest.mark.parametrize("flux,limiter", [("Roe", "vk"), ("AUSM+up", "minmod"), ("vanLeer", "vk"), ("Roe", "none"),
                                          ("SD-SLAU", "vk"), ("SW", "vk"), ("SW", "minmod")])
def test_jvp_matches_complex_step(family, flux, limiter, oracle_mod, fb):
    case = SMALL[family](flux=flux, limiter=limiter)
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    scale = np.abs(case.state).max(axis=0)
    for V in _dirs(case.state.shape, 99, 2):
        V = V * scale
        R, jv = ns.jvp(case.state, V, with_residual=True)
        cs_ref = o.residual_cstep(case.state, V)
        # the residual riding on the tangent chain against the plain residual
        # chain (on small meshes a two-warp gradient kernel with a different
        # summation order): momentum components share one scale, since the
        # z-momentum of the one-layer meshes is rounding noise
        assert res_err(R, ns.residual(case.state)).max() <= 1e-13
        cols = [k for k in range(5) if np.abs(cs_ref[:, k]).max() > 1e-12 * np.abs(cs_ref).max()]
        err = rel_err(jv[:, cols], cs_ref[:, cols])
        assert err.max() <= 1e-10, err


@pytest.mark.gpu
def test_jvp_matches_central_difference(oracle_mod, fb):
    """32 unit-norm seeded Gaussian directions (seed 99) on the cylinder mesh
    family, in-plane, with an unlimited AUSM+up residual (smooth)."""
    case = SMALL["cylinder"](flux="AUSM+up", limiter="none")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    scale = np.abs(case.state).max(axis=0) * np.array([1, 1, 1, 0, 1])
    worst = 0.0
    for V in _dirs(case.state.shape, 99, 32):
        V = V * scale
        jv = ns.jvp(case.state, V)
        h = 1e-7
        fd = (ns.residual(case.state + h * V) - ns.residual(case.state - h * V)) / (2 * h)
        cols = [0, 1, 2, 4]
        worst = max(worst, rel_err(jv[:, cols], fd[:, cols]).max())
    assert worst <= 1e-6, worst


@pytest.mark.gpu
def test_jvp_linearity(oracle_mod, fb):
    case = SMALL["wedge"](flux="Roe", limiter="vk")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    a, b = _dirs(case.state.shape, 5, 2)
    ja, jb = ns.jvp(case.state, a), ns.jvp(case.state, b)
    jab = ns.jvp(case.state, 2.0 * a - 3.0 * b)
    assert rel_err(jab, 2.0 * ja - 3.0 * jb).max() <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("family", sorted(SMALL))
def test_fp32_tangent_chain(family, oracle_mod, fb):
    """The FP32 tangent chain (mixed-precision Newton-Krylov) agrees with the
    FP64 tangent to single-precision accuracy: <= 1e-4 normwise per equation
    (the state itself is rounded to FP32, ~6e-8 relative, and the flux
    Jacobian amplifies that by the cancellation in the face differences)."""
    case = SMALL[family](limiter="none")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    scale = np.abs(case.state).max(axis=0) * np.array([1, 1, 1, 0, 1])
    for V in _dirs(case.state.shape, 17, 2):
        V = V * scale
        j64 = ns.jvp(case.state, V)
        j32 = ns.jvp(case.state, V, fp32=True)
        cols = [0, 1, 2, 4]
        err = rel_err(j32[:, cols], j64[:, cols])
        assert err.max() <= 1e-4, err


@pytest.mark.gpu
@pytest.mark.parametrize("family", sorted(ELEMENTS))
@pytest.mark.parametrize("flux", ["Roe", "SD-SLAU", "SW"])
def test_jvp_tets_pyramids(family, flux, oracle_mod, fb):
    """Tangent kernels on tetrahedra and pyramids vs the complex step."""
    case = ELEMENTS[family](flux=flux, limiter="vk")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    scale = np.abs(case.state).max(axis=0)
    for V in _dirs(case.state.shape, 23, 2):
        V = V * scale
        jv = ns.jvp(case.state, V)
        ref = o.residual_cstep(case.state, V)
        assert rel_err(jv, ref).max() <= 1e-10
