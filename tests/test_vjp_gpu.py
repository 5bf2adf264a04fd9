"""Adjoint (VJP) kernels of the residual and the boundary-load gradient.

The VJP transposes the same discrete residual the JVP differentiates (the
branches taken at W), so on small meshes J^T Rbar is compared entry by entry
with the transpose of the Jacobian assembled column by column from the
oracle's complex step (h = 1e-30, exact to rounding), and on larger ones by
the dot-product identity <Rbar, J V> = <J^T Rbar, V>.  The load gradient
(the adjoint/JVP benchmark check on the laminar cylinder at a converged
state) is compared with the oracle's complex-step loads and with FP64 central
differences (h = 1e-7) along 32 seeded unit Gaussian directions."""
import numpy as np
import pytest

from freecfd_b200 import cases
from tests.util import SMALL, build_pair

TINY = {
    "wedge": lambda **kw: cases.wedge_case(ni=12, nj=6, **kw),
    "cylinder": lambda **kw: cases.cylinder_case(ntheta=16, nr=8, **kw),
    "hypersonic": lambda **kw: cases.hypersonic_case(ntheta=16, nr=8, **kw),
    "plate": lambda **kw: cases.plate_case(ni=8, nj=4, nk=2, turbulent=False, **kw),
}


def _generic(case, seed=3):
    """The seeded states have v = w = 0 exactly (freestream along x).  Where
    two such zeros meet in a product (the minmod test dU * dUg < 0), the
    complex step's h^2 cross term decides the branch and its derivative is no
    longer that of the real computation; give v a small seeded perturbation
    so every comparison is decided by the real parts alone."""
    W = case.state.copy()
    rng = np.random.default_rng(seed)
    W[:, 2] = 0.02 * W[:, 1] * rng.uniform(-1.0, 1.0, W.shape[0])
    return W


def _jacobian_cs(o, W):
    """Dense dR/dW ([5nc] x [5nc], AoS order) from complex-step columns."""
    nc = W.shape[0]
    J = np.empty((5 * nc, 5 * nc))
    e = np.zeros((nc, 5))
    for k in range(5 * nc):
        e.flat[k] = 1.0
        J[:, k] = o.residual_cstep(W, e).ravel()
        e.flat[k] = 0.0
    return J


@pytest.mark.gpu
@pytest.mark.parametrize("family,flux,limiter", [("wedge", "Roe", "vk"), ("wedge", "AUSM+up", "minmod"),
                                                 ("wedge", "vanLeer", "bj"), ("cylinder", "Roe", "vk"),
                                                 ("cylinder", "AUSM+up", "none"), ("hypersonic", "AUSM+up", "minmod"),
                                                 ("plate", "Roe", "vk"), ("wedge", "SD-SLAU", "minmod"),
                                                 ("cylinder", "SW", "vk"), ("hypersonic", "SW", "none"),
                                                 ("plate", "SD-SLAU", "vk")])
def test_vjp_matches_jacobian_transpose(family, flux, limiter, oracle_mod, fb):
    case = TINY[family](flux=flux, limiter=limiter)
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    W = _generic(case)
    J = _jacobian_cs(o, W)
    rng = np.random.default_rng(7)
    for _ in range(2):
        Rb = rng.standard_normal(W.shape)
        ref = (J.T @ Rb.ravel()).reshape(W.shape)
        got = ns.vjp(W, Rb)
        # per-variable scale: the largest |J^T Rbar| entry of that variable
        scale = np.maximum(np.abs(ref).max(axis=0), 1e-300)
        # w is an inert direction on one-layer meshes (its column is noise)
        cols = [k for k in range(5) if np.abs(ref[:, k]).max() > 1e-9 * np.abs(ref).max()]
        err = (np.abs(got - ref).max(axis=0) / scale)[cols]
        assert err.max() <= 1e-9, (err, cols)


@pytest.mark.gpu
@pytest.mark.parametrize("family", sorted(SMALL))
def test_vjp_dot_product(family, oracle_mod, fb):
    """<Rbar, J V> (oracle complex step) = <J^T Rbar, V> on the parity meshes."""
    case = SMALL[family]()
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    W = _generic(case)
    rng = np.random.default_rng(11)
    scale = np.abs(W).max(axis=0)
    for _ in range(3):
        V = rng.standard_normal(W.shape) * scale
        Rb = rng.standard_normal(W.shape)
        jv = o.residual_cstep(W, V)
        wb = ns.vjp(W, Rb)
        lhs, rhs = float((Rb * jv).sum()), float((wb * V).sum())
        mag = float(np.abs(Rb * jv).sum())
        assert abs(lhs - rhs) <= 1e-11 * mag, (lhs, rhs, mag)


@pytest.mark.gpu
@pytest.mark.parametrize("family,limiter", [("wedge", "vk"), ("cylinder", "vk"), ("hypersonic", "minmod"),
                                            ("plate", "bj")])
def test_vjp_is_deterministic(family, limiter, oracle_mod, fb):
    """Every accumulation of the reverse sweep has a fixed order (limiter
    neighbours gathered per face side, stale densities summed per target in
    outlet order), so repeated adjoints are the same bits; the wedge's
    outlet leaves its right density to the state cache (the stale-density
    path)."""
    case = SMALL[family](limiter=limiter)
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    W = _generic(case)
    Rb = np.random.default_rng(13).standard_normal(W.shape)
    first = ns.vjp(W, Rb)
    for _ in range(4):
        assert np.array_equal(ns.vjp(W, Rb), first)


@pytest.mark.gpu
def test_vjp_agrees_with_device_jvp(fb, oracle_mod):
    """The forward/backward pair is consistent on the device alone."""
    case = SMALL["hypersonic"]()
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    W = case.state
    rng = np.random.default_rng(5)
    V = rng.standard_normal(W.shape) * np.abs(W).max(axis=0)
    Rb = rng.standard_normal(W.shape)
    lhs = float((Rb * ns.jvp(W, V)).sum())
    rhs = float((ns.vjp(W, Rb) * V).sum())
    assert abs(lhs - rhs) <= 1e-11 * float(np.abs(Rb * ns.jvp(W, V)).sum())


@pytest.fixture(scope="module")
def converged_cylinder(oracle_mod, fb):
    """Laminar cylinder 256x128x1 (Roe, unlimited second order) driven to
    |R_mass| <= 1e-10 |R_mass0|.  Unlimited: at a steady state the VK
    limiter's decisions sit on rounding-level gradients in the far field, where
    the device's and the oracle's last bits pick different branches."""
    case = cases.cylinder_case(limiter="none")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    W, rep = ns.newton_solve(case.state, tol=1e-10, max_newton=400, cfl0=2.0, cfl_max=1e6, krylov_rtol=1e-3,
                             precond_sweeps=4, krylov_cycles=3, jvp=False)
    return case, o, ns, W


@pytest.mark.gpu
def test_drag_and_gradient_converged_cylinder(converged_cylinder):
    """Wall force vs the oracle's loads; d(drag)/dW along 32 seeded unit
    Gaussian directions vs the oracle's complex step and FP64 central
    differences (h = 1e-7) of the device force."""
    case, o, ns, W = converged_cylinder
    F, G = ns.drag(W, [0], (1.0, 0.0, 0.0))
    Fo = o.loads(W)[0]
    assert np.abs(F - Fo).max() <= 1e-12 * np.abs(Fo).max()
    rng = np.random.default_rng(99)
    scale = np.abs(W).max(axis=0) * np.array([1, 1, 1, 0, 1])
    worst_cs, worst_fd = 0.0, 0.0
    for _ in range(32):
        V = rng.standard_normal(W.shape)
        V = V / np.linalg.norm(V) * scale
        adj = float((G * V).sum())
        cs_ = float(o.loads(W, V)[0, 0])
        h = 1e-7
        fd = (ns.drag(W + h * V, [0], gradient=False)[0][0] - ns.drag(W - h * V, [0], gradient=False)[0][0]) / (2 * h)
        ref = max(abs(cs_), 1e-12 * abs(Fo[0]))
        worst_cs = max(worst_cs, abs(adj - cs_) / ref)
        worst_fd = max(worst_fd, abs(adj - fd) / ref)
    assert worst_cs <= 1e-10, worst_cs
    # central differences of a force dominated by the absolute-pressure
    # integral (|F| ~ 1e4 x its directional derivative): rounding of F alone
    # is ~1e-16 |F| / h, so the difference quotient is good to ~1e-5
    assert worst_fd <= 1e-4, worst_fd


@pytest.mark.gpu
def test_jvp_converged_cylinder_32_directions(converged_cylinder):
    """JVP at the converged state vs complex step and central differences."""
    case, o, ns, W = converged_cylinder
    rng = np.random.default_rng(99)
    scale = np.abs(W).max(axis=0) * np.array([1, 1, 1, 0, 1])
    worst_cs, worst_fd = 0.0, 0.0
    cols = [0, 1, 2, 4]
    for _ in range(32):
        V = rng.standard_normal(W.shape)
        V = V / np.linalg.norm(V) * scale
        jv = ns.jvp(W, V)
        cs_ = o.residual_cstep(W, V)
        h = 1e-7
        fd = (ns.residual(W + h * V) - ns.residual(W - h * V)) / (2 * h)
        s = np.abs(cs_[:, cols]).max(axis=0)
        worst_cs = max(worst_cs, (np.abs(jv - cs_)[:, cols].max(axis=0) / s).max())
        worst_fd = max(worst_fd, (np.abs(jv - fd)[:, cols].max(axis=0) / s).max())
    assert worst_cs <= 1e-10, worst_cs
    assert worst_fd <= 1e-5, worst_fd
