"""Device Newton-Krylov solve (pseudo-transient, block preconditioner, GMRES).

The converged state is a steady solution of the reference discretisation: the
oracle's residual there is below the tolerance; plain FP64 (finite-difference
J.v) and tangent-kernel / FP32-Krylov runs reach the same state."""
import numpy as np
import pytest

from freecfd_b200 import cases
from tests.util import build_pair

KW = dict(tol=1e-10, max_newton=300, cfl0=2.0, cfl_max=1e6, krylov_rtol=1e-3, precond_sweeps=4, krylov_cycles=3)


@pytest.fixture(scope="module")
def cylinder(oracle_mod, fb):
    """Laminar cylinder family (64x32), Roe, unlimited second order."""
    case = cases.cylinder_case(ntheta=64, nr=32, limiter="none")
    o, cs, m = build_pair(case, oracle_mod, fb)
    return case, o, fb.NavierStokes(m, cs, 0)


@pytest.fixture(scope="module")
def wedge(oracle_mod, fb):
    """Supersonic wedge (30x15) with the VK limiter, bit-exact gradients.

    The reference's VK limiter uses eps^2 = (1e-6 K range/L)^2, so at local
    extrema it switches between ~0 and 1 over a band far narrower than a Newton
    step; whether the pseudo-transient iteration settles or chatters depends on
    the path (CFL schedule, Krylov tolerance, rounding of the gradients).  The
    settings below converge; others stall with the limiter chattering."""
    case = cases.wedge_case(ni=30, nj=15)
    o, cs, m = build_pair(case, oracle_mod, fb)
    return case, o, fb.NavierStokes(m, cs, 0, exact_gradients=True)


@pytest.mark.gpu
@pytest.mark.parametrize("label,opts", [("fd64", dict(jvp=False)),
                                        ("jvp64", dict(jvp=True, exact_jvp=True)),
                                        ("jvp_fp32_krylov", dict(jvp=True, exact_jvp=True, fp32_krylov=True)),
                                        ("mixed_fp32_tangent", dict(jvp=True, fp32_jvp=True, fp32_krylov=True))])
def test_newton_cylinder_converges(label, opts, cylinder):
    case, o, ns = cylinder
    W, rep = ns.newton_solve(case.state, **KW, **opts)
    assert rep["status"] == 0, rep
    r0 = np.linalg.norm(o.residual(case.state)[:, 0])
    r = np.linalg.norm(o.residual(W)[:, 0])
    assert r <= 1e-9 * r0, (r, r0)


@pytest.mark.gpu
def test_newton_variants_agree(cylinder):
    """Plain FP64 (finite-difference J.v, FP64 Krylov) and mixed (FP32 tangent
    J.v, FP32 Krylov, FP64 outer residual) reach the same steady state: to 1e-7 relative, since the 1e-10
    residual tolerance bounds the state error only through the conditioning of
    the Jacobian."""
    case, o, ns = cylinder
    Wa, _ = ns.newton_solve(case.state, jvp=False, **KW)
    Wb, _ = ns.newton_solve(case.state, jvp=True, fp32_jvp=True, fp32_krylov=True, **KW)
    # velocity components share one scale: w is rounding noise on this
    # one-layer mesh and its own maximum would divide by ~0
    scale = np.abs(Wa).max(axis=0)
    scale[1:4] = np.abs(Wa[:, 1:4]).max()
    assert (np.abs(Wa - Wb).max(axis=0) / scale).max() <= 1e-7


@pytest.mark.gpu
def test_newton_wedge_shock_fd(wedge):
    """Supersonic wedge with the VK limiter: plain FP64 converges to 1e-10."""
    case, o, ns = wedge
    W, rep = ns.newton_solve(case.state, tol=1e-10, max_newton=300, cfl0=5.0, cfl_max=1e5, krylov_rtol=1e-3,
                             jvp=False)
    assert rep["status"] == 0, rep
    r0 = np.linalg.norm(o.residual(case.state)[:, 0])
    assert np.linalg.norm(o.residual(W)[:, 0]) <= 1e-9 * r0


@pytest.mark.gpu
def test_newton_reports_nonconvergence(wedge, fb):
    """An iteration cap is reported as FCFD_ERR_NOT_CONVERGED with the report filled."""
    case, o, ns = wedge
    W, rep = ns.newton_solve(case.state, tol=1e-10, max_newton=3, raise_on_fail=False)
    assert rep["status"] == 4 and rep["newton_iterations"] == 3
    with pytest.raises(fb.FcfdError) as e:
        ns.newton_solve(case.state, tol=1e-10, max_newton=3)
    assert e.value.code == 4


@pytest.mark.gpu
@pytest.mark.parametrize("flux", ["SD-SLAU", "SW"])
@pytest.mark.parametrize("label,opts", [("fd64", dict(jvp=False)),
                                        ("mixed_fp32_tangent", dict(jvp=True, fp32_jvp=True, fp32_krylov=True))])
def test_newton_other_fluxes(flux, label, opts, oracle_mod, fb):
    """SD-SLAU and Steger-Warming through the whole Newton path (their face
    Jacobian kernels in the block preconditioner, tangent kernels in J.v):
    laminar cylinder 48x24, unlimited second order."""
    case = cases.cylinder_case(ntheta=48, nr=24, limiter="none", flux=flux)
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    W, rep = ns.newton_solve(case.state, **KW, **opts)
    assert rep["status"] == 0, rep
    r0 = np.linalg.norm(o.residual(case.state)[:, 0])
    r = np.linalg.norm(o.residual(W)[:, 0])
    assert r <= 1e-9 * r0, (r, r0)


@pytest.mark.gpu
def test_newton_drag_coefficient(cylinder):
    """The wall drag at the converged states: the plain FP64 arm's against the
    oracle's loads at that state (1e-12), and the mixed arm's against the plain
    arm's (1e-6: the states agree to ~1e-7 relative)."""
    case, o, ns = cylinder
    Wa, _ = ns.newton_solve(case.state, jvp=False, **KW)
    Wb, _ = ns.newton_solve(case.state, jvp=True, fp32_jvp=True, fp32_krylov=True, **KW)
    Fa = ns.drag(Wa, [0], gradient=False)[0]
    Fb = ns.drag(Wb, [0], gradient=False)[0]
    Fo = o.loads(Wa)[0]
    assert np.abs(Fa - Fo).max() <= 1e-12 * np.abs(Fo).max()
    assert abs(Fb[0] - Fa[0]) <= 1e-6 * abs(Fa[0])


@pytest.mark.gpu
@pytest.mark.parametrize("family", ["cylinder", "box_hexpyr"])
@pytest.mark.parametrize("label,opts", [("fd64", dict(jvp=False)),
                                        ("mixed_fp32_tangent", dict(jvp=True, fp32_jvp=True, fp32_krylov=True))])
def test_gauss_seidel_persistent_matches_per_colour(family, label, opts, oracle_mod, fb):
    """The Gauss-Seidel sweeps as one cooperative launch per preconditioner
    application (grid barriers between colour updates, couplings staged in
    shared memory where they fit) against one launch per colour update: the
    same updates in the same order with the same arithmetic per (cell, row),
    so six Newton steps give the same states and Krylov iteration counts.
    Families: the cylinder (four neighbour slots, two colours) and a 3D
    box of hexes and pyramids (six slots, more colours)."""
    if family == "cylinder":
        case = cases.cylinder_case(ntheta=64, nr=32, limiter="none")
    else:
        case = cases.box_case(kind="hexpyr", nx=8, ny=6, nz=5, flux="Roe", limiter="none")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    kw = dict(KW, max_newton=6, precond_sweeps=8, raise_on_fail=False)
    Wa, ra = ns.newton_solve(case.state, gs_persistent=False, **kw, **opts)
    Wb, rb = ns.newton_solve(case.state, gs_persistent=True, **kw, **opts)
    assert ra["newton_iterations"] == rb["newton_iterations"] == 6
    assert ra["krylov_iterations"] == rb["krylov_iterations"], (ra["krylov_iterations"], rb["krylov_iterations"])
    scale = np.abs(Wa).max(axis=0)
    scale[1:4] = np.abs(Wa[:, 1:4]).max()
    err = (np.abs(Wa - Wb).max(axis=0) / scale).max()
    assert err <= 1e-13, err


@pytest.mark.gpu
@pytest.mark.parametrize("family", ["wedge", "box_hexpyr"])
@pytest.mark.parametrize("label,opts", [("fd64", dict(jvp=False)),
                                        ("mixed_fp32_tangent", dict(jvp=True, fp32_jvp=True, fp32_krylov=True))])
def test_newton_block_ilu0(family, label, opts, oracle_mod, fb):
    """Block ILU(0) of the first-order operator in the multicolour order
    (precond_ilu0): the solve reaches the oracle's 1e-10 residual drop, with
    fewer Krylov iterations than the block-Jacobi preconditioner it
    refines (same settings, same number of Newton steps).  On the stretched
    cylinder O-grid neither converges its linear systems at these settings
    (the bench's 20 Gauss-Seidel sweeps do); the supersonic wedge at first
    order and the hexahedron / pyramid box are the cases here."""
    if family == "wedge":
        case = cases.wedge_case(ni=30, nj=15, order="first")
    else:
        case = cases.box_case(kind="hexpyr", nx=8, ny=6, nz=5, flux="Roe", limiter="none")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    kw = dict(KW, precond_sweeps=0, krylov_cycles=6)
    W, rep = ns.newton_solve(case.state, ilu0=True, **kw, **opts)
    assert rep["status"] == 0, rep
    r0 = np.linalg.norm(o.residual(case.state)[:, 0])
    assert np.linalg.norm(o.residual(W)[:, 0]) <= 1e-9 * r0
    _, rj = ns.newton_solve(case.state, ilu0=False, raise_on_fail=False, **dict(kw, max_newton=rep["newton_iterations"]),
                            **opts)
    assert rep["krylov_iterations"] < rj["krylov_iterations"], (rep["krylov_iterations"], rj["krylov_iterations"])


@pytest.mark.gpu
def test_newton_local_relaxation(cylinder):
    """Per-cell under-relaxation (each cell's p and T change clipped to 20 %
    on its own): the cylinder converges to the same steady state as with the
    global relaxation, since the clip is inactive once the steps are small."""
    case, o, ns = cylinder
    Wa, rep_a = ns.newton_solve(case.state, jvp=False, **KW)
    Wb, rep_b = ns.newton_solve(case.state, jvp=False, local_relax=True, **KW)
    assert rep_b["status"] == 0, rep_b
    r0 = np.linalg.norm(o.residual(case.state)[:, 0])
    assert np.linalg.norm(o.residual(Wb)[:, 0]) <= 1e-9 * r0
    scale = np.abs(Wa).max(axis=0)
    scale[1:4] = np.abs(Wa[:, 1:4]).max()
    assert (np.abs(Wa - Wb).max(axis=0) / scale).max() <= 1e-7


@pytest.mark.gpu
def test_newton_hypersonic_explicit_startup(oracle_mod, fb):
    """The explicit start-up of fcfd_newton_solve on the inviscid M = 8
    cylinder at first order, 64x32 prisms, from the vacuum-free start: local
    time steps at CFL 0.5 take the mass residual down by 1e-3 in the number
    of steps the same march with the reference's discretisation takes on the
    CPU (oracle residual and time-term blocks: 3123), the state stays
    physical, and the oracle's residual at the returned state (one Newton
    step later) confirms the drop."""
    case = cases.hypersonic_case(64, 32, ns_extra=" order=first;")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    W0 = cases.hypersonic_smooth_state(case, m.geometry()["cell_centroid"])
    r0 = np.linalg.norm(o.residual(W0)[:, 0])
    W, rep = ns.newton_solve(W0, tol=1e-10, max_newton=1, cfl_mode=0, cfl0=0.5, cfl_growth=1.3, cfl_max=1e5,
                             krylov_rtol=1e-3, precond_sweeps=8, krylov_cycles=3, startup_steps=20000,
                             startup_drop=1e-3, jvp=False, raise_on_fail=False)
    assert 3000 <= rep["startup_steps"] <= 3250, rep["startup_steps"]
    assert rep["status"] == 4
    assert np.isfinite(W).all() and (W[:, 0] > 0).all() and (W[:, 4] > 0).all()
    assert np.linalg.norm(o.residual(W)[:, 0]) <= 1.5e-3 * r0
