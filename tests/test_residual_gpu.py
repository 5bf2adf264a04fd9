"""Residual parity of the CUDA path (through the C ABI) against the CPU oracle.

Bar: integer/index work bit-exact (tests/test_mesh_parity.py).  Ghost states
bit-exact wherever the boundary conditions involved do not call pow() (the
ghost kernel is built without multiply-add contraction; CUDA's pow and libm's
pow may differ in the last bit).  Gradients and limiters bit-exact where the
limiter decides on the sign of rounding noise (minmod, Barth-Jespersen: the
gradient kernel then rebuilds the reference's rounded sums) and on request
(exact_gradients=True); with a continuous limiter the fused gradient is held
to 1e-12 of each variable's largest gradient.  The wedge and hypersonic
families have no pow in their BCs, so they are the bit-exact cases; the
cylinder and plate (subsonic outlets) are held to 1e-13.  The residual, mdot
and weightL within 1e-12 normwise relative per equation (FP64; the flux
arithmetic may contract multiply-adds and avoids the rotated frame, so it
differs from the reference at rounding level).
"""
import numpy as np
import pytest

from freecfd_b200 import cases
from tests.util import ELEMENTS, SMALL, build_pair, flux_scale, rel_err, res_err

TOL = 1e-12
BITWISE = {"wedge", "hypersonic"}


def tol(flux):
    """Steger-Warming adds two split fluxes A+ Q_L and A- Q_R that are each
    O(rho a H) while their sum is O(rho u H), and the reference forms them
    through 5x5 products; the rounding of the terms relative to the residual
    grows like 1/M (M = 0.2 on the cylinder and plate), so it is held to
    1e-11."""
    return 1e-11 if flux == "SW" else TOL


def _ctx(case, oracle_mod, fb, exact=False):
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0, exact_gradients=exact)
    return o, cs, m, ns


def grad_err(g, ref, nc):
    """Per-variable error of [nc][15] gradients relative to that variable's
    largest gradient component (one-layer meshes have a z column of pure
    rounding noise that a per-column norm would divide by ~0)."""
    g = np.asarray(g).reshape(nc, 5, 3)
    r = np.asarray(ref)[:nc].reshape(nc, 5, 3)
    scale = np.maximum(np.abs(r).max(axis=(0, 2)), 1e-300)
    return np.abs(g - r).max(axis=(0, 2)) / scale


def _check_stages(family, limiter, exact, st, ref, m):
    noise_limiter = limiter in ("minmod", "bj")
    if family in BITWISE:
        assert np.array_equal(st["ghost"], ref["ghost"]), "ghost states"
    else:
        assert rel_err(st["ghost"], ref["ghost"]).max() <= 1e-14
    if family in BITWISE and (noise_limiter or exact):
        assert np.array_equal(st["grads"], ref["grads"][: m.nc]), "gradients"
        assert np.array_equal(st["limiter"], ref["limiter"]), "limiters"
    elif noise_limiter or exact:
        assert grad_err(st["grads"], ref["grads"], m.nc).max() <= 1e-13
        assert rel_err(st["limiter"], ref["limiter"]).max() <= 1e-12
    else:
        assert grad_err(st["grads"], ref["grads"], m.nc).max() <= 1e-12
        assert rel_err(st["limiter"], ref["limiter"]).max() <= 1e-11


def _variants():
    out = []
    for fam in sorted(SMALL):
        for flux in ("Roe", "AUSM+up", "vanLeer", "SD-SLAU", "SW"):
            out.append((fam, flux, "vk"))
    out += [("wedge", "Roe", "minmod"), ("wedge", "Roe", "bj"), ("wedge", "AUSM+up", "none"),
            ("cylinder", "Roe", "minmod"), ("hypersonic", "AUSM+up", "minmod"), ("hypersonic", "Roe", "vk"),
            ("hypersonic", "SD-SLAU", "minmod"), ("wedge", "SW", "bj"), ("cylinder", "SW", "none")]
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("family,flux,limiter", _variants())
def test_residual_parity(family, flux, limiter, oracle_mod, fb):
    kw = dict(flux=flux, limiter=limiter)
    case = SMALL[family](**kw)
    o, cs, m, ns = _ctx(case, oracle_mod, fb)
    ref = o.residual(case.state, full=True)
    R = ns.residual(case.state)
    st = ns.stages()
    _check_stages(family, limiter, False, st, ref, m)
    err = res_err(R, ref["R"])
    assert err.max() <= tol(flux), err
    assert rel_err(st["mdot"], ref["mdot"]).max() <= tol(flux)
    _check_weights(flux, st, ref)


def _check_weights(flux, st, ref):
    """weightL is the upwind side (0 / 0.5 / 1) chosen by the sign of the mass
    flux; where that flux is at rounding level (symmetry and slip faces) the
    side is a rounding decision and mdot*weightL vanishes either way.  The
    Steger-Warming weight is the pressure-jump blend w (ns_stegger_warming.cc:
    38), a smooth function of the face pressures."""
    if flux == "SW":
        assert rel_err(st["weightL"], ref["weightL"]).max() <= 1e-13
        return
    big = np.abs(ref["mdot"]) > 1e-9 * np.abs(ref["mdot"]).max()
    assert np.array_equal(st["weightL"][big], ref["weightL"][big])


@pytest.mark.gpu
@pytest.mark.parametrize("family", sorted(ELEMENTS))
@pytest.mark.parametrize("flux,limiter", [("AUSM+up", "vk"), ("Roe", "minmod"), ("vanLeer", "bj"), ("Roe", "none"),
                                          ("SD-SLAU", "vk"), ("SW", "minmod")])
def test_residual_parity_tets_pyramids(family, flux, limiter, oracle_mod, fb):
    """Tetrahedra and pyramids (face tables, LSQ stencils of non-hex cells,
    triangle faces): residual parity on the jittered box meshes."""
    case = ELEMENTS[family](flux=flux, limiter=limiter)
    o, cs, m, ns = _ctx(case, oracle_mod, fb, exact=limiter in ("minmod", "bj"))
    ref = o.residual(case.state, full=True)
    R = ns.residual(case.state)
    st = ns.stages()
    assert rel_err(st["ghost"], ref["ghost"]).max() <= 1e-14
    assert grad_err(st["grads"], ref["grads"], m.nc).max() <= 1e-12
    assert rel_err(st["limiter"], ref["limiter"]).max() <= 1e-11
    assert res_err(R, ref["R"]).max() <= tol(flux)


@pytest.mark.gpu
@pytest.mark.parametrize("family,flux,limiter", [("wedge", "Roe", "vk"), ("hypersonic", "AUSM+up", "vk"),
                                                 ("wedge", "vanLeer", "none"), ("cylinder", "Roe", "vk"),
                                                 ("plate", "AUSM+up", "vk")])
def test_exact_gradients_on_request(family, flux, limiter, oracle_mod, fb):
    """exact_gradients=True rebuilds the reference's rounded gradient sums for
    a continuous limiter too (bit-exact on the wedge and hypersonic families),
    and the fused default agrees with it to rounding."""
    case = SMALL[family](flux=flux, limiter=limiter)
    o, cs, m, ns = _ctx(case, oracle_mod, fb, exact=True)
    ref = o.residual(case.state, full=True)
    R = ns.residual(case.state)
    _check_stages(family, limiter, True, ns.stages(), ref, m)
    assert res_err(R, ref["R"]).max() <= TOL
    fast = fb.NavierStokes(m, cs, 0)
    assert res_err(fast.residual(case.state), R).max() <= TOL


@pytest.mark.gpu
@pytest.mark.parametrize("family,limiter", [("cylinder", "vk"), ("plate", "vk"), ("hypersonic", "minmod"),
                                            ("wedge", "none")])
@pytest.mark.parametrize("extra", ["BLheight=0.05; walldissipation=0.5;", "BLheight=-1.;"])
def test_steger_warming_wall_dissipation(family, limiter, extra, oracle_mod, fb):
    """Steger-Warming with both dissipation branches (ns_stegger_warming.cc:
    92-93): faces farther from a no-slip wall than BLheight take
    wdiss (a + |V|), the others wdiss * dissipation_factor (a + |V.n|); the
    face wall distances and factors follow set_bcs.cc:228-249."""
    case = SMALL[family](flux="SW", limiter=limiter, ns_extra=" " + extra)
    o, cs, m, ns = _ctx(case, oracle_mod, fb)
    ref = o.residual(case.state, full=True)
    R = ns.residual(case.state)
    st = ns.stages()
    assert res_err(R, ref["R"]).max() <= tol("SW")
    assert rel_err(st["mdot"], ref["mdot"]).max() <= tol("SW")
    _check_weights("SW", st, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("family", sorted(SMALL))
@pytest.mark.parametrize("flux", [None, "SD-SLAU", "SW"])
def test_uniform_freestream(family, flux, oracle_mod, fb):
    """A uniform freestream state exercises every BC branch without limiter noise."""
    case = SMALL[family]() if flux is None else SMALL[family](flux=flux)
    o, cs, m, ns = _ctx(case, oracle_mod, fb)
    W = np.tile(np.asarray(case.freestream), (m.nc, 1))
    R, ref = ns.residual(W), o.residual(W)
    # the residual of a uniform state is mostly cancellation noise: bound the
    # difference by the size of the cancelling face fluxes
    assert (np.abs(R - ref).max(axis=0) <= tol(flux) * flux_scale(case, m.geometry())).all()


@pytest.mark.gpu
def test_determinism_and_device_pointers(oracle_mod, fb):
    """Two evaluations are bit-identical (atomic-free gather); device-pointer
    calls give the same bits as host-pointer calls."""
    import torch
    case = SMALL["cylinder"]()
    o, cs, m, ns = _ctx(case, oracle_mod, fb)
    R1 = ns.residual(case.state)
    R2 = ns.residual(case.state)
    assert np.array_equal(R1, R2)
    Wd = torch.from_numpy(case.state).cuda()
    Rd = ns.residual(Wd)
    torch.cuda.synchronize()
    assert np.array_equal(Rd.cpu().numpy(), R1)


@pytest.mark.gpu
@pytest.mark.parametrize("family", ["cylinder", "wedge", "hypersonic", "plate"])
def test_launch_overlap_same_bits(family, oracle_mod, fb):
    """Programmatic dependent launches of the gradient and face kernels (the
    default) and ordinary launches give the same residual bits, through the
    direct chain and through the pinned-buffer graph."""
    import torch
    case = SMALL[family]()
    o, cs, m, ns = _ctx(case, oracle_mod, fb)
    Wp = torch.empty((m.nc, 5), dtype=torch.float64, pin_memory=True)
    Rp = torch.empty((m.nc, 5), dtype=torch.float64, pin_memory=True)
    Wp.numpy()[:] = case.state
    out = {}
    for on in (True, False, True):
        ns.set_launch_overlap(on)
        r = ns.residual(case.state)
        ns.residual(Wp.numpy(), Rp.numpy())
        assert np.array_equal(Rp.numpy(), r)
        if on in out:
            assert np.array_equal(out[on], r)
        out[on] = r
    assert np.array_equal(out[True], out[False])


@pytest.mark.gpu
def test_pinned_host_buffers(oracle_mod, fb):
    """Page-locked W and R take the one-graph path (copies, chain and error
    flag replayed as a CUDA graph): same bits as pageable buffers, for a new
    state in the same buffers and for another buffer pair; a BC error raised
    inside the graph is reported and cleared."""
    import torch
    case = SMALL["cylinder"]()
    o, cs, m, ns = _ctx(case, oracle_mod, fb)
    ref = ns.residual(case.state)
    bufs = [(torch.empty((m.nc, 5), dtype=torch.float64, pin_memory=True),
             torch.empty((m.nc, 5), dtype=torch.float64, pin_memory=True)) for _ in range(2)]
    W2 = case.state * (1 + 1e-3 * np.random.default_rng(5).uniform(-1, 1, case.state.shape))
    ref2 = ns.residual(W2)
    for Wp, Rp in bufs:
        for W, r in ((case.state, ref), (W2, ref2), (case.state, ref)):
            Wp.numpy()[:] = W
            ns.residual(Wp.numpy(), Rp.numpy())
            assert np.array_equal(Rp.numpy(), r)
    # supersonic flow into the inlet, whose deck gives rho and V only
    Wbad = case.state.copy()
    Wbad[:, 1] = 1500.0
    Wp, Rp = bufs[0]
    Wp.numpy()[:] = Wbad
    with pytest.raises(fb.FcfdError) as e:
        ns.residual(Wp.numpy(), Rp.numpy())
    assert e.value.code == 8
    Wp.numpy()[:] = case.state
    ns.residual(Wp.numpy(), Rp.numpy())
    assert np.array_equal(Rp.numpy(), ref)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
def test_local_dt(mode, oracle_mod, fb):
    case = SMALL["wedge"]()
    o, cs, m, ns = _ctx(case, oracle_mod, fb)
    dt = ns.local_dt(case.state, 5.0, mode)
    ref = o.local_dt(case.state, 5.0, mode)
    assert np.abs(dt - ref).max() / np.abs(ref).max() <= 1e-15


@pytest.mark.gpu
@pytest.mark.parametrize("family", ["wedge", "hypersonic"])
def test_full_size_parity(family, oracle_mod, fb):
    """Configuration-sized meshes (7,200 and 262,144 cells): residual parity."""
    case = cases.wedge_case() if family == "wedge" else cases.hypersonic_case()
    o, cs, m, ns = _ctx(case, oracle_mod, fb)
    ref = o.residual(case.state, full=True)
    R = ns.residual(case.state)
    st = ns.stages()
    limiter = "minmod" if family == "hypersonic" else "vk"
    _check_stages(family, limiter, False, st, ref, m)
    assert res_err(R, ref["R"]).max() <= TOL


@pytest.mark.gpu
def test_conservation_full_cylinder(oracle_mod, fb):
    """Size-independent property at the benchmark size (256x128 cylinder):
    interior faces cancel, so the residual summed over cells equals the sum of
    boundary-face contributions; checked against the oracle's sum."""
    case = cases.cylinder_case()
    o, cs, m, ns = _ctx(case, oracle_mod, fb)
    R = ns.residual(case.state)
    ref = o.residual(case.state)
    s, sr = R.sum(axis=0), ref.sum(axis=0)
    scale = np.maximum(np.abs(ref).sum(axis=0), 1e-6 * np.abs(ref).sum(axis=0).max())
    assert (np.abs(s - sr) / scale).max() < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("family,limiter", [("wedge", "vk"), ("wedge", "minmod"), ("box_hexpyr", "vk"),
                                            ("box_tet", "minmod")])
def test_green_gauss_gradients(family, limiter, oracle_mod, fb):
    """gradients (... method=greengauss): empty gradient maps, so the gradient
    is the Green-Gauss fallback of Variable::cell_gradient (variable.h:204-213)
    with BC-fixed face values; evaluated with rounded operations in the
    reference's order, bit-exact where the ghosts are (wedge)."""
    if family == "wedge":
        case = cases.wedge_case(ni=24, nj=12, limiter=limiter, grad="greengauss")
    else:
        case = ELEMENTS[family](limiter=limiter, grad="greengauss")
    o, cs, m, ns = _ctx(case, oracle_mod, fb)
    assert m.n_grad_entries == 0
    ref = o.residual(case.state, full=True)
    R = ns.residual(case.state)
    st = ns.stages()
    if family == "wedge":
        assert np.array_equal(st["grads"], ref["grads"][: m.nc])
        assert np.array_equal(st["limiter"], ref["limiter"])
    else:
        assert grad_err(st["grads"], ref["grads"], m.nc).max() <= 1e-13
        assert rel_err(st["limiter"], ref["limiter"]).max() <= 1e-11
    assert res_err(R, ref["R"]).max() <= TOL
    # the tangent chain goes through the same fallback
    V = np.random.default_rng(3).standard_normal(case.state.shape) * np.abs(case.state).max(axis=0)
    jv, cs_ = ns.jvp(case.state, V), o.residual_cstep(case.state, V)
    cols = [k for k in range(5) if np.abs(cs_[:, k]).max() > 1e-12 * np.abs(cs_).max()]
    assert rel_err(jv[:, cols], cs_[:, cols]).max() <= 1e-10
    with pytest.raises(fb.FcfdError):          # the adjoint covers least-squares gradients only
        ns.vjp(case.state, np.ones_like(case.state))
