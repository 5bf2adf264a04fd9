"""The oracle pinned to the reference itself (CPU only).

oracle/_ref/freecfd_ref is Free CFD's own, unmodified source tree compiled
with single-process stand-ins for MPI, PETSc, ParMETIS and CGNS and driven by
oracle/ref/harness.cpp through the reference's set-up sequence (main.cc:
131-245) and member functions: Grid::setup, set_bcs, set_lengthScales,
face_interpolation_weights, gradient_maps, NavierStokes::calc_cell_grads,
calc_limiter, assemble_linear_system, time_terms, RANS::terms and
update_time_step.  Every test here requires the oracle's restatement to
reproduce the reference's doubles bit for bit on the same inputs.  The only
parts of the reference that are not its own code are the documented
reconstructions of the two missing update_boundaries sources, a one-rank
restatement of Grid::create_partition_ghosts (its source ends without a
return statement) and NONE for the BCregion fields set_bcs.cc leaves
uninitialised; the oracle makes the same choices.
"""
import numpy as np
import pytest

from freecfd_b200 import cases
from tests.util import ALL, ELEMENTS, SMALL


@pytest.fixture(scope="session")
def ref_mod():
    from oracle import reference
    if not reference.build():
        pytest.skip("the compiled reference is absent and its sources are not here to build it")
    return reference


def _pair(case, oracle_mod, ref_mod):
    return oracle_mod.Oracle(case), ref_mod.Reference(case)


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("family", sorted(ALL))
def test_mesh_bit_exact_against_reference(family, oracle_mod, ref_mod):
    """Connectivity, geometry and every LSQ weight.  Boundary ghosts' length
    scales are excluded: the reference copies a ghost's lengthScale before it
    is ever set (create_boundary_ghosts), so those doubles are indeterminate
    in the reference and unused on the path."""
    o, r = _pair(ALL[family](), oracle_mod, ref_mod)
    m = r.mesh()
    for k, v in o.connectivity().items():
        assert _same(v, m[k]), k
    geo = o.geometry()
    for k, v in geo.items():
        if k == "length_scale":
            assert v == m[k]
        elif k == "cell_length":
            assert _same(v[: o.nc], m[k][: o.nc]), k
        else:
            assert _same(v, m[k]), k
    assert _same(o.grad_weights(), m["grad_weights"])


def _variants():
    out = []
    for fam in sorted(SMALL):
        for flux in ("Roe", "AUSM+up", "vanLeer", "SD-SLAU", "SW"):
            out.append((fam, dict(flux=flux, limiter="vk")))
    for fam, flux, lim in (("wedge", "Roe", "minmod"), ("wedge", "Roe", "bj"), ("wedge", "AUSM+up", "none"),
                           ("cylinder", "Roe", "minmod"), ("cylinder", "SW", "none"), ("cylinder", "vanLeer", "bj"),
                           ("hypersonic", "AUSM+up", "minmod"), ("hypersonic", "SD-SLAU", "minmod"),
                           ("hypersonic", "Roe", "bj"), ("plate", "AUSM+up", "minmod")):
        out.append((fam, dict(flux=flux, limiter=lim)))
    out.append(("wedge", dict(order="first")))
    out.append(("wedge", dict(grad="greengauss", limiter="minmod")))
    out.append(("cylinder", dict(flux="SW", ns_extra=" BLheight=0.05; walldissipation=0.5;")))
    out.append(("hypersonic", dict(flux="SW", limiter="minmod", ns_extra=" BLheight=-1.;")))
    for fam in sorted(ELEMENTS):
        for flux, lim in (("AUSM+up", "vk"), ("Roe", "minmod"), ("vanLeer", "bj"), ("SD-SLAU", "none"),
                          ("SW", "vk")):
            out.append((fam, dict(flux=flux, limiter=lim)))
        out.append((fam, dict(grad="greengauss")))
    return out


def _make(family, kw):
    if family in ("box_tet", "box_hexpyr"):
        return ALL[family](**kw)
    if family == "wedge":
        return cases.wedge_case(ni=24, nj=12, **kw)
    return SMALL[family](**kw)


@pytest.mark.parametrize("family,kw", _variants(), ids=lambda v: v if isinstance(v, str) else
                         "-".join(f"{k}={x}".replace(" ", "") for k, x in v.items()))
def test_residual_bit_exact_against_reference(family, kw, oracle_mod, ref_mod):
    """Ghost states, gradients (ghost copies included), limiters, residual,
    mdot and weightL of the oracle equal the reference's doubles.

    One exception: with Steger-Warming the reference's stored weightL is the
    pressure-jump blend of the LAST flux evaluation of its face loop, and
    assemble_linear_system evaluates the flux again for each finite-
    difference perturbation of its Jacobian (get_jacobians,
    ns_assemble_linear_system.cc:197-267), so on boundary faces it holds the
    blend of a perturbed state.  The oracle (and the device) store the blend
    of the unperturbed state; the two differ by the perturbation's effect,
    held to 1e-8 here.  The other fluxes' weightL (0, 1/2, 1) is a sign
    decision on the mass flux, which a perturbation changes only where that
    flux is at rounding level (slip-wall and symmetry faces, |mdot| below
    1e-12 of the largest); there mdot * weightL vanishes either way, and
    weightL is compared on the other faces."""
    case = _make(family, kw)
    o, r = _pair(case, oracle_mod, ref_mod)
    want = r.residual(case.state)
    got = o.residual(case.state, full=True)
    for k in ("ghost", "grads", "limiter", "R", "mdot"):
        assert _same(got[k], want[k]), k
    if kw.get("flux") == "SW":
        assert np.abs(got["weightL"] - want["weightL"]).max() <= 1e-8
    else:
        live = np.abs(want["mdot"]) > 1e-12 * np.abs(want["mdot"]).max()
        assert _same(got["weightL"][live], want["weightL"][live])


@pytest.mark.parametrize("size", [(12, 8, 2), (24, 12, 3)])
def test_rans_residual_bit_exact_against_reference(size, oracle_mod, ref_mod):
    """k-omega plate: the NS residual with the eddy viscosity and
    RANS::terms' right-hand side (rans_terms.cc:39-275)."""
    case = cases.plate_case(ni=size[0], nj=size[1], nk=size[2])
    o, r = _pair(case, oracle_mod, ref_mod)
    want = r.residual(case.state, case.kstate)
    R, RK = o.rans_residual(case.state, case.kstate)
    assert _same(R, want["R"])
    assert _same(RK, want["RK"])


@pytest.mark.parametrize("family", ["wedge", "cylinder", "hypersonic", "plate", "box_tet"])
def test_time_terms_bit_exact_against_reference(family, oracle_mod, ref_mod):
    """cons2prim and the P V / dt blocks of NavierStokes::time_terms
    (ns_time_terms.cc:26-56,107-186) for seeded local time steps.  The
    reference ADDs each entry into a zeroed matrix, which turns a -0.0 entry
    (drho_dT * w with w = 0) into +0.0; signed zeros are compared as equal."""
    case = ALL[family]()
    o, r = _pair(case, oracle_mod, ref_mod)
    dt = np.random.default_rng(11).uniform(0.5, 2.0, o.nc) * 1e-5
    assert _same(o.time_terms(case.state, dt) + 0.0, r.time_terms(case.state, dt) + 0.0)


@pytest.mark.parametrize("family", ["wedge", "cylinder", "hypersonic", "plate"])
def test_time_step_bit_exact_against_reference(family, oracle_mod, ref_mod):
    """update_time_step at time step 1 (time_step.cc:143-224): every deck
    here uses CFLmax, with the ramp's initial value on step 1 where the deck
    ramps."""
    case = SMALL[family]()
    o, r = _pair(case, oracle_mod, ref_mod)
    dt, t, cfl = r.local_dt(case.state)
    deck = case.deck
    ramp = "ramp (initial=" in deck
    if ramp:
        c = float(deck.split("ramp (initial=")[1].split(";")[0])
    else:
        c = float(deck.split("CFLmax=")[1].split(";")[0])
    want = o.local_dt(case.state, c, mode=1)
    assert _same(dt, want)
    assert t == want[0]
