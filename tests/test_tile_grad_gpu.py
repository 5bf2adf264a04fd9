"""The shared-memory tile kernel of the gradient + limiter stage
(fcfd_ctx_set_gradient_kernel(ctx, 2)).

Tiles of 128 consecutive cells stage the states and centroids their
stencils and faces name in shared memory and run the same per-cell
arithmetic as the per-cell kernel (the bit-exact rebuild of the
least-squares weights for noise-deciding limiters, the fused form for
continuous ones).  Held: bit-identical residuals to the one-thread-per-cell
kernel, and the residual bar against the oracle, on every least-squares mesh
family; meshes with Green-Gauss or curvilinear cells are refused."""
import numpy as np
import pytest

from freecfd_b200 import cases
from tests.util import ALL, SMALL, build_pair, res_err


@pytest.mark.gpu
@pytest.mark.parametrize("family", sorted(ALL))
@pytest.mark.parametrize("limiter", ["vk", "minmod", "bj", "none"])
def test_tile_gradient_residual(family, limiter, oracle_mod, fb):
    case = ALL[family](limiter=limiter)
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    ns.set_gradient_kernel(2)
    R = ns.residual(case.state)
    assert res_err(R, o.residual(case.state)).max() <= 1e-12
    if limiter in ("minmod", "bj"):
        # bit-exact gradient path: the per-cell kernel gives the same doubles
        ns.set_gradient_kernel(1)
        assert np.array_equal(R, ns.residual(case.state))


@pytest.mark.gpu
def test_tile_gradient_full_plate_bit_identical(oracle_mod, fb):
    """Laminar plate 384x192x4 (fused gradient, one thread per cell in the
    per-cell kernel): the tile kernel's residual is the same doubles."""
    case = cases.plate_case(turbulent=False)
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    ns.set_gradient_kernel(1)
    R1 = ns.residual(case.state)
    ns.set_gradient_kernel(2)
    R2 = ns.residual(case.state)
    assert np.array_equal(R1, R2)
    assert res_err(R2, o.residual(case.state)).max() <= 1e-12


@pytest.mark.gpu
def test_tile_gradient_refused_without_lsq(oracle_mod, fb):
    for case in (cases.wedge_case(ni=12, nj=6, grad="greengauss"), cases.cylinder_case(ntheta=16, nr=8, grad="curvilinear")):
        o, cs, m = build_pair(case, oracle_mod, fb)
        ns = fb.NavierStokes(m, cs, 0)
        with pytest.raises(fb.FcfdError) as e:
            ns.set_gradient_kernel(2)
        assert e.value.code == 7
        ns.set_gradient_kernel(1)
        ns.set_gradient_kernel(0)


@pytest.mark.gpu
@pytest.mark.parametrize("family", ["cylinder", "wedge", "hypersonic"])
def test_folded_stencil_gradient(family, oracle_mod, fb):
    """Folded stencils (kind 3): on one-layer meshes the z-symmetry ghosts'
    terms join their parents' entries.  The residual equals the unfolded one
    to rounding and keeps the oracle bar, with the fused gradient (VK,
    K > 0); the automatic choice is the unfolded per-cell kernel."""
    case = SMALL[family](limiter="vk")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    ns.set_gradient_kernel(3)
    R3 = ns.residual(case.state)
    ns.set_gradient_kernel(1)
    R1 = ns.residual(case.state)
    ref = o.residual(case.state)
    assert res_err(R3, ref).max() <= 1e-12
    assert res_err(R3, R1).max() <= 1e-13
    ns.set_gradient_kernel(0)
    assert np.array_equal(ns.residual(case.state), R1)


@pytest.mark.gpu
def test_folded_stencil_not_built_for_layered_plate(oracle_mod, fb):
    case = cases.plate_case(ni=24, nj=12, nk=6, turbulent=False)
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    with pytest.raises(fb.FcfdError) as e:
        ns.set_gradient_kernel(3)
    assert e.value.code == 7
