"""The residual on an RCM-renumbered grid (device).

A shuffled grid renumbered by fcfd_mesh_rcm is the same discretisation in
another cell order: with a limiter that does not decide on rounding noise
(VK with K > 0, the fused gradient) the residual, taken back to the original
order, equals the original order's to rounding (1e-12 normwise per
equation).  With a noise-deciding limiter (minmod, bit-exact gradient) the
reference's own result depends on the cell numbering through the order of
its LSQ sums, so the device on the renumbered grid is compared with the
oracle on the same renumbered grid (the usual bar)."""
import tempfile

import numpy as np
import pytest

from freecfd_b200 import cases
from tests.util import res_err


def _ns(fb, case, exact=False):
    cs = fb.Case(case.write_deck(tempfile.mkdtemp(prefix="fcfd_rcm_")))
    m = fb.Mesh(case.mesh, cs)
    return m, fb.NavierStokes(m, cs, 0, exact_gradients=exact)


@pytest.mark.gpu
@pytest.mark.parametrize("make", [lambda: cases.plate_case(ni=48, nj=24, nk=4, turbulent=False),
                                  lambda: cases.cylinder_case(ntheta=64, nr=32)], ids=["plate", "cylinder"])
def test_rcm_residual_equals_original_order(make, fb):
    case = make()
    _, ns0 = _ns(fb, case)
    R0 = ns0.residual(case.state)
    sh = cases.shuffle_case(case, 2)
    msh, _ = _ns(fb, sh)
    perm_sh = np.random.default_rng(2).permutation(case.mesh.n_cells)  # shuffle_case's order
    rperm = msh.rcm_order()
    rc = cases.renumber_case(sh, rperm, "rcm")
    _, ns1 = _ns(fb, rc)
    R1 = ns1.residual(rc.state)
    # new cell i of the RCM grid is shuffled cell rperm[i], i.e. original cell perm_sh[rperm[i]]
    orig = perm_sh[rperm]
    back = np.empty_like(R1)
    back[orig] = R1
    assert res_err(back, R0).max() <= 1e-12


@pytest.mark.gpu
def test_rcm_residual_minmod_against_oracle(oracle_mod, fb):
    case = cases.shuffle_case(cases.hypersonic_case(ntheta=48, nr=24), 4)
    m, _ = _ns(fb, case)
    rc = cases.renumber_case(case, m.rcm_order(), "rcm")
    _, ns = _ns(fb, rc, exact=True)
    R = ns.residual(rc.state)
    o = oracle_mod.Oracle(rc, tempfile.mkdtemp(prefix="fcfd_rcm_"))
    ref = o.residual(rc.state)
    assert res_err(R, ref).max() <= 1e-12
