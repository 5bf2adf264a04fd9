"""Curvilinear gradient maps (CPU): the reference's default gradient method
for hexahedra and prisms (read_inputs.cc:47-48, curvilinear_grad_map.cc:
28-228).

The product's mesh builder stores each cell's map (up to six cells across
three face pairs, weights +-Jac^-T rows) and the device sums w . phi in key
order.  Held here bit for bit: the stored weights against the oracle's
restatement on every mesh family, and against the compiled reference itself
on prisms and tetrahedra.  The reference's hexahedron branch erases the
std::set element its loop iterator points at and then increments it
(undefined behaviour), so hexahedra are held to the oracle's restatement of
the pairing that loop is written to produce, not to the compiled reference."""
import tempfile

import numpy as np
import pytest

from freecfd_b200 import cases

CURV = {
    "wedge": lambda **kw: cases.wedge_case(ni=24, nj=12, grad="curvilinear", **kw),
    "cylinder": lambda **kw: cases.cylinder_case(ntheta=32, nr=16, grad="curvilinear", **kw),
    "hypersonic": lambda **kw: cases.hypersonic_case(ntheta=32, nr=16, grad="curvilinear", **kw),
    "plate": lambda **kw: cases.plate_case(ni=24, nj=12, nk=3, turbulent=False, grad="curvilinear", **kw),
    "box_tet": lambda **kw: cases.box_case("tet", grad="curvilinear", **kw),
    "box_hexpyr": lambda **kw: cases.box_case("hexpyr", grad="curvilinear", **kw),
}
# no hexahedra: the compiled reference's curvilinear map is defined here
REF_SAFE = ("hypersonic", "box_tet")


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("family", sorted(CURV))
def test_curvilinear_weights_bit_exact_against_oracle(family, oracle_mod, fb):
    case = CURV[family]()
    d = tempfile.mkdtemp(prefix="fcfd_curv_")
    o = oracle_mod.Oracle(case, d)
    cs = fb.Case(case.write_deck(d))
    m = fb.Mesh(case.mesh, cs)
    co, cp = o.connectivity(), m.connectivity()
    for k in co:
        assert np.array_equal(co[k], cp[k]), k
    assert _same(m.grad_weights(), o.grad_weights())
    # a curvilinear map holds at most the six cells across three face pairs
    idx = cp["grad_index"]
    assert int(np.diff(idx).max()) <= 6


@pytest.mark.parametrize("family", REF_SAFE)
def test_curvilinear_weights_bit_exact_against_reference(family, fb):
    from oracle import reference
    if not reference.build():
        pytest.skip("the compiled reference is absent and its sources are not here to build it")
    case = CURV[family]()
    cs = fb.Case(case.write_deck(tempfile.mkdtemp(prefix="fcfd_curv_")))
    m = fb.Mesh(case.mesh, cs)
    r = reference.Reference(case)
    rm = r.mesh()
    r.close()
    for k, v in m.connectivity().items():
        assert np.array_equal(np.asarray(v), np.asarray(rm[k])), k
    assert _same(m.grad_weights(), rm["grad_weights"])


@pytest.mark.parametrize("family,kw", [("hypersonic", dict(flux="AUSM+up", limiter="minmod")),
                                       ("hypersonic", dict(flux="Roe", limiter="vk")),
                                       ("box_tet", dict(flux="AUSM+up", limiter="vk")),
                                       ("box_tet", dict(flux="vanLeer", limiter="bj"))])
def test_curvilinear_residual_bit_exact_oracle_vs_reference(family, kw, oracle_mod):
    """The oracle's residual with curvilinear maps against the compiled
    reference's (gradients, limiters, residual) on prisms and tetrahedra."""
    from oracle import reference
    if not reference.build():
        pytest.skip("the compiled reference is absent and its sources are not here to build it")
    case = CURV[family](**kw)
    o = oracle_mod.Oracle(case, tempfile.mkdtemp(prefix="fcfd_curv_"))
    r = reference.Reference(case)
    want = r.residual(case.state)
    r.close()
    got = o.residual(case.state, full=True)
    for k in ("ghost", "grads", "limiter", "R", "mdot"):
        assert _same(got[k], want[k]), k


def test_lsqr_meshes_keep_no_weights(fb):
    """Without a curvilinear cell the least-squares weights are rebuilt on
    the device and none are stored."""
    case = cases.cylinder_case(ntheta=16, nr=8)
    cs = fb.Case(case.write_deck(tempfile.mkdtemp(prefix="fcfd_curv_")))
    m = fb.Mesh(case.mesh, cs)
    with pytest.raises(fb.FcfdError) as e:
        m.grad_weights()
    assert e.value.code == 7
