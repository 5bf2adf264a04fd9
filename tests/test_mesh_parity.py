"""Integer connectivity and geometry of the product's mesh builder against the
oracle's restatement of Grid::setup / set_bcs / set_lengthScales /
face_interpolation_weights / lsqr_grad_map — bit-exact (CPU only)."""
import numpy as np
import pytest

from tests.util import ALL, build_pair


@pytest.mark.parametrize("family", sorted(ALL))
def test_connectivity_bit_exact(family, oracle_mod, fb):
    o, cs, m = build_pair(ALL[family](), oracle_mod, fb)
    co, cp = o.connectivity(), m.connectivity()
    assert (o.nc, o.nf, o.nghost) == (m.nc, m.nf, m.nghost)
    for k in co:
        assert np.array_equal(co[k], cp[k]), k


@pytest.mark.parametrize("family", sorted(ALL))
def test_geometry_bit_exact(family, oracle_mod, fb):
    o, cs, m = build_pair(ALL[family](), oracle_mod, fb)
    go, gp = o.geometry(), m.geometry()
    for k in go:
        a, b = np.asarray(go[k]), np.asarray(gp[k])
        assert a.shape == b.shape, k
        assert np.array_equal(a.view(np.uint64) if a.dtype == np.float64 else a,
                              b.view(np.uint64) if b.dtype == np.float64 else b), k


@pytest.mark.parametrize("family", sorted(ALL))
def test_lsq_weights_bit_exact(family, oracle_mod, fb):
    """The gradient kernel rebuilds each lsqr_grad_map weight from centroids,
    per-cell cofactors/determinant and the precomputed self weight.  Redo that
    arithmetic here (numpy rounds every operation once, like the kernel's
    __dmul_rn/__dadd_rn/__ddiv_rn) and compare with the oracle's std::map."""
    o, cs, m = build_pair(ALL[family](), oracle_mod, fb)
    cof, selfw = m.lsq_data()
    g = m.geometry()
    conn = m.connectivity()
    x = g["cell_centroid"]
    w_or = o.grad_weights()
    idx, keys = conn["grad_index"], conn["grad_keys"]
    out = np.empty_like(w_or)
    for c in range(m.nc):
        C00, C01, C02, C11, C12, C22, det = cof[c]
        for j in range(idx[c], idx[c + 1]):
            k = keys[j]
            if k == c:
                out[j] = selfw[c]
                continue
            d0, d1, d2 = x[k, 0] - x[c, 0], x[k, 1] - x[c, 1], x[k, 2] - x[c, 2]
            w = (d0 * d0 + d1 * d1) + d2 * d2
            out[j, 0] = (w * ((d0 * C00 + d1 * C01) + d2 * C02)) / det
            out[j, 1] = (w * ((d0 * C01 + d1 * C11) + d2 * C12)) / det
            out[j, 2] = (w * ((d0 * C02 + d1 * C12) + d2 * C22)) / det
    assert np.array_equal(out.view(np.uint64), w_or.view(np.uint64))


@pytest.mark.parametrize("family", sorted(ALL))
def test_lsq_stencil_keys(family, oracle_mod, fb):
    o, cs, m = build_pair(ALL[family](), oracle_mod, fb)
    co, cp = o.connectivity(), m.connectivity()
    assert np.array_equal(co["grad_index"], cp["grad_index"])
    assert np.array_equal(co["grad_keys"], cp["grad_keys"])


@pytest.mark.parametrize("family", sorted(ALL))
def test_case_summary(family, oracle_mod, fb):
    o, cs, m = build_pair(ALL[family](), oracle_mod, fb)
    do, io = o.case_summary()
    dp, ip = cs.summary()
    assert np.array_equal(do[:12], dp[:12])
    assert np.array_equal(io, ip)


def test_full_size_wedge_connectivity(oracle_mod, fb):
    """Configuration-sized wedge (120x60x1): integer connectivity bit-exact."""
    from freecfd_b200 import cases
    o, cs, m = build_pair(cases.wedge_case(), oracle_mod, fb)
    co, cp = o.connectivity(), m.connectivity()
    assert (m.nc, m.nf) == (7200, 28980)
    for k in co:
        assert np.array_equal(co[k], cp[k]), k
