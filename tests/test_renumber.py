"""Reverse Cuthill-McKee renumbering of the cells (host only, CPU).

fcfd_mesh_rcm gives the order; cases.renumber_cells lists a grid's elements
in it and the mesh is built again.  Checked here: the order against the
plain-Python restatement in oracle/rcm.py (bit-exact integers), the
bandwidth it leaves on a shuffled grid, that the renumbered grid is the same
grid (every cell's volume and centroid, every face's nodes, area, centroid,
BC tag and its two cells, the normal's sign following the parent), and that
the mesh the product builds from the renumbered grid is the one the
reference builds from it (connectivity and geometry bit for bit against the
compiled reference)."""
import tempfile

import numpy as np
import pytest

from freecfd_b200 import cases
from oracle.rcm import rcm_order as rcm_restated
from tests.util import ALL


def _mesh(fb, case):
    cs = fb.Case(case.write_deck(tempfile.mkdtemp(prefix="fcfd_rcm_")))
    return cs, fb.Mesh(case.mesh, cs)


@pytest.mark.parametrize("family", sorted(ALL))
@pytest.mark.parametrize("shuffled", [False, True])
def test_rcm_matches_restatement(family, shuffled, fb):
    case = ALL[family]()
    if shuffled:
        case = cases.shuffle_case(case, 11)
    _, m = _mesh(fb, case)
    c = m.connectivity()
    perm = m.rcm_order()
    ref = rcm_restated(m.nc, c["face_parent"], c["face_neighbor"], c["face_bc"])
    assert np.array_equal(np.sort(perm), np.arange(m.nc))
    assert np.array_equal(perm, ref)


def test_rcm_bandwidth_of_shuffled_plate(fb):
    """A 96x48x4 plate listed in random order has bandwidth ~nc; after RCM it
    is below the structured i-j-k order's (ni*nj)."""
    case = cases.plate_case(ni=96, nj=48, nk=4, turbulent=False)
    sh = cases.shuffle_case(case, 3)
    _, m = _mesh(fb, sh)
    c = m.connectivity()
    assert cases.bandwidth(c["face_parent"], c["face_neighbor"], c["face_bc"]) > m.nc // 2
    r = cases.renumber_case(sh, m.rcm_order(), "rcm")
    _, m2 = _mesh(fb, r)
    c2 = m2.connectivity()
    assert cases.bandwidth(c2["face_parent"], c2["face_neighbor"], c2["face_bc"]) < 96 * 48 // 4


def _face_key(nodes, k):
    return tuple(sorted(int(v) for v in nodes[k] if v >= 0))


@pytest.mark.parametrize("family", sorted(ALL))
def test_renumbered_grid_is_the_same_grid(family, fb):
    """Same cells and faces under the permutation.  Integers exactly; the
    geometry to rounding, since a face takes the node order of the cell that
    lists it first (its parent) and the reference's area, centroid and
    volume sums follow that order."""
    case = cases.shuffle_case(ALL[family](), 5)
    _, m = _mesh(fb, case)
    perm = m.rcm_order()
    r = cases.renumber_case(case, perm, "rcm")
    _, m2 = _mesh(fb, r)
    assert (m.nc, m.nf, m.nghost) == (m2.nc, m2.nf, m2.nghost)
    g, g2 = m.geometry(), m2.geometry()
    c, c2 = m.connectivity(), m2.connectivity()
    nc = m.nc

    def close(a, b, tol=1e-14):
        a, b = np.asarray(a, float), np.asarray(b, float)
        return np.abs(a - b).max() <= tol * max(np.abs(b).max(), 1e-300)

    # cells: new i is old perm[i]
    assert close(g2["cell_volume"][:nc], g["cell_volume"][perm])
    assert close(g2["cell_centroid"][:nc], g["cell_centroid"][perm])
    # faces matched by centroid (mesh-local node ids differ: nodes are numbered
    # in first-seen order over the cell list)
    L = np.abs(g["face_centroid"]).max()
    key = lambda x: tuple(np.round(x / L * 1e10).astype(np.int64))
    where = {key(g["face_centroid"][f]): f for f in range(m.nf)}
    assert len(where) == m.nf
    for f2 in range(m2.nf):
        f = where[key(g2["face_centroid"][f2])]
        assert c2["face_bc"][f2] == c["face_bc"][f]
        assert close(g2["face_area"][f2], g["face_area"][f])
        p2, n2 = c2["face_parent"][f2], c2["face_neighbor"][f2]
        p, n = c["face_parent"][f], c["face_neighbor"][f]
        if c["face_bc"][f] >= 0:
            assert perm[p2] == p
            assert close(g2["face_normal"][f2], g["face_normal"][f])
        else:
            assert {perm[p2], perm[n2]} == {p, n}
            sgn = 1.0 if perm[p2] == p else -1.0
            assert close(g2["face_normal"][f2], sgn * g["face_normal"][f])


@pytest.mark.parametrize("family", ["cylinder", "hypersonic", "box_tet"])
def test_renumbered_grid_bit_exact_against_reference(family, fb):
    """The product's mesh of the RCM-renumbered grid against the compiled
    reference's Grid::setup of the same renumbered grid."""
    from oracle import reference
    if not reference.build():
        pytest.skip("the compiled reference is absent and its sources are not here to build it")
    case = cases.shuffle_case(ALL[family](), 9)
    _, m = _mesh(fb, case)
    r = cases.renumber_case(case, m.rcm_order(), "rcm")
    _, m2 = _mesh(fb, r)
    ref = reference.Reference(r)
    rm = ref.mesh()
    ref.close()
    for k, v in m2.connectivity().items():
        assert np.array_equal(np.asarray(v), np.asarray(rm[k])), k
    for k, v in m2.geometry().items():
        if k == "length_scale":
            assert v == rm[k]
        elif k == "cell_length":
            assert np.array_equal(v[: m2.nc].view(np.uint64), rm[k][: m2.nc].view(np.uint64)), k
        else:
            assert np.array_equal(np.asarray(v).view(np.uint64), np.asarray(rm[k]).view(np.uint64)), k
