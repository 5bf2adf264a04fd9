"""Tecplot FEPolyhedron grid files (Grid::readTEC + Grid::create_faces2).

The files are written by freecfd_b200.cases.write_tecplot from the synthetic
meshes, with faces in cell-visit order and shuffled.  The product's reader and
face-based builder are checked bit for bit against the oracle's restatement
(connectivity, geometry, LSQ stencils), and, for faces in cell-visit order,
against the cell-based builder of the same mesh (same faces, parents,
neighbours and BC tags; the cell node lists are sorted node sets, so cell
centroids differ by rounding only)."""
import os
import tempfile

import numpy as np
import pytest

from freecfd_b200 import cases
from tests.util import ALL, SMALL, build_pair, res_err

FAMILIES = ["wedge", "hypersonic", "plate", "box_tet", "box_hexpyr"]


def _pair(family, oracle_mod, fb, order, **kw):
    case = ALL[family](**kw)
    d = tempfile.mkdtemp(prefix="fcfd_tec_")
    path = cases.write_tecplot(case.mesh, os.path.join(d, "grid.dat"), order=order, seed=5)
    o = oracle_mod.Oracle(case, d, tecplot=path)
    cs = fb.Case(case.write_deck(d))
    m = fb.Mesh(None, cs, tecplot=path)
    return case, o, cs, m, path


@pytest.mark.parametrize("order", ["cells", "shuffled"])
@pytest.mark.parametrize("family", FAMILIES)
def test_tecplot_mesh_bit_exact(family, order, oracle_mod, fb):
    case, o, cs, m, _ = _pair(family, oracle_mod, fb, order)
    assert (o.nc, o.nf, o.nghost) == (m.nc, m.nf, m.nghost)
    co, cp = o.connectivity(), m.connectivity()
    for k in co:
        assert np.array_equal(co[k], cp[k]), k
    go, gp = o.geometry(), m.geometry()
    for k in go:
        a, b = np.asarray(go[k]), np.asarray(gp[k])
        assert np.array_equal(a.view(np.uint64) if a.dtype == np.float64 else a,
                              b.view(np.uint64) if b.dtype == np.float64 else b), k


@pytest.mark.parametrize("family", FAMILIES)
def test_tecplot_matches_cell_based_mesh(family, oracle_mod, fb):
    case, o, cs, m, _ = _pair(family, oracle_mod, fb, "cells")
    mc = fb.Mesh(case.mesh, cs)
    ct, cc = m.connectivity(), mc.connectivity()
    for k in ("face_parent", "face_neighbor", "face_bc", "cell_face_index", "cell_faces"):
        assert np.array_equal(ct[k], cc[k]), k
    gt, gc = m.geometry(), mc.geometry()
    for k in ("face_normal", "face_area", "face_centroid"):
        assert np.array_equal(gt[k], gc[k]), k
    for k in ("cell_centroid", "cell_volume", "face_avg"):
        scale = np.abs(gc[k]).max()
        assert np.abs(gt[k] - gc[k]).max() <= 1e-13 * scale, k


def test_tecplot_zone_names_and_errors(fb, tmp_path):
    case = SMALL["wedge"]()
    p = cases.write_tecplot(case.mesh, str(tmp_path / "g.dat"), ["inflow", "outflow", "symmetry", "ramp"])
    cs = fb.Case(case.write_deck(str(tmp_path)))
    m = fb.Mesh(None, cs, tecplot=p)
    assert m.bc_names == ["inflow", "outflow", "symmetry", "ramp"]
    text = open(p).read()
    bad = tmp_path / "bad.dat"
    bad.write_text(text.replace("ZONETYPE=FEPolyhedron", "ZONETYPE=FEBRICK"))
    with pytest.raises(fb.FcfdError) as e:
        fb.Mesh(None, cs, tecplot=str(bad))
    assert e.value.code == 7
    with pytest.raises(fb.FcfdError) as e:
        fb.Mesh(None, cs, tecplot=str(tmp_path / "missing.dat"))
    assert e.value.code == 1


@pytest.mark.gpu
@pytest.mark.parametrize("family,flux,limiter", [("wedge", "Roe", "minmod"), ("hypersonic", "AUSM+up", "vk"),
                                                 ("plate", "Roe", "vk"), ("box_hexpyr", "SD-SLAU", "vk")])
def test_tecplot_residual_parity(family, flux, limiter, oracle_mod, fb):
    """Residual on a shuffled-face Tecplot grid vs the oracle reading the same file."""
    case, o, cs, m, _ = _pair(family, oracle_mod, fb, "shuffled", flux=flux, limiter=limiter)
    ns = fb.NavierStokes(m, cs, 0)
    R = ns.residual(case.state)
    ref = o.residual(case.state)
    assert res_err(R, ref).max() <= 1e-12
