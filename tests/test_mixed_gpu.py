"""Mixed-precision residual (device): the face pass in FP32 where the flow is
smooth, FP64 at shocks.

fcfd_residual_mixed keeps ghosts, gradients, limiters and the gather in FP64
and sends a face to the FP64 pass when its two cell-centre absolute
pressures differ by more than shock_ratio.  Checked: every face in FP64
(shock_ratio < 1) reproduces the FP64 residual; with shocks present the
flagged faces are the ones crossing the jump; and the mixed residual stays
within 100 FP32 unit roundoffs (1.2e-5) of the face-flux scale of the FP64
oracle, per equation, on the hypersonic prisms (with a captured bow-shock
jump), the laminar cylinder and the wedge."""
import numpy as np
import pytest

from freecfd_b200 import cases
from tests.util import build_pair, flux_scale, res_err

BAR = 100 * 2.0 ** -23  # 1.19e-5 of the face-flux scale


def shocked_state(case, mesh_geometry, radius=1.2):
    W = cases.hypersonic_shock_state(case, mesh_geometry["cell_centroid"], radius)
    x = mesh_geometry["cell_centroid"][: W.shape[0]]
    return W, np.hypot(x[:, 0], x[:, 1]) < radius


def _abs_err(R, ref, scale):
    return np.abs(R - ref).max(axis=0) / scale


@pytest.mark.gpu
@pytest.mark.parametrize("family", ["hypersonic", "cylinder", "wedge"])
def test_mixed_all_fp64_equals_fp64_residual(family, oracle_mod, fb):
    mk = {"hypersonic": lambda: cases.hypersonic_case(ntheta=64, nr=32),
          "cylinder": lambda: cases.cylinder_case(ntheta=64, nr=32),
          "wedge": lambda: cases.wedge_case(ni=48, nj=24)}[family]
    case = mk()
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    R64 = ns.residual(case.state)
    R, n64 = ns.residual_mixed(case.state, shock_ratio=0.0)
    assert n64 > 0
    assert res_err(R, R64).max() <= 1e-14


@pytest.mark.gpu
@pytest.mark.parametrize("size", [(64, 32), (512, 256)])
def test_mixed_hypersonic_with_shock(size, oracle_mod, fb):
    case = cases.hypersonic_case(ntheta=size[0], nr=size[1])
    o, cs, m = build_pair(case, oracle_mod, fb)
    geo = m.geometry()
    W, inside = shocked_state(case, geo)
    ns = fb.NavierStokes(m, cs, 0)
    ref = o.residual(W)
    R, n64 = ns.residual_mixed(W, shock_ratio=2.0)
    # the flagged faces: interior faces between an inside and an outside cell
    conn = m.connectivity()
    fp, fn, fbc = conn["face_parent"], conn["face_neighbor"], conn["face_bc"]
    it = fbc < 0
    crossing = int((inside[fp[it]] != inside[fn[it]]).sum())
    assert crossing <= n64 <= crossing + int((fbc >= 0).sum())
    scale = flux_scale(case, geo)
    assert _abs_err(R, ref, scale).max() <= BAR
    # with the sensor off every face runs in FP32
    R32, n32 = ns.residual_mixed(W, shock_ratio=1e30)
    assert n32 == 0
    assert _abs_err(R32, ref, scale).max() <= BAR


@pytest.mark.gpu
@pytest.mark.parametrize("family", ["cylinder", "wedge"])
def test_mixed_smooth_flow(family, oracle_mod, fb):
    case = {"cylinder": lambda: cases.cylinder_case(ntheta=128, nr=64),
            "wedge": lambda: cases.wedge_case(ni=60, nj=30)}[family]()
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    ref = o.residual(case.state)
    R, n64 = ns.residual_mixed(case.state, shock_ratio=2.0)
    assert n64 == 0
    assert _abs_err(R, ref, flux_scale(case, m.geometry())).max() <= BAR
