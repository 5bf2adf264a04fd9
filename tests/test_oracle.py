"""Pins of the CPU oracle.

The reference ships no tests or golden outputs, and its build needs MPI,
PETSc, ParMETIS and CGNS.  Its path is nevertheless compiled here from its
own sources against single-process stand-ins for those libraries (oracle/ref,
`make -C oracle ref`), so the oracle is pinned against the reference's own
doubles, and in addition by the known-answer behaviour the reference relies
on and by identities of the discretisation:
  * LSQ gradient exactness for a linear field (the reference's gradient-test
    IC mode, ns.cc:161-185) — checked through the stored gradient weights;
  * flux consistency F(U,U) = physical flux (ns_roe.cc, ns_ausm_plus_up.cc,
    ns_vanleer.cc, ns_sd_slau.cc, ns_stegger_warming.cc): a uniform state
    leaves every cell away from non-symmetry boundaries with a zero residual up to the
    rounding of its cancelling face fluxes;
  * a closed symmetry box at rest has zero residual;
  * conservation: interior faces cancel in the sum of residuals;
  * committed golden vectors (tests/golden/) that tests/golden/make_golden.py
    produced by running the reference itself (its own sources compiled into
    oracle/_ref/freecfd_ref); tests/test_reference_pin.py compares the oracle
    with that compiled reference directly, over every mesh family, flux,
    limiter and the k-omega terms.
"""
import os

import numpy as np
import pytest

from freecfd_b200 import cases
from tests.conftest import ROOT
from tests.util import SMALL


@pytest.mark.parametrize("family", sorted(SMALL))
def test_lsq_exact_for_linear_field(family, oracle_mod):
    """sum_k w_k * phi_k reproduces grad(phi) for phi = a + b.x (all cells,
    ghosts included, as in the gradient-test mode) — except where a cell
    touches a symmetry face: there the reference's map drops the mirror
    point's value (lsqr_grad_map.cc:66-96), which the restatement keeps."""
    case = SMALL[family]()
    o = oracle_mod.Oracle(case)
    g = o.geometry()
    conn = o.connectivity()
    w = o.grad_weights()
    x = g["cell_centroid"]
    b = np.array([0.7, -1.3, 0.4])
    phi = 2.0 + x @ b
    idx, keys = conn["grad_index"], conn["grad_keys"]
    fbc = conn["face_bc"]
    cf, cfi = conn["cell_faces"], conn["cell_face_index"]
    sym = set(np.nonzero(fbc == 3)[0]) if family != "plate" else set(np.nonzero(fbc == 3)[0])
    checked = 0
    for c in range(o.nc):
        grad = np.zeros(3)
        for j in range(idx[c], idx[c + 1]):
            grad += w[j] * phi[keys[j]]
        faces = cf[cfi[c]:cfi[c + 1]]
        has_sym = any(fbc[f] >= 0 and _is_sym(case, fbc[f]) for f in faces)
        if not has_sym:
            assert np.allclose(grad, b, rtol=1e-8, atol=1e-8 * np.abs(phi).max()), (c, grad)
            checked += 1
    if family == "plate":
        assert checked > 0


def _is_sym(case, b):
    import re
    m = re.search(r"BC_%d\s*\(type=(\w+)" % (b + 1), case.deck)
    return m is not None and m.group(1) == "symmetry"


def test_symmetry_box_at_rest(oracle_mod, tmp_path):
    """All-symmetry box with uniform p, V=0: every cell's faces close, R = 0."""
    case = cases.plate_case(ni=6, nj=4, nk=2, turbulent=False)
    deck = case.deck.replace("BC_1 (type=inlet;", "BC_1 (type=symmetry; //").replace(
        "BC_2 (type=outlet;", "BC_2 (type=symmetry; //").replace("BC_3 (type=wall;", "BC_3 (type=symmetry; //")
    deck = "\n".join(line if not line.strip().startswith("BC_") else line.split("//")[0] + ");" for line in deck.split("\n"))
    case.deck = deck
    o = oracle_mod.Oracle(case, str(tmp_path))
    W = np.tile(np.array([101325.0, 0.0, 0.0, 0.0, 300.0]), (o.nc, 1))
    R = o.residual(W)
    assert np.abs(R[:, 0]).max() == 0.0
    assert np.abs(R[:, 1:4]).max() < 1e-9 * 101325.0
    assert np.abs(R[:, 4]).max() == 0.0


@pytest.mark.parametrize("family", sorted(SMALL))
def test_mass_conservation(family, oracle_mod):
    """Interior faces add +D to the parent and -D to the neighbour, so the
    continuity residual summed over cells equals the boundary-face mass flux
    -sum_b mdot_f*A_f (mdot is the per-face Variable of
    ns_assemble_linear_system.cc:123)."""
    case = SMALL[family]()
    o = oracle_mod.Oracle(case)
    out = o.residual(case.state, full=True)
    conn = o.connectivity()
    A = o.geometry()["face_area"]
    bnd = conn["face_bc"] >= 0
    total = out["R"][:, 0].sum()
    expect = -(out["mdot"][bnd] * A[bnd]).sum()
    scale = np.abs(out["mdot"] * A).sum()
    assert abs(total - expect) <= 1e-12 * scale


@pytest.mark.parametrize("flux", ["Roe", "AUSM+up", "vanLeer", "SD-SLAU", "SW"])
@pytest.mark.parametrize("family", ["wedge", "hypersonic", "plate"])
def test_freestream_preservation(family, flux, oracle_mod):
    """Flux consistency: with a uniform state every face flux is the physical
    flux of that state, so cells with no boundary face have R = 0 up to the
    rounding of their cancelling face fluxes (Steger-Warming: A+ Q + A- Q =
    A Q = F(Q), the eigen-split of the perfect-gas flux Jacobian with
    beta = gamma R / Cp = gamma - 1).  First order: the LSQ map's dropped
    symmetry-mirror values (lsqr_grad_map.cc:66-96) give a uniform field
    non-zero gradients next to symmetry planes, which second order would
    reconstruct into the face states."""
    from tests.util import flux_scale
    case = (SMALL[family](flux=flux, order="first") if family == "wedge"
            else SMALL[family](flux=flux, ns_extra=" order=first;"))
    o = oracle_mod.Oracle(case)
    W = np.tile(np.asarray(case.freestream), (o.nc, 1))
    R = o.residual(W)
    conn = o.connectivity()
    nc = o.nc
    fp, fn, fbc = conn["face_parent"], conn["face_neighbor"], conn["face_bc"]
    # symmetry ghosts mirror the uniform state onto itself (V tangential);
    # other ghosts (walls, inlets, outlets) differ from it and enter a cell's
    # residual through its boundary faces and through the LSQ gradients of
    # the cells on either side of its faces
    real = np.array([b >= 0 and not _is_sym(case, b) for b in fbc])
    bad_ghost = set(fn[real].tolist())
    gi, gk = conn["grad_index"], conn["grad_keys"]
    dirty = np.array([any(k in bad_ghost for k in gk[gi[c]:gi[c + 1]]) for c in range(nc)])
    inner = np.ones(nc, bool)
    for f in range(len(fp)):
        if real[f]:
            inner[fp[f]] = False
        elif fbc[f] < 0 and (dirty[fp[f]] or dirty[fn[f]]):
            inner[fp[f]] = inner[fn[f]] = False
    inner &= ~dirty
    assert inner.sum() > 0
    scale = flux_scale(case, o.geometry())
    assert (np.abs(R[inner]).max(axis=0) <= 1e-11 * scale).all(), np.abs(R[inner]).max(axis=0) / scale


@pytest.mark.parametrize("flux", ["SD-SLAU", "SW"])
@pytest.mark.parametrize("family", ["cylinder", "hypersonic"])
def test_complex_step_other_fluxes(family, flux, oracle_mod):
    """SD-SLAU and Steger-Warming: complex step vs central differences on a
    state with v perturbed (no face sits on the |V.n| = 0 kink) and an
    unlimited reconstruction."""
    from tests.test_vjp_gpu import _generic
    case = SMALL[family](flux=flux, limiter="none")
    o = oracle_mod.Oracle(case)
    W = _generic(case)
    rng = np.random.default_rng(7)
    dW = rng.standard_normal(W.shape) * np.abs(W).max(axis=0) * np.array([1.0, 1.0, 1.0, 0.0, 1.0])
    jv = o.residual_cstep(W, dW)
    h = 1e-7
    fd = (o.residual(W + h * dW) - o.residual(W - h * dW)) / (2 * h)
    cols = [0, 1, 2, 4]
    scale = np.abs(jv[:, cols]).max(axis=0)
    assert (np.abs(jv - fd)[:, cols].max(axis=0) / scale).max() < 1e-5


GOLDEN = {
    "wedge_12x6": lambda: cases.wedge_case(ni=12, nj=6),
    "hypersonic_16x8": lambda: cases.hypersonic_case(ntheta=16, nr=8),
    "cylinder_16x8": lambda: cases.cylinder_case(ntheta=16, nr=8),
    "box_tet_4x3x2": lambda: cases.box_case("tet", nx=4, ny=3, nz=2),
    "plate_komega_8x4x2": lambda: cases.plate_case(ni=8, nj=4, nk=2),
}


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_golden_vectors(name, oracle_mod):
    """The oracle reproduces, bit for bit, the doubles the reference itself
    computed (tests/golden/make_golden.py runs the compiled reference)."""
    gold = np.load(os.path.join(ROOT, "tests", "golden", name + ".npz"))
    o = oracle_mod.Oracle(GOLDEN[name]())
    if "RK" in gold.files:
        R, RK = o.rans_residual(gold["W"], gold["K"])
        assert np.array_equal(R, gold["R"])
        assert np.array_equal(RK, gold["RK"])
        return
    out = o.residual(gold["W"], full=True)
    for k in ("R", "limiter", "grads", "mdot", "ghost"):
        assert np.array_equal(out[k].view(np.uint64), gold[k].view(np.uint64)), k
    if "time_terms" in gold.files:
        assert np.array_equal(o.time_terms(gold["W"], gold["dt"]) + 0.0, gold["time_terms"] + 0.0)


@pytest.mark.parametrize("flux", ["AUSM+up", "vanLeer"])
def test_complex_step_matches_finite_difference(flux, oracle_mod):
    """The complex-step residual agrees with central differences where the
    residual is smooth: unlimited reconstruction and in-plane perturbations.
    (The reference's one-sided Roe flux switches branch at u = 0, which every
    radial face on the x axis of the O-grid sits on, and its entropy fix has a
    kink at du = 0 on symmetry planes; those are genuine non-differentiable
    points, so Roe is compared against complex step on the GPU instead.)"""
    case = SMALL["cylinder"](flux=flux, limiter="none")
    o = oracle_mod.Oracle(case)
    rng = np.random.default_rng(7)
    dW = rng.standard_normal(case.state.shape) * np.array([100.0, 1.0, 1.0, 0.0, 0.3])
    jv = o.residual_cstep(case.state, dW)
    h = 1e-6
    fd = (o.residual(case.state + h * dW) - o.residual(case.state - h * dW)) / (2 * h)
    cols = [0, 1, 2, 4]  # w stays identically zero in this 2-D case
    scale = np.abs(jv[:, cols]).max(axis=0)
    assert (np.abs(jv - fd)[:, cols].max(axis=0) / scale).max() < 1e-5


def test_oracle_rans_inlet_values(oracle_mod):
    """RANS::set_bcs inlet values (rans_set_bcs.cc:56-65): k = max(kLow,
    1.5 (I |V|)^2), omega = rho k / (ratio mu(T)), mu_t = ratio mu(T), with the
    flat plate's freestream (I = 1e-3, ratio 1); no-slip wall mu_t = 0."""
    import tempfile
    from freecfd_b200 import cases
    case = cases.plate_case(ni=8, nj=4, nk=2, turbulent=True)
    o = oracle_mod.Oracle(case, tempfile.mkdtemp())
    bcs = o.rans_bcs()
    k, omega = case.kfree
    assert bcs[0, 0] == 1 and abs(bcs[0, 1] - k) <= 1e-14 * k and abs(bcs[0, 2] - omega) <= 1e-12 * omega
    assert bcs[2, 3] == 1 and bcs[2, 4] == 0.0          # wall
    assert bcs[1, 0] == 0 and bcs[3, 0] == 0             # outlet, symmetry: extrapolated


def test_rans_complex_step_matches_finite_difference(oracle_mod):
    """The oracle's complex step of the coupled RANS residual agrees with
    central differences of its own residual (limiter off, v perturbed)."""
    case = cases.plate_case(ni=8, nj=4, nk=2, turbulent=True, limiter="none")
    o = oracle_mod.Oracle(case)
    W = case.state.copy()
    rng = np.random.default_rng(3)
    W[:, 2] = 0.02 * W[:, 1] * rng.uniform(-1.0, 1.0, W.shape[0])
    K = case.kstate
    dW = rng.standard_normal(W.shape) * np.abs(W).max(axis=0) * np.array([1, 1, 1, 0, 1]) * 1e-3
    dK = rng.standard_normal(K.shape) * np.abs(K).max(axis=0) * 1e-3
    dR, dRK = o.rans_residual_cstep(W, K, dW, dK)
    h = 1e-6
    Rp, RKp = o.rans_residual(W + h * dW, K + h * dK)
    Rm, RKm = o.rans_residual(W - h * dW, K - h * dK)
    cols = [0, 1, 2, 4]
    e1 = (np.abs(dR - (Rp - Rm) / (2 * h))[:, cols].max(axis=0) / np.abs(dR[:, cols]).max(axis=0)).max()
    e2 = (np.abs(dRK - (RKp - RKm) / (2 * h)).max(axis=0) / np.abs(dRK).max(axis=0)).max()
    assert e1 < 1e-5 and e2 < 1e-5, (e1, e2)
