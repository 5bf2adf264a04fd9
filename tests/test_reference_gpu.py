"""The CUDA path against the reference itself (B200).

The golden vectors in tests/golden/ are outputs of the reference compiled
from its own sources (tests/golden/make_golden.py), and oracle/_ref/freecfd_ref
is that compiled reference; both travel with the repository, so these tests
compare the device's results directly with the reference's doubles, without
the oracle in between.  Bars as in tests/test_residual_gpu.py: residual, mdot
and the k-omega right-hand side within 1e-12 normwise relative per equation;
ghost states 1e-14; gradients 1e-12 of each variable's largest component;
limiters 1e-11.
"""
import os
import tempfile

import numpy as np
import pytest

from freecfd_b200 import cases
from tests.conftest import ROOT
from tests.util import rel_err, res_err

GOLDEN = {
    "wedge_12x6": lambda: cases.wedge_case(ni=12, nj=6),
    "hypersonic_16x8": lambda: cases.hypersonic_case(ntheta=16, nr=8),
    "cylinder_16x8": lambda: cases.cylinder_case(ntheta=16, nr=8),
    "box_tet_4x3x2": lambda: cases.box_case("tet", nx=4, ny=3, nz=2),
    "plate_komega_8x4x2": lambda: cases.plate_case(ni=8, nj=4, nk=2),
}


def _ns(case, fb):
    d = tempfile.mkdtemp(prefix="fcfd_")
    cs = fb.Case(case.write_deck(d))
    m = fb.Mesh(case.mesh, cs)
    return m, fb.NavierStokes(m, cs, 0)


def grad_err(g, ref, nc):
    g = np.asarray(g).reshape(nc, 5, 3)
    r = np.asarray(ref)[:nc].reshape(nc, 5, 3)
    scale = np.maximum(np.abs(r).max(axis=(0, 2)), 1e-300)
    return np.abs(g - r).max(axis=(0, 2)) / scale


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_golden_vectors_from_the_reference(name, fb):
    gold = np.load(os.path.join(ROOT, "tests", "golden", name + ".npz"))
    case = GOLDEN[name]()
    m, ns = _ns(case, fb)
    if "RK" in gold.files:
        R, RK = ns.rans_residual(gold["W"], gold["K"])
        assert res_err(R, gold["R"]).max() <= 1e-12
        assert rel_err(RK, gold["RK"]).max() <= 1e-12
        return
    R = ns.residual(gold["W"])
    st = ns.stages()
    assert res_err(R, gold["R"]).max() <= 1e-12
    assert rel_err(st["ghost"], gold["ghost"]).max() <= 1e-14
    assert grad_err(st["grads"], gold["grads"], m.nc).max() <= 1e-12
    assert rel_err(st["limiter"], gold["limiter"]).max() <= 1e-11
    assert rel_err(st["mdot"], gold["mdot"]).max() <= 1e-12


def cs_types(case):
    """BC region types of a generated deck in region order (BC_1, BC_2, ...)."""
    out = []
    for line in case.deck.splitlines():
        line = line.strip()
        if line.startswith("BC_") and "type=" in line:
            out.append(line.split("type=")[1].split(";")[0].strip())
    return out


def _reference_or_oracle(case):
    """The compiled reference where it travelled with the repository, else the
    oracle (held bit-exact to it by tests/test_reference_pin.py)."""
    from oracle import reference
    if reference.available():
        return "reference", reference.Reference(case).residual(case.state, case.kstate)
    import oracle
    o = oracle.Oracle(case)
    return "oracle", o.residual(case.state, full=True)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cylinder_256x128", "plate_384x192x4"])
def test_full_size_per_cell_parity(name, fb):
    """The benchmarked cylinder (32,768 cells) and the laminar flat plate at
    384x192x4 (294,912 cells): every stage and every cell's residual."""
    case = cases.cylinder_case() if name.startswith("cylinder") else cases.plate_case(turbulent=False)
    m, ns = _ns(case, fb)
    R = ns.residual(case.state)
    st = ns.stages()
    kind, ref = _reference_or_oracle(case)
    assert res_err(R, ref["R"]).max() <= 1e-12, kind
    assert rel_err(st["ghost"], ref["ghost"]).max() <= 1e-14, kind
    assert grad_err(st["grads"], ref["grads"], m.nc).max() <= 1e-12, kind
    assert rel_err(st["limiter"], ref["limiter"]).max() <= 1e-11, kind
    assert rel_err(st["mdot"], ref["mdot"]).max() <= 1e-12, kind


@pytest.mark.gpu
def test_full_size_rans_plate_parity(fb):
    """The k-omega plate 384x192x4: NS residual with the eddy viscosity and
    the k-omega right-hand side of RANS::terms, every cell."""
    case = cases.plate_case()
    m, ns = _ns(case, fb)
    R, RK = ns.rans_residual(case.state, case.kstate)
    kind, ref = _reference_or_oracle(case)
    if kind == "oracle":
        import oracle
        ref = dict(zip(("R", "RK"), oracle.Oracle(case).rans_residual(case.state, case.kstate)))
    assert res_err(R, ref["R"]).max() <= 1e-12, kind
    assert rel_err(RK, ref["RK"]).max() <= 1e-12, kind


@pytest.mark.gpu
@pytest.mark.parametrize("family", ["wedge", "cylinder", "hypersonic"])
def test_diag_blocks_against_reference(family, fb, oracle_mod):
    """The preconditioner's diagonal blocks V P/dt - J_cc.  The time-term part
    (cons2prim, ns_time_terms.cc:26-56,107-186) is isolated by evaluating the
    blocks at dt and 2 dt: the difference is P V / (2 dt), compared with the
    oracle's restatement (bit-exact to the reference) at 1e-12 of each block
    row (two roundings of blocks that carry the Jacobian too).  J_cc is the
    exact derivative of the first-order face fluxes here and a one-sided
    finite difference with step 1.5e-7 in the reference (get_jacobians,
    ns_assemble_linear_system.cc:197-267), so the two agree to the finite
    difference's error: 1e-5 normwise per equation (largest difference over
    cells and columns over the equation's largest entry).  The seeded states
    have v = 0 exactly, which puts faces whose normal is along y on the kink
    of the upwind switches, where a one-sided difference and a derivative
    pick different branches; a small seeded v moves the state off the kinks.

    One exception is the reference's, on viscous cases: at a boundary face
    get_jacobians re-applies the BC to the perturbed left state (right.T of
    an inlet with rho and V given follows the left velocity through the
    Riemann invariant), but face_state_adjust (ns_assemble_linear_system.cc:
    460-500) refreshes the face temperature, viscosity and conductivity only
    when T itself is perturbed, so the reference's difference quotients of
    the energy flux with respect to u and v miss that response there.  The
    energy row of cells with an inlet or outlet face is therefore left out
    on the viscous case; everywhere else every row is held to 1e-5."""
    case = {"wedge": lambda: cases.wedge_case(ni=24, nj=12),
            "cylinder": lambda: cases.cylinder_case(ntheta=32, nr=16),
            "hypersonic": lambda: cases.hypersonic_case(ntheta=32, nr=16)}[family]()
    W = case.state.copy()
    W[:, 2] += 1e-3 * case.freestream[1] * np.random.default_rng(7).uniform(-1.0, 1.0, W.shape[0])
    m, ns = _ns(case, fb)
    dt = np.random.default_rng(5).uniform(0.5, 2.0, m.nc) * 1e-5
    B1 = ns.diag_blocks(W, dt)
    B2 = ns.diag_blocks(W, 2.0 * dt)
    o = oracle_mod.Oracle(case)
    tt = o.time_terms(W, dt)
    half = B1 - B2
    scale = np.maximum(np.abs(tt).max(axis=2, keepdims=True), 1e-300)
    assert (np.abs(half - 0.5 * tt) / scale).max() <= 1e-12
    Jdev = tt - B1
    from oracle import reference
    if not reference.available():
        pytest.skip("the compiled reference did not travel with the repository")
    Jref = tt - reference.Reference(case).diag_blocks(W, dt)
    scale = np.abs(Jref).max(axis=(0, 2))
    diff = np.abs(Jdev - Jref)
    if family == "cylinder":          # viscous: see above
        con = m.connectivity()
        bc_type = {b: t for b, t in enumerate(cs_types(case))}
        io = np.array([any(bc_type.get(int(con["face_bc"][f]), 0) in ("inlet", "outlet")
                           for f in con["cell_faces"][con["cell_face_index"][c]:con["cell_face_index"][c + 1]])
                       for c in range(m.nc)])
        diff[io, 4, :] = 0.
    err = diff.max(axis=(0, 2)) / scale
    assert err.max() <= 1e-5, err
