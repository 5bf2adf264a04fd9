"""Shared helpers for the parity tests: small instances of every benchmark
mesh family and the normwise comparison used throughout."""
import tempfile

import numpy as np

from freecfd_b200 import cases

# Small meshes of each family (the oracle finishes these in well under a second)
SMALL = {
    "wedge": lambda **kw: cases.wedge_case(ni=24, nj=12, **kw),
    "cylinder": lambda **kw: cases.cylinder_case(ntheta=32, nr=16, **kw),
    "hypersonic": lambda **kw: cases.hypersonic_case(ntheta=32, nr=16, **kw),
    "plate": lambda **kw: cases.plate_case(ni=24, nj=12, nk=3, turbulent=False, **kw),
}


# Tetrahedra and pyramids (the benchmark meshes are hexes and prisms only)
ELEMENTS = {
    "box_tet": lambda **kw: cases.box_case("tet", **kw),
    "box_hexpyr": lambda **kw: cases.box_case("hexpyr", **kw),
}
ALL = {**SMALL, **ELEMENTS}


def build_pair(case, oracle_mod, fb):
    """Oracle + product objects for the same case (decks in a temp dir)."""
    d = tempfile.mkdtemp(prefix="fcfd_")
    o = oracle_mod.Oracle(case, d)
    cs = fb.Case(case.write_deck(d))
    m = fb.Mesh(case.mesh, cs)
    return o, cs, m


def rel_err(a, b, floor=1e-300):
    """Normwise relative error per equation column: max|a-b| / max(max|b|, floor).

    ``floor`` keeps columns that are pure rounding noise (e.g. the z-momentum
    of a 2-D case) from being divided by ~0."""
    a = np.asarray(a).reshape(-1, np.asarray(a).shape[-1]) if np.asarray(a).ndim > 1 else np.asarray(a)[:, None]
    b = np.asarray(b).reshape(a.shape)
    scale = np.maximum(np.abs(b).max(axis=0), floor)
    return (np.abs(a - b).max(axis=0) / scale)


def res_err(a, b):
    """Normwise relative error of [n][5] residual-like arrays: per equation,
    with the three momentum components sharing one scale (on one-layer
    meshes the z-momentum column is rounding noise)."""
    a = np.asarray(a).reshape(-1, 5)
    b = np.asarray(b).reshape(a.shape)
    scale = np.abs(b).max(axis=0)
    scale[1:4] = scale[1:4].max()
    return np.abs(a - b).max(axis=0) / np.maximum(scale, 1e-300)


def flux_scale(case, mesh_geometry, gamma=1.4, R=287.0):
    """Per-equation magnitude of one face's freestream flux (mass, momentum,
    energy) times the largest face area: the size of the terms whose
    cancellation produces a residual."""
    p, u, v, w, T = case.freestream
    rho = p / (R * T)
    U = float(np.sqrt(u * u + v * v + w * w))
    H = gamma / (gamma - 1.0) * R * T + 0.5 * U * U
    A = float(np.max(mesh_geometry["face_area"]))
    mom = (rho * U * U + p) * A
    return np.array([rho * U * A, mom, mom, mom, rho * U * H * A])
