"""Synthetic benchmark cases: raw CELL-type meshes, input decks and seeded states.

Free CFD reads its meshes through ``Grid::readCGNS`` into a ``GridRawData``
record (grid/grid.h:61-78): node coordinates, a cell connectivity list in
CGNS element node order (HEXA_8 / PENTA_6) and, for every boundary-condition
region, the set of node ids on it.  The benchmark meshes of this project have
no CGNS file, so they are generated here in memory with exactly that shape:

* cells are listed in generation order (i fastest, then j, then k) and use the
  CGNS node order, so ``hexaFaces``/``prismFaces`` of
  grid/grid_create_elements.cc:187-201 give outward normals;
* boundary region ``b`` of the raw data is ``BC_{b+1}`` of the deck, as in
  grid/grid_reader_cgns.cc:100-102 (regions are numbered by first appearance);
* one-cell-thick 2-D meshes carry their front and back planes in a symmetry
  region, which is what ``set_lengthScales`` (main.cc:456-491) expects.

Every array is plain numpy; the same generated mesh feeds the CUDA library and
the CPU oracle.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

R_UNIV = 8314.47215          # material/material.h:26
R_AIR = 287.0
MW_AIR = R_UNIV / R_AIR


@dataclass
class RawMesh:
    """CELL-type raw grid (same meaning as ``GridRawData``, grid/grid.h:61-78)."""
    nodes: np.ndarray            # (N, 3) float64
    conn_index: np.ndarray       # (Nc+1,) int32, CSR offsets into conn
    conn: np.ndarray             # (sum,) int32, node ids in CGNS element order
    bc_nodes: list               # list of sorted int32 arrays, one per BC region
    dimension: int = 2

    @property
    def n_cells(self) -> int:
        return int(self.conn_index.shape[0] - 1)

    def bc_csr(self):
        idx = np.zeros(len(self.bc_nodes) + 1, dtype=np.int32)
        for b, s in enumerate(self.bc_nodes):
            idx[b + 1] = idx[b] + len(s)
        flat = (np.concatenate(self.bc_nodes).astype(np.int32)
                if self.bc_nodes else np.zeros(0, np.int32))
        return idx, flat


@dataclass
class Case:
    name: str
    mesh: RawMesh
    deck: str                    # input deck text (reference format)
    materials: dict = field(default_factory=dict)   # name -> .mat text
    state: np.ndarray = None     # (Nc, 5) float64 seeded primitive state p,u,v,w,T
    freestream: tuple = ()       # (p, u, v, w, T)
    workload: str = ""
    kstate: np.ndarray = None    # (Nc, 2) seeded turbulence state k, omega (k-omega decks)
    kfree: tuple = ()            # (k, omega) of the freestream

    def write_deck(self, directory: str) -> str:
        """Write the deck (and any .mat files) into ``directory``; return deck path."""
        os.makedirs(directory, exist_ok=True)
        for mname, text in self.materials.items():
            with open(os.path.join(directory, mname + ".mat"), "w") as fh:
                fh.write(text)
        path = os.path.join(directory, self.name + ".in")
        with open(path, "w") as fh:
            fh.write(self.deck)
        return path


# ----------------------------------------------------------------------------
# mesh builders
# ----------------------------------------------------------------------------

def _extrude_quads(xy: np.ndarray, quads: np.ndarray, z: np.ndarray):
    """Stack a 2-D node set over z levels and build HEXA_8 cells.

    ``xy`` is (n2, 2); ``quads`` (nq, 4) counter-clockwise seen from +z.
    Returns nodes (n2*len(z), 3) and hex connectivity (nq*(len(z)-1), 8).
    """
    n2 = xy.shape[0]
    nz = z.shape[0]
    nodes = np.empty((n2 * nz, 3), dtype=np.float64)
    for k in range(nz):
        nodes[k * n2:(k + 1) * n2, 0] = xy[:, 0]
        nodes[k * n2:(k + 1) * n2, 1] = xy[:, 1]
        nodes[k * n2:(k + 1) * n2, 2] = z[k]
    cells = []
    for k in range(nz - 1):
        lo = quads + k * n2
        hi = quads + (k + 1) * n2
        cells.append(np.concatenate([lo, hi], axis=1))
    return nodes, np.concatenate(cells, axis=0).astype(np.int32)


def _cells_to_csr(cells: np.ndarray):
    n, m = cells.shape
    idx = (np.arange(n + 1, dtype=np.int64) * m).astype(np.int32)
    return idx, cells.reshape(-1).astype(np.int32)


def _structured_quads(ni: int, nj: int, periodic_i: bool = False):
    """Quads over an (ni+1 or ni) x (nj+1) node lattice, node id = j*nI + i."""
    nI = ni if periodic_i else ni + 1
    i = np.arange(ni)
    j = np.arange(nj)
    I, J = np.meshgrid(i, j, indexing="xy")          # J rows, I fastest
    I = I.reshape(-1)
    J = J.reshape(-1)
    ip = (I + 1) % nI if periodic_i else I + 1
    n00 = J * nI + I
    n10 = J * nI + ip
    n11 = (J + 1) * nI + ip
    n01 = (J + 1) * nI + I
    return nI, n00, n10, n11, n01


def wedge_mesh(ni: int = 120, nj: int = 60, length: float = 3.0,
               height: float = 1.5, ramp_deg: float = 15.0, dz: float = 1.0 / 32.0):
    """Euler 15-degree wedge/ramp: inlet, outlet (right + top), symmetry, slip wall.

    BC regions (deck order): 1 inlet, 2 outlet, 3 symmetry (front/back), 4 slip wall.
    """
    nI, n00, n10, n11, n01 = _structured_quads(ni, nj)
    x1 = np.linspace(0.0, length, ni + 1)
    yb = np.maximum(0.0, x1 - length / 3.0) * math.tan(math.radians(ramp_deg))
    jj = np.arange(nj + 1) / nj
    X = np.repeat(x1[None, :], nj + 1, axis=0)
    Y = yb[None, :] + (height - yb[None, :]) * jj[:, None]
    xy = np.stack([X.reshape(-1), Y.reshape(-1)], axis=1)
    quads = np.stack([n00, n10, n11, n01], axis=1)     # ccw: +x then +y
    nodes, cells = _extrude_quads(xy, quads, np.array([0.0, dz]))
    n2 = xy.shape[0]
    ii = np.tile(np.arange(nI), nj + 1)
    jn = np.repeat(np.arange(nj + 1), nI)
    both = lambda mask: np.sort(np.concatenate([np.nonzero(mask)[0], np.nonzero(mask)[0] + n2])).astype(np.int32)
    inlet = both(ii == 0)
    outlet = both((ii == ni) | (jn == nj))
    sym = np.arange(2 * n2, dtype=np.int32)
    wall = both(jn == 0)
    idx, conn = _cells_to_csr(cells)
    return RawMesh(nodes, idx, conn, [inlet, outlet, sym, wall], dimension=2)


def _ogrid_radii(nr: int, r0: float, r1: float, dr0: float):
    """Geometric radial spacing with first step dr0 between r0 and r1."""
    span = r1 - r0
    if abs(dr0 * nr - span) < 1e-14:
        return r0 + dr0 * np.arange(nr + 1)
    lo, hi = 1.0 + 1e-12, 2.0
    f = lambda q: dr0 * (q ** nr - 1.0) / (q - 1.0) - span
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if f(mid) > 0:
            hi = mid
        else:
            lo = mid
    q = 0.5 * (lo + hi)
    steps = dr0 * q ** np.arange(nr)
    r = r0 + np.concatenate([[0.0], np.cumsum(steps)])
    r[-1] = r1
    return r


def cylinder_mesh(ntheta: int = 256, nr: int = 128, r0: float = 0.5,
                  r1: float = 15.0, dr0: float = 1e-3, dz: float = 1.0 / 32.0,
                  jitter: float = 0.0, seed: int = 4321, prisms: bool = False):
    """O-grid around a cylinder of diameter 1 (periodic in theta).

    BC regions (deck order): 1 wall (r=r0), 2 inlet (outer ring, x<=0),
    3 outlet (outer ring, x>=0), 4 symmetry (front/back).
    ``jitter`` moves interior nodes by U(-jitter, jitter) of the local spacing
    (seeded); ``prisms`` splits every hex into two PENTA_6 along its n00-n11
    diagonal.
    """
    assert ntheta % 4 == 0
    r = _ogrid_radii(nr, r0, r1, dr0)
    th = 2.0 * math.pi * np.arange(ntheta) / ntheta
    R = np.repeat(r[:, None], ntheta, axis=1)
    T = np.repeat(th[None, :], nr + 1, axis=0)
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        dr = np.diff(r)
        local_dr = np.minimum(np.concatenate([[dr[0]], dr]), np.concatenate([dr, [dr[-1]]]))
        dth = 2.0 * math.pi / ntheta
        ur = rng.uniform(-jitter, jitter, size=(nr + 1, ntheta))
        ut = rng.uniform(-jitter, jitter, size=(nr + 1, ntheta))
        R[1:nr] += ur[1:nr] * local_dr[1:nr, None]
        T[1:nr] += ut[1:nr] * dth
    xy = np.stack([(R * np.cos(T)).reshape(-1), (R * np.sin(T)).reshape(-1)], axis=1)
    nI, n00, n10, n11, n01 = _structured_quads(ntheta, nr, periodic_i=True)
    # i runs along +theta, j along +r: (i,j),(i,j+1),(i+1,j+1),(i+1,j) is ccw
    n2 = xy.shape[0]
    if not prisms:
        quads = np.stack([n00, n01, n11, n10], axis=1)
        nodes, cells = _extrude_quads(xy, quads, np.array([0.0, dz]))
    else:
        nodes = np.concatenate([np.c_[xy, np.zeros(n2)], np.c_[xy, np.full(n2, dz)]])
        a = np.stack([n00, n01, n11], axis=1)
        b = np.stack([n00, n11, n10], axis=1)
        tri = np.stack([a, b], axis=1).reshape(-1, 3)     # per quad: A then B
        cells = np.concatenate([tri, tri + n2], axis=1).astype(np.int32)
    jn = np.repeat(np.arange(nr + 1), ntheta)
    it = np.tile(np.arange(ntheta), nr + 1)
    q1, q3 = ntheta // 4, 3 * ntheta // 4
    both = lambda mask: np.sort(np.concatenate([np.nonzero(mask)[0], np.nonzero(mask)[0] + n2])).astype(np.int32)
    wall = both(jn == 0)
    inlet = both((jn == nr) & (it >= q1) & (it <= q3))
    outlet = both((jn == nr) & ((it >= q3) | (it <= q1)))
    sym = np.arange(2 * n2, dtype=np.int32)
    idx, conn = _cells_to_csr(cells)
    return RawMesh(nodes, idx, conn, [wall, inlet, outlet, sym], dimension=2)


def plate_mesh(ni: int = 384, nj: int = 192, nk: int = 4, plate: float = 2.0,
               upstream: float = 0.5, height: float = 1.0, y1: float = 1.1e-5,
               span: float = 0.1):
    """3-D flat plate: inlet, outlet (right + top), no-slip wall (y=0, x>=0),
    symmetry (y=0 upstream and the two z planes).

    BC regions (deck order): 1 inlet, 2 outlet, 3 wall, 4 symmetry.
    """
    nu = max(2, ni // 6)
    npl = ni - nu
    # plate: tanh clustering at the leading edge
    s = np.linspace(0.0, 1.0, npl + 1)
    beta = 2.5
    xp = plate * (1.0 + np.tanh(beta * (s - 1.0)) / math.tanh(beta))
    xp[0] = 0.0
    xp[-1] = plate
    # upstream: mirror of the first plate spacing, geometric toward the inlet
    d0 = xp[1] - xp[0]
    xu_r = _ogrid_radii(nu, 0.0, upstream, min(d0, upstream / nu))
    xu = -xu_r[::-1]
    x1 = np.concatenate([xu[:-1], xp])
    y = _ogrid_radii(nj, 0.0, height, min(y1, height / nj))
    nI = ni + 1
    X = np.repeat(x1[None, :], nj + 1, axis=0)
    Y = np.repeat(y[:, None], nI, axis=1)
    xy = np.stack([X.reshape(-1), Y.reshape(-1)], axis=1)
    _, n00, n10, n11, n01 = _structured_quads(ni, nj)
    quads = np.stack([n00, n10, n11, n01], axis=1)
    z = np.linspace(0.0, span, nk + 1)
    nodes, cells = _extrude_quads(xy, quads, z)
    n2 = xy.shape[0]
    ii = np.tile(np.arange(nI), nj + 1)
    jn = np.repeat(np.arange(nj + 1), nI)
    kk = np.repeat(np.arange(nk + 1), n2)
    i3 = np.tile(ii, nk + 1)
    j3 = np.tile(jn, nk + 1)
    xnode = nodes[:, 0]
    sel = lambda m: np.nonzero(m)[0].astype(np.int32)
    inlet = sel(i3 == 0)
    outlet = sel((i3 == ni) | (j3 == nj))
    wall = sel((j3 == 0) & (xnode >= 0.0))
    sym = sel(((j3 == 0) & (xnode <= 0.0)) | (kk == 0) | (kk == nk))
    idx, conn = _cells_to_csr(cells)
    return RawMesh(nodes, idx, conn, [inlet, outlet, wall, sym], dimension=3)


def box_mesh(nx: int = 6, ny: int = 4, nz: int = 3, kind: str = "tet", seed: int = 7,
             size=(1.0, 0.5, 0.375), jitter: float = 0.15):
    """3-D box of non-hex elements, for the element types the benchmark meshes
    do not use.  kind="tet": every hex split into six tetrahedra around its
    main diagonal (conforming across hexes); kind="hexpyr": a checkerboard of
    hexes and hexes split into six pyramids around a centre node (the quads
    still match).  Interior nodes are jittered by up to `jitter` x spacing.

    BC regions (deck order): 1 inlet x=0, 2 outlet x=Lx, 3 slip wall y=0,
    4 symmetry (y=Ly, z=0, z=Lz).
    """
    Lx, Ly, Lz = size
    xs, ys, zs = np.linspace(0, Lx, nx + 1), np.linspace(0, Ly, ny + 1), np.linspace(0, Lz, nz + 1)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    nodes = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1).astype(np.float64)
    nid = lambda i, j, k: (k * (ny + 1) + j) * (nx + 1) + i
    ii = np.tile(np.arange(nx + 1), (nz + 1) * (ny + 1))
    jj = np.tile(np.repeat(np.arange(ny + 1), nx + 1), nz + 1)
    kk = np.repeat(np.arange(nz + 1), (ny + 1) * (nx + 1))
    inner = (ii > 0) & (ii < nx) & (jj > 0) & (jj < ny) & (kk > 0) & (kk < nz)
    rng = np.random.default_rng(seed)
    h = np.array([Lx / nx, Ly / ny, Lz / nz])
    nodes[inner] += jitter * h * rng.uniform(-1.0, 1.0, size=(int(inner.sum()), 3))
    cells = []
    extra = []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                v = [nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k),
                     nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1), nid(i, j + 1, k + 1)]
                if kind == "tet":
                    for a, b, c in ((1, 2, 6), (2, 3, 6), (3, 7, 6), (7, 4, 6), (4, 5, 6), (5, 1, 6)):
                        t = [v[0], v[a], v[b], v[c]]
                        P = nodes[t]
                        if np.dot(np.cross(P[1] - P[0], P[2] - P[0]), P[3] - P[0]) < 0:
                            t[1], t[2] = t[2], t[1]
                        cells.append(t)
                elif (i + j + k) % 2 == 0:
                    cells.append(v)
                else:
                    ctr = len(nodes) + len(extra)
                    extra.append(nodes[v].mean(axis=0))
                    # hex faces (outward), each the base of one pyramid with the apex inside
                    for f in ((0, 3, 2, 1), (4, 5, 6, 7), (1, 2, 6, 5), (0, 4, 7, 3), (1, 5, 4, 0), (2, 3, 7, 6)):
                        a, b, c, d = (v[q] for q in f)
                        cells.append([a, d, c, b, ctr])
    if extra:
        nodes = np.vstack([nodes, np.array(extra)])
    idx = np.zeros(len(cells) + 1, dtype=np.int32)
    idx[1:] = np.cumsum([len(c) for c in cells])
    conn = np.concatenate([np.asarray(c, dtype=np.int32) for c in cells])
    nb = (nx + 1) * (ny + 1) * (nz + 1)
    sel = lambda m: np.nonzero(m)[0].astype(np.int32)
    inlet, outlet, wall = sel(ii == 0), sel(ii == nx), sel(jj == 0)
    sym = sel((jj == ny) | (kk == 0) | (kk == nz))
    assert nb == ii.size
    return RawMesh(nodes, idx, conn, [inlet, outlet, wall, sym], dimension=3)


def box_case(kind="tet", nx=6, ny=4, nz=3, seed=1234, flux="AUSM+up", limiter="vk", threshold=1.0,
             grad="lsqr") -> Case:
    """Inviscid M=0.6 flow through the non-hex box (parity coverage of the
    tetrahedron and pyramid face tables, LSQ stencils and geometry)."""
    mesh = box_mesh(nx, ny, nz, kind)
    p, T, M = 101325.0, 300.0, 0.6
    U = M * math.sqrt(1.4 * R_AIR * T)
    rho = p / (R_AIR * T)
    deck = f"""// Box {nx}x{ny}x{nz} split into {kind} elements, M={M}
reference {{Mach={_fmt(M)}; p=0.; T=0.;}}
time marching {{ CFLmax=50.; number of steps=500; }}
grid_1 {{
 file=box.cgns;
 dimension=3;
 equations=navier stokes;
 material (viscosity=0.; molar mass={_fmt(MW_AIR)}; gamma=1.4;);
 gradients (hex method={grad}; prism method={grad}; other method={grad};);
 navier stokes (limiter={limiter}; limiter threshold={_fmt(threshold)}; convective flux={flux};);
 write output ( volume variables=[V,p,T]; surface variables=[p]; );
 IC_1 (rho={_fmt(rho)}; V={_vec((U, 0.0, 0.0))}; p={_fmt(p)};);
 BC_1 (type=inlet; rho={_fmt(rho)}; V={_vec((U, 0.0, 0.0))};);
 BC_2 (type=outlet; p={_fmt(p)};);
 BC_3 (type=wall; kind=slip;);
 BC_4 (type=symmetry;);
}}
"""
    free = (p, U, 0.0, 0.0, T)
    st = seeded_state(mesh.n_cells, free, seed)
    st[:, 2] = 0.02 * U * np.random.default_rng(seed + 2).uniform(-1.0, 1.0, mesh.n_cells)
    st[:, 3] = 0.02 * U * np.random.default_rng(seed + 3).uniform(-1.0, 1.0, mesh.n_cells)
    return Case("box", mesh, deck, {}, st, free, f"euler_box_{nx}x{ny}x{nz}_{kind}_{flux}")


# ----------------------------------------------------------------------------
# decks
# ----------------------------------------------------------------------------

def _fmt(v: float) -> str:
    return repr(float(v))


def _vec(v) -> str:
    return "[" + ",".join(_fmt(x) for x in v) + "]"


def _air_mat(mu_ref: float, t_ref: float = 273.15, s: float = 110.4, pr: float = 0.72) -> str:
    return (
        f"molar mass={_fmt(MW_AIR)};\n"
        "gamma=1.4;\n"
        "equation of state { model=ideal gas; }\n"
        "viscosity {\n model=sutherlands;\n"
        f" reference viscosity={_fmt(mu_ref)};\n"
        f" reference temperature={_fmt(t_ref)};\n"
        f" sutherland temperature={_fmt(s)};\n}}\n"
        f"thermal conductivity {{\n model=constant Prandtl;\n Pr={_fmt(pr)};\n}}\n"
    )


def _sutherland_ref(mu_at_t: float, t: float, t_ref: float = 273.15, s: float = 110.4) -> float:
    return mu_at_t / (((t / t_ref) ** 1.5) * (t_ref + s) / (t + s))


def seeded_state(n_cells: int, free: tuple, seed: int, amp: float = 0.01) -> np.ndarray:
    """Freestream times (1 + amp*U(-1,1)) per component and cell (seeded)."""
    rng = np.random.default_rng(seed)
    base = np.asarray(free, dtype=np.float64)[None, :]
    return base * (1.0 + amp * rng.uniform(-1.0, 1.0, size=(n_cells, 5)))


def wedge_case(ni=120, nj=60, seed=1234, flux="Roe", limiter="vk", threshold=1.0,
               order="second", grad="lsqr", ns_extra="") -> Case:
    mesh = wedge_mesh(ni, nj)
    p, T, M = 101325.0, 300.0, 2.5
    a = math.sqrt(1.4 * R_AIR * T)
    U = M * a
    deck = f"""// Euler wedge/ramp {ni}x{nj}x1, M={M}
reference {{Mach={_fmt(M)}; p=0.; T=0.;}}
time marching {{ CFLmax=120.; number of steps=500; ramp (initial=5.0; growth=1.1;); }}
grid_1 {{
 file=wedge.cgns;
 dimension=2;
 equations=navier stokes;
 material (viscosity=0.; molar mass={_fmt(MW_AIR)}; gamma=1.4;);
 gradients (hex method={grad}; prism method={grad};);
 navier stokes (limiter={limiter}; limiter threshold={_fmt(threshold)}; order={order}; convective flux={flux};{ns_extra});
 write output ( volume variables=[V,p,T]; surface variables=[p]; );
 IC_1 (p={_fmt(p)}; T={_fmt(T)}; V={_vec((U, 0.0, 0.0))};);
 BC_1 (type=inlet; p={_fmt(p)}; T={_fmt(T)}; V={_vec((U, 0.0, 0.0))};);
 BC_2 (type=outlet;);
 BC_3 (type=symmetry;);
 BC_4 (type=wall; kind=slip;);
}}
"""
    free = (p, U, 0.0, 0.0, T)
    st = seeded_state(mesh.n_cells, free, seed)
    return Case("wedge", mesh, deck, {}, st, free,
                f"euler_wedge_{ni}x{nj}x1_hex_roe_lsq_vk")


def cylinder_case(ntheta=256, nr=128, seed=1234, flux="Roe", limiter="vk",
                  threshold=1.0, r1=15.0, dr0=1e-3, ns_extra="", grad="lsqr") -> Case:
    mesh = cylinder_mesh(ntheta, nr, r1=r1, dr0=dr0)
    p, T, M, Re, D = 101325.0, 300.0, 0.2, 40.0, 1.0
    a = math.sqrt(1.4 * R_AIR * T)
    U = M * a
    rho = p / (R_AIR * T)
    mu = rho * U * D / Re
    mat = _air_mat(_sutherland_ref(mu, T))
    deck = f"""// Laminar cylinder O-grid {ntheta}x{nr}x1, M={M}, Re_D={Re}
reference {{Mach={_fmt(M)}; p=0.; T=0.;}}
time marching {{ CFLmax=50.; number of steps=500; }}
grid_1 {{
 file=cylinder.cgns;
 dimension=2;
 equations=navier stokes;
 material=air;
 gradients (hex method={grad}; prism method={grad};);
 navier stokes (limiter={limiter}; limiter threshold={_fmt(threshold)}; convective flux={flux};{ns_extra});
 write output ( volume variables=[V,p,T]; surface variables=[p]; load frequency=1; include bcs=[1]; );
 IC_1 (rho={_fmt(rho)}; V={_vec((U, 0.0, 0.0))}; p={_fmt(p)};);
 BC_1 (type=wall;);
 BC_2 (type=inlet; rho={_fmt(rho)}; V={_vec((U, 0.0, 0.0))};);
 BC_3 (type=outlet; p={_fmt(p)};);
 BC_4 (type=symmetry;);
}}
"""
    free = (p, U, 0.0, 0.0, T)
    st = seeded_state(mesh.n_cells, free, seed)
    return Case("cylinder", mesh, deck, {"air": mat}, st, free,
                f"laminar_cylinder_{ntheta}x{nr}x1_hex_roe_viscous")


def hypersonic_case(ntheta=512, nr=256, seed=1234, flux="AUSM+up", limiter="minmod",
                    r1=2.5, dr0=2e-3, jitter_seed=4321, ns_extra="", grad="lsqr") -> Case:
    mesh = cylinder_mesh(ntheta, nr, r1=r1, dr0=dr0 * 256.0 / nr, jitter=0.1,
                         seed=jitter_seed, prisms=True)
    p, T, M = 2000.0, 220.0, 8.0
    a = math.sqrt(1.4 * R_AIR * T)
    U = M * a
    deck = f"""// Hypersonic cylinder O-grid {ntheta}x{nr}x1 split into prisms, M={M}
reference {{Mach={_fmt(M)}; p=0.; T=0.;}}
time marching {{ CFLmax=1.e3; number of steps=500; ramp (initial=0.1; growth=1.1;); }}
grid_1 {{
 file=cylinder.cgns;
 dimension=2;
 equations=navier stokes;
 material (viscosity=0.; molar mass={_fmt(MW_AIR)}; gamma=1.4;);
 gradients (hex method={grad}; prism method={grad};);
 navier stokes (limiter={limiter}; convective flux={flux};{ns_extra});
 write output ( volume variables=[V,p,T]; surface variables=[p]; );
 IC_1 (p={_fmt(p)}; T={_fmt(T)}; V={_vec((U, 0.0, 0.0))};);
 BC_1 (type=wall; kind=slip;);
 BC_2 (type=inlet; p={_fmt(p)}; T={_fmt(T)}; V={_vec((U, 0.0, 0.0))};);
 BC_3 (type=outlet;);
 BC_4 (type=symmetry;);
}}
"""
    free = (p, U, 0.0, 0.0, T)
    st = seeded_state(mesh.n_cells, free, seed)
    return Case("hypersonic", mesh, deck, {}, st, free,
                f"hypersonic_cylinder_{ntheta}x{nr}x1_prism_ausm_minmod")


def plate_case(ni=384, nj=192, nk=4, seed=1234, flux="Roe", limiter="vk",
               threshold=1.0, turbulent=True, ns_extra="", grad="lsqr") -> Case:
    L, ReL = 2.0, 5e6
    p, T, M = 101325.0, 300.0, 0.2
    a = math.sqrt(1.4 * R_AIR * T)
    U = M * a
    rho = p / (R_AIR * T)
    mu = rho * U * L / ReL
    cf = 0.0576 * ReL ** -0.2
    utau = U * math.sqrt(cf / 2.0)
    y1 = mu / rho / utau
    mesh = plate_mesh(ni, nj, nk, plate=L, y1=y1 * 192.0 / nj)
    mat = _air_mat(_sutherland_ref(mu, T))
    turb = (" turbulence (model=k-omega;);\n" if turbulent else "")
    tin = " turbulence intensity=1.e-3; eddy viscosity ratio=1.;" if turbulent else ""
    deck = f"""// Turbulent flat plate {ni}x{nj}x{nk}, M={M}, Re_L={ReL}
reference {{Mach={_fmt(M)}; p=0.; T=0.;}}
time marching {{ CFLmax=50.; number of steps=500; }}
grid_1 {{
 file=plate.cgns;
 dimension=3;
 equations=navier stokes;
 material=air;
 gradients (hex method={grad}; prism method={grad};);
{turb} navier stokes (limiter={limiter}; limiter threshold={_fmt(threshold)}; convective flux={flux};{ns_extra});
 write output ( volume variables=[V,p,T]; surface variables=[p]; );
 IC_1 (rho={_fmt(rho)}; V={_vec((U, 0.0, 0.0))}; p={_fmt(p)};{tin});
 BC_1 (type=inlet; rho={_fmt(rho)}; V={_vec((U, 0.0, 0.0))};{tin});
 BC_2 (type=outlet; p={_fmt(p)};);
 BC_3 (type=wall;);
 BC_4 (type=symmetry;);
}}
"""
    free = (p, U, 0.0, 0.0, T)
    st = seeded_state(mesh.n_cells, free, seed)
    case = Case("plate", mesh, deck, {"air": mat}, st, free,
                f"rans_flat_plate_{ni}x{nj}x{nk}_hex_roe_viscous_komega" if turbulent else
                f"laminar_flat_plate_{ni}x{nj}x{nk}_hex_roe_viscous")
    if turbulent:
        # freestream k, omega as the reference's inlet / IC formulas give them
        # (rans.cc:112-116, rans_set_bcs.cc:61-65): intensity 1e-3, ratio 1
        k = max(1e-10, 1.5 * (1e-3 * U) ** 2)
        omega = rho * k / (1.0 * mu)
        case.kfree = (k, omega)
        rng = np.random.default_rng(seed + 1)
        case.kstate = np.array([k, omega])[None, :] * (1.0 + 0.01 * rng.uniform(-1.0, 1.0, size=(mesh.n_cells, 2)))
    return case


CONFIGS = {
    "wedge": wedge_case,
    "cylinder": cylinder_case,
    "hypersonic": hypersonic_case,
    "plate": plate_case,
}


# ----------------------------------------------------------------------------
# Tecplot FEPolyhedron grid files (the face-based input of grid_reader_tec.cc)
# ----------------------------------------------------------------------------

# element face tables (local node numbers, normals pointing out of the cell)
_ELEMENT_FACES = {
    8: ((0, 3, 2, 1), (4, 5, 6, 7), (1, 2, 6, 5), (0, 4, 7, 3), (1, 5, 4, 0), (2, 3, 7, 6)),
    6: ((0, 2, 1), (3, 4, 5), (0, 3, 5, 2), (1, 2, 5, 4), (0, 1, 4, 3)),
    5: ((0, 3, 2, 1), (0, 1, 4), (1, 2, 4), (3, 4, 2), (0, 4, 3)),
    4: ((0, 2, 1), (1, 2, 3), (0, 3, 2), (0, 1, 3)),
}


def mesh_faces(mesh: RawMesh, order: str = "cells", seed: int = 0):
    """Faces of a CELL-type mesh: node lists oriented out of the left cell,
    left / right cells (0-based, -1 for a boundary face).  ``order`` "cells"
    lists them as the cells are visited (each face once, by its first cell);
    "shuffled" permutes that list with ``seed``."""
    first = {}
    faces, left, right = [], [], []
    for c in range(mesh.n_cells):
        nodes = mesh.conn[mesh.conn_index[c]:mesh.conn_index[c + 1]]
        for t in _ELEMENT_FACES[len(nodes)]:
            fn = tuple(int(nodes[k]) for k in t)
            key = tuple(sorted(fn))
            if key in first:
                right[first[key]] = c
            else:
                first[key] = len(faces)
                faces.append(fn)
                left.append(c)
                right.append(-1)
    if order == "shuffled":
        perm = np.random.default_rng(seed).permutation(len(faces))
        faces = [faces[i] for i in perm]
        left = [left[i] for i in perm]
        right = [right[i] for i in perm]
    return faces, np.array(left, np.int64), np.array(right, np.int64)


def write_tecplot(mesh: RawMesh, path: str, bc_names=None, order: str = "cells", seed: int = 0) -> str:
    """Write ``mesh`` as a Tecplot FEPolyhedron file in the layout
    grid_reader_tec.cc reads: volume zone (block-packed coordinates, face node
    counts, 1-based face nodes, left and right elements, each block after one
    comment line), then one zone per BC region (``ZONE T="name"`` on its own
    line, then its node count and the coordinates of its nodes)."""
    faces, left, right = mesh_faces(mesh, order, seed)
    names = bc_names or ["BC_%d" % (b + 1) for b in range(len(mesh.bc_nodes))]

    def block(vals, fmt):
        out = []
        for i in range(0, len(vals), 8):
            out.append(" ".join(fmt % v for v in vals[i:i + 8]))
        return "\n".join(out) + "\n"

    nn = mesh.nodes.shape[0]
    with open(path, "w") as fh:
        fh.write('TITLE="freecfd_b200 grid"\nVARIABLES="X","Y","Z"\nZONE T="volume"\n')
        fh.write("ZONETYPE=FEPolyhedron, DATAPACKING=BLOCK, Nodes=%d, Elements=%d, Faces=%d, TotalNumFaceNodes=%d, "
                 "NumConnectedBoundaryFaces=0, TotalNumBoundaryConnections=0\n"
                 % (nn, mesh.n_cells, len(faces), sum(len(f) for f in faces)))
        for i in range(3):
            fh.write(block([float(x) for x in mesh.nodes[:, i]], "%.17g"))
        fh.write("# node count per face\n")
        fh.write(block([len(f) for f in faces], "%d"))
        fh.write("# face nodes\n")
        fh.write(block([n + 1 for f in faces for n in f], "%d"))
        fh.write("# left elements\n")
        fh.write(block([int(c) + 1 for c in left], "%d"))
        fh.write("# right elements\n")
        fh.write(block([int(c) + 1 for c in right], "%d"))
        for b, nodes in enumerate(mesh.bc_nodes):
            nodes = np.asarray(nodes)
            fh.write('ZONE T="%s"\n' % names[b])
            fh.write("ZONETYPE=FEQUADRILATERAL, DATAPACKING=BLOCK, Nodes=%d, Elements=0\n" % len(nodes))
            for i in range(3):
                fh.write(block([float(x) for x in mesh.nodes[nodes, i]], "%.17g"))
    return path


# ----------------------------------------------------------------------------
# cell renumbering
# ----------------------------------------------------------------------------
def renumber_cells(mesh: RawMesh, perm) -> RawMesh:
    """The same grid with its elements listed in the order `perm` (perm[new]
    = old): new cell i is old cell perm[i], with its node list unchanged.
    Nodes and boundary regions are untouched, so every face, normal, area,
    centroid and volume is the same; only cell and face numbering change
    (faces are discovered in the new cell order)."""
    perm = np.asarray(perm, dtype=np.int64)
    n = mesh.n_cells
    if perm.shape != (n,) or not np.array_equal(np.sort(perm), np.arange(n)):
        raise ValueError("perm must be a permutation of the cell indices")
    ci = np.asarray(mesh.conn_index, dtype=np.int64)
    sizes = ci[1:] - ci[:-1]
    new_sizes = sizes[perm]
    idx = np.zeros(n + 1, dtype=np.int32)
    idx[1:] = np.cumsum(new_sizes)
    take = np.concatenate([np.arange(ci[o], ci[o + 1]) for o in perm]) if n else np.zeros(0, np.int64)
    return RawMesh(mesh.nodes, idx, np.ascontiguousarray(mesh.conn[take], dtype=np.int32),
                   list(mesh.bc_nodes), mesh.dimension)


def renumber_case(case: Case, perm, label: str = "renumbered") -> Case:
    """`case` on its grid renumbered by `perm` (perm[new] = old), with the
    seeded cell states permuted the same way."""
    perm = np.asarray(perm, dtype=np.int64)
    return Case(case.name, renumber_cells(case.mesh, perm), case.deck, dict(case.materials),
                None if case.state is None else np.ascontiguousarray(case.state[perm]), case.freestream,
                f"{case.workload}_{label}", None if case.kstate is None else np.ascontiguousarray(case.kstate[perm]),
                case.kfree)


def shuffle_case(case: Case, seed: int = 0) -> Case:
    """`case` with its cells listed in a seeded random order: a grid whose
    element order carries no locality (an unordered export)."""
    perm = np.random.default_rng(seed).permutation(case.mesh.n_cells)
    return renumber_case(case, perm, f"shuffled{seed}")


def bandwidth(face_parent, face_neighbor, face_bc) -> int:
    """Largest |parent - neighbour| over interior faces (matrix bandwidth)."""
    fp, fn = np.asarray(face_parent), np.asarray(face_neighbor)
    m = np.asarray(face_bc) < 0
    return int(np.abs(fp[m] - fn[m]).max()) if m.any() else 0


def hypersonic_smooth_state(case: Case, centroids, width: float = 2.0) -> np.ndarray:
    """A start for the hypersonic cylinder without the impulsive start's
    vacuum: the seeded freestream pressure and temperature, the velocity
    blended (smoothstep) from zero at the wall (r = 0.5) to the freestream
    over `width` in radius.  The impulsive start's lee-side wall faces pull
    the M = 8 flow away faster than 2a/(gamma-1) and open a vacuum."""
    W = case.state.copy()
    x = np.asarray(centroids)[: W.shape[0]]
    s = np.clip((np.hypot(x[:, 0], x[:, 1]) - 0.5) / width, 0.0, 1.0)
    s = s * s * (3.0 - 2.0 * s)
    W[:, 1:4] *= s[:, None]
    return W


def hypersonic_shock_state(case: Case, centroids, radius: float = 1.2, seed: int = 7, mach: float = 8.0,
                           gamma: float = 1.4) -> np.ndarray:
    """A state with a captured bow-shock jump for the hypersonic cylinder:
    the seeded freestream state, with the cells whose centroid lies within
    `radius` of the axis replaced by the normal-shock state of the freestream
    (Rankine-Hugoniot p2/p1, T2/T1, u2/u1 at `mach`), plus a 1 % seeded
    perturbation.  The pressure jumps ~75x across one ring of faces."""
    p1, u1, v1, w1, T1 = case.freestream
    M2 = mach * mach
    pr = 1.0 + 2.0 * gamma / (gamma + 1.0) * (M2 - 1.0)
    rr = (gamma + 1.0) * M2 / ((gamma - 1.0) * M2 + 2.0)
    W = case.state.copy()
    x = np.asarray(centroids)[: W.shape[0]]
    inside = np.hypot(x[:, 0], x[:, 1]) < radius
    rng = np.random.default_rng(seed)
    jit = 1.0 + 0.01 * rng.uniform(-1.0, 1.0, (int(inside.sum()), 5))
    post = np.array([p1 * pr, u1 / rr, v1 / rr, w1 / rr, T1 * pr / rr])
    W[inside] = post * jit
    return W
