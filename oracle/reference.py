"""The reference itself, compiled from its own sources — TEST INFRASTRUCTURE ONLY.

``oracle/_ref/freecfd_ref`` is Free CFD's unmodified source tree compiled
with single-process stand-ins for MPI, PETSc, ParMETIS and CGNS
(``oracle/ref/include``) and linked with the driver ``oracle/ref/harness.cpp``
(``make -C oracle ref``; it needs the reference's sources, so it is built
where they are and travels as a binary).  Each call runs the binary in a fresh
process: the reference keeps its grid, deck and solver state in process-wide
globals (main.cc:67-82), so one process holds one case.

Grids are handed over in the reference's own raw grid file ``grid.raw``
(``Grid::write_raw``, grid/grid.cc:346-394; read back by ``Grid::read_raw``,
grid/grid_reader_cgns.cc:433-489): node count and coordinates, cell count and
connectivity offsets, connectivity, the node set of each boundary region, and
the region names with their indices.

Only tests/ and bench.py's reference arm use this module, as the checker and
as the CPU baseline; the freecfd_b200 product never touches it.
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BINARY = os.path.join(HERE, "_ref", "freecfd_ref")


def available() -> bool:
    return os.path.exists(BINARY)


def build(ref_root: str = "/root/reference") -> bool:
    """Compile the reference into oracle/_ref when its sources are present."""
    if not os.path.isdir(os.path.join(ref_root, "src")):
        return available()
    subprocess.run(["make", "-C", HERE, "-s", "-j8", "ref", f"REF={ref_root}"], check=True)
    return available()


def write_grid_raw(mesh, path: str) -> None:
    """``Grid::write_raw`` layout (int32 counts, Vec3D = three doubles)."""
    nodes = np.ascontiguousarray(mesh.nodes, dtype=np.float64)
    cidx = np.ascontiguousarray(mesh.conn_index[:-1], dtype=np.int32)
    conn = np.ascontiguousarray(mesh.conn, dtype=np.int32)
    with open(path, "wb") as fh:
        fh.write(np.int32(nodes.shape[0]).tobytes())
        fh.write(nodes.tobytes())
        fh.write(np.int32(cidx.shape[0]).tobytes())
        fh.write(cidx.tobytes())
        fh.write(np.int32(conn.shape[0]).tobytes())
        fh.write(conn.tobytes())
        nbc = len(mesh.bc_nodes)
        fh.write(np.int32(nbc).tobytes())
        for s in mesh.bc_nodes:
            s = np.unique(np.asarray(s, dtype=np.int32))      # std::set order
            fh.write(np.int32(s.shape[0]).tobytes())
            fh.write(s.tobytes())
        names = sorted((f"BC_{b + 1}", b) for b in range(nbc))  # std::map<string,int> order
        for name, b in names:
            raw = name.encode()
            fh.write(np.int32(len(raw)).tobytes())
            fh.write(raw)
            fh.write(np.int32(b).tobytes())


class Reference:
    """One case (deck + CELL-type raw mesh) run through the compiled reference."""

    def __init__(self, case, workdir: str | None = None, timeout: float = 3600.0):
        if not available():
            raise RuntimeError("the compiled reference is missing (make -C oracle ref)")
        self._tmp = None
        if workdir is None:
            self._tmp = tempfile.mkdtemp(prefix="fcfd_ref_")
            workdir = self._tmp
        self.dir = workdir
        self.timeout = timeout
        deck_path = case.write_deck(workdir)
        self.deck = os.path.splitext(os.path.basename(deck_path))[0]
        write_grid_raw(case.mesh, os.path.join(workdir, "grid.raw"))
        self.sizes = None

    def close(self):
        if self._tmp is not None:
            shutil.rmtree(self._tmp, ignore_errors=True)
            self._tmp = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, cmd: str, *args: str) -> dict:
        p = subprocess.run([BINARY, self.dir, self.deck, cmd, *args], capture_output=True, text=True,
                           timeout=self.timeout)
        if p.returncode != 0:
            raise RuntimeError(f"freecfd_ref {cmd} failed (rc {p.returncode}): {p.stderr.strip()[-2000:]}")
        for line in p.stdout.splitlines():
            if line.startswith("FCFD_REF_RESULT "):
                self.sizes = json.loads(line[len("FCFD_REF_RESULT "):])
                return self.sizes
        raise RuntimeError(f"freecfd_ref {cmd}: no result line")

    def _out(self, name: str) -> str:
        d = os.path.join(self.dir, name)
        os.makedirs(d, exist_ok=True)
        return d

    def _put(self, name: str, a) -> str:
        path = os.path.join(self.dir, name)
        np.ascontiguousarray(a, dtype=np.float64).tofile(path)
        return path

    @staticmethod
    def _get(d: str, name: str, dtype=np.float64):
        return np.fromfile(os.path.join(d, name), dtype=dtype)

    def mesh(self) -> dict:
        """Connectivity, geometry and LSQ weights in reference order (the
        fields and layout of oracle.Oracle.connectivity / geometry /
        grad_weights)."""
        d = self._out("mesh")
        s = self.run("mesh", d)
        nf, nt = s["nf"], s["ntot"]
        g = lambda n: self._get(d, n + ".i32", np.int32)  # noqa: E731
        f = lambda n: self._get(d, n + ".f64")  # noqa: E731
        return dict(face_parent=g("face_parent"), face_neighbor=g("face_neighbor"), face_bc=g("face_bc"),
                    face_nodes=g("face_nodes").reshape(nf, 4), cell_face_index=g("cell_face_index"),
                    cell_faces=g("cell_faces"), nbr_index=g("nbr_index"), nbrs=g("nbrs"),
                    grad_index=g("grad_index"), grad_keys=g("grad_keys"),
                    grad_weights=f("grad_weights").reshape(-1, 3),
                    face_normal=f("face_normal").reshape(nf, 3), face_area=f("face_area"),
                    face_centroid=f("face_centroid").reshape(nf, 3), face_avg=f("face_avg").reshape(nf, 2),
                    cell_centroid=f("cell_centroid").reshape(nt, 3), cell_volume=f("cell_volume"),
                    cell_length=f("cell_length"), cell_wall_distance=f("cell_wall_distance"),
                    length_scale=float(f("length_scale")[0]))

    def residual(self, W, K=None) -> dict:
        """The rhs the reference assembles for state W[nc][5] (and, for a
        k-omega deck, K[nc][2]), with mdot, weightL, gradients, limiters and
        ghost states; RK[nc][2] and mu_t for k-omega."""
        d = self._out("residual")
        args = [self._put("W.bin", W), d]
        if K is not None:
            args.append(self._put("K.bin", K))
        s = self.run("residual", *args)
        nc, nf, nt = s["nc"], s["nf"], s["ntot"]
        out = dict(R=self._get(d, "R.f64").reshape(nc, 5), mdot=self._get(d, "mdot.f64"),
                   weightL=self._get(d, "weightL.f64"), grads=self._get(d, "grads.f64").reshape(nt, 15),
                   limiter=self._get(d, "limiter.f64").reshape(nc, 5),
                   ghost=self._get(d, "ghost.f64").reshape(nt - nc, 5))
        assert out["mdot"].shape[0] == nf
        if K is not None:
            out["RK"] = self._get(d, "RK.f64").reshape(nc, 2)
            out["mu_t"] = self._get(d, "mu_t.f64")
        return out

    def time_terms(self, W, dt):
        """The diagonal blocks P V / dt (nc, 5, 5) of NavierStokes::time_terms."""
        d = self._out("timeterms")
        s = self.run("timeterms", self._put("W.bin", W), self._put("dt.bin", dt), d)
        return self._get(d, "blocks.f64").reshape(s["nc"], 5, 5)

    def diag_blocks(self, W, dt):
        """Diagonal blocks (nc, 5, 5) of the reference's implicit operator:
        P V / dt minus the first-order finite-difference Jacobian of the
        cell's own residual (assemble_linear_system + time_terms)."""
        d = self._out("diagblocks")
        s = self.run("diagblocks", self._put("W.bin", W), self._put("dt.bin", dt), d)
        return self._get(d, "blocks.f64").reshape(s["nc"], 5, 5)

    def local_dt(self, W):
        """update_time_step at time step 1 with the deck's time-marching
        options: (dt per cell, time after the step, max CFL)."""
        d = self._out("dt")
        s = self.run("dt", self._put("W.bin", W), d)
        a = self._get(d, "dt.f64")
        nc = s["nc"]
        return a[:nc], float(a[nc]), float(a[nc + 1])

    def bench_command(self, W, evals: int, warmup: int, K=None) -> list:
        """Command line of `evals` timed residual evaluations after `warmup`
        untimed ones (one process; prints {'evaluations', 'seconds', ...})."""
        args = [self._put("W.bin", W), str(int(evals)), str(int(warmup))]
        if K is not None:
            args.append(self._put("K.bin", K))
        return [BINARY, self.dir, self.deck, "bench", *args]

    def bench(self, W, evals: int, warmup: int = 1, K=None) -> dict:
        cmd = self.bench_command(W, evals, warmup, K)
        return self.run("bench", *cmd[4:])
