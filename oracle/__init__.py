"""CPU oracle for Free CFD's residual path — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline/reference leg
may import this package, and only as the checker.  The freecfd_b200 product
never imports, links or executes anything here.

The oracle is a C++ restatement of the reference (oracle/oracle.cpp, with the
reference file:line it follows in each function's comment), built into
oracle/_build/liboracle.so by oracle/Makefile.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle shared library (g++, -ffp-contract=off)."""
    if force or not os.path.exists(_LIB_PATH) or (
            os.path.getmtime(_LIB_PATH) < max(os.path.getmtime(os.path.join(_HERE, f))
                                              for f in ("oracle.cpp", "deck.hpp"))):
        subprocess.run(["make", "-C", _HERE, "-s"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        vp = ctypes.c_void_p
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.orc_create.restype = vp
        L.orc_create_tecplot.restype = vp
        L.orc_create_tecplot.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
        L.orc_create.argtypes = [ctypes.c_char_p, ctypes.c_int, dp, ctypes.c_int, ip, ip, ctypes.c_int, ip, ip,
                                 ctypes.c_char_p, ctypes.c_int]
        L.orc_destroy.argtypes = [vp]
        L.orc_sizes.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
        L.orc_connectivity.argtypes = [vp] + [ip] * 10
        L.orc_nbr_total.argtypes = [vp]
        L.orc_nbr_total.restype = ctypes.c_int
        L.orc_geometry.argtypes = [vp] + [dp] * 9
        L.orc_grad_weights.argtypes = [vp, dp]
        L.orc_residual.argtypes = [vp] + [dp] * 7 + [ctypes.c_char_p, ctypes.c_int]
        L.orc_residual.restype = ctypes.c_int
        L.orc_residual_cstep.argtypes = [vp, dp, dp, ctypes.c_double, dp, ctypes.c_char_p, ctypes.c_int]
        L.orc_residual_cstep.restype = ctypes.c_int
        L.orc_local_dt.argtypes = [vp, dp, ctypes.c_double, ctypes.c_int, dp]
        L.orc_loads.argtypes = [vp, dp, dp, ctypes.c_double, dp, dp, ctypes.c_char_p, ctypes.c_int]
        L.orc_loads.restype = ctypes.c_int
        L.orc_rans_residual_cstep.argtypes = [vp, dp, dp, dp, dp, ctypes.c_double, dp, dp, ctypes.c_char_p, ctypes.c_int]
        L.orc_rans_residual_cstep.restype = ctypes.c_int
        L.orc_rans_residual.argtypes = [vp, dp, dp, dp, dp, ctypes.c_char_p, ctypes.c_int]
        L.orc_rans_residual.restype = ctypes.c_int
        L.orc_rans_bcs.argtypes = [vp, dp]
        L.orc_case_summary.argtypes = [vp, dp, ip]
        L.orc_time_terms.argtypes = [vp, dp, dp, dp]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


def _i(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) if a is not None else None


class Oracle:
    """Handle on one oracle grid + case (reference ordering throughout)."""

    def __init__(self, case, workdir: str | None = None, tecplot: str | None = None):
        """The case's deck with its CELL-type mesh, or (``tecplot`` = path) with
        the Tecplot FEPolyhedron grid file read by the restated readTEC."""
        L = lib()
        self._tmp = None
        if workdir is None:
            self._tmp = tempfile.TemporaryDirectory()
            workdir = self._tmp.name
        deck = case.write_deck(workdir)
        err = ctypes.create_string_buffer(512)
        if tecplot is not None:
            self.h = L.orc_create_tecplot(deck.encode(), str(tecplot).encode(), err, 512)
        else:
            m = case.mesh
            nodes = np.ascontiguousarray(m.nodes, dtype=np.float64)
            cidx = np.ascontiguousarray(m.conn_index, dtype=np.int32)
            conn = np.ascontiguousarray(m.conn, dtype=np.int32)
            bidx, bflat = m.bc_csr()
            self.h = L.orc_create(deck.encode(), nodes.shape[0], _d(nodes), m.n_cells, _i(cidx), _i(conn),
                                  len(m.bc_nodes), _i(bidx), _i(bflat), err, 512)
        if not self.h:
            raise RuntimeError("oracle: " + err.value.decode())
        s = (ctypes.c_longlong * 8)()
        L.orc_sizes(self.h, s)
        (self.nc, self.nf, self.nghost, self.ntot, self.nnodes, self.n_grad_entries,
         self.n_cell_faces, self.dimension) = [int(x) for x in s]

    def close(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None
        if self._tmp is not None:
            self._tmp.cleanup()
            self._tmp = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def connectivity(self):
        L = lib()
        nf, nc = self.nf, self.nc
        fp = np.empty(nf, np.int32); fn = np.empty(nf, np.int32); fb = np.empty(nf, np.int32)
        fnodes = np.empty(nf * 4, np.int32)
        cfi = np.empty(nc + 1, np.int32); cf = np.empty(self.n_cell_faces, np.int32)
        nbt = L.orc_nbr_total(self.h)
        ni = np.empty(nc + 1, np.int32); nb = np.empty(nbt, np.int32)
        gi = np.empty(nc + 1, np.int32); gk = np.empty(self.n_grad_entries, np.int32)
        L.orc_connectivity(self.h, _i(fp), _i(fn), _i(fb), _i(fnodes), _i(cfi), _i(cf), _i(ni), _i(nb), _i(gi), _i(gk))
        return dict(face_parent=fp, face_neighbor=fn, face_bc=fb, face_nodes=fnodes.reshape(nf, 4),
                    cell_face_index=cfi, cell_faces=cf, nbr_index=ni, nbrs=nb, grad_index=gi, grad_keys=gk)

    def geometry(self):
        nf, nt = self.nf, self.ntot
        out = dict(face_normal=np.empty((nf, 3)), face_area=np.empty(nf), face_centroid=np.empty((nf, 3)),
                   face_avg=np.empty((nf, 2)), cell_centroid=np.empty((nt, 3)), cell_volume=np.empty(nt),
                   cell_length=np.empty(nt), cell_wall_distance=np.empty(nt))
        lref = ctypes.c_double()
        lib().orc_geometry(self.h, _d(out["face_normal"]), _d(out["face_area"]), _d(out["face_centroid"]),
                           _d(out["face_avg"]), _d(out["cell_centroid"]), _d(out["cell_volume"]),
                           _d(out["cell_length"]), _d(out["cell_wall_distance"]), ctypes.byref(lref))
        out["length_scale"] = lref.value
        return out

    def grad_weights(self):
        w = np.empty((self.n_grad_entries, 3))
        lib().orc_grad_weights(self.h, _d(w))
        return w

    def residual(self, W, full: bool = False):
        W = np.ascontiguousarray(W, dtype=np.float64).reshape(self.nc, 5)
        R = np.empty((self.nc, 5))
        err = ctypes.create_string_buffer(512)
        if full:
            mdot = np.empty(self.nf); wl = np.empty(self.nf)
            grads = np.empty((self.ntot, 15)); lim = np.empty((self.nc, 5)); ghost = np.empty((self.nghost, 5))
            rc = lib().orc_residual(self.h, _d(W), _d(R), _d(mdot), _d(wl), _d(grads), _d(lim), _d(ghost), err, 512)
        else:
            rc = lib().orc_residual(self.h, _d(W), _d(R), None, None, None, None, None, err, 512)
        if rc != 0:
            raise RuntimeError("oracle: " + err.value.decode())
        if full:
            return dict(R=R, mdot=mdot, weightL=wl, grads=grads, limiter=lim, ghost=ghost)
        return R

    def residual_cstep(self, W, dW, h=1e-30):
        W = np.ascontiguousarray(W, dtype=np.float64).reshape(self.nc, 5)
        dW = np.ascontiguousarray(dW, dtype=np.float64).reshape(self.nc, 5)
        dR = np.empty((self.nc, 5))
        err = ctypes.create_string_buffer(512)
        rc = lib().orc_residual_cstep(self.h, _d(W), _d(dW), h, _d(dR), err, 512)
        if rc != 0:
            raise RuntimeError("oracle: " + err.value.decode())
        return dR

    def loads(self, W, dW=None, h=1e-30, moments=False):
        """Force on every boundary region [n_bc][3] (convective minus diffusive
        momentum flux summed over the region's faces); with dW, its
        complex-step directional derivative along dW.  moments=True returns
        (force, moment about the deck's moment center)."""
        W = np.ascontiguousarray(W, dtype=np.float64).reshape(self.nc, 5)
        nbc = int(self.case_summary()[1][5])
        out = np.empty((nbc, 3))
        err = ctypes.create_string_buffer(512)
        if dW is not None:
            dW = np.ascontiguousarray(dW, dtype=np.float64).reshape(self.nc, 5)
        mom = np.empty((nbc, 3)) if moments else None
        rc = lib().orc_loads(self.h, _d(W), None if dW is None else _d(dW), h, _d(out), None if mom is None else _d(mom),
                             err, 512)
        if rc != 0:
            raise RuntimeError("oracle: " + err.value.decode())
        return (out, mom) if moments else out

    def rans_residual(self, W, K):
        """k-omega RANS residual: (R[nc][5] with eddy viscosity, RK[nc][2])."""
        W = np.ascontiguousarray(W, dtype=np.float64).reshape(self.nc, 5)
        K = np.ascontiguousarray(K, dtype=np.float64).reshape(self.nc, 2)
        R = np.empty((self.nc, 5))
        RK = np.empty((self.nc, 2))
        err = ctypes.create_string_buffer(512)
        rc = lib().orc_rans_residual(self.h, _d(W), _d(K), _d(R), _d(RK), err, 512)
        if rc != 0:
            raise RuntimeError("oracle: " + err.value.decode())
        return R, RK

    def rans_residual_cstep(self, W, K, dW, dK, h=1e-30):
        """Complex-step directional derivative of the RANS residual along (dW, dK)."""
        a = [np.ascontiguousarray(x, dtype=np.float64).reshape(self.nc, n) for x, n in ((W, 5), (K, 2), (dW, 5), (dK, 2))]
        dR, dRK = np.empty((self.nc, 5)), np.empty((self.nc, 2))
        err = ctypes.create_string_buffer(512)
        rc = lib().orc_rans_residual_cstep(self.h, *[_d(x) for x in a], h, _d(dR), _d(dRK), err, 512)
        if rc != 0:
            raise RuntimeError("oracle: " + err.value.decode())
        return dR, dRK

    def rans_bcs(self):
        nbc = int(self.case_summary()[1][5])
        out = np.empty((nbc, 5))
        lib().orc_rans_bcs(self.h, _d(out))
        return out

    def local_dt(self, W, cfl, mode=0):
        W = np.ascontiguousarray(W, dtype=np.float64).reshape(self.nc, 5)
        dt = np.empty(self.nc)
        lib().orc_local_dt(self.h, _d(W), float(cfl), int(mode), _d(dt))
        return dt

    def time_terms(self, W, dt):
        """Diagonal blocks P(W_c) V_c / dt_c (nc, 5, 5) of NavierStokes::time_terms."""
        W = np.ascontiguousarray(W, dtype=np.float64).reshape(self.nc, 5)
        dt = np.ascontiguousarray(dt, dtype=np.float64).reshape(self.nc)
        out = np.empty((self.nc, 5, 5))
        lib().orc_time_terms(self.h, _d(W), _d(dt), _d(out))
        return out

    def case_summary(self):
        d = np.empty(13)
        i = np.zeros(7 + 4 * 64, np.int32)
        lib().orc_case_summary(self.h, _d(d), _i(i))
        nbc = int(i[5])
        return d, i[:7 + 4 * nbc]
