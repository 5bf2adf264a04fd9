"""Host-side mirror of the reference's residual interface.

``Case`` stands for the parsed input deck (read_inputs + MATERIAL::set +
NavierStokes::set_bcs), ``Mesh`` for ``Grid`` after ``setup``/``set_bcs``/
``gradient_maps`` and ``NavierStokes`` for the solver object whose residual
(``assemble_linear_system`` right-hand side), gradients (``calc_cell_grads``),
limiters (``calc_limiter``) and local time step (``update_time_step``) run on
the B200 through libfcfd_b200.  Arrays are in the reference's cell / face
order; states are [n_cells][5] = (p, u, v, w, T).
"""
from __future__ import annotations

import ctypes
import os
import tempfile

import numpy as np

from ._lib import (FCFD_DEVICE_PTRS, FCFD_NO_SYNC, NewtonOpts, NewtonReport, RunOpts, RunReport, _RawMesh, _d, _i, _ptr,
                   check, lib, FcfdError)


class Case:
    """Parsed input deck (src/read_inputs.cc schema and defaults)."""

    def __init__(self, deck_path: str):
        h = ctypes.c_void_p()
        check(lib.fcfd_case_from_deck(os.fsencode(deck_path), ctypes.byref(h)))
        self.h = h
        self.path = deck_path

    @classmethod
    def from_case(cls, case, workdir: str | None = None):
        """Write a synthetic ``cases.Case`` deck to ``workdir`` and parse it."""
        tmp = None
        if workdir is None:
            tmp = tempfile.TemporaryDirectory()
            workdir = tmp.name
        obj = cls(case.write_deck(workdir))
        obj._tmp = tmp
        return obj

    def summary(self):
        d = np.empty(13)
        i = np.zeros(7 + 4 * 64, np.int32)
        check(lib.fcfd_case_summary(self.h, _d(d), _i(i), i.size))
        return d, i[:7 + 4 * int(i[5])]

    def __del__(self):
        if getattr(self, "h", None):
            lib.fcfd_case_destroy(self.h)
            self.h = None


class Mesh:
    """Reference-order connectivity, geometry and LSQ stencils (Grid)."""

    def __init__(self, raw, case: Case, tecplot: str = None):
        """From a CELL-type raw grid, or (``tecplot`` = path, raw None) from a
        Tecplot FEPolyhedron grid file (Grid::readTEC + create_faces2)."""
        h = ctypes.c_void_p()
        self.bc_names = []
        if tecplot is not None:
            names = ctypes.create_string_buffer(4096)
            check(lib.fcfd_mesh_from_tecplot(os.fsencode(str(tecplot)), case.h, ctypes.byref(h), names, 4096))
            self.bc_names = [s for s in names.value.decode().split("\n") if s]
        else:
            self._keep = [np.ascontiguousarray(raw.nodes, np.float64), np.ascontiguousarray(raw.conn_index, np.int32),
                          np.ascontiguousarray(raw.conn, np.int32)]
            bidx, bflat = raw.bc_csr()
            self._keep += [np.ascontiguousarray(bidx, np.int32), np.ascontiguousarray(bflat, np.int32)]
            nodes, cidx, conn, bidx, bflat = self._keep
            r = _RawMesh(nodes.shape[0], _d(nodes), raw.n_cells, _i(cidx), _i(conn), len(raw.bc_nodes), _i(bidx),
                         _i(bflat))
            check(lib.fcfd_mesh_create(ctypes.byref(r), case.h, ctypes.byref(h)))
        self.h = h
        s = (ctypes.c_int64 * 8)()
        check(lib.fcfd_mesh_sizes(self.h, s))
        (self.nc, self.nf, self.nghost, self.ntot, self.nnodes, self.n_grad_entries, self.n_cell_faces,
         self.n_nbrs) = [int(x) for x in s]

    def connectivity(self):
        nf, nc = self.nf, self.nc
        out = dict(face_parent=np.empty(nf, np.int32), face_neighbor=np.empty(nf, np.int32),
                   face_bc=np.empty(nf, np.int32), face_nodes=np.empty((nf, 4), np.int32),
                   cell_face_index=np.empty(nc + 1, np.int32), cell_faces=np.empty(self.n_cell_faces, np.int32),
                   nbr_index=np.empty(nc + 1, np.int32), nbrs=np.empty(self.n_nbrs, np.int32),
                   grad_index=np.empty(nc + 1, np.int32), grad_keys=np.empty(self.n_grad_entries, np.int32))
        check(lib.fcfd_mesh_connectivity(self.h, *[_i(out[k]) for k in (
            "face_parent", "face_neighbor", "face_bc", "face_nodes", "cell_face_index", "cell_faces", "nbr_index",
            "nbrs", "grad_index", "grad_keys")]))
        return out

    def geometry(self):
        nf, nt = self.nf, self.ntot
        out = dict(face_normal=np.empty((nf, 3)), face_area=np.empty(nf), face_centroid=np.empty((nf, 3)),
                   face_avg=np.empty((nf, 2)), cell_centroid=np.empty((nt, 3)), cell_volume=np.empty(nt),
                   cell_length=np.empty(nt), cell_wall_distance=np.empty(nt))
        ls = np.empty(1)
        check(lib.fcfd_mesh_geometry(self.h, _d(out["face_normal"]), _d(out["face_area"]), _d(out["face_centroid"]),
                                     _d(out["face_avg"]), _d(out["cell_centroid"]), _d(out["cell_volume"]),
                                     _d(out["cell_length"]), _d(out["cell_wall_distance"]), _d(ls)))
        out["length_scale"] = float(ls[0])
        return out

    def lsq_data(self):
        cof = np.empty((self.nc, 7)); selfw = np.empty((self.nc, 3))
        check(lib.fcfd_mesh_lsq(self.h, _d(cof), _d(selfw)))
        return cof, selfw

    def grad_weights(self):
        """Stored gradient-map weights [E][3] in stencil-key order (meshes
        with curvilinear cells)."""
        w = np.empty((self.n_grad_entries, 3))
        check(lib.fcfd_mesh_grad_weights(self.h, _d(w)))
        return w

    def rcm_order(self):
        """Reverse Cuthill-McKee order of the interior cells (perm[new] =
        old) over the face-neighbour graph; `cases.renumber_cells` lists a
        grid's elements in this order."""
        perm = np.empty(self.nc, np.int32)
        check(lib.fcfd_mesh_rcm(self.h, _i(perm)))
        return perm

    def __del__(self):
        if getattr(self, "h", None):
            lib.fcfd_mesh_destroy(self.h)
            self.h = None


class NavierStokes:
    """Device residual context (one CUDA stream, device buffers)."""

    def __init__(self, mesh: Mesh, case: Case, device: int = 0, exact_gradients: bool = False):
        self.mesh, self.case = mesh, case
        h = ctypes.c_void_p()
        check(lib.fcfd_ctx_create(mesh.h, case.h, int(device), ctypes.byref(h)))
        self.h = h
        if exact_gradients:
            check(lib.fcfd_ctx_set_exact_gradients(self.h, 1))

    def residual(self, W, out=None):
        """R(W) for W [nc][5] (numpy host array or CUDA torch tensor)."""
        nc = self.mesh.nc
        if out is None:
            out = np.empty((nc, 5)) if isinstance(W, np.ndarray) else W.new_empty((nc, 5))
        if isinstance(W, np.ndarray):
            W = np.ascontiguousarray(W, dtype=np.float64)
        pw, fw = _ptr(W)
        pr, fr = _ptr(out)
        if fw != fr:
            raise ValueError("W and R must both be host arrays or both be device tensors")
        check(lib.fcfd_residual(self.h, pw, pr, fw))
        return out

    def residual_mixed(self, W, shock_ratio: float = 2.0, out=None):
        """R(W) with the face pass in FP32 except faces whose cell-centre
        absolute pressures differ by more than the factor shock_ratio (FP64);
        ghosts, gradients, limiters and the gather in FP64.  Returns (R,
        number of FP64 faces)."""
        nc = self.mesh.nc
        if out is None:
            out = np.empty((nc, 5)) if isinstance(W, np.ndarray) else W.new_empty((nc, 5))
        if isinstance(W, np.ndarray):
            W = np.ascontiguousarray(W, dtype=np.float64)
        pw, fw = _ptr(W)
        pr, fr = _ptr(out)
        if fw != fr:
            raise ValueError("W and R must both be host arrays or both be device tensors")
        n64 = ctypes.c_int64(0)
        check(lib.fcfd_residual_mixed(self.h, pw, pr, float(shock_ratio), fw, ctypes.byref(n64)))
        return out, int(n64.value)

    def time_residual_mixed(self, reps: int = 20, flush_l2: bool = True, shock_ratio: float = 2.0):
        """Mean device ms of the mixed-precision chain on the state of the
        last residual call, and its number of FP64 faces."""
        out = np.zeros(2)
        check(lib.fcfd_time_residual_mixed(self.h, int(reps), int(bool(flush_l2)), float(shock_ratio), _d(out)))
        return float(out[0]), int(out[1])

    def set_gradient_kernel(self, kind: int):
        """0 automatic, 1 per cell, 2 shared-memory tiles of 128 cells."""
        check(lib.fcfd_ctx_set_gradient_kernel(self.h, int(kind)))

    def set_launch_overlap(self, on: bool):
        """Programmatic dependent launches for the residual chain's gradient
        and face kernels (default on); the results are the same bits."""
        check(lib.fcfd_ctx_set_launch_overlap(self.h, int(bool(on))))

    def gradient_info(self):
        """dict(kind=1 per cell | 2 tiles | 3 folded stencils, fold_entries,
        fused) of the gradient kernel the residual runs."""
        out = (ctypes.c_int64 * 3)()
        check(lib.fcfd_ctx_gradient_info(self.h, out))
        return dict(kind=int(out[0]), fold_entries=int(out[1]), fused=bool(out[2]))

    def set_partition(self, lo: int, hi: int):
        """Evaluate only the part of the residual that owned cells [lo, hi)
        need (lo = hi = 0: the whole mesh again)."""
        check(lib.fcfd_ctx_set_partition(self.h, int(lo), int(hi)))
        self.partition = (int(lo), int(hi)) if hi > lo else None

    def partition_extrema(self, W, out=None):
        """Phase 1 of the partitioned residual: load W [nc][5] (owned and halo
        rows current), update this part's ghosts; returns the 8 VK extrema of
        the owned cells (combine over ranks: max of even, min of odd slots).
        For a CUDA tensor W the extrema are a CUDA tensor (``out``, 8
        doubles, if given) filled on the context's stream without a host
        synchronisation."""
        if isinstance(W, np.ndarray):
            W = np.ascontiguousarray(W, dtype=np.float64)
            ext = np.empty(8)
        else:
            ext = out if out is not None else W.new_empty(8)
        pw, fw = _ptr(W)
        pe, fe = _ptr(ext)
        check(lib.fcfd_partition_extrema(self.h, pw, pe, fw))
        return ext

    def partition_residual(self, ext, out, sync: bool = True):
        """Phase 2: rows [lo, hi) of R (numpy [nc][5] or CUDA tensor) from the
        extrema combined over all ranks (a CUDA tensor with a CUDA R).
        sync=False (CUDA R): enqueue only; check() reports a BC error."""
        if isinstance(out, np.ndarray):
            ext = np.ascontiguousarray(np.asarray(ext, dtype=np.float64))
        elif isinstance(ext, np.ndarray):
            import torch
            ext = torch.as_tensor(ext, device=out.device)
        pe, _ = _ptr(ext)
        pr, fr = _ptr(out)
        if not sync and fr & FCFD_DEVICE_PTRS:
            fr |= FCFD_NO_SYNC
        check(lib.fcfd_partition_residual(self.h, pe, pr, fr))
        return out

    def check(self):
        """Wait for the context's stream; raise for a BC error flagged by
        work enqueued without synchronisation."""
        check(lib.fcfd_ctx_check(self.h))

    def stream_handle(self) -> int:
        """The cudaStream_t this context enqueues its work on (as an int)."""
        s = ctypes.c_void_p()
        check(lib.fcfd_ctx_stream(self.h, ctypes.byref(s)))
        return int(s.value or 0)

    def jvp(self, W, V, with_residual: bool = False, fp32: bool = False):
        """Directional derivative (dR/dW).V of the residual (forward tangent);
        fp32=True evaluates the tangent chain in single precision."""
        nc = self.mesh.nc
        host = isinstance(W, np.ndarray)
        if host:
            W = np.ascontiguousarray(W, dtype=np.float64)
            V = np.ascontiguousarray(V, dtype=np.float64)
            JV = np.empty((nc, 5))
            R = np.empty((nc, 5)) if with_residual else None
        else:
            JV = W.new_empty((nc, 5))
            R = W.new_empty((nc, 5)) if with_residual else None
        pw, fw = _ptr(W)
        pv, _ = _ptr(V)
        pj, _ = _ptr(JV)
        pr = _ptr(R)[0] if R is not None else None
        check(lib.fcfd_jvp(self.h, pw, pv, pr, pj, fw | (4 if fp32 else 0)))
        return (R, JV) if with_residual else JV

    def vjp(self, W, Rbar):
        """Adjoint (dR/dW)^T . Rbar of the residual (backward half of jvp)."""
        nc = self.mesh.nc
        host = isinstance(W, np.ndarray)
        if host:
            W = np.ascontiguousarray(W, dtype=np.float64)
            Rbar = np.ascontiguousarray(Rbar, dtype=np.float64)
            Wb = np.empty((nc, 5))
        else:
            Wb = W.new_empty((nc, 5))
        pw, fw = _ptr(W)
        pr, _ = _ptr(Rbar)
        pb, _ = _ptr(Wb)
        check(lib.fcfd_vjp(self.h, pw, pr, pb, fw))
        return Wb

    def rans_residual(self, W, K):
        """k-omega RANS residual: (R[nc][5] with eddy viscosity, RK[nc][2])."""
        nc = self.mesh.nc
        W = np.ascontiguousarray(W, dtype=np.float64)
        K = np.ascontiguousarray(K, dtype=np.float64)
        R = np.empty((nc, 5))
        RK = np.empty((nc, 2))
        check(lib.fcfd_rans_residual(self.h, _d(W), _d(K), _d(R), _d(RK), 0))
        return R, RK

    def rans_jvp(self, W, K, V, VK, with_residual: bool = False, fp32: bool = False):
        """Tangent of the coupled residual along (V, VK): (JV[nc][5], JVK[nc][2]),
        with (R, RK) first when with_residual; fp32 runs the tangent chain in
        single precision."""
        nc = self.mesh.nc
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (W, K, V, VK)]
        JV, JVK = np.empty((nc, 5)), np.empty((nc, 2))
        R = np.empty((nc, 5)) if with_residual else None
        RK = np.empty((nc, 2)) if with_residual else None
        check(lib.fcfd_rans_jvp(self.h, *[_d(a) for a in arrs], _d(R), _d(RK), _d(JV), _d(JVK), 4 if fp32 else 0))
        return (R, RK, JV, JVK) if with_residual else (JV, JVK)

    def rans_vjp(self, W, K, Rbar, RKbar):
        """Adjoint of the coupled residual (backward half of rans_jvp):
        (Wbar[nc][5], Kbar[nc][2]) = (d(R, RK)/d(W, K))^T (Rbar, RKbar)."""
        nc = self.mesh.nc
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (W, K, Rbar, RKbar)]
        Wb, Kb = np.empty((nc, 5)), np.empty((nc, 2))
        check(lib.fcfd_rans_vjp(self.h, *[_d(a) for a in arrs], _d(Wb), _d(Kb), 0))
        return Wb, Kb

    def time_rans(self, reps: int = 50, flush_l2: bool = True):
        """[total, NS part, k-omega part] ms per coupled residual (device events)."""
        out = np.zeros(3)
        check(lib.fcfd_time_rans(self.h, int(reps), int(bool(flush_l2)), _d(out), out.size))
        return out

    def rans_bcs(self):
        """Per BC region: kw_fixed, k, omega, mut_fixed, mu_t."""
        nbc = int(self.case.summary()[1][5]) if hasattr(self.case, "summary") else 16
        out = np.zeros((16, 5))
        check(lib.fcfd_rans_bcs(self.h, _d(out), out.size))
        return out[:nbc]

    def drag(self, W, regions, direction=(1.0, 0.0, 0.0), gradient=True):
        """Force on the BC regions `regions` (0-based indices) and, with
        gradient=True, d(force . direction)/dW.  Returns (force[3], grad)."""
        nc = self.mesh.nc
        mask = 0
        for b in regions:
            mask |= 1 << int(b)
        W = np.ascontiguousarray(W, dtype=np.float64)
        d = np.ascontiguousarray(direction, dtype=np.float64)
        F = np.empty(3)
        G = np.empty((nc, 5)) if gradient else None
        check(lib.fcfd_drag(self.h, _d(W), mask, _d(d), _d(F), _d(G) if G is not None else None, 0))
        return F, G

    def newton_solve(self, W, tol=1e-10, max_newton=200, krylov_dim=30, krylov_rtol=1e-2, cfl0=1.0,
                     cfl_growth=1.2, cfl_max=1e6, cfl_mode=1, ser_exponent=1.0, jvp=True, fp32_krylov=False,
                     max_seconds=0.0, raise_on_fail=True, precond_sweeps=0, krylov_cycles=1, exact_jvp=False,
                     fp32_jvp=False, stop_all_rows=False, fp32_frozen_limiter=False, gs_persistent=False, ilu0=False,
                     local_relax=False, startup_steps=0, startup_drop=1e-3):
        """Steady solve R(W) = 0 (pseudo-transient Newton-Krylov on the device).
        stop_all_rows: also wait for the momentum and energy residuals to drop
        by tol.  fp32_frozen_limiter: with fp32_jvp, hold the limiter fixed in
        the FP32 tangent (jvp_mode 4).  gs_persistent: run all Gauss-Seidel
        colour updates of a preconditioner application in one cooperative
        launch with grid barriers instead of one launch per colour update.
        ilu0: block ILU(0) preconditioner in the multicolour order instead
        of block Jacobi / Gauss-Seidel.  local_relax: limit each cell's
        update to a 20 % change of p and T on its own instead of scaling the
        whole update.  startup_steps > 0: first up to that many explicit
        local-time-step steps at cfl0 until the mass residual has dropped by
        startup_drop.  Returns (W_converged, report dict)."""
        W = np.array(W, dtype=np.float64, order="C", copy=True)
        o = NewtonOpts(int(max_newton), float(tol), int(krylov_dim), float(krylov_rtol), float(cfl0), float(cfl_growth),
                       float(cfl_max), int(cfl_mode), float(ser_exponent),
                       ((4 if fp32_frozen_limiter else 3) if fp32_jvp else (2 if exact_jvp else 1)) if jvp else 0,
                       int(bool(fp32_krylov)), float(max_seconds), int(precond_sweeps), int(krylov_cycles),
                       int(bool(stop_all_rows)), int(bool(gs_persistent)), int(bool(ilu0)), int(bool(local_relax)),
                       int(startup_steps), float(startup_drop))
        r = NewtonReport()
        rc = lib.fcfd_newton_solve(self.h, _d(W), ctypes.byref(o), ctypes.byref(r))
        rep = dict(status=r.status, newton_iterations=r.newton_iterations, krylov_iterations=r.krylov_iterations,
                   res0=r.res0, res_final=r.res_final, wall_seconds=r.wall_seconds, last_cfl=r.last_cfl,
                   history=np.array(r.history[:r.newton_iterations + 1]), rows_final=list(r.rows_final),
                   seconds_to_tol=r.seconds_to_tol, startup_steps=r.startup_steps,
                   seconds_history=np.array(r.seconds_history[:r.newton_iterations + 1]))
        if rc != 0 and raise_on_fail:
            raise FcfdError(rc, lib.fcfd_last_error().decode() + f" after {r.newton_iterations} steps")
        return W, rep

    def rans_newton_solve(self, W, K, tol=1e-10, max_newton=200, krylov_dim=30, krylov_rtol=1e-2, cfl0=1.0,
                          cfl_max=1e6, ser_exponent=1.0, fp32_jvp=False, max_seconds=0.0, stop_all_rows=False,
                          raise_on_fail=True, cfl_mode=1):
        """Coupled steady solve of the flow and k-omega residuals (turbulent
        decks): pseudo-transient Newton-Krylov on (p,u,v,w,T,k,omega), J.v by
        FP64 finite differences or (fp32_jvp) the FP32 coupled tangent chain.
        Returns (W, K, report dict)."""
        W = np.array(W, dtype=np.float64, order="C", copy=True)
        K = np.array(K, dtype=np.float64, order="C", copy=True)
        o = NewtonOpts(int(max_newton), float(tol), int(krylov_dim), float(krylov_rtol), float(cfl0), 1.2,
                       float(cfl_max), int(cfl_mode), float(ser_exponent), 3 if fp32_jvp else 0, 0, float(max_seconds), 0, 1,
                       int(bool(stop_all_rows)))
        r = NewtonReport()
        rc = lib.fcfd_rans_newton_solve(self.h, _d(W), _d(K), ctypes.byref(o), ctypes.byref(r))
        n = r.newton_iterations
        rep = dict(status=r.status, newton_iterations=n, krylov_iterations=r.krylov_iterations, res0=r.res0,
                   res_final=r.res_final, wall_seconds=r.wall_seconds, last_cfl=r.last_cfl,
                   history=np.array(r.history[:n + 1]), seconds_history=np.array(r.seconds_history[:n + 1]),
                   rows_final=list(r.rows_final), kw_final=list(r.kw_final), seconds_to_tol=r.seconds_to_tol)
        if rc != 0 and raise_on_fail:
            raise FcfdError(rc, lib.fcfd_last_error().decode() + f" after {n} steps")
        return W, K, rep

    def run(self, W, work_dir=".", restart_step=0, max_steps=0, jvp=False, fp32_krylov=False, precond_sweeps=0,
            echo=False, raise_on_fail=True, K=None):
        """The deck's time loop (the reference's main program): per step the
        CFL schedule, one implicit backward-Euler step, convergence.dat,
        loads and restart files under ``work_dir``.  ``restart_step`` > 0
        starts from the restart files of that step (W is then only the
        output buffer).  Turbulent decks need ``K`` (k and omega per cell,
        [nc][2]); each step is then one coupled solve on the flow and k-omega
        variables.  Returns (W_final, report dict), with the final K under
        ``"K"`` for turbulent decks."""
        W = np.array(W, dtype=np.float64, order="C", copy=True)
        Kc = None if K is None else np.array(K, dtype=np.float64, order="C", copy=True)
        o = RunOpts(os.fsencode(str(work_dir)), int(restart_step), int(max_steps), 1 if jvp else 0,
                    int(bool(fp32_krylov)), int(precond_sweeps), int(bool(echo)), None if Kc is None else _d(Kc))
        r = RunReport()
        rc = lib.fcfd_run(self.h, _d(W), ctypes.byref(o), ctypes.byref(r))
        rep = dict(status=r.status, steps=r.steps, krylov_iterations=r.krylov_iterations, time=r.time, res=r.res,
                   wall_seconds=r.wall_seconds)
        if Kc is not None:
            rep["K"] = Kc
        if rc != 0 and raise_on_fail:
            raise FcfdError(rc, lib.fcfd_last_error().decode() + f" after {r.steps} steps")
        return W, rep

    def stages(self):
        m = self.mesh
        out = dict(grads=np.empty((m.nc, 15)), limiter=np.empty((m.nc, 5)), ghost=np.empty((m.nghost, 5)),
                   mdot=np.empty(m.nf), weightL=np.empty(m.nf))
        check(lib.fcfd_last_stages(self.h, _d(out["grads"]), _d(out["limiter"]), _d(out["ghost"]), _d(out["mdot"]),
                                   _d(out["weightL"])))
        return out

    def local_dt(self, W, cfl: float, mode: int = 0):
        nc = self.mesh.nc
        W = np.ascontiguousarray(W, dtype=np.float64)
        dt = np.empty(nc)
        pw, fw = _ptr(W)
        check(lib.fcfd_local_dt(self.h, pw, float(cfl), int(mode), ctypes.c_void_p(dt.ctypes.data), fw))
        return dt

    def diag_blocks(self, W, dt):
        """Diagonal blocks V P/dt - J_cc (nc, 5, 5) of the implicit operator
        at state W and local time steps dt: the counterpart of the diagonal
        of NavierStokes::time_terms (ns_time_terms.cc:107-186) plus
        assemble_linear_system's first-order Jacobian."""
        nc = self.mesh.nc
        W = np.ascontiguousarray(W, dtype=np.float64).reshape(nc, 5)
        dt = np.ascontiguousarray(dt, dtype=np.float64).reshape(nc)
        out = np.empty((nc, 5, 5))
        check(lib.fcfd_diag_blocks(self.h, _d(W), _d(dt), _d(out)))
        return out

    def time_terms(self, W, dt):
        """Time-term blocks V P/dt (nc, 5, 5) at state W and local time
        steps dt (NavierStokes::time_terms, ns_time_terms.cc:107-186)."""
        nc = self.mesh.nc
        W = np.ascontiguousarray(W, dtype=np.float64).reshape(nc, 5)
        dt = np.ascontiguousarray(dt, dtype=np.float64).reshape(nc)
        out = np.empty((nc, 5, 5))
        check(lib.fcfd_time_terms(self.h, _d(W), _d(dt), _d(out)))
        return out

    def time_residual(self, reps: int = 50, flush_l2: bool = True):
        out = np.zeros(8)
        check(lib.fcfd_time_residual(self.h, int(reps), int(bool(flush_l2)), _d(out), out.size))
        return out

    def __del__(self):
        if getattr(self, "h", None):
            lib.fcfd_ctx_destroy(self.h)
            self.h = None


def write_restart(work_dir, step: int, W, time: float, first_res, n_nodes: int, dt=None, K=None, mu_t=None,
                  rans_first_res=None, gid: int = 1):
    """Restart files in the reference's layout (write_restart.cc) under
    ``work_dir``/restart: partition map, <step>/time.dat, raw doubles per
    cell.  W[nc][5] = (p,u,v,w,T), K[nc][2] = (k, omega)."""
    W = np.ascontiguousarray(W, dtype=np.float64)
    nc = W.shape[0]
    first = np.ascontiguousarray(first_res, dtype=np.float64)
    rf = None if rans_first_res is None else np.ascontiguousarray(rans_first_res, dtype=np.float64)
    arr = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (dt, K, mu_t)]
    check(lib.fcfd_restart_write(os.fsencode(str(work_dir)), int(gid), int(step), float(time), _d(first), _d(rf),
                                 int(nc), int(n_nodes), _d(W), _d(arr[0]), _d(arr[1]), _d(arr[2])))


def read_restart(work_dir, step: int, n_cells: int, turbulent: bool = False, gid: int = 1):
    """Reads the files of write_restart (or of the reference's write_restart).
    Returns dict(time, first_res, rans_first_res, W[, K, mu_t])."""
    t = np.zeros(1)
    first = np.zeros(3)
    rf = np.zeros(2)
    W = np.zeros((n_cells, 5))
    K = np.zeros((n_cells, 2)) if turbulent else None
    mu_t = np.zeros(n_cells) if turbulent else None
    check(lib.fcfd_restart_read(os.fsencode(str(work_dir)), int(gid), int(step), int(n_cells), _d(t), _d(first), _d(rf),
                                _d(W), _d(K), _d(mu_t)))
    out = dict(time=float(t[0]), first_res=first, rans_first_res=rf, W=W)
    if turbulent:
        out.update(K=K, mu_t=mu_t)
    return out


def point_flux(flux: int, L, R, n, gamma=1.4, gas_R=287.0, Pref=0.0, Tref=0.0, Minf=1.0):
    """Convective flux per unit area through a face with unit normal n."""
    L = np.ascontiguousarray(L, np.float64); R = np.ascontiguousarray(R, np.float64)
    n = np.ascontiguousarray(n, np.float64)
    out = np.empty(5); wl = np.empty(1)
    check(lib.fcfd_point_flux(int(flux), _d(L), _d(R), _d(n), gamma, gas_R, Pref, Tref, Minf, _d(out), _d(wl)))
    return out, float(wl[0])
