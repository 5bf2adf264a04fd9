"""Domain-decomposed residual: one rank per GPU, halo states exchanged with
torch.distributed point-to-point (NCCL over NVLink on GPUs, gloo on CPU).

The reference runs one MPI rank per partition (ParMETIS, grid_partition.cc),
exchanges the primitives and gradients of its partition ghosts before every
residual (NavierStokes::mpi_update_ghost_primitives / _gradients,
navier_stokes/ns_mpi.cc:62-140, called from ns.cc:92-115) and all-reduces the
limiter extrema (find_min_max, ns.cc:425-427).  Here rank r owns the
contiguous global cell range ``ranges[r]``; the library
(``fcfd_partition_sets``) names the halo: every not-owned cell whose state
the owned rows of R depend on, so the state is exchanged once per residual and
gradients are recomputed on the halo instead of being exchanged.  The owned
rows equal the single-domain residual bit for bit.
"""
import numpy as np

from ._lib import _i, check, lib


def block_ranges(nc: int, nparts: int):
    """Contiguous cell ranges [lo, hi), sizes differing by at most one."""
    if not 1 <= nparts <= nc:
        raise ValueError("need 1 <= nparts <= cells")
    cuts = [(nc * r) // nparts for r in range(nparts + 1)]
    return [(cuts[r], cuts[r + 1]) for r in range(nparts)]


def partition_sets(mesh, case, lo: int, hi: int):
    """Host-side sets of the part owning [lo, hi): cells whose gradient is
    formed, faces whose flux is formed, halo cells (ascending global ids) and
    the number of ghosts updated."""
    counts = np.zeros(4, np.int32)
    check(lib.fcfd_partition_sets(mesh.h, case.h, int(lo), int(hi), _i(counts), None, None, None))
    grad, faces, halo = (np.empty(int(n), np.int32) for n in counts[:3])
    check(lib.fcfd_partition_sets(mesh.h, case.h, int(lo), int(hi), _i(counts), _i(grad), _i(faces), _i(halo)))
    return dict(grad_cells=grad, faces=faces, halo=halo, n_ghosts=int(counts[3]))


class HaloPlan:
    """Exchange lists of a contiguous-range partition: ``recv[r][q]`` = the
    halo cells of rank r owned by rank q; rank q sends exactly those."""

    def __init__(self, mesh, case, nparts: int):
        self.nc = mesh.nc
        self.ranges = block_ranges(mesh.nc, nparts)
        starts = np.array([lo for lo, _ in self.ranges])
        self.halo, self.recv = [], []
        for lo, hi in self.ranges:
            h = partition_sets(mesh, case, lo, hi)["halo"].astype(np.int64)
            self.halo.append(h)
            own = np.searchsorted(starts, h, side="right") - 1
            self.recv.append({int(q): h[own == q] for q in np.unique(own)})

    def send(self, q: int):
        """Cells rank q sends, per destination rank."""
        return {r: rv[q] for r, rv in enumerate(self.recv) if q in rv}

    def halo_cells(self, r: int):
        return self.halo[r]


class HaloExchange:
    """Halo update of one rank's state array W ([nc][5], float64, on the
    rank's device or the CPU): pack the owned rows the peers need, post all
    sends and receives at once, unpack into the halo rows."""

    def __init__(self, plan: HaloPlan, rank: int, W):
        import torch
        self.W, self.rank = W, rank
        dev = W.device
        self.sends = [(q, torch.as_tensor(idx, device=dev), torch.empty((len(idx), 5), dtype=W.dtype, device=dev))
                      for q, idx in sorted(plan.send(rank).items())]
        self.recvs = [(q, torch.as_tensor(idx, device=dev), torch.empty((len(idx), 5), dtype=W.dtype, device=dev))
                      for q, idx in sorted(plan.recv[rank].items())]
        self.bytes_per_exchange = 8 * 5 * sum(len(i) for _, i, _ in self.recvs)

    def exchange(self):
        import torch
        import torch.distributed as dist
        for _, idx, buf in self.sends:
            torch.index_select(self.W, 0, idx, out=buf)
        ops = [dist.P2POp(dist.isend, buf, q) for q, _, buf in self.sends]
        ops += [dist.P2POp(dist.irecv, buf, q) for q, _, buf in self.recvs]
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for _, idx, buf in self.recvs:
            self.W.index_copy_(0, idx, buf)


def combine_extrema(ext, device=None):
    """The VK extrema over all ranks: max of the even slots, min of the odd
    ones (one all-reduce, odd slots negated).  A torch tensor is combined in
    place on the current stream; host values come back as numpy."""
    import torch
    import torch.distributed as dist
    inplace = isinstance(ext, torch.Tensor)
    if not (dist.is_available() and dist.is_initialized()):
        return ext if inplace else np.asarray(ext, dtype=np.float64)
    t = ext if inplace else torch.as_tensor(np.asarray(ext, dtype=np.float64).copy(), device=device)
    t[1::2] = -t[1::2]
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    t[1::2] = -t[1::2]
    return t if inplace else t.cpu().numpy()


class PartitionedResidual:
    """R(W) of one rank: halo exchange, owned extrema, all-reduce, owned rows.

    ``W`` and ``R`` are [nc][5] float64 CUDA tensors on the rank's device;
    only the owned rows of R are written and only owned + halo rows of W are
    read.  Everything is enqueued on the library context's stream (the
    exchange's packing, the NCCL point-to-point and all-reduce, the two
    library phases), so a step has one host synchronisation: the error check
    at the end of phase 2."""

    def __init__(self, ns, plan: HaloPlan, rank: int, W):
        import torch
        self.ns, self.plan, self.rank = ns, plan, rank
        self.lo, self.hi = plan.ranges[rank]
        ns.set_partition(self.lo, self.hi)
        self.ex = HaloExchange(plan, rank, W)
        self.W = W
        self.ext = W.new_empty(8)
        self.stream = torch.cuda.ExternalStream(ns.stream_handle(), device=W.device)

    def __call__(self, R, sync: bool = True):
        """sync=False: enqueue the step only (no host synchronisation); a BC
        error is then reported by check()."""
        import torch
        # W may have been written on torch's stream (a state update)
        self.stream.wait_stream(torch.cuda.current_stream(self.W.device))
        with torch.cuda.stream(self.stream):
            self.ex.exchange()
            self.ns.partition_extrema(self.W, out=self.ext)
            combine_extrema(self.ext)
            self.ns.partition_residual(self.ext, R, sync=sync)
        return R

    def check(self):
        self.ns.check()


def gmres(matvec, precond, b, allreduce=None, m: int = 30, rtol: float = 1e-2, cycles: int = 1):
    """Right-preconditioned GMRES(m) on distributed vectors: each rank holds
    its owned rows (torch tensors, FP64); `matvec` and `precond` act on them
    (exchanging halos themselves); every dot product is a local sum followed
    by one all-reduce (SUM) of the column of dots, so all ranks take the
    same steps.  Classical Gram-Schmidt applied twice, Givens rotations on
    the host.  Returns (x, iterations, relative residual).  The distributed
    counterpart of the device GMRES of fcfd_newton_solve."""
    import torch

    def dots(vs, w):
        loc = torch.stack([(v * w).sum() for v in vs])
        if allreduce is not None:
            allreduce(loc)
        return loc.cpu().numpy()

    x = torch.zeros_like(b)
    bnorm = float(np.sqrt(dots([b], b)[0]))
    if not bnorm > 0.0:
        return x, 0, 0.0
    r = b.clone()
    its, rel = 0, 1.0
    for cyc in range(max(1, cycles)):
        beta = float(np.sqrt(dots([r], r)[0]))
        if not beta > 0.0:
            break
        V, Z = [r / beta], []
        H = np.zeros((m + 1, m))
        cs, sn, g = np.zeros(m), np.zeros(m), np.zeros(m + 1)
        g[0] = beta
        k = 0
        for j in range(m):
            z = precond(V[j])
            Z.append(z)
            w = matvec(z)
            h1 = dots(V, w)
            w = w - sum(float(h1[i]) * V[i] for i in range(j + 1))
            h2 = dots(V, w)
            w = w - sum(float(h2[i]) * V[i] for i in range(j + 1))
            hn = float(np.sqrt(dots([w], w)[0]))
            H[: j + 1, j] = h1 + h2
            H[j + 1, j] = hn
            for i in range(j):
                a, c = H[i, j], H[i + 1, j]
                H[i, j], H[i + 1, j] = cs[i] * a + sn[i] * c, -sn[i] * a + cs[i] * c
            a, c = H[j, j], H[j + 1, j]
            rr = float(np.hypot(a, c))
            cs[j], sn[j] = (a / rr, c / rr) if rr > 0.0 else (1.0, 0.0)
            H[j, j], H[j + 1, j] = rr, 0.0
            g[j + 1] = -sn[j] * g[j]
            g[j] = cs[j] * g[j]
            k = j + 1
            its += 1
            rel = abs(g[j + 1]) / bnorm
            if rel <= rtol or not hn > 0.0:
                break
            V.append(w / hn)
        y = np.zeros(k)
        for i in range(k - 1, -1, -1):
            y[i] = (g[i] - H[i, i + 1:k] @ y[i + 1:k]) / H[i, i]
        x = x + sum(float(y[i]) * Z[i] for i in range(k))
        if rel <= rtol or cyc + 1 == max(1, cycles):
            break
        r = b - matvec(x)
    return x, its, rel


class DecomposedNewton:
    """Pseudo-transient Newton-Krylov on one rank of a domain decomposition
    (the implicit step of NavierStokes::solve, ns.cc:104-118, run as the
    reference's MPI ranks would: every rank owns a cell range, exchanges its
    halo before each residual and takes part in every reduction).

    Per Newton step: the owned rows of R(W) (PartitionedResidual), the local
    time step and the owned cells' diagonal blocks V P/dt - J_cc and time
    terms V P/dt (fcfd_local_dt, fcfd_diag_blocks, fcfd_time_terms on this
    rank's state copy, whose owned and halo rows are current), then GMRES on
    (V P/dt - dR/dW) dW = R with J.v an FP64 finite difference of the
    partitioned residual (the perturbed state's halo exchanged like the
    state's), block-Jacobi preconditioning, equations weighted by their RMS
    row magnitudes and every dot product all-reduced (`gmres`).  The step is
    limited to a 20 % change of p and T (all-reduced maximum) and the CFL
    follows the mass residual (switched evolution / relaxation).  The block
    inverses of a rank use the VK extrema of its own state copy (its
    preconditioner only; the residual's extrema are all-reduced)."""

    def __init__(self, ns, mesh, case, plan: HaloPlan, rank: int, W):
        import torch
        self.ns, self.mesh, self.plan, self.rank = ns, mesh, plan, rank
        self.lo, self.hi = plan.ranges[rank]
        self.W = W
        self.Wp = W.clone()
        self.res = PartitionedResidual(ns, plan, rank, self.W)
        self.res_p = PartitionedResidual(ns, plan, rank, self.Wp)
        self.R = torch.zeros_like(W)
        self.Rp = torch.zeros_like(W)
        dv = np.zeros(13)
        iv = np.zeros(64, np.int32)
        from ._lib import _d
        check(lib.fcfd_case_summary(case.h, _d(dv), _i(iv), int(iv.size)))
        self.Pref, self.Tref = float(dv[2]), float(dv[3])

    def _allreduce(self, t, op=None):
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            dist.all_reduce(t, op=op or dist.ReduceOp.SUM)
        return t

    def _gnorm(self, x):
        import torch
        t = (x * x).sum().reshape(1).clone()
        self._allreduce(t)
        return float(torch.sqrt(t).item())

    def residual(self):
        self.res(self.R)
        import torch
        torch.cuda.synchronize(self.W.device)
        return self.R[self.lo:self.hi]

    def solve(self, tol=1e-10, max_newton=200, cfl0=1.0, cfl_max=1e6, ser_exponent=1.0, krylov_dim=30,
              krylov_rtol=1e-2, krylov_cycles=1):
        import torch
        import torch.distributed as dist
        lo, hi = self.lo, self.hi
        W, dev = self.W, self.W.device
        R0 = self.residual().clone()
        r0 = self._gnorm(R0[:, 0])
        rm, cfl = r0, cfl0
        history = [1.0]
        krylov = 0
        eps_mach = float(np.finfo(np.float64).eps)
        for it in range(max_newton):
            if rm <= tol * r0:
                break
            Wh = W.cpu().numpy()
            dt = self.ns.local_dt(Wh, cfl)
            D = torch.as_tensor(self.ns.diag_blocks(Wh, dt)[lo:hi], device=dev)
            T = torch.as_tensor(self.ns.time_terms(Wh, dt)[lo:hi], device=dev)
            Minv = torch.linalg.inv(D)
            # reference magnitudes of p, |V|, T and the RMS row magnitudes of D
            Wo = W[lo:hi]
            n_all = torch.tensor([float(hi - lo)], dtype=torch.float64, device=dev)
            self._allreduce(n_all)
            sq = (Wo * Wo).sum(dim=0)
            self._allreduce(sq)
            rms = torch.sqrt(sq / n_all)
            U = float(torch.sqrt(rms[1:4].pow(2).sum()).item()) or 1.0
            wref = torch.tensor([float(rms[0]) + abs(self.Pref), U, U, U, float(rms[4]) + abs(self.Tref)],
                                dtype=torch.float64, device=dev)
            rowmag = (D.abs() * wref.view(1, 1, 5)).sum(dim=2)
            rsq = (rowmag * rowmag).sum(dim=0)
            self._allreduce(rsq)
            wrow = 1.0 / torch.sqrt(rsq / n_all)
            Winv = 1.0 / wref
            wscale = self._gnorm(Wo * Winv)

            def matvec(z):
                zn = self._gnorm(z * Winv)
                eps = np.sqrt(eps_mach) * (1.0 + wscale) / zn if zn > 0.0 else np.sqrt(eps_mach)
                self.Wp.copy_(W)
                self.Wp[lo:hi] += eps * z
                self.res_p(self.Rp)
                Jz = (self.Rp[lo:hi] - R0) / eps
                y = torch.einsum("cij,cj->ci", T, z) - Jz
                return y * wrow

            def precond(v):
                return torch.einsum("cij,cj->ci", Minv, v / wrow)

            dW, its, rel = gmres(matvec, precond, R0 * wrow, allreduce=lambda t: self._allreduce(t), m=krylov_dim,
                                 rtol=krylov_rtol, cycles=krylov_cycles)
            krylov += its
            ch = torch.maximum((dW[:, 0] / (Wo[:, 0] + self.Pref)).abs().max(),
                               (dW[:, 4] / (Wo[:, 4] + self.Tref)).abs().max()).reshape(1).clone()
            self._allreduce(ch, dist.ReduceOp.MAX if dist.is_available() and dist.is_initialized() else None)
            dmax = float(ch.item())
            alpha = 0.2 / dmax if dmax > 0.2 else 1.0
            W[lo:hi] += alpha * dW
            R0 = self.residual().clone()
            rm = self._gnorm(R0[:, 0])
            history.append(rm / r0)
            if not np.isfinite(rm):
                break
            cfl = min(max(cfl0 * (r0 / rm) ** ser_exponent, 1e-3), cfl_max)
        return dict(newton_iterations=len(history) - 1, krylov_iterations=krylov, res0=r0, res_final=rm,
                    history=np.array(history), converged=bool(rm <= tol * r0))
