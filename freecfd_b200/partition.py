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

    def __call__(self, R):
        import torch
        # W may have been written on torch's stream (a state update)
        self.stream.wait_stream(torch.cuda.current_stream(self.W.device))
        with torch.cuda.stream(self.stream):
            self.ex.exchange()
            self.ns.partition_extrema(self.W, out=self.ext)
            combine_extrema(self.ext)
            self.ns.partition_residual(self.ext, R)
        return R
