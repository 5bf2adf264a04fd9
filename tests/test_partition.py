"""Domain decomposition, host side (no GPU): the partition sets are closed
under what the owned rows of R read, and the halo exchange delivers every
halo state from its owner (two gloo ranks on the CPU).

What the residual of an owned cell reads (the reference's face loop,
ns_assemble_linear_system.cc:75-140, and the stages before it): the fluxes of
its faces; for each, the reconstructed states of both sides (gradient and
limiter of the face's cells, ns.cc:301-336 and ns_limiters.cc) and, at
outlet faces, the state cache left by the previous faces; each gradient reads
the cell's LSQ stencil (lsqr_grad_map.cc:32-99) and each limiter the cell's
face neighbours; the VK extrema read T of cell 0 and w of the last cell
(find_min_max's indices, ns.cc:400-435)."""
import socket

import numpy as np
import pytest

from tests.util import ALL, SMALL


def _mesh(fb, family, **kw):
    import tempfile
    case = ALL[family](**kw)
    d = tempfile.mkdtemp(prefix="fcfd_part_")
    cs = fb.Case(case.write_deck(d))
    return case, cs, fb.Mesh(case.mesh, cs)


def _tecplot_mesh(fb, family):
    import os
    import tempfile

    from freecfd_b200 import cases
    case = ALL[family]()
    d = tempfile.mkdtemp(prefix="fcfd_partt_")
    path = cases.write_tecplot(case.mesh, os.path.join(d, "grid.dat"), order="shuffled", seed=7)
    cs = fb.Case(case.write_deck(d))
    return case, cs, fb.Mesh(None, cs, tecplot=path)


@pytest.mark.parametrize("family", sorted(ALL) + ["tecplot_wedge", "tecplot_hypersonic"])
@pytest.mark.parametrize("nparts", [2, 3])
def test_partition_sets_are_closed(family, nparts, fb):
    from freecfd_b200.partition import block_ranges, partition_sets
    if family.startswith("tecplot_"):
        case, cs, m = _tecplot_mesh(fb, family[len("tecplot_"):])  # faces in shuffled order
    else:
        case, cs, m = _mesh(fb, family)
    con = m.connectivity()
    nc, parent, nbr, fbc = m.nc, con["face_parent"], con["face_neighbor"], con["face_bc"]
    cfi, cfl = con["cell_face_index"], con["cell_faces"]
    gi, gk = con["grad_index"], con["grad_keys"]
    ghost_face = np.full(m.nghost, -1)
    bmask = fbc >= 0
    ghost_face[nbr[bmask] - nc] = np.nonzero(bmask)[0]
    covered = np.zeros(nc, bool)
    for lo, hi in block_ranges(nc, nparts):
        s = partition_sets(m, cs, lo, hi)
        covered[lo:hi] = True
        faces, grad, halo = set(s["faces"].tolist()), set(s["grad_cells"].tolist()), s["halo"]
        current = np.zeros(nc, bool)
        current[lo:hi] = True
        assert not current[halo].any()
        current[halo] = True
        assert current[0] and current[nc - 1]
        assert s["grad_cells"].tolist() == sorted(grad) and halo.tolist() == sorted(halo.tolist())
        for c in range(lo, hi):
            assert set(cfl[cfi[c]:cfi[c + 1]].tolist()) <= faces
        for f in faces:
            if fbc[f] < 0:
                assert parent[f] in grad and nbr[f] in grad
            else:
                assert parent[f] in grad
        for c in grad:
            for k in gk[gi[c]:gi[c + 1]]:
                assert current[k] if k < nc else current[parent[ghost_face[k - nc]]], (c, k)
            for f in cfl[cfi[c]:cfi[c + 1]]:
                if fbc[f] < 0:
                    assert current[nbr[f] if parent[f] == c else parent[f]]
    assert covered.all()


def test_partition_outlet_walk_cells(fb):
    """Outlet faces of owned cells read the right density of the previous
    faces in face order: the walk's cells are gradient cells of the part."""
    from freecfd_b200.partition import block_ranges, partition_sets
    case, cs, m = _mesh(fb, "cylinder")
    con = m.connectivity()
    fbc, parent, nbr = con["face_bc"], con["face_parent"], con["face_neighbor"]
    import re
    outlet_bc = {int(b) - 1 for b, t in re.findall(r"BC_(\d+)\s*\(\s*type=(\w+)", case.deck) if t == "outlet"}
    assert outlet_bc
    checked = 0
    for lo, hi in block_ranges(m.nc, 3):
        s = partition_sets(m, cs, lo, hi)
        grad = set(s["grad_cells"].tolist())
        for f in s["faces"]:
            if fbc[f] < 0 or fbc[f] not in outlet_bc:
                continue
            # the walk back to the first interior face is covered
            g = f - 1
            while g >= 0 and fbc[g] >= 0:
                assert parent[g] in grad
                g -= 1
            if g >= 0:
                assert nbr[g] in grad
            checked += 1
    assert checked > 0


def test_partition_range_errors(fb):
    from freecfd_b200.partition import block_ranges, partition_sets
    case, cs, m = _mesh(fb, "wedge")
    with pytest.raises(fb.FcfdError):
        partition_sets(m, cs, 5, 5)
    with pytest.raises(fb.FcfdError):
        partition_sets(m, cs, 0, m.nc + 1)
    with pytest.raises(ValueError):
        block_ranges(4, 5)
    assert block_ranges(10, 3) == [(0, 3), (3, 6), (6, 10)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _exchange_rank(rank, world, port, family, out_q):
    import tempfile

    import torch
    import torch.distributed as dist

    import freecfd_b200 as fb
    from freecfd_b200.partition import HaloExchange, HaloPlan, combine_extrema
    try:
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
        case = SMALL[family]()
        d = tempfile.mkdtemp(prefix=f"fcfd_gloo{rank}_")
        cs = fb.Case(case.write_deck(d))
        m = fb.Mesh(case.mesh, cs)
        plan = HaloPlan(m, cs, world)
        Wg = torch.as_tensor(case.state.copy())
        lo, hi = plan.ranges[rank]
        W = torch.full_like(Wg, -7.0)
        W[lo:hi] = Wg[lo:hi]
        ex = HaloExchange(plan, rank, W)
        ex.exchange()
        halo = torch.as_tensor(plan.halo_cells(rank))
        ok = bool(torch.equal(W[halo], Wg[halo])) and bool(torch.equal(W[lo:hi], Wg[lo:hi]))
        untouched = np.setdiff1d(np.arange(m.nc), np.concatenate([np.arange(lo, hi), plan.halo_cells(rank)]))
        ok = ok and bool((W[torch.as_tensor(untouched)] == -7.0).all()) if len(untouched) else ok
        # extrema combine: max of even slots, min of odd ones
        own = case.state[lo:hi]
        ext = np.array([own[:, 0].max(), own[:, 0].min(), own[:, 1].max(), own[:, 1].min(),
                        own[:, 2].max(), own[:, 2].min(), own[:, 4].max(), own[:, 4].min()])
        got = combine_extrema(ext)
        s = case.state
        ref = np.array([s[:, 0].max(), s[:, 0].min(), s[:, 1].max(), s[:, 1].min(), s[:, 2].max(), s[:, 2].min(),
                        s[:, 4].max(), s[:, 4].min()])
        ok = ok and np.array_equal(got, ref)
        out_q.put((rank, ok, ex.bytes_per_exchange))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent, which fails the test
        out_q.put((rank, repr(e), 0))


@pytest.mark.parametrize("family", ["cylinder", "hypersonic"])
def test_halo_exchange_gloo_two_ranks(family):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_exchange_rank, args=(r, 2, port, family, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    for rank, ok, nbytes in res:
        assert ok is True, (rank, ok)
        assert nbytes > 0


def _block_operator(m, seed=5):
    """A sparse block operator on the mesh's face graph: y_c = B_c x_c +
    sum over interior faces of C_f x_other, seeded 5x5 blocks with a
    dominant diagonal (the structure of the first-order implicit operator)."""
    conn = m.connectivity()
    fp, fn, fb_ = conn["face_parent"], conn["face_neighbor"], conn["face_bc"]
    it = np.nonzero(fb_ < 0)[0]
    rng = np.random.default_rng(seed)
    B = rng.standard_normal((m.nc, 5, 5)) * 0.3 + 12.0 * np.eye(5)
    CP = rng.standard_normal((len(it), 5, 5))  # parent row, neighbour column
    CN = rng.standard_normal((len(it), 5, 5))  # neighbour row, parent column
    return B, fp[it].astype(np.int64), fn[it].astype(np.int64), CP, CN


def _apply_rows(op, x, lo, hi):
    """Rows [lo, hi) of the operator applied to the full vector x (torch)."""
    import torch
    B, P, N, CP, CN = op
    y = torch.einsum("cij,cj->ci", torch.as_tensor(B[lo:hi]), x[lo:hi])
    sel = (P >= lo) & (P < hi)
    y.index_add_(0, torch.as_tensor(P[sel] - lo), torch.einsum("fij,fj->fi", torch.as_tensor(CP[sel]), x[torch.as_tensor(N[sel])]))
    sel = (N >= lo) & (N < hi)
    y.index_add_(0, torch.as_tensor(N[sel] - lo), torch.einsum("fij,fj->fi", torch.as_tensor(CN[sel]), x[torch.as_tensor(P[sel])]))
    return y


def _gmres_rank(rank, world, port, out_q):
    import tempfile

    import torch
    import torch.distributed as dist

    import freecfd_b200 as fb
    from freecfd_b200.partition import HaloExchange, HaloPlan, gmres
    try:
        if world > 1:
            dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
        case = SMALL["cylinder"]()
        cs = fb.Case(case.write_deck(tempfile.mkdtemp(prefix=f"fcfd_gm{rank}_")))
        m = fb.Mesh(case.mesh, cs)
        plan = HaloPlan(m, cs, world)
        lo, hi = plan.ranges[rank]
        op = _block_operator(m)
        xfull = torch.zeros((m.nc, 5), dtype=torch.float64)
        ex = HaloExchange(plan, rank, xfull) if world > 1 else None
        Binv = torch.linalg.inv(torch.as_tensor(op[0][lo:hi]))
        rng = np.random.default_rng(9)
        b = torch.as_tensor(rng.standard_normal((m.nc, 5))[lo:hi])

        def matvec(z):
            xfull[lo:hi] = z
            if ex is not None:
                ex.exchange()
            return _apply_rows(op, xfull, lo, hi)

        def precond(v):
            return torch.einsum("cij,cj->ci", Binv, v)

        ar = (lambda t: dist.all_reduce(t)) if world > 1 else None
        x, its, rel = gmres(matvec, precond, b, allreduce=ar, m=20, rtol=1e-10, cycles=3)
        out_q.put((rank, (lo, hi), x.numpy(), its, rel))
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
    except Exception as e:  # reported to the parent, which fails the test
        out_q.put((rank, repr(e), None, 0, 0.0))


def test_distributed_gmres_gloo_two_ranks():
    """GMRES over a two-rank decomposition (halo exchange of the Krylov
    direction inside the matvec, every dot product all-reduced over gloo)
    takes the same iterations as the single-domain solve and returns the
    same solution to rounding; the solution solves the system."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gmres_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=240) for _ in procs], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
    for rank, rng_, x, its, rel in res:
        assert x is not None, (rank, rng_)
    q1 = ctx.Queue()
    p1 = ctx.Process(target=_gmres_rank, args=(0, 1, 0, q1))
    p1.start()
    _, _, x1, its1, rel1 = q1.get(timeout=240)
    p1.join(timeout=60)
    assert x1 is not None
    xd = np.concatenate([x for _, _, x, _, _ in res])
    assert all(its == its1 for _, _, _, its, _ in res), ([r[3] for r in res], its1)
    assert np.abs(xd - x1).max() <= 1e-11 * np.abs(x1).max()
    assert rel1 <= 1e-10
