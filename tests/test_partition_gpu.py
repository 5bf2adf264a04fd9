"""Domain-decomposed residual on the device: every part of a 2- and 3-way
split evaluated in its own context, with the states of all cells outside the
part's owned range and halo replaced by a different (valid) state, the VK
extrema combined over the parts as the ranks' all-reduce does; the owned
rows equal the single-domain residual bit for bit (the reference's MPI runs
exchange partition ghosts, ns_mpi.cc:62-140, and all-reduce the extrema,
ns.cc:425-427, so each rank's residual rows are the global ones)."""
import numpy as np
import pytest

from freecfd_b200.partition import HaloPlan
from tests.util import ALL, SMALL


def _setup(fb, case):
    import tempfile
    d = tempfile.mkdtemp(prefix="fcfd_partg_")
    cs = fb.Case(case.write_deck(d))
    return cs, fb.Mesh(case.mesh, cs)


def _partitioned(fb, case, cs, m, nparts, exact=False, device=False):
    plan = HaloPlan(m, cs, nparts)
    state = case.state
    rng = np.random.default_rng(11)
    other = state * (1 + 0.05 * rng.uniform(-1, 1, state.shape))
    parts = []
    for r, (lo, hi) in enumerate(plan.ranges):
        ns = fb.NavierStokes(m, cs, 0, exact_gradients=exact)
        ns.set_partition(lo, hi)
        W = other.copy()
        W[lo:hi] = state[lo:hi]
        h = plan.halo_cells(r)
        W[h] = state[h]
        if device:
            import torch
            W = torch.as_tensor(W, device="cuda")
        parts.append((ns, W, lo, hi))
    if device:
        import torch
        e = torch.stack([ns.partition_extrema(W) for ns, W, _, _ in parts])
        torch.cuda.synchronize()
        ext = torch.where(torch.arange(8, device="cuda") % 2 == 0, e.max(dim=0).values, e.min(dim=0).values)
    else:
        exts = np.array([ns.partition_extrema(W) for ns, W, _, _ in parts])
        ext = np.where(np.arange(8) % 2 == 0, exts.max(axis=0), exts.min(axis=0))
    R = np.full((m.nc, 5), np.nan)
    for ns, W, lo, hi in parts:
        if device:
            import torch
            out = torch.full((m.nc, 5), float("nan"), dtype=torch.float64, device="cuda")
            ns.partition_residual(ext, out)
            out = out.cpu().numpy()
        else:
            out = np.full((m.nc, 5), np.nan)
            ns.partition_residual(ext, out)
        assert np.isnan(out[:lo]).all() and np.isnan(out[hi:]).all()
        R[lo:hi] = out[lo:hi]
    return R


@pytest.mark.gpu
@pytest.mark.parametrize("nparts", [2, 3])
@pytest.mark.parametrize("family", sorted(ALL))
def test_partitioned_residual_bit_exact(family, nparts, fb):
    case = ALL[family]()
    cs, m = _setup(fb, case)
    ref = fb.NavierStokes(m, cs, 0).residual(case.state)
    R = _partitioned(fb, case, cs, m, nparts)
    assert np.array_equal(R.view(np.uint64), ref.view(np.uint64))


@pytest.mark.gpu
@pytest.mark.parametrize("family,kw", [("wedge", dict(limiter="minmod")), ("cylinder", dict(flux="AUSM+up")),
                                       ("hypersonic", dict(limiter="vk")), ("plate", dict(flux="SD-SLAU"))])
def test_partitioned_residual_exact_gradients_and_fluxes(family, kw, fb):
    case = SMALL[family](**kw)
    cs, m = _setup(fb, case)
    ref = fb.NavierStokes(m, cs, 0, exact_gradients=True).residual(case.state)
    R = _partitioned(fb, case, cs, m, 4, exact=True)
    assert np.array_equal(R.view(np.uint64), ref.view(np.uint64))


@pytest.mark.gpu
@pytest.mark.parametrize("family", ["wedge", "hypersonic", "box_hexpyr"])
def test_partitioned_residual_tecplot_shuffled_faces(family, fb):
    """A Tecplot grid with its faces shuffled: the stale outlet density walks
    back over an arbitrary face order and the halo follows the file's
    connectivity; the owned rows stay bit-identical."""
    import os
    import tempfile

    from freecfd_b200 import cases
    case = ALL[family]()
    d = tempfile.mkdtemp(prefix="fcfd_partt_")
    path = cases.write_tecplot(case.mesh, os.path.join(d, "grid.dat"), order="shuffled", seed=7)
    cs = fb.Case(case.write_deck(d))
    m = fb.Mesh(None, cs, tecplot=path)
    ref = fb.NavierStokes(m, cs, 0).residual(case.state)
    R = _partitioned(fb, case, cs, m, 3)
    assert np.array_equal(R.view(np.uint64), ref.view(np.uint64))


@pytest.mark.gpu
def test_partitioned_residual_device_pointers(fb):
    case = SMALL["cylinder"]()
    cs, m = _setup(fb, case)
    ref = fb.NavierStokes(m, cs, 0).residual(case.state)
    R = _partitioned(fb, case, cs, m, 3, device=True)
    assert np.array_equal(R.view(np.uint64), ref.view(np.uint64))


@pytest.mark.gpu
def test_partitioned_residual_one_stream(fb):
    """PartitionedResidual (one rank, no process group): exchange, extrema and
    both phases enqueued on the context's stream; equals the single-domain
    residual, also after the state changes."""
    import torch
    from freecfd_b200.partition import PartitionedResidual
    case = SMALL["cylinder"]()
    cs, m = _setup(fb, case)
    ns0 = fb.NavierStokes(m, cs, 0)
    plan = HaloPlan(m, cs, 1)
    W = torch.as_tensor(case.state, device="cuda")
    R = torch.full_like(W, float("nan"))
    res = PartitionedResidual(fb.NavierStokes(m, cs, 0), plan, 0, W)
    for k in range(3):
        Wk = case.state * (1 + 1e-3 * k)
        W.copy_(torch.as_tensor(Wk))
        res(R)
        assert np.array_equal(R.cpu().numpy(), ns0.residual(Wk))


@pytest.mark.gpu
def test_partitioned_residual_without_sync(fb):
    """Steps enqueued without a host synchronisation (FCFD_NO_SYNC) give the
    same rows as synchronised ones; a boundary-condition error raised inside
    such a step stays flagged until check() reports it (FCFD_ERR_BC), and the
    flag is cleared afterwards."""
    import torch
    from freecfd_b200.partition import PartitionedResidual
    case = SMALL["cylinder"]()
    cs, m = _setup(fb, case)
    ns0 = fb.NavierStokes(m, cs, 0)
    W = torch.as_tensor(case.state, device="cuda")
    R = torch.full_like(W, float("nan"))
    res = PartitionedResidual(fb.NavierStokes(m, cs, 0), HaloPlan(m, cs, 1), 0, W)
    for k in range(3):
        Wk = case.state * (1 + 1e-3 * k)
        W.copy_(torch.as_tensor(Wk))
        res(R, sync=False)
        res.check()
        assert np.array_equal(R.cpu().numpy(), ns0.residual(Wk))
    # supersonic flow into the inlet, whose deck gives rho and V only
    Wbad = case.state.copy()
    Wbad[:, 1] = 1500.0
    W.copy_(torch.as_tensor(Wbad))
    res(R, sync=False)
    with pytest.raises(fb.FcfdError) as e:
        res.check()
    assert e.value.code == 8
    res.check()
    W.copy_(torch.as_tensor(case.state))
    res(R, sync=False)
    res.check()
    assert np.array_equal(R.cpu().numpy(), ns0.residual(case.state))


@pytest.mark.gpu
def test_partitioned_residual_nccl_process_group(fb):
    """The same step inside an NCCL process group (one rank): the extrema
    all-reduce runs on the library's stream through NCCL; the halo exchange
    has no peers.  Owned rows equal the single-domain residual."""
    import socket

    import torch
    import torch.distributed as dist
    from freecfd_b200.partition import PartitionedResidual
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        case = SMALL["wedge"]()
        cs, m = _setup(fb, case)
        ref = fb.NavierStokes(m, cs, 0).residual(case.state)
        W = torch.as_tensor(case.state, device="cuda")
        R = torch.full_like(W, float("nan"))
        res = PartitionedResidual(fb.NavierStokes(m, cs, 0), HaloPlan(m, cs, 1), 0, W)
        for _ in range(2):
            res(R)
        assert np.array_equal(R.cpu().numpy(), ref)
        del res
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_partition_errors(fb):
    case = SMALL["wedge"]()
    cs, m = _setup(fb, case)
    ns = fb.NavierStokes(m, cs, 0)
    with pytest.raises(fb.FcfdError):
        ns.partition_extrema(case.state)  # no partition selected
    with pytest.raises(fb.FcfdError):
        ns.set_partition(0, m.nc + 1)
    ns.set_partition(0, m.nc // 2)
    ns.set_partition(0, 0)
    from freecfd_b200 import cases
    plate = cases.plate_case(ni=8, nj=4, nk=2)  # k-omega deck
    pcs, pm = _setup(fb, plate)
    with pytest.raises(fb.FcfdError) as e:
        fb.NavierStokes(pm, pcs, 0).set_partition(0, pm.nc // 2)
    assert e.value.code == 7
    # the whole-mesh residual is unaffected by a partition set and cleared
    R = ns.residual(case.state)
    ref = fb.NavierStokes(m, cs, 0).residual(case.state)
    assert np.array_equal(R, ref)


@pytest.mark.gpu
def test_decomposed_newton_one_rank_nccl(oracle_mod, fb):
    """The decomposed Newton-Krylov solve (partitioned residual, FD J.v of
    the partitioned residual, block-Jacobi blocks and time terms from the
    library, GMRES with all-reduced dots) inside a one-rank NCCL group on a
    first-order supersonic wedge: it reaches a 1e-10 drop of the oracle's
    mass residual, and its state agrees with the library's single-domain
    Newton solve at the same tolerance."""
    import socket
    import tempfile

    import torch
    import torch.distributed as dist
    from freecfd_b200 import cases
    from freecfd_b200.partition import DecomposedNewton
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        case = cases.wedge_case(ni=30, nj=15, order="first")
        d = tempfile.mkdtemp(prefix="fcfd_dn_")
        cs = fb.Case(case.write_deck(d))
        m = fb.Mesh(case.mesh, cs)
        o = oracle_mod.Oracle(case, d)
        W = torch.as_tensor(case.state.copy(), device="cuda")
        dn = DecomposedNewton(fb.NavierStokes(m, cs, 0), m, cs, HaloPlan(m, cs, 1), 0, W)
        rep = dn.solve(tol=1e-10, max_newton=300, cfl0=2.0, cfl_max=1e6, krylov_dim=40, krylov_rtol=1e-3,
                       krylov_cycles=4)
        assert rep["converged"], rep["history"][-5:]
        Wd = W.cpu().numpy()
        r0 = np.linalg.norm(o.residual(case.state)[:, 0])
        assert np.linalg.norm(o.residual(Wd)[:, 0]) <= 1e-9 * r0
        Ws, rs = fb.NavierStokes(m, cs, 0).newton_solve(case.state, tol=1e-10, max_newton=300, cfl0=2.0,
                                                         cfl_max=1e6, krylov_rtol=1e-3, krylov_cycles=4, jvp=False,
                                                         precond_sweeps=0)
        scale = np.abs(Ws).max(axis=0)
        scale[1:4] = np.abs(Ws[:, 1:4]).max()
        assert (np.abs(Wd - Ws).max(axis=0) / scale).max() <= 1e-6
        del dn
    finally:
        dist.destroy_process_group()
