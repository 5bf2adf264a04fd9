"""The allocation-free CFL_MAX time step against the context-based one.

fcfd_local_dt_cflmax_noalloc exists for callers that cannot allocate device
memory (its scratch is a static __device__ array).  It must give the same
time steps as fcfd_local_dt in CFL_MAX mode, on consecutive calls (the shared
scratch keeps the previous call's contents), whether this file runs alone in
a fresh process or after every other test.  Collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from freecfd_b200 import cases
from tests.util import build_pair


@pytest.mark.gpu
def test_noalloc_cflmax_matches_context_path(oracle_mod, fb):
    import torch
    case = cases.wedge_case(ni=40, nj=20)
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    d, _ = cs.summary()
    gamma, gas_R, Pref, Tref = d[0], d[1], d[2], d[3]
    length = torch.from_numpy(np.ascontiguousarray(m.geometry()["cell_length"][: m.nc])).cuda()
    rng = np.random.default_rng(3)
    for call, cfl in enumerate((7.5, 0.8)):
        W = case.state * (1.0 + 0.02 * rng.uniform(-1, 1, size=case.state.shape))
        ref = ns.local_dt(W, cfl, mode=1)                      # existing entry point (context scratch)
        Wd = torch.from_numpy(np.ascontiguousarray(W)).cuda()
        dt = torch.full((m.nc,), -1.0, dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        rc = fb.lib.fcfd_local_dt_cflmax_noalloc(ctypes.c_void_p(Wd.data_ptr()), ctypes.c_void_p(length.data_ptr()),
                                                 m.nc, gamma, gas_R, Pref, Tref, cfl,
                                                 ctypes.c_void_p(dt.data_ptr()), ctypes.c_void_p(stream))
        assert rc == 0, fb.lib.fcfd_last_error()
        torch.cuda.synchronize()
        got = dt.cpu().numpy()
        assert np.abs(got - ref).max() <= 1e-15 * np.abs(ref).max(), (call, got[:3], ref[:3])
        assert np.all(got == got[0])


@pytest.mark.gpu
def test_noalloc_rejects_oversize(fb):
    import torch
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = fb.lib.fcfd_local_dt_cflmax_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                             1048577, 1.4, 287.0, 0.0, 0.0, 1.0, ctypes.c_void_p(x.data_ptr()), None)
    assert rc == 1
    assert b"static scratch limit" in fb.lib.fcfd_last_error()


def _torch_dt(W, length, cfl, gamma, gas_R, Pref, Tref):
    """The per-cell CFL_MAX time step formula of update_time_step
    (time_step.cc:181-186) evaluated in torch FP64."""
    import torch
    p, T = W[:, 0], W[:, 4]
    rho = (p + Pref) / (gas_R * (T + Tref))
    a = torch.sqrt(gamma * (p + Pref) / rho)
    return cfl * length / (torch.sqrt((W[:, 1:4] ** 2).sum(dim=1)) + a)


@pytest.mark.gpu
def test_noalloc_at_the_size_limit(fb):
    """1,048,576 cells, the largest size the static scratch accepts (4096
    partial minima): the time step equals a torch minimum over the per-cell
    steps, on two calls in a row."""
    import torch
    n = 1048576
    g = torch.Generator(device="cpu").manual_seed(17)
    W = torch.empty((n, 5), dtype=torch.float64)
    W[:, 0] = 101325.0 * (1 + 0.05 * torch.rand(n, generator=g, dtype=torch.float64))
    W[:, 1:4] = 300.0 * (torch.rand((n, 3), generator=g, dtype=torch.float64) - 0.5)
    W[:, 4] = 300.0 * (1 + 0.05 * torch.rand(n, generator=g, dtype=torch.float64))
    length = 1e-3 * (1 + torch.rand(n, generator=g, dtype=torch.float64))
    W, length = W.cuda(), length.cuda()
    dt = torch.full((n,), -1.0, dtype=torch.float64, device="cuda")
    for cfl in (3.0, 0.5):
        want = _torch_dt(W, length, cfl, 1.4, 287.0, 0.0, 0.0).min().item()
        rc = fb.lib.fcfd_local_dt_cflmax_noalloc(ctypes.c_void_p(W.data_ptr()), ctypes.c_void_p(length.data_ptr()),
                                                 n, 1.4, 287.0, 0.0, 0.0, cfl, ctypes.c_void_p(dt.data_ptr()), None)
        assert rc == 0, fb.lib.fcfd_last_error()
        torch.cuda.synchronize()
        assert abs(dt[0].item() - want) <= 1e-15 * want
        assert bool((dt == dt[0]).all())


@pytest.mark.gpu
def test_noalloc_skips_nan_cells_like_the_context_path(oracle_mod, fb):
    """A NaN cell drops out of the minimum in both entry points, as std::min
    drops it in the reference's update_time_step."""
    import torch
    case = cases.wedge_case(ni=40, nj=20)
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    d, _ = cs.summary()
    W = case.state.copy()
    W[17, 4] = np.nan
    ref = ns.local_dt(W, 2.0, mode=1)
    assert np.isfinite(ref).all()
    length = torch.from_numpy(np.ascontiguousarray(m.geometry()["cell_length"][: m.nc])).cuda()
    Wd = torch.from_numpy(np.ascontiguousarray(W)).cuda()
    dt = torch.empty((m.nc,), dtype=torch.float64, device="cuda")
    rc = fb.lib.fcfd_local_dt_cflmax_noalloc(ctypes.c_void_p(Wd.data_ptr()), ctypes.c_void_p(length.data_ptr()), m.nc,
                                             d[0], d[1], d[2], d[3], 2.0, ctypes.c_void_p(dt.data_ptr()), None)
    assert rc == 0
    torch.cuda.synchronize()
    assert np.abs(dt.cpu().numpy() - ref).max() <= 1e-15 * np.abs(ref).max()
