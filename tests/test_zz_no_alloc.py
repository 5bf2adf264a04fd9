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
