"""Deck-driven time loop (fcfd_run, the reference's main.cc:294-438).

Each step's state is recovered from the restart files the run writes
(restartfrequency=1), so every column of convergence.dat and every loads line
is checked against quantities recomputed here: the physical time and max CFL of
update_time_step (time_step.cc:143-224) from the device local time step, the
residual of update_variables (ns.cc:338-396) from the state differences and
the written dt, and the loads (ns_assemble_linear_system.cc:108-119) against
the oracle's forces and moments at the start-of-step state."""
import os
import re
import shutil

import numpy as np
import pytest

from freecfd_b200 import cases
from tests.util import build_pair

LINE = re.compile(r"^(\d+)\t1\t(\S+)\t(\S+)\t(\d+)\t(\S+)$")


def _cylinder(tm, wo, ntheta=32, nr=16, **kw):
    case = cases.cylinder_case(ntheta=ntheta, nr=nr, limiter="none", **kw)
    case.deck = case.deck.replace("time marching { CFLmax=50.; number of steps=500; }", "time marching { %s }" % tm)
    case.deck = case.deck.replace("load frequency=1; include bcs=[1];", wo)
    return case


def _states(run_dir, n, W0):
    """Start-of-step state k (k = 1..n) and the dt used in step k."""
    import freecfd_b200 as fb
    nc = W0.shape[0]
    Ws, dts = [W0], []
    for k in range(1, n + 1):
        r = fb.read_restart(run_dir, k, nc)
        Ws.append(r["W"])
        dts.append(np.fromfile(os.path.join(run_dir, "restart", str(k), "dt.1")))
    return Ws, dts


def _lines(run_dir):
    with open(os.path.join(run_dir, "convergence.dat")) as f:
        out = []
        for ln in f.read().splitlines():
            m = LINE.match(ln)
            assert m, ln
            out.append((int(m.group(1)), float(m.group(2)), float(m.group(3)), int(m.group(4)), float(m.group(5))))
    return out


def _close3(printed, value):
    """A %.3e column agrees with the recomputed value to its printed digits."""
    return abs(printed - value) <= 5.001e-4 * abs(value) + 1e-300


@pytest.mark.gpu
def test_run_cfl_max_ramp_columns_loads_and_restart(oracle_mod, fb, tmp_path):
    n = 8
    case = _cylinder("CFLmax=40.; number of steps=%d; ramp (initial=2.; growth=2.;);" % n,
                     "load frequency=1; restart frequency=1; include bcs=[1,3]; moment center=[0.25,0.5,0.];")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    a = tmp_path / "a"
    a.mkdir()
    W, rep = ns.run(case.state, work_dir=a)
    assert rep["status"] == 0 and rep["steps"] == n
    Ws, dts = _states(a, n, case.state)
    assert np.array_equal(Ws[-1], W)
    rows = _lines(a)
    assert [r[0] for r in rows] == list(range(1, n + 1))
    t = 0.0
    first = None
    for k in range(1, n + 1):
        cfl = min(2.0 * 2.0 ** (k - 1), 40.0)
        dt = ns.local_dt(Ws[k - 1], cfl, mode=1)
        assert np.array_equal(dts[k - 1], dt)  # CFL_MAX: every cell takes the global minimum
        t += dt[0]
        step, tcol, cflcol, nit, rescol = rows[k - 1]
        assert _close3(tcol, t) and _close3(cflcol, cfl)
        assert 1 <= nit <= 10
        d = Ws[k] - Ws[k - 1]
        tot = np.array([(d[:, 0] ** 2 / dt ** 2).sum(), (d[:, 1:4] ** 2 / dt[:, None] ** 2).sum(),
                        (d[:, 4] ** 2 / dt ** 2).sum()])
        if k == 1:
            first = np.sqrt(tot)
        assert _close3(rescol, (np.sqrt(tot) / first).mean())
    assert rep["time"] == pytest.approx(t, rel=1e-14)
    # loads: force and moment about (0.25, 0.5, 0) of BCs 1 and 3 at the
    # start-of-step state, written with the physical time after the step's dt
    for b in (1, 3):
        with open(a / "volume_output" / ("loads_grid_1_BC_%d.dat" % b)) as f:
            L = [ln.split("\t") for ln in f.read().splitlines()]
        assert [int(r[0]) for r in L] == list(range(1, n + 1))
        for k in range(1, n + 1):
            F, M = o.loads(Ws[k - 1], moments=True)
            got = np.array([float(v) for v in L[k - 1][2:8]])
            ref = np.concatenate([F[b - 1], M[b - 1]])
            # printed with 9 significant digits (scientific, precision 8)
            tol = 5.001e-9 * np.abs(ref) + 1e-13 * np.abs(ref).max()
            assert (np.abs(got - ref) <= tol).all(), (b, k, got, ref)
    # a restart continues with the ramp's target CFL: update_time_step sets
    # the initial value only at time step 1 (time_step.cc:145-156)
    bdir = tmp_path / "b"
    bdir.mkdir()
    shutil.copytree(a / "restart", bdir / "restart")
    ns.run(np.zeros_like(case.state), work_dir=bdir, restart_step=4, max_steps=2)
    assert [r[2] for r in _lines(bdir)] == [40.0, 40.0]


@pytest.mark.gpu
def test_run_restart_continuation_is_exact(oracle_mod, fb, tmp_path):
    """Without a ramp, 3 steps + restart + 3 steps = 6 steps, bit for bit
    (every reduction on the path has a fixed order), and convergence.dat is
    appended to."""
    case = _cylinder("CFLmax=10.; number of steps=6;", "restart frequency=3;")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    a, b = tmp_path / "a", tmp_path / "b"
    a.mkdir()
    b.mkdir()
    W, rep = ns.run(case.state, work_dir=a)
    shutil.copytree(a / "restart", b / "restart")
    with open(a / "convergence.dat") as f:
        head = f.read().splitlines()[:3]
    (b / "convergence.dat").write_text("\n".join(head) + "\n")
    W2, rep2 = ns.run(np.zeros_like(case.state), work_dir=b, restart_step=3, max_steps=3)
    assert rep2["steps"] == 3
    assert np.array_equal(W2, W)
    # time.dat keeps 6 significant digits of the physical time (default
    # stream precision), as the reference's does
    assert abs(rep2["time"] - rep["time"]) <= 1e-5 * rep["time"]
    ra, rb = _lines(a), _lines(b)
    assert [r[0] for r in rb] == list(range(1, 7))
    assert [r[2:4] for r in rb] == [r[2:4] for r in ra]
    assert all(_close3(x[1], y[1]) for x, y in zip(rb, ra))


@pytest.mark.gpu
def test_run_fixed_step_and_local_cfl(oracle_mod, fb, tmp_path):
    case = _cylinder("step size=2.e-6; number of steps=3;", "restart frequency=1;")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    W, rep = ns.run(case.state, work_dir=tmp_path)
    Ws, dts = _states(tmp_path, 3, case.state)
    for k, row in enumerate(_lines(tmp_path), start=1):
        assert _close3(row[1], 2e-6 * k)
        assert np.all(dts[k - 1] == 2e-6)
        # max CFL of the fixed step: max (|V| + a) dt / lengthScale
        ref = (2e-6 / ns.local_dt(Ws[k - 1], 1.0, mode=0)).max()
        assert _close3(row[2], ref)
    case = _cylinder("CFLlocal=8.; number of steps=3; ramp (initial=1.; growth=3.;);", "restart frequency=1;")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    d2 = tmp_path / "local"
    d2.mkdir()
    ns.run(case.state, work_dir=d2)
    Ws, dts = _states(d2, 3, case.state)
    t = 0.0
    for k, row in enumerate(_lines(d2), start=1):
        cfl = min(3.0 ** (k - 1), 8.0)
        dt = ns.local_dt(Ws[k - 1], cfl, mode=0)
        assert np.array_equal(dts[k - 1], dt)
        t += dt.min()
        assert _close3(row[1], t) and _close3(row[2], cfl)


@pytest.mark.gpu
def test_run_schedule_file_dump_restart_and_option_reread(oracle_mod, fb, tmp_path):
    """The CFL schedule file (time_step.cc:163-179: CFLmax = value of the last
    listed step below the current one, ramp off), a dump_restart request file
    and the re-read of the timemarching section every updatefrequency steps."""
    case = _cylinder("CFLmax=3.; number of steps=6; update frequency=4; schedule file=cfl.txt;", "")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    (tmp_path / "cfl.txt").write_text("2 5.\n3 7.5\n")
    (tmp_path / "dump_restart").write_text("")
    W, rep = ns.run(case.state, work_dir=tmp_path)
    rows = _lines(tmp_path)
    # steps 1-2: the deck's 3; step 3: 5 (3 > 2); steps 4..: 7.5 (> 3); the
    # re-read at step 4 keeps the schedule (the file still exists)
    assert [r[2] for r in rows] == [3.0, 3.0, 5.0, 7.5, 7.5, 7.5]
    assert not (tmp_path / "dump_restart").exists()
    assert sorted(os.listdir(tmp_path / "restart")) == ["1", "6", "partitionMap_1.dat"]


@pytest.mark.gpu
def test_run_converges_and_rejects_unsupported(oracle_mod, fb, tmp_path):
    """200 CFL-ramped implicit steps drive the laminar cylinder's update
    residual down by 5 orders; a turbulent deck without k and omega is
    refused."""
    case = _cylinder("CFLmax=1.e4; number of steps=200; ramp (initial=2.; growth=1.3;);", "")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    W, rep = ns.run(case.state, work_dir=tmp_path, precond_sweeps=2)
    assert rep["res"] < 1e-5, rep
    r0 = np.linalg.norm(o.residual(case.state)[:, 0])
    assert np.linalg.norm(o.residual(W)[:, 0]) < 1e-5 * r0
    plate = cases.plate_case(ni=8, nj=4, nk=2)
    o, cs, m = build_pair(plate, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    with pytest.raises(fb.FcfdError) as e:
        ns.run(plate.state, work_dir=tmp_path)
    assert e.value.code == 1


LINE_T = re.compile(r"^(\d+)\t1\t(\S+)\t(\S+)\t(\d+)\t(\S+)\t(\d+)\t(\S+)$")


def _plate_deck(tm, wo=""):
    case = cases.plate_case(ni=24, nj=12, nk=2)
    case.deck = case.deck.replace("time marching { CFLmax=50.; number of steps=500; }", "time marching { %s }" % tm)
    case.deck = case.deck.replace("surface variables=[p]; );", "surface variables=[p]; %s);" % wo)
    return case


def _lines_t(run_dir):
    with open(os.path.join(run_dir, "convergence.dat")) as f:
        out = []
        for ln in f.read().splitlines():
            m = LINE_T.match(ln)
            assert m, ln
            out.append(tuple(int(v) if i in (0, 3, 5) else float(v) for i, v in enumerate(m.groups())))
    return out


@pytest.mark.gpu
def test_run_turbulent_plate_columns_and_restart(oracle_mod, fb, tmp_path):
    """Turbulent decks: each time step is one coupled backward-Euler solve on
    (p, u, v, w, T, k, omega).  convergence.dat carries the reference's
    turbulent columns (main.cc:351-361): the flow residual of
    update_variables (ns.cc:338-396) and the k-omega residual of
    rans.cc:240-250, both recomputed here from the per-step restart states;
    the restart files hold k, omega and the eddy viscosity of
    update_eddy_viscosity (rans_update_eddy_viscosity.cc:26-50:
    min(rho k / omega, ratio limit x mu)); 3 steps + restart + 3 steps equal
    6 steps bit for bit."""
    n = 6
    case = _plate_deck("CFLmax=5.; number of steps=%d;" % n, "restart frequency=1; ")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    nc = m.nc
    a = tmp_path / "a"
    a.mkdir()
    W, rep = ns.run(case.state, work_dir=a, K=case.kstate)
    assert rep["status"] == 0 and rep["steps"] == n
    K = rep["K"]
    rs = [dict(W=case.state, K=case.kstate)] + [fb.read_restart(a, k, nc, turbulent=True) for k in range(1, n + 1)]
    assert np.array_equal(rs[-1]["W"], W) and np.array_equal(rs[-1]["K"], K)
    rows = _lines_t(a)
    assert [r[0] for r in rows] == list(range(1, n + 1))
    first = firstk = None
    for k in range(1, n + 1):
        dt = np.fromfile(os.path.join(a, "restart", str(k), "dt.1"))
        assert np.array_equal(dt, ns.local_dt(rs[k - 1]["W"], 5.0, mode=1))
        d = rs[k]["W"] - rs[k - 1]["W"]
        dk = rs[k]["K"] - rs[k - 1]["K"]
        tot = np.sqrt([(d[:, 0] ** 2 / dt ** 2).sum(), (d[:, 1:4] ** 2 / dt[:, None] ** 2).sum(),
                       (d[:, 4] ** 2 / dt ** 2).sum()])
        totk = np.sqrt((dk ** 2 / dt[:, None] ** 2).sum(axis=0))
        if k == 1:
            first, firstk = tot, totk
        step, tcol, cflcol, nit, rescol, nitk, rkcol = rows[k - 1]
        assert _close3(cflcol, 5.0) and 1 <= nit <= 10 and nitk == nit
        assert _close3(rescol, (tot / first).mean()) and _close3(rkcol, (totk / firstk).mean())
        # eddy viscosity of the updated state
        Wk, Kk = rs[k]["W"], rs[k]["K"]
        rho = Wk[:, 0] / (cases.R_AIR * Wk[:, 4])
        mt = rho * Kk[:, 0] / Kk[:, 1]
        mu_t = rs[k]["mu_t"]
        assert (mu_t > 0).all() and (mu_t <= mt * (1 + 1e-12)).all()
        assert np.mean(np.abs(mu_t - mt) <= 1e-12 * mt) > 0.5
    assert (K > 0).all() and np.isfinite(W).all()
    b = tmp_path / "b"
    b.mkdir()
    shutil.copytree(a / "restart", b / "restart")
    with open(a / "convergence.dat") as f:
        head = f.read().splitlines()[:3]
    (b / "convergence.dat").write_text("\n".join(head) + "\n")
    W2, rep2 = ns.run(np.zeros_like(case.state), work_dir=b, restart_step=3, max_steps=3,
                      K=np.zeros_like(case.kstate))
    assert rep2["steps"] == 3
    assert np.array_equal(W2, W) and np.array_equal(rep2["K"], K)
    assert [r[3:6:2] for r in _lines_t(b)] == [r[3:6:2] for r in rows]


@pytest.mark.gpu
def test_run_turbulent_plate_converges(oracle_mod, fb, tmp_path):
    """100 CFL-ramped coupled steps on the turbulent plate: the update
    residual of the flow falls below 1e-2 of its first value and the
    reference's residual (the oracle's, at the final state) by more than an
    order in mass and momentum and two in energy (measured: 3e-2, 3e-2,
    7e-3), with k and omega positive.  The k-omega update residual levels off
    near 5e-2, as in the coupled Newton solve, and GMRES reaches its
    10-vector cap at the top CFL."""
    case = _plate_deck("CFLmax=200.; number of steps=100; ramp (initial=1.; growth=1.15;);")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    W, rep = ns.run(case.state, work_dir=tmp_path, K=case.kstate)
    K = rep["K"]
    assert rep["status"] == 0 and (K > 0).all() and np.isfinite(W).all()
    rows = _lines_t(tmp_path)
    print("turbulent plate:", [(r[0], r[4], r[6]) for r in rows[::10]], rows[-1])
    R0, _ = o.rans_residual(case.state, case.kstate)
    R1, _ = o.rans_residual(W, K)
    red = np.linalg.norm(R1, axis=0) / np.linalg.norm(R0, axis=0)
    print("oracle residual reduction per equation:", red)
    assert (red[:3] < 0.1).all() and red[4] < 2e-2, red
    assert rows[-1][4] < 1e-2 and rows[-1][6] < 0.5, rows[-1]


@pytest.mark.gpu
def test_run_reports_nonphysical_state_as_divergence(oracle_mod, fb, tmp_path):
    """The impulsively started M = 8 cylinder at first order and CFL 0.5
    leaves negative pressures after its first implicit step; the next
    residual is then not finite, and the run ends with FCFD_ERR_DIVERGED
    (the reference's NaN check, ns.cc:349-355) instead of marching on with
    zero updates."""
    case = cases.hypersonic_case(128, 64, ns_extra=" order=first;")
    case.deck = case.deck.replace("time marching { CFLmax=1.e3; number of steps=500; ramp (initial=0.1; growth=1.1;); }",
                                  "time marching { CFLmax=0.5; number of steps=20; }")
    o, cs, m = build_pair(case, oracle_mod, fb)
    ns = fb.NavierStokes(m, cs, 0)
    W, rep = ns.run(case.state, work_dir=tmp_path, raise_on_fail=False)
    assert rep["status"] == 3, rep
    assert 1 <= rep["steps"] < 20
    b = tmp_path / "b"
    b.mkdir()
    with pytest.raises(fb.FcfdError) as e:
        ns.run(case.state, work_dir=b)
    assert e.value.code == 3
