"""Restart files in the reference's layout (host code, no GPU).

write_restart (write_restart.cc:45-100) / Variable::dump_cell_data
(variable.h:229-245) write raw native-endian doubles per cell in cell order,
a text partition map and a text time.dat with C++ default float formatting;
read_restart (read_restart.cc:44-102) / Variable::read_cell_data
(variable.h:248-271) place every value at the cell its global id names.  The
expected files here are built independently with numpy from that description."""
import os

import numpy as np
import pytest


def _state(nc, seed=0):
    rng = np.random.default_rng(seed)
    W = np.empty((nc, 5))
    W[:, 0] = 101325.0 * (1 + 0.01 * rng.uniform(-1, 1, nc))
    W[:, 1:4] = rng.standard_normal((nc, 3)) * 50.0
    W[:, 4] = 300.0 * (1 + 0.01 * rng.uniform(-1, 1, nc))
    return W


def _read(path):
    with open(path, "rb") as f:
        return f.read()


def test_restart_files_match_reference_layout(fb, tmp_path):
    nc, nn = 11, 37
    W = _state(nc)
    dt = np.linspace(1e-5, 2e-5, nc)
    first = np.array([1.25, 3.5e-7, 123456789.0])
    fb.write_restart(tmp_path, 40, W, 0.00123456789, first, n_nodes=nn, dt=dt)
    r = tmp_path / "restart"
    assert sorted(os.listdir(r)) == ["40", "partitionMap_1.dat"]
    assert sorted(os.listdir(r / "40")) == ["T.1", "V.1", "dt.1", "p.1", "time.dat"]
    # partition map: np, then "nodes\tcells", then one global id per line
    assert (r / "partitionMap_1.dat").read_text() == "1\n%d\t%d\n" % (nn, nc) + "".join("%d\n" % c for c in range(nc))
    # time.dat: default ostream formatting (precision 6)
    assert (r / "40" / "time.dat").read_text() == "0.00123457\n1.25\t3.5e-07\t1.23457e+08\n-1\t-1\n-1\n"
    assert _read(r / "40" / "p.1") == np.ascontiguousarray(W[:, 0]).tobytes()
    assert _read(r / "40" / "V.1") == np.ascontiguousarray(W[:, 1:4]).tobytes()
    assert _read(r / "40" / "T.1") == np.ascontiguousarray(W[:, 4]).tobytes()
    assert _read(r / "40" / "dt.1") == dt.tobytes()
    back = fb.read_restart(tmp_path, 40, nc)
    assert np.array_equal(back["W"], W)
    assert back["time"] == 0.00123457
    assert np.array_equal(back["first_res"], [1.25, 3.5e-7, 1.23457e8])
    assert np.array_equal(back["rans_first_res"], [-1.0, -1.0])


def test_restart_turbulent_variables(fb, tmp_path):
    nc = 9
    W = _state(nc, 1)
    rng = np.random.default_rng(2)
    K = rng.uniform(1e-3, 1.0, (nc, 2))
    mu_t = rng.uniform(1e-6, 1e-4, nc)
    fb.write_restart(tmp_path, 3, W, 1.5, [1.0, 2.0, 3.0], n_nodes=20, K=K, mu_t=mu_t, rans_first_res=[0.5, 0.25])
    d = tmp_path / "restart" / "3"
    assert _read(d / "k.1") == np.ascontiguousarray(K[:, 0]).tobytes()
    assert _read(d / "omega.1") == np.ascontiguousarray(K[:, 1]).tobytes()
    assert _read(d / "mu_t.1") == mu_t.tobytes()
    assert (d / "time.dat").read_text().split("\n")[2] == "0.5\t0.25"
    back = fb.read_restart(tmp_path, 3, nc, turbulent=True)
    assert np.array_equal(back["K"], K) and np.array_equal(back["mu_t"], mu_t)
    assert np.array_equal(back["rans_first_res"], [0.5, 0.25])


def test_restart_from_partitioned_run(fb, tmp_path):
    """Files of a 3-partition run (cells written partition by partition, each
    in its local order, global ids in the partition map) are scattered back
    to global cell order."""
    nc = 13
    W = _state(nc, 3)
    perm = np.random.default_rng(4).permutation(nc)
    parts = [perm[:5], perm[5:9], perm[9:]]
    r = tmp_path / "restart"
    (r / "7").mkdir(parents=True)
    with open(r / "partitionMap_1.dat", "w") as f:
        f.write("3\n")
        for q in parts:
            f.write("%d\t%d\n" % (10, len(q)))
            f.write("".join("%d\n" % g for g in q))
    (r / "7" / "time.dat").write_text("2.5\n1\t2\t3\n-1\t-1\n-1\n")
    order = np.concatenate(parts)
    (r / "7" / "p.1").write_bytes(np.ascontiguousarray(W[order, 0]).tobytes())
    (r / "7" / "V.1").write_bytes(np.ascontiguousarray(W[order, 1:4]).tobytes())
    (r / "7" / "T.1").write_bytes(np.ascontiguousarray(W[order, 4]).tobytes())
    back = fb.read_restart(tmp_path, 7, nc)
    assert np.array_equal(back["W"], W)
    assert back["time"] == 2.5


def test_restart_errors_are_status_codes(fb, tmp_path):
    with pytest.raises(fb.FcfdError) as e:
        fb.read_restart(tmp_path, 1, 5)
    assert e.value.code == 1
    W = _state(6)
    fb.write_restart(tmp_path, 2, W, 0.0, [1.0, 1.0, 1.0], n_nodes=8)
    with pytest.raises(fb.FcfdError):  # the mesh has another cell count
        fb.read_restart(tmp_path, 2, 7)
    p = tmp_path / "restart" / "2" / "T.1"
    p.write_bytes(p.read_bytes()[:-8])
    with pytest.raises(fb.FcfdError):  # truncated variable file
        fb.read_restart(tmp_path, 2, 6)


def test_time_marching_deck_errors(fb, tmp_path):
    """set_time_step_options (time_step.cc:34-47): CFLmax or CFLlocal together
    with stepsize is an input error."""
    from freecfd_b200 import cases
    c = cases.wedge_case(ni=4, nj=3)
    c.deck = c.deck.replace("CFLmax=120.;", "CFLmax=120.; step size=1.e-5;")
    with pytest.raises(fb.FcfdError) as e:
        fb.Case(c.write_deck(str(tmp_path)))
    assert e.value.code == 1
