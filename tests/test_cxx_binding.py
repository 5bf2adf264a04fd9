"""The C ABI as a C++ program links it: tests/cxx/binding_check.cpp is compiled
with g++ against include/fcfd.h and libfcfd_b200.so (no Python, no CUDA
headers) and calls deck parsing, mesh creation and context creation the way
INTEGRATION.md's binding does, including the error paths (status codes and
fcfd_last_error, never an exit).  Without a GPU the context creation must
fail with FCFD_ERR_CUDA; on a GPU the program also evaluates a residual,
which is compared with the oracle."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from freecfd_b200 import cases
from tests.conftest import ROOT
from tests.util import res_err

LIBDIR = os.path.join(ROOT, "freecfd_b200", "_build")


def _build(tmp):
    exe = os.path.join(tmp, "binding_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cxx", "binding_check.cpp"), "-L", LIBDIR, "-lfcfd_b200",
                    f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


def _mesh_file(mesh, path):
    idx, flat = mesh.bc_csr()
    hdr = np.array([mesh.nodes.shape[0], mesh.n_cells, len(mesh.bc_nodes), mesh.conn.shape[0], flat.shape[0]],
                   np.int32)
    with open(path, "wb") as fh:
        for a in (hdr, np.ascontiguousarray(mesh.nodes, np.float64), np.ascontiguousarray(mesh.conn_index, np.int32),
                  np.ascontiguousarray(mesh.conn, np.int32), idx.astype(np.int32), flat.astype(np.int32)):
            fh.write(a.tobytes())


def _run(case, with_state):
    tmp = tempfile.mkdtemp(prefix="fcfd_cxx_")
    exe = _build(tmp)
    deck = case.write_deck(tmp)
    mfile = os.path.join(tmp, "mesh.bin")
    _mesh_file(case.mesh, mfile)
    args = [exe, deck, mfile]
    rfile = os.path.join(tmp, "R.bin")
    if with_state:
        wfile = os.path.join(tmp, "W.bin")
        np.ascontiguousarray(case.state, np.float64).tofile(wfile)
        args += [wfile, rfile]
    p = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    kv = dict(x.split("=", 1) for x in p.stdout.split() if "=" in x)
    return kv, rfile, tmp


def test_cxx_caller_cpu_paths(oracle_mod):
    """Deck, mesh and their error paths from C++; the context creation's
    status matches whether a CUDA device is present."""
    import torch
    case = cases.cylinder_case(ntheta=32, nr=16)
    kv, _, tmp = _run(case, with_state=False)
    assert kv["missing_deck_rc"] == "1" and int(kv["missing_deck_msg_len"]) > 0
    assert kv["deck_rc"] == "0" and kv["mesh_rc"] == "0"
    assert kv["bad_mesh_rc"] in ("1", "2")
    o = oracle_mod.Oracle(case, tmp)
    assert (int(kv["n_cells"]), int(kv["n_faces"]), int(kv["n_ghosts"])) == (o.nc, o.nf, o.nghost)
    assert kv["ctx_rc"] == ("0" if torch.cuda.is_available() else "5")
    assert kv["rcm_rc"] == "0" and kv["rcm_permutation"] == "1"
    assert kv["grad_weights_rc"] == "1"  # null output pointer: FCFD_ERR_INPUT
    # a null context: FCFD_ERR_INPUT from every context-level entry point
    assert kv["null_ctx_rc"] == "1,1,1,1"


@pytest.mark.gpu
def test_cxx_caller_residual(oracle_mod):
    """On the GPU: the residual the C++ caller gets equals the oracle's."""
    case = cases.cylinder_case(ntheta=32, nr=16)
    kv, rfile, tmp = _run(case, with_state=True)
    assert kv["ctx_rc"] == "0" and kv["residual_rc"] == "0"
    R = np.fromfile(rfile).reshape(-1, 5)
    ref = oracle_mod.Oracle(case, tmp).residual(case.state)
    assert res_err(R, ref).max() <= 1e-12
    # the mixed-precision residual with every face in FP64 (shock ratio 0)
    # equals the FP64 residual; a bad gradient-kernel kind is FCFD_ERR_INPUT
    assert kv["mixed_rc"] == "0" and int(kv["mixed_fp64_faces"]) > 0
    assert float(kv["mixed_rel_diff"]) <= 1e-14
    assert kv["set_kernel_bad_rc"] == "1"
    # ordinary launches: the same bits, no flagged error; no k-omega adjoint
    # on a laminar case (FCFD_ERR_INPUT)
    assert kv["overlap_off_rc"] == "0,0" and kv["overlap_same_bits"] == "1" and kv["check_rc"] == "0"
    assert kv["rans_vjp_laminar_rc"] == "1"
