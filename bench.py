"""Benchmark: FP64 finite-volume residual throughput (M faces/s) on B200.

A step is one full residual evaluation R(W) — first-order ghost update, LSQ
gradients, limiter (with the global extrema), face fluxes and the atomic-free
cell gather — on the laminar cylinder workload (O-grid 256x128x1 hex, Roe +
viscous, Sutherland, Pr 0.72, VK limiter).  Timing: per-step CUDA events on
the library's stream, L2 flushed (512 MB memset) before every step, max over
ranks.  ``e2e`` is the same metric through the C ABI with pinned host input
and output copies inside the timed region.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
    python -m torch.distributed.run --nproc-per-node N bench.py --gpus N ...

Multi-GPU runs are replicas: every rank evaluates its own copy of the mesh
(weak scaling, no data-path collective).  ``--impl reference`` times the
reference itself -- Free CFD's own sources compiled into oracle/_ref/freecfd_ref
-- on the host cores instead, one process per core.  The default run also
checks the timed residual against the oracle (untimed) and prints residual
lines for the hypersonic, plate and plate64 workloads.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "cylinder": dict(fn="cylinder_case", kw={}),
    "wedge": dict(fn="wedge_case", kw={}),
    "hypersonic": dict(fn="hypersonic_case", kw={}),
    "plate": dict(fn="plate_case", kw=dict(turbulent=False)),
    "plate64": dict(fn="plate_case", kw=dict(nk=64, turbulent=False)),
    "plate_rans": dict(fn="plate_case", kw=dict(turbulent=True)),
    "plate64_rans": dict(fn="plate_case", kw=dict(nk=64, turbulent=True)),
}
METRIC = "M faces/s residual + % HBM peak; Newton wall time to 1e-10: mixed+JVP vs plain FP64"
UNIT = "M faces/s"


def load_cases():
    """freecfd_b200/cases.py on its own (it needs numpy only): the reference
    arm must not import the freecfd_b200 package, whose __init__ loads the
    CUDA library."""
    import importlib.util
    mod = sys.modules.get("fcfd_bench_cases")
    if mod is None:
        spec = importlib.util.spec_from_file_location("fcfd_bench_cases",
                                                      os.path.join(ROOT, "freecfd_b200", "cases.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules["fcfd_bench_cases"] = mod
        spec.loader.exec_module(mod)
    return mod


def make_case(name):
    w = WORKLOADS[name]
    return getattr(load_cases(), w["fn"])(**w["kw"])


def bench_config(case, counts, world):
    """The `config` object, identical in both arms: the workload and its sizes."""
    return {"workload": case.workload, "cells": int(counts["cells"]), "faces": int(counts["faces"]),
            "ghosts": int(counts["ghosts"]), "stencil_entries": int(counts["stencil_entries"]),
            "l2": "GPU arm: 512 MB memset flushes L2 before every step",
            "parallelism": f"replicas x{world}"}


def alg_bytes(m, s=8):
    """Algorithmic bytes of one residual (FP64): interior state read + residual
    write + cell geometry + LSQ matrix, ghost state write+read, face geometry and
    indices, stencil indices and the cell->face list."""
    return (m.nc * (5 * s + 5 * s + 4 * s + 6 * s) + m.nghost * (10 * s) + m.nf * (8 + 7 * s)
            + m.n_grad_entries * 4 + m.n_cell_faces * 4)


def kernel_bytes(m, name, viscous=True, exact_grad=False, s=8, fold_entries=0):
    """Algorithmic bytes of one launch of a residual kernel: every array it
    must read once and every array it writes (cell/face/stencil counts from
    the mesh).  Gradients and limiters are counted where a kernel reads or
    writes them.  fold_entries > 0: the gradient over folded stencils, which
    reads per entry a key and two weighted offsets instead of the entry
    cell's centroid, and the ghosts' states only in the limiter's face loops."""
    nc, nf, nb, nt = m.nc, m.nf, m.nghost, m.nc + m.nghost
    E, ncf = m.n_grad_entries, m.n_cell_faces
    if name == "grad_limiter" and fold_entries:
        b = nc * (5 * s + 3 * s)                     # interior states, own centroid
        b += nc * (7 * s + 4 + 4) + ncf * 4          # cofactors + det, stencil and cell->face CSR
        b += fold_entries * (4 + 6 * s)              # folded entries: key, w d of the cell and of its mirror ghosts
        b += nc * 3 * s                              # mirror weights
        b += nb * 5 * s                              # ghost states (limiter face loops)
        b += nf * (8 + 3 * s)                        # face parent/neighbour, face centroids
        b += nc * (15 * s + 5 * s)                   # gradient and limiter writes
        return b
    if name == "grad_limiter":
        b = nt * (5 * s + 3 * s)                    # states, centroids (stencils reach the ghosts)
        b += nc * (7 * s + 4 + 4) + E * 4 + ncf * 4  # cofactors + det, stencil and cell->face CSR
        b += nc * (4 * s if exact_grad else 3 * s)   # self weights + reciprocal, or mirror weights
        b += nf * (8 + 3 * s)                        # face parent/neighbour, face centroids
        b += nc * (15 * s + 5 * s)                   # gradient and limiter writes
        return b
    if name == "face_flux":
        b = nf * (12 + 3 * s + s + 3 * s + (2 * s if viscous else 0))  # indices, normal, area, centroid, weights
        b += nt * (5 * s + 3 * s)                    # states, centroids
        b += nc * (15 * s + 5 * s)                   # gradients, limiters
        b += nf * 5 * s                              # face differences written
        return b
    if name == "gather":
        return nc * (4 + 5 * s) + ncf * 4 + ncf * 5 * s
    if name == "ghost_minmax":
        return nb * (8 + 5 * s + 5 * s) + nc * 3 * s
    return 0


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampler for the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                self.samples.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 3 + i and "Active" in s[3 + i]
                          and not s[3 + i].startswith("Not")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def port_baseline(case, seconds=4.0):
    """The oracle (C++ restatement, right-hand side only) on one core."""
    import oracle
    o = oracle.Oracle(case)
    if case.kstate is not None:
        def step():
            o.rans_residual(case.state, case.kstate)
    else:
        def step():
            o.residual(case.state)
    step()
    n, t0 = 0, time.perf_counter()
    while True:
        step()
        n += 1
        el = time.perf_counter() - t0
        if el > seconds or n >= 200:
            break
    v = o.nf * n / el / 1e6
    o.close()
    return {"value": round(v, 4), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{n} residual evaluations (right-hand side only) of the same workload ({o.nf} faces) in "
                      f"{el:.1f} s, single-threaded C++ restatement (-O2, no FMA)"}


def _mem_available_gb():
    try:
        with open("/proc/meminfo") as fh:
            for line in fh:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) / 1048576.0
    except OSError:
        pass
    return None


def reference_workers(case, cap):
    """Processes for the reference: one per host core, at most `cap`, and no
    more than half the available memory holds (a process keeps one mesh copy:
    about 6.5 kB per cell)."""
    n = max(1, min(os.cpu_count() or 1, cap))
    mem = _mem_available_gb()
    if mem:
        per = max(0.05, 6.5e3 * case.mesh.n_cells / 1e9)
        n = max(1, min(n, int(0.5 * mem / per)))
    return n


def reference_throughput(case, procs, evals, warmup):
    """The reference itself (oracle/_ref/freecfd_ref: Free CFD's own sources)
    in `procs` concurrent processes, each holding its own copy of the mesh
    like one MPI rank per core without exchanges.  Each process times
    `evals` residual evaluations after `warmup` (the reference's
    calc_cell_grads, calc_limiter and assemble_linear_system, whose face loop
    also forms the first-order finite-difference Jacobian, with the matrix
    inserts switched off).  Throughput = procs x faces x evals / the slowest
    process's time."""
    from oracle import reference
    ref = reference.Reference(case)
    cmd = ref.bench_command(case.state, evals, warmup, case.kstate)
    ps = [subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True) for _ in range(procs)]
    outs = []
    for p in ps:
        out, err = p.communicate(timeout=7200)
        if p.returncode != 0:
            raise RuntimeError(f"freecfd_ref bench failed: {err.strip()[-500:]}")
        line = [x for x in out.splitlines() if x.startswith("FCFD_REF_RESULT ")][-1]
        outs.append(json.loads(line[len("FCFD_REF_RESULT "):]))
    ref.close()
    el = max(o["seconds"] for o in outs)
    nf = outs[0]["nf"]
    return {"value": procs * nf * evals / el / 1e6, "seconds": el, "sizes": outs[0], "procs": procs,
            "evals": evals, "setup_seconds": max(o["setup_seconds"] for o in outs)}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_baseline(case, seconds, cap):
    """The reference on the host cores for a bounded sample (about `seconds`
    of work per process)."""
    from oracle import reference
    if not reference.available():
        return port_baseline(case, seconds)
    procs = reference_workers(case, cap)
    evals = max(2, int(round(seconds * 0.3e6 / max(case.mesh.n_cells * 4, 1))))
    r = reference_throughput(case, procs, evals, 1)
    return {"value": round(r["value"], 4), "unit": UNIT, "cores": procs, "kind": "reference",
            "sample": f"{procs} processes x {evals} residual evaluations of the same workload "
                      f"({r['sizes']['nf']} faces) by the reference's own code (oracle/_ref/freecfd_ref), "
                      f"one mesh copy per process; each evaluation is the reference's calc_cell_grads + "
                      f"calc_limiter + assemble_linear_system, whose face loop also forms its finite-difference "
                      f"Jacobian", "host_cpu": cpu_model(), "nproc": os.cpu_count()}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    from oracle import reference
    case = make_case(args.workload)
    if reference.available():
        procs = reference_workers(case, args.ref_workers)
        r = reference_throughput(case, procs, args.steps, args.warmup)
        value, el, sz, kind = r["value"], r["seconds"], r["sizes"], "reference"
        sample = (f"{procs} processes x {args.steps} timed residual evaluations (after {args.warmup}) of the "
                  f"reference's own code, compiled from its sources (oracle/_ref/freecfd_ref), one mesh copy per "
                  f"process like one MPI rank per core; each evaluation is calc_cell_grads + calc_limiter + "
                  f"assemble_linear_system, whose face loop also forms the first-order finite-difference Jacobian "
                  f"(matrix inserts switched off)")
        counts = dict(cells=sz["nc"], faces=sz["nf"], ghosts=sz["nghost"], stencil_entries=sz["n_grad_entries"])
    else:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/freecfd_ref (the reference compiled from "
                                                              "its sources) was not built"}), flush=True)
        return
    line = {"metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * el / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": bench_config(case, counts, world),
            "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": procs, "kind": kind,
                             "sample": sample, "host_cpu": cpu_model(), "nproc": os.cpu_count()},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_cpu:
        line["port_residual_only"] = port_baseline(case, 4.0)
    print(json.dumps(line), flush=True)


def parity_check(ns, case):
    """Untimed: the timed workload's residual against the oracle (which the
    pin tests hold bit-exact to the compiled reference), normwise relative per
    equation with the three momentum components sharing one scale."""
    import oracle
    o = oracle.Oracle(case)
    if case.kstate is not None:
        R, RK = ns.rans_residual(case.state, case.kstate)
        ref, refk = o.rans_residual(case.state, case.kstate)
    else:
        R, ref = ns.residual(case.state), o.residual(case.state)
    o.close()
    scale = np.abs(ref).max(axis=0)
    scale[1:4] = scale[1:4].max()
    err = np.abs(R - ref).max(axis=0) / np.maximum(scale, 1e-300)
    out = {"max_normwise_rel": float(err.max()), "per_equation": [float(e) for e in err], "bar": 1e-12,
           "against": "oracle (bit-exact to the reference compiled from its sources)"}
    if case.kstate is not None:
        ek = np.abs(RK - refk).max(axis=0) / np.maximum(np.abs(refk).max(axis=0), 1e-300)
        out["komega_per_equation"] = [float(e) for e in ek]
        out["max_normwise_rel"] = float(max(err.max(), ek.max()))
    return out


def residual_subline(fb, name, dev, steps, warmup, parity):
    """One more workload's residual: M faces/s, the step's algorithmic bytes
    over its time, the dominant kernel's roofline fraction and, where the
    oracle finishes in seconds, its parity."""
    import tempfile
    case = make_case(name)
    cs = fb.Case(case.write_deck(tempfile.mkdtemp(prefix="fcfd_bench_")))
    mesh = fb.Mesh(case.mesh, cs)
    ns = fb.NavierStokes(mesh, cs, dev)
    ns.residual(case.state)
    ns.time_residual(max(warmup, 1), True)
    t = ns.time_residual(steps, True)
    ms = float(t[0])
    kern = {"ghost_minmax": t[1], "grad_limiter": t[2], "outlet_density": t[3], "face_flux": t[4], "gather": t[5]}
    peak, kind = peaks()
    B = alg_bytes(mesh)
    top = max(("grad_limiter", "face_flux", "gather", "ghost_minmax"), key=lambda k: kern[k])
    viscous = "viscosity=0." not in case.deck
    exact_grad = "limiter=minmod" in case.deck or "limiter=bj" in case.deck
    gi = ns.gradient_info()
    kb = kernel_bytes(mesh, top, viscous, exact_grad, fold_entries=gi["fold_entries"] if gi["kind"] == 3 else 0)
    out = {"workload": case.workload, "cells": mesh.nc, "faces": mesh.nf, "steps": steps,
           "ms_per_step": round(ms, 5), "value": round(mesh.nf / (ms * 1e-3) / 1e6, 3), "unit": UNIT,
           "step_roofline": {"achieved": round(B / (ms * 1e-3) / 1e9, 1), "frac": round(B / (ms * 1e-3) / 1e9 / peak, 4),
                             "alg_bytes": int(B), "peak": peak, "peak_kind": kind},
           "roofline": {"kernel": top, "alg_bytes_per_launch": int(kb), "ms_per_launch": round(float(kern[top]), 5),
                        "achieved": round(kb / (float(kern[top]) * 1e-3) / 1e9, 1),
                        "frac": round(kb / (float(kern[top]) * 1e-3) / 1e9 / peak, 4),
                        "traffic": NCU_TRAFFIC.get((name, top))},
           "kernels_ms": {k: round(float(v), 5) for k, v in kern.items()}}
    if parity:
        out["parity_err"] = parity_check(ns, case)
    if name == "hypersonic":
        out["mixed_precision"] = mixed_subline(ns, mesh, case, steps, parity)
    del ns
    return out


def flux_scale(case, geo, gamma=1.4, R=287.0):
    """Per-equation magnitude of one face's freestream flux times the
    largest face area (the terms whose cancellation forms the residual)."""
    p, u, v, w, T = case.freestream
    rho = p / (R * T)
    U = float(np.sqrt(u * u + v * v + w * w))
    H = gamma / (gamma - 1.0) * R * T + 0.5 * U * U
    A = float(np.max(geo["face_area"]))
    mom = (rho * U * U + p) * A
    return np.array([rho * U * A, mom, mom, mom, rho * U * H * A])


def mixed_subline(ns, mesh, case, steps, parity, shock_ratio=2.0):
    """The hypersonic residual with the face pass in FP32 and FP64 on the
    faces across a pressure jump (fcfd_residual_mixed, shock_ratio 2), on the
    seeded freestream state and on a state with a bow-shock jump; time per
    evaluation (L2 flushed), FP64 faces, and the error against the FP64
    oracle in units of the face-flux scale."""
    cm = load_cases()
    geo = mesh.geometry()
    out = {"shock_ratio": shock_ratio, "states": {}}
    for label, W in (("seeded_freestream", case.state),
                     ("bow_shock_jump", cm.hypersonic_shock_state(case, geo["cell_centroid"]))):
        W = np.ascontiguousarray(W)
        ns.residual(W)
        ns.time_residual(2, True)
        t64 = ns.time_residual(steps, True)
        R, n64 = ns.residual_mixed(W, shock_ratio)
        ns.time_residual_mixed(2, True, shock_ratio)
        ms, _ = ns.time_residual_mixed(steps, True, shock_ratio)
        d = {"fp64_ms_per_step": round(float(t64[0]), 5), "mixed_ms_per_step": round(ms, 5),
             "speedup": round(float(t64[0]) / ms, 3), "fp64_faces": n64, "faces": mesh.nf,
             "value": round(mesh.nf / (ms * 1e-3) / 1e6, 3), "unit": UNIT}
        if parity:
            import oracle
            o = oracle.Oracle(case)
            ref = o.residual(W)
            o.close()
            err = np.abs(R - ref).max(axis=0) / flux_scale(case, geo)
            d["err_vs_fp64_oracle_of_flux_scale"] = [float(e) for e in err]
        out["states"][label] = d
    return out


def renumber_subline(fb, dev, steps, warmup):
    """The laminar plate 384x192x4 residual in three cell orders: the
    generator's i-j-k order, a seeded random order (an unordered grid) and the
    reverse Cuthill-McKee order of the shuffled grid (fcfd_mesh_rcm).  Same
    discretisation each time; the times show what cell order costs the
    gathers."""
    import tempfile
    cm = load_cases()
    base = make_case("plate")
    out = {"workload": base.workload, "orders": {}}
    sh = cm.shuffle_case(base, 0)
    for label in ("generated", "shuffled", "rcm_of_shuffled"):
        if label == "generated":
            case = base
        elif label == "shuffled":
            case = sh
        cs = fb.Case(case.write_deck(tempfile.mkdtemp(prefix="fcfd_bench_")))
        if label == "rcm_of_shuffled":
            msh = fb.Mesh(sh.mesh, cs)
            t0 = time.perf_counter()
            perm = msh.rcm_order()
            out["rcm_host_seconds"] = round(time.perf_counter() - t0, 4)
            del msh
            case = cm.renumber_case(sh, perm, "rcm")
        mesh = fb.Mesh(case.mesh, cs)
        conn = mesh.connectivity()
        ns = fb.NavierStokes(mesh, cs, dev)
        ns.residual(case.state)
        ns.time_residual(max(warmup, 1), True)
        t = ns.time_residual(steps, True)
        ms = float(t[0])
        out["orders"][label] = {"ms_per_step": round(ms, 5), "value": round(mesh.nf / (ms * 1e-3) / 1e6, 3),
                                "unit": UNIT,
                                "bandwidth": cm.bandwidth(conn["face_parent"], conn["face_neighbor"], conn["face_bc"]),
                                "kernels_ms": {k: round(float(v), 5) for k, v in zip(
                                    ("ghost_minmax", "grad_limiter", "outlet_density", "face_flux", "gather"), t[1:6])}}
        del ns
    return out


def run_ours(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    import freecfd_b200 as fb
    case = make_case(args.workload)
    import tempfile
    tmp = tempfile.mkdtemp(prefix="fcfd_bench_")
    cs = fb.Case(case.write_deck(tmp))
    mesh = fb.Mesh(case.mesh, cs)
    ns = fb.NavierStokes(mesh, cs, dev)
    W = np.ascontiguousarray(case.state)
    rans = case.kstate is not None
    K = np.ascontiguousarray(case.kstate) if rans else None
    if rans:
        ns.rans_residual(W, K)                   # upload + first coupled evaluation
        ns.time_rans(max(args.warmup, 1), True)
    else:
        ns.residual(W)                           # upload + first evaluation (also checks BC errors)
        ns.time_residual(max(args.warmup, 1), True)  # warm-up steps
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    # the K timed steps are repeated until the block lasts a second, so the
    # clock sampler sees the GPU under this load; the median repeat is reported
    reps = []
    with Clocks(dev) as clk:
        t_start = time.perf_counter()
        while not reps or (time.perf_counter() - t_start < 1.0 and len(reps) < 2000):
            reps.append(ns.time_rans(args.steps, True) if rans else ns.time_residual(args.steps, True))
    torch.cuda.synchronize()
    reps.sort(key=lambda r: float(r[0]))
    t = reps[len(reps) // 2]
    ms = float(t[0])
    if rans:
        kern = {"ns_part_with_eddy_viscosity": t[1], "komega_part": t[2]}
    else:
        kern = {"ghost_minmax": t[1], "grad_limiter": t[2], "outlet_density": t[3], "face_flux": t[4], "gather": t[5]}
    if dist:
        x = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(x, op=dist.ReduceOp.MAX)
        ms = float(x.item())
    value = world * mesh.nf / (ms * 1e-3) / 1e6
    # end to end through the C ABI with pinned host buffers
    Wp = torch.empty((mesh.nc, 5), dtype=torch.float64, pin_memory=True)
    Rp = torch.empty((mesh.nc, 5), dtype=torch.float64, pin_memory=True)
    Wp.numpy()[:] = W
    Wn, Rn = Wp.numpy(), Rp.numpy()
    call = (lambda: ns.rans_residual(Wn, K)) if rans else (lambda: ns.residual(Wn, Rn))
    for _ in range(max(args.warmup, 1)):
        call()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        call()
    e2e_s = (time.perf_counter() - t0) / args.steps
    if dist:
        x = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(x, op=dist.ReduceOp.MAX)
        e2e_s = float(x.item())
    e2e = world * mesh.nf / e2e_s / 1e6
    peak, kind = peaks()
    B = alg_bytes(mesh)
    achieved = B / (ms * 1e-3) / 1e9
    n_kernels = 4 + (1 if ns_has_outlet(case) else 0)
    # dominant kernel: its own algorithmic bytes over its event-timed duration
    viscous = args.workload in ("cylinder", "plate", "plate64", "plate_rans", "plate64_rans")  # viscous materials
    exact_grad = "limiter=minmod" in case.deck or "limiter=bj" in case.deck
    gi = ns.gradient_info()
    if rans:
        # coupled step: flow arrays plus k, omega (read with ghosts), their
        # residual, the eddy viscosity per cell and face
        top = "rans_step"
        kb = B + mesh.nc * 2 * 8 * 2 + (mesh.nc + mesh.nghost) * 8 + mesh.nf * 8
        k_ms = ms
        n_kernels = 11
    else:
        top = max(("grad_limiter", "face_flux", "gather", "ghost_minmax"), key=lambda k: kern[k])
        kb = kernel_bytes(mesh, top, viscous, exact_grad, fold_entries=gi["fold_entries"] if gi["kind"] == 3 else 0)
        k_ms = float(kern[top])
    k_ach = kb / (k_ms * 1e-3) / 1e9
    traffic = NCU_TRAFFIC.get((args.workload, top))
    line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 5), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(case, dict(cells=mesh.nc, faces=mesh.nf, ghosts=mesh.nghost,
                                              stencil_entries=mesh.n_grad_entries), world),
            "e2e": {"value": round(e2e, 3), "unit": UNIT,
                    "h2d_bytes_per_step": int(W.nbytes + (K.nbytes if rans else 0)),
                    "d2h_bytes_per_step": int(W.nbytes + (K.nbytes if rans else 0))},
            "roofline": {"bound": "hbm", "achieved": round(k_ach, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(k_ach / peak, 4), "traffic": traffic, "peak_kind": kind, "kernel": top,
                         "gradient_kernel": {1: "per cell", 2: "tiles", 3: "per cell, folded stencils"}[gi["kind"]],
                         "alg_bytes_per_launch": int(kb), "ms_per_launch": round(k_ms, 5)},
            "step_roofline": {"achieved": round(achieved, 1), "frac": round(achieved / peak, 4), "alg_bytes": int(B),
                              "unit_of_work": "one residual evaluation (all kernels)"},
            "kernels_ms": {k: round(float(v), 5) for k, v in kern.items()},
            "gpu_launches": n_kernels * args.steps,
            "timed_repeats": {"count": len(reps), "reported": "median repeat of K steps",
                              "ms_per_step_min": round(float(reps[0][0]), 5),
                              "ms_per_step_max": round(float(reps[-1][0]), 5)},
            "clocks": clk.summary()}
    if rank == 0 and not args.no_parity:
        line["parity_err"] = parity_check(ns, case)
    if not args.no_sublines and args.workload == "cylinder":
        line["workloads"] = [residual_subline(fb, w, dev, min(args.steps, 20), args.warmup, w != "plate64")
                             for w in ("hypersonic", "plate", "plate64")]
        if world == 1:
            line["renumbering"] = renumber_subline(fb, dev, min(args.steps, 20), args.warmup)
    if (world > 1 or args.decomposed) and args.workload == "cylinder":
        line["decomposed"] = run_decomposed(fb, world, rank, dev, dist, args.steps, args.warmup)
    if not args.no_newton and not rans:
        line["newton"] = run_newton(fb, cs, mesh, case, dev, dist)
        if args.workload == "cylinder" and world == 1:
            line["rans_newton"] = run_rans_newton(fb, dev)
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(case, args.cpu_seconds, args.ref_workers)
    if rank == 0:
        print(json.dumps(line), flush=True)
    del ns
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_decomposed(fb, world, rank, dev, dist, steps, warmup):
    """One residual of a cylinder mesh N times as deep radially (256 x 128N
    cells, weak scaling) split over the N ranks in contiguous cell ranges:
    per step the halo states are exchanged (NCCL point-to-point), the VK
    extrema all-reduced and each rank evaluates its owned rows.  Every part
    of a step is enqueued on the library context's stream without a host
    synchronisation (the BC error flag is checked once after the timed
    steps), so the steps are timed by CUDA events on that stream; max over
    ranks."""
    import tempfile

    import torch
    from freecfd_b200 import cases
    from freecfd_b200.partition import HaloPlan, PartitionedResidual
    case = cases.cylinder_case(ntheta=256, nr=128 * world)
    cs = fb.Case(case.write_deck(tempfile.mkdtemp(prefix="fcfd_dd_")))
    mesh = fb.Mesh(case.mesh, cs)
    plan = HaloPlan(mesh, cs, world)
    ns = fb.NavierStokes(mesh, cs, dev)
    W = torch.as_tensor(np.ascontiguousarray(case.state), device="cuda")
    R = torch.empty_like(W)
    res = PartitionedResidual(ns, plan, rank, W)
    for _ in range(max(warmup, 1)):
        res(R)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(res.stream)
    for _ in range(steps):
        res(R, sync=False)
    ev1.record(res.stream)
    torch.cuda.synchronize()
    res.check()
    el = ev0.elapsed_time(ev1) * 1e-3
    halo = len(plan.halo_cells(rank))
    x = torch.tensor([el, float(res.ex.bytes_per_exchange), float(halo)], device="cuda", dtype=torch.float64)
    if dist:
        dist.all_reduce(x, op=dist.ReduceOp.MAX)
    el, nbytes, halo = (float(v) for v in x.cpu())
    del res, ns
    return {"workload": f"laminar_cylinder_256x{128 * world}x1_hex_roe_viscous split in {world} contiguous ranges",
            "cells": mesh.nc, "faces": mesh.nf, "value": round(mesh.nf * steps / el / 1e6, 3), "unit": UNIT,
            "ms_per_step": round(1e3 * el / steps, 5), "scaling": "weak",
            "timing": "CUDA events on the context stream, max over ranks",
            "halo_cells_max": int(halo), "halo_bytes_received_per_step_max": int(nbytes)}


# 20 symmetric Gauss-Seidel sweeps: the fastest setting of both arms within a
# few percent in a sweep-count scan (4 to 32 sweeps) on this workload
# The metric's time is the wall time to a 1e-10 drop of the mass residual.
# The solve then continues (final tightening) until the mass, momentum and
# energy residuals have all dropped by 1e-11 (stop_all_rows): the mass
# residual alone leaves the nearly passive low-Mach temperature field less
# converged, and the tightened state is the one compared with the FP64
# reference state.
NEWTON_TIME_TOL = 1e-10
NEWTON_KW = dict(tol=1e-11, max_newton=400, cfl0=2.0, cfl_max=1e6, krylov_rtol=1e-3, precond_sweeps=20,
                 krylov_cycles=3, stop_all_rows=True)


def time_to_drop(rep, drop):
    """Wall seconds of the first Newton step whose mass residual drop is at
    or below `drop` (from the solve's per-step history)."""
    for h, t in zip(rep["history"], rep["seconds_history"]):
        if h <= drop:
            return float(t)
    return -1.0


def profile_newton(args):
    """Only the two Newton arms, capped at --profile-newton steps (a short,
    reproducible run for launch-list profiles); prints their report."""
    import torch
    import tempfile
    import freecfd_b200 as fb
    torch.cuda.set_device(0)
    case = make_case(args.workload)
    cs = fb.Case(case.write_deck(tempfile.mkdtemp(prefix="fcfd_bench_")))
    mesh = fb.Mesh(case.mesh, cs)
    NEWTON_KW["max_newton"] = int(args.profile_newton)
    print(json.dumps({"workload": case.workload, "newton": run_newton(fb, cs, mesh, case, 0, None, False)}), flush=True)


def profile_mixed(args):
    """Only residual evaluations of the hypersonic workload with a bow-shock
    jump: each repeat one FP64 residual, then one mixed-precision residual
    (a short run for kernel profiles); prints the FP64 face count."""
    import tempfile
    import freecfd_b200 as fb
    case = make_case("hypersonic")
    cs = fb.Case(case.write_deck(tempfile.mkdtemp(prefix="fcfd_bench_")))
    mesh = fb.Mesh(case.mesh, cs)
    ns = fb.NavierStokes(mesh, cs, 0)
    W = np.ascontiguousarray(load_cases().hypersonic_shock_state(case, mesh.geometry()["cell_centroid"]))
    n = 0
    for _ in range(int(args.profile_mixed)):
        ns.residual(W)
        _, n = ns.residual_mixed(W, 2.0)
    print(json.dumps({"workload": case.workload, "state": "bow_shock_jump", "fp64_faces": n}), flush=True)


def run_newton(fb, cs, mesh, case, dev, dist, reference_state=True):
    """Steady solve from the seeded state until |R_mass|/|R_mass0| <= 1e-10:
    plain FP64 (finite-difference J.v, FP64 Krylov) against mixed (tangent
    J.v kernels evaluated in FP32, FP32 Krylov basis, FP32 Gauss-Seidel
    preconditioner; FP64 outer residual, dot products and Gram-Schmidt).  Wall time of the whole call (host state in, host state out);
    replicas under torchrun, max over ranks."""
    import torch
    out = {}
    states = {}
    variants = (("plain_fp64_fd", dict(jvp=False)),
                ("mixed_jvp_fp32", dict(jvp=True, fp32_jvp=True, fp32_krylov=True)))
    for label, opts in variants:
        ns = fb.NavierStokes(mesh, cs, dev)
        ns.newton_solve(case.state, **dict(NEWTON_KW, max_newton=2), raise_on_fail=False, **opts)  # warm-up
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        # two timed solves from the same seeded state (identical iterations);
        # the faster is reported, both are listed (host-side launch and
        # synchronisation noise differs between boxes)
        runs, runs_tol = [], []
        for _ in range(2 if NEWTON_KW["max_newton"] > 10 else 1):
            t0 = time.perf_counter()
            W, rep = ns.newton_solve(case.state, **NEWTON_KW, raise_on_fail=False, **opts)
            el = time.perf_counter() - t0
            el_tol = time_to_drop(rep, NEWTON_TIME_TOL)
            if dist:
                x = torch.tensor([el, el_tol], device="cuda", dtype=torch.float64)
                dist.all_reduce(x, op=dist.ReduceOp.MAX)
                el, el_tol = (float(v) for v in x.cpu())
            runs.append(round(el, 4))
            runs_tol.append(round(el_tol, 4))
        el = min(runs)
        states[label] = W
        out[label] = {"seconds_to_mass_1e-10": min(runs_tol), "seconds_to_mass_1e-10_runs": runs_tol,
                      "seconds_with_tightening": round(el, 4), "seconds_runs": runs, "converged": rep["status"] == 0,
                      "newton_iterations": rep["newton_iterations"], "krylov_iterations": rep["krylov_iterations"],
                      "mass_residual_drop": float(rep["res_final"] / rep["res0"]),
                      "final_drop_mass_momentum_energy": [float(x) for x in rep["rows_final"]]}
        if "type=wall;" in case.deck and case.name == "cylinder":
            # drag coefficient of the wall (BC_1): Fx / (0.5 rho U^2 D span), D = 1
            F, _ = ns.drag(W, [0], (1.0, 0.0, 0.0), gradient=False)
            p, U, T = case.freestream[0], case.freestream[1], case.freestream[4]
            rho = p / (287.0 * T)
            span = float(np.ptp(case.mesh.nodes[:, 2]))
            out[label]["drag_coefficient"] = float(F[0] / (0.5 * rho * U * U * 1.0 * span))
        del ns
    a, b = states["plain_fp64_fd"], states["mixed_jvp_fp32"]
    scale = np.abs(a).max(axis=0)
    scale[1:4] = np.abs(a[:, 1:4]).max()
    out["speedup_mixed_vs_plain"] = round(
        out["plain_fp64_fd"]["seconds_to_mass_1e-10"] / out["mixed_jvp_fp32"]["seconds_to_mass_1e-10"], 3)
    out["speedup_mixed_vs_plain_with_tightening"] = round(
        out["plain_fp64_fd"]["seconds_with_tightening"] / out["mixed_jvp_fp32"]["seconds_with_tightening"], 3)
    out["state_rel_diff_mixed_vs_plain"] = float((np.abs(a - b).max(axis=0) / scale).max())
    if "drag_coefficient" in out["plain_fp64_fd"]:
        cp, cm = out["plain_fp64_fd"]["drag_coefficient"], out["mixed_jvp_fp32"]["drag_coefficient"]
        out["drag_coefficient_rel_diff_mixed_vs_plain"] = abs(cm - cp) / abs(cp)
    # untimed: the plain arm continued to 1e-3 of its final residual (the
    # discrete steady state to round-off) as the FP64 reference state; the
    # error of each arm's 1e-10 state against it, per variable, relative to the
    # variable's magnitude (velocity components share one scale)
    if reference_state:
        ns = fb.NavierStokes(mesh, cs, dev)
        ref, rep = ns.newton_solve(a, **dict(NEWTON_KW, tol=1e-3, cfl0=1e6, max_newton=60), raise_on_fail=False,
                                   jvp=False)
        del ns
        out["fp64_reference_state"] = {"mass_residual_drop": float(out["plain_fp64_fd"]["mass_residual_drop"]
                                                                   * rep["res_final"] / rep["res0"]),
                                       "newton_iterations": rep["newton_iterations"]}
        # the reference state checked in the oracle's (the reference's) own
        # discretisation: its residual norm per equation over the seeded
        # state's
        import oracle
        o = oracle.Oracle(case)
        r_ref, r_0 = o.residual(ref), o.residual(case.state)
        o.close()
        out["fp64_reference_state"]["oracle_residual_drop"] = [
            float(np.linalg.norm(r_ref[:, v]) / max(np.linalg.norm(r_0[:, v]), 1e-300)) for v in range(5)]
        for label, W in states.items():
            err = np.abs(W - ref).max(axis=0) / scale
            out[label]["state_rel_err_vs_fp64_reference"] = dict(zip(("p", "u", "v", "w", "T"), map(float, err)))
    out["settings"] = dict(NEWTON_KW)
    return out


# coupled flow + k-omega Newton-Krylov on the turbulent plate: SER on the
# largest per-equation drop, k and omega clipped at their lower limits
RANS_NEWTON_KW = dict(tol=1e-10, max_newton=400, cfl0=1.0, cfl_max=1e6, krylov_dim=40, krylov_rtol=1e-2,
                      cfl_mode=2, stop_all_rows=True)


def run_rans_newton(fb, dev):
    """Config 5 (k-omega flat plate 384x192x4): the coupled Newton solve from
    the seeded state with FP64 finite-difference J.v (plain) and with the
    FP32 coupled tangent chain (mixed), the same settings and step cap; wall
    time, per-equation residual drops, and the skin-friction drag coefficient
    of the no-slip wall (BC_3) of each arm."""
    import tempfile
    case = make_case("plate_rans")
    cs = fb.Case(case.write_deck(tempfile.mkdtemp(prefix="fcfd_bench_")))
    mesh = fb.Mesh(case.mesh, cs)
    p, U, T = case.freestream[0], case.freestream[1], case.freestream[4]
    rho = p / (287.0 * T)
    nodes = case.mesh.nodes
    span = float(np.ptp(nodes[:, 2]))
    out, states = {}, {}
    for label, kw in (("plain_fp64_fd", {}), ("mixed_jvp_fp32", dict(fp32_jvp=True))):
        ns = fb.NavierStokes(mesh, cs, dev)
        t0 = time.perf_counter()
        W, K, rep = ns.rans_newton_solve(case.state, case.kstate, raise_on_fail=False, **RANS_NEWTON_KW, **kw)
        el = time.perf_counter() - t0
        F, _ = ns.drag(W, [2], (1.0, 0.0, 0.0), gradient=False)
        cf = float(F[0] / (0.5 * rho * U * U * 2.0 * span))
        states[label] = (W, K)
        out[label] = {"seconds": round(el, 3), "converged": rep["status"] == 0, "newton_iterations": rep["newton_iterations"],
                      "krylov_iterations": rep["krylov_iterations"],
                      "final_drop_mass_momentum_energy": [float(v) for v in rep["rows_final"]],
                      "final_drop_k_omega": [float(v) for v in rep["kw_final"]],
                      "skin_friction_drag_coefficient": cf}
        del ns
    (Wa, Ka), (Wb, Kb) = states["plain_fp64_fd"], states["mixed_jvp_fp32"]
    out["state_rel_diff_mixed_vs_plain"] = float(max((np.abs(Wa - Wb).max(axis=0) / np.abs(Wa).max(axis=0)).max(),
                                                    (np.abs(Ka - Kb).max(axis=0) / np.abs(Ka).max(axis=0)).max()))
    ca, cb = out["plain_fp64_fd"]["skin_friction_drag_coefficient"], out["mixed_jvp_fp32"]["skin_friction_drag_coefficient"]
    out["skin_friction_rel_diff_mixed_vs_plain"] = abs(cb - ca) / abs(ca)
    out["speedup_mixed_vs_plain"] = round(out["plain_fp64_fd"]["seconds"] / out["mixed_jvp_fp32"]["seconds"], 3)
    out["workload"] = case.workload
    out["settings"] = dict(RANS_NEWTON_KW)
    return out


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) from
# ncu captures of the same kernels; the capture commands are in profiles/.
NCU_TRAFFIC = {
    ("cylinder", "grad_limiter"): 17764096, ("cylinder", "face_flux"): 20554752,
    ("hypersonic", "grad_limiter"): 191846912, ("hypersonic", "face_flux"): 141227264,
    ("plate", "grad_limiter"): 155463936, ("plate", "face_flux"): 196130048,
}


def ns_has_outlet(case):
    return "type=outlet" in case.deck


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cylinder", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-workers", type=int, default=64)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-newton", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the untimed oracle check of the timed workload")
    ap.add_argument("--no-sublines", action="store_true",
                    help="skip the residual lines of the hypersonic, plate and plate64 workloads")
    ap.add_argument("--decomposed", action="store_true",
                    help="also time the domain-decomposed residual (always on under torchrun)")
    ap.add_argument("--profile-newton", type=int, default=0,
                    help="run only the two Newton arms, capped at this many Newton steps")
    ap.add_argument("--profile-mixed", type=int, default=0,
                    help="run only this many FP64 + mixed-precision residual pairs of the hypersonic workload")
    args = ap.parse_args()
    if args.profile_newton > 0:
        profile_newton(args)
    elif args.profile_mixed > 0:
        profile_mixed(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
