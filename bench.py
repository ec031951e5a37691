#!/usr/bin/env python3
"""Benchmark: global residual + Jacobian assembly of plane-stress Lagrange quads on B200.

Default workload: 1024x1024 order-3 quads on a 10x10 square (+-0.2h interior
perturbation, u in [-1e-3,1e-3], E=70e9, nu=0.3, 4x4 Gauss points; 18,886,658 DOF,
235,960,321 2x2 blocks).  One step = one complete residual + Jacobian assembly.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Prints one JSON line (rank 0).  `value` is elements/s of the plain FP64 plan
assembly (the reference's arithmetic) with device-resident inputs; `e2e` is the
same metric through the public API with a host->device copy of the state and a
device->host copy of the residual inside every timed step.  The MIXED-precision
form, the other paths (each timed for at least one second), a batched leg
(meshes of the many-mesh configuration in one captured graph) and a served leg
(Newton clients through the server at a fixed request rate) ride along as
sub-objects.  Multi-GPU runs are independent replicas (the assembly of one mesh
is not sharded).  --impl reference times the reference's own CPU assembly
(element/FEKernels.h compiled as oracle/_ref) on a bounded sample of the same
mesh with all host threads; it loads nothing from the library.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import pathlib
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    "square1024_p3": dict(kind="square", n=1024, p=3),
    "square512_p3": dict(kind="square", n=512, p=3),
    "square2048_p1": dict(kind="square", n=2048, p=1),
    "square1024_p2": dict(kind="square", n=1024, p=2),
    "square512_p4": dict(kind="square", n=512, p=4),
    "square64_p1": dict(kind="square64"),
    "annulus512x2048_p2": dict(kind="annulus"),
}


def make_mesh(mesh_mod, name):
    """The named workload from the package's mesh generator (pure numpy)."""
    w = WORKLOADS[name]
    if w["kind"] == "square64":
        return mesh_mod.square64_p1()
    if w["kind"] == "annulus":
        return mesh_mod.annulus512x2048_p2()
    if w["p"] == 3:
        return mesh_mod.square1024_p3(w["n"])
    return mesh_mod.square_mesh(w["n"], w["n"], w["p"], 1.0, 1.0, 0.1, 1e-3, 70e9, 0.3, 1.0, 0x5EED0006,
                                f"square{w['n']}_p{w['p']}")


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per assembly from ncu
# captures, keyed by workload, kernel label prefix and element layout.  The 1024^2
# order-3 figures are the sums over the four colour launches of the 512^2 case
# (colour layout 2.835 GB, the FP64 and BF16x6 kernels moving the same bytes; pair
# layout 2.592 GB) times 4: traffic grows with the element count.
MEASURED_TRAFFIC = {
    ("square1024_p3", "frag_kernel<3", "colours"): 4 * 2.835e9,
    ("square1024_p3", "frag_kernel<3>", "pairs"): 4 * 2.5917e9,
}


def algorithmic_bytes(mesh, nnzb):
    """Minimal HBM bytes of one residual+Jacobian assembly: read coords and states,
    read conn, write the residual and the BSR values once."""
    return 16 * mesh.num_nodes * 2 + 4 * mesh.num_elements * mesh.nodes_per_element + 16 * mesh.num_nodes + 32 * nnzb


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.dev)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]
        return False

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        load = [s for s in sm if s > 0.5 * (mx or max(sm))] or sm
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    """Replica ranks from the torchrun environment (one mesh per GPU, no sharding)."""
    import fem_pkg
    rep = fem_pkg.load_module("replicas")
    return rep.init_from_env("nccl" if args.impl == "ours" else "gloo")


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def log(msg):
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


# ----------------------------------------------------------------------------------------
def reference_sample(mesh_mod, orc, args):
    """The bounded CPU sample of the workload: its first elements, with the pattern
    and element map from the oracle's own builders (nothing from the library)."""
    mesh = make_mesh(mesh_mod, args.workload)
    sample = min(mesh.num_elements, args.ref_elements or 131072)
    sub = mesh_mod.submesh(mesh, 0, sample)
    rowp, cols = orc.bsr_pattern(sub.num_nodes, sub.conn_ptr, sub.conn)
    mp = orc.element_bsr_map(sub.conn_ptr, sub.conn, sub.nodes_per_element, rowp, cols)
    return mesh, sub, mp, int(cols.size)


def reference_assembler(orc, threads):
    """(kind, description, fn(sub, map, nnzb)) for the CPU baseline: the reference's
    own CPU assembly compiled with OpenMP (oracle/_ref/libfemref_omp.so) when it was
    built from the reference checkout, else the oracle port."""
    omp = ROOT / "oracle" / "_ref" / "libfemref_omp.so"
    if omp.exists():
        import ctypes as C
        lib = C.CDLL(str(omp))
        p, i, d = C.c_void_p, C.c_int, C.c_double
        lib.ref_run_jacobian.argtypes = [i, p, p, i, p, p, d, d, d, p, p, p]
        lib.ref_run_jacobian.restype = d
        lib.ref_set_num_threads.argtypes = [i]
        lib.ref_set_num_threads(threads)

        def run(sub, mp, nnzb):
            res = np.zeros(sub.num_nodes * 2)
            mat = np.zeros(nnzb * 4)
            cp, cn = np.ascontiguousarray(sub.conn_ptr, np.int32), np.ascontiguousarray(sub.conn, np.int32)
            st, xy = np.ascontiguousarray(sub.states), np.ascontiguousarray(sub.coords)
            lib.ref_run_jacobian(sub.order, cp.ctypes.data, cn.ctypes.data, sub.num_elements, st.ctypes.data,
                                 xy.ctypes.data, sub.E, sub.nu, sub.t, mp.ctypes.data, res.ctypes.data,
                                 mat.ctypes.data)

        return "reference", ("runJacobianKernel host build (element/FEKernels.h compiled from the reference "
                             "checkout, OpenMP over elements as written; A2D interface restated)"), run
    orc.set_threads(threads)
    return "port", "oracle restatement (OpenMP, atomic scatter)", (
        lambda sub, mp, nnzb: orc.assemble(sub, mp, nnzb, parallel=True))


def run_reference(args):
    """The reference's CPU assembly on a bounded sample, all host threads; rank 0 only."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if int(os.environ.get("RANK", "0")) != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import fem_pkg
    import oracle as orc
    mesh_mod = fem_pkg.load_module("mesh")
    if args.ref_elements is None:  # each step a bounded sample: about 20 x 131072 elements in all
        args.ref_elements = max(32768, min(131072, 131072 * 20 // max(1, args.steps)))
    mesh, sub, mp, nnzb = reference_sample(mesh_mod, orc, args)
    threads = os.cpu_count() or 1
    kind, what, run = reference_assembler(orc, threads)
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        run(sub, mp, nnzb)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    tot = sum(times)
    value = sub.num_elements * len(times) / tot
    line = {
        "impl": "reference", "metric": "assembled elements/s (res+Jac)", "value": value, "unit": "elements/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "order": mesh.order, "sample_elements": sub.num_elements,
                   "note": "each step assembles a bounded sample of the workload (its first elements); "
                           "elements/s is a per-element rate"},
        "cpu_baseline": {"value": value, "unit": "elements/s", "cores": threads, "kind": kind,
                         "sample": f"first {sub.num_elements} elements of {mesh.name}: {what}"},
        "e2e": {"value": value, "unit": "elements/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(mesh_mod, args):
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc
    mesh, sub, mp, nnzb = reference_sample(mesh_mod, orc, args)
    threads = os.cpu_count() or 1
    kind, what, run = reference_assembler(orc, threads)
    run(sub, mp, nnzb)
    t0 = time.perf_counter()
    reps = 0
    while True:
        run(sub, mp, nnzb)
        reps += 1
        if time.perf_counter() - t0 > args.cpu_seconds:
            break
    dt = (time.perf_counter() - t0) / reps
    return {"value": sub.num_elements / dt, "unit": "elements/s", "cores": threads, "kind": kind,
            "sample": f"first {sub.num_elements} elements of {mesh.name}, {reps} repeats: {what}"}


# ----------------------------------------------------------------------------------------
class Timer:
    """CUDA-event timing on one stream; max over ranks."""

    def __init__(self, stream, pg, dev):
        import fem_pkg
        self.stream, self.pg, self.dev = stream, pg, dev
        self.rep = fem_pkg.load_module("replicas")

    def steps(self, fn, steps, warmup):
        """ms per step over exactly `steps` steps after `warmup` untimed ones."""
        import torch
        for _ in range(warmup):
            fn()
        self.stream.synchronize()
        self.rep.barrier(self.pg)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(self.stream)
        for _ in range(steps):
            fn()
        ev1.record(self.stream)
        ev1.synchronize()
        return self.rep.max_over_ranks(ev0.elapsed_time(ev1) / steps, self.pg, self.dev)

    def window(self, fn, min_seconds=1.0, warmup=3, max_steps=20000):
        """(ms per step, steps) over a timed region of at least min_seconds."""
        est = self.steps(fn, 3, warmup)
        n = int(min(max_steps, max(5, math.ceil(min_seconds * 1e3 / max(est, 1e-3)))))
        n = int(self.rep.max_over_ranks(n, self.pg, self.dev))
        return self.steps(fn, n, 1), n


def run_ours(args):
    import torch
    world, rank, local, pg = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import fem_pkg
    fem = fem_pkg.load()
    mesh = make_mesh(fem.mesh, args.workload)
    stream = torch.cuda.Stream(device=dev)
    sptr = stream.cuda_stream
    with torch.cuda.stream(stream):
        d = fem.DeviceMesh(mesh, dev)
        plan = fem.Plan(mesh.order, mesh.num_nodes, mesh.conn_ptr, mesh.conn)
        nnzb = plan.nnzb
        res = torch.empty(mesh.num_nodes * 2, dtype=torch.float64, device=dev)
        mat = torch.empty(nnzb * 4, dtype=torch.float64, device=dev)
    stream.synchronize()
    E, nu, t = mesh.E, mesh.nu, mesh.t
    nE = mesh.num_elements
    T = Timer(stream, pg, dev)
    rate = lambda ms: world * nE / (ms * 1e-3)  # noqa: E731

    def assemble(prec="fp64", strain="linear", r=res, m=mat):
        plan.assemble(d.states, d.coords, E, nu, t, r, m, precision=prec, strain=strain, stream=sptr)

    if args.profile_run:
        # a short run for ncu captures: only the launches of the chosen path
        fn = {"jacobian": assemble, "mixed": lambda: assemble("mixed"),
              "residual": lambda: plan.assemble(d.states, d.coords, E, nu, t, res, None, stream=sptr)}[args.profile_path]
        log(f"{args.profile_path} {T.steps(fn, args.steps, args.warmup):.3f} ms")
        plan.close()
        if pg is not None:
            pg.destroy_process_group()
        return

    # headline: FP64 plan assembly, exactly K steps after W warm-up steps
    with ClockSampler(local) as clk:
        ms = T.steps(assemble, args.steps, args.warmup)
    value = rate(ms)
    launches = plan.launches() * args.steps
    log(f"plan fp64 {ms:.3f} ms")

    # end to end through the public API: pinned host state -> device, assemble, residual
    # -> pinned host, in one fem_plan_assemble_host call (state upload in node chunks,
    # band-split colour launches, residual download per chunk, all overlapped)
    h_states = torch.from_numpy(np.ascontiguousarray(mesh.states)).pin_memory()
    h_res = torch.empty(mesh.num_nodes * 2, dtype=torch.float64).pin_memory()
    h2d, d2h = h_states.numel() * 8, h_res.numel() * 8

    def e2e_step(prec="fp64"):
        plan.assemble_host(h_states, d.states, d.coords, E, nu, t, h_res, res, mat, precision=prec, bands=args.bands,
                           stream=sptr)

    def e2e_serial_step(prec="fp64"):
        d.states.copy_(h_states, non_blocking=True)
        assemble(prec)
        h_res.copy_(res, non_blocking=True)

    with torch.cuda.stream(stream):
        ms_e2e = T.steps(e2e_step, args.steps, args.warmup)
        ms_e2e_serial, _ = T.window(e2e_serial_step)
    ms_piped = pipelined(T, fem, plan, d, mesh, res, h_states, h_res, args, dev, stream)

    # every path timed over at least one second
    paths = {}

    def path(name, fn, **extra):
        with torch.cuda.stream(stream):
            pms, n = T.window(fn, args.min_seconds)
        paths[name] = {"ms": pms, "elements_per_s": rate(pms), "timed_steps": n, **extra}
        log(f"{name} {pms:.3f} ms ({n} steps)")
        return pms

    path("plan_fp64", assemble)
    layout = plan.layout()
    if layout[0] == "pairs":
        # the same launches with the element colouring (what batches and the server run)
        plan.set_layout("colours")
        path("plan_fp64_colour_layout", assemble)
        plan.set_layout("pairs")
    ms_mixed = path("plan_mixed", lambda: assemble("mixed"))
    path("plan_fp64_nonlinear", lambda: assemble("fp64", "nonlinear"))
    path("plan_fp64_residual_only", lambda: plan.assemble(d.states, d.coords, E, nu, t, res, None, stream=sptr))
    err = mixed_error(plan, d, mesh, res, mat, stream, sptr)
    with torch.cuda.stream(stream):
        ms_e2e_mixed, _ = T.window(lambda: e2e_step("mixed"), args.min_seconds)
    # plain drop-in FP64 (reference contract: caller zeroes, kernel accumulates via map)
    rowp_h, cols_h = plan.pattern()
    mp = fem.build_element_bsr_map(mesh.conn_ptr, mesh.conn, mesh.nodes_per_element, rowp_h, cols_h)
    with torch.cuda.stream(stream):
        dmap = torch.from_numpy(mp).to(dev)
    del mp, rowp_h, cols_h

    def dropin(zero=True):
        if zero:
            res.zero_()
            mat.zero_()
        fem.run_jacobian_kernel(mesh.order, d.conn_ptr, d.conn, nE, d.states, d.coords, E, nu, t, dmap, res, mat,
                                stream=sptr, timed=False)

    def dropin_residual():
        res.zero_()
        fem.run_residual_kernel(mesh.order, d.conn_ptr, d.conn, nE, d.states, d.coords, E, nu, t, res, stream=sptr,
                                timed=False)

    path("dropin_fp64_with_zeroing", dropin)
    path("dropin_fp64_kernel_only", lambda: dropin(False))
    path("dropin_fp64_residual_with_zeroing", dropin_residual)
    del dmap
    torch.cuda.synchronize(dev)

    hbm, peak_kind = peaks()
    abytes = algorithmic_bytes(mesh, nnzb)
    label = kernel_label(plan, mesh.order, "fp64")
    traffic = next((v for (w, k, lay), v in MEASURED_TRAFFIC.items()
                    if w == mesh.name and label.startswith(k) and label.endswith(f"({lay} layout)")), None)
    achieved = abytes / (ms * 1e-3) / 1e9
    line = {
        "metric": "assembled elements/s (res+Jac)", "value": value, "unit": "elements/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": mesh.name, "order": mesh.order, "elements": nE, "dof": mesh.num_dof, "nnzb": nnzb,
                   "path": "plan_fp64", "layout": {"order": layout[0], "pairs": layout[1], "colours": layout[2]},
                   "l2": "inputs and outputs larger than L2 (BSR values %.2f GB)" % (32 * nnzb / 1e9),
                   "parallelism": f"replicas{world}"},
        "dof_per_s": value * mesh.num_dof / nE,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": traffic, "peak_kind": peak_kind, "algorithmic_bytes_per_step": abytes, "kernel": label,
                     "traffic_note": ("DRAM bytes per step (all colour launches of one assembly) from an ncu capture "
                                      "of the 512^2 order-3 mesh scaled x4; above the algorithmic bytes: later "
                                      "colours' bulk reductions read the blocks an earlier colour stored"
                                      if traffic else "no ncu capture for this workload")},
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "e2e": {"value": rate(ms_e2e), "unit": "elements/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": ms_e2e,
                "api": (f"fem_plan_assemble_host, {args.bands} bands (copies overlapped with the assembly); the "
                        f"matrix ({32 * nnzb / 1e9:.2f} GB) stays on the device for a device solver -- a host "
                        f"consumer of the matrix would add that D2H per assembly"),
                "serial": {"value": rate(ms_e2e_serial), "ms_per_step": ms_e2e_serial,
                           "note": "state upload, fem_plan_assemble, residual download in sequence"},
                "pipelined": {"value": rate(ms_piped), "ms_per_step": ms_piped,
                              "note": "independent load cases: case k+1 uploads and case k-1 downloads "
                                      "while case k assembles (3 streams, 2 buffers); same copies per step"}},
        "mixed": {"value": rate(ms_mixed), "ms_per_step": ms_mixed, "dtype": mixed_dtype(mesh.order),
                  "kernel": kernel_label(plan, mesh.order, "mixed"), "rel_frobenius_err_vs_fp64": err,
                  "e2e": {"value": rate(ms_e2e_mixed), "ms_per_step": ms_e2e_mixed}},
        "paths": paths,
    }
    plan.close()
    del res, mat, d
    torch.cuda.synchronize(dev)
    torch.cuda.empty_cache()
    if rank == 0 and world == 1 and not args.no_legs:
        plain = paths["dropin_fp64_with_zeroing"]["elements_per_s"]
        line["batched"] = batch_leg(fem, dev, args, plain)
        line["served"] = serve_leg(fem, dev, args)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(fem.mesh, args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


def pipelined(T, fem, plan, d, mesh, res, h_states, h_res, args, dev, stream):
    """ms per load case when independent cases stream through the GPU: case k+1's
    state upload and case k-1's residual download overlap case k's assembly."""
    import torch
    sptr = stream.cuda_stream
    s_in, s_out = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    with torch.cuda.stream(stream):
        st2 = [d.states, torch.empty_like(d.states)]
        rs2 = [res, torch.empty_like(res)]
        mat = torch.empty(plan.nnzb * 4, dtype=torch.float64, device=dev)
    hs2 = [h_states, h_states.clone().pin_memory()]
    hr2 = [h_res, torch.empty_like(h_res).pin_memory()]
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_comp = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]
    for e in ev_comp + ev_out:
        e.record(stream)

    def piped_step(k):
        b = k % 2
        s_in.wait_event(ev_comp[b])  # buffer b's previous assembly has read its state
        with torch.cuda.stream(s_in):
            st2[b].copy_(hs2[b], non_blocking=True)
        ev_in[b].record(s_in)
        stream.wait_event(ev_in[b])
        stream.wait_event(ev_out[b])  # residual buffer b has been downloaded
        plan.assemble(st2[b], d.coords, mesh.E, mesh.nu, mesh.t, rs2[b], mat, stream=sptr)
        ev_comp[b].record(stream)
        s_out.wait_event(ev_comp[b])
        with torch.cuda.stream(s_out):
            hr2[b].copy_(rs2[b], non_blocking=True)
        ev_out[b].record(s_out)

    for k in range(args.warmup):
        piped_step(k)
    torch.cuda.synchronize(dev)
    T.rep.barrier(T.pg)
    steps = max(args.steps, 100)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(s_in)
    for k in range(steps):
        piped_step(k)
    s_in.wait_event(ev_out[0])
    s_in.wait_event(ev_out[1])
    p1.record(s_in)
    p1.synchronize()
    ms = T.rep.max_over_ranks(p0.elapsed_time(p1) / steps, T.pg, dev)
    torch.cuda.synchronize(dev)
    return ms


def mixed_error(plan, d, mesh, res, mat, stream, sptr):
    """Relative Frobenius error of the MIXED plan outputs against the FP64 ones."""
    import torch
    with torch.cuda.stream(stream):
        plan.assemble(d.states, d.coords, mesh.E, mesh.nu, mesh.t, res, mat, precision="fp64", stream=sptr)
        res64, mat64 = res.clone(), mat.clone()
        plan.assemble(d.states, d.coords, mesh.E, mesh.nu, mesh.t, res, mat, precision="mixed", stream=sptr)
        out = {"residual": float(torch.linalg.vector_norm(res - res64) / torch.linalg.vector_norm(res64)),
               "jacobian": float(torch.linalg.vector_norm(mat - mat64) / torch.linalg.vector_norm(mat64))}
    stream.synchronize()
    return out


def mixed_dtype(order):
    return {1: "f64", 2: "f64", 3: "bf16x6/f64", 4: "f32/f64"}[order]


def kernel_label(plan, order, prec):
    """The kernel that runs one assembly of `plan` (the dispatch of fem_plan_assemble)."""
    if plan.row_chunks > 0:
        return "rows_p1_kernel, 1 launch per step"
    # the fragment kernel serves orders 2-3 in both precisions (MIXED at order 3 with
    # its element stiffness as BF16x6 tensor-core products, at order 2 in FP64) and
    # order 4 in FP64; FP32 order 4 runs the element kernel
    n = plan.launches(precision=prec)
    lay = plan.layout()[0]
    if order == 3 and prec == "mixed":
        return f"frag_kernel<{order}, BF16x6 stiffness> x {n} colour launches per step ({lay} layout)"
    if order in (2, 3) or (order == 4 and prec == "fp64"):
        return f"frag_kernel<{order}> x {n} colour launches per step ({lay} layout)"
    return f"assemble_kernel<{order}, float> x {plan.num_colours} colour launches per step"


# ----------------------------------------------------------------------------------------
def mesh_bytes(spec, with_map=True):
    """Device bytes of one batched mesh: plan topology, coordinates/states/residual,
    BSR values and (for the single-mesh comparison) the reference element map."""
    n = (spec.order + 1) ** 2
    N, ne, nnzb = spec.num_nodes(), spec.num_elements, spec.nnzb()
    plan = 4 * (N + 1) + 4 * nnzb + 4 * ne * n + ne * n * n + ne * n
    data = 16 * N * 3 + 4 * ne * n + 4 * (ne + 1) + 32 * nnzb
    return plan + data + (4 * ne * n * n if with_map else 0)


def waves_of(specs, budget_bytes):
    waves, cur, used = [], [], 0
    for sp in specs:
        b = mesh_bytes(sp)
        if cur and used + b > budget_bytes:
            waves.append(cur)
            cur, used = [], 0
        cur.append(sp)
        used += b
    if cur:
        waves.append(cur)
    return waves


def batched_measure(fem, dev, waves, steps, warmup, precisions):
    """Each wave: plans, one tuned and captured graph per precision, replays timed
    with CUDA events; the plain FP64 drop-in (zero the outputs, fem_run_jacobian per
    mesh) on the same meshes; the MIXED error against FP64 on the first meshes."""
    import torch
    stream = torch.cuda.Stream(device=dev)
    sptr = stream.cuda_stream
    out = {"elements": 0, "ms": {p: 0.0 for p in precisions}, "ms_plain": 0.0, "launches": {p: 0 for p in precisions},
           "tiles": {p: [] for p in precisions}, "kernels": {p: [] for p in precisions},
           "ordered": {p: [] for p in precisions}, "errs": [],
           "wave_ms": {p: [] for p in precisions}}

    def ev_time(fn, reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    for wave in waves:
        meshes = [sp.build() for sp in wave]
        plans = [fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn) for m in meshes]
        with torch.cuda.stream(stream):
            devs = [fem.DeviceMesh(m, dev) for m in meshes]
            res = [torch.empty(m.num_nodes * 2, dtype=torch.float64, device=dev) for m in meshes]
            mat = [torch.empty(p.nnzb * 4, dtype=torch.float64, device=dev) for p in plans]
        stream.synchronize()
        for prec in precisions:
            batch = fem.Batch(plans)
            for i, (m, dm) in enumerate(zip(meshes, devs)):
                batch.bind(i, dm.states, dm.coords, m.E, m.nu, m.t, res[i], mat[i])
            batch.tune(precision=prec, stream=sptr, reps=2)
            out["tiles"][prec].append(batch.info()["tile_batches"])
            out["kernels"][prec].append(batch.kernels(prec))
            out["ordered"][prec].append(batch.ordered())
            batch.capture(precision=prec, stream=sptr)
            for _ in range(warmup):
                batch.replay(stream=sptr)
            ms = ev_time(lambda: batch.replay(stream=sptr), steps)
            out["ms"][prec] += ms
            out["wave_ms"][prec].append(ms)
            out["launches"][prec] += batch.info()["launches"] * steps
            if prec == "mixed":
                with torch.cuda.stream(stream):
                    keep = [(r.clone(), a.clone()) for r, a in zip(res[:8], mat[:8])]
                    b64 = fem.Batch(plans)
                    for i, (m, dm) in enumerate(zip(meshes, devs)):
                        b64.bind(i, dm.states, dm.coords, m.E, m.nu, m.t, res[i], mat[i])
                    b64.assemble(precision="fp64", stream=sptr)
                    for (r, a), r64, a64 in zip(keep, res[:8], mat[:8]):
                        out["errs"].append(max(
                            float(torch.linalg.vector_norm(r - r64) / torch.linalg.vector_norm(r64)),
                            float(torch.linalg.vector_norm(a - a64) / torch.linalg.vector_norm(a64))))
                    stream.synchronize()
                    b64.close()
                del keep
            batch.close()
        maps = []
        for m, p in zip(meshes, plans):
            rowp, cols = p.pattern()
            mp = fem.build_element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)
            with torch.cuda.stream(stream):
                maps.append(torch.from_numpy(mp).to(dev))

        def plain():
            for m, dm, r, a, mp in zip(meshes, devs, res, mat, maps):
                r.zero_()
                a.zero_()
                fem.run_jacobian_kernel(m.order, dm.conn_ptr, dm.conn, m.num_elements, dm.states, dm.coords, m.E,
                                        m.nu, m.t, mp, r, a, stream=sptr, timed=False)

        with torch.cuda.stream(stream):
            plain()
            out["ms_plain"] += ev_time(plain, max(1, steps // 2))
        out["elements"] += sum(m.num_elements for m in meshes)
        for p in plans:
            p.close()
        del meshes, plans, devs, res, mat, maps
        torch.cuda.synchronize(dev)
        torch.cuda.empty_cache()
    return out


def batch_leg(fem, dev, args, plain_single):
    """The batched configuration in the default run: the first meshes of the
    256-mesh mix (element counts log-uniform in [1e3, 1e6], orders 1-4) that fit
    args.leg_batch_gb, one wave, FP64 and MIXED graphs, against the plain FP64
    drop-in on the same meshes."""
    t0 = time.perf_counter()
    specs = fem.batch_specs(count=256)
    budget = args.leg_batch_gb * 1e9
    chosen, used = [], 0
    for sp in specs:
        b = mesh_bytes(sp)
        if used + b > budget:
            continue
        chosen.append(sp)
        used += b
    r = batched_measure(fem, dev, [chosen], args.leg_steps, 3, ("fp64", "mixed"))
    el = r["elements"]
    per_order = {p: sum(s.num_elements for s in chosen if s.order == p) for p in (1, 2, 3, 4)}
    log(f"batched leg {time.perf_counter() - t0:.1f} s")
    return {
        "workload": (f"{len(chosen)} of the 256 meshes (element counts log-uniform in [1e3, 1e6], orders 1-4), "
                     f"first in draw order within {args.leg_batch_gb:g} GB, one captured graph per precision"),
        "meshes": len(chosen), "elements": el, "elements_per_order": per_order,
        "fp64": {"elements_per_s": el / (r["ms"]["fp64"] * 1e-3), "ms_per_step": r["ms"]["fp64"],
                 "tuned_tile_batches": r["tiles"]["fp64"][0], "tuned_kernels": r["kernels"]["fp64"][0],
                 "tuned_ordered": r["ordered"]["fp64"][0]},
        "mixed": {"elements_per_s": el / (r["ms"]["mixed"] * 1e-3), "ms_per_step": r["ms"]["mixed"],
                  "tuned_tile_batches": r["tiles"]["mixed"][0], "tuned_kernels": r["kernels"]["mixed"][0],
                  "tuned_ordered": r["ordered"]["mixed"][0],
                  "rel_frobenius_err_vs_fp64_max": max(r["errs"]) if r["errs"] else None},
        "plain_fp64_dropin_same_meshes": {"elements_per_s": el / (r["ms_plain"] * 1e-3), "ms_per_step": r["ms_plain"],
                                          "note": "zero the outputs, fem_run_jacobian per mesh"},
        "batched_over_plain": {"fp64": r["ms_plain"] / r["ms"]["fp64"], "mixed": r["ms_plain"] / r["ms"]["mixed"]},
        "mixed_over_plain_single_mesh_headline": (el / (r["ms"]["mixed"] * 1e-3)) / plain_single,
        "timed_steps": args.leg_steps, "gpu_launches": r["launches"],
    }


def serve_sweep(fem, srv, ids, meshes, states, outs, rates, seconds, rng):
    """Poisson request streams at each aggregate rate; latency from each request's
    arrival to its completion (waiting behind the client's previous request included)."""
    import threading
    sweep = []
    for rate in rates:
        n_req = max(50, int(rate * seconds))
        arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n_req))
        who = rng.integers(0, len(meshes), size=n_req)
        per_client = [[] for _ in meshes]
        for t, c in zip(arrivals, who):
            per_client[c].append(t)
        lat, srv_lat, elems, sizes, arr = [], [], [0], [], []
        lock = threading.Lock()
        t0 = time.perf_counter() + 0.05
        st0 = srv.stats()

        def client(c):
            k = 0
            for t in per_client[c]:
                delay = t0 + t - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                tk = srv.submit(ids[c], states[c][k & 1], outs[c])
                sl = srv.wait(tk)
                done = time.perf_counter()
                k += 1
                with lock:
                    lat.append(done - (t0 + t))
                    srv_lat.append(sl)
                    sizes.append(meshes[c].num_elements)
                    arr.append(t)
                    elems[0] += meshes[c].num_elements

        threads = [threading.Thread(target=client, args=(c,)) for c in range(len(meshes)) if per_client[c]]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        wall = time.perf_counter() - t0
        st1 = srv.stats()
        lat_ms = np.array(lat) * 1e3
        sz = np.array(sizes)
        by_size = {}
        for name, lo, hi in (("small <3e4 el", 0, 3e4), ("medium 3e4-3e5 el", 3e4, 3e5), ("large >=3e5 el", 3e5, 1e12)):
            sel = lat_ms[(sz >= lo) & (sz < hi)]
            if sel.size:
                by_size[name] = {"requests": int(sel.size), "p50_ms": float(np.percentile(sel, 50)),
                                 "p99_ms": float(np.percentile(sel, 99))}
        sweep.append({"rate_req_s": rate, "requests": len(lat), "elements_per_s": elems[0] / wall,
                      "p50_ms": float(np.percentile(lat_ms, 50)), "p99_ms": float(np.percentile(lat_ms, 99)),
                      "server_p50_ms": float(np.percentile(np.array(srv_lat) * 1e3, 50)),
                      "server_p99_ms": float(np.percentile(np.array(srv_lat) * 1e3, 99)),
                      "by_request_size": by_size, "waves": st1["waves"] - st0["waves"], "wall_s": wall,
                      "slowest": [{"arrival_s": float(arr[i]), "ms": float(lat_ms[i]),
                                   "server_ms": float(srv_lat[i] * 1e3), "elements": int(sz[i])}
                                  for i in np.argsort(lat_ms)[::-1][:5]]})
    return sweep


def serve_setup(fem, clients, budget_gb, precision, max_batch):
    import torch
    specs = fem.batch_specs(count=clients, seed=fem.mesh.SEEDS["serve64"], max_dof=4e6)
    meshes = [sp.build() for sp in specs]
    srv = fem.Server(int(budget_gb * 1e9), precision=precision, max_batch=max_batch)
    ids, admitted = [], []
    for i, m in enumerate(meshes):
        try:
            ids.append(srv.add_mesh(m))
            admitted.append(i)
        except fem.FemError as e:
            if e.status != fem.FEM_ERR_BUDGET:
                raise
    meshes = [meshes[i] for i in admitted]
    states = []
    for m in meshes:
        s0 = torch.from_numpy(np.ascontiguousarray(m.states)).pin_memory()
        s1 = torch.from_numpy(np.ascontiguousarray(m.states * 1.01 + 1e-6)).pin_memory()
        states.append((s0, s1))
    outs = [torch.empty(m.num_nodes * 2, dtype=torch.float64).pin_memory() for m in meshes]
    for i in range(len(meshes)):  # warm-up: one request per client
        srv.wait(srv.submit(ids[i], states[i][0], outs[i]))
    return srv, ids, meshes, states, outs


def serve_plain(fem, dev, meshes, states, outs, rng, count):
    """Plain single-mesh FP64 drop-in for a sample of requests: H2D state, zero the
    outputs, fem_run_jacobian, D2H residual, one request at a time."""
    import torch
    sample = rng.integers(0, len(meshes), size=min(count, len(meshes)))
    stream = torch.cuda.Stream(device=dev)
    plain_el, plain_t = 0, 0.0
    for c in sorted(set(sample.tolist())):
        m = meshes[c]
        rowp, cols = fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
        mp = fem.build_element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)
        with torch.cuda.stream(stream):
            dm = fem.DeviceMesh(m, dev)
            dmap = torch.from_numpy(mp).to(dev)
            r = torch.empty(m.num_nodes * 2, dtype=torch.float64, device=dev)
            a = torch.empty(cols.size * 4, dtype=torch.float64, device=dev)
        reps = int((sample == c).sum())

        def one():
            dm.states.copy_(states[c][0], non_blocking=True)
            r.zero_()
            a.zero_()
            fem.run_jacobian_kernel(m.order, dm.conn_ptr, dm.conn, m.num_elements, dm.states, dm.coords, m.E, m.nu,
                                    m.t, dmap, r, a, stream=stream.cuda_stream, timed=False)
            outs[c].copy_(r, non_blocking=True)

        with torch.cuda.stream(stream):
            one()
            stream.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                one()
            e1.record(stream)
            e1.synchronize()
        plain_t += e0.elapsed_time(e1) * 1e-3
        plain_el += reps * m.num_elements
        del dm, dmap, r, a
        torch.cuda.empty_cache()
    return plain_el / plain_t, int(len(sample))


def serve_leg(fem, dev, args):
    """The serving configuration in the default run: the 64 Newton clients at one
    sub-saturation rate and at a saturating rate, FP64 and MIXED."""
    t0 = time.perf_counter()
    rng = np.random.default_rng(12345)
    out = {"workload": (f"{args.clients} Newton clients (meshes drawn like the batched set, <= 4M DOF each), "
                        f"Poisson arrivals, state H2D and residual D2H inside every request"),
           "rates_req_s": args.leg_rates, "seconds_per_rate": args.leg_serve_seconds}
    for prec in ("fp64", "mixed"):
        srv, ids, meshes, states, outs = serve_setup(fem, args.clients, args.budget_gb, prec, args.max_batch)
        sweep = serve_sweep(fem, srv, ids, meshes, states, outs, args.leg_rates, args.leg_serve_seconds, rng)
        out[prec] = {"clients_admitted": len(meshes), "device_bytes_used": srv.stats()["used_bytes"], "sweep": sweep}
        srv.close()
        if prec == "fp64":
            plain, n = serve_plain(fem, dev, meshes, states, outs, rng, 64)
            out["plain_fp64_dropin_per_request"] = {"elements_per_s": plain, "requests": n}
        del srv, meshes, states, outs
    log(f"served leg {time.perf_counter() - t0:.1f} s")
    return out


def run_batch(args):
    """Many meshes (log-uniform sizes 1e3..1e6 elements, orders 1..4) per graph launch,
    in waves that fit the device-memory budget, against the single-mesh FP64 drop-in."""
    import torch
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    import fem_pkg
    fem = fem_pkg.load()
    specs = fem.batch_specs(count=args.batch_meshes)
    waves = waves_of(specs, args.budget_gb * 1e9)
    prec = args.batch_precision
    r = batched_measure(fem, dev, waves, args.steps, args.warmup, (prec,))
    el = r["elements"]
    line = {
        "metric": "assembled elements/s (res+Jac)", "value": el / (r["ms"][prec] * 1e-3), "unit": "elements/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms"][prec],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if prec == "fp64" else "bf16x6 (p3) / f32 (p4) / f64", "data": "synthetic",
        "config": {"workload": f"batch{len(specs)}: element counts log-uniform in [1e3, 1e6], orders 1..4",
                   "meshes": len(specs), "elements": el, "waves": len(waves), "budget_gb": args.budget_gb,
                   "precision": prec, "l2": "per-wave inputs and outputs larger than L2"},
        "plain_fp64_single_mesh": {"elements_per_s": el / (r["ms_plain"] * 1e-3), "ms_per_step": r["ms_plain"]},
        "batched_over_plain": r["ms_plain"] / r["ms"][prec],
        "wave_graph_ms": r["wave_ms"][prec], "tuned_tile_batches": r["tiles"][prec],
        "tuned_kernels": r["kernels"][prec],
        "tuned_ordered": r["ordered"][prec],
        "mixed_rel_frobenius_err_max": max(r["errs"]) if r["errs"] else None,
        "gpu_launches": r["launches"][prec],
    }
    print(json.dumps(line), flush=True)


def run_serve(args):
    """64 Newton-solve clients with device-resident meshes issue requests as one
    Poisson stream at each swept aggregate rate; the server admits meshes under the
    HBM budget and batches concurrent requests."""
    import torch
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    import fem_pkg
    fem = fem_pkg.load()
    rng = np.random.default_rng(12345)
    srv, ids, meshes, states, outs = serve_setup(fem, args.clients, args.budget_gb, args.batch_precision,
                                                 args.max_batch)
    sweep = serve_sweep(fem, srv, ids, meshes, states, outs, args.rates, args.serve_seconds, rng)
    used = srv.stats()["used_bytes"]
    srv.close()
    plain, n = serve_plain(fem, dev, meshes, states, outs, rng, 64)
    best = max(sweep, key=lambda x: x["elements_per_s"])
    line = {
        "metric": "assembled elements/s (res+Jac); serve p50/p99 ms", "value": best["elements_per_s"],
        "unit": "elements/s", "n_gpus": 1, "steps": sum(x["requests"] for x in sweep), "warmup": len(meshes),
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.batch_precision == "fp64" else "bf16x6 (p3) / f32 (p4) / f64", "data": "synthetic",
        "config": {"workload": f"serve{args.clients}: Newton clients, meshes <= 4M DOF, Poisson arrivals",
                   "clients_admitted": len(meshes), "budget_gb": args.budget_gb, "device_bytes_used": used,
                   "max_batch": args.max_batch, "precision": args.batch_precision},
        "sweep": sweep,
        "plain_fp64_single_mesh": {"elements_per_s": plain, "requests": n},
    }
    print(json.dumps(line), flush=True)


def measure_peaks():
    """Arithmetic peaks of this GPU from the probe library (TFLOP/s)."""
    import ctypes as C

    import torch

    import fem_pkg
    fem_pkg.load_builder().build()
    probe = C.CDLL(str(ROOT / "gpu-fem-project_b200" / "libfemprobe.so"))
    probe.fem_probe_peak.argtypes = [C.c_int, C.POINTER(C.c_double)]
    torch.cuda.init()
    out = {}
    for kind, name in ((0, "fp64_fma_tflops"), (1, "fp32_fma_tflops"), (2, "fp64_mma_tflops"),
                       (3, "bf16_mma_sync_tflops")):
        v = C.c_double()
        rc = probe.fem_probe_peak(kind, C.byref(v))
        if rc != 0:
            raise RuntimeError(f"fem_probe_peak({kind}) returned {rc}")
        out[name] = v.value
    out["gpu"] = torch.cuda.get_device_name(0)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400, help="timed steps (400 x ~2.6 ms: a region of about 1 s)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="square1024_p3", choices=sorted(WORKLOADS) + ["batch256", "serve64"])
    ap.add_argument("--min-seconds", type=float, default=1.0, help="timed region of each comparison path")
    ap.add_argument("--clients", type=int, default=64)
    ap.add_argument("--rates", type=lambda v: [float(x) for x in v.split(",")], default=[100, 500, 1000, 2500, 5000])
    ap.add_argument("--serve-seconds", type=float, default=3.0)
    ap.add_argument("--max-batch", type=int, default=64)
    ap.add_argument("--batch-meshes", type=int, default=256)
    ap.add_argument("--budget-gb", type=float, default=100.0, help="device bytes per batched wave / server budget")
    ap.add_argument("--batch-precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-legs", action="store_true", help="skip the batched and served legs of the default run")
    ap.add_argument("--leg-batch-gb", type=float, default=40.0, help="device bytes of the batched leg's meshes")
    ap.add_argument("--leg-steps", type=int, default=10)
    ap.add_argument("--leg-rates", type=lambda v: [float(x) for x in v.split(",")], default=[1000, 5000])
    ap.add_argument("--leg-serve-seconds", type=float, default=2.0)
    ap.add_argument("--ref-elements", type=int, default=None,
                    help="elements of the CPU sample (default 131072; in --impl reference scaled down with "
                         "--steps so that the run stays near 20 steps of 131072 elements, at least 32768)")
    ap.add_argument("--bands", type=int, default=32, help="element bands / node chunks of the end-to-end call")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-run", action="store_true",
                    help="time one path's launches only and print no JSON line (for ncu captures)")
    ap.add_argument("--profile-path", default="jacobian", choices=["jacobian", "mixed", "residual"],
                    help="the plan path of --profile-run (FP64 residual+Jacobian, MIXED, FP64 residual only)")
    ap.add_argument("--peaks", action="store_true", help="print measured FP64/FP32/FP64-MMA/BF16-MMA peaks and exit")
    args = ap.parse_args()
    if args.peaks:
        print(json.dumps(measure_peaks()))
        return
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch256":
        run_batch(args)
    elif args.workload == "serve64":
        run_serve(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
