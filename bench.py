#!/usr/bin/env python3
"""Benchmark: global residual + Jacobian assembly of plane-stress Lagrange quads on B200.

Default workload: 1024x1024 order-3 quads on a 10x10 square (+-0.2h interior
perturbation, u in [-1e-3,1e-3], E=70e9, nu=0.3, 4x4 Gauss points; 18,886,658 DOF,
235,960,321 2x2 blocks).  One step = one complete residual + Jacobian assembly.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Prints one JSON line (rank 0).  `value` is elements/s of the fastest validated
path with device-resident inputs; `e2e` is the same metric through the public
API with a host->device copy of the state and a device->host copy of the
residual inside every timed step.  Multi-GPU runs are independent replicas (the
assembly of one mesh is not sharded).  --impl reference times the FP64 CPU
oracle (restatement of the reference's CPU assembly, element/FEKernels.h:317-508)
on a bounded sample of the same mesh with all host threads.
"""
from __future__ import annotations

import argparse
import json
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


def make_mesh(fem, name):
    w = WORKLOADS[name]
    if w["kind"] == "square64":
        return fem.square64_p1()
    if w["kind"] == "annulus":
        return fem.annulus512x2048_p2()
    if w["p"] == 3:
        return fem.square1024_p3(w["n"])
    return fem.square_mesh(w["n"], w["n"], w["p"], 1.0, 1.0, 0.1, 1e-3, 70e9, 0.3, 1.0, 0x5EED0006,
                           f"square{w['n']}_p{w['p']}")


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per assembly from ncu
# captures of the headline kernels, keyed by workload and kernel family.  The
# 1024^2 order-3 figure is the sum over the four colour launches of the 512^2 case
# (2.835 GB; BF16x6 and FP64 kernels move the same bytes), times 4: traffic grows
# with the element count.
MEASURED_TRAFFIC = {
    ("square1024_p3", "frag_kernel<3"): 4 * 2.835e9,
}


def algorithmic_bytes(mesh, nnzb):
    """Minimal HBM bytes of one residual+Jacobian assembly: read coords and states,
    read conn, write the residual and the BSR values once."""
    return 16 * mesh.num_nodes * 2 + 4 * mesh.num_elements * mesh.nodes_per_element + 16 * mesh.num_nodes + 32 * nnzb


def algorithmic_flops(mesh):
    """Per-element FP64 flop convention n_q*(24n^2 + 24n + 40) with n = n_q = (p+1)^2."""
    n = mesh.nodes_per_element
    return mesh.num_elements * n * (24 * n * n + 24 * n + 40)


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


# ----------------------------------------------------------------------------------------
def run_reference(args):
    """FP64 CPU oracle (restatement of the reference CPU assembly) on a bounded sample."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if int(os.environ.get("RANK", "0")) != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import fem_pkg
    import oracle as orc
    fem = fem_pkg.load()
    mesh = make_mesh(fem, args.workload)
    sample = min(mesh.num_elements, args.ref_elements)
    sub = fem.submesh(mesh, 0, sample)
    rowp, cols = fem.build_bsr_pattern(sub.num_nodes, sub.conn_ptr, sub.conn)
    mp = fem.build_element_bsr_map(sub.conn_ptr, sub.conn, sub.nodes_per_element, rowp, cols)
    threads = os.cpu_count() or 1
    orc.set_threads(threads)
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        orc.assemble(sub, mp, cols.size, parallel=True)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    tot = sum(times)
    value = sample * len(times) / tot
    line = {
        "impl": "reference", "metric": "assembled elements/s (res+Jac)", "value": value, "unit": "elements/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "sample_elements": sample, "order": mesh.order},
        "cpu_baseline": {"value": value, "unit": "elements/s", "cores": threads, "kind": "port",
                         "sample": f"first {sample} elements of {mesh.name} (OpenMP over elements, atomic scatter)"},
        "e2e": {"value": value, "unit": "elements/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------------------
def run_ours(args):
    import torch
    world, rank, local, pg = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import fem_pkg
    fem = fem_pkg.load()
    mesh = make_mesh(fem, args.workload)
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

    def time_steps(fn, steps, warmup, launches_per_step):
        for _ in range(warmup):
            fn()
        stream.synchronize()
        if pg is not None:
            pg.barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            fn()
        ev1.record(stream)
        ev1.synchronize()
        ms = ev0.elapsed_time(ev1) / steps
        ms = fem_pkg.load_module("replicas").max_over_ranks(ms, pg, dev)
        return ms, launches_per_step * steps

    paths = {}
    # plan path (overwrite, no zeroing), FP64 and mixed
    for prec in [x for x in ("fp64", "mixed") if f"plan_{x}" in args.paths]:
        fn = (lambda prec=prec: plan.assemble(d.states, d.coords, E, nu, t, res, mat, precision=prec, stream=sptr))
        ms, _ = time_steps(fn, max(2, args.steps // 2), args.warmup, plan.launches())
        paths[f"plan_{prec}"] = {"ms": ms, "elements_per_s": nE / (ms * 1e-3)}
    # GreenStrainType::NONLINEAR (FP64), same mesh and states; not a candidate for the headline
    # (the reference's dispatch always assembles LINEAR)
    if "plan_nonlinear" in args.paths:
        fn = (lambda: plan.assemble(d.states, d.coords, E, nu, t, res, mat, strain="nonlinear", stream=sptr))
        ms, _ = time_steps(fn, max(2, args.steps // 2), args.warmup, plan.launches("nonlinear"))
        paths["plan_fp64_nonlinear"] = {"ms": ms, "elements_per_s": nE / (ms * 1e-3)}
    # error of the mixed plan path against the FP64 plan path (FP64 path is oracle-checked in tests)
    err_res = err_mat = float("inf")
    if "plan_mixed" in paths:
        with torch.cuda.stream(stream):
            plan.assemble(d.states, d.coords, E, nu, t, res, mat, precision="fp64", stream=sptr)
            res64, mat64 = res.clone(), mat.clone()
            plan.assemble(d.states, d.coords, E, nu, t, res, mat, precision="mixed", stream=sptr)
            err_res = float(torch.linalg.vector_norm(res - res64) / torch.linalg.vector_norm(res64))
            err_mat = float(torch.linalg.vector_norm(mat - mat64) / torch.linalg.vector_norm(mat64))
            del res64, mat64
        paths["plan_mixed"]["rel_frobenius_err"] = {"residual": err_res, "jacobian": err_mat}
    stream.synchronize()
    # plain drop-in FP64 (reference contract: caller zeroes, kernel accumulates via map, atomics)
    if any(x.startswith("dropin") for x in args.paths):
        rowp_h, cols_h = plan.pattern()
        mp = fem.build_element_bsr_map(mesh.conn_ptr, mesh.conn, mesh.nodes_per_element, rowp_h, cols_h)
        with torch.cuda.stream(stream):
            dmap = torch.from_numpy(mp).to(dev)
        del mp, rowp_h, cols_h

        def dropin(prec="fp64", zero=True):
            if zero:
                res.zero_()
                mat.zero_()
            fem.run_jacobian_kernel(mesh.order, d.conn_ptr, d.conn, nE, d.states, d.coords, E, nu, t, dmap, res, mat,
                                    precision=prec, stream=sptr, timed=False)

        with torch.cuda.stream(stream):
            if "dropin_fp64" in args.paths:
                ms, _ = time_steps(lambda: dropin("fp64", True), max(2, args.steps // 2), args.warmup, 1)
                paths["dropin_fp64_with_zeroing"] = {"ms": ms, "elements_per_s": nE / (ms * 1e-3)}
                ms, _ = time_steps(lambda: dropin("fp64", False), max(2, args.steps // 2), args.warmup, 1)
                paths["dropin_fp64_kernel_only"] = {"ms": ms, "elements_per_s": nE / (ms * 1e-3)}
            if "dropin_mixed" in args.paths:
                ms, _ = time_steps(lambda: dropin("mixed", False), max(2, args.steps // 2), args.warmup, 1)
                paths["dropin_mixed_kernel_only"] = {"ms": ms, "elements_per_s": nE / (ms * 1e-3)}
        del dmap
    best = "plan_fp64"
    # MIXED is the headline only where it runs a kernel of its own and wins
    mixed_own = kernel_label(plan, mesh.order, "mixed") != kernel_label(plan, mesh.order, "fp64")
    if "plan_mixed" in paths and mixed_own and max(err_res, err_mat) <= 1e-6 and (
            "plan_fp64" not in paths or paths["plan_mixed"]["ms"] < paths["plan_fp64"]["ms"]):
        best = "plan_mixed"
    prec = "mixed" if best == "plan_mixed" else "fp64"

    def step():
        plan.assemble(d.states, d.coords, E, nu, t, res, mat, precision=prec, stream=sptr)

    with ClockSampler(local) as clk:
        ms, launches = time_steps(step, args.steps, args.warmup, plan.launches())
    value = world * nE / (ms * 1e-3)

    # end to end through the public API: pinned host state -> device, assemble, residual
    # -> pinned host, in one fem_plan_assemble_host call (state upload in node chunks,
    # band-split colour launches, residual download per chunk, all overlapped)
    h_states = torch.from_numpy(np.ascontiguousarray(mesh.states)).pin_memory()
    h_res = torch.empty(mesh.num_nodes * 2, dtype=torch.float64).pin_memory()

    def e2e_step():
        plan.assemble_host(h_states, d.states, d.coords, E, nu, t, h_res, res, mat, precision=prec, bands=args.bands,
                           stream=sptr)

    def e2e_serial_step():
        d.states.copy_(h_states, non_blocking=True)
        plan.assemble(d.states, d.coords, E, nu, t, res, mat, precision=prec, stream=sptr)
        h_res.copy_(res, non_blocking=True)

    band_launches = plan.launches() if plan.row_chunks > 0 else plan.num_colours * args.bands
    with torch.cuda.stream(stream):
        ms_e2e, _ = time_steps(e2e_step, args.steps, args.warmup, band_launches)
        ms_e2e_serial, _ = time_steps(e2e_serial_step, args.steps, args.warmup, plan.launches())
    h2d, d2h = h_states.numel() * 8, h_res.numel() * 8

    # the same per-step work for independent load cases streamed through the GPU:
    # case k+1's state upload and case k-1's residual download overlap case k's
    # assembly (copy-in, compute and copy-out streams, two state/residual buffers)
    s_in, s_out = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    with torch.cuda.stream(stream):
        st2 = [d.states, torch.empty_like(d.states)]
        rs2 = [res, torch.empty_like(res)]
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
        plan.assemble(st2[b], d.coords, E, nu, t, rs2[b], mat, precision=prec, stream=sptr)
        ev_comp[b].record(stream)
        s_out.wait_event(ev_comp[b])
        with torch.cuda.stream(s_out):
            hr2[b].copy_(rs2[b], non_blocking=True)
        ev_out[b].record(s_out)

    for k in range(args.warmup):
        piped_step(k)
    torch.cuda.synchronize(dev)
    if pg is not None:
        pg.barrier()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(s_in)
    for k in range(args.steps):
        piped_step(k)
    s_in.wait_event(ev_out[0])
    s_in.wait_event(ev_out[1])
    p1.record(s_in)
    p1.synchronize()
    ms_piped = fem_pkg.load_module("replicas").max_over_ranks(p0.elapsed_time(p1) / args.steps, pg, dev)
    torch.cuda.synchronize(dev)
    del st2, rs2, hs2, hr2

    hbm, peak_kind = peaks()
    abytes = algorithmic_bytes(mesh, nnzb)
    label = kernel_label(plan, mesh.order, prec)
    traffic = next((v for (w, k), v in MEASURED_TRAFFIC.items() if w == mesh.name and label.startswith(k)), None)
    achieved = abytes / (ms * 1e-3) / 1e9
    # FP64 side of the roofline: conventional element flops n_q (24 n^2 + 24 n + 40)
    # (a 2x2 block of D^T B products per node pair plus the J / grad u / sigma / R
    # work, no symmetry savings) against this GPU's FP64 tensor-core peak, probed live
    import ctypes as C
    nloc = (mesh.order + 1) ** 2
    aflops = float(nE) * nloc * (24 * nloc * nloc + 24 * nloc + 40)
    fp64_peak = C.c_double()
    fem.check(fem.lib.fem_probe_peak(2, C.byref(fp64_peak)), "fem_probe_peak")
    line = {
        "metric": "assembled elements/s (res+Jac)", "value": value, "unit": "elements/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if prec == "fp64" else {1: "f64", 2: "f64", 3: "bf16x6/f64"}.get(mesh.order, "f32/f64"),
        "data": "synthetic",
        "config": {"workload": mesh.name, "order": mesh.order, "elements": nE, "dof": mesh.num_dof, "nnzb": nnzb,
                   "path": best, "l2": "inputs and outputs larger than L2 (BSR values %.2f GB)" % (32 * nnzb / 1e9),
                   "parallelism": f"replicas{world}"},
        "dof_per_s": value * mesh.num_dof / nE,
        "paths": paths,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": traffic, "peak_kind": peak_kind, "algorithmic_bytes_per_step": abytes,
                     "kernel": kernel_label(plan, mesh.order, prec),
                     "traffic_note": ("DRAM bytes per step (all colour launches of one assembly) from an ncu capture "
                                      "of a 512^2 order-3 mesh scaled x4 (profiles/); above the algorithmic bytes: "
                                      "later colours' bulk reductions read the blocks an earlier colour stored"
                                      if traffic else "no ncu capture for this workload"),
                     "fp64": {"algorithmic_flops_per_step": aflops,
                              "achieved_tflops": aflops / (ms * 1e-3) / 1e12,
                              "peak_tflops": fp64_peak.value, "peak_kind": "measured (FP64 MMA probe)",
                              "frac": aflops / (ms * 1e-3) / 1e12 / fp64_peak.value,
                              "max_bound_frac": max(abytes / (hbm * 1e9), aflops / (fp64_peak.value * 1e12))
                              / (ms * 1e-3)}},
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "e2e": {"value": world * nE / (ms_e2e * 1e-3), "unit": "elements/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e,
                "api": f"fem_plan_assemble_host, {args.bands} bands (copies overlapped with the assembly)",
                "serial": {"value": world * nE / (ms_e2e_serial * 1e-3), "ms_per_step": ms_e2e_serial,
                           "note": "state upload, fem_plan_assemble, residual download in sequence"},
                "pipelined": {"value": world * nE / (ms_piped * 1e-3), "ms_per_step": ms_piped,
                              "note": "independent load cases: case k+1 uploads and case k-1 downloads "
                                      "while case k assembles (3 streams, 2 buffers); same copies per step"}},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(fem, mesh, args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    plan.close()
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


def kernel_label(plan, order, prec):
    """The kernel that runs one assembly of `plan` (the dispatch of fem_plan_assemble)."""
    if plan.row_chunks > 0:
        return "rows_p1_kernel, 1 launch per step"
    # the fragment kernel serves orders 2-3 in both precisions (MIXED at order 3 with
    # its element stiffness as BF16x6 tensor-core products, at order 2 in FP64) and
    # order 4 in FP64; FP32 order 4 runs the element kernel
    if order == 3 and prec == "mixed":
        return f"frag_kernel<{order}, BF16x6 stiffness> x {plan.num_colours} colour launches per step"
    if order in (2, 3) or (order == 4 and prec == "fp64"):
        return f"frag_kernel<{order}> x {plan.num_colours} colour launches per step"
    return f"assemble_kernel<{order}, float> x {plan.num_colours} colour launches per step"


def mesh_bytes(spec, with_map=True):
    """Device bytes of one batched mesh: plan topology, coordinates/states/residual,
    BSR values and (for the single-mesh comparison) the reference element map."""
    n = (spec.order + 1) ** 2
    N, ne, nnzb = spec.num_nodes(), spec.num_elements, spec.nnzb()
    plan = 4 * (N + 1) + 4 * nnzb + 4 * ne * n + ne * n * n + ne * n
    data = 16 * N * 3 + 4 * ne * n + 4 * (ne + 1) + 32 * nnzb
    return plan + data + (4 * ne * n * n if with_map else 0)


def run_batch(args):
    """Many meshes (log-uniform sizes 1e3..1e6 elements, orders 1..4) per graph launch,
    in waves that fit the device-memory budget, against the single-mesh FP64 drop-in."""
    import torch
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    import fem_pkg
    fem = fem_pkg.load()
    specs = fem.batch_specs(count=args.batch_meshes)
    budget = args.budget_gb * 1e9
    waves, cur, used = [], [], 0
    for sp in specs:
        b = mesh_bytes(sp)
        if cur and used + b > budget:
            waves.append(cur)
            cur, used = [], 0
        cur.append(sp)
        used += b
    if cur:
        waves.append(cur)
    stream = torch.cuda.Stream(device=dev)
    sptr = stream.cuda_stream
    tot_el, t_batch, t_plain, launches, graph_ms, errs, tiles = 0, 0.0, 0.0, 0, [], [], []

    def ev_time(fn, reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps * 1e-3

    for wave in waves:
        meshes = [sp.build() for sp in wave]
        plans = [fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn) for m in meshes]
        with torch.cuda.stream(stream):
            devs = [fem.DeviceMesh(m, dev) for m in meshes]
            res = [torch.empty(m.num_nodes * 2, dtype=torch.float64, device=dev) for m in meshes]
            mat = [torch.empty(p.nnzb * 4, dtype=torch.float64, device=dev) for p in plans]
        stream.synchronize()
        batch = fem.Batch(plans)
        for i, (m, d) in enumerate(zip(meshes, devs)):
            batch.bind(i, d.states, d.coords, m.E, m.nu, m.t, res[i], mat[i])
        prec = args.batch_precision
        batch.tune(precision=prec, stream=sptr, reps=2)
        tiles.append(batch.info()["tile_batches"])
        batch.capture(precision=prec, stream=sptr)
        for _ in range(args.warmup):
            batch.replay(stream=sptr)
        tb = ev_time(lambda: batch.replay(stream=sptr), args.steps)
        launches += batch.info()["launches"] * args.steps
        if prec == "mixed":
            with torch.cuda.stream(stream):
                keep = [(r.clone(), a.clone()) for r, a in zip(res[:8], mat[:8])]
                batch.assemble(precision="fp64", stream=sptr)
                for (r, a), r64, a64 in zip(keep, res[:8], mat[:8]):
                    errs.append(max(float(torch.linalg.vector_norm(r - r64) / torch.linalg.vector_norm(r64)),
                                    float(torch.linalg.vector_norm(a - a64) / torch.linalg.vector_norm(a64))))
            del keep
        # plain single-mesh FP64 drop-in (reference contract): zero outputs, one call per mesh
        maps = []
        for m, p in zip(meshes, plans):
            rowp, cols = p.pattern()
            mp = fem.build_element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)
            maps.append(torch.from_numpy(mp).to(dev))

        def plain():
            for m, d, r, a, mp in zip(meshes, devs, res, mat, maps):
                r.zero_()
                a.zero_()
                fem.run_jacobian_kernel(m.order, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu,
                                        m.t, mp, r, a, stream=sptr, timed=False)

        with torch.cuda.stream(stream):
            plain()
            tp = ev_time(plain, max(1, args.steps // 2))
        tot_el += sum(m.num_elements for m in meshes)
        t_batch += tb
        t_plain += tp
        graph_ms.append(tb * 1e3)
        batch.close()
        for p in plans:
            p.close()
        del meshes, plans, devs, res, mat, maps, batch
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    value = tot_el / t_batch
    line = {
        "metric": "assembled elements/s (res+Jac)", "value": value, "unit": "elements/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_batch * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.batch_precision == "fp64" else "bf16x6 (p3) / f32 (p4) / f64",
        "data": "synthetic",
        "config": {"workload": f"batch{len(specs)}: element counts log-uniform in [1e3, 1e6], orders 1..4",
                   "meshes": len(specs), "elements": tot_el, "waves": len(waves),
                   "budget_gb": args.budget_gb, "precision": args.batch_precision,
                   "l2": "per-wave inputs and outputs larger than L2"},
        "plain_fp64_single_mesh": {"elements_per_s": tot_el / t_plain, "ms_per_step": t_plain * 1e3},
        "batched_over_plain": t_plain / t_batch,
        "wave_graph_ms": graph_ms, "tuned_tile_batches": tiles,
        "mixed_rel_frobenius_err_max": max(errs) if errs else None,
        "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)


def run_serve(args):
    """64 Newton-solve clients with device-resident meshes (drawn like the batched
    workload, at most 4M DOF each) issue requests as one Poisson stream at each
    swept aggregate rate; the server admits meshes under the HBM budget and
    batches concurrent requests.  Latency is measured from each request's arrival
    (so it includes waiting behind the client's previous request)."""
    import threading

    import torch
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    import fem_pkg
    fem = fem_pkg.load()
    specs = fem.batch_specs(count=args.clients, seed=fem.mesh.SEEDS["serve64"], max_dof=4e6)
    meshes = [sp.build() for sp in specs]
    srv = fem.Server(int(args.budget_gb * 1e9), precision=args.batch_precision, max_batch=args.max_batch)
    ids, admitted = [], []
    for i, m in enumerate(meshes):
        try:
            ids.append(srv.add_mesh(m))
            admitted.append(i)
        except fem.FemError as e:
            if e.status != fem.FEM_ERR_BUDGET:
                raise
    meshes = [meshes[i] for i in admitted]
    rng = np.random.default_rng(12345)
    states = []
    for m in meshes:
        s0 = torch.from_numpy(np.ascontiguousarray(m.states)).pin_memory()
        s1 = torch.from_numpy(np.ascontiguousarray(m.states * 1.01 + 1e-6)).pin_memory()
        states.append((s0, s1))
    outs = [torch.empty(m.num_nodes * 2, dtype=torch.float64).pin_memory() for m in meshes]
    for i in range(len(meshes)):  # warm-up: one request per client
        srv.wait(srv.submit(ids[i], states[i][0], outs[i]))
    sweep = []
    for rate in args.rates:
        n_req = max(50, int(rate * args.serve_seconds))
        arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n_req))
        who = rng.integers(0, len(meshes), size=n_req)
        per_client = [[] for _ in meshes]
        for t, c in zip(arrivals, who):
            per_client[c].append(t)
        lat, srv_lat, elems = [], [], [0]
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
                    elems[0] += meshes[c].num_elements

        threads = [threading.Thread(target=client, args=(c,)) for c in range(len(meshes)) if per_client[c]]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        wall = time.perf_counter() - t0
        st1 = srv.stats()
        lat_ms = np.array(lat) * 1e3
        sweep.append({"rate_req_s": rate, "requests": len(lat), "elements_per_s": elems[0] / wall,
                      "p50_ms": float(np.percentile(lat_ms, 50)), "p99_ms": float(np.percentile(lat_ms, 99)),
                      "server_p50_ms": float(np.percentile(np.array(srv_lat) * 1e3, 50)),
                      "server_p99_ms": float(np.percentile(np.array(srv_lat) * 1e3, 99)),
                      "waves": st1["waves"] - st0["waves"], "wall_s": wall})
    used = srv.stats()["used_bytes"]
    srv.close()
    # plain single-mesh FP64 drop-in for a sample of the same requests: H2D state,
    # zero the outputs, fem_run_jacobian, D2H residual, one request at a time
    sample = rng.integers(0, len(meshes), size=min(64, len(meshes)))
    stream = torch.cuda.Stream(device=dev)
    plain_el, plain_t = 0, 0.0
    for c in sorted(set(sample.tolist())):
        m = meshes[c]
        rowp, cols = fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
        mp = fem.build_element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)
        with torch.cuda.stream(stream):
            d = fem.DeviceMesh(m, dev)
            dmap = torch.from_numpy(mp).to(dev)
            r = torch.empty(m.num_nodes * 2, dtype=torch.float64, device=dev)
            a = torch.empty(cols.size * 4, dtype=torch.float64, device=dev)
        reps = int((sample == c).sum())

        def one():
            d.states.copy_(states[c][0], non_blocking=True)
            r.zero_()
            a.zero_()
            fem.run_jacobian_kernel(m.order, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t,
                                    dmap, r, a, stream=stream.cuda_stream, timed=False)
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
        del d, dmap, r, a
        torch.cuda.empty_cache()
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
        "plain_fp64_single_mesh": {"elements_per_s": plain_el / plain_t, "requests": int(len(sample))},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(fem, mesh, args):
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc
    sample = min(mesh.num_elements, args.ref_elements)
    sub = fem.submesh(mesh, 0, sample)
    rowp, cols = fem.build_bsr_pattern(sub.num_nodes, sub.conn_ptr, sub.conn)
    mp = fem.build_element_bsr_map(sub.conn_ptr, sub.conn, sub.nodes_per_element, rowp, cols)
    threads = os.cpu_count() or 1
    orc.set_threads(threads)
    orc.assemble(sub, mp, cols.size, parallel=True)
    t0 = time.perf_counter()
    reps = 0
    while True:
        orc.assemble(sub, mp, cols.size, parallel=True)
        reps += 1
        if time.perf_counter() - t0 > args.cpu_seconds:
            break
    dt = (time.perf_counter() - t0) / reps
    return {"value": sample / dt, "unit": "elements/s", "cores": threads, "kind": "port",
            "sample": f"first {sample} elements of {mesh.name}, {reps} repeats (OpenMP, atomic scatter)"}


def measure_peaks():
    """Arithmetic peaks of this GPU from the library's probe kernels (TFLOP/s)."""
    import ctypes as C

    import torch

    import fem_pkg
    fem = fem_pkg.load()
    torch.cuda.init()
    out = {}
    for kind, name in ((0, "fp64_fma_tflops"), (1, "fp32_fma_tflops"), (2, "fp64_mma_tflops"),
                       (3, "bf16_mma_sync_tflops")):
        v = C.c_double()
        fem.check(fem.lib.fem_probe_peak(kind, C.byref(v)), "fem_probe_peak")
        out[name] = v.value
    out["gpu"] = torch.cuda.get_device_name(0)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="square1024_p3", choices=sorted(WORKLOADS) + ["batch256", "serve64"])
    ap.add_argument("--clients", type=int, default=64)
    ap.add_argument("--rates", type=lambda v: [float(x) for x in v.split(",")], default=[100, 500, 1000, 2500, 5000])
    ap.add_argument("--serve-seconds", type=float, default=3.0)
    ap.add_argument("--max-batch", type=int, default=64)
    ap.add_argument("--batch-meshes", type=int, default=256)
    ap.add_argument("--budget-gb", type=float, default=100.0, help="device bytes per batched wave")
    ap.add_argument("--batch-precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--ref-elements", type=int, default=131072)
    ap.add_argument("--bands", type=int, default=32, help="element bands / node chunks of the end-to-end call")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--paths", default="plan_fp64,plan_mixed,dropin_fp64,plan_nonlinear",
                    help="comma list of plan_fp64, plan_mixed, dropin_fp64, dropin_mixed, plan_nonlinear")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--peaks", action="store_true", help="print measured FP64/FP32/FP64-MMA/BF16-MMA peaks and exit")
    args = ap.parse_args()
    args.paths = set(args.paths.split(","))
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
