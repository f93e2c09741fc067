#!/usr/bin/env python
"""Benchmark: complex-Langevin steps/s on the 128^3, N = 50 polyelectrolyte
workload (L = 64 b, bead density 0.5 b^-3, v = 0.1 b^3, lB = 1 b, divalent
counterions, 1:1 salt at 0.05 b^-3, full stress tensor and isotropic
pressure every step, seeded Langevin noise, complex64 propagators and fields
with FP64 reductions).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one full predictor-corrector CL step (two density evaluations,
each one forward chain sweep plus the pair-density and pair-stress kernels,
since the uniform chain is mirror-symmetric; observables; update).  Under torchrun each rank
runs its own independent replica (different seed): weak scaling, no
collective in the data path; the elapsed time is the max over ranks.

Prints one JSON line.  `--impl reference` times the reference's own CUDA
build (oracle/_ref/ref_harness, built from the reference sources by
oracle/build_ref.sh) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "CL steps/s at 128^3 N=50"
UNIT = "steps/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp32", "fp64"], default="fp32")
    ap.add_argument("--scheme", choices=["si", "pc"], default="si")
    ap.add_argument("--checkpoint-every", type=int, default=10,
                    help="device checkpoint interval; a non-finite step rolls back to it (0: off)")
    ap.add_argument("--grid", type=int, default=128, help="override the grid (small smoke runs only)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-line", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cufft", action="store_true", help="skip the cuFFT segment-step comparison")
    ap.add_argument("--no-graph", action="store_true",
                    help="time the steps as individual launches instead of replaying a captured CUDA graph")
    ap.add_argument("--time-to-pi", action="store_true",
                    help="instead of the throughput line: time for Pi and mu to reach 1%% of the complex128 "
                         "semi-implicit dt=0.005 result, learned complex64 at dt=0.02 against plain runs")
    ap.add_argument("--ttp-time", type=float, default=20.0, help="simulated time of each time-to-Pi run")
    ap.add_argument("--ttp-case", choices=["w5", "w2"], default="w5",
                    help="time-to-Pi workload: w5 = the 128^3 divalent system (scaled by --grid), "
                         "w2 = the 64^3 N=50 monovalent system")
    ap.add_argument("--ttp-dts", type=lambda x: [float(v) for v in x.split(",")], default=[0.01, 0.02],
                    help="step sizes of the complex64 plain and learned runs (comma separated)")
    ap.add_argument("--ttp-checkpoint-every", type=int, default=100,
                    help="device checkpoint interval of the time-to-Pi runs (the reference's Ntmp)")
    ap.add_argument("--ttp-max-restarts", type=int, default=1000,
                    help="rollbacks allowed in a time-to-Pi run (the reference's max_nan_restarts)")
    ap.add_argument("--ttp-seed-runs", type=int, default=0,
                    help="extra complex128 runs at the target step with other noise seeds (spread of the target)")
    ap.add_argument("--ttp-train-steps", type=int, default=2000,
                    help="plain semi-implicit steps whose statistics train the network")
    ap.add_argument("--replicas", type=int, default=0,
                    help="instead of the throughput line: this many independent replicas of uneven grids "
                         "(32^3-96^3), spread over the ranks and stepped as one CUDA graph per rank")
    ap.add_argument("--steps-per-graph", type=int, default=2)
    ap.add_argument("--replica-seeds", type=int, default=1,
                    help="replicas per system (seeds), for the ensemble statistics of --replicas")
    ap.add_argument("--long-run", type=int, default=0,
                    help="instead of the throughput line: this many steps of the 128^3 workload with device "
                         "time averages of the record (Nss = 10, 10 blocks) and the capped rollback")
    ap.add_argument("--long-precision", choices=["fp32", "fp64"], default="fp32")
    ap.add_argument("--long-scheme", choices=["si", "pc"], default="si")
    ap.add_argument("--long-dt", type=float, default=0.005)
    ap.add_argument("--max-restarts", type=int, default=20,
                    help="rollbacks before a non-finite step ends a --long-run (the reference's max_nan_restarts)")
    ap.add_argument("--adaptive", type=float, default=0.0,
                    help="adaptive step bound u_ref for --long-run (0: fixed step)")
    ap.add_argument("--precision-report", action="store_true",
                    help="instead of the throughput line: complex64 against complex128 on the 64^3, N = 50 "
                         "workload, per observable (mean and standard error over 10 blocks)")
    ap.add_argument("--report-steps", type=int, default=5000)
    return ap.parse_args()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def step_roofline(prop_bytes, field, steps, npts, s_c, steps_per_s_gpu, peak):
    """Whole-step roofline: algorithmic bytes of one step = the propagator and
    pair passes (per-pass accounting in the engine) + the field-level passes
    (batched transforms, elementwise and reduction kernels, each counted by
    the fields it reads and writes), K_f = the latter in full-field units."""
    fbytes = sum(v["bytes"] for v in field.values()) / steps
    pbytes = prop_bytes / steps
    total = pbytes + fbytes
    achieved = total * steps_per_s_gpu / 1e9
    return {"bytes_per_step": total, "propagator_bytes_per_step": pbytes, "field_bytes_per_step": fbytes,
            "K_f": fbytes / (npts * s_c), "achieved": achieved, "unit": "GB/s", "frac": achieved / peak,
            "field_kinds": {k: {"launches": v["launches"] / steps, "bytes": v["bytes"] / steps,
                                "ms_per_step": v["ms"] / steps} for k, v in sorted(field.items())}}


def committed_traffic():
    """Per-launch DRAM bytes of the propagator passes from the committed ncu
    summary (profiles/propagator_passes_128cube_N50.md, lines 'traffic <kind> <bytes>')."""
    out = {}
    path = os.path.join(ROOT, "profiles", "propagator_passes_128cube_N50.md")
    if os.path.exists(path):
        for line in open(path):
            p = line.split()
            if len(p) == 3 and p[0] == "traffic":
                try:
                    out[p[1]] = float(p[2])
                except ValueError:
                    pass
    return out


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
        else:   # CPU runs of the rank logic (tests)
            dist.init_process_group("gloo", timeout=timedelta(seconds=120))
    return ws, rank, local


def dist_max(x: float, ws: int) -> float:
    if ws <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_sum(x: float, ws: int) -> float:
    if ws <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------
# CPU baseline: the FP64 oracle on the host cores
# ---------------------------------------------------------------------------
def cpu_baseline(case, derived, steps=2):
    """The FP64 oracle (the reference's step restated in C, OpenMP over all
    host cores) timed on `steps` full predictor-corrector steps of the
    workload itself, with noise and the full stress tensor and pressure (its
    observables re-solve the chains per component, as the reference does)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import pyoracle as po
    po.build()
    threads = po.lib().oracle_threads()
    o = po.Oracle(derived)
    om, ps = case.initial_fields()
    o.set_fields(om, ps)
    sigma = np.sqrt(2.0 * derived["dt"] / derived["dV"])
    rng = np.random.default_rng(3)
    times = []
    for _ in range(steps):
        eta = rng.standard_normal((len(derived["modes"]) + 1, case.size)) * sigma
        t0 = time.perf_counter()
        o.step(eta)
        times.append(time.perf_counter() - t0)
    o.close()
    step_s = sum(times) / len(times)
    return {"value": 1.0 / step_s, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": ("%d full FP64 predictor-corrector steps of the %s workload (%.1f s each, %s), timed one by "
                       "one; the oracle restates the reference's step including its per-component stress re-solves"
                       % (steps, case.name, step_s, ", ".join("%.1f" % t for t in times)))}


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------
def run_reference(args, ws, rank):
    if rank != 0:
        return 0
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    base = {"metric": METRIC, "unit": UNIT, "impl": "reference"}
    if not os.path.exists(harness):   # built by __graft_entry__.build() next to the reference sources
        base["unavailable"] = "reference CUDA build (oracle/_ref/ref_harness) is missing (run the build step first)"
        print(json.dumps(base))
        return 0
    from ftspolysol_b200.cases import workload
    case = workload(4, noise=True)
    if args.grid != 128:
        case = scaled_case(case, args.grid)
    work = tempfile.mkdtemp(prefix="ftsp_ref_")
    paths = case.write(work)
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    res = subprocess.run([harness, "time", os.path.basename(paths["param"]), paths["omega"], paths["psi"],
                          str(args.warmup), str(args.steps)], cwd=work, capture_output=True, text=True)
    ck = clocks.stop()
    if res.returncode != 0:
        base["unavailable"] = "reference CUDA build failed on this workload: " + res.stderr.strip()[-200:]
        print(json.dumps(base))
        return 0
    r = json.loads(res.stdout.strip().splitlines()[-1])
    value = r["steps_per_s"]
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["event_ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": case.name + ": 128^3 grid, L=64b, N=50, divalent counterions, 1:1 salt 0.05, "
                                                "full stress + isotropic pressure every step, seeded noise",
                       "scheme": "predictor-corrector (reference)", "l2": "inputs larger than L2"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                             "sample": "the reference's own CUDA build (FP64, cuFFT) on the same B200, %d timed steps"
                                       " after %d warm-up steps; one host thread drives it" % (args.steps, args.warmup)},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "clocks": ck, "restarts": r.get("restarts", 0)}
    print(json.dumps(line))
    return 0


def scaled_case(case, m):
    """The same chemistry on an m^3 grid (dL unchanged)."""
    c = case
    V = (m * c.dL) ** 3
    c.m = (m, m, m)
    c.species[0].num_chains = int(round(0.5 * V / c.species[0].N))
    if c.salt is not None:
        c.salt = dict(c.salt)
        c.salt["num_salt"] = int(round(0.05 * V))
    return c


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def graph_region(eng, steps, ws):
    """Steps replayed from a CUDA graph of two captured steps (launch gaps
    removed), CUDA events on the graph's stream; returns (ms, steps timed)."""
    import torch
    from ftspolysol_b200.engine import Batch
    b = Batch([eng], 2)
    stream = torch.cuda.ExternalStream(b.stream())
    b.step(1)
    b.sync()
    barrier(ws)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.step(steps // 2)
    e1.record(stream)
    b.sync()
    barrier(ws)
    b.close()
    return e0.elapsed_time(e1), 2 * (steps // 2)


def direct_region(eng, steps, ws, profile=False):
    """Steps launched kernel by kernel (no step graph); with profile, every
    propagator pass bracketed by CUDA events on the engine's stream."""
    import torch
    eng.set_step_graph(False)
    if profile:
        eng.profile(True)
    barrier(ws)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        eng.step_async()
    e1.record()
    torch.cuda.synchronize()
    barrier(ws)
    eng.set_step_graph(True)
    return e0.elapsed_time(e1)


def e2e_region(eng, om, ps, steps, ws):
    """End to end through the public API: every step copies its fields in
    from pinned host memory and its record out.  Pipelined (the value): the
    next step's fields go up with ftsp_set_fields_async while the current
    step runs (ftsp_step_async, a replay of the engine's captured step
    graph), then ftsp_read_status returns the record.  Serial (reported
    beside it): ftsp_set_fields then ftsp_step, one after the other."""
    import numpy as np
    import torch
    n_in = (eng.n_modes + 1) * eng.size
    host = torch.empty(2 * n_in, dtype=torch.float64, pin_memory=True)
    fields = np.concatenate([np.asarray(om).reshape(-1), np.asarray(ps).reshape(-1)])
    host.numpy()[:] = fields.view(np.float64)
    p_om = host.data_ptr()
    p_ps = host.data_ptr() + eng.n_modes * eng.size * 16
    ke = max(3, min(steps, 20))
    out_bytes = 16 * (eng.record_len + eng.n_species) + 8 * (eng.n_modes + 1)
    # serial
    eng.set_fields_ptr(p_om, p_ps)
    eng.step()
    torch.cuda.synchronize()
    barrier(ws)
    t0 = time.perf_counter()
    for _ in range(ke):
        eng.set_fields_ptr(p_om, p_ps)
        eng.step()
    t1 = time.perf_counter()
    barrier(ws)
    serial = ws * ke / dist_max(t1 - t0, ws)
    # pipelined
    eng.set_fields_async_ptr(p_om, p_ps)
    eng.step_async()
    eng.read_status()
    torch.cuda.synchronize()
    barrier(ws)
    t0 = time.perf_counter()
    eng.set_fields_async_ptr(p_om, p_ps)
    eng.step_async()
    for _ in range(ke - 1):
        eng.set_fields_async_ptr(p_om, p_ps)   # the next step's fields, beside the running step
        eng.read_status()                      # the running step's record
        eng.step_async()
    eng.read_status()
    t1 = time.perf_counter()
    barrier(ws)
    return {"value": ws * ke / dist_max(t1 - t0, ws), "unit": UNIT, "h2d_bytes_per_step": 16 * n_in,
            "d2h_bytes_per_step": out_bytes, "steps": ke,
            "api": "ftsp_set_fields_async (the next step's fields, host pinned, uploaded while the current step "
                   "runs) + ftsp_step_async + ftsp_read_status (record, Q, drift maxima out)",
            "serial": {"value": serial, "api": "ftsp_set_fields + ftsp_step, one after the other"}}


def cufft_segment(m, segments=49, reps=5):
    """The reference's segment step on the library FFT (polymer.cu:396-400,
    common.h:1079-1085): cuFFT forward C2C, one pointwise kernel (Phi/V), cuFFT
    inverse C2C, one pointwise kernel (exp(-W)) writing the next stored
    propagator; complex64, plans made once (torch.fft, which calls cuFFT),
    replayed from a CUDA graph of `segments` segment steps."""
    import torch
    dev = torch.device("cuda")
    g = torch.Generator(device=dev).manual_seed(5)
    k = 2 * torch.pi * torch.fft.fftfreq(m, d=0.5, device=dev, dtype=torch.float64)
    k2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2
    phiV = (torch.exp(-k2 / 6.0) / m ** 3).to(torch.float32)
    w = 0.1 * torch.randn((m, m, m), generator=g, device=dev, dtype=torch.float32)
    E = torch.exp(-w).to(torch.complex64)
    q = torch.ones((segments + 1, m, m, m), dtype=torch.complex64, device=dev)
    X = torch.empty((m, m, m), dtype=torch.complex64, device=dev)
    Y = torch.empty_like(X)

    def sweep():
        for s in range(segments):
            torch.fft.fftn(q[s], out=X)
            X.mul_(phiV)
            torch.fft.ifftn(X, norm="forward", out=Y)
            torch.mul(Y, E, out=q[s + 1])

    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(stream):
        for _ in range(2):
            sweep()
    torch.cuda.current_stream().wait_stream(stream)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        sweep()
    graph.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        graph.replay()
    e1.record()
    torch.cuda.synchronize()
    us_graph = e0.elapsed_time(e1) * 1e3 / (reps * segments)
    e0.record()
    for _ in range(reps):
        sweep()
    e1.record()
    torch.cuda.synchronize()
    us_eager = e0.elapsed_time(e1) * 1e3 / (reps * segments)
    del graph
    return {"us_per_segment_graph": us_graph, "us_per_segment_eager": us_eager, "segments": segments,
            "reps": reps, "grid": m, "dtype": "c64"}


def run_ours(args, ws, rank, local):
    import numpy as np
    import torch
    from ftspolysol_b200 import Engine, FP32, FP64, SCHEME_PC, SCHEME_SI
    from ftspolysol_b200.cases import workload
    from ftspolysol_b200.derive import derive

    torch.cuda.set_device(local)
    case = workload(4, noise=True)
    if args.grid != 128:
        case = scaled_case(case, args.grid)
    derived = derive(case)
    prec = FP32 if args.precision == "fp32" else FP64
    scheme = SCHEME_SI if args.scheme == "si" else SCHEME_PC
    eng = Engine(derived, precision=prec, noise=True, seed=1234 + rank, device=local, scheme=scheme,
                 restart_interval=args.checkpoint_every)
    om, ps = case.initial_fields()
    eng.set_fields(om, ps)
    for _ in range(args.warmup):
        eng.step_async()
    torch.cuda.synchronize()

    # timed region for `value`: no instrumentation
    clocks = ClockSampler(local)
    clocks.start()
    direct = args.no_graph or args.steps < 2
    if direct:
        ms = direct_region(eng, args.steps, ws)
        timed_steps = args.steps
    else:
        ms, timed_steps = graph_region(eng, args.steps, ws)
    ck = clocks.stop()
    ms_direct = None if direct else direct_region(eng, args.steps, ws)
    launches_per_step = eng.launches()
    status, rec, _ = eng.read_status()
    restarts = eng.restarts()
    ms_max = dist_max(ms, ws)
    value = ws * timed_steps / (ms_max * 1e-3)
    # a second timed region of the same length with every propagator pass
    # bracketed by CUDA events on the engine's stream: per-kernel durations
    ms_prof = direct_region(eng, args.steps, ws, profile=True)
    prof = eng.profile_read()
    eng.profile(False)

    # roofline of the dominant propagator pass (largest total device time)
    peak, peak_kind = measured_peak_hbm()
    field = {k: v for k, v in prof.items() if k.startswith("field_")}
    prof = {k: v for k, v in prof.items() if not k.startswith("field_")}
    dom = max(prof.items(), key=lambda kv: kv[1]["ms"])
    dname, dstat = dom
    per_launch_ms = dstat["ms"] / dstat["launches"]
    per_launch_bytes = dstat["bytes"] / dstat["launches"]
    achieved = per_launch_bytes / (per_launch_ms * 1e-3) / 1e9
    traffic = committed_traffic().get(dname)
    prop_ms = sum(v["ms"] for v in prof.values())
    prop_bytes = sum(v["bytes"] for v in prof.values())
    roofline = {"bound": "hbm", "kernel": dname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"
                if peak_kind == "measured" else "fallback 6650 GB/s",
                "traffic": traffic, "bytes_per_launch": per_launch_bytes, "ms_per_launch": per_launch_ms,
                "timing": "per-kernel CUDA events over a second timed region of %d steps (%.2f ms/step with "
                          "the events, %.2f ms/step without)" % (args.steps, ms_prof / args.steps, ms / timed_steps),
                "step": step_roofline(prop_bytes, field, args.steps, eng.size, 8 if prec == FP32 else 16,
                                      value / ws, peak),
                "all_propagator_passes": {"achieved": prop_bytes / (prop_ms * 1e-3) / 1e9,
                                          "share_of_step": prop_ms / ms_prof,
                                          "per_kind": {k: {"launches": v["launches"], "ms_per_launch": v["ms"] / v["launches"],
                                                           "GBps": v["bytes"] / v["ms"] * 1e-6}
                                                       for k, v in sorted(prof.items())}}}
    seg_us = None
    if "plane_fwd_mid" in prof and "bond_fwd" in prof:
        seg_us = 1e3 * (prof["plane_fwd_mid"]["ms"] / prof["plane_fwd_mid"]["launches"]
                        + prof["bond_fwd"]["ms"] / prof["bond_fwd"]["launches"])

    e2e = None if args.no_e2e else e2e_region(eng, om, ps, args.steps, ws)
    eng.close()

    extra = {}
    if not args.no_fp64_line and prec == FP32:
        # like for like with the reference build: complex128 throughout and the
        # reference's predictor-corrector scheme, timed exactly as `value`
        e64 = Engine(derived, precision=FP64, noise=True, seed=99 + rank, device=local, scheme=SCHEME_PC,
                     restart_interval=args.checkpoint_every)
        e64.set_fields(om, ps)
        for _ in range(args.warmup):
            e64.step_async()
        torch.cuda.synchronize()
        if direct:
            ms64, k64 = direct_region(e64, args.steps, ws), args.steps
        else:
            ms64, k64 = graph_region(e64, args.steps, ws)
        st64, _, _ = e64.read_status()
        ms64 = dist_max(ms64, ws)
        block = {"value": ws * k64 / (ms64 * 1e-3), "unit": UNIT, "ms_per_step": ms64 / k64, "steps": k64,
                 "warmup": args.warmup, "status": int(st64), "dtype": "c128",
                 "scheme": "predictor-corrector (the reference's scheme)",
                 "timed_as": "individual launches" if direct else "CUDA-graph replay of two captured steps"}
        if not args.no_e2e:
            block["e2e"] = e2e_region(e64, om, ps, args.steps, ws)
        e64.close()
        extra["fp64_pc"] = block

    if rank == 0 and ws == 1 and args.grid == 128 and not args.no_cufft:
        cf = cufft_segment(128)
        cf["ours_us_per_segment"] = seg_us
        cf["ours"] = ("plane_fwd_mid + bond_fwd per-launch CUDA-event times (one forward segment step: inverse yz, "
                      "exp(-W), store, forward yz; forward x, Phi/V, inverse x)")
        cf["speedup_graph"] = (cf["us_per_segment_graph"] / seg_us) if seg_us else None
        extra["cufft_segment_step"] = cf

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(case, derived)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": timed_steps,
                "warmup": args.warmup, "ms_per_step": ms_max / timed_steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "c64" if prec == FP32 else "c128",
                "data": "synthetic",
                "config": {"workload": case.name + ": %d^3 grid, L=%gb, N=50, divalent counterions, 1:1 salt 0.05, "
                                                   "full stress + isotropic pressure every step, seeded noise"
                                       % (case.m[0], case.L[0]),
                           "precision": ("complex64 fields and propagators, FP64 reductions" if prec == FP32
                                         else "complex128 throughout"),
                           "scheme": ("semi-implicit predictor-corrector (analytic linear-response preconditioner)"
                                      if scheme == SCHEME_SI else "predictor-corrector (reference scheme)"),
                           "replicas_per_gpu": 1,
                           "checkpoint_every": args.checkpoint_every,
                           "parallelism": "replicas (one independent system per GPU)",
                           "l2": "inputs larger than L2 (propagator storage %.2f GB per solve)"
                                 % (2 * 50 * derived_bytes(case, prec) / 1e9)},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches_per_step * timed_steps,
                "timed_as": ("individual launches" if direct else
                             "CUDA-graph replay of two captured steps (ftsp_batch_*); the same steps launched "
                             "one by one ran %.2f ms/step" % (ms_direct / args.steps)),
                "clocks": ck, "final_status": int(status), "restarts": int(restarts)}
        line.update(extra)
        print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# time to Pi: learned complex64 SI at dt = 0.02 against the plain runs
# ---------------------------------------------------------------------------
class _Trajectory:
    """Synchronous steps with a record each; rows get (wall s, sim time, Pi,
    mu, mu_ex), mu being the polymer's total chemical potential
    mu_ex + mu_self + mu_id (record entries idx).  A non-finite step is
    rolled back by the device on the next step to the last checkpoint (taken
    after every `every`-th step attempt that ends finite); the rows of the
    steps it undoes are dropped and the simulated time rewinds, as the
    reference rewrites its observable file after a restart
    (complexLangevin.cu:638-656).  After max_restarts rollbacks the run is
    over and `stopped` is set."""

    def __init__(self, eng, every, idx, t0, adaptive=False):
        self.eng, self.every, self.idx, self.t0, self.adaptive = eng, every, idx, t0, adaptive
        self.rows, self.attempts, self.ckpt_row, self.ckpt_sim = [], 0, 0, 0.0
        self.sim, self.bad, self.stopped = 0.0, 0, False

    def run(self, steps, dt):
        import time
        from ftspolysol_b200.engine import NonFinite
        for _ in range(steps):
            if self.stopped:
                return
            self.attempts += 1
            try:
                _, rec, _ = self.eng.step()
            except NonFinite:
                self.bad += 1
                del self.rows[self.ckpt_row:]
                self.sim = self.ckpt_sim
                if self.eng.rollback_exhausted():
                    self.stopped = True
                continue
            r = rec.real
            # with the adaptive step the step taken is dt_eff <= dt; records
            # are weighted by it (a time average), as the engine's own averages
            w = self.eng.step_info()[0] / dt if self.adaptive else 1.0
            self.sim += w * dt
            self.rows.append((time.perf_counter() - self.t0, self.sim, r[-1],
                              r[self.idx[0]] + r[self.idx[1]] + r[self.idx[2]], r[self.idx[0]], w))
            if self.attempts % self.every == 0:
                self.ckpt_row, self.ckpt_sim = len(self.rows), self.sim


def _wmean(h, c):
    return float((h[:, c] * h[:, 5]).sum() / h[:, 5].sum())


def _time_to_target(rows, target, tol=0.01, every=50, cols=(2, 3)):
    """Earliest wall time from which on every running estimate (time
    average of the observables `cols` (Pi, mu) over the second half of the
    trajectory so far, checked every `every` steps) stays within tol
    (relative) of target."""
    import numpy as np
    a = np.array(rows)
    checks = []
    for n in range(every, len(a) + 1, every):
        h = a[n // 2:n]
        ok = all(abs(_wmean(h, c) - target[c - 2]) <= tol * abs(target[c - 2]) for c in cols)
        checks.append((a[n - 1, 0], ok))
    t_hit = None
    for t, ok in reversed(checks):
        if not ok:
            break
        t_hit = t
    return t_hit


def run_time_to_pi(args, local):
    """Wall time for the running means of Pi and mu to settle within 1 % of
    the complex128 semi-implicit dt = 0.005 result: complex128 and complex64
    plain semi-implicit runs, and complex64 runs with the learned
    preconditioner at larger steps (trained on the force/increment
    statistics of plain dt = 0.005 steps, retrained online).  Every run
    covers the same simulated time; the target is the second-half mean of
    the complex128 run."""
    import time
    import numpy as np
    import torch
    from ftspolysol_b200 import Engine, FP32, FP64, SCHEME_SI
    from ftspolysol_b200.cases import workload
    from ftspolysol_b200.derive import derive

    torch.cuda.set_device(local)
    if args.ttp_case == "w2":
        case = workload(2, noise=True)
    else:
        case = workload(5, noise=True)
        if args.grid != 128:
            case = scaled_case(case, args.grid)
    d = derive(case)
    S, J = len(d["species"]), len(d["ions"])
    idx = (0, S + J, 2 * (S + J))   # mu_ex, mu_self, mu_id of the polymer
    om, ps = case.initial_fields()
    T = args.ttp_time
    salt = case.salt["num_salt"] / case.volume if case.salt else 0.0
    N = len(case.species[0].monomers)
    runs = {}

    every, cap = args.ttp_checkpoint_every, args.ttp_max_restarts

    def engine(prec, dt, seed=21):
        e = Engine(dict(d, dt=dt), precision=prec, scheme=SCHEME_SI, noise=True, seed=seed, device=local,
                   restart_interval=every, max_restarts=cap)
        e.set_fields(om, ps)
        if args.adaptive > 0:
            e.set_adaptive(args.adaptive)
        torch.cuda.synchronize()
        return e

    def plain(prec, dt, tag, seed=21):
        e = engine(prec, dt, seed)
        tr = _Trajectory(e, every, idx, time.perf_counter(), args.adaptive > 0)
        limit = 4 * int(round(T / dt))   # step attempts, rolled-back ones included
        while tr.sim < T - 0.5 * dt and not tr.stopped and tr.attempts < limit:
            tr.run(min(int(round((T - tr.sim) / dt)), limit - tr.attempts), dt)
        runs[tag] = {"rows": tr.rows, "dt": dt, "nonfinite_steps": tr.bad, "restarts": e.restarts(),
                     "stopped_at_cap": tr.stopped, "attempts": tr.attempts,
                     "wall_s": tr.rows[-1][0] if tr.rows else None}
        e.close()

    def learned(dt, tag):
        # plain SI steps at dt = 0.005 collect the statistics, Adam trains the
        # network, then steps of dt with the learned kernel, retrained online
        e = engine(FP32, 0.005)
        e.learn_configure(N=N, lB=case.lB, salt=salt, seed=11)
        tr = _Trajectory(e, every, idx, time.perf_counter(), args.adaptive > 0)
        ntrain = min(args.ttp_train_steps, int(round(T / 0.005)) // 2)
        e.learn_collect(True)
        tr.run(ntrain, 0.005)
        loss = e.learn_train(1500) if not tr.stopped else None
        valid = e.learn_stats()["valid_targets"]
        t_train = time.perf_counter() - tr.t0
        if not tr.stopped:
            e.set_dt(dt)
            e.learn_use(True)
            e.learn_reset()
        limit = tr.attempts + 4 * int(round((T - tr.sim) / dt))
        while tr.sim < T - 0.5 * dt and not tr.stopped and tr.attempts < limit:
            tr.run(min(200, int(round((T - tr.sim) / dt)), limit - tr.attempts), dt)
            if not tr.stopped:
                e.learn_train(200)
                e.learn_reset()
        st = e.learn_stats()
        runs[tag] = {"rows": tr.rows, "dt": dt, "nonfinite_steps": tr.bad, "restarts": e.restarts(),
                     "stopped_at_cap": tr.stopped, "attempts": tr.attempts,
                     "wall_s": tr.rows[-1][0] if tr.rows else None, "train_steps": ntrain, "train_wall_s": t_train,
                     "train_loss": loss, "valid_targets": valid, "fallback_steps": st["fallbacks"],
                     "judged_steps": st["checks"]}
        e.close()

    plain(FP64, 0.005, "c128_si_dt0.005")
    base_rows = np.array(runs["c128_si_dt0.005"]["rows"])
    half = base_rows[len(base_rows) // 2:]
    target = (_wmean(half, 2), _wmean(half, 3), _wmean(half, 4))
    bm = np.array([[_wmean(b, c) for c in (2, 3, 4)] for b in np.array_split(half, 10)])
    target_se = bm.std(axis=0, ddof=1) / np.sqrt(len(bm))
    # the target step with other noise seeds: how far apart independent
    # trajectories of the same length land (the resolution of the criterion)
    for k in range(args.ttp_seed_runs):
        plain(FP64, 0.005, "c128_si_dt0.005_seed%d" % (22 + k), seed=22 + k)
    plain(FP32, 0.005, "c64_si_dt0.005")
    for dt in args.ttp_dts:
        plain(FP32, dt, "c64_si_dt%g" % dt)
        learned(dt, "c64_learned_dt%g" % dt)

    out = {}
    for tag, r in runs.items():
        a = np.array(r["rows"])
        info = {k: v for k, v in r.items() if k != "rows"}
        if len(a) >= 2:
            h = a[len(a) // 2:]
            info.update({"steps": len(a), "Pi_mean": _wmean(h, 2), "mu_mean": _wmean(h, 3),
                         "mu_ex_mean": _wmean(h, 4),
                         "Pi_rel_err": _wmean(h, 2) / target[0] - 1.0,
                         "mu_rel_err": _wmean(h, 3) / target[1] - 1.0,
                         "mu_ex_abs_err": _wmean(h, 4) - target[2],
                         "time_to_1pct_s": _time_to_target(r["rows"], target),
                         "time_to_Pi_1pct_s": _time_to_target(r["rows"], target, cols=(2,))})
        else:
            info.update({"steps": len(a), "time_to_1pct_s": None})
        out[tag] = info
    base = out["c128_si_dt0.005"]["time_to_1pct_s"]
    best = None
    for tag, v in out.items():
        if tag.startswith("c64_learned") and v["time_to_1pct_s"] and (best is None or v["time_to_1pct_s"] < best[1]):
            best = (tag, v["time_to_1pct_s"])
    # the same with Pi alone (mu's statistical error can exceed 1 % at these lengths)
    base_pi = out["c128_si_dt0.005"].get("time_to_Pi_1pct_s")
    pi_only = {tag: v.get("time_to_Pi_1pct_s") for tag, v in out.items()}
    best_pi = min(((t, tag) for tag, t in pi_only.items() if tag.startswith("c64_learned") and t), default=None)
    print(json.dumps({"metric": "wall time for Pi and mu to settle within 1% of the complex128 semi-implicit "
                                "dt=0.005 result", "unit": "s", "higher_is_better": False,
                      "value": best[1] if best else None, "best_learned_run": best[0] if best else None,
                      "c128_time_to_1pct_s": base,
                      "speedup_vs_c128": (base / best[1]) if (base and best) else None,
                      "Pi_alone": {"time_to_1pct_s": pi_only, "best_learned_run": best_pi[1] if best_pi else None,
                                   "speedup_vs_c128": (base_pi / best_pi[0]) if (base_pi and best_pi) else None},
                      "seed_spread": {tag: {"Pi_rel_err": v.get("Pi_rel_err"), "mu_rel_err": v.get("mu_rel_err")}
                                      for tag, v in out.items() if tag.startswith("c128_si_dt0.005_seed")},
                      "target": {"Pi": target[0], "mu": target[1], "mu_ex": target[2],
                                 "Pi_se": float(target_se[0]), "mu_se": float(target_se[1]),
                                 "mu_ex_se": float(target_se[2])},
                      "criterion": "running means over the second half of each trajectory, checked every 50 steps, "
                                   "stay within 1% of the target from then on; mu = mu_ex + mu_self + mu_id of the "
                                   "polymer (mu_ex alone averages near zero: its absolute error is reported)",
                      "simulated_time": T,
                      "rollback": {"checkpoint_every": every, "max_restarts": cap,
                                   "adaptive_u_ref": args.adaptive or None},
                      "config": {"workload": case.name + ": %d^3, L=%gb, N=%d, %s counterions, salt %g"
                                 % (case.m[0], case.L[0], N,
                                    "divalent" if case.counterions["valence"] == 2.0 else "monovalent", salt)},
                      "data": "synthetic", "runs": out}))
    return 0


# ---------------------------------------------------------------------------
# long run: time-averaged observables of the 128^3 workload
# ---------------------------------------------------------------------------
def run_long(args, local):
    """`--long-run K` steps of the 128^3 workload (seeded noise, full stress),
    device time averages of the record (the reference's rule with Nss = 10,
    complexLangevin.cu:424-467, plus 10 blocks for the errors), device
    checkpoints every --checkpoint-every steps and the capped rollback
    (--max-restarts): the run stops when the cap is reached, as the
    reference's does.  With a checkpoint interval longer than the run, every
    rollback restores the initial fields (the policy of the reference
    harness's timing mode), so non-finite step counts compare directly."""
    import numpy as np
    import torch
    from ftspolysol_b200 import Engine, FP32, FP64, SCHEME_PC, SCHEME_SI
    from ftspolysol_b200.cases import workload
    from ftspolysol_b200.derive import derive

    torch.cuda.set_device(local)
    case = workload(4, noise=True, dt=args.long_dt)
    if args.grid != 128:
        case = scaled_case(case, args.grid)
    d = derive(case)
    prec = FP32 if args.long_precision == "fp32" else FP64
    scheme = SCHEME_SI if args.long_scheme == "si" else SCHEME_PC
    e = Engine(d, precision=prec, scheme=scheme, noise=True, seed=4321, device=local,
               restart_interval=args.checkpoint_every, max_restarts=args.max_restarts)
    om, ps = case.initial_fields()
    e.set_fields(om, ps)
    if args.adaptive > 0:
        e.set_adaptive(args.adaptive)
    K = args.long_run
    e.average_start(case.Nss, K, 10)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    done, stopped = 0, False
    while done < K and not stopped:
        n = min(200, K - done)
        for _ in range(n):
            e.step_async()
        done += n
        stopped = e.rollback_exhausted()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    mean, se, cnt = e.average_read()
    restarts = e.restarts()
    e.close()
    S, J = len(d["species"]), len(d["ions"])
    names = (["mu_ex_poly"] + ["mu_ex_ion%d" % j for j in range(J)] + ["mu_self_%d" % i for i in range(S + J)] +
             ["mu_id_%d" % i for i in range(S + J)] + ["H"] + ["stress_" + c for c in d["stress"]] + ["Pi"])
    print(json.dumps({"metric": "time-averaged observables of the 128^3 N=50 workload", "steps_requested": K,
                      "steps_taken": done, "records_averaged": cnt, "restarts": restarts, "stopped_at_cap": stopped,
                      "wall_s": wall, "steps_per_s": done / wall,
                      "config": {"workload": case.name + ": %d^3, L=%gb, N=50, divalent counterions, salt 0.05, "
                                 "full stress + Pi, seeded noise" % (case.m[0], case.L[0]),
                                 "precision": args.long_precision, "scheme": args.long_scheme, "dt": args.long_dt,
                                 "adaptive_u_ref": args.adaptive or None, "Nss": case.Nss,
                                 "checkpoint_every": args.checkpoint_every, "max_restarts": args.max_restarts},
                      "averages": {n: {"mean": float(m), "se": float(s)} for n, m, s in zip(names, mean, se)}}))
    return 0


# ---------------------------------------------------------------------------
# replicas: many independent systems of uneven size, one CUDA graph per rank
# ---------------------------------------------------------------------------
def run_replicas(args, ws, rank, local):
    import numpy as np
    import torch
    from ftspolysol_b200 import Engine, FP32, SCHEME_SI
    from ftspolysol_b200.derive import derive
    from ftspolysol_b200.engine import Batch
    from ftspolysol_b200 import replicas as R

    torch.cuda.set_device(local)
    cases_all = R.replica_set(args.replicas, seeds_per_system=args.replica_seeds)
    mine = R.assign([R.cost(c) for c in cases_all], ws)[rank]
    engines = []
    for i in mine:
        c = cases_all[i]
        e = Engine(derive(c), precision=FP32, scheme=SCHEME_SI, noise=True, seed=7000 + i, device=local,
                   restart_interval=10, autotune=True)
        om, ps = c.initial_fields()
        e.set_fields(om, ps)
        engines.append(e)
    K = max(1, args.steps // args.steps_per_graph)
    # the same steps launched one engine after another (no graph, one stream)
    for e in engines:
        e.step_async()
    torch.cuda.synchronize()
    barrier(ws)
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a0.record()
    for _ in range(K * args.steps_per_graph):
        for e in engines:
            e.step_async()
    a1.record()
    torch.cuda.synchronize()
    seq_ms = dist_max(a0.elapsed_time(a1), ws)
    # time averages of every replica's record over the timed steps (device
    # side, inside the graph): the batch warm-up steps are skipped
    warm = max(1, args.warmup // args.steps_per_graph)
    for e in engines:
        e.average_start(warm * args.steps_per_graph, K * args.steps_per_graph,
                        min(10, max(2, K * args.steps_per_graph // 4)))
    # one graph per rank: every replica on its own branch
    batch = Batch(engines, args.steps_per_graph)
    stream = torch.cuda.ExternalStream(batch.stream())
    batch.step(warm)
    batch.sync()
    barrier(ws)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    batch.step(K)
    e1.record(stream)
    batch.sync()
    ck = clocks.stop()
    barrier(ws)
    ms = dist_max(e0.elapsed_time(e1), ws)
    kernels = batch.launches_per_graph
    batch.close()
    tuned = {}
    for i, e in zip(mine, engines):
        t = e.tune_info()
        key = "%d^3" % cases_all[i].m[0]
        if key not in tuned or t["tuned"]:
            tuned[key] = {"compile_time_kernels": bool(t["compile_time"]), "max_radix": t["max_radix"],
                          "tile_width": t["tile_width"], "candidates": t["candidates"],
                          "fft_pair_ms": t["best_ms"], "default_fft_pair_ms": t["default_ms"]}
    results = {}
    for i, e in zip(mine, engines):
        st, rec, _ = e.read_status()
        mean, se, cnt = e.average_read()
        c = cases_all[i]
        h = 3 * (e.n_species + e.n_ions)   # record: mu_ex, mu_self, mu_id, H, Pi
        results[i] = {"status": int(st), "restarts": int(e.restarts()), "Pi_last": float(rec[-1].real),
                      "grid": c.m[0], "N": len(c.species[0].monomers), "salt": c.salt["num_salt"] / c.volume,
                      "records_averaged": cnt,
                      "Pi": (float(mean[-1]), float(se[-1])), "H": (float(mean[h]), float(se[h])),
                      "mu_ex": (float(mean[0]), float(se[0]))}
        e.close()
    results = R.gather(results, ws)
    keys = {i: R.system_key(cases_all[i]) for i in results}
    ens = R.ensemble(results, keys, ["Pi", "H", "mu_ex"])
    steps_done = dist_sum(len(mine) * K * args.steps_per_graph, ws)
    if rank == 0:
        by_grid = {}
        for r in results.values():
            g = by_grid.setdefault("%d^3" % r["grid"], {"replicas": 0, "restarts": 0})
            g["replicas"] += 1
            g["restarts"] += r["restarts"]
        print(json.dumps({
            "metric": "replica CL steps/s (%d independent replicas, 32^3-96^3 grids)" % args.replicas,
            "value": steps_done / (ms * 1e-3), "unit": "replica-steps/s", "n_gpus": ws,
            "steps": K * args.steps_per_graph, "warmup": args.warmup, "ms_per_step": ms / (K * args.steps_per_graph),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
            "config": {"workload": "%d replicas: grids 32/48/64/96^3 (a quarter each), L = 0.5 b x grid, N from "
                                   "{20, 32, 50}, salt 0.01-0.5 b^-3, own seeds; complex64 semi-implicit, dt 0.005"
                                   % args.replicas,
                       "placement": "longest-processing-time over %d rank(s)" % ws,
                       "graph": {"steps_per_graph": args.steps_per_graph, "kernels_per_graph_rank0": kernels},
                       "autotune_rank0": tuned},
            "sequential_value": steps_done / (seq_ms * 1e-3),
            "graph_speedup": seq_ms / ms,
            "clocks": ck,
            "replicas_by_grid": by_grid,
            "finite_replicas": sum(1 for r in results.values() if r["status"] == 0),
            "time_averages": {"rule": "records of the timed steps (the batch warm-up skipped), real parts, "
                                      "standard error from block means; per system: mean over its seeds and "
                                      "the standard error of that mean (a single seed keeps its block error)",
                              "seeds_per_system": args.replica_seeds,
                              "systems": {k: dict(v, **{"grid": results[min(i for i in results if keys[i] == k)]["grid"],
                                                        "N": results[min(i for i in results if keys[i] == k)]["N"],
                                                        "salt": results[min(i for i in results if keys[i] == k)]["salt"]})
                                          for k, v in sorted(ens.items())}}}))
    return 0


# ---------------------------------------------------------------------------
# precision report: complex64 propagators against complex128, same noise
# ---------------------------------------------------------------------------
def run_precision_report(args, local):
    import time
    import numpy as np
    import torch
    from ftspolysol_b200 import Engine, FP32, FP64, SCHEME_SI
    from ftspolysol_b200.cases import workload
    from ftspolysol_b200.derive import derive
    from ftspolysol_b200.engine import NonFinite

    torch.cuda.set_device(local)
    case = workload(2, noise=True)
    d = derive(case)
    om, ps = case.initial_fields()
    S, J = len(d["species"]), len(d["ions"])
    C = S + J
    names = ["mu_poly_ex", "H_real"] + ["stress_" + c for c in d["stress"]] + ["Pi"]
    idx = [0, 3 * C] + [3 * C + 1 + k for k in range(len(d["stress"]))] + [3 * C + 1 + len(d["stress"])]
    runs = {}
    for prec, tag in ((FP64, "c128"), (FP32, "c64")):
        e = Engine(d, precision=prec, scheme=SCHEME_SI, noise=True, seed=31, device=local)
        e.set_fields(om, ps)
        torch.cuda.synchronize()
        rows, first_bad = [], None
        t0 = time.perf_counter()
        for k in range(args.report_steps):
            try:
                _, rec, _ = e.step()
                rows.append([rec[i].real for i in idx])
            except NonFinite:
                first_bad = k + 1   # a runaway: the trajectory ends here
                break
        runs[tag] = {"rows": np.array(rows), "wall_s": time.perf_counter() - t0, "first_nonfinite_step": first_bad}
        e.close()
    L = min(len(runs["c128"]["rows"]), len(runs["c64"]["rows"]))
    a, b = runs["c128"]["rows"][:L], runs["c64"]["rows"][:L]
    start = L // 5   # equilibration discarded
    out = {}
    for j, n in enumerate(names):
        def blocks(x):
            x = x[start:, j]
            bl = np.array_split(x, 10)
            m = np.array([np.nanmean(q) for q in bl])
            return float(np.nanmean(m)), float(np.nanstd(m, ddof=1) / np.sqrt(len(m)))
        m64, s64 = blocks(a)
        m32, s32 = blocks(b)
        early = np.abs(b[:50, j] - a[:50, j]) / np.maximum(np.abs(a[:50, j]), 1e-12)
        out[n] = {"c128_mean": m64, "c128_se": s64, "c64_mean": m32, "c64_se": s32,
                  "difference": m32 - m64, "difference_in_se": (m32 - m64) / max(np.hypot(s64, s32), 1e-300),
                  "max_rel_diff_first_50_steps": float(np.nanmax(early))}
    print(json.dumps({"metric": "complex64 vs complex128 observables (block means)", "config": {
        "workload": case.name + ": 64^3, L=32b, N=50, monovalent counterions, salt 0.1, semi-implicit dt 0.005, "
                                "same noise in both runs; the steps both runs completed before a runaway, first "
                                "20% discarded, 10 blocks"},
        "steps_requested": args.report_steps, "steps_compared": L, "observables": out,
        "runs": {k: {kk: vv for kk, vv in v.items() if kk != "rows"} for k, v in runs.items()}}))
    return 0


def derived_bytes(case, prec):
    import numpy as np
    return int(np.prod(case.m)) * (8 if prec == 1 else 16)


def main():
    args = parse_args()
    ws, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            rc = run_reference(args, ws, rank)
        elif args.precision_report:
            rc = run_precision_report(args, local) if rank == 0 else 0
        elif args.replicas > 0:
            rc = run_replicas(args, ws, rank, local)
        elif args.time_to_pi:
            rc = run_time_to_pi(args, local) if rank == 0 else 0
        elif args.long_run > 0:
            rc = run_long(args, local) if rank == 0 else 0
        else:
            rc = run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
