#!/usr/bin/env python
"""Throughput of the explicit MPS step on B200: particle-updates/s.

A step is one pass of the dam-break time step (frsykzk/MPS_CUDA kernel.cu:1904-1941) over
all fluid particles of the workload; a particle-update is one fluid particle advanced
through one step. The default workload is the largest single-GPU scene: 6 144 000 fluid and
614 400 wall particles (l0 = 0.0025 m, 0.4 x 0.4 x 0.6 m column in a 1.6 x 0.4 x 0.8 m tank,
dt = 2.5e-5 s, bucket rebuild every step), FP32 (the reference's `typedef float real`), on
synthetic seeded inputs (there is no dataset).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours      : libmps_b200.so. `value` = device time of K steps (CUDA events on the solver's
            stream, L2 flushed between steps, max over ranks); `e2e` = the same steps
            through the C-ABI with the state uploaded from and read back into pinned host
            buffers every step; `roofline` = the dominant kernel group's algorithmic bytes
            per launch over its average launch time, timed live with CUDA events;
            `cpu_baseline` = the CPU oracle (OpenMP restatement of the reference's
            per-particle loops) on a bounded sample of the same workload, rank 0 only;
            `batched` = 64 uneven scenes in one handle against a per-scene loop;
            `adjoint` = the rollout adjoint's cost per step against a forward step at the
            48 000-particle adjoint workload, with its finite-difference agreement;
            `other_workloads` = the 384 000-particle dam break in FP32 and FP64.
reference : the reference's per-particle loops as that OpenMP CPU restatement (the
            reference itself has no CPU implementation), all host threads, rank 0 only, on
            the same workload built by the oracle's own scene generator (the product library
            is not loaded); `reference_cuda` adds the reference's own CUDA kernels (built for
            sm_100a from its sources) on the same workload and GPU, where that build is
            present.
Under torchrun (N > 1) each rank advances its own copy of the workload on its own GPU
(replicas: the step has no exchange between scenes), so `value` counts all ranks' updates.
"""
from __future__ import annotations

import argparse
import contextlib
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-updates/s"
WORKLOAD = "dambreak_l0.0025_6.1M"
L2_FLUSH_BYTES = 512 << 20  # > 126 MB L2

# Algorithmic bytes per unit (s = sizeof(real)): the state each kernel group must move,
# neighbour re-reads counted as cache hits.
#   pass A  (VscTrm + UpPcl1)  : read x, v; write x*, v*             12 s / fluid particle
#                                + read M1 mirrors                    3 s / mirror
#   pass B  (ChkCol + MkPrs)   : read x*, v*; write v**, P           10 s / fluid particle
#                                + read M1 mirrors                    3 s / mirror
#   pass C  (PrsGrdTrm+UpPcl2) : read x*, v**, P, pav; write x, v, pav 15 s / fluid particle
#                                + read M2 mirrors (x, P)              4 s / mirror
#   gen     (GenMRR + MRRinout): read x, P; write mirrors (x, P, slot) 4 s / fluid particle
#                                                                   + (4 s + 4) / mirror
#   bin     (bucket build)     : read key state, write sorted state  2 x payload / item


def alg_bytes(group: str, s: int, nf: int, m1: int, m2: int) -> float:
    return {
        "pass_a": 12 * s * nf + 3 * s * m1,
        "pass_b": 10 * s * nf + 3 * s * m1,
        "pass_c": 15 * s * nf + 4 * s * m2,
        "gen_cull": 4 * s * nf + (4 * s + 4) * (m1 + m2) / 2,
        "bin_fluid": 2 * (8 * s + 13) * nf,
        "bin_mirror": 2 * (4 * s + 4) * (m1 + m2) / 2,
    }[group]


# Arithmetic of the neighbour passes per unit of work (flops count a fused multiply-add as
# 2; square roots and divisions apart, since they cost several instructions each):
#   candidate test, list entry : dx, dy, dz and dot3                      8 flops
#   VscTrm pair                : d2 * d, u_j - u_i, 3 fma, sqrt, 2 l0 / t  10 flops, 1 sqrt, 1 div
#   ChkCol hit                 : u_i - u_j, dot3, f * (colfac / d2), 3 fma  15 flops, 1 div
#   MkPrs pair                 : sqrt, re/d - d/re                          1 flop, 1 sqrt, 2 div
#   PrsGrdTrm pair             : sqrt, (re/d - d/re) / d2, P_j - P_min,
#                                 (P_j - P_min) w, 3 fma                     9 flops, 1 sqrt, 3 div
# (kernel.cu:1062-1064, 1215-1220, 1346-1348, 1730-1735)
def pair_arith(work: dict, diag: dict) -> dict:
    """Per kernel group: (flops, square roots, divisions) of one step from the device's own
    counts (mps_get_work, mps_get_diag) of that step."""
    s = {k: float(np.sum(v, dtype=np.int64)) for k, v in diag.items() if k != "ndens"}
    va = s["vsc_f"] + s["vsc_m"]
    col = s["col_f"] + s["col_w"] + s["col_m"]
    prs = s["prs_f"] + s["prs_m"]
    grd = s["grd_f"] + s["grd_m"]
    n_list = float(work["list_entries"])
    return {
        "pass_a": (8 * float(work["visc_candidates"]) + 10 * va, va, va),
        "pass_b": (8 * float(work["list_candidates"]) + 8 * n_list + 15 * col + prs, prs,
                   col + 2 * prs),
        "pass_c": (16 * n_list + 9 * grd, grd, 3 * grd),
    }


NOMINAL_HBM_GBS = 8000.0  # B200 HBM3e, nominal (the measured copy bandwidth is the graded peak)


def step_roofline(groups: dict, steps: int, ms_per_step: float, peak_gbs: float) -> dict:
    """The whole step against HBM: the algorithmic bytes of every kernel group launched in
    `steps` timed steps (the table above, per launch, times its launches), per step, over the
    graph-replayed step time; as a fraction of the measured copy bandwidth and of the
    nominal 8 TB/s."""
    per_step = sum(v["alg_bytes"] * v["launches"] for v in groups.values()) / steps
    ach = per_step / (ms_per_step / 1e3) / 1e9
    return {"alg_bytes_per_step": per_step, "achieved": ach, "unit": "GB/s",
            "frac": ach / peak_gbs, "frac_nominal": ach / NOMINAL_HBM_GBS,
            "nominal_peak": NOMINAL_HBM_GBS,
            "floor_ms_per_step": per_step / (peak_gbs * 1e9) * 1e3}


def compute_roofline(ops, ms: float, ar: dict, f64: bool) -> dict:
    """Bound of one launch by the measured arithmetic rates: its flops at the fused
    multiply-add rate plus its square roots and divisions at theirs (they share the
    issue slots, so the times add)."""
    flops, nsq, ndv = ops
    pre = "fp64" if f64 else "fp32"
    t = (flops / ar[f"{pre}_fma_flops"] + nsq / ar[f"{pre}_sqrt_per_s"]
         + ndv / ar[f"{pre}_div_per_s"])
    ach = flops / (ms / 1e3)
    return {"flops_per_launch": flops, "sqrt_per_launch": nsq, "div_per_launch": ndv,
            "achieved_flops": ach, "flop_frac": ach / ar[f"{pre}_fma_flops"],
            "arith_bound_ms": 1e3 * t, "arith_frac": 1e3 * t / ms}


def issue_active(workload: str, precision: str):
    """Issue-active fraction per kernel group from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "issue_active.json")
    if not os.path.exists(p):
        return {}
    return json.load(open(p)).get(f"{workload}:{precision}", {})


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dram_traffic(workload: str, precision: str):
    """Per-launch DRAM bytes of each kernel group from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if not os.path.exists(p):
        return {}
    d = json.load(open(p))
    return d.get(f"{workload}:{precision}", {})


class ClockSampler:
    """nvidia-smi clocks and throttle reasons every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def setup_dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl" if os.environ.get("MPS_BENCH_BACKEND") != "gloo" else "gloo",
                                timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def allreduce_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def build_scene(workload: str, precision: str):
    from mps_cuda_b200 import F32, F32_N64, F64, configs, dambreak, dambreak_params
    desc, dt, _ = configs.WORKLOADS[workload]
    prec = {"f32": F32, "f64": F64, "f32n64": F32_N64}[precision]
    sc = dambreak(desc)
    p = dambreak_params(desc, dt=dt, precision=prec)
    rd = np.float64 if prec == F64 else np.float32
    return p, sc["typ"], sc["pos"].astype(rd), sc["vel"].astype(rd), sc["nrm"].astype(rd)


def build_scene_oracle(workload: str, precision: str):
    """The same workload from the oracle's own scene generator (tests/test_oracle_scene.py
    checks it byte for byte against build_scene), for the reference arm, which must not load
    the product library."""
    from oracle import scenes
    return scenes.workload(workload, precision)


def bench_config(workload: str, precision: str, nf: int, nw: int, world: int) -> dict:
    """The `config` object of both arms' JSON lines."""
    return {"workload": workload, "fluid_particles": nf, "wall_particles": nw,
            "precision": precision,
            "scene": "synthetic seeded dam break (walls on five tank faces, jittered lattice)",
            "l2": "state larger than the 126 MB L2; the GPU arm also flushes L2 (512 MiB "
                  "write) between timed steps",
            "parallelism": f"replicas x{world}"}


def cpu_oracle_rate(p, typ, pos, vel, nrm, budget_s: float, max_steps: int, warmup: int = 1):
    """Particle-updates/s of the OpenMP oracle over whole steps of the workload.

    `warmup` untimed steps, then at most `max_steps` timed steps, fewer where the warm-up
    steps' pace says they would take longer than `budget_s`. Returns (rate, steps timed,
    threads, seconds, warm-up steps run)."""
    from oracle.oracle import Oracle, lib, params_from
    threads = os.cpu_count() or 1
    lib().oracle_set_threads(threads)
    o = Oracle(params_from(p), typ, pos, vel, nrm)
    nf = int((typ == 0).sum())
    w = max(warmup, 1)
    t0 = time.perf_counter()
    o.step(1)
    t_step = time.perf_counter() - t0
    if w > 1:  # the remaining warm-up steps, as far as the budget allows
        w = 1 + int(min(w - 1, max(0.0, budget_s / 4) // max(t_step, 1e-9)))
        o.step(w - 1)
    k = int(max(1, min(max_steps, budget_s // max(t_step, 1e-9))))
    t0 = time.perf_counter()
    o.step(k)
    el = time.perf_counter() - t0
    o.close()
    return nf * k / el, k, threads, el, w


@contextlib.contextmanager
def _c_stdout_silenced():
    """Send what C code writes to file descriptor 1 to /dev/null for the duration."""
    import ctypes
    sys.stdout.flush()
    libc = ctypes.CDLL(None)
    saved = os.dup(1)
    null = os.open(os.devnull, os.O_WRONLY)
    os.dup2(null, 1)
    try:
        yield
    finally:
        libc.fflush(None)
        os.dup2(saved, 1)
        os.close(saved)
        os.close(null)


def reference_cuda_rate(p, typ, pos, vel, nrm, steps: int, warmup: int):
    """The reference's own CUDA kernels on the same workload, as a same-box reference point.

    oracle/_ref/libref_mps_{f32,f64}.so is `class MPS` built for sm_100a from the reference
    sources (oracle/ref_build.sh); its step is ClcMPS's loop body (kernel.cu:1904-1935),
    default stream, a device synchronise after every kernel as the reference does. Timed by
    wall clock around that synchronised loop, L2 not flushed. None where the library or a GPU
    is missing, or for the mixed precision the reference does not have.
    """
    if p.precision not in (0, 1):  # float or double: the reference has no mixed precision
        return None
    from oracle import refbind
    prec = p.precision
    if not refbind.available(prec):
        return None
    import torch
    if not torch.cuda.is_available():
        return None
    torch.cuda.set_device(0)
    with _c_stdout_silenced():  # SetPara prints its constants; keep stdout to the JSON line
        ref = refbind.Reference(p, typ, pos, vel, nrm)
        ref.step(max(warmup, 1))
        t0 = time.perf_counter()
        ref.step(steps)
        el = time.perf_counter() - t0
    nf = int((typ == 0).sum())
    return {"value": nf * steps / el, "unit": "particle-updates/s", "ms_per_step": 1e3 * el / steps,
            "steps": steps, "warmup": max(warmup, 1),
            "implementation": "the reference's class MPS kernels built for sm_100a, its own "
                              "synchronised step loop, timed by wall clock"}


def run_reference(args, world, rank):
    if rank != 0:
        return
    p, typ, pos, vel, nrm = build_scene_oracle(args.workload, args.precision)
    nf, nw = int((typ == 0).sum()), int((typ != 0).sum())
    rate, k, threads, el, w = cpu_oracle_rate(p, typ, pos, vel, nrm, budget_s=150.0,
                                              max_steps=args.steps, warmup=args.warmup)
    ref_cuda = reference_cuda_rate(p, typ, pos, vel, nrm, steps=args.steps,
                                   warmup=max(args.warmup, 3))
    sample = (f"{k} whole steps of the {args.workload} workload ({nf} fluid particles) after "
              f"{w} warm-up step(s), {threads} OpenMP threads")
    line = {"metric": METRIC, "value": rate, "unit": "particle-updates/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": k, "warmup": w,
            "ms_per_step": 1e3 * el / k, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
            "config": bench_config(args.workload, args.precision, nf, nw, world),
            "implementation": "OpenMP CPU restatement of the reference's per-particle loops "
                              "(the reference has no CPU path), scene from the oracle's own "
                              "generator",
            "cpu_baseline": {"value": rate, "unit": "particle-updates/s", "cores": threads,
                             "kind": "port", "sample": sample},
            "e2e": {"value": rate, "unit": "particle-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "reference_cuda": ref_cuda}
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local):
    import torch

    from mps_cuda_b200 import MPS, select_device
    from mps_cuda_b200 import _lib as L

    torch.cuda.set_device(local)
    select_device(local)
    p, typ, pos, vel, nrm = build_scene(args.workload, args.precision)
    nf = int((typ == 0).sum())
    s = 8 if args.precision == "f64" else 4
    g = MPS(p, typ, pos, vel, nrm)
    stream = torch.cuda.Stream()
    g.set_stream(stream.cuda_stream)
    # the library's tuned shapes for this scene (mps_autotune restores the state it tried
    # them on), as a user calls it once per handle
    tuned = None if args.no_tune else g.autotune(3)
    # shapes forced from the command line (profiling one variant), after the tuner
    if args.staging is not None:
        g.set_option(L.OPT_STAGING, args.staging)
    if args.candidate_batch is not None:
        g.set_option(L.OPT_CANDIDATE_BATCH, args.candidate_batch)
    g.set_option(L.OPT_GRAPH, 1)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    # warm-up (also captures the step graph)
    for _ in range(max(args.warmup, 3)):
        g.step(1)
    g.synchronize()

    # ---- timed region: K steps, L2 flushed between steps (outside the events) ----------
    K = args.steps
    # the state the timed steps start from: the per-kernel split below replays the same
    # simulated steps (a dam break's steps grow slower as the column collapses, so later
    # steps would not describe the timed ones)
    start = g.state()
    e0 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    e1 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    l0 = g.counters()["kernel_launches"]
    barrier(world)
    torch.cuda.synchronize()
    clk = ClockSampler(local).__enter__()  # sampled through every measured loop below
    w0 = time.perf_counter()
    # an NVTX range marks the timed steps, so that a profiler can be limited to them
    # (ncu --nvtx --nvtx-include "timed_steps/") past the tuner's trial steps
    torch.cuda.nvtx.range_push("timed_steps")
    with torch.cuda.stream(stream):
        for k in range(K):
            flush.fill_(float(k))
            e0[k].record(stream)
            g.step(1)
            e1[k].record(stream)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    barrier(world)
    launches = g.counters()["kernel_launches"] - l0
    dev_ms = sum(a.elapsed_time(b) for a, b in zip(e0, e1))
    dev_ms_max = allreduce_max(dev_ms, world)
    value = world * nf * K / (dev_ms_max / 1e3)
    cnt = g.counters()

    # ---- per-kernel device times (CUDA events on the solver's stream), same steps -----
    g.set_state(**start)
    g.set_option(L.OPT_TIMING, 1)
    g.timing(reset=True)
    with torch.cuda.stream(stream):
        for k in range(K):
            flush.fill_(float(k))
            g.step(1)
    tm = g.timing(reset=True)
    g.set_option(L.OPT_TIMING, 0)
    m1, m2 = cnt["n_mirror_1"], cnt["n_mirror_2"]
    groups = {}
    for name, (ms, n) in tm.items():
        if n:
            groups[name] = {"ms_per_launch": ms / n, "launches": n, "share": 0.0,
                            "alg_bytes": alg_bytes(name, s, nf, m1, m2)}
    total = sum(v["ms_per_launch"] * v["launches"] for v in groups.values())
    for v in groups.values():
        v["share"] = v["ms_per_launch"] * v["launches"] / total
    dom = max(groups, key=lambda k_: groups[k_]["ms_per_launch"] * groups[k_]["launches"])
    peak, peak_kind = peaks()
    ach = groups[dom]["alg_bytes"] / (groups[dom]["ms_per_launch"] / 1e3) / 1e9
    traffic = dram_traffic(args.workload, args.precision).get(dom)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": ach / peak, "traffic": traffic, "peak_source": peak_kind,
                "alg_bytes_per_launch": groups[dom]["alg_bytes"],
                "ms_per_launch": groups[dom]["ms_per_launch"]}

    # ---- companion compute roofline: the passes' pair arithmetic against the device's
    # own measured FMA / sqrt / division rates, the device counting its work in four
    # steps spread over the timed steps (replayed from their start) ---------------------
    compute = None
    if not args.no_compute:
        from mps_cuda_b200 import measure_arith
        ar = measure_arith()
        g.set_state(**start)
        samples = []
        for i in range(4):
            g.step(max(K // 4 - 1, 0))
            w0 = g.work()
            g.set_option(L.OPT_DIAG, 1)
            g.step(1)
            g.set_option(L.OPT_DIAG, 0)
            w1 = g.work()
            samples.append(pair_arith({k: w1[k] - w0[k] for k in w1}, g.diag()))
        ops = {k_: tuple(float(np.mean([sm[k_][j] for sm in samples])) for j in range(3))
               for k_ in samples[0]}
        ia = issue_active(args.workload, args.precision)
        compute = {"arith_peaks": ar, "issue_active_source": "profiles/issue_active.json (ncu)",
                   "groups": {}}
        for k_, o_ in ops.items():
            if k_ in groups:
                compute["groups"][k_] = compute_roofline(o_, groups[k_]["ms_per_launch"], ar,
                                                         args.precision == "f64")
                compute["groups"][k_]["issue_active"] = ia.get(k_)
        if dom in compute["groups"]:
            roofline["flop_frac"] = compute["groups"][dom]["flop_frac"]
            roofline["arith_frac"] = compute["groups"][dom]["arith_frac"]
            roofline["issue_active"] = compute["groups"][dom]["issue_active"]

    # ---- end to end through the C-ABI with pinned host buffers --------------------------
    e2e = None
    if not args.no_e2e:
        # A step reads typ, pos, vel and the running pav sum; it writes those and prs.
        # acc is ChkCol's scratch and zero between steps (kernel.cu:1146, 1826), and the
        # pressures a step starts from only reach the first mirror generation's PrsM, which
        # no later term reads (VscTrm, ChkCol and MkPrs use mirror positions only).
        st0 = start  # the same simulated steps as the timed region
        ins, outs = ("typ", "pos", "vel", "pav"), ("typ", "pos", "vel", "prs", "pav")

        def pinned_like(keys):
            return {k: torch.empty(st0[k].shape, dtype=torch.from_numpy(st0[k][:1].copy()).dtype,
                                   pin_memory=True).numpy() for k in keys}
        bufs = [pinned_like(outs), pinned_like(outs)]
        for k in outs:
            bufs[0][k][...] = st0[k]
        h2d = sum(bufs[0][k].nbytes for k in ins)
        d2h = sum(bufs[0][k].nbytes for k in outs)
        g.set_stream(0)
        barrier(world)
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        for k in range(K):
            src, dst = bufs[k % 2], bufs[(k + 1) % 2]
            g.set_state(**{f: src[f] for f in ins})  # this step's input from pinned host memory
            g.step(1)
            g.state(out=dst)                           # and its result back
        el = time.perf_counter() - w0
        el = allreduce_max(el, world)
        e2e = {"value": world * nf * K / el, "unit": "particle-updates/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": 1e3 * el / K}

    batched = None
    if not args.no_batched:
        batched = measure_batched(args, stream, flush, min(K, 50))
    adjoint = None
    if not args.no_adjoint:
        adjoint = measure_adjoint(stream)
    extra = None
    if not args.no_extra:
        # the 384 000-particle dam break in FP32 and FP64 (the reference dtype of its config)
        extra = [measure_workload(w_, pr_, stream, flush, min(K, 50))
                 for w_, pr_ in (("dambreak_l0.005_384k", "f32"), ("dambreak_l0.005_384k", "f64"))
                 if (w_, pr_) != (args.workload, args.precision)]
    clk.__exit__(None, None, None)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, k, threads, el, w = cpu_oracle_rate(p, typ, pos, vel, nrm, budget_s=20.0,
                                                  max_steps=200)
        cpu = {"value": rate, "unit": "particle-updates/s", "cores": threads, "kind": "port",
               "sample": f"{k} whole steps of the same workload after {w} warm-up step(s) "
                         f"({el:.1f} s)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "particle-updates/s", "n_gpus": world,
            "steps": K, "warmup": max(args.warmup, 3), "ms_per_step": dev_ms_max / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": args.precision, "data": "synthetic",
            "config": bench_config(args.workload, args.precision, nf, int((typ != 0).sum()),
                                   world),
            "graph": True, "tuned_shapes": tuned,
            "clocks": clk.summary(), "wall_ms_per_step": 1e3 * wall / K,
            "e2e": e2e, "gpu_launches": launches,
            "roofline": roofline, "compute_roofline": compute, "kernel_groups": groups,
            "step_roofline": step_roofline(groups, K, dev_ms_max / K, peak),
            "cpu_baseline": cpu,
            "batched": batched,
            "adjoint": adjoint,
            "other_workloads": extra,
            "counters": {k: v for k, v in cnt.items() if k != "kernel_launches"},
        }
        print(json.dumps(line), flush=True)
    g.close()


def measure_workload(workload: str, precision: str, stream, flush, K: int):
    """Device time of K graph-replayed steps of another workload or precision (L2 flushed
    between steps), with the step's per-group split."""
    import torch

    from mps_cuda_b200 import MPS
    from mps_cuda_b200 import _lib as L
    p, typ, pos, vel, nrm = build_scene(workload, precision)
    nf = int((typ == 0).sum())
    g = MPS(p, typ, pos, vel, nrm)
    g.set_stream(stream.cuda_stream)
    tuned = g.autotune(3)  # as for the headline workload: the handle's own tuned shapes
    g.set_option(L.OPT_GRAPH, 1)
    for _ in range(3):
        g.step(1)
    g.synchronize()
    e0 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    e1 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    with torch.cuda.stream(stream):
        for k in range(K):
            flush.fill_(float(k))
            e0[k].record(stream)
            g.step(1)
            e1[k].record(stream)
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in zip(e0, e1)) / K
    g.set_option(L.OPT_TIMING, 1)
    g.timing(reset=True)
    with torch.cuda.stream(stream):
        for k in range(min(K, 10)):
            flush.fill_(float(k))
            g.step(1)
    tm = g.timing(reset=True)
    cnt = g.counters()
    g.close()
    return {"workload": workload, "precision": precision, "fluid_particles": nf,
            "wall_particles": int((typ != 0).sum()), "steps": K, "ms_per_step": ms,
            "value": nf / (ms / 1e3), "unit": "particle-updates/s",
            "kernel_groups_ms_per_launch": {k: v[0] / v[1] for k, v in tm.items() if v[1]},
            "tuned_shapes": tuned, "deleted": cnt["n_deleted"], "errors": {k: v for k, v in cnt.items() if k.startswith("err")}}


def measure_adjoint(stream):
    """Adjoint workload: 48 000-particle dam break, FP64, 200 steps, checkpoints every 20.

    forward : device time of one graph-replayed step (CUDA events, 200 steps).
    adjoint : device time of mps_adjoint_backward over the recorded rollout (segment
              replays included) per step, CUDA events on the handle's stream.
    fd      : gradients of the dam-break loss (centroid and mean height beyond x = 0.7 m
              against the rollout at nu = 2e-6) against central differences: viscosity at
              the relative step 1e-4, the initial velocities along a uniform shift in x at 1e-7
              (collision onsets and wall events make the rollout piecewise smooth in them).
    """
    import math

    import torch

    from mps_cuda_b200 import _lib as L
    from mps_cuda_b200 import configs
    from mps_cuda_b200.adjoint import (RolloutProblem, dambreak_loss, loss_target, rollout,
                                       rollout_loss)

    desc, dt, steps = configs.WORKLOADS["adjoint_l0.01_48k"]
    pr = RolloutProblem(desc, dt=dt, steps=steps, every=20)
    f = pr.fluid
    v0 = pr.vel[:, f].copy()
    nu = configs.NU
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    h = pr.solver(nu, v0)
    h.set_stream(stream.cuda_stream)
    h.set_option(L.OPT_GRAPH, 1)
    h.step(3)
    h.synchronize()
    e0, e1 = ev(), ev()
    e0.record(stream)
    h.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    fwd = e0.elapsed_time(e1) / steps
    h.close()

    h = pr.solver(nu, v0)
    h.set_stream(stream.cuda_stream)
    h.set_option(L.OPT_GRAPH, 1)
    h.adjoint_record(steps, pr.every)
    lam = np.zeros((3, h.n))
    lam[:, f] = 1.0
    h.adjoint_backward(lam, None)  # warm-up
    e0, e1 = ev(), ev()
    e0.record(stream)
    h.adjoint_backward(lam, None)
    e1.record(stream)
    torch.cuda.synchronize()
    bwd = e0.elapsed_time(e1) / steps
    h.close()

    target = loss_target(pr, 2e-6, v0)
    nu_t = torch.tensor(nu, dtype=torch.float64, requires_grad=True)
    vel_t = torch.tensor(v0, dtype=torch.float64, requires_grad=True)
    pos, _, alive = rollout(nu_t, vel_t, pr)
    loss = dambreak_loss(pos, alive, torch.tensor(target))
    loss.backward()
    gnu, gv = float(nu_t.grad), vel_t.grad.numpy()
    hn = 1e-4 * nu
    fd_nu = (rollout_loss(pr, nu + hn, v0, target) - rollout_loss(pr, nu - hn, v0, target)) / (2 * hn)
    d = np.zeros(v0.shape)
    d[0] = 1.0  # every initial fluid velocity shifted in x
    eps = 1e-7 * float(np.sqrt(np.mean(v0 ** 2)))
    fd_v = (rollout_loss(pr, nu, v0 + eps * d, target)
            - rollout_loss(pr, nu, v0 - eps * d, target)) / (2 * eps)
    ad_v = math.fsum((gv * d).ravel())
    rel = lambda a, b: abs(a - b) / max(abs(a), abs(b), 1e-300)  # noqa: E731
    return {"workload": "adjoint_l0.01_48k", "fluid_particles": int(f.size), "steps": steps,
            "checkpoint_every": pr.every, "precision": "f64",
            "forward_ms_per_step": fwd, "adjoint_ms_per_step": bwd,
            "adjoint_over_forward": bwd / fwd,
            "loss": float(loss.detach()), "grad_nu": gnu, "fd_grad_nu": fd_nu,
            "fd_rel_err_nu": rel(gnu, fd_nu), "grad_vel0_dir": ad_v, "fd_grad_vel0_dir": fd_v,
            "fd_rel_err_vel0": rel(ad_v, fd_v),
            "fd_steps": {"nu": 1e-4, "vel0": 1e-7},
            "fd_direction_vel0": "every initial fluid velocity shifted in x"}


def measure_batched(args, stream, flush, K: int):
    """64 uneven dam breaks (FP32 state, FP64 number density, per-scene dt from CFL 0.2):
    one handle advancing all scenes per graph launch vs the per-scene loop (64 handles, one
    graph launch each per step, on the same stream). Device time, L2 flushed between steps."""
    import torch

    from mps_cuda_b200 import F32_N64, MPS, MPSBatch, configs, dambreak, dambreak_params
    from mps_cuda_b200 import _lib as L

    scenes = configs.batched_scenes()
    parts, params = [], []
    for desc, dt in scenes:
        sc = dambreak(desc)
        parts.append(sc)
        params.append(dambreak_params(desc, dt=dt, precision=F32_N64))
    counts = [p_["typ"].shape[0] for p_ in parts]
    nfl = sum(int((p_["typ"] == 0).sum()) for p_ in parts)
    cat = lambda k: np.concatenate([p_[k] for p_ in parts], axis=-1)
    f32 = lambda a: a.astype(np.float32)

    def timed(step_fn):
        e0 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
        e1 = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            for k in range(K):
                flush.fill_(float(k))
                e0[k].record(stream)
                step_fn()
                e1[k].record(stream)
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in zip(e0, e1))

    b = MPSBatch(params, cat("typ"), f32(cat("pos")), f32(cat("vel")), f32(cat("nrm")), counts=counts)
    b.set_stream(stream.cuda_stream)
    b.set_option(L.OPT_GRAPH, 1)
    b.step(3)
    ms_default = timed(lambda: b.step(1))  # default shapes: 128 threads, global walk
    tuned = b.autotune(3)
    b.set_option(L.OPT_GRAPH, 1)
    b.step(3)
    ms_batch = timed(lambda: b.step(1))
    # the kernels' own device time per step (CUDA events around each kernel group, no
    # graph): what a persistent step could at most save is the rest
    b.set_option(L.OPT_TIMING, 1)
    b.timing(reset=True)
    with torch.cuda.stream(stream):
        for k in range(min(K, 10)):
            flush.fill_(float(k))
            b.step(1)
    tm = b.timing(reset=True)
    b.set_option(L.OPT_TIMING, 0)
    kern_ms = sum(v[0] for v in tm.values()) / min(K, 10)
    hs = []
    for pp, pt in zip(params, parts):
        h = MPS(pp, pt["typ"], f32(pt["pos"]), f32(pt["vel"]), f32(pt["nrm"]))
        h.set_stream(stream.cuda_stream)
        h.set_option(L.OPT_GRAPH, 1)
        h.step(3)
        hs.append(h)

    def loop():
        for h in hs:
            h.step(1)
    ms_loop = timed(loop)
    for h in hs:
        h.close()
    b.close()
    return {"scenes": len(scenes), "fluid_particles": nfl,
            "particles_min": int(min(counts)), "particles_max": int(max(counts)),
            "precision": "f32 state, f64 number density", "steps": K,
            "value": nfl * K / (ms_batch / 1e3), "ms_per_step": ms_batch / K,
            "per_scene_loop_value": nfl * K / (ms_loop / 1e3), "per_scene_loop_ms_per_step": ms_loop / K,
            "speedup_vs_per_scene_loop": ms_loop / ms_batch, "tuned_shapes": tuned,
            "default_shapes_ms_per_step": ms_default / K, "tuned_gain": ms_default / ms_batch,
            "kernel_groups_ms_per_step": kern_ms,
            "launch_gap_ms_per_step": ms_batch / K - kern_ms,
            "unit": "particle-updates/s"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--precision", choices=["f32", "f64", "f32n64"], default="f32")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-extra", action="store_true")
    ap.add_argument("--no-compute", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--staging", type=int, choices=[0, 1, 2], default=None,
                    help="force pass A's staging mode (0 global, 1 positions, 2 velocities)")
    ap.add_argument("--candidate-batch", type=int, choices=[2, 4, 8], default=None,
                    help="force pass A's candidates per batch")
    args = ap.parse_args()
    world, rank, local = setup_dist()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
