"""bench.py's multi-rank plumbing on the CPU: two `gloo` ranks (no GPU needed).

`bench.py --gpus N` runs one replica per GPU and reports the whole job's throughput from the
slowest rank's device time (max over ranks). These tests run the same helpers as two
processes over `gloo`: the process group comes up from the torchrun environment, the
barrier returns on both ranks, the max reaches every rank, and a rank that never joins ends
the other's collective with an error instead of a hang.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank: int, world: int, port: int):
    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), MPS_BENCH_BACKEND="gloo")
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)


def _rank_main(rank: int, port: int, q):
    _env(rank, 2, port)
    import bench
    import torch.distributed as dist
    try:
        world, r, local = bench.setup_dist()
        bench.barrier(world)
        # per-rank device time of K steps: the job is as fast as its slowest replica
        ms = [120.0, 150.0][r]
        worst = bench.allreduce_max(ms, world)
        q.put((r, world, local, dist.get_backend(), worst))
    finally:
        dist.destroy_process_group()


def _lonely_rank(port: int, q):
    _env(0, 2, port)
    import datetime

    import torch.distributed as dist
    try:
        # the second rank never starts: the rendezvous must end with an error, not hang
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=3))
        q.put("joined")
    except Exception as e:  # noqa: BLE001 - any error is the expected outcome
        q.put(type(e).__name__)


def test_two_gloo_ranks_agree_on_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
    assert all(p.exitcode == 0 for p in ps), [p.exitcode for p in ps]
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert [g[0] for g in got] == [0, 1]
    for r, world, local, backend, worst in got:
        assert world == 2 and local == r and backend == "gloo"
        assert worst == 150.0
    # the bench's aggregate: every rank's particles over the slowest rank's time
    nf, K = 384000, 200
    assert 2 * nf * K / (150.0 / 1e3) == pytest.approx(1.024e9)


def test_missing_rank_ends_with_an_error():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_lonely_rank, args=(_free_port(), q))
    p.start()
    p.join(120)
    if p.is_alive():
        p.kill()
        pytest.fail("the rendezvous of a missing rank did not time out")
    assert q.get(timeout=5) != "joined"


def test_reference_arm_under_two_ranks():
    """`bench.py --impl reference` launched as two ranks: rank 0 times the CPU restatement and
    prints the one JSON line, rank 1 does no work, and both exit 0."""
    import json
    import subprocess
    env = dict(os.environ, MPS_BENCH_BACKEND="gloo")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--workload", "dambreak_l0.02_small", "--steps", "2", "--warmup", "1"]
    res = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    lines = [l for l in res.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, res.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["n_gpus"] == 2
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0


def test_reference_arm_does_not_load_the_product():
    """The reference arm builds its workload with the oracle's own scene generator: after a
    run, neither the product package nor libmps_b200.so is loaded in its process, and its
    `config` is the one the GPU arm prints for the same workload."""
    import json
    import subprocess
    code = r"""
import argparse, json, sys
sys.path.insert(0, '.')
import bench
args = argparse.Namespace(workload='dambreak_l0.02_small', precision='f32', steps=2, warmup=1,
                          gpus=1)
bench.run_reference(args, 1, 0)
maps = open('/proc/self/maps').read()
print(json.dumps({'pkg': 'mps_cuda_b200' in sys.modules, 'so': 'libmps_b200' in maps}))
"""
    res = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                         timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [json.loads(l) for l in res.stdout.splitlines() if l.startswith("{")]
    line, loaded = lines[0], lines[-1]
    assert loaded == {"pkg": False, "so": False}
    import bench
    from oracle import scenes
    _, typ, _, _, _ = scenes.workload("dambreak_l0.02_small", "f32")
    assert line["config"] == bench.bench_config("dambreak_l0.02_small", "f32",
                                                int((typ == 0).sum()), int((typ != 0).sum()), 1)
    assert line["steps"] == 2 and line["warmup"] == 1


def test_step_roofline_sums_the_groups_per_step():
    """The whole-step HBM figure: every group's algorithmic bytes per launch times its
    launches, per timed step, over the step time; against the measured and the nominal peak."""
    import bench
    s, nf, m1, m2, K = 4, 1000, 100, 120, 5
    launches = {"pass_a": K, "pass_b": K, "pass_c": K, "gen_cull": 2 * K - 1,
                "bin_fluid": 2 * K, "bin_mirror": 2 * K}
    groups = {g: {"alg_bytes": bench.alg_bytes(g, s, nf, m1, m2), "launches": n}
              for g, n in launches.items()}
    r = bench.step_roofline(groups, K, 2.0, 5000.0)
    per_step = sum(bench.alg_bytes(g, s, nf, m1, m2) * n for g, n in launches.items()) / K
    assert r["alg_bytes_per_step"] == per_step
    assert abs(r["achieved"] - per_step / 2e-3 / 1e9) < 1e-9 * r["achieved"]
    assert abs(r["frac"] * 5000.0 - r["achieved"]) < 1e-9 * r["achieved"]
    assert abs(r["frac_nominal"] * 8000.0 - r["achieved"]) < 1e-9 * r["achieved"]
    assert abs(r["floor_ms_per_step"] - per_step / 5e12 * 1e3) < 1e-12
