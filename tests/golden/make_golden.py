"""Generate the golden vectors of the reference's own kernels (run on a machine with a GPU).

Runs frsykzk/MPS_CUDA's `class MPS` (built by oracle/ref_build.sh, driven through
oracle/ref_harness.cu) on a small seeded dam break and records the state after every method
call of two time steps of ClcMPS's loop body (kernel.cu:1904-1935): the fluid particles'
type, position, velocity, acceleration, pressure and averaged pressure, the live mirror
particles (slot, position, pressure), and the bucket of every particle read back from the
reference's linked lists. The CPU tests replay each method of the oracle from the recorded
input state and compare with the recorded output state.

    python tests/golden/make_golden.py [outdir] [--corrected | --6k]

With --corrected the same record is made with the reference's corrected-matrix d_PrsGrdTrm
(the #if 0 variant, kernel.cu:1434-1648, built by oracle/ref_build.sh as libref_mps_corr_*)
into ref_small_corr_{f32,f64}.npz. With --6k: the 6 000-particle dam break in FP64, its
second step method by method, into ref_6k_f64.npz (see main_6k).
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from mps_cuda_b200.solver import SceneDesc, dambreak, dambreak_params  # noqa: E402
from oracle import refbind  # noqa: E402

SCENE = SceneDesc(0.02, (0.24, 0.12, 0.24), (6, 4, 8), seed=3)
DT = 2e-4
RECORD_STEPS = (0, 3)
FIELDS = ("typ", "pos", "vel", "acc", "prs", "pav")


def params_array(p) -> np.ndarray:
    return np.array([p.pcl_dst, *p.min, *p.max, *p.g, p.knm_vsc, p.col_rat, p.dst_lmt_rat, p.rho,
                     p.snd, p.dt, p.umax, p.pmax, p.precision], np.float64)


def snapshot(ref, nf, tag, out):
    st = ref.state()
    for k in FIELDS:
        a = st[k]
        out[f"{tag}_{k}"] = a[..., :nf].copy()
    m = ref.mirrors()
    out[f"{tag}_mslot"] = m["slot"]
    out[f"{tag}_mpos"] = m["pos"]
    out[f"{tag}_mprs"] = m["prs"]
    out[f"{tag}_cell"] = ref.buckets()


def main(outdir: str, corrected: bool = False):
    os.makedirs(outdir, exist_ok=True)
    for prec, name in ((0, "f32"), (1, "f64")):
        dty = np.float64 if prec == 1 else np.float32
        sc = dambreak(SCENE)
        p = dambreak_params(SCENE, dt=DT, precision=prec)
        args = (sc["typ"], sc["pos"].astype(dty), sc["vel"].astype(dty), sc["nrm"].astype(dty))
        ref = refbind.Reference(p, *args, corrected=corrected)
        nf = int(np.sum(sc["typ"] == 0))
        assert np.all(sc["typ"][:nf] == 0) and np.all(sc["typ"][nf:] != 0)
        out = {"params": params_array(p), "typ": sc["typ"], "pos": args[1], "vel": args[2],
               "nrm": args[3], "nf": np.array(nf), "wllse": ref.wall_flags(),
               "phases": np.array(refbind.STEP_PHASES, np.int32),
               "record_steps": np.array(RECORD_STEPS, np.int32)}
        info = ref.info()
        out["ref_info"] = np.array([info[k] for k in sorted(info)], np.float64)
        out["ref_info_keys"] = np.array(sorted(info))
        for step in range(max(RECORD_STEPS) + 1):
            rec = step in RECORD_STEPS
            if rec:
                snapshot(ref, nf, f"s{step}_k0", out)
            for k, ph in enumerate(refbind.STEP_PHASES):
                ref.phase(ph)
                if rec:
                    snapshot(ref, nf, f"s{step}_k{k + 1}", out)
        path = os.path.join(outdir, f"ref_small_{'corr_' if corrected else ''}{name}.npz")
        np.savez_compressed(path, **out)
        print(path, os.path.getsize(path))


# what each method of the step can change (the 6k record stores only these, and only where
# they differ from the state before the method)
CHANGES = {0: ("cell",), 2: ("mirrors",), 3: ("mirrors",), 4: ("mirrors",), 5: ("acc",),
           6: ("typ", "pos", "vel", "acc", "prs"), 7: ("vel", "acc"), 8: ("prs",), 9: ("acc",),
           10: ("typ", "pos", "vel", "acc", "prs", "pav")}
WORKLOAD_6K = "dambreak_l0.02_6k"


def main_6k(outdir: str):
    """The 6 000-particle dam break (FP64): its first step whole, then its second step method
    by method. The state before the second step is stored whole (fluid fields, mirrors,
    buckets), after each method only what that method changed. The particles are the
    workload's own seeded scene, regenerated by the test."""
    from mps_cuda_b200 import configs
    os.makedirs(outdir, exist_ok=True)
    desc, dt, _ = configs.WORKLOADS[WORKLOAD_6K]
    sc = dambreak(desc)
    p = dambreak_params(desc, dt=dt, precision=1)
    args = (sc["typ"], sc["pos"], sc["vel"], sc["nrm"])
    ref = refbind.Reference(p, *args)
    nf = int(np.sum(sc["typ"] == 0))
    out = {"params": params_array(p), "nf": np.array(nf), "wllse": ref.wall_flags(),
           "phases": np.array(refbind.STEP_PHASES, np.int32), "record_steps": np.array([1], np.int32),
           "workload": np.array(WORKLOAD_6K),
           "scene_sum": np.array([float(sc["pos"].sum()), float(sc["nrm"].sum()), nf])}
    info = ref.info()
    out["ref_info"] = np.array([info[k] for k in sorted(info)], np.float64)
    out["ref_info_keys"] = np.array(sorted(info))
    ref.step(1)

    def grab():
        st = ref.state()
        d = {k: st[k][..., :nf].copy() for k in FIELDS}
        m = ref.mirrors()
        d["mslot"], d["mpos"], d["mprs"] = m["slot"], m["pos"], m["prs"]
        d["cell"] = ref.buckets()
        return d

    prev = grab()
    for k, v in prev.items():
        out[f"s1_k0_{k}"] = v
    for k, ph in enumerate(refbind.STEP_PHASES):
        ref.phase(ph)
        cur = grab()
        for f in CHANGES[ph]:
            keys = ("mslot", "mpos", "mprs") if f == "mirrors" else (f,)
            if any(cur[q].shape != prev[q].shape or not np.array_equal(cur[q], prev[q]) for q in keys):
                for q in keys:
                    out[f"s1_k{k + 1}_{q}"] = cur[q]
        prev = cur
    path = os.path.join(outdir, "ref_6k_f64.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    outdir = args[0] if args else os.path.join(ROOT, "tests", "golden")
    if "--6k" in sys.argv:
        main_6k(outdir)
    else:
        main(outdir, "--corrected" in sys.argv)
