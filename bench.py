"""Benchmark of the spd_K B200 hydro step (one JSON line on rank 0).

Workload: the 2D point blast with the a-posteriori limiter -- 256x256
elements, p=3 (16 solution points per element, 1,048,576 DOF), gamma=1.4,
unit box with outflow (gradfree) boundaries, rho=1, v=0, P=1e-5 outside and
P=(gamma-1)E/(pi r^2) with E=1 inside r=0.01, ADER time stepping, LLF at SD
faces, NAD (relative tolerance 1e-5, Moore neighbourhood) + SED + PAD
detection with theta blending of MUSCL-Hancock/HLLC fallback fluxes. The
initial condition is generated, not read: data = "synthetic".

A step is one full ADER step (p+1 Picard passes + p+1 fallback slices +
dt reduction). The metric is DOF-updates/s = active solution points x steps
/ seconds (the reference's "zone-cycles/s", src/hydro_ader.hpp:263-271).

The timed form is, by default, the mixed + learned form: FP32 state,
transforms and fluxes with FP64 islands (pressure recovery, detector bounds,
dt) and the learned a-priori indicator (spd_k_b200/data/indicator_2d_p3.npz)
flagging elements for the fallback every step. The plain FP64 form (the
reference's arithmetic, bit-identical to it) and the mixed form without the
indicator are timed beside it on the same workload.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--precision fp32|fp64] [--learned PATH|none]
                  [--batch-problems P] [--batch-steps S] [--batch-wave-dof D]

N>1 runs N independent replicas (one per GPU, weak scaling); the headline
time is the max over ranks of CUDA-event time on each solver stream.

Beside the headline the line carries the batched ensemble (by default the
first 64 of the 512 four-quadrant problems, 20 steps; --batch-problems 512
--batch-wave-dof 1e8 runs the whole configuration in waves that fit the
device), the 2D field loop, the divergence-contraction study and the
reference CPU build's throughput.
"""
import argparse
import json
import math
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "blast2d-256x256-p3-ader-nad-muscl"
DEFAULT_INDICATOR = os.path.join(ROOT, "spd_k_b200", "data", "indicator_2d_p3.npz")
P0_BLAST = 0.4 / (math.pi * 0.01 ** 2)  # (gamma-1) E / (pi r^2), E = 1, r = 0.01
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def workload_overrides(N=256, p=3):
    from spd_k_b200.workloads import blast_overrides
    return blast_overrides(N, p, 2)


def workload_config(N=256, p=3):
    from spd_k_b200.api import apply_overrides, config_from_params
    return config_from_params(apply_overrides({}, workload_overrides(N, p)))


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                      "-i", str(self.index), "-lms", "100"],
                                     stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    try:
        with open(MEASURED_PEAKS) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ---------------------------------------------------------------------------
# algorithmic bytes per launch of each kernel kind (FP64 parity form)
# ---------------------------------------------------------------------------
def algorithmic_bytes(info, fallback, esz=8):
    """Compulsory HBM bytes of one launch of each kernel kind; S = one state
    array (E x V x NPT values of esz bytes; the (rho, p) candidates and the
    dt word stay FP64 in both forms)."""
    E, V, npt, nt, D, p = info.n_elements, info.nvar, info.n_points, info.n_time_slices, info.ndim, info.p
    n, nf = p + 1, p + 2
    S = E * V * npt * esz
    cells = E * npt
    ff_slice = D * E * V * (npt // n) * nf * esz        # FV face fluxes of one slice
    b = {}
    # predictor: first pass reads U once and writes nt slices; later passes
    # read nt slices + U and write nt slices; averaged over the p passes
    first = S + nt * S
    later = nt * S + S + nt * S
    b["predict"] = (first + (nt - 2) * later) / max(nt - 1, 1)
    b["correct"] = nt * S + S + S + S                    # U_ader, U (r+w), W_cv
    b["flux"] = nt * S + S + nt * ff_slice + S + 2 * cells * 16   # U_ader, U, FF, U_cv, candidates
    b["detect"] = 2 * cells * 16 + cells                  # (rho,p) candidates -> flags
    b["theta"] = cells + cells
    b["update"] = S + ff_slice + cells + S + (2 * cells * 16 if True else 0)
    return b


KINDS = ["predict", "correct", "flux", "detect", "theta", "update", "other"]


def traffic_from_profiles(kind, workload=WORKLOAD):
    """dram bytes per launch of a kernel kind from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            j = json.load(f)
        v = j.get(workload, {}).get(kind)
        return float(v) if v is not None else None
    except Exception:
        return None


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own CPU build (oracle/_ref) or the oracle port
# ---------------------------------------------------------------------------
def reference_cpu_run(steps, N=256, p=3, dt0=None):
    """Run the reference binary for `steps` full-size steps; returns
    (DOF-updates/s, ms/step, steps, threads, kind, sample)."""
    threads = os.cpu_count() or 1
    ref = os.path.join(ROOT, "oracle", "_ref", "spd_K_ref")
    if dt0 is None:
        dt0 = reference_dt0(N, p)
    tlim = (steps - 0.5) * dt0
    if os.path.exists(ref):
        with tempfile.TemporaryDirectory() as tmp:
            env = dict(os.environ, OMP_NUM_THREADS=str(threads), SPD_OUTPUT_DIR=tmp)
            cmd = [ref] + workload_overrides(N, p) + [f"time/tlim={tlim!r}"]
            r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=1800)
            m = re.search(r"evolution: (\d+) steps, ([\d.eE+-]+) s \(([\d.eE+-]+) ms/step\), ([\d.eE+-]+) zone-cycles/s",
                          r.stdout)
            if r.returncode == 0 and m:
                return (float(m.group(4)), float(m.group(3)), int(m.group(1)), threads, "reference",
                        f"reference CPU build (sources compiled unmodified with a Kokkos-subset OpenMP shim), "
                        f"{N}x{N} p={p}, {m.group(1)} full-size steps, OMP_NUM_THREADS={threads}")
    # oracle port (single thread) on the same workload
    from oracle import oracle as O
    c = O.config_from_params(O.apply_overrides({}, workload_overrides(N, p)))
    o = O.Oracle(c)
    dt = o.compute_dt()
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step(dt)
        dt = o.compute_dt()
    el = time.perf_counter() - t0
    dof = N * N * (p + 1) ** 2
    return (dof * steps / el, el / steps * 1e3, steps, 1, "port",
            f"C restatement of the reference path (oracle port), {N}x{N} p={p}, {steps} steps, 1 thread")


def reference_dt0(N=256, p=3):
    from oracle import oracle as O
    c = O.config_from_params(O.apply_overrides({}, workload_overrides(N, p)))
    # the initial dt depends only on the initial state; the oracle computes it exactly
    return O.Oracle(c).compute_dt()


# ---------------------------------------------------------------------------
def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
        return rank, world, local, dist
    return rank, world, local, None


def max_over_ranks(dist, value, device):
    """max of a per-rank value (device: "cuda:<local>" under NCCL, "cpu" under gloo)"""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_throughput(world, dof_per_rank, steps, ms_max):
    """whole-job DOF-updates/s of `world` replicas, timed by the slowest rank"""
    return world * dof_per_rank * steps / (ms_max * 1e-3)


def barrier(dist):
    if dist is not None:
        dist.barrier()


def batched_configs(count, seed=2024, precision="fp32", side=(64, 512)):
    """the seeded four-quadrant Riemann ensemble of the batched configuration
    (spd_k_b200.workloads.riemann_ensemble)"""
    from spd_k_b200.workloads import riemann_ensemble
    return riemann_ensemble(count, seed, precision, side)


def batched_leg(args, local, dist, world, rank=0):
    """the batched form on the ensemble: autotuned tiles, graph-replayed
    steps, DOF-updates/s of all problems together. With several ranks the
    ensemble is split across them (greedy size balance, the same split on
    every rank, no collective on the data path) and the throughput is the
    whole ensemble's DOF over the slowest rank's time (strong scaling)."""
    import ctypes
    import torch
    import spd_k_b200.batch as B
    cfgs = batched_configs(args.batch_problems)
    idx, mine = B.shard(cfgs, rank, world)
    total_dof = sum(B.problem_dof(c) for c in cfgs)

    def run(configs, tune=True):
        """(ms per step, launches per step, groups) of one batch of the given problems"""
        b = B.Batch(configs, device=local)
        if tune:
            b.autotune(2)
        info = b.info()
        st = torch.cuda.ExternalStream(b.stream(), device=f"cuda:{local}")
        b.steps(3)
        b.sync()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        b.steps(args.batch_steps)
        e1.record(st)
        e1.synchronize()
        b.sync()
        ms = e0.elapsed_time(e1) / args.batch_steps
        groups = {int(info.group_p[g]): {"problems": int(info.group_size[g]), "tile": int(info.group_tile[g])}
                  for g in range(info.n_groups)}
        out = (ms, info.launches_per_step, groups)
        b.close()
        return out

    # an ensemble larger than the device holds runs in waves of at most
    # batch_wave_dof DOF, one after the other; the step time is their sum
    waves = [mine] if mine else []
    if mine and args.batch_wave_dof > 0:
        waves = B.waves(mine, args.batch_wave_dof)
    ms_local, lps, groups = 0.0, None, None
    barrier(dist)       # every rank takes the same collective steps, with or without problems
    for w in waves:
        ms_w, lps, g = run(w)
        ms_local += ms_w
        groups = groups or {}
        for p, v in g.items():
            if p in groups:
                groups[p]["problems"] += v["problems"]   # the tile reported is the first wave's
            else:
                groups[p] = dict(v)
    ms = max_over_ranks(dist, ms_local * args.batch_steps, f"cuda:{local}")
    res = {"value": total_dof * args.batch_steps / (ms * 1e-3), "unit": "DOF-updates/s",
           "problems": len(cfgs), "dof": total_dof, "steps": args.batch_steps,
           "scaling": "strong (the ensemble split across ranks)" if world > 1 else "strong",
           "problems_on_rank": len(mine), "ms_per_step": ms / args.batch_steps,
           "workload": (f"the first {len(cfgs)} problems of the seeded four-quadrant Riemann ensemble: N per side "
                        "in {64..512} step 8, p in {2,3,5}, FP32 form, ADER + NAD/MUSCL, autotuned tiles, "
                        "graph-captured step"),
           "launches_per_step": lps, "groups": groups, "waves": len(waves)}
    # per order: the same problems batched by order alone, and one problem of
    # that order at the group's mean size stepped alone
    if world == 1 and mine and args.batch_groups and len(waves) == 1:
        per = {}
        for p in sorted({c["p"] for c in mine}):
            sub = [c for c in mine if c["p"] == p]
            dof = sum(B.problem_dof(c) for c in sub)
            ms_g, _, g = run(sub)
            side = int(round((sum(c["N"][0] * c["N"][1] for c in sub) / len(sub)) ** 0.5 / 8)) * 8
            one = dict(sub[0], N=[side, side, 1])
            ms_1, _, _ = run([one])
            per[p] = {"problems": len(sub), "dof": dof, "ms_per_step": ms_g, "value": dof * 1e3 / ms_g,
                      "tile": g[p]["tile"],
                      "single_problem": {"side": side, "value": B.problem_dof(one) * 1e3 / ms_1}}
        res["per_order"] = per
    return res


def kernel_profile(L, solver, steps, esz, workload):
    """per-kernel CUDA-event times of `steps` steps launched one by one with
    an event pair around every launch (no graph), the algorithmic GB/s of
    each kernel kind, and the roofline of the dominant kind"""
    import ctypes
    from spd_k_b200.api import _lib
    L.spdk_hydro_profile.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                     ctypes.POINTER(ctypes.c_longlong)]
    kms = (ctypes.c_double * 7)()
    kl = (ctypes.c_longlong * 7)()
    rc = L.spdk_hydro_profile(solver.h, steps, kms, kl)
    assert rc == 0, _lib.spdk_last_error()
    per_kind = {KINDS[i]: {"launches": int(kl[i]), "ms": float(kms[i]),
                           "avg_us": (1e3 * kms[i] / kl[i]) if kl[i] else None} for i in range(7)}
    info = solver.info
    alg = algorithmic_bytes(info, True, esz)
    dom = max((k for k in KINDS if k in alg and per_kind[k]["launches"]), key=lambda k: per_kind[k]["ms"])
    hbm, peak_kind = peaks()
    achieved = alg[dom] / (per_kind[dom]["avg_us"] * 1e-6) / 1e9
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_source": peak_kind, "traffic": traffic_from_profiles(dom, workload),
                "algorithmic_bytes": alg[dom]}
    table = {k: dict(v, algorithmic_gbs=(alg[k] / (v["avg_us"] * 1e-6) / 1e9 if k in alg and v["avg_us"] else None),
                     hbm_frac=(alg[k] / (v["avg_us"] * 1e-6) / 1e9 / hbm if k in alg and v["avg_us"] else None))
             for k, v in per_kind.items() if v["launches"]}
    table["note"] = (f"{steps} steps launched one by one with a CUDA-event pair around each launch (no graph, "
                     "no overlap between launches): the sum over kinds exceeds the graph-replayed step time")
    return table, roofline


def mid_run_state(c, t_mid, local):
    """the plain FP64 run's state at t_mid (first step end at or after it),
    stepped on the device by the time loop: (U_sp as doubles, t, steps)"""
    import spd_k_b200 as S
    sv = S.HydroSolver(dict(c, precision="fp64"), device=local)
    n = sv.evolve(t_mid)
    u = sv.read(S.FIELD_U_SP)
    t = sv.t
    sv.close()
    return u, t, n


def induction2d_leg(args, local, dist):
    """the 2D field-loop configuration (512^2 elements, p = 4, v = (2, 1),
    [-1, 1]^2 periodic as [0, 2]^2): graph-free steps of the native 2D
    induction solver in the plain FP64 and the FP32 form, CUDA events on the
    solver stream. DOF = elements x (p+1)^2 solution points; the algorithmic
    HBM bytes of an ADER step are the face fields' compulsory traffic of its
    fused passes: first pass B in, nt slices out; later passes nt slices + B
    in, nt slices out; corrector nt slices + B in, B out."""
    import torch
    from spd_k_b200.induction import Induction2D, field_loop_config
    hbm, peak_kind = peaks()
    out = {"workload": "field loop 2D, 512^2 elements, p=4, v=(2,1), A_z=1e-3 (0.3 - r), periodic, ADER",
           "unit": "DOF-updates/s"}
    for prec in ("fp64", "fp32"):
        c = field_loop_config(N=512, p=4, precision=prec)
        s = Induction2D(c)
        st = torch.cuda.ExternalStream(s.stream(), device=f"cuda:{local}")
        for _ in range(3):
            s.step()
        s.sync()
        barrier(dist)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.induction_steps):
            s.step()
        e1.record(st)
        e1.synchronize()
        ms = max_over_ranks(dist, e0.elapsed_time(e1), f"cuda:{local}") / args.induction_steps
        n, nf, nt = c["p"] + 1, c["p"] + 2, c["p"] + 1
        E = c["N"][0] * c["N"][1]
        S2 = 2 * E * n * nf * (8 if prec == "fp64" else 4)
        alg = (S2 + nt * S2) + (nt - 2) * (2 * nt + 1) * S2 + (nt + 2) * S2
        gbs = alg / (ms * 1e-3) / 1e9
        out[prec] = {"value": E * n * n / (ms * 1e-3), "ms_per_step": ms, "steps": args.induction_steps,
                     "launches_per_step": s.info.launches_per_step, "algorithmic_bytes_per_step": alg,
                     "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                                  "peak_source": peak_kind}}
        s.close()
    return out


def tensor_core_study(args, local):
    """the FP32 Picard pass's divergence contraction for one slice of the
    blast (N^2 elements x 4 variables, p = 3) on CUDA cores and on tensor
    cores (3xTF32 mma.sync), CUDA events, average over 20 calls"""
    import ctypes
    import torch
    import spd_k_b200 as S
    L = S.load_library()
    f = L.spdk_study_divergence
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_longlong] + [ctypes.c_void_p] * 4
    count = args.N * args.N * 4
    dev = torch.device(f"cuda:{local}")
    g = torch.Generator(device=dev)
    g.manual_seed(3)
    fx = torch.randn(count, 4, 5, device=dev, generator=g)
    fy = torch.randn(count, 4, 5, device=dev, generator=g)
    out = torch.empty(count, 4, 4, device=dev)
    st = torch.cuda.current_stream(dev)
    res = {"element_variables": count, "bytes_per_call": (fx.numel() + fy.numel() + out.numel()) * 4}
    for mode, name in ((0, "cuda_cores"), (1, "tensor_cores_3xtf32")):
        for _ in range(3):
            f(mode, 3, count, fx.data_ptr(), fy.data_ptr(), out.data_ptr(), st.cuda_stream)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        reps = 20
        e0.record(st)
        for _ in range(reps):
            f(mode, 3, count, fx.data_ptr(), fy.data_ptr(), out.data_ptr(), st.cuda_stream)
        e1.record(st)
        e1.synchronize()
        us = e0.elapsed_time(e1) * 1e3 / reps
        res[name] = {"us": us, "gbs": res["bytes_per_call"] / (us * 1e-6) / 1e9}
    res["tensor_over_cuda_cores_time"] = res["tensor_cores_3xtf32"]["us"] / res["cuda_cores"]["us"]
    return res


def run_reference_arm(args):
    rank, world, local, dist = (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                                int(os.environ.get("LOCAL_RANK", "0")), None)
    if rank != 0:
        return 0
    steps = max(1, min(args.steps, args.ref_steps))
    val, ms, ran, threads, kind, sample = reference_cpu_run(steps)
    line = {
        "impl": "reference", "metric": "DOF-updates/s", "value": val, "unit": "DOF-updates/s",
        "n_gpus": args.gpus, "steps": ran, "warmup": 0, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "elements": [256, 256], "p": 3, "dof": 256 * 256 * 16,
                   "integrator": "ader", "fallback": "NAD+SED+PAD, theta-blended MUSCL-Hancock/HLLC"},
        "cpu_baseline": {"value": val, "unit": "DOF-updates/s", "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": val, "unit": "DOF-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--profile-steps", type=int, default=20)
    ap.add_argument("--ref-steps", type=int, default=3, help="full-size steps of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--N", type=int, default=256)
    ap.add_argument("--no-graph", action="store_true",
                    help="launch the timed steps one by one instead of replaying the step graph")
    ap.add_argument("--precision", default="fp32", choices=["fp64", "fp32"],
                    help="arithmetic of the timed form (the plain fp64 form is timed beside any other)")
    ap.add_argument("--learned", default=DEFAULT_INDICATOR,
                    help="weights of the learned a-priori indicator ('none': without it)")
    ap.add_argument("--threshold", type=float, default=0.5)
    ap.add_argument("--batch-problems", type=int, default=64,
                    help="problems of the batched-ensemble leg, the first of its seeded ensemble (0: skip it)")
    ap.add_argument("--batch-steps", type=int, default=20)
    ap.add_argument("--batch-wave-dof", type=float, default=0,
                    help="run the ensemble in waves of at most this many DOF (0: one batch)")
    ap.add_argument("--batch-groups", type=int, default=1,
                    help="also time each order's problems as their own batch and one single problem per order")
    ap.add_argument("--tc-study", type=int, default=1,
                    help="time the divergence contraction on CUDA cores and on tensor cores (0: skip)")
    ap.add_argument("--induction-steps", type=int, default=20,
                    help="steps of the 2D field-loop leg (0: skip it)")
    ap.add_argument("--t-mid", type=float, default=0.025,
                    help="simulated time of the state the steps are timed from (0: the initial blast)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.warmup < 3:
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)

    rank, world, local, dist = dist_setup(args.gpus)
    import ctypes
    import numpy as np
    import spd_k_b200 as S
    from spd_k_b200.api import _lib

    c = dict(workload_config(args.N), precision=args.precision)
    esz = 4 if args.precision == "fp32" else 8
    learned = args.learned and args.learned != "none"
    ind = None
    if learned:
        from spd_k_b200.learned import Indicator, set_indicator
        torch_dev = f"cuda:{local}"
        import torch
        torch.cuda.set_device(local)
        ind = Indicator.load(args.learned)
    # the state the steps are timed from: the plain FP64 run at t_mid, where
    # the blast's shock ring keeps the fallback busy (untimed set-up)
    u_mid, t_mid, mid_steps = (None, 0.0, 0)
    if args.t_mid > 0:
        import torch
        torch.cuda.set_device(local)
        u_mid, t_mid, mid_steps = mid_run_state(c, args.t_mid, local)
    solver = S.HydroSolver(c, device=local)
    if u_mid is not None:
        solver.write_u(u_mid)
    if ind is not None:
        set_indicator(solver, ind, args.threshold)
    L = S.load_library()
    info = solver.info
    dof = info.n_dof
    form = ("mixed+learned" if learned else "mixed") if args.precision == "fp32" else (
        "plain+learned" if learned else "plain")

    # ---- headline: K graph-replayed steps, inputs resident in HBM ----
    import torch
    torch.cuda.set_device(local)
    sp = ctypes.c_void_p()
    L.spdk_hydro_get_stream.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
    rc = L.spdk_hydro_get_stream(solver.h, ctypes.byref(sp))
    assert rc == 0
    stream = torch.cuda.ExternalStream(sp.value, device=f"cuda:{local}")
    if args.no_graph:
        for _ in range(args.warmup):
            solver.step()
    else:
        solver.steps(args.warmup)
    solver.sync()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    barrier(dist)
    torch.cuda.synchronize()
    solver.sync()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    if args.no_graph:
        for _ in range(args.steps):
            solver.step()
    else:
        solver.steps(args.steps)
    e1.record(stream)
    e1.synchronize()
    solver.sync()
    torch.cuda.synchronize()
    barrier(dist)
    ms_local = e0.elapsed_time(e1)
    clk = clocks.stop()
    ms = max_over_ranks(dist, ms_local, f"cuda:{local}")
    value = aggregate_throughput(world, dof, args.steps, ms)

    # ---- per-kernel CUDA-event pass (same stream, no graph) ----
    kernel_table, roofline = kernel_profile(
        L, solver, args.profile_steps, esz, WORKLOAD if args.precision == "fp64" else f"{WORKLOAD}-{args.precision}")

    # ---- e2e through the C ABI with host buffers (reference driver loop) ----
    solver2 = S.HydroSolver(c, device=local)
    if ind is not None:
        set_indicator(solver2, ind, args.threshold)
    u_host = torch.empty(info.n_elements * info.nvar * info.n_points, dtype=torch.float64,
                         pin_memory=True).numpy()   # the C ABI exchanges doubles in both forms
    if u_mid is not None:
        u_host[:] = u_mid
    else:
        solver2.read(S.FIELD_U_SP, out=u_host)
    w_host = torch.empty_like(torch.from_numpy(u_host)).pin_memory().numpy()
    rc = L.spdk_hydro_get_stream(solver2.h, ctypes.byref(sp))
    stream2 = torch.cuda.ExternalStream(sp.value, device=f"cuda:{local}")
    e2e_steps = max(1, min(args.steps, 200))
    # simulated time the job runs to: t_mid plus the sum of the dts of
    # e2e_steps steps from the written state (untimed; the timed run repeats
    # the same dts)
    solver2.write_u(u_host)
    t_end = t_mid
    dt = solver2.dt()
    for _ in range(e2e_steps):
        solver2.step()
        t_end += dt
        dt = solver2.dt()
    barrier(dist)
    solver2.sync()

    def timed(run):
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream2)
        solver2.write_u(u_host)                 # H2D of the job's input state (pinned)
        n = run()
        solver2.read(S.FIELD_W_CV, out=w_host)  # D2H of the result
        f1.record(stream2)
        f1.synchronize()
        return n, max_over_ranks(dist, f0.elapsed_time(f1), f"cuda:{local}")

    def per_step():
        for _ in range(e2e_steps):
            solver2.step()                      # spdk_hydro_step
            solver2.dt()                        # blocking D2H of the step's dt (the reference's loop)
        return e2e_steps

    # time_evolution through the C ABI (spdk_hydro_evolve_from: the loop on
    # the device, resumed at t_mid)
    n_evolve, e2e_ms = timed(lambda: solver2.evolve(t_end, t0=t_mid))
    n_loop, loop_ms = timed(per_step)
    state_bytes = u_host.nbytes
    e2e = {"value": world * dof * n_evolve / (e2e_ms * 1e-3), "unit": "DOF-updates/s",
           "h2d_bytes_per_step": state_bytes / n_evolve, "d2h_bytes_per_step": state_bytes / n_evolve,
           "steps": n_evolve, "t0": t_mid, "t_end": t_end,
           "path": "spdk_hydro_write + spdk_hydro_evolve_from(t_mid, t_end) + spdk_hydro_read",
           "host_step_loop": {"value": world * dof * n_loop / (loop_ms * 1e-3),
                              "path": "spdk_hydro_step + blocking spdk_hydro_get_dt per step"}}
    solver2.close()

    # ---- the other forms on the same workload, beside the timed one ----
    def time_form(cf, u0=u_mid, profile=False, with_ind=False):
        sv = S.HydroSolver(cf, device=local)
        if u0 is not None:
            sv.write_u(u0)
        if with_ind:
            set_indicator(sv, ind, args.threshold)
        rc = L.spdk_hydro_get_stream(sv.h, ctypes.byref(sp))
        st = torch.cuda.ExternalStream(sp.value, device=f"cuda:{local}")
        sv.steps(args.warmup)
        sv.sync()
        barrier(dist)
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record(st)
        sv.steps(args.steps)
        g1.record(st)
        g1.synchronize()
        msf = max_over_ranks(dist, g0.elapsed_time(g1), f"cuda:{local}")
        res = {"value": aggregate_throughput(world, dof, args.steps, msf), "unit": "DOF-updates/s",
               "ms_per_step": msf / args.steps, "steps": args.steps,
               "timed_form_speedup": (msf / args.steps) / (ms / args.steps)}
        if profile:
            esz_f = 4 if cf["precision"] == "fp32" else 8
            wl = WORKLOAD if cf["precision"] == "fp64" else f"{WORKLOAD}-{cf['precision']}"
            res["kernels"], res["roofline"] = kernel_profile(L, sv, args.profile_steps, esz_f, wl)
        if with_ind:
            set_indicator(sv, None)
        sv.close()
        return res
    plain = time_form(dict(c, precision="fp64"), profile=True) if (args.precision != "fp64" or learned) else None
    mixed = time_form(dict(c, precision="fp32")) if (args.precision == "fp32" and learned) else None
    # the same forms timed from the initial blast (t = 0), where the shock
    # is small and the fallback nearly idle
    initial = None
    if u_mid is not None:
        initial = {"state": "t = 0, the initial blast",
                   "timed_form": dict(time_form(dict(c), u0=None, with_ind=learned), form=form),
                   "plain_fp64": time_form(dict(c, precision="fp64"), u0=None)}
        if args.precision == "fp32" and learned:
            initial["mixed_without_indicator"] = time_form(dict(c, precision="fp32"), u0=None)

    # ---- batched ensemble: independent four-quadrant Riemann problems ----
    batched = None
    if args.batch_problems > 0:
        batched = batched_leg(args, local, dist, world, rank)

    # ---- 2D field-loop advection (the native 2D induction solver) ----
    induction2d = induction2d_leg(args, local, dist) if args.induction_steps > 0 else None

    # ---- the divergence contraction on CUDA cores against tensor cores ----
    tc_study = tensor_core_study(args, local) if args.tc_study else None

    # ---- CPU baseline (rank 0, N=1 only) ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            val, ms_ref, ran, threads, kind, sample = reference_cpu_run(args.ref_steps)
            cpu = {"value": val, "unit": "DOF-updates/s", "cores": threads, "kind": kind, "sample": sample}
        except Exception as ex:  # reported, not fatal
            cpu = {"value": None, "unit": "DOF-updates/s", "cores": 0, "kind": "unavailable", "sample": str(ex)[:200]}

    barrier(dist)
    if rank == 0:
        state_gb = info.device_bytes / 1e9
        line = {
            "metric": "DOF-updates/s", "value": value, "unit": "DOF-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (f64 islands)" if args.precision == "fp32" else "f64",
            "form": form,
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "elements": [args.N, args.N], "p": 3, "dof_per_gpu": dof,
                       "integrator": "ader", "riemann": "LLF at SD faces, HLLC at fallback faces",
                       "fallback": "NAD(1e-5, Moore)+SED+PAD, theta-blended MUSCL-Hancock",
                       "precision": ("fp32 state/transforms/fluxes; fp64 pressure recovery, detector bounds, dt"
                                     if args.precision == "fp32" else "fp64, reference operation order (plain form)"),
                       "learned_indicator": (f"BF16 MLP {os.path.relpath(args.learned, ROOT)}, threshold "
                                             f"{args.threshold}: a-priori fallback flags every step"
                                             if learned else None),
                       "parallelism": f"replicas{world}",
                       "l2": f"no flush: device working set {state_gb:.2f} GB > 126 MB L2",
                       "state": (f"mid-run: the plain FP64 run's state at t = {t_mid:.6g} ({mid_steps} steps "
                                 f"from the initial blast, untimed), then {args.warmup} warm-up steps"
                                 if u_mid is not None else
                                 "steps continue from the initial blast after the warm-up")},
            "gpu_launches": info.launches_per_step * args.steps,
            "roofline": roofline,
            "kernels": kernel_table,
            "e2e": e2e,
            "plain_fp64": plain,
            "mixed_without_indicator": mixed,
            "initial_state": initial,
            "batched": batched,
            "induction2d": induction2d,
            "tensor_core_study": tc_study,
            "cpu_baseline": cpu,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    solver.close()
    if ind is not None:
        ind.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
