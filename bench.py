"""Benchmark of the FR residual + RK update path on B200.

Workload (N=1): 3-D Euler Taylor-Green vortex, gamma 1.4, Mach 0.1, periodic
[0, 2pi]^3, 32^3 straight hexes, P=3 Gauss-Legendre (64 solution points per
hex, 10,485,760 DOF), Rusanov flux, DG correction, classic RK4, dt from CFL 0.5
on the initial state, FP64 throughout (the plain form).  Inputs are larger than
L2 (the state alone is 84 MB, one stage touches ~1.2 GB), so no flush is needed.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

One JSON line (rank 0).  value = DOF * RK stages / s over all ranks with the
state resident in HBM; e2e = the same metric through the C ABI with the state
in pinned host memory, copied in and out every step.  N > 1 runs independent
replicas (one case per GPU, no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DECK_GPU = os.path.join(ROOT, "flurrypp_b200", "decks", "tgv3d_p3_32.deck")
DECK_CPU = os.path.join(ROOT, "flurrypp_b200", "decks", "tgv3d_p3_16.deck")
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "fr_ref_harness_omp")
METRIC = "DOF·RK-stage/s"
WORKLOAD = "3D Euler Taylor-Green vortex, 32^3 hexes, P=3, RK4, Rusanov, FP64 plain form"


def profiled_traffic(kernel_tag: str):
    """DRAM bytes per launch of a kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "fp64_stage_tgv32_p3.md")
    try:
        for line in open(p):
            if line.startswith(kernel_tag + ":"):
                return int(line.split(":")[1])
    except OSError:
        pass
    return None


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            t = [x.strip() for x in l.split(",")]
            if len(t) < 8:
                continue
            try:
                sm.append(float(t[0]))
                mx.append(float(t[1]))
            except ValueError:
                continue
            for n, v in zip(names, t[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def reference_sample(steps: int, warmup: int, threads: int):
    """The reference's own CPU path (oracle/_ref, OpenMP build) on the bounded
    sample: the same Taylor-Green problem on 16^3 hexes (same per-element work,
    1/8 of the elements; the reference's O(n^2) setup makes 32^3 take ~25 min)."""
    if not os.path.exists(REF_BIN):
        return None, "oracle/_ref/fr_ref_harness_omp not built"
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS="1")
    cmd = [REF_BIN, DECK_CPU, "-", "--ic", "tgv", "--tgv-mach", "0.1", "--cfl-dt", "0.5",
           "--time", f"{steps},{warmup}", "--threads", str(threads)]
    r = subprocess.run(cmd, capture_output=True, text=True, env=env)
    if r.returncode != 0:
        return None, f"reference harness failed: {r.stderr[-200:]}"
    line = [l for l in r.stdout.splitlines() if l.startswith("{")][-1]
    return json.loads(line), None


def ref_threads():
    n = os.cpu_count() or 1
    # the reference's omp_blocked_dgemm drops columns unless the thread count
    # divides N = nEles*nFields (global.cpp:229-230); 16^3*5 = 20480 = 2^12*5
    t = 1
    while t * 2 <= n and 20480 % (t * 2) == 0:
        t *= 2
    return t


def run_reference_arm(args, rank):
    if rank != 0:
        return
    thr = ref_threads()
    res, err = reference_sample(max(1, args.steps), max(1, args.warmup), thr)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return
    v = res["dof_stage_per_s"]
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * res["seconds"] / res["steps"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (Taylor-Green initial condition)",
        "config": {"workload": WORKLOAD, "sample": "16^3 hexes (reference CPU, OpenMP)"},
        "cpu_baseline": {"value": v, "unit": METRIC, "cores": res["threads"], "kind": "reference",
                         "sample": f"TGV P3 16^3 hexes, {res['steps']} RK4 steps after {args.warmup} warm-up, "
                                   f"OpenMP {res['threads']} threads, 1 BLAS thread"},
        "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, rank)
        return

    import numpy as np
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=120))
    import flurrypp_b200 as fb

    s = fb.Solver(DECK_GPU, device=local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    s.set_stream(stream.cuda_stream)
    s.initialize_solution(fb.IC_TGV, (0.1,))
    dt = s.calc_dt()  # CFL 0.5 in the deck, evaluated once on the initial state
    s.set_dt(dt)
    dof = s.nSpts * s.nEles * s.nFields
    nrk = s.nRKSteps

    # warm-up (includes the first, eager step and the graph capture)
    s.run(args.warmup)
    torch.cuda.synchronize()
    launches0 = s.info().launches
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        time.sleep(0.5)  # let the sampler start before the timed region
        ev0.record(stream)
        s.run(args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches = s.info().launches - launches0
    s.check_state()

    # dominant kernels timed alone (same stream)
    kt = {}
    for k in ("element_stage", "faces"):
        s.bench_kernel(k, 2)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 20
        a.record(stream)
        s.bench_kernel(k, reps)
        b.record(stream)
        torch.cuda.synchronize()
        kt[k] = a.elapsed_time(b) / reps

    # end to end through the C ABI with host buffers (pinned), every step:
    # state H2D, one update, state D2H
    U_host = torch.empty(s.shape, dtype=torch.float64, pin_memory=True).numpy()
    U_host[...] = s.get_state()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.set_state(U_host)
    s.update()
    U_host[...] = s.get_state()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.e2e_steps):
        s.set_state(U_host)
        s.update()
        U_host[...] = s.get_state()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1)

    t = torch.tensor([ms, ms_e2e], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms, ms_e2e = float(t[0]), float(t[1])

    if rank == 0:
        value = world * dof * nrk * args.steps / (ms / 1e3)
        e2e = world * dof * nrk * args.e2e_steps / (ms_e2e / 1e3)
        peak, peak_kind = measured_peak_hbm()
        # algorithmic bytes per launch of the element kernel (intermediate RK
        # stage, FP64): per element read U, U0, acc, Fn (nFpts*nF), JGinv
        # (nDims^2*nS), detJ (nS); write acc, U, U_fpts (nFpts*nF)
        nS, nFp, nF, nd, E = s.nSpts, s.nFpts, s.nFields, s.nDims, s.nEles
        elem_bytes = 8 * E * (5 * nS * nF + 2 * nFp * nF + nd * nd * nS + nS)
        inf = s.info()
        # face kernel: per face point read 2 slots, normal, dA L/R, U L/R;
        # write Fn L/R and the left wave speed
        nfp = inf.nFacePts
        face_bytes = nfp * (8 + 8 * nd + 16 + 2 * 8 * nF + 2 * 8 * nF + 8)
        ach = elem_bytes / (kt["element_stage"] / 1e3) / 1e9
        out = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (Taylor-Green initial condition, seeded-free analytic field)",
            "config": {"workload": WORKLOAD, "nEles": E, "order": s.order, "dof": dof, "rk_stages": nrk,
                       "dt": dt, "l2_flush": "inputs larger than L2 (no flush)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": dof * 8, "d2h_bytes_per_step": dof * 8},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                         "traffic": profiled_traffic("traffic_bytes_per_launch"),
                         "traffic_source": "profiles/fp64_stage_tgv32_p3.md (ncu, one launch)",
                         "kernel": "k_elem_tma<3, 3>" if inf.tensor_kernels == 2 else "k_elem_tp<3, 3>",
                         "kernel_ms": kt["element_stage"], "algorithmic_bytes": elem_bytes,
                         "peak_source": peak_kind},
            "kernels_ms": {"element_stage": kt["element_stage"], "faces": kt["faces"],
                           "faces_GBps": face_bytes / (kt["faces"] / 1e3) / 1e9},
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_cpu_baseline:
            thr = ref_threads()
            res, err = reference_sample(args.cpu_steps, 1, thr)
            if res:
                out["cpu_baseline"] = {
                    "value": res["dof_stage_per_s"], "unit": METRIC, "cores": res["threads"], "kind": "reference",
                    "sample": f"reference CPU (OpenMP {res['threads']} threads), TGV P3 16^3 hexes, "
                              f"{res['steps']} RK4 steps"}
            else:
                out["cpu_baseline"] = {"value": None, "unit": METRIC, "cores": 0, "kind": "reference",
                                       "sample": err}
        print(json.dumps(out))
    del s
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
