"""Benchmark of the FR residual + RK update path on B200.

Workload (N=1): 3-D Euler Taylor-Green vortex, gamma 1.4, Mach 0.1, periodic
[0, 2pi]^3, 32^3 straight hexes, P=3 Gauss-Legendre (64 solution points per
hex, 10,485,760 DOF), Rusanov flux, DG correction, classic RK4, dt from CFL 0.5
on the initial state, FP64 throughout (the plain form).  Inputs are larger than
L2 (the state alone is 84 MB, one stage touches ~1.2 GB), so no flush is needed.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--forms LIST]

One JSON line (rank 0).  value = DOF * RK stages / s over all ranks with the
state resident in HBM; e2e = the same metric through the C ABI with the state
in pinned host memory, copied in and out every step (three independent cases
in flight on their own streams, so copies and steps of different cases
overlap).  N > 1 runs independent
replicas (one case per GPU, no collective on the data path).

At N = 1 the line also carries "forms", the other workloads of the path,
each beside its plain-FP64 counterpart:
  precision_tgv32  the same 32^3 P3 Taylor-Green run in the precision form
                   (FP32 state/fluxes/operators, compensated RK sums), its
                   throughput and its L2/max error vs the FP64 run after 200
                   steps;
  precision_ns_tgv40  3-D Navier-Stokes Taylor-Green, Re 1600, Pr 0.71,
                   Mach 0.1, 40^3 hexes with interior vertices perturbed by
                   U(-0.05h, 0.05h) (seed 2024), P=4, LDG (tau 0.1, beta 0.5),
                   RK4: FP64 and precision form, 500 steps each, L2/max error;
  batch256         256 seeded 2-D vortex cases (N~U{8..96}, P~U{2..5},
                   strength~U(1,5), centre~U(-2,2)^2, Mach~U(0.2,0.6)), 500
                   RK4 steps: precision form batched (one launch per stage
                   per order, graph-captured step) vs the plain FP64 path
                   case by case, with the L2 error of every case;
  serve            Poisson streams (rates swept) of channel-over-bump steady
                   solves (h~U(0.02,0.1), nx~U{24..96}, ny=nx/3, P~U{1..4},
                   Mach~U(0.2,0.5), local-CFL RK4 + P-multigrid, residual
                   drop 1e-8) through the solve server: solves/s, p50/p99
                   latency, vs a sample of the same solves one at a time.
"""
from __future__ import annotations

import argparse
import json
import os

# 32 hardware work queues (CUDA's default is 8) before any CUDA context, for
# the many-stream serving and end-to-end forms; the package sets the same
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
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
E2E_CASES = 4  # cases in flight in the end-to-end measurement (default of --e2e-cases)
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


def max_over_ranks(values, device):
    """Each timing as the maximum over all ranks (replicas finish when the
    slowest does); identity with one process."""
    import torch
    import torch.distributed as dist

    t = torch.tensor(values, dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def whole_job_rate(world: int, dof: int, stages: int, steps: int, ms: float) -> float:
    """DOF x RK stages / s over all ranks: every rank advances its own case
    of `dof` unknowns by `steps` steps in `ms` (the slowest rank's time)."""
    return world * dof * stages * steps / (ms / 1e3)


TGV_ARGS = ["--ic", "tgv", "--tgv-mach", "0.1", "--cfl-dt", "0.5"]


def cpu_info():
    """The host CPU the reference runs on: model, logical CPUs, CPUs this
    process may use."""
    model = None
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    avail = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    return {"model": model, "logical_cpus": os.cpu_count(), "available_cpus": avail}


def ref_threads(n_cols: int) -> int:
    """OpenMP threads for the reference: the most that the available CPUs
    allow among those that divide N = nEles*nFields (the reference's
    omp_blocked_dgemm drops columns when the thread count does not divide N,
    src/global.cpp:229-230)."""
    avail = cpu_info()["available_cpus"]
    return max(t for t in range(1, avail + 1) if n_cols % t == 0)


def run_ref(deck: str, harness_args, steps: int, warmup: int, threads: int, time1: int = 0, cwd=None):
    """One timed run of the reference's own CPU path (oracle/_ref, OpenMP
    build): mesh setup, initial state, W untimed and K timed solver::update()
    steps (the driver's loop, P-multigrid cycle included), and optionally K1
    more on one thread.  Returns (the harness's JSON, None) or (None, why)."""
    if not os.path.exists(REF_BIN):
        return None, "oracle/_ref/fr_ref_harness_omp not built"
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS="1")
    cmd = [REF_BIN, deck, "-", *harness_args, "--time", f"{steps},{warmup}", "--threads", str(threads)]
    if time1:
        cmd += ["--time1", str(time1)]
    t0 = time.perf_counter()
    r = subprocess.run(cmd, capture_output=True, text=True, env=env, cwd=cwd)
    if r.returncode != 0:
        return None, f"reference harness failed: {r.stderr[-200:]}"
    line = [l for l in r.stdout.splitlines() if l.startswith("{")][-1]
    out = json.loads(line)
    out["wall_s"] = time.perf_counter() - t0
    return out, None


HEADLINE_ELES, HEADLINE_FIELDS = 32 ** 3, 5


def headline_config(world: int) -> dict:
    """The workload both arms measure (32^3 hexes, P3, TGV, RK4, FP64)."""
    return {"workload": WORKLOAD, "nEles": HEADLINE_ELES, "order": 3, "dof": HEADLINE_ELES * 64 * HEADLINE_FIELDS,
            "rk_stages": 4, "l2_flush": "inputs larger than L2 (no flush)",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


def headline_reference(steps: int, warmup: int, time1: int = 1):
    """The reference on the headline workload itself (32^3 hexes), all the
    threads that divide N; its mesh setup (not timed) takes a minute or two."""
    thr = ref_threads(HEADLINE_ELES * HEADLINE_FIELDS)
    res, err = run_ref(DECK_GPU, TGV_ARGS, steps, warmup, thr, time1=time1)
    if res is None:
        return None, err
    cpu = cpu_info()
    res["cpu"] = cpu
    res["sample"] = (f"the full workload (TGV P3 32^3 hexes), {res['steps']} RK4 steps after {warmup} warm-up, "
                     f"OpenMP {res['threads']} threads (the most of {cpu['available_cpus']} available CPUs that "
                     f"divide nEles*nFields), 1 BLAS thread; 1-thread figure over {res['steps_1thread']} step(s); "
                     "mesh setup untimed")
    return res, None


def run_reference_arm(args, rank):
    if rank != 0:
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    res, err = headline_reference(max(1, args.steps), max(1, args.warmup))
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return
    v = res["dof_stage_per_s"]
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * res["seconds"] / res["steps"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (Taylor-Green initial condition)",
        "config": headline_config(world),
        "cpu_baseline": {"value": v, "unit": METRIC, "cores": res["threads"], "kind": "reference",
                         "sample": res["sample"], "cpu": res["cpu"],
                         "value_1thread": res["dof_stage_per_s_1thread"]},
        "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


DECK_NS = os.path.join(ROOT, "flurrypp_b200", "decks", "ns_tgv3d_p4_40.deck")


def dev_ms(torch, stream, fn):
    """Device time of fn's work on `stream` (CUDA events, synchronized)."""
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b)


def state_errors(U, ref):
    """relative L2, max |diff| / max |ref|, and relative L2 per field."""
    import numpy as np

    d = U - ref
    per = [float(np.linalg.norm(d[..., k]) / max(np.linalg.norm(ref[..., k]), 1e-300)) for k in range(ref.shape[-1])]
    return {"l2_rel": float(np.linalg.norm(d) / np.linalg.norm(ref)),
            "max_rel": float(np.abs(d).max() / np.abs(ref).max()), "l2_rel_per_field": per}


def elem_bytes(s, wbytes):
    """Algorithmic bytes of one intermediate-stage element launch: read U, U0,
    acc (3 nS nF), Fn (nFp nF), JGinv (nDims^2 nS), detJ (nS); write acc, U
    (2 nS nF) and U_fpts (nFp nF); words of the working precision."""
    nS, nFp, nF, nd, E = s.nSpts, s.nFpts, s.nFields, s.nDims, s.nEles
    return wbytes * E * (5 * nS * nF + 2 * nFp * nF + nd * nd * nS + nS)


def kernel_ms(torch, stream, s, kernel, reps=20):
    s.bench_kernel(kernel, 2)
    return dev_ms(torch, stream, lambda: s.bench_kernel(kernel, reps)) / reps


def form_precision_tgv32(args, fb, torch, stream, dt):
    s = fb.Solver(DECK_GPU, precision=fb.FR_PREC_MIXED)
    s.set_stream(stream.cuda_stream)
    s.initialize_solution(fb.IC_TGV, (0.1,))
    s.set_dt(dt)
    dof, nrk = s.nSpts * s.nEles * s.nFields, s.nRKSteps
    s.run(args.warmup)
    ms = dev_ms(torch, stream, lambda: s.run(args.steps))
    inf = s.info()
    km = kernel_ms(torch, stream, s, "element_stage")
    fm = kernel_ms(torch, stream, s, "faces")
    peak, _ = measured_peak_hbm()
    eb = elem_bytes(s, 4)
    ach = eb / (km / 1e3) / 1e9
    del s
    # error after 200 steps vs the plain form, same initial state and dt
    runs = {}
    for prec in (fb.FR_PREC_FP64, fb.FR_PREC_MIXED):
        c = fb.Solver(DECK_GPU, precision=prec)
        c.set_stream(stream.cuda_stream)
        c.initialize_solution(fb.IC_TGV, (0.1,))
        c.set_dt(dt)
        c.run(args.err_steps)
        runs[prec] = c.get_state()
        del c
    return {
        "workload": "3D Euler TGV 32^3 P3 RK4, precision form (FP32 state/fluxes/operators, TwoSum RK sums)",
        "value": dof * nrk * args.steps / (ms / 1e3), "unit": METRIC, "ms_per_step": ms / args.steps,
        "dtype": "f32 (FP64 dt, metrics at setup, norms)",
        "tile_variant": inf.tile_variant, "elems_per_block": inf.elems_per_block,
        "kernels_ms": {"element_stage": km, "faces": fm},
        "roofline": {"bound": "hbm", "kernel": f"k_elem_tma<3, 3, float, {inf.tile_variant}>",
                     "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                     "algorithmic_bytes": eb},
        "error_vs_fp64": dict(steps=args.err_steps, **state_errors(runs[fb.FR_PREC_MIXED], runs[fb.FR_PREC_FP64])),
    }


def form_ns_tgv40(args, fb, torch, stream):
    opts = dict(perturb=1, seed=2024, perturb_frac=0.05, mu_override=1, mu_inf=1.0 / 1600.0)
    out, states, dt = {}, {}, None
    for prec, tag in ((fb.FR_PREC_FP64, "fp64"), (fb.FR_PREC_MIXED, "precision")):
        t0 = time.perf_counter()
        c = fb.Solver(DECK_NS, precision=prec, **opts)
        setup_s = time.perf_counter() - t0
        c.set_stream(stream.cuda_stream)
        c.initialize_solution(fb.IC_TGV, (0.1,))
        if dt is None:
            dt = c.calc_dt()
        c.set_dt(dt)
        dof, nrk = c.nSpts * c.nEles * c.nFields, c.nRKSteps
        w = min(3, args.ns_steps)
        c.run(w)
        ms = dev_ms(torch, stream, lambda: c.run(args.ns_steps - w))
        states[tag] = c.get_state()  # after exactly ns_steps steps
        km = kernel_ms(torch, stream, c, "element_stage", 5)
        fm = kernel_ms(torch, stream, c, "faces", 5)
        out[tag] = {"value": dof * nrk * (args.ns_steps - w) / (ms / 1e3), "unit": METRIC,
                    "ms_per_step": ms / (args.ns_steps - w), "setup_s": setup_s,
                    "kernels_ms": {"element_stage": km, "faces_ldg_grad_visc": fm}}
        del c
    out["workload"] = ("3D Navier-Stokes TGV Re 1600 Pr 0.71 Mach 0.1, 40^3 hexes perturbed U(-0.05h,0.05h) "
                       "seed 2024, P=4, LDG tau 0.1 beta 0.5, Rusanov, RK4")
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = ns_reference(args)
    out["dof"] = dof
    out["dt"] = dt
    out["speedup_precision_vs_fp64"] = out["precision"]["value"] / out["fp64"]["value"]
    out["error_vs_fp64"] = dict(steps=args.ns_steps, **state_errors(states["precision"], states["fp64"]))
    return out


def ns_reference(args):
    """The reference's CPU path on the Navier-Stokes TGV per RK stage, on a
    20^3 sample of the 40^3 mesh (same order, perturbation law and physics,
    1/8 of the elements: the reference's mesh setup grows with the square of
    the element count)."""
    import tempfile

    n = 20
    src = open(DECK_NS).read()
    for ax in ("nx", "ny", "nz"):
        src = src.replace(f"{ax}            40", f"{ax}            {n}")
    with tempfile.TemporaryDirectory() as td:
        deck = os.path.join(td, "ns20.deck")
        open(deck, "w").write(src)
        thr = ref_threads(n ** 3 * 5)
        res, err = run_ref(deck, ["--ic", "tgv", "--tgv-mach", "0.1", "--perturb", "2024,0.05",
                                  "--mu-inf", repr(1.0 / 1600.0), "--cfl-dt", "0.5"], 3, 1, thr)
    if res is None:
        return {"value": None, "sample": err}
    return {"value": res["dof_stage_per_s"], "unit": METRIC, "cores": res["threads"], "kind": "reference",
            "sample": f"NS TGV P4 on 20^3 perturbed hexes (1/8 of the elements), {res['steps']} RK4 steps "
                      f"after 1 warm-up, OpenMP {res['threads']} threads, per-stage rate"}


def vortex32_form(args, fb, torch, stream):
    """Config 1: 2-D Euler vortex (strength 5, Mach 0.5 along +x), periodic
    [-5,5]^2, 32x32 quads, P3, RK4, fixed dt at CFL 0.5, 1000 steps: the FP64
    GPU path and the reference's CPU path on the same run."""
    import tempfile

    from flurrypp_b200.decks import vortex_case

    deck = vortex_case(os.path.join(tempfile.mkdtemp(prefix="fr_v32_"), "vortex32.deck"), 32, 3, 0.5)
    s = fb.Solver(deck)
    s.set_stream(stream.cuda_stream)
    s.initialize_solution(fb.IC_VORTEX, (5.0, 0.0, 0.0, 0.5))
    dt = s.calc_dt()  # the CFL formula at CFL 0.5 on the initial state, then fixed
    s.set_dt(dt)
    dof, nrk = s.nSpts * s.nEles * s.nFields, s.nRKSteps
    steps = 1000
    s.run(3)
    ms = dev_ms(torch, stream, lambda: s.run(steps))
    out = {"workload": "2-D Euler vortex, 32x32 quads, P3, RK4, CFL 0.5 fixed dt, FP64", "dof": dof,
           "value": dof * nrk * steps / (ms / 1e3), "unit": METRIC, "ms_per_step": ms / steps, "steps": steps}
    if not args.no_cpu_baseline:
        thr = ref_threads(s.nEles * s.nFields)
        res, err = run_ref(deck, ["--ic", "vortex", "--vortex", "5,0,0,0.5", "--cfl-dt", "0.5"], steps, 3, thr)
        out["cpu_baseline"] = ({"value": res["dof_stage_per_s"], "unit": METRIC, "cores": res["threads"],
                                "kind": "reference", "sample": f"the whole run: {steps} RK4 steps, OpenMP "
                                                               f"{res['threads']} threads"}
                               if res else {"value": None, "sample": err})
    return out


def batch_reference(specs, decks, k: int, steps: int):
    """The reference's CPU path on the first k cases of the batch, one after
    another, each over `steps` RK4 steps: its DOF-stage rate over them."""
    dofs, secs, thr_used = 0.0, 0.0, set()
    for (n, P, eps, xc, yc, M), deck in list(zip(specs, decks))[:k]:
        thr = ref_threads(n * n * 4)
        res, err = run_ref(deck, ["--ic", "vortex", "--vortex", f"{eps!r},{xc!r},{yc!r},{M!r}", "--cfl-dt", "0.5"],
                           steps, 1, thr)
        if res is None:
            return {"value": None, "sample": err}
        dofs += res["dof"] * res["stages"]
        secs += res["seconds"]
        thr_used.add(res["threads"])
    return {"value": dofs / secs, "unit": METRIC, "cores": max(thr_used), "kind": "reference",
            "sample": f"the first {k} of the cases, one after another, {steps} RK4 steps each, OpenMP "
                      f"threads {sorted(thr_used)} (the most that divide each case's nEles*nFields)"}


def form_batch256(args, fb, torch, stream):
    import tempfile

    import numpy as np
    from flurrypp_b200.decks import vortex_case

    rng = np.random.default_rng(args.batch_seed)
    specs = []
    for _ in range(args.batch_cases):
        n = int(rng.integers(8, 97))
        P = int(rng.integers(2, 6))
        eps = float(rng.uniform(1, 5))
        xc, yc = (float(v) for v in rng.uniform(-2, 2, 2))
        M = float(rng.uniform(0.2, 0.6))
        specs.append((n, P, eps, xc, yc, M))
    tmp = tempfile.mkdtemp(prefix="fr_batch_")
    t0 = time.perf_counter()
    c64, c32, dofs, decks = [], [], [], []
    for i, (n, P, eps, xc, yc, M) in enumerate(specs):
        deck = vortex_case(os.path.join(tmp, f"b{i}.deck"), n, P, M)
        decks.append(deck)
        a = fb.Solver(deck)
        a.set_stream(stream.cuda_stream)
        a.initialize_solution(fb.IC_VORTEX, (eps, xc, yc, M))
        dt = a.calc_dt()
        a.set_dt(dt)
        b = fb.Solver(deck, precision=fb.FR_PREC_MIXED)
        b.initialize_solution(fb.IC_VORTEX, (eps, xc, yc, M))
        b.set_dt(dt)
        c64.append(a)
        c32.append(b)
        dofs.append(a.nSpts * a.nEles * a.nFields)
    setup_s = time.perf_counter() - t0
    nrk = c64[0].nRKSteps
    tot = float(sum(dofs))
    # plain FP64 path, case by case (each case its own graph-replayed run)
    ms_alone = 0.0
    for a in c64:
        a.run(3)
        ms_alone += dev_ms(torch, stream, lambda: a.run(args.alone_steps))
    for i, (n, P, eps, xc, yc, M) in enumerate(specs):
        c64[i].initialize_solution(fb.IC_VORTEX, (eps, xc, yc, M))
    res = {}
    forms = {fb.FR_BATCH_GROUPS: "groups", fb.FR_BATCH_MANY_ORDER: "many_order"}
    for tag, cs in (("fp64_batched", c64), ("precision_batched", c32)):
        bt = fb.Batch(cs)  # times both step forms on its own state and keeps the faster
        chosen = bt.form()
        w = 3
        bt.run(w)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        bt.run(args.batch_steps - w)
        torch.cuda.synchronize()
        sec = time.perf_counter() - t1
        bt.gather()
        inf = bt.info()
        res[tag] = {"value": tot * nrk * (args.batch_steps - w) / sec, "unit": METRIC,
                    "seconds": sec, "groups": inf["groups"], "form": forms[chosen["form"]],
                    "autotune_ms_per_step": {"groups": chosen["ms_groups"], "many_order": chosen["ms_many_order"]}}
        # the other form over 100 more steps (after the members took their state)
        other = fb.FR_BATCH_MANY_ORDER if chosen["form"] == fb.FR_BATCH_GROUPS else fb.FR_BATCH_GROUPS
        bt.set_form(other)
        bt.run(3)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        bt.run(100)
        torch.cuda.synchronize()
        res[tag]["other_form"] = {"form": forms[other],
                                  "value": tot * nrk * 100 / (time.perf_counter() - t2), "unit": METRIC}
        del bt
    errs = [state_errors(b.get_state(), a.get_state())["l2_rel"] for a, b in zip(c64, c32)]
    plain = tot * nrk * args.alone_steps / (ms_alone / 1e3)
    return {
        "workload": (f"{args.batch_cases} 2-D Euler vortex cases, seed {args.batch_seed}, N~U{{8..96}}, "
                     "P~U{2..5}, strength~U(1,5), centre~U(-2,2)^2, Mach~U(0.2,0.6), RK4, dt CFL 0.5 per case, "
                     f"{args.batch_steps} steps"),
        "total_dof": int(tot), "setup_s": setup_s,
        "plain_fp64_case_by_case": {"value": plain, "unit": METRIC, "steps_timed_per_case": args.alone_steps},
        "fp64_batched": res["fp64_batched"], "precision_batched": res["precision_batched"],
        "speedup_precision_batched_vs_plain_fp64": res["precision_batched"]["value"] / plain,
        # the same batching on both sides: what the precision form alone gains
        "speedup_precision_batched_vs_fp64_batched": (res["precision_batched"]["value"]
                                                      / res["fp64_batched"]["value"]),
        "cpu_baseline": (batch_reference(specs, decks, 8, 10) if not args.no_cpu_baseline else None),
        "timer": "host clock around a synchronized batch run (order groups run on their own streams)",
        "error_vs_fp64": {"steps": args.batch_steps, "l2_rel_max": max(errs),
                          "l2_rel_median": float(np.median(errs))},
    }


def form_serve(args, fb, torch):
    import tempfile

    import numpy as np
    from flurrypp_b200.decks import channel_case
    from flurrypp_b200.meshgen import channel_bump, write_gmsh

    rng = np.random.default_rng(args.serve_seed)
    tmp = tempfile.mkdtemp(prefix="fr_serve_")
    reqs, n_eles = [], {}
    for i in range(args.serve_requests):
        h = float(rng.uniform(0.02, 0.1))
        nx = int(rng.integers(24, 97))
        P = int(rng.integers(1, 5))
        M = float(rng.uniform(0.2, 0.5))
        msh = os.path.join(tmp, f"bump{i}.msh")
        write_gmsh(msh, channel_bump(nx, nx // 3, h))
        dof = nx * (nx // 3) * (P + 1) ** 2 * 4
        # residual evaluations per driver step on every P-multigrid level
        # (lowOrder 0, 2 smoothing steps, RK4): the fine update's 4 stages and
        # the cycle's fine residual; per coarse level p its source-term
        # residual, 2 x 2 smoothing updates of 4 stages and, above level 0,
        # the residual restricted downwards
        all_dof = dof * 5 + sum(nx * (nx // 3) * (p + 1) ** 2 * 4 * (1 + 2 * 2 * 4 + (1 if p > 0 else 0))
                                for p in range(P))
        reqs.append((channel_case(os.path.join(tmp, f"bump{i}.deck"), msh, P, M), dof, all_dof))
        n_eles[reqs[-1][0]] = nx * (nx // 3)

    def serve(subset, max_inflight, rate, precision=fb.FR_PREC_FP64):
        srv = fb.Server(budget_bytes=args.serve_budget_gb << 30, max_inflight=max_inflight, check_every=10,
                        precision=precision)
        gaps = np.random.default_rng(args.serve_seed + 1).exponential(1.0 / rate, len(subset)) if rate else None
        t0 = time.perf_counter()
        ids = []
        for k, (deck, dof, _) in enumerate(subset):
            if rate:
                time.sleep(float(gaps[k]))
            ids.append(srv.submit(deck, tol=1e-8, max_steps=args.serve_max_steps))
        polls, forms = [], []
        for r in ids:
            try:
                srv.wait(r, 3600)
            except fb.FrError:
                pass
            polls.append(srv.poll(r))
            forms.append(srv.poll_form(r))
        sec = time.perf_counter() - t0
        srv.close()
        lat = [p["latency_s"] for p in polls]
        done = [p for p in polls if p["status"] == 2]
        stages = sum(4 * p["steps"] * dof for p, (_, dof, _) in zip(polls, subset))
        all_stages = sum(p["steps"] * all_dof for p, (_, _, all_dof) in zip(polls, subset))
        return {"solves_per_s": len(done) / sec, "seconds": sec, "completed": len(done),
                "steps_each": [p["steps"] for p in polls],
                "converged_1e-8": sum(1 for p in done if p["res_ratio"] <= 1e-8),
                "median_residual_drop": float(np.median([p["res_ratio"] for p in done])) if done else None,
                "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
                "steps_mean": float(np.mean([p["steps"] for p in polls])),
                "steps_fp32_share": (sum(f["steps_fp32"] for f in forms) / max(1, sum(p["steps"] for p in polls))),
                "fine_dof_stage_per_s": stages / sec, "all_level_dof_stage_per_s": all_stages / sec}

    # warm-up: every request's deck for 20 steps in a throw-away server, so
    # that the kernels of every order and P-multigrid level are loaded before
    # the timed runs (CUDA loads a kernel's module at its first launch)
    warm = fb.Server(budget_bytes=args.serve_budget_gb << 30, max_inflight=args.serve_inflight, check_every=10)
    for rid in [warm.submit(deck, tol=1e-30, max_steps=20) for deck, _, _ in reqs]:
        try:
            warm.wait(rid, 600)
        except fb.FrError:
            pass
    warm.close()

    sweep = {}
    for rate in args.serve_rates:
        sweep[f"rate_{rate:g}_per_s"] = dict(max_inflight=args.serve_inflight, **serve(reqs, args.serve_inflight, rate))
        sweep[f"rate_{rate:g}_per_s"].pop("steps_each")
    top = max(args.serve_rates)
    precision = dict(max_inflight=args.serve_inflight, rate_per_s=top,
                     form="FR_PREC_MIXED_REFINE: precision form until the FP32 residual stops falling, then FP64",
                     **serve(reqs, args.serve_inflight, top, fb.FR_PREC_MIXED_REFINE))
    precision.pop("steps_each")
    k = min(args.serve_alone, len(reqs))
    alone = serve(reqs[:k], 1, 0.0)
    alone["sample"] = f"the first {k} requests, submitted together, one in flight"
    if not args.no_cpu_baseline:
        alone["cpu_baseline"] = serve_reference(reqs[:k], alone.pop("steps_each"), n_eles)
    else:
        alone.pop("steps_each")
    best = max(v["solves_per_s"] for v in sweep.values())
    return {
        "workload": (f"{len(reqs)} channel-over-bump requests, seed {args.serve_seed}, Poisson arrivals, "
                     "h~U(0.02,0.1), nx~U{24..96}, ny=nx/3, P~U{1..4}, Mach~U(0.2,0.5), local-CFL RK4 + "
                     "P-multigrid (lowOrder 0, 2 smoothing steps), run to a residual drop of 1e-8 "
                     f"(at most {args.serve_max_steps} steps), FP64, programmatic dependent launch"),
        "warm_up": "every request's deck run 20 steps in a throw-away server before the timed runs",
        "sweep": sweep,
        "precision_served": precision,
        "one_at_a_time": alone,
        "speedup_solves_per_s": best / max(alone["solves_per_s"], 1e-30),
    }


def serve_reference(subset, steps_each, n_eles):
    """The same requests solved serially by the reference's CPU path, one at a
    time: each request's time per driver step (update + P-multigrid cycle,
    the reference's own loop) over a sample of steps, times the steps the
    request took to converge here, gives its solve time; latencies are the
    completion times of the requests submitted together."""
    import numpy as np

    per_req = []
    for (deck, _, _), n in zip(subset, steps_each):
        thr = ref_threads(n_eles[deck] * 4)
        sample = 20
        res, err = run_ref(os.path.basename(deck), [], sample, 2, thr, cwd=os.path.dirname(deck))
        if res is None:
            return {"value": None, "sample": err}
        per_req.append(res["seconds"] / res["steps"] * n)
    done = np.cumsum(per_req)
    return {"solves_per_s": len(per_req) / float(done[-1]), "p50_latency_s": float(np.percentile(done, 50)),
            "p99_latency_s": float(np.percentile(done, 99)), "kind": "reference",
            "sample": f"the same {len(per_req)} requests, serially: the reference's time per driver step "
                      "(update + P-multigrid cycle) over 20 steps after 2 warm-up, times the steps each request "
                      "took to reach the 1e-8 drop here (extrapolated, not run to convergence on the CPU)",
            "solve_s_each": per_req}


def run_forms(args, fb, torch, stream, dt):
    forms = {}
    want = set(args.forms.split(",")) if args.forms else set()
    jobs = [("vortex32_1000", lambda: vortex32_form(args, fb, torch, stream)),
            ("precision_tgv32", lambda: form_precision_tgv32(args, fb, torch, stream, dt)),
            ("precision_ns_tgv40", lambda: form_ns_tgv40(args, fb, torch, stream)),
            ("batch256", lambda: form_batch256(args, fb, torch, stream)),
            ("serve", lambda: form_serve(args, fb, torch))]
    for name, fn in jobs:
        if name not in want:
            continue
        try:
            forms[name] = fn()
        except Exception as e:  # report, keep the headline line
            forms[name] = {"error": f"{type(e).__name__}: {e}"}
    return forms



PROFILE_CASES = {
    # name: (deck kind, order, size, precision, tile variant)
    "fp64_tgv32_p3": ("tgv", 3, 32, 0, -1),
    "fp32_tgv32_p3": ("tgv", 3, 32, 1, -1),
    "fp32_vortex256_p3": ("vortex", 3, 256, 1, -1),
    "fp64_vortex512_p3": ("vortex", 3, 512, 0, -1),
    "fp64_vortex512_p2": ("vortex", 2, 512, 0, -1),
    "fp64_vortex384_p4": ("vortex", 4, 384, 0, -1),
    "fp32_vortex384_p4": ("vortex", 4, 384, 1, -1),
    "fp64_vortex320_p5": ("vortex", 5, 320, 0, -1),
    "fp32_vortex320_p5": ("vortex", 5, 320, 1, -1),
    "tc_vortex256_p3": ("vortex", 3, 256, 1, 3),
    "fp32_tgv64_p1": ("tgv", 1, 64, 1, -1),
    "tc_tgv64_p1": ("tgv", 1, 64, 1, 3),
    "fp32_ns_tgv24_p4": ("ns", 4, 24, 1, -1),
    "fp64_ns_tgv24_p4": ("ns", 4, 24, 0, -1),
}


def profile_shard(fb, torch, nparts=4):
    """One RK step of the 16^3 P3 Taylor-Green case split into parts on this
    device (cut-face pack, exchange and flux kernels among the stage kernels)."""
    sh = fb.Shard(DECK_CPU, nparts)
    one = fb.Solver(DECK_CPU)
    one.initialize_solution(fb.IC_TGV, (0.1,))
    sh.set_state(one.get_state())
    sh.set_dt(one.calc_dt())
    sh.run(2)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    sh.run(1)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    return {"nparts": nparts, **sh.info()}


def profile_many_order(fb, torch, tmp):
    """One RK step of 32 vortex cases of orders 2..5 in the many-order batch
    form (one face and one element launch per stage for all orders)."""
    import numpy as np
    from flurrypp_b200.decks import vortex_case

    rng = np.random.default_rng(5)
    cs = []
    for i in range(32):
        n, P = int(rng.integers(16, 49)), 2 + i % 4
        s = fb.Solver(vortex_case(os.path.join(tmp, f"m{i}.deck"), n, P, 0.4))
        s.initialize_solution(fb.IC_VORTEX, (3.0, 0.0, 0.0, 0.4))
        s.set_dt(s.calc_dt())
        cs.append(s)
    b = fb.Batch(cs)
    b.set_form(fb.FR_BATCH_MANY_ORDER)
    b.run(2)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    b.run(1)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    return {"cases": len(cs), "dof": int(sum(c.nSpts * c.nEles * c.nFields for c in cs)), **b.form()}


def run_profile(names):
    """Set each case up, then launch its element stage and face pass once
    between cudaProfilerStart/Stop (for `ncu --profile-from-start off`);
    `shard4_tgv16` and `many_order_batch` profile one step of a split case
    and of the many-order batch form."""
    import tempfile

    import torch
    import flurrypp_b200 as fb
    from flurrypp_b200.decks import vortex_case, write_deck

    tmp = tempfile.mkdtemp(prefix="fr_prof_")
    out = {}
    for name in names.split(","):
        if name == "shard4_tgv16":
            out[name] = profile_shard(fb, torch)
            continue
        if name == "many_order_batch":
            out[name] = profile_many_order(fb, torch, tmp)
            continue
        kind, P, n, prec, var = PROFILE_CASES[name]
        opts = dict(precision=prec, tile_variant=var)
        if kind == "tgv":
            ic = (fb.IC_TGV, (0.1,))
            deck = DECK_GPU
            if n != 32 or P != 3:
                src = open(DECK_GPU).read().replace("order         3", f"order         {P}")
                for ax in ("nx", "ny", "nz"):
                    src = src.replace(f"{ax} 32", f"{ax} {n}")
                deck = os.path.join(tmp, f"{name}.deck")
                open(deck, "w").write(src)
        elif kind == "vortex":
            deck, ic = vortex_case(os.path.join(tmp, f"{name}.deck"), n, P, 0.5), (fb.IC_VORTEX, (5.0, 0.0, 0.0, 0.5))
        else:
            src = open(DECK_NS).read().replace("nx            40", f"nx            {n}")
            src = src.replace("ny            40", f"ny            {n}").replace("nz            40", f"nz            {n}")
            deck = os.path.join(tmp, f"{name}.deck")
            open(deck, "w").write(src)
            ic = (fb.IC_TGV, (0.1,))
            opts.update(perturb=1, seed=2024, perturb_frac=0.05, mu_override=1, mu_inf=1.0 / 1600.0)
        s = fb.Solver(deck, **opts)
        s.initialize_solution(*ic)
        s.set_dt(s.calc_dt())
        s.run(2)
        s.synchronize()
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        s.bench_kernel("element_stage", 1)
        s.bench_kernel("faces", 1)
        s.synchronize()
        torch.cuda.profiler.stop()
        inf = s.info()
        out[name] = {"nEles": s.nEles, "order": s.order, "nDims": s.nDims, "precision": prec,
                     "tile_variant": inf.tile_variant, "elems_per_block": inf.elems_per_block}
        del s
    print(json.dumps({"profile": out}))



def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=24)
    ap.add_argument("--e2e-cases", type=int, default=E2E_CASES,
                    help="independent cases in flight in the end-to-end measurement")
    ap.add_argument("--cpu-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--forms", default="vortex32_1000,precision_tgv32,precision_ns_tgv40,batch256,serve",
                    help="comma list of extra workloads measured at N=1 ('' for none)")
    ap.add_argument("--err-steps", type=int, default=200)
    ap.add_argument("--ns-steps", type=int, default=500)
    ap.add_argument("--batch-cases", type=int, default=256)
    ap.add_argument("--batch-steps", type=int, default=500)
    ap.add_argument("--batch-seed", type=int, default=2024)
    ap.add_argument("--alone-steps", type=int, default=20)
    ap.add_argument("--serve-requests", type=int, default=16)
    ap.add_argument("--serve-rates", type=float, nargs="+", default=[2.0, 32.0])
    ap.add_argument("--serve-alone", type=int, default=8)
    ap.add_argument("--serve-seed", type=int, default=7)
    ap.add_argument("--serve-max-steps", type=int, default=12000)
    ap.add_argument("--serve-inflight", type=int, default=16)
    ap.add_argument("--serve-budget-gb", type=int, default=64)
    ap.add_argument("--tile-variant", type=int, default=-1,
                    help="element tile variant of the headline case (-1: the autotuner's choice); for launch "
                         "lists under ncu, whose cold-cache serialised launches can sway the autotuner")
    ap.add_argument("--profile", default="", help="comma list of PROFILE_CASES: one element stage and one "
                    "face pass each between cudaProfilerStart/Stop, then exit")
    args = ap.parse_args()
    if args.profile:
        run_profile(args.profile)
        return

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

    s = fb.Solver(DECK_GPU, device=local, tile_variant=args.tile_variant)
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

    # end to end through the C ABI with host buffers (pinned): every step
    # copies its case's state in from pinned host memory, advances it one RK
    # step and copies the result back out, and the next step of that case
    # starts from the copy that came back.  --e2e-cases independent cases, each
    # on its own stream, are in flight together, so one case's copy in, another
    # case's step and a third case's copy out overlap (the two PCIe directions
    # and the SMs are separate engines).
    flight = [(s, stream)]
    for _ in range(args.e2e_cases - 1):
        sx, stx = fb.Solver(DECK_GPU, device=local, tile_variant=args.tile_variant), torch.cuda.Stream()
        sx.set_stream(stx.cuda_stream)
        sx.initialize_solution(fb.IC_TGV, (0.1,))
        sx.set_dt(dt)
        sx.run(2)  # first (eager) step and the graph capture
        flight.append((sx, stx))
    bufs = [torch.empty(s.shape, dtype=torch.float64, pin_memory=True).numpy() for _ in flight]
    for (sx, _), b in zip(flight, bufs):
        sx.get_state(out=b)

    def e2e_round(nsteps):
        for i in range(nsteps):
            k = i % len(flight)
            sx = flight[k][0]
            sx.set_state(bufs[k])         # pinned host -> device
            sx.run(1)                     # one RK step (graph replay)
            sx.get_state_async(bufs[k])   # device -> pinned host

    e2e_round(len(flight))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _, stx in flight[1:]:
        stx.wait_event(e0)
    e2e_round(args.e2e_steps)
    for _, stx in flight[1:]:
        ev = torch.cuda.Event()
        ev.record(stx)
        stream.wait_event(ev)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1)
    del flight[1:]

    # the same copies alone (a state in on one stream, a state out on
    # another, as in the end-to-end loop): the end-to-end rate if the RK
    # step itself took no time, i.e. the PCIe bound of that number
    hin = torch.empty(s.shape, dtype=torch.float64, pin_memory=True)
    hout = torch.empty(s.shape, dtype=torch.float64, pin_memory=True)
    din = torch.empty(s.shape, dtype=torch.float64, device=f"cuda:{local}")
    dout = torch.empty_like(din)
    cin, cout = torch.cuda.Stream(), torch.cuda.Stream()

    def copies(n):
        for _ in range(n):
            with torch.cuda.stream(cin):
                din.copy_(hin, non_blocking=True)
            with torch.cuda.stream(cout):
                hout.copy_(dout, non_blocking=True)

    copies(2)
    torch.cuda.synchronize()
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0.record(stream)
    cin.wait_event(c0)
    cout.wait_event(c0)
    copies(args.e2e_steps)
    for cs in (cin, cout):
        ev = torch.cuda.Event()
        ev.record(cs)
        stream.wait_event(ev)
    c1.record(stream)
    torch.cuda.synchronize()
    ms_copy = c0.elapsed_time(c1)
    del hin, hout, din, dout

    ms, ms_e2e, ms_copy = max_over_ranks([ms, ms_e2e, ms_copy], "cuda")

    if rank == 0:
        value = whole_job_rate(world, dof, nrk, args.steps, ms)
        e2e = whole_job_rate(world, dof, nrk, args.e2e_steps, ms_e2e)
        e2e_copy_bound = whole_job_rate(world, dof, nrk, args.e2e_steps, ms_copy)
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
            "config": headline_config(world), "dt": dt,
            "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": dof * 8, "d2h_bytes_per_step": dof * 8,
                    "cases_in_flight": args.e2e_cases, "steps": args.e2e_steps,
                    "copy_bound": e2e_copy_bound, "frac_of_copy_bound": e2e / e2e_copy_bound},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                         "traffic": profiled_traffic("traffic_bytes_per_launch"),
                         "traffic_source": "profiles/fp64_stage_tgv32_p3.md (ncu, one launch)",
                         "kernel": "k_elem_tma<3, 3>" if inf.tensor_kernels == 2 else "k_elem_tp<3, 3>",
                         "tile_variant": inf.tile_variant, "elems_per_block": inf.elems_per_block,
                         "kernel_ms": kt["element_stage"], "algorithmic_bytes": elem_bytes,
                         "peak_source": peak_kind},
            "kernels_ms": {"element_stage": kt["element_stage"], "faces": kt["faces"],
                           "faces_GBps": face_bytes / (kt["faces"] / 1e3) / 1e9},
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_cpu_baseline:
            res, err = headline_reference(args.cpu_steps, 2)
            if res:
                out["cpu_baseline"] = {
                    "value": res["dof_stage_per_s"], "unit": METRIC, "cores": res["threads"], "kind": "reference",
                    "sample": res["sample"], "cpu": res["cpu"], "value_1thread": res["dof_stage_per_s_1thread"]}
            else:
                out["cpu_baseline"] = {"value": None, "unit": METRIC, "cores": 0, "kind": "reference",
                                       "sample": err}
        if world == 1 and args.forms:
            out["forms"] = run_forms(args, fb, torch, stream, dt)
        print(json.dumps(out))
    del s
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
