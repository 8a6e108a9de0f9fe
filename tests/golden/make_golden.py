"""Generate the golden fixtures of the FR path from the reference itself.

Runs the reference solver (FlurryPP, built from its own sources by
``oracle/Makefile`` into ``oracle/_ref/fr_ref_harness``) on each deck under
``tests/golden/decks`` and stores its FP64 outputs as ``<case>.npz`` here:
setup arrays (operators, metrics, face connectivity), the initial state, the
intermediates of one residual evaluation (U_fpts, F_spts, Fn_fpts,
disFn_fpts, divF) and the state after N time steps.

    make -C oracle && python tests/golden/make_golden.py [case ...]

Requires the reference build (this container); the committed .npz files are
what the tests read.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "fr_ref_harness")
TWO_PI = "6.283185307179586"

SETUP = ["opp_spts_to_fpts", "opp_grad_spts_0", "opp_grad_spts_1", "opp_grad_spts_2",
         "opp_extrapolateFn_0", "opp_extrapolateFn_1", "opp_extrapolateFn_2",
         "opp_correction", "opp_correctU_0", "opp_correctU_1", "opp_correctU_2",
         "opp_prolong", "opp_restrict",
         "pos_spts", "detJac_spts", "JGinv_spts", "norm_fpts", "dA_fpts", "xv",
         "face_type", "face_eL", "face_locL", "face_eR", "face_locR", "face_relRot",
         "face_bc", "face_fptR"]
RESID = ["U_init", "U_fpts", "F_spts", "Fn_fpts", "disFn_fpts", "divF_0", "waveSp_fpts",
         "dU_spts", "dU_fpts", "dUc_fpts"]
FINAL = ["U_final", "time_dt", "ele_dt"]

# name -> (deck, harness args, steps, keep)
CASES = {
    "vortex2d_p3_8": ("vortex2d_p3_8", ["--ic", "vortex", "--vortex", "5,0,0,0.5", "--cfl-dt", "0.5"], 20, "all"),
    "vortex2d_p3_32_1000": ("vortex2d_p3_32", ["--ic", "vortex", "--vortex", "5,0,0,0.5", "--cfl-dt", "0.5"], 1000,
                            ["divF_0", "U_final", "time_dt"]),
    "tgv3d_p3_4": ("tgv3d_p3_4", ["--ic", "tgv", "--tgv-mach", "0.1", "--cfl-dt", "0.5"], 5, "all"),
    "tgv3d_p3_4_perturbed": ("tgv3d_p3_4", ["--ic", "tgv", "--tgv-mach", "0.1", "--perturb", "7,0.05",
                                            "--cfl-dt", "0.5"], 5, "all"),
    "tgv3d_p4_3_perturbed": ("tgv3d_p4_3", ["--ic", "tgv", "--tgv-mach", "0.1", "--perturb", "11,0.05",
                                            "--cfl-dt", "0.5"], 3, "all"),
    "tgv3d_p2_4": ("tgv3d_p2_4", ["--ic", "tgv", "--tgv-mach", "0.3", "--cfl-dt", "0.5"], 5, "all"),
    "channel2d_p2": ("channel2d_p2", ["--ic", "vortex", "--vortex", "0.5,0,0.4,0.35", "--cfl-dt", "0.5"], 10, "all"),
    "supsub2d_p3": ("supsub2d_p3", ["--ic", "vortex", "--vortex", "2,0,0,0.5", "--cfl-dt", "0.5"], 10, "all"),
    "roe2d_p2": ("roe2d_p2", ["--ic", "vortex", "--vortex", "5,0,0,0.5", "--cfl-dt", "0.5"], 10, "all"),
    "lobatto_sd2d_p4": ("lobatto_sd2d_p4", ["--ic", "vortex", "--vortex", "5,0.5,0,0.5", "--cfl-dt", "0.4"], 10, "all"),
    "hu2d_p3": ("hu2d_p3", ["--ic", "vortex", "--vortex", "4,0,0.5,0.3", "--cfl-dt", "0.5"], 10, "all"),
    "cplus2d_p2": ("cplus2d_p2", ["--ic", "vortex", "--vortex", "4,0,0,0.4", "--cfl-dt", "0.5"], 10, "all"),
    "localdt_jameson2d_p3": ("localdt_jameson2d_p3", ["--ic", "vortex", "--vortex", "5,0,0,0.5"], 10, "all"),
    "globalcfl_rk2_2d_p2": ("globalcfl_rk2_2d_p2", ["--ic", "vortex", "--vortex", "5,0,0,0.5"], 10, "all"),
    "euler_fwd2d_p1": ("euler_fwd2d_p1", ["--ic", "vortex", "--vortex", "3,0,0,0.5"], 10, "all"),
    "jameson5_2d_p2": ("jameson5_2d_p2", ["--ic", "vortex", "--vortex", "5,0,0,0.5"], 10, "all"),
    "p0_2d": ("p0_2d", ["--ic", "vortex", "--vortex", "5,0,0,0.5"], 10, "all"),
    "p5_2d": ("p5_2d", ["--ic", "vortex", "--vortex", "5,0,0,0.5", "--cfl-dt", "0.5"], 10, "all"),
    "p1_3d": ("p1_3d", ["--ic", "tgv", "--tgv-mach", "0.2", "--cfl-dt", "0.5"], 5, "all"),
    "ic1_2d_p3": ("ic1_2d_p3", ["--cfl-dt", "0.5"], 10, "all"),
    "ic2_2d_p3": ("ic2_2d_p3", ["--cfl-dt", "0.5"], 10, "all"),
    "ns_tgv3d_p2_4_perturbed": ("ns_tgv3d_p2_4", ["--ic", "tgv", "--tgv-mach", "0.1", "--perturb", "5,0.05",
                                                  "--cfl-dt", "0.3"], 4, "all"),
    "ns_tgv3d_p3_3": ("ns_tgv3d_p3_3", ["--ic", "tgv", "--tgv-mach", "0.1", "--cfl-dt", "0.3"], 3, "all"),
    "ns_vortex2d_p3_6": ("ns_vortex2d_p3_6", ["--ic", "vortex", "--vortex", "3,0,0,0.5", "--cfl-dt", "0.3"], 10, "all"),
    "ns_walls2d_p2": ("ns_walls2d_p2", ["--ic", "uniform", "--cfl-dt", "0.2"], 10, "all"),
    "ns_sutherland2d_p3": ("ns_sutherland2d_p3", ["--ic", "vortex", "--vortex", "2,0,0,0.3"], 10, "all"),
    "pmg_vortex2d_p3_8": ("pmg_vortex2d_p3_8", ["--ic", "vortex", "--vortex", "5,0,0,0.5"], 5, "all"),
    "pmg_tgv3d_p3_3": ("pmg_tgv3d_p3_3", ["--ic", "tgv", "--tgv-mach", "0.2", "--cfl-dt", "0.4"], 3, "all"),
    "chbump_p2_pmg": ("chbump_p2_pmg", [], 5, "all"),
    "chbump_p3": ("chbump_p3", [], 10, "all"),
    "wallchar3d_p2": ("wallchar3d_p2", ["--ic", "vortex", "--vortex", "0.3,0,0.4,0.35", "--cfl-dt", "0.5"], 5, "all"),
}


def read_dump(d: str) -> tuple[dict, dict]:
    arrays, meta = {}, {}
    with open(os.path.join(d, "manifest.txt")) as f:
        for line in f:
            t = line.split()
            if not t:
                continue
            if t[0] == "#meta":
                kv = t[1:]
                for k, v in zip(kv[0::2], kv[1::2]):
                    meta[k] = float(v) if k == "dt" else int(v)
                continue
            name, dt, dims = t[0], t[1], [int(x) for x in t[2:]]
            a = np.fromfile(os.path.join(d, name + ".bin"), dtype=np.float64 if dt == "f8" else np.int32)
            arrays[name] = a.reshape(dims)
    return arrays, meta


def run_case(name: str) -> None:
    deck, args, steps, keep = CASES[name]
    deck_path = os.path.join(HERE, "decks", deck + ".deck")
    with tempfile.TemporaryDirectory() as td:
        cmd = [HARNESS, deck_path, td] + args + ["--steps", str(steps)]
        # mesh files named in a deck are relative to the deck's directory
        subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL, cwd=os.path.join(HERE, "decks"))
        arrays, meta = read_dump(td)
    names = SETUP + RESID + FINAL if keep == "all" else keep
    out = {k: arrays[k] for k in names if k in arrays}
    meta.update({"case": name, "deck": deck, "harness_args": args, "steps": steps})
    out["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: {len(out) - 1} arrays, {os.path.getsize(os.path.join(HERE, name + '.npz')) / 1e3:.0f} kB")


def main(argv: list[str]) -> None:
    if not os.path.exists(HARNESS):
        sys.exit(f"{HARNESS} missing: run `make -C oracle` first")
    for name in argv or list(CASES):
        run_case(name)


if __name__ == "__main__":
    main(sys.argv[1:])
