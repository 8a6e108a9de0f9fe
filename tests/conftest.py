"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; the rest run on CPU."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
DECKS = os.path.join(GOLDEN, "decks")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden_cases(require=("U_init",)):
    out = []
    for f in sorted(os.listdir(GOLDEN)):
        if f.endswith(".npz"):
            z = np.load(os.path.join(GOLDEN, f))
            if all(r in z.files for r in require):
                out.append(f[:-4])
    return out


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    arrays = {k: z[k] for k in z.files if k != "meta"}
    meta = json.loads(str(z["meta"]))
    return arrays, meta


def deck_path(meta):
    return os.path.join(DECKS, meta["deck"] + ".deck")


def deck_option(meta, key, default=None):
    """First value of `key` in the fixture's deck (the reference's rule)."""
    for line in open(deck_path(meta)):
        t = line.split()
        if len(t) > 1 and t[0] == key:
            return t[1]
    return default


def has_pmg(meta):
    return int(float(deck_option(meta, "PMG", 0))) == 1


def has_motion(meta):
    return int(float(deck_option(meta, "motion", 0))) != 0


def harness_ic(meta):
    """(kind, params) of the product's fr_init_solution matching the fixture."""
    a = meta["harness_args"]
    if "--ic" not in a:
        return 0, ()
    ic = a[a.index("--ic") + 1]
    if ic == "vortex":
        v = [float(x) for x in a[a.index("--vortex") + 1].split(",")] if "--vortex" in a else [5, 0, 0, 0.5]
        return 1, tuple(v)
    if ic == "tgv":
        m = float(a[a.index("--tgv-mach") + 1]) if "--tgv-mach" in a else 0.1
        return 2, (m,)
    if ic == "uniform":
        return 3, ()
    return 0, ()


def perturb_opts(meta):
    a = meta["harness_args"]
    if "--perturb" not in a:
        return {}
    seed, frac = a[a.index("--perturb") + 1].split(",")
    return {"perturb": 1, "seed": int(seed), "perturb_frac": float(frac)}


def rel_err(a, b, scale=None):
    """max|a-b| / max(max|b|, scale)."""
    den = float(np.max(np.abs(b))) if b.size else 0.0
    if scale is not None:
        den = max(den, scale)
    return float(np.max(np.abs(a - b))) / max(den, 1e-300)


@pytest.fixture(scope="session")
def cuda_available():
    try:
        import ctypes
        rt = ctypes.CDLL("libcudart.so.12")
    except OSError:
        rt = None
    if rt is None:
        try:
            import torch
            return torch.cuda.is_available()
        except Exception:
            return False
    n = ctypes.c_int(0)
    return rt.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0
