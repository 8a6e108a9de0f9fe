"""The C-ABI library loads and exports every entry point include/*.h declares."""
import pytest
import ctypes
import glob
import os
import re

import flurrypp_b200 as fb
from conftest import ROOT


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(fr_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "fr_calc_residual" in names and "fr_update" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(fb.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_default_opts():
    o = fb.default_opts()
    assert o.precision == fb.FR_PREC_FP64 and o.visc_flux_quirk == 1 and o.perturb == 0


def test_server_reports_setup_failure_without_gpu_work(tmp_path):
    """A request whose deck cannot be read fails with FR_ERR_ARG (host path)."""
    srv = fb.Server(budget_bytes=1 << 20, max_inflight=1, check_every=1, device=0)
    r = srv.submit(str(tmp_path / "missing.deck"), tol=1e-3, max_steps=1)
    with pytest.raises(fb.FrError) as ei:
        srv.wait(r, 30)
    assert ei.value.code == fb.FR_ERR_ARG
    assert srv.poll(r)["status"] == 3
    srv.close()


def test_hardware_work_queues_default_and_caller_value_kept():
    """Importing the package asks for 32 CUDA hardware work queues unless the
    caller chose a value (checked in fresh interpreters, before any CUDA
    context)."""
    import subprocess
    import sys

    code = "import os, flurrypp_b200; print(os.environ['CUDA_DEVICE_MAX_CONNECTIONS'])"
    env = {k: v for k, v in os.environ.items() if k != "CUDA_DEVICE_MAX_CONNECTIONS"}
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "32"
    env["CUDA_DEVICE_MAX_CONNECTIONS"] = "4"
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True,
                         timeout=300)
    assert out.stdout.strip() == "4"
