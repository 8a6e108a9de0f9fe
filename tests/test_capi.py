"""The C-ABI library loads and exports every entry point include/*.h declares."""
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
