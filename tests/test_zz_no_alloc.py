"""fr_residual_norm_noalloc: the residual norm with its partial sums in a
fixed static device array, no device allocation by the library.

It must give what fr_residual_norm gives (the reference's writeResidual norm,
src/output.cpp:1011-1090) on the same residual, on two calls in a row (the
second one reuses the static array the first one filled), and refuse sizes
beyond the array.  The file sorts last so the GPU test also runs after every
other test in the same process; it passes alone as well.
"""
import ctypes

import numpy as np
import pytest

import flurrypp_b200 as fb
from conftest import deck_path, load_golden, perturb_opts

FR_OK, FR_ERR_ARG = 0, 1
FR_ERR_NONFINITE = fb.FR_ERR_NONFINITE
NORM_RTOL = 1e-12  # summation order differs (block tree vs element order)


def _entry():
    f = fb.lib.fr_residual_norm_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                  ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    return f


def test_noalloc_refuses_sizes_beyond_the_static_array():
    """Argument checks run before any device work (no GPU needed)."""
    f = _entry()
    out = np.zeros(5)
    fake = ctypes.c_void_p(256)  # never dereferenced: every call below is refused first
    optr = out.ctypes.data_as(ctypes.c_void_p)
    assert f(fake, fake, 3, 6, 10, 5, 2, optr, None) == FR_ERR_ARG   # order 6: 343 spts > 216
    assert f(fake, fake, 2, 3, 10, 5, 2, optr, None) == FR_ERR_ARG   # nFields != nDims + 2
    assert f(fake, fake, 2, 3, 0, 4, 2, optr, None) == FR_ERR_ARG    # no elements
    assert f(fake, fake, 2, 3, 10, 4, 4, optr, None) == FR_ERR_ARG   # resType 4
    assert f(None, fake, 2, 3, 10, 4, 2, optr, None) == FR_ERR_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["vortex2d_p3_8", "tgv3d_p3_4_perturbed", "p5_2d", "lobatto_hu3d_p3"])
def test_noalloc_norm_matches_residual_norm_twice(case):
    import torch

    a, meta = load_golden(case)
    s = fb.Solver(deck_path(meta), **perturb_opts(meta))
    s.set_state(a["U_init"])
    s.calc_residual(0)
    s.synchronize()
    divF, nbytes = s.device_ptr("divF_0")
    assert nbytes == s.nSpts * s.nEles * s.nFields * 8
    # the caller's own device copy of the Jacobian determinants, [nSpts][nEles]
    detJ = torch.from_numpy(s.get_array("detJac_spts")).to("cuda:0")
    assert detJ.numel() == s.nSpts * s.nEles
    torch.cuda.synchronize()
    f = _entry()
    for rt in (1, 2, 3):
        want = s.residual_norm(rt)
        for call in range(2):
            out = np.full(s.nFields, np.nan)
            st = f(divF, detJ.data_ptr(), s.nDims, s.order, s.nEles, s.nFields, rt,
                   out.ctypes.data_as(ctypes.c_void_p), None)
            assert st == FR_OK, (call, st)
            assert np.allclose(out, want, rtol=NORM_RTOL, atol=0), (rt, call, out, want)


@pytest.mark.gpu
def test_noalloc_refuses_the_precision_forms_fp32_arrays():
    """A precision-form case's divF_0 is FP32; read as FP64 it would be
    garbage, so the entry point refuses it before any device work."""
    a, meta = load_golden("vortex2d_p3_8")
    s = fb.Solver(deck_path(meta), precision=fb.FR_PREC_MIXED)
    s.set_state(a["U_init"])
    s.calc_residual(0)
    s.synchronize()
    divF, nbytes = s.device_ptr("divF_0")
    assert nbytes == s.nSpts * s.nEles * s.nFields * 4
    out = np.zeros(s.nFields)
    f = _entry()
    fp64 = fb.Solver(deck_path(meta))  # a real FP64 detJ-sized array to pass beside it
    fp64.set_state(a["U_init"])
    fp64.calc_residual(0)
    good, _ = fp64.device_ptr("divF_0")
    st = f(divF, good, s.nDims, s.order, s.nEles, s.nFields, 2, out.ctypes.data_as(ctypes.c_void_p), None)
    assert st == FR_ERR_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("rt", [1, 2, 3])
def test_noalloc_reports_a_nan_residual_for_every_norm(rt):
    """One NaN value of the state gives NaN residuals in a few elements only;
    every norm, the maximum included, must report it."""
    import torch

    a, meta = load_golden("vortex2d_p3_8")
    s = fb.Solver(deck_path(meta))
    U = a["U_init"].copy()
    U[3, 5, 1] = np.nan
    s.set_state(U)
    s.calc_residual(0)
    s.synchronize()
    divF, _ = s.device_ptr("divF_0")
    detJ = torch.from_numpy(s.get_array("detJac_spts")).to("cuda:0")
    torch.cuda.synchronize()
    out = np.zeros(s.nFields)
    st = _entry()(divF, detJ.data_ptr(), s.nDims, s.order, s.nEles, s.nFields, rt,
                  out.ctypes.data_as(ctypes.c_void_p), None)
    assert st == FR_ERR_NONFINITE
