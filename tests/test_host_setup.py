"""Product host setup (no GPU) against the reference's setup arrays.

The library is created in host-only mode (device = -1): mesh generation,
face connectivity (left/right choice and flux-point orientation), metrics
and the dense FR operators must match the reference's dumps.
"""
import numpy as np
import pytest

import flurrypp_b200 as fb
from conftest import deck_path, golden_cases, load_golden, perturb_opts, rel_err

OPS = ["opp_spts_to_fpts", "opp_correction"] + [f"opp_grad_spts_{d}" for d in range(3)] + \
      [f"opp_extrapolateFn_{d}" for d in range(3)]
GEOM = ["pos_spts", "detJac_spts", "JGinv_spts", "norm_fpts", "dA_fpts", "xv"]


def host_case(meta):
    return fb.Solver(deck_path(meta), device=-1, **perturb_opts(meta))


@pytest.mark.parametrize("case", golden_cases(require=("face_eL",)))
def test_operators_match(case):
    a, meta = load_golden(case)
    s = host_case(meta)
    for n in OPS:
        if n not in a:
            continue
        # the reference tabulates its 1-D nodes to 15 digits; ours are exact
        assert rel_err(s.get_array(n), a[n].ravel()) < 2e-14, n


@pytest.mark.parametrize("case", golden_cases(require=("face_eL",)))
def test_geometry_match(case):
    a, meta = load_golden(case)
    s = host_case(meta)
    for n in GEOM:
        assert rel_err(s.get_array(n), a[n].ravel()) < 1e-14, n


@pytest.mark.parametrize("case", golden_cases(require=("face_eL",)))
def test_faces_match(case):
    """Same faces, same left/right elements, same right flux-point map."""
    a, meta = load_golden(case)
    s = host_case(meta)
    eL, lL, eR, lR, bc = (s.get_array(n) for n in ["face_eL", "face_locL", "face_eR", "face_locR", "face_bc"])
    fptR = s.get_array("face_fptR").reshape(len(eL), -1)
    mine = {(x, y): (z, w, b if z < 0 else -1, tuple(f)) for x, y, z, w, b, f in zip(eL, lL, eR, lR, bc, fptR)}
    rf = a["face_fptR"].reshape(len(a["face_eL"]), -1)
    ref = {(x, y): (z, w, b if z < 0 else -1, tuple(f) if z >= 0 else tuple([-1] * rf.shape[1]))
           for x, y, z, w, b, f in zip(a["face_eL"], a["face_locL"], a["face_eR"], a["face_locR"], a["face_bc"], rf)}
    assert mine == ref


def test_bad_deck_is_an_error():
    with pytest.raises(fb.FrError) as ei:
        fb.Solver("/nonexistent/deck", device=-1)
    assert ei.value.code == fb.FR_ERR_ARG


def test_host_only_case_rejects_device_calls(tmp_path):
    a, meta = load_golden("vortex2d_p3_8")
    s = host_case(meta)
    with pytest.raises(fb.FrError) as ei:
        s.calc_residual(0)
    assert ei.value.code == fb.FR_ERR_STATE
    with pytest.raises(fb.FrError) as ei:
        s.set_state(a["U_init"])
    assert ei.value.code == fb.FR_ERR_STATE


def test_roe_3d_rejected(tmp_path):
    src = open(deck_path({"deck": "tgv3d_p3_4"})).read().replace("riemannType   0", "riemannType   1")
    p = tmp_path / "roe3d.deck"
    p.write_text(src)
    with pytest.raises(fb.FrError) as ei:
        fb.Solver(str(p), device=-1)
    assert ei.value.code == fb.FR_ERR_UNSUPPORTED
