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


SUMMARY_CASES = [c for c in golden_cases(require=("ref_face_eL",))]


@pytest.mark.parametrize("case", SUMMARY_CASES)
def test_reference_test_mesh_setup_matches(case, tmp_path):
    """The reference's own large test meshes (NACA 0012 of 9-node quads, the
    3-D cylinder of linear hexes), read from the Gmsh file: per-element sums of
    the metric arrays and the whole face table match the reference's setup."""
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from make_golden import setup_summary, stage_deck

    a, meta = load_golden(case)
    s = fb.Solver(stage_deck(meta["deck"], str(tmp_path)), device=-1)
    inf = s.info()
    nS, nFp, E, nd = inf.nSpts, inf.nFpts, inf.nEles, inf.nDims
    mine = setup_summary({
        "detJac_spts": s.get_array("detJac_spts").reshape(nS, E),
        "dA_fpts": s.get_array("dA_fpts").reshape(nFp, E),
        "norm_fpts": s.get_array("norm_fpts").reshape(nFp, E, nd),
        "pos_spts": s.get_array("pos_spts").reshape(nS, E, nd),
        "JGinv_spts": s.get_array("JGinv_spts").reshape(nd, nS, E, nd),
    })
    for k, v in mine.items():
        # a sum of unit normals cancels: its error is relative to the nFp terms summed
        scale = float(nFp) if k == "sum_norm_fpts" else None
        assert rel_err(v.ravel(), a[k].ravel(), scale) < 1e-13, k
    eL, lL, eR, lR, bc = (s.get_array(n) for n in ["face_eL", "face_locL", "face_eR", "face_locR", "face_bc"])
    fptR = s.get_array("face_fptR").reshape(len(eL), -1)
    got = {(x, y): (z, w, b if z < 0 else -1, tuple(f) if z >= 0 else ())
           for x, y, z, w, b, f in zip(eL, lL, eR, lR, bc, fptR)}
    rf = a["ref_face_fptR"].reshape(len(a["ref_face_eL"]), -1)
    want = {(x, y): (z, w, b if z < 0 else -1, tuple(f) if z >= 0 else ())
            for x, y, z, w, b, f in zip(a["ref_face_eL"], a["ref_face_locL"], a["ref_face_eR"],
                                        a["ref_face_locR"], a["ref_face_bc"], rf)}
    assert got == want


def test_curved_element_shapes_refused_like_the_reference(tmp_path):
    """8-node serendipity quads and triangles are not on the path: the
    reference stops in its shape functions (src/funcs.cpp:159-160) or reads
    simplices as collapsed quads; the product refuses both at setup."""
    from flurrypp_b200.meshgen import write_gmsh
    import shutil
    src = deck_path({"deck": "curved2d_q2_p3"})
    for typ, nodes in ((16, 8), (2, 3)):
        msh = tmp_path / "curved2d_q2.msh"
        lines = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$PhysicalNames", "2", '1 1 "bottom"',
                 '2 2 "fluid"', "$EndPhysicalNames", "$Nodes", "8"]
        lines += [f"{i + 1} {i} {i % 3} 0" for i in range(8)]
        lines += ["$EndNodes", "$Elements", "1", f"1 {typ} 2 2 2 " + " ".join(str(i + 1) for i in range(nodes)),
                  "$EndElements"]
        msh.write_text("\n".join(lines) + "\n")
        shutil.copyfile(src, tmp_path / "d.deck")
        with pytest.raises(fb.FrError) as ei:
            fb.Solver(str(tmp_path / "d.deck"), device=-1)
        assert ("Lagrange quad" in str(ei.value)) if typ == 16 else ("collapsed" in str(ei.value))


@pytest.mark.parametrize("extra", ["viscous 1\nRe 100\nMachBound 0.2\nMachWall 0\n", "riemannType 1\n",
                                   "motion 7\n"])
def test_moving_mesh_option_limits(extra, tmp_path):
    """Moving meshes run the inviscid Rusanov path (P-multigrid included),
    with one of the reference's laws 1..5; other combinations are refused."""
    d = tmp_path / "m.deck"
    d.write_text(("motion 2\n" if "motion" not in extra else "") + extra +
                 open(deck_path({"deck": "vortex2d_p3_8"})).read())
    with pytest.raises(fb.FrError) as ei:
        fb.Solver(str(d), device=-1)
    assert ei.value.code in (fb.FR_ERR_UNSUPPORTED, fb.FR_ERR_ARG)
