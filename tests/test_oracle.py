"""The numpy oracle against the reference's own outputs (golden fixtures).

This pins the oracle: its residual of the fixture's initial state and its
state after the fixture's N time steps must reproduce what the reference
solver (built from its sources) produced on the same mesh and state.
"""
import os

import numpy as np
import pytest

import fr_oracle as O
from conftest import ROOT, deck_path, golden_cases, has_motion, has_pmg, load_golden, rel_err

GOLDEN = os.path.join(ROOT, "tests", "golden")

# The residual is a difference of flux terms; rounding is relative to their
# size (the reference's own BLAS order is not reproducible), so residual
# errors are measured against the larger of max|divF| and max|F_spts|.
RESID_TOL = 1e-12
STATE_TOL = 1e-12


def oracle_for(arrays, meta):
    p = O.params_from_deck(deck_path(meta))
    if "--cfl-dt" in meta["harness_args"]:
        p["dtType"] = 0
    p["dt"] = meta["dt"] if p["dtType"] == 0 else 0.0
    return O.OracleCase(arrays, p)


@pytest.mark.parametrize("case", golden_cases())
def test_oracle_residual_matches_reference(case):
    a, meta = load_golden(case)
    if has_motion(meta):
        pytest.skip("the restatement covers static meshes; moving-mesh cases compare the GPU path with the reference")
    c = oracle_for(a, meta)
    keep = {}
    d = c.residual(a["U_init"], keep)
    fscale = float(np.max(np.abs(a["F_spts"])))
    assert rel_err(d, a["divF_0"], fscale) < RESID_TOL
    assert rel_err(keep["U_fpts"], a["U_fpts"]) < 1e-14
    assert rel_err(keep["Fn_fpts"], a["Fn_fpts"]) < 1e-13
    assert rel_err(keep["F_spts"], a["F_spts"]) < 1e-14
    assert rel_err(keep["disFn_fpts"], a["disFn_fpts"], fscale) < RESID_TOL


@pytest.mark.parametrize("case", golden_cases())
def test_oracle_steps_match_reference(case):
    a, meta = load_golden(case)
    if has_pmg(meta) or has_motion(meta):
        pytest.skip("the restatement has no P-multigrid levels or moving meshes; "
                    "the GPU path is compared with the reference directly")
    c = oracle_for(a, meta)
    U = a["U_init"].copy()
    for _ in range(meta["steps"]):
        U = c.update(U)
    assert rel_err(U, a["U_final"]) < STATE_TOL
    if "ele_dt" in a:
        assert rel_err(c.eleDt, a["ele_dt"]) < 1e-13


def test_oracle_flags_planted_error():
    """A planted sign error in the oracle's Rusanov dissipation is caught."""
    a, meta = load_golden("vortex2d_p3_8")
    c = oracle_for(a, meta)
    good = c.residual(a["U_init"])
    orig = O.rusanov

    def bad(UL, UR, n, gam):
        Fn, ws = orig(UL, UR, n, gam)
        return Fn + 1e-9 * (UR - UL), ws

    O.rusanov = bad
    try:
        planted = c.residual(a["U_init"])
    finally:
        O.rusanov = orig
    fscale = float(np.max(np.abs(a["F_spts"])))
    assert rel_err(good, a["divF_0"], fscale) < RESID_TOL
    assert rel_err(planted, a["divF_0"], fscale) > RESID_TOL


def test_residual_norm_definition():
    a, meta = load_golden("vortex2d_p3_8")
    c = oracle_for(a, meta)
    d = a["divF_0"]
    r2 = c.residual_norm(d, 2)
    w = O.spt_weights(2, 3)
    ref = np.sqrt(sum(d[s] ** 2 / a["detJac_spts"][s][:, None] * w[s] for s in range(d.shape[0])).sum(axis=0))
    assert np.allclose(r2, ref, rtol=1e-14)


NORM_CASES = ["vortex2d_p3_8", "lobatto_hu3d_p3", "chbump_p2_pmg", "tgv3d_p3_4_perturbed", "ns_tgv3d_p3_3", "p5_2d"]


@pytest.mark.parametrize("case", NORM_CASES)
def test_oracle_residual_norm_matches_reference(case):
    """The oracle's residual norm (resType 1, 2, 3) of the reference's own
    residual against writeResidual's norm as the reference computed it
    (ele::getNormResidual summed or maximised over the elements)."""
    a, meta = load_golden(case)
    ref = np.load(os.path.join(GOLDEN, "res_norms.npz"))[case + "__initial"]
    c = oracle_for(a, meta)
    for rt in (1, 2, 3):
        assert np.allclose(c.residual_norm(a["divF_0"], rt), ref[rt - 1], rtol=1e-13, atol=0), rt
