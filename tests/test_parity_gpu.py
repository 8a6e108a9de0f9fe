"""Parity of the CUDA path with the reference (golden fixtures) and the oracle.

Every case starts the GPU from the fixture's own initial state (the state the
reference ran from) and compares, through the C ABI:
  - one residual evaluation: divF, U_fpts, F_spts, Fn_fpts, disFn_fpts;
  - the state after the fixture's N time steps (reference: 1e-10 relative);
  - element time steps for the local-CFL case.
Residual tolerances are relative to the larger of max|divF| and max|F_spts|,
since the residual is a difference of flux terms of that size (the oracle and
the reference differ by up to ~2e-12 of max|divF| at Mach 0.1 for that reason).
"""
import numpy as np
import pytest

import flurrypp_b200 as fb
import fr_oracle as O
from conftest import deck_path, golden_cases, harness_ic, has_pmg, load_golden, perturb_opts, rel_err

pytestmark = pytest.mark.gpu

RESID_TOL = 1e-12   # per residual evaluation
STEP_TOL = 1e-10    # state after N steps


def gpu_case(meta, **kw):
    s = fb.Solver(deck_path(meta), debug_arrays=1, **perturb_opts(meta), **kw)
    if "--cfl-dt" in meta["harness_args"]:
        s.set_dt(meta["dt"])
    return s


@pytest.mark.parametrize("case", golden_cases())
def test_residual_matches_reference(case):
    a, meta = load_golden(case)
    s = gpu_case(meta)
    s.set_state(a["U_init"])
    s.calc_residual(0)
    fscale = float(np.max(np.abs(a["F_spts"])))
    shp = a["divF_0"].shape
    assert rel_err(s.get_residual(0), a["divF_0"], fscale) < RESID_TOL
    assert rel_err(s.get_array("U_fpts").reshape(a["U_fpts"].shape), a["U_fpts"]) < 1e-13
    assert rel_err(s.get_array("F_spts").reshape(a["F_spts"].shape), a["F_spts"]) < 1e-13
    assert rel_err(s.get_array("Fn_fpts").reshape(a["Fn_fpts"].shape), a["Fn_fpts"]) < 1e-12
    assert rel_err(s.get_array("disFn_fpts").reshape(a["disFn_fpts"].shape), a["disFn_fpts"], fscale) < RESID_TOL
    assert shp == s.shape
    if "dU_spts" in a:  # viscous: LDG jumps and corrected gradients
        # dUc = UC - U is a difference of nearly equal traces: measured
        # against the size of the traces
        uscale = float(np.max(np.abs(a["U_fpts"])))
        assert rel_err(s.get_array("dUc_fpts").reshape(a["dUc_fpts"].shape), a["dUc_fpts"], uscale) < 1e-13
        gscale = float(np.max(np.abs(a["dU_spts"])))
        assert rel_err(s.get_array("dU_spts").reshape(a["dU_spts"].shape), a["dU_spts"], gscale) < 1e-11
        assert rel_err(s.get_array("dU_fpts").reshape(a["dU_fpts"].shape), a["dU_fpts"], gscale) < 1e-11


@pytest.mark.parametrize("case", golden_cases())
def test_steps_match_reference(case):
    a, meta = load_golden(case)
    s = gpu_case(meta)
    s.set_state(a["U_init"])
    for _ in range(meta["steps"]):
        s.update()
        if has_pmg(meta):  # the driver's loop: update, then the V-cycle
            s.pmg_cycle()
    U = s.get_state()
    assert rel_err(U, a["U_final"]) < STEP_TOL
    if "ele_dt" in a:
        assert rel_err(s.get_array("ele_dt"), a["ele_dt"]) < 1e-12
    inf = s.info()
    assert inf.iter == meta["steps"]
    assert abs(inf.time - a["time_dt"][0]) <= 1e-12 * max(1.0, abs(a["time_dt"][0]))


@pytest.mark.parametrize("case", ["vortex2d_p3_8", "tgv3d_p3_4_perturbed", "localdt_jameson2d_p3",
                                  "channel2d_p2", "euler_fwd2d_p1", "pmg_vortex2d_p3_8", "ns_walls2d_p2",
                                  "motion2_2d_p3_jameson", "motion5_3d_p1"])
def test_graph_run_equals_update_loop(case):
    """fr_run (CUDA-graph steady state) gives the same bits as fr_update."""
    a, meta = load_golden(case)
    s1, s2 = gpu_case(meta), gpu_case(meta)
    s1.set_state(a["U_init"])
    s2.set_state(a["U_init"])
    for _ in range(meta["steps"]):
        s1.update()
        if has_pmg(meta):
            s1.pmg_cycle()
    s2.run(meta["steps"])
    assert np.array_equal(s1.get_state(), s2.get_state())


@pytest.mark.parametrize("precision", [fb.FR_PREC_FP64, fb.FR_PREC_MIXED])
@pytest.mark.parametrize("case", ["pmg_vortex2d_p3_8", "chbump_p2_pmg"])
def test_pmg_run_on_caller_stream_equals_update_loop(case, precision):
    """A P-multigrid case put on a stream of the caller's (fr_set_stream) and
    advanced by fr_run in one eager step, one ten-step graph and two one-step
    graphs gives the same bits as update() + pmg_cycle() on its own stream:
    the coarse levels move to the caller's stream with the case."""
    import torch

    a, meta = load_golden(case)
    s1, s2 = gpu_case(meta, precision=precision), gpu_case(meta, precision=precision)
    st = torch.cuda.Stream()
    s2.set_stream(st.cuda_stream)
    s1.set_state(a["U_init"])
    s2.set_state(a["U_init"])
    n = 13
    for _ in range(n):
        s1.update()
        s1.pmg_cycle()
    s2.run(n)
    assert np.array_equal(s1.get_state(), s2.get_state())


@pytest.mark.parametrize("case", golden_cases())
def test_initial_condition_matches_reference(case):
    a, meta = load_golden(case)
    kind, prm = harness_ic(meta)
    s = gpu_case(meta)
    s.initialize_solution(kind, prm)
    assert rel_err(s.get_state(), a["U_init"]) < 1e-14


def test_vortex_32x32_1000_steps():
    """2-D Euler vortex, 32x32 P3, CFL 0.5 fixed dt, 1000 RK4 steps, from the
    product's own initial condition: the reference's final state to 1e-10."""
    a, meta = load_golden("vortex2d_p3_32_1000")
    s = fb.Solver(deck_path(meta))
    s.initialize_solution(fb.IC_VORTEX, (5.0, 0.0, 0.0, 0.5))
    s.set_dt(meta["dt"])
    s.calc_residual(0)
    assert rel_err(s.get_residual(0), a["divF_0"]) < RESID_TOL
    s.run(meta["steps"])
    assert rel_err(s.get_state(), a["U_final"]) < STEP_TOL


def test_residual_norm_matches_oracle():
    a, meta = load_golden("vortex2d_p3_8")
    s = gpu_case(meta)
    s.set_state(a["U_init"])
    s.calc_residual(0)
    p = O.params_from_deck(deck_path(meta))
    c = O.OracleCase(a, p)
    for rt in (1, 2, 3):
        assert np.allclose(s.residual_norm(rt), c.residual_norm(a["divF_0"], rt), rtol=1e-12, atol=0)


@pytest.mark.parametrize("prec", [fb.FR_PREC_FP64, fb.FR_PREC_MIXED])
def test_nan_residual_fails_every_norm(prec):
    """One NaN value of the state makes the residual NaN in a few elements;
    every norm reports FR_ERR_NONFINITE, the maximum (resType 3) included,
    as the reference's writeResidual stops on a NaN residual."""
    a, meta = load_golden("vortex2d_p3_8")
    s = fb.Solver(deck_path(meta), precision=prec)
    U = a["U_init"].copy()
    U[3, 5, 1] = np.nan
    s.set_state(U)
    s.calc_residual(0)
    for rt in (1, 2, 3):
        with pytest.raises(fb.FrError) as ei:
            s.residual_norm(rt)
        assert ei.value.code == fb.FR_ERR_NONFINITE, rt


def test_nonfinite_state_is_reported():
    """Host-side fault injection: a poisoned state is caught, not trapped."""
    a, meta = load_golden("vortex2d_p3_8")
    s = gpu_case(meta)
    U = a["U_init"].copy()
    U[3, 5, 1] = np.nan
    s.set_state(U)
    with pytest.raises(fb.FrError) as ei:
        s.check_state()
    assert ei.value.code == fb.FR_ERR_NONFINITE
    U[3, 5, 1] = a["U_init"][3, 5, 1]
    U[0, 0, 0] = -1.0
    s.set_state(U)
    with pytest.raises(fb.FrError):
        s.check_state()
    s.set_state(a["U_init"])
    s.check_state()


def test_calc_dt_matches_reference_formula():
    """Global CFL dt on the initial state equals the harness's --cfl-dt value."""
    a, meta = load_golden("vortex2d_p3_8")
    src = open(deck_path(meta)).read().replace("dtType        0", "dtType 1\nCFL 0.5")
    import tempfile, os
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "d.deck")
        open(p, "w").write(src)
        s = fb.Solver(p)
        s.set_state(a["U_init"])
        dt = s.calc_dt()
    assert abs(dt - meta["dt"]) <= 1e-14 * meta["dt"]


@pytest.mark.parametrize("variant", [{"generic_kernels": 1}, {"no_tma": 1}, {}])
@pytest.mark.parametrize("case", ["tgv3d_p3_4_perturbed", "vortex2d_p3_8", "channel2d_p2", "tgv3d_p4_3_perturbed"])
def test_element_kernel_variants_agree(case, variant):
    """General sparse-operator, tensor-product and TMA element kernels all
    reproduce the reference (residual and N steps)."""
    a, meta = load_golden(case)
    s = gpu_case(meta, **variant)
    kind = s.info().tensor_kernels
    if variant.get("generic_kernels"):
        assert kind == 0
    elif variant.get("no_tma"):
        assert kind == 1
    s.set_state(a["U_init"])
    s.calc_residual(0)
    fscale = float(np.max(np.abs(a["F_spts"])))
    assert rel_err(s.get_residual(0), a["divF_0"], fscale) < RESID_TOL
    s.set_state(a["U_init"])
    for _ in range(meta["steps"]):
        s.update()
    assert rel_err(s.get_state(), a["U_final"]) < STEP_TOL


def test_cpp_driver_matches_python_binding():
    """The C++ solver adapter (include/fr_solver.hpp) driven like the
    reference's main loop gives the same residual history as the binding."""
    import os
    import subprocess
    from conftest import ROOT, DECKS
    exe = os.path.join(ROOT, "flurrypp_b200", "examples", "flurry_b200")
    deck = os.path.join(DECKS, "ic1_2d_p3.deck")
    out = subprocess.run([exe, deck, "10", "5"], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    last = [l for l in out.stdout.splitlines() if l.startswith("iter")][-1].split()
    res_cpp = np.array([float(x) for x in last[5:]])
    s = fb.Solver(deck)
    s.initialize_solution(fb.IC_DECK)
    for _ in range(10):
        s.update()
    res_py = s.residual_norm(2)
    assert np.allclose(res_cpp, res_py, rtol=1e-9, atol=0)


@pytest.mark.parametrize("case", ["vortex2d_p3_8", "tgv3d_p3_4_perturbed", "p5_2d", "channel2d_p2"])
def test_plain_tile_variants_bit_identical(case):
    """The plain form's autotuner chooses between element tile shapes that
    compute every point with the same operations: bit-identical states."""
    a, meta = load_golden(case)
    outs = []
    for v in (0, 1):
        s = gpu_case(meta, tile_variant=v)
        inf = s.info()
        if inf.tile_variant != v:
            pytest.skip("no TMA tiles for this case")
        s.set_state(a["U_init"])
        s.run(meta["steps"])
        outs.append(s.get_state())
    assert np.array_equal(outs[0], outs[1])
    assert rel_err(outs[0], a["U_final"]) < STEP_TOL


@pytest.mark.parametrize("precision", [fb.FR_PREC_FP64, fb.FR_PREC_MIXED])
@pytest.mark.parametrize("case", ["vortex2d_p3_8", "pmg_vortex2d_p3_8", "ns_vortex2d_p3_6", "tgv3d_p3_4_perturbed"])
def test_programmatic_launch_overlap_changes_nothing(case, precision):
    """Small cases chain their launches with programmatic dependent launch
    (each kernel's prologue overlaps the previous kernel's tail).  The same
    steps with plain stream order give bit-identical states, in the
    graph-replayed and the step-by-step loop."""
    a, meta = load_golden(case)
    outs = []
    for no_pdl in (0, 1):
        for graph in (True, False):
            s = gpu_case(meta, precision=precision, no_pdl=no_pdl)
            s.set_state(a["U_init"])
            if graph:
                s.run(4)
            else:
                for _ in range(4):
                    s.update()
                    if has_pmg(meta):  # fr_run's step: update, then the V-cycle
                        s.pmg_cycle()
            outs.append(s.get_state())
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])


@pytest.mark.parametrize("precision", [fb.FR_PREC_FP64, fb.FR_PREC_MIXED])
def test_async_state_copy(precision):
    """fr_get_state_async into pinned memory, read after the stream is
    reached, equals fr_get_state."""
    import torch

    a, meta = load_golden("tgv3d_p3_4")
    s = gpu_case(meta, precision=precision)
    s.set_state(a["U_init"])
    s.run(3)
    pinned = torch.empty(s.shape, dtype=torch.float64, pin_memory=True).numpy()
    s.get_state_async(pinned)
    s.synchronize()
    assert np.array_equal(pinned, s.get_state())


def test_moving_mesh_pmg_run_equals_update_loop():
    """A moving mesh with P-multigrid (every level moves its own mesh with its
    own time): the graph-replayed run, ten steps per graph launch and then
    single steps, equals update + pmg_cycle step by step, bit for bit, and
    the reference after its six steps."""
    a, meta = load_golden("pmg_motion2d_p2")
    outs = []
    for graph in (True, False):
        s = gpu_case(meta)
        s.set_state(a["U_init"])
        if graph:
            s.run(meta["steps"])
            s.run(11)
        else:
            for i in range(meta["steps"] + 11):
                s.update()
                s.pmg_cycle()
                if i == meta["steps"] - 1:
                    assert rel_err(s.get_state(), a["U_final"]) < STEP_TOL
        outs.append(s.get_state())
    assert np.isfinite(outs[0]).all()
    assert np.array_equal(outs[0], outs[1])


def test_moving_mesh_cases_are_not_batched():
    a, meta = load_golden("motion1_2d_p3")
    s = gpu_case(meta)
    s.set_state(a["U_init"])
    with pytest.raises(fb.FrError) as ei:
        fb.Batch([s])
    assert ei.value.code == fb.FR_ERR_UNSUPPORTED


def test_moving_mesh_precision_form_refused():
    a, meta = load_golden("motion1_2d_p3")
    with pytest.raises(fb.FrError) as ei:
        gpu_case(meta, precision=fb.FR_PREC_MIXED)
    assert ei.value.code == fb.FR_ERR_UNSUPPORTED


@pytest.mark.parametrize("case", golden_cases(require=("err_integrals", "U_init")))
def test_error_integrals_match_reference(case):
    """solver::integrateError (errorNorm 0, 1, 2) after the fixture's steps:
    the exact-solution error integrals of testCase 1 as the reference reports
    them, on straight, curved and moving meshes."""
    a, meta = load_golden(case)
    s = gpu_case(meta)
    s.set_state(a["U_init"])
    for _ in range(meta["steps"]):
        s.update()
    want = a["err_integrals"]
    for norm in range(3):
        got = s.integrate_error(norm)
        scale = float(np.max(np.abs(want[norm])))
        assert np.max(np.abs(got - want[norm])) <= 1e-9 * scale, (norm, got, want[norm])


def test_error_integrals_of_the_reference_vortex_run():
    """The reference's icType 1 vortex, 32x32 P3, 20 steps of the deck's dt,
    started from the deck's own initial condition: L1, L2 and conservation
    error integrals as the reference reports them."""
    a, meta = load_golden("err_ic1_2d_p3_32")
    s = fb.Solver(deck_path(meta))
    s.initialize_solution()
    s.run(meta["steps"])
    assert s.info().time == pytest.approx(a["time_dt"][0], rel=1e-14)
    for norm in range(3):
        got, want = s.integrate_error(norm), a["err_integrals"][norm]
        assert np.max(np.abs(got - want)) <= 1e-9 * np.max(np.abs(want)), (norm, got, want)


@pytest.mark.parametrize("case", golden_cases(require=("wall_force", "U_init")))
def test_boundary_monitors_match_reference(case):
    """Wall-force coefficients as writeResidual prints them and the testCase 2
    mass flux (errorNorm 0, 1, 2), on the face data of a residual evaluated
    after the fixture's steps (2-D/3-D, slip and viscous walls, far field,
    sub/supersonic boundaries, the reference's cylinder mesh)."""
    a, meta = load_golden(case)
    s = gpu_case(meta)
    s.set_state(a["U_init"])
    for _ in range(meta["steps"]):
        s.update()
        if has_pmg(meta):  # the driver's loop: update, then the V-cycle
            s.pmg_cycle()
    s.calc_residual(0)
    f, want = s.wall_force(), a["wall_force"]
    assert np.max(np.abs(f - want)) <= 1e-9 * max(np.max(np.abs(want)), 1e-3), (f, want)
    # inflow and outflow cancel in every norm (n_x carries its sign), so the
    # sums are measured against the unit scale of the non-dimensional fluxes
    flux = a["mass_flux"]
    for norm in range(3):
        got = s.mass_flux(norm)
        assert np.max(np.abs(got - flux[norm])) <= 1e-10 * max(1.0, np.max(np.abs(flux[norm]))), \
            (norm, got, flux[norm])


NORM_CASES = ["vortex2d_p3_8", "lobatto_hu3d_p3", "chbump_p2_pmg", "tgv3d_p3_4_perturbed", "ns_tgv3d_p3_3", "p5_2d"]


@pytest.mark.parametrize("case", NORM_CASES)
def test_residual_norm_matches_reference(case):
    """fr_residual_norm (resType 1, 2, 3) against the norms the reference's
    writeResidual computes, on the residual of the fixture's initial state and
    on that of its state after the fixture's N steps.  The residual itself
    agrees to 1e-12 of the flux scale, and the norms are of residuals up to
    two orders below that scale, hence the relative bounds."""
    import os

    from conftest import ROOT

    a, meta = load_golden(case)
    z = np.load(os.path.join(ROOT, "tests", "golden", "res_norms.npz"))
    s = gpu_case(meta)
    s.set_state(a["U_init"])
    s.calc_residual(0)
    for rt in (1, 2, 3):
        assert np.allclose(s.residual_norm(rt), z[case + "__initial"][rt - 1], rtol=1e-9, atol=0), rt
    s.run(meta["steps"])  # update() and, with PMG, the V-cycle: the reference driver's step
    s.calc_residual(0)
    for rt in (1, 2, 3):
        assert np.allclose(s.residual_norm(rt), z[case + "__final"][rt - 1], rtol=1e-7, atol=0), rt


@pytest.mark.parametrize("n", [16, 32])
def test_tgv_matches_reference_element_sums(n):
    """3-D Taylor-Green vortex, 16^3 and 32^3 hexes (the benchmark's own
    workload), P3, FP64, from the product's own initial condition:
    per-element sums of the initial state (1e-14), of the residual (1e-12 of
    the flux scale) and of the state after 5 RK4 steps (1e-10) against the
    reference's, and the residual norms."""
    import json
    import os

    from conftest import ROOT

    z = np.load(os.path.join(ROOT, "tests", "golden", f"tgv3d_p3_{n}_sums.npz"))
    meta = json.loads(str(z["meta"]))
    s = fb.Solver(deck_path(meta))
    s.initialize_solution(fb.IC_TGV, (0.1,))
    s.set_dt(meta["dt"])
    assert rel_err(s.get_state().sum(axis=0), z["U_init_elem_sum"]) < 1e-14
    s.calc_residual(0)
    fscale = 64 * max(float(z["divF_0_absmax"].max()), float(z["F_spts_absmax"].max()))
    assert rel_err(s.get_residual(0).sum(axis=0), z["divF_0_elem_sum"], fscale) < RESID_TOL
    for rt in (1, 2, 3):
        assert np.allclose(s.residual_norm(rt), z["res_norms"][rt - 1], rtol=1e-9, atol=0), rt
    s.run(meta["steps"])
    assert rel_err(s.get_state().sum(axis=0), z["U_final_elem_sum"]) < STEP_TOL
    s.calc_residual(0)
    for rt in (1, 2, 3):
        assert np.allclose(s.residual_norm(rt), z["res_norms_final"][rt - 1], rtol=1e-7, atol=0), rt


@pytest.mark.parametrize("case", ["naca_p4_sums", "cyl3d_p2_sums", "cyl3d_visc_p2_sums"])
def test_reference_test_meshes_match_element_sums(case, tmp_path):
    """The reference's own NACA 0012 (2,724 9-node quads, P4, CFL-based dt)
    and 3-D cylinder (3,756 hexes, P2) test meshes, from the deck's initial
    condition: per-element sums of the initial state (1e-14), of the
    residual (1e-12 of the flux scale) and of the state after the steps
    (1e-10) against the reference's, the residual norms before and after,
    and the boundary monitors after the steps."""
    import json
    import os

    from conftest import ROOT

    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_golden import stage_deck  # the meshes are kept gzip-compressed

    z = np.load(os.path.join(ROOT, "tests", "golden", f"{case}.npz"))
    meta = json.loads(str(z["meta"]))
    s = fb.Solver(stage_deck(meta["deck"], str(tmp_path)))
    s.initialize_solution()
    nS = s.shape[0]
    assert rel_err(s.get_state().sum(axis=0), z["U_init_elem_sum"]) < 1e-14
    s.calc_residual(0)
    fscale = nS * max(float(z["divF_0_absmax"].max()), float(z["F_spts_absmax"].max()))
    assert rel_err(s.get_residual(0).sum(axis=0), z["divF_0_elem_sum"], fscale) < RESID_TOL
    for rt in (1, 2, 3):
        assert np.allclose(s.residual_norm(rt), z["res_norms"][rt - 1], rtol=1e-9, atol=0), rt
    s.run(meta["steps"])
    assert rel_err(s.get_state().sum(axis=0), z["U_final_elem_sum"]) < STEP_TOL
    assert abs(s.info().time - z["time_dt"][0]) <= 1e-12 * max(1.0, abs(z["time_dt"][0]))
    s.calc_residual(0)
    for rt in (1, 2, 3):
        assert np.allclose(s.residual_norm(rt), z["res_norms_final"][rt - 1], rtol=1e-7, atol=0), rt
    want = z["wall_force"]
    assert np.max(np.abs(s.wall_force() - want)) <= 1e-9 * max(np.max(np.abs(want)), 1e-3)
    for norm in range(3):
        got, flux = s.mass_flux(norm), z["mass_flux"][norm]
        assert np.max(np.abs(got - flux)) <= 1e-10 * max(1.0, np.max(np.abs(flux))), (norm, got, flux)
