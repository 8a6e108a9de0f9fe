"""Precision form (FR_PREC_MIXED): FP32 state, fluxes and operator tables,
compensated RK sums, FP64 time step and norms.

Checked against the reference's FP64 fixtures and the plain form:
  - one residual evaluation within FP32 round-off of the reference's
    (relative to the flux scale, like the plain-form residual test);
  - the state after the fixture's N steps within 1e-6 relative L2 of the
    reference's (the precision form's stated bound);
  - every element tile shape (the autotuner's choices) gives bit-identical
    results, so the autotuner changes speed only;
  - the graph-replayed step equals the step-by-step loop bit for bit;
  - a batch of precision-form cases equals each case run alone, within FP32
    round-off.
"""
import numpy as np
import pytest

import flurrypp_b200 as fb
from conftest import deck_path, golden_cases, has_motion, load_golden, perturb_opts, rel_err

pytestmark = pytest.mark.gpu

RESID_TOL = 2e-5   # FP32 fluxes: residual error relative to max(|divF|, |F_spts|)
L2_TOL = 1e-6      # state after N steps, relative L2 vs the FP64 reference


def mixed_case(meta, **kw):
    s = fb.Solver(deck_path(meta), precision=fb.FR_PREC_MIXED, **perturb_opts(meta), **kw)
    if "--cfl-dt" in meta["harness_args"]:
        s.set_dt(meta["dt"])
    return s


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


# moving meshes run in the plain form only
MIXED_CASES = [c for c in golden_cases(("U_init", "U_final")) if not has_motion(load_golden(c)[1])]


@pytest.mark.parametrize("case", MIXED_CASES)
def test_mixed_residual_near_reference(case):
    a, meta = load_golden(case)
    s = mixed_case(meta, debug_arrays=1)
    s.set_state(a["U_init"])
    s.calc_residual(0)
    d = s.get_residual(0)
    scale = max(np.abs(a["divF_0"]).max(), np.abs(a["F_spts"]).max())
    assert np.abs(d - a["divF_0"]).max() / scale < RESID_TOL


@pytest.mark.parametrize("case", MIXED_CASES)
def test_mixed_steps_within_l2_bound(case):
    a, meta = load_golden(case)
    s = mixed_case(meta)
    s.set_state(a["U_init"])
    s.run(meta["steps"])
    assert rel_l2(s.get_state(), a["U_final"]) < L2_TOL


def test_mixed_vortex_32x32_1000_steps():
    """2-D vortex, 32x32 P3, 1000 RK4 steps from the product's own initial
    condition: within the L2 bound of the reference's final state."""
    a, meta = load_golden("vortex2d_p3_32_1000")
    s = fb.Solver(deck_path(meta), precision=fb.FR_PREC_MIXED)
    s.initialize_solution(fb.IC_VORTEX, (5.0, 0.0, 0.0, 0.5))
    s.set_dt(meta["dt"])
    s.run(meta["steps"])
    err = rel_l2(s.get_state(), a["U_final"])
    assert err < L2_TOL, err


@pytest.mark.parametrize("case", ["vortex2d_p3_8", "tgv3d_p3_4_perturbed", "p5_2d", "p1_3d"])
def test_tile_variants_bit_identical(case):
    a, meta = load_golden(case)
    outs = []
    for v in range(3):
        s = mixed_case(meta, tile_variant=v)
        assert s.info().tile_variant == v
        s.set_state(a["U_init"])
        s.run(5)
        outs.append(s.get_state())
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])


def test_autotuner_fixed_choice_on_a_small_case():
    a, meta = load_golden("tgv3d_p3_4")
    s = mixed_case(meta)
    inf = s.info()
    assert inf.tensor_kernels == 2 and inf.tile_variant == 0 and inf.elems_per_block % 4 == 0


def test_autotuner_times_variants_on_a_large_case(tmp_path):
    """2-D P3, 128^2 elements (2^18 solution points): every tile variant is
    timed at setup (the tensor-core one included) and the fastest CUDA-core
    shape is kept unless the tensor-core kernel is clearly faster."""
    from flurrypp_b200.decks import vortex_case

    s = fb.Solver(vortex_case(str(tmp_path / "v.deck"), 128, 3, 0.5), precision=fb.FR_PREC_MIXED)
    ms = s.get_array("tile_ms")
    v = s.info().tile_variant
    assert len(ms) == 4 and ms[3] > 0 and (ms[:3] > 0).sum() >= 2
    cuda_core = [m for m in ms[:3] if m > 0]
    if v == 3:
        assert ms[3] < 0.9 * min(cuda_core)
    else:
        assert ms[v] == min(cuda_core)


@pytest.mark.parametrize("case", ["vortex2d_p3_8", "tgv3d_p3_4_perturbed", "jameson5_2d_p2", "euler_fwd2d_p1"])
def test_mixed_graph_equals_update_loop(case):
    a, meta = load_golden(case)
    s1 = mixed_case(meta)
    s1.set_state(a["U_init"])
    s1.run(6)
    s2 = mixed_case(meta)
    s2.set_state(a["U_init"])
    for _ in range(6):
        s2.update()
    assert np.array_equal(s1.get_state(), s2.get_state())


def test_mixed_state_round_trip():
    a, meta = load_golden("tgv3d_p2_4")
    s = mixed_case(meta)
    s.set_state(a["U_init"])
    U = s.get_state()
    assert np.all(np.abs(U - a["U_init"]) <= 2.0 ** -46 * np.abs(a["U_init"]))


def test_mixed_batch_equals_alone(tmp_path):
    """Cases of uneven size and order in one batch give what each gives
    alone (alone, an element count that is not a multiple of 4 runs the
    non-TMA kernel, whose FMA contraction may differ: FP32 round-off)."""
    from test_batch_gpu import make_cases
    from flurrypp_b200.decks import vortex_case

    def build(sp, i):
        n, P, eps, xc, yc, M = sp
        s = fb.Solver(vortex_case(str(tmp_path / f"m{i}.deck"), n, P, M), precision=fb.FR_PREC_MIXED)
        s.initialize_solution(fb.IC_VORTEX, (eps, xc, yc, M))
        s.set_dt(s.calc_dt())
        return s

    specs = make_cases(tmp_path)
    alone = []
    for i, sp in enumerate(specs):
        s = build(sp, i)
        s.run(12)
        alone.append((s.get_state(), s.residual_norm(2)))
    members = [build(sp, i) for i, sp in enumerate(specs)]
    b = fb.Batch(members)
    b.run(12)
    norms = b.residual_norms(2)
    b.gather()
    for i, s in enumerate(members):
        U = s.get_state()
        Ua, ra = alone[i]
        assert np.max(np.abs(U - Ua)) <= 1e-6 * np.max(np.abs(Ua)), i
        assert np.allclose(norms[i], ra, rtol=1e-4, atol=0)


TC_CASES = ["vortex2d_p3_8", "channel2d_p2", "roe2d_p2", "hu2d_p3", "cplus2d_p2", "lobatto_sd2d_p4",
            "jameson5_2d_p2", "euler_fwd2d_p1", "localdt_jameson2d_p3", "ic1_2d_p3",
            "p1_3d"]  # 3-D: order 1 (24 elements and 120 of the 128 MMA rows per CTA)


def tensor_case(meta, **kw):
    s = mixed_case(meta, tile_variant=3, **kw)
    if s.info().tile_variant != 3:
        pytest.skip("element count not a multiple of 4 or order outside 1..4: no TMA tiles")
    return s


@pytest.mark.parametrize("case", TC_CASES)
def test_tensor_core_variant_residual_and_steps(case):
    """The tcgen05 (3xTF32) element stage: residual within FP32 round-off of
    the reference's and the state after N steps within the L2 bound."""
    a, meta = load_golden(case)
    s = tensor_case(meta, debug_arrays=1)
    s.set_state(a["U_init"])
    s.calc_residual(0)
    d = s.get_residual(0)
    scale = max(np.abs(a["divF_0"]).max(), np.abs(a["F_spts"]).max())
    assert np.abs(d - a["divF_0"]).max() / scale < RESID_TOL
    s2 = tensor_case(meta)
    s2.set_state(a["U_init"])
    s2.run(meta["steps"])
    assert rel_l2(s2.get_state(), a["U_final"]) < L2_TOL


@pytest.mark.parametrize("case", ["vortex2d_p3_8", "p1_3d"])
def test_tensor_core_variant_near_cuda_core_variant(case):
    a, meta = load_golden(case)
    out = []
    for v in (0, 3):
        s = mixed_case(meta, tile_variant=v)
        s.set_state(a["U_init"])
        s.run(20)
        out.append(s.get_state())
    assert rel_l2(out[1], out[0]) < 1e-7


@pytest.mark.parametrize("case", ["pmg_vortex2d_p3_8", "chbump_p2_pmg"])
def test_mixed_pmg_graph_equals_cycle_loop(case):
    """Precision-form P-multigrid: the graph-replayed step (update + V-cycle)
    equals update() followed by pmg_cycle() bit for bit."""
    a, meta = load_golden(case)
    s1 = mixed_case(meta)
    s1.set_state(a["U_init"])
    s1.run(4)
    s2 = mixed_case(meta)
    s2.set_state(a["U_init"])
    for _ in range(4):
        s2.update()
        s2.pmg_cycle()
    assert np.array_equal(s1.get_state(), s2.get_state())
