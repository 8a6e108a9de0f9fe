"""Serving form: continuous batching of steady channel solves.  Each result is
the same alone and in the mix; admission honours the memory budget."""
import os
import time

import numpy as np
import pytest

import flurrypp_b200 as fb
from flurrypp_b200.decks import channel_case
from flurrypp_b200.meshgen import channel_bump, write_gmsh

pytestmark = pytest.mark.gpu

SPECS = [(12, 2, 0.3, 0.06), (16, 3, 0.25, 0.04), (20, 1, 0.4, 0.08), (14, 2, 0.35, 0.05)]


def make_case(tmp_path, i, nx, P, M, h):
    msh = str(tmp_path / f"bump{i}.msh")
    write_gmsh(msh, channel_bump(nx, nx // 3, h))
    return channel_case(str(tmp_path / f"bump{i}.deck"), msh, P, M)


def shape_of(deck):
    s = fb.Solver(deck, device=-1)
    return s.shape


def test_results_same_alone_and_in_the_mix(tmp_path):
    decks = [make_case(tmp_path, i, *sp) for i, sp in enumerate(SPECS)]
    tol, max_steps = 1e-3, 120
    alone = fb.Server(budget_bytes=8 << 30, max_inflight=1, check_every=10)
    rid = alone.submit(decks[0], tol=tol, max_steps=max_steps)
    alone.wait(rid, 300)
    ua, pa = alone.result(rid, shape_of(decks[0])), alone.poll(rid)
    alone.close()
    mix = fb.Server(budget_bytes=8 << 30, max_inflight=4, check_every=10)
    ids = [mix.submit(d, tol=tol, max_steps=max_steps) for d in decks]
    for r in ids:
        mix.wait(r, 300)
    um, pm = mix.result(ids[0], shape_of(decks[0])), mix.poll(ids[0])
    assert pa["steps"] == pm["steps"]
    assert np.array_equal(ua, um)
    # the served result equals the same number of driver steps on a plain case
    s = fb.Solver(decks[0])
    s.initialize_solution(fb.IC_DECK)
    s.run(pa["steps"])
    assert np.array_equal(s.get_state(), ua)
    for r in ids:
        p = mix.poll(r)
        assert p["status"] == 2 and p["latency_s"] > 0
    mix.close()


def test_admission_respects_budget(tmp_path):
    deck = make_case(tmp_path, 0, *SPECS[0])
    # the device bytes one such case occupies, seen while it runs
    probe = fb.Server(budget_bytes=8 << 30, max_inflight=1, check_every=1)
    r = probe.submit(deck, tol=1e-30, max_steps=100000)
    one = 0
    t0 = time.time()
    while one == 0 and time.time() - t0 < 60:
        one = probe.stats()["inflight_bytes"]
    probe.cancel(r)
    probe.close()
    assert one > 0
    # a budget that holds one case at a time: the others wait in the queue
    srv = fb.Server(budget_bytes=int(1.5 * one), max_inflight=8, check_every=10)
    ids = [srv.submit(deck, tol=1e-2, max_steps=30) for _ in range(3)]
    peak = 0
    t0 = time.time()
    while time.time() - t0 < 120:
        st = srv.stats()
        peak = max(peak, st["inflight"])
        if all(srv.poll(r)["status"] >= 2 for r in ids):
            break
        time.sleep(0.001)
    assert peak == 1
    assert all(srv.poll(r)["status"] == 2 for r in ids)
    srv.close()


def test_over_budget_request_fails_cleanly(tmp_path):
    deck = make_case(tmp_path, 0, *SPECS[1])
    srv = fb.Server(budget_bytes=1 << 10, max_inflight=2, check_every=10)
    r = srv.submit(deck, tol=1e-2, max_steps=10)
    with pytest.raises(fb.FrError) as ei:
        srv.wait(r, 60)
    assert ei.value.code == fb.FR_ERR_BUDGET
    srv.close()


def test_precision_form_served(tmp_path):
    """The precision form (FP32 stages, P-multigrid included) through the
    server: the same alone and in the mix, equal to the same number of
    driver steps of a precision-form case, and within the precision form's
    L2 bound of the FP64 served result."""
    decks = [make_case(tmp_path, i, *sp) for i, sp in enumerate(SPECS)]
    tol, max_steps = 1e-3, 80
    alone = fb.Server(budget_bytes=8 << 30, max_inflight=1, check_every=10, precision=fb.FR_PREC_MIXED)
    rid = alone.submit(decks[1], tol=tol, max_steps=max_steps)
    alone.wait(rid, 300)
    ua, pa = alone.result(rid, shape_of(decks[1])), alone.poll(rid)
    alone.close()
    mix = fb.Server(budget_bytes=8 << 30, max_inflight=4, check_every=10, precision=fb.FR_PREC_MIXED)
    ids = [mix.submit(d, tol=tol, max_steps=max_steps) for d in decks]
    for r in ids:
        mix.wait(r, 300)
    um, pm = mix.result(ids[1], shape_of(decks[1])), mix.poll(ids[1])
    mix.close()
    assert pa["steps"] == pm["steps"]
    assert np.array_equal(ua, um)
    s = fb.Solver(decks[1], precision=fb.FR_PREC_MIXED)
    s.initialize_solution(fb.IC_DECK)
    s.run(pa["steps"])
    assert np.array_equal(s.get_state(), ua)
    d = fb.Solver(decks[1])
    d.initialize_solution(fb.IC_DECK)
    d.run(pa["steps"])
    ud = d.get_state()
    assert np.linalg.norm(ua - ud) / np.linalg.norm(ud) < 1e-6


def test_refining_precision_form_reaches_the_tight_drop(tmp_path):
    """FR_PREC_MIXED_REFINE served to a 1e-8 residual drop: the request runs
    in the precision form until its FP32 residual stops falling, then goes on
    in FP64; it reaches the drop, as the FP64 form does, and the FP64 steady
    state (L2 within 1e-6).  The all-FP32 form stays at its floor."""
    deck = make_case(tmp_path, 0, *SPECS[0])
    res = {}
    for prec in (fb.FR_PREC_FP64, fb.FR_PREC_MIXED_REFINE, fb.FR_PREC_MIXED):
        srv = fb.Server(budget_bytes=8 << 30, max_inflight=1, check_every=10, precision=prec)
        rid = srv.submit(deck, tol=1e-8, max_steps=20000)
        srv.wait(rid, 600)
        res[prec] = (srv.result(rid, shape_of(deck)), srv.poll(rid), srv.poll_form(rid))
        srv.close()
    (u64, p64, _), (umx, pmx, fmx), (_, p32, f32) = (res[fb.FR_PREC_FP64], res[fb.FR_PREC_MIXED_REFINE],
                                                      res[fb.FR_PREC_MIXED])
    assert p64["status"] == 2 and p64["res_ratio"] <= 1e-8
    assert pmx["status"] == 2 and pmx["res_ratio"] <= 1e-8, pmx
    assert fmx["precision"] == fb.FR_PREC_FP64 and 0 < fmx["steps_fp32"] < pmx["steps"], fmx
    assert np.linalg.norm(umx - u64) / np.linalg.norm(u64) < 1e-6
    assert f32["precision"] == fb.FR_PREC_MIXED and p32["res_ratio"] > 1e-8
