"""Batched form: many independent cases of uneven size and order advanced
together must give, case by case, what each gives alone."""
import numpy as np
import pytest

import flurrypp_b200 as fb
from flurrypp_b200.decks import vortex_case

pytestmark = pytest.mark.gpu


def make_cases(tmp_path, n_cases=7, seed=3):
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_cases):
        n = int(rng.integers(4, 13))
        P = int(rng.integers(2, 6))
        eps = float(rng.uniform(1, 5))
        xc, yc = rng.uniform(-2, 2, 2)
        M = float(rng.uniform(0.2, 0.6))
        specs.append((n, P, eps, float(xc), float(yc), M))
    return specs


def build(tmp_path, spec, i):
    n, P, eps, xc, yc, M = spec
    deck = vortex_case(str(tmp_path / f"c{i}.deck"), n, P, M)
    s = fb.Solver(deck)
    s.initialize_solution(fb.IC_VORTEX, (eps, xc, yc, M))
    s.set_dt(s.calc_dt())
    return s


def test_batch_equals_alone(tmp_path):
    specs = make_cases(tmp_path)
    steps = 12
    alone = []
    for i, sp in enumerate(specs):
        s = build(tmp_path, sp, i)
        s.run(steps)
        alone.append((s.get_state(), s.residual_norm(2)))
    members = [build(tmp_path, sp, i) for i, sp in enumerate(specs)]
    b = fb.Batch(members)
    assert b.info()["groups"] == len({sp[1] for sp in specs})
    b.run(steps)
    norms = b.residual_norms(2)
    b.gather()
    for i, s in enumerate(members):
        U = s.get_state()
        Ua, ra = alone[i]
        assert np.max(np.abs(U - Ua)) <= 1e-14 * np.max(np.abs(Ua)), i
        assert np.allclose(norms[i], ra, rtol=1e-12, atol=0)


def test_batch_rejects_unsupported(tmp_path):
    s = build(tmp_path, (6, 3, 2.0, 0.0, 0.0, 0.4), 0)
    h = fb.Solver(vortex_case(str(tmp_path / "h.deck"), 6, 3, 0.4), device=-1)
    with pytest.raises(fb.FrError) as ei:
        fb.Batch([s, h])
    assert ei.value.code == fb.FR_ERR_STATE


@pytest.mark.parametrize("prec", [fb.FR_PREC_FP64, fb.FR_PREC_MIXED])
def test_many_order_form_equals_alone(tmp_path, prec):
    """The many-order form (one face launch and one persistent element launch
    per RK stage for every order, blocks taken from a device work counter)
    gives, case by case, what each case gives alone; the creation-time choice
    between the forms is reported with both timings."""
    specs = make_cases(tmp_path, n_cases=9, seed=11)
    assert len({sp[1] for sp in specs}) >= 3
    steps = 10

    def built(i, sp):
        s = build(tmp_path, sp, i)
        if prec == fb.FR_PREC_FP64:
            return s
        m = fb.Solver(str(tmp_path / f"c{i}.deck"), precision=prec)
        m.initialize_solution(fb.IC_VORTEX, sp[2:])
        m.set_dt(s.calc_dt())
        return m

    alone = []
    for i, sp in enumerate(specs):
        s = built(i, sp)
        s.run(steps)
        alone.append(s.get_state())
    members = [built(i, sp) for i, sp in enumerate(specs)]
    b = fb.Batch(members)
    f = b.form()
    assert f["ms_groups"] > 0 and f["ms_many_order"] > 0
    b.set_form(fb.FR_BATCH_MANY_ORDER)
    b.run(steps)
    b.gather()
    tol = 1e-13 if prec == fb.FR_PREC_FP64 else 1e-5  # FP32: the two element kernels round alike only to FP32
    for i, s in enumerate(members):
        U, Ua = s.get_state(), alone[i]
        assert np.max(np.abs(U - Ua)) <= tol * np.max(np.abs(Ua)), i
