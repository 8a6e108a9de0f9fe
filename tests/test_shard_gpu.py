"""One case split into parts on one device (fr_shard_*): the parts exchange
the traces of the faces the partition cuts at every stage, as the
reference's MPI ranks do (mpiFace::communicate / getRightState,
src/mpiFace.cpp:122-175), and take the minimum time step over the parts
(src/solver.cpp:462-465).

The split case must give the unsplit case's residual and states: each side of
a cut face forms the flux with its own normal, so the two differ by round-off
only (bound 1e-14 relative to the flux scale per residual and to the state
after 10 steps), and both match the reference's fixtures as the unsplit case
does.
"""
import numpy as np
import pytest

import flurrypp_b200 as fb
from conftest import deck_path, load_golden, perturb_opts, rel_err

pytestmark = pytest.mark.gpu

SPLIT_TOL = 1e-14


def cases(meta, nparts):
    opts = perturb_opts(meta)
    one = fb.Solver(deck_path(meta), **opts)
    sh = fb.Shard(deck_path(meta), nparts, **opts)
    if "--cfl-dt" in meta["harness_args"]:
        one.set_dt(meta["dt"])
        sh.set_dt(meta["dt"])
    return one, sh


@pytest.mark.parametrize("nparts", [2, 3, 4])
@pytest.mark.parametrize("case", ["tgv3d_p3_4", "tgv3d_p3_4_perturbed", "chbump_p3", "vortex2d_p3_8", "roe2d_p2"])
def test_split_case_equals_unsplit(case, nparts):
    a, meta = load_golden(case)
    one, sh = cases(meta, nparts)
    inf = sh.info()
    assert inf["nparts"] == nparts and sum(inf["owned"]) == one.nEles
    assert all(c > 0 for c in inf["cut_points"])
    one.set_state(a["U_init"])
    sh.set_state(a["U_init"])
    assert np.array_equal(sh.get_state(), a["U_init"])
    one.calc_residual(0)
    sh.calc_residual(0)
    fscale = float(np.max(np.abs(a["F_spts"])))
    d1, ds = one.get_residual(0), sh.get_residual(0)
    assert rel_err(ds, d1, fscale) < SPLIT_TOL
    assert rel_err(ds, a["divF_0"], fscale) < 1e-12  # and the reference's
    steps = 10
    one.run(steps)
    sh.run(steps)
    assert rel_err(sh.get_state(), one.get_state()) < SPLIT_TOL
    t_one, dt_one = one.info().time, one.info().dt
    t_sh, dt_sh = sh.time()
    assert abs(t_sh - t_one) <= 1e-14 * abs(t_one) and abs(dt_sh - dt_one) <= 1e-14 * dt_one


@pytest.mark.parametrize("case", ["tgv3d_p3_4", "chbump_p3"])
def test_split_case_matches_reference_steps(case):
    """The fixture's N steps through the split case: the reference's state."""
    a, meta = load_golden(case)
    _, sh = cases(meta, 4)
    sh.set_state(a["U_init"])
    sh.run(meta["steps"])
    assert rel_err(sh.get_state(), a["U_final"]) < 1e-10


def test_split_refuses_what_it_does_not_cover():
    a, meta = load_golden("ns_tgv3d_p3_3")
    with pytest.raises(fb.FrError) as ei:
        fb.Shard(deck_path(meta), 2)
    assert ei.value.code == fb.FR_ERR_UNSUPPORTED
    a, meta = load_golden("vortex2d_p3_8")
    with pytest.raises(fb.FrError):
        fb.Shard(deck_path(meta), 2, precision=fb.FR_PREC_MIXED)


@pytest.mark.parametrize("case", ["chbump_p3", "tgv3d_p3_4"])
def test_rank_part_through_nccl_on_one_rank(case):
    """The rank form of a part (fr_part_create, one process and GPU per rank,
    traces by NCCL send/receive, dt by an NCCL minimum) on a one-rank
    communicator: the part is the whole case, the dt reduction goes through
    NCCL, and the result is the unsplit case's.  (More ranks need more GPUs
    than one call has; the in-process shard tests the cut exchange itself.)"""
    a, meta = load_golden(case)
    comm, _ = fb.nccl_comm(1, 0, 0)
    opts = perturb_opts(meta)
    p = fb.Solver(deck_path(meta), part=(1, 0, comm), **opts)
    one = fb.Solver(deck_path(meta), **opts)
    if "--cfl-dt" in meta["harness_args"]:
        p.set_dt(meta["dt"])
        one.set_dt(meta["dt"])
    p.set_state(a["U_init"])
    one.set_state(a["U_init"])
    p.run(10)
    one.run(10)
    assert fb.lib.fr_part_nccl_ok(p._c) == fb.FR_OK
    assert rel_err(p.get_state(), one.get_state()) < SPLIT_TOL
    assert abs(p.info().dt - one.info().dt) <= 1e-15 * one.info().dt
    del p
    fb.lib.fr_nccl_comm_destroy(comm)
