"""Solution files through the C ABI: the reference's ParaView (.vtu) and CSV
writers (src/output.cpp:43-512) and its restart reader
(src/solver.cpp:1789-1890, src/ele.cpp:1497-1921).

Checked against files the reference itself wrote after each fixture's N
steps: reading one restores the reference's state to the 16 printed digits;
writing the same state reproduces the reference's file (same tags and
layout, values to round-off); the reference reads the product's file back;
a P2 file restarts a P3 case as the reference interpolates it.  A checkpoint
holds the state of its own step while stepping goes on and changes nothing
in the run.
"""
import gzip
import os
import subprocess

import numpy as np
import pytest

import flurrypp_b200 as fb
from conftest import ROOT, deck_path, load_golden, perturb_opts, rel_err
from solution_files import read_csv, read_vtu

pytestmark = pytest.mark.gpu

OUTPUT_CASES = ["vortex2d_p3_8", "tgv3d_p2_4", "curved2d_q2_p3", "motion2_2d_p2_cfl"]
TEXT_TOL = 5e-15   # 16 printed digits, then primitive -> conservative rounding
FILE_TOL = 1e-13   # plot-point extrapolation: summation order differs from the reference's BLAS
HARNESS = os.path.join(ROOT, "oracle", "_ref", "fr_ref_harness")


def case_solver(meta, deck=None, **kw):
    s = fb.Solver(deck or deck_path(meta), **perturb_opts(meta), **kw)
    if "--cfl-dt" in meta["harness_args"]:
        s.set_dt(meta["dt"])
    return s


def ref_file(a, key, path):
    path.write_bytes(gzip.decompress(a[key].tobytes()))
    return str(path)


def deck_with(meta, tmp_path, head: str) -> str:
    """The fixture's deck with `head` lines first (first occurrence wins)."""
    d = tmp_path / "case.deck"
    d.write_text(head + open(deck_path(meta)).read())
    src = os.path.dirname(deck_path(meta))
    for line in open(deck_path(meta)):
        t = line.split()
        if len(t) > 1 and t[0] == "meshFileName":
            (tmp_path / t[1]).write_bytes(open(os.path.join(src, t[1]), "rb").read())
    return str(d)


def compare_vtu(mine: dict, ref: dict):
    assert float(mine["time"]) == pytest.approx(float(ref["time"]), rel=1e-15, abs=0)
    assert mine["iter"] == ref["iter"]
    no_time = lambda tags: [t for t in tags if "TIME" not in t]
    assert no_time(mine["tags"]) == no_time(ref["tags"])
    assert len(mine["pieces"]) == len(ref["pieces"])
    for name in ref["pieces"][0]:
        a = np.concatenate([p[name] for p in mine["pieces"]])
        b = np.concatenate([p[name] for p in ref["pieces"]])
        if b.dtype.kind == "i":
            assert np.array_equal(a, b), name
        else:
            assert rel_err(a, b) < FILE_TOL, name


@pytest.mark.parametrize("case", OUTPUT_CASES)
def test_restart_reads_the_reference_file(case, tmp_path):
    a, meta = load_golden(case)
    ref = read_vtu(gzip.decompress(a["ref_vtu_gz"].tobytes()).decode())
    s = case_solver(meta)
    s.read_restart(ref_file(a, "ref_vtu_gz", tmp_path / "ref.vtu"))
    assert rel_err(s.get_state(), a["U_final"]) < TEXT_TOL
    inf = s.info()
    assert inf.iter == meta["steps"] == ref["iter"]
    assert inf.time == float(ref["time"])


@pytest.mark.parametrize("case", OUTPUT_CASES)
def test_paraview_file_matches_the_reference(case, tmp_path):
    a, meta = load_golden(case)
    s = case_solver(meta)
    s.read_restart(ref_file(a, "ref_vtu_gz", tmp_path / "ref.vtu"))
    s.write_data(str(tmp_path / "mine.vtu"))
    compare_vtu(read_vtu((tmp_path / "mine.vtu").read_text()),
                read_vtu(gzip.decompress(a["ref_vtu_gz"].tobytes()).decode()))


@pytest.mark.parametrize("case", ["vortex2d_p3_8", "tgv3d_p2_4"])
def test_csv_file_matches_the_reference(case, tmp_path):
    a, meta = load_golden(case)
    s = case_solver(meta, deck=deck_with(meta, tmp_path, "plotType 0\n"))
    s.read_restart(ref_file(a, "ref_vtu_gz", tmp_path / "ref.vtu"))
    s.write_data(str(tmp_path / "mine.csv"))
    h1, mine = read_csv((tmp_path / "mine.csv").read_text())
    h2, ref = read_csv(gzip.decompress(a["ref_csv_gz"].tobytes()).decode())
    assert h1 == h2 and mine.shape == ref.shape
    assert np.max(np.abs(mine - ref)) <= FILE_TOL * max(1.0, np.max(np.abs(ref)))


def test_default_file_name_and_deck_restart(tmp_path):
    """dataFileName_<iter>.vtu by default; a deck with restart 1 starts from
    dataFileName_<restartIter>.vtu with the iteration count restartIter."""
    a, meta = load_golden("vortex2d_p3_8")
    prefix = str(tmp_path / "run")
    s = case_solver(meta, deck=deck_with(meta, tmp_path, f"dataFileName {prefix}\n"))
    s.set_state(a["U_init"])
    s.run(6)
    s.write_data()
    assert os.path.exists(prefix + "_000000006.vtu")
    r = case_solver(meta, deck=deck_with(meta, tmp_path, f"restart 1\nrestartIter 6\ndataFileName {prefix}\n"))
    r.initialize_solution()
    assert r.info().iter == 6
    assert rel_err(r.get_state(), s.get_state()) < TEXT_TOL
    r.run(3)
    s.run(3)
    assert rel_err(r.get_state(), s.get_state()) < 1e-12


def test_checkpoint_holds_its_step_and_changes_nothing(tmp_path):
    a, meta = load_golden("tgv3d_p3_4")
    s1 = case_solver(meta)
    s1.set_state(a["U_init"])
    s1.run(3)
    U3 = s1.get_state()
    s1.checkpoint()
    s1.run(4)  # stepping goes on while the copy is in flight
    s1.write_data(str(tmp_path / "cp.vtu"))
    s2 = case_solver(meta)
    s2.set_state(a["U_init"])
    s2.run(7)
    assert np.array_equal(s1.get_state(), s2.get_state())
    r = case_solver(meta)
    r.read_restart(str(tmp_path / "cp.vtu"))
    assert r.info().iter == 3
    assert rel_err(r.get_state(), U3) < TEXT_TOL


def test_precision_form_checkpoint(tmp_path):
    a, meta = load_golden("vortex2d_p3_8")
    s = case_solver(meta, precision=fb.FR_PREC_MIXED)
    s.set_state(a["U_init"])
    s.run(5)
    s.write_data(str(tmp_path / "m.vtu"))
    r = case_solver(meta)
    r.read_restart(str(tmp_path / "m.vtu"))
    assert rel_err(r.get_state(), s.get_state()) < TEXT_TOL


def test_restart_across_orders_matches_the_reference(tmp_path):
    """A P2 file into a P3 case: Lagrange interpolation in the P2 points."""
    a, meta = load_golden("restart_p2_to_p3")
    s = case_solver(meta)
    s.read_restart(ref_file(a, "ref_vtu_gz", tmp_path / "p2.vtu"))
    assert rel_err(s.get_state(), a["ref_U_restart"]) < 1e-14


def test_moving_mesh_pmg_restart_matches_the_reference(tmp_path):
    """A moving-mesh P-multigrid case restarted from the reference's file
    after 4 steps and run 4 more: the finest level takes the file's time and
    mesh position, the coarse levels keep their own time from zero (as the
    reference's levels, set up before the file is read); the reference's
    state and time after the 4 steps."""
    a, meta = load_golden("restart_pmg_motion2d_p2")
    s = case_solver(meta)
    s.read_restart(ref_file(a, "ref_vtu_gz", tmp_path / "w.vtu"))
    assert rel_err(s.get_state(), a["ref_U_restart"]) < 1e-14
    for _ in range(meta["steps"]):
        s.update()
        s.pmg_cycle()
    assert rel_err(s.get_state(), a["U_restarted_final"]) < 1e-10
    assert abs(s.info().time - a["time_dt_restarted"][0]) <= 1e-12


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="reference build not present")
@pytest.mark.parametrize("case", ["vortex2d_p3_8", "curved2d_q2_p3"])
def test_reference_reads_the_product_file(case, tmp_path):
    """The reference's restart reader (built from its sources) on a file the
    product wrote: it restores the product's state."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_golden import read_dump

    a, meta = load_golden(case)
    s = case_solver(meta)
    s.set_state(a["U_init"])
    s.run(7)
    s.write_data(str(tmp_path / "mine_000000007.vtu"))
    deck = deck_with(meta, tmp_path, f"restart 1\nrestartIter 7\ndataFileName {tmp_path / 'mine'}\n")
    out = tmp_path / "dump"
    out.mkdir()
    subprocess.run([HARNESS, deck, str(out)], check=True, stdout=subprocess.DEVNULL, cwd=str(tmp_path),
                   timeout=300)
    arrays, _ = read_dump(str(out))
    assert rel_err(arrays["U_init"].ravel(), s.get_state().ravel()) < TEXT_TOL
