"""The reference's solution files in the fixtures (no GPU): the layout that
the product's restart reader relies on.  The values at the solution points
of each element's (P+3)^d plot grid are the reference's state after the
fixture's steps, to the 16 digits printed (src/output.cpp:137-512 writes
them, src/ele.cpp:1497-1921 reads them back)."""
import gzip

import numpy as np
import pytest

from conftest import golden_cases, load_golden, rel_err
from solution_files import read_csv, read_vtu

CASES = golden_cases(require=("ref_vtu_gz", "U_final"))


def spts_of_plot_grid(nd, order):
    n, np3 = order + 1, order + 3
    idx = []
    for s in range(n ** nd):
        i, j, k = s % n, (s // n) % n, s // (n * n)
        idx.append((i + 1) + np3 * (j + 1) + (np3 * np3 * (k + 1) if nd == 3 else 0))
    return np.array(idx)


@pytest.mark.parametrize("case", CASES)
def test_reference_vtu_holds_the_state_at_its_solution_points(case):
    a, meta = load_golden(case)
    v = read_vtu(gzip.decompress(a["ref_vtu_gz"].tobytes()).decode())
    nd, order, E, gam = meta["nDims"], meta["order"], meta["nEles"], 1.4
    assert len(v["pieces"]) == E and v["iter"] == meta["steps"]
    at = spts_of_plot_grid(nd, order)
    U = np.empty_like(a["U_final"])
    for e, p in enumerate(v["pieces"]):
        rho, vel, pr = p["Density"][at], p["Velocity"].reshape(-1, 3)[at, :nd], p["Pressure"][at]
        U[:, e, 0] = rho
        U[:, e, 1:nd + 1] = rho[:, None] * vel
        U[:, e, nd + 1] = pr / (gam - 1) + 0.5 * rho * (vel ** 2).sum(axis=1)
    assert rel_err(U, a["U_final"]) < 5e-15
    assert float(v["time"]) == pytest.approx(a["time_dt"][0], rel=1e-15)


@pytest.mark.parametrize("case", golden_cases(require=("ref_csv_gz",)))
def test_reference_csv_rows(case):
    a, meta = load_golden(case)
    head, rows = read_csv(gzip.decompress(a["ref_csv_gz"].tobytes()).decode())
    assert head == "x,y,z,rho,u,v,p"
    assert rows.shape[0] == meta["nEles"] * (meta["nSpts"] + meta["nFpts"])
