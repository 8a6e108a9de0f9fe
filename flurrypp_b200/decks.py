"""Reference-format input decks for the path's workloads.

`deck_text(**opts)` writes "key value" lines with the reference's option names
(src/input.cpp:257-523); `vortex_case` and `channel_case` give the decks of the
batched 2-D vortex workload and of the channel-over-bump steady solve.
"""
from __future__ import annotations

import math
import os

BASE = {
    "equation": 1, "viscous": 0, "motion": 0, "nDims": 2, "order": 3, "riemannType": 0,
    "timeType": 4, "dtType": 0, "dt": 0.01, "CFL": 0.5, "iterMax": 1000000, "icType": 0, "restart": 0,
    "spts_type_quad": "Legendre", "vcjhSchemeQuad": 0, "gamma": 1.4,
    "rhoBound": 1, "uBound": 0.2, "vBound": 0, "wBound": 0, "pBound": 0.7142857143,
    "plotFreq": 100000000, "monitorResFreq": 100000000,
}


def deck_text(**opts) -> str:
    d = dict(BASE)
    extra = opts.pop("mesh_bound", [])
    d.update(opts)
    lines = [f"{k} {v}" for k, v in d.items()]
    lines += [f"mesh_bound {a} {b}" for a, b in extra]
    return "\n".join(lines) + "\n"


def write_deck(path: str, **opts) -> str:
    with open(path, "w") as f:
        f.write(deck_text(**opts))
    return path


def vortex_case(path: str, n: int, order: int, mach: float) -> str:
    """Periodic [-5,5]^2, n x n straight quads, free stream at `mach` (p = 1)."""
    return write_deck(path, order=order, meshType=1, nx=n, ny=n, xmin=-5, xmax=5, ymin=-5, ymax=5,
                      uBound=mach * math.sqrt(1.4), pBound=1)


def channel_case(path: str, mesh_file: str, order: int, mach: float, pmg: bool = True) -> str:
    """Channel over a bump: slip walls, characteristic inlet/outlet, rho = 1,
    p = 1/gamma, u = Mach; local-CFL RK4 with P-multigrid to lowOrder 0."""
    opts = dict(order=order, meshType=0, meshFileName=os.path.basename(mesh_file), dtType=2, CFL=0.5,
                maxTime=1e9, uBound=mach, pBound=0.7142857143, resType=2,
                mesh_bound=[("bottom", "slip_wall"), ("top", "slip_wall"), ("inlet", "char"),
                            ("outlet", "char"), ("fluid", "fluid")])
    if pmg:
        opts.update(PMG=1, lowOrder=0, smoothSteps=2)
    return write_deck(path, **opts)
