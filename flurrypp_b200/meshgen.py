"""Mesh generators for the path's workloads, with a Gmsh 2.2 ASCII writer.

`channel_bump` builds the structured channel-over-bump mesh of the steady
solve workload: x uniform on [-1.5, 1.5], lower wall y = h exp(-25 x^2),
upper wall y = 0.8, each column's points spaced linearly between the walls.
The same mesh goes to the library either as arrays (`fr_create_with_mesh`) or
as a Gmsh file named by a deck (`meshType 0`, read like the reference's
geo::readGmsh, src/geo.cpp:1021-1475).
"""
from __future__ import annotations

import numpy as np

BC_CODES = {"periodic": 0, "char": 1, "sup_in": 2, "sup_out": 3, "sub_in": 4, "sub_out": 5,
            "slip_wall": 8, "isothermal_noslip": 9, "adiabatic_noslip": 10, "symmetry": 12}


def channel_bump(nx: int, ny: int, h: float, x0: float = -1.5, x1: float = 1.5, ytop: float = 0.8):
    """Structured quads; returns a dict with xv [nVerts,2], c2v [nEles,4]
    (counter-clockwise), and boundary edges named bottom/top/inlet/outlet."""
    xs = np.linspace(x0, x1, nx + 1)
    yb = h * np.exp(-25.0 * xs * xs)
    xv = np.empty(((nx + 1) * (ny + 1), 2))
    vid = lambda i, j: j * (nx + 1) + i
    for j in range(ny + 1):
        for i in range(nx + 1):
            xv[vid(i, j)] = (xs[i], yb[i] + (ytop - yb[i]) * j / ny)
    c2v = np.array([[vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)]
                    for j in range(ny) for i in range(nx)], dtype=np.int32)
    edges = {
        "bottom": [(vid(i, 0), vid(i + 1, 0)) for i in range(nx)],
        "top": [(vid(i + 1, ny), vid(i, ny)) for i in range(nx)],
        "inlet": [(vid(0, j + 1), vid(0, j)) for j in range(ny)],
        "outlet": [(vid(nx, j), vid(nx, j + 1)) for j in range(ny)],
    }
    return {"xv": xv, "c2v": c2v, "edges": edges}


def mesh_arrays(m: dict, bcs: dict):
    """Arrays for fr_create_with_mesh: boundary faces listed by vertices."""
    verts, codes = [], []
    for name, lst in m["edges"].items():
        for a, b in lst:
            verts.append([a, b, -1, -1])
            codes.append(BC_CODES[bcs[name]])
    return {"xv": m["xv"], "c2v": m["c2v"], "bnd_face_verts": np.array(verts, dtype=np.int32),
            "bnd_face_bc": np.array(codes, dtype=np.int32)}


def write_gmsh(path: str, m: dict) -> None:
    """Gmsh 2.2 ASCII: physical lines bottom/top/inlet/outlet, surface fluid."""
    names = list(m["edges"].keys())
    xv, c2v = m["xv"], m["c2v"]
    lines = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$PhysicalNames", str(len(names) + 1)]
    for k, n in enumerate(names):
        lines.append(f'1 {k + 1} "{n}"')
    fluid = len(names) + 1
    lines.append(f'2 {fluid} "fluid"')
    lines += ["$EndPhysicalNames", "$Nodes", str(len(xv))]
    for i, (x, y) in enumerate(xv):
        lines.append(f"{i + 1} {float(x):.17g} {float(y):.17g} 0")
    lines += ["$EndNodes", "$Elements"]
    elems = []
    for k, n in enumerate(names):
        for a, b in m["edges"][n]:
            elems.append(f"1 2 {k + 1} {k + 1} {a + 1} {b + 1}")
    for q in c2v:
        elems.append(f"3 2 {fluid} {fluid} " + " ".join(str(v + 1) for v in q))
    lines.append(str(len(elems)))
    lines += [f"{i + 1} {e}" for i, e in enumerate(elems)]
    lines.append("$EndElements")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
