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


# --- curved (high-order) elements -------------------------------------------

def _quad_rings(lo: int, hi: int) -> list[tuple[int, int]]:
    """(a, b) 1-D indices of a Lagrange quad's nodes over [lo, hi], numbered
    the Gmsh way: corners, points inside each edge, then the inner quad."""
    out, n = [], hi - lo + 1
    for level in range(n // 2):
        a, b, m = lo + level, hi - level, n - 2 * (level + 1)
        out += [(a, a), (b, a), (b, b), (a, b)]
        out += [(a + 1 + k, a) for k in range(m)]
        out += [(b, a + 1 + k) for k in range(m)]
        out += [(b - 1 - k, b) for k in range(m)]
        out += [(a, b - 1 - k) for k in range(m)]
    if n % 2:
        out.append((lo + n // 2, lo + n // 2))
    return out


def lagrange_node_order(nd: int, q: int) -> list[tuple[int, ...]]:
    """1-D index tuples (along xi, eta[, mu]) of the nodes of a geometric-order
    q Lagrange quad or hex in Gmsh order."""
    ns = q + 1
    if nd == 2:
        return _quad_rings(0, ns - 1)
    out = []
    for level in range(ns // 2):
        i, j, m = level, ns - 1 - level, ns - 2 * (level + 1)
        out += [(i, i, i), (j, i, i), (j, j, i), (i, j, i), (i, i, j), (j, i, j), (j, j, j), (i, j, j)]
        edges = [lambda r, s: (r, i, i), lambda r, s: (i, r, i), lambda r, s: (i, i, r),
                 lambda r, s: (j, r, i), lambda r, s: (j, i, r), lambda r, s: (s, j, i),
                 lambda r, s: (j, j, r), lambda r, s: (i, j, r), lambda r, s: (r, i, j),
                 lambda r, s: (i, r, j), lambda r, s: (j, r, j), lambda r, s: (s, j, j)]
        for e in edges:
            out += [e(i + 1 + k, j - 1 - k) for k in range(m)]
        qr = _quad_rings(i + 1, j - 1)
        out += [(b, a, i) for a, b in qr]          # mu = low
        out += [(a, i, b) for a, b in qr]          # eta = low
        out += [(i, b, a) for a, b in qr]          # xi = low
        out += [(j, a, b) for a, b in qr]          # xi = high
        out += [(ns - 1 - a, j, b) for a, b in qr]  # eta = high
        out += [(a, b, j) for a, b in qr]          # mu = high
    if ns % 2:
        out.append((ns // 2,) * 3)
    return out


# 20-node serendipity hex: corners, then mid-edge nodes in Gmsh's edge order
# 0-1, 0-3, 0-4, 1-2, 1-5, 2-3, 2-6, 3-7, 4-5, 4-7, 5-6, 6-7 (indices on a
# 3-point grid per direction)
_SER20 = [(0, 0, 0), (2, 0, 0), (2, 2, 0), (0, 2, 0), (0, 0, 2), (2, 0, 2), (2, 2, 2), (0, 2, 2),
          (1, 0, 0), (0, 1, 0), (0, 0, 1), (2, 1, 0), (2, 0, 1), (1, 2, 0), (2, 2, 1), (0, 2, 1),
          (1, 0, 2), (0, 1, 2), (2, 1, 2), (1, 2, 2)]


def curved_box(nd: int, n: int, q: int, length: float, amp: float = 0.04, serendipity: bool = False):
    """A box [0, length]^nd of n^nd curved quads/hexes of geometric order q
    (serendipity: the 20-node hex, q = 2).  Every node sits on the smooth map
        x = X + amp L sin(2 pi X/L) sin(pi Y/L) [sin(pi Z/L)]
        y = Y + amp L (1 - Y/L) sin(pi X/L) [sin(pi Z/L)]
        z = Z + amp L sin(pi X/L) sin(2 pi Z/L) sin(pi Y/L)      (3-D)
    of the uniform grid, so the lower y face is curved, the x and z faces stay
    planar and every interior face is curved.  Boundaries: bottom/top (y),
    left/right (x), front/back (z, 3-D)."""
    if serendipity:
        assert nd == 3 and q == 2
    L, g = float(length), n * q + 1
    grid = np.linspace(0.0, L, g)
    idx = {}
    coords = []

    def node(I):
        if I not in idx:
            X = [grid[k] for k in I]
            s = lambda k, f=1.0: np.sin(f * np.pi * X[k] / L)
            if nd == 2:
                x = X[0] + amp * L * s(0, 2.0) * s(1)
                y = X[1] + amp * L * (1 - X[1] / L) * s(0)
                coords.append((x, y))
            else:
                x = X[0] + amp * L * s(0, 2.0) * s(1) * s(2)
                y = X[1] + amp * L * (1 - X[1] / L) * s(0) * s(2)
                z = X[2] + amp * L * s(0) * s(2, 2.0) * s(1)
                coords.append((x, y, z))
            idx[I] = len(coords) - 1
        return idx[I]

    order = _SER20 if serendipity else lagrange_node_order(nd, q)
    cells = []
    for e in np.ndindex(*[n] * nd):
        e = e[::-1]  # x fastest
        cells.append([node(tuple(e[d] * q + t[d] for d in range(nd))) for t in order])
    # boundary elements: all nodes of an edge (2-D), a quad face's nodes (3-D)
    faces = {}
    if nd == 2:
        line = [0, q] + list(range(1, q))
        for i in range(n):
            faces.setdefault("bottom", []).append([node((i * q + t, 0)) for t in line])
            faces.setdefault("top", []).append([node((i * q + t, n * q)) for t in line])
            faces.setdefault("left", []).append([node((0, i * q + t)) for t in line])
            faces.setdefault("right", []).append([node((n * q, i * q + t)) for t in line])
    else:
        fq = [(0, 0), (2, 0), (2, 2), (0, 2), (1, 0), (2, 1), (1, 2), (0, 1)] if serendipity else \
            _quad_rings(0, q)
        for i in range(n):
            for j in range(n):
                for name, ax, side in (("left", 0, 0), ("right", 0, n * q), ("bottom", 1, 0), ("top", 1, n * q),
                                       ("front", 2, 0), ("back", 2, n * q)):
                    pts = []
                    for a, b in fq:
                        I = [0, 0, 0]
                        o = [d for d in range(3) if d != ax]
                        I[ax], I[o[0]], I[o[1]] = side, i * q + a, j * q + b
                        pts.append(node(tuple(I)))
                    faces.setdefault(name, []).append(pts)
    return {"xv": np.array(coords), "cells": cells, "faces": faces, "nd": nd, "q": q,
            "serendipity": serendipity}


_CELL_TYPE = {(2, 4): 3, (2, 9): 10, (2, 16): 36, (2, 25): 37, (3, 8): 5, (3, 20): 17, (3, 27): 12, (3, 64): 92}
_FACE_TYPE = {(2, 2): 1, (2, 3): 8, (2, 4): 26, (2, 5): 27, (3, 4): 3, (3, 8): 16, (3, 9): 10, (3, 16): 36}


def write_gmsh_ho(path: str, m: dict) -> None:
    """Gmsh 2.2 ASCII of a `curved_box` mesh: one physical group per boundary
    name, the cells as the volume group "fluid"."""
    nd, xv = m["nd"], m["xv"]
    names = list(m["faces"].keys())
    lines = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$PhysicalNames", str(len(names) + 1)]
    for k, nm in enumerate(names):
        lines.append(f'{nd - 1} {k + 1} "{nm}"')
    fluid = len(names) + 1
    lines += [f'{nd} {fluid} "fluid"', "$EndPhysicalNames", "$Nodes", str(len(xv))]
    for i, p in enumerate(xv):
        c = list(p) + [0.0] * (3 - len(p))
        lines.append(f"{i + 1} " + " ".join(f"{float(v):.17g}" for v in c))
    lines += ["$EndNodes", "$Elements"]
    elems = []
    for k, nm in enumerate(names):
        for f in m["faces"][nm]:
            elems.append(f"{_FACE_TYPE[(nd, len(f))]} 2 {k + 1} {k + 1} " + " ".join(str(v + 1) for v in f))
    for c in m["cells"]:
        elems.append(f"{_CELL_TYPE[(nd, len(c))]} 2 {fluid} {fluid} " + " ".join(str(v + 1) for v in c))
    lines.append(str(len(elems)))
    lines += [f"{i + 1} {e}" for i, e in enumerate(elems)]
    lines.append("$EndElements")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
