"""Shared-memory bank model of the 3-D TMA element kernel's flux-tile reads.

A design aid, not part of the library: it counts the shared-memory
wavefronts that the line phases of `k_elem_tma` (stage_tma.cu) issue for a
given flux-tile layout, so the row and plane padding of the tile can be
chosen by search instead of by trial on the GPU.

Model: 32 banks of 4 bytes; a warp's access costs as many wavefronts as the
most distinct words any one bank must serve, and at least its distinct bytes
/ 128 (so a warp's 8-byte load of 32 distinct values costs 2).

Access patterns (thread t of a CTA is (solution point s, element el) with
t = s*EB + el in the point phases and (flux point f, element fe) with
t = f*EB + fe in the flux-point phases; a warp is 32 consecutive threads):
  C1  divergence: point s reads the flux tile of dimension d at the N points
      of its line along d, field by field;
  C2  extrapolated normal flux: flux point f reads the flux tile of its
      normal dimension at the N points of its line;
  E   extrapolation of the new state: as C2, from the copy of the state;
  own each point's own record (flux stores, the state copy).
Flux points are numbered face by face (x-, x+, y-, y+, z-, z+), N*N per face.

    python bank_model.py            # the search for FP64 P3 (2 and 4 elements)
"""
from __future__ import annotations

import math
from itertools import product


def wavefronts(byte_addrs, width):
    distinct = set(byte_addrs)
    banks = {}
    for a in distinct:
        for w in range(width // 4):
            word = a // 4 + w
            banks.setdefault(word % 32, set()).add(word)
    return max(max(len(v) for v in banks.values()), math.ceil(len(distinct) * width / 128))


def count(P, width, EB, row_pad, plane_pad, NF=5):
    """Wavefronts per CTA of the flux-tile line phases for a tile whose point
    p starts at p*EB*NF + (p//N)*row_pad + (p//N^2)*plane_pad values."""
    N = P + 1
    NS, NPF = N ** 3, N * N
    ROW = EB * NF

    def off(p):
        return p * ROW + (p // N) * row_pad + (p // NPF) * plane_pad

    slab = off(NS)

    def ijk(p):
        return [p % N, (p // N) % N, p // NPF]

    def pid(i):
        return i[0] + N * i[1] + NPF * i[2]

    out = {"C1": 0, "C2": 0, "E": 0, "own": 0}
    NT = NS * EB
    for w0 in range(0, NT, 32):
        lanes = [divmod(t, EB) for t in range(w0, min(w0 + 32, NT))]
        for d, m, k in product(range(3), range(N), range(NF)):
            addrs = []
            for s, el in lanes:
                i = ijk(s)
                i[d] = m
                addrs.append(width * (d * slab + off(pid(i)) + el * NF + k))
            out["C1"] += wavefronts(addrs, width)
        for k in range(NF):
            out["own"] += 4 * wavefronts([width * (off(s) + el * NF + k) for s, el in lanes], width)
    fpts = []
    for dn in range(3):
        free = [d for d in range(3) if d != dn]
        for _side, u, v in product(range(2), range(N), range(N)):
            i = [0, 0, 0]
            i[free[0]], i[free[1]] = v, u
            fpts.append((dn, i))
    for w0 in range(0, len(fpts) * EB, 32):
        lanes = [divmod(t, EB) for t in range(w0, min(w0 + 32, len(fpts) * EB))]
        for m, k in product(range(N), range(NF)):
            aF, aU = [], []
            for f, fe in lanes:
                dn, i = fpts[f]
                i = list(i)
                i[dn] = m
                aF.append(width * (dn * slab + off(pid(i)) + fe * NF + k))
                aU.append(width * (off(pid(i)) + fe * NF + k))
            out["C2"] += wavefronts(aF, width)
            out["E"] += wavefronts(aU, width)
    out["sum"] = sum(out.values())
    return out


def best_padding(P, width, EB, rows=range(9), planes=range(17)):
    """(row_pad, plane_pad) with the fewest wavefronts (smallest pads first)."""
    return min(((count(P, width, EB, a, b)["sum"], a + b, a, b) for a in rows for b in planes))


if __name__ == "__main__":
    for eb in (2, 4):
        base = count(3, 8, eb, 0, 0)
        total, _, a, b = best_padding(3, 8, eb)
        print(f"FP64 P3 EB{eb}: unpadded {base['sum']}, best row {a} plane {b}: {total}",
              count(3, 8, eb, a, b))
