"""Readers for the reference's solution files (test helpers).

`read_vtu` splits a ParaView file of the reference's layout
(src/output.cpp:137-512) into its header comments, its tag lines (everything
that is not a data line) and, per <Piece>, the data arrays by name;
`read_csv` reads the CSV writer's rows (src/output.cpp:60-135).
"""
from __future__ import annotations

import gzip
import re

import numpy as np


def read_vtu(text: str) -> dict:
    lines = text.splitlines()
    out = {"tags": [], "pieces": [], "time": None, "iter": None}
    i = 0
    piece = None
    while i < len(lines):
        ln = lines[i]
        s = ln.strip()
        if s.startswith("<!-- TIME"):
            out["time"] = s.split()[2]
        elif s.startswith("<!-- ITER"):
            out["iter"] = int(s.split()[2])
        if s.startswith("<Piece"):
            piece = {}
            out["pieces"].append(piece)
        out["tags"].append(ln)
        if s.startswith("<DataArray"):
            m = re.search(r'Name="([^"]+)"', s)
            name = m.group(1) if m else "Points"
            i += 1
            block = []
            while not lines[i].strip().startswith("</DataArray>"):
                block.append(lines[i])
                i += 1
            out["tags"].append(lines[i])
            dtype = np.int64 if name in ("connectivity", "offsets", "types") else np.float64
            piece[name] = np.array(" ".join(block).split(), dtype=dtype)
        i += 1
    return out


def read_vtu_gz(buf: np.ndarray) -> dict:
    return read_vtu(gzip.decompress(buf.tobytes()).decode())


def read_csv(text: str) -> tuple[str, np.ndarray]:
    lines = text.splitlines()
    return lines[0], np.array([[float(x) for x in ln.split(",")] for ln in lines[1:]])
