"""The two builds of the reference under oracle/_ref set meshes up alike.

The timing build (fr_ref_harness_omp) replaces the reference's O(n^2) row
de-duplication by a hashed one (oracle/refshim/fast_unique.cpp) so that its
32^3 mesh sets up in minutes; the parity build (fr_ref_harness) keeps the
reference's own.  Both must give the same face connectivity on every kind of
mesh the benchmarks use: periodic 2-D and 3-D boxes, and a Gmsh mesh with
walls and far-field boundaries.  CPU only; skipped where the reference was not
built.
"""
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_golden as MG  # noqa: E402

O2 = os.path.join(ROOT, "oracle", "_ref", "fr_ref_harness")
OMP = os.path.join(ROOT, "oracle", "_ref", "fr_ref_harness_omp")
BIG = os.path.join(ROOT, "oracle", "_ref", "fr_ref_harness_bigmesh")
FACE = ["face_type", "face_eL", "face_locL", "face_eR", "face_locR", "face_relRot", "face_bc", "face_fptR"]

pytestmark = pytest.mark.skipif(not (os.path.exists(O2) and os.path.exists(OMP)),
                                reason="reference builds (oracle/_ref) not present")


def dump(binary, deck, args=()):
    with tempfile.TemporaryDirectory() as td, tempfile.TemporaryDirectory() as wd:
        path = MG.stage_deck(deck, wd)
        env = dict(os.environ, OMP_NUM_THREADS="2")
        subprocess.run([binary, path, td, *args], check=True, stdout=subprocess.DEVNULL, cwd=wd, env=env)
        return MG.read_dump(td)


def dump_faces(binary, deck):
    arrays, meta = dump(binary, deck)
    return {k: arrays[k] for k in FACE}, meta


@pytest.mark.parametrize("deck", ["tgv3d_p3_4", "vortex2d_p3_8", "chbump_p2_pmg", "wallchar3d_p2"])
def test_timing_build_sets_up_the_same_faces(deck):
    a, ma = dump_faces(O2, deck)
    b, mb = dump_faces(OMP, deck)
    assert ma["nFaces"] == mb["nFaces"] and ma["nEles"] == mb["nEles"]
    for k in FACE:
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.skipif(not os.path.exists(BIG), reason="big-mesh parity build not present")
@pytest.mark.parametrize("deck", ["tgv3d_p3_4", "chbump_p2_pmg"])
def test_bigmesh_parity_build_equals_the_parity_build(deck):
    """The parity build with the hashed row de-duplication (used for the
    32^3 fixture) gives the parity build's dumps bit for bit: connectivity,
    metrics, one residual and the state after 3 steps."""
    args = ["--steps", "3"] + (["--ic", "tgv", "--cfl-dt", "0.5"] if deck.startswith("tgv") else [])
    a, ma = dump(O2, deck, args)
    b, mb = dump(BIG, deck, args)
    assert sorted(a) == sorted(b)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
