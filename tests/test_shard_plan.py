"""The sharding plan (fr_shard_plan, host only): the element partition covers
every element once and is balanced, and the halo of each part lists exactly
the points of the faces the partition cuts, both sides of every cut in the
same order; two gloo ranks exchange traces packed in that order and each
receives, point by point, the trace of the other side of the same face point
(the exchange mpiFace::communicate / getRightState make,
src/mpiFace.cpp:122-175)."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

import flurrypp_b200 as fb
from conftest import DECKS, ROOT

DECKS_USED = ["tgv3d_p3_4.deck", "vortex2d_p3_8.deck", "cyl2d_p2.deck", "curved3d_q2_p2.deck", "chbump_p3.deck"]


def host_case(deck):
    return fb.Solver(os.path.join(DECKS, deck), device=-1)


def face_table(s):
    """Both sides' global slots (fpt * nEles + element) of every interior face
    point, in face order and left point order."""
    eL, locL = s.get_array("face_eL"), s.get_array("face_locL")
    eR, fptR = s.get_array("face_eR"), s.get_array("face_fptR")
    nPF = fptR.size // eL.size
    fptR = fptR.reshape(-1, nPF)
    rows = []
    for f in range(eL.size):
        if eR[f] < 0:
            continue
        for j in range(nPF):
            rows.append((f, int(eL[f]), int(locL[f]) * nPF + j, int(eR[f]), int(fptR[f, j])))
    return rows


def global_slots(s, part, rank, slots):
    owned = np.nonzero(part == rank)[0]
    n = owned.size
    return [(int(sl // n), int(owned[sl % n])) for sl in slots]


@pytest.mark.parametrize("deck", DECKS_USED)
@pytest.mark.parametrize("nparts", [2, 3, 4])
def test_partition_and_halo_consistent(deck, nparts):
    s = host_case(deck)
    plans = [s.shard_plan(nparts, r) for r in range(nparts)]
    part = plans[0][0]
    for p in plans[1:]:
        assert np.array_equal(p[0], part)  # every rank computes the same partition
    sizes = np.bincount(part, minlength=nparts)
    assert sizes.sum() == s.nEles and sizes.min() >= 1 and sizes.max() - sizes.min() <= 1
    for r, (_, n_owned, peer, slot) in enumerate(plans):
        assert n_owned == sizes[r]
    rows = face_table(s)
    for a in range(nparts):
        for b in range(nparts):
            if a == b:
                continue
            # what each side must list, in face and point order
            want_a = [(fl, el) if part[el] == a else (fr, er)
                      for (_, el, fl, er, fr) in rows if {part[el], part[er]} == {a, b}]
            _, _, peer_a, slot_a = plans[a]
            got_a = global_slots(s, part, a, slot_a[peer_a == b])
            assert got_a == [(f, e) for (f, e) in want_a]
    # a part's halo holds nothing else than points on cut faces
    cut = sum(1 for (_, el, _, er, _) in rows if part[el] != part[er])
    assert sum(p[2].size for p in plans) == 2 * cut


def test_one_part_has_no_halo():
    s = host_case(DECKS_USED[0])
    part, n_owned, peer, slot = s.shard_plan(1, 0)
    assert n_owned == s.nEles and peer.size == 0 and not part.any()


def test_bad_arguments():
    s = host_case(DECKS_USED[0])
    with pytest.raises(fb.FrError):
        s.shard_plan(2, 2)
    with pytest.raises(fb.FrError):
        s.shard_plan(s.nEles + 1, 0)


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _rank(rank, world, port, deck, q):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        s = host_case(deck)
        part, n_owned, peer, slot = s.shard_plan(world, rank)
        owned = np.nonzero(part == rank)[0]
        # this part's traces: each local slot holds its global slot id
        nF = s.nFpts
        trace = np.array([(sl // n_owned) * s.nEles + owned[sl % n_owned] for sl in range(nF * n_owned)],
                         dtype=np.float64)
        ok = True
        for other in range(world):
            if other == rank:
                continue
            mine = slot[peer == other]
            send = torch.from_numpy(trace[mine].copy())
            recv = torch.empty_like(send)
            # lower rank sends first: every pair takes the same two steps
            if rank < other:
                dist.send(send, other)
                dist.recv(recv, other)
            else:
                dist.recv(recv, other)
                dist.send(send, other)
            # the other side of each listed point, from the global face table
            other_side = {}
            for (_, el, fl, er, fr) in face_table(s):
                other_side[(fl, el)] = fr * s.nEles + er
                other_side[(fr, er)] = fl * s.nEles + el
            want = [other_side[g] for g in global_slots(s, part, rank, mine)]
            ok = ok and np.array_equal(recv.numpy(), np.array(want, dtype=np.float64))
        q.put((rank, bool(ok), int(slot.size)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("deck", ["tgv3d_p3_4.deck", "chbump_p3.deck"])
def test_two_gloo_ranks_exchange_traces_in_plan_order(deck):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, deck, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        for p in procs:
            p.join(180)
    finally:
        for p in procs:  # a rank blocked on a dead peer must not outlive the test
            if p.is_alive():
                p.kill()
                p.join(10)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert all(ok for _, ok, _ in got)
    assert got[0][2] == got[1][2] > 0


def part_oracle(a, meta, part, rank, peer, slot):
    """The numpy oracle on one part: the fixture's arrays sliced to the part's
    elements, its interior and boundary faces renumbered, and its cut face
    points (halo order, stably sorted by peer as the library lists them), each
    formed with the part's own element as the left side and the received
    trace as the right state."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import fr_oracle as O
    from conftest import deck_path

    owned = np.nonzero(part == rank)[0]
    local = -np.ones(part.size, dtype=np.int64)
    local[owned] = np.arange(owned.size)
    b = {k: v for k, v in a.items() if k.startswith("opp_")}
    b["detJac_spts"] = a["detJac_spts"][:, owned]
    b["JGinv_spts"] = a["JGinv_spts"][:, :, owned, :]
    b["norm_fpts"] = a["norm_fpts"][:, owned, :]
    b["dA_fpts"] = a["dA_fpts"][:, owned]
    eL, eR = a["face_eL"], a["face_eR"]
    keep = (part[eL] == rank) & ((eR < 0) | (part[np.maximum(eR, 0)] == rank))
    b["face_eL"] = local[eL[keep]]
    b["face_locL"] = a["face_locL"][keep]
    b["face_eR"] = np.where(eR[keep] >= 0, local[np.maximum(eR[keep], 0)], -1)
    b["face_fptR"] = a["face_fptR"].reshape(eL.size, -1)[keep]
    b["face_bc"] = a["face_bc"][keep]
    p = O.params_from_deck(deck_path(meta))
    p["dt"] = meta["dt"]
    c = O.OracleCase(b, p)
    order = np.argsort(peer, kind="stable")
    c.cut_slot, c.cut_peer = slot[order], peer[order]
    base_faces = c.faces

    def faces(Uf):
        Fn = base_faces(Uf).reshape(-1, c.nF)
        Ufl = Uf.reshape(-1, c.nF)
        n = c.norm.reshape(-1, c.nd)[c.cut_slot]
        UL = Ufl[c.cut_slot]
        if c.nd == 2 and int(p.get("riemannType", 0)) == 1:
            F = O.roe2d(UL, c.recv, n, p["gamma"])
        else:
            F, _ = O.rusanov(UL, c.recv, n, p["gamma"])
        Fn[c.cut_slot] = F * c.dA.ravel()[c.cut_slot][:, None]
        return Fn.reshape(Uf.shape)

    c.faces = faces
    return c, owned


def _rank_residual(rank, world, port, case, q):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import fr_oracle as O
    from conftest import deck_path, load_golden

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        a, meta = load_golden(case)
        s = fb.Solver(deck_path(meta), device=-1)
        part, _, peer, slot = s.shard_plan(world, rank)
        c, owned = part_oracle(a, meta, part, rank, peer, slot)
        U = a["U_init"][:, owned, :]
        Uf = c.extrapolate(U).reshape(-1, c.nF)
        send = torch.from_numpy(np.ascontiguousarray(Uf[c.cut_slot]))
        recv = torch.empty_like(send)
        other = 1 - rank
        if rank == 0:
            dist.send(send, other)
            dist.recv(recv, other)
        else:
            dist.recv(recv, other)
            dist.send(send, other)
        c.recv = recv.numpy()
        d_part = c.residual(U)
        p = O.params_from_deck(deck_path(meta))
        p["dt"] = meta["dt"]
        d_full = O.OracleCase(a, p).residual(a["U_init"])[:, owned, :]
        fscale = float(np.max(np.abs(a["F_spts"])))
        err = float(np.max(np.abs(d_part - d_full))) / max(fscale, float(np.max(np.abs(d_full))))
        q.put((rank, err, int(c.cut_slot.size)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", ["tgv3d_p3_4", "chbump_p3", "roe2d_p2"])
def test_two_gloo_ranks_residual_through_the_partition(case):
    """Each of two gloo ranks computes the residual of its part with the numpy
    oracle, the right traces of its cut faces received from the other rank in
    the plan's order: together they give the whole case's residual (to the
    round-off of each side using its own normal)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_residual, args=(r, 2, port, case, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        for p in procs:
            p.join(180)
    finally:
        for p in procs:
            if p.is_alive():
                p.kill()
                p.join(10)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got[0][2] == got[1][2] > 0
    for _, err, _ in got:
        assert err < 1e-14, err
