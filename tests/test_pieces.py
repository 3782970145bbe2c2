"""Multi-piece decomposition on CPU: the partition (pnt_mesh_piece) and the
halo exchange (pennant_b200.pieces over gloo, world size 2 and 3).

A piece keeps every zone's and point's single-piece computation; what must
hold is that (1) the pieces cover the zones exactly once, (2) a piece holds
every point its zones touch, (3) each local point's corner list, local and
halo slots, is the global corner list in global side order, and (4) the
exchange fills every halo slot with the owning piece's value, so the
corner sums at shared points equal the single-piece sums bit for bit.
A rank lost between steps ends its neighbour's next exchange with an error,
not a wait without end."""
import os
import socket
import sys

import numpy as np
import pytest
from hypothesis import given, settings
from hypothesis import strategies as st
import torch.multiprocessing as mp

from conftest import DECKS, golden
import pennant_b200 as pb

sys.path.insert(0, DECKS)
from make_decks import sedov  # noqa: E402


def meshes():
    yield "sedov", pb.Mesh(deck=pb.Deck(text=sedov(12)))
    yield "noh-pie", pb.Mesh(deck=pb.Deck(path=golden("nohsmall.pnt")))


def slot_sides(info, nums, slots):
    """Global side of each corner slot (local side or halo slot)."""
    return np.where(slots < nums, slots + info["side0"], info["halo_side"][np.clip(slots - nums, 0, None)])


@pytest.mark.parametrize("npieces", [2, 3, 7])
def test_partition_covers_and_keeps_the_corner_order(npieces):
    for name, m in meshes():
        check_partition(name, m, npieces)


@settings(max_examples=40, deadline=None)
@given(kind=st.sampled_from(["rect", "pie"]), nx=st.integers(1, 12), ny=st.integers(1, 12),
       npieces=st.integers(2, 64))
def test_partition_of_random_meshes(kind, nx, ny, npieces):
    extra = "1.0 1.0" if kind == "rect" else "90.0 1.0"
    m = pb.Mesh(deck=pb.Deck(text=f"cstop 1\nmeshtype {kind}\nmeshparams {nx} {ny} {extra}\n"))
    if npieces > m.numz:
        with pytest.raises(pb.PntError):
            m.piece(npieces, 0)
        return
    check_partition(f"{kind} {nx}x{ny}", m, npieces)


def check_partition(name, m, npieces):
    """Invariants (1)-(3) of the module docstring and the pairing of send
    lists with halo slots, for `m` split into npieces."""
    goff, gsides = m.point_corners()
    gmapsp1, gmapsz = m.array("mapsp1"), m.array("mapsz")
    zone_owner = np.full(m.numz, -1)
    infos = []
    for q in range(npieces):
        pm = m.piece(npieces, q)
        info = pm.piece_info()
        infos.append((pm, info))
        z0 = info["zone0"]
        assert (zone_owner[z0:z0 + pm.numz] == -1).all(), name
        zone_owner[z0:z0 + pm.numz] = q
        # local zones' sides are the global sides side0 .. side0 + nums
        assert (pm.array("mapsz") + z0 == gmapsz[info["side0"]:info["side0"] + pm.nums]).all()
        # points: exactly those the zones touch, ascending global ids
        gp = info["gpoint"]
        assert (np.diff(gp) > 0).all()
        touched = np.unique(gmapsp1[info["side0"]:info["side0"] + pm.nums])
        assert np.array_equal(touched, gp), name
        assert (gp[pm.array("mapsp1")] == gmapsp1[info["side0"]:info["side0"] + pm.nums]).all()
        assert np.array_equal(pm.array("px"), m.array("px")[gp])
        # corner lists: the global list of each point, in global order
        off, slots = pm.point_corners()
        assert len(slots) == pm.nums + info["nhalo"]
        sides_of_slots = slot_sides(info, pm.nums, slots)
        for p in range(pm.nump):
            g = gp[p]
            assert np.array_equal(sides_of_slots[off[p]:off[p + 1]], gsides[goff[g]:goff[g + 1]]), (name, q, p)
    assert (zone_owner >= 0).all(), name
    # send lists of i to j = the halo slots j receives from i, same order
    for q, (pm, info) in enumerate(infos):
        for j, r in enumerate(info["nbr"]):
            rpm, rinfo = infos[r]
            k = list(rinfo["nbr"]).index(q)
            sent = info["send_side"][info["send_off"][j]:info["send_off"][j + 1]] + info["side0"]
            recv = rinfo["halo_side"][rinfo["recv_off"][k]:rinfo["recv_off"][k + 1]]
            assert np.array_equal(sent, recv), (name, q, r)


def test_one_piece_is_the_mesh():
    m = pb.Mesh(deck=pb.Deck(text=sedov(6)))
    pm = m.piece(1, 0)
    info = pm.piece_info()
    assert info["nhalo"] == 0 and len(info["nbr"]) == 0
    assert np.array_equal(pm.array("mapsp1"), m.array("mapsp1"))
    assert all(np.array_equal(a, b) for a, b in zip(pm.point_corners(), m.point_corners()))


def test_bad_piece_arguments():
    m = pb.Mesh(deck=pb.Deck(text=sedov(4)))
    for n, q in ((0, 0), (2, 2), (65, 0), (17, 0)):   # 17 pieces > 16 zones
        with pytest.raises(pb.PntError):
            m.piece(n, q)
    with pytest.raises(pb.PntError):
        m.piece(2, 0).piece(2, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _exchange_rank(rank, world, port, mixed, out):
    import torch
    import torch.distributed as dist
    from pennant_b200.pieces import HaloExchange
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        m = pb.Mesh(deck=pb.Deck(text=sedov(10)))
        pm = m.piece(world, rank)
        info = pm.piece_info()
        # per global side: a corner mass and force (seeded, the same on all ranks)
        rng = np.random.default_rng(5)
        dt = np.float32 if mixed else np.float64
        cmass_g = rng.standard_normal(m.nums).astype(dt)
        cforce_g = rng.standard_normal((m.nums, 2)).astype(dt)
        cmb, cfb = cmass_g.itemsize, 2 * cmass_g.itemsize
        s0 = info["side0"]
        local_m, local_f = cmass_g[s0:s0 + pm.nums], cforce_g[s0:s0 + pm.nums]
        nsend = int(info["send_off"][-1])
        foff = (nsend * cmb + 15) // 16 * 16
        send = np.zeros(foff + nsend * cfb, np.uint8)
        send[:nsend * cmb] = local_m[info["send_side"]].view(np.uint8)
        send[foff:] = np.ascontiguousarray(local_f[info["send_side"]]).view(np.uint8).ravel()
        halo_m = torch.zeros(info["nhalo"] * cmb, dtype=torch.uint8)
        halo_f = torch.zeros(info["nhalo"] * cfb, dtype=torch.uint8)
        HaloExchange(info, cmb, cfb, foff).exchange(torch.from_numpy(send), halo_m, halo_f)
        hm = halo_m.numpy().view(dt)
        hf = halo_f.numpy().view(dt).reshape(-1, 2)
        # every halo slot holds its owner's value
        assert np.array_equal(hm, cmass_g[info["halo_side"]])
        assert np.array_equal(hf, cforce_g[info["halo_side"]])
        # the corner sums at the piece's points, in slot order, equal the
        # single-piece sums in global order, bit for bit
        allm = np.concatenate([local_m, hm])
        allf = np.concatenate([local_f, hf])
        off, slots = pm.point_corners()
        goff, gsides = m.point_corners()
        for p, g in enumerate(info["gpoint"]):
            a, b = dt(0), np.zeros(2, dt)
            for c in range(off[p], off[p + 1]):
                a = dt(a + allm[slots[c]])
                b = (b + allf[slots[c]]).astype(dt)
            ga, gb = dt(0), np.zeros(2, dt)
            for c in range(goff[g], goff[g + 1]):
                ga = dt(ga + cmass_g[gsides[c]])
                gb = (gb + cforce_g[gsides[c]]).astype(dt)
            assert a.tobytes() == ga.tobytes() and b.tobytes() == gb.tobytes()
        out[rank] = 1
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,mixed", [(2, False), (3, True)])
def test_halo_exchange_over_gloo(world, mixed):
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    mp.start_processes(_exchange_rank, args=(world, _free_port(), mixed, out), nprocs=world, join=True,
                       start_method="spawn")
    assert sorted(out.keys()) == list(range(world))


def test_pieces_driver_arguments_and_no_device():
    """pnt_pieces_create: fewer than two pieces is an argument error; without
    a GPU it fails cleanly (no device), after building the pieces on the
    host."""
    import torch
    m = pb.Mesh(deck=pb.Deck(text=sedov(6)))
    d = pb.Deck(text=sedov(6))
    with pytest.raises(pb.PntError) as e:
        pb.Pieces(m, d.params(), 1)
    assert e.value.status == pb.PNT_ERR_INVALID_ARG
    if not torch.cuda.is_available():
        with pytest.raises(pb.PntError) as e:
            pb.Pieces(m, d.params(), 2)
        assert e.value.status == pb.PNT_ERR_NO_DEVICE


def _lost_rank(rank, world, port, mode, out):
    import time
    import torch
    import torch.distributed as dist
    from pennant_b200.pieces import HaloExchange, reduce_scalars
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=5))
    m = pb.Mesh(deck=pb.Deck(text=sedov(8)))
    info = m.piece(world, rank).piece_info()
    if rank == 1:
        # this rank leaves between steps (exits, or stays alive and never
        # takes the next step): no exchange, no reduction
        if mode == "stall":
            time.sleep(12)
        out[rank] = "left"
        return
    nsend, nhalo = int(info["send_off"][-1]), int(info["nhalo"])
    send = torch.zeros(16 + nsend * 24, dtype=torch.uint8)
    t0 = time.monotonic()
    for step in (lambda: HaloExchange(info, 8, 16, 16 + nsend * 8).exchange(
                     send, torch.zeros(nhalo * 8, dtype=torch.uint8), torch.zeros(nhalo * 16, dtype=torch.uint8)),
                 lambda: reduce_scalars(torch.zeros(4, dtype=torch.float64))):
        try:
            step()
            out[rank] = "no error"
            return
        except RuntimeError as e:
            out[rank] = ("error", time.monotonic() - t0, str(e)[:200])
            break


@pytest.mark.parametrize("mode", ["exit", "stall"])
def test_a_lost_rank_ends_the_exchange_with_an_error(mode):
    """A rank that leaves between steps: its neighbour's next exchange ends
    with an error (the closed connection, or the process group's 5 s
    timeout) instead of waiting for good."""
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    mp.start_processes(_lost_rank, args=(2, _free_port(), mode, out), nprocs=2, join=True, start_method="spawn")
    assert out[1] == "left"
    assert out[0][0] == "error", out[0]
    assert out[0][1] < 11, out[0]


def _reduce_rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from pennant_b200.pieces import reduce_scalars
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        # {dtnew, -dvovmax, inverted sides in pass A, in pass C} of this piece
        red = torch.tensor([1e-3 * (rank + 2), -0.01 * (rank + 1), float(rank), 2.0 * rank], dtype=torch.float64)
        reduce_scalars(red)
        out[rank] = red.tolist()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_piece_scalars_reduce_over_gloo(world):
    """The per-cycle scalars: minimum dtnew and -dvovmax (the maximum dV/V),
    summed inverted-side counts, the same on every rank."""
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    mp.start_processes(_reduce_rank, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    want = [2e-3, -0.01 * world, float(sum(range(world))), 2.0 * sum(range(world))]
    for r in range(world):
        assert out[r] == want, (r, out[r])
