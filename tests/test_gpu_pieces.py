"""Multi-piece runs on the GPU (needs a GPU): the mesh split over 2 or 3
ranks (processes; on one GPU they share it and exchange through gloo and
host memory, so no kernel waits on another), every rank stepping its piece
with pennant_b200.pieces.PieceHydro.  Each piece's zones and points must be
bit-identical to the single-piece run of the same deck, for the FP64 cycle
(rect and pie meshes), the mixed cycle and the learned cycle."""
import datetime
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import DECKS, PKG, golden
import pennant_b200 as pb

sys.path.insert(0, DECKS)
from make_decks import sedov  # noqa: E402

pytestmark = pytest.mark.gpu

CLOSURE = os.path.join(PKG, "closure", "qcs_mlp.bin")
ZONE = ("zr", "ze", "zetot", "zvol", "zwrate")
POINT = ("px", "pu")


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _deck(text, precision):
    d = pb.Deck(text=text)
    d.set("precision", precision)
    return d


def _rank(rank, world, port, text, precision, out):
    import torch.distributed as dist
    from pennant_b200.pieces import PieceHydro
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        d = _deck(text, precision)
        clo = pb.Closure(path=CLOSURE) if precision == "learned" else None
        ph = PieceHydro(pb.Mesh(deck=d), d.params(), device=0, closure=clo)
        s = ph.run()
        out[rank] = (s, ph.fields(ZONE + POINT), ph.info)
        ph.close()
    finally:
        dist.destroy_process_group()


def single(text, precision):
    d = _deck(text, precision)
    h = pb.Hydro(pb.Mesh(deck=d), d.params())
    if precision == "learned":
        h.set_closure(pb.Closure(path=CLOSURE))
    s = h.run()
    f = {k: h.download(k) for k in ZONE + POINT}
    h.close()
    return s, f


CASES = {
    "sedov-fp64": (sedov(24, tstop=0.05), "fp64", 2),
    "sedov-fp64-3": (sedov(20, tstop=0.05), "fp64", 3),
    "noh-pie-fp64": (open(golden("nohsmall.pnt")).read().replace("cstop   10", "cstop   60"), "fp64", 2),
    "sedov-mixed": (sedov(24, tstop=0.05), "mixed", 2),
    "sedov-learned": (sedov(32, tstop=0.2), "learned", 2),
}


@pytest.mark.timeout(600)
@pytest.mark.parametrize("case", sorted(CASES))
def test_pieces_match_the_single_piece_run_bitwise(case):
    text, precision, world = CASES[case]
    s1, f1 = single(text, precision)
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_rank, args=(world, _port(), text, precision, out), nprocs=world, join=True,
                       start_method="spawn")
    assert sorted(out.keys()) == list(range(world))
    for r in range(world):
        s, f, info = out[r]
        assert s["cycle"] == s1["cycle"] and s["time"] == s1["time"] and s["done"] == 1, (case, r, s, s1)
        z = slice(info["zone0"], info["zone0"] + len(f["zr"]))
        for k in ZONE:
            assert f[k].tobytes() == f1[k][z].tobytes(), (case, r, k)
        for k in POINT:
            assert f[k].tobytes() == f1[k][info["gpoint"]].tobytes(), (case, r, k)


def test_a_piece_refuses_whole_cycles_and_a_mesh_the_piece_calls():
    """Whole cycles on a piece (no exchange) and piece steps on a mesh object
    are state errors, not silent wrong answers."""
    d = pb.Deck(text=sedov(8, tstop=0.01))
    m = pb.Mesh(deck=d)
    h = pb.Hydro(m.piece(2, 0), d.params())
    for call in (h.cycle, lambda: h.run(), lambda: h.enqueue(1), lambda: h.time_cycles(1)):
        with pytest.raises(pb.PntError) as e:
            call()
        assert e.value.status == pb.PNT_ERR_STATE
    h.close()
    whole = pb.Hydro(m, d.params())
    with pytest.raises(pb.PntError) as e:
        pb.check(pb.lib.pnt_hydro_piece_forces(whole.h))
    assert e.value.status == pb.PNT_ERR_STATE
    whole.close()


@pytest.mark.parametrize("case,npieces", [("sedov-fp64", 2), ("sedov-fp64-3", 3), ("noh-pie-fp64", 4),
                                          ("sedov-mixed", 3), ("sedov-learned", 2)])
def test_native_pieces_match_the_single_piece_run_bitwise(case, npieces, tmp_path):
    """pnt_pieces (one process; peer copies, host reductions), gathered back
    to the whole mesh: equal to the single-piece run bit for bit."""
    text, precision, _ = CASES[case]
    s1, f1 = single(text, precision)
    d = _deck(text, precision)
    m = pb.Mesh(deck=d)
    ps = pb.Pieces(m, d.params(), npieces, devices=(0,))
    if precision == "learned":
        ps.set_closure(pb.Closure(path=CLOSURE))
    s = ps.run()
    assert s["cycle"] == s1["cycle"] and s["time"] == s1["time"] and s["done"] == 1, (case, s, s1)
    for k in ZONE + POINT:
        assert ps.download(k).tobytes() == f1[k].tobytes(), (case, k)
    ps.write_xy(str(tmp_path / "p.xy"))
    assert (tmp_path / "p.xy").stat().st_size > 0
    ps.close()


def _graph_rank(rank, port, text, precision, cycles_per_graph, out):
    import torch
    import torch.distributed as dist
    from pennant_b200.pieces import PieceHydro
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device("cuda", 0))
    try:
        d = _deck(text, precision)
        clo = pb.Closure(path=CLOSURE) if precision == "learned" else None
        ph = PieceHydro(pb.Mesh(deck=d), d.params(), device=0, closure=clo)
        ph.cycle()                       # one eager cycle first, as bench.py's warm-up does
        ph.capture(cycles_per_graph)
        for _ in range(100000):
            ph.replay()
            if ph.scalars()["done"]:
                break
        out[0] = (ph.scalars(), ph.fields(ZONE + POINT))
        ph.close()                       # releases the graph before the group goes
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(600)
@pytest.mark.parametrize("case", ["sedov-fp64", "sedov-learned"])
def test_graph_captured_piece_cycles_match_the_single_piece_run_bitwise(case):
    """One rank over NCCL: whole piece cycles (kernels, halo send/receive,
    both reductions) captured in a CUDA graph and replayed until the run
    ends give the single-piece run bit for bit (cycles the graph runs past
    the end are skipped on the device)."""
    text, precision, _ = CASES[case]
    s1, f1 = single(text, precision)
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_graph_rank, args=(_port(), text, precision, 7, out), nprocs=1, join=True,
                       start_method="spawn")
    s, f = out[0]
    assert s["cycle"] == s1["cycle"] and s["time"] == s1["time"] and s["done"] == 1, (case, s, s1)
    for k in ZONE + POINT:
        assert f[k].tobytes() == f1[k].tobytes(), (case, k)
