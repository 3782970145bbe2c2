"""Batched meshes (needs a GPU): every instance of a batch must be bit-identical
to its own single-mesh run (itself bit-identical to the CPU oracle),
whatever the work-list shape and after the autotuner has run."""
import sys

import numpy as np
import pytest

from conftest import DECKS, golden
from oracle import Oracle
import pennant_b200 as pb

sys.path.insert(0, DECKS)
from make_decks import sedov, sedov_batch  # noqa: E402

pytestmark = pytest.mark.gpu

STATE = ("px", "pu", "zr", "ze", "zetot", "zvol", "zwrate")


def instance_decks():
    rng = np.random.default_rng(7)
    texts = []
    for n, tstop in ((16, 0.05), (24, 0.02), (33, 0.05), (20, 0.01), (40, 0.03)):
        texts.append(sedov(n, e0=float(rng.uniform(0.1, 1.0)), tstop=tstop,
                           gamma=float(rng.uniform(1.4, 5 / 3))))
    # a pie mesh among the quads: the general (non-quad) path and 3-sided zones
    texts.insert(2, open(golden("nohsmall.pnt")).read().replace("cstop   10", "cstop   60"))
    return texts


def make_batch(texts):
    decks = [pb.Deck(text=t) for t in texts]
    meshes = [pb.Mesh(deck=d) for d in decks]
    return pb.Batch(meshes, [d.params() for d in decks]), meshes, decks


def single_runs(texts):
    out = []
    for t in texts:
        d = pb.Deck(text=t)
        h = pb.Hydro(pb.Mesh(deck=d), d.params())
        s = h.run()
        out.append((s, {k: h.download(k) for k in STATE}))
        h.close()
    return out


def check_batch(b, ref):
    for i, (s, fields) in enumerate(ref):
        sb = b.scalars(i)
        assert sb["done"] == 1 and sb["status"] == 0, (i, sb)
        assert sb["cycle"] == s["cycle"] and sb["time"] == s["time"], (i, sb, s)
        for k in STATE:
            assert b.download(i, k).tobytes() == fields[k].tobytes(), (i, k)


def test_batch_matches_single_mesh_runs_bitwise():
    texts = instance_decks()
    ref = single_runs(texts)
    b, _, _ = make_batch(texts)
    assert b.run() == 0
    check_batch(b, ref)
    # and two of them against the oracle directly
    for i in (0, 2):
        o = Oracle(text=texts[i])
        assert o.run() == 0
        for k in ("zr", "px"):
            assert o.field(k).tobytes() == ref[i][1][k].tobytes()


@pytest.mark.parametrize("shape", [(64, 2), (128, 4), (1024, 3)])
def test_batch_results_do_not_depend_on_shape(shape):
    texts = instance_decks()
    ref = single_runs(texts)
    b, _, _ = make_batch(texts)
    b.set_shape(*shape)
    assert b.shape() == shape
    assert b.run() == 0
    check_batch(b, ref)


def test_batch_autotuner_picks_a_shape_and_keeps_results():
    texts = instance_decks()
    ref = single_runs(texts)
    b, _, _ = make_batch(texts)
    zpt, cps, ms = b.tune(2)
    assert zpt % 64 == 0 and 1 <= cps <= 8 and ms > 0
    assert b.shape() == (zpt, cps)
    assert b.run() == 0
    check_batch(b, ref)


def test_batch_partial_run_and_instances_finishing_early():
    texts = instance_decks()
    b, _, _ = make_batch(texts)
    left = b.run(max_cycles=5)
    assert left == len(texts)
    assert all(b.scalars(i)["cycle"] == 5 for i in range(len(texts)))
    b.run()
    cycles = [b.scalars(i)["cycle"] for i in range(len(texts))]
    assert len(set(cycles)) > 1   # uneven meshes and stop times finish apart


@pytest.mark.timeout(900)
def test_seeded_batch_workload_subset_matches_single_runs_bitwise():
    """The first 32 instances of the seeded 256-instance Sedov batch (sizes
    log-uniform in [32, 512], E0 in [0.1, 1], gamma in [1.4, 5/3], to
    t = 0.5) with the autotuned shape: every instance ends exactly as its
    own single-mesh run."""
    insts = sedov_batch(256)[:32]
    texts = [i["text"] for i in insts]
    assert min(i["n"] for i in insts) < 64 and max(i["n"] for i in insts) > 256
    ref = single_runs(texts)
    b, _, _ = make_batch(texts)
    zpt, cps, _ = b.tune(2)
    b.close()
    b, _, _ = make_batch(texts)
    b.set_shape(zpt, cps)
    assert b.run() == 0
    check_batch(b, ref)
    assert all(abs(b.scalars(i)["time"] - 0.5) < 1e-12 for i in range(len(texts)))


def _with_precision(texts, precision):
    out = []
    for t in texts:
        d = pb.Deck(text=t)
        d.set("precision", precision)
        out.append(d)
    return out


def test_mixed_batch_matches_single_mixed_runs_bitwise():
    """The mixed-precision cycle in a batch: every instance (quad and pie
    meshes together) ends exactly as its own single-mesh mixed run."""
    texts = instance_decks()
    ref = []
    for d in _with_precision(texts, "mixed"):
        h = pb.Hydro(pb.Mesh(deck=d), d.params())
        s = h.run()
        ref.append((s, {k: h.download(k) for k in STATE}))
        h.close()
    decks = _with_precision(texts, "mixed")
    b = pb.Batch([pb.Mesh(deck=d) for d in decks], [d.params() for d in decks])
    assert b.run() == 0
    check_batch(b, ref)
    # and differs from the FP64 batch: the instances really ran the mixed cycle
    fp = single_runs(texts[:1])
    assert b.download(0, "ze").tobytes() != fp[0][1]["ze"].tobytes()


def test_batch_rejects_learned_and_mixed_precisions():
    d = pb.Deck(text=sedov(16, tstop=0.01))
    d.set("precision", "learned")
    with pytest.raises(pb.PntError) as e:
        pb.Batch([pb.Mesh(deck=d)], [d.params()])
    assert e.value.status == pb.PNT_ERR_UNSUPPORTED
    d1, d2 = pb.Deck(text=sedov(16, tstop=0.01)), pb.Deck(text=sedov(16, tstop=0.01))
    d2.set("precision", "mixed")
    with pytest.raises(pb.PntError) as e:
        pb.Batch([pb.Mesh(deck=d1), pb.Mesh(deck=d2)], [d1.params(), d2.params()])
    assert e.value.status == pb.PNT_ERR_UNSUPPORTED
