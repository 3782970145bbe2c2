"""Parity of the CUDA cycle against the CPU oracle (needs a GPU).

The FP64 path is built to reproduce a serial run of the reference bit for
bit: every state field and the dt sequence are compared with exact equality
after every cycle.  The accuracy bound of the FP64 path is 1e-11 relative per field after
the run; bitwise equality is the stronger claim tested here, and the
fingerprint test measures the relative error explicitly.
"""
import hashlib
import json

import numpy as np
import pytest

from conftest import deck, golden
from oracle import Oracle
import pennant_b200 as pb

pytestmark = pytest.mark.gpu

STATE = ("px", "pu", "zr", "ze", "zp", "zetot", "zvol", "zwrate")
REL_TOL = 1e-11   # accuracy bound of the FP64 path


def make_pair(path=None, text=None, **overrides):
    o = Oracle(path=path, text=text)
    d = pb.Deck(path=path, text=text)
    for k, v in overrides.items():
        d.set(k, v)
    h = pb.Hydro(pb.Mesh(deck=d), d.params())
    return o, h


def assert_state_equal(o, h, where=""):
    for k in STATE:
        a, b = o.field(k), h.download(k)
        if a.tobytes() != b.tobytes():
            rel = np.abs(a - b) / np.maximum(np.abs(a), 1e-300)
            i = np.unravel_index(np.argmax(rel), rel.shape)
            raise AssertionError(f"{where} field {k} differs: max rel {rel[i]:.3e} at {i}, "
                                 f"{int((a != b).sum())} of {a.size} values")


@pytest.mark.parametrize("name", ["sedov.pnt", "sedovsmall.pnt", "noh.pnt", "nohsmall.pnt",
                                  "leblanc.pnt"])
def test_cycle_by_cycle_bitwise(name):
    o, h = make_pair(golden(name))
    assert_state_equal(o, h, "init")
    for c in range(10):
        assert o.cycle() == 0
        s = h.cycle()
        assert s["cycle"] == o.num("cycle") == c + 1
        for k in ("time", "dt", "dtrec", "dtnew", "dvovmax"):
            assert s[k] == o.scalar(k), (c, k, s[k], o.scalar(k))
        assert_state_equal(o, h, f"cycle {c + 1}")
    assert s["done"] == 1   # cstop 10


def test_sedov_golden_xy_through_gpu(tmp_path):
    """The GPU run of the reference deck writes the same .xy bytes as the
    oracle (which is pinned to the reference's gold)."""
    o, h = make_pair(golden("sedov.pnt"))
    assert o.run() == 0
    s = h.run()
    assert s["cycle"] == 10
    o.write_xy(str(tmp_path / "o.xy"))
    h.write_xy(str(tmp_path / "g.xy"))
    assert (tmp_path / "o.xy").read_bytes() == (tmp_path / "g.xy").read_bytes()
    o.write_gold(str(tmp_path / "o"))
    h.write_gold(str(tmp_path / "g"))
    for ext in ("geo", "zr", "ze", "zp"):
        assert (tmp_path / f"o.{ext}").read_bytes() == (tmp_path / f"g.{ext}").read_bytes(), ext


def test_sedov48_to_t1_graph_path_bitwise():
    """CPU-runnable case (48^2 Sedov to t = 1.0) through the CUDA-graph run
    loop, reports at cycle 1 and every dtreport cycles."""
    o, h = make_pair(deck("sedov48.pnt"))
    assert o.run() == 0
    seen = []
    s = h.run(report=lambda sc, us: seen.append(sc["cycle"]))
    assert s["cycle"] == o.num("cycle") and s["done"] == 1
    assert s["time"] == o.scalar("time") == 1.0
    assert seen[0] == 1 and all(c % 100 == 0 for c in seen[1:])
    assert_state_equal(o, h, "t=1")


def test_pie_noh_to_stop_bitwise():
    o, h = make_pair(golden("noh.pnt"), cstop=200)
    o2 = Oracle(text=open(golden("noh.pnt")).read().replace("cstop   10", "cstop   200"))
    assert o2.run() == 0
    s = h.run()
    assert s["cycle"] == o2.num("cycle") == 200
    assert_state_equal(o2, h, "noh 200")


def test_tstop_termination_matches_oracle():
    text = open(golden("sedovsmall.pnt")).read().replace("cstop   10", "cstop   100000").replace(
        "tstop   1.0", "tstop   0.05")
    o, h = make_pair(text=text)
    assert o.run() == 0
    s = h.run()
    assert s["cycle"] == o.num("cycle")
    assert s["time"] == o.scalar("time")
    assert not (s["time"] < 0.05)
    assert_state_equal(o, h, "tstop")
    # further calls are no-ops once done
    s2 = h.cycle()
    assert s2["cycle"] == s["cycle"]


def test_max_cycles_and_enqueue_semantics():
    o, h = make_pair(deck("sedov48.pnt"))
    s = h.run(max_cycles=7)
    assert s["cycle"] == 7 and s["done"] == 0
    h.enqueue(33)
    h.synchronize()
    assert h.scalars()["cycle"] == 40
    assert o.run(40) == 0
    assert_state_equal(o, h, "40")


def test_negative_volume_reports_badsides_like_oracle():
    """A deposit far too strong for dtinit inverts zones on the first cycle;
    both paths stop with the bad-side error (the reference exits,
    Mesh.cc:1531-1550)."""
    text = open(golden("sedovsmall.pnt")).read().replace("dtinit  0.0025", "dtinit  0.5")
    o, h = make_pair(text=text)
    st = 0
    while not o.done:
        st = o.cycle()
        if st:
            break
    assert st == 3
    with pytest.raises(pb.PntError) as e:
        h.run()
    assert e.value.status == pb.PNT_ERR_BADSIDES
    s = h.scalars()
    assert s["status"] == pb.PNT_ERR_BADSIDES and s["done"] == 1
    assert s["cycle"] == o.num("cycle") and s["nbad"] == o.num("nbad")


def test_upload_download_round_trip():
    o, h = make_pair(golden("sedovsmall.pnt"))
    pu = h.download("pu")
    pu[:, :] = 0.25
    h.upload("pu", pu)
    np.testing.assert_array_equal(h.download("pu"), pu)
    with pytest.raises(pb.PntError):
        h.upload("smf", np.zeros(h.mesh.nums))
    wrong = np.empty(3)
    assert pb.lib.pnt_hydro_download(h.h, pb.FIELDS["zr"], wrong.ctypes.data, wrong.nbytes) == \
        pb.PNT_ERR_INVALID_ARG


def _fp_compare(fp, h, name):
    for k, ref in fp["fields"].items():
        a = h.download(k).reshape(-1)
        sha = hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()
        vals = np.array([float.fromhex(v) for v in ref["val"]])
        got = a[np.array(ref["idx"])]
        rel = np.abs(got - vals) / np.maximum(np.abs(vals), 1e-300)
        assert rel.max() <= REL_TOL, (name, k, rel.max())
        assert abs(a.sum() - ref["sum"]) <= REL_TOL * max(ref["l1"], 1e-300), (name, k)
        assert sha == ref["sha256"], (name, k, "not bit-identical (within 1e-11 on samples)")


@pytest.mark.slow
def test_sedov480_to_t1_matches_oracle_fingerprint():
    """480^2 Sedov to t = 1.0 (the FP64 drop-in case) against the oracle's
    final state, generated by tests/golden/make_fingerprint.py."""
    fp_path = golden("sedov480_fingerprint.json")
    fp = json.load(open(fp_path))
    d = pb.Deck(path=deck("sedov480.pnt"))
    h = pb.Hydro(pb.Mesh(deck=d), d.params())
    s = h.run()
    assert s["cycle"] == fp["cycle"]
    assert s["time"] == float.fromhex(fp["time"])
    _fp_compare(fp, h, "sedov480")


@pytest.mark.slow
@pytest.mark.parametrize("fp_name,deck_name", [("leblanc2880x288_c400_fingerprint.json", "leblanc2880x288.pnt"),
                                               ("sedov1920_c100_fingerprint.json", "sedov1920.pnt")])
def test_full_size_meshes_match_oracle_fingerprints(fp_name, deck_name):
    """The FP64 cycle on the full-size meshes of the mixed-precision and
    learned-closure workloads (2880x288 Leblanc, 1920^2 Sedov), from the
    deck's initial state for the fingerprint's cycles, bit for bit against
    the oracle's final state (tests/golden/make_fingerprint.py with cstop)."""
    fp = json.load(open(golden(fp_name)))
    d = pb.Deck(path=deck(deck_name))
    d.set("cstop", fp["cstop"])
    h = pb.Hydro(pb.Mesh(deck=d), d.params())
    s = h.run()
    assert s["cycle"] == fp["cycle"] == fp["cstop"]
    assert s["time"] == float.fromhex(fp["time"])
    _fp_compare(fp, h, deck_name)
    h.close()


def test_copy_state_restarts_bitwise():
    """pnt_hydro_copy_state: an object restarted from another's state
    continues exactly as the source does (same fields after the same cycles),
    and refuses objects of another mesh."""
    text = open(golden("sedov.pnt")).read().replace("cstop   10", "cstop   60")
    d = pb.Deck(text=text)
    src = pb.Hydro(pb.Mesh(deck=d), d.params())
    src.run(max_cycles=25)
    dst = pb.Hydro(pb.Mesh(deck=pb.Deck(text=text)), d.params())
    dst.copy_state_from(src)
    assert dst.scalars()["cycle"] == 25 and dst.scalars()["time"] == src.scalars()["time"]
    s1, s2 = src.run(), dst.run()
    assert s1["cycle"] == s2["cycle"] == 60 and s1["time"] == s2["time"]
    for k in ("px", "pu", "zr", "ze", "zp", "zetot", "zvol", "zwrate"):
        assert src.download(k).tobytes() == dst.download(k).tobytes(), k
    other = pb.Hydro(pb.Mesh(deck=pb.Deck(path=golden("sedovsmall.pnt"))), d.params())
    with pytest.raises(pb.PntError):
        other.copy_state_from(src)


def test_check_finite_finds_the_first_non_finite_value():
    """pnt_hydro_check_finite (the NAN_CHECK analogue): none after a clean
    run, then the first field in field order and its smallest bad index."""
    d = pb.Deck(path=golden("sedov.pnt"))
    h = pb.Hydro(pb.Mesh(deck=d), d.params())
    h.run()
    assert h.check_finite() == (None, -1)
    ze = h.download("ze")
    ze[90] = np.inf
    ze[37] = np.nan
    h.upload("ze", ze)
    assert h.check_finite() == ("ze", 37)
    px = h.download("px")
    px[5, 1] = -np.inf
    h.upload("px", px)
    assert h.check_finite() == ("px", 5)
    h.close()
