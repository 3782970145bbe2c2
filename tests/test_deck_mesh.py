"""Host-side parity (no GPU): deck parsing, mesh generation, derived maps.

The product's mesh builder (libpennant_b200.so, C++) and the oracle (C)
restate GenMesh independently; connectivity, coordinates, boundary point
sets and the point->corner CSR must agree bit for bit.
"""
import os

import numpy as np
import pytest

from conftest import golden
from oracle import Oracle, OracleError
import pennant_b200 as pb

DECKS = ["sedov.pnt", "sedovsmall.pnt", "noh.pnt", "nohsmall.pnt", "leblanc.pnt", "nohsquare.pnt"]


def test_abi_version():
    assert pb.lib.pnt_abi_version() == 1


# ---------------------------------------------------------------- deck
def test_deck_values_and_defaults():
    d = pb.Deck(text="# comment\ncstop 10\n  tstop   1.0e-1 trailing\nmeshparams 4 5 1.5 2.0\n"
                     "meshtype rect\n\nbcx 0.0 1.5\nq1 .25\n")
    assert d.get_int("cstop", 0) == 10
    assert d.get_double("tstop", 0) == pytest.approx(0.1)
    assert d.get_double_list("meshparams") == [4.0, 5.0, 1.5, 2.0]
    assert d.get_string("meshtype") == "rect"
    assert d.get_double_list("missing") is None
    assert d.get_int("missing", 7) == 7
    p = d.params()
    assert (p.cstop, p.nbcx, p.nbcy) == (10, 2, 0)
    assert p.q1 == 0.25 and p.q2 == 2.0 and p.alfa == 0.5     # QCS/TTS defaults
    assert p.cfl == 0.6 and p.cflv == 0.1 and p.dtfac == 1.2  # Hydro/Driver defaults
    assert p.gamma == pytest.approx(5.0 / 3.0)


def test_deck_get_int_truncates_like_stream_extraction():
    d = pb.Deck(text="cstop 12.7\n")
    assert d.get_int("cstop", 0) == 12


def test_deck_duplicate_key_is_an_error():
    with pytest.raises(pb.PntError) as e:
        pb.Deck(text="cstop 1\ncstop 2\n")
    assert e.value.status == pb.PNT_ERR_DECK
    with pytest.raises(OracleError):
        Oracle(text="cstop 1\ncstop 2\nmeshtype rect\nmeshparams 2\n")


def test_deck_unterminated_last_line_is_dropped():
    # InputFile's getline loop stops at EOF before storing the last line
    d = pb.Deck(text="cstop 5\ntstop 2.0")
    assert d.get_double("tstop", -1.0) == -1.0


def test_deck_needs_stop_condition():
    d = pb.Deck(text="meshtype rect\nmeshparams 2\n")
    with pytest.raises(pb.PntError) as e:
        d.params()
    assert e.value.status == pb.PNT_ERR_DECK


def test_deck_missing_file():
    with pytest.raises(pb.PntError) as e:
        pb.Deck(path="/nonexistent/deck.pnt")
    assert e.value.status == pb.PNT_ERR_DECK


@pytest.mark.parametrize("text,status", [
    ("cstop 1\nmeshparams 2\n", pb.PNT_ERR_DECK),                      # no meshtype
    ("cstop 1\nmeshtype tri\nmeshparams 2\n", pb.PNT_ERR_DECK),        # invalid meshtype
    ("cstop 1\nmeshtype rect\n", pb.PNT_ERR_DECK),                     # no meshparams
    ("cstop 1\nmeshtype rect\nmeshparams 1 2 3 4 5\n", pb.PNT_ERR_DECK),
    ("cstop 1\nmeshtype rect\nmeshparams 0 2\n", pb.PNT_ERR_DECK),
    ("cstop 1\nmeshtype pie\nmeshparams 4 4 360\n", pb.PNT_ERR_DECK),  # theta must be < 360
    ("cstop 1\nmeshtype hex\nmeshparams 4\n", pb.PNT_ERR_UNSUPPORTED),
])
def test_mesh_generate_rejects_bad_decks(text, status):
    d = pb.Deck(text=text)
    with pytest.raises(pb.PntError) as e:
        pb.Mesh(deck=d)
    assert e.value.status == status


def test_subregion_needs_four_values():
    d = pb.Deck(text="cstop 1\nmeshtype rect\nmeshparams 2\nsubregion 0 1 0\n")
    with pytest.raises(pb.PntError):
        d.params()


# ---------------------------------------------------------------- mesh
@pytest.mark.parametrize("name", DECKS)
def test_mesh_connectivity_bit_exact_vs_oracle(name):
    d = pb.Deck(path=golden(name))
    m = pb.Mesh(deck=d)
    o = Oracle(golden(name))
    assert (m.nump, m.numz, m.nums) == (o.nump, o.numz, o.nums)
    for k in ("znump", "mapsp1", "mapsp2", "mapsz", "mapss3", "mapss4"):
        np.testing.assert_array_equal(m.array(k), o.field(k), err_msg=k)
    px = m.array("px")
    assert px.tobytes() == o.field("px").tobytes()


def test_rect_numbering_matches_reference_layout():
    m = pb.Mesh(deck=pb.Deck(text="cstop 1\nmeshtype rect\nmeshparams 3 2 3.0 2.0\n"))
    assert (m.nump, m.numz, m.nums) == (12, 6, 24)
    # zone 4 = row 1, col 1: sides bottom, right, top, left
    np.testing.assert_array_equal(m.array("mapsp1")[16:20], [5, 6, 10, 9])
    np.testing.assert_array_equal(m.array("mapsp2")[16:20], [6, 10, 9, 5])
    np.testing.assert_array_equal(m.array("px")[6], [2.0, 1.0])


@pytest.mark.parametrize("params", ["3 2 3.0 2.0", "1 5", "7 1", "16 9 1.0 2.0"])
def test_rect_point_indices_follow_from_the_zone_index(params):
    """The FP64 pass A and the batch read a rect mesh's points without
    mapsp1: side 4z + k of zone z = (i, j) starts at point
    j (nzx + 1) + i + {0, 1, nzx + 2, nzx + 1}[k].  Checked against the
    mesh's own mapsp1 for every zone."""
    m = pb.Mesh(deck=pb.Deck(text=f"cstop 1\nmeshtype rect\nmeshparams {params}\n"))
    nzx = int(params.split()[0])
    z = np.arange(m.numz)
    p0 = (z // nzx) * (nzx + 1) + z % nzx
    want = p0[:, None] + np.array([0, 1, nzx + 2, nzx + 1])[None, :]
    np.testing.assert_array_equal(m.array("mapsp1").reshape(-1, 4), want)


@pytest.mark.parametrize("params", ["3 2 3.0 2.0", "1 5", "7 1", "16 9 1.0 2.0"])
def test_rect_point_corners_follow_from_the_point_index(params):
    """The point passes read a rect mesh's corners without the CSR: point
    (i, j) gathers side 2 of the zone below-left, 3 of the zone below, 1 of
    the zone to the left and 0 of its own zone, those that exist, in that
    order.  Checked against the mesh's CSR (ascending side order) for every
    point."""
    m = pb.Mesh(deck=pb.Deck(text=f"cstop 1\nmeshtype rect\nmeshparams {params}\n"))
    nzx = int(params.split()[0])
    nzy = m.numz // nzx
    off, sides = m.point_corners()
    for p in range(m.nump):
        j, i = divmod(p, nzx + 1)
        want = []
        if j > 0:
            if i > 0:
                want.append(4 * ((j - 1) * nzx + i - 1) + 2)
            if i < nzx:
                want.append(4 * ((j - 1) * nzx + i) + 3)
        if j < nzy:
            if i > 0:
                want.append(4 * (j * nzx + i - 1) + 1)
            if i < nzx:
                want.append(4 * (j * nzx + i))
        assert list(sides[off[p]:off[p + 1]]) == want, (p, i, j)


def test_pie_mesh_structure():
    m = pb.Mesh(deck=pb.Deck(path=golden("nohsmall.pnt")))   # pie 2 x 20
    z = m.array("znump")
    assert (z[:2] == 3).all() and (z[2:] == 4).all()
    assert m.nums == 3 * 2 + 4 * 2 * 19
    assert m.nump == 3 * 20 + 1
    # every triangle touches the origin
    sp1 = m.array("mapsp1")
    assert (sp1[[0, 3]] == 0).all()


@pytest.mark.parametrize("name", ["sedov.pnt", "noh.pnt", "leblanc.pnt"])
def test_point_corner_csr(name):
    m = pb.Mesh(deck=pb.Deck(path=golden(name)))
    off, sides = m.point_corners()
    sp1 = m.array("mapsp1")
    assert off[0] == 0 and off[-1] == m.nums
    ref_order = np.argsort(sp1, kind="stable")      # ascending side within each point
    np.testing.assert_array_equal(sides, ref_order)
    np.testing.assert_array_equal(np.diff(off), np.bincount(sp1, minlength=m.nump))


def test_mesh_invariants_circulate():
    m = pb.Mesh(deck=pb.Deck(path=golden("noh.pnt")))
    sp1, sp2, ss4 = m.array("mapsp1"), m.array("mapsp2"), m.array("mapss4")
    np.testing.assert_array_equal(sp2, sp1[ss4])


def test_mesh_create_from_arrays_round_trip():
    src = pb.Mesh(deck=pb.Deck(path=golden("nohsmall.pnt")))
    desc = {k: src.array(k) for k in ("znump", "mapsp1", "mapsp2", "mapsz", "mapss3", "mapss4")}
    desc["px"] = src.array("px").reshape(-1)
    m = pb.Mesh(desc=desc)
    for k in ("znump", "mapsp1", "mapss4"):
        np.testing.assert_array_equal(m.array(k), src.array(k))


def test_mesh_create_rejects_broken_connectivity():
    src = pb.Mesh(deck=pb.Deck(path=golden("sedovsmall.pnt")))
    desc = {k: src.array(k) for k in ("znump", "mapsp1", "mapsp2", "mapsz", "mapss3", "mapss4")}
    desc["px"] = src.array("px").reshape(-1)
    bad = dict(desc)
    bad["mapss4"] = desc["mapss4"].copy()
    bad["mapss4"][5] = 0
    with pytest.raises(pb.PntError) as e:
        pb.Mesh(desc=bad)
    assert e.value.status == pb.PNT_ERR_INVALID_ARG
    bad = dict(desc)
    bad["mapsp1"] = desc["mapsp1"].copy()
    bad["mapsp1"][3] = 10 ** 6
    with pytest.raises(pb.PntError):
        pb.Mesh(desc=bad)
    bad = dict(desc)
    bad["znump"] = desc["znump"].copy()
    bad["znump"][0] = 5
    with pytest.raises(pb.PntError) as e:
        pb.Mesh(desc=bad)
    assert e.value.status in (pb.PNT_ERR_UNSUPPORTED, pb.PNT_ERR_INVALID_ARG)


def test_inverted_initial_mesh_reports_bad_sides():
    src = pb.Mesh(deck=pb.Deck(path=golden("sedovsmall.pnt")))
    desc = {k: src.array(k) for k in ("znump", "mapsp1", "mapsp2", "mapsz", "mapss3", "mapss4")}
    px = src.array("px")
    px[:, 1] = -px[:, 1]   # mirror in y: zones turn clockwise, r stays >= 0
    desc["px"] = px.reshape(-1)
    with pytest.raises(pb.PntError) as e:
        pb.Mesh(desc=desc)
    assert e.value.status == pb.PNT_ERR_BADSIDES


@pytest.mark.parametrize("name", ["sedov.pnt", "noh.pnt", "leblanc.pnt", "nohsquare.pnt"])
def test_bc_point_sets_match_oracle(name):
    """Boundary point lists (HydroBC) are the points within 1e-12 of each
    plane, ascending; the oracle builds them the reference's way."""
    o = Oracle(golden(name))
    d = pb.Deck(path=golden(name))
    p = d.params()
    px = pb.Mesh(deck=d).array("px")
    planes = [(0, v) for v in p.bcx[:p.nbcx]] + [(1, v) for v in p.bcy[:p.nbcy]]
    assert o.num("nbc") == len(planes)
    for b, (axis, bound) in enumerate(planes):
        mine = np.nonzero(np.abs(px[:, axis] - bound) < 1e-12)[0]
        np.testing.assert_array_equal(mine, o.field(f"bcpts{b}"))


def test_committed_decks_are_what_make_decks_writes():
    """The benchmark decks in the package are exactly make_decks.py's output
    (no hand edits), and the batch workload is reproducible from its seed:
    256 instances, N in [32, 512], E0 in [0.1, 1], gamma in [1.4, 5/3]."""
    import sys
    from conftest import DECKS as DECK_DIR
    sys.path.insert(0, DECK_DIR)
    import make_decks
    for name, text in make_decks.DECKS.items():
        with open(os.path.join(DECK_DIR, name)) as f:
            assert f.read() == text, name
    a, b = make_decks.sedov_batch(), make_decks.sedov_batch()
    assert a == b and len(a) == 256
    assert all(32 <= i["n"] <= 512 and 0.1 <= i["e0"] <= 1.0 and 1.4 <= i["gamma"] <= 5 / 3 for i in a)
    assert len({i["n"] for i in a}) > 50   # uneven sizes


@pytest.mark.parametrize("name", ["leblanc.pnt", "leblancbig.pnt", "noh.pnt", "nohpoly.pnt", "nohsmall.pnt",
                                  "nohsquare.pnt", "sedov.pnt", "sedovbig.pnt", "sedovsmall.pnt"])
def test_every_reference_deck_is_handled_like_the_oracle(name):
    """Each deck of the reference's test/ directory: the library and the
    oracle build the same mesh and parameters, or both refuse it with the
    same status (nohpoly's hex mesh: unsupported, as the reference's parallel
    generator asserts)."""
    try:
        o, oerr = Oracle(golden(name)), None
    except OracleError as e:
        o, oerr = None, e
    try:
        d = pb.Deck(path=golden(name))
        m, perr = pb.Mesh(deck=d), None
    except pb.PntError as e:
        m, perr = None, e
    if o is None or m is None:
        assert o is None and m is None, (name, oerr, perr)
        assert perr.status == oerr.status == pb.PNT_ERR_UNSUPPORTED, (name, oerr, perr)
        return
    assert (m.nump, m.numz, m.nums) == (o.nump, o.numz, o.nums)
    for k in ("znump", "mapsp1", "mapsp2", "mapsz", "mapss3", "mapss4"):
        np.testing.assert_array_equal(m.array(k), o.field(k), err_msg=k)
    assert m.array("px").tobytes() == o.field("px").tobytes()
    p = d.params()
    assert p.cstop == o.num("cstop") and p.dtreport == o.num("dtreport")
    for k in ("tstop", "dtmax", "dtinit", "dtfac", "cfl", "cflv", "rinit", "einit", "rinitsub", "einitsub",
              "uinitradial", "gamma", "pgas_ssmin", "alfa", "tts_ssmin", "qgamma", "q1", "q2"):
        assert getattr(p, k) == o.scalar(k), k
