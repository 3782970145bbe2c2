"""Differential tests (no GPU) over random small decks: the product's deck
parser and mesh builder (libpennant_b200.so, C++) against the oracle's
independent C restatement of InputFile and GenMesh.  For every generated
deck both accept or both reject it, and when they accept, the connectivity,
the coordinates (bitwise) and the parameters agree.  Random junk text never
crashes the parser: it answers with a status."""
import numpy as np
from hypothesis import HealthCheck, event, given, settings
from hypothesis import strategies as st

from oracle import Oracle, OracleError
import pennant_b200 as pb

SETTINGS = settings(max_examples=60, deadline=None, suppress_health_check=[HealthCheck.too_slow])

extent = st.floats(min_value=0.05, max_value=20.0, allow_nan=False, allow_infinity=False)


@st.composite
def mesh_decks(draw):
    kind = draw(st.sampled_from(["rect", "rect", "pie"]))
    nx = draw(st.integers(1, 14))
    ny = draw(st.integers(1, 14))
    if kind == "rect":
        params = f"{nx} {ny} {draw(extent)!r} {draw(extent)!r}"
    else:
        theta = draw(st.floats(min_value=1.0, max_value=359.0, allow_nan=False))
        params = f"{nx} {ny} {theta!r} {draw(extent)!r}"
    lines = [f"cstop {draw(st.integers(1, 50))}", f"meshtype {kind}", f"meshparams {params}"]
    if draw(st.booleans()):
        lines.append(f"dtreport {draw(st.integers(1, 1000))}")
    if draw(st.booleans()):
        lines.append(f"tstop {draw(extent)!r}")
    if draw(st.booleans()):
        a, b = sorted(draw(st.lists(extent, min_size=2, max_size=2)))
        c, d = sorted(draw(st.lists(extent, min_size=2, max_size=2)))
        lines.append(f"subregion {a!r} {b!r} {c!r} {d!r}")
    for key in ("dtinit", "dtmax", "dtfac", "cfl", "cflv", "q1", "q2", "qgamma", "alfa", "ssmin", "gamma", "rinit",
                "einit", "rinitsub", "einitsub", "uinitradial"):
        if draw(st.booleans()):
            lines.append(f"{key} {draw(extent)!r}")
    for key in ("bcx", "bcy"):
        if draw(st.booleans()):
            vals = draw(st.lists(st.floats(min_value=0.0, max_value=20.0, allow_nan=False), min_size=1, max_size=3))
            lines.append(f"{key} " + " ".join(repr(v) for v in vals))
    order = draw(st.permutations(lines))
    return "\n".join(order) + "\n"


def _oracle(text):
    try:
        return Oracle(text=text), None
    except OracleError as e:
        return None, e


def _product(text):
    try:
        d = pb.Deck(text=text)
        return d, pb.Mesh(deck=d), None
    except pb.PntError as e:
        return None, None, e


@SETTINGS
@given(mesh_decks())
def test_random_decks_build_the_same_mesh_as_the_oracle(text):
    o, oerr = _oracle(text)
    d, m, perr = _product(text)
    assert (o is None) == (m is None), (text, oerr, perr)
    event("rejected by both" if m is None else "accepted by both")
    if m is None:
        return
    assert (m.nump, m.numz, m.nums) == (o.nump, o.numz, o.nums), text
    for k in ("znump", "mapsp1", "mapsp2", "mapsz", "mapss3", "mapss4"):
        np.testing.assert_array_equal(m.array(k), o.field(k), err_msg=f"{k}\n{text}")
    assert m.array("px").tobytes() == o.field("px").tobytes(), text
    p = d.params()
    assert p.cstop == o.num("cstop") and p.dtreport == o.num("dtreport"), text
    for k in ("tstop", "dtmax", "dtinit", "dtfac", "cfl", "cflv", "rinit", "einit", "rinitsub", "einitsub",
              "uinitradial", "gamma", "pgas_ssmin", "alfa", "tts_ssmin", "qgamma", "q1", "q2"):
        assert getattr(p, k) == o.scalar(k), (k, getattr(p, k), o.scalar(k), text)
    # the boundary point sets
    px = m.array("px")
    planes = [(0, v) for v in p.bcx[:p.nbcx]] + [(1, v) for v in p.bcy[:p.nbcy]]
    assert o.num("nbc") == len(planes), text
    for b, (axis, bound) in enumerate(planes):
        np.testing.assert_array_equal(np.nonzero(np.abs(px[:, axis] - bound) < 1e-12)[0], o.field(f"bcpts{b}"))


junk = st.text(alphabet=st.sampled_from(list("abcdefgmnprstxyz0123456789.-+e \t\n#")), max_size=200)


@SETTINGS
@given(junk)
def test_junk_text_gets_a_status_not_a_crash(text):
    try:
        d = pb.Deck(text=text)
    except pb.PntError as e:
        assert e.status == pb.PNT_ERR_DECK
        return
    try:
        d.params()
    except pb.PntError as e:
        assert e.status in (pb.PNT_ERR_DECK, pb.PNT_ERR_INVALID_ARG)
