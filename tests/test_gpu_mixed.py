"""Mixed-precision cycle (FP32 side forces, sound speed and zone dt; FP64
kinematics, pressure, work and the dt reduction) against the FP64 cycle,
which is itself bit-identical to the CPU oracle.

Every case states its relative L1 errors (sum |a - b| / sum |b|) of density,
specific energy and point velocity; the bound asserted is the accuracy
target of the reduced-precision paths, 1e-3 relative L1 density error,
applied to all three fields.
"""
import numpy as np
import pytest

from conftest import deck, golden
import pennant_b200 as pb

pytestmark = pytest.mark.gpu

L1_BOUND = 1e-3


def run(text, precision):
    d = pb.Deck(text=text)
    d.set("precision", precision)
    h = pb.Hydro(pb.Mesh(deck=d), d.params())
    s = h.run()
    out = {k: h.download(k) for k in ("zr", "ze", "pu", "px")}
    h.close()
    return s, out


def l1(a, b):
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))


def compare(text):
    s64, f64 = run(text, "fp64")
    s32, f32 = run(text, "mixed")
    assert s64["status"] == 0 and s32["status"] == 0
    err = {"zr": l1(f32["zr"], f64["zr"]), "ze": l1(f32["ze"], f64["ze"]),
           "u": l1(np.hypot(*f32["pu"].T), np.hypot(*f64["pu"].T))}
    print(f"cycles fp64 {s64['cycle']} mixed {s32['cycle']}, L1 errors {err}")
    return s64, s32, err


def leblanc(nx, ny, tstop):
    return (f"tstop {tstop}\nmeshtype rect\nmeshparams {nx} {ny} 9.0 0.9\nsubregion 3.0 9.0 0.0 0.9\n"
            "rinit 1.0\neinit 0.1\nrinitsub 1.0e-3\neinitsub 1.0e-7\nbcx 0.0 9.0\nbcy 0.0 0.9\n"
            "ssmin 0.1\nq1 0.3\nq2 2.0\ndtinit 1.e-3\n")


def test_mixed_sedov48_to_t1():
    s64, s32, err = compare(open(deck("sedov48.pnt")).read())
    assert s32["time"] == s64["time"] == 1.0
    assert max(err.values()) <= L1_BOUND, err


def test_mixed_leblanc_shock_tube():
    """Leblanc-type tube of the mixed-precision config (x < 3 dense and hot,
    x >= 3 rarefied), reduced to 576 x 58 zones, run to t = 6.0."""
    s64, s32, err = compare(leblanc(576, 58, 6.0))
    assert abs(s32["time"] - 6.0) < 1e-12
    assert max(err.values()) <= L1_BOUND, err


@pytest.mark.timeout(300)
def test_mixed_leblanc_full_size_config():
    """The mixed-precision workload at its full size: the Leblanc-type tube
    on 2880 x 288 zones over [0, 9] x [0, 0.9] to t = 6.0 (~9300 cycles a
    path), the mixed cycle against the FP64 cycle; the same deck as
    decks/leblanc2880x288.pnt and bench.py --workload leblanc."""
    s64, s32, err = compare(leblanc(2880, 288, 6.0))
    assert abs(s32["time"] - 6.0) < 1e-12 and abs(s64["time"] - 6.0) < 1e-12
    assert s64["cycle"] > 9000 and s32["cycle"] > 9000
    assert max(err.values()) <= L1_BOUND, err


def test_mixed_pie_noh():
    """Noh on the pie mesh (3-sided zones and 3-degree corners at the centre)
    up to cycle 150, before the stagnation zone at the origin starts to
    bounce.  Past that bounce (cycle ~200) the mixed run departs from the
    FP64 run in the central zones (relative L1 density error ~7e-3 at cycle
    400) while FP64 runs perturbed by 1e-6 stay within 1e-6; that departure
    is an open limitation of the mixed path on pie meshes."""
    text = open(golden("noh.pnt")).read().replace("cstop   10", "cstop   150")
    s64, s32, err = compare(text)
    assert max(err.values()) <= L1_BOUND, err


def test_mixed_reports_badsides_too():
    text = open(golden("sedovsmall.pnt")).read().replace("dtinit  0.0025", "dtinit  0.5")
    d = pb.Deck(text=text)
    d.set("precision", "mixed")
    h = pb.Hydro(pb.Mesh(deck=d), d.params())
    with pytest.raises(pb.PntError) as e:
        h.run()
    assert e.value.status == pb.PNT_ERR_BADSIDES
