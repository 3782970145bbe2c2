"""The drop-in boundary from plain C: a C99 program (no C++, no Python)
includes include/pennant_b200.h, links libpennant_b200.so and drives the
host-side half of the API -- the deck (InputFile), the mesh (Mesh + GenMesh),
the parameters, a piece of the mesh -- then asks for a Hydro object, which
without a GPU must fail with PNT_ERR_NO_DEVICE rather than fall back to
anything.  Its output is compared with the same calls made through the
Python binding."""
import os
import subprocess

import pytest

from conftest import ROOT, golden
import pennant_b200 as pb

C_SOURCE = r"""
#include <stdio.h>
#include <stdlib.h>
#include "pennant_b200.h"

#define CHECK(x) do { pnt_status s_ = (x); if (s_ != PNT_OK) { \
    fprintf(stderr, "%s: %s (%s)\n", #x, pnt_status_string(s_), pnt_last_error()); return 2; } } while (0)

int main(int argc, char** argv) {
    pnt_deck* deck = NULL;
    pnt_mesh* mesh = NULL;
    pnt_mesh* piece = NULL;
    pnt_mesh_desc md;
    pnt_piece_desc pd;
    pnt_params prm;
    pnt_hydro* hydro = NULL;
    pnt_status st;
    if (argc != 2) return 1;
    if (pnt_abi_version() != PNT_ABI_VERSION) return 3;
    CHECK(pnt_deck_load(argv[1], &deck));
    CHECK(pnt_mesh_generate(deck, &mesh));
    CHECK(pnt_mesh_describe(mesh, &md));
    CHECK(pnt_params_from_deck(deck, &prm));
    printf("mesh %d %d %d\n", md.numz, md.nums, md.nump);
    printf("params %d %.17g %.17g %.17g %.17g %d %d\n", prm.cstop, prm.tstop, prm.dtinit, prm.q1, prm.alfa,
           prm.nbcx, prm.nbcy);
    CHECK(pnt_mesh_piece(mesh, 2, 1, &piece));
    CHECK(pnt_mesh_piece_describe(piece, &pd));
    printf("piece %d %d %d %d\n", pd.piece, pd.zone0, pd.nhalo, pd.nnbr);
    st = pnt_hydro_create(mesh, &prm, 0, &hydro);
    printf("hydro %d\n", (int)st);
    if (hydro) pnt_hydro_destroy(hydro);
    pnt_mesh_destroy(piece);
    pnt_mesh_destroy(mesh);
    pnt_deck_destroy(deck);
    return 0;
}
"""


def _has_device():
    import ctypes
    try:
        rt = ctypes.CDLL("libcudart.so")
    except OSError:
        return False
    n = ctypes.c_int(0)
    return rt.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0


@pytest.mark.skipif(_has_device(), reason="checks the no-device answer of the C boundary")
def test_plain_c_client_against_the_python_binding(tmp_path):
    src = tmp_path / "client.c"
    src.write_text(C_SOURCE)
    exe = tmp_path / "client"
    pkg = os.path.dirname(pb.LIB_PATH)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe), "-L", pkg, "-lpennant_b200", f"-Wl,-rpath,{pkg}"], check=True)
    deck_path = golden("sedov.pnt")
    r = subprocess.run([str(exe), deck_path], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lines = dict(line.split(" ", 1) for line in r.stdout.strip().splitlines())

    d = pb.Deck(path=deck_path)
    m = pb.Mesh(deck=d)
    p = d.params()
    assert lines["mesh"].split() == [str(m.numz), str(m.nums), str(m.nump)]
    want = [p.cstop, p.tstop, p.dtinit, p.q1, p.alfa, p.nbcx, p.nbcy]
    got = lines["params"].split()
    assert [int(got[0])] + [float(v) for v in got[1:5]] + [int(v) for v in got[5:]] == want
    info = m.piece(2, 1).piece_info()
    assert lines["piece"].split() == [str(info["piece"]), str(info["zone0"]), str(info["nhalo"]),
                                      str(len(info["nbr"]))]
    assert int(lines["hydro"]) == pb.PNT_ERR_NO_DEVICE


CPP_SOURCE = r"""
#include <cstdio>
#include "pennant.hh"

int main(int argc, char** argv) {
    if (argc != 2) return 1;
    pnt::InputFile inp(argv[1]);
    pnt::Mesh mesh(&inp);
    pnt::PolyGas pgas(&inp, nullptr);
    pnt::TTS tts(&inp, nullptr);
    pnt::QCS qcs(&inp, nullptr);
    std::printf("mesh %d %d %d %d\n", mesh.nump, mesh.numz, mesh.nums, mesh.numc);
    std::printf("side %d %d %d %d %d\n", mesh.mapsp1()[5], mesh.mapsp2()[5], mesh.mapsz()[5], mesh.mapss3()[5],
                mesh.mapss4()[5]);
    std::printf("coef %.17g %.17g %.17g %.17g %.17g %.17g %.17g\n", pgas.gamma, pgas.ssmin, tts.alfa, tts.ssmin,
                qcs.qgamma, qcs.q1, qcs.q2);
    const std::vector<double> bcx = inp.getDoubleList("bcx", {}), bcy = inp.getDoubleList("bcy", {});
    for (double b : bcx) {
        pnt::HydroBC bc(&mesh, pnt::double2{1., 0.}, b, true);
        std::printf("bc %d", bc.numb);
        for (int p : bc.mapbp) std::printf(" %d", p);
        std::printf("\n");
    }
    for (double b : bcy) {
        pnt::HydroBC bc(&mesh, pnt::double2{0., 1.}, b, false);
        std::printf("bc %d", bc.numb);
        for (int p : bc.mapbp) std::printf(" %d", p);
        std::printf("\n");
    }
    try {
        pnt::Driver drv(&inp, "client");
        std::printf("driver %d\n", 0);
    } catch (const pnt::Error& e) {
        std::printf("driver %d\n", (int)e.status);
    }
    return 0;
}
"""


@pytest.mark.skipif(_has_device(), reason="checks the no-device answer of the C++ classes")
def test_cpp_classes_against_the_oracle(tmp_path):
    """The reference's class surface in C++ (pennant.hh): InputFile, Mesh
    with its side maps, PolyGas / TTS / QCS coefficients, HydroBC boundary
    point lists, and Driver, which without a GPU throws pnt::Error with
    PNT_ERR_NO_DEVICE.  Coefficients and boundary lists agree with the
    oracle's independent restatement."""
    from oracle import Oracle
    src = tmp_path / "client.cpp"
    src.write_text(CPP_SOURCE)
    exe = tmp_path / "client"
    pkg = os.path.dirname(pb.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(pkg, "csrc"), str(src), "-o", str(exe), "-L", pkg, "-lpennant_b200",
                    f"-Wl,-rpath,{pkg}"], check=True)
    for name in ("sedov.pnt", "leblanc.pnt", "nohsquare.pnt"):
        deck_path = golden(name)
        r = subprocess.run([str(exe), deck_path], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        rows = [line.split() for line in r.stdout.strip().splitlines()]
        o = Oracle(deck_path)
        mesh = next(r[1:] for r in rows if r[0] == "mesh")
        assert [int(v) for v in mesh] == [o.nump, o.numz, o.nums, o.nums]
        side = [int(v) for v in next(r[1:] for r in rows if r[0] == "side")]
        assert side == [int(o.field(k)[5]) for k in ("mapsp1", "mapsp2", "mapsz", "mapss3", "mapss4")]
        coef = [float(v) for v in next(r[1:] for r in rows if r[0] == "coef")]
        assert coef == [o.scalar(k) for k in ("gamma", "pgas_ssmin", "alfa", "tts_ssmin", "qgamma", "q1", "q2")]
        bcs = [r[1:] for r in rows if r[0] == "bc"]
        assert len(bcs) == o.num("nbc")
        for b, row in enumerate(bcs):
            pts = [int(v) for v in row[1:]]
            assert int(row[0]) == len(pts) and pts == o.field(f"bcpts{b}").tolist(), (name, b)
        assert int(next(r[1] for r in rows if r[0] == "driver")) == pb.PNT_ERR_NO_DEVICE
