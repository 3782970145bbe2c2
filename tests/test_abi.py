"""The C-ABI library loads and exports every symbol include/*.h declares."""
import ctypes
import glob
import os
import subprocess

import pytest

from conftest import ROOT
import pennant_b200 as pb


def _header_symbols():
    syms = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        syms.update(pb.exported_symbols_from_header(h))
    return sorted(syms)


def test_every_declared_symbol_is_exported():
    syms = _header_symbols()
    assert len(syms) >= 30
    lib = ctypes.CDLL(pb.LIB_PATH)
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_dynamic_symbol_table_has_c_linkage():
    out = subprocess.run(["nm", "-D", "--defined-only", pb.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    names = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for s in _header_symbols():
        assert s in names, s


def test_only_the_c_abi_is_exported():
    """Internal C++ symbols stay local (csrc/exports.map): a client's own
    classes of the same names cannot interpose on them."""
    out = subprocess.run(["nm", "-D", "--defined-only", pb.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    names = [line.split()[-1] for line in out.splitlines() if line.strip()]
    assert names and all(n.startswith("pnt_") for n in names), [n for n in names if not n.startswith("pnt_")]
    assert sorted(names) == _header_symbols()


def test_status_strings():
    for st in range(0, 10):
        assert pb.lib.pnt_status_string(st)
    assert pb.lib.pnt_status_string(999) == b"unknown status"


def test_null_arguments_are_rejected():
    assert pb.lib.pnt_deck_parse(None, None) == pb.PNT_ERR_INVALID_ARG
    assert b"null" in pb.lib.pnt_last_error()
    assert pb.lib.pnt_hydro_cycle(None, None) == pb.PNT_ERR_INVALID_ARG
    assert pb.lib.pnt_mesh_generate(None, None) == pb.PNT_ERR_INVALID_ARG


def test_cli_binary_exists():
    exe = os.path.join(ROOT, "pennant-legion_b200", "pennant")
    assert os.access(exe, os.X_OK)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 1 and "No Pennant input file" in r.stderr


def test_cli_skips_legion_arguments_and_accepts_debug_flag(tmp_path):
    """Run scripts of the reference put Legion runtime arguments first
    (-ll:cpu 4 -ll:gpu 1 ...); they are skipped, -d is accepted, and the
    deck is read and meshed before the GPU is asked for (without one, the
    run stops there with an error)."""
    exe = os.path.join(ROOT, "pennant-legion_b200", "pennant")
    deck = tmp_path / "sedovsmall.pnt"      # outputs land beside the deck
    deck.write_text(open(os.path.join(ROOT, "tests", "golden", "sedovsmall.pnt")).read())
    r = subprocess.run([exe, "-ll:cpu", "4", "-ll:gpu", "1", "-lg:prof", "0", "-d", "-f", str(deck)],
                       capture_output=True, text=True, timeout=120)
    assert "Usage" not in r.stderr
    assert "Zones:   81" in r.stdout and "Sides:   324" in r.stdout
    if not _has_device():
        assert r.returncode == 1 and "no CUDA device" in r.stderr


def _has_device():
    n = ctypes.c_int(0)
    try:
        rt = ctypes.CDLL("libcudart.so.12")
    except OSError:
        return False
    return rt.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0


@pytest.mark.skipif(_has_device(), reason="checks the no-device error path")
def test_hydro_create_without_device_fails_loudly():
    d = pb.Deck(path=os.path.join(ROOT, "tests", "golden", "sedovsmall.pnt"))
    m = pb.Mesh(deck=d)
    with pytest.raises(pb.PntError) as e:
        pb.Hydro(m, d.params())
    assert e.value.status == pb.PNT_ERR_NO_DEVICE


def test_wait_probe_arguments_and_no_device():
    """pnt_closure_wait_probe: bad arguments are rejected before any device
    work; without a device it fails with PNT_ERR_NO_DEVICE."""
    for arrive, limit in ((2, 10), (-1, 10), (0, 0), (1, (1 << 20) + 1)):
        assert pb.lib.pnt_closure_wait_probe(0, arrive, limit) == pb.PNT_ERR_INVALID_ARG
    if not _has_device():
        assert pb.lib.pnt_closure_wait_probe(0, 0, 10) == pb.PNT_ERR_NO_DEVICE
