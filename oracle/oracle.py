"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker / timed reference, never by the
product library.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_DIR, "_build", "liboracle.so")

_D2 = {"px", "pxp", "px0", "pu", "pu0", "pf", "pap", "zx", "zxp", "zuc", "ex", "exp",
       "ssurfp", "sfp", "sfq", "sft", "cqe1", "cqe2"}
_INT = {"znump", "mapsp1", "mapsp2", "mapsz", "mapss3", "mapss4"}
_POINT = {"px", "pxp", "px0", "pu", "pu0", "pf", "pap", "pmaswt"}
_ZONE = {"znump", "zx", "zxp", "zuc", "zarea", "zvol", "zareap", "zvolp", "zvol0", "zdl",
         "zm", "zr", "zrp", "ze", "zetot", "zw", "zwrate", "zp", "zss", "zdu", "ztmp"}


def build() -> None:
    subprocess.run(["make", "-s", "-C", _DIR], check=True)


def _load():
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    lib.orc_create.restype = C.c_int
    lib.orc_create.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(vp), C.c_char_p, C.c_size_t]
    lib.orc_destroy.argtypes = [vp]
    lib.orc_cycle.argtypes = [vp]
    lib.orc_run.argtypes = [vp, C.c_int]
    lib.orc_done.argtypes = [vp]
    lib.orc_set_threads.argtypes = [vp, C.c_int]
    lib.orc_num.restype = C.c_int64
    lib.orc_num.argtypes = [vp, C.c_char_p]
    lib.orc_scalar.restype = C.c_double
    lib.orc_scalar.argtypes = [vp, C.c_char_p]
    lib.orc_field.restype = vp
    lib.orc_field.argtypes = [vp, C.c_char_p]
    lib.orc_bc_count.argtypes = [vp, C.c_int]
    lib.orc_write_xy.argtypes = [vp, C.c_char_p]
    lib.orc_write_gold.argtypes = [vp, C.c_char_p]
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


class OracleError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"oracle status {status}: {msg}")
        self.status = status


class Oracle:
    """Serial CPU restatement of the reference's hydro cycle."""

    def __init__(self, path: str | None = None, text: str | None = None, threads: int = 1):
        L = lib()
        h = C.c_void_p()
        err = C.create_string_buffer(512)
        st = L.orc_create(path.encode() if path else None, text.encode() if text else None,
                          C.byref(h), err, 512)
        if st:
            raise OracleError(st, err.value.decode())
        self.h = h
        L.orc_set_threads(h, threads)
        self.nump = L.orc_num(h, b"nump")
        self.numz = L.orc_num(h, b"numz")
        self.nums = L.orc_num(h, b"nums")

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def cycle(self) -> int:
        return lib().orc_cycle(self.h)

    def run(self, max_cycles: int = 0) -> int:
        return lib().orc_run(self.h, max_cycles)

    @property
    def done(self) -> bool:
        return bool(lib().orc_done(self.h))

    def num(self, what: str) -> int:
        return lib().orc_num(self.h, what.encode())

    def scalar(self, what: str) -> float:
        return lib().orc_scalar(self.h, what.encode())

    def field(self, name: str) -> np.ndarray:
        """Copy of a field in reference numbering (double2 fields as (n, 2))."""
        ptr = lib().orc_field(self.h, name.encode())
        if not ptr:
            raise KeyError(name)
        if name.startswith("bcpts"):
            n = lib().orc_bc_count(self.h, int(name[5:]))
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_int32)), shape=(n,)).copy()
        n = self.nump if name in _POINT else (self.numz if name in _ZONE else self.nums)
        if name in _INT:
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_int32)), shape=(n,)).copy()
        if name in _D2:
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_double)), shape=(2 * n,)).reshape(n, 2).copy()
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_double)), shape=(n,)).copy()

    def write_xy(self, path: str) -> None:
        lib().orc_write_xy(self.h, path.encode())

    def write_gold(self, base: str) -> None:
        lib().orc_write_gold(self.h, base.encode())
