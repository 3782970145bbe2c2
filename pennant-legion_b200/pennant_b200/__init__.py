"""ctypes binding of libpennant_b200.so (C ABI: include/pennant_b200.h).

The compute path is the CUDA library; this module only marshals arguments.
Importing it loads the in-tree shared library and raises if it is missing:
there is no CPU fallback.

Objects mirror the reference's classes: ``Deck`` (InputFile), ``Mesh``
(Mesh + GenMesh, one piece), ``Hydro`` (Hydro + the Driver loop).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_PKG_DIR), "libpennant_b200.so")

PNT_OK = 0
PNT_ERR_INVALID_ARG = 1
PNT_ERR_DECK = 2
PNT_ERR_BADSIDES = 3
PNT_ERR_CUDA = 4
PNT_ERR_UNSUPPORTED = 5
PNT_ERR_TIMEOUT = 6
PNT_ERR_NOMEM = 7
PNT_ERR_NO_DEVICE = 8
PNT_ERR_STATE = 9

PREC_FP64 = 0
PREC_MIXED = 1
PREC_LEARNED = 2
MAX_BC = 16

CLOSURE_PARAMS = 5380
CLOSURE_NORM = 36
CLOSURE_IN = 14
CLOSURE_CLASSES = ("zero", "dead", "mlp", "fallback", "ood", "acute", "error", "zones")

FIELDS = {"px": 0, "pu": 1, "zr": 2, "ze": 3, "zp": 4, "zm": 5, "zetot": 6,
          "zvol": 7, "zwrate": 8, "smf": 9}
_POINT2 = {"px", "pu"}
_SIDE = {"smf"}


class PntError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"pnt status {status}: {msg}")
        self.status = status


class Params(C.Structure):
    _fields_ = [
        ("cstop", C.c_int32), ("dtreport", C.c_int32),
        ("tstop", C.c_double), ("dtmax", C.c_double), ("dtinit", C.c_double), ("dtfac", C.c_double),
        ("cfl", C.c_double), ("cflv", C.c_double), ("rinit", C.c_double), ("einit", C.c_double),
        ("rinitsub", C.c_double), ("einitsub", C.c_double), ("uinitradial", C.c_double),
        ("has_subregion", C.c_int32), ("subregion", C.c_double * 4),
        ("nbcx", C.c_int32), ("nbcy", C.c_int32),
        ("bcx", C.c_double * MAX_BC), ("bcy", C.c_double * MAX_BC),
        ("gamma", C.c_double), ("pgas_ssmin", C.c_double),
        ("alfa", C.c_double), ("tts_ssmin", C.c_double),
        ("qgamma", C.c_double), ("q1", C.c_double), ("q2", C.c_double),
        ("precision", C.c_int32), ("graph_cycles", C.c_int32),
        ("reserved", C.c_int32 * 14),
    ]


class Scalars(C.Structure):
    _fields_ = [
        ("cycle", C.c_int32), ("done", C.c_int32), ("status", C.c_int32), ("nbad", C.c_int32),
        ("time", C.c_double), ("dt", C.c_double), ("dtrec", C.c_double),
        ("dtnew", C.c_double), ("dvovmax", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class MeshDesc(C.Structure):
    _fields_ = [
        ("nump", C.c_int32), ("numz", C.c_int32), ("nums", C.c_int32),
        ("px", C.POINTER(C.c_double)), ("znump", C.POINTER(C.c_int32)),
        ("mapsp1", C.POINTER(C.c_int32)), ("mapsp2", C.POINTER(C.c_int32)),
        ("mapsz", C.POINTER(C.c_int32)), ("mapss3", C.POINTER(C.c_int32)),
        ("mapss4", C.POINTER(C.c_int32)),
    ]


class PieceDesc(C.Structure):
    _fields_ = [
        ("piece", C.c_int32), ("npieces", C.c_int32), ("zone0", C.c_int32), ("side0", C.c_int32),
        ("gpoint", C.POINTER(C.c_int32)), ("nhalo", C.c_int32), ("halo_side", C.POINTER(C.c_int32)),
        ("nnbr", C.c_int32), ("nbr", C.POINTER(C.c_int32)), ("recv_off", C.POINTER(C.c_int32)),
        ("send_off", C.POINTER(C.c_int32)), ("send_side", C.POINTER(C.c_int32)),
    ]


class PieceBuffers(C.Structure):
    _fields_ = [
        ("send", C.c_void_p), ("send_cforce_offset", C.c_size_t),
        ("halo_cmass", C.c_void_p), ("halo_cforce", C.c_void_p),
        ("cmass_bytes", C.c_int32), ("cforce_bytes", C.c_int32),
        ("red", C.c_void_p), ("stream", C.c_void_p),
    ]


REPORT_FN = C.CFUNCTYPE(None, C.POINTER(Scalars), C.c_double, C.c_void_p)


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C pennant-legion_b200` "
                          "(or __graft_entry__.build()); there is no fallback path")
    lib = C.CDLL(LIB_PATH)
    vp, i32, dbl, sz = C.c_void_p, C.c_int32, C.c_double, C.c_size_t
    pp = C.POINTER(C.c_void_p)
    sig = {
        "pnt_status_string": (C.c_char_p, [i32]),
        "pnt_last_error": (C.c_char_p, []),
        "pnt_abi_version": (i32, []),
        "pnt_deck_load": (i32, [C.c_char_p, pp]),
        "pnt_deck_parse": (i32, [C.c_char_p, pp]),
        "pnt_deck_set": (i32, [vp, C.c_char_p, C.c_char_p]),
        "pnt_deck_has": (i32, [vp, C.c_char_p]),
        "pnt_deck_get_int": (i32, [vp, C.c_char_p, i32]),
        "pnt_deck_get_double": (dbl, [vp, C.c_char_p, dbl]),
        "pnt_deck_get_string": (i32, [vp, C.c_char_p, C.c_char_p, C.c_char_p, sz]),
        "pnt_deck_get_double_list": (i32, [vp, C.c_char_p, C.POINTER(C.c_double), i32]),
        "pnt_deck_destroy": (None, [vp]),
        "pnt_mesh_generate": (i32, [vp, pp]),
        "pnt_mesh_create": (i32, [C.POINTER(MeshDesc), pp]),
        "pnt_mesh_describe": (i32, [vp, C.POINTER(MeshDesc)]),
        "pnt_mesh_point_corners": (i32, [vp, C.POINTER(C.POINTER(C.c_int32)),
                                         C.POINTER(C.POINTER(C.c_int32))]),
        "pnt_mesh_destroy": (None, [vp]),
        "pnt_mesh_piece": (i32, [vp, i32, i32, pp]),
        "pnt_mesh_piece_describe": (i32, [vp, C.POINTER(PieceDesc)]),
        "pnt_params_default": (i32, [C.POINTER(Params)]),
        "pnt_params_from_deck": (i32, [vp, C.POINTER(Params)]),
        "pnt_hydro_create": (i32, [vp, C.POINTER(Params), i32, pp]),
        "pnt_hydro_destroy": (None, [vp]),
        "pnt_hydro_cycle": (i32, [vp, C.POINTER(Scalars)]),
        "pnt_hydro_run": (i32, [vp, i32, REPORT_FN, vp, C.POINTER(Scalars)]),
        "pnt_hydro_enqueue": (i32, [vp, i32]),
        "pnt_hydro_synchronize": (i32, [vp]),
        "pnt_hydro_time_kernels": (i32, [vp, i32, C.POINTER(C.c_double), i32]),
        "pnt_hydro_time_cycles": (i32, [vp, i32, C.POINTER(C.c_double)]),
        "pnt_hydro_copy_state": (i32, [vp, vp]),
        "pnt_hydro_get_scalars": (i32, [vp, C.POINTER(Scalars)]),
        "pnt_hydro_download": (i32, [vp, i32, vp, sz]),
        "pnt_hydro_upload": (i32, [vp, i32, vp, sz]),
        "pnt_hydro_device_ptr": (i32, [vp, i32, pp]),
        "pnt_hydro_stream": (i32, [vp, pp]),
        "pnt_hydro_check_finite": (i32, [vp, C.POINTER(i32), C.POINTER(C.c_int64)]),
        "pnt_hydro_piece_buffers": (i32, [vp, C.POINTER(PieceBuffers)]),
        "pnt_hydro_piece_forces": (i32, [vp]),
        "pnt_hydro_piece_advance": (i32, [vp]),
        "pnt_hydro_piece_finish": (i32, [vp]),
        "pnt_batch_create": (i32, [C.POINTER(vp), C.POINTER(Params), i32, i32, pp]),
        "pnt_batch_destroy": (None, [vp]),
        "pnt_batch_set_shape": (i32, [vp, i32, i32]),
        "pnt_batch_get_shape": (i32, [vp, C.POINTER(i32), C.POINTER(i32)]),
        "pnt_batch_tune": (i32, [vp, i32, C.POINTER(i32), C.POINTER(i32), C.POINTER(dbl)]),
        "pnt_batch_run": (i32, [vp, i32, C.POINTER(i32)]),
        "pnt_batch_enqueue": (i32, [vp, i32]),
        "pnt_batch_time_cycles": (i32, [vp, i32, C.POINTER(dbl)]),
        "pnt_batch_scalars": (i32, [vp, i32, C.POINTER(Scalars)]),
        "pnt_batch_download": (i32, [vp, i32, i32, vp, sz]),
        "pnt_op_calc_dt": (i32, [vp, vp, vp, vp, vp, C.c_int64, dbl, dbl, dbl, vp, vp]),
        "pnt_op_calc_dt_noalloc": (i32, [vp, vp, vp, vp, vp, C.c_int64, dbl, dbl, dbl, vp, vp]),
        "pnt_closure_create": (i32, [i32, C.c_uint64, pp]),
        "pnt_closure_load": (i32, [C.c_char_p, i32, pp]),
        "pnt_closure_save": (i32, [vp, C.c_char_p]),
        "pnt_closure_destroy": (None, [vp]),
        "pnt_closure_get": (i32, [vp, vp, vp, vp]),
        "pnt_closure_set": (i32, [vp, vp, vp, vp]),
        "pnt_hydro_harvest": (i32, [vp, dbl, dbl, C.c_uint64, vp, vp, vp, C.c_int64, C.POINTER(C.c_int64)]),
        "pnt_closure_fit_normalization": (i32, [vp, vp, vp, C.c_int64]),
        "pnt_closure_prepare": (i32, [vp, vp, vp, C.c_int64, vp, vp]),
        "pnt_closure_train": (i32, [vp, vp, vp, C.c_int64, C.c_int64, i32, i32, C.c_float, vp]),
        "pnt_closure_gradient": (i32, [vp, vp, vp, C.c_int64, vp, C.POINTER(C.c_float)]),
        "pnt_closure_forward": (i32, [vp, vp, C.c_int64, vp]),
        "pnt_closure_wait_probe": (i32, [i32, i32, i32]),
        "pnt_hydro_set_closure": (i32, [vp, vp, i32]),
        "pnt_hydro_closure_counts": (i32, [vp, C.POINTER(C.c_uint64), i32]),
        "pnt_hydro_write_xy": (i32, [vp, C.c_char_p]),
        "pnt_pieces_create": (i32, [vp, C.POINTER(Params), i32, C.POINTER(i32), i32, pp]),
        "pnt_pieces_set_closure": (i32, [vp, vp, i32]),
        "pnt_pieces_cycle": (i32, [vp, C.POINTER(Scalars)]),
        "pnt_pieces_run": (i32, [vp, i32, REPORT_FN, vp, C.POINTER(Scalars)]),
        "pnt_pieces_download": (i32, [vp, i32, vp, sz]),
        "pnt_pieces_write_xy": (i32, [vp, C.c_char_p]),
        "pnt_pieces_destroy": (None, [vp]),
        "pnt_hydro_write_gold": (i32, [vp, C.c_char_p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status: int) -> None:
    if status != PNT_OK:
        raise PntError(status, (lib.pnt_last_error() or b"").decode())


def _b(s: str) -> bytes:
    return s.encode()


class Deck:
    """InputFile: a parsed .pnt deck."""

    def __init__(self, path: str | None = None, text: str | None = None):
        h = C.c_void_p()
        if text is not None:
            check(lib.pnt_deck_parse(_b(text), C.byref(h)))
        else:
            check(lib.pnt_deck_load(_b(path), C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            lib.pnt_deck_destroy(self.h)
            self.h = None

    def set(self, key: str, value) -> "Deck":
        check(lib.pnt_deck_set(self.h, _b(key), _b(str(value))))
        return self

    def get_int(self, key, dflt=0):
        return lib.pnt_deck_get_int(self.h, _b(key), dflt)

    def get_double(self, key, dflt=0.0):
        return lib.pnt_deck_get_double(self.h, _b(key), dflt)

    def get_string(self, key, dflt=""):
        buf = C.create_string_buffer(4096)
        lib.pnt_deck_get_string(self.h, _b(key), _b(dflt), buf, 4096)
        return buf.value.decode()

    def get_double_list(self, key):
        n = lib.pnt_deck_get_double_list(self.h, _b(key), None, 0)
        if n < 0:
            return None
        arr = (C.c_double * max(n, 1))()
        lib.pnt_deck_get_double_list(self.h, _b(key), arr, n)
        return list(arr[:n])

    def params(self) -> Params:
        p = Params()
        check(lib.pnt_params_from_deck(self.h, C.byref(p)))
        return p


class Mesh:
    """Mesh + GenMesh for one piece, reference numbering (or a piece of a
    mesh: Mesh.piece)."""

    def __init__(self, deck: Deck | None = None, desc: dict | None = None, _handle=None):
        h = C.c_void_p()
        if _handle is not None:
            h = _handle
        elif deck is not None:
            check(lib.pnt_mesh_generate(deck.h, C.byref(h)))
        else:
            arrs = {k: np.ascontiguousarray(desc[k], dtype=np.float64 if k == "px" else np.int32)
                    for k in ("px", "znump", "mapsp1", "mapsp2", "mapsz", "mapss3", "mapss4")}
            d = MeshDesc()
            d.nump = len(arrs["px"]) // 2 if arrs["px"].ndim == 1 else arrs["px"].shape[0]
            d.numz = len(arrs["znump"])
            d.nums = len(arrs["mapsp1"])
            d.px = arrs["px"].ctypes.data_as(C.POINTER(C.c_double))
            for k in ("znump", "mapsp1", "mapsp2", "mapsz", "mapss3", "mapss4"):
                setattr(d, k, arrs[k].ctypes.data_as(C.POINTER(C.c_int32)))
            check(lib.pnt_mesh_create(C.byref(d), C.byref(h)))
        self.h = h
        d = MeshDesc()
        check(lib.pnt_mesh_describe(self.h, C.byref(d)))
        self.nump, self.numz, self.nums = d.nump, d.numz, d.nums
        self._desc = d

    def __del__(self):
        if getattr(self, "h", None):
            lib.pnt_mesh_destroy(self.h)
            self.h = None

    def array(self, name: str) -> np.ndarray:
        """Copy of a connectivity array (px as (nump, 2))."""
        d = self._desc
        if name == "px":
            return np.ctypeslib.as_array(d.px, shape=(2 * d.nump,)).reshape(-1, 2).copy()
        n = d.numz if name == "znump" else d.nums
        return np.ctypeslib.as_array(getattr(d, name), shape=(n,)).copy()

    def point_corners(self):
        """Point -> corner CSR (offsets, slots); for a piece the slots past
        nums are halo slots."""
        off = C.POINTER(C.c_int32)()
        sides = C.POINTER(C.c_int32)()
        check(lib.pnt_mesh_point_corners(self.h, C.byref(off), C.byref(sides)))
        offs = np.ctypeslib.as_array(off, shape=(self.nump + 1,)).copy()
        return offs, np.ctypeslib.as_array(sides, shape=(int(offs[-1]),)).copy()

    def piece(self, npieces: int, piece: int) -> "Mesh":
        """Piece `piece` of `npieces`: a contiguous zone range with its
        points, local numbering in global order, halo corner slots."""
        h = C.c_void_p()
        check(lib.pnt_mesh_piece(self.h, npieces, piece, C.byref(h)))
        return Mesh(_handle=h)

    def piece_info(self) -> dict:
        """Global ids and halo exchange lists of a piece mesh (numpy copies)."""
        d = PieceDesc()
        check(lib.pnt_mesh_piece_describe(self.h, C.byref(d)))

        def arr(ptr, n):
            return np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n > 0 and ptr else np.zeros(0, np.int32)

        nn = d.nnbr
        info = {"piece": d.piece, "npieces": d.npieces, "zone0": d.zone0, "side0": d.side0,
                "nhalo": d.nhalo, "nbr": arr(d.nbr, nn)}
        info["gpoint"] = arr(d.gpoint, self.nump) if d.npieces > 1 else np.arange(self.nump, dtype=np.int32)
        info["halo_side"] = arr(d.halo_side, d.nhalo)
        info["recv_off"] = arr(d.recv_off, nn + 1) if d.npieces > 1 else np.zeros(1, np.int32)
        info["send_off"] = arr(d.send_off, nn + 1) if d.npieces > 1 else np.zeros(1, np.int32)
        info["send_side"] = arr(d.send_side, int(info["send_off"][-1]))
        return info


class Hydro:
    """Hydro state on one GPU plus the Driver loop."""

    def __init__(self, mesh: Mesh, params: Params, device: int = 0):
        h = C.c_void_p()
        check(lib.pnt_hydro_create(mesh.h, C.byref(params), device, C.byref(h)))
        self.h = h
        self.mesh = mesh
        self.params = params

    def close(self):
        if getattr(self, "h", None):
            lib.pnt_hydro_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def cycle(self) -> dict:
        s = Scalars()
        check(lib.pnt_hydro_cycle(self.h, C.byref(s)))
        return s.as_dict()

    def run(self, max_cycles: int = 0, report=None) -> dict:
        s = Scalars()
        if report is None:
            cb = REPORT_FN()
        else:
            cb = REPORT_FN(lambda sp, us, _u: report(sp.contents.as_dict(), us))
        check(lib.pnt_hydro_run(self.h, max_cycles, cb, None, C.byref(s)))
        return s.as_dict()

    def enqueue(self, ncycles: int) -> None:
        check(lib.pnt_hydro_enqueue(self.h, ncycles))

    def time_kernels(self, ncycles: int) -> list:
        """Mean ms of passes A, B, C (which ends the cycle), a separate
        end-of-cycle step (none: about 0) and the closure pass over `ncycles`
        (these cycles advance the run)."""
        out = (C.c_double * 5)()
        check(lib.pnt_hydro_time_kernels(self.h, ncycles, out, 5))
        return list(out)

    def copy_state_from(self, src: "Hydro") -> None:
        check(lib.pnt_hydro_copy_state(self.h, src.h))

    def time_cycles(self, ncycles: int) -> float:
        """Device milliseconds of `ncycles` graph-replayed cycles (CUDA events on the stream)."""
        ms = C.c_double()
        check(lib.pnt_hydro_time_cycles(self.h, ncycles, C.byref(ms)))
        return ms.value

    def synchronize(self) -> None:
        check(lib.pnt_hydro_synchronize(self.h))

    def scalars(self) -> dict:
        s = Scalars()
        check(lib.pnt_hydro_get_scalars(self.h, C.byref(s)))
        return s.as_dict()

    def _shape(self, name):
        if name in _POINT2:
            return (self.mesh.nump, 2)
        if name in _SIDE:
            return (self.mesh.nums,)
        return (self.mesh.numz,)

    def download(self, name: str) -> np.ndarray:
        out = np.empty(self._shape(name), dtype=np.float64)
        check(lib.pnt_hydro_download(self.h, FIELDS[name], out.ctypes.data, out.nbytes))
        return out

    def upload(self, name: str, arr) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(self._shape(name))
        check(lib.pnt_hydro_upload(self.h, FIELDS[name], a.ctypes.data, a.nbytes))

    def device_ptr(self, name: str) -> int:
        p = C.c_void_p()
        check(lib.pnt_hydro_device_ptr(self.h, FIELDS[name], C.byref(p)))
        return p.value

    def stream(self) -> int:
        p = C.c_void_p()
        check(lib.pnt_hydro_stream(self.h, C.byref(p)))
        return p.value or 0

    def check_finite(self):
        """(field name, index) of the first NaN/Inf in the state, or (None, -1)."""
        f, i = C.c_int32(), C.c_int64()
        check(lib.pnt_hydro_check_finite(self.h, C.byref(f), C.byref(i)))
        if f.value < 0:
            return None, -1
        name = next(k for k, v in FIELDS.items() if v == f.value)
        return name, i.value

    def set_closure(self, closure: "Closure", mode: int = 0) -> None:
        """Learned cycle: 0 the network, 1 no force on its corners, 2 plain QCS there."""
        check(lib.pnt_hydro_set_closure(self.h, closure.h, mode))
        self.closure = closure

    def closure_counts(self, reset: bool = False) -> dict:
        out = (C.c_uint64 * len(CLOSURE_CLASSES))()
        check(lib.pnt_hydro_closure_counts(self.h, out, 1 if reset else 0))
        return dict(zip(CLOSURE_CLASSES, [int(v) for v in out]))

    def harvest(self, dead: float, keep: float, seed: int, feats: int, targets: int, sides: int,
                capacity: int, count: int) -> int:
        """Appends closure training samples (device addresses) at `count`; returns the new count."""
        n = C.c_int64(count)
        check(lib.pnt_hydro_harvest(self.h, dead, keep, seed, feats, targets, sides, capacity, C.byref(n)))
        return n.value

    def write_xy(self, path: str) -> None:
        check(lib.pnt_hydro_write_xy(self.h, _b(path)))

    def write_gold(self, base: str) -> None:
        check(lib.pnt_hydro_write_gold(self.h, _b(base)))


class Batch:
    """Many independent meshes advanced together on one GPU (FP64 cycle)."""

    def __init__(self, meshes, params, device: int = 0):
        n = len(meshes)
        harr = (C.c_void_p * n)(*[m.h.value for m in meshes])
        parr = (Params * n)(*params)
        h = C.c_void_p()
        check(lib.pnt_batch_create(harr, parr, n, device, C.byref(h)))
        self.h = h
        self.meshes = list(meshes)

    def close(self):
        if getattr(self, "h", None):
            lib.pnt_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_shape(self, zones_per_tile: int, ctas_per_sm: int) -> None:
        check(lib.pnt_batch_set_shape(self.h, zones_per_tile, ctas_per_sm))

    def shape(self):
        a, b = C.c_int32(), C.c_int32()
        check(lib.pnt_batch_get_shape(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def tune(self, trial_cycles: int = 4):
        a, b, ms = C.c_int32(), C.c_int32(), C.c_double()
        check(lib.pnt_batch_tune(self.h, trial_cycles, C.byref(a), C.byref(b), C.byref(ms)))
        return a.value, b.value, ms.value

    def run(self, max_cycles: int = 0) -> int:
        left = C.c_int32()
        check(lib.pnt_batch_run(self.h, max_cycles, C.byref(left)))
        return left.value

    def time_cycles(self, n: int) -> float:
        ms = C.c_double()
        check(lib.pnt_batch_time_cycles(self.h, n, C.byref(ms)))
        return ms.value

    def scalars(self, i: int) -> dict:
        s = Scalars()
        check(lib.pnt_batch_scalars(self.h, i, C.byref(s)))
        return s.as_dict()

    def download(self, i: int, name: str) -> np.ndarray:
        m = self.meshes[i]
        shape = (m.nump, 2) if name in _POINT2 else (m.numz,)
        out = np.empty(shape, dtype=np.float64)
        check(lib.pnt_batch_download(self.h, i, FIELDS[name], out.ctypes.data, out.nbytes))
        return out


class Pieces:
    """numpcs pieces of one mesh stepped together by the library (peer
    copies between the pieces' devices, host reductions): bit-identical to
    one Hydro over the whole mesh."""

    def __init__(self, mesh: Mesh, params: Params, npieces: int, devices=(0,)):
        h = C.c_void_p()
        devs = (C.c_int32 * len(devices))(*devices)
        check(lib.pnt_pieces_create(mesh.h, C.byref(params), npieces, devs, len(devices), C.byref(h)))
        self.h = h
        self.mesh = mesh

    def close(self):
        if getattr(self, "h", None):
            lib.pnt_pieces_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_closure(self, closure: "Closure", mode: int = 0) -> None:
        check(lib.pnt_pieces_set_closure(self.h, closure.h, mode))

    def cycle(self) -> dict:
        s = Scalars()
        check(lib.pnt_pieces_cycle(self.h, C.byref(s)))
        return s.as_dict()

    def run(self, max_cycles: int = 0) -> dict:
        s = Scalars()
        check(lib.pnt_pieces_run(self.h, max_cycles, REPORT_FN(), None, C.byref(s)))
        return s.as_dict()

    def download(self, name: str) -> np.ndarray:
        shape = (self.mesh.nump, 2) if name in _POINT2 else (self.mesh.numz,)
        out = np.empty(shape, dtype=np.float64)
        check(lib.pnt_pieces_download(self.h, FIELDS[name], out.ctypes.data, out.nbytes))
        return out

    def write_xy(self, path: str) -> None:
        check(lib.pnt_pieces_write_xy(self.h, _b(path)))


class Closure:
    """The learned QCS closure: 14-64-64-4 network, its normalisation and thresholds."""

    def __init__(self, seed: int = 0, device: int = 0, path: str | None = None):
        h = C.c_void_p()
        if path is not None:
            check(lib.pnt_closure_load(_b(path), device, C.byref(h)))
        else:
            check(lib.pnt_closure_create(device, seed, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib.pnt_closure_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def save(self, path: str) -> None:
        check(lib.pnt_closure_save(self.h, _b(path)))

    def get(self):
        p = np.empty(CLOSURE_PARAMS, np.float32)
        nm = np.empty(CLOSURE_NORM, np.float32)
        th = np.empty(3, np.float32)
        check(lib.pnt_closure_get(self.h, p.ctypes.data, nm.ctypes.data, th.ctypes.data))
        return p, nm, th

    def set(self, params=None, norm=None, thresholds=None) -> None:
        arrs = [None if a is None else np.ascontiguousarray(a, np.float32) for a in (params, norm, thresholds)]
        ptrs = [None if a is None else a.ctypes.data for a in arrs]
        check(lib.pnt_closure_set(self.h, *ptrs))

    def fit_normalization(self, feats: int, targets: int, n: int) -> None:
        check(lib.pnt_closure_fit_normalization(self.h, feats, targets, n))

    def prepare(self, feats: int, targets: int, n: int, x: int, t: int) -> None:
        check(lib.pnt_closure_prepare(self.h, feats, targets, n, x, t))

    def train(self, x: int, t: int, n: int, first: int, steps: int, rows_per_step: int, lr: float) -> np.ndarray:
        losses = np.zeros(max(steps, 1), np.float32)
        check(lib.pnt_closure_train(self.h, x, t, n, first, steps, rows_per_step, lr, losses.ctypes.data))
        return losses[:steps]

    def gradient(self, x: int, t: int, n: int):
        g = np.empty(CLOSURE_PARAMS, np.float32)
        loss = C.c_float()
        check(lib.pnt_closure_gradient(self.h, x, t, n, g.ctypes.data, C.byref(loss)))
        return g, loss.value

    def forward(self, feats: int, n: int, out: int) -> None:
        check(lib.pnt_closure_forward(self.h, feats, n, out))


def op_calc_dt(zdl: int, zdu: int, zss: int, zvol: int, zvol0: int, numz: int, cfl: float,
               cflv: float, dtlast: float, out: int, stream: int = 0) -> None:
    """pnt_op_calc_dt on device addresses (ints); out receives dtrec, dtnew, dvovmax."""
    check(lib.pnt_op_calc_dt(zdl, zdu, zss, zvol, zvol0, numz, cfl, cflv, dtlast, out, stream))


def exported_symbols_from_header(header_path: str) -> list[str]:
    """Function names declared in include/pennant_b200.h."""
    import re
    txt = open(header_path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(pnt_[a-z0-9_]+)\s*\(", txt)))
