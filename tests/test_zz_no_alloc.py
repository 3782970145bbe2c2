"""pnt_op_calc_dt_noalloc: the dt reduction without any device allocation.

Some callers cannot allocate device memory: code running inside a runtime
that owns all GPU memory (a Legion GPU task, where the mapper accounts for
every instance), loops that cannot risk an allocation stalling or failing
under memory pressure, processes capped by a pool they do not control.  The
entry point keeps its per-block partials in a fixed device array instead,
so its results must equal those of the allocating pnt_op_calc_dt bit for
bit -- including on back-to-back calls, since every call reuses that array.

This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

import pennant_b200 as pb

pytestmark = pytest.mark.gpu

MAX_ZONES = 16777216   # PNT_OP_CALC_DT_NOALLOC_MAX_ZONES


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    zvol0 = rng.uniform(0.5, 1.5, n)
    arrs = [rng.uniform(1e-3, 1e-1, n), rng.uniform(0, 2, n), rng.uniform(0, 1, n),
            zvol0 * (1 + rng.normal(0, 1e-3, n)), zvol0]
    return [torch.from_numpy(a).cuda() for a in arrs]


def _call(fn, dev, cfl, cflv, dtlast):
    out = torch.full((3,), -1.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = fn(*(t.data_ptr() for t in dev), dev[0].numel(), cfl, cflv, dtlast, out.data_ptr(), stream)
    pb.check(st)
    torch.cuda.synchronize()
    return out.cpu().numpy().tolist()


def test_noalloc_matches_allocating_entry_on_two_calls_in_a_row():
    a = _inputs(3_000_017, 1)      # 1465 blocks of partials
    b = _inputs(123_457, 2)        # fewer blocks: must not read the first call's leftovers
    ref_a = _call(pb.lib.pnt_op_calc_dt, a, 0.6, 0.1, 2e-3)
    ref_b = _call(pb.lib.pnt_op_calc_dt, b, 0.5, 0.2, 1e-3)
    got_a = _call(pb.lib.pnt_op_calc_dt_noalloc, a, 0.6, 0.1, 2e-3)
    got_b = _call(pb.lib.pnt_op_calc_dt_noalloc, b, 0.5, 0.2, 1e-3)
    assert got_a == ref_a
    assert got_b == ref_b
    assert ref_a != ref_b


def test_noalloc_rejects_sizes_beyond_its_limit():
    dev = _inputs(16, 3)
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    st = pb.lib.pnt_op_calc_dt_noalloc(*(t.data_ptr() for t in dev), MAX_ZONES + 1, 0.6, 0.1, 1e-3,
                                       out.data_ptr(), None)
    assert st == pb.PNT_ERR_INVALID_ARG
    assert b"no-allocation limit" in pb.lib.pnt_last_error()


def test_noalloc_takes_nothing_from_the_device_memory_pool():
    """The allocating entry point takes its partials from the device's default
    stream-ordered pool (cudaMallocAsync); the no-allocation one must leave
    the pool's high-water mark where it was.  Inputs and outputs are
    allocated before the mark is reset."""
    rt = ctypes.CDLL("libcudart.so.12")   # the runtime torch has loaded
    used_mem_high = ctypes.c_int(8)       # cudaMemPoolAttrUsedMemHigh
    pool = ctypes.c_void_p()
    assert rt.cudaDeviceGetDefaultMemPool(ctypes.byref(pool), ctypes.c_int(torch.cuda.current_device())) == 0

    def high():
        v = ctypes.c_uint64(0)
        assert rt.cudaMemPoolGetAttribute(pool, used_mem_high, ctypes.byref(v)) == 0
        return v.value

    dev = _inputs(3_000_017, 4)
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    args = [t.data_ptr() for t in dev] + [dev[0].numel(), 0.6, 0.1, 2e-3, out.data_ptr(),
                                          torch.cuda.current_stream().cuda_stream]
    torch.cuda.synchronize()
    zero = ctypes.c_uint64(0)
    assert rt.cudaMemPoolSetAttribute(pool, used_mem_high, ctypes.byref(zero)) == 0
    before = high()
    for _ in range(2):
        pb.check(pb.lib.pnt_op_calc_dt_noalloc(*args))
    torch.cuda.synchronize()
    assert high() == before
    # the control: the allocating entry point does move the mark
    pb.check(pb.lib.pnt_op_calc_dt(*args))
    torch.cuda.synchronize()
    assert high() > before
