"""Per-task operators on caller device arrays (needs a GPU)."""
import numpy as np
import pytest
import torch

from conftest import golden
from oracle import Oracle
import pennant_b200 as pb

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def calc_dt_ref(zdl, zdu, zss, zvol, zvol0, cfl, cflv, dtlast):
    """calcDtNew/calcDvol/calcDt (Hydro.cc:1591-1667) in numpy: same per-zone
    IEEE operations; min/max folds that skip NaN, as the serial loops do."""
    inner = np.where(zss < 1e-99, 1e-99, zss)
    cdu = np.where(zdu < inner, inner, zdu)
    zdthyd = zdl * cfl / cdu
    dvov = np.abs((zvol - zvol0) / zvol0)
    ok = ~np.isnan(zdthyd)
    dtnew = min(1e99, zdthyd[ok].min()) if ok.any() else 1e99
    ok = ~np.isnan(dvov)
    dvovmax = max(1e-99, dvov[ok].max()) if ok.any() else 1e-99
    dtrec = 1e99
    if dtnew < dtrec:
        dtrec = dtnew
    d2 = dtlast * cflv / dvovmax
    if d2 < dtrec:
        dtrec = d2
    return dtrec, dtnew, dvovmax


def run_op(arrs, cfl, cflv, dtlast):
    dev = [_dev(a) for a in arrs]
    out = torch.full((3,), -1.0, dtype=torch.float64, device="cuda")
    n = len(arrs[0])
    stream = torch.cuda.current_stream().cuda_stream
    pb.op_calc_dt(*(t.data_ptr() for t in dev), n, cfl, cflv, dtlast, out.data_ptr(), stream)
    torch.cuda.synchronize()
    return tuple(out.cpu().numpy().tolist())


@pytest.mark.parametrize("name", ["sedov.pnt", "noh.pnt", "leblanc.pnt"])
def test_op_calc_dt_matches_oracle_cycle(name):
    o = Oracle(golden(name))
    for _ in range(3):
        assert o.cycle() == 0
    arrs = [o.field(k) for k in ("zdl", "zdu", "zss", "zvol", "zvol0")]
    p = pb.Deck(path=golden(name)).params()
    got = run_op(arrs, p.cfl, p.cflv, o.scalar("dt"))
    assert got == (o.scalar("dtrec"), o.scalar("dtnew"), o.scalar("dvovmax"))


@pytest.mark.parametrize("n", [1, 2047, 2048, 2049, 1_000_003])
def test_op_calc_dt_ragged_sizes(n):
    rng = np.random.default_rng(n)
    zdl = rng.uniform(1e-3, 1e-1, n)
    zdu = rng.uniform(0, 2, n)
    zss = rng.uniform(0, 1, n)
    zvol0 = rng.uniform(0.5, 1.5, n)
    zvol = zvol0 * (1 + rng.normal(0, 1e-3, n))
    got = run_op([zdl, zdu, zss, zvol, zvol0], 0.6, 0.1, 1e-3)
    assert got == calc_dt_ref(zdl, zdu, zss, zvol, zvol0, 0.6, 0.1, 1e-3)


def test_op_calc_dt_empty_and_nan():
    got = run_op([np.zeros(0)] * 5, 0.6, 0.1, 1e-3)
    assert got == calc_dt_ref(*([np.zeros(0)] * 5), 0.6, 0.1, 1e-3)
    n = 5000
    rng = np.random.default_rng(7)
    zdl, zdu, zss = rng.uniform(1e-3, 1e-1, n), rng.uniform(0, 2, n), rng.uniform(0, 1, n)
    zvol0 = rng.uniform(0.5, 1.5, n)
    zvol = zvol0 * 1.01
    zdl[17] = np.nan           # NaN terms never win the fold
    zvol0[99] = 0.0            # |dV/0| = inf wins the max, as in the reference
    got = run_op([zdl, zdu, zss, zvol, zvol0], 0.6, 0.1, 1e-3)
    assert got == calc_dt_ref(zdl, zdu, zss, zvol, zvol0, 0.6, 0.1, 1e-3)


def test_op_calc_dt_rejects_bad_arguments():
    assert pb.lib.pnt_op_calc_dt(None, None, None, None, None, 5, 0.6, 0.1, 1.0, None, None) == \
        pb.PNT_ERR_INVALID_ARG
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    assert pb.lib.pnt_op_calc_dt(None, None, None, None, None, -1, 0.6, 0.1, 1.0, out.data_ptr(), None) == \
        pb.PNT_ERR_INVALID_ARG
