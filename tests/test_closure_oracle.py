"""CPU checks of the closure oracle (oracle/closure_oracle.py), the checker
the GPU closure tests compare against."""
import sys

import numpy as np

from conftest import DECKS
from oracle import Oracle
import closure_oracle as co

sys.path.insert(0, DECKS)
from make_decks import sedov  # noqa: E402


def random_net(seed, scale=1.0):
    rng = np.random.default_rng(seed)
    p = (rng.standard_normal(co.N_PARAMS) * 0.3 * scale).astype(np.float32)
    return p


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7, 1.0 + 3 * 2 ** -8, -2.5, 0.0, 1e-30], np.float32)
    r = co.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: even mantissa (1.0) wins;
    # 1 + 3*2^-8 ties between 1 + 2^-7 and 1 + 2^-6: even (1 + 2^-6) wins
    assert list(r[:4]) == [1.0, 1.0, 1.0 + 2 ** -7, 1.0 + 2 ** -6]
    assert r[4] == -2.5 and r[5] == 0.0
    assert abs(r[6] - 1e-30) / 1e-30 < 2 ** -8


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = random_net(1).astype(np.float64)
    x = rng.standard_normal((24, 14))
    t = rng.standard_normal((24, 4))
    _, g = co.loss_grad(p, x, t, bf16_round=False)
    idx = rng.choice(co.N_PARAMS, 60, replace=False)
    idx = np.concatenate([idx, [co.B1, co.B2 + 3, co.B3 + 1, co.W3 + 5]])
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (co.loss_grad(pp, x, t, False)[0] - co.loss_grad(pm, x, t, False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])) + 1e-8, (i, fd, g[i])


def test_bf16_gradient_close_to_exact():
    """The rounded form differs from the exact gradient only by BF16 noise."""
    rng = np.random.default_rng(4)
    p = random_net(2)
    x = co.bf16(rng.standard_normal((512, 14)).astype(np.float32))
    t = rng.standard_normal((512, 4)).astype(np.float32)
    l0, g0 = co.loss_grad(p, x, t, bf16_round=False)
    l1, g1 = co.loss_grad(p, x, t, bf16_round=True)
    assert abs(l1 - l0) / l0 < 1e-2
    assert np.linalg.norm(g1 - g0) / np.linalg.norm(g0) < 3e-2


def test_corner_features_of_an_oracle_run():
    o = Oracle(text=sedov(24, tstop=1.0))
    o.run(60)
    f, tg, elig = co.corner_features(o, 1e-6, 1.0 * 0.25 * (5 / 3 + 1), 0.1)
    assert elig.sum() > 50
    fe, te = f[elig], tg[elig]
    assert np.all(np.isfinite(fe)) and np.all(np.isfinite(te))
    # unit-scaled velocity differences, rho in (0, 1), unit direction
    assert np.abs(fe[:, :6]).max() <= 1.0 + 1e-6
    assert fe[:, 11].min() > 0 and fe[:, 11].max() < 1
    assert np.allclose(np.hypot(fe[:, 12], fe[:, 13])[np.hypot(fe[:, 12], fe[:, 13]) > 0], 1.0, atol=1e-5)
    # targets are the QCS corner forces in the corner frame over zrp D (a D + b c): bounded
    assert np.abs(te).max() < 20
