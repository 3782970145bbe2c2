"""CPU restatement of the learned QCS closure (numpy).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the GPU
harvest, inference and training kernels; never by the product library.

* corner_features(): the 14 inputs and the normalised QCS targets of every
  corner, from the oracle's fields of one cycle (pxp, pu0, zxp, zuc, zss,
  zrp, cqe1, cqe2; QCS.cc:116-327 for the targets' source, setCornerDiv
  and setQCnForce).
* forward() / loss_grad(): the 14-64-64-4 GELU network with the GPU
  kernels' rounding points -- inputs, hidden activations and the backward
  deltas rounded to BF16, products accumulated exactly (float64 here, FP32
  on the GPU) -- or with no rounding at all (bf16=False), the form the
  finite-difference check uses.
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID, N_OUT = 14, 64, 4
W1, B1 = 0, 64 * 14
W2 = B1 + 64
B2 = W2 + 64 * 64
W3 = B2 + 64
B3 = W3 + 4 * 64
N_PARAMS = B3 + 4
GELU_C = np.float32(0.7978845608028654)
GELU_A = np.float32(0.044715)


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest bfloat16 (ties to even), as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def unpack(p: np.ndarray):
    p = np.asarray(p)
    return (p[W1:B1].reshape(64, 14), p[B1:W2], p[W2:B2].reshape(64, 64), p[B2:W3],
            p[W3:B3].reshape(4, 64), p[B3:N_PARAMS])


def gelu(x, dtype=np.float32):
    x = x.astype(dtype)
    c, a = dtype(GELU_C), dtype(GELU_A)
    th = np.tanh(c * (x + a * x * x * x))
    y = dtype(0.5) * x * (dtype(1) + th)
    dy = dtype(0.5) * (dtype(1) + th) + dtype(0.5) * x * (dtype(1) - th * th) * c * (dtype(1) + dtype(3) * a * x * x)
    return y, dy


def normalise(feats: np.ndarray, norm: np.ndarray) -> np.ndarray:
    """(f - mean) * (1 / std) in float32, as the GPU forms it."""
    mean = norm[:14].astype(np.float32)
    istd = (np.float32(1) / norm[14:28].astype(np.float32)).astype(np.float32)
    return ((feats.astype(np.float32) - mean) * istd).astype(np.float32)


def forward(params: np.ndarray, x: np.ndarray, bf16_round: bool = True):
    """Network on normalised inputs x [n][14]; returns normalised outputs and
    the intermediates (z1, h1, z2, h2)."""
    w1, b1, w2, b2, w3, b3 = unpack(params)
    if bf16_round:
        r = bf16
        w1, w2, w3 = r(w1).astype(np.float64), r(w2).astype(np.float64), r(w3).astype(np.float64)
        xin = r(x).astype(np.float64)
        z1 = (xin @ w1.T).astype(np.float32) + b1.astype(np.float32)
        h1f, _ = gelu(z1)
        h1 = r(h1f).astype(np.float64)
        z2 = (h1 @ w2.T).astype(np.float32) + b2.astype(np.float32)
        h2f, _ = gelu(z2)
        h2 = r(h2f).astype(np.float64)
        y = (h2 @ w3.T).astype(np.float32) + b3.astype(np.float32)
        return y, (xin, z1, h1, z2, h2)
    xin = x.astype(np.float64)
    z1 = xin @ w1.T.astype(np.float64) + b1
    h1, _ = gelu(z1, np.float64)
    z2 = h1 @ w2.T.astype(np.float64) + b2
    h2, _ = gelu(z2, np.float64)
    y = h2 @ w3.T.astype(np.float64) + b3
    return y, (xin, z1, h1, z2, h2)


def loss_grad(params: np.ndarray, x: np.ndarray, t: np.ndarray, bf16_round: bool = True):
    """Mean squared error over n rows x 4 outputs and its gradient, with the
    GPU training kernel's rounding points when bf16_round."""
    n = x.shape[0]
    w1, b1, w2, b2, w3, b3 = unpack(params)
    y, (xin, z1, h1, z2, h2) = forward(params, x, bf16_round)
    if bf16_round:
        r = bf16
        w2b, w3b = r(w2).astype(np.float64), r(w3).astype(np.float64)
        inv = np.float32(1.0) / np.float32(n * 4)
        d = (y - t.astype(np.float32)).astype(np.float32)
        loss = float(np.sum(d.astype(np.float64) ** 2) * float(inv))
        dy = (np.float32(2) * d * inv).astype(np.float32)
        dyb = r(dy).astype(np.float64)
        _, g2 = gelu(z2)
        dz2 = ((dyb @ w3b).astype(np.float32) * g2).astype(np.float32)
        dz2b = r(dz2).astype(np.float64)
        _, g1 = gelu(z1)
        dz1 = ((dz2b @ w2b).astype(np.float32) * g1).astype(np.float32)
        dz1b = r(dz1).astype(np.float64)
        gw3 = dyb.T @ h2
        gw2 = dz2b.T @ h1
        gw1 = dz1b.T @ xin
        gb3, gb2, gb1 = dy.astype(np.float64).sum(0), dz2.astype(np.float64).sum(0), dz1.astype(np.float64).sum(0)
    else:
        d = y - t
        loss = float(np.mean(d ** 2))
        dy = 2.0 * d / (n * 4)
        _, g2 = gelu(z2, np.float64)
        dz2 = (dy @ w3.astype(np.float64)) * g2
        _, g1 = gelu(z1, np.float64)
        dz1 = (dz2 @ w2.astype(np.float64)) * g1
        gw3, gw2, gw1 = dy.T @ h2, dz2.T @ h1, dz1.T @ xin
        gb3, gb2, gb1 = dy.sum(0), dz2.sum(0), dz1.sum(0)
    g = np.concatenate([gw1.ravel(), gb1, gw2.ravel(), gb2, gw3.ravel(), gb3])
    return loss, g


def corner_features(o, dead: float, qa: float, qb: float):
    """Inputs and normalised targets of every corner of the oracle's last
    cycle.  Returns (feats [ns][14], targets [ns][4], eligible [ns]) where
    eligible marks the corners the closure covers (cdiv < 0, outside the
    dead zone, zone without an acute corner)."""
    mapsp1, mapsp2 = o.field("mapsp1"), o.field("mapsp2")
    mapsz, mapss3 = o.field("mapsz"), o.field("mapss3")
    pxp, pu0 = o.field("pxp"), o.field("pu0")
    zxp, zuc, zss, zrp = o.field("zxp"), o.field("zuc"), o.field("zss"), o.field("zrp")
    cqe1, cqe2 = o.field("cqe1"), o.field("cqe2")
    z = mapsz
    p, pprev, pnext = mapsp1, mapsp1[mapss3], mapsp2
    xp, xpp, xpn, xz = pxp[p], pxp[pprev], pxp[pnext], zxp[z]
    up, upp, upn, uz = pu0[p], pu0[pprev], pu0[pnext], zuc[z]
    up1, up3 = 0.5 * (up + upn), 0.5 * (upp + up)
    uav = 0.25 * (((up + up1) + uz) + up3)
    css = zss[z]
    d = xz - xp
    il = 1.0 / np.hypot(d[:, 0], d[:, 1])
    cx, cy = d[:, 0] * il, d[:, 1] * il

    def rot(v):
        return np.stack([cx * v[:, 0] + cy * v[:, 1], cx * v[:, 1] - cy * v[:, 0]], axis=1)

    e1, e2 = xpp - xp, xpn - xp
    iL = 2.0 / (np.hypot(*e1.T) + np.hypot(*e2.T))
    d1, d2, dc = up - upp, upn - up, uz - up
    m2 = np.maximum(np.maximum((d1 ** 2).sum(1), (d2 ** 2).sum(1)), (dc ** 2).sum(1))
    D = np.sqrt(m2)
    live = m2 > (dead * css) ** 2
    Ds = np.where(live, D, 1.0)
    Q = qa * Ds + qb * css
    scale = Ds * Q
    am = np.hypot(*uav.T)
    ia = np.where(am > 0, 1.0 / np.where(am > 0, am, 1.0), 0.0)
    f = np.concatenate([rot(d1) / Ds[:, None], rot(d2) / Ds[:, None], rot(dc) / Ds[:, None],
                        rot(e1) * iL[:, None], rot(e2) * iL[:, None], (1.0 / il * iL)[:, None],
                        (qa * Ds / Q)[:, None], rot(uav) * ia[:, None]], axis=1)
    inv = 1.0 / (zrp[z] * scale)
    tg = np.concatenate([rot(cqe1) * inv[:, None], rot(cqe2) * inv[:, None]], axis=1)
    # cdiv < 0 (QCS.cc:193-198 form) and the acute-corner test per zone
    xq1 = 0.5 * (xp + xpn)
    xq3 = 0.5 * (xpp + xp)
    up2 = uz

    def cross(a, b):
        return a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]

    cvol = 0.5 * cross(xz - xp, xq3 - xq1)
    cdiv = (cross(up2 - up, xq3 - xq1) - cross(up3 - up1, xz - xp)) / (2.0 * cvol)
    v1, v2 = xq3 - xp, xq1 - xp
    de1, de2 = np.hypot(*(xp - xpp).T), np.hypot(*(xpn - xp).T)
    ssin = 4.0 * cross(v1, v2) / (de1 * de2)
    acute_side = ssin * ssin < 0.25
    acute_zone = np.zeros(len(zss), bool)
    np.logical_or.at(acute_zone, z, acute_side)
    eligible = (cdiv < 0) & live & ~acute_zone[z]
    return f.astype(np.float32), tg.astype(np.float32), eligible
