"""Writes the benchmark decks of this project (generated, not from the reference).

Sedov: rect N x N over [0, 1.125]^2, a total energy E0 = 0.25 deposited in
the single zone at the origin.  The zone's RZ volume per radian is h^3/2
(h = 1.125/N; the volume formula of Mesh.cc:976-977), so the specific energy
is einitsub = E0 / (2*pi * h^3/2) = E0 / (pi*h^3).  By the same mapping the
reference's test/sedov/sedov.pnt (45^2, einitsub 5027.7) deposits E0 ~= 0.247.
dtinit scales as 1e-4 * (48/N)^2.5 so the first step resolves the deposit.

Leblanc: rect 2880 x 288 over [0, 9] x [0, 0.9], rho 1 / e 0.1 for x < 3 and
rho 1e-3 / e 1e-7 for x >= 3 (x is the radial coordinate), reflecting walls,
q1/q2/ssmin/dtinit of test/leblancbig/leblancbig.pnt.

Usage: python make_decks.py  (rewrites the .pnt files next to this script)
"""
import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def sedov(n: int, e0: float = 0.25, tstop: float = 1.0, dtinit: float | None = None,
          gamma: float | None = None, extra: str = "") -> str:
    h = 1.125 / n
    einit = e0 / (math.pi * h ** 3)
    if dtinit is None:
        dtinit = 1e-4 * (48.0 / n) ** 2.5
    g = f"gamma   {gamma!r}\n" if gamma is not None else ""
    return (f"tstop   {tstop!r}\n"
            f"meshtype rect\n"
            f"meshparams {n} {n} 1.125 1.125\n"
            f"subregion 0.0 {h!r}  0.0 {h!r}\n"
            f"rinit   1.0\neinit   0.0\n"
            f"rinitsub 1.0\n"
            f"einitsub {einit!r}\n"
            f"{g}"
            f"bcx     0.0 1.125\nbcy     0.0 1.125\n"
            f"ssmin   0.1\nq1      0.1\nq2      1.0\nalfa    0.5\n"
            f"cfl     0.6\ncflv    0.1\n"
            f"dtinit  {dtinit!r}\n"
            f"dtreport 100\n{extra}")


def leblanc(nx: int = 2880, ny: int = 288, tstop: float = 6.0, extra: str = "") -> str:
    return (f"tstop   {tstop!r}\n"
            f"meshtype rect\n"
            f"meshparams {nx} {ny} 9.0 0.9\n"
            f"subregion 3.0 9.0  0.0 0.9\n"
            f"rinit   1.0\neinit   0.1\n"
            f"rinitsub 1.0e-3\neinitsub 1.0e-7\n"
            f"bcx     0.0 9.0\nbcy     0.0 0.9\n"
            f"ssmin   0.1\nq1      0.3\nq2      2.0\n"
            f"dtinit  1.e-3\n"
            f"dtreport 100\n{extra}")


def sedov_batch(count: int = 256, seed: int = 20240601, nmin: int = 32, nmax: int = 512,
                tstop: float = 0.5) -> list[dict]:
    """The batched workload: `count` Sedov instances, side length N drawn
    log-uniform in [nmin, nmax], deposited energy E0 uniform in [0.1, 1.0],
    gamma uniform in [1.4, 5/3], each run to `tstop`; numpy's PCG64 seeded
    with `seed`.  dtinit = min(1e-4, 1e-4 (48/N)^2.5 sqrt(0.25/E0)): the 48^2
    deck's 1e-4 rescaled by the first step's CFL limit h/c, c ~ sqrt(E0/h^3),
    so that no instance inverts a zone on its first step.  Returns dicts with
    keys n, e0, gamma, text."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        e0 = float(rng.uniform(0.1, 1.0))
        gamma = float(rng.uniform(1.4, 5.0 / 3.0))
        dtinit = min(1e-4, 1e-4 * (48.0 / n) ** 2.5 * math.sqrt(0.25 / e0))
        out.append({"n": n, "e0": e0, "gamma": gamma,
                    "text": sedov(n, e0=e0, tstop=tstop, dtinit=dtinit, gamma=gamma)})
    return out


DECKS = {
    "sedov48.pnt": sedov(48),      # CPU-runnable case, FP64, t = 1.0
    "sedov480.pnt": sedov(480),    # FP64 drop-in parity case, t = 1.0
    "sedov1920.pnt": sedov(1920),  # headline case
    "sedov1024.pnt": sedov(1024),  # profiling case: ~0.4 GB on the device, > L2
    "leblanc2880x288.pnt": leblanc(),
}


def main() -> None:
    for name, text in DECKS.items():
        with open(os.path.join(HERE, name), "w") as f:
            f.write(text)


if __name__ == "__main__":
    main()
