"""Runs the CPU oracle on a deck to its stop condition and writes a compact
fingerprint of the final state (JSON) for the GPU parity tests.

The fingerprint holds, per field, the SHA-256 of the float64 array bytes
(bit-exact check), its sum and L1 norm, and the exact values (float.hex) at
evenly spaced indices, so a mismatch can still be measured against the 1e-11
relative bound.

Usage: python tests/golden/make_fingerprint.py <deck.pnt> <out.json> [cstop]

With cstop the run stops after that many cycles (a "cstop N" line is added
to the deck text; the decks used this way have no cstop of their own).
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
from oracle import Oracle  # noqa: E402

FIELDS = ("zr", "ze", "zp", "zetot", "zvol", "zwrate", "px", "pu")
NSAMPLE = 256


def fingerprint(arrays: dict, meta: dict) -> dict:
    out = dict(meta)
    out["fields"] = {}
    for k, a in arrays.items():
        a = np.ascontiguousarray(a, dtype="<f8")
        flat = a.reshape(-1)
        idx = np.unique(np.linspace(0, flat.size - 1, NSAMPLE).astype(np.int64))
        out["fields"][k] = {
            "sha256": hashlib.sha256(flat.tobytes()).hexdigest(),
            "sum": float(flat.sum()),
            "l1": float(np.abs(flat).sum()),
            "idx": idx.tolist(),
            "val": [float(v).hex() for v in flat[idx]],
        }
    return out


def main(deck: str, out_json: str, cstop: int = 0) -> None:
    t0 = time.time()
    if cstop:
        text = open(deck).read()
        if any(line.split()[:1] == ["cstop"] for line in text.splitlines()):
            raise SystemExit(f"{deck} has a cstop of its own")
        o = Oracle(text=text.rstrip("\n") + f"\ncstop {cstop}\n")
    else:
        o = Oracle(deck)
    st = o.run()
    if st:
        raise SystemExit(f"oracle failed with status {st}")
    meta = {"deck": os.path.basename(deck), "cycle": o.num("cycle"),
            "time": float(o.scalar("time")).hex(), "dt": float(o.scalar("dt")).hex(),
            "oracle_seconds": round(time.time() - t0, 1)}
    if cstop:
        meta["cstop"] = cstop
    fp = fingerprint({k: o.field(k) for k in FIELDS}, meta)
    with open(out_json, "w") as f:
        json.dump(fp, f, indent=0)
    print(f"{deck}: {meta['cycle']} cycles, {meta['oracle_seconds']} s")


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2], int(sys.argv[3]) if len(sys.argv) > 3 else 0)
