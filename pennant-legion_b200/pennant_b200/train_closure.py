"""Trains the learned QCS closure on the GPU and writes its parameter file.

Training data are harvested from seeded FP64 runs (pnt_hydro_harvest: the
exact QCS corner forces of the cycle about to run):

  * Sedov 480 x 480 to t = 1.0 (the FP64 drop-in case),
  * the Leblanc-type tube 2880 x 288 to t = 6.0 (the mixed-precision case),
  * instances of the seeded 256-instance Sedov batch (N log-uniform in
    [32, 512], E0 in [0.1, 1], gamma in [1.4, 5/3]) to t = 0.5,

every `every` cycles, each eligible corner kept with a per-run probability.
The network is trained with the library's own BF16 tensor-core forward and
backward kernels (pnt_closure_train, Adam, cosine learning-rate decay) on
the samples whose compression lies within the closure's range, with 2% held
out for the validation loss.  PyTorch provides device buffers and the
shuffle only.

Usage:  python -m pennant_b200.train_closure [--out PATH] [--samples N] ...
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time

import numpy as np
import torch

import pennant_b200 as pb

_HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(os.path.dirname(_HERE), "closure", "qcs_mlp.bin")
sys.path.insert(0, os.path.join(os.path.dirname(_HERE), "decks"))
from make_decks import leblanc, sedov, sedov_batch  # noqa: E402


def harvest_runs(quick: bool):
    """(name, deck text, harvest every k cycles, share of the sample budget)."""
    if quick:
        return [("sedov96", sedov(96, tstop=0.5), 10, 1.0),
                ("leblanc576x58", leblanc(576, 58, tstop=2.0), 10, 1.0)]
    runs = [("sedov480", sedov(480, tstop=1.0), 20, 0.35),
            ("leblanc2880x288", leblanc(2880, 288, tstop=6.0), 20, 0.30)]
    insts = sedov_batch(256)
    for i in range(0, 256, 16):   # 16 instances of the batch, every 16th
        runs.append((f"batch{i}_n{insts[i]['n']}", insts[i]["text"], 10, 0.35 / 16))
    return runs


def harvest(args, dev):
    """Harvests every run with a keep probability steered so that its share of
    the budget is spread over its whole simulated time."""
    cap = int(args.samples)
    feats = torch.empty((cap, pb.CLOSURE_IN), dtype=torch.float32, device=dev)
    targs = torch.empty((cap, 4), dtype=torch.float32, device=dev)
    sides = torch.empty((cap,), dtype=torch.int32, device=dev)
    count = 0
    log = []
    runs = harvest_runs(args.quick)
    wsum = sum(r[3] for r in runs)
    for k, (name, text, every, share) in enumerate(runs):
        t0 = time.time()
        d = pb.Deck(text=text)
        tstop = d.get_double("tstop", 1e99)
        h = pb.Hydro(pb.Mesh(deck=d), d.params())
        start = count
        budget = int(cap * share / wsum)
        limit = min(cap, start + budget)
        keep, per_harvest = 0.01, None
        nharv = 0
        while True:
            s = h.scalars()
            if s["done"] or count >= limit:
                break
            if per_harvest is not None:
                left = max(tstop - s["time"], 0.0)
                harvests_left = max(left / max(s["dt"], 1e-300) / every, 1.0)
                keep = min(1.0, (limit - count) / (harvests_left * max(per_harvest, 1.0)))
            before = count
            count = h.harvest(args.dead, keep, args.seed + 7919 * k + nharv, feats.data_ptr(), targs.data_ptr(),
                              sides.data_ptr(), limit, count)
            nharv += 1
            est = (count - before) / keep
            per_harvest = est if per_harvest is None else 0.7 * per_harvest + 0.3 * est
            h.run(max_cycles=every)
        s = h.scalars()
        log.append({"run": name, "cycles": s["cycle"], "time": s["time"], "harvests": nharv,
                    "samples": count - start, "seconds": time.time() - t0})
        print(f"harvest {name}: {s['cycle']} cycles to t={s['time']:.4g}, {nharv} harvests, "
              f"{count - start} samples", flush=True)
        h.close()
    return feats[:count], targs[:count], log


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--samples", type=float, default=5e7)
    ap.add_argument("--epochs", type=float, default=12)
    ap.add_argument("--rows-per-step", type=int, default=32768)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--dead", type=float, default=1e-6)
    ap.add_argument("--rho-max", type=float, default=0.5)
    ap.add_argument("--ood-kappa", type=float, default=6.0)
    ap.add_argument("--seed", type=int, default=12345)
    ap.add_argument("--quick", action="store_true", help="small harvest for a smoke run")
    args = ap.parse_args(argv)
    dev = torch.device("cuda:0")
    t_start = time.time()

    feats, targs, hlog = harvest(args, dev)
    # the closure's range: compression rho <= rho_max (input 11), with a margin
    keep = feats[:, 11] <= args.rho_max * 1.1
    feats, targs = feats[keep], targs[keep]
    n_all = feats.shape[0]
    g = torch.Generator(device=dev)
    g.manual_seed(args.seed)
    perm = torch.randperm(n_all, generator=g, device=dev)
    feats, targs = feats[perm].contiguous(), targs[perm].contiguous()
    n_val = max(1024, n_all // 50)
    n_tr = n_all - n_val

    clo = pb.Closure(seed=args.seed)
    clo.set(thresholds=np.array([args.dead, args.rho_max, args.ood_kappa], np.float32))
    clo.fit_normalization(feats.data_ptr(), targs.data_ptr(), n_tr)
    x = torch.empty((n_all, 16), dtype=torch.bfloat16, device=dev)
    t = torch.empty((n_all, 4), dtype=torch.float32, device=dev)
    clo.prepare(feats.data_ptr(), targs.data_ptr(), n_all, x.data_ptr(), t.data_ptr())
    xv, tv = x[n_tr:], t[n_tr:]

    steps = int(math.ceil(args.epochs * n_tr / args.rows_per_step))
    chunk = 100
    losses, val = [], []
    t0 = time.time()
    done = 0
    while done < steps:
        k = min(chunk, steps - done)
        lr = 1e-5 + 0.5 * (args.lr - 1e-5) * (1 + math.cos(math.pi * done / steps))
        ls = clo.train(x.data_ptr(), t.data_ptr(), n_tr, (done * args.rows_per_step) % n_tr, k,
                       args.rows_per_step, lr)
        losses.append(float(ls.mean()))
        done += k
        if (done // chunk) % 10 == 0 or done == steps:
            _, vl = clo.gradient(xv.data_ptr(), tv.data_ptr(), n_val)
            val.append((done, vl))
            print(f"step {done}/{steps} lr {lr:.2e} train {losses[-1]:.4e} val {vl:.4e}", flush=True)
    torch.cuda.synchronize()
    train_s = time.time() - t0
    _, vl = clo.gradient(xv.data_ptr(), tv.data_ptr(), n_val)
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    clo.save(args.out)
    info = {
        "samples_harvested": sum(r["samples"] for r in hlog), "samples_in_range": n_all,
        "train_rows": n_tr, "val_rows": n_val, "steps": steps, "rows_per_step": args.rows_per_step,
        "epochs": args.epochs, "lr": args.lr, "seed": args.seed, "dead": args.dead,
        "rho_max": args.rho_max, "ood_kappa": args.ood_kappa, "final_val_mse": vl,
        "train_seconds": train_s, "total_seconds": time.time() - t_start,
        "train_loss_per_100_steps": losses, "val_loss": val, "harvest": hlog,
    }
    with open(os.path.splitext(args.out)[0] + ".json", "w") as f:
        json.dump(info, f, indent=1)
    print(json.dumps({k: v for k, v in info.items() if not isinstance(v, list)}), flush=True)


if __name__ == "__main__":
    main()
