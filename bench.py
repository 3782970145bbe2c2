#!/usr/bin/env python
"""Benchmark of the hydro cycle: zone-cycles/s on the 1920^2 Sedov deck.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one hydro cycle (Hydro::doCycle plus the Driver's dt update) over
the whole mesh.  `value` is device-timed throughput with the state resident
in HBM (CUDA events on the library's stream around K graph-replayed cycles,
barrier + synchronize on both sides, max over ranks).  With N > 1 (torchrun,
one rank per GPU) each rank runs an independent replica: the single-mesh
path has no multi-GPU decomposition in this build, so scaling is weak.

The headline path is the mixed-precision cycle (FP32 side forces, FP64
kinematics/volumes/work/dt; `--precision fp64` selects the plain cycle); the
plain FP64 cycle is timed beside it on the same deck and the headline path's
relative L1 errors against it are reported.

`e2e` runs the same K cycles through the C ABI from host buffers: state
uploaded from pinned host memory, one pnt_hydro_cycle call per step (each
returns that step's dt/time to the host), final fields downloaded.

`--impl reference` times the reference's CPU path on this machine's host
cores: the oracle (a restatement of the reference's *OMPTask loops; the
reference itself needs the Legion runtime and cannot be built here) with
all host threads, one cycle of the same deck per step.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "pennant-legion_b200")
ORACLE_DIR = os.path.join(ROOT, "oracle")
sys.path.insert(0, PKG)

METRIC = "zone-cycles/s on 1920² Sedov, learned+FP32 vs plain FP64 GPU at ≤1e-3 L1 err"
UNIT = "zone-cycles/s"
DEFAULT_DECK = os.path.join(PKG, "decks", "sedov1920.pnt")


def algorithmic_bytes(nump, nums, numz):
    """Compulsory HBM bytes of the 3-pass schedule (per cycle and per pass)."""
    a = 32 * nump + 44 * numz + 52 * nums   # pass A: px0,pu0; 4 zone fields + offsets; mapsp1,smf; 3 side outputs; zp
    b = 68 * nump + 28 * nums               # pass B: CSR offsets, corner ids, corner mass/force, px0,pu0 -> px,pu
    c = 64 * nump + 20 * nums + 60 * numz   # pass C: 4 point fields; mapsp1, sfp+sfq; zone fields in/out
    return {"cycle": a + b + c, "A": a, "B": b, "C": c}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: str):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.gpu, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        smax = [num(r[2]) for r in rows if num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        pw = [num(r[3]) for r in rows if num(r[3]) is not None]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows), "power_w_max": max(pw) if pw else None}


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_baseline(deck_path, seconds=15.0, threads=None, warmup=1, max_cycles=None):
    """Times the oracle (OpenMP restatement of the reference's CPU loops)."""
    sys.path.insert(0, ORACLE_DIR)
    from oracle import Oracle
    threads = threads or host_cores()
    o = Oracle(deck_path, threads=threads)
    numz = o.numz
    for _ in range(warmup):
        o.cycle()
    n, t0 = 0, time.perf_counter()
    while True:
        st = o.cycle()
        n += 1
        el = time.perf_counter() - t0
        if st or o.done or el >= seconds or (max_cycles and n >= max_cycles):
            break
    return {"value": numz * n / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} cycles of {os.path.basename(deck_path)} ({numz} zones) after {warmup} warm-up "
                      f"cycle(s), {el:.1f} s, oracle with OpenMP loops of the reference's *OMPTask shape"}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    sys.path.insert(0, ORACLE_DIR)
    from oracle import Oracle
    threads = host_cores()
    o = Oracle(args.deck, threads=threads)
    numz = o.numz
    for _ in range(args.warmup):
        o.cycle()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        st = o.cycle()
        times.append(time.perf_counter() - t0)
        if st or o.done:
            break
    total = sum(times)
    val = numz * len(times) / total
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": world,
        "steps": len(times), "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": os.path.basename(args.deck), "zones": numz, "path": "cpu-openmp-port"},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{len(times)} cycles of {os.path.basename(args.deck)} after {args.warmup} "
                                   f"warm-up cycles; oracle restating the reference's *OMPTask loops "
                                   f"(the reference needs Legion and cannot be built here)"},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--deck", default=DEFAULT_DECK)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="path of the headline value; the plain FP64 cycle is always timed beside it")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, rank, world)

    import numpy as np
    import torch
    import torch.distributed as dist
    import pennant_b200 as pb

    torch.cuda.set_device(local_rank)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local_rank))

    mesh = pb.Mesh(deck=pb.Deck(path=args.deck))
    nump, numz, nums = mesh.nump, mesh.numz, mesh.nums
    ab = algorithmic_bytes(nump, nums, numz)

    def make(precision):
        d = pb.Deck(path=args.deck)
        d.set("precision", precision)
        return pb.Hydro(mesh, d.params(), device=local_rank)

    def barrier_sync():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    gpu_index = os.environ.get("CUDA_VISIBLE_DEVICES", str(local_rank)).split(",")[local_rank if world > 1 else 0]

    def timed(h, sample_clocks):
        h.time_cycles(args.warmup)      # graph capture + W cycles
        barrier_sync()
        clocks = None
        if sample_clocks:
            with ClockSampler(gpu_index) as clk:
                barrier_sync()
                ms = h.time_cycles(args.steps)
                barrier_sync()
            clocks = clk.summary()
        else:
            barrier_sync()
            ms = h.time_cycles(args.steps)
            barrier_sync()
        s = h.scalars()
        if s["status"] or s["cycle"] < args.warmup + args.steps:
            raise SystemExit(f"run stopped early: {s}")
        return max_over_ranks(ms), clocks

    names = ["A", "B", "C", "finalize"]
    head = make(args.precision)
    ms_head, clocks = timed(head, True)
    kms_head = head.time_kernels(10)
    if args.precision == "fp64":
        ref64, ms_64, kms_64 = head, ms_head, kms_head
    else:
        ref64 = make("fp64")
        ms_64, _ = timed(ref64, False)
        kms_64 = ref64.time_kernels(10)
    value = world * numz * args.steps / (ms_head / 1e3)
    value_64 = world * numz * args.steps / (ms_64 / 1e3)

    # accuracy of the headline path against the FP64 cycle after the same
    # number of cycles (the FP64 cycle is bit-identical to the CPU oracle)
    def l1(a, b):
        return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))

    err = None
    if ref64 is not head:
        c1, c2 = head.scalars()["cycle"], ref64.scalars()["cycle"]
        assert c1 == c2, (c1, c2)
        err = {"zr": l1(head.download("zr"), ref64.download("zr")),
               "ze": l1(head.download("ze"), ref64.download("ze")),
               "u": l1(np.hypot(*head.download("pu").T), np.hypot(*ref64.download("pu").T)),
               "cycles": c1, "time": head.scalars()["time"]}
        ref64.close()

    hbm, peak_kind = measured_peaks()
    dom = int(np.argmax(kms_head[:3]))
    if args.precision == "mixed":
        per_launch = {"A": 32 * nump + 44 * numz + 32 * nums, "B": 68 * nump + 16 * nums,
                      "C": 64 * nump + 12 * nums + 60 * numz}
    else:
        per_launch = {k: ab[k] for k in ("A", "B", "C")}
    ach_dom = per_launch[names[dom]] / (kms_head[dom] / 1e3) / 1e9
    ach_cycle = ab["cycle"] * args.steps / (ms_head / 1e3) / 1e9

    # end to end through the C ABI with pinned host buffers
    fields = ["px", "pu", "zr", "ze", "zm", "zetot", "zwrate", "zvol"]
    host = {}
    for k in fields:
        arr = head.download(k)
        pin = torch.empty(arr.shape, dtype=torch.float64, pin_memory=True).numpy()
        pin[...] = arr
        host[k] = pin
    outs = {k: torch.empty(head._shape(k), dtype=torch.float64, pin_memory=True).numpy()
            for k in ("zr", "ze", "zp", "px", "pu")}
    barrier_sync()
    t0 = time.perf_counter()
    for k in fields:
        pb.check(pb.lib.pnt_hydro_upload(head.h, pb.FIELDS[k], host[k].ctypes.data, host[k].nbytes))
    for _ in range(args.steps):
        head.cycle()
    for k, arr in outs.items():
        pb.check(pb.lib.pnt_hydro_download(head.h, pb.FIELDS[k], arr.ctypes.data, arr.nbytes))
    barrier_sync()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    h2d = sum(a.nbytes for a in host.values())
    d2h = sum(a.nbytes for a in outs.values()) + 72 * args.steps
    head.close()

    result = None
    if rank == 0:
        path = ("mixed precision: FP32 edge/corner geometry and TTS/QCS side forces, FP64 point kinematics, "
                "volumes, EOS, work and dt; plain QCS" if args.precision == "mixed"
                else "plain FP64 (bitwise parity path)")
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_head / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if args.precision == "mixed" else "f64", "data": "synthetic",
            "config": {"workload": f"{os.path.basename(args.deck)} ({numz} zones, {nums} sides, {nump} points)",
                       "path": path, "cycles_per_step": 1, "parallelism": f"replicas x{world}",
                       "l2": "working set > 1 GB per GPU >> 126 MB L2 (no flush needed)",
                       "fp64_plain": {"value": value_64, "ms_per_step": ms_64 / args.steps,
                                      "kernel_ms": dict(zip(names, kms_64))},
                       "speedup_vs_fp64": value / value_64,
                       "l1_rel_err_vs_fp64": err},
            "roofline": {"bound": "hbm", "kernel": f"pass {names[dom]} ({args.precision})", "achieved": ach_dom,
                         "peak": hbm, "unit": "GB/s", "frac": ach_dom / hbm, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": per_launch[names[dom]], "launch_ms": kms_head[dom],
                         "traffic": None},
            "roofline_cycle": {"achieved": ach_cycle, "peak": hbm, "unit": "GB/s", "frac": ach_cycle / hbm,
                               "algorithmic_bytes_per_cycle": ab["cycle"],
                               "note": "FP64 schedule bytes B = 164 Np + 100 Ns + 104 Nz for every path"},
            "kernel_ms": dict(zip(names, kms_head)),
            "e2e": {"value": world * numz * args.steps / e2e_s, "unit": UNIT,
                    "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                    "note": "state uploaded from pinned host memory once per timed run, one pnt_hydro_cycle "
                            "call per step (returns the step's dt/time), final fields downloaded; "
                            "bytes per step are run totals / steps"},
            "gpu_launches": 4 * args.steps,
            "clocks": clocks,
        }
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            result["cpu_baseline"] = cpu_baseline(args.deck, seconds=args.cpu_seconds)
        print(json.dumps(result), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
