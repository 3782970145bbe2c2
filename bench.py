#!/usr/bin/env python
"""Benchmark of the hydro cycle: zone-cycles/s on the 1920^2 Sedov deck.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--precision learned|mixed|fp64] [--no-full-run]

A step is one hydro cycle (Hydro::doCycle plus the Driver's dt update) over
the whole mesh.  Every path is timed from the same state: the plain FP64
cycle run from the deck's initial state to cycle --start-cycles (30000,
t ~ 0.197: a developed blast whose shock has crossed a third of the mesh;
the first cycles of the deck have almost no compressing corners and would
flatter the learned closure) and copied into each path's object.  `value`
is device-timed throughput with the state resident in HBM (CUDA events on
the library's stream around K graph-replayed cycles, barrier + synchronize
on both sides, max over ranks).  With N > 1 (torchrun, one rank per GPU)
each rank runs an independent replica (weak scaling).

The headline path is the learned cycle: the mixed-precision cycle (FP32
side geometry, TTS and QCS forces; FP64 point kinematics, volumes, EOS,
work and dt) with the learned closure in place of QCS on its corners.  The
plain FP64 cycle and the mixed cycle with the plain QCS are timed beside it.
The metric's accuracy condition is measured in the same run: after the
timed windows the FP64 run continues to t = 1, the learned and mixed cycles
run the deck from its initial state to t = 1, and the line's `accuracy`
holds their relative L1 errors in density, energy and speed against the
FP64 run, with the closure's fallback fraction (--no-full-run skips this).

`e2e` runs the same K cycles through the C ABI from host buffers: state
uploaded from pinned host memory, one pnt_hydro_cycle call per step (each
returns that step's dt/time to the host), final fields downloaded.

`--impl reference` times the reference's CPU path on this machine's host
cores: the oracle (a restatement of the reference's *OMPTask loops; the
reference itself needs the Legion runtime and cannot be built here) with
all host threads, one cycle of the same deck per step from its initial
state (the plain QCS does the same work per cycle whatever the state).
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
sys.path.insert(0, os.path.join(PKG, "decks"))

METRIC = "zone-cycles/s on 1920² Sedov, learned+FP32 vs plain FP64 GPU at ≤1e-3 L1 err"
UNIT = "zone-cycles/s"
DEFAULT_DECK = os.path.join(PKG, "decks", "sedov1920.pnt")
DEFAULT_CLOSURE = os.path.join(PKG, "closure", "qcs_mlp.bin")
MLP_FLOP_PER_ROW = 2 * (16 * 64 + 64 * 64 + 64 * 16)   # tensor-core MMA shapes, padded
# DRAM bytes (read + write) of one pass A launch per zone, from the ncu
# captures of profiles/pass_a_rows_learned_sedov1024.md (learned, mixed)
# and profiles/pass_a_fp64_sedov1024.md (FP64), 1,048,576 zones each; the
# bench scales them by its zone count
PASS_A_TRAFFIC_PER_ZONE = {"learned": (109.723e6 + 81.982e6) / 1048576,
                           "mixed": (109.362e6 + 76.070e6) / 1048576,
                           "fp64": (125.973e6 + 130.137e6) / 1048576}


# FP64 thread-instructions a zone of one FP64 pass A launch (ncu
# sm__sass_thread_inst_executed_op_fp64_pred_on, 1024^2 Sedov at cycle
# 16000: profiles/pass_a_fp64_sedov1024.md), and the B200's FP64 rate a
# clock per SM (sm__sass_thread_inst_executed_op_dfma_pred_on peak)
FP64_PASS_A_INST_PER_ZONE = 907.6
FP64_INST_PER_CLOCK_PER_SM = 64


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
    """SM clocks, power and throttle reasons sampled during the timed region:
    NVML polled every 10 ms from a thread (a 100 ms window still gets ~10
    samples), else `nvidia-smi -lms 200`.  Reads only; changes nothing."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_index: str, period_s: float = 0.01):
        self.gpu = gpu_index
        self.period = period_s
        self.proc = None
        self.path = None
        self.thread = None
        self.rows = []          # (sm MHz, max sm MHz, power W, set of reasons)
        self.stop = None

    def _nvml_open(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
        except Exception:
            return None
        try:
            h = (nv.nvmlDeviceGetHandleByUUID(self.gpu) if self.gpu.startswith(("GPU-", "MIG-"))
                 else nv.nvmlDeviceGetHandleByIndex(int(self.gpu)))
            reasons_fn = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons",
                                 getattr(nv, "nvmlDeviceGetCurrentClocksThrottleReasons", None))
            bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                    nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
            smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            # one trial read of every query the thread makes: any failure
            # falls back to nvidia-smi rather than an empty record
            nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            nv.nvmlDeviceGetPowerUsage(h)
            if reasons_fn is None:
                raise RuntimeError("NVML without a clock-event reasons query")
            reasons_fn(h)
            return nv, h, reasons_fn, bits, smax
        except Exception:
            try:
                nv.nvmlShutdown()
            except Exception:
                pass
            return None

    def _poll(self, nv, h, reasons_fn, bits, smax):
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1e3
                r = reasons_fn(h)
                self.rows.append((float(sm), float(smax), pw,
                                  {n for n, b in zip(self.REASONS, bits) if r & b}))
            except Exception:
                pass
            self.stop.wait(self.period)

    def __enter__(self):
        opened = self._nvml_open()
        if opened:
            import threading
            self.stop = threading.Event()
            self.nv = opened[0]
            self.thread = threading.Thread(target=self._poll, args=opened, daemon=True)
            self.thread.start()
            time.sleep(0.05)
            return self
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
        if self.thread:
            self.stop.set()
            self.thread.join(timeout=5)
            try:
                self.nv.nvmlShutdown()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def _smi_rows(self):
        rows = []
        if not self.path or not os.path.exists(self.path):
            return rows

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9 and num(parts[1]) is not None:
                rows.append((num(parts[1]), num(parts[2]), num(parts[3]),
                             {n for i, n in enumerate(self.REASONS) if parts[5 + i].lower().startswith("active")}))
        os.unlink(self.path)
        return rows

    def summary(self):
        rows = self.rows if self.thread else self._smi_rows()
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        smax = [r[1] for r in rows if r[1] is not None]
        pw = [r[2] for r in rows if r[2] is not None]
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(set().union(*(r[3] for r in rows))), "samples": len(rows),
                "sampler": "nvml 10 ms" if self.thread else "nvidia-smi 200 ms",
                "power_w_max": max(pw) if pw else None}


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
        "config": workload_config(args.deck, numz, o.nums, o.nump, world),
        "details": {"path": "cpu-openmp-port"},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{len(times)} cycles of {os.path.basename(args.deck)} after {args.warmup} "
                                   f"warm-up cycles; oracle restating the reference's *OMPTask loops "
                                   f"(the reference needs Legion and cannot be built here)"},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(deck, numz, nums, nump, world):
    """The `config` object of the line, identical in both arms."""
    return {"workload": f"{os.path.basename(deck)} ({numz} zones, {nums} sides, {nump} points)",
            "cycles_per_step": 1, "parallelism": f"replicas x{world}",
            "l2": "working set > 1 GB per GPU >> 126 MB L2 (no flush needed)"}


def l1_rel(a, b):
    import numpy as np
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))


def run_leblanc(args, pb, np, torch):
    """The Leblanc-type tube (2880 x 288 over [0,9] x [0,0.9], rho 1 / e 0.1 for
    x < 3, rho 1e-3 / e 1e-7 beyond) to t = 6 with the FP64, mixed and learned
    cycles: whole-run zone-cycles/s (wall clock around pnt_hydro_run, which
    replays graphs and polls the done flag) and the L1 errors of rho, e, |u|
    against the FP64 run."""
    from make_decks import leblanc
    text = leblanc()
    closure = pb.Closure(path=args.closure)
    out = {"metric": "whole-run zone-cycles/s and L1 errors vs FP64", "workload": "leblanc2880x288 to t=6",
           "unit": "zone-cycles/s", "data": "synthetic"}
    ref = None
    for p in ("fp64", "mixed", "learned"):
        d = pb.Deck(text=text)
        d.set("precision", p)
        m = pb.Mesh(deck=d)
        h = pb.Hydro(m, d.params())
        if p == "learned":
            h.set_closure(closure)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s = h.run()
        wall = time.perf_counter() - t0
        r = {"cycles": s["cycle"], "time": s["time"], "wall_s": wall, "value": m.numz * s["cycle"] / wall}
        f = {k: h.download(k) for k in ("zr", "ze", "pu")}
        if p == "fp64":
            ref = f
        else:
            r["l1_rel_err_vs_fp64"] = {"rho": l1_rel(f["zr"], ref["zr"]), "e": l1_rel(f["ze"], ref["ze"]),
                                       "u": l1_rel(np.hypot(*f["pu"].T), np.hypot(*ref["pu"].T))}
        if p == "learned":
            c = h.closure_counts()
            tot = sum(v for k, v in c.items() if k not in ("error", "zones"))
            r["corner_fractions"] = {k: v / max(tot, 1) for k, v in c.items() if k not in ("error", "zones")}
        out[p] = r
        h.close()
    print(json.dumps(out), flush=True)
    return 0


def batch_record(pb, torch, count=256):
    """The seeded 256-instance Sedov batch (decks/make_decks.py sedov_batch:
    N log-uniform in [32, 512], E0 in [0.1, 1], gamma in [1.4, 5/3], t = 0.5)
    in one pnt_batch (autotuned tile shape, persistent launches, CUDA graph),
    against the same instances run one after another as single-mesh objects
    (graph replay each).  Both timings are wall clock around the runs with
    the objects already created; every 16th instance is compared bit for
    bit with its single run."""
    from make_decks import sedov_batch
    insts = sedov_batch(count)
    decks = [pb.Deck(text=i["text"]) for i in insts]
    meshes = [pb.Mesh(deck=d) for d in decks]
    params = [d.params() for d in decks]
    tuner = pb.Batch(meshes, params)
    zpt, cps, ms_tune = tuner.tune(4)
    tuner.close()
    b = pb.Batch(meshes, params)
    b.set_shape(zpt, cps)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    left = b.run()
    t_batch = time.perf_counter() - t0
    sc = [b.scalars(i) for i in range(len(insts))]
    zc = sum(m.numz * s["cycle"] for m, s in zip(meshes, sc))
    hs = [pb.Hydro(m, p) for m, p in zip(meshes, params)]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for h in hs:
        h.run()
    t_seq = time.perf_counter() - t0
    mismatch = 0
    for i in range(0, len(insts), 16):
        for k in ("zr", "ze", "px", "pu"):
            mismatch += int(hs[i].download(k).tobytes() != b.download(i, k).tobytes())
    for h in hs:
        h.close()
    b.close()
    return {"metric": f"zone-cycles/s, {len(insts)}-instance Sedov batch to t=0.5", "unit": "zone-cycles/s",
            "value": zc / t_batch, "dtype": "f64",
            "config": {"instances": len(insts), "zones": sum(m.numz for m in meshes), "zone_cycles": zc,
                       "cycles_min": min(s["cycle"] for s in sc), "cycles_max": max(s["cycle"] for s in sc),
                       "tile_zones": zpt, "ctas_per_sm": cps, "tuned_ms_per_cycle": ms_tune,
                       "left_running": left},
            "batch_wall_s": t_batch, "sequential_wall_s": t_seq, "sequential_value": zc / t_seq,
            "speedup_vs_sequential": t_seq / t_batch, "sampled_instances_bitwise_mismatches": mismatch,
            "status_nonzero": sum(1 for s in sc if s["status"])}


def run_batch(args, pb, np, torch):
    """--workload batch: the config-3 batch record alone (batch_record)."""
    out = batch_record(pb, torch)
    out["data"] = "synthetic"
    print(json.dumps(out), flush=True)
    return 0


def run_pieces(args, pb, np, torch, dist, rank, world, local_rank):
    """--decomp pieces: the deck's mesh split into `world` pieces, one per
    rank (pnt_mesh_piece; the reference's numpcs decomposition), stepped
    over NCCL with the halo sums of corner mass and force and the dt
    reductions every cycle.  Every rank replays CUDA graphs of whole cycles
    (kernels, NCCL sends/receives and all-reduces); `value` = zones of the
    whole mesh x K / (max over ranks of the CUDA-event time of K cycles):
    strong scaling.  The start state is the FP64 pieces' run to
    --start-cycles, copied into the timed path's pieces."""
    from datetime import timedelta
    from pennant_b200.pieces import PieceHydro
    if world == 1:   # a single piece run without a launcher
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29517")
        os.environ.setdefault("RANK", "0")
        os.environ.setdefault("WORLD_SIZE", "1")
    dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local_rank))
    deck = pb.Deck(path=args.deck)
    mesh = pb.Mesh(deck=deck)
    numz, nums, nump = mesh.numz, mesh.nums, mesh.nump
    closure = pb.Closure(path=args.closure, device=local_rank) if args.precision == "learned" else None

    def params(precision):
        d = pb.Deck(path=args.deck)
        d.set("precision", precision)
        return d.params()

    chunk = 10
    t0 = time.perf_counter()
    base = PieceHydro(mesh, params("fp64"), device=local_rank)
    base.capture(chunk)
    for _ in range(args.start_cycles // chunk):
        base.replay()
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    start = base.scalars()
    head = PieceHydro(mesh, params(args.precision), device=local_rank, closure=closure)
    head.hydro.copy_state_from(base.hydro)
    base.close()
    # host cost of one eagerly stepped cycle (library calls and NCCL
    # launches from Python), then the graph of `chunk` cycles
    torch.cuda.synchronize()
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.warmup):
        head.cycle()
    torch.cuda.synchronize()
    eager_ms = (time.perf_counter() - t0) * 1e3 / args.warmup
    head.capture(chunk)
    for _ in range(max(1, args.warmup // chunk)):
        head.replay()
    nrep = max(1, args.steps // chunk)
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(head.stream)
    for _ in range(nrep):
        head.replay()
    ev1.record(head.stream)
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    steps = nrep * chunk
    s = head.scalars()
    head.close()
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        line = {"metric": METRIC, "value": numz * steps / (ms / 1e3), "unit": UNIT, "n_gpus": world,
                "steps": steps, "warmup": args.warmup, "ms_per_step": ms / steps, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None,
                "dtype": {"learned": "bf16+f32+f64", "mixed": "f32+f64", "fp64": "f64"}[args.precision],
                "data": "synthetic",
                "config": dict(workload_config(args.deck, numz, nums, nump, world),
                               parallelism=f"pieces x{world}"),
                "details": {"decomp": "pnt_mesh_piece zone strips, halo corner sums over NCCL, graph-replayed "
                                      f"cycles ({chunk} a graph)", "path": args.precision,
                            "start_state": {"cycle": start["cycle"], "time": start["time"], "setup_s": setup_s},
                            "end_cycle": s["cycle"], "eager_ms_per_cycle": eager_ms},
                "gpu_launches": None}
        print(json.dumps(line), flush=True)
    return 0


def run_probe(args, pb, sedov, torch):
    """A developed state (the FP64 cycle to --start-cycles on Sedov N^2) and one
    single-launch cycle of each path from it inside the NVTX range 'prof',
    after one unmarked cycle: the small case the pass A profiles capture."""
    text = sedov(args.probe)
    closure = pb.Closure(path=args.closure)

    def make(p, **keys):
        d = pb.Deck(text=text)
        d.set("precision", p)
        for k, v in keys.items():
            d.set(k, v)
        h = pb.Hydro(pb.Mesh(deck=d), d.params())
        if p == "learned":
            h.set_closure(closure)
        return h

    base = make("fp64", cstop=args.start_cycles)
    base.run()
    out = {"probe": args.probe, "start_cycle": base.scalars()["cycle"], "time": base.scalars()["time"]}
    for p in ("mixed", "learned", "fp64"):
        h = make(p)
        h.copy_state_from(base)
        h.cycle()
        torch.cuda.nvtx.range_push("prof")
        h.cycle()
        torch.cuda.nvtx.range_pop()
        out[p] = h.scalars()["cycle"]
        h.close()
    print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--deck", default=DEFAULT_DECK)
    ap.add_argument("--precision", default="learned", choices=["learned", "mixed", "fp64"],
                    help="path of the headline value; the plain FP64 cycle is always timed beside it")
    ap.add_argument("--closure", default=DEFAULT_CLOSURE)
    ap.add_argument("--start-cycles", type=int, default=30000)
    ap.add_argument("--no-full-run", action="store_true",
                    help="skip the whole runs of the deck to t = 1 with each path (the accuracy record)")
    ap.add_argument("--no-full-480", action="store_true",
                    help="skip the 480^2 whole runs (short profiling runs)")
    ap.add_argument("--workload", default="sedov1920", choices=["sedov1920", "leblanc", "batch"],
                    help="sedov1920: the headline line; leblanc: the 2880x288 Leblanc-type tube to t = 6 "
                         "with each path (accuracy of the mixed cycle); batch: the seeded 256-instance "
                         "Sedov batch to t = 0.5, batched against one instance at a time")
    ap.add_argument("--probe", type=int, default=0, metavar="N",
                    help="profiling probe instead of the benchmark: Sedov N^2, the FP64 cycle to "
                         "--start-cycles, then one single-launch cycle of each path inside NVTX range 'prof'")
    ap.add_argument("--decomp", default="replicas", choices=["replicas", "pieces"],
                    help="N > 1: independent replicas (weak scaling) or the mesh split into N pieces that "
                         "exchange halo corner sums over NCCL every cycle (strong scaling)")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the seeded 256-instance batch record of the default line")
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
    from make_decks import sedov

    torch.cuda.set_device(local_rank)
    if args.probe:
        return run_probe(args, pb, sedov, torch)
    if args.workload == "leblanc":
        return run_leblanc(args, pb, np, torch)
    if args.workload == "batch":
        return run_batch(args, pb, np, torch)
    if args.decomp == "pieces":
        return run_pieces(args, pb, np, torch, dist, rank, world, local_rank)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local_rank))

    mesh = pb.Mesh(deck=pb.Deck(path=args.deck))
    nump, numz, nums = mesh.nump, mesh.numz, mesh.nums
    ab = algorithmic_bytes(nump, nums, numz)
    closure = pb.Closure(path=args.closure, device=local_rank) if args.precision == "learned" else None

    def make(precision, text=None, **keys):
        d = pb.Deck(text=text) if text is not None else pb.Deck(path=args.deck)
        d.set("precision", precision)
        for k, v in keys.items():
            d.set(k, v)
        h = pb.Hydro(mesh if text is None else pb.Mesh(deck=d), d.params(), device=local_rank)
        if precision == "learned":
            h.set_closure(closure)
        return h

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

    def l1(a, b):
        return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))

    def errors(h, ref):
        return {"zr": l1(h.download("zr"), ref.download("zr")), "ze": l1(h.download("ze"), ref.download("ze")),
                "u": l1(np.hypot(*h.download("pu").T), np.hypot(*ref.download("pu").T)),
                "cycles": h.scalars()["cycle"], "cycles_fp64": ref.scalars()["cycle"], "time": h.scalars()["time"]}

    def fractions(c):
        tot = sum(v for k, v in c.items() if k not in ("error", "zones"))
        return {k: v / max(tot, 1) for k, v in c.items() if k not in ("error", "zones")}

    gpu_index = os.environ.get("CUDA_VISIBLE_DEVICES", str(local_rank)).split(",")[local_rank if world > 1 else 0]

    def timed(h, learned, sample_clocks, name):
        h.time_cycles(args.warmup)      # graph capture + W cycles
        if learned:
            h.closure_counts(reset=True)
        barrier_sync()
        clocks = None
        # NVTX range "timed_<path>": lets a profiler select the timed kernels
        if sample_clocks:
            with ClockSampler(gpu_index) as clk:
                barrier_sync()
                torch.cuda.nvtx.range_push(f"timed_{name}")
                ms = h.time_cycles(args.steps)
                torch.cuda.nvtx.range_pop()
                barrier_sync()
            clocks = clk.summary()
        else:
            barrier_sync()
            torch.cuda.nvtx.range_push(f"timed_{name}")
            ms = h.time_cycles(args.steps)
            torch.cuda.nvtx.range_pop()
            barrier_sync()
        s = h.scalars()
        if s["status"] or s["done"]:
            raise SystemExit(f"run stopped early: {s}")
        return max_over_ranks(ms), clocks

    # the common start state: the FP64 cycle to cycle --start-cycles (this
    # object is the FP64 whole run: it continues to t = 1 after the windows)
    t0 = time.perf_counter()
    base = make("fp64")
    s0 = base.run(max_cycles=args.start_cycles)
    t_base = time.perf_counter() - t0
    start = {"cycle": s0["cycle"], "time": s0["time"], "setup_s": t_base,
             "note": "plain FP64 run from the deck's initial state, copied into every timed path"}

    order = [args.precision] + [p for p in ("fp64", "mixed") if p != args.precision]
    heads, res = {}, {}
    for p in order:
        h = make(p)
        h.copy_state_from(base)
        heads[p] = h
        ms, clocks = timed(h, p == "learned", p == args.precision, p)
        cnt = h.closure_counts(reset=True) if p == "learned" else None
        kms = h.time_kernels(10)
        res[p] = {"ms": ms, "clocks": clocks, "kernel_ms": kms, "counts": cnt,
                  "value": world * numz * args.steps / (ms / 1e3)}
    head = heads[args.precision]
    window_err = {p: errors(heads[p], heads["fp64"]) for p in order if p != "fp64"}
    for p in order:
        if p != args.precision:
            heads[p].close()

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

    def whole_run(p, text=None):
        h = make(p, text=text)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        h.run()
        return h, time.perf_counter() - t1

    def compare(p, h, ref, wall):
        out = {"wall_s": wall, "cycles": h.scalars()["cycle"], "time": h.scalars()["time"],
               "l1_rel_err_vs_fp64": errors(h, ref)}
        if p == "learned":
            c = h.closure_counts()
            out["corner_fractions"] = fractions(c)
            out["fallback_fraction"] = (c["fallback"] + c["ood"]) / max(c["mlp"] + c["fallback"] + c["ood"], 1)
            out["wait_timeouts"] = c["error"]
        return out

    # whole runs to t = 1 against the FP64 cycle: 480^2, and the metric's
    # 1920^2 (the FP64 one continues the start-state run)
    def full_run_480():
        text = sedov(480, tstop=1.0)
        ref, wall = whole_run("fp64", text)
        out = {"fp64": {"wall_s": wall, "cycles": ref.scalars()["cycle"]}}
        for p in order:
            if p != "fp64":
                h, wall = whole_run(p, text)
                out[p] = compare(p, h, ref, wall)
                h.close()
        ref.close()
        return out

    full = {} if args.no_full_480 else {"480": full_run_480()}
    accuracy = None
    if not args.no_full_run:
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        base.run()
        wall = t_base + time.perf_counter() - t1
        f1920 = {"fp64": {"wall_s": wall, "cycles": base.scalars()["cycle"], "time": base.scalars()["time"],
                          "value": numz * base.scalars()["cycle"] / wall}}
        for p in order:
            if p != "fp64":
                h, wall = whole_run(p)
                f1920[p] = compare(p, h, base, wall)
                f1920[p]["value"] = numz * f1920[p]["cycles"] / wall
                h.close()
        full["1920"] = f1920
        hp = f1920[args.precision] if args.precision != "fp64" else None
        if hp:
            err = hp["l1_rel_err_vs_fp64"]
            accuracy = {"mesh": f"{os.path.basename(args.deck)} to t = {hp['time']:.6g} from its initial state",
                        "l1_rel_err_vs_fp64": {"rho": err["zr"], "e": err["ze"], "u": err["u"]},
                        "bound": 1e-3, "within_bound": max(err["zr"], err["ze"], err["u"]) <= 1e-3,
                        "cycles": hp["cycles"], "cycles_fp64": f1920["fp64"]["cycles"],
                        "whole_run_speedup_vs_fp64": f1920["fp64"]["wall_s"] / hp["wall_s"]}
            if "fallback_fraction" in hp:
                accuracy["fallback_fraction"] = hp["fallback_fraction"]
                accuracy["wait_timeouts"] = hp["wait_timeouts"]
    base.close()
    batch = None if (args.no_batch or rank != 0) else batch_record(pb, torch)

    hbm, peak_kind = measured_peaks()
    names = ["A", "B", "C", "end_of_cycle", "closure"]   # the order of pnt_hydro_time_kernels

    def kernel_ms(path, kms):
        """The launches the path makes: passes A, B, C (C's last CTA ends the
        cycle; time_kernels' separate end-of-cycle slot holds only the event
        gap) and, in the learned cycle, the closure pass."""
        d = {"A": kms[0], "B": kms[1], "C": kms[2]}
        if path == "learned":
            d["closure"] = kms[4]
        return d

    def fp64_pipe_roofline(ms, nz):
        """The FP64 pass A against the FP64 pipe: its FP64 instructions (ncu
        count a zone x zones) per second over 64 a clock per SM."""
        nsm = torch.cuda.get_device_properties(local_rank).multi_processor_count
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
                mhz = float(json.load(f)["sm_max_mhz"])
        except Exception:
            mhz = 1965.0
        peak = FP64_INST_PER_CLOCK_PER_SM * nsm * mhz * 1e6 / 1e12
        ach = FP64_PASS_A_INST_PER_ZONE * nz / (ms / 1e3) / 1e12
        return {"bound": "fp64 pipe", "kernel": "pass A (fp64)", "achieved": ach, "peak": peak,
                "unit": "T FP64 thread-instructions/s", "frac": ach / peak, "launch_ms": ms,
                "note": "FP64 instructions a zone from profiles/pass_a_fp64_sedov1024.md (1024^2 at cycle "
                        "16000); the count depends on how much of the mesh is quiescent"}

    kms_head = res[args.precision]["kernel_ms"]
    dom = int(np.argmax(kms_head[:3]))
    if args.precision in ("mixed", "learned"):
        per_launch = {"A": 32 * nump + 44 * numz + 32 * nums, "B": 68 * nump + 16 * nums,
                      "C": 64 * nump + 12 * nums + 60 * numz}
    else:
        per_launch = {k: ab[k] for k in ("A", "B", "C")}
    ach_dom = per_launch[names[dom]] / (kms_head[dom] / 1e3) / 1e9
    ms_head = res[args.precision]["ms"]
    ach_cycle = ab["cycle"] * args.steps / (ms_head / 1e3) / 1e9

    closure_info = None
    if args.precision == "learned":
        cnt = res["learned"]["counts"]
        zones_per_cycle = cnt["zones"] / args.steps
        cl_ms = kms_head[4]
        closure_info = {
            "corner_fractions": fractions(cnt),
            # plain-QCS share of the compressing corners the network could take
            # (zones with an acute corner keep the FP64 QCS whatever the compression)
            "fallback_fraction": (cnt["fallback"] + cnt["ood"]) / max(cnt["mlp"] + cnt["fallback"] + cnt["ood"], 1),
            # the closure pass runs the network on the network's corners only
            "zones_per_cycle": zones_per_cycle, "network_rows_per_cycle": cnt["mlp"] / args.steps,
            "closure_pass_ms": cl_ms,
            "tensor_tflops": (cnt["mlp"] / args.steps * MLP_FLOP_PER_ROW) / (cl_ms / 1e3) / 1e12 if cl_ms > 0 else None,
            "wait_timeouts": cnt["error"], "weights": os.path.relpath(args.closure, ROOT)}

    result = None
    if rank == 0:
        paths = {
            "learned": "learned closure + mixed precision: the 14-64-64-4 BF16 network (tcgen05) in place of QCS "
                       "on compressing corners within its range, plain QCS elsewhere; FP32 side geometry, "
                       "TTS/QCS forces, sound speed and zone dt, FP64 point kinematics, volumes, pressure, "
                       "work and the dt reduction",
            "mixed": "mixed precision: FP32 edge/corner geometry, TTS/QCS side forces, sound speed and zone dt, "
                     "FP64 point kinematics, volumes, pressure, work and the dt reduction; plain QCS",
            "fp64": "plain FP64 (bitwise parity path)"}
        # passes A, B, C (which ends the cycle), and the closure pass
        launches = 4 if args.precision == "learned" else 3
        others = {p: {"value": res[p]["value"], "ms_per_step": res[p]["ms"] / args.steps,
                      "kernel_ms": kernel_ms(p, res[p]["kernel_ms"])} for p in order if p != args.precision}
        result = {
            "metric": METRIC, "value": res[args.precision]["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_head / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"learned": "bf16+f32+f64", "mixed": "f32+f64", "fp64": "f64"}[args.precision],
            "data": "synthetic",
            "config": workload_config(args.deck, numz, nums, nump, world),
            "accuracy": accuracy,
            "batch": batch,
            "details": {"path": paths[args.precision], "start_state": start, "others": others,
                        "speedup_vs_fp64": res[args.precision]["value"] / res["fp64"]["value"],
                        "l1_rel_err_vs_fp64_window": window_err,
                        "full_runs_to_t1": full,
                        "closure": closure_info},
            "roofline": {"bound": "hbm", "kernel": f"pass {names[dom]} ({args.precision})", "achieved": ach_dom,
                         "peak": hbm, "unit": "GB/s", "frac": ach_dom / hbm, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": per_launch[names[dom]], "launch_ms": kms_head[dom],
                         "traffic": PASS_A_TRAFFIC_PER_ZONE[args.precision] * numz if names[dom] == "A" else None,
                         "traffic_note": "ncu DRAM read+write of one pass A launch at 1024^2 (cycle 16000), "
                                         "scaled by the zone count (writes still in L2 at the kernel's end "
                                         "are not counted)"},
            "roofline_fp64_pass_a": fp64_pipe_roofline(res["fp64"]["kernel_ms"][0], numz),
            "roofline_cycle": {"achieved": ach_cycle, "peak": hbm, "unit": "GB/s", "frac": ach_cycle / hbm,
                               "algorithmic_bytes_per_cycle": ab["cycle"],
                               "note": "FP64 schedule bytes B = 164 Np + 100 Ns + 104 Nz for every path"},
            "kernel_ms": kernel_ms(args.precision, kms_head),
            "e2e": {"value": world * numz * args.steps / e2e_s, "unit": UNIT,
                    "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                    "note": "state uploaded from pinned host memory once per timed run, one pnt_hydro_cycle "
                            "call per step (returns the step's dt/time), final fields downloaded; "
                            "bytes per step are run totals / steps"},
            "gpu_launches": launches * args.steps,
            "clocks": res[args.precision]["clocks"],
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
