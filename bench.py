"""Benchmark of the strip list-mode TOF MLEM path on B200.

Workload (the at-scale configuration): two 800 mm strips at y = +-400 mm,
800 x 400 image of 1 mm pixels, sigma_z 5 mm, sigma_dl 25 mm, 2e8 seeded
synthetic events from a 10-ellipse Shepp-like phantom (activities 0.1-2.0).
A step is one full-set MLEM iteration over all events; the metric is
Mevent*iter/s (events x iterations / device time).  Events stay resident in
HBM (2.4 GB > L2), so no L2 flush is needed between iterations.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 (torchrun, one rank per GPU): each rank holds its own 2e8 events
(seed + rank); after every iteration's backprojection the ranks all-reduce
the binary64 accumulator over NCCL and apply the same update (weak scaling).
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "j-pet-mlem-old_b200"))

METRIC = "Strip TOF-MLEM Mevent·iter/s on 1 B200 at ≤1e-4 rel-L2 vs FP64 oracle"
UNIT = "Mevent*iter/s"
GEOM = dict(radius=400.0, length=800.0, n_y=400, n_z=800, p=1.0, s_z=5.0, s_dl=25.0)
PHANTOM = [
    (-150, 60, 40, 25, 20, 2.0),
    (150, -60, 50, 30, -30, 0.1),
    (0, 100, 60, 20, 0, 1.5),
    (0, -110, 70, 25, 10, 0.5),
    (-250, -40, 30, 30, 0, 1.8),
    (250, 50, 35, 20, 45, 0.3),
    (80, 40, 20, 15, 0, 2.0),
    (-80, -60, 25, 15, -15, 0.8),
    (0, 0, 300, 150, 0, 1.0),
    (0, 0, 360, 175, 0, 0.2),
]
SEED = 20260101
# DRAM bytes (read + write) per event of one k_tile pass, from an ncu capture
# of one launch over this workload's first 2e7 events (dram__bytes_read.sum
# 244.7 MB + dram__bytes_write.sum 5.1 MB); the traffic grows with the event
# count.
TILE_DRAM_BYTES_PER_EVENT = (244.702464e6 + 5.090304e6) / 2e7


def workload_config(n_events, e2e_iters, world=1):
    return {
        "workload": "strip MLEM, 800x400 image of 1 mm pixels, R=400 mm, L=800 mm, "
                    "sigma_z=5 mm, sigma_dl=25 mm, 10-ellipse Shepp-like phantom",
        "n_events": n_events,
        "image": [GEOM["n_y"], GEOM["n_z"]],
        "pixel_mm": GEOM["p"],
        "mode": "cpu-compat (GaussianKernel, no sensitivity)",
        "accumulation": "kahan per lane + binary64 across lanes and images",
        "step": "one full-set MLEM iteration over all events",
        "e2e_step": f"set_events from pinned host + {e2e_iters} iterations + image D2H",
        "l2": "inputs (12 B/event, 2.4 GB) larger than the 126 MB L2; no flush",
        "parallelism": ("single GPU" if world == 1 else
                        f"{world} ranks: events sharded per rank (each its own 2e8), "
                        "image replicated, NCCL all-reduce of the binary64 "
                        "backprojection every iteration"),
        "seed": SEED,
    }


def scanner():
    import stripmlem as sm
    return sm.Scanner(GEOM["radius"], GEOM["length"], GEOM["n_y"], GEOM["n_z"],
                      GEOM["p"], GEOM["p"], GEOM["s_z"], GEOM["s_dl"])


def measured_peak(key):
    """A peak of MEASURED_PEAKS.json (written per machine), or None."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)[key])
    except Exception:
        return None


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# ---------------------------------------------------------------------------
# reference arm / cpu baseline: the reference's own CPU binary
# ---------------------------------------------------------------------------
def run_reference_cpu(n_sample, iters, warmup, cores, events=None):
    """Times the reference 2d_strip_reconstruction (oracle/_ref, built from the
    reference sources with its default flags) on the first n_sample events of
    the workload.  Returns (Mevent*iter/s, kind, detail).  Without `events`
    the sample comes from the oracle's statement of the workload generator
    (oracle/strip_events.c, the same events bit for bit), so this arm loads
    nothing of the product library."""
    from oracle import oracle as orc
    g = orc.geometry(GEOM["radius"], GEOM["length"], GEOM["n_y"], GEOM["n_z"],
                     GEOM["p"], GEOM["p"], GEOM["s_z"], GEOM["s_dl"])
    if events is None:
        zu, zd, dl = orc.generate_events(g, PHANTOM, n_sample, SEED)
    else:
        zu, zd, dl = (a[:n_sample] for a in events)
    if orc.ref_available(nocontract=False):
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "events.bin")
            orc.write_events_bin(path, zu, zd, dl)
            _, out = orc.ref_benchmark(g, path, iters + warmup, cores)
        times = [float(m.group(2)) for m in
                 re.finditer(r"^\s*(\d+)\s+([0-9.]+)\s*$", out, flags=re.M)]
        times = times[warmup:] if len(times) > warmup else times
        t = sum(times) / 1000.0
        return n_sample * len(times) / t / 1e6, "reference", \
            f"first {n_sample} events of the workload, {len(times)} timed iterations " \
            f"(+{warmup} warm-up) of oracle/_ref/2d_strip_reconstruction -T {cores} -vv"
    # oracle port (single thread) when the reference binary was not built
    t0 = time.perf_counter()
    n = min(n_sample, 20000)
    orc.mlem_f32(g, zu[:n], zd[:n], dl[:n], iters)
    t = time.perf_counter() - t0
    return n * iters / t / 1e6, "port", \
        f"first {n} events, {iters} iterations of the oracle's binary32 restatement, 1 thread"


def reference_arm(args, rank, world):
    if rank != 0:
        return 0
    cores = host_cores()
    n_sample = args.ref_events or min(args.events, 60000 * cores)
    value, kind, sample = run_reference_cpu(n_sample, args.steps, args.warmup, cores)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": n_sample / (value * 1e6) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args.events, args.e2e_iters, world),
        "cpu_baseline": {"value": value, "unit": UNIT,
                         "cores": cores if kind == "reference" else 1,
                         "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def pinned_empty(n):
    import torch
    t = torch.empty(n, dtype=torch.float32, pin_memory=True)
    return t, t.numpy()


def differentiable_throughput(rec, n, reps=2):
    """Device time of the forward projection (strip_forward_device) and the
    adjoint (strip_adjoint_device) over the resident events; returns ms of
    each (mean over reps), at the geometry's sigmas."""
    import torch
    dev = rec.torch_device
    n_pix = GEOM["n_y"] * GEOM["n_z"]
    rho = torch.ones(n_pix, dtype=torch.float32, device=dev)
    y = torch.empty(n, dtype=torch.float64, device=dev)
    w = torch.empty(n, dtype=torch.float64, device=dev)
    g = torch.empty(n_pix, dtype=torch.float64, device=dev)
    sz, sdl = GEOM["s_z"], GEOM["s_dl"]
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    tf = ta = 0.0
    for r in range(reps + 1):
        torch.cuda.synchronize()
        ev[0].record()
        rec._check(rec.lib.strip_forward_device(rec._ctx, rho.data_ptr(), sz, sdl, 0,
                                                y.data_ptr()))
        ev[1].record()
        torch.reciprocal(y, out=w)
        torch.cuda.synchronize()
        ev[1].synchronize()
        t_fwd = ev[0].elapsed_time(ev[1])
        ev[0].record()
        rec._check(rec.lib.strip_adjoint_device(rec._ctx, w.data_ptr(), sz, sdl, 0,
                                                g.data_ptr()))
        ev[2].record()
        ev[2].synchronize()
        if r > 0:  # the first pass is a warm-up
            tf += t_fwd
            ta += ev[0].elapsed_time(ev[2])
    return tf / reps, ta / reps


def accuracy_vs_fp64(events, n_sample, iters, local_rank, n_subsets=1):
    """Error of the benchmark's kernel configuration against the FP64 oracle
    (the checker): the first n_sample events of the workload reconstructed on
    the GPU -- MLEM with 8000-event work items, the full run's item size, or
    n_subsets-subset OSEM -- for `iters` iterations, and the same in binary64
    on the host (oracle/strip_oracle.c, all host threads)."""
    import stripmlem as sm
    from oracle import oracle as orc
    zu, zd, dl = (a[:n_sample] for a in events)
    g = orc.geometry(GEOM["radius"], GEOM["length"], GEOM["n_y"], GEOM["n_z"],
                     GEOM["p"], GEOM["p"], GEOM["s_z"], GEOM["s_dl"])
    with sm.Reconstruction(scanner(), device=local_rank, mode=sm.MODE_CPU,
                           accumulation=sm.ACCUM_KAHAN) as r:
        if n_subsets == 1:
            r.set_item_events(8000)
        r.set_events(zu, zd, dl, n_subsets=n_subsets)
        max_item = r.stats()["max_item_events"]
        r(None, iters, n_subsets=n_subsets)
        img = r.rho.astype(np.float64)
    ref = orc.mlem_f64(g, zu, zd, dl, iters, n_subsets=n_subsets, sets_f32=True)

    def rel(b):
        return float(np.linalg.norm(img - b) / np.linalg.norm(b))

    out = {"rel_l2_vs_fp64": rel(ref),
           "max_pixel_err_rel_peak": float(np.abs(img - ref).max() / np.abs(ref).max()),
           "sample": f"first {n_sample} events of the workload, {iters} "
                     + ("MLEM iterations, 8000-event work items (largest item "
                        f"{max_item}), the benchmark's kernel configuration"
                        if n_subsets == 1 else f"{n_subsets}-subset OSEM iterations")
                     + "; FP64 oracle with the reference's binary32 pixel sets"}
    if n_subsets == 1:
        out["rel_l2_vs_full_fp64"] = rel(orc.mlem_f64(g, zu, zd, dl, iters, sets_f32=False))
    return out


def osem_throughput(rec, n, n_subsets, warmup, steps):
    """Device time of `steps` OSEM iterations (each a sweep over all events
    in n_subsets subset updates) on the resident events; Mevent*iter/s."""
    rec(None, warmup, n_subsets=n_subsets)  # the first call re-bins
    rec(None, steps, n_subsets=n_subsets)
    st = rec.stats()
    ms = st["last_iterate_ms"]
    return {"subsets": n_subsets, "steps": steps, "ms_per_iteration": ms / steps,
            "Mevent_iter_per_s": n * steps / (ms / 1e3) / 1e6,
            "launches_per_iteration": st["kernel_launches"] / steps,
            "what": f"{n_subsets}-subset OSEM (subset = event index mod {n_subsets}); "
                    "an iteration visits every subset once"}


def write_event_file(path, zu, zd, dl, chunk=10_000_000):
    """The events as the reference's binary event file (raw f32 triples)."""
    with open(path, "wb") as f:
        for a in range(0, zu.shape[0], chunk):
            b = min(zu.shape[0], a + chunk)
            np.stack([zu[a:b], zd[a:b], dl[a:b]], axis=1).astype("<f4").tofile(f)


def io_throughput(zu, zd, dl, local_rank, iters):
    """Event input from a file (page cache warm, the file just written):
    strip_load_responses_file (file -> pinned staging -> HBM -> binning),
    the pageable path (np.fromfile, then the AoS setter), and the drop-in CLI
    end to end (process start, file -> HBM, `iters` iterations, image file)
    timed by the wall clock."""
    import stripmlem as sm
    n = zu.shape[0]
    d = tempfile.mkdtemp(prefix="strip_io_")
    path = os.path.join(d, "events.bin")
    out = {"events": n, "file_bytes": 12 * n, "page_cache": "warm (file just written)"}
    try:
        write_event_file(path, zu, zd, dl)
        with sm.Reconstruction(scanner(), device=local_rank) as rec:
            times = []
            for _ in range(2):
                t0 = time.perf_counter()
                rec.load_responses_file(path)
                times.append(time.perf_counter() - t0)
            out["file_to_hbm_binned_s"] = min(times)
            out["file_to_hbm_binned_GBps"] = 12 * n / min(times) / 1e9
            out["binning_ms"] = rec.stats()["last_setup_ms"]
            t0 = time.perf_counter()
            t = np.fromfile(path, dtype="<f4").reshape(-1, 3)
            t1 = time.perf_counter()
            rec.responses = t
            t2 = time.perf_counter()
            del t
            out["pageable_read_s"] = t1 - t0
            out["pageable_set_responses_s"] = t2 - t1
            out["pageable_total_GBps"] = 12 * n / (t2 - t0) / 1e9
        cli = os.path.join(ROOT, "j-pet-mlem-old_b200", "bin", "2d_strip_reconstruction")
        if os.access(cli, os.X_OK):
            img = os.path.join(d, "r.bin")
            cmd = [cli, path, "-r", repr(GEOM["radius"]), "-l", repr(GEOM["length"]),
                   "-p", repr(GEOM["p"]), "--n-y-pixels", str(GEOM["n_y"]),
                   "--n-z-pixels", str(GEOM["n_z"]), "--s-z", repr(GEOM["s_z"]),
                   "--s-dl", repr(GEOM["s_dl"]), "-i", "1", "-I", str(iters), "-o", img,
                   "--cuda-device", str(local_rank)]
            t0 = time.perf_counter()
            p = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
            wall = time.perf_counter() - t0
            if p.returncode == 0:
                out["cli_e2e"] = {
                    "value": n * iters / wall / 1e6, "unit": UNIT, "wall_s": wall,
                    "iterations": iters,
                    "what": "bin/2d_strip_reconstruction <file> -i 1 -I %d -o r.bin: process "
                            "start, CUDA context, file -> HBM, binning, iterations, image "
                            "file, wall clock" % iters}
            else:
                out["cli_e2e"] = {"error": p.stderr[-300:]}
    finally:
        for f in os.listdir(d):
            os.unlink(os.path.join(d, f))
        os.rmdir(d)
    return out


def batch_instances(n_inst=64):
    """The batched workload: n_inst reconstructions, instance i seeded by i --
    image n_y x n_z with n in [100, 800], pixel p in {1, 2, 3, 4} mm, strips
    L = n_z p long at R = n_y p / 2, sigma_z 10 mm, sigma_dl 42 mm, 3-10
    ellipses (the last a body covering most of the field), events
    log-uniform in [1e5, 2e7]."""
    out = []
    for i in range(n_inst):
        rng = np.random.default_rng(i)
        n_y, n_z = (int(v) for v in rng.integers(100, 801, size=2))
        p = float(rng.integers(1, 5))
        R, L = n_y * p / 2.0, n_z * p
        k = int(rng.integers(3, 11))
        ph = []
        for _ in range(k - 1):
            ph.append((float(rng.uniform(-0.3, 0.3) * L), float(rng.uniform(-0.3, 0.3) * R),
                       float(rng.uniform(0.04, 0.15) * L), float(rng.uniform(0.04, 0.15) * R),
                       float(rng.uniform(0, 180)), float(rng.uniform(0.1, 2.0))))
        ph.append((0.0, 0.0, 0.42 * L, 0.42 * R, 0.0, 1.0))
        n_ev = int(np.exp(rng.uniform(np.log(1e5), np.log(2e7))))
        out.append(dict(R=R, L=L, n_y=n_y, n_z=n_z, p=p, phantom=ph, events=n_ev, seed=i))
    return out


def batched_throughput(local_rank, n_inst, warmup, steps, autotune=True):
    """The same instances advanced one context at a time (strip_iterate) and
    as one batch (strip_batch_*): Mevent*iter/s of each over all events.
    With autotune, every instance first gets its own tile / grab schedule
    from strip_autotune (timed on its own events); both legs use it."""
    import torch
    import stripmlem as sm
    recs = []
    total = 0
    schedules = {}
    tune_s = 0.0
    try:
        for inst in batch_instances(n_inst):
            sc = sm.Scanner(inst["R"], inst["L"], inst["n_y"], inst["n_z"], inst["p"],
                            inst["p"], 10.0, 42.0)
            ev = sm.generate_events_device(sc, inst["phantom"], inst["events"],
                                           seed=inst["seed"], device=local_rank)
            rec = sm.Reconstruction(sc, device=local_rank, mode=sm.MODE_CPU)
            rec.set_events_device(*ev)
            del ev
            if autotune:
                t0 = time.perf_counter()
                best = rec.autotune()
                tune_s += time.perf_counter() - t0
                key = f"tile{best['tile']}_grab{best['grab']}"
                schedules[key] = schedules.get(key, 0) + 1
            recs.append(rec)
            total += inst["events"]
        torch.cuda.empty_cache()
        import ctypes
        flops = 0.0
        overflow = 0
        for rec in recs:
            bb, inn, ne = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
            rec._check(rec.lib.strip_count_work(rec._ctx, ctypes.byref(bb), ctypes.byref(inn),
                                                ctypes.byref(ne)))
            flops += 10.0 * bb.value + 18.0 * inn.value
            overflow += rec.stats()["n_overflow"]
        seq_ms = 0.0
        for rec in recs:
            rec(None, warmup)
            rec(None, steps)
            seq_ms += rec.stats()["last_iterate_ms"]
        with sm.Batch(recs) as batch:
            batch(warmup)
            batch(steps)
            st = batch.stats()
        bat_ms = st["last_iterate_ms"]
        return {"instances": n_inst, "events": total, "steps": steps,
                "sequential_Mevent_per_s": total * steps / (seq_ms / 1e3) / 1e6,
                "batched_Mevent_per_s": total * steps / (bat_ms / 1e3) / 1e6,
                "ratio_batched_vs_sequential": seq_ms / bat_ms,
                "batched_ms_per_step": bat_ms / steps,
                "work_model_tflops_batched": flops * steps / (bat_ms / 1e3) / 1e12,
                "work_model_tflops_sequential": flops * steps / (seq_ms / 1e3) / 1e12,
                "events_on_global_path": overflow,
                "tile_work_items": st["n_work_items"],
                "launches_per_step": st["launches_per_iteration"],
                "autotuned": autotune,
                "schedules": schedules,
                "autotune_s": tune_s,
                "what": "64 seeded instances (image 100-800 px per side, 1-4 mm pixels, "
                        "1e5-2e7 events each): one MLEM step of every instance -- own tile "
                        "launches of the large instances on side streams beside a "
                        "persistent tile launch over the small ones, one update launch -- "
                        "replayed from a CUDA graph, against strip_iterate on each context "
                        "in turn"}
    finally:
        for r in recs:
            r.close()


def secondary_rates(n_in, tile_ms, clocks, n_sm=148):
    """The work model's special-function and atomic rates: one ex2 and one
    scatter-add per in-ellipse pixel and iteration.  The SFU peak is the
    nominal 16 MUFU results per SM and clock at the sampled SM clock."""
    per_s = n_in / (tile_ms / 1e3)
    mhz = clocks.get("sm_mhz") or 1965.0
    sfu_peak = n_sm * 16 * mhz * 1e6
    return {
        "model_ex2_per_s": per_s, "sfu_nominal_peak_per_s": sfu_peak,
        "sfu_frac": per_s / sfu_peak,
        "scatter_adds_per_s": per_s,
        "note": "per the work model (one ex2 and one scatter-add per in-ellipse pixel); "
                "the kernel evaluates the Gaussian along a run by a two-multiply "
                "recurrence (one ex2 pair per row) and scatters with one 32-bit "
                "shared-memory reduction per pixel, flushed to HBM once per work item",
    }


def ours(args, rank, world, local_rank):
    import torch
    import stripmlem as sm

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    torch.cuda.set_device(local_rank)
    sc = scanner()
    n = args.events

    # seeded workload (rank r: seed + r), generated on the GPU by the library's
    # device generator (the host generator's events) and kept in pinned host
    # memory for the end-to-end leg
    import ctypes
    tz, zu = pinned_empty(n)
    td, zd = pinned_empty(n)
    tl, dl = pinned_empty(n)
    gen = sm.generate_events_device(sc, PHANTOM, n, seed=SEED + rank, device=local_rank)
    for host, dev in zip((tz, td, tl), gen):
        host.copy_(dev)
    del gen
    torch.cuda.empty_cache()

    rec = sm.Reconstruction(sc, device=local_rank, mode=sm.MODE_CPU,
                            accumulation=sm.ACCUM_KAHAN)
    rec.set_events(zu, zd, dl)
    work_bb, work_in, nonempty = [ctypes.c_int64() for _ in range(3)]
    rec._check(rec.lib.strip_count_work(rec._ctx, ctypes.byref(work_bb),
                                        ctypes.byref(work_in), ctypes.byref(nonempty)))
    flops_per_iter = 10.0 * work_bb.value + 18.0 * work_in.value  # work model

    peak = ctypes.c_double()
    rec._check(rec.lib.strip_probe_fp32_peak(local_rank, ctypes.byref(peak)))

    # N = 1: strip_iterate runs the K iterations in one call.  N > 1: each
    # iteration is strip_accumulate on the rank's events, an NCCL all-reduce
    # of the binary64 accumulator, and strip_update on every rank.
    shd = None
    if world > 1:
        from stripmlem.distributed import ShardedReconstruction
        shd = ShardedReconstruction(rec, exchange="device")

    def iterate(k):
        if shd is None:
            rec(None, k)
        else:
            shd(k)

    iterate(args.warmup)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        t0.record()
        iterate(args.steps)
        t1.record()
        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    st = rec.stats()
    if shd is None:
        t_ms = st["last_iterate_ms"]   # library stream, CUDA events
        tile_ms = st["last_tile_ms"]
        launches = st["kernel_launches"]
    else:
        t_ms = t0.elapsed_time(t1)
        tile_ms = None
        launches = None
    if dist is not None:
        tt = torch.tensor([t_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_ms = float(tt.item())
    value = world * n * args.steps / (t_ms / 1e3) / 1e6
    clocks = clk.summary()

    # the tile kernel's own time: from the multi-rank run when N = 1, else
    # from one more local pass of the same events
    if tile_ms is None:
        rec(None, 1)
        st1 = rec.stats()
        tile_ms = st1["last_tile_ms"] * args.steps
        launches = st1["kernel_launches"] * args.steps  # tile (+ global) + update

    # end to end through the public API with host buffers
    e2e = None
    if args.e2e_steps > 0:
        img = np.empty((GEOM["n_y"], GEOM["n_z"]), np.float32)
        times = []
        # host wall time of each phase (every call returns once its work is
        # done), summed over the timed steps
        phases = {"set_events": 0.0, "set_image": 0.0, "iterations": 0.0, "get_image": 0.0}
        # within set_events: the host -> device copy (wall) and the binning
        # (device time), from the context's statistics
        sub = {"set_events_upload": 0.0, "set_events_binning": 0.0}
        # two untimed steps: the context's memory pool reaches its working
        # size on the second set_events (first 0.2-1.4 s, second about 0.1 s,
        # then 0.068 s at 2e8 events)
        e2e_warm = 2
        with ClockSampler(local_rank) as clk_e2e:
            for s in range(args.e2e_steps + e2e_warm):
                if dist is not None:
                    dist.barrier()
                torch.cuda.synchronize()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                w0 = time.perf_counter()
                rec.set_events(zu, zd, dl)
                w1 = time.perf_counter()
                rec.rho = np.ones_like(img)
                w2 = time.perf_counter()
                iterate(args.e2e_iters)
                w3 = time.perf_counter()
                img[...] = rec.rho
                w4 = time.perf_counter()
                b.record()
                torch.cuda.synchronize()
                if s >= e2e_warm:
                    times.append(a.elapsed_time(b) / 1e3)
                    for k, dt in zip(phases, (w1 - w0, w2 - w1, w3 - w2, w4 - w3)):
                        phases[k] += dt
                    st_e = rec.stats()
                    sub["set_events_upload"] += st_e["last_upload_ms"] / 1e3
                    sub["set_events_binning"] += st_e["last_setup_ms"] / 1e3
        e2e_t = sum(times) / len(times)
        if dist is not None:
            tt = torch.tensor([e2e_t], dtype=torch.float64, device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            e2e_t = float(tt.item())
        e2e = {"value": world * n * args.e2e_iters / e2e_t / 1e6,
               "unit": UNIT, "h2d_bytes_per_step": int(3 * 4 * n),
               "d2h_bytes_per_step": int(img.nbytes), "steps": len(times),
               "iterations_per_step": args.e2e_iters,
               "phases_s_per_step": {k: v / len(times)
                                     for k, v in list(phases.items()) + list(sub.items())},
               "clocks": clk_e2e.summary(),
               "timed": "set_events (pinned host -> HBM, binning) + iterations + image D2H, "
                        "CUDA events, max over ranks"}

    diff = None
    if world == 1 and not args.no_differentiable:
        tf, ta = differentiable_throughput(rec, n)
        mlem_ms = t_ms / args.steps
        diff = {"forward_ms": tf, "adjoint_ms": ta,
                "forward_plus_adjoint_Mevent_per_s": n / ((tf + ta) / 1e3) / 1e6,
                "mlem_Mevent_per_s": n / (mlem_ms / 1e3) / 1e6,
                "ratio_vs_mlem": mlem_ms / (tf + ta),
                "what": "strip_forward_device then strip_adjoint_device over the same "
                        "events (y_e = sum_j K_ej rho_j, g_j = sum_e K_ej / y_e)"}

    error = None
    osem = None
    if rank == 0 and world == 1 and args.error_events > 0:
        error = accuracy_vs_fp64((zu, zd, dl), min(n, args.error_events), args.e2e_iters,
                                 local_rank)
    if world == 1 and not args.no_osem:
        osem = osem_throughput(rec, n, 8, 1, 2)
        if rank == 0 and args.error_events > 0:
            osem["error"] = accuracy_vs_fp64((zu, zd, dl), min(n, args.error_events // 2), 2,
                                             local_rank, n_subsets=8)

    io = None
    if rank == 0 and world == 1 and not args.no_io:
        io = io_throughput(zu, zd, dl, local_rank, args.e2e_iters)

    batched = None
    achieved_plain = flops_per_iter / (tile_ms / args.steps / 1e3) / 1e12
    if world == 1 and not args.no_batched:
        batched = batched_throughput(local_rank, 64, max(1, args.warmup // 3), 3)
        batched["ratio_vs_plain_workload_by_work"] = (
            batched["work_model_tflops_batched"] / achieved_plain)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = host_cores()
        n_sample = min(n, args.ref_events or 60000 * cores)
        v, kind, sample = run_reference_cpu(n_sample, 1, 0, cores, events=(zu, zd, dl))
        cpu = {"value": v, "unit": UNIT, "cores": cores if kind == "reference" else 1,
               "kind": kind, "sample": sample}

    achieved = flops_per_iter / (tile_ms / args.steps / 1e3) / 1e12
    hbm_peak = measured_peak("hbm_gbs")
    hbm_achieved = (12 * n) / (tile_ms / args.steps / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": workload_config(n, args.e2e_iters, world),
        "roofline": {
            "bound": "fp32", "achieved": achieved, "peak": peak.value,
            "unit": "TFLOP/s", "frac": achieved / peak.value if peak.value else None,
            "traffic": TILE_DRAM_BYTES_PER_EVENT * n,
            "traffic_unit": "bytes per launch (ncu capture at 2e7 events, scaled)",
            "algorithmic_bytes": 12 * n + 4 * GEOM["n_y"] * GEOM["n_z"],
            "hbm": {"achieved_gbs": hbm_achieved, "peak_gbs": hbm_peak,
                    "frac": hbm_achieved / hbm_peak if hbm_peak else None,
                    "peak_source": "MEASURED_PEAKS.json hbm_gbs"},
            "kernel": "k_tile (tile-window MLEM kernel)",
            "work_model": "10 flops per bbox pixel + 18 per in-ellipse pixel",
            "bbox_pixels_per_iter": work_bb.value, "ellipse_pixels_per_iter": work_in.value,
            "tile_ms_per_step": tile_ms / args.steps,
            "peak_source": "measured live: strip_probe_fp32_peak (FMA chains, this GPU)",
            "secondary": secondary_rates(work_in.value, tile_ms / args.steps, clocks),
        },
        "clocks": clocks,
        "gpu_launches": launches,
        "binning": {k: st[k] for k in ("n_tiles_z", "n_tiles_y", "tile_z", "tile_y",
                                       "halo_z", "halo_y", "n_work_items", "n_overflow",
                                       "n_empty", "smem_bytes", "last_setup_ms")},
    }
    if error is not None:
        line["error"] = error
    if e2e is not None:
        line["e2e"] = e2e
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if diff is not None:
        line["differentiable"] = diff
    if osem is not None:
        line["osem8"] = osem
    if io is not None:
        line["io"] = io
    if batched is not None:
        line["batched"] = batched
    if rank == 0 and world == 1 and not args.no_hybrid:
        # the 3D hybrid path (the next scope row, bench.py --path hybrid for the full line)
        import bench_hybrid
        line["hybrid"] = bench_hybrid.summary(local_rank, host_cores,
                                              cpu_baseline=not args.no_cpu_baseline)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if shd is not None:
        shd.close()
    rec.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--events", type=int, default=200_000_000)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--e2e-iters", type=int, default=20)
    ap.add_argument("--ref-events", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-differentiable", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-osem", action="store_true")
    ap.add_argument("--no-io", action="store_true")
    ap.add_argument("--error-events", type=int, default=1_000_000,
                    help="events of the prefix whose 20-iteration image is checked "
                         "against the FP64 oracle (0: no check)")
    ap.add_argument("--path", default="strip", choices=["strip", "hybrid", "precision"],
                    help="strip: the 2D strip MLEM headline; hybrid: the 3D hybrid MLEM; "
                         "precision: the accumulation-mode error study")
    ap.add_argument("--precision-events", type=int, default=1_000_000)
    ap.add_argument("--hybrid-events", type=int, default=10_000_000)
    ap.add_argument("--no-hybrid", action="store_true",
                    help="strip path: leave out the 3D hybrid summary")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", args.gpus))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if world > 1 and "RANK" not in os.environ:
        sys.exit("for --gpus N > 1 launch under torchrun (one rank per GPU)")
    if args.path == "precision":
        import bench_precision
        if rank != 0:
            return 0
        return bench_precision.run(args, local_rank, host_cores)
    if args.path == "hybrid":
        import bench_hybrid
        if args.e2e_iters == 20:
            args.e2e_iters = 10
        if args.impl == "reference":
            return bench_hybrid.reference_arm(args, rank, world, host_cores())
        return bench_hybrid.ours(args, rank, world, local_rank, ClockSampler, host_cores)
    if args.impl == "reference":
        return reference_arm(args, rank, world)
    return ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
