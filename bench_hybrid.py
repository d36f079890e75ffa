"""Benchmark of the 3D hybrid list-mode TOF MLEM path on B200 (bench.py --path hybrid).

Workload: the J-PET big barrel (three rings of 48, 48 and 96 square
scintillators, 7 x 19 mm, at 425 / 467.5 / 575 mm inner radius, the second
and third turned by half a detector), a 200 x 200 grid of 4 mm pixels
(field of view radius 400 mm) x 125 planes of 4 mm covering the 500 mm barrel
length, sigma_z 15 mm, sigma_dl 60 mm (the reference CLI's defaults); the
analytic stand-in system matrix of stripmlem.hybrid.synthetic_matrix (7.15e6
LOR pixel infos) and 1e7 seeded synthetic responses of a three-cylinder
phantom.  A step is one MLEM iteration over all responses; the metric is
Mevent*iter/s (frame events x iterations / device time).  The responses'
frame events (320 MB) exceed L2; the 20 MB volume stays L2-resident by
design.
"""
import json
import os
import re
import subprocess
import tempfile
import time

import numpy as np

METRIC = ("3D hybrid TOF-MLEM Mevent·iter/s on 1 B200 (big barrel, 200x200x125 voxels "
          "of 4 mm) at ≤1e-4 rel-L2 vs FP64 oracle")
UNIT = "Mevent*iter/s"
N_PIX, PIXEL, N_PLANES, Z_LEFT = 200, 0.004, 125, -0.25
LENGTH, SIGMA_Z, SIGMA_DL, FOV = 0.5, 0.015, 0.06, 0.4
PHANTOM = [(0.1, 0.05, 0.02, 0.05, 0.05, 3.0), (-0.15, 0.0, -0.05, 0.04, 0.08, 0.2),
           (0.0, 0.0, 0.0, 0.3, 0.2, 1.0)]
SEED = 20260202
# Algorithmic FP32 work per voxel and iteration: GaussianKernel::normalized
# as the reference evaluates it per voxel (distance 2, the a and b vectors 12,
# a'Sa and b'Sb 16, c / sqrt 2, exponent and exp 2, product 1, sensitivity
# 19 with its two arctangents, quotient 1), weight 2, denominator 2, scatter 2.
FLOPS_PER_VOXEL = 63.0
# DRAM bytes (read + write) per frame event of one k_mlem launch, from an ncu
# capture of the first 1e6 responses of this workload (149.6 MB read + 893.6
# MB written, dram__bytes_read.sum / dram__bytes_write.sum of one launch): frame
# events, LOR pixel infos and weights, and the per-warp weight slabs' lines
# that L2 writes back before they are read again.
MLEM_DRAM_BYTES_PER_EVENT = (149.592576e6 + 893.551104e6) / 1e6


def config(n, e2e_iters):
    return {"workload": "3D hybrid big barrel: 3 rings (48/48/96) of 7x19 mm detectors, "
                        "200x200 pixels of 4 mm x 125 planes, sigma_z 15 mm, sigma_dl 60 mm, "
                        "analytic system matrix, 3-cylinder phantom",
            "responses": n, "voxels": N_PIX * N_PIX * N_PLANES,
            "l2": "frame events (32 B x responses) exceed L2; no flush",
            "e2e_iterations_per_step": e2e_iters}


def setup(n, device):
    from stripmlem import hybrid as hy
    b = hy.Barrel()
    m = hy.synthetic_matrix(b, N_PIX, PIXEL, FOV)
    r = hy.generate_responses(b, PHANTOM, n, LENGTH, SIGMA_Z, SIGMA_DL, seed=SEED,
                              device=device)
    return b, m, r


def run_reference(b, m, r, n_sample, iters, warmup, cores):
    """oracle/_ref/3d_hybrid_reconstruction (the reference's own CPU binary,
    default flags) on the first n_sample responses: per-iteration times from
    its -vv benchmark lines."""
    from oracle import hybrid as oh
    from stripmlem import hybrid as hy
    if not oh.ref_available(nocontract=False):
        return None
    with tempfile.TemporaryDirectory() as td:
        paths = {k: os.path.join(td, f) for k, f in
                 (("m", "m.bin"), ("det", "det.txt"), ("sym", "sym.txt"), ("r", "r.bin"))}
        m.write(paths["m"])
        b.write_detector_file(paths["det"])
        hy.write_symmetry_file(paths["sym"], b.n_detectors)
        hy.write_responses(paths["r"], *(a[:n_sample] for a in r))
        cmd = [oh.REF_BIN, "--system", paths["m"], "--detector-file", paths["det"],
               "--detector-file-sym", paths["sym"], "-n", str(N_PIX), "-p", repr(PIXEL),
               "--n-planes", str(N_PLANES), "--z-left", repr(Z_LEFT), "--length", repr(LENGTH),
               "--s-z", repr(SIGMA_Z), "--s-dl", repr(SIGMA_DL), "-i", "1",
               "-I", str(iters + warmup), "-T", str(cores), "-vv", paths["r"]]
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=3600, cwd=td)
    if p.returncode != 0:
        raise RuntimeError(f"reference failed: {p.stderr[-1000:]}")
    times = [float(x.group(2)) for x in
             re.finditer(r"^\s*(\d+)\s+([0-9.]+)\s*$", p.stdout, flags=re.M)]
    events = int(re.search(r"event count = (\d+)", p.stderr).group(1))
    times = times[warmup:] if len(times) > warmup else times
    value = events * len(times) / (sum(times) / 1e3) / 1e6
    sample = (f"first {n_sample} responses of the workload ({events} frame events), "
              f"{len(times)} timed iterations (+{warmup} warm-up) of "
              f"oracle/_ref/3d_hybrid_reconstruction -T {cores} -vv")
    return value, sample


def reference_arm(args, rank, world, cores):
    if rank != 0:
        return 0
    b, m, r = setup(args.hybrid_events, -1)
    n_sample = args.ref_events or min(args.hybrid_events, 2000 * cores)
    out = run_reference(b, m, r, n_sample, args.steps, args.warmup, cores)
    if out is None:
        print(json.dumps({"impl": "reference", "path": "hybrid",
                          "unavailable": "oracle/_ref/3d_hybrid_reconstruction was not built"}))
        return 0
    value, sample = out
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
            "path": "hybrid", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config(args.hybrid_events, args.e2e_iters),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def ours(args, rank, world, local_rank, clock_sampler, host_cores):
    import ctypes

    import torch
    from stripmlem import _lib
    from stripmlem import hybrid as hy
    if world > 1:
        raise SystemExit("--path hybrid runs on one GPU")
    torch.cuda.set_device(local_rank)
    n = args.hybrid_events
    b, m, r = setup(n, local_rank)
    # pinned host copies of the responses for the end-to-end leg
    pin = [torch.empty(len(a), dtype={np.int16: torch.int16, np.float32: torch.float32}[a.dtype.type],
                       pin_memory=True) for a in r]
    for t, a in zip(pin, r):
        t.numpy()[:] = a
    host = [t.numpy() for t in pin]
    rec = hy.HybridReconstruction(N_PIX, N_PIX, N_PLANES, PIXEL, Z_LEFT, LENGTH, SIGMA_Z, SIGMA_DL,
                                  device=local_rank)
    rec.set_geometry_from_matrix(b.centers, m)
    rec.set_sensitivity()
    rec.set_responses(*host)
    st = rec.stats()
    n_events, voxels = st["n_events"], st["used_voxels"]
    peak = ctypes.c_double()
    lib = _lib.load()
    if lib.strip_probe_fp32_peak(local_rank, ctypes.byref(peak)) != 0:
        peak.value = float("nan")

    rec(args.warmup)
    torch.cuda.synchronize()
    ms = []
    with clock_sampler(local_rank) as clk:
        for _ in range(args.steps):
            rec(1)
            ms.append(rec.stats()["last_iteration_ms"])  # CUDA events on the library stream
    t_ms = float(sum(ms))
    value = n_events * args.steps / (t_ms / 1e3) / 1e6
    achieved = FLOPS_PER_VOXEL * voxels / (t_ms / args.steps / 1e3) / 1e12
    clocks = clk.summary()

    # end to end through the public API: responses from pinned host memory,
    # e2e_iters iterations, the image back to the host, every step
    e2e_val = None
    h2d = 16 * n
    d2h = 4 * N_PIX * N_PIX * N_PLANES
    if args.e2e_steps > 0:
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            rec.set_responses(*host)
            rec(args.e2e_iters)
            img = rec.rho
        t = time.perf_counter() - t0
        e2e_val = n_events * args.e2e_iters * args.e2e_steps / t / 1e6
        assert np.isfinite(img).all()

    cpu = None
    if not args.no_cpu_baseline:
        cores = host_cores()
        out = run_reference(b, m, r, args.ref_events or min(n, 2000 * cores), 2, 1, cores)
        if out is not None:
            cpu = {"value": out[0], "unit": UNIT, "cores": cores, "kind": "reference",
                   "sample": out[1]}
    rec.close()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "path": "hybrid", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": config(n, args.e2e_iters),
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak.value,
                     "unit": "TFLOP/s", "frac": achieved / peak.value if peak.value else None,
                     "traffic": MLEM_DRAM_BYTES_PER_EVENT * n_events,
                     "model": f"{FLOPS_PER_VOXEL:.0f} flop x {voxels} voxels per iteration; "
                              "peak = live FP32 FMA probe"},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": args.steps,
        "clocks": clocks,
        "work": {"frame_events": n_events, "voxels_per_iteration": voxels,
                 "pixel_infos": st["n_pixel_infos"]},
    }
    print(json.dumps(line), flush=True)
    return 0


def summary(local_rank, host_cores, n=10_000_000, warmup=3, steps=3, e2e_iters=3,
            cpu_baseline=True):
    """A compact measurement of the hybrid workload for the strip bench's JSON
    line: device-timed iterations, one end-to-end step and the reference's
    CPU binary on a bounded sample."""
    import ctypes

    from stripmlem import _lib
    from stripmlem import hybrid as hy
    b, m, r = setup(n, local_rank)
    with hy.HybridReconstruction(N_PIX, N_PIX, N_PLANES, PIXEL, Z_LEFT, LENGTH, SIGMA_Z,
                                 SIGMA_DL, device=local_rank) as rec:
        rec.set_geometry_from_matrix(b.centers, m)
        rec.set_sensitivity()
        rec.set_responses(*r)
        st = rec.stats()
        rec(warmup)
        ms = []
        for _ in range(steps):
            rec(1)
            ms.append(rec.stats()["last_iteration_ms"])
        t_ms = float(sum(ms))
        t0 = time.perf_counter()
        rec.set_responses(*r)
        rec(e2e_iters)
        img = rec.rho
        t_e2e = time.perf_counter() - t0
        assert np.isfinite(img).all()
    peak = ctypes.c_double()
    if _lib.load().strip_probe_fp32_peak(local_rank, ctypes.byref(peak)) != 0:
        peak.value = float("nan")
    value = st["n_events"] * steps / (t_ms / 1e3) / 1e6
    achieved = FLOPS_PER_VOXEL * st["used_voxels"] / (t_ms / steps / 1e3) / 1e12
    out = {"metric": METRIC, "value": value, "unit": UNIT, "steps": steps, "warmup": warmup,
           "ms_per_step": t_ms / steps, "config": config(n, e2e_iters),
           "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak.value,
                        "unit": "TFLOP/s",
                        "frac": achieved / peak.value if peak.value else None,
                        "traffic": MLEM_DRAM_BYTES_PER_EVENT * st["n_events"],
                        "model": f"{FLOPS_PER_VOXEL:.0f} flop x {st['used_voxels']} voxels"},
           "e2e": {"value": st["n_events"] * e2e_iters / t_e2e / 1e6, "unit": UNIT,
                   "h2d_bytes_per_step": 16 * n, "d2h_bytes_per_step": 4 * N_PIX * N_PIX * N_PLANES},
           "gpu_launches": steps, "dtype": "f32", "data": "synthetic"}
    if cpu_baseline:
        cores = host_cores()
        ref = run_reference(b, m, r, min(n, 2000 * cores), 2, 1, cores)
        if ref is not None:
            out["cpu_baseline"] = {"value": ref[0], "unit": UNIT, "cores": cores,
                                   "kind": "reference", "sample": ref[1]}
    return out
