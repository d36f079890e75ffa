"""Precision study of the strip MLEM accumulation modes (bench.py --path precision).

Workload: the 250 x 200 geometry of 2 mm pixels (two 500 mm strips at
y = +-200 mm, sigma_z 10 mm, sigma_dl 42 mm), the 3-ellipse phantom, seed 1;
the first --precision-events events (default 1e6) of the 5e7-event stream --
the full-FP64 oracle over 5e7 events and 50 iterations would take hours on
the host, and the per-event normalisation sums whose rounding the modes
differ in do not depend on how many events there are.

Columns, each after 5, 20 and 50 MLEM iterations (reference CPU semantics),
against the full-binary64 oracle (binary64 pixel sets and arithmetic,
oracle/strip_oracle.c):
  gpu_fp32    kernel and scatter in binary32, per-lane row sums in binary32
  gpu_kahan   ... compensated (Kahan) binary32 per-lane sums (the default)
  gpu_fp64    ... binary64 per-lane sums
              (all three: binary64 across lanes, binary64 image reductions)
  reference   the reference's own CPU binary (oracle/_ref/2d_strip_reconstruction,
              default flags, all host threads): binary32 everywhere, the
              per-event sum in y-then-z order, per-thread images summed
              serially in binary32 (src/2d/strip/reconstruction.h:143-149,
              255-290)
  oracle_f64_sets32  the FP64 oracle with the reference's binary32 pixel
              sets (what the 1e-4 parity bar is stated against)
Errors: rel_l2 = |x - x64| / |x64|; max_abs_rel_peak = max |x - x64| /
max x64; max_rel_1pct = max |x - x64| / x64 over pixels above 1 % of the
peak.  table_vs_f64_sets32 holds the same against oracle_f64_sets32, and
mode_spread_rel_l2 the largest rel-L2 between gpu_fp32 / gpu_kahan and
gpu_fp64.
"""
import json
import os
import re
import subprocess
import tempfile
import time

import numpy as np

GEOM = dict(radius=200.0, length=500.0, n_y=200, n_z=250, p=2.0, s_z=10.0, s_dl=42.0)
PHANTOM = [(40, 30, 30, 20, 0, 3.0), (-50, -20, 25, 40, 0, 0.3), (0, 0, 150, 100, 0, 1.0)]
SEED = 1
CHECKPOINTS = (5, 20, 50)


def errors(x, ref):
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    d = np.abs(x - ref)
    peak = ref.max()
    big = ref > 0.01 * peak
    return {"rel_l2": float(np.linalg.norm(x - ref) / np.linalg.norm(ref)),
            "max_abs_rel_peak": float(d.max() / peak),
            "max_rel_1pct": float((d[big] / ref[big]).max())}


def oracle_series(orc, g, ev, sets_f32):
    out, rho, done = {}, None, 0
    for it in CHECKPOINTS:
        rho = orc.mlem_f64(g, *ev, it - done, rho=rho, sets_f32=sets_f32)
        done = it
        out[it] = rho.copy()
    return out


def reference_series(orc, g, ev, cores):
    """The reference binary, 10 blocks of 5 iterations: images after 5, 10,
    ..., 50 (reconstruction_cmd.cpp:270-293 writes one per block)."""
    if not orc.ref_available(nocontract=False):
        return None, None
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "events.bin")
        orc.write_events_bin(path, *ev)
        out = os.path.join(td, "r.bin")
        cmd = [orc.REF_RECON, path, "-r", repr(g.radius), "-l", repr(g.scintillator_length),
               "-p", repr(g.pixel_width), "--n-y-pixels", str(g.n_y_pixels),
               "--n-z-pixels", str(g.n_z_pixels), "--s-z", repr(g.sigma_z),
               "--s-dl", repr(g.sigma_dl), "-i", "10", "-I", "5", "-T", str(cores),
               "-o", out]
        t0 = time.perf_counter()
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=3600)
        secs = time.perf_counter() - t0
        if p.returncode != 0:
            raise RuntimeError(f"reference failed: {p.stderr[-500:]}")
        imgs = {}
        for f in os.listdir(td):
            m = re.match(r"r_0*(\d+)\.bin$", f)
            if m and int(m.group(1)) in CHECKPOINTS:
                imgs[int(m.group(1))] = np.fromfile(os.path.join(td, f), dtype="<f4").reshape(
                    g.n_y_pixels, g.n_z_pixels)
    return imgs, secs


def run(args, local_rank, host_cores):
    import stripmlem as sm
    from oracle import oracle as orc
    n = args.precision_events
    g = orc.geometry(GEOM["radius"], GEOM["length"], GEOM["n_y"], GEOM["n_z"], GEOM["p"],
                     GEOM["p"], GEOM["s_z"], GEOM["s_dl"])
    ev = orc.generate_events(g, PHANTOM, n, SEED)
    sc = sm.Scanner(GEOM["radius"], GEOM["length"], GEOM["n_y"], GEOM["n_z"], GEOM["p"],
                    GEOM["p"], GEOM["s_z"], GEOM["s_dl"])
    cols = {}
    for name, acc in (("gpu_fp32", sm.ACCUM_FP32), ("gpu_kahan", sm.ACCUM_KAHAN),
                      ("gpu_fp64", sm.ACCUM_FP64)):
        with sm.Reconstruction(sc, device=local_rank, mode=sm.MODE_CPU, accumulation=acc) as r:
            r.set_events(*ev)
            imgs, done = {}, 0
            for it in CHECKPOINTS:
                r(None, it - done)
                done = it
                imgs[it] = r.rho
        cols[name] = imgs
    t0 = time.perf_counter()
    ref64 = oracle_series(orc, g, ev, sets_f32=False)
    t64 = time.perf_counter() - t0
    cols["oracle_f64_sets32"] = oracle_series(orc, g, ev, sets_f32=True)
    cores = host_cores()
    ref_imgs, ref_s = reference_series(orc, g, ev, cores)
    if ref_imgs is not None:
        cols["reference"] = ref_imgs
    table = {name: {str(it): errors(imgs[it], ref64[it]) for it in CHECKPOINTS if it in imgs}
             for name, imgs in cols.items()}
    # against the FP64 oracle with the reference's binary32 sets (the parity bar's reference),
    # and the spread between the three GPU accumulation modes
    sets32 = cols["oracle_f64_sets32"]
    table_sets32 = {name: {str(it): errors(imgs[it], sets32[it]) for it in CHECKPOINTS
                           if it in imgs}
                    for name, imgs in cols.items() if name != "oracle_f64_sets32"}
    spread = {str(it): max(errors(cols[a][it], cols["gpu_fp64"][it])["rel_l2"]
                           for a in ("gpu_fp32", "gpu_kahan")) for it in CHECKPOINTS}
    line = {"metric": "strip MLEM image error vs the full-FP64 oracle", "path": "precision",
            "config": {"workload": "strip MLEM, 250x200 image of 2 mm pixels, R=200 mm, "
                                   "L=500 mm, sigma_z=10 mm, sigma_dl=42 mm, 3-ellipse phantom",
                       "events": n, "seed": SEED,
                       "sample": f"first {n} events of the 5e7-event stream",
                       "iterations": list(CHECKPOINTS)},
            "data": "synthetic", "table": table, "table_vs_f64_sets32": table_sets32,
            "mode_spread_rel_l2": spread,
            "oracle_full_fp64_s": t64, "reference_s": ref_s,
            "reference_threads": cores if ref_imgs is not None else None}
    print(json.dumps(line), flush=True)
    return 0
