"""Drop-in command line for the reference's 3d_hybrid_reconstruction
(src/3d/hybrid/reconstruction_cmd.cpp:147-680, its --system matrix path) on
the B200:

    python -m stripmlem.hybrid_cli --system matrix_full.bin \\
        --detector-file det.txt --detector-file-sym sym.txt -p 0.004 \\
        --n-planes 125 --z-left -0.25 --length 0.5 -i 1 -I 10 -o rho.bin responses.bin

Same flags, defaults and file formats as the reference: a full (PETP) system
matrix; the detector description file (detector centres from its polygons);
responses `first second z_up z_dn dl`, binary (16-byte records) or, for
*.txt, text; --sens-to-one, --sensitivity (a 2D map, binary or *.txt),
--inactive; --rho to start from an image; -i blocks x -I iterations.  With
-o base.ext it writes, as the reference's CPU branch does, the naive image of
the events' points `base.ext` (int32) and after each block
`base_NN.ext` (binary32, or text for .txt), each with an NRRD header.
Text responses are parsed as the reference's fast text parser parses them
(its own binary32 rounding, stripmlem.hybrid.read_responses_text).
"""
import argparse
import os
import sys

import numpy as np

from . import hybrid as hy


def _ints(text):
    return [int(v) for v in str(text).replace(",", " ").split()]


def parse(argv=None):
    ap = argparse.ArgumentParser(prog="3d_hybrid_reconstruction")
    ap.add_argument("--system", "-s", required=True, help="system matrix file (full form)")
    ap.add_argument("--detector-file", default=None, help="detector description file")
    ap.add_argument("--geometry", default=None,
                    help="LOR geometry file (weights from --system)")
    ap.add_argument("--detector-file-sym", default=None,
                    help="detector symmetries description file (accepted, not used)")
    ap.add_argument("--n-pixels", "-n", type=int, default=None)
    ap.add_argument("--s-pixel", "-p", type=float, default=None)
    ap.add_argument("--n-planes", type=int, default=None)
    ap.add_argument("--z-left", type=float, default=None)
    ap.add_argument("--length", "-l", type=float, default=2.0)
    ap.add_argument("--s-z", type=float, default=0.015)
    ap.add_argument("--s-dl", type=float, default=0.060)
    ap.add_argument("--blocks", "-i", type=int, default=0)
    ap.add_argument("--iterations", "-I", type=int, default=1)
    ap.add_argument("--output", "-o", default=None)
    ap.add_argument("--sens-to-one", action="store_true")
    ap.add_argument("--sensitivity", default=None, help="external 2D sensitivity")
    ap.add_argument("--inactive", default=None, help="list of inactive detectors")
    ap.add_argument("--rho", default=None, help="start rho")
    ap.add_argument("--cuda-device", "-D", type=int, default=0)
    ap.add_argument("--verbose", "-v", action="count", default=0)
    ap.add_argument("responses", nargs="*")
    return ap.parse_args(argv)


def _read_map(path, n):
    if path.endswith(".txt"):
        return np.loadtxt(path, dtype=np.float32).reshape(-1)[:n]
    return np.fromfile(path, np.float32, n)


def _write_map(base, ext, data, dims, kind):
    fn = base + ext
    if ext == ".txt":
        with open(fn, "w") as f:
            width = dims[0]
            flat = data.reshape(-1)
            for r in range(0, flat.size, width):
                f.write(" ".join(("%d" if kind == "int" else "%g") % v
                                 for v in flat[r:r + width]) + "\n")
    else:
        data.astype(np.int32 if kind == "int" else np.float32).tofile(fn)
    with open(base + ".nrrd", "w") as f:
        f.write("NRRD0001\ntype: %s\nendian: little\ndimension: 3\nsizes: %d %d %d\n"
                "data file: ./%s\nencoding: %s\n"
                % (kind, dims[0], dims[1], dims[2], os.path.basename(fn),
                   "ascii" if ext == ".txt" else "raw"))


def lor_segments(centers):
    """Per LOR index first * (first + 1) / 2 + second: the segment from the
    centre of detector `second` to that of `first` (start x, y, end x, y)."""
    c = np.asarray(centers, np.float32)
    nd = len(c)
    seg = np.zeros(((nd + 1) * nd // 2, 4), np.float32)
    for a in range(nd):
        for b in range(a + 1):
            seg[a * (a + 1) // 2 + b] = (c[b, 0], c[b, 1], c[a, 0], c[a, 1])
    return seg


def naive_image(kept, resp, nc, nr, n_planes, p, llx, lly, z_left, segments):
    """Reconstruction::naive (reconstruction.h:394-405): the count of kept
    events per voxel of their point (the LOR's mid point + up along it, z =
    right), binary32 as the reference computes it.  kept: the kept responses'
    indices."""
    f32 = np.float32
    idx = np.asarray(kept, np.int64)
    first, second = resp[0][idx].astype(np.int64), resp[1][idx].astype(np.int64)
    zu, zd, dl = (np.asarray(a, f32)[idx] for a in resp[2:])
    sg = np.asarray(segments, f32)[first * (first + 1) // 2 + second]
    cs, ce = sg[:, 0:2], sg[:, 2:4]
    mid = (cs + ce) / f32(2)
    v = ce - cs
    ln = np.sqrt(v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1])
    d = v / ln[:, None]
    R = ln / f32(2)
    tan = (zu - zd) / (f32(2) * R)
    up = f32(-0.5) * (dl / np.sqrt(f32(1) + tan * tan))
    right = f32(0.5) * (zu + zd + (f32(2) * up * tan))
    x = mid[:, 0] + d[:, 0] * up
    y = mid[:, 1] + d[:, 1] * up
    # PixelGrid::pixel_at (pixel_grid.h:59-62) on the grid's lower-left corner
    ix = np.floor((x - f32(llx)) / f32(p)).astype(np.int64)
    iy = np.floor((y - f32(lly)) / f32(p)).astype(np.int64)
    iz = np.floor((right - f32(z_left)) / f32(p)).astype(np.int64)
    ok = (ix >= 0) & (ix < nc) & (iy >= 0) & (iy < nr) & (iz >= 0) & (iz < n_planes)
    img = np.zeros((n_planes, nr, nc), np.int32)
    np.add.at(img, (iz[ok], iy[ok], ix[ok]), 1)
    return img


def main(argv=None):
    a = parse(argv)
    m = hy.SystemMatrix.read(a.system)
    inactive = _ints(a.inactive) if a.inactive else None
    geom = None
    if a.geometry:
        # run_with_geometry (reconstruction_cmd.cpp:281-363): the pixel grid
        # (size and lower-left corner) from the file, the weights from the
        # matrix; --s-pixel (default: the file's pixel size) only sets the
        # default z_left, as there
        if "," in a.system:
            raise SystemExit("per-plane system matrices (a comma-separated --system list) "
                             "are not supported; give one matrix")
        geom = hy.read_geometry(a.geometry)
        nc, nr, gp, llx, lly = geom["grid"]
        if abs(llx + gp * nc / 2) > 1e-6 * gp or abs(lly + gp * nr / 2) > 1e-6 * gp:
            raise SystemExit("the geometry's pixel grid must be centred on the origin "
                             f"(lower left {llx}, {lly} for {nc} x {nr} pixels of {gp})")
        n = a.n_pixels or max(nc, nr)
        if a.s_pixel is None:
            a.s_pixel = gp
        p_grid = gp
    else:
        if a.s_pixel is None or a.detector_file is None:
            raise SystemExit("--s-pixel and --detector-file are required with --system")
        n = a.n_pixels or m.n_pixels_in_row
        nc = nr = n
        p_grid = a.s_pixel
        llx = lly = -p_grid * n / 2
    n_planes = a.n_planes if a.n_planes is not None else n
    z_left = a.z_left if a.z_left is not None else -n_planes * a.s_pixel / 2
    if a.verbose:
        print(f"3D hybrid reconstruction:\n    detectors = {m.n_detectors}", file=sys.stderr)
        print(f"   pixel grid = {nc} x {nr} / {p_grid}", file=sys.stderr)
    rec = hy.HybridReconstruction(nc, nr, n_planes, p_grid, z_left, a.length, a.s_z, a.s_dl,
                                  device=a.cuda_device)
    if geom is not None:
        soa = hy.geometry_soa_from_file(geom, m)
        rec.set_geometry_soa(soa["n_detectors"], soa["segments"], soa["pixels"],
                             soa["positions"], soa["weights"], soa["lor_begin"],
                             soa["lor_end"])
        segments = soa["segments"]
    else:
        polygons = hy.read_detector_file(a.detector_file)
        if len(polygons) != m.n_detectors:
            raise SystemExit("n_detectors mismatch")
        centers = hy.detector_centers(polygons)
        rec.set_geometry_from_matrix(centers, m, inactive)
        segments = lor_segments(centers)
    if a.sensitivity:
        rec.set_sensitivity(_read_map(a.sensitivity, nc * nr))
    elif a.sens_to_one:
        rec.set_sensitivity("one")
    else:
        rec.set_sensitivity()
    parts = [hy.read_responses(fn) for fn in a.responses]
    resp = tuple(np.concatenate([p[k] for p in parts]) if parts else np.zeros(0)
                 for k in range(5))
    rec.set_responses(*resp)
    st = rec.stats()
    if a.verbose:
        print(f"       events = {st['n_events']}", file=sys.stderr)
    start = 0
    if a.rho:
        rec.rho = _read_map(a.rho, nc * nr * n_planes)
        base = os.path.splitext(a.rho)[0]
        digits = len(base) - len(base.rstrip("0123456789"))
        start = int(base[len(base) - digits:]) if digits else 0
    out_base, out_ext = os.path.splitext(a.output) if a.output else (None, None)
    dims = (nc, nr, n_planes)
    if out_base:
        _write_map(out_base, out_ext,
                   naive_image(rec.frames()["index"], resp, nc, nr, n_planes, p_grid, llx, lly,
                               z_left, segments), dims, "int")
    n_total = a.blocks * a.iterations
    digits = len(str(n_total)) if n_total > 0 else 1
    for block in range(a.blocks):
        first_it = block * a.iterations
        todo = [i for i in range(first_it, first_it + a.iterations) if i >= start]
        if todo:
            rec(len(todo))
        it = (block + 1) * a.iterations
        if it <= start or not out_base:
            continue
        _write_map(f"{out_base}_{it:0{digits}d}", out_ext, rec.rho, dims, "float")
    st = rec.stats()
    print(f"  event count = {st['n_events']}", file=sys.stderr)
    if st["n_events"]:
        print(f"  voxel count = {st['used_voxels']}"
              f"({st['used_voxels'] / st['n_events']:g} / event)", file=sys.stderr)
        print(f"  pixel count = {st['used_pixels']}"
              f"({st['used_pixels'] / st['n_events']:g} / event)", file=sys.stderr)
    rec.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
