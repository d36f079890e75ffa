"""Writes tests/golden/hybrid_small.npz by running the reference's own
3d_hybrid_reconstruction (compiled from the reference sources into oracle/_ref
by `make -C oracle ref`; the -ffp-contract=off parity build).  Run here,
where the reference checkout exists:

    python tests/golden/make_hybrid_golden.py

The inputs are seeded synthetic stand-ins (the reference ships no 3D hybrid
data): a two-ring barrel of 64 square detectors, the analytic system matrix
of stripmlem.hybrid.synthetic_matrix on a 24 x 24 grid of 1 cm pixels, and
3000 responses of stripmlem.hybrid.generate_responses (host generator,
seed 5) in a two-cylinder phantom; 24 planes, z_left -0.12 m, L 0.3 m,
sigma_z 0.01 m, sigma_dl 0.04 m.  The npz holds the inputs (detector
polygons, matrix elements, responses, setup) and, per case, the reference's
image, its naive image (event points per voxel) and its event / pixel / voxel
counts:
  calc     calculate_sensitivity, 3 iterations
  one      --sens-to-one, 2 iterations
  inactive --inactive 3,40, 2 iterations
  geom     --geometry: a LOR geometry file of the same flattened geometry
           (tests rebuild it with write_golden_geometry), weights loaded from
           the matrix, 3 iterations
  text     the same responses as text in mixed number formats (text_in),
           calculate_sensitivity, 3 iterations
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "j-pet-mlem-old_b200"))
sys.path.insert(0, ROOT)

from stripmlem import hybrid as hy  # noqa: E402
from oracle import hybrid as oh  # noqa: E402

SETUP = dict(n=24, p=0.01, n_planes=24, z_left=-0.12, length=0.3, sigma_z=0.01, sigma_dl=0.04)
CASES = {"calc": (3, ()), "one": (2, ("--sens-to-one",)), "inactive": (2, ("--inactive", "3,40"))}


def counts(stderr):
    g = lambda k: int(re.search(rf"{k} count = (\d+)", stderr).group(1))  # noqa: E731
    return np.array([g("event"), g("pixel"), g("voxel")], np.int64)


def write_golden_geometry(path, b, m):
    """The LOR geometry file of the --geometry case: the oracle's flattened
    geometry of the matrix (segments between detector centres, pixel infos
    sorted by position), distance 0, fill 1, weight 0."""
    s = SETUP
    setup = oh.setup(s["n"], s["n"], s["n_planes"], s["p"], s["z_left"], s["length"],
                     s["sigma_z"], s["sigma_dl"])
    geo = oh.soa_from_matrix(setup, b.centers, m)
    lors = {}
    for li in range(len(geo["lbeg"])):
        lb, le = int(geo["lbeg"][li]), int(geo["lend"][li])
        infos = np.zeros(le - lb, hy._PIXEL_INFO)
        infos["x"], infos["y"] = geo["pix"][lb:le, 0], geo["pix"][lb:le, 1]
        infos["t"] = geo["pos"][lb:le]
        infos["fill"] = 1.0
        lors[li] = (geo["seg"][li, :4], 0.0, infos)
    p = np.float32(s["p"])
    ll = float(-p * np.float32(s["n"]) / np.float32(2))
    hy.write_geometry(path, b.n_detectors, (s["n"], s["n"], s["p"], ll, ll), lors)


def main():
    if not oh.ref_available():
        sys.exit("build the reference first: make -C oracle ref")
    b = hy.Barrel(radius=(0.15, 0.17), n_detectors=(32, 32), rotation=(0, 0.5),
                  w_detector=0.009, h_detector=0.015)
    s = SETUP
    m = hy.synthetic_matrix(b, s["n"], s["p"], 0.12)
    phantom = [(0.02, 0.01, 0.0, 0.05, 0.06, 2.0), (0.0, 0.0, 0.0, 0.1, 0.12, 1.0)]
    r = hy.generate_responses(b, phantom, 3000, s["length"], s["sigma_z"], s["sigma_dl"],
                              seed=5)
    out = {"polygons": b.polygons, "m_lor_a": m.lor_a, "m_lor_b": m.lor_b, "m_px": m.px,
           "m_py": m.py, "m_hits": m.hits,
           "m_meta": np.array([m.n_pixels_in_row, m.n_emissions, m.n_detectors], np.int64),
           "r_first": r[0], "r_second": r[1], "r_z_up": r[2], "r_z_dn": r[3], "r_dl": r[4],
           "setup": np.array([s["n"], s["n_planes"]], np.int64),
           "setup_f": np.array([s["p"], s["z_left"], s["length"], s["sigma_z"], s["sigma_dl"]])}
    for name, (n_iter, extra) in CASES.items():
        d = oh.tempdir()
        paths = {k: os.path.join(d, f) for k, f in
                 (("m", "m.bin"), ("det", "det.txt"), ("sym", "sym.txt"), ("resp", "r.bin"))}
        m.write(paths["m"])
        b.write_detector_file(paths["det"])
        hy.write_symmetry_file(paths["sym"], b.n_detectors)
        hy.write_responses(paths["resp"], *r)
        img, err = oh.run_ref(d, paths["m"], paths["det"], paths["sym"], paths["resp"], s["n"],
                              s["p"], s["n_planes"], s["z_left"], s["length"], s["sigma_z"],
                              s["sigma_dl"], n_iter, extra=extra)
        out[f"{name}_rho"] = img
        out[f"{name}_naive"] = oh.ref_naive(d, s["n"], s["n_planes"])
        out[f"{name}_counts"] = counts(err)
        print(name, out[f"{name}_counts"], float(img.sum()))
    # the --geometry path: a LOR geometry file holding the calc case's
    # flattened geometry (weights left 0), the weights loaded from the matrix
    geom_path = os.path.join(oh.tempdir(), "g.bin")
    write_golden_geometry(geom_path, b, m)
    d = oh.tempdir()
    paths = {k: os.path.join(d, f) for k, f in
             (("m", "m.bin"), ("det", "det.txt"), ("sym", "sym.txt"), ("resp", "r.bin"))}
    m.write(paths["m"])
    b.write_detector_file(paths["det"])
    hy.write_symmetry_file(paths["sym"], b.n_detectors)
    hy.write_responses(paths["resp"], *r)
    img, err = oh.run_ref(d, paths["m"], paths["det"], paths["sym"], paths["resp"], s["n"],
                          s["p"], s["n_planes"], s["z_left"], s["length"], s["sigma_z"],
                          s["sigma_dl"], 3, extra=("--geometry", geom_path))
    out["geom_rho"] = img
    out["geom_counts"] = counts(err)
    print("geometry", out["geom_counts"], float(img.sum()))
    # text responses in mixed number formats, read by the reference's fast
    # text parser (its own binary32 rounding)
    rng = np.random.default_rng(6)
    fmts = ["%.9g", "%.4e", "%+.6f", "%.7g"]
    lines = []
    for i in range(len(r[0])):
        f = fmts[rng.integers(0, len(fmts))]
        lines.append(f"{int(r[0][i])} {int(r[1][i])} " +
                     " ".join(f % float(v) for v in (r[2][i], r[3][i], r[4][i])))
    text = "\n".join(lines) + "\n"
    d = oh.tempdir()
    paths = {k: os.path.join(d, f) for k, f in
             (("m", "m.bin"), ("det", "det.txt"), ("sym", "sym.txt"), ("resp", "r.txt"))}
    m.write(paths["m"])
    b.write_detector_file(paths["det"])
    hy.write_symmetry_file(paths["sym"], b.n_detectors)
    with open(paths["resp"], "w") as f:
        f.write(text)
    img, err = oh.run_ref(d, paths["m"], paths["det"], paths["sym"], paths["resp"], s["n"],
                          s["p"], s["n_planes"], s["z_left"], s["length"], s["sigma_z"],
                          s["sigma_dl"], 3)
    out["text_in"] = np.array(text)
    out["text_rho"] = img
    out["text_counts"] = counts(err)
    print("text", out["text_counts"], float(img.sum()))
    np.savez_compressed(os.path.join(HERE, "hybrid_small.npz"), **out)


if __name__ == "__main__":
    main()
