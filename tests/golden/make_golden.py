"""Writes the golden fixtures of tests/golden/ by running the reference's own
2d_strip_reconstruction (compiled from the reference sources into oracle/_ref
by `make -C oracle ref`).  Run here, where the reference checkout exists:

    python tests/golden/make_golden.py

Fixtures (events in the reference binary format: raw little-endian f32
triples z_u z_d dl; images raw f32, n_y rows of n_z):
  c1_small.events.bin      4000 seeded C1 events (generator seed 11)
  c1_small.ref3.npz        reference images after 3 iterations, -T 1:
                           'nocontract' (-ffp-contract=off build) and
                           'default' (GCC's default FMA contraction)
  edge.events.bin          hand-picked and random edge events (out of FOV,
                           NaN/Inf, int16 wrap-around of the centre pixel,
                           extreme tan, clamped boxes)
  edge.ref1.npz            reference image after 1 iteration (nocontract)
  metre.events.bin         2000 events in metres (the reference CLI defaults:
                           R 0.5, L 1, p 0.01, s_z 0.015, s_dl 0.06)
  metre.ref2.npz           reference image after 2 iterations (nocontract)
  text.events.txt          1500 C1 events as text in mixed number formats
  text.ref1.npz            reference image after 1 iteration of the text file
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "j-pet-mlem-old_b200"))

from oracle import oracle as orc  # noqa: E402
import stripmlem as sm  # noqa: E402

C1 = (200.0, 500.0, 200, 250, 2.0, 2.0, 10.0, 42.0)
C1_PHANTOM = [(40, 30, 30, 20, 0, 3.0), (-50, -20, 25, 40, 0, 0.3), (0, 0, 150, 100, 0, 1.0)]
METRE = (0.5, 1.0, 100, 100, 0.01, 0.01, 0.015, 0.06)


def edge_events():
    ev = [
        (0.0, 0.0, 0.0),
        (249.0, 249.0, 0.0),
        (-260.0, -260.0, 10.0),
        (1e5, 1e5, 0.0),
        (131022.0, 131022.0, 0.0),      # centre pixel wraps to column 100
        (-130522.0, -130522.0, 0.0),    # wraps from the other side
        (float("nan"), 0.0, 0.0),
        (0.0, 0.0, float("inf")),
        (0.0, 0.0, float("-inf")),
        (250.0, -250.0, 0.0),           # tan = 1.25
        (-250.0, 250.0, 30.0),
        (1e30, -1e30, 0.0),             # tan overflows
        (0.0, 0.0, 400.0),              # y = -200 (bottom edge)
        (0.0, 0.0, -400.0),             # y = +200 (top edge)
        (0.0, 0.0, -399.0),
        (1.0, -1.0, 0.0),
        (-0.0, 0.0, -0.0),
        (3e9, 3e9, 0.0),                # beyond int32 in pixel units
        (0.0, 0.0, 9e9),
        (600.0, -600.0, 0.0),           # tan = 3
    ]
    rng = np.random.default_rng(5)
    r = rng.uniform(-700, 700, size=(400, 3))
    r[:, 2] *= 0.8
    ev += [tuple(x) for x in r]
    a = np.array(ev, dtype=np.float32)
    return a[:, 0], a[:, 1], a[:, 2]


def main():
    if not orc.ref_available(True) or not orc.ref_available(False):
        sys.exit("build the reference first: make -C oracle ref")
    g = orc.geometry(*C1)
    sc = sm.Scanner(*C1)
    zu, zd, dl = sm.generate_events(sc, C1_PHANTOM, 4000, seed=11)
    orc.write_events_bin(os.path.join(HERE, "c1_small.events.bin"), zu, zd, dl)
    nc, _ = orc.run_ref(g, zu, zd, dl, 3, threads=1, nocontract=True)
    df, _ = orc.run_ref(g, zu, zd, dl, 3, threads=1, nocontract=False)
    np.savez_compressed(os.path.join(HERE, "c1_small.ref3.npz"), nocontract=nc, default=df)

    ezu, ezd, edl = edge_events()
    orc.write_events_bin(os.path.join(HERE, "edge.events.bin"), ezu, ezd, edl)
    ei, _ = orc.run_ref(g, ezu, ezd, edl, 1, threads=1, nocontract=True)
    np.savez_compressed(os.path.join(HERE, "edge.ref1.npz"), nocontract=ei)

    # text events: mixed number formats, '+' signs, exponents (the reference
    # parser turns e>=2 into 10*0.1^(e-1)), and a last line without '\n'
    tzu, tzd, tdl = sm.generate_events(sc, C1_PHANTOM, 1500, seed=12)
    fmts = ["{:.6f}", "{:.3e}", "{:g}", "{:+.4f}", "{:.2E}", "{:.9f}"]
    lines = []
    for i in range(len(tzu)):
        f = fmts[i % len(fmts)]
        lines.append(" ".join(f.format(float(v)) for v in (tzu[i], tzd[i], tdl[i])))
    lines[7] = "1.5e2 -2.0e1 3e-1"
    lines[8] = "12 -7 0"
    lines[9] = "+.5 -.25 10.125"
    with open(os.path.join(HERE, "text.events.txt"), "w") as f:
        f.write("\n".join(lines))  # no newline after the last line
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "r.bin")
        exe = orc.REF_RECON_NOCONTRACT
        subprocess.run([exe, os.path.join(HERE, "text.events.txt"), "-r", "200", "-l", "500",
                        "-p", "2", "--n-y-pixels", "200", "--n-z-pixels", "250", "--s-z", "10",
                        "--s-dl", "42", "-i", "1", "-I", "1", "-T", "1", "-o", out],
                       check=True, capture_output=True)
        ti = np.fromfile(os.path.join(td, "r_1.bin"), dtype="<f4").reshape(200, 250)
    np.savez_compressed(os.path.join(HERE, "text.ref1.npz"), nocontract=ti)

    gm = orc.geometry(*METRE)
    scm = sm.Scanner(*METRE)
    mzu, mzd, mdl = sm.generate_events(
        scm, [(0.1, 0.05, 0.08, 0.05, 30, 2.0), (0.0, 0.0, 0.3, 0.2, 0, 1.0)], 2000, seed=3)
    orc.write_events_bin(os.path.join(HERE, "metre.events.bin"), mzu, mzd, mdl)
    mi, _ = orc.run_ref(gm, mzu, mzd, mdl, 2, threads=1, nocontract=True)
    np.savez_compressed(os.path.join(HERE, "metre.ref2.npz"), nocontract=mi)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
