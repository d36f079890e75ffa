"""Writes tests/golden/gate_small.npz by running the reference's own
3d_tool_convert (compiled from the reference sources into oracle/_ref by
`make -C oracle ref`).  Run here, where the reference checkout exists:

    python tests/golden/make_gate_golden.py

Inputs (seeded synthetic, in the GATE text layouts the converter reads):
  warsaw      600 hit pairs `x1 y1 z1 t1 x2 y2 z2 t2 e1 e2 scatter` (cm, ps):
              points near detector centres of the big barrel, points between
              detectors, |z| beyond the barrel, scatter flags 0..3
  tbednarski  300 records `du dd t_ul t_ur t_dl t_dr` (detectors from 1, ps)
Outputs, the reference's stdout parsed as numbers (it prints 6 significant
digits): warsaw with --s-z 0 --s-dl 0 (all pairs, and --only 1) and with
--s-z 0.01 --s-dl 0.05 --seed 5 (smeared), tbednarski default and
--relative-time.
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "j-pet-mlem-old_b200"))

from stripmlem import hybrid as hy  # noqa: E402

EXE = os.path.join(ROOT, "oracle", "_ref", "3d_tool_convert")
SCANNER = ["--w-detector", "0.007", "--h-detector", "0.019", "--radius", "0.4155,0.458,0.5655",
           "--n-detectors", "48,48,96", "--rotation", "0,0.5,0.5", "--length", "0.5"]


def warsaw_lines(rng, n):
    b = hy.Barrel()
    c = b.centers.astype(np.float64)
    lines = []
    for i in range(n):
        k1, k2 = rng.integers(0, b.n_detectors, 2)
        p1 = c[k1] + rng.uniform(-0.002, 0.002, 2)
        p2 = c[k2] + rng.uniform(-0.002, 0.002, 2)
        if i % 17 == 0:  # between detectors of the inner ring
            a = 2 * np.pi * (rng.integers(0, 48) + 0.5) / 48
            p1 = 0.425 * np.array([np.cos(a), np.sin(a)])
        z1, z2 = rng.uniform(-30, 30, 2)
        if i % 23 == 0:
            z2 = 26.0  # beyond L/2 = 25 cm
        t1, t2 = rng.uniform(0, 3000, 2)
        sc = i % 4
        lines.append(f"{p1[0]*100:.6f} {p1[1]*100:.6f} {z1:.4f} {t1:.3f} "
                     f"{p2[0]*100:.6f} {p2[1]*100:.6f} {z2:.4f} {t2:.3f} 0.511 0.34 {sc}")
    return lines


def tbednarski_lines(rng, n):
    lines = []
    for _ in range(n):
        du, dd = rng.integers(1, 385, 2)
        t = rng.uniform(0, 5000, 4)
        lines.append(f"{du} {dd} {t[0]:.3f} {t[1]:.3f} {t[2]:.3f} {t[3]:.3f}")
    return lines


def run(args, lines, tmp):
    path = os.path.join(tmp, "in.txt")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    p = subprocess.run([EXE] + args + [path], capture_output=True, text=True, check=True)
    rows = [ln.split() for ln in p.stdout.splitlines() if ln.strip()]
    return np.array([[float(v) for v in r] for r in rows]).reshape(-1, len(rows[0]) if rows else 5)


def main():
    import tempfile
    if not os.path.exists(EXE):
        sys.exit("build the reference first: make -C oracle ref")
    rng = np.random.default_rng(42)
    w = warsaw_lines(rng, 600)
    t = tbednarski_lines(rng, 300)
    with tempfile.TemporaryDirectory() as tmp:
        out = {
            "warsaw_in": np.array(w), "tbednarski_in": np.array(t),
            "warsaw_all": run(SCANNER + ["--warsaw", "--s-z", "0", "--s-dl", "0"], w, tmp),
            "warsaw_only1": run(SCANNER + ["--warsaw", "--s-z", "0", "--s-dl", "0",
                                           "--only", "1"], w, tmp),
            "warsaw_smeared": run(SCANNER + ["--warsaw", "--s-z", "0.01", "--s-dl", "0.05",
                                             "--seed", "5"], w, tmp),
            "tbednarski": run(SCANNER + ["--tbednarski"], t, tmp),
            "tbednarski_rel": run(SCANNER + ["--tbednarski", "--relative-time"], t, tmp),
        }
    for k, v in out.items():
        print(k, v.shape)
    np.savez_compressed(os.path.join(HERE, "gate_small.npz"), **out)


if __name__ == "__main__":
    main()
