"""Coefficients of the 3D hybrid kernel's arctangent (atan2_pos in
j-pet-mlem-old_b200/csrc/hybrid_kernels.cu).

atan(t) on [0, 1] is approximated by the odd polynomial t * P(t^2), P of
degree 7 in s = t^2 (degree 15 in t), fitted toward the minimax absolute
error by Lawson's iteratively reweighted least squares (C. L. Lawson,
"Contributions to the theory of linear least maximum approximation", 1961):
weighted least squares on 20001 Chebyshev-spaced nodes, each weight
multiplied by that node's absolute error after every solve; the best
maximum error over 200 rounds is kept.  The coefficients are then rounded
to binary32, highest degree first, the order of the kernel's Horner chain.

    python tests/golden/fit_atan.py            # prints the coefficients
    python tests/golden/fit_atan.py --check    # compares them with the kernel

The fit is deterministic (numpy's least squares on fixed nodes), so the
kernel's constants are reproducible from this file.
"""
import os
import re
import sys

import numpy as np

N_TERMS = 8
N_NODES = 20001
ROUNDS = 200
KERNEL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "..",
                      "j-pet-mlem-old_b200", "csrc", "hybrid_kernels.cu")


def fit():
    """Returns (max abs error in binary64, binary32 coefficients of s^7 .. s^0)."""
    k = np.arange(N_NODES)
    t = 0.5 - 0.5 * np.cos(np.pi * k / (N_NODES - 1))
    f = np.arctan(t)
    V = np.stack([t ** (2 * j + 1) for j in range(N_TERMS)], axis=1)
    w = np.ones(N_NODES)
    best_err, best = None, None
    for _ in range(ROUNDS):
        sw = np.sqrt(w)
        c, *_ = np.linalg.lstsq(V * sw[:, None], f * sw, rcond=None)
        e = np.abs(V @ c - f)
        if best_err is None or e.max() < best_err:
            best_err, best = float(e.max()), c.copy()
        w = w * e
        w /= w.sum()
    return best_err, [np.float32(x) for x in best[::-1]]


def fma32(a, b, c):
    """Binary32 fused multiply-add (the product of two binary32 values is
    exact in binary64; the sum is rounded once more, to binary32)."""
    return np.float32(np.float64(a) * np.float64(b) + np.float64(c))


def eval32(coef, t):
    """The kernel's evaluation: Horner in s = t*t with binary32 FMAs, then t*p."""
    t = np.float32(t)
    s = np.float32(t * t)
    p = coef[0]
    for c in coef[1:]:
        p = fma32(p, s, c)
    return np.float32(t * p)


def kernel_coefficients(path=KERNEL):
    """The Horner chain's constants in atan2_pos, highest degree first."""
    src = open(path).read()
    body = src[src.index("float atan2_pos("):]
    body = body[:body.index("float r = t * p;")]
    return [np.float32(float(x)) for x in
            re.findall(r"p = (?:fmaf\(p, s, )?(-?[0-9.]+(?:e-?[0-9]+)?)f", body)]


def main():
    err, coef = fit()
    ts = np.linspace(0.0, 1.0, 200001, dtype=np.float32)
    e32 = max(abs(float(eval32(coef, x)) - np.arctan(np.float64(x))) for x in ts[::20])
    print(f"max |error|: {err:.3g} in binary64, {e32:.3g} evaluated in binary32")
    for c in coef:
        print(f"  {float(c)!r}f")
    if "--check" in sys.argv:
        have = kernel_coefficients()
        if [float(c) for c in have] != [float(c) for c in coef]:
            print("kernel coefficients differ:", [float(c) for c in have])
            return 1
        print("kernel coefficients match")
    return 0


if __name__ == "__main__":
    sys.exit(main())
