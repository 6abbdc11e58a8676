"""Statistical image comparison for the path-tracer parity tests.

Renders are Monte Carlo estimates, and this build's random numbers differ
from the reference's mt19937 streams, so images can only agree in
expectation.  Each side provides two independent halves (different seeds).
Over B x B pixel blocks and each channel:

    X = sum_R (A_R - B_R)^2 / sum_R ((a0_R - a1_R)^2 + (b0_R - b1_R)^2) / 4

where A = (a0 + a1) / 2.  If both renders have the same expectation the
numerator and denominator have the same mean, so X is close to 1; a bias
between the renderers makes X grow with the sample count.  The relative RMSE
of the block means is reported alongside.
"""
from __future__ import annotations

import numpy as np


def blocks(img, b):
    h, w, c = img.shape
    h2, w2 = h // b * b, w // b * b
    return img[:h2, :w2].reshape(h2 // b, b, w2 // b, b, c).mean(axis=(1, 3))


def compare(a0, a1, b0, b1, block=8):
    A0, A1, B0, B1 = (blocks(np.asarray(x, np.float64), block) for x in (a0, a1, b0, b1))
    A, B = (A0 + A1) / 2, (B0 + B1) / 2
    num = ((A - B) ** 2).sum(axis=(0, 1))
    den = (((A0 - A1) ** 2 + (B0 - B1) ** 2) / 4).sum(axis=(0, 1))
    X = num / np.maximum(den, 1e-30)
    rel_rmse = np.sqrt(((A - B) ** 2).mean()) / max(B.mean(), 1e-30)
    mean_rel = (A.mean(axis=(0, 1)) - B.mean(axis=(0, 1))) / np.maximum(B.mean(axis=(0, 1)), 1e-30)
    return {"X": X, "rel_rmse_blocks": float(rel_rmse), "mean_rel": mean_rel}


def rel_rmse(x, ref):
    x, ref = np.asarray(x, np.float64), np.asarray(ref, np.float64)
    return float(np.sqrt(((x - ref) ** 2).mean()) / ref.mean())
