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


def forked_pixels(x, ref, tol=1e-4):
    """Pixels of two renders of the same paths (same random numbers) that
    differ by more than tol x the reference's mean.  Two kernels compile
    the same arithmetic with different fused multiply-adds, so a path that
    grazes an edge or a critical angle can take another branch in one of
    them; every other pixel agrees to float rounding."""
    d = np.abs(np.asarray(x, np.float64) - ref).max(axis=-1)
    return int((d > tol * float(np.mean(ref))).sum())


def compare_blocks(A0, A1, B0, B1):
    """compare() on images already reduced to block means."""
    A0, A1, B0, B1 = (np.asarray(x, np.float64) for x in (A0, A1, B0, B1))
    A, B = (A0 + A1) / 2, (B0 + B1) / 2
    num = ((A - B) ** 2).sum(axis=(0, 1))
    den = (((A0 - A1) ** 2 + (B0 - B1) ** 2) / 4).sum(axis=(0, 1))
    X = num / np.maximum(den, 1e-30)
    mean_rel = (A.mean(axis=(0, 1)) - B.mean(axis=(0, 1))) / np.maximum(B.mean(axis=(0, 1)), 1e-30)
    # per block: squared difference over its own noise estimate (channels
    # summed); without bias its distribution is F-like with median ~1, and a
    # few caustic or firefly blocks cannot move the median
    nb = ((A - B) ** 2).sum(axis=-1)
    db = (((A0 - A1) ** 2 + (B0 - B1) ** 2) / 4).sum(axis=-1)
    noisy = db > 1e-12 * max(float(db.max()), 1e-30)
    Xmed = float(np.median(nb[noisy] / db[noisy])) if noisy.any() else 0.0
    # difference of the channel means over its standard error (blocks are
    # independent; each block's variance estimated from the halves)
    nblk = A.shape[0] * A.shape[1]
    se = np.sqrt((((A0 - A1) ** 2 + (B0 - B1) ** 2) / 4).sum(axis=(0, 1))) / nblk
    mean_z = (A.mean(axis=(0, 1)) - B.mean(axis=(0, 1))) / np.maximum(se, 1e-30)
    return {"X": X, "mean_rel": mean_rel, "Xmed": Xmed, "mean_z": mean_z}


def compare_single(A0, A1, B, b_var_ratio):
    """compare_blocks() against one image B instead of two halves, for a
    reference whose renders cannot be made independent: B's noise is taken as
    b_var_ratio times the noise of the mean of A0 and A1 (the ratio of their
    sample counts when both come from the same estimator)."""
    A0, A1, B = (np.asarray(x, np.float64) for x in (A0, A1, B))
    A = (A0 + A1) / 2
    va = (A0 - A1) ** 2 / 4                      # noise of A, per block and channel
    v = va * (1.0 + b_var_ratio)                 # noise of A - B
    num = ((A - B) ** 2).sum(axis=(0, 1))
    X = num / np.maximum(v.sum(axis=(0, 1)), 1e-30)
    mean_rel = (A.mean(axis=(0, 1)) - B.mean(axis=(0, 1))) / np.maximum(B.mean(axis=(0, 1)), 1e-30)
    nb = ((A - B) ** 2).sum(axis=-1)
    db = v.sum(axis=-1)
    noisy = db > 1e-12 * max(float(db.max()), 1e-30)
    Xmed = float(np.median(nb[noisy] / db[noisy])) if noisy.any() else 0.0
    nblk = A.shape[0] * A.shape[1]
    se = np.sqrt(v.sum(axis=(0, 1))) / nblk
    mean_z = (A.mean(axis=(0, 1)) - B.mean(axis=(0, 1))) / np.maximum(se, 1e-30)
    return {"X": X, "mean_rel": mean_rel, "Xmed": Xmed, "mean_z": mean_z}


def block_means(img, block=16):
    """Mean RGB of block x block pixel blocks; the last row / column of blocks
    is ragged when the size does not divide the image."""
    img = np.asarray(img, np.float64)
    h, w = img.shape[:2]
    by, bx = (h + block - 1) // block, (w + block - 1) // block
    out = np.zeros((by, bx, img.shape[2]), np.float64)
    for j in range(by):
        for i in range(bx):
            out[j, i] = img[j * block:(j + 1) * block, i * block:(i + 1) * block].reshape(
                -1, img.shape[2]).mean(0)
    return out


def normal_cdf_inverse(p: float) -> float:
    """Abramowitz & Stegun 26.2.23, as the reference's math.cpp:4-19 uses."""
    def approx(t):
        c0, c1, c2 = 2.515517, 0.802853, 0.010328
        d0, d1, d2 = 1.432788, 0.189269, 0.001308
        return t - ((c2 * t + c1) * t + c0) / (((d2 * t + d1) * t + d0) * t + 1.0)
    if p < 0.5:
        return -approx(np.sqrt(-2.0 * np.log(p)))
    return approx(np.sqrt(-2.0 * np.log(1.0 - p)))


def convergence_tiles(w: int, h: int, min_tile_size: int = 32) -> np.ndarray:
    """Tiles test_convergence checks (convergence_test.cpp:31-35,69-83): the
    image, then tiles of size min(w, h) >> depth down to min_tile_size."""
    max_depth = 0
    while (min(w, h) >> (max_depth + 1)) >= min_tile_size:
        max_depth += 1
    tiles = []
    for depth in range(max_depth + 1):
        size = min(w, h) >> depth
        for ty in range((h + size - 1) // size):
            for tx in range((w + size - 1) // size):
                tiles.append((tx * size, ty * size, min((tx + 1) * size, w),
                              min((ty + 1) * size, h)))
    return np.asarray(tiles, np.int32)


def tile_means(img, tiles):
    img = np.asarray(img, np.float64)
    return np.asarray([img[y0:y1, x0:x1].reshape(-1, 3).mean(0) for x0, y0, x1, y1 in tiles])


def reference_convergence(ref_tmeans, tiles, tested, variation=8.0, bias=0.0, p_value=0.01,
                          min_tile_size=32):
    """The reference's own image test, test_convergence
    (src/dort/convergence_test.cpp:10-101), from the reference image's tile
    means.  Returns the largest |mean_diff| / threshold over all tiles (the
    test passes when it is <= 1) and the first failing tile (or None)."""
    h, w = tested.shape[:2]
    max_depth = 0
    while (min(w, h) >> (max_depth + 1)) >= min_tile_size:
        max_depth += 1
    test_count = float(((1 << (2 * max_depth + 2)) - 1) // 3)
    test_p = 1.0 - (1.0 - p_value) ** (1.0 / test_count)
    inv_phi = normal_cdf_inverse(test_p * 0.5)
    ref_mean = np.asarray(ref_tmeans[0], np.float64)     # tile 0 is the whole image
    ours = tile_means(tested, tiles)
    worst, first_fail = 0.0, None
    for k, (x0, y0, x1, y1) in enumerate(tiles):
        tref = np.asarray(ref_tmeans[k], np.float64)
        mean_diff = (ours[k] - tref).max()
        stddev = max((ref_mean * variation).max(), (tref * variation).max())
        b = min((ref_mean * bias).max(), (tref * bias).max())
        count = float(x1 - x0) * float(y1 - y0)
        max_diff = -stddev / np.sqrt(count) * inv_phi + b
        r = abs(mean_diff) / max(max_diff, 1e-30)
        worst = max(worst, r)
        if r > 1.0 and first_fail is None:
            first_fail = (int(x0), int(y0), int(x1), int(y1), float(mean_diff), float(max_diff))
    return worst, first_fail
