"""CPU checks of bench.py's measurement arithmetic.

The equal-RMSE figure compares a frame with a converged frame that still has
Monte Carlo noise of its own; bench.py subtracts that noise (estimated from
the spread of the converged frame's independent sub-frames).  Here the truth
is known: synthetic frames are a fixed image plus Gaussian noise of known
variance, and the corrected relative RMSE must recover the noise of the frame
under test, where the uncorrected one overestimates it.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _frames(truth, sigma, count, rng):
    return [truth + rng.normal(0.0, sigma, truth.shape) for _ in range(count)]


@pytest.mark.parametrize("ref_frames", [4, 16, 64])
def test_equal_rmse_subtracts_the_references_own_noise(ref_frames):
    rng = np.random.default_rng(3)
    truth = rng.uniform(0.5, 1.5, (96, 128, 3))
    sigma = 0.05                        # noise of one 256-spp frame
    subs = _frames(truth, sigma, ref_frames, rng)
    acc = np.sum(subs, axis=0)
    acc2 = np.sum([f * f for f in subs], axis=0)
    mean = acc / ref_frames
    var_frame = (acc2 / ref_frames - mean * mean) * ref_frames / (ref_frames - 1)
    x = truth + rng.normal(0.0, sigma, truth.shape)
    eq = bench.equal_rmse({"wavefront": x, "megakernel": x.copy()}, mean, var_frame / ref_frames,
                          ref_frames * 256, 256, {"wavefront": 2.0, "megakernel": 1.0})
    want = sigma / truth.mean()
    assert eq["rel_rmse_wavefront"] == pytest.approx(want, rel=0.03)
    assert eq["rel_rmse_wavefront_uncorrected"] > eq["rel_rmse_wavefront"]
    assert eq["reference_rel_rmse"] == pytest.approx(want / np.sqrt(ref_frames), rel=0.05)
    assert eq["rel_rmse_expected_from_spread"] == pytest.approx(want, rel=0.05)
    # 1/sqrt(spp): the spp that brings the error to 1 %
    assert eq["spp_for_1pct_wavefront"] == pytest.approx(256 * (want / 0.01) ** 2, rel=0.07)
    assert eq["equal_rmse_spp"] >= 256
    assert eq["wavefront_over_megakernel_at_equal_rmse"] == 2.0


def test_equal_rmse_halves_report_each_renderers_converged_half():
    rng = np.random.default_rng(5)
    truth = rng.uniform(0.5, 1.5, (64, 96, 3))
    sigma, k = 0.05, 32
    halves = {}
    for name, secs in (("wavefront", 10.0), ("megakernel", 25.0)):
        subs = _frames(truth, sigma, k, rng)
        mean = np.mean(subs, axis=0)
        var_frame = np.var(subs, axis=0, ddof=1)
        halves[name] = {"mean": mean, "var_mean": var_frame / k, "spp": k * 256,
                        "seconds": secs}
    ref = (halves["wavefront"]["mean"] + halves["megakernel"]["mean"]) / 2
    var_ref = (halves["wavefront"]["var_mean"] + halves["megakernel"]["var_mean"]) / 4
    x = truth + rng.normal(0.0, sigma, truth.shape)
    eq = bench.equal_rmse({"wavefront": x, "megakernel": x}, ref, var_ref, 2 * k * 256, 256,
                          {"wavefront": 2.0, "megakernel": 1.0}, halves, 64 * 96)
    at = eq["at_1pct"]
    want = sigma / truth.mean() / np.sqrt(k)
    assert at["wavefront"]["rel_rmse"] == pytest.approx(want, rel=0.05)
    assert at["megakernel"]["rel_rmse"] == pytest.approx(want, rel=0.05)
    assert at["rel_rmse_between"] == pytest.approx(at["rel_rmse_between_expected"], rel=0.05)
    assert at["wavefront_over_megakernel"] == 2.5
    assert at["wavefront"]["samples_per_s"] == pytest.approx(64 * 96 * k * 256 / 10.0)
    assert eq["rel_rmse_wavefront"] == pytest.approx(sigma / truth.mean(), rel=0.05)


def test_ref_procs_and_host_info():
    n = bench.ref_procs()
    assert 1 <= n <= (os.cpu_count() or 1)
    info = bench.host_info()
    assert info["host_cores"] == os.cpu_count()


def test_scene_input_bytes_counts_the_arrays():
    sd = {"verts": np.zeros((10, 3), np.float32), "tris": np.zeros((4, 3), np.uint32),
          "sky_rgb": np.zeros((2, 4, 3), np.float32), "camera": {}}
    assert bench.scene_input_bytes(sd) == 120 + 48 + 96
