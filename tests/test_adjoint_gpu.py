"""Adjoint (path replay backpropagation) against central finite differences.

The backward pass uses the forward pass's seed, so the gradient is that of
the loss of this estimator with its random numbers held fixed (common random
numbers).  Central differences of the same estimator along a random
direction v must then match <grad, v>.  With max_depth <= 2 no Russian
roulette decision exists and the only difference is float rounding: the bar
is 2 % relative.  At the workload's depth 6, roulette probabilities depend on
the albedo and are held fixed by the adjoint (unbiased in expectation); the
bar there is statistical.
"""
import numpy as np
import pytest

import dort_b200 as db
from dort_b200 import scenes

pytestmark = pytest.mark.gpu


def _setup(n_tris=20000, w=64, spp=16, depth=2, seed=7):
    sd = scenes.adjoint_scene(n_tris=n_tris)
    sc = db.scene_from_dict(sd)
    p = db.render_params(sd["camera"], w, w, spp, max_depth=depth, seed=seed)
    return sd, sc, p


def _loss(sc, p, alb, em, target):
    img = sc.adjoint_forward(p, alb, em)
    loss, g = db.loss_l2(img, target)
    return loss, g, img


@pytest.mark.parametrize("which", ["albedo", "emission"])
def test_directional_derivative_matches_fd_depth2(cuda, which):
    sd, sc, p = _setup()
    alb0, em0 = sd["tri_albedo"], sd["tri_emission"]
    rng = np.random.default_rng(3)
    # target: the same scene with perturbed albedo / emission
    alb_t = np.clip(alb0 * rng.uniform(0.7, 1.3, alb0.shape), 0, 1).astype(np.float32)
    em_t = (em0 * rng.uniform(0.7, 1.3, em0.shape)).astype(np.float32)
    target = sc.adjoint_forward(p, alb_t, em_t)
    loss, g, img = _loss(sc, p, alb0, em0, target)
    da, de = sc.adjoint_backward(p, g, alb0, em0)
    if which == "albedo":
        v = rng.normal(size=alb0.shape).astype(np.float32) * (alb0 > 0)
        h = 1e-2
        lp = _loss(sc, p, (alb0 + h * v).astype(np.float32), em0, target)[0]
        lm = _loss(sc, p, (alb0 - h * v).astype(np.float32), em0, target)[0]
        analytic = float((da.astype(np.float64) * v).sum())
    else:
        v = np.zeros_like(em0)
        lights = sd["lights"]
        v[lights] = rng.normal(size=(len(lights), 3))
        h = 1e-1
        lp = _loss(sc, p, alb0, (em0 + h * v).astype(np.float32), target)[0]
        lm = _loss(sc, p, alb0, (em0 - h * v).astype(np.float32), target)[0]
        analytic = float((de.astype(np.float64) * v).sum())
    fd = (lp - lm) / (2 * h)
    assert abs(fd) > 0
    assert abs(analytic - fd) <= 0.02 * abs(fd), (analytic, fd)


def test_gradient_is_linear_in_image_adjoint(cuda):
    sd, sc, p = _setup(n_tris=5000, w=32, spp=8)
    rng = np.random.default_rng(1)
    g1 = rng.normal(size=(32, 32, 3)).astype(np.float32)
    g2 = rng.normal(size=(32, 32, 3)).astype(np.float32)
    a1, e1 = sc.adjoint_backward(p, g1, sd["tri_albedo"], sd["tri_emission"])
    a2, e2 = sc.adjoint_backward(p, g2, sd["tri_albedo"], sd["tri_emission"])
    a3, e3 = sc.adjoint_backward(p, g1 + 2 * g2, sd["tri_albedo"], sd["tri_emission"])
    np.testing.assert_allclose(a3, a1 + 2 * a2, rtol=1e-3, atol=1e-6)
    np.testing.assert_allclose(e3, e1 + 2 * e2, rtol=1e-3, atol=1e-4)


def test_emission_gradient_of_mean_pixel(cuda):
    """With dLoss/dI = 1 everywhere the emission gradient is the derivative of
    the image sum, which is linear in the emission: sum(dI/dLe * Le) equals
    the image sum (every path term is proportional to exactly one Le)."""
    sd, sc, p = _setup(n_tris=5000, w=32, spp=8, depth=4)
    img = sc.adjoint_forward(p, sd["tri_albedo"], sd["tri_emission"])
    ones = np.ones_like(img)
    _, de = sc.adjoint_backward(p, ones, sd["tri_albedo"], sd["tri_emission"])
    total = float((de.astype(np.float64) * sd["tri_emission"]).sum())
    assert abs(total - float(img.sum(dtype=np.float64))) <= 1e-3 * float(img.sum())


def test_depth6_statistical(cuda):
    sd, sc, p0 = _setup(n_tris=20000, w=48, spp=64, depth=6)
    alb0, em0 = sd["tri_albedo"], sd["tri_emission"]
    rng = np.random.default_rng(5)
    target = sc.adjoint_forward(p0, np.clip(alb0 * 1.2, 0, 1).astype(np.float32), em0)
    v = rng.normal(size=alb0.shape).astype(np.float32) * (alb0 > 0)
    h = 2e-2
    fds, ans = [], []
    for seed in range(4):
        p = db.render_params(sd["camera"], 48, 48, 64, max_depth=6, seed=100 + seed)
        loss, g, img = _loss(sc, p, alb0, em0, target)
        da, _ = sc.adjoint_backward(p, g, alb0, em0, want_emission=False)
        ans.append(float((da.astype(np.float64) * v).sum()))
        lp = _loss(sc, p, (alb0 + h * v).astype(np.float32), em0, target)[0]
        lm = _loss(sc, p, (alb0 - h * v).astype(np.float32), em0, target)[0]
        fds.append((lp - lm) / (2 * h))
    fd, an = np.mean(fds), np.mean(ans)
    assert abs(an - fd) <= 0.1 * abs(fd), (ans, fds)


def test_l2_loss(cuda):
    rng = np.random.default_rng(0)
    a = rng.random((17, 13, 3)).astype(np.float32)
    b = rng.random((17, 13, 3)).astype(np.float32)
    loss, g = db.loss_l2(a, b)
    np.testing.assert_allclose(loss, ((a.astype(np.float64) - b) ** 2).sum(), rtol=1e-6)
    np.testing.assert_allclose(g, 2 * (a - b), rtol=1e-6)
