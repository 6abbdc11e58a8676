"""Adjoint (path replay backpropagation) against central finite differences
and against the float64 CPU gradient.

The backward pass uses the forward pass's seed, so the gradient is that of
the loss of this estimator with its random numbers held fixed (common random
numbers).  Central differences of the same estimator along a random
direction v must then match <grad, v> within 2 %:
  * at max_depth 2, where no Russian roulette decision exists;
  * at the workload's depth 6 with roulette off (DORT_PT_NO_ROULETTE): a
    roulette decision depends on the albedo, so under a perturbation a
    decision can flip and its sample jump, which finite differences see and
    the gradient (decisions held fixed, unbiased in expectation) does not;
  * at the full workload size (500k triangles, 512 x 512, 64 spp, depth 6).
With roulette on, the gradient is checked statistically (seed averages).

The float64 CPU gradient (oracle/pt64.c: the same estimator on the same
random numbers, each path term differentiated directly) must equal the GPU's
path-replay gradient to 2 % in norm (with roulette on: the same decisions).
"""
import numpy as np
import pytest

import dort_b200 as db
from dort_b200 import scenes
from oracle import pyoracle as po

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


@pytest.mark.parametrize("roulette,depth", [(True, 6), (False, 6), (False, 14)])
def test_gradient_equals_the_float64_cpu_gradient(cuda, roulette, depth):
    """depth 14 without roulette: long paths record more terms than the
    per-sample log holds, and those samples take the two-pass replay."""
    w, spp = 24, 8
    sd = scenes.adjoint_scene(n_tris=2000)
    sc = db.scene_from_dict(sd)
    p = db.render_params(sd["camera"], w, w, spp, max_depth=depth, seed=13, roulette=roulette)
    alb, em = sd["tri_albedo"], sd["tri_emission"]
    rng = np.random.default_rng(4)
    target = rng.uniform(0.0, 0.3, (w, w, 3)).astype(np.float32)
    img = sc.adjoint_forward(p, alb, em)
    _, g = db.loss_l2(img, target)
    da, de = sc.adjoint_backward(p, g, alb, em)
    img64, da64, de64 = po.pt64(sd, w, w, spp, depth, 13, alb, em, dl_dimage=g,
                                no_roulette=not roulette)
    assert np.sqrt(((img - img64) ** 2).mean()) / img64.mean() < 1e-3
    for got, want in ((da, da64), (de, de64)):
        assert np.abs(want).sum() > 0
        err = np.linalg.norm(got.astype(np.float64) - want) / np.linalg.norm(want)
        assert err < 0.02, err
    # the light gradients one by one
    lights = sd["lights"]
    np.testing.assert_allclose(de[lights], de64[lights], rtol=0.02,
                               atol=0.02 * np.abs(de64[lights]).max())


@pytest.mark.parametrize("which", ["albedo", "emission"])
def test_directional_derivative_matches_fd_depth6_no_roulette(cuda, which):
    sd, sc, p = _setup(n_tris=20000, w=48, spp=16, depth=6)
    p = db.render_params(sd["camera"], 48, 48, 16, max_depth=6, seed=7, roulette=False)
    alb0, em0 = sd["tri_albedo"], sd["tri_emission"]
    rng = np.random.default_rng(8)
    alb_t = np.clip(alb0 * rng.uniform(0.7, 1.3, alb0.shape), 0, 1).astype(np.float32)
    target = sc.adjoint_forward(p, alb_t, em0)
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
        v[sd["lights"]] = rng.normal(size=(len(sd["lights"]), 3))
        h = 1e-1
        lp = _loss(sc, p, alb0, (em0 + h * v).astype(np.float32), target)[0]
        lm = _loss(sc, p, alb0, (em0 - h * v).astype(np.float32), target)[0]
        analytic = float((de.astype(np.float64) * v).sum())
    fd = (lp - lm) / (2 * h)
    assert abs(fd) > 0
    assert abs(analytic - fd) <= 0.02 * abs(fd), (analytic, fd)


def test_workload_size_fd_no_roulette(cuda):
    """The adjoint workload itself: 500k triangles, 512 x 512, 64 spp, depth 6."""
    sd = scenes.adjoint_scene()
    sc = db.scene_from_dict(sd)
    p = db.render_params(sd["camera"], 512, 512, 64, max_depth=6, seed=1, roulette=False)
    alb0, em0 = sd["tri_albedo"], sd["tri_emission"]
    rng = np.random.default_rng(9)
    target = sc.adjoint_forward(p, np.clip(alb0 * rng.uniform(0.8, 1.2, alb0.shape), 0, 1)
                                .astype(np.float32), em0)
    loss, g, img = _loss(sc, p, alb0, em0, target)
    da, de = sc.adjoint_backward(p, g, alb0, em0)
    assert np.isfinite(da).all() and np.isfinite(de).all()
    v = rng.normal(size=alb0.shape).astype(np.float32) * (alb0 > 0)
    h = 1e-2
    lp = _loss(sc, p, (alb0 + h * v).astype(np.float32), em0, target)[0]
    lm = _loss(sc, p, (alb0 - h * v).astype(np.float32), em0, target)[0]
    fd = (lp - lm) / (2 * h)
    analytic = float((da.astype(np.float64) * v).sum())
    assert abs(analytic - fd) <= 0.02 * abs(fd), (analytic, fd)
    ve = np.zeros_like(em0)
    ve[sd["lights"]] = rng.normal(size=(len(sd["lights"]), 3))
    h = 1e-1
    lp = _loss(sc, p, alb0, (em0 + h * ve).astype(np.float32), target)[0]
    lm = _loss(sc, p, alb0, (em0 - h * ve).astype(np.float32), target)[0]
    fd = (lp - lm) / (2 * h)
    analytic = float((de.astype(np.float64) * ve).sum())
    assert abs(analytic - fd) <= 0.02 * abs(fd), (analytic, fd)


def test_wavefront_renders_with_the_triangle_overrides(cuda):
    """The per-triangle albedo / emission set by the adjoint entry points
    belong to the scene: a wavefront frame rendered after them uses them
    (its cached graph is rebuilt), and after they are replaced, the new ones."""
    sd, sc, p = _setup(n_tris=2000, w=32, spp=16, depth=4)
    alb, em = sd["tri_albedo"], sd["tri_emission"]
    plain, _ = sc.render_wavefront(p)
    for k in (0.5, 0.25):
        a = (alb * k).astype(np.float32)
        img = sc.adjoint_forward(p, a, em)
        wf, _ = sc.render_wavefront(p)
        assert np.sqrt(((wf - img) ** 2).mean()) / img.mean() < 2e-3
        assert img.mean() < 0.9 * plain.mean()


@pytest.mark.parametrize("roulette", [True, False])
def test_wavefront_backward_equals_megakernel_backward(cuda, roulette):
    """The backward pass as a wavefront (per-slot term logs, applied by the
    regeneration stage) and as a megakernel trace the same paths: the same
    gradients to float rounding (atomics add in any order; a path that forks
    at a rounding difference between the two kernels is rare)."""
    sd, sc, p = _setup(n_tris=20000, w=48, spp=16, depth=6)
    pw = db.render_params(sd["camera"], 48, 48, 16, max_depth=6, seed=11, roulette=roulette)
    pm = db.render_params(sd["camera"], 48, 48, 16, max_depth=6, seed=11, roulette=roulette,
                          adjoint_megakernel=True)
    alb, em = sd["tri_albedo"], sd["tri_emission"]
    rng = np.random.default_rng(12)
    target = rng.uniform(0.0, 0.3, (48, 48, 3)).astype(np.float32)
    img = sc.adjoint_forward(pw, alb, em)
    _, g = db.loss_l2(img, target)
    wa, we = sc.adjoint_backward(pw, g, alb, em)
    st = sc.adjoint_stats()
    assert st["engine"] == "wavefront" and st["retraced"] == 0 and st["waves"] > 0
    ma, me = sc.adjoint_backward(pm, g, alb, em)
    assert sc.adjoint_stats()["engine"] == "megakernel"
    for got, want in ((wa, ma), (we, me)):
        assert np.abs(want).sum() > 0
        assert np.linalg.norm(got - want) <= 5e-3 * np.linalg.norm(want)


def _closed_box():
    """The Cornell box closed by a front wall, the camera inside it: without
    roulette every path runs to max_depth."""
    sd = scenes.cornell_box()
    P = np.array([[552.8, 0, 0], [0, 0, 0], [556, 548.8, 0], [0, 548.8, 0]], np.float32) * 0.01
    base = len(sd["verts"])
    sd["verts"] = np.concatenate([sd["verts"], P]).astype(np.float32)
    sd["tris"] = np.concatenate([sd["tris"], np.array([[base, base + 1, base + 3],
                                                       [base, base + 3, base + 2]],
                                                      np.uint32)]).astype(np.uint32)
    sd["tri_material"] = np.concatenate([sd["tri_material"],
                                         np.zeros(2, np.uint32)]).astype(np.uint32)
    sd["tri_emission"] = np.concatenate([sd["tri_emission"],
                                         np.zeros((2, 3), np.float32)]).astype(np.float32)
    sd["camera"] = scenes.look_at_camera((2.78, 2.73, 0.2), (2.78, 2.73, 5.0), (0.0, 1.0, 0.0),
                                         1.2)
    return sd


@pytest.mark.parametrize("list_cap,engine", [(None, "wavefront"), (100, "wavefront+megakernel")])
def test_wavefront_backward_log_overflow(cuda, list_cap, engine):
    """In a closed box without roulette every path reaches depth 14 and
    records more terms than a slot's log holds: those samples are traced
    again from a list, or, when they outnumber the list (capped here), the
    megakernel form runs for every sample.  Both give the megakernel's
    gradients."""
    sd = _closed_box()
    sc = db.scene_from_dict(sd)
    n = len(sd["tris"])
    rng = np.random.default_rng(6)
    alb = rng.uniform(0.3, 0.8, (n, 3)).astype(np.float32)
    em = sd["tri_emission"]
    args = dict(max_depth=14, seed=5, roulette=False)
    pw = db.render_params(sd["camera"], 32, 32, 4, **args)
    pm = db.render_params(sd["camera"], 32, 32, 4, adjoint_megakernel=True, **args)
    img = sc.adjoint_forward(pw, alb, em)
    _, g = db.loss_l2(img, np.zeros_like(img))
    if list_cap is not None:
        db.debug_adjoint_list(list_cap)
    try:
        wa, we = sc.adjoint_backward(pw, g, alb, em)
    finally:
        db.debug_adjoint_list(-1)
    st = sc.adjoint_stats()
    assert st["engine"] == engine, st
    assert st["retraced"] > 0.9 * 32 * 32 * 4, st
    ma, me = sc.adjoint_backward(pm, g, alb, em)
    for got, want in ((wa, ma), (we, me)):
        assert np.abs(want).sum() > 0
        assert np.linalg.norm(got - want) <= 5e-3 * np.linalg.norm(want)


def test_forward_is_deterministic_and_equals_megakernel_forward(cuda):
    """The forward pass renders the path tracer as a wavefront with
    deterministic sums: repeated calls give the same bits (finite
    differences of the loss rely on it), and the megakernel form
    (DORT_ADJOINT_MEGAKERNEL) the same image up to rounding."""
    sd, sc, p = _setup(n_tris=20000, w=40, spp=12, depth=6)
    alb, em = sd["tri_albedo"], sd["tri_emission"]
    a = sc.adjoint_forward(p, alb, em)
    b = sc.adjoint_forward(p, alb, em)
    assert np.array_equal(a, b)
    pm = db.render_params(sd["camera"], 40, 40, 12, max_depth=2, seed=7, adjoint_megakernel=True)
    m = sc.adjoint_forward(pm, alb, em)
    pw = db.render_params(sd["camera"], 40, 40, 12, max_depth=2, seed=7)
    w = sc.adjoint_forward(pw, alb, em)
    assert np.sqrt(((w - m) ** 2).mean()) / m.mean() < 1e-3
