"""The float64 path-tracing oracle (oracle/pt64.c), checked on the CPU before
it checks the GPU adjoint.

* Its image equals the device path sampler compiled for the host
  (dort_gpu_host_check_render) on the same random numbers: the same paths,
  float against double rounding.
* Its gradient (forward mode per path term) equals central finite
  differences of its own image loss in double precision, with roulette off
  (a roulette decision that flips under a perturbation makes a sample jump;
  with it on, the gradient holds the decisions fixed).
"""
import numpy as np
import pytest

import dort_b200 as db
from dort_b200 import scenes
from oracle import pyoracle as po

W, H, SPP, DEPTH, SEED = 12, 10, 4, 6, 5


@pytest.fixture(scope="module")
def scene():
    return scenes.adjoint_scene(n_tris=400)


@pytest.mark.parametrize("roulette", [True, False])
def test_image_equals_the_host_compiled_sampler(scene, roulette):
    sd = scene
    n = len(sd["tris"])
    alb, em = sd["tri_albedo"], sd["tri_emission"]
    # per-triangle albedo as one material per triangle (the host check has no
    # per-triangle override)
    sd2 = dict(sd)
    sd2["materials"] = [{"kind": 0, "color": tuple(map(float, alb[k]))} for k in range(n)]
    sd2["tri_material"] = np.arange(n, dtype=np.uint32)
    p = db.render_params(sd["camera"], 20, 16, 8, max_depth=DEPTH, seed=SEED, roulette=roulette)
    host = db.host_check_render(sd2, p)
    img, _, _ = po.pt64(sd, 20, 16, 8, DEPTH, SEED, alb, em, no_roulette=not roulette)
    assert img.mean() > 0
    assert np.sqrt(((host - img) ** 2).mean()) / img.mean() < 1e-4


def _loss(sd, alb, em, target):
    img, _, _ = po.pt64(sd, W, H, SPP, DEPTH, SEED, alb, em, no_roulette=True)
    return float(((img - target) ** 2).sum()), img


def test_gradient_equals_finite_differences(scene):
    sd = scene
    alb0 = sd["tri_albedo"].astype(np.float64)
    em0 = sd["tri_emission"].astype(np.float64)
    rng = np.random.default_rng(2)
    target = rng.uniform(0.0, 0.3, (H, W, 3))
    loss, img = _loss(sd, alb0, em0, target)
    _, da, de = po.pt64(sd, W, H, SPP, DEPTH, SEED, alb0, em0, dl_dimage=2 * (img - target),
                        no_roulette=True)
    assert np.abs(da).sum() > 0 and np.abs(de).sum() > 0
    # directional derivatives (the oracle takes float32 parameters: steps of
    # 1e-3 keep the rounding of the perturbed values far below the change)
    va = rng.normal(size=alb0.shape) * (alb0 > 0)
    ve = np.zeros_like(em0)
    ve[sd["lights"]] = rng.normal(size=(len(sd["lights"]), 3))
    for v, g, h, which in ((va, da, 1e-3, "albedo"), (ve, de, 1e-2, "emission")):
        if which == "albedo":
            lp, _ = _loss(sd, (alb0 + h * v), em0, target)
            lm, _ = _loss(sd, (alb0 - h * v), em0, target)
        else:
            lp, _ = _loss(sd, alb0, em0 + h * v, target)
            lm, _ = _loss(sd, alb0, em0 - h * v, target)
        fd = (lp - lm) / (2 * h)
        an = float((g * v).sum())
        assert abs(an - fd) <= 1e-3 * abs(fd), (which, an, fd)
