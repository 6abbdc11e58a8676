"""The GGX conductor on the GPU (the material of a third of the 1080p
benchmark scene's patches), against the float64 oracle (oracle/microfacet.py,
whose GGX terms are pinned to the reference's MicrofacetDistrib in
tests/test_bsdf.py).

* Values: f and pdf at random direction pairs; sampled directions, values and
  pdfs from given uniforms.
* Distribution: 2^20 sampled directions per case binned over the hemisphere
  in (cos theta, phi); expected bin probabilities integrate the oracle's pdf
  on a fine grid; chi-square with sparse bins merged, p > 1e-4.
* Energy: with F0 = 1 the directional albedo E[f cos / pdf] is at most 1
  (the Smith term only removes energy) and equals the oracle's quadrature of
  f cos over the hemisphere.
"""
import numpy as np
import pytest

import dort_b200 as db
from oracle import microfacet as mf

pytestmark = pytest.mark.gpu

F0 = (0.95, 0.64, 0.54)


def unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def conductor(alpha, f0=F0):
    return {"kind": db.MAT_CONDUCTOR, "color": f0, "param": (alpha,)}


def wo_at(theta_deg):
    t = np.radians(theta_deg)
    return np.array([np.sin(t) * 0.6, np.sin(t) * 0.8, np.cos(t)])


@pytest.mark.parametrize("alpha", [0.05, 0.2, 0.5])
def test_device_conductor_matches_the_oracle(cuda, alpha):
    rng = np.random.default_rng(21)
    n = 1 << 16
    wo = unit(rng.normal(size=(n, 3)))
    wo[:, 2] = np.maximum(np.abs(wo[:, 2]), 0.05)
    wo = unit(wo).astype(np.float32)
    wi = unit(rng.normal(size=(n, 3)))
    wi[:, 2] = np.maximum(np.abs(wi[:, 2]), 0.05)
    wi = unit(wi).astype(np.float32)
    u = rng.uniform(1e-3, 1 - 1e-3, (n, 3)).astype(np.float32)
    got = db.bsdf_probe(conductor(alpha), wo, wi=wi, u=u)
    w64o, w64i = wo.astype(np.float64), wi.astype(np.float64)
    np.testing.assert_allclose(got["f"], mf.conductor_f(F0, alpha, w64i, w64o), rtol=2e-3,
                               atol=1e-6)
    np.testing.assert_allclose(got["pdf"], mf.conductor_pdf(alpha, w64i, w64o), rtol=2e-3,
                               atol=1e-6)
    swi, sf, spdf = mf.conductor_sample(F0, alpha, w64o, u[:, 0].astype(np.float64),
                                        u[:, 1].astype(np.float64))
    both = (spdf > 0) & (got["spdf"] > 0)
    assert np.mean((spdf > 0) != (got["spdf"] > 0)) < 1e-3
    np.testing.assert_allclose(got["wi"][both], swi[both], atol=5e-4)
    np.testing.assert_allclose(got["spdf"][both], spdf[both], rtol=5e-3)
    np.testing.assert_allclose(got["sf"][both], sf[both], rtol=5e-3, atol=1e-6)
    # the host-compiled code gives the same numbers
    host = db.bsdf_probe(conductor(alpha), wo[:4096], wi=wi[:4096], u=u[:4096], device=False)
    np.testing.assert_allclose(got["f"][:4096], host["f"], rtol=1e-4, atol=1e-7)
    np.testing.assert_allclose(got["wi"][:4096], host["wi"], atol=1e-5)


def _expected_bins(alpha, wo, n_cos, n_phi, sub=48):
    """Probability of each (cos theta, phi) bin of the upper hemisphere under
    the oracle pdf, by the midpoint rule on a grid `sub` times finer."""
    grid, dw = mf.hemisphere_grid(n_cos * sub, n_phi * sub)
    pdf = mf.conductor_pdf(alpha, grid.reshape(-1, 3), np.broadcast_to(wo, (grid.size // 3, 3)))
    pdf = pdf.reshape(n_cos, sub, n_phi, sub) * dw
    return pdf.sum(axis=(1, 3))


@pytest.mark.parametrize("alpha,theta", [(0.5, 10), (0.5, 60), (0.2, 30), (0.2, 75),
                                         (0.1, 45)])
def test_sampled_directions_follow_the_pdf(cuda, alpha, theta):
    from scipy import stats
    n = 1 << 20
    n_cos, n_phi = 16, 32
    wo = wo_at(theta)
    rng = np.random.default_rng(100 + theta)
    u = rng.uniform(size=(n, 3)).astype(np.float32)
    got = db.bsdf_probe(conductor(alpha), np.tile(wo.astype(np.float32), (n, 1)), u=u)
    valid = got["spdf"] > 0
    wi = got["wi"][valid].astype(np.float64)
    ci = np.minimum((wi[:, 2] * n_cos).astype(int), n_cos - 1)
    phi = np.mod(np.arctan2(wi[:, 1], wi[:, 0]), 2 * np.pi)
    pi_ = np.minimum((phi / (2 * np.pi) * n_phi).astype(int), n_phi - 1)
    obs = np.bincount(ci * n_phi + pi_, minlength=n_cos * n_phi).astype(np.float64)
    exp = _expected_bins(alpha, wo, n_cos, n_phi).reshape(-1) * n
    # the samples that leave the hemisphere are the probability the bins miss
    obs = np.append(obs, n - valid.sum())
    exp = np.append(exp, max(n - exp.sum(), 0.0))
    order = np.argsort(exp)
    # merge the sparsest bins until every merged bin expects at least 20
    o_m, e_m, acc_o, acc_e = [], [], 0.0, 0.0
    for k in order:
        acc_o += obs[k]
        acc_e += exp[k]
        if acc_e >= 20:
            o_m.append(acc_o)
            e_m.append(acc_e)
            acc_o = acc_e = 0.0
    if acc_e > 0:
        o_m[-1] += acc_o
        e_m[-1] += acc_e
    o_m, e_m = np.array(o_m), np.array(e_m)
    chi2 = float(((o_m - e_m) ** 2 / e_m).sum())
    p = stats.chi2.sf(chi2, len(o_m) - 1)
    assert len(o_m) > 10
    assert p > 1e-4, (chi2, len(o_m), p)


@pytest.mark.parametrize("alpha", [0.05, 0.2, 0.5])
@pytest.mark.parametrize("theta", [5, 45, 80])
def test_furnace_albedo(cuda, alpha, theta):
    n = 1 << 20
    wo = wo_at(theta)
    rng = np.random.default_rng(7 * theta + int(alpha * 100))
    u = rng.uniform(size=(n, 3)).astype(np.float32)
    got = db.bsdf_probe(conductor(alpha, (1.0, 1.0, 1.0)),
                        np.tile(wo.astype(np.float32), (n, 1)), u=u)
    ok = got["spdf"] > 0
    est = np.zeros(n)
    est[ok] = got["sf"][ok, 0] * np.abs(got["wi"][ok, 2]) / got["spdf"][ok]
    albedo = est.mean()
    err = est.std() / np.sqrt(n)
    assert albedo <= 1.0 + 4 * err
    quad = _albedo_quadrature(alpha, wo)
    assert abs(albedo - quad) < max(5 * err, 3e-3 * quad), (albedo, quad, err)


def _albedo_quadrature(alpha, wo, n_t=2048, n_p=512):
    """Integral of f cos over the hemisphere, taken over half vectors (where
    the peaked D lives near the pole of a theta-uniform grid): each upper-
    hemisphere wi is the reflection of wo about exactly one h with wo.h > 0,
    and d(omega_i) = 4 (wo.h) d(omega_h)."""
    t = (np.arange(n_t) + 0.5) / n_t * (np.pi / 2)
    p = (np.arange(n_p) + 0.5) / n_p * 2 * np.pi
    T, P = np.meshgrid(t, p, indexing="ij")
    h = np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], -1).reshape(-1, 3)
    dw_h = np.sin(T).reshape(-1) * (np.pi / 2 / n_t) * (2 * np.pi / n_p)
    d = h @ wo
    wi = 2 * d[:, None] * h - wo
    ok = (d > 0) & (wi[:, 2] > 0)
    f = mf.conductor_f((1.0, 1.0, 1.0), alpha, wi[ok], np.broadcast_to(wo, wi[ok].shape))[:, 0]
    return float((f * wi[ok, 2] * 4 * d[ok] * dw_h[ok]).sum())
