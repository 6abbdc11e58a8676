"""The GGX distribution and the GGX conductor, checked on the CPU.

* The oracle's float64 restatement of GGX D, G1 and the half-vector sampler
  (oracle/microfacet.py) is pinned against the reference's own
  MicrofacetDistrib (src/dort/microfacet.cpp:19-86) compiled from its sources
  into oracle/_ref: equal to float rounding.
* The BxDF code the renderers run (pt.cuh), compiled for the host and reached
  through dort_gpu_bsdf_probe, against that oracle: the conductor's value,
  pdf and sampled directions, and Lambert as a control.  The same checks on
  the GPU, plus the sampling distribution and the energy bound, are in
  tests/test_bsdf_gpu.py.
"""
import numpy as np
import pytest

import dort_b200 as db
from oracle import microfacet as mf
from oracle import pyoracle as po

ALPHAS = (0.05, 0.2, 0.5)
F0 = (0.95, 0.64, 0.54)


def unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def upper_dirs(rng, n, min_z=0.02):
    v = unit(rng.normal(size=(n, 3)))
    v[:, 2] = np.maximum(np.abs(v[:, 2]), min_z)
    return unit(v).astype(np.float32)


def conductor(alpha):
    return {"kind": db.MAT_CONDUCTOR, "color": F0, "param": (alpha,)}


needs_ref = pytest.mark.skipif(not po.ref_available(), reason="compiled reference not built")


@needs_ref
@pytest.mark.parametrize("alpha", ALPHAS)
def test_oracle_ggx_matches_the_reference(alpha):
    rng = np.random.default_rng(7)
    uv = rng.uniform(1e-3, 1 - 1e-3, (4096, 2)).astype(np.float32)
    m_ref, pdf_ref = po.ref_ggx_sample_m(alpha, uv)
    m, pdf = mf.ggx_sample_m(uv[:, 0].astype(np.float64), uv[:, 1].astype(np.float64), alpha)
    np.testing.assert_allclose(m, m_ref, atol=1e-4)
    np.testing.assert_allclose(pdf, pdf_ref, rtol=1e-3)
    mm = m_ref.astype(np.float64)
    np.testing.assert_allclose(mf.ggx_d(mm, alpha), po.ref_ggx_d(alpha, m_ref), rtol=1e-3)
    v = upper_dirs(rng, 4096)
    np.testing.assert_allclose(mf.ggx_g1(v.astype(np.float64), mm, alpha),
                               po.ref_ggx_g1(alpha, v, m_ref), atol=1e-5)
    # G1 is zero where v sees the back of the microfacet (v.m and v.z of
    # opposite signs)
    va = unit(rng.normal(size=(4096, 3))).astype(np.float32)
    back = np.sum(va * m_ref, axis=1) * va[:, 2] <= 0
    assert back.sum() > 50
    assert np.all(po.ref_ggx_g1(alpha, va, m_ref)[back] == 0.0)
    assert np.all(mf.ggx_g1(va.astype(np.float64), mm, alpha)[back] == 0.0)


@pytest.mark.parametrize("alpha", ALPHAS)
def test_host_conductor_values_match_the_oracle(alpha):
    rng = np.random.default_rng(11)
    wo = upper_dirs(rng, 4096, 0.05)
    wi = upper_dirs(rng, 4096, 0.05)
    got = db.bsdf_probe(conductor(alpha), wo, wi=wi, device=False)
    f = mf.conductor_f(F0, alpha, wi.astype(np.float64), wo.astype(np.float64))
    pdf = mf.conductor_pdf(alpha, wi.astype(np.float64), wo.astype(np.float64))
    np.testing.assert_allclose(got["f"], f, rtol=2e-3, atol=1e-6)
    np.testing.assert_allclose(got["pdf"], pdf, rtol=2e-3, atol=1e-6)
    # opposite sides: nothing
    got = db.bsdf_probe(conductor(alpha), wo, wi=-wi, device=False)
    assert np.all(got["f"] == 0.0) and np.all(got["pdf"] == 0.0)


@pytest.mark.parametrize("alpha", ALPHAS)
def test_host_conductor_sampling_matches_the_oracle(alpha):
    rng = np.random.default_rng(13)
    n = 4096
    wo = upper_dirs(rng, n, 0.05)
    wo[: n // 2, 2] *= -1.0                      # both sides of the surface
    u = rng.uniform(1e-3, 1 - 1e-3, (n, 3)).astype(np.float32)
    got = db.bsdf_probe(conductor(alpha), wo, u=u, device=False)
    wi, f, pdf = mf.conductor_sample(F0, alpha, wo.astype(np.float64),
                                     u[:, 0].astype(np.float64), u[:, 1].astype(np.float64))
    ok = pdf > 0
    assert np.array_equal(got["spdf"] > 0, ok) or np.mean((got["spdf"] > 0) != ok) < 1e-3
    both = ok & (got["spdf"] > 0)
    np.testing.assert_allclose(got["wi"][both], wi[both], atol=5e-4)
    np.testing.assert_allclose(got["spdf"][both], pdf[both], rtol=5e-3)
    np.testing.assert_allclose(got["sf"][both], f[both], rtol=5e-3, atol=1e-6)
    # sampled directions stay on wo's side; the pdf of the sample is the
    # pdf of evaluating it
    assert np.all(got["wi"][both, 2] * wo[both, 2] > 0)
    ev = db.bsdf_probe(conductor(alpha), wo[both], wi=got["wi"][both], device=False)
    np.testing.assert_allclose(ev["pdf"], got["spdf"][both], rtol=2e-3)


def test_host_lambert_matches_cosine_sampling():
    rng = np.random.default_rng(5)
    n = 2048
    wo = upper_dirs(rng, n)
    wi = upper_dirs(rng, n)
    u = rng.uniform(size=(n, 3)).astype(np.float32)
    lam = {"kind": db.MAT_LAMBERT, "color": (0.5, 0.25, 0.75)}
    got = db.bsdf_probe(lam, wo, wi=wi, u=u, device=False)
    np.testing.assert_allclose(got["f"], np.tile([0.5, 0.25, 0.75], (n, 1)) / np.pi, rtol=1e-6)
    np.testing.assert_allclose(got["pdf"], wi[:, 2] / np.pi, rtol=1e-5)
    np.testing.assert_allclose(got["spdf"], got["wi"][:, 2] / np.pi, rtol=1e-4)
