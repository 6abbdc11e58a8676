"""Float64 restatement of the GGX microfacet distribution and of the GGX
conductor built on it.

TEST INFRASTRUCTURE ONLY: the checker for the device BxDF code (through the
dort_gpu_bsdf_probe diagnostic), never imported by the product package.

* GGX D, Smith G1 and the half-vector sampler restate the reference's
  MicrofacetDistrib of type GGX (src/dort/microfacet.cpp:19-36, 38-58,
  64-86); tests pin this restatement against the reference's own float code
  compiled into oracle/_ref (pyoracle.ref_ggx_*).
* The conductor has no reference counterpart (the reference has no GGX
  conductor; its Tungsten importer maps one elsewhere, lua/tungsten.lua:
  119-124).  It is the microfacet reflection model of Walter, Marschner, Li
  and Torrance, "Microfacet Models for Refraction through Rough Surfaces"
  (EGSR 2007): f = F(wi.h) D(h) G1(wi, h) G1(wo, h) / (4 |cos wi| |cos wo|)
  with h the normalised half vector (their eq. 20), Schlick's Fresnel
  approximation F = F0 + (1 - F0)(1 - |cos|)^5 (Schlick, "An Inexpensive BRDF
  Model for Physically-based Rendering", 1994), half vectors sampled from
  D(h) cos(h) and mirrored to the side of wo, so the direction pdf is
  D(h) |cos h| / (4 |wo.h|) (their eq. 14 and the reflection Jacobian,
  eq. 13).

Directions are arrays of shape (..., 3) in the local shading frame (z = the
normal).
"""
from __future__ import annotations

import numpy as np

INV_PI = 1.0 / np.pi


def _dot(a, b):
    return np.sum(np.asarray(a, np.float64) * np.asarray(b, np.float64), axis=-1)


def ggx_d(m, alpha):
    """D(m) (microfacet.cpp:19-36, GGX branch): 1 / (pi a^2 cos^4 (1 + tan^2/a^2)^2)
    written as INV_PI a^2 / (cos^2 (a^2 + tan^2))^2."""
    m = np.asarray(m, np.float64)
    c2 = m[..., 2] ** 2
    with np.errstate(divide="ignore", invalid="ignore"):
        t2 = (1.0 - c2) / c2
        return INV_PI * alpha ** 2 / (c2 * (alpha ** 2 + t2)) ** 2


def ggx_g1(v, m, alpha):
    """Smith G1(v, m) (microfacet.cpp:38-58): 0 when v and m lie on opposite
    sides of the surface as seen from v, else 2 / (1 + sqrt(1 + a^2 tan^2 v))."""
    v = np.asarray(v, np.float64)
    c2 = v[..., 2] ** 2
    with np.errstate(divide="ignore", invalid="ignore"):
        t2 = (1.0 - c2) / c2
        g = 2.0 / (1.0 + np.sqrt(1.0 + alpha ** 2 * t2))
    return np.where(_dot(v, m) * v[..., 2] <= 0.0, 0.0, g)


def ggx_sample_m(u1, u2, alpha):
    """Half vector from two uniforms and its pdf D(m) cos(m)
    (microfacet.cpp:64-86): cos theta = 1 / sqrt(a^2 u1 / (1 - u1) + 1),
    phi = 2 pi u2, m = (sin t sin p, sin t cos p, cos t)."""
    u1 = np.asarray(u1, np.float64)
    u2 = np.asarray(u2, np.float64)
    ct = 1.0 / np.sqrt(alpha ** 2 * u1 / (1.0 - u1) + 1.0)
    st = np.sqrt(np.maximum(0.0, 1.0 - ct * ct))
    phi = 2.0 * np.pi * u2
    m = np.stack([st * np.sin(phi), st * np.cos(phi), ct], axis=-1)
    return m, ggx_d(m, alpha) * ct


def schlick(f0, cos_i):
    """Schlick's Fresnel for a conductor tinted f0 (RGB)."""
    x = 1.0 - np.minimum(np.abs(np.asarray(cos_i, np.float64)), 1.0)
    k = x ** 5
    f0 = np.asarray(f0, np.float64)
    return f0 + (1.0 - f0) * k[..., None]


def _half(wi, wo):
    h = np.asarray(wi, np.float64) + np.asarray(wo, np.float64)
    n = np.linalg.norm(h, axis=-1, keepdims=True)
    with np.errstate(divide="ignore", invalid="ignore"):
        h = h / n
    h = np.where(h[..., 2:3] < 0.0, -h, h)
    return h, n[..., 0] > 0.0


def conductor_f(f0, alpha, wi, wo):
    """The conductor's BRDF value (RGB), zero unless wi and wo lie on the same
    side of the surface."""
    wi = np.asarray(wi, np.float64)
    wo = np.asarray(wo, np.float64)
    h, ok = _half(wi, wo)
    same = wi[..., 2] * wo[..., 2] > 0.0
    with np.errstate(divide="ignore", invalid="ignore"):
        s = ggx_d(h, alpha) * ggx_g1(wi, h, alpha) * ggx_g1(wo, h, alpha) / (
            4.0 * np.abs(wi[..., 2]) * np.abs(wo[..., 2]))
    s = np.where(same & ok, s, 0.0)
    return schlick(f0, _dot(wi, h)) * s[..., None]


def conductor_pdf(alpha, wi, wo):
    """Density of sampling wi given wo: D(h) |cos h| / (4 |wo.h|)."""
    wi = np.asarray(wi, np.float64)
    wo = np.asarray(wo, np.float64)
    h, ok = _half(wi, wo)
    same = wi[..., 2] * wo[..., 2] > 0.0
    dwo = np.abs(_dot(wo, h))
    with np.errstate(divide="ignore", invalid="ignore"):
        p = ggx_d(h, alpha) * np.abs(h[..., 2]) / (4.0 * dwo)
    return np.where(same & ok & (dwo > 0.0), p, 0.0)


def conductor_sample(f0, alpha, wo, u1, u2):
    """Sampled direction (half vector mirrored to wo's side, wo reflected
    about it), its BRDF value and pdf; pdf = 0 where the reflection leaves
    wo's side of the surface."""
    wo = np.asarray(wo, np.float64)
    h, pm = ggx_sample_m(u1, u2, alpha)
    h = np.where(wo[..., 2:3] < 0.0, h * np.array([1.0, 1.0, -1.0]), h)
    d = _dot(wo, h)
    wi = 2.0 * d[..., None] * h - wo
    valid = (wi[..., 2] * wo[..., 2] > 0.0) & (d != 0.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        pdf = np.where(valid, pm / (4.0 * np.abs(d)), 0.0)
    f = np.where(valid[..., None], conductor_f(f0, alpha, wi, wo), 0.0)
    return wi, f, pdf


def hemisphere_grid(n_cos: int, n_phi: int, upper: bool = True):
    """Midpoints of an (cos theta, phi) grid over a hemisphere and the solid
    angle of each cell (dcos * dphi)."""
    c = (np.arange(n_cos) + 0.5) / n_cos
    p = (np.arange(n_phi) + 0.5) / n_phi * 2.0 * np.pi
    C, P = np.meshgrid(c, p, indexing="ij")
    s = np.sqrt(1.0 - C * C)
    w = np.stack([s * np.cos(P), s * np.sin(P), C if upper else -C], axis=-1)
    return w, (1.0 / n_cos) * (2.0 * np.pi / n_phi)
