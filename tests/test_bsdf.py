"""Analytic checks of the physical estimator's BSDFs: Lambert, GGX with visible-normal
sampling (Heitz 2018) and the smooth dielectric, evaluated in double precision by
the oracle's restatement -- the same formulas the GPU kernels evaluate, tied to
them by the GPU parity tests. The reference has none of these materials, so these
known-answer properties pin them: sampling densities that integrate to the kept
fraction, sampling weights equal to f cos / pdf, reciprocity, energy bounds
(white furnace), the law of reflection, Snell's law and Fresnel reflectance.
CPU only.
"""
import numpy as np
import pytest

import oracle

N = np.array([0.0, 0.0, 1.0])


def wo_at(deg):
    t = np.radians(deg)
    return np.array([np.sin(t), 0.0, np.cos(t)])


def hemisphere_grid(n_theta, n_phi):
    """Midpoint rule over the upper hemisphere: directions and their solid angles."""
    th = (np.arange(n_theta) + 0.5) * (np.pi / 2) / n_theta
    ph = (np.arange(n_phi) + 0.5) * 2 * np.pi / n_phi
    t, p = np.meshgrid(th, ph, indexing="ij")
    d = np.stack([np.sin(t) * np.cos(p), np.sin(t) * np.sin(p), np.cos(t)], -1).reshape(-1, 3)
    dw = (np.sin(t) * (np.pi / 2 / n_theta) * (2 * np.pi / n_phi)).reshape(-1)
    return d, dw


def test_lambert_density_weight_and_furnace():
    d, dw = hemisphere_grid(300, 600)
    fc, pdf, ok = oracle.bsdf_eval(0, [0.5, 0.25, 1.0], 0.0, N, wo_at(30), d)
    assert ok.all()
    assert abs((pdf * dw).sum() - 1.0) < 1e-4
    assert np.allclose((fc * dw[:, None]).sum(0), [0.5, 0.25, 1.0], atol=1e-4)  # directional albedo = albedo
    u = np.random.default_rng(0).random((20000, 3))
    wi, w, p, good = oracle.bsdf_sample(0, [0.5, 0.25, 1.0], 0.0, N, wo_at(30), u)
    assert good.mean() > 0.999
    assert np.allclose(w[good], [0.5, 0.25, 1.0])
    assert np.allclose(p[good], wi[good, 2] / np.pi)
    assert np.allclose(np.linalg.norm(wi[good], axis=1), 1.0)


@pytest.mark.parametrize("alpha", [0.1, 0.3, 0.7, 1.0])
@pytest.mark.parametrize("theta", [0, 40, 75])
def test_ggx_sampling_density_and_furnace(alpha, theta):
    wo = wo_at(theta)
    n = 200000
    wi, w, p, good = oracle.bsdf_sample(1, [1.0, 1.0, 1.0], alpha, N, wo, np.random.default_rng(7).random((n, 3)))
    # every kept sample: the density and weight the evaluator gives for that direction
    fc, pe, ok = oracle.bsdf_eval(1, [1.0, 1.0, 1.0], alpha, N, wo, wi[good])
    assert ok.all()
    assert np.allclose(pe, p[good], rtol=1e-9)
    assert np.allclose(fc[:, 0] / pe, w[good, 0], rtol=1e-9)
    # the density integrates over the upper hemisphere to the fraction of samples kept
    d, dw = hemisphere_grid(600, 1200)
    fq, pq, _ = oracle.bsdf_eval(1, [1.0, 1.0, 1.0], alpha, N, wo, d)
    kept = good.mean()
    assert abs((pq * dw).sum() - kept) < 4 * np.sqrt(kept * (1 - kept) / n) + 2e-3
    # white furnace (F0 = 1): directional albedo <= 1, and the mean weight estimates it
    a_q = (fq[:, 0] * dw).sum()
    a_mc = np.where(good, w[:, 0], 0.0)
    assert a_q <= 1.0 + 2e-3
    assert abs(a_q - a_mc.mean()) < 4 * a_mc.std() / np.sqrt(n) + 2e-3
    # at normal incidence the sampled microfacet normal leans past 45 degrees (and
    # the reflection leaves below the horizon) with probability a^2 / (1 + a^2)
    if theta == 0:
        expect = 1.0 / (1.0 + alpha * alpha)
        assert abs(kept - expect) < 4 * np.sqrt(expect * (1 - expect) / n)


@pytest.mark.parametrize("mat,param", [(0, 0.0), (1, 0.05), (1, 0.4), (1, 1.0)])
def test_reciprocity(mat, param):
    rng = np.random.default_rng(3)
    for _ in range(200):
        a = rng.normal(size=3)
        b = rng.normal(size=3)
        a[2], b[2] = abs(a[2]) + 0.05, abs(b[2]) + 0.05
        a /= np.linalg.norm(a)
        b /= np.linalg.norm(b)
        f_ab, _, ok1 = oracle.bsdf_eval(mat, [0.8, 0.5, 0.2], param, N, a, b[None])
        f_ba, _, ok2 = oracle.bsdf_eval(mat, [0.8, 0.5, 0.2], param, N, b, a[None])
        assert ok1[0] == ok2[0]
        if ok1[0]:
            # f cos(wi) / cos(wi) is the BRDF, symmetric in its arguments
            assert np.allclose(f_ab[0] / b[2], f_ba[0] / a[2], rtol=1e-10)


def test_dielectric_reflection_refraction_and_fresnel():
    eta = 1.5
    for deg in (0, 30, 60, 80):
        wo = wo_at(deg)
        wi, w, p, good = oracle.bsdf_sample(2, [1, 1, 1], eta, N, wo, [[0.5, 0.5, 0.0], [0.5, 0.5, 0.999999]])
        assert good.all() and np.allclose(w, 1.0) and np.all(p == 0.0)
        assert np.allclose(wi[0], [-wo[0], -wo[1], wo[2]])  # law of reflection
        sin_t = np.sin(np.radians(deg)) / eta
        assert np.isclose(np.linalg.norm(wi[1]), 1.0)
        assert wi[1, 2] < 0 and np.isclose(np.hypot(wi[1, 0], wi[1, 1]), sin_t)  # Snell
        assert wi[1, 0] <= 1e-12  # continues away from the incoming side
    # Fresnel at normal incidence: ((1 - 1.5) / (1 + 1.5))^2 = 0.04 of uniform choices reflect
    uf = (np.arange(100000) + 0.5) / 100000
    u = np.stack([np.full_like(uf, 0.5), np.full_like(uf, 0.5), uf], -1)
    wi, _, _, _ = oracle.bsdf_sample(2, [1, 1, 1], eta, N, wo_at(0), u)
    assert abs((wi[:, 2] > 0).mean() - 0.04) < 1e-4
    # total internal reflection from inside beyond the critical angle (41.8 degrees)
    t = np.radians(60)
    wo_inside = np.array([np.sin(t), 0.0, -np.cos(t)])
    wi, _, _, _ = oracle.bsdf_sample(2, [1, 1, 1], eta, N, wo_inside, u[::1000])
    assert np.allclose(wi, [-wo_inside[0], -wo_inside[1], wo_inside[2]])  # mirrored, stays inside


def test_sincos_turn_accuracy():
    """The FP32 estimator's sin(2 pi u), cos(2 pi u) (quarter-turn reduction, Taylor
    polynomials): within 2 float ulps of 1 of the exact values on every 24-bit uniform
    the estimator can draw, and s^2 + c^2 = 1 to float rounding."""
    u = (np.arange(1 << 24, dtype=np.float64) / (1 << 24)).astype(np.float32)
    s, c = oracle.sincos_turn(u)
    a = 2 * np.pi * u.astype(np.float64)
    ulp1 = np.spacing(np.float32(1.0))
    assert np.abs(s - np.sin(a)).max() < 2 * ulp1
    assert np.abs(c - np.cos(a)).max() < 2 * ulp1
    norm = s.astype(np.float64) ** 2 + c.astype(np.float64) ** 2
    assert np.abs(norm - 1).max() < 4 * ulp1
    # exact at the quarter turns
    q = np.array([0.0, 0.25, 0.5, 0.75], np.float32)
    sq, cq = oracle.sincos_turn(q)
    assert np.array_equal(sq, [0, 1, 0, -1]) and np.array_equal(cq, [1, 0, -1, 0])
