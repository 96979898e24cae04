"""The reference's own known-answer checks (tests/test_materials.cpp, tests/test_core.cpp),
restated at the Material level and applied to the CPU restatement and to the GPU's device
functions: furnace tests, sample/evaluate/pdf consistency, energy conservation, glass weights,
total internal reflection, emissive materials, power-heuristic edge values."""
import math

import numpy as np
import pytest

import helpers
from rbr_b200 import abi

F32 = np.float32


def direction_from_cos(c, phi=0.3):
    s = math.sqrt(max(0.0, 1.0 - c * c))
    return np.array([s * math.cos(phi), s * math.sin(phi), c], F32)


class Impl:
    def __init__(self, eval_fn, sample_fn, mis_fn):
        self.eval, self.sample, self.mis = eval_fn, sample_fn, mis_fn


@pytest.fixture(params=["restatement", pytest.param("gpu", marks=pytest.mark.gpu)])
def impl(request):
    if request.param == "restatement":
        r = request.getfixturevalue("restatement")

        def ev(m, wo, wi):
            f, pdf, info = r.bsdf_eval(m, wo, wi)
            return f, pdf, info

        return Impl(ev, r.bsdf_sample, lambda a, b: r.power_heuristic(1, a, 1, b))
    ctx = request.getfixturevalue("ctx")

    def ev(m, wo, wi):
        e = ctx.bsdf_eval(m, wo, wi)
        return e[:, :3], e[:, 3], np.array([e[0, 4], e[0, 5]], np.uint32)

    return Impl(ev, ctx.bsdf_sample, lambda a, b: float(ctx.mis_weights(np.array([[a, b]], F32))[0]))


def sampled_albedo(impl, m, wo, n, seed):
    """Mean of f.x |cos| / pdf over BSDF::sample (test_materials.cpp:49-58)."""
    rng = np.random.default_rng(seed)
    u = np.minimum(rng.random((n, 2), dtype=F32), F32(0.99999994))
    s = impl.sample(m, np.tile(wo, (n, 1)), u)
    ok = s[:, 6] > 0
    return float(np.sum(s[ok, 3] * np.abs(s[ok, 2]) / s[ok, 6]) / n)


def test_white_diffuse_furnace(impl):
    m = helpers.material((1, 1, 1), roughness=1.0, ior=1.0)
    for c in (1.0, 0.6, 0.15, -0.5):
        assert abs(sampled_albedo(impl, m, direction_from_cos(c), 200000, 1) - 1.0) < 0.01


def test_glass_weights(impl):
    """Smooth glass: reflection + refraction weights add up to F + (1 - F) / 1.5^2; rough glass
    keeps about the same total (test_materials.cpp:229-243)."""
    wo = direction_from_cos(0.6)
    cos_i, eta = 0.6, 1.0 / 1.5
    sin_t = eta * math.sqrt(1 - cos_i ** 2)
    cos_t = math.sqrt(1 - sin_t ** 2)
    rpar = (1.5 * cos_i - cos_t) / (1.5 * cos_i + cos_t)
    rper = (cos_i - 1.5 * cos_t) / (cos_i + 1.5 * cos_t)
    F = 0.5 * (rpar ** 2 + rper ** 2)
    glass = helpers.material((1, 1, 1), roughness=0.0, transmission=1.0)
    assert abs(sampled_albedo(impl, glass, wo, 400000, 2) - (F + (1 - F) / 2.25)) < 0.01
    f, pdf, info = impl.eval(glass, wo[None], direction_from_cos(0.5)[None])
    assert info[0] == 1, "smooth glass is a delta BSDF"
    rough = helpers.material((1, 1, 1), roughness=0.3, transmission=1.0)
    assert abs(sampled_albedo(impl, rough, wo, 400000, 3) - (F + (1 - F) / 2.25)) < 0.08


def test_total_internal_reflection(impl):
    """Leaving glass beyond the critical angle nothing is transmitted (test_materials.cpp:150-151)."""
    glass = helpers.material((1, 1, 1), roughness=0.0, transmission=1.0)
    wo = direction_from_cos(-0.5)
    rng = np.random.default_rng(4)
    s = impl.sample(glass, np.tile(wo, (1000, 1)), rng.random((1000, 2), dtype=F32))
    ok = s[:, 6] > 0
    assert ok.all() and (s[:, 2] < 0).all(), "every sample stays on the incident side"


@pytest.mark.parametrize("name,mat", helpers.material_grid(), ids=[n for n, _ in helpers.material_grid()])
def test_energy_conservation_and_consistency(impl, name, mat):
    """Sampled albedo <= 1 (+1e-2) and sample() agrees with evaluate()/pdf() for non-delta
    samples to 1e-3 (test_materials.cpp:86-102, 197-221)."""
    wo = direction_from_cos(0.6)
    albedo = sampled_albedo(impl, mat, wo, 100000, 5)
    assert albedo <= 1.0 + 1e-2
    rng = np.random.default_rng(6)
    u = np.minimum(rng.random((20000, 2), dtype=F32), F32(0.99999994))
    s = impl.sample(mat, np.tile(wo, (20000, 1)), u)
    nd = (s[:, 6] > 0) & (s[:, 7] == 0)
    if nd.any():
        f, pdf, _ = impl.eval(mat, np.tile(wo, (nd.sum(), 1)), s[nd, :3])
        assert np.all(np.abs(pdf - s[nd, 6]) <= 1e-3 * np.maximum(1, s[nd, 6]))
        assert np.all(np.abs(f[:, 0] - s[nd, 3]) <= 1e-3 * np.maximum(1, s[nd, 3]))


def test_emissive_material_does_not_scatter(impl):
    m = helpers.material((0, 0, 0), ior=1.0, emission=(5, 5, 5))
    wo = direction_from_cos(0.6)
    s = impl.sample(m, wo[None], np.array([[0.3, 0.6]], F32))
    assert s[0, 6] == 0.0
    f, pdf, _ = impl.eval(m, wo[None], direction_from_cos(0.5)[None])
    assert (f <= 0).all() and pdf[0] == 0.0


def test_power_heuristic_edges(impl):
    """test_core.cpp:80-93."""
    inf = float("inf")
    assert abs(impl.mis(1.0, 1.0) - 0.5) < 1e-5
    assert impl.mis(inf, 1.0) == 1.0
    assert impl.mis(1.0, inf) == 0.0
    assert impl.mis(0.0, 0.0) == 0.0
    assert not math.isnan(impl.mis(1e30, 1e30))
