"""Volumetric path tracing on the GPU (RBR_RENDER_VOLUMETRIC: VolumetricPathIntegrator's
estimator with a HomogeneousMedium and the Henyey-Greenstein phase function) against the CPU
restatement (same random numbers) and the reference's own integrator (statistically)."""
import numpy as np
import pytest

import helpers
from rbr_b200 import abi, render_params, scenes
from test_oracle_pin import foggy_small, moments_z

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("g", [0.0, 0.0005, 0.5, -0.3, 0.9])
def test_phase_function_matches_reference(ctx, reference, g):
    """evaluate is exactly rounded (bit-identical); sample uses cos/sin of 2 pi u2, which CUDA
    and glibc may round an ulp apart: directions within 1e-5 for 99.9 %, within 1e-4 for all."""
    rng = np.random.default_rng(helpers.name_seed(str(g), 1000))
    wo = helpers.unit_vectors(rng, 8192)
    wi = helpers.unit_vectors(rng, 8192)
    u = rng.random((8192, 2), dtype=np.float32)
    assert np.array_equal(bits(ctx.phase_eval(g, wo, wi)), bits(reference.hg_eval(g, wo, wi)))
    dev = np.abs(ctx.phase_sample(g, wo, u) - reference.hg_sample(g, wo, u)).max(axis=1)
    assert dev.max() <= 1e-4 and (dev <= 1e-5).mean() >= 0.999


def test_medium_distance_sampling_matches_reference(ctx, reference):
    """HomogeneousMedium::sampleDistance: logf / expf may differ by an ulp between CUDA and
    glibc, so distances and weights agree to 1e-6 relative; the scatter decision agrees except
    where the sampled distance lies within that of the maximum distance."""
    m = abi.rbr_medium()
    m.sigma_a = abi.f3((0.02, 0.03, 0.01))
    m.sigma_s = abi.f3((0.08, 0.07, 0.09))
    m.g = 0.5
    rng = np.random.default_rng(3)
    n = 8192
    md = np.where(rng.random(n) < 0.1, np.inf, rng.uniform(0.01, 40.0, n)).astype(np.float32)
    u = rng.random(n, dtype=np.float32)
    got, want = ctx.medium_sample(m, md, u), reference.medium_sample(m, md, u)
    same = got[:, 4] == want[:, 4]
    assert same.mean() > 0.999
    np.testing.assert_allclose(got[same], want[same], rtol=2e-6, atol=1e-12)


def test_transparent_medium_never_scatters(ctx, reference):
    m = abi.rbr_medium()
    m.sigma_a = abi.f3((0, 0, 0))
    m.sigma_s = abi.f3((1e-7, 1e-7, 1e-7))
    m.g = 0.0
    u = np.linspace(0, 0.999, 64, dtype=np.float32)
    md = np.full(64, 5.0, np.float32)
    got = ctx.medium_sample(m, md, u)
    assert np.array_equal(got, reference.medium_sample(m, md, u))
    assert (got[:, 4] == 0).all() and (got[:, 1:4] == 1).all()


def path_agreement(a, b, rtol=1e-3, atol=1e-4):
    return np.isclose(a, b, rtol=rtol, atol=atol).all(axis=-1).mean()


@pytest.mark.parametrize("depth", [1, 3, 8])
def test_foggy_cornell_single_paths_match_restatement(ctx, restatement, depth):
    """spp = 1 with identical counter-RNG streams: every pixel is the same path on both sides
    up to logf / expf / cos / sin ulps, which rarely flip a decision (a scatter distance against
    a hit distance, a Russian-roulette draw)."""
    s = foggy_small(48, 48)
    ctx.upload(s)
    p = render_params(spp=1, max_depth=depth, seed=77, flags=abi.RBR_RENDER_VOLUMETRIC)
    gpu = ctx.render_host(s.camera, p)
    cpu = restatement.render(restatement.scene(s), s.camera, p)
    assert np.isfinite(gpu).all()
    frac = path_agreement(gpu, cpu)
    assert frac > 0.97, frac


def test_volumetric_flag_without_medium_matches_restatement(ctx, restatement):
    """Without a medium the volumetric estimator still differs from the path tracer (emission
    at every hit, no MIS weights); the GPU follows the restatement path for path."""
    s = scenes.cornell_box()
    s.camera = scenes.look_at_camera(40, 40, (0.0, 1.0, 3.5), (0.0, 1.0, 0.0), (0.0, 1.0, 0.0), 40.0)
    ctx.upload(s)
    p = render_params(spp=1, max_depth=8, seed=5, flags=abi.RBR_RENDER_VOLUMETRIC)
    gpu = ctx.render_host(s.camera, p)
    cpu = restatement.render(restatement.scene(s), s.camera, p)
    assert path_agreement(gpu, cpu, rtol=1e-4, atol=1e-5) > 0.99
    plain = ctx.render_host(s.camera, render_params(spp=1, max_depth=8, seed=5))
    assert not np.allclose(gpu, plain)


@pytest.mark.slow
@pytest.mark.parametrize("sigma_t,albedo,g,depth", [(0.1, 0.8, 0.5, 3), (1.5, 0.6, 0.3, 8)],
                         ids=["foggy-config-depth3", "dense-medium"])
def test_foggy_cornell_converges_to_reference_integrator(ctx, reference, sigma_t, albedo, g, depth):
    """Per-pixel means of the GPU and of the reference's VolumetricPathIntegrator::Li agree
    within 3 standard errors, and so does the image mean. Both sides take the same number of
    samples: the per-pixel distributions are strongly skewed (rare paths to the light carry
    most of the value), so a small sample underestimates its own variance, and with unequal
    counts the smaller side's standard error would be the one taken too small."""
    s = foggy_small(32, 32, sigma_t=sigma_t, albedo=albedo, g=g)
    ctx.upload(s)
    n_gpu = 2048
    p = render_params(spp=n_gpu, max_depth=depth, seed=2024, flags=abi.RBR_RENDER_VOLUMETRIC)
    mean, m2 = ctx.render_host(s.camera, p, second_moment=True)
    n_ref = 2048
    acc = reference.render_moments(reference.scene(s), s.camera, render_params(spp=n_ref, max_depth=depth), batch=1,
                                   volumetric=True)
    z, z_img = moments_z(mean.astype(np.float64) * n_gpu, m2, n_gpu, acc[0], acc[1], n_ref)
    assert (z > 3).mean() < 0.015
    assert z_img < 3.0, z_img
