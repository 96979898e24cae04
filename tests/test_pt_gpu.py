"""GPU wavefront path tracer (rbr_render) against the CPU restatement and the reference.

1. Same random numbers: the CPU restatement (oracle/rbr_oracle.c) draws the same counter-RNG
   streams (pixel, sample, bounce, purpose) as the GPU, so with spp = 1 every pixel is one and
   the same path on both sides. Arithmetic is rounded identically except cosf/sinf (CUDA vs
   glibc, an ulp apart), so nearly all paths agree to float precision; a few diverge where an
   ulp flips a decision (a grazing hit, a Russian-roulette draw at the threshold).
2. Monte-Carlo agreement with the reference's own integrator (PathTracingIntegrator::Li
   through the reference library): per-pixel means within 3 standard errors, with the tail
   fraction bounded.
"""
import numpy as np
import pytest

import helpers
from rbr_b200 import RbrError, abi, render_params, scenes

pytestmark = pytest.mark.gpu


def small_cornell(w=64, h=64):
    s = scenes.cornell_box()
    s.camera = scenes.look_at_camera(w, h, (0.0, 1.0, 3.5), (0.0, 1.0, 0.0), (0.0, 1.0, 0.0), 40.0)
    return s


def path_agreement(a, b, rtol=1e-4, atol=1e-5):
    """Fraction of pixels whose three channels agree within rtol/atol."""
    close = np.isclose(a, b, rtol=rtol, atol=atol).all(axis=-1)
    return close.mean()


@pytest.mark.parametrize("nee,mis", [(True, True), (True, False), (False, False)])
def test_cornell_single_paths_match_restatement(ctx, restatement, nee, mis):
    s = small_cornell()
    ctx.upload(s)
    p = render_params(spp=1, max_depth=8, use_nee=nee, use_mis=mis, seed=1234)
    gpu = ctx.render_host(s.camera, p)
    cpu = restatement.render(restatement.scene(s), s.camera, p)
    assert np.isfinite(gpu).all()
    frac = path_agreement(gpu, cpu)
    assert frac > 0.99, f"only {frac:.4f} of single-sample paths agree"
    # the image as a whole agrees far below Monte-Carlo noise
    assert abs(gpu.mean() - cpu.mean()) < 1e-3 * cpu.mean()


def test_cornell_multi_sample_film_matches_restatement(ctx, restatement):
    s = small_cornell(48, 40)
    ctx.upload(s)
    p = render_params(spp=16, max_depth=8, seed=7, sample_offset=32)
    gpu = ctx.render_host(s.camera, p)
    cpu = restatement.render(restatement.scene(s), s.camera, p)
    assert path_agreement(gpu, cpu, rtol=1e-3, atol=1e-4) > 0.97
    assert abs(gpu.mean() - cpu.mean()) < 2e-3 * cpu.mean()


def test_second_moment_and_stats(ctx, restatement):
    s = small_cornell(32, 32)
    ctx.upload(s)
    p = render_params(spp=8, max_depth=8, seed=3)
    mean, m2 = ctx.render_host(s.camera, p, second_moment=True)
    _, sm, sq = restatement.render(restatement.scene(s), s.camera, p, moments=True)
    assert np.allclose(mean * 8, sm, rtol=2e-3, atol=1e-3)
    close = np.isclose(m2, sq, rtol=2e-3, atol=1e-3).all(-1).mean()
    assert close > 0.97
    st = ctx.render_stats()
    assert st.paths == 32 * 32 * 8 and st.waves == 2  # a one-wave image runs as two halves in flight
    assert st.extension_rays >= st.paths and st.shadow_rays > 0 and st.milliseconds > 0


def test_waves_do_not_change_results(ctx):
    """Every path's random numbers depend only on (pixel, sample): splitting a render into
    sample ranges, or into several waves, gives the same film up to summation order."""
    s = scenes.cornell_box(1400, 1400)  # 7.84 M paths at 4 spp: two waves
    ctx.upload(s)
    full = ctx.render_host(s.camera, render_params(spp=4, seed=11))
    assert ctx.render_stats().waves >= 2
    a = ctx.render_host(s.camera, render_params(spp=2, seed=11, sample_offset=0))
    b = ctx.render_host(s.camera, render_params(spp=2, seed=11, sample_offset=2))
    assert np.allclose(full, 0.5 * (a + b), rtol=1e-5, atol=1e-5)


def test_two_waves_in_flight_match_one(ctx):
    """pt.streams 2 (waves alternate between two path-buffer sets and two streams) renders the
    same film and counts the same rays as one wave at a time, up to summation order; a small
    wave size makes four waves, so both buffer sets are reused."""
    s = scenes.cornell_box(256, 256)
    ctx.upload(s)
    wave_paths = ctx.get_param("pt.wave_paths")
    ctx.set_param("pt.wave_paths", 65536)
    try:
        p = render_params(spp=4, seed=21)
        ctx.set_param("pt.streams", 1)
        one = ctx.render_host(s.camera, p)
        st1 = ctx.render_stats()
        ctx.set_param("pt.streams", 2)
        two = ctx.render_host(s.camera, p)
        st2 = ctx.render_stats()
    finally:
        ctx.set_param("pt.streams", 2)
        ctx.set_param("pt.wave_paths", wave_paths)
    assert st1.waves == st2.waves == 4
    assert st1.extension_rays == st2.extension_rays and st1.shadow_rays == st2.shadow_rays
    assert np.allclose(one, two, rtol=1e-5, atol=1e-5)
    with pytest.raises(RbrError):
        ctx.set_param("pt.streams", 3)


@pytest.mark.parametrize("split", [0, 1])
def test_claimed_work_matches_grid_stride(ctx, split):
    """pt.fetch 1 (long queues handed out by claims on per-depth cursors) traces, shades
    and counts exactly the work of the fixed grid-stride order (pt.fetch 0): the same rays, nodes
    and records, and the same film up to the order of the shadow rays' atomic additions. Three
    lights and GGX materials; 5.2 M paths in two waves of up to 2^22, so the queues of the first
    depths are long enough for claims (eight grid rounds and more) and the later ones are not,
    and the cursors are reset between depths and waves; with pt.shade_split 1 the per-class
    shading launches keep the grid-stride order beside claimed extension and shadow launches."""
    s = scenes.ggx_scene(1024, 640, n_spheres=24, mesh_n=400, seed=3)
    ctx.upload(s)
    wave_paths = ctx.get_param("pt.wave_paths")
    ctx.set_param("pt.wave_paths", 1 << 22)
    ctx.set_param("pt.shade_split", split)
    films, stats = {}, {}
    try:
        for fetch in (0, 1):
            ctx.set_param("pt.fetch", fetch)
            p = render_params(spp=8, max_depth=12, seed=17, flags=abi.RBR_RENDER_COUNT_TRAFFIC)
            films[fetch] = ctx.render_host(s.camera, p)
            stats[fetch] = ctx.render_stats()
    finally:
        ctx.set_param("pt.fetch", 1)
        ctx.set_param("pt.shade_split", 0)
        ctx.set_param("pt.wave_paths", wave_paths)
    a, b = stats[0], stats[1]
    assert a.waves == b.waves == 2 and a.ext_nodes > 0 and a.shadow_nodes > 0
    for f in ("extension_rays", "shadow_rays", "shaded_vertices", "ext_nodes", "ext_records", "shadow_nodes",
              "shadow_records"):
        assert getattr(a, f) == getattr(b, f), f
    assert np.isfinite(films[1]).all()
    np.testing.assert_allclose(films[1], films[0], rtol=1e-5, atol=1e-6)
    with pytest.raises(RbrError):
        ctx.set_param("pt.fetch", 2)


def test_edge_parameters(ctx, restatement):
    s = small_cornell(16, 16)
    s.background = (0.25, 0.5, 1.0)  # camera rays leaving through the open front see it
    ctx.upload(s)
    zero = ctx.render_host(s.camera, render_params(spp=2, max_depth=0))
    assert (zero == 0).all()
    p = render_params(spp=4, max_depth=1, seed=5)
    gpu = ctx.render_host(s.camera, p)
    cpu = restatement.render(restatement.scene(s), s.camera, p)
    assert path_agreement(gpu, cpu) > 0.99
    with pytest.raises(RbrError) as e:
        ctx.render_host(s.camera, render_params(spp=0))
    assert e.value.status == abi.RBR_ERR_INVALID_ARGUMENT


def test_thin_lens_point_light_glass(ctx, restatement):
    """Thin-lens camera, a point light beside the area light, glass, mirror and rough metal."""
    s = small_cornell(48, 48)
    glass = s.add_material(base_color=(1, 1, 1), roughness=0.0, ior=1.5, transmission=1.0)
    rough_glass = s.add_material(base_color=(0.9, 1, 0.9), roughness=0.3, ior=1.5, transmission=1.0)
    mirror = s.add_material(base_color=(0.9, 0.9, 0.9), metallic=1.0, roughness=0.0)
    metal = s.add_material(base_color=(0.9, 0.7, 0.4), metallic=1.0, roughness=0.4)
    plastic = s.add_material(base_color=(0.2, 0.4, 0.8), roughness=0.2, ior=1.5)
    s.spheres = np.array([[-0.4, 0.4, 0.0, 0.35], [0.45, 0.3, 0.3, 0.3], [0.0, 1.3, -0.4, 0.25],
                          [-0.5, 1.2, 0.3, 0.2], [0.5, 1.0, -0.5, 0.22]], np.float32)
    s.sphere_materials = np.array([glass, mirror, metal, rough_glass, plastic], np.uint32)
    s.point_light((0.0, 1.8, 0.5), (1.0, 1.0, 1.0), 2.0)
    s.camera = scenes.look_at_camera(48, 48, (0.0, 1.0, 3.5), (0.0, 1.0, 0.0), (0, 1, 0), 40.0,
                                     lens_radius=0.05, focal_distance=3.5)
    ctx.upload(s)
    p = render_params(spp=1, max_depth=12, seed=99)
    gpu = ctx.render_host(s.camera, p)
    cpu = restatement.render(restatement.scene(s), s.camera, p)
    assert path_agreement(gpu, cpu) > 0.98


@pytest.mark.slow
def test_cornell_converges_to_reference_integrator(ctx, reference):
    """Cornell box on the configured 256x256 camera (pinhole, fov 40), central 96x96 crop: per-pixel
    means of the GPU and of the reference's PathTracingIntegrator::Li agree within 3 standard
    errors (independent random numbers on the two sides), and so do the image means."""
    s = scenes.cornell_box()
    assert (s.camera.width, s.camera.height) == (256, 256)
    cam = helpers.crop_camera(s.camera, 80, 80, 96, 96)
    ctx.upload(s)
    n_gpu = 4096
    mean, m2 = ctx.render_host(cam, render_params(spp=n_gpu, max_depth=8, seed=2024), second_moment=True)
    n_ref = 512
    acc = reference.render_moments(reference.scene(s), cam, render_params(spp=n_ref, max_depth=8), batch=0)
    z, z_img = helpers.moments_z(mean.astype(np.float64) * n_gpu, m2, n_gpu, acc[0], acc[1], n_ref)
    tail = (z > 3).mean()
    assert tail < 0.01, f"{tail:.4f} of pixel channels beyond 3 standard errors"
    assert z_img < 3.0, f"image means differ by {z_img:.2f} standard errors"


@pytest.mark.slow
def test_ggx_scene_converges_to_reference_integrator(ctx, reference):
    """The GGX material scene at 64x36 (mound of 7,200 triangles, 260 spheres of every material
    class including smooth glass, a mirror and smooth dielectrics, two area lights with emissive
    quads, a point light, thin-lens camera, max depth 16): the GPU path tracer and the
    reference's own PathTracingIntegrator::Li agree per pixel channel within 3 standard errors
    (independent random numbers) and in the image mean. This pins the GPU estimator on the
    delta / transmission / MIS paths directly against the reference, not only against the
    restatement that shares its random numbers."""
    s = helpers.ggx_small(64, 36, mesh_n=60)
    ctx.upload(s)
    n_gpu = 16384
    mean, m2 = ctx.render_host(s.camera, render_params(spp=n_gpu, max_depth=16, seed=2025), second_moment=True)
    n_ref = 2048
    acc = reference.render_moments(reference.scene(s), s.camera, render_params(spp=n_ref, max_depth=16), batch=0)
    z, z_img = helpers.moments_z(mean.astype(np.float64) * n_gpu, m2, n_gpu, acc[0], acc[1], n_ref)
    assert (acc[0] > 0).mean() > 0.5
    tail = (z > 3).mean()
    assert tail < 0.01, f"{tail:.4f} of pixel channels beyond 3 standard errors"
    assert z_img < 3.0, f"image means differ by {z_img:.2f} standard errors"
