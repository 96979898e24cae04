"""Pins the CPU restatement (oracle/rbr_oracle.c) to the reference library built from its own
sources (oracle/_ref): identical inputs must give bit-identical outputs for every function
the GPU path restates. Runs on CPU."""
import numpy as np
import pytest

import helpers
from rbr_b200 import abi, render_params, scenes


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("name,mat", helpers.material_grid(), ids=[n for n, _ in helpers.material_grid()])
def test_bsdf_eval_and_sample_bit_exact(restatement, reference, name, mat):
    wo, wi, u = helpers.bsdf_inputs(4096, seed=helpers.name_seed(name, 1000))
    f1, p1, i1 = restatement.bsdf_eval(mat, wo, wi)
    f2, p2, i2 = reference.bsdf_eval(mat, wo, wi)
    assert np.array_equal(bits(f1), bits(f2)) and np.array_equal(bits(p1), bits(p2))
    assert np.array_equal(i1, i2), "isDelta / BSDFType bits"
    s1 = restatement.bsdf_sample(mat, wo, u)
    s2 = reference.bsdf_sample(mat, wo, u)
    assert np.array_equal(bits(s1), bits(s2))


@pytest.mark.parametrize("name,mat", helpers.material_grid(), ids=[n for n, _ in helpers.material_grid()])
def test_bsdf_eval_edge_directions(restatement, reference, name, mat):
    """The restatement's evaluate() and pdf() on the direction pairs where their checks decide."""
    wo, wi = helpers.edge_directions()
    f1, p1, _ = restatement.bsdf_eval(mat, wo, wi)
    f2, p2, _ = reference.bsdf_eval(mat, wo, wi)
    assert np.array_equal(bits(f1), bits(f2)) and np.array_equal(bits(p1), bits(p2))


def test_light_samples_bit_exact(restatement, reference):
    p, u = helpers.light_points(4096, seed=4)
    for l in helpers.lights():
        assert np.array_equal(bits(restatement.light_sample(l, p, u)), bits(reference.light_sample(l, p, u)))


@pytest.mark.parametrize("lens", [0.0, 0.1])
def test_camera_rays_bit_exact(restatement, reference, lens):
    cam = reference.camera(200, 100, (0, 1, 5), (0, 1, 0), (0, 1, 0), 40.0, lens_radius=lens, focal_distance=4.0)
    s = helpers.camera_samples(cam, 4096, seed=5)
    assert np.array_equal(bits(restatement.camera_rays(cam, s)), bits(reference.camera_rays(cam, s)))


def test_camera_setup_matches_reference_lookat():
    """look_at_camera (float32 numpy) reproduces CameraExtrinsics::lookAt + fromVerticalFov."""
    from oracle import Reference, have_reference

    if not have_reference():
        pytest.skip("reference library not built")
    ref = Reference()
    for args in [((0.0, 1.0, 3.5), (0.0, 1.0, 0.0), 40.0), ((0.0, 3.0, 14.0), (0.0, 0.8, 0.0), 40.0),
                 ((1.0, 2.0, 3.0), (-1.0, 0.5, 0.2), 65.0)]:
        mine = scenes.look_at_camera(256, 192, args[0], args[1], (0, 1, 0), args[2])
        theirs = ref.camera(256, 192, args[0], args[1], (0, 1, 0), args[2])
        for f in ("position", "forward", "right", "up"):
            assert np.array_equal(np.array(getattr(mine, f)[:], np.float32), np.array(getattr(theirs, f)[:], np.float32)), f
        assert abs(mine.fy - theirs.fy) <= 1e-6 * theirs.fy and mine.cx == theirs.cx and mine.cy == theirs.cy


def test_power_heuristic_bit_exact(restatement, reference):
    for a, b in helpers.mis_pairs():
        x, y = restatement.power_heuristic(1, float(a), 1, float(b)), reference.power_heuristic(1, float(a), 1, float(b))
        assert np.float32(x).view(np.uint32) == np.float32(y).view(np.uint32) or (np.isnan(x) and np.isnan(y))


@pytest.mark.parametrize("ns,nt,nq,plane,seed", [(30, 30, 10, False, 1), (400, 1500, 100, False, 2),
                                                  (60, 200, 20, True, 3)])
def test_ray_queries_bit_exact(restatement, reference, ns, nt, nq, plane, seed):
    w = scenes.random_world(ns, nt, plane, seed=seed, n_quads=nq)
    rays = scenes.random_test_rays(4000, seed=seed + 10)
    o, r = restatement.scene(w), reference.scene(w)
    a, b = restatement.trace_closest(o, rays), reference.trace_closest(r, rays, brute=True)
    assert np.array_equal(a["prim"], b["prim"]) and np.array_equal(bits(a["t"]), bits(b["t"]))
    assert np.array_equal(restatement.trace_any(o, rays), reference.trace_any(r, rays, brute=True))


def test_integrator_matches_reference_statistically(restatement, reference):
    """The restated PathTracingIntegrator::Li (with the counter RNG) and the reference's own
    (with mt19937_64) converge to the same image: per-pixel 3-sigma test."""
    s = scenes.cornell_box()
    s.camera = scenes.look_at_camera(32, 32, (0.0, 1.0, 3.5), (0.0, 1.0, 0.0), (0.0, 1.0, 0.0), 40.0)
    n = 512
    _, S, Q = restatement.render(restatement.scene(s), s.camera, render_params(spp=n, seed=5), moments=True)
    acc = reference.render_moments(reference.scene(s), s.camera, render_params(spp=n), batch=3)
    mu_o, mu_r = S / n, acc[0] / n
    var_o = np.maximum(Q / n - mu_o ** 2, 0) * n / (n - 1)
    var_r = np.maximum(acc[1] / n - mu_r ** 2, 0) * n / (n - 1)
    se = np.sqrt(var_o / n + var_r / n)
    z = np.abs(mu_o - mu_r) / np.maximum(se, 1e-12)
    z[(se == 0) & (np.abs(mu_o - mu_r) < 1e-6)] = 0
    assert (z > 3).mean() < 0.01


def test_integrator_matches_reference_on_ggx_scene(restatement, reference):
    """The GGX material scene reduced to a 32x18 film (every material class, smooth glass,
    mirror and smooth dielectrics included; two area lights and a point light; thin-lens camera;
    max depth 16): the restated PathTracingIntegrator::Li and the reference's own converge to the
    same image, per pixel channel within 3 standard errors and in the image mean."""
    s = helpers.ggx_small(32, 18, mesh_n=40)
    n = 256
    _, S, Q = restatement.render(restatement.scene(s), s.camera, render_params(spp=n, max_depth=16, seed=5),
                                 moments=True)
    acc = reference.render_moments(reference.scene(s), s.camera, render_params(spp=n, max_depth=16), batch=3)
    z, z_img = helpers.moments_z(S, Q, n, acc[0], acc[1], n)
    assert (S > 0).mean() > 0.5  # most pixel channels see light
    assert (z > 3).mean() < 0.01
    assert z_img < 3.0, z_img


@pytest.mark.parametrize("g", [0.0, 0.0005, 0.5, -0.3, 0.9])
def test_phase_function_bit_exact(restatement, reference, g):
    """HenyeyGreensteinPhase::evaluate and ::sample restated (phase_function.cpp:17-41)."""
    rng = np.random.default_rng(helpers.name_seed(str(g), 1000))
    wo = helpers.unit_vectors(rng, 4096)
    wi = helpers.unit_vectors(rng, 4096)
    u = rng.random((4096, 2), dtype=np.float32)
    assert np.array_equal(restatement.hg_eval(g, wo, wi), reference.hg_eval(g, wo, wi))
    assert np.array_equal(restatement.hg_sample(g, wo, u), reference.hg_sample(g, wo, u))


def foggy_small(w=24, h=24, **kw):
    s = scenes.foggy_cornell_box(**kw)
    s.camera = scenes.look_at_camera(w, h, (0.0, 1.0, 3.5), (0.0, 1.0, 0.0), (0.0, 1.0, 0.0), 40.0)
    return s


def moments_z(S1, Q1, n1, S2, Q2, n2):
    """Per-pixel z scores and the z score of the image mean of two sets of sample moments."""
    mu1, mu2 = S1 / n1, S2 / n2
    var1 = np.maximum(Q1 / n1 - mu1 ** 2, 0) * n1 / (n1 - 1)
    var2 = np.maximum(Q2 / n2 - mu2 ** 2, 0) * n2 / (n2 - 1)
    se = np.sqrt(var1 / n1 + var2 / n2)
    z = np.abs(mu1 - mu2) / np.maximum(se, 1e-12)
    z[(se == 0) & (np.abs(mu1 - mu2) < 1e-6)] = 0
    m = mu1.size
    z_img = abs(mu1.mean() - mu2.mean()) / max(np.sqrt((var1 / n1 + var2 / n2).sum()) / m, 1e-12)
    return z, z_img


@pytest.mark.parametrize("sigma_t,albedo,g,depth", [(0.1, 0.8, 0.5, 3), (1.5, 0.6, 0.3, 8)],
                         ids=["foggy-config-depth3", "dense-medium"])
def test_volumetric_integrator_matches_reference_statistically(restatement, reference, sigma_t, albedo, g, depth):
    """The restated VolumetricPathIntegrator::Li (counter RNG) and the reference's own converge
    to the same image of the foggy Cornell box: per-pixel 3-sigma test and the image mean within
    3 standard errors. The reference's scatter weight sigma_s * Tr / mean(sigma_t)^2 has mean
    albedo / (2 mean(sigma_t)) = 4 per event for the configured fog, so its variance grows
    geometrically with depth; the configured medium is compared at depth 3, a dense one
    (weight <= 0.27) at depth 8."""
    s = foggy_small(sigma_t=sigma_t, albedo=albedo, g=g)
    n = 512
    p = render_params(spp=n, max_depth=depth, seed=5, flags=abi.RBR_RENDER_VOLUMETRIC)
    _, S, Q = restatement.render(restatement.scene(s), s.camera, p, moments=True)
    acc = reference.render_moments(reference.scene(s), s.camera, render_params(spp=n, max_depth=depth), batch=5,
                                   volumetric=True)
    z, z_img = moments_z(S, Q, n, acc[0], acc[1], n)
    assert (z > 3).mean() < 0.015
    assert z_img < 3.0, z_img
