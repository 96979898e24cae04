"""The CPU restatement and the GPU library against the golden fixtures in tests/golden/
(outputs of the reference library itself, made by tests/golden/make_golden.py). These tests
need neither the reference sources nor the reference library at run time."""
from pathlib import Path

import numpy as np
import pytest

from rbr_b200 import abi, render_params, scenes

GOLDEN = Path(__file__).resolve().parent / "golden"


def load(name):
    return np.load(GOLDEN / name)


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def material(p):
    m = abi.rbr_material()
    m.base_color = abi.f3(p[0:3])
    m.metallic, m.roughness, m.ior, m.transmission = (float(x) for x in p[3:7])
    m.emission = abi.f3(p[7:10])
    return m


def light(p):
    l = abi.rbr_light()
    l.type = int(p[0])
    l.position, l.u, l.v, l.color = abi.f3(p[1:4]), abi.f3(p[4:7]), abi.f3(p[7:10]), abi.f3(p[10:13])
    l.intensity = float(p[13])
    return l


def camera(p):
    c = abi.rbr_camera()
    c.width, c.height, c.model = int(p[0]), int(p[1]), int(p[2])
    c.position, c.forward, c.right, c.up = abi.f3(p[3:6]), abi.f3(p[6:9]), abi.f3(p[9:12]), abi.f3(p[12:15])
    c.fx, c.fy, c.cx, c.cy, c.lens_radius, c.focal_distance = (float(x) for x in p[15:21])
    return c


def golden_world():
    g = load("golden_rays.npz")
    s = scenes.Scene()
    m = s.diffuse((0.5, 0.5, 0.5))
    s.triangles, s.triangle_ids = g["triangles"], g["triangle_ids"]
    s.spheres, s.sphere_ids = g["spheres"], g["sphere_ids"]
    s.quads, s.quad_ids = g["quads"], g["quad_ids"]
    s.planes, s.plane_ids = g["planes"], g["plane_ids"]
    s.triangle_materials = np.full(len(s.triangles), m, np.uint32)
    s.sphere_materials = np.full(len(s.spheres), m, np.uint32)
    s.quad_materials = np.full(len(s.quads), m, np.uint32)
    s.plane_materials = np.full(len(s.planes), m, np.uint32)
    return s, g["rays"].view(abi.RAY_DTYPE), g


def z_fraction(mean, m2_or_var, n, golden, from_moments):
    if from_moments:
        var = np.maximum(m2_or_var / n - mean.astype(np.float64) ** 2, 0) * n / (n - 1)
    else:
        var = m2_or_var
    se = np.sqrt(var / n + golden["var"] / int(golden["n"]))
    z = np.abs(mean - golden["mean"]) / np.maximum(se, 1e-12)
    z[(se == 0) & (np.abs(mean - golden["mean"]) < 1e-6)] = 0
    return (z > 3).mean()


# ------------------------------------------------------------------------------------------ CPU
def test_restatement_rays(restatement):
    s, rays, g = golden_world()
    h = restatement.scene(s)
    hits = restatement.trace_closest(h, rays)
    assert np.array_equal(hits["prim"], g["prim"]) and np.array_equal(bits(hits["t"]), bits(g["t"]))
    assert np.array_equal(restatement.trace_any(h, rays), g["occluded"])


def test_restatement_bsdf(restatement):
    g = load("golden_bsdf.npz")
    for k, p in enumerate(g["params"]):
        m = material(p)
        f, pdf, info = restatement.bsdf_eval(m, g["wo"][k], g["wi"][k])
        assert np.array_equal(bits(f), bits(g["eval"][k][:, :3])) and np.array_equal(bits(pdf), bits(g["eval"][k][:, 3]))
        assert np.array_equal(info, g["info"][k])
        assert np.array_equal(bits(restatement.bsdf_sample(m, g["wo"][k], g["u"][k])), bits(g["sample"][k])), g["names"][k]


def test_restatement_lights_cameras_mis(restatement):
    g = load("golden_lights.npz")
    for p, out in zip(g["params"], g["out"]):
        assert np.array_equal(bits(restatement.light_sample(light(p), g["points"], g["u"])), bits(out))
    g = load("golden_camera.npz")
    for p, out in zip(g["params"], g["out"]):
        assert np.array_equal(bits(restatement.camera_rays(camera(p), g["samples"])), bits(out))
    g = load("golden_mis.npz")
    got = np.array([restatement.power_heuristic(1, float(a), 1, float(b)) for a, b in g["pairs"]], np.float32)
    assert np.array_equal(bits(got), bits(g["weights"]))


def test_restatement_cornell_converges_to_golden(restatement):
    g = load("golden_cornell.npz")
    s = scenes.cornell_box()
    cam = camera(g["camera"])
    n = 1024
    _, S, Q = restatement.render(restatement.scene(s), cam, render_params(spp=n, seed=9), moments=True)
    assert z_fraction(S / n, Q, n, g, True) < 0.01


def fog_z(mean, var_or_m2, n, g, from_moments):
    """z scores of a foggy-Cornell estimate against golden_volume.npz, and of the image mean."""
    if from_moments:
        var = np.maximum(var_or_m2 / n - mean.astype(np.float64) ** 2, 0) * n / (n - 1)
    else:
        var = var_or_m2
    ng = int(g["fog_n"])
    se = np.sqrt(var / n + g["fog_var"] / ng)
    z = np.abs(mean - g["fog_mean"]) / np.maximum(se, 1e-12)
    z[(se == 0) & (np.abs(mean - g["fog_mean"]) < 1e-6)] = 0
    z_img = abs(mean.mean() - g["fog_mean"].mean()) / max(np.sqrt((var / n + g["fog_var"] / ng).sum()) / mean.size, 1e-12)
    return (z > 3).mean(), z_img


def test_restatement_volume(restatement):
    g = load("golden_volume.npz")
    for k, gv in enumerate(g["g"]):
        assert np.array_equal(bits(restatement.hg_eval(float(gv), g["wo"], g["wi"])), bits(g["hg_eval"][k]))
        assert np.array_equal(bits(restatement.hg_sample(float(gv), g["wo"], g["u"])), bits(g["hg_sample"][k]))
    s = scenes.foggy_cornell_box()
    n = 4096
    p = render_params(spp=n, max_depth=3, seed=19, flags=abi.RBR_RENDER_VOLUMETRIC)
    _, S, Q = restatement.render(restatement.scene(s), camera(g["fog_camera"]), p, moments=True)
    tail, z_img = fog_z(S / n, Q, n, g, True)
    assert tail < 0.015 and z_img < 3.0, (tail, z_img)


def test_obj_meshes_golden():
    from rbr_b200 import parse_obj

    g = load("golden_obj.npz")
    for i, (name, text) in enumerate(zip(g["names"], g["texts"])):
        v, nn = parse_obj(bytes(text))
        assert np.array_equal(bits(v), bits(g[f"v{i}"])), name
        want_n = g[f"n{i}"]
        assert (nn is None) == (len(want_n) == 0), name
        if nn is not None:
            assert np.array_equal(bits(nn), bits(want_n)), name


# ------------------------------------------------------------------------------------------ GPU
@pytest.mark.gpu
def test_gpu_rays(ctx):
    s, rays, g = golden_world()
    ctx.upload(s)
    hits = ctx.trace_host(rays)
    assert np.array_equal(hits["prim"], g["prim"]) and np.array_equal(bits(hits["t"]), bits(g["t"]))
    assert np.array_equal(ctx.trace_host(rays, any_hit=True), g["occluded"])


@pytest.mark.gpu
def test_gpu_bsdf_lights_cameras_mis(ctx):
    g = load("golden_bsdf.npz")
    for k, p in enumerate(g["params"]):
        m = material(p)
        e = ctx.bsdf_eval(m, g["wo"][k], g["wi"][k])
        assert np.array_equal(bits(e[:, :4]), bits(g["eval"][k])), g["names"][k]
        assert (e[:, 4] == g["info"][k][0]).all() and (e[:, 5] == g["info"][k][1]).all()
        smp, want = ctx.bsdf_sample(m, g["wo"][k], g["u"][k]), g["sample"][k]
        valid = (smp[:, 6] > 0) & (want[:, 6] > 0)
        assert ((smp[:, 6] > 0) == (want[:, 6] > 0)).mean() >= 0.99, g["names"][k]
        assert np.abs(smp[valid, :3] - want[valid, :3]).max(initial=0.0) <= 1e-5, g["names"][k]
        if valid.any():
            assert np.isclose(smp[valid, 3:7], want[valid, 3:7], rtol=1e-5).all(axis=1).mean() >= 0.97, g["names"][k]
    g = load("golden_lights.npz")
    for p, out in zip(g["params"], g["out"]):
        assert np.array_equal(bits(ctx.light_sample(light(p), g["points"], g["u"])), bits(out))
    g = load("golden_camera.npz")
    pin, thin = (camera(p) for p in g["params"])
    assert np.array_equal(bits(ctx.camera_rays(pin, g["samples"])), bits(g["out"][0]))
    assert np.allclose(ctx.camera_rays(thin, g["samples"]), g["out"][1], rtol=1e-5, atol=1e-6)
    g = load("golden_mis.npz")
    assert np.array_equal(bits(ctx.mis_weights(g["pairs"])), bits(g["weights"]))


@pytest.mark.gpu
def test_gpu_cornell_converges_to_golden(ctx):
    g = load("golden_cornell.npz")
    s = scenes.cornell_box()
    ctx.upload(s)
    n = 8192
    mean, m2 = ctx.render_host(camera(g["camera"]), render_params(spp=n, seed=10), second_moment=True)
    assert z_fraction(mean, m2, n, g, True) < 0.01


@pytest.mark.gpu
def test_gpu_volume(ctx):
    g = load("golden_volume.npz")
    for k, gv in enumerate(g["g"]):
        assert np.array_equal(bits(ctx.phase_eval(float(gv), g["wo"], g["wi"])), bits(g["hg_eval"][k]))
        d = np.abs(ctx.phase_sample(float(gv), g["wo"], g["u"]) - g["hg_sample"][k]).max(axis=1)
        assert d.max() <= 1e-4 and (d <= 1e-5).mean() >= 0.99
    med = abi.rbr_medium()
    med.sigma_a, med.sigma_s, med.g = abi.f3(g["medium"][0:3]), abi.f3(g["medium"][3:6]), float(g["medium"][6])
    got, want = ctx.medium_sample(med, g["max_dist"], g["u_medium"]), g["medium_sample"]
    same = got[:, 4] == want[:, 4]
    assert same.mean() >= 0.99
    np.testing.assert_allclose(got[same], want[same], rtol=2e-6, atol=1e-12)
    s = scenes.foggy_cornell_box()
    ctx.upload(s)
    n = 4096
    p = render_params(spp=n, max_depth=3, seed=23, flags=abi.RBR_RENDER_VOLUMETRIC)
    mean, m2 = ctx.render_host(camera(g["fog_camera"]), p, second_moment=True)
    tail, z_img = fog_z(mean, m2, n, g, True)
    assert tail < 0.015 and z_img < 3.0, (tail, z_img)


@pytest.mark.gpu
def test_gpu_film_export(ctx):
    g = load("golden_film.npz")
    for (t, e, gam), want in zip(g["modes"], g["rgb8"]):
        got = ctx.film_to_rgb8(g["film"], float(e), float(gam), bool(t))
        d = np.abs(got.astype(int) - want.astype(int))
        assert d.max() <= 1 and (d == 0).mean() >= 0.999
