"""Shared inputs for the unit-parity tests and the golden-fixture script."""
from __future__ import annotations

import zlib

import numpy as np

from rbr_b200 import abi

F32 = np.float32


def name_seed(name: str, modulus: int) -> int:
    """A seed derived from a test-case name that is the same in every process (str hashes are
    salted per process)."""
    return zlib.crc32(name.encode()) % modulus


def material(base=(0.8, 0.8, 0.8), metallic=0.0, roughness=1.0, ior=1.5, transmission=0.0, emission=(0, 0, 0)):
    m = abi.rbr_material()
    m.base_color = abi.f3(base)
    m.metallic = metallic
    m.roughness = roughness
    m.ior = ior
    m.transmission = transmission
    m.emission = abi.f3(emission)
    return m


def material_grid():
    """Materials covering every branch of Material::createBSDF (material.cpp:69-108): the presets
    of material.cpp:9-55 and of the reference's tests/test_materials.cpp:197-209, the smooth /
    rough boundary (roughness 0.03), partial metal and transmission, index 1, black, emissive."""
    return [
        ("diffuse", material((0.7, 0.7, 0.7), roughness=1.0, ior=1.0)),
        ("plastic", material((0.7, 0.7, 0.7), roughness=0.3)),
        ("rough plastic", material((0.7, 0.5, 0.3), roughness=0.8)),
        ("smooth plastic", material((0.7, 0.7, 0.7), roughness=0.0)),
        ("rough metal", material((0.9, 0.7, 0.4), metallic=1.0, roughness=0.4)),
        ("mirror", material((0.9, 0.9, 0.9), metallic=1.0, roughness=0.0)),
        ("half metal", material((0.8, 0.8, 0.8), metallic=0.5, roughness=0.3)),
        ("glass", material((1, 1, 1), roughness=0.0, transmission=1.0)),
        ("rough glass", material((1, 1, 1), roughness=0.3, transmission=1.0)),
        ("tinted rough glass", material((0.5, 0.9, 0.8), roughness=0.6, transmission=1.0)),
        ("half transmissive", material((0.5, 0.9, 0.8), roughness=0.5, transmission=0.4)),
        ("almost smooth", material((0.2, 0.3, 0.4), roughness=0.0299, transmission=0.5)),
        ("just rough", material((0.2, 0.3, 0.4), roughness=0.0301, transmission=0.5)),
        ("pass-through", material((0.2, 0.3, 0.4), roughness=0.5, ior=1.0, transmission=0.5)),
        ("metal glass mix", material((0.6, 0.6, 0.9), metallic=0.3, roughness=0.2, transmission=0.7)),
        ("dense glass", material((1, 1, 1), roughness=0.15, ior=2.4, transmission=1.0)),
        ("black", material((0, 0, 0), roughness=0.5)),
        ("emissive", material((0, 0, 0), ior=1.0, emission=(15, 15, 15))),
        ("alpha floor", material((0.9, 0.9, 0.9), metallic=1.0, roughness=0.031)),
    ]


def unit_dirs(n, rng, z_sign=0):
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    if z_sign:
        v[:, 2] = np.abs(v[:, 2]) * z_sign
    return v.astype(F32)


def bsdf_inputs(n, seed):
    """wo, wi on the whole sphere plus grazing and normal-incidence cases, and uniforms u."""
    rng = np.random.default_rng(seed)
    wo = unit_dirs(n, rng)
    wi = unit_dirs(n, rng)
    wo[:8] = [[0, 0, 1], [0, 0, -1], [1, 0, 0], [0.6, 0.0, 0.8], [0.6, 0.0, -0.8], [0.999, 0, 0.0447],
              [0, 0.1, 0.995], [0.3, -0.3, 0.9055]]
    wi[:8] = [[0, 0, 1], [0, 0, 1], [0, 0, 1], [-0.6, 0.0, 0.8], [-0.6, 0.0, 0.8], [0.0, 0.999, 0.0447],
              [0, 0, -1], [-0.3, 0.3, 0.9055]]
    u = rng.random((n, 2), dtype=F32)
    u[:4] = [[0, 0], [0.99999994, 0.99999994], [0.5, 0.5], [0.25, 0.75]]
    return np.ascontiguousarray(wo, F32), np.ascontiguousarray(wi, F32), np.ascontiguousarray(u, F32)


def edge_directions():
    """(wo, wi) pairs on which the checks inside BSDF evaluate() and pdf() decide: wi = -wo,
    a direction on the horizon, normal incidence into either hemisphere, wi = wo."""
    wo = [[0.6, 0.0, 0.8], [0.0, 0.0, 1.0], [1.0, 0.0, 0.0], [0.6, 0.0, -0.8], [0.0, 0.6, 0.8], [0.28, 0.96, 0.0],
          [0.0, 0.0, -1.0], [0.8, 0.0, 0.6]]
    wi = [[-0.6, 0.0, -0.8], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0], [-0.6, 0.0, 0.8], [0.0, -0.6, -0.8], [0.0, 0.0, -1.0],
          [0.0, 0.0, -1.0], [0.8, 0.0, 0.6]]
    return np.ascontiguousarray(wo, F32), np.ascontiguousarray(wi, F32)


def lights():
    out = []
    for (t, pos, u, v, col, inten) in [
        (abi.RBR_LIGHT_AREA, (0.0, 1.99, 0.0), (0.5, 0, 0), (0, 0, 0.5), (17, 12, 4), 1.0),
        (abi.RBR_LIGHT_AREA, (1.0, 3.0, -2.0), (0.3, 0.4, 0.0), (0.0, 0.2, 1.1), (1, 2, 3), 2.5),
        (abi.RBR_LIGHT_POINT, (0.0, 1.8, 0.5), (0, 0, 0), (0, 0, 0), (1, 1, 1), 2.0),
    ]:
        l = abi.rbr_light()
        l.type = t
        l.position = abi.f3(pos)
        l.u = abi.f3(u)
        l.v = abi.f3(v)
        l.color = abi.f3(col)
        l.intensity = inten
        out.append(l)
    return out


def light_points(n, seed):
    rng = np.random.default_rng(seed)
    p = rng.uniform(-2.0, 2.0, (n, 3)).astype(F32)
    u = rng.random((n, 2), dtype=F32)
    return p, u


def camera_samples(cam, n, seed):
    rng = np.random.default_rng(seed)
    s = np.empty((n, 4), F32)
    s[:, 0] = rng.uniform(0, cam.width, n)
    s[:, 1] = rng.uniform(0, cam.height, n)
    s[:, 2:] = rng.random((n, 2))
    s[:4] = [[0, 0, 0.5, 0.5], [cam.width / 2, cam.height / 2, 0.5, 0.5], [cam.width, cam.height, 0.0, 1.0],
             [0.5, 0.5, 0.25, 0.75]]
    return s


def mis_pairs():
    inf = np.inf
    base = [(1.0, 1.0), (inf, 1.0), (1.0, inf), (0.0, 0.0), (1e30, 1e30), (0.0, 1.0), (1.0, 0.0), (3.5, 0.25),
            (1e-30, 1e-30), (2.0, 7.0)]
    rng = np.random.default_rng(3)
    extra = rng.lognormal(0, 3, (200, 2))
    return np.concatenate([np.array(base), extra]).astype(F32)


def unit_vectors(rng, n):
    v = rng.normal(size=(n, 3))
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(F32)


def ggx_small(width=64, height=36, mesh_n=60):
    """The GGX material scene (rbr_b200.scenes.ggx_scene: 256 spheres of random materials with
    20 % glass, rough metals and rough dielectrics, a mound mesh on a ground quad, two quad area
    lights with coincident emissive quads, a point light, a thin-lens camera) on a reduced film
    and mesh, plus four spheres in front of the mound with the smooth (delta-lobe) materials the
    random draw never produces (roughness below 0.03): clear glass, a mirror, smooth plastic and a
    smooth half-transmissive dielectric."""
    from rbr_b200 import scenes

    s = scenes.ggx_scene(width=width, height=height, mesh_n=mesh_n, seed=0)
    extra = [((-2.2, 0.6, 6.0, 0.6), dict(base_color=(1, 1, 1), roughness=0.0, ior=1.5, transmission=1.0)),
             ((-0.7, 0.5, 7.0, 0.5), dict(base_color=(0.9, 0.9, 0.9), metallic=1.0, roughness=0.0)),
             ((0.8, 0.5, 7.0, 0.5), dict(base_color=(0.2, 0.4, 0.8), roughness=0.0, ior=1.5)),
             ((2.3, 0.6, 6.0, 0.6), dict(base_color=(0.8, 0.9, 0.7), roughness=0.0, ior=1.5, transmission=0.5))]
    sph, mats = list(s.spheres), list(s.sphere_materials)
    for geom, m in extra:
        sph.append(geom)
        mats.append(s.add_material(**m))
    s.spheres = np.asarray(sph, F32)
    s.sphere_materials = np.asarray(mats, np.uint32)
    return s


def moments_z(S1, Q1, n1, S2, Q2, n2):
    """Per-pixel-channel z scores of two sets of sample moments (sums and sums of squares of n1
    and n2 independent samples), and the z score of the difference of their image means."""
    mu1, mu2 = S1 / n1, S2 / n2
    var1 = np.maximum(Q1 / n1 - mu1 ** 2, 0) * n1 / (n1 - 1)
    var2 = np.maximum(Q2 / n2 - mu2 ** 2, 0) * n2 / (n2 - 1)
    se = np.sqrt(var1 / n1 + var2 / n2)
    z = np.abs(mu1 - mu2) / np.maximum(se, 1e-12)
    z[(se == 0) & (np.abs(mu1 - mu2) < 1e-6)] = 0
    m = mu1.size
    z_img = abs(mu1.mean() - mu2.mean()) / max(np.sqrt((var1 / n1 + var2 / n2).sum()) / m, 1e-12)
    return z, z_img


def crop_camera(cam, x0, y0, width, height):
    """The pixels [x0, x0 + width) x [y0, y0 + height) of `cam`'s film as a camera of their own:
    the same rays per pixel, principal point shifted by the crop origin."""
    import ctypes as C

    c = abi.rbr_camera()
    C.memmove(C.byref(c), C.byref(cam), C.sizeof(cam))
    c.width, c.height = width, height
    c.cx = cam.cx - x0
    c.cy = cam.cy - y0
    return c

