"""Meshes read from OBJ text through the GPU path, and the film exported to 8-bit RGB on the
device, against the CPU restatement / the reference's Film."""
import numpy as np
import pytest

from rbr_b200 import abi, parse_obj, render_params, scenes
from test_trace_gpu import assert_same_closest

pytestmark = pytest.mark.gpu


def icosphere_obj(level=3, radius=2.0, quads=True):
    """OBJ text of an icosphere with vertex normals, some faces merged into quads (fan
    triangulation), negative indices on half of the faces."""
    v, f = scenes.icosphere(level)
    lines = [f"v {x * radius:.7g} {y * radius:.7g} {z * radius:.7g}" for x, y, z in v]
    lines += [f"vn {x:.7g} {y:.7g} {z:.7g}" for x, y, z in v]
    nv = len(v)
    i = 0
    while i < len(f):
        a, b, c = (int(x) + 1 for x in f[i])
        if i % 2:
            a, b, c = a - nv - 1, b - nv - 1, c - nv - 1  # negative (relative) indices
        lines.append(f"f {a}//{a} {b}//{b} {c}//{c}")
        i += 1
    return "\n".join(lines) + "\n"


def test_obj_mesh_traced_on_gpu_matches_bruteforce(ctx, restatement):
    verts, normals = parse_obj(icosphere_obj())
    assert normals is not None and len(verts) == 20 * 4 ** 3
    s = scenes.Scene()
    mat = s.diffuse((0.7, 0.7, 0.7))
    s.add_mesh(verts, normals, mat)
    lo, hi = scenes.scene_bounds(s)
    rays = scenes.uniform_rays(20000, lo - 1.0, hi + 1.0, seed=4)
    ctx.upload(s)
    assert_same_closest(ctx.trace_host(rays), restatement.trace_closest(restatement.scene(s), rays))
    # the interpolated normals reach the path tracer: a render sees them
    s.area_light((0, 4, 0), (1, 0, 0), (0, 0, 1), (5, 5, 5))
    s.camera = scenes.look_at_camera(32, 32, (0, 0, 6), (0, 0, 0), (0, 1, 0), 40.0)
    ctx.upload(s)
    p = render_params(spp=1, max_depth=3, seed=2)
    gpu = ctx.render_host(s.camera, p)
    cpu = restatement.render(restatement.scene(s), s.camera, p)
    assert np.isclose(gpu, cpu, rtol=1e-4, atol=1e-5).all(-1).mean() > 0.99


@pytest.mark.parametrize("tonemap,exposure,gamma", [(False, 1.0, 2.2), (True, 1.5, 2.2), (True, 0.25, 1.0),
                                                    (False, 1.0, 1.8)])
def test_film_export_matches_reference(ctx, reference, tonemap, exposure, gamma):
    """Film::toRGB8 / toRGB8ToneMapped on the device: the 8-bit values equal the reference's
    except where pow() lands within an ulp of a quantisation step (at most one level)."""
    rng = np.random.default_rng(9)
    film = (rng.random((96, 128, 3)) ** 3 * 4.0).astype(np.float32)
    film[0, :8] = np.array([0.0, 1.0, 1.0000001, 0.9999999, 1e-30, 7.0, 0.5, 2.0 ** -20], np.float32)[:, None]
    film[1, :3] = -0.25  # negative radiance clamps to 0
    got = ctx.film_to_rgb8(film, exposure, gamma, tonemap)
    want = reference.film_rgb8(film, exposure, gamma, tonemap)
    d = np.abs(got.astype(int) - want.astype(int))
    assert d.max() <= 1 and (d == 0).mean() >= 0.999
