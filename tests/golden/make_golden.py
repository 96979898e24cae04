"""Generates the golden fixtures in tests/golden/ from the reference library itself.

    python tests/golden/make_golden.py

Needs oracle/_ref/librbr_ref.so (the unmodified reference compiled from its own sources by
oracle/Makefile). Every expected value below is an output of the reference's code:
  golden_rays.npz     a seeded world (spheres, triangles, tilted quads, a plane) and 3000 rays;
                      brute-force closest hit (primitive index, t) and any hit
                      (the loop of tests/test_accelerators.cpp:58-74)
  golden_bsdf.npz     Material::createBSDF + evaluate/pdf/sample on the material grid of
                      tests/helpers.py (128 inputs per material)
  golden_lights.npz   AreaLight / PointLight ::sample
  golden_camera.npz   PinholeCamera / ThinLensCamera ::generateRay
  golden_mis.npz      sampling::powerHeuristic
  golden_cornell.npz  per-pixel mean and variance of PathTracingIntegrator::Li on the Cornell
                      box at 24x24, 2048 samples per pixel (independent seeds)
  golden_volume.npz   HenyeyGreensteinPhase::evaluate / sample, HomogeneousMedium::sampleDistance,
                      and per-pixel mean and variance of VolumetricPathIntegrator::Li on the
                      foggy Cornell box at 16x16, depth 3, 4096 samples per pixel
  golden_obj.npz      ObjImporter::parse + TriangleMesh::toPrimitives on small OBJ texts
  golden_film.npz     Film::toRGB8 / toRGB8ToneMapped of a seeded film
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO / "ray-based-rendering_b200"))
sys.path.insert(0, str(REPO / "oracle"))
sys.path.insert(0, str(HERE.parent))

import helpers  # noqa: E402
from oracle import Reference  # noqa: E402
from rbr_b200 import abi, render_params, scenes  # noqa: E402


def mat_params(m):
    return np.array(list(m.base_color) + [m.metallic, m.roughness, m.ior, m.transmission] + list(m.emission),
                    np.float32)


def light_params(l):
    return np.array([l.type] + list(l.position) + list(l.u) + list(l.v) + list(l.color) + [l.intensity], np.float32)


def camera_params(c):
    return np.array([c.width, c.height, c.model] + list(c.position) + list(c.forward) + list(c.right) + list(c.up)
                    + [c.fx, c.fy, c.cx, c.cy, c.lens_radius, c.focal_distance], np.float32)


def main():
    ref = Reference()
    # rays
    w = scenes.random_world(60, 200, True, seed=3, n_quads=20)
    rays = scenes.random_test_rays(3000, seed=33)
    h = ref.scene(w)
    hits = ref.trace_closest(h, rays, brute=True)
    occ = ref.trace_any(h, rays, brute=True)
    np.savez_compressed(HERE / "golden_rays.npz", triangles=w.triangles, triangle_ids=w.triangle_ids,
                        spheres=w.spheres, sphere_ids=w.sphere_ids, quads=w.quads, quad_ids=w.quad_ids,
                        planes=w.planes, plane_ids=w.plane_ids, rays=rays.view(np.uint8), prim=hits["prim"],
                        t=hits["t"], occluded=occ)
    # BSDFs
    names, params, wos, wis, us, evals, infos, samples = [], [], [], [], [], [], [], []
    for k, (name, m) in enumerate(helpers.material_grid()):
        wo, wi, u = helpers.bsdf_inputs(128, seed=100 + k)
        f, pdf, info = ref.bsdf_eval(m, wo, wi)
        names.append(name)
        params.append(mat_params(m))
        wos.append(wo)
        wis.append(wi)
        us.append(u)
        evals.append(np.concatenate([f, pdf[:, None]], 1))
        infos.append(info)
        samples.append(ref.bsdf_sample(m, wo, u))
    np.savez_compressed(HERE / "golden_bsdf.npz", names=np.array(names), params=np.array(params), wo=np.array(wos),
                        wi=np.array(wis), u=np.array(us), eval=np.array(evals), info=np.array(infos),
                        sample=np.array(samples))
    # lights
    p, u = helpers.light_points(256, seed=7)
    ls = helpers.lights()
    np.savez_compressed(HERE / "golden_lights.npz", params=np.array([light_params(l) for l in ls]), points=p, u=u,
                        out=np.array([ref.light_sample(l, p, u) for l in ls]))
    # cameras
    cams = [ref.camera(200, 100, (0, 1, 5), (0, 1, 0), (0, 1, 0), 40.0),
            ref.camera(200, 100, (0, 1, 5), (0, 1, 0), (0, 1, 0), 40.0, lens_radius=0.1, focal_distance=4.0)]
    s = helpers.camera_samples(cams[0], 256, seed=8)
    np.savez_compressed(HERE / "golden_camera.npz", params=np.array([camera_params(c) for c in cams]), samples=s,
                        out=np.array([ref.camera_rays(c, s) for c in cams]))
    # MIS
    pairs = helpers.mis_pairs()
    np.savez_compressed(HERE / "golden_mis.npz", pairs=pairs,
                        weights=np.array([ref.power_heuristic(1, float(a), 1, float(b)) for a, b in pairs], np.float32))
    # Cornell moments
    c = scenes.cornell_box()
    cam = scenes.look_at_camera(24, 24, (0.0, 1.0, 3.5), (0.0, 1.0, 0.0), (0.0, 1.0, 0.0), 40.0)
    c.camera = cam
    n = 2048
    acc = ref.render_moments(ref.scene(c), cam, render_params(spp=n, max_depth=8), batch=11)
    mean = acc[0] / n
    var = np.maximum(acc[1] / n - mean ** 2, 0) * n / (n - 1)
    np.savez_compressed(HERE / "golden_cornell.npz", mean=mean, var=var, n=np.array(n), camera=camera_params(cam))
    # participating medium
    gs = np.array([0.0, 0.0005, 0.5, -0.3, 0.9], np.float32)
    rng = np.random.default_rng(77)
    wo = helpers.unit_vectors(rng, 256)
    wi = helpers.unit_vectors(rng, 256)
    u2 = rng.random((256, 2), dtype=np.float32)
    med = abi.rbr_medium()
    med.sigma_a = abi.f3((0.02, 0.03, 0.01))
    med.sigma_s = abi.f3((0.08, 0.07, 0.09))
    med.g = 0.5
    md = np.where(rng.random(256) < 0.1, np.inf, rng.uniform(0.01, 40.0, 256)).astype(np.float32)
    um = rng.random(256, dtype=np.float32)
    fog = scenes.foggy_cornell_box()
    fcam = scenes.look_at_camera(16, 16, (0.0, 1.0, 3.5), (0.0, 1.0, 0.0), (0.0, 1.0, 0.0), 40.0)
    fog.camera = fcam
    nf = 4096
    facc = ref.render_moments(ref.scene(fog), fcam, render_params(spp=nf, max_depth=3), batch=13, volumetric=True)
    fmean = facc[0] / nf
    fvar = np.maximum(facc[1] / nf - fmean ** 2, 0) * nf / (nf - 1)
    np.savez_compressed(HERE / "golden_volume.npz", g=gs, wo=wo, wi=wi, u=u2,
                        hg_eval=np.array([ref.hg_eval(g, wo, wi) for g in gs]),
                        hg_sample=np.array([ref.hg_sample(g, wo, u2) for g in gs]),
                        medium=np.array(list(med.sigma_a) + list(med.sigma_s) + [med.g], np.float32),
                        max_dist=md, u_medium=um, medium_sample=ref.medium_sample(med, md, um),
                        fog_mean=fmean, fog_var=fvar, fog_n=np.array(nf), fog_camera=camera_params(fcam))
    # OBJ meshes
    import test_mesh_obj

    texts, verts, norms = [], [], []
    for name, text in test_mesh_obj.CASES.items():
        v, nn = ref.obj_triangles(text)
        texts.append(text)
        verts.append(v)
        norms.append(nn if nn is not None else np.zeros((0, 9), np.float32))
    np.savez_compressed(HERE / "golden_obj.npz", names=np.array(list(test_mesh_obj.CASES)),
                        texts=np.array(texts), **{f"v{i}": v for i, v in enumerate(verts)},
                        **{f"n{i}": nn for i, nn in enumerate(norms)})
    # film export
    film = (np.random.default_rng(9).random((48, 64, 3)) ** 3 * 4.0).astype(np.float32)
    modes = [(False, 1.0, 2.2), (True, 1.5, 2.2), (True, 0.25, 1.0)]
    np.savez_compressed(HERE / "golden_film.npz", film=film, modes=np.array(modes, np.float32),
                        rgb8=np.array([ref.film_rgb8(film, e, g, t) for t, e, g in modes]))
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
