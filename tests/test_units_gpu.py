"""The path tracer's device functions against the reference's CPU code on identical inputs.

BSDF values and densities, light samples, pinhole camera rays and MIS weights are exactly
rounded restatements: bit-identical. Sampling routines that call cosf/sinf (Lambertian cosine
sampling, GGX visible-normal sampling, thin-lens disk sampling) may differ by an ulp of those
functions; they must agree within 1e-5 relative (the bar the parity target states).
"""
import numpy as np
import pytest

import helpers

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


GRID = helpers.material_grid()


@pytest.mark.parametrize("name,mat", GRID, ids=[n for n, _ in GRID])
def test_bsdf_eval_pdf_bit_exact(ctx, reference, name, mat):
    wo, wi, _ = helpers.bsdf_inputs(8192, seed=hash(name) % 997)
    got = ctx.bsdf_eval(mat, wo, wi)
    f, pdf, info = reference.bsdf_eval(mat, wo, wi)
    assert np.array_equal(bits(got[:, :3]), bits(f)), "BSDF values"
    assert np.array_equal(bits(got[:, 3]), bits(pdf)), "pdfs"
    assert (got[:, 4] == info[0]).all() and (got[:, 5] == info[1]).all(), "isDelta / type bits"


@pytest.mark.parametrize("name,mat", GRID, ids=[n for n, _ in GRID])
def test_bsdf_sample_within_1e5(ctx, reference, name, mat):
    wo, _, u = helpers.bsdf_inputs(8192, seed=hash(name) % 991)
    got = ctx.bsdf_sample(mat, wo, u)
    want = reference.bsdf_sample(mat, wo, u)
    close = np.isclose(got, want, rtol=1e-5, atol=1e-6).all(axis=1)
    # an ulp of cosf/sinf can flip a sample across a hemisphere test at grazing angles
    assert close.mean() >= 0.999, f"{(~close).sum()} of {len(close)} samples differ; first {np.flatnonzero(~close)[:5]}"
    exact = (bits(got) == bits(want)).all(axis=1)
    if mat.metallic == 1.0 and mat.roughness == 0.0:  # delta lobes: no transcendental involved
        assert exact.all()


def test_light_samples_bit_exact(ctx, reference):
    p, u = helpers.light_points(8192, seed=14)
    for l in helpers.lights():
        assert np.array_equal(bits(ctx.light_sample(l, p, u)), bits(reference.light_sample(l, p, u)))


def test_camera_rays(ctx, reference):
    pin = reference.camera(256, 192, (0, 1, 3.5), (0, 1, 0), (0, 1, 0), 40.0)
    s = helpers.camera_samples(pin, 8192, seed=15)
    assert np.array_equal(bits(ctx.camera_rays(pin, s)), bits(reference.camera_rays(pin, s)))
    thin = reference.camera(256, 192, (0, 3, 14), (0, 0.8, 0), (0, 1, 0), 40.0, lens_radius=0.05,
                            focal_distance=14.2)
    got, want = ctx.camera_rays(thin, s), reference.camera_rays(thin, s)
    assert np.allclose(got, want, rtol=1e-5, atol=1e-6)


def test_mis_weights_bit_exact(ctx, reference):
    pairs = helpers.mis_pairs()
    got = ctx.mis_weights(pairs)
    want = np.array([reference.power_heuristic(1, float(a), 1, float(b)) for a, b in pairs], np.float32)
    assert np.array_equal(bits(got), bits(want))
