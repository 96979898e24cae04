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
    wo, wi, _ = helpers.bsdf_inputs(8192, seed=helpers.name_seed(name, 997))
    got = ctx.bsdf_eval(mat, wo, wi)
    f, pdf, info = reference.bsdf_eval(mat, wo, wi)
    assert np.array_equal(bits(got[:, :3]), bits(f)), "BSDF values"
    assert np.array_equal(bits(got[:, 3]), bits(pdf)), "pdfs"
    assert (got[:, 4] == info[0]).all() and (got[:, 5] == info[1]).all(), "isDelta / type bits"


@pytest.mark.parametrize("name,mat", GRID, ids=[n for n, _ in GRID])
def test_bsdf_eval_pdf_edge_directions(ctx, reference, name, mat):
    """Direction pairs where the checks inside evaluate() and pdf() decide: wi = -wo (the
    reflection half vector vanishes), a direction on the horizon (cos = 0), normal incidence
    into both hemispheres, wi = wo. The one-pass value and pdf equal the reference's two calls."""
    wo, wi = helpers.edge_directions()
    got = ctx.bsdf_eval(mat, wo, wi)
    f, pdf, _ = reference.bsdf_eval(mat, wo, wi)
    assert np.array_equal(bits(got[:, :3]), bits(f)) and np.array_equal(bits(got[:, 3]), bits(pdf))


def check_samples(ctx_or_none, reference, mat, wo, got, want, min_close=0.99):
    """Well-posed comparison of BSDF::sample outputs (8 floats each) from two implementations
    whose sin/cos may differ in the last bit:
      - the same samples are valid (pdf > 0) on both sides, up to 0.1 %;
      - sampled directions agree within 1e-5 (unit vectors) for all but 0.1 % of the samples and
        within 1e-3 for all (refraction close to total internal reflection magnifies an ulp of
        sin/cos);
      - every non-delta GPU sample carries exactly (bit for bit) the reference's
        evaluate() and pdf() at the GPU's own direction;
      - f and pdf agree within 1e-5 relative for at least `min_close` of the samples (sharp GGX
        lobes, alpha down to 1e-3, turn a 1e-7 change of direction into a large change of value:
        two accurate CPU libraries disagree there too);
      - delta samples are bit-exact."""
    vg, vw = got[:, 6] > 0, want[:, 6] > 0
    assert (vg == vw).mean() >= 0.999
    both = vg & vw
    dev = np.abs(got[both, :3] - want[both, :3]).max(axis=1, initial=0.0)
    assert dev.max(initial=0.0) <= 1e-3
    assert (dev <= 1e-5).mean() >= 0.999 if both.any() else True
    nd = vg & (got[:, 7] == 0)
    if nd.any():
        f, pdf, _ = reference.bsdf_eval(mat, wo[nd], got[nd, :3])
        assert np.array_equal(bits(got[nd, 3:6]), bits(f)) and np.array_equal(bits(got[nd, 6]), bits(pdf))
    close = np.isclose(got[both, 3:7], want[both, 3:7], rtol=1e-5, atol=0.0).all(axis=1)
    if both.any():  # materials without lobes (black, lights) produce no samples at all
        assert close.mean() >= min_close, f"{(~close).sum()} of {both.sum()} samples beyond 1e-5"
    delta = both & (got[:, 7] == 1) & (want[:, 7] == 1)
    assert np.array_equal(bits(got[delta]), bits(want[delta]))


@pytest.mark.parametrize("name,mat", GRID, ids=[n for n, _ in GRID])
def test_bsdf_sample_matches_reference(ctx, reference, name, mat):
    wo, _, u = helpers.bsdf_inputs(8192, seed=helpers.name_seed(name, 991))
    check_samples(ctx, reference, mat, wo, ctx.bsdf_sample(mat, wo, u), reference.bsdf_sample(mat, wo, u))


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


def test_l2_read_bandwidth(ctx):
    """The L2 roofline's denominator: a 32 MiB buffer read from L2 is faster than any HBM copy
    (B200: about 6.5 TB/s), and sizes outside 4 KiB..1 GiB are refused."""
    from rbr_b200 import RbrError

    bw = ctx.l2_read_bandwidth(32 << 20, 20)
    assert 7000.0 < bw < 100000.0, bw
    with pytest.raises(RbrError):
        ctx.l2_read_bandwidth(1024, 20)
