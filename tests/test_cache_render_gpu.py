"""Path tracing with the radiance cache (rbr_cache_render) on small scenes: paths end into the
cache, training paths train it, and on the GGX scene the trained cache gives a lower RelMSE
against a converged render than the plain path tracer at the same number of samples."""
import numpy as np
import pytest
import torch

from rbr_b200 import render_params, scenes

pytestmark = pytest.mark.gpu


def relmse(x, ref):
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))


def small_ggx(w=192, h=108):
    s = scenes.ggx_scene(mesh_n=200)
    s.camera.width, s.camera.height = w, h
    s.camera.cx, s.camera.cy = w / 2, h / 2
    s.camera.fx *= w / 1920
    s.camera.fy *= h / 1080
    return s


def cached_render(ctx, cam, frames, depth, seed, train=True):
    film = torch.zeros(cam.width * cam.height * 3, device="cuda")
    ctx.cache_render_dev(cam, render_params(spp=1, max_depth=depth, seed=seed), frames, film.data_ptr(), 0, train)
    torch.cuda.synchronize()
    return film.cpu().numpy().reshape(cam.height, cam.width, 3)


def test_cache_render_trains_and_queries(ctx):
    s = scenes.cornell_box()
    s.camera = scenes.look_at_camera(64, 64, (0.0, 1.0, 3.5), (0.0, 1.0, 0.0), (0.0, 1.0, 0.0), 40.0)
    ctx.upload(s)
    ctx.cache_create(train_paths=512, seed=1)
    img = cached_render(ctx, s.camera, 8, 8, 5)
    info = ctx.cache_info()
    assert np.isfinite(img).all() and (img >= 0).all()
    assert info.optimiser_steps == 8 * 4
    # paths that leave the box or hit the light end without a query
    assert info.last_queries > 0.5 * (64 * 64 - 512) and info.last_train_records > 512
    assert np.isfinite(info.last_loss) and info.last_loss > 0
    # without training the parameters stay as they are
    before = ctx.cache_get_params()
    cached_render(ctx, s.camera, 2, 8, 6, train=False)
    assert np.array_equal(before, ctx.cache_get_params()) and ctx.cache_info().optimiser_steps == 8 * 4


def test_cache_beats_plain_at_equal_samples_on_ggx(ctx):
    s = small_ggx()
    ctx.upload(s)
    ref = ctx.render_host(s.camera, render_params(spp=1024, max_depth=16, seed=99))
    plain = ctx.render_host(s.camera, render_params(spp=64, max_depth=16, seed=5))
    ctx.cache_create(train_paths=(192 * 108) // 8, seed=1)
    cached = cached_render(ctx, s.camera, 64, 16, 5)
    r_plain, r_cache = relmse(plain, ref), relmse(cached, ref)
    assert r_cache < 0.7 * r_plain, (r_cache, r_plain)
    assert abs(cached.mean() / ref.mean() - 1.0) < 0.05


def test_two_waves_in_flight_gather_the_same_paths(ctx):
    """pt.streams 2 renders a cached frame as two half-image waves with their own query records
    and training lists: every frame ends the same paths into the cache and gathers the same
    training vertices as one wave at a time (only the order of the training list differs, so
    the trained cache and the image agree statistically, not bit for bit)."""
    s = small_ggx(96, 54)
    ctx.upload(s)
    out = {}
    try:
        for streams in (1, 2):
            ctx.set_param("pt.streams", streams)
            ctx.cache_create(train_paths=(96 * 54) // 8, seed=1)
            img = cached_render(ctx, s.camera, 16, 16, 5)
            info = ctx.cache_info()
            out[streams] = (img, info.last_queries, info.last_train_records, info.optimiser_steps)
    finally:
        ctx.set_param("pt.streams", 2)
    (a, qa, ta, sa), (b, qb, tb, sb) = out[1], out[2]
    assert qa == qb and ta == tb and sa == sb == 16 * 4
    assert np.isfinite(b).all() and (b >= 0).all()
    assert abs(b.mean() / a.mean() - 1.0) < 0.05


def test_self_training_suffix(ctx):
    """train_suffix k > 0 ends training paths into the cache k bounces after the termination
    depth: fewer training vertices and more queries per frame than full training paths
    (train_suffix 0), and an image of the same brightness."""
    s = small_ggx(96, 54)
    ctx.upload(s)
    out = {}
    for k in (0, 2):
        ctx.cache_create(train_paths=(96 * 54) // 8, seed=1, train_suffix=k)
        img = cached_render(ctx, s.camera, 16, 16, 5)
        info = ctx.cache_info()
        out[k] = (img, info.last_queries, info.last_train_records)
    (a, q0, t0), (b, q2, t2) = out[0], out[2]
    assert t2 < t0 and q2 > q0, (t0, t2, q0, q2)
    assert np.isfinite(b).all() and abs(b.mean() / a.mean() - 1.0) < 0.05


def test_spatially_sorted_queries_render_the_same_frame(ctx):
    """cache.sort_queries: the inference serves a wave's queries cell by cell; each query's
    prediction and its path's radiance are the same, so frames rendered without training agree
    (up to the order of the shadow rays' atomic sums)."""
    s = small_ggx()
    ctx.upload(s)
    ctx.cache_create(train_paths=(192 * 108) // 8, seed=3)
    cached_render(ctx, s.camera, 4, 16, 7)  # train a little first
    try:
        ctx.set_param("cache.sort_queries", 0)
        a = cached_render(ctx, s.camera, 2, 16, 8, train=False)
        ctx.set_param("cache.sort_queries", 1)
        b = cached_render(ctx, s.camera, 2, 16, 8, train=False)
    finally:
        ctx.set_param("cache.sort_queries", 0)
    assert np.isfinite(b).all()
    np.testing.assert_allclose(b, a, rtol=1e-4, atol=1e-5)
