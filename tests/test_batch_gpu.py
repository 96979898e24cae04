"""Batched request loop (rbr_batch_*): requests of several scenes, resolutions, sample counts,
depths and integrators packed into shared waves give the same images as rendering each request
alone with rbr_render (the same random numbers per (pixel, sample, seed)), whether the waves
are replayed from captured CUDA graphs, launched directly, or rendered by one persistent
cooperative launch, however a request is split over waves, and with staggered arrival times;
per-request latency (from arrival, on the device clock) and batch statistics are reported."""
import numpy as np
import pytest
import torch

from rbr_b200 import Batch, Context, RbrError, abi, render_params, scenes

pytestmark = pytest.mark.gpu


def small_ggx(w, h, seed=0):
    s = scenes.ggx_scene(width=w, height=h, mesh_n=60, seed=seed)
    return s


def cornell(w, h):
    s = scenes.cornell_box()
    s.camera = scenes.look_at_camera(w, h, (0.0, 1.0, 3.5), (0.0, 1.0, 0.0), (0.0, 1.0, 0.0), 40.0)
    return s


def foggy(w, h):
    s = scenes.foggy_cornell_box()
    s.camera = scenes.look_at_camera(w, h, (0.0, 1.0, 3.5), (0.0, 1.0, 0.0), (0.0, 1.0, 0.0), 40.0)
    return s


@pytest.fixture(scope="module")
def bctx():
    c = Context(0)
    yield c
    c.close()


def requests():
    """(scene key, width, height, params) of a mixed set of requests."""
    vol = abi.RBR_RENDER_VOLUMETRIC
    return [
        ("cornell", 48, 40, render_params(spp=3, max_depth=8, seed=11)),
        ("ggx", 64, 36, render_params(spp=5, max_depth=16, seed=12, sample_offset=7)),
        ("cornell", 32, 32, render_params(spp=1, max_depth=3, seed=13, use_mis=False)),
        ("fog", 40, 40, render_params(spp=4, max_depth=6, seed=14, flags=vol)),
        ("ggx", 50, 30, render_params(spp=2, max_depth=5, seed=15, use_nee=False)),
        ("cornell", 20, 70, render_params(spp=9, max_depth=8, seed=16)),
        ("fog", 24, 24, render_params(spp=2, max_depth=3, seed=17, flags=vol)),
    ]


def build_scenes():
    return {"cornell": cornell, "ggx": small_ggx, "fog": foggy}


def alone(ctx, key, w, h, p):
    s = build_scenes()[key](w, h)
    ctx.upload(s)
    return ctx.render_host(s.camera, p)


def batched(ctx, arrivals=None, **cfg):
    b = Batch(ctx, **cfg)
    ids = {}
    for key, fn in build_scenes().items():
        ids[key] = b.add_scene(fn(16, 16))
    films, rids = [], []
    for i, (key, w, h, p) in enumerate(requests()):
        cam = build_scenes()[key](w, h).camera
        f = torch.zeros(w * h * 3, device="cuda")
        films.append(f)
        rids.append(b.submit(ids[key], cam, p, f.data_ptr(), arrival_us=0 if arrivals is None else arrivals[i]))
    b.run()
    torch.cuda.synchronize()
    stats = [b.request_stats(r) for r in rids]
    return b, [f.cpu().numpy().reshape(h, w, 3) for f, (_, w, h, _) in zip(films, requests())], stats


@pytest.mark.parametrize("cfg", [dict(), dict(use_graphs=0), dict(wave_paths=4096), dict(wave_paths=1000, blocks_per_sm=2),
                                 dict(wave_paths=4096, waves_in_flight=1), dict(persistent=1),
                                 dict(persistent=1, wave_paths=1000)],
                         ids=["graphs", "direct", "small-waves", "split-requests", "one-wave-in-flight", "persistent",
                              "persistent-split-requests"])
def test_packed_requests_equal_single_renders(bctx, cfg):
    b, films, stats = batched(bctx, **cfg)
    for (key, w, h, p), got in zip(requests(), films):
        want = alone(bctx, key, w, h, p)
        assert np.isfinite(got).all()
        np.testing.assert_allclose(got, want, rtol=2e-5, atol=2e-6, err_msg=key)
    bs = b.stats()
    assert bs.requests == len(requests()) and bs.waves >= 3  # three scenes x modes at least
    assert bs.paths == sum(w * h * p.samples_per_pixel for _, w, h, p in requests())
    if cfg.get("persistent"):
        assert bs.persistent_launches == 1 and bs.kernel_launches == 1 and bs.graph_launches == 0
    elif cfg.get("use_graphs", 1):
        assert bs.graph_launches == bs.waves and 1 <= bs.graphs_captured <= bs.waves and bs.persistent_launches == 0
    lat = [s.latency_ms for s in stats]
    assert all(s.latency_ms > 0 and s.start_ms <= s.latency_ms for s in stats)
    assert max(lat) <= bs.milliseconds + 0.01
    if cfg.get("wave_paths") == 1000:
        assert any(s.waves > 1 for s in stats)  # a request spread over several waves
    b.close()


def test_graph_replay_across_runs_and_autotune(bctx):
    b = Batch(bctx)
    sid = b.add_scene(cornell(16, 16))
    cam = cornell(64, 64).camera
    f = torch.zeros(64 * 64 * 3, device="cuda")
    p = render_params(spp=4, max_depth=8, seed=3)
    for _ in range(3):
        b.submit(sid, cam, p, f.data_ptr())
        b.run()
    st = b.stats()
    assert st.graphs_captured == 0 and st.graph_launches == st.waves  # replayed from the first run
    first = f.cpu().numpy().copy()
    b.submit(sid, cam, p, f.data_ptr())
    b.autotune()
    b.run()
    torch.cuda.synchronize()
    np.testing.assert_allclose(f.cpu().numpy(), first, rtol=2e-5, atol=2e-6)
    st = b.stats()
    assert st.wave_paths in (1 << 20, 1 << 21, 1 << 22, 1 << 23) and st.blocks_per_sm in (4, 8, 16)
    b.close()


def test_cached_requests_in_a_batch(bctx):
    b = Batch(bctx)
    sid = b.add_scene(small_ggx(16, 16))
    b.cache_create(sid, train_paths=4096, seed=1)
    cam = small_ggx(96, 54).camera
    films = [torch.zeros(96 * 54 * 3, device="cuda") for _ in range(4)]
    for i, f in enumerate(films):
        b.submit(sid, cam, render_params(spp=1, max_depth=16, seed=5, sample_offset=i), f.data_ptr(),
                 use_cache=True, train_cache=True)
    b.run()
    torch.cuda.synchronize()
    for f in films:
        img = f.cpu().numpy()
        assert np.isfinite(img).all() and (img >= 0).all() and img.mean() > 0
    assert b.stats().waves == 1


def test_invalid_requests_are_rejected(bctx):
    from rbr_b200 import RbrError

    b = Batch(bctx)
    sid = b.add_scene(cornell(16, 16))
    cam = cornell(8, 8).camera
    f = torch.zeros(8 * 8 * 3, device="cuda")
    with pytest.raises(RbrError):
        b.submit(sid + 5, cam, render_params(spp=1), f.data_ptr())
    with pytest.raises(RbrError):
        b.submit(sid, cam, render_params(spp=1, max_depth=0), f.data_ptr())
    with pytest.raises(RbrError):
        b.submit(sid, cam, render_params(spp=1), f.data_ptr(), use_cache=True)  # no cache on the scene
    with pytest.raises(RbrError):
        b.submit(sid, cam, render_params(spp=1, flags=abi.RBR_RENDER_SECOND_MOMENT), f.data_ptr())


def test_scene_variants_share_geometry(bctx):
    """A variant (other materials and lights on the base scene's resident BVH) renders what a
    full upload of the variant renders."""
    base = small_ggx(16, 16)
    var = scenes.ggx_variant(base, 3)
    b = Batch(bctx)
    bid = b.add_scene(base)
    vid = b.add_scene_variant(bid, var)
    cam = small_ggx(64, 48).camera
    f = torch.zeros(64 * 48 * 3, device="cuda")
    p = render_params(spp=4, max_depth=8, seed=21)
    b.submit(vid, cam, p, f.data_ptr())
    b.run()
    torch.cuda.synchronize()
    var.camera = cam
    bctx.upload(var)
    want = bctx.render_host(cam, p)
    np.testing.assert_allclose(f.cpu().numpy().reshape(48, 64, 3), want, rtol=2e-5, atol=2e-6)
    base.camera = cam
    bctx.upload(base)
    assert not np.allclose(bctx.render_host(cam, p), want)
    b.close()


@pytest.mark.parametrize("persistent", [0, 1], ids=["graphs", "persistent"])
def test_staggered_arrivals(bctx, persistent):
    """Requests arriving over 30 ms (seeded): the same images; no request's wave starts before
    it arrives, so the run lasts past the last arrival; latency counts from the arrival."""
    rng = np.random.default_rng(41)
    arrivals = np.sort(rng.integers(0, 30000, len(requests()))).tolist()
    arrivals = list(rng.permutation(arrivals))  # submitted out of arrival order
    b, films, stats = batched(bctx, arrivals=arrivals, persistent=persistent)
    for (key, w, h, p), got in zip(requests(), films):
        np.testing.assert_allclose(got, alone(bctx, key, w, h, p), rtol=2e-5, atol=2e-6, err_msg=key)
    bs = b.stats()
    assert bs.milliseconds >= max(arrivals) / 1000.0
    assert all(s.latency_ms > 0 and 0 <= s.start_ms <= s.latency_ms for s in stats)
    # a request is done within its arrival plus the whole run
    assert all(a / 1000.0 + s.latency_ms <= bs.milliseconds + 0.01 for a, s in zip(arrivals, stats))
    b.close()


def test_persistent_barrier_wait_runs_out_and_recovers(bctx):
    """A grid-barrier limit of 1 us makes the persistent run's barrier waits give up: the run
    reports RBR_ERR_DEVICE_TIMEOUT (every block leaves the kernel, nothing waits without bound)
    and the same context renders correctly afterwards."""
    from rbr_b200 import RbrError

    b = Batch(bctx, persistent=1, barrier_timeout_us=1)
    sid = b.add_scene(cornell(16, 16))
    cam = cornell(64, 64).camera
    f = torch.zeros(64 * 64 * 3, device="cuda")
    p = render_params(spp=4, max_depth=8, seed=3)
    b.submit(sid, cam, p, f.data_ptr())
    b.run()
    with pytest.raises(RbrError) as e:
        b.stats()
    assert e.value.status == abi.RBR_ERR_DEVICE_TIMEOUT
    b.close()
    b = Batch(bctx, persistent=1)
    sid = b.add_scene(cornell(16, 16))
    b.submit(sid, cam, p, f.data_ptr())
    b.run()
    torch.cuda.synchronize()
    assert b.stats().persistent_launches == 1
    np.testing.assert_allclose(f.cpu().numpy().reshape(64, 64, 3), alone(bctx, "cornell", 64, 64, p), rtol=2e-5,
                               atol=2e-6)
    b.close()



@pytest.mark.parametrize("cfg", [dict(), dict(wave_paths=1000), dict(persistent=1)],
                         ids=["graphs", "split-requests", "persistent"])
def test_host_films_arrive_after_the_run(bctx, cfg):
    """rbr_batch_set_host_film: the run copies each registered request's film to its
    page-locked host buffer after the request's last wave; the host copy equals the device
    film, requests without a host buffer are untouched, and an unknown request id is rejected."""
    b = Batch(bctx, **cfg)
    ids = {key: b.add_scene(fn(16, 16)) for key, fn in build_scenes().items()}
    films, hosts, rids = [], [], []
    for i, (key, w, h, p) in enumerate(requests()):
        cam = build_scenes()[key](w, h).camera
        f = torch.zeros(w * h * 3, device="cuda")
        films.append(f)
        rid = b.submit(ids[key], cam, p, f.data_ptr())
        rids.append(rid)
        if i % 2 == 0:  # every other request gets a host buffer
            hb = torch.full((w * h * 3,), -1.0).pin_memory()
            b.set_host_film(rid, hb.data_ptr())
            hosts.append(hb)
        else:
            hosts.append(None)
    with pytest.raises(RbrError):
        b.set_host_film(max(rids) + 100, hosts[0].data_ptr())
    b.run()
    torch.cuda.synchronize()
    for f, hb in zip(films, hosts):
        if hb is not None:
            assert torch.equal(hb, f.cpu())
    b.close()


def test_host_film_of_a_request_over_many_waves(bctx):
    """A request spread over many waves on both stream slots: its host copy waits for the waves
    of the other slot too, so it equals the device film (and a single render)."""
    b = Batch(bctx, wave_paths=1 << 15)
    sid = b.add_scene(cornell(16, 16))
    w, h, p = 192, 160, render_params(spp=8, max_depth=8, seed=21)
    cam = cornell(w, h).camera
    f = torch.zeros(w * h * 3, device="cuda")
    rid = b.submit(sid, cam, p, f.data_ptr())
    hb = torch.full((w * h * 3,), -1.0).pin_memory()
    b.set_host_film(rid, hb.data_ptr())
    b.run()
    torch.cuda.synchronize()
    assert b.request_stats(rid).waves >= 6
    assert torch.equal(hb, f.cpu())
    np.testing.assert_allclose(hb.numpy().reshape(h, w, 3), alone(bctx, "cornell", w, h, p), rtol=2e-5, atol=2e-6)
    b.close()
