"""GPU ray queries (rbr_trace_*) against the CPU oracle and the reference library.

Closest hit must equal the brute-force loop over the primitives bit for bit (primitive id and
the bits of t); any hit must equal the brute-force any-hit answer. Worlds and rays have the
shape of the reference's accelerator tests (tests/test_accelerators.cpp:37-105).
"""
import numpy as np
import pytest

from rbr_b200 import RbrError, abi, scenes

pytestmark = pytest.mark.gpu

MISS = abi.RBR_MISS


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def assert_same_closest(got, want):
    miss_g, miss_w = got["prim"] == MISS, want["prim"] == MISS
    assert np.array_equal(miss_g, miss_w), f"hit/miss differs on {np.sum(miss_g != miss_w)} rays"
    hit = ~miss_w
    bad = np.flatnonzero(got["prim"][hit] != want["prim"][hit])
    assert bad.size == 0, f"{bad.size} primitive ids differ"
    assert np.array_equal(bits(got["t"][hit]), bits(want["t"][hit])), "hit distances differ in bits"


WORLDS = [(30, 30, False, 1), (400, 1500, False, 2), (60, 200, True, 3)]
# (trace.kernel, trace.order): one thread per ray, persistent lane refill, warp-cooperative,
# and one thread per ray on rays sorted by the five key layouts (direction octant and origin
# cell of 512^3 or 64^3, or cell first; octahedral direction cell and origin cell of 8^3, in
# either order)
# (trace.kernel, trace.order, trace.node_test): the last case is the register-lean node test
# (trace.kernel, trace.order, trace.node_test, trace.refill_min)
KERNELS = [(0, 0, 0, 1), (1, 0, 0, 1), (2, 0, 0, 1), (0, 1, 0, 1), (0, 2, 0, 1), (0, 3, 0, 1), (0, 4, 0, 1),
           (0, 5, 0, 1), (1, 4, 0, 1), (0, 5, 1, 1), (1, 5, 0, 12)]


@pytest.fixture(params=KERNELS, ids=["kernel0", "kernel1", "kernel2", "kernel0-sorted", "kernel0-sorted64",
                                     "kernel0-cellfirst", "kernel0-dirfirst", "kernel0-originfirst",
                                     "kernel1-dirfirst", "kernel0-originfirst-lean", "kernel1-originfirst-refill12"])
def kctx(ctx, request):
    """The shared context with each traversal variant in turn."""
    ctx.set_param("trace.kernel", request.param[0])
    ctx.set_param("trace.order", request.param[1])
    ctx.set_param("trace.node_test", request.param[2])
    ctx.set_param("trace.refill_min", request.param[3])
    yield ctx
    ctx.set_param("trace.kernel", 0)
    ctx.set_param("trace.order", 0)
    ctx.set_param("trace.node_test", 0)
    ctx.set_param("trace.refill_min", 1)


@pytest.mark.parametrize("ns,nt,plane,seed", WORLDS)
def test_closest_and_any_match_bruteforce(kctx, restatement, ns, nt, plane, seed):
    ctx = kctx
    w = scenes.random_world(ns, nt, plane, seed=seed)
    rays = scenes.random_test_rays(6000, seed=seed + 100)
    ctx.upload(w)
    h = restatement.scene(w)
    want = restatement.trace_closest(h, rays)
    assert (want["prim"] != MISS).sum() > len(rays) // 20, "test rays hit nothing"
    assert_same_closest(ctx.trace_host(rays), want)
    assert np.array_equal(ctx.trace_host(rays, any_hit=True), restatement.trace_any(h, rays))


def test_chunked_host_pipeline_matches(kctx, restatement):
    """rbr_trace_host in chunks of 500 rays rotating over 2, 3 or 4 streams (trace.host_chunk,
    trace.host_streams) gives the answers of one piece, with a last chunk shorter than the
    others."""
    ctx = kctx
    w = scenes.random_world(400, 1500, False, seed=9)
    rays = scenes.random_test_rays(6500, seed=109)
    ctx.upload(w)
    h = restatement.scene(w)
    want = restatement.trace_closest(h, rays)
    want_any = restatement.trace_any(h, rays)
    chunk, streams = ctx.get_param("trace.host_chunk"), ctx.get_param("trace.host_streams")
    try:
        for c, ns in ((500, 2), (500, 3), (500, 4), (0, 2)):
            ctx.set_param("trace.host_chunk", c)
            ctx.set_param("trace.host_streams", ns)
            assert_same_closest(ctx.trace_host(rays), want)
            assert np.array_equal(ctx.trace_host(rays, any_hit=True), want_any)
        for bad in (1, 5):
            with pytest.raises(RbrError):
                ctx.set_param("trace.host_streams", bad)
    finally:
        ctx.set_param("trace.host_chunk", chunk)
        ctx.set_param("trace.host_streams", streams)


def test_sorted_queries_with_few_distinct_keys(ctx, restatement):
    """The counting sort of orders 4 and 5 with heavily repeated keys: rays from one point into a
    narrow cone from outside the scene box (one boundary origin cell, one or two direction cells),
    from two such points. Whole warps share a key and take their slots from one aggregated
    atomic; the answers equal brute force."""
    w = scenes.random_world(400, 1500, False, seed=31)
    ctx.upload(w)
    h = restatement.scene(w)
    rng = np.random.default_rng(131)
    n = 70_000
    o = np.tile(np.array([[0.5, 0.3, 13.0]], np.float32), (n, 1))
    d = np.stack([rng.uniform(-0.02, 0.02, n), rng.uniform(-0.02, 0.02, n), -np.ones(n)], 1).astype(np.float32)
    # the second half from beside the box in x (the world spans about +-11.4), towards -x
    o[n // 2:] = np.array([14.0, 0.3, 0.5], np.float32)
    d[n // 2:] = np.stack([-np.ones(n - n // 2), d[n // 2:, 0], d[n // 2:, 1]], 1)
    rays = abi.make_rays(o, d)
    want = restatement.trace_closest(h, rays)
    want_any = restatement.trace_any(h, rays)
    try:
        for order, lean in ((4, 0), (5, 0), (5, 1)):
            ctx.set_param("trace.kernel", 0)
            ctx.set_param("trace.order", order)
            ctx.set_param("trace.node_test", lean)
            assert_same_closest(ctx.trace_host(rays), want)
            assert np.array_equal(ctx.trace_host(rays, any_hit=True), want_any)
    finally:
        ctx.set_param("trace.order", 0)
        ctx.set_param("trace.node_test", 0)


@pytest.mark.parametrize("ns,nt,plane,seed", WORLDS)
def test_matches_reference_bvh_and_bruteforce(ctx, reference, ns, nt, plane, seed):
    """The same worlds through the reference library itself: its brute-force loop and its BVH."""
    w = scenes.random_world(ns, nt, plane, seed=seed)
    rays = scenes.random_test_rays(6000, seed=seed + 200)
    ctx.upload(w)
    r = reference.scene(w)
    got = ctx.trace_host(rays)
    assert_same_closest(got, reference.trace_closest(r, rays, brute=True))
    bvh = reference.trace_closest(r, rays)
    assert np.array_equal(got["prim"] == MISS, bvh["prim"] == MISS)
    hit = got["prim"] != MISS
    assert np.array_equal(bits(got["t"][hit]), bits(bvh["t"][hit]))
    assert np.array_equal(ctx.trace_host(rays, any_hit=True), reference.trace_any(r, rays))


@pytest.mark.parametrize("ns,nt,nq,plane,seed", [(30, 30, 10, False, 21), (400, 1500, 100, False, 22),
                                                  (60, 200, 20, True, 23)])
def test_tilted_quads_match_bruteforce(kctx, reference, ns, nt, nq, plane, seed):
    """Quads with non-orthogonal edges: Quad::intersect accepts a parallelogram that
    Quad::getBounds does not contain, so the reference's own BVH misses some of their hits.
    The GPU returns exactly what brute force over the primitives returns."""
    ctx = kctx
    w = scenes.random_world(ns, nt, plane, seed=seed, n_quads=nq)
    rays = scenes.random_test_rays(6000, seed=seed + 300)
    ctx.upload(w)
    r = reference.scene(w)
    brute = reference.trace_closest(r, rays, brute=True)
    got = ctx.trace_host(rays)
    assert_same_closest(got, brute)
    assert np.array_equal(ctx.trace_host(rays, any_hit=True), reference.trace_any(r, rays, brute=True))
    bvh = reference.trace_closest(r, rays)
    ref_bvh_misses = int(np.sum(bvh["prim"] != brute["prim"]))
    print(f"reference BVH disagrees with brute force on {ref_bvh_misses} of {len(rays)} rays; GPU on 0")


def test_empty_scene(kctx):
    ctx = kctx
    ctx.upload(scenes.Scene())
    rays = abi.make_rays(np.array([[0, 0, 5]], np.float32), np.array([[0, 0, -1]], np.float32))
    assert ctx.trace_host(rays)["prim"][0] == MISS
    assert ctx.trace_host(rays, any_hit=True)[0] == 0
    lo, hi = ctx.world_bounds()
    assert (lo > hi).all(), "an empty scene has an empty (inverted) bounding box"


def test_single_sphere(kctx, restatement):
    ctx = kctx
    s = scenes.Scene()
    m = s.diffuse((0.5, 0.5, 0.5))
    s.spheres = np.array([[0, 0, 0, 1]], np.float32)
    s.sphere_materials = np.array([m], np.uint32)
    ctx.upload(s)
    rays = abi.make_rays(np.array([[0, 0, 5]], np.float32), np.array([[0, 0, -1]], np.float32))
    got = ctx.trace_host(rays)
    assert got["prim"][0] == 0 and abs(got["t"][0] - 4.0) < 1e-3
    assert_same_closest(got, restatement.trace_closest(restatement.scene(s), rays))


def test_rebuild_replaces_previous_contents(ctx, restatement):
    small = scenes.random_world(30, 30, seed=11)
    big = scenes.random_world(400, 1500, seed=12)
    ctx.upload(big)
    ctx.upload(small)
    probe = abi.make_rays(np.array([[0, 0, 50]], np.float32), np.array([[0, 0, -1]], np.float32))
    rays = np.concatenate([probe, scenes.random_test_rays(2000, seed=13)])
    assert_same_closest(ctx.trace_host(rays), restatement.trace_closest(restatement.scene(small), rays))


def test_icosphere_bruteforce(kctx, restatement):
    """Displaced icosphere (level 5, 20,480 triangles): bit-exact against brute force."""
    ctx = kctx
    s = scenes.ray_query_scene(level=5)
    lo, hi = scenes.scene_bounds(s)
    rays = scenes.uniform_rays(40000, lo, hi, seed=5)
    finite = rays.copy()
    finite["tmax"] = np.random.default_rng(6).uniform(0.5, 15.0, len(rays)).astype(np.float32)
    ctx.upload(s)
    h = restatement.scene(s)
    assert_same_closest(ctx.trace_host(rays), restatement.trace_closest(h, rays))
    assert_same_closest(ctx.trace_host(finite), restatement.trace_closest(h, finite))
    assert np.array_equal(ctx.trace_host(finite, any_hit=True), restatement.trace_any(h, finite))


@pytest.mark.slow
def test_icosphere_full_size_vs_reference_bvh(kctx, reference):
    """Full ray-query workload (1,310,720 triangles, 2^22 rays) against the reference's BVH:
    identical hit/miss and hit distances for every ray; primitive ids may differ only where
    two primitives are hit at exactly the same t (the reference BVH keeps the one it visits
    last, the GPU keeps the highest id, as brute force does)."""
    ctx = kctx
    s = scenes.ray_query_scene(level=8)
    lo, hi = scenes.scene_bounds(s)
    rays = scenes.uniform_rays(1 << 22, lo, hi, seed=0)
    ctx.upload(s)
    got = ctx.trace_host(rays)
    r = reference.scene(s)
    want = reference.trace_closest(r, rays)
    miss_g, miss_w = got["prim"] == MISS, want["prim"] == MISS
    assert np.array_equal(miss_g, miss_w), f"hit/miss differs on {np.sum(miss_g != miss_w)} of {len(rays)} rays"
    hit = ~miss_w
    assert np.array_equal(bits(got["t"][hit]), bits(want["t"][hit]))
    ties = int(np.sum(got["prim"][hit] != want["prim"][hit]))
    print(f"equal-t ties resolved differently from the reference BVH: {ties} of {len(rays)} rays")
    assert ties <= len(rays) * 1e-4, f"{ties} equal-t ties resolved differently"
    # shadow queries: segments ending halfway to the hit (never occluded by it) and unbounded
    seg = rays.copy()
    seg["tmax"] = np.where(hit, got["t"] * np.float32(0.5), np.float32(np.inf))
    assert np.array_equal(ctx.trace_host(seg, any_hit=True), reference.trace_any(r, seg))
    assert np.array_equal(ctx.trace_host(rays, any_hit=True), (~miss_w).astype(np.uint8))


def test_device_and_host_entry_points_agree(ctx):
    torch = pytest.importorskip("torch")
    s = scenes.ray_query_scene(level=4)
    lo, hi = scenes.scene_bounds(s)
    rays = scenes.uniform_rays(10000, lo, hi, seed=9)
    ctx.upload(s)
    d_rays = torch.from_numpy(rays.view(np.uint8)).cuda()
    d_hits = torch.zeros(len(rays) * 8, dtype=torch.uint8, device="cuda")
    d_occ = torch.zeros(len(rays), dtype=torch.uint8, device="cuda")
    ctx.trace_closest_dev(d_rays.data_ptr(), len(rays), d_hits.data_ptr())
    ctx.trace_any_dev(d_rays.data_ptr(), len(rays), d_occ.data_ptr())
    torch.cuda.synchronize()
    got = d_hits.cpu().numpy().view(abi.HIT_DTYPE)
    host = ctx.trace_host(rays)
    assert np.array_equal(got["prim"], host["prim"]) and np.array_equal(bits(got["t"]), bits(host["t"]))
    assert np.array_equal(d_occ.cpu().numpy(), ctx.trace_host(rays, any_hit=True))
    nodes, recs = ctx.trace_counts_dev(d_rays.data_ptr(), len(rays))
    assert nodes >= len(rays) and recs > 0


def test_invalid_scenes_are_rejected(ctx):
    s = scenes.random_world(5, 5, seed=1)
    s.triangle_materials = s.triangle_materials + 7  # no such material
    with pytest.raises(RbrError) as e:
        ctx.upload(s)
    assert e.value.status == abi.RBR_ERR_INVALID_ARGUMENT
    s = scenes.random_world(5, 5, seed=1)
    s.triangles = s.triangles.copy()
    s.triangles[2, 4] = np.nan
    with pytest.raises(RbrError) as e:
        ctx.upload(s)
    assert e.value.status == abi.RBR_ERR_INVALID_ARGUMENT
    s = scenes.random_world(5, 5, seed=1)
    s.sphere_ids = s.sphere_ids.copy()
    s.sphere_ids[0] = s.sphere_ids[1]  # not a permutation
    with pytest.raises(RbrError) as e:
        ctx.upload(s)
    assert e.value.status == abi.RBR_ERR_INVALID_ARGUMENT
    s = scenes.random_world(5, 5, seed=1)
    s.point_light((0, 0, 0), (1, 1, 1))
    s.lights[-1]["type"] = 9
    with pytest.raises(RbrError) as e:
        ctx.upload(s)
    assert e.value.status == abi.RBR_ERR_UNSUPPORTED


def test_trace_before_upload_is_an_error():
    from rbr_b200 import Context

    with Context(0) as c:
        rays = abi.make_rays(np.zeros((1, 3), np.float32), np.array([[0, 0, 1]], np.float32))
        with pytest.raises(RbrError) as e:
            c.trace_host(rays)
        assert e.value.status == abi.RBR_ERR_NO_SCENE
