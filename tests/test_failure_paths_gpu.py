"""Failure detection without a GPU fault: the errors the library reports when a bounded device
wait runs out or a device allocation fails, and that the context stays usable afterwards.

The tensor-core kernels of the radiance cache wait for MMA completion on an mbarrier with a
bounded number of polls ("cache.wait_limit"). With the limit at 0 every such wait gives up at
once: the kernel records kErrDeviceTimeout, stops issuing work, drains the MMA it already
issued with the full bound and frees its tensor memory, so nothing hangs and nothing is left in
flight. Allocation failures are injected on the host ("debug.fail_alloc"): the next device
allocation of the context reports RBR_ERR_OUT_OF_MEMORY instead of calling cudaMalloc."""
import numpy as np
import pytest

from rbr_b200 import Context, RbrError, abi, render_params, scenes

pytestmark = pytest.mark.gpu


def records(n, seed=3):
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 16), np.float32)
    r[:, 0:3] = rng.uniform(-1, 1, (n, 3))
    d = rng.normal(size=(n, 6))
    r[:, 3:6] = d[:, :3] / np.linalg.norm(d[:, :3], axis=1, keepdims=True)
    r[:, 6:9] = d[:, 3:] / np.linalg.norm(d[:, 3:], axis=1, keepdims=True)
    r[:, 9:16] = rng.uniform(0, 1, (n, 7))
    return r


def test_tensor_core_wait_runs_out_and_context_recovers():
    with Context(0) as c:
        c.cache_create(log2_table_size=12, bounds_min=(-1, -1, -1), bounds_max=(1, 1, 1), seed=1)
        recs = records(1000)
        want = c.cache_infer(recs)
        t = np.random.default_rng(4).uniform(0, 2, (1000, 3)).astype(np.float32)
        assert c.get_param("cache.wait_limit") == 1 << 22
        c.set_param("cache.wait_limit", 0)
        with pytest.raises(RbrError) as e:
            c.cache_infer(recs)
        assert e.value.status == abi.RBR_ERR_DEVICE_TIMEOUT
        assert "bounded device wait" in c.last_error()
        with pytest.raises(RbrError) as e:
            c.cache_train(recs, t, apply=False)
        assert e.value.status == abi.RBR_ERR_DEVICE_TIMEOUT
        # the same context, with the normal bound again: inference is unchanged
        c.set_param("cache.wait_limit", 1 << 22)
        got = c.cache_infer(recs)
        assert np.array_equal(got, want)
        c.cache_train(recs, t, apply=False)
        with pytest.raises(RbrError):
            c.set_param("cache.wait_limit", (1 << 22) + 1)


def test_injected_allocation_failure_and_recovery():
    s = scenes.cornell_box(64, 48)
    with Context(0) as c:
        c.upload(s)
        p = render_params(spp=4, max_depth=8, seed=9)
        # rbr_render_host's first allocation is its film staging, the second the path rays
        c.set_param("debug.fail_alloc", 2)
        with pytest.raises(RbrError) as e:
            c.render_host(s.camera, p)
        assert e.value.status == abi.RBR_ERR_OUT_OF_MEMORY
        assert "path rays" in c.last_error() and "failure injected" in c.last_error()
        assert c.get_param("debug.fail_alloc") == 0
        got = c.render_host(s.camera, p)  # nothing left half-allocated
    with Context(0) as c2:
        c2.upload(s)
        want = c2.render_host(s.camera, p)
    assert np.array_equal(got, want)


def test_injected_failure_of_a_later_allocation():
    """The n-th allocation fails: when the second path-buffer set (two waves in flight) cannot be
    allocated, the render runs its waves one at a time in the first set and gives the film of
    pt.streams 1; the next render allocates the second set again."""
    s = scenes.cornell_box(64, 48)
    with Context(0) as c:
        c.upload(s)
        p = render_params(spp=2, max_depth=4, seed=1)
        # the film staging, nine buffers of the first set, then the second set's
        c.set_param("debug.fail_alloc", 12)
        fallback = c.render_host(s.camera, p)
        assert c.get_param("debug.fail_alloc") == 0  # the injected failure happened
        st = c.render_stats()
        assert st.paths == 64 * 48 * 2 and st.waves == 2
        c.set_param("pt.streams", 1)
        one = c.render_host(s.camera, p)
        c.set_param("pt.streams", 2)
        two = c.render_host(s.camera, p)
    assert np.allclose(fallback, one, rtol=1e-5, atol=1e-5)
    assert np.allclose(one, two, rtol=1e-5, atol=1e-5)
