"""rbr_render_noalloc: rendering without any device allocation inside the call.

Callers that manage the GPU's memory themselves (a fixed pool reserved at start-up, or a frame
loop that must not stall on cudaMalloc/cudaFree) use this entry point instead of rbr_render,
which allocates its per-path working memory on demand. It must produce the film rbr_render
produces, call after call, although every call reuses (and finds dirty) the same fixed scratch
array. This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from rbr_b200 import Context, abi, load_library, render_params, scenes

pytestmark = pytest.mark.gpu


def test_noalloc_render_matches_render_on_consecutive_calls():
    torch = pytest.importorskip("torch")
    lib = load_library()
    with Context(0) as ctx:
        s = scenes.cornell_box(96, 80)  # 7,680 pixels: several waves of the fixed scratch at 64 spp
        ctx.upload(s)
        cam = s.camera
        n = cam.width * cam.height * 3
        stream = torch.cuda.current_stream().cuda_stream
        for params in (render_params(spp=64, max_depth=8, seed=77),
                       render_params(spp=16, max_depth=6, seed=5, sample_offset=100)):
            want = torch.zeros(n, dtype=torch.float32, device="cuda")
            ctx.render_dev(cam, params, want.data_ptr(), 0, stream)
            got = torch.full((n,), -1.0, dtype=torch.float32, device="cuda")  # stale values must be overwritten
            st = lib.rbr_render_noalloc(ctx.h, C.byref(cam), C.byref(params), C.c_void_p(got.data_ptr()),
                                        C.c_void_p(stream))
            assert st == abi.RBR_OK, ctx.last_error()
            torch.cuda.synchronize()
            np.testing.assert_allclose(got.cpu().numpy(), want.cpu().numpy(), rtol=1e-5, atol=1e-6)


def test_noalloc_render_rejects_what_does_not_fit():
    lib = load_library()
    with Context(0) as ctx:
        s = scenes.cornell_box(8, 8)
        ctx.upload(s)
        film = np.zeros(8 * 8 * 3, np.float32)  # never written: the call is rejected first
        st = lib.rbr_render_noalloc(ctx.h, C.byref(s.camera), C.byref(render_params(spp=1 << 20)),
                                    C.c_void_p(film.ctypes.data), None)
        assert st == abi.RBR_ERR_INVALID_ARGUMENT
        assert "scratch" in ctx.last_error()
