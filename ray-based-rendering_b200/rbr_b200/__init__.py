"""Python binding of librbr_b200.so, the B200 path-tracing hot path (C ABI: include/rbr_b200.h).

The library is the GPU side of the reference framework's Accelerator / Integrator drop-ins;
this module is a thin ctypes layer used by the tests and the benchmark. There is no CPU
fallback: without the built library or without a CUDA device every call raises.
"""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np

from . import abi
from .abi import RAY_DTYPE, HIT_DTYPE

LIB_PATH = Path(__file__).resolve().parent / "librbr_b200.so"
HEADER = Path(__file__).resolve().parents[2] / "include" / "rbr_b200.h"

_lib = None


class RbrError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def header_functions() -> list[str]:
    """Names of the functions include/rbr_b200.h declares."""
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rbr_[a-z_0-9]+)\s*\(", text)))


def load_library() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                           "(python -m rbr_b200.build); there is no CPU fallback")
    lib = C.CDLL(str(LIB_PATH))
    P = C.c_void_p
    sig = {
        "rbr_abi_version": (C.c_uint32, []),
        "rbr_struct_size": (C.c_size_t, [C.c_char_p]),
        "rbr_ctx_create": (C.c_int, [C.c_int, C.POINTER(P)]),
        "rbr_ctx_destroy": (None, [P]),
        "rbr_last_error": (C.c_char_p, [P]),
        "rbr_scene_upload": (C.c_int, [P, C.POINTER(abi.rbr_scene_desc)]),
        "rbr_scene_stats_get": (C.c_int, [P, C.POINTER(abi.rbr_scene_stats)]),
        "rbr_world_bounds": (C.c_int, [P, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
        "rbr_trace_closest": (C.c_int, [P, P, C.c_uint32, P, P]),
        "rbr_trace_any": (C.c_int, [P, P, C.c_uint32, P, P]),
        "rbr_trace_host": (C.c_int, [P, P, C.c_uint32, C.c_int, P]),
        "rbr_trace_counts": (C.c_int, [P, P, C.c_uint32, C.c_int, C.POINTER(C.c_uint64)]),
        "rbr_render": (C.c_int, [P, C.POINTER(abi.rbr_camera), C.POINTER(abi.rbr_render_params), P, P, P]),
        "rbr_render_host": (C.c_int, [P, C.POINTER(abi.rbr_camera), C.POINTER(abi.rbr_render_params), P, P]),
        "rbr_render_stats_get": (C.c_int, [P, C.POINTER(abi.rbr_render_stats)]),
        "rbr_render_noalloc": (C.c_int, [P, C.POINTER(abi.rbr_camera), C.POINTER(abi.rbr_render_params), P, P]),
        "rbr_bsdf_eval_host": (C.c_int, [P, C.POINTER(abi.rbr_material), C.c_uint32, P, P, P]),
        "rbr_bsdf_sample_host": (C.c_int, [P, C.POINTER(abi.rbr_material), C.c_uint32, P, P, P]),
        "rbr_light_sample_host": (C.c_int, [P, C.POINTER(abi.rbr_light), C.c_uint32, P, P, P]),
        "rbr_camera_rays_host": (C.c_int, [P, C.POINTER(abi.rbr_camera), C.c_uint32, P, P]),
        "rbr_mis_weights_host": (C.c_int, [P, C.c_uint32, P, P]),
        "rbr_phase_eval_host": (C.c_int, [P, C.c_float, C.c_uint32, P, P, P]),
        "rbr_phase_sample_host": (C.c_int, [P, C.c_float, C.c_uint32, P, P, P]),
        "rbr_medium_sample_host": (C.c_int, [P, C.POINTER(abi.rbr_medium), C.c_uint32, P, P, P]),
        "rbr_l2_read_bandwidth": (C.c_int, [P, C.c_uint64, C.c_uint32, C.POINTER(C.c_double)]),
        "rbr_param_set": (C.c_int, [P, C.c_char_p, C.c_int64]),
        "rbr_param_get": (C.c_int, [P, C.c_char_p, C.POINTER(C.c_int64)]),
        "rbr_autotune_trace": (C.c_int, [P, P, C.c_uint32, C.c_int, C.POINTER(C.c_int64)]),
        "rbr_cache_config_default": (None, [C.POINTER(abi.rbr_cache_config)]),
        "rbr_cache_create": (C.c_int, [P, C.POINTER(abi.rbr_cache_config)]),
        "rbr_cache_destroy": (None, [P]),
        "rbr_cache_info_get": (C.c_int, [P, C.POINTER(abi.rbr_cache_info)]),
        "rbr_cache_set_params": (C.c_int, [P, P, P]),
        "rbr_cache_get_params": (C.c_int, [P, P, P]),
        "rbr_cache_grads_get": (C.c_int, [P, P, P]),
        "rbr_cache_encode_host": (C.c_int, [P, C.c_uint32, P, P]),
        "rbr_cache_infer_host": (C.c_int, [P, C.c_uint32, P, P]),
        "rbr_cache_train_host": (C.c_int, [P, C.c_uint32, P, P, C.c_int, C.POINTER(C.c_float)]),
        "rbr_cache_render": (C.c_int, [P, C.POINTER(abi.rbr_camera), C.POINTER(abi.rbr_render_params), C.c_uint32,
                                       C.c_int, P, P, P]),
        "rbr_mesh_load_obj": (C.c_int, [C.c_char_p, C.POINTER(P), C.c_char_p, C.c_size_t]),
        "rbr_mesh_parse_obj": (C.c_int, [C.c_char_p, C.c_size_t, C.POINTER(P), C.c_char_p, C.c_size_t]),
        "rbr_mesh_triangles": (C.c_uint32, [P]),
        "rbr_mesh_triangle_vertices": (C.POINTER(C.c_float), [P]),
        "rbr_mesh_triangle_normals": (C.POINTER(C.c_float), [P]),
        "rbr_mesh_destroy": (None, [P]),
        "rbr_film_to_rgb8": (C.c_int, [P, P, C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_int, P, P]),
        "rbr_film_to_rgb8_host": (C.c_int, [P, P, C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_int, P]),
        "rbr_batch_config_default": (None, [C.POINTER(abi.rbr_batch_config)]),
        "rbr_batch_create": (C.c_int, [P, C.POINTER(abi.rbr_batch_config), C.POINTER(P)]),
        "rbr_batch_destroy": (None, [P]),
        "rbr_batch_last_error": (C.c_char_p, [P]),
        "rbr_batch_add_scene": (C.c_int, [P, C.POINTER(abi.rbr_scene_desc), C.POINTER(C.c_uint32)]),
        "rbr_batch_cache_create": (C.c_int, [P, C.c_uint32, C.POINTER(abi.rbr_cache_config)]),
        "rbr_batch_add_scene_variant": (C.c_int, [P, C.c_uint32, C.POINTER(abi.rbr_material), C.c_uint32,
                                                  C.POINTER(abi.rbr_light), C.c_uint32, C.POINTER(abi.rbr_medium),
                                                  C.POINTER(C.c_uint32)]),
        "rbr_batch_submit": (C.c_int, [P, C.POINTER(abi.rbr_request), C.POINTER(C.c_uint32)]),
        "rbr_batch_run": (C.c_int, [P, P]),
        "rbr_batch_set_host_film": (C.c_int, [P, C.c_uint32, P]),
        "rbr_batch_request_stats": (C.c_int, [P, C.c_uint32, C.POINTER(abi.rbr_request_stats)]),
        "rbr_batch_stats_get": (C.c_int, [P, C.POINTER(abi.rbr_batch_stats)]),
        "rbr_batch_autotune": (C.c_int, [P, P]),
    }
    for name, (res, args) in sig.items():
        if hasattr(lib, name):
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
    _lib = lib
    return lib


def _mesh_arrays(lib, h):
    n = lib.rbr_mesh_triangles(h)
    v = np.ctypeslib.as_array(lib.rbr_mesh_triangle_vertices(h), shape=(n * 9,)).reshape(n, 9).copy()
    np_ = lib.rbr_mesh_triangle_normals(h)
    nn = np.ctypeslib.as_array(np_, shape=(n * 9,)).reshape(n, 9).copy() if np_ else None
    return v, nn


def parse_obj(text):
    """Triangles of an OBJ text (ObjImporter::parse + toPrimitives): vertices [n, 9] and unit
    vertex normals [n, 9] or None. Raises ValueError on a malformed file."""
    lib = load_library()
    data = text.encode() if isinstance(text, str) else bytes(text)
    h = C.c_void_p()
    err = C.create_string_buffer(256)
    st = lib.rbr_mesh_parse_obj(data, len(data), C.byref(h), err, 256)
    if st != abi.RBR_OK:
        raise ValueError(err.value.decode())
    try:
        return _mesh_arrays(lib, h)
    finally:
        lib.rbr_mesh_destroy(h)


def load_obj(path):
    """parse_obj of a file (ObjImporter::load)."""
    lib = load_library()
    h = C.c_void_p()
    err = C.create_string_buffer(256)
    st = lib.rbr_mesh_load_obj(str(path).encode(), C.byref(h), err, 256)
    if st != abi.RBR_OK:
        raise ValueError(err.value.decode())
    try:
        return _mesh_arrays(lib, h)
    finally:
        lib.rbr_mesh_destroy(h)


def render_params(spp=16, max_depth=8, use_nee=True, use_mis=True, seed=0, sample_offset=0, flags=0):
    p = abi.rbr_render_params()
    p.samples_per_pixel = spp
    p.max_depth = max_depth
    p.use_nee = int(use_nee)
    p.use_mis = int(use_mis)
    p.seed = seed
    p.sample_offset = sample_offset
    p.flags = flags
    return p


class Context:
    """One rbr_ctx: a device, a resident scene, and the path tracer's working memory."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        st = self.lib.rbr_ctx_create(device, C.byref(h))
        if st != abi.RBR_OK:
            raise RbrError(st, f"rbr_ctx_create({device}) failed (no usable CUDA device?)")
        self.h = h
        self._scene_keep = None

    def close(self):
        if getattr(self, "h", None):
            self.lib.rbr_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st):
        if st != abi.RBR_OK:
            raise RbrError(st, self.lib.rbr_last_error(self.h).decode())

    # scene ---------------------------------------------------------------------------------
    def upload(self, scene) -> abi.rbr_scene_stats:
        desc = scene.desc() if hasattr(scene, "desc") and callable(scene.desc) else scene
        self._check(self.lib.rbr_scene_upload(self.h, C.byref(desc.desc)))
        self._scene_keep = desc
        return self.stats()

    def upload_raw(self, desc: abi.rbr_scene_desc) -> int:
        return self.lib.rbr_scene_upload(self.h, C.byref(desc))

    def set_param(self, name: str, value: int):
        self._check(self.lib.rbr_param_set(self.h, name.encode(), int(value)))

    def get_param(self, name: str) -> int:
        v = C.c_int64()
        self._check(self.lib.rbr_param_get(self.h, name.encode(), C.byref(v)))
        return int(v.value)

    def autotune_trace(self, rays_ptr: int, n: int, any_hit: bool = False) -> dict:
        """Times the traversal variants on these device rays; keeps the fastest. Returns the choice."""
        us = C.c_int64()
        self._check(self.lib.rbr_autotune_trace(self.h, C.c_void_p(rays_ptr), n, int(any_hit), C.byref(us)))
        return {"trace.kernel": self.get_param("trace.kernel"), "trace.min_blocks": self.get_param("trace.min_blocks"),
                "trace.order": self.get_param("trace.order"), "trace.node_test": self.get_param("trace.node_test"),
                "us_per_launch": us.value}

    def l2_read_bandwidth(self, nbytes: int = 32 << 20, passes: int = 50) -> float:
        """Read bandwidth (GB/s) of an L2-resident buffer: the traversal roofline's denominator."""
        v = C.c_double()
        self._check(self.lib.rbr_l2_read_bandwidth(self.h, nbytes, passes, C.byref(v)))
        return v.value

    def last_error(self) -> str:
        return self.lib.rbr_last_error(self.h).decode()

    def stats(self) -> abi.rbr_scene_stats:
        s = abi.rbr_scene_stats()
        self._check(self.lib.rbr_scene_stats_get(self.h, C.byref(s)))
        return s

    def world_bounds(self):
        lo = (C.c_float * 3)()
        hi = (C.c_float * 3)()
        self._check(self.lib.rbr_world_bounds(self.h, lo, hi))
        return np.array(lo[:], np.float32), np.array(hi[:], np.float32)

    # ray queries ---------------------------------------------------------------------------
    def trace_closest_dev(self, rays_ptr: int, n: int, hits_ptr: int, stream: int = 0):
        self._check(self.lib.rbr_trace_closest(self.h, C.c_void_p(rays_ptr), n, C.c_void_p(hits_ptr),
                                               C.c_void_p(stream)))

    def trace_any_dev(self, rays_ptr: int, n: int, occ_ptr: int, stream: int = 0):
        self._check(self.lib.rbr_trace_any(self.h, C.c_void_p(rays_ptr), n, C.c_void_p(occ_ptr),
                                           C.c_void_p(stream)))

    def trace_host(self, rays: np.ndarray, any_hit: bool = False, out: np.ndarray | None = None) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=RAY_DTYPE)
        n = len(rays)
        if out is None:
            out = np.zeros(n, dtype=np.uint8 if any_hit else HIT_DTYPE)
        self._check(self.lib.rbr_trace_host(self.h, C.c_void_p(rays.ctypes.data), n, int(any_hit),
                                            C.c_void_p(out.ctypes.data)))
        return out

    def trace_counts_dev(self, rays_ptr: int, n: int, any_hit: bool = False):
        """(wide nodes fetched, leaf records tested) summed over the n rays."""
        out = (C.c_uint64 * 2)()
        self._check(self.lib.rbr_trace_counts(self.h, C.c_void_p(rays_ptr), n, int(any_hit), out))
        return int(out[0]), int(out[1])

    # rendering -----------------------------------------------------------------------------
    def render_dev(self, camera, params, film_mean_ptr: int, film_m2_ptr: int = 0, stream: int = 0):
        self._check(self.lib.rbr_render(self.h, C.byref(camera), C.byref(params), C.c_void_p(film_mean_ptr),
                                        C.c_void_p(film_m2_ptr or None), C.c_void_p(stream)))

    def render_host(self, camera, params, second_moment: bool = False, out: np.ndarray | None = None):
        """Renders into host memory: `out` (float32, H x W x 3, e.g. a view of pinned memory) or a
        new array."""
        W, H = camera.width, camera.height
        if out is not None and (out.dtype != np.float32 or out.size != H * W * 3 or not out.flags.c_contiguous):
            raise ValueError("out must be a C-contiguous float32 array of H x W x 3")
        mean = out.reshape(H, W, 3) if out is not None else np.zeros((H, W, 3), np.float32)
        m2 = np.zeros((H, W, 3), np.float32) if second_moment else None
        if second_moment:
            params.flags |= abi.RBR_RENDER_SECOND_MOMENT
        self._check(self.lib.rbr_render_host(self.h, C.byref(camera), C.byref(params),
                                             C.c_void_p(mean.ctypes.data),
                                             C.c_void_p(m2.ctypes.data) if m2 is not None else None))
        return (mean, m2) if second_moment else mean

    # device functions on caller inputs (unit parity) -----------------------------------------
    def _unit(self, fn, args, n, width):
        out = np.zeros((n, width), np.float32)
        keep = [np.ascontiguousarray(a, np.float32) for a in args]
        self._check(fn(self.h, *[C.c_void_p(k.ctypes.data) for k in keep], C.c_void_p(out.ctypes.data)))
        return out

    def bsdf_eval(self, material: abi.rbr_material, wo, wi):
        """(n, 6): f[3], pdf, isDelta, type bits."""
        n = len(wo)
        return self._unit(lambda h, a, b, o: self.lib.rbr_bsdf_eval_host(h, C.byref(material), n, a, b, o),
                          [wo, wi], n, 6)

    def bsdf_sample(self, material: abi.rbr_material, wo, u):
        """(n, 8): wi[3], f[3], pdf, isDelta."""
        n = len(wo)
        return self._unit(lambda h, a, b, o: self.lib.rbr_bsdf_sample_host(h, C.byref(material), n, a, b, o),
                          [wo, u], n, 8)

    def light_sample(self, light: abi.rbr_light, points, u):
        """(n, 9): wi[3], Li[3], pdf, distance, isDelta."""
        n = len(points)
        return self._unit(lambda h, a, b, o: self.lib.rbr_light_sample_host(h, C.byref(light), n, a, b, o),
                          [points, u], n, 9)

    def camera_rays(self, camera: abi.rbr_camera, samples):
        """(n, 6): origin[3], direction[3]."""
        n = len(samples)
        return self._unit(lambda h, a, o: self.lib.rbr_camera_rays_host(h, C.byref(camera), n, a, o),
                          [samples], n, 6)

    def mis_weights(self, pdf_pairs):
        n = len(pdf_pairs)
        return self._unit(lambda h, a, o: self.lib.rbr_mis_weights_host(h, n, a, o), [pdf_pairs], n, 1)[:, 0]

    # radiance cache ------------------------------------------------------------------------
    def cache_config(self, **kw) -> abi.rbr_cache_config:
        cfg = abi.rbr_cache_config()
        self.lib.rbr_cache_config_default(C.byref(cfg))
        for k, v in kw.items():
            if k in ("bounds_min", "bounds_max"):
                getattr(cfg, k)[:] = [float(x) for x in v]
            else:
                setattr(cfg, k, v)
        return cfg

    def cache_create(self, cfg: abi.rbr_cache_config | None = None, **kw):
        cfg = cfg if cfg is not None else self.cache_config(**kw)
        self._check(self.lib.rbr_cache_create(self.h, C.byref(cfg)))
        return self.cache_info()

    def cache_info(self) -> abi.rbr_cache_info:
        info = abi.rbr_cache_info()
        self._check(self.lib.rbr_cache_info_get(self.h, C.byref(info)))
        return info

    def cache_set_params(self, mlp_bf16: np.ndarray | None = None, grid_f16: np.ndarray | None = None):
        m = None if mlp_bf16 is None else np.ascontiguousarray(mlp_bf16, np.uint16)
        g = None if grid_f16 is None else np.ascontiguousarray(grid_f16, np.uint16)
        self._check(self.lib.rbr_cache_set_params(self.h, None if m is None else C.c_void_p(m.ctypes.data),
                                                  None if g is None else C.c_void_p(g.ctypes.data)))

    def cache_get_params(self, grid: bool = False):
        info = self.cache_info()
        m = np.zeros(abi.CACHE_MLP_WEIGHTS, np.uint16)
        g = np.zeros(info.levels * info.table_size * 2, np.uint16) if grid else None
        self._check(self.lib.rbr_cache_get_params(self.h, C.c_void_p(m.ctypes.data),
                                                  None if g is None else C.c_void_p(g.ctypes.data)))
        return (m, g) if grid else m

    def cache_grads(self, grid: bool = True):
        info = self.cache_info()
        m = np.zeros(abi.CACHE_MLP_WEIGHTS, np.float32)
        g = np.zeros(info.levels * info.table_size * 2, np.float32) if grid else None
        self._check(self.lib.rbr_cache_grads_get(self.h, C.c_void_p(m.ctypes.data),
                                                 None if g is None else C.c_void_p(g.ctypes.data)))
        return m, g

    def cache_encode(self, records: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(records, np.float32).reshape(-1, abi.CACHE_RECORD_FLOATS)
        out = np.zeros((len(r), abi.CACHE_INPUTS), np.float32)
        self._check(self.lib.rbr_cache_encode_host(self.h, len(r), C.c_void_p(r.ctypes.data), C.c_void_p(out.ctypes.data)))
        return out

    def cache_infer(self, records: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(records, np.float32).reshape(-1, abi.CACHE_RECORD_FLOATS)
        out = np.zeros((len(r), 3), np.float32)
        self._check(self.lib.rbr_cache_infer_host(self.h, len(r), C.c_void_p(r.ctypes.data), C.c_void_p(out.ctypes.data)))
        return out

    def cache_train(self, records: np.ndarray, targets: np.ndarray, apply: bool = True) -> float:
        r = np.ascontiguousarray(records, np.float32).reshape(-1, abi.CACHE_RECORD_FLOATS)
        t = np.ascontiguousarray(targets, np.float32).reshape(-1, 3)
        loss = C.c_float()
        self._check(self.lib.rbr_cache_train_host(self.h, len(r), C.c_void_p(r.ctypes.data), C.c_void_p(t.ctypes.data),
                                                  int(apply), C.byref(loss)))
        return float(loss.value)

    def cache_render_dev(self, camera, params, frames: int, film_mean_ptr: int, film_m2_ptr: int = 0,
                         train: bool = True, stream: int = 0):
        self._check(self.lib.rbr_cache_render(self.h, C.byref(camera), C.byref(params), frames, int(train),
                                              C.c_void_p(film_mean_ptr), C.c_void_p(film_m2_ptr or None),
                                              C.c_void_p(stream)))

    def film_to_rgb8(self, film: np.ndarray, exposure=1.0, gamma=2.2, tonemap=False) -> np.ndarray:
        film = np.ascontiguousarray(film, np.float32)
        h, w = film.shape[:2]
        out = np.zeros((h, w, 3), np.uint8)
        self._check(self.lib.rbr_film_to_rgb8_host(self.h, C.c_void_p(film.ctypes.data), w, h, exposure, gamma,
                                                   int(tonemap), C.c_void_p(out.ctypes.data)))
        return out

    def phase_eval(self, g, wo, wi):
        n = len(wo)
        return self._unit(lambda h, a, b, o: self.lib.rbr_phase_eval_host(h, g, n, a, b, o), [wo, wi], n, 1)[:, 0]

    def phase_sample(self, g, wo, u):
        n = len(wo)
        return self._unit(lambda h, a, b, o: self.lib.rbr_phase_sample_host(h, g, n, a, b, o), [wo, u], n, 3)

    def medium_sample(self, medium: abi.rbr_medium, max_dist, u):
        """(n, 5): t, weight[3], scattered."""
        n = len(max_dist)
        return self._unit(lambda h, a, b, o: self.lib.rbr_medium_sample_host(h, C.byref(medium), n, a, b, o),
                          [max_dist, u], n, 5)

    def render_stats(self) -> abi.rbr_render_stats:
        s = abi.rbr_render_stats()
        self._check(self.lib.rbr_render_stats_get(self.h, C.byref(s)))
        return s


class Batch:
    """An rbr_batch: the batched request loop on a Context's device and path buffers."""

    def __init__(self, ctx: Context, **cfg):
        self.ctx = ctx
        self.lib = ctx.lib
        c = abi.rbr_batch_config()
        self.lib.rbr_batch_config_default(C.byref(c))
        for k, v in cfg.items():
            setattr(c, k, v)
        h = C.c_void_p()
        st = self.lib.rbr_batch_create(ctx.h, C.byref(c), C.byref(h))
        if st != abi.RBR_OK:
            raise RbrError(st, "rbr_batch_create failed")
        self.h = h
        self._keep = []

    def _check(self, st):
        if st != abi.RBR_OK:
            raise RbrError(st, self.lib.rbr_batch_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.rbr_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_scene(self, scene) -> int:
        desc = scene.desc() if hasattr(scene, "desc") and callable(scene.desc) else scene
        sid = C.c_uint32()
        self._check(self.lib.rbr_batch_add_scene(self.h, C.byref(desc.desc), C.byref(sid)))
        self._keep.append(desc)
        return int(sid.value)

    def add_scene_variant(self, base_id: int, scene) -> int:
        """A scene sharing base_id's geometry and BVH, with `scene`'s materials, lights, medium."""
        desc = scene.desc() if hasattr(scene, "desc") and callable(scene.desc) else scene
        d = desc.desc
        sid = C.c_uint32()
        self._check(self.lib.rbr_batch_add_scene_variant(self.h, base_id, d.materials, d.num_materials, d.lights,
                                                         d.num_lights, d.medium, C.byref(sid)))
        self._keep.append(desc)
        return int(sid.value)

    def cache_create(self, scene_id: int, **kw):
        cfg = self.ctx.cache_config(**kw)
        self._check(self.lib.rbr_batch_cache_create(self.h, scene_id, C.byref(cfg)))

    def submit(self, scene_id, camera, params, film_ptr, use_cache=False, train_cache=False, arrival_us=0) -> int:
        r = abi.rbr_request()
        r.scene = scene_id
        r.camera = camera
        r.params = params
        r.use_cache = int(use_cache)
        r.train_cache = int(train_cache)
        r.film = film_ptr
        r.arrival_us = int(arrival_us)
        rid = C.c_uint32()
        self._check(self.lib.rbr_batch_submit(self.h, C.byref(r), C.byref(rid)))
        return int(rid.value)

    def set_host_film(self, rid: int, host_ptr: int):
        """The next run also copies request `rid`'s film to host memory at `host_ptr` (page-locked
        for an asynchronous copy) right after the request's last wave."""
        self._check(self.lib.rbr_batch_set_host_film(self.h, rid, C.c_void_p(host_ptr)))

    def run(self, stream: int = 0):
        self._check(self.lib.rbr_batch_run(self.h, C.c_void_p(stream)))

    def autotune(self, stream: int = 0):
        self._check(self.lib.rbr_batch_autotune(self.h, C.c_void_p(stream)))

    def request_stats(self, rid: int) -> abi.rbr_request_stats:
        s = abi.rbr_request_stats()
        self._check(self.lib.rbr_batch_request_stats(self.h, rid, C.byref(s)))
        return s

    def stats(self) -> abi.rbr_batch_stats:
        s = abi.rbr_batch_stats()
        self._check(self.lib.rbr_batch_stats_get(self.h, C.byref(s)))
        return s


__all__ = ["Context", "Batch", "load_obj", "parse_obj", "RbrError", "load_library", "header_functions", "render_params", "abi", "RAY_DTYPE",
           "HIT_DTYPE"]
