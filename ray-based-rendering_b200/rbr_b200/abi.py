"""ctypes mirror of include/rbr_b200.h (the C ABI of librbr_b200.so).

Structures here must match the header field for field; tests/test_abi.py checks the sizes
and offsets against the compiled library (rbr_abi_layout).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

RBR_OK = 0
RBR_ERR_INVALID_ARGUMENT = 1
RBR_ERR_CUDA = 2
RBR_ERR_OUT_OF_MEMORY = 3
RBR_ERR_NO_SCENE = 4
RBR_ERR_UNSUPPORTED = 5
RBR_ERR_DEVICE_TIMEOUT = 6
RBR_ERR_INTERNAL = 7

STATUS_NAMES = {
    0: "RBR_OK",
    1: "RBR_ERR_INVALID_ARGUMENT",
    2: "RBR_ERR_CUDA",
    3: "RBR_ERR_OUT_OF_MEMORY",
    4: "RBR_ERR_NO_SCENE",
    5: "RBR_ERR_UNSUPPORTED",
    6: "RBR_ERR_DEVICE_TIMEOUT",
    7: "RBR_ERR_INTERNAL",
}

RBR_MISS = 0xFFFFFFFF
RBR_LIGHT_AREA = 0
RBR_LIGHT_POINT = 1
RBR_CAMERA_PINHOLE = 0
RBR_CAMERA_THIN_LENS = 1
RBR_RENDER_CORRECTED_MIS = 1 << 0
RBR_RENDER_SECOND_MOMENT = 1 << 1
RBR_RENDER_VOLUMETRIC = 1 << 2
RBR_RENDER_COUNT_TRAFFIC = 1 << 3

_f3 = C.c_float * 3
_u32p = C.POINTER(C.c_uint32)
_f32p = C.POINTER(C.c_float)


class rbr_material(C.Structure):
    _fields_ = [
        ("base_color", _f3),
        ("metallic", C.c_float),
        ("roughness", C.c_float),
        ("ior", C.c_float),
        ("transmission", C.c_float),
        ("emission", _f3),
    ]


class rbr_light(C.Structure):
    _fields_ = [
        ("type", C.c_uint32),
        ("position", _f3),
        ("u", _f3),
        ("v", _f3),
        ("color", _f3),
        ("intensity", C.c_float),
    ]


class rbr_medium(C.Structure):
    _fields_ = [("sigma_a", _f3), ("sigma_s", _f3), ("g", C.c_float)]


class rbr_scene_desc(C.Structure):
    _fields_ = [
        ("num_triangles", C.c_uint32),
        ("triangle_vertices", _f32p),
        ("triangle_normals", _f32p),
        ("triangle_materials", _u32p),
        ("triangle_ids", _u32p),
        ("num_spheres", C.c_uint32),
        ("spheres", _f32p),
        ("sphere_materials", _u32p),
        ("sphere_ids", _u32p),
        ("num_quads", C.c_uint32),
        ("quads", _f32p),
        ("quad_materials", _u32p),
        ("quad_ids", _u32p),
        ("num_planes", C.c_uint32),
        ("planes", _f32p),
        ("plane_materials", _u32p),
        ("plane_ids", _u32p),
        ("num_materials", C.c_uint32),
        ("materials", C.POINTER(rbr_material)),
        ("num_lights", C.c_uint32),
        ("lights", C.POINTER(rbr_light)),
        ("background", _f3),
        ("medium", C.POINTER(rbr_medium)),
    ]


class rbr_scene_stats(C.Structure):
    _fields_ = [
        ("num_primitives", C.c_uint32),
        ("num_bounded", C.c_uint32),
        ("num_unbounded", C.c_uint32),
        ("num_wide_nodes", C.c_uint32),
        ("num_leaf_records", C.c_uint32),
        ("max_depth", C.c_uint32),
        ("wrapped_leaves", C.c_uint32),
        ("record_cost_milli", C.c_uint32),
        ("device_bytes", C.c_uint64),
        ("build_seconds", C.c_double),
    ]


class rbr_camera(C.Structure):
    _fields_ = [
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("model", C.c_uint32),
        ("position", _f3),
        ("forward", _f3),
        ("right", _f3),
        ("up", _f3),
        ("fx", C.c_float),
        ("fy", C.c_float),
        ("cx", C.c_float),
        ("cy", C.c_float),
        ("lens_radius", C.c_float),
        ("focal_distance", C.c_float),
    ]


class rbr_render_params(C.Structure):
    _fields_ = [
        ("samples_per_pixel", C.c_int32),
        ("max_depth", C.c_int32),
        ("use_nee", C.c_int32),
        ("use_mis", C.c_int32),
        ("seed", C.c_uint64),
        ("sample_offset", C.c_uint32),
        ("flags", C.c_uint32),
    ]


class rbr_render_stats(C.Structure):
    _fields_ = [
        ("paths", C.c_uint64),
        ("extension_rays", C.c_uint64),
        ("shadow_rays", C.c_uint64),
        ("waves", C.c_uint32),
        ("launches", C.c_uint32),
        ("milliseconds", C.c_float),
        ("shaded_vertices", C.c_uint64),
        ("ext_nodes", C.c_uint64),
        ("ext_records", C.c_uint64),
        ("shadow_nodes", C.c_uint64),
        ("shadow_records", C.c_uint64),
    ]


# numpy views of the ray / hit records
CACHE_LEVELS = 16
CACHE_INPUTS = 64
CACHE_MLP_WEIGHTS = 4 * 64 * 64 + 16 * 64
CACHE_RECORD_FLOATS = 16


class rbr_cache_config(C.Structure):
    _fields_ = [
        ("log2_table_size", C.c_int32),
        ("min_resolution", C.c_int32),
        ("max_resolution", C.c_int32),
        ("learning_rate", C.c_float),
        ("beta1", C.c_float),
        ("beta2", C.c_float),
        ("epsilon", C.c_float),
        ("train_batch", C.c_uint32),
        ("train_steps", C.c_uint32),
        ("train_paths", C.c_uint32),
        ("termination_depth", C.c_uint32),
        ("seed", C.c_uint64),
        ("bounds_min", _f3),
        ("bounds_max", _f3),
        ("train_suffix", C.c_uint32),
    ]


class rbr_cache_info(C.Structure):
    _fields_ = [
        ("levels", C.c_uint32),
        ("table_size", C.c_uint32),
        ("resolution", C.c_uint32 * CACHE_LEVELS),
        ("dense_levels", C.c_uint32),
        ("optimiser_steps", C.c_uint32),
        ("bounds_min", _f3),
        ("bounds_max", _f3),
        ("last_loss", C.c_float),
        ("last_queries", C.c_uint32),
        ("last_train_records", C.c_uint32),
    ]


class rbr_batch_config(C.Structure):
    _fields_ = [
        ("path_memory_bytes", C.c_uint64),
        ("wave_paths", C.c_uint32),
        ("blocks_per_sm", C.c_uint32),
        ("use_graphs", C.c_int32),
        ("waves_in_flight", C.c_uint32),
        ("persistent", C.c_uint32),
        ("barrier_timeout_us", C.c_uint32),
    ]


class rbr_request(C.Structure):
    _fields_ = [
        ("scene", C.c_uint32),
        ("camera", rbr_camera),
        ("params", rbr_render_params),
        ("use_cache", C.c_int32),
        ("train_cache", C.c_int32),
        ("film", C.c_void_p),
        ("arrival_us", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


class rbr_request_stats(C.Structure):
    _fields_ = [
        ("start_ms", C.c_float),
        ("latency_ms", C.c_float),
        ("waves", C.c_uint32),
        ("segments", C.c_uint32),
        ("paths", C.c_uint64),
    ]


class rbr_batch_stats(C.Structure):
    _fields_ = [
        ("milliseconds", C.c_float),
        ("requests", C.c_uint32),
        ("waves", C.c_uint32),
        ("segments", C.c_uint32),
        ("graphs_captured", C.c_uint32),
        ("graph_launches", C.c_uint32),
        ("kernel_launches", C.c_uint32),
        ("wave_paths", C.c_uint32),
        ("blocks_per_sm", C.c_uint32),
        ("persistent_launches", C.c_uint32),
        ("paths", C.c_uint64),
    ]


# rbr_cache_record as 16 float32 columns: position[3], direction[3], normal[3], roughness,
# diffuse[3], specular[3]
CACHE_RECORD_DTYPE = np.dtype((np.float32, (CACHE_RECORD_FLOATS,)))

RAY_DTYPE = np.dtype(
    [("origin", np.float32, 3), ("tmax", np.float32), ("direction", np.float32, 3), ("pad", np.float32)]
)
HIT_DTYPE = np.dtype([("prim", np.uint32), ("t", np.float32)])
assert RAY_DTYPE.itemsize == 32 and HIT_DTYPE.itemsize == 8


def f3(v) -> "C.Array":
    return _f3(*[float(x) for x in v])


def make_rays(origins: np.ndarray, directions: np.ndarray, tmax=np.inf) -> np.ndarray:
    """Packs origins/directions (n,3 float32) and tmax (scalar or n) into rbr_ray records."""
    n = origins.shape[0]
    rays = np.zeros(n, dtype=RAY_DTYPE)
    rays["origin"] = origins.astype(np.float32)
    rays["direction"] = directions.astype(np.float32)
    rays["tmax"] = np.broadcast_to(np.asarray(tmax, dtype=np.float32), (n,))
    return rays


def ptr(a: np.ndarray | None, ctype):
    if a is None:
        return C.cast(None, C.POINTER(ctype))
    assert a.flags["C_CONTIGUOUS"], "arrays passed to the C ABI must be C-contiguous"
    return a.ctypes.data_as(C.POINTER(ctype))
