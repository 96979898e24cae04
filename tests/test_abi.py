"""The C-ABI library loads, exports every function include/rbr_b200.h declares, and its struct
layouts match the ctypes mirrors. No compute calls (runs without a GPU)."""
import ctypes as C

import pytest

from rbr_b200 import abi, header_functions, load_library


def test_library_exports_every_declared_function():
    lib = load_library()
    declared = header_functions()
    assert "rbr_trace_closest" in declared and "rbr_render" in declared
    missing = [name for name in declared if not hasattr(lib, name)]
    assert not missing, f"declared in include/rbr_b200.h but not exported: {missing}"


def test_abi_version():
    assert load_library().rbr_abi_version() == 1


@pytest.mark.parametrize(
    "name,cls",
    [
        ("rbr_material", abi.rbr_material),
        ("rbr_light", abi.rbr_light),
        ("rbr_scene_desc", abi.rbr_scene_desc),
        ("rbr_scene_stats", abi.rbr_scene_stats),
        ("rbr_camera", abi.rbr_camera),
        ("rbr_render_params", abi.rbr_render_params),
        ("rbr_render_stats", abi.rbr_render_stats),
        ("rbr_cache_config", abi.rbr_cache_config),
        ("rbr_cache_info", abi.rbr_cache_info),
        ("rbr_medium", abi.rbr_medium),
        ("rbr_batch_config", abi.rbr_batch_config),
        ("rbr_request", abi.rbr_request),
        ("rbr_request_stats", abi.rbr_request_stats),
        ("rbr_batch_stats", abi.rbr_batch_stats),
    ],
)
def test_struct_sizes_match(name, cls):
    assert load_library().rbr_struct_size(name.encode()) == C.sizeof(cls)


def test_record_sizes():
    lib = load_library()
    assert lib.rbr_struct_size(b"rbr_ray") == abi.RAY_DTYPE.itemsize == 32
    assert lib.rbr_struct_size(b"rbr_hit") == abi.HIT_DTYPE.itemsize == 8
    assert lib.rbr_struct_size(b"rbr_cache_record") == abi.CACHE_RECORD_DTYPE.itemsize == 64
    assert lib.rbr_struct_size(b"no_such_struct") == 0


def test_null_arguments_are_rejected_without_a_device():
    lib = load_library()
    assert lib.rbr_ctx_create(0, None) == abi.RBR_ERR_INVALID_ARGUMENT
    assert lib.rbr_scene_upload(None, None) == abi.RBR_ERR_INVALID_ARGUMENT
    assert lib.rbr_trace_closest(None, None, 0, None, None) == abi.RBR_ERR_INVALID_ARGUMENT
    assert lib.rbr_render(None, None, None, None, None, None) == abi.RBR_ERR_INVALID_ARGUMENT
    assert lib.rbr_last_error(None) == b"no context"


def test_no_cpu_fallback_without_a_device():
    """Without a CUDA device context creation fails loudly (there is no CPU path)."""
    lib = load_library()
    h = C.c_void_p()
    st = lib.rbr_ctx_create(0, C.byref(h))
    if st == abi.RBR_OK:
        lib.rbr_ctx_destroy(h)
        pytest.skip("a CUDA device is present")
    assert st == abi.RBR_ERR_CUDA and not h.value


def test_every_tunable_is_documented_and_accepted():
    """The tunables rbr_param_set and rbr_param_get accept (capi.cpp) are exactly the ones the
    header documents, each accepted by both calls."""
    import re
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    header = (root / "include" / "rbr_b200.h").read_text()
    block = header[header.index("Tunables of a context"):header.index("Results do not depend on them")]
    documented = set(re.findall(r'^ \*   "([a-z_0-9.]+)"', block, re.M))
    src = (root / "ray-based-rendering_b200" / "csrc" / "capi.cpp").read_text()
    setter = src[src.index("rbr_status rbr_param_set("):src.index("rbr_status rbr_param_get(")]
    getter = src[src.index("rbr_status rbr_param_get("):]
    getter = getter[:getter.index("\n}\n")]
    accepted_set = set(re.findall(r'n == "([a-z_0-9.]+)"', setter))
    accepted_get = set(re.findall(r'n == "([a-z_0-9.]+)"', getter))
    assert "pt.fetch" in documented and "trace.order" in documented
    assert accepted_set == documented, (accepted_set ^ documented)
    assert accepted_get == documented, (accepted_get ^ documented)
