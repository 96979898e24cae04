"""TEST INFRASTRUCTURE: ctypes access to the two CPU checkers of the GPU library.

  Restatement  oracle/_build/librbr_oracle.so  (oracle/rbr_oracle.c: a C restatement of the
               reference's hot path with the GPU library's counter RNG)
  Reference    oracle/_ref/librbr_ref.so       (the UNMODIFIED reference library compiled from
               its own sources by oracle/Makefile, plus oracle/ref_harness.cpp)

Only tests/, __graft_entry__.smoke() and bench.py's CPU arms import this module. Both libraries
are built by `make -C oracle` (the reference one only where the reference sources exist; the
built file travels with the repository).
"""
from __future__ import annotations

import ctypes as C
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
sys.path.insert(0, str(REPO / "ray-based-rendering_b200"))

from rbr_b200 import abi  # noqa: E402
from rbr_b200.abi import HIT_DTYPE, RAY_DTYPE  # noqa: E402

ORACLE_LIB = HERE / "_build" / "librbr_oracle.so"
REF_LIB = HERE / "_ref" / "librbr_ref.so"


def reference_dir() -> Path:
    """Where the reference's sources lie (only where they were cloned; never on the GPU box):
    the RBR_REFERENCE setting, the same one oracle/Makefile and adapters/Makefile read."""
    return Path(os.environ.get("RBR_REFERENCE", "/root/reference"))

P = C.c_void_p
_i64 = C.c_int64


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def have_reference() -> bool:
    return REF_LIB.exists()


# ------------------------------------------------------------------------------------------
class Restatement:
    """The C restatement (oracle/rbr_oracle.c)."""

    def __init__(self):
        if not ORACLE_LIB.exists():
            raise RuntimeError(f"{ORACLE_LIB} missing: run `make -C oracle`")
        L = C.CDLL(str(ORACLE_LIB))
        L.orc_scene_create.restype = P
        L.orc_scene_create.argtypes = [C.POINTER(abi.rbr_scene_desc)]
        L.orc_scene_destroy.argtypes = [P]
        L.orc_trace_closest.argtypes = [P, P, _i64, P, C.c_int]
        L.orc_trace_any.argtypes = [P, P, _i64, P, C.c_int]
        L.orc_bsdf_eval.argtypes = [C.POINTER(abi.rbr_material), _i64, P, P, P, P, P]
        L.orc_bsdf_sample.argtypes = [C.POINTER(abi.rbr_material), _i64, P, P, P]
        L.orc_light_sample.argtypes = [C.POINTER(abi.rbr_light), _i64, P, P, P]
        L.orc_camera_rays.argtypes = [C.POINTER(abi.rbr_camera), _i64, P, P]
        L.orc_power_heuristic.restype = C.c_float
        L.orc_power_heuristic.argtypes = [C.c_int, C.c_float, C.c_int, C.c_float]
        L.orc_philox.argtypes = [P, P, P]
        L.orc_render.argtypes = [P, C.POINTER(abi.rbr_camera), C.POINTER(abi.rbr_render_params), P, P, P, C.c_int]
        L.orc_path.argtypes = [P, C.POINTER(abi.rbr_camera), C.POINTER(abi.rbr_render_params), C.c_int, C.c_int,
                               C.c_uint32, P]
        L.orc_hg_eval.restype = C.c_float
        L.orc_hg_eval.argtypes = [C.c_float, P, P]
        L.orc_hg_sample.argtypes = [C.c_float, _i64, P, P, P]
        self.L = L

    def scene(self, scene):
        return _Handle(self.L.orc_scene_create, self.L.orc_scene_destroy, scene)

    def trace_closest(self, h, rays, threads=0):
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        out = np.zeros(len(rays), HIT_DTYPE)
        self.L.orc_trace_closest(h.h, _ptr(rays), len(rays), _ptr(out), threads)
        return out

    def trace_any(self, h, rays, threads=0):
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        out = np.zeros(len(rays), np.uint8)
        self.L.orc_trace_any(h.h, _ptr(rays), len(rays), _ptr(out), threads)
        return out

    def bsdf_eval(self, mat, wo, wi):
        wo, wi = _f(wo), _f(wi)
        n = len(wo)
        f = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        info = np.zeros(2, np.uint32)
        self.L.orc_bsdf_eval(C.byref(mat), n, _ptr(wo), _ptr(wi), _ptr(f), _ptr(pdf), _ptr(info))
        return f, pdf, info

    def bsdf_sample(self, mat, wo, u):
        wo, u = _f(wo), _f(u)
        out = np.zeros((len(wo), 8), np.float32)
        self.L.orc_bsdf_sample(C.byref(mat), len(wo), _ptr(wo), _ptr(u), _ptr(out))
        return out

    def light_sample(self, light, points, u):
        points, u = _f(points), _f(u)
        out = np.zeros((len(points), 9), np.float32)
        self.L.orc_light_sample(C.byref(light), len(points), _ptr(points), _ptr(u), _ptr(out))
        return out

    def camera_rays(self, cam, samples):
        samples = _f(samples)
        out = np.zeros((len(samples), 6), np.float32)
        self.L.orc_camera_rays(C.byref(cam), len(samples), _ptr(samples), _ptr(out))
        return out

    def power_heuristic(self, nf, fp, ng, gp):
        return self.L.orc_power_heuristic(nf, fp, ng, gp)

    def hg_eval(self, g, wo, wi):
        wo, wi = _f(wo), _f(wi)
        return np.array([self.L.orc_hg_eval(g, _ptr(wo[i]), _ptr(wi[i])) for i in range(len(wo))], np.float32)

    def hg_sample(self, g, wo, u):
        wo, u = _f(wo), _f(u)
        out = np.zeros((len(wo), 3), np.float32)
        self.L.orc_hg_sample(g, len(wo), _ptr(wo), _ptr(u), _ptr(out))
        return out

    def philox(self, ctr, key):
        c = np.ascontiguousarray(ctr, np.uint32)
        k = np.ascontiguousarray(key, np.uint32)
        o = np.zeros(4, np.uint32)
        self.L.orc_philox(_ptr(c), _ptr(k), _ptr(o))
        return o

    def render(self, h, cam, params, threads=0, moments=False):
        W, H = cam.width, cam.height
        mean = np.zeros((H, W, 3), np.float32)
        s = np.zeros((H, W, 3), np.float64) if moments else None
        q = np.zeros((H, W, 3), np.float64) if moments else None
        self.L.orc_render(h.h, C.byref(cam), C.byref(params), _ptr(mean), _ptr(s), _ptr(q), threads)
        return (mean, s, q) if moments else mean

    def path(self, h, cam, params, x, y, sample):
        out = np.zeros(3, np.float32)
        self.L.orc_path(h.h, C.byref(cam), C.byref(params), x, y, sample, _ptr(out))
        return out


# ------------------------------------------------------------------------------------------
class Reference:
    """The unmodified reference library behind oracle/ref_harness.cpp."""

    def __init__(self):
        if not REF_LIB.exists():
            raise RuntimeError(f"{REF_LIB} missing: run `make -C oracle ref` where the reference sources exist")
        L = C.CDLL(str(REF_LIB))
        L.ref_max_threads.restype = C.c_int
        L.ref_scene_create.restype = P
        L.ref_scene_create.argtypes = [C.POINTER(abi.rbr_scene_desc), C.c_int]
        L.ref_scene_destroy.argtypes = [P]
        L.ref_scene_set_medium.argtypes = [P, P, P, C.c_float]
        for n in ("ref_trace_closest", "ref_brute_closest"):
            getattr(L, n).argtypes = [P, P, _i64, P, C.c_int]
        for n in ("ref_trace_any", "ref_brute_any"):
            getattr(L, n).argtypes = [P, P, _i64, P, C.c_int]
        L.ref_hit_details.argtypes = [P, P, _i64, P]
        L.ref_world_bounds.argtypes = [P, P, P]
        L.ref_bsdf_eval.argtypes = [C.POINTER(abi.rbr_material), _i64, P, P, P, P, P]
        L.ref_bsdf_sample.argtypes = [C.POINTER(abi.rbr_material), _i64, P, P, P]
        L.ref_light_sample.argtypes = [C.POINTER(abi.rbr_light), _i64, P, P, P]
        L.ref_camera_setup.argtypes = [C.c_int, C.c_int, P, P, P, C.c_float, C.c_float, C.c_float,
                                       C.POINTER(abi.rbr_camera)]
        L.ref_camera_rays.argtypes = [C.POINTER(abi.rbr_camera), _i64, P, P]
        L.ref_render.argtypes = [P, C.POINTER(abi.rbr_camera), C.POINTER(abi.rbr_render_params), C.c_int, P,
                                 C.c_int]
        L.ref_render_moments.argtypes = [P, C.POINTER(abi.rbr_camera), C.POINTER(abi.rbr_render_params), C.c_int,
                                         C.c_uint64, P, P, C.c_int]
        L.ref_power_heuristic.restype = C.c_float
        L.ref_power_heuristic.argtypes = [C.c_int, C.c_float, C.c_int, C.c_float]
        L.ref_frame.argtypes = [P, P, P]
        L.ref_film_rgb8.argtypes = [P, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, P]
        L.ref_hg_eval.argtypes = [C.c_float, _i64, P, P, P]
        L.ref_hg_sample.argtypes = [C.c_float, _i64, P, P, P]
        L.ref_medium_sample.argtypes = [C.POINTER(abi.rbr_medium), _i64, P, P, P]
        self.L = L

    def max_threads(self):
        return self.L.ref_max_threads()

    def scene(self, scene, accel=0):
        return _Handle(lambda d: self.L.ref_scene_create(d, accel), self.L.ref_scene_destroy, scene)

    def trace_closest(self, h, rays, threads=0, brute=False):
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        out = np.zeros(len(rays), HIT_DTYPE)
        f = self.L.ref_brute_closest if brute else self.L.ref_trace_closest
        f(h.h, _ptr(rays), len(rays), _ptr(out), threads)
        return out

    def trace_any(self, h, rays, threads=0, brute=False):
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        out = np.zeros(len(rays), np.uint8)
        f = self.L.ref_brute_any if brute else self.L.ref_trace_any
        f(h.h, _ptr(rays), len(rays), _ptr(out), threads)
        return out

    def hit_details(self, h, rays):
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        out = np.zeros((len(rays), 10), np.float32)
        self.L.ref_hit_details(h.h, _ptr(rays), len(rays), _ptr(out))
        return out

    def world_bounds(self, h):
        lo = np.zeros(3, np.float32)
        hi = np.zeros(3, np.float32)
        self.L.ref_world_bounds(h.h, _ptr(lo), _ptr(hi))
        return lo, hi

    def bsdf_eval(self, mat, wo, wi):
        wo, wi = _f(wo), _f(wi)
        n = len(wo)
        f = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        info = np.zeros(2, np.uint32)
        self.L.ref_bsdf_eval(C.byref(mat), n, _ptr(wo), _ptr(wi), _ptr(f), _ptr(pdf), _ptr(info))
        return f, pdf, info

    def bsdf_sample(self, mat, wo, u):
        wo, u = _f(wo), _f(u)
        out = np.zeros((len(wo), 8), np.float32)
        self.L.ref_bsdf_sample(C.byref(mat), len(wo), _ptr(wo), _ptr(u), _ptr(out))
        return out

    def light_sample(self, light, points, u):
        points, u = _f(points), _f(u)
        out = np.zeros((len(points), 9), np.float32)
        self.L.ref_light_sample(C.byref(light), len(points), _ptr(points), _ptr(u), _ptr(out))
        return out

    def camera(self, width, height, position, look_at, up, fov, lens_radius=0.0, focal_distance=1.0):
        cam = abi.rbr_camera()
        p, t, u = _f(position), _f(look_at), _f(up)  # keep the arrays alive during the call
        self.L.ref_camera_setup(width, height, _ptr(p), _ptr(t), _ptr(u), fov, lens_radius, focal_distance,
                                C.byref(cam))
        return cam

    def camera_rays(self, cam, samples):
        samples = _f(samples)
        out = np.zeros((len(samples), 6), np.float32)
        self.L.ref_camera_rays(C.byref(cam), len(samples), _ptr(samples), _ptr(out))
        return out

    def render(self, h, cam, params, volumetric=False, threads=0):
        film = np.zeros((cam.height, cam.width, 3), np.float32)
        self.L.ref_render(h.h, C.byref(cam), C.byref(params), int(volumetric), _ptr(film), threads)
        return film

    def render_moments(self, h, cam, params, batch=0, volumetric=False, threads=0, acc=None):
        if acc is None:
            acc = (np.zeros((cam.height, cam.width, 3)), np.zeros((cam.height, cam.width, 3)))
        self.L.ref_render_moments(h.h, C.byref(cam), C.byref(params), int(volumetric), batch, _ptr(acc[0]),
                                  _ptr(acc[1]), threads)
        return acc

    def power_heuristic(self, nf, fp, ng, gp):
        return self.L.ref_power_heuristic(nf, fp, ng, gp)

    def frame(self, n):
        t = np.zeros(3, np.float32)
        b = np.zeros(3, np.float32)
        n = _f(n)
        self.L.ref_frame(_ptr(n), _ptr(t), _ptr(b))
        return t, b

    def hg_eval(self, g, wo, wi):
        wo, wi = _f(wo), _f(wi)
        out = np.zeros(len(wo), np.float32)
        self.L.ref_hg_eval(g, len(wo), _ptr(wo), _ptr(wi), _ptr(out))
        return out

    def film_rgb8(self, film, exposure=1.0, gamma=2.2, tonemap=False):
        film = _f(film)
        h, w = film.shape[:2]
        out = np.zeros((h, w, 3), np.uint8)
        self.L.ref_film_rgb8(_ptr(film), w, h, exposure, gamma, int(tonemap), _ptr(out))
        return out

    def obj_triangles(self, text: bytes):
        """(vertices [n, 9], normals [n, 9] or None) of the reference's ObjImporter::load +
        toPrimitives on `text` (run by oracle/_ref/ref_obj_dump), None when it fails."""
        import subprocess
        import tempfile

        with tempfile.NamedTemporaryFile(suffix=".obj") as f:
            f.write(text)
            f.flush()
            out = subprocess.run([str(HERE / "_ref" / "ref_obj_dump"), f.name], capture_output=True, check=True).stdout
        n = int(np.frombuffer(out[:8], np.int64)[0])
        if n < 0:
            return None
        has = int(np.frombuffer(out[8:12], np.int32)[0])
        data = np.frombuffer(out[12:], np.float32)
        v = data[:9 * n].reshape(n, 9).copy()
        return v, (data[9 * n:18 * n].reshape(n, 9).copy() if has else None)

    def hg_sample(self, g, wo, u):
        wo, u = _f(wo), _f(u)
        out = np.zeros((len(wo), 3), np.float32)
        self.L.ref_hg_sample(g, len(wo), _ptr(wo), _ptr(u), _ptr(out))
        return out

    def medium_sample(self, medium, max_dist, u):
        """(n, 5): t, weight[3], scattered (HomogeneousMedium::sampleDistance)."""
        md, u = _f(max_dist), _f(u)
        out = np.zeros((len(md), 5), np.float32)
        self.L.ref_medium_sample(C.byref(medium), len(md), _ptr(md), _ptr(u), _ptr(out))
        return out

    def set_medium(self, h, sigma_a, sigma_s, g):
        sa, ss = _f(sigma_a), _f(sigma_s)
        self.L.ref_scene_set_medium(h.h, _ptr(sa), _ptr(ss), g)


class _Handle:
    def __init__(self, create, destroy, scene):
        self._desc = scene.desc() if hasattr(scene, "desc") and callable(scene.desc) else scene
        self.h = create(C.byref(self._desc.desc))
        if not self.h:
            raise ValueError("scene creation failed (ids not a permutation?)")
        self._destroy = destroy

    def close(self):
        if self.h:
            self._destroy(self.h)
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
