"""Seeded synthetic scenes and ray sets for the hot path's workloads.

A `Scene` holds plain numpy arrays in the rbr_scene_desc layout (include/rbr_b200.h); the
same arrays feed the GPU library, the CPU restatement and the reference library, so every
side sees bit-identical inputs. Workloads (all seeded, no external data):

  cornell_box()        2x2x2 quad box, coloured walls, 0.5x0.5 ceiling light (AreaLight plus a
                       coincident emissive quad, emission (17,12,4)), two boxes rotated +-17 deg;
                       pinhole camera, fov 40, (0,1,3.5) -> (0,1,0).
  ray_query_scene()    icosphere subdivided 8 times (1,310,720 triangles), radius 10, radially
                       displaced by 4-octave value noise of amplitude 0.1 of the radius.
  uniform_rays()       origins uniform in a box, directions uniform on the sphere.
  ggx_scene()          256 spheres (radius U[0.1,0.5]) and a 2M-triangle displaced mound on a
                       ground quad; per-object random materials (20% glass); 2 quad area lights
                       with coincident emissive quads and a point light; thin-lens camera.

Radius 10 for the icosphere: triangle tests reject |e1 . (d x e2)| < 1e-4 (an absolute
EPSILON, src/geometry/triangle.cpp:12), which on a unit-radius level-8 icosphere culls every
triangle (2*area ~ 1.5e-5); at radius 10 only rays within ~4 degrees of grazing are culled.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import abi

F32 = np.float32


# ----------------------------------------------------------------------------------------
# float32 vector helpers that round like the reference's Vec3 (include/render/core/vector.h)
# ----------------------------------------------------------------------------------------
def _f(x):
    return np.asarray(x, dtype=F32)


def dot3(a, b):
    """Vec3::dot: (x*x' + y*y') + z*z' with float32 rounding at every step."""
    a = _f(a)
    b = _f(b)
    return (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]


def cross3(a, b):
    a = _f(a)
    b = _f(b)
    return np.stack(
        [
            a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
            a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
            a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0],
        ],
        axis=-1,
    ).astype(F32)


def normalize3(v):
    """Vec3::normalized: v * (1 / sqrt(dot(v, v))), zero for a zero vector."""
    v = _f(v)
    ln = np.sqrt(dot3(v, v)).astype(F32)
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = (F32(1.0) / ln).astype(F32)
        out = (v * inv[..., None]).astype(F32)
    return np.where((ln > 0)[..., None], out, F32(0)).astype(F32)


# ----------------------------------------------------------------------------------------
# Scene container
# ----------------------------------------------------------------------------------------
@dataclass
class Scene:
    """Primitives, materials and lights in the rbr_scene_desc layout.

    ids: global primitive index of every primitive of a type (Scene::primitives() order).
    """

    triangles: np.ndarray = field(default_factory=lambda: np.zeros((0, 9), F32))
    triangle_normals: np.ndarray | None = None
    triangle_materials: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))
    triangle_ids: np.ndarray | None = None
    spheres: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), F32))
    sphere_materials: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))
    sphere_ids: np.ndarray | None = None
    quads: np.ndarray = field(default_factory=lambda: np.zeros((0, 9), F32))
    quad_materials: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))
    quad_ids: np.ndarray | None = None
    planes: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), F32))
    plane_materials: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))
    plane_ids: np.ndarray | None = None
    materials: list = field(default_factory=list)  # list of dicts
    lights: list = field(default_factory=list)  # list of dicts
    background: tuple = (0.0, 0.0, 0.0)
    medium: dict | None = None  # sigma_a, sigma_s, g (a homogeneous medium filling all space)
    camera: object = None  # rbr_camera or None
    name: str = "scene"

    @property
    def num_primitives(self) -> int:
        return len(self.triangles) + len(self.spheres) + len(self.quads) + len(self.planes)

    def add_material(self, base_color=(0.8, 0.8, 0.8), metallic=0.0, roughness=1.0, ior=1.5,
                     transmission=0.0, emission=(0.0, 0.0, 0.0)) -> int:
        self.materials.append(dict(base_color=tuple(base_color), metallic=metallic, roughness=roughness,
                                   ior=ior, transmission=transmission, emission=tuple(emission)))
        return len(self.materials) - 1

    # Material presets (src/materials/material.cpp:9-55)
    def diffuse(self, albedo):
        return self.add_material(base_color=albedo, roughness=1.0, ior=1.0)

    def emissive(self, emission, intensity=1.0):
        return self.add_material(base_color=(0, 0, 0), ior=1.0, emission=tuple(F32(e) * F32(intensity) for e in emission))

    def area_light(self, position, u, v, color, intensity=1.0):
        self.lights.append(dict(type=abi.RBR_LIGHT_AREA, position=tuple(position), u=tuple(u), v=tuple(v),
                                color=tuple(color), intensity=float(intensity)))

    def point_light(self, position, color, intensity=1.0):
        self.lights.append(dict(type=abi.RBR_LIGHT_POINT, position=tuple(position), u=(0, 0, 0), v=(0, 0, 0),
                                color=tuple(color), intensity=float(intensity)))

    def add_mesh(self, vertices, normals, material: int):
        """Appends triangles ([n, 9] vertices, optional [n, 9] unit normals) with one material,
        as TriangleMesh::toPrimitives adds a mesh (src/geometry/mesh.cpp:14-38)."""
        v = np.asarray(vertices, F32).reshape(-1, 9)
        old = len(self.triangles)
        if normals is not None and old and self.triangle_normals is None:
            raise ValueError("mixing triangles with and without normals")
        self.triangles = np.concatenate([self.triangles.reshape(-1, 9), v]).astype(F32)
        if normals is not None:
            nn = np.asarray(normals, F32).reshape(-1, 9)
            self.triangle_normals = nn if self.triangle_normals is None else np.concatenate([self.triangle_normals, nn])
        elif self.triangle_normals is not None:
            raise ValueError("mixing triangles with and without normals")
        self.triangle_materials = np.concatenate([self.triangle_materials, np.full(len(v), material, np.uint32)])

    def set_medium(self, sigma_a, sigma_s, g=0.0):
        """SceneBuilder::medium (src/scene/scene_builder.cpp:102-105): a HomogeneousMedium."""
        self.medium = dict(sigma_a=tuple(sigma_a), sigma_s=tuple(sigma_s), g=float(g))

    def desc(self) -> "SceneDesc":
        return SceneDesc(self)


class SceneDesc:
    """An rbr_scene_desc that keeps the arrays it points to alive."""

    def __init__(self, s: Scene):
        def arr(a, dt, cols=None):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=dt)
            if cols is not None:
                a = a.reshape(-1, cols)
            return a

        self._keep = []

        def keep(a):
            self._keep.append(a)
            return a

        d = abi.rbr_scene_desc()
        tri = keep(arr(s.triangles, F32, 9))
        d.num_triangles = len(tri)
        d.triangle_vertices = abi.ptr(tri, C.c_float)
        d.triangle_normals = abi.ptr(keep(arr(s.triangle_normals, F32, 9)), C.c_float)
        d.triangle_materials = abi.ptr(keep(arr(s.triangle_materials, np.uint32)), C.c_uint32)
        d.triangle_ids = abi.ptr(keep(arr(s.triangle_ids, np.uint32)), C.c_uint32)
        sph = keep(arr(s.spheres, F32, 4))
        d.num_spheres = len(sph)
        d.spheres = abi.ptr(sph, C.c_float)
        d.sphere_materials = abi.ptr(keep(arr(s.sphere_materials, np.uint32)), C.c_uint32)
        d.sphere_ids = abi.ptr(keep(arr(s.sphere_ids, np.uint32)), C.c_uint32)
        qd = keep(arr(s.quads, F32, 9))
        d.num_quads = len(qd)
        d.quads = abi.ptr(qd, C.c_float)
        d.quad_materials = abi.ptr(keep(arr(s.quad_materials, np.uint32)), C.c_uint32)
        d.quad_ids = abi.ptr(keep(arr(s.quad_ids, np.uint32)), C.c_uint32)
        pl = keep(arr(s.planes, F32, 4))
        d.num_planes = len(pl)
        d.planes = abi.ptr(pl, C.c_float)
        d.plane_materials = abi.ptr(keep(arr(s.plane_materials, np.uint32)), C.c_uint32)
        d.plane_ids = abi.ptr(keep(arr(s.plane_ids, np.uint32)), C.c_uint32)
        mats = (abi.rbr_material * max(1, len(s.materials)))()
        for i, m in enumerate(s.materials):
            mats[i].base_color = abi.f3(m["base_color"])
            mats[i].metallic = m["metallic"]
            mats[i].roughness = m["roughness"]
            mats[i].ior = m["ior"]
            mats[i].transmission = m["transmission"]
            mats[i].emission = abi.f3(m["emission"])
        keep(mats)
        d.num_materials = len(s.materials)
        d.materials = C.cast(mats, C.POINTER(abi.rbr_material))
        lts = (abi.rbr_light * max(1, len(s.lights)))()
        for i, l in enumerate(s.lights):
            lts[i].type = l["type"]
            lts[i].position = abi.f3(l["position"])
            lts[i].u = abi.f3(l["u"])
            lts[i].v = abi.f3(l["v"])
            lts[i].color = abi.f3(l["color"])
            lts[i].intensity = l["intensity"]
        keep(lts)
        d.num_lights = len(s.lights)
        d.lights = C.cast(lts, C.POINTER(abi.rbr_light))
        d.background = abi.f3(s.background)
        if s.medium is not None:
            med = abi.rbr_medium()
            med.sigma_a = abi.f3(s.medium["sigma_a"])
            med.sigma_s = abi.f3(s.medium["sigma_s"])
            med.g = s.medium["g"]
            keep(med)
            d.medium = C.pointer(med)
        self.desc = d

    @property
    def ref(self):
        return C.byref(self.desc)


# ----------------------------------------------------------------------------------------
# Camera (CameraExtrinsics::lookAt, camera_extrinsics.h:28-45; fromVerticalFov,
# perspective_intrinsics.h:33-36), float32 arithmetic
# ----------------------------------------------------------------------------------------
def look_at_camera(width, height, position, target, up=(0.0, 1.0, 0.0), fov=60.0, lens_radius=0.0,
                   focal_distance=1.0, thin_lens=None) -> abi.rbr_camera:
    position = _f(position)
    forward = normalize3(_f(target) - position)
    r = cross3(forward, _f(up))
    if dot3(r, r) < F32(1e-12):
        alt = _f((0, 1, 0)) if abs(forward[1]) < F32(0.99) else _f((0, 0, 1))
        r = cross3(forward, alt)
    right = normalize3(r)
    cup = cross3(right, forward)
    pi = F32(3.14159265358979323846)
    rad = F32(F32(fov) * pi) / F32(180.0)
    f = F32(F32(0.5) * F32(height)) / F32(math.tan(float(F32(rad * F32(0.5)))))
    cam = abi.rbr_camera()
    cam.width, cam.height = int(width), int(height)
    if thin_lens is None:
        thin_lens = lens_radius > 0
    cam.model = abi.RBR_CAMERA_THIN_LENS if thin_lens else abi.RBR_CAMERA_PINHOLE
    cam.position = abi.f3(position)
    cam.forward = abi.f3(forward)
    cam.right = abi.f3(right)
    cam.up = abi.f3(cup)
    cam.fx = cam.fy = float(f)
    cam.cx = float(F32(0.5) * F32(width))
    cam.cy = float(F32(0.5) * F32(height))
    cam.lens_radius = float(lens_radius)
    cam.focal_distance = float(focal_distance)
    return cam


# ----------------------------------------------------------------------------------------
# Cornell box (cornell box configuration of the path-tracer workload)
# ----------------------------------------------------------------------------------------
def _box_quads(center, half, angle_deg):
    """Six quads (origin, u, v) of a box rotated about +y, outward normals u x v."""
    a = math.radians(angle_deg)
    ca, sa = math.cos(a), math.sin(a)

    def rot(p):
        x, y, z = p
        return np.array([ca * x + sa * z, y, -sa * x + ca * z])

    c = np.asarray(center, dtype=np.float64)
    hx, hy, hz = half
    ex, ey, ez = rot((2 * hx, 0, 0)), rot((0, 2 * hy, 0)), rot((0, 0, 2 * hz))
    p000 = c + rot((-hx, -hy, -hz))
    p100, p010, p001 = p000 + ex, p000 + ey, p000 + ez
    faces = [
        (p000, ez, ey),  # -x
        (p100, ey, ez),  # +x
        (p000, ex, ez),  # -y
        (p010, ez, ex),  # +y
        (p000, ey, ex),  # -z
        (p001, ex, ey),  # +z
    ]
    return [np.concatenate([o, u, v]) for o, u, v in faces]


def cornell_box(width=256, height=256) -> Scene:
    s = Scene(name="cornell")
    white = s.diffuse((0.73, 0.73, 0.73))
    red = s.diffuse((0.65, 0.05, 0.05))
    green = s.diffuse((0.12, 0.45, 0.15))
    light = s.emissive((17.0, 12.0, 4.0))
    quads, mats = [], []

    def q(o, u, v, m):
        quads.append(np.concatenate([o, u, v]))
        mats.append(m)

    q((-1, 0, -1), (2, 0, 0), (0, 0, 2), white)  # floor
    q((-1, 2, -1), (2, 0, 0), (0, 0, 2), white)  # ceiling
    q((-1, 0, -1), (2, 0, 0), (0, 2, 0), white)  # back wall
    q((-1, 0, -1), (0, 0, 2), (0, 2, 0), red)  # left wall
    q((1, 0, -1), (0, 0, 2), (0, 2, 0), green)  # right wall
    q((-0.25, 1.99, -0.25), (0.5, 0, 0), (0, 0, 0.5), light)  # emissive quad under the area light
    for face in _box_quads((0.33, 0.3, 0.3), (0.3, 0.3, 0.3), -17.0):  # short box
        q(face[:3], face[3:6], face[6:], white)
    for face in _box_quads((-0.33, 0.6, -0.3), (0.3, 0.6, 0.3), 17.0):  # tall box
        q(face[:3], face[3:6], face[6:], white)
    s.quads = np.asarray(quads, dtype=F32)
    s.quad_materials = np.asarray(mats, dtype=np.uint32)
    # AreaLight is centre-based (area_light.cpp:13-16); u x v = -y faces the room
    s.area_light((0.0, 1.99, 0.0), (0.5, 0, 0), (0, 0, 0.5), (17.0, 12.0, 4.0), 1.0)
    s.camera = look_at_camera(width, height, (0.0, 1.0, 3.5), (0.0, 1.0, 0.0), (0.0, 1.0, 0.0), 40.0)
    return s


def foggy_cornell_box(width=256, height=256, sigma_t=0.1, albedo=0.8, g=0.5, point_light=True) -> Scene:
    """The Cornell box filled with a homogeneous medium: sigma_t 0.1, single-scattering albedo
    0.8 (sigma_s 0.08, sigma_a 0.02 per channel), Henyey-Greenstein g = 0.5, rendered with the
    volumetric path integrator. The volumetric integrator's next-event estimation from scatter
    points reaches point lights only (volumetric_path_integrator.cpp:97-116), so a point light
    below the ceiling lamp lights the fog directly."""
    s = cornell_box(width, height)
    ss = F32(sigma_t) * F32(albedo)
    sa = F32(sigma_t) - ss
    s.set_medium((sa, sa, sa), (ss, ss, ss), g)
    if point_light:
        s.point_light((0.0, 1.8, 0.0), (1.0, 0.85, 0.6), 2.0)
    return s


# ----------------------------------------------------------------------------------------
# Icosphere + value noise (ray-query workload)
# ----------------------------------------------------------------------------------------
def icosphere(level: int):
    """Unit icosphere: vertices (V,3) float64 and faces (F,3) int64, F = 20 * 4**level."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array(
        [[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
         [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array(
        [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
         [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
         [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    for _ in range(level):
        nv = len(v)
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        lo, hi = np.minimum(e[:, 0], e[:, 1]), np.maximum(e[:, 0], e[:, 1])
        key = lo * nv + hi
        uniq, inv = np.unique(key, return_inverse=True)
        a, b = uniq // nv, uniq % nv
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        v = np.concatenate([v, mid])
        nf = len(f)
        m01, m12, m20 = nv + inv[:nf], nv + inv[nf:2 * nf], nv + inv[2 * nf:]
        f = np.concatenate([
            np.stack([f[:, 0], m01, m20], 1),
            np.stack([f[:, 1], m12, m01], 1),
            np.stack([f[:, 2], m20, m12], 1),
            np.stack([m01, m12, m20], 1),
        ])
    return v, f


def _hash3(ix, iy, iz, seed):
    with np.errstate(over="ignore"):
        return _hash3_impl(ix, iy, iz, seed)


def _hash3_impl(ix, iy, iz, seed):
    h = (ix.astype(np.uint64) * np.uint64(0x8DA6B343) ^ iy.astype(np.uint64) * np.uint64(0xD8163841)
         ^ iz.astype(np.uint64) * np.uint64(0xCB1AB31F) ^ np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15))
    h &= np.uint64(0xFFFFFFFFFFFFFFFF)
    h ^= h >> np.uint64(33)
    h = (h * np.uint64(0xFF51AFD7ED558CCD)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    h ^= h >> np.uint64(33)
    h = (h * np.uint64(0xC4CEB9FE1A85EC53)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    h ^= h >> np.uint64(33)
    return (h >> np.uint64(11)).astype(np.float64) * (2.0 / 9007199254740992.0) - 1.0


def value_noise(p: np.ndarray, seed: int) -> np.ndarray:
    """Trilinear value noise in [-1, 1] with smoothstep weights, lattice values from a hash."""
    i = np.floor(p)
    fr = p - i
    w = fr * fr * (3.0 - 2.0 * fr)
    i = i.astype(np.int64)
    out = np.zeros(len(p))
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                val = _hash3(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz, seed)
                wx = w[:, 0] if dx else 1 - w[:, 0]
                wy = w[:, 1] if dy else 1 - w[:, 1]
                wz = w[:, 2] if dz else 1 - w[:, 2]
                out += val * wx * wy * wz
    return out


def fbm(p: np.ndarray, octaves: int = 4, seed: int = 0, base_frequency: float = 4.0) -> np.ndarray:
    """Sum of octaves of value noise (frequency x2, amplitude /2), normalised to [-1, 1]."""
    total = np.zeros(len(p))
    amp, freq, norm = 1.0, base_frequency, 0.0
    for o in range(octaves):
        total += amp * value_noise(p * freq, seed * 131 + o)
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return total / norm


def displaced_icosphere(level=8, radius=10.0, amplitude=0.1, octaves=4, seed=0):
    v, f = icosphere(level)
    r = radius * (1.0 + amplitude * fbm(v, octaves=octaves, seed=seed))
    pos = (v * r[:, None]).astype(F32)
    return pos, f


def ray_query_scene(level=8, radius=10.0, seed=0) -> Scene:
    pos, f = displaced_icosphere(level=level, radius=radius, seed=seed)
    s = Scene(name=f"icosphere{level}")
    m = s.diffuse((0.7, 0.7, 0.7))
    s.triangles = np.ascontiguousarray(pos[f].reshape(-1, 9))
    s.triangle_materials = np.full(len(f), m, np.uint32)
    return s


def scene_bounds(s: Scene):
    pts = [s.triangles.reshape(-1, 3)]
    if len(s.spheres):
        c, r = s.spheres[:, :3], s.spheres[:, 3:4]
        pts += [c - r, c + r]
    if len(s.quads):
        o, u, v = s.quads[:, :3], s.quads[:, 3:6], s.quads[:, 6:9]
        pts += [o, o + u, o + v, o + u + v]
    p = np.concatenate([x for x in pts if len(x)]) if any(len(x) for x in pts) else np.zeros((1, 3), F32)
    return p.min(0).astype(F32), p.max(0).astype(F32)


def uniform_sphere_dirs(u1: np.ndarray, u2: np.ndarray) -> np.ndarray:
    """sampling::uniformSphere (include/render/core/sampler.h:58-63) in float32."""
    u1 = _f(u1)
    u2 = _f(u2)
    z = F32(1.0) - F32(2.0) * u1
    r = np.sqrt(np.maximum(F32(0.0), F32(1.0) - z * z)).astype(F32)
    phi = (F32(2.0) * F32(3.14159265358979323846)) * u2
    d = np.stack([r * np.cos(phi).astype(F32), r * np.sin(phi).astype(F32), z], 1).astype(F32)
    return normalize3(d)  # a render::Ray normalises its direction


def uniform_rays(n: int, lo, hi, seed=0, tmax=np.inf) -> np.ndarray:
    """n rays: origins uniform in [lo, hi], directions uniform on the sphere (seeded)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    lo, hi = _f(lo), _f(hi)
    o = (lo + rng.random((n, 3), dtype=F32) * (hi - lo)).astype(F32)
    d = uniform_sphere_dirs(rng.random(n, dtype=F32), rng.random(n, dtype=F32))
    return abi.make_rays(o, d, tmax)


# ----------------------------------------------------------------------------------------
# Random worlds and rays in the shape of the reference's accelerator tests
# (tests/test_accelerators.cpp:37-55 and :84-93): spheres and triangles in [-10,10]^3,
# 20 axis-aligned flat triangles, optionally an infinite plane y = -12; a third of the rays
# axis-aligned along z, every 7th (of the rest) with a zero y component, every 4th a finite
# segment with tmax in [0.5, 40].
# ----------------------------------------------------------------------------------------
def random_world(n_spheres: int, n_triangles: int, with_plane: bool = False, seed: int = 0,
                 flat_triangles: int = 20, n_quads: int = 0) -> Scene:
    rng = np.random.default_rng(seed)
    s = Scene(name=f"world{n_spheres}_{n_triangles}{'_plane' if with_plane else ''}")
    m = s.diffuse((0.5, 0.5, 0.5))
    pos = lambda *sh: rng.uniform(-10.0, 10.0, sh).astype(F32)
    size = lambda *sh: rng.uniform(0.1, 1.5, sh).astype(F32)
    sph = np.concatenate([pos(n_spheres, 3), size(n_spheres, 1)], 1) if n_spheres else np.zeros((0, 4), F32)
    c = pos(n_triangles, 1, 3)
    tri = (c + (size(n_triangles, 3, 3) - F32(0.8))).astype(F32).reshape(-1, 9)
    flat = []
    for _ in range(flat_triangles):
        z, x, y = pos(3)
        flat.append([x, y, z, x + 2, y, z, x, y + 2, z])
    tri = np.concatenate([tri, np.asarray(flat, F32).reshape(-1, 9)]).astype(F32)
    s.triangles = np.ascontiguousarray(tri)
    s.triangle_materials = np.full(len(tri), m, np.uint32)
    s.spheres = np.ascontiguousarray(sph)
    s.sphere_materials = np.full(len(sph), m, np.uint32)
    # the reference test adds spheres first, then triangles, then the plane
    n_sph = len(sph)
    s.sphere_ids = np.arange(n_sph, dtype=np.uint32)
    s.triangle_ids = np.arange(n_sph, n_sph + len(tri), dtype=np.uint32)
    nxt = n_sph + len(tri)
    if n_quads:  # tilted quads: origin in the box, u = (a, 0, 0.3), v = (0, b, b)
        o = pos(n_quads, 3)
        a, b = size(n_quads), size(n_quads)
        z = np.zeros(n_quads, F32)
        u = np.stack([a, z, np.full(n_quads, 0.3, F32)], 1)
        v = np.stack([z, b, b], 1)
        s.quads = np.ascontiguousarray(np.concatenate([o, u, v], 1).astype(F32))
        s.quad_materials = np.full(n_quads, m, np.uint32)
        s.quad_ids = np.arange(nxt, nxt + n_quads, dtype=np.uint32)
        nxt += n_quads
    if with_plane:
        s.planes = np.array([[0.0, 1.0, 0.0, 12.0]], F32)  # Plane(Vec3(0,1,0), 12): y = -12
        s.plane_materials = np.array([m], np.uint32)
        s.plane_ids = np.array([nxt], np.uint32)
    return s


def random_test_rays(n: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    o = rng.uniform(-14.0, 14.0, (n, 3)).astype(F32)
    d = rng.uniform(-1.0, 1.0, (n, 3)).astype(F32)
    i = np.arange(n)
    axis = i % 3 == 0
    d[axis] = 0.0
    d[axis, 2] = np.where(i[axis] % 2 == 1, 1.0, -1.0)
    flat = (~axis) & (i % 7 == 0)
    d[flat, 1] = 0.0
    keep = np.sqrt(dot3(d, d)) >= F32(1e-3)
    d = normalize3(d)
    tmax = np.full(n, np.inf, F32)
    seg = i % 4 == 0
    tmax[seg] = rng.uniform(0.5, 40.0, seg.sum()).astype(F32)
    rays = abi.make_rays(o[keep], d[keep], tmax[keep])
    return rays


# ----------------------------------------------------------------------------------------
# GGX material scene
# ----------------------------------------------------------------------------------------
def _random_material(s: Scene, rng):
    base = tuple(float(x) for x in rng.random(3))
    rough = float(rng.uniform(0.05, 1.0))
    if rng.random() < 0.2:  # glass
        return s.add_material(base_color=base, metallic=0.0, roughness=rough, ior=1.5, transmission=1.0)
    metallic = float(rng.integers(0, 2))
    return s.add_material(base_color=base, metallic=metallic, roughness=rough, ior=1.5, transmission=0.0)


def mound_mesh(n=1000, size=8.0, height=2.0, seed=0):
    """n x n grid of quads split into 2*n*n triangles, displaced into a noisy mound."""
    xs = np.linspace(-size / 2, size / 2, n + 1)
    X, Z = np.meshgrid(xs, xs, indexing="ij")
    r2 = (X * X + Z * Z) / (size * size / 16.0)
    p = np.stack([X.ravel(), np.zeros(X.size), Z.ravel()], 1) * 0.5
    Y = height * np.exp(-r2) * (1.0 + 0.25 * fbm(p, octaves=4, seed=seed + 7, base_frequency=1.0).reshape(X.shape))
    Y = np.maximum(Y, 0.0) + 1e-3
    V = np.stack([X, Y, Z], -1).reshape(-1, 3).astype(F32)
    i = np.arange(n)
    a = (i[:, None] * (n + 1) + i[None, :]).ravel()
    b, c, d = a + 1, a + (n + 1), a + (n + 2)
    f = np.concatenate([np.stack([a, b, d], 1), np.stack([a, d, c], 1)])
    return V, f


def ggx_scene(width=1920, height=1080, n_spheres=256, mesh_n=1000, seed=0) -> Scene:
    rng = np.random.default_rng(seed)
    s = Scene(name="ggx")
    ground = s.diffuse((0.5, 0.5, 0.5))
    # ground: a large quad (bounded) instead of an infinite Plane
    quads = [np.array([-20, 0, -20, 40, 0, 0, 0, 0, 40], F32)]
    qmats = [ground]
    # lights: 2 area lights facing down + coincident emissive quads, 1 point light
    for pos, col in (((-3.0, 7.0, 2.0), (12.0, 10.0, 8.0)), ((4.0, 6.0, -2.0), (6.0, 8.0, 12.0))):
        u, v = (2.0, 0.0, 0.0), (0.0, 0.0, 2.0)
        s.area_light(pos, u, v, col, 1.0)
        corner = np.array(pos) - 0.5 * np.array(u) - 0.5 * np.array(v)
        quads.append(np.concatenate([corner, u, v]).astype(F32))
        qmats.append(s.emissive(col))
    s.point_light((0.0, 5.0, 6.0), (1.0, 1.0, 1.0), 20.0)
    # mound mesh
    V, f = mound_mesh(n=mesh_n, seed=seed)
    s.triangles = np.ascontiguousarray(V[f].reshape(-1, 9))
    s.triangle_materials = np.full(len(f), _random_material(s, rng), np.uint32)
    # spheres resting on the ground
    sph = np.zeros((n_spheres, 4), F32)
    smat = np.zeros(n_spheres, np.uint32)
    for k in range(n_spheres):
        r = rng.uniform(0.1, 0.5)
        while True:
            x, z = rng.uniform(-9, 9, 2)
            if x * x + z * z > 16.0:  # outside the mound
                break
        sph[k] = (x, r, z, r)
        smat[k] = _random_material(s, rng)
    s.spheres = sph
    s.sphere_materials = smat
    s.quads = np.asarray(quads, F32)
    s.quad_materials = np.asarray(qmats, np.uint32)
    pos, tgt = (0.0, 3.0, 14.0), (0.0, 0.8, 0.0)
    dist = float(np.linalg.norm(np.subtract(tgt, pos)))
    s.camera = look_at_camera(width, height, pos, tgt, (0, 1, 0), 40.0, lens_radius=0.05, focal_distance=dist)
    return s


def ggx_variant(base: Scene, seed: int) -> Scene:
    """A seeded material and light perturbation of a GGX scene with the same geometry: base
    colours scaled by U[0.7, 1.3] per channel (clamped to 1), roughness shifted by U[-0.1, 0.1]
    (kept in [0.05, 1]), light intensities scaled by U[0.5, 1.5] and area-light colours tinted."""
    import copy

    rng = np.random.default_rng(1000 + seed)
    v = copy.copy(base)
    v.materials = []
    for m in base.materials:
        m = dict(m)
        if max(m["emission"]) <= 0.0:
            m["base_color"] = tuple(float(min(1.0, c * rng.uniform(0.7, 1.3))) for c in m["base_color"])
            m["roughness"] = float(np.clip(m["roughness"] + rng.uniform(-0.1, 0.1), 0.05, 1.0))
        v.materials.append(m)
    v.lights = []
    for l in base.lights:
        l = dict(l)
        l["intensity"] = float(l["intensity"] * rng.uniform(0.5, 1.5))
        if l["type"] == abi.RBR_LIGHT_AREA:
            l["color"] = tuple(float(c * rng.uniform(0.8, 1.2)) for c in l["color"])
        v.lights.append(l)
    return v


def square_camera(cam: abi.rbr_camera, size: int) -> abi.rbr_camera:
    """The same camera with a size x size film and the vertical field of view kept."""
    c = abi.rbr_camera()
    C.memmove(C.byref(c), C.byref(cam), C.sizeof(cam))
    scale = size / cam.height
    c.width = c.height = size
    c.fx = cam.fx * scale
    c.fy = cam.fy * scale
    c.cx = size / 2.0
    c.cy = size / 2.0
    return c
