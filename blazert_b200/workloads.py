"""Seeded synthetic scenes and ray batches for the closest-hit workloads.

No public dataset is involved: every workload is generated here from a recorded seed, so the
GPU path, the CPU oracle and the CPU baseline all consume byte-identical float64 arrays.

Workloads (names used by bench.py and the tests):

* ``icosphere_pinhole``  -- unit icosphere subdivided 4 times (5,120 triangles, 5,112 vertices,
  built like the reference's benchmark helper benchmarks/benchmark_helper/OriginSphere.h:12-119),
  512 x 512 pinhole rays from (0, 0, 3), 60 degree vertical field of view.
* ``mixed_primitives``   -- 10,000 spheres, 1,000 cylinders, 100 finite planes in
  [-100, 100]^3; 1,048,576 incoherent rays from [-120, 120]^3 with isotropic directions.
* ``heightfield``        -- 1024 x 1024 vertex grid over [0, 1000]^2 (2,093,058 triangles),
  6-octave value-noise fBm heights; secondary rays leaving the surface (cosine-weighted).
* ``batched_icospheres`` -- 256 radially perturbed icospheres (levels 3-7) with ray batches of
  log-uniform size.
* ``adjoint_scene``      -- perturbed level-6 icosphere with 10,000 extra split triangles plus
  500 spheres, rays from a radius-4 sphere toward the unit ball.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

KINDS = ("mesh", "spheres", "planes", "cylinders")


@dataclass
class SceneSpec:
    """Geometry of one scene, in the order the kinds are added (the order fixes geom ids)."""

    order: List[str] = field(default_factory=list)
    mesh: Optional[Dict[str, np.ndarray]] = None
    spheres: Optional[Dict[str, np.ndarray]] = None
    planes: Optional[Dict[str, np.ndarray]] = None
    cylinders: Optional[Dict[str, np.ndarray]] = None

    def add_mesh(self, vertices, faces):
        self.mesh = dict(vertices=np.ascontiguousarray(vertices, np.float64).reshape(-1, 3),
                         faces=np.ascontiguousarray(faces, np.uint32).reshape(-1, 3))
        self.order.append("mesh")
        return self

    def add_spheres(self, centers, radii):
        self.spheres = dict(centers=np.ascontiguousarray(centers, np.float64).reshape(-1, 3),
                            radii=np.ascontiguousarray(radii, np.float64).reshape(-1))
        self.order.append("spheres")
        return self

    def add_planes(self, centers, dxs, dys, rotations):
        self.planes = dict(centers=np.ascontiguousarray(centers, np.float64).reshape(-1, 3),
                           dxs=np.ascontiguousarray(dxs, np.float64).reshape(-1),
                           dys=np.ascontiguousarray(dys, np.float64).reshape(-1),
                           rotations=np.ascontiguousarray(rotations, np.float64).reshape(-1, 3, 3))
        self.order.append("planes")
        return self

    def add_cylinders(self, centers, semi_axes_a, semi_axes_b, heights, rotations):
        self.cylinders = dict(
            centers=np.ascontiguousarray(centers, np.float64).reshape(-1, 3),
            semi_axes_a=np.ascontiguousarray(semi_axes_a, np.float64).reshape(-1),
            semi_axes_b=np.ascontiguousarray(semi_axes_b, np.float64).reshape(-1),
            heights=np.ascontiguousarray(heights, np.float64).reshape(-1),
            rotations=np.ascontiguousarray(rotations, np.float64).reshape(-1, 3, 3))
        self.order.append("cylinders")
        return self

    def nbytes(self):
        tot = 0
        for k in KINDS:
            d = getattr(self, k)
            if d:
                tot += sum(v.nbytes for v in d.values())
        return tot


@dataclass
class RayBatch:
    origins: np.ndarray      # n x 3 float64
    directions: np.ndarray   # n x 3 float64 (need not be unit length)
    tmin: Optional[np.ndarray] = None
    tmax: Optional[np.ndarray] = None

    @property
    def n(self):
        return int(self.origins.shape[0])

    def slice(self, a, b):
        return RayBatch(self.origins[a:b], self.directions[a:b],
                        None if self.tmin is None else self.tmin[a:b],
                        None if self.tmax is None else self.tmax[a:b])


@dataclass
class Workload:
    name: str
    scene: SceneSpec
    rays: RayBatch
    meta: dict = field(default_factory=dict)


# ------------------------------------------------------------------------------------ helpers
def _normalize_rows(v):
    """Row-wise v * (1 / |v|) with |v| = sqrt((x*x + y*y) + z*z): the vector-normalisation
    order used throughout this package."""
    x, y, z = v[:, 0], v[:, 1], v[:, 2]
    n = np.sqrt((x * x + y * y) + z * z)
    il = np.where(n != 0.0, 1.0 / np.where(n != 0.0, n, 1.0), 0.0)
    return v * il[:, None]


def icosphere(level: int):
    """Unit icosphere with the vertex and face order of the reference's OriginSphere helper
    (benchmarks/benchmark_helper/OriginSphere.h:12-119): the golden ratio computed in float32,
    midpoint vertices appended per triangle and edge without de-duplication (so level k has
    12 + 3 * sum_{i<k} 20 * 4^i vertices), and four children per triangle in the order
    (f0, f3, f5), (f3, f1, f4), (f4, f2, f5), (f3, f4, f5)."""
    t = float((np.float32(1.0) + np.sqrt(np.float32(5.0))) / np.float32(2.0))
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                  [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]],
                 dtype=np.float64)
    v = _normalize_rows(v)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9],
                  [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2],
                  [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10],
                  [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    for _ in range(level):
        nv, nf = v.shape[0], f.shape[0]
        v0, v1, v2 = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
        m01 = _normalize_rows((v0 + v1) * 0.5)
        m12 = _normalize_rows((v1 + v2) * 0.5)
        m20 = _normalize_rows((v2 + v0) * 0.5)
        newv = np.stack([m01, m12, m20], axis=1).reshape(-1, 3)
        base = nv + 3 * np.arange(nf)
        f3, f4, f5 = base, base + 1, base + 2
        f0, f1, f2 = f[:, 0], f[:, 1], f[:, 2]
        f = np.stack([np.stack([f0, f3, f5], 1), np.stack([f3, f1, f4], 1),
                      np.stack([f4, f2, f5], 1), np.stack([f3, f4, f5], 1)], axis=1).reshape(-1, 3)
        v = np.concatenate([v, newv], axis=0)
    return np.ascontiguousarray(v), np.ascontiguousarray(f.astype(np.uint32))


def rotation_to(axis):
    """Rotation matrices R (n x 3 x 3, row-major) with R @ e_z = axis, by the Rodrigues formula
    about e_z x axis (the construction of test/test_helpers.h:438-451 with the angle between
    e_z and the axis)."""
    axis = np.asarray(axis, np.float64).reshape(-1, 3)
    n = axis.shape[0]
    ez = np.array([0.0, 0.0, 1.0])
    k = np.cross(np.broadcast_to(ez, axis.shape), axis)
    s = np.linalg.norm(k, axis=1)
    c = axis[:, 2]
    R = np.zeros((n, 3, 3))
    for i in range(n):
        if s[i] < 1e-12:
            R[i] = np.eye(3) if c[i] > 0 else np.diag([1.0, -1.0, -1.0])
            continue
        kk = k[i] / s[i]
        ang = math.atan2(s[i], c[i])
        K = np.array([[0, -kk[2], kk[1]], [kk[2], 0, -kk[0]], [-kk[1], kk[0], 0]])
        R[i] = np.eye(3) + math.sin(ang) * K + (1 - math.cos(ang)) * (K @ K)
    return R


def _unit_sphere(rng, n):
    g = rng.standard_normal((n, 3))
    return g / np.linalg.norm(g, axis=1, keepdims=True)


# ------------------------------------------------------------------------------------ workloads
def icosphere_pinhole(level=4, width=512, height=512, fov_deg=60.0, n_rays=None):
    if n_rays:  # square image with about n_rays pixels
        width = height = max(1, int(round(math.sqrt(n_rays))))
    verts, faces = icosphere(level)
    scene = SceneSpec().add_mesh(verts, faces)
    tan = math.tan(math.radians(fov_deg) / 2.0)
    i = np.arange(width, dtype=np.float64)
    j = np.arange(height, dtype=np.float64)
    u = (2.0 * (i + 0.5) / width - 1.0) * tan
    v = (1.0 - 2.0 * (j + 0.5) / height) * tan
    U, V = np.meshgrid(u, v)  # row-major over pixels (j, i)
    d = np.stack([U.ravel(), V.ravel(), -np.ones(width * height)], axis=1)
    d = d / np.linalg.norm(d, axis=1, keepdims=True)
    o = np.broadcast_to(np.array([0.0, 0.0, 3.0]), d.shape).copy()
    rays = RayBatch(o, np.ascontiguousarray(d), np.zeros(d.shape[0]),
                    np.full(d.shape[0], np.inf))
    return Workload("icosphere_pinhole", scene, rays,
                    dict(level=level, triangles=int(faces.shape[0]), width=width, height=height))


def mixed_primitives(n_rays=1 << 20, n_spheres=10_000, n_cylinders=1_000, n_planes=100, seed=2):
    rng = np.random.Generator(np.random.PCG64(seed))
    sc = rng.uniform(-100.0, 100.0, (n_spheres, 3))
    sr = np.exp(rng.uniform(math.log(0.1), math.log(2.0), n_spheres))
    cc = rng.uniform(-100.0, 100.0, (n_cylinders, 3))
    cax = _unit_sphere(rng, n_cylinders)
    crad = rng.uniform(0.1, 1.0, n_cylinders)
    chalf = rng.uniform(0.5, 5.0, n_cylinders)
    pc = rng.uniform(-100.0, 100.0, (n_planes, 3))
    pn = _unit_sphere(rng, n_planes)
    pdx = rng.uniform(1.0, 20.0, n_planes)
    pdy = rng.uniform(1.0, 20.0, n_planes)
    scene = SceneSpec()
    scene.add_spheres(sc, sr)
    scene.add_cylinders(cc, crad, crad, 2.0 * chalf, rotation_to(cax))
    scene.add_planes(pc, pdx, pdy, rotation_to(pn))
    o = rng.uniform(-120.0, 120.0, (n_rays, 3))
    d = _unit_sphere(rng, n_rays)
    rays = RayBatch(o, d, np.zeros(n_rays), np.full(n_rays, np.inf))
    return Workload("mixed_primitives", scene, rays,
                    dict(spheres=n_spheres, cylinders=n_cylinders, planes=n_planes, seed=seed))


def _value_noise(x, y, rng_seed, octave):
    """Value noise in [-1, 1]: seeded random values on the integer lattice, smoothstep blend."""
    rng = np.random.Generator(np.random.PCG64([rng_seed, octave]))
    ix, iy = np.floor(x).astype(np.int64), np.floor(y).astype(np.int64)
    fx, fy = x - ix, y - iy
    size = int(max(ix.max(), iy.max())) + 2
    lattice = rng.uniform(-1.0, 1.0, (size + 1, size + 1))
    sx, sy = fx * fx * (3 - 2 * fx), fy * fy * (3 - 2 * fy)
    a = lattice[ix, iy] + sx * (lattice[ix + 1, iy] - lattice[ix, iy])
    b = lattice[ix, iy + 1] + sx * (lattice[ix + 1, iy + 1] - lattice[ix, iy + 1])
    return a + sy * (b - a)


def heightfield_mesh(n=1024, extent=1000.0, amplitude=100.0, octaves=6, lacunarity=2.0, gain=0.5,
                     base_frequency=4.0 / 1000.0, seed=3):
    """n x n vertex grid over [0, extent]^2, heights from fBm value noise; two triangles per
    quad with a fixed diagonal: 2 (n-1)^2 triangles."""
    xs = np.linspace(0.0, extent, n)
    X, Y = np.meshgrid(xs, xs, indexing="xy")
    Z = np.zeros_like(X)
    amp, freq, norm = 1.0, base_frequency, 0.0
    for o in range(octaves):
        Z += amp * _value_noise(X * freq, Y * freq, seed, o)
        norm += amp
        amp *= gain
        freq *= lacunarity
    Z *= amplitude / norm
    v = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    j, i = np.meshgrid(np.arange(n - 1), np.arange(n - 1), indexing="ij")
    a = (j * n + i).ravel()
    f = np.concatenate([np.stack([a, a + 1, a + n + 1], 1), np.stack([a, a + n + 1, a + n], 1)])
    f = f.reshape(2, -1, 3).transpose(1, 0, 2).reshape(-1, 3)  # interleave the two per quad
    return np.ascontiguousarray(v), np.ascontiguousarray(f.astype(np.uint32))


def _cosine_dirs(rng, normals):
    """Cosine-weighted directions about each unit normal."""
    n = normals.shape[0]
    r1, r2 = rng.random(n), rng.random(n)
    phi = 2.0 * np.pi * r1
    sr = np.sqrt(r2)
    local = np.stack([sr * np.cos(phi), sr * np.sin(phi), np.sqrt(1.0 - r2)], 1)
    # orthonormal frame (t, b, n) per normal
    helper = np.where(np.abs(normals[:, 2:3]) < 0.9, [[0.0, 0.0, 1.0]], [[1.0, 0.0, 0.0]])
    t = np.cross(helper, normals)
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    b = np.cross(normals, t)
    return local[:, :1] * t + local[:, 1:2] * b + local[:, 2:3] * normals


def heightfield(n_rays=1 << 23, grid=1024, seed=3):
    verts, faces = heightfield_mesh(grid, seed=seed)
    scene = SceneSpec().add_mesh(verts, faces)
    rng = np.random.Generator(np.random.PCG64(seed + 1000))
    v0, v1, v2 = verts[faces[:, 0]], verts[faces[:, 1]], verts[faces[:, 2]]
    cr = np.cross(v1 - v0, v2 - v0)
    area = 0.5 * np.linalg.norm(cr, axis=1)
    nf = cr / (2.0 * area[:, None])
    nf *= np.sign(nf[:, 2:3])  # oriented +z
    cdf = np.cumsum(area)
    tri = np.minimum(np.searchsorted(cdf, rng.random(n_rays) * cdf[-1]), len(area) - 1)
    r1, r2 = np.sqrt(rng.random(n_rays)), rng.random(n_rays)
    p = ((1 - r1)[:, None] * v0[tri] + (r1 * (1 - r2))[:, None] * v1[tri]
         + (r1 * r2)[:, None] * v2[tri])
    nrm = nf[tri]
    o = p + 1e-6 * nrm
    d = _cosine_dirs(rng, nrm)
    rays = RayBatch(np.ascontiguousarray(o), np.ascontiguousarray(d), np.zeros(n_rays),
                    np.full(n_rays, np.inf))
    return Workload("heightfield", scene, rays,
                    dict(triangles=int(faces.shape[0]), grid=grid, seed=seed))


def _dedup_noise(v, rng_seed, sigma, radial):
    """Perturbation that moves bitwise-identical vertex positions together (the icosphere
    helper duplicates midpoint vertices per triangle), so the mesh stays watertight."""
    uniq, inv = np.unique(v, axis=0, return_inverse=True)
    rng = np.random.Generator(np.random.PCG64(rng_seed))
    if radial:
        eps = rng.normal(0.0, sigma, uniq.shape[0])
        return uniq[inv.ravel()] * (1.0 + eps[inv.ravel()])[:, None]
    return uniq[inv.ravel()] + rng.normal(0.0, sigma, uniq.shape)[inv.ravel()]


def _rays_to_ball(rng, n, radius):
    """Origins uniform on a sphere of the given radius, directions toward points uniform in
    the unit ball."""
    o = _unit_sphere(rng, n) * radius
    q = _unit_sphere(rng, n) * np.cbrt(rng.random(n))[:, None]
    d = q - o
    return o, d / np.linalg.norm(d, axis=1, keepdims=True)


def batched_icospheres(n_scenes=256, seed=4, min_rays=1_000, max_rays=1_000_000, scale=1.0):
    """Per scene: a target triangle count log-uniform in [1k, 500k] mapped to the nearest
    icosphere level in 3..7, radial perturbation N(0, 0.02) per unique vertex; a ray batch of
    log-uniform size in [min_rays, max_rays] (times scale) from a radius-3 sphere toward the
    unit ball."""
    rng = np.random.Generator(np.random.PCG64(seed))
    cache = {}
    out = []
    for sidx in range(n_scenes):
        target = math.exp(rng.uniform(math.log(1e3), math.log(5e5)))
        level = int(np.clip(np.round(np.log(target / 20.0) / np.log(4.0)), 3, 7))
        if level not in cache:
            cache[level] = icosphere(level)
        v, f = cache[level]
        v = _dedup_noise(v, seed * 100003 + sidx, 0.02, radial=True)
        n = max(1, int(math.exp(rng.uniform(math.log(min_rays), math.log(max_rays))) * scale))
        o, d = _rays_to_ball(rng, n, 3.0)
        out.append(Workload(f"icosphere_{sidx}", SceneSpec().add_mesh(v, f),
                            RayBatch(o, d, np.zeros(n), np.full(n, np.inf)),
                            dict(level=level, triangles=int(f.shape[0]))))
    return out


def adjoint_scene(n_rays=1 << 22, seed=5, level=6, n_split=10_000, n_spheres=500):
    """Level-6 icosphere with n_split triangles split at an edge midpoint (one more triangle
    each), isotropic vertex noise N(0, 0.01) per unique vertex, plus spheres with centres in
    [-2, 2]^3 and radii in [0.05, 0.2]; rays from a radius-4 sphere toward the unit ball and
    per-ray loss weights w ~ N(0, 1)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    v, f = icosphere(level)
    v = _dedup_noise(v, seed * 7919, 0.01, radial=False)
    pick = rng.choice(f.shape[0], n_split, replace=False)
    a, b, c = f[pick, 0], f[pick, 1], f[pick, 2]
    mid = 0.5 * (v[a] + v[b])
    m = v.shape[0] + np.arange(n_split)
    v = np.concatenate([v, mid])
    f = f.astype(np.int64).copy()
    f[pick] = np.stack([a, m, c], 1)
    f = np.concatenate([f, np.stack([m, b, c], 1)])
    sc = rng.uniform(-2.0, 2.0, (n_spheres, 3))
    sr = rng.uniform(0.05, 0.2, n_spheres)
    scene = SceneSpec().add_mesh(v, f.astype(np.uint32)).add_spheres(sc, sr)
    o, d = _rays_to_ball(rng, n_rays, 4.0)
    w = rng.standard_normal(n_rays)
    return Workload("adjoint_scene", scene, RayBatch(o, d, np.zeros(n_rays), np.full(n_rays, np.inf)),
                    dict(triangles=int(f.shape[0]), spheres=n_spheres, seed=seed, weights=w))


def distance_points(spec, kind, rng, n):
    """(ids, points) of distance queries on one kind: random points around random primitives at
    several scales, plus special points -- centres, axis points, shell and cap points of
    cylinders (in the cylinder's frame), surface points of spheres, vertices, edge midpoints
    and centroids of triangles."""
    col = getattr(spec, kind)
    if kind == "mesh":
        v, f = col["vertices"], col["faces"]
        m = len(f)
        ids = rng.integers(0, m, n).astype(np.uint32)
        tri = v[f[ids]]  # n x 3 x 3
        w = rng.dirichlet([1.0, 1.0, 1.0], n)
        base = np.einsum("ni,nij->nj", w, tri)
        scale = rng.choice([0.0, 1e-3, 0.1, 1.0, 10.0], (n, 1))
        pts = base + rng.standard_normal((n, 3)) * scale
        k = n // 8
        pts[:k] = tri[:k, 0]                                   # vertices
        pts[k:2 * k] = 0.5 * (tri[k:2 * k, 0] + tri[k:2 * k, 1])  # edge midpoints
        pts[2 * k:3 * k] = tri[2 * k:3 * k].mean(1)            # centroids
        return ids, pts
    c = col["centers"]
    m = len(c)
    ids = rng.integers(0, m, n).astype(np.uint32)
    scale = rng.choice([0.01, 0.3, 1.0, 5.0, 50.0], (n, 1))
    pts = c[ids] + rng.standard_normal((n, 3)) * scale
    k = n // 10
    pts[:k] = c[ids[:k]]  # centres
    if kind == "spheres":
        u = rng.standard_normal((k, 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        r = col["radii"][ids[k:2 * k]]
        pts[k:2 * k] = c[ids[k:2 * k]] + u * r[:, None]
    if kind == "cylinders":
        R = col["rotations"].reshape(-1, 3, 3)
        a, b, h = col["semi_axes_a"], col["semi_axes_b"], col["heights"]
        for j in range(k, min(n, 6 * k)):
            i = ids[j]
            th = rng.uniform(0, 2 * np.pi)
            sel = j % 5
            if sel == 0:    # on the axis at several heights
                loc = np.array([0.0, 0.0, rng.choice([0.0, h[i] / 2, -h[i] / 2, h[i], 0.3 * h[i]])])
            elif sel == 1:  # on the shell
                loc = np.array([a[i] * np.cos(th), b[i] * np.sin(th), rng.uniform(-h[i], h[i])])
            elif sel == 2:  # on a cap
                rr = rng.uniform(0, 1)
                loc = np.array([rr * a[i] * np.cos(th), rr * b[i] * np.sin(th), h[i] / 2])
            elif sel == 3:  # inside, near the shell
                loc = np.array([0.9 * a[i] * np.cos(th), 0.9 * b[i] * np.sin(th), 0.1 * h[i]])
            else:           # outside beside and above
                loc = np.array([2 * a[i] * np.cos(th), 2 * b[i] * np.sin(th), rng.choice([0.0, h[i]])])
            pts[j] = c[i] + R[i] @ loc
    return ids, pts


def distance_queries(n_per_kind=1 << 22, seed=6):
    """Per-primitive distance queries on the mixed-primitive scene (10,000 spheres, 1,000
    cylinders, 100 planes): n_per_kind (primitive id, point) pairs for each kind, from
    distance_points (points around random primitives at scales 0.01 to 50 plus centres, axis,
    shell and cap points)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    scene = mixed_primitives(n_rays=1).scene
    queries = {k: distance_points(scene, k, rng, n_per_kind) for k in scene.order}
    return Workload("distance_queries", scene, RayBatch(np.zeros((1, 3)), np.ones((1, 3))),
                    dict(queries=queries, n_per_kind=n_per_kind, seed=seed))


def closest_surface_points(n_points=1 << 20, seed=7):
    """Nearest-surface queries on the differentiation scene (91,920 triangles and 500 spheres):
    points uniform in [-2.5, 2.5]^3."""
    rng = np.random.Generator(np.random.PCG64(seed))
    scene = adjoint_scene(n_rays=1).scene
    pts = rng.uniform(-2.5, 2.5, (n_points, 3))
    return Workload("closest_surface", scene, RayBatch(np.zeros((1, 3)), np.ones((1, 3))),
                    dict(points=pts, seed=seed))


WORKLOADS = {
    "icosphere_pinhole": icosphere_pinhole,
    "mixed_primitives": mixed_primitives,
    "heightfield": heightfield,
    "adjoint_scene": adjoint_scene,
}

# query workloads of the distance kernels (not ray batches)
DISTANCE_WORKLOADS = {
    "distance_queries": distance_queries,
    "closest_surface": closest_surface_points,
}
