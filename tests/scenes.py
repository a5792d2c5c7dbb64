"""Small hand-made and randomised scenes for the edge-case tests (shared by CPU and GPU tests).

Edge cases follow the reference's own test suite (test/test_primitives/*.cpp,
test/test_bvh/test_intersect.cpp): axis-aligned rays whose origins lie on box planes (the
0 * inf slab cases), rays along edges and through corners, origins inside primitives, finite
tmin / tmax, overlapping cylinders (a later cylinder overwrites an earlier hit,
blazert/primitives/cylinder.h:181-495), and degenerate boxes."""
from __future__ import annotations

import numpy as np

from blazert_b200.workloads import RayBatch, SceneSpec, rotation_to


def cube_mesh(center=(0.0, 0.0, 0.0), half=1.0):
    """Axis-aligned cube of 12 triangles (counter-clockwise seen from outside)."""
    c = np.asarray(center, np.float64)
    v = np.array([[-1, -1, -1], [1, -1, -1], [1, -1, 1], [-1, -1, 1],
                  [-1, 1, -1], [1, 1, -1], [1, 1, 1], [-1, 1, 1]], np.float64) * half + c
    f = np.array([[1, 5, 4], [0, 1, 4], [2, 6, 5], [1, 2, 5], [3, 7, 6], [2, 3, 6],
                  [4, 7, 3], [0, 4, 3], [5, 6, 7], [4, 5, 7], [3, 2, 1], [0, 3, 1]], np.uint32)
    return v, f


def grid_mesh(n=8, spacing=1.0):
    """Flat n x n vertex grid in the z = 0 plane (many shared edges, exact coordinates)."""
    xs = np.arange(n, dtype=np.float64) * spacing
    X, Y = np.meshgrid(xs, xs)
    v = np.stack([X.ravel(), Y.ravel(), np.zeros(n * n)], 1)
    faces = []
    for j in range(n - 1):
        for i in range(n - 1):
            a = j * n + i
            faces += [[a, a + 1, a + n + 1], [a, a + n + 1, a + n]]
    return v, np.array(faces, np.uint32)


def axis_rays(rng, lo, hi, n, snap=0.5):
    """Rays with axis-aligned (or partly zero) directions and origins snapped to a lattice, so
    that many origins lie exactly on box planes and edges."""
    o = np.round(rng.uniform(lo, hi, (n, 3)) / snap) * snap
    d = np.zeros((n, 3))
    ax = rng.integers(0, 3, n)
    d[np.arange(n), ax] = rng.choice([-1.0, 1.0], n)
    mix = rng.random(n) < 0.3  # second nonzero component
    ax2 = (ax + 1 + rng.integers(0, 2, n)) % 3
    d[np.arange(n)[mix], ax2[mix]] = rng.choice([-0.5, 0.5, -1.0, 1.0], int(mix.sum()))
    neg0 = rng.random(n) < 0.2  # negative zeros: sign 0 but inverse -inf
    d[neg0 & (d[:, 0] == 0), 0] = -0.0
    return o, d


def edge_case_scenes(seed=11):
    """(name, SceneSpec, RayBatch) triples covering the reference's special cases."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    # 1. cubes and a flat grid hit by axis-aligned rays from lattice points
    v1, f1 = cube_mesh()
    v2, f2 = grid_mesh(9)
    v2 = v2 + np.array([-4.0, -4.0, 2.0])
    v = np.concatenate([v1, v2]); f = np.concatenate([f1, f2 + len(v1)])
    o, d = axis_rays(rng, -5, 5, 4000)
    out.append(("mesh_axis", SceneSpec().add_mesh(v, f), RayBatch(o, d)))
    # 2. the same with finite tmin / tmax
    tmin = rng.choice([0.0, 0.5, 1.0, 3.0], o.shape[0])
    tmax = rng.choice([np.inf, 2.0, 4.0, 1.7976931348623157e308, 0.25], o.shape[0])
    out.append(("mesh_axis_trange", SceneSpec().add_mesh(v, f), RayBatch(o, d, tmin, tmax)))
    # 3. spheres on a lattice (touching boxes), axis rays and random rays, some from inside
    c = np.stack(np.meshgrid(*[np.arange(-3, 4, 2.0)] * 3), -1).reshape(-1, 3)
    r = np.full(len(c), 1.0)
    o2, d2 = axis_rays(rng, -6, 6, 3000)
    o3 = rng.uniform(-6, 6, (3000, 3)); d3 = rng.standard_normal((3000, 3))
    sp = SceneSpec().add_spheres(c, r)
    out.append(("spheres_lattice", sp, RayBatch(np.concatenate([o2, o3]), np.concatenate([d2, d3]))))
    # 4. overlapping cylinders along x (later cylinders overwrite earlier hits) + axis rays
    n_c = 40
    cc = np.stack([np.linspace(-4, 4, n_c), np.zeros(n_c), np.zeros(n_c)], 1)
    ax = np.tile([[1.0, 0.0, 0.0]], (n_c, 1)); ax[::3] = [0, 0, 1.0]; ax[1::3] = [0, 1.0, 0]
    rot = rotation_to(ax)
    ca = rng.uniform(0.3, 1.0, n_c); cb = rng.uniform(0.3, 1.0, n_c); ch = rng.uniform(0.5, 3.0, n_c)
    o4, d4 = axis_rays(rng, -5, 5, 4000, snap=0.25)
    o5 = rng.uniform(-5, 5, (2000, 3)); d5 = rng.standard_normal((2000, 3))
    cy = SceneSpec().add_cylinders(cc, ca, cb, ch, rot)
    out.append(("cylinders_overlap", cy, RayBatch(np.concatenate([o4, o5]), np.concatenate([d4, d5]))))
    # 5. planes, axis-aligned and rotated, rays hitting edges and corners exactly
    pc = np.array([[0, 0, 0], [0, 0, 1.0], [2, 0, 0], [0, 3, 0], [-2, -2, -1]], np.float64)
    pn = np.array([[0, 0, 1], [0, 0, 1], [1, 0, 0], [0, 1, 0], [1, 1, 1]], np.float64)
    pn /= np.linalg.norm(pn, axis=1, keepdims=True)
    prot = rotation_to(pn)
    pdx = np.array([2.0, 4.0, 2.0, 1.0, 3.0]); pdy = np.array([2.0, 1.0, 4.0, 2.0, 3.0])
    o6, d6 = axis_rays(rng, -4, 4, 4000, snap=0.5)
    pl = SceneSpec().add_planes(pc, pdx, pdy, prot)
    out.append(("planes_edges", pl, RayBatch(o6, d6)))
    # 6. all four kinds together, random geometry, mixed rays, geom ids in a shuffled order
    vi, fi = cube_mesh((1.0, 1.0, 1.0), 0.75)
    mix = SceneSpec()
    mix.add_cylinders(cc[:10], ca[:10], cb[:10], ch[:10], rot[:10])
    mix.add_mesh(vi, fi)
    mix.add_planes(pc, pdx, pdy, prot)
    mix.add_spheres(c[:20] * 0.8, r[:20] * 0.5)
    o7, d7 = axis_rays(rng, -5, 5, 3000)
    o8 = rng.uniform(-6, 6, (3000, 3)); d8 = rng.standard_normal((3000, 3))
    out.append(("all_kinds", mix, RayBatch(np.concatenate([o7, o8]), np.concatenate([d7, d8]))))
    # 7. single primitives (root is a leaf) and degenerate geometry
    deg = SceneSpec()
    deg.add_mesh(np.array([[0, 0, 0], [1, 0, 0], [2, 0, 0], [0, 1, 0]], np.float64),
                 np.array([[0, 1, 2], [0, 1, 3]], np.uint32))  # a zero-area triangle
    deg.add_spheres(np.array([[0.0, 0.0, 2.0]]), np.array([0.0]))  # zero radius
    o9, d9 = axis_rays(rng, -2, 2, 2000, snap=0.5)
    out.append(("degenerate", deg, RayBatch(o9, d9)))
    return out


from blazert_b200.workloads import distance_points as distance_queries  # noqa: E402,F401
