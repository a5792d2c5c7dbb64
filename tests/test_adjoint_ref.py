"""The host analytic gradient (tests/adjoint_ref.py) against FP64 central finite differences of
the CPU oracle's forward pass, so that the GPU adjoint can be checked against it."""
import numpy as np

from blazert_b200 import workloads as W
from oracle.oracle import Oracle
from tests import adjoint_ref

H = 1e-6


def small_scene(seed=3):
    rng = np.random.Generator(np.random.PCG64(seed))
    v, f = W.icosphere(2)
    v = W._dedup_noise(v, seed, 0.01, radial=False)
    s = W.SceneSpec().add_mesh(v, f)
    s.add_spheres(rng.uniform(-1.5, 1.5, (12, 3)), rng.uniform(0.1, 0.3, 12))
    o, d = W._rays_to_ball(rng, 400, 4.0)
    d = d * rng.uniform(0.5, 2.0, (400, 1))  # raw directions of varied length
    return s, o, d, rng


def loss_parts(out, wt, wuv, wn):
    t = np.where(out["hit"].astype(bool), out["t"], 0.0)
    return float(np.sum(wt * t * t) + np.sum(wuv * out["uv"]) + np.sum(wn * out["normal"]))


def test_analytic_gradient_matches_finite_differences():
    spec, o, d, rng = small_scene()
    base = Oracle(spec).intersect(o, d)
    hit = base["hit"].astype(bool)
    wt = rng.standard_normal(len(o)) * hit
    wuv = rng.standard_normal((len(o), 2)) * hit[:, None]
    wn = rng.standard_normal((len(o), 3)) * hit[:, None]
    g = adjoint_ref.gradients(spec, o, d, base, 2 * wt * base["t"] * hit, wuv, wn)

    def L(spec_, o_, d_, stable):
        out = Oracle(spec_).intersect(o_, d_)
        assert np.array_equal(out["prim"][stable], base["prim"][stable])
        return loss_parts({k: v[stable] for k, v in out.items()}, wt[stable], wuv[stable], wn[stable])

    def check(fd, an):
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)) + 1e-7, (fd, an)

    def fd_geometry(kind, key, index):
        vals = getattr(spec, kind)[key]
        outs = []
        for sgn in (1, -1):
            s2 = W.SceneSpec()
            for k in spec.order:
                arrs = {n: a.copy() for n, a in getattr(spec, k).items()}
                if k == kind:
                    arrs[key][index] += sgn * H
                getattr(s2, "add_" + k)(*arrs.values())
            outs.append(s2)
        # rays whose hit primitive is the same under both perturbations
        a, b = Oracle(outs[0]).intersect(o, d), Oracle(outs[1]).intersect(o, d)
        stable = (a["prim"] == base["prim"]) & (b["prim"] == base["prim"]) & \
                 (a["geom"] == base["geom"]) & (b["geom"] == base["geom"])
        return (L(outs[0], o, d, stable) - L(outs[1], o, d, stable)) / (2 * H)

    for vi in rng.choice(len(spec.mesh["vertices"]), 6, replace=False):
        for ax in range(3):
            check(fd_geometry("mesh", "vertices", (vi, ax)), g["vertices"][vi, ax])
    for si in range(3):
        check(fd_geometry("spheres", "centers", (si, 1)), g["centers"][si, 1])
        check(fd_geometry("spheres", "radii", si), g["radii"][si])
    rays = np.nonzero(hit)[0][:8]
    for ri in rays:
        for arr, key in ((o, "origins"), (d, "directions")):
            for ax in range(3):
                vals = []
                for sgn in (1, -1):
                    a2 = arr.copy()
                    a2[ri, ax] += sgn * H
                    o_, d_ = (a2, d) if key == "origins" else (o, a2)
                    out = Oracle(spec).intersect(o_[ri:ri + 1], d_[ri:ri + 1])
                    assert out["prim"][0] == base["prim"][ri]
                    vals.append(loss_parts(out, wt[ri:ri + 1], wuv[ri:ri + 1], wn[ri:ri + 1]))
                check((vals[0] - vals[1]) / (2 * H), g[key][ri, ax])
