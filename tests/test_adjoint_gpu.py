"""The CUDA adjoint (bzr_adjoint_hit) and its torch.autograd wrapper against the host analytic
FP64 gradient and FP64 central finite differences of the GPU forward pass (h = 1e-6,
Richardson-extrapolated with h/2)."""
import numpy as np
import pytest

from blazert_b200 import workloads as W
from tests import adjoint_ref
from tests.helpers import product_scene, to_numpy
from tests.test_adjoint_ref import small_scene

pytestmark = pytest.mark.gpu
H = 1e-6


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _adjoint_vs_analytic(spec, o, d, rng, with_uv_normal):
    s = product_scene(spec)
    to, td = _dev(o), _dev(d)
    fwd = s.intersectN(to, td)
    f = to_numpy(fwd)
    hit = f["hit"].astype(bool)
    wt = rng.standard_normal(len(o)) * hit
    gt = 2 * wt * f["t"] * hit
    guv = rng.standard_normal((len(o), 2)) * hit[:, None] if with_uv_normal else None
    gn = rng.standard_normal((len(o), 3)) * hit[:, None] if with_uv_normal else None
    nv = len(spec.mesh["vertices"])
    ns = len(spec.spheres["radii"])
    g = s.adjoint(to, td, fwd, grad_t=_dev(gt), grad_uv=None if guv is None else _dev(guv),
                  grad_normal=None if gn is None else _dev(gn), n_vertices=nv, n_spheres=ns)
    assert s.check() == 0
    ref = adjoint_ref.gradients(spec, o, d, f, gt, guv, gn)
    for k in ("origins", "directions", "vertices", "centers", "radii"):
        assert_close(g[k].cpu().numpy(), ref[k], k)
    return s, f, wt


def assert_close(got, ref, what):
    """Two independent FP64 evaluations of the same gradient: per element within 1e-7
    relative (rays that graze a triangle have 1/(n.d) condition numbers near 1e8), plus an
    absolute floor of 1e-10 of the largest magnitude."""
    tol = 1e-7 * np.abs(ref) + 1e-10 * (np.abs(ref).max() + 1e-300)
    bad = np.abs(got - ref) > tol
    assert not bad.any(), (what, int(bad.sum()), float(np.abs(got - ref).max()))


def test_adjoint_matches_analytic_small():
    spec, o, d, rng = small_scene()
    _adjoint_vs_analytic(spec, o, d, rng, with_uv_normal=True)


def test_adjoint_scene_analytic_and_finite_differences():
    """The differentiation workload (91,920-triangle perturbed icosphere + 500 spheres), loss
    L = sum w_i t_i^2: CUDA adjoint vs the host analytic gradient on all rays, and vs central
    differences on a seeded subsample of parameters (rays whose hit primitive changes under the
    perturbation, and grazing hits, are left out of the difference quotient)."""
    wl = W.adjoint_scene(n_rays=1 << 20)
    spec, R = wl.scene, wl.rays
    rng = np.random.Generator(np.random.PCG64(55))
    s, f, wt = _adjoint_vs_analytic(spec, R.origins, R.directions, rng, with_uv_normal=False)
    to, td = _dev(R.origins), _dev(R.directions)
    fwd = s.intersectN(to, td)
    nv, ns = len(spec.mesh["vertices"]), len(spec.spheres["radii"])
    hit = f["hit"].astype(bool)
    g = s.adjoint(to, td, fwd, grad_t=_dev(2 * wt * f["t"] * hit), n_vertices=nv, n_spheres=ns)
    gv, gc, gr = (g[k].cpu().numpy() for k in ("vertices", "centers", "radii"))

    # Grazing hits (|cos| between ray and normal below 0.05) are left out of the difference
    # quotient: dt/dparameter grows like 1/cos there, and the truncation error of the
    # difference quotient faster still.
    dn = R.directions / np.linalg.norm(R.directions, axis=1, keepdims=True)
    well = np.abs(np.einsum("ij,ij->i", dn, f["normal"])) >= 0.05

    def fd(kind, key, index):
        """Central differences at h and h/2 over the rays whose hit is unchanged in all four
        perturbed scenes, combined as (4 D(h/2) - D(h)) / 3 (the O(h^2) terms cancel)."""
        specs = []
        for step in (H, -H, H / 2, -H / 2):
            s2 = W.SceneSpec()
            for k in spec.order:
                arrs = {n: a.copy() for n, a in getattr(spec, k).items()}
                if k == kind:
                    arrs[key][index] += step
                getattr(s2, "add_" + k)(*arrs.values())
            specs.append(s2)
        outs = [to_numpy(product_scene(x).intersectN(to, td)) for x in specs]
        stable = well.copy()
        for out in outs:
            stable &= (out["prim"] == f["prim"]) & (out["geom"] == f["geom"])
        t2 = [np.where(o_["hit"][stable].astype(bool), o_["t"][stable], 0.0) ** 2 for o_ in outs]
        # per-ray differences first: rays the perturbation leaves alone contribute exactly 0
        d1 = float(np.sum(wt[stable] * (t2[0] - t2[1]))) / (2 * H)
        d2 = float(np.sum(wt[stable] * (t2[2] - t2[3]))) / H
        return (4 * d2 - d1) / 3, stable

    used = 0
    vert_candidates = np.unique(f["prim"][hit & (f["geom"] == 0)])
    for face in rng.choice(vert_candidates, 4, replace=False):
        vi = int(spec.mesh["faces"][face][0])
        for ax in range(3):
            fdv, stable = fd("mesh", "vertices", (vi, ax))
            # the adjoint restricted to the same stable rays
            g2 = s.adjoint(to, td, fwd, grad_t=_dev(2 * wt * f["t"] * hit * stable),
                           n_vertices=nv, n_spheres=ns)["vertices"].cpu().numpy()
            an = g2[vi, ax]
            assert abs(fdv - an) <= 1e-6 * max(abs(an), 1e-3), (vi, ax, fdv, an)
            used += 1
    sph_candidates = np.unique(f["prim"][hit & (f["geom"] == 1)])
    for si in rng.choice(sph_candidates, 3, replace=False):
        for key, index in (("centers", (si, 0)), ("radii", si)):
            fdv, stable = fd("spheres", key, index)
            g2 = s.adjoint(to, td, fwd, grad_t=_dev(2 * wt * f["t"] * hit * stable),
                           n_vertices=nv, n_spheres=ns)[key].cpu().numpy()
            an = g2[index]
            assert abs(fdv - an) <= 1e-6 * max(abs(an), 1e-3), (key, index, fdv, an)
            used += 1
    assert used == 18


def test_autograd_wrapper():
    import torch

    from blazert_b200.autograd import trace

    spec, o, d, rng = small_scene(seed=7)
    s = product_scene(spec)
    to = _dev(o).requires_grad_(True)
    td = _dev(d).requires_grad_(True)
    verts = _dev(spec.mesh["vertices"]).requires_grad_(True)
    cen = _dev(spec.spheres["centers"]).requires_grad_(True)
    rad = _dev(spec.spheres["radii"]).requires_grad_(True)
    t, uv, nrm, prim, geom, hit = trace(s, to, td, verts, cen, rad)
    w = _dev(rng.standard_normal(len(o)))
    hm = hit.to(torch.float64)
    loss = (w * torch.where(hit.bool(), t, torch.zeros_like(t)) ** 2).sum() + (uv * hm[:, None]).sum() \
        + (nrm[:, 2] * hm).sum()
    loss.backward()
    f = {k: v.detach().cpu().numpy() for k, v in dict(t=t, prim=prim, geom=geom, hit=hit).items()}
    hnp = f["hit"].astype(bool)
    gt = 2 * w.cpu().numpy() * f["t"] * hnp
    guv = np.ones((len(o), 2)) * hnp[:, None]
    gn = np.zeros((len(o), 3))
    gn[:, 2] = hnp
    ref = adjoint_ref.gradients(spec, o, d, {k: v for k, v in f.items()}, gt, guv, gn)
    for got, k in ((to.grad, "origins"), (td.grad, "directions"), (verts.grad, "vertices"),
                   (cen.grad, "centers"), (rad.grad, "radii")):
        assert_close(got.cpu().numpy(), ref[k], k)
