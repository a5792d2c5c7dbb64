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


def assert_close(got, ref, what, scale=None):
    """Two independent FP64 evaluations of the same gradient: per element within 1e-7
    relative (rays that graze a triangle have 1/(n.d) condition numbers near 1e8), plus an
    absolute floor of 1e-10 of the largest magnitude.  With `scale` (the same sums taken over
    the absolute values of their terms), also 1e-8 of that scale: a sum whose terms cancel
    keeps the rounding of its terms, not a fraction of its own size."""
    tol = 1e-7 * np.abs(ref) + 1e-10 * (np.abs(ref).max() + 1e-300)
    if scale is not None:
        tol = tol + 1e-8 * scale
    bad = np.abs(got - ref) > tol
    assert not bad.any(), (what, int(bad.sum()), float(np.abs(got - ref).max()))


def test_adjoint_matches_analytic_small():
    spec, o, d, rng = small_scene()
    _adjoint_vs_analytic(spec, o, d, rng, with_uv_normal=True)


@pytest.fixture(scope="module")
def adjoint_case():
    """The differentiation workload at full size (91,920-triangle perturbed icosphere + 500
    spheres, 4,194,304 rays): its scene, rays, forward results and the loss weights."""
    wl = W.adjoint_scene()
    spec, R = wl.scene, wl.rays
    assert R.n == 4_194_304
    rng = np.random.Generator(np.random.PCG64(55))
    s = product_scene(spec)
    to, td = _dev(R.origins), _dev(R.directions)
    fwd = s.intersectN(to, td)
    f = to_numpy(fwd)
    hit = f["hit"].astype(bool)
    w = {"t": rng.standard_normal(R.n) * hit,
         "uv": rng.standard_normal((R.n, 2)) * hit[:, None],
         "normal": rng.standard_normal((R.n, 3)) * hit[:, None]}
    yield dict(spec=spec, R=R, s=s, to=to, td=td, fwd=fwd, f=f, hit=hit, w=w, rng=rng)
    s.close()


def _upstream(case, loss, mask):
    """dL/dt, dL/duv, dL/dnormal of the chosen loss, restricted to the rays in `mask`."""
    f, w = case["f"], case["w"]
    m = mask.astype(np.float64)
    gt = 2 * w["t"] * f["t"] * m if loss == "t" else np.zeros(len(m))
    guv = w["uv"] * m[:, None] if loss == "uv" else None
    gn = w["normal"] * m[:, None] if loss == "normal" else None
    return gt, guv, gn


def _loss_of(out, case, loss, mask):
    """Per-ray terms of L over the rays in `mask`: w t^2, w . uv or w . normal (misses 0)."""
    w = case["w"]
    h = out["hit"][mask].astype(bool)
    if loss == "t":
        return w["t"][mask] * np.where(h, out["t"][mask], 0.0) ** 2
    key = "uv" if loss == "uv" else "normal"
    return np.einsum("ij,ij->i", w[key][mask], np.where(h[:, None], out[key][mask], 0.0))


def _geometric_cos(spec, R, f):
    """|cos| between each ray's direction and the geometric normal of the surface it hits
    (the face normal for triangles, the returned normal for spheres); 1 for misses."""
    d = R.directions / np.linalg.norm(R.directions, axis=1, keepdims=True)
    hit = f["hit"].astype(bool)
    n = np.array(f["normal"], copy=True)
    tri = hit & (f["geom"] == 0)
    if tri.any():
        V, F = spec.mesh["vertices"], spec.mesh["faces"].astype(np.int64)
        P = F[f["prim"][tri].astype(np.int64)]
        n[tri] = np.cross(V[P[:, 1]] - V[P[:, 0]], V[P[:, 2]] - V[P[:, 0]])
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-300)
    return np.where(hit, np.abs(np.einsum("ij,ij->i", d, n)), 1.0)


def test_adjoint_scene_analytic_full_size(adjoint_case):
    """All 4,194,304 rays: the CUDA adjoint of t, uv and normal (together) against the host
    analytic FP64 gradient.  Both sides are FP64 evaluations of the same closed form in
    different operation orders, so they agree to about eps times the condition number, which
    grows like a power of 1/cos of the angle between the ray and the surface (up to 1/cos^3
    for the barycentric and normal terms, measured).  Rays with |cos| >= 1e-3
    (all but about one in a thousand) are compared on every output at 1e-7 relative; the
    grazing rest, in a call of their own, on their per-ray origin and direction gradient
    vectors at max(1e-7, 64 eps / cos^3) of the vector's length.  Per-vertex and per-sphere
    sums also get 1e-8 of the sum of their terms' magnitudes, since terms of both signs cancel
    in them."""
    c = adjoint_case
    spec, R, s = c["spec"], c["R"], c["s"]
    cos = _geometric_cos(spec, R, c["f"])
    nv, ns = len(spec.mesh["vertices"]), len(spec.spheres["radii"])
    for part in ("well", "grazing"):
        mask = c["hit"] & ((cos >= 1e-3) if part == "well" else (cos < 1e-3))
        gt, _, _ = _upstream(c, "t", mask)
        guv = c["w"]["uv"] * mask[:, None]
        gn = c["w"]["normal"] * mask[:, None]
        g = s.adjoint(c["to"], c["td"], c["fwd"], grad_t=_dev(gt), grad_uv=_dev(guv),
                      grad_normal=_dev(gn), n_vertices=nv, n_spheres=ns)
        assert s.check() == 0
        ref = adjoint_ref.gradients(spec, R.origins, R.directions, c["f"], gt, guv, gn)
        if part == "well":
            assert mask.sum() > 0.99 * c["hit"].sum()
            scale = adjoint_ref.gradients(spec, R.origins, R.directions, c["f"], gt, guv, gn,
                                          absolute=True)
            for k in ("origins", "directions", "vertices", "centers", "radii"):
                assert_close(g[k].cpu().numpy(), ref[k], k, scale[k])
        else:
            rel = np.maximum(1e-7, 64 * np.finfo(np.float64).eps / np.maximum(cos, 1e-300) ** 3)
            for k in ("origins", "directions"):
                got = g[k].cpu().numpy()
                size = np.linalg.norm(ref[k], axis=1)
                err = np.linalg.norm(got - ref[k], axis=1)
                bad = err > rel * size + 1e-300
                worst = int(np.argmax(err / (rel * size + 1e-300)))
                assert not bad.any(), (k, int(bad.sum()), float(cos[worst]), float(err[worst]),
                                       float(size[worst]))


@pytest.mark.parametrize("loss", ["t", "uv", "normal"])
def test_adjoint_scene_finite_differences(adjoint_case, loss):
    """Losses L = sum w_i t_i^2, sum w_i . uv_i and sum w_i . normal_i over the full workload:
    the CUDA adjoint against FP64 central differences of the GPU forward pass (h = 1e-6 and
    h/2, Richardson-extrapolated) on a seeded subsample of vertex coordinates, sphere centres
    and radii, to 1e-6 relative.  Rays whose hit primitive changes in any perturbed scene, and
    grazing hits (|cos| between ray and normal below 0.05, where the difference quotient's
    truncation error grows like 1/cos^2), are left out of both sides."""
    c = adjoint_case
    spec, R, s, f, hit = c["spec"], c["R"], c["s"], c["f"], c["hit"]
    to, td, fwd = c["to"], c["td"], c["fwd"]
    rng = np.random.Generator(np.random.PCG64({"t": 55, "uv": 56, "normal": 57}[loss]))
    nv, ns = len(spec.mesh["vertices"]), len(spec.spheres["radii"])
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
        outs = []
        for x in specs:
            sx = product_scene(x)
            outs.append(to_numpy(sx.intersectN(to, td)))
            sx.close()
        stable = well.copy()
        for out in outs:
            stable &= (out["prim"] == f["prim"]) & (out["geom"] == f["geom"])
        terms = [_loss_of(o_, c, loss, stable) for o_ in outs]
        # per-ray differences first: rays the perturbation leaves alone contribute exactly 0
        d1 = float(np.sum(terms[0] - terms[1])) / (2 * H)
        d2 = float(np.sum(terms[2] - terms[3])) / H
        return (4 * d2 - d1) / 3, stable

    used = 0
    vert_candidates = np.unique(f["prim"][hit & (f["geom"] == 0)])
    for face in rng.choice(vert_candidates, 4, replace=False):
        vi = int(spec.mesh["faces"][face][0])
        for ax in range(3):
            fdv, stable = fd("mesh", "vertices", (vi, ax))
            gt, guv, gn = _upstream(c, loss, hit & stable)
            g2 = s.adjoint(to, td, fwd, grad_t=_dev(gt),
                           grad_uv=None if guv is None else _dev(guv),
                           grad_normal=None if gn is None else _dev(gn),
                           n_vertices=nv, n_spheres=ns)["vertices"].cpu().numpy()
            an = g2[vi, ax]
            assert abs(fdv - an) <= 1e-6 * max(abs(an), 1e-3), (loss, vi, ax, fdv, an)
            used += 1
    sph_candidates = np.unique(f["prim"][hit & (f["geom"] == 1)])
    for si in rng.choice(sph_candidates, 3, replace=False):
        for key, index in (("centers", (si, 0)), ("radii", si)):
            fdv, stable = fd("spheres", key, index)
            gt, guv, gn = _upstream(c, loss, hit & stable)
            g2 = s.adjoint(to, td, fwd, grad_t=_dev(gt),
                           grad_uv=None if guv is None else _dev(guv),
                           grad_normal=None if gn is None else _dev(gn),
                           n_vertices=nv, n_spheres=ns)[key].cpu().numpy()
            an = g2[index]
            assert abs(fdv - an) <= 1e-6 * max(abs(an), 1e-3), (loss, key, index, fdv, an)
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
