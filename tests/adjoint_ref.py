"""Analytic FP64 gradient of the closest-hit outputs on the host (numpy), written independently
of the CUDA adjoint, for the differentiation tests.

The forward model is the reference's (blazert/primitives/trimesh.h:133-181, sphere.h:107-177,
ray.h:59): for a triangle (a, b, c) hit by a ray (o, w), d = w / |w|,
    t = n.q / n.d, u = (d x q).e2 / n.d, v = (d x q).e1 / n.d,
    e1 = a - b, e2 = c - a, n = e1 x e2, q = a - o,
    normal = normalize((1-u-v) N_a + u N_b + v N_c),  N_x = sum_f normalize(m_f) / 3;
for a sphere (c, R): T = |t_r| |d| with t_r the root taken, normal = normalize(o + T d - c).
Gradients are built with explicit Jacobians (numpy einsum), not by reverse accumulation.
"""
from __future__ import annotations

import numpy as np


def _normalize_jac(x):
    """Jacobian of x / |x| (rows: n x 3 x 3)."""
    n = np.linalg.norm(x, axis=1)
    u = x / n[:, None]
    return (np.eye(3)[None] - u[:, :, None] * u[:, None, :]) / n[:, None, None]


def _cross_mat(a):
    """Matrix [a]_x with [a]_x b = a x b (n x 3 x 3)."""
    z = np.zeros(len(a))
    return np.stack([np.stack([z, -a[:, 2], a[:, 1]], 1),
                     np.stack([a[:, 2], z, -a[:, 0]], 1),
                     np.stack([-a[:, 1], a[:, 0], z], 1)], 1)


def gradients(spec, origins, directions, fwd, gt, guv=None, gnormal=None, absolute=False):
    """fwd: dict with t, prim, geom, hit (numpy).  Returns dict like Scene.adjoint.  With
    absolute=True every per-ray and per-face contribution is accumulated by its absolute value
    instead: the scale against which the rounding of the sums is measured."""
    def acc(X, i, v):
        np.add.at(X, i, np.abs(v) if absolute else v)

    n = origins.shape[0]
    g_o = np.zeros((n, 3))
    g_w = np.zeros((n, 3))
    gv = np.zeros_like(spec.mesh["vertices"]) if spec.mesh else None
    gvn = np.zeros_like(spec.mesh["vertices"]) if spec.mesh else None
    gc = np.zeros_like(spec.spheres["centers"]) if spec.spheres else None
    gr = np.zeros_like(spec.spheres["radii"]) if spec.spheres else None
    guv = np.zeros((n, 2)) if guv is None else guv
    gnormal = np.zeros((n, 3)) if gnormal is None else gnormal
    geom_ids = {k: i for i, k in enumerate(spec.order)}
    w = directions
    wn = np.linalg.norm(w, axis=1)
    d = w / wn[:, None]
    Jw = _normalize_jac(w)  # dd/dw
    hit = fwd["hit"].astype(bool)

    if spec.mesh is not None:
        m = hit & (fwd["geom"] == geom_ids["mesh"])
        idx = np.nonzero(m)[0]
        V, F = spec.mesh["vertices"], spec.mesh["faces"].astype(np.int64)
        # vertex normals exactly as the forward model defines them
        f0, f1, f2 = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
        mf = np.cross(f1 - f0, f2 - f0)
        fn = mf / np.linalg.norm(mf, axis=1)[:, None]
        VN = np.zeros_like(V)
        for j in range(3):
            np.add.at(VN, F[:, j], fn / 3.0)
        P = fwd["prim"][idx].astype(np.int64)
        ia, ib, ic = F[P, 0], F[P, 1], F[P, 2]
        a, b, c = V[ia], V[ib], V[ic]
        o, dd = origins[idx], d[idx]
        e1, e2 = a - b, c - a
        nn = np.cross(e1, e2)
        q = a - o
        r = np.cross(dd, q)
        den = np.einsum("ij,ij->i", nn, dd)
        A = np.einsum("ij,ij->i", nn, q)
        B = np.einsum("ij,ij->i", r, e2)
        Cc = np.einsum("ij,ij->i", r, e1)
        t, u, v = A / den, B / den, Cc / den
        # derivatives of (A, B, C, den) w.r.t. a, b, c, o, d (each n x 3)
        # A = (e1 x e2).q ; B = (d x q).e2 ; C = (d x q).e1 ; den = (e1 x e2).d
        def dot_grads(vec_n, vec_q):
            return vec_n, vec_q
        # partials via closed forms
        dA_de1 = np.cross(e2, q); dA_de2 = np.cross(q, e1); dA_dq = nn
        dB_dd = np.cross(q, e2); dB_dq = np.cross(e2, dd); dB_de2 = r
        dC_dd = np.cross(q, e1); dC_dq = np.cross(e1, dd); dC_de1 = r
        dden_de1 = np.cross(e2, dd); dden_de2 = np.cross(dd, e1); dden_dd = nn

        def to_abcod(de1, de2, dq, dd_):
            # e1 = a - b, e2 = c - a, q = a - o
            ga = de1 - de2 + dq
            gb = -de1
            gc_ = de2
            go = -dq
            return ga, gb, gc_, go, dd_

        z = np.zeros_like(a)
        JA = to_abcod(dA_de1, dA_de2, dA_dq, z)
        JB = to_abcod(z, dB_de2, dB_dq, dB_dd)
        JC = to_abcod(dC_de1, z, dC_dq, dC_dd)
        JD = to_abcod(dden_de1, dden_de2, z, dden_dd)
        # normal = normalize(s), s = (1-u-v) Na + u Nb + v Nc
        Na, Nb, Nc = VN[ia], VN[ib], VN[ic]
        s = Na * (1 - u - v)[:, None] + Nb * u[:, None] + Nc * v[:, None]
        ds = np.einsum("nij,ni->nj", _normalize_jac(s), gnormal[idx])  # dL/ds
        gu = guv[idx, 0] + np.einsum("ij,ij->i", ds, Nb - Na)
        gvv = guv[idx, 1] + np.einsum("ij,ij->i", ds, Nc - Na)
        gtt = gt[idx]
        # t = A/den etc.
        cA, cB, cC = gtt / den, gu / den, gvv / den
        cD = -(gtt * t + gu * u + gvv * v) / den
        grads = [sum(coef[:, None] * J[k] for coef, J in ((cA, JA), (cB, JB), (cC, JC), (cD, JD)))
                 for k in range(5)]
        ga, gb, gcc, go, gd = grads
        acc(gv, ia, ga)
        acc(gv, ib, gb)
        acc(gv, ic, gcc)
        acc(gvn, ia, ds * (1 - u - v)[:, None])
        acc(gvn, ib, ds * u[:, None])
        acc(gvn, ic, ds * v[:, None])
        g_o[idx] += np.abs(go) if absolute else go
        gw_ = np.einsum("nij,ni->nj", Jw[idx], gd)
        g_w[idx] += np.abs(gw_) if absolute else gw_
        # vertex normals back to vertices: N_x = sum_f normalize(m_f)/3
        gfn = (gvn[F[:, 0]] + gvn[F[:, 1]] + gvn[F[:, 2]]) / 3.0
        gm = np.einsum("nij,ni->nj", _normalize_jac(mf), gfn)
        E1, E2 = f1 - f0, f2 - f0
        gE1 = np.cross(E2, gm)
        gE2 = np.cross(gm, E1)
        acc(gv, F[:, 0], -(gE1 + gE2))
        acc(gv, F[:, 1], gE1)
        acc(gv, F[:, 2], gE2)

    if spec.spheres is not None:
        m = hit & (fwd["geom"] == geom_ids["spheres"])
        idx = np.nonzero(m)[0]
        P = fwd["prim"][idx].astype(np.int64)
        C0 = spec.spheres["centers"][P]
        R = spec.spheres["radii"][P]
        o, dd = origins[idx], d[idx]
        vv = o - C0
        Aq = np.einsum("ij,ij->i", dd, dd)
        B = 2 * np.einsum("ij,ij->i", vv, dd)
        Cq = np.einsum("ij,ij->i", vv, vv) - R * R
        sD = np.sqrt(B * B - 4 * Aq * Cq)
        t0, t1 = (-B - sD) / (2 * Aq), (-B + sD) / (2 * Aq)
        dn = np.sqrt(Aq)
        T = fwd["t"][idx]
        sigma = np.where(np.abs(np.abs(t0) * dn - T) <= np.abs(np.abs(t1) * dn - T), -1.0, 1.0)
        tr = np.where(sigma < 0, t0, t1)
        # d tr / d (o, c, R, d): tr = (-B + sigma sqrt(D)) / (2A)
        dtr_dB = (-1 + sigma * B / sD) / (2 * Aq)
        dtr_dC = -sigma / sD
        dtr_dA = -sigma * Cq / (Aq * sD) - tr / Aq
        dtr_dv = dtr_dB[:, None] * 2 * dd + dtr_dC[:, None] * 2 * vv
        dtr_dd = dtr_dB[:, None] * 2 * vv + dtr_dA[:, None] * 2 * dd
        dtr_dR = dtr_dC * (-2 * R)
        sg = np.sign(tr)
        # T = |tr| |d|
        dT_dv = (sg * dn)[:, None] * dtr_dv
        dT_dd = (sg * dn)[:, None] * dtr_dd + (np.abs(tr) / dn)[:, None] * dd
        dT_dR = sg * dn * dtr_dR
        # normal = normalize(p), p = o + T d - c = v + T d
        p = vv + T[:, None] * dd
        gp = np.einsum("nij,ni->nj", _normalize_jac(p), gnormal[idx])
        gT = gt[idx] + np.einsum("ij,ij->i", gp, dd)
        gvv_ = gp + gT[:, None] * dT_dv
        gd = T[:, None] * gp + gT[:, None] * dT_dd
        acc(gc, P, -gvv_)
        acc(gr, P, gT * dT_dR)
        g_o[idx] += np.abs(gvv_) if absolute else gvv_
        gw_ = np.einsum("nij,ni->nj", Jw[idx], gd)
        g_w[idx] += np.abs(gw_) if absolute else gw_

    return dict(origins=g_o, directions=g_w, vertices=gv, centers=gc, radii=gr)
