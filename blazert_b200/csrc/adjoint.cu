// Adjoint (reverse-mode gradient) of the closest-hit outputs, for sm_100a.
//
// Given the forward results of a batch (prim_id, geom_id, t, uv, normal as returned by
// bzr_intersectN) and upstream gradients dL/dt, dL/duv, dL/dnormal per ray, this computes
// dL/d(triangle vertices), dL/d(sphere centres), dL/d(sphere radii), dL/d(ray origins) and
// dL/d(raw ray directions).  The hit primitive is held fixed: its intersection is recomputed
// from the stored prim_id, without re-traversal.
//
// Forward model differentiated (the reference's formulas, blazert/primitives/trimesh.h:153-181,
// sphere.h:135-177, their post_traversal, and ray.h:59 d = w / |w|):
//   triangle  e1 = a - b, e2 = c - a, n = e1 x e2, q = a - o, r = d x q, den = n . d,
//             t = (n . q) / den, u = (r . e2) / den, v = (r . e1) / den   (the product_sign
//             factors of the reference cancel), normal = normalize((1-u-v) N_a + u N_b + v N_c)
//             with N the accumulated vertex normals, N_x = sum over faces f at x of
//             normalize((v1_f - v0_f) x (v2_f - v0_f)) / 3 (trimesh.h:91-93, :126-130);
//   sphere    v = o - c, A = d.d, B = 2 v.d, C = v.v - R^2, root t_r = (-B -+ sqrt(B^2-4AC))/(2A)
//             (the root the reference took: the one whose norm(t_r d) equals the stored t),
//             T = norm(t_r d) = |t_r| |d|, normal = normalize(o + T d - c), uv = 0.
// Planes and cylinders are not differentiated: their rays get zero gradients and the call
// reports BZR_EDEVICE_FLAG with kErrAdjointKind set if any ray's hit was one of them.
//
// Gradients are accumulated with double-precision atomics (summation order, and so the last
// bits of a sum over many rays, may vary between runs).
#include <cuda_runtime.h>

#include <cstdint>

#include "adjoint.h"
#include "layout.h"

namespace bzr {
namespace {

struct V {
  double x, y, z;
};
__device__ __forceinline__ V v3(const double *p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ V operator+(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V operator-(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V operator*(V a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V cross(V a, V b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double len(V a) { return sqrt(dot(a, a)); }
// Jacobian-transpose of x -> x / |x| applied to g (x given through its norm and direction).
__device__ __forceinline__ V normalize_back(V dir, double norm, V g) {
  return (g - dir * dot(dir, g)) * (1.0 / norm);
}
__device__ __forceinline__ void atomic_add3(double *p, V g) {
  atomicAdd(p, g.x);
  atomicAdd(p + 1, g.y);
  atomicAdd(p + 2, g.z);
}

__global__ void adjoint_ray_kernel(AdjointView A, AdjointIO io) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < io.n;
       i += uint64_t(gridDim.x) * blockDim.x) {
    V go = {0, 0, 0}, gw = {0, 0, 0};
    const uint32_t geom = io.geom[i], prim = io.prim[i];
    if (io.hit[i] && geom != 0xFFFFFFFFu) {
      const V o = v3(io.org + 3 * i), w = v3(io.dir + 3 * i);
      const double wn = len(w);
      const V d = w * (1.0 / wn);
      const double gt = io.grad_t ? io.grad_t[i] : 0.0;
      const double gu_in = io.grad_uv ? io.grad_uv[2 * i] : 0.0;
      const double gv_in = io.grad_uv ? io.grad_uv[2 * i + 1] : 0.0;
      const V gN = io.grad_normal ? v3(io.grad_normal + 3 * i) : V{0, 0, 0};
      V gd = {0, 0, 0};
      if (geom == A.mesh_geom && A.faces) {
        const uint32_t *F = A.faces + 3 * size_t(prim);
        const V a = v3(A.verts + 3 * size_t(F[0])), b = v3(A.verts + 3 * size_t(F[1])),
                c = v3(A.verts + 3 * size_t(F[2]));
        const V e1 = a - b, e2 = c - a, n = cross(e1, e2), q = a - o, r = cross(d, q);
        const double den = dot(n, d);
        const double t = dot(n, q) / den, u = dot(r, e2) / den, v = dot(r, e1) / den;
        // normal = normalize(s), s = (1-u-v) Na + u Nb + v Nc
        const V Na = v3(A.vert_n + 3 * size_t(F[0])), Nb = v3(A.vert_n + 3 * size_t(F[1])),
                Nc = v3(A.vert_n + 3 * size_t(F[2]));
        const V s = Na * (1.0 - u - v) + Nb * u + Nc * v;
        const double sn = len(s);
        const V ds = normalize_back(s * (1.0 / sn), sn, gN);
        const double gu = gu_in + dot(ds, Nb - Na), gv = gv_in + dot(ds, Nc - Na);
        if (io.grad_vert_n) {
          atomic_add3(io.grad_vert_n + 3 * size_t(F[0]), ds * (1.0 - u - v));
          atomic_add3(io.grad_vert_n + 3 * size_t(F[1]), ds * u);
          atomic_add3(io.grad_vert_n + 3 * size_t(F[2]), ds * v);
        }
        const double gA = gt / den, gB = gu / den, gC = gv / den;
        const double gden = -(gt * t + gu * u + gv * v) / den;
        V gn = q * gA + d * gden, gq = n * gA;
        const V gr = e2 * gB + e1 * gC;
        V ge2 = r * gB, ge1 = r * gC;
        gd = gd + n * gden + cross(q, gr);
        gq = gq + cross(gr, d);
        ge1 = ge1 + cross(e2, gn);
        ge2 = ge2 + cross(gn, e1);
        const V ga = gq + ge1 - ge2;
        go = go - gq;
        if (io.grad_verts) {
          atomic_add3(io.grad_verts + 3 * size_t(F[0]), ga);
          atomic_add3(io.grad_verts + 3 * size_t(F[1]), ge1 * -1.0);
          atomic_add3(io.grad_verts + 3 * size_t(F[2]), ge2);
        }
      } else if (geom == A.sphere_geom && A.centers) {
        const V c = v3(A.centers + 3 * size_t(prim));
        const double R = A.radii[prim];
        const V vv = o - c;
        const double Aq = dot(d, d), B = 2.0 * dot(vv, d), C = dot(vv, vv) - R * R;
        const double D = B * B - 4.0 * Aq * C, sD = sqrt(D);
        const double t0 = (-B - sD) / (2.0 * Aq), t1 = (-B + sD) / (2.0 * Aq);
        const double dn = len(d), T = io.t[i];
        const double T0 = fabs(t0) * dn, T1 = fabs(t1) * dn;
        const double sigma = fabs(T0 - T) <= fabs(T1 - T) ? -1.0 : 1.0;
        const double tr = sigma < 0 ? t0 : t1;
        // normal = normalize(p), p = o + T d - c
        const V p = o + d * T - c;
        const double pn = len(p);
        const V gp = normalize_back(p * (1.0 / pn), pn, gN);
        go = go + gp;
        V gc = gp * -1.0;
        gd = gd + gp * T;
        const double gT = gt + dot(gp, d);
        // T = |tr| |d|
        const double sg = tr < 0 ? -1.0 : 1.0;
        const double gtr = gT * sg * dn;
        gd = gd + d * (gT * fabs(tr) / dn);
        const double gB = gtr * (-1.0 + sigma * B / sD) / (2.0 * Aq);
        const double gCq = gtr * (-sigma / sD);
        const double gAq = gtr * (-sigma * C / (Aq * sD) - tr / Aq);
        gd = gd + d * (2.0 * gAq) + vv * (2.0 * gB);
        const V gvv = d * (2.0 * gB) + vv * (2.0 * gCq);
        go = go + gvv;
        gc = gc - gvv;
        if (io.grad_centers) atomic_add3(io.grad_centers + 3 * size_t(prim), gc);
        if (io.grad_radii) atomicAdd(io.grad_radii + prim, -2.0 * gCq * R);
      } else {
        atomicOr(io.error_word, kErrAdjointKind);
      }
      gw = normalize_back(d, wn, gd);
    }
    if (io.grad_org) {
      io.grad_org[3 * i] = go.x;
      io.grad_org[3 * i + 1] = go.y;
      io.grad_org[3 * i + 2] = go.z;
    }
    if (io.grad_dir) {
      io.grad_dir[3 * i] = gw.x;
      io.grad_dir[3 * i + 1] = gw.y;
      io.grad_dir[3 * i + 2] = gw.z;
    }
  }
}

// dL/d(vertex normals) -> dL/d(vertices) through N_x = sum_f normalize(m_f) / 3,
// m_f = (v1 - v0) x (v2 - v0).
__global__ void adjoint_face_kernel(AdjointView A, AdjointIO io) {
  for (uint64_t f = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; f < A.n_faces;
       f += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t *F = A.faces + 3 * f;
    const V g = (v3(io.grad_vert_n + 3 * size_t(F[0])) + v3(io.grad_vert_n + 3 * size_t(F[1])) +
                 v3(io.grad_vert_n + 3 * size_t(F[2]))) * (1.0 / 3.0);
    if (g.x == 0.0 && g.y == 0.0 && g.z == 0.0) continue;
    const V a = v3(A.verts + 3 * size_t(F[0])), b = v3(A.verts + 3 * size_t(F[1])),
            c = v3(A.verts + 3 * size_t(F[2]));
    const V E1 = b - a, E2 = c - a, m = cross(E1, E2);
    const double mn = len(m);
    const V gm = normalize_back(m * (1.0 / mn), mn, g);
    const V gE1 = cross(E2, gm), gE2 = cross(gm, E1);
    atomic_add3(io.grad_verts + 3 * size_t(F[0]), (gE1 + gE2) * -1.0);
    atomic_add3(io.grad_verts + 3 * size_t(F[1]), gE1);
    atomic_add3(io.grad_verts + 3 * size_t(F[2]), gE2);
  }
}

}  // namespace

cudaError_t launch_adjoint(const AdjointView &A, const AdjointIO &io, int sms,
                           cudaStream_t stream) {
  const int threads = 256;
  const uint64_t want = (io.n + threads - 1) / threads;
  const int blocks = int(want < uint64_t(sms) * 16 ? (want ? want : 1) : uint64_t(sms) * 16);
  adjoint_ray_kernel<<<blocks, threads, 0, stream>>>(A, io);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !A.faces || !io.grad_verts || !io.grad_vert_n) return e;
  const uint64_t fw = (A.n_faces + threads - 1) / threads;
  const int fblocks = int(fw < uint64_t(sms) * 16 ? (fw ? fw : 1) : uint64_t(sms) * 16);
  adjoint_face_kernel<<<fblocks, threads, 0, stream>>>(A, io);
  return cudaGetLastError();
}

}  // namespace bzr
