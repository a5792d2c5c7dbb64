// Host interface of the adjoint kernels (adjoint.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace bzr {

// Scene arrays the adjoint reads (device, input order).
struct AdjointView {
  const double *verts = nullptr;    // n_vertices x 3
  const uint32_t *faces = nullptr;  // n_faces x 3
  const double *vert_n = nullptr;   // n_vertices x 3 accumulated vertex normals
  uint64_t n_faces = 0;
  uint32_t mesh_geom = 0xFFFFFFFFu;
  const double *centers = nullptr;  // spheres: n x 3
  const double *radii = nullptr;    // spheres: n
  uint32_t sphere_geom = 0xFFFFFFFFu;
};

// Device pointers of one backward batch.  Forward results as returned by bzr_intersectN;
// upstream gradients may be null (zero).  grad_verts, grad_centers, grad_radii, grad_vert_n
// are accumulated into (zeroed by the caller); grad_org / grad_dir are written per ray.
struct AdjointIO {
  uint64_t n = 0;
  const double *org = nullptr, *dir = nullptr;
  const double *t = nullptr;
  const uint32_t *prim = nullptr, *geom = nullptr;
  const uint8_t *hit = nullptr;
  const double *grad_t = nullptr, *grad_uv = nullptr, *grad_normal = nullptr;
  double *grad_verts = nullptr, *grad_vert_n = nullptr;
  double *grad_centers = nullptr, *grad_radii = nullptr;
  double *grad_org = nullptr, *grad_dir = nullptr;
  uint32_t *error_word = nullptr;
};

cudaError_t launch_adjoint(const AdjointView &A, const AdjointIO &io, int sms,
                           cudaStream_t stream);

}  // namespace bzr
