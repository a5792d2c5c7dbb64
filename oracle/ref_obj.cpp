// C-ABI driver around the reference's vendored OBJ loader (test infrastructure, not product
// code): examples/common/tiny_obj_loader.cc (tiny_obj_loader 0.9.14) compiled where it lies,
// and the mesh assembly of examples/scene_mesh/main.cc:15-43 (shapes concatenated, face
// indices offset by the vertices of the shapes before, float positions widened to double).
// Pins bzr_obj_load.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "tiny_obj_loader.h"

extern "C" {

// Returns 0 and fills malloc'd arrays (release with ref_obj_free), or 1 with the loader's
// message in `why`.
int ref_obj_load(const char *path, double **vertices, long *n_vertices, uint32_t **faces,
                 long *n_faces, char *why, long why_cap) {
  std::vector<tinyobj::shape_t> shapes;
  const std::string err = tinyobj::LoadObj(shapes, path);
  if (!err.empty()) {
    if (why && why_cap > 0) {
      std::strncpy(why, err.c_str(), size_t(why_cap) - 1);
      why[why_cap - 1] = 0;
    }
    return 1;
  }
  std::vector<double> v;
  std::vector<uint32_t> f;
  size_t offset = 0;
  for (const tinyobj::shape_t &shape : shapes) {
    for (size_t i = 0; i < shape.mesh.indices.size(); ++i)
      f.push_back(uint32_t(shape.mesh.indices[i] + offset));
    for (size_t i = 0; i < shape.mesh.positions.size(); ++i)
      v.push_back(double(shape.mesh.positions[i]));
    offset += shape.mesh.positions.size() / 3;
  }
  *vertices = static_cast<double *>(std::malloc((v.size() + 1) * sizeof(double)));
  *faces = static_cast<uint32_t *>(std::malloc((f.size() + 1) * sizeof(uint32_t)));
  if (!v.empty()) std::memcpy(*vertices, v.data(), v.size() * sizeof(double));
  if (!f.empty()) std::memcpy(*faces, f.data(), f.size() * sizeof(uint32_t));
  *n_vertices = long(v.size() / 3);
  *n_faces = long(f.size() / 3);
  return 0;
}

void ref_obj_free(void *p) { std::free(p); }

}  // extern "C"
