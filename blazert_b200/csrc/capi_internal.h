// Internal accessors of a committed scene for C-ABI entry points defined outside capi.cpp.
#pragma once
#include <cstdint>

#include "../../include/blazert_b200.h"
#include "layout.h"
#include "trace.h"

namespace bzr {

struct SceneHandles {
  int device;
  const SceneView *view;
  const LaunchPlan *plan;
  uint32_t *error_word;  // the scene's sticky kernel error word (read by bzr_scene_check)
};

// BZR_OK, or BZR_EINVAL / BZR_ESTATE (with the thread's error string set) when the scene is
// null or not committed.
int scene_handles(const bzr_scene *scene, SceneHandles *out);
int set_error(int code, const char *msg);
bool is_device_pointer(const void *p);

}  // namespace bzr
