// Camera sensor entry points of the reference's libmjmlx (include/mjmlx/mjmlx.h
// of the reference, lines 272-295: a Vulkan rasteriser drawing every env's
// cameras).  Rendering needs a graphics stack, which this CUDA engine does
// not have; the functions exist so that callers built against the
// reference's API link unchanged, and each refuses at run time.
#include "capi_internal.h"

namespace {
const char* kNoCamera = "mjmlx_camera_*: camera rendering needs a graphics stack (the reference's Vulkan renderer); this CUDA engine has none";
}

extern "C" {

MJMLX_API MjmlxCameraRenderer* mjmlx_camera_create(MjmlxBatchedSim*, int, int) {
  mjb::set_error(kNoCamera);
  return nullptr;
}
MJMLX_API void mjmlx_camera_free(MjmlxCameraRenderer*) {}
MJMLX_API int mjmlx_camera_count(const MjmlxCameraRenderer*) { return 0; }
MJMLX_API int mjmlx_camera_render(MjmlxCameraRenderer*) {
  mjb::set_error(kNoCamera);
  return -1;
}
MJMLX_API int mjmlx_camera_draw_call_count(const MjmlxCameraRenderer*) { return 0; }
MJMLX_API int mjmlx_camera_get_rgb(MjmlxCameraRenderer*, uint8_t*) {
  mjb::set_error(kNoCamera);
  return -1;
}
MJMLX_API int mjmlx_camera_get_depth(MjmlxCameraRenderer*, float*) {
  mjb::set_error(kNoCamera);
  return -1;
}
MJMLX_API int mjmlx_camera_gpu_supported(const MjmlxCameraRenderer*) { return 0; }
MJMLX_API int mjmlx_camera_gpu_copy(MjmlxCameraRenderer*) {
  mjb::set_error(kNoCamera);
  return -1;
}
MJMLX_API int mjmlx_camera_gpu_export_fd(MjmlxCameraRenderer*, int, uint64_t*) {
  mjb::set_error(kNoCamera);
  return -1;
}

}  // extern "C"
