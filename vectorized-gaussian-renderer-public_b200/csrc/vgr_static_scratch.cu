// Allocation-free render entry point: the render's scratch lives in a
// file-scope device array instead of a caller-provided buffer.
//
// Who needs this: callers that are not allowed to call cudaMalloc on their
// render path -- for example a sensor plug-in running inside a host
// simulator that owns all device memory through its own pool, a real-time
// loop that must not take the allocator's latency or fragmentation, or code
// being captured into a CUDA graph, where a fresh cudaMalloc is not an
// operation the capture can record.  Such a caller can still hand over the
// buffers it already owns (inputs, outputs and the record/key/value/range
// workspace), but has nowhere to get the queue tickets, per-camera plans and
// projection constants from.  Those fit in a fixed array that
// the library carries itself.
//
// Limits and rules:
//  * The array is VGR_STATIC_SCRATCH_BYTES (16 MiB).  Every GPU on which the
//    library is loaded holds it until the process exits.  The scratch grows
//    with the active cameras (176 bytes each: a 56-byte plan, 112 bytes of
//    projection constants and an 8-byte tile prefix entry) plus about 9 KB
//    (header and sort histogram), not with the scene or the intersections.
//    vgr_static_scratch_max_cameras() returns the exact limit (95,275
//    active cameras); a larger render is rejected with
//    VGR_ERR_SCRATCH_TOO_SMALL before anything is launched.
//  * Every call on a device shares the one array, and it keeps the previous
//    call's contents.  vgr_render clears everything that must start at zero
//    (counters, queue tickets, reserved totals, tile counts) on the
//    stream, so back-to-back calls on one stream are correct; calls whose
//    work overlaps on the GPU (different streams, or different host threads
//    without ordering) race on the array and produce wrong results.
//  * reuse_projection is refused: it would composite from the plans left in
//    the array by whichever static-scratch call ran last on the device, which
//    need not be the caller's previous render.
//  * The first call on each device looks up the array's device address with
//    cudaGetSymbolAddress while that device is current, and caches it for the
//    process.  Make that first call before any stream capture begins.  The
//    cached address belongs to the device's primary context: after
//    cudaDeviceReset (which unloads the library's module) or from a
//    driver-API context of one's own, do not call this entry point.
//  * Nothing here allocates: no cudaMalloc, cudaFree or allocating library
//    routine is called on any path.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/vgr_b200.h"
#include "vgr_api_internal.h"
#include "vgr_camera.cuh"

namespace {

static __device__ __align__(256) unsigned char g_static_scratch[VGR_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_static_mutex;
void* g_static_address[kMaxDevices] = {};

int static_scratch_address(void** address) {
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) {
    cudaGetLastError();
    return vgr::fail(VGR_ERR_CUDA, "static scratch: no usable current CUDA device");
  }
  std::lock_guard<std::mutex> lock(g_static_mutex);
  if (g_static_address[device] == nullptr) {
    void* ptr = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&ptr, g_static_scratch);
    if (err != cudaSuccess || ptr == nullptr) {
      cudaGetLastError();
      return vgr::fail(VGR_ERR_CUDA, "static scratch: cudaGetSymbolAddress failed: %s",
                       cudaGetErrorString(err));
    }
    g_static_address[device] = ptr;
  }
  *address = g_static_address[device];
  return VGR_OK;
}

}  // namespace

extern "C" int64_t vgr_static_scratch_max_cameras(void) {
  int64_t lo = 0;
  int64_t hi = VGR_STATIC_SCRATCH_BYTES / 64;
  while (lo < hi) {  // largest count whose layout fits in the array
    const int64_t mid = (lo + hi + 1) / 2;
    if (vgr::make_scratch_layout(1, mid, false).total <= VGR_STATIC_SCRATCH_BYTES) {
      lo = mid;
    } else {
      hi = mid - 1;
    }
  }
  return lo;
}

extern "C" int vgr_render_static_scratch(const vgr_scene* scene, const vgr_cameras* cameras,
                                         const vgr_outputs* outputs,
                                         const vgr_workspace* workspace,
                                         const vgr_render_options* options, void* stream,
                                         int64_t* sorted_buffer_selector) {
  if (!workspace) return vgr::fail(VGR_ERR_INVALID_ARGUMENT, "render arguments must be non-null");
  if (options && options->reuse_projection) {
    return vgr::fail(VGR_ERR_INVALID_ARGUMENT,
                     "vgr_render_static_scratch does not support reuse_projection: the shared "
                     "static array may hold another call's camera plans; use vgr_render");
  }
  void* address = nullptr;
  const int rc = static_scratch_address(&address);
  if (rc != VGR_OK) return rc;
  vgr_workspace with_static = *workspace;
  with_static.scratch = address;
  with_static.scratch_bytes = VGR_STATIC_SCRATCH_BYTES;
  const int result =
      vgr_render(scene, cameras, outputs, &with_static, options, stream, sorted_buffer_selector);
  if (result == VGR_ERR_SCRATCH_TOO_SMALL) {
    char detail[512];
    std::snprintf(detail, sizeof(detail), "%s", vgr_last_error());
    return vgr::fail(VGR_ERR_SCRATCH_TOO_SMALL,
                     "this render needs more scratch than the %lld-byte static array of "
                     "vgr_render_static_scratch; use vgr_render with a caller-provided scratch "
                     "buffer (%s)",
                     static_cast<long long>(VGR_STATIC_SCRATCH_BYTES), detail);
  }
  return result;
}
