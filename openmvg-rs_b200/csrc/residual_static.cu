// residual_static.cu — omvgba_residual_vjp_f32_static: the residual adjoint for callers that cannot
// allocate device memory.
//
// Who needs it. Some hosts own all of the GPU's memory up front — an engine or framework that
// reserves device memory at start-up and routes every later request through its own pool, or a
// certified or real-time loop that allows no driver allocation after initialisation — and a
// cudaMalloc / cudaFree may also synchronise the device, which a latency-bound loop cannot afford.
// Such callers still own their inputs and outputs; what they cannot provide is the adjoint's
// scratch: the per-camera table and the fixed-point accumulators of omvgba_residual_vjp_f32.
//
// How. The scratch is one file-scope device array of OMVGBA_RESIDUAL_STATIC_SCRATCH_BYTES (16 MiB),
// which every GPU that loads this library holds until the process exits. Host code cannot use the
// array's name as a device address, so every call resolves the address on the current device with
// cudaGetSymbolAddress (cheap, allocates nothing). Resolving it per call rather than caching it per
// device ordinal keeps it right when the module is loaded again at another address: after a
// cudaDeviceReset, or for a driver-API caller whose current context is not the primary one.
// The entry then runs the ordinary omvgba_residual_vjp_f32 with the array as its workspace: that
// path clears the accumulators on the stream before use and overwrites the camera table, so the
// previous call's leftovers never leak into a result. Nothing here calls cudaMalloc, cudaFree or any
// allocating routine.
//
// Module loading. CUDA loads a library's modules lazily by default, so the driver reserves the
// array's 16 MiB when the first call on a device loads this file's module (the symbol lookup does
// that), not at process start. Callers that allow no driver allocation after start-up make one
// warm-up call at start-up, or set CUDA_MODULE_LOADING=EAGER.
//
// Because every call shares the one array, calls that overlap on the GPU (on different streams, or
// from different threads without ordering) race on it; order them on one stream or synchronise.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <string>

#include "../../include/ba_cuda.h"

static __device__ __align__(256) unsigned char g_vjp_scratch[OMVGBA_RESIDUAL_STATIC_SCRATCH_BYTES];

namespace {

int report(omvgba_error* e, int code, const std::string& msg) {
  if (e) {
    e->code = code;
    e->detail = -1;
    std::strncpy(e->message, msg.c_str(), sizeof(e->message) - 1);
    e->message[sizeof(e->message) - 1] = 0;
  }
  return code;
}

// Device address of the scratch array in the current context.
int scratch_on_current_device(void** out, omvgba_error* error) {
  void* ptr = nullptr;
  const cudaError_t st = cudaGetSymbolAddress((void**)&ptr, g_vjp_scratch);
  if (st != cudaSuccess || !ptr)
    return report(error, OMVGBA_CUDA_ERROR,
                  std::string("cudaGetSymbolAddress of the static scratch: ") + cudaGetErrorString(st));
  *out = ptr;
  return OMVGBA_OK;
}

}  // namespace

extern "C" int32_t omvgba_residual_vjp_f32_static(
    void* stream, uint64_t observation_count, const uint32_t* camera_index, const uint32_t* point_index,
    const float* pixel, uint64_t camera_count, const float* rotvec, const float* translation, const float* intrinsics,
    uint64_t point_count, const float* points, const float* grad_residual, float* grad_rotvec, float* grad_translation,
    float* grad_intrinsics, float* grad_points, omvgba_error* error) {
  if (error) {
    error->code = 0;
    error->detail = -1;
    error->message[0] = 0;
  }
  if (observation_count == 0) return OMVGBA_OK;
  const uint64_t need = omvgba_residual_vjp_workspace_bytes(observation_count, camera_count, point_count);
  if (need > (uint64_t)OMVGBA_RESIDUAL_STATIC_SCRATCH_BYTES)
    return report(error, OMVGBA_INVALID_ARGUMENT,
                  "problem too large for the static scratch: " + std::to_string(camera_count) + " cameras and " +
                      std::to_string(point_count) + " points need " + std::to_string(need) +
                      " bytes, the library's static scratch holds " +
                      std::to_string((uint64_t)OMVGBA_RESIDUAL_STATIC_SCRATCH_BYTES) +
                      " bytes; use omvgba_residual_vjp_f32 with a caller-provided workspace");
  void* scratch = nullptr;
  int code = scratch_on_current_device(&scratch, error);
  if (code != OMVGBA_OK) return code;
  return omvgba_residual_vjp_f32(stream, observation_count, camera_index, point_index, pixel, camera_count, rotvec,
                                 translation, intrinsics, point_count, points, grad_residual, grad_rotvec,
                                 grad_translation, grad_intrinsics, grad_points, scratch,
                                 (uint64_t)OMVGBA_RESIDUAL_STATIC_SCRATCH_BYTES, error);
}
