// k_noalloc.cu -- an allocation-free form of the 3-iteration a-trous chain.
//
// Some callers cannot allocate device memory at the moment they need the
// denoiser: an engine's render thread whose device memory is owned by its
// own allocator and admission budget, or a frame loop that must not call
// cudaMalloc/cudaFree because those synchronize the device and stall the
// other streams.  vrt_denoise_atrous_noalloc serves them: the caller passes
// the history (input), the G-buffer (input) and the output image, and the one
// intermediate image the chain needs lives in the file-scope array below.
//
// Limits and sharing rules:
//   * at most kNoAllocMaxPixels pixels (1920 x 1080); larger images are
//     rejected with VRT_ERR_INVALID before anything is launched;
//   * the output may not overlap the history or the G-buffer (the first
//     iteration reads the neighbours of every pixel it writes); overlapping
//     ranges are rejected with VRT_ERR_INVALID;
//   * every GPU that loads this library holds the array (16,588,800 bytes)
//     until the process exits;
//   * all calls on a device share the one array, and it keeps the last call's
//     contents: calls whose work overlaps on the GPU (different streams, no
//     ordering between them) race on it and must be serialised by the caller;
//   * the array needs no clearing: every pixel of it is written before it is
//     read within one call.
//
// The iterations run the TMA-staged a-trous kernel (k_atrous_tma.cu), which
// needs no memory beyond its tensor maps (kernel parameters); buffers that do
// not meet its copy constraints (16-byte alignment; an even width for an
// rgba16f source) take the unstaged kernel, which allocates nothing either.
#include <cuda_runtime.h>
#include <cstdint>
#include "vrt_internal.h"

namespace vrt {

constexpr size_t kNoAllocMaxPixels = 1920u * 1080u;

// One rgba16f image (8 bytes per pixel) of the a-trous chain.
static __device__ __align__(256) uint2 g_noalloc_scratch[kNoAllocMaxPixels];

// Device address of g_noalloc_scratch on the current device.  In host code the
// symbol name is only a stand-in for the device array, so the address is
// looked up with the device current -- on every call: the lookup allocates
// nothing, and a cached address would go stale if the host recreated the
// device's primary context.
static cudaError_t scratch_address(void** out) { return cudaGetSymbolAddress(out, g_noalloc_scratch); }

static bool ranges_overlap(const void* a, size_t na, const void* b, size_t nb) {
  const uintptr_t a0 = reinterpret_cast<uintptr_t>(a), b0 = reinterpret_cast<uintptr_t>(b);
  return a0 < b0 + nb && b0 < a0 + na;
}

}  // namespace vrt

using namespace vrt;

static int vrt_noalloc_fail(int code, const char* msg) { return vrt::set_error(code, msg); }

extern "C" int vrt_denoise_atrous_noalloc(const void* accum, int accum_f32, const float* gbuf, void* out, int width,
                                          int height, void* stream) {
  if (!accum || !gbuf || !out) return vrt_noalloc_fail(VRT_ERR_INVALID, "vrt_denoise_atrous_noalloc: NULL buffer");
  if (width < 1 || height < 1)
    return vrt_noalloc_fail(VRT_ERR_INVALID, "vrt_denoise_atrous_noalloc: empty image");
  if ((size_t)width * (size_t)height > kNoAllocMaxPixels)
    return vrt_noalloc_fail(VRT_ERR_INVALID,
                            "vrt_denoise_atrous_noalloc: image larger than its fixed scratch "
                            "(at most 1920x1080 = 2073600 pixels)");
  const size_t px = (size_t)width * (size_t)height;
  if (ranges_overlap(out, px * 8, accum, px * (accum_f32 ? 16 : 8)) || ranges_overlap(out, px * 8, gbuf, px * 16))
    return vrt_noalloc_fail(VRT_ERR_INVALID,
                            "vrt_denoise_atrous_noalloc: the output overlaps the history or the G-buffer "
                            "(the first iteration reads the neighbours of the pixels it writes)");
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess)
    return vrt_noalloc_fail(VRT_ERR_NO_DEVICE, "vrt_denoise_atrous_noalloc: no current CUDA device");
  void* scratch = nullptr;
  cudaError_t e = scratch_address(&scratch);
  if (e != cudaSuccess) return vrt_noalloc_fail(VRT_ERR_CUDA, cudaGetErrorString(e));
  cudaStream_t st = (cudaStream_t)stream;
  // history -> out (step 1) -> scratch (step 2) -> out (step 4), the chain
  // accum -> dA -> dB -> dA of the frame loop with dA = out, dB = scratch.
  // No error word is passed to the staged kernel: a tile whose bounded copy
  // wait ran out is left unwritten and the call still returns.
  e = launch_atrous_staged(width, height, accum, accum_f32 != 0, gbuf, out, 1, nullptr, st);
  if (e == cudaSuccess) e = launch_atrous_staged(width, height, out, false, gbuf, scratch, 2, nullptr, st);
  if (e == cudaSuccess) e = launch_atrous_staged(width, height, scratch, false, gbuf, out, 4, nullptr, st);
  if (e != cudaSuccess) return vrt_noalloc_fail(VRT_ERR_CUDA, cudaGetErrorString(e));
  return VRT_OK;
}
