// trace_kernel.cuh -- per-block helpers shared by the one-thread-per-pixel
// kernels (plain path megakernel, ray batches, ReSTIR passes).
#pragma once
#include "vrt_device.cuh"
#include "vrt_internal.h"
#include <cstring>

namespace vrt {

// Largest occupancy bitmap staged in shared memory (512^3 grid = 32 KB).
constexpr size_t kMaxSmemOccBytes = 64 * 1024;

// Stage the 1-bit-per-brick occupancy bitmap in shared memory (kSmem) or use
// the global copy.  Every thread of the block must call it.
template <bool kSmem>
VRT_DI const uint32_t* stage_occupancy(const DScene& S, uint32_t* s_occ) {
  if (!kSmem) return S.bits;
  const int nwords = (S.BG * S.BG * S.BG + 31) >> 5;
  for (int i = threadIdx.x; i < nwords; i += blockDim.x) s_occ[i] = __ldg(S.bits + i);
  __syncthreads();
  return s_occ;
}


inline DScene to_dscene(const SceneDev& s) {
  DScene d;
  d.vox = s.vox; d.masks = s.masks; d.bits = s.bits; d.N = s.N; d.BG = s.BG;
  return d;
}

inline Uni to_uni(const VrtUniforms& u) {
  Uni r;
  static_assert(sizeof(Uni) == sizeof(VrtUniforms), "uniform layouts differ");
  std::memcpy(&r, &u, sizeof(Uni));
  return r;
}

// Pixel of thread `threadIdx.x` in a 16 x 16 block whose eight warps each
// cover an 8 x 4 tile (coherent primary rays within a warp).
VRT_DI void block_pixel_16x16(int& gx, int& gy) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  gx = blockIdx.x * 16 + (warp & 1) * 8 + (lane & 7);
  gy = blockIdx.y * 16 + (warp >> 1) * 4 + (lane >> 3);
}

}  // namespace vrt
