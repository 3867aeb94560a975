// k_lights.cu -- the scene's emissive-face light list and per-brick light
// grid (scene.js:58-200, 435-461) built on the device, for scenes that are
// edited at run time (the reference builds them once on the CPU).
//
// Light list: every exposed face of an emissive voxel, voxels in z, y, x
// order and faces +x,-x,+y,-y,+z,-z within a voxel -- an ordered compaction:
// per-voxel face counts, a scan of per-block totals, then each block writes
// its lights at its offset.  Weights (emissiveFaceWeight) in double, as the
// reference's JavaScript numbers.
//
// Light grid: one thread per brick cell ranks every light by power /
// max(d^2, (BRICK/2)^2) with a facing test and keeps the top 16, replaying
// the reference's insertion order and its Float32Array roundings exactly.
#include "vrt_device.cuh"
#include "vrt_internal.h"

namespace vrt {

constexpr int kLgK = 16, kLgStride = 2 + 2 * kLgK;

__device__ __forceinline__ double light_weight_d(uint32_t m) {
  const double e = (double)((m >> 24) & 0xffu) / 255.0;
  if (e <= 0.0) return 0.0;
  const double r = (double)(m & 0xffu) / 255.0;
  const double g = (double)((m >> 8) & 0xffu) / 255.0;
  const double b = (double)((m >> 16) & 0xffu) / 255.0;
  return e * (((0.2126 * r) * r + (0.7152 * g) * g) + (0.0722 * b) * b);
}

// Exposed-face bit mask (bit f = face f is a light) of voxel i.
__device__ __forceinline__ uint32_t light_faces(const uint32_t* __restrict__ vox, int N, long long i) {
  const uint32_t m = __ldg(vox + i);
  if (((m >> 24) & 0xffu) == 0u || m == 0u) return 0u;
  const int x = (int)(i % N), y = (int)((i / N) % N), z = (int)(i / ((long long)N * N));
  const int d[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  uint32_t bits = 0u;
#pragma unroll
  for (int f = 0; f < 6; f++) {
    const int nx = x + d[f][0], ny = y + d[f][1], nz = z + d[f][2];
    const bool in = nx >= 0 && ny >= 0 && nz >= 0 && nx < N && ny < N && nz < N;
    if (!in || __ldg(vox + (size_t)nx + (size_t)ny * N + (size_t)nz * N * N) == 0u) bits |= 1u << f;
  }
  return bits;
}

// Block-wide exclusive scan of v over 1024 threads; returns the prefix, *total the sum.
__device__ __forceinline__ uint32_t block_scan_1024(uint32_t v, uint32_t* total) {
  __shared__ uint32_t warp_sums[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t s = warp_sums[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += t;
    }
    warp_sums[lane] = s;   // inclusive over warps
  }
  __syncthreads();
  const uint32_t before = warp == 0 ? 0u : warp_sums[warp - 1];
  *total = warp_sums[31];
  return before + incl - v;
}

__global__ void __launch_bounds__(1024) k_light_count(const uint32_t* __restrict__ vox, int N,
                                                      uint32_t* __restrict__ bsum) {
  const long long n3 = (long long)N * N * N;
  const long long i = (long long)blockIdx.x * 1024 + threadIdx.x;
  const uint32_t c = i < n3 ? (uint32_t)__popc(light_faces(vox, N, i)) : 0u;
  uint32_t total;
  block_scan_1024(c, &total);
  if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// Exclusive scan of the block totals by one block; total count to *count.
__global__ void __launch_bounds__(1024) k_light_offsets(uint32_t* __restrict__ bsum, int nb,
                                                        uint32_t* __restrict__ count) {
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0u;
  __syncthreads();
  for (int base = 0; base < nb; base += 1024) {
    const int i = base + threadIdx.x;
    const uint32_t v = i < nb ? bsum[i] : 0u;
    uint32_t total;
    const uint32_t ex = block_scan_1024(v, &total);
    const uint32_t c0 = carry;
    if (i < nb) bsum[i] = c0 + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry = c0 + total;
    __syncthreads();
  }
  if (threadIdx.x == 0) *count = carry;
}

__global__ void __launch_bounds__(1024) k_light_write(const uint32_t* __restrict__ vox, int N,
                                                      const uint32_t* __restrict__ boff, uint32_t* __restrict__ words,
                                                      double* __restrict__ weights) {
  const long long n3 = (long long)N * N * N;
  const long long i = (long long)blockIdx.x * 1024 + threadIdx.x;
  const uint32_t bits = i < n3 ? light_faces(vox, N, i) : 0u;
  uint32_t total;
  uint32_t slot = boff[blockIdx.x] + block_scan_1024((uint32_t)__popc(bits), &total);
  if (!bits) return;
  const uint32_t m = __ldg(vox + i);
  const double w = light_weight_d(m);
  const uint32_t x = (uint32_t)(i % N), y = (uint32_t)((i / N) % N), z = (uint32_t)(i / ((long long)N * N));
  for (int f = 0; f < 6; f++) {
    if (!((bits >> f) & 1u)) continue;
    words[2 * (size_t)slot] = x | (y << 9) | (z << 18) | ((uint32_t)f << 27);
    words[2 * (size_t)slot + 1] = m;
    weights[slot] = w;
    slot++;
  }
}

__global__ void __launch_bounds__(128) k_light_grid(int N, const uint32_t* __restrict__ words,
                                                    const double* __restrict__ weights, int n,
                                                    uint32_t* __restrict__ grid) {
  const int BG = N / kBrick;
  const int cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= BG * BG * BG) return;
  const int bx = cell % BG, by = (cell / BG) % BG, bz = cell / (BG * BG);
  const double ccx = (bx + 0.5) * kBrick, ccy = (by + 0.5) * kBrick, ccz = (bz + 0.5) * kBrick;
  const double eps = (kBrick / 2.0) * (kBrick / 2.0);
  uint32_t topIdx[kLgK];
  float topW[kLgK];
  int count = 0, minAt = 0;
  double minW = 0.0;
  for (int i = 0; i < n; i++) {
    const uint32_t w0 = __ldg(words + 2 * (size_t)i);
    const int v[3] = {(int)(w0 & 0x1ffu), (int)((w0 >> 9) & 0x1ffu), (int)((w0 >> 18) & 0x1ffu)};
    const int face = (int)((w0 >> 27) & 7u), axis = face >> 1, pos = (face & 1) == 0 ? 1 : 0;
    double c[3] = {v[0] + 0.5, v[1] + 0.5, v[2] + 0.5}, nn[3] = {0.0, 0.0, 0.0};
    c[axis] = (double)(v[axis] + pos);
    nn[axis] = pos ? 1.0 : -1.0;
    const double dx = ccx - c[0], dy = ccy - c[1], dz = ccz - c[2];
    if ((dx * nn[0] + dy * nn[1]) + dz * nn[2] <= 0.0) continue;
    const double d2 = (dx * dx + dy * dy) + dz * dz;
    const double w = __ldg(weights + i) / (d2 > eps ? d2 : eps);
    if (count < kLgK) {
      topIdx[count] = (uint32_t)i;
      topW[count] = (float)w;
      count++;
      if (count == kLgK) {
        minW = topW[0]; minAt = 0;
        for (int k = 1; k < kLgK; k++) if ((double)topW[k] < minW) { minW = topW[k]; minAt = k; }
      }
    } else if (w > minW) {
      topIdx[minAt] = (uint32_t)i;
      topW[minAt] = (float)w;
      minW = topW[0]; minAt = 0;
      for (int k = 1; k < kLgK; k++) if ((double)topW[k] < minW) { minW = topW[k]; minAt = k; }
    }
  }
  uint32_t* g = grid + (size_t)cell * kLgStride;
  double wSum = 0.0;
  for (int k = 0; k < count; k++) wSum += (double)topW[k];
  g[0] = (uint32_t)count;
  g[1] = __float_as_uint((float)wSum);
  for (int k = 0; k < kLgK; k++) {
    g[2 + 2 * k] = k < count ? topIdx[k] : 0u;
    g[3 + 2 * k] = k < count ? __float_as_uint(topW[k]) : 0u;
  }
}

int light_blocks(int N) { return (int)(((long long)N * N * N + 1023) / 1024); }

cudaError_t launch_light_count(const uint32_t* vox, int N, uint32_t* bsum, uint32_t* count, cudaStream_t st) {
  const int nb = light_blocks(N);
  k_light_count<<<nb, 1024, 0, st>>>(vox, N, bsum);
  k_light_offsets<<<1, 1024, 0, st>>>(bsum, nb, count);
  return cudaGetLastError();
}

cudaError_t launch_light_write(const uint32_t* vox, int N, const uint32_t* boff, uint32_t* words, double* weights,
                               cudaStream_t st) {
  k_light_write<<<light_blocks(N), 1024, 0, st>>>(vox, N, boff, words, weights);
  return cudaGetLastError();
}

cudaError_t launch_light_grid(int N, const uint32_t* words, const double* weights, int n, uint32_t* grid,
                              cudaStream_t st) {
  const int cells = (N / kBrick) * (N / kBrick) * (N / kBrick);
  k_light_grid<<<(cells + 127) / 128, 128, 0, st>>>(N, words, weights, n, grid);
  return cudaGetLastError();
}

}  // namespace vrt
