// k_atrous_tma.cu -- the a-trous iteration (atrous.wgsl:26-83) with its
// input tile staged in shared memory by TMA (cp.async.bulk.tensor).
//
// A CTA of 256 threads produces a 32 x 16 tile of output pixels (32 x 8 at
// step 4, whose halo is widest).  One thread
// issues two tiled bulk copies -- the G-buffer (rgba32f) and the source image
// (rgba16f or rgba32f) of the tile plus a halo of 2 * step pixels on each
// side -- completing on one mbarrier; pixels outside the image arrive as zeros
// (a zero normal gives a zero edge weight, the same as skipping the tap).
// The threads then convert the staged source to fp32 once per pixel, with its
// luminance in .w, over the copied tile itself (each thread reads its pixels
// before the block rewrites them: 32 bytes of shared memory per staged pixel,
// 49 KB at step 4), read their centre pixel with its history alpha from global
// memory, and evaluate the 24 taps from shared memory.  The per-tap
// arithmetic and its order are those of atrous_pixel (image_core.cuh), so the
// output is bit-identical to the plain kernel's.
//
// Constraints (checked by the launcher, which otherwise uses the plain
// kernel): 16-byte aligned buffers and, for an rgba16f source (8-byte pixels
// copied as 64-bit elements), an even width so that rows start on 16 bytes.
// The x coordinate of every copy is the tile origin minus the halo, an even
// pixel index, i.e. a multiple of 16 bytes for both element sizes.
#include <cuda.h>
#include <mutex>
#include "image_core.cuh"
#include "umma.cuh"
#include "vrt_device.cuh"
#include "vrt_internal.h"

namespace vrt {

constexpr int kTX = 32;                      // output tile width; height kTY: 16, or 8 at step 4
constexpr uint32_t kTmaSpin = 1u << 22;      // bounded wait for the copies (try_wait iterations)

__host__ __device__ constexpr int align128(int x) { return (x + 127) & ~127; }
__host__ __device__ constexpr int tile_px(int step, int ty) { return (kTX + 4 * step) * (ty + 4 * step); }
__host__ __device__ constexpr int tile_rows(int step) { return step >= 4 ? 8 : 16; }
// G-buffer tile + source tile (rgba16f or rgba32f as copied, expanded in place
// to fp32 with its luminance); the steps are 1, 2, 4.
__host__ __device__ constexpr int tile_smem(int step, int ty) {
  return align128(tile_px(step, ty) * 16) + tile_px(step, ty) * 16;
}
constexpr int kMaxTilePx = 1280;   // staged pixels of the largest tile (step 4, 8 rows: 1,152), rounded to 256
static_assert(tile_px(1, 16) <= kMaxTilePx && tile_px(2, 16) <= kMaxTilePx && tile_px(4, 8) <= kMaxTilePx, "tile");
static_assert(kMaxTilePx % 256 == 0, "staged pixels per thread");

__device__ __forceinline__ void mbar_expect_tx(uint64_t* mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(umma::smem_u32(mbar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* tm, int c0, int c1, uint64_t* mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          umma::smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(umma::smem_u32(mbar))
      : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* tm, int c0, int c1, int c2,
                                            uint64_t* mbar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(umma::smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(umma::smem_u32(mbar))
      : "memory");
}

// kTY: output rows per CTA (16, or 8 at step 4, where the halo is widest: 49 KB of
// shared memory per CTA at 16 rows, 37 KB at 8).
template <bool kSrcF32, int kTY>
__global__ void __launch_bounds__(256) k_atrous_tma(const __grid_constant__ CUtensorMap tm_src,
                                                    const __grid_constant__ CUtensorMap tm_g, int W, int H,
                                                    const void* __restrict__ src, uint2* __restrict__ dst, int step,
                                                    unsigned long long* err) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ uint64_t mbar;
  const int hx = 2 * step;
  const int RW = kTX + 2 * hx, RH = kTY + 2 * hx, npx = RW * RH;
  float4* sg = reinterpret_cast<float4*>(smem);
  uint8_t* ssrc = smem + align128(npx * 16);          // the source tile as copied, expanded in place below
  float4* sc = reinterpret_cast<float4*>(ssrc);
  const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
  const int t = threadIdx.x;
  if (t == 0) umma::mbar_init(&mbar, 1);
  __syncthreads();
  if (t == 0) {
    mbar_expect_tx(&mbar, (uint32_t)(npx * 16 + npx * (kSrcF32 ? 16 : 8)));
    tma_load_3d(sg, &tm_g, 0, x0 - hx, y0 - hx, &mbar);
    if (kSrcF32) tma_load_3d(ssrc, &tm_src, 0, x0 - hx, y0 - hx, &mbar);
    else tma_load_2d(ssrc, &tm_src, x0 - hx, y0 - hx, &mbar);
  }
  if (!__syncthreads_and(umma::mbar_wait(&mbar, 0, kTmaSpin) ? 1 : 0)) {
    // record the failure and give the copies in flight a last bounded wait
    if (t == 0 && err) atomicExch(err, 1ull);
    umma::mbar_wait(&mbar, 0, kTmaSpin);
    return;
  }
  // fp32 source with its luminance in .w, once per staged pixel, written over
  // the copied tile: an rgba32f pixel in its own slot; rgba16f pixels (half
  // the size) are read by every thread before the block rewrites them.
  if (kSrcF32) {
    for (int i = t; i < npx; i += 256) {
      float4 c = sc[i];
      c.w = luminance(c.x, c.y, c.z);
      sc[i] = c;
    }
  } else {
    uint2 raw[kMaxTilePx / 256];
#pragma unroll
    for (int k = 0; k < kMaxTilePx / 256; k++) {
      const int i = t + 256 * k;
      if (i < npx) raw[k] = reinterpret_cast<const uint2*>(ssrc)[i];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kMaxTilePx / 256; k++) {
      const int i = t + 256 * k;
      if (i < npx) {
        float4 c = unpack_h4(raw[k]);
        c.w = luminance(c.x, c.y, c.z);
        sc[i] = c;
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int half = 0; half < kTY / 8; half++) {
    const int lx = t & 31, ly = (t >> 5) + 8 * half;
    const int px = x0 + lx, py = y0 + ly;
    if (px >= W || py >= H) continue;
    const int ci = (ly + hx) * RW + (lx + hx);
    const size_t p = (size_t)py * W + px;
    const float4 center = kSrcF32 ? __ldg(reinterpret_cast<const float4*>(src) + p)
                                  : unpack_h4(__ldg(reinterpret_cast<const uint2*>(src) + p));
    const float4 v = atrous_pixel_tile(center, sg[ci], sg, sc, ci, RW, step);
    dst[p] = pack_h4(v.x, v.y, v.z, v.w);
  }
}

// ---------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// rgba32f image {4 channels, W, H} in boxes of {4, bw, bh}.
static bool map_f32x4(CUtensorMap* m, const void* base, int W, int H, int bw, int bh) {
  const cuuint64_t dims[3] = {4, (cuuint64_t)W, (cuuint64_t)H};
  const cuuint64_t strides[2] = {16, (cuuint64_t)W * 16};
  const cuuint32_t box[3] = {4, (cuuint32_t)bw, (cuuint32_t)bh};
  const cuuint32_t es[3] = {1, 1, 1};
  return encode_fn()(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(base), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// rgba16f image as one 64-bit element per pixel {W, H} in boxes of {bw, bh}.
static bool map_h4(CUtensorMap* m, const void* base, int W, int H, int bw, int bh) {
  const cuuint64_t dims[2] = {(cuuint64_t)W, (cuuint64_t)H};
  const cuuint64_t strides[1] = {(cuuint64_t)W * 8};
  const cuuint32_t box[2] = {(cuuint32_t)bw, (cuuint32_t)bh};
  const cuuint32_t es[2] = {1, 1};
  return encode_fn()(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, const_cast<void*>(base), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

cudaError_t launch_atrous_staged(int W, int H, const void* src, bool src_f32, const void* gbuf, void* dst, int step,
                                 unsigned long long* err, cudaStream_t st, int rows) {
  const bool aligned = ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(gbuf)) & 15u) == 0u;
  const bool ok = encode_fn() && aligned && (src_f32 || W % 2 == 0) && step >= 1 && step <= 4 && W > 0 && H > 0;
  if (!ok) return launch_atrous(W, H, src, src_f32, gbuf, dst, step, st);
  // rows: 16 = 16 at steps 1-2 and 8 at step 4; 0 (default) or 8 = 8 at every step (the whole frame measured
  // 1.918 against 1.942 ms per 1080p frame with the shading grids at 32 blocks per SM)
  const int ty = rows == 16 ? tile_rows(step) : 8;
  const int hx = 2 * step, bw = kTX + 2 * hx, bh = ty + 2 * hx;
  CUtensorMap tg, ts;
  const bool enc = map_f32x4(&tg, gbuf, W, H, bw, bh) &&
                   (src_f32 ? map_f32x4(&ts, src, W, H, bw, bh) : map_h4(&ts, src, W, H, bw, bh));
  if (!enc) return launch_atrous(W, H, src, src_f32, gbuf, dst, step, st);
  const int smem = tile_smem(step, ty);
  dim3 grid((W + kTX - 1) / kTX, (H + ty - 1) / ty);
  auto run = [&](auto* fn) -> cudaError_t {
    cudaError_t r = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (r != cudaSuccess) return r;
    fn<<<grid, 256, smem, st>>>(ts, tg, W, H, src, (uint2*)dst, step, err);
    return cudaGetLastError();
  };
  cudaError_t e;
  if (src_f32) e = ty == 8 ? run(k_atrous_tma<true, 8>) : run(k_atrous_tma<true, 16>);
  else e = ty == 8 ? run(k_atrous_tma<false, 8>) : run(k_atrous_tma<false, 16>);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

}  // namespace vrt
