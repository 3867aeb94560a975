// k_batch.cu -- many independent views rendered in one launch sequence.
//
// A batch frame renders one frame for each of n sessions (different scenes,
// sizes, bounce counts, cameras).  The sessions' pixels are laid out back to
// back in one global index space; every kernel finds the job of a pixel by a
// binary search over the jobs' first pixels.  The wavefront path tracer runs
// over all jobs at once -- one persistent trace launch per wave serves rays
// of every scene -- followed by one temporal, three a-trous and one present
// launch over all jobs.  Per-pixel arithmetic is the single-session code
// (wavefront_core.cuh, image_core.cuh), so each job's image is bit-identical
// to rendering that session alone.
#include <cstddef>
#include "wavefront_core.cuh"
#include "image_core.cuh"

namespace vrt {

static_assert(sizeof(JobDev) == sizeof(JobHost), "job table layouts differ");
static_assert(offsetof(JobDev, S) == offsetof(JobHost, vox), "job table layouts differ");
static_assert(offsetof(JobDev, out) == offsetof(JobHost, rad16), "job table layouts differ");
static_assert(offsetof(JobDev, W) == offsetof(JobHost, W), "job table layouts differ");
static_assert(offsetof(JobDev, acc_prev) == offsetof(JobHost, acc_prev), "job table layouts differ");
static_assert(offsetof(JobDev, acc_f32) == offsetof(JobHost, acc_f32), "job table layouts differ");
static_assert(offsetof(JobDev, cache) == offsetof(JobHost, cache), "job table layouts differ");

// temporal.wgsl:17-77 over all jobs.
__global__ void __launch_bounds__(256) k_b_temporal(MultiJob J, uint32_t P) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= P) return;
  const int j = J.job_of(g);
  const JobDev& jd = J.jobs[j];
  const int W = jd.W, H = jd.H;
  const uint32_t lp = g - jd.first;
  const int x = (int)(lp % (uint32_t)W), y = (int)(lp / (uint32_t)W);
  const float4 res = temporal_pixel(jd.u, W, H, x, y, jd.out.rad16, jd.out.gbuf, jd.acc_prev, jd.acc_f32 != 0,
                                    jd.gbuf_prev);
  store_px(jd.acc_cur, jd.acc_f32 != 0, lp, res);
}

// atrous.wgsl:26-83 iteration `it` (step 1 << it) of every job whose denoise
// flag is set; chain accum -> dA -> dB -> dA (main.js:503-507).
__global__ void __launch_bounds__(256) k_b_atrous(MultiJob J, uint32_t P, int it) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= P) return;
  const int j = J.job_of(g);
  const JobDev& jd = J.jobs[j];
  if ((jd.u.params0[2] & 2u) == 0u) return;
  const int W = jd.W, H = jd.H;
  const uint32_t lp = g - jd.first;
  const int x = (int)(lp % (uint32_t)W), y = (int)(lp / (uint32_t)W);
  const void* src = it == 0 ? jd.acc_cur : (it == 1 ? (const void*)jd.den0 : (const void*)jd.den1);
  const bool srcF32 = it == 0 && jd.acc_f32 != 0;
  uint2* dst = it == 1 ? jd.den1 : jd.den0;
  const float4 v = atrous_pixel(W, H, x, y, src, srcF32, jd.out.gbuf, 1 << it);
  dst[lp] = pack_h4(v.x, v.y, v.z, v.w);
}

// The same iteration over shared-memory tiles: a CTA of 256 threads produces a
// 32 x kTY tile of one job (kTY = 16 at steps 1-2, 8 at step 4), staging the
// tile and its halo of 2 step pixels -- G-buffer as copied, source in fp32
// with its luminance in .w, zeros outside the image, whose zero normal drops
// the tap as the plain kernel's bounds test does -- with coalesced loads,
// then evaluating the taps from shared memory (atrous_pixel_tile: the
// arithmetic and order of atrous_pixel, so the same bits).  tiles: m + 1
// prefix counts of the jobs' tiles; CTA b finds its job by binary search.
template <int kTY>
__global__ void __launch_bounds__(256) k_b_atrous_tiled(MultiJob J, const uint32_t* __restrict__ tiles, int it) {
  extern __shared__ __align__(16) uint8_t smem[];
  const uint32_t b = blockIdx.x;
  int lo = 0, hi = J.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(tiles + mid) <= b) lo = mid;
    else hi = mid - 1;
  }
  const JobDev& jd = J.jobs[lo];
  if ((jd.u.params0[2] & 2u) == 0u) return;
  const int W = jd.W, H = jd.H, step = 1 << it;
  const int tb = (int)(b - __ldg(tiles + lo)), tw = (W + 31) / 32;
  const int x0 = (tb % tw) * 32, y0 = (tb / tw) * kTY;
  const int hx = 2 * step, RW = 32 + 2 * hx, RH = kTY + 2 * hx, npx = RW * RH;
  float4* sg = reinterpret_cast<float4*>(smem);
  float4* sc = sg + npx;
  const void* src = it == 0 ? jd.acc_cur : (it == 1 ? (const void*)jd.den0 : (const void*)jd.den1);
  const bool srcF32 = it == 0 && jd.acc_f32 != 0;
  uint2* dst = it == 1 ? jd.den1 : jd.den0;
  const float4* gb = jd.out.gbuf;
  for (int i = threadIdx.x; i < npx; i += 256) {
    const int qx = x0 - hx + i % RW, qy = y0 - hx + i / RW;
    float4 g4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), c4 = g4;
    if (qx >= 0 && qy >= 0 && qx < W && qy < H) {
      const size_t q = (size_t)qy * W + qx;
      g4 = __ldg(gb + q);
      c4 = load_px(src, srcF32, q);
      c4.w = luminance(c4.x, c4.y, c4.z);
    }
    sg[i] = g4;
    sc[i] = c4;
  }
  __syncthreads();
#pragma unroll
  for (int half = 0; half < kTY / 8; half++) {
    const int lx = threadIdx.x & 31, ly = (threadIdx.x >> 5) + 8 * half;
    const int px = x0 + lx, py = y0 + ly;
    if (px >= W || py >= H) continue;
    const int ci = (ly + hx) * RW + (lx + hx);
    const size_t p = (size_t)py * W + px;
    const float4 center = load_px(src, srcF32, p);
    const float4 v = atrous_pixel_tile(center, sg[ci], sg, sc, ci, RW, step);
    dst[p] = pack_h4(v.x, v.y, v.z, v.w);
  }
}

// present.wgsl:40-55 over all jobs.
__global__ void __launch_bounds__(256) k_b_present(MultiJob J, uint32_t P, const float* __restrict__ lut) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= P) return;
  const int j = J.job_of(g);
  const JobDev& jd = J.jobs[j];
  const uint32_t lp = g - jd.first;
  const bool denoise = (jd.u.params0[2] & 2u) != 0u;
  const float4 il = denoise ? load_px(jd.den0, false, lp) : load_px(jd.acc_cur, jd.acc_f32 != 0, lp);
  jd.ldr[lp] = present_pixel(jd.u.params1[2], il, __ldg(jd.out.alb8 + lp), lut);
}

cudaError_t launch_batch_frame(const void* d_jobs, const uint32_t* d_firsts, int n, uint32_t P, int waves,
                               const WavefrontBufs& wb, const WavefrontTuning& tune, unsigned long long* stats,
                               cudaStream_t st, uint32_t* launches, const float* present_lut, const CacheLaunch* cls,
                               int ncl, const AtrousTiles* at) {
  MultiJob J;
  J.jobs = (const JobDev*)d_jobs;
  J.firsts = d_firsts;
  J.n = n;
  J.cache_jobs = ncl;
  // tail wave: as tuned; automatic (-1) = wave 2 when every job is cache-assisted (only the
  // training paths remain after the first bounce), else never
  const int tail = tune.tail_wave >= 0 ? tune.tail_wave : (ncl > 0 && ncl == n ? 2 : 0);
  cudaError_t e = wf_launch_frame(J, P, waves, 0, wb, tune, stats, st, launches, nullptr, 0, nullptr, n, tail);
  if (e != cudaSuccess) return e;
  // the cache jobs' inference, resolve and training, all jobs per launch
  if (ncl > 0 && (e = launch_cache_post(J, wf_view(wb), cls, ncl, stats, st, launches)) != cudaSuccess) return e;
  const unsigned blocks = (P + 255) / 256;
  k_b_temporal<<<blocks, 256, 0, st>>>(J, P);
  for (int it = 0; it < 3; it++) {
    if (at && at->d16) {   // shared-memory tiles: 32 x 8 (tile rows 16: 32 x 16 at steps 1-2)
      const int step = 1 << it, hx = 2 * step;
      if (it < 2 && tune.atrous_rows == 16) {
        const int smem = (32 + 2 * hx) * (16 + 2 * hx) * 32;
        k_b_atrous_tiled<16><<<at->n16, 256, smem, st>>>(J, at->d16, it);
      } else {
        const int smem = (32 + 2 * hx) * (8 + 2 * hx) * 32;
        k_b_atrous_tiled<8><<<at->n8, 256, smem, st>>>(J, at->d8, it);
      }
    } else {
      k_b_atrous<<<blocks, 256, 0, st>>>(J, P, it);
    }
  }
  k_b_present<<<blocks, 256, 0, st>>>(J, P, present_lut);
  if (launches) *launches += 5;
  return cudaGetLastError();
}

}  // namespace vrt
