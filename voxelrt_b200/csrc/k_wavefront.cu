// k_wavefront.cu -- wavefront form of the plain path tracer (sm_100a), for
// one session.
//
// The megakernel (k_trace.cu) runs one path per thread; its warps idle on
// sky pixels, skipped shadow rays and on the longest DDA walk of each warp
// (ncu: ~11% of lanes active per instruction).  Here a frame is split into
// waves:
//
//   generate  : per pixel RNG init, sub-pixel jitter, camera ray
//   trace(0)  : primary rays (implicit queue = all pixels)
//   shade(0)  : G-buffer/albedo, vertex 0 (emission, sun NEE sample, bounce
//               sample) -> shadow + bounce rays appended to queue 1
//   trace(k)  : queue k;  shade(k): resolve vertex k-1's shadow ray, shade
//               vertex k, append queue k+1 ... until every path terminated.
//
// Queues and active-path lists are compacted with warp ballots (one atomic
// per warp).  The trace kernel is persistent: each warp owns 32 lanes that
// walk the DDA as a flat state machine shared by brick-level and voxel-level
// lanes; lanes whose ray ended are refilled from the queue once enough of
// them are idle, so warps stay full until the queue drains.  The kernels are
// defined in wavefront_core.cuh and shared with the batched form (k_batch.cu).
//
// The per-path arithmetic (RNG draws, shading, order of radiance sums) is
// exactly the megakernel's, so results are bit-identical to it and to the
// CPU oracle.
#include "wavefront_core.cuh"
#include <algorithm>
#include <cstring>

namespace vrt {

// Queue capacity: a plain path appends at most a shadow and a bounce ray per
// wave; with several slots a path (or the spatial pass's pixel) up to four.
static size_t queue_entries(size_t P, int slots) { return (slots > 1 ? 4 : 2) * P; }

size_t wavefront_bytes(int W, int H, int max_waves, int slots) {
  const size_t P = (size_t)W * H;
  return P * 16 * (4 + 3 * (size_t)slots) + queue_entries(P, slots) * 4 * 2 + P * 4 * 2 + (size_t)max_waves * 16;
}

void carve_wavefront(void* mem, size_t P, int max_waves, WavefrontBufs& wb, int slots) {
  char* m = (char*)mem;
  const size_t big = (size_t)slots * P;
  void** f4[7] = {&wb.R0, &wb.R1, &wb.R2, &wb.S0, &wb.S1, &wb.S2, &wb.hit};
  for (auto* f : f4) {
    const bool twice = f == &wb.R0 || f == &wb.R2 || f == &wb.hit;
    *f = m;
    m += (twice ? big : P) * 16;
  }
  for (int i = 0; i < 2; i++) { wb.q[i] = (uint32_t*)m; m += queue_entries(P, slots) * 4; }
  wb.qcap = queue_entries(P, slots);
  for (int i = 0; i < 2; i++) { wb.act[i] = (uint32_t*)m; m += P * 4; }
  wb.ctr = (int*)m;
  wb.max_waves = max_waves;
  wb.slots = slots;
}

static SingleJob make_job(const SceneDev& s, const VrtUniforms& uu, float fclamp, int W, int H, const PathOut& out) {
  SingleJob job;
  std::memcpy(&job.u, &uu, sizeof(Uni));
  job.S.vox = s.vox; job.S.masks = s.masks; job.S.bits = s.bits; job.S.N = s.N; job.S.BG = s.BG;
  job.out.rad16 = (uint2*)out.rad16;
  job.out.rad32 = (float4*)out.rad32;
  job.out.alb8 = out.alb8;
  job.out.gbuf = (float4*)out.gbuf;
  job.fclamp = fclamp;
  job.W = W;
  job.H = H;
  return job;
}

cudaError_t launch_wavefront(const SceneDev& s, const VrtUniforms& uu, float fclamp, int W, int H,
                             const PathOut& out, const WavefrontBufs& wb, const WavefrontTuning& tune,
                             cudaStream_t st, uint32_t* launches, cudaEvent_t* trace_ev, int max_timed_waves,
                             int* timed_waves, const CacheLaunch* cache, cudaEvent_t* cache_ev) {
  SingleJob job = make_job(s, uu, fclamp, W, H, out);
  std::memset(&job.cc, 0, sizeof job.cc);
  if (cache) job.cc = cache->cd;
  // cache-assisted frames run as many waves as their training paths need
  const int waves = (job.cc.on ? (int)job.cc.train_bounces : (int)job.u.params0[1]) + 2;
  const int smem_occ = (int)(occ_words(s.BG) * sizeof(uint32_t));
  const int smem = smem_occ <= 64 * 1024 ? smem_occ : 0;
  // cache frames: every path but the training paths ends at its first bounce
  // (wave 1), so by default the few paths left after it run to their end one
  // thread each
  const int tail = tune.tail_wave >= 0 ? tune.tail_wave : (job.cc.on ? 2 : 0);
  cudaError_t e = wf_launch_frame(job, (uint32_t)(W * H), waves, smem, wb, tune, out.stats, st, launches, trace_ev,
                                  max_timed_waves, timed_waves, 1, tail);
  if (e != cudaSuccess || !job.cc.on) return e;
  if (cache_ev && (e = cudaEventRecord(cache_ev[0], st)) != cudaSuccess) return e;
  e = launch_cache_post(job, wf_view(wb), cache, 1, out.stats, st, launches);
  if (e != cudaSuccess) return e;
  if (cache_ev) e = cudaEventRecord(cache_ev[1], st);
  return e;
}

}  // namespace vrt
