// vrt_internal.h -- launch wrappers shared by the C-ABI layer and the kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/vrt.h"

namespace vrt {

// Device-resident scene: packed voxels, per-brick words and masks, plus the
// 1-bit-per-brick occupancy bitmap the traversal stages in shared memory.
struct SceneDev {
  uint32_t* vox = nullptr;     // N^3
  uint32_t* bricks = nullptr;  // BG^3
  uint32_t* masks = nullptr;   // 16 * BG^3
  uint32_t* bits = nullptr;    // ceil(BG^3 / 32)
  int N = 0, BG = 0;
};

inline size_t occ_words(int BG) { return ((size_t)BG * BG * BG + 31) / 32; }

// Per-frame counters written by the path kernel (u64 each).
enum StatSlot {
  kStatRays = 0, kStatOuter, kStatInner, kStatVReads, kStatPixels, kStatCacheQueries, kStatCacheSamples,
  kStatError,   // nonzero: a bounded wait on staged copies ran out
  kStatTraceSlots,   // lane step slots of the queue tracer: 32 x steps per pass x passes, per warp
  kStatCount = 9
};
static_assert(kStatRays == 0 && kStatOuter == 1 && kStatInner == 2 && kStatVReads == 3 && kStatPixels == 4,
              "block_flush_stats adds to the first five counters in this order");

// Device pointers of one frame's path-trace outputs.
struct PathOut {
  void* rad16 = nullptr;       // rgba16f  (uint2 per pixel)
  void* rad32 = nullptr;       // rgba32f  (optional)
  uint32_t* alb8 = nullptr;    // rgba8
  void* gbuf = nullptr;        // rgba32f  (float4 per pixel)
  unsigned long long* stats = nullptr;
};

// Scratch of the wavefront path tracer (per session, carved from one
// allocation): per-pixel path state, ray queues, active lists, counters.
struct WavefrontBufs {
  void *R0 = nullptr, *R1 = nullptr, *R2 = nullptr;   // float4 per pixel (R0, R2: slots x P)
  void *S0 = nullptr, *S1 = nullptr, *S2 = nullptr;   // float4 per pixel
  void* hit = nullptr;                                // uint4 per pixel (slots x P)
  uint32_t* q[2] = {nullptr, nullptr};                // 2P entries each (4P with several slots)
  uint32_t* act[2] = {nullptr, nullptr};              // P entries each
  int* ctr = nullptr;                                 // 4 ints per wave
  size_t qcap = 0;                                    // entries per queue
  int max_waves = 0;
  int slots = 1;                                      // shadow-ray slots per path: ray k of path g is
                                                      // traced as path g + k P
};

// Radiance-cache state of one cache-assisted wavefront frame (device
// pointers; see wavefront_core.cuh for how the kernels use it).
constexpr int kCacheMaxRec = 8;   // record slots per training path

struct CacheDev {
  int on;
  uint32_t train_bounces;   // bounce count of training paths
  int rec_vertices;         // vertices 0..rec_vertices-1 give training samples
  uint32_t phase;           // training pixels: (x & 3, y & 3) == (phase & 3, phase >> 2)
  int TW;                   // training paths per image row: ceil(W / 4)
  float tclamp;             // per-channel clamp of training targets (<= 0: none)
  float4* rec;              // [T][kCacheMaxRec][4]: (pos, R.x) (normal, R.y) (albedo, R.z) (tp, 0)
  int* rec_n;               // [T] records written by the training path
  float* qbuf;              // [P][9] cache queries: position, normal, albedo
  uint32_t* qpix;           // [P] path id of each query
  int* qcount;
  float* cand_q9;           // [cap][9] training samples
  float* cand_y3;           // [cap][3]
  int* cand_count;          // samples produced this frame (may exceed cap)
  int cand_cap;
};


// Launch-shape knobs of the wavefront tracer (chosen by the autotuner).
struct WavefrontTuning {
  int refill_min = 8;           // idle lanes that trigger a warp refill
  int trace_blocks_per_sm = 0;  // 0 = occupancy maximum
  int shade_blocks_per_sm = 32;
  int trace_variant = 0;        // (DDA iterations per warp-bookkeeping pass, min blocks/SM):
                                // 0: (8, 5)  1: (6, 5)  2: (6, 4)  3: (4, 4)  4: (2, 1)  5: (1, 1);
                                // 6, 7, 8: (8, 5) with the step loop unrolled 1, 2, 4 times
  int atrous_rows = 0;          // a-trous output tile rows: 0 or 8 = 8 at all steps, 16 = 16 at steps 1-2 and 8 at step 4
  int tail_wave = -1;           // first wave whose paths finish one thread each (k_wf_tail); 0 = never;
                                // -1 = automatic: wave 2 for cache-assisted frames (a session's, or a
                                // batch's whose every job has the cache on), else never
};

// Host mirror of the device job table entry (JobDev in wavefront_core.cuh):
// one session rendered inside a batch frame.  Same field order and layout.
struct JobHost {
  VrtUniforms u;
  const uint32_t* vox;
  const uint32_t* masks;
  const uint32_t* bits;
  int N, BG;
  void* rad16;
  void* rad32;
  uint32_t* alb8;
  void* gbuf;
  int W, H;
  uint32_t first;
  float fclamp;
  const void* acc_prev;
  void* acc_cur;
  const void* gbuf_prev;
  void* den0;
  void* den1;
  uint32_t* ldr;
  int acc_f32;
  int pad[3];
  CacheDev cache;
};

// The batch a-trous tile tables: per job, the prefix counts of its 32 x 16 and
// 32 x 8 output tiles (m + 1 entries each, in device memory) and their totals.
struct AtrousTiles {
  const uint32_t* d16;
  const uint32_t* d8;
  uint32_t n16, n8;
};


// Post-wave cache work of one job: its queries, network and training state.
struct CacheLaunch {
  CacheDev cd;
  uint16_t* wb = nullptr;     // bf16 weights
  float* wm = nullptr;        // fp32 masters
  float* m = nullptr;
  float* v = nullptr;
  float* grad = nullptr;
  float* partial = nullptr;
  float* loss = nullptr;
  int* err = nullptr;
  int* step = nullptr;        // device Adam step counter
  float* pred = nullptr;      // [P][3]
  int P = 0;
  float extent = 0.0f;
  int train_batch = 0, train_steps = 0;
  float lr = 0.0f;
};

// One batch frame over n jobs of P pixels in total: wavefront path trace
// (waves = max bounces + 2), the cache jobs' post-wave work, temporal,
// 3x a-trous, present.
cudaError_t launch_batch_frame(const void* d_jobs, const uint32_t* d_firsts, int n, uint32_t P, int waves,
                               const WavefrontBufs& wb, const WavefrontTuning& tune, unsigned long long* stats,
                               cudaStream_t st, uint32_t* launches, const float* present_lut,
                               const CacheLaunch* cls = nullptr, int ncl = 0, const AtrousTiles* at = nullptr);

// Radiance-cache MLP kernels (k_mlp.cu).  q9: n x 9 floats (position in
// metres, normal, albedo); y3: n x 3 target radiance; weights bf16 row-major.
int mlp_num_params();
int mlp_max_ctas();
cudaError_t mlp_encode(const float* q9, int n, float extent, uint16_t* out, cudaStream_t st);
// One network's share of an MLP launch.  A launch serves up to
// kMaxMlpTasks networks (the sessions of a batch); the task table travels as
// a kernel parameter, so a captured graph needs no table upload.
struct MlpTask {
  const uint16_t* wb;       // bf16 weights as the kernels' shared-memory image (k_mlp.cu)
  const float* q9;          // inputs [n][9]: position (metres), normal, albedo
  const float* y3;          // training targets [n][3]
  float* out3;              // inference output [n][3]
  const int* n_dev;         // count on the device (may be null: n_max is the count)
  int n_max;                // inference: bound on *n_dev; training: samples per step
  int pop_cap;              // training: population = min(*n_dev, pop_cap)
  uint32_t seed;            // training: sample draws (mixed with *step)
  float extent;             // world size in metres
  int* step;                // Adam step counter (advanced by the reduction)
  float* partial;           // per-CTA gradient partials [mlp_max_ctas()][params]
  float* loss;              // per-CTA loss sums
  float* grad;              // reduced gradient
  float* wm;                // fp32 masters
  float* m;
  float* v;
  uint16_t* wbw;            // bf16 copy written by Adam (= wb)
  float lr;
  int* err;                 // a bounded tensor-core wait ran out
  int cta0, ctas;           // CTA range of the task (set by the launcher)
};
constexpr int kMaxMlpTasks = 48;
struct MlpTaskSet {
  int n;
  int pad[3];
  MlpTask t[kMaxMlpTasks];
};
// Inference over every task's queries (count *n_dev, bounded by n_max).
cudaError_t mlp_infer_tasks(MlpTaskSet& ts, cudaStream_t st);
// Gradient of every task (per-CTA partials, then the fixed-order reduction,
// which advances *step when the step had samples).  Sample selection: with
// n_dev null the n_max samples in order; otherwise the population is
// min(*n_dev, pop_cap) samples and the step uses min(population, n_max) of
// them -- all in order when they fit, else uniform draws with replacement.
cudaError_t mlp_gradient_tasks(MlpTaskSet& ts, cudaStream_t st);
// Adam step number *step of every task (skipped when *n_dev == 0).
cudaError_t mlp_adam_tasks(const MlpTaskSet& ts, cudaStream_t st);
cudaError_t mlp_to_bf16(const float* wm, uint16_t* wb, cudaStream_t st);

// HDR reference pipeline (k_hdr.cu): FP64 sums of the capture's HDR value
// (demodulated radiance x (albedo byte / 255)^2) and per-block partial sums
// of squared errors (mode 0: last frame vs ref; mode 1: acc * inv_count vs ref).
int hdr_blocks(int P);
cudaError_t launch_hdr_add(int P, const void* rad32, const uint32_t* alb8, double* acc, cudaStream_t st);
cudaError_t launch_hdr_sq_err(int P, int mode, const void* rad32, const uint32_t* alb8, const double* acc,
                              double inv_count, const float* ref, double* part, cudaStream_t st);

// Scene lights (k_lights.cu): ordered light-list compaction and light grid.
int light_blocks(int N);
cudaError_t launch_light_count(const uint32_t* vox, int N, uint32_t* bsum, uint32_t* count, cudaStream_t st);
cudaError_t launch_light_write(const uint32_t* vox, int N, const uint32_t* boff, uint32_t* words, double* weights,
                               cudaStream_t st);
cudaError_t launch_light_grid(int N, const uint32_t* words, const double* weights, int n, uint32_t* grid,
                              cudaStream_t st);

// Records `msg` as the calling thread's vrt_last_error_string(); returns code.
int set_error(int code, const char* msg);

// slots: shadow-ray slots per path (1 for the plain path; the ReSTIR passes
// use up to 4: ray k of path g is traced as path g + k P in R0, R2 and hit).
size_t wavefront_bytes(int W, int H, int max_waves, int slots = 1);
// Lays the wavefront scratch of P pixels out in mem (wavefront_bytes(P, 1, max_waves, slots) bytes).
void carve_wavefront(void* mem, size_t P, int max_waves, WavefrontBufs& wb, int slots = 1);
// When trace_ev is non-null, events trace_ev[2w], trace_ev[2w+1] bracket the
// trace kernel of wave w (w < max_timed_waves); *timed_waves receives the count.
// cache (may be null): cache-assisted frame (training + query paths),
// followed by its post-wave work (events cache_ev[0..1] around it when given).
cudaError_t launch_wavefront(const SceneDev& s, const VrtUniforms& u, float fclamp, int W, int H,
                             const PathOut& out, const WavefrontBufs& wb, const WavefrontTuning& tune,
                             cudaStream_t st, uint32_t* launches, cudaEvent_t* trace_ev = nullptr,
                             int max_timed_waves = 0, int* timed_waves = nullptr, const CacheLaunch* cache = nullptr,
                             cudaEvent_t* cache_ev = nullptr);

cudaError_t launch_build_bricks(const SceneDev& s, int bx0, int by0, int bz0, int bx1, int by1, int bz1,
                                cudaStream_t st);
cudaError_t launch_build_bits(const SceneDev& s, cudaStream_t st);
cudaError_t launch_fill_box(const SceneDev& s, int x0, int y0, int z0, int x1, int y1, int z1, uint32_t value,
                            cudaStream_t st);
cudaError_t launch_pathtrace(const SceneDev& s, const VrtUniforms& u, float fclamp, int W, int H,
                             const PathOut& out, cudaStream_t st);
cudaError_t launch_trace_rays(const SceneDev& s, const float* o, const float* d, const float* tmax, int n,
                              VrtHit* out, cudaStream_t st);
cudaError_t launch_temporal(const VrtUniforms& u, int W, int H, const void* rad16, const void* gcur,
                            const void* acc_prev, const void* gprev, void* acc_out, bool acc_f32,
                            cudaStream_t st);
// The a-trous iteration with its input tile staged by TMA (falls back to
// launch_atrous when the buffers do not meet the copy constraints); err
// (may be null) is set when a bounded wait for the copies ran out.
cudaError_t launch_atrous_staged(int W, int H, const void* src, bool src_f32, const void* gbuf, void* dst, int step,
                                 unsigned long long* err, cudaStream_t st, int rows = 0);
cudaError_t launch_atrous(int W, int H, const void* src, bool src_f32, const void* gbuf, void* dst, int step,
                          cudaStream_t st);
// Present with the context's lookup table (kPresentLut 4-byte words: albedo
// factor per byte, the code thresholds and windows, the scan's scratch), built
// once per context by launch_present_lut.
constexpr int kPresentLut = 256 + 257 + 257 + 512;
cudaError_t launch_present(const VrtUniforms& u, int W, int H, const void* fin, bool fin_f32,
                           const uint32_t* alb8, uint32_t* ldr, const float* lut, cudaStream_t st);
cudaError_t launch_present_lut(float* lut, cudaStream_t st);
// Counts the floats of the table's range where the table path and the exact
// arithmetic give different codes (bad), and the smallest such bit pattern.
cudaError_t launch_present_check(const float* lut, unsigned long long* bad, unsigned int* first, cudaStream_t st);

// Reservoir flags of params2.x (common.wgsl:40-59).
constexpr uint32_t kRfRestir = 1u, kRfTemporal = 2u, kRfSpatial = 4u, kRfPaired = 8u, kRfDupmap = 16u,
                   kRfFootprint = 32u, kRfVector = 64u, kRfUnified = 128u, kRfPlane = 256u, kRfRescue = 512u,
                   kRfFullV = 1024u, kRfClamp = 2048u, kRfLightPower = 4096u, kRfMixSigma = 8192u,
                   kRfAdaptCand = 16384u, kRfConfDenoise = 32768u, kRfLightGrid = 65536u, kRfMutate = 131072u,
                   kRfHistIsolate = 262144u, kRfWorldGi = 524288u;
// The flags the library implements: every flag of the `gi`, `lin`, `ours` and
// `ours_motion` presets (main.js:40-62) plus footprint, mixed sigma, adaptive
// candidate counts and the light grid.
constexpr uint32_t kRestirFlagsImplemented =
    kRfRestir | kRfTemporal | kRfSpatial | kRfPaired | kRfDupmap | kRfFootprint | kRfVector | kRfUnified | kRfPlane |
    kRfRescue | kRfFullV | kRfClamp | kRfLightPower | kRfMixSigma | kRfAdaptCand | kRfLightGrid | kRfHistIsolate;

// Pairing textures of paired spatial reuse (pairing.js:74): sizes and offsets.
constexpr int kPairSizes[3] = {254, 230, 210};
constexpr uint32_t kPairingWords = 254u * 254u + 230u * 230u + 210u * 210u;
// pairing.js:26-70 restated: the three textures for sigmas[0..2] (uint32
// words of two i16 coordinate deltas), into out[kPairingWords].
void make_pairing_buffer(const double sigmas[3], uint32_t* out);

// ReSTIR reservoirs of one session (32 bytes per pixel each, the reference's
// record layout) and the pass-through radiance of the initial pass.
struct RestirBufs {
  void* resA = nullptr;             // working set: initial, then temporal merge
  void* resB = nullptr;             // post-spatial = next frame's history
  void* direct = nullptr;           // rgba16f
  const void* gbuf_prev = nullptr;  // previous frame's G-buffer
  void* scratch = nullptr;          // 80 B per pixel: wavefront path state (x2, RIS state)
  float* dup = nullptr;             // duplication score per pixel (dupmap.wgsl)
  const uint32_t* pairing = nullptr;      // kPairingWords (RF_PAIRED)
  const uint32_t* light_words = nullptr;  // 2 per light (RF_UNIFIED)
  const float* light_alias = nullptr;     // 4 per light
  const uint32_t* light_grid = nullptr;   // 34 per brick cell
};
cudaError_t launch_restir_initial(const SceneDev& s, const VrtUniforms& u, float fclamp, int W, int H,
                                  const PathOut& out, const RestirBufs& rb, cudaStream_t st);
// The initial pass on the wavefront tracer (bit-identical to launch_restir_initial).
cudaError_t launch_restir_initial_wavefront(const SceneDev& s, const VrtUniforms& u, float fclamp, int W, int H,
                                            const PathOut& out, const RestirBufs& rb, const WavefrontBufs& wb,
                                            const WavefrontTuning& tune, cudaStream_t st, uint32_t* launches,
                                            cudaEvent_t* trace_ev, int max_timed_waves, int* timed_waves);
// The unified (RF_UNIFIED) initial pass on the wavefront tracer.
cudaError_t launch_restir_unified_wavefront(const SceneDev& s, const VrtUniforms& u, float fclamp, int W, int H,
                                            const PathOut& out, const RestirBufs& rb, const WavefrontBufs& wb,
                                            const WavefrontTuning& tune, cudaStream_t st, uint32_t* launches,
                                            cudaEvent_t* trace_ev, int max_timed_waves, int* timed_waves);
cudaError_t launch_restir_temporal(const SceneDev& s, const VrtUniforms& u, int W, int H, const PathOut& out,
                                   const RestirBufs& rb, cudaStream_t st);
cudaError_t launch_restir_spatial(const SceneDev& s, const VrtUniforms& u, int W, int H, const PathOut& out,
                                  const RestirBufs& rb, cudaStream_t st);
// dupmap.wgsl: duplication score of every pixel from reservoirs B.
cudaError_t launch_restir_dupmap(const VrtUniforms& u, int W, int H, const RestirBufs& rb, cudaStream_t st);
// The spatial pass with its visibility rays on the wavefront tracer (select,
// trace, resolve; bit-identical to launch_restir_spatial).
cudaError_t launch_restir_spatial_wavefront(const SceneDev& s, const VrtUniforms& u, int W, int H, const PathOut& out,
                                            const RestirBufs& rb, const WavefrontBufs& wb,
                                            const WavefrontTuning& tune, cudaStream_t st, uint32_t* launches);

// One frame of the VoxelBench technique adapter (k_vb.cu).
struct VbLaunch {
  SceneDev scene;            // the harness's grid in the packed layout (material id in the low byte)
  int nx, ny, nz;            // the harness's grid size
  int W, H;
  const void* px;            // 3 float4 per pixel (VrtVbPixel)
  void* hist;                // float4 per pixel
  void* out;                 // float4 per pixel
  const int* emitters;       // 4 ints per emissive face
  int n_emitters;
  float albedo[16][3], emission[16][3];
  int sky;
  float sun_dir[3], sun_e[3], zenith[3], horizon[3];
  unsigned long long* rays;
  uint32_t fcount;
  int base_paths;
  double frac_p;
  int stride;
};
cudaError_t launch_vb_frame(const VbLaunch& L, cudaStream_t st);

}  // namespace vrt
