/*
 * vrt.h -- C ABI of voxelrt_b200, a B200 (sm_100a) implementation of
 * VoxelRT's plain per-frame global-illumination path:
 *
 *   pathtrace (two-level brick->voxel DDA, 1-spp path, sun-cone NEE,
 *   emissive pickup, firefly clamp, albedo demodulation)
 *   -> temporal reprojection -> 3x edge-aware a-trous -> present.
 *
 * Buffer formats follow the reference renderer (src/main.js:335-360,
 * src/scene.js:411-433):
 *   voxels     u32[N^3], index x + y*N + z*N*N, packed R | G<<8 | B<<16 | E<<24
 *              (0 = air)                                   (voxel.wgsl:8-11)
 *   bricks     u32[(N/8)^3], non-zero when any voxel of the 8^3 brick is solid
 *   brickMasks u32[16*(N/8)^3], bit lx + 8*ly + 64*lz of brick bi in word
 *              bi*16 + (bit>>5)
 *   radiance   rgba16f (demodulated), albedo rgba8unorm (sqrt albedo),
 *   gbuffer    rgba32f (normal, hit distance; sky = (-rd, -1)),
 *   accum      rgba16f or rgba32f (history length in alpha), denoise rgba16f,
 *   ldr        rgba8 (the headless stand-in for the canvas present pass).
 *
 * Conventions: every call returns VRT_OK (0) or a VRT_ERR_* code and never
 * throws; vrt_last_error_string() describes the last failure on the calling
 * thread.  Each context owns one CUDA stream; calls on one context are
 * serialised by the caller (host-thread-safe per context).  Host pointers are
 * plain host memory; "_device" entry points take device pointers.
 */
#ifndef VRT_H_
#define VRT_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VRT_ABI_VERSION 1

enum {
  VRT_OK = 0,
  VRT_ERR_INVALID = 1,     /* bad argument or size                       */
  VRT_ERR_CUDA = 2,        /* CUDA runtime error (message has details)   */
  VRT_ERR_OOM = 3,         /* device allocation failed                   */
  VRT_ERR_NO_DEVICE = 4,   /* no CUDA device / extension unusable        */
  VRT_ERR_BUDGET = 5,      /* HBM admission budget exceeded              */
  VRT_ERR_TIMEOUT = 6,     /* a bounded device wait gave up              */
  VRT_ERR_STATE = 7        /* call not valid in the object's state       */
};

typedef struct VrtCtx VrtCtx;
typedef struct VrtScene VrtScene;
typedef struct VrtSession VrtSession;
typedef struct VrtBatch VrtBatch;
typedef struct VrtServer VrtServer;
typedef struct VrtMlp VrtMlp;

/* Uniform block, byte-identical to the reference's 304-byte UBO
 * (common.wgsl:13-35, packed by main.js:399-426). */
typedef struct VrtUniforms {
  float invViewProj[16];   /* column-major, WebGPU clip z in [0,1]            */
  float prevViewProj[16];
  float camPos[4];         /* xyz metres, w = time                             */
  float prevCamPos[4];
  float sunDir[4];         /* xyz towards the sun, w = cos(angular radius)     */
  float sunRadiance[4];    /* rgb irradiance, w = sky intensity                */
  uint32_t params0[4];     /* x frame index (RNG stream), y bounces,
                              z flags: bit0 temporal, bit1 denoise             */
  float params1[4];        /* x width, y height, z exposure                    */
  uint32_t params2[4];     /* x restir flags (common.wgsl:40-59): 0 = preset
                              base; with RF_RESTIR (1) any of TEMPORAL 2,
                              SPATIAL 4, PAIRED 8, DUPMAP 16, FOOTPRINT 32,
                              VECTOR 64, UNIFIED 128, PLANE 256, RESCUE 512,
                              FULLV 1024, CLAMP 2048, LIGHTPOWER 4096,
                              MIXSIGMA 8192, ADAPTCAND 16384, LIGHTGRID
                              65536, HISTISOLATE 262144; y light count;
                              z spatial taps                                  */
  float params3[4];        /* x = temporal confidence cap (default 20)         */
  float params4[4];        /* x = spatial disk radius in pixels (default 30),
                              y = max temporal history (default 64)            */
  float params5[4];
  float params6[4];
} VrtUniforms;

typedef struct VrtDeviceConfig {
  int device;                 /* CUDA ordinal                                  */
  uint64_t hbm_budget_bytes;  /* 0 = no admission limit                        */
} VrtDeviceConfig;

typedef struct VrtSessionConfig {
  int width, height;          /* render size in pixels                         */
  float firefly_clamp;        /* FCLAMP_VALUE (pathtrace.wgsl:35); <=0 = off   */
  int accum_f32;              /* 1: rgba32f history, 0: rgba16f                */
  int keep_radiance_f32;      /* 1: also store fp32 demodulated radiance       */
  int path_kernel;            /* VRT_PATH_WAVEFRONT (default) or _MEGAKERNEL   */
} VrtSessionConfig;

enum {
  VRT_PATH_WAVEFRONT = 0,     /* queued waves + persistent refilling DDA       */
  VRT_PATH_MEGAKERNEL = 1,    /* one thread walks a whole path                 */
  VRT_PATH_BATCH_ONLY = 2     /* rendered only through a VrtBatch: the session
                                 holds no path-tracing scratch of its own      */
};

/* Launch-shape knobs of the wavefront path tracer; 0 keeps the default. */
typedef struct VrtTuning {
  int refill_min;             /* idle lanes of a warp that trigger a refill    */
  int trace_blocks_per_sm;    /* persistent DDA blocks per SM (0 = max)        */
  int shade_blocks_per_sm;    /* shading kernel blocks per SM                  */
  int trace_variant;          /* tracer variant: (DDA iterations per pass of the
                                 warp bookkeeping, min blocks per SM) =
                                 0: (8,5) default, 1: (6,5), 2: (6,4), 3: (4,4),
                                 4: (2,1), 5: (1,1); 6, 7, 8: (8,5) with the
                                 step loop unrolled 1, 2, 4 times (not 8)        */
  int atrous_tile_rows;       /* a-trous output tile rows: 0 (default) or 8 = 8
                                 at every step, 16 = 16 at steps 1-2 and 8 at
                                 step 4                                          */
  int tail_wave;              /* first wave whose remaining paths each finish on
                                 one thread (their rays traced in turn, not in
                                 per-wave launches); 0 = never, -1 = automatic
                                 (wave 2 for a cache-assisted session, or for a
                                 batch whose every job is cache-assisted; else
                                 never); the image is the same either way      */
} VrtTuning;

/* One traced ray (vrt_trace_rays).  face: 0..5 = +x,-x,+y,-y,+z,-z normal,
 * -1 on miss.  steps = brick iterations + voxel iterations entered;
 * bytes = 4 * (brick words + mask words + voxel words read). */
typedef struct VrtHit {
  float t;                    /* metres, < 0 on miss                           */
  float n[3];
  uint32_t mat;
  int32_t voxel[3];
  int32_t face;
  uint32_t steps;
  uint32_t bytes;
  uint32_t pad;
} VrtHit;

typedef struct VrtFrameStats {
  uint64_t rays;              /* trace() invocations (primary+bounce+shadow)   */
  uint64_t dda_outer;         /* brick iterations                              */
  uint64_t dda_inner;         /* voxel iterations                              */
  uint64_t voxel_reads;
  uint64_t pixels;
  float ms_pathtrace, ms_temporal, ms_atrous, ms_present, ms_total;
  uint32_t launches;          /* kernels launched by the frame                 */
  uint32_t trace_launches;    /* wavefront trace launches timed in ms_trace    */
  float ms_trace;             /* summed duration of those trace launches       */
  uint32_t cache_on;          /* 1: the frame was cache-assisted               */
  uint64_t cache_queries;     /* paths that ended in a cache query             */
  uint64_t cache_samples;     /* training samples produced by training paths   */
  float ms_cache;             /* cache inference + resolve + training steps    */
  float ms_reuse;             /* ReSTIR frames: reuse passes (inside
                                 ms_pathtrace, which covers all three)         */
  uint64_t trace_step_slots;  /* wavefront tracer: lane slots of its DDA steps
                                 (32 x steps per pass x warp passes); the
                                 brick + voxel iterations over this is the
                                 tracer's SIMT (warp execution) efficiency     */
} VrtFrameStats;

/* Camera pose of the reference's fly camera (camera.js:1-57). */
typedef struct VrtCameraPose {
  double pos[3];              /* metres                                        */
  double yaw, pitch;          /* radians; yaw 0 faces +Z                       */
  double fov_y;               /* radians (reference default 70 deg)            */
  double near_z, far_z;       /* 0.05, 400 in the reference                    */
} VrtCameraPose;

typedef struct VrtLighting {
  float sun_dir[3];           /* towards the sun, normalised by the callee     */
  float sun_cos_radius;       /* cos(angular radius)                           */
  float sun_irradiance[3];
  float sky_intensity;
} VrtLighting;

/* Scene generators (host only; no GPU needed). */
enum {
  VRT_SCENE_VOXELRT = 0,      /* scene.js 'default' world (noise seed = seed)  */
  VRT_SCENE_SMALL = 1,        /* 64^3 terrain + 24^3 Cornell box              */
  VRT_SCENE_FULL = 2,         /* terrain, room, 40 trees, RGB lanterns        */
  VRT_SCENE_RANDOM = 3,       /* terrain + boxes, 0.1% emissive U(1,20)       */
  VRT_SCENE_VOXELRT_LAMPS = 4 /* scene.js 'lamps' variant (scene.js:303-409)  */
};

/* ---- context ----------------------------------------------------------- */
/* Replaces WebGPU requestAdapter/requestDevice (main.js:138-159).  Creates
 * the context's stream and builds its present lookup table on it (an
 * exhaustive pass over the floats below 8, ~5 ms of GPU time, asynchronous). */
int vrt_create(const VrtDeviceConfig* cfg, VrtCtx** out);
int vrt_destroy(VrtCtx* ctx);
int vrt_ctx_synchronize(VrtCtx* ctx);
/* Bytes of device memory currently held by scenes and sessions of ctx. */
uint64_t vrt_ctx_bytes_in_use(const VrtCtx* ctx);
const char* vrt_last_error_string(void);
int vrt_abi_version(void);

/* ---- scene ------------------------------------------------------------- */
/* Replaces generateScene() upload + brick build (main.js:188-203,
 * scene.js:411-433): uploads voxels and builds bricks/masks on the device. */
int vrt_scene_upload(VrtCtx* ctx, const uint32_t* voxels, int N, VrtScene** out);
/* Same, with caller-built bricks and masks (reference writeBuffer path). */
int vrt_scene_upload_prebuilt(VrtCtx* ctx, const uint32_t* voxels, const uint32_t* bricks,
                              const uint32_t* brick_masks, int N, VrtScene** out);
/* Sets every voxel of the inclusive box to value and updates the affected
 * bricks and masks (VoxelBench scene events, scenes.h:8-12). */
int vrt_scene_edit_box(VrtScene* scene, int x0, int y0, int z0, int x1, int y1, int z1,
                       uint32_t value);
int vrt_scene_read(VrtScene* scene, uint32_t* voxels, uint32_t* bricks, uint32_t* brick_masks);
int vrt_scene_destroy(VrtScene* scene);

/* ---- DDA parity entry (voxel.wgsl:73-157 trace/traceShadow) ------------ */
int vrt_trace_rays(VrtScene* scene, const float* origins, const float* dirs, const float* tmax,
                   int n, VrtHit* out);
int vrt_trace_rays_device(VrtScene* scene, const float* d_origins, const float* d_dirs,
                          const float* d_tmax, int n, VrtHit* d_out);

/* ---- session (per-view render targets, main.js:335-360) ---------------- */
int vrt_session_create(VrtCtx* ctx, VrtScene* scene, const VrtSessionConfig* cfg, VrtSession** out);
int vrt_session_destroy(VrtSession* s);
int vrt_session_set_scene(VrtSession* s, VrtScene* scene);
/* Clears history (next frame starts with parity 0 and empty history). */
int vrt_session_reset(VrtSession* s);
/* One frame: pathtrace -> [ReSTIR: reuse_temporal (RF_TEMPORAL) ->
 * reuse_spatial] -> temporal -> (if params0.z bit1) a-trous x3 -> present,
 * ping-ponging G-buffer/history by frame parity (main.js:680-772). */
int vrt_frame(VrtSession* s, const VrtUniforms* u);
/* Individual passes of the same frame (parity of the frame in flight).
 * With RF_RESTIR in params2.x the path-trace pass is the reservoir pass of
 * pathtrace.wgsl:332-457 (initial candidates -> reservoirs A, pass-through
 * radiance -> direct); reuse_temporal merges the reprojected history
 * reservoirs B into A (reuse_temporal.wgsl, no-op without RF_TEMPORAL) and
 * reuse_spatial merges neighbours, shades the radiance and writes B
 * (reuse_spatial.wgsl). */
int vrt_pass_pathtrace(VrtSession* s, const VrtUniforms* u);
int vrt_pass_reuse_temporal(VrtSession* s, const VrtUniforms* u);
int vrt_pass_reuse_spatial(VrtSession* s, const VrtUniforms* u);
/* dupmap.wgsl: the duplication map of reservoirs B (no-op without
 * RF_DUPMAP); vrt_frame runs it after reuse_spatial (main.js:741). */
int vrt_pass_dupmap(VrtSession* s, const VrtUniforms* u);
/* Base sigma of the pairing textures of RF_PAIRED (main.js:73 `sigma`,
 * default 16); the wide tap's sigma under RF_MIXSIGMA is params5.x. */
int vrt_session_set_pairing_sigma(VrtSession* s, float sigma);
/* The pairing buffer itself (pairing.js:80-89, seeds 0xc0ffee + 7919 i):
 * 254^2 + 230^2 + 210^2 words for sigmas[0..2]; host only. */
int vrt_make_pairing(const double* sigmas, uint32_t* out, size_t words);
int vrt_pass_temporal(VrtSession* s, const VrtUniforms* u);
int vrt_pass_atrous(VrtSession* s, const VrtUniforms* u, int iteration /*0,1,2*/);
int vrt_pass_present(VrtSession* s, const VrtUniforms* u);
/* Ends a frame driven pass by pass (advances parity). */
int vrt_end_frame(VrtSession* s);
int vrt_session_set_tuning(VrtSession* s, const VrtTuning* t);
int vrt_session_get_tuning(VrtSession* s, VrtTuning* t);
/* Autotuner (no counterpart in the reference): times `frames` path-trace
 * passes of `u` for each candidate launch shape of the wavefront tracer and
 * keeps the fastest (returned in *best, its median pass time in *best_ms).
 * Resets the session's history. */
int vrt_session_autotune(VrtSession* s, const VrtUniforms* u, int frames, VrtTuning* best, float* best_ms);
/* Per-pass CUDA-event timings and in-kernel ray/step counters. */
int vrt_session_set_timing(VrtSession* s, int enable);
int vrt_session_last_stats(VrtSession* s, VrtFrameStats* out);

/* Readbacks of the last frame (HDR capture, main.js:571-661). bytes must be
 * at least W*H*bpp; returns VRT_ERR_INVALID otherwise. */
int vrt_read_radiance(VrtSession* s, void* host, size_t bytes);      /* rgba16f */
int vrt_read_radiance_f32(VrtSession* s, void* host, size_t bytes);  /* rgba32f */
int vrt_read_albedo(VrtSession* s, void* host, size_t bytes);        /* rgba8   */
int vrt_read_gbuffer(VrtSession* s, void* host, size_t bytes);       /* rgba32f */
int vrt_read_accum(VrtSession* s, void* host, size_t bytes);         /* f16/f32 */
int vrt_read_denoise(VrtSession* s, int index, void* host, size_t bytes); /* rgba16f */
int vrt_read_final(VrtSession* s, void* host, size_t bytes);         /* rgba16f/32f */
int vrt_read_ldr(VrtSession* s, void* host, size_t bytes);           /* rgba8   */
int vrt_read_hdr(VrtSession* s, float* host_rgb, size_t bytes);      /* f32 RGB */
/* ReSTIR state: reservoirs (which 0 = A, 1 = B; W*H records of 32 bytes in
 * the layout of restir.wgsl:14-27: posW f32 x 4, data u32 x 4) and the
 * pass-through radiance (rgba16f).  VRT_ERR_STATE before the first ReSTIR
 * frame of the session. */
int vrt_read_reservoirs(VrtSession* s, int which, void* host, size_t bytes);
int vrt_read_direct(VrtSession* s, void* host, size_t bytes);
int vrt_read_dupmap(VrtSession* s, void* host, size_t bytes);       /* f32 per pixel */
/* Writes history buffers (resume from a saved session state). */
int vrt_write_history(VrtSession* s, const void* accum_prev, const float* gbuf_prev);

/* ---- VoxelBench technique adapter (VoxelBench/pipeline/technique.h:8-14) --
 * A VoxelBench Technique estimates the indirect radiance of every G-buffer
 * pixel of the harness under a per-frame ray budget.  This object holds the
 * harness's world on the device and runs the estimator of its baseline
 * technique (techniques/pt.h: NEE paths, exponential history, edge-aware 5x5
 * filter) on this library's DDA.  Units are the harness's (voxels). */
typedef struct VrtVb VrtVb;

typedef struct VrtVbWorld {
  int nx, ny, nz;                /* grid size (core.h:64), any size up to 1024     */
  const uint8_t* grid;           /* material ids 0..15, index (z*ny + y)*nx + x    */
  float albedo[16][3];           /* MAT[m].alb                                     */
  float emission[16][3];         /* MAT[m].emi (emissive when the sum is > 0)      */
  const int32_t* emitters;       /* 5 per exposed emissive face: x, y, z, face, m  */
  int n_emitters;                /* (collectEmitters, core.cpp:133-141)            */
  int sky_enabled;               /* SKY (core.h:85-95)                             */
  float sun_dir[3], sun_e[3], zenith[3], horizon[3];
} VrtVbWorld;

typedef struct VrtVbPixel {      /* one GPix (core.h:119)                           */
  float pos[3];                  /* hit point (voxels)                              */
  float depth;
  float n[3];                    /* face normal                                     */
  uint32_t flags;                /* bit0 hit, bit1 the hit material is emissive     */
  float albedo[3];
  uint32_t pad;
} VrtVbPixel;

int vrt_vb_create(VrtCtx* ctx, int width, int height, VrtVb** out);
int vrt_vb_destroy(VrtVb* vb);
/* Uploads the world (Technique::init, and after a geometry or light event). */
int vrt_vb_set_world(VrtVb* vb, const VrtVbWorld* world);
/* Uploads the harness's G-buffer (width*height pixels, row-major). */
int vrt_vb_set_gbuffer(VrtVb* vb, const VrtVbPixel* pixels);
/* Clears the history (the next frame starts the estimate afresh). */
int vrt_vb_reset(VrtVb* vb);
/* Technique::frame(budget): one frame within `budget` rays; out_rgb (may be
 * NULL) receives width*height indirect radiances (RGB f32), *rays the rays
 * traced. */
int vrt_vb_frame(VrtVb* vb, long long budget, float* out_rgb, uint64_t* rays);

/* ---- batched frames (no counterpart in the reference) ------------------ */
/* A batch renders one frame for each of n sessions of one context in a
 * single launch sequence: one wavefront path trace over all sessions' pixels
 * (one persistent trace launch per wave serving every scene), then one
 * temporal, three a-trous and one present launch over all sessions.  Each
 * session keeps its own buffers, history and frame parity; every image is
 * bit-identical to rendering the session alone with vrt_frame.  The launch
 * sequence is captured once as a CUDA graph and replayed (re-captured when
 * the largest bounce count or the tuning changes). */
int vrt_batch_create(VrtCtx* ctx, VrtSession* const* sessions, int n, VrtBatch** out);
int vrt_batch_destroy(VrtBatch* b);
/* u: n uniform blocks, one per session, in creation order. */
int vrt_batch_frame(VrtBatch* b, const VrtUniforms* u);
/* One frame for the m sessions idx[0..m) of the batch (indices in creation
 * order), uniforms u[0..m); launched directly, without the graph. */
int vrt_batch_frame_subset(VrtBatch* b, const int* idx, int m, const VrtUniforms* u);
int vrt_batch_set_graph(VrtBatch* b, int enable);
int vrt_batch_set_tuning(VrtBatch* b, const VrtTuning* t);
/* Autotuner over whole batch frames (resets every session's history). */
int vrt_batch_autotune(VrtBatch* b, const VrtUniforms* u, int frames, VrtTuning* best, float* best_ms);
/* Counters of the last batch frame; ms_total = device time of the frame. */
int vrt_batch_last_stats(VrtBatch* b, VrtFrameStats* out);

/* ---- serving (no counterpart in the reference) -------------------------- */
/* A voxel edit applied to a session's scene before its frame renders. */
typedef struct VrtEditBox {
  int x0, y0, z0, x1, y1, z1;   /* inclusive voxel box (clipped to the grid)    */
  uint32_t value;               /* packed voxel written (0 = carve to air)      */
  int pad;
} VrtEditBox;

typedef struct VrtCompletion {
  uint64_t ticket;
  int session;
  int pad;
  double t_arrival;             /* seconds on the server clock                  */
  double t_done;                /* device completion time on the same clock     */
} VrtCompletion;

/* Continuous batching over device-resident sessions (each should own its
 * scene when requests carry edits).  A request renders the next frame of one
 * session after applying its edits.  Requests queue in arrival order; every
 * launch takes the oldest pending request of each idle session into one batch
 * frame, so requests that arrive while others are on the GPU join the next
 * launch; up to max_in_flight batch frames are queued on the device at once.
 * Frames of one session are rendered in request order, so each result equals
 * rendering the same request sequence alone. */
int vrt_server_create(VrtCtx* ctx, VrtSession* const* sessions, int n, int max_in_flight, VrtServer** out);
int vrt_server_destroy(VrtServer* sv);
/* Seconds since the server was created (clock of t_arrival / t_done). */
double vrt_server_now(VrtServer* sv);
/* t_arrival < 0 means now.  ldr_out (may be NULL) receives the frame's rgba8
 * image (W*H*4 bytes) when the request completes; pinned memory keeps the
 * copy asynchronous. */
int vrt_server_submit(VrtServer* sv, int session, const VrtUniforms* u, const VrtEditBox* edits, int n_edits,
                      double t_arrival, void* ldr_out, uint64_t* ticket);
/* Non-blocking: retires finished requests into out[0..max_out) and launches
 * new batch frames while device slots are free. */
int vrt_server_poll(VrtServer* sv, VrtCompletion* out, int max_out, int* n_out);
/* Blocks until every submitted request completed (or out[] is full). */
int vrt_server_drain(VrtServer* sv, VrtCompletion* out, int max_out, int* n_out);
int vrt_server_pending(VrtServer* sv, int* queued, int* in_flight);
/* No counterpart in the reference (a browser renderer serves one view).
 * A server whose sessions come and go: `max_sessions` slots and a scratch
 * pool for `max_pixels` pixels per batch launch (a launch takes the oldest
 * request of each idle session while their pixels fit).  Sessions enter
 * through the admission queue below. */
int vrt_server_create_dynamic(VrtCtx* ctx, int max_sessions, long long max_pixels, int max_in_flight,
                              VrtServer** out);
/* Admission by the context's HBM budget: queues a session (scene, config)
 * and creates it as soon as a slot is free and the budget has room for its
 * buffers, in arrival order -- immediately when it fits.  The server owns
 * the session.  *ticket names the open request. */
int vrt_server_open_session(VrtServer* sv, VrtScene* scene, const VrtSessionConfig* cfg, uint64_t* ticket);
/* The slot of an admitted session (VRT_ERR_STATE while it still waits). */
int vrt_server_session_of(VrtServer* sv, uint64_t ticket, int* slot);
/* Closes the session in `slot`: no new requests; once its queued and
 * in-flight requests are done it is destroyed (if the server created it),
 * its memory returns to the budget and waiting sessions are admitted. */
int vrt_server_close_session(VrtServer* sv, int slot);
/* Open sessions and sessions waiting for admission. */
int vrt_server_sessions(VrtServer* sv, int* open, int* waiting);
/* Sequential mode (on = 1): each launch renders the single oldest request
 * through its session's own frame path (vrt_frame), one after another --
 * the unbatched form the batched server is measured against.  Every session
 * needs its own path scratch (not VRT_PATH_BATCH_ONLY).  Only while idle. */
int vrt_server_set_sequential(VrtServer* sv, int on);
/* Batched mode with large sessions apart: a request of a session of at least
 * `pixels` pixels that has its own path scratch renders alone through its
 * frame path (a batch gains nothing from a view that fills the GPU by
 * itself); smaller sessions are batched together.  0 (default): every
 * request is batched. */
int vrt_server_set_solo_pixels(VrtServer* sv, long long pixels);
/* Batched mode: while fewer than `sessions` sessions have pending requests,
 * each launch renders the oldest request of a session with its own path
 * scratch alone through its frame path (a small batch costs a whole frame's
 * launch sequence and wave tails for a few views).  1 (default): always
 * batch. */
int vrt_server_set_min_batch(VrtServer* sv, int sessions);

/* ---- scene lights -------------------------------------------------------- */
/* The emissive-face light list, its power alias table and the per-brick
 * top-16 light grid of the scene (scene.js:58-200, 435-461: `lights`,
 * `lightAlias`, `lightGrid`), built from the scene's current voxels -- the
 * list and grid on the device, the O(n) alias pass on the host -- so a host
 * that edits the world can rebuild them per edit.  Same contents as the
 * reference's buffers: words (x | y<<9 | z<<18 | face<<27, material) per
 * light, (q, alias, pdf, 0) floats per light (4 floats when there are no
 * lights), 34 words per brick cell (count, f32 weight sum, 16 x (index, f32
 * weight)).  Grids up to 512^3. */
typedef struct VrtLightStats {
  uint32_t count;             /* emissive faces                                 */
  uint32_t pad;
  double total_weight;        /* sum of the face weights (emitted power proxy)  */
  float ms_list, ms_alias, ms_grid, pad2;   /* device list / host alias / device grid */
} VrtLightStats;
int vrt_scene_build_lights(VrtScene* s, VrtLightStats* stats);
int vrt_scene_read_lights(VrtScene* s, uint32_t* words, size_t words_bytes, float* alias, size_t alias_bytes,
                          uint32_t* grid, size_t grid_bytes);

/* ---- HDR reference pipeline -------------------------------------------- */
/* The reference's HDR capture (main.js:571-661: final illumination x (albedo
 * byte / 255)^2) and its converged-reference accumulation (test/bench.mjs
 * reference(), preset=base with a very long history), done on the device:
 * per-frame HDR radiance of the path-trace pass (the session must keep fp32
 * radiance) summed in FP64 -- the same double operations, in the same order,
 * as a CPU FP64 accumulation, so the sums are bit-identical to it -- plus
 * squared errors against a reference image, summed on the device. */
int vrt_hdr_accum_reset(VrtSession* s);
/* Adds the last path-trace pass's HDR radiance. */
int vrt_hdr_accum_add(VrtSession* s);
/* spp path-trace passes of u with frame indices frame0 .. frame0+spp-1, each added. */
int vrt_hdr_accumulate(VrtSession* s, const VrtUniforms* u, uint32_t frame0, int spp);
/* The FP64 sums (W*H*3 doubles) and the number of frames added. */
int vrt_hdr_accum_read(VrtSession* s, double* rgb, size_t bytes, uint32_t* count);
/* Reference image for the error calls: W*H*3 floats (HDR RGB). */
int vrt_hdr_set_reference(VrtSession* s, const float* rgb, size_t bytes);
/* Sum over pixels and channels of (last frame's HDR - reference)^2. */
int vrt_hdr_frame_error(VrtSession* s, double* sum_sq);
/* Sum over pixels and channels of (sums / count - reference)^2. */
int vrt_hdr_accum_error(VrtSession* s, double* sum_sq);

/* ---- radiance cache MLP (no counterpart in the reference) --------------- */
/* A 4-layer MLP (80 -> 64 -> 64 -> 64 -> 3, ReLU, no biases) mapping an
 * encoded path vertex to outgoing radiance.  Input per query: 9 floats --
 * position (metres), normal, albedo; the position is normalised by `extent`
 * (the world size in metres) and encoded as sin/cos of 12 octaves per axis.
 * BF16 weights and activations on the tensor cores (tcgen05, FP32
 * accumulation in TMEM); FP32 master weights and Adam (b1 0.9, b2 0.99).
 * Loss: relative L2, sum_c (o - y)^2 / (o^2 + 0.01), mean over samples.
 * Parameters: row-major W_l [K_in x N_out] back to back, the output layer
 * padded to 16 columns (columns 3..15 stay 0): vrt_mlp_num_params() floats. */
int vrt_mlp_create(VrtCtx* ctx, uint32_t seed, VrtMlp** out);
int vrt_mlp_destroy(VrtMlp* m);
int vrt_mlp_num_params(void);
int vrt_mlp_get_params(VrtMlp* m, float* host);
/* Sets the FP32 master weights and resets the Adam state. */
int vrt_mlp_set_params(VrtMlp* m, const float* host);
/* Encoded inputs (n x 80 bf16 bit patterns). */
int vrt_mlp_encode_device(VrtMlp* m, const float* d_q9, int n, float extent, uint16_t* d_feat);
/* d_out3: n x 3 predicted radiance. */
int vrt_mlp_infer_device(VrtMlp* m, const float* d_q9, int n, float extent, float* d_out3);
/* Gradient of the mean loss (d_grad: vrt_mlp_num_params() floats, may be NULL);
 * *loss_out (may be NULL) receives the mean loss. */
int vrt_mlp_gradient_device(VrtMlp* m, const float* d_q9, const float* d_y3, int n, float extent, float* d_grad,
                            float* loss_out);
/* `steps` Adam steps on the samples; *loss_out (may be NULL): loss before the first step. */
int vrt_mlp_train_device(VrtMlp* m, const float* d_q9, const float* d_y3, int n, float extent, float lr, int steps,
                         float* loss_out);
/* Reports a tensor-core wait that ran out in any earlier call (VRT_ERR_TIMEOUT). */
int vrt_mlp_check(VrtMlp* m);

/* ---- cache-assisted path tracing (no counterpart in the reference) ------- */
/* With the cache enabled a session's path-trace pass works as follows:
 *  - one pixel of every 4x4 block (rotating with the frame index) traces a
 *    full training path of `train_bounces` bounces (the plain estimator);
 *    its vertices 0..train_vertices-1 become training samples
 *    (position, normal, albedo -> reflected radiance gathered after it);
 *  - every other path ends at its first bounce hit: emission is picked up
 *    there and the reflected radiance is the network's prediction;
 *  - after the waves: one inference over the queries, then `train_steps`
 *    Adam steps of `train_batch` samples drawn from this frame's samples.
 * The uniforms' bounce count is ignored while the cache is on.  Wavefront
 * sessions only. */
typedef struct VrtCacheConfig {
  int enabled;
  int train_bounces;          /* default 6                                     */
  int train_vertices;         /* 1..8, default 3                               */
  int train_batch;            /* samples per Adam step, default 65536          */
  int train_steps;            /* Adam steps per frame, default 1               */
  float learning_rate;        /* default 1e-2                                  */
  uint32_t seed;              /* initial weights                               */
  int pad;
} VrtCacheConfig;
int vrt_session_set_cache(VrtSession* s, const VrtCacheConfig* cfg);
/* The session's network (owned by the session; NULL before the cache was enabled). */
int vrt_session_cache_mlp(VrtSession* s, VrtMlp** out);
/* Training samples of the last cache-assisted frame (in production order):
 * up to `cap` rows of q9 (position, normal, albedo) and y3 (target);
 * *count receives the number produced. */
int vrt_session_read_cache_samples(VrtSession* s, float* q9, float* y3, int cap, int* count);

/* ---- radiance cache tensor-core diagnostics ----------------------------- */
/* No counterpart in the reference.  Runs one tcgen05 GEMM on host data to check
 * the shared-memory operand layouts: mode 0: D[128 x N] = A[128 x K] B[N x K]^T;
 * mode 1: D[K x N] = A[128 x K]^T B[128 x N]; mode 2: D[128 x N] = A[128 x K] B[K x N]
 * (B read MN-major).  A, B are bf16 bit patterns. */
int vrt_mlp_selftest_gemm(int mode, int K, int N, const uint16_t* A, const uint16_t* B, float* D);
/* No counterpart in the reference.  Exercises the failure path of the
 * kernels' bounded waits: waits `spins` rounds on an mbarrier that nothing
 * arrives on, with TMEM held.  Returns VRT_ERR_TIMEOUT (the expected outcome);
 * the context stays usable. */
int vrt_selftest_bounded_wait(unsigned int spins);
/* No counterpart in the reference.  The present pass maps each channel value
 * below 8 to its rgba8 code through the context's threshold table instead of
 * evaluating ACES and pow(1/2.2) (present.wgsl:40-55); this runs every float
 * of [0, 8) through both and reports how many differ (*mismatches, 0 when the
 * table path is exact) and the smallest differing bit pattern (*first_bits,
 * 0xffffffff when none). */
int vrt_selftest_present(VrtCtx* ctx, uint64_t* mismatches, uint32_t* first_bits);

/* ---- session checkpoint / resume ----------------------------------------- */
/* No counterpart in the browser renderer; VoxelBench resumes its reference
 * accumulations from disk (VoxelBench/pipeline/harness.cpp:241-256).  A
 * checkpoint holds what the session's next frames depend on: the scene's
 * voxels, both history and G-buffer parities and the frame parity, the
 * radiance cache's network (fp32 weights, Adam moments and step), the ReSTIR
 * history (reservoirs, duplication map) and the HDR reference accumulation.
 * vrt_session_restore loads one into a session of the same size, history
 * format and scene size (the scene's bricks, masks and bitmap are rebuilt;
 * its lights are rebuilt on next use); the session then renders the same
 * frames the checkpointed one would -- bit for bit without the radiance
 * cache; with it the network comes back exactly, and later frames agree to
 * the order in which a frame's training samples are gathered, which is not
 * fixed in the original session either.  Host buffers; the calls
 * synchronize the context's stream.  VRT_ERR_INVALID for a buffer that is
 * not a checkpoint of a matching session. */
int vrt_session_checkpoint_size(VrtSession* s, uint64_t* bytes);
int vrt_session_checkpoint(VrtSession* s, void* host, uint64_t bytes);
int vrt_session_restore(VrtSession* s, const void* host, uint64_t bytes);

/* ---- allocation-free denoise ------------------------------------------- */
/* No counterpart in the reference.  The 3-iteration a-trous chain (steps
 * 1, 2, 4) on caller-owned device buffers, for callers that cannot allocate
 * device memory when they denoise (an engine whose device memory belongs to
 * its own allocator/budget, or a frame loop that must not call cudaMalloc,
 * which synchronizes the device).  d_accum: history, rgba16f (accum_f32 = 0)
 * or rgba32f (1); d_gbuf: rgba32f normal + distance; d_out: rgba16f result.
 * At most 1920x1080 pixels, and d_out may not overlap d_accum or d_gbuf
 * (VRT_ERR_INVALID otherwise, before anything is queued).  The intermediate
 * image lives in a fixed 16,588,800-byte device array of the library, held on
 * every GPU that loads it; each call looks up that array's address on the
 * current device, and the first call on a device also loads the library's
 * kernels there (make the first call before any stream capture).  Calls share
 * the array: calls that overlap on the GPU race and must be ordered by the
 * caller.  Work is queued on `stream` (a cudaStream_t, NULL = legacy default);
 * nothing is allocated or freed. */
int vrt_denoise_atrous_noalloc(const void* d_accum, int accum_f32, const float* d_gbuf, void* d_out, int width,
                               int height, void* stream);

/* ---- host helpers (no GPU) --------------------------------------------- */
/* Fills the uniform block like main.js writeUniforms (399-426). */
int vrt_make_uniforms(const VrtCameraPose* cur, const VrtCameraPose* prev, const VrtLighting* light,
                      uint32_t frame, uint32_t bounces, uint32_t flags, int width, int height,
                      float exposure, float max_history, VrtUniforms* out);
/* viewProj / invViewProj of camera.js:47-57 (column-major). */
int vrt_camera_matrices(const VrtCameraPose* pose, double aspect, float* view_proj,
                        float* inv_view_proj);
/* Benchmark camera path from a spawn pose: per frame the yaw advances
 * 0.5 degree and the position moves 0.05 m along the horizontal heading. */
int vrt_camera_spline(const VrtCameraPose* spawn, int frame, VrtCameraPose* out);
/* Procedural scenes; out_voxels holds N^3 words; spawn (may be NULL)
 * receives the default camera pose for the scene. */
int vrt_scene_generate(int kind, int N, uint32_t seed, uint32_t* out_voxels, VrtCameraPose* spawn);

#ifdef __cplusplus
}
#endif
#endif /* VRT_H_ */
