// wavefront.cuh -- building blocks of the wavefront path tracer shared by the
// single-session kernels (k_wavefront.cu) and the batched kernels
// (k_batch.cu): path-state layout, block-aggregated queue appends, the flat
// two-level DDA, and per-vertex shading.
#pragma once
#include "vrt_device.cuh"
#include "vrt_internal.h"
#include <algorithm>
#include <cstring>

namespace vrt {


constexpr uint32_t kFlagShadow = 1u;     // a shadow ray of the previous vertex is pending
constexpr uint32_t kFlagTerminal = 2u;   // no bounce ray: finalize after the shadow ray
constexpr uint32_t kShadowBit = 0x80000000u;
constexpr uint32_t kFlagShadow2 = 4u;           // a second shadow ray of the previous vertex is pending

struct WfDev {
  float4* R0;      // ray origin of waves 1..: surf = pos + n*1e-3 (primary rays start at the camera)
  float4* R1;      // primary / bounce direction
  float4* R2;      // direction (xyz) and maxT (w) of the pending shadow ray
  float4* S0;      // radiance xyz, w = RNG state bits
  float4* S1;      // throughput xyz, w = primary material bits
  float4* S2;      // pending sun contribution xyz, w = flags
  uint4* hit;      // x = t bits, y = material, z = entry axis, w = shadow occluded
  uint32_t* q0;    // ray queues (entry = path | kShadowBit for shadow rays), capacity 3P; a path's second
                   // shadow ray uses path index g + P (R0, R2 and hit hold 2P entries where it is used)
  uint32_t* q1;
  uint32_t* a0;    // active path lists, capacity P
  uint32_t* a1;
  int* ctr;        // per wave k: [4k] shadow rays (queue front), [4k+1] queue head, [4k+2] active count,
                   // [4k+3] bounce rays (queue back)
  uint32_t qcap;   // queue capacity in entries: bounce ray i of a wave sits at qcap - 1 - i
};

// Ray queues: a wave's shadow rays are appended from the front, its bounce
// rays from the back (bounce ray i at qcap - 1 - i), so a tracer warp takes
// runs of one kind -- shadow rays of neighbouring paths share the sun
// direction and much of their walks.

VRT_DI uint32_t* queue_of(const WfDev& b, int wave) { return (wave & 1) ? b.q1 : b.q0; }
VRT_DI uint32_t* active_of(const WfDev& b, int wave) { return (wave & 1) ? b.a1 : b.a0; }

// Warp-aggregated append: one atomicAdd per warp, slots in lane order.  All
// 32 lanes must call it (pred false for lanes with nothing to append).
VRT_DI uint32_t warp_append(int* counter, bool pred) {
  const unsigned mask = __ballot_sync(0xffffffffu, pred);
  if (!mask) return 0u;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(counter, __popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  return (uint32_t)base + (uint32_t)__popc(mask & ((1u << lane) - 1u));
}

VRT_DI F3 xyz(float4 v) { return f3(v.x, v.y, v.z); }

// Normal of a hit on entry axis `vax` for direction rd (same value the DDA
// returns: -vmask * sign(rd)).
VRT_DI F3 hit_normal(int vax, F3 rd) {
  const int sx = rd.x > 0.0f ? 1 : (rd.x < 0.0f ? -1 : 0);
  const int sy = rd.y > 0.0f ? 1 : (rd.y < 0.0f ? -1 : 0);
  const int sz = rd.z > 0.0f ? 1 : (rd.z < 0.0f ? -1 : 0);
  return f3(face_normal_component(vax == 0, sx), face_normal_component(vax == 1, sy),
            face_normal_component(vax == 2, sz));
}

// ---------------------------------------------------------------------------
// Two-level DDA as one resumable iteration shared by both levels
// (voxel.wgsl:73-153).  Each call performs
//   [pending step at the current level] + [test of the current cell],
// so lanes walking bricks and lanes walking voxels execute the same code.
// Transitions reproduce the nested loops:
//   brick test occupied  -> descend (entry voxel from t + 1e-4, next call
//                           tests it without stepping)
//   voxel test occupied  -> hit (voxel read, maxT check)
//   voxel step leaves the brick, or 24 voxel tests done -> brick step pending
// Steps use fma(|invRd|, scale, tMax), which equals the reference's
// tMax + |invRd|*8 (brick) and tMax + |invRd| (voxel) bit for bit because
// |invRd|*8 and |invRd|*1 are exact.
// Counters follow the oracle: outer = brick iterations entered, inner =
// voxel iterations entered, vreads = voxel words read.
// ---------------------------------------------------------------------------
enum : int { kLevelVoxel = 1, kPending = 2, kDone = 4, kHitCell = 8 };

// Register layout: tm / (cx, cy, cz) / t / ax hold the current level's state
// -- the brick level's tMaxB, brick cell, t and ax while walking bricks, the
// voxel level's tMaxV, local cell, tCur and vax while walking voxels -- so the
// step reads no level-selected operands; the brick level's tMax and cell are
// saved in tmB / (bx, by, bz) on descent and restored when the voxel walk ends
// (t and ax need no restore: the brick step that follows rewrites them).  The
// step's scale (8 or 1) and the cells per axis (BG or 8, which is also the
// stride of the test's bit index) are per-level registers, and only the
// stepped coordinate is bounds-checked (the others did not move).  The entry axis left in ax after a miss is not meaningful; every
// consumer reads it for hits only.  Against a layout with both levels' state
// and per-operand level selects: 1.61 -> 1.48 ms of trace on the 1080p frame.
struct FlatDDA {
  F3 ro, invRd;
  float maxT, tExit;
  F3 tm, tmB;
  int cx, cy, cz;               // current cell (brick, or voxel local to the brick)
  int bx, by, bz;               // brick cell while walking voxels
  int sx, sy, sz;
  float t, sc;
  int ext, ax, iter, j, state;   // ext: cells per axis of the current level (BG, or 8 in a brick)
  uint32_t bi16;                // 16 x the brick index while walking voxels (its first mask word)
  float tHit;
  uint32_t mat;

  VRT_DI bool done() const { return (state & kDone) != 0; }
  VRT_DI int hit_axis() const { return ax; }

  // Counters: brick iterations entered = iter at the end of the walk; voxel
  // iterations = the sum of j over the bricks walked (added as each voxel
  // walk ends), so the steps count nothing.
  VRT_DI void finish(const DScene& S, DCount& c) {
    tHit = -1.0f;
    mat = 0u;
    c.outer += (uint32_t)iter;
    if (state & kHitCell) {
      c.inner += (uint32_t)j;
      const uint32_t vx = (uint32_t)(bx * kBrick + cx), vy = (uint32_t)(by * kBrick + cy),
                     vz = (uint32_t)(bz * kBrick + cz);
      mat = __ldg(S.vox + (vx + vy * (uint32_t)S.N + vz * (uint32_t)(S.N * S.N)));
      c.vreads++;
      if (!(t > maxT)) tHit = t * kVoxelSize;
      else mat = 0u;
    }
  }

  VRT_DI void init(const DScene& S, F3 roW, F3 rd, float maxTW) {
    ro = roW * kInvVoxel;
    maxT = maxTW * kInvVoxel;
    const float sgx = rd.x >= 0.0f ? 1.0f : -1.0f;
    const float sgy = rd.y >= 0.0f ? 1.0f : -1.0f;
    const float sgz = rd.z >= 0.0f ? 1.0f : -1.0f;
    invRd = f3(safe_inv(sgx, rd.x), safe_inv(sgy, rd.y), safe_inv(sgz, rd.z));
    sx = rd.x > 0.0f ? 1 : (rd.x < 0.0f ? -1 : 0);
    sy = rd.y > 0.0f ? 1 : (rd.y < 0.0f ? -1 : 0);
    sz = rd.z > 0.0f ? 1 : (rd.z < 0.0f ? -1 : 0);
    const F3 stepGE = f3(rd.x >= 0.0f ? 1.0f : 0.0f, rd.y >= 0.0f ? 1.0f : 0.0f, rd.z >= 0.0f ? 1.0f : 0.0f);
    const float G = (float)S.N;
    const F3 t0 = f3(__fsub_rn(0.0f, ro.x), __fsub_rn(0.0f, ro.y), __fsub_rn(0.0f, ro.z)) * invRd;
    const F3 t1 = (f3(G, G, G) - ro) * invRd;
    const F3 tmin3 = min3(t0, t1);
    const F3 tmax3 = max3(t0, t1);
    const float tEnter = fmax_(fmax_(tmin3.x, tmin3.y), fmax_(tmin3.z, 0.0f));
    tExit = fmin_(fmin_(tmax3.x, tmax3.y), fmin_(tmax3.z, maxT));
    iter = 0;
    j = 0;
    ax = 0;
    if (tEnter > tExit) { state = kDone; return; }
    if (tmin3.x >= tmin3.y && tmin3.x >= tmin3.z) ax = 0;
    else if (tmin3.y >= tmin3.z) ax = 1;
    else ax = 2;
    t = tEnter;
    const F3 sp = ro + rd * (t + 1e-4f);
    // x / 8 as x * 0.125: the same real number, so the same rounding
    cx = iclamp_(ifloor_(sp.x * 0.125f), 0, S.BG - 1);
    cy = iclamp_(ifloor_(sp.y * 0.125f), 0, S.BG - 1);
    cz = iclamp_(ifloor_(sp.z * 0.125f), 0, S.BG - 1);
    tm = ((f3((float)cx, (float)cy, (float)cz) + stepGE) * 8.0f - ro) * invRd;
    sc = 8.0f;
    ext = S.BG;
    state = 0;   // brick level, test first
  }

  // The voxel walk of the current brick ends: brick step next.
  VRT_DI void leave_brick(const DScene& S, DCount& c) {
    c.inner += (uint32_t)j;
    cx = bx; cy = by; cz = bz;
    tm = tmB;
    sc = 8.0f;
    ext = S.BG;
    state = kPending;
  }

  // kSharedOcc: occ is the block's shared-memory copy of the occupancy bitmap;
  // otherwise it is the scene's bitmap in global memory, read through the
  // read-only path.
  template <bool kSharedOcc>
  VRT_DI void step(const DScene& S, const uint32_t* occ, F3 rd, DCount& c) {
    const bool lv = (state & kLevelVoxel) != 0;
    if (state & kPending) {
      const bool px = tm.x <= tm.y && tm.x <= tm.z;
      const bool py = !px && tm.y <= tm.z;
      const float tn = px ? tm.x : (py ? tm.y : tm.z);
      const float ia = fabsf(px ? invRd.x : (py ? invRd.y : invRd.z));
      const float nv = __fmaf_rn(ia, sc, tn);
      int cn;
      if (px) { tm.x = nv; cx += sx; cn = cx; }
      else if (py) { tm.y = nv; cy += sy; cn = cy; }
      else { tm.z = nv; cz += sz; cn = cz; }
      t = tn;
      ax = px ? 0 : (py ? 1 : 2);
      if ((unsigned)cn >= (unsigned)ext) {   // left the brick (voxel walk) or the grid (brick walk)
        if (lv) leave_brick(S, c);
        else state = kDone;
        return;
      }
      state &= ~kPending;
    }
    if (lv) {
      if (j >= 3 * kBrick) { leave_brick(S, c); return; }   // voxel loop exhausted
      j++;
    } else {
      if (iter >= 3 * S.BG + 2 || t > tExit) { state = kDone; return; }
      iter++;
    }
    // the cell's bit index: the brick index bx + BG (by + BG bz) at brick level,
    // the mask bit lx + 8 (ly + 8 lz) in a brick
    const uint32_t idx = (uint32_t)cx + (uint32_t)ext * ((uint32_t)cy + (uint32_t)ext * (uint32_t)cz);
    // two typed loads (the bitmap may be in shared memory, the masks are in
    // global memory) rather than one load through a selected pointer
    const uint32_t word = lv ? __ldg(S.masks + (size_t)bi16 + (idx >> 5))
                             : (kSharedOcc ? occ[idx >> 5] : __ldg(occ + (idx >> 5)));
    if (!((word >> (idx & 31u)) & 1u)) {
      state |= kPending;
      return;
    }
    if (lv) {
      state = kDone | kHitCell;   // finish() reads the voxel
      return;
    }
    // descend into the occupied brick (voxel.wgsl:104-109); t and ax carry over as tCur and vax
    bx = cx; by = cy; bz = cz;
    bi16 = idx * 16u;
    tmB = tm;
    const int mnx = bx * kBrick, mny = by * kBrick, mnz = bz * kBrick;
    const F3 p = ro + rd * (t + 1e-4f);
    const int vx = iclamp_(ifloor_(p.x), mnx, mnx + 7);
    const int vy = iclamp_(ifloor_(p.y), mny, mny + 7);
    const int vz = iclamp_(ifloor_(p.z), mnz, mnz + 7);
    const F3 stepGE = f3(rd.x >= 0.0f ? 1.0f : 0.0f, rd.y >= 0.0f ? 1.0f : 0.0f, rd.z >= 0.0f ? 1.0f : 0.0f);
    tm = ((f3((float)vx, (float)vy, (float)vz) + stepGE) - ro) * invRd;
    cx = vx - mnx; cy = vy - mny; cz = vz - mnz;
    j = 0;
    sc = 1.0f;
    ext = kBrick;
    state = kLevelVoxel;
  }
};

// ---------------------------------------------------------------------------
// Job policies.  A "job" is one view (session) rendered in a wave: uniforms,
// scene, size and output buffers.  Path state is indexed by a global pixel id
// g (jobs are laid out back to back); outputs by the job-local pixel id.
// ---------------------------------------------------------------------------
struct JobOut {
  uint2* rad16;     // rgba16f demodulated radiance
  float4* rad32;    // optional fp32 copy
  uint32_t* alb8;   // rgba8 sqrt albedo
  float4* gbuf;     // rgba32f normal + distance of this frame
};

// One session: everything in kernel parameters, occupancy bitmap staged in
// shared memory by the tracer.
struct SingleJob {
  Uni u;
  DScene S;
  JobOut out;
  CacheDev cc;             // radiance cache (cc.on == 0: plain path)
  float fclamp;
  int W, H;
  __host__ __device__ bool any_cache() const { return cc.on != 0; }
  VRT_DI const CacheDev& cache(int) const { return cc; }
  VRT_DI int job_of(uint32_t) const { return 0; }
  VRT_DI int job_of_cached(uint32_t, int&, uint32_t&, uint32_t&) const { return 0; }
  VRT_DI const Uni& uni(int) const { return u; }
  VRT_DI DScene scene(int) const { return S; }
  VRT_DI JobOut outs(int) const { return out; }
  VRT_DI float clamp(int) const { return fclamp; }
  VRT_DI int width(int) const { return W; }
  VRT_DI int height(int) const { return H; }
  VRT_DI uint32_t first(int) const { return 0u; }
};

// Device job table entry of a batch (one per session in the batch).
struct JobDev {
  Uni u;
  DScene S;
  JobOut out;
  int W, H;
  uint32_t first;          // first global pixel of the job
  float fclamp;
  // image passes of the frame
  const void* acc_prev;    // history read by temporal (rgba16f / rgba32f)
  void* acc_cur;           // history written by temporal
  const float4* gbuf_prev;
  uint2* den0;             // a-trous ping-pong (dA, dB)
  uint2* den1;
  uint32_t* ldr;
  int acc_f32;
  int pad[3];
  CacheDev cache;          // radiance cache of the job's session (cache.on == 0: plain path)
};

// Many sessions: job table in device memory, job found by binary search on
// the sorted first-pixel array.
struct MultiJob {
  const JobDev* jobs;
  const uint32_t* firsts;  // n entries, ascending
  int n;
  int cache_jobs;          // jobs with the cache on
  __host__ __device__ bool any_cache() const { return cache_jobs != 0; }
  VRT_DI const CacheDev& cache(int j) const { return jobs[j].cache; }
  VRT_DI int job_of(uint32_t g) const {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(firsts + mid) <= g) lo = mid;
      else hi = mid - 1;
    }
    return lo;
  }
  // job_of with the caller's last answer (job jc for pixels [lo, hi), lo <= hi; lo == hi: none)
  // tried first
  VRT_DI int job_of_cached(uint32_t g, int& jc, uint32_t& lo, uint32_t& hi) const {
    if (g - lo < hi - lo) return jc;
    jc = job_of(g);
    lo = __ldg(firsts + jc);
    hi = jc + 1 < n ? __ldg(firsts + jc + 1) : 0xffffffffu;
    return jc;
  }
  VRT_DI const Uni& uni(int j) const { return jobs[j].u; }
  VRT_DI DScene scene(int j) const { return jobs[j].S; }
  VRT_DI JobOut outs(int j) const { return jobs[j].out; }
  VRT_DI float clamp(int j) const { return jobs[j].fclamp; }
  VRT_DI int width(int j) const { return jobs[j].W; }
  VRT_DI int height(int j) const { return jobs[j].H; }
  VRT_DI uint32_t first(int j) const { return jobs[j].first; }
};

// ---------------------------------------------------------------------------
// radiance cache hooks (single session).  With the cache on, 1/16 of the
// pixels (one position of every 4x4 block, rotating per frame) trace full
// training paths of `train_bounces` bounces and record their first
// `rec_vertices` vertices; every other path ends at its first bounce hit
// (vertex 1): its emission is picked up there and the reflected radiance at
// that point is queried from the network after the waves.
// ---------------------------------------------------------------------------
enum : int { kRolePlain = 0, kRoleTrain = 1, kRoleQuery = 2 };

VRT_DI int cache_role(const CacheDev& c, uint32_t lp, int W) {
  if (!c.on) return kRolePlain;
  const uint32_t x = lp % (uint32_t)W, y = lp / (uint32_t)W;
  return ((x & 3u) == (c.phase & 3u) && (y & 3u) == (c.phase >> 2)) ? kRoleTrain : kRoleQuery;
}

VRT_DI uint32_t train_index(const CacheDev& c, uint32_t lp, int W) {
  const uint32_t x = lp % (uint32_t)W, y = lp / (uint32_t)W;
  return (y >> 2) * (uint32_t)c.TW + (x >> 2);
}

// Record slot of vertex k of a training path (nullptr: nothing to record).
VRT_DI float4* rec_slot(const CacheDev& c, int role, uint32_t lp, int W, uint32_t k) {
  if (role != kRoleTrain || (int)k >= c.rec_vertices) return nullptr;
  const uint32_t ti = train_index(c, lp, W);
  c.rec_n[ti] = (int)k + 1;
  return c.rec + ((size_t)ti * kCacheMaxRec + k) * 4;
}

VRT_DI float cache_target(float rfin, float rk, float tpk, float clampv) {
  float v = tpk > 1e-6f ? (rfin - rk) / tpk : 0.0f;
  v = fmax_(v, 0.0f);
  if (clampv > 0.0f) v = fmin_(v, clampv);
  return v;
}

// The counter that every thread of the block with want set appends to, when
// it is one counter (a single job's), or null when no thread appends; false
// when the threads append to different counters (several jobs of a batch in
// one block).  All threads of the block call it.
VRT_DI bool block_common_counter(int* mine, bool want, int*& common) {
  __shared__ int* s_c;
  if (threadIdx.x == 0) s_c = nullptr;
  __syncthreads();
  if (want) s_c = mine;   // any of the writers
  __syncthreads();
  common = s_c;
  return __syncthreads_and(!want || mine == common) != 0;
}

// One atomicAdd on ctr for the n entries of every thread of the block; the
// thread's first slot (its n slots are consecutive).  All threads call it.
VRT_DI uint32_t block_append1(int* ctr, int n) {
  __shared__ int s_cnt[8];
  __shared__ int s_base;
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int incl = n;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(full, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) s_cnt[w] = incl;
  __syncthreads();
  if (threadIdx.x == 0) {
    int tot = 0;
    const int nw = (int)(blockDim.x >> 5);   // blocks of up to 256 threads
    for (int k = 0; k < nw; k++) {
      const int v = s_cnt[k];
      s_cnt[k] = tot;
      tot += v;
    }
    s_base = tot ? atomicAdd(ctr, tot) : 0;
  }
  __syncthreads();
  const uint32_t slot = (uint32_t)(s_base + s_cnt[w] + incl - n);
  __syncthreads();   // s_cnt / s_base are rewritten by the block's next call
  return slot;
}

// Writes the nrec training samples of training path ti from sample slot
// `slot` on (slots at or past the buffer's capacity are dropped).
VRT_DI void cache_write_samples(const CacheDev& c, uint32_t ti, int nrec, int slot, F3 rfin) {
  for (int k = 0; k < nrec && slot < c.cand_cap; k++, slot++) {
    const float4* r = c.rec + ((size_t)ti * kCacheMaxRec + k) * 4;
    const float4 r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3];
    float* q = c.cand_q9 + (size_t)slot * 9;
    q[0] = r0.x; q[1] = r0.y; q[2] = r0.z;
    q[3] = r1.x; q[4] = r1.y; q[5] = r1.z;
    q[6] = r2.x; q[7] = r2.y; q[8] = r2.z;
    float* y = c.cand_y3 + (size_t)slot * 3;
    y[0] = cache_target(rfin.x, r0.w, r3.x, c.tclamp);
    y[1] = cache_target(rfin.y, r1.w, r3.y, c.tclamp);
    y[2] = cache_target(rfin.z, r2.w, r3.z, c.tclamp);
  }
}

// Training samples of finished training paths: for each recorded vertex k,
// the radiance the path gathered after vertex k's emission pickup per unit
// of the throughput that reached it, (R_final - R_k) / tp_k -- the reflected
// radiance estimate at x_k.  All threads of the block call it: one atomic per
// block when its samples go to one job's buffer; otherwise per warp, or per
// lane when a warp's lanes belong to different jobs.
VRT_DI void cache_emit_samples(const CacheDev& c, bool fin, uint32_t ti, F3 rfin) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int nrec = fin ? c.rec_n[ti] : 0;
  int* common = nullptr;
  int slot = 0;
  if (block_common_counter(c.cand_count, nrec > 0, common)) {
    if (!common) return;
    slot = (int)block_append1(common, nrec);
  } else {
    const unsigned any = __ballot_sync(full, nrec > 0);
    if (!any) return;
    const unsigned long long key = (unsigned long long)c.cand_count;
    const unsigned grp = __match_any_sync(full, nrec > 0 ? key : 0ull) & any;
    const bool one_job = nrec > 0 ? grp == any : true;
    if (__all_sync(full, one_job)) {
      int incl = nrec;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(full, incl, o);
        if (lane >= o) incl += v;
      }
      const int total = __shfl_sync(full, incl, 31);
      const int leader = __ffs(any) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(c.cand_count, total);
      base = __shfl_sync(full, base, leader);
      slot = base + incl - nrec;
    } else if (nrec > 0) {
      slot = atomicAdd(c.cand_count, nrec);
    }
  }
  cache_write_samples(c, ti, nrec, slot, rfin);
}

// Appends a cache query of path g at its vertex 1.  All threads of the block
// call it; one atomic per block when its queries go to one job's buffer.
VRT_DI void cache_emit_query(const CacheDev& c, bool q, uint32_t g, F3 pos, F3 n, F3 alb) {
  const unsigned full = 0xffffffffu;
  int* common = nullptr;
  uint32_t slot = 0u;
  if (block_common_counter(c.qcount, q, common)) {
    if (!common) return;
    slot = block_append1(common, q ? 1 : 0);
  } else {
    const unsigned any = __ballot_sync(full, q);
    if (!any) return;
    const unsigned grp = __match_any_sync(full, q ? (unsigned long long)c.qcount : 0ull) & any;
    if (__all_sync(full, q ? grp == any : true)) slot = warp_append(c.qcount, q);
    else slot = q ? (uint32_t)atomicAdd(c.qcount, 1) : 0u;
  }
  if (q) {
    float* d = c.qbuf + (size_t)slot * 9;
    d[0] = pos.x; d[1] = pos.y; d[2] = pos.z;
    d[3] = n.x; d[4] = n.y; d[5] = n.z;
    d[6] = alb.x; d[7] = alb.y; d[8] = alb.z;
    c.qpix[slot] = g;
  }
}

// ---------------------------------------------------------------------------
// shading
// ---------------------------------------------------------------------------
VRT_DI void finalize(const JobOut& out, uint32_t lp, F3 radiance, uint32_t mat1bits, float fclamp) {
  const Mat mat1 = unpack_material(mat1bits);
  if (!(fclamp <= 0.0f)) radiance = min3(radiance, f3(fclamp, fclamp, fclamp));
  const F3 den = max3(mat1.albedo, f3(1e-3f, 1e-3f, 1e-3f));
  const float4 rad = make_float4(radiance.x / den.x, radiance.y / den.y, radiance.z / den.z, 1.0f);
  out.rad16[lp] = pack_h4(rad.x, rad.y, rad.z, rad.w);
  if (out.rad32) out.rad32[lp] = rad;
}

// Vertex k of a path (pathtrace.wgsl:297-320 loop body up to the trace call),
// path state at index g.  Returns whether the path stays active.
// kmax: the path's last vertex (the uniforms' bounce count for plain paths).
// rec (may be null): training record of this vertex, written after the
// emission pickup.
VRT_DI bool shade_vertex(const Uni& u, const WfDev& b, uint32_t g, uint32_t k, F3 pos, F3 n, Mat mat,
                         F3& radiance, F3& tp, uint32_t& rng, uint32_t mat1bits, bool& want_shadow,
                         bool& want_bounce, uint32_t kmax, float4* rec) {
  if (mat.emissive > 0.0f) radiance = radiance + (tp * mat.albedo) * (mat.emissive * kEmissiveScale);
  if (rec) {
    rec[0] = make_float4(pos.x, pos.y, pos.z, radiance.x);
    rec[1] = make_float4(n.x, n.y, n.z, radiance.y);
    rec[2] = make_float4(mat.albedo.x, mat.albedo.y, mat.albedo.z, radiance.z);
    rec[3] = make_float4(tp.x, tp.y, tp.z, 0.0f);
  }
  const F3 surf = pos + n * 1e-3f;
  const F3 l = sample_sun_dir(u, rng);
  const float ndl = dot3(n, l);
  uint32_t flags = 0u;
  F3 sunc = f3(0.0f, 0.0f, 0.0f);
  want_shadow = ndl > 0.0f && l.y > 0.0f;
  if (want_shadow) {
    const F3 sunRad = f3(u.sunRadiance[0], u.sunRadiance[1], u.sunRadiance[2]);
    sunc = (((tp * mat.albedo) * kInvPi) * ndl) * sunRad;
    flags |= kFlagShadow;
    b.R2[g] = make_float4(l.x, l.y, l.z, 1e4f);
  }
  want_bounce = false;
  if (k == kmax) {
    flags |= kFlagTerminal;
  } else {
    const F3 rd = cosine_hemisphere(n, rng);
    tp = tp * mat.albedo;
    bool alive = true;
    if (k >= 2u) {
      const float pr = clamp_(fmax_(tp.x, fmax_(tp.y, tp.z)), 0.05f, 0.95f);
      if (rand_(rng) > pr) alive = false;
      else tp = f3(tp.x / pr, tp.y / pr, tp.z / pr);
    }
    if (alive) {
      want_bounce = true;
      b.R1[g] = make_float4(rd.x, rd.y, rd.z, 0.0f);
    } else {
      flags |= kFlagTerminal;
    }
  }
  b.R0[g] = make_float4(surf.x, surf.y, surf.z, 0.0f);
  b.S0[g] = make_float4(radiance.x, radiance.y, radiance.z, __uint_as_float(rng));
  b.S1[g] = make_float4(tp.x, tp.y, tp.z, __uint_as_float(mat1bits));
  b.S2[g] = make_float4(sunc.x, sunc.y, sunc.z, __uint_as_float(flags));
  return want_shadow || want_bounce;
}

// Block-aggregated appends: each thread of a block of 256 adds nf entries to
// the list counted by c_front, nb to the list counted by c_back and, if act,
// one to the list counted by c_act; one atomicAdd per counter per block, since
// every block of the grid appends to the same counters.  Returns the thread's
// first slot in each (its nf / nb slots are consecutive).  All threads of the
// block call it (block-uniform control flow).  Entries of a block are in
// thread order; a path's results do not depend on the order of the queues.
VRT_DI void block_append(int* c_front, int* c_back, int* c_act, int nf, int nb, bool act, uint32_t& fslot,
                         uint32_t& bslot, uint32_t& aslot) {
  __shared__ int s_cnt[3][8];
  __shared__ int s_base[3];
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int incf = nf, incb = nb;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int vf = __shfl_up_sync(full, incf, o);
    const int vb = __shfl_up_sync(full, incb, o);
    if (lane >= o) { incf += vf; incb += vb; }
  }
  const unsigned ma = __ballot_sync(full, act);
  if (lane == 31) { s_cnt[0][w] = incf; s_cnt[1][w] = incb; }
  if (lane == 0) s_cnt[2][w] = __popc(ma);
  __syncthreads();
  if (threadIdx.x < 3) {   // thread 0: front, 1: back, 2: list
    int tot = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const int v = s_cnt[threadIdx.x][k];
      s_cnt[threadIdx.x][k] = tot;
      tot += v;
    }
    int* c = threadIdx.x == 0 ? c_front : (threadIdx.x == 1 ? c_back : c_act);
    s_base[threadIdx.x] = tot ? atomicAdd(c, tot) : 0;
  }
  __syncthreads();
  fslot = (uint32_t)(s_base[0] + s_cnt[0][w] + incf - nf);
  bslot = (uint32_t)(s_base[1] + s_cnt[1][w] + incb - nb);
  aslot = (uint32_t)(s_base[2] + s_cnt[2][w]) + (uint32_t)__popc(ma & ((1u << lane) - 1u));
  __syncthreads();   // s_cnt / s_base are rewritten by the block's next call
}

// Appends the new rays (shadow ray of path g, its bounce ray) and the active
// path of wave `next`.  Block-uniform, see block_append.
VRT_DI void emit_block(const WfDev& b, int next, uint32_t g, bool shadow, bool bounce, bool keep) {
  uint32_t fs, bs, as;
  int* c = b.ctr + 4 * next;
  block_append(c, c + 3, c + 2, (int)shadow, (int)bounce, keep, fs, bs, as);
  uint32_t* q = queue_of(b, next);
  if (shadow) q[fs] = g | kShadowBit;
  if (bounce) q[b.qcap - 1u - bs] = g;
  if (keep) active_of(b, next)[as] = g;
}

// emit_block() with a second shadow ray of the path, traced as path g + P.
VRT_DI void emit2_block(const WfDev& b, int next, uint32_t g, uint32_t P, bool shadow, bool shadow2, bool bounce,
                        bool keep) {
  uint32_t fs, bs, as;
  int* c = b.ctr + 4 * next;
  block_append(c, c + 3, c + 2, (int)shadow2 + (int)shadow, (int)bounce, keep, fs, bs, as);
  uint32_t* q = queue_of(b, next);
  if (shadow2) q[fs++] = (g + P) | kShadowBit;
  if (shadow) q[fs] = g | kShadowBit;
  if (bounce) q[b.qcap - 1u - bs] = g;
  if (keep) active_of(b, next)[as] = g;
}

// ---------------------------------------------------------------------------
// kernels (templated on the job policy)
// ---------------------------------------------------------------------------
// generate: RNG stream, jitter, camera ray (pathtrace.wgsl:249-263)
template <class J>
__global__ void __launch_bounds__(256) k_wf_generate(J jobs, uint32_t P, WfDev b) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= P) return;
  const int j = jobs.job_of(g);
  const Uni& u = jobs.uni(j);
  const int W = jobs.width(j), H = jobs.height(j);
  const uint32_t lp = g - jobs.first(j);
  const uint32_t gx = lp % (uint32_t)W, gy = lp / (uint32_t)W;
  uint32_t rng = init_rng(gx, gy, u.params0[0]);
  const float jx = rand_(rng) - 0.5f;
  const float jy = rand_(rng) - 0.5f;
  const float uvx = (((float)gx + 0.5f) + jx) / (float)W;
  const float uvy = (((float)gy + 0.5f) + jy) / (float)H;
  const F3 rd = camera_ray(u, uvx, uvy);
  b.R1[g] = make_float4(rd.x, rd.y, rd.z, 0.0f);
  b.S0[g] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(rng));
}

// Persistent queue tracer.  kSmem: stage the (single) scene's occupancy
// bitmap in shared memory.  kSteps DDA iterations per pass of the warp
// bookkeeping (idle-lane ballot, refill, drain check).  kVarMaxT: shadow rays
// carry their own maxT in R2.w (otherwise every ray ends at 1e4 m, the plain
// path's bound, and the tracer keeps its register budget).
template <class J, bool kSmem, int kSteps, int kMinB, bool kVarMaxT, int kUnroll = kSteps>
__global__ void __launch_bounds__(256, kMinB) k_wf_trace(J jobs, WfDev b, int wave, int implicit_n,
                                                              int refill_min, unsigned long long* stats) {
  extern __shared__ uint32_t s_occ[];
  if (kSmem) {
    const DScene S0 = jobs.scene(0);
    const int nwords = (S0.BG * S0.BG * S0.BG + 31) >> 5;
    for (int i = threadIdx.x; i < nwords; i += blockDim.x) s_occ[i] = __ldg(S0.bits + i);
    __syncthreads();
  }
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int nf = implicit_n > 0 ? 0 : b.ctr[4 * wave];   // shadow rays at the queue's front
  const int n = implicit_n > 0 ? implicit_n : nf + b.ctr[4 * wave + 3];
  int* head = b.ctr + 4 * wave + 1;
  const uint32_t* queue = queue_of(b, wave);
  DCount c{0u, 0u, 0u, 0u};
  FlatDDA d;
  DScene S = jobs.scene(0);
  F3 rd = f3(0.0f, 0.0f, 0.0f);
  uint32_t entry = 0u;
  int jc = 0;                     // the lane's last job and its pixel range [jlo, jhi) (empty: none yet)
  uint32_t jlo = 0u, jhi = 0u;
  uint32_t passes = 0u;   // passes of the step loop with a lane walking (warp-uniform)
  bool active = false, drained = false;
  while (true) {
    const unsigned idle = __ballot_sync(full, !active);
    const int nidle = __popc(idle);
    if (!drained && (nidle >= refill_min || nidle == 32)) {
      int base = 0;
      if (lane == 0) base = atomicAdd(head, nidle);
      base = __shfl_sync(full, base, 0);
      if (base + nidle >= n) drained = true;
      if (!active) {
        const int slot = base + __popc(idle & ((1u << lane) - 1u));
        if (slot < n) {
          entry = implicit_n > 0 ? (uint32_t)slot
                                 : (slot < nf ? queue[slot] : queue[b.qcap - 1u - (uint32_t)(slot - nf)]);
          const uint32_t g = entry & ~kShadowBit;
          const int j = jobs.job_of_cached(g, jc, jlo, jhi);   // consecutive rays mostly share a job
          S = jobs.scene(j);
          // primary rays start at the camera: its position comes from the job's
          // uniforms (k_wf_generate writes no R0, so no wave-0 shading kernel
          // may read R0 either); later waves read the origin their shading stored
          F3 ro;
          if (implicit_n > 0) {
            const Uni& uj = jobs.uni(j);
            ro = f3(uj.camPos[0], uj.camPos[1], uj.camPos[2]);
          } else {
            ro = xyz(b.R0[g]);
          }
          if (kVarMaxT) {
            float maxT = 1e4f;   // bounce rays; shadow rays carry theirs in R2.w
            if (entry & kShadowBit) {
              const float4 r2 = b.R2[g];
              rd = xyz(r2);
              maxT = r2.w;
            } else {
              rd = xyz(b.R1[g]);
            }
            d.init(S, ro, rd, maxT);
          } else {
            rd = (entry & kShadowBit) ? xyz(b.R2[g]) : xyz(b.R1[g]);
            d.init(S, ro, rd, 1e4f);
          }
          c.rays++;
          active = true;
        }
      }
    }
    if (!__any_sync(full, active)) {
      if (drained) break;
      continue;
    }
    passes++;
    if (active) {
#pragma unroll kUnroll
      for (int k = 0; k < kSteps; k++)
        if (!d.done()) d.step<kSmem>(S, kSmem ? s_occ : S.bits, rd, c);
      if (d.done()) {
        d.finish(S, c);
        const uint32_t g = entry & ~kShadowBit;
        uint32_t* h = reinterpret_cast<uint32_t*>(b.hit + g);
        if (entry & kShadowBit) {
          h[3] = d.tHit >= 0.0f ? 1u : 0u;
        } else {
          *reinterpret_cast<uint2*>(h) = make_uint2(__float_as_uint(d.tHit), d.mat);
          h[2] = (uint32_t)d.hit_axis();
        }
        active = false;
      }
    }
  }
  if (stats) {
    block_flush_stats(stats, c, 0u);   // kStatRays..kStatVReads
    block_flush_one(stats + kStatTraceSlots, lane == 0 ? passes * (uint32_t)(32 * kSteps) : 0u);
  }
}

// shade(0): primary hits over all pixels.  The shading kernels stream the path
// state and run at 5 blocks per SM (48 registers): 2.034 -> 2.019 ms per
// 1080p frame against 4 (55-64 registers); 6 blocks (40 registers) spill
// and gain nothing further.
template <class J>
__global__ void __launch_bounds__(256, 5) k_wf_shade_primary(J jobs, uint32_t P, WfDev b, unsigned long long* stats) {
  const bool any_cache = jobs.any_cache();
  const CacheDev* ccp = nullptr;
  const uint32_t stride = gridDim.x * blockDim.x;
  if (stats && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(stats + kStatPixels, (unsigned long long)P);
  for (uint32_t base = blockIdx.x * blockDim.x; base < P; base += stride) {
    const uint32_t g = base + threadIdx.x;
    bool shadow = false, bounce = false, keep = false;
    bool fin_train = false;
    uint32_t ti = 0u;
    F3 rfin = f3(0.0f, 0.0f, 0.0f);
    if (g < P) {
      const int j = jobs.job_of(g);
      const Uni& u = jobs.uni(j);
      const JobOut out = jobs.outs(j);
      const uint32_t lp = g - jobs.first(j);
      const uint4 h = b.hit[g];
      const F3 rd = xyz(b.R1[g]);
      const float s0w = b.S0[g].w;   // RNG state, loaded with the hit rather than after the sky test
      const float t = __uint_as_float(h.x);
      if (t < 0.0f) {
        const F3 sky = sky_color(u, rd, true);
        out.rad16[lp] = pack_h4(sky.x, sky.y, sky.z, 1.0f);
        if (out.rad32) out.rad32[lp] = make_float4(sky.x, sky.y, sky.z, 1.0f);
        out.alb8[lp] = 0xffffffffu;
        out.gbuf[lp] = make_float4(-rd.x, -rd.y, -rd.z, -1.0f);
      } else {
        const Mat mat1 = unpack_material(h.y);
        const F3 ro = f3(u.camPos[0], u.camPos[1], u.camPos[2]);
        const F3 x1 = ro + rd * t;
        const F3 n1 = hit_normal((int)h.z, rd);
        out.alb8[lp] = unorm8_(__fsqrt_rn(mat1.albedo.x)) | (unorm8_(__fsqrt_rn(mat1.albedo.y)) << 8) |
                       (unorm8_(__fsqrt_rn(mat1.albedo.z)) << 16) | (255u << 24);
        out.gbuf[lp] = make_float4(n1.x, n1.y, n1.z, t);
        uint32_t rng = __float_as_uint(s0w);
        F3 radiance = f3(0.0f, 0.0f, 0.0f), tp = f3(1.0f, 1.0f, 1.0f);
        const int W = jobs.width(j);
        const CacheDev& cc = jobs.cache(j);
        ccp = &cc;
        const int role = cache_role(cc, lp, W);
        const uint32_t kmax = role == kRolePlain ? u.params0[1] : (role == kRoleTrain ? cc.train_bounces : 1u);
        keep = shade_vertex(u, b, g, 0u, x1, n1, mat1, radiance, tp, rng, h.y, shadow, bounce, kmax,
                            rec_slot(cc, role, lp, W, 0u));
        if (!keep) {
          finalize(out, lp, radiance, h.y, jobs.clamp(j));
          if (role == kRoleTrain) { fin_train = true; ti = train_index(cc, lp, W); rfin = radiance; }
        }
      }
    }
    emit_block(b, 1, g, shadow, bounce, keep);
    if (any_cache) cache_emit_samples(fin_train ? *ccp : jobs.cache(0), fin_train, ti, rfin);
  }
}

// shade(k), k >= 1: resolve vertex k-1's shadow ray, then the bounce hit.
template <class J>
__global__ void __launch_bounds__(256, 5) k_wf_shade(J jobs, WfDev b, int wave) {
  const bool any_cache = jobs.any_cache();
  const int n = b.ctr[4 * wave + 2];
  const uint32_t* list = active_of(b, wave);
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
    const int i = base + threadIdx.x;
    bool shadow = false, bounce = false, keep = false;
    bool fin_train = false, query = false;
    uint32_t ti = 0u;
    F3 rfin = f3(0.0f, 0.0f, 0.0f), qpos = rfin, qn = rfin, qalb = rfin;
    uint32_t g = 0u;
    int jc = 0;
    if (i < n) {
      g = list[i];
      const int j = jobs.job_of(g);
      jc = j;
      const uint32_t lp = g - jobs.first(j);
      const int W = jobs.width(j);
      const CacheDev& cc = jobs.cache(j);
      const int role = cache_role(cc, lp, W);
      const float4 s0 = b.S0[g];
      const float4 s1 = b.S1[g];
      const float4 s2 = b.S2[g];
      const uint4 h = b.hit[g];
      // loaded with the state above rather than after the terminal check, so a
      // path's reads are one round trip instead of two
      const float4 r1 = b.R1[g];
      const float4 r0 = b.R0[g];
      F3 radiance = xyz(s0);
      F3 tp = xyz(s1);
      uint32_t rng = __float_as_uint(s0.w);
      const uint32_t mat1bits = __float_as_uint(s1.w);
      const uint32_t flags = __float_as_uint(s2.w);
      if ((flags & kFlagShadow) && h.w == 0u) radiance = radiance + xyz(s2);
      bool done = (flags & kFlagTerminal) != 0u;
      if (!done) {
        const Uni& u = jobs.uni(j);
        const F3 rd = xyz(r1);
        const F3 surf = xyz(r0);
        const float t = __uint_as_float(h.x);
        if (t < 0.0f) {
          radiance = radiance + tp * sky_color(u, rd, false);
          done = true;
        } else {
          const F3 pos = surf + rd * t;
          const F3 nrm = hit_normal((int)h.z, rd);
          const Mat mat = unpack_material(h.y);
          if (role == kRoleQuery) {
            // path ends at vertex 1: emission here, reflected radiance from the cache
            if (mat.emissive > 0.0f) radiance = radiance + (tp * mat.albedo) * (mat.emissive * kEmissiveScale);
            b.S0[g] = make_float4(radiance.x, radiance.y, radiance.z, __uint_as_float(rng));
            query = true;
            qpos = pos; qn = nrm; qalb = mat.albedo;
          } else {
            const uint32_t kmax = role == kRolePlain ? u.params0[1] : cc.train_bounces;
            keep = shade_vertex(u, b, g, (uint32_t)wave, pos, nrm, mat, radiance, tp, rng, mat1bits, shadow, bounce,
                                kmax, rec_slot(cc, role, lp, W, (uint32_t)wave));
            done = !keep;
          }
        }
      }
      if (done) {
        finalize(jobs.outs(j), lp, radiance, mat1bits, jobs.clamp(j));
        if (role == kRoleTrain) { fin_train = true; ti = train_index(cc, lp, W); rfin = radiance; }
      }
    }
    emit_block(b, wave + 1, g, shadow, bounce, keep);
    if (any_cache) {
      const CacheDev& cc = jobs.cache(jc);
      cache_emit_query(cc, query, g, qpos, qn, qalb);
      cache_emit_samples(cc, fin_train, ti, rfin);
    }
  }
}

// The tail of a frame whose remaining paths are few -- the radiance cache's
// training paths after every other path ended at its first bounce: one
// thread finishes each path of wave `wave`'s active list, tracing its pending
// shadow and bounce rays with the same resumable DDA the queue tracer runs
// (FlatDDA: same walk, hits and counters) and shading each vertex as
// k_wf_shade does, until the path ends.  The per-wave form would launch a
// trace and a shade kernel for every remaining bounce, each waiting for the
// slowest of ~10^5 latency-bound walks; here each path runs its own
// sequence.  Same per-path arithmetic and RNG draws, so the same image.
// (A per-lane state machine -- lanes stepping their walks together, each
// shading when its own ray ends and then taking the next path -- ran 447
// against 305 us per 1080p cache frame: some lane shades in nearly every pass,
// so the warp runs the shading code far more often than once per bounce.)
template <class J, bool kSmem>
__global__ void __launch_bounds__(128, 6) k_wf_tail(J jobs, WfDev b, int wave, unsigned long long* stats) {
  extern __shared__ uint32_t s_occ[];
  if (kSmem) {
    const DScene S0 = jobs.scene(0);
    const int nwords = (S0.BG * S0.BG * S0.BG + 31) >> 5;
    for (int i = threadIdx.x; i < nwords; i += blockDim.x) s_occ[i] = __ldg(S0.bits + i);
    __syncthreads();
  }
  const bool any_cache = jobs.any_cache();
  const int n = b.ctr[4 * wave + 2];
  const uint32_t* list = active_of(b, wave);
  const int stride = gridDim.x * blockDim.x;
  DCount c{0u, 0u, 0u, 0u};
  for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
    const int i = base + threadIdx.x;
    bool fin_train = false;
    uint32_t ti = 0u;
    F3 rfin = f3(0.0f, 0.0f, 0.0f);
    int jc = 0;
    if (i < n) {
      const uint32_t g = list[i];
      const int j = jobs.job_of(g);
      jc = j;
      const uint32_t lp = g - jobs.first(j);
      const int W = jobs.width(j);
      const CacheDev& cc = jobs.cache(j);
      const int role = cache_role(cc, lp, W);
      const Uni& u = jobs.uni(j);
      const DScene S = jobs.scene(j);
      const uint32_t* occ = kSmem ? s_occ : S.bits;
      for (int w = wave;; w++) {
        const float4 s0 = b.S0[g];
        const float4 s1 = b.S1[g];
        const float4 s2 = b.S2[g];
        const float4 r0 = b.R0[g];
        const float4 r1 = b.R1[g];
        F3 radiance = xyz(s0);
        F3 tp = xyz(s1);
        uint32_t rng = __float_as_uint(s0.w);
        const uint32_t mat1bits = __float_as_uint(s1.w);
        const uint32_t flags = __float_as_uint(s2.w);
        const F3 surf = xyz(r0);
        if (flags & kFlagShadow) {   // the previous vertex's sun shadow ray
          const float4 r2 = b.R2[g];
          const F3 ld = xyz(r2);
          FlatDDA d;
          d.init(S, surf, ld, r2.w);
          c.rays++;
          while (!d.done()) d.step<kSmem>(S, occ, ld, c);
          d.finish(S, c);
          if (!(d.tHit >= 0.0f)) radiance = radiance + xyz(s2);
        }
        bool done = (flags & kFlagTerminal) != 0u;
        if (!done) {
          const F3 rd = xyz(r1);
          FlatDDA d;
          d.init(S, surf, rd, 1e4f);
          c.rays++;
          while (!d.done()) d.step<kSmem>(S, occ, rd, c);
          d.finish(S, c);
          if (d.tHit < 0.0f) {
            radiance = radiance + tp * sky_color(u, rd, false);
            done = true;
          } else {
            const F3 pos = surf + rd * d.tHit;
            const F3 nrm = hit_normal(d.hit_axis(), rd);
            const Mat mat = unpack_material(d.mat);
            const uint32_t kmax = role == kRolePlain ? u.params0[1] : cc.train_bounces;
            bool shadow = false, bounce = false;
            done = !shade_vertex(u, b, g, (uint32_t)w, pos, nrm, mat, radiance, tp, rng, mat1bits, shadow, bounce,
                                 kmax, rec_slot(cc, role, lp, W, (uint32_t)w));
          }
        }
        if (done) {
          finalize(jobs.outs(j), lp, radiance, mat1bits, jobs.clamp(j));
          if (role == kRoleTrain) { fin_train = true; ti = train_index(cc, lp, W); rfin = radiance; }
          break;
        }
      }
    }
    if (any_cache) cache_emit_samples(jobs.cache(jc), fin_train, ti, rfin);
  }
  if (stats) block_flush_stats(stats, c, 0u);   // kStatRays..kStatVReads
}

// Zeroes the per-frame query and sample counters of every cache job.
template <class J>
__global__ void k_cache_reset(J jobs, int njobs) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= njobs) return;
  const CacheDev& c = jobs.cache(j);
  if (c.on) {
    *c.qcount = 0;
    *c.cand_count = 0;
  }
}

// Cache-terminated paths of up to kMaxMlpTasks jobs (blockIdx.y = entry):
// radiance += throughput at vertex 1 * predicted reflected radiance there,
// then the usual clamp / demodulation / store.
struct ResolveEntry {
  const int* qcount;
  const uint32_t* qpix;
  const int* cand_count;
  const float* pred;
  int cand_cap;
  int pad;
};
struct ResolveSet {
  int n;
  int pad[3];
  ResolveEntry e[kMaxMlpTasks];
};

template <class J>
__global__ void __launch_bounds__(256) k_cache_resolve(J jobs, WfDev b, const __grid_constant__ ResolveSet rs,
                                                       unsigned long long* stats) {
  const ResolveEntry& r = rs.e[blockIdx.y];
  const int n = *r.qcount;
  if (stats && blockIdx.x == 0 && threadIdx.x == 0) {
    atomicAdd(stats + kStatCacheQueries, (unsigned long long)n);
    atomicAdd(stats + kStatCacheSamples, (unsigned long long)min(*r.cand_count, r.cand_cap));
  }
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t g = r.qpix[i];
    const int j = jobs.job_of(g);
    const float4 s0 = b.S0[g];
    const float4 s1 = b.S1[g];
    const float* p = r.pred + 3 * (size_t)i;
    const F3 L = f3(fmax_(p[0], 0.0f), fmax_(p[1], 0.0f), fmax_(p[2], 0.0f));
    const F3 radiance = xyz(s0) + xyz(s1) * L;
    finalize(jobs.outs(j), g - jobs.first(j), radiance, __float_as_uint(s1.w), jobs.clamp(j));
  }
}

// ---------------------------------------------------------------------------
// host: one frame's wave sequence for a job set of P pixels
// ---------------------------------------------------------------------------
inline WfDev wf_view(const WavefrontBufs& w) {
  WfDev d;
  d.R0 = (float4*)w.R0; d.R1 = (float4*)w.R1; d.R2 = (float4*)w.R2;
  d.S0 = (float4*)w.S0; d.S1 = (float4*)w.S1; d.S2 = (float4*)w.S2;
  d.hit = (uint4*)w.hit;
  d.q0 = w.q[0]; d.q1 = w.q[1]; d.a0 = w.act[0]; d.a1 = w.act[1];
  d.ctr = w.ctr;
  d.qcap = (uint32_t)w.qcap;
  return d;
}

inline int wf_sm_count() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 1;
}

// ---------------------------------------------------------------------------
// host: post-wave cache work of one job -- inference over its queries, the
// resolve of its cache-terminated paths, then its training steps.  Every
// per-frame quantity (counts, Adam step, sample draws) lives on the device,
// so the sequence can be captured in a CUDA graph and replayed.
// ---------------------------------------------------------------------------
// The MLP task of a cache job: inference (k < 0) or training step k.
inline MlpTask mlp_task_of(const CacheLaunch& cl, int k) {
  MlpTask t;
  std::memset(&t, 0, sizeof t);
  t.wb = cl.wb;
  t.extent = cl.extent;
  t.err = cl.err;
  if (k < 0) {
    t.q9 = cl.cd.qbuf;
    t.out3 = cl.pred;
    t.n_dev = cl.cd.qcount;
    t.n_max = cl.P;
  } else {
    t.q9 = cl.cd.cand_q9;
    t.y3 = cl.cd.cand_y3;
    t.n_dev = cl.cd.cand_count;
    t.n_max = cl.train_batch;
    t.pop_cap = cl.cd.cand_cap;
    t.seed = 0x9e3779b9u * (uint32_t)(k + 1);
    t.step = cl.step;
    t.partial = cl.partial;
    t.loss = cl.loss;
    t.grad = cl.grad;
    t.wm = cl.wm;
    t.m = cl.m;
    t.v = cl.v;
    t.wbw = cl.wb;
    t.lr = cl.lr;
  }
  return t;
}

// Post-wave cache work of `n` jobs, up to kMaxMlpTasks per launch: one
// inference launch over all their queries, one resolve launch, then per
// training step one gradient (+ reduction) and one Adam launch serving every
// job that still has steps to take.
template <class J>
cudaError_t launch_cache_post(const J& jobs, const WfDev& b, const CacheLaunch* cls, int n,
                              unsigned long long* stats, cudaStream_t st, uint32_t* launches) {
  uint32_t nl = 0;
  for (int c0 = 0; c0 < n; c0 += kMaxMlpTasks) {
    const int cn = std::min(kMaxMlpTasks, n - c0);
    MlpTaskSet ts;
    std::memset(&ts, 0, sizeof ts);
    ResolveSet rs;
    std::memset(&rs, 0, sizeof rs);
    int maxP = 1, steps = 0;
    for (int k = 0; k < cn; k++) {
      const CacheLaunch& cl = cls[c0 + k];
      ts.t[ts.n++] = mlp_task_of(cl, -1);
      rs.e[rs.n++] = ResolveEntry{cl.cd.qcount, cl.cd.qpix, cl.cd.cand_count, cl.pred, cl.cd.cand_cap, 0};
      maxP = std::max(maxP, cl.P);
      steps = std::max(steps, cl.train_steps);
    }
    cudaError_t e = mlp_infer_tasks(ts, st);
    if (e != cudaSuccess) return e;
    const int bx = std::max(1, std::min((maxP + 255) / 256, wf_sm_count() * 8 / cn));
    k_cache_resolve<J><<<dim3(bx, rs.n), 256, 0, st>>>(jobs, b, rs, stats);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    nl += 2;
    for (int k = 0; k < steps; k++) {
      MlpTaskSet tr;
      std::memset(&tr, 0, sizeof tr);
      for (int q = 0; q < cn; q++)
        if (k < cls[c0 + q].train_steps) tr.t[tr.n++] = mlp_task_of(cls[c0 + q], k);
      if ((e = mlp_gradient_tasks(tr, st)) != cudaSuccess) return e;
      if ((e = mlp_adam_tasks(tr, st)) != cudaSuccess) return e;
      nl += 4;   // gradient, the reduction's two stages, Adam
    }
  }
  if (launches) *launches += nl;
  return cudaSuccess;
}

template <class J, bool kSmem, int kSteps, int kMinB, bool kVarMaxT, int kUnroll = kSteps>
cudaError_t wf_launch_trace(const J& jobs, int smem, int blocks_per_sm, int sms, const WfDev& b, int w,
                            int implicit_n, int refill, unsigned long long* stats, cudaStream_t st) {
  auto* fn = k_wf_trace<J, kSmem, kSteps, kMinB, kVarMaxT, kUnroll>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
  }
  int per = blocks_per_sm;
  if (per <= 0) {
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, 256, smem);
    if (e != cudaSuccess || per < 1) per = 1;
  }
  fn<<<sms * per, 256, smem, st>>>(jobs, b, w, implicit_n, refill, stats);
  return cudaGetLastError();
}

// Tracer variants (the autotuner's trace_variant): DDA iterations per pass of
// the warp bookkeeping x minimum resident blocks per SM (register cap).
// Measured on the 1080p / 256^3 frame with FlatDDA's current-level register
// layout: 8 x 5 (48 registers) 1.48 ms of trace, 6 x 5 1.49, 12 x 5 1.63,
// 16 x 5 1.69 ms; with the typed test loads 8 x 5 1.436, 8 x 6 (40 registers,
// spilling) 1.491, 8 x 4 (59 registers) 1.497 ms; with the earlier layout 8 x 5 1.60-1.66, 6 x 5 1.67,
// 6 x 4 (57 registers) 1.71, 4 x 4 1.74, 2 x 1 (69) 1.98, 1 x 1 2.20 ms.
// (Stepping until enough lanes are idle, with a ballot after every iteration,
// ran 1.88 ms: the per-iteration ballot costs more than the idle lanes of a
// fixed pass.)  Also measured with the earlier layout and dropped, each
// bit-identical: a step with every outcome selected instead of branched (only
// the descent branched) 2.02 ms; descents parked until the end of each pass,
// so that a warp runs the descent block once per pass, 1.71 (4 x 5) - 1.80 ms
// (8 x 5); an exact empty-space skip (brick distance field and 4^3 sub-block
// masks, the skipped steps replayed in closed form per axis: 41% fewer step
// calls on this frame) 2.2 - 3.3 ms, because a warp runs the ~100-instruction
// replay in nearly every step in which one of its lanes needs it.
template <class J, bool kSmem, bool kVarMaxT = false>
cudaError_t wf_dispatch_trace(int variant, const J& jobs, int smem, int tb, int sms, const WfDev& b, int w, int impl,
                              int refill, unsigned long long* stats, cudaStream_t st) {
  if (kVarMaxT)   // the ReSTIR passes: the default shape only
    return wf_launch_trace<J, kSmem, 8, 5, kVarMaxT>(jobs, smem, tb, sms, b, w, impl, refill, stats, st);
  switch (variant) {
    case 1: return wf_launch_trace<J, kSmem, 6, 5, false>(jobs, smem, tb, sms, b, w, impl, refill, stats, st);
    case 2: return wf_launch_trace<J, kSmem, 6, 4, false>(jobs, smem, tb, sms, b, w, impl, refill, stats, st);
    case 3: return wf_launch_trace<J, kSmem, 4, 4, false>(jobs, smem, tb, sms, b, w, impl, refill, stats, st);
    case 4: return wf_launch_trace<J, kSmem, 2, 1, false>(jobs, smem, tb, sms, b, w, impl, refill, stats, st);
    case 5: return wf_launch_trace<J, kSmem, 1, 1, false>(jobs, smem, tb, sms, b, w, impl, refill, stats, st);
    // the default shape with the step loop unrolled 1, 2 or 4 times instead of 8 (smaller code;
    // measured 1.396 / 1.354 / 1.358 ms of trace per 1080p frame against 1.349 fully unrolled)
    case 6: return wf_launch_trace<J, kSmem, 8, 5, false, 1>(jobs, smem, tb, sms, b, w, impl, refill, stats, st);
    case 7: return wf_launch_trace<J, kSmem, 8, 5, false, 2>(jobs, smem, tb, sms, b, w, impl, refill, stats, st);
    case 8: return wf_launch_trace<J, kSmem, 8, 5, false, 4>(jobs, smem, tb, sms, b, w, impl, refill, stats, st);
    default: return wf_launch_trace<J, kSmem, 8, 5, false>(jobs, smem, tb, sms, b, w, impl, refill, stats, st);
  }
}

// Launches generate + (trace, shade) x waves; shade(b, w, blocks) launches
// the shading kernel of wave w.  smem > 0 selects the shared-memory bitmap
// tracer (single scene only).
constexpr int kPrimaryRefill = 32;   // idle lanes that trigger a refill in the primary wave (at least)

template <class J, class ShadeFn, bool kVarMaxT = false>
cudaError_t wf_run_waves(const J& jobs, uint32_t P, int waves, int smem, const WavefrontBufs& wb,
                         const WavefrontTuning& tune, unsigned long long* stats, cudaStream_t st, uint32_t* launches,
                         cudaEvent_t* trace_ev, int max_timed_waves, int* timed_waves, ShadeFn shade,
                         int tail_from = 0) {
  if (waves + 1 > wb.max_waves) return cudaErrorInvalidValue;
  const WfDev b = wf_view(wb);
  cudaError_t e = cudaMemsetAsync(wb.ctr, 0, (size_t)wb.max_waves * 16, st);
  if (e != cudaSuccess) return e;
  const int sms = wf_sm_count();
  const int refill = tune.refill_min > 0 ? tune.refill_min : 8;
  const int sblocks = sms * (tune.shade_blocks_per_sm > 0 ? tune.shade_blocks_per_sm : 32);
  uint32_t nl = 0;
  k_wf_generate<J><<<(P + 255) / 256, 256, 0, st>>>(jobs, P, b);
  nl++;
  int timed = 0;
  for (int w = 0; w < waves; w++) {
    if (tail_from > 0 && w == tail_from) {   // the remaining paths, one thread each
      // a resident grid of 128-thread blocks: 260 us per 1080p cache frame against 282 with 256-thread
      // blocks (a block's round waits for its slowest path) and 262 with 64; a grid of one block per 256
      // training paths, blocks without paths returning at once, ran 291
      const int tblocks = sms * 6;
      if (smem > 0) {
        e = cudaFuncSetAttribute(k_wf_tail<J, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e == cudaSuccess) k_wf_tail<J, true><<<tblocks, 128, smem, st>>>(jobs, b, w, stats);
      } else {
        k_wf_tail<J, false><<<tblocks, 128, 0, st>>>(jobs, b, w, stats);
      }
      if (e != cudaSuccess || (e = cudaGetLastError()) != cudaSuccess) return e;
      nl++;
      break;
    }
    const bool tm = trace_ev && w < max_timed_waves;
    if (tm && (e = cudaEventRecord(trace_ev[2 * w], st)) != cudaSuccess) return e;
    const int impl = w == 0 ? (int)P : 0;
    const int tb = tune.trace_blocks_per_sm;
    // the coherent primary rays refill later: the 1080p primary wave took 299 / 290 / 285 / 277 / 271 us at
    // 8 / 12 / 16 / 24 / 32 idle lanes (32: only whole warps refill), while the later waves are fastest at 8
    // (490 / 426 / 143 us against 530 / 479 / 153 at 24)
    const int rf = w == 0 ? std::max(refill, kPrimaryRefill) : refill;
    if (smem > 0)
      e = wf_dispatch_trace<J, true, kVarMaxT>(tune.trace_variant, jobs, smem, tb, sms, b, w, impl, rf, stats, st);
    else
      e = wf_dispatch_trace<J, false, kVarMaxT>(tune.trace_variant, jobs, 0, tb, sms, b, w, impl, rf, stats, st);
    if (e != cudaSuccess) return e;
    if (tm && (e = cudaEventRecord(trace_ev[2 * w + 1], st)) != cudaSuccess) return e;
    if (tm) timed++;
    nl++;
    if ((e = shade(b, w, sblocks)) != cudaSuccess) return e;
    nl++;
  }
  if (launches) *launches += nl;
  if (timed_waves) *timed_waves = timed;
  return cudaGetLastError();
}

// The plain path's wave sequence (with the radiance cache's counter reset
// when any job has the cache on).
template <class J>
cudaError_t wf_launch_frame(const J& jobs, uint32_t P, int waves, int smem, const WavefrontBufs& wb,
                            const WavefrontTuning& tune, unsigned long long* stats, cudaStream_t st,
                            uint32_t* launches, cudaEvent_t* trace_ev, int max_timed_waves, int* timed_waves,
                            int njobs = 1, int tail_from = 0) {
  if (waves + 1 > wb.max_waves) return cudaErrorInvalidValue;
  if (jobs.any_cache()) {
    k_cache_reset<J><<<(njobs + 127) / 128, 128, 0, st>>>(jobs, njobs);
    if (launches) (*launches)++;
  }
  return wf_run_waves(jobs, P, waves, smem, wb, tune, stats, st, launches, trace_ev, max_timed_waves, timed_waves,
                      [&](const WfDev& b, int w, int sblocks) {
                        if (w == 0) k_wf_shade_primary<J><<<sblocks, 256, 0, st>>>(jobs, P, b, stats);
                        else k_wf_shade<J><<<sblocks, 256, 0, st>>>(jobs, b, w);
                        return cudaGetLastError();
                      }, tail_from);
}

}  // namespace vrt
