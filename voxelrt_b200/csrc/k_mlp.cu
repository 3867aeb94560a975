// k_mlp.cu -- the radiance cache's BF16 tensor-core kernels (tcgen05, TMEM).
//
// This file starts with a GEMM self-test of the two operand forms the MLP
// uses: K-major A [128 x K] times K-major B [N x K] (forward and input
// gradients), and MN-major views of two row-chunked tiles X [128 x C],
// Y [128 x N] giving X^T Y (weight gradients).
#include <cuda_runtime.h>
#include <cstdint>
#include "umma.cuh"
#include "vrt_device.cuh"
#include "vrt_internal.h"
#include <cuda_bf16.h>
#include <vector>
#include <cmath>
#include <algorithm>

namespace vrt {

constexpr uint32_t kMbarSpin = 1u << 20;   // bounded mbarrier wait (iterations)

// mode 0: D[128 x N] = A[128 x K] * B[N x K]^T   (A, B row-major in global)
// mode 1: D[C x N]   = X[128 x C]^T * Y[128 x N] (rows 0..C-1 of the 128-row tile)
__global__ void __launch_bounds__(128, 1) k_umma_selftest(int mode, int K, int N, const uint16_t* __restrict__ A,
                                                          const uint16_t* __restrict__ B, float* __restrict__ D,
                                                          int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5;
  // operand A at smem[0 .. 32 KB), operand B at smem[32 KB .. 64 KB); 4 KB slack after each
  uint8_t* sA = smem;
  uint8_t* sB = smem + 36 * 1024;
  if (warp == 0) umma::tmem_alloc(&tmem_base, 64);
  if (tid == 0) umma::mbar_init(&mbar, 1);
  if (mode == 0 || mode == 2) {
    for (int i = tid; i < 128 * K; i += 128) {
      const int r = i / K, c = i % K;
      *reinterpret_cast<uint16_t*>(sA + umma::canon_off(r, c, K)) = A[i];
    }
    for (int i = tid; i < N * K; i += 128) {
      if (mode == 0) {
        const int r = i / K, c = i % K;
        *reinterpret_cast<uint16_t*>(sB + umma::canon_off(r, c, K)) = B[i];
      } else {   // B given as [K x N], rows = K: read MN-major
        const int r = i / N, c = i % N;
        *reinterpret_cast<uint16_t*>(sB + umma::canon_off(r, c, N)) = B[i];
      }
    }
  } else {
    const int C = K;   // X has C columns
    for (int i = tid; i < 128 * C; i += 128) {
      const int r = i / C, c = i % C;
      *reinterpret_cast<uint16_t*>(sA + umma::canon_off(r, c, C)) = A[i];
    }
    for (int i = tid; i < 128 * N; i += 128) {
      const int r = i / N, c = i % N;
      *reinterpret_cast<uint16_t*>(sB + umma::canon_off(r, c, N)) = B[i];
    }
  }
  umma::fence_smem_to_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = tmem_base;
  if (tid == 0) {
    const uint32_t a0 = umma::smem_u32(sA), b0 = umma::smem_u32(sB);
    if (mode == 0) {
      const uint32_t id = umma::idesc_bf16(128, N, false, false);
      for (int ks = 0; ks < K / 16; ks++)
        umma::mma_bf16(tbase, umma::desc_kmajor(a0 + 256u * ks, K), umma::desc_kmajor(b0 + 256u * ks, K), id,
                       ks > 0 ? 1u : 0u);
    } else if (mode == 2) {
      const uint32_t id = umma::idesc_bf16(128, N, false, true);
      for (int ks = 0; ks < K / 16; ks++)
        umma::mma_bf16(tbase, umma::desc_kmajor(a0 + 256u * ks, K), umma::desc_mnmajor(b0 + 32u * N * ks, N), id,
                       ks > 0 ? 1u : 0u);
    } else {
      const int C = K;
      const uint32_t id = umma::idesc_bf16(128, N, true, true);
      for (int ks = 0; ks < 128 / 16; ks++)
        umma::mma_bf16(tbase, umma::desc_mnmajor(a0 + 2u * 16u * C * ks, C),
                       umma::desc_mnmajor(b0 + 2u * 16u * N * ks, N), id, ks > 0 ? 1u : 0u);
    }
    umma::commit(&mbar);
  }
  const bool ok = __syncthreads_and(umma::mbar_wait(&mbar, 0, kMbarSpin) ? 1 : 0);
  umma::fence_after_sync();
  if (ok) {
    const int rows = mode == 1 ? K : 128;
    for (int c0 = 0; c0 < N; c0 += 16) {
      float v[16];
      umma::tmem_ld16(tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (tid < rows)
        for (int j = 0; j < 16 && c0 + j < N; j++) D[(size_t)tid * N + c0 + j] = v[j];
    }
  } else if (tid == 0) {
    atomicExch(err, 1);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tbase, 64);
}


// ===========================================================================
// The radiance-cache MLP: 80 -> 64 -> 64 -> 64 -> 3 (output padded to 16),
// ReLU on the hidden layers, no biases (the encoding carries a constant 1).
// Parameters: W_l row-major [K_in x N_out], fp32 masters + bf16 copy.
// ===========================================================================
namespace mlp {
constexpr int kIn = 80, kHid = 64, kOutPad = 16, kOut = 3;
constexpr int kL0 = kIn * kHid, kL1 = kHid * kHid, kL2 = kHid * kHid, kL3 = kHid * kOutPad;
constexpr int kOff0 = 0, kOff1 = kL0, kOff2 = kL0 + kL1, kOff3 = kL0 + kL1 + kL2;
constexpr int kParams = kL0 + kL1 + kL2 + kL3;   // 14336
constexpr int kFreqs = 12;

// forward weight copies (bytes): W_l^T as [N_out rows x K_in columns], K-major
constexpr int kWf0 = 0, kWf1 = kWf0 + kHid * kIn * 2, kWf2 = kWf1 + kHid * kHid * 2, kWf3 = kWf2 + kHid * kHid * 2;
constexpr int kWEnd = kWf3 + kOutPad * kHid * 2;   // 28 KB
// training kernel: two groups of 128 samples (threads 0-127, 128-255), each
// with its own input, activation and gradient tiles
constexpr int kGA0 = 0, kGA1 = kGA0 + 128 * kIn * 2, kGA2 = kGA1 + 128 * kHid * 2, kGA3 = kGA2 + 128 * kHid * 2;
constexpr int kGDY = kGA3 + 128 * kHid * 2, kGStride = kGDY + 128 * kHid * 2;   // 84 KB per group
constexpr int kGBase = kWEnd, kGEnd = kGBase + 2 * kGStride;
constexpr int kTrainSmem = kGEnd + 1024;   // slack: MN-major views read up to 1 KB past a tile
// inference kernel: forward weights + per tile (two groups of threads, two
// tiles in flight each) one operand tile X: the 80-column input, then each
// hidden layer's 64 columns written over it once the MMAs that read it have
// completed
constexpr int kITile = 128 * kIn * 2;
constexpr int kIX = kWEnd, kIEnd = kIX + 4 * kITile;
constexpr int kInferSmem = kIEnd;   // 108 KB: two CTAs per SM

// TMEM columns (fp32): layer outputs / input gradients of group g at 64 g,
// weight gradients accumulated over all of a CTA's samples at kTW*
constexpr uint32_t kTFwd = 0, kTW0 = 128, kTW1 = 192, kTW2 = 256, kTW3 = 320;

__device__ __forceinline__ uint16_t f2bf(float x) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}
__device__ __forceinline__ float bf2f(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }

// Input encoding of one query: position (metres) normalised by the world
// extent, then per axis sin/cos(2 pi 2^k frac(p / 2)) for octaves k = 0..11,
// followed by normal, albedo, 1, 0.  Only octave 0 calls sincos_; each
// higher octave follows by the double-angle identities
//   sin 2a = 2 sin a cos a,  cos 2a = (cos a - sin a)(cos a + sin a),
// which keeps the per-query cost at 3 sincos_ calls (the rounding error
// doubles per octave: ~2e-4 at octave 11, far below the bf16 step).
__device__ __forceinline__ void encode(const float* q, float extent, float* f) {
  float sn[3], cs[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const float x = (q[a] / extent) * 0.5f;
    const float t = x - floorf(x);
    sincos_(kTwoPi * t, sn[a], cs[a]);
  }
  // the x and y axes' recurrences as packed pairs, z alone; same roundings
  float2 s01 = make_float2(sn[0], sn[1]), c01 = make_float2(cs[0], cs[1]);
  float s2 = sn[2], c2 = cs[2];
  const float2 two = make_float2(2.0f, 2.0f);
#pragma unroll
  for (int k = 0; k < kFreqs; k++) {
    f[6 * k + 0] = s01.x; f[6 * k + 1] = s01.y; f[6 * k + 2] = s2;
    f[6 * k + 3] = c01.x; f[6 * k + 4] = c01.y; f[6 * k + 5] = c2;
    const float2 ns01 = f2_mul(f2_mul(s01, c01), two);
    const float2 nc01 = f2_mul(f2_sub(c01, s01), f2_add(c01, s01));
    const float ns2 = (s2 * c2) * 2.0f;
    const float nc2 = (c2 - s2) * (c2 + s2);
    s01 = ns01; c01 = nc01; s2 = ns2; c2 = nc2;
  }
  f[72] = q[3]; f[73] = q[4]; f[74] = q[5];
  f[75] = q[6]; f[76] = q[7]; f[77] = q[8];
  f[78] = 1.0f; f[79] = 0.0f;
}

// Packs 8 floats as bf16 (RNE) into one 16-byte chunk, element 0 lowest.
__device__ __forceinline__ uint4 pack8(const float* v) {
  uint4 r;
  uint32_t* w = &r.x;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    w[i] = *reinterpret_cast<const uint32_t*>(&h);
  }
  return r;
}

// Row `row` of a row-chunked tile with C columns from C floats (16-byte stores).
__device__ __forceinline__ void store_row(uint8_t* tile, int row, int C, const float* v) {
#pragma unroll
  for (int cg = 0; cg < C / 8; cg++)
    *reinterpret_cast<uint4*>(tile + umma::canon_off(row, 8 * cg, C)) = pack8(v + 8 * cg);
}

// pack8 of max(v, 0): the conversion's .relu form clamps negative values to
// zero in the same instruction (bf16 rounding keeps the sign, so the result
// equals rounding after the ReLU).
__device__ __forceinline__ uint4 pack8_relu(const float* v) {
  uint4 r;
  uint32_t* w = &r.x;
#pragma unroll
  for (int i = 0; i < 4; i++)
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(w[i]) : "f"(v[2 * i + 1]), "f"(v[2 * i]));
  return r;
}

// store_row of ReLU(v).
__device__ __forceinline__ void store_row_relu(uint8_t* tile, int row, int C, const float* v) {
#pragma unroll
  for (int cg = 0; cg < C / 8; cg++)
    *reinterpret_cast<uint4*>(tile + umma::canon_off(row, 8 * cg, C)) = pack8_relu(v + 8 * cg);
}

// The bf16 weight copy is kept in global memory as the kernels' shared-memory
// image of the weights: for each layer W^T (rows N_out, columns K_in) in the
// canonical no-swizzle layout at byte offset kWf<l>, kWEnd bytes in all.
// Read K-major it is the B operand of the forward GEMMs; read MN-major it is
// the B operand W of the input-gradient GEMMs dX = dH W^T.  image_index maps
// parameter i (row-major W_l[K_in x N_out]) to its u16 position in the image.
__device__ __forceinline__ int image_index(int i) {
  int kin, nout, off, fbase;
  if (i < kOff1) { kin = kIn; nout = kHid; off = kOff0; fbase = kWf0; }
  else if (i < kOff2) { kin = kHid; nout = kHid; off = kOff1; fbase = kWf1; }
  else if (i < kOff3) { kin = kHid; nout = kHid; off = kOff2; fbase = kWf2; }
  else { kin = kHid; nout = kOutPad; off = kOff3; fbase = kWf3; }
  const int k = (i - off) / nout, n = (i - off) % nout;
  return (int)((fbase + umma::canon_off(n, k, kin)) >> 1);
}
static_assert(kWEnd == kParams * 2, "the weight image holds every parameter once");

// Copies the weight image (kWEnd bytes) into shared memory, 16 bytes per access.
__device__ __forceinline__ void load_weights(uint8_t* smem, const uint16_t* __restrict__ w) {
  const uint4* src = reinterpret_cast<const uint4*>(w);
  uint4* dst = reinterpret_cast<uint4*>(smem);
  for (int i = threadIdx.x; i < kWEnd / 16; i += blockDim.x) dst[i] = __ldg(src + i);
}

struct Ctl {
  uint64_t* mbar;
  uint32_t phase;
  bool ok;
};

// One elected thread issues `nk` K-steps of D = A * B (both K-major).
__device__ __forceinline__ void issue_fwd(uint32_t tmem, uint32_t a, uint32_t b, int K, int N, bool acc0) {
  const uint32_t id = umma::idesc_bf16(128, N, false, false);
  for (int ks = 0; ks < K / 16; ks++)
    umma::mma_bf16(tmem, umma::desc_kmajor(a + 256u * ks, K), umma::desc_kmajor(b + 256u * ks, K), id,
                   (acc0 || ks > 0) ? 1u : 0u);
}

// dW[K_in x N] (+)= X^T Y over the 128 samples of the tile (MN-major views).
__device__ __forceinline__ void issue_dw(uint32_t tmem, uint32_t x, int Cx, uint32_t y, int N, bool acc0) {
  const uint32_t id = umma::idesc_bf16(128, N, true, true);
  for (int ks = 0; ks < 128 / 16; ks++)
    umma::mma_bf16(tmem, umma::desc_mnmajor(x + 32u * Cx * ks, Cx), umma::desc_mnmajor(y + 32u * N * ks, N), id,
                   (acc0 || ks > 0) ? 1u : 0u);
}

// dX[128 x N] = dH[128 x K] * W^T from the forward weight copy read MN-major
// (W^T stored with rows K = N_out and columns N = K_in).
__device__ __forceinline__ void issue_dx(uint32_t tmem, uint32_t a, int K, uint32_t w, int N) {
  const uint32_t id = umma::idesc_bf16(128, N, false, true);
  for (int ks = 0; ks < K / 16; ks++)
    umma::mma_bf16(tmem, umma::desc_kmajor(a + 256u * ks, K), umma::desc_mnmajor(w + 32u * N * ks, N), id,
                   ks > 0 ? 1u : 0u);
}

// All threads: commit (thread 0) and wait for the MMAs, bounded.
__device__ __forceinline__ void sync_mma(Ctl& c) {
  if (threadIdx.x == 0) umma::commit(c.mbar);
  const bool ok = umma::mbar_wait(c.mbar, c.phase, kMbarSpin);
  c.phase ^= 1u;
  c.ok = __syncthreads_and(ok ? 1 : 0) && c.ok;
  umma::fence_after_sync();
}

// Thread-to-smem handoff before the tensor core reads what threads wrote.
__device__ __forceinline__ void publish() {
  umma::fence_smem_to_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
}

// publish() that also agrees on `ok` across the block (false if any thread's
// bounded wait ran out).
__device__ __forceinline__ bool publish_and(bool ok) {
  umma::fence_smem_to_async();
  umma::fence_before_sync();
  const bool all = __syncthreads_and(ok ? 1 : 0) != 0;
  umma::fence_after_sync();
  return all;
}

// Reads `n` (16 or 64) fp32 columns [col, col+n) of this thread's TMEM lane:
// all loads issued, then one wait.
template <int n>
__device__ __forceinline__ void tmem_row(uint32_t tbase, uint32_t col, float* out) {
  const uint32_t lane = (uint32_t)(((threadIdx.x >> 5) & 3) * 32) << 16;   // warp w: lanes 32 (w % 4) ..
  uint32_t r[n];
#pragma unroll
  for (int c0 = 0; c0 < n; c0 += 16) umma::tmem_ld16_raw(tbase + lane + col + (uint32_t)c0, r + c0);
#pragma unroll
  for (int c0 = 0; c0 < n; c0 += 16) umma::tmem_wait_dep(r + c0);
#pragma unroll
  for (int i = 0; i < n; i++) out[i] = __uint_as_float(r[i]);
}

// Forward of G tiles of 128 samples (thread t: group t / 128, row t % 128):
// activations written to A1..A3 (bf16) of the thread's group (group g's
// tiles at +g * gstride), output o[16].  With kMasks, returns the three
// hidden layers' ReLU masks (training).  Thread 0 issues every group's MMAs.
template <int G, bool kMasks>
__device__ __forceinline__ void forward_tile(uint8_t* smem, uint32_t tbase, Ctl& c, int a_in, int a1, int a2, int a3,
                                             int gstride, float* o, uint64_t* mask) {
  const uint32_t s0 = umma::smem_u32(smem);
  const int ain[3] = {a_in, a1, a2};
  const int aout[3] = {a1, a2, a3};
  const int wf[3] = {kWf0, kWf1, kWf2};
  const int t = threadIdx.x, g = t >> 7, r = t & 127;
  const uint32_t tcol = kTFwd + 64u * (uint32_t)g;
#pragma unroll
  for (int l = 0; l < 3; l++) {
    const int K = l == 0 ? kIn : kHid;
    if (t == 0)
      for (int q = 0; q < G; q++)
        issue_fwd(tbase + kTFwd + 64u * q, s0 + ain[l] + q * gstride, s0 + wf[l], K, kHid, false);
    sync_mma(c);
    float h[kHid];
    tmem_row<kHid>(tbase, tcol, h);
    if (kMasks) {
      uint32_t lo = 0u, hi = 0u;
#pragma unroll
      for (int j = 0; j < 32; j++) lo |= (h[j] > 0.0f ? 1u : 0u) << j;
#pragma unroll
      for (int j = 0; j < 32; j++) hi |= (h[32 + j] > 0.0f ? 1u : 0u) << j;
      mask[l] = ((uint64_t)hi << 32) | lo;
    }
#pragma unroll
    for (int j = 0; j < kHid; j++) h[j] = h[j] > 0.0f ? h[j] : 0.0f;
    store_row(smem + aout[l] + g * gstride, r, kHid, h);
    publish();
  }
  if (t == 0)
    for (int q = 0; q < G; q++) issue_fwd(tbase + kTFwd + 64u * q, s0 + a3 + q * gstride, s0 + kWf3, kHid, kOutPad, false);
  sync_mma(c);
  tmem_row<kOutPad>(tbase, tcol, o);
}

// Writes the encoded input of sample `src` (zeros when idx >= n) into row
// `row` of the input tile.
__device__ __forceinline__ void stage_input(uint8_t* tile, int row, const float* __restrict__ q9, int n, int idx,
                                            float extent, int src) {
  float f[kIn];
  if (idx < n) {
    float q[9];
#pragma unroll
    for (int j = 0; j < 9; j++) q[j] = q9[(size_t)src * 9 + j];
    encode(q, extent, f);
  } else {
#pragma unroll
    for (int j = 0; j < kIn; j++) f[j] = 0.0f;
  }
  store_row(tile, row, kIn, f);
}

// As stage_input with the query already in registers (valid: row holds a sample).
__device__ __forceinline__ void stage_query(uint8_t* tile, int row, const float* q, bool valid, float extent) {
  float f[kIn];
  if (valid) {
    encode(q, extent, f);
  } else {
#pragma unroll
    for (int j = 0; j < kIn; j++) f[j] = 0.0f;
  }
  store_row(tile, row, kIn, f);
}

// Source index of training sample idx: in order when the population fits the
// step, else a uniform draw (with replacement) from the population.
__device__ __forceinline__ int sample_source(int idx, int pop, bool draw, uint32_t seed) {
  if (!draw) return idx;
  const uint32_t h = pcg_hash(seed ^ pcg_hash((uint32_t)idx * 2654435761u + 0x9e3779b9u));
  return (int)(((uint64_t)h * (uint64_t)(uint32_t)pop) >> 32);
}

// (samples used by a step, population, draw?) for the selection rule of mlp_gradient.
__device__ __forceinline__ void sample_counts(int n, const int* n_dev, int pop_cap, int& nn, int& pop, bool& draw) {
  if (!n_dev) { nn = n; pop = n; draw = false; return; }
  pop = min(max(*n_dev, 0), pop_cap);
  nn = min(pop, n);
  draw = pop > n;
}

}  // namespace mlp

// Encoded inputs as bf16 (for checking against the CPU restatement).
__global__ void k_mlp_encode(const float* __restrict__ q9, int n, float extent, uint16_t* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float q[9], f[mlp::kIn];
  for (int j = 0; j < 9; j++) q[j] = q9[(size_t)i * 9 + j];
  mlp::encode(q, extent, f);
  for (int j = 0; j < mlp::kIn; j++) out[(size_t)i * mlp::kIn + j] = mlp::f2bf(f[j]);
}

// The task of CTA b: tasks own contiguous CTA ranges [cta0, cta0 + ctas).
__device__ __forceinline__ int task_of(const MlpTaskSet& ts, int b) {
  int j = 0;
  while (j + 1 < ts.n && b >= ts.t[j + 1].cta0) j++;
  return j;
}

// Barrier of the 128 threads of group g (named barrier 1 + g) that also
// agrees on `ok` across them, with the handoff fences of publish_and.
__device__ __forceinline__ bool group_publish_and(int g, bool ok) {
  umma::fence_smem_to_async();
  umma::fence_before_sync();
  uint32_t all;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, %2, 128, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(all)
      : "r"(ok ? 1u : 0u), "r"(1 + g)
      : "memory");
  umma::fence_after_sync();
  return all != 0u;
}

// Inference: out3[i*3 + c] = MLP(encode(q_i)) for every task of the set.
// A CTA of 256 threads is two groups of 128 (threads 128 g .. 128 g + 127)
// that share the weights in shared memory and otherwise run independently,
// synchronising on their own named barrier.  Each group keeps two 128-query
// tiles in flight, each with its own TMEM accumulator (columns 64 (2g + u)),
// its own operand tile and its own mbarrier: while the tensor core runs one
// tile's layer, the group's threads unpack the other tile's previous layer
// (TMEM load, ReLU, bf16 pack into the next operand tile), so the MMA latency
// hides behind the epilogue work, and the other group's tiles fill the
// tensor core's remaining gaps.  A layer's output overwrites its input tile:
// every thread waits for the layer's MMA completion (which covers the MMAs'
// shared-memory reads) before it stores.  Thread r of a group owns row r of
// its tiles; the first thread of each group issues the group's MMAs.  The
// groups of a task's CTAs stride over its tile pairs.  (Handing each operand
// over through a per-tile mbarrier instead -- one arrival per thread, only the
// issuing thread waiting -- ran 70.7 against 65.8 us for 983 K queries: the
// issuer's polling and the warps it holds back cost more than the barrier.)
__global__ void __launch_bounds__(256, 2) k_mlp_infer(const __grid_constant__ MlpTaskSet ts) {
  using namespace mlp;
  const MlpTask& tk = ts.t[task_of(ts, blockIdx.x)];
  int n = tk.n_max;
  if (tk.n_dev) n = min(*tk.n_dev, n);
  const int tiles = (n + 127) / 128;
  const int cb = blockIdx.x - tk.cta0;
  if (2 * cb >= tiles) return;   // nothing for this CTA (before any TMEM allocation)
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t mbar[4];
  __shared__ uint32_t tmem_base;
  const int warp = threadIdx.x >> 5, g = threadIdx.x >> 7, t = threadIdx.x & 127;
  if (warp == 0) umma::tmem_alloc(&tmem_base, 256);
  if (threadIdx.x < 4) umma::mbar_init(&mbar[threadIdx.x], 1);
  load_weights(smem, tk.wb);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = tmem_base;
  const uint32_t s0 = umma::smem_u32(smem);
  // this group's tiles: X (input, 80 columns; then each hidden layer, 64 columns)
  const int X[2] = {kIX + (2 * g) * kITile, kIX + (2 * g + 1) * kITile};
  const uint32_t acc[2] = {tbase + 64u * (uint32_t)(2 * g), tbase + 64u * (uint32_t)(2 * g + 1)};
  uint64_t* mb = mbar + 2 * g;
  uint32_t phase[2] = {0u, 0u};
  bool ok = true;
  const int vctas = 2 * tk.ctas;           // groups of the task: pairs (pt, pt + vctas), pt = vb + k stride
  const int vb = 2 * cb + g;
  const int stride = 2 * vctas;
  float q[2][9];
  auto fetch = [&](int pair_tile) {
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int idx = (pair_tile + u * vctas) * 128 + t;
      if (idx < n) {
#pragma unroll
        for (int j = 0; j < 9; j++) q[u][j] = __ldg(tk.q9 + (size_t)idx * 9 + j);
      }
    }
  };
  // tensor-core work of layer l of tile u (the group's first thread), completion on mb[u]
  auto issue = [&](int u, int l) {
    if (t != 0) return;
    if (l == 0) issue_fwd(acc[u], s0 + X[u], s0 + kWf0, kIn, kHid, false);
    else if (l == 1) issue_fwd(acc[u], s0 + X[u], s0 + kWf1, kHid, kHid, false);
    else if (l == 2) issue_fwd(acc[u], s0 + X[u], s0 + kWf2, kHid, kHid, false);
    else issue_fwd(acc[u], s0 + X[u], s0 + kWf3, kHid, kOutPad, false);
    umma::commit(&mb[u]);
  };
  auto wait = [&](int u) {
    ok = umma::mbar_wait(&mb[u], phase[u], kMbarSpin) && ok;
    phase[u] ^= 1u;
    umma::fence_after_sync();
  };
  if (vb < tiles) fetch(vb);
  // The loop runs while the group agrees on `ok` (every exit is decided on a
  // value its barrier made uniform).  No barrier closes a pair: the next
  // pair's first MMA is issued after the staging barrier, which each thread
  // reaches after reading its last TMEM rows, and each thread writes the next
  // input tile only after it has seen the MMAs that read the tile complete.
  for (int pt = vb; pt < tiles; pt += stride) {
    int idx[2];
    float qq[2][9];
#pragma unroll
    for (int u = 0; u < 2; u++) {
      idx[u] = (pt + u * vctas) * 128 + t;
#pragma unroll
      for (int j = 0; j < 9; j++) qq[u][j] = q[u][j];
    }
    // stage both tiles, then start both first layers (one barrier for the pair: 65.0 -> 63.1 us for 983 K
    // queries; a barrier per tile within the layers is kept -- unpacking both tiles of a layer before one
    // barrier ran 70.0 us, the tensor core then waits for both epilogues)
    // the group's last pair may hold one tile only (its second lies past the
    // queries): then the second tile is neither staged nor computed
    const int nu = pt + vctas < tiles ? 2 : 1;
    stage_query(smem + X[0], t, qq[0], idx[0] < n, tk.extent);
    if (nu == 2) stage_query(smem + X[1], t, qq[1], idx[1] < n, tk.extent);
    ok = group_publish_and(g, ok);
    if (!ok) break;
    issue(0, 0);
    if (nu == 2) issue(1, 0);
    fetch(pt + stride);                    // the next pair's queries, in flight during this pair
#pragma unroll 1
    for (int l = 0; l < 4 && ok; l++) {
#pragma unroll
      for (int u = 0; u < 2; u++) {
        if (u >= nu) continue;
        wait(u);
        if (l < 3) {
          float h[kHid];
          tmem_row<kHid>(acc[u], 0u, h);
          store_row_relu(smem + X[u], t, kHid, h);
          ok = group_publish_and(g, ok);
          if (ok) issue(u, l + 1);
        } else {
          float o[kOutPad];
          tmem_row<kOutPad>(acc[u], 0u, o);
          if (ok && idx[u] < n)
            for (int j = 0; j < kOut; j++) tk.out3[(size_t)idx[u] * 3 + j] = o[j];
        }
      }
    }
  }
  ok = group_publish_and(g, ok);           // the last pair's output waits, agreed
  if (!ok && t == 0) atomicExch(tk.err, 1);
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tbase, 256);
}

// One gradient pass: per-CTA partial dW (sum over the CTA's samples) of the
// relative L2 loss sum_c (o_c - y_c)^2 / (o_c^2 + 0.01), the denominator held
// constant (not differentiated).  256 threads work on 256 samples per
// iteration as two groups of 128; thread 0 issues all MMAs, so the weight
// gradients of both groups accumulate in order into the same TMEM columns.
// Input gradients dX = dH W^T read the forward weight copy MN-major; weight
// gradients dW = X^T dH read the activation tiles MN-major (no transposes).
__global__ void __launch_bounds__(256, 1) k_mlp_grad(const __grid_constant__ MlpTaskSet ts) {
  using namespace mlp;
  const MlpTask& tk = ts.t[task_of(ts, blockIdx.x)];
  const int cb = blockIdx.x - tk.cta0;
  const float* __restrict__ q9 = tk.q9;
  const float* __restrict__ y3 = tk.y3;
  const float extent = tk.extent;
  int n, pop;
  bool draw;
  sample_counts(tk.n_max, tk.n_dev, tk.pop_cap, n, pop, draw);
  uint32_t seed = tk.seed;
  if (tk.step) seed ^= pcg_hash((uint32_t)*tk.step + 0x6a09e667u);
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_base;
  __shared__ float s_loss[8];
  const int t = threadIdx.x, warp = t >> 5, g = t >> 7, r = t & 127;
  if (warp == 0) umma::tmem_alloc(&tmem_base, 512);
  if (t == 0) umma::mbar_init(&mbar, 1);
  load_weights(smem, tk.wb);
  for (int i = t; i < (kTrainSmem - kGEnd) / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(smem + kGEnd)[i] = 0u;
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = tmem_base;
  const uint32_t s0 = umma::smem_u32(smem);
  const uint32_t gs = (uint32_t)kGStride;
  uint8_t* mine = smem + kGBase + g * kGStride;   // this thread's group tiles
  Ctl c{&mbar, 0u, true};
  float lsum = 0.0f;
  const int tiles = (n + 255) / 256;
  bool first = true;
  // the next tile's sample (query + target) is loaded one tile ahead, so its
  // scattered read overlaps the current tile's tensor-core work
  float qn[9], yn[3];
  auto fetch = [&](int tile_) {
    const int idx_ = tile_ * 256 + t;
    if (tile_ < tiles && idx_ < n) {
      const int src_ = sample_source(idx_, pop, draw, seed);
#pragma unroll
      for (int j = 0; j < 9; j++) qn[j] = __ldg(q9 + (size_t)src_ * 9 + j);
#pragma unroll
      for (int j = 0; j < 3; j++) yn[j] = __ldg(y3 + (size_t)src_ * 3 + j);
    }
  };
  fetch(cb);
  for (int tile = cb; tile < tiles && c.ok; tile += tk.ctas) {
    const int idx = tile * 256 + t;
    float q[9], yv[3];
#pragma unroll
    for (int j = 0; j < 9; j++) q[j] = qn[j];
#pragma unroll
    for (int j = 0; j < 3; j++) yv[j] = yn[j];
    fetch(tile + tk.ctas);
    stage_query(mine + kGA0, r, q, idx < n, extent);
    publish();
    float o[kOutPad];
    uint64_t mask[3];
    forward_tile<2, true>(smem, tbase, c, kGBase + kGA0, kGBase + kGA1, kGBase + kGA2, kGBase + kGA3, kGStride, o, mask);
    // loss gradient dL/do (rows of padding samples are zero)
    float gy[kOutPad];
#pragma unroll
    for (int j = 0; j < kOutPad; j++) {
      float gv = 0.0f;
      if (idx < n && j < kOut) {
        const float d = o[j] - yv[j];
        const float den = o[j] * o[j] + 0.01f;
        gv = 2.0f * d / den;
        lsum += d * d / den;
      }
      gy[j] = gv;
    }
    store_row(mine + kGDY, r, kOutPad, gy);
    publish();
    const uint32_t A[4] = {s0 + kGBase + kGA0, s0 + kGBase + kGA1, s0 + kGBase + kGA2, s0 + kGBase + kGA3};
    const uint32_t DY = s0 + kGBase + kGDY;
    // layer 3: dW3 += A3^T dO ; dX3 = dO W3^T
    if (t == 0) {
      issue_dw(tbase + kTW3, A[3], kHid, DY, kOutPad, !first);
      issue_dw(tbase + kTW3, A[3] + gs, kHid, DY + gs, kOutPad, true);
      for (int q = 0; q < 2; q++) issue_dx(tbase + kTFwd + 64u * q, DY + q * gs, kOutPad, s0 + kWf3, kHid);
    }
    sync_mma(c);
    const uint32_t wf[3] = {kWf1, kWf2, kWf3};
    const uint32_t tw[3] = {kTW0, kTW1, kTW2};
#pragma unroll
    for (int l = 2; l >= 0; l--) {
      // dH_{l+1} = dX_{l+1} * relu'(h_{l+1}) -> the group's dY tile (C = 64)
      float dx[kHid];
      tmem_row<kHid>(tbase, kTFwd + 64u * (uint32_t)g, dx);
#pragma unroll
      for (int j = 0; j < kHid; j++)
        if (!((mask[l] >> j) & 1ull)) dx[j] = 0.0f;
      store_row(mine + kGDY, r, kHid, dx);
      publish();
      if (t == 0) {
        // dW_l += A_l^T dH_{l+1}   (A_0 has 80 columns);  dX_l = dH_{l+1} W_l^T
        const int cx = l == 0 ? kIn : kHid;
        issue_dw(tbase + tw[l], A[l], cx, DY, kHid, !first);
        issue_dw(tbase + tw[l], A[l] + gs, cx, DY + gs, kHid, true);
        if (l > 0)
          for (int q = 0; q < 2; q++) issue_dx(tbase + kTFwd + 64u * q, DY + q * gs, kHid, s0 + wf[l - 1], kHid);
      }
      sync_mma(c);
    }
    first = false;
  }
  // partial gradients of this CTA: TMEM lane = input feature row, columns = outputs
  float* pc = tk.partial + (size_t)cb * kParams;
  if (c.ok) {
    const int kin[4] = {kIn, kHid, kHid, kHid};
    const int nout[4] = {kHid, kHid, kHid, kOutPad};
    const int off[4] = {kOff0, kOff1, kOff2, kOff3};
    const uint32_t twa[4] = {kTW0, kTW1, kTW2, kTW3};
#pragma unroll
    for (int l = 0; l < 4; l++) {
      float row[kHid];
      if (l < 3) tmem_row<kHid>(tbase, twa[l], row);
      else tmem_row<kOutPad>(tbase, twa[l], row);
      // both groups read the same TMEM lanes; group g stores half of the row's
      // columns, 16 bytes at a time (row offsets are multiples of 4 floats)
      if (r < kin[l]) {
        const int half = (l < 3 ? kHid : kOutPad) / 2;   // a constant once the layer loop is unrolled
        float4* dst = reinterpret_cast<float4*>(pc + off[l] + r * nout[l] + g * half);
#pragma unroll
        for (int j = 0; j < kHid / 2; j += 4) {
          if (j < half) {
            const float4 lo = make_float4(row[j], row[j + 1], row[j + 2], row[j + 3]);
            const float4 hi = make_float4(row[half + j], row[half + j + 1], row[half + j + 2], row[half + j + 3]);
            dst[j / 4] = first ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : (g ? hi : lo);
          }
        }
      }
    }
  }
  // loss of this CTA
  for (int o2 = 16; o2 > 0; o2 >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o2);
  if ((t & 31) == 0) s_loss[warp] = lsum;
  __syncthreads();
  if (t == 0) {
    float a = 0.0f;
    for (int i = 0; i < 8; i++) a += s_loss[i];
    tk.loss[cb] = a;
    if (!c.ok) atomicExch(tk.err, 1);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tbase, 512);
}

// grad[i] = sum over the task's CTAs of partial[cta][i] / n, in two stages
// with a fixed order (deterministic): k_mlp_reduce sums each run of
// kReduceRows partial rows into the run's first row (blockIdx.y = run,
// blockIdx.z = task); k_mlp_reduce_final sums the runs' first rows in order
// and scales by 1/n (blockIdx.y = task).  Thread 0 of the final stage
// advances the task's Adam step counter when the step has samples.
constexpr int kReduceRows = 16;

__global__ void k_mlp_reduce(const __grid_constant__ MlpTaskSet ts) {
  const MlpTask& tk = ts.t[blockIdx.z];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int c0 = blockIdx.y * kReduceRows;
  if (i >= mlp::kParams || c0 >= tk.ctas) return;
  const int c1 = min(c0 + kReduceRows, tk.ctas);
  float s = 0.0f;
  for (int c = c0; c < c1; c++) s += tk.partial[(size_t)c * mlp::kParams + i];
  tk.partial[(size_t)c0 * mlp::kParams + i] = s;
}

__global__ void k_mlp_reduce_final(const __grid_constant__ MlpTaskSet ts) {
  const MlpTask& tk = ts.t[blockIdx.y];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= mlp::kParams) return;
  int n, pop;
  bool draw;
  mlp::sample_counts(tk.n_max, tk.n_dev, tk.pop_cap, n, pop, draw);
  const float inv_n = n > 0 ? 1.0f / (float)n : 0.0f;
  if (i == 0 && tk.step && n > 0) *tk.step += 1;
  float s = 0.0f;
  for (int c = 0; c < tk.ctas; c += kReduceRows) s += tk.partial[(size_t)c * mlp::kParams + i];
  tk.grad[i] = s * inv_n;
}

// Adam on fp32 masters (step number *step, bias corrections from it); writes
// the bf16 copy.  Output columns >= 3 stay 0.  Skipped when the step had no
// samples.  blockIdx.y = task.
__global__ void k_mlp_adam(const __grid_constant__ MlpTaskSet ts, float b1, float b2, float eps) {
  const MlpTask& tk = ts.t[blockIdx.y];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= mlp::kParams) return;
  if (tk.n_dev && *tk.n_dev <= 0) return;
  float* __restrict__ wm = tk.wm;
  uint16_t* __restrict__ wb = tk.wbw;
  if (i >= mlp::kOff3 && ((i - mlp::kOff3) % mlp::kOutPad) >= mlp::kOut) {
    wm[i] = 0.0f;
    wb[mlp::image_index(i)] = 0;
    return;
  }
  const float t = (float)*tk.step;
  const float bc1 = 1.0f - powf(b1, t), bc2 = 1.0f - powf(b2, t);
  const float g = tk.grad[i];
  const float mi = b1 * tk.m[i] + (1.0f - b1) * g;
  const float vi = b2 * tk.v[i] + (1.0f - b2) * g * g;
  tk.m[i] = mi;
  tk.v[i] = vi;
  const float mh = mi / bc1, vh = vi / bc2;
  const float w = wm[i] - tk.lr * mh / (sqrtf(vh) + eps);
  wm[i] = w;
  wb[mlp::image_index(i)] = mlp::f2bf(w);
}

__global__ void k_mlp_to_bf16(const float* __restrict__ wm, uint16_t* __restrict__ wb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < mlp::kParams) wb[mlp::image_index(i)] = mlp::f2bf(wm[i]);
}


// ---------------------------------------------------------------------------
// launch wrappers
// ---------------------------------------------------------------------------
int mlp_num_params() { return mlp::kParams; }

static int sm_count_mlp() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 1;
}

int mlp_max_ctas() { return sm_count_mlp(); }

cudaError_t mlp_encode(const float* q9, int n, float extent, uint16_t* out, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_mlp_encode<<<(n + 127) / 128, 128, 0, st>>>(q9, n, extent, out);
  return cudaGetLastError();
}

// Splits `total` CTAs over the tasks in proportion to their work (at least
// one each, at most one per tile) and sets cta0/ctas; returns the grid.
static int task_work(const MlpTask& t) {
  const int w = (t.n_dev && t.pop_cap > 0) ? std::min(t.n_max, t.pop_cap) : t.n_max;
  return std::max(w, 1);
}

static int assign_ctas(MlpTaskSet& ts, int total, int tile_samples) {
  double work = 0.0;
  for (int k = 0; k < ts.n; k++) work += (double)task_work(ts.t[k]);
  int next = 0;
  for (int k = 0; k < ts.n; k++) {
    const int tiles = std::max(1, (task_work(ts.t[k]) + tile_samples - 1) / tile_samples);
    int c = (int)((double)total * (double)task_work(ts.t[k]) / work);
    c = std::max(1, std::min(c, tiles));
    ts.t[k].cta0 = next;
    ts.t[k].ctas = c;
    next += c;
  }
  return next;
}

cudaError_t mlp_infer_tasks(MlpTaskSet& ts, cudaStream_t st) {
  if (ts.n <= 0) return cudaSuccess;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, mlp::kInferSmem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const int grid = assign_ctas(ts, sm_count_mlp() * 2, 512);   // 2 x 108 KB of shared memory per SM
  k_mlp_infer<<<grid, 256, mlp::kInferSmem, st>>>(ts);
  return cudaGetLastError();
}

cudaError_t mlp_gradient_tasks(MlpTaskSet& ts, cudaStream_t st) {
  if (ts.n <= 0) return cudaSuccess;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, mlp::kTrainSmem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  // partial buffers hold mlp_max_ctas() rows per network
  const int grid = assign_ctas(ts, sm_count_mlp(), 256);
  k_mlp_grad<<<grid, 256, mlp::kTrainSmem, st>>>(ts);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int runs = (sm_count_mlp() + kReduceRows - 1) / kReduceRows;   // partial rows per network: one per CTA
  k_mlp_reduce<<<dim3((mlp::kParams + 255) / 256, runs, ts.n), 256, 0, st>>>(ts);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_mlp_reduce_final<<<dim3((mlp::kParams + 255) / 256, ts.n), 256, 0, st>>>(ts);
  return cudaGetLastError();
}

cudaError_t mlp_adam_tasks(const MlpTaskSet& ts, cudaStream_t st) {
  if (ts.n <= 0) return cudaSuccess;
  k_mlp_adam<<<dim3((mlp::kParams + 255) / 256, ts.n), 256, 0, st>>>(ts, 0.9f, 0.99f, 1e-8f);
  return cudaGetLastError();
}

cudaError_t mlp_to_bf16(const float* wm, uint16_t* wb, cudaStream_t st) {
  k_mlp_to_bf16<<<(mlp::kParams + 255) / 256, 256, 0, st>>>(wm, wb);
  return cudaGetLastError();
}

}  // namespace vrt

using namespace vrt;

// Diagnostic of the tensor-core operand layouts (see k_umma_selftest).
// The failure path of the bounded waits: an mbarrier that nothing arrives on,
// waited on for `spins` try_wait rounds, with a TMEM allocation held across
// the wait as the MLP kernels hold one.  The wait runs out, the kernel sets
// the error flag, frees TMEM and returns.
__global__ void __launch_bounds__(128) k_wait_selftest(uint32_t spins, int* __restrict__ err) {
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_base;
  const int t = threadIdx.x, warp = t >> 5;
  if (warp == 0) umma::tmem_alloc(&tmem_base, 32);
  if (t == 0) umma::mbar_init(&mbar, 1);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const bool ok = __syncthreads_and(umma::mbar_wait(&mbar, 0, spins) ? 1 : 0) != 0;
  if (!ok && t == 0) atomicExch(err, 1);
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_free(tmem_base, 32);
}

extern "C" int vrt_selftest_bounded_wait(unsigned int spins) {
  if (spins == 0 || spins > (1u << 20)) return set_error(VRT_ERR_INVALID, "vrt_selftest_bounded_wait: spins out of range");
  int* d = nullptr;
  cudaError_t e = cudaMalloc(&d, 4);
  if (e != cudaSuccess) return set_error(VRT_ERR_OOM, cudaGetErrorString(e));
  e = cudaMemset(d, 0, 4);
  if (e == cudaSuccess) {
    k_wait_selftest<<<1, 128>>>(spins, d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  int h = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&h, d, 4, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return set_error(VRT_ERR_CUDA, cudaGetErrorString(e));
  if (h) return set_error(VRT_ERR_TIMEOUT, "vrt_selftest_bounded_wait: the wait ran out (expected)");
  return VRT_OK;
}

extern "C" int vrt_mlp_selftest_gemm(int mode, int K, int N, const uint16_t* A, const uint16_t* B, float* D) {
  if (!A || !B || !D || mode < 0 || mode > 2 || N < 16 || N > 64 || N % 16 || K < 16 || K > 128 || K % 16)
    return set_error(VRT_ERR_INVALID, "vrt_mlp_selftest_gemm: bad argument");
  const size_t na = (size_t)128 * K, nb = mode == 1 ? (size_t)128 * N : (size_t)N * K;
  const size_t nd = (size_t)128 * N;
  void* buf = nullptr;
  cudaError_t e = cudaMalloc(&buf, (na + nb) * 2 + nd * 4 + 16);
  if (e != cudaSuccess) return set_error(VRT_ERR_OOM, cudaGetErrorString(e));
  uint16_t* dA = (uint16_t*)buf;
  uint16_t* dB = dA + na;
  float* dD = (float*)(dB + nb);
  int* dErr = (int*)(dD + nd);
  e = cudaMemcpy(dA, A, na * 2, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dB, B, nb * 2, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(dD, 0, nd * 4 + 16);
  const int smem = 72 * 1024;
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_umma_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess) {
    k_umma_selftest<<<1, 128, smem>>>(mode, K, N, dA, dB, dD, dErr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  int herr = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&herr, dErr, 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(D, dD, nd * 4, cudaMemcpyDeviceToHost);
  cudaFree(buf);
  if (e != cudaSuccess) return set_error(VRT_ERR_CUDA, cudaGetErrorString(e));
  if (herr) return set_error(VRT_ERR_TIMEOUT, "vrt_mlp_selftest_gemm: tensor-core completion wait ran out");
  return VRT_OK;
}
