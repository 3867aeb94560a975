// k_vb.cu -- the VoxelBench technique adapter's estimator (no counterpart in
// the browser renderer; VoxelBench/pipeline/technique.h:8-14 is the interface
// it serves).
//
// VoxelBench techniques estimate the INDIRECT radiance L_ind = alb/pi * E_ind
// of every G-buffer pixel of the harness (core.h:118-141) under a per-frame ray
// budget, in VoxelBench's own lighting model: a delta sun of irradiance sunE,
// a two-colour sky gradient, emissive voxel faces with RGB emission
// (core.h:85-116, core.cpp:143-171).  This kernel runs the estimator of the
// harness's baseline technique (techniques/pt.h:24-68: NEE paths of up to 8
// bounces with Russian roulette from the second, an exponential history and an
// edge-aware 5x5 filter) on the two-level DDA of this library over the
// harness's grid, converted to the packed-u32 layout (material id in the low
// byte).  Coordinates stay in voxel units; the DDA works in metres, so rays are
// scaled by 1/16 (exact) on the way in and hit distances by 16 on the way out.
// Random numbers follow the harness's stateless SplitMix64 streams, one per
// (pixel, frame), so the estimator is the harness's in distribution; the
// traversal is this library's (float arithmetic, 8^3 bricks), so single paths
// can part ways with the CPU's at grazing ties.
#include "trace_kernel.cuh"

namespace vrt {

constexpr int kVbMaxMat = 16;

struct VbDev {
  DScene S;
  int nx, ny, nz;          // the harness's grid (embedded at the origin of the N^3 grid)
  int W, H;
  const float4* px;        // 3 per pixel: (pos, depth), (n, flags), (alb, 0); flags bit0 hit, bit1 emissive
  float4* hist;            // xyz history, w sample count
  float4* out;             // indirect radiance
  const int4* em;          // emissive faces: (x, y, z, face | material << 8)
  int nem;
  float3 alb[kVbMaxMat], emi[kVbMaxMat];
  int sky;                 // SKY.enabled
  float3 sunDir, sunE, zenith, horizon;
  unsigned long long* rays;
};

// VoxelBench's stateless RNG (core.h:48-58): a SplitMix64 stream seeded from
// (a, b, c).
struct VbRng {
  uint64_t s;
  VRT_DI VbRng(uint64_t a, uint64_t b, uint64_t c) {
    s = a * 0x9E3779B97F4A7C15ull ^ (b + 0xBF58476D1CE4E5B9ull) * 0x94D049BB133111EBull ^ c * 0xD6E8FEB86659FD93ull;
    next();
    next();
  }
  VRT_DI uint64_t next() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  VRT_DI uint32_t u32() { return (uint32_t)(next() >> 32); }
  VRT_DI float uf() { return (float)(u32() >> 8) * (1.0f / 16777216.0f); }
};

VRT_DI F3 v3(float3 a) { return f3(a.x, a.y, a.z); }
VRT_DI F3 vb_norm(F3 a) {
  const float l = __fsqrt_rn(dot3(a, a));
  return a * (1.0f / (l + 1e-20f));
}
VRT_DI F3 face_n(int f) {   // FN[] (core.h:98): +x, -x, +y, -y, +z, -z
  const float s = (f & 1) ? -1.0f : 1.0f;
  return f3(f >> 1 == 0 ? s : 0.0f, f >> 1 == 1 ? s : 0.0f, f >> 1 == 2 ? s : 0.0f);
}
VRT_DI F3 face_point(int vx, int vy, int vz, int f) {   // core.h:111-113
  return (f3((float)vx, (float)vy, (float)vz) + f3(0.5f, 0.5f, 0.5f)) + face_n(f) * 0.501f;
}
VRT_DI bool vb_emissive(const VbDev& D, int m) {
  const F3 e = v3(D.emi[m]);
  return (e.x + e.y) + e.z > 0.0f;
}
VRT_DI F3 sky_l(const VbDev& D, F3 d) {   // SkyLight::skyL (core.h:89-94)
  if (!D.sky) return f3(0.0f, 0.0f, 0.0f);
  const float t = __fsqrt_rn(fmax_(0.0f, d.y));
  return v3(D.horizon) * (1.0f - t) + v3(D.zenith) * t;
}

struct VbHit {
  bool hit;
  int vx, vy, vz, face, m;
  float t;   // voxel units
};

// One traversal in voxel units on this library's DDA (metres inside).  As
// the harness's trace (core.cpp:52-56), an origin outside its grid is a miss.
VRT_DI VbHit vb_trace(const VbDev& D, const uint32_t* occ, F3 o, F3 d, float tmax, uint32_t& nrays) {
  nrays++;
  const int ox = (int)floorf(o.x), oy = (int)floorf(o.y), oz = (int)floorf(o.z);
  if (ox < 0 || oy < 0 || oz < 0 || ox >= D.nx || oy >= D.ny || oz >= D.nz) {
    VbHit miss;
    miss.hit = false;
    miss.vx = miss.vy = miss.vz = miss.face = -1;
    miss.m = 0;
    miss.t = -1.0f;
    return miss;
  }
  DCount c{0u, 0u, 0u, 0u};
  const DHit h = trace<false>(D.S, occ, o * (1.0f / 16.0f), d, tmax * (1.0f / 16.0f), c);
  VbHit r;
  r.hit = h.t >= 0.0f;
  r.vx = h.vx; r.vy = h.vy; r.vz = h.vz;
  r.face = r.hit ? face_of(h.n) : -1;
  r.m = (int)(h.mat & 0xffu);
  r.t = h.t * 16.0f;
  return r;
}

// cosDir (core.h:103-110)
VRT_DI F3 cos_dir(F3 n, VbRng& rng) {
  const float u1 = rng.uf(), u2 = rng.uf();
  const float r = __fsqrt_rn(u1), phi = 6.2831853f * u2;
  const float lx = r * cosf(phi), ly = r * sinf(phi), lz = __fsqrt_rn(fmax_(0.0f, 1.0f - u1));
  F3 tu = fabsf(n.x) > 0.5f ? f3(0.0f, 1.0f, 0.0f) : f3(1.0f, 0.0f, 0.0f);
  const F3 tv = vb_norm(cross3(n, tu));
  tu = cross3(tv, n);
  return vb_norm((tu * lx + tv * ly) + n * lz);
}

// neeIrr (core.cpp:143-171): one emissive-face sample and the sun, <= 2 rays.
VRT_DI F3 nee_irr(const VbDev& D, const uint32_t* occ, F3 p, F3 n, VbRng& rng, uint32_t& nrays) {
  F3 acc = f3(0.0f, 0.0f, 0.0f);
  if (D.nem > 0) {
    const int i = (int)(rng.u32() % (uint32_t)D.nem);
    const int4 e = D.em[i];
    const int ef = e.w & 0xff, em = e.w >> 8;
    const F3 fn = face_n(ef);
    F3 q = face_point(e.x, e.y, e.z, ef);
    const F3 tu = fabsf(fn.x) > 0.5f ? f3(0.0f, 1.0f, 0.0f) : f3(1.0f, 0.0f, 0.0f);
    const F3 tv = cross3(fn, tu);
    const float j0 = rng.uf() - 0.5f;
    const float j1 = rng.uf() - 0.5f;
    q = q + (tu * j0 + tv * j1);
    F3 w = q - p;
    const float d2 = dot3(w, w), d = __fsqrt_rn(d2);
    w = w * (1.0f / d);
    const float cs = dot3(w, n), cl = -dot3(w, fn);
    if (cs > 0.0f && cl > 0.0f) {
      const VbHit h = vb_trace(D, occ, p, w, d + 1.0f, nrays);
      if (h.hit && vb_emissive(D, h.m) && h.t >= d - 0.87f) {
        const float pdfA = 1.0f / (float)D.nem;
        acc = acc + v3(D.emi[em]) * ((cs * cl) / (d2 * pdfA + 1e-9f));
      }
    }
  }
  const F3 sE = v3(D.sunE);
  if (D.sky && (sE.x + sE.y) + sE.z > 0.0f) {
    const F3 sd = v3(D.sunDir);
    const float cs = dot3(sd, n);
    if (cs > 0.0f && !vb_trace(D, occ, p, sd, 1e9f, nrays).hit) acc = acc + sE * cs;
  }
  return acc;
}

// One frame of MethodPT's estimator per pixel (techniques/pt.h:24-52).
template <bool kSmem>
__global__ void __launch_bounds__(128) k_vb_paths(const __grid_constant__ VbDev D, uint32_t fcount, int basePaths,
                                                  double fracP, int stride) {
  extern __shared__ uint32_t s_occ[];
  const uint32_t* occ = stage_occupancy<kSmem>(D.S, s_occ);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t nrays = 0u;
  if (i < D.W * D.H) {
    const float4 p0 = D.px[3 * i], p1 = D.px[3 * i + 1];
    const uint32_t flags = __float_as_uint(p1.w);
    const bool live = (flags & 1u) && !(flags & 2u) && !(stride > 1 && ((uint32_t)i + fcount) % (uint32_t)stride != 0u);
    if (live) {
      VbRng rng((uint64_t)i, (uint64_t)fcount, 101ull);
      const int paths = basePaths + ((double)rng.uf() < fracP ? 1 : 0);
      F3 E = f3(0.0f, 0.0f, 0.0f);
      for (int s = 0; s < paths; s++) {
        F3 p = f3(p0.x, p0.y, p0.z), nn = f3(p1.x, p1.y, p1.z), tp = f3(1.0f, 1.0f, 1.0f);
        F3 acc = f3(0.0f, 0.0f, 0.0f);
        for (int b = 0; b < 8; b++) {
          const F3 d = cos_dir(nn, rng);
          const VbHit h = vb_trace(D, occ, p, d, 1e9f, nrays);
          if (!h.hit) {
            acc = acc + tp * (sky_l(D, d) * 3.14159265f);
            break;
          }
          if (vb_emissive(D, h.m)) break;
          const F3 hp = face_point(h.vx, h.vy, h.vz, h.face);
          const F3 hn = face_n(h.face);
          tp = tp * v3(D.alb[h.m]);
          acc = acc + tp * nee_irr(D, occ, hp, hn, rng, nrays);
          if (b >= 1) {
            const float rr = 0.7f;
            if (rng.uf() >= rr) break;
            tp = tp * (1.0f / rr);
          }
          p = hp;
          nn = hn;
        }
        E = E + acc;
      }
      E = E * (1.0f / (float)paths);
      float4 hs = D.hist[i];
      const float a = hs.w < 1.0f ? 1.0f : 0.15f;
      const F3 hv = f3(hs.x, hs.y, hs.z) * (1.0f - a) + E * a;
      D.hist[i] = make_float4(hv.x, hv.y, hv.z, hs.w + 1.0f);
    }
  }
  const uint32_t r = __reduce_add_sync(0xffffffffu, nrays);
  if ((threadIdx.x & 31) == 0 && r) atomicAdd(D.rays, (unsigned long long)r);
}

// The edge-aware 5x5 filter and the remodulation (techniques/pt.h:54-68).
__global__ void __launch_bounds__(256) k_vb_filter(const __grid_constant__ VbDev D) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= D.W * D.H) return;
  const int x = i % D.W, y = i / D.W;
  const float4 g0 = D.px[3 * i], g1 = D.px[3 * i + 1], g2 = D.px[3 * i + 2];
  const float4 hi = D.hist[i];
  if (!(__float_as_uint(g1.w) & 1u)) {
    D.out[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    return;
  }
  F3 acc = f3(0.0f, 0.0f, 0.0f);
  float ws = 0.0f;
  for (int dy = -2; dy <= 2; dy++)
    for (int dx = -2; dx <= 2; dx++) {
      const int xx = x + dx, yy = y + dy;
      if (xx < 0 || xx >= D.W || yy < 0 || yy >= D.H) continue;
      const int j = yy * D.W + xx;
      const float4 q0 = D.px[3 * j], q1 = D.px[3 * j + 1];
      if (!(__float_as_uint(q1.w) & 1u)) continue;
      if (dot3(f3(q1.x, q1.y, q1.z), f3(g1.x, g1.y, g1.z)) < 0.9f) continue;
      if (fabsf(q0.w - g0.w) > 2.5f) continue;
      const float w = expf(-(float)(dx * dx + dy * dy) / 4.5f);
      const float4 hj = D.hist[j];
      acc = acc + f3(hj.x, hj.y, hj.z) * w;
      ws = ws + w;
    }
  const F3 f = ws > 0.0f ? acc * (1.0f / ws) : f3(hi.x, hi.y, hi.z);
  const F3 o = f3(g2.x, g2.y, g2.z) * (f * (1.0f / 3.14159265f));
  D.out[i] = make_float4(o.x, o.y, o.z, 0.0f);
}

cudaError_t launch_vb_frame(const VbLaunch& L, cudaStream_t st) {
  VbDev D;
  D.S = to_dscene(L.scene);
  D.nx = L.nx;
  D.ny = L.ny;
  D.nz = L.nz;
  D.W = L.W;
  D.H = L.H;
  D.px = (const float4*)L.px;
  D.hist = (float4*)L.hist;
  D.out = (float4*)L.out;
  D.em = (const int4*)L.emitters;
  D.nem = L.n_emitters;
  for (int m = 0; m < kVbMaxMat; m++) {
    D.alb[m] = make_float3(L.albedo[m][0], L.albedo[m][1], L.albedo[m][2]);
    D.emi[m] = make_float3(L.emission[m][0], L.emission[m][1], L.emission[m][2]);
  }
  D.sky = L.sky;
  D.sunDir = make_float3(L.sun_dir[0], L.sun_dir[1], L.sun_dir[2]);
  D.sunE = make_float3(L.sun_e[0], L.sun_e[1], L.sun_e[2]);
  D.zenith = make_float3(L.zenith[0], L.zenith[1], L.zenith[2]);
  D.horizon = make_float3(L.horizon[0], L.horizon[1], L.horizon[2]);
  D.rays = L.rays;
  const int P = L.W * L.H;
  const size_t smem = occ_words(L.scene.BG) * sizeof(uint32_t);
  if (smem <= kMaxSmemOccBytes) {
    if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(k_vb_paths<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
    }
    k_vb_paths<true><<<(P + 127) / 128, 128, smem, st>>>(D, L.fcount, L.base_paths, L.frac_p, L.stride);
  } else {
    k_vb_paths<false><<<(P + 127) / 128, 128, 0, st>>>(D, L.fcount, L.base_paths, L.frac_p, L.stride);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_vb_filter<<<(P + 255) / 256, 256, 0, st>>>(D);
  return cudaGetLastError();
}

}  // namespace vrt
