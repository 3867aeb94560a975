// k_trace.cu -- path-trace pass and the DDA parity entry (sm_100a).
//
// k_pathtrace is the plain branch of pathtrace.wgsl (lines 248-330): one
// thread per pixel, 16x16-pixel blocks whose warps cover 8x4 pixel tiles so
// primary rays of a warp stay coherent.  The brick occupancy bitmap (one bit
// per 8^3 brick, 4 KB at 256^3, 32 KB at 512^3) is staged once per block in
// shared memory; brick masks and voxels are read through the read-only path
// (L1/L2 resident: 2 MB + 64 MB at 256^3 fit the 126 MB L2).
#include "trace_kernel.cuh"

namespace vrt {

// One pixel of the plain path (pathtrace.wgsl:248-330).
VRT_DI void path_pixel(const DScene& S, const uint32_t* occ, const Uni& u, float fclamp, uint32_t gx, uint32_t gy,
                       uint32_t W, uint32_t H, float4& rad, uint32_t& alb, float4& gb, DCount& cnt) {
  uint32_t rng = init_rng(gx, gy, u.params0[0]);
  const float jx = rand_(rng) - 0.5f;
  const float jy = rand_(rng) - 0.5f;
  const float uvx = (((float)gx + 0.5f) + jx) / (float)W;
  const float uvy = (((float)gy + 0.5f) + jy) / (float)H;
  const F3 ro = f3(u.camPos[0], u.camPos[1], u.camPos[2]);
  F3 rd = camera_ray(u, uvx, uvy);

  const DHit h0 = trace<true>(S, occ, ro, rd, 1e4f, cnt);
  if (h0.t < 0.0f) {
    const F3 sky = sky_color(u, rd, true);
    rad = make_float4(sky.x, sky.y, sky.z, 1.0f);
    alb = 0xffffffffu;
    gb = make_float4(-rd.x, -rd.y, -rd.z, -1.0f);
    return;
  }
  const Mat mat1 = unpack_material(h0.mat);
  const F3 x1 = ro + rd * h0.t;
  const F3 n1 = h0.n;
  alb = unorm8_(__fsqrt_rn(mat1.albedo.x)) | (unorm8_(__fsqrt_rn(mat1.albedo.y)) << 8) |
        (unorm8_(__fsqrt_rn(mat1.albedo.z)) << 16) | (255u << 24);
  gb = make_float4(n1.x, n1.y, n1.z, h0.t);

  F3 radiance = f3(0.0f, 0.0f, 0.0f);
  F3 tp = f3(1.0f, 1.0f, 1.0f);
  F3 pos = x1, n = n1;
  Mat mat = mat1;
  const uint32_t nB = u.params0[1];
  const F3 sunRad = f3(u.sunRadiance[0], u.sunRadiance[1], u.sunRadiance[2]);
  for (uint32_t bounce = 0; bounce <= nB; bounce++) {
    if (mat.emissive > 0.0f) radiance = radiance + (tp * mat.albedo) * (mat.emissive * kEmissiveScale);
    const F3 surf = pos + n * 1e-3f;
    const F3 l = sample_sun_dir(u, rng);
    const float ndl = dot3(n, l);
    if (ndl > 0.0f && l.y > 0.0f) {
      const DHit hs = trace<true>(S, occ, surf, l, 1e4f, cnt);
      if (!(hs.t >= 0.0f)) radiance = radiance + (((tp * mat.albedo) * kInvPi) * ndl) * sunRad;
    }
    if (bounce == nB) break;
    rd = cosine_hemisphere(n, rng);
    tp = tp * mat.albedo;
    if (bounce >= 2u) {
      const float p = clamp_(fmax_(tp.x, fmax_(tp.y, tp.z)), 0.05f, 0.95f);
      if (rand_(rng) > p) break;
      tp = f3(tp.x / p, tp.y / p, tp.z / p);
    }
    const DHit h = trace<true>(S, occ, surf, rd, 1e4f, cnt);
    if (h.t < 0.0f) {
      radiance = radiance + tp * sky_color(u, rd, false);
      break;
    }
    pos = surf + rd * h.t;
    n = h.n;
    mat = unpack_material(h.mat);
  }
  if (!(fclamp <= 0.0f)) radiance = min3(radiance, f3(fclamp, fclamp, fclamp));
  const F3 den = max3(mat1.albedo, f3(1e-3f, 1e-3f, 1e-3f));
  rad = make_float4(radiance.x / den.x, radiance.y / den.y, radiance.z / den.z, 1.0f);
}

template <bool kSmem>
__global__ void __launch_bounds__(256) k_pathtrace(DScene S, Uni u, float fclamp, int W, int H, PathOut out) {
  extern __shared__ uint32_t s_occ[];
  const uint32_t* occ = stage_occupancy<kSmem>(S, s_occ);
  int gx, gy;
  block_pixel_16x16(gx, gy);
  DCount cnt{0u, 0u, 0u, 0u};
  uint32_t pix = 0;
  if (gx < W && gy < H) {
    float4 rad, gb;
    uint32_t alb;
    path_pixel(S, occ, u, fclamp, (uint32_t)gx, (uint32_t)gy, (uint32_t)W, (uint32_t)H, rad, alb, gb, cnt);
    const size_t p = (size_t)gy * W + gx;
    reinterpret_cast<uint2*>(out.rad16)[p] = pack_h4(rad.x, rad.y, rad.z, rad.w);
    if (out.rad32) reinterpret_cast<float4*>(out.rad32)[p] = rad;
    out.alb8[p] = alb;
    reinterpret_cast<float4*>(out.gbuf)[p] = gb;
    pix = 1;
  }
  if (out.stats) block_flush_stats(out.stats, cnt, pix);
}

template <bool kSmem>
__global__ void __launch_bounds__(256) k_trace_rays(DScene S, const float* __restrict__ o, const float* __restrict__ d,
                                                    const float* __restrict__ tmax, int n, VrtHit* __restrict__ out) {
  extern __shared__ uint32_t s_occ[];
  const uint32_t* occ = stage_occupancy<kSmem>(S, s_occ);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  DCount cnt{0u, 0u, 0u, 0u};
  const F3 ro = f3(o[3 * i], o[3 * i + 1], o[3 * i + 2]);
  const F3 rd = f3(d[3 * i], d[3 * i + 1], d[3 * i + 2]);
  const DHit h = trace<true>(S, occ, ro, rd, tmax[i], cnt);
  VrtHit r;
  r.t = h.t; r.n[0] = h.n.x; r.n[1] = h.n.y; r.n[2] = h.n.z; r.mat = h.mat;
  r.voxel[0] = h.vx; r.voxel[1] = h.vy; r.voxel[2] = h.vz;
  r.face = h.t >= 0.0f ? face_of(h.n) : -1;
  r.steps = cnt.outer + cnt.inner;
  r.bytes = 4u * (cnt.outer + cnt.inner + cnt.vreads);
  r.pad = 0u;
  out[i] = r;
}

cudaError_t launch_pathtrace(const SceneDev& s, const VrtUniforms& u, float fclamp, int W, int H,
                             const PathOut& out, cudaStream_t st) {
  const size_t smem = occ_words(s.BG) * sizeof(uint32_t);
  dim3 grid((W + 15) / 16, (H + 15) / 16);
  if (smem <= kMaxSmemOccBytes) {
    if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(k_pathtrace<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
    }
    k_pathtrace<true><<<grid, 256, smem, st>>>(to_dscene(s), to_uni(u), fclamp, W, H, out);
  } else {
    k_pathtrace<false><<<grid, 256, 0, st>>>(to_dscene(s), to_uni(u), fclamp, W, H, out);
  }
  return cudaGetLastError();
}

cudaError_t launch_trace_rays(const SceneDev& s, const float* o, const float* d, const float* tmax, int n,
                              VrtHit* out, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const size_t smem = occ_words(s.BG) * sizeof(uint32_t);
  const int blocks = (n + 255) / 256;
  if (smem <= kMaxSmemOccBytes) {
    if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(k_trace_rays<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
    }
    k_trace_rays<true><<<blocks, 256, smem, st>>>(to_dscene(s), o, d, tmax, n, out);
  } else {
    k_trace_rays<false><<<blocks, 256, 0, st>>>(to_dscene(s), o, d, tmax, n, out);
  }
  return cudaGetLastError();
}

}  // namespace vrt
