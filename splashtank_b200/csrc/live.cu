// live.cu - what the viewer and the bake take from the solver besides the water frame, packed on the device:
//  * the live view (dispPack, src/flip/sim.js:381-404: subsample, sprayDisp, deepPick, packDisp,
//    src/flip/wgsl-solver.js:141-147 and src/flip/wgsl-whitewater.js:196-297), in the WGSL's f32 arithmetic;
//  * a frame's whitewater part (packSprayFrame with packSprayJS, src/flip/bake.js:4-15, 43-58) and deep-water part
//    (readDeep + packDeep, src/flip/sim.js:408-421, src/gpu.js:512-524), in the JavaScript double arithmetic.
// The reference compacts the whitewater sample and the deep points with atomic counters in arbitrary order; here both
// keep ascending order (sampled slot, then tile-major cell), numbered by block scans.
#include <algorithm>

#include "common.cuh"
#include "jsnum.cuh"
#include "kernels.h"

namespace st {

// ---- JavaScript Math.min / Math.max (NaN in, NaN out) ----
__device__ __forceinline__ double jsMin(double a, double b) { return (a != a || b != b) ? __longlong_as_double(0x7ff8000000000000ll) : fmin(a, b); }
__device__ __forceinline__ double jsMax(double a, double b) { return (a != a || b != b) ? __longlong_as_double(0x7ff8000000000000ll) : fmax(a, b); }

// packSprayJS (src/flip/bake.js:4-15): top bit whitewater, two bits of kind, 8 bits of speed in quarter units, then for
// spray and mist an octahedral direction (10 + 10 bits), for foam and bubbles the life left (10 bits). Math.hypot is the
// square root of the sum of squares (ECMAScript leaves its last bit to the engine).
__device__ uint32_t packSprayJS(double vx, double vy, double vz, double kindRounded, double lifeFrac) {
  const int32_t kind = toInt32(kindRounded);
  const double s = sqrt(vx * vx + vy * vy + vz * vz);
  uint32_t code = 0x80000000u | ((uint32_t)toInt32(jsMin(floor(s * 4.0), 255.0)) << 21);
  const uint32_t kbits[4] = {0u, 0x40000000u, 0x20000000u, 0x60000000u};
  code |= kbits[kind & 3];
  if (kind >= 2) {
    const double lf = (lifeFrac == lifeFrac && lifeFrac != 0.0) ? lifeFrac : 0.0;   // lifeFrac || 0
    return code | (uint32_t)toInt32(jsRound(jsMax(0.0, jsMin(1.0, lf)) * 1023.0));
  }
  double nx = 0.0, ny = 1.0, nz = 0.0;
  if (s > 1e-6) { nx = vx / s; ny = vy / s; nz = vz / s; }
  const double l = fabs(nx) + fabs(ny) + fabs(nz);
  double px = nx / l, py = ny / l;
  if (nz < 0.0) {
    const double qx = (1.0 - fabs(py)) * (px >= 0.0 ? 1.0 : -1.0), qy = (1.0 - fabs(px)) * (py >= 0.0 ? 1.0 : -1.0);
    px = qx;
    py = qy;
  }
  const double u = jsMax(0.0, jsMin(1023.0, jsRound((px * 0.5 + 0.5) * 1023.0)));
  const double w = jsMax(0.0, jsMin(1023.0, jsRound((py * 0.5 + 0.5) * 1023.0)));
  return code | ((uint32_t)toInt32(w) << 10) | (uint32_t)toInt32(u);
}

// packSpray (src/flip/wgsl-whitewater.js:183-193), the same code in the shader's f32 arithmetic (round: ties to even)
__device__ uint32_t packSprayF(V3 v, uint32_t kind, float lifeFrac) {
  const float s = len3(v);
  uint32_t code = 0x80000000u | (min(u32f(s * 4.0f), 255u) << 21);
  if (kind == 1u) code |= 0x40000000u;
  else if (kind == 2u) code |= 0x20000000u;
  else if (kind == 3u) code |= 0x60000000u;
  if (kind >= 2u) return code | u32f(clampf(lifeFrac, 0.0f, 1.0f) * 1023.0f);
  V3 n = v3(0.0f, 1.0f, 0.0f);
  if (s > 1e-6f) n = v / s;
  const float l = fabsf(n.x) + fabsf(n.y) + fabsf(n.z);
  float px = n.x / l, py = n.y / l;
  if (n.z < 0.0f) {
    const float qx = (1.0f - fabsf(py)) * (px >= 0.0f ? 1.0f : -1.0f), qy = (1.0f - fabsf(px)) * (py >= 0.0f ? 1.0f : -1.0f);
    px = qx;
    py = qy;
  }
  const uint32_t u = u32f(clampf(rintf((px * 0.5f + 0.5f) * 1023.0f), 0.0f, 1023.0f));
  const uint32_t w = u32f(clampf(rintf((py * 0.5f + 0.5f) * 1023.0f), 0.0f, 1023.0f));
  return code | (w << 10) | u;
}
// q16 of packDisp (src/flip/wgsl-whitewater.js:202), f32
__device__ __forceinline__ uint16_t q16f(float v, float lo, float k) { return (uint16_t)u32f(clampf(rintf((v - lo) * k), 0.0f, 65535.0f)); }

// ---- one-CTA exclusive scan of n counts in place (n capped by *ndev when given); *total receives the sum ----
__global__ void __launch_bounds__(1024) k_scan_u32(uint32_t* a, uint32_t n, const uint32_t* ndev, uint32_t* total) {
  __shared__ uint32_t sm[33];
  if (ndev) n = min(n, *ndev);
  uint32_t carry = 0;
  for (uint32_t c0 = 0; c0 < n; c0 += blockDim.x) {
    const uint32_t i = c0 + threadIdx.x;
    const uint32_t v = i < n ? a[i] : 0u;
    uint32_t tot;
    const uint32_t ex = blockExclusive(v, sm, &tot);
    if (i < n) a[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) *total = carry;
}

// ---- packSprayFrame: alive slots, then every step-th slot's alive points in slot order ----
__global__ void k_sf_alive(const float4* __restrict__ sPos, uint32_t nslots, uint32_t* alive) {
  uint32_t c = 0;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nslots; j += gridDim.x * blockDim.x) c += sPos[j].w > 0.0f ? 1u : 0u;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(alive, c);
}
// pass 0: per-block counts of sampled living slots; pass 1: write them (blk holds the scanned offsets)
__global__ void __launch_bounds__(256) k_sf_pick(const float4* __restrict__ sPos, const float4* __restrict__ sVel, uint32_t nslots,
                                                 uint32_t step, uint32_t nsample, int pass, uint32_t* blk, FrameBox F, double foamLife,
                                                 uint16_t* __restrict__ pos16, uint32_t* __restrict__ pk) {
  __shared__ uint32_t sm[33];
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t j = (uint64_t)t * step;
  const bool pick = t < nsample && j < nslots && sPos[j].w > 0.0f;
  if (pass == 0) {
    const uint32_t c = __syncthreads_count(pick);
    if (threadIdx.x == 0) blk[blockIdx.x] = c;
    return;
  }
  const uint32_t k = blk[blockIdx.x] + blockExclusive(pick ? 1u : 0u, sm, nullptr);
  if (!pick) return;
  const float4 p = sPos[j], v = sVel[j];
  pos16[3 * (size_t)k] = q16((double)p.x, F.x0, F.kx);
  pos16[3 * (size_t)k + 1] = q16((double)p.y, F.y0, F.ky);
  pos16[3 * (size_t)k + 2] = q16((double)p.z, F.z0, F.kz);
  pk[k] = packSprayJS((double)v.x, (double)v.y, (double)v.z, jsRound((double)v.w), (double)p.w / foamLife);
}

// ---- deepPick (src/flip/wgsl-whitewater.js:284-295): fluid cells with no particles (narrow band deep water) ----
// Above DEEPMAX such cells (counted by the previous pass, prev) a fixed hashed sample of them is kept.
constexpr uint32_t DEEPMAX = 200000u;
__device__ __forceinline__ bool deepCell(const FlipParams& P, const Bufs& B, uint32_t t, uint32_t local, uint32_t prev, bool& counted) {
  int i, j, k;
  tileCoord(P, t, local, i, j, k);
  const uint32_t c = t * 512u + local;
  counted = inDom(P, i, j, k) && (B.ctype[c] & 0xffu) == 1u && B.cnt[c] <= 0;
  if (!counted) return false;
  return !(prev > DEEPMAX && hash1(c * 2654435761u + 7u) * (float)prev >= (float)DEEPMAX);
}
// pass 0: per active tile, picked cells into tcount and all deep cells into *seen; pass 1: write the picked points
__global__ void __launch_bounds__(512) k_deep(Bufs B, uint32_t prev, int pass, uint32_t* tcount, uint32_t* seen, float4* __restrict__ out) {
  __shared__ FlipParams P;
  __shared__ uint32_t sm[33];
  loadParams(P, B.P);
  const uint32_t nA = B.ctl->nActive;
  for (uint32_t a = blockIdx.x; a < nA; a += gridDim.x) {
    const uint32_t t = B.active[a];
    bool counted;
    const bool pick = deepCell(P, B, t, threadIdx.x, prev, counted);
    if (pass == 0) {
      const uint32_t nc = __syncthreads_count(counted), np = __syncthreads_count(pick);
      if (threadIdx.x == 0) {
        tcount[a] = np;
        if (nc) atomicAdd(seen, nc);
      }
      continue;
    }
    const uint32_t k = tcount[a] + blockExclusive(pick ? 1u : 0u, sm, nullptr);
    if (pick && k < DEEPMAX) {
      int i, j, kk;
      tileCoord(P, t, threadIdx.x, i, j, kk);
      const V3 x = cellCenter(P, i, j, kk);
      out[k] = make_float4(x.x, x.y, x.z, 4096.0f + fmn(len3(velGVec(P, B.velG, B.ncell, x)), 63.0f));
    }
  }
}
// packDeep (src/gpu.js:512-524): positions and speed bytes of the deep points, JavaScript doubles
__global__ void k_pack_deep(const float4* __restrict__ dp, uint32_t n, FrameBox F, uint16_t* __restrict__ pos16, uint8_t* __restrict__ spd) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 p = dp[i];
    pos16[3 * (size_t)i] = q16((double)p.x, F.x0, F.kx);
    pos16[3 * (size_t)i + 1] = q16((double)p.y, F.y0, F.ky);
    pos16[3 * (size_t)i + 2] = q16((double)p.z, F.z0, F.kz);
    const double s = ((double)p.w - 4096.0) * F.ks;
    spd[i] = s > 191.0 ? (uint8_t)191 : toU8(jsMax(0.0, s));
  }
}

// ---- the packed live view (packDisp, src/flip/wgsl-whitewater.js:207-253) ----
// water: every stride-th particle of the storage order (subsample) or the first nW (straight from pos)
__global__ void k_live_water(const Part* __restrict__ pa, uint32_t nW, uint32_t stride, LiveBox K, uint32_t* __restrict__ out) {
  uint16_t* p16 = reinterpret_cast<uint16_t*>(out + K.oWp);
  uint8_t* s8 = reinterpret_cast<uint8_t*>(out + K.oWs);
  uint8_t* f8 = reinterpret_cast<uint8_t*>(out + K.oWf);
  const uint32_t n4 = ((nW + 3u) / 4u) * 4u;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += gridDim.x * blockDim.x) {
    float4 v = make_float4(0.0f, -1.0e6f, 0.0f, 0.0f);
    if (i < nW) v = pa[(size_t)i * stride].p;
    uint16_t q[3] = {0, 0, 0};
    uint32_t s = 255u, f = 0u;
    if (v.y > DEADY) {
      q[0] = q16f(v.x, K.x0, K.kx); q[1] = q16f(v.y, K.y0, K.ky); q[2] = q16f(v.z, K.z0, K.kz);
      const float lv = floorf(v.w / 64.0f);
      s = u32f(clampf((v.w - lv * 64.0f) * 16.0f * K.vs, 0.0f, 191.0f));
      f = u32f(clampf(lv, 0.0f, 15.0f)) * 17u;
    }
    p16[3 * (size_t)i] = q[0]; p16[3 * (size_t)i + 1] = q[1]; p16[3 * (size_t)i + 2] = q[2];
    s8[i] = (uint8_t)s;
    f8[i] = (uint8_t)f;
  }
}
// whitewater (sprayDisp): every stride-th slot handed out, the living ones in slot order; pass 0 counts per block
__global__ void __launch_bounds__(256) k_live_spray(Bufs B, uint32_t sdMax, float foamLife, int pass, uint32_t* blk, LiveBox K,
                                                    uint32_t* __restrict__ out) {
  __shared__ uint32_t sm[33];
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t used = min(B.ctl->sctl0, K.smax), stride = max(1u, (used + sdMax - 1u) / sdMax);
  const uint64_t j = (uint64_t)k * stride;
  const bool pick = k < sdMax && j < used && B.sPos[j].w > 0.0f;
  if (pass == 0) {
    const uint32_t c = __syncthreads_count(pick);
    if (threadIdx.x == 0) blk[blockIdx.x] = c;
    return;
  }
  const uint32_t o = blk[blockIdx.x] + blockExclusive(pick ? 1u : 0u, sm, nullptr);
  if (!pick || o >= K.nS) return;
  const float4 p = B.sPos[j], v = B.sVel[j];
  uint16_t* p16 = reinterpret_cast<uint16_t*>(out + K.oSp);
  p16[3 * (size_t)o] = q16f(p.x, K.x0, K.kx);
  p16[3 * (size_t)o + 1] = q16f(p.y, K.y0, K.ky);
  p16[3 * (size_t)o + 2] = q16f(p.z, K.z0, K.kz);
  out[K.oSk + o] = packSprayF(xyz(v), u32f(v.w + 0.5f), p.w / fmx(foamLife, 0.01f));
}
// deep water points into the live view
__global__ void k_live_deep(const float4* __restrict__ dp, uint32_t n, LiveBox K, uint32_t* __restrict__ out) {
  uint16_t* p16 = reinterpret_cast<uint16_t*>(out + K.oDp);
  uint8_t* s8 = reinterpret_cast<uint8_t*>(out + K.oDs);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 v = dp[i];
    if (!(v.y > DEADY)) continue;
    p16[3 * (size_t)i] = q16f(v.x, K.x0, K.kx); p16[3 * (size_t)i + 1] = q16f(v.y, K.y0, K.ky); p16[3 * (size_t)i + 2] = q16f(v.z, K.z0, K.kz);
    s8[i] = (uint8_t)u32f(clampf((v.w - 4096.0f) * 16.0f * K.vs, 0.0f, 191.0f));
  }
}

// ---- launchers ----
int launch_spray_frame(const float4* sPos, const float4* sVel, uint32_t nslots, uint32_t maxPoints, const FrameBox& F, double foamLife,
                       uint32_t* scratch, uint16_t* pos16, uint32_t* pk, uint32_t* counts, cudaStream_t s) {
  // counts[0]: alive slots; counts[1]: points written. scratch: one count per block of 256 samples
  cudaMemsetAsync(counts, 0, 8, s);
  k_sf_alive<<<std::max<uint32_t>(1, std::min<uint32_t>((nslots + 255) / 256, 148 * 8)), 256, 0, s>>>(sPos, nslots, counts);
  uint32_t alive = 0;
  cudaMemcpyAsync(&alive, counts, 4, cudaMemcpyDeviceToHost, s);
  cudaStreamSynchronize(s);
  const uint32_t step = std::max<uint32_t>(1u, (uint32_t)std::ceil((double)alive / (double)std::max<uint32_t>(maxPoints, 1)));
  const uint32_t nsample = (uint32_t)(((uint64_t)nslots + step - 1) / step), nb = (nsample + 255) / 256;
  if (!nb) return 2;
  k_sf_pick<<<nb, 256, 0, s>>>(sPos, sVel, nslots, step, nsample, 0, scratch, F, foamLife, pos16, pk);
  k_scan_u32<<<1, 1024, 0, s>>>(scratch, nb, nullptr, counts + 1);
  k_sf_pick<<<nb, 256, 0, s>>>(sPos, sVel, nslots, step, nsample, 1, scratch, F, foamLife, pos16, pk);
  return 5;
}
int launch_deep(const Bufs& B, uint32_t prev, uint32_t nActiveMax, int grid, uint32_t* tcount, uint32_t* counts, float4* out, cudaStream_t s) {
  // counts[0]: deep cells seen; counts[1]: points picked (the first DEEPMAX are written)
  cudaMemsetAsync(counts, 0, 8, s);
  k_deep<<<grid, 512, 0, s>>>(B, prev, 0, tcount, counts, out);
  k_scan_u32<<<1, 1024, 0, s>>>(tcount, nActiveMax, &B.ctl->nActive, counts + 1);
  k_deep<<<grid, 512, 0, s>>>(B, prev, 1, tcount, counts, out);
  return 3;
}
int launch_pack_deep(const float4* dp, uint32_t n, const FrameBox& F, uint16_t* pos16, uint8_t* spd, cudaStream_t s) {
  if (!n) return 0;
  k_pack_deep<<<std::min<uint32_t>((n + 255) / 256, 148 * 8), 256, 0, s>>>(dp, n, F, pos16, spd);
  return 1;
}
int launch_live(const Bufs& B, const LiveBox& K, uint32_t nW, uint32_t stride, uint32_t sdMax, float foamLife, const float4* deep, uint32_t nDeep,
                uint32_t* scratch, uint32_t* out, cudaStream_t s) {
  int nl = 0;
  if (nW) {
    const uint32_t n4 = ((nW + 3u) / 4u) * 4u;
    k_live_water<<<std::min<uint32_t>((n4 + 255) / 256, 148 * 8), 256, 0, s>>>(B.pa, nW, stride, K, out);
    nl++;
  }
  if (K.nS && sdMax) {
    const uint32_t nb = (sdMax + 255) / 256;
    k_live_spray<<<nb, 256, 0, s>>>(B, sdMax, foamLife, 0, scratch, K, out);
    k_scan_u32<<<1, 1024, 0, s>>>(scratch, nb, nullptr, out);   // header word 0: whitewater points
    k_live_spray<<<nb, 256, 0, s>>>(B, sdMax, foamLife, 1, scratch, K, out);
    nl += 3;
  }
  if (nDeep) {
    k_live_deep<<<std::min<uint32_t>((nDeep + 255) / 256, 148 * 8), 256, 0, s>>>(deep, nDeep, K, out);
    nl++;
  }
  return nl;
}

}  // namespace st
