// frames.cu - the particles as a cache frame and the bake's per-frame measurements, on the device.
//
// A frame is what a bake stores per frame and the live view draws (packFrameBuf, src/gpu.js:525-560; the cache layout
// of writeCacheParts, src/shared.js:688-705): in id order, each point's position as 3 x uint16 across the box, a speed
// byte (16ths of the solver's speed times vs, at most 191; 255 = gone) and a white-water byte (level x 17). The
// reference computes it in JavaScript doubles from a float readback; the kernel does the same double arithmetic
// (Math.round is round-half-up, a Uint8Array store truncates), so the bytes are identical, and only 8 bytes per point
// cross PCIe instead of 16.
#include "common.cuh"
#include "jsnum.cuh"
#include "kernels.h"

namespace st {

// meta[0]: last water point + 1 (atomicMax of index + 1), meta[1]: any white water
__global__ void k_pack_frame(const float4* __restrict__ pos4, uint32_t n, FrameBox F, uint16_t* __restrict__ pos16,
                             uint8_t* __restrict__ spd, uint8_t* __restrict__ fm, uint32_t* meta) {
  uint32_t last = 0, foam = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 p = pos4[i];
    const uint32_t wb = __float_as_uint(p.w);
    uint16_t q[3] = {0, 0, 0};
    uint8_t s = 255, f = 0;
    const bool gone = (double)p.y < -1e5;
    const bool other = wb >= 0x80000000u || (double)p.w >= 4096.0;   // whitewater or deep-water codes (live view only)
    if (!gone && !other) {
      q[0] = q16((double)p.x, F.x0, F.kx);
      q[1] = q16((double)p.y, F.y0, F.ky);
      q[2] = q16((double)p.z, F.z0, F.kz);
      const double w = (double)p.w, lv = floor(w / 64.0), sv = (w - lv * 64.0) * F.ks;
      s = sv > 191.0 ? (uint8_t)191 : toU8(sv);
      if (lv != 0.0) { f = toU8(lv * 17.0); foam = 1; }
    }
    if (!((double)p.y <= -1e5) && !other) last = max(last, i + 1);
    pos16[3 * (size_t)i] = q[0];
    pos16[3 * (size_t)i + 1] = q[1];
    pos16[3 * (size_t)i + 2] = q[2];
    spd[i] = s;
    fm[i] = f;
  }
  for (int o = 16; o > 0; o >>= 1) {
    last = max(last, __shfl_xor_sync(0xffffffffu, last, o));
    foam |= __shfl_xor_sync(0xffffffffu, foam, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (last) atomicMax(&meta[0], last);
    if (foam) atomicOr(&meta[1], 1u);
  }
}

// bakeDiag (src/flip/bake.js:60-83) over the particle slots: counts, sums, extremes and a 16-bin height histogram.
// Sums of doubles are reduced in a different order than the reference's loop, so they agree to rounding, not bit for bit.
__device__ __forceinline__ unsigned long long ordKey(double v) {   // doubles in order as unsigned integers
  const unsigned long long u = (unsigned long long)__double_as_longlong(v);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__global__ void k_bake_diag(const Part* __restrict__ pa, uint32_t n, DiagBox D, DiagAcc* acc) {
  __shared__ uint32_t hist[16];
  if (threadIdx.x < 16) hist[threadIdx.x] = 0;
  __syncthreads();
  uint32_t alive = 0, bad = 0, out = 0, capped = 0, foamy = 0;
  double sx = 0, sy = 0, sz = 0, ss = 0, fl = 0, smax = 0;
  unsigned long long mn[3] = {~0ull, ~0ull, ~0ull}, mx[3] = {0, 0, 0};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 p = pa[i].p;
    const double x = p.x, y = p.y, z = p.z, w = p.w;
    if (!(isfinite(x) && isfinite(y) && isfinite(z) && isfinite(w))) { bad++; continue; }
    if (y < -1e5) continue;
    alive++;
    const double lv = floor(w / 64.0), sp = w - lv * 64.0;
    sx += x; sy += y; sz += z; ss += sp; smax = fmax(smax, sp); fl += lv;
    if (lv >= 8.0) foamy++;
    if (sp >= D.cap) capped++;
    const double e = 1e-3;
    if (x < D.x0 - e || x > D.x1 + e || y < D.y0 - e || y > D.y1 + e || z < D.z0 - e || z > D.z1 + e) out++;
    const double c[3] = {x, y, z};
    for (int k = 0; k < 3; k++) { const unsigned long long o = ordKey(c[k]); mn[k] = min(mn[k], o); mx[k] = max(mx[k], o); }
    const double b = floor((y - D.y0) / D.hy);
    atomicAdd(&hist[(int)fmin(15.0, fmax(0.0, b))], 1u);
  }
  for (int o = 16; o > 0; o >>= 1) {
    alive += __shfl_xor_sync(0xffffffffu, alive, o); bad += __shfl_xor_sync(0xffffffffu, bad, o);
    out += __shfl_xor_sync(0xffffffffu, out, o); capped += __shfl_xor_sync(0xffffffffu, capped, o);
    foamy += __shfl_xor_sync(0xffffffffu, foamy, o);
    sx += __shfl_xor_sync(0xffffffffu, sx, o); sy += __shfl_xor_sync(0xffffffffu, sy, o); sz += __shfl_xor_sync(0xffffffffu, sz, o);
    ss += __shfl_xor_sync(0xffffffffu, ss, o); fl += __shfl_xor_sync(0xffffffffu, fl, o);
    smax = fmax(smax, __shfl_xor_sync(0xffffffffu, smax, o));
    for (int k = 0; k < 3; k++) {
      mn[k] = min(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
      mx[k] = max(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
    }
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&acc->count[0], alive); atomicAdd(&acc->count[1], bad); atomicAdd(&acc->count[2], out);
    atomicAdd(&acc->count[3], capped); atomicAdd(&acc->count[4], foamy);
    atomicAdd(&acc->sum[0], sx); atomicAdd(&acc->sum[1], sy); atomicAdd(&acc->sum[2], sz); atomicAdd(&acc->sum[3], ss); atomicAdd(&acc->sum[4], fl);
    atomicMax(&acc->smax, (unsigned long long)__double_as_longlong(smax));   // speeds are not negative
    for (int k = 0; k < 3; k++) { atomicMin(&acc->mn[k], mn[k]); atomicMax(&acc->mx[k], mx[k]); }
  }
  __syncthreads();
  if (threadIdx.x < 16 && hist[threadIdx.x]) atomicAdd(&acc->hist[threadIdx.x], hist[threadIdx.x]);
}

int launch_pack_frame(const float4* pos4, uint32_t n, const FrameBox& F, uint16_t* pos16, uint8_t* spd, uint8_t* fm, uint32_t* meta,
                      cudaStream_t s) {
  if (!n) return 0;
  k_pack_frame<<<std::min<uint32_t>((n + 255) / 256, 148 * 16), 256, 0, s>>>(pos4, n, F, pos16, spd, fm, meta);
  return 1;
}
int launch_bake_diag(const Part* pa, uint32_t n, const DiagBox& D, DiagAcc* acc, cudaStream_t s) {
  if (!n) return 0;
  k_bake_diag<<<std::min<uint32_t>((n + 255) / 256, 148 * 8), 256, 0, s>>>(pa, n, D, acc);
  return 1;
}

}  // namespace st
