// flip_extra.cu - narrow band (src/flip/wgsl-narrowband.js) and whitewater (src/flip/wgsl-whitewater.js) kernels.
//
// Where the reference compacts with atomics in arbitrary order (nbDead, nbDeficit, nbSpawn, sprayEmit), these
// kernels use a fixed order built from block scans: dead slots in ascending storage index, deficit cells in
// ascending cell key, whitewater ring slots in ascending storage index of the emitting particle.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace st {

// ---- phiInitAll (wgsl-narrowband.js:20-35) ----
__global__ void __launch_bounds__(512) k_nb_init(Bufs B) {
  __shared__ FlipParams P;
  loadParams(P, B.P);
  const uint32_t nA = B.ctl->nActive, nc = B.ncell;
  for (uint32_t a = blockIdx.x; a < nA; a += gridDim.x) {
    const uint32_t t = B.active[a], c = t * 512u + threadIdx.x;
    int i, j, k;
    tileCoord(P, t, threadIdx.x, i, j, k);
    float ph = clampf(fillPhi(P, B.waves, B.cols, B.sdf, cellCenter(P, i, j, k)), -7.9f, 7.9f);
    if (ph < 0.0f) ph = fmn(ph, -1.5f);
    if (!inDom(P, i, j, k)) ph = 8.0f;
    const uint32_t ct = B.ctype[c];
    if (P.nbInit == 2u) ph = fmn(ph, phiOfBits(ct));
    B.ctype[c] = phiPutBits(ct, ph);
    if (P.nbInit == 1u) {   // the starting velocity: the waves' under the ocean's surface, else at rest
      for (int ax = 0; ax < 3; ax++) {
        const V3 fp = facePos(P, i, j, k, ax);
        float v = 0.0f;
        if (P.ocean != 0u && fp.y < oceanEta(P, B.waves, fp.x, fp.z)) v = comp3(oceanVel(P, B.waves, fp), ax);
        B.velG[ax * nc + c] = v;
      }
    }
  }
}

// ---- depth passes: nbPhi (wgsl-narrowband.js:38-49), jacNb / nbJacA / nbJacB (:50-68) ----
__device__ __forceinline__ float phiSampleX(const FlipParams& P, const uint32_t* __restrict__ ctype, V3 x) {
  const V3 g = (x - v3(P.x0, P.y0, P.z0)) * P.ih - v3(0.5f, 0.5f, 0.5f);
  const V3 gc = vclamp(g, v3(0.0f, 0.0f, 0.0f), v3((float)P.nx - 1.001f, (float)P.ny - 1.001f, (float)P.nz - 1.001f));
  const V3 f0 = vfloor(gc), fr = gc - f0;
  const int i0 = gidx(f0.x), j0 = gidx(f0.y), k0 = gidx(f0.z);
  float s = 0.0f, ws = 0.0f;
  for (int c = 0; c < 8; c++) {
    const int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
    const float w = (dx == 1 ? fr.x : 1.0f - fr.x) * (dy == 1 ? fr.y : 1.0f - fr.y) * (dz == 1 ? fr.z : 1.0f - fr.z);
    const uint32_t ct = ctype[cellIdx(P, i0 + dx, j0 + dy, k0 + dz)];
    if (((ct >> 8) & 0xffu) != 0u || w <= 0.0f) continue;
    s += w * phiOfBits(ct);
    ws += w;
  }
  if (ws < 1.0e-4f) return 0.5f;
  return s / ws;
}
__global__ void __launch_bounds__(512) k_nb_phi(Bufs B) {
  __shared__ FlipParams P;
  loadParams(P, B.P);
  const uint32_t nA = B.ctl->nActive, nc = B.ncell;
  for (uint32_t a = blockIdx.x; a < nA; a += gridDim.x) {
    const uint32_t t = B.active[a], c = t * 512u + threadIdx.x;
    int i, j, k;
    tileCoord(P, t, threadIdx.x, i, j, k);
    if (!inDom(P, i, j, k)) { B.rhs[c] = 8.0f; continue; }
    if (((B.ctype[c] >> 8) & 0xffu) != 0u) { B.rhs[c] = 0.5f; continue; }
    const V3 x = cellCenter(P, i, j, k);
    const float phA = phiSampleX(P, B.ctype, x - velGVec(P, B.velG, nc, x) * P.dt);
    bool inside = B.cnt[c] > 0 || phA < -1.0f;
    if (P.ocean != 0u && layerW(P, x) >= 0.5f) inside = x.y < oceanEta(P, B.waves, x.x, x.z);   // the ocean's boundary decides
    B.rhs[c] = inside ? clampf(phA, -7.9f, -0.5f) : clampf(phA, 0.5f, 7.9f);
  }
}
__device__ __forceinline__ float jacNb(const FlipParams& P, const Bufs& B, int i, int j, int k, float cur, bool fromRhs) {
  if (!inDom(P, i, j, k)) return 8.0f;
  if (cur >= 0.0f) return cur;
  // the six neighbours' words are loaded together from addresses that are always valid (a neighbour outside the domain
  // reads the cell itself and is skipped below); the maximum then runs in the reference's order
  uint32_t ct[6];
  float rv[6];
  bool in[6];
  const uint32_t self = cellIdx(P, i, j, k);
#pragma unroll
  for (int q = 0; q < 6; q++) {
    int a = i, b = j, c = k;
    if (q == 0) a -= 1; else if (q == 1) a += 1; else if (q == 2) b -= 1; else if (q == 3) b += 1; else if (q == 4) c -= 1; else c += 1;
    in[q] = inDom(P, a, b, c);
    const uint32_t cq = in[q] ? cellIdx(P, a, b, c) : self;
    ct[q] = B.ctype[cq];
    rv[q] = fromRhs ? B.rhs[cq] : 0.0f;
  }
  float m = -8.0f;
#pragma unroll
  for (int q = 0; q < 6; q++) {
    if (!in[q] || ((ct[q] >> 8) & 0xffu) != 0u) continue;
    m = fmx(m, fromRhs ? rv[q] : phiOfBits(ct[q]));
  }
  return clampf(m - 1.0f, -7.9f, -0.5f);
}
// pass A: depth (ctype bits) from rhs; pass B: rhs from depth
__global__ void __launch_bounds__(512) k_nb_jac(Bufs B, int passA) {
  __shared__ FlipParams P;
  loadParams(P, B.P);
  const uint32_t nA = B.ctl->nActive;
  for (uint32_t a = blockIdx.x; a < nA; a += gridDim.x) {
    const uint32_t t = B.active[a], c = t * 512u + threadIdx.x;
    int i, j, k;
    tileCoord(P, t, threadIdx.x, i, j, k);
    if (passA) {
      const float v = jacNb(P, B, i, j, k, B.rhs[c], true);
      B.ctype[c] = phiPutBits(B.ctype[c], v);
    } else {
      B.rhs[c] = jacNb(P, B, i, j, k, phiOfBits(B.ctype[c]), false);
    }
  }
}

// ---- nbVel (wgsl-narrowband.js:70-85): water faces with no particle weight take the carried grid velocity ----
__global__ void __launch_bounds__(512) k_nb_vel(Bufs B) {
  __shared__ FlipParams P;
  loadParams(P, B.P);
  const uint32_t nA = B.ctl->nActive, nc = B.ncell;
  for (uint32_t a = blockIdx.x; a < nA; a += gridDim.x) {
    const uint32_t t = B.active[a], c = t * 512u + threadIdx.x;
    int i, j, k;
    tileCoord(P, t, threadIdx.x, i, j, k);
    if (!inDom(P, i, j, k) || (B.ctype[c] & 0xffu) != 1u) continue;
    // the three lower neighbours' types and the three face weights, loaded together (a neighbour outside the domain
    // reads the cell itself and is skipped)
    uint32_t nt[3];
    int32_t wsum[3];
    bool in[3];
#pragma unroll
    for (int ax = 0; ax < 3; ax++) {
      const int li = ax == 0 ? i - 1 : i, lj = ax == 1 ? j - 1 : j, lk = ax == 2 ? k - 1 : k;
      in[ax] = inDom(P, li, lj, lk);
      nt[ax] = B.ctype[in[ax] ? cellIdx(P, li, lj, lk) : c];
      wsum[ax] = B.acc[(3 + ax) * nc + c];
    }
    for (int ax = 0; ax < 3; ax++) {
      if (!in[ax] || (nt[ax] & 0xffu) != 1u || wsum[ax] > 0) continue;
      const V3 fp = facePos(P, i, j, k, ax);
      const float vc = velGAxis(P, B.velG, nc, fp - velGVec(P, B.velG, nc, fp) * P.dt, ax);
      B.acc[ax * nc + c] = (int32_t)rintf(vc * P.scale);
      B.acc[(3 + ax) * nc + c] = (int32_t)P.scale;
    }
  }
}

// ---- refill: nbDead (wgsl-narrowband.js:106-110), nbDeficit (:112-130), nbSpawn (:134-148); nbKill is in g2p ----
// which: 0 particles killed per tile, 1 deficit (cells and need per tile), 2 whitewater points per tile
__global__ void __launch_bounds__(1024) k_scan_x(Bufs B, int which) {
  __shared__ uint32_t sm[33];
  const uint32_t nA = B.ctl->nActive;
  if (which == 0) scanOne(B.tileDead, nA, &B.ctl->nKilled, sm);
  else if (which == 1) {
    if (blockIdx.x == 0) scanOne(B.tileAux, nA, &B.ctl->defCount, sm);
    else scanOne(B.tileAux2, nA, &B.ctl->defNeed, sm);
  } else scanOne(B.tileEmit, nA, &B.ctl->emitTried, sm);
}
// the dead slots, in ascending storage index: this step's kills inside the tiles' segments (listed here), then the slots
// that were already dead when the step sorted them ([nLive, N), no list needed)
__global__ void __launch_bounds__(512) k_killed_list(Bufs B) {
  __shared__ FlipParams P;
  __shared__ uint32_t sm[33];
  loadParams(P, B.P);
  const uint32_t nA = B.ctl->nActive;
  __shared__ uint32_t walk[2];
  TileWalk w{B.ctl, walk};
  for (uint32_t a = w.begin(); a < nA; a = w.next()) {
    w.fetch();
    if (B.tileDead[a + 1] == B.tileDead[a]) continue;   // uniform per block: no kills in this tile
    const uint32_t s0 = B.tileCnt[a], s1 = B.tileCnt[a + 1];
    uint32_t base = B.tileDead[a];
    for (uint32_t c0 = s0; c0 < s1; c0 += blockDim.x) {
      const uint32_t i = c0 + threadIdx.x;
      const bool d = i < s1 && B.deadF[i];
      uint32_t tot;
      const uint32_t r = blockExclusive(d ? 1u : 0u, sm, &tot);
      if (d && base + r < P.lcap) B.deadList[base + r] = i;
      base += tot;
    }
  }
  w.done();
}
__device__ __forceinline__ uint32_t deadSlot(const Bufs& B, uint32_t k, uint32_t nKilled, uint32_t nLive) {
  return k < nKilled ? B.deadList[k] : nLive + (k - nKilled);
}
// the deficit test of one cell; returns the particles it asks for (0: none)
__device__ __forceinline__ uint32_t deficitNeed(const FlipParams& P, const Bufs& B, uint32_t c, int i, int j, int k) {
  if (!inDom(P, i, j, k)) return 0;
  const uint32_t ct = B.ctype[c];
  if (((ct >> 8) & 0xffu) != 0u) return 0;
  const float ph = phiOfBits(ct);
  const V3 cx = cellCenter(P, i, j, k);
  const float lw = layerW(P, cx);
  if (lw > 0.25f && lw < 0.5f) {   // the inner half of the ocean's boundary is full below the ocean's surface
    if (cx.y > oceanEta(P, B.waves, cx.x, cx.z) - 0.25f * P.h || ph < -P.band) return 0;
  } else {
    if ((ct & 0xffu) != 1u || ph > -1.0f || ph < -P.band) return 0;
  }
  // the count test before the calm test (both only ever return 0, so the order is free): a full cell skips the
  // 24-corner velocity sample
  const uint32_t n = (uint32_t)max(B.cnt[c], 0);
  if ((float)n >= 0.55f * P.rest) return 0;
  if (!(lw > 0.25f && lw < 0.5f) && !(len3(velGVec(P, B.velG, B.ncell, cx)) < 9.0f * P.h)) return 0;
  return min((uint32_t)rintf(0.85f * P.rest) - n, 64u);
}
// three CTAs per SM (40 registers, a short spill): the deficit test's dependent loads overlap more (0.284 -> 0.266 ms
// for the reseed stage at 256^3)
__global__ void __launch_bounds__(512, 3) k_def_count(Bufs B) {
  __shared__ FlipParams P;
  __shared__ uint32_t sm[33];
  loadParams(P, B.P);
  const uint32_t nA = B.ctl->nActive;
  __shared__ uint32_t walk[2];
  TileWalk w{B.ctl, walk};
  for (uint32_t a = w.begin(); a < nA; a = w.next()) {
    w.fetch();
    const uint32_t t = B.active[a], c = t * 512u + threadIdx.x;
    int i, j, k;
    tileCoord(P, t, threadIdx.x, i, j, k);
    const uint32_t nd = deficitNeed(P, B, c, i, j, k);
    // one scan of two 16-bit fields: cells asking (at most 512) and particles asked for (at most 64 a cell)
    uint32_t tot;
    blockExclusive((nd ? 1u : 0u) | (nd << 16), sm, &tot);
    if (threadIdx.x == 0) { B.tileAux[a] = tot & 0xffffu; B.tileAux2[a] = tot >> 16; }
  }
  w.done();
}
__global__ void __launch_bounds__(512) k_spawn(Bufs B) {
  __shared__ FlipParams P;
  __shared__ uint32_t sm[33];
  loadParams(P, B.P);
  const uint32_t nA = B.ctl->nActive, nc = B.ncell;
  const uint32_t nKilled = B.ctl->nKilled, nLive = B.ctl->nLive;
  const uint32_t avail = min(nKilled + (P.n - nLive), P.lcap);
  __shared__ uint32_t walk[2];
  TileWalk w{B.ctl, walk};
  for (uint32_t a = w.begin(); a < nA; a = w.next()) {
    w.fetch();
    if (B.tileAux2[a + 1] == B.tileAux2[a]) continue;   // no cell of this tile asks (the whole CTA skips it)
    const uint32_t t = B.active[a], c = t * 512u + threadIdx.x;
    int i, j, k;
    tileCoord(P, t, threadIdx.x, i, j, k);
    const uint32_t nd = deficitNeed(P, B, c, i, j, k);
    const uint32_t ex = blockExclusive((nd ? 1u : 0u) | (nd << 16), sm, nullptr);
    const uint32_t e = B.tileAux[a] + (ex & 0xffffu), base = B.tileAux2[a] + (ex >> 16);
    if (!nd || e >= P.lcap / 2u) continue;
    const V3 cp = v3((float)i, (float)j, (float)k);
    for (uint32_t m = 0; m < nd; m++) {
      const uint32_t kk = base + m;
      if (kk >= avail) break;
      const uint32_t pi = deadSlot(B, kk, nKilled, nLive);
      const uint32_t hh = (e * 9781u + m * 6271u + 17u) ^ (P.seed * 2654435761u);
      const V3 x = v3(P.x0, P.y0, P.z0) + (cp + v3(hash1(hh + 1u), hash1(hh + 2u), hash1(hh + 3u))) * P.h;
      const V3 v = layerW(P, x) > 0.25f ? oceanVel(P, B.waves, x) : velGVec(P, B.velG, nc, x);
      Part q;
      q.p = make_float4(x.x, x.y, x.z, fmn(len3(v), 63.0f));
      q.v = make_float4(v.x, v.y, v.z, 0.0f);
      B.pa[pi] = q;
    }
  }
  w.done();
}

// ---- whitewater: wetCell / wetAt (wgsl-whitewater.js:7-23) ----
// the per-cell values are computed once a step by the divergence pass (0 for tiles without storage)
__device__ __forceinline__ float wetCell(const FlipParams& P, const Bufs& B, int i, int j, int k) { return wetCellAt(P, B.wet, i, j, k); }
__device__ __forceinline__ float wetAt(const FlipParams& P, const Bufs& B, V3 p) {
  const V3 g = (p - v3(P.x0, P.y0, P.z0)) * P.ih - v3(0.5f, 0.5f, 0.5f);
  const V3 f0 = vfloor(g), fr = g - f0;
  const int i0 = gidx(f0.x), j0 = gidx(f0.y), k0 = gidx(f0.z);
  float s = 0.0f;
  for (int c = 0; c < 8; c++) {
    const int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
    const float w = (dx == 1 ? fr.x : 1.0f - fr.x) * (dy == 1 ? fr.y : 1.0f - fr.y) * (dz == 1 ? fr.z : 1.0f - fr.z);
    if (w > 0.0f) s += w * wetCell(P, B, i0 + dx, j0 + dy, k0 + dz);
  }
  return s;
}
// ---- air field (wgsl-whitewater.js:24-89): a coarse grid of air velocity at cell centres (cells P.airH wide from the
// box's low corner) that water near the surface and flying spray drag along; spray and mist drift with it ----
// WGSL i32(f32): truncation towards zero, saturating at the ends of the range; NaN gives 0
__device__ __forceinline__ int32_t i32f(float f) {
  if (!(f == f)) return 0;
  if (f >= 2147483648.0f) return 2147483647;
  if (f <= -2147483648.0f) return (int32_t)0x80000000u;
  return (int32_t)f;
}
__device__ __forceinline__ uint32_t airIdx(const FlipParams& P, int x, int y, int z) {   // airIdx (:25-28)
  const int qx = clampi(x, 0, (int)P.aNx - 1), qy = clampi(y, 0, (int)P.aNy - 1), qz = clampi(z, 0, (int)P.aNz - 1);
  return (uint32_t)qx + P.aNx * ((uint32_t)qy + P.aNy * (uint32_t)qz);
}
__device__ __forceinline__ V3 airAt(const FlipParams& P, const float4* __restrict__ air, V3 p) {   // airAt (:30-40)
  const V3 g = (p - v3(P.x0, P.y0, P.z0)) / P.airH - v3(0.5f, 0.5f, 0.5f);
  const V3 f0 = vfloor(g), fr = g - f0;
  const int i0 = gidx(f0.x), j0 = gidx(f0.y), k0 = gidx(f0.z);
  V3 s = v3(0.0f, 0.0f, 0.0f);
  for (int c = 0; c < 8; c++) {
    const int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
    const float w = (dx == 1 ? fr.x : 1.0f - fr.x) * (dy == 1 ? fr.y : 1.0f - fr.y) * (dz == 1 ? fr.z : 1.0f - fr.z);
    s = s + xyz(__ldg(&air[airIdx(P, i0 + dx, j0 + dy, k0 + dz)])) * w;
  }
  return s;
}
// airPush (:41-45) for a warp at once: the lanes that push into the same air cell add their fixed-point values first
// (integer sums, so the result does not depend on the order), and one lane per cell does the atomics
__device__ __forceinline__ void airPushWarp(const FlipParams& P, int32_t* __restrict__ acc, bool valid, V3 p, V3 v, float w) {
  uint32_t key = 0xffffffffu, q0 = 0, q1 = 0, q2 = 0, q3 = 0;
  if (valid) {
    const V3 g = vfloor((p - v3(P.x0, P.y0, P.z0)) / P.airH);
    key = airIdx(P, gidx(g.x), gidx(g.y), gidx(g.z));
    q0 = (uint32_t)i32f(v.x * w * 256.0f);
    q1 = (uint32_t)i32f(v.y * w * 256.0f);
    q2 = (uint32_t)i32f(v.z * w * 256.0f);
    q3 = (uint32_t)i32f(w * 256.0f);
  }
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t pend = __ballot_sync(0xffffffffu, valid);
  while (pend) {
    const int lead = __ffs(pend) - 1;
    const uint32_t k = __shfl_sync(0xffffffffu, key, lead);
    const bool mine = valid && key == k;
    const uint32_t grp = __ballot_sync(0xffffffffu, mine);
    const uint32_t s0 = __reduce_add_sync(0xffffffffu, mine ? q0 : 0u), s1 = __reduce_add_sync(0xffffffffu, mine ? q1 : 0u);
    const uint32_t s2 = __reduce_add_sync(0xffffffffu, mine ? q2 : 0u), s3 = __reduce_add_sync(0xffffffffu, mine ? q3 : 0u);
    if (lane == (uint32_t)lead) {
      uint32_t* a = reinterpret_cast<uint32_t*>(acc) + 4ull * k;
      atomicAdd(a, s0); atomicAdd(a + 1, s1); atomicAdd(a + 2, s2); atomicAdd(a + 3, s3);
    }
    pend &= ~grp;
  }
}
// airSplatW (:51-57) over the live particles, then airSplatS (:59-64) over the whitewater slots handed out, in one
// launch. g2p held back the narrow band trim of particles that throw off no points (their kill belongs to the
// reseed stage, after the air has felt them); they are removed here once pushed.
__global__ void __launch_bounds__(256) k_air_splat(Bufs B) {
  __shared__ FlipParams P;
  loadParams(P, B.P);
  const uint32_t nL = B.ctl->nLive, m = min(B.ctl->sctl0, P.smax), tot = nL + m;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); i0 < tot; i0 += stride) {
    const uint32_t i = i0 + (threadIdx.x & 31u);
    bool valid = false;
    V3 p = v3(0.0f, 0.0f, 0.0f), v = p;
    float w = 1.0f;
    if (i < nL) {
      const Part q = B.pa[i];
      p = xyz(q.p);
      v = xyz(q.v);
      valid = !(q.p.y < DEADY);
      if (valid) {
        int ci, cj, ck;
        particleCell(P, p, ci, cj, ck);
        if (B.on[tileOf(P, ci, cj, ck)] && (float)B.cnt[cellIdx(P, ci, cj, ck)] > 0.85f * P.rest) valid = false;
        const uint8_t ek = B.emitK[i];
        if ((ek & EMIT_KILL) && (ek & 7u) == 0u) {
          Part d;
          d.p = make_float4(0.0f, -1.0e6f, 0.0f, 0.0f);
          d.v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
          B.pa[i] = d;
        }
      }
    } else if (i < tot) {
      const uint32_t j = i - nL;
      const float4 sp = B.sPos[j], sv = B.sVel[j];
      p = xyz(sp);
      v = xyz(sv);
      w = 0.25f;
      valid = !(sp.w <= 0.0f) && !(sv.w > 1.5f);
    }
    airPushWarp(P, B.airAcc, valid, p, v, w);
  }
}
// airUpdate (:67-86): blur towards the six neighbours, pull towards what pushed the cell, take the velocity of an
// object the cell is inside, settle back to the wind
__global__ void __launch_bounds__(256) k_air_update(Bufs B) {
  __shared__ FlipParams P;
  loadParams(P, B.P);
  const uint32_t nax = P.aNx, nay = P.aNy, na = nax * nay * P.aNz;
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < na; c += gridDim.x * blockDim.x) {
    const int ci = (int)(c % nax), cj = (int)((c / nax) % nay), ck = (int)(c / (nax * nay));
    V3 a = xyz(B.air[c]);
    const V3 nb = (xyz(B.air[airIdx(P, ci + 1, cj, ck)]) + xyz(B.air[airIdx(P, ci - 1, cj, ck)]) + xyz(B.air[airIdx(P, ci, cj + 1, ck)]) +
                   xyz(B.air[airIdx(P, ci, cj - 1, ck)]) + xyz(B.air[airIdx(P, ci, cj, ck + 1)]) + xyz(B.air[airIdx(P, ci, cj, ck - 1)])) / 6.0f;
    a = vmix(a, nb, P.airBlur);
    const int4 ac = reinterpret_cast<const int4*>(B.airAcc)[c];
    const float w = (float)ac.w / 256.0f;
    if (w > 0.0f) {
      const V3 vt = v3((float)ac.x, (float)ac.y, (float)ac.z) / (w * 256.0f);
      a = vmix(a, vt, 1.0f - st_expf(-P.airCouple * fmn(w, 8.0f) * P.dt));
    }
    const V3 x = v3(P.x0, P.y0, P.z0) + (v3((float)ci, (float)cj, (float)ck) + v3(0.5f, 0.5f, 0.5f)) * P.airH;
    for (uint32_t k = 0; k < P.ncols; k++) {
      if (!colNear(P, B.cols, k, x)) continue;
      float phi;
      V3 wn;
      sdfEval(B.cols, B.sdf, k, x, phi, wn);
      if (phi < 0.6f * P.airH) { a = colSurfVel(B.cols, k, x); break; }
    }
    a = vmix(a, v3(P.q1, P.q2, P.q3), 1.0f - st_expf(-P.airDecay * P.dt));
    B.air2[c] = make_float4(a.x, a.y, a.z, 0.0f);
  }
}
__global__ void __launch_bounds__(256) k_air_copy(Bufs B, uint32_t na) {   // airCopy (:88)
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < na; c += gridDim.x * blockDim.x) B.air[c] = B.air2[c];
}

// wwSample (wgsl-whitewater.js:91-98) fused with sprayStep (:134-179): each point reads only its own sample
__global__ void __launch_bounds__(256) k_ww_step(Bufs B) {
  __shared__ FlipParams P;
  loadParams(P, B.P);
  const uint32_t m = min(B.ctl->sctl0, P.smax), nc = B.ncell;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
    float4 sp = B.sPos[j];
    if (sp.w <= 0.0f) continue;
    const V3 p = xyz(sp);
    // sample: water velocity (vn) and wetness
    V3 vf = v3(0.0f, 0.0f, 0.0f);
    int ci, cj, ck;
    particleCell(P, p, ci, cj, ck);
    if (B.on[tileOf(P, ci, cj, ck)]) {
      float r[3];
      for (int axis = 0; axis < 3; axis++) {
        V3 g = (p - v3(P.x0, P.y0, P.z0)) * P.ih;
        if (axis == 0) { g.y -= 0.5f; g.z -= 0.5f; } else if (axis == 1) { g.x -= 0.5f; g.z -= 0.5f; } else { g.x -= 0.5f; g.y -= 0.5f; }
        const V3 f0 = vfloor(g), fr = g - f0;
        const int i0 = gidx(f0.x), j0 = gidx(f0.y), k0 = gidx(f0.z);
        float sn = 0.0f;
        for (int c = 0; c < 8; c++) {
          const int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
          const float w = (dx == 1 ? fr.x : 1.0f - fr.x) * (dy == 1 ? fr.y : 1.0f - fr.y) * (dz == 1 ? fr.z : 1.0f - fr.z);
          sn += w * B.vn[axis * nc + faceCell(P, axis, i0 + dx, j0 + dy, k0 + dz)];
        }
        r[axis] = sn;
      }
      vf = v3(r[0], r[1], r[2]);
    }
    const float wet = wetAt(P, B, p);
    // step
    float4 sv = B.sVel[j];
    V3 v = xyz(sv);
    const float kw = sv.w;
    uint32_t kind = u32f(kw + 0.5f);
    float tk = (kw - (float)kind) / 0.4f * WWHOLD;
    const bool settled = tk >= WWHOLD * 0.999f;
    const uint32_t k0 = kind;
    float life = sp.w;
    const uint32_t h0 = j * 2654435761u + P.seed * 974711u;
    if (kind == 0u && v.y < vf.y && wet > 0.55f && tk > 0.05f) { kind = 2u; life = P.wwFoamLife * (0.6f + 0.8f * hash1(h0)); v = vf; }
    else if (kind == 1u && wet > 0.55f) { life = 0.0f; }
    else if (kind == 2u && wet > 0.97f && settled) { kind = 3u; }
    else if (kind == 2u && wet < 0.04f && settled) { kind = 0u; life = fmn(life, P.sprLife); }
    else if (kind == 3u && wet < 0.6f && settled) { kind = 2u; life = fmx(life, 0.5f * P.wwFoamLife); }
    if (kind != k0) tk = 0.0f; else tk = fmn(tk + P.dt, WWHOLD);
    if (kind <= 1u) {
      const bool mist = kind == 1u;
      V3 gust = v3(0.0f, 0.0f, 0.0f);
      if (P.q7 > 0.0f) {
        const V3 gp = p * 0.55f * P.vs;
        const float tt = P.q8 * 0.6f;
        gust = v3(vnz(gp + v3(tt, 0.0f, 0.0f)), vnz(gp + v3(17.3f, tt, 4.1f)), vnz(gp + v3(5.7f, 9.2f, tt))) * 2.0f - v3(1.0f, 1.0f, 1.0f);
      }
      const V3 base = P.airOn != 0u ? airAt(P, B.air, p) : v3(P.q1, P.q2, P.q3);
      const V3 airv = base + gust * P.q7 * (mist ? 2.5f : 1.0f);
      v.y -= P.gravity * P.dt;
      v = v + (airv - v) * (1.0f - st_expf(-(mist ? P.mistDrag : P.sprDrag) * P.dt));
      life -= P.dt;
    } else if (kind == 2u) {
      const float vy = vf.y + clampf((wet - 0.5f) * 4.0f, -1.0f, 1.0f) * P.h * 4.0f;
      v = vmix(v, v3(vf.x, vy, vf.z), 1.0f - st_expf(-10.0f * P.dt));
      life -= P.dt;
    } else {
      v = vmix(v, vf + v3(0.0f, P.wwRise, 0.0f), 1.0f - st_expf(-6.0f * P.dt));
      life -= 0.3f * P.dt;
    }
    const V3 np = p + v * P.dt;
    if (np.x < P.x0 || np.x > P.x1 || np.y < P.y0 || np.y > P.y1 || np.z < P.z0 || np.z > P.z1) life = 0.0f;
    else if (P.ncols > 0u && colAt(P, B.cols, B.sdf, np) >= 0) life = 0.0f;
    else if (P.ocean != 0u && kind >= 2u && layerW(P, np) > 0.6f) life = 0.0f;   // foam and bubbles end at the ocean's boundary
    B.sPos[j] = make_float4(np.x, np.y, np.z, life);
    B.sVel[j] = make_float4(v.x, v.y, v.z, (float)kind + 0.4f * tk / WWHOLD);
  }
}
// sprayEmit (wgsl-whitewater.js:99-133): g2p counted each particle's points (emitK) and their sum per tile; here the
// points go into ring slots (sctl[0] + run) % smax that are not alive, run counting in storage order
__global__ void __launch_bounds__(256) k_emit_write(Bufs B) {
  __shared__ FlipParams P;
  __shared__ uint32_t sm[33];
  loadParams(P, B.P);
  const uint32_t nA = B.ctl->nActive, s0ring = B.ctl->sctl0;
  for (uint32_t a = blockIdx.x; a < nA; a += gridDim.x) {
    if (B.tileEmit[a + 1] == B.tileEmit[a]) continue;   // uniform per block: nothing thrown off in this tile
    const uint32_t s0 = B.tileCnt[a], s1 = B.tileCnt[a + 1];
    uint32_t base = B.tileEmit[a];
    for (uint32_t c0 = s0; c0 < s1; c0 += blockDim.x) {
      const uint32_t i = c0 + threadIdx.x;
      const uint32_t ek = i < s1 ? B.emitK[i] : 0u;
      const uint32_t kc = ek & 7u;
      uint32_t tot;
      const uint32_t run0 = base + blockExclusive(kc, sm, &tot);
      base += tot;
      if (!kc) continue;
      Part q = B.pa[i];
      float rho, fast, e;
      emitTerms(P, B.wet, q.p, q.v, rho, fast, e);
      const V3 qp = xyz(q.p), v = xyz(q.v);
      const float spd = len3(v);
      const uint32_t h0 = B.ida[i] * 747796405u + P.seed * 2891336453u;
      for (uint32_t mm = 0; mm < kc; mm++) {
        const uint32_t run = run0 + mm;
        if (run >= P.smax) break;   // more points tried in one step than the ring holds: the rest are dropped
        const uint32_t slot = (uint32_t)(((uint64_t)s0ring + run) % P.smax);
        if (B.sPos[slot].w > 0.0f) continue;   // never replace a living point
        const uint32_t hh = h0 ^ ((mm + 1u) * 0x9E3779B9u);
        const float z = hash1(hh + 1u) * 2.0f - 1.0f;
        const float an = hash1(hh + 2u) * 6.2831853f;
        const float s = sqrtf(fmx(0.0f, 1.0f - z * z));
        float sa, ca;
        st_sincosf(an, &sa, &ca);
        const V3 dir = v3(s * ca, s * sa, z);
        const bool under = rho > 0.7f && hash1(hh + 7u) < 0.7f;
        const bool mist = !under && hash1(hh + 3u) < P.mistFrac * fast;
        V3 nv = v * (0.9f + 0.2f * hash1(hh + 4u)) + dir * spd * (mist ? 0.2f : 0.06f);
        float life = P.sprLife * (0.6f + 0.8f * hash1(hh + 5u)) * (mist ? 1.6f : 1.0f);
        float kind = mist ? 1.0f : 0.0f;
        if (under) { nv = v + dir * spd * 0.05f; life = P.wwFoamLife * (0.6f + 0.8f * hash1(hh + 5u)); kind = 3.0f; }
        const V3 np = qp + nv * P.dt + dir * P.h * 0.3f * hash1(hh + 6u);
        B.sPos[slot] = make_float4(np.x, np.y, np.z, life);
        B.sVel[slot] = make_float4(nv.x, nv.y, nv.z, kind);
      }
      if (ek & EMIT_KILL) {   // the narrow band trim g2p held back until the points were written
        q.p = make_float4(0.0f, -1.0e6f, 0.0f, 0.0f);
        q.v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        B.pa[i] = q;
      }
    }
  }
}
__global__ void k_emit_done(Bufs B) {
  const FlipParams* P = B.P;
  const uint32_t tried = B.ctl->emitTried;
  if (tried > P->smax) B.ctl->sprayOvf += 1u;
  B.ctl->sctl0 = B.ctl->sctl0 + tried;
}
// dripStep (wgsl-whitewater.js:254-278): drip samples over the colliders' surfaces stay wet in water and dry over
// P.dripDry seconds out of it, letting go of drops while they dry. The reference hands out ring slots with an atomic in
// arbitrary order; here one CTA walks the samples in ascending order and numbers the drops with block scans, so drop
// r goes to slot (sctl[0] + r) % smax. Drops beyond smax in one pass are not written (their slots would repeat).
// Three passes so that every SM takes part: each CTA tests one chunk of DRIP_T samples and counts its drops, one CTA
// turns the counts into offsets, then each chunk writes its drops into the ring in sample order (the order of the
// reference's single loop, so the slots are the same).
__global__ void __launch_bounds__(DRIP_T) k_drip_test(Bufs B) {
  __shared__ FlipParams P;
  loadParams(P, B.P);
  const uint32_t nd = P.ndrip, s = blockIdx.x * DRIP_T + threadIdx.x;
  if (blockIdx.x * DRIP_T >= nd) return;   // a chunk past the samples (the grid covers the buffer's capacity)
  uint32_t want = 0;
  V3 probe = v3(0.0f, 0.0f, 0.0f), nv = probe;
  if (s < nd) {
    const float4 a = B.drip[2 * s], b = B.drip[2 * s + 1];
    const uint32_t k = u32f(a.w);
    if (k < P.ncols) {
      const V3 r0 = xyz(B.cols[k * 8 + 2]), r1 = xyz(B.cols[k * 8 + 3]), r2 = xyz(B.cols[k * 8 + 4]);
      const V3 wp = xyz(B.cols[k * 8 + 5]) + r0 * a.x + r1 * a.y + r2 * a.z;
      const V3 wr = r0 * b.x + r1 * b.y + r2 * b.z;
      const V3 wn = wr / len3(wr);
      probe = wp + wn * P.h * 0.75f;
      const float here = wetAt(P, B, probe);
      if (here > 0.4f) {
        B.drip[2 * s + 1] = make_float4(b.x, b.y, b.z, 1.0f);
      } else {
        const float wetness = fmx(0.0f, b.w - P.dt / fmx(P.dripDry, 0.05f));
        B.drip[2 * s + 1] = make_float4(b.x, b.y, b.z, wetness);
        if (!(wetness <= 0.0f || here > 0.1f || P.smax == 0u || P.dripRate <= 0.0f)) {
          const float down = clampf(-wn.y, 0.0f, 1.0f);
          const float rate = P.dripRate * wetness * wetness * (0.15f + 0.85f * down);
          const uint32_t h0 = s * 747796405u + P.seed * 2891336453u + 17u;
          if (hash1(h0) < rate * P.dt) {
            want = 1;
            nv = colSurfVel(B.cols, k, wp) + wn * P.h * 2.0f * hash1(h0 + 1u);
          }
        }
      }
    }
    B.dripTmp[2 * s] = make_float4(probe.x, probe.y, probe.z, want ? 1.0f : 0.0f);
    B.dripTmp[2 * s + 1] = make_float4(nv.x, nv.y, nv.z, 0.0f);
  }
  const uint32_t cnt = (uint32_t)__syncthreads_count(want != 0u);
  if (threadIdx.x == 0) B.dripCnt[blockIdx.x] = cnt;
}
__global__ void __launch_bounds__(1024) k_drip_scan(Bufs B) {
  __shared__ uint32_t sm[33];
  const uint32_t nd = B.P->ndrip, nch = (nd + DRIP_T - 1) / DRIP_T;
  const uint32_t s0ring = B.ctl->sctl0;
  scanOne(B.dripCnt, nch, nullptr, sm);   // dripCnt[nch] = the drops of this step
  if (threadIdx.x == 0) {
    B.dripCnt[nch + 1] = s0ring;
    B.ctl->sctl0 = s0ring + B.dripCnt[nch];
  }
}
__global__ void __launch_bounds__(DRIP_T) k_drip_write(Bufs B) {
  __shared__ FlipParams P;
  __shared__ uint32_t sm[33];
  loadParams(P, B.P);
  const uint32_t nd = P.ndrip, nch = (nd + DRIP_T - 1) / DRIP_T, s = blockIdx.x * DRIP_T + threadIdx.x;
  if (blockIdx.x >= nch) return;
  const float4 pr = s < nd ? B.dripTmp[2 * s] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const uint32_t want = pr.w > 0.5f ? 1u : 0u;
  const uint32_t run = B.dripCnt[blockIdx.x] + blockExclusive(want, sm, nullptr);
  if (want && run < P.smax) {
    const uint32_t slot = (uint32_t)(((uint64_t)B.dripCnt[nch + 1] + run) % P.smax);
    if (!(B.sPos[slot].w > 0.0f)) {
      const float4 nv = B.dripTmp[2 * s + 1];
      B.sPos[slot] = make_float4(pr.x, pr.y, pr.z, P.sprLife * 2.0f);
      B.sVel[slot] = make_float4(nv.x, nv.y, nv.z, 0.0f);
    }
  }
}

// ---- launchers: each returns how many kernels it launched ----
int launch_nb_init(const Bufs& B, int grid, cudaStream_t s) { k_nb_init<<<grid, 512, 0, s>>>(B); return 1; }
int launch_nb_phi(const Bufs& B, int grid, cudaStream_t s) {
  k_nb_phi<<<grid, 512, 0, s>>>(B);
  k_nb_jac<<<grid, 512, 0, s>>>(B, 1);
  k_nb_jac<<<grid, 512, 0, s>>>(B, 0);
  k_nb_jac<<<grid, 512, 0, s>>>(B, 1);
  return 4;
}
int launch_nb_vel(const Bufs& B, int grid, cudaStream_t s) { k_nb_vel<<<grid, 512, 0, s>>>(B); return 1; }
int launch_nb_reseed(const Bufs& B, int grid, cudaStream_t s) {
  k_scan_x<<<1, 1024, 0, s>>>(B, 0);
  k_killed_list<<<walk_grid((const void*)k_killed_list, 512, grid), 512, 0, s>>>(B);
  k_def_count<<<walk_grid((const void*)k_def_count, 512, grid), 512, 0, s>>>(B);
  k_scan_x<<<2, 1024, 0, s>>>(B, 1);
  k_spawn<<<walk_grid((const void*)k_spawn, 512, grid), 512, 0, s>>>(B);
  return 5;
}
void warm_walk_grids_extra() {
  walk_grid((const void*)k_killed_list, 512, 1);
  walk_grid((const void*)k_def_count, 512, 1);
  walk_grid((const void*)k_spawn, 512, 1);
}
int launch_spray(const Bufs& B, uint32_t smax, bool emit, uint32_t airCells, uint32_t dripCap, int grid, cudaStream_t s) {
  if (!smax) return 0;
  int nl = 0;
  if (airCells) {   // the air field first, so the whitewater moves with this step's air (src/flip/sim.js:297-301)
    cudaMemsetAsync(B.airAcc, 0, (size_t)airCells * 16, s);
    k_air_splat<<<grid * 4, 256, 0, s>>>(B);   // a particle stream: more CTAs keep more loads in flight (0.42 -> 0.40 ms)
    const int ga = (int)std::min<uint32_t>((airCells + 255) / 256, 148u * 8u);
    k_air_update<<<ga, 256, 0, s>>>(B);
    k_air_copy<<<ga, 256, 0, s>>>(B, airCells);
    nl += 3;
  }
  k_ww_step<<<grid, 256, 0, s>>>(B);
  nl++;
  if (emit) {
    k_scan_x<<<1, 1024, 0, s>>>(B, 2);
    k_emit_write<<<grid, 256, 0, s>>>(B);
    k_emit_done<<<1, 1, 0, s>>>(B);
    nl += 3;
  }
  if (dripCap) {
    const int nch = (int)((dripCap + DRIP_T - 1) / DRIP_T);
    k_drip_test<<<nch, DRIP_T, 0, s>>>(B);
    k_drip_scan<<<1, 1024, 0, s>>>(B);
    k_drip_write<<<nch, DRIP_T, 0, s>>>(B);
    nl += 3;
  }
  return nl;
}

}  // namespace st
