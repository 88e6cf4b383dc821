// common.cuh - device-side data layout and helpers shared by the FLIP kernels.
//
// Grid storage is tile-indexed: tile t = ti + tx*(tj + ty*tk) owns cells t*512 + (i&7) + 8*((j&7) + 8*(k&7)).
// The whole tile box of every workload fits in HBM, so every tile has a fixed home and no kernel needs the
// reference's tile -> slot indirection (tmap, src/flip/wgsl-core.js:80-83). Tiles without storage in the
// reference sense ("inactive") are kept in the state the reference's spare slot 0 reads as: cnt 0, type air,
// pressure 0, rhs 8, velocities 0 (src/flip/wgsl-solver.js:6-15).
//
// All arithmetic follows the reference WGSL operation by operation (left-to-right sums, no fused multiply-add:
// the library is built with -fmad=false) so that integer and discrete results are bit-identical to the oracle.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/st_math.h"

namespace st {

// the text st_last_error() returns on this thread (capi.cu)
void set_error_text(const char* text);

constexpr float DEADY = -1.0e5f;
constexpr uint32_t DEADKEY = 0xffffffffu;
constexpr float WWHOLD = 0.2f;

// The solver's parameter block (src/flip/wgsl-core.js:3-20, packed by src/flip/sim.js:196-231), resident in device
// memory so that a captured launch sequence reads each step's values.
struct FlipParams {
  uint32_t n, nx, ny, nz, ncols, open, tx, ty, tz, ntiles;
  float dt, h, ih, gravity, flip, rest, comp, omega;
  float x0, y0, z0, vmax, margin, scale, x1, y1, z1;
  float q0, q1, q2, q3, q4, q5, q6, q7, q8, q9, q10, q12;
  float sheetMin, sprRate, sprMin, sprLife, mistFrac, sprDrag, mistDrag, vs;
  uint32_t smax, seed, nb, nbInit, nfill, lcap, stamp, sprayOn;
  float band, wwFoamLife, wwRise, wwCrest, wwImpact;
  uint32_t airOn, aNx, aNy, aNz;          // air field (words 72-83 of the reference's block)
  float airCouple, airDecay, airH, airBlur;
  uint32_t ndrip;                         // drips (words 79-81)
  float dripRate, dripDry;
  uint32_t ocean, nwave;                  // ocean (words 57-61, 63, 66; the waves follow the collider records)
  float otime, olevel, olayer, oy0, odepth;
  uint32_t nfv;                           // water-mesh fill volumes after the colliders (word 67), on a restart step
  uint32_t padW[1];
  float fills[16][4];
};
// the collider records follow the block in the upload buffer and are read as float4
static_assert(sizeof(FlipParams) % 16 == 0, "FlipParams must keep 16-byte multiples");

// Device counters (the reference's ctl words, src/flip/wgsl-core.js:38-40, plus this design's own).
struct Ctl {
  uint32_t nActive;     // tiles with storage (ctl[4])
  uint32_t fluid;       // fluid cells (ctl[0] + ctl[1])
  uint32_t vmaxBits;    // fastest particle (ctl[6])
  uint32_t nLive;       // live particles this step (sum of cell counts)
  uint32_t nDropped;    // tiles that lost storage this step
  uint32_t nDead;       // dead particle slots (narrow band refill list length)
  uint32_t sctl0;       // whitewater slots handed out (sctl[0])
  uint32_t sprayOvf;    // steps whose emission tried more points than the ring holds
  uint32_t defCount;    // narrow band deficit cells
  uint32_t defNeed;     // particles they ask for
  uint32_t emitTried;   // whitewater points tried this step
  uint32_t nFluidTiles; // tiles holding at least one fluid cell
  uint32_t nKilled;     // particles g2p killed this step (open faces, narrow band trim)
  uint32_t tileNext;    // p2g / g2p: the next tile a CTA takes (nextTile), 0 between launches
  uint32_t tileDone;    // p2g / g2p: CTAs that have run out of tiles, 0 between launches
  uint32_t pad;
};
// Dynamic tile assignment for the per-tile kernels whose tiles differ widely in work (p2g, g2p): a CTA takes the next
// tile of the list when it has finished one, so the SMs that drew light tiles take more of them (a fixed stride left
// SMs idle for the last sixth of g2p). Launch these kernels with only as many CTAs as can be resident. The call is a
// barrier of the CTA; `slot` is a shared word.
__device__ __forceinline__ uint32_t nextTile(Ctl* ctl, uint32_t* slot) {
  if (threadIdx.x == 0) *slot = atomicAdd(&ctl->tileNext, 1u);
  __syncthreads();
  return *slot;
}
// The same assignment for kernels whose tiles are short: the index of the next tile is fetched when the CTA starts a
// tile, so its latency hides behind the tile's work, and handed over at a barrier that ends the tile (two shared
// words, so a slow warp still reading the current index is never overwritten).
//   TileWalk w{B.ctl, words};
//   for (uint32_t a = w.begin(); a < nA; a = w.next()) { w.fetch(); ...the tile... }
//   w.done();
struct TileWalk {
  Ctl* ctl;
  uint32_t* slot;
  uint32_t k = 0, pre = 0;
  __device__ __forceinline__ uint32_t begin() { return nextTile(ctl, slot); }
  __device__ __forceinline__ void fetch() { if (threadIdx.x == 0) pre = atomicAdd(&ctl->tileNext, 1u); }
  __device__ __forceinline__ uint32_t next() {
    k ^= 1u;
    if (threadIdx.x == 0) slot[k] = pre;
    __syncthreads();
    return slot[k];
  }
  __device__ __forceinline__ void done();
};
// After a CTA's last nextTile: the last CTA to leave puts the counters back to 0 for the next launch on the stream
// (every other CTA has taken its last tile by then: each one's fetch is fenced before it counts itself out).
__device__ __forceinline__ void tilesDone(Ctl* ctl) {
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&ctl->tileDone, 1u) == gridDim.x - 1u) {
      ctl->tileNext = 0u;
      ctl->tileDone = 0u;
    }
  }
}
__device__ __forceinline__ void TileWalk::done() { tilesDone(ctl); }

struct Part { float4 p, v; };   // one particle: position (w: speed + 64 x foam level), velocity (w: foam)

// Pointers to every device buffer of one simulator.
struct Bufs {
  const FlipParams* P;
  Ctl* ctl;
  Part* pa;             // particles, storage order of this step (written by p2g)
  Part* pb;             // particles, previous order (read by the sort)
  uint32_t* ida;        // ids matching pa
  uint32_t* idb;        // ids matching pb
  uint32_t* key;        // per particle: cell key, DEADKEY when dead
  uint32_t* rank;       // per particle: rank inside its cell (or dead rank inside its block)
  uint32_t* srcIdx;     // per sorted position: index into pb
  uint32_t* spid;       // per sorted position: id
  uint32_t* blkDead;    // per particle block: dead count, then exclusive offsets
  // tiles
  uint32_t* need;       // stamp of the last step that marked the tile
  uint8_t* on;          // tile has storage this step
  uint8_t* tstate;      // bit0 had storage last step, bit1 has it now
  uint32_t* blkTiles;   // per 1024-tile chunk: tiles with storage
  uint32_t* active;     // tiles with storage, ascending
  uint32_t* prevActive; // last step's list (narrow band marking)
  uint32_t* tileSlot;   // tile -> position in active
  uint32_t* dropped;    // tiles that lost storage this step
  uint32_t* fluidTiles; // tiles holding fluid this step (any order)
  uint32_t* tileCnt;    // per active position: particles, then exclusive offsets (size ntiles + 1)
  uint32_t* tileAux;    // per active position: scratch counts (deficit cells), then offsets
  uint32_t* tileAux2;   // per active position: scratch sums (deficit need), then offsets
  // cells (ncell = ntiles * 512)
  int32_t* cnt;         // particles per cell, this step (two buffers alternate by step)
  int32_t* cntOther;    // the other buffer: cleared during this step for the next one
  uint32_t* cellOff;    // exclusive prefix of cnt inside the tile
  uint32_t* ctype;      // bits 0-7 type, 8-15 collider + 1, 16-31 depth (src/flip/wgsl-core.js:33)
  float* pres;
  float* rhs;
  int32_t* acc;         // 6 planes of ncell: summed v (x, y, z), summed weight (x, y, z), fixed point
  float* vn;            // 3 planes: new face velocity
  float* vo;            // 3 planes: old face velocity
  float* velG;          // 3 planes: kept grid velocity (narrow band)
  uint16_t* sorInfo;    // per fluid cell: bits 0-5 neighbour is fluid, bits 8-10 non-solid neighbours
  // the pressure sweeps' compact copy: per fluid tile (position a in fluidTiles) 512 values, red cells then black
  // ones, each half ordered (lx / 2) + 4 (ly + 8 lz); nbs: the positions of its 6 face neighbours (own when none)
  float* cp;
  float* crhs;
  uint16_t* cinfo;
  uint32_t* nbs;
  uint32_t* slotOf;     // per tile: position in fluidTiles, or 0xffffffff
  // where this tank's fluid tiles start in the compact copy (0 for a tank alone; a tank of a pooled batch shares one
  // copy with the others, at the offset the batch's plan kernel writes); pomega: the SOR factor of each copied tile
  const uint32_t* poolOff;
  float* pomega;
  float* wet;           // per cell: how much water (wetCell, src/flip/wgsl-whitewater.js:7-12), 0 outside the domain
  // air field (src/flip/wgsl-whitewater.js:24-89): velocity at air-cell centres, its next value, fixed-point pushes
  float4* air;
  float4* air2;
  int32_t* airAcc;      // 4 per air cell: sum of v w 256 (x, y, z) and of w 256
  float4* drip;         // 2 per drip sample (dripSamples, src/flip/bake.js:19-40): local position + collider, local normal + wetness
  float4* dripTmp;      // 2 per drip sample: the probe point (w: 1 when it drips this step) and the drop's velocity
  uint32_t* dripCnt;    // drops per chunk of DRIP_T samples, then their exclusive offsets, the total and the ring start
  const float4* waves;  // ocean: 2 per wave, (kx, kz, amplitude, angular frequency) and (phase, wavenumber, 0, 0)
  // colliders
  const float4* cols;   // 8 per collider (src/gpu.js:3-4)
  const float* sdf;
  // whitewater
  float4* sPos;
  float4* sVel;
  uint8_t* emitK;       // per particle: points to emit
  uint32_t* blkEmit;    // per particle block: points, then offsets
  uint8_t* deadF;       // per particle: killed by g2p this step (narrow band runs)
  uint32_t* tileEmit;   // per active position: whitewater points its particles throw off, then offsets
  uint32_t* tileDead;   // per active position: particles killed in it, then offsets
  // narrow band refill
  uint32_t* deadList;   // this step's killed particles in storage order
  uint32_t ncell;
  uint32_t nblk;        // particle blocks of PBLK
};

constexpr int PBLK = 1024;     // particles per block in the order-defining passes (count, scatter, dead lists)

// The compact copy shared by the tanks of a pooled batch (capi.cu's ST_BATCH_POOLED): every tank's fluid tiles one after
// another in tank order, with their SOR factors; the offsets and total come from the plan kernel each step.
struct PoolBufs {
  float* cp;
  float* crhs;
  uint16_t* cinfo;
  uint32_t* nbs;
  float* pomega;
  uint32_t* off;          // per tank
  uint32_t* total;
  unsigned int* bar;      // the persistent sweep's grid barrier
  unsigned int* err;      // set when a barrier wait ran out
};

// the parameter block into a CTA's shared copy (every thread of the CTA calls it; it ends with a barrier)
__device__ __forceinline__ void loadParams(FlipParams& s, const FlipParams* g) {
  const uint32_t* src = reinterpret_cast<const uint32_t*>(g);
  uint32_t* dst = reinterpret_cast<uint32_t*>(&s);
  for (int i = threadIdx.x; i < (int)(sizeof(FlipParams) / 4); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
}

// ---- small vector math: every operation spelled out so the order matches the oracle ----
struct V3 { float x, y, z; };
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float len3(V3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ float fmn(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float fmx(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fmn(fmx(x, lo), hi); }
__device__ __forceinline__ V3 vmin(V3 a, V3 b) { return v3(fmn(a.x, b.x), fmn(a.y, b.y), fmn(a.z, b.z)); }
__device__ __forceinline__ V3 vmax(V3 a, V3 b) { return v3(fmx(a.x, b.x), fmx(a.y, b.y), fmx(a.z, b.z)); }
__device__ __forceinline__ V3 vclamp(V3 a, V3 lo, V3 hi) { return vmin(vmax(a, lo), hi); }
__device__ __forceinline__ V3 vfloor(V3 a) { return v3(floorf(a.x), floorf(a.y), floorf(a.z)); }
__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ V3 vmix(V3 a, V3 b, float t) { return v3(mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t)); }
__device__ __forceinline__ V3 cross3(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
__device__ __forceinline__ float smoothstepf(float e0, float e1, float x) {
  float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
__device__ __forceinline__ float comp3(V3 a, int ax) { return ax == 0 ? a.x : (ax == 1 ? a.y : a.z); }
__device__ __forceinline__ uint32_t u32f(float f) { return f <= 0.0f ? 0u : (uint32_t)f; }
__device__ __forceinline__ V3 xyz(float4 a) { return v3(a.x, a.y, a.z); }

// hash1 (src/flip/wgsl-solver.js:181-184)
__device__ __forceinline__ float hash1(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
  return (float)x * 2.3283064e-10f;
}

// ---- addressing ----
__device__ __forceinline__ uint32_t tileOf(const FlipParams& P, int i, int j, int k) {
  return (uint32_t)(i >> 3) + P.tx * ((uint32_t)(j >> 3) + P.ty * (uint32_t)(k >> 3));
}
__device__ __forceinline__ uint32_t cellIdx(const FlipParams& P, int i, int j, int k) {
  return tileOf(P, i, j, k) * 512u + (uint32_t)(i & 7) + 8u * ((uint32_t)(j & 7) + 8u * (uint32_t)(k & 7));
}
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
// a floored grid coordinate as an index, held in [-2, 2^24] so that index + 1 cannot overflow for huge or infinite
// positions (the conversion saturates); in-range values are unchanged
__device__ __forceinline__ int gidx(float f) { return clampi((int)f, -2, 1 << 24); }
// the cell holding face (axis, i, j, k) after the reference's clamping (src/flip/wgsl-core.js:84-89)
__device__ __forceinline__ uint32_t faceCell(const FlipParams& P, int axis, int i, int j, int k) {
  int nx = (int)P.nx, ny = (int)P.ny, nz = (int)P.nz;
  if (axis == 0) return cellIdx(P, clampi(i, 0, nx), clampi(j, 0, ny - 1), clampi(k, 0, nz - 1));
  if (axis == 1) return cellIdx(P, clampi(i, 0, nx - 1), clampi(j, 0, ny), clampi(k, 0, nz - 1));
  return cellIdx(P, clampi(i, 0, nx - 1), clampi(j, 0, ny - 1), clampi(k, 0, nz));
}
__device__ __forceinline__ void tileCoord(const FlipParams& P, uint32_t t, uint32_t local, int& i, int& j, int& k) {
  uint32_t tt = t / P.tx;
  i = (int)((t % P.tx) * 8u + (local & 7u));
  j = (int)((tt % P.ty) * 8u + ((local >> 3) & 7u));
  k = (int)((tt / P.ty) * 8u + (local >> 6));
}
__device__ __forceinline__ bool inDom(const FlipParams& P, int i, int j, int k) {
  return i >= 0 && j >= 0 && k >= 0 && i < (int)P.nx && j < (int)P.ny && k < (int)P.nz;
}
// ctypeOf (src/flip/wgsl-core.js:104-112)
__device__ __forceinline__ uint32_t ctypeOf(const FlipParams& P, const uint32_t* __restrict__ ctype, int i, int j, int k) {
  if (i < 0) return (P.open & 1u) ? 0u : 2u;
  if (i >= (int)P.nx) return (P.open & 2u) ? 0u : 2u;
  if (j < 0) return (P.open & 4u) ? 0u : 2u;
  if (j >= (int)P.ny) return (P.open & 8u) ? 0u : 2u;
  if (k < 0) return (P.open & 16u) ? 0u : 2u;
  if (k >= (int)P.nz) return (P.open & 32u) ? 0u : 2u;
  return ctype[cellIdx(P, i, j, k)] & 0xffu;
}
__device__ __forceinline__ V3 cellCenter(const FlipParams& P, int i, int j, int k) {
  return v3(P.x0 + ((float)i + 0.5f) * P.h, P.y0 + ((float)j + 0.5f) * P.h, P.z0 + ((float)k + 0.5f) * P.h);
}
__device__ __forceinline__ void particleCell(const FlipParams& P, V3 p, int& ci, int& cj, int& ck) {
  V3 g = vfloor((p - v3(P.x0, P.y0, P.z0)) * P.ih);
  ci = clampi((int)g.x, 0, (int)P.nx - 1);
  cj = clampi((int)g.y, 0, (int)P.ny - 1);
  ck = clampi((int)g.z, 0, (int)P.nz - 1);
}
__device__ __forceinline__ V3 facePos(const FlipParams& P, int i, int j, int k, int axis) {
  return v3(P.x0 + ((float)i + (axis == 0 ? 0.0f : 0.5f)) * P.h, P.y0 + ((float)j + (axis == 1 ? 0.0f : 0.5f)) * P.h,
            P.z0 + ((float)k + (axis == 2 ? 0.0f : 0.5f)) * P.h);
}
__device__ __forceinline__ float phiOfBits(uint32_t ct) { return 8.0f - (float)(ct >> 16) / 4096.0f; }
__device__ __forceinline__ uint32_t phiPutBits(uint32_t ct, float v) {
  uint32_t q = (uint32_t)clampf(rintf((8.0f - v) * 4096.0f), 0.0f, 65535.0f);
  return (ct & 0xffffu) | (q << 16);
}

// ---- velGAxis (src/flip/wgsl-core.js:185-197): the kept grid velocity (narrow band), trilinear on the MAC faces ----
__device__ __forceinline__ float velGAxis(const FlipParams& P, const float* __restrict__ velG, uint32_t nc, V3 x, int axis) {
  V3 g = (x - v3(P.x0, P.y0, P.z0)) * P.ih;
  if (axis == 0) { g.y -= 0.5f; g.z -= 0.5f; } else if (axis == 1) { g.x -= 0.5f; g.z -= 0.5f; } else { g.x -= 0.5f; g.y -= 0.5f; }
  const V3 f0 = vfloor(g), fr = g - f0;
  const int i0 = gidx(f0.x), j0 = gidx(f0.y), k0 = gidx(f0.z);
  float s = 0.0f;
  for (int c = 0; c < 8; c++) {
    const int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
    const float w = (dx == 1 ? fr.x : 1.0f - fr.x) * (dy == 1 ? fr.y : 1.0f - fr.y) * (dz == 1 ? fr.z : 1.0f - fr.z);
    s += w * velG[axis * nc + faceCell(P, axis, i0 + dx, j0 + dy, k0 + dz)];
  }
  return s;
}
__device__ __forceinline__ V3 velGVec(const FlipParams& P, const float* __restrict__ velG, uint32_t nc, V3 x) {
  return v3(velGAxis(P, velG, nc, x, 0), velGAxis(P, velG, nc, x, 1), velGAxis(P, velG, nc, x, 2));
}

// ---- value noise (wgsl-solver.js:198-207): the gusts of g2p and of the whitewater step ----
__device__ __forceinline__ float hsh3(V3 p) {
  V3 q = p * 0.3183099f + v3(0.1f, 0.2f, 0.3f);
  q = q - vfloor(q);
  q = q * 17.0f;
  const float r = q.x * q.y * q.z * (q.x + q.y + q.z);
  return r - floorf(r);
}
static __device__ float vnz(V3 x) {
  const V3 i = vfloor(x), fr = x - vfloor(x);
  const V3 u = fr * fr * (v3(3.0f, 3.0f, 3.0f) - fr * 2.0f);
  const float a = mixf(mixf(hsh3(i), hsh3(i + v3(1, 0, 0)), u.x), mixf(hsh3(i + v3(0, 1, 0)), hsh3(i + v3(1, 1, 0)), u.x), u.y);
  const float b = mixf(mixf(hsh3(i + v3(0, 0, 1)), hsh3(i + v3(1, 0, 1)), u.x), mixf(hsh3(i + v3(0, 1, 1)), hsh3(i + v3(1, 1, 1)), u.x), u.y);
  return mixf(a, b, u.z);
}

// ---- ocean (src/flip/wgsl-core.js:201-226): a sum of linear (Airy) waves ----
// Out of line: inlined, the wave loops raise the register count of the kernels that call them.
static __device__ __noinline__ float oceanEta(const FlipParams& P, const float4* __restrict__ W, float x, float z) {
  float e = 0.0f;
  for (uint32_t k = 0; k < P.nwave; k++) {
    const float4 A = W[2 * k], Bw = W[2 * k + 1];
    float sn, cs;
    st_sincosf(A.x * x + A.y * z - A.w * P.otime + Bw.x, &sn, &cs);
    e += A.z * cs;
  }
  return P.olevel + e;
}
// the water velocity under the waves over a floor at depth odepth, the height stretched so a crest gets the surface value
static __device__ __noinline__ V3 oceanVel(const FlipParams& P, const float4* __restrict__ W, V3 p) {
  const float D = fmx(P.odepth, 1.0e-3f), eta = oceanEta(P, W, p.x, p.z);
  const float ys = clampf((p.y - P.oy0) * D / fmx(D + eta - P.olevel, 0.1f * D), 0.0f, D);
  V3 v = v3(0.0f, 0.0f, 0.0f);
  for (uint32_t k = 0; k < P.nwave; k++) {
    const float4 A = W[2 * k], Bw = W[2 * k + 1];
    const float kk = fmx(Bw.y, 1.0e-4f);
    const float th = A.x * p.x + A.y * p.z - A.w * P.otime + Bw.x;
    const float e1 = st_expf(kk * (ys - D)), e2 = st_expf(-kk * (ys + D)), dn = fmx(1.0f - st_expf(-2.0f * kk * D), 1.0e-4f);
    const float aw = A.z * A.w;
    float sn, cs;
    st_sincosf(th, &sn, &cs);
    const float hc = aw * (e1 + e2) / dn * cs / kk;
    v = v + v3(hc * A.x, aw * (e1 - e2) / dn * sn, hc * A.y);
  }
  return v;
}
// 1 at the side walls, 0 a boundary width in from them: above 0.5 the ocean is prescribed, below it particles are nudged
__device__ __forceinline__ float layerW(const FlipParams& P, V3 p) {
  if (P.ocean == 0u) return 0.0f;
  const float dw = fmn(fmn(p.x - P.x0, P.x1 - p.x), fmn(p.z - P.z0, P.z1 - p.z));
  return clampf(1.0f - dw / fmx(P.olayer, 1.0e-4f), 0.0f, 1.0f);
}
// ---- colliders (src/gpu.js:6-38, src/flip/wgsl-core.js:113-126) ----
__device__ __forceinline__ void sdfEval(const float4* __restrict__ cols, const float* __restrict__ sdf, uint32_t k, V3 p,
                                        float& phi, V3& wn) {
  float4 a = cols[k * 8], b = cols[k * 8 + 1];
  V3 r0 = xyz(cols[k * 8 + 2]), r1 = xyz(cols[k * 8 + 3]), r2 = xyz(cols[k * 8 + 4]);
  V3 d = p - xyz(cols[k * 8 + 5]);
  V3 lp = v3(dot3(r0, d), dot3(r1, d), dot3(r2, d));
  V3 g = v3((lp.x - b.x) / b.w, (lp.y - b.y) / b.w, (lp.z - b.z) / b.w);
  V3 dims = v3(a.y, a.z, a.w);
  V3 gc = vclamp(g, v3(0.0f, 0.0f, 0.0f), dims - v3(1.0001f, 1.0001f, 1.0001f));
  V3 fl = vfloor(gc);
  V3 f = gc - fl;
  uint32_t nx = u32f(a.y), ny = u32f(a.z);
  uint32_t base = u32f(a.x) + u32f(fl.x) + nx * (u32f(fl.y) + ny * u32f(fl.z));
  uint32_t s = nx * ny;
  float v000 = sdf[base], v100 = sdf[base + 1], v010 = sdf[base + nx], v110 = sdf[base + nx + 1];
  float v001 = sdf[base + s], v101 = sdf[base + s + 1], v011 = sdf[base + s + nx], v111 = sdf[base + s + nx + 1];
  float c00 = mixf(v000, v100, f.x), c10 = mixf(v010, v110, f.x), c01 = mixf(v001, v101, f.x), c11 = mixf(v011, v111, f.x);
  float c0 = mixf(c00, c10, f.y), c1 = mixf(c01, c11, f.y);
  phi = mixf(c0, c1, f.z);
  V3 out = g - gc;
  V3 gl;
  if (dot3(out, out) > 0.0f) {
    float l = len3(out);
    phi += l * b.w;
    gl = out / l;
  } else {
    gl = v3(mixf(mixf(v100 - v000, v110 - v010, f.y), mixf(v101 - v001, v111 - v011, f.y), f.z), mixf(c10 - c00, c11 - c01, f.z), c1 - c0);
    float l = len3(gl);
    gl = gl / fmx(l, 1e-9f);
  }
  wn = r0 * gl.x + r1 * gl.y + r2 * gl.z;
}
// fillPhi (wgsl-core.js:227-238): signed distance in cells to the starting water: boxes, spheres, water meshes (the
// distance grids of the fill volumes, records ncols .. ncols + nfv - 1 after the colliders) and the ocean
__device__ __forceinline__ float fillPhi(const FlipParams& P, const float4* __restrict__ W, const float4* __restrict__ cols,
                                         const float* __restrict__ sdf, V3 x) {
  float d = 1.0e9f;
  for (uint32_t k = 0; k < P.nfill; k++) {
    const float* A = P.fills[k * 2];
    const float* Bq = P.fills[k * 2 + 1];
    if (A[0] < 1.5f) {
      V3 q = vmax(v3(A[1], A[2], A[3]) - x, x - v3(Bq[0], Bq[1], Bq[2]));
      d = fmn(d, len3(vmax(q, v3(0.0f, 0.0f, 0.0f))) + fmn(fmx(q.x, fmx(q.y, q.z)), 0.0f));
    } else {
      d = fmn(d, len3(x - v3(A[1], A[2], A[3])) - Bq[0]);
    }
  }
  for (uint32_t k = P.ncols; k < P.ncols + P.nfv; k++) {
    float phi;
    V3 wn;
    sdfEval(cols, sdf, k, x, phi, wn);
    d = fmn(d, phi);
  }
  if (P.ocean != 0u) d = fmn(d, x.y - oceanEta(P, W, x.x, x.z));
  return d * P.ih;
}

__device__ __forceinline__ V3 colSurfVel(const float4* __restrict__ cols, uint32_t k, V3 p) {
  V3 c = xyz(cols[k * 8 + 5]);
  return xyz(cols[k * 8 + 6]) + cross3(xyz(cols[k * 8 + 7]), p - c);
}
__device__ __forceinline__ bool colNear(const FlipParams& P, const float4* __restrict__ cols, uint32_t k, V3 p) {
  if (P.q10 > 0.5f) return true;
  float4 b = cols[k * 8 + 1];
  V3 d = p - xyz(cols[k * 8 + 5]);
  V3 lp = v3(dot3(xyz(cols[k * 8 + 2]), d), dot3(xyz(cols[k * 8 + 3]), d), dot3(xyz(cols[k * 8 + 4]), d));
  V3 g = v3((lp.x - b.x) / b.w, (lp.y - b.y) / b.w, (lp.z - b.z) / b.w);
  float4 a = cols[k * 8];
  float lo = -1.0f - P.q0 / b.w, hi = P.q0 / b.w;
  return g.x > lo && g.y > lo && g.z > lo && g.x < a.y + hi && g.y < a.z + hi && g.z < a.w + hi;
}
__device__ __forceinline__ int colAt(const FlipParams& P, const float4* __restrict__ cols, const float* __restrict__ sdf, V3 p) {
  for (uint32_t k = 0; k < P.ncols; k++) {
    if (!colNear(P, cols, k, p)) continue;
    float phi; V3 wn;
    sdfEval(cols, sdf, k, p, phi, wn);
    if (phi < P.q0) return (int)k;
  }
  return -1;
}

// collideP (src/flip/wgsl-solver.js:185-197): out of every collider near p by q0, then the walls less the margin
__device__ __forceinline__ V3 collideP(const FlipParams& P, const float4* __restrict__ cols, const float* __restrict__ sdf, V3 pin) {
  V3 p = pin;
  const float m = P.margin;
  for (uint32_t k = 0; k < P.ncols; k++) {
    if (!colNear(P, cols, k, p)) continue;
    float phi; V3 wn;
    sdfEval(cols, sdf, k, p, phi, wn);
    if (phi < P.q0) p = p + wn * (P.q0 - phi);
  }
  const float big = 1.0e9f;
  const V3 lo = v3((P.open & 1u) ? -big : P.x0 + m, (P.open & 4u) ? -big : P.y0 + m, (P.open & 16u) ? -big : P.z0 + m);
  const V3 hi = v3((P.open & 2u) ? big : P.x1 - m, (P.open & 8u) ? big : P.y1 - m, (P.open & 32u) ? big : P.z1 - m);
  return vclamp(p, lo, hi);
}
// ---- whitewater emission terms (sprayEmit, src/flip/wgsl-whitewater.js:101-117), shared by g2p and the emit pass ----
constexpr uint8_t EMIT_KILL = 0x80;   // emitK flag: the narrow band trims this particle once its points are written
__device__ __forceinline__ float wetCellAt(const FlipParams& P, const float* __restrict__ wet, int i, int j, int k) {
  if (!inDom(P, i, j, k)) return 0.0f;
  return wet[cellIdx(P, i, j, k)];
}
// wetAt(i, j, k) gives wetCellAt for the eight cells around the particle (from HBM, or a staged window)
template <class WetAt>
__device__ __forceinline__ void emitTermsT(const FlipParams& P, const WetAt& wetAt, float4 qp, float4 qv, float& rho, float& fast, float& e,
                                           float settle) {
  const V3 p = xyz(qp), v = xyz(qv);
  const float foam = qv.w, spd = len3(v);
  fast = clampf((spd * P.vs - P.sprMin) / (2.0f * P.sprMin), 0.0f, 1.0f);
  const V3 bcf = vfloor((p - v3(P.x0, P.y0, P.z0)) * P.ih - v3(0.5f, 0.5f, 0.5f));
  const int bi = gidx(bcf.x), bj = gidx(bcf.y), bk = gidx(bcf.z);
  rho = 0.0f;
  for (int dz = 0; dz <= 1; dz++)
    for (int dy = 0; dy <= 1; dy++)
      for (int dx = 0; dx <= 1; dx++) rho += wetAt(bi + dx, bj + dy, bk + dz);
  rho = rho / 8.0f;
  const float crest = (1.0f - smoothstepf(0.3f, 0.75f, rho)) * fast * (0.3f + 0.7f * foam);
  const float churn = (1.0f - smoothstepf(0.8f, 1.0f, rho)) * clampf((foam - 0.55f) / 0.45f, 0.0f, 1.0f) * smoothstepf(0.5f, 1.5f, spd * P.vs);
  e = (P.wwCrest * crest + P.wwImpact * churn) * settle;
}
struct WetGlobal {
  const FlipParams& P;
  const float* __restrict__ wet;
  __device__ __forceinline__ float operator()(int i, int j, int k) const { return wetCellAt(P, wet, i, j, k); }
};
__device__ __forceinline__ void emitTerms(const FlipParams& P, const float* __restrict__ wet, float4 qp, float4 qv, float& rho, float& fast, float& e) {
  emitTermsT(P, WetGlobal{P, wet}, qp, qv, rho, fast, e, smoothstepf(0.1f, 0.5f, P.q8));
}

// ---- block-wide scans (blockDim.x a multiple of 32, at most 1024) ----
__device__ __forceinline__ uint32_t warpInclusive(uint32_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t n = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += n;
  }
  return v;
}
// exclusive prefix of v over the block; *total gets the block sum. smem must hold 33 words. Ends with a barrier.
__device__ __forceinline__ uint32_t blockExclusive(uint32_t v, uint32_t* smem, uint32_t* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t inc = warpInclusive(v);
  if (lane == 31) smem[w] = inc;
  __syncthreads();
  if (w == 0) {
    uint32_t s = lane < nw ? smem[lane] : 0u;
    uint32_t si = warpInclusive(s);
    if (lane < nw) smem[lane] = si - s;
    if (lane == nw - 1) smem[32] = si;
  }
  __syncthreads();
  uint32_t r = smem[w] + inc - v;
  if (total) *total = smem[32];
  __syncthreads();
  return r;
}
// exclusive scan of arr[0, n) in place by one CTA (contiguous chunks per thread), arr[n] and *total (when given) = sum
__device__ __forceinline__ void scanOne(uint32_t* arr, uint32_t n, uint32_t* total, uint32_t* sm) {
  const uint32_t chunk = (n + blockDim.x - 1) / blockDim.x;
  const uint32_t beg = min(threadIdx.x * chunk, n), end = min(beg + chunk, n);
  uint32_t s = 0;
  for (uint32_t x = beg; x < end; x++) s += arr[x];
  uint32_t tot;
  uint32_t run = blockExclusive(s, sm, &tot);
  for (uint32_t x = beg; x < end; x++) { const uint32_t v = arr[x]; arr[x] = run; run += v; }
  if (threadIdx.x == 0) { arr[n] = tot; if (total) *total = tot; }
}

}  // namespace st
