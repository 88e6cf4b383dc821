// flip_kernels.cu - the FLIP step on B200: tile activation, particle sort, P2G, classify, normalise + divergence,
// red-black SOR, projection and G2P. Narrow band and whitewater kernels are in flip_extra.cu.
//
// Every kernel is either one thread per particle (storage order) or one CTA per tile with storage, striding over
// device-side counts, so a step needs no host round trip. Citations name the WGSL kernel each one restates.
#include <algorithm>
#include <mutex>
#include <unordered_map>

#include "common.cuh"
#include "kernels.h"

namespace st {

// markAround (wgsl-core.js:239-246): every tile within two cells of cell (ci, cj, ck) gets this step's stamp.
__device__ __forceinline__ void markAround(const FlipParams& P, uint32_t* __restrict__ need, int ci, int cj, int ck) {
  int lox = max(ci - 2, 0) >> 3, loy = max(cj - 2, 0) >> 3, loz = max(ck - 2, 0) >> 3;
  int hix = min(ci + 2, (int)P.tx * 8 - 1) >> 3, hiy = min(cj + 2, (int)P.ty * 8 - 1) >> 3, hiz = min(ck + 2, (int)P.tz * 8 - 1) >> 3;
  for (int tk = loz; tk <= hiz; tk++)
    for (int tj = loy; tj <= hiy; tj++)
      for (int ti = lox; ti <= hix; ti++) {
        uint32_t t = (uint32_t)ti + P.tx * ((uint32_t)tj + P.ty * (uint32_t)tk);
        if (need[t] != P.stamp) need[t] = P.stamp;
      }
}

// ---- 1. tileMark + count per cell (wgsl-blocks.js:10-14, the cell count of wgsl-solver.js:39) ----
// One pass over the particles in storage order: mark tiles near live particles, count particles per cell with
// warp-aggregated atomics (the returned base gives each particle a rank in its cell), count dead slots per block,
// and the fastest speed (ctl[6], wgsl-solver.js:24).
// A CTA of CM_T threads takes one block of PBLK particles, CM_U per thread (a warp's lanes on consecutive particles),
// and keeps all of them in flight (loads, then the atomics, then the tile marks); several CTAs per SM overlap the
// dependent steps and barriers of one another.
constexpr int CM_T = 256, CM_U = PBLK / CM_T;
static_assert(CM_U == 4, "k_scatter packs the dead counts of four slices into two scans");
__global__ void __launch_bounds__(CM_T, 5) k_count_mark(Bufs B) {
  __shared__ FlipParams P;
  __shared__ float wmax[CM_T / 32];
  __shared__ uint32_t wdead[CM_T / 32];
  loadParams(P, B.P);
  const int lane = threadIdx.x & 31;
  Part q[CM_U];
  uint32_t key[CM_U], idx[CM_U], peers[CM_U], base[CM_U];
  bool live[CM_U], dead[CM_U];
  int ci[CM_U], cj[CM_U], ck[CM_U];
  float sp = 0.0f;
#pragma unroll
  for (int u = 0; u < CM_U; u++) {
    idx[u] = blockIdx.x * PBLK + u * CM_T + threadIdx.x;
    if (idx[u] < P.n) q[u] = B.pb[idx[u]];
  }
#pragma unroll
  for (int u = 0; u < CM_U; u++) {
    key[u] = DEADKEY;
    live[u] = dead[u] = false;
    ci[u] = cj[u] = ck[u] = 0;
    if (idx[u] < P.n) {
      if (q[u].p.y < DEADY) dead[u] = true;
      else {
        live[u] = true;
        particleCell(P, xyz(q[u].p), ci[u], cj[u], ck[u]);
        key[u] = cellIdx(P, ci[u], cj[u], ck[u]);
        sp = fmx(sp, len3(xyz(q[u].v)));
      }
      B.key[idx[u]] = key[u];
    }
    peers[u] = __match_any_sync(0xffffffffu, key[u]);
  }
  // the group's first lane counts for all of them, and marks the tiles (lanes in one cell mark the same tiles)
#pragma unroll
  for (int u = 0; u < CM_U; u++) {
    base[u] = 0;
    if (live[u] && lane == __ffs(peers[u]) - 1) base[u] = (uint32_t)atomicAdd(&B.cnt[key[u]], __popc(peers[u]));
  }
#pragma unroll
  for (int u = 0; u < CM_U; u++)
    if (live[u] && lane == __ffs(peers[u]) - 1) markAround(P, B.need, ci[u], cj[u], ck[u]);
#pragma unroll
  for (int u = 0; u < CM_U; u++) {
    const uint32_t b = __shfl_sync(0xffffffffu, base[u], __ffs(peers[u]) - 1);
    if (live[u]) B.rank[idx[u]] = b + __popc(peers[u] & ((1u << lane) - 1u));
  }
  // the block's dead slots, and the fastest speed: lengths are non-negative, so their bit patterns order like the
  // floats; one atomic per CTA
  uint32_t nd = 0;
#pragma unroll
  for (int u = 0; u < CM_U; u++) nd += (uint32_t)__popc(__ballot_sync(0xffffffffu, dead[u]));
  float m = sp;
  for (int o = 16; o > 0; o >>= 1) m = fmx(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) { wmax[threadIdx.x >> 5] = m; wdead[threadIdx.x >> 5] = nd; }
  __syncthreads();
  if (threadIdx.x < 32) {
    float b = threadIdx.x < CM_T / 32 ? wmax[threadIdx.x] : 0.0f;
    uint32_t d = threadIdx.x < CM_T / 32 ? wdead[threadIdx.x] : 0u;
    for (int o = 16; o > 0; o >>= 1) b = fmx(b, __shfl_xor_sync(0xffffffffu, b, o));
    d = __reduce_add_sync(0xffffffffu, d);
    if (threadIdx.x == 0) {
      B.blkDead[blockIdx.x] = d;
      if (b > 0.0f) atomicMax(&B.ctl->vmaxBits, __float_as_uint(b));
    }
  }
}

// tileMarkPhi (wgsl-narrowband.js:6-10): last step's tiles that hold water by depth keep storage.
__global__ void __launch_bounds__(512) k_mark_phi(Bufs B) {
  __shared__ FlipParams P;
  loadParams(P, B.P);
  const uint32_t nA = B.ctl->nActive;   // still last step's count: read before the new list is built
  for (uint32_t a = blockIdx.x; a < nA; a += gridDim.x) {
    uint32_t t = B.active[a], c = t * 512u + threadIdx.x;
    int i, j, k;
    tileCoord(P, t, threadIdx.x, i, j, k);
    if (inDom(P, i, j, k) && phiOfBits(B.ctype[c]) < 0.5f) markAround(P, B.need, i, j, k);
  }
}

// tileMarkFill (wgsl-narrowband.js:12-18): on a restart every tile the starting water reaches
__global__ void k_mark_fill(Bufs B) {
  __shared__ FlipParams P;
  loadParams(P, B.P);
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < P.ntiles; t += gridDim.x * blockDim.x) {
    uint32_t tt = t / P.tx;
    V3 tc = v3((float)(t % P.tx), (float)(tt % P.ty), (float)(tt / P.ty)) * 8.0f + v3(4.0f, 4.0f, 4.0f);
    if (fillPhi(P, B.waves, B.cols, B.sdf, v3(P.x0, P.y0, P.z0) + tc * P.h) < 9.0f) B.need[t] = P.stamp;
  }
}

// ---- 2. which tiles keep, get or lose storage (tileFree / tileAlloc / slotListBuild, wgsl-blocks.js:16-53) ----
// Chunks of 1024 tiles: flags and per-chunk counts; tiles that lose storage go on the dropped list.
__global__ void __launch_bounds__(1024) k_tile_flags(Bufs B) {
  __shared__ FlipParams P;
  loadParams(P, B.P);
  uint32_t t = blockIdx.x * 1024u + threadIdx.x;
  bool now = false;
  if (t < P.ntiles) {
    uint8_t was = B.on[t];
    now = B.need[t] == P.stamp;
    B.on[t] = now ? 1 : 0;
    B.tstate[t] = (uint8_t)((was ? 1 : 0) | (now ? 2 : 0));
    if (was && !now) B.dropped[atomicAdd(&B.ctl->nDropped, 1u)] = t;
  }
  uint32_t c = __syncthreads_count(now);
  if (threadIdx.x == 0) B.blkTiles[blockIdx.x] = c;
}
// The list of tiles with storage in ascending tile order, and each tile's position in it.
__global__ void __launch_bounds__(1024) k_tile_list(Bufs B) {
  __shared__ FlipParams P;
  __shared__ uint32_t sm[33];
  loadParams(P, B.P);
  uint32_t part = 0;
  for (uint32_t b = threadIdx.x; b < blockIdx.x; b += 1024) part += B.blkTiles[b];
  uint32_t off;
  blockExclusive(part, sm, &off);
  uint32_t t = blockIdx.x * 1024u + threadIdx.x;
  bool now = t < P.ntiles && B.on[t];
  uint32_t tot;
  uint32_t r = blockExclusive(now ? 1u : 0u, sm, &tot);
  if (now) { B.active[off + r] = t; B.tileSlot[t] = off + r; }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) B.ctl->nActive = off + tot;
}

// ---- 3. new tiles (initNew, wgsl-blocks.js:37-47), tiles leaving storage, and per-tile counts ----
// Active tiles: a new one starts with pressure 0, air, its collider per cell and no kept velocity.
// Each active tile also gets the exclusive prefix of its cell counts and its particle total.
// Dropped tiles go back to the state the reference's spare slot reads as.
__global__ void __launch_bounds__(512) k_tile_prep(Bufs B) {
  __shared__ FlipParams P;
  __shared__ uint32_t sm[33];
  loadParams(P, B.P);
  const uint32_t nA = B.ctl->nActive, nD = B.ctl->nDropped, nc = B.ncell;
  for (uint32_t a = blockIdx.x; a < nA + nD; a += gridDim.x) {
    if (a < nA) {
      uint32_t t = B.active[a], c = t * 512u + threadIdx.x;
      if (B.tstate[t] == 2) {
        int i, j, k;
        tileCoord(P, t, threadIdx.x, i, j, k);
        B.pres[c] = 0.0f;
        B.ctype[c] = (uint32_t)(colAt(P, B.cols, B.sdf, cellCenter(P, i, j, k)) + 1) << 8;   // depth bits 0: air
        B.velG[c] = 0.0f; B.velG[nc + c] = 0.0f; B.velG[2 * nc + c] = 0.0f;
      }
      uint32_t tot;
      uint32_t ex = blockExclusive((uint32_t)B.cnt[c], sm, &tot);
      B.cellOff[c] = ex;
      if (threadIdx.x == 0) B.tileCnt[a] = tot;
    } else {
      uint32_t t = B.dropped[a - nA], c = t * 512u + threadIdx.x;
      B.cnt[c] = 0; B.cntOther[c] = 0; B.ctype[c] = 0u; B.pres[c] = 0.0f; B.rhs[c] = 8.0f; B.sorInfo[c] = 0; B.wet[c] = 0.0f;
      for (int p = 0; p < 6; p++) B.acc[p * nc + c] = 0;
      for (int p = 0; p < 3; p++) { B.vn[p * nc + c] = 0.0f; B.vo[p * nc + c] = 0.0f; B.velG[p * nc + c] = 0.0f; }
    }
  }
}

// Exclusive scan of up to a few hundred thousand counts by one CTA; block 0 scans the per-tile particle counts
// (total = live particles), block 1 the per-block dead counts. arr[n] receives the total.
__global__ void __launch_bounds__(1024) k_scan_counts(Bufs B) {
  __shared__ uint32_t sm[33];
  if (blockIdx.x == 0) scanOne(B.tileCnt, B.ctl->nActive, &B.ctl->nLive, sm);
  else scanOne(B.blkDead, B.nblk, nullptr, sm);
}

// ---- 4. scatter: sorted position of every particle ----
// Live: (tile offset + cell offset + rank from the atomic count); the order inside a cell is fixed to ascending id by
// p2g. Dead: after all live ones, in storage order (a block scan keeps it stable); they are moved here directly.
__global__ void __launch_bounds__(CM_T, 6) k_scatter(Bufs B) {
  __shared__ FlipParams P;
  __shared__ uint32_t sm[33];
  loadParams(P, B.P);
  uint32_t idx[CM_U], k[CM_U], r[CM_U], rk[CM_U], id[CM_U], a[CM_U], off[CM_U];
  bool dead[CM_U];
#pragma unroll
  for (int u = 0; u < CM_U; u++) {
    idx[u] = blockIdx.x * PBLK + u * CM_T + threadIdx.x;
    k[u] = idx[u] < P.n ? B.key[idx[u]] : 0u;
  }
#pragma unroll
  for (int u = 0; u < CM_U; u++) {
    dead[u] = idx[u] < P.n && k[u] == DEADKEY;
    if (idx[u] < P.n) {
      id[u] = B.idb[idx[u]];
      if (!dead[u]) { a[u] = B.tileSlot[k[u] >> 9]; off[u] = B.cellOff[k[u]]; rk[u] = B.rank[idx[u]]; }
    }
  }
  // dead ranks in storage order (slice by slice): two slices per scan in 16-bit fields (a slice has at most CM_T)
  uint32_t t01, t23;
  const uint32_t e01 = blockExclusive((dead[0] ? 1u : 0u) | (dead[1] ? 0x10000u : 0u), sm, &t01);
  const uint32_t e23 = blockExclusive((dead[2] ? 1u : 0u) | (dead[3] ? 0x10000u : 0u), sm, &t23);
  r[0] = e01 & 0xffffu;
  r[1] = (t01 & 0xffffu) + (e01 >> 16);
  r[2] = (t01 & 0xffffu) + (t01 >> 16) + (e23 & 0xffffu);
  r[3] = (t01 & 0xffffu) + (t01 >> 16) + (t23 & 0xffffu) + (e23 >> 16);
#pragma unroll
  for (int u = 0; u < CM_U; u++) {
    if (idx[u] >= P.n) continue;
    if (!dead[u]) {
      const uint32_t pos = B.tileCnt[a[u]] + off[u] + rk[u];
      B.srcIdx[pos] = idx[u];
      B.spid[pos] = id[u];
    } else {
      const uint32_t pos = B.ctl->nLive + B.blkDead[blockIdx.x] + r[u];
      B.pa[pos] = B.pb[idx[u]];
      B.ida[pos] = id[u];
    }
  }
}

// ---- 5. p2g (wgsl-solver.js:17-40) ----
// One CTA per tile with storage. Its particles (a contiguous sorted segment) are gathered from the previous order,
// written to their final place (ascending id inside each cell) and splatted into a 10^3-cell shared-memory window
// (the tile plus one cell around it) in the reference's fixed point: i32(round(w * v * 65536)) and i32(round(w * 65536)).
// Integer sums do not depend on order, so the window is flushed to HBM with plain atomic adds.
// The tile's cell offsets and counts are staged in shared memory first; the in-cell rank is the number of ids below
// the particle's in its cell. A particle whose corner faces need no clamping (the usual case) splats with window offsets
// fixed at compile time. Chunks of 256 particles go through two phases. The move (gather from the previous order, in-cell rank, write to the
// final place) runs with a warp's lanes on consecutive particles, so its global loads and stores are coalesced and
// the lanes of one cell read the same ids (L1 broadcasts); it leaves each particle's position and velocity in shared
// memory. The splat then takes them back with a warp's lanes 8 particles apart (different cells, so the window atomics
// rarely collide), from a layout padded by one word per 32 so those reads hit 32 different banks. Five CTAs share an
// SM (48 registers, 34 KB of shared memory each; with the tiles taken dynamically five beat four, 1.42 -> 1.37 ms at
// 256^3, and six spill); staging the tile's ids in shared memory, a second staging buffer and window strides padded
// against bank conflicts (24 / 256 words) all measured slower.
constexpr int P2G_T = 256;
constexpr int P2G_SW = P2G_T + P2G_T / 32;
struct P2GSmem {
  int32_t win[6][1000];
  uint32_t soff[512];
  int32_t scnt[512];
  float stg[6][P2G_SW];
};
__device__ __forceinline__ int p2gSlot(uint32_t r) { return (int)(r + (r >> 5)); }
// The 8 corners of one axis for a particle whose corner faces all lie in the window without clamping (the tile is at
// least a cell away from every wall, and corner (0,0,0) has window coordinates in [0, 8]): window offsets are
// compile-time constants from the base, weights are the reference's ((wx * wy) * wz) with the xy products shared, and
// each sum is i32(round(w * v * 65536)) / i32(round(w * 65536)) as in the general path.
__device__ __forceinline__ void splatAxisFast(int32_t* __restrict__ pv, int32_t* __restrict__ pw, V3 fr, float vc, float scale) {
  const float wx0 = 1.0f - fr.x, wx1 = fr.x, wy0 = 1.0f - fr.y, wy1 = fr.y, wz0 = 1.0f - fr.z, wz1 = fr.z;
  const float wxy[4] = {wx0 * wy0, wx1 * wy0, wx0 * wy1, wx1 * wy1};
#pragma unroll
  for (int c = 0; c < 8; c++) {
    const int off = (c & 1) + 10 * ((c >> 1) & 1) + 100 * (c >> 2);
    const float w = wxy[c & 3] * ((c & 4) ? wz1 : wz0);
    if (!(w <= 0.0f)) {
      atomicAdd(pv + off, __float2int_rn(w * vc * scale));
      atomicAdd(pw + off, __float2int_rn(w * scale));
    }
  }
}
__device__ __forceinline__ void p2gSplat(const FlipParams& P, P2GSmem& S, V3 p, V3 v, int ox, int oy, int oz, bool inner) {
  for (int axis = 0; axis < 3; axis++) {
    V3 g = (p - v3(P.x0, P.y0, P.z0)) * P.ih;
    if (axis == 0) { g.y -= 0.5f; g.z -= 0.5f; } else if (axis == 1) { g.x -= 0.5f; g.z -= 0.5f; } else { g.x -= 0.5f; g.y -= 0.5f; }
    const V3 f0 = vfloor(g), fr = g - f0;
    const int i0 = gidx(f0.x), j0 = gidx(f0.y), k0 = gidx(f0.z);
    const float vc = comp3(v, axis);
    const int bx = i0 - ox + 1, by = j0 - oy + 1, bz = k0 - oz + 1;
    if (inner && (unsigned)bx <= 8u && (unsigned)by <= 8u && (unsigned)bz <= 8u) {
      const int wb = bx + 10 * (by + 10 * bz);
      splatAxisFast(&S.win[axis][wb], &S.win[3 + axis][wb], fr, vc, P.scale);
      continue;
    }
    for (int c = 0; c < 8; c++) {
      const int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
      const float w = (dx == 1 ? fr.x : 1.0f - fr.x) * (dy == 1 ? fr.y : 1.0f - fr.y) * (dz == 1 ? fr.z : 1.0f - fr.z);
      if (w <= 0.0f) continue;
      int fi = i0 + dx, fj = j0 + dy, fk = k0 + dz;   // the face's cell, clamped as faceIndex does
      if (axis == 0) { fi = clampi(fi, 0, (int)P.nx); fj = clampi(fj, 0, (int)P.ny - 1); fk = clampi(fk, 0, (int)P.nz - 1); }
      else if (axis == 1) { fi = clampi(fi, 0, (int)P.nx - 1); fj = clampi(fj, 0, (int)P.ny); fk = clampi(fk, 0, (int)P.nz - 1); }
      else { fi = clampi(fi, 0, (int)P.nx - 1); fj = clampi(fj, 0, (int)P.ny - 1); fk = clampi(fk, 0, (int)P.nz); }
      const int widx = (fi - ox + 1) + 10 * ((fj - oy + 1) + 10 * (fk - oz + 1));
      atomicAdd(&S.win[axis][widx], (int32_t)rintf(w * vc * P.scale));
      atomicAdd(&S.win[3 + axis][widx], (int32_t)rintf(w * P.scale));
    }
  }
}
__global__ void __launch_bounds__(P2G_T, 5) k_p2g(Bufs B) {
  extern __shared__ __align__(16) unsigned char p2gRaw[];
  P2GSmem& S = *reinterpret_cast<P2GSmem*>(p2gRaw);
  __shared__ FlipParams P;
  loadParams(P, B.P);
  const uint32_t nA = B.ctl->nActive, nc = B.ncell;
  const uint32_t tid = threadIdx.x, splatPos = (tid & 31) * 8 + (tid >> 5);
  __shared__ uint32_t tileSlot;
  for (;;) {
    const uint32_t a = nextTile(B.ctl, &tileSlot);
    if (a >= nA) break;
    const uint32_t t = B.active[a];
    const uint32_t tt = t / P.tx;
    const int ox = (int)((t % P.tx) * 8u), oy = (int)((tt % P.ty) * 8u), oz = (int)((tt / P.ty) * 8u);
    const uint32_t s0 = B.tileCnt[a], s1 = B.tileCnt[a + 1], n = s1 - s0;
    // clamping of face indices (faceIndex) is the identity for every corner of this tile's particles
    const bool inner = ox >= 1 && oy >= 1 && oz >= 1 && ox + 9 <= (int)P.nx && oy + 9 <= (int)P.ny && oz + 9 <= (int)P.nz;
    for (int r = tid; r < 6000; r += P2G_T) (&S.win[0][0])[r] = 0;
    for (int r = tid; r < 512; r += P2G_T) { S.soff[r] = B.cellOff[t * 512u + r]; S.scnt[r] = B.cnt[t * 512u + r]; }
    __syncthreads();
    // the move of one chunk: particle s = s0 + chunk * 256 + tid, already loaded into q
    auto move = [&](uint32_t ch, const Part& q) {
      const uint32_t s = s0 + ch * P2G_T + tid;
      if (s >= s1) return;
      const uint32_t myid = B.spid[s];
      int ci, cj, ck;
      particleCell(P, xyz(q.p), ci, cj, ck);
      const uint32_t key = cellIdx(P, ci, cj, ck), lk = key - t * 512u;
      uint32_t cs, ce;
      if (lk < 512u) { cs = s0 + S.soff[lk]; ce = cs + (uint32_t)S.scnt[lk]; }
      else { cs = s0 + B.cellOff[key]; ce = cs + (uint32_t)B.cnt[key]; }
      uint32_t rk = 0;
      for (uint32_t u = cs; u < ce; u++) rk += B.spid[u] < myid ? 1u : 0u;
      B.pa[cs + rk] = q;
      B.ida[cs + rk] = myid;
      const int k = p2gSlot(tid);
      S.stg[0][k] = q.p.x; S.stg[1][k] = q.p.y; S.stg[2][k] = q.p.z;
      S.stg[3][k] = q.v.x; S.stg[4][k] = q.v.y; S.stg[5][k] = q.v.z;
    };
    const uint32_t nch = (n + P2G_T - 1) / P2G_T;
    // the next chunk's particle is loaded while this chunk is splatted
    Part qn;
    if (tid < n) qn = B.pb[B.srcIdx[s0 + tid]];
    for (uint32_t ch = 0; ch < nch; ch++) {
      move(ch, qn);
      if ((ch + 1) * P2G_T + tid < n) qn = B.pb[B.srcIdx[s0 + (ch + 1) * P2G_T + tid]];
      __syncthreads();
      if (ch * P2G_T + splatPos < n) {
        const int k = p2gSlot(splatPos);
        const V3 p = v3(S.stg[0][k], S.stg[1][k], S.stg[2][k]);
        const V3 v = v3(S.stg[3][k], S.stg[4][k], S.stg[5][k]);
        p2gSplat(P, S, p, v, ox, oy, oz, inner);
      }
      __syncthreads();
    }
    for (int r = tid; r < 1000; r += P2G_T) {
      const int gi = ox + (r % 10) - 1, gj = oy + (r / 10) % 10 - 1, gk = oz + r / 100 - 1;
      if (gi < 0 || gj < 0 || gk < 0 || gi >= (int)P.tx * 8 || gj >= (int)P.ty * 8 || gk >= (int)P.tz * 8) continue;
      const uint32_t c = cellIdx(P, gi, gj, gk);
      for (int pl = 0; pl < 6; pl++) {
        const int32_t v = S.win[pl][r];
        if (v != 0) atomicAdd(&B.acc[pl * nc + c], v);
      }
    }
    __syncthreads();
  }
  tilesDone(B.ctl);
}

// ---- 6. collider bits (solidBuild, wgsl-solver.js:42-45) + classify (wgsl-solver.js:47-74) ----
// OCEAN: compiled with the ocean's boundary (an ocean scene) or without it, so the other scenes' kernels carry none
// of its code or registers
template <bool OCEAN>
__global__ void __launch_bounds__(512) k_classify(Bufs B) {
  __shared__ FlipParams P;
  loadParams(P, B.P);
  const uint32_t nA = B.ctl->nActive, nc = B.ncell;
  for (uint32_t a = blockIdx.x; a < nA; a += gridDim.x) {
    const uint32_t t = B.active[a], c = t * 512u + threadIdx.x;
    int i, j, k;
    tileCoord(P, t, threadIdx.x, i, j, k);
    const V3 cx = cellCenter(P, i, j, k);
    uint32_t ct = B.ctype[c];
    ct = (ct & 0xffff00ffu) | ((uint32_t)(colAt(P, B.cols, B.sdf, cx) + 1) << 8);
    const uint32_t sb = ct & 0xffffff00u;
    const int32_t n = B.cnt[c];
    uint32_t ty = 0;
    if (!inDom(P, i, j, k)) ty = 0;
    else if ((sb & 0xff00u) != 0u) ty = 2;
    else if (OCEAN && P.ocean != 0u && layerW(P, cx) >= 0.5f)   // the ocean's boundary: a wall moving with the waves
      ty = cx.y < oceanEta(P, B.waves, cx.x, cx.z) ? 2u : 0u;
    else {
      // fluid when the narrow band holds deep water here (deeper than the band, or calm) or when particles are here
      // and the sheet does not tear. Either makes the cell fluid, so the particle test runs first: the calm test's 24
      // kept-velocity loads are only needed for a cell that the particles leave air (in a full-depth band, few).
      bool fl = false;
      if (n > 0) {
        fl = true;
        if ((float)n < P.sheetMin) {
          const int32_t dth = (int32_t)ceilf(0.6f * P.rest);
          bool dense = false;
          for (int q = 0; q < 6; q++) {
            int qi = i, qj = j, qk = k;
            if (q == 0) qi -= 1; else if (q == 1) qi += 1; else if (q == 2) qj -= 1; else if (q == 3) qj += 1; else if (q == 4) qk -= 1; else qk += 1;
            if (!inDom(P, qi, qj, qk)) continue;
            if (B.cnt[cellIdx(P, qi, qj, qk)] >= dth) dense = true;
          }
          fl = dense;
        }
      }
      if (!fl && P.nb != 0u && phiOfBits(ct) < -1.0f &&
          (phiOfBits(ct) < -P.band || len3(velGVec(P, B.velG, nc, cx)) < 9.0f * P.h)) fl = true;
      ty = fl ? 1u : 0u;
    }
    B.ctype[c] = ty | sb;
    if (ty != 1u) B.pres[c] = 0.0f;
    const uint32_t nf = __syncthreads_count(ty == 1u);
    if (threadIdx.x == 0 && nf) {
      atomicAdd(&B.ctl->fluid, nf);
      B.fluidTiles[atomicAdd(&B.ctl->nFluidTiles, 1u)] = t;   // the pressure sweeps visit only these (order free)
    }
  }
}

// ---- 7. normFaces (wgsl-solver.js:75-105) fused with divergence (wgsl-solver.js:107-123) ----
// normBody: the face velocity from the fixed-point sums, gravity on y faces, collider or wall velocity on solid faces.
__device__ __forceinline__ int colAtCell(const FlipParams& P, const uint32_t* __restrict__ ctype, int i, int j, int k) {
  if (!inDom(P, i, j, k)) return -1;
  return (int)((ctype[cellIdx(P, i, j, k)] >> 8) & 0xffu) - 1;
}
template <bool OCEAN>
__device__ __forceinline__ void normBody(const FlipParams& P, const Bufs& B, int axis, int i, int j, int k, uint32_t c, float& vOut, float& oldOut) {
  int li = i, lj = j, lk = k;
  if (axis == 0) li -= 1; else if (axis == 1) lj -= 1; else lk -= 1;
  const uint32_t tl = ctypeOf(P, B.ctype, li, lj, lk), th = ctypeOf(P, B.ctype, i, j, k);
  const int32_t ws = B.acc[(3 + axis) * B.ncell + c], vs = B.acc[axis * B.ncell + c];
  float v = ws > 0 ? (float)vs / (float)max(ws, 1) : 0.0f;
  float old = v;
  if (axis == 1) v -= P.gravity * P.dt;
  if (tl == 2u || th == 2u) {
    float sv = 0.0f;
    int ci = -1;
    if (tl == 2u) ci = colAtCell(P, B.ctype, li, lj, lk);
    if (ci < 0 && th == 2u) ci = colAtCell(P, B.ctype, i, j, k);
    if (ci >= 0) sv = comp3(colSurfVel(B.cols, (uint32_t)ci, facePos(P, i, j, k, axis)), axis);
    else if (OCEAN && P.ocean != 0u && ((tl == 2u && inDom(P, li, lj, lk)) || (th == 2u && inDom(P, i, j, k))))
      sv = comp3(oceanVel(P, B.waves, facePos(P, i, j, k, axis)), axis);
    v = sv;
    old = sv;
  }
  vOut = v;
  oldOut = old;
}
template <bool OCEAN>
__global__ void __launch_bounds__(512, 3) k_norm_div(Bufs B) {
  __shared__ FlipParams P;
  __shared__ float svn[3][512];
  __shared__ float shi[3][64];   // the faces just past the tile's high side, per axis, (other two local coordinates)
  loadParams(P, B.P);
  const uint32_t nA = B.ctl->nActive, nc = B.ncell;
  const int lx = threadIdx.x & 7, ly = (threadIdx.x >> 3) & 7, lz = threadIdx.x >> 6;
  const int NX = (int)P.tx * 8, NY = (int)P.ty * 8, NZ = (int)P.tz * 8;
  __shared__ uint32_t walk[2];
  TileWalk w{B.ctl, walk};
  for (uint32_t a = w.begin(); a < nA; a = w.next()) {
    w.fetch();
    const uint32_t t = B.active[a], c = t * 512u + threadIdx.x;
    int i, j, k;
    tileCoord(P, t, threadIdx.x, i, j, k);
    for (int axis = 0; axis < 3; axis++) {
      float v, old;
      normBody<OCEAN>(P, B, axis, i, j, k, c, v, old);
      B.vn[axis * nc + c] = v;
      B.vo[axis * nc + c] = old;
      svn[axis][threadIdx.x] = v;
    }
    // the divergence of the tile's high layer needs the neighbour tiles' first faces: six whole warps compute them
    // (a face outside the tile box is never read: fluid cells lie inside the domain, which the box exceeds by a cell)
    if (threadIdx.x < 192) {
      const int ax = threadIdx.x >> 6, f0 = threadIdx.x & 7, f1 = (threadIdx.x >> 3) & 7;
      const int fi = i - lx + (ax == 0 ? 8 : f0), fj = j - ly + (ax == 0 ? f0 : ax == 1 ? 8 : f1), fk = k - lz + (ax == 2 ? 8 : f1);
      float d = 0.0f, o2;
      if (fi < NX && fj < NY && fk < NZ) normBody<OCEAN>(P, B, ax, fi, fj, fk, cellIdx(P, fi, fj, fk), d, o2);
      shi[ax][threadIdx.x & 63] = d;
    }
    __syncthreads();
    const uint32_t ct = B.ctype[c];
    {   // wetCell (wgsl-whitewater.js:7-12): types, depth and counts are final for this step from here on
      float wv = 0.0f;
      if (inDom(P, i, j, k)) wv = (P.nb != 0u && (ct & 0xffu) == 1u && phiOfBits(ct) < -1.0f) ? 1.0f : fmn((float)B.cnt[c] / P.rest, 1.0f);
      B.wet[c] = wv;
    }
    if ((ct & 0xffu) != 1u) {
      B.rhs[c] = 0.0f;
      B.sorInfo[c] = 0;
    } else {
      const float vxp = lx < 7 ? svn[0][threadIdx.x + 1] : shi[0][ly + 8 * lz];
      const float vyp = ly < 7 ? svn[1][threadIdx.x + 8] : shi[1][lx + 8 * lz];
      const float vzp = lz < 7 ? svn[2][threadIdx.x + 64] : shi[2][lx + 8 * ly];
      const float div = (vxp - svn[0][threadIdx.x] + vyp - svn[1][threadIdx.x] + vzp - svn[2][threadIdx.x]) * P.ih;
      bool interior = true;
      uint32_t mask = 0, nns = 0;
      for (int q = 0; q < 6; q++) {
        int qi = i, qj = j, qk = k;
        if (q == 0) qi -= 1; else if (q == 1) qi += 1; else if (q == 2) qj -= 1; else if (q == 3) qj += 1; else if (q == 4) qk -= 1; else qk += 1;
        const uint32_t ty = ctypeOf(P, B.ctype, qi, qj, qk);
        if (ty == 0u) interior = false;
        if (ty != 2u) nns++;
        if (ty == 1u) mask |= 1u << q;
      }
      const float dens = (float)B.cnt[c] / P.rest - 1.0f;
      float tgt = P.comp * (interior ? dens : fmx(dens, 0.0f));
      if (P.nb != 0u && phiOfBits(ct) < -1.0f) tgt = 0.0f;
      B.rhs[c] = (tgt - div) * P.h * P.h / P.dt;
      B.sorInfo[c] = (uint16_t)(0x8000u | (nns << 8) | mask);
    }
  }
  w.done();
}

// ---- 8. red-black SOR (relax, wgsl-solver.js:124-140; rbRed/rbBlack :162-164) ----
// One CTA per tile holding fluid, one thread per cell of the colour. sorInfo (from classify's types) says which
// neighbours are fluid and how many are not solid. All eight loads of a cell are issued together from addresses that
// are always valid (a missing neighbour reads the cell itself); the sum then adds only the fluid neighbours, in the
// reference's order, so the arithmetic is unchanged.
// The sweeps run on a compact copy of the fluid tiles: per tile its red cells then its black ones, each half ordered
// (lx / 2) + 4 (ly + 8 lz). A warp's cells and each of its six neighbour loads are then contiguous runs of the other
// colour's half (a face neighbour across the tile boundary comes from the neighbour tile's copy), instead of touching
// whole 32-byte sectors of neighbour tiles for one value each. Same arithmetic, same order per cell.
__global__ void k_sor_slots(Bufs B) {
  const uint32_t nT = B.ctl->nFluidTiles;
  for (uint32_t a = blockIdx.x * blockDim.x + threadIdx.x; a < nT; a += gridDim.x * blockDim.x) B.slotOf[B.fluidTiles[a]] = a;
}
__device__ __forceinline__ uint32_t splitIdx(uint32_t local) {
  const uint32_t lx = local & 7u, ly = (local >> 3) & 7u, lz = local >> 6;
  return ((lx + ly + lz) & 1u) * 256u + (lx >> 1) + 4u * (ly + 8u * lz);
}
__global__ void __launch_bounds__(512) k_sor_pack(Bufs B) {
  __shared__ FlipParams P;
  loadParams(P, B.P);
  const uint32_t nT = B.ctl->nFluidTiles, O = *B.poolOff;
  for (uint32_t a = blockIdx.x; a < nT; a += gridDim.x) {
    const uint32_t t = B.fluidTiles[a], c = t * 512u + threadIdx.x, d = (O + a) * 512u + splitIdx(threadIdx.x);
    B.cp[d] = B.pres[c];
    B.crhs[d] = B.rhs[c];
    B.cinfo[d] = B.sorInfo[c];
    if (threadIdx.x == 6) B.pomega[O + a] = P.omega;
    if (threadIdx.x < 6) {
      const uint32_t tt = t / P.tx, ti = t % P.tx, tj = tt % P.ty, tk = tt / P.ty;
      const int dir = threadIdx.x;
      uint32_t n = 0xffffffffu;
      if (dir == 0 && ti > 0) n = t - 1u;
      if (dir == 1 && ti + 1 < P.tx) n = t + 1u;
      if (dir == 2 && tj > 0) n = t - P.tx;
      if (dir == 3 && tj + 1 < P.ty) n = t + P.tx;
      if (dir == 4 && tk > 0) n = t - P.tx * P.ty;
      if (dir == 5 && tk + 1 < P.tz) n = t + P.tx * P.ty;
      const uint32_t sl = n != 0xffffffffu ? B.slotOf[n] : 0xffffffffu;
      B.nbs[(O + a) * 6u + dir] = O + (sl != 0xffffffffu ? sl : a);   // no fluid there: never summed, any valid cell will do
    }
  }
}
// one colour of one red-black iteration on the copied tile at position a (neighbour positions in nbs are absolute)
__device__ __forceinline__ void sorTile(float* cp, const float* __restrict__ crhs, const uint16_t* __restrict__ cinfo,
                                        const uint32_t* __restrict__ nbs, uint32_t a, float omega, uint32_t color, uint32_t j) {
  const uint32_t lz = j >> 5, ly = (j >> 2) & 7u;
  const uint32_t lx = 2u * (j & 3u) + ((ly + lz + color) & 1u), row = j & ~3u;
  const uint32_t own = color * 256u + j, oth = (color ^ 1u) * 256u;
  const uint32_t* nb = nbs + a * 6u;
  const uint32_t base = a * 512u + oth;
  const uint32_t ixm = lx > 0 ? base + row + ((lx - 1u) >> 1) : nb[0] * 512u + oth + row + 3u;
  const uint32_t ixp = lx < 7 ? base + row + ((lx + 1u) >> 1) : nb[1] * 512u + oth + row;
  const uint32_t iym = ly > 0 ? base + j - 4u : nb[2] * 512u + oth + j + 28u;
  const uint32_t iyp = ly < 7 ? base + j + 4u : nb[3] * 512u + oth + j - 28u;
  const uint32_t izm = lz > 0 ? base + j - 32u : nb[4] * 512u + oth + j + 224u;
  const uint32_t izp = lz < 7 ? base + j + 32u : nb[5] * 512u + oth + j - 224u;
  const uint32_t c = a * 512u + own;
  const uint32_t info = cinfo[c];
  const float p0 = cp[c], r0 = crhs[c];
  const float pxm = cp[ixm], pxp = cp[ixp], pym = cp[iym], pyp = cp[iyp], pzm = cp[izm], pzp = cp[izp];
  if (!(info & 0x8000u)) return;
  const uint32_t nns = (info >> 8) & 7u;
  if (nns == 0u) { cp[c] = 0.0f; return; }
  float sum = 0.0f;
  if (info & 1u) sum += pxm;
  if (info & 2u) sum += pxp;
  if (info & 4u) sum += pym;
  if (info & 8u) sum += pyp;
  if (info & 16u) sum += pzm;
  if (info & 32u) sum += pzp;
  const float pg = (r0 + sum) / (float)nns;
  cp[c] = p0 + omega * (pg - p0);
}
__global__ void __launch_bounds__(256) k_sor_c(Bufs B, uint32_t color) {
  // launched as a programmatic dependent of the previous sweep: its CTAs may become resident early, and wait here until
  // that sweep has finished and its writes are visible
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const uint32_t nT = B.ctl->nFluidTiles, O = *B.poolOff;
  const float omega = B.P->omega;
  for (uint32_t a = blockIdx.x; a < nT; a += gridDim.x) sorTile(B.cp, B.crhs, B.cinfo, B.nbs, O + a, omega, color, threadIdx.x);
}
// the sweeps of a pooled batch: every tank's copied tiles in one launch, each with its own tank's SOR factor
__global__ void __launch_bounds__(256) k_sor_pool(const PoolBufs Q, uint32_t color) {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const uint32_t nT = *Q.total;
  for (uint32_t a = blockIdx.x; a < nT; a += gridDim.x) sorTile(Q.cp, Q.crhs, Q.cinfo, Q.nbs, a, Q.pomega[a], color, threadIdx.x);
}
// The same sweeps as one persistent cooperative launch: every CTA walks its share of the pool, then waits for all CTAs
// at a grid barrier between colours. Each wait is bounded (limit_ns of the global timer): a barrier that runs out sets
// Q.err and every CTA returns after its current sweep, so the host gets ST_TIMEOUT and the context stays usable.
__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool gridBarrier(unsigned int* bar, unsigned int expect, unsigned int& gen, unsigned int* err, uint64_t limit_ns) {
  __syncthreads();
  if (threadIdx.x == 0) {
    gen++;
    __threadfence();
    atomicAdd(bar, 1u);
    const uint64_t t0 = gtimer();
    while (true) {
      unsigned int v;
      asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
      if (v >= gen * expect) break;
      if (*(volatile unsigned int*)err) break;
      if (gtimer() - t0 > limit_ns) { atomicOr(err, 1u); break; }
      __nanosleep(64);
    }
    __threadfence();
  }
  __syncthreads();
  return *(volatile unsigned int*)err == 0u;
}
__global__ void __launch_bounds__(256) k_sor_persist(const PoolBufs Q, int iters, unsigned int expect, uint64_t limit_ns) {
  const uint32_t nT = *Q.total;
  unsigned int gen = 0;
  for (int it = 0; it < iters; it++)
    for (uint32_t color = 0; color < 2; color++) {
      for (uint32_t a = blockIdx.x; a < nT; a += gridDim.x) sorTile(Q.cp, Q.crhs, Q.cinfo, Q.nbs, a, Q.pomega[a], color, threadIdx.x);
      __threadfence();
      if (!gridBarrier(Q.bar, expect, gen, Q.err, limit_ns)) return;
    }
}
// offsets of every tank's copied tiles in the pool (ascending tank order) and the pool's total; the barrier word cleared
__global__ void k_pool_plan(const PoolBufs Q, const Ctl* const* ctls, uint32_t ntanks) {
  if (threadIdx.x != 0) return;
  uint32_t o = 0;
  for (uint32_t k = 0; k < ntanks; k++) {
    Q.off[k] = o;
    o += ctls[k]->nFluidTiles;
  }
  *Q.total = o;
  *Q.bar = 0u;
}
// a barrier that expects more arrivals than the launch has: every wait runs out (the test of the bounded wait)
__global__ void __launch_bounds__(256) k_barrier_test(unsigned int* bar, unsigned int* err, unsigned int expect, uint64_t limit_ns) {
  unsigned int gen = 0;
  gridBarrier(bar, expect, gen, err, limit_ns);
}
// back into the grid; the slot map goes back to empty for the next step
__global__ void __launch_bounds__(512) k_sor_unpack(Bufs B) {
  const uint32_t nT = B.ctl->nFluidTiles, O = *B.poolOff;
  for (uint32_t a = blockIdx.x; a < nT; a += gridDim.x) {
    const uint32_t t = B.fluidTiles[a];
    B.pres[t * 512u + threadIdx.x] = B.cp[(O + a) * 512u + splitIdx(threadIdx.x)];
    if (threadIdx.x == 0) B.slotOf[t] = 0xffffffffu;
  }
}

// ---- 9. project (wgsl-solver.js:165-180) + saveVel (wgsl-narrowband.js:88-91) ----
// Also clears this step's fixed-point sums and the other cell-count buffer, ready for the next step.
__global__ void __launch_bounds__(512) k_project(Bufs B) {
  __shared__ FlipParams P;
  loadParams(P, B.P);
  const uint32_t nA = B.ctl->nActive, nc = B.ncell;
  for (uint32_t a = blockIdx.x; a < nA; a += gridDim.x) {
    const uint32_t t = B.active[a], c = t * 512u + threadIdx.x;
    int i, j, k;
    tileCoord(P, t, threadIdx.x, i, j, k);
    const uint32_t th = ctypeOf(P, B.ctype, i, j, k);
    for (int axis = 0; axis < 3; axis++) {
      int li = i, lj = j, lk = k;
      if (axis == 0) li -= 1; else if (axis == 1) lj -= 1; else lk -= 1;
      const uint32_t tl = ctypeOf(P, B.ctype, li, lj, lk);
      float vnew = B.vn[axis * nc + c];
      if (!(tl == 2u || th == 2u) && (tl == 1u || th == 1u)) {
        float pl = 0.0f, ph = 0.0f;
        if (tl == 1u) pl = B.pres[cellIdx(P, li, lj, lk)];
        if (th == 1u) ph = B.pres[c];
        vnew = vnew - P.dt * P.ih * (ph - pl);
        B.vn[axis * nc + c] = vnew;
      }
      if (P.nb) B.velG[axis * nc + c] = vnew;
    }
    for (int pl = 0; pl < 6; pl++) B.acc[pl * nc + c] = 0;
    B.cntOther[c] = 0;
  }
}

// ---- 10. g2p (wgsl-solver.js:208-275) with sampleBoth (wgsl-core.js:138-154) and collideP (wgsl-solver.js:185-197) ----
__device__ __forceinline__ void sampleBoth(const FlipParams& P, const Bufs& B, V3 p, V3& vn, V3& vo) {
  const uint32_t nc = B.ncell;
  float rn[3], ro[3];
  for (int axis = 0; axis < 3; axis++) {
    V3 g = (p - v3(P.x0, P.y0, P.z0)) * P.ih;
    if (axis == 0) { g.y -= 0.5f; g.z -= 0.5f; } else if (axis == 1) { g.x -= 0.5f; g.z -= 0.5f; } else { g.x -= 0.5f; g.y -= 0.5f; }
    const V3 f0 = vfloor(g), fr = g - f0;
    const int i0 = gidx(f0.x), j0 = gidx(f0.y), k0 = gidx(f0.z);
    float sn = 0.0f, so = 0.0f;
    for (int c = 0; c < 8; c++) {
      const int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
      const float w = (dx == 1 ? fr.x : 1.0f - fr.x) * (dy == 1 ? fr.y : 1.0f - fr.y) * (dz == 1 ? fr.z : 1.0f - fr.z);
      const uint32_t f = faceCell(P, axis, i0 + dx, j0 + dy, k0 + dz);
      sn += w * B.vn[axis * nc + f];
      so += w * B.vo[axis * nc + f];
    }
    rn[axis] = sn;
    ro[axis] = so;
  }
  vn = v3(rn[0], rn[1], rn[2]);
  vo = v3(ro[0], ro[1], ro[2]);
}
// Cheap tests that only skip colliders colNear (src/flip/wgsl-core.js:113-126) rejects, so collideP's result is
// unchanged. s: a world-space sphere around the near box (xyz centre, w radius^2; w = +inf when the rows are not a
// rotation): in exact arithmetic colNear(p) puts the local point inside the box centre cL +- half extents h, so
// |p - (pos + R^T cL)| < |h|. lo/hi: the near box in local coordinates, before colNear's division by the voxel size.
// Both carry slack (1% and one voxel) that covers rounding; wlo/whi bound the near box in world space and go first,
// six compares that reject most particles of a tank near a long collider such as a wall piston, whose sphere covers
// them. on = 0 when colNear always holds.
struct ColPre {
  float4 s, r0, r1, r2, pos, lo, hi;
  float4 wlo, whi;   // the near box's world-space bounding box (a tenth of a percent and 1e-5 wider), +-inf when unused
  int on;
};
__device__ ColPre colPre(const FlipParams& P, const float4* __restrict__ cols, uint32_t k) {
  ColPre X;
  const float4 a = cols[k * 8], b = cols[k * 8 + 1];
  X.r0 = cols[k * 8 + 2]; X.r1 = cols[k * 8 + 3]; X.r2 = cols[k * 8 + 4]; X.pos = cols[k * 8 + 5];
  const V3 r0 = xyz(X.r0), r1 = xyz(X.r1), r2 = xyz(X.r2), pos = xyz(X.pos);
  const float tol = 1.0e-4f, hw = b.w, m = fabsf(P.q0);
  X.on = (P.q10 > 0.5f || !(hw > 0.0f)) ? 0 : 1;
  const bool rot = fabsf(dot3(r0, r0) - 1.0f) < tol && fabsf(dot3(r1, r1) - 1.0f) < tol && fabsf(dot3(r2, r2) - 1.0f) < tol &&
                   fabsf(dot3(r0, r1)) < tol && fabsf(dot3(r0, r2)) < tol && fabsf(dot3(r1, r2)) < tol;
  const float sl = 0.01f * hw + hw;
  X.lo = make_float4(b.x - hw - m - sl, b.y - hw - m - sl, b.z - hw - m - sl, 0.0f);
  X.hi = make_float4(b.x + a.y * hw + m + sl, b.y + a.z * hw + m + sl, b.z + a.w * hw + m + sl, 0.0f);
  const V3 cL = v3(b.x + (a.y - 1.0f) * 0.5f * hw, b.y + (a.z - 1.0f) * 0.5f * hw, b.z + (a.w - 1.0f) * 0.5f * hw);
  const V3 h = v3((a.y + 1.0f) * 0.5f * hw + m, (a.z + 1.0f) * 0.5f * hw + m, (a.w + 1.0f) * 0.5f * hw + m);
  const V3 c = pos + r0 * cL.x + r1 * cL.y + r2 * cL.z;
  const float rad = len3(h) * 1.01f + hw;
  X.s = (X.on && rot) ? make_float4(c.x, c.y, c.z, rad * rad) : make_float4(0.0f, 0.0f, 0.0f, __int_as_float(0x7f800000));
  // world bounds of the local box [lo, hi]: the rows are orthonormal to 1e-4, so pos + R^T lp covers it up to that
  // relative error, far inside the box's voxel of slack; widened once more against the bounds' own rounding
  const float inf = __int_as_float(0x7f800000);
  X.wlo = make_float4(-inf, -inf, -inf, 0.0f);
  X.whi = make_float4(inf, inf, inf, 0.0f);
  if (X.on && rot) {
    const V3 cl = v3((X.lo.x + X.hi.x) * 0.5f, (X.lo.y + X.hi.y) * 0.5f, (X.lo.z + X.hi.z) * 0.5f);
    const V3 hl = v3((X.hi.x - X.lo.x) * 0.5f, (X.hi.y - X.lo.y) * 0.5f, (X.hi.z - X.lo.z) * 0.5f);
    const V3 wc = pos + r0 * cl.x + r1 * cl.y + r2 * cl.z;
    const V3 wh = v3(fabsf(r0.x) * hl.x + fabsf(r1.x) * hl.y + fabsf(r2.x) * hl.z, fabsf(r0.y) * hl.x + fabsf(r1.y) * hl.y + fabsf(r2.y) * hl.z,
                     fabsf(r0.z) * hl.x + fabsf(r1.z) * hl.y + fabsf(r2.z) * hl.z);
    const float e = 1.0e-5f * (1.0f + fabsf(wc.x) + fabsf(wc.y) + fabsf(wc.z) + len3(hl));
    X.wlo = make_float4(wc.x - wh.x * 1.001f - e, wc.y - wh.y * 1.001f - e, wc.z - wh.z * 1.001f - e, 0.0f);
    X.whi = make_float4(wc.x + wh.x * 1.001f + e, wc.y + wh.y * 1.001f + e, wc.z + wh.z * 1.001f + e, 0.0f);
  }
  return X;
}
// collideP (src/flip/wgsl-solver.js:185-197) with the cheap tests first; wall[0], wall[1]: the clamp box (wallBox).
// cmask: the colliders whose near box the tile's particles can reach (tileColliders); the others are skipped until a
// push-out has moved the particle, after which every later collider is tested as the reference tests it.
__device__ __forceinline__ V3 collidePB(const FlipParams& P, const Bufs& B, const ColPre* pre, const float4* wall, uint32_t cmask,
                                        V3 pin) {
  V3 p = pin;
  bool moved = false;
  for (uint32_t k = 0; cmask != 0u && k < P.ncols; k++) {
    if (!moved && !((cmask >> k) & 1u)) continue;
    const ColPre& X = pre[k];
    if (p.x < X.wlo.x || p.y < X.wlo.y || p.z < X.wlo.z || p.x > X.whi.x || p.y > X.whi.y || p.z > X.whi.z) continue;
    const V3 d0 = p - xyz(X.s);
    if (dot3(d0, d0) > X.s.w) continue;
    if (X.on) {
      const V3 d = p - xyz(X.pos);
      const V3 lp = v3(dot3(xyz(X.r0), d), dot3(xyz(X.r1), d), dot3(xyz(X.r2), d));
      if (lp.x < X.lo.x || lp.y < X.lo.y || lp.z < X.lo.z || lp.x > X.hi.x || lp.y > X.hi.y || lp.z > X.hi.z) continue;
    }
    if (!colNear(P, B.cols, k, p)) continue;
    float phi; V3 wn;
    sdfEval(B.cols, B.sdf, k, p, phi, wn);
    if (phi < P.q0) { p = p + wn * (P.q0 - phi); moved = true; }
  }
  const float4 lo = wall[0], hi = wall[1];
  return vclamp(p, xyz(lo), xyz(hi));
}
// The colliders a particle of the tile at cell (ox, oy, oz) can reach before a push-out moves it: their near boxes'
// world bounds (ColPre wlo/whi) against the tile's cells grown by a cell (particleCell's rounding) and by the furthest
// a particle moves in a step (vmax dt: the speed is limited before the move), with slack for the bounds' rounding.
__device__ __forceinline__ uint32_t tileColliders(const FlipParams& P, const ColPre* pre, int ox, int oy, int oz) {
  const float pad = P.h * 1.01f + fabsf(P.vmax) * P.dt * 1.01f +
                    1.0e-5f * (1.0f + fabsf(P.x0) + fabsf(P.y0) + fabsf(P.z0) + fabsf(P.x1) + fabsf(P.y1) + fabsf(P.z1));
  const V3 lo = v3(P.x0 + (float)ox * P.h - pad, P.y0 + (float)oy * P.h - pad, P.z0 + (float)oz * P.h - pad);
  const V3 hi = v3(P.x0 + (float)(ox + 8) * P.h + pad, P.y0 + (float)(oy + 8) * P.h + pad, P.z0 + (float)(oz + 8) * P.h + pad);
  uint32_t m = 0;
  for (uint32_t k = 0; k < P.ncols; k++) {
    const ColPre& X = pre[k];
    if (!(hi.x < X.wlo.x || hi.y < X.wlo.y || hi.z < X.wlo.z || lo.x > X.whi.x || lo.y > X.whi.y || lo.z > X.whi.z)) m |= 1u << k;
  }
  return m;
}
// collideP's wall clamp box, the same for every particle: faces left open do not clamp
__device__ __forceinline__ void wallBox(const FlipParams& P, float4* wall) {
  const float big = 1.0e9f, m = P.margin;
  wall[0] = make_float4((P.open & 1u) ? -big : P.x0 + m, (P.open & 4u) ? -big : P.y0 + m, (P.open & 16u) ? -big : P.z0 + m, 0.0f);
  wall[1] = make_float4((P.open & 2u) ? big : P.x1 - m, (P.open & 8u) ? big : P.y1 - m, (P.open & 32u) ? big : P.z1 - m, 0.0f);
}
constexpr int G2P_T = 256;
// dynamic shared memory: the foam terms of count sums 0 .. G2P_LUT - 1 (float4), the tile's 729 count sums (int, padded
// to 16 bytes), then two particle slots per thread
constexpr int G2P_LUT = G2P_T;
constexpr int G2P_CSUM_OFF = G2P_LUT * 16, G2P_SLOT_OFF = G2P_CSUM_OFF + 2928;
constexpr int G2P_DYN = G2P_SLOT_OFF + 2 * G2P_T * 32;
// The particle update of g2p: p, v0 in; vn/vo and the counts come from the tile's shared-memory window.
struct G2PWin {
  const float2* v;   // [3][1000]: (vn, vo) of each face, one 64-bit load per corner
  const int32_t* csum;   // [9][9][9]: the summed counts of the 2 x 2 x 2 cells from (ox - 1, oy - 1, oz - 1) + (x, y, z)
  const float4* lut;     // [G2P_LUT]: foamCell of the count sums 0 .. G2P_LUT - 1
  const int32_t* cnt;
  const float* wet;      // wetCellAt of each window cell (0 outside the domain)
  const uint8_t* kill;   // the narrow band's trim test of each window cell
  const ColPre* cpre;    // collider pre-tests (colPre)
  const float4* wall;    // collideP's wall clamp box (wallBox)
  uint32_t cmask;        // the colliders this tile's particles can reach (tileColliders)
  int ox, oy, oz;
  __device__ __forceinline__ int idx(int i, int j, int k) const { return (i - ox + 1) + 10 * ((j - oy + 1) + 10 * (k - oz + 1)); }
  __device__ __forceinline__ bool has(int i, int j, int k) const {
    return (unsigned)(i - ox + 1) < 10u && (unsigned)(j - oy + 1) < 10u && (unsigned)(k - oz + 1) < 10u;
  }
};
struct WetWin {
  const G2PWin& W;
  __device__ __forceinline__ float operator()(int i, int j, int k) const { return W.wet[W.idx(i, j, k)]; }
};
__device__ __forceinline__ void sampleWin(const FlipParams& P, const G2PWin& W, V3 p, V3& vn, V3& vo) {
  float rn[3], ro[3];
  for (int axis = 0; axis < 3; axis++) {
    V3 g = (p - v3(P.x0, P.y0, P.z0)) * P.ih;
    if (axis == 0) { g.y -= 0.5f; g.z -= 0.5f; } else if (axis == 1) { g.x -= 0.5f; g.z -= 0.5f; } else { g.x -= 0.5f; g.y -= 0.5f; }
    const V3 f0 = vfloor(g), fr = g - f0;
    const int i0 = gidx(f0.x), j0 = gidx(f0.y), k0 = gidx(f0.z);
    // the clamped corner cells of faceIndex (wgsl-core.js:84-89): two candidates per axis
    const int hx = axis == 0 ? (int)P.nx : (int)P.nx - 1, hy = axis == 1 ? (int)P.ny : (int)P.ny - 1, hz = axis == 2 ? (int)P.nz : (int)P.nz - 1;
    const int xa = clampi(i0, 0, hx), xb = clampi(i0 + 1, 0, hx);
    const int ya = clampi(j0, 0, hy), yb = clampi(j0 + 1, 0, hy);
    const int za = clampi(k0, 0, hz), zb = clampi(k0 + 1, 0, hz);
    const float2* wv = W.v + axis * 1000;
    float sn = 0.0f, so = 0.0f;
    for (int c = 0; c < 8; c++) {
      const int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
      const float w = (dx == 1 ? fr.x : 1.0f - fr.x) * (dy == 1 ? fr.y : 1.0f - fr.y) * (dz == 1 ? fr.z : 1.0f - fr.z);
      const int f = W.idx(dx ? xb : xa, dy ? yb : ya, dz ? zb : za);
      const float2 fv = wv[f];
      sn += w * fv.x;
      so += w * fv.y;
    }
    rn[axis] = sn;
    ro[axis] = so;
  }
  vn = v3(rn[0], rn[1], rn[2]);
  vo = v3(ro[0], ro[1], ro[2]);
}
// The gust noise's hash lattice has spacing 1 in units of p * 0.55, so a whole tank spans only a few lattice points.
// Each CTA hashes them once into a table (the same hsh3 on the same integer-valued inputs, so the values are identical);
// points outside the table are hashed directly.
constexpr int GT_MAX = 256;   // lattice points per noise: 6^3 covers boxes up to about 3.5 m a side
struct GustTab {
  float2 v[3][GT_MAX];   // (hash at a lattice point, hash at the next point along x): one 64-bit load per pair
  int lo[3][3], n[3][3];
  bool on;
};
__device__ __forceinline__ float vnzTab(const GustTab& T, int which, V3 x) {
  const V3 i = vfloor(x), fr = x - vfloor(x);
  const V3 u = fr * fr * (v3(3.0f, 3.0f, 3.0f) - fr * 2.0f);
  const int ix = (int)i.x - T.lo[which][0], iy = (int)i.y - T.lo[which][1], iz = (int)i.z - T.lo[which][2];
  const int nx = T.n[which][0], ny = T.n[which][1], nz = T.n[which][2];
  if (!T.on || ix < 0 || iy < 0 || iz < 0 || ix + 1 >= nx || iy + 1 >= ny || iz + 1 >= nz) return vnz(x);
  const float2* t = T.v[which];
  const int b = ix + nx * (iy + ny * iz), sy = nx, sz = nx * ny;
  const float2 t0 = t[b], t1 = t[b + sy], t2 = t[b + sz], t3 = t[b + sz + sy];
  const float a = mixf(mixf(t0.x, t0.y, u.x), mixf(t1.x, t1.y, u.x), u.y);
  const float c = mixf(mixf(t2.x, t2.y, u.x), mixf(t3.x, t3.y, u.x), u.y);
  return mixf(a, c, u.z);
}
__device__ void buildGust(const FlipParams& P, GustTab& T) {
  const float tt = P.q8 * 0.6f;
  const float off[3][3] = {{tt, 0.0f, 0.0f}, {17.3f, tt, 4.1f}, {5.7f, 9.2f, tt}};
  const float lo3[3] = {P.x0, P.y0, P.z0}, hi3[3] = {P.x1, P.y1, P.z1};
  if (threadIdx.x == 0) {
    bool ok = P.q7 > 0.0f && P.q4 > 0.0f;
    for (int w = 0; w < 3; w++) {
      int cells = 1;
      for (int a = 0; a < 3; a++) {
        const int l = (int)floorf(lo3[a] * 0.55f + off[w][a]) - 1, h = (int)floorf(hi3[a] * 0.55f + off[w][a]) + 2;
        T.lo[w][a] = l;
        T.n[w][a] = h - l + 1;
        cells *= T.n[w][a];
      }
      if (cells > GT_MAX) ok = false;
    }
    T.on = ok;
  }
  __syncthreads();
  if (!T.on) return;
  for (int w = 0; w < 3; w++) {
    const int nx = T.n[w][0], ny = T.n[w][1], nz = T.n[w][2];
    for (int r = threadIdx.x; r < nx * ny * nz; r += blockDim.x) {
      const int ix = r % nx, iy = (r / nx) % ny, iz = r / (nx * ny);
      const V3 x = v3((float)(ix + T.lo[w][0]), (float)(iy + T.lo[w][1]), (float)(iz + T.lo[w][2]));
      T.v[w][r] = make_float2(hsh3(x), hsh3(v3((float)(ix + 1 + T.lo[w][0]), x.y, x.z)));
    }
  }
  __syncthreads();
}
// The three value-noise lookups of the gust, out of line: inlined, the scheduler hoists their table loads into the face
// sampling and g2p needs 156 registers; with this one call per particle it fits 80, so three CTAs of 256 threads share
// an SM (24 warps instead of 16; g2p 2.39 -> 2.10 ms at 256^3).
__device__ __noinline__ V3 gustAt(const GustTab& T, V3 gp, float tt) {
  return v3(vnzTab(T, 0, gp + v3(tt, 0.0f, 0.0f)), vnzTab(T, 1, gp + v3(17.3f, tt, 4.1f)), vnzTab(T, 2, gp + v3(5.7f, 9.2f, tt)));
}
// values of the particle update that depend only on the parameters, computed once per thread
struct G2PUni {
  float sens, settle, tau0, tt, v2lo, imp2lo, trb2lo;
};
__device__ __forceinline__ G2PUni g2pUni(const FlipParams& P) {
  // v2lo: below it |v|^2 cannot round to a speed above vmax (vmax^2 (1 - 2^-20) leaves room for both roundings).
  // imp2lo, trb2lo: below them |vn - vo|^2 and |v0 - vo|^2 cannot round to an impact or turbulence term above 0 (their
  // clamped ramps start at 15 sens / dt and 0.35 sens; the factor 1 - 2^-16 leaves room for every rounding on the way)
  const float sens = fmx(P.q6, 0.05f), a = 15.0f * sens * P.dt, b = 0.35f * sens;
  return G2PUni{sens, smoothstepf(0.1f, 0.5f, P.q8), fmx(P.q5, 0.05f), P.q8 * 0.6f, P.vmax * P.vmax * (1.0f - 1.0f / 1048576.0f),
                a * a * (1.0f - 1.0f / 65536.0f), b * b * (1.0f - 1.0f / 65536.0f)};
}
// The terms of g2p's particle update that depend only on the local density rho = csum / (8 rest) of the particle's
// 2 x 2 x 2 count sum (wgsl-solver.js:222-240): air, the foam decay exp(-dt / tau), the drag factor
// 1 - exp(-kd dt) and shield, in the reference's operations. In the default mode every particle of a tile takes its
// count sum from one of 729 corner cells, so g2p evaluates them once per corner cell into a shared-memory table instead
// of once per particle (two exp and five divisions).
__device__ __forceinline__ float4 foamCell(const FlipParams& P, const G2PUni& U, float csum) {
  const float rho = csum / (8.0f * P.rest);
  const float air = 1.0f - smoothstepf(0.008f, 0.1f, rho);
  const float shield = smoothstepf(0.1f, 0.65f, rho);
  const float exposure = 1.0f - 0.97f * shield;
  const float tau = U.tau0 * mixf(1.0f, 0.35f, smoothstepf(0.7f, 1.0f, rho)) * mixf(1.0f, 2.5f, air);
  const float kd = P.q4 * (0.04f + 1.5f * exposure * exposure);
  return make_float4(air, st_expf(-P.dt / tau), 1.0f - st_expf(-kd * P.dt), shield);
}
template <bool OCEAN>
__device__ __forceinline__ void g2pOne(const FlipParams& P, const Bufs& B, const G2PWin& W, const GustTab& T, const G2PUni& U, Part& q,
                                       float& speed) {
  const V3 p = xyz(q.p), v0 = xyz(q.v);
  V3 vn, vo;
  sampleWin(P, W, p, vn, vo);    // the particle's own tile has storage: it marked it this step
  V3 v = vmix(vn, v0 + (vn - vo), P.flip);
  if (OCEAN && P.ocean != 0u) {   // near the ocean's boundary, ease into the waves
    const float lw = layerW(P, p);
    if (lw > 0.0f) {
      const float s = clampf(lw * 2.0f, 0.0f, 1.0f);
      v = vmix(v, oceanVel(P, B.waves, p), s * s * (1.0f - st_expf(-8.0f * P.dt)));
    }
  }
  const V3 bcf = vfloor((p - v3(P.x0, P.y0, P.z0)) * P.ih - v3(0.5f, 0.5f, 0.5f));
  const int bi = gidx(bcf.x), bj = gidx(bcf.y), bk = gidx(bcf.z);
  const bool fast = P.q12 > 0.5f;
  float4 fc;
  float csum;
  bool direct = true;
  if (P.q9 < 0.5f && !fast) {
    // the sum depends on the corner only through its clamp into [-1, n - 1], which the tile's particles keep within
    // the staged 9^3 block (the outer clamp only keeps the shared-memory index in bounds)
    const int x = clampi(clampi(bi, -1, (int)P.nx - 1) - (W.ox - 1), 0, 8), y = clampi(clampi(bj, -1, (int)P.ny - 1) - (W.oy - 1), 0, 8);
    const int z = clampi(clampi(bk, -1, (int)P.nz - 1) - (W.oz - 1), 0, 8);
    const int32_t cs = W.csum[x + 9 * (y + 9 * z)];
    if ((uint32_t)cs < (uint32_t)G2P_LUT) { fc = W.lut[cs]; direct = false; }
    else csum = (float)cs;
  } else {
    int fi, fj, fk;
    particleCell(P, p, fi, fj, fk);
    csum = P.q9 < 0.5f ? 8.0f * (float)W.cnt[W.idx(fi, fj, fk)] : 8.0f * P.rest;
  }
  if (direct) fc = foamCell(P, U, csum);
  const float air = fc.x, shield = fc.w;
  const float sens = U.sens;
  const float settle = U.settle;
  // impact and turbulence are 0 unless |vn - vo| / dt and |v0 - vo| reach their ramps: the common calm particle skips
  // their square roots and divisions
  const V3 dvn = vn - vo, dv0 = v0 - vo;
  const float dvn2 = dot3(dvn, dvn), dv02 = dot3(dv0, dv0);
  float impact = 0.0f, turb = 0.0f;
  if (!(dvn2 < U.imp2lo)) {
    const float pacc = sqrtf(dvn2) / P.dt;
    impact = clampf((pacc / sens - 15.0f) / 80.0f, 0.0f, 1.0f) * settle;
  }
  if (!(dv02 < U.trb2lo)) turb = clampf((sqrtf(dv02) / sens - 0.35f) / 1.5f, 0.0f, 1.0f) * settle;
  // with no air around (air 0, the deep water) the spray term is 0 whatever the speed: its square root is skipped
  const float spray = air == 0.0f ? 0.0f : air * (0.25f + 0.75f * clampf(len3(v) / 4.0f, 0.0f, 1.0f));
  float foam = q.v.w * fc.y;
  foam = fmx(foam, fmx(spray * 0.9f, fmx(impact, turb * 0.8f)));
  if (OCEAN && P.ocean != 0u) foam *= 1.0f - clampf(layerW(P, p) * 2.0f, 0.0f, 1.0f);   // easing into the waves is not churning
  V3 gust = v3(0.0f, 0.0f, 0.0f);
  if (P.q7 > 0.0f && P.q4 > 0.0f && (!fast || shield < 0.9f)) {
    const V3 gp = p * 0.55f;
    const float tt = U.tt;
    gust = gustAt(T, gp, tt) * 2.0f - v3(1.0f, 1.0f, 1.0f);
  }
  const V3 airv = v3(P.q1, P.q2, P.q3) + gust * P.q7;
  v = v + (airv - v) * fc.z;
  const float sp2 = dot3(v, v);
  if (!(sp2 < U.v2lo)) {   // the speed limit; the common slow particle skips its square root
    const float sp = sqrtf(sp2);
    if (sp > P.vmax) v = v * (P.vmax / sp);
  }
  const V3 pt = p + v * P.dt;
  const V3 pc = collidePB(P, B, W.cpre, W.wall, W.cmask, pt);
  const V3 dsp = pc - pt;
  if (dot3(dsp, dsp) > 1.0e-12f) {
    const V3 nrm = dsp / len3(dsp);
    const float vd = dot3(v, nrm);
    if (vd < 0.0f) v = v - nrm * vd;
  }
  const uint32_t o = P.open;
  if (o != 0u && (((o & 1u) && pc.x < P.x0) || ((o & 2u) && pc.x > P.x1) || ((o & 4u) && pc.y < P.y0) ||
                  ((o & 8u) && pc.y > P.y1) || ((o & 16u) && pc.z < P.z0) || ((o & 32u) && pc.z > P.z1))) {
    q.p = make_float4(0.0f, -1.0e6f, 0.0f, 0.0f);
    q.v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    speed = 0.0f;
  } else {
    speed = len3(v);   // |q.v.xyz|, also for the emission and trim tests after the update
    q.p = make_float4(pc.x, pc.y, pc.z, fmn(speed, 63.0f) + 64.0f * floorf(foam * 15.0f + 0.5f));
    q.v = make_float4(v.x, v.y, v.z, foam);
  }
}
// One CTA per tile with storage: the tile's particles are one contiguous sorted segment, and every face and count they
// sample lies in the 10^3-cell window (the tile plus one cell around it), staged once in shared memory.
// 16-byte asynchronous copies from global to shared memory (cp.async): the data lands without passing through
// registers, and the issuing thread waits for it with cpAsyncWait before reading the slot
__device__ __forceinline__ void cpAsync16(void* smem, const void* gmem) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cpAsyncWait() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void cpAsyncPart(Part* slot, const Part* src) {
  cpAsync16(&slot->p, &src->p);
  cpAsync16(&slot->v, &src->v);
}
template <bool OCEAN>
__global__ void __launch_bounds__(G2P_T, 3) k_g2p(Bufs B) {
  __shared__ FlipParams P;
  __shared__ float2 wv[3 * 1000];
  __shared__ int32_t wcnt[1000];
  extern __shared__ __align__(16) unsigned char g2pDyn[];   // dynamic: the static arrays fill the 48 KB
  float4* const wlut = reinterpret_cast<float4*>(g2pDyn);
  int32_t* const wcsum = reinterpret_cast<int32_t*>(g2pDyn + G2P_CSUM_OFF);
  Part* const pslot = reinterpret_cast<Part*>(g2pDyn + G2P_SLOT_OFF);   // [2][G2P_T]: this thread's next particles
  __shared__ float wwet[1000];
  __shared__ uint8_t wkill[1000];
  __shared__ ColPre cpre[32];
  __shared__ float4 wall[2];
  __shared__ GustTab gtab;
  __shared__ uint32_t sm[33];
  loadParams(P, B.P);
  if (threadIdx.x < P.ncols) cpre[threadIdx.x] = colPre(P, B.cols, threadIdx.x);
  if (threadIdx.x == 0) wallBox(P, wall);
  // g2p's density terms depend on the local density only through the integer count sum of the particle's 2 x 2 x 2
  // corner cells: evaluated once per CTA for the sums below G2P_LUT, in the reference's operations (the same values)
  if (P.q9 < 0.5f && !(P.q12 > 0.5f)) {
    const G2PUni U0 = g2pUni(P);
    for (int r = threadIdx.x; r < G2P_LUT; r += G2P_T) wlut[r] = foamCell(P, U0, (float)r);
  }
  buildGust(P, gtab);   // its barriers also publish cpre, wall and wlut
  const uint32_t nA = B.ctl->nActive, nc = B.ncell;
  const int NX = (int)P.tx * 8, NY = (int)P.ty * 8, NZ = (int)P.tz * 8;
  __shared__ uint32_t tileSlot;
  for (;;) {
    const uint32_t a = nextTile(B.ctl, &tileSlot);
    if (a >= nA) break;
    const uint32_t t = B.active[a], tt = t / P.tx;
    const int ox = (int)((t % P.tx) * 8u), oy = (int)((tt % P.ty) * 8u), oz = (int)((tt / P.ty) * 8u);
    G2PWin W{wv, wcsum, wlut, wcnt, wwet, wkill, cpre, wall, tileColliders(P, cpre, ox, oy, oz), ox, oy, oz};
    // the trim (depth below the band) needs a band shallower than the deepest depth a cell word holds (8 - 65535 / 4096):
    // at full depth (band 1e4) no particle is ever trimmed and the test is left out
    const bool needWet = P.sprayOn != 0u && P.smax != 0u && P.sprRate > 0.0f, needKill = P.nb != 0u && P.band < 8.0f;
    const G2PUni U = g2pUni(P);
    for (int r = threadIdx.x; r < 1000; r += G2P_T) {
      const int gi = W.ox + r % 10 - 1, gj = W.oy + (r / 10) % 10 - 1, gk = W.oz + r / 100 - 1;
      if (gi < 0 || gj < 0 || gk < 0 || gi >= NX || gj >= NY || gk >= NZ) {   // faces here are never sampled (clamped)
        wwet[r] = 0.0f;
        wkill[r] = 0;
        continue;
      }
      const uint32_t c = cellIdx(P, gi, gj, gk);
      for (int ax = 0; ax < 3; ax++) wv[ax * 1000 + r] = make_float2(B.vn[ax * nc + c], B.vo[ax * nc + c]);
      wcnt[r] = B.cnt[c];
      if (needWet) wwet[r] = inDom(P, gi, gj, gk) ? B.wet[c] : 0.0f;
      if (needKill) wkill[r] = (B.on[c >> 9] && phiOfBits(B.ctype[c]) < -P.band) ? 1 : 0;
    }
    __syncthreads();
    // the local density's count sums (g2p's foam terms, wgsl-solver.js:222-229) of every corner a particle of this tile
    // can have (integers; the reference sums them as floats, exactly, so the float of this sum is its value)
    if (P.q9 < 0.5f && !(P.q12 > 0.5f)) {
      for (int r = threadIdx.x; r < 729; r += G2P_T) {
        const int bi = W.ox - 1 + r % 9, bj = W.oy - 1 + (r / 9) % 9, bk = W.oz - 1 + r / 81;
        const int xa = clampi(bi, 0, (int)P.nx - 1), xb = clampi(bi + 1, 0, (int)P.nx - 1);
        const int ya = clampi(bj, 0, (int)P.ny - 1), yb = clampi(bj + 1, 0, (int)P.ny - 1);
        const int za = clampi(bk, 0, (int)P.nz - 1), zb = clampi(bk + 1, 0, (int)P.nz - 1);
        int32_t cs = 0;
        for (int dz = 0; dz <= 1; dz++)
          for (int dy = 0; dy <= 1; dy++)
            for (int dx = 0; dx <= 1; dx++) cs += wcnt[W.idx(dx ? xb : xa, dy ? yb : ya, dz ? zb : za)];
        wcsum[r] = cs;
      }
      __syncthreads();
    }
    const uint32_t s0 = B.tileCnt[a], s1 = B.tileCnt[a + 1];
    uint32_t emitSum = 0, deadSum = 0;
    // each thread's next particle is copied into its shared-memory slot while it updates the current one (no registers
    // held for it); two slots, so a copy never lands in the slot being read
    if (s0 + threadIdx.x < s1) cpAsyncPart(&pslot[threadIdx.x], &B.pa[s0 + threadIdx.x]);
    cpAsyncCommit();
    uint32_t slot = 0;
    for (uint32_t i = s0 + threadIdx.x; i < s1; i += G2P_T) {
      cpAsyncWait();
      Part q = pslot[slot * G2P_T + threadIdx.x];
      slot ^= 1u;
      if (i + G2P_T < s1) cpAsyncPart(&pslot[slot * G2P_T + threadIdx.x], &B.pa[i + G2P_T]);
      cpAsyncCommit();
      float speed;
      g2pOne<OCEAN>(P, B, W, gtab, U, q, speed);
      // the whitewater each particle will throw off (sprayEmit's count, wgsl-whitewater.js:101-117) and the narrow band
      // trim of deep calm particles (nbKill, wgsl-narrowband.js:93-102), both from the moved particle
      const bool gone = q.p.y < DEADY;
      uint32_t kc = 0;
      // e is 0 (or NaN) unless the particle is fast enough for crest (speed over sprMin) or churn (over 0.5): the
      // common slow particle skips the eight wetness reads (kc stays 0 either way)
      const float xs = speed * P.vs;
      const bool oceanSide = OCEAN && P.ocean != 0u && !gone && layerW(P, xyz(q.p)) > 0.0f;   // no whitewater from the ocean's boundary
      if (!gone && needWet && !oceanSide && U.settle != 0.0f && (xs - P.sprMin > 0.0f || xs > 0.5f)) {
        float rho, fast, e;
        // the eight cells around the moved particle: from the window when it holds them
        const V3 bcf = vfloor((xyz(q.p) - v3(P.x0, P.y0, P.z0)) * P.ih - v3(0.5f, 0.5f, 0.5f));
        const int bi = gidx(bcf.x), bj = gidx(bcf.y), bk = gidx(bcf.z);
        if (W.has(bi, bj, bk) && W.has(bi + 1, bj + 1, bk + 1)) emitTermsT(P, WetWin{W}, q.p, q.v, rho, fast, e, U.settle);
        else emitTerms(P, B.wet, q.p, q.v, rho, fast, e);
        if (e > 0.0f) {
          const uint32_t h0 = B.ida[i] * 747796405u + P.seed * 2891336453u;
          kc = min(u32f(floorf(P.sprRate * e * P.dt + hash1(h0))), 4u);
        }
      }
      bool kill = false;
      if (oceanSide) {   // inside the ocean's boundary, or above the ocean's surface in its inner half
        const float lw = layerW(P, xyz(q.p));
        kill = lw >= 0.5f || (lw > 0.25f && q.p.y > oceanEta(P, B.waves, q.p.x, q.p.z) + 0.5f * P.h);
      }
      if (!kill && !gone && needKill && speed < 9.0f * P.h) {
        int ci, cj, ck;
        particleCell(P, xyz(q.p), ci, cj, ck);
        if (W.has(ci, cj, ck)) kill = W.kill[W.idx(ci, cj, ck)] != 0;
        else {
          const uint32_t cc = cellIdx(P, ci, cj, ck);
          kill = B.on[cc >> 9] && phiOfBits(B.ctype[cc]) < -P.band;
        }
      }
      // the trim waits for the points this particle throws off (written by the emit pass) and, with the air field
      // on, for the air splat, which still sees the particle (the reference trims in the reseed stage)
      const bool holdKill = kc != 0 || P.airOn != 0u;
      if (kill && !holdKill) {
        q.p = make_float4(0.0f, -1.0e6f, 0.0f, 0.0f);
        q.v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      }
      B.pa[i] = q;
      if (P.sprayOn != 0u) B.emitK[i] = (uint8_t)(kc | (kill && holdKill ? EMIT_KILL : 0u));
      if (P.nb != 0u) B.deadF[i] = (gone || kill) ? 1 : 0;
      emitSum += kc;
      deadSum += (gone || kill) ? 1u : 0u;
    }
    if (P.sprayOn != 0u || P.nb != 0u) {
      uint32_t te, td;
      blockExclusive(emitSum, sm, &te);
      blockExclusive(deadSum, sm, &td);
      if (threadIdx.x == 0) { B.tileEmit[a] = te; B.tileDead[a] = td; }
    }
    __syncthreads();
  }
  tilesDone(B.ctl);
}

// unsort for readback (wgsl-blocks.js:97-99): id order into dst (pos and vel)
__global__ void k_unsort(const Part* __restrict__ src, const uint32_t* __restrict__ ids, uint32_t n, float4* __restrict__ pos, float4* __restrict__ vel) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t id = ids[i];
    if (id >= n) continue;
    const Part q = src[i];
    pos[id] = q.p;
    if (vel) vel[id] = q.v;
  }
}

// the state an inactive tile holds (the reference's spare slot): rhs 8, everything else 0
__global__ void k_fill_f32(float* p, float v, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}
__global__ void k_iota(uint32_t* p, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = i;
}

// ---- launchers: each returns how many kernels it launched ----
int launch_count_mark(const Bufs& B, cudaStream_t s) { k_count_mark<<<B.nblk, CM_T, 0, s>>>(B); return 1; }
int launch_mark_phi(const Bufs& B, int grid, cudaStream_t s) { k_mark_phi<<<grid, 512, 0, s>>>(B); return 1; }
int launch_mark_fill(const Bufs& B, int grid, cudaStream_t s) { k_mark_fill<<<grid, 256, 0, s>>>(B); return 1; }
int launch_tiles(const Bufs& B, uint32_t ntiles, int grid, cudaStream_t s) {
  uint32_t nb = (ntiles + 1023) / 1024;
  k_tile_flags<<<nb, 1024, 0, s>>>(B);
  k_tile_list<<<nb, 1024, 0, s>>>(B);
  k_tile_prep<<<grid, 512, 0, s>>>(B);
  return 3;
}
int launch_scan_counts(const Bufs& B, cudaStream_t s) { k_scan_counts<<<2, 1024, 0, s>>>(B); return 1; }
int launch_scatter(const Bufs& B, cudaStream_t s) { k_scatter<<<B.nblk, CM_T, 0, s>>>(B); return 1; }
// CTAs of a kernel that fit on one SM at once (the dynamic-tile kernels are launched with no more than these)
static int residentPerSm(const void* fn, int threads, size_t dyn) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, dyn) != cudaSuccess || n < 1) n = 1;
  return n;
}
// The grid of a kernel that walks the tile list dynamically (TileWalk): no more CTAs than fit on the SMs at once (a CTA
// that starts after the list is taken only loads its parameters and leaves). Resident counts are cached per kernel.
static std::mutex g_walk_mu;
static std::unordered_map<const void*, int> g_walk_res;
int walk_grid(const void* fn, int threads, int grid) {
  int res;
  {
    std::lock_guard<std::mutex> lk(g_walk_mu);
    auto it = g_walk_res.find(fn);
    if (it == g_walk_res.end()) res = g_walk_res[fn] = residentPerSm(fn, threads, 0);
    else res = it->second;
  }
  int dev = 0, sms = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return std::max(1, std::min(grid, sms * res));
}
void warm_walk_grids_flip() {
  walk_grid((const void*)k_norm_div<false>, 512, 1);
  walk_grid((const void*)k_norm_div<true>, 512, 1);
}
int p2g_ctas_per_sm() {
  // the window, ids, offsets and staging buffers take more than the 48 KB of static shared memory
  cudaFuncSetAttribute(k_p2g, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(P2GSmem));
  static const int n = residentPerSm((const void*)k_p2g, P2G_T, sizeof(P2GSmem));
  return n;
}
int launch_p2g(const Bufs& B, int grid, cudaStream_t s) {
  cudaFuncSetAttribute(k_p2g, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(P2GSmem));
  k_p2g<<<grid, P2G_T, sizeof(P2GSmem), s>>>(B);
  return 1;
}
int launch_classify(const Bufs& B, int grid, bool ocean, cudaStream_t s) {
  if (ocean) k_classify<true><<<grid, 512, 0, s>>>(B);
  else k_classify<false><<<grid, 512, 0, s>>>(B);
  return 1;
}
int launch_norm_div(const Bufs& B, int grid, bool ocean, cudaStream_t s) {
  if (ocean) k_norm_div<true><<<walk_grid((const void*)k_norm_div<true>, 512, grid), 512, 0, s>>>(B);
  else k_norm_div<false><<<walk_grid((const void*)k_norm_div<false>, 512, grid), 512, 0, s>>>(B);
  return 1;
}
int launch_sor_pack(const Bufs& B, int grid4, cudaStream_t s) {
  k_sor_slots<<<64, 256, 0, s>>>(B);
  k_sor_pack<<<grid4, 512, 0, s>>>(B);
  return 2;
}
// iters red-black iterations, each colour a programmatic dependent launch of the one before (its launch overlaps the
// previous sweep's tail); the kernel is either a tank's own sweep or a pooled batch's
template <class Arg>
static int launch_sweeps(void (*kern)(Arg, uint32_t), const Arg& A, int grid, int iters, cudaStream_t s) {
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  for (int it = 0; it < iters; it++)
    for (uint32_t color = 0; color < 2; color++) cudaLaunchKernelEx(&cfg, kern, A, color);
  return 2 * iters;
}
int launch_sor_unpack(const Bufs& B, int grid4, cudaStream_t s) {
  k_sor_unpack<<<grid4, 512, 0, s>>>(B);
  return 1;
}
int launch_sor_compact(const Bufs& B, int grid, int grid4, int iters, cudaStream_t s) {
  int nl = launch_sor_pack(B, grid4, s);
  nl += launch_sweeps(k_sor_c, B, grid, iters, s);
  return nl + launch_sor_unpack(B, grid4, s);
}
int launch_pool_plan(const PoolBufs& Q, const Ctl* const* ctls, uint32_t ntanks, cudaStream_t s) {
  k_pool_plan<<<1, 32, 0, s>>>(Q, ctls, ntanks);
  return 1;
}
int launch_pool_sweeps(const PoolBufs& Q, int grid, int iters, cudaStream_t s) { return launch_sweeps(k_sor_pool, Q, grid, iters, s); }
cudaError_t launch_pool_persistent(const PoolBufs& Q, int grid, int iters, uint64_t limit_ns, cudaStream_t s) {
  unsigned int expect = (unsigned int)grid;
  int it = iters;
  void* args[] = {(void*)&Q, (void*)&it, (void*)&expect, (void*)&limit_ns};
  return cudaLaunchCooperativeKernel((const void*)k_sor_persist, dim3((unsigned)grid), dim3(256), args, 0, s);
}
int persistent_ctas_per_sm() {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_sor_persist, 256, 0);
  return n;
}
cudaError_t launch_barrier_test(unsigned int* bar, unsigned int* err, int grid, unsigned int expect, uint64_t limit_ns, cudaStream_t s) {
  void* args[] = {(void*)&bar, (void*)&err, (void*)&expect, (void*)&limit_ns};
  return cudaLaunchCooperativeKernel((const void*)k_barrier_test, dim3((unsigned)grid), dim3(256), args, 0, s);
}
int launch_project(const Bufs& B, int grid, cudaStream_t s) { k_project<<<grid, 512, 0, s>>>(B); return 1; }
static void g2pAttributes(bool ocean) {
  // three CTAs of about 68 KB each share an SM: ask for the largest shared-memory carveout
  if (ocean) {
    cudaFuncSetAttribute(k_g2p<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, G2P_DYN);
    cudaFuncSetAttribute(k_g2p<true>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  } else {
    cudaFuncSetAttribute(k_g2p<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, G2P_DYN);
    cudaFuncSetAttribute(k_g2p<false>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  }
}
int g2p_ctas_per_sm(bool ocean) {
  g2pAttributes(ocean);
  if (ocean) {
    static const int n = residentPerSm((const void*)k_g2p<true>, G2P_T, G2P_DYN);
    return n;
  }
  static const int n = residentPerSm((const void*)k_g2p<false>, G2P_T, G2P_DYN);
  return n;
}
int launch_g2p(const Bufs& B, int grid, bool ocean, cudaStream_t s) {
  g2pAttributes(ocean);
  if (ocean) k_g2p<true><<<grid, G2P_T, G2P_DYN, s>>>(B);
  else k_g2p<false><<<grid, G2P_T, G2P_DYN, s>>>(B);
  return 1;
}
int launch_unsort(const Part* src, const uint32_t* ids, uint32_t n, float4* pos, float4* vel, cudaStream_t s) {
  if (!n) return 0;
  k_unsort<<<(n + 255) / 256, 256, 0, s>>>(src, ids, n, pos, vel);
  return 1;
}
int launch_fill_f32(float* p, float v, size_t n, cudaStream_t s) {
  if (!n) return 0;
  k_fill_f32<<<1024, 256, 0, s>>>(p, v, n);
  return 1;
}
int launch_iota(uint32_t* p, uint32_t n, cudaStream_t s) {
  if (!n) return 0;
  k_iota<<<1024, 256, 0, s>>>(p, n);
  return 1;
}

}  // namespace st
