// pbf_core.cuh - position-based fluid passes on sm_100a with the semantics of GpuSim (src/gpu.js:102-353), shared by
// the PBF engine (st_pbf_*) and the density stage of the FLIP step, whose kernels are in pbf.cu.
//
// Design: every step sorts the live particles by uniform-grid cell (cell size h = 2.2 d) into a cell-sorted copy of
// their positions, so each solver pass is one thread per sorted slot and the 27-cell neighbour loops read contiguous
// runs of that copy: the lanes of a warp sit in one or two cells and read the same neighbours (L1 broadcasts), instead
// of the reference's gathers through an index list. Inside a cell the order is ascending particle index (the
// reference's atomic scatter leaves it open), fixed by a rank pass after the scatter, so every float sum is
// reproducible and equal to the oracle's. delta and applyDelta are one kernel writing a second position buffer (the
// neighbours' positions of the same iteration stay intact), so an iteration is two launches.
// Arithmetic: f32 in the reference's source order, no contraction (-fmad=false), inverseSqrt as 1 / sqrt.
#pragma once
#include "common.cuh"

namespace st {

// GpuSim's uniform block (struct Params, src/gpu.js:73-82), plus 1 / h and 1 / rho0 (computed in f32 by the shaders)
struct PbfParams {
  uint32_t n, nx, ny, nz, ncols, open, ncell, pad;
  float dt, h, h2, d, rho0, poly, spiky, W0, eps, c0, Gh, margin, gravity, visc, rest, relax;
  float bx0, bx1, by0, by1, bz0, bz1, maxD, vmax, inv, irho;
};
constexpr uint32_t PBF_DEAD = 0xffffffffu;
// the uniform block into the CTA's shared copy (every thread calls it; it ends with a barrier)
__device__ __forceinline__ void loadPbf(PbfParams& s, const PbfParams* g) {
  const uint32_t* src = reinterpret_cast<const uint32_t*>(g);
  uint32_t* dst = reinterpret_cast<uint32_t*>(&s);
  for (int i = threadIdx.x; i < (int)(sizeof(PbfParams) / 4); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
}
constexpr int PBF_T = 256;
constexpr int PBF_SCAN = 2048;   // cells per block of the grid scan

// Gf (src/gpu.js:116-121)
__device__ __forceinline__ float pbfGf(const PbfParams& P, float s) {
  const float h2 = P.h2, h4 = h2 * h2, h6 = h4 * h2, h8 = h4 * h4;
  const float s2 = s * s, s3 = s2 * s, s5 = s3 * s2, s7 = s5 * s2, s9 = s7 * s2;
  return h8 * s - (4.0f / 3.0f) * h6 * s3 + (6.0f / 5.0f) * h4 * s5 - (4.0f / 7.0f) * h2 * s7 + s9 / 9.0f;
}
// surf (src/gpu.js:123-128)
__device__ __forceinline__ void pbfSurf(const PbfParams& P, float phi0, float& rho, float& drho) {
  const float p = fmx(phi0, 0.0f);
  const float t = P.h2 - p * p;
  const float t2 = t * t;
  rho = P.c0 * (P.Gh - pbfGf(P, p));
  drho = -P.c0 * t2 * t2;
}
// bnd (src/gpu.js:129-148): boundary density and its gradient from the closed walls and every collider's grid
__device__ __forceinline__ void pbfBnd(const PbfParams& P, const float4* __restrict__ cols, const float* __restrict__ sdf, V3 x, float& rho, V3& g) {
  const float h = P.h;
  rho = 0.0f;
  g = v3(0.0f, 0.0f, 0.0f);
  float r, dr;
  float ph = x.x - P.bx0; if ((P.open & 1u) == 0u && ph < h) { pbfSurf(P, ph, r, dr); rho += r; g.x += dr; }
  ph = P.bx1 - x.x; if ((P.open & 2u) == 0u && ph < h) { pbfSurf(P, ph, r, dr); rho += r; g.x -= dr; }
  ph = x.y - P.by0; if ((P.open & 4u) == 0u && ph < h) { pbfSurf(P, ph, r, dr); rho += r; g.y += dr; }
  ph = P.by1 - x.y; if ((P.open & 8u) == 0u && ph < h) { pbfSurf(P, ph, r, dr); rho += r; g.y -= dr; }
  ph = x.z - P.bz0; if ((P.open & 16u) == 0u && ph < h) { pbfSurf(P, ph, r, dr); rho += r; g.z += dr; }
  ph = P.bz1 - x.z; if ((P.open & 32u) == 0u && ph < h) { pbfSurf(P, ph, r, dr); rho += r; g.z -= dr; }
  for (uint32_t k = 0; k < P.ncols; k++) {
    float phi; V3 wn;
    sdfEval(cols, sdf, k, x, phi, wn);
    if (phi >= h) continue;
    pbfSurf(P, phi, r, dr);
    rho += r;
    g = g + wn * dr;
  }
}
// collide (src/gpu.js:102-114): out of every collider by the margin, then the closed walls
__device__ __forceinline__ V3 pbfCollide(const PbfParams& P, const float4* __restrict__ cols, const float* __restrict__ sdf, V3 pin) {
  V3 p = pin;
  const float m = P.margin;
  for (uint32_t k = 0; k < P.ncols; k++) {
    float phi; V3 wn;
    sdfEval(cols, sdf, k, p, phi, wn);
    if (phi < m) p = p + wn * (m - phi);
  }
  const float big = 1.0e9f;
  const V3 lo = v3((P.open & 1u) ? -big : P.bx0 + m, (P.open & 4u) ? -big : P.by0 + m, (P.open & 16u) ? -big : P.bz0 + m);
  const V3 hi = v3((P.open & 2u) ? big : P.bx1 - m, (P.open & 8u) ? big : P.by1 - m, (P.open & 32u) ? big : P.bz1 - m);
  return vclamp(p, lo, hi);
}
// WGSL i32(f) (truncation, saturating) clamped into [0, n - 1]
__device__ __forceinline__ int pbfAxisCell(float f, uint32_t n) {
  int c = (f == f) ? (f >= 2147483648.0f ? 2147483647 : (f <= -2147483648.0f ? (int)0x80000000 : (int)f)) : 0;
  return c < 0 ? 0 : (c > (int)n - 1 ? (int)n - 1 : c);
}
// cellOf (src/gpu.js:149-155)
__device__ __forceinline__ uint32_t pbfCellOf(const PbfParams& P, V3 p) {
  const int cx = pbfAxisCell((p.x - P.bx0) * P.inv, P.nx), cy = pbfAxisCell((p.y - P.by0) * P.inv, P.ny);
  const int cz = pbfAxisCell((p.z - P.bz0) * P.inv, P.nz);
  return (uint32_t)cx + P.nx * ((uint32_t)cy + P.ny * (uint32_t)cz);
}
// Slots past the last one that the neighbour walk may read (and then ignores): the sorted-position arrays it walks are
// allocated with them.
constexpr uint32_t PBF_PAD = 8;
// A buffer of sorted positions: float4 records (each neighbour's own read and every other pass) and the same positions
// split into x, y and z arrays (the neighbour walk's test reads two slots per 8-byte load). Each holds PBF_PAD more slots.
struct PbfPos {
  float4* v;
  float *x, *y, *z;
};
__device__ __forceinline__ void pbfPut(const PbfPos& b, uint32_t t, float qx, float qy, float qz) {
  b.v[t] = make_float4(qx, qy, qz, 0.0f);
  b.x[t] = qx;
  b.y[t] = qy;
  b.z[t] = qz;
}
// The candidates of a particle in cell c that may lie inside the kernel radius, handed to f in the loop order of lambda,
// delta and viscosity (src/gpu.js:220-224): the 27-cell neighbourhood as 9 rows of three x-adjacent cells, which are
// contiguous runs of the sorted slots, z outer, y inner, slots ascending. Two phases: the lane first tests every slot of
// its rows (two slots per paired f32 operation on the split x, y, z arrays, in groups of eight with a bit per slot at a
// fixed position) into 64-slot masks kept in shared memory (PBF_ENT per thread), then walks all set bits of all masks
// in one loop, calling f with the slot and its position (loaded one neighbour ahead). A warp thus runs the
// per-neighbour work (square root, division) once per neighbour of its busiest lane over the whole neighbourhood,
// instead of once per slot where any lane has a neighbour (about 45 of the 290 slots of a 27-cell neighbourhood are
// within h); a lane whose masks fill the buffer walks them before it tests on. The test is a superset: its fused r2
// stays within a few units of rounding of the unfused one and the bound is h2 (1 + 2^-20), so every slot that the
// reference's loop does not skip reaches f (a NaN distance too). f makes that loop's own tests (the slot itself, the
// unfused r2 against h2) before its sums, so every sum gets the same terms in the same order. Blocks of PBF_T threads.
constexpr int PBF_ENT = 12;
template <class F>
__device__ __forceinline__ void pbfNear(const PbfParams& P, const PbfPos& xs, const uint32_t* __restrict__ start, uint32_t c, V3 qi,
                                        F&& f) {
  __shared__ uint32_t entBase[PBF_ENT][PBF_T];
  __shared__ uint2 entMask[PBF_ENT][PBF_T];
  const uint32_t tid = threadIdx.x;
  int nent = 0;
  // the bits of all masks in order; the next neighbour's position is loaded before f works on the current one
  auto walk = [&]() {
    int j = 0;
    unsigned long long m = 0ull;
    uint32_t base = 0;
    auto next = [&](uint32_t& slot) {
      while (m == 0ull && j < nent) {
        const uint2 mm = entMask[j][tid];
        m = ((unsigned long long)mm.y << 32) | mm.x;
        base = entBase[j][tid];
        j++;
      }
      if (m == 0ull) return false;
      slot = base + (uint32_t)__ffsll((long long)m) - 1u;
      m &= m - 1ull;
      return true;
    };
    uint32_t cur;
    if (next(cur)) {
      float4 xc = xs.v[cur];
      while (true) {
        uint32_t nx;
        const bool more = next(nx);
        float4 xn;
        if (more) xn = xs.v[nx];
        f(cur, xc);
        if (!more) break;
        cur = nx;
        xc = xn;
      }
    }
    nent = 0;
  };
  const int cx = (int)(c % P.nx);
  const uint32_t cq = c / P.nx;
  const int cy = (int)(cq % P.ny), cz = (int)(cq / P.ny);
  const uint32_t xa = (uint32_t)max(cx - 1, 0), xe = (uint32_t)min(cx + 1, (int)P.nx - 1) + 1u;
  const int ya = max(cy - 1, 0), yb = min(cy + 1, (int)P.ny - 1), za = max(cz - 1, 0), zb = min(cz + 1, (int)P.nz - 1);
  const float lim = P.h2 * (1.0f + 1.0f / 1048576.0f);
  const float2 nqx = make_float2(-qi.x, -qi.x), nqy = make_float2(-qi.y, -qi.y), nqz = make_float2(-qi.z, -qi.z);
  const float* __restrict__ sx = xs.x;
  const float* __restrict__ sy = xs.y;
  const float* __restrict__ sz = xs.z;
  for (int z = za; z <= zb; z++)
    for (int y = ya; y <= yb; y++) {
      const uint32_t row = P.nx * (uint32_t)(y + (int)P.ny * z);
      const uint32_t sb = start[row + xa], e = start[row + xe];
      // runs start at even slots, so each pair of slots is one aligned 8-byte load per axis (paired f32 arithmetic);
      // a slot before the row's start is masked off below
      for (uint32_t s = sb & ~1u; s < e; s += 64u) {
        const uint32_t n = min(e - s, 64u);
        unsigned long long m = 0ull;
        for (uint32_t g = 0; g < n; g += 8u) {
          uint32_t gm = 0;
#pragma unroll
          for (uint32_t k = 0; k < 8u; k += 2u) {
            const uint32_t i = s + g + k;
            const float2 dx = __fadd2_rn(*reinterpret_cast<const float2*>(sx + i), nqx);
            const float2 dy = __fadd2_rn(*reinterpret_cast<const float2*>(sy + i), nqy);
            const float2 dz = __fadd2_rn(*reinterpret_cast<const float2*>(sz + i), nqz);
            const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
            if (!(r2.x >= lim)) gm |= 1u << k;
            if (!(r2.y >= lim)) gm |= 2u << k;
          }
          m |= (unsigned long long)gm << g;
        }
        if (n < 64u) m &= (1ull << n) - 1ull;
        if (s < sb) m &= ~1ull;
        if (m == 0ull) continue;
        entBase[nent][tid] = s;
        entMask[nent][tid] = make_uint2((uint32_t)m, (uint32_t)(m >> 32));
        if (++nent == PBF_ENT) walk();
      }
    }
  walk();
}

// ---- the grid of one step: count (warp-aggregated atomics), scan, scatter, canonical order ----
// One particle per lane: its cell (or PBF_DEAD), and a provisional rank in the cell from the count's atomic.
// Every lane of the warp must call it (the aggregation is warp-wide).
__device__ __forceinline__ void pbfCount(uint32_t key, bool valid, uint32_t* __restrict__ cnt, uint32_t& rank) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t peers = __match_any_sync(0xffffffffu, valid && key != PBF_DEAD ? key : PBF_DEAD);
  const uint32_t lead = (uint32_t)__ffs(peers) - 1u;
  uint32_t base = 0;
  if (valid && key != PBF_DEAD && lane == lead) base = atomicAdd(&cnt[key], (uint32_t)__popc(peers));
  base = __shfl_sync(0xffffffffu, base, lead);
  rank = base + (uint32_t)__popc(peers & ((1u << lane) - 1u));
}
// ---- one solver iteration in sorted space ----
// lambda (src/gpu.js:208-251) for sorted slot t
__device__ __forceinline__ void pbfLambdaOne(const PbfParams& P, const PbfPos& xs, const uint32_t* __restrict__ start, uint32_t c,
                                             uint32_t t, const float4* __restrict__ cols, const float* __restrict__ sdf, float& lam, V3& bgr) {
  const V3 qi = xyz(xs.v[t]);
  const float irho = P.irho;
  float rho = P.W0, sg = 0.0f;
  V3 g = v3(0.0f, 0.0f, 0.0f);
  pbfNear(P, xs, start, c, qi, [&](uint32_t s, float4 xsS) {
    if (s == t) return;
    const V3 dd = qi - xyz(xsS);
    const float r2 = dot3(dd, dd);
    if (r2 >= P.h2) return;
    const float tt = P.h2 - r2;
    rho += P.poly * tt * tt * tt;
    const float r = sqrtf(r2);
    if (r < 1e-7f) return;
    const float hr = P.h - r;
    const float f = P.spiky * hr * hr / r * irho;
    const V3 fv = dd * f;
    g = g + fv;
    sg += dot3(fv, fv);
  });
  float br; V3 bg;
  pbfBnd(P, cols, sdf, qi, br, bg);
  rho += br;
  bg = bg * irho;
  bgr = bg;
  g = g + bg;
  sg += dot3(bg, bg);
  const float C = rho * irho - 1.0f;
  lam = C > 0.0f ? -C / (sg + dot3(g, g) + P.eps) : 0.0f;
}
// delta (src/gpu.js:253-286) for sorted slot t: the clamped correction
__device__ __forceinline__ V3 pbfDeltaOne(const PbfParams& P, const PbfPos& xs, const uint32_t* __restrict__ start, uint32_t c,
                                          uint32_t t, const float* __restrict__ lamS, const float4* __restrict__ bgrS) {
  const V3 qi = xyz(xs.v[t]);
  const float irho = P.irho, li = lamS[t];
  V3 s = xyz(bgrS[t]) * li;
  pbfNear(P, xs, start, c, qi, [&](uint32_t q, float4 xsQ) {
    if (q == t) return;
    const float sj = li + lamS[q];
    if (sj == 0.0f) return;
    const V3 dd = qi - xyz(xsQ);
    const float r2 = dot3(dd, dd);
    if (r2 >= P.h2) return;
    const float r = sqrtf(r2);
    if (r < 1e-7f) return;
    const float hr = P.h - r;
    s = s + dd * (P.spiky * hr * hr / r * irho * sj);
  });
  s = s * P.relax;
  const float m2 = dot3(s, s);
  if (m2 > P.maxD * P.maxD) s = s * (P.maxD * (1.0f / sqrtf(m2)));
  return s;
}

// Device buffers of one solver (the engine's, or the FLIP step's density stage)
struct PbfDev {
  PbfParams* P = nullptr;                   // the uniform block, uploaded each step
  uint32_t *key = nullptr, *rank = nullptr, *tmp = nullptr, *sidx = nullptr, *cellS = nullptr;   // per particle / slot
  PbfPos xs[2] = {};                        // sorted positions, two iteration buffers
  float4* bgrS = nullptr;                   // boundary gradient / rho0 per slot
  float* lamS = nullptr;                    // lambda per slot
  uint32_t *cnt = nullptr, *start = nullptr, *bsum = nullptr;   // per cell; scan blocks
  uint32_t ncell = 0;
};
// FluidSim's constants in double (src/shared.js:236-270)
struct PbfHostConsts { double h, h2, poly, spiky, W0, rho0, eps, c0, Gh, margin; };
PbfHostConsts pbf_consts(double d, double epsK, double wallK);
PbfParams pbf_params(const PbfHostConsts& c, double d, const double lo[3], const double hi[3], double dt, double g, double visc, uint32_t n,
                     uint32_t ncols, uint32_t open);
cudaError_t pbf_dev_alloc(PbfDev& D, uint32_t maxN, uint32_t ncell);
void pbf_dev_free(PbfDev& D);
size_t pbf_dev_bytes(uint32_t maxN, uint32_t ncell);
// the FLIP step's density stage on the particles of B.pa (D.P->n slots): grid, iters x (lambda, delta + collideP), write back
int launch_flip_pbf(const Bufs& B, const PbfDev& D, int iters, int grid, cudaStream_t s);

}  // namespace st
