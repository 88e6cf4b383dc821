// pbf.cu - position-based fluids on sm_100a with GpuSim's semantics (src/gpu.js:357-476): the PBF engine behind
// st_pbf_* of include/splashtank_cuda.h, and the density stage the FLIP step runs on its particles when
// st_step_opts.pbf_iters > 0. The passes themselves are in pbf_core.cuh.
//
// A step of the engine (GpuSim.step, src/gpu.js:409-428):
//   predict + count   one thread per particle (index order): gravity, collide, grid cell, warp-aggregated cell count
//   scan (3 launches) cell counts -> cell starts
//   scatter + order   provisional slots, then the canonical slot (ascending index in the cell) and the sorted copy
//   iterations        lambda, then delta + collide into the other position buffer (sorted space)
//   finalize          velocity from the move, restitution against the boundary gradient, speed limit, open faces
//   viscosity         XSPH over the neighbours, written back to index order
// Particles stay in index order between steps, as the reference keeps them. The neighbour-loop kernels run four CTAs
// per SM (at most 64 registers): two per SM measured 1.4x slower, five no faster.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/splashtank_cuda.h"
#include "kernels.h"
#include "pbf_core.cuh"

namespace st {

// ---- grid scan and the solver pass shared by both users ----
// exclusive scan of cnt[0, n) into start[0, n], start[n] = total: blocks of PBF_SCAN cells, then the block totals by one
// CTA, then each block adds its offset
__global__ void __launch_bounds__(1024) k_pbf_scan_blk(const uint32_t* __restrict__ cnt, uint32_t n, uint32_t* __restrict__ start,
                                                       uint32_t* __restrict__ bsum) {
  __shared__ uint32_t sm[33];
  const uint32_t i0 = blockIdx.x * PBF_SCAN + 2u * threadIdx.x;
  const uint32_t a = i0 < n ? cnt[i0] : 0u, b = i0 + 1 < n ? cnt[i0 + 1] : 0u;
  uint32_t tot;
  const uint32_t ex = blockExclusive(a + b, sm, &tot);
  if (i0 < n) start[i0] = ex;
  if (i0 + 1 < n) start[i0 + 1] = ex + a;
  if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}
__global__ void __launch_bounds__(1024) k_pbf_scan_top(uint32_t* __restrict__ bsum, uint32_t nb) {
  __shared__ uint32_t sm[33];
  scanOne(bsum, nb, nullptr, sm);
}
__global__ void __launch_bounds__(1024) k_pbf_scan_add(uint32_t* __restrict__ start, uint32_t n, const uint32_t* __restrict__ bsum, uint32_t nb) {
  const uint32_t i0 = blockIdx.x * PBF_SCAN + 2u * threadIdx.x, off = bsum[blockIdx.x];
  if (i0 < n) start[i0] += off;
  if (i0 + 1 < n) start[i0 + 1] += off;
  if (blockIdx.x == 0 && threadIdx.x == 0) start[n] = bsum[nb];
}
// provisional slots from the count's ranks
__global__ void __launch_bounds__(PBF_T) k_pbf_scatter(const PbfParams* __restrict__ Pg, const uint32_t* __restrict__ key,
                                                       const uint32_t* __restrict__ rank, const uint32_t* __restrict__ start,
                                                       uint32_t* __restrict__ tmp) {
  const uint32_t n = Pg->n;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t k = key[i];
    if (k != PBF_DEAD) tmp[start[k] + rank[i]] = i;
  }
}
// the canonical order: a particle's slot in its cell is the number of the cell's particles with a smaller index; its
// position (x: float4 records `stride` float4 apart) goes to the sorted copy
__global__ void __launch_bounds__(PBF_T) k_pbf_order(const PbfParams* __restrict__ Pg, const uint32_t* __restrict__ tmp, const uint32_t* __restrict__ key,
                                                     const uint32_t* __restrict__ start, const float4* __restrict__ x, uint32_t stride,
                                                     uint32_t* __restrict__ sidx, uint32_t* __restrict__ cellS, PbfPos xs) {
  const uint32_t nLive = start[Pg->ncell];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nLive; t += gridDim.x * blockDim.x) {
    const uint32_t i = tmp[t], c = key[i];
    const uint32_t a = start[c], b = start[c + 1];
    uint32_t r = 0;
    for (uint32_t u = a; u < b; u++) r += tmp[u] < i ? 1u : 0u;
    const float4 q = x[(size_t)i * stride];
    sidx[a + r] = i;
    cellS[a + r] = c;
    pbfPut(xs, a + r, q.x, q.y, q.z);
  }
}

__global__ void __launch_bounds__(PBF_T, 4) k_pbf_lambda(const PbfParams* __restrict__ Pg, const PbfPos xs, const uint32_t* __restrict__ cellS,
                                                      const uint32_t* __restrict__ start, const float4* __restrict__ cols, const float* __restrict__ sdf,
                                                      float* __restrict__ lamS, float4* __restrict__ bgrS) {
  __shared__ PbfParams P;
  loadPbf(P, Pg);
  const uint32_t nLive = start[P.ncell];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nLive; t += gridDim.x * blockDim.x) {
    float lam; V3 bg;
    pbfLambdaOne(P, xs, start, cellS[t], t, cols, sdf, lam, bg);
    lamS[t] = lam;
    bgrS[t] = make_float4(bg.x, bg.y, bg.z, 0.0f);
  }
}

// ---- the engine's own passes ----
// predict (src/gpu.js:155-161) fused with countCells (src/gpu.js:168-174). Dead particles keep their place and get
// velocity 0 (their finalize and viscosity write 0, src/gpu.js:295, 326). The loop bounds are warp-uniform (the count
// aggregates over the warp).
__global__ void __launch_bounds__(PBF_T) k_pbf_predict(const PbfParams* __restrict__ Pg, float4* __restrict__ pos, float4* __restrict__ vel,
                                                       float4* __restrict__ prd, uint32_t* __restrict__ key, uint32_t* __restrict__ rank,
                                                       uint32_t* __restrict__ cnt, const float4* __restrict__ cols, const float* __restrict__ sdf) {
  __shared__ PbfParams P;
  loadPbf(P, Pg);
  for (uint32_t b = blockIdx.x * blockDim.x; b < P.n; b += gridDim.x * blockDim.x) {
    const uint32_t i = b + threadIdx.x;
    const bool valid = i < P.n;
    uint32_t k = PBF_DEAD;
    if (valid) {
      const float4 p = pos[i];
      if (p.y < DEADY) {
        prd[i] = p;
        vel[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      } else {
        const float4 v0 = vel[i];
        const V3 v = xyz(v0) + v3(0.0f, -P.gravity * P.dt, 0.0f);
        vel[i] = make_float4(v.x, v.y, v.z, 0.0f);
        const V3 q = pbfCollide(P, cols, sdf, xyz(p) + v * P.dt);
        prd[i] = make_float4(q.x, q.y, q.z, 0.0f);
        k = pbfCellOf(P, q);
      }
      key[i] = k;
    }
    uint32_t r;
    pbfCount(k, valid, cnt, r);
    if (valid && k != PBF_DEAD) rank[i] = r;
  }
}
// delta (src/gpu.js:253-286) + applyDelta (:288-292): the corrected, collided position into the other buffer
__global__ void __launch_bounds__(PBF_T, 4) k_pbf_delta(const PbfParams* __restrict__ Pg, const PbfPos xs, const uint32_t* __restrict__ cellS,
                                                     const uint32_t* __restrict__ start, const float* __restrict__ lamS, const float4* __restrict__ bgrS,
                                                     const float4* __restrict__ cols, const float* __restrict__ sdf, const PbfPos xsOut) {
  __shared__ PbfParams P;
  loadPbf(P, Pg);
  const uint32_t nLive = start[P.ncell];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nLive; t += gridDim.x * blockDim.x) {
    const V3 s = pbfDeltaOne(P, xs, start, cellS[t], t, lamS, bgrS);
    const V3 q = pbfCollide(P, cols, sdf, xyz(xs.v[t]) + s);
    pbfPut(xsOut, t, q.x, q.y, q.z);
  }
}
// finalize (src/gpu.js:293-322) in sorted space: the velocity of the move, restitution where the boundary pushes,
// the speed limit of 12, and open faces; the result goes to the sorted final positions and velocities
__global__ void __launch_bounds__(PBF_T) k_pbf_finalize(const PbfParams* __restrict__ Pg, const float4* __restrict__ pos, const float4* __restrict__ vel,
                                                        const uint32_t* __restrict__ sidx, const float4* __restrict__ xs, const float4* __restrict__ bgrS,
                                                        const uint32_t* __restrict__ start, const PbfPos posF, float4* __restrict__ vel2S) {
  __shared__ PbfParams P;
  loadPbf(P, Pg);
  const uint32_t nLive = start[P.ncell];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nLive; t += gridDim.x * blockDim.x) {
    const uint32_t i = sidx[t];
    const V3 p = xyz(pos[i]), q = xyz(xs[t]), vo = xyz(vel[i]);
    V3 v = (q - p) / P.dt;
    const V3 g = xyz(bgrS[t]);
    const float gm2 = dot3(g, g);
    if (gm2 > 1e-6f) {
      const V3 nrm = (v3(0.0f, 0.0f, 0.0f) - g) * (1.0f / sqrtf(gm2));
      const float vn0 = dot3(vo, nrm);
      if (vn0 < 0.0f) {
        const float vn = dot3(v, nrm);
        const float lim = -vn0 * P.rest;
        if (vn > lim) v = v - nrm * (vn - lim);
      }
    }
    const float s2 = dot3(v, v);
    if (s2 > P.vmax * P.vmax) v = v * (P.vmax * (1.0f / sqrtf(s2)));
    const uint32_t o = P.open;
    if (o != 0u && (((o & 1u) && q.x < P.bx0) || ((o & 2u) && q.x > P.bx1) || ((o & 4u) && q.y < P.by0) || ((o & 8u) && q.y > P.by1) ||
                    ((o & 16u) && q.z < P.bz0) || ((o & 32u) && q.z > P.bz1))) {
      pbfPut(posF, t, 0.0f, -1.0e6f, 0.0f);
      vel2S[t] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    } else {
      pbfPut(posF, t, q.x, q.y, q.z);
      vel2S[t] = make_float4(v.x, v.y, v.z, 0.0f);
    }
  }
}
// viscosity (src/gpu.js:323-353): XSPH over the neighbours found through the step's grid, at the final positions;
// written back to index order with the speed in pos.w
__global__ void __launch_bounds__(PBF_T, 4) k_pbf_visc(const PbfParams* __restrict__ Pg, const uint32_t* __restrict__ sidx, const uint32_t* __restrict__ cellS,
                                                    const uint32_t* __restrict__ start, const PbfPos posF, const float4* __restrict__ vel2S,
                                                    float4* __restrict__ pos, float4* __restrict__ vel) {
  __shared__ PbfParams P;
  loadPbf(P, Pg);
  const uint32_t nLive = start[P.ncell];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nLive; t += gridDim.x * blockDim.x) {
    const uint32_t i = sidx[t];
    const float4 pf = posF.v[t];
    if (pf.y < DEADY) {
      pos[i] = pf;
      vel[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      continue;
    }
    const V3 pi = xyz(pf), vi = xyz(vel2S[t]);
    const float irho = P.irho;
    V3 a = v3(0.0f, 0.0f, 0.0f);
    if (P.visc > 0.0f) {
      pbfNear(P, posF, start, cellS[t], pi, [&](uint32_t s, float4 pfS) {
        if (s == t) return;
        const V3 dd = pi - xyz(pfS);
        const float r2 = dot3(dd, dd);
        if (r2 >= P.h2) return;
        const float tt = P.h2 - r2;
        a = a + (xyz(vel2S[s]) - vi) * (P.poly * tt * tt * tt * irho);
      });
    }
    const V3 nv = vi + a * P.visc;
    vel[i] = make_float4(nv.x, nv.y, nv.z, 0.0f);
    pos[i] = make_float4(pi.x, pi.y, pi.z, len3(nv));
  }
}

// ---- the FLIP step's density stage: the FLIP particles after g2p (storage order), FLIP's collider response ----
// count over the FLIP particles (Part records): dead ones (y below DEADY) take no cell
__global__ void __launch_bounds__(PBF_T) k_fpbf_count(const PbfParams* __restrict__ Pg, const Part* __restrict__ pa, uint32_t* __restrict__ key,
                                                      uint32_t* __restrict__ rank, uint32_t* __restrict__ cnt) {
  __shared__ PbfParams P;
  loadPbf(P, Pg);
  for (uint32_t b = blockIdx.x * blockDim.x; b < P.n; b += gridDim.x * blockDim.x) {
    const uint32_t i = b + threadIdx.x;
    const bool valid = i < P.n;
    uint32_t k = PBF_DEAD;
    if (valid) {
      const float4 p = pa[i].p;
      if (!(p.y < DEADY)) k = pbfCellOf(P, xyz(p));
      key[i] = k;
    }
    uint32_t r;
    pbfCount(k, valid, cnt, r);
    if (valid && k != PBF_DEAD) rank[i] = r;
  }
}
// delta + the FLIP step's collideP (src/flip/wgsl-solver.js:185-197) as the projection after each correction
__global__ void __launch_bounds__(PBF_T, 4) k_fpbf_delta(const PbfParams* __restrict__ Pg, Bufs B, const PbfPos xs, const uint32_t* __restrict__ cellS,
                                                      const uint32_t* __restrict__ start, const float* __restrict__ lamS, const float4* __restrict__ bgrS,
                                                      const PbfPos xsOut) {
  __shared__ FlipParams FP;
  loadParams(FP, B.P);
  __shared__ PbfParams P;
  loadPbf(P, Pg);
  const uint32_t nLive = start[P.ncell];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nLive; t += gridDim.x * blockDim.x) {
    const V3 s = pbfDeltaOne(P, xs, start, cellS[t], t, lamS, bgrS);
    const V3 q = collideP(FP, B.cols, B.sdf, xyz(xs.v[t]) + s);
    pbfPut(xsOut, t, q.x, q.y, q.z);
  }
}
// back to the FLIP particles: position q, velocity v + (q - p) / dt, pos.w from the new speed and the foam level (the
// encoding g2p writes)
__global__ void __launch_bounds__(PBF_T) k_fpbf_write(const PbfParams* __restrict__ Pg, const uint32_t* __restrict__ sidx, const float4* __restrict__ xs,
                                                      const uint32_t* __restrict__ start, Part* __restrict__ pa) {
  __shared__ PbfParams P;
  loadPbf(P, Pg);
  const uint32_t nLive = start[P.ncell];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nLive; t += gridDim.x * blockDim.x) {
    const uint32_t i = sidx[t];
    Part q = pa[i];
    const V3 x = xyz(xs[t]);
    const V3 v = xyz(q.v) + (x - xyz(q.p)) / P.dt;
    const float foam = q.v.w;
    q.p = make_float4(x.x, x.y, x.z, fmn(len3(v), 63.0f) + 64.0f * floorf(foam * 15.0f + 0.5f));
    q.v = make_float4(v.x, v.y, v.z, foam);
    pa[i] = q;
  }
}

// grid build shared by both: scan, scatter, order (counts are zeroed by the caller before the count pass)
static int launch_pbf_grid(const PbfParams* dP, const PbfDev& D, const float4* x, uint32_t stride, int grid, cudaStream_t s) {
  const uint32_t nb = (D.ncell + PBF_SCAN - 1) / PBF_SCAN;
  k_pbf_scan_blk<<<nb, 1024, 0, s>>>(D.cnt, D.ncell, D.start, D.bsum);
  k_pbf_scan_top<<<1, 1024, 0, s>>>(D.bsum, nb);
  k_pbf_scan_add<<<nb, 1024, 0, s>>>(D.start, D.ncell, D.bsum, nb);
  k_pbf_scatter<<<grid, PBF_T, 0, s>>>(dP, D.key, D.rank, D.start, D.tmp);
  k_pbf_order<<<grid, PBF_T, 0, s>>>(dP, D.tmp, D.key, D.start, x, stride, D.sidx, D.cellS, D.xs[0]);
  return 5;
}

int launch_flip_pbf(const Bufs& B, const PbfDev& D, int iters, int grid, cudaStream_t s) {
  int nl = 0;
  cudaMemsetAsync(D.cnt, 0, (size_t)D.ncell * 4, s);
  k_fpbf_count<<<grid, PBF_T, 0, s>>>(D.P, B.pa, D.key, D.rank, D.cnt);
  nl += 1 + launch_pbf_grid(D.P, D, &B.pa[0].p, 2, grid, s);
  int cur = 0;
  for (int it = 0; it < iters; it++) {
    k_pbf_lambda<<<grid, PBF_T, 0, s>>>(D.P, D.xs[cur], D.cellS, D.start, B.cols, B.sdf, D.lamS, D.bgrS);
    k_fpbf_delta<<<grid, PBF_T, 0, s>>>(D.P, B, D.xs[cur], D.cellS, D.start, D.lamS, D.bgrS, D.xs[cur ^ 1]);
    cur ^= 1;
    nl += 2;
  }
  k_fpbf_write<<<grid, PBF_T, 0, s>>>(D.P, D.sidx, D.xs[cur].v, D.start, B.pa);
  return nl + 1;
}

// FluidSim's constants (src/shared.js:236-270), computed in double as the JavaScript does
PbfHostConsts pbf_consts(double d, double epsK, double wallK) {
  PbfHostConsts c{};
  const double PI = 3.141592653589793;
  c.h = 2.2 * d;
  const double h = c.h, h2 = h * h;
  c.h2 = h2;
  c.poly = 315.0 / (64.0 * PI * std::pow(h, 9));
  c.spiky = -45.0 / (PI * std::pow(h, 6));
  c.W0 = c.poly * std::pow(h2, 3);
  auto G = [h2](double s) {
    const double h4 = h2 * h2, h6 = h4 * h2, h8 = h4 * h4;
    const double s2 = s * s, s3 = s2 * s, s5 = s3 * s2, s7 = s5 * s2, s9 = s7 * s2;
    return h8 * s - (4.0 / 3.0) * h6 * s3 + (6.0 / 5.0) * h4 * s5 - (4.0 / 7.0) * h2 * s7 + s9 / 9.0;
  };
  double rho0 = 0, below = 0, sgRest = 0;
  for (int i = -3; i <= 3; i++)
    for (int j = -3; j <= 3; j++)
      for (int k = -3; k <= 3; k++) {
        const double r2 = (double)(i * i + j * j + k * k) * d * d;
        if (r2 < h2) {
          const double w = c.poly * std::pow(h2 - r2, 3);
          rho0 += w;
          if (k < 0) below += w;
        }
      }
  c.rho0 = rho0;
  for (int i = -3; i <= 3; i++)
    for (int j = -3; j <= 3; j++)
      for (int k = -3; k <= 3; k++) {
        const double r = std::sqrt((double)(i * i + j * j + k * k)) * d;
        if (r > 1e-9 && r < h) {
          const double f = c.spiky * (h - r) * (h - r) / r / rho0 * r;
          sgRest += f * f;
        }
      }
  c.eps = (epsK > 0 ? epsK : 0.64) * sgRest;
  c.Gh = G(h);
  const double c0 = (1.0 / (d * d * d)) * (PI / 4.0) * c.poly;
  const double cont = c0 * (c.Gh - G(d / 2.0));
  c.c0 = c0 * (below / cont) * (wallK > 0 ? wallK : 1.8);
  c.margin = 0.15 * d;
  return c;
}
// the uniform block as GpuSim.step packs it (src/gpu.js:410-416): each value rounded once to f32
PbfParams pbf_params(const PbfHostConsts& c, double d, const double lo[3], const double hi[3], double dt, double g, double visc, uint32_t n,
                     uint32_t ncols, uint32_t open) {
  PbfParams P{};
  P.n = n; P.ncols = ncols; P.open = open;
  P.nx = (uint32_t)std::ceil((hi[0] - lo[0]) / c.h) + 1u;
  P.ny = (uint32_t)std::ceil((hi[1] - lo[1]) / c.h) + 1u;
  P.nz = (uint32_t)std::ceil((hi[2] - lo[2]) / c.h) + 1u;
  P.ncell = P.nx * P.ny * P.nz;
  P.dt = (float)dt; P.h = (float)c.h; P.h2 = (float)c.h2; P.d = (float)d; P.rho0 = (float)c.rho0; P.poly = (float)c.poly;
  P.spiky = (float)c.spiky; P.W0 = (float)c.W0; P.eps = (float)c.eps; P.c0 = (float)c.c0; P.Gh = (float)c.Gh;
  P.margin = (float)c.margin; P.gravity = (float)g; P.visc = (float)visc; P.rest = 0.1f; P.relax = 1.0f;
  P.bx0 = (float)lo[0]; P.bx1 = (float)hi[0]; P.by0 = (float)lo[1]; P.by1 = (float)hi[1]; P.bz0 = (float)lo[2]; P.bz1 = (float)hi[2];
  P.maxD = (float)(0.5 * d); P.vmax = 12.0f;
  P.inv = 1.0f / P.h;
  P.irho = 1.0f / P.rho0;
  return P;
}

// a sorted-position buffer of n slots (and PBF_PAD more) in one allocation: the float4 records, then x, y and z, each
// array an even number of floats long so every even slot starts an aligned pair
static size_t pbf_pos_slots(size_t n) { return (n + PBF_PAD + 1) & ~(size_t)1; }
static cudaError_t pbf_pos_alloc(PbfPos& b, size_t n) {
  const size_t np = pbf_pos_slots(n);
  char* m = nullptr;
  const cudaError_t e = cudaMalloc((void**)&m, np * 28);
  if (e != cudaSuccess) return e;
  b.v = reinterpret_cast<float4*>(m);
  b.x = reinterpret_cast<float*>(m + np * 16);
  b.y = b.x + np;
  b.z = b.y + np;
  return cudaSuccess;
}
static void pbf_pos_free(PbfPos& b) {
  if (b.v) cudaFree(b.v);
  b = PbfPos{};
}
cudaError_t pbf_dev_alloc(PbfDev& D, uint32_t maxN, uint32_t ncell) {
  D.ncell = ncell;
  const uint32_t nb = (ncell + PBF_SCAN - 1) / PBF_SCAN;
  cudaError_t e = cudaSuccess;
  auto A = [&](void** p, size_t bytes) { if (e == cudaSuccess) e = cudaMalloc(p, std::max<size_t>(bytes, 16)); };
  const size_t N = std::max<uint32_t>(maxN, 1);
  A((void**)&D.P, sizeof(PbfParams));
  A((void**)&D.key, N * 4); A((void**)&D.rank, N * 4); A((void**)&D.tmp, N * 4); A((void**)&D.sidx, N * 4); A((void**)&D.cellS, N * 4);
  for (PbfPos& b : D.xs)
    if (e == cudaSuccess) e = pbf_pos_alloc(b, N);
  A((void**)&D.bgrS, N * 16); A((void**)&D.lamS, N * 4);
  A((void**)&D.cnt, (size_t)ncell * 4); A((void**)&D.start, ((size_t)ncell + 1) * 4); A((void**)&D.bsum, ((size_t)nb + 1) * 4);
  return e;
}
void pbf_dev_free(PbfDev& D) {
  for (PbfPos& b : D.xs) pbf_pos_free(b);
  void* ps[] = {D.P, D.key, D.rank, D.tmp, D.sidx, D.cellS, D.bgrS, D.lamS, D.cnt, D.start, D.bsum};
  for (void* p : ps)
    if (p) cudaFree(p);
  D = PbfDev{};
}
size_t pbf_dev_bytes(uint32_t maxN, uint32_t ncell) {
  const size_t N = std::max<uint32_t>(maxN, 1);
  return N * (5 * 4 + 16 + 4) + 2 * pbf_pos_slots(N) * 28 + (size_t)ncell * 8 + ((size_t)ncell / PBF_SCAN + 2) * 4 + sizeof(PbfParams);
}

}  // namespace st

using namespace st;

// ---- the engine's handle ----
struct st_pbf {
  int device = 0;
  cudaStream_t stream = nullptr;
  int sms = 148;
  double d = 0, lo[3] = {}, hi[3] = {};
  PbfHostConsts c{};
  uint32_t open = 0, maxN = 0, cap = 0, N = 0, ring = 0, ncell = 0;
  bool recycle = true;
  float4 *pos = nullptr, *vel = nullptr, *prd = nullptr, *vel2S = nullptr;
  PbfPos posF{};             // the final sorted positions, walked by the viscosity pass
  PbfDev D{};
  float4* cols = nullptr;    // 8 float4 per collider (packColliders, src/gpu.js:57-67)
  float* sdf = nullptr;
  size_t sdfCap = 0;
  std::string sdfSig;
  PbfParams* hP = nullptr;   // pinned: the block uploaded each step
  float* hCols = nullptr;    // pinned: collider records
};

static thread_local char g_perr[256];
#define PK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { snprintf(g_perr, sizeof(g_perr), "%s: %s", #x, cudaGetErrorString(e_)); set_error_text(g_perr); return ST_DEVICE_ERROR; } } while (0)

void st_pbf_destroy(st_pbf* s) {
  if (!s) return;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  pbf_pos_free(s->posF);
  void* ps[] = {s->pos, s->vel, s->prd, s->vel2S, s->cols, s->sdf};
  for (void* p : ps)
    if (p) cudaFree(p);
  pbf_dev_free(s->D);
  if (s->hP) cudaFreeHost(s->hP);
  if (s->hCols) cudaFreeHost(s->hCols);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

// new GpuSim(device, {d, maxN, size, open}) (src/gpu.js:357-380): FluidSim's constants and grid (src/shared.js:220-270)
st_status st_pbf_create(const st_pbf_desc* ds, st_pbf** out) {
  if (!ds || !out || ds->size != sizeof(st_pbf_desc) || !(ds->d > 0) || ds->max_n == 0) return ST_BAD_ARG;
  *out = nullptr;
  st_pbf* s = new st_pbf();
  s->device = ds->device;
  s->d = ds->d;
  const double sz[3] = {ds->box[0] > 0 ? ds->box[0] : 3.0, ds->box[1] > 0 ? ds->box[1] : 2.6, ds->box[2] > 0 ? ds->box[2] : 3.0};
  s->lo[0] = -sz[0] / 2; s->hi[0] = sz[0] / 2; s->lo[1] = 0.0; s->hi[1] = sz[1]; s->lo[2] = -sz[2] / 2; s->hi[2] = sz[2] / 2;
  s->open = ds->open;
  s->maxN = s->cap = ds->max_n;
  s->c = pbf_consts(s->d, ds->eps_k, ds->wall_k);
  const PbfParams P0 = pbf_params(s->c, s->d, s->lo, s->hi, 1.0, 0.0, 0.0, 0, 0, s->open);
  s->ncell = P0.ncell;
  if ((double)P0.nx * P0.ny * P0.nz > 2.0e9) { delete s; set_error_text("pbf create: the grid has too many cells"); return ST_BAD_ARG; }
  auto fail = [&](const char* what, cudaError_t e) {
    snprintf(g_perr, sizeof(g_perr), "pbf create: %s: %s", what, cudaGetErrorString(e));
    set_error_text(g_perr);
    st_pbf_destroy(s);
    return e == cudaErrorMemoryAllocation ? ST_OOM : ST_DEVICE_ERROR;
  };
  cudaError_t e = cudaSetDevice(s->device);
  if (e != cudaSuccess) return fail("device", e);
  cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, s->device);
  if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail("stream", e);
  const size_t N = s->maxN;
  for (float4** p : {&s->pos, &s->vel, &s->prd, &s->vel2S})
    if ((e = cudaMalloc((void**)p, N * 16)) != cudaSuccess) return fail("particles", e);
  if ((e = pbf_pos_alloc(s->posF, N)) != cudaSuccess) return fail("particles", e);
  if ((e = cudaMemsetAsync(s->pos, 0, N * 16, s->stream)) != cudaSuccess) return fail("memset", e);
  if ((e = cudaMemsetAsync(s->vel, 0, N * 16, s->stream)) != cudaSuccess) return fail("memset", e);
  if ((e = pbf_dev_alloc(s->D, s->maxN, s->ncell)) != cudaSuccess) return fail("solver buffers", e);
  if ((e = cudaMalloc((void**)&s->cols, 32 * 8 * 16)) != cudaSuccess) return fail("colliders", e);
  if ((e = cudaMallocHost((void**)&s->hP, sizeof(PbfParams))) != cudaSuccess) return fail("pinned", e);
  if ((e = cudaMallocHost((void**)&s->hCols, 32 * 32 * 4)) != cudaSuccess) return fail("pinned", e);
  if ((e = cudaStreamSynchronize(s->stream)) != cudaSuccess) return fail("sync", e);
  *out = s;
  return ST_OK;
}

void* st_pbf_stream(st_pbf* s) { return s ? (void*)s->stream : nullptr; }

st_status st_pbf_set_cap(st_pbf* s, uint32_t c) {
  if (!s) return ST_BAD_ARG;
  s->cap = std::min(c, s->maxN);
  if (s->N > s->cap) s->N = s->cap;
  if (s->ring >= s->cap) s->ring = 0;
  return ST_OK;
}
st_status st_pbf_clear(st_pbf* s) {
  if (!s) return ST_BAD_ARG;
  s->N = 0;
  s->ring = 0;
  return ST_OK;
}
st_status st_pbf_set_recycle(st_pbf* s, int32_t on) {
  if (!s) return ST_BAD_ARG;
  s->recycle = on != 0;
  return ST_OK;
}

// GpuSim.add (src/gpu.js:390-402) for n particles: slots past N, then the ring once the cap is reached; the speed in
// pos.w (Math.sqrt in double, stored as f32), vel.w 0
st_status st_pbf_add(st_pbf* s, const float* p3, const float* v3_, uint32_t n, uint32_t* added) {
  if (!s || (n && !p3)) return ST_BAD_ARG;
  PK(cudaSetDevice(s->device));
  std::vector<float4> hp(n), hv(n);
  std::vector<uint32_t> slot(n);
  uint32_t k = 0;
  for (; k < n; k++) {
    uint32_t i;
    if (s->N < s->cap) i = s->N++;
    else if (s->recycle && s->cap) { i = s->ring++; if (s->ring >= s->cap) s->ring = 0; }
    else break;
    const float vx = v3_ ? v3_[k * 3] : 0.0f, vy = v3_ ? v3_[k * 3 + 1] : 0.0f, vz = v3_ ? v3_[k * 3 + 2] : 0.0f;
    hp[k] = make_float4(p3[k * 3], p3[k * 3 + 1], p3[k * 3 + 2], (float)std::sqrt((double)vx * vx + (double)vy * vy + (double)vz * vz));
    hv[k] = make_float4(vx, vy, vz, 0.0f);
    slot[k] = i;
  }
  uint32_t a = 0;
  while (a < k) {   // contiguous runs of slots go up in one copy each (flushRun, src/gpu.js:403-408)
    uint32_t b = a + 1;
    while (b < k && slot[b] == slot[b - 1] + 1) b++;
    PK(cudaMemcpyAsync(s->pos + slot[a], hp.data() + a, (size_t)(b - a) * 16, cudaMemcpyHostToDevice, s->stream));
    PK(cudaMemcpyAsync(s->vel + slot[a], hv.data() + a, (size_t)(b - a) * 16, cudaMemcpyHostToDevice, s->stream));
    a = b;
  }
  PK(cudaStreamSynchronize(s->stream));
  if (added) *added = k;
  return ST_OK;
}

// packColliders (src/gpu.js:42-70): 32 floats per collider; distance grids uploaded when the set of ids changes
static st_status pbf_pack(st_pbf* s, const st_pbf_opts* o, uint32_t& nc) {
  nc = std::min(o->ncols, 32u);
  std::string sig;
  std::map<uint32_t, uint32_t> offs;
  uint32_t off = 0;
  for (uint32_t k = 0; k < nc; k++) {
    const st_sdf* sd = o->cols[k].sdf;
    if (!sd || !sd->data || !sd->dims[0] || !sd->dims[1] || !sd->dims[2]) return ST_BAD_ARG;
    if (!offs.count(sd->id)) { offs[sd->id] = off; off += sd->dims[0] * sd->dims[1] * sd->dims[2]; sig += std::to_string(sd->id) + ","; }
  }
  if (sig != s->sdfSig) {
    PK(cudaStreamSynchronize(s->stream));
    if (off > s->sdfCap) {
      if (s->sdf) cudaFree(s->sdf);
      s->sdf = nullptr;
      s->sdfCap = (size_t)std::ceil(off * 1.3) + 16;
      PK(cudaMalloc((void**)&s->sdf, s->sdfCap * 4));
    }
    std::map<uint32_t, bool> seen;
    for (uint32_t k = 0; k < nc; k++) {
      const st_sdf* sd = o->cols[k].sdf;
      if (seen[sd->id]) continue;
      seen[sd->id] = true;
      PK(cudaMemcpyAsync(s->sdf + offs[sd->id], sd->data, 4ull * sd->dims[0] * sd->dims[1] * sd->dims[2], cudaMemcpyHostToDevice, s->stream));
    }
    PK(cudaStreamSynchronize(s->stream));
    s->sdfSig = sig;
  }
  if (!s->sdf) {
    s->sdfCap = 16;
    PK(cudaMalloc((void**)&s->sdf, s->sdfCap * 4));
  }
  for (uint32_t k = 0; k < nc; k++) {
    const st_collider& c = o->cols[k];
    const st_sdf* sd = c.sdf;
    float* f = s->hCols + k * 32;
    f[0] = (float)offs[sd->id]; f[1] = (float)sd->dims[0]; f[2] = (float)sd->dims[1]; f[3] = (float)sd->dims[2];
    f[4] = sd->origin[0]; f[5] = sd->origin[1]; f[6] = sd->origin[2]; f[7] = sd->cell;
    f[8] = c.R[0]; f[9] = c.R[3]; f[10] = c.R[6]; f[11] = 0;
    f[12] = c.R[1]; f[13] = c.R[4]; f[14] = c.R[7]; f[15] = 0;
    f[16] = c.R[2]; f[17] = c.R[5]; f[18] = c.R[8]; f[19] = 0;
    f[20] = c.pos[0]; f[21] = c.pos[1]; f[22] = c.pos[2]; f[23] = 0;
    f[24] = c.vel[0]; f[25] = c.vel[1]; f[26] = c.vel[2]; f[27] = 0;
    f[28] = c.ang[0]; f[29] = c.ang[1]; f[30] = c.ang[2]; f[31] = 0;
  }
  if (nc) PK(cudaMemcpyAsync(s->cols, s->hCols, nc * 32 * 4, cudaMemcpyHostToDevice, s->stream));
  return ST_OK;
}

// GpuSim.step (src/gpu.js:409-428)
st_status st_pbf_step(st_pbf* s, double dt, const st_pbf_opts* o) {
  if (!s || !o || o->size != sizeof(st_pbf_opts) || (o->ncols && !o->cols) || o->iters < 1 || !(dt > 0)) return ST_BAD_ARG;
  if (!s->N) return ST_NOT_READY;
  PK(cudaSetDevice(s->device));
  uint32_t nc = 0;
  const st_status st = pbf_pack(s, o, nc);
  if (st != ST_OK) return st;
  PK(cudaStreamSynchronize(s->stream));   // the pinned block is rewritten only after the last step's copy ran
  *s->hP = pbf_params(s->c, s->d, s->lo, s->hi, dt, o->g, o->visc, s->N, nc, s->open);
  cudaStream_t q = s->stream;
  PK(cudaMemcpyAsync(s->D.P, s->hP, sizeof(PbfParams), cudaMemcpyHostToDevice, q));
  PK(cudaMemsetAsync(s->D.cnt, 0, (size_t)s->ncell * 4, q));
  const int grid = std::max(1, std::min<int>(s->sms * 8, (int)((s->N + PBF_T - 1) / PBF_T)));
  k_pbf_predict<<<grid, PBF_T, 0, q>>>(s->D.P, s->pos, s->vel, s->prd, s->D.key, s->D.rank, s->D.cnt, s->cols, s->sdf);
  launch_pbf_grid(s->D.P, s->D, s->prd, 1, grid, q);
  int cur = 0;
  for (int it = 0; it < o->iters; it++) {
    k_pbf_lambda<<<grid, PBF_T, 0, q>>>(s->D.P, s->D.xs[cur], s->D.cellS, s->D.start, s->cols, s->sdf, s->D.lamS, s->D.bgrS);
    k_pbf_delta<<<grid, PBF_T, 0, q>>>(s->D.P, s->D.xs[cur], s->D.cellS, s->D.start, s->D.lamS, s->D.bgrS, s->cols, s->sdf, s->D.xs[cur ^ 1]);
    cur ^= 1;
  }
  k_pbf_finalize<<<grid, PBF_T, 0, q>>>(s->D.P, s->pos, s->vel, s->D.sidx, s->D.xs[cur].v, s->D.bgrS, s->D.start, s->posF, s->vel2S);
  k_pbf_visc<<<grid, PBF_T, 0, q>>>(s->D.P, s->D.sidx, s->D.cellS, s->D.start, s->posF, s->vel2S, s->pos, s->vel);
  PK(cudaGetLastError());
  return ST_OK;
}

// positions (xyz, speed in w) and velocities of the N slots in index order (readbackInto, src/gpu.js:430-443)
st_status st_pbf_read(st_pbf* s, float* pos4, float* vel4, uint32_t cap, uint32_t* n) {
  if (!s || (!pos4 && !vel4)) return ST_BAD_ARG;
  PK(cudaSetDevice(s->device));
  const uint32_t m = std::min(cap, s->N);
  if (n) *n = s->N;
  if (m && pos4) PK(cudaMemcpyAsync(pos4, s->pos, (size_t)m * 16, cudaMemcpyDeviceToHost, s->stream));
  if (m && vel4) PK(cudaMemcpyAsync(vel4, s->vel, (size_t)m * 16, cudaMemcpyDeviceToHost, s->stream));
  PK(cudaStreamSynchronize(s->stream));
  return ST_OK;
}
