// pbf.cu - the position-based fluid step (GpuSim, src/gpu.js:357-428; its CPU twin Sim::step, native/splash.cpp:212-247)
// on sm_100a, behind st_pbf_* of include/splashtank_cuda.h.
//
// Particles stay in index order. Each step sorts particle indices by uniform-grid cell (cell size h = 2.2 d): an atomic
// scatter, then every cell's short index list is put in ascending order, which is exactly the order the reference's
// serial counting sort produces (native/splash.cpp:157-159). Neighbour lists then hold the first 48 particles within h,
// scanning cells z, y, x as the reference does (:161-175), so the capped lists - and every floating-point sum over
// them - match the CPU restatement bit for bit (no contraction: -fmad=false).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/splashtank_cuda.h"
#include "common.cuh"

namespace {

constexpr int MAXNB = 48;
constexpr int MAXCOL = 32;

struct PCol { int t; float x, y, z, r, hx, hy, hz, c, s; };   // native/splash.cpp:22

struct PbfParams {
  float d, h, h2, poly, spiky, W0, rho0, eps, c0, Gh, margin, rest;
  float X0, X1, Y0, Y1, Z0, Z1;
  float dt, g, visc, inv;
  int nx, ny, nz, n, ncols;
  PCol cols[MAXCOL];
};

__device__ __forceinline__ float fminx(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float fmaxx(float a, float b) { return a > b ? a : b; }
__device__ double Gd(double h, double s) {
  double h2 = h * h, h4 = h2 * h2, h6 = h4 * h2, h8 = h4 * h4;
  double s2 = s * s, s3 = s2 * s, s5 = s3 * s2, s7 = s5 * s2, s9 = s7 * s2;
  return h8 * s - (4.0 / 3) * h6 * s3 + (6.0 / 5) * h4 * s5 - (4.0 / 7) * h2 * s7 + s9 / 9;
}

// collide (native/splash.cpp:95-116): push out of spheres and rotated boxes, then clamp to the walls
__global__ void k_collide(PbfParams P, float* __restrict__ Q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const float m = P.margin, x0 = P.X0 + m, x1 = P.X1 - m, y0 = P.Y0 + m, y1 = P.Y1 - m, z0 = P.Z0 + m, z1 = P.Z1 - m;
  const int i3 = i * 3;
  float x = Q[i3], y = Q[i3 + 1], z = Q[i3 + 2];
  for (int k = 0; k < P.ncols; k++) {
    const PCol c = P.cols[k];
    if (c.t == 0) {
      float dx = x - c.x, dy = y - c.y, dz = z - c.z, R = c.r + m, d2 = dx * dx + dy * dy + dz * dz;
      if (d2 < R * R) {
        float dd = sqrtf(d2);
        if (dd < 1e-6f) y = c.y + R;
        else { float s = R / dd; x = c.x + dx * s; y = c.y + dy * s; z = c.z + dz * s; }
      }
    } else {
      float ox = x - c.x, oy = y - c.y, oz = z - c.z, lx = ox * c.c + oz * c.s, lz = -ox * c.s + oz * c.c;
      float ax = c.hx + m, ay = c.hy + m, az = c.hz + m, alx = fabsf(lx), aly = fabsf(oy), alz = fabsf(lz);
      if (alx < ax && aly < ay && alz < az) {
        float px = ax - alx, py = ay - aly, pz = az - alz;
        if (px <= py && px <= pz) lx = lx < 0 ? -ax : ax; else if (py <= pz) oy = oy < 0 ? -ay : ay; else lz = lz < 0 ? -az : az;
        x = c.x + lx * c.c - lz * c.s; z = c.z + lx * c.s + lz * c.c; y = c.y + oy;
      }
    }
  }
  Q[i3] = fminx(fmaxx(x, x0), x1); Q[i3 + 1] = fminx(fmaxx(y, y0), y1); Q[i3 + 2] = fminx(fmaxx(z, z0), z1);
}

__device__ __forceinline__ float bR(const PbfParams& P, float p) { return P.c0 * (P.Gh - (float)Gd((double)P.h, (double)p)); }
__device__ __forceinline__ float bD(const PbfParams& P, float p) { float t = P.h2 - p * p; t *= t; return -P.c0 * t * t; }
// bnd (native/splash.cpp:117-148): density of the walls and colliders at a point, and its gradient
__device__ void bnd(const PbfParams& P, float x, float y, float z, float& rho, float& gx, float& gy, float& gz) {
  rho = gx = gy = gz = 0.0f;
  float p;
  const float h = P.h;
  p = x - P.X0; if (p < h) { if (p < 0) p = 0; rho += bR(P, p); gx += bD(P, p); }
  p = P.X1 - x; if (p < h) { if (p < 0) p = 0; rho += bR(P, p); gx -= bD(P, p); }
  p = y - P.Y0; if (p < h) { if (p < 0) p = 0; rho += bR(P, p); gy += bD(P, p); }
  p = P.Y1 - y; if (p < h) { if (p < 0) p = 0; rho += bR(P, p); gy -= bD(P, p); }
  p = z - P.Z0; if (p < h) { if (p < 0) p = 0; rho += bR(P, p); gz += bD(P, p); }
  p = P.Z1 - z; if (p < h) { if (p < 0) p = 0; rho += bR(P, p); gz -= bD(P, p); }
  for (int k = 0; k < P.ncols; k++) {
    const PCol c = P.cols[k];
    if (c.t == 0) {
      float dx = x - c.x, dy = y - c.y, dz = z - c.z, dist = sqrtf(dx * dx + dy * dy + dz * dz), phi = dist - c.r;
      if (phi >= h) continue;
      if (phi < 0) phi = 0;
      float dd = bD(P, phi);
      rho += bR(P, phi);
      if (dist > 1e-6f) { float s = dd / dist; gx += dx * s; gy += dy * s; gz += dz * s; } else gy += dd;
    } else {
      float ox = x - c.x, oy = y - c.y, oz = z - c.z, lx = ox * c.c + oz * c.s, lz = -ox * c.s + oz * c.c;
      float qx = fabsf(lx) - c.hx, qy = fabsf(oy) - c.hy, qz = fabsf(lz) - c.hz, nlx, nly, nlz, phi;
      if (qx < 0 && qy < 0 && qz < 0) {
        phi = 0; nlx = nly = nlz = 0;
        if (qx >= qy && qx >= qz) nlx = lx < 0 ? -1 : 1; else if (qy >= qz) nly = oy < 0 ? -1 : 1; else nlz = lz < 0 ? -1 : 1;
      } else {
        float mx = fmaxx(qx, 0.f), my = fmaxx(qy, 0.f), mz = fmaxx(qz, 0.f);
        phi = sqrtf(mx * mx + my * my + mz * mz);
        if (phi >= h) continue;
        float inv = phi > 1e-9f ? 1 / phi : 0;
        nlx = (lx < 0 ? -mx : mx) * inv; nly = (oy < 0 ? -my : my) * inv; nlz = (lz < 0 ? -mz : mz) * inv;
      }
      float dd = bD(P, phi);
      rho += bR(P, phi);
      gx += dd * (nlx * c.c - nlz * c.s); gy += dd * nly; gz += dd * (nlx * c.s + nlz * c.c);
    }
  }
}

// predict (native/splash.cpp:214-215)
__global__ void k_predict(PbfParams P, const float* __restrict__ Pp, float* __restrict__ V, float* __restrict__ Q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const int i3 = i * 3;
  V[i3 + 1] -= P.g * P.dt;
  for (int a = 0; a < 3; a++) Q[i3 + a] = Pp[i3 + a] + V[i3 + a] * P.dt;
}
// grid cell of each particle and the count per cell (native/splash.cpp:152-156)
__global__ void k_cells(PbfParams P, const float* __restrict__ Q, int* __restrict__ cid, int* __restrict__ count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const int i3 = i * 3;
  int cx = (int)((Q[i3] - P.X0) * P.inv), cy = (int)((Q[i3 + 1] - P.Y0) * P.inv), cz = (int)((Q[i3 + 2] - P.Z0) * P.inv);
  cx = min(max(cx, 0), P.nx - 1); cy = min(max(cy, 0), P.ny - 1); cz = min(max(cz, 0), P.nz - 1);
  const int c = cx + P.nx * (cy + P.ny * cz);
  cid[i] = c;
  atomicAdd(&count[c], 1);
}
// exclusive scan of the cell counts: per-block sums, one CTA over them, then per-block prefixes
__global__ void __launch_bounds__(1024) k_blocksum(const int* __restrict__ in, int n, int* __restrict__ bs) {
  __shared__ uint32_t sm[33];
  const int i = blockIdx.x * 1024 + threadIdx.x;
  uint32_t tot;
  st::blockExclusive(i < n ? (uint32_t)in[i] : 0u, sm, &tot);
  if (threadIdx.x == 0) bs[blockIdx.x] = (int)tot;
}
__global__ void __launch_bounds__(1024) k_scanblocks(int* bs, int nb) {
  __shared__ uint32_t sm[33];
  uint32_t chunk = (nb + 1023) / 1024, beg = min(threadIdx.x * chunk, (uint32_t)nb), end = min(beg + chunk, (uint32_t)nb);
  uint32_t s = 0;
  for (uint32_t x = beg; x < end; x++) s += (uint32_t)bs[x];
  uint32_t tot, run = st::blockExclusive(s, sm, &tot);
  for (uint32_t x = beg; x < end; x++) { uint32_t v = (uint32_t)bs[x]; bs[x] = (int)run; run += v; }
}
__global__ void __launch_bounds__(1024) k_prefix(const int* __restrict__ in, int n, const int* __restrict__ bs, int* __restrict__ start,
                                                 int* __restrict__ cursor) {
  __shared__ uint32_t sm[33];
  const int i = blockIdx.x * 1024 + threadIdx.x;
  uint32_t tot;
  uint32_t ex = st::blockExclusive(i < n ? (uint32_t)in[i] : 0u, sm, &tot);
  if (i < n) { start[i] = bs[blockIdx.x] + (int)ex; cursor[i] = start[i]; }
  if (i == n - 1) start[n] = bs[blockIdx.x] + (int)ex + in[i];
}
__global__ void k_scatter_idx(PbfParams P, const int* __restrict__ cid, int* __restrict__ cursor, int* __restrict__ sorted) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  sorted[atomicAdd(&cursor[cid[i]], 1)] = i;
}
// each cell's indices in ascending order: the order of the reference's serial scatter
__global__ void k_cell_order(int cells, const int* __restrict__ start, int* __restrict__ sorted) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cells) return;
  const int a = start[c], b = start[c + 1];
  for (int u = a + 1; u < b; u++) {
    const int v = sorted[u];
    int w = u - 1;
    while (w >= a && sorted[w] > v) { sorted[w + 1] = sorted[w]; w--; }
    sorted[w + 1] = v;
  }
}
// neighbour lists (native/splash.cpp:160-175): the first MAXNB particles within h, cells scanned z, y, then a row of x
__global__ void k_neighbors(PbfParams P, const float* __restrict__ Q, const int* __restrict__ cid, const int* __restrict__ start,
                            const int* __restrict__ sorted, int* __restrict__ nb, int* __restrict__ nc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const int c = cid[i], cx = c % P.nx, t = c / P.nx, cy = t % P.ny, cz = t / P.ny, i3 = i * 3;
  const float xi = Q[i3], yi = Q[i3 + 1], zi = Q[i3 + 2];
  const int xa = max(cx - 1, 0), xb = min(cx + 1, P.nx - 1), ya = max(cy - 1, 0), yb = min(cy + 1, P.ny - 1);
  const int za = max(cz - 1, 0), zb = min(cz + 1, P.nz - 1);
  int* out = nb + (size_t)i * MAXNB;
  int n = 0;
  for (int z = za; z <= zb; z++)
    for (int y = ya; y <= yb; y++) {
      const int row = P.nx * (y + P.ny * z);
      const int s1 = start[row + xb + 1];
      for (int s = start[row + xa]; s < s1; s++) {
        const int j = sorted[s];
        if (j == i) continue;
        const int j3 = j * 3;
        const float dx = xi - Q[j3], dy = yi - Q[j3 + 1], dz = zi - Q[j3 + 2];
        if (dx * dx + dy * dy + dz * dz < P.h2 && n < MAXNB) out[n++] = j;
      }
    }
  nc[i] = n;
}
// solve, first loop (native/splash.cpp:179-194): density constraint and its lambda
__global__ void k_lambda(PbfParams P, const float* __restrict__ Q, const int* __restrict__ nb, const int* __restrict__ nc,
                         float* __restrict__ BG, float* __restrict__ lam) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const float irho = 1 / P.rho0;
  const int i3 = i * 3;
  const float xi = Q[i3], yi = Q[i3 + 1], zi = Q[i3 + 2];
  float rho = P.W0, gx = 0, gy = 0, gz = 0, sg = 0;
  const int* lst = nb + (size_t)i * MAXNB;
  const int cnt = nc[i];
  for (int k = 0; k < cnt; k++) {
    const int j3 = lst[k] * 3;
    const float dx = xi - Q[j3], dy = yi - Q[j3 + 1], dz = zi - Q[j3 + 2], r2 = dx * dx + dy * dy + dz * dz;
    if (r2 >= P.h2) continue;
    const float t = P.h2 - r2;
    rho += P.poly * t * t * t;
    const float r = sqrtf(r2);
    if (r < 1e-7f) continue;
    const float hr = P.h - r, f = P.spiky * hr * hr / r * irho, fx = f * dx, fy = f * dy, fz = f * dz;
    gx += fx; gy += fy; gz += fz; sg += fx * fx + fy * fy + fz * fz;
  }
  float br, bgx, bgy, bgz;
  bnd(P, xi, yi, zi, br, bgx, bgy, bgz);
  rho += br; bgx *= irho; bgy *= irho; bgz *= irho;
  BG[i3] = bgx; BG[i3 + 1] = bgy; BG[i3 + 2] = bgz;
  gx += bgx; gy += bgy; gz += bgz; sg += bgx * bgx + bgy * bgy + bgz * bgz;
  const float C = rho * irho - 1;
  lam[i] = C > 0 ? -C / (sg + gx * gx + gy * gy + gz * gz + P.eps) : 0;
}
// solve, second loop (native/splash.cpp:195-208): position correction, limited to half a spacing
__global__ void k_delta(PbfParams P, const float* __restrict__ Q, const int* __restrict__ nb, const int* __restrict__ nc,
                        const float* __restrict__ BG, const float* __restrict__ lam, float* __restrict__ D) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const float irho = 1 / P.rho0, maxD = 0.5f * P.d, maxD2 = maxD * maxD;
  const int i3 = i * 3;
  const float xi = Q[i3], yi = Q[i3 + 1], zi = Q[i3 + 2], li = lam[i];
  float sx = li * BG[i3], sy = li * BG[i3 + 1], sz = li * BG[i3 + 2];
  const int* lst = nb + (size_t)i * MAXNB;
  const int cnt = nc[i];
  for (int k = 0; k < cnt; k++) {
    const int j = lst[k], j3 = j * 3;
    const float s = li + lam[j];
    if (s == 0) continue;
    const float dx = xi - Q[j3], dy = yi - Q[j3 + 1], dz = zi - Q[j3 + 2], r2 = dx * dx + dy * dy + dz * dz;
    if (r2 >= P.h2) continue;
    const float r = sqrtf(r2);
    if (r < 1e-7f) continue;
    const float hr = P.h - r, f = P.spiky * hr * hr / r * irho * s;
    sx += f * dx; sy += f * dy; sz += f * dz;
  }
  const float m2 = sx * sx + sy * sy + sz * sz;
  if (m2 > maxD2) { const float k = maxD / sqrtf(m2); sx *= k; sy *= k; sz *= k; }
  D[i3] = sx; D[i3 + 1] = sy; D[i3 + 2] = sz;
}
__global__ void k_apply(int n3, float* __restrict__ Q, const float* __restrict__ D) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n3) Q[i] += D[i];
}
// velocity from the move, inelastic contact, speed limit (native/splash.cpp:218-229)
__global__ void k_velocity(PbfParams P, const float* __restrict__ Pp, const float* __restrict__ Q, const float* __restrict__ BG, float* __restrict__ V) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const float idt = 1 / P.dt, vmax = 12;
  const int i3 = i * 3;
  float vx = (Q[i3] - Pp[i3]) * idt, vy = (Q[i3 + 1] - Pp[i3 + 1]) * idt, vz = (Q[i3 + 2] - Pp[i3 + 2]) * idt;
  const float gx = BG[i3], gy = BG[i3 + 1], gz = BG[i3 + 2], gm2 = gx * gx + gy * gy + gz * gz;
  if (gm2 > 1e-6f) {
    const float gm = 1 / sqrtf(gm2), nx_ = -gx * gm, ny_ = -gy * gm, nz_ = -gz * gm;
    const float vo = V[i3] * nx_ + V[i3 + 1] * ny_ + V[i3 + 2] * nz_;
    if (vo < 0) {
      const float vn = vx * nx_ + vy * ny_ + vz * nz_, lim = -vo * P.rest;
      if (vn > lim) { const float k = vn - lim; vx -= k * nx_; vy -= k * ny_; vz -= k * nz_; }
    }
  }
  const float s2 = vx * vx + vy * vy + vz * vz;
  if (s2 > vmax * vmax) { const float k = vmax / sqrtf(s2); vx *= k; vy *= k; vz *= k; }
  V[i3] = vx; V[i3 + 1] = vy; V[i3 + 2] = vz;
}
// XSPH viscosity (native/splash.cpp:230-244)
__global__ void k_visc(PbfParams P, const float* __restrict__ Q, const float* __restrict__ V, const int* __restrict__ nb,
                       const int* __restrict__ nc, float* __restrict__ NV) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const float irho = 1 / P.rho0;
  const int i3 = i * 3;
  const float xi = Q[i3], yi = Q[i3 + 1], zi = Q[i3 + 2];
  float ax = 0, ay = 0, az = 0;
  const int* lst = nb + (size_t)i * MAXNB;
  const int cnt = nc[i];
  for (int k = 0; k < cnt; k++) {
    const int j3 = lst[k] * 3;
    const float dx = xi - Q[j3], dy = yi - Q[j3 + 1], dz = zi - Q[j3 + 2], r2 = dx * dx + dy * dy + dz * dz;
    if (r2 >= P.h2) continue;
    const float t = P.h2 - r2, w = P.poly * t * t * t * irho;
    ax += (V[j3] - V[i3]) * w; ay += (V[j3 + 1] - V[i3 + 1]) * w; az += (V[j3 + 2] - V[i3 + 2]) * w;
  }
  NV[i3] = V[i3] + P.visc * ax; NV[i3 + 1] = V[i3 + 1] + P.visc * ay; NV[i3 + 2] = V[i3 + 2] + P.visc * az;
}
__global__ void k_commit(PbfParams P, float* __restrict__ Pp, const float* __restrict__ Q, const float* __restrict__ V, float* __restrict__ S) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const int i3 = i * 3;
  Pp[i3] = Q[i3]; Pp[i3 + 1] = Q[i3 + 1]; Pp[i3 + 2] = Q[i3 + 2];
  S[i] = sqrtf(V[i3] * V[i3] + V[i3 + 1] * V[i3 + 1] + V[i3 + 2] * V[i3 + 2]);
}
__global__ void k_pack(int n, const float* __restrict__ Pp, const float* __restrict__ S, const float* __restrict__ V, float4* pos, float4* vel) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  pos[i] = make_float4(Pp[i * 3], Pp[i * 3 + 1], Pp[i * 3 + 2], S[i]);
  if (vel) vel[i] = make_float4(V[i * 3], V[i * 3 + 1], V[i * 3 + 2], 0.0f);
}

thread_local char g_perr[256] = "";

}  // namespace

struct st_pbf {
  int device = 0;
  cudaStream_t stream = nullptr;
  PbfParams hp{};
  uint32_t cap = 0;
  int n = 0, cells = 0, nblocks = 0;
  float *P = nullptr, *V = nullptr, *Q = nullptr, *D = nullptr, *NV = nullptr, *BG = nullptr, *S = nullptr, *lam = nullptr;
  int *cid = nullptr, *sorted = nullptr, *nb = nullptr, *nc = nullptr, *count = nullptr, *start = nullptr, *cursor = nullptr, *bs = nullptr;
  float4* out = nullptr;
};

#define PK(call)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) {                                                                  \
      snprintf(g_perr, sizeof(g_perr), "%s: %s", #call, cudaGetErrorString(e_)); st::set_error_text(g_perr);              \
      return e_ == cudaErrorMemoryAllocation ? ST_OOM : ST_DEVICE_ERROR;                      \
    }                                                                                         \
  } while (0)

extern "C" {

void st_pbf_destroy(st_pbf* s) {
  if (!s) return;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  void* ptrs[] = {s->P, s->V, s->Q, s->D, s->NV, s->BG, s->S, s->lam, s->cid, s->sorted, s->nb, s->nc, s->count, s->start, s->cursor, s->bs, s->out};
  for (void* p : ptrs) if (p) cudaFree(p);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

// constants of new FluidSim / Sim (src/shared.js:220-271, native/splash.cpp:50-71)
st_status st_pbf_create(const st_pbf_desc* ds, st_pbf** out) {
  if (!ds || !out || ds->size != sizeof(st_pbf_desc) || !(ds->d > 0) || ds->max_n == 0) return ST_BAD_ARG;
  st_pbf* s = new st_pbf();
  *out = nullptr;
  s->device = ds->device;
  if (cudaSetDevice(s->device) != cudaSuccess) { delete s; return ST_DEVICE_ERROR; }
  PbfParams& P = s->hp;
  P.d = (float)ds->d;
  double bx = ds->box[0] > 0 ? ds->box[0] : 3.0, by = ds->box[1] > 0 ? ds->box[1] : 2.6, bz = ds->box[2] > 0 ? ds->box[2] : 3.0;
  P.X0 = (float)(-bx / 2); P.X1 = (float)(bx / 2); P.Y0 = 0.0f; P.Y1 = (float)by; P.Z0 = (float)(-bz / 2); P.Z1 = (float)(bz / 2);
  P.h = 2.2f * P.d; P.h2 = P.h * P.h;
  const double hh = P.h, dd = P.d;
  const double polyD = 315.0 / (64.0 * M_PI * pow(hh, 9)), spikyD = -45.0 / (M_PI * pow(hh, 6));
  P.poly = (float)polyD; P.spiky = (float)spikyD; P.W0 = (float)(polyD * pow(hh * hh, 3));
  P.nx = (int)ceil((P.X1 - P.X0) / P.h) + 1; P.ny = (int)ceil((P.Y1 - P.Y0) / P.h) + 1; P.nz = (int)ceil((P.Z1 - P.Z0) / P.h) + 1;
  double r0 = 0, below = 0, sgRest = 0;
  for (int i = -3; i <= 3; i++) for (int j = -3; j <= 3; j++) for (int k = -3; k <= 3; k++) {
    double r2 = (i * i + j * j + k * k) * dd * dd;
    if (r2 < hh * hh) { double w = polyD * pow(hh * hh - r2, 3); r0 += w; if (k < 0) below += w; }
  }
  P.rho0 = (float)r0;
  for (int i = -3; i <= 3; i++) for (int j = -3; j <= 3; j++) for (int k = -3; k <= 3; k++) {
    double r = sqrt((double)(i * i + j * j + k * k)) * dd;
    if (r > 1e-9 && r < hh) { double f = spikyD * (hh - r) * (hh - r) / r / r0 * r; sgRest += f * f; }
  }
  const double epsK = ds->eps_k != 0 ? ds->eps_k : 0.64, wallK = ds->wall_k != 0 ? ds->wall_k : 1.8;
  P.eps = (float)(epsK * sgRest);
  auto Gh = [](double h, double x) {
    double h2 = h * h, h4 = h2 * h2, h6 = h4 * h2, h8 = h4 * h4, s2 = x * x, s3 = s2 * x, s5 = s3 * s2, s7 = s5 * s2, s9 = s7 * s2;
    return h8 * x - (4.0 / 3) * h6 * s3 + (6.0 / 5) * h4 * s5 - (4.0 / 7) * h2 * s7 + s9 / 9;
  };
  const double c0d = (1.0 / (dd * dd * dd)) * (M_PI / 4) * polyD, Ghd = Gh(hh, hh), cont = c0d * (Ghd - Gh(hh, dd / 2));
  P.c0 = (float)(c0d * (below / cont) * wallK); P.Gh = (float)Ghd; P.margin = 0.15f * P.d; P.rest = 0.1f;
  P.inv = 1 / P.h;
  s->cap = ds->max_n;
  s->cells = P.nx * P.ny * P.nz;
  s->nblocks = (s->cells + 1023) / 1024;
  const size_t M = s->cap;
  cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  auto A = [&](void** p, size_t b) { if (e == cudaSuccess) e = cudaMalloc(p, std::max<size_t>(b, 16)); };
  A((void**)&s->P, M * 12); A((void**)&s->V, M * 12); A((void**)&s->Q, M * 12); A((void**)&s->D, M * 12); A((void**)&s->NV, M * 12);
  A((void**)&s->BG, M * 12); A((void**)&s->S, M * 4); A((void**)&s->lam, M * 4); A((void**)&s->cid, M * 4); A((void**)&s->sorted, M * 4);
  A((void**)&s->nb, M * MAXNB * 4); A((void**)&s->nc, M * 4); A((void**)&s->count, (size_t)s->cells * 4);
  A((void**)&s->start, ((size_t)s->cells + 1) * 4); A((void**)&s->cursor, (size_t)s->cells * 4); A((void**)&s->bs, ((size_t)s->nblocks + 1) * 4);
  A((void**)&s->out, M * 32);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->BG, 0, M * 12, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) {
    snprintf(g_perr, sizeof(g_perr), "create: %s", cudaGetErrorString(e)); st::set_error_text(g_perr);
    st_pbf_destroy(s);
    return e == cudaErrorMemoryAllocation ? ST_OOM : ST_DEVICE_ERROR;
  }
  *out = s;
  return ST_OK;
}

void* st_pbf_stream(st_pbf* s) { return s ? (void*)s->stream : nullptr; }

// Sim::add (native/splash.cpp:78-83) for n particles
st_status st_pbf_add(st_pbf* s, const float* p3, const float* v3, uint32_t n, uint32_t* added) {
  if (!s || (n && !p3)) return ST_BAD_ARG;
  PK(cudaSetDevice(s->device));
  uint32_t k = std::min<uint32_t>(n, s->cap - (uint32_t)s->n);
  std::vector<float> vel(k * 3, 0.0f), spd(k);
  for (uint32_t i = 0; i < k; i++) {
    if (v3) for (int a = 0; a < 3; a++) vel[i * 3 + a] = v3[i * 3 + a];
    float vx = vel[i * 3], vy = vel[i * 3 + 1], vz = vel[i * 3 + 2];
    spd[i] = sqrtf(vx * vx + vy * vy + vz * vz);
  }
  if (k) {
    PK(cudaMemcpyAsync(s->P + (size_t)s->n * 3, p3, (size_t)k * 12, cudaMemcpyHostToDevice, s->stream));
    PK(cudaMemcpyAsync(s->V + (size_t)s->n * 3, vel.data(), (size_t)k * 12, cudaMemcpyHostToDevice, s->stream));
    PK(cudaMemcpyAsync(s->S + s->n, spd.data(), (size_t)k * 4, cudaMemcpyHostToDevice, s->stream));
    PK(cudaStreamSynchronize(s->stream));
  }
  s->n += (int)k;
  if (added) *added = k;
  return ST_OK;
}

// Sim::step (native/splash.cpp:212-247)
st_status st_pbf_step(st_pbf* s, double dt, const st_pbf_opts* o) {
  if (!s || !o || o->size != sizeof(st_pbf_opts) || o->ncols > MAXCOL || (o->ncols && !o->cols)) return ST_BAD_ARG;
  if (!s->n) return ST_NOT_READY;
  PK(cudaSetDevice(s->device));
  PbfParams P = s->hp;
  P.dt = (float)dt; P.g = o->g; P.visc = o->visc; P.n = s->n; P.ncols = (int)o->ncols;
  for (uint32_t k = 0; k < o->ncols; k++) {   // Runner::step's records (native/splash.cpp:258-259)
    const st_pbf_col& c = o->cols[k];
    if (c.kind == 1) P.cols[k] = PCol{1, c.x, c.y, c.z, 0.0f, c.hx, c.hy, c.hz, cosf(c.yaw), sinf(c.yaw)};
    else P.cols[k] = PCol{0, c.x, c.y, c.z, c.r, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  }
  const int T = 256, G = (s->n + T - 1) / T, q3 = (3 * s->n + T - 1) / T;
  cudaStream_t q = s->stream;
  k_predict<<<G, T, 0, q>>>(P, s->P, s->V, s->Q);
  k_collide<<<G, T, 0, q>>>(P, s->Q);
  PK(cudaMemsetAsync(s->count, 0, (size_t)s->cells * 4, q));
  k_cells<<<G, T, 0, q>>>(P, s->Q, s->cid, s->count);
  k_blocksum<<<s->nblocks, 1024, 0, q>>>(s->count, s->cells, s->bs);
  k_scanblocks<<<1, 1024, 0, q>>>(s->bs, s->nblocks);
  k_prefix<<<s->nblocks, 1024, 0, q>>>(s->count, s->cells, s->bs, s->start, s->cursor);
  k_scatter_idx<<<G, T, 0, q>>>(P, s->cid, s->cursor, s->sorted);
  k_cell_order<<<(s->cells + T - 1) / T, T, 0, q>>>(s->cells, s->start, s->sorted);
  k_neighbors<<<G, T, 0, q>>>(P, s->Q, s->cid, s->start, s->sorted, s->nb, s->nc);
  for (int it = 0; it < o->iters; it++) {
    k_lambda<<<G, T, 0, q>>>(P, s->Q, s->nb, s->nc, s->BG, s->lam);
    k_delta<<<G, T, 0, q>>>(P, s->Q, s->nb, s->nc, s->BG, s->lam, s->D);
    k_apply<<<q3, T, 0, q>>>(3 * s->n, s->Q, s->D);
    k_collide<<<G, T, 0, q>>>(P, s->Q);
  }
  k_velocity<<<G, T, 0, q>>>(P, s->P, s->Q, s->BG, s->V);
  if (o->visc > 0) {
    k_visc<<<G, T, 0, q>>>(P, s->Q, s->V, s->nb, s->nc, s->NV);
    PK(cudaMemcpyAsync(s->V, s->NV, (size_t)s->n * 12, cudaMemcpyDeviceToDevice, q));
  }
  k_commit<<<G, T, 0, q>>>(P, s->P, s->Q, s->V, s->S);
  PK(cudaGetLastError());
  return ST_OK;
}

st_status st_pbf_read(st_pbf* s, float* pos4, float* vel4, uint32_t cap, uint32_t* n) {
  if (!s || !pos4) return ST_BAD_ARG;
  PK(cudaSetDevice(s->device));
  if (n) *n = (uint32_t)s->n;
  const uint32_t m = std::min<uint32_t>(cap, (uint32_t)s->n);
  if (!m) return ST_OK;
  k_pack<<<(s->n + 255) / 256, 256, 0, s->stream>>>(s->n, s->P, s->S, s->V, s->out, vel4 ? s->out + s->cap : nullptr);
  PK(cudaGetLastError());
  PK(cudaMemcpyAsync(pos4, s->out, (size_t)m * 16, cudaMemcpyDeviceToHost, s->stream));
  if (vel4) PK(cudaMemcpyAsync(vel4, s->out + s->cap, (size_t)m * 16, cudaMemcpyDeviceToHost, s->stream));
  PK(cudaStreamSynchronize(s->stream));
  return ST_OK;
}

}  // extern "C"
