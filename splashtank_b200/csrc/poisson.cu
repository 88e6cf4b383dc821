// poisson.cu - the pressure projection's linear solve on its own (st_poisson_*), for the precision study: the reference's
// red-black SOR (relax, src/flip/wgsl-solver.js:124-140) in FP32, the same FP32 sweeps inside FP64 iterative refinement,
// and FP64 SOR.
//
// Operator: for a fluid cell c, nns = neighbours that are not solid (outside the box counts as solid unless that face is
// open) and A p(c) = nns p(c) - sum of fluid neighbours' p; air neighbours are p = 0. SOR: p += omega ((rhs + sum)/nns - p).
// Refinement: x (FP64) = 0, r = b; repeat: e = FP32 SOR sweeps on A e = (float) r from e = 0, x += e, r = b - A x in FP64,
// until ||r|| / ||b|| <= tol. Only the residual and the correction use FP64.
//
// Layout: the tile-major layout of the FLIP grid (8^3 tiles, cell t*512 + local); only tiles holding fluid are visited.
// Norms are summed per tile in cell order, then over tiles in tile order by one CTA, so they are reproducible.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/splashtank_cuda.h"
#include "common.cuh"

namespace {

struct PGeo { uint32_t nx, ny, nz, tx, ty, tz; };

__device__ __forceinline__ void neighbours(const PGeo& G, uint32_t t, uint32_t local, uint32_t* nb) {
  const uint32_t c = t * 512u + local;
  const int lx = local & 7, ly = (local >> 3) & 7, lz = local >> 6;
  const uint32_t tt = t / G.tx, ti = t % G.tx, tj = tt % G.ty, tk = tt / G.ty;
  const uint32_t slab = 512u * G.tx * G.ty;
  nb[0] = lx > 0 ? c - 1u : (ti > 0 ? c - 512u + 7u : c);
  nb[1] = lx < 7 ? c + 1u : (ti + 1 < G.tx ? c + 512u - 7u : c);
  nb[2] = ly > 0 ? c - 8u : (tj > 0 ? c - 512u * G.tx + 56u : c);
  nb[3] = ly < 7 ? c + 8u : (tj + 1 < G.ty ? c + 512u * G.tx - 56u : c);
  nb[4] = lz > 0 ? c - 64u : (tk > 0 ? c - slab + 448u : c);
  nb[5] = lz < 7 ? c + 64u : (tk + 1 < G.tz ? c + slab - 448u : c);
}

// one colour sweep in FP32 (same arithmetic as the FLIP step's k_sor)
__global__ void __launch_bounds__(256) k_ps_sor32(PGeo G, const uint32_t* __restrict__ tiles, uint32_t nT, const uint16_t* __restrict__ info,
                                                  float* __restrict__ p, const float* __restrict__ rhs, float omega, uint32_t color) {
  const int lz = threadIdx.x >> 5, ly = (threadIdx.x >> 2) & 7;
  const int lx = 2 * (threadIdx.x & 3) + (int)((ly + lz + color) & 1);
  const uint32_t local = (uint32_t)(lx + 8 * (ly + 8 * lz));
  for (uint32_t a = blockIdx.x; a < nT; a += gridDim.x) {
    const uint32_t t = tiles[a], c = t * 512u + local;
    uint32_t nb[6];
    neighbours(G, t, local, nb);
    const uint32_t in = info[c];
    const float p0 = p[c], r0 = rhs[c];
    const float q0 = p[nb[0]], q1 = p[nb[1]], q2 = p[nb[2]], q3 = p[nb[3]], q4 = p[nb[4]], q5 = p[nb[5]];
    if (!(in & 0x8000u)) continue;
    const uint32_t nns = (in >> 8) & 7u;
    if (nns == 0u) { p[c] = 0.0f; continue; }
    float sum = 0.0f;
    if (in & 1u) sum += q0;
    if (in & 2u) sum += q1;
    if (in & 4u) sum += q2;
    if (in & 8u) sum += q3;
    if (in & 16u) sum += q4;
    if (in & 32u) sum += q5;
    const float pg = (r0 + sum) / (float)nns;
    p[c] = p0 + omega * (pg - p0);
  }
}
// one colour sweep in FP64
__global__ void __launch_bounds__(256) k_ps_sor64(PGeo G, const uint32_t* __restrict__ tiles, uint32_t nT, const uint16_t* __restrict__ info,
                                                  double* __restrict__ p, const double* __restrict__ rhs, double omega, uint32_t color) {
  const int lz = threadIdx.x >> 5, ly = (threadIdx.x >> 2) & 7;
  const int lx = 2 * (threadIdx.x & 3) + (int)((ly + lz + color) & 1);
  const uint32_t local = (uint32_t)(lx + 8 * (ly + 8 * lz));
  for (uint32_t a = blockIdx.x; a < nT; a += gridDim.x) {
    const uint32_t t = tiles[a], c = t * 512u + local;
    uint32_t nb[6];
    neighbours(G, t, local, nb);
    const uint32_t in = info[c];
    const double p0 = p[c], r0 = rhs[c];
    const double q0 = p[nb[0]], q1 = p[nb[1]], q2 = p[nb[2]], q3 = p[nb[3]], q4 = p[nb[4]], q5 = p[nb[5]];
    if (!(in & 0x8000u)) continue;
    const uint32_t nns = (in >> 8) & 7u;
    if (nns == 0u) { p[c] = 0.0; continue; }
    double sum = 0.0;
    if (in & 1u) sum += q0;
    if (in & 2u) sum += q1;
    if (in & 4u) sum += q2;
    if (in & 8u) sum += q3;
    if (in & 16u) sum += q4;
    if (in & 32u) sum += q5;
    const double pg = (r0 + sum) / (double)nns;
    p[c] = p0 + omega * (pg - p0);
  }
}
// r = b - A x in FP64 for x in FP64 (x64) or FP32 (x32); per-tile sums of r^2 in cell order (and b^2 when asked)
template <class T>
__global__ void __launch_bounds__(512) k_ps_resid(PGeo G, const uint32_t* __restrict__ tiles, uint32_t nT, const uint16_t* __restrict__ info,
                                                  const T* __restrict__ x, const double* __restrict__ b, double* __restrict__ r,
                                                  double* __restrict__ tileR2, double* __restrict__ tileB2) {
  __shared__ double sr[512], sb[512];
  for (uint32_t a = blockIdx.x; a < nT; a += gridDim.x) {
    const uint32_t t = tiles[a], c = t * 512u + threadIdx.x;
    uint32_t nb[6];
    neighbours(G, t, threadIdx.x, nb);
    const uint32_t in = info[c];
    double rv = 0.0, bv = 0.0;
    if (in & 0x8000u) {
      const uint32_t nns = (in >> 8) & 7u;
      double s = 0.0;
      for (int q = 0; q < 6; q++) if (in & (1u << q)) s += (double)x[nb[q]];
      bv = b[c];
      rv = bv - ((double)nns * (double)x[c] - s);
    }
    r[c] = rv;
    sr[threadIdx.x] = rv * rv;
    sb[threadIdx.x] = bv * bv;
    __syncthreads();
    // fixed-order tree over the tile's 512 cells
    for (int w = 256; w > 0; w >>= 1) {
      if ((int)threadIdx.x < w) { sr[threadIdx.x] += sr[threadIdx.x + w]; sb[threadIdx.x] += sb[threadIdx.x + w]; }
      __syncthreads();
    }
    if (threadIdx.x == 0) { tileR2[a] = sr[0]; if (tileB2) tileB2[a] = sb[0]; }
    __syncthreads();
  }
}
// sum of per-tile partials in tile order (one CTA, fixed tree): out[0] = sum tileR2, out[1] = sum tileB2
__global__ void __launch_bounds__(1024) k_ps_norms(const double* __restrict__ tileR2, const double* __restrict__ tileB2, uint32_t nT, double* out) {
  __shared__ double s1[1024], s2[1024];
  double a = 0.0, b = 0.0;
  const uint32_t chunk = (nT + 1023) / 1024, beg = min(threadIdx.x * chunk, nT), end = min(beg + chunk, nT);
  for (uint32_t k = beg; k < end; k++) { a += tileR2[k]; if (tileB2) b += tileB2[k]; }
  s1[threadIdx.x] = a;
  s2[threadIdx.x] = b;
  __syncthreads();
  for (int w = 512; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) { s1[threadIdx.x] += s1[threadIdx.x + w]; s2[threadIdx.x] += s2[threadIdx.x + w]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { out[0] = s1[0]; out[1] = s2[0]; }
}
// refinement helpers: inner right-hand side and zero start; correction x += e
__global__ void k_ps_inner(const uint32_t* __restrict__ tiles, uint32_t nT, const double* __restrict__ r, float* __restrict__ rhs32, float* __restrict__ e) {
  for (uint32_t a = blockIdx.x; a < nT; a += gridDim.x) {
    const uint32_t c = tiles[a] * 512u + threadIdx.x;
    rhs32[c] = (float)r[c];
    e[c] = 0.0f;
  }
}
__global__ void k_ps_correct(const uint32_t* __restrict__ tiles, uint32_t nT, const float* __restrict__ e, double* __restrict__ x) {
  for (uint32_t a = blockIdx.x; a < nT; a += gridDim.x) {
    const uint32_t c = tiles[a] * 512u + threadIdx.x;
    x[c] = x[c] + (double)e[c];
  }
}
__global__ void k_ps_copy(const uint32_t* __restrict__ tiles, uint32_t nT, const float* __restrict__ p32, double* __restrict__ x) {
  for (uint32_t a = blockIdx.x; a < nT; a += gridDim.x) {
    const uint32_t c = tiles[a] * 512u + threadIdx.x;
    x[c] = (double)p32[c];
  }
}

thread_local char g_serr[256] = "";

}  // namespace

struct st_poisson {
  int device = 0;
  cudaStream_t stream = nullptr;
  int sms = 148;
  PGeo G{};
  uint32_t open = 0, nT = 0;
  size_t ncell = 0;
  uint32_t* tiles = nullptr;
  uint16_t* info = nullptr;
  float *p32 = nullptr, *rhs32 = nullptr;
  double *x64 = nullptr, *b64 = nullptr, *r64 = nullptr, *tileR2 = nullptr, *tileB2 = nullptr, *norms = nullptr;
  double bnorm2 = 0.0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
};

#define SK(call)                                                                            \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) {                                                                \
      snprintf(g_serr, sizeof(g_serr), "%s: %s", #call, cudaGetErrorString(e_)); st::set_error_text(g_serr);            \
      return e_ == cudaErrorMemoryAllocation ? ST_OOM : ST_DEVICE_ERROR;                    \
    }                                                                                       \
  } while (0)

extern "C" {

void st_poisson_destroy(st_poisson* s) {
  if (!s) return;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  void* ptrs[] = {s->tiles, s->info, s->p32, s->rhs32, s->x64, s->b64, s->r64, s->tileR2, s->tileB2, s->norms};
  for (void* p : ptrs) if (p) cudaFree(p);
  if (s->e0) cudaEventDestroy(s->e0);
  if (s->e1) cudaEventDestroy(s->e1);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

st_status st_poisson_create(const st_poisson_desc* d, st_poisson** out) {
  if (!d || !out || d->size != sizeof(st_poisson_desc) || !d->n[0] || !d->n[1] || !d->n[2]) return ST_BAD_ARG;
  st_poisson* s = new st_poisson();
  *out = nullptr;
  s->device = d->device;
  if (cudaSetDevice(s->device) != cudaSuccess) { delete s; return ST_DEVICE_ERROR; }
  cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, s->device);
  s->G = PGeo{d->n[0], d->n[1], d->n[2], (d->n[0] + 7) / 8, (d->n[1] + 7) / 8, (d->n[2] + 7) / 8};
  s->open = d->open;
  const size_t T = (size_t)s->G.tx * s->G.ty * s->G.tz;
  s->ncell = T * 512;
  cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  auto A = [&](void** p, size_t b) { if (e == cudaSuccess) e = cudaMalloc(p, std::max<size_t>(b, 16)); };
  A((void**)&s->tiles, T * 4); A((void**)&s->info, s->ncell * 2); A((void**)&s->p32, s->ncell * 4); A((void**)&s->rhs32, s->ncell * 4);
  A((void**)&s->x64, s->ncell * 8); A((void**)&s->b64, s->ncell * 8); A((void**)&s->r64, s->ncell * 8);
  A((void**)&s->tileR2, T * 8); A((void**)&s->tileB2, T * 8); A((void**)&s->norms, 16);
  if (e == cudaSuccess) e = cudaEventCreate(&s->e0);
  if (e == cudaSuccess) e = cudaEventCreate(&s->e1);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->p32, 0, s->ncell * 4, s->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->x64, 0, s->ncell * 8, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) {
    snprintf(g_serr, sizeof(g_serr), "create: %s", cudaGetErrorString(e)); st::set_error_text(g_serr);
    st_poisson_destroy(s);
    return e == cudaErrorMemoryAllocation ? ST_OOM : ST_DEVICE_ERROR;
  }
  *out = s;
  return ST_OK;
}

// cell types (0 air, 1 fluid, 2 solid) and right-hand side, dense over n[0] x n[1] x n[2], x fastest
st_status st_poisson_set(st_poisson* s, const uint8_t* type, const double* rhs) {
  if (!s || !type || !rhs) return ST_BAD_ARG;
  SK(cudaSetDevice(s->device));
  const PGeo& G = s->G;
  const size_t T = (size_t)G.tx * G.ty * G.tz;
  std::vector<uint16_t> info(s->ncell, 0);
  std::vector<double> b(s->ncell, 0.0);
  std::vector<uint8_t> tileOn(T, 0);
  auto ty = [&](long i, long j, long k) -> int {   // ctypeOf (src/flip/wgsl-core.js:104-112)
    if (i < 0) return (s->open & 1u) ? 0 : 2;
    if (i >= (long)G.nx) return (s->open & 2u) ? 0 : 2;
    if (j < 0) return (s->open & 4u) ? 0 : 2;
    if (j >= (long)G.ny) return (s->open & 8u) ? 0 : 2;
    if (k < 0) return (s->open & 16u) ? 0 : 2;
    if (k >= (long)G.nz) return (s->open & 32u) ? 0 : 2;
    return type[(size_t)i + G.nx * ((size_t)j + (size_t)G.ny * k)];
  };
  for (long k = 0; k < (long)G.nz; k++)
    for (long j = 0; j < (long)G.ny; j++)
      for (long i = 0; i < (long)G.nx; i++) {
        const size_t o = (size_t)i + G.nx * ((size_t)j + (size_t)G.ny * k);
        if (type[o] != 1) continue;
        const size_t t = (size_t)(i >> 3) + G.tx * ((size_t)(j >> 3) + (size_t)G.ty * (k >> 3));
        const size_t c = t * 512 + (i & 7) + 8 * ((j & 7) + 8 * (k & 7));
        const long q[6][3] = {{i - 1, j, k}, {i + 1, j, k}, {i, j - 1, k}, {i, j + 1, k}, {i, j, k - 1}, {i, j, k + 1}};
        uint32_t mask = 0, nns = 0;
        for (int a = 0; a < 6; a++) {
          const int tq = ty(q[a][0], q[a][1], q[a][2]);
          if (tq != 2) nns++;
          if (tq == 1) mask |= 1u << a;
        }
        info[c] = (uint16_t)(0x8000u | (nns << 8) | mask);
        b[c] = rhs[o];
        tileOn[t] = 1;
      }
  std::vector<uint32_t> tiles;
  for (size_t t = 0; t < T; t++) if (tileOn[t]) tiles.push_back((uint32_t)t);
  s->nT = (uint32_t)tiles.size();
  cudaStream_t q = s->stream;
  SK(cudaMemcpyAsync(s->info, info.data(), s->ncell * 2, cudaMemcpyHostToDevice, q));
  SK(cudaMemcpyAsync(s->b64, b.data(), s->ncell * 8, cudaMemcpyHostToDevice, q));
  SK(cudaMemcpyAsync(s->tiles, tiles.data(), std::max<size_t>(tiles.size(), 1) * 4, cudaMemcpyHostToDevice, q));
  SK(cudaMemsetAsync(s->p32, 0, s->ncell * 4, q));
  SK(cudaMemsetAsync(s->x64, 0, s->ncell * 8, q));
  SK(cudaStreamSynchronize(q));
  return ST_OK;
}

static st_status norms(st_poisson* s, bool withB, double* r2, double* b2) {
  cudaStream_t q = s->stream;
  k_ps_norms<<<1, 1024, 0, q>>>(s->tileR2, withB ? s->tileB2 : nullptr, s->nT, s->norms);
  double h[2];
  SK(cudaMemcpyAsync(h, s->norms, 16, cudaMemcpyDeviceToHost, q));
  SK(cudaStreamSynchronize(q));
  *r2 = h[0];
  if (b2) *b2 = h[1];
  return ST_OK;
}

// Solve from zero. mode 0: FP32 SOR (the residual is measured in FP64 every check_every iterations);
// 1: FP32 SOR inside FP64 refinement (inner_sweeps iterations per refinement); 2: FP64 SOR.
st_status st_poisson_solve(st_poisson* s, const st_poisson_opts* o, st_poisson_result* res) {
  if (!s || !o || !res || o->size != sizeof(st_poisson_opts)) return ST_BAD_ARG;
  SK(cudaSetDevice(s->device));
  memset(res, 0, sizeof(*res));
  if (!s->nT) { res->converged = 1; return ST_OK; }
  cudaStream_t q = s->stream;
  const int grid = std::max(1, std::min<int>(s->sms * 8, (int)s->nT)), grid4 = std::max(1, std::min<int>(s->sms * 4, (int)s->nT));
  const int check = std::max(1, o->check_every), maxIt = std::max(1, o->max_sweeps);
  const float om = o->omega;
  SK(cudaMemsetAsync(s->p32, 0, s->ncell * 4, q));
  SK(cudaMemsetAsync(s->x64, 0, s->ncell * 8, q));
  // ||b|| once, from the residual of x = 0
  k_ps_resid<double><<<grid4, 512, 0, q>>>(s->G, s->tiles, s->nT, s->info, s->x64, s->b64, s->r64, s->tileR2, s->tileB2);
  double r2 = 0, b2 = 0;
  st_status st = norms(s, true, &r2, &b2);
  if (st != ST_OK) return st;
  s->bnorm2 = b2;
  const double bn = std::sqrt(b2);
  if (bn == 0.0) { res->converged = 1; return ST_OK; }
  SK(cudaEventRecord(s->e0, q));
  int it = 0, ref = 0;
  double rel = 1.0;
  if (o->mode == 0) {
    k_ps_inner<<<grid4, 512, 0, q>>>(s->tiles, s->nT, s->b64, s->rhs32, s->p32);
    while (it < maxIt) {
      for (int k = 0; k < check && it < maxIt; k++, it++) {
        k_ps_sor32<<<grid, 256, 0, q>>>(s->G, s->tiles, s->nT, s->info, s->p32, s->rhs32, om, 0u);
        k_ps_sor32<<<grid, 256, 0, q>>>(s->G, s->tiles, s->nT, s->info, s->p32, s->rhs32, om, 1u);
      }
      k_ps_resid<float><<<grid4, 512, 0, q>>>(s->G, s->tiles, s->nT, s->info, s->p32, s->b64, s->r64, s->tileR2, nullptr);
      st = norms(s, false, &r2, nullptr);
      if (st != ST_OK) return st;
      rel = std::sqrt(r2) / bn;
      if (rel <= o->tol) break;
    }
    k_ps_copy<<<grid4, 512, 0, q>>>(s->tiles, s->nT, s->p32, s->x64);
  } else if (o->mode == 1) {
    const int inner = std::max(1, o->inner_sweeps);
    while (it < maxIt) {
      k_ps_inner<<<grid4, 512, 0, q>>>(s->tiles, s->nT, s->r64, s->rhs32, s->p32);
      for (int k = 0; k < inner && it < maxIt; k++, it++) {
        k_ps_sor32<<<grid, 256, 0, q>>>(s->G, s->tiles, s->nT, s->info, s->p32, s->rhs32, om, 0u);
        k_ps_sor32<<<grid, 256, 0, q>>>(s->G, s->tiles, s->nT, s->info, s->p32, s->rhs32, om, 1u);
      }
      k_ps_correct<<<grid4, 512, 0, q>>>(s->tiles, s->nT, s->p32, s->x64);
      k_ps_resid<double><<<grid4, 512, 0, q>>>(s->G, s->tiles, s->nT, s->info, s->x64, s->b64, s->r64, s->tileR2, nullptr);
      ref++;
      st = norms(s, false, &r2, nullptr);
      if (st != ST_OK) return st;
      rel = std::sqrt(r2) / bn;
      if (rel <= o->tol) break;
    }
  } else if (o->mode == 2) {
    while (it < maxIt) {
      for (int k = 0; k < check && it < maxIt; k++, it++) {
        k_ps_sor64<<<grid, 256, 0, q>>>(s->G, s->tiles, s->nT, s->info, s->x64, s->b64, (double)om, 0u);
        k_ps_sor64<<<grid, 256, 0, q>>>(s->G, s->tiles, s->nT, s->info, s->x64, s->b64, (double)om, 1u);
      }
      k_ps_resid<double><<<grid4, 512, 0, q>>>(s->G, s->tiles, s->nT, s->info, s->x64, s->b64, s->r64, s->tileR2, nullptr);
      st = norms(s, false, &r2, nullptr);
      if (st != ST_OK) return st;
      rel = std::sqrt(r2) / bn;
      if (rel <= o->tol) break;
    }
  } else {
    return ST_BAD_ARG;
  }
  SK(cudaEventRecord(s->e1, q));
  SK(cudaEventSynchronize(s->e1));
  SK(cudaGetLastError());
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, s->e0, s->e1);
  res->rel_residual = rel;
  res->sweeps = it;
  res->refinements = ref;
  res->converged = rel <= o->tol ? 1 : 0;
  res->ms = ms;
  return ST_OK;
}

// FP32 SOR iterations (red + black) on (float) b from p = 0, nothing else: the unit the parity tests compare
st_status st_poisson_sweeps32(st_poisson* s, float omega, int32_t iters, float* ms) {
  if (!s) return ST_BAD_ARG;
  SK(cudaSetDevice(s->device));
  if (ms) *ms = 0.0f;
  if (!s->nT) return ST_OK;
  cudaStream_t q = s->stream;
  const int grid = std::max(1, std::min<int>(s->sms * 8, (int)s->nT)), grid4 = std::max(1, std::min<int>(s->sms * 4, (int)s->nT));
  k_ps_inner<<<grid4, 512, 0, q>>>(s->tiles, s->nT, s->b64, s->rhs32, s->p32);
  SK(cudaEventRecord(s->e0, q));
  for (int k = 0; k < iters; k++) {
    k_ps_sor32<<<grid, 256, 0, q>>>(s->G, s->tiles, s->nT, s->info, s->p32, s->rhs32, omega, 0u);
    k_ps_sor32<<<grid, 256, 0, q>>>(s->G, s->tiles, s->nT, s->info, s->p32, s->rhs32, omega, 1u);
  }
  SK(cudaEventRecord(s->e1, q));
  k_ps_copy<<<grid4, 512, 0, q>>>(s->tiles, s->nT, s->p32, s->x64);
  SK(cudaStreamSynchronize(q));
  SK(cudaGetLastError());
  if (ms) SK(cudaEventElapsedTime(ms, s->e0, s->e1));
  return ST_OK;
}

// the solution (FP64, dense, x fastest) and the relative residual of a given dense FP64 field
st_status st_poisson_read(st_poisson* s, double* p) {
  if (!s || !p) return ST_BAD_ARG;
  SK(cudaSetDevice(s->device));
  const PGeo& G = s->G;
  std::vector<double> x(s->ncell);
  SK(cudaMemcpyAsync(x.data(), s->x64, s->ncell * 8, cudaMemcpyDeviceToHost, s->stream));
  SK(cudaStreamSynchronize(s->stream));
  for (size_t k = 0; k < G.nz; k++)
    for (size_t j = 0; j < G.ny; j++)
      for (size_t i = 0; i < G.nx; i++) {
        const size_t t = (i >> 3) + G.tx * ((j >> 3) + (size_t)G.ty * (k >> 3));
        p[i + G.nx * (j + (size_t)G.ny * k)] = x[t * 512 + (i & 7) + 8 * ((j & 7) + 8 * (k & 7))];
      }
  return ST_OK;
}

void* st_poisson_stream(st_poisson* s) { return s ? (void*)s->stream : nullptr; }

}  // extern "C"

// ---- residual norm without allocation (st_poisson_residual_noalloc) ----
// Its scratch is this fixed array: per-tile partial sums of r^2 and b^2, the two totals and an error word. One copy
// per device; the host looks its address up once per device.
namespace {

constexpr uint32_t kNoAllocTiles = ST_NOALLOC_MAX_TILES;
static __device__ __align__(256) double g_noalloc_scratch[2 * kNoAllocTiles + 4];

// r = b - A x in FP64 summed per tile (the same arithmetic and tree as k_ps_resid), without storing r; a tile index
// outside the box sets the error word and its partials to zero instead of reading
__global__ void __launch_bounds__(512) k_ps_resid_norm(PGeo G, const uint32_t* __restrict__ tiles, uint32_t nT, uint32_t nTiles,
                                                       const uint16_t* __restrict__ info, const double* __restrict__ x,
                                                       const double* __restrict__ b, double* __restrict__ tileR2,
                                                       double* __restrict__ tileB2, unsigned long long* __restrict__ bad) {
  __shared__ double sr[512], sb[512];
  for (uint32_t a = blockIdx.x; a < nT; a += gridDim.x) {
    const uint32_t t = tiles[a];
    double rv = 0.0, bv = 0.0;
    if (t < nTiles) {
      const uint32_t c = t * 512u + threadIdx.x;
      uint32_t nb[6];
      neighbours(G, t, threadIdx.x, nb);
      const uint32_t in = info[c];
      if (in & 0x8000u) {
        const uint32_t nns = (in >> 8) & 7u;
        double s = 0.0;
        for (int q = 0; q < 6; q++) if (in & (1u << q)) s += x[nb[q]];
        bv = b[c];
        rv = bv - ((double)nns * x[c] - s);
      }
    } else if (threadIdx.x == 0) {
      atomicExch(bad, 1ull);
    }
    sr[threadIdx.x] = rv * rv;
    sb[threadIdx.x] = bv * bv;
    __syncthreads();
    for (int w = 256; w > 0; w >>= 1) {
      if ((int)threadIdx.x < w) { sr[threadIdx.x] += sr[threadIdx.x + w]; sb[threadIdx.x] += sb[threadIdx.x + w]; }
      __syncthreads();
    }
    if (threadIdx.x == 0) { tileR2[a] = sr[0]; tileB2[a] = sb[0]; }
    __syncthreads();
  }
}

struct NoAllocDev {
  double* scratch = nullptr;
  int sms = 0;
};
constexpr int kNoAllocMaxDevices = 64;
NoAllocDev g_noalloc_dev[kNoAllocMaxDevices];
std::mutex g_noalloc_mu;

void noalloc_err(const char* text) { st::set_error_text(text); }

}  // namespace

extern "C" st_status st_poisson_residual_noalloc(const st_poisson_system* sys, const double* x, void* stream, double* rel,
                                                double* r2, double* b2) {
  char msg[256];
  if (!sys || !rel || sys->size != sizeof(st_poisson_system) || !sys->n[0] || !sys->n[1] || !sys->n[2]) {
    noalloc_err("st_poisson_residual_noalloc: null argument, wrong st_poisson_system.size or an empty box");
    return ST_BAD_ARG;
  }
  const uint64_t tx = (sys->n[0] + 7) / 8, ty = (sys->n[1] + 7) / 8, tz = (sys->n[2] + 7) / 8, nTiles = tx * ty * tz;
  if (nTiles * 512u > 0xffffffffull) {
    noalloc_err("st_poisson_residual_noalloc: box too large for 32-bit cell indices");
    return ST_BAD_ARG;
  }
  if (sys->n_tiles > kNoAllocTiles) {
    snprintf(msg, sizeof(msg), "st_poisson_residual_noalloc: n_tiles %u exceeds the fixed scratch of %u tiles", sys->n_tiles, kNoAllocTiles);
    noalloc_err(msg);
    return ST_BAD_ARG;
  }
  if (sys->n_tiles && (!sys->tiles || !sys->info || !sys->b || !x)) {
    noalloc_err("st_poisson_residual_noalloc: null device array");
    return ST_BAD_ARG;
  }
  *rel = 0.0;
  if (r2) *r2 = 0.0;
  if (b2) *b2 = 0.0;
  if (!sys->n_tiles) return ST_OK;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) {
    snprintf(msg, sizeof(msg), "st_poisson_residual_noalloc: current device %d: %s", dev, cudaGetErrorString(e));
    noalloc_err(msg);
    return ST_DEVICE_ERROR;
  }
  NoAllocDev d;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_dev[dev].scratch) {   // first call on this device: look the scratch up with the device current
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      int sms = 0;
      if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) {
        snprintf(msg, sizeof(msg), "st_poisson_residual_noalloc: scratch lookup on device %d: %s", dev, cudaGetErrorString(e));
        noalloc_err(msg);
        return ST_DEVICE_ERROR;
      }
      g_noalloc_dev[dev].scratch = (double*)p;
      g_noalloc_dev[dev].sms = sms;
    }
    d = g_noalloc_dev[dev];
  }
  double* tileR2 = d.scratch;
  double* tileB2 = d.scratch + kNoAllocTiles;
  double* tot = d.scratch + 2 * kNoAllocTiles;                                      // [0] r^2, [1] b^2
  unsigned long long* bad = (unsigned long long*)(d.scratch + 2 * kNoAllocTiles + 2);  // must start at zero
  cudaStream_t q = (cudaStream_t)stream;
  const PGeo G{sys->n[0], sys->n[1], sys->n[2], (uint32_t)tx, (uint32_t)ty, (uint32_t)tz};
  const int grid = std::max(1, std::min<int>(d.sms * 4, (int)sys->n_tiles));
  double h[3] = {0.0, 0.0, 0.0};
  e = cudaMemsetAsync(bad, 0, sizeof(unsigned long long), q);
  if (e == cudaSuccess) {
    k_ps_resid_norm<<<grid, 512, 0, q>>>(G, sys->tiles, sys->n_tiles, (uint32_t)nTiles, sys->info, x, sys->b, tileR2, tileB2, bad);
    k_ps_norms<<<1, 1024, 0, q>>>(tileR2, tileB2, sys->n_tiles, tot);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, tot, 3 * sizeof(double), cudaMemcpyDeviceToHost, q);
  if (e == cudaSuccess) e = cudaStreamSynchronize(q);
  if (e != cudaSuccess) {
    snprintf(msg, sizeof(msg), "st_poisson_residual_noalloc: %s", cudaGetErrorString(e));
    noalloc_err(msg);
    return ST_DEVICE_ERROR;
  }
  unsigned long long badv = 0;
  memcpy(&badv, &h[2], sizeof(badv));
  if (badv) {
    noalloc_err("st_poisson_residual_noalloc: a tile index is outside the box");
    return ST_BAD_ARG;
  }
  *rel = h[1] > 0.0 ? std::sqrt(h[0]) / std::sqrt(h[1]) : 0.0;
  if (r2) *r2 = h[0];
  if (b2) *b2 = h[1];
  return ST_OK;
}
