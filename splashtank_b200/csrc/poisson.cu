// poisson.cu - the pressure projection's linear solve on its own (st_poisson_*), for the precision study: the reference's
// red-black SOR (relax, src/flip/wgsl-solver.js:124-140) in FP32, the same FP32 sweeps inside FP64 iterative refinement,
// and FP64 SOR.
//
// Operator: for a fluid cell c, nns = neighbours that are not solid (outside the box counts as solid unless that face is
// open) and A p(c) = nns p(c) - sum of fluid neighbours' p; air neighbours are p = 0. SOR: p += omega ((rhs + sum)/nns - p).
// Refinement: x (FP64) = 0, r = b; repeat: e = FP32 SOR sweeps on A e = (float) r from e = 0, x += e, r = b - A x in FP64,
// until ||r|| / ||b|| <= tol. Only the residual and the correction use FP64.
//
// Layout: only the 8^3 tiles holding fluid are stored, in ascending tile order (slot a); a slot holds its tile's red
// cells then its black ones, each half ordered (lx / 2) + 4 (ly + 8 lz), and nbs gives the slots of its 6 face
// neighbours (its own slot when a neighbour holds no fluid: such values are never summed). A sweep's loads are then
// contiguous per warp. Norms are summed per tile over the cells in (lx, ly, lz) order by a fixed tree, then over tiles
// in tile order by one CTA, so they are reproducible.
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

// standard tile-major neighbours (used by the residual on caller arrays below)
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

// position of local cell l inside its slot
__host__ __device__ __forceinline__ uint32_t splitIdx(uint32_t l) {
  const uint32_t lx = l & 7u, ly = (l >> 3) & 7u, lz = l >> 6;
  return ((lx + ly + lz) & 1u) * 256u + (lx >> 1) + 4u * (ly + 8u * lz);
}
// compact index of the face neighbour of local cell l of slot a in direction dir (-x, +x, -y, +y, -z, +z)
__device__ __forceinline__ uint32_t nbIdx(const uint32_t* __restrict__ nbs, uint32_t a, uint32_t l, int dir) {
  const uint32_t lx = l & 7u, ly = (l >> 3) & 7u, lz = l >> 6;
  uint32_t sl = a, nl = l;
  switch (dir) {
    case 0: if (lx > 0) nl = l - 1u; else { sl = nbs[a * 6u]; nl = l + 7u; } break;
    case 1: if (lx < 7) nl = l + 1u; else { sl = nbs[a * 6u + 1u]; nl = l - 7u; } break;
    case 2: if (ly > 0) nl = l - 8u; else { sl = nbs[a * 6u + 2u]; nl = l + 56u; } break;
    case 3: if (ly < 7) nl = l + 8u; else { sl = nbs[a * 6u + 3u]; nl = l - 56u; } break;
    case 4: if (lz > 0) nl = l - 64u; else { sl = nbs[a * 6u + 4u]; nl = l + 448u; } break;
    default: if (lz < 7) nl = l + 64u; else { sl = nbs[a * 6u + 5u]; nl = l - 448u; } break;
  }
  return sl * 512u + splitIdx(nl);
}

// one colour sweep (thread j: the colour's cell (lx / 2) + 4 (ly + 8 lz) = j), same arithmetic as the FLIP step's
template <class T>
__global__ void __launch_bounds__(256) k_ps_sor(uint32_t nT, const uint32_t* __restrict__ nbs, const uint16_t* __restrict__ info,
                                                T* __restrict__ p, const T* __restrict__ rhs, T omega, uint32_t color) {
  const uint32_t j = threadIdx.x, lz = j >> 5, ly = (j >> 2) & 7u;
  const uint32_t lx = 2u * (j & 3u) + ((ly + lz + color) & 1u), row = j & ~3u;
  const uint32_t own = color * 256u + j, oth = (color ^ 1u) * 256u;
  for (uint32_t a = blockIdx.x; a < nT; a += gridDim.x) {
    const uint32_t* nb = nbs + a * 6u;
    const uint32_t base = a * 512u + oth;
    const uint32_t ixm = lx > 0 ? base + row + ((lx - 1u) >> 1) : nb[0] * 512u + oth + row + 3u;
    const uint32_t ixp = lx < 7 ? base + row + ((lx + 1u) >> 1) : nb[1] * 512u + oth + row;
    const uint32_t iym = ly > 0 ? base + j - 4u : nb[2] * 512u + oth + j + 28u;
    const uint32_t iyp = ly < 7 ? base + j + 4u : nb[3] * 512u + oth + j - 28u;
    const uint32_t izm = lz > 0 ? base + j - 32u : nb[4] * 512u + oth + j + 224u;
    const uint32_t izp = lz < 7 ? base + j + 32u : nb[5] * 512u + oth + j - 224u;
    const uint32_t c = a * 512u + own;
    const uint32_t in = info[c];
    const T p0 = p[c], r0 = rhs[c];
    const T q0 = p[ixm], q1 = p[ixp], q2 = p[iym], q3 = p[iyp], q4 = p[izm], q5 = p[izp];
    if (!(in & 0x8000u)) continue;
    const uint32_t nns = (in >> 8) & 7u;
    if (nns == 0u) { p[c] = (T)0; continue; }
    T sum = (T)0;
    if (in & 1u) sum += q0;
    if (in & 2u) sum += q1;
    if (in & 4u) sum += q2;
    if (in & 8u) sum += q3;
    if (in & 16u) sum += q4;
    if (in & 32u) sum += q5;
    const T pg = (r0 + sum) / (T)nns;
    p[c] = p0 + omega * (pg - p0);
  }
}
// r = b - A x in FP64 for x in FP64 or FP32; per-tile sums of r^2 (and b^2 when asked) over the cells in local order
template <class T>
__global__ void __launch_bounds__(512) k_ps_resid(uint32_t nT, const uint32_t* __restrict__ nbs, const uint16_t* __restrict__ info,
                                                  const T* __restrict__ x, const double* __restrict__ b, double* __restrict__ r,
                                                  double* __restrict__ tileR2, double* __restrict__ tileB2) {
  __shared__ double sr[512], sb[512];
  for (uint32_t a = blockIdx.x; a < nT; a += gridDim.x) {
    const uint32_t l = threadIdx.x, c = a * 512u + splitIdx(l);
    const uint32_t in = info[c];
    double rv = 0.0, bv = 0.0;
    if (in & 0x8000u) {
      const uint32_t nns = (in >> 8) & 7u;
      double s = 0.0;
      for (int q = 0; q < 6; q++) if (in & (1u << q)) s += (double)x[nbIdx(nbs, a, l, q)];
      bv = b[c];
      rv = bv - ((double)nns * (double)x[c] - s);
    }
    r[c] = rv;
    sr[l] = rv * rv;
    sb[l] = bv * bv;
    __syncthreads();
    // fixed-order tree over the tile's 512 cells
    for (int w = 256; w > 0; w >>= 1) {
      if ((int)l < w) { sr[l] += sr[l + w]; sb[l] += sb[l + w]; }
      __syncthreads();
    }
    if (l == 0) { tileR2[a] = sr[0]; if (tileB2) tileB2[a] = sb[0]; }
    __syncthreads();
  }
}
// One refinement step in one pass: the corrected solution x + e (xo), its FP64 residual (as k_ps_resid<double> computes
// it from the corrected values: the same sums in the same order, the same per-tile tree), and the next inner
// right-hand side rhs32 = (float) r. The corrected solution goes to a second buffer, since neighbours still read x and
// e; the caller swaps the two and clears e.
__global__ void __launch_bounds__(512) k_ps_refine(uint32_t nT, const uint32_t* __restrict__ nbs, const uint16_t* __restrict__ info,
                                                   const double* __restrict__ x, const float* __restrict__ e, const double* __restrict__ b,
                                                   double* __restrict__ xo, float* __restrict__ rhs32, double* __restrict__ tileR2) {
  __shared__ double sr[512];
  for (uint32_t a = blockIdx.x; a < nT; a += gridDim.x) {
    const uint32_t l = threadIdx.x, c = a * 512u + splitIdx(l);
    const uint32_t in = info[c];
    const double xc = x[c] + (double)e[c];
    double rv = 0.0;
    if (in & 0x8000u) {
      const uint32_t nns = (in >> 8) & 7u;
      double s = 0.0;
      for (int q = 0; q < 6; q++)
        if (in & (1u << q)) {
          const uint32_t nb = nbIdx(nbs, a, l, q);
          s += x[nb] + (double)e[nb];
        }
      rv = b[c] - ((double)nns * xc - s);
    }
    xo[c] = xc;
    rhs32[c] = (float)rv;
    sr[l] = rv * rv;
    __syncthreads();
    for (int w = 256; w > 0; w >>= 1) {
      if ((int)l < w) sr[l] += sr[l + w];
      __syncthreads();
    }
    if (l == 0) tileR2[a] = sr[0];
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
// over all stored cells: the first inner right-hand side with a zero start; FP32 -> FP64 copy
__global__ void k_ps_inner(size_t n, const double* __restrict__ r, float* __restrict__ rhs32, float* __restrict__ e) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    rhs32[i] = (float)r[i];
    e[i] = 0.0f;
  }
}
__global__ void k_ps_copy(size_t n, const float* __restrict__ p32, double* __restrict__ x) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) x[i] = (double)p32[i];
}

thread_local char g_serr[256] = "";

}  // namespace

struct st_poisson {
  int device = 0;
  cudaStream_t stream = nullptr;
  int sms = 148;
  PGeo G{};
  uint32_t open = 0, nT = 0, capT = 0;
  std::vector<uint32_t> tiles;   // host copy: tile of each slot
  uint32_t* nbs = nullptr;
  uint16_t* info = nullptr;
  float *p32 = nullptr, *rhs32 = nullptr;
  double *x64 = nullptr, *b64 = nullptr, *r64 = nullptr, *tileR2 = nullptr, *tileB2 = nullptr, *norms = nullptr;
  double* x64b = nullptr;   // the refinement's second solution buffer
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  size_t cells() const { return (size_t)nT * 512; }
};

#define SK(call)                                                                            \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) {                                                                \
      snprintf(g_serr, sizeof(g_serr), "%s: %s", #call, cudaGetErrorString(e_)); st::set_error_text(g_serr);            \
      return e_ == cudaErrorMemoryAllocation ? ST_OOM : ST_DEVICE_ERROR;                    \
    }                                                                                       \
  } while (0)

static void poisson_free(st_poisson* s) {
  void* ptrs[] = {s->nbs, s->info, s->p32, s->rhs32, s->x64, s->x64b, s->b64, s->r64, s->tileR2, s->tileB2};
  for (void* p : ptrs) if (p) cudaFree(p);
  s->nbs = nullptr; s->info = nullptr; s->p32 = s->rhs32 = nullptr; s->x64 = s->x64b = s->b64 = s->r64 = s->tileR2 = s->tileB2 = nullptr;
  s->capT = 0;
}

extern "C" {

void st_poisson_destroy(st_poisson* s) {
  if (!s) return;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  poisson_free(s);
  if (s->norms) cudaFree(s->norms);
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
  cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc((void**)&s->norms, 4 * sizeof(double));
  if (e == cudaSuccess) e = cudaEventCreate(&s->e0);
  if (e == cudaSuccess) e = cudaEventCreate(&s->e1);
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
  auto ty = [&](long i, long j, long k) -> int {   // ctypeOf (src/flip/wgsl-core.js:104-112)
    if (i < 0) return (s->open & 1u) ? 0 : 2;
    if (i >= (long)G.nx) return (s->open & 2u) ? 0 : 2;
    if (j < 0) return (s->open & 4u) ? 0 : 2;
    if (j >= (long)G.ny) return (s->open & 8u) ? 0 : 2;
    if (k < 0) return (s->open & 16u) ? 0 : 2;
    if (k >= (long)G.nz) return (s->open & 32u) ? 0 : 2;
    return type[(size_t)i + G.nx * ((size_t)j + (size_t)G.ny * k)];
  };
  // the tiles holding fluid, ascending, and each one's slot
  std::vector<uint32_t> slot(T, 0xffffffffu);
  for (long k = 0; k < (long)G.nz; k++)
    for (long j = 0; j < (long)G.ny; j++)
      for (long i = 0; i < (long)G.nx; i++)
        if (type[(size_t)i + G.nx * ((size_t)j + (size_t)G.ny * k)] == 1)
          slot[(size_t)(i >> 3) + G.tx * ((size_t)(j >> 3) + (size_t)G.ty * (k >> 3))] = 0;
  s->tiles.clear();
  for (size_t t = 0; t < T; t++) if (slot[t] == 0) { slot[t] = (uint32_t)s->tiles.size(); s->tiles.push_back((uint32_t)t); }
  const uint32_t nT = (uint32_t)s->tiles.size();
  const size_t n = (size_t)nT * 512;
  std::vector<uint16_t> info(n, 0);
  std::vector<double> b(n, 0.0);
  std::vector<uint32_t> nbs((size_t)nT * 6);
  for (uint32_t a = 0; a < nT; a++) {
    const uint32_t t = s->tiles[a], tt = t / G.tx, ti = t % G.tx, tj = tt % G.ty, tk = tt / G.ty;
    const long nt[6] = {ti > 0 ? (long)t - 1 : -1, ti + 1 < G.tx ? (long)t + 1 : -1, tj > 0 ? (long)(t - G.tx) : -1,
                        tj + 1 < G.ty ? (long)(t + G.tx) : -1, tk > 0 ? (long)(t - G.tx * G.ty) : -1,
                        tk + 1 < G.tz ? (long)(t + G.tx * G.ty) : -1};
    for (int d = 0; d < 6; d++) nbs[(size_t)a * 6 + d] = (nt[d] >= 0 && slot[nt[d]] != 0xffffffffu) ? slot[nt[d]] : a;
    for (uint32_t l = 0; l < 512; l++) {
      const long i = (long)ti * 8 + (l & 7), j = (long)tj * 8 + ((l >> 3) & 7), k = (long)tk * 8 + (l >> 6);
      if (i >= (long)G.nx || j >= (long)G.ny || k >= (long)G.nz) continue;
      const size_t o = (size_t)i + G.nx * ((size_t)j + (size_t)G.ny * k);
      if (type[o] != 1) continue;
      const long q[6][3] = {{i - 1, j, k}, {i + 1, j, k}, {i, j - 1, k}, {i, j + 1, k}, {i, j, k - 1}, {i, j, k + 1}};
      uint32_t mask = 0, nns = 0;
      for (int d = 0; d < 6; d++) {
        const int tq = ty(q[d][0], q[d][1], q[d][2]);
        if (tq != 2) nns++;
        if (tq == 1) mask |= 1u << d;
      }
      const size_t c = (size_t)a * 512 + splitIdx(l);
      info[c] = (uint16_t)(0x8000u | (nns << 8) | mask);
      b[c] = rhs[o];
    }
  }
  if (nT > s->capT) {
    SK(cudaStreamSynchronize(s->stream));
    poisson_free(s);
    const size_t m = (size_t)std::max(nT, 1u) * 512;
    SK(cudaMalloc((void**)&s->nbs, (size_t)std::max(nT, 1u) * 6 * 4));
    SK(cudaMalloc((void**)&s->info, m * 2));
    SK(cudaMalloc((void**)&s->p32, m * 4));
    SK(cudaMalloc((void**)&s->rhs32, m * 4));
    SK(cudaMalloc((void**)&s->x64, m * 8));
    SK(cudaMalloc((void**)&s->x64b, m * 8));
    SK(cudaMalloc((void**)&s->b64, m * 8));
    SK(cudaMalloc((void**)&s->r64, m * 8));
    SK(cudaMalloc((void**)&s->tileR2, (size_t)std::max(nT, 1u) * 8));
    SK(cudaMalloc((void**)&s->tileB2, (size_t)std::max(nT, 1u) * 8));
    s->capT = std::max(nT, 1u);
  }
  s->nT = nT;
  cudaStream_t q = s->stream;
  if (nT) {
    SK(cudaMemcpyAsync(s->info, info.data(), n * 2, cudaMemcpyHostToDevice, q));
    SK(cudaMemcpyAsync(s->b64, b.data(), n * 8, cudaMemcpyHostToDevice, q));
    SK(cudaMemcpyAsync(s->nbs, nbs.data(), (size_t)nT * 6 * 4, cudaMemcpyHostToDevice, q));
    SK(cudaMemsetAsync(s->p32, 0, n * 4, q));
    SK(cudaMemsetAsync(s->x64, 0, n * 8, q));
  }
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

static void sweeps32(st_poisson* s, int grid, float om, int iters) {
  for (int k = 0; k < iters; k++) {
    k_ps_sor<float><<<grid, 256, 0, s->stream>>>(s->nT, s->nbs, s->info, s->p32, s->rhs32, om, 0u);
    k_ps_sor<float><<<grid, 256, 0, s->stream>>>(s->nT, s->nbs, s->info, s->p32, s->rhs32, om, 1u);
  }
}

// Solve from zero. mode 0: FP32 SOR (the residual is measured in FP64 every check_every iterations);
// 1: FP32 SOR inside FP64 refinement (inner_sweeps iterations per refinement); 2: FP64 SOR.
st_status st_poisson_solve(st_poisson* s, const st_poisson_opts* o, st_poisson_result* res) {
  if (!s || !o || !res || o->size != sizeof(st_poisson_opts)) return ST_BAD_ARG;
  SK(cudaSetDevice(s->device));
  memset(res, 0, sizeof(*res));
  if (!s->nT) { res->converged = 1; return ST_OK; }
  cudaStream_t q = s->stream;
  const size_t n = s->cells();
  const int grid = std::max(1, std::min<int>(s->sms * 8, (int)s->nT)), grid4 = std::max(1, std::min<int>(s->sms * 4, (int)s->nT));
  const int gridE = s->sms * 8;
  const int check = std::max(1, o->check_every), maxIt = std::max(1, o->max_sweeps);
  const float om = o->omega;
  SK(cudaMemsetAsync(s->p32, 0, n * 4, q));
  SK(cudaMemsetAsync(s->x64, 0, n * 8, q));
  // ||b|| once, from the residual of x = 0
  k_ps_resid<double><<<grid4, 512, 0, q>>>(s->nT, s->nbs, s->info, s->x64, s->b64, s->r64, s->tileR2, s->tileB2);
  double r2 = 0, b2 = 0;
  st_status st = norms(s, true, &r2, &b2);
  if (st != ST_OK) return st;
  const double bn = std::sqrt(b2);
  if (bn == 0.0) { res->converged = 1; return ST_OK; }
  SK(cudaEventRecord(s->e0, q));
  int it = 0, ref = 0;
  double rel = 1.0;
  // iterations before the next residual check: fixed blocks, or (ST_SCHEDULE_PREDICT) the count the last block's
  // reduction per iteration says reaches the tolerance, with 2% and one iteration to spare, between 8 and the block
  double lastRel = 1.0;
  int lastK = 0;
  auto nextBlock = [&](int block) {
    if (o->schedule != ST_SCHEDULE_PREDICT || lastK == 0 || !(rel < lastRel) || !(rel > 0.0)) return block;
    const double rho = std::pow(rel / lastRel, 1.0 / lastK);
    if (!(rho > 0.0 && rho < 1.0)) return block;
    const double need = std::log(o->tol / rel) / std::log(rho);
    return std::max(std::min(8, block), std::min(block, (int)std::ceil(need * 1.02) + 1));
  };
  auto checked = [&](double before, int k) { lastRel = before; lastK = k; };
  if (o->mode == 0) {
    k_ps_inner<<<gridE, 256, 0, q>>>(n, s->b64, s->rhs32, s->p32);
    while (it < maxIt) {
      const int k = std::min(nextBlock(check), maxIt - it);
      sweeps32(s, grid, om, k);
      it += k;
      k_ps_resid<float><<<grid4, 512, 0, q>>>(s->nT, s->nbs, s->info, s->p32, s->b64, s->r64, s->tileR2, nullptr);
      st = norms(s, false, &r2, nullptr);
      if (st != ST_OK) return st;
      checked(rel, k);
      rel = std::sqrt(r2) / bn;
      if (rel <= o->tol) break;
    }
    k_ps_copy<<<gridE, 256, 0, q>>>(n, s->p32, s->x64);
  } else if (o->mode == 1) {
    const int inner = std::max(1, o->inner_sweeps);
    k_ps_inner<<<gridE, 256, 0, q>>>(n, s->b64, s->rhs32, s->p32);   // x = 0: the first correction solves A e = b
    while (it < maxIt) {
      const int k = std::min(nextBlock(inner), maxIt - it);
      sweeps32(s, grid, om, k);
      it += k;
      k_ps_refine<<<grid4, 512, 0, q>>>(s->nT, s->nbs, s->info, s->x64, s->p32, s->b64, s->x64b, s->rhs32, s->tileR2);
      std::swap(s->x64, s->x64b);
      SK(cudaMemsetAsync(s->p32, 0, n * 4, q));
      ref++;
      st = norms(s, false, &r2, nullptr);
      if (st != ST_OK) return st;
      checked(rel, k);
      rel = std::sqrt(r2) / bn;
      if (rel <= o->tol) break;
    }
  } else if (o->mode == 2) {
    while (it < maxIt) {
      const int blk = nextBlock(check);
      int k = 0;
      for (; k < blk && it < maxIt; k++, it++) {
        k_ps_sor<double><<<grid, 256, 0, q>>>(s->nT, s->nbs, s->info, s->x64, s->b64, (double)om, 0u);
        k_ps_sor<double><<<grid, 256, 0, q>>>(s->nT, s->nbs, s->info, s->x64, s->b64, (double)om, 1u);
      }
      k_ps_resid<double><<<grid4, 512, 0, q>>>(s->nT, s->nbs, s->info, s->x64, s->b64, s->r64, s->tileR2, nullptr);
      st = norms(s, false, &r2, nullptr);
      if (st != ST_OK) return st;
      checked(rel, k);
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
  const size_t n = s->cells();
  const int grid = std::max(1, std::min<int>(s->sms * 8, (int)s->nT)), gridE = s->sms * 8;
  k_ps_inner<<<gridE, 256, 0, q>>>(n, s->b64, s->rhs32, s->p32);
  SK(cudaEventRecord(s->e0, q));
  sweeps32(s, grid, omega, iters);
  SK(cudaEventRecord(s->e1, q));
  k_ps_copy<<<gridE, 256, 0, q>>>(n, s->p32, s->x64);
  SK(cudaStreamSynchronize(q));
  SK(cudaGetLastError());
  if (ms) SK(cudaEventElapsedTime(ms, s->e0, s->e1));
  return ST_OK;
}

// the solution (FP64, dense, x fastest; 0 outside the tiles holding fluid)
st_status st_poisson_read(st_poisson* s, double* p) {
  if (!s || !p) return ST_BAD_ARG;
  SK(cudaSetDevice(s->device));
  const PGeo& G = s->G;
  memset(p, 0, sizeof(double) * (size_t)G.nx * G.ny * G.nz);
  if (!s->nT) return ST_OK;
  std::vector<double> x(s->cells());
  SK(cudaMemcpyAsync(x.data(), s->x64, s->cells() * 8, cudaMemcpyDeviceToHost, s->stream));
  SK(cudaStreamSynchronize(s->stream));
  for (uint32_t a = 0; a < s->nT; a++) {
    const uint32_t t = s->tiles[a], tt = t / G.tx, ti = t % G.tx, tj = tt % G.ty, tk = tt / G.ty;
    for (uint32_t l = 0; l < 512; l++) {
      const size_t i = (size_t)ti * 8 + (l & 7), j = (size_t)tj * 8 + ((l >> 3) & 7), k = (size_t)tk * 8 + (l >> 6);
      if (i >= G.nx || j >= G.ny || k >= G.nz) continue;
      p[i + G.nx * (j + (size_t)G.ny * k)] = x[(size_t)a * 512 + splitIdx(l)];
    }
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
