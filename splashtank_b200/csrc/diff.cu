// diff.cu - a differentiable FLIP rollout with its hand-written adjoint (st_diff_*).
//
// The step follows the reference's FLIP step (src/flip/wgsl-solver.js: p2g :17-40, normFaces :75-105, divergence
// :107-123, relax/project :124-180, g2p/collideP :181-275) on a dense n^3 MAC grid over the unit box, with the parts that
// have a derivative: P2G as float sums (mass-weighted face velocity), gravity, collider and wall face velocities, the
// pressure projection (the Poisson system of the step, solved by Jacobi-preconditioned conjugate gradients), FLIP/PIC
// G2P, advection, the push-out of a box collider (analytic, or its distance grid sampled as sdfEval does) and the wall
// clamp. Its discrete decisions (cell types,
// which faces carry mass, which particles touch the collider or a wall, which piece of the box's distance field each
// particle is on) are recorded by a forward pass and then held
// fixed: the adjoint differentiates the step with those decisions as constants, and a frozen forward pass evaluates
// exactly that function, so central differences check the adjoint.
//
// Parameters (27): the collider's centre at 8 keyframes (xyz, linear in time over the rollout) and the initial fluid
// velocity. Loss: sum over cells of (splatted particle density - target)^2. The reverse pass restores a checkpoint of
// the particles every ckpt_every steps, recomputes that segment forward keeping its tape, and runs the segment
// backwards. The adjoint pressure solve reuses the same symmetric operator. Everything is templated on the precision:
// FP32 for speed, FP64 for the reference gradient and the finite differences.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/splashtank_cuda.h"
#include "common.cuh"

namespace {

thread_local char g_derr[256] = "";
#define DK(call)                                                                                          \
  do {                                                                                                    \
    cudaError_t e_ = (call);                                                                              \
    if (e_ != cudaSuccess) {                                                                              \
      snprintf(g_derr, sizeof(g_derr), "%s: %s", #call, cudaGetErrorString(e_));                          \
      st::set_error_text(g_derr);                                                                         \
      return e_ == cudaErrorMemoryAllocation ? ST_OOM : ST_DEVICE_ERROR;                                  \
    }                                                                                                     \
  } while (0)

// ---- geometry ----
struct DGeo {
  int n;
  double h, ih;
  __host__ __device__ size_t nf(int a) const { return (size_t)(n + 1) * n * n; (void)a; }
  __host__ __device__ size_t cells() const { return (size_t)n * n * n; }
  // face (i, j, k) of axis a: the face on the low side of cell (i, j, k) along a; i ranges to n along a
  __host__ __device__ size_t face(int a, int i, int j, int k) const {
    if (a == 0) return (size_t)i + (size_t)(n + 1) * ((size_t)j + (size_t)n * k);
    if (a == 1) return (size_t)i + (size_t)n * ((size_t)j + (size_t)(n + 1) * k);
    return (size_t)i + (size_t)n * ((size_t)j + (size_t)n * k);
  }
  __host__ __device__ size_t cell(int i, int j, int k) const { return (size_t)i + (size_t)n * ((size_t)j + (size_t)n * k); }
};
enum : uint8_t { T_AIR = 0, T_FLUID = 1, T_SOLID = 2 };

// trilinear stencil of axis-a faces (a < 3) or cell centres (a == 3) at x: 8 indices, weights and d(weight)/dx
template <class T>
__device__ __forceinline__ void stencil(const DGeo& G, int a, const T* x, size_t* idx, T* w, T (*dw)[3]) {
  T g[3];
  int hi[3];
  for (int d = 0; d < 3; d++) {
    const bool shift = (a == 3) || d != a;
    g[d] = x[d] * (T)G.ih - (shift ? (T)0.5 : (T)0);
    hi[d] = (a < 3 && d == a) ? G.n : G.n - 1;
  }
  int i0[3];
  T fr[3];
  for (int d = 0; d < 3; d++) {
    const T f = floor(g[d]);
    i0[d] = (int)f;
    fr[d] = g[d] - f;
  }
  for (int c = 0; c < 8; c++) {
    int ii[3];
    T wd[3], dd[3];
    for (int d = 0; d < 3; d++) {
      const int o = (c >> d) & 1;
      ii[d] = min(max(i0[d] + o, 0), hi[d]);
      wd[d] = o ? fr[d] : (T)1 - fr[d];
      dd[d] = (o ? (T)1 : (T)-1) * (T)G.ih;
    }
    idx[c] = a < 3 ? G.face(a, ii[0], ii[1], ii[2]) : G.cell(ii[0], ii[1], ii[2]);
    w[c] = wd[0] * wd[1] * wd[2];
    dw[c][0] = dd[0] * wd[1] * wd[2];
    dw[c][1] = wd[0] * dd[1] * wd[2];
    dw[c][2] = wd[0] * wd[1] * dd[2];
  }
}

// analytic box signed distance at q = x - centre, half extents hb: phi, unit gradient n, Hessian H (3x3, row major).
// Its piece of the box's distance field is a discrete choice like the others: outside, which coordinates lie beyond
// the box (bits 0-2 of the regime); inside, which face is nearest (bits 3-4, with bits 0-2 clear). record != 0 picks
// it from q and returns it in *regime; otherwise the recorded piece is evaluated (extended past its own region).
template <class T>
__device__ __forceinline__ void boxSdf(const T* q, const T* hb, uint8_t* regime, int record, T& phi, T* n, T* H) {
  T d[3], s[3];
  for (int k = 0; k < 3; k++) { s[k] = q[k] < (T)0 ? (T)-1 : (T)1; d[k] = fabs(q[k]) - hb[k]; }
  for (int k = 0; k < 9; k++) H[k] = (T)0;
  if (record) {
    uint8_t out = 0;
    for (int k = 0; k < 3; k++) if (d[k] > (T)0) out |= (uint8_t)(1u << k);
    int m = 0;
    for (int k = 1; k < 3; k++) if (d[k] > d[m]) m = k;
    *regime = out ? out : (uint8_t)(m << 3);
  }
  const uint8_t out = *regime & 7u;
  if (out) {   // outside: distance to the nearest point of the box
    T o[3], l2 = (T)0;
    for (int k = 0; k < 3; k++) { o[k] = (out >> k) & 1u ? d[k] : (T)0; l2 += o[k] * o[k]; }
    const T l = sqrt(l2);
    phi = l;
    for (int k = 0; k < 3; k++) n[k] = s[k] * o[k] / l;
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++) {
        if (!((out >> r) & 1u) || !((out >> c) & 1u)) continue;
        const T e = (r == c ? (T)1 : (T)0) - (o[r] / l) * (o[c] / l);
        H[r * 3 + c] = s[r] * s[c] * e / l;
      }
  } else {     // inside: the nearest face
    const int m = (*regime >> 3) & 3u;
    phi = d[m];
    for (int k = 0; k < 3; k++) n[k] = k == m ? s[k] : (T)0;
  }
}

// The collider's distance grid (collider_grid = 1): nodes `cell` apart from `origin` (relative to the collider centre),
// dims nodes per axis, the box's exact distance at each node.
struct DGrid {
  int mode;            // 0 analytic box, 1 its distance grid
  int dims[3];
  double origin[3], cell;
  const float* data;
};
// The collider at q = x - centre: distance phi, unit normal n, d phi / dq (dphi) and d n / dq (J, row major). The
// analytic box gives dphi = n and J = its Hessian. The grid follows sdfEval (src/gpu.js:6-33): the trilinear distance at
// the clamped grid coordinate plus the distance outside the grid, the normal the normalised trilinear gradient (in grid
// units, raw = d phi / d f), so dphi = raw / cell and J = (I - n n^T) H_f / (|raw| cell) with H_f the trilinear Hessian
// (zero diagonal). Outside the grid the normal points out of it and J is left 0: the grid's margin exceeds q0, so no
// contact happens there.
template <class T>
__device__ __forceinline__ void colEval(const DGrid& Gd, const T* q, const T* hb, uint8_t* regime, int record, T& phi, T* n, T* dphi, T* J) {
  if (Gd.mode == 0) {
    boxSdf<T>(q, hb, regime, record, phi, n, J);
    for (int k = 0; k < 3; k++) dphi[k] = n[k];
    return;
  }
  if (record) *regime = 0;
  T g[3], gc[3], f[3];
  int fl[3];
  T out2 = (T)0;
  for (int d = 0; d < 3; d++) {
    g[d] = (q[d] - (T)Gd.origin[d]) / (T)Gd.cell;
    gc[d] = fmin(fmax(g[d], (T)0), (T)Gd.dims[d] - (T)1.0001);
    const T fv = floor(gc[d]);
    fl[d] = (int)fv;
    f[d] = gc[d] - fv;
    out2 += (g[d] - gc[d]) * (g[d] - gc[d]);
  }
  const int nx = Gd.dims[0], nxy = Gd.dims[0] * Gd.dims[1];
  const size_t b0 = (size_t)fl[0] + (size_t)nx * fl[1] + (size_t)nxy * fl[2];
  const T v000 = (T)Gd.data[b0], v100 = (T)Gd.data[b0 + 1], v010 = (T)Gd.data[b0 + nx], v110 = (T)Gd.data[b0 + nx + 1];
  const T v001 = (T)Gd.data[b0 + nxy], v101 = (T)Gd.data[b0 + nxy + 1], v011 = (T)Gd.data[b0 + nxy + nx], v111 = (T)Gd.data[b0 + nxy + nx + 1];
  auto mix = [](T a, T b, T t) { return a * ((T)1 - t) + b * t; };
  const T c00 = mix(v000, v100, f[0]), c10 = mix(v010, v110, f[0]), c01 = mix(v001, v101, f[0]), c11 = mix(v011, v111, f[0]);
  const T c0 = mix(c00, c10, f[1]), c1 = mix(c01, c11, f[1]);
  phi = mix(c0, c1, f[2]);
  for (int k = 0; k < 9; k++) J[k] = (T)0;
  if (out2 > (T)0) {
    const T l = sqrt(out2);
    phi += l * (T)Gd.cell;
    for (int d = 0; d < 3; d++) { n[d] = (g[d] - gc[d]) / l; dphi[d] = n[d]; }
    return;
  }
  const T ax0 = v100 - v000, ax1 = v110 - v010, ax2 = v101 - v001, ax3 = v111 - v011;
  const T raw[3] = {mix(mix(ax0, ax1, f[1]), mix(ax2, ax3, f[1]), f[2]), mix(c10 - c00, c11 - c01, f[2]), c1 - c0};
  const T l = sqrt(raw[0] * raw[0] + raw[1] * raw[1] + raw[2] * raw[2]);
  const T il = (T)1 / fmax(l, (T)1e-9);
  for (int d = 0; d < 3; d++) { n[d] = raw[d] * il; dphi[d] = raw[d] / (T)Gd.cell; }
  // trilinear Hessian in grid units (symmetric, zero diagonal)
  const T hxy = mix(ax1 - ax0, ax3 - ax2, f[2]);
  const T hxz = mix(ax2, ax3, f[1]) - mix(ax0, ax1, f[1]);
  const T hyz = (c11 - c01) - (c10 - c00);
  const T Hf[9] = {(T)0, hxy, hxz, hxy, (T)0, hyz, hxz, hyz, (T)0};
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) {
      T acc = (T)0;
      for (int m = 0; m < 3; m++) acc += (((r == m) ? (T)1 : (T)0) - n[r] * n[m]) * Hf[m * 3 + c];
      J[r * 3 + c] = acc * il / (T)Gd.cell;
    }
}

// ---- forward kernels ----
template <class T>
__global__ void k_d_p2g(DGeo G, size_t np, const T* __restrict__ x, const T* __restrict__ v, T* mom, T* mass, int* count) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < np; p += (size_t)gridDim.x * blockDim.x) {
    const T* xp = x + 3 * p;
    for (int a = 0; a < 3; a++) {
      size_t idx[8];
      T w[8], dw[8][3];
      stencil<T>(G, a, xp, idx, w, dw);
      const T va = v[3 * p + a];
      for (int c = 0; c < 8; c++) {
        atomicAdd(&mom[a * G.nf(a) + idx[c]], w[c] * va);
        atomicAdd(&mass[a * G.nf(a) + idx[c]], w[c]);
      }
    }
    if (count) {
      int ci[3];
      for (int d = 0; d < 3; d++) ci[d] = min(max((int)floor(xp[d] * (T)G.ih), 0), G.n - 1);
      atomicAdd(&count[G.cell(ci[0], ci[1], ci[2])], 1);
    }
  }
}
// cell types: outside the box nothing (walls are handled by the neighbour logic); collider cells solid (inside the
// analytic box, or a distance below q0 at the centre for the grid, as colAt decides); cells with a particle fluid
template <class T>
__global__ void k_d_types(DGeo G, const int* __restrict__ count, const T* c, const T* hb, DGrid Gd, T q0, uint8_t* types) {
  const size_t nc = G.cells();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nc; i += (size_t)gridDim.x * blockDim.x) {
    const int ci = (int)(i % G.n), cj = (int)((i / G.n) % G.n), ck = (int)(i / ((size_t)G.n * G.n));
    const T q[3] = {((T)ci + (T)0.5) * (T)G.h - c[0], ((T)cj + (T)0.5) * (T)G.h - c[1], ((T)ck + (T)0.5) * (T)G.h - c[2]};
    bool inside = true;
    if (Gd.mode == 0) {
      for (int k = 0; k < 3; k++) inside = inside && fabs(q[k]) < hb[k];
    } else {
      T phi, n[3], dphi[3], J[9];
      uint8_t rg = 0;
      colEval<T>(Gd, q, hb, &rg, 1, phi, n, dphi, J);
      inside = phi < q0;   // colAt's test (src/flip/wgsl-core.js:127-131), as the step classifies collider cells
    }
    types[i] = inside ? T_SOLID : (count[i] > 0 ? T_FLUID : T_AIR);
  }
}
// the two cells either side of face f of axis a; -1 when outside the box (a wall)
__device__ __forceinline__ void faceCells(const DGeo& G, int a, size_t f, long& lo, long& hi) {
  int i, j, k;
  if (a == 0) { i = (int)(f % (G.n + 1)); j = (int)((f / (G.n + 1)) % G.n); k = (int)(f / ((size_t)(G.n + 1) * G.n)); }
  else if (a == 1) { i = (int)(f % G.n); j = (int)((f / G.n) % (G.n + 1)); k = (int)(f / ((size_t)G.n * (G.n + 1))); }
  else { i = (int)(f % G.n); j = (int)((f / G.n) % G.n); k = (int)(f / ((size_t)G.n * G.n)); }
  int lo3[3] = {i, j, k}, hi3[3] = {i, j, k};
  lo3[a] -= 1;
  lo = lo3[a] < 0 ? -1 : (long)G.cell(lo3[0], lo3[1], lo3[2]);
  hi = hi3[a] >= G.n ? -1 : (long)G.cell(hi3[0], hi3[1], hi3[2]);
}
// face velocity: mass-weighted mean (recorded or frozen: which faces carry mass), gravity on y, collider velocity on
// faces touching a collider cell, 0 on wall faces; the old velocity u0 (the FLIP term's) is the mean, or the boundary's
// velocity on those faces (normFaces, src/flip/wgsl-solver.js:75-105)
template <class T>
__global__ void k_d_norm(DGeo G, const T* __restrict__ mom, const T* __restrict__ mass, uint8_t* mask, int record,
                         const uint8_t* __restrict__ types, const T* vc, T gdt, T* u0, T* u1) {
  const size_t nf = G.nf(0);
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < 3 * nf; t += (size_t)gridDim.x * blockDim.x) {
    const int a = (int)(t / nf);
    const size_t f = t % nf;
    if (record) mask[t] = mass[t] > (T)0 ? 1 : 0;
    const T u = (mask[t] && mass[t] > (T)0) ? mom[t] / mass[t] : (T)0;
    long lo, hi;
    faceCells(G, a, f, lo, hi);
    T r = u - (a == 1 ? gdt : (T)0), old = u;
    if (lo < 0 || hi < 0) r = old = (T)0;                                                   // a wall
    else if (types[lo] == T_SOLID || types[hi] == T_SOLID) r = old = vc[a];                // the collider's velocity
    u0[t] = old;   // the step's old face velocity (vo): on a boundary face the boundary's, as normFaces sets it
    u1[t] = r;
  }
}
// right-hand side of the pressure system on fluid cells: -(h / dt) * sum of face flux differences
template <class T>
__global__ void k_d_rhs(DGeo G, const uint8_t* __restrict__ types, const T* __restrict__ u1, T hdt, T* b) {
  const size_t nc = G.cells(), nf = G.nf(0);
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
    if (types[c] != T_FLUID) { b[c] = (T)0; continue; }
    const int i = (int)(c % G.n), j = (int)((c / G.n) % G.n), k = (int)(c / ((size_t)G.n * G.n));
    T d = (T)0;
    d += u1[0 * nf + G.face(0, i + 1, j, k)] - u1[0 * nf + G.face(0, i, j, k)];
    d += u1[1 * nf + G.face(1, i, j + 1, k)] - u1[1 * nf + G.face(1, i, j, k)];
    d += u1[2 * nf + G.face(2, i, j, k + 1)] - u1[2 * nf + G.face(2, i, j, k)];
    b[c] = -hdt * d;
  }
}
// y = A x on fluid cells (nns x_c - sum of fluid neighbours), and the Jacobi preconditioner 1 / nns
__device__ __forceinline__ int cellType(const DGeo& G, const uint8_t* types, int i, int j, int k) {
  if (i < 0 || j < 0 || k < 0 || i >= G.n || j >= G.n || k >= G.n) return T_SOLID;
  return types[G.cell(i, j, k)];
}
template <class T>
__global__ void k_d_apply(DGeo G, const uint8_t* __restrict__ types, const T* __restrict__ xv, T* y, T* dinv) {
  const size_t nc = G.cells();
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
    if (types[c] != T_FLUID) { y[c] = (T)0; if (dinv) dinv[c] = (T)0; continue; }
    const int i = (int)(c % G.n), j = (int)((c / G.n) % G.n), k = (int)(c / ((size_t)G.n * G.n));
    const int nb[6][3] = {{i - 1, j, k}, {i + 1, j, k}, {i, j - 1, k}, {i, j + 1, k}, {i, j, k - 1}, {i, j, k + 1}};
    int nns = 0;
    T s = (T)0;
    for (int q = 0; q < 6; q++) {
      const int t = cellType(G, types, nb[q][0], nb[q][1], nb[q][2]);
      if (t != T_SOLID) nns++;
      if (t == T_FLUID) s += xv[G.cell(nb[q][0], nb[q][1], nb[q][2])];
    }
    y[c] = (T)nns * xv[c] - s;
    if (dinv) dinv[c] = nns ? (T)1 / (T)nns : (T)0;
  }
}
// dot products in FP64 (block sums then one atomic per block)
template <class T>
__global__ void k_d_dot(size_t n, const T* __restrict__ a, const T* __restrict__ b, double* out) {
  __shared__ double s[256];
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) acc += (double)a[i] * (double)b[i];
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(out, s[0]);
}
template <class T>
__global__ void k_d_axpy(size_t n, T alpha, const T* __restrict__ xv, T* y) {   // y += alpha x
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) y[i] += alpha * xv[i];
}
template <class T>
__global__ void k_d_xpby(size_t n, const T* __restrict__ xv, T beta, T* y) {    // y = x + beta y
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) y[i] = xv[i] + beta * y[i];
}
template <class T>
__global__ void k_d_mul(size_t n, const T* __restrict__ a, const T* __restrict__ b, T* y) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) y[i] = a[i] * b[i];
}
// projection: faces with no solid side and a fluid side lose dt/h times the pressure difference (air p = 0)
template <class T>
__global__ void k_d_project(DGeo G, const uint8_t* __restrict__ types, const T* __restrict__ p, const T* __restrict__ u1, T dth, T* u2) {
  const size_t nf = G.nf(0);
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < 3 * nf; t += (size_t)gridDim.x * blockDim.x) {
    const int a = (int)(t / nf);
    long lo, hi;
    faceCells(G, a, t % nf, lo, hi);
    T r = u1[t];
    if (lo >= 0 && hi >= 0 && types[lo] != T_SOLID && types[hi] != T_SOLID && (types[lo] == T_FLUID || types[hi] == T_FLUID)) {
      const T ph = types[hi] == T_FLUID ? p[hi] : (T)0, pl = types[lo] == T_FLUID ? p[lo] : (T)0;
      r -= dth * (ph - pl);
    }
    u2[t] = r;
  }
}
// G2P + advection + collider push-out + wall clamp, then the step's velocity response (g2p after collideP,
// src/flip/wgsl-solver.js:259-265): the displacement dsp = x_out - x_a of the push-out and the clamp together, and when
// it is not negligible the velocity's component into it removed (v -= nrm min(v . nrm, 0), nrm = dsp / |dsp|).
// flags (recorded or frozen) per particle: bit 0 touches the collider, bit 1 the velocity response applies (moved and
// v . nrm < 0), bits 2-7 the position was clamped on (x lo, x hi, y lo, ...).
template <class T>
__global__ void k_d_g2p(DGeo G, size_t np, const T* __restrict__ x, const T* __restrict__ v, const T* __restrict__ u2,
                        const T* __restrict__ u0, T beta, T dt, const T* c, const T* hb, DGrid Gd, T q0, T lo, T hi, uint8_t* flags,
                        uint8_t* regimes, int record, T* xo, T* vo) {
  const size_t nf = G.nf(0);
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < np; p += (size_t)gridDim.x * blockDim.x) {
    const T* xp = x + 3 * p;
    T vn[3];
    for (int a = 0; a < 3; a++) {
      size_t idx[8];
      T w[8], dw[8][3];
      stencil<T>(G, a, xp, idx, w, dw);
      T s2 = (T)0, s0 = (T)0;
      for (int k = 0; k < 8; k++) { s2 += w[k] * u2[a * nf + idx[k]]; s0 += w[k] * u0[a * nf + idx[k]]; }
      vn[a] = s2 + beta * (v[3 * p + a] - s0);
    }
    T xa[3];
    for (int a = 0; a < 3; a++) xa[a] = xp[a] + vn[a] * dt;
    uint8_t fl = record ? 0 : flags[p];
    T q[3] = {xa[0] - c[0], xa[1] - c[1], xa[2] - c[2]}, phi, n[3], dphi[3], J[9];
    uint8_t rg = regimes[p];
    colEval<T>(Gd, q, hb, &rg, record, phi, n, dphi, J);
    if (record) regimes[p] = rg;
    if (record && phi < q0) fl |= 1;
    T xc[3] = {xa[0], xa[1], xa[2]}, dsp[3] = {(T)0, (T)0, (T)0};
    if (fl & 1)
      for (int a = 0; a < 3; a++) {
        xc[a] += n[a] * (q0 - phi);
        dsp[a] = n[a] * fabs(q0 - phi);   // = the push where it was recorded (phi < q0); a frozen pass that no longer
                                          // reaches q0 keeps the normal's side, so the response does not flip
      }
    for (int a = 0; a < 3; a++) {
      if (record) { if (xc[a] < lo) fl |= (uint8_t)(4u << (2 * a)); else if (xc[a] > hi) fl |= (uint8_t)(8u << (2 * a)); }
      const T before = xc[a];
      if (fl & (4u << (2 * a))) xc[a] = lo;
      else if (fl & (8u << (2 * a))) xc[a] = hi;
      dsp[a] += xc[a] - before;
    }
    const T d2 = dsp[0] * dsp[0] + dsp[1] * dsp[1] + dsp[2] * dsp[2];
    if (record && d2 > (T)1e-12) {
      const T il = (T)1 / sqrt(d2);
      const T vd = (vn[0] * dsp[0] + vn[1] * dsp[1] + vn[2] * dsp[2]) * il;
      if (vd < (T)0) fl |= 2;
    }
    if (fl & 2) {
      const T il = (T)1 / sqrt(d2);
      const T nr[3] = {dsp[0] * il, dsp[1] * il, dsp[2] * il};
      const T vd = vn[0] * nr[0] + vn[1] * nr[1] + vn[2] * nr[2];
      for (int a = 0; a < 3; a++) vn[a] -= nr[a] * vd;
    }
    for (int a = 0; a < 3; a++) {
      xo[3 * p + a] = xc[a];
      vo[3 * p + a] = vn[a];
    }
    if (record) flags[p] = fl;
  }
}
template <class T>
__global__ void k_d_splat(DGeo G, size_t np, const T* __restrict__ x, T* rho) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < np; p += (size_t)gridDim.x * blockDim.x) {
    size_t idx[8];
    T w[8], dw[8][3];
    stencil<T>(G, 3, x + 3 * p, idx, w, dw);
    for (int k = 0; k < 8; k++) atomicAdd(&rho[idx[k]], w[k]);
  }
}
template <class T>
__global__ void k_d_resid(size_t n, const T* __restrict__ rho, const float* __restrict__ tgt, T* g, double* loss) {
  __shared__ double s[256];
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const T d = rho[i] - (T)tgt[i];
    acc += (double)d * (double)d;
    if (g) g[i] = (T)2 * d;
  }
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, s[0]);
}
template <class T>
__global__ void k_d_fillv(size_t np, const T* v0, T* v) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < np; p += (size_t)gridDim.x * blockDim.x)
    for (int a = 0; a < 3; a++) v[3 * p + a] = v0[a];
}

// ---- adjoint kernels ----
// density loss -> particle positions
template <class T>
__global__ void k_d_splat_b(DGeo G, size_t np, const T* __restrict__ x, const T* __restrict__ grho, T* gx) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < np; p += (size_t)gridDim.x * blockDim.x) {
    size_t idx[8];
    T w[8], dw[8][3];
    stencil<T>(G, 3, x + 3 * p, idx, w, dw);
    T g[3] = {(T)0, (T)0, (T)0};
    for (int k = 0; k < 8; k++) for (int d = 0; d < 3; d++) g[d] += dw[k][d] * grho[idx[k]];
    for (int d = 0; d < 3; d++) gx[3 * p + d] = g[d];
  }
}
// back through wall clamp, collider response, advection and G2P. In: gx, gv of the step's outputs. Out: gx, gv of its
// inputs (in place), face adjoints of u2 and u0 (atomics), the collider centre's adjoint (atomics into gc[3]).
template <class T>
__global__ void k_d_g2p_b(DGeo G, size_t np, const T* __restrict__ x, const T* __restrict__ v, const T* __restrict__ u2,
                          const T* __restrict__ u0, T beta, T dt, const T* c, const T* hb, DGrid Gd, T q0, T lo, T hi,
                          const uint8_t* __restrict__ flags,
                          const uint8_t* __restrict__ regimes, T* gx, T* gv, T* gu2, T* gu0, double* gc) {
  const size_t nf = G.nf(0);
  T gcx = 0, gcy = 0, gcz = 0;
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < np; p += (size_t)gridDim.x * blockDim.x) {
    const T* xp = x + 3 * p;
    // recompute the forward values this particle needs
    size_t idx[3][8];
    T w[3][8], dw[3][8][3], vn[3];
    for (int a = 0; a < 3; a++) {
      stencil<T>(G, a, xp, idx[a], w[a], dw[a]);
      T s2 = (T)0, t0 = (T)0;
      for (int k = 0; k < 8; k++) { s2 += w[a][k] * u2[a * nf + idx[a][k]]; t0 += w[a][k] * u0[a * nf + idx[a][k]]; }
      vn[a] = s2 + beta * (v[3 * p + a] - t0);
    }
    T xa[3];
    for (int a = 0; a < 3; a++) xa[a] = xp[a] + vn[a] * dt;
    const uint8_t fl = flags[p];
    T q[3] = {xa[0] - c[0], xa[1] - c[1], xa[2] - c[2]}, phi, n[3], dphi[3], J[9];
    uint8_t rg = regimes[p];
    colEval<T>(Gd, q, hb, &rg, 0, phi, n, dphi, J);
    T gxo[3] = {gx[3 * p], gx[3 * p + 1], gx[3 * p + 2]}, gvo[3] = {gv[3 * p], gv[3 * p + 1], gv[3 * p + 2]};
    // the forward's output position again: push-out, then the clamp
    T xc[3] = {xa[0], xa[1], xa[2]};
    if (fl & 1)
      for (int a = 0; a < 3; a++) xc[a] += n[a] * (q0 - phi);
    for (int a = 0; a < 3; a++) {
      if (fl & (4u << (2 * a))) xc[a] = lo;
      else if (fl & (8u << (2 * a))) xc[a] = hi;
    }
    // velocity response: v_out = v' - nrm (v' . nrm), nrm = dsp / |dsp|, dsp = x_out - x_a
    T gvp[3] = {gvo[0], gvo[1], gvo[2]}, gxa[3] = {(T)0, (T)0, (T)0};
    if (fl & 2) {
      const T dsp[3] = {xc[0] - xa[0], xc[1] - xa[1], xc[2] - xa[2]};
      const T l = sqrt(dsp[0] * dsp[0] + dsp[1] * dsp[1] + dsp[2] * dsp[2]);
      const T nr[3] = {dsp[0] / l, dsp[1] / l, dsp[2] / l};
      const T vd = vn[0] * nr[0] + vn[1] * nr[1] + vn[2] * nr[2];
      const T ng = nr[0] * gvo[0] + nr[1] * gvo[1] + nr[2] * gvo[2];
      T gnr[3];
      for (int a = 0; a < 3; a++) {
        gvp[a] = gvo[a] - nr[a] * ng;
        gnr[a] = -(vd * gvo[a] + ng * vn[a]);
      }
      const T nd = nr[0] * gnr[0] + nr[1] * gnr[1] + nr[2] * gnr[2];
      for (int a = 0; a < 3; a++) {
        const T gd = (gnr[a] - nr[a] * nd) / l;   // through nrm = dsp / |dsp|
        gxo[a] += gd;                            // dsp = x_out - x_a
        gxa[a] -= gd;
      }
    }
    // wall clamp: a clamped coordinate is constant
    for (int a = 0; a < 3; a++) if (fl & (12u << (2 * a))) gxo[a] = (T)0;
    // collider: x_c = x_a + n (q0 - phi)
    for (int a = 0; a < 3; a++) gxa[a] += gxo[a];
    if (fl & 1) {
      T gn[3] = {gxo[0] * (q0 - phi), gxo[1] * (q0 - phi), gxo[2] * (q0 - phi)};
      T gphi = -(gxo[0] * n[0] + gxo[1] * n[1] + gxo[2] * n[2]);
      // phi and n are functions of q = x_a - c: d phi = dphi . dq, d n = J dq
      T gq[3];
      for (int r = 0; r < 3; r++) gq[r] = gphi * dphi[r] + J[r] * gn[0] + J[3 + r] * gn[1] + J[6 + r] * gn[2];
      for (int a = 0; a < 3; a++) gxa[a] += gq[a];
      gcx -= gq[0]; gcy -= gq[1]; gcz -= gq[2];
    }
    // advection: x_a = x + v' dt
    for (int a = 0; a < 3; a++) gvp[a] += gxa[a] * dt;
    T gxi[3] = {gxa[0], gxa[1], gxa[2]};
    // G2P: v'_a = U2_a(x) + beta (v_a - U0_a(x))
    for (int a = 0; a < 3; a++) {
      const T g = gvp[a];
      gv[3 * p + a] = beta * g;
      for (int k = 0; k < 8; k++) {
        atomicAdd(&gu2[a * nf + idx[a][k]], w[a][k] * g);
        atomicAdd(&gu0[a * nf + idx[a][k]], -beta * w[a][k] * g);
        const T uu = u2[a * nf + idx[a][k]] - beta * u0[a * nf + idx[a][k]];
        for (int d = 0; d < 3; d++) gxi[d] += dw[a][k][d] * uu * g;
      }
    }
    for (int a = 0; a < 3; a++) gx[3 * p + a] = gxi[a];
  }
  // one atomic per warp for the collider centre
  for (int o = 16; o > 0; o >>= 1) {
    gcx += __shfl_xor_sync(0xffffffffu, gcx, o);
    gcy += __shfl_xor_sync(0xffffffffu, gcy, o);
    gcz += __shfl_xor_sync(0xffffffffu, gcz, o);
  }
  if ((threadIdx.x & 31) == 0) { atomicAdd(&gc[0], (double)gcx); atomicAdd(&gc[1], (double)gcy); atomicAdd(&gc[2], (double)gcz); }
}
// projection backwards: gu1 = gu2; gp_c = dt/h * (sum of gu2 over active faces where c is the low cell - where it is
// the high cell), for fluid cells
template <class T>
__global__ void k_d_project_b(DGeo G, const uint8_t* __restrict__ types, const T* __restrict__ gu2, T dth, T* gp) {
  const size_t nc = G.cells(), nf = G.nf(0);
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
    if (types[c] != T_FLUID) { gp[c] = (T)0; continue; }
    const int i = (int)(c % G.n), j = (int)((c / G.n) % G.n), k = (int)(c / ((size_t)G.n * G.n));
    T s = (T)0;
    for (int a = 0; a < 3; a++) {
      int lo[3] = {i, j, k}, hi[3] = {i, j, k};
      hi[a] += 1;   // face on the high side of c: c is its low cell
      // low-side face (index i along a): c is its high cell
      const int tl = cellType(G, types, a == 0 ? i - 1 : i, a == 1 ? j - 1 : j, a == 2 ? k - 1 : k);
      const int th = cellType(G, types, a == 0 ? i + 1 : i, a == 1 ? j + 1 : j, a == 2 ? k + 1 : k);
      const bool inLo = (a == 0 ? i : (a == 1 ? j : k)) > 0, inHi = (a == 0 ? i : (a == 1 ? j : k)) + 1 < G.n;
      if (inLo && tl != T_SOLID) s -= gu2[a * nf + G.face(a, lo[0], lo[1], lo[2])];   // this cell is the face's high side
      if (inHi && th != T_SOLID) s += gu2[a * nf + G.face(a, hi[0], hi[1], hi[2])];   // low side
    }
    gp[c] = dth * s;
  }
}
// right-hand side backwards into u1, then the face velocity rule backwards into u0 and the collider velocity
template <class T>
__global__ void k_d_norm_b(DGeo G, const uint8_t* __restrict__ types, const T* __restrict__ gb, T hdt, const T* __restrict__ gu2,
                           const uint8_t* __restrict__ mask, const T* __restrict__ u0, const T* __restrict__ mass, T* gu0,
                           T* gmom, T* gmass, double* gvc) {
  const size_t nf = G.nf(0);
  T gva = 0, gvb = 0, gvcz = 0;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < 3 * nf; t += (size_t)gridDim.x * blockDim.x) {
    const int a = (int)(t / nf);
    long lo, hi;
    faceCells(G, a, t % nf, lo, hi);
    T g = gu2[t];   // projection passes u1 through
    // b_c = -(h/dt) (u1[c's high face] - u1[c's low face]) for fluid c
    if (lo >= 0 && types[lo] == T_FLUID) g += -hdt * gb[lo];
    if (hi >= 0 && types[hi] == T_FLUID) g -= -hdt * gb[hi];
    // the G2P's FLIP term reads u0 directly: on a boundary face u0 is the boundary's velocity like u1
    T g0 = (T)0;
    if (lo < 0 || hi < 0) g0 = (T)0;
    else if (types[lo] == T_SOLID || types[hi] == T_SOLID) {
      const T gb2 = g + gu0[t];
      if (a == 0) gva += gb2; else if (a == 1) gvb += gb2; else gvcz += gb2;
    } else g0 = g + gu0[t];
    const bool m = mask[t] && mass[t] > (T)0;
    gmom[t] = m ? g0 / mass[t] : (T)0;
    gmass[t] = m ? -g0 * u0[t] / mass[t] : (T)0;
  }
  for (int o = 16; o > 0; o >>= 1) {
    gva += __shfl_xor_sync(0xffffffffu, gva, o);
    gvb += __shfl_xor_sync(0xffffffffu, gvb, o);
    gvcz += __shfl_xor_sync(0xffffffffu, gvcz, o);
  }
  if ((threadIdx.x & 31) == 0) { atomicAdd(&gvc[0], (double)gva); atomicAdd(&gvc[1], (double)gvb); atomicAdd(&gvc[2], (double)gvcz); }
}
// P2G backwards: gv_a += sum w gmom; gx += sum dw (v_a gmom + gmass)
template <class T>
__global__ void k_d_p2g_b(DGeo G, size_t np, const T* __restrict__ x, const T* __restrict__ v, const T* __restrict__ gmom,
                          const T* __restrict__ gmass, T* gx, T* gv) {
  const size_t nf = G.nf(0);
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < np; p += (size_t)gridDim.x * blockDim.x) {
    const T* xp = x + 3 * p;
    T gxi[3] = {gx[3 * p], gx[3 * p + 1], gx[3 * p + 2]};
    for (int a = 0; a < 3; a++) {
      size_t idx[8];
      T w[8], dw[8][3];
      stencil<T>(G, a, xp, idx, w, dw);
      const T va = v[3 * p + a];
      T g = (T)0;
      for (int k = 0; k < 8; k++) {
        const T gm = gmom[a * nf + idx[k]], gw = gmass[a * nf + idx[k]];
        g += w[k] * gm;
        for (int d = 0; d < 3; d++) gxi[d] += dw[k][d] * (va * gm + gw);
      }
      gv[3 * p + a] += g;
    }
    for (int d = 0; d < 3; d++) gx[3 * p + d] = gxi[d];
  }
}
template <class T>
__global__ void k_d_sumv(size_t np, const T* __restrict__ gv, double* out) {
  double s[3] = {0, 0, 0};
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < np; p += (size_t)gridDim.x * blockDim.x)
    for (int a = 0; a < 3; a++) s[a] += (double)gv[3 * p + a];
  for (int a = 0; a < 3; a++) {
    double x = s[a];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&out[a], x);
  }
}

}  // namespace

// ---- the rollout ----
struct st_diff {
  st_diff_desc d{};
  DGeo G{};
  cudaStream_t stream = nullptr;
  int grid = 1184;
  size_t np = 0;
  bool fp64 = false;
  bool recorded = false;
  std::vector<double> params;   // of the recorded forward
  void* mem = nullptr;          // all device memory in one block
  size_t memBytes = 0;
  // device pointers (element type T = float or double, cast at use)
  void *x0 = nullptr, *x = nullptr, *v = nullptr, *xn = nullptr, *vn = nullptr;
  void *mom = nullptr, *mass = nullptr, *u0 = nullptr, *u1 = nullptr, *u2 = nullptr;
  void *b = nullptr, *p = nullptr, *r = nullptr, *z = nullptr, *pd = nullptr, *q = nullptr, *dinv = nullptr, *rho = nullptr;
  void *gx = nullptr, *gv = nullptr, *gu2 = nullptr, *gu0 = nullptr, *gmom = nullptr, *gmass = nullptr, *gp = nullptr, *gb = nullptr;
  void *cbuf = nullptr;         // per step: collider centre (3), collider velocity (3), half extents (3)
  float* tgt = nullptr;
  int* count = nullptr;
  double* red = nullptr;        // reduction scratch of the solver and the loss (8 doubles)
  double* cred = nullptr;       // the collider centre and velocity adjoints of one step (8 doubles)
  uint8_t *types = nullptr, *mask = nullptr, *flags = nullptr, *regimes = nullptr;   // per step: n^3, 3 nf, np, np
  // per segment tape: particles at each step start, u0, mass, u2, p per step
  void *tx = nullptr, *tv = nullptr, *tu0 = nullptr, *tmass = nullptr, *tu2 = nullptr, *tp = nullptr;
  void *ckx = nullptr, *ckv = nullptr;   // checkpoints: particles at every segment start
  int cgIters = 0;
  DGrid col{};                  // the collider's distance grid (mode 1), or mode 0
  float* gridData = nullptr;
  DGrid grid_() const { return col; }
};

static size_t esz(const st_diff* s) { return s->fp64 ? 8 : 4; }

// centre of the collider at time t (keyframes K[8][3] at t_k = k T / 7), and the step's collider records
static void collider_path(const st_diff* s, const double* K, std::vector<double>& cs, std::vector<double>& vs) {
  const int S = (int)s->d.steps;
  const double T = S * (double)s->d.dt;
  auto at = [&](double t, double* o) {
    double u = t / T * 7.0;
    int i = std::min(6, std::max(0, (int)std::floor(u)));
    double a = u - i;
    for (int d = 0; d < 3; d++) o[d] = (1 - a) * K[i * 3 + d] + a * K[(i + 1) * 3 + d];
  };
  cs.assign((size_t)S * 3, 0.0);
  vs.assign((size_t)S * 3, 0.0);
  for (int k = 0; k < S; k++) {
    double c0[3], c1[3];
    at(k * (double)s->d.dt, c0);
    at((k + 1) * (double)s->d.dt, c1);
    for (int d = 0; d < 3; d++) { cs[k * 3 + d] = c1[d]; vs[k * 3 + d] = (c1[d] - c0[d]) / s->d.dt; }
  }
}
// d c(t) / d K: the two keyframes and weights
static void path_weights(const st_diff* s, double t, int& i, double& wa, double& wb) {
  const double T = s->d.steps * (double)s->d.dt;
  double u = t / T * 7.0;
  i = std::min(6, std::max(0, (int)std::floor(u)));
  double a = u - i;
  wa = 1 - a;
  wb = a;
}

template <class T>
static T* P(void* p) { return static_cast<T*>(p); }

// PCG on A y = rhs (fluid cells), from y = 0. The scalars stay on the device (red: 0 rz, 1 rr, 2 pAp, 3 new rz, 4 new rr,
// 5 alpha, 6 beta); the host reads the residual every 16 iterations.
__global__ void k_d_zero(double* a, int n) { if (threadIdx.x < n) a[threadIdx.x] = 0.0; }
__global__ void k_d_alpha(double* red) { red[5] = red[2] > 0.0 ? red[0] / red[2] : 0.0; red[3] = 0.0; red[4] = 0.0; }
__global__ void k_d_beta(double* red) { red[6] = red[0] > 0.0 ? red[3] / red[0] : 0.0; red[0] = red[3]; red[1] = red[4]; red[2] = 0.0; }
template <class T>
__global__ void k_d_step(size_t n, const double* __restrict__ red, const T* __restrict__ pd, const T* __restrict__ Ap,
                         const T* __restrict__ dinv, T* y, T* r, T* z) {   // y += alpha p; r -= alpha Ap; z = r / diag
  const T alpha = (T)red[5];
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    y[i] += alpha * pd[i];
    const T ri = r[i] - alpha * Ap[i];
    r[i] = ri;
    z[i] = dinv[i] * ri;
  }
}
template <class T>
__global__ void k_d_dir(size_t n, const double* __restrict__ red, const T* __restrict__ z, T* pd) {   // p = z + beta p
  const T beta = (T)red[6];
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) pd[i] = z[i] + beta * pd[i];
}
template <class T>
static st_status pcg(st_diff* s, const uint8_t* types, const T* rhs, T* y) {
  const DGeo& G = s->G;
  const size_t n = G.cells();
  cudaStream_t q = s->stream;
  const int gr = s->grid;
  T *r = P<T>(s->r), *z = P<T>(s->z), *pd = P<T>(s->pd), *Ap = P<T>(s->q), *dinv = P<T>(s->dinv);
  double* red = s->red;
  DK(cudaMemsetAsync(y, 0, n * sizeof(T), q));
  DK(cudaMemcpyAsync(r, rhs, n * sizeof(T), cudaMemcpyDeviceToDevice, q));
  k_d_apply<T><<<gr, 256, 0, q>>>(G, types, y, Ap, dinv);   // fills the preconditioner
  k_d_mul<T><<<gr, 256, 0, q>>>(n, dinv, r, z);
  DK(cudaMemcpyAsync(pd, z, n * sizeof(T), cudaMemcpyDeviceToDevice, q));
  k_d_zero<<<1, 32, 0, q>>>(red, 8);
  k_d_dot<T><<<gr, 256, 0, q>>>(n, r, z, red);
  k_d_dot<T><<<gr, 256, 0, q>>>(n, r, r, red + 1);
  double h[8];
  DK(cudaMemcpyAsync(h, red, 2 * sizeof(double), cudaMemcpyDeviceToHost, q));
  DK(cudaStreamSynchronize(q));
  const double b2 = h[1];
  if (b2 == 0.0) return ST_OK;
  const double tol2 = (double)s->d.cg_tol * (double)s->d.cg_tol * b2;
  int it = 0;
  while (it < (int)s->d.cg_maxit) {
    const int chunk = std::min(16, (int)s->d.cg_maxit - it);
    for (int k = 0; k < chunk; k++) {
      k_d_apply<T><<<gr, 256, 0, q>>>(G, types, pd, Ap, nullptr);
      k_d_dot<T><<<gr, 256, 0, q>>>(n, pd, Ap, red + 2);
      k_d_alpha<<<1, 1, 0, q>>>(red);
      k_d_step<T><<<gr, 256, 0, q>>>(n, red, pd, Ap, dinv, y, r, z);
      k_d_dot<T><<<gr, 256, 0, q>>>(n, r, z, red + 3);
      k_d_dot<T><<<gr, 256, 0, q>>>(n, r, r, red + 4);
      k_d_beta<<<1, 1, 0, q>>>(red);
      k_d_dir<T><<<gr, 256, 0, q>>>(n, red, z, pd);
    }
    it += chunk;
    DK(cudaMemcpyAsync(h, red, 2 * sizeof(double), cudaMemcpyDeviceToHost, q));
    DK(cudaStreamSynchronize(q));
    if (h[1] <= tol2 || h[0] == 0.0) break;
  }
  s->cgIters += it;
  return ST_OK;
}

// one forward step k from (x, v) into (xn, vn); record: decide the discrete choices, else reuse them. tapeSlot >= 0:
// keep u0, mass, u2, p of the step in the tape.
template <class T>
static st_status step_fwd(st_diff* s, int k, bool record, const double* cs, const double* vs, int tapeSlot) {
  const DGeo& G = s->G;
  const size_t nf = G.nf(0), nc = G.cells();
  cudaStream_t q = s->stream;
  const int gr = s->grid;
  T* cb = P<T>(s->cbuf) + (size_t)k * 9;
  T hcb[9];
  for (int d = 0; d < 3; d++) { hcb[d] = (T)cs[k * 3 + d]; hcb[3 + d] = (T)vs[k * 3 + d]; hcb[6 + d] = (T)s->d.box_half[d]; }
  DK(cudaMemcpyAsync(cb, hcb, 9 * sizeof(T), cudaMemcpyHostToDevice, q));
  uint8_t* types = s->types + (size_t)k * nc;
  uint8_t* mask = s->mask + (size_t)k * 3 * nf;
  uint8_t* flags = s->flags + (size_t)k * s->np;
  uint8_t* regimes = s->regimes + (size_t)k * s->np;
  DK(cudaMemsetAsync(s->mom, 0, 3 * nf * sizeof(T), q));
  DK(cudaMemsetAsync(s->mass, 0, 3 * nf * sizeof(T), q));
  if (record) DK(cudaMemsetAsync(s->count, 0, nc * sizeof(int), q));
  k_d_p2g<T><<<gr, 256, 0, q>>>(G, s->np, P<T>(s->x), P<T>(s->v), P<T>(s->mom), P<T>(s->mass), record ? s->count : nullptr);
  if (record) k_d_types<T><<<gr, 256, 0, q>>>(G, s->count, cb, cb + 6, s->grid_(), (T)s->d.q0, types);
  T* u0 = tapeSlot >= 0 ? P<T>(s->tu0) + (size_t)tapeSlot * 3 * nf : P<T>(s->u0);
  T* u2 = tapeSlot >= 0 ? P<T>(s->tu2) + (size_t)tapeSlot * 3 * nf : P<T>(s->u2);
  T* pp = tapeSlot >= 0 ? P<T>(s->tp) + (size_t)tapeSlot * nc : P<T>(s->p);
  if (tapeSlot >= 0) DK(cudaMemcpyAsync(P<T>(s->tmass) + (size_t)tapeSlot * 3 * nf, s->mass, 3 * nf * sizeof(T), cudaMemcpyDeviceToDevice, q));
  k_d_norm<T><<<gr, 256, 0, q>>>(G, P<T>(s->mom), P<T>(s->mass), mask, record ? 1 : 0, types, cb + 3, (T)(s->d.g * s->d.dt), u0, P<T>(s->u1));
  k_d_rhs<T><<<gr, 256, 0, q>>>(G, types, P<T>(s->u1), (T)(G.h / s->d.dt), P<T>(s->b));
  st_status st = pcg<T>(s, types, P<T>(s->b), pp);
  if (st != ST_OK) return st;
  k_d_project<T><<<gr, 256, 0, q>>>(G, types, pp, P<T>(s->u1), (T)(s->d.dt / G.h), u2);
  const T lo = (T)s->d.margin, hi = (T)(1.0 - s->d.margin);
  k_d_g2p<T><<<gr, 256, 0, q>>>(G, s->np, P<T>(s->x), P<T>(s->v), u2, u0, (T)s->d.flip, (T)s->d.dt, cb, cb + 6, s->grid_(), (T)s->d.q0, lo, hi,
                                flags, regimes, record ? 1 : 0, P<T>(s->xn), P<T>(s->vn));
  std::swap(s->x, s->xn);
  std::swap(s->v, s->vn);
  return ST_OK;
}

template <class T>
static st_status forward(st_diff* s, const double* params, bool record, double* loss) {
  const DGeo& G = s->G;
  cudaStream_t q = s->stream;
  std::vector<double> cs, vs;
  collider_path(s, params, cs, vs);
  DK(cudaMemcpyAsync(s->x, s->x0, s->np * 3 * sizeof(T), cudaMemcpyDeviceToDevice, q));
  T v0[3] = {(T)params[24], (T)params[25], (T)params[26]};
  DK(cudaMemcpyAsync(s->red, v0, sizeof(v0), cudaMemcpyHostToDevice, q));
  k_d_fillv<T><<<s->grid, 256, 0, q>>>(s->np, reinterpret_cast<const T*>(s->red), P<T>(s->v));
  const int ck = (int)s->d.ckpt_every;
  for (int k = 0; k < (int)s->d.steps; k++) {
    if (record && k % ck == 0) {
      const size_t seg = (size_t)(k / ck);
      DK(cudaMemcpyAsync(P<T>(s->ckx) + seg * s->np * 3, s->x, s->np * 3 * sizeof(T), cudaMemcpyDeviceToDevice, q));
      DK(cudaMemcpyAsync(P<T>(s->ckv) + seg * s->np * 3, s->v, s->np * 3 * sizeof(T), cudaMemcpyDeviceToDevice, q));
    }
    st_status st = step_fwd<T>(s, k, record, cs.data(), vs.data(), -1);
    if (st != ST_OK) return st;
  }
  DK(cudaMemsetAsync(s->rho, 0, G.cells() * sizeof(T), q));
  k_d_splat<T><<<s->grid, 256, 0, q>>>(G, s->np, P<T>(s->x), P<T>(s->rho));
  DK(cudaMemsetAsync(s->red, 0, sizeof(double), q));
  k_d_resid<T><<<s->grid, 256, 0, q>>>(G.cells(), P<T>(s->rho), s->tgt, nullptr, s->red);
  DK(cudaMemcpyAsync(loss, s->red, sizeof(double), cudaMemcpyDeviceToHost, q));
  DK(cudaStreamSynchronize(q));
  DK(cudaGetLastError());
  if (record) { s->recorded = true; s->params.assign(params, params + 27); }
  return ST_OK;
}

template <class T>
static st_status backward(st_diff* s, double* grad) {
  const DGeo& G = s->G;
  const size_t nf = G.nf(0), nc = G.cells(), np = s->np;
  cudaStream_t q = s->stream;
  const int gr = s->grid, S = (int)s->d.steps, ck = (int)s->d.ckpt_every;
  std::vector<double> cs, vs;
  collider_path(s, s->params.data(), cs, vs);
  // loss -> final positions (s->x holds them after the recorded forward)
  DK(cudaMemsetAsync(s->rho, 0, nc * sizeof(T), q));
  k_d_splat<T><<<gr, 256, 0, q>>>(G, np, P<T>(s->x), P<T>(s->rho));
  DK(cudaMemsetAsync(s->red, 0, sizeof(double), q));
  k_d_resid<T><<<gr, 256, 0, q>>>(nc, P<T>(s->rho), s->tgt, P<T>(s->rho), s->red);   // rho becomes d loss / d rho
  k_d_splat_b<T><<<gr, 256, 0, q>>>(G, np, P<T>(s->x), P<T>(s->rho), P<T>(s->gx));
  DK(cudaMemsetAsync(s->gv, 0, np * 3 * sizeof(T), q));
  std::vector<double> gc((size_t)S * 3, 0.0), gvc((size_t)S * 3, 0.0);
  double hred[8];
  for (int seg = (S - 1) / ck; seg >= 0; seg--) {
    const int k0 = seg * ck, k1 = std::min(S, k0 + ck);
    // recompute the segment from its checkpoint, keeping the tape
    DK(cudaMemcpyAsync(s->x, P<T>(s->ckx) + (size_t)seg * np * 3, np * 3 * sizeof(T), cudaMemcpyDeviceToDevice, q));
    DK(cudaMemcpyAsync(s->v, P<T>(s->ckv) + (size_t)seg * np * 3, np * 3 * sizeof(T), cudaMemcpyDeviceToDevice, q));
    for (int k = k0; k < k1; k++) {
      const int slot = k - k0;
      DK(cudaMemcpyAsync(P<T>(s->tx) + (size_t)slot * np * 3, s->x, np * 3 * sizeof(T), cudaMemcpyDeviceToDevice, q));
      DK(cudaMemcpyAsync(P<T>(s->tv) + (size_t)slot * np * 3, s->v, np * 3 * sizeof(T), cudaMemcpyDeviceToDevice, q));
      st_status st = step_fwd<T>(s, k, false, cs.data(), vs.data(), slot);
      if (st != ST_OK) return st;
    }
    for (int k = k1 - 1; k >= k0; k--) {
      const int slot = k - k0;
      const T* tx = P<T>(s->tx) + (size_t)slot * np * 3;
      const T* tv = P<T>(s->tv) + (size_t)slot * np * 3;
      const T* u0 = P<T>(s->tu0) + (size_t)slot * 3 * nf;
      const T* u2 = P<T>(s->tu2) + (size_t)slot * 3 * nf;
      const T* mass = P<T>(s->tmass) + (size_t)slot * 3 * nf;
      const uint8_t* types = s->types + (size_t)k * nc;
      const uint8_t* mask = s->mask + (size_t)k * 3 * nf;
      const uint8_t* flags = s->flags + (size_t)k * np;
      const uint8_t* regimes = s->regimes + (size_t)k * np;
      const T* cb = P<T>(s->cbuf) + (size_t)k * 9;
      T hcb[9];
      for (int d = 0; d < 3; d++) { hcb[d] = (T)cs[k * 3 + d]; hcb[3 + d] = (T)vs[k * 3 + d]; hcb[6 + d] = (T)s->d.box_half[d]; }
      DK(cudaMemcpyAsync(const_cast<T*>(cb), hcb, 9 * sizeof(T), cudaMemcpyHostToDevice, q));
      DK(cudaMemsetAsync(s->gu2, 0, 3 * nf * sizeof(T), q));
      DK(cudaMemsetAsync(s->gu0, 0, 3 * nf * sizeof(T), q));
      DK(cudaMemsetAsync(s->cred, 0, 8 * sizeof(double), q));
      k_d_g2p_b<T><<<gr, 256, 0, q>>>(G, np, tx, tv, u2, u0, (T)s->d.flip, (T)s->d.dt, cb, cb + 6, s->grid_(), (T)s->d.q0,
                                      (T)s->d.margin, (T)(1.0 - s->d.margin), flags,
                                      regimes, P<T>(s->gx), P<T>(s->gv), P<T>(s->gu2), P<T>(s->gu0), s->cred);
      k_d_project_b<T><<<gr, 256, 0, q>>>(G, types, P<T>(s->gu2), (T)(s->d.dt / G.h), P<T>(s->gp));
      st_status st = pcg<T>(s, types, P<T>(s->gp), P<T>(s->gb));   // A is symmetric: the adjoint solve uses it again
      if (st != ST_OK) return st;
      k_d_norm_b<T><<<gr, 256, 0, q>>>(G, types, P<T>(s->gb), (T)(G.h / s->d.dt), P<T>(s->gu2), mask, u0, mass, P<T>(s->gu0),
                                       P<T>(s->gmom), P<T>(s->gmass), s->cred + 3);
      k_d_p2g_b<T><<<gr, 256, 0, q>>>(G, np, tx, tv, P<T>(s->gmom), P<T>(s->gmass), P<T>(s->gx), P<T>(s->gv));
      DK(cudaMemcpyAsync(hred, s->cred, 6 * sizeof(double), cudaMemcpyDeviceToHost, q));
      DK(cudaStreamSynchronize(q));
      for (int d = 0; d < 3; d++) { gc[k * 3 + d] = hred[d]; gvc[k * 3 + d] = hred[3 + d]; }
    }
  }
  // initial velocity: every particle starts with v0
  DK(cudaMemsetAsync(s->red, 0, 3 * sizeof(double), q));
  k_d_sumv<T><<<gr, 256, 0, q>>>(np, P<T>(s->gv), s->red);
  DK(cudaMemcpyAsync(hred, s->red, 3 * sizeof(double), cudaMemcpyDeviceToHost, q));
  DK(cudaStreamSynchronize(q));
  DK(cudaGetLastError());
  for (int i = 0; i < 27; i++) grad[i] = 0.0;
  for (int d = 0; d < 3; d++) grad[24 + d] = hred[d];
  // collider centre c_k = c(t_{k+1}), velocity (c(t_{k+1}) - c(t_k)) / dt, both linear in the keyframes
  for (int k = 0; k < S; k++) {
    int i1, i0;
    double a1, b1, a0, b0;
    path_weights(s, (k + 1) * (double)s->d.dt, i1, a1, b1);
    path_weights(s, k * (double)s->d.dt, i0, a0, b0);
    for (int d = 0; d < 3; d++) {
      const double g1 = gc[k * 3 + d] + gvc[k * 3 + d] / s->d.dt, g0 = -gvc[k * 3 + d] / s->d.dt;
      grad[i1 * 3 + d] += a1 * g1;
      grad[(i1 + 1) * 3 + d] += b1 * g1;
      grad[i0 * 3 + d] += a0 * g0;
      grad[(i0 + 1) * 3 + d] += b0 * g0;
    }
  }
  return ST_OK;
}

extern "C" {

void st_diff_destroy(st_diff* s) {
  if (!s) return;
  cudaSetDevice(s->d.device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->mem) cudaFree(s->mem);
  if (s->gridData) cudaFree(s->gridData);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

st_status st_diff_create(const st_diff_desc* d, const float* pos3, uint32_t np, const float* target, st_diff** out) {
  if (!d || !pos3 || !np || !target || !out || d->size != sizeof(st_diff_desc) || d->n < 4 || d->n > 512 || !d->steps ||
      !d->ckpt_every || d->dt <= 0.0f)
    return ST_BAD_ARG;
  *out = nullptr;
  st_diff* s = new st_diff();
  s->d = *d;
  s->G = DGeo{(int)d->n, 1.0 / d->n, (double)d->n};
  s->np = np;
  s->fp64 = d->fp64 != 0;
  cudaError_t e = cudaSetDevice(d->device);
  int sms = 148;
  if (e == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d->device);
  s->grid = sms * 8;
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  const size_t E = esz(s), nf = s->G.nf(0), nc = s->G.cells(), S = d->steps, ck = d->ckpt_every, segs = (S + ck - 1) / ck;
  struct Item { void** p; size_t bytes; };
  std::vector<Item> items = {
      {&s->x0, np * 3 * E}, {&s->x, np * 3 * E}, {&s->v, np * 3 * E}, {&s->xn, np * 3 * E}, {&s->vn, np * 3 * E},
      {&s->mom, 3 * nf * E}, {&s->mass, 3 * nf * E}, {&s->u0, 3 * nf * E}, {&s->u1, 3 * nf * E}, {&s->u2, 3 * nf * E},
      {&s->b, nc * E}, {&s->p, nc * E}, {&s->r, nc * E}, {&s->z, nc * E}, {&s->pd, nc * E}, {&s->q, nc * E}, {&s->dinv, nc * E},
      {&s->rho, nc * E}, {&s->gx, np * 3 * E}, {&s->gv, np * 3 * E}, {&s->gu2, 3 * nf * E}, {&s->gu0, 3 * nf * E},
      {&s->gmom, 3 * nf * E}, {&s->gmass, 3 * nf * E}, {&s->gp, nc * E}, {&s->gb, nc * E}, {&s->cbuf, S * 9 * E},
      {(void**)&s->tgt, nc * 4}, {(void**)&s->count, nc * 4}, {(void**)&s->red, 64}, {(void**)&s->cred, 64},
      {(void**)&s->types, S * nc}, {(void**)&s->mask, S * 3 * nf}, {(void**)&s->flags, S * np}, {(void**)&s->regimes, S * np},
      {&s->tx, ck * np * 3 * E}, {&s->tv, ck * np * 3 * E}, {&s->tu0, ck * 3 * nf * E}, {&s->tmass, ck * 3 * nf * E},
      {&s->tu2, ck * 3 * nf * E}, {&s->tp, ck * nc * E}, {&s->ckx, segs * np * 3 * E}, {&s->ckv, segs * np * 3 * E}};
  size_t tot = 0;
  for (auto& it : items) tot += (it.bytes + 255) & ~(size_t)255;
  if (e == cudaSuccess) e = cudaMalloc(&s->mem, tot);
  if (e == cudaSuccess) {
    char* m = static_cast<char*>(s->mem);
    for (auto& it : items) { *it.p = m; m += (it.bytes + 255) & ~(size_t)255; }
    s->memBytes = tot;
    if (s->fp64) {
      std::vector<double> x(np * 3);
      for (size_t i = 0; i < np * 3; i++) x[i] = pos3[i];
      e = cudaMemcpy(s->x0, x.data(), np * 3 * 8, cudaMemcpyHostToDevice);
    } else {
      e = cudaMemcpy(s->x0, pos3, np * 3 * 4, cudaMemcpyHostToDevice);
    }
  }
  if (e == cudaSuccess) e = cudaMemcpy(s->tgt, target, nc * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && d->collider_grid) {
    // the box's exact signed distance at grid nodes, 3 cells of margin around it (as a mesh collider's grid is built)
    const double cell = d->grid_cell > 0.0f ? (double)d->grid_cell : 0.5 / d->n, m = 3.0 * cell;
    DGrid& Gd = s->col;
    Gd.mode = 1;
    Gd.cell = cell;
    for (int k = 0; k < 3; k++) {
      Gd.origin[k] = -((double)d->box_half[k] + m);
      Gd.dims[k] = (int)std::floor(2.0 * ((double)d->box_half[k] + m) / cell + 1e-9) + 1;
    }
    const size_t ng = (size_t)Gd.dims[0] * Gd.dims[1] * Gd.dims[2];
    std::vector<float> h(ng);
    for (int k = 0; k < Gd.dims[2]; k++)
      for (int j = 0; j < Gd.dims[1]; j++)
        for (int i = 0; i < Gd.dims[0]; i++) {
          const double x[3] = {Gd.origin[0] + i * cell, Gd.origin[1] + j * cell, Gd.origin[2] + k * cell};
          double o2 = 0.0, in = -1e30;
          for (int a = 0; a < 3; a++) {
            const double qd = std::fabs(x[a]) - d->box_half[a];
            o2 += std::max(qd, 0.0) * std::max(qd, 0.0);
            in = std::max(in, qd);
          }
          h[(size_t)i + (size_t)Gd.dims[0] * ((size_t)j + (size_t)Gd.dims[1] * k)] = (float)(std::sqrt(o2) + std::min(in, 0.0));
        }
    e = cudaMalloc((void**)&s->gridData, ng * 4);
    if (e == cudaSuccess) e = cudaMemcpy(s->gridData, h.data(), ng * 4, cudaMemcpyHostToDevice);
    Gd.data = s->gridData;
  }
  if (e != cudaSuccess) {
    snprintf(g_derr, sizeof(g_derr), "diff create: %s", cudaGetErrorString(e));
    st::set_error_text(g_derr);
    st_diff_destroy(s);
    return e == cudaErrorMemoryAllocation ? ST_OOM : ST_DEVICE_ERROR;
  }
  *out = s;
  return ST_OK;
}

st_status st_diff_forward(st_diff* s, const double* params, int32_t record, double* loss) {
  if (!s || !params || !loss) return ST_BAD_ARG;
  if (!record && !s->recorded) {
    st::set_error_text("st_diff_forward: a frozen pass needs a recorded one first");
    return ST_BAD_ARG;
  }
  DK(cudaSetDevice(s->d.device));
  s->cgIters = 0;
  return s->fp64 ? forward<double>(s, params, record != 0, loss) : forward<float>(s, params, record != 0, loss);
}

st_status st_diff_backward(st_diff* s, double* grad) {
  if (!s || !grad) return ST_BAD_ARG;
  if (!s->recorded) {
    st::set_error_text("st_diff_backward: no recorded forward pass");
    return ST_BAD_ARG;
  }
  DK(cudaSetDevice(s->d.device));
  // the final state of the recorded pass: recompute it (a frozen pass may have run since) as a frozen pass, so the
  // decisions stay those of the recording (recording again could flip one whose test sits at rounding level, such as
  // the sign of v.n of a particle sliding along the collider, since the FP64 sums are atomic)
  double loss;
  std::vector<double> prm = s->params;
  st_status st = s->fp64 ? forward<double>(s, prm.data(), false, &loss) : forward<float>(s, prm.data(), false, &loss);
  if (st != ST_OK) return st;
  s->cgIters = 0;
  return s->fp64 ? backward<double>(s, grad) : backward<float>(s, grad);
}

void* st_diff_stream(st_diff* s) { return s ? (void*)s->stream : nullptr; }

st_status st_diff_read_state(st_diff* s, float* pos3, float* vel3) {
  if (!s || !pos3) return ST_BAD_ARG;
  DK(cudaSetDevice(s->d.device));
  DK(cudaStreamSynchronize(s->stream));
  const size_t n = s->np * 3;
  for (int w = 0; w < 2; w++) {
    float* out = w == 0 ? pos3 : vel3;
    if (!out) continue;
    const void* src = w == 0 ? s->x : s->v;
    if (s->fp64) {
      std::vector<double> h(n);
      DK(cudaMemcpy(h.data(), src, n * 8, cudaMemcpyDeviceToHost));
      for (size_t i = 0; i < n; i++) out[i] = (float)h[i];
    } else {
      DK(cudaMemcpy(out, src, n * 4, cudaMemcpyDeviceToHost));
    }
  }
  return ST_OK;
}

st_status st_diff_stats(st_diff* s, uint64_t* device_bytes, int32_t* cg_iters) {
  if (!s) return ST_BAD_ARG;
  if (device_bytes) *device_bytes = s->memBytes;
  if (cg_iters) *cg_iters = s->cgIters;
  return ST_OK;
}

}  // extern "C"
