// poisson_oracle.cpp - CPU checker of the pressure solve study (st_poisson_*), test infrastructure only.
//
// The system is the reference's pressure solve (relax, src/flip/wgsl-solver.js:124-140; neighbour types as ctypeOf,
// src/flip/wgsl-core.js:104-112): for a fluid cell nns p - sum(fluid neighbours p) = rhs. This file provides
//   * FP32 red-black SOR sweeps from zero, the same operations as the kernels (bit-exact comparison);
//   * the FP64 residual and its norm, summed per tile by the same tree and over tiles in tile order;
//   * the all-FP64 reference solution by conjugate gradients (the operator is symmetric positive definite when every
//     fluid region touches air), to which the FP32, refined and FP64-SOR solutions are compared.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/splashtank_cuda.h"

namespace {

struct Pois {
  uint32_t nx, ny, nz, tx, ty, tz, open;
  std::vector<uint32_t> tiles;          // tiles holding fluid, ascending
  std::vector<uint16_t> info;           // per cell of the tile box: fluid flag, fluid neighbour mask, non-solid count
  std::vector<double> b;
  int nthreads = 1;
  size_t cell(long i, long j, long k) const {
    size_t t = (size_t)(i >> 3) + tx * ((size_t)(j >> 3) + (size_t)ty * (k >> 3));
    return t * 512 + (i & 7) + 8 * ((j & 7) + 8 * (k & 7));
  }
  void coords(size_t c, long& i, long& j, long& k) const {
    size_t t = c >> 9, l = c & 511, tt = t / tx;
    i = (long)((t % tx) * 8 + (l & 7)); j = (long)((tt % ty) * 8 + ((l >> 3) & 7)); k = (long)((tt / ty) * 8 + (l >> 6));
  }
  int ty_(const uint8_t* type, long i, long j, long k) const {
    if (i < 0) return (open & 1u) ? 0 : 2;
    if (i >= (long)nx) return (open & 2u) ? 0 : 2;
    if (j < 0) return (open & 4u) ? 0 : 2;
    if (j >= (long)ny) return (open & 8u) ? 0 : 2;
    if (k < 0) return (open & 16u) ? 0 : 2;
    if (k >= (long)nz) return (open & 32u) ? 0 : 2;
    return type[(size_t)i + nx * ((size_t)j + (size_t)ny * k)];
  }
  void set(const uint8_t* type, const double* rhs) {
    size_t T = (size_t)tx * ty * tz;
    info.assign(T * 512, 0); b.assign(T * 512, 0.0);
    std::vector<uint8_t> on(T, 0);
    for (long k = 0; k < (long)nz; k++) for (long j = 0; j < (long)ny; j++) for (long i = 0; i < (long)nx; i++) {
      size_t o = (size_t)i + nx * ((size_t)j + (size_t)ny * k);
      if (type[o] != 1) continue;
      const long q[6][3] = {{i - 1, j, k}, {i + 1, j, k}, {i, j - 1, k}, {i, j + 1, k}, {i, j, k - 1}, {i, j, k + 1}};
      uint32_t mask = 0, nns = 0;
      for (int a = 0; a < 6; a++) { int t = ty_(type, q[a][0], q[a][1], q[a][2]); if (t != 2) nns++; if (t == 1) mask |= 1u << a; }
      size_t c = cell(i, j, k);
      info[c] = (uint16_t)(0x8000u | (nns << 8) | mask);
      b[c] = rhs[o];
      on[c >> 9] = 1;
    }
    tiles.clear();
    for (size_t t = 0; t < T; t++) if (on[t]) tiles.push_back((uint32_t)t);
  }
  size_t nbr(size_t c, int a) const {
    long i, j, k; coords(c, i, j, k);
    if (a == 0) i--; else if (a == 1) i++; else if (a == 2) j--; else if (a == 3) j++; else if (a == 4) k--; else k++;
    return cell(i, j, k);
  }
  // FP32 red-black SOR iterations from zero on (float) b (same operations as k_ps_sor32)
  void sweeps32(float omega, int iters, std::vector<float>& p) const {
    p.assign(info.size(), 0.0f);
    std::vector<float> rhs(info.size(), 0.0f);
    for (uint32_t t : tiles) for (int l = 0; l < 512; l++) rhs[(size_t)t * 512 + l] = (float)b[(size_t)t * 512 + l];
    for (int it = 0; it < iters; it++) for (uint32_t color = 0; color < 2; color++) {
#pragma omp parallel for schedule(static) num_threads(nthreads)
      for (long ti = 0; ti < (long)tiles.size(); ti++) {
        uint32_t t = tiles[ti];
        for (int l = 0; l < 512; l++) {
          size_t c = (size_t)t * 512 + l;
          int lx = l & 7, ly = (l >> 3) & 7, lz = l >> 6;
          if ((uint32_t)((lx + ly + lz) & 1) != color) continue;
          uint32_t in = info[c];
          if (!(in & 0x8000u)) continue;
          uint32_t nns = (in >> 8) & 7u;
          if (nns == 0u) { p[c] = 0.0f; continue; }
          float sum = 0.0f;
          for (int a = 0; a < 6; a++) if (in & (1u << a)) sum += p[nbr(c, a)];
          float pg = (rhs[c] + sum) / (float)nns;
          p[c] = p[c] + omega * (pg - p[c]);
        }
      }
    }
  }
  // ||b - A x||^2 and ||b||^2, per tile by the kernels' tree, tiles in order
  void norms(const std::vector<double>& x, double& r2, double& b2) const {
    std::vector<double> tr(tiles.size()), tb(tiles.size());
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (long ti = 0; ti < (long)tiles.size(); ti++) {
      double sr[512], sb[512];
      uint32_t t = tiles[ti];
      for (int l = 0; l < 512; l++) {
        size_t c = (size_t)t * 512 + l; uint32_t in = info[c];
        double rv = 0.0, bv = 0.0;
        if (in & 0x8000u) {
          uint32_t nns = (in >> 8) & 7u; double s = 0.0;
          for (int a = 0; a < 6; a++) if (in & (1u << a)) s += x[nbr(c, a)];
          bv = b[c]; rv = bv - ((double)nns * x[c] - s);
        }
        sr[l] = rv * rv; sb[l] = bv * bv;
      }
      for (int w = 256; w > 0; w >>= 1) for (int l = 0; l < w; l++) { sr[l] += sr[l + w]; sb[l] += sb[l + w]; }
      tr[ti] = sr[0]; tb[ti] = sb[0];
    }
    // the kernels' final sum: 1024 threads each summing a contiguous chunk, then a halving tree
    size_t nT = tiles.size(), chunk = (nT + 1023) / 1024;
    double s1[1024], s2[1024];
    for (size_t th = 0; th < 1024; th++) {
      size_t beg = std::min(th * chunk, nT), end = std::min(beg + chunk, nT);
      double a = 0.0, bb = 0.0;
      for (size_t k = beg; k < end; k++) { a += tr[k]; bb += tb[k]; }
      s1[th] = a; s2[th] = bb;
    }
    for (int w = 512; w > 0; w >>= 1) for (int l = 0; l < w; l++) { s1[l] += s1[l + w]; s2[l] += s2[l + w]; }
    r2 = s1[0]; b2 = s2[0];
  }
  void applyA(const std::vector<double>& x, std::vector<double>& y) const {
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (long ti = 0; ti < (long)tiles.size(); ti++) {
      uint32_t t = tiles[ti];
      for (int l = 0; l < 512; l++) {
        size_t c = (size_t)t * 512 + l; uint32_t in = info[c];
        if (!(in & 0x8000u)) { y[c] = 0.0; continue; }
        double s = 0.0;
        for (int a = 0; a < 6; a++) if (in & (1u << a)) s += x[nbr(c, a)];
        y[c] = (double)((in >> 8) & 7u) * x[c] - s;
      }
    }
  }
  double dotp(const std::vector<double>& a, const std::vector<double>& b2) const {
    double s = 0.0;
    for (uint32_t t : tiles) for (int l = 0; l < 512; l++) { size_t c = (size_t)t * 512 + l; s += a[c] * b2[c]; }
    return s;
  }
  // all-FP64 reference: conjugate gradients from zero to ||r|| / ||b|| <= tol
  int cg(double tol, int maxit, std::vector<double>& x) const {
    size_t n = info.size();
    x.assign(n, 0.0);
    std::vector<double> r = b, p = b, Ap(n, 0.0);
    double rr = dotp(r, r), bb = rr;
    if (bb == 0.0) return 0;
    int it = 0;
    for (; it < maxit && std::sqrt(rr / bb) > tol; it++) {
      applyA(p, Ap);
      double alpha = rr / dotp(p, Ap);
      for (uint32_t t : tiles) for (int l = 0; l < 512; l++) { size_t c = (size_t)t * 512 + l; x[c] += alpha * p[c]; r[c] -= alpha * Ap[c]; }
      double rn = dotp(r, r), beta = rn / rr;
      rr = rn;
      for (uint32_t t : tiles) for (int l = 0; l < 512; l++) { size_t c = (size_t)t * 512 + l; p[c] = r[c] + beta * p[c]; }
    }
    return it;
  }
  void toDense(const std::vector<double>& x, double* out) const {
    for (long k = 0; k < (long)nz; k++) for (long j = 0; j < (long)ny; j++) for (long i = 0; i < (long)nx; i++)
      out[(size_t)i + nx * ((size_t)j + (size_t)ny * k)] = x[cell(i, j, k)];
  }
  void fromDense(const double* in, std::vector<double>& x) const {
    x.assign(info.size(), 0.0);
    for (long k = 0; k < (long)nz; k++) for (long j = 0; j < (long)ny; j++) for (long i = 0; i < (long)nx; i++)
      x[cell(i, j, k)] = in[(size_t)i + nx * ((size_t)j + (size_t)ny * k)];
  }
};

}  // namespace

extern "C" {
void* oracle_poisson_create(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t open, int threads) {
  Pois* s = new Pois();
  s->nx = nx; s->ny = ny; s->nz = nz; s->tx = (nx + 7) / 8; s->ty = (ny + 7) / 8; s->tz = (nz + 7) / 8; s->open = open;
  s->nthreads = threads < 1 ? 1 : threads;
  return s;
}
void oracle_poisson_destroy(void* h) { delete (Pois*)h; }
void oracle_poisson_set(void* h, const uint8_t* type, const double* rhs) { ((Pois*)h)->set(type, rhs); }
// FP32 SOR iterations from zero; the dense result as doubles
void oracle_poisson_sweeps32(void* h, float omega, int iters, double* out) {
  Pois* s = (Pois*)h; std::vector<float> p; s->sweeps32(omega, iters, p);
  std::vector<double> x(p.begin(), p.end()); s->toDense(x, out);
}
// ||b - A x|| / ||b|| for a dense FP64 field (the kernels' summation order), and the squared norms
double oracle_poisson_rel_residual(void* h, const double* dense, double* r2out, double* b2out) {
  Pois* s = (Pois*)h; std::vector<double> x; s->fromDense(dense, x);
  double r2, b2; s->norms(x, r2, b2);
  if (r2out) *r2out = r2;
  if (b2out) *b2out = b2;
  return b2 > 0 ? std::sqrt(r2) / std::sqrt(b2) : 0.0;
}
int oracle_poisson_cg(void* h, double tol, int maxit, double* out) {
  Pois* s = (Pois*)h; std::vector<double> x; int it = s->cg(tol, maxit, x); s->toDense(x, out); return it;
}
}
