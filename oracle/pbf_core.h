// pbf_core.h - CPU restatement of GpuSim's position-based fluid passes (src/gpu.js:102-353), test infrastructure only:
// the parity checker of the sm_100a PBF kernels and a timed CPU baseline, never linked into the product.
//
// Each function restates one WGSL function or dispatch of GPU_WGSL with its f32 arithmetic in source order (built with
// -ffp-contract=off, so nothing is fused). Two choices fix what the reference leaves open:
//   * scatter (src/gpu.js:201-206) hands out a cell's slots with an atomic counter, so the order of the particles of a
//     cell - and with it the order of every neighbour sum - varies from run to run; here it is ascending particle
//     index, one of the orders the reference can produce;
//   * inverseSqrt(x) is computed as 1 / sqrt(x) (WGSL leaves its rounding to the implementation).
// The constants are FluidSim's (src/shared.js:236-270), computed in double as the JavaScript does and rounded to f32
// as GpuSim's Float32Array upload does (src/gpu.js:414-416).
#ifndef ORACLE_PBF_CORE_H
#define ORACLE_PBF_CORE_H
#include <cmath>
#include <cstdint>
#include <vector>

#include "oracle_math.h"

// the f32 uniform block of GpuSim.step (struct Params, src/gpu.js:73-82), plus 1/h and 1/rho0, which the shaders
// compute in f32 (cellOf, lambda, delta, viscosity)
struct PbfP {
  uint32_t n, nx, ny, nz, ncols, open;
  float dt, h, h2, d, rho0, poly, spiky, W0, eps, c0, Gh, margin, gravity, visc, rest, relax;
  float bx0, bx1, by0, by1, bz0, bz1, maxD, vmax, inv, irho;
};
const uint32_t PBF_DEADC = 0xffffffffu;

// FluidSim's derived constants in double (src/shared.js:236-270)
struct PbfConsts { double h, h2, poly, spiky, W0, rho0, eps, c0, Gh, margin, relax, rest; };
inline double pbfG(double h2, double s) {
  const double h4 = h2 * h2, h6 = h4 * h2, h8 = h4 * h4;
  const double s2 = s * s, s3 = s2 * s, s5 = s3 * s2, s7 = s5 * s2, s9 = s7 * s2;
  return h8 * s - (4.0 / 3.0) * h6 * s3 + (6.0 / 5.0) * h4 * s5 - (4.0 / 7.0) * h2 * s7 + s9 / 9.0;
}
inline PbfConsts pbfConsts(double d, double epsK, double wallK) {
  PbfConsts c;
  const double PI = 3.141592653589793;
  c.h = 2.2 * d;
  const double h = c.h, h2 = h * h;
  c.h2 = h2;
  c.poly = 315.0 / (64.0 * PI * std::pow(h, 9));
  c.spiky = -45.0 / (PI * std::pow(h, 6));
  c.W0 = c.poly * std::pow(h2, 3);
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
  c.relax = 1.0;
  c.rest = 0.1;
  c.Gh = pbfG(h2, h);
  const double c0 = (1.0 / (d * d * d)) * (PI / 4.0) * c.poly;
  const double cont = c0 * (c.Gh - pbfG(h2, d / 2.0));
  c.c0 = c0 * (below / cont) * (wallK > 0 ? wallK : 1.8);
  c.margin = 0.15 * d;
  return c;
}
// the uniform block as GpuSim.step packs it (src/gpu.js:410-416): every value rounded once to f32
inline PbfP pbfParams(const PbfConsts& c, double d, const double lo[3], const double hi[3], double dt, double g, double visc,
                      uint32_t n, uint32_t ncols, uint32_t open) {
  PbfP P{};
  P.n = n; P.ncols = ncols; P.open = open;
  P.nx = (uint32_t)std::ceil((hi[0] - lo[0]) / c.h) + 1u;
  P.ny = (uint32_t)std::ceil((hi[1] - lo[1]) / c.h) + 1u;
  P.nz = (uint32_t)std::ceil((hi[2] - lo[2]) / c.h) + 1u;
  P.dt = (float)dt; P.h = (float)c.h; P.h2 = (float)c.h2; P.d = (float)d; P.rho0 = (float)c.rho0; P.poly = (float)c.poly;
  P.spiky = (float)c.spiky; P.W0 = (float)c.W0; P.eps = (float)c.eps; P.c0 = (float)c.c0; P.Gh = (float)c.Gh;
  P.margin = (float)c.margin; P.gravity = (float)g; P.visc = (float)visc; P.rest = (float)c.rest; P.relax = (float)c.relax;
  P.bx0 = (float)lo[0]; P.bx1 = (float)hi[0]; P.by0 = (float)lo[1]; P.by1 = (float)hi[1]; P.bz0 = (float)lo[2]; P.bz1 = (float)hi[2];
  P.maxD = (float)(0.5 * d); P.vmax = 12.0f;
  P.inv = 1.0f / P.h;
  P.irho = 1.0f / P.rho0;
  return P;
}

// Gf (src/gpu.js:116-121), in f32
inline float pbfGf(const PbfP& P, float s) {
  const float h2 = P.h2, h4 = h2 * h2, h6 = h4 * h2, h8 = h4 * h4;
  const float s2 = s * s, s3 = s2 * s, s5 = s3 * s2, s7 = s5 * s2, s9 = s7 * s2;
  return h8 * s - (4.0f / 3.0f) * h6 * s3 + (6.0f / 5.0f) * h4 * s5 - (4.0f / 7.0f) * h2 * s7 + s9 / 9.0f;
}
// surf (src/gpu.js:123-128): (density, d density / d distance) of a solid surface at distance phi0
inline void pbfSurf(const PbfP& P, float phi0, float& rho, float& drho) {
  const float p = fmax_(phi0, 0.0f);
  const float t = P.h2 - p * p;
  const float t2 = t * t;
  rho = P.c0 * (P.Gh - pbfGf(P, p));
  drho = -P.c0 * t2 * t2;
}
// bnd (src/gpu.js:129-148): boundary density of the closed walls and of every collider's distance grid.
// sdf(k, x, phi, wn) evaluates collider k (sdfEval).
template <class Sdf>
inline void pbfBnd(const PbfP& P, const Sdf& sdf, uint32_t ncols, V3 x, float& rho, V3& g) {
  const float h = P.h;
  rho = 0.0f;
  g = v3(0, 0, 0);
  float r, dr;
  float ph = x.x - P.bx0; if ((P.open & 1u) == 0u && ph < h) { pbfSurf(P, ph, r, dr); rho += r; g.x += dr; }
  ph = P.bx1 - x.x; if ((P.open & 2u) == 0u && ph < h) { pbfSurf(P, ph, r, dr); rho += r; g.x -= dr; }
  ph = x.y - P.by0; if ((P.open & 4u) == 0u && ph < h) { pbfSurf(P, ph, r, dr); rho += r; g.y += dr; }
  ph = P.by1 - x.y; if ((P.open & 8u) == 0u && ph < h) { pbfSurf(P, ph, r, dr); rho += r; g.y -= dr; }
  ph = x.z - P.bz0; if ((P.open & 16u) == 0u && ph < h) { pbfSurf(P, ph, r, dr); rho += r; g.z += dr; }
  ph = P.bz1 - x.z; if ((P.open & 32u) == 0u && ph < h) { pbfSurf(P, ph, r, dr); rho += r; g.z -= dr; }
  for (uint32_t k = 0; k < ncols; k++) {
    float phi; V3 wn;
    sdf(k, x, phi, wn);
    if (phi >= h) continue;
    pbfSurf(P, phi, r, dr);
    rho += r;
    g = g + wn * dr;
  }
}
// collide (src/gpu.js:102-114): out of every collider by the margin, then the closed walls
template <class Sdf>
inline V3 pbfCollide(const PbfP& P, const Sdf& sdf, uint32_t ncols, V3 pin) {
  V3 p = pin;
  const float m = P.margin;
  for (uint32_t k = 0; k < ncols; k++) {
    float phi; V3 wn;
    sdf(k, p, phi, wn);
    if (phi < m) p = p + wn * (m - phi);
  }
  const float big = 1.0e9f;
  const V3 lo = v3((P.open & 1u) ? -big : P.bx0 + m, (P.open & 4u) ? -big : P.by0 + m, (P.open & 16u) ? -big : P.bz0 + m);
  const V3 hi = v3((P.open & 2u) ? big : P.bx1 - m, (P.open & 8u) ? big : P.by1 - m, (P.open & 32u) ? big : P.bz1 - m);
  return vclamp(p, lo, hi);
}
// cellOf (src/gpu.js:149-155)
inline uint32_t pbfCellOf(const PbfP& P, V3 p) {
  const int cx = std::min(std::max(i32f((p.x - P.bx0) * P.inv), 0), (int)P.nx - 1);
  const int cy = std::min(std::max(i32f((p.y - P.by0) * P.inv), 0), (int)P.ny - 1);
  const int cz = std::min(std::max(i32f((p.z - P.bz0) * P.inv), 0), (int)P.nz - 1);
  return (uint32_t)cx + P.nx * ((uint32_t)cy + P.ny * (uint32_t)cz);
}

// the uniform grid of one step: countCells + scanCells + scatter (src/gpu.js:168-206) with ascending particle index
// inside each cell. x: positions, `stride` floats apart; a particle with y < DEADY is dead (cid DEADC, in no cell).
struct PbfGrid {
  std::vector<uint32_t> cid, cstart, sorted;
};
inline void pbfBuildGrid(const PbfP& P, const float* x, size_t stride, uint32_t n, PbfGrid& G) {
  const size_t cells = (size_t)P.nx * P.ny * P.nz;
  G.cid.assign(n, 0);
  G.cstart.assign(cells + 1, 0);
  std::vector<uint32_t> count(cells, 0);
  for (uint32_t i = 0; i < n; i++) {
    const float* q = x + (size_t)i * stride;
    if (q[1] < DEADY) { G.cid[i] = PBF_DEADC; continue; }
    const uint32_t c = pbfCellOf(P, v3(q[0], q[1], q[2]));
    G.cid[i] = c;
    count[c]++;
  }
  uint32_t acc = 0;
  for (size_t c = 0; c < cells; c++) { G.cstart[c] = acc; acc += count[c]; }
  G.cstart[cells] = acc;
  G.sorted.assign(acc, 0);
  std::vector<uint32_t> cur(G.cstart.begin(), G.cstart.end() - 1);
  for (uint32_t i = 0; i < n; i++)
    if (G.cid[i] != PBF_DEADC) G.sorted[cur[G.cid[i]]++] = i;
}
// the neighbour cells' rows of particle cell c (the loops of lambda, delta and viscosity): visit(s) for every sorted slot
template <class F>
inline void pbfRows(const PbfP& P, const PbfGrid& G, uint32_t c, F&& visit) {
  const int cx = (int)(c % P.nx); const uint32_t t = c / P.nx; const int cy = (int)(t % P.ny), cz = (int)(t / P.ny);
  const uint32_t xa = (uint32_t)std::max(cx - 1, 0), xb = (uint32_t)std::min(cx + 1, (int)P.nx - 1);
  for (int z = std::max(cz - 1, 0); z <= std::min(cz + 1, (int)P.nz - 1); z++)
    for (int y = std::max(cy - 1, 0); y <= std::min(cy + 1, (int)P.ny - 1); y++) {
      const uint32_t row = P.nx * (uint32_t)(y + (int)P.ny * z);
      const uint32_t s1 = G.cstart[row + xb + 1u];
      for (uint32_t s = G.cstart[row + xa]; s < s1; s++) visit(s);
    }
}
// lambda (src/gpu.js:208-251) for particle i: its constraint multiplier and its boundary-density gradient / rho0.
// prd: predicted positions (4 floats each).
template <class Sdf>
inline void pbfLambdaOne(const PbfP& P, const Sdf& sdf, uint32_t ncols, const PbfGrid& G, const float* prd, uint32_t i, float& lam, V3& bgr) {
  const V3 qi = v3(prd[i * 4], prd[i * 4 + 1], prd[i * 4 + 2]);
  const float irho = P.irho;
  float rho = P.W0, sg = 0.0f;
  V3 g = v3(0, 0, 0);
  pbfRows(P, G, G.cid[i], [&](uint32_t s) {
    const uint32_t j = G.sorted[s];
    if (j == i) return;
    const V3 dd = qi - v3(prd[j * 4], prd[j * 4 + 1], prd[j * 4 + 2]);
    const float r2 = dot(dd, dd);
    if (r2 >= P.h2) return;
    const float tt = P.h2 - r2;
    rho += P.poly * tt * tt * tt;
    const float r = sqrtf(r2);
    if (r < 1e-7f) return;
    const float hr = P.h - r;
    const float f = P.spiky * hr * hr / r * irho;
    const V3 fv = dd * f;
    g = g + fv;
    sg += dot(fv, fv);
  });
  float br; V3 bg;
  pbfBnd(P, sdf, ncols, qi, br, bg);
  rho += br;
  bg = bg * irho;
  bgr = bg;
  g = g + bg;
  sg += dot(bg, bg);
  const float C = rho * irho - 1.0f;
  lam = C > 0.0f ? -C / (sg + dot(g, g) + P.eps) : 0.0f;
}
// delta (src/gpu.js:253-286) for particle i: the position correction, relaxed and clamped to maxD
inline V3 pbfDeltaOne(const PbfP& P, const PbfGrid& G, const float* prd, const float* lam, const float* bgr, uint32_t i) {
  const V3 qi = v3(prd[i * 4], prd[i * 4 + 1], prd[i * 4 + 2]);
  const float irho = P.irho, li = lam[i];
  V3 s = v3(bgr[i * 4], bgr[i * 4 + 1], bgr[i * 4 + 2]) * li;
  pbfRows(P, G, G.cid[i], [&](uint32_t q) {
    const uint32_t j = G.sorted[q];
    if (j == i) return;
    const float sj = li + lam[j];
    if (sj == 0.0f) return;
    const V3 dd = qi - v3(prd[j * 4], prd[j * 4 + 1], prd[j * 4 + 2]);
    const float r2 = dot(dd, dd);
    if (r2 >= P.h2) return;
    const float r = sqrtf(r2);
    if (r < 1e-7f) return;
    const float hr = P.h - r;
    s = s + dd * (P.spiky * hr * hr / r * irho * sj);
  });
  s = s * P.relax;
  const float m2 = dot(s, s);
  if (m2 > P.maxD * P.maxD) s = s * (P.maxD * (1.0f / sqrtf(m2)));
  return s;
}
// one solver iteration (lambda, delta, applyDelta: src/gpu.js:208-292) over n particles: prd moves in place;
// collide(p) is the projection applied after each correction
template <class Sdf, class Col>
inline void pbfIteration(const PbfP& P, const Sdf& sdf, uint32_t ncols, const Col& collide, const PbfGrid& G, float* prd, uint32_t n,
                         std::vector<float>& lam, std::vector<float>& bgr, std::vector<float>& dlt, int threads) {
  lam.resize(n); bgr.resize((size_t)n * 4); dlt.resize((size_t)n * 4);
#pragma omp parallel for schedule(static) num_threads(threads)
  for (int64_t ii = 0; ii < (int64_t)n; ii++) {
    const uint32_t i = (uint32_t)ii;
    if (G.cid[i] == PBF_DEADC) continue;
    V3 bg;
    pbfLambdaOne(P, sdf, ncols, G, prd, i, lam[i], bg);
    bgr[i * 4] = bg.x; bgr[i * 4 + 1] = bg.y; bgr[i * 4 + 2] = bg.z; bgr[i * 4 + 3] = 0.0f;
  }
#pragma omp parallel for schedule(static) num_threads(threads)
  for (int64_t ii = 0; ii < (int64_t)n; ii++) {
    const uint32_t i = (uint32_t)ii;
    if (G.cid[i] == PBF_DEADC) continue;
    const V3 s = pbfDeltaOne(P, G, prd, lam.data(), bgr.data(), i);
    dlt[i * 4] = s.x; dlt[i * 4 + 1] = s.y; dlt[i * 4 + 2] = s.z;
  }
#pragma omp parallel for schedule(static) num_threads(threads)
  for (int64_t ii = 0; ii < (int64_t)n; ii++) {
    const uint32_t i = (uint32_t)ii;
    if (G.cid[i] == PBF_DEADC) continue;
    const V3 q = collide(v3(prd[i * 4], prd[i * 4 + 1], prd[i * 4 + 2]) + v3(dlt[i * 4], dlt[i * 4 + 1], dlt[i * 4 + 2]));
    prd[i * 4] = q.x; prd[i * 4 + 1] = q.y; prd[i * 4 + 2] = q.z; prd[i * 4 + 3] = 0.0f;
  }
}
#endif
