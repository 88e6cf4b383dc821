// flip_oracle.cpp - CPU restatement of SplashTank's FLIP step, used ONLY as the parity checker and as the
// timed CPU baseline. It is test infrastructure: the product (splashtank_b200) never links or calls it.
//
// It restates the WGSL kernels of src/flip/wgsl-{core,blocks,solver,narrowband,whitewater}.js and the host
// logic of src/flip/sim.js:179-310 kernel by kernel, in the reference's stage order, with the reference's
// numerics (f32, fixed-point P2G at scale 65536, red-black SOR in place, 16-bit depth field).
// Every function cites the reference file:line it follows.
//
// Parity status: the reference runs only as WGSL in a browser (WebGPU); it has no CPU FLIP code and its tests
// hold no golden vectors for the step. This restatement is therefore "parity unpinned" against the reference
// itself: it is pinned by reading, by the invariant tests in tests/ and by the golden fixtures it generated.
//
// Storage: a dense tile box ((tx*8) x (ty*8) x (tz*8) cells, 512 per tile, x fastest inside a tile) plus one
// spare block at index ntiles, which plays the reference's spare slot 0: every read of a cell whose tile has
// no storage lands there (wgsl-core.js:79-83). Order-dependent parts of the reference (atomic compaction) use
// a canonical order here, the same the CUDA path uses:
//   * particles are stored sorted by (cell key, id) each step, dead ones after them in their previous order;
//   * narrow-band refill: deficit cells in ascending cell key, dead slots in ascending storage index;
//   * whitewater emission: ring slots handed out in ascending storage index of the emitting particle.
// Build with -ffp-contract=off (no FMA) so float results are bit-reproducible.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/splashtank_cuda.h"
#include "../include/st_math.h"
#include "oracle_math.h"
#include "pbf_core.h"

namespace {

const uint32_t NONE = 0xffffffffu;
const float WWHOLD = 0.2f;

// hash1 (wgsl-solver.js:181-184)
inline float hash1(uint32_t n0) {
  uint32_t x = n0; x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
  return (float)x * 2.3283064e-10f;
}

// The parameter block, f32 words as packed by sim.js:196-231 (wgsl-core.js:3-20).
struct Params {
  uint32_t n, nx, ny, nz, ncols, open, ncell;
  float dt, h, ih, gravity, flip, rest, comp, omega;
  float x0, y0, z0, vmax, margin, scale, x1, y1, z1;
  float q0, q1, q2, q3, q4, q5, q6, q7, q8, q9, q10, q11, q12;
  uint32_t lcap, tx, ty, tz, scap;
  float sheetMin, sprRate, sprMin, sprLife, mistFrac, sprDrag, mistDrag, vs;
  uint32_t smax, seed;
  uint32_t nb; float band; uint32_t nbInit, nfill;
  float wwFoamLife, wwRise, wwCrest, wwImpact;
  uint32_t airOn, aNx, aNy, aNz; float airCouple, airDecay, airH, airBlur;   // words 72-76, 82
  uint32_t ndrip; float dripRate, dripDry;                                    // words 79-81
  uint32_t ocean, nwave; float otime, olevel, olayer, oy0, odepth;            // words 57-61, 63, 66
  uint32_t nfv;                                                               // word 67: fill volumes after the colliders
  float waves[24 * 8];                                                        // oceanWaves: 8 floats per wave
  float fills[16][4];
};

struct Oracle {
  // fixed at create (sim.js:47-61)
  double d, ratio, h, rest;
  int nx, ny, nz, tx, ty, tz, ntiles;
  double bx0, bx1, by0, by1, bz0, bz1;
  uint32_t open, maxN, cap, N = 0, ring = 0, sprayCap;
  bool recycle = true;
  // particles in storage order: pos/vel 4 floats, id
  std::vector<float> pos, vel;
  std::vector<uint32_t> pid;
  // tiles and cells ((ntiles + 1) * 512: spare block last)
  std::vector<uint8_t> alloc, need;
  std::vector<int32_t> cnt, accV, accW;   // acc: 3 per cell (x, y, z lower faces)
  std::vector<uint32_t> ctype;
  std::vector<float> pres, rhs, velG;
  std::vector<uint32_t> active;           // tiles with storage, ascending
  // colliders (packColliders, gpu.js:42-70): 32 floats each, sdf grids back to back
  std::vector<float> cols, sdf;
  uint32_t ncols = 0;
  std::string sdfSig;
  // whitewater (sim.js:71, 333-341)
  std::vector<float> sPos, sVel, sAux;
  uint32_t sctl0 = 0;
  // air field (sim.js:342-350): 4 floats per air cell (air, air2), 4 fixed-point sums (airAcc)
  std::vector<float> air, air2;
  std::vector<int32_t> airAcc;
  uint32_t aNx = 0, aNy = 0, aNz = 0, airCells = 0;
  double airH = 1.0;
  // drip samples (sim.js:352-363): 8 floats each (local position, collider, local normal, wetness)
  std::vector<float> drip;
  uint32_t ndrip = 0;
  std::string dripSig;
  // narrow band state (sim.js:92, 120-126)
  bool velGOn = false;
  uint32_t nbInit = 0;
  std::vector<float> fillsPacked;  // 8 floats per fill
  // water-mesh fill volumes of the next restart (sim.nbFillVols, src/shared.js:849-850): records with owned grids
  struct FillVol { st_sdf sd; std::vector<float> data; st_collider c; };
  std::vector<FillVol> fillVols;
  uint32_t nfv = 0;
  // time and seed (sim.js:200, 207)
  double tm = 0;
  uint32_t seed = 0, steps = 0;
  // the live view's state (sim.js:80, 184, 406): deep look, the last step's particle count and narrow band, and
  // how many deep cells the previous deep pass saw (ctl[12])
  bool deepOn = false, lastNb = false;
  uint32_t lastN = 0, deepPrev = 0;
  // stats
  uint32_t st_sc = 0, st_fluid = 0, st_ovf = 0, spray_ovf = 0, st_live = 0;
  float st_vmax = 0;
  Params P;
  int nthreads = 1;

  uint32_t spare() const { return (uint32_t)ntiles; }
  // ---- addressing (wgsl-core.js:76-135) ----
  uint32_t tileOf(int i, int j, int k) const { return (uint32_t)(i >> 3) + P.tx * ((uint32_t)(j >> 3) + P.ty * (uint32_t)(k >> 3)); }
  uint32_t cellIdx(int i, int j, int k) const {
    uint32_t t = tileOf(i, j, k);
    uint32_t s = alloc[t] ? t : spare();
    return s * 512u + (uint32_t)(i & 7) + 8u * ((uint32_t)(j & 7) + 8u * (uint32_t)(k & 7));
  }
  uint32_t faceIndex(int axis, int i, int j, int k) const {
    int nx_ = (int)P.nx, ny_ = (int)P.ny, nz_ = (int)P.nz;
    auto cl = [](int v, int lo, int hi) { return std::min(std::max(v, lo), hi); };
    if (axis == 0) return cellIdx(cl(i, 0, nx_), cl(j, 0, ny_ - 1), cl(k, 0, nz_ - 1)) * 3u;
    if (axis == 1) return cellIdx(cl(i, 0, nx_ - 1), cl(j, 0, ny_), cl(k, 0, nz_ - 1)) * 3u + 1u;
    return cellIdx(cl(i, 0, nx_ - 1), cl(j, 0, ny_ - 1), cl(k, 0, nz_)) * 3u + 2u;
  }
  void tileCoord(uint32_t t, uint32_t local, int& i, int& j, int& k) const {
    uint32_t tt = t / P.tx;
    i = (int)((t % P.tx) * 8u + (local & 7u)); j = (int)((tt % P.ty) * 8u + ((local >> 3) & 7u)); k = (int)((tt / P.ty) * 8u + (local >> 6));
  }
  uint32_t ctypeOf(int i, int j, int k) const {
    if (i < 0) return (P.open & 1u) ? 0u : 2u;
    if (i >= (int)P.nx) return (P.open & 2u) ? 0u : 2u;
    if (j < 0) return (P.open & 4u) ? 0u : 2u;
    if (j >= (int)P.ny) return (P.open & 8u) ? 0u : 2u;
    if (k < 0) return (P.open & 16u) ? 0u : 2u;
    if (k >= (int)P.nz) return (P.open & 32u) ? 0u : 2u;
    return ctype[cellIdx(i, j, k)] & 0xffu;
  }
  bool inDom(int i, int j, int k) const { return i >= 0 && j >= 0 && k >= 0 && i < (int)P.nx && j < (int)P.ny && k < (int)P.nz; }
  V3 cellCenter(int i, int j, int k) const {
    return v3(P.x0 + ((float)i + 0.5f) * P.h, P.y0 + ((float)j + 0.5f) * P.h, P.z0 + ((float)k + 0.5f) * P.h);
  }
  void particleCell(V3 p, int& ci, int& cj, int& ck) const {
    V3 g = vfloor((p - v3(P.x0, P.y0, P.z0)) * P.ih);
    ci = std::min(std::max((int)g.x, 0), (int)P.nx - 1);
    cj = std::min(std::max((int)g.y, 0), (int)P.ny - 1);
    ck = std::min(std::max((int)g.z, 0), (int)P.nz - 1);
  }
  bool hasStorage(int i, int j, int k) const { return alloc[tileOf(i, j, k)] != 0; }
  float gvR(uint32_t f) const { return bitsf(accV[f]); }
  float gv0R(uint32_t f) const { return bitsf(accW[f]); }

  // ---- colliders (gpu.js:6-38, wgsl-core.js:113-131) ----
  const float* col(uint32_t k, int m) const { return &cols[(size_t)k * 32 + (size_t)m * 4]; }
  void sdfEval(uint32_t k, V3 p, float& phi, V3& wn) const { sdfEvalRec(cols.data(), sdf.data(), k, p, phi, wn); }
  V3 colSurfVel(uint32_t k, V3 p) const {
    V3 c = v3(col(k, 5)[0], col(k, 5)[1], col(k, 5)[2]);
    return v3(col(k, 6)[0], col(k, 6)[1], col(k, 6)[2]) + cross(v3(col(k, 7)[0], col(k, 7)[1], col(k, 7)[2]), p - c);
  }
  bool colNear(uint32_t k, V3 p) const {
    if (P.q10 > 0.5f) return true;
    const float* b = col(k, 1);
    V3 d_ = p - v3(col(k, 5)[0], col(k, 5)[1], col(k, 5)[2]);
    V3 lp = v3(dot(v3(col(k, 2)[0], col(k, 2)[1], col(k, 2)[2]), d_), dot(v3(col(k, 3)[0], col(k, 3)[1], col(k, 3)[2]), d_),
               dot(v3(col(k, 4)[0], col(k, 4)[1], col(k, 4)[2]), d_));
    V3 g = (lp - v3(b[0], b[1], b[2])) / b[3];
    V3 dims = v3(col(k, 0)[1], col(k, 0)[2], col(k, 0)[3]);
    float lo = -1.0f - P.q0 / b[3], hi = P.q0 / b[3];
    return g.x > lo && g.y > lo && g.z > lo && g.x < dims.x + hi && g.y < dims.y + hi && g.z < dims.z + hi;
  }
  int colAt(V3 p) const {
    for (uint32_t k = 0; k < P.ncols; k++) {
      if (!colNear(k, p)) continue;
      float phi; V3 wn; sdfEval(k, p, phi, wn);
      if (phi < P.q0) return (int)k;
    }
    return -1;
  }
  int colAtCell(int i, int j, int k) const {
    if (!inDom(i, j, k)) return -1;
    return (int)((ctype[cellIdx(i, j, k)] >> 8) & 0xffu) - 1;
  }

  // ---- narrow band helpers (wgsl-core.js:160-200, 228-238) ----
  uint32_t colBits(uint32_t c) const { return (ctype[c] >> 8) & 0xffu; }
  float phiOf(uint32_t c) const { return 8.0f - (float)(ctype[c] >> 16) / 4096.0f; }
  void phiPut(uint32_t c, float v) {
    uint32_t q = (uint32_t)clampf(rintf((8.0f - v) * 4096.0f), 0.0f, 65535.0f);
    ctype[c] = (ctype[c] & 0xffffu) | (q << 16);
  }
  V3 facePos(int i, int j, int k, int axis) const {
    return v3(P.x0 + ((float)i + (axis == 0 ? 0.0f : 0.5f)) * P.h, P.y0 + ((float)j + (axis == 1 ? 0.0f : 0.5f)) * P.h,
              P.z0 + ((float)k + (axis == 2 ? 0.0f : 0.5f)) * P.h);
  }
  float phiSample(V3 x) const {
    V3 g = (x - v3(P.x0, P.y0, P.z0)) * P.ih - v3(0.5f, 0.5f, 0.5f);
    V3 gc = vclamp(g, v3(0, 0, 0), v3((float)P.nx - 1.001f, (float)P.ny - 1.001f, (float)P.nz - 1.001f));
    V3 f0 = vfloor(gc); V3 fr = gc - f0; int i0 = (int)f0.x, j0 = (int)f0.y, k0 = (int)f0.z;
    float s = 0.0f, ws = 0.0f;
    for (int c = 0; c < 8; c++) {
      int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
      float w = (dx == 1 ? fr.x : 1.0f - fr.x) * (dy == 1 ? fr.y : 1.0f - fr.y) * (dz == 1 ? fr.z : 1.0f - fr.z);
      uint32_t ci = cellIdx(i0 + dx, j0 + dy, k0 + dz);
      if (colBits(ci) != 0u || w <= 0.0f) continue;
      s += w * phiOf(ci); ws += w;
    }
    if (ws < 1.0e-4f) return 0.5f;
    return s / ws;
  }
  float velGAxis(V3 x, int axis) const {
    V3 g = (x - v3(P.x0, P.y0, P.z0)) * P.ih;
    if (axis == 0) { g.y -= 0.5f; g.z -= 0.5f; } else if (axis == 1) { g.x -= 0.5f; g.z -= 0.5f; } else { g.x -= 0.5f; g.y -= 0.5f; }
    V3 f0 = vfloor(g); V3 fr = g - f0; int i0 = (int)f0.x, j0 = (int)f0.y, k0 = (int)f0.z;
    float s = 0.0f;
    for (int c = 0; c < 8; c++) {
      int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
      float w = (dx == 1 ? fr.x : 1.0f - fr.x) * (dy == 1 ? fr.y : 1.0f - fr.y) * (dz == 1 ? fr.z : 1.0f - fr.z);
      s += w * velG[faceIndex(axis, i0 + dx, j0 + dy, k0 + dz)];
    }
    return s;
  }
  V3 velGVec(V3 x) const { return v3(velGAxis(x, 0), velGAxis(x, 1), velGAxis(x, 2)); }
  bool calmV(V3 v) const { return length(v) < 9.0f * P.h; }
  // ---- ocean (wgsl-core.js:201-226) ----
  float oceanEta(float x, float z) const {
    float e = 0.0f;
    for (uint32_t k = 0; k < P.nwave; k++) {
      const float* A = &P.waves[k * 8]; const float* Bw = A + 4;
      float sn, cs; st_sincosf(A[0] * x + A[1] * z - A[3] * P.otime + Bw[0], &sn, &cs);
      e += A[2] * cs;
    }
    return P.olevel + e;
  }
  V3 oceanVel(V3 p) const {
    float D = fmax_(P.odepth, 1.0e-3f), eta = oceanEta(p.x, p.z);
    float ys = clampf((p.y - P.oy0) * D / fmax_(D + eta - P.olevel, 0.1f * D), 0.0f, D);
    V3 v = v3(0, 0, 0);
    for (uint32_t k = 0; k < P.nwave; k++) {
      const float* A = &P.waves[k * 8]; const float* Bw = A + 4;
      float kk = fmax_(Bw[1], 1.0e-4f);
      float th = A[0] * p.x + A[1] * p.z - A[3] * P.otime + Bw[0];
      float e1 = st_expf(kk * (ys - D)), e2 = st_expf(-kk * (ys + D)), dn = fmax_(1.0f - st_expf(-2.0f * kk * D), 1.0e-4f);
      float aw = A[2] * A[3];
      float sn, cs; st_sincosf(th, &sn, &cs);
      float hc = aw * (e1 + e2) / dn * cs / kk;
      v = v + v3(hc * A[0], aw * (e1 - e2) / dn * sn, hc * A[1]);
    }
    return v;
  }
  float layerW(V3 p) const {
    if (P.ocean == 0u) return 0.0f;
    float dw = fmin_(fmin_(p.x - P.x0, P.x1 - p.x), fmin_(p.z - P.z0, P.z1 - p.z));
    return clampf(1.0f - dw / fmax_(P.olayer, 1.0e-4f), 0.0f, 1.0f);
  }
  float fillPhi(V3 x) const {
    float dd = 1.0e9f;
    for (uint32_t k = 0; k < P.nfill; k++) {
      const float* A = P.fills[k * 2]; const float* B = P.fills[k * 2 + 1];
      if (A[0] < 1.5f) {
        V3 q = vmax(v3(A[1], A[2], A[3]) - x, x - v3(B[0], B[1], B[2]));
        dd = fmin_(dd, length(vmax(q, v3(0, 0, 0))) + fmin_(fmax_(q.x, fmax_(q.y, q.z)), 0.0f));
      } else {
        dd = fmin_(dd, length(x - v3(A[1], A[2], A[3])) - B[0]);
      }
    }
    for (uint32_t k = P.ncols; k < P.ncols + P.nfv; k++) { float phi; V3 wn; sdfEval(k, x, phi, wn); dd = fmin_(dd, phi); }
    if (P.ocean != 0u) dd = fmin_(dd, x.y - oceanEta(x.x, x.z));
    return dd * P.ih;
  }
  // markAround (wgsl-core.js:239-246)
  void markAround(int ci, int cj, int ck) {
    int lox = std::max(ci - 2, 0) >> 3, loy = std::max(cj - 2, 0) >> 3, loz = std::max(ck - 2, 0) >> 3;
    int hix = std::min(ci + 2, (int)P.tx * 8 - 1) >> 3, hiy = std::min(cj + 2, (int)P.ty * 8 - 1) >> 3, hiz = std::min(ck + 2, (int)P.tz * 8 - 1) >> 3;
    for (int tk = loz; tk <= hiz; tk++) for (int tj = loy; tj <= hiy; tj++) for (int ti = lox; ti <= hix; ti++)
      need[(uint32_t)ti + P.tx * ((uint32_t)tj + P.ty * (uint32_t)tk)] = 1;
  }
  V3 ppos(uint32_t i) const { return v3(pos[i * 4], pos[i * 4 + 1], pos[i * 4 + 2]); }
  V3 pvel(uint32_t i) const { return v3(vel[i * 4], vel[i * 4 + 1], vel[i * 4 + 2]); }
  template <class F> void forActive(F fn) {
    const int64_t nc = (int64_t)active.size() * 512;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t t = 0; t < nc; t++) {
      uint32_t tile = active[(size_t)(t >> 9)], local = (uint32_t)(t & 511);
      int i, j, k; tileCoord(tile, local, i, j, k);
      fn(tile * 512u + local, i, j, k);
    }
  }
  template <class F> void forParticles(F fn) {
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t i = 0; i < (int64_t)P.n; i++) fn((uint32_t)i);
  }

  // ---- create (sim.js:47-98) ----
  void create(const st_flip_desc* dsc) {
    d = dsc->d;
    double r = dsc->ratio != 0 ? dsc->ratio : 2.0;
    ratio = std::max(1.4, std::min(4.0, r));
    h = ratio * d; rest = ratio * ratio * ratio;
    double sz[3] = {3, 2.6, 3};
    if (dsc->box[0] > 0 && dsc->box[1] > 0 && dsc->box[2] > 0) { sz[0] = dsc->box[0]; sz[1] = dsc->box[1]; sz[2] = dsc->box[2]; }
    nx = std::max(4, (int)std::floor(sz[0] / h + 0.5)); ny = std::max(4, (int)std::floor(sz[1] / h + 0.5)); nz = std::max(4, (int)std::floor(sz[2] / h + 0.5));
    double W = nx * h, H = ny * h, D = nz * h;
    bx0 = -W / 2; bx1 = W / 2; by0 = 0; by1 = H; bz0 = -D / 2; bz1 = D / 2;
    open = dsc->open; maxN = dsc->max_n; cap = maxN; sprayCap = dsc->spray_cap;
    tx = (nx + 1 + 7) / 8; ty = (ny + 1 + 7) / 8; tz = (nz + 1 + 7) / 8; ntiles = tx * ty * tz;
    pos.assign((size_t)maxN * 4, 0.0f); vel.assign((size_t)maxN * 4, 0.0f); pid.resize(maxN);
    for (uint32_t k = 0; k < maxN; k++) pid[k] = k;
    size_t ncell = (size_t)(ntiles + 1) * 512;
    alloc.assign(ntiles, 0); need.assign(ntiles, 0);
    cnt.assign(ncell, 0); ctype.assign(ncell, 0); pres.assign(ncell, 0.0f); rhs.assign(ncell, 0.0f);
    accV.assign(ncell * 3, 0); accW.assign(ncell * 3, 0); velG.assign(ncell * 3, 0.0f);
    sPos.assign((size_t)std::max(sprayCap, 1u) * 4, 0.0f); sVel = sPos; sAux = sPos;
    if (sprayCap) {   // airAlloc (sim.js:343-350), made up front: it stays zero until the air field is first on
      int r = std::max(2, (int)std::ceil(std::cbrt((double)nx * ny * nz / 260000.0)));
      airH = h * r;
      aNx = (uint32_t)((nx + r - 1) / r + 1); aNy = (uint32_t)((ny + r - 1) / r + 1); aNz = (uint32_t)((nz + r - 1) / r + 1);
      airCells = aNx * aNy * aNz;
      air.assign((size_t)airCells * 4, 0.0f); air2 = air; airAcc.assign((size_t)airCells * 4, 0);
    }
    memset(&P, 0, sizeof(P));
    P.tx = tx; P.ty = ty; P.tz = tz; P.nx = nx; P.ny = ny; P.nz = nz;
  }
  // FlipSim.clear (sim.js:539-547, gpu.js:389)
  void clear() {
    N = 0; ring = 0; tm = 0; nbInit = 1; fillsPacked.clear(); fillVols.clear();
    std::fill(sPos.begin(), sPos.end(), 0.0f); sctl0 = 0;
    std::fill(air.begin(), air.end(), 0.0f);
    dripSig.clear();   // drip samples come back dry
    for (uint32_t k = 0; k < maxN; k++) pid[k] = k;
    steps = 0;
  }
  // FlipSim.add (gpu.js:390-402)
  bool add(float x, float y, float z, float vx, float vy, float vz) {
    uint32_t i;
    if (N < cap) i = N++;
    else if (recycle) { i = ring++; if (ring >= cap) ring = 0; }
    else return false;
    pos[i * 4] = x; pos[i * 4 + 1] = y; pos[i * 4 + 2] = z;
    pos[i * 4 + 3] = (float)std::sqrt((double)vx * vx + (double)vy * vy + (double)vz * vz);
    vel[i * 4] = vx; vel[i * 4 + 1] = vy; vel[i * 4 + 2] = vz; vel[i * 4 + 3] = 0.0f;
    return true;
  }
  // packColliders (gpu.js:42-70)
  void packCols(const st_step_opts* o) {
    uint32_t nc = std::min(o->ncols, 32u);
    std::string sig; std::map<uint32_t, uint32_t> offs; uint32_t off = 0;
    for (uint32_t k = 0; k < nc; k++) {
      const st_sdf* sd = o->cols[k].sdf;
      if (!offs.count(sd->id)) { offs[sd->id] = off; off += sd->dims[0] * sd->dims[1] * sd->dims[2]; sig += std::to_string(sd->id) + ","; }
    }
    if (sig != sdfSig) {
      sdf.assign(std::max(off, 16u), 0.0f);
      std::map<uint32_t, bool> seen;
      for (uint32_t k = 0; k < nc; k++) {
        const st_sdf* sd = o->cols[k].sdf;
        if (seen[sd->id]) continue;
        seen[sd->id] = true;
        memcpy(&sdf[offs[sd->id]], sd->data, sizeof(float) * sd->dims[0] * sd->dims[1] * sd->dims[2]);
      }
      sdfSig = sig;
    }
    cols.assign((size_t)std::max(nc, 1u) * 32, 0.0f);
    for (uint32_t k = 0; k < nc; k++) {
      const st_collider& c = o->cols[k]; const st_sdf* sd = c.sdf; float* cf = &cols[k * 32];
      cf[0] = (float)offs[sd->id]; cf[1] = (float)sd->dims[0]; cf[2] = (float)sd->dims[1]; cf[3] = (float)sd->dims[2];
      cf[4] = sd->origin[0]; cf[5] = sd->origin[1]; cf[6] = sd->origin[2]; cf[7] = sd->cell;
      cf[8] = c.R[0]; cf[9] = c.R[3]; cf[10] = c.R[6]; cf[11] = 0;
      cf[12] = c.R[1]; cf[13] = c.R[4]; cf[14] = c.R[7]; cf[15] = 0;
      cf[16] = c.R[2]; cf[17] = c.R[5]; cf[18] = c.R[8]; cf[19] = 0;
      cf[20] = c.pos[0]; cf[21] = c.pos[1]; cf[22] = c.pos[2]; cf[23] = 0;
      cf[24] = c.vel[0]; cf[25] = c.vel[1]; cf[26] = c.vel[2]; cf[27] = 0;
      cf[28] = c.ang[0]; cf[29] = c.ang[1]; cf[30] = c.ang[2]; cf[31] = 0;
    }
    ncols = nc;
  }
  double omegaAuto() const { return std::min(1.9, 2.0 / (1.0 + std::sin(M_PI / std::max(nx, std::max(ny, nz))))); }

  // ---- parameter block (sim.js:196-231) ----
  void packParams(double dt, const st_step_opts* o, uint32_t init, bool nbOn, bool sprOn) {
    P.n = N; P.nx = nx; P.ny = ny; P.nz = nz; P.ncols = ncols; P.open = open; P.ncell = (uint32_t)(nx * ny * nz);
    P.dt = (float)dt; P.h = (float)h; P.ih = (float)(1.0 / h); P.gravity = o->g; P.flip = o->flip; P.rest = (float)rest; P.comp = o->comp;
    P.omega = o->omega != 0.0f ? o->omega : (float)omegaAuto();
    P.x0 = (float)bx0; P.y0 = (float)by0; P.z0 = (float)bz0; P.vmax = o->vmax != 0.0f ? o->vmax : 14.0f; P.margin = (float)(0.3 * d); P.scale = 65536.0f;
    P.x1 = (float)bx1; P.y1 = (float)by1; P.z1 = (float)bz1; P.q0 = (float)(0.3 * h);
    P.q1 = o->wind[0]; P.q2 = o->wind[1]; P.q3 = o->wind[2]; P.q4 = o->drag; P.q5 = o->foam_tau != 0.0f ? o->foam_tau : 1.2f;
    P.q6 = o->foam_sens != 0.0f ? o->foam_sens : 1.0f; P.q7 = o->gust; P.q8 = (float)tm;
    P.q9 = (o->flags & ST_OPT_NO_FOAM) ? 1.0f : 0.0f; P.q10 = (o->flags & ST_OPT_NO_CULL) ? 1.0f : 0.0f; P.q11 = 1.0f;
    P.q12 = (o->flags & ST_OPT_FAST_AIR) ? 1.0f : 0.0f;
    uint64_t pool = (uint64_t)(ntiles + 1) * 512;
    P.lcap = velGOn ? (uint32_t)pool : (uint32_t)std::min<uint64_t>(pool, maxN);
    P.tx = tx; P.ty = ty; P.tz = tz; P.scap = (uint32_t)(ntiles + 1);
    const st_spray_opts& sp = o->spray;
    P.sheetMin = o->tear; P.sprRate = sprOn ? sp.rate : 0.0f; P.sprMin = sprOn ? std::max(0.05f, sp.min) : 1.0f; P.sprLife = sprOn ? sp.life : 1.0f;
    P.mistFrac = sprOn ? sp.mist : 0.0f; P.sprDrag = sprOn ? sp.drag : 1.0f; P.mistDrag = sprOn ? sp.mdrag : 4.0f; P.vs = o->vs != 0.0f ? o->vs : 1.0f;
    P.smax = sprayCap; P.seed = seed;
    P.nb = nbOn ? 1u : 0u; P.band = std::max(2.0f, o->nb_band != 0.0f ? o->nb_band : 3.0f); P.nbInit = init;
    uint32_t nf = init ? (uint32_t)std::min<size_t>(fillsPacked.size() / 8, 8) : 0u; P.nfill = nf; P.nfv = nfv;
    memset(P.fills, 0, sizeof(P.fills));
    for (uint32_t k = 0; k < nf; k++) memcpy(P.fills[k * 2], &fillsPacked[k * 8], 8 * sizeof(float));
    P.wwFoamLife = sp.foam_life != 0.0f ? sp.foam_life : 3.0f; P.wwRise = sp.rise != 0.0f ? sp.rise : 0.3f;
    P.wwCrest = sp.crest; P.wwImpact = sp.impact;
    bool airo = sprOn && o->air_on != 0 && airCells != 0;   // sim.js:222-229
    P.airOn = airo ? 1u : 0u; P.airCouple = airo ? o->air_couple : 0.0f; P.airDecay = airo ? o->air_decay : 0.0f;
    P.airH = airCells ? (float)airH : 1.0f; P.airBlur = airo ? o->air_blur : 0.0f;
    P.aNx = airCells ? aNx : 1u; P.aNy = airCells ? aNy : 1u; P.aNz = airCells ? aNz : 1u;
    // ocean (sim.js:210-218; oceanWaves, shared.js:760-780)
    bool oc = o->ocean_on != 0;
    P.ocean = oc ? 1u : 0u; P.otime = o->time; P.olevel = oc ? o->ocean_level : 0.0f; P.olayer = oc ? o->ocean_layer : 0.0f;
    P.oy0 = (float)by0; P.odepth = oc ? (float)std::max((double)o->ocean_level - by0, 1e-3) : 1.0f;
    P.nwave = oc ? oceanWaves(o, (double)o->g, (double)o->ocean_level - by0, P.waves) : 0u;
    bool dr = sprOn && o->drip_on != 0;
    P.ndrip = dr ? ndrip : 0u; P.dripRate = dr ? o->drip_rate : 0.0f; P.dripDry = dr ? o->drip_dry : 1.0f;
  }

  // oceanWaves (shared.js:760-780): mulberry32 draws, Pierson-Moskowitz amplitudes, dispersion by fixed-point iteration
  static uint32_t oceanWaves(const st_step_opts* o, double g, double depth, float* w) {
    auto toI32 = [](double x) -> int32_t {
      if (!std::isfinite(x)) return 0;
      double m = std::fmod(std::trunc(x), 4294967296.0); if (m < 0) m += 4294967296.0;
      return (int32_t)(uint32_t)m;
    };
    int32_t sd = toI32((double)o->ocean_seed); if (sd == 0) sd = 1;
    uint32_t a = (uint32_t)toI32((double)sd * 7919.0 + 13.0);
    auto rnd = [&]() {
      a += 0x6D2B79F5u;
      uint32_t t = (a ^ (a >> 15)) * (1u | a);
      t = (t + (t ^ (t >> 7)) * (61u | t)) ^ t;
      return (double)(t ^ (t >> 14)) / 4294967296.0;
    };
    const int N = 24; const double PI = 3.141592653589793;
    double D = std::max(depth, 1e-3), G = std::max(g, 1e-4), lp = std::max((double)o->ocean_length, 1e-3);
    double kp = 2 * PI / lp, wp = std::sqrt(G * kp * std::tanh(kp * D));
    auto kOf = [&](double om) { double k = om * om / G; for (int i = 0; i < 40; i++) k = om * om / (G * std::tanh(std::max(k * D, 1e-6))); return k; };
    double dir = o->ocean_dir == o->ocean_dir ? o->ocean_dir : 0.0, sp = o->ocean_spread == o->ocean_spread ? o->ocean_spread : 0.0;
    double th0 = dir * PI / 180, spr = std::max(0.0, sp) * PI / 180;
    double K[N], OM[N], S[N], TH[N], PH[N], sum = 0;
    for (int i = 0; i < N; i++) {
      double r = 0.6 + 1.6 * (i + rnd()) / N;
      OM[i] = r * wp; K[i] = kOf(OM[i]); S[i] = std::pow(r, -5) * std::exp(-1.25 * std::pow(r, -4));
      double r1 = rnd(), r2 = rnd(), r3 = rnd();
      TH[i] = th0 + spr * (r1 + r2 + r3 - 1.5) / 1.5; PH[i] = rnd() * 2 * PI; sum += S[i];
    }
    double hs = o->ocean_height == o->ocean_height ? o->ocean_height : 0.0, m0 = std::pow(std::max(hs, 0.0) / 4, 2);
    for (int i = 0; i < N; i++) {
      double amp = std::min(std::sqrt(2 * m0 * S[i] / sum), 0.3 / K[i]);
      double rec[8] = {K[i] * std::cos(TH[i]), K[i] * std::sin(TH[i]), amp, OM[i], PH[i], K[i], 0, 0};
      for (int q = 0; q < 8; q++) w[i * 8 + q] = (float)rec[q];
    }
    return N;
  }

  // ---- drip samples (dripSamples, bake.js:19-40, in JavaScript doubles; dripUpdate, sim.js:352-363) ----
  static double jsRound(double x) { double r = std::floor(x); return x - r >= 0.5 ? r + 1.0 : r; }
  void dripSamplesOf(const st_sdf* sd, uint32_t k, std::vector<float>& out) const {
    int sx = (int)sd->dims[0], sy = (int)sd->dims[1], sz = (int)sd->dims[2];
    double c = sd->cell;
    auto D = [&](int i, int j, int q) { return (double)sd->data[(size_t)i + (size_t)sx * ((size_t)j + (size_t)sy * (size_t)q)]; };
    auto at = [&](int i, int j, int q) { return D(std::min(sx - 1, std::max(0, i)), std::min(sy - 1, std::max(0, j)), std::min(sz - 1, std::max(0, q))); };
    std::vector<double> pts;
    for (int q = 1; q < sz - 1; q++) for (int j = 1; j < sy - 1; j++) for (int i = 1; i < sx - 1; i++) {
      double v = D(i, j, q);
      if (std::fabs(v) > 0.6 * c) continue;
      double gx = at(i + 1, j, q) - at(i - 1, j, q), gy = at(i, j + 1, q) - at(i, j - 1, q), gz = at(i, j, q + 1) - at(i, j, q - 1);
      double gl = std::sqrt(gx * gx + gy * gy + gz * gz);   // Math.hypot
      if (gl < 1e-9) continue;
      gx /= gl; gy /= gl; gz /= gl;
      double rec[6] = {(double)sd->origin[0] + i * c - gx * v, (double)sd->origin[1] + j * c - gy * v, (double)sd->origin[2] + q * c - gz * v, gx, gy, gz};
      pts.insert(pts.end(), rec, rec + 6);
    }
    double nsurf = (double)(pts.size() / 6);
    double want = std::max(100.0, std::min(6000.0, jsRound(nsurf * c * c / (h * h))));
    double step = std::max(1.0, nsurf / want);
    double seedv = 7.0 + (double)(int32_t)sd->id;
    auto rnd = [&]() { seedv = std::fmod(seedv * 16807.0, 2147483647.0); return seedv / 2147483647.0; };
    for (double t = rnd() * step; t < nsurf; t += step) {
      size_t i = (size_t)std::floor(t) * 6;
      float rec[8] = {(float)pts[i], (float)pts[i + 1], (float)pts[i + 2], (float)k, (float)pts[i + 3], (float)pts[i + 4], (float)pts[i + 5], 0.0f};
      out.insert(out.end(), rec, rec + 8);
    }
  }
  void dripUpdate(const st_step_opts* o, uint32_t nc) {
    std::string sig;
    for (uint32_t k = 0; k < nc; k++) sig += std::to_string(o->cols[k].sdf->id) + ",";
    if (sig == dripSig) return;
    dripSig = sig;
    drip.clear();
    for (uint32_t k = 0; k < nc; k++) dripSamplesOf(o->cols[k].sdf, k, drip);
    ndrip = (uint32_t)(drip.size() / 8);
  }

  // ---- blocks (wgsl-blocks.js:5-55, wgsl-narrowband.js:6-18, sim.js:253-261) ----
  void stageBlocks(bool nb, uint32_t init) {
    std::fill(need.begin(), need.end(), 0);
    for (uint32_t i = 0; i < P.n; i++) {              // tileMark
      if (pos[i * 4 + 1] < DEADY) continue;
      int ci, cj, ck; particleCell(ppos(i), ci, cj, ck); markAround(ci, cj, ck);
    }
    if (nb && init != 1) {                             // tileMarkPhi: last step's blocks holding water by depth
      for (uint32_t tile : active) for (uint32_t local = 0; local < 512; local++) {
        int i, j, k; tileCoord(tile, local, i, j, k);
        if (!inDom(i, j, k) || phiOf(tile * 512 + local) >= 0.5f) continue;
        markAround(i, j, k);
      }
    }
    if (init) {                                        // tileMarkFill
      for (uint32_t t = 0; t < (uint32_t)ntiles; t++) {
        uint32_t tt = t / P.tx;
        V3 tc = v3((float)(t % P.tx), (float)(tt % P.ty), (float)(tt / P.ty)) * 8.0f + v3(4.0f, 4.0f, 4.0f);
        if (fillPhi(v3(P.x0, P.y0, P.z0) + tc * P.h) < 9.0f) need[t] = 1;
      }
    }
    // tileFree + tileAlloc + initNew (a new block: pres 0, collider id per cell, depth bits 0, velG 0)
    for (uint32_t t = 0; t < (uint32_t)ntiles; t++) {
      if (!need[t] && alloc[t]) alloc[t] = 0;
      else if (need[t] && !alloc[t]) {
        alloc[t] = 1;
        for (uint32_t local = 0; local < 512; local++) {
          int i, j, k; tileCoord(t, local, i, j, k);
          uint32_t c = t * 512 + local;
          pres[c] = 0.0f;
          ctype[c] = (uint32_t)(colAt(cellCenter(i, j, k)) + 1) << 8;
          velG[c * 3] = 0.0f; velG[c * 3 + 1] = 0.0f; velG[c * 3 + 2] = 0.0f;
        }
      }
    }
    active.clear();
    for (uint32_t t = 0; t < (uint32_t)ntiles; t++) if (alloc[t]) active.push_back(t);
    st_sc = (uint32_t)active.size(); st_ovf = 0; st_vmax = 0.0f;
    if (init) {                                         // phiInitAll (wgsl-narrowband.js:21-35)
      forActive([&](uint32_t c, int i, int j, int k) {
        float ph = clampf(fillPhi(cellCenter(i, j, k)), -7.9f, 7.9f);
        if (ph < 0.0f) ph = fmin_(ph, -1.5f);
        if (!inDom(i, j, k)) ph = 8.0f;
        if (P.nbInit == 2u) ph = fmin_(ph, phiOf(c));
        phiPut(c, ph);
        if (P.nbInit == 1u)
          for (int ax = 0; ax < 3; ax++) {
            V3 fp = facePos(i, j, k, ax); float v = 0.0f;
            if (P.ocean != 0u && fp.y < oceanEta(fp.x, fp.z)) v = comp(oceanVel(fp), ax);
            velG[c * 3 + ax] = v;
          }
      });
    }
  }
  // clearSlots (wgsl-solver.js:6-15): blocks in use and the spare block
  void stageClear() {
    auto clr = [&](uint32_t c) { cnt[c] = 0; for (int a = 0; a < 3; a++) { accV[c * 3 + a] = 0; accW[c * 3 + a] = 0; } };
    forActive([&](uint32_t c, int, int, int) { clr(c); });
    for (uint32_t l = 0; l < 512; l++) { uint32_t c = spare() * 512 + l; clr(c); rhs[c] = 8.0f; }
  }
  // canonical storage order: live particles by (cell key, id), dead ones after them keeping their order
  void stageSort() {
    uint32_t n = P.n;
    std::vector<uint64_t> key(n);
    std::vector<uint32_t> order(n);
    for (uint32_t i = 0; i < n; i++) {
      order[i] = i;
      if (pos[i * 4 + 1] < DEADY) { key[i] = ~0ull; continue; }
      int ci, cj, ck; particleCell(ppos(i), ci, cj, ck);
      key[i] = ((uint64_t)cellIdx(ci, cj, ck) << 32) | pid[i];
    }
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
    st_live = 0;
    for (uint32_t i = 0; i < n; i++) if (key[i] != ~0ull) st_live++;
    std::vector<float> np((size_t)n * 4), nv((size_t)n * 4); std::vector<uint32_t> nid(n);
    for (uint32_t k = 0; k < n; k++) {
      uint32_t s = order[k];
      memcpy(&np[k * 4], &pos[s * 4], 16); memcpy(&nv[k * 4], &vel[s * 4], 16); nid[k] = pid[s];
    }
    memcpy(pos.data(), np.data(), (size_t)n * 16); memcpy(vel.data(), nv.data(), (size_t)n * 16);
    memcpy(pid.data(), nid.data(), (size_t)n * 4);
  }
  // p2g (wgsl-solver.js:17-40)
  void stageP2G() {
    std::vector<float> vm(nthreads, 0.0f);
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t ii = 0; ii < (int64_t)P.n; ii++) {
      uint32_t i = (uint32_t)ii;
      V3 p = ppos(i);
      if (pos[i * 4 + 1] < DEADY) continue;
      int ci, cj, ck; particleCell(p, ci, cj, ck);
      if (!hasStorage(ci, cj, ck)) continue;
      V3 v = pvel(i);
#ifdef _OPENMP
      int th = omp_get_thread_num();
#else
      int th = 0;
#endif
      vm[th] = fmax_(vm[th], length(v));
      for (int axis = 0; axis < 3; axis++) {
        V3 q = (p - v3(P.x0, P.y0, P.z0)) * P.ih;
        if (axis == 0) { q.y -= 0.5f; q.z -= 0.5f; } else if (axis == 1) { q.x -= 0.5f; q.z -= 0.5f; } else { q.x -= 0.5f; q.y -= 0.5f; }
        V3 f0 = vfloor(q); V3 fr = q - f0; int i0 = (int)f0.x, j0 = (int)f0.y, k0 = (int)f0.z;
        float vc = comp(v, axis);
        for (int c = 0; c < 8; c++) {
          int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
          float w = (dx == 1 ? fr.x : 1.0f - fr.x) * (dy == 1 ? fr.y : 1.0f - fr.y) * (dz == 1 ? fr.z : 1.0f - fr.z);
          if (w <= 0.0f) continue;
          uint32_t idx = faceIndex(axis, i0 + dx, j0 + dy, k0 + dz);
          int32_t av = (int32_t)rintf(w * vc * P.scale), aw = (int32_t)rintf(w * P.scale);
#pragma omp atomic
          accV[idx] += av;
#pragma omp atomic
          accW[idx] += aw;
        }
      }
      uint32_t cc = cellIdx(ci, cj, ck);
#pragma omp atomic
      cnt[cc] += 1;
    }
    for (float x : vm) st_vmax = fmax_(st_vmax, x);
  }
  // narrow band depth passes (wgsl-narrowband.js:38-68)
  float jacNb(int i, int j, int k, float cur, bool fromRhs) const {
    if (!inDom(i, j, k)) return 8.0f;
    if (cur >= 0.0f) return cur;
    float m = -8.0f;
    for (int q = 0; q < 6; q++) {
      int a = i, b = j, c = k;
      if (q == 0) a -= 1; else if (q == 1) a += 1; else if (q == 2) b -= 1; else if (q == 3) b += 1; else if (q == 4) c -= 1; else c += 1;
      if (!inDom(a, b, c)) continue;
      uint32_t cq = cellIdx(a, b, c);
      if (colBits(cq) != 0u) continue;
      m = fmax_(m, fromRhs ? rhs[cq] : phiOf(cq));
    }
    return clampf(m - 1.0f, -7.9f, -0.5f);
  }
  void stageNarrowBand() {
    forActive([&](uint32_t c, int i, int j, int k) {          // nbPhi
      if (!inDom(i, j, k)) { rhs[c] = 8.0f; return; }
      if (colBits(c) != 0u) { rhs[c] = 0.5f; return; }
      V3 x = cellCenter(i, j, k);
      float phA = phiSample(x - velGVec(x) * P.dt);
      bool inside = cnt[c] > 0 || phA < -1.0f;
      if (P.ocean != 0u && layerW(x) >= 0.5f) inside = x.y < oceanEta(x.x, x.z);
      rhs[c] = inside ? clampf(phA, -7.9f, -0.5f) : clampf(phA, 0.5f, 7.9f);
    });
    auto jacA = [&]() { forActive([&](uint32_t c, int i, int j, int k) { phiPut(c, jacNb(i, j, k, rhs[c], true)); }); };
    jacA();
    forActive([&](uint32_t c, int i, int j, int k) { rhs[c] = jacNb(i, j, k, phiOf(c), false); });
    jacA();
  }
  // collider bits (solidBuild, wgsl-solver.js:42-45) then classify (wgsl-solver.js:47-74)
  void stageClassify() {
    forActive([&](uint32_t c, int i, int j, int k) {
      ctype[c] = (ctype[c] & 0xffff00ffu) | ((uint32_t)(colAt(cellCenter(i, j, k)) + 1) << 8);
    });
    forActive([&](uint32_t c, int i, int j, int k) {
      uint32_t ty = 0;
      uint32_t sb = ctype[c] & 0xffffff00u;
      int32_t n = cnt[c];
      V3 cx = cellCenter(i, j, k);
      if (!inDom(i, j, k)) ty = 0;
      else if ((sb & 0xff00u) != 0u) ty = 2;
      else if (P.ocean != 0u && layerW(cx) >= 0.5f) ty = cx.y < oceanEta(cx.x, cx.z) ? 2u : 0u;
      else if (P.nb != 0u && phiOf(c) < -1.0f && (phiOf(c) < -P.band || calmV(velGVec(cx)))) ty = 1;
      else if (n > 0) {
        ty = 1;
        if ((float)n < P.sheetMin) {
          int32_t dth = (int32_t)ceilf(0.6f * P.rest); bool dense = false;
          for (int q = 0; q < 6; q++) {
            int a = i, b = j, cc = k;
            if (q == 0) a -= 1; else if (q == 1) a += 1; else if (q == 2) b -= 1; else if (q == 3) b += 1; else if (q == 4) cc -= 1; else cc += 1;
            if (!inDom(a, b, cc)) continue;
            if (cnt[cellIdx(a, b, cc)] >= dth) dense = true;
          }
          if (!dense) ty = 0;
        }
      }
      ctype[c] = ty | sb;
      if (ty != 1u) pres[c] = 0.0f;
    });
    uint32_t fl = 0;
    for (uint32_t t : active) for (uint32_t l = 0; l < 512; l++) if ((ctype[t * 512 + l] & 0xffu) == 1u) fl++;
    st_fluid = fl;
  }
  // nbVel (wgsl-narrowband.js:71-85)
  void stageNbVel() {
    forActive([&](uint32_t c, int i, int j, int k) {
      if (!inDom(i, j, k)) return;
      if ((ctype[c] & 0xffu) != 1u) return;
      for (int ax = 0; ax < 3; ax++) {
        int a = i, b = j, cc = k;
        if (ax == 0) a -= 1; else if (ax == 1) b -= 1; else cc -= 1;
        if (!inDom(a, b, cc)) continue;
        if ((ctype[cellIdx(a, b, cc)] & 0xffu) != 1u) continue;
        uint32_t f = c * 3 + ax;
        if (accW[f] > 0) continue;
        V3 fp = facePos(i, j, k, ax);
        float vc = velGAxis(fp - velGVec(fp) * P.dt, ax);
        accV[f] = (int32_t)rintf(vc * P.scale); accW[f] = (int32_t)P.scale;
      }
    });
  }
  // normFaces / normBody (wgsl-solver.js:75-105)
  void stageNormFaces() {
    forActive([&](uint32_t c, int i, int j, int k) {
      for (int axis = 0; axis < 3; axis++) {
        uint32_t f = c * 3 + axis;
        int li = i, lj = j, lk = k;
        if (axis == 0) li -= 1; else if (axis == 1) lj -= 1; else lk -= 1;
        uint32_t tl = ctypeOf(li, lj, lk), th = ctypeOf(i, j, k);
        int32_t ws = accW[f], vs = accV[f];
        float v = ws > 0 ? (float)vs / (float)std::max(ws, 1) : 0.0f;
        float old = v;
        if (axis == 1) v -= P.gravity * P.dt;
        if (tl == 2u || th == 2u) {
          float sv = 0.0f; int ci = -1;
          if (tl == 2u) ci = colAtCell(li, lj, lk);
          if (ci < 0 && th == 2u) ci = colAtCell(i, j, k);
          V3 fp = facePos(i, j, k, axis);
          if (ci >= 0) sv = comp(colSurfVel((uint32_t)ci, fp), axis);
          else if (P.ocean != 0u && ((tl == 2u && inDom(li, lj, lk)) || (th == 2u && inDom(i, j, k)))) sv = comp(oceanVel(fp), axis);
          v = sv; old = sv;
        }
        accW[f] = fbits(old); accV[f] = fbits(v);
      }
    });
  }
  // divergence (wgsl-solver.js:107-123)
  void stageDivergence() {
    forActive([&](uint32_t c, int i, int j, int k) {
      if ((ctype[c] & 0xffu) != 1u) { rhs[c] = 0.0f; return; }
      float div = (gvR(faceIndex(0, i + 1, j, k)) - gvR(faceIndex(0, i, j, k)) + gvR(faceIndex(1, i, j + 1, k)) - gvR(faceIndex(1, i, j, k)) +
                   gvR(faceIndex(2, i, j, k + 1)) - gvR(faceIndex(2, i, j, k))) * P.ih;
      bool interior = true;
      if (ctypeOf(i - 1, j, k) == 0u || ctypeOf(i + 1, j, k) == 0u || ctypeOf(i, j - 1, k) == 0u || ctypeOf(i, j + 1, k) == 0u ||
          ctypeOf(i, j, k - 1) == 0u || ctypeOf(i, j, k + 1) == 0u) interior = false;
      float dens = (float)cnt[c] / P.rest - 1.0f;
      float tgt = P.comp * (interior ? dens : fmax_(dens, 0.0f));
      if (P.nb != 0u && phiOf(c) < -1.0f) tgt = 0.0f;
      rhs[c] = (tgt - div) * P.h * P.h / P.dt;
    });
  }
  // relax / rbRed / rbBlack (wgsl-solver.js:124-140, 162-164), iters x (red, black)
  void stagePressure(int iters) {
    for (int it = 0; it < iters; it++) for (uint32_t color = 0; color < 2; color++) {
      forActive([&](uint32_t c, int i, int j, int k) {
        if ((uint32_t)((i + j + k) & 1) != color) return;
        if ((ctype[c] & 0xffu) != 1u) return;
        float sum = 0.0f, nns = 0.0f;
        for (int a = 0; a < 6; a++) {
          int qi = i, qj = j, qk = k;
          if (a == 0) qi -= 1; else if (a == 1) qi += 1; else if (a == 2) qj -= 1; else if (a == 3) qj += 1; else if (a == 4) qk -= 1; else qk += 1;
          uint32_t ty = ctypeOf(qi, qj, qk);
          if (ty == 2u) continue;
          nns += 1.0f;
          if (ty == 1u) sum += pres[cellIdx(qi, qj, qk)];
        }
        if (nns < 0.5f) { pres[c] = 0.0f; return; }
        float pg = (rhs[c] + sum) / nns;
        pres[c] = pres[c] + P.omega * (pg - pres[c]);
      });
    }
  }
  // project / projBody (wgsl-solver.js:165-180), then saveVel (wgsl-narrowband.js:88-91)
  void stageProject(bool nb) {
    forActive([&](uint32_t c, int i, int j, int k) {
      for (int axis = 0; axis < 3; axis++) {
        uint32_t f = c * 3 + axis;
        int li = i, lj = j, lk = k;
        if (axis == 0) li -= 1; else if (axis == 1) lj -= 1; else lk -= 1;
        uint32_t tl = ctypeOf(li, lj, lk), th = ctypeOf(i, j, k);
        if (tl == 2u || th == 2u) continue;
        if (tl != 1u && th != 1u) continue;
        float pl = 0.0f, ph = 0.0f;
        if (tl == 1u) pl = pres[cellIdx(li, lj, lk)];
        if (th == 1u) ph = pres[cellIdx(i, j, k)];
        accV[f] = fbits(gvR(f) - P.dt * P.ih * (ph - pl));
      }
    });
    if (nb) forActive([&](uint32_t c, int, int, int) { for (int a = 0; a < 3; a++) velG[c * 3 + a] = gvR(c * 3 + a); });
  }
  // sampleBoth (wgsl-core.js:138-154)
  void sampleBoth(V3 p, V3& vn, V3& vo) const {
    for (int axis = 0; axis < 3; axis++) {
      V3 g = (p - v3(P.x0, P.y0, P.z0)) * P.ih;
      if (axis == 0) { g.y -= 0.5f; g.z -= 0.5f; } else if (axis == 1) { g.x -= 0.5f; g.z -= 0.5f; } else { g.x -= 0.5f; g.y -= 0.5f; }
      V3 f0 = vfloor(g); V3 fr = g - f0; int i0 = (int)f0.x, j0 = (int)f0.y, k0 = (int)f0.z;
      float sn = 0.0f, so = 0.0f;
      for (int c = 0; c < 8; c++) {
        int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
        float w = (dx == 1 ? fr.x : 1.0f - fr.x) * (dy == 1 ? fr.y : 1.0f - fr.y) * (dz == 1 ? fr.z : 1.0f - fr.z);
        uint32_t f = faceIndex(axis, i0 + dx, j0 + dy, k0 + dz);
        sn += w * gvR(f); so += w * gv0R(f);
      }
      setc(vn, axis, sn); setc(vo, axis, so);
    }
  }
  // collideP (wgsl-solver.js:185-197)
  V3 collideP(V3 pin) const {
    V3 p = pin; float m = P.margin;
    for (uint32_t k = 0; k < P.ncols; k++) {
      if (!colNear(k, p)) continue;
      float phi; V3 wn; sdfEval(k, p, phi, wn);
      if (phi < P.q0) p = p + wn * (P.q0 - phi);
    }
    float big = 1.0e9f;
    V3 lo = v3((P.open & 1u) ? -big : P.x0 + m, (P.open & 4u) ? -big : P.y0 + m, (P.open & 16u) ? -big : P.z0 + m);
    V3 hi = v3((P.open & 2u) ? big : P.x1 - m, (P.open & 8u) ? big : P.y1 - m, (P.open & 32u) ? big : P.z1 - m);
    return vclamp(p, lo, hi);
  }
  static float hsh3(V3 p) {
    V3 q = p * 0.3183099f + v3(0.1f, 0.2f, 0.3f); q = q - vfloor(q); q = q * 17.0f;
    float r = q.x * q.y * q.z * (q.x + q.y + q.z);
    return r - floorf(r);
  }
  static float vnz(V3 x) {    // value noise (wgsl-solver.js:202-207)
    V3 i = vfloor(x); V3 fr = x - vfloor(x); V3 u = fr * fr * (v3(3, 3, 3) - fr * 2.0f);
    float a = mixf(mixf(hsh3(i), hsh3(i + v3(1, 0, 0)), u.x), mixf(hsh3(i + v3(0, 1, 0)), hsh3(i + v3(1, 1, 0)), u.x), u.y);
    float b = mixf(mixf(hsh3(i + v3(0, 0, 1)), hsh3(i + v3(1, 0, 1)), u.x), mixf(hsh3(i + v3(0, 1, 1)), hsh3(i + v3(1, 1, 1)), u.x), u.y);
    return mixf(a, b, u.z);
  }
  // g2p (wgsl-solver.js:208-275)
  void stageG2P() {
    forParticles([&](uint32_t i) {
      if (pos[i * 4 + 1] < DEADY) return;
      V3 p = ppos(i); V3 v0 = pvel(i);
      int fi, fj, fk; particleCell(p, fi, fj, fk);
      V3 vn = v0 - v3(0.0f, P.gravity * P.dt, 0.0f); V3 vo = v0;
      if (hasStorage(fi, fj, fk)) sampleBoth(p, vn, vo);
      V3 v = vmix(vn, v0 + (vn - vo), P.flip);
      if (P.ocean != 0u) { float lw = layerW(p); if (lw > 0.0f) { float s = clampf(lw * 2.0f, 0.0f, 1.0f); v = vmix(v, oceanVel(p), s * s * (1.0f - st_expf(-8.0f * P.dt))); } }
      V3 bcf = vfloor((p - v3(P.x0, P.y0, P.z0)) * P.ih - v3(0.5f, 0.5f, 0.5f));
      int bi = (int)bcf.x, bj = (int)bcf.y, bk = (int)bcf.z;
      float csum = 8.0f * P.rest;
      bool fast = P.q12 > 0.5f;
      if (P.q9 < 0.5f && fast) csum = 8.0f * (float)cnt[cellIdx(fi, fj, fk)];
      else if (P.q9 < 0.5f) {
        csum = 0.0f;
        for (int dz = 0; dz <= 1; dz++) for (int dy = 0; dy <= 1; dy++) for (int dx = 0; dx <= 1; dx++) {
          int a = std::min(std::max(bi + dx, 0), (int)P.nx - 1), b = std::min(std::max(bj + dy, 0), (int)P.ny - 1), c = std::min(std::max(bk + dz, 0), (int)P.nz - 1);
          csum += (float)cnt[cellIdx(a, b, c)];
        }
      }
      float rho = csum / (8.0f * P.rest);
      float air = 1.0f - smoothstep(0.008f, 0.1f, rho);
      float shield = smoothstep(0.1f, 0.65f, rho);
      float exposure = 1.0f - 0.97f * shield;
      float spd0 = length(v);
      float sens = fmax_(P.q6, 0.05f);
      float pacc = length(vn - vo) / P.dt;
      float settle = smoothstep(0.1f, 0.5f, P.q8);
      float impact = clampf((pacc / sens - 15.0f) / 80.0f, 0.0f, 1.0f) * settle;
      float turb = clampf((length(v0 - vo) / sens - 0.35f) / 1.5f, 0.0f, 1.0f) * settle;
      float spray = air * (0.25f + 0.75f * clampf(spd0 / 4.0f, 0.0f, 1.0f));
      float tau = fmax_(P.q5, 0.05f) * mixf(1.0f, 0.35f, smoothstep(0.7f, 1.0f, rho)) * mixf(1.0f, 2.5f, air);
      float foam = vel[i * 4 + 3] * st_expf(-P.dt / tau);
      foam = fmax_(foam, fmax_(spray * 0.9f, fmax_(impact, turb * 0.8f)));
      if (P.ocean != 0u) foam *= 1.0f - clampf(layerW(p) * 2.0f, 0.0f, 1.0f);
      V3 gust = v3(0, 0, 0);
      if (P.q7 > 0.0f && P.q4 > 0.0f && (!fast || shield < 0.9f)) {
        V3 gp = p * 0.55f; float tt = P.q8 * 0.6f;
        gust = v3(vnz(gp + v3(tt, 0.0f, 0.0f)), vnz(gp + v3(17.3f, tt, 4.1f)), vnz(gp + v3(5.7f, 9.2f, tt))) * 2.0f - v3(1, 1, 1);
      }
      float kd = P.q4 * (0.04f + 1.5f * exposure * exposure);
      V3 airv = v3(P.q1, P.q2, P.q3) + gust * P.q7;
      v = v + (airv - v) * (1.0f - st_expf(-kd * P.dt));
      float sp = length(v);
      if (sp > P.vmax) v = v * (P.vmax / sp);
      V3 pt = p + v * P.dt;
      V3 pc = collideP(pt);
      V3 dsp = pc - pt;
      if (dot(dsp, dsp) > 1.0e-12f) {
        V3 nrm = dsp / length(dsp); float vd = dot(v, nrm);
        if (vd < 0.0f) v = v - nrm * vd;
      }
      uint32_t o = P.open;
      if (o != 0u && (((o & 1u) && pc.x < P.x0) || ((o & 2u) && pc.x > P.x1) || ((o & 4u) && pc.y < P.y0) ||
                      ((o & 8u) && pc.y > P.y1) || ((o & 16u) && pc.z < P.z0) || ((o & 32u) && pc.z > P.z1))) {
        pos[i * 4] = 0.0f; pos[i * 4 + 1] = -1.0e6f; pos[i * 4 + 2] = 0.0f; pos[i * 4 + 3] = 0.0f;
        vel[i * 4] = 0.0f; vel[i * 4 + 1] = 0.0f; vel[i * 4 + 2] = 0.0f; vel[i * 4 + 3] = 0.0f;
        return;
      }
      pos[i * 4] = pc.x; pos[i * 4 + 1] = pc.y; pos[i * 4 + 2] = pc.z;
      pos[i * 4 + 3] = fmin_(length(v), 63.0f) + 64.0f * floorf(foam * 15.0f + 0.5f);
      vel[i * 4] = v.x; vel[i * 4 + 1] = v.y; vel[i * 4 + 2] = v.z; vel[i * 4 + 3] = foam;
    });
  }

  // ---- whitewater (wgsl-whitewater.js:7-23, 92-180) ----
  float wetCell(int i, int j, int k) const {
    if (!inDom(i, j, k) || !hasStorage(i, j, k)) return 0.0f;
    uint32_t ci = cellIdx(i, j, k);
    if (P.nb != 0u && (ctype[ci] & 0xffu) == 1u && phiOf(ci) < -1.0f) return 1.0f;
    return fmin_((float)cnt[ci] / P.rest, 1.0f);
  }
  float wetAt(V3 p) const {
    V3 g = (p - v3(P.x0, P.y0, P.z0)) * P.ih - v3(0.5f, 0.5f, 0.5f);
    V3 f0 = vfloor(g); V3 fr = g - f0; int i0 = (int)f0.x, j0 = (int)f0.y, k0 = (int)f0.z;
    float s = 0.0f;
    for (int c = 0; c < 8; c++) {
      int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
      float w = (dx == 1 ? fr.x : 1.0f - fr.x) * (dy == 1 ? fr.y : 1.0f - fr.y) * (dz == 1 ? fr.z : 1.0f - fr.z);
      if (w > 0.0f) s += w * wetCell(i0 + dx, j0 + dy, k0 + dz);
    }
    return s;
  }
  // ---- air field (wgsl-whitewater.js:24-89) ----
  uint32_t airIdx(int x, int y, int z) const {   // :25-28
    int qx = std::min(std::max(x, 0), (int)P.aNx - 1), qy = std::min(std::max(y, 0), (int)P.aNy - 1), qz = std::min(std::max(z, 0), (int)P.aNz - 1);
    return (uint32_t)qx + P.aNx * ((uint32_t)qy + P.aNy * (uint32_t)qz);
  }
  V3 airV(uint32_t c) const { return v3(air[c * 4], air[c * 4 + 1], air[c * 4 + 2]); }
  V3 airAt(V3 p) const {   // :30-40
    V3 g = (p - v3(P.x0, P.y0, P.z0)) / P.airH - v3(0.5f, 0.5f, 0.5f);
    V3 f0 = vfloor(g); V3 fr = g - f0; int i0 = i32idx(f0.x), j0 = i32idx(f0.y), k0 = i32idx(f0.z);
    V3 s = v3(0, 0, 0);
    for (int c = 0; c < 8; c++) {
      int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
      float w = (dx == 1 ? fr.x : 1.0f - fr.x) * (dy == 1 ? fr.y : 1.0f - fr.y) * (dz == 1 ? fr.z : 1.0f - fr.z);
      s = s + airV(airIdx(i0 + dx, j0 + dy, k0 + dz)) * w;
    }
    return s;
  }
  void airPush(V3 p, V3 v, float w) {   // :41-45 (integer sums: any order gives the same result)
    V3 g = vfloor((p - v3(P.x0, P.y0, P.z0)) / P.airH);
    uint32_t c = airIdx(i32idx(g.x), i32idx(g.y), i32idx(g.z)) * 4u;
    uint32_t q[4] = {(uint32_t)i32f(v.x * w * 256.0f), (uint32_t)i32f(v.y * w * 256.0f), (uint32_t)i32f(v.z * w * 256.0f), (uint32_t)i32f(w * 256.0f)};
    for (int a = 0; a < 4; a++) {
      uint32_t* t = reinterpret_cast<uint32_t*>(&airAcc[c + a]);
#pragma omp atomic
      *t += q[a];
    }
  }
  void stageAir() {
    std::fill(airAcc.begin(), airAcc.end(), 0);                                   // airClear
    forParticles([&](uint32_t i) {                                                // airSplatW (:51-57)
      if (pos[i * 4 + 1] < DEADY) return;
      V3 p = ppos(i);
      int ci, cj, ck; particleCell(p, ci, cj, ck);
      if (hasStorage(ci, cj, ck) && (float)cnt[cellIdx(ci, cj, ck)] > 0.85f * P.rest) return;
      airPush(p, pvel(i), 1.0f);
    });
    uint32_t m = std::min(sctl0, P.smax);                                         // airSplatS (:59-64), over the slots handed out
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t jj = 0; jj < (int64_t)m; jj++) {
      uint32_t j = (uint32_t)jj;
      if (sPos[j * 4 + 3] <= 0.0f || sVel[j * 4 + 3] > 1.5f) continue;
      airPush(v3(sPos[j * 4], sPos[j * 4 + 1], sPos[j * 4 + 2]), v3(sVel[j * 4], sVel[j * 4 + 1], sVel[j * 4 + 2]), 0.25f);
    }
    uint32_t na = P.aNx * P.aNy * P.aNz;                                          // airUpdate (:67-86)
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t cc = 0; cc < (int64_t)na; cc++) {
      uint32_t c = (uint32_t)cc;
      int ci = (int)(c % P.aNx), cj = (int)((c / P.aNx) % P.aNy), ck = (int)(c / (P.aNx * P.aNy));
      V3 a = airV(c);
      V3 nb = (airV(airIdx(ci + 1, cj, ck)) + airV(airIdx(ci - 1, cj, ck)) + airV(airIdx(ci, cj + 1, ck)) + airV(airIdx(ci, cj - 1, ck)) +
               airV(airIdx(ci, cj, ck + 1)) + airV(airIdx(ci, cj, ck - 1))) / 6.0f;
      a = vmix(a, nb, P.airBlur);
      float w = (float)airAcc[c * 4 + 3] / 256.0f;
      if (w > 0.0f) {
        V3 vt = v3((float)airAcc[c * 4], (float)airAcc[c * 4 + 1], (float)airAcc[c * 4 + 2]) / (w * 256.0f);
        a = vmix(a, vt, 1.0f - st_expf(-P.airCouple * fmin_(w, 8.0f) * P.dt));
      }
      V3 x = v3(P.x0, P.y0, P.z0) + (v3((float)ci, (float)cj, (float)ck) + v3(0.5f, 0.5f, 0.5f)) * P.airH;
      for (uint32_t k = 0; k < P.ncols; k++) {
        if (!colNear(k, x)) continue;
        float phi; V3 wn; sdfEval(k, x, phi, wn);
        if (phi < 0.6f * P.airH) { a = colSurfVel(k, x); break; }
      }
      a = vmix(a, v3(P.q1, P.q2, P.q3), 1.0f - st_expf(-P.airDecay * P.dt));
      air2[c * 4] = a.x; air2[c * 4 + 1] = a.y; air2[c * 4 + 2] = a.z; air2[c * 4 + 3] = 0.0f;
    }
    std::copy(air2.begin(), air2.begin() + (size_t)na * 4, air.begin());        // airCopy
  }

  // PBF density constraints on the particles at the end of the step (st_step_opts.pbf_iters; the reference's FLIP step
  // has none): GpuSim's grid, lambda and delta (src/gpu.js:162-292, restated in pbf_core.h) with kernel radius 2.2 d,
  // the walls' and colliders' boundary density, collideP after each correction; then v += (x - p) / dt, pos.w again
  void stagePbf(double dt, int iters) {
    const PbfConsts pc = pbfConsts(d, 0.0, 0.0);
    const double lo[3] = {bx0, by0, bz0}, hi[3] = {bx1, by1, bz1};
    const PbfP Q = pbfParams(pc, d, lo, hi, dt, 0.0, 0.0, N, P.ncols, open);
    std::vector<float> prd((size_t)N * 4), lam, bgr, dlt;
    for (size_t i = 0; i < (size_t)N; i++) {
      prd[i * 4] = pos[i * 4]; prd[i * 4 + 1] = pos[i * 4 + 1]; prd[i * 4 + 2] = pos[i * 4 + 2]; prd[i * 4 + 3] = 0.0f;
    }
    PbfGrid G;
    pbfBuildGrid(Q, prd.data(), 4, N, G);
    auto sdfOf = [&](uint32_t k, V3 x, float& phi, V3& wn) { sdfEval(k, x, phi, wn); };
    auto col = [&](V3 p) { return collideP(p); };
    for (int it = 0; it < iters; it++) pbfIteration(Q, sdfOf, P.ncols, col, G, prd.data(), N, lam, bgr, dlt, nthreads);
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t ii = 0; ii < (int64_t)N; ii++) {
      const size_t i = (size_t)ii;
      if (G.cid[i] == PBF_DEADC) continue;
      const V3 x = v3(prd[i * 4], prd[i * 4 + 1], prd[i * 4 + 2]);
      const V3 v = pvel((uint32_t)i) + (x - ppos((uint32_t)i)) / Q.dt;
      const float foam = vel[i * 4 + 3];
      pos[i * 4] = x.x; pos[i * 4 + 1] = x.y; pos[i * 4 + 2] = x.z; pos[i * 4 + 3] = fmin_(length(v), 63.0f) + 64.0f * floorf(foam * 15.0f + 0.5f);
      vel[i * 4] = v.x; vel[i * 4 + 1] = v.y; vel[i * 4 + 2] = v.z;
    }
  }

  void stageSpray(bool emit) {
    if (P.airOn != 0u) stageAir();   // the air field first, so the whitewater moves with this step's air (sim.js:297-301)
    uint32_t m = std::min(sctl0, P.smax);
    // wwSample
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t jj = 0; jj < (int64_t)m; jj++) {
      uint32_t j = (uint32_t)jj;
      if (sPos[j * 4 + 3] <= 0.0f) continue;
      V3 p = v3(sPos[j * 4], sPos[j * 4 + 1], sPos[j * 4 + 2]); V3 vf = v3(0, 0, 0);
      int ci, cj, ck; particleCell(p, ci, cj, ck);
      if (hasStorage(ci, cj, ck)) { V3 vo; sampleBoth(p, vf, vo); }
      sAux[j * 4] = vf.x; sAux[j * 4 + 1] = vf.y; sAux[j * 4 + 2] = vf.z; sAux[j * 4 + 3] = wetAt(p);
    }
    // sprayStep
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t jj = 0; jj < (int64_t)m; jj++) {
      uint32_t j = (uint32_t)jj;
      float life = sPos[j * 4 + 3];
      if (life <= 0.0f) continue;
      V3 v = v3(sVel[j * 4], sVel[j * 4 + 1], sVel[j * 4 + 2]); float kw = sVel[j * 4 + 3]; uint32_t kind = u32f(kw + 0.5f);
      float tk = (kw - (float)kind) / 0.4f * WWHOLD; bool settled = tk >= WWHOLD * 0.999f; uint32_t k0 = kind;
      float wet = sAux[j * 4 + 3]; V3 vf = v3(sAux[j * 4], sAux[j * 4 + 1], sAux[j * 4 + 2]);
      uint32_t h0 = j * 2654435761u + P.seed * 974711u;
      if (kind == 0u && v.y < vf.y && wet > 0.55f && tk > 0.05f) { kind = 2u; life = P.wwFoamLife * (0.6f + 0.8f * hash1(h0)); v = vf; }
      else if (kind == 1u && wet > 0.55f) { life = 0.0f; }
      else if (kind == 2u && wet > 0.97f && settled) { kind = 3u; }
      else if (kind == 2u && wet < 0.04f && settled) { kind = 0u; life = fmin_(life, P.sprLife); }
      else if (kind == 3u && wet < 0.6f && settled) { kind = 2u; life = fmax_(life, 0.5f * P.wwFoamLife); }
      if (kind != k0) tk = 0.0f; else tk = fmin_(tk + P.dt, WWHOLD);
      V3 p = v3(sPos[j * 4], sPos[j * 4 + 1], sPos[j * 4 + 2]);
      if (kind <= 1u) {
        bool mist = kind == 1u;
        V3 gust = v3(0, 0, 0);
        if (P.q7 > 0.0f) {
          V3 gp = p * 0.55f * P.vs; float tt = P.q8 * 0.6f;
          gust = v3(vnz(gp + v3(tt, 0.0f, 0.0f)), vnz(gp + v3(17.3f, tt, 4.1f)), vnz(gp + v3(5.7f, 9.2f, tt))) * 2.0f - v3(1, 1, 1);
        }
        V3 base = P.airOn != 0u ? airAt(p) : v3(P.q1, P.q2, P.q3);
        V3 airv = base + gust * P.q7 * (mist ? 2.5f : 1.0f);
        v.y -= P.gravity * P.dt;
        v = v + (airv - v) * (1.0f - st_expf(-(mist ? P.mistDrag : P.sprDrag) * P.dt));
        life -= P.dt;
      } else if (kind == 2u) {
        float vy = vf.y + clampf((wet - 0.5f) * 4.0f, -1.0f, 1.0f) * P.h * 4.0f;
        v = vmix(v, v3(vf.x, vy, vf.z), 1.0f - st_expf(-10.0f * P.dt));
        life -= P.dt;
      } else {
        v = vmix(v, vf + v3(0.0f, P.wwRise, 0.0f), 1.0f - st_expf(-6.0f * P.dt));
        life -= 0.3f * P.dt;
      }
      V3 np = p + v * P.dt;
      if (np.x < P.x0 || np.x > P.x1 || np.y < P.y0 || np.y > P.y1 || np.z < P.z0 || np.z > P.z1) life = 0.0f;
      else if (P.ncols > 0u && colAt(np) >= 0) life = 0.0f;
      else if (P.ocean != 0u && kind >= 2u && layerW(np) > 0.6f) life = 0.0f;
      sPos[j * 4] = np.x; sPos[j * 4 + 1] = np.y; sPos[j * 4 + 2] = np.z; sPos[j * 4 + 3] = life;
      sVel[j * 4] = v.x; sVel[j * 4 + 1] = v.y; sVel[j * 4 + 2] = v.z; sVel[j * 4 + 3] = (float)kind + 0.4f * tk / WWHOLD;
    }
    if (emit) stageEmit();
    if (P.ndrip) stageDrip();
  }

  // dripStep (wgsl-whitewater.js:254-278). Canonical order: samples ascending; the ring counter advances once per drop;
  // drops beyond smax in one pass are not written.
  void stageDrip() {
    uint32_t run = 0;
    for (uint32_t s = 0; s < P.ndrip; s++) {
      float* a = &drip[(size_t)s * 8]; float* b = a + 4;
      uint32_t k = u32f(a[3]); if (k >= P.ncols) continue;
      V3 r0 = v3(col(k, 2)[0], col(k, 2)[1], col(k, 2)[2]), r1 = v3(col(k, 3)[0], col(k, 3)[1], col(k, 3)[2]), r2 = v3(col(k, 4)[0], col(k, 4)[1], col(k, 4)[2]);
      V3 wp = v3(col(k, 5)[0], col(k, 5)[1], col(k, 5)[2]) + r0 * a[0] + r1 * a[1] + r2 * a[2];
      V3 wr = r0 * b[0] + r1 * b[1] + r2 * b[2];
      V3 wn = wr / length(wr);
      V3 probe = wp + wn * P.h * 0.75f;
      float here = wetAt(probe);
      if (here > 0.4f) { b[3] = 1.0f; continue; }
      float wetness = fmax_(0.0f, b[3] - P.dt / fmax_(P.dripDry, 0.05f));
      b[3] = wetness;
      if (wetness <= 0.0f || here > 0.1f || P.smax == 0u || P.dripRate <= 0.0f) continue;
      float down = clampf(-wn.y, 0.0f, 1.0f);
      float rate = P.dripRate * wetness * wetness * (0.15f + 0.85f * down);
      uint32_t h0 = s * 747796405u + P.seed * 2891336453u + 17u;
      if (hash1(h0) >= rate * P.dt) continue;
      uint32_t r = run++;
      if (r >= P.smax) continue;
      uint32_t slot = (uint32_t)(((uint64_t)sctl0 + r) % P.smax);
      if (sPos[slot * 4 + 3] > 0.0f) continue;
      V3 nv = colSurfVel(k, wp) + wn * P.h * 2.0f * hash1(h0 + 1u);
      sPos[slot * 4] = probe.x; sPos[slot * 4 + 1] = probe.y; sPos[slot * 4 + 2] = probe.z; sPos[slot * 4 + 3] = P.sprLife * 2.0f;
      sVel[slot * 4] = nv.x; sVel[slot * 4 + 1] = nv.y; sVel[slot * 4 + 2] = nv.z; sVel[slot * 4 + 3] = 0.0f;
    }
    sctl0 = sctl0 + run;
  }

  void stageEmit() {
    // sprayEmit (wgsl-whitewater.js:101-133). Canonical order: particles by storage index, points by m; the ring
    // counter advances once per point tried; a slot is taken only if it was not living before this pass.
    if (P.smax == 0u || P.sprRate <= 0.0f) return;
    std::vector<uint32_t> kcount(P.n, 0);
    std::vector<float> rhov(P.n, 0.0f);
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t ii = 0; ii < (int64_t)P.n; ii++) {
      uint32_t i = (uint32_t)ii;
      if (pos[i * 4 + 1] < DEADY) continue;
      if (P.ocean != 0u && layerW(ppos(i)) > 0.0f) continue;
      V3 q = ppos(i); V3 v = pvel(i); float foam = vel[i * 4 + 3]; float spd = length(v);
      float fast = clampf((spd * P.vs - P.sprMin) / (2.0f * P.sprMin), 0.0f, 1.0f);
      V3 bcf = vfloor((q - v3(P.x0, P.y0, P.z0)) * P.ih - v3(0.5f, 0.5f, 0.5f));
      int bi = (int)bcf.x, bj = (int)bcf.y, bk = (int)bcf.z;
      float rho = 0.0f;
      for (int dz = 0; dz <= 1; dz++) for (int dy = 0; dy <= 1; dy++) for (int dx = 0; dx <= 1; dx++) rho += wetCell(bi + dx, bj + dy, bk + dz);
      rho = rho / 8.0f;
      float crest = (1.0f - smoothstep(0.3f, 0.75f, rho)) * fast * (0.3f + 0.7f * foam);
      float churn = (1.0f - smoothstep(0.8f, 1.0f, rho)) * clampf((foam - 0.55f) / 0.45f, 0.0f, 1.0f) * smoothstep(0.5f, 1.5f, spd * P.vs);
      float e = (P.wwCrest * crest + P.wwImpact * churn) * smoothstep(0.1f, 0.5f, P.q8);
      if (e <= 0.0f) continue;
      uint32_t h0 = pid[i] * 747796405u + P.seed * 2891336453u;
      float kf = floorf(P.sprRate * e * P.dt + hash1(h0));
      kcount[i] = std::min(u32f(kf), 4u); rhov[i] = rho;
    }
    uint64_t tried = 0; for (uint32_t i = 0; i < P.n; i++) tried += kcount[i];
    if (tried > P.smax) spray_ovf++;
    std::vector<float> lifeBefore(P.smax);
    for (uint32_t j = 0; j < P.smax; j++) lifeBefore[j] = sPos[j * 4 + 3];
    uint64_t run = 0;
    for (uint32_t i = 0; i < P.n; i++) {
      for (uint32_t mm = 0; mm < kcount[i]; mm++, run++) {
        if (run >= P.smax) continue;   // more points tried in one step than the ring holds: the rest are dropped
        uint32_t slot = (uint32_t)((sctl0 + run) % P.smax);
        if (lifeBefore[slot] > 0.0f) continue;
        V3 q = ppos(i); V3 v = pvel(i); float spd = length(v); float rho = rhov[i];
        float fast = clampf((spd * P.vs - P.sprMin) / (2.0f * P.sprMin), 0.0f, 1.0f);
        uint32_t h0 = pid[i] * 747796405u + P.seed * 2891336453u;
        uint32_t hh = h0 ^ ((mm + 1u) * 0x9E3779B9u);
        float z = hash1(hh + 1u) * 2.0f - 1.0f; float a = hash1(hh + 2u) * 6.2831853f; float s = sqrtf(fmax_(0.0f, 1.0f - z * z));
        float sa, ca; st_sincosf(a, &sa, &ca);
        V3 dir = v3(s * ca, s * sa, z);
        bool under = rho > 0.7f && hash1(hh + 7u) < 0.7f;
        bool mist = !under && hash1(hh + 3u) < P.mistFrac * fast;
        V3 nv = v * (0.9f + 0.2f * hash1(hh + 4u)) + dir * spd * (mist ? 0.2f : 0.06f);
        float life = P.sprLife * (0.6f + 0.8f * hash1(hh + 5u)) * (mist ? 1.6f : 1.0f);
        float kind = mist ? 1.0f : 0.0f;
        if (under) { nv = v + dir * spd * 0.05f; life = P.wwFoamLife * (0.6f + 0.8f * hash1(hh + 5u)); kind = 3.0f; }
        V3 np = q + nv * P.dt + dir * P.h * 0.3f * hash1(hh + 6u);
        sPos[slot * 4] = np.x; sPos[slot * 4 + 1] = np.y; sPos[slot * 4 + 2] = np.z; sPos[slot * 4 + 3] = life;
        sVel[slot * 4] = nv.x; sVel[slot * 4 + 1] = nv.y; sVel[slot * 4 + 2] = nv.z; sVel[slot * 4 + 3] = kind;
      }
    }
    sctl0 = (uint32_t)(sctl0 + tried);
  }

  // ---- narrow band reseed (wgsl-narrowband.js:93-148) ----
  void stageReseed() {
    forParticles([&](uint32_t i) {                       // nbKill
      if (pos[i * 4 + 1] < DEADY) return;
      V3 q = ppos(i);
      float lw = layerW(q);
      bool kill = lw >= 0.5f || (lw > 0.25f && q.y > oceanEta(q.x, q.z) + 0.5f * P.h);
      if (!kill && P.nb != 0u && calmV(pvel(i))) {
        int ci, cj, ck; particleCell(q, ci, cj, ck);
        if (hasStorage(ci, cj, ck) && phiOf(cellIdx(ci, cj, ck)) < -P.band) kill = true;
      }
      if (kill) { for (int a = 0; a < 4; a++) { pos[i * 4 + a] = 0.0f; vel[i * 4 + a] = 0.0f; } pos[i * 4 + 1] = -1.0e6f; }
    });
    std::vector<uint32_t> dead;                          // nbDead: ascending storage index
    for (uint32_t i = 0; i < P.n; i++) if (pos[i * 4 + 1] < DEADY && dead.size() < P.lcap) dead.push_back(i);
    struct Def { int i, j, k; uint32_t need; };
    std::vector<Def> defs;                               // nbDeficit: ascending cell key
    for (uint32_t tile : active) for (uint32_t local = 0; local < 512; local++) {
      int i, j, k; tileCoord(tile, local, i, j, k); uint32_t c = tile * 512 + local;
      if (!inDom(i, j, k) || colBits(c) != 0u) continue;
      V3 cx = cellCenter(i, j, k); float ph = phiOf(c); float lw = layerW(cx);
      if (lw > 0.25f && lw < 0.5f) {
        if (cx.y > oceanEta(cx.x, cx.z) - 0.25f * P.h || ph < -P.band) continue;
      } else {
        if ((ctype[c] & 0xffu) != 1u || ph > -1.0f || ph < -P.band) continue;
        if (!calmV(velGVec(cx))) continue;
      }
      uint32_t n = (uint32_t)std::max(cnt[c], 0);
      if ((float)n >= 0.55f * P.rest) continue;
      uint32_t nd = std::min((uint32_t)rintf(0.85f * P.rest) - n, 64u);
      if (defs.size() >= P.lcap / 2u) continue;
      defs.push_back({i, j, k, nd});
    }
    uint32_t avail = std::min((uint32_t)dead.size(), P.lcap);
    uint32_t base = 0;
    for (uint32_t e = 0; e < (uint32_t)defs.size(); e++) {   // nbSpawn
      V3 cp = v3((float)defs[e].i, (float)defs[e].j, (float)defs[e].k);
      for (uint32_t m = 0; m < defs[e].need; m++) {
        uint32_t k = base + m; if (k >= avail) break;
        uint32_t i = dead[k];
        uint32_t hh = (e * 9781u + m * 6271u + 17u) ^ (P.seed * 2654435761u);
        V3 x = v3(P.x0, P.y0, P.z0) + (cp + v3(hash1(hh + 1u), hash1(hh + 2u), hash1(hh + 3u))) * P.h;
        V3 v = velGVec(x);
        if (layerW(x) > 0.25f) v = oceanVel(x);
        pos[i * 4] = x.x; pos[i * 4 + 1] = x.y; pos[i * 4 + 2] = x.z; pos[i * 4 + 3] = fmin_(length(v), 63.0f);
        vel[i * 4] = v.x; vel[i * 4 + 1] = v.y; vel[i * 4 + 2] = v.z; vel[i * 4 + 3] = 0.0f;
      }
      base += defs[e].need;
    }
  }

  // ---- deepClear + deepPick + deepFin (wgsl-whitewater.js:282-297): fluid cells with no particles, as points at their
  // centres (x, y, z, 4096 + speed), in ascending tile then cell order; above DEEPMAX cells seen by the previous pass, a
  // fixed hashed sample ----
  std::vector<float> deepPass() {
    const uint32_t DEEPMAX = 200000u;
    std::vector<float> out;
    uint32_t seen = 0, picked = 0;
    for (uint32_t tile : active) for (uint32_t local = 0; local < 512; local++) {
      int i, j, k; tileCoord(tile, local, i, j, k); uint32_t c = tile * 512u + local;
      if (!inDom(i, j, k) || (ctype[c] & 0xffu) != 1u || cnt[c] > 0) continue;
      seen++;
      if (deepPrev > DEEPMAX && hash1(c * 2654435761u + 7u) * (float)deepPrev >= (float)DEEPMAX) continue;
      if (picked++ >= DEEPMAX) continue;
      V3 x = cellCenter(i, j, k);
      float rec[4] = {x.x, x.y, x.z, 4096.0f + fmin_(length(velGVec(x)), 63.0f)};
      out.insert(out.end(), rec, rec + 4);
    }
    deepPrev = seen;
    return out;
  }

  // ---- FlipSim.step (sim.js:179-241, stage list :245-310) ----
  st_status step(double dt, const st_step_opts* o) {
    if (N == 0) return ST_NOT_READY;
    bool nbOn = o->nb_on != 0 || o->ocean_on != 0;
    if (nbOn && !velGOn) velGOn = true;
    uint32_t init = nbOn && nbInit ? nbInit : 0;
    // a restart packs the fill volumes after the step's colliders (FlipSim.step, src/flip/sim.js:189-190)
    const uint32_t ncStep = std::min(o->ncols, 32u);
    nfv = 0;
    if (init && !fillVols.empty()) {
      std::vector<st_collider> all(o->cols, o->cols + ncStep);
      for (auto& f : fillVols) { all.push_back(f.c); all.back().sdf = &f.sd; f.sd.data = f.data.data(); }
      st_step_opts o2 = *o;
      o2.cols = all.data();
      o2.ncols = (uint32_t)all.size();
      packCols(&o2);
      nfv = ncols - std::min(ncStep, ncols);
      ncols -= nfv;
    } else {
      packCols(o);
    }
    bool sprOn = o->spray_on != 0 && sprayCap > 0;
    if (sprOn && o->drip_on != 0) dripUpdate(o, ncols);
    lastN = N; lastNb = nbOn;
    seed = seed + 1u;
    packParams(dt, o, init, nbOn, sprOn);
    tm = tm + dt;
    if (init) { nbInit = 0; fillsPacked.clear(); fillVols.clear(); }
    int iters = std::max(1, o->iters);
    stageBlocks(nbOn, init);
    stageClear();
    stageSort();
    stageP2G();
    if (nbOn) stageNarrowBand();
    stageClassify();
    if (nbOn) stageNbVel();
    stageNormFaces();
    stageDivergence();
    stagePressure(iters);
    stageProject(nbOn);
    stageG2P();
    if (sprayCap > 0) stageSpray(sprOn);
    if (nbOn) stageReseed();
    if (o->pbf_iters > 0) stagePbf(dt, std::min(o->pbf_iters, 64));
    steps++;
    return ST_OK;
  }
};

}  // namespace

extern "C" {

void oracle_step_opts_default(st_step_opts* o);

st_status oracle_flip_create(const st_flip_desc* desc, void** out) {
  if (!desc || !out || desc->size != sizeof(st_flip_desc) || desc->d <= 0 || desc->max_n == 0) return ST_BAD_ARG;
  Oracle* s = new Oracle();
  s->create(desc);
  *out = s;
  return ST_OK;
}
void oracle_flip_destroy(void* h) { delete (Oracle*)h; }
void oracle_flip_set_threads(void* h, int n) { ((Oracle*)h)->nthreads = n < 1 ? 1 : n; }
st_status oracle_flip_clear(void* h) { ((Oracle*)h)->clear(); return ST_OK; }
st_status oracle_flip_set_cap(void* h, uint32_t c) {
  Oracle* s = (Oracle*)h; s->cap = std::min(c, s->maxN); if (s->N > s->cap) s->N = s->cap; if (s->ring >= s->cap) s->ring = 0; return ST_OK;
}
st_status oracle_flip_add(void* h, const float* p3, const float* v3_, uint32_t n, uint32_t* added) {
  Oracle* s = (Oracle*)h; uint32_t k = 0;
  for (; k < n; k++) if (!s->add(p3[k * 3], p3[k * 3 + 1], p3[k * 3 + 2], v3_[k * 3], v3_[k * 3 + 1], v3_[k * 3 + 2])) break;
  if (added) *added = k;
  return ST_OK;
}
st_status oracle_flip_step(void* h, double dt, const st_step_opts* o) {
  if (!o || o->size != sizeof(st_step_opts)) return ST_BAD_ARG;
  return ((Oracle*)h)->step(dt, o);
}
st_status oracle_flip_read_particles(void* h, float* pos4, float* vel4, uint32_t cap, uint32_t* n) {
  Oracle* s = (Oracle*)h; if (n) *n = s->N;
  for (uint32_t i = 0; i < s->N; i++) {
    uint32_t id = s->pid[i]; if (id >= cap) continue;
    if (pos4) memcpy(&pos4[(size_t)id * 4], &s->pos[(size_t)i * 4], 16);
    if (vel4) memcpy(&vel4[(size_t)id * 4], &s->vel[(size_t)i * 4], 16);
  }
  return ST_OK;
}
st_status oracle_flip_read_spray(void* h, float* pos4, float* vel4, uint32_t cap, uint32_t* n) {
  Oracle* s = (Oracle*)h; uint32_t m = std::max(1u, std::min(s->sprayCap, s->sctl0)); if (!s->sprayCap) m = 0;
  if (n) *n = m;
  for (uint32_t j = 0; j < m && j < cap; j++) {
    if (pos4) memcpy(&pos4[j * 4], &s->sPos[j * 4], 16);
    if (vel4) memcpy(&vel4[j * 4], &s->sVel[j * 4], 16);
  }
  return ST_OK;
}
st_status oracle_flip_read_air(void* h, float* vel4, uint32_t cap, uint32_t* dims3) {
  Oracle* s = (Oracle*)h;
  if (dims3) { dims3[0] = s->aNx; dims3[1] = s->aNy; dims3[2] = s->aNz; }
  uint32_t m = std::min(cap, s->airCells);
  if (vel4 && m) memcpy(vel4, s->air.data(), (size_t)m * 16);
  return ST_OK;
}
st_status oracle_flip_read_drips(void* h, float* out8, uint32_t cap, uint32_t* n) {
  Oracle* s = (Oracle*)h;
  if (n) *n = s->ndrip;
  uint32_t m = std::min(cap, s->ndrip);
  if (out8 && m) memcpy(out8, s->drip.data(), (size_t)m * 32);
  return ST_OK;
}
int oracle_ocean_waves(const st_step_opts* o, double depth, float* w) { return (int)Oracle::oceanWaves(o, (double)o->g, depth, w); }
st_status oracle_flip_set_recycle(void* h, int on) { ((Oracle*)h)->recycle = on != 0; return ST_OK; }
// FlipSim.setSprayCap (sim.js:326-334): a new empty pool; sctl keeps counting. The first pool also brings the air field.
st_status oracle_flip_set_spray_cap(void* h, uint32_t n) {
  Oracle* s = (Oracle*)h;
  if (n == s->sprayCap) return ST_OK;
  s->sprayCap = n;
  s->sPos.assign((size_t)std::max(n, 1u) * 4, 0.0f); s->sVel = s->sPos; s->sAux = s->sPos;
  if (n && !s->airCells) {
    int r = std::max(2, (int)std::ceil(std::cbrt((double)s->nx * s->ny * s->nz / 260000.0)));
    s->airH = s->h * r;
    s->aNx = (uint32_t)((s->nx + r - 1) / r + 1); s->aNy = (uint32_t)((s->ny + r - 1) / r + 1); s->aNz = (uint32_t)((s->nz + r - 1) / r + 1);
    s->airCells = s->aNx * s->aNy * s->aNz;
    s->air.assign((size_t)s->airCells * 4, 0.0f); s->air2 = s->air; s->airAcc.assign((size_t)s->airCells * 4, 0);
  }
  return ST_OK;
}
st_status oracle_flip_set_deep_look(void* h, int on) { ((Oracle*)h)->deepOn = on != 0; return ST_OK; }
// one deep pass when the deep look applies (deep look on, narrow band and kept velocities on at the last step), as
// float4 points; *n receives the count (0 when it does not apply)
st_status oracle_flip_deep_points(void* h, float* out4, uint32_t cap, uint32_t* n) {
  Oracle* s = (Oracle*)h;
  if (n) *n = 0;
  if (!(s->deepOn && s->lastNb && s->velGOn && s->lastN)) return ST_OK;
  std::vector<float> d = s->deepPass();
  uint32_t m = (uint32_t)(d.size() / 4);
  if (n) *n = m;
  if (out4) memcpy(out4, d.data(), (size_t)std::min(m, cap) * 16);
  return ST_OK;
}
st_status oracle_flip_stats(void* h, st_stats* o) {
  Oracle* s = (Oracle*)h;
  o->sc = s->st_sc; o->ovf = s->st_ovf; o->fluid = s->st_fluid; o->vmax = s->st_vmax; o->n = s->N;
  // particles alive at the start of the last step's sort (all slots before the first step)
  o->live = s->steps ? s->st_live : s->N; o->spray_used = s->sctl0; o->steps = s->steps; o->spray_overflow = s->spray_ovf; o->launches = 0;
  return ST_OK;
}
st_status oracle_flip_get_dims(void* h, st_flip_dims* o) {
  Oracle* s = (Oracle*)h;
  o->nx = s->nx; o->ny = s->ny; o->nz = s->nz; o->tx = s->tx; o->ty = s->ty; o->tz = s->tz;
  o->h = (float)s->h; o->x0 = (float)s->bx0; o->y0 = (float)s->by0; o->z0 = (float)s->bz0; o->x1 = (float)s->bx1; o->y1 = (float)s->by1; o->z1 = (float)s->bz1;
  return ST_OK;
}
st_status oracle_flip_read_grid(void* h, const st_flip_grid* g) {
  Oracle* s = (Oracle*)h;
  uint32_t NX = s->tx * 8, NY = s->ty * 8, NZ = s->tz * 8;
  if (g->tile_on) for (int t = 0; t < s->ntiles; t++) g->tile_on[t] = s->alloc[t];
  for (uint32_t k = 0; k < NZ; k++) for (uint32_t j = 0; j < NY; j++) for (uint32_t i = 0; i < NX; i++) {
    size_t o = (size_t)i + NX * ((size_t)j + NY * k);
    uint32_t c = s->cellIdx((int)i, (int)j, (int)k);
    bool spare = (c >> 9) == s->spare();
    if (g->cnt) g->cnt[o] = spare ? 0 : s->cnt[c];
    if (g->ctype) g->ctype[o] = spare ? 0 : s->ctype[c];
    if (g->pres) g->pres[o] = spare ? 0.0f : s->pres[c];
    if (g->rhs) g->rhs[o] = spare ? 8.0f : s->rhs[c];
    for (int a = 0; a < 3; a++) {
      if (g->vn) g->vn[o * 3 + a] = spare ? 0.0f : bitsf(s->accV[c * 3 + a]);
      if (g->vo) g->vo[o * 3 + a] = spare ? 0.0f : bitsf(s->accW[c * 3 + a]);
      if (g->velg) g->velg[o * 3 + a] = spare ? 0.0f : s->velG[c * 3 + a];
    }
  }
  return ST_OK;
}
st_status oracle_flip_save_state(void* h, float* pos4, float* vel4, uint32_t* pid, uint32_t cap, uint32_t* n) {
  Oracle* s = (Oracle*)h; if (n) *n = s->N;
  uint32_t m = std::min(cap, s->N);
  if (pos4) memcpy(pos4, s->pos.data(), (size_t)m * 16);
  if (vel4) memcpy(vel4, s->vel.data(), (size_t)m * 16);
  if (pid) memcpy(pid, s->pid.data(), (size_t)m * 4);
  return ST_OK;
}
st_status oracle_flip_load_state(void* h, const float* pos4, const float* vel4, const uint32_t* pid, uint32_t n, double t, uint32_t seed) {
  Oracle* s = (Oracle*)h; if (n > s->maxN) return ST_BAD_ARG;
  s->N = n; s->ring = 0;
  memcpy(s->pos.data(), pos4, (size_t)n * 16); memcpy(s->vel.data(), vel4, (size_t)n * 16); memcpy(s->pid.data(), pid, (size_t)n * 4);
  s->tm = t; s->seed = seed;
  return ST_OK;
}
st_status oracle_flip_nb_fills(void* h, const float* boxes6, uint32_t nbox, const float* sph4, uint32_t nsph, uint32_t mode) {
  Oracle* s = (Oracle*)h;
  if (mode != 2) s->fillsPacked.clear();   // water added to a running tank adds to the fills (src/shared.js:849)
  for (uint32_t k = 0; k < nbox; k++) {
    const float* b = &boxes6[k * 6];
    float f[8] = {1, b[0], b[1], b[2], b[3], b[4], b[5], 0}; s->fillsPacked.insert(s->fillsPacked.end(), f, f + 8);
  }
  for (uint32_t k = 0; k < nsph; k++) {
    const float* q = &sph4[k * 4];
    float f[8] = {2, q[0], q[1], q[2], q[3], 0, 0, 0}; s->fillsPacked.insert(s->fillsPacked.end(), f, f + 8);
  }
  s->nbInit = mode ? mode : 1;
  return ST_OK;
}
// nbSeed's sim.nbFillVols (src/shared.js:849-850): water meshes whose distance grids start the depth field
st_status oracle_flip_nb_fill_vols(void* h, const st_collider* vols, uint32_t n, uint32_t mode) {
  Oracle* s = (Oracle*)h;
  if (n && !vols) return ST_BAD_ARG;
  for (uint32_t k = 0; k < n; k++)
    if (!vols[k].sdf || !vols[k].sdf->data) return ST_BAD_ARG;
  if (mode != 2) s->fillVols.clear();
  for (uint32_t k = 0; k < n; k++) {
    Oracle::FillVol f;
    f.sd = *vols[k].sdf;
    f.data.assign(vols[k].sdf->data, vols[k].sdf->data + (size_t)f.sd.dims[0] * f.sd.dims[1] * f.sd.dims[2]);
    f.c = vols[k];
    for (int a = 0; a < 3; a++) { f.c.vel[a] = 0.0f; f.c.ang[a] = 0.0f; }
    s->fillVols.push_back(std::move(f));
  }
  s->nbInit = mode ? mode : 1;
  return ST_OK;
}
uint32_t oracle_flip_spray_overflow(void* h) { return ((Oracle*)h)->spray_ovf; }

}  // extern "C"
