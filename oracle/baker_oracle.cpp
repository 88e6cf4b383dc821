// baker_oracle.cpp - CPU restatement of the reference's native PBF baker (native/splash.cpp), test infrastructure only:
// it pins the GpuSim restatement (pbf_oracle.cpp) to the reference's own compiled code where the two engines define
// the same computation, and it is the CPU baseline of the baker's scenes. Never linked into the product.
//
// It restates Sim of native/splash.cpp (constants :50-71, collide :95-116, bnd :117-148, buildNeighbors :149-176,
// solve :177-211, step :212-247) and its fillBox jitter (:84-89, mt19937 seeded 12345). Parity status: pinned
// against the reference itself - tests build native/splash.cpp unchanged (oracle/Makefile -> oracle/_ref/splash),
// run it on a scene file and compare its SPLC frames (16-bit positions) with this restatement. The reference binary
// is built with -O3 -march=native, so the compiler may fuse multiply-adds; this file does not
// (-ffp-contract=off), so the comparison with the binary is to the frame quantum, while the CUDA kernels match this
// file bit for bit.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/splashtank_cuda.h"

// the baker's analytic colliders and step options (Runner's objects, native/splash.cpp:22, 255-262)
struct baker_desc { uint32_t size; double d; double box[3]; uint32_t max_n; };
struct baker_col { int32_t kind; float x, y, z, r, hx, hy, hz, yaw; };   // kind 0 sphere (r), 1 box (half extents, yaw)
struct baker_opts { uint32_t size; float g, visc; int32_t iters; uint32_t ncols; const baker_col* cols; };

namespace {

struct Col { int t; float x, y, z, r, hx, hy, hz, c, s; };   // native/splash.cpp:22

struct Pbf {
  float d, h, h2, poly, spiky, W0, rho0, eps, c0, Gh, margin, rest = 0.1f;
  float X0, X1, Y0, Y1, Z0, Z1;
  int nx, ny, nz, N = 0;
  uint32_t cap;
  static const int MAXNB = 48;
  std::vector<float> P, V, Q, D, NV, BG, S, lam;
  std::vector<int> cid, sorted, nb, nc, cellStart, cellCount, cursor;
  std::mt19937 rng{12345};
  int nthreads = 1;

  static double Gd(double h, double s) {
    double h2 = h * h, h4 = h2 * h2, h6 = h4 * h2, h8 = h4 * h4;
    double s2 = s * s, s3 = s2 * s, s5 = s3 * s2, s7 = s5 * s2, s9 = s7 * s2;
    return h8 * s - (4.0 / 3) * h6 * s3 + (6.0 / 5) * h4 * s5 - (4.0 / 7) * h2 * s7 + s9 / 9;
  }
  double Gfun(double s) const { return Gd(h, s); }

  void init(const baker_desc* ds) {
    d = (float)ds->d;
    double bx = ds->box[0] > 0 ? ds->box[0] : 3.0, by = ds->box[1] > 0 ? ds->box[1] : 2.6, bz = ds->box[2] > 0 ? ds->box[2] : 3.0;
    X0 = (float)(-bx / 2); X1 = (float)(bx / 2); Y0 = 0.0f; Y1 = (float)by; Z0 = (float)(-bz / 2); Z1 = (float)(bz / 2);
    cap = ds->max_n;
    h = 2.2f * d; h2 = h * h;
    double hh = h;
    double polyD = 315.0 / (64.0 * M_PI * pow(hh, 9)), spikyD = -45.0 / (M_PI * pow(hh, 6));
    poly = (float)polyD; spiky = (float)spikyD; W0 = (float)(polyD * pow(hh * hh, 3));
    nx = (int)ceil((X1 - X0) / h) + 1; ny = (int)ceil((Y1 - Y0) / h) + 1; nz = (int)ceil((Z1 - Z0) / h) + 1;
    size_t cells = (size_t)nx * ny * nz;
    cellCount.assign(cells, 0); cellStart.assign(cells + 1, 0); cursor.assign(cells, 0);
    double r0 = 0, below = 0, sgRest = 0, dd = d;
    for (int i = -3; i <= 3; i++) for (int j = -3; j <= 3; j++) for (int k = -3; k <= 3; k++) {
      double r2 = (i * i + j * j + k * k) * dd * dd;
      if (r2 < hh * hh) { double w = polyD * pow(hh * hh - r2, 3); r0 += w; if (k < 0) below += w; }
    }
    rho0 = (float)r0;
    for (int i = -3; i <= 3; i++) for (int j = -3; j <= 3; j++) for (int k = -3; k <= 3; k++) {
      double r = sqrt((double)(i * i + j * j + k * k)) * dd;
      if (r > 1e-9 && r < hh) { double f = spikyD * (hh - r) * (hh - r) / r / r0 * r; sgRest += f * f; }
    }
    const double epsK = 0.64, wallK = 1.8;   // native/splash.cpp:67-70
    eps = (float)(epsK * sgRest);
    double c0d = (1.0 / (dd * dd * dd)) * (M_PI / 4) * polyD, Ghd = Gd(hh, hh);
    double cont = c0d * (Ghd - Gd(hh, dd / 2));
    c0 = (float)(c0d * (below / cont) * wallK); Gh = (float)Ghd; margin = 0.15f * d;
    P.assign((size_t)cap * 3, 0); V = P; Q = P; D = P; NV = P; BG = P;
    S.assign(cap, 0); lam.assign(cap, 0); cid.assign(cap, 0); sorted.assign(cap, 0); nc.assign(cap, 0); nb.assign((size_t)cap * MAXNB, 0);
  }
  bool add(float x, float y, float z, float vx, float vy, float vz) {
    if ((uint32_t)N >= cap) return false;
    int i3 = N * 3; P[i3] = x; P[i3 + 1] = y; P[i3 + 2] = z; V[i3] = vx; V[i3 + 1] = vy; V[i3 + 2] = vz;
    S[N] = sqrtf(vx * vx + vy * vy + vz * vz); N++; return true;
  }
  float jit() { return (float)(rng() % 10000) / 10000.0f - 0.5f; }
  void fillBox(float x0, float x1, float y0, float y1, float z0, float z1) {   // native/splash.cpp:85-89
    float j = 0.01f * d / 0.12f;
    for (float y = y0 + d / 2; y < y1; y += d) for (float x = x0 + d / 2; x < x1; x += d) for (float z = z0 + d / 2; z < z1; z += d)
      add(x + jit() * j, y + jit() * j, z + jit() * j, 0, 0, 0);
  }
  void collide(const std::vector<Col>& cols) {
    float m = margin, x0 = X0 + m, x1 = X1 - m, y0 = Y0 + m, y1 = Y1 - m, z0 = Z0 + m, z1 = Z1 - m;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int i = 0; i < N; i++) {
      int i3 = i * 3; float x = Q[i3], y = Q[i3 + 1], z = Q[i3 + 2];
      for (const Col& c : cols) {
        if (c.t == 0) {
          float dx = x - c.x, dy = y - c.y, dz = z - c.z, R = c.r + m, d2 = dx * dx + dy * dy + dz * dz;
          if (d2 < R * R) { float dd = sqrtf(d2); if (dd < 1e-6f) y = c.y + R; else { float s = R / dd; x = c.x + dx * s; y = c.y + dy * s; z = c.z + dz * s; } }
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
      Q[i3] = std::min(std::max(x, x0), x1); Q[i3 + 1] = std::min(std::max(y, y0), y1); Q[i3 + 2] = std::min(std::max(z, z0), z1);
    }
  }
  float bR(float p) const { return c0 * (Gh - (float)Gfun(p)); }
  float bD(float p) const { float t = h2 - p * p; t *= t; return -c0 * t * t; }
  void bnd(float x, float y, float z, const std::vector<Col>& cols, float& rho, float& gx, float& gy, float& gz) const {
    rho = gx = gy = gz = 0; float p;
    p = x - X0; if (p < h) { if (p < 0) p = 0; rho += bR(p); gx += bD(p); }
    p = X1 - x; if (p < h) { if (p < 0) p = 0; rho += bR(p); gx -= bD(p); }
    p = y - Y0; if (p < h) { if (p < 0) p = 0; rho += bR(p); gy += bD(p); }
    p = Y1 - y; if (p < h) { if (p < 0) p = 0; rho += bR(p); gy -= bD(p); }
    p = z - Z0; if (p < h) { if (p < 0) p = 0; rho += bR(p); gz += bD(p); }
    p = Z1 - z; if (p < h) { if (p < 0) p = 0; rho += bR(p); gz -= bD(p); }
    for (const Col& c : cols) {
      if (c.t == 0) {
        float dx = x - c.x, dy = y - c.y, dz = z - c.z, dist = sqrtf(dx * dx + dy * dy + dz * dz), phi = dist - c.r;
        if (phi >= h) continue;
        if (phi < 0) phi = 0;
        float dd = bD(phi); rho += bR(phi);
        if (dist > 1e-6f) { float s = dd / dist; gx += dx * s; gy += dy * s; gz += dz * s; } else gy += dd;
      } else {
        float ox = x - c.x, oy = y - c.y, oz = z - c.z, lx = ox * c.c + oz * c.s, lz = -ox * c.s + oz * c.c;
        float qx = fabsf(lx) - c.hx, qy = fabsf(oy) - c.hy, qz = fabsf(lz) - c.hz, nlx, nly, nlz, phi;
        if (qx < 0 && qy < 0 && qz < 0) {
          phi = 0; nlx = nly = nlz = 0;
          if (qx >= qy && qx >= qz) nlx = lx < 0 ? -1 : 1; else if (qy >= qz) nly = oy < 0 ? -1 : 1; else nlz = lz < 0 ? -1 : 1;
        } else {
          float mx = std::max(qx, 0.f), my = std::max(qy, 0.f), mz = std::max(qz, 0.f); phi = sqrtf(mx * mx + my * my + mz * mz);
          if (phi >= h) continue;
          float inv = phi > 1e-9f ? 1 / phi : 0; nlx = (lx < 0 ? -mx : mx) * inv; nly = (oy < 0 ? -my : my) * inv; nlz = (lz < 0 ? -mz : mz) * inv;
        }
        float dd = bD(phi); rho += bR(phi);
        gx += dd * (nlx * c.c - nlz * c.s); gy += dd * nly; gz += dd * (nlx * c.s + nlz * c.c);
      }
    }
  }
  void buildNeighbors() {
    float inv = 1 / h;
    std::fill(cellCount.begin(), cellCount.end(), 0);
    for (int i = 0; i < N; i++) {
      int i3 = i * 3, cx = (int)((Q[i3] - X0) * inv), cy = (int)((Q[i3 + 1] - Y0) * inv), cz = (int)((Q[i3 + 2] - Z0) * inv);
      cx = std::min(std::max(cx, 0), nx - 1); cy = std::min(std::max(cy, 0), ny - 1); cz = std::min(std::max(cz, 0), nz - 1);
      int c = cx + nx * (cy + ny * cz); cid[i] = c; cellCount[c]++;
    }
    size_t cells = (size_t)nx * ny * nz; cellStart[0] = 0;
    for (size_t c = 0; c < cells; c++) { cellStart[c + 1] = cellStart[c] + cellCount[c]; cursor[c] = cellStart[c]; }
    for (int i = 0; i < N; i++) sorted[cursor[cid[i]]++] = i;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int i = 0; i < N; i++) {
      int c = cid[i], cx = c % nx, t = c / nx, cy = t % ny, cz = t / ny, i3 = i * 3;
      float xi = Q[i3], yi = Q[i3 + 1], zi = Q[i3 + 2];
      int xa = std::max(cx - 1, 0), xb = std::min(cx + 1, nx - 1), ya = std::max(cy - 1, 0), yb = std::min(cy + 1, ny - 1), za = std::max(cz - 1, 0), zb = std::min(cz + 1, nz - 1);
      int base = i * MAXNB, n = 0;
      for (int z = za; z <= zb; z++) for (int y = ya; y <= yb; y++) {
        int row = nx * (y + ny * z);
        for (int s = cellStart[row + xa]; s < cellStart[row + xb + 1]; s++) {
          int j = sorted[s]; if (j == i) continue; int j3 = j * 3;
          float dx = xi - Q[j3], dy = yi - Q[j3 + 1], dz = zi - Q[j3 + 2];
          if (dx * dx + dy * dy + dz * dz < h2 && n < MAXNB) nb[base + n++] = j;
        }
      }
      nc[i] = n;
    }
  }
  void solve(const std::vector<Col>& cols) {
    float irho = 1 / rho0, maxD = 0.5f * d, maxD2 = maxD * maxD;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int i = 0; i < N; i++) {
      int i3 = i * 3; float xi = Q[i3], yi = Q[i3 + 1], zi = Q[i3 + 2], rho = W0, gx = 0, gy = 0, gz = 0, sg = 0;
      int base = i * MAXNB, cnt = nc[i];
      for (int k = 0; k < cnt; k++) {
        int j3 = nb[base + k] * 3; float dx = xi - Q[j3], dy = yi - Q[j3 + 1], dz = zi - Q[j3 + 2], r2 = dx * dx + dy * dy + dz * dz;
        if (r2 >= h2) continue;
        float t = h2 - r2; rho += poly * t * t * t; float r = sqrtf(r2); if (r < 1e-7f) continue;
        float hr = h - r, f = spiky * hr * hr / r * irho, fx = f * dx, fy = f * dy, fz = f * dz;
        gx += fx; gy += fy; gz += fz; sg += fx * fx + fy * fy + fz * fz;
      }
      float br, bgx, bgy, bgz; bnd(xi, yi, zi, cols, br, bgx, bgy, bgz);
      rho += br; bgx *= irho; bgy *= irho; bgz *= irho; BG[i3] = bgx; BG[i3 + 1] = bgy; BG[i3 + 2] = bgz;
      gx += bgx; gy += bgy; gz += bgz; sg += bgx * bgx + bgy * bgy + bgz * bgz;
      float C = rho * irho - 1; lam[i] = C > 0 ? -C / (sg + gx * gx + gy * gy + gz * gz + eps) : 0;
    }
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int i = 0; i < N; i++) {
      int i3 = i * 3; float xi = Q[i3], yi = Q[i3 + 1], zi = Q[i3 + 2], li = lam[i];
      float sx = li * BG[i3], sy = li * BG[i3 + 1], sz = li * BG[i3 + 2];
      int base = i * MAXNB, cnt = nc[i];
      for (int k = 0; k < cnt; k++) {
        int j = nb[base + k], j3 = j * 3; float s = li + lam[j]; if (s == 0) continue;
        float dx = xi - Q[j3], dy = yi - Q[j3 + 1], dz = zi - Q[j3 + 2], r2 = dx * dx + dy * dy + dz * dz;
        if (r2 >= h2) continue; float r = sqrtf(r2); if (r < 1e-7f) continue;
        float hr = h - r, f = spiky * hr * hr / r * irho * s; sx += f * dx; sy += f * dy; sz += f * dz;
      }
      float m2 = sx * sx + sy * sy + sz * sz; if (m2 > maxD2) { float k = maxD / sqrtf(m2); sx *= k; sy *= k; sz *= k; }
      D[i3] = sx; D[i3 + 1] = sy; D[i3 + 2] = sz;
    }
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int i = 0; i < N * 3; i++) Q[i] += D[i];
  }
  void step(float dt, float g, int iters, float visc, const std::vector<Col>& cols) {
    if (!N) return;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int i = 0; i < N; i++) { int i3 = i * 3; V[i3 + 1] -= g * dt; for (int a = 0; a < 3; a++) Q[i3 + a] = P[i3 + a] + V[i3 + a] * dt; }
    collide(cols); buildNeighbors();
    for (int it = 0; it < iters; it++) { solve(cols); collide(cols); }
    float idt = 1 / dt, vmax = 12;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int i = 0; i < N; i++) {
      int i3 = i * 3; float vx = (Q[i3] - P[i3]) * idt, vy = (Q[i3 + 1] - P[i3 + 1]) * idt, vz = (Q[i3 + 2] - P[i3 + 2]) * idt;
      float gx = BG[i3], gy = BG[i3 + 1], gz = BG[i3 + 2], gm2 = gx * gx + gy * gy + gz * gz;
      if (gm2 > 1e-6f) {
        float gm = 1 / sqrtf(gm2), nx_ = -gx * gm, ny_ = -gy * gm, nz_ = -gz * gm, vo = V[i3] * nx_ + V[i3 + 1] * ny_ + V[i3 + 2] * nz_;
        if (vo < 0) { float vn = vx * nx_ + vy * ny_ + vz * nz_, lim = -vo * rest; if (vn > lim) { float k = vn - lim; vx -= k * nx_; vy -= k * ny_; vz -= k * nz_; } }
      }
      float s2 = vx * vx + vy * vy + vz * vz; if (s2 > vmax * vmax) { float k = vmax / sqrtf(s2); vx *= k; vy *= k; vz *= k; }
      V[i3] = vx; V[i3 + 1] = vy; V[i3 + 2] = vz;
    }
    if (visc > 0) {
      float irho = 1 / rho0;
#pragma omp parallel for schedule(static) num_threads(nthreads)
      for (int i = 0; i < N; i++) {
        int i3 = i * 3; float xi = Q[i3], yi = Q[i3 + 1], zi = Q[i3 + 2], ax = 0, ay = 0, az = 0; int base = i * MAXNB, cnt = nc[i];
        for (int k = 0; k < cnt; k++) {
          int j3 = nb[base + k] * 3; float dx = xi - Q[j3], dy = yi - Q[j3 + 1], dz = zi - Q[j3 + 2], r2 = dx * dx + dy * dy + dz * dz;
          if (r2 >= h2) continue; float t = h2 - r2, w = poly * t * t * t * irho;
          ax += (V[j3] - V[i3]) * w; ay += (V[j3 + 1] - V[i3 + 1]) * w; az += (V[j3 + 2] - V[i3 + 2]) * w;
        }
        NV[i3] = V[i3] + visc * ax; NV[i3 + 1] = V[i3 + 1] + visc * ay; NV[i3 + 2] = V[i3 + 2] + visc * az;
      }
#pragma omp parallel for schedule(static) num_threads(nthreads)
      for (int i = 0; i < N * 3; i++) V[i] = NV[i];
    }
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int i = 0; i < N; i++) { int i3 = i * 3; P[i3] = Q[i3]; P[i3 + 1] = Q[i3 + 1]; P[i3 + 2] = Q[i3 + 2]; S[i] = sqrtf(V[i3] * V[i3] + V[i3 + 1] * V[i3 + 1] + V[i3 + 2] * V[i3 + 2]); }
  }
};

// Runner::step's collider records (native/splash.cpp:258-259): cos and sin of the yaw taken on the host
std::vector<Col> cols_of(const baker_opts* o) {
  std::vector<Col> cols;
  for (uint32_t k = 0; k < o->ncols; k++) {
    const baker_col& c = o->cols[k];
    if (c.kind == 1) cols.push_back({1, c.x, c.y, c.z, 0, c.hx, c.hy, c.hz, cosf(c.yaw), sinf(c.yaw)});
    else cols.push_back({0, c.x, c.y, c.z, c.r, 0, 0, 0, 0, 0});
  }
  return cols;
}

}  // namespace

extern "C" {
st_status oracle_baker_create(const baker_desc* desc, void** out) {
  if (!desc || !out || desc->size != sizeof(baker_desc) || !(desc->d > 0) || desc->max_n == 0) return ST_BAD_ARG;
  Pbf* s = new Pbf();
  s->init(desc);
  *out = s;
  return ST_OK;
}
void oracle_baker_destroy(void* h) { delete (Pbf*)h; }
void oracle_baker_set_threads(void* h, int n) { ((Pbf*)h)->nthreads = n < 1 ? 1 : n; }
st_status oracle_baker_add(void* h, const float* p3, const float* v3, uint32_t n, uint32_t* added) {
  Pbf* s = (Pbf*)h; uint32_t k = 0;
  for (; k < n; k++) if (!s->add(p3[k * 3], p3[k * 3 + 1], p3[k * 3 + 2], v3 ? v3[k * 3] : 0.f, v3 ? v3[k * 3 + 1] : 0.f, v3 ? v3[k * 3 + 2] : 0.f)) break;
  if (added) *added = k;
  return ST_OK;
}
// the baker's fillBox with its own seeded jitter, so a test can start both sides from the baker's particles
uint32_t oracle_baker_fill_box(void* h, float x0, float x1, float y0, float y1, float z0, float z1) {
  Pbf* s = (Pbf*)h; int n0 = s->N; s->fillBox(x0, x1, y0, y1, z0, z1); return (uint32_t)(s->N - n0);
}
st_status oracle_baker_step(void* h, double dt, const baker_opts* o) {
  if (!o || o->size != sizeof(baker_opts)) return ST_BAD_ARG;
  Pbf* s = (Pbf*)h;
  s->step((float)dt, o->g, o->iters, o->visc, cols_of(o));
  return ST_OK;
}
st_status oracle_baker_read(void* h, float* pos4, float* vel4, uint32_t cap, uint32_t* n) {
  Pbf* s = (Pbf*)h; if (n) *n = (uint32_t)s->N;
  for (int i = 0; i < s->N && (uint32_t)i < cap; i++) {
    if (pos4) { pos4[i * 4] = s->P[i * 3]; pos4[i * 4 + 1] = s->P[i * 3 + 1]; pos4[i * 4 + 2] = s->P[i * 3 + 2]; pos4[i * 4 + 3] = s->S[i]; }
    if (vel4) { vel4[i * 4] = s->V[i * 3]; vel4[i * 4 + 1] = s->V[i * 3 + 1]; vel4[i * 4 + 2] = s->V[i * 3 + 2]; vel4[i * 4 + 3] = 0; }
  }
  return ST_OK;
}
}
