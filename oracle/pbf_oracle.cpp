// pbf_oracle.cpp - CPU restatement of the app's WebGPU position-based fluid engine GpuSim (src/gpu.js:357-476), test
// infrastructure only: the parity checker of the sm_100a PBF engine (st_pbf_*) and a timed CPU baseline. Never linked
// into the product.
//
// GpuSim.step (src/gpu.js:409-428) dispatch by dispatch: predict (:155-161), the grid (:162-206), iterations of lambda
// (:208-251), delta (:253-286) and applyDelta (:288-292), finalize (:293-322), viscosity (:323-353), over particles in
// index order; the passes are in pbf_core.h. packColliders (src/gpu.js:42-70) packs the collider records.
// Parity status: GpuSim runs only as WGSL through WebGPU in a browser, which cannot run here (no graphics stack, no
// Node), so this restatement is not run against the reference itself; where GpuSim and the native baker define the
// same arithmetic (a ball of water away from walls and colliders) the tests compare it with the baker built from the
// reference's own source (baker_oracle.cpp and oracle/_ref/splash_nofma).
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
#include "oracle_math.h"
#include "pbf_core.h"

namespace {

struct Gpbf {
  double d = 0, lo[3] = {}, hi[3] = {};
  PbfConsts c{};
  uint32_t open = 0, maxN = 0, cap = 0, N = 0, ring = 0;
  bool recycle = true;
  int nthreads = 1;
  std::vector<float> pos, vel;   // 4 floats per particle (pos.w speed)
  std::vector<float> cols, sdf;  // packColliders records (32 floats), grids back to back
  std::string sdfSig;

  void pack(const st_pbf_opts* o, uint32_t& nc) {
    nc = std::min(o->ncols, 32u);
    std::string sig;
    std::map<uint32_t, uint32_t> offs;
    uint32_t off = 0;
    for (uint32_t k = 0; k < nc; k++) {
      const st_sdf* sd = o->cols[k].sdf;
      if (!offs.count(sd->id)) { offs[sd->id] = off; off += sd->dims[0] * sd->dims[1] * sd->dims[2]; sig += std::to_string(sd->id) + ","; }
    }
    if (sig != sdfSig) {
      sdf.assign(off, 0.0f);
      for (uint32_t k = 0; k < nc; k++) {
        const st_sdf* sd = o->cols[k].sdf;
        memcpy(&sdf[offs[sd->id]], sd->data, 4ull * sd->dims[0] * sd->dims[1] * sd->dims[2]);
      }
      sdfSig = sig;
    }
    cols.assign((size_t)nc * 32, 0.0f);
    for (uint32_t k = 0; k < nc; k++) {
      const st_collider& cc = o->cols[k];
      const st_sdf* sd = cc.sdf;
      float* f = &cols[(size_t)k * 32];
      f[0] = (float)offs[sd->id]; f[1] = (float)sd->dims[0]; f[2] = (float)sd->dims[1]; f[3] = (float)sd->dims[2];
      f[4] = sd->origin[0]; f[5] = sd->origin[1]; f[6] = sd->origin[2]; f[7] = sd->cell;
      f[8] = cc.R[0]; f[9] = cc.R[3]; f[10] = cc.R[6];
      f[12] = cc.R[1]; f[13] = cc.R[4]; f[14] = cc.R[7];
      f[16] = cc.R[2]; f[17] = cc.R[5]; f[18] = cc.R[8];
      f[20] = cc.pos[0]; f[21] = cc.pos[1]; f[22] = cc.pos[2];
      f[24] = cc.vel[0]; f[25] = cc.vel[1]; f[26] = cc.vel[2];
      f[28] = cc.ang[0]; f[29] = cc.ang[1]; f[30] = cc.ang[2];
    }
  }

  void step(double dt, const st_pbf_opts* o) {
    if (N == 0) return;
    uint32_t nc = 0;
    pack(o, nc);
    const PbfP P = pbfParams(c, d, lo, hi, dt, o->g, o->visc, N, nc, open);
    auto sdfOf = [&](uint32_t k, V3 x, float& phi, V3& wn) { sdfEvalRec(cols.data(), sdf.data(), k, x, phi, wn); };
    auto collide = [&](V3 p) { return pbfCollide(P, sdfOf, nc, p); };
    std::vector<float> prd((size_t)N * 4), bgr((size_t)N * 4, 0.0f), lam(N, 0.0f), dlt, vel2((size_t)N * 4, 0.0f);
    // predict (src/gpu.js:155-161)
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t ii = 0; ii < (int64_t)N; ii++) {
      const size_t i = (size_t)ii;
      if (pos[i * 4 + 1] < DEADY) { for (int a = 0; a < 4; a++) prd[i * 4 + a] = pos[i * 4 + a]; continue; }
      const V3 v = v3(vel[i * 4], vel[i * 4 + 1], vel[i * 4 + 2]) + v3(0.0f, -P.gravity * P.dt, 0.0f);
      vel[i * 4] = v.x; vel[i * 4 + 1] = v.y; vel[i * 4 + 2] = v.z; vel[i * 4 + 3] = 0.0f;
      const V3 q = collide(v3(pos[i * 4], pos[i * 4 + 1], pos[i * 4 + 2]) + v * P.dt);
      prd[i * 4] = q.x; prd[i * 4 + 1] = q.y; prd[i * 4 + 2] = q.z; prd[i * 4 + 3] = 0.0f;
    }
    // the grid (src/gpu.js:162-206), then the iterations (src/gpu.js:425)
    PbfGrid G;
    pbfBuildGrid(P, prd.data(), 4, N, G);
    for (int it = 0; it < o->iters; it++) pbfIteration(P, sdfOf, nc, collide, G, prd.data(), N, lam, bgr, dlt, nthreads);
    // finalize (src/gpu.js:293-322)
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t ii = 0; ii < (int64_t)N; ii++) {
      const size_t i = (size_t)ii;
      if (pos[i * 4 + 1] < DEADY) { for (int a = 0; a < 4; a++) vel2[i * 4 + a] = 0.0f; continue; }
      const V3 p = v3(pos[i * 4], pos[i * 4 + 1], pos[i * 4 + 2]), q = v3(prd[i * 4], prd[i * 4 + 1], prd[i * 4 + 2]);
      const V3 vo = v3(vel[i * 4], vel[i * 4 + 1], vel[i * 4 + 2]);
      V3 v = (q - p) / P.dt;
      const V3 g = v3(bgr[i * 4], bgr[i * 4 + 1], bgr[i * 4 + 2]);
      const float gm2 = dot(g, g);
      if (gm2 > 1e-6f) {
        const V3 nrm = (v3(0, 0, 0) - g) * (1.0f / sqrtf(gm2));
        const float vn0 = dot(vo, nrm);
        if (vn0 < 0.0f) {
          const float vn = dot(v, nrm);
          const float lim = -vn0 * P.rest;
          if (vn > lim) v = v - nrm * (vn - lim);
        }
      }
      const float s2 = dot(v, v);
      if (s2 > P.vmax * P.vmax) v = v * (P.vmax * (1.0f / sqrtf(s2)));
      vel2[i * 4] = v.x; vel2[i * 4 + 1] = v.y; vel2[i * 4 + 2] = v.z; vel2[i * 4 + 3] = 0.0f;
      const uint32_t ob = P.open;
      if (ob != 0u && (((ob & 1u) && q.x < P.bx0) || ((ob & 2u) && q.x > P.bx1) || ((ob & 4u) && q.y < P.by0) || ((ob & 8u) && q.y > P.by1) ||
                       ((ob & 16u) && q.z < P.bz0) || ((ob & 32u) && q.z > P.bz1))) {
        pos[i * 4] = 0.0f; pos[i * 4 + 1] = -1.0e6f; pos[i * 4 + 2] = 0.0f; pos[i * 4 + 3] = 0.0f;
        for (int a = 0; a < 4; a++) vel2[i * 4 + a] = 0.0f;
        continue;
      }
      pos[i * 4] = q.x; pos[i * 4 + 1] = q.y; pos[i * 4 + 2] = q.z; pos[i * 4 + 3] = 0.0f;
    }
    // viscosity (src/gpu.js:323-353)
    std::vector<float> nvel((size_t)N * 4, 0.0f), npos(pos);
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t ii = 0; ii < (int64_t)N; ii++) {
      const uint32_t i = (uint32_t)ii;
      if (pos[i * 4 + 1] < DEADY) continue;   // vel 0
      const V3 pi = v3(pos[i * 4], pos[i * 4 + 1], pos[i * 4 + 2]), vi = v3(vel2[i * 4], vel2[i * 4 + 1], vel2[i * 4 + 2]);
      V3 a = v3(0, 0, 0);
      if (P.visc > 0.0f) {
        pbfRows(P, G, G.cid[i], [&](uint32_t s) {
          const uint32_t j = G.sorted[s];
          if (j == i) return;
          const V3 dd = pi - v3(pos[j * 4], pos[j * 4 + 1], pos[j * 4 + 2]);
          const float r2 = dot(dd, dd);
          if (r2 >= P.h2) return;
          const float tt = P.h2 - r2;
          a = a + (v3(vel2[j * 4], vel2[j * 4 + 1], vel2[j * 4 + 2]) - vi) * (P.poly * tt * tt * tt * P.irho);
        });
      }
      const V3 nv = vi + a * P.visc;
      nvel[i * 4] = nv.x; nvel[i * 4 + 1] = nv.y; nvel[i * 4 + 2] = nv.z;
      npos[i * 4 + 3] = length(nv);
    }
    vel.swap(nvel);
    pos.swap(npos);
  }
};

}  // namespace

extern "C" {
st_status oracle_pbf_create(const st_pbf_desc* ds, void** out) {
  if (!ds || !out || ds->size != sizeof(st_pbf_desc) || !(ds->d > 0) || ds->max_n == 0) return ST_BAD_ARG;
  Gpbf* s = new Gpbf();
  s->d = ds->d;
  const double sz[3] = {ds->box[0] > 0 ? ds->box[0] : 3.0, ds->box[1] > 0 ? ds->box[1] : 2.6, ds->box[2] > 0 ? ds->box[2] : 3.0};
  s->lo[0] = -sz[0] / 2; s->hi[0] = sz[0] / 2; s->lo[1] = 0.0; s->hi[1] = sz[1]; s->lo[2] = -sz[2] / 2; s->hi[2] = sz[2] / 2;
  s->open = ds->open;
  s->maxN = s->cap = ds->max_n;
  s->c = pbfConsts(s->d, ds->eps_k, ds->wall_k);
  s->pos.assign((size_t)s->maxN * 4, 0.0f);
  s->vel.assign((size_t)s->maxN * 4, 0.0f);
  *out = s;
  return ST_OK;
}
void oracle_pbf_destroy(void* h) { delete (Gpbf*)h; }
void oracle_pbf_set_threads(void* h, int n) { ((Gpbf*)h)->nthreads = n < 1 ? 1 : n; }
// GpuSim.add (src/gpu.js:390-402)
st_status oracle_pbf_add(void* h, const float* p3, const float* v3_, uint32_t n, uint32_t* added) {
  Gpbf* s = (Gpbf*)h;
  uint32_t k = 0;
  for (; k < n; k++) {
    uint32_t i;
    if (s->N < s->cap) i = s->N++;
    else if (s->recycle && s->cap) { i = s->ring++; if (s->ring >= s->cap) s->ring = 0; }
    else break;
    const float vx = v3_ ? v3_[k * 3] : 0.0f, vy = v3_ ? v3_[k * 3 + 1] : 0.0f, vz = v3_ ? v3_[k * 3 + 2] : 0.0f;
    float* p = &s->pos[(size_t)i * 4];
    float* v = &s->vel[(size_t)i * 4];
    p[0] = p3[k * 3]; p[1] = p3[k * 3 + 1]; p[2] = p3[k * 3 + 2]; p[3] = (float)std::sqrt((double)vx * vx + (double)vy * vy + (double)vz * vz);
    v[0] = vx; v[1] = vy; v[2] = vz; v[3] = 0.0f;
  }
  if (added) *added = k;
  return ST_OK;
}
st_status oracle_pbf_set_cap(void* h, uint32_t c) {
  Gpbf* s = (Gpbf*)h;
  s->cap = std::min(c, s->maxN);
  if (s->N > s->cap) s->N = s->cap;
  if (s->ring >= s->cap) s->ring = 0;
  return ST_OK;
}
st_status oracle_pbf_clear(void* h) { Gpbf* s = (Gpbf*)h; s->N = 0; s->ring = 0; return ST_OK; }
st_status oracle_pbf_set_recycle(void* h, int32_t on) { ((Gpbf*)h)->recycle = on != 0; return ST_OK; }
st_status oracle_pbf_step(void* h, double dt, const st_pbf_opts* o) {
  if (!o || o->size != sizeof(st_pbf_opts) || (o->ncols && !o->cols) || o->iters < 1 || !(dt > 0)) return ST_BAD_ARG;
  Gpbf* s = (Gpbf*)h;
  if (!s->N) return ST_NOT_READY;
  s->step(dt, o);
  return ST_OK;
}
st_status oracle_pbf_read(void* h, float* pos4, float* vel4, uint32_t cap, uint32_t* n) {
  Gpbf* s = (Gpbf*)h;
  if (n) *n = s->N;
  const uint32_t m = std::min(cap, s->N);
  if (pos4) memcpy(pos4, s->pos.data(), (size_t)m * 16);
  if (vel4) memcpy(vel4, s->vel.data(), (size_t)m * 16);
  return ST_OK;
}
void* oracle_pbf_stream(void*) { return nullptr; }
}
