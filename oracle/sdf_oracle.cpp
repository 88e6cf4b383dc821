// sdf_oracle.cpp - CPU restatement of buildSDF (src/shared.js:98-181), used ONLY as the checker of the device builder
// (st_build_sdf). Test infrastructure: the product never links or calls it.
//
// It follows the reference step by step in doubles into a float array, in the reference's order: exact squared
// distances within 2.5 voxels of each triangle (ptTriDist2, src/shared.js:69-96: Ericson's closest point on a
// triangle), square roots, the forward and backward chamfer sweeps in raster order, then the inside test from the
// sorted crossings of lines along x. Math.hypot is written as the square root of the sum of squares.
// Build with -ffp-contract=off (no FMA).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../include/splashtank_cuda.h"

namespace {

double ptTriDist2(double px, double py, double pz, const double* a, const double* b, const double* c) {
  const double abx = b[0] - a[0], aby = b[1] - a[1], abz = b[2] - a[2], acx = c[0] - a[0], acy = c[1] - a[1], acz = c[2] - a[2];
  const double apx = px - a[0], apy = py - a[1], apz = pz - a[2];
  const double d1 = abx * apx + aby * apy + abz * apz, d2 = acx * apx + acy * apy + acz * apz;
  double q[3];
  auto set = [&](double x, double y, double z) { q[0] = x; q[1] = y; q[2] = z; };
  if (d1 <= 0 && d2 <= 0) { set(a[0], a[1], a[2]); }
  else {
    const double bpx = px - b[0], bpy = py - b[1], bpz = pz - b[2];
    const double d3 = abx * bpx + aby * bpy + abz * bpz, d4 = acx * bpx + acy * bpy + acz * bpz;
    if (d3 >= 0 && d4 <= d3) { set(b[0], b[1], b[2]); }
    else {
      const double vc = d1 * d4 - d3 * d2;
      if (vc <= 0 && d1 >= 0 && d3 <= 0) { const double v = d1 / (d1 - d3); set(a[0] + abx * v, a[1] + aby * v, a[2] + abz * v); }
      else {
        const double cpx = px - c[0], cpy = py - c[1], cpz = pz - c[2];
        const double d5 = abx * cpx + aby * cpy + abz * cpz, d6 = acx * cpx + acy * cpy + acz * cpz;
        if (d6 >= 0 && d5 <= d6) { set(c[0], c[1], c[2]); }
        else {
          const double vb = d5 * d2 - d1 * d6;
          if (vb <= 0 && d2 >= 0 && d6 <= 0) { const double w = d2 / (d2 - d6); set(a[0] + acx * w, a[1] + acy * w, a[2] + acz * w); }
          else {
            const double va = d3 * d6 - d5 * d4;
            if (va <= 0 && d4 - d3 >= 0 && d5 - d6 >= 0) {
              const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
              set(b[0] + (c[0] - b[0]) * w, b[1] + (c[1] - b[1]) * w, b[2] + (c[2] - b[2]) * w);
            } else {
              const double den = 1 / (va + vb + vc), v = vb * den, w = vc * den;
              set(a[0] + abx * v + acx * w, a[1] + aby * v + acy * w, a[2] + abz * v + acz * w);
            }
          }
        }
      }
    }
  }
  const double dx = px - q[0], dy = py - q[1], dz = pz - q[2];
  return dx * dx + dy * dy + dz * dz;
}

}  // namespace

extern "C" st_status oracle_build_sdf(const st_mesh* mesh, st_sdf_build* b) {
  if (!mesh || !b || b->size != sizeof(st_sdf_build)) return ST_BAD_ARG;
  double lo[3] = {1e9, 1e9, 1e9}, hi[3] = {-1e9, -1e9, -1e9};   // meshBounds
  for (uint32_t p = 0; p < mesh->nv; p++)
    for (int k = 0; k < 3; k++) { const double x = mesh->v[3 * p + k]; if (x < lo[k]) lo[k] = x; if (x > hi[k]) hi[k] = x; }
  if (mesh->nv == 0) return ST_BAD_ARG;   // the reference's grid would have a negative size (a RangeError)
  double cell = b->cell != 0.0 ? b->cell : 0.025;
  for (int k = 0; k < 3; k++) { lo[k] -= b->margin; hi[k] += b->margin; }
  if (!(cell > 0) || !(hi[0] - lo[0] >= 0) || !(hi[1] - lo[1] >= 0) || !(hi[2] - lo[2] >= 0)) return ST_BAD_ARG;
  int dims[3];
  auto setDims = [&]() { for (int k = 0; k < 3; k++) dims[k] = (int)std::ceil((hi[k] - lo[k]) / cell) + 1; };
  setDims();
  while ((double)dims[0] * dims[1] * dims[2] > 2.6e6) { cell *= 1.25; setDims(); }
  for (int k = 0; k < 3; k++) { b->dims[k] = (uint32_t)dims[k]; b->origin[k] = lo[k]; }
  b->cell = cell;
  const int nx = dims[0], ny = dims[1], nz = dims[2];
  const size_t nxy = (size_t)nx * ny, N = nxy * nz;
  if (!b->data) return ST_OK;
  if (b->cap < N) return ST_OVERFLOW;
  const double ic = 1 / cell;
  std::vector<double> T;   // meshTris: fan triangulation
  {
    size_t at = 0;
    for (uint32_t f = 0; f < mesh->nf; f++) {
      for (uint32_t k = 1; k + 1 < mesh->len[f]; k++)
        for (uint32_t id : {mesh->idx[at], mesh->idx[at + k], mesh->idx[at + k + 1]}) T.insert(T.end(), mesh->v + 3 * id, mesh->v + 3 * id + 3);
      at += mesh->len[f];
    }
  }
  const size_t nt = T.size() / 9;
  float* data = b->data;
  std::fill(data, data + N, 1e30f);
  const double B = 2.5 * cell, B2 = B * B;
  for (size_t q = 0; q < nt; q++) {
    const double *a = &T[9 * q], *bb = a + 3, *c = a + 6;
    const double ux = bb[0] - a[0], uy = bb[1] - a[1], uz = bb[2] - a[2], vx = c[0] - a[0], vy = c[1] - a[1], vz = c[2] - a[2];
    double px = uy * vz - uz * vy, py = uz * vx - ux * vz, pz = ux * vy - uy * vx;
    const double pl = std::sqrt(px * px + py * py + pz * pz);
    if (pl > 0) { px /= pl; py /= pl; pz /= pl; }
    int r0[3], r1[3];
    for (int k = 0; k < 3; k++) {
      const double mn = std::min(std::min(a[k], bb[k]), c[k]), mx = std::max(std::max(a[k], bb[k]), c[k]);
      r0[k] = (int)std::max(0.0, std::min((double)(dims[k] - 1), std::floor((mn + -B - lo[k]) * ic)));
      r1[k] = (int)std::max(0.0, std::min((double)(dims[k] - 1), std::ceil((mx + B - lo[k]) * ic)));
    }
    for (int k = r0[2]; k <= r1[2]; k++) {
      const double z = lo[2] + k * cell;
      for (int j = r0[1]; j <= r1[1]; j++) {
        const double y = lo[1] + j * cell;
        const size_t base = (size_t)j * nx + (size_t)k * nxy;
        for (int i = r0[0]; i <= r1[0]; i++) {
          const double x = lo[0] + i * cell;
          if (pl > 0) { const double e = (x - a[0]) * px + (y - a[1]) * py + (z - a[2]) * pz; if (e * e > B2) continue; }
          const double d2 = ptTriDist2(x, y, z, a, bb, c);
          if (d2 < (double)data[base + i]) data[base + i] = (float)d2;
        }
      }
    }
  }
  for (size_t i = 0; i < N; i++) if ((double)data[i] < 1e29) data[i] = (float)std::sqrt((double)data[i]);
  int oi[13], oj[13], ok[13];
  float ow[13];
  {
    int o = 0;
    for (int dk = -1; dk <= 0; dk++)
      for (int dj = -1; dj <= 1; dj++)
        for (int di = -1; di <= 1; di++)
          if (dk < 0 || dj < 0 || (dj == 0 && di < 0)) {
            oi[o] = di; oj[o] = dj; ok[o] = dk; ow[o] = (float)(cell * std::sqrt((double)(di * di + dj * dj + dk * dk))); o++;
          }
  }
  for (int pass = 0; pass < 2; pass++) {   // raster order, then reversed
    const int sg = pass ? -1 : 1;
    for (int kk = 0; kk < nz; kk++) {
      const int k = pass ? nz - 1 - kk : kk;
      for (int jj = 0; jj < ny; jj++) {
        const int j = pass ? ny - 1 - jj : jj;
        for (int ii = 0; ii < nx; ii++) {
          const int i = pass ? nx - 1 - ii : ii;
          const size_t idx = (size_t)i + (size_t)j * nx + (size_t)k * nxy;
          double v = data[idx];
          if (v <= B) continue;
          for (int o = 0; o < 13; o++) {
            const int ni = i + sg * oi[o], nj = j + sg * oj[o], nk = k + sg * ok[o];
            if (ni < 0 || nj < 0 || nk < 0 || ni >= nx || nj >= ny || nk >= nz) continue;
            const double c2 = (double)data[(size_t)ni + (size_t)nj * nx + (size_t)nk * nxy] + (double)ow[o];
            if (c2 < v) v = c2;
          }
          data[idx] = (float)v;
        }
      }
    }
  }
  const double ey = 0.000137 * cell, ez = 0.000271 * cell;
  std::vector<std::vector<double>> rows((size_t)ny * nz);
  for (size_t q = 0; q < nt; q++) {
    const double *a = &T[9 * q], *bb = a + 3, *c = a + 6;
    const double area = (bb[1] - a[1]) * (c[2] - a[2]) - (bb[2] - a[2]) * (c[1] - a[1]);
    if (std::fabs(area) < 1e-14) continue;
    const int jlo = (int)std::max(0.0, std::ceil((std::min(std::min(a[1], bb[1]), c[1]) - lo[1] - ey) * ic));
    const int jhi = (int)std::min((double)(ny - 1), std::floor((std::max(std::max(a[1], bb[1]), c[1]) - lo[1] - ey) * ic));
    const int klo = (int)std::max(0.0, std::ceil((std::min(std::min(a[2], bb[2]), c[2]) - lo[2] - ez) * ic));
    const int khi = (int)std::min((double)(nz - 1), std::floor((std::max(std::max(a[2], bb[2]), c[2]) - lo[2] - ez) * ic));
    for (int k = klo; k <= khi; k++) {
      const double z = lo[2] + k * cell + ez;
      for (int j = jlo; j <= jhi; j++) {
        const double y = lo[1] + j * cell + ey;
        const double w0 = ((c[1] - bb[1]) * (z - bb[2]) - (c[2] - bb[2]) * (y - bb[1])) / area;
        const double w1 = ((a[1] - c[1]) * (z - c[2]) - (a[2] - c[2]) * (y - c[1])) / area, w2 = 1 - w0 - w1;
        if (w0 < 0 || w1 < 0 || w2 < 0) continue;
        rows[(size_t)j + (size_t)ny * k].push_back(w0 * a[0] + w1 * bb[0] + w2 * c[0]);
      }
    }
  }
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++) {
      std::vector<double>& xs = rows[(size_t)j + (size_t)ny * k];
      if (xs.empty()) continue;
      std::sort(xs.begin(), xs.end());
      size_t m = 0;
      const size_t base = (size_t)j * nx + (size_t)k * nxy;
      for (int i = 0; i < nx; i++) {
        const double x = lo[0] + i * cell;
        while (m < xs.size() && xs[m] < x) m++;
        if (m & 1) data[base + i] = -data[base + i];
      }
    }
  return ST_OK;
}
