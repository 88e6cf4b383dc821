// drips.cpp - drip samples on a collider's surface (dripSamples, src/flip/bake.js:19-40), computed on the host once per
// set of colliders, as the reference does.
//
// The reference computes them in JavaScript doubles from the distance grid and stores them as a Float32Array; the
// same double operations are done here, in the same order, with the same seeded generator (the Park-Miller minimal
// standard, seed 7 + id). Math.hypot is written as the square root of the sum of squares: ECMAScript leaves the last
// bit of Math.hypot to the engine, and the result is rounded to f32 afterwards.
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/splashtank_cuda.h"

namespace st {

static double js_round(double x) {   // Math.round: the nearest integer, halves up
  const double r = std::floor(x);
  return x - r >= 0.5 ? r + 1.0 : r;
}

// 8 floats per sample: local position, collider number k, local normal, wetness 0 (dry)
void drip_samples(const st_sdf* sdf, double h, uint32_t k, std::vector<float>& out) {
  const int nx = (int)sdf->dims[0], ny = (int)sdf->dims[1], nz = (int)sdf->dims[2];
  const double c = sdf->cell;
  const double o0 = sdf->origin[0], o1 = sdf->origin[1], o2 = sdf->origin[2];
  const float* d = sdf->data;
  auto at = [&](int i, int j, int q) -> double {
    const int ci = std::min(nx - 1, std::max(0, i)), cj = std::min(ny - 1, std::max(0, j)), cq = std::min(nz - 1, std::max(0, q));
    return (double)d[(size_t)ci + (size_t)nx * ((size_t)cj + (size_t)ny * (size_t)cq)];
  };
  std::vector<double> pts;
  for (int q = 1; q < nz - 1; q++)
    for (int j = 1; j < ny - 1; j++)
      for (int i = 1; i < nx - 1; i++) {
        const double v = (double)d[(size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * (size_t)q)];
        if (std::fabs(v) > 0.6 * c) continue;
        double gx = at(i + 1, j, q) - at(i - 1, j, q), gy = at(i, j + 1, q) - at(i, j - 1, q), gz = at(i, j, q + 1) - at(i, j, q - 1);
        const double gl = std::sqrt(gx * gx + gy * gy + gz * gz);
        if (gl < 1e-9) continue;
        gx /= gl;
        gy /= gl;
        gz /= gl;
        pts.push_back(o0 + i * c - gx * v);
        pts.push_back(o1 + j * c - gy * v);
        pts.push_back(o2 + q * c - gz * v);
        pts.push_back(gx);
        pts.push_back(gy);
        pts.push_back(gz);
      }
  const double nsurf = (double)(pts.size() / 6);
  const double want = std::max(100.0, std::min(6000.0, js_round(nsurf * c * c / (h * h))));
  const double step = std::max(1.0, nsurf / want);
  double sd = 7.0 + (double)(int32_t)sdf->id;
  auto rnd = [&]() { sd = std::fmod(sd * 16807.0, 2147483647.0); return sd / 2147483647.0; };
  for (double t = rnd() * step; t < nsurf; t += step) {
    const size_t i = (size_t)std::floor(t) * 6;
    const float rec[8] = {(float)pts[i], (float)pts[i + 1], (float)pts[i + 2], (float)k,
                          (float)pts[i + 3], (float)pts[i + 4], (float)pts[i + 5], 0.0f};
    out.insert(out.end(), rec, rec + 8);
  }
}

}  // namespace st
