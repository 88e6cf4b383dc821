// ocean.cpp - the ocean's wave list (oceanWaves, src/shared.js:760-780), computed on the host as the reference does.
//
// 24 linear waves around the peak wavelength, amplitudes from a Pierson-Moskowitz shaped spectrum scaled to the
// significant height (4 standard deviations of the surface), directions spread around the mean direction, wavenumbers
// from the dispersion relation at the water depth (fixed-point iteration). The reference draws the frequencies,
// directions and phases from mulberry32 (Tommy Ettinger's public-domain generator) seeded from the ocean's seed; the
// same integer steps are done here, and the double arithmetic in the reference's order, rounded to f32 at the end.
#include <algorithm>
#include <cmath>
#include <cstdint>

#include "../../include/splashtank_cuda.h"

namespace st {

namespace {
struct Mulberry32 {
  uint32_t a;
  double next() {
    a += 0x6D2B79F5u;
    uint32_t t = (a ^ (a >> 15)) * (1u | a);
    t = (t + (t ^ (t >> 7)) * (61u | t)) ^ t;
    return (double)(t ^ (t >> 14)) / 4294967296.0;
  }
};
int32_t to_int32(double x) {   // ToInt32
  if (!std::isfinite(x)) return 0;
  double m = std::fmod(std::trunc(x), 4294967296.0);
  if (m < 0) m += 4294967296.0;
  return (int32_t)(uint32_t)m;
}
}  // namespace

// 8 floats per wave: kx, kz, amplitude, angular frequency, phase, wavenumber, 0, 0. Returns the number of waves.
int ocean_waves(const st_step_opts* o, double g, double depth, float* w) {
  const int N = 24;
  const double pi = 3.141592653589793;
  int32_t sd = to_int32((double)o->ocean_seed);
  if (sd == 0) sd = 1;                                   // (oc.seed | 0) || 1
  Mulberry32 rnd{(uint32_t)to_int32((double)sd * 7919.0 + 13.0)};
  const double D = std::max(depth, 1e-3), G = std::max(g, 1e-4), lp = std::max((double)o->ocean_length, 1e-3);
  const double kp = 2 * pi / lp, wp = std::sqrt(G * kp * std::tanh(kp * D));
  auto kOf = [&](double om) {
    double k = om * om / G;
    for (int i = 0; i < 40; i++) k = om * om / (G * std::tanh(std::max(k * D, 1e-6)));
    return k;
  };
  const double dir = o->ocean_dir == o->ocean_dir ? (double)o->ocean_dir : 0.0;   // oc.dir || 0
  const double spreadIn = o->ocean_spread == o->ocean_spread ? (double)o->ocean_spread : 0.0;
  const double th0 = dir * pi / 180, spr = std::max(0.0, spreadIn) * pi / 180;
  double k[N], om[N], S[N], th[N], ph[N], sum = 0;
  for (int i = 0; i < N; i++) {
    const double r = 0.6 + 1.6 * (i + rnd.next()) / N;
    om[i] = r * wp;
    k[i] = kOf(om[i]);
    S[i] = std::pow(r, -5) * std::exp(-1.25 * std::pow(r, -4));
    const double r1 = rnd.next(), r2 = rnd.next(), r3 = rnd.next();
    th[i] = th0 + spr * (r1 + r2 + r3 - 1.5) / 1.5;
    ph[i] = rnd.next() * 2 * pi;
    sum += S[i];
  }
  const double hs = o->ocean_height == o->ocean_height ? (double)o->ocean_height : 0.0;
  const double m0 = std::pow(std::max(hs, 0.0) / 4, 2);
  for (int i = 0; i < N; i++) {
    const double a = std::min(std::sqrt(2 * m0 * S[i] / sum), 0.3 / k[i]);
    const double rec[8] = {k[i] * std::cos(th[i]), k[i] * std::sin(th[i]), a, om[i], ph[i], k[i], 0, 0};
    for (int q = 0; q < 8; q++) w[i * 8 + q] = (float)rec[q];
  }
  return N;
}

}  // namespace st

extern "C" int st_ocean_waves(const st_step_opts* o, double depth, float* w) {
  if (!o || !w) return 0;
  return st::ocean_waves(o, (double)o->g, depth, w);
}
