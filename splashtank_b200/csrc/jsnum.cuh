// jsnum.cuh - JavaScript number arithmetic on the device, for outputs the reference computes in JS doubles
// (packFrameBuf, packSprayFrame / packSprayJS, packDeep): Math.round, ToInt32, ToUint8 and the uint16 quantiser.
#pragma once
#include <cstdint>

namespace st {

// Math.round: the nearest integer, halves up (x - floor(x) is exact, so this is the rounding of the value itself)
__device__ __forceinline__ double jsRound(double x) {
  const double r = floor(x);
  return x - r >= 0.5 ? r + 1.0 : r;
}
// Math.max(0, Math.min(65535, Math.round((v - lo) * k)))
__device__ __forceinline__ uint16_t q16(double v, double lo, double k) {
  const double r = jsRound((v - lo) * k);
  return (uint16_t)(r < 0.0 ? 0.0 : (r > 65535.0 ? 65535.0 : r));
}
// ToInt32 (what `| 0`, `<<` and `|` do to a number): NaN and infinities give 0, the rest is truncated modulo 2^32
__device__ __forceinline__ int32_t toInt32(double s) {
  if (!(s == s) || isinf(s)) return 0;
  double m = fmod(trunc(s), 4294967296.0);
  if (m < 0.0) m += 4294967296.0;
  return (int32_t)(uint32_t)m;
}
// a Uint8Array store: ToUint8 (truncate, then modulo 256)
__device__ __forceinline__ uint8_t toU8(double s) { return (uint8_t)(toInt32(s) & 0xff); }

}  // namespace st
