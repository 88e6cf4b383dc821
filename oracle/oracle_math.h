// oracle_math.h - f32 vector helpers and the collider distance lookup shared by the CPU restatements (test
// infrastructure only: the oracle is the parity checker and the timed CPU baseline, never part of the product).
// WGSL semantics where C differs: select/clamp/min/max as written below, i32()/u32() saturating truncation.
#ifndef ORACLE_MATH_H
#define ORACLE_MATH_H
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

struct V3 { float x, y, z; };
inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
inline V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
inline V3 operator/(V3 a, V3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float length(V3 a) { return sqrtf(dot(a, a)); }
inline float fmin_(float a, float b) { return a < b ? a : b; }
inline float fmax_(float a, float b) { return a > b ? a : b; }
inline float clampf(float x, float lo, float hi) { return fmin_(fmax_(x, lo), hi); }
inline V3 vmin(V3 a, V3 b) { return v3(fmin_(a.x, b.x), fmin_(a.y, b.y), fmin_(a.z, b.z)); }
inline V3 vmax(V3 a, V3 b) { return v3(fmax_(a.x, b.x), fmax_(a.y, b.y), fmax_(a.z, b.z)); }
inline V3 vclamp(V3 a, V3 lo, V3 hi) { return vmin(vmax(a, lo), hi); }
inline V3 vfloor(V3 a) { return v3(floorf(a.x), floorf(a.y), floorf(a.z)); }
inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline V3 vmix(V3 a, V3 b, float t) { return v3(mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t)); }
inline V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline float smoothstep(float e0, float e1, float x) { float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f); return t * t * (3.0f - 2.0f * t); }
inline float comp(V3 a, int ax) { return ax == 0 ? a.x : (ax == 1 ? a.y : a.z); }
inline void setc(V3& a, int ax, float v) { if (ax == 0) a.x = v; else if (ax == 1) a.y = v; else a.z = v; }
inline float bitsf(int32_t i) { float f; memcpy(&f, &i, 4); return f; }
inline int32_t fbits(float f) { int32_t i; memcpy(&i, &f, 4); return i; }
// WGSL u32(f): truncation, saturating at 0 for negative values
inline uint32_t u32f(float f) { return f <= 0.0f ? 0u : (uint32_t)f; }
// WGSL i32(f): truncation, saturating at the ends of the range; NaN gives 0
inline int32_t i32f(float f) {
  if (!(f == f)) return 0;
  if (f >= 2147483648.0f) return 2147483647;
  if (f <= -2147483648.0f) return (int32_t)0x80000000u;
  return (int32_t)f;
}
// a floored coordinate as an index, held in [-2, 2^24] so that index + 1 cannot overflow (in-range values unchanged)
inline int i32idx(float f) { return std::min(std::max(i32f(f), -2), 1 << 24); }

const float DEADY = -1.0e5f;

// sdfEval (src/gpu.js:6-33) on the packed collider records (32 floats each, packColliders src/gpu.js:57-67):
// trilinear distance in the collider's grid frame, extended outside the grid by the distance to it, and the normal
// (the grid gradient inside, the direction out of the grid outside) turned back to world space.
inline void sdfEvalRec(const float* cols, const float* sdfData, uint32_t k, V3 p, float& phi, V3& wn) {
  const float* c = cols + (size_t)k * 32;
  const float* a = c; const float* b = c + 4;
  V3 r0 = v3(c[8], c[9], c[10]), r1 = v3(c[12], c[13], c[14]), r2 = v3(c[16], c[17], c[18]);
  V3 d_ = p - v3(c[20], c[21], c[22]);
  V3 lp = v3(dot(r0, d_), dot(r1, d_), dot(r2, d_));
  V3 g = (lp - v3(b[0], b[1], b[2])) / b[3];
  V3 dims = v3(a[1], a[2], a[3]);
  V3 gc = vclamp(g, v3(0, 0, 0), dims - v3(1.0001f, 1.0001f, 1.0001f));
  V3 fl = vfloor(gc); V3 f = gc - fl;
  uint32_t nx_ = u32f(a[1]), ny_ = u32f(a[2]);
  uint32_t base = u32f(a[0]) + u32f(fl.x) + nx_ * (u32f(fl.y) + ny_ * u32f(fl.z));
  uint32_t s = nx_ * ny_;
  const float* sd = sdfData;
  float v000 = sd[base], v100 = sd[base + 1], v010 = sd[base + nx_], v110 = sd[base + nx_ + 1];
  float v001 = sd[base + s], v101 = sd[base + s + 1], v011 = sd[base + s + nx_], v111 = sd[base + s + nx_ + 1];
  float c00 = mixf(v000, v100, f.x), c10 = mixf(v010, v110, f.x), c01 = mixf(v001, v101, f.x), c11 = mixf(v011, v111, f.x);
  float c0 = mixf(c00, c10, f.y), c1 = mixf(c01, c11, f.y);
  phi = mixf(c0, c1, f.z);
  V3 out = g - gc; V3 gl;
  if (dot(out, out) > 0.0f) {
    float l = length(out); phi += l * b[3]; gl = out / l;
  } else {
    gl = v3(mixf(mixf(v100 - v000, v110 - v010, f.y), mixf(v101 - v001, v111 - v011, f.y), f.z), mixf(c10 - c00, c11 - c01, f.z), c1 - c0);
    float l = length(gl); gl = gl / fmax_(l, 1e-9f);
  }
  wn = r0 * gl.x + r1 * gl.y + r2 * gl.z;
}
#endif
