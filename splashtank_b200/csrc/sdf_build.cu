// sdf_build.cu - the signed distance grid of a closed mesh (buildSDF, src/shared.js:98-181), built on the device.
//
// The reference runs three passes in JavaScript doubles into a Float32Array:
//  1. exact squared distances near the surface: each triangle visits the voxels of its box grown by 2.5 cells and
//     keeps the smaller of the stored value and its distance (ptTriDist2, Ericson's closest point on a triangle);
//  2. a forward and a backward chamfer sweep over 13 neighbours each, for the voxels farther than 2.5 cells;
//  3. the sign, from the crossings of lines along x with the mesh.
// Here pass 1 is one CTA per triangle with a 32-bit atomic minimum: the stored value is the f32 rounding of a double,
// and rounding is monotonic, so the minimum over triangles of the rounded distances is what any visiting order stores.
// Pass 2 depends on the raster order (each voxel reads 13 neighbours the same sweep already updated); a voxel (i, j, k)
// only reads voxels with a smaller i + 2 j + 4 k, so one CTA walks those diagonal planes in order with a barrier between
// them and does exactly the reference's arithmetic per voxel. Pass 3 collects each line's crossings (any order: only
// the count of crossings below a voxel matters) and flips the voxels with an odd count.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/splashtank_cuda.h"
#include "common.cuh"

namespace st {

struct SdfGrid {
  double lo[3], cell, ic, B, B2;
  int nx, ny, nz;
};

// Ericson's closest point on a triangle (Real-Time Collision Detection, 5.1.5), the reference's ptTriDist2
// (src/shared.js:69-96) operation for operation in doubles
__device__ double ptTriDist2(double px, double py, double pz, const double* a, const double* b, const double* c) {
  const double abx = b[0] - a[0], aby = b[1] - a[1], abz = b[2] - a[2], acx = c[0] - a[0], acy = c[1] - a[1], acz = c[2] - a[2];
  const double apx = px - a[0], apy = py - a[1], apz = pz - a[2];
  const double d1 = abx * apx + aby * apy + abz * apz, d2 = acx * apx + acy * apy + acz * apz;
  double qx, qy, qz;
  if (d1 <= 0 && d2 <= 0) { qx = a[0]; qy = a[1]; qz = a[2]; }
  else {
    const double bpx = px - b[0], bpy = py - b[1], bpz = pz - b[2];
    const double d3 = abx * bpx + aby * bpy + abz * bpz, d4 = acx * bpx + acy * bpy + acz * bpz;
    if (d3 >= 0 && d4 <= d3) { qx = b[0]; qy = b[1]; qz = b[2]; }
    else {
      const double vc = d1 * d4 - d3 * d2;
      if (vc <= 0 && d1 >= 0 && d3 <= 0) {
        const double v = d1 / (d1 - d3);
        qx = a[0] + abx * v; qy = a[1] + aby * v; qz = a[2] + abz * v;
      } else {
        const double cpx = px - c[0], cpy = py - c[1], cpz = pz - c[2];
        const double d5 = abx * cpx + aby * cpy + abz * cpz, d6 = acx * cpx + acy * cpy + acz * cpz;
        if (d6 >= 0 && d5 <= d6) { qx = c[0]; qy = c[1]; qz = c[2]; }
        else {
          const double vb = d5 * d2 - d1 * d6;
          if (vb <= 0 && d2 >= 0 && d6 <= 0) {
            const double w = d2 / (d2 - d6);
            qx = a[0] + acx * w; qy = a[1] + acy * w; qz = a[2] + acz * w;
          } else {
            const double va = d3 * d6 - d5 * d4;
            if (va <= 0 && d4 - d3 >= 0 && d5 - d6 >= 0) {
              const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
              qx = b[0] + (c[0] - b[0]) * w; qy = b[1] + (c[1] - b[1]) * w; qz = b[2] + (c[2] - b[2]) * w;
            } else {
              const double den = 1 / (va + vb + vc), v = vb * den, w = vc * den;
              qx = a[0] + abx * v + acx * w; qy = a[1] + aby * v + acy * w; qz = a[2] + abz * v + acz * w;
            }
          }
        }
      }
    }
  }
  const double dx = px - qx, dy = py - qy, dz = pz - qz;
  return dx * dx + dy * dy + dz * dz;
}

__global__ void k_sdf_fill(uint32_t* data, size_t n, uint32_t bits) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) data[i] = bits;
}

// pass 1: one CTA per triangle, its threads over the voxels of the triangle's grown box
__global__ void __launch_bounds__(256) k_sdf_band(const double* __restrict__ tri, uint32_t nt, SdfGrid G, uint32_t* __restrict__ data) {
  for (uint32_t q = blockIdx.x; q < nt; q += gridDim.x) {
    const double* a = tri + 9 * (size_t)q;
    const double* b = a + 3;
    const double* c = a + 6;
    const double ux = b[0] - a[0], uy = b[1] - a[1], uz = b[2] - a[2], vx = c[0] - a[0], vy = c[1] - a[1], vz = c[2] - a[2];
    double px = uy * vz - uz * vy, py = uz * vx - ux * vz, pz = ux * vy - uy * vx;
    const double pl = sqrt(px * px + py * py + pz * pz);   // Math.hypot
    if (pl > 0) { px /= pl; py /= pl; pz /= pl; }
    int r0[3], r1[3];
    const int dims[3] = {G.nx, G.ny, G.nz};
    for (int k = 0; k < 3; k++) {
      const double mn = fmin(fmin(a[k], b[k]), c[k]), mx = fmax(fmax(a[k], b[k]), c[k]);
      const double f0 = floor((mn + -G.B - G.lo[k]) * G.ic), f1 = ceil((mx + G.B - G.lo[k]) * G.ic);
      r0[k] = (int)fmax(0.0, fmin((double)(dims[k] - 1), f0));
      r1[k] = (int)fmax(0.0, fmin((double)(dims[k] - 1), f1));
    }
    const int bx = r1[0] - r0[0] + 1, by = r1[1] - r0[1] + 1, bz = r1[2] - r0[2] + 1;
    const long long nb = (long long)bx * by * bz;
    for (long long e = threadIdx.x; e < nb; e += blockDim.x) {
      const int i = r0[0] + (int)(e % bx), j = r0[1] + (int)((e / bx) % by), k = r0[2] + (int)(e / ((long long)bx * by));
      const double x = G.lo[0] + i * G.cell, y = G.lo[1] + j * G.cell, z = G.lo[2] + k * G.cell;
      if (pl > 0) {
        const double ee = (x - a[0]) * px + (y - a[1]) * py + (z - a[2]) * pz;
        if (ee * ee > G.B2) continue;
      }
      const float d2 = (float)ptTriDist2(x, y, z, a, b, c);
      atomicMin(&data[(size_t)i + (size_t)G.nx * ((size_t)j + (size_t)G.ny * k)], __float_as_uint(d2));
    }
  }
}

__global__ void k_sdf_sqrt(float* data, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float v = data[i];
    if ((double)v < 1e29) data[i] = (float)sqrt((double)v);
  }
}

// pass 2: the chamfer sweeps. Neighbour o of the forward sweep is (di, dj, dk) with dk < 0, or dk = 0 and dj < 0, or
// dk = dj = 0 and di < 0; the backward sweep mirrors them. Plane t holds the voxels with i + 2 j + 4 k = t (mirrored
// coordinates for the backward sweep): every neighbour a voxel reads lies on an earlier plane.
struct Chamfer { int oi[13], oj[13], ok[13]; float ow[13]; };
__global__ void __launch_bounds__(1024) k_sdf_sweep(float* data, SdfGrid G, Chamfer W, int pass) {
  const int nx = G.nx, ny = G.ny, nz = G.nz;
  const int sg = pass ? -1 : 1;
  const int tmax = (nx - 1) + 2 * (ny - 1) + 4 * (nz - 1);
  const int njk = ny * nz;
  for (int t = 0; t <= tmax; t++) {
    for (int r = threadIdx.x; r < njk; r += blockDim.x) {
      const int jj = r % ny, kk = r / ny;
      const int ii = t - 2 * jj - 4 * kk;
      if (ii < 0 || ii >= nx) continue;
      const int i = pass ? nx - 1 - ii : ii, j = pass ? ny - 1 - jj : jj, k = pass ? nz - 1 - kk : kk;
      const size_t idx = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k);
      double v = data[idx];
      if (v <= G.B) continue;   // exact already
      for (int o = 0; o < 13; o++) {
        const int ni = i + sg * W.oi[o], nj = j + sg * W.oj[o], nk = k + sg * W.ok[o];
        if (ni < 0 || nj < 0 || nk < 0 || ni >= nx || nj >= ny || nk >= nz) continue;
        const double c2 = (double)data[(size_t)ni + (size_t)nx * ((size_t)nj + (size_t)ny * nk)] + (double)W.ow[o];
        if (c2 < v) v = c2;
      }
      data[idx] = (float)v;
    }
    __syncthreads();
  }
}

// pass 3: the crossings of the line (j, k), nudged off the grid by (ey, ez), with each triangle; pass 0 counts them per
// line, pass 1 stores their x (any order) from the scanned line offsets
__global__ void __launch_bounds__(256) k_sdf_cross(const double* __restrict__ tri, uint32_t nt, SdfGrid G, int pass, uint32_t* rowCount,
                                                   const uint32_t* rowOff, double* xs) {
  const double ey = 0.000137 * G.cell, ez = 0.000271 * G.cell;
  for (uint32_t q = blockIdx.x; q < nt; q += gridDim.x) {
    const double* a = tri + 9 * (size_t)q;
    const double* b = a + 3;
    const double* c = a + 6;
    const double area = (b[1] - a[1]) * (c[2] - a[2]) - (b[2] - a[2]) * (c[1] - a[1]);
    if (fabs(area) < 1e-14) continue;   // edge-on to the lines
    const int jlo = (int)fmax(0.0, ceil((fmin(fmin(a[1], b[1]), c[1]) - G.lo[1] - ey) * G.ic));
    const int jhi = (int)fmin((double)(G.ny - 1), floor((fmax(fmax(a[1], b[1]), c[1]) - G.lo[1] - ey) * G.ic));
    const int klo = (int)fmax(0.0, ceil((fmin(fmin(a[2], b[2]), c[2]) - G.lo[2] - ez) * G.ic));
    const int khi = (int)fmin((double)(G.nz - 1), floor((fmax(fmax(a[2], b[2]), c[2]) - G.lo[2] - ez) * G.ic));
    if (jhi < jlo || khi < klo) continue;
    const int nj = jhi - jlo + 1;
    const long long n = (long long)nj * (khi - klo + 1);
    for (long long e = threadIdx.x; e < n; e += blockDim.x) {
      const int j = jlo + (int)(e % nj), k = klo + (int)(e / nj);
      const double z = G.lo[2] + k * G.cell + ez, y = G.lo[1] + j * G.cell + ey;
      const double w0 = ((c[1] - b[1]) * (z - b[2]) - (c[2] - b[2]) * (y - b[1])) / area;
      const double w1 = ((a[1] - c[1]) * (z - c[2]) - (a[2] - c[2]) * (y - c[1])) / area;
      const double w2 = 1 - w0 - w1;
      if (w0 < 0 || w1 < 0 || w2 < 0) continue;
      const uint32_t row = (uint32_t)j + (uint32_t)G.ny * (uint32_t)k;
      if (pass == 0) { atomicAdd(&rowCount[row], 1u); continue; }
      xs[rowOff[row] + atomicAdd(&rowCount[row], 1u)] = w0 * a[0] + w1 * b[0] + w2 * c[0];
    }
  }
}
__global__ void __launch_bounds__(1024) k_sdf_scan(const uint32_t* cnt, uint32_t n, uint32_t* off) {
  __shared__ uint32_t sm[33];
  uint32_t carry = 0;
  for (uint32_t c0 = 0; c0 < n; c0 += blockDim.x) {
    const uint32_t i = c0 + threadIdx.x;
    const uint32_t v = i < n ? cnt[i] : 0u;
    uint32_t tot;
    const uint32_t ex = blockExclusive(v, sm, &tot);
    if (i < n) off[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) off[n] = carry;
}
__global__ void k_sdf_sign(float* data, SdfGrid G, const uint32_t* __restrict__ rowOff, const double* __restrict__ xs) {
  const size_t n = (size_t)G.nx * G.ny * G.nz;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % G.nx);
    const uint32_t row = (uint32_t)(e / G.nx);
    const uint32_t s0 = rowOff[row], s1 = rowOff[row + 1];
    if (s0 == s1) continue;
    const double x = G.lo[0] + i * G.cell;
    uint32_t m = 0;
    for (uint32_t q = s0; q < s1; q++) m += xs[q] < x ? 1u : 0u;
    if (m & 1u) data[e] = -data[e];
  }
}

}  // namespace st

using namespace st;

#define SB_CK(x)                                                         \
  do {                                                                   \
    cudaError_t e_ = (x);                                                \
    if (e_ != cudaSuccess) {                                             \
      st::set_error_text(cudaGetErrorString(e_));                        \
      st = e_ == cudaErrorMemoryAllocation ? ST_OOM : ST_DEVICE_ERROR;   \
      goto done;                                                         \
    }                                                                    \
  } while (0)

extern "C" st_status st_build_sdf(int device, const st_mesh* mesh, st_sdf_build* b) {
  if (!mesh || !b || b->size != sizeof(st_sdf_build) || (mesh->nf && (!mesh->idx || !mesh->len)) || (mesh->nv && !mesh->v)) return ST_BAD_ARG;
  // meshBounds and the grid (src/shared.js:63-67, 103-106), in doubles
  double lo[3] = {1e9, 1e9, 1e9}, hi[3] = {-1e9, -1e9, -1e9};
  for (uint32_t p = 0; p < mesh->nv; p++)
    for (int k = 0; k < 3; k++) { const double x = mesh->v[3 * (size_t)p + k]; if (x < lo[k]) lo[k] = x; if (x > hi[k]) hi[k] = x; }
  if (mesh->nv == 0) return ST_BAD_ARG;   // the reference's grid would have a negative size (a RangeError)
  double cell = b->cell != 0.0 ? b->cell : 0.025;
  const double margin = b->margin;
  for (int k = 0; k < 3; k++) { lo[k] = lo[k] - margin; hi[k] = hi[k] + margin; }
  if (!(cell > 0) || !(hi[0] - lo[0] >= 0) || !(hi[1] - lo[1] >= 0) || !(hi[2] - lo[2] >= 0)) return ST_BAD_ARG;
  int dims[3];
  auto setDims = [&]() { for (int k = 0; k < 3; k++) dims[k] = (int)std::ceil((hi[k] - lo[k]) / cell) + 1; };
  setDims();
  while ((double)dims[0] * dims[1] * dims[2] > 2.6e6) { cell *= 1.25; setDims(); }
  for (int k = 0; k < 3; k++) { b->dims[k] = (uint32_t)dims[k]; b->origin[k] = lo[k]; }
  b->cell = cell;
  const size_t N = (size_t)dims[0] * dims[1] * dims[2];
  if (!b->data) return ST_OK;
  if (b->cap < N) return ST_OVERFLOW;
  // meshTris (src/shared.js:45-49): fan triangulation of each face
  std::vector<double> tri;
  {
    size_t at = 0;
    for (uint32_t f = 0; f < mesh->nf; f++) {
      const uint32_t L = mesh->len[f];
      for (uint32_t k = 1; k + 1 < L; k++) {
        const uint32_t id[3] = {mesh->idx[at], mesh->idx[at + k], mesh->idx[at + k + 1]};
        for (uint32_t vtx : id) {
          if (vtx >= mesh->nv) return ST_BAD_ARG;
          tri.insert(tri.end(), mesh->v + 3 * (size_t)vtx, mesh->v + 3 * (size_t)vtx + 3);
        }
      }
      at += L;
    }
  }
  const uint32_t nt = (uint32_t)(tri.size() / 9);
  st_status st = ST_OK;
  cudaStream_t q = nullptr;
  double *dTri = nullptr, *dXs = nullptr;
  float* dData = nullptr;
  uint32_t *dCnt = nullptr, *dOff = nullptr;
  SdfGrid G{{lo[0], lo[1], lo[2]}, cell, 1 / cell, 2.5 * cell, (2.5 * cell) * (2.5 * cell), dims[0], dims[1], dims[2]};
  Chamfer W{};
  {
    int o = 0;
    for (int dk = -1; dk <= 0; dk++)
      for (int dj = -1; dj <= 1; dj++)
        for (int di = -1; di <= 1; di++)
          if (dk < 0 || dj < 0 || (dj == 0 && di < 0)) {
            W.oi[o] = di; W.oj[o] = dj; W.ok[o] = dk;
            W.ow[o] = (float)(cell * std::sqrt((double)(di * di + dj * dj + dk * dk)));   // cell * Math.hypot(di, dj, dk)
            o++;
          }
  }
  const uint32_t rows = (uint32_t)dims[1] * (uint32_t)dims[2];
  uint32_t nx2 = 0;
  SB_CK(cudaSetDevice(device));
  SB_CK(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking));
  SB_CK(cudaMalloc((void**)&dData, N * sizeof(float)));
  SB_CK(cudaMalloc((void**)&dTri, std::max<size_t>(tri.size(), 1) * sizeof(double)));
  SB_CK(cudaMalloc((void**)&dCnt, (size_t)rows * sizeof(uint32_t)));
  SB_CK(cudaMalloc((void**)&dOff, ((size_t)rows + 1) * sizeof(uint32_t)));
  if (!tri.empty()) SB_CK(cudaMemcpyAsync(dTri, tri.data(), tri.size() * sizeof(double), cudaMemcpyHostToDevice, q));
  {
    const uint32_t g = (uint32_t)std::min<size_t>((N + 255) / 256, 148 * 16);
    const float big = 1e30f;   // Float32Array(N).fill(1e30)
    uint32_t bigBits;
    memcpy(&bigBits, &big, 4);
    k_sdf_fill<<<g, 256, 0, q>>>(reinterpret_cast<uint32_t*>(dData), N, bigBits);
    if (nt) k_sdf_band<<<std::min<uint32_t>(nt, 148 * 16), 256, 0, q>>>(dTri, nt, G, reinterpret_cast<uint32_t*>(dData));
    k_sdf_sqrt<<<g, 256, 0, q>>>(dData, N);
    k_sdf_sweep<<<1, 1024, 0, q>>>(dData, G, W, 0);
    k_sdf_sweep<<<1, 1024, 0, q>>>(dData, G, W, 1);
    SB_CK(cudaMemsetAsync(dCnt, 0, (size_t)rows * sizeof(uint32_t), q));
    if (nt) k_sdf_cross<<<std::min<uint32_t>(nt, 148 * 16), 256, 0, q>>>(dTri, nt, G, 0, dCnt, nullptr, nullptr);
    k_sdf_scan<<<1, 1024, 0, q>>>(dCnt, rows, dOff);
    SB_CK(cudaMemcpyAsync(&nx2, dOff + rows, sizeof(uint32_t), cudaMemcpyDeviceToHost, q));
    SB_CK(cudaStreamSynchronize(q));
    if (nx2) {
      SB_CK(cudaMalloc((void**)&dXs, (size_t)nx2 * sizeof(double)));
      SB_CK(cudaMemsetAsync(dCnt, 0, (size_t)rows * sizeof(uint32_t), q));
      k_sdf_cross<<<std::min<uint32_t>(nt, 148 * 16), 256, 0, q>>>(dTri, nt, G, 1, dCnt, dOff, dXs);
      k_sdf_sign<<<g, 256, 0, q>>>(dData, G, dOff, dXs);
    }
    SB_CK(cudaMemcpyAsync(b->data, dData, N * sizeof(float), cudaMemcpyDeviceToHost, q));
    SB_CK(cudaStreamSynchronize(q));
    SB_CK(cudaGetLastError());
  }
done:
  if (dData) cudaFree(dData);
  if (dTri) cudaFree(dTri);
  if (dCnt) cudaFree(dCnt);
  if (dOff) cudaFree(dOff);
  if (dXs) cudaFree(dXs);
  if (q) cudaStreamDestroy(q);
  return st;
}
