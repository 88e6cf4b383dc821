// kernels.h - host-side launchers of the FLIP and PBF kernels (defined next to the kernels they launch).
#pragma once
#include <vector>

#include "../../include/splashtank_cuda.h"
#include "common.cuh"

namespace st {
int launch_count_mark(const Bufs& B, cudaStream_t s);
int launch_mark_phi(const Bufs& B, int grid, cudaStream_t s);
int launch_mark_fill(const Bufs& B, int grid, cudaStream_t s);
int launch_tiles(const Bufs& B, uint32_t ntiles, int grid, cudaStream_t s);
int launch_scan_counts(const Bufs& B, cudaStream_t s);
int launch_scatter(const Bufs& B, cudaStream_t s);
int launch_p2g(const Bufs& B, int grid, cudaStream_t s);
int p2g_ctas_per_sm();   // CTAs of k_p2g resident on one SM (its launches use no more)
// the grid of a kernel that walks the tile list dynamically: at most its resident CTAs (cached per kernel)
int walk_grid(const void* fn, int threads, int grid);
void warm_walk_grids_flip();    // fill that cache for the kernels of flip_kernels.cu / flip_extra.cu (outside any
void warm_walk_grids_extra();   // graph capture)
// ocean: the kernels compiled with the ocean's boundary (only an ocean scene needs them)
int launch_classify(const Bufs& B, int grid, bool ocean, cudaStream_t s);
int launch_norm_div(const Bufs& B, int grid, bool ocean, cudaStream_t s);
int launch_sor_compact(const Bufs& B, int grid, int grid4, int iters, cudaStream_t s);
int launch_sor_pack(const Bufs& B, int grid4, cudaStream_t s);
int launch_sor_unpack(const Bufs& B, int grid4, cudaStream_t s);
// a pooled batch's pressure sweeps (capi.cu's ST_BATCH_POOLED): the plan of offsets, then the sweeps over every tank's
// copied tiles, as launches chained by programmatic dependence or as one persistent cooperative launch
int launch_pool_plan(const PoolBufs& Q, const Ctl* const* ctls, uint32_t ntanks, cudaStream_t s);
int launch_pool_sweeps(const PoolBufs& Q, int grid, int iters, cudaStream_t s);
cudaError_t launch_pool_persistent(const PoolBufs& Q, int grid, int iters, uint64_t limit_ns, cudaStream_t s);
int persistent_ctas_per_sm();
cudaError_t launch_barrier_test(unsigned int* bar, unsigned int* err, int grid, unsigned int expect, uint64_t limit_ns, cudaStream_t s);
int launch_project(const Bufs& B, int grid, cudaStream_t s);
int launch_g2p(const Bufs& B, int grid, bool ocean, cudaStream_t s);
int g2p_ctas_per_sm(bool ocean);   // CTAs of k_g2p resident on one SM (its launches use no more)
int launch_unsort(const Part* src, const uint32_t* ids, uint32_t n, float4* pos, float4* vel, cudaStream_t s);
int launch_fill_f32(float* p, float v, size_t n, cudaStream_t s);
int launch_iota(uint32_t* p, uint32_t n, cudaStream_t s);
// narrow band (flip_extra.cu)
int launch_nb_init(const Bufs& B, int grid, cudaStream_t s);
int launch_nb_phi(const Bufs& B, int grid, cudaStream_t s);
int launch_nb_vel(const Bufs& B, int grid, cudaStream_t s);
int launch_nb_reseed(const Bufs& B, int grid, cudaStream_t s);
// whitewater (flip_extra.cu)
// airCells: air-field cells to step first (0 when the air field is off this step); drip: step the drip samples last
constexpr uint32_t DRIP_T = 1024;   // drip samples per chunk (one CTA)
int launch_spray(const Bufs& B, uint32_t smax, bool emit, uint32_t airCells, uint32_t dripCap, int grid, cudaStream_t s);
// drip samples of one collider's distance grid (drips.cpp), appended to out: 8 floats each
void drip_samples(const st_sdf* sdf, double h, uint32_t k, std::vector<float>& out);
// the ocean's wave list (ocean.cpp): 8 floats per wave into w (room for 24); returns the number of waves
int ocean_waves(const st_step_opts* o, double g, double depth, float* w);
// frames and bake measurements (frames.cu)
struct FrameBox { double x0, y0, z0, kx, ky, kz, ks; };
struct DiagBox { double x0, y0, z0, x1, y1, z1, hy, cap; };
struct DiagAcc {
  uint32_t count[5];            // alive, non-finite, outside the box, at the speed limit, foamy
  uint32_t hist[16];            // heights
  double sum[5];                // x, y, z, speed, foam level
  unsigned long long smax;      // fastest speed (bits of a non-negative double)
  unsigned long long mn[3], mx[3];   // bounding box (doubles as ordered integers)
};
int launch_pack_frame(const float4* pos4, uint32_t n, const FrameBox& F, uint16_t* pos16, uint8_t* spd, uint8_t* fm, uint32_t* meta,
                      cudaStream_t s);
int launch_bake_diag(const Part* pa, uint32_t n, const DiagBox& D, DiagAcc* acc, cudaStream_t s);
// the live view and a frame's whitewater and deep-water parts (live.cu)
struct LiveBox {
  float x0, y0, z0, kx, ky, kz, vs;            // the box and the speed scale, f32 as the shader has them
  uint32_t smax, nS;                           // whitewater slots; whitewater points the view holds
  uint32_t oWp, oWs, oWf, oSp, oSk, oDp, oDs;  // word offsets of the parts (packLayout)
};
int launch_spray_frame(const float4* sPos, const float4* sVel, uint32_t nslots, uint32_t maxPoints, const FrameBox& F, double foamLife,
                       uint32_t* scratch, uint16_t* pos16, uint32_t* pk, uint32_t* counts, cudaStream_t s);
int launch_deep(const Bufs& B, uint32_t prev, uint32_t nActiveMax, int grid, uint32_t* tcount, uint32_t* counts, float4* out, cudaStream_t s);
int launch_pack_deep(const float4* dp, uint32_t n, const FrameBox& F, uint16_t* pos16, uint8_t* spd, cudaStream_t s);
int launch_live(const Bufs& B, const LiveBox& K, uint32_t nW, uint32_t stride, uint32_t sdMax, float foamLife, const float4* deep, uint32_t nDeep,
                uint32_t* scratch, uint32_t* out, cudaStream_t s);
}  // namespace st
