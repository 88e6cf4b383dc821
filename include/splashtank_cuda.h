/*
 * splashtank_cuda.h - C ABI of the B200 FLIP water step (SplashTank's FlipSim) and the PBF solver.
 *
 * Plain C: pointers, sizes and POD structs only; no CUDA or torch types. One handle owns one CUDA
 * stream and all device memory it needs. A handle is not thread-safe: call it from one host thread.
 * Calls that only enqueue GPU work (st_flip_step) return before the GPU finishes; read calls
 * (st_flip_read_*, st_flip_stats) synchronise the handle's stream.
 *
 * Each entry point names the reference interface it replaces (paths inside the SplashTank repo).
 */
#ifndef SPLASHTANK_CUDA_H
#define SPLASHTANK_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ST_ABI_VERSION 1u

typedef enum st_status {
  ST_OK = 0,
  ST_NOT_READY = 1,     /* nothing to do: no particles (FlipSim.step returns early, src/flip/sim.js:181) */
  ST_POOL_GREW = 2,     /* reserved: the tile pool grew (src/flip/sim.js:137-159) */
  ST_OVERFLOW = 3,      /* a bounded list (whitewater ring, spawn list, cell bucket) was cut short */
  ST_OOM = 4,           /* device allocation failed */
  ST_BAD_ARG = 5,       /* null pointer, wrong struct size, out-of-range value */
  ST_DEVICE_ERROR = 6,  /* a CUDA call failed; the message is in st_last_error() */
  ST_TIMEOUT = 7,       /* a bounded device wait gave up */
  ST_UNSUPPORTED = 8
} st_status;

/* Open faces of the box: particles leave through them (src/shared.js:229). */
enum { ST_OPEN_X0 = 1, ST_OPEN_X1 = 2, ST_OPEN_Y0 = 4, ST_OPEN_Y1 = 8, ST_OPEN_Z0 = 16, ST_OPEN_Z1 = 32 };

/* Step option switches: FlipSim.opt (src/flip/sim.js:49). */
enum { ST_OPT_NO_FOAM = 1, ST_OPT_NO_CULL = 2, ST_OPT_FAST_AIR = 4 };

typedef struct st_flip st_flip;

/* new FlipSim(device, {d, maxN, size, open, ratio}) (src/flip/sim.js:47-58). */
typedef struct st_flip_desc {
  uint32_t size;        /* sizeof(st_flip_desc) */
  double d;             /* particle spacing */
  double ratio;         /* cell size over spacing; 0 means 2; clamped to [1.4, 4] */
  double box[3];        /* box extent (W, H, D); zeros mean (3, 2.6, 3) */
  uint32_t open;        /* ST_OPEN_* bits */
  uint32_t max_n;       /* particle capacity (MAXN) */
  uint32_t spray_cap;   /* whitewater points (FlipSim.setSprayCap, src/flip/sim.js:333); 0: off */
  int32_t device;       /* CUDA device ordinal */
} st_flip_desc;

/* A collider's signed distance grid: the object passed as cols[k].sdf (src/shared.js:98, src/gpu.js:42-56).
 * Grids are uploaded when the set of ids changes; data must stay valid only during the call. */
typedef struct st_sdf {
  uint32_t id;
  uint32_t dims[3];
  float origin[3];
  float cell;
  const float* data;    /* dims[0]*dims[1]*dims[2] floats, x fastest */
} st_sdf;

/* One collider record for a step: SceneRunner.step's colOf (src/shared.js:531-544). */
typedef struct st_collider {
  const st_sdf* sdf;
  float pos[3];         /* x, y, z */
  float R[9];           /* rotation, row major (eulerMat, src/shared.js:9-14) */
  float vel[3];         /* vx, vy, vz */
  float ang[3];         /* wx, wy, wz */
} st_collider;

/* Whitewater options: o.spr (src/flip/sim.js:203-205, 225). */
typedef struct st_spray_opts {
  float rate, min, life, mist, drag, mdrag;
  float foam_life, rise, crest, impact;
} st_spray_opts;

/* The per-step options object o (src/flip/sim.js:185-230). Fill with st_step_opts_default first. */
typedef struct st_step_opts {
  uint32_t size;        /* sizeof(st_step_opts) */
  float g;              /* gravity (o.g) */
  float flip;           /* FLIP ratio (default 0.95) */
  float comp;           /* density correction (default 6) */
  float omega;          /* SOR factor; 0 picks min(1.9, 2/(1+sin(pi/max n))) */
  float vmax;           /* speed limit; 0 means 14 */
  float wind[3];
  float drag;
  float foam_tau;       /* default 1.2 */
  float foam_sens;      /* default 1 */
  float gust;
  float tear;           /* sheet tearing threshold (particles per cell) */
  float vs;             /* metres per scene unit (default 1) */
  int32_t iters;        /* SOR iterations (red + black) */
  uint32_t flags;       /* ST_OPT_* */
  uint32_t ncols;       /* colliders (at most 32) */
  const st_collider* cols;
  int32_t spray_on;     /* o.spr present */
  st_spray_opts spray;
  int32_t nb_on;        /* o.nb.on: narrow band */
  float nb_band;        /* o.nb.band (cells, at least 2) */
  int32_t air_on;       /* o.air.on: air field dragged by water and spray, moving the whitewater (needs spray_on) */
  float air_couple;     /* o.air.couple */
  float air_decay;      /* o.air.decay */
  float air_blur;       /* o.air.blur (default 0.35) */
  int32_t drip_on;      /* o.drip.on: wet colliders drip after they leave the water (needs spray_on) */
  float drip_rate;      /* o.drip.rate: drops a second from a fully wet surface sample */
  float drip_dry;       /* o.drip.dry: seconds a surface stays wet out of the water */
  /* o.ocean (src/flip/sim.js:185-217, oceanWaves src/shared.js:760-780): 24 linear waves around the peak wavelength
   * with a Pierson-Moskowitz shaped spectrum; a boundary layer of width `layer` at the side walls holds the water to
   * them. Turns the narrow band on. */
  int32_t ocean_on;
  float ocean_level;    /* mean surface height */
  float ocean_layer;    /* boundary width */
  float ocean_length;   /* peak wavelength */
  float ocean_height;   /* significant wave height */
  float ocean_dir;      /* direction, degrees */
  float ocean_spread;   /* directional spread, degrees */
  int32_t ocean_seed;
  float time;           /* o.time: scene time, the waves' phase */
  /* PBF density constraints on the FLIP particles at the end of the step, after the whitewater and narrow-band
   * stages (no counterpart in the reference's FLIP step; the constraint is GpuSim's, src/gpu.js:208-292): iterations
   * of lambda + delta with kernel radius 2.2 d, the boundary density of the walls and colliders, FLIP's collider
   * response after each correction, and the particle velocity changed by the correction over dt. 0: off. */
  int32_t pbf_iters;
} st_step_opts;

/* Counters read back after a step: FlipSim.stats (src/flip/sim.js:160-168). */
typedef struct st_stats {
  uint32_t sc;          /* tiles (8^3 blocks) with storage */
  uint32_t ovf;         /* tiles that did not fit (always 0: every tile has storage) */
  uint32_t fluid;       /* fluid cells */
  float vmax;           /* fastest particle speed seen by P2G */
  uint32_t n;           /* particle slots in use (N) */
  uint32_t live;        /* particles alive when the last step sorted them (N before the first step) */
  uint32_t spray_used;  /* whitewater slots handed out (sctl[0]) */
  uint32_t steps;       /* steps taken since create/clear */
  uint32_t spray_overflow; /* steps whose whitewater emission tried more points than the ring holds */
  uint64_t launches;    /* CUDA kernels launched by steps since create */
} st_stats;

/* Dense debug export of the grid (FlipSim.dbgColumn/dbgRow, src/flip/sim.js:457-482), per cell of the
 * tile box (tx*8) x (ty*8) x (tz*8), x fastest. Null pointers are skipped. Cells of tiles without storage
 * read as the spare block does in the reference (cnt 0, ctype 0, pres 0). */
typedef struct st_flip_grid {
  uint8_t* tile_on;     /* tx*ty*tz */
  int32_t* cnt;
  uint32_t* ctype;
  float* pres;
  float* rhs;
  float* vn;            /* 3 per cell: the cell's lower x, y, z faces (new velocity) */
  float* vo;            /* 3 per cell: old velocity */
  float* velg;          /* 3 per cell: kept grid velocity (narrow band) */
} st_flip_grid;

typedef struct st_flip_dims {
  uint32_t nx, ny, nz, tx, ty, tz;
  float h, x0, y0, z0, x1, y1, z1;
} st_flip_dims;

/* Per-stage device milliseconds of the last step (FlipSim.stepTimed, src/flip/sim.js:312-331). Stage
 * names as in src/app/14-bench.js:17; pbf is the density stage of st_step_opts.pbf_iters (0 when off). */
typedef struct st_stage_times {
  float sort, blocks, clear, p2g, narrow_band, classify, norm_faces, divergence, pressure, project, g2p, pbf, spray, reseed, total;
} st_stage_times;

/* ---- FLIP ---- */

/* Fill an options struct with the reference defaults (src/flip/sim.js:197-230). */
void st_step_opts_default(st_step_opts* o);

/* new FlipSim(device, opt) (src/flip/sim.js:47-105). */
st_status st_flip_create(const st_flip_desc* desc, st_flip** out);
/* FlipSim.destroy (src/flip/sim.js:496-501). */
void st_flip_destroy(st_flip* s);
/* FlipSim.clear (src/flip/sim.js:539-547, src/gpu.js:389). */
st_status st_flip_clear(st_flip* s);
/* FlipSim.setCap (src/gpu.js:388). */
st_status st_flip_set_cap(st_flip* s, uint32_t cap);
/* n calls of FlipSim.add(x,y,z,vx,vy,vz) then flushRun (src/gpu.js:390-408). pos3 and vel3 hold n xyz
 * triples. *added receives how many were taken (the ring recycles slots when full). */
st_status st_flip_add(st_flip* s, const float* pos3, const float* vel3, uint32_t n, uint32_t* added);
/* FlipSim.step(dt, o) (src/flip/sim.js:179-241). Enqueues the step on the handle's stream. */
st_status st_flip_step(st_flip* s, double dt, const st_step_opts* o);
/* FlipSim.stepTimed (src/flip/sim.js:312-331): one step, returning device ms per stage. */
st_status st_flip_step_timed(st_flip* s, double dt, const st_step_opts* o, st_stage_times* t);
/* Stage timing without stalls (the per-stage numbers of src/app/14-bench.js, measured in place): while on, every step
 * records its stage boundaries as CUDA events; st_flip_read_timing waits for them and returns the summed stage times
 * of the steps recorded since timing was turned on or last read (at most the last 256). */
st_status st_flip_set_timing(st_flip* s, int on);
st_status st_flip_read_timing(st_flip* s, st_stage_times* sum, uint32_t* nsteps);
/* FlipSim.readbackInto (src/flip/sim.js:439-455): particles in id order, 4 floats each.
 * vel4 may be null. *n receives N; at most cap particles are written. */
st_status st_flip_read_particles(st_flip* s, float* pos4, float* vel4, uint32_t cap, uint32_t* n);
/* FlipSim.readSpray (src/flip/sim.js:423-437): whitewater slots handed out (positions with life in w,
 * velocities with kind in w). */
st_status st_flip_read_spray(st_flip* s, float* pos4, float* vel4, uint32_t cap, uint32_t* n);
/* The live view (FlipSim.dispPack + pump, src/flip/sim.js:381-404, 506-525; kernels subsample, sprayDisp, deepPick and
 * packDisp, src/flip/wgsl-solver.js:141-147, src/flip/wgsl-whitewater.js:196-297): a sample of the water (the first
 * n_water particles of the storage order, or every stride-th one when there are more than 300,000 or when whitewater
 * or deep water is shown), up to 200,000 whitewater points (every stride-th slot handed out, the living ones) and, with
 * the deep look on, up to 200,000 deep-water points, packed in packLayout's 32-bit words: word 0 whitewater points,
 * word 1 deep points, 2 zero words, then the parts at the offsets below (positions 3 x uint16 across the box, water
 * speed and white-water bytes, whitewater codes, deep speed bytes). The reference's order of the compacted
 * whitewater and deep points is that of its atomics; here it is ascending slot and tile-major cell. With words null
 * only the layout is filled; a smaller cap_words returns ST_OVERFLOW. */
typedef struct st_live_layout {
  uint32_t size;        /* sizeof(st_live_layout) */
  uint32_t n_water, n_spray, n_deep;   /* capacities of the parts, in points */
  uint32_t from_pos;    /* 1: the water part is the first n_water particles; 0: every stride-th */
  uint32_t o_wp, o_ws, o_wf, o_sp, o_sk, o_dp, o_ds;   /* word offsets: water positions, speeds, white water; whitewater
                                                          positions, codes; deep positions, speeds */
  uint32_t words;       /* words in all */
} st_live_layout;
st_status st_flip_pack_live(st_flip* s, float vs, uint32_t* words, uint64_t cap_words, st_live_layout* layout);
/* FlipSim.readDeep (src/flip/sim.js:408-421): the deep-water points of the last step as float4 (x, y, z, 4096 +
 * speed), compacted; *n = 0 when the deep look does not apply. At most cap are written (ST_OVERFLOW when more). */
st_status st_flip_read_deep_points(st_flip* s, float* out4, uint32_t cap, uint32_t* n);
/* FlipSim.setSprayCap (src/flip/sim.js:326-334): room for n whitewater points (0 turns whitewater off); the pool starts
 * empty, the slot counter keeps counting. The first pool also brings the air field (airAlloc). */
st_status st_flip_set_spray_cap(st_flip* s, uint32_t n);
/* FlipSim.recycle (src/gpu.js:393): when on (the default), FlipSim.add reuses slots in a ring once the cap is reached. */
st_status st_flip_set_recycle(st_flip* s, int on);
/* FlipSim.memBytes (src/flip/sim.js:492-495): device memory this handle holds, in bytes (its own count of what it
 * allocated, not the reference's estimate). */
st_status st_flip_mem_bytes(st_flip* s, uint64_t* bytes);
/* FlipSim.setDeepLook (src/flip/sim.js:406): show the narrow band's deep water (fluid cells with no particles). */
st_status st_flip_set_deep_look(st_flip* s, int on);
/* readDeep + packDeep (src/flip/sim.js:408-421, src/gpu.js:512-524): the deep-water points of the last step for a
 * frame (deep look on and the narrow band on in that step; else *n = 0): positions 3 x uint16 across the box and speed
 * bytes (16ths of the speed times vs, at most 191). Above 200,000 deep cells a fixed hashed sample is kept, sized from
 * the previous call's count. *n receives the count; at most cap are written (ST_OVERFLOW when more). */
st_status st_flip_read_deep(st_flip* s, float vs, uint16_t* pos, uint8_t* spd, uint32_t cap, uint32_t* n);
/* packSprayFrame (src/flip/bake.js:43-58): the whitewater part of a frame. Of the slots handed out, every step-th
 * (step = max(1, ceil(alive / max_points))) that is alive, in slot order: positions 3 x uint16 across the box and the
 * 32-bit codes of packSprayJS (foam_life 0 means 3). *n receives the points, *alive the living slots; at most cap are
 * written (ST_OVERFLOW when more). */
st_status st_flip_read_spray_frame(st_flip* s, uint32_t max_points, float foam_life, uint16_t* pos, uint32_t* pk, uint32_t cap,
                                   uint32_t* n, uint32_t* alive);
/* The air field (src/flip/wgsl-whitewater.js:24-89, grid made by airAlloc, src/flip/sim.js:342-350): air velocity at
 * each air-cell centre, x fastest, 4 floats per cell (w 0). dims3 receives the air grid's cells per axis (0 0 0 when
 * the handle has no whitewater pool, which the air field needs); at most cap cells are written. */
st_status st_flip_read_air(st_flip* s, float* vel4, uint32_t cap, uint32_t* dims3);
/* The drip samples (dripSamples, src/flip/bake.js:19-40; bDrip, src/flip/sim.js:352-363): 8 floats each, the
 * position on the collider in its own frame, the collider number, the normal in its own frame and the wetness (1 in
 * water, falling to 0 over o.drip.dry seconds out of it). *n receives the count; at most cap are written. */
st_status st_flip_read_drips(st_flip* s, float* out8, uint32_t cap, uint32_t* n);
/* oceanWaves (src/shared.js:760-780), host only: the ocean's 24 waves for o's ocean settings, gravity o->g and water
 * depth `depth` (the mean level above the floor), 8 floats each (kx, kz, amplitude, angular frequency, phase,
 * wavenumber, 0, 0) into w (room for 192 floats). Returns the number of waves. The viewer draws the same sums. */
int st_ocean_waves(const st_step_opts* o, double depth, float* w);
/* ---- mesh colliders: buildSDF (src/shared.js:98-181) on the device ---- */
/* A closed mesh as the reference's {v, f}: vertex positions and polygon faces, fan-triangulated as meshTris
 * (src/shared.js:45-49). */
typedef struct st_mesh {
  const double* v;      /* nv x 3 vertex positions */
  uint32_t nv;
  const uint32_t* idx;  /* the faces' vertex indices, face after face */
  const uint32_t* len;  /* vertices of each face (3 or more) */
  uint32_t nf;
} st_mesh;
/* in: cell (voxel size; 0 means 0.025) and margin (how far outside the mesh the grid reaches; the reference's default
 * is 0.16); out: the voxel size used (grown by 1.25 until the grid has at most 2.6M voxels), dims and origin. With data
 * null only the grid is computed; otherwise data (cap floats, x fastest) receives the signed distances: exact within
 * 2.5 voxels of the surface, chamfer distances farther out, negative inside. Results equal the reference's double
 * arithmetic into a Float32Array (Math.hypot taken as the square root of the sum of squares). */
typedef struct st_sdf_build {
  uint32_t size;        /* sizeof(st_sdf_build) */
  uint32_t dims[3];
  double cell, margin;
  double origin[3];
  float* data;
  uint64_t cap;
} st_sdf_build;
st_status st_build_sdf(int device, const st_mesh* mesh, st_sdf_build* b);
/* FlipSim.stats via readStats (src/flip/sim.js:160-168). Synchronises. */
st_status st_flip_stats(st_flip* s, st_stats* out);
/* The counters without waiting, as the reference reads them (readStats, src/flip/sim.js:160-168: the copy is encoded
 * into the step's submission and mapped later): st_flip_stats_async enqueues a copy of the counters as they will be
 * after the work queued so far into pinned host memory and returns a ticket (1, 2, ...); st_flip_stats_wait blocks
 * until that copy has landed and fills *out as st_flip_stats would have at that point. The last 4 tickets are held: a
 * fifth call first waits for the oldest copy, and a ticket older than that gives ST_BAD_ARG. */
/* The step timer of the reference's FlipSim (track, src/gpu.js:444-454): *inflight = steps queued but not finished,
 * *last_ms = the median device time of the last 31 finished steps (0 before the first), *slow_ms = the slowest step
 * so far. Each step records an event before and after itself; this call reads those of the finished steps without
 * waiting for the others. */
st_status st_flip_track(st_flip* s, uint32_t* inflight, float* last_ms, float* slow_ms);
st_status st_flip_stats_async(st_flip* s, uint64_t* ticket);
st_status st_flip_stats_wait(st_flip* s, uint64_t ticket, st_stats* out);
/* FlipSim.dbgColumn/dbgRow/activeCells (src/flip/sim.js:457-490), all cells at once. */
st_status st_flip_read_grid(st_flip* s, const st_flip_grid* g);
st_status st_flip_get_dims(st_flip* s, st_flip_dims* out);
/* The particle state in storage order (the order after the last step's sort): pos4, vel4, ids.
 * Pointers may be null. Together with st_flip_load_state this is the checkpoint of the particles. */
st_status st_flip_save_state(st_flip* s, float* pos4, float* vel4, uint32_t* pid, uint32_t cap, uint32_t* n);
/* Replace every particle (storage order, with ids); resets time-since-start to t and the seed counter. */
st_status st_flip_load_state(st_flip* s, const float* pos4, const float* vel4, const uint32_t* pid, uint32_t n,
                             double t, uint32_t seed);
/* Full checkpoint (no reference counterpart: the reference's cache stores frames, not solver state): everything a step
 * reads before it writes (particles in storage order, pressure warm start, cell types with the narrow band's depth,
 * kept grid velocity, both count buffers, tile flags and list, face velocities, the whitewater ring, the device
 * counters) and the host step state (time, seed, stamps, buffer parity). Restoring it into a handle created with the
 * same desc continues bit-identically. save: with buf null, *size receives the bytes needed; a smaller cap returns
 * ST_OVERFLOW. load: collider distance grids are uploaded again by the next step. */
st_status st_flip_save_full(st_flip* s, void* buf, uint64_t cap, uint64_t* size);
st_status st_flip_load_full(st_flip* s, const void* buf, uint64_t size);
/* Narrow band start (nbSeed's sim.nbFills, src/shared.js:849-851): boxes as {x0,y0,z0,x1,y1,z1} and spheres as
 * {x,y,z,r}; the next step initialises the depth field from them (nbInit = mode). mode 2 (water added to a running
 * tank) adds to the fills given since the last restart step; other modes replace them. */
st_status st_flip_nb_fills(st_flip* s, const float* boxes6, uint32_t nbox, const float* spheres4, uint32_t nsph,
                           uint32_t mode);
/* The water meshes of the same start (sim.nbFillVols, src/shared.js:829-831, 849-850): each a collider-shaped record
 * (distance grid, position, rotation; velocities are ignored) whose negative distance is water. The next restart step
 * packs them after its colliders (FlipSim.step, src/flip/sim.js:189-190) for fillPhi (wgsl-core.js:235) and then drops
 * them; the grids are copied at the call. mode as for st_flip_nb_fills. Fill volumes pending at a full checkpoint are
 * stored in it. */
st_status st_flip_nb_fill_vols(st_flip* s, const st_collider* vols, uint32_t n, uint32_t mode);
/* The CUDA stream the handle enqueues on (a cudaStream_t), for events and graph capture by the caller. */
void* st_flip_stream(st_flip* s);

/* ---- PBF (GpuSim, src/gpu.js:357-476) ----
 * The app's WebGPU position-based fluid engine: constants of FluidSim (src/shared.js:220-270), colliders as signed
 * distance grids (the same st_collider records as the FLIP step), open faces, dead particles (y below -1e5) kept in
 * place, particles in index order. The order inside a grid cell, which the reference leaves to an atomic counter, is
 * ascending particle index here. */

typedef struct st_pbf st_pbf;

/* new GpuSim(device, {d, maxN, size, open}) (src/gpu.js:357-380) */
typedef struct st_pbf_desc {
  uint32_t size;        /* sizeof(st_pbf_desc) */
  double d;             /* particle spacing; kernel radius h = 2.2 d */
  double box[3];        /* zeros mean (3, 2.6, 3) */
  uint32_t open;        /* ST_OPEN_* bits */
  uint32_t max_n;
  int32_t device;
  double eps_k;         /* FluidSim opt.epsK; 0 means 0.64 (src/shared.js:259) */
  double wall_k;        /* FluidSim opt.wallK; 0 means 1.8 (src/shared.js:268) */
} st_pbf_desc;

/* GpuSim.step's options o (src/gpu.js:409-416): gravity, XSPH viscosity, solver iterations (at least 1), colliders */
typedef struct st_pbf_opts {
  uint32_t size;        /* sizeof(st_pbf_opts) */
  float g;
  float visc;
  int32_t iters;
  uint32_t ncols;       /* at most 32 are used */
  const st_collider* cols;
} st_pbf_opts;

st_status st_pbf_create(const st_pbf_desc* desc, st_pbf** out);
void st_pbf_destroy(st_pbf* s);
/* GpuSim.add (src/gpu.js:390-402) for n particles (vel3 may be NULL: at rest); the ring overwrites slots once the cap is
 * reached while recycling is on. *added: how many were taken. */
st_status st_pbf_add(st_pbf* s, const float* pos3, const float* vel3, uint32_t n, uint32_t* added);
/* GpuSim.setCap / clear / recycle (src/gpu.js:387-389) */
st_status st_pbf_set_cap(st_pbf* s, uint32_t cap);
st_status st_pbf_clear(st_pbf* s);
st_status st_pbf_set_recycle(st_pbf* s, int32_t on);
/* GpuSim.step (src/gpu.js:409-428): predict, grid, iters x (lambda, delta, applyDelta), finalize, viscosity. Enqueues. */
st_status st_pbf_step(st_pbf* s, double dt, const st_pbf_opts* o);
/* readbackInto (src/gpu.js:430-443): positions (xyz, speed in w) and velocities of the N slots in index order. */
st_status st_pbf_read(st_pbf* s, float* pos4, float* vel4, uint32_t cap, uint32_t* n);
void* st_pbf_stream(st_pbf* s);

/* ---- the pressure projection's solve on its own: precision study ---- */

/* The linear system of the reference's pressure solve (relax, src/flip/wgsl-solver.js:124-140): for a fluid cell,
 * nns p - sum(fluid neighbours p) = rhs, with air neighbours at p = 0 and solid (walls, unless open) left out. */
typedef struct st_poisson st_poisson;
typedef struct st_poisson_desc {
  uint32_t size;        /* sizeof(st_poisson_desc) */
  uint32_t n[3];        /* cells per axis */
  uint32_t open;        /* ST_OPEN_* bits: box faces that are air instead of wall */
  int32_t device;
} st_poisson_desc;
enum { ST_SOLVE_SOR32 = 0, ST_SOLVE_REFINE = 1, ST_SOLVE_SOR64 = 2 };
typedef struct st_poisson_opts {
  uint32_t size;        /* sizeof(st_poisson_opts) */
  int32_t mode;         /* ST_SOLVE_*: FP32 red-black SOR; FP32 SOR inside FP64 residual/correction refinement; FP64 SOR */
  double tol;           /* stop at ||b - A x|| / ||b|| <= tol (measured in FP64) */
  float omega;          /* SOR factor */
  int32_t max_sweeps;   /* red + black iterations, all refinements together */
  int32_t inner_sweeps; /* iterations per refinement (mode 1) */
  int32_t check_every;  /* iterations between residual checks (modes 0 and 2) */
  int32_t schedule;     /* ST_SCHEDULE_*: blocks of check_every / inner_sweeps iterations between checks, or blocks sized
                           from the last block's measured reduction per iteration to end at the tolerance (at least 8
                           iterations, at most check_every / inner_sweeps); the same rule for every mode */
} st_poisson_opts;
enum { ST_SCHEDULE_FIXED = 0, ST_SCHEDULE_PREDICT = 1 };
typedef struct st_poisson_result {
  double rel_residual;
  int32_t sweeps;
  int32_t refinements;
  int32_t converged;
  float ms;             /* device time of the solve */
} st_poisson_result;
st_status st_poisson_create(const st_poisson_desc* d, st_poisson** out);
void st_poisson_destroy(st_poisson* s);
/* dense cell types (0 air, 1 fluid, 2 solid) and right-hand side, n[0] x n[1] x n[2], x fastest */
st_status st_poisson_set(st_poisson* s, const uint8_t* type, const double* rhs);
/* solve from zero */
st_status st_poisson_solve(st_poisson* s, const st_poisson_opts* o, st_poisson_result* res);
/* iters FP32 red-black SOR iterations from zero on (float) rhs; the result is readable with st_poisson_read.
 * ms (optional): device time of the sweeps alone. */
st_status st_poisson_sweeps32(st_poisson* s, float omega, int32_t iters, float* ms);
/* the current solution in FP64, dense, x fastest */
st_status st_poisson_read(st_poisson* s, double* p);
void* st_poisson_stream(st_poisson* s);

/* ---- frames and bake measurements ----
 * The particles as a cache frame (packFrameBuf, src/gpu.js:525-560; format of writeCacheParts, src/shared.js:688-705),
 * packed on the device in id order: pos 3 x uint16 per point across the box, spd one byte (16ths of speed x vs, at most
 * 191, 255 = gone), fm one byte (white-water level x 17). *n: points in the frame (the last live id + 1); *any_foam:
 * whether any point has white water (the frame stores fm only then). Arrays need room for cap points; at most
 * min(cap, n) are written. vs: metres per scene unit (the bake's scale; 0 means 1). */
st_status st_flip_read_frame(st_flip* s, float vs, uint16_t* pos, uint8_t* spd, uint8_t* fm, uint32_t cap, uint32_t* n,
                             int32_t* any_foam);
/* The same frame without waiting for it, as the reference's readback is a mapAsync that the bake awaits later
 * (readbackInto, src/gpu.js:430-443, awaited by the bake loops, src/gpu.js:577-587 and src/flip/bake.js:103-115): the
 * frame of the particles as they are now is packed on the step stream and copied to pos/spd/fm on a second stream
 * while the caller goes on stepping. st_flip_frame_wait blocks until it has landed and gives *n and *any_foam as st_flip_read_frame would. The copy covers
 * min(cap, slots) points whatever *n turns out to be (points from *n on are unspecified) and fm always (all zero when
 * no point has white water). The host buffers must stay valid until the wait; pinned memory lets the copy overlap the
 * steps. One frame is pending at a time: another frame call first waits for it. A wait with nothing pending gives 0. */
st_status st_flip_read_frame_async(st_flip* s, float vs, uint16_t* pos, uint8_t* spd, uint8_t* fm, uint32_t cap);
st_status st_flip_frame_wait(st_flip* s, uint32_t* n, int32_t* any_foam);
/* bakeDiag (src/flip/bake.js:60-83) of the current particles, on the device: the same counts; sums agree to rounding. */
typedef struct st_bake_diag {
  uint32_t alive, gone, non_finite, outside_box, at_speed_limit, foamy;
  double mean_speed, max_speed, mean_foam;
  double center[3];
  int32_t has_bbox;
  double bbox[6];       /* x0, y0, z0, x1, y1, z1 of the live points */
  uint32_t height_hist[16];
} st_bake_diag;
/* vcap: the step's speed limit (o.vmax; 0 means 14) */
st_status st_flip_bake_diag(st_flip* s, float vcap, st_bake_diag* out);

/* ---- launch shape of a tank's kernels (no reference counterpart: WebGPU picks no grid sizes) ----
 * CTAs per SM of the per-tile kernels: heavy (p2g, g2p; default 8), light (classify, normalise, project, narrow band;
 * default 4) and the pressure sweeps (default 8), each capped at the tile count. The kernels that take their tiles from
 * a counter (p2g, g2p, normalise + divergence, the narrow band's refill) are also capped at the CTAs that fit on the
 * SMs at once. Results do not depend on them; an autotuner picks them for many tanks sharing one GPU. */
st_status st_flip_set_launch(st_flip* s, int32_t tile_ctas_per_sm, int32_t light_ctas_per_sm, int32_t sor_ctas_per_sm);

/* ---- many independent tanks stepped together (no reference counterpart; the reference steps one tank) ----
 * The tanks are st_flip handles on one device, created and owned by the caller. st_batch_step does each tank's
 * st_flip_step (same options, same result, bit for bit) in one of four ways:
 *  ST_BATCH_GRAPH       every tank's step graph as a parallel branch of one CUDA graph launch;
 *  ST_BATCH_SEQUENTIAL  the step graphs one after another on the batch stream;
 *  ST_BATCH_POOLED      one graph: parallel tank branches up to the pressure sweeps, then every tank's fluid tiles
 *                       in one shared pool (tank order, tiles ascending; the reference's slot pool,
 *                       src/flip/wgsl-blocks.js:16-35, shared by all tanks) swept by one launch per colour for all
 *                       tanks, then parallel tank branches to the end of the step;
 *  ST_BATCH_PERSISTENT  as POOLED, with all sweeps of the step in one persistent cooperative launch whose grid-barrier
 *                       waits are bounded: a wait that runs out makes the next st_batch_step return ST_TIMEOUT.
 * The pooled modes need the same SOR iteration count on every tank; a step where a tank restarts its narrow band
 * runs as ST_BATCH_GRAPH. The batch's work is ordered after each tank's earlier work and before its later work. */
typedef struct st_batch st_batch;
enum { ST_BATCH_GRAPH = 0, ST_BATCH_SEQUENTIAL = 1, ST_BATCH_POOLED = 2, ST_BATCH_PERSISTENT = 3 };
typedef struct st_batch_desc {
  uint32_t size;   /* sizeof(st_batch_desc) */
  int32_t mode;    /* ST_BATCH_* */
} st_batch_desc;
st_status st_batch_create(const st_batch_desc* d, st_flip* const* tanks, uint32_t n, st_batch** out);
void st_batch_destroy(st_batch* b);
/* opts[i]: the options of tank i (its colliders included) */
st_status st_batch_step(st_batch* b, double dt, const st_step_opts* const* opts);
st_status st_batch_set_mode(st_batch* b, int32_t mode);
void* st_batch_stream(st_batch* b);
/* kernels launched by batch steps so far */
uint64_t st_batch_launches(st_batch* b);
/* the pooled modes' sweeps: CTAs per SM (capped by residency in ST_BATCH_PERSISTENT) and the limit of each grid-barrier
 * wait in microseconds (default 1,000,000) */
st_status st_batch_set_sweeps(st_batch* b, int32_t ctas_per_sm, uint32_t wait_limit_us);
/* The persistent sweep's bounded grid barrier on its own, expecting `missing` more CTAs than it launches, so every wait
 * runs out after about limit_us: *timed_out = 1 when the kernel reported it and returned (the check of the bound). */
st_status st_batch_barrier_test(int32_t device, uint32_t missing, uint32_t limit_us, uint32_t* timed_out);

/* ---- differentiable rollout and its adjoint (no reference counterpart: the reference has no gradients) ----
 * A FLIP rollout on a dense n^3 MAC grid over the unit box (P2G, gravity, collider and wall face velocities, pressure
 * projection by preconditioned conjugate gradients, FLIP/PIC G2P, advection, analytic box collider push-out, wall
 * clamp) whose loss is sum over cells of (splatted particle density - target)^2. Parameters (27 doubles): the box
 * collider's centre at 8 keyframes spread evenly over the rollout (xyz each, linear in between), then the initial
 * fluid velocity. A recording forward pass fixes the discrete decisions (cell types, faces with mass, collider and
 * wall contacts, the piece of the box's distance field each particle is on); st_diff_backward returns the exact gradient of the rollout with those decisions held, by a
 * hand-written adjoint with checkpoint-and-recompute every ckpt_every steps; a frozen forward pass (record 0)
 * evaluates that same function for finite differences. fp64 selects double precision throughout. */
typedef struct st_diff st_diff;
typedef struct st_diff_desc {
  uint32_t size;          /* sizeof(st_diff_desc) */
  uint32_t n;             /* cells per axis (cell size 1/n) */
  uint32_t steps;
  uint32_t ckpt_every;    /* particle checkpoint interval of the reverse pass */
  int32_t fp64;
  int32_t device;
  float dt, flip, g;      /* time step, FLIP ratio, gravity */
  float q0;               /* collider push-out distance */
  float margin;           /* particles stay in [margin, 1 - margin] */
  float box_half[3];      /* collider half extents */
  uint32_t cg_maxit;
  float cg_tol;           /* relative residual of the pressure solves */
  /* 1: the collider is the box's signed distance grid (nodes grid_cell apart, 3 cells of margin) sampled as sdfEval
   * does (src/gpu.js:6-33: trilinear distance, the normalised trilinear gradient as the normal), and the adjoint
   * differentiates that response (the trilinear gradient and Hessian); 0: the analytic box */
  int32_t collider_grid;
  float grid_cell;
} st_diff_desc;
/* pos3: initial particle positions; target: n^3 densities, x fastest */
st_status st_diff_create(const st_diff_desc* d, const float* pos3, uint32_t np, const float* target, st_diff** out);
void st_diff_destroy(st_diff* s);
st_status st_diff_forward(st_diff* s, const double* params, int32_t record, double* loss);
/* gradient of the loss at the parameters of the last recording forward pass */
st_status st_diff_backward(st_diff* s, double* grad);
/* the particles after the last forward pass (positions, then velocities when vel3 is not NULL), np x 3 floats each */
st_status st_diff_read_state(st_diff* s, float* pos3, float* vel3);
/* device bytes held; conjugate-gradient iterations of the last forward or backward call */
st_status st_diff_stats(st_diff* s, uint64_t* device_bytes, int32_t* cg_iters);
void* st_diff_stream(st_diff* s);

/* ---- pressure residual that allocates nothing (no reference counterpart: the reference measures no residual) ----
 * ||b - A x|| / ||b|| of the pressure system above, in FP64, on arrays the caller owns on the device, in the tile-major
 * layout (tile t = ti + tx (tj + ty tk) with tx = ceil(n[0]/8) ..., cell t*512 + lx + 8 (ly + 8 lz)). For callers that
 * cannot allocate device memory at the call: a process whose free device memory is held by another allocator (a
 * caching allocator such as PyTorch's reserves it, so a cudaMalloc here can fail although the caller has room), or a
 * stepping loop that must not take the device-wide synchronisation that cudaMalloc/cudaFree can imply.
 * It calls no cudaMalloc/cudaFree and no allocating library routine. Its scratch is a fixed device array inside the
 * library, one per device: 2 x ST_NOALLOC_MAX_TILES + 4 doubles (1 MiB), holding per-tile partial sums.
 *  - n_tiles above ST_NOALLOC_MAX_TILES is rejected with ST_BAD_ARG and a message in st_last_error().
 *  - The first call on each device, made with that device current, looks up the scratch address
 *    (cudaGetSymbolAddress).
 *  - Every call synchronises `stream` and copies the result into host memory, so no call can be captured into a
 *    graph: do not call it while `stream` (or, under global capture mode, any stream on the device) is capturing.
 *  - The scratch's error word must start at zero: each call clears it on `stream` before its kernels. The partial sums
 *    need no clearing; each call writes every one it reads.
 *  - Calls on one device share the scratch: calls that overlap in time (on other streams or host threads) race and
 *    return wrong numbers. Serialise them.
 * Runs on the current device, on `stream` (NULL: the default stream), and waits for that stream before returning. A
 * tile index outside the box returns ST_BAD_ARG (nothing outside the arrays is read). */
#define ST_NOALLOC_MAX_TILES 65536u
typedef struct st_poisson_system {
  uint32_t size;         /* sizeof(st_poisson_system) */
  uint32_t n[3];         /* cells per axis */
  uint32_t n_tiles;      /* tiles holding fluid (at most ST_NOALLOC_MAX_TILES) */
  const uint32_t* tiles; /* device: the n_tiles tiles holding fluid, ascending */
  const uint16_t* info;  /* device, tx*ty*tz*512 words: 0x8000 fluid | non-solid neighbours << 8 | fluid-neighbour bits
                            (-x, +x, -y, +y, -z, +z), 0 for other cells */
  const double* b;       /* device, tx*ty*tz*512: right-hand side on fluid cells */
} st_poisson_system;
/* x: device, tx*ty*tz*512 FP64 values. rel = ||r|| / ||b|| (0 when b = 0); r2, b2 (optional) = ||r||^2, ||b||^2. */
st_status st_poisson_residual_noalloc(const st_poisson_system* sys, const double* x, void* stream, double* rel, double* r2,
                                      double* b2);

/* ---- common ---- */
uint32_t st_abi_version(void);
/* Text of the last error on this thread (static storage). */
const char* st_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
