// capi.cu - the C ABI of include/splashtank_cuda.h for the FLIP step: handle, device memory, the parameter block
// and the stage sequence of one step (FlipSim.step, src/flip/sim.js:179-310).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>
#include <algorithm>

#include "../../include/splashtank_cuda.h"
#include "common.cuh"
#include "kernels.h"
#include "pbf_core.cuh"

using namespace st;

namespace {

thread_local char g_err[512] = "";

void set_err(const char* what, cudaError_t e) {
  snprintf(g_err, sizeof(g_err), "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call)                                  \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) {                      \
      set_err(#call, e_);                         \
      return e_ == cudaErrorMemoryAllocation ? ST_OOM : ST_DEVICE_ERROR; \
    }                                             \
  } while (0)

thread_local size_t g_alloc_bytes = 0;   // bytes dalloc handed out on this thread (a handle's create sums its own)
template <class T>
cudaError_t dalloc(T** p, size_t count) {
  const size_t b = std::max<size_t>(count, 1) * sizeof(T);
  const cudaError_t e = cudaMalloc((void**)p, b);
  if (e == cudaSuccess) g_alloc_bytes += b;
  return e;
}

}  // namespace

void st::set_error_text(const char* text) { snprintf(g_err, sizeof(g_err), "%s", text); }

struct st_flip {
  int device = 0;
  cudaStream_t stream = nullptr;
  int sms = 148;
  // geometry, fixed at create (src/flip/sim.js:47-61)
  double d = 0, ratio = 2, h = 0, rest = 8;
  int nx = 0, ny = 0, nz = 0, tx = 0, ty = 0, tz = 0;
  uint32_t ntiles = 0, ncell = 0;
  double bx0 = 0, bx1 = 0, by0 = 0, by1 = 0, bz0 = 0, bz1 = 0;
  uint32_t open = 0, maxN = 0, cap = 0, N = 0, ring = 0, sprayCap = 0;
  bool recycle = true;
  // host-side step state
  double tm = 0;
  uint32_t seed = 0, steps = 0, stamp = 0, parity = 0;
  bool velGOn = false;
  uint32_t nbInit = 0;
  std::vector<float> fills;
  // water-mesh fill volumes of the next restart (sim.nbFillVols, src/shared.js:849-850): records with owned grids
  struct FillVol { st_sdf sd; std::vector<float> data; st_collider c; };
  std::vector<FillVol> fillVols;
  std::string sdfSig;
  size_t sdfCap = 0;
  FlipParams hp{};
  float waves[32 * 8] = {};   // this step's ocean waves (oceanWaves)
  // per-step uploads (parameter block + collider records) come from a ring of pinned host blocks, so the copies are
  // asynchronous and a block is rewritten only after the copy that read it has run
  static constexpr int RING = 16;
  // cols and waves: float4 reads; pbf: the density stage's block (st_step_opts.pbf_iters)
  struct Upload { FlipParams P; alignas(16) float cols[32 * 32]; alignas(16) float waves[32 * 8]; alignas(16) PbfParams pbf; };
  Upload* ring_h = nullptr;
  cudaEvent_t ring_ev[RING] = {};
  int ring_i = 0;
  // stage timing without stalls: each step records its stage events into a ring; st_flip_read_timing sums them
  static constexpr int TSLOTS = 256, TEV = 12;
  bool timing = false;
  cudaEvent_t tev[TSLOTS][TEV] = {};
  uint32_t tcount = 0;
  // device memory
  Ctl* dCtl = nullptr;
  Ctl* hCtl = nullptr;   // pinned
  Upload* dUp = nullptr;
  Part* part[2] = {nullptr, nullptr};
  uint32_t* ids[2] = {nullptr, nullptr};
  uint32_t *key = nullptr, *rank = nullptr, *srcIdx = nullptr, *spid = nullptr, *blkDead = nullptr;
  uint32_t *need = nullptr, *blkTiles = nullptr, *active = nullptr, *tileSlot = nullptr, *dropped = nullptr, *fluidTiles = nullptr;
  uint32_t *tileCnt = nullptr, *tileAux = nullptr, *tileAux2 = nullptr, *tileEmit = nullptr, *tileDead = nullptr;
  uint8_t* deadF = nullptr;
  uint8_t *on = nullptr, *tstate = nullptr;
  int32_t* cnt[2] = {nullptr, nullptr};
  uint32_t *cellOff = nullptr, *ctype = nullptr;
  float *pres = nullptr, *rhs = nullptr, *vn = nullptr, *vo = nullptr, *velG = nullptr;
  int32_t* acc = nullptr;
  uint16_t* sorInfo = nullptr;
  float *cp = nullptr, *crhs = nullptr;
  uint16_t* cinfo = nullptr;
  uint32_t *nbs = nullptr, *slotOf = nullptr;
  uint32_t* poolZero = nullptr;   // offset 0 of a tank alone in its own compact copy
  float* pomega = nullptr;        // SOR factor of each copied tile
  uint8_t* frame = nullptr;   // packed frame (allocated by the first st_flip_read_frame)
  // an asynchronous frame (st_flip_read_frame_async): copied to the host on its own stream while later steps run
  cudaStream_t copyStream = nullptr;
  cudaEvent_t frameReady = nullptr, frameCopied = nullptr;
  uint32_t* frameMeta = nullptr;   // pinned: the frame's point count and any-foam flag
  bool framePending = false;
  // step tracking (track, src/gpu.js:444-454): an event before and after each step, read once the step is done
  static constexpr int TRK = 64;
  cudaEvent_t trkStart[TRK] = {}, trkDone[TRK] = {};
  uint64_t trkHead = 0, trkTail = 0;   // steps recorded, steps read back
  float trkMs[31] = {};
  int trkN = 0, trkPos = 0;
  float lastMs = 0.0f, slowMs = 0.0f;
  // counters read without waiting (st_flip_stats_async): a ring of pinned copies, each with its ticket and event
  static constexpr int STAT_SLOTS = 4;
  struct StatSlot { Ctl* h = nullptr; cudaEvent_t ev = nullptr; uint64_t ticket = 0, steps = 0, launches = 0; uint32_t n = 0; bool pending = false; };
  StatSlot stat[STAT_SLOTS];
  uint64_t statNext = 1;
  DiagAcc* diag = nullptr;
  float* wet = nullptr;
  float* sdf = nullptr;
  float4 *sPos = nullptr, *sVel = nullptr;
  // air field (src/flip/sim.js:342-350): cells r solver cells wide, r = max(2, ceil(cbrt(cells / 260000)))
  float4 *air = nullptr, *air2 = nullptr;
  int32_t* airAcc = nullptr;
  uint32_t aNx = 0, aNy = 0, aNz = 0, airCells = 0;
  double airH = 1.0;
  // drip samples on the colliders (dripUpdate, src/flip/sim.js:352-363): 2 float4 each, rebuilt (dry) when the
  // colliders' distance grids change
  float4* drip = nullptr;
  uint32_t ndrip = 0, dripCap = 0;
  std::string dripSig;
  std::map<uint32_t, std::vector<float>> dripCache;   // per grid id: its samples (collider number 0)
  uint8_t* emitK = nullptr;
  uint32_t *blkEmit = nullptr, *deadList = nullptr;
  // the live view and a frame's whitewater / deep-water parts (allocated by their first call)
  static constexpr uint32_t DISP_MAX = 300000, SPRAY_DISP_MAX = 200000, DEEP_MAX = 200000;
  bool deepOn = false, lastNb = false;
  uint32_t lastN = 0, stride = 1, deepPrev = 0;
  float4* deepBuf = nullptr;       // DEEP_MAX deep-water points of the last pass
  uint32_t* viewScratch = nullptr; // per-block or per-tile counts, then 2 counters
  size_t viewScratchN = 0;
  uint32_t* liveOut = nullptr;     // the packed live view
  size_t liveWords = 0;
  uint8_t* framePart = nullptr;    // packed whitewater or deep-water points of a frame
  size_t framePartBytes = 0;
  size_t createBytes = 0;          // device bytes allocated by create
  cudaEvent_t ev[16] = {};
  int cur = 0;   // part[cur] holds this step's storage order
  uint64_t launches = 0;   // kernels launched by steps since create
  struct Graph { uint64_t key = 0; cudaGraph_t graph = nullptr; cudaGraphExec_t exec = nullptr; cudaGraphNode_t evnode[TEV] = {}; int launches = 0; };
  std::vector<Graph> graphs;
  // the PBF density stage's buffers, made on the first step that asks for it
  PbfDev pbf{};
  PbfHostConsts pbfc{};
  uint32_t pbfCells = 0;
  bool use_graphs = true;
  // CTAs per SM of the per-tile kernels (heavy: p2g, g2p; light: the rest) and of the pressure sweeps
  int gridT = 8, gridT4 = 4, gridSor = 8;
  uint64_t gen = 0;   // bumped whenever the captured steps are dropped (their buffers or launch shapes changed)

  Bufs bufs() const {
    Bufs B{};
    B.P = &dUp->P; B.ctl = dCtl;
    B.pa = part[cur]; B.pb = part[cur ^ 1]; B.ida = ids[cur]; B.idb = ids[cur ^ 1];
    B.key = key; B.rank = rank; B.srcIdx = srcIdx; B.spid = spid; B.blkDead = blkDead;
    B.need = need; B.on = on; B.tstate = tstate; B.blkTiles = blkTiles; B.active = active; B.prevActive = nullptr;
    B.tileSlot = tileSlot; B.dropped = dropped; B.fluidTiles = fluidTiles; B.wet = wet; B.tileCnt = tileCnt; B.tileAux = tileAux; B.tileAux2 = tileAux2; B.tileEmit = tileEmit; B.tileDead = tileDead; B.deadF = deadF;
    B.cnt = cnt[parity]; B.cntOther = cnt[parity ^ 1]; B.cellOff = cellOff; B.ctype = ctype; B.pres = pres; B.rhs = rhs;
    B.acc = acc; B.vn = vn; B.vo = vo; B.velG = velG; B.sorInfo = sorInfo; B.cp = cp; B.crhs = crhs; B.cinfo = cinfo; B.nbs = nbs; B.slotOf = slotOf; B.poolOff = poolZero; B.pomega = pomega; B.cols = reinterpret_cast<const float4*>(dUp->cols); B.sdf = sdf;
    B.waves = reinterpret_cast<const float4*>(dUp->waves);
    B.sPos = sPos; B.sVel = sVel; B.air = air; B.air2 = air2; B.airAcc = airAcc; B.drip = drip; B.dripTmp = drip ? drip + 2 * (size_t)dripCap : nullptr;
    B.dripCnt = drip ? reinterpret_cast<uint32_t*>(drip + 4 * (size_t)dripCap) : nullptr; B.emitK = emitK; B.blkEmit = blkEmit; B.deadList = deadList;
    B.ncell = ncell; B.nblk = (N + PBLK - 1) / PBLK;
    return B;
  }
  int tileGrid(int per_sm) const { return std::max(1, std::min<int>(sms * per_sm, (int)ntiles)); }
};

static void drop_graphs(st_flip* s);

extern "C" {

uint32_t st_abi_version(void) { return ST_ABI_VERSION; }
const char* st_last_error(void) { return g_err; }

void st_step_opts_default(st_step_opts* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->size = sizeof(st_step_opts);
  o->g = 9.81f; o->flip = 0.95f; o->comp = 6.0f; o->omega = 0.0f; o->vmax = 14.0f;
  o->foam_tau = 1.2f; o->foam_sens = 1.0f; o->vs = 1.0f; o->iters = 30;
  o->spray.foam_life = 3.0f; o->spray.rise = 0.3f; o->spray.crest = 1.0f; o->spray.impact = 0.5f;
  o->nb_band = 3.0f;
  o->air_blur = 0.35f;
  o->drip_dry = 1.0f;
}

void st_flip_destroy(st_flip* s) {
  if (!s) return;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->copyStream) cudaStreamSynchronize(s->copyStream);
  drop_graphs(s);
  void* ptrs[] = {s->dCtl, s->part[0], s->part[1], s->ids[0], s->ids[1], s->key, s->rank, s->srcIdx, s->spid, s->blkDead,
                  s->need, s->blkTiles, s->active, s->tileSlot, s->dropped, s->fluidTiles, s->wet, s->tileCnt, s->tileAux, s->tileAux2, s->tileEmit, s->tileDead, s->deadF, s->on, s->tstate,
                  s->cnt[0], s->cnt[1], s->cellOff, s->ctype, s->pres, s->rhs, s->vn, s->vo, s->velG, s->acc, s->sorInfo,
                  s->sdf, s->sPos, s->sVel, s->air, s->air2, s->airAcc, s->drip, s->deepBuf, s->viewScratch, s->liveOut, s->framePart, s->emitK, s->blkEmit, s->deadList, s->cp, s->crhs, s->cinfo, s->nbs, s->slotOf, s->frame, s->diag, s->poolZero, s->pomega};
  for (void* p : ptrs) if (p) cudaFree(p);
  if (s->hCtl) cudaFreeHost(s->hCtl);
  if (s->ring_h) cudaFreeHost(s->ring_h);
  if (s->dUp) cudaFree(s->dUp);
  if (s->pbf.key) { s->pbf.P = nullptr; pbf_dev_free(s->pbf); }   // P points into the upload buffer
  for (auto& e : s->ring_ev) if (e) cudaEventDestroy(e);
  for (auto& row : s->tev) for (auto& e : row) if (e) cudaEventDestroy(e);
  for (auto& e : s->ev) if (e) cudaEventDestroy(e);
  if (s->frameReady) cudaEventDestroy(s->frameReady);
  if (s->frameCopied) cudaEventDestroy(s->frameCopied);
  if (s->frameMeta) cudaFreeHost(s->frameMeta);
  for (auto& q : s->stat) {
    if (q.ev) cudaEventDestroy(q.ev);
    if (q.h) cudaFreeHost(q.h);
  }
  for (int k = 0; k < st_flip::TRK; k++) {
    if (s->trkStart[k]) cudaEventDestroy(s->trkStart[k]);
    if (s->trkDone[k]) cudaEventDestroy(s->trkDone[k]);
  }
  if (s->copyStream) cudaStreamDestroy(s->copyStream);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

static st_status reset_ids(st_flip* s) {
  for (int b = 0; b < 2; b++) launch_iota(s->ids[b], s->maxN, s->stream);
  return ST_OK;
}

st_status st_flip_create(const st_flip_desc* desc, st_flip** out) {
  if (!desc || !out || desc->size != sizeof(st_flip_desc) || !(desc->d > 0) || desc->max_n == 0) return ST_BAD_ARG;
  st_flip* s = new st_flip();
  *out = nullptr;
  s->device = desc->device;
  cudaError_t e = cudaSetDevice(s->device);
  if (e != cudaSuccess) { set_err("cudaSetDevice", e); delete s; return ST_DEVICE_ERROR; }
  cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, s->device);
  // the resident-CTA counts of the dynamic-tile kernels, queried once here rather than first inside a graph capture
  (void)p2g_ctas_per_sm(); (void)g2p_ctas_per_sm(false); (void)g2p_ctas_per_sm(true);
  warm_walk_grids_flip(); warm_walk_grids_extra();
  s->d = desc->d;
  double r = desc->ratio != 0 ? desc->ratio : 2.0;
  s->ratio = std::max(1.4, std::min(4.0, r));
  s->h = s->ratio * s->d;
  s->rest = s->ratio * s->ratio * s->ratio;
  double sz[3] = {3, 2.6, 3};
  if (desc->box[0] > 0 && desc->box[1] > 0 && desc->box[2] > 0) { sz[0] = desc->box[0]; sz[1] = desc->box[1]; sz[2] = desc->box[2]; }
  // Math.round in the reference rounds halves up
  s->nx = std::max(4, (int)std::floor(sz[0] / s->h + 0.5));
  s->ny = std::max(4, (int)std::floor(sz[1] / s->h + 0.5));
  s->nz = std::max(4, (int)std::floor(sz[2] / s->h + 0.5));
  double W = s->nx * s->h, H = s->ny * s->h, D = s->nz * s->h;
  s->bx0 = -W / 2; s->bx1 = W / 2; s->by0 = 0; s->by1 = H; s->bz0 = -D / 2; s->bz1 = D / 2;
  s->tx = (s->nx + 1 + 7) / 8; s->ty = (s->ny + 1 + 7) / 8; s->tz = (s->nz + 1 + 7) / 8;
  s->ntiles = (uint32_t)(s->tx * s->ty * s->tz);
  s->ncell = s->ntiles * 512u;
  s->open = desc->open; s->maxN = desc->max_n; s->cap = desc->max_n; s->sprayCap = desc->spray_cap;
  const size_t M = s->maxN, T = s->ntiles, C = s->ncell, NB = (M + PBLK - 1) / PBLK;
  st_status st = ST_OK;
  auto A = [&](cudaError_t ee, const char* what) { if (ee != cudaSuccess && st == ST_OK) { set_err(what, ee); st = ee == cudaErrorMemoryAllocation ? ST_OOM : ST_DEVICE_ERROR; } };
  A(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "stream");
  g_alloc_bytes = 0;
  A(dalloc(&s->dCtl, 1), "ctl"); A(cudaMallocHost((void**)&s->hCtl, sizeof(Ctl)), "ctl host");
  for (int b = 0; b < 2; b++) { A(dalloc(&s->part[b], M), "particles"); A(dalloc(&s->ids[b], M), "ids"); A(dalloc(&s->cnt[b], C), "cnt"); }
  A(dalloc(&s->key, M), "key"); A(dalloc(&s->rank, M), "rank"); A(dalloc(&s->srcIdx, M), "srcIdx"); A(dalloc(&s->spid, M), "spid");
  A(dalloc(&s->blkDead, NB + 1), "blkDead"); A(dalloc(&s->blkEmit, NB + 1), "blkEmit"); A(dalloc(&s->emitK, M), "emitK");
  A(dalloc(&s->deadList, M), "deadList");
  A(dalloc(&s->need, T), "need"); A(dalloc(&s->on, T), "on"); A(dalloc(&s->tstate, T), "tstate"); A(dalloc(&s->blkTiles, (T + 1023) / 1024 + 1), "blkTiles");
  A(dalloc(&s->active, T), "active"); A(dalloc(&s->fluidTiles, T), "fluidTiles"); A(dalloc(&s->wet, C), "wet"); A(dalloc(&s->tileSlot, T), "tileSlot"); A(dalloc(&s->dropped, T), "dropped");
  A(dalloc(&s->tileCnt, T + 1), "tileCnt"); A(dalloc(&s->tileAux, T + 1), "tileAux"); A(dalloc(&s->tileAux2, T + 1), "tileAux2");
  A(dalloc(&s->tileEmit, T + 1), "tileEmit"); A(dalloc(&s->tileDead, T + 1), "tileDead"); A(dalloc(&s->deadF, M), "deadF");
  A(dalloc(&s->cellOff, C), "cellOff"); A(dalloc(&s->ctype, C), "ctype"); A(dalloc(&s->pres, C), "pres"); A(dalloc(&s->rhs, C), "rhs");
  A(dalloc(&s->acc, 6 * C), "acc"); A(dalloc(&s->vn, 3 * C), "vn"); A(dalloc(&s->vo, 3 * C), "vo"); A(dalloc(&s->velG, 3 * C), "velG");
  A(dalloc(&s->sorInfo, C), "sorInfo");
  A(dalloc(&s->cp, C), "sweep p"); A(dalloc(&s->crhs, C), "sweep rhs"); A(dalloc(&s->cinfo, C), "sweep info");
  A(dalloc(&s->nbs, 6 * T), "sweep neighbours"); A(dalloc(&s->slotOf, T), "sweep slots");
  A(dalloc(&s->poolZero, 1), "pool offset"); A(dalloc(&s->pomega, T), "sweep omega"); A(dalloc(&s->sdf, 16), "sdf"); s->sdfCap = 16;
  A(dalloc(&s->sPos, std::max<size_t>(s->sprayCap, 1)), "sPos"); A(dalloc(&s->sVel, std::max<size_t>(s->sprayCap, 1)), "sVel");
  if (s->sprayCap) {   // the air field exists only with whitewater: it is stepped in the whitewater stage
    const double cells = (double)s->nx * (double)s->ny * (double)s->nz;
    const int r = std::max(2, (int)std::ceil(std::cbrt(cells / 260000.0)));
    s->airH = s->h * r;
    s->aNx = (uint32_t)((s->nx + r - 1) / r + 1); s->aNy = (uint32_t)((s->ny + r - 1) / r + 1); s->aNz = (uint32_t)((s->nz + r - 1) / r + 1);
    s->airCells = s->aNx * s->aNy * s->aNz;
    A(dalloc(&s->air, s->airCells), "air"); A(dalloc(&s->air2, s->airCells), "air2"); A(dalloc(&s->airAcc, 4 * (size_t)s->airCells), "air acc");
  }
  for (auto& ev : s->ev) A(cudaEventCreate(&ev), "event");
  A(cudaMallocHost((void**)&s->ring_h, sizeof(st_flip::Upload) * st_flip::RING), "upload ring"); A(dalloc(&s->dUp, 1), "upload");
  for (auto& ev : s->ring_ev) A(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "ring event");
  if (st != ST_OK) { st_flip_destroy(s); return st; }
  s->createBytes = g_alloc_bytes;
  // every tile starts in the state the reference's spare slot reads as
  cudaStream_t q = s->stream;
  A(cudaMemsetAsync(s->dCtl, 0, sizeof(Ctl), q), "memset");
  A(cudaMemsetAsync(s->dUp, 0, sizeof(st_flip::Upload), q), "memset");
  for (int b = 0; b < 2; b++) { A(cudaMemsetAsync(s->part[b], 0, M * sizeof(Part), q), "memset"); A(cudaMemsetAsync(s->cnt[b], 0, C * 4, q), "memset"); }
  A(cudaMemsetAsync(s->need, 0, T * 4, q), "memset"); A(cudaMemsetAsync(s->on, 0, T, q), "memset");
  A(cudaMemsetAsync(s->ctype, 0, C * 4, q), "memset"); A(cudaMemsetAsync(s->pres, 0, C * 4, q), "memset");
  A(cudaMemsetAsync(s->acc, 0, 6 * C * 4, q), "memset"); A(cudaMemsetAsync(s->vn, 0, 3 * C * 4, q), "memset");
  A(cudaMemsetAsync(s->vo, 0, 3 * C * 4, q), "memset"); A(cudaMemsetAsync(s->velG, 0, 3 * C * 4, q), "memset");
  A(cudaMemsetAsync(s->sorInfo, 0, C * 2, q), "memset");
  A(cudaMemsetAsync(s->slotOf, 0xff, T * 4, q), "memset");
  A(cudaMemsetAsync(s->poolZero, 0, 4, q), "memset");
  A(cudaMemsetAsync(s->wet, 0, C * 4, q), "memset");
  A(cudaMemsetAsync(s->sPos, 0, std::max<size_t>(s->sprayCap, 1) * 16, q), "memset");
  A(cudaMemsetAsync(s->sVel, 0, std::max<size_t>(s->sprayCap, 1) * 16, q), "memset");
  if (s->airCells) { A(cudaMemsetAsync(s->air, 0, (size_t)s->airCells * 16, q), "memset"); A(cudaMemsetAsync(s->air2, 0, (size_t)s->airCells * 16, q), "memset"); }
  launch_fill_f32(s->rhs, 8.0f, C, q);
  reset_ids(s);
  A(cudaStreamSynchronize(q), "create sync");
  A(cudaGetLastError(), "create kernels");
  if (st != ST_OK) { st_flip_destroy(s); return st; }
  *out = s;
  return ST_OK;
}

st_status st_flip_get_dims(st_flip* s, st_flip_dims* o) {
  if (!s || !o) return ST_BAD_ARG;
  o->nx = s->nx; o->ny = s->ny; o->nz = s->nz; o->tx = s->tx; o->ty = s->ty; o->tz = s->tz;
  o->h = (float)s->h; o->x0 = (float)s->bx0; o->y0 = (float)s->by0; o->z0 = (float)s->bz0;
  o->x1 = (float)s->bx1; o->y1 = (float)s->by1; o->z1 = (float)s->bz1;
  return ST_OK;
}

void* st_flip_stream(st_flip* s) { return s ? (void*)s->stream : nullptr; }

st_status st_flip_clear(st_flip* s) {
  if (!s) return ST_BAD_ARG;
  cudaSetDevice(s->device);
  s->N = 0; s->ring = 0; s->tm = 0; s->nbInit = 1; s->fills.clear(); s->fillVols.clear(); s->steps = 0;
  if (s->sprayCap) {
    CK(cudaMemsetAsync(s->sPos, 0, (size_t)s->sprayCap * 16, s->stream));
    CK(cudaMemsetAsync(&s->dCtl->sctl0, 0, 4, s->stream));
  }
  if (s->airCells) CK(cudaMemsetAsync(s->air, 0, (size_t)s->airCells * 16, s->stream));
  s->dripSig.clear();   // drip samples come back dry
  reset_ids(s);
  CK(cudaStreamSynchronize(s->stream));
  return ST_OK;
}

st_status st_flip_set_cap(st_flip* s, uint32_t c) {
  if (!s) return ST_BAD_ARG;
  s->cap = std::min(c, s->maxN);
  if (s->N > s->cap) s->N = s->cap;
  if (s->ring >= s->cap) s->ring = 0;
  return ST_OK;
}

// FlipSim.add for n particles (src/gpu.js:390-408): the speed goes in pos.w, foam 0. Slots past N take the next
// ids; once the cap is reached the ring overwrites storage slots, keeping the id each slot holds.
st_status st_flip_add(st_flip* s, const float* p3, const float* v3_, uint32_t n, uint32_t* added) {
  if (!s || (n && (!p3 || !v3_))) return ST_BAD_ARG;
  cudaSetDevice(s->device);
  std::vector<Part> host(n);
  std::vector<uint32_t> slot(n);
  uint32_t k = 0;
  for (; k < n; k++) {
    uint32_t i;
    if (s->N < s->cap) i = s->N++;
    else if (s->recycle) { i = s->ring++; if (s->ring >= s->cap) s->ring = 0; }
    else break;
    float vx = v3_[k * 3], vy = v3_[k * 3 + 1], vz = v3_[k * 3 + 2];
    host[k].p = make_float4(p3[k * 3], p3[k * 3 + 1], p3[k * 3 + 2], (float)std::sqrt((double)vx * vx + (double)vy * vy + (double)vz * vz));
    host[k].v = make_float4(vx, vy, vz, 0.0f);
    slot[k] = i;
  }
  // contiguous runs of slots go up in one copy each
  uint32_t a = 0;
  while (a < k) {
    uint32_t b = a + 1;
    while (b < k && slot[b] == slot[b - 1] + 1) b++;
    CK(cudaMemcpyAsync(s->part[s->cur] + slot[a], host.data() + a, (size_t)(b - a) * sizeof(Part), cudaMemcpyHostToDevice, s->stream));
    a = b;
  }
  CK(cudaStreamSynchronize(s->stream));
  if (added) *added = k;
  return ST_OK;
}

// packColliders (src/gpu.js:42-70): 32 floats per collider, SDF grids uploaded when the set of ids changes
static st_status pack_colliders(st_flip* s, const st_step_opts* o, uint32_t& nc, float* cf, cudaStream_t q) {
  nc = std::min(o->ncols, 32u);
  if (nc && !o->cols) return ST_BAD_ARG;
  std::string sig;
  std::map<uint32_t, uint32_t> offs;
  uint32_t off = 0;
  for (uint32_t k = 0; k < nc; k++) {
    const st_sdf* sd = o->cols[k].sdf;
    if (!sd || !sd->data) return ST_BAD_ARG;
    if (!offs.count(sd->id)) { offs[sd->id] = off; off += sd->dims[0] * sd->dims[1] * sd->dims[2]; sig += std::to_string(sd->id) + ","; }
  }
  if (sig != s->sdfSig) {
    if (off > s->sdfCap) {
      CK(cudaStreamSynchronize(q));
      drop_graphs(s);   // captured steps hold the old grid pointer
      cudaFree(s->sdf);
      s->sdfCap = (size_t)std::ceil(off * 1.3);
      CK(dalloc(&s->sdf, s->sdfCap));
    }
    std::map<uint32_t, bool> seen;
    for (uint32_t k = 0; k < nc; k++) {
      const st_sdf* sd = o->cols[k].sdf;
      if (seen[sd->id]) continue;
      seen[sd->id] = true;
      CK(cudaMemcpyAsync(s->sdf + offs[sd->id], sd->data, sizeof(float) * sd->dims[0] * sd->dims[1] * sd->dims[2], cudaMemcpyHostToDevice, q));
    }
    CK(cudaStreamSynchronize(q));   // in stream order after the steps that read the old grids; data is the caller's
    s->sdfSig = sig;
  }
  if (nc) {
    for (uint32_t k = 0; k < nc; k++) {
      const st_collider& c = o->cols[k];
      const st_sdf* sd = c.sdf;
      float* f = &cf[k * 32];
      f[0] = (float)offs[sd->id]; f[1] = (float)sd->dims[0]; f[2] = (float)sd->dims[1]; f[3] = (float)sd->dims[2];
      f[4] = sd->origin[0]; f[5] = sd->origin[1]; f[6] = sd->origin[2]; f[7] = sd->cell;
      f[8] = c.R[0]; f[9] = c.R[3]; f[10] = c.R[6]; f[11] = 0;
      f[12] = c.R[1]; f[13] = c.R[4]; f[14] = c.R[7]; f[15] = 0;
      f[16] = c.R[2]; f[17] = c.R[5]; f[18] = c.R[8]; f[19] = 0;
      f[20] = c.pos[0]; f[21] = c.pos[1]; f[22] = c.pos[2]; f[23] = 0;
      f[24] = c.vel[0]; f[25] = c.vel[1]; f[26] = c.vel[2]; f[27] = 0;
      f[28] = c.ang[0]; f[29] = c.ang[1]; f[30] = c.ang[2]; f[31] = 0;
    }
  }
  return ST_OK;
}

// float4s of the drip buffer for n samples: the samples (2 each), the pass's scratch (2 each) and the chunk counts
static size_t drip_words(uint32_t n) { return 4 * (size_t)n + ((size_t)n / DRIP_T + 4 + 3) / 4; }

// dripUpdate (src/flip/sim.js:352-363): the samples of every collider's distance grid, rebuilt when the grids of the
// colliders (in collider order) change; a rebuilt set starts dry
static st_status drip_update(st_flip* s, const st_step_opts* o, uint32_t nc, cudaStream_t q) {
  std::string sig;
  for (uint32_t k = 0; k < nc; k++) sig += std::to_string(o->cols[k].sdf->id) + ",";
  if (sig == s->dripSig) return ST_OK;
  std::vector<float> all;
  for (uint32_t k = 0; k < nc; k++) {
    const st_sdf* sd = o->cols[k].sdf;
    auto it = s->dripCache.find(sd->id);
    if (it == s->dripCache.end()) {
      std::vector<float> v;
      drip_samples(sd, s->h, 0, v);
      if (s->dripCache.size() >= 32) s->dripCache.erase(s->dripCache.begin());
      it = s->dripCache.emplace(sd->id, std::move(v)).first;
    }
    const size_t at = all.size();
    all.insert(all.end(), it->second.begin(), it->second.end());
    for (size_t i = at + 3; i < all.size(); i += 8) all[i] = (float)k;
  }
  const uint32_t n = (uint32_t)(all.size() / 8);
  if (n > s->dripCap) {
    CK(cudaStreamSynchronize(q));
    drop_graphs(s);   // captured steps hold the old buffer
    if (s->drip) cudaFree(s->drip);
    s->drip = nullptr;
    s->dripCap = 0;
    CK(dalloc(&s->drip, drip_words(n)));
    s->dripCap = n;
  }
  if (n) {
    CK(cudaMemcpyAsync(s->drip, all.data(), all.size() * sizeof(float), cudaMemcpyHostToDevice, q));
    CK(cudaStreamSynchronize(q));
  }
  s->ndrip = n;
  s->dripSig = sig;
  return ST_OK;
}

// the parameter block (src/flip/sim.js:196-231): host values in double, rounded once to f32
static void pack_params(st_flip* s, double dt, const st_step_opts* o, uint32_t nc, uint32_t init, bool nbOn, bool sprOn) {
  FlipParams& P = s->hp;
  memset(&P, 0, sizeof(P));
  P.n = s->N; P.nx = s->nx; P.ny = s->ny; P.nz = s->nz; P.ncols = nc; P.open = s->open;
  P.tx = s->tx; P.ty = s->ty; P.tz = s->tz; P.ntiles = s->ntiles;
  P.dt = (float)dt; P.h = (float)s->h; P.ih = (float)(1.0 / s->h); P.gravity = o->g; P.flip = o->flip; P.rest = (float)s->rest;
  P.comp = o->comp;
  double omAuto = std::min(1.9, 2.0 / (1.0 + std::sin(M_PI / std::max(s->nx, std::max(s->ny, s->nz)))));
  P.omega = o->omega != 0.0f ? o->omega : (float)omAuto;
  P.x0 = (float)s->bx0; P.y0 = (float)s->by0; P.z0 = (float)s->bz0; P.vmax = o->vmax != 0.0f ? o->vmax : 14.0f;
  P.margin = (float)(0.3 * s->d); P.scale = 65536.0f; P.x1 = (float)s->bx1; P.y1 = (float)s->by1; P.z1 = (float)s->bz1;
  P.q0 = (float)(0.3 * s->h); P.q1 = o->wind[0]; P.q2 = o->wind[1]; P.q3 = o->wind[2]; P.q4 = o->drag;
  P.q5 = o->foam_tau != 0.0f ? o->foam_tau : 1.2f; P.q6 = o->foam_sens != 0.0f ? o->foam_sens : 1.0f; P.q7 = o->gust;
  P.q8 = (float)s->tm; P.q9 = (o->flags & ST_OPT_NO_FOAM) ? 1.0f : 0.0f; P.q10 = (o->flags & ST_OPT_NO_CULL) ? 1.0f : 0.0f;
  P.q12 = (o->flags & ST_OPT_FAST_AIR) ? 1.0f : 0.0f;
  const st_spray_opts& sp = o->spray;
  P.sheetMin = o->tear; P.sprRate = sprOn ? sp.rate : 0.0f; P.sprMin = sprOn ? std::max(0.05f, sp.min) : 1.0f;
  P.sprLife = sprOn ? sp.life : 1.0f; P.mistFrac = sprOn ? sp.mist : 0.0f; P.sprDrag = sprOn ? sp.drag : 1.0f;
  P.mistDrag = sprOn ? sp.mdrag : 4.0f; P.vs = o->vs != 0.0f ? o->vs : 1.0f;
  P.smax = s->sprayCap; P.seed = s->seed; P.nb = nbOn ? 1u : 0u; P.nbInit = init; P.sprayOn = sprOn ? 1u : 0u;
  uint64_t pool = (uint64_t)(s->ntiles + 1) * 512;
  P.lcap = s->velGOn ? (uint32_t)std::min<uint64_t>(pool, 0xffffffffu) : (uint32_t)std::min<uint64_t>(pool, s->maxN);
  P.stamp = s->stamp;
  P.band = std::max(2.0f, o->nb_band != 0.0f ? o->nb_band : 3.0f);
  P.wwFoamLife = sp.foam_life != 0.0f ? sp.foam_life : 3.0f; P.wwRise = sp.rise != 0.0f ? sp.rise : 0.3f;
  P.wwCrest = sp.crest; P.wwImpact = sp.impact;
  // air field (words 72-76, 82): on only with whitewater on this step
  const bool airOn = sprOn && o->air_on != 0 && s->airCells != 0;
  P.airOn = airOn ? 1u : 0u; P.airCouple = airOn ? o->air_couple : 0.0f; P.airDecay = airOn ? o->air_decay : 0.0f;
  P.airH = s->airCells ? (float)s->airH : 1.0f; P.airBlur = airOn ? o->air_blur : 0.0f;
  P.aNx = s->airCells ? s->aNx : 1u; P.aNy = s->airCells ? s->aNy : 1u; P.aNz = s->airCells ? s->aNz : 1u;
  // ocean (words 57-61, 63, 66 and the wave list, src/flip/sim.js:210-218)
  const bool oc = o->ocean_on != 0;
  P.ocean = oc ? 1u : 0u;
  P.nwave = oc ? (uint32_t)ocean_waves(o, (double)o->g, (double)o->ocean_level - s->by0, s->waves) : 0u;
  P.otime = o->time; P.olevel = oc ? o->ocean_level : 0.0f; P.olayer = oc ? o->ocean_layer : 0.0f; P.oy0 = (float)s->by0;
  P.odepth = oc ? (float)std::max((double)o->ocean_level - s->by0, 1e-3) : 1.0f;
  // drips (words 79-81): on only with whitewater on this step
  const bool drOn = sprOn && o->drip_on != 0;
  P.ndrip = drOn ? s->ndrip : 0u; P.dripRate = drOn ? o->drip_rate : 0.0f; P.dripDry = drOn ? o->drip_dry : 1.0f;
  uint32_t nf = init ? (uint32_t)std::min<size_t>(s->fills.size() / 8, 8) : 0u;
  P.nfill = nf;
  for (uint32_t k = 0; k < nf; k++) memcpy(P.fills[k * 2], &s->fills[k * 8], 8 * sizeof(float));
}

}  // extern "C"

static void stage_fill(st_stage_times* t, const float* ms, float total) {
  t->sort = 0.0f; t->blocks = ms[0]; t->clear = 0.0f; t->p2g = ms[1]; t->narrow_band = ms[2]; t->classify = ms[3];
  t->norm_faces = ms[4]; t->divergence = 0.0f; t->pressure = ms[5]; t->project = ms[6]; t->g2p = ms[7]; t->spray = ms[8];
  t->reseed = ms[9]; t->pbf = ms[10]; t->total = total;
}

// The device work of one step after the uploads: counters reset, then the stages in the reference's order
// (src/flip/sim.js:253-309), then the PBF density stage when pbfIters > 0. mark(k) is called at the 12 stage
// boundaries. The front half runs up to the pressure sweeps, the back half from the projection on; a pooled batch
// runs its tanks' sweeps between the two. Each returns the kernels it launched.
template <class Mark>
static int enqueue_front(st_flip* s, const Bufs& B, cudaStream_t q, bool nbOn, uint32_t init, Mark mark) {
  cudaMemsetAsync(&s->dCtl->fluid, 0, 3 * sizeof(uint32_t), q);        // fluid, vmaxBits, nLive (nActive is kept)
  cudaMemsetAsync(&s->dCtl->nDropped, 0, sizeof(uint32_t), q);
  cudaMemsetAsync(&s->dCtl->emitTried, 0, 2 * sizeof(uint32_t), q);     // emitTried, nFluidTiles
  const int gT4 = s->tileGrid(s->gridT4);
  int nl = 0;
  mark(0);
  // blocks + sort: mark and count, activate tiles, offsets, scatter (the sort is part of the blocks stage)
  nl += launch_count_mark(B, q);
  if (nbOn && init != 1) nl += launch_mark_phi(B, gT4, q);
  if (init) nl += launch_mark_fill(B, std::max(1, (int)std::min<uint32_t>((s->ntiles + 255) / 256, 4096)), q);
  nl += launch_tiles(B, s->ntiles, gT4, q);
  if (init) nl += launch_nb_init(B, gT4, q);
  nl += launch_scan_counts(B, q);
  nl += launch_scatter(B, q);
  mark(1);
  nl += launch_p2g(B, s->tileGrid(std::min(s->gridT, p2g_ctas_per_sm())), q);   // dynamic tiles: resident CTAs only
  mark(2);
  if (nbOn) nl += launch_nb_phi(B, gT4, q);
  mark(3);
  const bool ocean = s->hp.ocean != 0;
  nl += launch_classify(B, gT4, ocean, q);
  if (nbOn) nl += launch_nb_vel(B, gT4, q);
  mark(4);
  nl += launch_norm_div(B, gT4, ocean, q);
  mark(5);
  return nl;
}
template <class Mark>
static int enqueue_back(st_flip* s, const Bufs& B, cudaStream_t q, bool nbOn, bool sprOn, int pbfIters, Mark mark) {
  const int gT4 = s->tileGrid(s->gridT4);
  const bool ocean = s->hp.ocean != 0;
  int nl = 0;
  mark(6);
  nl += launch_project(B, gT4, q);
  mark(7);
  nl += launch_g2p(B, s->tileGrid(std::min(s->gridT, g2p_ctas_per_sm(ocean))), ocean, q);   // dynamic tiles: resident CTAs only
  mark(8);
  if (s->sprayCap > 0) nl += launch_spray(B, s->sprayCap, sprOn, s->hp.airOn ? s->airCells : 0u, s->hp.ndrip != 0 ? s->dripCap : 0u, gT4, q);
  mark(9);
  if (nbOn) nl += launch_nb_reseed(B, gT4, q);
  mark(10);
  // the density stage last: the whitewater, the air field and the narrow band's trim and refill above all see the
  // particles g2p moved (their emission counts and trim tests are fused into g2p)
  if (pbfIters > 0) nl += launch_flip_pbf(B, s->pbf, pbfIters, std::max(1, std::min<int>(s->sms * 8, (int)((s->N + PBF_T - 1) / PBF_T))), q);
  mark(11);
  return nl;
}
template <class Mark>
static int enqueue_step(st_flip* s, const Bufs& B, cudaStream_t q, bool nbOn, uint32_t init, bool sprOn, int iters, int pbfIters, Mark mark) {
  int nl = enqueue_front(s, B, q, nbOn, init, mark);
  nl += launch_sor_compact(B, s->tileGrid(s->gridSor), s->tileGrid(s->gridT4), iters, q);
  return nl + enqueue_back(s, B, q, nbOn, sprOn, pbfIters, mark);
}

// A step's kernels as a CUDA graph, keyed by everything that changes what is launched: the particle buffer parity,
// the particle count (grid sizes), SOR iterations, narrow band, whitewater emission, the air field, drips, the ocean
// and stage timing. Stage markers are external event-record nodes, pointed at the timing ring's events before each
// launch.
static uint64_t graph_key(const st_flip* s, bool nbOn, bool sprOn, int iters, int pbfIters, bool timing) {
  return (uint64_t)s->cur | ((uint64_t)s->parity << 1) | ((uint64_t)nbOn << 2) | ((uint64_t)sprOn << 3) | ((uint64_t)timing << 4) |
         ((uint64_t)(s->hp.airOn != 0) << 5) | ((uint64_t)(s->hp.ndrip != 0) << 6) | ((uint64_t)(s->hp.ocean != 0) << 7) |
         ((uint64_t)(iters & 0xffff) << 8) | ((uint64_t)s->N << 24) | ((uint64_t)(pbfIters & 0xff) << 56);
}
static st_status get_graph(st_flip* s, const Bufs& B, bool nbOn, bool sprOn, int iters, int pbfIters, bool timing, st_flip::Graph** out) {
  const uint64_t key = graph_key(s, nbOn, sprOn, iters, pbfIters, timing);
  for (auto& g : s->graphs) if (g.exec && g.key == key) { *out = &g; return ST_OK; }
  if (s->graphs.size() >= 8) {   // a small cache: drop the oldest
    if (s->graphs.front().exec) cudaGraphExecDestroy(s->graphs.front().exec);
    if (s->graphs.front().graph) cudaGraphDestroy(s->graphs.front().graph);
    s->graphs.erase(s->graphs.begin());
  }
  cudaStream_t q = s->stream;
  cudaGraph_t graph = nullptr;
  CK(cudaStreamBeginCapture(q, cudaStreamCaptureModeThreadLocal));
  int nl = enqueue_step(s, B, q, nbOn, 0, sprOn, iters, pbfIters, [&](int k) {
    if (timing) cudaEventRecordWithFlags(s->tev[0][k], q, cudaEventRecordExternal);
  });
  cudaError_t e = cudaStreamEndCapture(q, &graph);
  if (e != cudaSuccess) { set_err("graph capture", e); return ST_DEVICE_ERROR; }
  st_flip::Graph g;
  g.key = key;
  g.launches = nl;
  e = cudaGraphInstantiate(&g.exec, graph, 0);
  if (e == cudaSuccess && timing) {
    size_t n = 0;
    cudaGraphGetNodes(graph, nullptr, &n);
    std::vector<cudaGraphNode_t> nodes(n);
    cudaGraphGetNodes(graph, nodes.data(), &n);
    int found = 0;
    for (size_t k = 0; k < n && found < st_flip::TEV; k++) {
      cudaGraphNodeType ty;
      cudaGraphNodeGetType(nodes[k], &ty);
      if (ty != cudaGraphNodeTypeEventRecord) continue;
      cudaEvent_t ev;
      cudaGraphEventRecordNodeGetEvent(nodes[k], &ev);
      for (int j = 0; j < st_flip::TEV; j++) if (ev == s->tev[0][j]) { g.evnode[j] = nodes[k]; found++; }
    }
    if (found != st_flip::TEV) e = cudaErrorInvalidValue;
  }
  if (e != cudaSuccess) {
    set_err("graph instantiate", e);
    if (g.exec) cudaGraphExecDestroy(g.exec);
    cudaGraphDestroy(graph);
    return ST_DEVICE_ERROR;
  }
  g.graph = graph;   // kept: its event-record node handles are updated before each launch
  s->graphs.push_back(g);
  *out = &s->graphs.back();
  return ST_OK;
}
static void drop_graphs(st_flip* s) {
  for (auto& g : s->graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
  }
  s->graphs.clear();
  s->gen++;
}

// The host half of a step: parameter block, collider records and counters, with the uploads enqueued on q.
struct StepPrep { bool nbOn = false, sprOn = false; uint32_t init = 0; int iters = 1, pbfIters = 0; };
static st_status prepare_step(st_flip* s, double dt, const st_step_opts* o, cudaStream_t q, StepPrep* pr) {
  const bool nbOn = o->nb_on != 0 || o->ocean_on != 0;   // the ocean keeps its water by depth: it turns the narrow band on
  if (nbOn) s->velGOn = true;
  const uint32_t init = nbOn && s->nbInit ? s->nbInit : 0;
  // the next pinned upload block: wait for the copy that last read it
  st_flip::Upload* up = &s->ring_h[s->ring_i];
  cudaEvent_t upEv = s->ring_ev[s->ring_i];
  s->ring_i = (s->ring_i + 1) % st_flip::RING;
  CK(cudaEventSynchronize(upEv));
  uint32_t nc = 0, nfv = 0;
  st_status st;
  if (init && !s->fillVols.empty()) {   // a restart packs the fill volumes after the colliders (src/flip/sim.js:189-190)
    const uint32_t ncStep = std::min(o->ncols, 32u);
    if (ncStep && !o->cols) return ST_BAD_ARG;
    std::vector<st_collider> all;
    if (ncStep) all.assign(o->cols, o->cols + ncStep);
    for (auto& f : s->fillVols) {
      f.sd.data = f.data.data();
      all.push_back(f.c);
      all.back().sdf = &f.sd;
    }
    st_step_opts o2 = *o;
    o2.cols = all.data();
    o2.ncols = (uint32_t)all.size();
    st = pack_colliders(s, &o2, nc, up->cols, q);
    if (st != ST_OK) return st;
    nfv = nc - std::min(ncStep, nc);
    nc -= nfv;
  } else {
    st = pack_colliders(s, o, nc, up->cols, q);
    if (st != ST_OK) return st;
  }
  const bool sprOn = o->spray_on != 0 && s->sprayCap > 0;
  if (sprOn && o->drip_on) {
    st = drip_update(s, o, nc, q);
    if (st != ST_OK) return st;
  }
  s->seed = s->seed + 1u;
  s->stamp = s->stamp + 1u;
  pack_params(s, dt, o, nc, init, nbOn, sprOn);
  s->hp.nfv = nfv;
  s->tm = s->tm + dt;
  // the live view's water sample (src/flip/sim.js:184): every stride-th particle, at most about DISP_MAX
  s->stride = std::max<uint32_t>(1u, (uint32_t)((s->N + st_flip::DISP_MAX - 1) / st_flip::DISP_MAX));
  s->lastN = s->N;
  s->lastNb = nbOn;
  if (init) { s->nbInit = 0; s->fills.clear(); s->fillVols.clear(); }
  const int iters = std::max(1, o->iters);
  // the PBF density stage: its block (FluidSim's constants for this spacing, the tank's box and walls, this step's dt
  // and colliders) and, on first use, its buffers (outside any graph capture)
  const int pbfIters = std::min(std::max(o->pbf_iters, 0), 64);
  if (pbfIters > 0) {
    if (!s->pbf.key) {
      s->pbfc = pbf_consts(s->d, 0.0, 0.0);
      const double lo[3] = {s->bx0, s->by0, s->bz0}, hi[3] = {s->bx1, s->by1, s->bz1};
      const PbfParams P0 = pbf_params(s->pbfc, s->d, lo, hi, dt, 0.0, 0.0, 0, 0, s->open);
      s->pbfCells = P0.ncell;
      cudaError_t e = pbf_dev_alloc(s->pbf, s->maxN, s->pbfCells);
      if (e != cudaSuccess) { pbf_dev_free(s->pbf); set_err("pbf stage buffers", e); return e == cudaErrorMemoryAllocation ? ST_OOM : ST_DEVICE_ERROR; }
      cudaFree(s->pbf.P);   // the block lives in the upload buffer
    }
    s->pbf.P = &s->dUp->pbf;
    const double lo[3] = {s->bx0, s->by0, s->bz0}, hi[3] = {s->bx1, s->by1, s->bz1};
    up->pbf = pbf_params(s->pbfc, s->d, lo, hi, dt, 0.0, 0.0, s->N, nc, s->open);
  }
  // this step's storage order goes into the other particle buffer; cell counts alternate buffers
  s->cur ^= 1;
  s->parity ^= 1;
  up->P = s->hp;
  CK(cudaMemcpyAsync(&s->dUp->P, &up->P, sizeof(FlipParams), cudaMemcpyHostToDevice, q));
  if (nc + nfv) CK(cudaMemcpyAsync(s->dUp->cols, up->cols, (nc + nfv) * 32 * sizeof(float), cudaMemcpyHostToDevice, q));
  if (s->hp.nwave) {
    memcpy(up->waves, s->waves, s->hp.nwave * 8 * sizeof(float));
    CK(cudaMemcpyAsync(s->dUp->waves, up->waves, s->hp.nwave * 8 * sizeof(float), cudaMemcpyHostToDevice, q));
  }
  if (pbfIters > 0) CK(cudaMemcpyAsync(&s->dUp->pbf, &up->pbf, sizeof(PbfParams), cudaMemcpyHostToDevice, q));
  CK(cudaEventRecord(upEv, q));
  pr->nbOn = nbOn; pr->sprOn = sprOn; pr->init = init; pr->iters = iters; pr->pbfIters = pbfIters;
  return ST_OK;
}

// a finished step's device time joins the last 31 (the median is lastMs) and the slowest so far (slowMs)
static void trk_take(st_flip* s) {
  const int k = (int)(s->trkTail % st_flip::TRK);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, s->trkStart[k], s->trkDone[k]);
  s->trkMs[s->trkPos] = ms;
  s->trkPos = (s->trkPos + 1) % 31;
  if (s->trkN < 31) s->trkN++;
  float r[31];
  for (int i = 0; i < s->trkN; i++) r[i] = s->trkMs[i];
  std::sort(r, r + s->trkN);
  s->lastMs = r[s->trkN >> 1];
  s->slowMs = std::max(s->slowMs, ms);
  s->trkTail++;
}
// read back every finished step, in order; wait for the oldest first when the ring is full
static st_status trk_poll(st_flip* s, bool full) {
  if (full && s->trkHead - s->trkTail == (uint64_t)st_flip::TRK) {
    CK(cudaEventSynchronize(s->trkDone[s->trkTail % st_flip::TRK]));
    trk_take(s);
  }
  while (s->trkTail < s->trkHead) {
    const cudaError_t e = cudaEventQuery(s->trkDone[s->trkTail % st_flip::TRK]);
    if (e == cudaErrorNotReady) break;
    CK(e);
    trk_take(s);
  }
  return ST_OK;
}

// one step; t (optional) receives device ms per stage
static st_status do_step(st_flip* s, double dt, const st_step_opts* o, st_stage_times* t) {
  if (!s || !o || o->size != sizeof(st_step_opts)) return ST_BAD_ARG;
  if (s->N == 0) return ST_NOT_READY;
  CK(cudaSetDevice(s->device));
  cudaStream_t q = s->stream;
  StepPrep pr;
  st_status st = prepare_step(s, dt, o, q, &pr);
  if (st != ST_OK) return st;
  const bool nbOn = pr.nbOn, sprOn = pr.sprOn;
  const uint32_t init = pr.init;
  const int iters = pr.iters;
  const Bufs B = s->bufs();
  cudaEvent_t* tslot = nullptr;
  if (s->timing) {
    if (s->tcount >= (uint32_t)st_flip::TSLOTS) CK(cudaEventSynchronize(s->tev[s->tcount % st_flip::TSLOTS][st_flip::TEV - 1]));
    tslot = s->tev[s->tcount % st_flip::TSLOTS];
  }
  if (!s->trkStart[0])
    for (int k = 0; k < st_flip::TRK; k++) {
      CK(cudaEventCreate(&s->trkStart[k]));
      CK(cudaEventCreate(&s->trkDone[k]));
    }
  if ((st = trk_poll(s, true)) != ST_OK) return st;
  const int tk = (int)(s->trkHead % st_flip::TRK);
  int nl = 0;
  if (s->use_graphs && !t && !init) {
    st_flip::Graph* g = nullptr;
    st = get_graph(s, B, nbOn, sprOn, iters, pr.pbfIters, tslot != nullptr, &g);
    if (st != ST_OK) return st;
    if (tslot)
      for (int k = 0; k < st_flip::TEV; k++) CK(cudaGraphExecEventRecordNodeSetEvent(g->exec, g->evnode[k], tslot[k]));
    CK(cudaEventRecord(s->trkStart[tk], q));   // after the host work, so a new graph's instantiation is not timed
    CK(cudaGraphLaunch(g->exec, q));
    nl = g->launches;
  } else {
    CK(cudaEventRecord(s->trkStart[tk], q));
    nl = enqueue_step(s, B, q, nbOn, init, sprOn, iters, pr.pbfIters, [&](int k) {
      if (t) cudaEventRecord(s->ev[k], q);
      if (tslot) cudaEventRecord(tslot[k], q);
    });
  }
  s->launches += (uint64_t)nl;
  CK(cudaGetLastError());
  CK(cudaEventRecord(s->trkDone[tk], q));
  s->trkHead++;
  s->steps++;
  if (tslot) s->tcount++;
  if (t) {
    constexpr int L = st_flip::TEV - 1;
    CK(cudaEventSynchronize(s->ev[L]));
    float ms[L];
    for (int k = 0; k < L; k++) cudaEventElapsedTime(&ms[k], s->ev[k], s->ev[k + 1]);
    float tot = 0.0f;
    cudaEventElapsedTime(&tot, s->ev[0], s->ev[L]);
    stage_fill(t, ms, tot);
  }
  return ST_OK;
}

extern "C" {

st_status st_flip_step(st_flip* s, double dt, const st_step_opts* o) { return do_step(s, dt, o, nullptr); }

st_status st_flip_set_timing(st_flip* s, int on) {
  if (!s) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  if (on && !s->tev[0][0])
    for (auto& row : s->tev) for (auto& e : row) CK(cudaEventCreate(&e));
  s->timing = on != 0;
  s->tcount = 0;
  return ST_OK;
}
// sum of the stage times of the steps recorded since st_flip_set_timing (at most the last 256)
st_status st_flip_read_timing(st_flip* s, st_stage_times* sum, uint32_t* nsteps) {
  if (!s || !sum) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  memset(sum, 0, sizeof(*sum));
  uint32_t n = std::min<uint32_t>(s->tcount, st_flip::TSLOTS);
  if (n) CK(cudaStreamSynchronize(s->stream));
  constexpr int L = st_flip::TEV - 1;
  float acc[L] = {0}, tot = 0.0f;
  for (uint32_t k = 0; k < n; k++) {
    cudaEvent_t* e = s->tev[(s->tcount - 1 - k) % st_flip::TSLOTS];
    for (int j = 0; j < L; j++) { float ms = 0.0f; CK(cudaEventElapsedTime(&ms, e[j], e[j + 1])); acc[j] += ms; }
    float ms = 0.0f; CK(cudaEventElapsedTime(&ms, e[0], e[L])); tot += ms;
  }
  stage_fill(sum, acc, tot);
  if (nsteps) *nsteps = n;
  s->tcount = 0;
  return ST_OK;
}
st_status st_flip_step_timed(st_flip* s, double dt, const st_step_opts* o, st_stage_times* t) {
  if (!t) return ST_BAD_ARG;
  return do_step(s, dt, o, t);
}

static void stats_fill(const Ctl& c, uint32_t n, uint64_t steps, uint64_t launches, st_stats* out) {
  out->sc = c.nActive; out->ovf = 0; out->fluid = c.fluid;
  uint32_t vb = c.vmaxBits; float vm; memcpy(&vm, &vb, 4); out->vmax = vm;
  out->n = n; out->live = steps ? c.nLive : n; out->spray_used = c.sctl0; out->steps = steps;
  out->launches = launches; out->spray_overflow = c.sprayOvf;
}

st_status st_flip_stats(st_flip* s, st_stats* out) {
  if (!s || !out) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  CK(cudaMemcpyAsync(s->hCtl, s->dCtl, sizeof(Ctl), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  stats_fill(*s->hCtl, s->N, s->steps, s->launches, out);
  return ST_OK;
}

st_status st_flip_track(st_flip* s, uint32_t* inflight, float* last_ms, float* slow_ms) {
  if (!s) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  st_status st = trk_poll(s, false);
  if (st != ST_OK) return st;
  if (inflight) *inflight = (uint32_t)(s->trkHead - s->trkTail);
  if (last_ms) *last_ms = s->lastMs;
  if (slow_ms) *slow_ms = s->slowMs;
  return ST_OK;
}

st_status st_flip_stats_async(st_flip* s, uint64_t* ticket) {
  if (!s || !ticket) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  st_flip::StatSlot& q = s->stat[s->statNext % st_flip::STAT_SLOTS];
  if (q.pending) {   // the ring is full: the oldest copy has to land before its slot is reused
    q.pending = false;
    CK(cudaEventSynchronize(q.ev));
  }
  if (!q.h) {
    CK(cudaHostAlloc((void**)&q.h, sizeof(Ctl), cudaHostAllocDefault));
    CK(cudaEventCreateWithFlags(&q.ev, cudaEventDisableTiming));
  }
  CK(cudaMemcpyAsync(q.h, s->dCtl, sizeof(Ctl), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaEventRecord(q.ev, s->stream));
  q.ticket = s->statNext; q.n = s->N; q.steps = s->steps; q.launches = s->launches; q.pending = true;
  *ticket = s->statNext++;
  return ST_OK;
}

st_status st_flip_stats_wait(st_flip* s, uint64_t ticket, st_stats* out) {
  if (!s || !out) return ST_BAD_ARG;
  st_flip::StatSlot& q = s->stat[ticket % st_flip::STAT_SLOTS];
  if (ticket == 0 || q.ticket != ticket) {   // never issued, or its slot has been reused since
    st::set_error_text("st_flip_stats_wait: ticket not issued or no longer held");
    return ST_BAD_ARG;
  }
  CK(cudaSetDevice(s->device));
  CK(cudaEventSynchronize(q.ev));
  q.pending = false;
  stats_fill(*q.h, q.n, q.steps, q.launches, out);
  return ST_OK;
}

// particles in id order: unsort on the device into the free particle buffer, then copy out
st_status st_flip_read_particles(st_flip* s, float* pos4, float* vel4, uint32_t cap, uint32_t* n) {
  if (!s || !pos4) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  if (n) *n = s->N;
  uint32_t m = std::min(cap, s->N);
  if (m == 0) return ST_OK;
  float4* tmp = reinterpret_cast<float4*>(s->part[s->cur ^ 1]);   // 2 float4 per particle of room
  launch_unsort(s->part[s->cur], s->ids[s->cur], s->N, tmp, vel4 ? tmp + s->N : nullptr, s->stream);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(pos4, tmp, (size_t)m * 16, cudaMemcpyDeviceToHost, s->stream));
  if (vel4) CK(cudaMemcpyAsync(vel4, tmp + s->N, (size_t)m * 16, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return ST_OK;
}

// ---- the live view and a frame's whitewater / deep-water parts (live.cu) ----
}  // extern "C"
template <class T>
static cudaError_t grow(T** p, size_t& have, size_t need) {   // a device buffer of at least need elements
  if (need <= have && *p) return cudaSuccess;
  if (*p) cudaFree(*p);
  *p = nullptr;
  have = 0;
  cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(need, 1) * sizeof(T));
  if (e == cudaSuccess) have = need;
  return e;
}
extern "C" {
static FrameBox frame_box(const st_flip* s, float vs) {
  return FrameBox{s->bx0, s->by0, s->bz0, 65535.0 / (s->bx1 - s->bx0), 65535.0 / (s->by1 - s->by0), 65535.0 / (s->bz1 - s->bz0),
                  16.0 * (vs != 0.0f ? (double)vs : 1.0)};
}
static bool deep_ready(const st_flip* s) { return s->deepOn && s->lastNb && s->velGOn && s->lastN; }
// deepClear + deepPick + deepFin (src/flip/wgsl-whitewater.js:282-297): the deep points into deepBuf; returns how many
static st_status deep_pass(st_flip* s, uint32_t* n) {
  if (!s->deepBuf) CK(cudaMalloc((void**)&s->deepBuf, (size_t)st_flip::DEEP_MAX * sizeof(float4)));
  CK(grow(&s->viewScratch, s->viewScratchN, std::max<size_t>(s->ntiles, 1) + 2));
  uint32_t* counts = s->viewScratch + std::max<size_t>(s->ntiles, 1);
  const Bufs B = s->bufs();
  launch_deep(B, s->deepPrev, s->ntiles, s->tileGrid(s->gridT4), s->viewScratch, counts, s->deepBuf, s->stream);
  uint32_t h[2];
  CK(cudaMemcpyAsync(h, counts, 8, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaGetLastError());
  s->deepPrev = h[0];
  *n = std::min(h[1], st_flip::DEEP_MAX);
  return ST_OK;
}

st_status st_flip_read_deep_points(st_flip* s, float* out4, uint32_t cap, uint32_t* n) {
  if (!s || !n) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  *n = 0;
  if (!deep_ready(s)) return ST_OK;
  uint32_t nd = 0;
  st_status st = deep_pass(s, &nd);
  if (st != ST_OK) return st;
  *n = nd;
  const uint32_t m = std::min(nd, cap);
  if (out4 && m) {
    CK(cudaMemcpyAsync(out4, s->deepBuf, (size_t)m * sizeof(float4), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
  }
  return m < nd ? ST_OVERFLOW : ST_OK;
}

st_status st_flip_set_recycle(st_flip* s, int on) {
  if (!s) return ST_BAD_ARG;
  s->recycle = on != 0;
  return ST_OK;
}

st_status st_flip_set_spray_cap(st_flip* s, uint32_t n) {
  if (!s) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  if (n == s->sprayCap) return ST_OK;
  CK(cudaStreamSynchronize(s->stream));
  drop_graphs(s);   // captured steps hold the old pool
  float4 *p = nullptr, *v = nullptr;
  cudaError_t e = dalloc(&p, std::max<size_t>(n, 1));
  if (e == cudaSuccess) e = dalloc(&v, std::max<size_t>(n, 1));
  if (e != cudaSuccess) {
    if (p) cudaFree(p);
    set_err("spray pool", e);
    return e == cudaErrorMemoryAllocation ? ST_OOM : ST_DEVICE_ERROR;
  }
  CK(cudaMemsetAsync(p, 0, std::max<size_t>(n, 1) * 16, s->stream));
  CK(cudaMemsetAsync(v, 0, std::max<size_t>(n, 1) * 16, s->stream));
  if (n && !s->airCells) {   // the air field comes with the first pool (airAlloc, src/flip/sim.js:343-350)
    const double cells = (double)s->nx * (double)s->ny * (double)s->nz;
    const int r = std::max(2, (int)std::ceil(std::cbrt(cells / 260000.0)));
    const uint32_t ax = (uint32_t)((s->nx + r - 1) / r + 1), ay = (uint32_t)((s->ny + r - 1) / r + 1), az = (uint32_t)((s->nz + r - 1) / r + 1);
    const uint32_t na = ax * ay * az;
    CK(dalloc(&s->air, na)); CK(dalloc(&s->air2, na)); CK(dalloc(&s->airAcc, 4 * (size_t)na));
    CK(cudaMemsetAsync(s->air, 0, (size_t)na * 16, s->stream));
    CK(cudaMemsetAsync(s->air2, 0, (size_t)na * 16, s->stream));
    s->airH = s->h * r; s->aNx = ax; s->aNy = ay; s->aNz = az; s->airCells = na;
    s->createBytes += (size_t)na * 48;
  }
  s->createBytes += 32 * std::max<size_t>(n, 1);
  s->createBytes -= 32 * std::max<size_t>(s->sprayCap, 1);
  CK(cudaStreamSynchronize(s->stream));
  cudaFree(s->sPos);
  cudaFree(s->sVel);
  s->sPos = p;
  s->sVel = v;
  s->sprayCap = n;   // the ring counter keeps counting, as the reference's sctl does
  return ST_OK;
}

st_status st_flip_mem_bytes(st_flip* s, uint64_t* bytes) {
  if (!s || !bytes) return ST_BAD_ARG;
  uint64_t b = s->createBytes;
  b += (uint64_t)s->sdfCap * 4 - 64;                                     // distance grids beyond the first 16 floats
  b += s->frame ? (uint64_t)s->maxN * 8 + 16 : 0;
  b += s->diag ? sizeof(DiagAcc) : 0;
  b += s->deepBuf ? (uint64_t)st_flip::DEEP_MAX * sizeof(float4) : 0;
  b += (uint64_t)s->viewScratchN * 4 + (uint64_t)s->liveWords * 4 + s->framePartBytes + (uint64_t)drip_words(s->dripCap) * 16;
  *bytes = b;
  return ST_OK;
}

st_status st_flip_set_deep_look(st_flip* s, int on) {
  if (!s) return ST_BAD_ARG;
  s->deepOn = on != 0;
  return ST_OK;
}

st_status st_flip_read_deep(st_flip* s, float vs, uint16_t* pos, uint8_t* spd, uint32_t cap, uint32_t* n) {
  if (!s || !n) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  *n = 0;
  if (!deep_ready(s)) return ST_OK;
  uint32_t nd = 0;
  st_status st = deep_pass(s, &nd);
  if (st != ST_OK) return st;
  *n = nd;
  const uint32_t m = std::min(nd, cap);
  if (!m) return nd ? ST_OVERFLOW : ST_OK;
  CK(grow(&s->framePart, s->framePartBytes, (size_t)st_flip::DEEP_MAX * 7));
  uint16_t* p16 = reinterpret_cast<uint16_t*>(s->framePart);
  uint8_t* s8 = s->framePart + (size_t)st_flip::DEEP_MAX * 6;
  launch_pack_deep(s->deepBuf, nd, frame_box(s, vs), p16, s8, s->stream);
  if (pos) CK(cudaMemcpyAsync(pos, p16, (size_t)m * 6, cudaMemcpyDeviceToHost, s->stream));
  if (spd) CK(cudaMemcpyAsync(spd, s8, m, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaGetLastError());
  return m < nd ? ST_OVERFLOW : ST_OK;
}

st_status st_flip_read_spray_frame(st_flip* s, uint32_t max_points, float foam_life, uint16_t* pos, uint32_t* pk, uint32_t cap,
                                   uint32_t* n, uint32_t* alive) {
  if (!s || !n) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  *n = 0;
  if (alive) *alive = 0;
  if (!s->sprayCap) return ST_OK;
  uint32_t used = 0;
  CK(cudaMemcpyAsync(&used, &s->dCtl->sctl0, 4, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  const uint32_t nslots = std::max(1u, std::min(s->sprayCap, used));
  const double fl = (foam_life == foam_life && foam_life != 0.0f) ? (double)foam_life : 3.0;   // foamLife || 3
  CK(grow(&s->viewScratch, s->viewScratchN, std::max<size_t>((nslots + 255) / 256, s->ntiles) + 2));
  uint32_t* counts = s->viewScratch + (s->viewScratchN - 2);
  const size_t codesAt = ((size_t)s->sprayCap * 6 + 15) & ~(size_t)15;   // the codes start 16-byte aligned
  CK(grow(&s->framePart, s->framePartBytes, std::max<size_t>(codesAt + (size_t)s->sprayCap * 4, (size_t)st_flip::DEEP_MAX * 7)));
  uint16_t* p16 = reinterpret_cast<uint16_t*>(s->framePart);
  uint32_t* k32 = reinterpret_cast<uint32_t*>(s->framePart + codesAt);
  launch_spray_frame(s->sPos, s->sVel, nslots, max_points, frame_box(s, 1.0f), fl, s->viewScratch, p16, k32, counts, s->stream);
  uint32_t h[2];
  CK(cudaMemcpyAsync(h, counts, 8, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaGetLastError());
  if (alive) *alive = h[0];
  *n = h[1];
  const uint32_t m = std::min(h[1], cap);
  if (m && pos) CK(cudaMemcpyAsync(pos, p16, (size_t)m * 6, cudaMemcpyDeviceToHost, s->stream));
  if (m && pk) CK(cudaMemcpyAsync(pk, k32, (size_t)m * 4, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return m < h[1] ? ST_OVERFLOW : ST_OK;
}

// packLayout (src/flip/sim.js:371-376)
static void live_layout(uint32_t nW, uint32_t nS, uint32_t nD, st_live_layout* L) {
  const uint32_t gW = (nW + 3) / 4, gS = (nS + 3) / 4, gD = (nD + 3) / 4;
  L->n_water = nW; L->n_spray = nS; L->n_deep = nD;
  L->o_wp = 4; L->o_ws = L->o_wp + gW * 6; L->o_wf = L->o_ws + gW; L->o_sp = L->o_wf + gW; L->o_sk = L->o_sp + gS * 6;
  L->o_dp = L->o_sk + gS * 4; L->o_ds = L->o_dp + gD * 6; L->words = L->o_ds + gD;
}

st_status st_flip_pack_live(st_flip* s, float vs, uint32_t* words, uint64_t cap_words, st_live_layout* L) {
  if (!s || !L || L->size != sizeof(st_live_layout)) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  const uint32_t sdMax = std::min(s->sprayCap, st_flip::SPRAY_DISP_MAX);
  const bool spr = sdMax > 0 && s->lastN, deep = deep_ready(s);
  const bool fromPos = !spr && !deep && (s->stride <= 1 || !s->lastN);
  const uint32_t nW = fromPos ? std::min(std::min(s->N, st_flip::DISP_MAX + 1), s->maxN) : (s->lastN + s->stride - 1) / s->stride;
  live_layout(nW, spr ? sdMax : 0, deep ? st_flip::DEEP_MAX : 0, L);
  L->from_pos = fromPos ? 1u : 0u;
  if (!words) return ST_OK;
  if (cap_words < L->words) return ST_OVERFLOW;
  uint32_t nDeep = 0;
  if (deep) {
    st_status st = deep_pass(s, &nDeep);
    if (st != ST_OK) return st;
  }
  CK(grow(&s->liveOut, s->liveWords, L->words));
  CK(grow(&s->viewScratch, s->viewScratchN, std::max<size_t>((sdMax + 255) / 256, s->ntiles) + 2));
  CK(cudaMemsetAsync(s->liveOut, 0, (size_t)L->words * 4, s->stream));
  if (L->n_deep) CK(cudaMemsetAsync(s->liveOut + L->o_ds, 0xff, (size_t)(L->words - L->o_ds) * 4, s->stream));   // speed 255: no point
  LiveBox K{(float)s->bx0, (float)s->by0, (float)s->bz0, (float)(65535.0 / (s->bx1 - s->bx0)), (float)(65535.0 / (s->by1 - s->by0)),
            (float)(65535.0 / (s->bz1 - s->bz0)), vs != 0.0f ? vs : 1.0f, s->sprayCap, L->n_spray,
            L->o_wp, L->o_ws, L->o_wf, L->o_sp, L->o_sk, L->o_dp, L->o_ds};
  const Bufs B = s->bufs();
  launch_live(B, K, nW, fromPos ? 1u : s->stride, spr ? sdMax : 0u, s->hp.wwFoamLife, s->deepBuf, nDeep, s->viewScratch, s->liveOut, s->stream);
  CK(cudaMemcpyAsync(words, s->liveOut, (size_t)L->words * 4, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaGetLastError());
  words[1] = nDeep;   // header: whitewater points (written by the device), deep points, two zero words
  return ST_OK;
}

// the frame unsorted into the spare particle buffer and packed into s->frame, on the step stream
struct FramePtrs { uint32_t* meta; uint16_t* p16; uint8_t* sp; uint8_t* f8; };
static st_status frame_pack(st_flip* s, float vs, FramePtrs* f) {
  if (!s->frame) {   // packed frame: 6 + 1 + 1 bytes per slot, plus 2 counters
    CK(cudaMalloc((void**)&s->frame, (size_t)s->maxN * 8 + 16));
  }
  f->meta = reinterpret_cast<uint32_t*>(s->frame);
  f->p16 = reinterpret_cast<uint16_t*>(s->frame + 16);
  f->sp = s->frame + 16 + (size_t)s->maxN * 6;
  f->f8 = f->sp + s->maxN;
  float4* tmp = reinterpret_cast<float4*>(s->part[s->cur ^ 1]);
  launch_unsort(s->part[s->cur], s->ids[s->cur], s->N, tmp, nullptr, s->stream);
  FrameBox F{s->bx0, s->by0, s->bz0, 65535.0 / (s->bx1 - s->bx0), 65535.0 / (s->by1 - s->by0), 65535.0 / (s->bz1 - s->bz0),
             16.0 * (vs != 0.0f ? (double)vs : 1.0)};
  CK(cudaMemsetAsync(f->meta, 0, 8, s->stream));
  launch_pack_frame(tmp, s->N, F, f->p16, f->sp, f->f8, f->meta, s->stream);
  CK(cudaGetLastError());
  return ST_OK;
}
// the host has the pending asynchronous frame (s->frame is free again)
static st_status frame_settle(st_flip* s) {
  if (!s->framePending) return ST_OK;
  s->framePending = false;
  CK(cudaEventSynchronize(s->frameCopied));
  return ST_OK;
}

st_status st_flip_read_frame(st_flip* s, float vs, uint16_t* pos, uint8_t* spd, uint8_t* fm, uint32_t cap, uint32_t* n,
                             int32_t* any_foam) {
  if (!s || !n) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  *n = 0;
  if (any_foam) *any_foam = 0;
  if (s->N == 0) return ST_OK;
  st_status r = frame_settle(s);
  if (r != ST_OK) return r;
  FramePtrs f;
  if ((r = frame_pack(s, vs, &f)) != ST_OK) return r;
  uint32_t h[2];
  CK(cudaMemcpyAsync(h, f.meta, 8, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  *n = h[0];
  if (any_foam) *any_foam = (int32_t)h[1];
  const uint32_t m = std::min(cap, h[0]);
  if (m) {
    if (pos) CK(cudaMemcpyAsync(pos, f.p16, (size_t)m * 6, cudaMemcpyDeviceToHost, s->stream));
    if (spd) CK(cudaMemcpyAsync(spd, f.sp, m, cudaMemcpyDeviceToHost, s->stream));
    if (fm && h[1]) CK(cudaMemcpyAsync(fm, f.f8, m, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
  }
  return ST_OK;
}

st_status st_flip_read_frame_async(st_flip* s, float vs, uint16_t* pos, uint8_t* spd, uint8_t* fm, uint32_t cap) {
  if (!s) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  st_status r = frame_settle(s);
  if (r != ST_OK) return r;
  if (!s->copyStream) {
    CK(cudaStreamCreateWithFlags(&s->copyStream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&s->frameReady, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&s->frameCopied, cudaEventDisableTiming));
    CK(cudaHostAlloc((void**)&s->frameMeta, 16, cudaHostAllocDefault));
  }
  s->frameMeta[0] = s->frameMeta[1] = 0;
  if (s->N == 0) return ST_OK;   // nothing pending: the wait gives 0 points
  FramePtrs f;
  if ((r = frame_pack(s, vs, &f)) != ST_OK) return r;
  CK(cudaEventRecord(s->frameReady, s->stream));
  CK(cudaStreamWaitEvent(s->copyStream, s->frameReady, 0));
  CK(cudaMemcpyAsync(s->frameMeta, f.meta, 8, cudaMemcpyDeviceToHost, s->copyStream));
  const uint32_t m = std::min(cap, s->N);   // the point count is not known yet: every slot the caller has room for
  if (m) {
    if (pos) CK(cudaMemcpyAsync(pos, f.p16, (size_t)m * 6, cudaMemcpyDeviceToHost, s->copyStream));
    if (spd) CK(cudaMemcpyAsync(spd, f.sp, m, cudaMemcpyDeviceToHost, s->copyStream));
    if (fm) CK(cudaMemcpyAsync(fm, f.f8, m, cudaMemcpyDeviceToHost, s->copyStream));
  }
  CK(cudaEventRecord(s->frameCopied, s->copyStream));
  s->framePending = true;
  return ST_OK;
}

st_status st_flip_frame_wait(st_flip* s, uint32_t* n, int32_t* any_foam) {
  if (!s) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  if (n) *n = 0;
  if (any_foam) *any_foam = 0;
  if (!s->framePending) return ST_OK;
  st_status r = frame_settle(s);
  if (r != ST_OK) return r;
  if (n) *n = s->frameMeta[0];
  if (any_foam) *any_foam = (int32_t)s->frameMeta[1];
  return ST_OK;
}

st_status st_flip_bake_diag(st_flip* s, float vcap, st_bake_diag* out) {
  if (!s || !out) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  memset(out, 0, sizeof(*out));
  if (!s->diag) CK(cudaMalloc((void**)&s->diag, sizeof(DiagAcc)));
  DiagAcc h{};
  for (int k = 0; k < 3; k++) { h.mn[k] = ~0ull; h.mx[k] = 0; }
  CK(cudaMemcpyAsync(s->diag, &h, sizeof(h), cudaMemcpyHostToDevice, s->stream));
  const double vc = vcap != 0.0f ? (double)vcap : 14.0;
  DiagBox D{s->bx0, s->by0, s->bz0, s->bx1, s->by1, s->bz1, (s->by1 - s->by0) / 16.0, std::min(vc, 63.0) * 0.98};
  launch_bake_diag(s->part[s->cur], s->N, D, s->diag, s->stream);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(&h, s->diag, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  const uint32_t alive = h.count[0];
  const double a = std::max<double>(alive, 1.0);
  auto dbl = [](unsigned long long k) {   // back from the ordered integer
    const unsigned long long u = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    double d;
    memcpy(&d, &u, 8);
    return d;
  };
  out->alive = alive; out->non_finite = h.count[1]; out->gone = s->N - alive - h.count[1];
  out->outside_box = h.count[2]; out->at_speed_limit = h.count[3]; out->foamy = h.count[4];
  out->mean_speed = h.sum[3] / a;
  double smax;
  memcpy(&smax, &h.smax, 8);
  out->max_speed = smax;
  out->mean_foam = h.sum[4] / a / 15.0;
  for (int k = 0; k < 3; k++) out->center[k] = h.sum[k] / a;
  out->has_bbox = alive ? 1 : 0;
  if (alive) for (int k = 0; k < 3; k++) { out->bbox[k] = dbl(h.mn[k]); out->bbox[3 + k] = dbl(h.mx[k]); }
  for (int k = 0; k < 16; k++) out->height_hist[k] = h.hist[k];
  return ST_OK;
}

st_status st_flip_read_spray(st_flip* s, float* pos4, float* vel4, uint32_t cap, uint32_t* n) {
  if (!s) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  if (!s->sprayCap) { if (n) *n = 0; return ST_OK; }
  CK(cudaMemcpyAsync(s->hCtl, s->dCtl, sizeof(Ctl), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  uint32_t m = std::max(1u, std::min(s->sprayCap, s->hCtl->sctl0));
  if (n) *n = m;
  uint32_t c = std::min(m, cap);
  if (pos4 && c) CK(cudaMemcpyAsync(pos4, s->sPos, (size_t)c * 16, cudaMemcpyDeviceToHost, s->stream));
  if (vel4 && c) CK(cudaMemcpyAsync(vel4, s->sVel, (size_t)c * 16, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return ST_OK;
}

st_status st_flip_read_air(st_flip* s, float* vel4, uint32_t cap, uint32_t* dims3) {
  if (!s) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  if (dims3) { dims3[0] = s->aNx; dims3[1] = s->aNy; dims3[2] = s->aNz; }
  const uint32_t m = std::min(cap, s->airCells);
  if (vel4 && m) {
    CK(cudaMemcpyAsync(vel4, s->air, (size_t)m * 16, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
  }
  return ST_OK;
}

st_status st_flip_read_drips(st_flip* s, float* out8, uint32_t cap, uint32_t* n) {
  if (!s) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  if (n) *n = s->ndrip;
  const uint32_t m = std::min(cap, s->ndrip);
  if (out8 && m) {
    CK(cudaMemcpyAsync(out8, s->drip, (size_t)m * 32, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
  }
  return ST_OK;
}

st_status st_flip_read_grid(st_flip* s, const st_flip_grid* g) {
  if (!s || !g) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  const size_t C = s->ncell, T = s->ntiles;
  std::vector<uint8_t> on(T);
  std::vector<int32_t> cnt(C);
  std::vector<uint32_t> ct(C);
  std::vector<float> pr(C), rh(C), vn(3 * C), vo(3 * C), vg(3 * C);
  cudaStream_t q = s->stream;
  CK(cudaMemcpyAsync(on.data(), s->on, T, cudaMemcpyDeviceToHost, q));
  CK(cudaMemcpyAsync(cnt.data(), s->cnt[s->parity], C * 4, cudaMemcpyDeviceToHost, q));
  CK(cudaMemcpyAsync(ct.data(), s->ctype, C * 4, cudaMemcpyDeviceToHost, q));
  CK(cudaMemcpyAsync(pr.data(), s->pres, C * 4, cudaMemcpyDeviceToHost, q));
  CK(cudaMemcpyAsync(rh.data(), s->rhs, C * 4, cudaMemcpyDeviceToHost, q));
  CK(cudaMemcpyAsync(vn.data(), s->vn, 3 * C * 4, cudaMemcpyDeviceToHost, q));
  CK(cudaMemcpyAsync(vo.data(), s->vo, 3 * C * 4, cudaMemcpyDeviceToHost, q));
  CK(cudaMemcpyAsync(vg.data(), s->velG, 3 * C * 4, cudaMemcpyDeviceToHost, q));
  CK(cudaStreamSynchronize(q));
  const uint32_t NX = s->tx * 8, NY = s->ty * 8, NZ = s->tz * 8;
  if (g->tile_on) memcpy(g->tile_on, on.data(), T);
  for (uint32_t k = 0; k < NZ; k++)
    for (uint32_t j = 0; j < NY; j++)
      for (uint32_t i = 0; i < NX; i++) {
        size_t o = (size_t)i + NX * ((size_t)j + NY * k);
        uint32_t t = (i >> 3) + s->tx * ((j >> 3) + s->ty * (k >> 3));
        size_t c = (size_t)t * 512 + (i & 7) + 8 * ((j & 7) + 8 * (k & 7));
        bool live = on[t] != 0;
        if (g->cnt) g->cnt[o] = live ? cnt[c] : 0;
        if (g->ctype) g->ctype[o] = live ? ct[c] : 0;
        if (g->pres) g->pres[o] = live ? pr[c] : 0.0f;
        if (g->rhs) g->rhs[o] = live ? rh[c] : 8.0f;
        for (int a = 0; a < 3; a++) {
          if (g->vn) g->vn[o * 3 + a] = live ? vn[a * C + c] : 0.0f;
          if (g->vo) g->vo[o * 3 + a] = live ? vo[a * C + c] : 0.0f;
          if (g->velg) g->velg[o * 3 + a] = live ? vg[a * C + c] : 0.0f;
        }
      }
  return ST_OK;
}

st_status st_flip_save_state(st_flip* s, float* pos4, float* vel4, uint32_t* pid, uint32_t cap, uint32_t* n) {
  if (!s) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  if (n) *n = s->N;
  uint32_t m = std::min(cap, s->N);
  if (m == 0) return ST_OK;
  std::vector<Part> host(m);
  CK(cudaMemcpyAsync(host.data(), s->part[s->cur], (size_t)m * sizeof(Part), cudaMemcpyDeviceToHost, s->stream));
  if (pid) CK(cudaMemcpyAsync(pid, s->ids[s->cur], (size_t)m * 4, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  for (uint32_t i = 0; i < m; i++) {
    if (pos4) memcpy(&pos4[i * 4], &host[i].p, 16);
    if (vel4) memcpy(&vel4[i * 4], &host[i].v, 16);
  }
  return ST_OK;
}

st_status st_flip_load_state(st_flip* s, const float* pos4, const float* vel4, const uint32_t* pid, uint32_t n, double t, uint32_t seed) {
  if (!s || n > s->maxN || (n && (!pos4 || !vel4 || !pid))) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  std::vector<Part> host(n);
  for (uint32_t i = 0; i < n; i++) { memcpy(&host[i].p, &pos4[i * 4], 16); memcpy(&host[i].v, &vel4[i * 4], 16); }
  if (n) {
    CK(cudaMemcpyAsync(s->part[s->cur], host.data(), (size_t)n * sizeof(Part), cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(s->ids[s->cur], pid, (size_t)n * 4, cudaMemcpyHostToDevice, s->stream));
  }
  CK(cudaStreamSynchronize(s->stream));
  s->N = n; s->ring = 0; s->tm = t; s->seed = seed;
  return ST_OK;
}

st_status st_flip_nb_fills(st_flip* s, const float* boxes6, uint32_t nbox, const float* sph4, uint32_t nsph, uint32_t mode) {
  if (!s || (nbox && !boxes6) || (nsph && !sph4)) return ST_BAD_ARG;
  if (mode != 2) s->fills.clear();   // water added to a running tank adds to the fills (src/shared.js:849)
  for (uint32_t k = 0; k < nbox; k++) {
    const float* b = &boxes6[k * 6];
    float f[8] = {1, b[0], b[1], b[2], b[3], b[4], b[5], 0};
    s->fills.insert(s->fills.end(), f, f + 8);
  }
  for (uint32_t k = 0; k < nsph; k++) {
    const float* q = &sph4[k * 4];
    float f[8] = {2, q[0], q[1], q[2], q[3], 0, 0, 0};
    s->fills.insert(s->fills.end(), f, f + 8);
  }
  s->nbInit = mode ? mode : 1;
  return ST_OK;
}


st_status st_flip_nb_fill_vols(st_flip* s, const st_collider* vols, uint32_t n, uint32_t mode) {
  if (!s || (n && !vols)) return ST_BAD_ARG;
  for (uint32_t k = 0; k < n; k++)
    if (!vols[k].sdf || !vols[k].sdf->data) return ST_BAD_ARG;
  if (mode != 2) s->fillVols.clear();
  for (uint32_t k = 0; k < n; k++) {
    st_flip::FillVol f;
    f.sd = *vols[k].sdf;
    f.data.assign(vols[k].sdf->data, vols[k].sdf->data + (size_t)f.sd.dims[0] * f.sd.dims[1] * f.sd.dims[2]);
    f.c = vols[k];
    for (int a = 0; a < 3; a++) { f.c.vel[a] = 0.0f; f.c.ang[a] = 0.0f; }
    s->fillVols.push_back(std::move(f));
  }
  s->nbInit = mode ? mode : 1;
  return ST_OK;
}

// ---- full checkpoint: every buffer a step reads before it writes, plus the host step state ----
// Layout: header, pending fills (floats), drip-grid signature (padded to 4 bytes), pending fill volumes (per volume 20
// words of record - id, dims, origin, cell, pos, R - then its grid), then the device buffers of full_parts in order.
struct FullHdr {
  uint32_t magic, version, nx, ny, nz, ntiles, ncell, maxN, sprayCap;
  uint32_t N, cap, ring, seed, steps, stamp, parity, cur, velGOn, nbInit, nfills, ndrip, nsig, airCells, nvols;
  uint64_t volWords;
  double tm;
};
static constexpr uint32_t FULL_MAGIC = 0x53544650u;   // "PFTS"
static constexpr uint32_t FULL_VERSION = 4;           // 4: air-field size and the pending fill volumes in the header
static constexpr uint32_t VOL_REC = 20;               // words of one fill volume's record
// the device parts of a checkpoint for N particles, the current buffer cur and ndrip drip samples
static void full_parts(st_flip* s, uint32_t N, int cur, uint32_t ndrip, std::vector<std::pair<void*, size_t>>& v) {
  const size_t C = s->ncell, T = s->ntiles, SC = std::max<size_t>(s->sprayCap, 1);
  v = {{s->dCtl, sizeof(Ctl)}, {s->part[cur], (size_t)N * sizeof(Part)}, {s->ids[cur], (size_t)N * 4}, {s->need, T * 4}, {s->on, T},
       {s->tstate, T}, {s->active, T * 4}, {s->cnt[0], C * 4}, {s->cnt[1], C * 4}, {s->ctype, C * 4}, {s->pres, C * 4},
       {s->rhs, C * 4}, {s->acc, 6 * C * 4}, {s->vn, 3 * C * 4}, {s->vo, 3 * C * 4}, {s->velG, 3 * C * 4}, {s->sorInfo, C * 2},
       {s->wet, C * 4}, {s->sPos, SC * 16}, {s->sVel, SC * 16}};
  if (s->airCells) v.push_back({s->air, (size_t)s->airCells * 16});
  if (ndrip) v.push_back({s->drip, (size_t)ndrip * 32});
}
static size_t pad4(size_t n) { return (n + 3) & ~(size_t)3; }
static uint64_t vol_words(const st_flip* s) {
  uint64_t w = 0;
  for (auto& f : s->fillVols) w += VOL_REC + f.data.size();
  return w;
}

st_status st_flip_save_full(st_flip* s, void* buf, uint64_t cap, uint64_t* size) {
  if (!s || !size) return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  std::vector<std::pair<void*, size_t>> parts;
  full_parts(s, s->N, s->cur, s->ndrip, parts);
  const uint64_t vw = vol_words(s);
  uint64_t need = sizeof(FullHdr) + s->fills.size() * sizeof(float) + pad4(s->dripSig.size()) + vw * 4;
  for (auto& p : parts) need += p.second;
  *size = need;
  if (!buf) return ST_OK;
  if (cap < need) return ST_OVERFLOW;
  FullHdr h{};
  h.magic = FULL_MAGIC; h.version = FULL_VERSION; h.nx = (uint32_t)s->nx; h.ny = (uint32_t)s->ny; h.nz = (uint32_t)s->nz; h.ntiles = s->ntiles;
  h.ncell = s->ncell; h.maxN = s->maxN; h.sprayCap = s->sprayCap; h.N = s->N; h.cap = s->cap; h.ring = s->ring; h.seed = s->seed;
  h.steps = s->steps; h.stamp = s->stamp; h.parity = s->parity; h.cur = (uint32_t)s->cur; h.velGOn = s->velGOn ? 1u : 0u;
  h.nbInit = s->nbInit; h.nfills = (uint32_t)s->fills.size(); h.tm = s->tm;
  h.ndrip = s->ndrip; h.nsig = (uint32_t)s->dripSig.size(); h.airCells = s->airCells;
  h.nvols = (uint32_t)s->fillVols.size(); h.volWords = vw;
  char* out = static_cast<char*>(buf);
  memcpy(out, &h, sizeof(h));
  out += sizeof(h);
  if (!s->fills.empty()) { memcpy(out, s->fills.data(), s->fills.size() * sizeof(float)); out += s->fills.size() * sizeof(float); }
  memset(out, 0, pad4(s->dripSig.size()));
  memcpy(out, s->dripSig.data(), s->dripSig.size());
  out += pad4(s->dripSig.size());
  for (auto& f : s->fillVols) {
    uint32_t rec[VOL_REC];
    rec[0] = f.sd.id; rec[1] = f.sd.dims[0]; rec[2] = f.sd.dims[1]; rec[3] = f.sd.dims[2];
    memcpy(&rec[4], f.sd.origin, 12); memcpy(&rec[7], &f.sd.cell, 4); memcpy(&rec[8], f.c.pos, 12); memcpy(&rec[11], f.c.R, 36);
    memcpy(out, rec, sizeof(rec));
    out += sizeof(rec);
    memcpy(out, f.data.data(), f.data.size() * 4);
    out += f.data.size() * 4;
  }
  for (auto& p : parts) {
    if (p.second) CK(cudaMemcpyAsync(out, p.first, p.second, cudaMemcpyDeviceToHost, s->stream));
    out += p.second;
  }
  CK(cudaStreamSynchronize(s->stream));
  return ST_OK;
}

// Every header field and every length is checked against this handle and the blob's size before anything of the
// handle changes, so a rejected blob leaves the tank as it was (and steppable).
st_status st_flip_load_full(st_flip* s, const void* buf, uint64_t size) {
  if (!s || !buf || size < sizeof(FullHdr)) return ST_BAD_ARG;
  FullHdr h;
  memcpy(&h, buf, sizeof(h));
  if (h.magic != FULL_MAGIC || h.version != FULL_VERSION || h.nx != (uint32_t)s->nx || h.ny != (uint32_t)s->ny || h.nz != (uint32_t)s->nz ||
      h.ntiles != s->ntiles || h.ncell != s->ncell || h.maxN != s->maxN || h.sprayCap != s->sprayCap || h.airCells != s->airCells) {
    snprintf(g_err, sizeof(g_err), "load_full: the checkpoint is not of a simulator with this geometry and capacity");
    return ST_BAD_ARG;
  }
  if (h.cap > s->maxN || h.N > h.cap || (h.cap ? h.ring >= h.cap : h.ring != 0) || h.cur > 1 || h.parity > 1 || h.nbInit > 2 ||
      h.nfills % 8 != 0 || h.nfills > (1u << 20) || h.nsig > (1u << 24) || h.ndrip > (1u << 26) || h.nvols > 4096) {
    snprintf(g_err, sizeof(g_err), "load_full: the checkpoint's counters are out of range (N %u, cap %u, ring %u)", h.N, h.cap, h.ring);
    return ST_BAD_ARG;
  }
  // the sizes of every part from the header alone
  const char* base = static_cast<const char*>(buf);
  uint64_t off = sizeof(FullHdr) + (uint64_t)h.nfills * sizeof(float) + pad4(h.nsig);
  if (off > size) goto short_blob;
  {
    // fill volumes: walk the records, checking each grid's length against what is left
    const uint64_t volStart = off;
    uint64_t words = 0;
    for (uint32_t k = 0; k < h.nvols; k++) {
      if (off + VOL_REC * 4 > size) goto short_blob;
      uint32_t rec[VOL_REC];
      memcpy(rec, base + off, sizeof(rec));
      const uint64_t n = (uint64_t)rec[1] * rec[2] * rec[3];
      if (!rec[1] || !rec[2] || !rec[3] || rec[1] > 4096 || rec[2] > 4096 || rec[3] > 4096 || off + VOL_REC * 4 + n * 4 > size) goto short_blob;
      off += VOL_REC * 4 + n * 4;
      words += VOL_REC + n;
    }
    if (words != h.volWords) goto short_blob;
    std::vector<std::pair<void*, size_t>> parts;
    full_parts(s, h.N, (int)h.cur, h.ndrip, parts);   // sizes only: the drip pointer may change below
    uint64_t need = off;
    for (auto& p : parts) need += p.second;
    if (size < need) {
      snprintf(g_err, sizeof(g_err), "load_full: %llu bytes given, %llu needed", (unsigned long long)size, (unsigned long long)need);
      return ST_BAD_ARG;
    }
    // everything checked: commit
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    if (h.ndrip > s->dripCap) {
      drop_graphs(s);
      float4* nd = nullptr;
      CK(dalloc(&nd, drip_words(h.ndrip)));
      if (s->drip) cudaFree(s->drip);
      s->drip = nd;
      s->dripCap = h.ndrip;
    }
    s->N = h.N; s->cap = h.cap; s->ring = h.ring; s->seed = h.seed; s->steps = h.steps; s->stamp = h.stamp; s->parity = h.parity;
    s->cur = (int)h.cur; s->velGOn = h.velGOn != 0; s->nbInit = h.nbInit; s->tm = h.tm;
    s->ndrip = h.ndrip;
    const char* in = base + sizeof(FullHdr);
    s->fills.assign(reinterpret_cast<const float*>(in), reinterpret_cast<const float*>(in) + h.nfills);
    in += (size_t)h.nfills * sizeof(float);
    s->dripSig.assign(in, h.nsig);
    in = base + volStart;
    s->fillVols.clear();
    for (uint32_t k = 0; k < h.nvols; k++) {
      uint32_t rec[VOL_REC];
      memcpy(rec, in, sizeof(rec));
      in += sizeof(rec);
      st_flip::FillVol f{};
      f.sd.id = rec[0]; f.sd.dims[0] = rec[1]; f.sd.dims[1] = rec[2]; f.sd.dims[2] = rec[3];
      memcpy(f.sd.origin, &rec[4], 12); memcpy(&f.sd.cell, &rec[7], 4); memcpy(f.c.pos, &rec[8], 12); memcpy(f.c.R, &rec[11], 36);
      const size_t n = (size_t)rec[1] * rec[2] * rec[3];
      f.data.assign(reinterpret_cast<const float*>(in), reinterpret_cast<const float*>(in) + n);
      in += n * 4;
      s->fillVols.push_back(std::move(f));
    }
    full_parts(s, s->N, s->cur, s->ndrip, parts);
    for (auto& p : parts) {
      if (p.second) CK(cudaMemcpyAsync(p.first, in, p.second, cudaMemcpyHostToDevice, s->stream));
      in += p.second;
    }
    // the dynamic-tile counters are 0 between launches; a checkpoint cannot change that
    CK(cudaMemsetAsync(&s->dCtl->tileNext, 0, 2 * sizeof(uint32_t), s->stream));
    CK(cudaStreamSynchronize(s->stream));
    drop_graphs(s);
    s->sdfSig.clear();   // the next step uploads its colliders' distance grids again
    return ST_OK;
  }
short_blob:
  snprintf(g_err, sizeof(g_err), "load_full: the checkpoint is truncated or its fill volumes are malformed");
  return ST_BAD_ARG;
}

st_status st_flip_set_launch(st_flip* s, int32_t tile_ctas_per_sm, int32_t light_ctas_per_sm, int32_t sor_ctas_per_sm) {
  if (!s || tile_ctas_per_sm < 1 || light_ctas_per_sm < 1 || sor_ctas_per_sm < 1 || tile_ctas_per_sm > 64 ||
      light_ctas_per_sm > 64 || sor_ctas_per_sm > 64)
    return ST_BAD_ARG;
  CK(cudaSetDevice(s->device));
  if (s->gridT == tile_ctas_per_sm && s->gridT4 == light_ctas_per_sm && s->gridSor == sor_ctas_per_sm) return ST_OK;
  CK(cudaStreamSynchronize(s->stream));
  drop_graphs(s);
  s->gridT = tile_ctas_per_sm; s->gridT4 = light_ctas_per_sm; s->gridSor = sor_ctas_per_sm;
  return ST_OK;
}

}  // extern "C"

// ---- many tanks per step (st_batch_*) ----
// Each tank keeps its own buffers and its captured step graph. A batch step does the host half of every tank's step
// (uploads on the batch stream), then runs the tanks' step graphs either as the parallel branches of one CUDA graph
// (ST_BATCH_GRAPH: one launch; independent tanks run concurrently and fill the GPU together) or one after another on
// the batch stream (ST_BATCH_SEQUENTIAL). Both orders give every tank the same result as st_flip_step.
struct st_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  int mode = ST_BATCH_GRAPH;
  std::vector<st_flip*> tanks;
  std::vector<cudaEvent_t> tankEv;
  cudaEvent_t evOut = nullptr;
  struct Combined {
    std::vector<uint64_t> key;   // per tank: step graph key and generation
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
  };
  std::vector<Combined> cache;
  uint64_t launches = 0, graph_launches = 0;
  // pooled modes: one compact copy of every tank's fluid tiles, swept by one launch per colour (ST_BATCH_POOLED) or
  // by one persistent cooperative launch (ST_BATCH_PERSISTENT)
  PoolBufs pool{};
  const Ctl** dCtls = nullptr;     // device: each tank's counters
  unsigned int* hErr = nullptr;    // pinned: the persistent sweep's error word after its launch
  bool errPending = false;
  int poolGrid = 8;                // CTAs per SM of the pooled sweeps
  uint64_t limitNs = 1000000000ull;
  struct Pooled {
    std::vector<uint64_t> key;
    cudaGraph_t g[2] = {nullptr, nullptr};
    cudaGraphExec_t x[2] = {nullptr, nullptr};
    int launches = 0;
  };
  std::vector<Pooled> pcache;
};

static void batch_drop(st_batch* b) {
  for (auto& c : b->cache) {
    if (c.exec) cudaGraphExecDestroy(c.exec);
    if (c.graph) cudaGraphDestroy(c.graph);
  }
  b->cache.clear();
  for (auto& c : b->pcache)
    for (int k = 0; k < 2; k++) {
      if (c.x[k]) cudaGraphExecDestroy(c.x[k]);
      if (c.g[k]) cudaGraphDestroy(c.g[k]);
    }
  b->pcache.clear();
}
static void pool_free(st_batch* b) {
  void* ps[] = {b->pool.cp, b->pool.crhs, b->pool.cinfo, b->pool.nbs, b->pool.pomega, b->pool.off, b->pool.total, b->pool.bar, b->pool.err,
                (void*)b->dCtls};
  for (void* p : ps)
    if (p) cudaFree(p);
  b->pool = PoolBufs{};
  b->dCtls = nullptr;
}
// the pool holds every tile of every tank (an upper bound on their fluid tiles)
static cudaError_t pool_alloc(st_batch* b) {
  size_t T = 0;
  for (auto* s : b->tanks) T += s->ntiles;
  cudaError_t e = cudaSuccess;
  auto A = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
  A(dalloc(&b->pool.cp, T * 512)); A(dalloc(&b->pool.crhs, T * 512)); A(dalloc(&b->pool.cinfo, T * 512)); A(dalloc(&b->pool.nbs, T * 6));
  A(dalloc(&b->pool.pomega, T)); A(dalloc(&b->pool.off, b->tanks.size())); A(dalloc(&b->pool.total, 1)); A(dalloc(&b->pool.bar, 1));
  A(dalloc(&b->pool.err, 1)); A(dalloc(&b->dCtls, b->tanks.size()));
  if (e == cudaSuccess) {
    std::vector<const Ctl*> h(b->tanks.size());
    for (size_t i = 0; i < h.size(); i++) h[i] = b->tanks[i]->dCtl;
    e = cudaMemcpy((void*)b->dCtls, h.data(), h.size() * sizeof(Ctl*), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaMemset(b->pool.err, 0, 4);
  return e;
}
// a tank's buffers with its compact copy in the pool, at the offset the plan kernel writes
static Bufs pooled_bufs(const st_batch* b, size_t i) {
  Bufs B = b->tanks[i]->bufs();
  B.cp = b->pool.cp; B.crhs = b->pool.crhs; B.cinfo = b->pool.cinfo; B.nbs = b->pool.nbs; B.pomega = b->pool.pomega;
  B.poolOff = b->pool.off + i;
  return B;
}

// One pooled batch step after every tank's host half: a graph of parallel per-tank branches up to the pressure
// sweeps, the plan of pool offsets, every tank's copy into the pool (parallel), then the sweeps over the whole pool, then
// parallel per-tank branches unpacking and finishing the step. ST_BATCH_POOLED captures the sweeps into the graph as
// chained launches; ST_BATCH_PERSISTENT runs them as one cooperative launch between two graphs (its grid barrier waits
// are bounded; a wait that ran out is reported as ST_TIMEOUT by the next batch call).
static st_status batch_pooled(st_batch* b, const std::vector<StepPrep>& prs) {
  const size_t n = b->tanks.size();
  cudaStream_t q = b->stream;
  const bool persist = b->mode == ST_BATCH_PERSISTENT;
  int sms = b->tanks[0]->sms;
  const int iters = prs[0].iters;
  int grid = sms * b->poolGrid;
  if (persist) grid = sms * std::max(1, std::min(b->poolGrid, persistent_ctas_per_sm()));
  std::vector<uint64_t> key;
  for (size_t i = 0; i < n; i++) {
    st_flip* s = b->tanks[i];
    key.push_back(graph_key(s, prs[i].nbOn, prs[i].sprOn, prs[i].iters, prs[i].pbfIters, false));
    key.push_back(s->gen);
  }
  key.push_back((uint64_t)b->mode | ((uint64_t)grid << 8));
  st_batch::Pooled* c = nullptr;
  for (auto& x : b->pcache) if (x.key == key) c = &x;
  if (!c) {
    if (b->pcache.size() >= 4) {
      auto& f = b->pcache.front();
      for (int k = 0; k < 2; k++) { if (f.x[k]) cudaGraphExecDestroy(f.x[k]); if (f.g[k]) cudaGraphDestroy(f.g[k]); }
      b->pcache.erase(b->pcache.begin());
    }
    st_batch::Pooled nc;
    nc.key = key;
    int nl = 0;
    auto fork = [&](auto&& body) -> cudaError_t {   // body(i, stream) on every tank's stream, joined back into q
      cudaError_t e = cudaEventRecord(b->evOut, q);
      for (size_t i = 0; i < n && e == cudaSuccess; i++) {
        st_flip* s = b->tanks[i];
        e = cudaStreamWaitEvent(s->stream, b->evOut, 0);
        if (e == cudaSuccess) nl += body(i, s->stream);
        if (e == cudaSuccess) e = cudaEventRecord(b->tankEv[i], s->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(q, b->tankEv[i], 0);
      }
      return e;
    };
    auto sweeps = [&]() { nl += launch_pool_sweeps(b->pool, grid, iters, q); };
    for (int part = 0; part < (persist ? 2 : 1); part++) {
      cudaError_t e = cudaStreamBeginCapture(q, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess && part == 0) {
        e = fork([&](size_t i, cudaStream_t sq) {
          st_flip* s = b->tanks[i];
          return enqueue_front(s, pooled_bufs(b, i), sq, prs[i].nbOn, 0u, [](int) {});
        });
        if (e == cudaSuccess) nl += launch_pool_plan(b->pool, b->dCtls, (uint32_t)n, q);
        if (e == cudaSuccess)
          e = fork([&](size_t i, cudaStream_t sq) { return launch_sor_pack(pooled_bufs(b, i), b->tanks[i]->tileGrid(b->tanks[i]->gridT4), sq); });
        if (e == cudaSuccess && !persist) sweeps();
      }
      if (e == cudaSuccess && (part == 1 || !persist)) {
        e = fork([&](size_t i, cudaStream_t sq) {
          st_flip* s = b->tanks[i];
          const Bufs B = pooled_bufs(b, i);
          return launch_sor_unpack(B, s->tileGrid(s->gridT4), sq) + enqueue_back(s, B, sq, prs[i].nbOn, prs[i].sprOn, prs[i].pbfIters, [](int) {});
        });
      }
      cudaGraph_t g = nullptr;
      const cudaError_t e2 = cudaStreamEndCapture(q, &g);
      if (e == cudaSuccess) e = e2;
      if (e == cudaSuccess) e = cudaGraphInstantiate(&nc.x[part], g, 0);
      nc.g[part] = g;
      if (e != cudaSuccess) {
        set_err("pooled batch graph", e);
        for (int k = 0; k < 2; k++) { if (nc.x[k]) cudaGraphExecDestroy(nc.x[k]); if (nc.g[k]) cudaGraphDestroy(nc.g[k]); }
        return ST_DEVICE_ERROR;
      }
    }
    nc.launches = nl + (persist ? 1 : 0);
    b->pcache.push_back(nc);
    c = &b->pcache.back();
  }
  CK(cudaGraphLaunch(c->x[0], q));
  b->graph_launches++;
  if (persist) {
    CK(launch_pool_persistent(b->pool, grid, iters, b->limitNs, q));
    CK(cudaMemcpyAsync(b->hErr, b->pool.err, 4, cudaMemcpyDeviceToHost, q));
    b->errPending = true;
    CK(cudaGraphLaunch(c->x[1], q));
    b->graph_launches++;
  }
  for (size_t i = 0; i < n; i++) {
    b->tanks[i]->launches += (uint64_t)(c->launches / std::max<size_t>(n, 1));
    b->tanks[i]->steps++;
  }
  b->launches += (uint64_t)c->launches;
  CK(cudaGetLastError());
  CK(cudaEventRecord(b->evOut, q));
  for (size_t i = 0; i < n; i++) CK(cudaStreamWaitEvent(b->tanks[i]->stream, b->evOut, 0));
  return ST_OK;
}

extern "C" {

void st_batch_destroy(st_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_drop(b);
  pool_free(b);
  if (b->hErr) cudaFreeHost(b->hErr);
  for (auto e : b->tankEv) if (e) cudaEventDestroy(e);
  if (b->evOut) cudaEventDestroy(b->evOut);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

st_status st_batch_create(const st_batch_desc* d, st_flip* const* tanks, uint32_t n, st_batch** out) {
  if (!d || !out || d->size != sizeof(st_batch_desc) || !tanks || !n || d->mode < ST_BATCH_GRAPH || d->mode > ST_BATCH_PERSISTENT)
    return ST_BAD_ARG;
  *out = nullptr;
  for (uint32_t i = 0; i < n; i++)
    if (!tanks[i] || tanks[i]->device != tanks[0]->device) return ST_BAD_ARG;
  st_batch* b = new st_batch();
  b->device = tanks[0]->device;
  b->mode = d->mode;
  b->tanks.assign(tanks, tanks + n);
  b->tankEv.assign(n, nullptr);
  cudaError_t e = cudaSetDevice(b->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->evOut, cudaEventDisableTiming);
  for (uint32_t i = 0; i < n && e == cudaSuccess; i++) e = cudaEventCreateWithFlags(&b->tankEv[i], cudaEventDisableTiming);
  if (e == cudaSuccess) e = pool_alloc(b);
  if (e == cudaSuccess) e = cudaMallocHost((void**)&b->hErr, 4);
  if (e == cudaSuccess) *b->hErr = 0u;
  if (e != cudaSuccess) {
    set_err("batch create", e);
    st_batch_destroy(b);
    return ST_DEVICE_ERROR;
  }
  *out = b;
  return ST_OK;
}

st_status st_batch_set_mode(st_batch* b, int32_t mode) {
  if (!b || mode < ST_BATCH_GRAPH || mode > ST_BATCH_PERSISTENT) return ST_BAD_ARG;
  b->mode = mode;
  return ST_OK;
}

st_status st_batch_set_sweeps(st_batch* b, int32_t ctas_per_sm, uint32_t wait_limit_us) {
  if (!b || ctas_per_sm < 1 || ctas_per_sm > 64 || wait_limit_us == 0) return ST_BAD_ARG;
  if (b->poolGrid != ctas_per_sm) {
    CK(cudaSetDevice(b->device));
    CK(cudaStreamSynchronize(b->stream));
    batch_drop(b);
  }
  b->poolGrid = ctas_per_sm;
  b->limitNs = (uint64_t)wait_limit_us * 1000ull;
  return ST_OK;
}

// The bounded grid barrier of the persistent sweep, run on its own with more arrivals expected than the launch has
// (missing > 0): every CTA's wait must run out within about limit_us and report it. *timed_out = 1 when it did.
st_status st_batch_barrier_test(int32_t device, uint32_t missing, uint32_t limit_us, uint32_t* timed_out) {
  if (!timed_out || limit_us == 0 || limit_us > 10000000u) return ST_BAD_ARG;
  CK(cudaSetDevice(device));
  int sms = 148;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  unsigned int* w = nullptr;
  CK(cudaMalloc((void**)&w, 8));
  cudaError_t e = cudaMemset(w, 0, 8);
  const int grid = sms;   // one CTA per SM: all resident
  if (e == cudaSuccess) e = launch_barrier_test(w, w + 1, grid, (unsigned int)grid + missing, (uint64_t)limit_us * 1000ull, 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  unsigned int h[2] = {0, 0};
  if (e == cudaSuccess) e = cudaMemcpy(h, w, 8, cudaMemcpyDeviceToHost);
  cudaFree(w);
  CK(e);
  *timed_out = h[1] != 0u ? 1u : 0u;
  return ST_OK;
}

void* st_batch_stream(st_batch* b) { return b ? (void*)b->stream : nullptr; }

uint64_t st_batch_launches(st_batch* b) { return b ? b->launches : 0; }

st_status st_batch_step(st_batch* b, double dt, const st_step_opts* const* opts) {
  if (!b || !opts) return ST_BAD_ARG;
  const size_t n = b->tanks.size();
  for (size_t i = 0; i < n; i++)
    if (!opts[i] || opts[i]->size != sizeof(st_step_opts)) return ST_BAD_ARG;
  CK(cudaSetDevice(b->device));
  cudaStream_t q = b->stream;
  // after whatever each tank's own stream still has queued (adds, reads)
  for (size_t i = 0; i < n; i++) {
    CK(cudaEventRecord(b->tankEv[i], b->tanks[i]->stream));
    CK(cudaStreamWaitEvent(q, b->tankEv[i], 0));
  }
  if (b->errPending) {   // the last persistent sweep's error word has landed by now (this call waited above)
    CK(cudaStreamSynchronize(q));
    b->errPending = false;
    if (*b->hErr) {
      *b->hErr = 0u;
      CK(cudaMemsetAsync(b->pool.err, 0, 4, q));
      snprintf(g_err, sizeof(g_err), "batch: a grid barrier of the persistent pressure sweeps ran out of time");
      return ST_TIMEOUT;
    }
  }
  std::vector<StepPrep> prs(n);
  bool pooled = b->mode == ST_BATCH_POOLED || b->mode == ST_BATCH_PERSISTENT;
  if (pooled) {
    // every tank's host half first; a tank that restarts this step (or cannot use graphs) sends the step down the
    // branch path below, as do differing iteration counts
    for (size_t i = 0; i < n; i++) {
      st_flip* s = b->tanks[i];
      if (s->N == 0) { pooled = false; continue; }
      st_status st = prepare_step(s, dt, opts[i], q, &prs[i]);
      if (st != ST_OK) return st;
      if (prs[i].init || !s->use_graphs || prs[i].iters != prs[0].iters) pooled = false;
    }
    if (pooled) return batch_pooled(b, prs);
  }
  std::vector<cudaGraph_t> kids;
  std::vector<uint64_t> key;
  const bool prepared = b->mode == ST_BATCH_POOLED || b->mode == ST_BATCH_PERSISTENT;
  for (size_t i = 0; i < n; i++) {
    st_flip* s = b->tanks[i];
    if (s->N == 0) continue;
    StepPrep pr = prs[i];
    st_status st = prepared ? ST_OK : prepare_step(s, dt, opts[i], q, &pr);
    if (st != ST_OK) return st;
    const Bufs B = s->bufs();
    int nl = 0;
    if (pr.init || !s->use_graphs) {
      nl = enqueue_step(s, B, q, pr.nbOn, pr.init, pr.sprOn, pr.iters, pr.pbfIters, [](int) {});
    } else {
      st_flip::Graph* g = nullptr;
      st = get_graph(s, B, pr.nbOn, pr.sprOn, pr.iters, pr.pbfIters, false, &g);
      if (st != ST_OK) return st;
      nl = g->launches;
      if (b->mode == ST_BATCH_SEQUENTIAL) {
        CK(cudaGraphLaunch(g->exec, q));
        b->graph_launches++;
      } else {
        kids.push_back(g->graph);
        key.push_back(g->key);
        key.push_back(s->gen);
        key.push_back((uint64_t)i);
      }
    }
    s->launches += (uint64_t)nl;
    b->launches += (uint64_t)nl;
    s->steps++;
  }
  if (!kids.empty()) {
    st_batch::Combined* c = nullptr;
    for (auto& x : b->cache) if (x.key == key) c = &x;
    if (!c) {
      if (b->cache.size() >= 4) {
        if (b->cache.front().exec) cudaGraphExecDestroy(b->cache.front().exec);
        if (b->cache.front().graph) cudaGraphDestroy(b->cache.front().graph);
        b->cache.erase(b->cache.begin());
      }
      st_batch::Combined nc;
      nc.key = key;
      cudaError_t e = cudaGraphCreate(&nc.graph, 0);
      for (size_t k = 0; k < kids.size() && e == cudaSuccess; k++) {
        cudaGraphNode_t node;
        e = cudaGraphAddChildGraphNode(&node, nc.graph, nullptr, 0, kids[k]);
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&nc.exec, nc.graph, 0);
      if (e != cudaSuccess) {
        set_err("batch graph", e);
        if (nc.exec) cudaGraphExecDestroy(nc.exec);
        if (nc.graph) cudaGraphDestroy(nc.graph);
        return ST_DEVICE_ERROR;
      }
      b->cache.push_back(nc);
      c = &b->cache.back();
    }
    CK(cudaGraphLaunch(c->exec, q));
    b->graph_launches++;
  }
  CK(cudaGetLastError());
  // each tank's later work (reads, the next single step) waits for this batch step
  CK(cudaEventRecord(b->evOut, q));
  for (size_t i = 0; i < n; i++) CK(cudaStreamWaitEvent(b->tanks[i]->stream, b->evOut, 0));
  return ST_OK;
}

}  // extern "C"
