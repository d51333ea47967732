// C ABI of the B200 pressure projection (declared in include/shkz_b200.h).
//
// One context owns one CUDA stream and every device buffer; nothing is
// allocated per iteration. A projection runs:
//   label unknowns -> build the 8^3 tile pool -> weights/rhs -> MIC(0) factor
//   -> FP32 PCG with FP64 reductions inside an FP64 refinement loop
//   -> pressure scatter and velocity update.
// The PCG runs in batches of `check_interval` iterations; each kernel reads
// the device-side solver state and returns at once after convergence, so the
// host only synchronises once per batch.
#include "common.cuh"
#include "kernels.h"
#include "solver.h"
#include "learned.h"
#include "csr_mic0.h"
#include "../../include/shkz_b200.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

using namespace shkz;

static thread_local char g_last_error[512] = {0};

void shkz_set_cuda_error(cudaError_t e, const char *expr, const char *file, int line) {
  std::snprintf(g_last_error, sizeof(g_last_error), "%s (%d) at %s:%d: %s", cudaGetErrorString(e), (int)e, file, line,
                expr);
}

struct shkz_b200_ctx {
  shkz_b200_config cfg;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[12] = {};
  // dense capacities
  size_t cap_cells = 0;
  size_t cap_h_cells = 0, cap_h_nodes = 0, cap_h_faces[3] = {0, 0, 0};
  long long cap_tiles = 0;
  int cap_pool = 0;
  // dense staging buffers for the host path
  float *h_fluid = nullptr, *h_solid = nullptr, *h_vel[3] = {}, *h_svel[3] = {}, *h_pressure = nullptr;
  uint8_t *h_fluid_active = nullptr, *h_solid_active = nullptr, *h_vact[3] = {}, *h_pact = nullptr;
  // assembly
  int *flags = nullptr;
  uint8_t *unk = nullptr;
  int *tile_count = nullptr, *tile_state = nullptr, *pool_tile = nullptr, *nbr = nullptr, *level_count = nullptr,
      *sched = nullptr, *bsum = nullptr, *total = nullptr;
  // pool arrays
  float *diag = nullptr, *offx = nullptr, *offy = nullptr, *offz = nullptr, *d32 = nullptr;
  float *upx = nullptr, *upy = nullptr, *upz = nullptr;  // upper weights of the backward sweep
  double *diag64 = nullptr, *offx64 = nullptr, *offy64 = nullptr, *offz64 = nullptr, *rhs64 = nullptr,
         *colsum = nullptr, *dmic64 = nullptr, *x64 = nullptr, *r64 = nullptr, *xref64 = nullptr,
         *p64 = nullptr, *q64 = nullptr, *z64 = nullptr;
  float *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *z = nullptr, *t = nullptr, *p32 = nullptr;
  float *pb = nullptr;  // second direction buffer: the fused stencil writes the new p beside the old one
  // reductions and wavefront sync
  double *partials = nullptr, *out4 = nullptr;
  unsigned *counter = nullptr;
  SolverState *st = nullptr;
  int *wflags = nullptr;  // factor wavefront flags [cap_pool]
  unsigned long long *faces_f = nullptr, *faces_b = nullptr;  // [cap_pool][3][64] epoch-tagged sweep faces
  // 16^3 macro tiles of the MIC(0) sweeps
  int KM = 0, cap_macro = 0;
  int *mcount = nullptr, *mstate = nullptr, *mtile = nullptr, *mnbr = nullptr, *msched = nullptr, *msub = nullptr;
  unsigned long long *mfaces_f = nullptr, *mfaces_b = nullptr;  // [cap_macro][3][256]
  void *ws = nullptr;     // 3 WaveSync
  // last projection
  Geometry G{};
  int K = 0;
  long long unknowns = 0;
  int has_system = 0;
  int mic_ready = 0;  // d32 holds the MIC(0) factor of the current system
  LearnedModel *model = nullptr;
  int model_ready = 0;  // block activity computed for the current system
  AssemblyInputs last_in{};
  SolverState *st_scratch = nullptr;
  // optional terms: surface tension curvature, volume correction, warm start
  float *curv = nullptr;
  size_t cap_curv = 0;
  double vol_target = 0.0, vol_current = 0.0, vol_yprev = 0.0;
  double *prev = nullptr;          // warm-start vector by reference unknown number
  long long prev_n = 0, cap_prev = 0;
  int *rank_pool = nullptr, *rank_cnt = nullptr;
  long long *rank_total = nullptr;
  double *xw = nullptr;            // warm-start x0 over the pool
  int cap_warm_pool = 0;
  size_t cap_rank_cnt = 0;
  float *h_dens[3] = {};           // staging of the solid density faces (host path)
  float *ext_v[3] = {};            // velocity extension: side buffer of new values per component
  uint8_t *ext_a[3] = {};          // and its flags
  size_t cap_ext[3] = {0, 0, 0};
  int *ext_flag = nullptr;         // levelset_exist(solid) of the extension's constraint
  // FLIP splat (splat.cu)
  unsigned char *sp_raw = nullptr;  // particle records (host path)
  size_t cap_sp_raw = 0;
  float4 *sp_posm = nullptr, *sp_vc[3] = {};
  int *sp_key = nullptr, *sp_rank = nullptr, *sp_list = nullptr;
  float4 *sp_sposm = nullptr, *sp_svc = nullptr;
  long long cap_sp_particles = 0;
  int *sp_faces = nullptr, *sp_sorted = nullptr, *sp_face_bin = nullptr, *sp_nfaces = nullptr, *sp_work = nullptr;
  long long cap_sp_list = 0;
  int *sp_count = nullptr, *sp_tile_start = nullptr, *sp_tiles = nullptr;
  uint8_t *sp_tile_act = nullptr;
  long long cap_sp_tiles = 0;
  bool sp_dirty = false;  // bucket counters may be nonzero: a call stopped before clearing them
  uint8_t *sp_act[3] = {};
  size_t cap_sp_faces[3] = {0, 0, 0};
  float *sp_mass[3] = {}, *sp_mom[3] = {};  // optional outputs (host path)
  uint8_t *sp_sact[3] = {};
  size_t cap_sp_out[3] = {0, 0, 0};
  void *flush = nullptr;           // 256 MB written between timed kernel launches (> L2)
  size_t cap_h_dens[3] = {0, 0, 0};
  std::unordered_map<void *, size_t> held;  // buffers allocated by grow() and their bytes
  size_t held_bytes = 0;
};

extern "C" void shkz_b200_default_config(shkz_b200_config *c) {
  std::memset(c, 0, sizeof(*c));
  c->residual = 1e-4;
  c->max_iterations = 30000;
  c->preconditioner = SHKZ_B200_PRECOND_MIC0;
  c->mic_omega = 0.97;
  c->mic_min_diag_ratio = 0.25;
  c->eps_fluid = 1e-2;
  c->eps_solid = 1e-2;
  c->second_order_fluid = 1;
  c->second_order_solid = 1;
  c->refine = 1;
  c->fp64_reference = 0;
  c->fp64_tol = 1e-12;
  c->check_interval = 16;
  c->stall_window = 8;
  c->device = 0;
  c->mic_block = 16;
  c->gain = 1.0;
  c->warm_start = 0;
  c->index_tile = 16;
}

extern "C" const char *shkz_b200_errstr(int code) {
  switch (code) {
    case SHKZ_B200_OK: return "ok";
    case SHKZ_B200_ERR_ARG: return "invalid argument";
    case SHKZ_B200_ERR_CUDA: return "CUDA runtime error";
    case SHKZ_B200_ERR_NOMEM: return "device allocation failed";
    case SHKZ_B200_ERR_TIMEOUT: return "a bounded device wait gave up";
    case SHKZ_B200_ERR_NAN: return "NaN in the system or the iterates";
    case SHKZ_B200_ERR_NODEVICE: return "no usable sm_100 device";
    case SHKZ_B200_ERR_STATE: return "invalid call order";
    case SHKZ_B200_ERR_LIMIT: return "size beyond a documented limit";
    default: return "unknown error";
  }
}

extern "C" const char *shkz_b200_last_error(shkz_b200_ctx *) { return g_last_error; }

extern "C" void *shkz_b200_host_alloc(size_t bytes) {
  void *p = nullptr;
  if (!bytes) return nullptr;
  const cudaError_t e = cudaMallocHost(&p, bytes);
  if (e != cudaSuccess) {
    shkz_set_cuda_error(e, "cudaMallocHost", __FILE__, __LINE__);
    return nullptr;
  }
  return p;
}

extern "C" void shkz_b200_host_free(void *p) {
  if (p) cudaFreeHost(p);
}

// Grid and tile-pool buffers of the context: freed and reallocated when a
// call needs more. Their bytes are counted against cfg.device_mem_limit_mb
// (when set), which refuses an allocation with SHKZ_B200_ERR_NOMEM before
// cudaMalloc is asked.
static void release(shkz_b200_ctx *ctx, void *p) {
  if (!p) return;
  auto it = ctx->held.find(p);
  if (it != ctx->held.end()) {
    ctx->held_bytes -= it->second;
    ctx->held.erase(it);
  }
  cudaFree(p);
}

template <class T>
static int grow(shkz_b200_ctx *ctx, T **ptr, size_t need, const char *what) {
  release(ctx, *ptr);
  *ptr = nullptr;
  if (need == 0) return 0;
  const size_t bytes = need * sizeof(T);
  const size_t cap = (size_t)(ctx->cfg.device_mem_limit_mb > 0 ? ctx->cfg.device_mem_limit_mb : 0) << 20;
  if (cap && ctx->held_bytes + bytes > cap) {
    std::snprintf(g_last_error, sizeof(g_last_error),
                  "device memory cap of %d MiB reached: %zu bytes held, %zu more requested for %s",
                  ctx->cfg.device_mem_limit_mb, ctx->held_bytes, bytes, what);
    return SHKZ_B200_ERR_NOMEM;
  }
  cudaError_t e = cudaMalloc((void **)ptr, bytes);
  if (e != cudaSuccess) {
    shkz_set_cuda_error(e, "cudaMalloc", __FILE__, __LINE__);
    *ptr = nullptr;
    return SHKZ_B200_ERR_NOMEM;
  }
  ctx->held[*ptr] = bytes;
  ctx->held_bytes += bytes;
  return 0;
}

#define GROW(field, n)                                    \
  do {                                                    \
    int _rc = grow(ctx, &ctx->field, (size_t)(n), #field); \
    if (_rc) return _rc;                                  \
  } while (0)

static Geometry make_geometry(int nx, int ny, int nz) {
  Geometry G;
  G.nx = nx;
  G.ny = ny;
  G.nz = nz;
  G.bx = (nx + SHKZ_T - 1) / SHKZ_T;
  G.by = (ny + SHKZ_T - 1) / SHKZ_T;
  G.bz = (nz + SHKZ_T - 1) / SHKZ_T;
  G.ntiles = (long long)G.bx * G.by * G.bz;
  return G;
}

static int ensure_grid(shkz_b200_ctx *ctx, const Geometry &G) {
  const size_t cells = (size_t)G.nx * G.ny * G.nz;
  if (cells > ctx->cap_cells) {
    GROW(unk, cells);
    ctx->cap_cells = cells;
  }
  if (G.ntiles > ctx->cap_tiles) {
    GROW(tile_count, G.ntiles);
    GROW(tile_state, G.ntiles);
    GROW(bsum, (G.ntiles + 1023) / 1024 + 1);
    GROW(mcount, G.ntiles);
    GROW(mstate, G.ntiles);
    ctx->cap_tiles = G.ntiles;
  }
  if (!ctx->level_count) {
    // levels bx+by+bz <= 3 * 65536 / 8 for any grid this ABI accepts
    GROW(level_count, 3 * 8192 + 8);
  }
  return 0;
}

static int ensure_host_staging(shkz_b200_ctx *ctx, const Geometry &G, bool solid, const bool svel[3]) {
  const size_t cells = (size_t)G.nx * G.ny * G.nz;
  const size_t nodes = (size_t)(G.nx + 1) * (G.ny + 1) * (G.nz + 1);
  if (cells > ctx->cap_h_cells) {
    GROW(h_fluid, cells);
    GROW(h_fluid_active, cells);
    GROW(h_pressure, cells);
    GROW(h_pact, cells);
    ctx->cap_h_cells = cells;
  }
  if (solid && nodes > ctx->cap_h_nodes) {
    GROW(h_solid, nodes);
    GROW(h_solid_active, nodes);
    ctx->cap_h_nodes = nodes;
  }
  for (int d = 0; d < 3; ++d) {
    const size_t nf = (size_t)(G.nx + (d == 0)) * (G.ny + (d == 1)) * (G.nz + (d == 2));
    if (nf > ctx->cap_h_faces[d]) {
      GROW(h_vel[d], nf);
      GROW(h_vact[d], nf);
      if (ctx->h_svel[d]) { release(ctx, ctx->h_svel[d]); ctx->h_svel[d] = nullptr; }
      ctx->cap_h_faces[d] = nf;
    }
    if (svel[d] && !ctx->h_svel[d]) GROW(h_svel[d], ctx->cap_h_faces[d]);
  }
  return 0;
}

static int ensure_pool(shkz_b200_ctx *ctx, int K) {
  if (K <= ctx->cap_pool) return 0;
  int cap = K + K / 4 + 16;
  const size_t n = (size_t)cap * SHKZ_TC;
  GROW(pool_tile, cap);
  GROW(nbr, (size_t)cap * 6);
  GROW(sched, cap);
  GROW(diag, n); GROW(offx, n); GROW(offy, n); GROW(offz, n); GROW(d32, n);
  GROW(diag64, n); GROW(offx64, n); GROW(offy64, n); GROW(offz64, n); GROW(rhs64, n);
  GROW(colsum, n); GROW(dmic64, n); GROW(x64, n); GROW(r64, n); GROW(xref64, n);
  GROW(p64, n); GROW(q64, n); GROW(z64, n);
  GROW(x, n); GROW(r, n); GROW(p, n); GROW(q, n); GROW(z, n); GROW(t, n); GROW(p32, n); GROW(pb, n);
  GROW(upx, n); GROW(upy, n); GROW(upz, n);
  GROW(partials, (size_t)2 * cap + 4 * 8192);
  GROW(wflags, (size_t)cap);
  GROW(faces_f, (size_t)cap * 3 * 64);
  GROW(faces_b, (size_t)cap * 3 * 64);
  SHKZ_CUDA_TRY(cudaMemsetAsync(ctx->wflags, 0, sizeof(int) * (size_t)cap, ctx->stream));
  SHKZ_CUDA_TRY(cudaMemsetAsync(ctx->faces_f, 0, sizeof(unsigned long long) * (size_t)cap * 3 * 64, ctx->stream));
  SHKZ_CUDA_TRY(cudaMemsetAsync(ctx->faces_b, 0, sizeof(unsigned long long) * (size_t)cap * 3 * 64, ctx->stream));
  if (ctx->ws) {
    // flags were reset: restart the epochs (macro faces too, so no stale tag matches)
    SHKZ_CUDA_TRY(cudaMemsetAsync(ctx->ws, 0, 3 * wave_sync_bytes(), ctx->stream));
    if (ctx->mfaces_f) {
      SHKZ_CUDA_TRY(cudaMemsetAsync(ctx->mfaces_f, 0, sizeof(unsigned long long) * (size_t)ctx->cap_macro * 768,
                                    ctx->stream));
      SHKZ_CUDA_TRY(cudaMemsetAsync(ctx->mfaces_b, 0, sizeof(unsigned long long) * (size_t)ctx->cap_macro * 768,
                                    ctx->stream));
    }
  }
  ctx->cap_pool = cap;
  return 0;
}

static int ensure_macro(shkz_b200_ctx *ctx, int KM) {
  if (KM <= ctx->cap_macro) return 0;
  const int cap = KM + KM / 4 + 16;
  GROW(mtile, cap);
  GROW(mnbr, (size_t)cap * 6);
  GROW(msched, cap);
  GROW(msub, (size_t)cap * 8);
  GROW(mfaces_f, (size_t)cap * 768);
  GROW(mfaces_b, (size_t)cap * 768);
  // new face words carry epoch 0, which no sweep uses
  SHKZ_CUDA_TRY(cudaMemsetAsync(ctx->mfaces_f, 0, sizeof(unsigned long long) * (size_t)cap * 768, ctx->stream));
  SHKZ_CUDA_TRY(cudaMemsetAsync(ctx->mfaces_b, 0, sizeof(unsigned long long) * (size_t)cap * 768, ctx->stream));
  ctx->cap_macro = cap;
  return 0;
}

// 16^3 macro tiles over the pool (2x2x2 tiles each) for the MIC(0) sweeps:
// the pool kernels run again on a grid twice as coarse, with the summed
// unknown counts of each macro tile's eight tiles.
static int build_macro_tiles(shkz_b200_ctx *ctx, const Geometry &G, int K, cudaStream_t s) {
  ctx->KM = 0;
  if (K <= 0 || ctx->cfg.mic_block == 8) return 0;
  Geometry M = G;
  M.bx = (G.bx + 1) / 2;
  M.by = (G.by + 1) / 2;
  M.bz = (G.bz + 1) / 2;
  M.ntiles = (long long)M.bx * M.by * M.bz;
  launch_macro_count(G, ctx->tile_count, M, ctx->mcount, s);
  const int KM = pool_count(M, ctx->mcount, ctx->bsum, ctx->total, s);
  if (KM < 0) {
    shkz_set_cuda_error(cudaGetLastError(), "pool_count (macro)", __FILE__, __LINE__);
    return SHKZ_B200_ERR_CUDA;
  }
  int rc = ensure_macro(ctx, KM > 0 ? KM : 1);
  if (rc) return rc;
  build_macro(G, M, ctx->tile_count, ctx->tile_state, ctx->mcount, ctx->mstate, ctx->mtile, ctx->mnbr,
              ctx->level_count, ctx->msched, ctx->msub, KM, ctx->bsum, s);
  SHKZ_CUDA_TRY(cudaGetLastError());
  ctx->KM = KM;
  return 0;
}

extern "C" int shkz_b200_create(shkz_b200_ctx **out, const shkz_b200_config *cfg) {
  if (!out) return SHKZ_B200_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return SHKZ_B200_ERR_NODEVICE;
  shkz_b200_ctx *ctx = new shkz_b200_ctx();
  if (cfg) ctx->cfg = *cfg;
  else shkz_b200_default_config(&ctx->cfg);
  ctx->device = ctx->cfg.device;
  if (ctx->device < 0 || ctx->device >= ndev) {
    delete ctx;
    return SHKZ_B200_ERR_ARG;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, ctx->device) != cudaSuccess || prop.major < 10) {
    delete ctx;
    return SHKZ_B200_ERR_NODEVICE;
  }
  cudaSetDevice(ctx->device);
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return SHKZ_B200_ERR_CUDA;
  }
  for (auto &e : ctx->ev) cudaEventCreate(&e);
  if (cudaMalloc(&ctx->flags, sizeof(int)) != cudaSuccess || cudaMalloc(&ctx->total, sizeof(int)) != cudaSuccess ||
      cudaMalloc(&ctx->counter, sizeof(unsigned) * 8) != cudaSuccess ||
      cudaMalloc(&ctx->st, sizeof(SolverState)) != cudaSuccess || cudaMalloc(&ctx->out4, sizeof(double) * 8) != cudaSuccess ||
      cudaMalloc(&ctx->ws, 3 * wave_sync_bytes()) != cudaSuccess ||
      cudaMalloc(&ctx->st_scratch, sizeof(SolverState)) != cudaSuccess) {
    shkz_b200_destroy(ctx);
    return SHKZ_B200_ERR_NOMEM;
  }
  cudaMemsetAsync(ctx->counter, 0, sizeof(unsigned) * 8, ctx->stream);
  cudaMemsetAsync(ctx->ws, 0, 3 * wave_sync_bytes(), ctx->stream);
  cudaMemsetAsync(ctx->st, 0, sizeof(SolverState), ctx->stream);
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
    shkz_b200_destroy(ctx);
    return SHKZ_B200_ERR_CUDA;
  }
  *out = ctx;
  return 0;
}

extern "C" void shkz_b200_destroy(shkz_b200_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  void *ptrs[] = {ctx->h_fluid, ctx->h_solid, ctx->h_vel[0], ctx->h_vel[1], ctx->h_vel[2], ctx->h_svel[0],
                  ctx->h_svel[1], ctx->h_svel[2], ctx->h_pressure, ctx->h_fluid_active, ctx->h_solid_active,
                  ctx->h_vact[0], ctx->h_vact[1], ctx->h_vact[2], ctx->h_pact, ctx->flags, ctx->unk, ctx->tile_count,
                  ctx->tile_state, ctx->pool_tile, ctx->nbr, ctx->level_count, ctx->sched, ctx->bsum, ctx->total,
                  ctx->diag, ctx->offx, ctx->offy, ctx->offz, ctx->d32, ctx->diag64, ctx->offx64, ctx->offy64,
                  ctx->offz64, ctx->rhs64, ctx->upx, ctx->upy, ctx->upz, ctx->colsum, ctx->dmic64, ctx->x64,
                  ctx->r64, ctx->xref64, ctx->p64, ctx->q64, ctx->z64, ctx->x, ctx->r, ctx->p, ctx->q, ctx->z,
                  ctx->t, ctx->p32, ctx->partials, ctx->out4, ctx->counter, ctx->st,
                  ctx->wflags, ctx->faces_f, ctx->faces_b, ctx->ws, ctx->st_scratch, ctx->mcount, ctx->mstate,
                  ctx->mtile, ctx->mnbr, ctx->msched, ctx->msub, ctx->mfaces_f, ctx->mfaces_b, ctx->curv,
                  ctx->prev, ctx->rank_pool, ctx->rank_cnt, ctx->rank_total, ctx->xw, ctx->h_dens[0],
                  ctx->h_dens[1], ctx->h_dens[2], ctx->flush, ctx->pb, ctx->ext_v[0], ctx->ext_v[1], ctx->ext_v[2],
                  ctx->ext_a[0], ctx->ext_a[1], ctx->ext_a[2], ctx->ext_flag, ctx->sp_raw, ctx->sp_posm,
                  ctx->sp_vc[0], ctx->sp_vc[1], ctx->sp_vc[2], ctx->sp_key, ctx->sp_rank, ctx->sp_list, ctx->sp_sposm,
                  ctx->sp_svc, ctx->sp_faces, ctx->sp_sorted, ctx->sp_face_bin, ctx->sp_nfaces, ctx->sp_work,
                  ctx->sp_count, ctx->sp_tile_start, ctx->sp_tile_act, ctx->sp_tiles, ctx->sp_act[0],
                  ctx->sp_act[1], ctx->sp_act[2], ctx->sp_mass[0], ctx->sp_mass[1], ctx->sp_mass[2], ctx->sp_mom[0],
                  ctx->sp_mom[1], ctx->sp_mom[2],
                  ctx->sp_sact[0], ctx->sp_sact[1], ctx->sp_sact[2]};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (ctx->model) learned_free(ctx->model);
  for (auto &e : ctx->ev)
    if (e) cudaEventDestroy(e);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

extern "C" int shkz_b200_set_config(shkz_b200_ctx *ctx, const shkz_b200_config *cfg) {
  if (!ctx || !cfg) return SHKZ_B200_ERR_ARG;
  ctx->cfg = *cfg;
  return 0;
}

extern "C" void *shkz_b200_stream(shkz_b200_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

static PoolSystem pool_system(shkz_b200_ctx *ctx) {
  PoolSystem S;
  S.K = ctx->K;
  S.nbr = ctx->nbr;
  S.sched = ctx->sched;
  S.KM = ctx->cfg.mic_block == 8 ? 0 : ctx->KM;
  S.msched = ctx->msched;
  S.mnbr = ctx->mnbr;
  S.msub = ctx->msub;
  S.mfaces_f = ctx->mfaces_f;
  S.mfaces_b = ctx->mfaces_b;
  S.diag = ctx->diag;
  S.offx = ctx->offx;
  S.offy = ctx->offy;
  S.offz = ctx->offz;
  S.diag64 = ctx->diag64;
  S.offx64 = ctx->offx64;
  S.offy64 = ctx->offy64;
  S.offz64 = ctx->offz64;
  S.upx = ctx->upx;
  S.upy = ctx->upy;
  S.upz = ctx->upz;
  return S;
}

static char *wsync(shkz_b200_ctx *ctx, int which) { return (char *)ctx->ws + which * wave_sync_bytes(); }

// Before a call's wavefront kernels: clear the three wave-sync error words
// (a timed-out call leaves one set) and write the configured spin limit and
// the fault-injection slot (forward sweep only). The words are
// error, spin_limit, skip_publish at byte offset 12 of each WaveSync; the
// slot, epoch and finished words are left alone, so face tags stay valid.
static int arm_waves(shkz_b200_ctx *ctx) {
  for (int w = 0; w < 3; ++w) {
    const int words[3] = {0, ctx->cfg.spin_limit > 0 ? ctx->cfg.spin_limit : 0,
                          w == 1 && ctx->cfg.fault_skip_publish > 0 ? ctx->cfg.fault_skip_publish : 0};
    SHKZ_CUDA_TRY(cudaMemcpyAsync(wsync(ctx, w) + 3 * sizeof(int), words, sizeof(words), cudaMemcpyHostToDevice,
                                  ctx->stream));
  }
  return 0;
}

// Wave-sync error word (offset of `error` inside WaveSync is 3 ints).
static int wave_errors(shkz_b200_ctx *ctx) {
  std::vector<char> h(3 * wave_sync_bytes());
  if (cudaMemcpy(h.data(), ctx->ws, h.size(), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  int any = 0;
  for (int w = 0; w < 3; ++w) {
    int err;
    std::memcpy(&err, h.data() + w * wave_sync_bytes() + 3 * sizeof(int), sizeof(int));
    any |= (err != 0);
  }
  return any;
}

// --------------------------------------------------------------------------
// FP32 PCG with FP64 reductions and reliable updates.
//
// One PCG recurrence (the reference loop, pcg_solver.h:246-295) runs on FP32
// vectors scaled by 1/||b||inf. The solution is accumulated in FP64: each time
// the recursive residual has dropped by `kReliableDrop` since the last update,
// and whenever it meets the tolerance, the FP32 increment is added to x64, the
// true residual b - A x64 is recomputed in FP64 and replaces the recursive one,
// and the search direction is kept. The stopping test is always decided on the
// true FP64 residual, so FP32 rounding never ends a solve early and the
// iteration count stays that of the FP64 recurrence.

static const double kReliableDrop = 0.1;

// z = M^-1 r, rho_new, beta, p = z + beta p (or the identity-preconditioned variant)
static void launch_iteration_tail(shkz_b200_ctx *ctx, const PoolSystem &S, int n, int precond, cudaStream_t s) {
  if (precond == SHKZ_B200_PRECOND_MIC0) {
    launch_mic_apply(S, ctx->d32, ctx->r, ctx->t, ctx->z, ctx->partials, ctx->faces_f,
                     ctx->faces_b, wsync(ctx, 1), wsync(ctx, 2), ctx->st, s);
    launch_finish_rho(ctx->partials, mic_partial_count(S), ctx->st, 0, s);
    launch_update_p(n, ctx->z, ctx->p, ctx->st, s);
  } else {
    launch_finish_rho_r2(ctx->st, 0, s);
    launch_update_p(n, ctx->r, ctx->p, ctx->st, s);
  }
}

static int solve_system(shkz_b200_ctx *ctx, double tol, int precond, shkz_b200_result *res) {
  cudaStream_t s = ctx->stream;
  const PoolSystem S = pool_system(ctx);
  const int n = ctx->K * SHKZ_TC;
  SHKZ_CUDA_TRY(cudaMemsetAsync(ctx->x64, 0, sizeof(double) * n, s));
  double h4[4];
  launch_residual64(S, ctx->rhs64, ctx->x64, ctx->r64, ctx->partials, ctx->counter + 2, ctx->out4, s);
  SHKZ_CUDA_TRY(cudaMemcpyAsync(h4, ctx->out4, sizeof(h4), cudaMemcpyDeviceToHost, s));
  SHKZ_CUDA_TRY(cudaStreamSynchronize(s));
  const double bmax = h4[2], b2 = h4[3];
  double rmax = h4[0], r2 = h4[1];
  res->outer_steps = 0;
  if (bmax == 0.0) {
    res->iterations = 0;
    res->reresid = 0.0;
    res->reresid_l2 = 0.0;
    return 0;
  }
  if (!(b2 == b2)) {
    res->iterations = 0;
    return SHKZ_B200_ERR_NAN;
  }
  const double scale = bmax;
  const bool reliable = ctx->cfg.refine != 0;
  launch_inner_init(n, ctx->r64, 1.0 / scale, ctx->r, ctx->x, s);
  launch_inner_setup(n, ctx->r, ctx->partials, ctx->counter, ctx->st, tol, s);
  launch_state_resume(ctx->st, reliable ? kReliableDrop : 0.0, s);
  // z0 = M^-1 r0, rho0, p0 = z0
  if (precond == SHKZ_B200_PRECOND_MIC0) {
    launch_mic_apply(S, ctx->d32, ctx->r, ctx->t, ctx->z, ctx->partials, ctx->faces_f,
                     ctx->faces_b, wsync(ctx, 1), wsync(ctx, 2), ctx->st, s);
    launch_finish_rho(ctx->partials, mic_partial_count(S), ctx->st, 1, s);
    SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->p, ctx->z, sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
  } else {
    launch_finish_rho_r2(ctx->st, 1, s);
    SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->p, ctx->r, sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
  }
  const int max_it = ctx->cfg.max_iterations;
  const int batch = ctx->cfg.check_interval > 0 ? ctx->cfg.check_interval : 16;
  SolverState hst;
  int rc = 0, updates = 0;
  bool true_checked = false;
  // MIC(0) on macro tiles: the direction update p = z + beta p rides in the
  // next iteration's stencil (ping-pong between two p buffers) and the x/r
  // update in the forward sweep's staging, so an iteration is three passes
  // (stencil, forward sweep, backward sweep; the backward sweep's last CTA
  // also finishes rho and beta)
  // (the current direction is in ctx->p after an even number of completed
  // iterations and in ctx->pb after an odd one; the kernels pick it on the
  // device, where retired launches leave the count alone)
  const bool fused = precond == SHKZ_B200_PRECOND_MIC0 && S.KM > 0;
  for (;;) {
    for (int b = 0; b < batch; ++b) {
      if (fused) {
        launch_spmv_update(S, ctx->p, ctx->pb, ctx->z, ctx->q, ctx->partials, ctx->counter, ctx->st, s);
        launch_mic_apply_update(S, ctx->d32, ctx->r, ctx->t, ctx->z, ctx->partials, ctx->p, ctx->pb, ctx->q, ctx->x,
                                ctx->counter + 1, ctx->st, max_it, wsync(ctx, 1), wsync(ctx, 2), ctx->counter + 5, s);
        continue;
      }
      launch_spmv(S, ctx->p, ctx->q, ctx->partials, ctx->counter, ctx->st, 0, s);
      launch_update_xr(n, ctx->p, ctx->q, ctx->x, ctx->r, ctx->partials, ctx->counter + 1, ctx->st, max_it, s);
      launch_iteration_tail(ctx, S, n, precond, s);
    }
    SHKZ_CUDA_TRY(cudaMemcpyAsync(&hst, ctx->st, sizeof(hst), cudaMemcpyDeviceToHost, s));
    SHKZ_CUDA_TRY(cudaStreamSynchronize(s));
    // a bounded wait that gave up leaves its iterate undefined: stop here
    if (wave_errors(ctx)) { rc = SHKZ_B200_ERR_TIMEOUT; break; }
    if (hst.done == 0) continue;
    if (hst.done == 3 || hst.status == -5) { rc = SHKZ_B200_ERR_NAN; break; }
    if (hst.done == 2) break;
    if (hst.done == 1 && !reliable) break;
    // reliable update: fold the FP32 increment into x64 and replace r by b - A x64
    launch_accumulate(n, ctx->x, scale, ctx->x64, s);
    launch_residual64(S, ctx->rhs64, ctx->x64, ctx->r64, ctx->partials, ctx->counter + 2, ctx->out4, s);
    SHKZ_CUDA_TRY(cudaMemcpyAsync(h4, ctx->out4, sizeof(h4), cudaMemcpyDeviceToHost, s));
    SHKZ_CUDA_TRY(cudaStreamSynchronize(s));
    rmax = h4[0];
    r2 = h4[1];
    ++updates;
    true_checked = true;
    if (!(rmax == rmax)) { rc = SHKZ_B200_ERR_NAN; break; }
    if (rmax <= tol * bmax) break;
    launch_inner_init(n, ctx->r64, 1.0 / scale, ctx->r, ctx->x, s);
    launch_state_resume(ctx->st, kReliableDrop * rmax / scale, s);
    true_checked = false;
    // complete the interrupted iteration with the replaced residual (the
    // fused loop leaves the direction update to its next stencil)
    if (fused) {
      launch_mic_apply(S, ctx->d32, ctx->r, ctx->t, ctx->z, ctx->partials, ctx->faces_f, ctx->faces_b, wsync(ctx, 1),
                       wsync(ctx, 2), ctx->st, s);
      launch_finish_rho(ctx->partials, mic_partial_count(S), ctx->st, 0, s);
    } else {
      launch_iteration_tail(ctx, S, n, precond, s);
    }
  }
  if (!true_checked) {
    // plain FP32 finish (refine off) or max iterations: report the true residual
    launch_accumulate(n, ctx->x, scale, ctx->x64, s);
    launch_residual64(S, ctx->rhs64, ctx->x64, ctx->r64, ctx->partials, ctx->counter + 2, ctx->out4, s);
    SHKZ_CUDA_TRY(cudaMemcpyAsync(h4, ctx->out4, sizeof(h4), cudaMemcpyDeviceToHost, s));
    SHKZ_CUDA_TRY(cudaStreamSynchronize(s));
    rmax = h4[0];
    r2 = h4[1];
  }
  if (wave_errors(ctx)) rc = SHKZ_B200_ERR_TIMEOUT;
  res->iterations = hst.iter;
  res->outer_steps = updates;
  res->reresid = rmax / bmax;
  res->reresid_l2 = std::sqrt(r2 / b2);
  return rc;
}

// FP64 tight reference solve: flexible CG (Polak-Ribiere beta) in FP64 whose
// preconditioner is the FP32 MIC(0) applied to the scaled residual. It
// solves the same FP64 system the reference assembles, to fp64_tol, into
// xref64, and reports ||x64 - xref64||inf / ||xref64||inf.
// x0 (may be null): warm-start vector already added to x64; the reference
// solution of the shifted system gets it too before the comparison.
static int fp64_reference_solve(shkz_b200_ctx *ctx, shkz_b200_result *res, const double *x0) {
  cudaStream_t s = ctx->stream;
  const PoolSystem S = pool_system(ctx);
  const int n = ctx->K * SHKZ_TC;
  const double tol = ctx->cfg.fp64_tol > 0 ? ctx->cfg.fp64_tol : 1e-12;
  double h[4];
  auto dots = [&](const double *a, const double *b, const double *c, const double *d) -> int {
    launch_dots64(n, a, b, c, d, ctx->partials, ctx->counter + 3, ctx->out4, s);
    if (cudaMemcpyAsync(h, ctx->out4, sizeof(double) * 3, cudaMemcpyDeviceToHost, s) != cudaSuccess) return -1;
    return cudaStreamSynchronize(s) == cudaSuccess ? 0 : -1;
  };
  auto precond = [&](const double *r, double rmax) {
    // z = rmax * M^-1 (r / rmax) with M^-1 the FP32 MIC(0)
    launch_scale_f64_f32(n, r, 1.0 / rmax, ctx->r, s);
    launch_mic_apply(S, ctx->d32, ctx->r, ctx->t, ctx->z, nullptr, ctx->faces_f,
                     ctx->faces_b, wsync(ctx, 1), wsync(ctx, 2), nullptr, s);
    launch_scale_f32_f64(n, ctx->z, rmax, ctx->z64, s);
  };
  SHKZ_CUDA_TRY(cudaMemsetAsync(ctx->xref64, 0, sizeof(double) * n, s));
  SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->r64, ctx->rhs64, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  if (dots(ctx->r64, ctx->r64, nullptr, nullptr)) return SHKZ_B200_ERR_CUDA;
  const double bmax = h[2];
  if (bmax == 0.0) {
    res->fp64_reresid = 0.0;
    res->err_fp64_inf = 0.0;
    return 0;
  }
  double rmax = bmax;
  precond(ctx->r64, rmax);
  if (dots(ctx->z64, ctx->r64, nullptr, nullptr)) return SHKZ_B200_ERR_CUDA;
  double rho = h[0];
  SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->p64, ctx->z64, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  int it = 0;
  const int max_it = ctx->cfg.max_iterations;
  for (; it < max_it; ++it) {
    launch_apply64(S, ctx->p64, ctx->q64, s);
    if (dots(ctx->p64, ctx->q64, nullptr, nullptr)) return SHKZ_B200_ERR_CUDA;
    const double alpha = rho / h[0];
    launch_axpy2_64(n, alpha, ctx->p64, ctx->xref64, ctx->q64, ctx->r64, s);
    if (dots(ctx->r64, ctx->r64, nullptr, nullptr)) return SHKZ_B200_ERR_CUDA;
    rmax = h[2];
    if (!(rmax == rmax)) return SHKZ_B200_ERR_NAN;
    if (rmax <= tol * bmax) break;
    precond(ctx->r64, rmax);
    if (dots(ctx->z64, ctx->r64, ctx->z64, ctx->q64)) return SHKZ_B200_ERR_CUDA;
    const double rho_new = h[0];
    const double beta = -alpha * h[1] / rho;
    launch_xpby64(n, ctx->z64, beta, ctx->p64, s);
    rho = rho_new;
  }
  // true residual of the reference solution and the error of x64
  launch_residual64(S, ctx->rhs64, ctx->xref64, ctx->r64, ctx->partials, ctx->counter + 2, ctx->out4, s);
  SHKZ_CUDA_TRY(cudaMemcpyAsync(h, ctx->out4, sizeof(double) * 4, cudaMemcpyDeviceToHost, s));
  SHKZ_CUDA_TRY(cudaStreamSynchronize(s));
  res->fp64_reresid = h[0] / h[2];
  if (x0) launch_axpy2_64(n, 1.0, x0, ctx->xref64, x0, ctx->p64, s);  // xref64 += x0 (p64 scratch)
  // error: ||x64 - xref64||inf over ||xref64||inf  (q64 = x64 - xref64)
  SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->q64, ctx->x64, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  launch_axpy2_64(n, -1.0, ctx->xref64, ctx->q64, ctx->xref64, ctx->p64, s);  // second pair is a scratch write
  if (dots(ctx->q64, ctx->q64, ctx->xref64, ctx->xref64)) return SHKZ_B200_ERR_CUDA;
  const double emax = h[2];
  if (dots(ctx->xref64, ctx->xref64, nullptr, nullptr)) return SHKZ_B200_ERR_CUDA;
  res->err_fp64_inf = h[2] > 0 ? emax / h[2] : 0.0;
  return 0;
}

static int learned_solve(shkz_b200_ctx *ctx, double tol, shkz_b200_result *res);

static int validate(const shkz_b200_project_args *a) {
  if (!a || a->nx <= 0 || a->ny <= 0 || a->nz <= 0 || !a->fluid || !a->fluid_active) return SHKZ_B200_ERR_ARG;
  if (a->nx > 65536 || a->ny > 65536 || a->nz > 65536) return SHKZ_B200_ERR_LIMIT;
  if ((size_t)a->nx * a->ny * a->nz > ((size_t)1 << 31)) return SHKZ_B200_ERR_LIMIT;
  if ((a->solid == nullptr) != (a->solid_active == nullptr)) return SHKZ_B200_ERR_ARG;
  for (int d = 0; d < 3; ++d)
    if (!a->velocity[d] || !a->velocity_active[d]) return SHKZ_B200_ERR_ARG;
  if (!(a->dx > 0.0)) return SHKZ_B200_ERR_ARG;
  const bool dens = a->solid_density[0] || a->solid_density[1] || a->solid_density[2];
  if (dens && !(a->solid_density[0] && a->solid_density[1] && a->solid_density[2])) return SHKZ_B200_ERR_ARG;
  return 0;
}

static float ms_between(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

// warm-start buffers: pool-sized rank and x0, reference-tile counts, and the
// previous vector (kept across growth)
static int ensure_warm(shkz_b200_ctx *ctx, const Geometry &G, int T, long long unknowns_bound) {
  if (ctx->cap_warm_pool < ctx->cap_pool) {
    GROW(rank_pool, (size_t)ctx->cap_pool * SHKZ_TC);
    GROW(xw, (size_t)ctx->cap_pool * SHKZ_TC);
    ctx->cap_warm_pool = ctx->cap_pool;
  }
  const size_t nref = unknown_rank_scratch(G, T);
  if (nref > ctx->cap_rank_cnt) {
    GROW(rank_cnt, nref);
    ctx->cap_rank_cnt = nref;
  }
  if (!ctx->rank_total) GROW(rank_total, 1);
  if (unknowns_bound > ctx->cap_prev) {
    const long long cap = unknowns_bound + unknowns_bound / 4 + 1024;
    double *np = nullptr;
    cudaError_t e = cudaMalloc(&np, sizeof(double) * (size_t)cap);
    if (e != cudaSuccess) {
      shkz_set_cuda_error(e, "cudaMalloc", __FILE__, __LINE__);
      return SHKZ_B200_ERR_NOMEM;
    }
    if (ctx->prev && ctx->prev_n > 0)
      SHKZ_CUDA_TRY(cudaMemcpyAsync(np, ctx->prev, sizeof(double) * (size_t)ctx->prev_n, cudaMemcpyDeviceToDevice,
                                    ctx->stream));
    SHKZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (ctx->prev) cudaFree(ctx->prev);
    ctx->prev = np;
    ctx->cap_prev = cap;
  }
  return 0;
}

static int project_device(shkz_b200_ctx *ctx, const shkz_b200_project_args *a, shkz_b200_result *res) {
  cudaStream_t s = ctx->stream;
  const Geometry G = make_geometry(a->nx, a->ny, a->nz);
  // the previous system's buffers may be regrown (or fail to be) below:
  // nothing may inspect or reuse that system until this call completes one
  ctx->has_system = 0;
  int rc = ensure_grid(ctx, G);
  if (rc) return rc;
  AssemblyInputs in;
  in.G = G;
  in.fluid = a->fluid;
  in.fluid_active = a->fluid_active;
  in.solid = a->solid;
  in.solid_active = a->solid_active;
  for (int d = 0; d < 3; ++d) {
    in.vel[d] = a->velocity[d];
    in.svel[d] = a->solid_velocity[d];
  }
  in.dx = a->dx;
  in.dt = a->dt;
  in.eps_solid = ctx->cfg.eps_solid;
  in.eps_fluid = ctx->cfg.eps_fluid;
  in.second_order_fluid = ctx->cfg.second_order_fluid;
  in.second_order_solid = ctx->cfg.second_order_solid;
  for (int d = 0; d < 3; ++d) in.density[d] = a->solid_density[d];
  in.rhs_add = 0.0;

  ctx->last_in = in;
  const long long launches0 = launches_so_far();
  cudaEventRecord(ctx->ev[0], s);
  launch_label(in, ctx->flags, ctx->unk, ctx->tile_count, s);
  cudaEventRecord(ctx->ev[8], s);
  if (a->surface_tension != 0.0) {
    // velocity += surface tension force before the system is built (it reads the new velocity)
    const size_t cells = (size_t)G.nx * G.ny * G.nz;
    if (cells > ctx->cap_curv) {
      GROW(curv, cells);
      ctx->cap_curv = cells;
    }
    float *vel[3] = {a->velocity[0], a->velocity[1], a->velocity[2]};
    const uint8_t *vact[3] = {a->velocity_active[0], a->velocity_active[1], a->velocity_active[2]};
    launch_surface_tension(in, ctx->flags, ctx->curv, a->surface_tension, vel, vact, s);
  }
  // pool size (one small host read), then the pool itself
  const int K = pool_count(G, ctx->tile_count, ctx->bsum, ctx->total, s);
  if (K < 0) {
    shkz_set_cuda_error(cudaGetLastError(), "pool_count", __FILE__, __LINE__);
    return SHKZ_B200_ERR_CUDA;
  }
  rc = ensure_pool(ctx, K > 0 ? K : 1);
  if (rc) return rc;
  pool_assign(G, ctx->tile_count, K, ctx->bsum, ctx->tile_state, ctx->pool_tile, ctx->nbr, ctx->level_count,
              ctx->sched, s);
  SHKZ_CUDA_TRY(cudaGetLastError());
  rc = build_macro_tiles(ctx, G, K, s);
  if (rc) return rc;
  rc = arm_waves(ctx);
  if (rc) return rc;
  cudaEventRecord(ctx->ev[9], s);
  ctx->K = K;
  ctx->G = G;
  ctx->model_ready = 0;
  res->tiles = K;
  res->volume_rhs_correct = 0.0;
  if (K > 0 && ctx->cfg.gain != 0.0 && ctx->vol_target != 0.0) {
    // PI volume correction (macpressuresolver3.cpp:219-234), state advanced once per solved projection
    const double x = (ctx->vol_current - ctx->vol_target) / ctx->vol_target;
    const double y = ctx->vol_yprev + x * a->dt;
    ctx->vol_yprev = y;
    const double kp = ctx->cfg.gain * 2.3 / (25.0 * 0.01);
    const double ki = kp * kp / 16.0;
    in.rhs_add = -(kp * x + ki * y) / (x + 1.0);
    res->volume_rhs_correct = in.rhs_add;
    ctx->last_in = in;
  }
  CoeffOutputs co{ctx->diag, ctx->offx, ctx->offy, ctx->offz, ctx->diag64, ctx->offx64, ctx->offy64, ctx->offz64,
                  ctx->rhs64};
  launch_coeff(in, ctx->flags, ctx->pool_tile, K, ctx->unk, co, s);
  if (K > 0) launch_upper_weights(pool_system(ctx), ctx->upx, ctx->upy, ctx->upz, s);
  cudaEventRecord(ctx->ev[10], s);
  const bool warm = K > 0 && ctx->cfg.warm_start;
  if (warm) {
    // b <- b - A x_prev with x_prev read by the reference's unknown number
    const int T = ctx->cfg.index_tile > 0 ? ctx->cfg.index_tile : 16;
    rc = ensure_warm(ctx, G, T, (long long)K * SHKZ_TC);
    if (rc) return rc;
    const PoolSystem S0 = pool_system(ctx);
    launch_unknown_rank(G, K, ctx->unk, T, ctx->tile_state, ctx->rank_pool, ctx->rank_cnt, ctx->rank_total, s);
    launch_warm_gather((long long)K * SHKZ_TC, ctx->rank_pool, ctx->prev, ctx->prev_n, ctx->xw, s);
    launch_residual64(S0, ctx->rhs64, ctx->xw, ctx->r64, ctx->partials, ctx->counter + 2, ctx->out4, s);
    SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->rhs64, ctx->r64, sizeof(double) * (size_t)K * SHKZ_TC,
                                  cudaMemcpyDeviceToDevice, s));
  }
  const int precond = ctx->cfg.preconditioner;
  const PoolSystem S = pool_system(ctx);
  ctx->mic_ready = 0;
  if (K > 0 && (precond == SHKZ_B200_PRECOND_MIC0 || precond == SHKZ_B200_PRECOND_LEARNED)) {
    launch_mic_factor(S, ctx->colsum, ctx->cfg.mic_omega, ctx->cfg.mic_min_diag_ratio, ctx->dmic64, ctx->d32,
                      ctx->wflags, wsync(ctx, 0), s);
    ctx->mic_ready = 1;
  }
  SHKZ_CUDA_TRY(cudaGetLastError());
  cudaEventRecord(ctx->ev[1], s);
  ctx->has_system = 1;
  // unknown count (for the result)
  {
    std::vector<int> tc((size_t)G.ntiles);
    SHKZ_CUDA_TRY(cudaMemcpyAsync(tc.data(), ctx->tile_count, sizeof(int) * G.ntiles, cudaMemcpyDeviceToHost, s));
    SHKZ_CUDA_TRY(cudaStreamSynchronize(s));
    long long u = 0;
    for (int v : tc) u += v;
    ctx->unknowns = u;
    res->unknowns = u;
  }
  int solve_rc = 0;
  if (K > 0) {
    if (precond == SHKZ_B200_PRECOND_LEARNED && ctx->model)
      solve_rc = learned_solve(ctx, ctx->cfg.residual, res);
    else
      solve_rc = solve_system(ctx, ctx->cfg.residual, precond == SHKZ_B200_PRECOND_LEARNED ? SHKZ_B200_PRECOND_MIC0 : precond, res);
  } else {
    res->iterations = 0;
    res->reresid = 0.0;
  }
  cudaEventRecord(ctx->ev[2], s);
  // FP32 pressure of the solution, then the velocity update
  const int n = K * SHKZ_TC;
  if (warm) {
    // x = d + x_prev, and the new previous vector (length = unknown count)
    launch_warm_finish(n, ctx->rank_pool, ctx->xw, ctx->x64, ctx->prev, s);
    ctx->prev_n = ctx->unknowns;
  }
  if (K > 0) launch_to_float(n, ctx->x64, ctx->p32, s);
  float *vel[3] = {a->velocity[0], a->velocity[1], a->velocity[2]};
  uint8_t *vact[3] = {a->velocity_active[0], a->velocity_active[1], a->velocity_active[2]};
  if (K > 0) launch_velocity_update(in, ctx->flags, ctx->tile_state, ctx->p32, vel, vact, s);
  if (a->pressure || a->pressure_active)
    launch_scatter_pressure(G, ctx->tile_state, ctx->p32, ctx->unk, a->pressure, a->pressure_active, s);
  cudaEventRecord(ctx->ev[3], s);
  SHKZ_CUDA_TRY(cudaGetLastError());
  // optional FP64 tight reference solve
  res->err_fp64_inf = -1.0;
  res->fp64_reresid = -1.0;
  if (K > 0 && ctx->cfg.fp64_reference) {
    int rrc = fp64_reference_solve(ctx, res, warm ? ctx->xw : nullptr);
    if (rrc && !solve_rc) solve_rc = rrc;
  }
  SHKZ_CUDA_TRY(cudaStreamSynchronize(s));
  res->ms_assemble = ms_between(ctx->ev[0], ctx->ev[1]);
  res->ms_solve = ms_between(ctx->ev[1], ctx->ev[2]);
  res->ms_update = ms_between(ctx->ev[2], ctx->ev[3]);
  res->ms_total = ms_between(ctx->ev[0], ctx->ev[3]);
  res->ms_fractions = ms_between(ctx->ev[0], ctx->ev[8]);
  res->ms_labelling = ms_between(ctx->ev[8], ctx->ev[9]);
  res->ms_build = ms_between(ctx->ev[9], ctx->ev[10]);
  res->kernel_launches = launches_so_far() - launches0;
  res->status = solve_rc;
  return solve_rc;
}

extern "C" int shkz_b200_project_device(shkz_b200_ctx *ctx, const shkz_b200_project_args *a, shkz_b200_result *res) {
  if (!ctx || !res) return SHKZ_B200_ERR_ARG;
  std::memset(res, 0, sizeof(*res));
  int rc = validate(a);
  if (rc) return res->status = rc;
  cudaSetDevice(ctx->device);
  rc = project_device(ctx, a, res);
  res->status = rc;
  return rc;
}

extern "C" int shkz_b200_project_host(shkz_b200_ctx *ctx, const shkz_b200_project_args *a, shkz_b200_result *res) {
  if (!ctx || !res) return SHKZ_B200_ERR_ARG;
  std::memset(res, 0, sizeof(*res));
  int rc = validate(a);
  if (rc) return res->status = rc;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const Geometry G = make_geometry(a->nx, a->ny, a->nz);
  const bool svel[3] = {a->solid_velocity[0] != nullptr, a->solid_velocity[1] != nullptr,
                        a->solid_velocity[2] != nullptr};
  rc = ensure_grid(ctx, G);
  if (rc) return res->status = rc;
  rc = ensure_host_staging(ctx, G, a->solid != nullptr, svel);
  if (rc) return res->status = rc;
  const size_t cells = (size_t)G.nx * G.ny * G.nz;
  const size_t nodes = (size_t)(G.nx + 1) * (G.ny + 1) * (G.nz + 1);
  cudaEvent_t e0 = ctx->ev[4], e1 = ctx->ev[5], e2 = ctx->ev[6], e3 = ctx->ev[7];
  cudaEventRecord(e0, s);
  SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->h_fluid, a->fluid, cells * 4, cudaMemcpyHostToDevice, s));
  SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->h_fluid_active, a->fluid_active, cells, cudaMemcpyHostToDevice, s));
  if (a->solid) {
    SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->h_solid, a->solid, nodes * 4, cudaMemcpyHostToDevice, s));
    SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->h_solid_active, a->solid_active, nodes, cudaMemcpyHostToDevice, s));
  }
  size_t nf[3];
  for (int d = 0; d < 3; ++d) {
    nf[d] = (size_t)(G.nx + (d == 0)) * (G.ny + (d == 1)) * (G.nz + (d == 2));
    SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->h_vel[d], a->velocity[d], nf[d] * 4, cudaMemcpyHostToDevice, s));
    SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->h_vact[d], a->velocity_active[d], nf[d], cudaMemcpyHostToDevice, s));
    if (svel[d])
      SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->h_svel[d], a->solid_velocity[d], nf[d] * 4, cudaMemcpyHostToDevice, s));
    if (a->solid_density[d]) {
      if (nf[d] > ctx->cap_h_dens[d]) {
        GROW(h_dens[d], nf[d]);
        ctx->cap_h_dens[d] = nf[d];
      }
      SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->h_dens[d], a->solid_density[d], nf[d] * 4, cudaMemcpyHostToDevice, s));
    }
  }
  cudaEventRecord(e1, s);
  shkz_b200_project_args da = *a;
  da.fluid = ctx->h_fluid;
  da.fluid_active = ctx->h_fluid_active;
  da.solid = a->solid ? ctx->h_solid : nullptr;
  da.solid_active = a->solid ? ctx->h_solid_active : nullptr;
  for (int d = 0; d < 3; ++d) {
    da.velocity[d] = ctx->h_vel[d];
    da.velocity_active[d] = ctx->h_vact[d];
    da.solid_velocity[d] = svel[d] ? ctx->h_svel[d] : nullptr;
    da.solid_density[d] = a->solid_density[d] ? ctx->h_dens[d] : nullptr;
  }
  da.pressure = ctx->h_pressure;
  da.pressure_active = ctx->h_pact;
  rc = project_device(ctx, &da, res);
  if (rc && rc != SHKZ_B200_ERR_NAN && rc != SHKZ_B200_ERR_TIMEOUT) return res->status = rc;
  cudaEventRecord(e2, s);
  for (int d = 0; d < 3; ++d) {
    SHKZ_CUDA_TRY(cudaMemcpyAsync(a->velocity[d], ctx->h_vel[d], nf[d] * 4, cudaMemcpyDeviceToHost, s));
    SHKZ_CUDA_TRY(cudaMemcpyAsync(a->velocity_active[d], ctx->h_vact[d], nf[d], cudaMemcpyDeviceToHost, s));
  }
  if (a->pressure) SHKZ_CUDA_TRY(cudaMemcpyAsync(a->pressure, ctx->h_pressure, cells * 4, cudaMemcpyDeviceToHost, s));
  if (a->pressure_active)
    SHKZ_CUDA_TRY(cudaMemcpyAsync(a->pressure_active, ctx->h_pact, cells, cudaMemcpyDeviceToHost, s));
  cudaEventRecord(e3, s);
  SHKZ_CUDA_TRY(cudaStreamSynchronize(s));
  res->ms_h2d = ms_between(e0, e1);
  res->ms_d2h = ms_between(e2, e3);
  res->ms_total = ms_between(e0, e3);
  res->status = rc;
  return rc;
}

// --------------------------------------------------------------------------
// Velocity extension after a projection (macliquid3::extend_both,
// src/liquid/macliquid3.cpp:330-340): kernels in extend.cu.

static int validate_extend(const shkz_b200_extend_args *a) {
  if (!a || a->nx < 2 || a->ny < 2 || a->nz < 2) return SHKZ_B200_ERR_ARG;
  if (a->nx > 65536 || a->ny > 65536 || a->nz > 65536) return SHKZ_B200_ERR_LIMIT;
  if ((size_t)a->nx * a->ny * a->nz > ((size_t)1 << 31)) return SHKZ_B200_ERR_LIMIT;
  if (a->width < 0 || a->width > 4096) return SHKZ_B200_ERR_ARG;
  if (a->constrain && !(a->dx > 0.0)) return SHKZ_B200_ERR_ARG;
  if ((a->solid == nullptr) != (a->solid_active == nullptr)) return SHKZ_B200_ERR_ARG;
  for (int d = 0; d < 3; ++d)
    if (!a->velocity[d] || !a->velocity_active[d]) return SHKZ_B200_ERR_ARG;
  // the kernels read masks 16 bytes and the solid 4 values at a time
  auto aligned16 = [](const void *p) { return ((uintptr_t)p & 15u) == 0; };
  for (int d = 0; d < 3; ++d)
    if (!aligned16(a->velocity_active[d])) return SHKZ_B200_ERR_ARG;
  if (a->solid && !(aligned16(a->solid) && aligned16(a->solid_active))) return SHKZ_B200_ERR_ARG;
  return 0;
}

static int extend_device(shkz_b200_ctx *ctx, const shkz_b200_extend_args *a) {
  cudaStream_t s = ctx->stream;
  size_t nf[3];
  for (int d = 0; d < 3; ++d) {
    nf[d] = (size_t)(a->nx + (d == 0)) * (a->ny + (d == 1)) * (a->nz + (d == 2));
    if (nf[d] > ctx->cap_ext[d]) {
      GROW(ext_v[d], nf[d]);
      GROW(ext_a[d], nf[d]);
      ctx->cap_ext[d] = nf[d];
    }
  }
  if (!ctx->ext_flag) GROW(ext_flag, 1);
  // ext_v / ext_a are a side buffer and its flags; the flags start (and end) zero
  for (int d = 0; d < 3; ++d) SHKZ_CUDA_TRY(cudaMemsetAsync(ctx->ext_a[d], 0, nf[d], s));
  for (int d = 0; d < 3; ++d) {
    const int W = a->nx + (d == 0), H = a->ny + (d == 1), D = a->nz + (d == 2);
    for (int w = 0; w < a->width; ++w)
      launch_extrapolate(W, H, D, a->velocity[d], a->velocity_active[d], ctx->ext_v[d], ctx->ext_a[d], s);
  }
  if (a->constrain) {
    ConstrainFields f;
    for (int d = 0; d < 3; ++d) {
      f.save[d] = a->velocity[d];
      f.act[d] = a->velocity_active[d];
    }
    SHKZ_CUDA_TRY(cudaMemsetAsync(ctx->ext_flag, 0, sizeof(int), s));
    if (a->solid) {
      const size_t nodes = (size_t)(a->nx + 1) * (a->ny + 1) * (a->nz + 1);
      launch_solid_exists(a->solid, a->solid_active, nodes, ctx->ext_flag, s);
    }
    // all three components are found on the unchanged field, then committed
    for (int d = 0; d < 3; ++d)
      launch_constrain_find(d, a->nx, a->ny, a->nz, a->dx, a->solid, ctx->ext_flag, f, ctx->ext_v[d], ctx->ext_a[d], s);
    for (int d = 0; d < 3; ++d) launch_apply_side(nf[d], a->velocity[d], ctx->ext_v[d], ctx->ext_a[d], s);
  }
  SHKZ_CUDA_TRY(cudaGetLastError());
  SHKZ_CUDA_TRY(cudaStreamSynchronize(s));
  return 0;
}

extern "C" int shkz_b200_extend_velocity_device(shkz_b200_ctx *ctx, const shkz_b200_extend_args *a) {
  if (!ctx) return SHKZ_B200_ERR_ARG;
  int rc = validate_extend(a);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  return extend_device(ctx, a);
}

extern "C" int shkz_b200_extend_velocity_host(shkz_b200_ctx *ctx, const shkz_b200_extend_args *a) {
  if (!ctx || !a) return SHKZ_B200_ERR_ARG;
  // host arrays may have any alignment: they are staged into the context's buffers
  shkz_b200_extend_args chk = *a;
  static const float f16[4] __attribute__((aligned(16))) = {0.f, 0.f, 0.f, 0.f};
  static const uint8_t b16[16] __attribute__((aligned(16))) = {};
  for (int d = 0; d < 3; ++d)
    if (chk.velocity_active[d]) chk.velocity_active[d] = const_cast<uint8_t *>(b16);
  if (chk.solid) {
    chk.solid = f16;
    chk.solid_active = chk.solid_active ? b16 : nullptr;
  }
  int rc = validate_extend(&chk);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const Geometry G = make_geometry(a->nx, a->ny, a->nz);
  const bool svel[3] = {false, false, false};
  rc = ensure_host_staging(ctx, G, a->solid != nullptr, svel);
  if (rc) return rc;
  const size_t nodes = (size_t)(a->nx + 1) * (a->ny + 1) * (a->nz + 1);
  shkz_b200_extend_args da = *a;
  if (a->solid) {
    SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->h_solid, a->solid, nodes * 4, cudaMemcpyHostToDevice, s));
    SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->h_solid_active, a->solid_active, nodes, cudaMemcpyHostToDevice, s));
    da.solid = ctx->h_solid;
    da.solid_active = ctx->h_solid_active;
  }
  size_t nf[3];
  for (int d = 0; d < 3; ++d) {
    nf[d] = (size_t)(a->nx + (d == 0)) * (a->ny + (d == 1)) * (a->nz + (d == 2));
    SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->h_vel[d], a->velocity[d], nf[d] * 4, cudaMemcpyHostToDevice, s));
    SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->h_vact[d], a->velocity_active[d], nf[d], cudaMemcpyHostToDevice, s));
    da.velocity[d] = ctx->h_vel[d];
    da.velocity_active[d] = ctx->h_vact[d];
  }
  rc = extend_device(ctx, &da);
  if (rc) return rc;
  for (int d = 0; d < 3; ++d) {
    SHKZ_CUDA_TRY(cudaMemcpyAsync(a->velocity[d], ctx->h_vel[d], nf[d] * 4, cudaMemcpyDeviceToHost, s));
    SHKZ_CUDA_TRY(cudaMemcpyAsync(a->velocity_active[d], ctx->h_vact[d], nf[d], cudaMemcpyDeviceToHost, s));
  }
  SHKZ_CUDA_TRY(cudaStreamSynchronize(s));
  return 0;
}

// --------------------------------------------------------------------------
// FLIP splat before the projection (macflipliquid3.cpp:135-151): kernels in
// splat.cu.

// 8x8x8 tiles of the three axes' edge grids, numbered one axis after another
static long long splat_tiles(int nx, int ny, int nz, long long base[3]) {
  long long total = 0;
  for (int d = 0; d < 3; ++d) {
    base[d] = total;
    total += (long long)((nx + (d != 0) + 7) / 8) * ((ny + (d != 1) + 7) / 8) * ((nz + (d != 2) + 7) / 8);
  }
  return total;
}

static int validate_splat(const shkz_b200_splat_args *a) {
  if (!a || a->nx < 1 || a->ny < 1 || a->nz < 1 || !(a->dx > 0.0) || a->count < 0) return SHKZ_B200_ERR_ARG;
  if (a->nx > 65536 || a->ny > 65536 || a->nz > 65536) return SHKZ_B200_ERR_LIMIT;
  long long base[3];
  const long long tiles = splat_tiles(a->nx, a->ny, a->nz, base);
  if (512 * tiles >= ((long long)1 << 31) || 3 * a->count >= ((long long)1 << 31)) return SHKZ_B200_ERR_LIMIT;
  // the velocity (in/out) and the splat grid (out) are each all three axes or
  // none, and at least one of them is given
  const bool vel0 = a->velocity[0] != nullptr;
  for (int d = 0; d < 3; ++d)
    if ((a->velocity[d] != nullptr) != vel0 || (a->velocity_active[d] != nullptr) != vel0) return SHKZ_B200_ERR_ARG;
  const bool out0 = a->mass[0] != nullptr;
  for (int d = 0; d < 3; ++d)
    if ((a->mass[d] != nullptr) != out0 || (a->momentum[d] != nullptr) != out0 ||
        (a->splat_active[d] != nullptr) != out0)
      return SHKZ_B200_ERR_ARG;
  if (!vel0 && !out0) return SHKZ_B200_ERR_ARG;
  if (a->count == 0) return 0;
  if (!a->particles || a->stride < 4 || (a->stride & 3)) return SHKZ_B200_ERR_ARG;
  auto field = [&](int off, int bytes) { return off >= 0 && (off & 3) == 0 && off + bytes <= a->stride; };
  if (!field(a->offset_position, 12) || !field(a->offset_velocity, 12) || !field(a->offset_mass, 4))
    return SHKZ_B200_ERR_ARG;
  if (a->offset_apic != -1 && !field(a->offset_apic, 36)) return SHKZ_B200_ERR_ARG;
  if (a->offset_bullet != -1 && (a->offset_bullet < 0 || a->offset_bullet >= a->stride)) return SHKZ_B200_ERR_ARG;
  return 0;
}

// particles: device records; grid: device face arrays (outputs optional)
static int splat_device(shkz_b200_ctx *ctx, const shkz_b200_splat_args *a, const void *particles,
                        const SplatGrid &grid) {
  cudaStream_t s = ctx->stream;
  SplatBuffers B{};
  B.tiles = splat_tiles(a->nx, a->ny, a->nz, B.tile_base);
  B.apic = a->offset_apic >= 0;
  const long long n = a->count;
  if (n > ctx->cap_sp_particles) {
    GROW(sp_posm, n);
    for (int d = 0; d < 3; ++d) GROW(sp_vc[d], n);
    GROW(sp_key, 3 * n);
    GROW(sp_rank, 3 * n);
    GROW(sp_list, 3 * n);
    GROW(sp_sposm, 3 * n);
    GROW(sp_svc, 3 * n);
    ctx->cap_sp_particles = n;
  }
  if (!ctx->sp_nfaces) GROW(sp_nfaces, 4);
  if (!ctx->sp_work) GROW(sp_work, 3 * kSplatWorkBins);
  if (B.tiles > ctx->cap_sp_tiles) {
    GROW(sp_count, 512 * B.tiles);
    GROW(sp_tile_act, B.tiles);
    GROW(sp_tile_start, B.tiles + 1);
    GROW(sp_tiles, scan_tile_count(B.tiles + 1));
    ctx->cap_sp_tiles = B.tiles;
    ctx->sp_dirty = true;
  }
  // counters and tile flags are zero between calls; set them once when new
  // or after a call that stopped before its clear pass
  if (ctx->sp_dirty) {
    SHKZ_CUDA_TRY(cudaMemsetAsync(ctx->sp_count, 0, (size_t)ctx->cap_sp_tiles * 512 * sizeof(int), s));
    SHKZ_CUDA_TRY(cudaMemsetAsync(ctx->sp_tile_act, 0, (size_t)ctx->cap_sp_tiles, s));
  }
  // a particle activates at most 8 faces per axis
  size_t nf[3];
  long long listed = 0;
  for (int d = 0; d < 3; ++d) {
    nf[d] = (size_t)(a->nx + (d == 0)) * (a->ny + (d == 1)) * (a->nz + (d == 2));
    B.face_off[d] = listed;
    listed += std::min((long long)nf[d], 8 * n);
  }
  if (listed > ctx->cap_sp_list) {
    GROW(sp_faces, listed);
    GROW(sp_sorted, listed);
    GROW(sp_face_bin, listed);
    ctx->cap_sp_list = listed;
  }
  for (int d = 0; d < 3; ++d) {
    if (nf[d] > ctx->cap_sp_faces[d]) {
      GROW(sp_act[d], nf[d]);
      ctx->cap_sp_faces[d] = nf[d];
    }
    B.vc[d] = ctx->sp_vc[d];
    B.act[d] = ctx->sp_act[d];
    SHKZ_CUDA_TRY(cudaMemsetAsync(ctx->sp_act[d], 0, nf[d], s));
  }
  B.posm = ctx->sp_posm;
  B.key = ctx->sp_key;
  B.rank = ctx->sp_rank;
  B.count = ctx->sp_count;
  B.tile_act = ctx->sp_tile_act;
  B.tile_start = ctx->sp_tile_start;
  B.list = ctx->sp_list;
  B.sposm = ctx->sp_sposm;
  B.svc = ctx->sp_svc;
  B.faces = ctx->sp_faces;
  B.sorted = ctx->sp_sorted;
  B.face_bin = ctx->sp_face_bin;
  B.work = ctx->sp_work;
  B.nfaces = ctx->sp_nfaces;
  SHKZ_CUDA_TRY(cudaMemsetAsync(ctx->sp_nfaces, 0, 4 * sizeof(int), s));
  SHKZ_CUDA_TRY(cudaMemsetAsync(ctx->sp_work, 0, 3 * kSplatWorkBins * sizeof(int), s));
  SplatRecords R{static_cast<const unsigned char *>(particles), n, a->stride, a->offset_position,
                 a->offset_velocity, a->offset_mass, a->offset_apic, a->offset_bullet, a->splat_bullet != 0};
  ctx->sp_dirty = true;
  launch_splat_bin(R, a->nx, a->ny, a->nz, a->dx, B, s);
  launch_splat_bucket_scan(B, ctx->sp_tiles, s);
  launch_splat_scatter(n, B, s);
  launch_splat_gather(a->nx, a->ny, a->nz, a->dx, B, grid, s);
  launch_splat_clear(B, s);
  SHKZ_CUDA_TRY(cudaGetLastError());
  int over = 0;
  SHKZ_CUDA_TRY(cudaMemcpyAsync(&over, ctx->sp_nfaces + 3, sizeof(int), cudaMemcpyDeviceToHost, s));
  SHKZ_CUDA_TRY(cudaStreamSynchronize(s));
  ctx->sp_dirty = false;
  return over ? SHKZ_B200_ERR_LIMIT : 0;
}

extern "C" int shkz_b200_splat_device(shkz_b200_ctx *ctx, const shkz_b200_splat_args *a) {
  if (!ctx) return SHKZ_B200_ERR_ARG;
  int rc = validate_splat(a);
  if (rc) return rc;
  // the kernels read the records' floats and write the face floats 4 bytes at a time
  auto aligned4 = [](const void *p) { return ((uintptr_t)p & 3u) == 0; };
  if (a->count && !aligned4(a->particles)) return SHKZ_B200_ERR_ARG;
  for (int d = 0; d < 3; ++d)
    if (!aligned4(a->velocity[d]) || !aligned4(a->mass[d]) || !aligned4(a->momentum[d])) return SHKZ_B200_ERR_ARG;
  cudaSetDevice(ctx->device);
  SplatGrid G{};
  for (int d = 0; d < 3; ++d) {
    G.velocity[d] = a->velocity[d];
    G.velocity_active[d] = a->velocity_active[d];
    G.mass[d] = a->mass[d];
    G.momentum[d] = a->momentum[d];
    G.splat_active[d] = a->splat_active[d];
  }
  return splat_device(ctx, a, a->particles, G);
}

extern "C" int shkz_b200_splat_host(shkz_b200_ctx *ctx, const shkz_b200_splat_args *a) {
  if (!ctx) return SHKZ_B200_ERR_ARG;
  int rc = validate_splat(a);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const Geometry G = make_geometry(a->nx, a->ny, a->nz);
  const bool svel[3] = {false, false, false};
  rc = ensure_host_staging(ctx, G, false, svel);
  if (rc) return rc;
  const size_t raw = (size_t)a->count * (size_t)(a->count ? a->stride : 0);
  if (raw > ctx->cap_sp_raw) {
    GROW(sp_raw, raw);
    ctx->cap_sp_raw = raw;
  }
  if (raw) SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->sp_raw, a->particles, raw, cudaMemcpyHostToDevice, s));
  const bool outs = a->mass[0] != nullptr;
  SplatGrid D{};
  size_t nf[3];
  const bool vel = a->velocity[0] != nullptr;
  for (int d = 0; d < 3; ++d) {
    nf[d] = (size_t)(a->nx + (d == 0)) * (a->ny + (d == 1)) * (a->nz + (d == 2));
    if (vel) {
      SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->h_vel[d], a->velocity[d], nf[d] * 4, cudaMemcpyHostToDevice, s));
      SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->h_vact[d], a->velocity_active[d], nf[d], cudaMemcpyHostToDevice, s));
      D.velocity[d] = ctx->h_vel[d];
      D.velocity_active[d] = ctx->h_vact[d];
    }
    if (outs) {
      if (nf[d] > ctx->cap_sp_out[d]) {
        GROW(sp_mass[d], nf[d]);
        GROW(sp_mom[d], nf[d]);
        GROW(sp_sact[d], nf[d]);
        ctx->cap_sp_out[d] = nf[d];
      }
      D.mass[d] = ctx->sp_mass[d];
      D.momentum[d] = ctx->sp_mom[d];
      D.splat_active[d] = ctx->sp_sact[d];
    }
  }
  rc = splat_device(ctx, a, ctx->sp_raw, D);
  if (rc) return rc;
  for (int d = 0; d < 3; ++d) {
    if (vel) {
      SHKZ_CUDA_TRY(cudaMemcpyAsync(a->velocity[d], ctx->h_vel[d], nf[d] * 4, cudaMemcpyDeviceToHost, s));
      SHKZ_CUDA_TRY(cudaMemcpyAsync(a->velocity_active[d], ctx->h_vact[d], nf[d], cudaMemcpyDeviceToHost, s));
    }
    if (outs) {
      SHKZ_CUDA_TRY(cudaMemcpyAsync(a->mass[d], ctx->sp_mass[d], nf[d] * 4, cudaMemcpyDeviceToHost, s));
      SHKZ_CUDA_TRY(cudaMemcpyAsync(a->momentum[d], ctx->sp_mom[d], nf[d] * 4, cudaMemcpyDeviceToHost, s));
      SHKZ_CUDA_TRY(cudaMemcpyAsync(a->splat_active[d], ctx->sp_sact[d], nf[d], cudaMemcpyDeviceToHost, s));
    }
  }
  SHKZ_CUDA_TRY(cudaStreamSynchronize(s));
  return 0;
}

// --------------------------------------------------------------------------
// inspection helpers (dense <-> pool)

__global__ void k_pool_to_dense_f32(Geometry G, const int *tile_state, const float *pool, float *dense) {
  const size_t n = (size_t)G.nx * G.ny * G.nz;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % G.nx), j = (int)((c / G.nx) % G.ny), k = (int)(c / ((size_t)G.nx * G.ny));
    const long long t = (long long)(i >> 3) + (long long)G.bx * ((long long)(j >> 3) + (long long)G.by * (k >> 3));
    const int pt = tile_state[t];
    dense[c] = pt >= 0 ? pool[(size_t)pt * SHKZ_TC + (i & 7) + 8 * (j & 7) + 64 * (k & 7)] : 0.0f;
  }
}
__global__ void k_pool_to_dense_f64(Geometry G, const int *tile_state, const double *pool, double *dense) {
  const size_t n = (size_t)G.nx * G.ny * G.nz;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % G.nx), j = (int)((c / G.nx) % G.ny), k = (int)(c / ((size_t)G.nx * G.ny));
    const long long t = (long long)(i >> 3) + (long long)G.bx * ((long long)(j >> 3) + (long long)G.by * (k >> 3));
    const int pt = tile_state[t];
    dense[c] = pt >= 0 ? pool[(size_t)pt * SHKZ_TC + (i & 7) + 8 * (j & 7) + 64 * (k & 7)] : 0.0;
  }
}
__global__ void k_dense_to_pool_f32(Geometry G, const int *pool_tile, int K, const float *dense, float *pool) {
  const size_t n = (size_t)K * SHKZ_TC;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    const int pt = (int)(o >> 9), c = (int)(o & 511);
    const long long t = pool_tile[pt];
    const int i = (int)(t % G.bx) * 8 + (c & 7), j = (int)((t / G.bx) % G.by) * 8 + ((c >> 3) & 7),
              k = (int)(t / ((long long)G.bx * G.by)) * 8 + (c >> 6);
    float v = 0.0f;
    if (i < G.nx && j < G.ny && k < G.nz) v = dense[(size_t)i + (size_t)G.nx * ((size_t)j + (size_t)G.ny * k)];
    pool[o] = v;
  }
}

extern "C" int shkz_b200_inspect(shkz_b200_ctx *ctx, int what, void *host_out, size_t bytes) {
  if (!ctx || !host_out) return SHKZ_B200_ERR_ARG;
  if (!ctx->has_system) return SHKZ_B200_ERR_STATE;
  const Geometry &G = ctx->G;
  const size_t cells = (size_t)G.nx * G.ny * G.nz;
  const bool f64 = (what >= 5);
  if (bytes < cells * (f64 ? 8 : 4)) return SHKZ_B200_ERR_ARG;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  void *dense = nullptr;
  SHKZ_CUDA_TRY(cudaMalloc(&dense, cells * (f64 ? 8 : 4)));
  const float *src32 = nullptr;
  const double *src64 = nullptr;
  switch (what) {
    case 0: src32 = ctx->diag; break;
    case 1: src32 = ctx->offx; break;
    case 2: src32 = ctx->offy; break;
    case 3: src32 = ctx->offz; break;
    case 4: src32 = ctx->d32; break;
    case 5: src64 = ctx->rhs64; break;
    case 6: src64 = ctx->x64; break;
    case 7: src64 = ctx->xref64; break;
    default: cudaFree(dense); return SHKZ_B200_ERR_ARG;
  }
  count_launches(1);
  if (src32) k_pool_to_dense_f32<<<148 * 8, 256, 0, s>>>(G, ctx->tile_state, src32, (float *)dense);
  else k_pool_to_dense_f64<<<148 * 8, 256, 0, s>>>(G, ctx->tile_state, src64, (double *)dense);
  cudaError_t e = cudaMemcpyAsync(host_out, dense, cells * (f64 ? 8 : 4), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(dense);
  if (e != cudaSuccess) {
    shkz_set_cuda_error(e, "inspect", __FILE__, __LINE__);
    return SHKZ_B200_ERR_CUDA;
  }
  return 0;
}

static int dense_roundtrip(shkz_b200_ctx *ctx, const float *in_cells, float *out_cells, int op) {
  if (!ctx || !in_cells || !out_cells) return SHKZ_B200_ERR_ARG;
  if (!ctx->has_system) return SHKZ_B200_ERR_STATE;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const Geometry &G = ctx->G;
  const size_t cells = (size_t)G.nx * G.ny * G.nz;
  const int n = ctx->K * SHKZ_TC;
  float *dense = nullptr;
  int rc = arm_waves(ctx);
  if (rc) return rc;
  SHKZ_CUDA_TRY(cudaMalloc(&dense, cells * 4));
  cudaMemcpyAsync(dense, in_cells, cells * 4, cudaMemcpyHostToDevice, s);
  if (ctx->K > 0) {
    count_launches(1);
    k_dense_to_pool_f32<<<148 * 8, 256, 0, s>>>(G, ctx->pool_tile, ctx->K, dense, ctx->r);
    const PoolSystem S = pool_system(ctx);
    if (op == 0) {
      launch_spmv(S, ctx->r, ctx->z, ctx->partials, ctx->counter, nullptr, 1, s);
    } else if (ctx->cfg.preconditioner == SHKZ_B200_PRECOND_MIC0 || ctx->cfg.preconditioner == SHKZ_B200_PRECOND_LEARNED) {
      launch_mic_apply(S, ctx->d32, ctx->r, ctx->t, ctx->z, nullptr, ctx->faces_f,
                       ctx->faces_b, wsync(ctx, 1), wsync(ctx, 2), nullptr, s);
    } else {
      cudaMemcpyAsync(ctx->z, ctx->r, sizeof(float) * n, cudaMemcpyDeviceToDevice, s);
    }
    count_launches(1);
    k_pool_to_dense_f32<<<148 * 8, 256, 0, s>>>(G, ctx->tile_state, ctx->z, dense);
  } else {
    cudaMemsetAsync(dense, 0, cells * 4, s);
  }
  cudaError_t e = cudaMemcpyAsync(out_cells, dense, cells * 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(dense);
  if (e != cudaSuccess) {
    shkz_set_cuda_error(e, "roundtrip", __FILE__, __LINE__);
    return SHKZ_B200_ERR_CUDA;
  }
  if (wave_errors(ctx)) return SHKZ_B200_ERR_TIMEOUT;
  return 0;
}

extern "C" int shkz_b200_apply_preconditioner(shkz_b200_ctx *ctx, const float *r_cells, float *z_cells) {
  return dense_roundtrip(ctx, r_cells, z_cells, 1);
}
extern "C" int shkz_b200_apply_matrix(shkz_b200_ctx *ctx, const float *x_cells, float *y_cells) {
  return dense_roundtrip(ctx, x_cells, y_cells, 0);
}

// --------------------------------------------------------------------------
// Generic CSR path for LinSolver=: the shipped pcg_solver algorithm
// (PCGSolver::solve, local/include/pcgsolver/pcg_solver.h:246-295) whose
// preconditioner result is discarded (:379-384), i.e. CG in FP64 with
// x0 = 0 and the stopping rule ||r||inf <= Residual * ||b||inf.

__global__ void k_csr_spmv64(int n, const int *__restrict__ indptr, const int *__restrict__ indices,
                             const double *__restrict__ data, const double *__restrict__ x, double *__restrict__ y,
                             const CsrState *st) {
  if (st->done) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int p = indptr[i]; p < indptr[i + 1]; ++p) s += data[p] * x[indices[p]];
    y[i] = s;
  }
}

// Iterations of one CUDA graph launched between host checks of the CSR solve.
// Every kernel returns at once after the stop, so launches past it cost only
// their (empty) launch.
constexpr int kCsrIterationsPerCheck = 16;

extern "C" int shkz_b200_solve_csr(shkz_b200_ctx *ctx, long long n, const long long *indptr,
                                   const long long *indices, const double *data, const double *b, double *x,
                                   shkz_b200_result *res) {
  if (!ctx || !indptr || !indices || !data || !b || !x || !res || n < 0) return SHKZ_B200_ERR_ARG;
  std::memset(res, 0, sizeof(*res));
  if (n == 0) return 0;
  const long long nnz = indptr[n];
  if (n > INT32_MAX || nnz > INT32_MAX) return res->status = SHKZ_B200_ERR_LIMIT;
  const bool mic = ctx->cfg.csr_preconditioner == SHKZ_B200_PRECOND_MIC0;
  if (!mic && ctx->cfg.csr_preconditioner != SHKZ_B200_PRECOND_NONE) return res->status = SHKZ_B200_ERR_ARG;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  std::vector<int> hp((size_t)n + 1), hi((size_t)nnz);
  for (long long i = 0; i <= n; ++i) hp[i] = (int)indptr[i];
  for (long long i = 0; i < nnz; ++i) hi[i] = (int)indices[i];
  int *dp = nullptr, *di = nullptr;
  double *dd = nullptr, *vb = nullptr;
  CsrState *dst = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  auto cleanup = [&]() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (dp) cudaFree(dp);
    if (di) cudaFree(di);
    if (dd) cudaFree(dd);
    if (vb) cudaFree(vb);
    if (dst) cudaFree(dst);
  };
  // vectors: r, x, s(p), z(q), the preconditioned residual and reduction scratch
  if (cudaMalloc(&dp, sizeof(int) * (n + 1)) != cudaSuccess || cudaMalloc(&di, sizeof(int) * (nnz ? nnz : 1)) != cudaSuccess ||
      cudaMalloc(&dd, sizeof(double) * (nnz ? nnz : 1)) != cudaSuccess ||
      cudaMalloc(&vb, sizeof(double) * (5 * (size_t)n + 3 * 8192 + 8)) != cudaSuccess ||
      cudaMalloc(&dst, sizeof(CsrState)) != cudaSuccess) {
    cleanup();
    return res->status = SHKZ_B200_ERR_NOMEM;
  }
  double *r = vb, *xv = vb + n, *p = vb + 2 * n, *q = vb + 3 * n, *zv = vb + 4 * n, *part = vb + 5 * n,
         *out = part + 3 * 8192;
  unsigned *cnt = ctx->counter + 4;
  cudaMemcpyAsync(dp, hp.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(di, hi.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(dd, data, sizeof(double) * nnz, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(r, b, sizeof(double) * n, cudaMemcpyHostToDevice, s);
  cudaMemsetAsync(xv, 0, sizeof(double) * n, s);
  CsrMic0 M;
  if (ctx->cfg.spin_limit > 0) M.set_wait_limit(ctx->cfg.spin_limit);
  if (ctx->cfg.fault_skip_publish > 0) M.set_fault_skip(ctx->cfg.fault_skip_publish - 1);
  if (mic) {
    int rc = M.build((int)n, hp.data(), hi.data(), dp, di, s);
    if (!rc) rc = M.factor(dd, ctx->cfg.mic_omega, ctx->cfg.mic_min_diag_ratio, s);
    if (rc) {
      cleanup();
      return res->status = rc;
    }
  }
  // z = M^-1 r (pcg_solver.h:378-385 with the MIC(0) result kept), or z = r
  const double *z = mic ? zv : r;
  if (mic && M.apply(r, zv, s)) {
    cleanup();
    return res->status = SHKZ_B200_ERR_CUDA;
  }
  // out = {r.r, z.r, max|r|}
  double h[3];
  launch_dots64((int)n, r, r, z, r, part, cnt, out, s);
  if (cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cleanup();
    return res->status = SHKZ_B200_ERR_CUDA;
  }
  const double r0 = h[2];
  int rc = 0;
  res->iterations = 0;
  res->reresid = r0 != 0.0 ? 1.0 : 0.0;
  if (r0 != 0.0 && ctx->cfg.max_iterations > 0) {
    // pcg_solver.h:252-295 on the device: q = A p, alpha = rho / p.q,
    // x += alpha p, r -= alpha q, z = M^-1 r, stop on max|r| <= tol, else
    // beta = z.r / rho, p = z + beta p
    CsrState st{};
    st.rho = h[1];
    st.tol = ctx->cfg.residual * r0;
    st.rmax = r0;
    st.max_it = ctx->cfg.max_iterations;
    cudaMemcpyAsync(dst, &st, sizeof(st), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(p, z, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
    const int grid = (int)std::min<long long>((n + 255) / 256, 148 * 16);
    const long long counted = launches_so_far();
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      k_csr_spmv64<<<grid, 256, 0, s>>>((int)n, dp, di, dd, p, q, dst);
      count_launches(1);
      launch_csr_dots((int)n, p, q, nullptr, nullptr, part, cnt, dst, 0, s);
      launch_csr_axpy2((int)n, dst, p, xv, q, r, s);
      if (mic) M.apply(r, zv, s, &dst->done);
      launch_csr_dots((int)n, r, r, z, r, part, cnt, dst, 1, s);
      launch_csr_xpby((int)n, z, dst, p, s);
      e = cudaStreamEndCapture(s, &graph);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    // nodes of one iteration; counted again for every launch of the graph
    const long long nodes = launches_so_far() - counted;
    count_launches((int)-nodes);
    while (e == cudaSuccess) {
      for (int k = 0; k < kCsrIterationsPerCheck && e == cudaSuccess; ++k) {
        e = cudaGraphLaunch(exec, s);
        count_launches((int)nodes);
      }
      if (e == cudaSuccess) e = cudaMemcpyAsync(&st, dst, sizeof(st), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess || st.done) break;
    }
    if (e != cudaSuccess) {
      shkz_set_cuda_error(e, "csr solve graph", __FILE__, __LINE__);
      rc = SHKZ_B200_ERR_CUDA;
    } else if (st.done == 3) {
      rc = SHKZ_B200_ERR_NAN;
    }
    res->iterations = st.it;
    res->reresid = st.rmax / r0;
  }
  if (cudaMemcpyAsync(x, xv, sizeof(double) * n, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    rc = SHKZ_B200_ERR_CUDA;
  // a triangular solve's bounded wait that ran out outranks the NaN it left
  if (mic && (!rc || rc == SHKZ_B200_ERR_NAN)) {
    const int we = M.wait_error(s);
    if (we) rc = we;
  }
  cleanup();
  res->unknowns = n;
  res->outer_steps = mic ? M.levels() : 0;
  res->status = rc;
  return rc;
}

static LearnedSystem learned_system(shkz_b200_ctx *ctx);
static int learned_ready(shkz_b200_ctx *ctx);

extern "C" int shkz_b200_time_kernel(shkz_b200_ctx *ctx, int which, int reps, double *ms, long long *cells_out) {
  if (!ctx || !ms || reps <= 0) return SHKZ_B200_ERR_ARG;
  if (!ctx->has_system) return SHKZ_B200_ERR_STATE;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const PoolSystem S = pool_system(ctx);
  const int n = ctx->K * SHKZ_TC;
  SolverState init{};
  init.rho = 1.0;
  init.alpha = 1e-30;  // keeps x and r unchanged to rounding while timing the update
  init.beta = 0.0;
  init.tol_abs = -1.0;
  const int arm = arm_waves(ctx);
  if (arm) return arm;
  SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->st_scratch, &init, sizeof(init), cudaMemcpyHostToDevice, s));
  auto launch = [&]() {
    switch (which) {
      case 0: launch_spmv(S, ctx->p, ctx->q, ctx->partials, ctx->counter, ctx->st_scratch, 0, s); break;
      case 1:
      case 2: {
        // forward and backward are timed as a pair; the split uses two event pairs below
        launch_mic_apply(S, ctx->d32, ctx->r, ctx->t, ctx->z, ctx->partials, ctx->faces_f,
                         ctx->faces_b, wsync(ctx, 1), wsync(ctx, 2), nullptr, s);
        break;
      }
      case 3: launch_update_xr(n, ctx->p, ctx->q, ctx->x, ctx->r, ctx->partials, ctx->counter + 1, ctx->st_scratch,
                               1 << 30, s); break;
      case 4: launch_update_p(n, ctx->z, ctx->p, ctx->st_scratch, s); break;
      case 5: launch_label(ctx->last_in, ctx->flags, ctx->unk, ctx->tile_count, s); break;
      case 6: {
        CoeffOutputs co{ctx->diag, ctx->offx, ctx->offy, ctx->offz, ctx->diag64, ctx->offx64, ctx->offy64,
                        ctx->offz64, ctx->rhs64};
        launch_coeff(ctx->last_in, ctx->flags, ctx->pool_tile, ctx->K, ctx->unk, co, s);
        break;
      }
      case 7: launch_mic_factor(S, ctx->colsum, ctx->cfg.mic_omega, ctx->cfg.mic_min_diag_ratio, ctx->dmic64,
                                ctx->d32, ctx->wflags, wsync(ctx, 0), s); break;
      case 8: learned_apply(ctx->model, learned_system(ctx), ctx->r, 1.0, ctx->t, s); break;
      case 9:
        launch_spmv_update(S, ctx->p, ctx->pb, ctx->z, ctx->q, ctx->partials, ctx->counter, ctx->st_scratch, s);
        break;
      case 10:
        launch_mic_apply_update(S, ctx->d32, ctx->r, ctx->t, ctx->z, ctx->partials, ctx->p, ctx->pb, ctx->q, ctx->x,
                                ctx->counter + 1, ctx->st_scratch, 1 << 30, wsync(ctx, 1), wsync(ctx, 2),
                                ctx->counter + 5, s);
        break;
      default: break;
    }
  };
  if (which < 0 || which > 10) return SHKZ_B200_ERR_ARG;
  if (which >= 9 && (!ctx->pb || S.KM <= 0)) return SHKZ_B200_ERR_STATE;
  if (which == 8) {
    const int rc = learned_ready(ctx);
    if (rc) return rc;
  }
  launch();  // warm-up
  SHKZ_CUDA_TRY(cudaStreamSynchronize(s));
  // Each launch is timed alone between events, after a write of a buffer
  // larger than the 126 MB L2: a kernel whose arrays would fit in L2 (the p
  // update at 256^3 touches 69 MB) is then timed from HBM as it runs inside an
  // iteration, not from the previous repetition's cache.
  const size_t flush_bytes = (size_t)256 << 20;
  if (!ctx->flush) {
    if (cudaMalloc(&ctx->flush, flush_bytes) != cudaSuccess) {
      ctx->flush = nullptr;
      return SHKZ_B200_ERR_NOMEM;
    }
  }
  double total = 0.0;
  for (int i = 0; i < reps; ++i) {
    SHKZ_CUDA_TRY(cudaMemsetAsync(ctx->flush, i & 0xff, flush_bytes, s));
    cudaEventRecord(ctx->ev[4], s);
    launch();
    cudaEventRecord(ctx->ev[5], s);
    SHKZ_CUDA_TRY(cudaEventSynchronize(ctx->ev[5]));
    total += ms_between(ctx->ev[4], ctx->ev[5]);
  }
  *ms = total / reps;
  SHKZ_CUDA_TRY(cudaGetLastError());
  if (cells_out) *cells_out = (which == 5) ? (long long)ctx->G.nx * ctx->G.ny * ctx->G.nz : (long long)n;
  if (wave_errors(ctx)) return SHKZ_B200_ERR_TIMEOUT;
  return 0;
}

// --------------------------------------------------------------------------
// Learned preconditioner: flexible PCG and the model entry points

static LearnedSystem learned_system(shkz_b200_ctx *ctx) {
  LearnedSystem L;
  L.G = ctx->G;
  L.tile_state = ctx->tile_state;
  L.pool_tile = ctx->pool_tile;
  L.K = ctx->K;
  L.unk = ctx->unk;
  L.fluid = ctx->last_in.fluid;
  L.solid = ctx->last_in.solid;
  L.dx = ctx->last_in.dx;
  return L;
}

static int learned_ready(shkz_b200_ctx *ctx) {
  if (!ctx->model) return SHKZ_B200_ERR_STATE;
  if (!ctx->has_system) return SHKZ_B200_ERR_STATE;
  if (!ctx->model_ready) {
    int rc = learned_prepare(ctx->model, ctx->G, ctx->tile_state, ctx->stream);
    if (rc) return rc;
    ctx->model_ready = 1;
  }
  return 0;
}

// Flexible PCG (Polak-Ribiere beta) with the learned preconditioner on FP32
// vectors, FP64 reductions and reliable updates (as solve_system). When the
// residual stalls -- less than a 10 % reduction over `stall_window`
// iterations -- the solve falls back to the reference's MIC(0) for the rest
// of the solve and restarts the direction from the current residual.
static int learned_solve(shkz_b200_ctx *ctx, double tol, shkz_b200_result *res) {
  int rc = learned_ready(ctx);
  if (rc) return rc;
  cudaStream_t s = ctx->stream;
  const PoolSystem S = pool_system(ctx);
  const LearnedSystem LS = learned_system(ctx);
  const int n = ctx->K * SHKZ_TC;
  SHKZ_CUDA_TRY(cudaMemsetAsync(ctx->x64, 0, sizeof(double) * n, s));
  double h4[4];
  launch_residual64(S, ctx->rhs64, ctx->x64, ctx->r64, ctx->partials, ctx->counter + 2, ctx->out4, s);
  SHKZ_CUDA_TRY(cudaMemcpyAsync(h4, ctx->out4, sizeof(h4), cudaMemcpyDeviceToHost, s));
  SHKZ_CUDA_TRY(cudaStreamSynchronize(s));
  const double bmax = h4[2], b2 = h4[3];
  double rmax_true = h4[0], r2 = h4[1];
  res->outer_steps = 0;
  res->fallbacks = 0;
  if (bmax == 0.0) {
    res->iterations = 0;
    res->reresid = 0.0;
    res->reresid_l2 = 0.0;
    return 0;
  }
  const double scale = bmax;
  launch_inner_init(n, ctx->r64, 1.0 / scale, ctx->r, ctx->x, s);
  launch_inner_setup(n, ctx->r, ctx->partials, ctx->counter, ctx->st, tol, s);
  launch_state_resume(ctx->st, kReliableDrop, s);
  bool use_mic = false;
  auto precondition = [&](double rmax_scaled) -> int {
    if (use_mic) {
      launch_mic_apply(S, ctx->d32, ctx->r, ctx->t, ctx->z, nullptr, ctx->faces_f, ctx->faces_b, wsync(ctx, 1),
                       wsync(ctx, 2), ctx->st, s);
      return 0;
    }
    return learned_apply(ctx->model, LS, ctx->r, rmax_scaled, ctx->z, s);
  };
  if ((rc = precondition(1.0))) return rc;
  launch_fpcg_dots(n, ctx->z, ctx->r, ctx->q, ctx->partials, ctx->counter + 5, ctx->st, 1 | 2, s);
  SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->p, ctx->z, sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
  const int max_it = ctx->cfg.max_iterations;
  const int W = ctx->cfg.stall_window > 0 ? ctx->cfg.stall_window : 8;
  std::vector<double> hist;
  SolverState hst;
  int updates = 0;
  bool true_checked = false;
  for (;;) {
    launch_spmv(S, ctx->p, ctx->q, ctx->partials, ctx->counter, ctx->st, 0, s);
    launch_update_xr(n, ctx->p, ctx->q, ctx->x, ctx->r, ctx->partials, ctx->counter + 1, ctx->st, max_it, s);
    SHKZ_CUDA_TRY(cudaMemcpyAsync(&hst, ctx->st, sizeof(hst), cudaMemcpyDeviceToHost, s));
    SHKZ_CUDA_TRY(cudaStreamSynchronize(s));
    if (use_mic && wave_errors(ctx)) { rc = SHKZ_B200_ERR_TIMEOUT; break; }
    if (hst.done == 5) {
      // the learned z broke down (z.r <= 0 or not finite): x and r are those of
      // the last completed iteration; continue with MIC(0) from r
      use_mic = true;
      res->fallbacks += 1;
      launch_state_resume(ctx->st, hst.ru_threshold, s);
      if ((rc = precondition(hst.rmax))) break;
      launch_fpcg_dots(n, ctx->z, ctx->r, ctx->q, ctx->partials, ctx->counter + 5, ctx->st, 1, s);
      SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->p, ctx->z, sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
      continue;
    }
    if (hst.done == 3 || hst.status == -5) { rc = SHKZ_B200_ERR_NAN; break; }
    if (hst.done == 2) break;
    true_checked = false;
    double rmax = hst.rmax;
    if (hst.done == 1 || hst.done == 4) {
      launch_accumulate(n, ctx->x, scale, ctx->x64, s);
      launch_residual64(S, ctx->rhs64, ctx->x64, ctx->r64, ctx->partials, ctx->counter + 2, ctx->out4, s);
      SHKZ_CUDA_TRY(cudaMemcpyAsync(h4, ctx->out4, sizeof(h4), cudaMemcpyDeviceToHost, s));
      SHKZ_CUDA_TRY(cudaStreamSynchronize(s));
      rmax_true = h4[0];
      r2 = h4[1];
      ++updates;
      true_checked = true;
      if (!(rmax_true == rmax_true)) { rc = SHKZ_B200_ERR_NAN; break; }
      if (rmax_true <= tol * bmax) break;
      launch_inner_init(n, ctx->r64, 1.0 / scale, ctx->r, ctx->x, s);
      launch_state_resume(ctx->st, kReliableDrop * rmax_true / scale, s);
      rmax = rmax_true / scale;
    }
    hist.push_back(rmax);
    const int k = (int)hist.size() - 1;
    bool restart = false;
    if (!use_mic && k >= W && rmax > 0.9 * hist[k - W]) {
      use_mic = true;  // stall: fall back to MIC(0)
      res->fallbacks += 1;
      restart = true;
    }
    if ((rc = precondition(rmax))) break;
    launch_fpcg_dots(n, ctx->z, ctx->r, ctx->q, ctx->partials, ctx->counter + 5, ctx->st,
                     (restart ? 1 : 0) | (use_mic ? 0 : 2), s);
    if (restart) SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->p, ctx->z, sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
    else launch_update_p(n, ctx->z, ctx->p, ctx->st, s);
  }
  if (!true_checked && rc == 0) {
    launch_accumulate(n, ctx->x, scale, ctx->x64, s);
    launch_residual64(S, ctx->rhs64, ctx->x64, ctx->r64, ctx->partials, ctx->counter + 2, ctx->out4, s);
    SHKZ_CUDA_TRY(cudaMemcpyAsync(h4, ctx->out4, sizeof(h4), cudaMemcpyDeviceToHost, s));
    SHKZ_CUDA_TRY(cudaStreamSynchronize(s));
    rmax_true = h4[0];
    r2 = h4[1];
  }
  if (!rc && learned_error(ctx->model)) rc = SHKZ_B200_ERR_TIMEOUT;
  if (!rc && wave_errors(ctx)) rc = SHKZ_B200_ERR_TIMEOUT;
  res->iterations = hst.iter;
  res->outer_steps = updates;
  res->reresid = rmax_true / bmax;
  res->reresid_l2 = std::sqrt(r2 / b2);
  return rc;
}

extern "C" int shkz_b200_set_target_volume(shkz_b200_ctx *ctx, double current_volume, double target_volume) {
  if (!ctx) return SHKZ_B200_ERR_ARG;
  ctx->vol_current = current_volume;
  ctx->vol_target = target_volume;
  return 0;
}

extern "C" int shkz_b200_get_volume_state(shkz_b200_ctx *ctx, double state[3]) {
  if (!ctx || !state) return SHKZ_B200_ERR_ARG;
  state[0] = ctx->vol_target;
  state[1] = ctx->vol_current;
  state[2] = ctx->vol_yprev;
  return 0;
}

extern "C" int shkz_b200_set_volume_state(shkz_b200_ctx *ctx, const double state[3]) {
  if (!ctx || !state) return SHKZ_B200_ERR_ARG;
  ctx->vol_target = state[0];
  ctx->vol_current = state[1];
  ctx->vol_yprev = state[2];
  return 0;
}

extern "C" long long shkz_b200_warm_start_size(shkz_b200_ctx *ctx) { return ctx ? ctx->prev_n : -1; }

extern "C" int shkz_b200_get_warm_start(shkz_b200_ctx *ctx, double *out, size_t n) {
  if (!ctx || (n && !out) || (long long)n != ctx->prev_n) return SHKZ_B200_ERR_ARG;
  if (n == 0) return 0;
  cudaSetDevice(ctx->device);
  SHKZ_CUDA_TRY(cudaMemcpyAsync(out, ctx->prev, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  SHKZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return 0;
}

extern "C" int shkz_b200_set_warm_start(shkz_b200_ctx *ctx, const double *in, size_t n) {
  if (!ctx || (n && !in)) return SHKZ_B200_ERR_ARG;
  cudaSetDevice(ctx->device);
  if ((long long)n > ctx->cap_prev) {
    const long long cap = (long long)n + 1024;
    double *np = nullptr;
    cudaError_t e = cudaMalloc(&np, sizeof(double) * (size_t)cap);
    if (e != cudaSuccess) {
      shkz_set_cuda_error(e, "cudaMalloc", __FILE__, __LINE__);
      return SHKZ_B200_ERR_NOMEM;
    }
    SHKZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (ctx->prev) cudaFree(ctx->prev);
    ctx->prev = np;
    ctx->cap_prev = cap;
  }
  if (n) SHKZ_CUDA_TRY(cudaMemcpyAsync(ctx->prev, in, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  SHKZ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  ctx->prev_n = (long long)n;
  return 0;
}

extern "C" int shkz_b200_learned_init(shkz_b200_ctx *ctx, unsigned seed) {
  if (!ctx) return SHKZ_B200_ERR_ARG;
  cudaSetDevice(ctx->device);
  if (!ctx->model) {
    ctx->model = learned_create(ctx->device);
    if (!ctx->model) return SHKZ_B200_ERR_NOMEM;
  }
  ctx->model_ready = 0;
  return learned_init_params(ctx->model, seed, ctx->stream);
}

extern "C" double shkz_b200_learned_flops(shkz_b200_ctx *ctx) {
  if (!ctx || !ctx->model) return -1.0;
  if (learned_ready(ctx)) return -1.0;
  return learned_forward_flops(ctx->model);
}

extern "C" long long shkz_b200_learned_param_count(shkz_b200_ctx *ctx) {
  return (ctx && ctx->model) ? (long long)learned_param_count(ctx->model) : -1;
}

extern "C" int shkz_b200_learned_set_params(shkz_b200_ctx *ctx, const float *blob, size_t n) {
  if (!ctx || !blob) return SHKZ_B200_ERR_ARG;
  if (!ctx->model) return SHKZ_B200_ERR_STATE;
  cudaSetDevice(ctx->device);
  return learned_set_params(ctx->model, blob, n, ctx->stream);
}

extern "C" int shkz_b200_learned_get_params(shkz_b200_ctx *ctx, float *blob, size_t n, int gradients) {
  if (!ctx || !blob) return SHKZ_B200_ERR_ARG;
  if (!ctx->model) return SHKZ_B200_ERR_STATE;
  cudaSetDevice(ctx->device);
  return learned_get_params(ctx->model, blob, n, gradients, ctx->stream);
}

// z = s N(r/s) at unknown cells for a dense host residual (FP32 cells).
extern "C" int shkz_b200_learned_apply(shkz_b200_ctx *ctx, const float *r_cells, float *z_cells) {
  if (!ctx || !r_cells || !z_cells) return SHKZ_B200_ERR_ARG;
  cudaSetDevice(ctx->device);
  int rc = learned_ready(ctx);
  if (rc) return rc;
  cudaStream_t s = ctx->stream;
  const Geometry &G = ctx->G;
  const size_t cells = (size_t)G.nx * G.ny * G.nz;
  double rmax = 0.0;
  for (size_t i = 0; i < cells; ++i) rmax = std::fmax(rmax, std::fabs((double)r_cells[i]));
  float *dense = nullptr;
  SHKZ_CUDA_TRY(cudaMalloc(&dense, cells * 4));
  cudaMemcpyAsync(dense, r_cells, cells * 4, cudaMemcpyHostToDevice, s);
  if (ctx->K > 0) {
    count_launches(1);
    k_dense_to_pool_f32<<<148 * 8, 256, 0, s>>>(G, ctx->pool_tile, ctx->K, dense, ctx->r);
    rc = learned_apply(ctx->model, learned_system(ctx), ctx->r, rmax, ctx->z, s);
    count_launches(1);
    k_pool_to_dense_f32<<<148 * 8, 256, 0, s>>>(G, ctx->tile_state, ctx->z, dense);
  }
  cudaError_t e = cudaMemcpyAsync(z_cells, dense, cells * 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(dense);
  if (e != cudaSuccess) {
    shkz_set_cuda_error(e, "learned_apply", __FILE__, __LINE__);
    return SHKZ_B200_ERR_CUDA;
  }
  if (!rc) rc = learned_error(ctx->model);
  return rc;
}

// Dense level-0 network dimensions (grid rounded up to multiples of 4).
extern "C" int shkz_b200_learned_dims(shkz_b200_ctx *ctx, int *dims) {
  if (!ctx || !dims) return SHKZ_B200_ERR_ARG;
  int rc = learned_ready(ctx);
  if (rc) return rc;
  learned_dense_dims(ctx->model, &dims[0], &dims[1], &dims[2]);
  return 0;
}

// Inspection of the last network application: which = 0 .. 12 are the
// stored activations X0, A1, S1, P1, A2, S2, P2, A3, B3, C2, D2, C1, D1
// (dense channels-last FP32, shape4 = z, y, x, channels); which = 13 is the
// raw FP32 output Z of the last layer (channels = 1); 14 .. 26 are the
// FP32 gradients w.r.t. tensors 0 .. 12 after the last backward pass.
extern "C" int shkz_b200_learned_tensor(shkz_b200_ctx *ctx, int which, float *out, size_t count, int *shape4) {
  if (!ctx || which < 0 || which > 26) return SHKZ_B200_ERR_ARG;
  int rc = learned_ready(ctx);
  if (rc) return rc;
  cudaStream_t s = ctx->stream;
  size_t need;
  int shp[4];
  if (which == 13) {
    learned_tensor_shape(ctx->model, 0, shp);
    shp[3] = 1;
    need = learned_dense_cells(ctx->model);
  } else {
    learned_tensor_shape(ctx->model, which % 14, shp);
    need = learned_tensor_size(ctx->model, which % 14);
  }
  if (shape4) std::memcpy(shape4, shp, sizeof(shp));
  if (!out) return 0;
  if (count < need) return SHKZ_B200_ERR_ARG;
  float *d = nullptr;
  SHKZ_CUDA_TRY(cudaMalloc(&d, need * 4));
  rc = which == 13 ? learned_output_dense(ctx->model, d, s)
                   : (which > 13 ? learned_grad_dense(ctx->model, which - 14, d, s)
                                 : learned_tensor_dense(ctx->model, which, d, s));
  cudaError_t e = cudaMemcpyAsync(out, d, need * 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(d);
  if (e != cudaSuccess) return SHKZ_B200_ERR_CUDA;
  return rc;
}

// Weight gradients of sum(gZ * Z) for the last application (gZ dense level-0 FP32, host).
extern "C" int shkz_b200_learned_backward(shkz_b200_ctx *ctx, const float *gZ_dense, size_t count) {
  if (!ctx || !gZ_dense) return SHKZ_B200_ERR_ARG;
  int rc = learned_ready(ctx);
  if (rc) return rc;
  cudaStream_t s = ctx->stream;
  const size_t nv = learned_dense_cells(ctx->model);
  if (count < nv) return SHKZ_B200_ERR_ARG;
  float *d = nullptr;
  SHKZ_CUDA_TRY(cudaMalloc(&d, nv * 4));
  cudaMemcpyAsync(d, gZ_dense, nv * 4, cudaMemcpyHostToDevice, s);
  rc = learned_backward_dense(ctx->model, d, s);
  cudaError_t e = cudaStreamSynchronize(s);
  cudaFree(d);
  if (e != cudaSuccess) return SHKZ_B200_ERR_CUDA;
  if (!rc) rc = learned_error(ctx->model);
  return rc;
}

// Training on the last projection's system: step i uses a residual that is
// the right-hand side (i % 3 == 0), A e for white noise e (i % 3 == 1), or
// b + A e (i % 3 == 2), scaled to ||r||inf = 1; energy loss, Adam(lr).
extern "C" int shkz_b200_learned_train(shkz_b200_ctx *ctx, int steps, double lr, unsigned seed, double *losses) {
  if (!ctx || steps < 0) return SHKZ_B200_ERR_ARG;
  cudaSetDevice(ctx->device);
  int rc = learned_ready(ctx);
  if (rc) return rc;
  if (ctx->K == 0) return 0;
  cudaStream_t s = ctx->stream;
  const PoolSystem S = pool_system(ctx);
  const LearnedSystem LS = learned_system(ctx);
  const int n = ctx->K * SHKZ_TC;
  if (!ctx->mic_ready) {
    launch_mic_factor(S, ctx->colsum, ctx->cfg.mic_omega, ctx->cfg.mic_min_diag_ratio, ctx->dmic64, ctx->d32,
                      ctx->wflags, wsync(ctx, 0), s);
    ctx->mic_ready = 1;
  }
  const int np = mic_partial_count(S);
  std::vector<double> hp((size_t)np);
  for (int i = 0; i < steps; ++i) {
    const int kind = i % 3;
    // r (FP32 pool) in ctx->r; scratch: ctx->t (noise), ctx->q (A e)
    if (kind != 1) launch_to_float(n, ctx->rhs64, ctx->r, s);
    else SHKZ_CUDA_TRY(cudaMemsetAsync(ctx->r, 0, sizeof(float) * n, s));
    if (kind != 0) {
      launch_rand_unknowns(n, ctx->diag, seed * 7919u + (unsigned)i, ctx->t, s);
      launch_spmv(S, ctx->t, ctx->q, ctx->partials, ctx->counter, nullptr, 1, s);
      // balance the two parts by their sizes
      launch_inner_setup(n, ctx->q, ctx->partials, ctx->counter, ctx->st_scratch, 1.0, s);
      SolverState a1;
      cudaMemcpyAsync(&a1, ctx->st_scratch, sizeof(a1), cudaMemcpyDeviceToHost, s);
      launch_inner_setup(n, ctx->r, ctx->partials, ctx->counter, ctx->st_scratch, 1.0, s);
      SolverState a2;
      cudaMemcpyAsync(&a2, ctx->st_scratch, sizeof(a2), cudaMemcpyDeviceToHost, s);
      SHKZ_CUDA_TRY(cudaStreamSynchronize(s));
      const float w = (kind == 1 || a1.rmax0 == 0.0) ? 1.0f : (float)(a2.rmax0 / a1.rmax0);
      launch_axpby_f32(n, w, ctx->q, 1.0f, ctx->r, s);
    }
    launch_inner_setup(n, ctx->r, ctx->partials, ctx->counter, ctx->st_scratch, 1.0, s);
    SolverState a3;
    SHKZ_CUDA_TRY(cudaMemcpyAsync(&a3, ctx->st_scratch, sizeof(a3), cudaMemcpyDeviceToHost, s));
    SHKZ_CUDA_TRY(cudaStreamSynchronize(s));
    if (a3.rmax0 > 0) launch_scale_f32(n, ctx->r, (float)(1.0 / a3.rmax0), s);
    // loss scale: the MIC(0) energy 1/2 r.M^-1 r estimates 1/2 r.A^-1 r, so the
    // normalised loss is near -1 at the optimum whatever the system and residual
    launch_mic_apply(S, ctx->d32, ctx->r, ctx->t, ctx->z, ctx->partials, ctx->faces_f, ctx->faces_b, wsync(ctx, 1),
                     wsync(ctx, 2), nullptr, s);
    SHKZ_CUDA_TRY(cudaMemcpyAsync(hp.data(), ctx->partials, sizeof(double) * np, cudaMemcpyDeviceToHost, s));
    SHKZ_CUDA_TRY(cudaStreamSynchronize(s));
    double rz = 0.0;
    for (double v : hp) rz += v;
    const double gscale = (rz > 0.0 && rz < 1e300) ? 2.0 / rz : 1.0;
    double loss = 0.0;
    rc = learned_train_step(ctx->model, LS, S, ctx->r, ctx->z, ctx->q, ctx->partials, ctx->counter, (float)lr,
                            gscale, &loss, s);
    if (rc) return rc;
    if (losses) losses[i] = loss;
  }
  return 0;
}

extern "C" int shkz_b200_learned_save(shkz_b200_ctx *ctx, const char *path) {
  if (!ctx || !path) return SHKZ_B200_ERR_ARG;
  if (!ctx->model) return SHKZ_B200_ERR_STATE;
  const size_t n = learned_param_count(ctx->model);
  std::vector<float> blob(n);
  int rc = learned_get_params(ctx->model, blob.data(), n, 0, ctx->stream);
  if (rc) return rc;
  FILE *f = std::fopen(path, "wb");
  if (!f) return SHKZ_B200_ERR_ARG;
  const unsigned long long nn = n;
  std::fwrite("SHKZNET1", 1, 8, f);
  std::fwrite(&nn, 8, 1, f);
  std::fwrite(blob.data(), 4, n, f);
  std::fclose(f);
  return 0;
}

extern "C" int shkz_b200_learned_load(shkz_b200_ctx *ctx, const char *path) {
  if (!ctx || !path) return SHKZ_B200_ERR_ARG;
  cudaSetDevice(ctx->device);
  if (!ctx->model) {
    ctx->model = learned_create(ctx->device);
    if (!ctx->model) return SHKZ_B200_ERR_NOMEM;
  }
  FILE *f = std::fopen(path, "rb");
  if (!f) return SHKZ_B200_ERR_ARG;
  char magic[8];
  unsigned long long nn = 0;
  const bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "SHKZNET1", 8) == 0 &&
                  std::fread(&nn, 8, 1, f) == 1 && nn == learned_param_count(ctx->model);
  if (!ok) {
    std::fclose(f);
    return SHKZ_B200_ERR_ARG;
  }
  std::vector<float> blob(nn);
  const size_t got = std::fread(blob.data(), 4, nn, f);
  std::fclose(f);
  if (got != nn) return SHKZ_B200_ERR_ARG;
  ctx->model_ready = 0;
  return learned_set_params(ctx->model, blob.data(), nn, ctx->stream);
}

// One 3^3 convolution on the tensor cores with host arrays (unit tests of the
// kernel): in0 (nz,ny,nx,c0), in1 (nz/2,ny/2,nx/2,c1) nearest-upsampled and
// concatenated, w[27][cout][c0+c1], bias[cout] (may be NULL); out (nz,ny,nx,cout),
// BF16-rounded values as FP32.
extern "C" int shkz_b200_conv3d(int nx, int ny, int nz, int c0, int c1, int cout, int planes, const float *in0,
                                const float *in1, const float *w, const float *bias, int relu, float *out) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || c0 <= 0 || c0 % 16 || c1 < 0 || c1 % 16 || cout <= 0 || cout > 128 ||
      (planes != 4 && planes != 8) || !in0 || !w || !out || (c1 && !in1) || (nx | ny | nz) & 1)
    return SHKZ_B200_ERR_ARG;
  // the kernel runs with cout padded to a power of two (at least 16); one
  // CTA's accumulators take planes x that (each plane on a 32-column
  // boundary) of the SM's 512 tensor-memory columns
  int n_pad = 16;
  while (n_pad < cout) n_pad <<= 1;
  if (planes * ((n_pad + 31) & ~31) > 512) return SHKZ_B200_ERR_LIMIT;
  return conv3d_run(nx, ny, nz, c0, c1, cout, planes, in0, in1, w, bias, relu, out);
}
