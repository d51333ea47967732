/*
 * shkz_b200.h -- C ABI of the B200 MAC pressure projection.
 *
 * This is the boundary between host code written against Shiokaze's module
 * API and the sm_100a CUDA implementation. Signatures use plain pointers and
 * sizes only; no CUDA, C++ or torch types cross it. Every function returns
 * 0 on success or a negative SHKZ_B200_ERR_* code, never throws and never
 * exits the process.
 *
 * Reference interfaces replaced (paths relative to the Shiokaze tree):
 *   shkz_b200_project*   macproject3_interface::project
 *                        (include/shiokaze/projection/macproject3_interface.h:84-91),
 *                        implemented by macpressuresolver3::project
 *                        (src/projection/macpressuresolver3.cpp:54-299)
 *   shkz_b200_solve_csr  RCMatrix_solver_interface<size_t,double>::solve
 *                        (include/shiokaze/linsolver/RCMatrix_solver.h:44-77),
 *                        implemented by pcg_solver::solve
 *                        (src/linsolver/pcg.cpp:45-73)
 *   shkz_b200_config     the configuration keys those modules read:
 *                        Residual, MaxIterations, ModifiedIC, MinDiagRatio
 *                        (src/linsolver/pcg.cpp:39-44), EpsFluid, EpsSolid
 *                        (src/utility/macutility3.cpp:503-504),
 *                        SecondOrderAccurateFluid/Solid
 *                        (src/projection/macpressuresolver3.cpp:301-307)
 *
 * Grid conventions (same as the reference array3/macarray3 index space):
 *   cells      nx*ny*nz, index i + nx*(j + ny*k)
 *   nodes      (nx+1)*(ny+1)*(nz+1)            (solid level set)
 *   faces dim0 (nx+1)*ny*nz, dim1 nx*(ny+1)*nz, dim2 nx*ny*(nz+1)
 * Level-set and velocity inputs are the values array3::operator() returns
 * for every cell (active value, fill value or background), plus one byte per
 * cell that is 1 where the reference grid holds an active value.
 */
#ifndef SHKZ_B200_H
#define SHKZ_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SHKZ_B200_ABI_VERSION 1

enum {
  SHKZ_B200_OK = 0,
  SHKZ_B200_ERR_ARG = -1,        /* bad argument (null pointer, size) */
  SHKZ_B200_ERR_CUDA = -2,       /* CUDA runtime error; see shkz_b200_last_error */
  SHKZ_B200_ERR_NOMEM = -3,      /* device allocation failed */
  SHKZ_B200_ERR_TIMEOUT = -4,    /* a bounded device wait gave up */
  SHKZ_B200_ERR_NAN = -5,        /* NaN in the system or the iterates */
  SHKZ_B200_ERR_NODEVICE = -6,   /* no usable sm_100 device */
  SHKZ_B200_ERR_STATE = -7,      /* call order (e.g. no model loaded) */
  SHKZ_B200_ERR_LIMIT = -8       /* size beyond a documented limit */
};

/* Preconditioner choice. NONE is what the shipped reference runs (its
 * MIC(0) result is discarded, local/include/pcgsolver/pcg_solver.h:379-384);
 * MIC0 applies the reference's own MIC(0) factor (pcg_solver.h:88-223);
 * LEARNED is the conv-net preconditioner inside flexible PCG with MIC(0)
 * fallback. */
enum { SHKZ_B200_PRECOND_NONE = 0, SHKZ_B200_PRECOND_MIC0 = 1, SHKZ_B200_PRECOND_LEARNED = 2 };

typedef struct shkz_b200_config {
  double residual;            /* Residual (default 1e-4): stop at ||r||inf <= residual*||b||inf */
  int max_iterations;         /* MaxIterations (default 30000) */
  int preconditioner;         /* SHKZ_B200_PRECOND_* (default MIC0) */
  double mic_omega;           /* ModifiedIC (default 0.97) */
  double mic_min_diag_ratio;  /* MinDiagRatio (default 0.25) */
  double eps_fluid;           /* EpsFluid (default 1e-2) */
  double eps_solid;           /* EpsSolid (default 1e-2) */
  int second_order_fluid;     /* SecondOrderAccurateFluid (default 1) */
  int second_order_solid;     /* SecondOrderAccurateSolid (default 1) */
  int refine;                 /* FP64 outer refinement of the FP32 solve (default 1) */
  int fp64_reference;         /* also run an FP64 tight solve and report the error (default 0) */
  double fp64_tol;            /* tolerance of that solve (default 1e-12) */
  int check_interval;         /* iterations per device-side batch between host checks (default 16) */
  int stall_window;           /* learned FPCG: iterations without progress before MIC(0) fallback */
  int device;                 /* CUDA device ordinal (default 0) */
  int mic_block;              /* MIC(0) sweep block edge: 16 (default, 2x2x2 tiles per CTA) or 8 */
  double gain;                /* Gain of the volume correction (default 1.0) */
  int warm_start;             /* WarmStart (default 0) */
  int index_tile;             /* tile edge of the caller's grids (TileSize, default 16): unknown numbering of
                                 the warm-start vector */
  int spin_limit;             /* polling rounds of every bounded device wait (tile faces and flags of the MIC(0)
                                 wavefronts, row values of shkz_b200_solve_csr's MIC(0) triangular solves) before
                                 it gives up and the call returns SHKZ_B200_ERR_TIMEOUT; 0 = the default, 2^21
                                 (about 0.15 s) for the wavefronts, 2^22 for the CSR solves */
  int fault_skip_publish;     /* fault injection, 0 = off: k > 0 makes the forward MIC(0) sweep's k-th wavefront
                                 slot skip publishing its faces (and, in shkz_b200_solve_csr, the forward
                                 triangular solve's k-th row in level order skip storing its value), so the
                                 bounded waits on it run out */
  int device_mem_limit_mb;    /* cap on the device memory of the context's grid and tile-pool buffers, in MiB;
                                 a call that would exceed it returns SHKZ_B200_ERR_NOMEM (0 = no cap) */
  int csr_preconditioner;     /* shkz_b200_solve_csr: SHKZ_B200_PRECOND_NONE (default: what the shipped pcg
                                 runs) or SHKZ_B200_PRECOND_MIC0 (the header's MIC(0) applied) */
} shkz_b200_config;

/* Fill *cfg with the defaults listed above. */
void shkz_b200_default_config(shkz_b200_config *cfg);

typedef struct shkz_b200_ctx shkz_b200_ctx;

int shkz_b200_create(shkz_b200_ctx **out, const shkz_b200_config *cfg);
void shkz_b200_destroy(shkz_b200_ctx *ctx);
int shkz_b200_set_config(shkz_b200_ctx *ctx, const shkz_b200_config *cfg);
const char *shkz_b200_errstr(int code);
/* Text of the last CUDA error seen by this thread's context, or "". */
const char *shkz_b200_last_error(shkz_b200_ctx *ctx);

/* Arguments of one projection: project(dt, velocity, solid, solid_velocity,
 * fluid) of macproject3_interface. All arrays are either all host pointers
 * (shkz_b200_project_host) or all device pointers (shkz_b200_project_device).
 * solid / solid_active may be NULL for "no solid level set" (the reference's
 * solid cleared to 1); solid_velocity may be NULL for zero solid velocity.
 * velocity[] and velocity_active[] are updated in place; pressure (cells) and
 * pressure_active (cells, 1 where an unknown was solved) are written. */
typedef struct shkz_b200_project_args {
  int nx, ny, nz;
  double dx, dt;
  const float *fluid;                  /* cells */
  const uint8_t *fluid_active;         /* cells */
  const float *solid;                  /* nodes, may be NULL */
  const uint8_t *solid_active;         /* nodes, may be NULL */
  float *velocity[3];                  /* faces, in/out */
  uint8_t *velocity_active[3];         /* faces, in/out */
  const float *solid_velocity[3];      /* faces, each may be NULL */
  float *pressure;                     /* cells, out, may be NULL */
  uint8_t *pressure_active;            /* cells, out, may be NULL */
  double surface_tension;              /* surface_tension argument of project(); 0 = none */
  const float *solid_density[3];       /* faces (set_solid_density), all NULL = none */
} shkz_b200_project_args;

typedef struct shkz_b200_result {
  int status;                /* 0 or SHKZ_B200_ERR_* */
  int iterations;            /* total inner PCG iterations (reference: Result.count) */
  int outer_steps;           /* FP64 refinement passes */
  int fallbacks;             /* learned FPCG -> MIC(0) fallbacks */
  long long unknowns;        /* number of pressure unknowns */
  long long tiles;           /* tiles in the pool (8^3 tiles with >= 1 unknown) */
  double reresid;            /* true ||r||inf/||b||inf after the solve (reference: Result.reresid) */
  double reresid_l2;         /* true ||r||2/||b||2 */
  double err_fp64_inf;       /* ||x - x_fp64||inf/||x_fp64||inf when fp64_reference, else -1 */
  double fp64_reresid;       /* reached residual of the FP64 tight solve, else -1 */
  double ms_assemble;        /* device time per phase (CUDA events) */
  double ms_solve;
  double ms_update;
  double ms_total;
  double ms_h2d, ms_d2h;     /* host paths only */
  long long kernel_launches; /* CUDA kernels this library launched for the call */
  double volume_rhs_correct; /* volume correction added to every rhs row (record _volume_correct_rhs), else 0 */
  /* sub-phases of ms_assemble, under the reference's record names
   * (macpressuresolver3.cpp:95,168,218): face fractions and the unknown mask
   * (one kernel; solid_fluid_fractions), the unknown numbering by tile-pool
   * compaction (labelling_cells), the system's weights and rhs
   * (build_highres_linsystem, with the volume correction inside) */
  double ms_fractions;
  double ms_labelling;
  double ms_build;
  double reserved[3];
} shkz_b200_result;

/* macproject3_interface::set_target_volume (macpressuresolver3.cpp:46-49):
 * with Gain != 0 and a non-zero target, each projection adds the PI volume
 * correction of macpressuresolver3.cpp:219-234 to every rhs row. */
int shkz_b200_set_target_volume(shkz_b200_ctx *ctx, double current_volume, double target_volume);
/* Volume-correction state {target_volume, current_volume, y_prev} as the
 * reference serialises it (macpressuresolver3.cpp:320-342); post_initialize
 * clears it. */
int shkz_b200_get_volume_state(shkz_b200_ctx *ctx, double state[3]);
int shkz_b200_set_volume_state(shkz_b200_ctx *ctx, const double state[3]);
/* Warm-start vector (WarmStart=Yes): the previous solution indexed by the
 * reference's unknown number, as m_prev_pressure holds it. size returns its
 * length (0 before the first warm-started projection). */
long long shkz_b200_warm_start_size(shkz_b200_ctx *ctx);
int shkz_b200_get_warm_start(shkz_b200_ctx *ctx, double *out, size_t n);
int shkz_b200_set_warm_start(shkz_b200_ctx *ctx, const double *in, size_t n);

/* One pressure projection with host buffers: uploads, assembles, solves,
 * updates the velocities and downloads. Host arrays may be pageable; pinned
 * memory copies faster. */
int shkz_b200_project_host(shkz_b200_ctx *ctx, const shkz_b200_project_args *args, shkz_b200_result *out);

/* Same, with every array already resident on the context's device. */
int shkz_b200_project_device(shkz_b200_ctx *ctx, const shkz_b200_project_args *args, shkz_b200_result *out);

/* Velocity extension after a projection: what the liquid solver does right
 * after project() (macliquid3::extend_both, src/liquid/macliquid3.cpp:330-340)
 * -- `width` passes of macarray_extrapolator3::extrapolate
 * (include/shiokaze/array/macarray_extrapolator3.h: each inactive face next
 * to an active one takes the mean of its active neighbours and becomes
 * active), then, when constrain != 0, macutility3::constrain_velocity
 * (src/utility/macutility3.cpp:61-92: no flow into the solid at faces inside
 * it, none out through the domain's floor and ceiling). Same grid layouts as
 * shkz_b200_project_args; solid / solid_active (nodes) may be NULL for no
 * solid. Results are bit-identical to the reference's. nx, ny, nz >= 2,
 * 0 <= width <= 4096. */
typedef struct shkz_b200_extend_args {
  int nx, ny, nz;
  double dx;
  int width;                      /* extrapolation passes */
  int constrain;                  /* 1: constrain_velocity after the passes */
  const float *solid;             /* nodes, may be NULL */
  const uint8_t *solid_active;    /* nodes, may be NULL */
  float *velocity[3];             /* faces, in/out */
  uint8_t *velocity_active[3];    /* faces, in/out */
} shkz_b200_extend_args;

/* Host buffers (copied to the device and back). */
int shkz_b200_extend_velocity_host(shkz_b200_ctx *ctx, const shkz_b200_extend_args *args);

/* Device pointers on the context's device, e.g. the arrays just passed to
 * shkz_b200_project_device: the velocity stays on the GPU between the
 * projection and its extension. The masks and the solid arrays must start on
 * 16-byte boundaries (cudaMalloc's are), else SHKZ_B200_ERR_ARG. */
int shkz_b200_extend_velocity_device(shkz_b200_ctx *ctx, const shkz_b200_extend_args *args);

/* FLIP splat before the projection: what the FLIP liquid solver does right
 * before project() (macflipliquid3, src/liquid/macflipliquid3.cpp:135-151):
 * macnbflip3::splat (src/flip/macnbflip3.cpp:103-148) -- every face within
 * reach of a splatting particle gets the tent-weighted sums of particle mass
 * and momentum (the APIC term c[d].(x_face - p) included), gathered over the
 * particles' edge hash (pointgridhash3, src/pointgridhash/pointgridhash3.cpp:
 * 90-100, 218-231) -- and then the combined grid velocity on every face with
 * non-zero mass: u = (g u + momentum) / (g + mass), g = max(0, 1 - mass) on
 * faces the velocity held active, else 0; the face becomes active.
 * Results are bit-identical to the reference's.
 *
 * Particles are `count` records of `stride` bytes, read in place: a maintainer
 * passes macnbflip3's own particle vector with stride sizeof(Particle) and the
 * offsetof() of its fields. The float fields (p[3], velocity[3], mass,
 * c[3][3]) must lie at offsets that are multiples of 4 with stride a multiple
 * of 4; offset_apic = -1 turns APIC off (macnbflip3's APIC=No);
 * offset_bullet = -1 means no bullet flags. Bullet particles splat only when
 * splat_bullet != 0 (SplatBulletParticle). Face grids use the layouts of
 * shkz_b200_project_args. mass, momentum and splat_active are optional outputs
 * (all three or none): the splat grid itself, zero and inactive where the
 * splatted mass is zero. velocity and velocity_active may be NULL (all of
 * them) when the splat grid is asked for: the splat alone, as
 * macflip3_interface::splat returns it, without the combined velocity. nx, ny, nz >= 1; the three axes' edge grids together
 * and 3 * count stay below 2^31. An edge bucket (the particles whose
 * positions round to one edge cell; about 8 to 12 in a FLIP simulation) of
 * more than 4096 particles returns SHKZ_B200_ERR_LIMIT with the grids left
 * as they were. */
typedef struct shkz_b200_splat_args {
  int nx, ny, nz;
  double dx;
  long long count;                /* particles */
  const void *particles;          /* count records of stride bytes */
  int stride;
  int offset_position;            /* float[3] */
  int offset_velocity;            /* float[3] */
  int offset_mass;                /* float */
  int offset_apic;                /* float[3][3], row d = c[d]; -1: APIC off */
  int offset_bullet;              /* uint8 (nonzero = bullet); -1: none */
  int splat_bullet;
  float *velocity[3];             /* faces, in/out, optional (see above) */
  uint8_t *velocity_active[3];    /* faces, in/out, optional */
  float *mass[3];                 /* faces, out, optional */
  float *momentum[3];             /* faces, out, optional */
  uint8_t *splat_active[3];       /* faces, out, optional */
} shkz_b200_splat_args;

/* Host buffers (particle records and grids copied to the device and back). */
int shkz_b200_splat_host(shkz_b200_ctx *ctx, const shkz_b200_splat_args *args);

/* Device pointers on the context's device (the particle records and the
 * float face grids 4-byte aligned, else SHKZ_B200_ERR_ARG): the grid velocity
 * can go straight on to shkz_b200_project_device. */
int shkz_b200_splat_device(shkz_b200_ctx *ctx, const shkz_b200_splat_args *args);

/* The CUDA stream the context launches on (as an opaque pointer), so callers
 * can order their own work against it. */
void *shkz_b200_stream(shkz_b200_ctx *ctx);

/* Page-locked host memory for the buffers of the host-buffer entry points:
 * the host<->device copies of shkz_b200_project_host (and the other *_host
 * calls) run at full link speed from it, where pageable memory is first
 * copied through a bounce buffer by the CUDA driver. Returns NULL on failure;
 * free with shkz_b200_host_free. No counterpart in the reference (its grids
 * live in host memory only). */
void *shkz_b200_host_alloc(size_t bytes);
void shkz_b200_host_free(void *p);

/* Generic solver path for LinSolver= (replaces pcg_solver::solve,
 * src/linsolver/pcg.cpp:45-73): solves A x = b for a symmetric CSR matrix
 * given on the host (row-sorted, 0-based, FP64) with the reference's PCG loop
 * (local/include/pcgsolver/pcg_solver.h:246-295), x0 = 0, stop at
 * ||r||inf <= residual * ||b||inf, iterations = iteration + 1, in FP64 on the
 * device. With csr_preconditioner = NONE (default) the preconditioner is the
 * identity, which is what the shipped pcg module runs (its MIC(0) result is
 * overwritten, pcg_solver.h:379-384); with MIC0 it is the header's own
 * modified incomplete Cholesky (pcg_solver.h:88-223, mic_omega and
 * mic_min_diag_ratio), factored and applied on the device over level
 * schedules of the factor's pattern. The config's preconditioner field is
 * not used here. */
int shkz_b200_solve_csr(shkz_b200_ctx *ctx, long long n, const long long *indptr, const long long *indices,
                        const double *data, const double *b, double *x, shkz_b200_result *out);

/* Inspection of the last projection's device state in dense grid layout
 * (host buffers). what: 0 = diagonal (f32 cells), 1..3 = lower off-diagonal
 * x/y/z (f32 cells), 4 = MIC(0) inverse pivot d (f32 cells), 5 = rhs (f64 cells),
 * 6 = pressure (f64 cells, FP64 iterate), 7 = FP64 reference solution (f64 cells). */
int shkz_b200_inspect(shkz_b200_ctx *ctx, int what, void *host_out, size_t bytes);

/* Apply the preconditioner selected in the config once to a dense host
 * residual (f32 cells) of the last projection's system and return z (f32
 * cells); used to check the MIC(0) sweeps against a CPU restatement. */
int shkz_b200_apply_preconditioner(shkz_b200_ctx *ctx, const float *r_cells, float *z_cells);

/* y = A x on the last projection's system, dense f32 cells in and out. */
int shkz_b200_apply_matrix(shkz_b200_ctx *ctx, const float *x_cells, float *y_cells);

/* Device timing of one kernel on the last projection's system: launches it
 * `reps` times on the context stream, each launch between CUDA events after a
 * 256 MB write that evicts the L2, and stores the mean milliseconds per
 * launch. which: 0 = stencil q = A p with fused p.q, 1 (or 2) = the MIC(0)
 * forward and backward sweep pair with fused z.r, 3 = fused x/r update with
 * norms, 4 = p update, 5 = unknown labelling, 6 = weights/rhs assembly,
 * 7 = MIC(0) factor, 8 = one application of the learned preconditioner's
 * network (needs a loaded or initialised network), and the two passes of
 * the fused MIC(0)-PCG iteration on 16^3 macro tiles: 9 = stencil with the
 * direction update p = z + beta p, 10 = sweep pair with the x/r update in
 * the forward sweep (9 and 10 need a MIC(0) projection on macro tiles
 * first, else SHKZ_B200_ERR_STATE). *cells_out (may be NULL)
 * receives the cells the kernel sweeps per launch (pool cells, or grid cells
 * for 5). No reference counterpart: it is the measurement hook for the
 * roofline figures. */
int shkz_b200_time_kernel(shkz_b200_ctx *ctx, int which, int reps, double *ms_per_launch, long long *cells_out);

/* ---- learned preconditioner (3-level conv encoder-decoder used in a flexible PCG) ----
 * No counterpart in the reference: the network is the second preconditioner
 * of the projection (config preconditioner = SHKZ_B200_PRECOND_LEARNED);
 * the entry points below create, train, inspect and persist it. Training and
 * inspection act on the system of the last projection. */
int shkz_b200_learned_init(shkz_b200_ctx *ctx, unsigned seed);
long long shkz_b200_learned_param_count(shkz_b200_ctx *ctx);
/* FLOPs of one network application on the last projection's system as the
 * tensor cores execute it (2 * 27 * C_in * C_out per voxel of every active
 * 8x16x8 block of each layer's level); -1 without a network. */
double shkz_b200_learned_flops(shkz_b200_ctx *ctx);
/* parameters blob: per layer w[27][cout][cin] then b[cout], FP32 */
int shkz_b200_learned_set_params(shkz_b200_ctx *ctx, const float *blob, size_t n);
int shkz_b200_learned_get_params(shkz_b200_ctx *ctx, float *blob, size_t n, int gradients);
/* z = s N(r / s), s = ||r||inf, for a dense host residual (f32 cells) */
int shkz_b200_learned_apply(shkz_b200_ctx *ctx, const float *r_cells, float *z_cells);
/* dense level-0 network grid (cells rounded up to multiples of 4) */
int shkz_b200_learned_dims(shkz_b200_ctx *ctx, int *dims);
/* which = 0..12: stored activations X0, A1, S1, P1, A2, S2, P2, A3, B3, C2,
 * D2, C1, D1 (dense channels-last f32); 13: raw output Z; 14..26: gradients
 * w.r.t. activations 0..12 after the last backward. shape4 (may be
 * NULL) receives z, y, x, channels; out may be NULL to query the shape. */
int shkz_b200_learned_tensor(shkz_b200_ctx *ctx, int which, float *out, size_t count, int *shape4);
/* weight gradients of sum(gZ * Z) for the last application */
int shkz_b200_learned_backward(shkz_b200_ctx *ctx, const float *gZ_dense, size_t count);
/* `steps` Adam steps (learning rate lr) on the energy loss 1/2 z.Az - z.r */
int shkz_b200_learned_train(shkz_b200_ctx *ctx, int steps, double lr, unsigned seed, double *losses);
int shkz_b200_learned_save(shkz_b200_ctx *ctx, const char *path);
/* One 3^3 convolution of the network's tensor-core kernel on host arrays
 * (checking the kernel in isolation): in0 (nz,ny,nx,c0), in1 at half
 * resolution (nz/2,ny/2,nx/2,c1) nearest-upsampled and concatenated (may be
 * NULL when c1 = 0), w[27][cout][c0+c1], bias[cout] (may be NULL), planes = 4
 * or 8 output z planes per CTA; out (nz,ny,nx,cout). c0, c1 multiples of 16,
 * cout <= 128, even grid sizes. The accumulators of one CTA take planes x
 * (cout rounded up to a power of two, at least 32) tensor-memory columns, at
 * most 512: planes = 8 allows cout <= 64; a larger product returns
 * SHKZ_B200_ERR_LIMIT before any device work. No reference counterpart. */
int shkz_b200_conv3d(int nx, int ny, int nz, int c0, int c1, int cout, int planes, const float *in0,
                     const float *in1, const float *w, const float *bias, int relu, float *out);

/* The same convolution for callers that cannot allocate device memory (for
 * example an application that has reserved the whole GPU for its own pool
 * allocator, or a time-critical loop that must not pay the device-wide
 * synchronisation cudaMalloc/cudaFree may imply). It allocates nothing: all
 * pointers are DEVICE arrays the caller owns -- in0 (nz,ny,nx,c0) and in1
 * (nz/2,ny/2,nx/2,c1) BF16 bit patterns channels-last, w[27][cout][c0+c1]
 * FP32, bias[cout] FP32 (may be NULL), out (nz,ny,nx,cout) BF16 bit patterns
 * -- and `stream` is a cudaStream_t (NULL = the default stream); the call
 * waits for the stream to drain and reads the kernel's error word back before
 * it returns. in0, in1 and out must start on 16-byte boundaries and w, bias on
 * 4-byte boundaries (SHKZ_B200_ERR_ARG otherwise). Its scratch (packed
 * weights, block flags, an error word) is a fixed 1.1 MiB array in the library
 * that each GPU holds until exit. Limits: cout in {16, 32, 64, 128}, c0 + c1 <=
 * 128 (both multiples of 16), planes x max(cout, 32) <= 512 tensor-memory
 * columns (planes = 8 only with cout <= 64), at most 2^18 output blocks of
 * 8x16x8 voxels (a 512^3 grid); larger sizes return SHKZ_B200_ERR_LIMIT. All
 * checks come before any device work. The first call on a device (with
 * that device current) looks up the array's device address; make it before
 * any stream capture. Calls share the array, so calls that overlap on the GPU
 * race: serialise them. No counterpart in the reference. */
int shkz_b200_conv3d_noalloc(int nx, int ny, int nz, int c0, int c1, int cout, int planes, const uint16_t *in0,
                             const uint16_t *in1, const float *w, const float *bias, int relu, uint16_t *out,
                             void *stream);
int shkz_b200_learned_load(shkz_b200_ctx *ctx, const char *path);

#ifdef __cplusplus
}
#endif
#endif
