// Host-side launch interfaces shared by the CUDA translation units.
#pragma once
#include "common.cuh"

namespace shkz {

struct AssemblyInputs {
  Geometry G;
  const float *fluid;
  const uint8_t *fluid_active;
  const float *solid;          // may be null
  const uint8_t *solid_active; // may be null
  const float *vel[3];
  const float *svel[3];        // each may be null
  double dx, dt;
  double eps_solid, eps_fluid;
  int second_order_fluid, second_order_solid;
  const float *density[3];     // per-face solid density, each may be null
  double rhs_add;              // volume correction added to every rhs row
};

struct CoeffOutputs {
  float *diag, *offx, *offy, *offz;
  double *diag64, *offx64, *offy64, *offz64;   // may be null
  double *rhs64;
};

// Pool-resident system in 8^3 tiles.
struct PoolSystem {
  int K;                 // tiles in the pool
  const int *nbr;        // [K][6] pool index of neighbour tiles or -1
  const int *sched;      // [K] pool indices ordered by wavefront level
  const float *diag, *offx, *offy, *offz;
  // upper weights: the lower weight of the +x/+y/+z neighbour cell (across
  // the tile face where needed), for the backward MIC(0) sweep
  const float *upx, *upy, *upz;
  const double *diag64, *offx64, *offy64, *offz64;
  // 16^3 macro tiles (2x2x2 pool tiles) for the MIC(0) sweeps
  int KM;
  const int *msched;     // [KM] macro tiles ordered by wavefront level
  const int *mnbr;       // [KM][6] neighbour macro tiles or -1
  const int *msub;       // [KM][8] pool index of sub-tile (x + 2y + 4z) or -1
  unsigned long long *mfaces_f, *mfaces_b;  // [KM][3][256] epoch-tagged sweep faces
};

// assemble.cu
void launch_label(const AssemblyInputs &in, int *flags, uint8_t *unk, int *tile_count, cudaStream_t s);
void launch_coeff(const AssemblyInputs &in, const int *flags, const int *pool_tile, int K, const uint8_t *unk,
                  const CoeffOutputs &out, cudaStream_t s);
void launch_velocity_update(const AssemblyInputs &in, const int *flags, const int *tile_state,
                            const float *pressure_pool, float *const vel[3], uint8_t *const vact[3], cudaStream_t s);
// velocity extension after a projection (extend.cu)
struct ConstrainFields {
  const float *save[3];    // the velocity components (read-only while the constraint is found)
  const uint8_t *act[3];   // their active masks
};
// one extrapolation pass in place: frontier values into side/flag, then committed
// (flag must be all zero on entry and is all zero again on return)
void launch_extrapolate(int W, int H, int D, float *v, uint8_t *a, float *side, uint8_t *flag, cudaStream_t s);
void launch_solid_exists(const float *solid, const uint8_t *act, size_t n, int *flag, cudaStream_t s);
// constrained values of component d that differ from the field, into side/flag
void launch_constrain_find(int d, int nx, int ny, int nz, double dx, const float *solid, const int *solid_flag,
                           const ConstrainFields &f, float *side, uint8_t *flag, cudaStream_t s);
void launch_apply_side(size_t n, float *v, const float *side, uint8_t *flag, cudaStream_t s);

// FLIP splat (splat.cu). Particle records read in place: float fields at byte
// offsets (multiples of 4) of `stride`-byte records.
constexpr int kSplatWorkBins = 64;  // work classes of 4 particle visits each
// Largest edge bucket the splat accepts (particles of one edge cell, about 8
// to 12 in a FLIP simulation): ordering a bucket costs its size squared.
constexpr int kSplatBucketLimit = 4096;
struct SplatRecords {
  const unsigned char *base;
  long long count;
  int stride, off_p, off_v, off_m, off_c, off_bullet;  // off_c / off_bullet < 0: absent
  int splat_bullet;
};
struct SplatBuffers {
  float4 *posm;            // per particle: p, mass
  float4 *vc[3];           // per particle and axis d: u_d, c[d]
  int *key, *rank;         // [3][count]: edge bucket slot (-1: does not splat), arrival rank in it
  // Edge buckets live in 8x8x8 tiles of each axis' edge grid, 512 slots a
  // tile (splat.cu: bucket_slot). count holds a bucket's particles, then its
  // offset inside the tile's run; tile_start the first list position of each
  // tile. count and tile_act are zero between calls: a call touches and then
  // clears only the tiles its particles reach.
  int *count;              // [tiles * 512]
  uint8_t *tile_act;       // [tiles] the tile holds a particle
  int *tile_start;         // [tiles + 1], exclusive scan of the tiles' particle counts
  int *list;               // [3 count] d * count + particle index, bucket by bucket, arrival order inside one
  float4 *sposm, *svc;     // [3 count] posm and vc[d] bucket by bucket, index order inside one
  uint8_t *act[3];         // faces activated by the splat
  int *faces;              // active faces of each axis, listed from face_off[d]
  int *sorted;             // the same lists, faces with more particles to visit first
  int *face_bin;           // work class of each listed face
  int *work;               // [3][kSplatWorkBins] work-class counts, then cursors
  int *nfaces;             // [4]: list lengths of the three axes, then a bucket over kSplatBucketLimit (flag)
  long long face_off[3];
  long long tile_base[3];  // first tile of each axis
  long long tiles;
  int apic;
};
struct SplatGrid {
  float *velocity[3];            // optional (velocity[0] == nullptr: no combined velocity)
  uint8_t *velocity_active[3];
  float *mass[3], *momentum[3];  // optional (mass[0] == nullptr: none)
  uint8_t *splat_active[3];
};
void launch_splat_bin(const SplatRecords &R, int nx, int ny, int nz, double dx, const SplatBuffers &B,
                      cudaStream_t s);
size_t scan_tile_count(long long n);
void launch_exclusive_scan(int *data, long long n, int *tile_sums, cudaStream_t s);
// each reached tile's bucket counts into offsets inside it, then the tiles'
// starts (tile_sums: scratch of scan_tile_count(tiles + 1) ints)
void launch_splat_bucket_scan(const SplatBuffers &B, int *tile_sums, cudaStream_t s);
// bucket lists, then the particles' data copied into bucket order
void launch_splat_scatter(long long count, const SplatBuffers &B, cudaStream_t s);
// counts and tile flags of the reached tiles back to zero
void launch_splat_clear(const SplatBuffers &B, cudaStream_t s);
// active-face lists ordered by work, then the per-face sums and the combined velocity
void launch_splat_gather(int nx, int ny, int nz, double dx, const SplatBuffers &B, const SplatGrid &G,
                         cudaStream_t s);
void launch_surface_tension(const AssemblyInputs &in, const int *flags, float *curv, double kappa, float *const vel[3],
                            const uint8_t *const vact[3], cudaStream_t s);
void launch_scatter_pressure(const Geometry &G, const int *tile_state, const float *pressure_pool, const uint8_t *unk,
                             float *pressure, uint8_t *pressure_active, cudaStream_t s);

// warmstart.cu: reference unknown numbering (tiles of edge T, x fastest) and
// the warm-start gather/finish over the pool
size_t unknown_rank_scratch(const Geometry &G, int T);
long long launch_unknown_rank(const Geometry &G, int K, const uint8_t *unk, int T, const int *tile_state,
                              int *rank_pool, int *cnt, long long *d_total, cudaStream_t s);
void launch_warm_gather(long long n, const int *rank_pool, const double *prev, long long prev_n, double *x0,
                        cudaStream_t s);
void launch_warm_finish(long long n, const int *rank_pool, const double *x0, double *x, double *prev, cudaStream_t s);

}  // namespace shkz
