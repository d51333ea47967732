// Shared definitions for the B200 pressure-projection kernels.
//
// Device layout ("tile pool"): the grid is cut into 8^3-cell tiles. Only
// tiles that contain at least one pressure unknown are kept; they are
// compacted into a pool of K tiles. Every per-cell solver array is stored
// pool-major, [K][512] floats, cell (ii,jj,kk) of a tile at ii + 8*jj + 64*kk
// (x fastest, like the reference's in-tile order, src/array/tiledarray3.cpp:806-808).
// A tile is 2 KB per FP32 field, so one CTA moves whole tiles with
// coalesced 16-byte accesses.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define SHKZ_T 8
#define SHKZ_TC 512          // cells per tile
#define SHKZ_LOG_T 3

namespace shkz {

// Neighbour slots in the per-tile neighbour table.
enum { NB_XM = 0, NB_XP = 1, NB_YM = 2, NB_YP = 3, NB_ZM = 4, NB_ZP = 5 };

struct Geometry {
  int nx, ny, nz;          // cells
  int bx, by, bz;          // tiles per axis
  long long ntiles;        // bx*by*bz
};

// Device-resident solver scalars. Kernels read alpha/beta from here so the
// host never waits inside an iteration; once `done` is set the remaining
// launched iterations return at once.
struct SolverState {
  double rho;              // z.r of the current iterate
  double rho_new;
  double pq;               // p.Ap
  double alpha, beta;
  double rmax;             // ||r||_inf (recursive residual)
  double rmax0;            // ||b||_inf
  double r2;               // ||r||_2^2
  double tol_abs;          // tol * ||b||_inf
  double ru_threshold;     // request an FP64 residual replacement below this ||r||inf
  int iter;                // iterations completed
  int done;                // 1 = converged, 2 = max iterations, 3 = breakdown, 4 = replace residual
  int status;              // 0 ok, <0 error (wait timeout, NaN)
  int pad;
};

// Block-wide sum of one double; every thread gets the result.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *smem) {
  #pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) smem[w] = v;
  __syncthreads();
  double s = 0.0;
  #pragma unroll
  for (int i = 0; i < NT / 32; ++i) s += smem[i];
  return s;
}

template <int NT>
__device__ __forceinline__ double block_max(double v, double *smem) {
  #pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) smem[w] = v;
  __syncthreads();
  double s = 0.0;
  #pragma unroll
  for (int i = 0; i < NT / 32; ++i) s = fmax(s, smem[i]);
  return s;
}

}  // namespace shkz

#define SHKZ_CUDA_TRY(expr)                                       \
  do {                                                            \
    cudaError_t _e = (expr);                                      \
    if (_e != cudaSuccess) {                                      \
      shkz_set_cuda_error(_e, #expr, __FILE__, __LINE__);         \
      return SHKZ_B200_ERR_CUDA;                                  \
    }                                                             \
  } while (0)

void shkz_set_cuda_error(cudaError_t e, const char *expr, const char *file, int line);

// Number of kernels this library has launched (host-side count, all threads).
namespace shkz {
void count_launches(int n);
long long launches_so_far();
}
