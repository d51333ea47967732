// Warm start of the pressure solve (macpressuresolver3.cpp:236-259, 292-296).
//
// The reference keeps the previous solution as an RCMatrix vector indexed by
// unknown number, resizes it to the new unknown count, solves
// A d = b - A x_prev and returns x = d + x_prev. The unknown numbering is the
// order in which mark_body visits the liquid (macpressuresolver3.cpp:159-167):
// tiles of the grid's tile edge T in x-fastest tile order
// (tiledarray3.cpp:314-340, 466-492), x fastest inside a tile. The kernels
// below compute that number for every unknown of the pool, so the previous
// vector is read and written exactly as the reference indexes it.
#include "common.cuh"
#include "kernels.h"

namespace shkz {

struct RefTiles {
  int T, rbx, rby, rbz;
  long long n;
};

static RefTiles ref_tiles(const Geometry &G, int T) {
  RefTiles R;
  R.T = T;
  R.rbx = (G.nx + T - 1) / T;
  R.rby = (G.ny + T - 1) / T;
  R.rbz = (G.nz + T - 1) / T;
  R.n = (long long)R.rbx * R.rby * R.rbz;
  return R;
}

// unknowns per tile of edge T
__global__ void __launch_bounds__(256) k_rank_count(Geometry G, RefTiles R, const uint8_t *unk, int *cnt) {
  __shared__ int wsum[8];
  const long long t = blockIdx.x;
  const int oi = (int)(t % R.rbx) * R.T, oj = (int)((t / R.rbx) % R.rby) * R.T,
            ok = (int)(t / ((long long)R.rbx * R.rby)) * R.T;
  const int cells = R.T * R.T * R.T;
  int c = 0;
  for (int l = threadIdx.x; l < cells; l += blockDim.x) {
    const int i = oi + l % R.T, j = oj + (l / R.T) % R.T, k = ok + l / (R.T * R.T);
    if (i < G.nx && j < G.ny && k < G.nz) c += unk[(size_t)i + (size_t)G.nx * ((size_t)j + (size_t)G.ny * k)];
  }
  c = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int w = 0; w < 8; ++w) s += wsum[w];
    cnt[t] = s;
  }
}

// In-place exclusive scan of n ints by one CTA of 1024 threads (chunked).
__global__ void __launch_bounds__(1024) k_scan_exclusive(int *v, long long n, long long *total) {
  __shared__ long long part[1024];
  const long long chunk = (n + 1023) / 1024;
  const long long b = threadIdx.x * chunk, e = b + chunk < n ? b + chunk : n;
  long long s = 0;
  for (long long i = b; i < e; ++i) s += v[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const long long add = threadIdx.x >= off ? part[threadIdx.x - off] : 0;
    __syncthreads();
    part[threadIdx.x] += add;
    __syncthreads();
  }
  long long run = part[threadIdx.x] - s;  // exclusive prefix of this chunk
  for (long long i = b; i < e; ++i) {
    const int x = v[i];
    v[i] = (int)run;
    run += x;
  }
  if (threadIdx.x == 1023) *total = part[1023];
}

// Reference number of every unknown, written into the pool layout (-1 elsewhere).
__global__ void __launch_bounds__(256) k_rank_assign(Geometry G, RefTiles R, const uint8_t *unk, const int *base,
                                                     const int *tile_state, int *rank_pool) {
  __shared__ int wsum[8];
  __shared__ int run;
  const long long t = blockIdx.x;
  const int oi = (int)(t % R.rbx) * R.T, oj = (int)((t / R.rbx) % R.rby) * R.T,
            ok = (int)(t / ((long long)R.rbx * R.rby)) * R.T;
  const int cells = R.T * R.T * R.T;
  if (threadIdx.x == 0) run = base[t];
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int l0 = 0; l0 < cells; l0 += 256) {
    const int l = l0 + threadIdx.x;
    int i = 0, j = 0, k = 0;
    bool f = false;
    if (l < cells) {
      i = oi + l % R.T;
      j = oj + (l / R.T) % R.T;
      k = ok + l / (R.T * R.T);
      f = i < G.nx && j < G.ny && k < G.nz && unk[(size_t)i + (size_t)G.nx * ((size_t)j + (size_t)G.ny * k)];
    }
    const unsigned m = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wsum[w] = __popc(m);
    __syncthreads();
    int before = 0, total = 0;
    for (int q = 0; q < 8; ++q) {
      before += q < w ? wsum[q] : 0;
      total += wsum[q];
    }
    if (f) {
      const int r = run + before + __popc(m & ((1u << lane) - 1u));
      const long long tt = (long long)(i >> 3) + (long long)G.bx * ((long long)(j >> 3) + (long long)G.by * (k >> 3));
      const int pt = tile_state[tt];
      if (pt >= 0) rank_pool[(size_t)pt * SHKZ_TC + (i & 7) + 8 * (j & 7) + 64 * (k & 7)] = r;
    }
    __syncthreads();
    if (threadIdx.x == 0) run += total;
    __syncthreads();
  }
}

__global__ void k_warm_gather(long long n, const int *rank_pool, const double *prev, long long prev_n, double *x0) {
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
    const int r = rank_pool[o];
    x0[o] = (r >= 0 && r < prev_n) ? prev[r] : 0.0;
  }
}

// x += x0, then prev[rank] = x
__global__ void k_warm_finish(long long n, const int *rank_pool, const double *x0, double *x, double *prev) {
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
    const int r = rank_pool[o];
    if (r < 0) continue;
    const double v = x[o] + x0[o];
    x[o] = v;
    prev[r] = v;
  }
}

size_t unknown_rank_scratch(const Geometry &G, int T) { return (size_t)ref_tiles(G, T).n; }

long long launch_unknown_rank(const Geometry &G, int K, const uint8_t *unk, int T, const int *tile_state,
                              int *rank_pool, int *cnt, long long *d_total, cudaStream_t s) {
  const RefTiles R = ref_tiles(G, T);
  cudaMemsetAsync(rank_pool, 0xff, sizeof(int) * (size_t)K * SHKZ_TC, s);
  count_launches(3);
  k_rank_count<<<(unsigned)R.n, 256, 0, s>>>(G, R, unk, cnt);
  k_scan_exclusive<<<1, 1024, 0, s>>>(cnt, R.n, d_total);
  k_rank_assign<<<(unsigned)R.n, 256, 0, s>>>(G, R, unk, cnt, tile_state, rank_pool);
  return R.n;
}

static int grid_cells(long long n) {
  long long g = (n + 1023) / 1024;
  if (g > 148 * 8) g = 148 * 8;
  return g < 1 ? 1 : (int)g;
}

void launch_warm_gather(long long n, const int *rank_pool, const double *prev, long long prev_n, double *x0,
                        cudaStream_t s) {
  count_launches(1);
  k_warm_gather<<<grid_cells(n), 256, 0, s>>>(n, rank_pool, prev, prev_n, x0);
}

void launch_warm_finish(long long n, const int *rank_pool, const double *x0, double *x, double *prev, cudaStream_t s) {
  count_launches(1);
  k_warm_finish<<<grid_cells(n), 256, 0, s>>>(n, rank_pool, x0, x, prev);
}

}  // namespace shkz
