// Matrix-free PCG on the 8^3 tile pool.
//
// Reference algorithm: PCGSolver::solve (local/include/pcgsolver/pcg_solver.h:246-295)
// with the MIC(0) factor of factor_modified_incomplete_cholesky0 (:88-189)
// and the sweeps solve_lower / solve_lower_transpose_in_place (:195-223).
//
// Per-cell system data (pool-major [K][512]):
//   diag        A_ii
//   offx/y/z    w = -A(i, i-e) for the lower neighbour along x/y/z, zero unless
//               both cells are unknowns
// The upper couplings of a cell are the lower weights of its +x/+y/+z
// neighbours, so the 7-point row is diag, three own weights and three
// neighbour weights.
//
// MIC(0) in this storage. With d = invdiag^2 = 1/pivot, the reference factor
// (lower neighbours k of j all precede j in its tile-major numbering) is
//   pivot_j = A_jj - sum_k d_k w_jk (w_jk + omega * (S_k - w_jk)),
//   S_k = sum of k's upper weights;  d_j = 1/pivot_j, or 1/A_jj when
//   pivot_j < min_ratio * A_jj,
// and M^-1 r is
//   t_j = d_j (r_j + sum_{k lower} w_jk t_k)            (forward)
//   z_j = t_j + d_j sum_{a upper} w_aj z_a               (backward)
// which equals invdiag*(...) of solve_lower and solve_lower_transpose with
// L_jk = A_jk invdiag_k.
//
// The sweeps run as a tile wavefront: CTAs take tiles in level order
// (bi+bj+bk ascending for the forward sweep) from an atomic slot counter and
// wait, with a bounded spin, for the flags of the three lower (upper)
// neighbour tiles. A CTA only waits on tiles whose slot was handed out
// earlier, i.e. to CTAs that are already running, so the wait always ends;
// if it does not within the spin limit the kernel records an error and
// finishes without waiting.
#include "common.cuh"
#include "kernels.h"
#include "solver.h"
#include <math_constants.h>
#include <atomic>

namespace shkz {

static std::atomic<long long> g_launches{0};
void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launches_so_far() { return g_launches.load(std::memory_order_relaxed); }

#define SPIN_LIMIT (1 << 21)   // ~0.15 s with the back-off below

__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }
__device__ __forceinline__ float comp(const float4 &v, int e) { return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w)); }

// Deterministic finish of a grid reduction: every block writes its partial;
// the last block to arrive sums them in block order.
__device__ __forceinline__ bool last_block(unsigned *counter) {
  __shared__ bool s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned ticket = atomicAdd(counter, 1u);
    s_last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  return s_last;
}

template <int NT>
__device__ double sum_partials(const double *part, int n, double *red) {
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += NT) s += part[i];
  return block_sum<NT>(s, red);
}
template <int NT>
__device__ double max_partials(const double *part, int n, double *red) {
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += NT) s = fmax(s, part[i]);
  return block_max<NT>(s, red);
}

// ---------------------------------------------------------------------------
// Tile pool construction

__global__ void k_pool_blocksum(const int *tile_count, long long nt, int *bsum) {
  __shared__ double red[8];
  const long long base = (long long)blockIdx.x * 1024;
  int c = 0;
  for (int i = threadIdx.x; i < 1024; i += 256) {
    const long long t = base + i;
    if (t < nt && tile_count[t] > 0) ++c;
  }
  const double s = block_sum<256>((double)c, red);
  if (threadIdx.x == 0) bsum[blockIdx.x] = (int)s;
}

__global__ void k_pool_scan_blocks(int *bsum, int nb, int *total) {
  // one block: exclusive scan of up to a few thousand block sums
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int i = 0; i < nb; ++i) {
      const int v = bsum[i];
      bsum[i] = acc;
      acc += v;
    }
    *total = acc;
  }
}

__global__ void k_pool_assign(const int *tile_count, long long nt, const int *boff, int *tile_state, int *pool_tile) {
  // 1024 tiles per block, 1024 threads: in-block exclusive scan
  __shared__ int warp_tot[32];
  const long long t = (long long)blockIdx.x * 1024 + threadIdx.x;
  const int flag = (t < nt && tile_count[t] > 0) ? 1 : 0;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int incl = flag;
  #pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_tot[w] = incl;
  __syncthreads();
  if (w == 0) {
    int v = warp_tot[lane];
    #pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += y;
    }
    warp_tot[lane] = v;  // inclusive
  }
  __syncthreads();
  const int excl = incl - flag + (w > 0 ? warp_tot[w - 1] : 0) + boff[blockIdx.x];
  if (t < nt) {
    tile_state[t] = flag ? excl : -1;
    if (flag) pool_tile[excl] = (int)t;
  }
}

__global__ void k_pool_neighbours(Geometry G, const int *tile_state, const int *pool_tile, int K, int *nbr,
                                  int *level_count) {
  const int pt = blockIdx.x * blockDim.x + threadIdx.x;
  if (pt >= K) return;
  const long long t = pool_tile[pt];
  const int ti = (int)(t % G.bx), tj = (int)((t / G.bx) % G.by), tk = (int)(t / ((long long)G.bx * G.by));
  auto look = [&](int i, int j, int k) -> int {
    if (i < 0 || j < 0 || k < 0 || i >= G.bx || j >= G.by || k >= G.bz) return -1;
    return tile_state[(long long)i + (long long)G.bx * ((long long)j + (long long)G.by * k)];
  };
  nbr[pt * 6 + NB_XM] = look(ti - 1, tj, tk);
  nbr[pt * 6 + NB_XP] = look(ti + 1, tj, tk);
  nbr[pt * 6 + NB_YM] = look(ti, tj - 1, tk);
  nbr[pt * 6 + NB_YP] = look(ti, tj + 1, tk);
  nbr[pt * 6 + NB_ZM] = look(ti, tj, tk - 1);
  nbr[pt * 6 + NB_ZP] = look(ti, tj, tk + 1);
  atomicAdd(&level_count[ti + tj + tk], 1);
}

__global__ void k_level_scan(int *level_count, int nlev) {
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int i = 0; i < nlev; ++i) {
      const int v = level_count[i];
      level_count[i] = acc;
      acc += v;
    }
  }
}

__global__ void k_level_scatter(Geometry G, const int *pool_tile, int K, int *level_cursor, int *sched) {
  const int pt = blockIdx.x * blockDim.x + threadIdx.x;
  if (pt >= K) return;
  const long long t = pool_tile[pt];
  const int ti = (int)(t % G.bx), tj = (int)((t / G.bx) % G.by), tk = (int)(t / ((long long)G.bx * G.by));
  const int pos = atomicAdd(&level_cursor[ti + tj + tk], 1);
  sched[pos] = pt;
}

// ---------------------------------------------------------------------------
// q = A p over the pool, p staged in shared memory with its six halo faces,
// fused with p.q. One tile per loop trip, 128 threads, four x-consecutive
// cells per thread.

struct SpmvSmem {
  float xs[10][10][16];  // (kk+1, jj+1, ii+4); halos at kk/jj 0,9 and ii 3,12
};

// zu != null: the pending direction update p <- z + beta p is applied on the
// fly (k_update_p's arithmetic) to the tile and its halo, and the tile's new
// p is written to pout (a different buffer: other CTAs still read the old p
// for their halos).
__device__ __forceinline__ void stage_tile(const PoolSystem &S, const float *__restrict__ p, int pt, SpmvSmem &sm,
                                           float4 &xv, const float *__restrict__ zu = nullptr,
                                           float *__restrict__ pout = nullptr, float beta = 0.0f) {
  const int tid = threadIdx.x;
  const int q4 = tid & 1, jj = (tid >> 1) & 7, kk = tid >> 4;
  const size_t base = (size_t)pt * SHKZ_TC + kk * 64 + jj * 8 + q4 * 4;
  xv = ld4(p + base);
  if (zu) {
    const float4 zv = ld4(zu + base);
    xv.x = zv.x + beta * xv.x; xv.y = zv.y + beta * xv.y; xv.z = zv.z + beta * xv.z; xv.w = zv.w + beta * xv.w;
    st4(pout + base, xv);
  }
  st4(&sm.xs[kk + 1][jj + 1][4 + 4 * q4], xv);
  // The 6 x 64 halo values: three per thread, faces XM, YM, ZM for threads
  // 0-63 and XP, YP, ZP for 64-127. Every load is issued before any is used,
  // so the three neighbour lookups and the value loads each cost one round
  // trip, not one per value.
  const int a = tid & 63, u = a & 7, v = a >> 3, side = tid >> 6;
  int nb[3];
  #pragma unroll
  for (int q = 0; q < 3; ++q) nb[q] = S.nbr[pt * 6 + 2 * q + side];
  float hv[3], hz[3];
  #pragma unroll
  for (int q = 0; q < 3; ++q) {
    // cell of the neighbour tile next to this tile's face
    const int cell = q == 0 ? (side ? 0 : 7) + 8 * u + 64 * v
                   : q == 1 ? u + (side ? 0 : 56) + 64 * v
                            : u + 8 * v + (side ? 0 : 448);
    const size_t o = (size_t)(nb[q] >= 0 ? nb[q] : 0) * SHKZ_TC + cell;
    hv[q] = nb[q] >= 0 ? p[o] : 0.0f;
    hz[q] = (zu && nb[q] >= 0) ? zu[o] : 0.0f;
  }
  #pragma unroll
  for (int q = 0; q < 3; ++q) {
    const float val = (zu && nb[q] >= 0) ? hz[q] + beta * hv[q] : hv[q];
    if (q == 0) sm.xs[v + 1][u + 1][side ? 12 : 3] = val;
    else if (q == 1) sm.xs[v + 1][side ? 9 : 0][u + 4] = val;
    else sm.xs[side ? 9 : 0][v + 1][u + 4] = val;
  }
}

struct Coef4 {
  float4 dg, ox, oy, oz;
  // upper weights that no lane of this warp holds: the +x neighbour's first
  // column (q4 == 1), the +y row (jj == 7), the +z plane (odd kk)
  float oxf;
  float4 oyf, ozf;
};

// All coefficient loads of a tile, issued before the tile's barrier so their
// latency overlaps the staging of p.
__device__ __forceinline__ Coef4 load_coef4(const PoolSystem &S, int pt) {
  const int tid = threadIdx.x;
  const int q4 = tid & 1, jj = (tid >> 1) & 7, kk = tid >> 4;
  const size_t base = (size_t)pt * SHKZ_TC + kk * 64 + jj * 8 + q4 * 4;
  Coef4 c;
  c.dg = ld4(S.diag + base);
  c.ox = ld4(S.offx + base);
  c.oy = ld4(S.offy + base);
  c.oz = ld4(S.offz + base);
  const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
  c.oxf = 0.0f;
  if (q4 == 1) {
    const int nb = S.nbr[pt * 6 + NB_XP];
    if (nb >= 0) c.oxf = S.offx[(size_t)nb * SHKZ_TC + kk * 64 + jj * 8];
  }
  c.oyf = zero4;
  if (jj == 7) {
    const int nb = S.nbr[pt * 6 + NB_YP];
    if (nb >= 0) c.oyf = ld4(S.offy + (size_t)nb * SHKZ_TC + kk * 64 + q4 * 4);
  }
  c.ozf = zero4;
  if (kk & 1) {
    if (kk < 7) c.ozf = ld4(S.offz + base + 64);
    else {
      const int nb = S.nbr[pt * 6 + NB_ZP];
      if (nb >= 0) c.ozf = ld4(S.offz + (size_t)nb * SHKZ_TC + jj * 8 + q4 * 4);
    }
  }
  return c;
}

// Computes the four outputs of this thread for tile pt (after staging and a barrier).
__device__ __forceinline__ float4 stencil4(const SpmvSmem &sm, float4 xv, const Coef4 &cf) {
  const int tid = threadIdx.x;
  const int q4 = tid & 1, jj = (tid >> 1) & 7, kk = tid >> 4;
  const float4 dg = cf.dg, ox = cf.ox, oy = cf.oy, oz = cf.oz;
  // upper weights: lower weights of the +x/+y/+z neighbour cells
  const float oxn = __shfl_down_sync(0xffffffffu, ox.x, 1);
  float4 oyn, ozn;
  oyn.x = __shfl_down_sync(0xffffffffu, oy.x, 2);
  oyn.y = __shfl_down_sync(0xffffffffu, oy.y, 2);
  oyn.z = __shfl_down_sync(0xffffffffu, oy.z, 2);
  oyn.w = __shfl_down_sync(0xffffffffu, oy.w, 2);
  ozn.x = __shfl_down_sync(0xffffffffu, oz.x, 16);
  ozn.y = __shfl_down_sync(0xffffffffu, oz.y, 16);
  ozn.z = __shfl_down_sync(0xffffffffu, oz.z, 16);
  ozn.w = __shfl_down_sync(0xffffffffu, oz.w, 16);
  const float oxu3 = q4 == 0 ? oxn : cf.oxf;
  const float4 oyu = jj < 7 ? oyn : cf.oyf;
  const float4 ozu = (kk & 1) == 0 ? ozn : cf.ozf;
  const float oxu[4] = {ox.y, ox.z, ox.w, oxu3};
  float out[4];
  #pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int c = 4 + 4 * q4 + e;
    const float xc = comp(xv, e);
    const float xm = sm.xs[kk + 1][jj + 1][c - 1];
    const float xp = sm.xs[kk + 1][jj + 1][c + 1];
    const float ym = sm.xs[kk + 1][jj][c];
    const float yp = sm.xs[kk + 1][jj + 2][c];
    const float zm = sm.xs[kk][jj + 1][c];
    const float zp = sm.xs[kk + 2][jj + 1][c];
    float off = comp(ox, e) * xm + oxu[e] * xp;
    off += comp(oy, e) * ym + comp(oyu, e) * yp;
    off += comp(oz, e) * zm + comp(ozu, e) * zp;
    out[e] = comp(dg, e) * xc - off;
  }
  return make_float4(out[0], out[1], out[2], out[3]);
}

// mode 0: q = A p and pq = p.q -> st->pq, st->alpha = rho/pq
// mode 1: q = A p only
#define SPMV_CTAS_PER_SM 8
// With zu != null, p and pout are the two direction buffers and the one
// holding the current direction is chosen by the parity of the completed
// iteration count on the device, so launches that the loop control retires
// (done != 0) do not flip it.
__global__ void __launch_bounds__(128, SPMV_CTAS_PER_SM) k_spmv(PoolSystem S, const float *p, float *__restrict__ q,
                                              double *partials, unsigned *counter, SolverState *st, int mode,
                                              const float *__restrict__ zu, float *pout) {
  __shared__ SpmvSmem sm;
  __shared__ double red[4];
  if (st && st->done) return;
  double acc = 0.0;
  const int tid = threadIdx.x;
  const int q4 = tid & 1, jj = (tid >> 1) & 7, kk = tid >> 4;
  const float beta = zu ? (float)st->beta : 0.0f;
  if (zu && (st->iter & 1)) {
    float *t = const_cast<float *>(p);
    p = pout;
    pout = t;
  }
  for (int pt = blockIdx.x; pt < S.K; pt += gridDim.x) {
    float4 xv;
    const Coef4 cf = load_coef4(S, pt);
    __syncthreads();
    stage_tile(S, p, pt, sm, xv, zu, pout, beta);
    __syncthreads();
    const float4 y = stencil4(sm, xv, cf);
    st4(q + (size_t)pt * SHKZ_TC + kk * 64 + jj * 8 + q4 * 4, y);
    acc += (double)xv.x * y.x + (double)xv.y * y.y + (double)xv.z * y.z + (double)xv.w * y.w;
  }
  if (mode != 0) return;
  const double s = block_sum<128>(acc, red);
  if (tid == 0) partials[blockIdx.x] = s;
  if (last_block(counter)) {
    const double pq = sum_partials<128>(partials, gridDim.x, red);
    if (tid == 0) {
      st->pq = pq;
      st->alpha = st->rho / pq;
      if (!(pq == pq) || pq == 0.0) {
        st->done = 3;
        if (!(pq == pq)) st->status = -5;
      }
      *counter = 0;
    }
  }
}

// x += alpha p; r -= alpha q; ||r||inf, ||r||2^2 -> st; convergence check.
__global__ void __launch_bounds__(256) k_update_xr(int n4, const float4 *__restrict__ p, const float4 *__restrict__ q,
                                                   float4 *__restrict__ x, float4 *__restrict__ r, double *partials,
                                                   unsigned *counter, SolverState *st, int max_iterations) {
  __shared__ double red[8];
  if (st->done) return;
  const float alpha = (float)st->alpha;
  double m = 0.0, s2 = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += gridDim.x * blockDim.x) {
    const float4 pv = p[i], qv = q[i];
    float4 xv = x[i], rv = r[i];
    xv.x += alpha * pv.x; xv.y += alpha * pv.y; xv.z += alpha * pv.z; xv.w += alpha * pv.w;
    rv.x -= alpha * qv.x; rv.y -= alpha * qv.y; rv.z -= alpha * qv.z; rv.w -= alpha * qv.w;
    x[i] = xv;
    r[i] = rv;
    m = fmax(m, fmax(fmax(fabs((double)rv.x), fabs((double)rv.y)), fmax(fabs((double)rv.z), fabs((double)rv.w))));
    s2 += (double)rv.x * rv.x + (double)rv.y * rv.y + (double)rv.z * rv.z + (double)rv.w * rv.w;
  }
  const double bm = block_max<256>(m, red);
  const double bs = block_sum<256>(s2, red);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = bm;
    partials[gridDim.x + blockIdx.x] = bs;
  }
  if (last_block(counter)) {
    double mm = 0.0, ss = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += 256) {
      mm = fmax(mm, partials[i]);
      ss += partials[gridDim.x + i];
    }
    mm = block_max<256>(mm, red);
    ss = block_sum<256>(ss, red);
    // a NaN anywhere in r makes the (ordered) sum of squares NaN
    const bool nan = !(ss == ss);
    if (threadIdx.x == 0) {
      st->rmax = nan ? CUDART_NAN : mm;
      st->r2 = ss;
      st->iter += 1;
      if (nan) { st->done = 3; st->status = -5; }
      else if (mm <= st->tol_abs) st->done = 1;
      else if (st->iter >= max_iterations) st->done = 2;
      else if (mm < st->ru_threshold) st->done = 4;
      *counter = 0;
    }
  }
}

// rho_new from partials (one per pool tile or block), beta = rho_new/rho, rho = rho_new.
__global__ void __launch_bounds__(1024) k_finish_rho(const double *partials, int n, SolverState *st, int init) {
  __shared__ double red[32];
  if (st->done) return;
  const double s = sum_partials<1024>(partials, n, red);
  if (threadIdx.x == 0) {
    if (init) {
      st->rho = s;
      st->beta = 0.0;
      if (s == 0.0 || !(s == s)) {
        st->done = 3;
        if (!(s == s)) st->status = -5;
      }
    } else {
      st->beta = s / st->rho;
      st->rho = s;
    }
  }
}

// Unpreconditioned path: rho_new = r.r from the update kernel.
__global__ void k_finish_rho_r2(SolverState *st, int init) {
  if (st->done) return;
  if (init) {
    st->rho = st->r2;
    st->beta = 0.0;
  } else {
    st->beta = st->r2 / st->rho;
    st->rho = st->r2;
  }
}

// p = z + beta p (beta from st; init: p = z)
__global__ void __launch_bounds__(256) k_update_p(int n4, const float4 *__restrict__ z, float4 *__restrict__ p,
                                                  const SolverState *st) {
  if (st->done) return;
  const float beta = (float)st->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += gridDim.x * blockDim.x) {
    const float4 zv = z[i];
    float4 pv = p[i];
    pv.x = zv.x + beta * pv.x; pv.y = zv.y + beta * pv.y; pv.z = zv.z + beta * pv.z; pv.w = zv.w + beta * pv.w;
    p[i] = pv;
  }
}

// ---------------------------------------------------------------------------
// MIC(0)

// S_k = offx(k+x) + offy(k+y) + offz(k+z), FP64, per pool cell.
__global__ void __launch_bounds__(512) k_mic_colsum(PoolSystem S, double *colsum) {
  const int pt = blockIdx.x, c = threadIdx.x;
  const int ii = c & 7, jj = (c >> 3) & 7, kk = c >> 6;
  const size_t o = (size_t)pt * SHKZ_TC + c;
  double s = 0.0;
  {
    int nb = pt, cell = c + 1;
    if (ii == 7) { nb = S.nbr[pt * 6 + NB_XP]; cell = c - 7; }
    if (nb >= 0) s += S.offx64[(size_t)nb * SHKZ_TC + cell];
  }
  {
    int nb = pt, cell = c + 8;
    if (jj == 7) { nb = S.nbr[pt * 6 + NB_YP]; cell = c - 56; }
    if (nb >= 0) s += S.offy64[(size_t)nb * SHKZ_TC + cell];
  }
  {
    int nb = pt, cell = c + 64;
    if (kk == 7) { nb = S.nbr[pt * 6 + NB_ZP]; cell = c - 448; }
    if (nb >= 0) s += S.offz64[(size_t)nb * SHKZ_TC + cell];
  }
  colsum[o] = s;
}

struct WaveSync {
  int slot;
  unsigned finished;
  int epoch;
  int error;         // 0, or the slot that gave up waiting + 1
  int spin_limit;    // polling rounds of a bounded wait (0: SPIN_LIMIT); set by the host
  int skip_publish;  // fault injection (0: off): wavefront slot k - 1 of a forward macro sweep does not publish
};

// Rounds a bounded wait polls before it gives up.
__device__ __forceinline__ int spin_rounds(const WaveSync *ws) {
  const int v = *((volatile const int *)&ws->spin_limit);
  return v > 0 ? v : SPIN_LIMIT;
}

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Bounded wait for flag >= target. Returns false when the limit was hit.
__device__ __forceinline__ bool wait_flag(const int *flag, int target, int limit) {
  for (int it = 0; it < limit; ++it) {
    if (ld_acquire(flag) >= target) return true;
    if (it > 64) __nanosleep(64);
  }
  return false;
}

// Common prologue of a wavefront kernel: take a slot, read the epoch.
__device__ __forceinline__ void wave_begin(WaveSync *ws, int &slot, int &target) {
  __shared__ int s_slot, s_epoch;
  if (threadIdx.x == 0) {
    s_slot = atomicAdd(&ws->slot, 1);
    s_epoch = *((volatile int *)&ws->epoch) + 1;
  }
  __syncthreads();
  slot = s_slot;
  target = s_epoch;
}

// Producer side: every thread's stores precede the barrier; thread 0's
// fence then orders them (cumulatively) before the releasing flag store.
__device__ __forceinline__ void wave_end(WaveSync *ws, int *flags, int pt, int target) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    st_release(&flags[pt], target);
    const unsigned f = atomicAdd(&ws->finished, 1u);
    if (f == gridDim.x - 1) {
      ws->slot = 0;
      ws->finished = 0;
      __threadfence();
      atomicExch(&ws->epoch, target);
    }
  }
}

// Wait (thread 0) for the given neighbour tiles, then release the CTA.
__device__ __forceinline__ void wave_wait(WaveSync *ws, const int *flags, const int *nb3, int target, int slot) {
  if (threadIdx.x == 0) {
    bool ok = true;
    const int limit = spin_rounds(ws);
    #pragma unroll
    for (int i = 0; i < 3; ++i)
      if (nb3[i] >= 0 && ok) ok = wait_flag(&flags[nb3[i]], target, limit);
    if (!ok) atomicCAS(&ws->error, 0, slot + 1);
  }
  // consumer side: thread 0's acquire, then the barrier, orders the other
  // threads' (L2) loads of the neighbour tiles after the flag
  __syncthreads();
}

// Tile rows are staged in shared memory; in step s of the in-tile wavefront
// thread (jj,kk) handles cell ii = s - jj - kk of its x-row, so each cell's
// -x/-y/-z (or +x/+y/+z) neighbours were finished one barrier earlier.
__device__ __forceinline__ void load_tile_f32(float *dst, const float *src) {
  for (int v = threadIdx.x; v < SHKZ_TC / 4; v += blockDim.x)
    reinterpret_cast<float4 *>(dst)[v] = reinterpret_cast<const float4 *>(src)[v];
}
__device__ __forceinline__ void load_tile_f64(double *dst, const double *src) {
  for (int v = threadIdx.x; v < SHKZ_TC / 2; v += blockDim.x)
    reinterpret_cast<double2 *>(dst)[v] = reinterpret_cast<const double2 *>(src)[v];
}

// Factor: FP64 pivots, forward wavefront. 64 threads, thread = (jj, kk) row.
__global__ void __launch_bounds__(64) k_mic_factor(PoolSystem S, const int *sched, const double *colsum, double omega,
                                                   double min_ratio, double *d64, float *d32, int *flags,
                                                   WaveSync *ws) {
  __shared__ __align__(16) double D[SHKZ_TC], Sc[SHKZ_TC], A[SHKZ_TC], WX[SHKZ_TC], WY[SHKZ_TC], WZ[SHKZ_TC];
  __shared__ double hx[64], hy[64], hz[64], hsx[64], hsy[64], hsz[64];
  int slot, target;
  wave_begin(ws, slot, target);
  const int pt = sched[slot];
  const int tid = threadIdx.x, jj = tid & 7, kk = tid >> 3;
  const size_t tb = (size_t)pt * SHKZ_TC;
  load_tile_f64(Sc, colsum + tb);
  load_tile_f64(A, S.diag64 + tb);
  load_tile_f64(WX, S.offx64 + tb);
  load_tile_f64(WY, S.offy64 + tb);
  load_tile_f64(WZ, S.offz64 + tb);
  const int nb3[3] = {S.nbr[pt * 6 + NB_XM], S.nbr[pt * 6 + NB_YM], S.nbr[pt * 6 + NB_ZM]};
  wave_wait(ws, flags, nb3, target, slot);
  {
    // -x face (ii=7) indexed jj+8kk; -y face (jj=7) indexed ii+8kk; -z face (kk=7) indexed ii+8jj
    const int u = tid & 7, v = tid >> 3;
    const size_t cx = 7 + 8 * u + 64 * v, cy = u + 56 + 64 * v, cz = u + 8 * v + 448;
    hx[tid] = nb3[0] >= 0 ? __ldcg(d64 + (size_t)nb3[0] * SHKZ_TC + cx) : 0.0;
    hsx[tid] = nb3[0] >= 0 ? colsum[(size_t)nb3[0] * SHKZ_TC + cx] : 0.0;
    hy[tid] = nb3[1] >= 0 ? __ldcg(d64 + (size_t)nb3[1] * SHKZ_TC + cy) : 0.0;
    hsy[tid] = nb3[1] >= 0 ? colsum[(size_t)nb3[1] * SHKZ_TC + cy] : 0.0;
    hz[tid] = nb3[2] >= 0 ? __ldcg(d64 + (size_t)nb3[2] * SHKZ_TC + cz) : 0.0;
    hsz[tid] = nb3[2] >= 0 ? colsum[(size_t)nb3[2] * SHKZ_TC + cz] : 0.0;
  }
  __syncthreads();
  for (int s = 0; s < 22; ++s) {
    const int ii = s - jj - kk;
    if (ii >= 0 && ii < 8) {
      const int c = ii + 8 * jj + 64 * kk;
      const double dx_ = ii > 0 ? D[c - 1] : hx[jj + 8 * kk];
      const double sx_ = ii > 0 ? Sc[c - 1] : hsx[jj + 8 * kk];
      const double dy_ = jj > 0 ? D[c - 8] : hy[ii + 8 * kk];
      const double sy_ = jj > 0 ? Sc[c - 8] : hsy[ii + 8 * kk];
      const double dz_ = kk > 0 ? D[c - 64] : hz[ii + 8 * jj];
      const double sz_ = kk > 0 ? Sc[c - 64] : hsz[ii + 8 * jj];
      const double a = A[c], wx = WX[c], wy = WY[c], wz = WZ[c];
      double dv = 0.0;
      if (a != 0.0) {
        double piv = a;
        piv -= dx_ * wx * (wx + omega * (sx_ - wx));
        piv -= dy_ * wy * (wy + omega * (sy_ - wy));
        piv -= dz_ * wz * (wz + omega * (sz_ - wz));
        dv = (piv < min_ratio * a) ? 1.0 / a : 1.0 / piv;
      }
      D[c] = dv;
    }
    __syncthreads();
  }
  for (int c = tid; c < SHKZ_TC; c += 64) {
    d64[tb + c] = D[c];
    d32[tb + c] = (float)D[c];
  }
  wave_end(ws, flags, pt, target);
}

// Tile faces published with an epoch tag: entry = (epoch << 32) | float bits.
// A 64-bit store is single-copy atomic, so a consumer that reads the current
// epoch in an entry also reads that entry's value; no separate flag, fence or
// second load is needed between neighbouring tiles.
__device__ __forceinline__ void face_put(unsigned long long *e, int epoch, float v) {
  const unsigned long long w = ((unsigned long long)(unsigned)epoch << 32) | (unsigned long long)__float_as_uint(v);
  asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(e), "l"(w) : "memory");
}
// The three upstream (downstream) face entries of one thread, polled
// together: every round issues the loads of the entries still missing before
// it checks any of them, so once the last face lands the thread sees it one
// L2 round trip later, not one per face. e0/e1/e2 null: no neighbour (0).
__device__ __forceinline__ void face_get3(const unsigned long long *e0, const unsigned long long *e1,
                                          const unsigned long long *e2, int epoch, int limit, float &v0, float &v1,
                                          float &v2, bool &ok) {
  bool r0 = !e0, r1 = !e1, r2 = !e2;
  v0 = v1 = v2 = 0.0f;
  for (int it = 0; it < limit && !(r0 && r1 && r2); ++it) {
    unsigned long long w0 = 0ull, w1 = 0ull, w2 = 0ull;
    if (!r0) asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(w0) : "l"(e0) : "memory");
    if (!r1) asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(w1) : "l"(e1) : "memory");
    if (!r2) asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(w2) : "l"(e2) : "memory");
    if (!r0 && (int)(w0 >> 32) == epoch) { v0 = __uint_as_float((unsigned)(w0 & 0xffffffffu)); r0 = true; }
    if (!r1 && (int)(w1 >> 32) == epoch) { v1 = __uint_as_float((unsigned)(w1 & 0xffffffffu)); r1 = true; }
    if (!r2 && (int)(w2 >> 32) == epoch) { v2 = __uint_as_float((unsigned)(w2 & 0xffffffffu)); r2 = true; }
    if (it > 32) __nanosleep(32);
  }
  if (!(r0 && r1 && r2)) ok = false;
}

__device__ __forceinline__ void sweep_begin(WaveSync *ws, int &slot, int &epoch, int &limit) {
  __shared__ int s_slot, s_epoch, s_limit;
  if (threadIdx.x == 0) {
    s_slot = atomicAdd(&ws->slot, 1);
    s_epoch = *((volatile int *)&ws->epoch) + 1;
    s_limit = spin_rounds(ws);
  }
  __syncthreads();
  slot = s_slot;
  epoch = s_epoch;
  limit = s_limit;
}

__device__ __forceinline__ void sweep_end(WaveSync *ws, int epoch) {
  if (threadIdx.x == 0) {
    const unsigned f = atomicAdd(&ws->finished, 1u);
    if (f == gridDim.x - 1) {
      ws->slot = 0;
      ws->finished = 0;
      __threadfence();
      atomicExch(&ws->epoch, epoch);
    }
  }
}

// Forward sweep t = d (r + sum_lower w t) in FP32. faces: [K][3][64]
// (+x face ii=7 by jj+8kk, +y face jj=7 by ii+8kk, +z face kk=7 by ii+8jj).
__global__ void __launch_bounds__(64) k_mic_forward(PoolSystem S, const int *sched, const float *__restrict__ d32,
                                                    const float *__restrict__ r, float *__restrict__ t,
                                                    unsigned long long *faces, WaveSync *ws, const SolverState *st) {
  __shared__ __align__(16) float T[SHKZ_TC], R[SHKZ_TC], Dd[SHKZ_TC], WX[SHKZ_TC], WY[SHKZ_TC], WZ[SHKZ_TC];
  __shared__ float hx[64], hy[64], hz[64];
  if (st && st->done) return;
  int slot, epoch, limit;
  sweep_begin(ws, slot, epoch, limit);
  const int pt = sched[slot];
  const int tid = threadIdx.x, jj = tid & 7, kk = tid >> 3;
  const size_t tb = (size_t)pt * SHKZ_TC;
  load_tile_f32(R, r + tb);
  load_tile_f32(Dd, d32 + tb);
  load_tile_f32(WX, S.offx + tb);
  load_tile_f32(WY, S.offy + tb);
  load_tile_f32(WZ, S.offz + tb);
  {
    const int nxm = S.nbr[pt * 6 + NB_XM], nym = S.nbr[pt * 6 + NB_YM], nzm = S.nbr[pt * 6 + NB_ZM];
    bool ok = true;
    face_get3(nxm >= 0 ? faces + ((size_t)nxm * 3 + 0) * 64 + tid : nullptr,
              nym >= 0 ? faces + ((size_t)nym * 3 + 1) * 64 + tid : nullptr,
              nzm >= 0 ? faces + ((size_t)nzm * 3 + 2) * 64 + tid : nullptr, epoch, limit, hx[tid], hy[tid], hz[tid], ok);
    if (!ok) atomicCAS(&ws->error, 0, slot + 1);
  }
  __syncthreads();
  for (int s = 0; s < 22; ++s) {
    const int ii = s - jj - kk;
    if (ii >= 0 && ii < 8) {
      const int c = ii + 8 * jj + 64 * kk;
      const float tx = ii > 0 ? T[c - 1] : hx[jj + 8 * kk];
      const float ty = jj > 0 ? T[c - 8] : hy[ii + 8 * kk];
      const float tz = kk > 0 ? T[c - 64] : hz[ii + 8 * jj];
      T[c] = Dd[c] * (R[c] + WX[c] * tx + WY[c] * ty + WZ[c] * tz);
    }
    __syncthreads();
  }
  {
    unsigned long long *f = faces + (size_t)pt * 3 * 64;
    const int u = tid & 7, v = tid >> 3;
    face_put(f + 0 * 64 + tid, epoch, T[7 + 8 * u + 64 * v]);
    face_put(f + 1 * 64 + tid, epoch, T[u + 56 + 64 * v]);
    face_put(f + 2 * 64 + tid, epoch, T[u + 8 * v + 448]);
  }
  for (int v = tid; v < SHKZ_TC / 4; v += 64)
    reinterpret_cast<float4 *>(t + tb)[v] = reinterpret_cast<const float4 *>(T)[v];
  sweep_end(ws, epoch);
}

// Backward sweep z = t + d * sum_upper w z, reverse level order; fused z.r
// partial per tile into partials[pt]. faces: [K][3][64] (-x face ii=0,
// -y face jj=0, -z face kk=0, same indexing as the forward faces).
__global__ void __launch_bounds__(64) k_mic_backward(PoolSystem S, const int *sched, const float *__restrict__ d32,
                                                     const float *__restrict__ t, const float *__restrict__ r,
                                                     float *__restrict__ z, double *partials,
                                                     unsigned long long *faces, WaveSync *ws, const SolverState *st) {
  __shared__ __align__(16) float Z[SHKZ_TC], Tt[SHKZ_TC], Dd[SHKZ_TC], WX[SHKZ_TC], WY[SHKZ_TC], WZ[SHKZ_TC];
  __shared__ float hx[64], hy[64], hz[64], ux[64], uy[64], uz[64];
  __shared__ double red[2];
  if (st && st->done) return;
  int slot, epoch, limit;
  sweep_begin(ws, slot, epoch, limit);
  const int pt = sched[S.K - 1 - slot];
  const int tid = threadIdx.x, jj = tid & 7, kk = tid >> 3;
  const size_t tb = (size_t)pt * SHKZ_TC;
  const int nxp = S.nbr[pt * 6 + NB_XP], nyp = S.nbr[pt * 6 + NB_YP], nzp = S.nbr[pt * 6 + NB_ZP];
  load_tile_f32(Tt, t + tb);
  load_tile_f32(Dd, d32 + tb);
  load_tile_f32(WX, S.offx + tb);
  load_tile_f32(WY, S.offy + tb);
  load_tile_f32(WZ, S.offz + tb);
  {
    // upper weights across the tile faces: +x tile column ii=0, +y row jj=0, +z plane kk=0
    const int u = tid & 7, v = tid >> 3;
    ux[tid] = nxp >= 0 ? S.offx[(size_t)nxp * SHKZ_TC + 8 * u + 64 * v] : 0.0f;
    uy[tid] = nyp >= 0 ? S.offy[(size_t)nyp * SHKZ_TC + u + 64 * v] : 0.0f;
    uz[tid] = nzp >= 0 ? S.offz[(size_t)nzp * SHKZ_TC + u + 8 * v] : 0.0f;
    bool ok = true;
    face_get3(nxp >= 0 ? faces + ((size_t)nxp * 3 + 0) * 64 + tid : nullptr,
              nyp >= 0 ? faces + ((size_t)nyp * 3 + 1) * 64 + tid : nullptr,
              nzp >= 0 ? faces + ((size_t)nzp * 3 + 2) * 64 + tid : nullptr, epoch, limit, hx[tid], hy[tid], hz[tid], ok);
    if (!ok) atomicCAS(&ws->error, 0, slot + 1);
  }
  __syncthreads();
  for (int s = 21; s >= 0; --s) {
    const int ii = s - jj - kk;
    if (ii >= 0 && ii < 8) {
      const int c = ii + 8 * jj + 64 * kk;
      const float zx = ii < 7 ? Z[c + 1] : hx[jj + 8 * kk];
      const float wx = ii < 7 ? WX[c + 1] : ux[jj + 8 * kk];
      const float zy = jj < 7 ? Z[c + 8] : hy[ii + 8 * kk];
      const float wy = jj < 7 ? WY[c + 8] : uy[ii + 8 * kk];
      const float zz = kk < 7 ? Z[c + 64] : hz[ii + 8 * jj];
      const float wz = kk < 7 ? WZ[c + 64] : uz[ii + 8 * jj];
      Z[c] = Tt[c] + Dd[c] * (wx * zx + wy * zy + wz * zz);
    }
    __syncthreads();
  }
  {
    unsigned long long *f = faces + (size_t)pt * 3 * 64;
    const int u = tid & 7, v = tid >> 3;
    face_put(f + 0 * 64 + tid, epoch, Z[8 * u + 64 * v]);
    face_put(f + 1 * 64 + tid, epoch, Z[u + 64 * v]);
    face_put(f + 2 * 64 + tid, epoch, Z[u + 8 * v]);
  }
  double dot = 0.0;
  for (int v = tid; v < SHKZ_TC / 4; v += 64) {
    const float4 zv = reinterpret_cast<const float4 *>(Z)[v];
    const float4 rv = reinterpret_cast<const float4 *>(r + tb)[v];
    reinterpret_cast<float4 *>(z + tb)[v] = zv;
    dot += (double)zv.x * rv.x + (double)zv.y * rv.y + (double)zv.z * rv.z + (double)zv.w * rv.w;
  }
  #pragma unroll
  for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
  if ((tid & 31) == 0) red[tid >> 5] = dot;
  __syncthreads();
  if (tid == 0 && partials) partials[pt] = red[0] + red[1];
  sweep_end(ws, epoch);
}

// ---------------------------------------------------------------------------
// MIC(0) sweeps over 16^3 macro tiles (2x2x2 pool tiles per CTA).
//
// Same recurrences as the 8^3 kernels above, on four times as many cells per
// CTA (256 threads, one per x-row of 16 cells, 46 in-tile diagonals): the
// wavefront then crosses half as many tile levels, and the hand-off between
// levels -- not the arithmetic -- is what bounds a sweep. Shared memory holds
// the macro tile's six FP32 fields (96 KB); faces are 256 epoch-tagged words.

#define MT 16
#define MTC 4096
// Solution array of a macro tile with one ghost layer: cell (x, y, z),
// x, y, z in [-1, 16], at (x + 1) + 18 (y + 1) + 337 (z + 1). The ghosts hold
// the upstream faces, so the sweep's neighbour reads are unconditional. Along
// a diagonal (x = s - y - z) consecutive rows are 17 floats apart and the
// warp's second plane 336 = 16 (mod 32) further, so its 32 rows fall in 32
// distinct banks.
#define MGY 18
#define MGZ 337
#define MGC 6080            // >= 18 * 337, padded to 16 bytes
__device__ __forceinline__ int mghost(int x, int y, int z) { return (x + 1) + MGY * (y + 1) + MGZ * (z + 1); }

// macro tile counts = sum of the counts of its (up to) eight tiles
__global__ void k_macro_count(Geometry G, const int *tile_count, Geometry M, int *macro_count) {
  const long long n = M.ntiles;
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n; m += (long long)gridDim.x * blockDim.x) {
    const int mi = (int)(m % M.bx), mj = (int)((m / M.bx) % M.by), mk = (int)(m / ((long long)M.bx * M.by));
    int c = 0;
    for (int s = 0; s < 8; ++s) {
      const int ti = 2 * mi + (s & 1), tj = 2 * mj + ((s >> 1) & 1), tk = 2 * mk + (s >> 2);
      if (ti < G.bx && tj < G.by && tk < G.bz) c += tile_count[(long long)ti + (long long)G.bx * ((long long)tj + (long long)G.by * tk)];
    }
    macro_count[m] = c;
  }
}

__global__ void k_macro_sub(Geometry G, Geometry M, const int *macro_tile, int KM, const int *tile_state, int *msub) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= KM * 8) return;
  const int pm = e >> 3, s = e & 7;
  const long long m = macro_tile[pm];
  const int mi = (int)(m % M.bx), mj = (int)((m / M.bx) % M.by), mk = (int)(m / ((long long)M.bx * M.by));
  const int ti = 2 * mi + (s & 1), tj = 2 * mj + ((s >> 1) & 1), tk = 2 * mk + (s >> 2);
  int pt = -1;
  if (ti < G.bx && tj < G.by && tk < G.bz) pt = tile_state[(long long)ti + (long long)G.bx * ((long long)tj + (long long)G.by * tk)];
  msub[e] = pt;
}

// Stage five pool fields of the macro tile's sub-tiles into shared memory
// (index x + 16y + 256z); absent sub-tiles read as zero.
__device__ __forceinline__ void macro_load5(const int *sub, const float *s0, const float *s1, const float *s2,
                                            const float *s3, const float *s4, float *d0, float *d1, float *d2,
                                            float *d3, float *d4) {
  for (int e = threadIdx.x; e < 8 * 128; e += blockDim.x) {
    const int v = e & 127, st = e >> 7;
    const int pt = sub[st];
    const int c = v * 4;
    const int x = (c & 7) + (st & 1) * 8, y = ((c >> 3) & 7) + ((st >> 1) & 1) * 8, z = (c >> 6) + (st >> 2) * 8;
    const int o = x + 16 * y + 256 * z;
    float4 a0 = make_float4(0.f, 0.f, 0.f, 0.f), a1 = a0, a2 = a0, a3 = a0, a4 = a0;
    if (pt >= 0) {
      const size_t b = (size_t)pt * (SHKZ_TC / 4) + v;
      a0 = reinterpret_cast<const float4 *>(s0)[b];
      a1 = reinterpret_cast<const float4 *>(s1)[b];
      a2 = reinterpret_cast<const float4 *>(s2)[b];
      a3 = reinterpret_cast<const float4 *>(s3)[b];
      a4 = reinterpret_cast<const float4 *>(s4)[b];
    }
    *reinterpret_cast<float4 *>(d0 + o) = a0;
    *reinterpret_cast<float4 *>(d1 + o) = a1;
    *reinterpret_cast<float4 *>(d2 + o) = a2;
    *reinterpret_cast<float4 *>(d3 + o) = a3;
    *reinterpret_cast<float4 *>(d4 + o) = a4;
  }
}
// Fused PCG update while staging (forward sweep of an iteration): r -= alpha q
// and x += alpha p on the macro tile's cells, the new r staged for the sweep,
// written back, and its inf-norm / squared 2-norm returned for this thread.
__device__ __forceinline__ void macro_load_update(const int *sub, float *r, const float *q, const float *p, float *x,
                                                  float alpha, const float *s1, const float *s2, const float *s3,
                                                  const float *s4, float *d0, float *d1, float *d2, float *d3,
                                                  float *d4, double &m, double &s2sum) {
  for (int e = threadIdx.x; e < 8 * 128; e += blockDim.x) {
    const int v = e & 127, st = e >> 7;
    const int pt = sub[st];
    const int c = v * 4;
    const int xx = (c & 7) + (st & 1) * 8, y = ((c >> 3) & 7) + ((st >> 1) & 1) * 8, z = (c >> 6) + (st >> 2) * 8;
    const int o = xx + 16 * y + 256 * z;
    float4 a0 = make_float4(0.f, 0.f, 0.f, 0.f), a1 = a0, a2 = a0, a3 = a0, a4 = a0;
    if (pt >= 0) {
      const size_t b = (size_t)pt * (SHKZ_TC / 4) + v;
      float4 rv = reinterpret_cast<const float4 *>(r)[b];
      const float4 qv = reinterpret_cast<const float4 *>(q)[b];
      const float4 pv = reinterpret_cast<const float4 *>(p)[b];
      float4 xv = reinterpret_cast<const float4 *>(x)[b];
      a1 = reinterpret_cast<const float4 *>(s1)[b];
      a2 = reinterpret_cast<const float4 *>(s2)[b];
      a3 = reinterpret_cast<const float4 *>(s3)[b];
      a4 = reinterpret_cast<const float4 *>(s4)[b];
      // the expressions of k_update_xr
      xv.x += alpha * pv.x; xv.y += alpha * pv.y; xv.z += alpha * pv.z; xv.w += alpha * pv.w;
      rv.x -= alpha * qv.x; rv.y -= alpha * qv.y; rv.z -= alpha * qv.z; rv.w -= alpha * qv.w;
      reinterpret_cast<float4 *>(x)[b] = xv;
      reinterpret_cast<float4 *>(r)[b] = rv;
      m = fmax(m, fmax(fmax(fabs((double)rv.x), fabs((double)rv.y)), fmax(fabs((double)rv.z), fabs((double)rv.w))));
      s2sum += (double)rv.x * rv.x + (double)rv.y * rv.y + (double)rv.z * rv.z + (double)rv.w * rv.w;
      a0 = rv;
    }
    *reinterpret_cast<float4 *>(d0 + o) = a0;
    *reinterpret_cast<float4 *>(d1 + o) = a1;
    *reinterpret_cast<float4 *>(d2 + o) = a2;
    *reinterpret_cast<float4 *>(d3 + o) = a3;
    *reinterpret_cast<float4 *>(d4 + o) = a4;
  }
}

// Write the interior of a ghosted solution array back to the pool sub-tiles.
__device__ __forceinline__ void macro_store_ghosted(const int *sub, const float *srcg, float *dst) {
  for (int e = threadIdx.x; e < 8 * 128; e += blockDim.x) {
    const int v = e & 127, st = e >> 7;
    const int pt = sub[st];
    if (pt < 0) continue;
    const int c = v * 4;
    const int x = (c & 7) + (st & 1) * 8, y = ((c >> 3) & 7) + ((st >> 1) & 1) * 8, z = (c >> 6) + (st >> 2) * 8;
    const int o = mghost(x, y, z);
    reinterpret_cast<float4 *>(dst + (size_t)pt * SHKZ_TC)[v] = make_float4(srcg[o], srcg[o + 1], srcg[o + 2], srcg[o + 3]);
  }
}

__device__ __forceinline__ void macro_store(const int *sub, const float *srcs, float *dst) {
  for (int e = threadIdx.x; e < 8 * 128; e += blockDim.x) {
    const int v = e & 127, st = e >> 7;
    const int pt = sub[st];
    if (pt < 0) continue;
    const int c = v * 4;
    const int x = (c & 7) + (st & 1) * 8, y = ((c >> 3) & 7) + ((st >> 1) & 1) * 8, z = (c >> 6) + (st >> 2) * 8;
    reinterpret_cast<float4 *>(dst + (size_t)pt * SHKZ_TC)[v] = *reinterpret_cast<const float4 *>(srcs + x + 16 * y + 256 * z);
  }
}

// With fu != null the kernel also performs the preceding x/r update of the
// PCG iteration (k_update_xr's arithmetic and convergence bookkeeping, the
// last CTA reducing the norms); the update's extra loads sit in the staging
// phase, which overlaps the wait for the upstream faces.
struct SweepUpdate {
  const float *p, *q;
  const float *p_alt;  // non-null: p / p_alt are the two direction buffers, the current one
                       // chosen by the parity of st->iter + 1 (the stencil of this iteration wrote it)
  float *x, *r;
  SolverState *st;
  unsigned *counter;
  double *part;        // [2 * KM]: per-tile inf-norm, squared 2-norm
  int max_iterations;
};

__global__ void __launch_bounds__(256, 2) k_mic_forward16(PoolSystem S, const float *__restrict__ d32,
                                                       const float *__restrict__ r, float *__restrict__ t,
                                                       unsigned long long *faces, WaveSync *ws, const SolverState *st,
                                                       SweepUpdate fu) {
  extern __shared__ __align__(16) float smf[];
  float *Tg = smf, *R = Tg + MGC, *Dd = R + MTC, *WX = Dd + MTC, *WY = WX + MTC, *WZ = WY + MTC;
  __shared__ int sub[8];
  if (st && st->done) return;
  int slot, epoch, limit;
  sweep_begin(ws, slot, epoch, limit);
  const int mt = S.msched[slot];
  const int tid = threadIdx.x, jj = tid & 15, kk = tid >> 4;
  if (tid < 8) sub[tid] = S.msub[mt * 8 + tid];
  __syncthreads();
  if (fu.st) {
    __shared__ double red[8];
    double m = 0.0, s2 = 0.0;
    const float *pcur = (fu.p_alt && ((fu.st->iter + 1) & 1)) ? fu.p_alt : fu.p;
    macro_load_update(sub, fu.r, fu.q, pcur, fu.x, (float)fu.st->alpha, d32, S.offx, S.offy, S.offz, R, Dd, WX, WY,
                      WZ, m, s2);
    m = block_max<256>(m, red);
    s2 = block_sum<256>(s2, red);
    if (tid == 0) {
      fu.part[mt] = m;
      fu.part[S.KM + mt] = s2;
    }
  } else {
    macro_load5(sub, r, d32, S.offx, S.offy, S.offz, R, Dd, WX, WY, WZ);
  }
  __syncthreads();
  // The thread's x-row in registers, rotated by its wavefront offset
  // o = jj + kk: slot k holds cell (k - o) mod 16, so the cell of step s
  // (x = s - o) sits in slot s mod 16, a constant of the unrolled step loop.
  const int o = jj + kk;
  float cd[MT], cr[MT], cx[MT], cy[MT], cz[MT];
  {
    const int rb = MT * jj + MT * MT * kk;
    #pragma unroll
    for (int k = 0; k < MT; ++k) {
      const int c = rb + ((k - o) & (MT - 1));
      cd[k] = Dd[c]; cr[k] = R[c]; cx[k] = WX[c]; cy[k] = WY[c]; cz[k] = WZ[c];
    }
  }
  float tx;
  {
    const int nxm = S.mnbr[mt * 6 + NB_XM], nym = S.mnbr[mt * 6 + NB_YM], nzm = S.mnbr[mt * 6 + NB_ZM];
    const int u = tid & 15, v = tid >> 4;
    bool ok = true;
    float gx, gy, gz;
    face_get3(nxm >= 0 ? faces + ((size_t)nxm * 3 + 0) * 256 + tid : nullptr,
              nym >= 0 ? faces + ((size_t)nym * 3 + 1) * 256 + tid : nullptr,
              nzm >= 0 ? faces + ((size_t)nzm * 3 + 2) * 256 + tid : nullptr, epoch, limit, gx, gy, gz, ok);
    Tg[mghost(-1, u, v)] = gx;
    Tg[mghost(u, -1, v)] = gy;
    Tg[mghost(u, v, -1)] = gz;
    tx = gx;
    if (!ok) atomicCAS(&ws->error, 0, slot + 1);
  }
  __syncthreads();
  {
    const int gb = mghost(0, jj, kk) - o;
    #pragma unroll
    for (int s = 0; s < 3 * MT - 2; ++s) {
      if ((unsigned)(s - o) < (unsigned)MT) {
        const int g = s + gb, k = s & (MT - 1);
        const float ty = Tg[g - MGY], tz = Tg[g - MGZ];
        tx = cd[k] * (cr[k] + cx[k] * tx + cy[k] * ty + cz[k] * tz);
        Tg[g] = tx;
      }
      __syncthreads();
    }
  }
  if (*((volatile const int *)&ws->skip_publish) != slot + 1) {
    unsigned long long *f = faces + (size_t)mt * 3 * 256;
    const int u = tid & 15, v = tid >> 4;
    face_put(f + 0 * 256 + tid, epoch, Tg[mghost(15, u, v)]);
    face_put(f + 1 * 256 + tid, epoch, Tg[mghost(u, 15, v)]);
    face_put(f + 2 * 256 + tid, epoch, Tg[mghost(u, v, 15)]);
  }
  macro_store_ghosted(sub, Tg, t);
  if (fu.st && last_block(fu.counter)) {
    // the convergence bookkeeping of k_update_xr, on the new residual
    __shared__ double red2[8];
    double mm = 0.0, ss = 0.0;
    for (int i = tid; i < S.KM; i += 256) {
      mm = fmax(mm, fu.part[i]);
      ss += fu.part[S.KM + i];
    }
    mm = block_max<256>(mm, red2);
    ss = block_sum<256>(ss, red2);
    const bool nan = !(ss == ss);
    if (tid == 0) {
      SolverState *sw = fu.st;
      sw->rmax = nan ? CUDART_NAN : mm;
      sw->r2 = ss;
      sw->iter += 1;
      if (nan) { sw->done = 3; sw->status = -5; }
      else if (mm <= sw->tol_abs) sw->done = 1;
      else if (sw->iter >= fu.max_iterations) sw->done = 2;
      else if (mm < sw->ru_threshold) sw->done = 4;
      *fu.counter = 0;
    }
  }
  sweep_end(ws, epoch);
}

__global__ void __launch_bounds__(256, 2) k_mic_backward16(PoolSystem S, const float *__restrict__ d32,
                                                        const float *__restrict__ t, const float *__restrict__ r,
                                                        float *__restrict__ z, double *partials,
                                                        unsigned long long *faces, WaveSync *ws,
                                                        SolverState *st, unsigned *finish) {
  extern __shared__ __align__(16) float smb[];
  float *Zg = smb, *Tt = Zg + MGC, *Dd = Tt + MTC, *WX = Dd + MTC, *WY = WX + MTC, *WZ = WY + MTC;
  __shared__ int sub[8];
  __shared__ double red[8];
  if (st && st->done) return;
  int slot, epoch, limit;
  sweep_begin(ws, slot, epoch, limit);
  const int mt = S.msched[S.KM - 1 - slot];
  const int tid = threadIdx.x, jj = tid & 15, kk = tid >> 4;
  if (tid < 8) sub[tid] = S.msub[mt * 8 + tid];
  __syncthreads();
  // the upper weights come precomputed (launch_upper_weights): W?[c] is the
  // lower weight of the +x/+y/+z neighbour cell, across the macro face where
  // needed, so the sweep reads them at the cell's own index
  macro_load5(sub, t, d32, S.upx, S.upy, S.upz, Tt, Dd, WX, WY, WZ);
  const int nxp = S.mnbr[mt * 6 + NB_XP], nyp = S.mnbr[mt * 6 + NB_YP], nzp = S.mnbr[mt * 6 + NB_ZP];
  __syncthreads();
  // the thread's x-row in registers, rotated as in the forward sweep: slot k
  // holds cell (k - o) mod 16
  const int o = jj + kk;
  float ct[MT], cd[MT], cx[MT], cy[MT], cz[MT];
  {
    const int rb = MT * jj + MT * MT * kk;
    #pragma unroll
    for (int k = 0; k < MT; ++k) {
      const int c = rb + ((k - o) & (MT - 1));
      ct[k] = Tt[c]; cd[k] = Dd[c]; cx[k] = WX[c]; cy[k] = WY[c]; cz[k] = WZ[c];
    }
  }
  float zx;
  {
    const int u = tid & 15, v = tid >> 4;
    bool ok = true;
    float gx, gy, gz;
    face_get3(nxp >= 0 ? faces + ((size_t)nxp * 3 + 0) * 256 + tid : nullptr,
              nyp >= 0 ? faces + ((size_t)nyp * 3 + 1) * 256 + tid : nullptr,
              nzp >= 0 ? faces + ((size_t)nzp * 3 + 2) * 256 + tid : nullptr, epoch, limit, gx, gy, gz, ok);
    Zg[mghost(MT, u, v)] = gx;
    Zg[mghost(u, MT, v)] = gy;
    Zg[mghost(u, v, MT)] = gz;
    zx = gx;
    if (!ok) atomicCAS(&ws->error, 0, slot + 1);
  }
  __syncthreads();
  {
    const int gb = mghost(0, jj, kk) - o;
    #pragma unroll
    for (int s = 3 * MT - 3; s >= 0; --s) {
      if ((unsigned)(s - o) < (unsigned)MT) {
        const int g = s + gb, k = s & (MT - 1);
        const float zy = Zg[g + MGY], zz = Zg[g + MGZ];
        zx = ct[k] + cd[k] * (cx[k] * zx + cy[k] * zy + cz[k] * zz);
        Zg[g] = zx;
      }
      __syncthreads();
    }
  }
  {
    unsigned long long *f = faces + (size_t)mt * 3 * 256;
    const int u = tid & 15, v = tid >> 4;
    face_put(f + 0 * 256 + tid, epoch, Zg[mghost(0, u, v)]);
    face_put(f + 1 * 256 + tid, epoch, Zg[mghost(u, 0, v)]);
    face_put(f + 2 * 256 + tid, epoch, Zg[mghost(u, v, 0)]);
  }
  macro_store_ghosted(sub, Zg, z);
  // fused z.r over the macro tile's cells (absent sub-tiles contribute zero)
  double dot = 0.0;
  for (int e = tid; e < 8 * 128; e += 256) {
    const int v = e & 127, stt = e >> 7;
    const int pt = sub[stt];
    if (pt < 0) continue;
    const int c = v * 4;
    const int x = (c & 7) + (stt & 1) * 8, y = ((c >> 3) & 7) + ((stt >> 1) & 1) * 8, zc = (c >> 6) + (stt >> 2) * 8;
    const int o = mghost(x, y, zc);
    const float4 rv = reinterpret_cast<const float4 *>(r + (size_t)pt * SHKZ_TC)[v];
    dot += (double)Zg[o] * rv.x + (double)Zg[o + 1] * rv.y + (double)Zg[o + 2] * rv.z + (double)Zg[o + 3] * rv.w;
  }
  const double tot = block_sum<256>(dot, red);
  if (tid == 0 && partials) partials[mt] = tot;
  if (finish && last_block(finish)) {
    // k_finish_rho of the PCG iteration: rho_new = z.r from the macro-tile
    // partials in tile order, beta = rho_new / rho
    const double rho_new = sum_partials<256>(partials, S.KM, red);
    if (tid == 0) {
      st->beta = rho_new / st->rho;
      st->rho = rho_new;
      *finish = 0;
    }
  }
  sweep_end(ws, epoch);
}

// Upper weights of every pool cell: the lower weight of the +x/+y/+z
// neighbour cell (A(i, i+e) = -off?(i+e)), from the neighbour tile across a
// tile face, zero where that tile is not in the pool. They depend on the
// matrix only, so the backward MIC(0) sweep stages them instead of shifting
// the lower weights every iteration.
__global__ void __launch_bounds__(256) k_upper_weights(PoolSystem S, float *__restrict__ upx,
                                                       float *__restrict__ upy, float *__restrict__ upz) {
  const long long n = (long long)S.K * SHKZ_TC;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int pt = (int)(i >> 9), c = (int)(i & 511);
    const int ii = c & 7, jj = (c >> 3) & 7, kk = c >> 6;
    const size_t base = (size_t)pt * SHKZ_TC;
    float ux = 0.f, uy = 0.f, uz = 0.f;
    if (ii < 7) ux = S.offx[base + c + 1];
    else if (S.nbr[pt * 6 + NB_XP] >= 0) ux = S.offx[(size_t)S.nbr[pt * 6 + NB_XP] * SHKZ_TC + c - 7];
    if (jj < 7) uy = S.offy[base + c + 8];
    else if (S.nbr[pt * 6 + NB_YP] >= 0) uy = S.offy[(size_t)S.nbr[pt * 6 + NB_YP] * SHKZ_TC + c - 56];
    if (kk < 7) uz = S.offz[base + c + 64];
    else if (S.nbr[pt * 6 + NB_ZP] >= 0) uz = S.offz[(size_t)S.nbr[pt * 6 + NB_ZP] * SHKZ_TC + c - 448];
    upx[i] = ux;
    upy[i] = uy;
    upz[i] = uz;
  }
}

static int grid_for(long long n, int per, int cap);
void launch_upper_weights(const PoolSystem &S, float *upx, float *upy, float *upz, cudaStream_t s) {
  if (S.K <= 0) return;
  count_launches(1);
  k_upper_weights<<<grid_for((long long)S.K * SHKZ_TC, 256 * 4, 148 * 8), 256, 0, s>>>(S, upx, upy, upz);
}

size_t mic16_smem_forward() { return sizeof(float) * (MGC + 5 * MTC); }
size_t mic16_smem_backward() { return sizeof(float) * (MGC + 5 * MTC); }

// ---------------------------------------------------------------------------
// FP64 residual r64 = b64 - A64 x64 (x64 in FP64), its norms, and the FP32
// scaled copy r32 = r64 / ||r64||inf for the next inner solve.
__global__ void __launch_bounds__(256) k_residual64(PoolSystem S, const double *__restrict__ b, const double *__restrict__ x,
                                                    double *__restrict__ r, double *partials, unsigned *counter,
                                                    double *out3) {
  __shared__ double red[8];
  double m = 0.0, s2 = 0.0, bm = 0.0, b2 = 0.0;
  const size_t n = (size_t)S.K * SHKZ_TC;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    const int pt = (int)(o >> 9), c = (int)(o & 511);
    const int ii = c & 7, jj = (c >> 3) & 7, kk = c >> 6;
    auto xat = [&](int nbslot, int cell, bool inside) -> double {
      if (inside) return x[(size_t)pt * SHKZ_TC + cell];
      const int nb = S.nbr[pt * 6 + nbslot];
      return nb >= 0 ? x[(size_t)nb * SHKZ_TC + cell] : 0.0;
    };
    auto wat = [&](const double *w, int nbslot, int cell, bool inside) -> double {
      if (inside) return w[(size_t)pt * SHKZ_TC + cell];
      const int nb = S.nbr[pt * 6 + nbslot];
      return nb >= 0 ? w[(size_t)nb * SHKZ_TC + cell] : 0.0;
    };
    const double xc = x[o];
    double y = S.diag64[o] * xc;
    y -= S.offx64[o] * xat(NB_XM, ii > 0 ? c - 1 : c + 7, ii > 0);
    y -= S.offy64[o] * xat(NB_YM, jj > 0 ? c - 8 : c + 56, jj > 0);
    y -= S.offz64[o] * xat(NB_ZM, kk > 0 ? c - 64 : c + 448, kk > 0);
    {
      const int cell = ii < 7 ? c + 1 : c - 7;
      y -= wat(S.offx64, NB_XP, cell, ii < 7) * xat(NB_XP, cell, ii < 7);
    }
    {
      const int cell = jj < 7 ? c + 8 : c - 56;
      y -= wat(S.offy64, NB_YP, cell, jj < 7) * xat(NB_YP, cell, jj < 7);
    }
    {
      const int cell = kk < 7 ? c + 64 : c - 448;
      y -= wat(S.offz64, NB_ZP, cell, kk < 7) * xat(NB_ZP, cell, kk < 7);
    }
    const double bv = b[o];
    const double rv = S.diag64[o] != 0.0 ? bv - y : 0.0;
    r[o] = rv;
    m = fmax(m, fabs(rv));
    s2 += rv * rv;
    bm = fmax(bm, fabs(bv));
    b2 += bv * bv;
  }
  const double v0 = block_max<256>(m, red);
  const double v1 = block_sum<256>(s2, red);
  const double v2 = block_max<256>(bm, red);
  const double v3 = block_sum<256>(b2, red);
  if (threadIdx.x == 0) {
    partials[4 * blockIdx.x + 0] = v0;
    partials[4 * blockIdx.x + 1] = v1;
    partials[4 * blockIdx.x + 2] = v2;
    partials[4 * blockIdx.x + 3] = v3;
  }
  if (last_block(counter)) {
    double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += 256) {
      a0 = fmax(a0, partials[4 * i]);
      a1 += partials[4 * i + 1];
      a2 = fmax(a2, partials[4 * i + 2]);
      a3 += partials[4 * i + 3];
    }
    a0 = block_max<256>(a0, red);
    a1 = block_sum<256>(a1, red);
    a2 = block_max<256>(a2, red);
    a3 = block_sum<256>(a3, red);
    if (threadIdx.x == 0) {
      out3[0] = a0;
      out3[1] = a1;
      out3[2] = a2;
      out3[3] = a3;
      *counter = 0;
    }
  }
}

// Start of an inner FP32 solve on r32 = r64 * inv_scale; x32 = 0.
__global__ void __launch_bounds__(256) k_inner_init(int n, const double *__restrict__ r64, double inv_scale,
                                                    float *__restrict__ r32, float *__restrict__ x32) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    r32[i] = (float)(r64[i] * inv_scale);
    x32[i] = 0.0f;
  }
}

// x64 += scale * x32
__global__ void __launch_bounds__(256) k_accumulate(int n, const float *__restrict__ x32, double scale,
                                                    double *__restrict__ x64) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x64[i] += scale * (double)x32[i];
}

__global__ void __launch_bounds__(256) k_to_float(int n, const double *__restrict__ a, float *__restrict__ b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = (float)a[i];
}

// rmax0 and the absolute tolerance of an inner solve from r32 (= its rhs).
__global__ void __launch_bounds__(256) k_inner_setup(int n, const float *__restrict__ r, double *partials,
                                                     unsigned *counter, SolverState *st, double tol) {
  __shared__ double red[8];
  double m = 0.0, s2 = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    m = fmax(m, fabs((double)r[i]));
    s2 += (double)r[i] * r[i];
  }
  const double bm = block_max<256>(m, red);
  const double bs = block_sum<256>(s2, red);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = bm;
    partials[gridDim.x + blockIdx.x] = bs;
  }
  if (last_block(counter)) {
    double mm = 0.0, ss = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += 256) {
      mm = fmax(mm, partials[i]);
      ss += partials[gridDim.x + i];
    }
    mm = block_max<256>(mm, red);
    ss = block_sum<256>(ss, red);
    if (threadIdx.x == 0) {
      st->rmax0 = mm;
      st->rmax = mm;
      st->r2 = ss;
      st->tol_abs = tol * mm;
      st->iter = 0;
      st->done = (mm == 0.0) ? 1 : 0;
      st->status = (ss == ss) ? 0 : -5;
      if (!(ss == ss)) st->done = 3;
      st->rho = 0.0;
      st->beta = 0.0;
      st->ru_threshold = 0.0;
      *counter = 0;
    }
  }
}

// Host-directed state edits between batches (one thread).
__global__ void k_state_resume(SolverState *st, double ru_threshold, int iter_offset) {
  st->done = 0;
  st->ru_threshold = ru_threshold;
  (void)iter_offset;
}

// ---------------------------------------------------------------------------
// FP64 vector kernels (FP64 reference solve)

__global__ void __launch_bounds__(256) k_apply64(PoolSystem S, const double *__restrict__ x, double *__restrict__ y) {
  const size_t n = (size_t)S.K * SHKZ_TC;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    const int pt = (int)(o >> 9), c = (int)(o & 511);
    const int ii = c & 7, jj = (c >> 3) & 7, kk = c >> 6;
    auto at = [&](const double *v, int nbslot, int cell, bool inside) -> double {
      if (inside) return v[(size_t)pt * SHKZ_TC + cell];
      const int nb = S.nbr[pt * 6 + nbslot];
      return nb >= 0 ? v[(size_t)nb * SHKZ_TC + cell] : 0.0;
    };
    double v = S.diag64[o] * x[o];
    v -= S.offx64[o] * at(x, NB_XM, ii > 0 ? c - 1 : c + 7, ii > 0);
    v -= S.offy64[o] * at(x, NB_YM, jj > 0 ? c - 8 : c + 56, jj > 0);
    v -= S.offz64[o] * at(x, NB_ZM, kk > 0 ? c - 64 : c + 448, kk > 0);
    { const int cell = ii < 7 ? c + 1 : c - 7; v -= at(S.offx64, NB_XP, cell, ii < 7) * at(x, NB_XP, cell, ii < 7); }
    { const int cell = jj < 7 ? c + 8 : c - 56; v -= at(S.offy64, NB_YP, cell, jj < 7) * at(x, NB_YP, cell, jj < 7); }
    { const int cell = kk < 7 ? c + 64 : c - 448; v -= at(S.offz64, NB_ZP, cell, kk < 7) * at(x, NB_ZP, cell, kk < 7); }
    y[o] = v;
  }
}

// out[0] = a.b, out[1] = c.d (c may be null), out[2] = max|a|
__global__ void __launch_bounds__(256) k_dots64(int n, const double *__restrict__ a, const double *__restrict__ b,
                                                const double *__restrict__ c, const double *__restrict__ d,
                                                double *partials, unsigned *counter, double *out) {
  __shared__ double red[8];
  double s0 = 0.0, s1 = 0.0, m = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    s0 += a[i] * b[i];
    if (c) s1 += c[i] * d[i];
    m = fmax(m, fabs(a[i]));
  }
  s0 = block_sum<256>(s0, red);
  s1 = block_sum<256>(s1, red);
  m = block_max<256>(m, red);
  if (threadIdx.x == 0) {
    partials[3 * blockIdx.x] = s0;
    partials[3 * blockIdx.x + 1] = s1;
    partials[3 * blockIdx.x + 2] = m;
  }
  if (last_block(counter)) {
    double t0 = 0, t1 = 0, tm = 0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += 256) {
      t0 += partials[3 * i];
      t1 += partials[3 * i + 1];
      tm = fmax(tm, partials[3 * i + 2]);
    }
    t0 = block_sum<256>(t0, red);
    t1 = block_sum<256>(t1, red);
    tm = block_max<256>(tm, red);
    if (threadIdx.x == 0) {
      out[0] = t0;
      out[1] = t1;
      out[2] = tm;
      *counter = 0;
    }
  }
}

// y += alpha x ; r -= alpha q (fused, FP64)
__global__ void __launch_bounds__(256) k_axpy2_64(int n, double alpha, const double *__restrict__ x, double *__restrict__ y,
                                                  const double *__restrict__ q, double *__restrict__ r) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    y[i] += alpha * x[i];
    r[i] -= alpha * q[i];
  }
}
// y = x + beta y
__global__ void __launch_bounds__(256) k_xpby64(int n, const double *__restrict__ x, double beta, double *__restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = x[i] + beta * y[i];
}
// CSR loop on the device (CsrState): the reductions of k_dots64 in the same
// order, with the scalar updates of the host loop in the last block
__global__ void __launch_bounds__(256) k_csr_dots(int n, const double *__restrict__ a, const double *__restrict__ b,
                                                  const double *__restrict__ c, const double *__restrict__ d,
                                                  double *partials, unsigned *counter, CsrState *st, int phase) {
  __shared__ double red[8];
  if (st->done) return;
  double s0 = 0.0, s1 = 0.0, m = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    s0 += a[i] * b[i];
    if (c) s1 += c[i] * d[i];
    m = fmax(m, fabs(a[i]));
  }
  s0 = block_sum<256>(s0, red);
  s1 = block_sum<256>(s1, red);
  m = block_max<256>(m, red);
  if (threadIdx.x == 0) {
    partials[3 * blockIdx.x] = s0;
    partials[3 * blockIdx.x + 1] = s1;
    partials[3 * blockIdx.x + 2] = m;
  }
  if (last_block(counter)) {
    double t0 = 0, t1 = 0, tm = 0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += 256) {
      t0 += partials[3 * i];
      t1 += partials[3 * i + 1];
      tm = fmax(tm, partials[3 * i + 2]);
    }
    t0 = block_sum<256>(t0, red);
    t1 = block_sum<256>(t1, red);
    tm = block_max<256>(tm, red);
    if (threadIdx.x == 0) {
      if (phase == 0) {
        st->alpha = st->rho / t0;
      } else {
        // t1 = z.r, tm = max|r| (pcg_solver.h:262-281)
        st->rmax = tm;
        if (!(tm == tm)) {
          st->done = 3;
        } else if (tm <= st->tol) {
          st->it += 1;
          st->done = 1;
        } else {
          st->beta = t1 / st->rho;
          st->rho = t1;
          st->it += 1;
          if (st->it >= st->max_it) st->done = 2;
        }
      }
      *counter = 0;
    }
  }
}
__global__ void __launch_bounds__(256) k_csr_axpy2(int n, const CsrState *st, const double *__restrict__ x,
                                                   double *__restrict__ y, const double *__restrict__ q,
                                                   double *__restrict__ r) {
  if (st->done) return;
  const double alpha = st->alpha;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    y[i] += alpha * x[i];
    r[i] -= alpha * q[i];
  }
}
__global__ void __launch_bounds__(256) k_csr_xpby(int n, const double *__restrict__ x, const CsrState *st,
                                                  double *__restrict__ y) {
  if (st->done) return;
  const double beta = st->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = x[i] + beta * y[i];
}
// b32 = (float)(a64 * s)
__global__ void __launch_bounds__(256) k_scale_f64_f32(int n, const double *__restrict__ a, double s, float *__restrict__ b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = (float)(a[i] * s);
}
// b64 = (double)a32 * s
__global__ void __launch_bounds__(256) k_scale_f32_f64(int n, const float *__restrict__ a, double s, double *__restrict__ b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = (double)a[i] * s;
}

// ---------------------------------------------------------------------------
// Flexible PCG pieces (learned preconditioner)

// z.r and z.q (FP64); init: rho = z.r, beta = 0; else Polak-Ribiere
// beta = z.(r_new - r_old)/rho = -alpha z.q / rho (r_old = r_new + alpha q).
__global__ void __launch_bounds__(256) k_fpcg_dots(int n4, const float4 *__restrict__ z, const float4 *__restrict__ r,
                                                   const float4 *__restrict__ q, double *partials, unsigned *counter,
                                                   SolverState *st, int init) {
  __shared__ double red[8];
  if (st->done) return;
  double a = 0.0, b = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += gridDim.x * blockDim.x) {
    const float4 zv = z[i], rv = r[i];
    a += (double)zv.x * rv.x + (double)zv.y * rv.y + (double)zv.z * rv.z + (double)zv.w * rv.w;
    if (!(init & 1)) {
      const float4 qv = q[i];
      b += (double)zv.x * qv.x + (double)zv.y * qv.y + (double)zv.z * qv.z + (double)zv.w * qv.w;
    }
  }
  a = block_sum<256>(a, red);
  b = block_sum<256>(b, red);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = a;
    partials[2 * blockIdx.x + 1] = b;
  }
  if (last_block(counter)) {
    double ta = 0.0, tb = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += 256) {
      ta += partials[2 * i];
      tb += partials[2 * i + 1];
    }
    ta = block_sum<256>(ta, red);
    tb = block_sum<256>(tb, red);
    if (threadIdx.x == 0) {
      if (init & 1) {
        st->rho = ta;
        st->beta = 0.0;
      } else {
        st->beta = -st->alpha * tb / st->rho;
        st->rho = ta;
      }
      if (init & 2) {
        // guarded (learned) preconditioner: z.r not positive and finite is a
        // breakdown of the preconditioner, not of the solve (done = 5)
        if (!(ta > 0.0) || !(tb == tb) || ta > 1e300) st->done = 5;
      } else if (!(ta == ta) || ta == 0.0) {
        st->done = 3;
        if (!(ta == ta)) st->status = -5;
      }
      *counter = 0;
    }
  }
}

// Standard normal samples at unknown cells (diag != 0) from a counter-based hash.
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352dU; x ^= x >> 15; x *= 0x846ca68bU; x ^= x >> 16;
  return x;
}
__global__ void k_rand_unknowns(int n, const float *diag, uint32_t seed, float *e) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float v = 0.f;
    if (diag[i] != 0.f) {
      const uint32_t h1 = mix32((uint32_t)i * 2654435761u ^ seed), h2 = mix32(h1 ^ 0x9e3779b9u);
      const float u1 = ((h1 >> 8) + 1) * (1.0f / 16777217.0f), u2 = (h2 >> 8) * (1.0f / 16777216.0f);
      v = sqrtf(-2.f * logf(u1)) * cospif(2.f * u2);
    }
    e[i] = v;
  }
}
__global__ void k_scale_f32(int n, float *a, float s) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] *= s;
}
__global__ void k_axpby_f32(int n, float a, const float *x, float b, float *y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = a * x[i] + b * y[i];
}

// ---------------------------------------------------------------------------
// host launchers

static int grid_for(long long n, int per, int cap) {
  long long g = (n + per - 1) / per;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

int pool_count(const Geometry &G, const int *tile_count, int *scratch_bsum, int *d_total, cudaStream_t s) {
  const long long nt = G.ntiles;
  const int nb = (int)((nt + 1023) / 1024);
  count_launches(1);
  k_pool_blocksum<<<nb, 256, 0, s>>>(tile_count, nt, scratch_bsum);
  count_launches(1);
  k_pool_scan_blocks<<<1, 32, 0, s>>>(scratch_bsum, nb, d_total);
  int K = -1;
  if (cudaMemcpyAsync(&K, d_total, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return -1;
  if (cudaStreamSynchronize(s) != cudaSuccess) return -1;
  return K;
}

void pool_assign(const Geometry &G, const int *tile_count, int K, const int *scratch_bsum, int *tile_state,
                 int *pool_tile, int *nbr, int *level_count, int *sched, cudaStream_t s) {
  const long long nt = G.ntiles;
  const int nb = (int)((nt + 1023) / 1024);
  count_launches(1);
  k_pool_assign<<<nb, 1024, 0, s>>>(tile_count, nt, scratch_bsum, tile_state, pool_tile);
  const int nlev = G.bx + G.by + G.bz;
  cudaMemsetAsync(level_count, 0, sizeof(int) * (nlev + 1), s);
  if (K > 0) {
    count_launches(1);
    k_pool_neighbours<<<(K + 255) / 256, 256, 0, s>>>(G, tile_state, pool_tile, K, nbr, level_count);
    count_launches(1);
    k_level_scan<<<1, 32, 0, s>>>(level_count, nlev);
    count_launches(1);
    k_level_scatter<<<(K + 255) / 256, 256, 0, s>>>(G, pool_tile, K, level_count, sched);
  }
}

size_t wave_sync_bytes() { return sizeof(WaveSync); }

void launch_spmv(const PoolSystem &S, const float *p, float *q, double *partials, unsigned *counter, SolverState *st,
                 int mode, cudaStream_t s) {
  if (S.K <= 0) return;
  count_launches(1);
  k_spmv<<<spmv_grid(S.K), 128, 0, s>>>(S, p, q, partials, counter, st, mode, nullptr, nullptr);
}

void launch_spmv_update(const PoolSystem &S, float *p0, float *p1, const float *z, float *q, double *partials,
                        unsigned *counter, SolverState *st, cudaStream_t s) {
  if (S.K <= 0) return;
  count_launches(1);
  k_spmv<<<spmv_grid(S.K), 128, 0, s>>>(S, p0, q, partials, counter, st, 0, z, p1);
}

// one wave of resident CTAs looping over the tiles
int spmv_grid(int K) { return K < 148 * SPMV_CTAS_PER_SM ? K : 148 * SPMV_CTAS_PER_SM; }

void launch_update_xr(int n, const float *p, const float *q, float *x, float *r, double *partials, unsigned *counter,
                      SolverState *st, int max_iterations, cudaStream_t s) {
  const int n4 = n / 4;
  count_launches(1);
  k_update_xr<<<grid_for(n4, 256 * 4, 148 * 8), 256, 0, s>>>(n4, (const float4 *)p, (const float4 *)q, (float4 *)x,
                                                               (float4 *)r, partials, counter, st, max_iterations);
}

void launch_finish_rho(const double *partials, int n, SolverState *st, int init, cudaStream_t s) {
  count_launches(1);
  k_finish_rho<<<1, 1024, 0, s>>>(partials, n, st, init);
}
void launch_finish_rho_r2(SolverState *st, int init, cudaStream_t s) {
  count_launches(1);
  k_finish_rho_r2<<<1, 1, 0, s>>>(st, init);
}

void launch_update_p(int n, const float *z, float *p, const SolverState *st, cudaStream_t s) {
  const int n4 = n / 4;
  count_launches(1);
  k_update_p<<<grid_for(n4, 256 * 4, 148 * 8), 256, 0, s>>>(n4, (const float4 *)z, (float4 *)p, st);
}

void launch_mic_factor(const PoolSystem &S, double *colsum, double omega, double min_ratio, double *d64, float *d32,
                       int *flags, void *ws, cudaStream_t s) {
  if (S.K <= 0) return;
  count_launches(1);
  k_mic_colsum<<<S.K, 512, 0, s>>>(S, colsum);
  count_launches(1);
  k_mic_factor<<<S.K, 64, 0, s>>>(S, S.sched, colsum, omega, min_ratio, d64, d32, flags, (WaveSync *)ws);
}

void launch_mic_apply(const PoolSystem &S, const float *d32, const float *r, float *t, float *z, double *partials,
                      unsigned long long *faces_f, unsigned long long *faces_b, void *ws_f, void *ws_b,
                      const SolverState *st, cudaStream_t s) {
  if (S.K <= 0) return;
  if (S.KM > 0) {
    static bool attr[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr[dev]) {
      cudaFuncSetAttribute(k_mic_forward16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mic16_smem_forward());
      cudaFuncSetAttribute(k_mic_backward16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mic16_smem_backward());
      if (dev >= 0 && dev < 64) attr[dev] = true;
    }
    count_launches(2);
    k_mic_forward16<<<S.KM, 256, mic16_smem_forward(), s>>>(S, d32, r, t, S.mfaces_f, (WaveSync *)ws_f, st,
                                                             SweepUpdate{});
    k_mic_backward16<<<S.KM, 256, mic16_smem_backward(), s>>>(S, d32, t, r, z, partials, S.mfaces_b,
                                                               (WaveSync *)ws_b, const_cast<SolverState *>(st),
                                                               nullptr);
    return;
  }
  count_launches(1);
  k_mic_forward<<<S.K, 64, 0, s>>>(S, S.sched, d32, r, t, faces_f, (WaveSync *)ws_f, st);
  count_launches(1);
  k_mic_backward<<<S.K, 64, 0, s>>>(S, S.sched, d32, t, r, z, partials, faces_b, (WaveSync *)ws_b, st);
}

bool launch_mic_apply_update(const PoolSystem &S, const float *d32, float *r, float *t, float *z, double *partials,
                             const float *p, const float *p_alt, const float *q, float *x, unsigned *counter,
                             SolverState *st, int max_iterations, void *ws_f, void *ws_b, unsigned *finish,
                             cudaStream_t s) {
  if (S.K <= 0 || S.KM <= 0) return false;
  static bool attr[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || !attr[dev]) {
    cudaFuncSetAttribute(k_mic_forward16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mic16_smem_forward());
    cudaFuncSetAttribute(k_mic_backward16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mic16_smem_backward());
    if (dev >= 0 && dev < 64) attr[dev] = true;
  }
  SweepUpdate fu;
  fu.p = p;
  fu.p_alt = p_alt;
  fu.q = q;
  fu.x = x;
  fu.r = r;
  fu.st = st;
  fu.counter = counter;
  fu.part = partials;  // [2 KM]; the backward sweep then writes its z.r partials over [0, KM)
  fu.max_iterations = max_iterations;
  count_launches(2);
  k_mic_forward16<<<S.KM, 256, mic16_smem_forward(), s>>>(S, d32, r, t, S.mfaces_f, (WaveSync *)ws_f, st, fu);
  k_mic_backward16<<<S.KM, 256, mic16_smem_backward(), s>>>(S, d32, t, r, z, partials, S.mfaces_b, (WaveSync *)ws_b,
                                                             st, finish);
  return true;
}

void build_macro(const Geometry &G, const Geometry &M, const int *tile_count, const int *tile_state, int *macro_count,
                 int *macro_state, int *macro_tile, int *mnbr, int *level_count, int *msched, int *msub, int KM,
                 const int *bsum, cudaStream_t s) {
  pool_assign(M, macro_count, KM, bsum, macro_state, macro_tile, mnbr, level_count, msched, s);
  if (KM > 0) {
    count_launches(1);
    k_macro_sub<<<(KM * 8 + 255) / 256, 256, 0, s>>>(G, M, macro_tile, KM, tile_state, msub);
  }
}

void launch_macro_count(const Geometry &G, const int *tile_count, const Geometry &M, int *macro_count, cudaStream_t s) {
  count_launches(1);
  k_macro_count<<<grid_for(M.ntiles, 256, 148 * 8), 256, 0, s>>>(G, tile_count, M, macro_count);
}

void launch_residual64(const PoolSystem &S, const double *b, const double *x, double *r, double *partials,
                       unsigned *counter, double *out4, cudaStream_t s) {
  const long long n = (long long)S.K * SHKZ_TC;
  count_launches(1);
  k_residual64<<<grid_for(n, 256 * 4, 148 * 8), 256, 0, s>>>(S, b, x, r, partials, counter, out4);
}

void launch_inner_init(int n, const double *r64, double inv_scale, float *r32, float *x32, cudaStream_t s) {
  count_launches(1);
  k_inner_init<<<grid_for(n, 256 * 4, 148 * 8), 256, 0, s>>>(n, r64, inv_scale, r32, x32);
}
void launch_accumulate(int n, const float *x32, double scale, double *x64, cudaStream_t s) {
  count_launches(1);
  k_accumulate<<<grid_for(n, 256 * 4, 148 * 8), 256, 0, s>>>(n, x32, scale, x64);
}
void launch_to_float(int n, const double *a, float *b, cudaStream_t s) {
  count_launches(1);
  k_to_float<<<grid_for(n, 256 * 4, 148 * 8), 256, 0, s>>>(n, a, b);
}
void launch_state_resume(SolverState *st, double ru_threshold, cudaStream_t s) {
  count_launches(1);
  k_state_resume<<<1, 1, 0, s>>>(st, ru_threshold, 0);
}

void launch_inner_setup(int n, const float *r, double *partials, unsigned *counter, SolverState *st, double tol,
                        cudaStream_t s) {
  count_launches(1);
  k_inner_setup<<<grid_for(n, 256 * 4, 148 * 8), 256, 0, s>>>(n, r, partials, counter, st, tol);
}

}  // namespace shkz

namespace shkz {
void launch_apply64(const PoolSystem &S, const double *x, double *y, cudaStream_t s) {
  const long long n = (long long)S.K * SHKZ_TC;
  count_launches(1);
  k_apply64<<<grid_for(n, 256 * 4, 148 * 8), 256, 0, s>>>(S, x, y);
}
void launch_dots64(int n, const double *a, const double *b, const double *c, const double *d, double *partials,
                   unsigned *counter, double *out, cudaStream_t s) {
  count_launches(1);
  k_dots64<<<grid_for(n, 256 * 4, 148 * 8), 256, 0, s>>>(n, a, b, c, d, partials, counter, out);
}
void launch_axpy2_64(int n, double alpha, const double *x, double *y, const double *q, double *r, cudaStream_t s) {
  count_launches(1);
  k_axpy2_64<<<grid_for(n, 256 * 4, 148 * 8), 256, 0, s>>>(n, alpha, x, y, q, r);
}
void launch_xpby64(int n, const double *x, double beta, double *y, cudaStream_t s) {
  count_launches(1);
  k_xpby64<<<grid_for(n, 256 * 4, 148 * 8), 256, 0, s>>>(n, x, beta, y);
}
void launch_csr_dots(int n, const double *a, const double *b, const double *c, const double *d, double *partials,
                     unsigned *counter, CsrState *st, int phase, cudaStream_t s) {
  count_launches(1);
  k_csr_dots<<<grid_for(n, 256 * 4, 148 * 8), 256, 0, s>>>(n, a, b, c, d, partials, counter, st, phase);
}
void launch_csr_axpy2(int n, const CsrState *st, const double *x, double *y, const double *q, double *r,
                      cudaStream_t s) {
  count_launches(1);
  k_csr_axpy2<<<grid_for(n, 256 * 4, 148 * 8), 256, 0, s>>>(n, st, x, y, q, r);
}
void launch_csr_xpby(int n, const double *x, const CsrState *st, double *y, cudaStream_t s) {
  count_launches(1);
  k_csr_xpby<<<grid_for(n, 256 * 4, 148 * 8), 256, 0, s>>>(n, x, st, y);
}
void launch_scale_f64_f32(int n, const double *a, double sc, float *b, cudaStream_t s) {
  count_launches(1);
  k_scale_f64_f32<<<grid_for(n, 256 * 4, 148 * 8), 256, 0, s>>>(n, a, sc, b);
}
void launch_scale_f32_f64(int n, const float *a, double sc, double *b, cudaStream_t s) {
  count_launches(1);
  k_scale_f32_f64<<<grid_for(n, 256 * 4, 148 * 8), 256, 0, s>>>(n, a, sc, b);
}
}  // namespace shkz

namespace shkz {
void launch_fpcg_dots(int n, const float *z, const float *r, const float *q, double *partials, unsigned *counter,
                      SolverState *st, int init, cudaStream_t s) {
  const int n4 = n / 4;
  count_launches(1);
  k_fpcg_dots<<<grid_for(n4, 256 * 4, 148 * 8), 256, 0, s>>>(n4, (const float4 *)z, (const float4 *)r,
                                                               (const float4 *)q, partials, counter, st, init);
}
void launch_rand_unknowns(int n, const float *diag, unsigned seed, float *e, cudaStream_t s) {
  count_launches(1);
  k_rand_unknowns<<<grid_for(n, 256 * 4, 148 * 8), 256, 0, s>>>(n, diag, seed, e);
}
void launch_scale_f32(int n, float *a, float sc, cudaStream_t s) {
  count_launches(1);
  k_scale_f32<<<grid_for(n, 256 * 4, 148 * 8), 256, 0, s>>>(n, a, sc);
}
void launch_axpby_f32(int n, float a, const float *x, float b, float *y, cudaStream_t s) {
  count_launches(1);
  k_axpby_f32<<<grid_for(n, 256 * 4, 148 * 8), 256, 0, s>>>(n, a, x, b, y);
}
}  // namespace shkz
