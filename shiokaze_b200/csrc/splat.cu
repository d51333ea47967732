// FLIP splat before the projection, as the liquid solver runs it
// (src/liquid/macflipliquid3.cpp:135-151): macnbflip3::splat
// (src/flip/macnbflip3.cpp:103-148) over the edge hash of
// pointgridhash3 (src/pointgridhash/pointgridhash3.cpp:90-100, 218-231),
// then the combined grid velocity.
//
// Built with -fmad=false: the reference accumulates FP64 products into FP32
// sums in a fixed order (each bucket's particles by index, buckets in its
// neighbour-query order); these kernels keep that order and round after every
// operation, so the splatted mass, momentum and velocity are bit-identical.
//
// Device pipeline, one call:
//   bin      one thread per particle: reads its record (the reference's own
//            84-byte layout, or any stride), packs (p, mass) and per axis
//            (u_d, c_d) into float4s, finds its edge bucket per axis and
//            takes a slot in it with an atomic counter, and marks the 8 faces
//            per axis it activates;
//   scan     in each tile of buckets a particle reached, the counters into
//            offsets inside the tile; then the tiles' starts;
//   scatter  every particle index into its bucket's slot;
//   sort     one thread per slot: the slot's particle goes to the rank its
//            index has in the bucket (the atomic slots are in arrival order)
//            and its packed data is copied there, so each bucket is
//            contiguous and in the reference's order;
//   compact  the activated faces of each axis into a list, then the list
//            ordered by work class (particle visits per face);
//   gather   one thread per listed face: visits the 16 buckets of the
//            neighbour query in the reference's loop order (8 distinct ones,
//            each twice: the query's loops run over all three axes but the
//            bucket does not move along the face's own axis), sums
//            tent-weighted mass and momentum (APIC term included), and
//            combines with the grid velocity in place;
//   clear    the reached tiles' counters back to zero.
// Faces are dense, x fastest; axis d has (nx+(d==0)) x (ny+(d==1)) x
// (nz+(d==2)) entries. Edge buckets of axis d cover (nx+(d!=0)) x
// (ny+(d!=1)) x (nz+(d!=2)) edges, grouped in 8x8x8 tiles (bucket_slot); the
// three axes' tiles are numbered one after another. Only tiles that hold a
// particle are scanned and cleared, so the bucket bookkeeping costs in
// proportion to the particles' band, not to the grid.
#include <cmath>

#include "common.cuh"
#include "kernels.h"

namespace shkz {

namespace {

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ float rec_f(const unsigned char *rec, int off, int k) {
  return __ldg(reinterpret_cast<const float *>(rec + off) + k);
}

// Division by the cell size. When dx is a power of two, a / dx and
// a * (1 / dx) are the same real number, so their correctly rounded results
// are equal: the multiply stands in for the FP64 divide, bit for bit.
struct DxDiv {
  double dx, inv;
  int pow2;
};

template <bool POW2>
__device__ __forceinline__ double div_dx(double a, const DxDiv &X) {
  return POW2 ? a * X.inv : a / X.dx;
}

// shape3::find_edge(p/dx, dim) on one axis (include/shiokaze/math/shape.h:
// 748-750): p/dx rounded to FP32, plus 0.5 off the edge's own axis rounded to
// FP32, truncated, clamped to the edge grid.
__device__ __forceinline__ int edge_axis(float pc, const DxDiv &X, bool half, int extent) {
  const double pd = X.pow2 ? div_dx<true>((double)pc, X) : div_dx<false>((double)pc, X);
  const float q = __double2float_rn(pd);
  const float t = __double2float_rn((double)q + (half ? 0.5 : 0.0));
  return clampi((int)t, 0, extent - 1);
}

// one factor of macnbflip3::grid_kernel (macnbflip3.cpp:44-49)
template <bool POW2>
__device__ __forceinline__ double tent(float r, const DxDiv &X) {
  const double v = 1.0 - div_dx<POW2>(fabs((double)r), X);
  return 0.0 < v ? v : 0.0;
}

// Slot of the edge bucket e (edge coordinates on axis d, extents E): the
// edge's 8x8x8 tile, numbered x fastest after the earlier axes' tiles, times
// 512, plus the edge's place in the tile (x fastest).
__device__ __forceinline__ int bucket_slot(const SplatBuffers &B, int d, const int E[3], const int e[3]) {
  const long long T0 = (E[0] + 7) >> 3, T1 = (E[1] + 7) >> 3;
  const long long tile = B.tile_base[d] + (e[0] >> 3) + T0 * ((e[1] >> 3) + T1 * (e[2] >> 3));
  return (int)((tile << 9) | (e[0] & 7) | ((e[1] & 7) << 3) | ((e[2] & 7) << 6));
}

// [first, end) of a bucket's particles in the bucket-ordered list. In a tile
// no particle reached every count is zero, so the range is empty.
__device__ __forceinline__ int2 bucket_range(const SplatBuffers &B, int slot) {
  const int t = slot >> 9;
  const int t0 = __ldg(B.tile_start + t);
  const int first = t0 + __ldg(B.count + slot);
  const int end = (slot & 511) == 511 ? __ldg(B.tile_start + t + 1) : t0 + __ldg(B.count + slot + 1);
  return make_int2(first, end);
}

__global__ void k_splat_bin(SplatRecords R, int nx, int ny, int nz, DxDiv X, SplatBuffers B) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= R.count) return;
  const unsigned char *rec = R.base + (size_t)n * R.stride;
  const float p[3] = {rec_f(rec, R.off_p, 0), rec_f(rec, R.off_p, 1), rec_f(rec, R.off_p, 2)};
  B.posm[n] = make_float4(p[0], p[1], p[2], rec_f(rec, R.off_m, 0));
  const bool splats = R.splat_bullet || R.off_bullet < 0 || rec[R.off_bullet] == 0;
  const int n3[3] = {nx, ny, nz};
  #pragma unroll
  for (int d = 0; d < 3; ++d) {
    float4 vc = make_float4(rec_f(rec, R.off_v, d), 0.f, 0.f, 0.f);
    if (R.off_c >= 0) {
      vc.y = rec_f(rec, R.off_c, 3 * d + 0);
      vc.z = rec_f(rec, R.off_c, 3 * d + 1);
      vc.w = rec_f(rec, R.off_c, 3 * d + 2);
    }
    B.vc[d][n] = vc;
    const size_t slot = (size_t)d * R.count + n;
    if (!splats) {
      B.key[slot] = -1;
      continue;
    }
    int e[3], E[3];
    #pragma unroll
    for (int c = 0; c < 3; ++c) {
      E[c] = n3[c] + (c != d);
      e[c] = edge_axis(p[c], X, c != d, E[c]);
    }
    const int key = bucket_slot(B, d, E, e);
    B.key[slot] = key;
    const int rank = atomicAdd(&B.count[key], 1);
    B.rank[slot] = rank;
    if (rank == 0) B.tile_act[key >> 9] = 1;
    // faces this particle activates (macnbflip3.cpp:109-120): the cell below
    // the face-centred position and its +1 neighbours, clamped to the cells
    int pi[3];
    #pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double pd = X.pow2 ? div_dx<true>((double)p[c], X) : div_dx<false>((double)p[c], X);
      pi[c] = (int)(pd - (c != d ? 0.5 : 0.0));
    }
    const int fw = nx + (d == 0), fh = ny + (d == 1);
    uint8_t *act = B.act[d];
    #pragma unroll
    for (int o = 0; o < 8; ++o) {
      const int i = clampi(pi[0] + (o >> 2), 0, nx - 1);
      const int j = clampi(pi[1] + ((o >> 1) & 1), 0, ny - 1);
      const int k = clampi(pi[2] + (o & 1), 0, nz - 1);
      act[(size_t)i + (size_t)fw * ((size_t)j + (size_t)fh * k)] = 1;
    }
  }
}

// --- exclusive scan of int counters, in place (three launches) -------------
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// exclusive prefix sum over the NT threads of a block; total = block sum
template <int NT>
__device__ __forceinline__ int block_exclusive(int v, int *warp_sums, int &total) {
  constexpr int NW = NT / 32;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
  #pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = lane < NW ? warp_sums[lane] : 0;
    #pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < NW) warp_sums[lane] = s;
  }
  __syncthreads();
  total = warp_sums[NW - 1];
  const int before = (w > 0 ? warp_sums[w - 1] : 0) + x - v;
  __syncthreads();
  return before;
}

// 8 consecutive counters of one thread: two 16-byte accesses when all are in
// range (the buffer starts 16-byte aligned and every thread's run starts on
// a 32-byte boundary), else one at a time
__device__ __forceinline__ void load8(const int *data, long long base, long long n, int v[kScanItems]) {
  if (base + kScanItems <= n) {
    const int4 a = *reinterpret_cast<const int4 *>(data + base);
    const int4 b = *reinterpret_cast<const int4 *>(data + base + 4);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
  } else {
    #pragma unroll
    for (int q = 0; q < kScanItems; ++q) v[q] = base + q < n ? data[base + q] : 0;
  }
}

__device__ __forceinline__ void store8(int *data, long long base, long long n, const int v[kScanItems]) {
  if (base + kScanItems <= n) {
    *reinterpret_cast<int4 *>(data + base) = make_int4(v[0], v[1], v[2], v[3]);
    *reinterpret_cast<int4 *>(data + base + 4) = make_int4(v[4], v[5], v[6], v[7]);
  } else {
    #pragma unroll
    for (int q = 0; q < kScanItems; ++q)
      if (base + q < n) data[base + q] = v[q];
  }
}

// each tile of kScanTile counters: local exclusive scan, tile total out
__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(int *data, long long n, int *tile_sums) {
  __shared__ int warp_sums[32];
  const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
  int v[kScanItems];
  load8(data, base, n, v);
  int s = 0;
  #pragma unroll
  for (int q = 0; q < kScanItems; ++q) s += v[q];
  int total;
  int run = block_exclusive<kScanThreads>(s, warp_sums, total);
  #pragma unroll
  for (int q = 0; q < kScanItems; ++q) {
    const int c = v[q];
    v[q] = run;
    run += c;
  }
  store8(data, base, n, v);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// the tile totals, in one block, chunk by chunk with a carry
__global__ void __launch_bounds__(kScanThreads) k_scan_tile_sums(int *tile_sums, int tiles) {
  __shared__ int warp_sums[32];
  int carry = 0;
  for (int c0 = 0; c0 < tiles; c0 += kScanThreads) {
    const int i = c0 + threadIdx.x;
    const int v = i < tiles ? tile_sums[i] : 0;
    int total;
    const int ex = block_exclusive<kScanThreads>(v, warp_sums, total);
    if (i < tiles) tile_sums[i] = carry + ex;
    carry += total;
  }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_add(int *data, long long n, const int *tile_sums) {
  const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
  const int add = tile_sums[blockIdx.x];
  int v[kScanItems];
  load8(data, base, n, v);
  #pragma unroll
  for (int q = 0; q < kScanItems; ++q) v[q] += add;
  store8(data, base, n, v);
}

// One warp per tile of 512 bucket counters. A tile that a particle reached
// turns its counters into offsets inside the tile and writes its particle
// total; every other tile's total is zero without reading its counters. The
// entry after the last tile is zero as well, so that the exclusive scan of the
// totals leaves the particle total there.
constexpr int kTileWarps = 8;

__global__ void __launch_bounds__(32 * kTileWarps) k_splat_tile_scan(SplatBuffers B) {
  const long long t = (long long)blockIdx.x * kTileWarps + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (t > B.tiles) return;
  if (t == B.tiles || !B.tile_act[t]) {
    if (lane == 0) B.tile_start[t] = 0;
    return;
  }
  // 16 counters a lane: the buffer is 16-byte aligned and a tile is 2 KB
  int4 *c = reinterpret_cast<int4 *>(B.count + (t << 9) + lane * 16);
  int v[16];
  #pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int4 a = c[q];
    v[4 * q] = a.x;
    v[4 * q + 1] = a.y;
    v[4 * q + 2] = a.z;
    v[4 * q + 3] = a.w;
  }
  int sum = 0;
  #pragma unroll
  for (int q = 0; q < 16; ++q) sum += v[q];
  int x = sum;
  #pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  int run = x - sum;
  #pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int k = v[q];
    v[q] = run;
    run += k;
  }
  #pragma unroll
  for (int q = 0; q < 4; ++q) c[q] = make_int4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
  if (lane == 31) B.tile_start[t] = x;
}

// the reached tiles' counters and flags back to zero for the next call
__global__ void __launch_bounds__(32 * kTileWarps) k_splat_tile_clear(SplatBuffers B) {
  const long long t = (long long)blockIdx.x * kTileWarps + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (t >= B.tiles || !B.tile_act[t]) return;
  int4 *c = reinterpret_cast<int4 *>(B.count + (t << 9) + lane * 16);
  #pragma unroll
  for (int q = 0; q < 4; ++q) c[q] = make_int4(0, 0, 0, 0);
  __syncwarp();
  if (lane == 0) B.tile_act[t] = 0;
}

__global__ void k_splat_scatter(long long count, SplatBuffers B) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= count) return;
  #pragma unroll
  for (int d = 0; d < 3; ++d) {
    const size_t slot = (size_t)d * count + n;
    const int key = B.key[slot];
    if (key >= 0) B.list[bucket_range(B, key).x + B.rank[slot]] = (int)slot;
  }
}

// One thread per bucket slot: the slot's particle goes to the position its
// index takes among its bucket's particles (the atomic slots are in arrival
// order), and its packed data is copied there, so that the gather reads each
// bucket contiguously and in the reference's order.
__global__ void k_splat_sort_copy(long long count, SplatBuffers B) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int total = B.tile_start[B.tiles];
  if (s >= total) return;
  const int sl = B.list[s];  // d * count + particle
  const int d = (int)(sl / count);
  const long long n = sl - d * count;
  const int2 range = bucket_range(B, B.key[sl]);
  const int s0 = range.x, s1 = range.y;
  if (s1 - s0 > kSplatBucketLimit) {
    // refused (the call returns SHKZ_B200_ERR_LIMIT and the gather writes nothing)
    if (s == s0) B.nfaces[3] = 1;
    return;
  }
  // one bucket holds one axis' entries, so d * count + particle orders them by particle
  int r = 0;
  for (int t = s0; t < s1; ++t) r += B.list[t] < sl;
  B.sposm[s0 + r] = B.posm[n];
  B.svc[s0 + r] = B.vc[d][n];
}

// active faces of axis D into a list: 16 faces a thread, one atomic a block
// (the order of blocks is arbitrary: every face is computed on its own, so
// the order only affects locality)
constexpr int kCompactThreads = 256;

template <int D>
__global__ void __launch_bounds__(kCompactThreads) k_splat_compact(int nx, int ny, int nz, SplatBuffers B) {
  __shared__ int warp_sums[kCompactThreads / 32];
  __shared__ int block_base;
  const size_t nf = (size_t)(nx + (D == 0)) * (ny + (D == 1)) * (nz + (D == 2));
  const size_t f0 = ((size_t)blockIdx.x * kCompactThreads + threadIdx.x) * 16;
  uint8_t a[16];
  if (f0 + 16 <= nf) {
    // act[D] comes from cudaMalloc and f0 is a multiple of 16
    const uint4 q = *reinterpret_cast<const uint4 *>(B.act[D] + f0);
    memcpy(a, &q, 16);
  } else {
    #pragma unroll
    for (int k = 0; k < 16; ++k) a[k] = f0 + k < nf ? B.act[D][f0 + k] : 0;
  }
  int c = 0;
  #pragma unroll
  for (int k = 0; k < 16; ++k) c += a[k] != 0;
  int total;
  int at = block_exclusive<kCompactThreads>(c, warp_sums, total);
  if (threadIdx.x == 0) block_base = total ? atomicAdd(&B.nfaces[D], total) : 0;
  __syncthreads();
  int *out = B.faces + B.face_off[D] + block_base;
  #pragma unroll
  for (int k = 0; k < 16; ++k)
    if (a[k]) out[at++] = (int)(f0 + k);
}

// Coordinates of the 8 distinct buckets a face of axis D reads, numbered
// 4 * (dir + 1) + 2 * ra + rb with ra, rb the offsets along the two other
// axes in increasing axis order.
template <int D>
__device__ __forceinline__ void bucket_coords(int k, const int fi[3], int q[3]) {
  const int dir = (k >> 2) - 1, ra = (k >> 1) & 1, rb = k & 1;
  if (D == 0) { q[0] = fi[0] + dir; q[1] = fi[1] + ra; q[2] = fi[2] + rb; }
  if (D == 1) { q[0] = fi[0] + ra; q[1] = fi[1] + dir; q[2] = fi[2] + rb; }
  if (D == 2) { q[0] = fi[0] + ra; q[1] = fi[1] + rb; q[2] = fi[2] + dir; }
}

// Work classes: a face's particle visits (twice the particles of its 8
// distinct buckets) in classes of 4, heaviest first. Listing the faces class
// by class gives the 32 faces of a warp nearly equal work, so its lanes
// finish together.
template <int D>
__device__ __forceinline__ int face_visits(size_t f, int nx, int ny, int nz, const SplatBuffers &B) {
  const int fw = nx + (D == 0), fh = ny + (D == 1);
  const int E[3] = {nx + (D != 0), ny + (D != 1), nz + (D != 2)};
  const int fi[3] = {(int)(f % fw), (int)((f / fw) % fh), (int)(f / ((size_t)fw * fh))};
  int total = 0;
  #pragma unroll
  for (int k = 0; k < 8; ++k) {
    int q[3];
    bucket_coords<D>(k, fi, q);
    if (q[0] < 0 || q[0] >= E[0] || q[1] < 0 || q[1] >= E[1] || q[2] < 0 || q[2] >= E[2]) continue;
    const int2 r = bucket_range(B, bucket_slot(B, D, E, q));
    total += r.y - r.x;
  }
  return 2 * total;
}

template <int D>
__global__ void __launch_bounds__(256) k_splat_face_work(int nx, int ny, int nz, SplatBuffers B) {
  __shared__ int hist[kSplatWorkBins];
  for (int i = threadIdx.x; i < kSplatWorkBins; i += blockDim.x) hist[i] = 0;
  __syncthreads();
  const int nact = B.nfaces[D];
  const int *faces = B.faces + B.face_off[D];
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nact; t += gridDim.x * blockDim.x) {
    const int visits = face_visits<D>((size_t)faces[t], nx, ny, nz, B);
    const int bin = kSplatWorkBins - 1 - min(visits >> 2, kSplatWorkBins - 1);
    B.face_bin[B.face_off[D] + t] = bin;
    atomicAdd(&hist[bin], 1);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kSplatWorkBins; i += blockDim.x)
    if (hist[i]) atomicAdd(&B.work[D * kSplatWorkBins + i], hist[i]);
}

// class counts into class cursors (exclusive), one warp per axis
__global__ void k_splat_work_scan(SplatBuffers B) {
  const int d = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (d >= 3) return;
  int *w = B.work + d * kSplatWorkBins;
  int carry = 0;
  for (int c0 = 0; c0 < kSplatWorkBins; c0 += 32) {
    const int v = w[c0 + lane];
    int x = v;
    #pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    w[c0 + lane] = carry + x - v;
    carry += __shfl_sync(0xffffffffu, x, 31);
  }
}

// Faces into class order. A block counts its faces per class in shared
// memory, reserves each class's run in one global atomic, and places its
// faces with shared-memory cursors (the global cursors would serialise on a
// few addresses).
template <int D>
__global__ void __launch_bounds__(256) k_splat_face_sort(SplatBuffers B) {
  __shared__ int cnt[kSplatWorkBins];
  __shared__ int cur[kSplatWorkBins];
  const int nact = B.nfaces[D];
  const int *faces = B.faces + B.face_off[D];
  const int *bins = B.face_bin + B.face_off[D];
  const int stride = gridDim.x * blockDim.x;
  for (int c0 = blockIdx.x * blockDim.x; c0 < nact; c0 += stride) {
    for (int i = threadIdx.x; i < kSplatWorkBins; i += blockDim.x) cnt[i] = 0;
    __syncthreads();
    const int t = c0 + threadIdx.x;
    const int bin = t < nact ? bins[t] : -1;
    if (bin >= 0) atomicAdd(&cnt[bin], 1);
    __syncthreads();
    for (int i = threadIdx.x; i < kSplatWorkBins; i += blockDim.x)
      cur[i] = cnt[i] ? atomicAdd(&B.work[D * kSplatWorkBins + i], cnt[i]) : 0;
    __syncthreads();
    if (bin >= 0) B.sorted[B.face_off[D] + atomicAdd(&cur[bin], 1)] = faces[t];
    __syncthreads();
  }
}

// The 16 visits of get_face_neighbors (pointgridhash3.cpp:218-231), in its
// loop order dir, ri, rj, rk, reach the 8 distinct buckets of bucket_coords:
// the loop variable of the face's own axis D does not move the bucket.
// Distinct bucket of visit v:
template <int D>
__device__ __forceinline__ int visit_bucket(int v) {
  if (D == 0) return 4 * (v >> 3) + (v & 3);                            // rj, rk
  if (D == 1) return 4 * (v >> 3) + 2 * ((v >> 2) & 1) + (v & 1);       // ri, rk
  return 4 * (v >> 3) + ((v >> 1) & 3);                                 // ri, rj
}

constexpr int kGatherThreads = 256;
constexpr int kGatherBatch = 4;

// One lane per listed face, a warp over 32 of them. A lane first loads the
// ranges of its face's 8 distinct buckets (into shared memory, all at once),
// then walks the 16 visits as one flat sequence of particles, so the lanes of
// a warp stay busy until the longest sequence ends.
template <int D, bool POW2>
__global__ void __launch_bounds__(kGatherThreads) k_splat_gather(int nx, int ny, int nz, DxDiv X, SplatBuffers B,
                                                                 SplatGrid G) {
  __shared__ int2 range[8][kGatherThreads];
  if (B.nfaces[3]) return;  // a bucket was over the limit: leave the grids as they are
  const int fw = nx + (D == 0), fh = ny + (D == 1);
  const int E[3] = {nx + (D != 0), ny + (D != 1), nz + (D != 2)};
  const int nact = B.nfaces[D];
  const int *__restrict__ faces = B.sorted + B.face_off[D];
  const float4 *__restrict__ sposm = B.sposm;
  const float4 *__restrict__ svc = B.svc;
  const bool apic = B.apic;
  const double dx = X.dx;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = blockIdx.x * (kGatherThreads >> 5) + (tid >> 5);
  const int warps = gridDim.x * (kGatherThreads >> 5);
  // warp-uniform loop: every lane runs every trip, lanes past the list idle
  for (int t0 = warp * 32; t0 < nact; t0 += warps * 32) {
    const int t = t0 + lane;
    const bool has = t < nact;
    const size_t f = has ? (size_t)__ldg(faces + t) : 0;
    const int fi[3] = {(int)(f % fw), (int)((f / fw) % fh), (int)(f / ((size_t)fw * fh))};
    double pos[3];
    #pragma unroll
    for (int c = 0; c < 3; ++c) pos[c] = ((double)fi[c] + (c != D ? 0.5 : 0.0)) * dx;
    // the 8 distinct buckets (empty where out of the edge grid)
    #pragma unroll
    for (int k = 0; k < 8; ++k) {
      int q[3];
      bucket_coords<D>(k, fi, q);
      const bool out = !has || q[0] < 0 || q[0] >= E[0] || q[1] < 0 || q[1] >= E[1] || q[2] < 0 || q[2] >= E[2];
      const int2 r = out ? make_int2(0, 0) : bucket_range(B, bucket_slot(B, D, E, q));
      range[k][tid] = r;
    }
    float m = 0.0f, mom = 0.0f;
    int v = -1, s = 0, e = 0;
    bool live = has;
    while (true) {
      // the lane's next kGatherBatch particles of its visit sequence: their
      // loads go out together so the L2 latencies overlap, and they are
      // summed in sequence order
      int at[kGatherBatch];
      #pragma unroll
      for (int u = 0; u < kGatherBatch; ++u) {
        while (live && s == e) {
          if (++v == 16) {
            live = false;
            break;
          }
          const int2 r = range[visit_bucket<D>(v)][tid];
          s = r.x;
          e = r.y;
        }
        at[u] = live ? s++ : -1;
      }
      if (!__any_sync(0xffffffffu, at[0] >= 0)) break;
      float4 pmb[kGatherBatch], ub[kGatherBatch];
      #pragma unroll
      for (int u = 0; u < kGatherBatch; ++u) {
        pmb[u] = at[u] >= 0 ? __ldg(sposm + at[u]) : make_float4(0.f, 0.f, 0.f, 0.f);
        ub[u] = at[u] >= 0 ? __ldg(svc + at[u]) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
      #pragma unroll
      for (int u = 0; u < kGatherBatch; ++u) {
        if (at[u] < 0) continue;
        const float4 pm = pmb[u], uv = ub[u];
        const float r0 = __double2float_rn((double)pm.x - pos[0]);
        const float r1 = __double2float_rn((double)pm.y - pos[1]);
        const float r2 = __double2float_rn((double)pm.z - pos[2]);
        const double w = tent<POW2>(r0, X) * tent<POW2>(r1, X) * tent<POW2>(r2, X);
        if (w != 0.0) {
          const double wm = w * (double)pm.w;
          mom = __double2float_rn((double)mom + wm * (double)uv.x);
          m = __double2float_rn((double)m + wm);
          if (apic) {
            double dot = 0.0;
            dot += (double)uv.y * (pos[0] - (double)pm.x);
            dot += (double)uv.z * (pos[1] - (double)pm.y);
            dot += (double)uv.w * (pos[2] - (double)pm.z);
            mom = __double2float_rn((double)mom + wm * dot);
          }
        }
      }
    }
    if (!has) continue;
    const bool on = m != 0.0f;
    if (G.mass[D]) {
      G.mass[D][f] = on ? m : 0.0f;
      G.momentum[D][f] = on ? mom : 0.0f;
      G.splat_active[D][f] = on ? 1 : 0;
    }
    if (on && G.velocity[D]) {
      // combined grid velocity (macflipliquid3.cpp:141-150)
      float *u = G.velocity[D];
      uint8_t *ua = G.velocity_active[D];
      const double g64 = 1.0 - (double)m;
      const float gm = ua[f] ? __double2float_rn(0.0 < g64 ? g64 : 0.0) : 0.0f;
      const float num = __fadd_rn(__fmul_rn(gm, u[f]), mom);
      u[f] = __fdiv_rn(num, __fadd_rn(gm, m));
      ua[f] = 1;
    }
  }
}

// The splat grid of axis D is zero and inactive wherever no particle
// reaches; the gather writes only the faces the particles activate, so the
// rest is cleared first (not after a refused bucket: then the call leaves
// every grid as it was).
template <int D>
__global__ void k_splat_clear_grid(int nx, int ny, int nz, SplatBuffers B, SplatGrid G) {
  if (B.nfaces[3]) return;
  const size_t nf = (size_t)(nx + (D == 0)) * (ny + (D == 1)) * (nz + (D == 2));
  for (size_t f = (size_t)blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += (size_t)gridDim.x * blockDim.x) {
    G.mass[D][f] = 0.0f;
    G.momentum[D][f] = 0.0f;
    G.splat_active[D][f] = 0;
  }
}

}  // namespace

static DxDiv make_dxdiv(double dx) {
  int ex = 0;
  const double mant = std::frexp(dx, &ex);
  const double inv = 1.0 / dx;
  const bool pow2 = mant == 0.5 && std::isnormal(dx) && std::isfinite(inv) && inv * dx == 1.0;
  return DxDiv{dx, inv, pow2 ? 1 : 0};
}

void launch_splat_bin(const SplatRecords &R, int nx, int ny, int nz, double dx, const SplatBuffers &B,
                      cudaStream_t s) {
  if (R.count <= 0) return;
  const unsigned blocks = (unsigned)((R.count + 255) / 256);
  k_splat_bin<<<blocks, 256, 0, s>>>(R, nx, ny, nz, make_dxdiv(dx), B);
}

size_t scan_tile_count(long long n) { return (size_t)((n + kScanTile - 1) / kScanTile); }

void launch_exclusive_scan(int *data, long long n, int *tile_sums, cudaStream_t s) {
  const unsigned tiles = (unsigned)scan_tile_count(n);
  if (!tiles) return;
  k_scan_tiles<<<tiles, kScanThreads, 0, s>>>(data, n, tile_sums);
  k_scan_tile_sums<<<1, kScanThreads, 0, s>>>(tile_sums, (int)tiles);
  k_scan_add<<<tiles, kScanThreads, 0, s>>>(data, n, tile_sums);
}

void launch_splat_bucket_scan(const SplatBuffers &B, int *tile_sums, cudaStream_t s) {
  const unsigned blocks = (unsigned)((B.tiles + 1 + kTileWarps - 1) / kTileWarps);
  k_splat_tile_scan<<<blocks, 32 * kTileWarps, 0, s>>>(B);
  launch_exclusive_scan(B.tile_start, B.tiles + 1, tile_sums, s);
}

void launch_splat_clear(const SplatBuffers &B, cudaStream_t s) {
  const unsigned blocks = (unsigned)((B.tiles + kTileWarps - 1) / kTileWarps);
  if (blocks) k_splat_tile_clear<<<blocks, 32 * kTileWarps, 0, s>>>(B);
}

void launch_splat_scatter(long long count, const SplatBuffers &B, cudaStream_t s) {
  if (count <= 0) return;
  k_splat_scatter<<<(unsigned)((count + 255) / 256), 256, 0, s>>>(count, B);
  k_splat_sort_copy<<<(unsigned)((3 * count + 255) / 256), 256, 0, s>>>(count, B);
}

void launch_splat_gather(int nx, int ny, int nz, double dx, const SplatBuffers &B, const SplatGrid &G,
                         cudaStream_t s) {
  for (int d = 0; d < 3; ++d) {
    const size_t nf = (size_t)(nx + (d == 0)) * (ny + (d == 1)) * (nz + (d == 2));
    const unsigned blocks = (unsigned)((nf + 16 * kCompactThreads - 1) / (16 * kCompactThreads));
    if (d == 0) k_splat_compact<0><<<blocks, kCompactThreads, 0, s>>>(nx, ny, nz, B);
    if (d == 1) k_splat_compact<1><<<blocks, kCompactThreads, 0, s>>>(nx, ny, nz, B);
    if (d == 2) k_splat_compact<2><<<blocks, kCompactThreads, 0, s>>>(nx, ny, nz, B);
  }
  // the face lists' lengths stay on the device: a fixed grid strides over them
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const unsigned blocks = (unsigned)sms * 8;
  k_splat_face_work<0><<<blocks, 256, 0, s>>>(nx, ny, nz, B);
  k_splat_face_work<1><<<blocks, 256, 0, s>>>(nx, ny, nz, B);
  k_splat_face_work<2><<<blocks, 256, 0, s>>>(nx, ny, nz, B);
  k_splat_work_scan<<<1, 96, 0, s>>>(B);
  k_splat_face_sort<0><<<blocks, 256, 0, s>>>(B);
  k_splat_face_sort<1><<<blocks, 256, 0, s>>>(B);
  k_splat_face_sort<2><<<blocks, 256, 0, s>>>(B);
  if (G.mass[0]) {
    k_splat_clear_grid<0><<<blocks, 256, 0, s>>>(nx, ny, nz, B, G);
    k_splat_clear_grid<1><<<blocks, 256, 0, s>>>(nx, ny, nz, B, G);
    k_splat_clear_grid<2><<<blocks, 256, 0, s>>>(nx, ny, nz, B, G);
  }
  const DxDiv X = make_dxdiv(dx);
  if (X.pow2) {
    k_splat_gather<0, true><<<blocks, kGatherThreads, 0, s>>>(nx, ny, nz, X, B, G);
    k_splat_gather<1, true><<<blocks, kGatherThreads, 0, s>>>(nx, ny, nz, X, B, G);
    k_splat_gather<2, true><<<blocks, kGatherThreads, 0, s>>>(nx, ny, nz, X, B, G);
  } else {
    k_splat_gather<0, false><<<blocks, kGatherThreads, 0, s>>>(nx, ny, nz, X, B, G);
    k_splat_gather<1, false><<<blocks, kGatherThreads, 0, s>>>(nx, ny, nz, X, B, G);
    k_splat_gather<2, false><<<blocks, kGatherThreads, 0, s>>>(nx, ny, nz, X, B, G);
  }
}

}  // namespace shkz
