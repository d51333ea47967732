// Velocity extension after a projection, as macliquid3::extend_both runs it
// (src/liquid/macliquid3.cpp:330-340): macarray_extrapolator3::extrapolate
// followed by macutility3::constrain_velocity.
//
// Built with -fmad=false: the reference's double expressions (trilinear
// weights, products added into FP32 sums, the normal projection) round after
// every operation, and so do these, so the results are bit-identical.
//
// Grids are dense, x fastest; a face component d has
// (nx + (d == 0)) x (ny + (d == 1)) x (nz + (d == 2)) entries with a uint8
// active mask; the solid level set is nodal, (nx+1) x (ny+1) x (nz+1), holding
// the values the reference's array3 returns for every node (active value,
// flood-fill value or background), with its active mask.
#include "common.cuh"
#include "kernels.h"

namespace shkz {

// One pass of array_extrapolator3::extrapolate
// (include/shiokaze/array/array_extrapolator3.h) through array3::dilate
// (src/array/dilate3.h): every inactive cell with an active 6-neighbour in the
// state before the pass becomes active with the FP32 mean of its active
// neighbours, summed in the reference's query order (i+1, i-1, j+1, j-1, k-1,
// k+1). The reference defers the writes to the end of the pass; here the find
// kernel writes the frontier's values into a side buffer with a flag, and the
// apply kernel commits them. A pass thus reads the mask (1 B/face) and the
// flags (1 B/face) and touches values only on the frontier, instead of
// copying the whole field between two buffers.
__device__ __forceinline__ void extrapolate_face(size_t o, int W, int H, int D, size_t WH,
                                                 const float *__restrict__ v, const uint8_t *__restrict__ a,
                                                 float *__restrict__ side, uint8_t *__restrict__ flag) {
  const int i = (int)(o % W), j = (int)((o / W) % H), k = (int)(o / WH);
  float s = 0.0f;
  int w = 0;
  if (i + 1 < W && a[o + 1]) { s += v[o + 1]; ++w; }
  if (i > 0 && a[o - 1]) { s += v[o - 1]; ++w; }
  if (j + 1 < H && a[o + W]) { s += v[o + W]; ++w; }
  if (j > 0 && a[o - W]) { s += v[o - W]; ++w; }
  if (k > 0 && a[o - WH]) { s += v[o - WH]; ++w; }
  if (k + 1 < D && a[o + WH]) { s += v[o + WH]; ++w; }
  if (w) {
    side[o] = __fdiv_rn(s, (float)w);
    flag[o] = 1;
  }
}

// The masks are read 16 faces at a time (one 16-byte load per thread, so a
// warp keeps 512 bytes in flight per load); a group of 16 active faces is
// skipped at once. The arrays start 16-byte aligned (cudaMalloc, torch).
__device__ __forceinline__ bool all_set(uint4 m) {
  return m.x == 0x01010101u && m.y == 0x01010101u && m.z == 0x01010101u && m.w == 0x01010101u;
}
__device__ __forceinline__ bool none_set(uint4 m) { return (m.x | m.y | m.z | m.w) == 0u; }
__device__ __forceinline__ unsigned byte_of(uint4 m, int e) {
  const unsigned w = e < 4 ? m.x : (e < 8 ? m.y : (e < 12 ? m.z : m.w));
  return (w >> (8 * (e & 3))) & 0xffu;
}

__global__ void __launch_bounds__(256) k_extrapolate_find(int W, int H, int D, const float *__restrict__ v,
                                                          const uint8_t *__restrict__ a, float *__restrict__ side,
                                                          uint8_t *__restrict__ flag) {
  const size_t n = (size_t)W * H * D, WH = (size_t)W * H, n16 = n / 16;
  const size_t stride = (size_t)gridDim.x * blockDim.x, t0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  for (size_t b = t0; b < n16; b += stride) {
    const uint4 m = reinterpret_cast<const uint4 *>(a)[b];
    if (all_set(m)) continue;
    for (int e = 0; e < 16; ++e)
      if (!byte_of(m, e)) extrapolate_face(16 * b + e, W, H, D, WH, v, a, side, flag);
  }
  for (size_t o = 16 * n16 + t0; o < n; o += stride)
    if (!a[o]) extrapolate_face(o, W, H, D, WH, v, a, side, flag);
}

// Commit flagged values (and activate the faces when act != null), clearing
// the flags for the next use.
__global__ void __launch_bounds__(256) k_apply_side(size_t n, float *__restrict__ v, uint8_t *__restrict__ act,
                                                    const float *__restrict__ side, uint8_t *__restrict__ flag) {
  const size_t n16 = n / 16, stride = (size_t)gridDim.x * blockDim.x;
  const size_t t0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  for (size_t b = t0; b < n16; b += stride) {
    const uint4 f = reinterpret_cast<const uint4 *>(flag)[b];
    if (none_set(f)) continue;
    for (int e = 0; e < 16; ++e) {
      if (!byte_of(f, e)) continue;
      const size_t o = 16 * b + e;
      v[o] = side[o];
      if (act) act[o] = 1;
    }
    reinterpret_cast<uint4 *>(flag)[b] = make_uint4(0u, 0u, 0u, 0u);
  }
  for (size_t o = 16 * n16 + t0; o < n; o += stride) {
    if (!flag[o]) continue;
    v[o] = side[o];
    if (act) act[o] = 1;
    flag[o] = 0;
  }
}

// levelset_exist (include/shiokaze/array/array_utility3.h:112-123): an active
// node with a negative value.
__global__ void k_solid_exists(const float *__restrict__ solid, const uint8_t *__restrict__ act, size_t n,
                               int *flag) {
  int f = 0;
  const size_t n4 = n / 4, stride = (size_t)gridDim.x * blockDim.x;
  const size_t t0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  for (size_t b = t0; b < n4; b += stride) {
    const float4 v = reinterpret_cast<const float4 *>(solid)[b];
    const unsigned m = reinterpret_cast<const unsigned *>(act)[b];
    if (((m & 0xffu) && v.x < 0.0f) || ((m & 0xff00u) && v.y < 0.0f) || ((m & 0xff0000u) && v.z < 0.0f) ||
        ((m & 0xff000000u) && v.w < 0.0f))
      f = 1;
  }
  for (size_t o = 4 * n4 + t0; o < n; o += stride)
    if (act[o] && solid[o] < 0.0f) f = 1;
  if (__any_sync(0xffffffffu, f) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

// array_interpolator3::interpolate_coef's cell and fractions for one point
// (include/shiokaze/array/array_interpolator3.h): clamp into the grid, corner
// (i, j, k), and the weights' factors (i+1-x, x-i, ...).
struct Trilinear {
  int i, j, k;
  double ax, bx, ay, by, az, bz;
};
__device__ __forceinline__ Trilinear trilinear(int W, int H, int D, double px, double py, double pz) {
  Trilinear t;
  const double x = fmax(0.0, fmin(W - 1.0, px));
  const double y = fmax(0.0, fmin(H - 1.0, py));
  const double z = fmax(0.0, fmin(D - 1.0, pz));
  t.i = (int)fmin(x, W - 2.0);
  t.j = (int)fmin(y, H - 2.0);
  t.k = (int)fmin(z, D - 2.0);
  t.ax = (double)(t.i + 1) - x; t.bx = x - (double)t.i;
  t.ay = (double)(t.j + 1) - y; t.by = y - (double)t.j;
  t.az = (double)(t.k + 1) - z; t.bz = z - (double)t.k;
  return t;
}

// The 8 corner values of a grid (0 where the optional mask is off: the
// background of an inactive face is 0).
__device__ __forceinline__ void corners(const float *a, const uint8_t *m, int W, int H, const Trilinear &t,
                                        float v[8]) {
  #pragma unroll
  for (int n = 0; n < 8; ++n) {
    const size_t o = (size_t)(t.i + (n & 1)) + (size_t)W * ((size_t)(t.j + ((n >> 1) & 1)) +
                                                              (size_t)H * (size_t)(t.k + (n >> 2)));
    v[n] = (m && !m[o]) ? 0.0f : a[o];
  }
}

// array_interpolator3::interpolate (only_actives false): FP32 value, each
// corner with a non-zero weight added as value += corner * weight in FP64.
__device__ __forceinline__ float interpolate(const float v[8], const Trilinear &t) {
  const double c[8] = {t.az * t.ax * t.ay, t.az * t.bx * t.ay, t.az * t.ax * t.by, t.az * t.bx * t.by,
                       t.bz * t.ax * t.ay, t.bz * t.bx * t.ay, t.bz * t.ax * t.by, t.bz * t.bx * t.by};
  float r = 0.0f;
  #pragma unroll
  for (int n = 0; n < 8; ++n)
    if (c[n] != 0.0) r = (float)((double)r + (double)v[n] * c[n]);
  return r;
}

// array_derivative3::derivative (include/shiokaze/array/array_derivative3.h):
// FP32 gradient in index space, every term coef * corner in FP64.
__device__ __forceinline__ void derivative(const float v[8], const Trilinear &t, float g[3]) {
  const double cx[8] = {-t.az * t.ay, t.az * t.ay, -t.az * t.by, t.az * t.by,
                        -t.bz * t.ay, t.bz * t.ay, -t.bz * t.by, t.bz * t.by};
  const double cy[8] = {-t.az * t.ax, -t.az * t.bx, t.az * t.ax, t.az * t.bx,
                        -t.bz * t.ax, -t.bz * t.bx, t.bz * t.ax, t.bz * t.bx};
  const double cz[8] = {-t.ax * t.ay, -t.bx * t.ay, -t.ax * t.by, -t.bx * t.by,
                        t.ax * t.ay, t.bx * t.ay, t.ax * t.by, t.bx * t.by};
  float rx = 0.0f, ry = 0.0f, rz = 0.0f;
  #pragma unroll
  for (int n = 0; n < 8; ++n) rx = (float)((double)rx + cx[n] * (double)v[n]);
  #pragma unroll
  for (int n = 0; n < 8; ++n) ry = (float)((double)ry + cy[n] * (double)v[n]);
  #pragma unroll
  for (int n = 0; n < 8; ++n) rz = (float)((double)rz + cz[n] * (double)v[n]);
  g[0] = rx;
  g[1] = ry;
  g[2] = rz;
}

// macutility3::constrain_velocity for the active faces of component d
// (src/utility/macutility3.cpp:61-92): where the solid level set interpolated
// at the face centre is negative, a velocity (interpolated from the field as
// it was before the constraint) that points into the solid loses its normal
// part; then no active y-face lets flow out through the floor or the ceiling.
// The field is not modified here: a changed value goes to side with a flag
// (committed by k_apply_side once all three components are done), so every
// interpolation reads the pre-constraint field, as the reference's
// velocity_save copy provides. Faces whose 8 solid corners are all positive
// are outside the solid without the FP64 interpolation (its weights are
// non-negative and sum to one).
__global__ void __launch_bounds__(128) k_constrain_find(int d, int nx, int ny, int nz, double dx,
                                                        const float *__restrict__ solid, const int *solid_flag,
                                                        ConstrainFields f, float *__restrict__ side,
                                                        uint8_t *__restrict__ flag) {
  const int W = nx + (d == 0), H = ny + (d == 1), D = nz + (d == 2);
  const size_t n = (size_t)W * H * D, WH = (size_t)W * H;
  const bool has_solid = solid && solid_flag && *solid_flag;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    if (!f.act[d][o]) continue;
    const int i = (int)(o % W), j = (int)((o / W) % H), k = (int)(o / WH);
    const float v0 = f.save[d][o];
    float v = v0;
    if (has_solid) {
      const double px = i + 0.5 * (d != 0), py = j + 0.5 * (d != 1), pz = k + 0.5 * (d != 2);
      const Trilinear ts = trilinear(nx + 1, ny + 1, nz + 1, px, py, pz);
      float sv[8];
      corners(solid, nullptr, nx + 1, ny + 1, ts, sv);
      bool near = false;
      #pragma unroll
      for (int c = 0; c < 8; ++c) near = near || !(sv[c] > 0.0f);
      if (near && interpolate(sv, ts) < 0.0f) {
        float g[3];
        derivative(sv, ts, g);
        const double nrm0 = (double)g[0] / dx, nrm1 = (double)g[1] / dx, nrm2 = (double)g[2] / dx;
        const double norm2 = ((0.0 + nrm0 * nrm0) + nrm1 * nrm1) + nrm2 * nrm2;
        if (norm2 != 0.0) {
          double u[3];
          #pragma unroll
          for (int c = 0; c < 3; ++c) {
            const int Wc = nx + (c == 0), Hc = ny + (c == 1), Dc = nz + (c == 2);
            const Trilinear tc = trilinear(Wc, Hc, Dc, px - 0.5 * (c != 0), py - 0.5 * (c != 1), pz - 0.5 * (c != 2));
            float cv[8];
            corners(f.save[c], f.act[c], Wc, Hc, tc, cv);
            u[c] = (double)interpolate(cv, tc);
          }
          const double un = ((0.0 + u[0] * nrm0) + u[1] * nrm1) + u[2] * nrm2;
          if (un < 0.0) {
            const double ud = d == 0 ? u[0] : (d == 1 ? u[1] : u[2]);
            const double nd = d == 0 ? nrm0 : (d == 1 ? nrm1 : nrm2);
            v = (float)(ud - nd * un);
          }
        }
      }
    }
    if (d == 1) {
      if (j == 0 && v < 0.0f) v = 0.0f;
      if (j == ny && v > 0.0f) v = 0.0f;
    }
    if (__float_as_uint(v) != __float_as_uint(v0)) {
      side[o] = v;
      flag[o] = 1;
    }
  }
}

static int ext_grid(size_t n, int threads) {
  const size_t b = (n + threads - 1) / threads;
  return (int)(b < (size_t)148 * 16 ? (b ? b : 1) : (size_t)148 * 16);
}

void launch_extrapolate(int W, int H, int D, float *v, uint8_t *a, float *side, uint8_t *flag, cudaStream_t s) {
  const size_t n = (size_t)W * H * D;
  if (!n) return;
  count_launches(2);
  k_extrapolate_find<<<ext_grid(n, 256), 256, 0, s>>>(W, H, D, v, a, side, flag);
  k_apply_side<<<ext_grid(n, 256), 256, 0, s>>>(n, v, a, side, flag);
}

void launch_solid_exists(const float *solid, const uint8_t *act, size_t n, int *flag, cudaStream_t s) {
  if (!n) return;
  count_launches(1);
  k_solid_exists<<<ext_grid(n, 256), 256, 0, s>>>(solid, act, n, flag);
}

void launch_constrain_find(int d, int nx, int ny, int nz, double dx, const float *solid, const int *solid_flag,
                           const ConstrainFields &f, float *side, uint8_t *flag, cudaStream_t s) {
  const size_t n = (size_t)(nx + (d == 0)) * (ny + (d == 1)) * (nz + (d == 2));
  count_launches(1);
  k_constrain_find<<<ext_grid(n, 128), 128, 0, s>>>(d, nx, ny, nz, dx, solid, solid_flag, f, side, flag);
}

void launch_apply_side(size_t n, float *v, const float *side, uint8_t *flag, cudaStream_t s) {
  if (!n) return;
  count_launches(1);
  k_apply_side<<<ext_grid(n, 256), 256, 0, s>>>(n, v, nullptr, side, flag);
}

}  // namespace shkz
