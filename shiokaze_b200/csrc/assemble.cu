// Assembly of the variational pressure system and the velocity update.
//
// This translation unit is compiled with -fmad=false: the face areas, liquid
// fractions, matrix weights and right-hand side are evaluated in FP64 with
// the same operation order as the reference CPU code, so masks are bit-exact
// and the FP64 system equals the reference's RCMatrix values.
//
//   face solid area   macutility3::compute_area_fraction (src/utility/macutility3.cpp:98-171)
//                     + utility::get_area (include/shiokaze/utility/utility.h:191-226)
//   face liquid rho   macutility3::compute_fluid_fraction (macutility3.cpp:172-200)
//                     + utility::fraction (utility.h:174-182)
//   unknowns          mark_body (src/projection/macpressuresolver3.cpp:134-158)
//   weights, rhs      macpressuresolver3.cpp:179-216
//   velocity update   macpressuresolver3.cpp:262-284
//   solid density     macpressuresolver3.cpp:75-80 (areas), 286-293 (velocity scale)
//   surface tension   macpressuresolver3.cpp:98-128
//   volume correction macpressuresolver3.cpp:219-234 (constant added to every rhs row)
#include "common.cuh"
#include "kernels.h"
#include <float.h>

namespace shkz {

struct FaceParams {
  const float *solid;          // nodal effective values, or null (no solid level set)
  const uint8_t *solid_active;
  const float *fluid;          // cell effective values
  int nx, ny, nz;
  int solid_exists, fluid_exists;
  double eps_solid, eps_fluid;
  int second_order_fluid, second_order_solid;
  const float *density[3];     // per-face solid density (set_solid_density), or null
};

// Marching-squares area of the negative region on the unit square, corners
// in (0,0),(1,0),(1,1),(0,1) order, followed by the shoelace sum.
__device__ __forceinline__ double get_area4(const double v[4]) {
  const double qx[4] = {0.0, 1.0, 1.0, 0.0};
  const double qy[4] = {0.0, 0.0, 1.0, 1.0};
  bool all_neg = true, all_nonneg = true;
  #pragma unroll
  for (int n = 0; n < 4; ++n) {
    all_neg &= (v[n] < 0.0);
    all_nonneg &= !(v[n] < 0.0);
  }
  // Uniform corners give no crossing points: an empty list (area 0) or the
  // unit square (shoelace sum 2, area 1), exactly as the general path does.
  if (all_nonneg) return 0.0;
  if (all_neg) return 1.0;
  double px[8], py[8];
  int pnum = 0;
  #pragma unroll
  for (int n = 0; n < 4; ++n) {
    if (v[n] < 0.0) {
      px[pnum] = qx[n];
      py[pnum] = qy[n];
      pnum++;
    }
    const int m = (n + 1) & 3;
    if (v[n] * v[m] < 0) {
      const double y0 = v[n], y1 = v[m];
      if (y0 - y1 != 0.0) {
        const double a = y0 / (y0 - y1);
        px[pnum] = (1.0 - a) * qx[n] + a * qx[m];
        py[pnum] = (1.0 - a) * qy[n] + a * qy[m];
        pnum++;
      }
    }
  }
  double sum = 0.0;
  for (int m = 0; m < pnum; m++) {
    const int m1 = (m + 1 == pnum) ? 0 : m + 1;
    sum += px[m] * py[m1] - py[m] * px[m1];
  }
  return 0.5 * sum;
}

__device__ __forceinline__ size_t nidx(const FaceParams &P, int i, int j, int k) {
  return (size_t)i + (size_t)(P.nx + 1) * ((size_t)j + (size_t)(P.ny + 1) * (size_t)k);
}
__device__ __forceinline__ size_t cidx(const FaceParams &P, int i, int j, int k) {
  return (size_t)i + (size_t)P.nx * ((size_t)j + (size_t)P.ny * (size_t)k);
}

// Solid area of face (d; i,j,k) as the reference stores it (float).
__device__ float face_area(const FaceParams &P, int d, int i, int j, int k) {
  const int pd = d == 0 ? i : (d == 1 ? j : k);
  const int nd = d == 0 ? P.nx : (d == 1 ? P.ny : P.nz);
  double a;
  bool act = false;  // face active in the reference's area grid
  if (!P.solid_exists) {
    // areas.clear(1.0) with the domain walls closed (macutility3.cpp:158-170)
    a = (pd == 0 || pd == nd) ? 0.0 : 1.0;
  } else {
    int n0[3] = {i, j, k}, n1[3], n2[3], n3[3];
    if (d == 0) {
      n1[0] = i; n1[1] = j + 1; n1[2] = k;
      n2[0] = i; n2[1] = j + 1; n2[2] = k + 1;
      n3[0] = i; n3[1] = j;     n3[2] = k + 1;
    } else if (d == 1) {
      n1[0] = i + 1; n1[1] = j; n1[2] = k;
      n2[0] = i + 1; n2[1] = j; n2[2] = k + 1;
      n3[0] = i;     n3[1] = j; n3[2] = k + 1;
    } else {
      n1[0] = i + 1; n1[1] = j;     n1[2] = k;
      n2[0] = i + 1; n2[1] = j + 1; n2[2] = k;
      n3[0] = i;     n3[1] = j + 1; n3[2] = k;
    }
    const size_t s0 = nidx(P, n0[0], n0[1], n0[2]), s1 = nidx(P, n1[0], n1[1], n1[2]);
    const size_t s2 = nidx(P, n2[0], n2[1], n2[2]), s3 = nidx(P, n3[0], n3[1], n3[2]);
    // quadsolid[0][0], [1][0], [1][1], [0][1] -> corners (0,0),(1,0),(1,1),(0,1)
    const double v[4] = {(double)P.solid[s0], (double)P.solid[s1], (double)P.solid[s2], (double)P.solid[s3]};
    act = P.solid_active[s0] | P.solid_active[s1] | P.solid_active[s2] | P.solid_active[s3];
    if (act) {
      if (pd == 0 || pd == nd) a = 0.0;
      else a = 1.0 - get_area4(v);
      if (a != 0.0 && a < P.eps_solid) a = P.eps_solid;
    } else {
      // inactive face: the flood-filled value, 1 outside the solid and the
      // background 0 inside; all four corners lie on one side of the band
      a = 1.0 - get_area4(v);
    }
  }
  float af = (float)a;
  if (act && P.density[d]) {
    // solid density on the active faces of the area grid: density*area + (1 - density)
    const int fw = P.nx + (d == 0), fh = P.ny + (d == 1);
    const float dens = P.density[d][(size_t)i + (size_t)fw * ((size_t)j + (size_t)fh * (size_t)k)];
    const float da = dens * af;
    af = (float)((double)da + (1.0 - (double)dens));
  }
  if (!P.second_order_solid && af != 0.0f) af = 1.0f;
  return af;
}

__device__ __forceinline__ double fraction(double phi0, double phi1) {
  if (phi0 * phi1 >= 0.0) {
    if (phi0 < 0.0 || phi1 < 0.0) return 1.0;
    return 0.0;
  }
  return -fmin(phi0, phi1) / fmax(fabs(phi1 - phi0), DBL_MIN);
}

// Liquid fraction of face (d; i,j,k) as the reference stores it (float).
__device__ float face_rho(const FaceParams &P, int d, int i, int j, int k) {
  double r;
  if (!P.fluid_exists) {
    r = 1.0;
  } else {
    const int ci = min(max(i, 0), P.nx - 1), cj = min(max(j, 0), P.ny - 1), ck = min(max(k, 0), P.nz - 1);
    const int bi = min(max(i - (d == 0), 0), P.nx - 1), bj = min(max(j - (d == 1), 0), P.ny - 1),
              bk = min(max(k - (d == 2), 0), P.nz - 1);
    r = fraction((double)P.fluid[cidx(P, ci, cj, ck)], (double)P.fluid[cidx(P, bi, bj, bk)]);
    if (r != 0.0 && r < P.eps_fluid) r = P.eps_fluid;
  }
  float rf = (float)r;
  if (!P.second_order_fluid && rf != 0.0f) rf = 1.0f;
  return rf;
}

// ---------------------------------------------------------------------------
// levelset_exist (include/shiokaze/array/array_utility3.h:112-122) for the
// liquid (flag bit 0) and solid (bit 1) grids.
__global__ void k_levelset_exist(const float *fluid, const uint8_t *fluid_active, size_t ncell, const float *solid,
                                 const uint8_t *solid_active, size_t nnode, int *flags) {
  int f = 0;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < ncell; c += (size_t)gridDim.x * blockDim.x)
    if (fluid_active[c] && fluid[c] < 0.0f) { f |= 1; break; }
  if (solid) {
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nnode; c += (size_t)gridDim.x * blockDim.x)
      if (solid_active[c] && solid[c] < 0.0f) { f |= 2; break; }
  }
  f = __reduce_or_sync(0xffffffffu, f);
  if ((threadIdx.x & 31) == 0 && f) atomicOr(flags, f);
}

// ---------------------------------------------------------------------------
// Unknown labelling, one CTA per 8^3 tile of the grid. Writes the dense
// unknown mask and the number of unknowns per tile.
__global__ void __launch_bounds__(256) k_label(FaceParams P, Geometry G, const int *flags, uint8_t *unk, int *tile_count) {
  __shared__ double red[8];
  P.fluid_exists = (*flags) & 1;
  P.solid_exists = P.solid ? (((*flags) >> 1) & 1) : 0;
  const long long t = blockIdx.x;
  const int ti = (int)(t % G.bx), tj = (int)((t / G.bx) % G.by), tk = (int)(t / ((long long)G.bx * G.by));
  int count = 0;
  for (int c = threadIdx.x; c < SHKZ_TC; c += blockDim.x) {
    const int i = ti * SHKZ_T + (c & 7), j = tj * SHKZ_T + ((c >> 3) & 7), k = tk * SHKZ_T + (c >> 6);
    if (i >= G.nx || j >= G.ny || k >= G.nz) continue;
    const size_t ci = cidx(P, i, j, k);
    bool inside = false;
    if (P.fluid[ci] < 0.0f) {
      // neighbours in the reference's order: +x, -x, +y, -y, +z, -z
      #pragma unroll 1
      for (int nq = 0; nq < 6 && !inside; ++nq) {
        const int d = nq >> 1, s = (nq & 1) ? -1 : 1;
        const int qi = i + (d == 0) * s, qj = j + (d == 1) * s, qk = k + (d == 2) * s;
        if (qi < 0 || qj < 0 || qk < 0 || qi >= G.nx || qj >= G.ny || qk >= G.nz) continue;
        if (!(P.fluid[cidx(P, qi, qj, qk)] < 0.0f)) continue;
        const int fi = s > 0 ? qi : i, fj = s > 0 ? qj : j, fk = s > 0 ? qk : k;
        if (face_area(P, d, fi, fj, fk) != 0.0f && face_rho(P, d, fi, fj, fk) != 0.0f) inside = true;
      }
    }
    unk[ci] = inside ? 1 : 0;
    count += inside;
  }
  const double total = block_sum<256>((double)count, red);
  if (threadIdx.x == 0) tile_count[t] = (int)total;
}

// ---------------------------------------------------------------------------
// Weights and right-hand side per pool tile. For every unknown cell:
//   w_f   = dt*area/(dx*dx*rho) for in-domain faces with area, rho != 0
//   A_ii  = sum of w_f in the order +x,-x,+y,-y,+z,-z
//   A_i,i-e = -w_f when the neighbour is liquid (it is then an unknown);
//             stored as the positive lower weight off_e
//   b_i   = sum_f -sgn*area*u_f/dx (+ -sgn*(1-area)*u_solid/dx where area<1)
// Non-unknown cells get zeros everywhere, which keeps y = A x zero there.
__global__ void __launch_bounds__(256) k_coeff(FaceParams P, Geometry G, const int *flags, const int *pool_tile,
                                               const uint8_t *unk, const float *vel0, const float *vel1,
                                               const float *vel2, const float *svel0, const float *svel1,
                                               const float *svel2, double dx, double dt, float *diag, float *offx,
                                               float *offy, float *offz, double *diag64, double *offx64,
                                               double *offy64, double *offz64, double *rhs64, double rhs_add) {
  P.fluid_exists = (*flags) & 1;
  P.solid_exists = P.solid ? (((*flags) >> 1) & 1) : 0;
  const int pt = blockIdx.x;
  const long long t = pool_tile[pt];
  const int ti = (int)(t % G.bx), tj = (int)((t / G.bx) % G.by), tk = (int)(t / ((long long)G.bx * G.by));
  const float *vel[3] = {vel0, vel1, vel2};
  const float *svel[3] = {svel0, svel1, svel2};
  for (int c = threadIdx.x; c < SHKZ_TC; c += blockDim.x) {
    const int i = ti * SHKZ_T + (c & 7), j = tj * SHKZ_T + ((c >> 3) & 7), k = tk * SHKZ_T + (c >> 6);
    const size_t o = (size_t)pt * SHKZ_TC + c;
    double dg = 0.0, b = 0.0, lo[3] = {0.0, 0.0, 0.0};
    const bool in_grid = i < G.nx && j < G.ny && k < G.nz;
    if (in_grid && unk[cidx(P, i, j, k)]) {
      #pragma unroll 1
      for (int nq = 0; nq < 6; ++nq) {
        const int d = nq >> 1, s = (nq & 1) ? -1 : 1;
        const int qi = i + (d == 0) * s, qj = j + (d == 1) * s, qk = k + (d == 2) * s;
        const int fi = s > 0 ? qi : i, fj = s > 0 ? qj : j, fk = s > 0 ? qk : k;
        const double area = (double)face_area(P, d, fi, fj, fk);
        const bool oob = qi < 0 || qj < 0 || qk < 0 || qi >= G.nx || qj >= G.ny || qk >= G.nz;
        if (!oob && area != 0.0) {
          const double rho = (double)face_rho(P, d, fi, fj, fk);
          if (rho != 0.0) {
            const double value = dt * area / (dx * dx * rho);
            if (s < 0 && P.fluid[cidx(P, qi, qj, qk)] < 0.0f) lo[d] = value;
            dg += value;
          }
        }
        const int fw = G.nx + (d == 0), fh = G.ny + (d == 1);
        const size_t f = (size_t)fi + (size_t)fw * ((size_t)fj + (size_t)fh * (size_t)fk);
        b += -s * area * (double)vel[d][f] / dx;
        if (area < 1.0) {
          const double us = svel[d] ? (double)svel[d][f] : 0.0;
          b += -s * (1.0 - area) * us / dx;
        }
      }
      b += rhs_add;
    }
    diag[o] = (float)dg;
    offx[o] = (float)lo[0];
    offy[o] = (float)lo[1];
    offz[o] = (float)lo[2];
    if (diag64) {
      diag64[o] = dg;
      offx64[o] = lo[0];
      offy64[o] = lo[1];
      offz64[o] = lo[2];
    }
    rhs64[o] = b;
  }
}

// ---------------------------------------------------------------------------
// Velocity update over every face of dimension d (macpressuresolver3.cpp:269-284):
// active faces with area and rho != 0 get u -= dt*(p_i - p_{i-1})/(rho*dx)
// (u = u_solid on the domain walls); other active faces are switched off.
// The pressure is read as the FP32 grid the reference stores (m_pressure).
__global__ void k_velocity_update(FaceParams P, Geometry G, const int *flags, int d, const int *tile_state,
                                  const float *pressure_pool, const float *svel, double dx, double dt, float *vel,
                                  uint8_t *vact) {
  P.fluid_exists = (*flags) & 1;
  P.solid_exists = P.solid ? (((*flags) >> 1) & 1) : 0;
  const int fw = G.nx + (d == 0), fh = G.ny + (d == 1), fd = G.nz + (d == 2);
  const size_t nf = (size_t)fw * fh * fd;
  const int nd = d == 0 ? G.nx : (d == 1 ? G.ny : G.nz);
  for (size_t f = blockIdx.x * (size_t)blockDim.x + threadIdx.x; f < nf; f += (size_t)gridDim.x * blockDim.x) {
    if (!vact[f]) continue;
    const int i = (int)(f % fw), j = (int)((f / fw) % fh), k = (int)(f / ((size_t)fw * fh));
    const float area = face_area(P, d, i, j, k);
    const float rhof = face_rho(P, d, i, j, k);
    const int pd = d == 0 ? i : (d == 1 ? j : k);
    if (area != 0.0f && rhof != 0.0f) {
      if (pd == 0 || pd == nd) {
        vel[f] = svel ? svel[f] : 0.0f;
      } else {
        auto pread = [&](int ci, int cj, int ck) -> float {
          const long long t = (long long)(ci >> SHKZ_LOG_T) +
                              (long long)G.bx * ((long long)(cj >> SHKZ_LOG_T) + (long long)G.by * (ck >> SHKZ_LOG_T));
          const int pt = tile_state[t];
          if (pt < 0) return 0.0f;
          return pressure_pool[(size_t)pt * SHKZ_TC + (ci & 7) + 8 * (cj & 7) + 64 * (ck & 7)];
        };
        const float p1 = pread(i, j, k);
        const float p0 = pread(i - (d == 0), j - (d == 1), k - (d == 2));
        const float diff = p1 - p0;
        const float value = (float)(dt * (double)diff / ((double)rhof * dx));
        vel[f] = vel[f] - value;
      }
      if (P.density[d]) {
        const float scale = (float)(1.0 - (1.0 - (double)area) * (double)P.density[d][f]);
        vel[f] = scale * vel[f];
      }
    } else {
      vel[f] = 0.0f;
      vact[f] = 0;
    }
  }
}

// ---------------------------------------------------------------------------
// Surface tension (macpressuresolver3.cpp:98-128): curvature as the 7-point
// Laplacian of the liquid level set with clamped neighbours, then every active
// face with 0 < rho < 1 gets u += -sgn*dt/(dx*rho)*kappa*kappa_face, the face
// curvature interpolated by the liquid fraction.
__global__ void k_curvature(FaceParams P, double dx, float *curv) {
  const size_t n = (size_t)P.nx * P.ny * P.nz;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % P.nx), j = (int)((c / P.nx) % P.ny), k = (int)(c / ((size_t)P.nx * P.ny));
    auto f = [&](int a, int b, int e) -> float {
      a = min(max(a, 0), P.nx - 1);
      b = min(max(b, 0), P.ny - 1);
      e = min(max(e, 0), P.nz - 1);
      return P.fluid[cidx(P, a, b, e)];
    };
    // the six neighbours are summed in FP32, as the reference's float operands are
    const float s6 = f(i - 1, j, k) + f(i + 1, j, k) + f(i, j - 1, k) + f(i, j + 1, k) + f(i, j, k - 1) + f(i, j, k + 1);
    const double value = ((double)s6 - 6.0 * (double)P.fluid[c]) / (dx * dx);
    curv[c] = (float)value;
  }
}

__global__ void k_surface_tension(FaceParams P, Geometry G, const int *flags, int d, const float *curv, double kappa,
                                  double dx, double dt, float *vel, const uint8_t *vact) {
  P.fluid_exists = (*flags) & 1;
  P.solid_exists = P.solid ? (((*flags) >> 1) & 1) : 0;
  const int fw = G.nx + (d == 0), fh = G.ny + (d == 1), fd = G.nz + (d == 2);
  const size_t nf = (size_t)fw * fh * fd;
  for (size_t f = blockIdx.x * (size_t)blockDim.x + threadIdx.x; f < nf; f += (size_t)gridDim.x * blockDim.x) {
    if (!vact[f]) continue;
    const int i = (int)(f % fw), j = (int)((f / fw) % fh), k = (int)(f / ((size_t)fw * fh));
    const double rho = (double)face_rho(P, d, i, j, k);
    if (rho != 0.0 && rho < 1.0) {
      const int ci = min(i, G.nx - 1), cj = min(j, G.ny - 1), ck = min(k, G.nz - 1);
      const int bi = max(i - (d == 0), 0), bj = max(j - (d == 1), 0), bk = max(k - (d == 2), 0);
      const size_t c1 = cidx(P, ci, cj, ck), c0 = cidx(P, min(bi, G.nx - 1), min(bj, G.ny - 1), min(bk, G.nz - 1));
      const double sgn = P.fluid[c1] < 0.0f ? -1.0 : 1.0;
      const double theta = sgn < 0 ? 1.0 - rho : rho;
      const double face_c = theta * (double)curv[c1] + (1.0 - theta) * (double)curv[c0];
      const float inc = (float)(-sgn * dt / (dx * rho) * kappa * face_c);
      vel[f] = vel[f] + inc;
    }
  }
}

// Dense pressure grid (FP32, 0 outside unknowns) from the pool.
__global__ void k_scatter_pressure(Geometry G, const int *tile_state, const float *pressure_pool, const uint8_t *unk,
                                   float *pressure, uint8_t *pressure_active) {
  const size_t n = (size_t)G.nx * G.ny * G.nz;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % G.nx), j = (int)((c / G.nx) % G.ny), k = (int)(c / ((size_t)G.nx * G.ny));
    const long long t = (long long)(i >> 3) + (long long)G.bx * ((long long)(j >> 3) + (long long)G.by * (k >> 3));
    const int pt = tile_state[t];
    float v = 0.0f;
    if (pt >= 0 && unk[c]) v = pressure_pool[(size_t)pt * SHKZ_TC + (i & 7) + 8 * (j & 7) + 64 * (k & 7)];
    if (pressure) pressure[c] = v;
    if (pressure_active) pressure_active[c] = unk[c];
  }
}

// ---------------------------------------------------------------------------
// host launchers

static FaceParams make_params(const AssemblyInputs &in) {
  FaceParams P;
  P.solid = in.solid;
  P.solid_active = in.solid_active;
  P.fluid = in.fluid;
  P.nx = in.G.nx;
  P.ny = in.G.ny;
  P.nz = in.G.nz;
  P.solid_exists = 0;
  P.fluid_exists = 0;
  P.eps_solid = in.eps_solid;
  P.eps_fluid = in.eps_fluid;
  P.second_order_fluid = in.second_order_fluid;
  P.second_order_solid = in.second_order_solid;
  for (int d = 0; d < 3; ++d) P.density[d] = in.density[d];
  return P;
}

void launch_label(const AssemblyInputs &in, int *flags, uint8_t *unk, int *tile_count, cudaStream_t s) {
  const size_t ncell = (size_t)in.G.nx * in.G.ny * in.G.nz;
  const size_t nnode = (size_t)(in.G.nx + 1) * (in.G.ny + 1) * (in.G.nz + 1);
  cudaMemsetAsync(flags, 0, sizeof(int), s);
  count_launches(1);
  k_levelset_exist<<<148 * 8, 256, 0, s>>>(in.fluid, in.fluid_active, ncell, in.solid, in.solid_active, nnode, flags);
  count_launches(1);
  k_label<<<(unsigned)in.G.ntiles, 256, 0, s>>>(make_params(in), in.G, flags, unk, tile_count);
}

void launch_coeff(const AssemblyInputs &in, const int *flags, const int *pool_tile, int K, const uint8_t *unk,
                  const CoeffOutputs &out, cudaStream_t s) {
  if (K <= 0) return;
  count_launches(1);
  k_coeff<<<K, 256, 0, s>>>(make_params(in), in.G, flags, pool_tile, unk, in.vel[0], in.vel[1], in.vel[2],
                             in.svel[0], in.svel[1], in.svel[2], in.dx, in.dt, out.diag, out.offx, out.offy, out.offz,
                             out.diag64, out.offx64, out.offy64, out.offz64, out.rhs64, in.rhs_add);
}

void launch_surface_tension(const AssemblyInputs &in, const int *flags, float *curv, double kappa, float *const vel[3],
                            const uint8_t *const vact[3], cudaStream_t s) {
  count_launches(1);
  k_curvature<<<148 * 16, 256, 0, s>>>(make_params(in), in.dx, curv);
  for (int d = 0; d < 3; ++d) {
    count_launches(1);
    k_surface_tension<<<148 * 16, 256, 0, s>>>(make_params(in), in.G, flags, d, curv, kappa, in.dx, in.dt, vel[d],
                                               vact[d]);
  }
}

void launch_velocity_update(const AssemblyInputs &in, const int *flags, const int *tile_state,
                            const float *pressure_pool, float *const vel[3], uint8_t *const vact[3], cudaStream_t s) {
  for (int d = 0; d < 3; ++d) {
    count_launches(1);
    k_velocity_update<<<148 * 16, 256, 0, s>>>(make_params(in), in.G, flags, d, tile_state, pressure_pool, in.svel[d],
                                               in.dx, in.dt, vel[d], vact[d]);
  }
}

void launch_scatter_pressure(const Geometry &G, const int *tile_state, const float *pressure_pool, const uint8_t *unk,
                             float *pressure, uint8_t *pressure_active, cudaStream_t s) {
  count_launches(1);
  k_scatter_pressure<<<148 * 16, 256, 0, s>>>(G, tile_state, pressure_pool, unk, pressure, pressure_active);
}

}  // namespace shkz
