// Learned preconditioner: a 3-level 3D conv encoder-decoder (16/32/64
// channels, 3^3 kernels, BF16 weights and activations, FP32 accumulation)
// that maps (residual, liquid level set, solid fraction) to a correction z,
// used as the preconditioner of a flexible PCG (Polak-Ribiere beta) with the
// reference's MIC(0) as the fallback when the residual stalls.
//
// Layers (level 0 = grid resolution, 1 = half, 2 = quarter):
//   e1a X0(16)->16, e1b 16->16 = S1          level 0
//   e2a avgpool(S1)(16)->32, e2b 32->32 = S2  level 1
//   e3a avgpool(S2)(32)->64, e3b 64->64 = B3  level 2
//   d2a [S2, up(B3)](96)->32, d2b 32->32 = D2 level 1
//   d1a [S1, up(D2)](48)->16, d1b 16->16 = D1 level 0
//   out 16->1 (linear, FP32)                  level 0
// Activations are dense channels-last BF16 tensors per level, zero outside
// the active 8x16x8 blocks (blocks that touch a tile of the solver's pool).
// Every 3^3 convolution (forward, and the input gradient with flipped and
// transposed weights) runs on the tcgen05 implicit-GEMM kernel of tc_conv.cuh;
// weight gradients run on tcgen05 too (k_wgrad_tc, voxels as the reduction
// dimension). Adam keeps FP32 master weights and moments.
#include "common.cuh"
#include "kernels.h"
#include "learned.h"
#include "solver.h"
#include "tc_conv.cuh"

#include <cudaTypedefs.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

namespace shkz {

// ---------------------------------------------------------------------------
// tcgen05 convolution kernel

__global__ void __launch_bounds__(128, 1) k_conv_tc(ConvArgs a, const __grid_constant__ ConvMaps maps) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const int P = a.planes;
  const uint32_t LBO_A = (uint32_t)(P + 2) * 18 * 10 * 16;
  const uint32_t wbytes = 27u * a.cout * 32u;
  uint8_t *halo = smem;
  uint8_t *wsm = smem + 2 * LBO_A;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(wsm + wbytes);
  uint64_t *mbar_tma = mbar + 1;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mbar + 2);

  const int zsplit = 8 / P;
  int bid = blockIdx.x;
  const int zpart = bid % zsplit;
  bid /= zsplit;
  const int bxi = bid % a.gbx;
  bid /= a.gbx;
  const int byi = bid % a.gby;
  const int bzi = bid / a.gby;
  if (!a.block_act[((size_t)bzi * a.gby + byi) * a.gbx + bxi]) return;  // whole CTA
  const int X0 = bxi * 8, Y0 = byi * 16, Z0 = bzi * 8 + zpart * P;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // each plane's accumulator starts on a 32-column boundary of TMEM
  const int pstride = (a.cout + 31) & ~31;
  uint32_t ncols = 32;
  while (ncols < (uint32_t)(P * pstride)) ncols <<= 1;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar_tma)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  const int nchunk = (a.c0 + a.c1) / 16;
  const uint32_t idesc = umma_idesc_bf16(a.cout);
  const uint32_t halo_s = smem_u32(halo), w_s = smem_u32(wsm), bar_s = smem_u32(mbar);
  bool ok = true;
  const uint32_t tma_s = smem_u32(mbar_tma);
  int tma_uses = 0;
  for (int ch = 0; ch < nchunk; ++ch) {
    const bool first = ch * 16 < a.c0;  // chunk from in0 (else the upsampled in1)
    const bool by_tma = a.tma && first;
    if (by_tma) {
      // both 8-channel halves of the halo by two 4D TMA loads; the tensor maps
      // cover the grid exactly, so halo voxels outside it arrive as zeros
      if (tid == 0) {
        const uint32_t bytes = 2 * LBO_A;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tma_s), "r"(bytes) : "memory");
        #pragma unroll
        for (int h = 0; h < 2; ++h) {
          const CUtensorMap *map = &maps.m[2 * ch + h];
          asm volatile(
              "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::
                  "r"(halo_s + (uint32_t)h * LBO_A), "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(X0 - 1),
                  "r"(Y0 - 1), "r"(Z0 - 1), "r"(tma_s)
              : "memory");
        }
      }
    }
    // halo of the chunk (unless by TMA): each thread owns one or two of the
    // 18 x 10 (y, x) columns and walks its P + 2 planes and both 8-channel
    // halves, so the index arithmetic is done once per column
    for (int pp = by_tma ? 180 : tid; pp < 180; pp += 128) {
      const int yy = pp / 10, xx = pp - yy * 10;
      const int X = X0 + xx - 1, Y = Y0 + yy - 1;
      const bool inxy = X >= 0 && Y >= 0 && X < a.nx && Y < a.ny;
      const int hX = X >> 1, hY = Y >> 1;
      const bool inxy1 = inxy && hX < a.hx && hY < a.hy;
      const uint32_t dcol = halo_s + (uint32_t)(yy * 10 + xx) * 16;
      for (int zz = 0; zz < P + 2; ++zz) {
        const int Z = Z0 + zz - 1;
        const void *src0 = a.in0, *src1 = a.in0;
        int bytes = 0;
        if (first) {
          if (inxy && Z >= 0 && Z < a.nz) {
            src0 = a.in0 + ((size_t)((size_t)Z * a.ny + Y) * a.nx + X) * a.c0 + ch * 16;
            src1 = static_cast<const __nv_bfloat16 *>(src0) + 8;
            bytes = 16;
          }
        } else {
          const int hZ = Z >> 1;
          if (inxy1 && Z >= 0 && Z < a.nz && hZ < a.hz) {
            src0 = a.in1 + ((size_t)((size_t)hZ * a.hy + hY) * a.hx + hX) * a.c1 + (ch * 16 - a.c0);
            src1 = static_cast<const __nv_bfloat16 *>(src0) + 8;
            bytes = 16;
          }
        }
        const uint32_t d = dcol + (uint32_t)zz * 180 * 16;
        cp_async16(d, src0, bytes);
        cp_async16(d + LBO_A, src1, bytes);
      }
    }
    const __nv_bfloat16 *wsrc = a.wpk + (size_t)ch * 27 * a.cout * 16;
    for (int e = tid; e < 27 * a.cout * 2; e += 128) cp_async16(w_s + e * 16, wsrc + (size_t)e * 8, 16);
    cp_async_wait_all();
    if (by_tma) {
      if (mbar_wait(tma_s, (uint32_t)(tma_uses & 1))) ++tma_uses;
      else ok = false;  // tma_uses keeps the parity still in flight for the error path
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (!ok) break;
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      // The descriptors' start-address field holds (address >> 4) in its low
      // 14 bits and shared addresses stay below 2^18, so a tap's descriptor is
      // the base descriptor plus the tap's offset in 16-byte units.
      const uint64_t da0 = umma_desc(halo_s, LBO_A, 160);
      const uint64_t db0 = umma_desc(w_s, (uint32_t)a.cout * 16, 128);
      for (int zo = 0; zo < P; ++zo) {
        const uint32_t d_tmem = tmem + (uint32_t)(zo * pstride);
        int t = 0;
        for (int dz = 0; dz < 3; ++dz)
          for (int dy = 0; dy < 3; ++dy)
            for (int dx = 0; dx < 3; ++dx, ++t) {
              const uint64_t da = da0 + (uint64_t)(((zo + dz) * 18 + dy) * 10 + dx);
              const uint64_t db = db0 + (uint64_t)(t * a.cout * 2);
              const uint32_t acc = (ch > 0 || t > 0) ? 1u : 0u;
              asm volatile(
                  "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                  "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d_tmem),
                  "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0)
                  : "memory");
            }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_s)
                   : "memory");
    }
    __syncwarp();
    if (!mbar_wait(bar_s, (uint32_t)(ch & 1))) {
      ok = false;
      break;
    }
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    const int m = warp * 32 + lane;
    const int x = m & 7, y = m >> 3;
    for (int zo = 0; zo < P; ++zo) {
      const int X = X0 + x, Y = Y0 + y, Z = Z0 + zo;
      const bool inside = X < a.nx && Y < a.ny && Z < a.nz;
      for (int cb = 0; cb < a.cout; cb += 16) {
        uint32_t r[16];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(zo * pstride + cb);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr)
            : "memory");
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (!inside) continue;
        const size_t vox = ((size_t)Z * a.ny + Y) * a.nx + X;
        float v[16];
        #pragma unroll
        for (int i = 0; i < 16; ++i) {
          v[i] = __uint_as_float(r[i]) + ((a.bias && cb + i < a.bias_n) ? a.bias[cb + i] : 0.0f);
          if (a.relu) v[i] = fmaxf(v[i], 0.0f);
        }
        if (a.out32 && cb == 0) a.out32[vox] = v[0];
        if (a.out) {
          __align__(16) __nv_bfloat16 h[16];
          #pragma unroll
          for (int i = 0; i < 16; ++i) h[i] = __float2bfloat16_rn(v[i]);
          uint4 *dst = reinterpret_cast<uint4 *>(a.out + vox * a.cout + cb);
          dst[0] = reinterpret_cast<const uint4 *>(h)[0];
          dst[1] = reinterpret_cast<const uint4 *>(h)[1];
        }
      }
    }
  } else {
    if (tid == 0) atomicExch(a.err, 1);
    // give the outstanding MMAs and halo copies a bounded chance to finish
    // before TMEM and shared memory are released
    mbar_wait(bar_s, 0);
    mbar_wait(bar_s, 1);
    if (a.tma) mbar_wait(tma_s, (uint32_t)(tma_uses & 1));
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

static size_t conv_smem_bytes(int planes, int cout) {
  return (size_t)2 * (planes + 2) * 18 * 10 * 16 + (size_t)27 * cout * 32 + 32;
}

// cuTensorMapEncodeTiled from the driver, looked up once.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// Tensor maps for the in0 chunks of a convolution; false (a.tma stays 0, all
// halos by cp.async) when the driver entry point is missing, the channel
// count exceeds the maps' capacity or the driver rejects a map.
static bool make_conv_maps(ConvArgs &a, ConvMaps &M) {
  a.tma = 0;
  auto enc = tensor_map_encoder();
  const int nch0 = a.c0 / 16;
  if (!enc || nch0 > CONV_MAX_TMA_CHUNKS || a.c0 % 16) return false;
  for (int ch = 0; ch < nch0; ++ch)
    for (int h = 0; h < 2; ++h) {
      const __nv_bfloat16 *base = a.in0 + ch * 16 + h * 8;  // 16-byte aligned: 32 ch + 16 h bytes past the tensor
      const cuuint64_t dims[4] = {8, (cuuint64_t)a.nx, (cuuint64_t)a.ny, (cuuint64_t)a.nz};
      const cuuint64_t strides[3] = {(cuuint64_t)a.c0 * 2, (cuuint64_t)a.nx * a.c0 * 2,
                                     (cuuint64_t)a.ny * a.nx * a.c0 * 2};
      const cuuint32_t box[4] = {8, 10, 18, (cuuint32_t)(a.planes + 2)};
      const cuuint32_t es[4] = {1, 1, 1, 1};
      if (enc(&M.m[2 * ch + h], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16 *>(base), dims, strides,
              box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    }
  a.tma = 1;
  return true;
}

static void launch_conv_tc(ConvArgs a, int nblocks, size_t smem, cudaStream_t s) {
  ConvMaps maps;  // the launch copies it into the kernel's parameter buffer
  std::memset(&maps, 0, sizeof(maps));
  make_conv_maps(a, maps);
  count_launches(1);
  k_conv_tc<<<nblocks, 128, smem, s>>>(a, maps);
}

// ---------------------------------------------------------------------------
// elementwise kernels

// Packs FP32 weights w[27][cout][cin] into the per-chunk canonical layout;
// transposed = 1 packs the input-gradient weights W'[t][ci][co] = W[26-t][co][ci]
// (padded so that both channel counts are multiples of 16).
__global__ void k_pack_weights(const float *w, int cout_real, int cin_real, int n_pad, int k_pad, int transposed,
                               __nv_bfloat16 *out) {
  // out element (chunk, t, kh, n/8, n%8, k8) for n < n_pad, k = chunk*16 + kh*8 + k8 < k_pad
  const int total = 27 * n_pad * k_pad;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    int r = e;
    const int k8 = r & 7; r >>= 3;
    const int n8 = r & 7; r >>= 3;
    const int ng = r % (n_pad / 8); r /= (n_pad / 8);
    const int kh = r & 1; r >>= 1;
    const int t = r % 27;
    const int chunk = r / 27;
    const int n = ng * 8 + n8, k = chunk * 16 + kh * 8 + k8;
    float v = 0.0f;
    if (!transposed) {
      if (n < cout_real && k < cin_real) v = w[((size_t)t * cout_real + n) * cin_real + k];
    } else {
      // n = input channel of the forward layer, k = its output channel
      if (n < cin_real && k < cout_real) v = w[((size_t)(26 - t) * cout_real + k) * cin_real + n];
    }
    out[e] = __float2bfloat16_rn(v);
  }
}

// Block activity for the three levels from the pool tiles of the solver.
__global__ void k_block_activity(Geometry G, const int *tile_state, int level, int gbx, int gby, int gbz,
                                 uint8_t *act) {
  const int nb = gbx * gby * gbz;
  const int f = 1 << level;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    const int bx = b % gbx, by = (b / gbx) % gby, bz = b / (gbx * gby);
    // level-0 cell range of the block, in 8^3 solver tiles
    const int x0 = bx * 8 * f, y0 = by * 16 * f, z0 = bz * 8 * f;
    const int tx0 = x0 >> 3, ty0 = y0 >> 3, tz0 = z0 >> 3;
    const int tx1 = min((x0 + 8 * f - 1) >> 3, G.bx - 1), ty1 = min((y0 + 16 * f - 1) >> 3, G.by - 1),
              tz1 = min((z0 + 8 * f - 1) >> 3, G.bz - 1);
    uint8_t a = 0;
    for (int tz = tz0; tz <= tz1 && !a; ++tz)
      for (int ty = ty0; ty <= ty1 && !a; ++ty)
        for (int tx = tx0; tx <= tx1 && !a; ++tx)
          if (tile_state[(long long)tx + (long long)G.bx * ((long long)ty + (long long)G.by * tz)] >= 0) a = 1;
    act[b] = a;
  }
}

// Blocks that are active or touch an active block (26-neighbourhood): the
// input gradient of a convolution reaches one voxel beyond the active blocks.
__global__ void k_block_dilate(const uint8_t *act, int gbx, int gby, int gbz, uint8_t *out) {
  const int nb = gbx * gby * gbz;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    const int bx = b % gbx, by = (b / gbx) % gby, bz = b / (gbx * gby);
    uint8_t a = 0;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int x = bx + dx, y = by + dy, z = bz + dz;
          if (x >= 0 && y >= 0 && z >= 0 && x < gbx && y < gby && z < gbz && act[((size_t)z * gby + y) * gbx + x])
            a = 1;
        }
    out[b] = a;
  }
}

__device__ __forceinline__ bool vox_active(const uint8_t *act, int gbx, int gby, int x, int y, int z) {
  return act[((size_t)(z >> 3) * gby + (y >> 4)) * gbx + (x >> 3)] != 0;
}

// X0 channels: r/s at unknowns, phi/dx, solid node fraction; zero outside active blocks.
__global__ void k_make_input(Geometry G, int NX, int NY, int NZ, const int *tile_state, const float *r_pool,
                             const uint8_t *unk, const float *fluid, const float *solid, double inv_scale,
                             double inv_dx, const uint8_t *act, int gbx, int gby, __nv_bfloat16 *X0) {
  const size_t n = (size_t)NX * NY * NZ;
  for (size_t v = blockIdx.x * (size_t)blockDim.x + threadIdx.x; v < n; v += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(v % NX), y = (int)((v / NX) % NY), z = (int)(v / ((size_t)NX * NY));
    float c0 = 0.f, c1 = 0.f, c2 = 0.f;
    if (vox_active(act, gbx, gby, x, y, z) && x < G.nx && y < G.ny && z < G.nz) {
      const size_t c = (size_t)x + (size_t)G.nx * ((size_t)y + (size_t)G.ny * z);
      const long long t = (long long)(x >> 3) + (long long)G.bx * ((long long)(y >> 3) + (long long)G.by * (z >> 3));
      const int pt = tile_state[t];
      if (pt >= 0 && unk[c]) c0 = (float)(r_pool[(size_t)pt * SHKZ_TC + (x & 7) + 8 * (y & 7) + 64 * (z & 7)] * inv_scale);
      c1 = fminf(fmaxf((float)(fluid[c] * inv_dx), -4.f), 4.f);
      if (solid) {
        int in = 0;
        for (int dz = 0; dz < 2; ++dz)
          for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx)
              in += solid[(size_t)(x + dx) + (size_t)(G.nx + 1) * ((size_t)(y + dy) + (size_t)(G.ny + 1) * (z + dz))] < 0.f;
        c2 = in * 0.125f;
      }
    }
    __align__(16) __nv_bfloat16 h[16];
    h[0] = __float2bfloat16_rn(c0);
    h[1] = __float2bfloat16_rn(c1);
    h[2] = __float2bfloat16_rn(c2);
    #pragma unroll
    for (int i = 3; i < 16; ++i) h[i] = __float2bfloat16_rn(0.f);
    uint4 *dst = reinterpret_cast<uint4 *>(X0 + v * 16);
    dst[0] = reinterpret_cast<const uint4 *>(h)[0];
    dst[1] = reinterpret_cast<const uint4 *>(h)[1];
  }
}

// z_pool = scale * Z at unknown cells, 0 elsewhere.
__global__ void k_gather_output(Geometry G, int NX, int NY, const int *pool_tile, int K, const uint8_t *unk,
                                const float *Z, double scale, float *z_pool) {
  const size_t n = (size_t)K * SHKZ_TC;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    const int pt = (int)(o >> 9), c = (int)(o & 511);
    const long long t = pool_tile[pt];
    const int x = (int)(t % G.bx) * 8 + (c & 7), y = (int)((t / G.bx) % G.by) * 8 + ((c >> 3) & 7),
              z = (int)(t / ((long long)G.bx * G.by)) * 8 + (c >> 6);
    float v = 0.f;
    if (x < G.nx && y < G.ny && z < G.nz && unk[(size_t)x + (size_t)G.nx * ((size_t)y + (size_t)G.ny * z)])
      v = (float)(scale * Z[((size_t)z * NY + y) * NX + x]);
    z_pool[o] = v;
  }
}

// 2x2x2 average pooling, channels-last; zero outside active blocks of the output level.
__global__ void k_avgpool(const __nv_bfloat16 *in, int NX, int NY, int C, __nv_bfloat16 *out, int hx, int hy, int hz,
                          const uint8_t *act, int gbx, int gby) {
  const size_t n = (size_t)hx * hy * hz * C;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(e % C);
    const size_t v = e / C;
    const int x = (int)(v % hx), y = (int)((v / hx) % hy), z = (int)(v / ((size_t)hx * hy));
    float s = 0.f;
    if (vox_active(act, gbx, gby, x, y, z)) {
      for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
          for (int dx = 0; dx < 2; ++dx)
            s += __bfloat162float(in[(((size_t)(2 * z + dz) * NY + (2 * y + dy)) * NX + (2 * x + dx)) * C + c]);
      s *= 0.125f;
    }
    out[e] = __float2bfloat16_rn(s);
  }
}

// ---------------------------------------------------------------------------
// backward helpers

// gpre (BF16, cpad channels) = G (FP32, C channels) * relu'(act) * mask
__global__ void k_grad_pre(const float *G, const __nv_bfloat16 *act, int C, int cpad, int relu, size_t nvox, int NX,
                           int NY, const uint8_t *blk, int gbx, int gby, __nv_bfloat16 *gpre) {
  const size_t n = nvox * cpad;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(e % cpad);
    const size_t v = e / cpad;
    const int x = (int)(v % NX), y = (int)((v / NX) % NY), z = (int)(v / ((size_t)NX * NY));
    float g = 0.f;
    if (c < C && vox_active(blk, gbx, gby, x, y, z)) {
      g = G[v * C + c];
      if (relu && !(__bfloat162float(act[v * C + c]) > 0.f)) g = 0.f;
    }
    gpre[e] = __float2bfloat16_rn(g);
  }
}

// G0 += gx[..., :c0] (level res); G1 += sum over 2^3 children of gx[..., c0:] (half res)
__global__ void k_split_grad(const __nv_bfloat16 *gx, int cin, int c0, size_t nvox, float *G0, const uint8_t *blk,
                             int NX, int NY, int gbx, int gby) {
  const size_t n = nvox * c0;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(e % c0);
    const size_t v = e / c0;
    const int x = (int)(v % NX), y = (int)((v / NX) % NY), z = (int)(v / ((size_t)NX * NY));
    if (vox_active(blk, gbx, gby, x, y, z)) G0[e] += __bfloat162float(gx[v * cin + c]);
  }
}
__global__ void k_up_grad(const __nv_bfloat16 *gx, int cin, int c0, int NX, int NY, int NZ, float *G1, int c1, int hx,
                          int hy, int hz, const uint8_t *blk1, int gbx1, int gby1) {
  const size_t n = (size_t)hx * hy * hz * c1;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(e % c1);
    const size_t v = e / c1;
    const int x = (int)(v % hx), y = (int)((v / hx) % hy), z = (int)(v / ((size_t)hx * hy));
    if (!vox_active(blk1, gbx1, gby1, x, y, z)) continue;
    float s = 0.f;
    for (int dz = 0; dz < 2; ++dz)
      for (int dy = 0; dy < 2; ++dy)
        for (int dx = 0; dx < 2; ++dx) {
          const int X = 2 * x + dx, Y = 2 * y + dy, Z = 2 * z + dz;
          if (X < NX && Y < NY && Z < NZ) s += __bfloat162float(gx[(((size_t)Z * NY + Y) * NX + X) * cin + c0 + c]);
        }
    G1[e] += s;
  }
}
// avgpool backward: G_fine += G_coarse / 8 (coarse masked)
__global__ void k_pool_grad(const float *Gc, int C, int hx, int hy, int hz, const uint8_t *blkc, int gbxc, int gbyc,
                            float *Gf, int NX, int NY) {
  const size_t n = (size_t)hx * hy * hz * C;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(e % C);
    const size_t v = e / C;
    const int x = (int)(v % hx), y = (int)((v / hx) % hy), z = (int)(v / ((size_t)hx * hy));
    if (!vox_active(blkc, gbxc, gbyc, x, y, z)) continue;
    const float g = Gc[e] * 0.125f;
    for (int dz = 0; dz < 2; ++dz)
      for (int dy = 0; dy < 2; ++dy)
        for (int dx = 0; dx < 2; ++dx)
          Gf[(((size_t)(2 * z + dz) * NY + (2 * y + dy)) * NX + (2 * x + dx)) * C + c] += g;
  }
}

// Weight gradient on the tensor cores (tcgen05, kind::f16, M = 64, N = 16,
// K = voxels): for one active block (8 x 16 x 8 voxels) and one 16-channel
// input chunk,
//   D_t[co][ci] = sum_v gpre[v][co] * X(v + off_t)[ci]      for the 27 taps t,
// accumulated in TMEM (tap t in columns 16 t .. 16 t + 15) over four
// sub-blocks of two z planes (256 voxels). Both operands are MN-major, so the
// staged data keep their channels-last order:
//   A = gpre: 8-channel groups g of 256 voxels x 16 B, byte g * 4096 + k * 16
//       (k = x + 8 y + 128 z); SBO = 4096 B between channel groups, LBO = 128 B
//       between the 8-voxel groups of a K step;
//   B = the input halo of the sub-block, (4 z) x 18 x 10 voxels x 16 B per
//       8-channel half, the canonical layout of the forward kernel; a tap is
//       the same layout shifted, so only the start address changes; SBO = the
//       half's size between the channel halves, LBO = 160 B (one y row)
//       between the 8-voxel groups of a K step.
// The next sub-block is staged (cp.async) while the tensor cores work on the
// current one. Row co of D sits in TMEM lane (co % 16) + 32 (co / 16), so warp
// w reads output channels 16 w .. 16 w + 15 in its first 16 lanes, adds them
// to dW with atomics, and the bias gradient is summed from the staged gpre.
__global__ void __launch_bounds__(128, 1) k_wgrad_tc(const __nv_bfloat16 *gpre, int cout_pad, int cout_real,
                                                     const __nv_bfloat16 *in0, int c0, const __nv_bfloat16 *in1,
                                                     int c1, int nx, int ny, int nz, int hx, int hy, int hz,
                                                     const uint8_t *blk, int gbx, int gby, int gbz, float *dW,
                                                     float *db, int *err) {
  constexpr uint32_t kG = 8 * 256 * 16;        // staged gpre of a sub-block
  constexpr uint32_t kHH = 4 * 18 * 10 * 16;   // one 8-channel half of the halo
  constexpr uint32_t kBuf = kG + 2 * kHH;      // one stage (55,808 bytes)
  extern __shared__ __align__(1024) uint8_t smem[];
  uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + 2 * kBuf);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mbar + 1);
  const int cin = c0 + c1;
  const int nchunk = cin / 16;
  int bid = blockIdx.x;
  const int chunk = bid % nchunk;
  bid /= nchunk;
  const int bxi = bid % gbx, byi = (bid / gbx) % gby, bzi = bid / (gbx * gby);
  if (!blk[((size_t)bzi * gby + byi) * gbx + bxi]) return;  // whole CTA
  const int X0 = bxi * 8, Y0 = byi * 16, Z0 = bzi * 8;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t s0 = smem_u32(smem), bar_s = smem_u32(mbar);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_s) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  // D FP32, A/B BF16, both MN-major, N = 16, M = 64
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((uint32_t)(16 >> 3) << 17) |
                         ((uint32_t)(64 >> 4) << 24);
  auto stage = [&](int sb, uint32_t buf) {
    for (int e = tid; e < 2048; e += 128) {
      const int g = e >> 8, k = e & 255;
      const int X = X0 + (k & 7), Y = Y0 + ((k >> 3) & 15), Z = Z0 + 2 * sb + (k >> 7);
      const bool in = 8 * g < cout_pad && X < nx && Y < ny && Z < nz;
      const __nv_bfloat16 *src = in ? gpre + (((size_t)Z * ny + Y) * nx + X) * cout_pad + 8 * g : gpre;
      cp_async16(buf + (uint32_t)(g * 4096 + k * 16), src, in ? 16 : 0);
    }
    for (int e = tid; e < 1440; e += 128) {
      const int kh = e / 720, r = e % 720, zz = r / 180, yy = (r % 180) / 10, xx = r % 10;
      const int X = X0 + xx - 1, Y = Y0 + yy - 1, Z = Z0 + 2 * sb + zz - 1;
      const int c = chunk * 16 + kh * 8;
      const __nv_bfloat16 *src = in0;
      int bytes = 0;
      if (X >= 0 && Y >= 0 && Z >= 0 && X < nx && Y < ny && Z < nz) {
        if (c < c0) {
          src = in0 + (((size_t)Z * ny + Y) * nx + X) * c0 + c;
          bytes = 16;
        } else {
          const int hX = X >> 1, hY = Y >> 1, hZ = Z >> 1;
          if (hX < hx && hY < hy && hZ < hz) {
            src = in1 + (((size_t)hZ * hy + hY) * hx + hX) * c1 + (c - c0);
            bytes = 16;
          }
        }
      }
      cp_async16(buf + kG + (uint32_t)kh * kHH + (uint32_t)((zz * 18 + yy) * 10 + xx) * 16, src, bytes);
    }
  };
  bool ok = true;
  float bsum = 0.0f;
  const bool bias = chunk == 0 && db != nullptr;
  stage(0, s0);
  cp_async_wait_all();
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  for (int sb = 0; sb < 4; ++sb) {
    const uint32_t buf = s0 + (uint32_t)(sb & 1) * kBuf;
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int t = 0; t < 27; ++t) {
        const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
        #pragma unroll 4
        for (int j = 0; j < 16; ++j) {
          const int y0 = (2 * j) & 15, zl = j >> 3;
          const uint64_t da = umma_desc(buf + 256u * (uint32_t)j, 128, 4096);
          const uint64_t dbd =
              umma_desc(buf + kG + (uint32_t)(((zl + dz) * 18 + (y0 + dy)) * 10 + dx) * 16, 160, kHH);
          const uint32_t acc = (sb > 0 || j > 0) ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem + (uint32_t)(t * 16)),
              "l"(da), "l"(dbd), "r"(idesc), "r"(acc)
              : "memory");
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_s)
                   : "memory");
    }
    __syncwarp();
    // the next sub-block into the other stage while the tensor cores read this one
    if (sb + 1 < 4) stage(sb + 1, s0 + (uint32_t)((sb + 1) & 1) * kBuf);
    if (bias) {
      // bias gradient: thread (co, half) sums half of the sub-block's voxels
      const int co = tid & 63, half = tid >> 6;
      if (co < cout_pad) {
        const __nv_bfloat16 *G = reinterpret_cast<const __nv_bfloat16 *>(smem + (sb & 1) * kBuf);
        for (int k = half * 128; k < half * 128 + 128; ++k) bsum += __bfloat162float(G[(co >> 3) * 2048 + k * 8 + (co & 7)]);
      }
    }
    if (!mbar_wait(bar_s, (uint32_t)(sb & 1))) {
      ok = false;
      break;
    }
    cp_async_wait_all();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    const int co = 16 * warp + (lane & 15);
    for (int t = 0; t < 27; ++t) {
      uint32_t r[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(t * 16);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr)
          : "memory");
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (lane < 16 && co < cout_real) {
        float *dst = dW + ((size_t)t * cout_real + co) * cin + chunk * 16;
        #pragma unroll
        for (int i = 0; i < 16; ++i) atomicAdd(dst + i, __uint_as_float(r[i]));
      }
    }
    if (bias && (tid & 63) < cout_real) atomicAdd(&db[tid & 63], bsum);
  } else {
    if (tid == 0) atomicExch(err, 1);
    // a bounded chance for the outstanding MMAs and copies to finish before
    // TMEM and shared memory are released
    mbar_wait(bar_s, 0);
    mbar_wait(bar_s, 1);
    cp_async_wait_all();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
}

__global__ void k_adam(float *w, const float *g, float *m, float *v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// Scale-invariant energy loss: L(z) = g E(c z) with E(y) = 1/2 y.A y - y.r
// and c = z.r / z.A z the best step along z, i.e. -g/2 (z.r)^2 / z.A z, the
// energy a conjugate-direction step along z removes. Its gradient is
// dL/dz = g c (c A z - r); it does not reward shrinking z, which the plain
// energy does while the output is still uncorrelated with the error. Writes
// the gradient into the dense FP32 output gradient and the loss terms.
__global__ void k_energy_grad(Geometry G, int NX, int NY, const int *pool_tile, int K, const uint8_t *unk,
                              const float *Az, const float *zp, const float *rp, float cz, float gscale, float *gZ,
                              double *partials) {
  __shared__ double red[8];
  double e = 0.0;
  const size_t n = (size_t)K * SHKZ_TC;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    const int pt = (int)(o >> 9), c = (int)(o & 511);
    const long long t = pool_tile[pt];
    const int x = (int)(t % G.bx) * 8 + (c & 7), y = (int)((t / G.bx) % G.by) * 8 + ((c >> 3) & 7),
              z = (int)(t / ((long long)G.bx * G.by)) * 8 + (c >> 6);
    if (x >= G.nx || y >= G.ny || z >= G.nz) continue;
    if (!unk[(size_t)x + (size_t)G.nx * ((size_t)y + (size_t)G.ny * z)]) continue;
    const float q = cz * Az[o] - rp[o];
    gZ[((size_t)z * NY + y) * NX + x] = gscale * q;
    e += 0.5 * (double)cz * cz * zp[o] * Az[o] - (double)cz * zp[o] * rp[o];
  }
  e = block_sum<256>(e, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = e;
}

// z.r and z.A z over the pool (both zero outside unknowns)
__global__ void k_dot2_pool(size_t n, const float *z, const float *r, const float *Az, double *partials) {
  __shared__ double red[8];
  double a = 0.0, b = 0.0;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    a += (double)z[o] * r[o];
    b += (double)z[o] * Az[o];
  }
  a = block_sum<256>(a, red);
  b = block_sum<256>(b, red);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = a;
    partials[2 * blockIdx.x + 1] = b;
  }
}

// ---------------------------------------------------------------------------
// model

struct LayerDef {
  const char *name;
  int level;
  int in0, c0, in1, c1;  // tensor ids and channel counts
  int cout, relu, out;   // output tensor id
};
// tensor ids
enum { T_X0, T_A1, T_S1, T_P1, T_A2, T_S2, T_P2, T_A3, T_B3, T_C2, T_D2, T_C1, T_D1, T_COUNT };
static const int kTensorLevel[T_COUNT] = {0, 0, 0, 1, 1, 1, 2, 2, 2, 1, 1, 0, 0};
static const int kTensorC[T_COUNT] = {16, 16, 16, 16, 32, 32, 32, 64, 64, 32, 32, 16, 16};
static const LayerDef kLayers[11] = {
    {"e1a", 0, T_X0, 16, -1, 0, 16, 1, T_A1}, {"e1b", 0, T_A1, 16, -1, 0, 16, 1, T_S1},
    {"e2a", 1, T_P1, 16, -1, 0, 32, 1, T_A2}, {"e2b", 1, T_A2, 32, -1, 0, 32, 1, T_S2},
    {"e3a", 2, T_P2, 32, -1, 0, 64, 1, T_A3}, {"e3b", 2, T_A3, 64, -1, 0, 64, 1, T_B3},
    {"d2a", 1, T_S2, 32, T_B3, 64, 32, 1, T_C2}, {"d2b", 1, T_C2, 32, -1, 0, 32, 1, T_D2},
    {"d1a", 0, T_S1, 16, T_D2, 32, 16, 1, T_C1}, {"d1b", 0, T_C1, 16, -1, 0, 16, 1, T_D1},
    {"out", 0, T_D1, 16, -1, 0, 1, 0, -1},
};

struct LayerParams {
  int cin, cout, n_pad;
  int nt_pad;  // N of the input-gradient MMA: cin rounded up to a power of two (>= 16)
  size_t nw;
  float *w = nullptr, *b = nullptr;          // FP32 master
  float *gw = nullptr, *gb = nullptr;        // gradients
  float *mw = nullptr, *vw = nullptr, *mb = nullptr, *vb = nullptr;
  __nv_bfloat16 *wpk = nullptr, *wpk_t = nullptr;
};

struct LearnedModel {
  int device = 0;
  LayerParams L[11];
  int adam_t = 0;
  // grid-dependent
  int NX[3] = {0, 0, 0}, NY[3] = {0, 0, 0}, NZ[3] = {0, 0, 0};
  int gb[3][3] = {};
  size_t cap_vox0 = 0;
  uint8_t *blk[3] = {nullptr, nullptr, nullptr};
  uint8_t *blkd[3] = {nullptr, nullptr, nullptr};  // dilated by one block
  __nv_bfloat16 *T[T_COUNT] = {};
  float *Gt[T_COUNT] = {};
  float *Z = nullptr, *gZ = nullptr;
  __nv_bfloat16 *gpre = nullptr, *gx = nullptr;
  int *err = nullptr;
  double *partials = nullptr;
  size_t params_total = 0;
  long long nactive[3] = {0, 0, 0};  // active 8x16x8 blocks per level (last prepare)
};

static size_t nvox(const LearnedModel *m, int l) { return (size_t)m->NX[l] * m->NY[l] * m->NZ[l]; }

void learned_free(LearnedModel *m) {
  if (!m) return;
  for (auto &L : m->L) {
    void *p[] = {L.w, L.b, L.gw, L.gb, L.mw, L.vw, L.mb, L.vb, L.wpk, L.wpk_t};
    for (void *q : p)
      if (q) cudaFree(q);
  }
  for (int l = 0; l < 3; ++l) {
    if (m->blk[l]) cudaFree(m->blk[l]);
    if (m->blkd[l]) cudaFree(m->blkd[l]);
  }
  for (int t = 0; t < T_COUNT; ++t) {
    if (m->T[t]) cudaFree(m->T[t]);
    if (m->Gt[t]) cudaFree(m->Gt[t]);
  }
  void *q[] = {m->Z, m->gZ, m->gpre, m->gx, m->err, m->partials};
  for (void *p : q)
    if (p) cudaFree(p);
  delete m;
}

static int grid_blocks(size_t n, int per, int cap) {
  size_t g = (n + per - 1) / per;
  if (g > (size_t)cap) g = cap;
  return g < 1 ? 1 : (int)g;
}

static int repack(LearnedModel *m, int li, cudaStream_t s) {
  LayerParams &P = m->L[li];
  const LayerDef &D = kLayers[li];
  const int cin = D.c0 + D.c1;
  count_launches(2);
  k_pack_weights<<<grid_blocks((size_t)27 * P.n_pad * cin, 256, 1024), 256, 0, s>>>(P.w, P.cout, cin, P.n_pad, cin, 0,
                                                                                     P.wpk);
  // input-gradient weights: n = forward input channel (rows padded to nt_pad),
  // k = forward output channel padded to 16
  k_pack_weights<<<grid_blocks((size_t)27 * P.nt_pad * P.n_pad, 256, 1024), 256, 0, s>>>(P.w, P.cout, cin, P.nt_pad,
                                                                                           P.n_pad, 1, P.wpk_t);
  return cudaGetLastError() == cudaSuccess ? 0 : SHKZ_B200_ERR_CUDA;
}

LearnedModel *learned_create(int device) {
  LearnedModel *m = new LearnedModel();
  m->device = device;
  bool ok = cudaMalloc(&m->err, sizeof(int)) == cudaSuccess &&
            cudaMalloc(&m->partials, sizeof(double) * 8192) == cudaSuccess;
  size_t total = 0;
  for (int li = 0; li < 11 && ok; ++li) {
    const LayerDef &D = kLayers[li];
    LayerParams &P = m->L[li];
    P.cin = D.c0 + D.c1;
    P.cout = D.cout;
    P.n_pad = D.cout < 16 ? 16 : D.cout;
    P.nt_pad = 16;
    while (P.nt_pad < P.cin) P.nt_pad <<= 1;
    P.nw = (size_t)27 * P.cout * P.cin;
    total += P.nw + P.cout;
    ok = ok && cudaMalloc(&P.w, P.nw * 4) == cudaSuccess && cudaMalloc(&P.b, P.cout * 4) == cudaSuccess &&
         cudaMalloc(&P.gw, P.nw * 4) == cudaSuccess && cudaMalloc(&P.gb, P.cout * 4) == cudaSuccess &&
         cudaMalloc(&P.mw, P.nw * 4) == cudaSuccess && cudaMalloc(&P.vw, P.nw * 4) == cudaSuccess &&
         cudaMalloc(&P.mb, P.cout * 4) == cudaSuccess && cudaMalloc(&P.vb, P.cout * 4) == cudaSuccess &&
         cudaMalloc(&P.wpk, (size_t)27 * P.n_pad * P.cin * 2) == cudaSuccess &&
         cudaMalloc(&P.wpk_t, (size_t)27 * P.nt_pad * P.n_pad * 2) == cudaSuccess;
    if (ok) {
      cudaMemset(P.mw, 0, P.nw * 4);
      cudaMemset(P.vw, 0, P.nw * 4);
      cudaMemset(P.mb, 0, P.cout * 4);
      cudaMemset(P.vb, 0, P.cout * 4);
      cudaMemset(P.b, 0, P.cout * 4);
    }
  }
  m->params_total = total;
  if (!ok) {
    learned_free(m);
    return nullptr;
  }
  return m;
}

size_t learned_param_count(const LearnedModel *m) { return m->params_total; }

// weights blob: per layer w[27][cout][cin] then b[cout], FP32, layer order above
int learned_set_params(LearnedModel *m, const float *blob, size_t n, cudaStream_t s) {
  if (n != m->params_total) return SHKZ_B200_ERR_ARG;
  size_t off = 0;
  for (int li = 0; li < 11; ++li) {
    LayerParams &P = m->L[li];
    if (cudaMemcpyAsync(P.w, blob + off, P.nw * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return SHKZ_B200_ERR_CUDA;
    off += P.nw;
    if (cudaMemcpyAsync(P.b, blob + off, P.cout * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return SHKZ_B200_ERR_CUDA;
    off += P.cout;
    int rc = repack(m, li, s);
    if (rc) return rc;
  }
  return cudaStreamSynchronize(s) == cudaSuccess ? 0 : SHKZ_B200_ERR_CUDA;
}

int learned_get_params(LearnedModel *m, float *blob, size_t n, int grads, cudaStream_t s) {
  if (n != m->params_total) return SHKZ_B200_ERR_ARG;
  size_t off = 0;
  for (int li = 0; li < 11; ++li) {
    LayerParams &P = m->L[li];
    if (cudaMemcpyAsync(blob + off, grads ? P.gw : P.w, P.nw * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess)
      return SHKZ_B200_ERR_CUDA;
    off += P.nw;
    if (cudaMemcpyAsync(blob + off, grads ? P.gb : P.b, P.cout * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess)
      return SHKZ_B200_ERR_CUDA;
    off += P.cout;
  }
  return cudaStreamSynchronize(s) == cudaSuccess ? 0 : SHKZ_B200_ERR_CUDA;
}

// He-normal initialisation (same rule as the CPU restatement), from a seed.
int learned_init_params(LearnedModel *m, unsigned seed, cudaStream_t s) {
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> nd(0.f, 1.f);
  std::vector<float> blob(m->params_total);
  size_t off = 0;
  for (int li = 0; li < 11; ++li) {
    const LayerDef &D = kLayers[li];
    LayerParams &P = m->L[li];
    const float fan = 27.f * (li == 0 ? 3.f : (float)P.cin);
    const float sc = std::sqrt(2.f / fan) * (li == 10 ? 0.1f : 1.f);
    for (size_t i = 0; i < P.nw; ++i) {
      const int ci = (int)(i % P.cin);
      blob[off + i] = (li == 0 && ci >= 3) ? 0.f : nd(rng) * sc;
    }
    off += P.nw;
    for (int c = 0; c < P.cout; ++c) blob[off + c] = 0.f;
    off += P.cout;
    (void)D;
  }
  return learned_set_params(m, blob.data(), blob.size(), s);
}

// (Re)size tensors for the grid and recompute block activity from the pool.
int learned_prepare(LearnedModel *m, const Geometry &G, const int *tile_state, cudaStream_t s) {
  int NX = (G.nx + 3) & ~3, NY = (G.ny + 3) & ~3, NZ = (G.nz + 3) & ~3;
  const bool resize = NX != m->NX[0] || NY != m->NY[0] || NZ != m->NZ[0];
  for (int l = 0; l < 3; ++l) {
    m->NX[l] = NX >> l;
    m->NY[l] = NY >> l;
    m->NZ[l] = NZ >> l;
    m->gb[l][0] = (m->NX[l] + 7) / 8;
    m->gb[l][1] = (m->NY[l] + 15) / 16;
    m->gb[l][2] = (m->NZ[l] + 7) / 8;
  }
  if (resize) {
    for (int l = 0; l < 3; ++l) {
      if (m->blk[l]) cudaFree(m->blk[l]);
      if (m->blkd[l]) cudaFree(m->blkd[l]);
      const size_t nb = (size_t)m->gb[l][0] * m->gb[l][1] * m->gb[l][2];
      if (cudaMalloc(&m->blk[l], nb) != cudaSuccess || cudaMalloc(&m->blkd[l], nb) != cudaSuccess)
        return SHKZ_B200_ERR_NOMEM;
    }
    for (int t = 0; t < T_COUNT; ++t) {
      if (m->T[t]) cudaFree(m->T[t]);
      if (m->Gt[t]) cudaFree(m->Gt[t]);
      const size_t n = nvox(m, kTensorLevel[t]) * kTensorC[t];
      if (cudaMalloc(&m->T[t], n * 2) != cudaSuccess || cudaMalloc(&m->Gt[t], n * 4) != cudaSuccess)
        return SHKZ_B200_ERR_NOMEM;
    }
    if (m->Z) cudaFree(m->Z);
    if (m->gZ) cudaFree(m->gZ);
    if (m->gpre) cudaFree(m->gpre);
    if (m->gx) cudaFree(m->gx);
    const size_t n0 = nvox(m, 0);
    if (cudaMalloc(&m->Z, n0 * 4) != cudaSuccess || cudaMalloc(&m->gZ, n0 * 4) != cudaSuccess ||
        cudaMalloc(&m->gpre, n0 * 64 * 2) != cudaSuccess || cudaMalloc(&m->gx, n0 * 64 * 2) != cudaSuccess)
      return SHKZ_B200_ERR_NOMEM;
  }
  for (int l = 0; l < 3; ++l) {
    count_launches(1);
    k_block_activity<<<grid_blocks((size_t)m->gb[l][0] * m->gb[l][1] * m->gb[l][2], 256, 1024), 256, 0, s>>>(
        G, tile_state, l, m->gb[l][0], m->gb[l][1], m->gb[l][2], m->blk[l]);
    count_launches(1);
    k_block_dilate<<<grid_blocks((size_t)m->gb[l][0] * m->gb[l][1] * m->gb[l][2], 256, 1024), 256, 0, s>>>(
        m->blk[l], m->gb[l][0], m->gb[l][1], m->gb[l][2], m->blkd[l]);
  }
  // tensors are zero outside active blocks: clear them once per system
  for (int t = 0; t < T_COUNT; ++t)
    cudaMemsetAsync(m->T[t], 0, nvox(m, kTensorLevel[t]) * kTensorC[t] * 2, s);
  cudaMemsetAsync(m->Z, 0, nvox(m, 0) * 4, s);
  cudaMemsetAsync(m->gpre, 0, nvox(m, 0) * 64 * 2, s);
  cudaMemsetAsync(m->gx, 0, nvox(m, 0) * 64 * 2, s);
  cudaMemsetAsync(m->err, 0, sizeof(int), s);
  {
    // active blocks per level, for the FLOP count of an application
    for (int l = 0; l < 3; ++l) {
      const size_t nb = (size_t)m->gb[l][0] * m->gb[l][1] * m->gb[l][2];
      std::vector<uint8_t> h(nb);
      if (cudaMemcpyAsync(h.data(), m->blk[l], nb, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess)
        return SHKZ_B200_ERR_CUDA;
      long long c = 0;
      for (uint8_t v : h) c += v != 0;
      m->nactive[l] = c;
    }
  }
  return cudaGetLastError() == cudaSuccess ? 0 : SHKZ_B200_ERR_CUDA;
}

static int conv_launch(LearnedModel *m, int level, const __nv_bfloat16 *in0, int c0, const __nv_bfloat16 *in1, int c1,
                       const __nv_bfloat16 *wpk, const float *bias, int bias_n, int cout, int relu,
                       __nv_bfloat16 *out, float *out32, cudaStream_t s, bool dilated = false) {
  ConvArgs a;
  a.in0 = in0;
  a.in1 = in1;
  a.c0 = c0;
  a.c1 = c1;
  a.nx = m->NX[level];
  a.ny = m->NY[level];
  a.nz = m->NZ[level];
  a.hx = level < 2 ? m->NX[level + 1] : 0;
  a.hy = level < 2 ? m->NY[level + 1] : 0;
  a.hz = level < 2 ? m->NZ[level + 1] : 0;
  a.wpk = wpk;
  a.bias = bias;
  a.bias_n = bias_n;
  a.cout = cout;
  a.relu = relu;
  a.out = out;
  a.out32 = out32;
  a.block_act = dilated ? m->blkd[level] : m->blk[level];
  a.gbx = m->gb[level][0];
  a.gby = m->gb[level][1];
  a.gbz = m->gb[level][2];
  a.planes = cout <= 32 ? 8 : 4;
  a.err = m->err;
  const size_t smem = conv_smem_bytes(a.planes, cout);
  cudaFuncSetAttribute(k_conv_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  const int nblocks = a.gbx * a.gby * a.gbz * (8 / a.planes);
  launch_conv_tc(a, nblocks, smem, s);
  return cudaGetLastError() == cudaSuccess ? 0 : SHKZ_B200_ERR_CUDA;
}

// Forward pass; X0 already built. Output Z (FP32 dense, level 0).
static int forward(LearnedModel *m, cudaStream_t s) {
  for (int li = 0; li < 11; ++li) {
    const LayerDef &D = kLayers[li];
    const LayerParams &P = m->L[li];
    if (li == 2) {
      count_launches(1);
      k_avgpool<<<grid_blocks(nvox(m, 1) * 16, 256, 148 * 16), 256, 0, s>>>(
          m->T[T_S1], m->NX[0], m->NY[0], 16, m->T[T_P1], m->NX[1], m->NY[1], m->NZ[1], m->blk[1], m->gb[1][0],
          m->gb[1][1]);
    }
    if (li == 4) {
      count_launches(1);
      k_avgpool<<<grid_blocks(nvox(m, 2) * 32, 256, 148 * 16), 256, 0, s>>>(
          m->T[T_S2], m->NX[1], m->NY[1], 32, m->T[T_P2], m->NX[2], m->NY[2], m->NZ[2], m->blk[2], m->gb[2][0],
          m->gb[2][1]);
    }
    int rc = conv_launch(m, D.level, m->T[D.in0], D.c0, D.in1 >= 0 ? m->T[D.in1] : nullptr, D.c1, P.wpk, P.b,
                         P.cout, P.n_pad, D.relu, D.out >= 0 ? m->T[D.out] : nullptr, D.out >= 0 ? nullptr : m->Z, s);
    if (rc) return rc;
  }
  return 0;
}

// Backward of sum(gZ * Z): weight/bias gradients into L[].gw/gb (zeroed first).
static int backward(LearnedModel *m, cudaStream_t s) {
  for (int li = 0; li < 11; ++li) {
    cudaMemsetAsync(m->L[li].gw, 0, m->L[li].nw * 4, s);
    cudaMemsetAsync(m->L[li].gb, 0, m->L[li].cout * 4, s);
  }
  for (int t = 0; t < T_COUNT; ++t) cudaMemsetAsync(m->Gt[t], 0, nvox(m, kTensorLevel[t]) * kTensorC[t] * 4, s);
  for (int li = 10; li >= 0; --li) {
    const LayerDef &D = kLayers[li];
    const LayerParams &P = m->L[li];
    const int lv = D.level;
    const size_t nv = nvox(m, lv);
    // pre-activation gradient (BF16, n_pad channels)
    if (li == 10) {
      count_launches(1);
      k_grad_pre<<<grid_blocks(nv * P.n_pad, 256, 148 * 16), 256, 0, s>>>(
          m->gZ, nullptr, 1, P.n_pad, 0, nv, m->NX[lv], m->NY[lv], m->blk[lv], m->gb[lv][0], m->gb[lv][1], m->gpre);
    } else {
      count_launches(1);
      k_grad_pre<<<grid_blocks(nv * P.n_pad, 256, 148 * 16), 256, 0, s>>>(
          m->Gt[D.out], m->T[D.out], P.cout, P.n_pad, D.relu, nv, m->NX[lv], m->NY[lv], m->blk[lv], m->gb[lv][0],
          m->gb[lv][1], m->gpre);
    }
    // weight and bias gradients on the tensor cores (one CTA per SM: it holds
    // all 512 TMEM columns, and its 120 KB of shared memory keeps a second
    // CTA from waiting in the allocation)
    {
      const int cin = D.c0 + D.c1;
      const size_t smem = 120 * 1024;
      cudaFuncSetAttribute(k_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      const int nb = m->gb[lv][0] * m->gb[lv][1] * m->gb[lv][2] * (cin / 16);
      count_launches(1);
      k_wgrad_tc<<<nb, 128, smem, s>>>(m->gpre, P.n_pad, P.cout, m->T[D.in0], D.c0,
                                       D.in1 >= 0 ? m->T[D.in1] : nullptr, D.c1, m->NX[lv], m->NY[lv], m->NZ[lv],
                                       lv < 2 ? m->NX[lv + 1] : 0, lv < 2 ? m->NY[lv + 1] : 0,
                                       lv < 2 ? m->NZ[lv + 1] : 0, m->blk[lv], m->gb[lv][0], m->gb[lv][1],
                                       m->gb[lv][2], P.gw, P.gb, m->err);
    }
    if (li == 0) break;  // no input gradient needed for the first layer
    // input gradient: conv of gpre with the flipped, transposed weights
    // (N = nt_pad channels per voxel in gx; the first cin are meaningful),
    // over the active blocks and their neighbours, zero elsewhere
    cudaMemsetAsync(m->gx, 0, nv * P.nt_pad * 2, s);
    int rc = conv_launch(m, lv, m->gpre, P.n_pad, nullptr, 0, P.wpk_t, nullptr, 0, P.nt_pad, 0, m->gx, nullptr, s,
                         true);
    if (rc) return rc;
    count_launches(1);
    k_split_grad<<<grid_blocks(nv * D.c0, 256, 148 * 16), 256, 0, s>>>(m->gx, P.nt_pad, D.c0, nv, m->Gt[D.in0],
                                                                         m->blk[lv], m->NX[lv], m->NY[lv],
                                                                         m->gb[lv][0], m->gb[lv][1]);
    if (D.in1 >= 0) {
      const int l1 = lv + 1;
      count_launches(1);
      k_up_grad<<<grid_blocks(nvox(m, l1) * D.c1, 256, 148 * 16), 256, 0, s>>>(
          m->gx, P.nt_pad, D.c0, m->NX[lv], m->NY[lv], m->NZ[lv], m->Gt[D.in1], D.c1, m->NX[l1], m->NY[l1],
          m->NZ[l1], m->blk[l1], m->gb[l1][0], m->gb[l1][1]);
    }
    if (li == 2 || li == 4) {
      // pooled input: propagate to the finer skip tensor
      const int tc = li == 2 ? T_P1 : T_P2, tf = li == 2 ? T_S1 : T_S2, lc = lv, lf = lv - 1;
      count_launches(1);
      k_pool_grad<<<grid_blocks(nvox(m, lc) * kTensorC[tc], 256, 148 * 16), 256, 0, s>>>(
          m->Gt[tc], kTensorC[tc], m->NX[lc], m->NY[lc], m->NZ[lc], m->blk[lc], m->gb[lc][0], m->gb[lc][1], m->Gt[tf],
          m->NX[lf], m->NY[lf]);
    }
  }
  return cudaGetLastError() == cudaSuccess ? 0 : SHKZ_B200_ERR_CUDA;
}

static int adam_step(LearnedModel *m, float lr, cudaStream_t s) {
  m->adam_t += 1;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.f - std::pow(b1, (float)m->adam_t), c2 = 1.f - std::pow(b2, (float)m->adam_t);
  for (int li = 0; li < 11; ++li) {
    LayerParams &P = m->L[li];
    count_launches(2);
    k_adam<<<grid_blocks(P.nw, 256, 1024), 256, 0, s>>>(P.w, P.gw, P.mw, P.vw, (int)P.nw, lr, b1, b2, eps, c1, c2);
    k_adam<<<1, 64, 0, s>>>(P.b, P.gb, P.mb, P.vb, P.cout, lr, b1, b2, eps, c1, c2);
    int rc = repack(m, li, s);
    if (rc) return rc;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Stand-alone run of the convolution kernel (unit tests): host arrays in and
// out; weights w[27][cout][c0+c1] FP32 are packed on the device, every block
// is active.
int conv3d_run(int nx, int ny, int nz, int c0, int c1, int cout, int planes, const float *in0_h, const float *in1_h,
               const float *w_h, const float *bias_h, int relu, float *out_h) {
  const int cin = c0 + c1;
  int n_pad = 16;
  while (n_pad < cout) n_pad <<= 1;
  const size_t n0 = (size_t)nx * ny * nz, n1 = (size_t)(nx / 2) * (ny / 2) * (nz / 2);
  std::vector<__nv_bfloat16> b0(n0 * c0), b1(n1 * (c1 ? c1 : 1));
  for (size_t i = 0; i < n0 * c0; ++i) b0[i] = __float2bfloat16_rn(in0_h[i]);
  for (size_t i = 0; c1 && i < n1 * c1; ++i) b1[i] = __float2bfloat16_rn(in1_h[i]);
  __nv_bfloat16 *d0 = nullptr, *d1 = nullptr, *dw = nullptr, *dout = nullptr;
  float *dwf = nullptr, *db = nullptr;
  uint8_t *act = nullptr;
  int *err = nullptr;
  const int gbx = (nx + 7) / 8, gby = (ny + 15) / 16, gbz = (nz + 7) / 8;
  bool ok = cudaMalloc(&d0, b0.size() * 2) == cudaSuccess && cudaMalloc(&d1, b1.size() * 2) == cudaSuccess &&
            cudaMalloc(&dwf, (size_t)27 * cout * cin * 4) == cudaSuccess &&
            cudaMalloc(&dw, (size_t)27 * n_pad * cin * 2) == cudaSuccess &&
            cudaMalloc(&db, (size_t)n_pad * 4) == cudaSuccess && cudaMalloc(&dout, n0 * n_pad * 2) == cudaSuccess &&
            cudaMalloc(&act, (size_t)gbx * gby * gbz) == cudaSuccess && cudaMalloc(&err, 4) == cudaSuccess;
  int rc = ok ? 0 : SHKZ_B200_ERR_NOMEM;
  if (ok) {
    cudaMemcpy(d0, b0.data(), b0.size() * 2, cudaMemcpyHostToDevice);
    cudaMemcpy(d1, b1.data(), b1.size() * 2, cudaMemcpyHostToDevice);
    cudaMemcpy(dwf, w_h, (size_t)27 * cout * cin * 4, cudaMemcpyHostToDevice);
    cudaMemset(db, 0, (size_t)n_pad * 4);
    if (bias_h) cudaMemcpy(db, bias_h, (size_t)cout * 4, cudaMemcpyHostToDevice);
    cudaMemset(act, 1, (size_t)gbx * gby * gbz);
    cudaMemset(err, 0, 4);
    cudaMemset(dout, 0, n0 * n_pad * 2);
    count_launches(1);
    k_pack_weights<<<256, 256>>>(dwf, cout, cin, n_pad, cin, 0, dw);
    ConvArgs a;
    a.in0 = d0;
    a.in1 = c1 ? d1 : nullptr;
    a.c0 = c0;
    a.c1 = c1;
    a.nx = nx; a.ny = ny; a.nz = nz;
    a.hx = nx / 2; a.hy = ny / 2; a.hz = nz / 2;
    a.wpk = dw;
    a.bias = db;
    a.bias_n = cout;
    a.cout = n_pad;
    a.relu = relu;
    a.out = dout;
    a.out32 = nullptr;
    a.block_act = act;
    a.gbx = gbx; a.gby = gby; a.gbz = gbz;
    a.planes = planes;
    a.err = err;
    cudaFuncSetAttribute(k_conv_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    launch_conv_tc(a, gbx * gby * gbz * (8 / planes), conv_smem_bytes(planes, n_pad), 0);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) rc = SHKZ_B200_ERR_CUDA;
    int herr = 0;
    cudaMemcpy(&herr, err, 4, cudaMemcpyDeviceToHost);
    if (herr) rc = SHKZ_B200_ERR_TIMEOUT;
    std::vector<__nv_bfloat16> ho(n0 * n_pad);
    cudaMemcpy(ho.data(), dout, ho.size() * 2, cudaMemcpyDeviceToHost);
    for (size_t v = 0; v < n0; ++v)
      for (int c = 0; c < cout; ++c) out_h[v * cout + c] = __bfloat162float(ho[v * n_pad + c]);
  }
  void *ptrs[] = {d0, d1, dw, dout, dwf, db, act, err};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  return rc;
}

__global__ void k_fill_u8(uint8_t *a, int n, uint8_t v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = v;
}

// The same convolution on device arrays with caller-provided scratch (packed
// weights, block activity, error word); launches on `s` and returns without
// synchronising. cout must be 16, 32, 64 or 128 (output stride = cout).
int conv3d_launch_scratch(int nx, int ny, int nz, int c0, int c1, int cout, int planes, const __nv_bfloat16 *in0,
                          const __nv_bfloat16 *in1, const float *w, const float *bias, int relu, __nv_bfloat16 *out,
                          __nv_bfloat16 *wpk, uint8_t *act, int *err, cudaStream_t s) {
  const int cin = c0 + c1;
  const int gbx = (nx + 7) / 8, gby = (ny + 15) / 16, gbz = (nz + 7) / 8;
  const int nb = gbx * gby * gbz;
  count_launches(2);
  k_pack_weights<<<256, 256, 0, s>>>(w, cout, cin, cout, cin, 0, wpk);
  k_fill_u8<<<grid_blocks((size_t)nb, 256, 1024), 256, 0, s>>>(act, nb, 1);
  if (cudaMemsetAsync(err, 0, sizeof(int), s) != cudaSuccess) return SHKZ_B200_ERR_CUDA;
  ConvArgs a;
  a.in0 = in0;
  a.in1 = c1 ? in1 : nullptr;
  a.c0 = c0;
  a.c1 = c1;
  a.nx = nx; a.ny = ny; a.nz = nz;
  a.hx = nx / 2; a.hy = ny / 2; a.hz = nz / 2;
  a.wpk = wpk;
  a.bias = bias;
  a.bias_n = cout;
  a.cout = cout;
  a.relu = relu;
  a.out = out;
  a.out32 = nullptr;
  a.block_act = act;
  a.gbx = gbx; a.gby = gby; a.gbz = gbz;
  a.planes = planes;
  a.err = err;
  if (cudaFuncSetAttribute(k_conv_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess)
    return SHKZ_B200_ERR_CUDA;
  launch_conv_tc(a, nb * (8 / planes), conv_smem_bytes(planes, cout), s);
  return cudaGetLastError() == cudaSuccess ? 0 : SHKZ_B200_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// entry points used by the context (api.cu)

int learned_apply(LearnedModel *m, const LearnedSystem &sys, const float *r_pool, double rmax, float *z_pool,
                  cudaStream_t s) {
  const double inv = rmax > 0 ? 1.0 / rmax : 0.0;
  count_launches(1);
  k_make_input<<<grid_blocks(nvox(m, 0), 256, 148 * 16), 256, 0, s>>>(
      sys.G, m->NX[0], m->NY[0], m->NZ[0], sys.tile_state, r_pool, sys.unk, sys.fluid, sys.solid, inv, 1.0 / sys.dx,
      m->blk[0], m->gb[0][0], m->gb[0][1], m->T[T_X0]);
  int rc = forward(m, s);
  if (rc) return rc;
  count_launches(1);
  k_gather_output<<<grid_blocks((size_t)sys.K * SHKZ_TC, 256, 148 * 16), 256, 0, s>>>(
      sys.G, m->NX[0], m->NY[0], sys.pool_tile, sys.K, sys.unk, m->Z, rmax, z_pool);
  return cudaGetLastError() == cudaSuccess ? 0 : SHKZ_B200_ERR_CUDA;
}

int learned_backward_dense(LearnedModel *m, const float *gZ_dense, cudaStream_t s) {
  cudaMemcpyAsync(m->gZ, gZ_dense, nvox(m, 0) * 4, cudaMemcpyDeviceToDevice, s);
  return backward(m, s);
}

int learned_output_dense(LearnedModel *m, float *Z_dense_dev, cudaStream_t s) {
  return cudaMemcpyAsync(Z_dense_dev, m->Z, nvox(m, 0) * 4, cudaMemcpyDeviceToDevice, s) == cudaSuccess
             ? 0 : SHKZ_B200_ERR_CUDA;
}

size_t learned_dense_cells(const LearnedModel *m) { return nvox(m, 0); }

// FLOPs of one application as the tensor cores execute it: every layer's 3^3
// convolution over the active 8x16x8 blocks of its level, 2 * 27 * C_in * C_out
// per voxel.
double learned_forward_flops(const LearnedModel *m) {
  double f = 0.0;
  for (int li = 0; li < 11; ++li) {
    const LayerDef &d = kLayers[li];
    const double vox = (double)m->nactive[d.level] * 8 * 16 * 8;
    f += vox * 2.0 * 27.0 * (double)(d.c0 + d.c1) * (double)d.cout;
  }
  return f;
}

__global__ void k_bf16_to_f32(const __nv_bfloat16 *a, size_t n, float *b) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = __bfloat162float(a[i]);
}
// Stored activation tensor `t` (0 = X0 ... 12 = D1) as FP32 into a device
// buffer of learned_tensor_size(t) floats.
size_t learned_tensor_size(const LearnedModel *m, int t) {
  if (t < 0 || t >= T_COUNT) return 0;
  return nvox(m, kTensorLevel[t]) * kTensorC[t];
}
void learned_tensor_shape(const LearnedModel *m, int t, int *shape4) {
  const int l = kTensorLevel[t];
  shape4[0] = m->NZ[l];
  shape4[1] = m->NY[l];
  shape4[2] = m->NX[l];
  shape4[3] = kTensorC[t];
}
int learned_grad_dense(LearnedModel *m, int t, float *out, cudaStream_t s) {
  const size_t n = learned_tensor_size(m, t);
  if (!n) return SHKZ_B200_ERR_ARG;
  return cudaMemcpyAsync(out, m->Gt[t], n * 4, cudaMemcpyDeviceToDevice, s) == cudaSuccess ? 0 : SHKZ_B200_ERR_CUDA;
}
int learned_tensor_dense(LearnedModel *m, int t, float *out, cudaStream_t s) {
  const size_t n = learned_tensor_size(m, t);
  if (!n) return SHKZ_B200_ERR_ARG;
  count_launches(1);
  k_bf16_to_f32<<<grid_blocks(n, 256, 148 * 16), 256, 0, s>>>(m->T[t], n, out);
  return cudaGetLastError() == cudaSuccess ? 0 : SHKZ_B200_ERR_CUDA;
}
void learned_dense_dims(const LearnedModel *m, int *nx, int *ny, int *nz) {
  *nx = m->NX[0];
  *ny = m->NY[0];
  *nz = m->NZ[0];
}

// One training step on the energy loss 1/2 z.A z - z.r (gradient A z - r, the
// gradient of the A-norm error 1/2 (z - A^-1 r).A (z - A^-1 r)), r scaled to
// ||r||inf = 1. Az_pool and z_pool are scratch pool vectors.
int learned_train_step(LearnedModel *m, const LearnedSystem &sys, const PoolSystem &S, const float *r_pool,
                       float *z_pool, float *Az_pool, double *partials, unsigned *counter, float lr, double gscale,
                       double *loss, cudaStream_t s) {
  int rc = learned_apply(m, sys, r_pool, 1.0, z_pool, s);
  if (rc) return rc;
  launch_spmv(S, z_pool, Az_pool, partials, counter, nullptr, 1, s);
  const int nb = 148 * 4;
  // best step c along z (plain energy gradient while z.A z is not yet positive)
  std::vector<double> hd(2 * nb);
  count_launches(1);
  k_dot2_pool<<<nb, 256, 0, s>>>((size_t)sys.K * SHKZ_TC, z_pool, r_pool, Az_pool, m->partials);
  if (cudaMemcpyAsync(hd.data(), m->partials, sizeof(double) * 2 * nb, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return SHKZ_B200_ERR_CUDA;
  double zr = 0.0, zaz = 0.0;
  for (int i = 0; i < nb; ++i) {
    zr += hd[2 * i];
    zaz += hd[2 * i + 1];
  }
  const double c = (zaz > 0.0 && zaz < 1e300 && zr == zr) ? zr / zaz : 1.0;
  cudaMemsetAsync(m->gZ, 0, nvox(m, 0) * 4, s);
  count_launches(1);
  k_energy_grad<<<nb, 256, 0, s>>>(sys.G, m->NX[0], m->NY[0], sys.pool_tile, sys.K, sys.unk, Az_pool, z_pool, r_pool,
                                   (float)c, (float)(gscale * c), m->gZ, m->partials);
  std::vector<double> hp(nb);
  cudaMemcpyAsync(hp.data(), m->partials, sizeof(double) * nb, cudaMemcpyDeviceToHost, s);
  rc = backward(m, s);
  if (rc) return rc;
  rc = adam_step(m, lr, s);
  if (rc) return rc;
  if (cudaStreamSynchronize(s) != cudaSuccess) return SHKZ_B200_ERR_CUDA;
  double e = 0.0;
  for (double v : hp) e += v;
  if (loss) *loss = e * gscale;
  int herr = 0;
  cudaMemcpy(&herr, m->err, sizeof(int), cudaMemcpyDeviceToHost);
  return herr ? SHKZ_B200_ERR_TIMEOUT : 0;
}

int learned_error(LearnedModel *m) {
  int herr = 0;
  cudaMemcpy(&herr, m->err, sizeof(int), cudaMemcpyDeviceToHost);
  return herr ? SHKZ_B200_ERR_TIMEOUT : 0;
}

}  // namespace shkz
