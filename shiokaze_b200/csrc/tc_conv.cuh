// 3^3 convolution as an implicit GEMM on the 5th-generation tensor cores.
//
// One CTA (128 threads) computes an output block of 8 (x) x 16 (y) x P (z)
// voxels, P = 8 or 4 planes, for all Cout channels:
//   D[plane][m = 8*y + x][co] = sum_tap sum_ci W[tap][co][ci] * X[voxel(m) + off(tap)][ci]
// Each plane is one M = 128 MMA tile; N = Cout (16..96); K runs over input
// channels in chunks of 16 (one kind::f16 MMA per tap and chunk).
//
// For a chunk, the halo of the block, (P+2) x 18 x 10 voxels x 16 channels of
// BF16, is staged in shared memory in the canonical K-major no-swizzle UMMA
// layout (core matrix = 8 consecutive x voxels x 8 channels = 8 x 16 B):
//   byte(kh, z, y, x) = kh * LBO + ((z * 18 + y) * 10 + x) * 16,  LBO = (P+2)*18*10*16
// so the A operand of tap (dx,dy,dz) for plane zo is the same layout shifted by
// ((zo+dz)*18 + dy)*10 + dx entries: only the descriptor's start address
// changes (SBO = 160 B between groups of 8 rows, i.e. between y rows). The
// weights of the chunk, 27 x Cout x 16 BF16, are staged in the same canonical
// layout (SBO = 128 B between groups of 8 output channels, LBO = Cout*16 B
// between the two 8-channel halves). One thread issues all MMAs; FP32
// accumulators live in TMEM (P x Cout columns); tcgen05.commit signals an
// mbarrier that all threads wait on (bounded) before the next chunk is staged.
// The epilogue reads each warp's 32 TMEM lanes (rows) with tcgen05.ld, adds
// the bias, applies ReLU and stores BF16 channels-last (or channel 0 in FP32).
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace shkz {

struct ConvArgs {
  const __nv_bfloat16 *in0;   // channels-last at the output resolution, c0 channels
  const __nv_bfloat16 *in1;   // channels-last at half the output resolution (nearest upsampled), or null
  int c0, c1;                 // multiples of 16
  int nx, ny, nz;             // output grid
  int hx, hy, hz;             // in1 grid
  const __nv_bfloat16 *wpk;   // packed weights [chunk][tap][kh][co/8][co%8][k%8]
  const float *bias;          // [bias_n] or null (channels >= bias_n get no bias)
  int bias_n;
  int cout;                   // N of the MMA: 16, 32, 64 or 128
  int relu;
  __nv_bfloat16 *out;         // channels-last, cout channels (or null)
  float *out32;               // FP32 channel 0 (or null)
  const uint8_t *block_act;   // per 8x16x8 block, 1 = compute
  int gbx, gby, gbz;          // blocks per axis
  int planes;                 // 8 or 4 z planes per CTA
  int *err;                   // set on a bounded-wait timeout
  int tma;                    // 1: in0 halos by TMA through the tensor maps of ConvMaps
};

// Tensor maps of the in0 halos: chunk ch, 8-channel half h at m[2 ch + h],
// each a 4D view (8 channels, x, y, z) of the channels-last tensor starting at
// channel 16 ch + 8 h, box (8, 10, 18, P + 2), no swizzle, zero fill outside
// the grid. Passed as a __grid_constant__ kernel parameter.
#define CONV_MAX_TMA_CHUNKS 8
struct ConvMaps {
  CUtensorMap m[2 * CONV_MAX_TMA_CHUNKS];
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  // base offset 0, lbo mode 0, layout type 0 (no swizzle)
  return d;
}

// kind::f16 instruction descriptor: D FP32, A/B BF16, both K-major, M = 128.
__host__ __device__ __forceinline__ uint32_t umma_idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (int it = 0; it < (1 << 22); ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

}  // namespace shkz
