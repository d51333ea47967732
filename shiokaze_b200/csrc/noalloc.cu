// shkz_b200_conv3d_noalloc: the network's tensor-core 3^3 convolution for
// callers that cannot allocate device memory.
//
// Some host programs cannot call cudaMalloc: an application that has already
// reserved the whole device for its own pool allocator, or a time-critical
// loop that must not pay the device-wide synchronisation cudaMalloc/cudaFree
// may imply. This entry point allocates nothing. The caller passes the inputs
// and the output; the only scratch the kernel needs -- the weights packed in
// the tensor-core layout, the block-activity array and an error word -- lives
// in the file-scope array below, which every GPU that loads this library holds
// until the process exits (1.1 MiB).
//
// Host code must not hand the array's name to a kernel: on the host it is a
// stand-in symbol, not a device address. The first call on each device
// (made with that device current) looks its device address up once with
// cudaGetSymbolAddress; make that first call before any stream capture. Each
// call waits for its stream to drain and reads the error word back before it
// returns. All calls share the array and it keeps the last call's contents: each call
// rewrites the packed weights and the activity bytes it uses and clears the
// error word. Calls that overlap on the GPU (other streams, other host
// threads) race on the array; serialise them.
#include "common.cuh"
#include "learned.h"
#include "../../include/shkz_b200.h"

#include <mutex>

namespace {

constexpr int kMaxCin = 128;                            // c0 + c1
constexpr int kMaxCout = 128;
constexpr size_t kWpkBytes = (size_t)27 * kMaxCout * kMaxCin * 2;  // packed BF16 weights
constexpr size_t kMaxBlocks = (size_t)1 << 18;          // 8x16x8 output blocks (a 512^3 grid)
constexpr size_t kScratchBytes = kWpkBytes + kMaxBlocks + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_base[kMaxDevices] = {};

// Device address of the scratch array on the current device (set up once).
int scratch_base(int dev, unsigned char **out) {
  if (dev < 0 || dev >= kMaxDevices) return SHKZ_B200_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_base[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      shkz_set_cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
      return SHKZ_B200_ERR_CUDA;
    }
    g_base[dev] = p;
  }
  *out = static_cast<unsigned char *>(g_base[dev]);
  return 0;
}

}  // namespace

extern "C" int shkz_b200_conv3d_noalloc(int nx, int ny, int nz, int c0, int c1, int cout, int planes,
                                        const uint16_t *in0, const uint16_t *in1, const float *w,
                                        const float *bias, int relu, uint16_t *out, void *stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || c0 <= 0 || c0 % 16 || c1 < 0 || c1 % 16 || !in0 || !w || !out ||
      (c1 && !in1) || (c1 && ((nx | ny | nz) & 1)) || (planes != 4 && planes != 8))
    return SHKZ_B200_ERR_ARG;
  // the kernel's vector loads and stores and its tensor map need 16-byte
  // aligned activations; the weight packing reads FP32 words
  const auto misaligned = [](const void *p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) != 0; };
  if (misaligned(in0, 16) || (c1 && misaligned(in1, 16)) || misaligned(out, 16) || misaligned(w, 4) ||
      (bias && misaligned(bias, 4)))
    return SHKZ_B200_ERR_ARG;
  if (cout != 16 && cout != 32 && cout != 64 && cout != 128) return SHKZ_B200_ERR_LIMIT;
  if (c0 + c1 > kMaxCin) return SHKZ_B200_ERR_LIMIT;
  // one CTA's accumulators: planes x cout FP32 columns of tensor memory (each
  // plane on a 32-column boundary), at most the 512 columns of an SM
  if (planes * ((cout + 31) & ~31) > 512) return SHKZ_B200_ERR_LIMIT;
  const size_t nb = (size_t)((nx + 7) / 8) * ((ny + 15) / 16) * ((nz + 7) / 8);
  if (nb > kMaxBlocks) return SHKZ_B200_ERR_LIMIT;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return SHKZ_B200_ERR_NODEVICE;
  unsigned char *base = nullptr;
  int rc = scratch_base(dev, &base);
  if (rc) return rc;
  __nv_bfloat16 *wpk = reinterpret_cast<__nv_bfloat16 *>(base);
  uint8_t *act = base + kWpkBytes;
  int *err = reinterpret_cast<int *>(base + kWpkBytes + kMaxBlocks);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  rc = shkz::conv3d_launch_scratch(nx, ny, nz, c0, c1, cout, planes, reinterpret_cast<const __nv_bfloat16 *>(in0),
                                   reinterpret_cast<const __nv_bfloat16 *>(in1), w, bias, relu,
                                   reinterpret_cast<__nv_bfloat16 *>(out), wpk, act, err, s);
  if (rc) return rc;
  if (cudaStreamSynchronize(s) != cudaSuccess) return SHKZ_B200_ERR_CUDA;
  int herr = 0;
  if (cudaMemcpy(&herr, err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return SHKZ_B200_ERR_CUDA;
  return herr ? SHKZ_B200_ERR_TIMEOUT : 0;
}
