// MIC(0) preconditioner for the generic CSR solver path (LinSolver=pcg_b200
// with B200.Preconditioner=mic0): the reference header's own factorisation
// and triangular solves (local/include/pcgsolver/pcg_solver.h:88-223) on the
// device, for any symmetric row-sorted CSR matrix.
//
// The lower factor L keeps A's lower pattern, stored by column as the header
// stores it (column i = row i's entries right of the diagonal). The
// factorisation is left-looking: column j takes the update of every column
// k < j with L(j,k) != 0, in increasing k, exactly the updates (and their
// order) the header's right-looking loop applies to it, then is finalised.
// Columns are grouped into levels (level(j) = 1 + the largest level of its
// k's); the columns of a level are independent and run in one launch. The
// triangular solves run row-wise in one launch each (k_csrmic_lower_sf,
// k_csrmic_upper_sf): warps take chunks of up to 32 rows of one level from an
// atomic counter in level order (reverse order for the transpose solve), and
// a row polls each value it depends on until the warp that owns that row has
// stored it. Each row's subtractions keep the header's order. Every product
// and sum is rounded on its own (no fused multiply-add), as the host code the
// header compiles to computes them.
#include "common.cuh"
#include "kernels.h"
#include "csr_mic0.h"

#include <algorithm>
#include <vector>

namespace shkz {

__global__ void k_csrmic_init(int nnzl, const int *__restrict__ src, int n, const int *__restrict__ dpos,
                              const double *__restrict__ data, double *val, double *invdiag, double *adiag) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nnzl; p += gridDim.x * blockDim.x) val[p] = data[src[p]];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double a = dpos[i] >= 0 ? data[dpos[i]] : 0.0;
    invdiag[i] = a;
    adiag[i] = a;
  }
}

// factor_modified_incomplete_cholesky0 (pcg_solver.h:122-189) for the columns
// of one level: all updates into column j, then its finalisation.
__global__ void k_csrmic_factor(CsrMicDevice M, const int *__restrict__ cols, int count, double omega,
                                double min_ratio) {
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < count; w += gridDim.x * blockDim.x) {
    const int j = cols[w];
    const int jb = M.colstart[j], je = M.colstart[j + 1];
    const int ab = M.a_ptr[j], ae = M.a_ptr[j + 1];
    double inv = M.invdiag[j];
    for (int qq = M.lrow_start[j]; qq < M.lrow_start[j + 1]; ++qq) {
      const int k = M.lrow_col[qq];
      if (M.adiag[k] == 0.0) continue;  // a null column eliminates nothing
      const int kb = M.colstart[k], ke = M.colstart[k + 1];
      const double mult = M.val[M.lrow_pos[qq]];
      double missing = 0.0;
      int a = kb;
      // dropped entries above row j of column j (pcg_solver.h:140-155)
      int b = ab;
      while (a < ke && M.rowindex[a] < j) {
        while (b < ae) {
          const int ib = M.a_idx[b], ra = M.rowindex[a];
          if (ib < ra) ++b;
          else if (ib == ra) break;
          else {
            missing = __dadd_rn(missing, M.val[a]);
            break;
          }
        }
        ++a;
      }
      if (a < ke && M.rowindex[a] == j) inv = __dsub_rn(inv, __dmul_rn(mult, M.val[a]));
      ++a;
      // eliminate into column j's entries below the diagonal (pcg_solver.h:160-176)
      b = jb;
      while (a < ke && b < je) {
        const int rb = M.rowindex[b], ra = M.rowindex[a];
        if (rb < ra) ++b;
        else if (rb == ra) {
          M.val[b] = __dsub_rn(M.val[b], __dmul_rn(mult, M.val[a]));
          ++a;
          ++b;
        } else {
          missing = __dadd_rn(missing, M.val[a]);
          ++a;
        }
      }
      while (a < ke) {
        missing = __dadd_rn(missing, M.val[a]);
        ++a;
      }
      inv = __dsub_rn(inv, __dmul_rn(__dmul_rn(omega, mult), missing));
    }
    // finalise column j (pcg_solver.h:126-135)
    const double ad = M.adiag[j];
    if (ad == 0.0) {
      M.invdiag[j] = inv;
      continue;
    }
    inv = inv < __dmul_rn(min_ratio, ad) ? __ddiv_rn(1.0, __dsqrt_rn(ad)) : __ddiv_rn(1.0, __dsqrt_rn(inv));
    M.invdiag[j] = inv;
    for (int p = jb; p < je; ++p) M.val[p] = __dmul_rn(M.val[p], inv);
  }
}

// Sync-free triangular solves. Output values start as a signalling-NaN
// pattern that no arithmetic produces; a 64-bit store of the final value is
// single-copy atomic, so the value is its own ready flag. A chunk holds rows
// of one level and waits only on rows of earlier chunks, which warps that are
// already running hold, so every wait ends; each is still bounded, and on
// expiry the row stores a quiet NaN (its dependants then finish at once and
// the solve's NaN check stops it) and sets the error word.
constexpr unsigned long long kPending = 0x7ff4000000000001ull;
constexpr int kSolveWarpsPerSm = 8;

__device__ __forceinline__ double poll_value(const double *p, int limit, int *err) {
  unsigned long long w;
  for (int it = 0;; ++it) {
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(w) : "l"(p) : "memory");
    if (w != kPending) return __longlong_as_double((long long)w);
    if (it >= limit) {
      atomicExch(err, 1);
      return __longlong_as_double(0x7ff8000000000000ll);
    }
    __nanosleep(32);
  }
}

__device__ __forceinline__ void store_value(double *p, double v) {
  asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(__double_as_longlong(v)) : "memory");
}

// both solves' outputs to pending, both chunk counters to zero
__global__ void k_csrmic_pending(int n, double *t, double *z, unsigned *counters, const int *done) {
  if (done && *done) return;
  const double pend = __longlong_as_double((long long)kPending);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    t[i] = pend;
    z[i] = pend;
  }
  if (blockIdx.x == 0 && threadIdx.x < 2) counters[threadIdx.x] = 0;
}

__device__ __forceinline__ unsigned long long load_word(const double *p) {
  unsigned long long w;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(w) : "l"(p) : "memory");
  return w;
}

// s - sum_q val[pos(q)] * x[col(q)] over q in [q0, q1), in q order. The first
// kDepBatch values are loaded together and re-polled together until none is
// pending, so a row waits about one L2 round trip once its dependencies are
// stored; any further ones are polled one by one.
constexpr int kDepBatch = 8;
template <class Col, class Pos>
__device__ __forceinline__ double row_update(double s, int q0, int q1, const double *x, const double *val, Col col,
                                             Pos pos, int limit, int *err) {
  unsigned long long w[kDepBatch];
  #pragma unroll
  for (int k = 0; k < kDepBatch; ++k) w[k] = q0 + k < q1 ? load_word(x + col(q0 + k)) : 0ull;
  for (int it = 0;; ++it) {
    bool pending = false;
    #pragma unroll
    for (int k = 0; k < kDepBatch; ++k) pending |= w[k] == kPending;
    if (!pending) break;
    if (it >= limit) {
      atomicExch(err, 1);
      #pragma unroll
      for (int k = 0; k < kDepBatch; ++k)
        if (w[k] == kPending) w[k] = 0x7ff8000000000000ull;
      break;
    }
    __nanosleep(32);
    #pragma unroll
    for (int k = 0; k < kDepBatch; ++k)
      if (w[k] == kPending) w[k] = load_word(x + col(q0 + k));
  }
  #pragma unroll
  for (int k = 0; k < kDepBatch; ++k)
    if (q0 + k < q1) s = __dsub_rn(s, __dmul_rn(val[pos(q0 + k)], __longlong_as_double((long long)w[k])));
  for (int q = q0 + kDepBatch; q < q1; ++q) s = __dsub_rn(s, __dmul_rn(val[pos(q)], poll_value(x + col(q), limit, err)));
  return s;
}

// solve_lower (pcg_solver.h:195-209): y[r] = (b[r] - sum_k L(r,k) y[k]) * invdiag[r]
__global__ void __launch_bounds__(128) k_csrmic_lower_sf(CsrMicDevice M, const int *__restrict__ cols,
                                                         const int *__restrict__ chunks, int nchunks,
                                                         const double *__restrict__ b, double *y, unsigned *counter,
                                                         int *err, int limit, const int *done, int skip) {
  if (done && *done) return;
  const int lane = threadIdx.x & 31;
  while (true) {
    int c = 0;
    if (lane == 0) c = (int)atomicAdd(counter, 1u);
    c = __shfl_sync(0xffffffffu, c, 0);
    if (c >= nchunks) return;
    const int first = chunks[c], count = chunks[c + 1] - first;
    if (lane < count) {
      const int r = cols[first + lane];
      const double s = row_update(
          b[r], M.lrow_start[r], M.lrow_start[r + 1], y, M.val, [&](int q) { return M.lrow_col[q]; },
          [&](int q) { return M.lrow_pos[q]; }, limit, err);
      // fault injection (tests only): the row at level-order position skip
      // never stores, so the waits on it run out
      if (first + lane != skip) store_value(y + r, __dmul_rn(s, M.invdiag[r]));
    }
  }
}

// solve_lower_transpose_in_place (pcg_solver.h:211-223), out of place:
// z[i] = (t[i] - sum L(r,i) z[r]) * invdiag[i], chunks in reverse level order
__global__ void __launch_bounds__(128) k_csrmic_upper_sf(CsrMicDevice M, const int *__restrict__ cols,
                                                         const int *__restrict__ chunks, int nchunks,
                                                         const double *__restrict__ t, double *z, unsigned *counter,
                                                         int *err, int limit, const int *done) {
  if (done && *done) return;
  const int lane = threadIdx.x & 31;
  while (true) {
    int c = 0;
    if (lane == 0) c = (int)atomicAdd(counter, 1u);
    c = __shfl_sync(0xffffffffu, c, 0);
    if (c >= nchunks) return;
    c = nchunks - 1 - c;
    const int first = chunks[c], count = chunks[c + 1] - first;
    if (lane < count) {
      const int i = cols[first + lane];
      const double s = row_update(
          t[i], M.colstart[i], M.colstart[i + 1], z, M.val, [&](int p) { return M.rowindex[p]; },
          [](int p) { return p; }, limit, err);
      store_value(z + i, __dmul_rn(s, M.invdiag[i]));
    }
  }
}

static int level_grid(int count) { return std::min((count + 127) / 128, 148 * 8); }

CsrMic0::~CsrMic0() { release(); }

void CsrMic0::release() {
  void *ptrs[] = {d_colstart, d_rowindex, d_val, d_invdiag, d_adiag, d_lrow_start, d_lrow_col, d_lrow_pos, d_src,
                  d_dpos, d_cols, d_chunks, d_t, d_sync};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  d_colstart = d_rowindex = d_lrow_start = d_lrow_col = d_lrow_pos = d_src = d_dpos = d_cols = d_chunks = d_sync = nullptr;
  d_val = d_invdiag = d_adiag = d_t = nullptr;
  nchunks = 0;
}

int CsrMic0::build(int n_, const int *indptr, const int *indices, const int *d_indptr, const int *d_indices,
                   cudaStream_t s) {
  release();
  n = n_;
  // pattern of L by column (row i right of the diagonal) and of the diagonal
  std::vector<int> colstart(n + 1), rowindex, src, dpos(n, -1);
  for (int i = 0; i < n; ++i) {
    colstart[i] = (int)rowindex.size();
    for (int p = indptr[i]; p < indptr[i + 1]; ++p) {
      if (indices[p] > i) {
        rowindex.push_back(indices[p]);
        src.push_back(p);
      } else if (indices[p] == i) {
        dpos[i] = p;
      }
    }
  }
  colstart[n] = (int)rowindex.size();
  nnzl = colstart[n];
  // L by row: for row j the columns k < j with L(j,k) != 0, increasing k, and
  // where L(j,k) sits in column k
  std::vector<int> lrow_start(n + 1, 0), lrow_col(nnzl), lrow_pos(nnzl);
  for (int p = 0; p < nnzl; ++p) ++lrow_start[rowindex[p] + 1];
  for (int j = 0; j < n; ++j) lrow_start[j + 1] += lrow_start[j];
  {
    std::vector<int> cur(lrow_start.begin(), lrow_start.end() - 1);
    for (int k = 0; k < n; ++k)
      for (int p = colstart[k]; p < colstart[k + 1]; ++p) {
        const int j = rowindex[p];
        lrow_col[cur[j]] = k;
        lrow_pos[cur[j]] = p;
        ++cur[j];
      }
  }
  // levels: a column (row) after every column it depends on
  std::vector<int> level(n, 0);
  int nlev = 0;
  for (int j = 0; j < n; ++j) {
    int l = 0;
    for (int q = lrow_start[j]; q < lrow_start[j + 1]; ++q) l = std::max(l, level[lrow_col[q]] + 1);
    level[j] = l;
    nlev = std::max(nlev, l + 1);
  }
  level_start.assign(nlev + 1, 0);
  for (int j = 0; j < n; ++j) ++level_start[level[j] + 1];
  for (int l = 0; l < nlev; ++l) level_start[l + 1] += level_start[l];
  std::vector<int> cols(n);
  {
    std::vector<int> cur(level_start.begin(), level_start.end() - 1);
    for (int j = 0; j < n; ++j) cols[cur[level[j]]++] = j;
  }
  // chunks of up to 32 rows, never across a level boundary
  std::vector<int> chunks;
  for (int l = 0; l < nlev; ++l)
    for (int q = level_start[l]; q < level_start[l + 1]; q += 32) chunks.push_back(q);
  chunks.push_back(n);
  nchunks = (int)chunks.size() - 1;
  auto upload = [&](int **d, const std::vector<int> &h) -> bool {
    if (cudaMalloc(d, sizeof(int) * std::max<size_t>(1, h.size())) != cudaSuccess) return false;
    return h.empty() || cudaMemcpyAsync(*d, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice, s) == cudaSuccess;
  };
  bool ok = upload(&d_colstart, colstart) && upload(&d_rowindex, rowindex) && upload(&d_lrow_start, lrow_start) &&
            upload(&d_lrow_col, lrow_col) && upload(&d_lrow_pos, lrow_pos) && upload(&d_src, src) &&
            upload(&d_dpos, dpos) && upload(&d_cols, cols) && upload(&d_chunks, chunks) &&
            cudaMalloc(&d_t, sizeof(double) * std::max(1, n)) == cudaSuccess &&
            cudaMalloc(&d_sync, sizeof(int) * 4) == cudaSuccess && cudaMemsetAsync(d_sync, 0, sizeof(int) * 4, s) == cudaSuccess &&
            cudaMalloc(&d_val, sizeof(double) * std::max(1, nnzl)) == cudaSuccess &&
            cudaMalloc(&d_invdiag, sizeof(double) * std::max(1, n)) == cudaSuccess &&
            cudaMalloc(&d_adiag, sizeof(double) * std::max(1, n)) == cudaSuccess;
  // the host vectors must outlive the asynchronous uploads
  if (cudaStreamSynchronize(s) != cudaSuccess) ok = false;
  if (!ok) {
    release();
    return SHKZ_B200_ERR_NOMEM;
  }
  a_ptr = d_indptr;
  a_idx = d_indices;
  return 0;
}

CsrMicDevice CsrMic0::device() const {
  CsrMicDevice M;
  M.n = n;
  M.colstart = d_colstart;
  M.rowindex = d_rowindex;
  M.val = d_val;
  M.invdiag = d_invdiag;
  M.adiag = d_adiag;
  M.lrow_start = d_lrow_start;
  M.lrow_col = d_lrow_col;
  M.lrow_pos = d_lrow_pos;
  M.a_ptr = a_ptr;
  M.a_idx = a_idx;
  return M;
}

int CsrMic0::factor(const double *d_data, double omega, double min_ratio, cudaStream_t s) {
  count_launches(1);
  k_csrmic_init<<<std::min((std::max(nnzl, n) + 255) / 256, 148 * 8) + 1, 256, 0, s>>>(nnzl, d_src, n, d_dpos, d_data,
                                                                                       d_val, d_invdiag, d_adiag);
  const CsrMicDevice M = device();
  const int nlev = (int)level_start.size() - 1;
  for (int l = 0; l < nlev; ++l) {
    const int c = level_start[l + 1] - level_start[l];
    count_launches(1);
    k_csrmic_factor<<<level_grid(c), 128, 0, s>>>(M, d_cols + level_start[l], c, omega, min_ratio);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : SHKZ_B200_ERR_CUDA;
}

int CsrMic0::apply(const double *r, double *z, cudaStream_t s, const int *done) {
  const CsrMicDevice M = device();
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = sms * kSolveWarpsPerSm / 4;
  unsigned *counters = reinterpret_cast<unsigned *>(d_sync);
  int *err = d_sync + 2;
  count_launches(3);
  k_csrmic_pending<<<std::max(1, std::min((n + 255) / 256, 148 * 8)), 256, 0, s>>>(n, d_t, z, counters, done);
  k_csrmic_lower_sf<<<blocks, 128, 0, s>>>(M, d_cols, d_chunks, nchunks, r, d_t, counters, err, wait_limit, done,
                                           skip_pos);
  k_csrmic_upper_sf<<<blocks, 128, 0, s>>>(M, d_cols, d_chunks, nchunks, d_t, z, counters + 1, err, wait_limit,
                                           done);
  return cudaGetLastError() == cudaSuccess ? 0 : SHKZ_B200_ERR_CUDA;
}

int CsrMic0::wait_error(cudaStream_t s) const {
  if (!d_sync) return 0;
  int e = 0;
  if (cudaMemcpyAsync(&e, d_sync + 2, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return SHKZ_B200_ERR_CUDA;
  return e ? SHKZ_B200_ERR_TIMEOUT : 0;
}

}  // namespace shkz
