// MIC(0) on a generic CSR matrix (csr_mic0.cu).
#pragma once
#include "common.cuh"
#include "../../include/shkz_b200.h"

#include <vector>

namespace shkz {

struct CsrMicDevice {
  int n;
  const int *colstart, *rowindex;                 // L by column: rows right of the diagonal
  double *val, *invdiag, *adiag;
  const int *lrow_start, *lrow_col, *lrow_pos;    // L by row: columns k < j and positions in column k
  const int *a_ptr, *a_idx;                       // A's pattern (CSR)
};

class CsrMic0 {
 public:
  ~CsrMic0();
  // Pattern analysis on the host (row-sorted, symmetric pattern, 0-based);
  // d_indptr/d_indices: the same pattern on the device (kept by the caller).
  int build(int n, const int *indptr, const int *indices, const int *d_indptr, const int *d_indices,
            cudaStream_t s);
  // Factor the values of A (device, CSR order) with the header's parameters.
  int factor(const double *d_data, double omega, double min_ratio, cudaStream_t s);
  // z = (L L^T)^-1 r (z must not alias r); every launch returns at once
  // while *done != 0
  int apply(const double *r, double *z, cudaStream_t s, const int *done = nullptr);
  // SHKZ_B200_ERR_TIMEOUT when a triangular solve's wait ran out (since build)
  int wait_error(cudaStream_t s) const;
  // polling rounds of each wait in the triangular solves
  void set_wait_limit(int limit) { wait_limit = limit; }
  // fault injection for tests: the forward solve's row at level-order
  // position pos (-1: none) never stores its value
  void set_fault_skip(int pos) { skip_pos = pos; }
  int levels() const { return (int)level_start.size() - 1; }

 private:
  void release();
  CsrMicDevice device() const;
  int n = 0, nnzl = 0, nchunks = 0, wait_limit = 1 << 22, skip_pos = -1;
  std::vector<int> level_start;
  int *d_colstart = nullptr, *d_rowindex = nullptr, *d_lrow_start = nullptr, *d_lrow_col = nullptr,
      *d_lrow_pos = nullptr, *d_src = nullptr, *d_dpos = nullptr, *d_cols = nullptr, *d_chunks = nullptr;
  int *d_sync = nullptr;  // two chunk counters, the wait error word
  double *d_val = nullptr, *d_invdiag = nullptr, *d_adiag = nullptr, *d_t = nullptr;
  const int *a_ptr = nullptr, *a_idx = nullptr;
};

}  // namespace shkz
