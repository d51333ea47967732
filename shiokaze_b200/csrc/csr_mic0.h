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
  // z = (L L^T)^-1 r
  int apply(const double *r, double *z, cudaStream_t s);
  int levels() const { return (int)level_start.size() - 1; }

 private:
  void release();
  CsrMicDevice device() const;
  int n = 0, nnzl = 0;
  std::vector<int> level_start;
  int *d_colstart = nullptr, *d_rowindex = nullptr, *d_lrow_start = nullptr, *d_lrow_col = nullptr,
      *d_lrow_pos = nullptr, *d_src = nullptr, *d_dpos = nullptr, *d_cols = nullptr;
  double *d_val = nullptr, *d_invdiag = nullptr, *d_adiag = nullptr;
  const int *a_ptr = nullptr, *a_idx = nullptr;
};

}  // namespace shkz
