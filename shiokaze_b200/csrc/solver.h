// Launch interfaces of the PCG / MIC(0) kernels (solver.cu).
#pragma once
#include "common.cuh"
#include "kernels.h"

namespace shkz {

// Number of tiles holding unknowns (synchronises the stream), then the pool itself.
int pool_count(const Geometry &G, const int *tile_count, int *scratch_bsum, int *d_total, cudaStream_t s);
void pool_assign(const Geometry &G, const int *tile_count, int K, const int *scratch_bsum, int *tile_state,
                 int *pool_tile, int *nbr, int *level_count, int *sched, cudaStream_t s);
size_t wave_sync_bytes();
int spmv_grid(int K);
// q = A p with p = z + beta p_old formed on the fly (beta from st, the pending
// update of the previous iteration): p_old is p0 after an even number of
// completed iterations (st->iter) and p1 after an odd one, the new p goes to
// the other buffer; fused p.q -> alpha as launch_spmv mode 0.
void launch_spmv_update(const PoolSystem &S, float *p0, float *p1, const float *z, float *q, double *partials,
                        unsigned *counter, SolverState *st, cudaStream_t s);
void launch_spmv(const PoolSystem &S, const float *p, float *q, double *partials, unsigned *counter, SolverState *st,
                 int mode, cudaStream_t s);
void launch_update_xr(int n, const float *p, const float *q, float *x, float *r, double *partials, unsigned *counter,
                      SolverState *st, int max_iterations, cudaStream_t s);
void launch_finish_rho(const double *partials, int n, SolverState *st, int init, cudaStream_t s);
void launch_finish_rho_r2(SolverState *st, int init, cudaStream_t s);
void launch_update_p(int n, const float *z, float *p, const SolverState *st, cudaStream_t s);
void launch_mic_factor(const PoolSystem &S, double *colsum, double omega, double min_ratio, double *d64, float *d32,
                       int *flags, void *ws, cudaStream_t s);
void launch_mic_apply(const PoolSystem &S, const float *d32, const float *r, float *t, float *z, double *partials,
                      unsigned long long *faces_f, unsigned long long *faces_b, void *ws_f, void *ws_b,
                      const SolverState *st, cudaStream_t s);
// One PCG iteration's x/r update fused into the MIC(0) application on 16^3
// macro tiles (r -= alpha q, x += alpha p, norms and stopping bookkeeping as
// launch_update_xr, then z = M^-1 r with the z.r partials). False (nothing
// launched) when the macro-tile sweeps are not in use. finish (may be null): a
// zeroed counter; the backward sweep's last CTA then also computes
// rho_new = z.r, beta = rho_new / rho, rho = rho_new (k_finish_rho's update).
bool launch_mic_apply_update(const PoolSystem &S, const float *d32, float *r, float *t, float *z, double *partials,
                             const float *p, const float *p_alt, const float *q, float *x, unsigned *counter,
                             SolverState *st, int max_iterations, void *ws_f, void *ws_b, unsigned *finish,
                             cudaStream_t s);
void launch_residual64(const PoolSystem &S, const double *b, const double *x, double *r, double *partials,
                       unsigned *counter, double *out4, cudaStream_t s);
void launch_inner_init(int n, const double *r64, double inv_scale, float *r32, float *x32, cudaStream_t s);
void launch_accumulate(int n, const float *x32, double scale, double *x64, cudaStream_t s);
void launch_to_float(int n, const double *a, float *b, cudaStream_t s);
void launch_state_resume(SolverState *st, double ru_threshold, cudaStream_t s);
void launch_inner_setup(int n, const float *r, double *partials, unsigned *counter, SolverState *st, double tol,
                        cudaStream_t s);

void launch_apply64(const PoolSystem &S, const double *x, double *y, cudaStream_t s);
void launch_dots64(int n, const double *a, const double *b, const double *c, const double *d, double *partials,
                   unsigned *counter, double *out, cudaStream_t s);
void launch_axpy2_64(int n, double alpha, const double *x, double *y, const double *q, double *r, cudaStream_t s);
void launch_xpby64(int n, const double *x, double beta, double *y, cudaStream_t s);
// The generic CSR solve's PCG loop kept on the device, so that one iteration
// can be a CUDA graph launched many times between host checks. The kernels do
// the arithmetic of k_dots64 / k_axpy2_64 / k_xpby64 with alpha and beta taken
// from CsrState, and return at once when done != 0.
struct CsrState {
  double rho, alpha, beta, tol, rmax;
  int it, done, status, max_it;  // done: 1 converged, 2 iteration limit, 3 NaN
};
// phase 0: alpha = rho / a.b; phase 1 (a = r, c = z, d = r): stop test on
// max|r|, then rho, beta and the iteration count
void launch_csr_dots(int n, const double *a, const double *b, const double *c, const double *d, double *partials,
                     unsigned *counter, CsrState *st, int phase, cudaStream_t s);
void launch_csr_axpy2(int n, const CsrState *st, const double *x, double *y, const double *q, double *r,
                      cudaStream_t s);
void launch_csr_xpby(int n, const double *x, const CsrState *st, double *y, cudaStream_t s);
void launch_scale_f64_f32(int n, const double *a, double sc, float *b, cudaStream_t s);
void launch_scale_f32_f64(int n, const float *a, double sc, double *b, cudaStream_t s);

// partial sums written by one MIC(0) apply (one per CTA of the backward sweep)
inline int mic_partial_count(const PoolSystem &S) { return S.KM > 0 ? S.KM : S.K; }
void launch_macro_count(const Geometry &G, const int *tile_count, const Geometry &M, int *macro_count, cudaStream_t s);
void build_macro(const Geometry &G, const Geometry &M, const int *tile_count, const int *tile_state, int *macro_count,
                 int *macro_state, int *macro_tile, int *mnbr, int *level_count, int *msched, int *msub, int KM,
                 const int *bsum, cudaStream_t s);
void launch_fpcg_dots(int n, const float *z, const float *r, const float *q, double *partials, unsigned *counter,
                      SolverState *st, int init, cudaStream_t s);
// upx/upy/upz of every pool cell from the lower weights and the tile neighbours
void launch_upper_weights(const PoolSystem &S, float *upx, float *upy, float *upz, cudaStream_t s);
void launch_rand_unknowns(int n, const float *diag, unsigned seed, float *e, cudaStream_t s);
void launch_scale_f32(int n, float *a, float sc, cudaStream_t s);
void launch_axpby_f32(int n, float a, const float *x, float b, float *y, cudaStream_t s);

}  // namespace shkz
