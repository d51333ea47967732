// Learned preconditioner (conv encoder-decoder) used inside flexible PCG.
#pragma once
#include "common.cuh"
#include "kernels.h"
#include <cuda_bf16.h>
#include "../../include/shkz_b200.h"

namespace shkz {
struct LearnedModel;

// The solver system the network runs on (device pointers of the context).
struct LearnedSystem {
  Geometry G;
  const int *tile_state, *pool_tile;
  int K;
  const uint8_t *unk;
  const float *fluid, *solid;  // dense effective level sets of the last projection (solid may be null)
  double dx;
};

LearnedModel *learned_create(int device);
void learned_free(LearnedModel *m);
size_t learned_param_count(const LearnedModel *m);
int learned_set_params(LearnedModel *m, const float *blob, size_t n, cudaStream_t s);
int learned_get_params(LearnedModel *m, float *blob, size_t n, int grads, cudaStream_t s);
int learned_init_params(LearnedModel *m, unsigned seed, cudaStream_t s);
int learned_prepare(LearnedModel *m, const Geometry &G, const int *tile_state, cudaStream_t s);
// z_pool = rmax * N(r_pool / rmax) at unknown cells
double learned_forward_flops(const LearnedModel *m);
int learned_apply(LearnedModel *m, const LearnedSystem &sys, const float *r_pool, double rmax, float *z_pool,
                  cudaStream_t s);
int learned_backward_dense(LearnedModel *m, const float *gZ_dense, cudaStream_t s);
int learned_output_dense(LearnedModel *m, float *Z_dense_dev, cudaStream_t s);
size_t learned_dense_cells(const LearnedModel *m);
void learned_dense_dims(const LearnedModel *m, int *nx, int *ny, int *nz);
int learned_train_step(LearnedModel *m, const LearnedSystem &sys, const PoolSystem &S, const float *r_pool,
                       float *z_pool, float *Az_pool, double *partials, unsigned *counter, float lr, double gscale,
                       double *loss, cudaStream_t s);
int learned_error(LearnedModel *m);
size_t learned_tensor_size(const LearnedModel *m, int t);
void learned_tensor_shape(const LearnedModel *m, int t, int *shape4);
int learned_tensor_dense(LearnedModel *m, int t, float *out, cudaStream_t s);
int learned_grad_dense(LearnedModel *m, int t, float *out, cudaStream_t s);
int conv3d_launch_scratch(int nx, int ny, int nz, int c0, int c1, int cout, int planes, const __nv_bfloat16 *in0,
                          const __nv_bfloat16 *in1, const float *w, const float *bias, int relu, __nv_bfloat16 *out,
                          __nv_bfloat16 *wpk, uint8_t *act, int *err, cudaStream_t s);
int conv3d_run(int nx, int ny, int nz, int c0, int c1, int cout, int planes, const float *in0_h, const float *in1_h,
               const float *w_h, const float *bias_h, int relu, float *out_h);
}  // namespace shkz
