// Learned preconditioner (conv encoder-decoder) used inside flexible PCG.
#pragma once
#include "common.cuh"
#include "../../include/shkz_b200.h"

struct shkz_b200_ctx;

namespace shkz {
struct LearnedModel;
void learned_free(LearnedModel *m);
int learned_solve(LearnedModel *m, shkz_b200_ctx *ctx, shkz_b200_result *res);
}  // namespace shkz
