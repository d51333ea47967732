// Learned preconditioner: placeholder translation unit, filled in with the
// conv encoder-decoder kernels.
#include "learned.h"

namespace shkz {
struct LearnedModel {
  int dummy;
};
void learned_free(LearnedModel *m) { delete m; }
int learned_solve(LearnedModel *, shkz_b200_ctx *, shkz_b200_result *) { return SHKZ_B200_ERR_STATE; }
}  // namespace shkz
