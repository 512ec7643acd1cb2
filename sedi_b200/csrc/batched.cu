// Batched (RHS-interleaved) forms -- placeholder until the batched kernels land.
#include "sedi_internal.h"

namespace sedi {
int batched_alloc(Ctx *c) { c->error = "batched form not built"; return SEDI_ERR_UNSUPPORTED; }
void batched_free(Ctx *) {}
int batched_solve_dev(Ctx *, int, const double *, double *, int, double, double *, int *, int *) { return SEDI_ERR_UNSUPPORTED; }
int batched_estimate_dev(Ctx *, int, const double *, int, double, int, double *, double *, double *, int *, double *, int *) { return SEDI_ERR_UNSUPPORTED; }
}  // namespace sedi
