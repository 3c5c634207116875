// stubs.cu -- entry points not yet implemented (return KET_ERR_UNSUPPORTED).
#include "ctx.h"

using namespace ket;

extern "C" {

int ket_adjoint_gradient(ket_ctx*, int, uint64_t, const ket_op*, size_t, const double*, size_t,
                         const ket_param_binding*, size_t, const double*, int, int, int, const double*, const char*, int,
                         double*, double*) {
  return fail(KET_ERR_UNSUPPORTED, "adjoint gradient not built");
}

int ket_batch_qaoa(ket_ctx*, int, const int*, const int*, const int64_t*, const int*, int, const double*,
                   const double*, int, double*) {
  return fail(KET_ERR_UNSUPPORTED, "batch qaoa not built");
}

}
