// stubs.cu -- entry points whose implementation is not built yet.
#include "smoq_internal.h"
extern "C" {
smoq_status smoq_energy_grad(smoq_ctx* ctx, int, smoq_dtype, const smoq_op*, int, int, const smoq_pauli_term*, int,
                             int, const double*, double*, double*) {
    if (ctx) ctx->last_error = "smoq_energy_grad: not implemented";
    return SMOQ_ERR_UNSUPPORTED;
}
smoq_status smoq_energy(smoq_ctx* ctx, int, smoq_dtype, const smoq_op*, int, int, const smoq_pauli_term*, int, int,
                        const double*, double*) {
    if (ctx) ctx->last_error = "smoq_energy: not implemented";
    return SMOQ_ERR_UNSUPPORTED;
}
}
