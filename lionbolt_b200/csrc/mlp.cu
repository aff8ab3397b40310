// Learned right preconditioner for FGMRES (per-cell MLP).  Hooks used by the Krylov driver.
#include "lb_internal.h"

namespace lb {

bool mlp_ready(Handle* h) { return h->mlp != nullptr; }

int mlp_apply_precond(Handle* h, const double* v, double* z) {
    (void)v; (void)z;
    return fail(h, LB_ERR_STATE, "learned preconditioner not loaded");
}

void mlp_destroy(Handle* h) { h->mlp = nullptr; }

}  // namespace lb
