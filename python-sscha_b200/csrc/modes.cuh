// modes.cuh -- the Lanczos inputs built on the GPU (modes.cu).
#pragma once

namespace tdscha {

// X = (u o sqrt(m)) . pols, Y = (f / sqrt(m)) . pols; u, f (N, 3 nat), pols (3 nat, n); host buffers.
int project_ensemble(const double *u, const double *f, const double *masses, const double *pols, int N, int nat3, int n,
                     double *X_out, double *Y_out);

// Per degenerate block b: (N_sym, d_b, d_b) tables S_b^j = E_b^T P_j E_b; host buffers.
int symmetries_on_modes(const double *pols, int nat, int n, int N_sym, const int *perm, const double *rot, int n_blocks,
                        const int *n_deg, const int *const *deg_space, double *const *sym_out);

}  // namespace tdscha
