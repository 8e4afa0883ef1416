// apply.cuh -- the apply_full_L pipeline, the bi-conjugate step and the continued fraction
// (apply.cu), shared by the C ABI (capi.cu) and the multi-step run (run.cu).
#pragma once

#include <cuda_runtime.h>

#include "ensemble.cuh"

namespace tdscha {

int apply_full_L_device(tdscha_ensemble *e, int nb, const double *psi, const int *transpose_h, const tdscha_apply_opts *opts,
                        int precision, double *out, cudaStream_t st, void *scratch, size_t scratch_bytes);
int apply_full_L_device_flags(tdscha_ensemble *e, int nb, const double *psi, const int *tr_d, const tdscha_apply_opts *opts,
                              int precision, double *out, cudaStream_t st, double *work, size_t work_bytes);
size_t apply_scratch_bytes(const tdscha_ensemble *e, int nb);
int apply_prologue_device(tdscha_ensemble *e, int nb, const double *psi, const int *tr_d, const tdscha_apply_opts *opts,
                          double *R, double *Ys, cudaStream_t st);
int apply_epilogue_device(tdscha_ensemble *e, int nb, const double *psi, const int *tr_d, const tdscha_apply_opts *opts,
                          const double *fav, const double *dav, double *out, cudaStream_t st);
int lanczos_step_device(int nc, long long len, const double *Lq, const double *pL, const double *q, const double *p,
                        const double *q_prev, const double *p_prev, const double *sc_in, const double *mask, double *q_next,
                        double *p_next, double *sc_out, cudaStream_t st, double *scratch, size_t scratch_bytes);
size_t lanczos_scratch_bytes(int nc);
int apply_L1_static_device(tdscha_ensemble *e, int nb, const double *psi, double power, double *out, cudaStream_t st);
int apply_static_L_device(tdscha_ensemble *e, int nb, const double *psi, int ignore_v4, int include_L1, int precision,
                          double *out, cudaStream_t st, double *work, size_t work_bytes);
size_t static_work_bytes(const tdscha_ensemble *e, int nb);
int lanczos_run_device(int ns, const tdscha_run_system *sys, int n_steps, int use_graph, cudaStream_t st);
int continued_fraction_device(int n_iter, const double *a, const double *b, const double *c, int n_b, int n_c, int n_w,
                              const double *omega, int use_terminator, int last_average, double smearing, int use_wigner,
                              int reverse_L, double shift_value, double modulus, double *gf_out, cudaStream_t st);

}  // namespace tdscha
