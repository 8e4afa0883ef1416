// capi.cu -- extern "C" entry points declared in include/tdscha_b200.h.
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

#include "apply.cuh"
#include "common.cuh"
#include "ensemble.cuh"
#include "freq.cuh"
#include "modes.cuh"
#include "tc_gemm.cuh"

namespace tdscha {

static thread_local char g_err[1024] = "";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}
void clear_error() { g_err[0] = 0; }

// Temporaries of the allocating entry points: library-owned buffers, grown on demand, one per
// (slot, device, stream) and host thread.  Calls from one thread on one stream reuse a buffer in
// stream order; calls on different streams or from different threads never share one.
struct Scratch {
    void *p = nullptr;
    size_t bytes = 0;
};
static thread_local std::map<std::tuple<int, int, cudaStream_t>, Scratch> g_scratch;

static int scratch_get(int slot, size_t bytes, cudaStream_t st, void **out) {
    int dev = 0;
    TD_CUDA(cudaGetDevice(&dev));
    Scratch &s = g_scratch[std::make_tuple(slot, dev, st)];
    if (s.p && s.bytes < bytes) {
        TD_CUDA(cudaStreamSynchronize(st));   // the old buffer may still be read by this stream's work
        cudaFree(s.p);
        s = Scratch();
    }
    if (!s.p) {
        TD_CUDA(cudaMalloc(&s.p, bytes));
        s.bytes = bytes;
    }
    *out = s.p;
    return 0;
}

// Per-call reading of the error word (tdscha_set_error_check); off: tdscha_check_errors reads it.
static std::atomic<int> g_check_per_call{1};

static int read_err_word(tdscha_ensemble *e, cudaStream_t st) {
    unsigned h = 0;
    TD_CUDA(cudaMemcpyAsync(&h, e->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    TD_CUDA(cudaStreamSynchronize(st));
    if (h) {
        cudaMemsetAsync(e->d_err, 0, sizeof(unsigned), st);
        set_error("a tensor-core kernel hit its bounded-wait limit and aborted (error word 0x%x)", h);
        return TDSCHA_ETIMEOUT;
    }
    return 0;
}

static int check_err_word(tdscha_ensemble *e, cudaStream_t st) {
    return g_check_per_call.load() ? read_err_word(e, st) : 0;
}

}  // namespace tdscha

using namespace tdscha;

extern "C" {

const char *tdscha_last_error(void) { return g_err; }

const char *tdscha_version(void) { return "tdscha_b200 0.1.0 (sm_100a)"; }

int tdscha_ensemble_create(const double *X, const double *Y, const double *w, const double *rho, int N, int n, double T,
                           int N_sym, int n_blocks, const int *n_deg, const int *const *deg_space,
                           const double *const *sym_blocks, const int *blocks_ids, tdscha_ensemble **out) {
    clear_error();
    return ensemble_create(X, Y, w, rho, N, n, T, N_sym, n_blocks, n_deg, deg_space, sym_blocks, blocks_ids, out);
}

int tdscha_ensemble_destroy(tdscha_ensemble *ens) { return ensemble_destroy(ens); }

int tdscha_ensemble_info(const tdscha_ensemble *e, int *n, int *N, int *N_sym, int *n_blocks, double *T, double *N_eff) {
    TD_CHECK(e != nullptr, TDSCHA_EINVAL, "NULL ensemble");
    if (n) *n = e->n;
    if (N) *N = e->N;
    if (N_sym) *N_sym = e->N_sym;
    if (n_blocks) *n_blocks = e->n_blocks;
    if (T) *T = e->T;
    if (N_eff) *N_eff = e->N_eff;
    return 0;
}

int tdscha_ensemble_cosets(const tdscha_ensemble *e, int *rotated, int *n_cosets, int *coset_size, double *offpattern) {
    TD_CHECK(e != nullptr, TDSCHA_EINVAL, "NULL ensemble");
    if (rotated) *rotated = e->Rrow != nullptr;
    if (n_cosets) *n_cosets = e->cosets ? e->cosets->n_cos : 0;
    if (coset_size) *coset_size = e->cosets ? e->cosets->sub : 0;
    if (offpattern) *offpattern = e->cosets ? e->cosets->offpattern : 0.0;
    return 0;
}

int tdscha_ensemble_classes(const tdscha_ensemble *e, int *n_class, int *Kq, int *Kmq, double *flops_ratio) {
    TD_CHECK(e != nullptr, TDSCHA_EINVAL, "NULL ensemble");
    const FreqTables *f = e->freq;
    if (n_class) *n_class = f ? f->n_class : 0;
    if (Kq) *Kq = f ? f->Kq : 0;
    if (Kmq) *Kmq = f ? f->Kmq : 0;
    if (flops_ratio) *flops_ratio = f ? f->flops_ratio : 1.0;
    return 0;
}

int tdscha_symmetry_classes(int N_sym, int n_blocks, const int *n_deg, const double *const *sym_blocks, int *sizes,
                            double *flops_ratio, int *cls, int *pcol_i, double *pcol_d, int *pp_i, double *pp_d, int *mcol_i,
                            double *mcol_d, int *mode_col) {
    clear_error();
    TD_CHECK(N_sym > 0 && n_blocks > 0 && n_deg && sym_blocks && sizes, TDSCHA_EINVAL, "bad arguments");
    std::vector<int> dim(n_deg, n_deg + n_blocks), start(n_blocks);
    int n = 0;
    for (int b = 0; b < n_blocks; ++b) {
        TD_CHECK(dim[b] > 0 && sym_blocks[b], TDSCHA_EINVAL, "block %d empty", b);
        start[b] = n;
        n += dim[b];
    }
    const long long P = (long long)n * (n + 1) / 2;
    sizes[0] = sizes[1] = sizes[2] = 0;
    sizes[3] = (int)P;
    CosetAnalysis ca;
    TD_TRY(analyse_cosets(N_sym, dim, sym_blocks, ca));
    if (!ca.ok) {
        set_error("%s", ca.why.c_str());
        return 0;
    }
    FreqLayout L;
    TD_TRY(build_freq_layout(n, dim, start, sym_blocks, ca, L));
    if (!L.ok) return 0;
    sizes[0] = L.n_class;
    sizes[1] = L.Kq;
    sizes[2] = L.Kmq;
    if (flops_ratio) *flops_ratio = L.flops_ratio;
    if (!cls) return 0;
    for (int g = 0; g < L.n_class; ++g) {
        const int v[5] = {L.cls_real[g], L.pcol_off[g], L.pcol_cnt[g], L.mcol_off[g], L.mcol_cnt[g]};
        std::memcpy(cls + 5 * g, v, sizeof(v));
    }
    for (int c = 0; c < L.Kq; ++c) {
        if (pcol_i) {
            const int v[5] = {L.pc_mu0[c], L.pc_nu0[c], L.pc_mu1[c], L.pc_nu1[c], L.pc_partner[c]};
            std::memcpy(pcol_i + 5 * c, v, sizeof(v));
        }
        if (pcol_d) {
            const double v[5] = {L.pc_c0[c], L.pc_c1[c], L.pc_re[c], L.pc_im[c], L.pc_zc[c]};
            std::memcpy(pcol_d + 5 * c, v, sizeof(v));
        }
    }
    for (long long p = 0; p < P; ++p) {
        if (pp_i) { pp_i[2 * p] = L.pp_col0[p]; pp_i[2 * p + 1] = L.pp_col1[p]; }
        if (pp_d) { pp_d[2 * p] = L.pp_c0[p]; pp_d[2 * p + 1] = L.pp_c1[p]; }
    }
    for (int c = 0; c < L.Kmq; ++c) {
        if (mcol_i) { mcol_i[2 * c] = L.mc_mode[c]; mcol_i[2 * c + 1] = L.mc_partner[c]; }
        if (mcol_d) {
            const double v[4] = {L.mc_sign[c], L.mc_re[c], L.mc_im[c], L.mc_zc[c]};
            std::memcpy(mcol_d + 4 * c, v, sizeof(v));
        }
    }
    if (mode_col) std::memcpy(mode_col, L.mode_col.data(), n * sizeof(int));
    return 0;
}

int tdscha_symmetry_cosets(int N_sym, int n_blocks, const int *n_deg, const double *const *sym_blocks, int *n_cosets,
                           int *coset_size, int *order, int *partner, double *R, double *offpattern) {
    clear_error();
    TD_CHECK(N_sym > 0 && n_blocks > 0 && n_deg && sym_blocks && n_cosets && coset_size, TDSCHA_EINVAL, "bad arguments");
    std::vector<int> dim(n_deg, n_deg + n_blocks);
    for (int b = 0; b < n_blocks; ++b) TD_CHECK(dim[b] > 0 && sym_blocks[b], TDSCHA_EINVAL, "block %d empty", b);
    CosetAnalysis ca;
    TD_TRY(analyse_cosets(N_sym, dim, sym_blocks, ca));
    *n_cosets = ca.ok ? ca.n_cos : 0;
    *coset_size = ca.ok ? ca.sub : 0;
    if (!ca.ok) {
        set_error("%s", ca.why.c_str());
        return 0;
    }
    if (order) std::memcpy(order, ca.order.data(), ca.order.size() * sizeof(int));
    if (partner) std::memcpy(partner, ca.partner.data(), ca.partner.size() * sizeof(int));
    if (R) std::memcpy(R, ca.R.data(), ca.R.size() * sizeof(double));
    if (offpattern) *offpattern = ca.offpattern;
    return 0;
}

int tdscha_ensemble_device_bytes(const tdscha_ensemble *e, long long *bytes) {
    TD_CHECK(e != nullptr && bytes != nullptr, TDSCHA_EINVAL, "NULL argument");
    size_t b = e->base_bytes + e->ws.bytes;
    for (const auto &o : e->ops) b += o.bytes;
    for (const auto &o : e->fops) b += o.bytes;
    for (const auto &o : e->fhalf) b += o.bytes;
    b += e->chunk_ops.bytes;
    *bytes = (long long)b;
    return 0;
}

int tdscha_perturb_average_sym_device(tdscha_ensemble *e, int nb, const double *R1, const double *Y1, int apply_d4,
                                      int precision, double *f_out, double *d2v_out, void *stream) {
    clear_error();
    TD_CHECK(e && R1 && Y1 && f_out && d2v_out, TDSCHA_EINVAL, "NULL argument");
    TD_CHECK(nb > 0, TDSCHA_EINVAL, "nb must be positive");
    TD_CUDA(cudaSetDevice(e->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    void *ys = nullptr;
    TD_TRY(scratch_get(0, (size_t)nb * e->n * e->n * sizeof(double), st, &ys));
    TD_TRY(symmetrize_device(nb, e->n, Y1, static_cast<double *>(ys), st));
    TD_TRY(perturb_average_device(e, nb, R1, static_cast<const double *>(ys), apply_d4, precision, f_out, d2v_out, st));
    return check_err_word(e, st);
}

int tdscha_perturb_average_sym(tdscha_ensemble *e, const double *R1, const double *Y1, int apply_d4, int precision,
                               double *f_out, double *d2v_out) {
    clear_error();
    TD_CHECK(e && R1 && Y1 && f_out && d2v_out, TDSCHA_EINVAL, "NULL argument");
    TD_CUDA(cudaSetDevice(e->device));
    const size_t n = e->n;
    void *buf = nullptr;
    TD_TRY(scratch_get(1, (2 * n + 2 * n * n) * sizeof(double), nullptr, &buf));
    double *dR = static_cast<double *>(buf), *dY = dR + n, *df = dY + n * n, *dD = df + n;
    TD_CUDA(cudaMemcpy(dR, R1, n * sizeof(double), cudaMemcpyHostToDevice));
    TD_CUDA(cudaMemcpy(dY, Y1, n * n * sizeof(double), cudaMemcpyHostToDevice));
    TD_TRY(tdscha_perturb_average_sym_device(e, 1, dR, dY, apply_d4, precision, df, dD, nullptr));
    TD_CUDA(cudaMemcpy(f_out, df, n * sizeof(double), cudaMemcpyDeviceToHost));
    TD_CUDA(cudaMemcpy(d2v_out, dD, n * n * sizeof(double), cudaMemcpyDeviceToHost));
    return 0;
}

int tdscha_GetPerturbAverageSym(const double *X, const double *Y, const double *w, const double *rho, const double *R1,
                                const double *Y1, double T, int apply_D4, int N_syms, int n_blocks,
                                const double *const *sym_list, const int *n_deg, const int *const *deg_space_list,
                                const int *blocks_ids, int N_configs, int N_modes, double *f_out, double *d2v_out) {
    clear_error();
    TD_CHECK(apply_D4 == 0 || apply_D4 == 1, TDSCHA_EINVAL, "the apply_D4 value passed must be either 0 or 1 (got %d)", apply_D4);
    tdscha_ensemble *e = nullptr;
    TD_TRY(ensemble_create(X, Y, w, rho, N_configs, N_modes, T, N_syms, n_blocks, n_deg, deg_space_list, sym_list, blocks_ids, &e));
    int rc = tdscha_perturb_average_sym(e, R1, Y1, apply_D4, TDSCHA_PREC_FP64, f_out, d2v_out);
    ensemble_destroy(e);
    return rc;
}

int tdscha_apply_full_L_device(tdscha_ensemble *e, int nb, const double *psi, const int *transpose,
                               const tdscha_apply_opts *opts, int precision, double *out, void *stream) {
    clear_error();
    TD_CHECK(e != nullptr, TDSCHA_EINVAL, "NULL ensemble");
    TD_CUDA(cudaSetDevice(e->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t need = apply_scratch_bytes(e, nb);
    void *buf = nullptr;
    TD_TRY(scratch_get(0, need, st, &buf));
    TD_TRY(apply_full_L_device(e, nb, psi, transpose, opts, precision, out, st, buf, need));
    return check_err_word(e, st);
}

static int upload_flags(int nb, const int *transpose, cudaStream_t st, int **tr_d) {
    TD_CHECK(transpose && nb > 0 && nb <= 4096, TDSCHA_EINVAL, "bad transpose flags");
    void *buf = nullptr;
    TD_TRY(scratch_get(2, 4096 * sizeof(int), st, &buf));
    TD_CUDA(cudaMemcpyAsync(buf, transpose, nb * sizeof(int), cudaMemcpyHostToDevice, st));
    *tr_d = static_cast<int *>(buf);
    return 0;
}

int tdscha_apply_prologue_device(tdscha_ensemble *e, int nb, const double *psi, const int *transpose,
                                 const tdscha_apply_opts *opts, double *R1_out, double *Y1_out, void *stream) {
    clear_error();
    TD_CHECK(e != nullptr, TDSCHA_EINVAL, "NULL ensemble");
    TD_CUDA(cudaSetDevice(e->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int *tr_d = nullptr;
    TD_TRY(upload_flags(nb, transpose, st, &tr_d));
    return apply_prologue_device(e, nb, psi, tr_d, opts, R1_out, Y1_out, st);
}

int tdscha_apply_epilogue_device(tdscha_ensemble *e, int nb, const double *psi, const int *transpose,
                                 const tdscha_apply_opts *opts, const double *f_av, const double *d2v_av, double *out,
                                 void *stream) {
    clear_error();
    TD_CHECK(e != nullptr, TDSCHA_EINVAL, "NULL ensemble");
    TD_CUDA(cudaSetDevice(e->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int *tr_d = nullptr;
    TD_TRY(upload_flags(nb, transpose, st, &tr_d));
    return apply_epilogue_device(e, nb, psi, tr_d, opts, f_av, d2v_av, out, st);
}

int tdscha_apply_L1_static_device(tdscha_ensemble *e, int nb, const double *psi, double power, double *out, void *stream) {
    clear_error();
    TD_CHECK(e != nullptr, TDSCHA_EINVAL, "NULL ensemble");
    TD_CUDA(cudaSetDevice(e->device));
    return apply_L1_static_device(e, nb, psi, power, out, static_cast<cudaStream_t>(stream));
}

int tdscha_apply_static_L_device(tdscha_ensemble *e, int nb, const double *psi, int ignore_v4, int include_L1, int precision,
                                 double *out, void *stream) {
    clear_error();
    TD_CHECK(e != nullptr, TDSCHA_EINVAL, "NULL ensemble");
    TD_CHECK(nb > 0 && nb <= 64, TDSCHA_EINVAL, "1..64 vectors per static apply (got %d)", nb);
    TD_CUDA(cudaSetDevice(e->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t need = static_work_bytes(e, nb);
    void *buf = nullptr;
    TD_TRY(scratch_get(0, need, st, &buf));
    TD_TRY(apply_static_L_device(e, nb, psi, ignore_v4, include_L1, precision, out, st, static_cast<double *>(buf), need));
    return check_err_word(e, st);
}

int tdscha_lanczos_run_device(int n_systems, const tdscha_run_system *systems, int n_steps, int use_graph, void *stream) {
    clear_error();
    return lanczos_run_device(n_systems, systems, n_steps, use_graph, static_cast<cudaStream_t>(stream));
}

int tdscha_lanczos_step_device(int nc, long long len, const double *Lq, const double *pL, const double *q, const double *p,
                               const double *q_prev, const double *p_prev, const double *sc_in, const double *mask,
                               double *q_next, double *p_next, double *sc_out, void *stream) {
    clear_error();
    const size_t need = lanczos_scratch_bytes(nc);
    void *buf = nullptr;
    TD_TRY(scratch_get(3, need, static_cast<cudaStream_t>(stream), &buf));
    return lanczos_step_device(nc, len, Lq, pL, q, p, q_prev, p_prev, sc_in, mask, q_next, p_next, sc_out,
                               static_cast<cudaStream_t>(stream), static_cast<double *>(buf), need);
}

int tdscha_continued_fraction_device(int n_iter, const double *a, const double *b, const double *c, int n_b, int n_c, int n_w,
                                     const double *omega, int use_terminator, int last_average, double smearing,
                                     int use_wigner, int reverse_L, double shift_value, double perturbation_modulus,
                                     double *gf_out, void *stream) {
    clear_error();
    return continued_fraction_device(n_iter, a, b, c, n_b, n_c, n_w, omega, use_terminator, last_average, smearing, use_wigner,
                                     reverse_L, shift_value, perturbation_modulus, gf_out, static_cast<cudaStream_t>(stream));
}

int tdscha_set_profiling(tdscha_ensemble *e, int enable) {
    TD_CHECK(e != nullptr, TDSCHA_EINVAL, "NULL ensemble");
    e->prof.enabled = enable != 0;
    return 0;
}

int tdscha_read_profile(tdscha_ensemble *e, double *ms, long long *launches, int n_stages) {
    TD_CHECK(e != nullptr && n_stages > 0, TDSCHA_EINVAL, "bad arguments");
    TD_CUDA(cudaSetDevice(e->device));
    for (int s = 0; s < n_stages && s < ST_COUNT; ++s) {
        if (ms) ms[s] = 0.0;
        if (launches) launches[s] = e->prof.launches[s];
    }
    for (auto &r : e->prof.recs) {
        float t = 0.f;
        TD_CUDA(cudaEventSynchronize(r.b));
        TD_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
        if (ms && r.stage < n_stages) ms[r.stage] += t;
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    e->prof.recs.clear();
    for (int s = 0; s < ST_COUNT; ++s) e->prof.launches[s] = 0;
    return 0;
}

int tdscha_set_wait_budget(double seconds) {
    clear_error();
    TD_CHECK(seconds >= 1e-6 && seconds <= 60.0, TDSCHA_EINVAL, "wait budget must lie in [1e-6, 60] s (got %g)", seconds);
    tc::set_wait_budget_ns((unsigned long long)(seconds * 1e9));
    return 0;
}

int tdscha_debug_stall_next_contraction(void) {
    clear_error();
    tc::stall_next_launch();
    return 0;
}

int tdscha_set_error_check(int per_call) {
    clear_error();
    g_check_per_call.store(per_call ? 1 : 0);
    return 0;
}

int tdscha_check_errors(tdscha_ensemble *e, void *stream) {
    clear_error();
    TD_CHECK(e != nullptr, TDSCHA_EINVAL, "NULL ensemble");
    TD_CUDA(cudaSetDevice(e->device));
    return read_err_word(e, static_cast<cudaStream_t>(stream));
}

int tdscha_tc_contract(int precision, int M, int N, int K, const void *A_hi, const void *A_lo, long long lda,
                       const void *B_hi, const void *B_lo, long long ldb, float *D, long long ldd, void *stream) {
    clear_error();
    TD_CHECK(precision != TDSCHA_PREC_FP64 && precision >= 0 && precision <= TDSCHA_PREC_BF16, TDSCHA_EINVAL,
             "tdscha_tc_contract: precision %d is not a tensor-core mode", precision);
    static thread_local unsigned *err = nullptr;
    if (!err) TD_CUDA(cudaMalloc(&err, sizeof(unsigned)));
    TD_CUDA(cudaMemsetAsync(err, 0, sizeof(unsigned), static_cast<cudaStream_t>(stream)));
    tc::GemmOperands op{format_of(precision), products_of(precision), A_hi, A_lo, lda, B_hi, B_lo, ldb};
    TD_TRY(tc::gemm(op, M, N, K, D, ldd, static_cast<cudaStream_t>(stream), err));
    unsigned h = 0;
    TD_CUDA(cudaMemcpyAsync(&h, err, sizeof(unsigned), cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(stream)));
    TD_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    TD_CHECK(h == 0, TDSCHA_ETIMEOUT, "tensor-core contraction hit its bounded-wait limit (error word 0x%x)", h);
    return 0;
}

}  // extern "C"

extern "C" int tdscha_project_ensemble(const double *u, const double *f, const double *masses, const double *pols, int N,
                                       int nat3, int n, double *X_out, double *Y_out) {
    clear_error();
    return tdscha::project_ensemble(u, f, masses, pols, N, nat3, n, X_out, Y_out);
}

extern "C" int tdscha_symmetries_on_modes(const double *pols, int nat, int n, int N_sym, const int *perm, const double *rot,
                                          int n_blocks, const int *n_deg, const int *const *deg_space,
                                          double *const *sym_out) {
    clear_error();
    return tdscha::symmetries_on_modes(pols, nat, n, N_sym, perm, rot, n_blocks, n_deg, deg_space, sym_out);
}

extern "C" int tdscha_perturb_average_vjp_precision_device(tdscha_ensemble *e, int nb, const double *R1, const double *Ys,
                                                           int apply_d4, int precision, const double *fbar,
                                                           const double *Dbar, double *Ybar, double *rhobar, void *stream) {
    clear_error();
    TD_CHECK(e != nullptr, TDSCHA_EINVAL, "NULL ensemble");
    TD_CUDA(cudaSetDevice(e->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    TD_TRY(tdscha::perturb_average_vjp_device(e, nb, R1, Ys, apply_d4, fbar, Dbar, Ybar, rhobar, st, precision));
    return precision == TDSCHA_PREC_FP64 ? 0 : tdscha::check_err_word(e, st);
}

extern "C" int tdscha_perturb_average_vjp_device(tdscha_ensemble *e, int nb, const double *R1, const double *Ys, int apply_d4,
                                                 const double *fbar, const double *Dbar, double *Ybar, double *rhobar,
                                                 void *stream) {
    clear_error();
    TD_CHECK(e != nullptr, TDSCHA_EINVAL, "NULL ensemble");
    TD_CUDA(cudaSetDevice(e->device));
    return tdscha::perturb_average_vjp_device(e, nb, R1, Ys, apply_d4, fbar, Dbar, Ybar, rhobar,
                                              static_cast<cudaStream_t>(stream));
}
