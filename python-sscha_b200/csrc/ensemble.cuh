// ensemble.cuh -- device-resident ensemble and the symmetrised perturbed averages.
//
// Reformulation of the reference's per-(configuration, symmetry) loop
// (CModules/LanczosFunctions.c:2082-2754) used by every precision mode.  With u = S_j x_i,
// f = S_j y_i, ups/psi thermal factors (commuting with S_j inside a degenerate block),
// x~ = ups o x, g = psi o y, R~_j = S_j^T R1, Ys = (Y1 + Y1^T)/2, Y~_j = S_j^T Ys S_j:
//     a_ij = x_i^T Y~_j x_i            b_ij = x_i^T Y~_j g_i
//     c_ij = r1_j . x_i                d_ij = r1_j . g_i        (r1_j = ups o R~_j)
//     gamma = rho(-c/3 + a/8 [d4]),  delta = rho(-d/3 + b/4 [d4]),  alpha = -rho a/6,  beta = -rho b/3
//     f_av  = 1/(N_eff N_sym) sum_j S_j [ sum_i alpha_ij y_i + beta_ij x~_i ]
//     D_av  = 1/(N_eff N_sym) sum_j S_j W_j S_j^T,
//     W_j[mu,nu] = ups_mu ups_nu sum_i gamma_ij (x_mu g_nu + g_mu x_nu) + delta_ij x_mu x_nu.
// Over the packed pair index p = (mu <= nu) both O(N N_sym n^2) pieces become dense contractions
// with the per-ensemble matrix V (2N x P):
//     V[i, p]   = c_p x_i,mu x_i,nu            (c_p = 2 off the diagonal, 1 on it)
//     V[N+i, p] = x_i,mu g_i,nu + x_i,nu g_i,mu (off diagonal), x_i,mu g_i,mu (diagonal)
//   GEMM1  [a | b] (N_sym x 2N)   = B1 (N_sym x P) . V^T,        B1[j, p] = Y~_j[mu, nu]
//   GEMM2  Z (N_sym x P)          = Cw (N_sym x 2N) . V,         Cw[j] = [delta_j/2 | gamma_j]
//   W_j[mu,nu] = e_p ups_mu ups_nu Z[j, p]   (e_p = 2 on the diagonal, 1 off it)
// and two thin ones (K = n and N = n): [c | d] = r1 . [X; G]^T and F = [alpha | beta] . [Y^T | X~^T]^T.
// No symmetry image of any configuration is ever formed: S_j acts on n x n objects only.
#pragma once
#include <cublas_v2.h>
#include <vector>
#include "common.cuh"
#include "symmetry.cuh"
#include "cosets.cuh"
#include "freq.cuh"

struct tdscha_ensemble;

namespace tdscha {

struct OperandSet {          // the per-ensemble GEMM operands in one storage format
    bool built = false;
    bool has_lo = false;
    void *V_hi = nullptr, *V_lo = nullptr;       // 2N x Kp
    void *VT_hi = nullptr, *VT_lo = nullptr;     // P x N2p
    void *XG_hi = nullptr, *XG_lo = nullptr;     // 2N x np
    void *YXt_hi = nullptr, *YXt_lo = nullptr;   // n x N2p
    size_t bytes = 0;
};

struct Workspace {
    void *base = nullptr;
    size_t bytes = 0;
};

// Chunking plan of the last averages call (reused verbatim while a CUDA graph is being captured,
// when neither device memory queries nor allocations may happen).
struct AvgPlan {
    bool valid = false;
    int nb = 0, fmt = -1;
    bool lo = false;
    bool cosets = false;
    bool freq = false;
    bool half = false;   // configuration chunks over resident row-major class operands
    long long Nc = 0;
    int Jc = 0;
};

// Stages of one averages call, for the optional CUDA-event profile.
enum Stage : int { ST_TRANSFORM = 0, ST_GEMM_AB, ST_GEMM_CD, ST_WEIGHTS, ST_GEMM_Z, ST_GEMM_F, ST_FOLD, ST_OTHER, ST_OPERANDS, ST_COUNT };

struct ProfRec {
    int stage;
    cudaEvent_t a, b;
};

struct Profile {
    bool enabled = false;
    std::vector<ProfRec> recs;
    long long launches[ST_COUNT] = {0};
    void begin(int stage, cudaStream_t st, ProfRec *r);
    void end(ProfRec *r, cudaStream_t st);
};

}  // namespace tdscha

struct tdscha_ensemble {
    int device = 0;
    int n = 0, N = 0, N_sym = 0, n_blocks = 0;
    long long P = 0, Kp = 0, N2 = 0, N2p = 0, np = 0;
    double T = 0, N_eff = 0;
    int dmax = 0;
    std::vector<int> blk_start, blk_dim;
    std::vector<long long> blk_sym_off;
    std::vector<int> bp_b, bp_c;                   // block pairs b <= c
    // device arrays
    double *X = nullptr, *Y = nullptr, *G = nullptr, *Xt = nullptr;
    double *rho = nullptr, *w = nullptr, *ups = nullptr, *psi = nullptr, *sym = nullptr;
    float *symP = nullptr, *symPT = nullptr;       // padded fp32 symmetry tables (as given, transposed)
    long long *d_offP = nullptr;                   // block offsets into symP / symPT
    int *d_blk_start = nullptr, *d_blk_dim = nullptr, *d_blocks_ids = nullptr, *d_bp_b = nullptr, *d_bp_c = nullptr;
    long long *d_blk_sym_off = nullptr;
    int *d_pair_mu = nullptr, *d_pair_nu = nullptr;
    unsigned *d_err = nullptr;
    tdscha::OperandSet ops[3];                     // indexed by Format
    tdscha::Workspace ws;
    tdscha::Workspace vjp_ws;                      // workspace of the averages' VJP
    tdscha::Workspace chunk_ops;                   // operands of one configuration chunk (large ensembles)
    tdscha::AvgPlan plan;                          // chunking plan of the last averages call
    double *YX = nullptr;                          // [Y; X~] (2N x np), FP64, built by the first VJP
    double *XGT = nullptr;                         // [X^T; G^T] (2n x N), FP64, built by the first operand build
    double *d_static_lam = nullptr;                // Lambda of the static L1 per packed pair (P), built on first use
    cublasHandle_t cublas = nullptr;
    size_t base_bytes = 0;
    tdscha::Profile prof;
    tdscha::PairClasses pairs;
    tdscha::SymUmma *umma = nullptr;               // tcgen05 symmetry transform / fold tables (bf16 formats)
    void *YXm_hi[3] = {nullptr, nullptr, nullptr};  // [Y; X~] (2N x np) per storage format (mixed VJP)
    void *YXm_lo[3] = {nullptr, nullptr, nullptr};
    // Rotated mode basis (inside degenerate blocks) in which a subgroup of the symmetries is 2 x 2
    // sparse: X, Y, G, X~ and the symmetry tables are stored in it, and the averages and their VJP
    // rotate their inputs in and their outputs back.  nullptr: the basis as given.
    double *Rrow = nullptr;                        // n x dmax, Rrow[mu][q] = R_b[mu - s_b][q]
    tdscha::SymCosets *cosets = nullptr;           // factorised symmetry transform / fold (mixed formats)
    tdscha::FreqTables *freq = nullptr;            // character classes of the subgroup (freq.cuh)
    tdscha::FreqOps fops[3];                       // character-basis operands per storage format (resident)
    tdscha::FreqOps fhalf[3];                      // resident row-major class operands of chunked ensembles
    void *fyx_hi[3] = {nullptr, nullptr, nullptr};  // [Y; X~] mode components (2N x Kmq) per format (class VJP)
    void *fyx_lo[3] = {nullptr, nullptr, nullptr};
    tdscha::Workspace rot_ws;                      // rotated inputs / outputs of the VJP
};

namespace tdscha {

int ensemble_create(const double *X, const double *Y, const double *w, const double *rho, int N, int n, double T,
                    int N_sym, int n_blocks, const int *n_deg, const int *const *deg_space,
                    const double *const *sym_blocks, const int *blocks_ids, tdscha_ensemble **out);
int ensemble_destroy(tdscha_ensemble *e);

// nb perturbations, device pointers.  Ys: (nb, n, n) SYMMETRIC upsilon; R1: (nb, n).
int perturb_average_device(tdscha_ensemble *e, int nb, const double *R1, const double *Ys, int apply_d4,
                           int precision, double *f_out, double *d_out, cudaStream_t st);

// Vector-Jacobian product of the averages with respect to the ensemble's forces Y and weights rho:
// for cotangents (fbar, Dbar) of (f_av, D_av) at the perturbations (R1, Ys), writes
//   Ybar (N, n) = d<fbar, f_av> + <Dbar, D_av> / dY,   rhobar (N) = same / drho   (summed over nb)
// FP64 (cuBLAS DGEMM) by default; a mixed `precision` runs its eight contractions on the tcgen05
// kernel in that storage format (the rest stays FP64).  Dbar must be symmetric (the Frobenius
// product is used).
int perturb_average_vjp_device(tdscha_ensemble *e, int nb, const double *R1, const double *Ys, int apply_d4,
                               const double *fbar, const double *Dbar, double *Ybar, double *rhobar, cudaStream_t st,
                               int precision = TDSCHA_PREC_FP64);

// (nb, n, n) -> (Y + Y^T)/2 on the device
int symmetrize_device(int nb, int n, const double *Y, double *Ys, cudaStream_t st);

}  // namespace tdscha
