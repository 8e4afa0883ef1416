// symmetry.cuh -- the O(N_sym n^2 d) symmetry work of one averages call.
//
//   transform: B1[(k,j), p(mu,nu)] = (S_j^T Ys_k S_j)[mu, nu]  (packed, in the GEMM storage format)
//              r1[(k,j), mu]       = ups_mu (S_j^T R1_k)_mu
//   fold:      D_k = sum_j S_j W_kj S_j^T,  f_k = sum_j S_j F_kj   (FP64 partial sums per j-chunk)
// S_j is block diagonal over degenerate blocks, so both run per block pair (b <= c): the products
// S_b^T Ys[b,c] S_c and S_b W[b,c] S_c^T are d_b x d_c matrices.  Block pairs are grouped into
// classes by max(d_b, d_c) so that each class runs with a register micro-tile (MT x MT outputs per
// thread of a 16 x 16 grid) that covers it with little waste.
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "common.cuh"

namespace tdscha {

constexpr int SYM_THREADS = 256;
constexpr int SYM_MT_MAX = 5;                      // blocks up to 16 * 5 = 80 modes
constexpr int DMAX_SUPPORTED = 16 * SYM_MT_MAX;

struct SymUmma;

struct SymTables {
    const double *sym;         // per-block (N_sym, d, d) tables, concatenated
    const long long *off;      // offset of block b's table
    const int *start, *dim;    // first mode and size of block b
    int n_blocks, n, dmax;
    // fp32 copies for the tensor-core kernels of the mixed-precision modes: block b's (N_sym, DP, DP)
    // tables with DP = d_b rounded up to 4 (zero padded), as given (symP) and transposed (symPT),
    // starting at element offP[b]
    const float *symP, *symPT;
    const long long *offP;
    // tensor-core (tcgen05) transform / fold of the bf16 formats (symmetry_umma.cu), when built
    SymUmma *umma = nullptr;
    const int *blocks_ids = nullptr;   // block of each mode (device)
    unsigned *err = nullptr;           // error word of the call (bounded waits)
};

// bf16 hi / lo symmetry tables with their TMA descriptors and the work items of the tcgen05
// transform / fold (symmetry_umma.cu); one per ensemble, built on the first bf16-format call.
int sym_umma_create(const SymTables &t, int N_sym, const std::vector<int> &dim, const std::vector<long long> &sym_off,
                    SymUmma **out);
void sym_umma_destroy(SymUmma *u);
int sym_transform_umma(SymUmma *u, const SymTables &t, const int *blocks_ids, int nb, int nj, int j0, const double *Ys,
                       const double *R1, const double *ups, long long Kp, long long np, Format fmt, void *B1_hi, void *B1_lo,
                       void *r1_hi, void *r1_lo, unsigned *err, cudaStream_t st);
int sym_fold_umma(SymUmma *u, const SymTables &t, const int *blocks_ids, int nb, int nj, int j0, int Jf, int nf_total,
                  const float *Z, long long ldz, const float *F, long long ldf, const double *ups, double *partD,
                  double *partF, unsigned *err, cudaStream_t st);

// Block pairs (b <= c) grouped by micro-tile class MT = ceil(max(d_b, d_c) / 16).
struct PairClasses {
    int count[SYM_MT_MAX + 1] = {0};
    int *b[SYM_MT_MAX + 1] = {nullptr};
    int *c[SYM_MT_MAX + 1] = {nullptr};
};

int build_pair_classes(const std::vector<int> &dim, PairClasses &pc, size_t *bytes);
void free_pair_classes(PairClasses &pc);

// rows r = k * nj + (j - j0); compute in FP32 when fp32_compute (mixed-precision storage formats)
int sym_transform(const SymTables &t, const PairClasses &pc, int nb, int nj, int j0, const double *Ys, const double *R1,
                  const double *ups, long long P, long long Kp, long long np, Format fmt, void *B1_hi, void *B1_lo,
                  void *r1_hi, void *r1_lo, bool fp32_compute, cudaStream_t st);

// The same two stages on the tensor pipe (mma.sync, three-term tf32 splitting), used by the
// mixed-precision modes; FP64 keeps sym_transform / sym_fold with T = double.
int sym_transform_tc(const SymTables &t, const PairClasses &pc, int nb, int nj, int j0, const double *Ys, const double *R1,
                     const double *ups, long long Kp, long long np, Format fmt, void *B1_hi, void *B1_lo, void *r1_hi,
                     void *r1_lo, cudaStream_t st);
int sym_fold_tc(const SymTables &t, const PairClasses &pc, int nb, int nj, int j0, int Jf, int nf_total, const float *Z,
                long long ldz, const float *F, long long ldf, const double *ups, double *partD, double *partF, cudaStream_t st);

// Z (rows r as above, packed pairs, ldz), F (rows r, ldf); partials per (k, fold chunk fg).  The
// per-symmetry block products run in FP32 when fp32_compute and are summed over symmetries in FP64.
template <typename AccT>
int sym_fold(const SymTables &t, const PairClasses &pc, const int *blocks_ids, int nb, int nj, int j0, int Jf, int nf_total,
             const AccT *Z, long long ldz, const AccT *F, long long ldf, const double *ups, double *partD, double *partF,
             bool fp32_compute, cudaStream_t st);

}  // namespace tdscha
