// cosets.cuh -- the symmetry group factorised over the cosets of a subgroup that is 2 x 2 sparse
// in a rotated mode basis.
//
// The averages need, for every symmetry j, Y~_j = S_j^T Ys S_j (transform) and S_j W_j S_j^T,
// S_j F_j (fold), restricted to degenerate blocks.  Let K be the kernel of the representation on one
// degenerate block b0 (for a crystal in a supercell with a Gamma-point block: the lattice
// translations).  K is a normal subgroup, its left cosets are the classes of equal S_j on b0, and
// with one representative p per coset every symmetry is S_j = S_p D_j, D_j = S_p^T S_j in K.  If K
// is abelian, an orthogonal change of basis inside every degenerate block (R_b, built here from K's
// matrices) brings all of K's matrices to 1 x 1 / 2 x 2 blocks: each rotated mode q has a partner
// pi(q) (itself for a real character) and D_j has non-zeros only at (q, q) and (pi(q), q).  Then
//     Y~_j = D_j^T U_p D_j,          U_p = S_p^T Ys S_p           (dense only per coset)
//     S_j W_j S_j^T = S_p (D_j W_j D_j^T) S_p^T,   S_j F_j = S_p (D_j F_j)
// and the dense work runs over the cosets only; the expansion to the symmetries of a coset is
// four-term arithmetic per packed pair, bound by the memory traffic of B1 and Z.
#pragma once
#include <string>
#include <vector>
#include "common.cuh"

namespace tdscha {

// Host analysis of the symmetry tables (sym_blocks[b]: N_sym x d_b x d_b, row-major, as given).
struct CosetAnalysis {
    bool ok = false;
    int b0 = -1;                   // block whose representation's kernel is the subgroup
    int sub = 0;                   // order of the subgroup = rows per coset
    int n_cos = 0;                 // number of cosets
    std::vector<int> order;        // internal symmetry row -> symmetry index (coset-major)
    std::vector<int> kset;         // the subgroup's symmetry indices
    std::vector<int> partner;      // n: partner of each rotated mode (global index)
    std::vector<double> R;         // per block d x d, R_b[q'][q] = component q' of rotated mode q
    std::vector<long long> R_off;  // offset of block b's R_b in R
    double offpattern = 0;         // largest entry of R^T D R outside the 2 x 2 pattern (subgroup)
    std::string why;               // reason when !ok
};

int analyse_cosets(int N_sym, const std::vector<int> &dim, const double *const *sym_blocks, CosetAnalysis &out);

// Device data of the rotated basis and of the factorised symmetry path of one ensemble.
struct SymCosets {
    int n_cos = 0, sub = 0;
    int *order = nullptr;          // N_sym
    int *partner = nullptr;        // n
    float *c0 = nullptr;           // (N_sym internal rows) x n: D_j[q, q]
    float *c1 = nullptr;           // (N_sym internal rows) x n: D_j[pi(q), q] (0 without a partner)
    float *repP = nullptr, *repPT = nullptr;   // padded fp32 tables of the representatives (as given / transposed)
    long long *d_offRep = nullptr;             // block offsets into repP / repPT
    double *repS = nullptr;                    // FP64 tables of the representatives (n_cos, d, d) per block
    long long *d_offRepS = nullptr;            // block offsets into repS
    double offpattern = 0;         // device check over all symmetries
};

// Rotation to / from the rotated basis of an (rows x n) row-vector array (every row transformed):
// to_rot: out = in . R, else out = in . R^T.  Rrow is n x dmax with Rrow[mu][q] = R_b[mu - s_b][q].
int rotate_rows_of(long long rows, int n, int dmax, const double *Rrow, const int *blocks_ids, const int *blk_start,
                   const int *blk_dim, const double *in, double *out, bool to_rot, cudaStream_t st);
// (nb x n x n): to_rot: out = R^T A R, else out = R A R^T (tmp: nb x n x n scratch)
int rotate_mats(int nb, int n, int dmax, const double *Rrow, const int *blocks_ids, const int *blk_start, const int *blk_dim,
                const double *in, double *tmp, double *out, bool to_rot, cudaStream_t st);

// Set-up on the device (ensemble creation): tables (N_sym, d, d) of block b rotated in place,
// M' = R_b^T M R_b.
int rotate_sym_tables(double *sym_b, int N_sym, int d, const double *Rb, cudaStream_t st);
// Coefficients c0, c1 of every internal row from the rotated FP64 tables; returns the largest
// entry outside the pattern in *offmax (device, as the bits of a non-negative double).
int coset_coefficients(int N_sym, int n, int sub, const int *order, const int *partner, const int *blocks_ids,
                       const int *blk_start, const int *blk_dim, const double *sym, const long long *blk_sym_off, float *c0,
                       float *c1, unsigned long long *offmax, cudaStream_t st);

// Transform expansion: B1 rows r = k * nj + l (l in [0, nj), nj = ncj * sub, coset l / sub) from
// U rows k * ncj + l / sub (fp32, packed pairs, ld Kp); writes every column of [0, Kp) (zeros past P).
int coset_expand(int nb, int ncj, int sub, int j0, long long P, long long Kp, int n, const float *U, const int *pmu,
                 const int *pnu, const int *partner, const float *c0, const float *c1, Format fmt, void *B1_hi, void *B1_lo,
                 cudaStream_t st);
// r1 rows (ld np) from the representatives' r1p rows (fp32, ld np); zeros past n.
int coset_expand_r1(int nb, int ncj, int sub, int j0, int n, long long np, const float *r1p, const int *partner,
                    const float *c0, const float *c1, Format fmt, void *r1_hi, void *r1_lo, cudaStream_t st);
// Fold, inner part: Zs rows k * ncj + c = (1/e) sum over the coset's rows of D_j (e o Z_j) D_j^T
// (packed pairs, ld ldz, e = 2 on the diagonal), Fs rows = sum of D_j F_j (ld ldf).
int coset_fold_inner(int nb, int ncj, int sub, int j0, long long P, long long ldz, long long ldf, int n, const float *Z,
                     const float *F, const int *pmu, const int *pnu, const int *partner, const float *c0, const float *c1,
                     float *Zs, float *Fs, cudaStream_t st);

}  // namespace tdscha
