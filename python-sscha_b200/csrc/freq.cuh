// freq.cuh -- the two big contractions of the averages over the characters of the subgroup K.
//
// On the factorised symmetry path every symmetry is S_j = S_p D_t (p a coset representative, D_t in
// the abelian subgroup K, 2 x 2 sparse in the rotated basis), and the per-row quantities only enter
// through
//     a_(p,t),i = <U_p, D_t M_i D_t^T>_F,   U_p = S_p^T Ys S_p,   M_i = x_i x_i^T or sym(x_i g_i^T)
//     c_(p,t),i = r1_p . D_t x_i            (and b, d with g_i)
//     N~_p = sum_t D_t (sum_i w_(p,t),i M_i) D_t^T,   F~_p = sum_t D_t (sum_i w'_(p,t),i v_i).
// In the rotated basis symmetric matrices decompose into components xi_k, each a real number or a
// complex number (a 2 x 2 block's linear / antilinear part, or a real mode times a complex pair)
// that D_t multiplies by a character chi(t) of K.  Grouping the components by character class
// (chi and its conjugate; the stored "canonical" component is conjugated where needed):
//     a_(p,t) = sum_K Re( conj(chi_K(t)) H_K ),   H_K = sum_{k in K} m_k u_k conj(xi_k(M_i))
// (m_k the Frobenius multiplicity of the component) and, because every weight is linear in a, b, c,
// d with per-configuration coefficients, the weights' transforms over t are
//     sum_t a_(p,t) chi_K(t) = s_K H_K,   s_K = |K| / 2 (complex class) or |K| Re (real class),
// so the weights can be formed class by class without ever leaving the character basis, and
//     xi_k(N~_p) = sum_i w^_K,i xi_k(M_i),     the same for the mode components of F~_p.
// Each character class is one contraction over only its own components: the two big contractions
// shrink from N_sym rows x all P pairs to (2 x cosets) rows per class x the class's pairs, about
// |K| / 2 times fewer flops.  Layouts (NR = nb x cosets in the chunk):
//   pair columns: the P components (complex ones as a real and an imaginary column) sorted by
//     class, each class padded to a multiple of 64 columns (Kq in all);
//   mode columns: the n mode components (complex orbits as two columns) by class, padded (Kmq);
//   left operands / outputs: rows (comp, v, c) = comp * NR + v * ncos + c, comp 0 the real part.
#pragma once
#include <vector>
#include "common.cuh"
#include "cosets.cuh"

namespace tdscha {

// Host description of the character classes and the component layouts.
struct FreqLayout {
    bool ok = false;
    int n_class = 0, Kq = 0, Kmq = 0;
    std::vector<int> cls_real;                        // class is a real character
    std::vector<int> pcol_off, pcol_cnt;              // pair columns of each class (padded)
    std::vector<int> mcol_off, mcol_cnt;              // mode columns of each class (padded; 0 when none)
    std::vector<int> mcol_used;                       // the class's mode columns before padding
    // per pair column: own value = c0 M[mu0, nu0] + c1 M[mu1, nu1] of a symmetric matrix M
    std::vector<int> pc_mu0, pc_nu0, pc_mu1, pc_nu1;
    std::vector<double> pc_c0, pc_c1;
    std::vector<int> pc_partner;                      // the other column of a complex component (-1: none)
    std::vector<double> pc_re, pc_im;                 // left rows: Re = pc_re own(c), Im = pc_im own(partner)
    std::vector<double> pc_zc;                        // output: own(c) = O1[c] + pc_zc O2[partner]
    // per packed pair (mu <= nu): N~[mu, nu] = pp_c0 own(pp_col0) + pp_c1 own(pp_col1)
    std::vector<int> pp_col0, pp_col1;
    std::vector<double> pp_c0, pp_c1;
    // per mode column: own value of a mode vector v = mc_sign v[mc_mode]
    std::vector<int> mc_mode, mc_partner;
    std::vector<double> mc_sign, mc_re, mc_im, mc_zc;
    std::vector<int> mode_col;                        // column of each mode
    double flops_ratio = 0;                           // big-contraction work relative to all symmetries
};

// Classes and layouts from the analysis of the symmetry tables (sym_blocks as given, host).
int build_freq_layout(int n, const std::vector<int> &dim, const std::vector<int> &blk_start, const double *const *sym_blocks,
                      const CosetAnalysis &ca, FreqLayout &out);

// Device copy of the layout tables.
struct FreqTables {
    int n_class = 0, Kq = 0, Kmq = 0;
    std::vector<int> cls_real, pcol_off, pcol_cnt, mcol_off, mcol_cnt, mcol_used;
    int *d_mcol_off = nullptr, *d_mcol_used = nullptr;   // per class (device)
    int *pc_mu0 = nullptr, *pc_nu0 = nullptr, *pc_mu1 = nullptr, *pc_nu1 = nullptr, *pc_partner = nullptr;
    double *pc_c0 = nullptr, *pc_c1 = nullptr, *pc_re = nullptr, *pc_im = nullptr, *pc_zc = nullptr;
    int *pp_col0 = nullptr, *pp_col1 = nullptr;
    double *pp_c0 = nullptr, *pp_c1 = nullptr;
    int *mc_mode = nullptr, *mc_partner = nullptr, *mode_col = nullptr;
    double *mc_sign = nullptr, *mc_re = nullptr, *mc_im = nullptr, *mc_zc = nullptr;
    int *d_cls_real = nullptr;
    double flops_ratio = 0;
    size_t bytes = 0;
};
int freq_tables_create(const FreqLayout &L, FreqTables **out);
void freq_tables_destroy(FreqTables *t);

// Per-ensemble operands in the character basis, one storage format (hi, lo):
//   Vq  (2Nc x Kq):  [xi(x x^T) ; xi(sym(x g^T))] rows per configuration
//   VqT (Kq x N2pc): the same transposed (zero columns past 2Nc)
//   XGq (2Nc x Kmq): [mode components of x ; of g]
//   YXq (Kmq x N2pc): [mode components of y | of x~] transposed
struct FreqOps {
    bool built = false, has_lo = false;
    void *V_hi = nullptr, *V_lo = nullptr, *VT_hi = nullptr, *VT_lo = nullptr;
    void *XG_hi = nullptr, *XG_lo = nullptr, *YX_hi = nullptr, *YX_lo = nullptr;
    size_t bytes = 0;
};
size_t freq_operand_bytes(const FreqTables &t, long long Nc, Format fmt, bool lo);
// Operands of configurations [c0, c0 + Nc) into caller-provided storage `buf` (freq_operand_bytes).
// X, G, Y, Xt: (N x n) rotated-basis ensemble (row c0 first); XGT: [X^T; G^T] (2n x ldT, column c0
// first) or nullptr (the split formats build from it when given).
int freq_build_operands(const FreqTables &t, const double *X, const double *G, const double *Y, const double *Xt,
                        const double *XGT, long long ldT, int n, long long Nc, Format fmt, bool lo, void *buf, FreqOps &o,
                        cudaStream_t st);

// Configuration chunks over a resident row-major operand (split formats): Vq and XGq of all N
// configurations stay resident (freq_build_rows, freq_resident_rows_bytes), and per chunk only the
// transposed operands are formed: VqT by a tiled transpose of the chunk's two row ranges of Vq
// (rows c0.. and N + c0..), YXq from Y, X~ (freq_build_chunk_cols, freq_chunk_cols_bytes).  The
// chunk's FreqOps then points at the resident Vq / XGq, whose chunk rows the [a|b] and [c|d]
// contractions address as two row ranges.
size_t freq_resident_rows_bytes(const FreqTables &t, long long N, Format fmt, bool lo);
size_t freq_chunk_cols_bytes(const FreqTables &t, long long Nc, Format fmt, bool lo);
int freq_build_rows(const FreqTables &t, const double *X, const double *G, const double *XGT, long long ldT, int n, long long N,
                    Format fmt, bool lo, void *buf, FreqOps &o, cudaStream_t st);
int freq_build_chunk_cols(const FreqTables &t, const FreqOps &rows, long long N, long long c0, long long Nc, const double *Y,
                          const double *Xt, int n, Format fmt, bool lo, void *buf, FreqOps &o, cudaStream_t st);

// Left operands from the representatives' transforms (InT float or double):
//   Lab (2 NR x Kq) from U (NR x ldu, packed pairs), Lcd (2 NR x Kmq) from r1p (NR x ldr).
template <typename InT>
int freq_left(const FreqTables &t, int NR, int n, const InT *U, long long ldu, const InT *r1p, long long ldr, Format fmt,
              void *Lab_hi, void *Lab_lo, void *Lcd_hi, void *Lcd_lo, cudaStream_t st);

// Weights of the character basis, class by class: from [a|b] (H) and [c|d] (Ch), rows
// g * 2NR + (comp, v, c) with ld, columns i < Nc and Nc + i, write Cw = [delta/2 | gamma] and
// AB = [alpha | beta] (ld N2pc, zero columns from 2Nc on); the imaginary rows of real classes are
// skipped (their contractions never read them).
template <typename AccT>
int freq_weights(const FreqTables &t, const AccT *H, const AccT *Ch, long long ld, const double *rho, long long Nc, int NR,
                 long long N2pc, int d4, Format fmt, void *Cw_hi, void *Cw_lo, void *AB_hi, void *AB_lo, cudaStream_t st);

// ---- the averages' VJP in the character basis -------------------------------------------------
// With the hatted class-basis quantities (H = [a|b], Ch = [c|d] from U / r1; HQ = [A'|B'], Cp =
// [C'|D'] from the cotangent transforms Q / phi) the VJP's per-row coefficients are linear:
//   K1 = d4 A'/8 - D'/3,  K2 = -c/3 + d4 a/8,  K3 = -A'/6,  K4 = -a/6,
// and the transposed contractions over the rows give the components of the configuration-side
// cotangents: xi(Vbar_i) = sum_p conj(K1) xi(U_p) + conj(K2) xi(Q_p), z(gbar_i) += sum_p conj(K3)
// z(r1_p), z(ypart_i) = sum_p conj(K4) z(phi_p), real GEMMs whose right operands are the left
// operands L (their columns scaled by s_K m, undone in freq_vjp_reconstruct).  The weights'
// pairing sum over the symmetry rows (rho's cotangent) is a sum over rows of products / s_K.

// Row-major mode components of two (Nc x n) arrays, [A ; B] (2Nc x Kmq): [X; G] or [Y; X~].
int freq_build_mode_rows(const FreqTables &t, const double *A, const double *B, int n, long long Nc, Format fmt, void *hi,
                         void *lo, cudaStream_t st);
// out (cols x 2 NRp) = L^T with the rows comp * NR + j moved to comp * NRp + j (zeros elsewhere).
int freq_transpose_left(Format fmt, const void *L, int NR, int NRp, long long cols, void *out, cudaStream_t st);
// Coefficients of the VJP from H, Ch, HQ, Cp (rows g * 2NR + comp * NR + j, ld, columns i and N + i):
//   trans: K1..K4 transposed (N x nC * 2NRp, row g * 2NRp + comp * NRp + j), split into fmt
//          (zeroed first by the caller: padding and the imaginary rows of real classes stay zero);
//   else:  K1..K4 row-major like H (rows x ldk, FP64).
//   BR (rows x N, FP64): the rho-pairing terms of every row, 1 / s_K included (0 for unused rows).
template <typename AccT>
int freq_vjp_coef(const FreqTables &t, int sub, const AccT *H, const AccT *Ch, const AccT *HQ, const AccT *Cp, long long ld,
                  int N, int NR, int NRp, int d4, bool trans, Format fmt, void *const *K_hi, void *const *K_lo, long long ldk,
                  double *BR, cudaStream_t st);
// Vbar (N x ldv, packed entries), gbar / ypart (N x ldg, mode entries; gbar accumulated) from the
// component outputs VbarQ (N x Kq), GQ and YQ (N x Kmq).
template <typename T>
int freq_vjp_reconstruct(const FreqTables &t, int N, int n, long long P, const T *VbarQ, const T *GQ, const T *YQ, T *Vbar,
                         long long ldv, T *gbar, T *ypart, long long ldg, cudaStream_t st);

// The weights with the thin [c|d] contraction folded in (split formats): c and d of row r and
// configuration i are the dot products of the row's left operand Lcd (2NR x Kmq, hi + lo) with the
// configuration's mode components XGq (2Nc x Kmq, hi + lo) over the row's class columns, formed in
// fp32 next to [a|b] (H) instead of being stored by a contraction and read back.
int freq_weights_cd(const FreqTables &t, const float *H, long long ld, const void *Lcd_hi, const void *Lcd_lo, const void *XG_hi,
                    const void *XG_lo, const double *rho, long long Nc, int NR, long long N2pc, int d4, Format fmt, void *Cw_hi,
                    void *Cw_lo, void *AB_hi, void *AB_lo, cudaStream_t st);

// Back from the character basis: Zs (NR x ldz, packed c_p N~) from O (2 NR x Kq), Fs (NR x ldf)
// from OF (2 NR x Kmq).
template <typename AccT>
int freq_reconstruct(const FreqTables &t, int NR, int n, long long P, const int *pmu, const int *pnu, const AccT *O,
                     const AccT *OF, AccT *Zs, long long ldz, AccT *Fs, long long ldf, cudaStream_t st);

}  // namespace tdscha
