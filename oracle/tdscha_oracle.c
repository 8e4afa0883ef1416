/*
 * tdscha_oracle.c -- CPU restatement of the reference's symmetrised perturbed ensemble averages.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links, loads or calls this file; it is used by
 * tests/, by __graft_entry__.smoke() and by bench.py's cpu_baseline leg, and only as the checker.
 *
 * It restates, pair by pair, what the reference computes in
 *   CModules/LanczosFunctions.c:2082-2254  get_f_average_from_Y_pert_sym_fast   (f average, "D3 from Y1")
 *   CModules/LanczosFunctions.c:2257-2438  get_d2v_dR2_from_R_pert_sym_fast     (<d2V/dR2> from R1, overwrite)
 *   CModules/LanczosFunctions.c:2615-2754  get_d2v_dR2_from_Y_pert_sym_fast     (<d2V/dR2> from Y1, "D4", add)
 * as called by the CPython binding CModules/odd_corr_module.c:491-634 (GetPerturbAverageSym).
 *
 * For every configuration i and symmetry j the image u = S_j x_i, f = S_j y_i is formed with the
 * block gather of LanczosFunctions.c:2158-2170 (S_j is block diagonal over degenerate subspaces;
 * block b acts on the contiguous modes deg_space[b][0] .. deg_space[b][0]+n_deg[b]-1), then
 *     W1 = -1/2 sum_{mu,nu} u_mu u_nu Y1[mu,nu]
 *     W2 = -1/4 sum_{mu,nu} Y1[mu,nu] (u_mu psi_nu f_nu + u_nu psi_mu f_mu)
 *     f_av  += rho_i W1 f / 3 + rho_i W2 (ups o u) 2/3
 *     W3 = R1 . (ups o u),  W4 = R1 . f
 *     D_av  -= rho_i W3/3 ((ups o u) f^T + f (ups o u)^T) + rho_i W4/3 (ups o u)(ups o u)^T
 *   and, when apply_d4,
 *     W5 = -(rho_i/8) u^T Y1 u,  W6 = -(rho_i/8) sum Y1[mu,nu] (psi_mu f_mu u_nu + psi_nu f_nu u_mu)
 *     D_av  -= W5 ((ups o u) f^T + f (ups o u)^T) + W6 (ups o u)(ups o u)^T
 * and both averages are divided by N_eff * N_sym with N_eff = sum rho.
 * ups(w) = 2w/(1+2n(w)), psi = 1/ups, n(w) = 1/(exp(w*RY_TO_K/T) - 1) (LanczosFunctions.c:14-30).
 *
 * Differences from the reference that do not change the result beyond rounding: the thermal
 * factors are tabulated once instead of calling exp() inside the n^2 loops, Y1 u and Y1^T u are
 * formed once per pair, and configurations are split over OpenMP threads (contiguous slices, the
 * same partition the reference uses over MPI ranks at LanczosFunctions.c:2123-2136) with the
 * per-thread partial sums added in thread order.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_RY_TO_K 157887.32400374097

static double bose(double w, double T) {
    if (T > 0) return 1.0 / (exp(w * ORACLE_RY_TO_K / T) - 1.0);
    return 0.0;
}

/*
 * Returns 0 on success, a negative code on bad arguments.
 *   X, Y     : (N, n) C order
 *   sym_flat : concatenation over blocks b of the (N_sym, d_b, d_b) tables
 *   deg_flat : concatenation over blocks of their mode indices (contiguous ascending per block)
 *   n_deg    : (n_blocks) block sizes;  blocks_ids : (n) block of each mode
 *   i_start, i_stop : configuration slice to accumulate (pass 0, N for the whole ensemble);
 *                     the normalisation always uses the N_eff of the whole ensemble.
 *   n_threads: <= 0 means the OpenMP default.
 */
int oracle_perturb_average_sym(const double *X, const double *Y, const double *w, const double *rho,
                               const double *R1, const double *Y1, double T, int apply_d4,
                               int N, int n, int N_sym, int n_blocks, const int *n_deg,
                               const int *deg_flat, const double *sym_flat, const int *blocks_ids,
                               int i_start, int i_stop, int n_threads,
                               double *f_out, double *d2v_out) {
    if (N <= 0 || n <= 0 || N_sym <= 0 || n_blocks <= 0) return -1;
    if (apply_d4 != 0 && apply_d4 != 1) return -2;
    if (i_start < 0 || i_stop > N || i_start > i_stop) return -3;

    int *blk_first = (int *)malloc(sizeof(int) * n_blocks);
    size_t *blk_sym_off = (size_t *)malloc(sizeof(size_t) * n_blocks);
    int off = 0;
    size_t soff = 0;
    for (int b = 0; b < n_blocks; ++b) {
        blk_first[b] = deg_flat[off];
        blk_sym_off[b] = soff;
        off += n_deg[b];
        soff += (size_t)N_sym * n_deg[b] * n_deg[b];
    }
    if (off != n) { free(blk_first); free(blk_sym_off); return -4; }

    double *ups = (double *)malloc(sizeof(double) * n);
    double *psi = (double *)malloc(sizeof(double) * n);
    for (int m = 0; m < n; ++m) {
        double nb = bose(w[m], T);
        ups[m] = 2.0 * w[m] / (1.0 + 2.0 * nb);
        psi[m] = (1.0 + 2.0 * nb) / (2.0 * w[m]);
    }
    double N_eff = 0;
    for (int i = 0; i < N; ++i) N_eff += rho[i];

    int nthr = 1;
#ifdef _OPENMP
    nthr = n_threads > 0 ? n_threads : omp_get_max_threads();
#endif
    double *f_part = (double *)calloc((size_t)nthr * n, sizeof(double));
    double *d_part = (double *)calloc((size_t)nthr * n * n, sizeof(double));

#ifdef _OPENMP
#pragma omp parallel num_threads(nthr)
#endif
    {
        int tid = 0, nt = 1;
#ifdef _OPENMP
        tid = omp_get_thread_num();
        nt = omp_get_num_threads();
#endif
        int count = (i_stop - i_start) / nt, rem = (i_stop - i_start) % nt;
        int s0 = i_start + (tid < rem ? tid * (count + 1) : tid * count + rem);
        int s1 = s0 + count + (tid < rem ? 1 : 0);
        double *u = (double *)malloc(sizeof(double) * n);
        double *f = (double *)malloc(sizeof(double) * n);
        double *ut = (double *)malloc(sizeof(double) * n);   /* ups o u */
        double *g = (double *)malloc(sizeof(double) * n);    /* psi o f */
        double *t = (double *)malloc(sizeof(double) * n);    /* Y1 u    */
        double *s = (double *)malloc(sizeof(double) * n);    /* Y1^T u  */
        double *fp = f_part + (size_t)tid * n;
        double *dp = d_part + (size_t)tid * n * n;

        for (int i = s0; i < s1; ++i) {
            const double *xi = X + (size_t)i * n;
            const double *yi = Y + (size_t)i * n;
            for (int j = 0; j < N_sym; ++j) {
                /* symmetry image, LanczosFunctions.c:2158-2170 */
                for (int mu = 0; mu < n; ++mu) {
                    int b = blocks_ids[mu];
                    int d = n_deg[b];
                    int r = mu - blk_first[b];
                    const double *S = sym_flat + blk_sym_off[b] + ((size_t)j * d + r) * d;
                    double su = 0, sf = 0;
                    for (int k = 0; k < d; ++k) {
                        su += S[k] * xi[blk_first[b] + k];
                        sf += S[k] * yi[blk_first[b] + k];
                    }
                    u[mu] = su;
                    f[mu] = sf;
                    ut[mu] = ups[mu] * su;
                    g[mu] = psi[mu] * sf;
                }
                for (int mu = 0; mu < n; ++mu) { t[mu] = 0; s[mu] = 0; }
                for (int mu = 0; mu < n; ++mu) {
                    const double *row = Y1 + (size_t)mu * n;
                    double acc = 0;
                    for (int nu = 0; nu < n; ++nu) {
                        acc += row[nu] * u[nu];
                        s[nu] += row[nu] * u[mu];
                    }
                    t[mu] = acc;
                }
                double uYu = 0, gYu = 0, R1ut = 0, R1f = 0;
                for (int mu = 0; mu < n; ++mu) {
                    uYu += u[mu] * t[mu];
                    gYu += g[mu] * (t[mu] + s[mu]);
                    R1ut += R1[mu] * ut[mu];
                    R1f += R1[mu] * f[mu];
                }
                double ri = rho[i];
                /* f average: W1 = -uYu/2, W2 = -gYu/4 (LanczosFunctions.c:2194-2231) */
                double W1 = -0.5 * uYu, W2 = -0.25 * gYu;
                for (int mu = 0; mu < n; ++mu)
                    fp[mu] += ri * W1 * f[mu] / 3.0 + ri * W2 * ut[mu] * 2.0 / 3.0;
                /* <d2V/dR2>: R part (LanczosFunctions.c:2374-2407) and D4 part (:2687-2725) */
                double cf = ri * R1ut / 3.0;          /* multiplies (ut f^T + f ut^T) */
                double cu = ri * R1f / 3.0;           /* multiplies ut ut^T          */
                if (apply_d4) {
                    cf += -ri / 8.0 * uYu;            /* W5 */
                    cu += -ri / 8.0 * gYu;            /* W6 */
                }
                for (int mu = 0; mu < n; ++mu) {
                    double *drow = dp + (size_t)mu * n;
                    double a1 = cf * ut[mu], a2 = cf * f[mu], a3 = cu * ut[mu];
                    for (int nu = 0; nu < n; ++nu)
                        drow[nu] -= a1 * f[nu] + a2 * ut[nu] + a3 * ut[nu];
                }
            }
        }
        free(u); free(f); free(ut); free(g); free(t); free(s);
    }

    double norm = N_eff * (double)N_sym;
    for (int m = 0; m < n; ++m) {
        double acc = 0;
        for (int th = 0; th < nthr; ++th) acc += f_part[(size_t)th * n + m];
        f_out[m] = acc / norm;
    }
    for (size_t e = 0; e < (size_t)n * n; ++e) {
        double acc = 0;
        for (int th = 0; th < nthr; ++th) acc += d_part[(size_t)th * n * n + e];
        d2v_out[e] = acc / norm;
    }
    free(f_part); free(d_part); free(ups); free(psi); free(blk_first); free(blk_sym_off);
    return 0;
}
