/*
 * tdscha_b200.h -- C ABI of the B200 (sm_100a) TD-SCHA linear-response engine.
 *
 * Plain pointers and sizes only.  Every entry point returns 0 on success and a negative
 * TDSCHA_E* code on failure (never exit()); tdscha_last_error() gives the message of the last
 * failure on the calling thread.  "_device" entry points take device pointers and an optional
 * cudaStream_t passed as void* (NULL = the legacy default stream) and are asynchronous with respect
 * to the host unless stated otherwise; the other entry points take host buffers and synchronise.
 * Temporaries of the entry points that need them live in library-owned device buffers, one per
 * (host thread, device, stream), grown on demand: calls issued from one thread on one stream reuse
 * them in stream order, and calls on different streams or threads never share one.
 *
 * Reference interfaces replaced (mesonepigreco/python-sscha, tdscha package):
 *   sscha_HP_odd.GetPerturbAverageSym          CModules/odd_corr_module.c:491-634
 *     -> tdscha_GetPerturbAverageSym (same argument list), tdscha_perturb_average_sym (resident)
 *   get_f_average_from_Y_pert_sym_fast          CModules/LanczosFunctions.c:2082-2254
 *   get_d2v_dR2_from_R_pert_sym_fast            CModules/LanczosFunctions.c:2257-2438
 *   get_d2v_dR2_from_Y_pert_sym_fast            CModules/LanczosFunctions.c:2615-2754
 *     -> the three are computed together by tdscha_perturb_average_sym[_device]
 *   Lanczos.apply_full_L / apply_L1_FT / apply_anharmonic_FT
 *                                               Modules/DynamicalLanczos.py:3467-3570, 2227-2385, 2891-3281
 *     -> tdscha_apply_full_L_device
 *   Lanczos.run_FT (one bi-conjugate step, n_rep_orth = 0)
 *                                               Modules/DynamicalLanczos.py:6026-6153
 *     -> tdscha_lanczos_step_device
 *   Lanczos.get_green_function_continued_fraction
 *                                               Modules/DynamicalLanczos.py:4951-5047
 *     -> tdscha_continued_fraction_device
 */
#ifndef TDSCHA_B200_H
#define TDSCHA_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* error codes */
#define TDSCHA_OK 0
#define TDSCHA_EINVAL (-1)     /* bad argument (shape, value, layout)                       */
#define TDSCHA_ECUDA (-2)      /* CUDA runtime / driver error                               */
#define TDSCHA_ENOMEM (-3)     /* device allocation failed                                  */
#define TDSCHA_ENOSUPPORT (-4) /* no sm_100 device, or precision not available              */
#define TDSCHA_ETIMEOUT (-5)   /* a device-side bounded wait expired (kernel aborted cleanly) */

/* arithmetic of the two O(N * N_sym * n^2) ensemble contractions; everything else is FP64 */
#define TDSCHA_PREC_FP64 0     /* FP64 throughout                                            */
#define TDSCHA_PREC_TF32 1     /* tcgen05 kind::tf32, one product, FP32 accumulation        */
#define TDSCHA_PREC_BF16X3 2   /* tcgen05 kind::f16 on bf16 hi/lo splits, 3 products, FP32 acc */
#define TDSCHA_PREC_TF32X3 3   /* tcgen05 kind::tf32 on tf32 hi/lo splits, 3 products, FP32 acc */
#define TDSCHA_PREC_BF16 4     /* tcgen05 kind::f16, one bf16 product (accuracy reference)     */

typedef struct tdscha_ensemble tdscha_ensemble;

/* Message of the last failure on this thread ("" if none). */
const char *tdscha_last_error(void);

/* Library version string. */
const char *tdscha_version(void);

/*
 * Upload an ensemble and its mode-space symmetries to the current CUDA device and keep them
 * resident.  Argument meaning follows GetPerturbAverageSym (odd_corr_module.c:519-520):
 *   X, Y        (N, n) C order, mass-rescaled displacements / anharmonic forces in the mode basis
 *   w           (n) frequencies [Ry];  rho (N) weights;  T temperature [K]
 *   N_sym       number of symmetry operations
 *   n_blocks    number of degenerate blocks;  n_deg (n_blocks) block sizes
 *   deg_space   n_blocks pointers, each to n_deg[b] int mode indices (contiguous, ascending)
 *   sym_blocks  n_blocks pointers, each to an (N_sym, n_deg[b], n_deg[b]) C-order table
 *   blocks_ids  (n) block of each mode
 * Every frequency inside a block must be equal to within 1e-10 relative (degenerate subspace).
 */
int tdscha_ensemble_create(const double *X, const double *Y, const double *w, const double *rho,
                           int N, int n, double T, int N_sym, int n_blocks, const int *n_deg,
                           const int *const *deg_space, const double *const *sym_blocks,
                           const int *blocks_ids, tdscha_ensemble **out);

int tdscha_ensemble_destroy(tdscha_ensemble *ens);

/* Sizes of a resident ensemble (any pointer may be NULL). */
int tdscha_ensemble_info(const tdscha_ensemble *ens, int *n, int *N, int *N_sym, int *n_blocks,
                         double *T, double *N_eff);

/*
 * Factorised symmetry path of a resident ensemble.  When the symmetry group has a subgroup K (the
 * kernel of its representation on one degenerate block: the lattice translations of a supercell)
 * whose matrices an orthogonal change of basis inside every degenerate block brings to 1 x 1 / 2 x 2
 * blocks, the ensemble is stored in that basis (inputs and outputs of the averages and of their VJP
 * stay in the given basis) and the mixed-precision averages run their dense symmetry transform /
 * fold over the cosets of K only.  rotated: 1 when the basis is rotated; n_cosets, coset_size: the
 * factorisation (0 when the general path is used); offpattern: the largest matrix entry outside the
 * 2 x 2 pattern over the whole group (at most 1e-7 for the factorised path).
 * TDSCHA_SYM_COSETS=0 in the environment at creation keeps the given basis and the general path.
 * Any pointer may be NULL.
 */
int tdscha_ensemble_cosets(const tdscha_ensemble *ens, int *rotated, int *n_cosets, int *coset_size,
                           double *offpattern);

/*
 * The analysis behind it, on host arrays (no device): sym_blocks as for tdscha_ensemble_create.
 * Outputs n_cosets, coset_size (0 when the group has no such structure; tdscha_last_error says
 * why) and, when non-NULL: order (N_sym) the symmetries coset by coset, partner (n) the partner of
 * each rotated mode (itself for a real character), R (sum of n_deg[b]^2) the rotation of every block,
 * R_b[q'][q] = component q' of rotated mode q, row-major; offpattern the largest entry of
 * R^T S_t R outside the pattern over the subgroup's matrices.
 */
int tdscha_symmetry_cosets(int N_sym, int n_blocks, const int *n_deg, const double *const *sym_blocks,
                           int *n_cosets, int *coset_size, int *order, int *partner, double *R,
                           double *offpattern);

/*
 * Character classes of the factorised path (no counterpart in the reference: its averaging loop runs
 * over every symmetry).  On the factorised path the subgroup K is abelian, so every component of a
 * symmetric matrix in the rotated basis is multiplied by a character of K under its matrices; the
 * averages' two big contractions then run class by class over only that class's components, in
 * every precision (TDSCHA_SYM_FREQ=0 at creation keeps the contractions over every symmetry row).
 * n_class: classes in use (0 when the path is off); Kq / Kmq: padded pair / mode columns;
 * flops_ratio: the class contractions' work relative to the same contractions over all symmetries
 * and all pairs.  Any pointer may be NULL.
 */
int tdscha_ensemble_classes(const tdscha_ensemble *ens, int *n_class, int *Kq, int *Kmq, double *flops_ratio);

/*
 * The tables behind it, on host arrays (no device), for tests: sizes[4] = {n_class, Kq, Kmq, P}
 * always; when cls is non-NULL also
 *   cls (n_class x 5): real, pair-column offset, count, mode-column offset, count;
 *   pcol_i (Kq x 5): mu0, nu0, mu1, nu1, partner;  pcol_d (Kq x 5): c0, c1, re, im, zc
 *     (own value of a pair column on a symmetric matrix M: c0 M[mu0,nu0] + c1 M[mu1,nu1]; left
 *     rows Re = re own(c), Im = im own(partner); outputs own(c) = O1[c] + zc O2[partner]);
 *   pp_i (P x 2), pp_d (P x 2): entry (mu <= nu) of N from the outputs' own values;
 *   mcol_i (Kmq x 2): mode, partner;  mcol_d (Kmq x 4): sign, re, im, zc;  mode_col (n).
 * Returns sizes[0] = 0 when the group has no such structure.
 */
int tdscha_symmetry_classes(int N_sym, int n_blocks, const int *n_deg, const double *const *sym_blocks,
                            int *sizes, double *flops_ratio, int *cls, int *pcol_i, double *pcol_d, int *pp_i,
                            double *pp_d, int *mcol_i, double *mcol_d, int *mode_col);

/* Device bytes the ensemble holds now (operands of every precision built so far included). */
int tdscha_ensemble_device_bytes(const tdscha_ensemble *ens, long long *bytes);

/*
 * Symmetrised perturbed averages on host buffers: f_out (n), d2v_out (n, n) C order, exactly the
 * outputs of GetPerturbAverageSym (d2v overwritten, D4 part added when apply_d4 = 1).
 * Only the symmetric part of Y1 enters the reference's formulas; Y1 may be non-symmetric.
 */
int tdscha_perturb_average_sym(tdscha_ensemble *ens, const double *R1, const double *Y1, int apply_d4,
                               int precision, double *f_out, double *d2v_out);

/* Batched, device-resident: nb perturbations R1 (nb, n), Y1 (nb, n, n) -> f (nb, n), d2v (nb, n, n). */
int tdscha_perturb_average_sym_device(tdscha_ensemble *ens, int nb, const double *R1, const double *Y1,
                                      int apply_d4, int precision, double *f_out, double *d2v_out,
                                      void *stream);

/*
 * One-shot drop-in with the argument list of sscha_HP_odd.GetPerturbAverageSym
 * (odd_corr_module.c:519-520), FP64: uploads, computes, downloads, frees.
 */
int tdscha_GetPerturbAverageSym(const double *X, const double *Y, const double *w, const double *rho,
                                const double *R1, const double *Y1, double T, int apply_D4, int N_syms,
                                int n_blocks, const double *const *sym_list, const int *n_deg,
                                const int *const *deg_space_list, const int *blocks_ids, int N_configs,
                                int N_modes, double *f_out, double *d2v_out);

/* Flags of Lanczos.apply_full_L (DynamicalLanczos.py:241-271, 494). */
typedef struct tdscha_apply_opts {
    int use_wigner;       /* Wigner representation (a', b') instead of (Upsilon, ReA)         */
    int ignore_harmonic;  /* drop L1                                                          */
    int ignore_v3;        /* drop the whole anharmonic part (Python semantics, :3532)          */
    int ignore_v4;        /* drop the D4 part of the averages                                  */
    int reverse_L;        /* output *= -1                                                      */
    double shift_value;   /* output += shift_value * psi                                       */
} tdscha_apply_opts;

/*
 * apply_full_L on nb device vectors psi (nb, n + n(n+1)) -> out (nb, n + n(n+1)).
 * transpose (nb ints, host) selects L or L^T per vector; opts may be NULL (all defaults).
 */
int tdscha_apply_full_L_device(tdscha_ensemble *ens, int nb, const double *psi, const int *transpose,
                               const tdscha_apply_opts *opts, int precision, double *out, void *stream);

/*
 * The two halves of apply_full_L around the averages (Modules/DynamicalLanczos.py:2936-2993 and
 * :3195-3281 / 2227-2385), for a caller that computes the averages of configuration slices on
 * several devices and reduces them (the reference's MPI_Allreduce, CModules/LanczosFunctions.c:2237,
 * 2417, 2731):
 *   prologue: psi (nb, len) -> R1 (nb, n), Y1 (nb, n, n)  (unpacking, transpose mixing, Wigner alpha)
 *   epilogue: psi, f_av (nb, n), d2v_av (nb, n, n) -> out (nb, len)  (L1, packing, signs, reverse, shift)
 * prologue -> tdscha_perturb_average_sym_device -> epilogue equals tdscha_apply_full_L_device.
 */
int tdscha_apply_prologue_device(tdscha_ensemble *ens, int nb, const double *psi, const int *transpose,
                                 const tdscha_apply_opts *opts, double *R1_out, double *Y1_out, void *stream);
int tdscha_apply_epilogue_device(tdscha_ensemble *ens, int nb, const double *psi, const int *transpose,
                                 const tdscha_apply_opts *opts, const double *f_av, const double *d2v_av,
                                 double *out, void *stream);

/*
 * One bi-conjugate Lanczos step (DynamicalLanczos.py:6059-6153, n_rep_orth = 0) for nc chains,
 * all FP64 on the device.  Per chain c the arrays hold vectors of length len:
 *   Lq, pL        L q_k and L^T p_k;   q, p   current q_k, p_k;   q_prev, p_prev   q_{k-1}, p_{k-1}
 *   sc_in  (nc, 6) : [c_{k-1}, b_{k-1}, s_norm_k, s_norm_{k-1}, c_{k-2}, step_k]  (step 0 ignores the
 *                    history terms exactly as the reference's len(basis) checks do)
 *   mask   optional (len) scalar-product weights (mask_dot_wigner, run_simm), NULL otherwise
 * Outputs: q_next, p_next (nc, len) and sc_out (nc, 4) = [a_k, b_k, c_k, s_norm_{k+1}].
 */
int tdscha_lanczos_step_device(int nc, long long len, const double *Lq, const double *pL,
                               const double *q, const double *p, const double *q_prev,
                               const double *p_prev, const double *sc_in, const double *mask,
                               double *q_next, double *p_next, double *sc_out, void *stream);

/*
 * tdscha_lanczos_step_device with no device allocation at all.  There is no counterpart in the
 * reference.  It is meant for host programs that cannot call cudaMalloc while they drive the
 * recurrence: applications that hand out all device memory from their own fixed arena, code that
 * must not add an implicit device synchronisation (cudaMalloc/cudaFree synchronise), and real-time
 * or embedded runners with a fixed memory budget.  The step's reduction partials live instead in a
 * fixed array inside this library (4 doubles per chain per reduction block, 303 KB), which every GPU
 * that loads the library holds until the process exits.
 *   - nc must be at most 32; larger requests fail with TDSCHA_EINVAL and a message.
 *   - Runs on the current device.  The first call on each device looks up the array's device
 *     address (cudaGetSymbolAddress), and so does the first call after that device's context
 *     changed (e.g. after cudaDeviceReset); make such a call before any stream capture.
 *   - All calls share the one array: calls that overlap on the GPU (e.g. on different streams)
 *     race and give wrong results.  Each call writes every partial it reads, so no clearing is
 *     needed between calls.
 *   - Arguments, outputs and errors are those of tdscha_lanczos_step_device.
 */
int tdscha_lanczos_step_device_noalloc(int nc, long long len, const double *Lq, const double *pL,
                                       const double *q, const double *p, const double *q_prev,
                                       const double *p_prev, const double *sc_in, const double *mask,
                                       double *q_next, double *p_next, double *sc_out, void *stream);

/*
 * The static (zero-frequency) L operator of the free-energy Hessian on nb static vectors
 * psi (nb, n + n(n+1)/2) = (R, Upsilon packed upper row-major), FP64 device arrays:
 *   tdscha_apply_L1_static_device  Lanczos.apply_L1_static(psi, inverse, power)
 *                                  (Modules/DynamicalLanczos.py:2502-2565) with the exponent
 *                                  already signed: power = -p for inverse = True
 *   tdscha_apply_static_L_device   apply_anharmonic_static() (:3287-3354), plus apply_L1_static(psi)
 *                                  when include_L1: the matvec of run_hessian_calculation
 *                                  (:3973-4235) and of StaticHessian.apply_L
 *                                  (Modules/StaticHessian.py:561-623); nb <= 64; averages in
 *                                  `precision`, D4 term unless ignore_v4
 */
int tdscha_apply_L1_static_device(tdscha_ensemble *ens, int nb, const double *psi, double power, double *out,
                                  void *stream);
int tdscha_apply_static_L_device(tdscha_ensemble *ens, int nb, const double *psi, int ignore_v4, int include_L1,
                                 int precision, double *out, void *stream);

/*
 * Many bi-conjugate steps of many chains over several systems, without returning to the host:
 * the step loop of Lanczos.run_FT (Modules/DynamicalLanczos.py:5843-6374, n_rep_orth = 0) for
 * every chain of every system, advanced in lockstep.  The reference runs one chain per call; this
 * entry point has no single counterpart (run_FT per chain is the reference-side equivalent).
 *
 * Per system (one resident ensemble, nc = n_chains <= 32 chains, len = n + n(n+1)):
 *   qp    device (4, nc, len): q_k, p_k, q_{k-1}, p_{k-1} of every chain (in, advanced in place)
 *   sc    device (nc, 6): the recurrence history of tdscha_lanczos_step_device's sc_in (in/out)
 *   coef  device (n_steps, nc, 4): [a_k, b_k, c_k, s_norm_{k+1}] of every step (out)
 * Each step is one batched apply of the 2 nc vectors [q; p] (transpose 0 for q, 1 for p), one
 * batched recurrence and the history update.  Systems run on their own streams forked from and
 * joined into `stream`.  With use_graph != 0 the first two steps run eagerly and every remaining
 * step of all systems is captured into one CUDA graph, launched once.  A chain whose |b| or
 * |c| falls below 1e-12 ends there as in run_FT (:6129-6141): its last coef row is that step's,
 * later rows are left untouched, its qp and sc stay at that step (its vectors still go through
 * the batched apply, whose other chains are unaffected).  Returns after the last step completed.
 */
typedef struct tdscha_run_system {
    tdscha_ensemble *ens;
    int n_chains;
    double *qp;
    double *sc;
    double *coef;
    tdscha_apply_opts opts;
    int precision;
} tdscha_run_system;

int tdscha_lanczos_run_device(int n_systems, const tdscha_run_system *systems, int n_steps, int use_graph,
                              void *stream);

/*
 * Continued-fraction Green function (DynamicalLanczos.py:4951-5047) on the device.
 * a (n_iter), b (n_iter-1 or more), c (same as b or NULL = symmetric) FP64 device arrays;
 * omega (n_w) device; gf_out (2 * n_w) interleaved re, im.
 */
int tdscha_continued_fraction_device(int n_iter, const double *a, const double *b, const double *c,
                                     int n_b, int n_c, int n_w, const double *omega, int use_terminator,
                                     int last_average, double smearing, int use_wigner, int reverse_L,
                                     double shift_value, double perturbation_modulus, double *gf_out,
                                     void *stream);

/*
 * Profiling hooks (no counterpart in the reference, whose only timers are wall clocks printed per
 * apply, DynamicalLanczos.py:3521-3551).  When enabled, every averages call records CUDA events on
 * its launching stream around each stage.  tdscha_read_profile synchronises, returns the summed
 * milliseconds and the launch counts of the n_stages stages (0 transform, 1 contraction [a|b],
 * 2 contraction [c|d], 3 weights, 4 contraction Z, 5 contraction F, 6 fold, 7 other, 8 the
 * operand rebuilds of configuration-chunked ensembles) since the last read, and resets them.
 * Launch counts are kept even with profiling disabled.
 */
int tdscha_set_profiling(tdscha_ensemble *ens, int enable);
int tdscha_read_profile(tdscha_ensemble *ens, double *ms, long long *launches, int n_stages);

/*
 * The tensor-core contraction used by the averages, exposed for testing and reuse (no counterpart
 * in the reference): D (M x N, fp32, row-major, leading dimension ldd) = A (M x K) . B (N x K)^T
 * on device operands stored row-major with K contiguous.  precision TF32 / TF32X3: fp32 elements
 * already rounded to tf32; BF16 / BF16X3: bf16 elements; the X3 modes also read A_lo / B_lo and
 * accumulate hi.hi + hi.lo + lo.hi.  K must be a multiple of 64 (bf16) or 32 (tf32); lda / ldb in
 * elements with 16-byte aligned rows.
 */
int tdscha_tc_contract(int precision, int M, int N, int K, const void *A_hi, const void *A_lo, long long lda,
                       const void *B_hi, const void *B_lo, long long ldb, float *D, long long ldd, void *stream);

/*
 * Failure detection of the tensor-core kernels (no counterpart in the reference, whose kernels have
 * no waits).  Every pipeline wait inside the tcgen05 contraction is bounded; when one runs out the
 * kernel stops its CTA cleanly (its copies in flight drained, its MMAs retired, its tensor memory
 * freed) and the call returns TDSCHA_ETIMEOUT, after which the library stays usable.
 *   tdscha_set_wait_budget               budget of each wait of later launches, seconds in
 *                                        [1e-6, 60] (default 4); process-wide
 *   tdscha_debug_stall_next_contraction  the next contraction launch issues no operand copy, so that
 *                                        its first wait can only end by running out (tests of the
 *                                        abort path); one-shot, process-wide
 *   tdscha_set_error_check               per_call = 1 (default): every device entry point that runs
 *                                        tensor-core kernels reads the ensemble's error word when its
 *                                        work is done (one stream synchronisation per call);
 *                                        per_call = 0: the calls return as soon as their work is
 *                                        queued and the error word keeps every expiry until
 *                                        tdscha_check_errors reads it; process-wide
 *   tdscha_check_errors                  waits for `stream`, returns TDSCHA_ETIMEOUT (and clears the
 *                                        word) when a wait of an earlier call on this ensemble ran out
 */
int tdscha_set_wait_budget(double seconds);
int tdscha_debug_stall_next_contraction(void);
int tdscha_set_error_check(int per_call);
int tdscha_check_errors(tdscha_ensemble *ens, void *stream);

/*
 * Vector-Jacobian product of the averages (the outputs of tdscha_perturb_average_sym_device)
 * with respect to the ensemble's forces Y and weights rho -- the building block of dG(w)/dY,
 * dG(w)/drho (the reference has no derivatives; no counterpart there).  For nb perturbations
 * (R1 (nb, n), Ys (nb, n, n) symmetric, device) and cotangents fbar (nb, n), Dbar (nb, n, n)
 * symmetric (device) it writes, summed over the nb vectors,
 *   Ybar (N, n)  = d[ sum_k <fbar_k, f_k> + <Dbar_k, D_k>_F ] / dY,   rhobar (N) = the same / drho
 * (device buffers, overwritten).  FP64 throughout; N_eff = sum(rho) is differentiated too.
 */
int tdscha_perturb_average_vjp_device(tdscha_ensemble *ens, int nb, const double *R1, const double *Ys, int apply_d4,
                                      const double *fbar, const double *Dbar, double *Ybar, double *rhobar,
                                      void *stream);

/*
 * The same vector-Jacobian product with its eight ensemble contractions (four like the averages'
 * [a|b], [c|d] and four transposed ones over the symmetry rows) in `precision`: TDSCHA_PREC_FP64 is
 * tdscha_perturb_average_vjp_device; the mixed modes run them on the tcgen05 contraction kernel in
 * that storage format, the cotangent algebra and the reductions staying FP64.  No counterpart in
 * the reference.
 */
int tdscha_perturb_average_vjp_precision_device(tdscha_ensemble *ens, int nb, const double *R1, const double *Ys,
                                                int apply_d4, int precision, const double *fbar, const double *Dbar,
                                                double *Ybar, double *rhobar, void *stream);

/*
 * Inputs of the Lanczos from an ensemble, computed on the GPU (host buffers in and out).
 *
 * tdscha_project_ensemble: X = (u o sqrt(m)) . pols and Y = (f / sqrt(m)) . pols, the
 * mass-rescaled displacements and forces in the polarisation basis -- the projection at
 * Modules/DynamicalLanczos.py:431-435 (u in Bohr, f in Ry/Bohr after the reference's subtraction
 * of the SSCHA and mean forces, :389-425).  u, f (N, 3 nat); masses (3 nat); pols (3 nat, n);
 * X_out, Y_out (N, n); all C order, FP64.
 *
 * tdscha_symmetries_on_modes: the symmetry group on the degenerate blocks of the modes,
 * S_b^j = E_b^T P_j E_b (N_sym, d_b, d_b) per block, with (P_j v)[perm_j(a)] = R_j v[a] on
 * mass-weighted displacements.  This replaces the tables that DynamicalLanczos.py:749-756
 * takes from cellconstructor's GetSymmetriesOnModesDeg.  perm (N_sym, nat) image atoms, rot
 * (N_sym, 3, 3) Cartesian rotations, pols (3 nat, n); blocks of at most 80 modes.
 */
int tdscha_project_ensemble(const double *u, const double *f, const double *masses, const double *pols, int N,
                            int nat3, int n, double *X_out, double *Y_out);
int tdscha_symmetries_on_modes(const double *pols, int nat, int n, int N_sym, const int *perm, const double *rot,
                               int n_blocks, const int *n_deg, const int *const *deg_space, double *const *sym_out);

#ifdef __cplusplus
}
#endif
#endif /* TDSCHA_B200_H */
