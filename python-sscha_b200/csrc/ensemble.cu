// ensemble.cu -- resident ensemble, operand builders, symmetry transform/fold kernels and the
// orchestration of the symmetrised perturbed averages (the algebra is in ensemble.cuh).
#include <cublas_v2.h>
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "ensemble.cuh"
#include "symmetry.cuh"
#include "tc_gemm.cuh"

namespace tdscha {


// ------------------------------------------------------------------------------------------------
// operand builders (once per ensemble and storage format)
// ------------------------------------------------------------------------------------------------
// V (2N x Kp): rows < N -> c_p x_mu x_nu ; rows >= N -> x_mu g_nu + x_nu g_mu (x g on the diagonal).
// One CTA row per operand row (blockIdx.y strides over rows), threads over the packed pairs p: the
// pair tables are read coalesced and x, g come from one row of X / G (L1).
__global__ void build_V_kernel(const double *__restrict__ X, const double *__restrict__ G,
                               const int *__restrict__ pmu, const int *__restrict__ pnu, int N, int n,
                               long long P, long long Kp, Format fmt, void *hi, void *lo) {
    for (long long k = blockIdx.y; k < 2LL * N; k += gridDim.y) {
        const bool second = k >= N;
        const double *x = X + (second ? k - N : k) * n;
        const double *g = G + (second ? k - N : k) * n;
        for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < Kp; p += (long long)gridDim.x * blockDim.x) {
            double v = 0.0;
            if (p < P) {
                const int mu = pmu[p], nu = pnu[p];
                if (!second) v = (mu == nu ? 1.0 : 2.0) * x[mu] * x[nu];
                else v = (mu == nu) ? x[mu] * g[mu] : x[mu] * g[nu] + x[nu] * g[mu];
            }
            store_split(fmt, hi, lo, k * Kp + p, v);
        }
    }
}

// VT (P x N2p) = V^T with zero columns beyond 2N, from the transposed ensemble XGT = [X^T ; G^T]
// (2n x ldT, configuration-contiguous): one CTA row per pair p, threads over configurations, so
// every read and write is coalesced.
__global__ void build_VT_kernel(const double *__restrict__ XGT, long long ldT, const int *__restrict__ pmu,
                                const int *__restrict__ pnu, int N, int n, long long P, long long N2p, Format fmt, void *hi,
                                void *lo) {
    for (long long p = blockIdx.y; p < P; p += gridDim.y) {
        const int mu = pmu[p], nu = pnu[p];
        const double *xm = XGT + (long long)mu * ldT, *xn = XGT + (long long)nu * ldT;
        const double *gm = XGT + (long long)(n + mu) * ldT, *gn = XGT + (long long)(n + nu) * ldT;
        const double c = mu == nu ? 1.0 : 2.0;
        for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < N2p; k += (long long)gridDim.x * blockDim.x) {
            double v = 0.0;
            if (k < N) {
                v = c * xm[k] * xn[k];
            } else if (k < 2LL * N) {
                const long long i = k - N;
                v = (mu == nu) ? xm[i] * gm[i] : xm[i] * gn[i] + xn[i] * gm[i];
            }
            store_split(fmt, hi, lo, p * N2p + k, v);
        }
    }
}

// XGT (2n x N) = [X^T ; G^T], tiled transpose through shared memory
__global__ void transpose_XG_kernel(const double *__restrict__ X, const double *__restrict__ G, int N, int n,
                                    double *__restrict__ XGT) {
    __shared__ double tile[32][33];
    const int which = blockIdx.z;                       // 0: X, 1: G
    const double *src = which ? G : X;
    const int i0 = blockIdx.y * 32, m0 = blockIdx.x * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = i0 + r, m = m0 + threadIdx.x;
        tile[r][threadIdx.x] = (i < N && m < n) ? src[(long long)i * n + m] : 0.0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int m = m0 + r, i = i0 + threadIdx.x;
        if (m < n && i < N) XGT[((long long)which * n + m) * N + i] = tile[threadIdx.x][r];
    }
}

// grid of the row-wise builders: x over a row's columns (256 threads a CTA), y over rows
static dim3 rows_grid(long long cols, long long rows) {
    const long long gx = std::min<long long>(ceil_div(cols, 256), 64);
    const long long gy = std::min<long long>(std::max<long long>(rows, 1), 65535);
    return dim3((unsigned)std::max<long long>(gx, 1), (unsigned)gy);
}

// XG (2N x np) = [X ; G] ; YXt (n x N2p) = [Y^T | X~^T]
__global__ void build_XG_kernel(const double *X, const double *G, int N, int n, long long np, Format fmt, void *hi, void *lo) {
    const long long total = 2LL * N * np;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long k = idx / np, m = idx % np;
        double v = 0.0;
        if (m < n) v = (k < N) ? X[k * n + m] : G[(k - N) * n + m];
        store_split(fmt, hi, lo, idx, v);
    }
}
__global__ void build_YXt_kernel(const double *Y, const double *Xt, int N, int n, long long N2p, Format fmt, void *hi, void *lo) {
    const long long total = (long long)n * N2p;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long m = idx / N2p, k = idx % N2p;
        double v = 0.0;
        if (k < N) v = Y[k * n + m];
        else if (k < 2LL * N) v = Xt[(k - N) * n + m];
        store_split(fmt, hi, lo, idx, v);
    }
}

__global__ void thermal_kernel(const double *w, int n, double T, double *ups, double *psi) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    double nb = T > 0 ? 1.0 / (exp(w[m] * RY_TO_K / T) - 1.0) : 0.0;
    ups[m] = 2.0 * w[m] / (1.0 + 2.0 * nb);
    psi[m] = (1.0 + 2.0 * nb) / (2.0 * w[m]);
}

// (N_sym, d, d) fp64 table -> (N_sym, dp, dp) fp32 zero-padded copies, as given and transposed
__global__ void pad_sym_kernel(const double *S, int N_sym, int d, int dp, float *P, float *PT) {
    const long long total = (long long)N_sym * dp * dp;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long j = idx / ((long long)dp * dp);
        const int e = (int)(idx % ((long long)dp * dp)), p = e / dp, q = e % dp;
        const bool in = p < d && q < d;
        P[idx] = in ? (float)S[(j * d + p) * d + q] : 0.f;
        PT[idx] = in ? (float)S[(j * d + q) * d + p] : 0.f;
    }
}

__global__ void scale_rows_kernel(const double *A, const double *s, int N, int n, double *out) {
    long long total = (long long)N * n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x)
        out[idx] = A[idx] * s[idx % n];
}

__global__ void symmetrize_kernel(int nb, int n, const double *Y, double *Ys) {
    long long total = (long long)nb * n * n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        long long k = idx / ((long long)n * n), e = idx % ((long long)n * n);
        int r = (int)(e / n), c = (int)(e % n);
        const double *Yk = Y + k * n * n;
        Ys[idx] = 0.5 * (Yk[(long long)r * n + c] + Yk[(long long)c * n + r]);
    }
}

// ------------------------------------------------------------------------------------------------
// weights: from [a | b] (D1) and [c | d] (Dcd) build Cw = [delta/2 | gamma] and AB = [alpha | beta]
// ------------------------------------------------------------------------------------------------
template <typename AccT>
__global__ void weights_kernel(const AccT *__restrict__ D1, const AccT *__restrict__ Dcd, long long ld, const double *__restrict__ rho,
                               int N, int M, long long N2p, int d4, Format fmt, void *Cw_hi, void *Cw_lo, void *AB_hi,
                               void *AB_lo) {
    const long long per_row = N + (N2p - 2LL * N);
    const long long total = (long long)M * per_row;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long r = idx / per_row, i = idx % per_row;
        if (i < N) {
            const double a = (double)D1[r * ld + i], b = (double)D1[r * ld + N + i];
            const double c = (double)Dcd[r * ld + i], d = (double)Dcd[r * ld + N + i];
            const double rh = rho[i];
            const double gam = rh * (-c / 3.0 + (d4 ? a / 8.0 : 0.0));
            const double del = rh * (-d / 3.0 + (d4 ? b / 4.0 : 0.0));
            store_split(fmt, Cw_hi, Cw_lo, r * N2p + i, 0.5 * del);
            store_split(fmt, Cw_hi, Cw_lo, r * N2p + N + i, gam);
            store_split(fmt, AB_hi, AB_lo, r * N2p + i, -rh * a / 6.0);
            store_split(fmt, AB_hi, AB_lo, r * N2p + N + i, -rh * b / 3.0);
        } else {
            const long long col = 2LL * N + (i - N);
            store_split(fmt, Cw_hi, Cw_lo, r * N2p + col, 0.0);
            store_split(fmt, AB_hi, AB_lo, r * N2p + col, 0.0);
        }
    }
}

__global__ void fold_reduce_kernel(const double *partD, const double *partF, int nf, int n, int nb,
                                   const int *blocks_ids, double norm, double *D_out, double *f_out) {
    const long long nn = (long long)n * n;
    const long long total = (long long)nb * nn;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long k = idx / nn, e = idx % nn;
        int mu = (int)(e / n), nu = (int)(e % n);
        if (blocks_ids[mu] > blocks_ids[nu]) { int s = mu; mu = nu; nu = s; }
        const double *src = partD + k * nf * nn + (long long)mu * n + nu;
        double s = 0.0;
        for (int f = 0; f < nf; ++f) s += src[f * nn];
        D_out[idx] = s * norm;
    }
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < (long long)nb * n;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long k = idx / n, m = idx % n;
        double s = 0.0;
        for (int f = 0; f < nf; ++f) s += partF[(k * nf + f) * n + m];
        f_out[idx] = s * norm;
    }
}

// ------------------------------------------------------------------------------------------------
// host orchestration
// ------------------------------------------------------------------------------------------------
void Profile::begin(int stage, cudaStream_t st, ProfRec *r) {
    r->stage = stage;
    r->a = r->b = nullptr;
    if (!enabled) return;
    cudaEventCreate(&r->a);
    cudaEventCreate(&r->b);
    cudaEventRecord(r->a, st);
}
void Profile::end(ProfRec *r, cudaStream_t st) {
    if (!enabled || !r->a) return;
    cudaEventRecord(r->b, st);
    recs.push_back(*r);
}

// Profile one stage: records CUDA events around the launches on the launching stream when enabled,
// counts launches always.
struct StageScope {
    tdscha_ensemble *e;
    cudaStream_t st;
    ProfRec r;
    StageScope(tdscha_ensemble *e_, int stage, cudaStream_t st_, int n_launch = 1) : e(e_), st(st_) {
        e->prof.launches[stage] += n_launch;
        e->prof.begin(stage, st, &r);
    }
    ~StageScope() { e->prof.end(&r, st); }
};

static int grid_for(long long total, int threads = 256) {
    long long g = (total + threads - 1) / threads;
    return (int)std::min<long long>(std::max<long long>(g, 1), 148LL * 32);
}

static int dev_alloc(void **p, size_t bytes, size_t *acc) {
    TD_CUDA(cudaMalloc(p, bytes));
    if (acc) *acc += bytes;
    return 0;
}

int symmetrize_device(int nb, int n, const double *Y, double *Ys, cudaStream_t st) {
    symmetrize_kernel<<<grid_for((long long)nb * n * n), 256, 0, st>>>(nb, n, Y, Ys);
    TD_CUDA(cudaGetLastError());
    return 0;
}

static void free_cosets(SymCosets *c) {
    if (!c) return;
    void *ps[] = {c->order, c->partner, c->c0, c->c1, c->repP, c->repPT, c->d_offRep, c->repS, c->d_offRepS};
    for (void *p : ps)
        if (p) cudaFree(p);
    delete c;
}

// TDSCHA_SYM_COSETS=0 keeps the ensemble in the given basis and the averages on the general
// symmetry kernels (read when an ensemble is created, and again by every averages call).
static bool cosets_enabled() {
    const char *env = getenv("TDSCHA_SYM_COSETS");
    return !(env && atoi(env) == 0);
}

// TDSCHA_SYM_FREQ=0 keeps the coset path's contractions over every symmetry row instead of the
// character classes of freq.cuh (read when an ensemble is created, and again by every averages call).
static bool freq_enabled() {
    const char *env = getenv("TDSCHA_SYM_FREQ");
    return !(env && atoi(env) == 0);
}

// Rotated basis and factorised symmetry path (cosets.cuh) when the symmetry group has the structure;
// on the legacy stream, before the fp32 tables, G and X~ are derived from X, Y and the tables.
static int setup_cosets(tdscha_ensemble *e, const std::vector<int> &dim, const double *const *sym_blocks) {
    CosetAnalysis ca;
    TD_TRY(analyse_cosets(e->N_sym, dim, sym_blocks, ca));
    if (!ca.ok) return 0;
    const int n = e->n, dmax = e->dmax, nblk = e->n_blocks;
    std::vector<double> Rrow((size_t)n * dmax, 0.0);
    for (int b = 0; b < nblk; ++b)
        for (int q = 0; q < dim[b]; ++q)
            for (int r = 0; r < dim[b]; ++r)
                Rrow[(size_t)(e->blk_start[b] + q) * dmax + r] = ca.R[ca.R_off[b] + (size_t)q * dim[b] + r];
    double *Rblk = nullptr;
    TD_CUDA(cudaMalloc(&e->Rrow, Rrow.size() * sizeof(double)));
    TD_CUDA(cudaMemcpy(e->Rrow, Rrow.data(), Rrow.size() * sizeof(double), cudaMemcpyHostToDevice));
    TD_CUDA(cudaMalloc(&Rblk, ca.R.size() * sizeof(double)));
    TD_CUDA(cudaMemcpy(Rblk, ca.R.data(), ca.R.size() * sizeof(double), cudaMemcpyHostToDevice));
    // X, Y into the rotated basis (G is free scratch until it is derived from Y)
    TD_TRY(rotate_rows_of(e->N, n, dmax, e->Rrow, e->d_blocks_ids, e->d_blk_start, e->d_blk_dim, e->X, e->G, true, 0));
    std::swap(e->X, e->G);
    TD_TRY(rotate_rows_of(e->N, n, dmax, e->Rrow, e->d_blocks_ids, e->d_blk_start, e->d_blk_dim, e->Y, e->G, true, 0));
    std::swap(e->Y, e->G);
    for (int b = 0; b < nblk; ++b)
        TD_TRY(rotate_sym_tables(e->sym + e->blk_sym_off[b], e->N_sym, dim[b], Rblk + ca.R_off[b], 0));
    TD_CUDA(cudaDeviceSynchronize());
    cudaFree(Rblk);
    // coefficients of every symmetry, checked against the 2 x 2 pattern over the whole group
    auto *c = new SymCosets();
    c->n_cos = ca.n_cos;
    c->sub = ca.sub;
    auto fail = [&](int rc) { free_cosets(c); return rc; };
    unsigned long long *offmax = nullptr;
    const size_t cb = (size_t)e->N_sym * n * sizeof(float);
    if (cudaMalloc(&c->order, e->N_sym * sizeof(int)) != cudaSuccess || cudaMalloc(&c->partner, n * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&c->c0, cb) != cudaSuccess || cudaMalloc(&c->c1, cb) != cudaSuccess ||
        cudaMalloc(&offmax, sizeof(unsigned long long)) != cudaSuccess) {
        if (offmax) cudaFree(offmax);
        set_error("allocation of the symmetry cosets failed");
        return fail(TDSCHA_ENOMEM);
    }
    cudaMemcpy(c->order, ca.order.data(), e->N_sym * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(c->partner, ca.partner.data(), n * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemset(offmax, 0, sizeof(unsigned long long));
    int rc = coset_coefficients(e->N_sym, n, ca.sub, c->order, c->partner, e->d_blocks_ids, e->d_blk_start, e->d_blk_dim, e->sym,
                                e->d_blk_sym_off, c->c0, c->c1, offmax, 0);
    unsigned long long bits = 0;
    if (!rc && cudaMemcpy(&bits, offmax, sizeof(bits), cudaMemcpyDeviceToHost) != cudaSuccess) rc = TDSCHA_ECUDA;
    cudaFree(offmax);
    if (rc) return fail(rc);
    std::memcpy(&c->offpattern, &bits, sizeof(double));
    if (!(c->offpattern <= 1e-7)) { free_cosets(c); return 0; }   // not a factorisation to working accuracy
    // the representatives' tables in the padded fp32 layouts of the tensor-core kernels
    std::vector<long long> offR(nblk), offS(nblk);
    long long tot = 0, totd = 0;
    for (int b = 0; b < nblk; ++b) {
        const long long dp = (dim[b] + 3) & ~3;
        offR[b] = tot;
        tot += (long long)ca.n_cos * dp * dp;
        offS[b] = totd;
        totd += (long long)ca.n_cos * dim[b] * dim[b];
    }
    if (cudaMalloc(&c->repP, tot * sizeof(float)) != cudaSuccess || cudaMalloc(&c->repPT, tot * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&c->d_offRep, nblk * sizeof(long long)) != cudaSuccess ||
        cudaMalloc(&c->repS, totd * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->d_offRepS, nblk * sizeof(long long)) != cudaSuccess) {
        set_error("allocation of the coset tables failed");
        return fail(TDSCHA_ENOMEM);
    }
    cudaMemcpy(c->d_offRep, offR.data(), nblk * sizeof(long long), cudaMemcpyHostToDevice);
    cudaMemcpy(c->d_offRepS, offS.data(), nblk * sizeof(long long), cudaMemcpyHostToDevice);
    for (int b = 0; b < nblk; ++b) {
        // the representatives' FP64 tables (rotated basis), then their padded fp32 copies
        const size_t blk = (size_t)dim[b] * dim[b];
        double *reps = c->repS + offS[b];
        for (int p = 0; p < ca.n_cos; ++p)
            cudaMemcpy(reps + p * blk, e->sym + e->blk_sym_off[b] + (size_t)ca.order[(size_t)p * ca.sub] * blk, blk * sizeof(double),
                       cudaMemcpyDeviceToDevice);
        const long long dp = (dim[b] + 3) & ~3;
        pad_sym_kernel<<<grid_for((long long)ca.n_cos * dp * dp), 256>>>(reps, ca.n_cos, dim[b], (int)dp, c->repP + offR[b],
                                                                         c->repPT + offR[b]);
        if (cudaDeviceSynchronize() != cudaSuccess) {
            set_error("coset tables: %s", cudaGetErrorString(cudaGetLastError()));
            return fail(TDSCHA_ECUDA);
        }
    }
    e->cosets = c;
    // character classes of the subgroup: the big contractions class by class (freq.cuh)
    if (freq_enabled()) {
        FreqLayout fl;
        TD_TRY(build_freq_layout(n, dim, e->blk_start, sym_blocks, ca, fl));
        if (fl.ok) TD_TRY(freq_tables_create(fl, &e->freq));
    }
    return 0;
}

int ensemble_create(const double *X, const double *Y, const double *w, const double *rho, int N, int n, double T,
                    int N_sym, int n_blocks, const int *n_deg, const int *const *deg_space,
                    const double *const *sym_blocks, const int *blocks_ids, tdscha_ensemble **out) {
    TD_CHECK(out != nullptr, TDSCHA_EINVAL, "out handle pointer is NULL");
    *out = nullptr;
    TD_CHECK(X && Y && w && rho && n_deg && deg_space && sym_blocks && blocks_ids, TDSCHA_EINVAL, "NULL input array");
    TD_CHECK(N > 0 && n > 0 && N_sym > 0 && n_blocks > 0 && n_blocks <= n, TDSCHA_EINVAL,
             "bad sizes N=%d n=%d N_sym=%d n_blocks=%d", N, n, N_sym, n_blocks);
    int dev = 0;
    TD_CUDA(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    TD_CUDA(cudaGetDeviceProperties(&prop, dev));
    TD_CHECK(prop.major == 10, TDSCHA_ENOSUPPORT, "device %d is sm_%d%d; this library is built for sm_100a", dev, prop.major, prop.minor);

    // validate the block structure (contiguous, ascending, covering 0..n-1 in order) and degeneracy
    std::vector<int> start(n_blocks), dim(n_blocks);
    int expect = 0, dmax = 0;
    for (int b = 0; b < n_blocks; ++b) {
        TD_CHECK(n_deg[b] > 0 && deg_space[b] && sym_blocks[b], TDSCHA_EINVAL, "block %d empty", b);
        start[b] = deg_space[b][0];
        dim[b] = n_deg[b];
        TD_CHECK(start[b] == expect, TDSCHA_EINVAL,
                 "degenerate blocks must be contiguous and ordered: block %d starts at mode %d, expected %d", b, start[b], expect);
        for (int q = 0; q < n_deg[b]; ++q)
            TD_CHECK(deg_space[b][q] == start[b] + q, TDSCHA_EINVAL, "block %d is not a contiguous ascending mode range", b);
        double wmin = w[start[b]], wmax = w[start[b]];
        for (int q = 0; q < n_deg[b]; ++q) {
            TD_CHECK(blocks_ids[start[b] + q] == b, TDSCHA_EINVAL, "blocks_ids[%d] != %d", start[b] + q, b);
            wmin = std::min(wmin, w[start[b] + q]);
            wmax = std::max(wmax, w[start[b] + q]);
        }
        TD_CHECK(wmax - wmin <= 1e-10 * std::fabs(wmax), TDSCHA_EINVAL,
                 "block %d is not degenerate: frequency spread %.3e (relative) > 1e-10", b, (wmax - wmin) / std::fabs(wmax));
        expect += n_deg[b];
        dmax = std::max(dmax, n_deg[b]);
    }
    TD_CHECK(expect == n, TDSCHA_EINVAL, "blocks cover %d modes, n = %d", expect, n);
    TD_CHECK(dmax <= DMAX_SUPPORTED, TDSCHA_EINVAL, "degenerate block of %d modes exceeds the supported %d", dmax, DMAX_SUPPORTED);
    for (int m = 0; m < n; ++m) TD_CHECK(w[m] > 0, TDSCHA_EINVAL, "frequency %d is not positive (%g)", m, w[m]);

    auto *e = new tdscha_ensemble();
    e->device = dev;
    e->n = n; e->N = N; e->N_sym = N_sym; e->n_blocks = n_blocks; e->T = T; e->dmax = dmax;
    e->P = (long long)n * (n + 1) / 2;
    e->Kp = round_up(e->P, 64);
    e->N2 = 2LL * N;
    e->N2p = round_up(e->N2, 64);
    e->np = round_up(n, 64);
    e->blk_start = start; e->blk_dim = dim;
    e->blk_sym_off.resize(n_blocks);
    long long soff = 0;
    for (int b = 0; b < n_blocks; ++b) { e->blk_sym_off[b] = soff; soff += (long long)N_sym * dim[b] * dim[b]; }
    std::vector<long long> offP(n_blocks);
    long long soffP = 0;
    for (int b = 0; b < n_blocks; ++b) {
        const long long dp = (dim[b] + 3) & ~3;
        offP[b] = soffP;
        soffP += (long long)N_sym * dp * dp;
    }
    for (int b = 0; b < n_blocks; ++b)
        for (int c = b; c < n_blocks; ++c) { e->bp_b.push_back(b); e->bp_c.push_back(c); }
    double neff = 0;
    for (int i = 0; i < N; ++i) neff += rho[i];
    e->N_eff = neff;

    auto fail = [&](int rc) { ensemble_destroy(e); return rc; };
    size_t acc = 0;
    const size_t xb = (size_t)N * n * sizeof(double);
    int rc;
    if ((rc = dev_alloc((void **)&e->X, xb, &acc)) || (rc = dev_alloc((void **)&e->Y, xb, &acc)) ||
        (rc = dev_alloc((void **)&e->G, xb, &acc)) || (rc = dev_alloc((void **)&e->Xt, xb, &acc)) ||
        (rc = dev_alloc((void **)&e->rho, N * sizeof(double), &acc)) || (rc = dev_alloc((void **)&e->w, n * sizeof(double), &acc)) ||
        (rc = dev_alloc((void **)&e->ups, n * sizeof(double), &acc)) || (rc = dev_alloc((void **)&e->psi, n * sizeof(double), &acc)) ||
        (rc = dev_alloc((void **)&e->sym, soff * sizeof(double), &acc)) ||
        (rc = dev_alloc((void **)&e->symP, soffP * sizeof(float), &acc)) ||
        (rc = dev_alloc((void **)&e->symPT, soffP * sizeof(float), &acc)) ||
        (rc = dev_alloc((void **)&e->d_offP, n_blocks * sizeof(long long), &acc)) ||
        (rc = dev_alloc((void **)&e->d_blk_start, n_blocks * sizeof(int), &acc)) ||
        (rc = dev_alloc((void **)&e->d_blk_dim, n_blocks * sizeof(int), &acc)) ||
        (rc = dev_alloc((void **)&e->d_blk_sym_off, n_blocks * sizeof(long long), &acc)) ||
        (rc = dev_alloc((void **)&e->d_blocks_ids, n * sizeof(int), &acc)) ||
        (rc = dev_alloc((void **)&e->d_bp_b, e->bp_b.size() * sizeof(int), &acc)) ||
        (rc = dev_alloc((void **)&e->d_bp_c, e->bp_c.size() * sizeof(int), &acc)) ||
        (rc = dev_alloc((void **)&e->d_pair_mu, e->P * sizeof(int), &acc)) ||
        (rc = dev_alloc((void **)&e->d_pair_nu, e->P * sizeof(int), &acc)) ||
        (rc = dev_alloc((void **)&e->d_err, sizeof(unsigned), &acc)))
        return fail(rc);
    e->base_bytes = acc;
    std::vector<int> pmu(e->P), pnu(e->P);
    {
        long long p = 0;
        for (int mu = 0; mu < n; ++mu)
            for (int nu = mu; nu < n; ++nu) { pmu[p] = mu; pnu[p] = nu; ++p; }
    }
#define TD_UP(dst, src, bytes)                                                         \
    do {                                                                               \
        cudaError_t ce = cudaMemcpy((dst), (src), (bytes), cudaMemcpyHostToDevice);    \
        if (ce != cudaSuccess) { set_error("upload: %s", cudaGetErrorString(ce)); return fail(TDSCHA_ECUDA); } \
    } while (0)
    TD_UP(e->X, X, xb);
    TD_UP(e->Y, Y, xb);
    TD_UP(e->rho, rho, N * sizeof(double));
    TD_UP(e->w, w, n * sizeof(double));
    for (int b = 0; b < n_blocks; ++b)
        TD_UP(e->sym + e->blk_sym_off[b], sym_blocks[b], (size_t)N_sym * dim[b] * dim[b] * sizeof(double));
    TD_UP(e->d_blk_start, start.data(), n_blocks * sizeof(int));
    TD_UP(e->d_blk_dim, dim.data(), n_blocks * sizeof(int));
    TD_UP(e->d_blk_sym_off, e->blk_sym_off.data(), n_blocks * sizeof(long long));
    TD_UP(e->d_offP, offP.data(), n_blocks * sizeof(long long));
    TD_UP(e->d_blocks_ids, blocks_ids, n * sizeof(int));
    TD_UP(e->d_bp_b, e->bp_b.data(), e->bp_b.size() * sizeof(int));
    TD_UP(e->d_bp_c, e->bp_c.data(), e->bp_c.size() * sizeof(int));
    TD_UP(e->d_pair_mu, pmu.data(), e->P * sizeof(int));
    TD_UP(e->d_pair_nu, pnu.data(), e->P * sizeof(int));
#undef TD_UP
    if (cudaMemset(e->d_err, 0, sizeof(unsigned)) != cudaSuccess) return fail(TDSCHA_ECUDA);
    if (cosets_enabled()) {
        const int crc = setup_cosets(e, dim, sym_blocks);
        if (crc) return fail(crc);
    }
    thermal_kernel<<<ceil_div(n, 128), 128>>>(e->w, n, T, e->ups, e->psi);
    for (int b = 0; b < n_blocks; ++b) {
        const long long dp = (dim[b] + 3) & ~3;
        pad_sym_kernel<<<grid_for((long long)N_sym * dp * dp), 256>>>(e->sym + e->blk_sym_off[b], N_sym, dim[b], (int)dp,
                                                                      e->symP + offP[b], e->symPT + offP[b]);
    }
    scale_rows_kernel<<<grid_for((long long)N * n), 256>>>(e->Y, e->psi, N, n, e->G);
    scale_rows_kernel<<<grid_for((long long)N * n), 256>>>(e->X, e->ups, N, n, e->Xt);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
        set_error("ensemble set-up kernels failed");
        return fail(TDSCHA_ECUDA);
    }
    {
        size_t pcb = 0;
        int prc = build_pair_classes(dim, e->pairs, &pcb);
        if (prc) return fail(prc);
        e->base_bytes += pcb;
    }
    if (cublasCreate(&e->cublas) != CUBLAS_STATUS_SUCCESS) {
        set_error("cublasCreate failed");
        return fail(TDSCHA_ECUDA);
    }
    *out = e;
    return 0;
}

static void free_ops(OperandSet &o) {
    void *ps[] = {o.V_hi, o.V_lo, o.VT_hi, o.VT_lo, o.XG_hi, o.XG_lo, o.YXt_hi, o.YXt_lo};
    for (void *p : ps)
        if (p) cudaFree(p);
    o = OperandSet();
}

int ensemble_destroy(tdscha_ensemble *e) {
    if (!e) return 0;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(e->device);
    cudaDeviceSynchronize();
    void *ps[] = {e->X, e->Y, e->G, e->Xt, e->rho, e->w, e->ups, e->psi, e->sym, e->symP, e->symPT, e->d_offP, e->d_blk_start, e->d_blk_dim,
                  e->d_blk_sym_off, e->d_blocks_ids, e->d_bp_b, e->d_bp_c, e->d_pair_mu, e->d_pair_nu, e->d_err, e->ws.base,
                  e->vjp_ws.base, e->YX, e->chunk_ops.base, e->XGT, e->d_static_lam, e->Rrow, e->rot_ws.base};
    for (void *p : ps)
        if (p) cudaFree(p);
    for (auto &o : e->ops) free_ops(o);
    for (int f = 0; f < 3; ++f) {
        if (e->YXm_hi[f]) cudaFree(e->YXm_hi[f]);
        if (e->YXm_lo[f]) cudaFree(e->YXm_lo[f]);
    }
    free_pair_classes(e->pairs);
    free_cosets(e->cosets);
    freq_tables_destroy(e->freq);
    for (auto &fo : e->fops)
        if (fo.V_hi) cudaFree(fo.V_hi);   // one allocation per format, V_hi first
    for (auto &fo : e->fhalf)
        if (fo.V_hi) cudaFree(fo.V_hi);   // one allocation per format, V_hi first
    for (int f = 0; f < 3; ++f) {
        if (e->fyx_hi[f]) cudaFree(e->fyx_hi[f]);
        if (e->fyx_lo[f]) cudaFree(e->fyx_lo[f]);
    }
    sym_umma_destroy(e->umma);
    if (e->cublas) cublasDestroy(e->cublas);
    delete e;
    cudaSetDevice(prev);
    return 0;
}

// The transposed ensemble [X^T ; G^T] (2n x N) of the VT builder, built once.
static int ensure_XGT(tdscha_ensemble *e, cudaStream_t st) {
    if (e->XGT) return 0;
    TD_CHECK(ceil_div(e->N, 32) <= 65535, TDSCHA_EINVAL, "ensemble of %d configurations exceeds the transpose grid", e->N);
    TD_CUDA(cudaMalloc(&e->XGT, (size_t)2 * e->n * e->N * sizeof(double)));
    dim3 grid((unsigned)ceil_div(e->n, 32), (unsigned)ceil_div(e->N, 32), 2);
    transpose_XG_kernel<<<grid, dim3(32, 8), 0, st>>>(e->X, e->G, e->N, e->n, e->XGT);
    TD_CUDA(cudaGetLastError());
    return 0;
}

// Build (once) the V / VT / XG / YXt operands in storage format fmt; lo splits when with_lo.
static int ensure_operands(tdscha_ensemble *e, Format fmt, bool with_lo, cudaStream_t st) {
    OperandSet &o = e->ops[fmt];
    if (o.built && (o.has_lo || !with_lo)) return 0;
    free_ops(o);
    const size_t es = format_bytes(fmt);
    const long long nV = e->N2 * e->Kp, nVT = e->P * e->N2p, nXG = e->N2 * e->np, nYX = (long long)e->n * e->N2p;
    size_t acc = 0;
    TD_TRY(dev_alloc(&o.V_hi, nV * es, &acc));
    TD_TRY(dev_alloc(&o.VT_hi, nVT * es, &acc));
    TD_TRY(dev_alloc(&o.XG_hi, nXG * es, &acc));
    TD_TRY(dev_alloc(&o.YXt_hi, nYX * es, &acc));
    if (with_lo) {
        TD_TRY(dev_alloc(&o.V_lo, nV * es, &acc));
        TD_TRY(dev_alloc(&o.VT_lo, nVT * es, &acc));
        TD_TRY(dev_alloc(&o.XG_lo, nXG * es, &acc));
        TD_TRY(dev_alloc(&o.YXt_lo, nYX * es, &acc));
    }
    TD_TRY(ensure_XGT(e, st));
    build_V_kernel<<<rows_grid(e->Kp, e->N2), 256, 0, st>>>(e->X, e->G, e->d_pair_mu, e->d_pair_nu, e->N, e->n, e->P, e->Kp, fmt,
                                                           o.V_hi, o.V_lo);
    build_VT_kernel<<<rows_grid(e->N2p, e->P), 256, 0, st>>>(e->XGT, e->N, e->d_pair_mu, e->d_pair_nu, e->N, e->n, e->P, e->N2p,
                                                            fmt, o.VT_hi, o.VT_lo);
    build_XG_kernel<<<grid_for(nXG), 256, 0, st>>>(e->X, e->G, e->N, e->n, e->np, fmt, o.XG_hi, o.XG_lo);
    build_YXt_kernel<<<grid_for(nYX), 256, 0, st>>>(e->Y, e->Xt, e->N, e->n, e->N2p, fmt, o.YXt_hi, o.YXt_lo);
    TD_CUDA(cudaGetLastError());
    o.built = true;
    o.has_lo = with_lo;
    o.bytes = acc;
    return 0;
}

// Layout of one call's workspace for M = nb * Jc rows.
struct WsLayout {
    size_t B1_hi, B1_lo, r1_hi, r1_lo, D1, Dcd, Cw_hi, Cw_lo, AB_hi, AB_lo, Z, F, partD, partF;
    size_t Ucos, r1cos, Ysr, R1r, rtmp;   // coset path and rotated basis (0 when unused)
    size_t total;
    long long ld1, ldz, ldf;
};

// ncj > 0: the coset path with ncj cosets per symmetry chunk (U / Zs and r1p / Fs share buffers)
static WsLayout layout(const tdscha_ensemble *e, int nb, int Jc, int nf_total, Format fmt, bool lo, long long Nc, int ncj = 0) {
    WsLayout L{};
    const size_t es = format_bytes(fmt);
    const size_t as = (fmt == FMT_F64) ? 8 : 4;
    const long long M = (long long)nb * Jc;
    const long long N2pc = round_up(2 * Nc, 64);
    L.ld1 = round_up(2 * Nc, 4);
    L.ldz = round_up(e->P, 4);
    L.ldf = round_up(e->n, 4);
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) / 256 * 256; return o; };
    L.B1_hi = take(M * e->Kp * es);
    L.B1_lo = lo ? take(M * e->Kp * es) : 0;
    L.r1_hi = take(M * e->np * es);
    L.r1_lo = lo ? take(M * e->np * es) : 0;
    L.D1 = take(M * L.ld1 * as);
    L.Dcd = take(M * L.ld1 * as);
    L.Cw_hi = take(M * N2pc * es);
    L.Cw_lo = lo ? take(M * N2pc * es) : 0;
    L.AB_hi = take(M * N2pc * es);
    L.AB_lo = lo ? take(M * N2pc * es) : 0;
    L.Z = take(M * L.ldz * as);
    L.F = take(M * L.ldf * as);
    L.partD = take((size_t)nb * nf_total * e->n * e->n * 8);
    L.partF = take((size_t)nb * nf_total * e->n * 8);
    if (ncj > 0) {
        const long long Mc = (long long)nb * ncj;
        L.Ucos = take(Mc * std::max<long long>(e->Kp, L.ldz) * 4);
        L.r1cos = take(Mc * std::max<long long>(e->np, L.ldf) * 4);
    }
    if (e->Rrow) {
        L.Ysr = take((size_t)nb * e->n * e->n * 8);
        L.R1r = take((size_t)nb * e->n * 8);
        L.rtmp = take((size_t)nb * e->n * e->n * 8);
    }
    L.total = off;
    return L;
}

static int ensure_ws(tdscha_ensemble *e, size_t bytes) {
    if (e->ws.bytes >= bytes) return 0;
    if (e->ws.base) { TD_CUDA(cudaDeviceSynchronize()); cudaFree(e->ws.base); e->ws = Workspace(); }
    TD_CUDA(cudaMalloc(&e->ws.base, bytes));
    e->ws.bytes = bytes;
    return 0;
}

// C (M x N) row-major = A (M x K) . B (N x K)^T
static int gemm_abt(tdscha_ensemble *e, Format fmt, int nprod, const void *A_hi, const void *A_lo, long long lda, long long M,
                    const void *B_hi, const void *B_lo, long long ldb, long long N, long long K, void *Cout, long long ldc,
                    cudaStream_t st, bool accumulate = false) {
    if (fmt == FMT_F64) {
        const double one = 1.0, zero = accumulate ? 1.0 : 0.0;
        cublasSetStream(e->cublas, st);
        cublasStatus_t s = cublasDgemm(e->cublas, CUBLAS_OP_T, CUBLAS_OP_N, (int)N, (int)M, (int)K, &one,
                                       static_cast<const double *>(B_hi), (int)ldb, static_cast<const double *>(A_hi), (int)lda,
                                       &zero, static_cast<double *>(Cout), (int)ldc);
        TD_CHECK(s == CUBLAS_STATUS_SUCCESS, TDSCHA_ECUDA, "cublasDgemm failed (%d)", (int)s);
        return 0;
    }
    // Split K: a contraction over a K longer than about 72k runs as launches over K slices, the
    // later ones accumulating into the output.  Within one launch the co-resident tiles walk K in
    // near-lockstep and share the operand slices through L2; over a very long K they drift apart
    // (the L2 holds only a few thousand K of the tiles' panels), so the slices bound the drift.
    // TDSCHA_KSPLIT sets the slice length (elements; 0 disables).
    const char *kv = getenv("TDSCHA_KSPLIT");
    const long long kslice = kv ? atoll(kv) : 73728LL;
    const size_t es = format_bytes(fmt);
    long long chunk = K;
    if (kslice > 0 && K > kslice) chunk = round_up(ceil_div(K, ceil_div(K, kslice)), 64);
    for (long long k0 = 0; k0 < K; k0 += chunk) {
        const long long kc = std::min(chunk, K - k0);
        auto off = [&](const void *p) -> const void * {
            return p ? static_cast<const uint8_t *>(p) + k0 * es : nullptr;
        };
        tc::GemmOperands op{fmt, nprod, off(A_hi), off(A_lo), lda, off(B_hi), off(B_lo), ldb};
        op.accumulate = accumulate || k0 > 0;
        TD_TRY(tc::gemm(op, (int)M, (int)N, (int)kc, static_cast<float *>(Cout), ldc, st, e->d_err));
    }
    return 0;
}

// Bytes of the V / VT / XG / YXt operands for Nc configurations in format fmt.
static size_t operand_bytes(const tdscha_ensemble *e, long long Nc, Format fmt, bool lo) {
    const long long N2pc = round_up(2 * Nc, 64);
    const size_t per = (size_t)(2 * Nc * e->Kp + e->P * N2pc + 2 * Nc * e->np + (long long)e->n * N2pc);
    return per * format_bytes(fmt) * (lo ? 2 : 1) + 8 * 256;
}

// Operands of configurations [c0, c0 + Nc) built into `buf` (the configuration-chunked path).
static int build_chunk_operands(tdscha_ensemble *e, long long c0, long long Nc, Format fmt, bool lo, void *buf, OperandSet &o,
                                cudaStream_t st) {
    const size_t es = format_bytes(fmt);
    const long long N2pc = round_up(2 * Nc, 64);
    const long long nV = 2 * Nc * e->Kp, nVT = e->P * N2pc, nXG = 2 * Nc * e->np, nYX = (long long)e->n * N2pc;
    uint8_t *b = static_cast<uint8_t *>(buf);
    size_t off = 0;
    auto take = [&](long long count) { void *p = b + off; off += ((size_t)count * es + 255) / 256 * 256; return p; };
    o = OperandSet();
    o.V_hi = take(nV);
    o.VT_hi = take(nVT);
    o.XG_hi = take(nXG);
    o.YXt_hi = take(nYX);
    if (lo) {
        o.V_lo = take(nV);
        o.VT_lo = take(nVT);
        o.XG_lo = take(nXG);
        o.YXt_lo = take(nYX);
    }
    const int n = e->n, Ni = (int)Nc;
    const double *X = e->X + c0 * n, *G = e->G + c0 * n, *Y = e->Y + c0 * n, *Xt = e->Xt + c0 * n;
    TD_TRY(ensure_XGT(e, st));
    build_V_kernel<<<rows_grid(e->Kp, 2 * Nc), 256, 0, st>>>(X, G, e->d_pair_mu, e->d_pair_nu, Ni, n, e->P, e->Kp, fmt, o.V_hi,
                                                            o.V_lo);
    build_VT_kernel<<<rows_grid(N2pc, e->P), 256, 0, st>>>(e->XGT + c0, e->N, e->d_pair_mu, e->d_pair_nu, Ni, n, e->P, N2pc, fmt,
                                                          o.VT_hi, o.VT_lo);
    build_XG_kernel<<<grid_for(nXG), 256, 0, st>>>(X, G, Ni, n, e->np, fmt, o.XG_hi, o.XG_lo);
    build_YXt_kernel<<<grid_for(nYX), 256, 0, st>>>(Y, Xt, Ni, n, N2pc, fmt, o.YXt_hi, o.YXt_lo);
    TD_CUDA(cudaGetLastError());
    o.built = true;
    o.has_lo = lo;
    return 0;
}

// TDSCHA_SYM_UMMA=1 runs the bf16 formats' symmetry transform / fold on the tcgen05 kernels of
// symmetry_umma.cu instead of the mma.sync kernels of symmetry_tc.cu (read at every call).  Off by
// default: on the 4x4x4 benchmark the tcgen05 version is correct but slower (96 + 112 ms against
// 69 + 105 ms per 16-vector step) and less accurate (bf16 instead of tf32 splitting); its profile
// shows one 14-warp CTA per SM waiting on the per-symmetry chain copy -> MMA -> TMEM read-back ->
// MMA -> store (tensor pipe active 2 %, issue active 13 %).
static bool sym_umma_enabled() {
    const char *env = getenv("TDSCHA_SYM_UMMA");
    return env && atoi(env) == 1;
}

// ------------------------------------------------------------------------------------------------
// The averages on the character classes of the subgroup (freq.cuh): dense transform and fold over
// the coset representatives, the four contractions class by class.
// ------------------------------------------------------------------------------------------------
// k-blocks accumulated in tensor memory per drain of the class [a|b] contraction.  Its K is one
// class's components (a few thousand), so its tiles are short and a drain after every k-block leaves
// the tile's final store exposed; four k-blocks per drain overlap it with the next tile's MMAs at
// the split modes' accuracy of single-k-block drains (measured on the 4x4x4 benchmark system).
// TDSCHA_FREQ_DRAIN_AB overrides (0: the contraction default).
static int freq_ab_drain() {
    const char *env = getenv("TDSCHA_FREQ_DRAIN_AB");
    return env ? std::max(0, atoi(env)) : 4;
}

// TDSCHA_FREQ_FUSED_CD=1 forms the thin [c|d] contraction of the split formats inside the weights
// kernel instead of a grouped contraction plus a separate weights kernel (read at every call).  Off
// by default: on the 4x4x4 benchmark system the fused kernel takes 6.7 ms per 16-vector step against
// 2.1 + 3.1 ms for the two launches (same results).
static bool fused_cd_enabled() {
    const char *env = getenv("TDSCHA_FREQ_FUSED_CD");
    return env && atoi(env) == 1;
}

static bool use_freq_path(const tdscha_ensemble *e, Format fmt) {
    return e->freq && e->cosets && cosets_enabled() && freq_enabled() && !(fmt == FMT_BF16 && sym_umma_enabled());
}

// Resident character-basis operands of all configurations in format fmt (one allocation).
static int ensure_freq_operands(tdscha_ensemble *e, Format fmt, bool lo, cudaStream_t st) {
    FreqOps &o = e->fops[fmt];
    if (o.built && (o.has_lo || !lo)) return 0;
    if (o.V_hi) { TD_CUDA(cudaDeviceSynchronize()); cudaFree(o.V_hi); o = FreqOps(); }
    void *buf = nullptr;
    TD_CUDA(cudaMalloc(&buf, freq_operand_bytes(*e->freq, e->N, fmt, lo)));
    TD_TRY(ensure_XGT(e, st));
    const int rc = freq_build_operands(*e->freq, e->X, e->G, e->Y, e->Xt, e->XGT, e->N, e->n, e->N, fmt, lo, buf, o, st);
    if (rc) { cudaFree(buf); o = FreqOps(); return rc; }
    return 0;
}

struct FreqWs {
    size_t U, r1, Lab_hi, Lab_lo, Lcd_hi, Lcd_lo, H, Ch, Cw_hi, Cw_lo, AB_hi, AB_lo, O, OF, partD, partF, Ysr, R1r, rtmp;
    size_t total;
    long long ld1, ldz, ldf, N2pc;
};

static FreqWs freq_ws_layout(const tdscha_ensemble *e, int nb, int ncj, int nf_total, Format fmt, bool lo, long long Nc) {
    const FreqTables &t = *e->freq;
    FreqWs L{};
    const size_t es = format_bytes(fmt), as = fmt == FMT_F64 ? 8 : 4;
    const long long NR = (long long)nb * ncj, nC = t.n_class, Kmq = std::max(t.Kmq, 1);
    L.N2pc = round_up(2 * Nc, 64);
    L.ld1 = round_up(2 * Nc, 4);
    L.ldz = round_up(e->P, 4);
    L.ldf = round_up(e->n, 4);
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) / 256 * 256; return o; };
    L.U = take(NR * std::max<long long>(e->Kp, L.ldz) * as);
    L.r1 = take(NR * std::max<long long>(e->np, L.ldf) * as);
    L.Lab_hi = take(2 * NR * t.Kq * es);
    L.Lab_lo = lo ? take(2 * NR * t.Kq * es) : 0;
    L.Lcd_hi = take(2 * NR * Kmq * es);
    L.Lcd_lo = lo ? take(2 * NR * Kmq * es) : 0;
    L.H = take(nC * 2 * NR * L.ld1 * as);
    L.Ch = take(nC * 2 * NR * L.ld1 * as);
    L.Cw_hi = take(nC * 2 * NR * L.N2pc * es);
    L.Cw_lo = lo ? take(nC * 2 * NR * L.N2pc * es) : 0;
    L.AB_hi = take(nC * 2 * NR * L.N2pc * es);
    L.AB_lo = lo ? take(nC * 2 * NR * L.N2pc * es) : 0;
    L.O = take(2 * NR * t.Kq * as);
    L.OF = take(2 * NR * Kmq * as);
    L.partD = take((size_t)nb * nf_total * e->n * e->n * 8);
    L.partF = take((size_t)nb * nf_total * e->n * 8);
    L.Ysr = take((size_t)nb * e->n * e->n * 8);
    L.R1r = take((size_t)nb * e->n * 8);
    L.rtmp = take((size_t)nb * e->n * e->n * 8);
    L.total = off;
    return L;
}

// C (row-major) (+)= A . B^T for every group, FP64 (cuBLAS DGEMM per group)
static int gemm_groups_f64(tdscha_ensemble *e, const std::vector<tc::GemmGroup> &gs, const double *A, long long lda,
                           const double *B, long long ldb, double *C, long long ldc, bool accumulate, cudaStream_t st) {
    const double one = 1.0, beta = accumulate ? 1.0 : 0.0;
    cublasSetStream(e->cublas, st);
    for (const auto &g : gs) {
        cublasStatus_t s = cublasDgemm(e->cublas, CUBLAS_OP_T, CUBLAS_OP_N, g.N, g.M, g.K, &one, B + (long long)g.b_row * ldb + g.b_k,
                                       (int)ldb, A + (long long)g.a_row * lda + g.a_k, (int)lda, &beta, C + g.d_off, (int)ldc);
        TD_CHECK(s == CUBLAS_STATUS_SUCCESS, TDSCHA_ECUDA, "cublasDgemm failed (%d)", (int)s);
    }
    return 0;
}

static int gemm_groups(tdscha_ensemble *e, Format fmt, int nprod, const void *A_hi, const void *A_lo, long long a_rows,
                       long long lda, const void *B_hi, const void *B_lo, long long b_rows, long long ldb,
                       const std::vector<tc::GemmGroup> &gs, void *C, long long ldc, bool accumulate, cudaStream_t st,
                       int drain_kb = 0) {
    if (gs.empty()) return 0;
    if (fmt == FMT_F64)
        return gemm_groups_f64(e, gs, static_cast<const double *>(A_hi), lda, static_cast<const double *>(B_hi), ldb,
                               static_cast<double *>(C), ldc, accumulate, st);
    tc::GemmOperands op{fmt, nprod, A_hi, A_lo, lda, B_hi, B_lo, ldb};
    op.accumulate = accumulate;
    op.drain_kb = drain_kb;
    return tc::gemm_grouped(op, a_rows, lda, b_rows, ldb, gs.data(), (int)gs.size(), static_cast<float *>(C), ldc, st, e->d_err);
}

static int perturb_average_freq(tdscha_ensemble *e, int nb, const double *R1, const double *Ys, int apply_d4, Format fmt,
                                int nprod, bool lo, double *f_out, double *d_out, cudaStream_t st) {
    const FreqTables &ft = *e->freq;
    const SymCosets *cs = e->cosets;
    const int n_cos = cs->n_cos, sub = cs->sub, nC = ft.n_class;
    // fold partials: Jf representatives per fold CTA (eight partials of 6 at 48 representatives), so
    // that each CTA reuses its W block over several representatives
    const int Jf = std::max(1, ceil_div(n_cos, 8));
    const int nf_total = ceil_div(n_cos, Jf);
    const size_t es = format_bytes(fmt);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    TD_CUDA(cudaStreamIsCapturing(st, &cap));
    long long Nc = e->N;
    int ncj = 0;
    bool half = false;   // chunks over resident row-major class operands
    FreqOps co;
    if (cap != cudaStreamCaptureStatusNone) {
        const AvgPlan &pl = e->plan;
        TD_CHECK(pl.valid && pl.nb == nb && pl.fmt == (int)fmt && pl.lo == lo && pl.cosets && pl.freq, TDSCHA_EINVAL,
                 "graph capture of the averages needs an earlier call with the same batch (%d) and precision", nb);
        Nc = pl.Nc;
        ncj = pl.Jc / sub;
        half = pl.half;
        if (Nc < e->N) {
            const size_t need = half ? freq_chunk_cols_bytes(ft, Nc, fmt, lo) : freq_operand_bytes(ft, Nc, fmt, lo);
            TD_CHECK(e->chunk_ops.bytes >= need, TDSCHA_EINVAL, "chunk buffer changed since the plan");
            TD_CHECK(!half || (e->fhalf[fmt].built && (e->fhalf[fmt].has_lo || !lo)), TDSCHA_EINVAL, "resident rows released since the plan");
        } else {
            TD_CHECK(e->fops[fmt].built && (e->fops[fmt].has_lo || !lo), TDSCHA_EINVAL, "operands released since the plan");
            co = e->fops[fmt];
        }
    } else {
        size_t free_b = 0, tot_b = 0;
        TD_CUDA(cudaMemGetInfo(&free_b, &tot_b));
        const size_t avail = free_b + e->ws.bytes + e->chunk_ops.bytes;
        const char *env_chunk = getenv("TDSCHA_CONFIG_CHUNK");
        // Configuration chunks: all configurations when their operands fit in half of the memory this
        // call may use; else every class operand is rebuilt per chunk, or, with
        // TDSCHA_CHUNK_RESIDENT_ROWS=1 and a split format, the row-major class operands of all
        // configurations stay resident (when they fit in 55 % of that memory) and only the transposed
        // ones are formed per chunk.  Off by default: on the 5x5x5 system the per-chunk transposes
        // took 263 ms per 16-vector step against 143 ms for the full rebuilds.
        const char *env_rows = getenv("TDSCHA_CHUNK_RESIDENT_ROWS");
        const bool may_half = fmt != FMT_F64 && env_rows && atoi(env_rows) == 1;
        const size_t resident = freq_resident_rows_bytes(ft, e->N, fmt, lo);
        const bool rows_fit = may_half && (e->fhalf[fmt].built || resident < (size_t)(avail * 0.55));
        if (env_chunk && atoll(env_chunk) > 0 && atoll(env_chunk) < e->N) {
            Nc = atoll(env_chunk);
            half = rows_fit;
        } else if (!e->fops[fmt].built && freq_operand_bytes(ft, e->N, fmt, lo) > avail / 2) {
            half = rows_fit;
            const long long per_conf = (half ? 2LL : 4LL) * (ft.Kq + ft.Kmq) * (long long)es * (lo ? 2 : 1);
            const size_t room = half ? (e->fhalf[fmt].built ? avail : avail - resident) : avail;
            const long long fit = (long long)(room * 0.4) / per_conf;
            Nc = std::min<long long>(e->N, std::max<long long>(32, fit / 32 * 32));
        }
        if (Nc < e->N) {
            if (half && !(e->fhalf[fmt].built && (e->fhalf[fmt].has_lo || !lo))) {
                if (e->fhalf[fmt].V_hi) { TD_CUDA(cudaDeviceSynchronize()); cudaFree(e->fhalf[fmt].V_hi); e->fhalf[fmt] = FreqOps(); }
                void *buf = nullptr;
                TD_CUDA(cudaMalloc(&buf, resident));
                TD_TRY(ensure_XGT(e, st));
                const int rc = freq_build_rows(ft, e->X, e->G, e->XGT, e->N, e->n, e->N, fmt, lo, buf, e->fhalf[fmt], st);
                if (rc) { cudaFree(buf); e->fhalf[fmt] = FreqOps(); return rc; }
            }
            const size_t need = half ? freq_chunk_cols_bytes(ft, Nc, fmt, lo) : freq_operand_bytes(ft, Nc, fmt, lo);
            if (e->chunk_ops.bytes < need) {
                if (e->chunk_ops.base) { TD_CUDA(cudaDeviceSynchronize()); cudaFree(e->chunk_ops.base); e->chunk_ops = Workspace(); }
                TD_CUDA(cudaMalloc(&e->chunk_ops.base, need));
                e->chunk_ops.bytes = need;
            }
        } else {
            TD_TRY(ensure_freq_operands(e, fmt, lo, st));
            co = e->fops[fmt];
        }
        TD_CUDA(cudaMemGetInfo(&free_b, &tot_b));
        // coset chunk: the largest multiple of Jf whose workspace fits in the budget
        const size_t budget = std::max<size_t>((size_t)2 << 30, (size_t)((free_b + e->ws.bytes) * 0.6));
        ncj = (int)round_up(n_cos, Jf);
        while (ncj > Jf && freq_ws_layout(e, nb, ncj, nf_total, fmt, lo, Nc).total > budget) ncj -= Jf;
        const char *env_sym = getenv("TDSCHA_SYM_CHUNK");   // in symmetries; forces a smaller chunk (tuning and tests)
        if (env_sym && atoi(env_sym) > 0) ncj = std::min(ncj, std::max(Jf, atoi(env_sym) / sub / Jf * Jf));
        e->plan.valid = true;
        e->plan.nb = nb;
        e->plan.fmt = (int)fmt;
        e->plan.lo = lo;
        e->plan.cosets = true;
        e->plan.freq = true;
        e->plan.half = half;
        e->plan.Nc = Nc;
        e->plan.Jc = ncj * sub;
    }
    const bool chunked = Nc < e->N;
    const FreqWs L = freq_ws_layout(e, nb, ncj, nf_total, fmt, lo, Nc);
    if (cap != cudaStreamCaptureStatusNone)
        TD_CHECK(e->ws.bytes >= L.total, TDSCHA_EINVAL, "workspace changed since the plan");
    else
        TD_TRY(ensure_ws(e, L.total));
    uint8_t *W = static_cast<uint8_t *>(e->ws.base);
    auto at = [&](size_t off) -> void * { return W + off; };
    void *U = at(L.U), *r1 = at(L.r1), *H = at(L.H), *Ch = at(L.Ch), *O = at(L.O), *OF = at(L.OF);
    void *Lab_hi = at(L.Lab_hi), *Lab_lo = lo ? at(L.Lab_lo) : nullptr, *Lcd_hi = at(L.Lcd_hi), *Lcd_lo = lo ? at(L.Lcd_lo) : nullptr;
    void *Cw_hi = at(L.Cw_hi), *Cw_lo = lo ? at(L.Cw_lo) : nullptr, *AB_hi = at(L.AB_hi), *AB_lo = lo ? at(L.AB_lo) : nullptr;
    double *partD = static_cast<double *>(at(L.partD)), *partF = static_cast<double *>(at(L.partF));
    double *Ysr = static_cast<double *>(at(L.Ysr)), *R1r = static_cast<double *>(at(L.R1r)), *rtmp = static_cast<double *>(at(L.rtmp));
    const bool f64 = fmt == FMT_F64;
    const size_t as = f64 ? 8 : 4;
    {
        StageScope sc(e, ST_OTHER, st, 3);
        TD_TRY(rotate_mats(nb, e->n, e->dmax, e->Rrow, e->d_blocks_ids, e->d_blk_start, e->d_blk_dim, Ys, rtmp, Ysr, true, st));
        TD_TRY(rotate_rows_of(nb, e->n, e->dmax, e->Rrow, e->d_blocks_ids, e->d_blk_start, e->d_blk_dim, R1, R1r, true, st));
    }
    SymTables tr{e->sym, e->d_blk_sym_off, e->d_blk_start, e->d_blk_dim, e->n_blocks, e->n, e->dmax, cs->repP, cs->repPT, cs->d_offRep};
    SymTables t64{cs->repS, cs->d_offRepS, e->d_blk_start, e->d_blk_dim, e->n_blocks, e->n, e->dmax, nullptr, nullptr, nullptr};
    int n_classes = 0;
    for (int m = 1; m <= SYM_MT_MAX; ++m) n_classes += e->pairs.count[m] > 0 ? 1 : 0;
    const long long Kmq1 = std::max(ft.Kmq, 1);
    bool fused_cd = !f64 && ft.Kmq > 0 && fused_cd_enabled();
    for (int u : ft.mcol_used) fused_cd = fused_cd && u <= 64;
    for (int p0 = 0; p0 < n_cos; p0 += ncj) {
        const int nc = std::min(ncj, n_cos - p0);
        const int NR = nb * nc;
        {
            StageScope sc(e, ST_TRANSFORM, st, n_classes + 3);
            if (f64) {
                TD_TRY(sym_transform(t64, e->pairs, nb, nc, p0, Ysr, R1r, e->ups, e->P, e->Kp, e->np, FMT_F64, U, nullptr, r1,
                                     nullptr, false, st));
                TD_TRY(freq_left<double>(ft, NR, e->n, (const double *)U, e->Kp, (const double *)r1, e->np, fmt, Lab_hi, Lab_lo,
                                         Lcd_hi, Lcd_lo, st));
            } else {
                TD_TRY(sym_transform_tc(tr, e->pairs, nb, nc, p0, Ysr, R1r, e->ups, e->Kp, e->np, FMT_F32, U, nullptr, r1, nullptr,
                                        st));
                TD_TRY(freq_left<float>(ft, NR, e->n, (const float *)U, e->Kp, (const float *)r1, e->np, fmt, Lab_hi, Lab_lo,
                                        Lcd_hi, Lcd_lo, st));
            }
        }
        for (long long c0 = 0; c0 < e->N; c0 += Nc) {
            const long long Ncur = std::min(Nc, e->N - c0);
            const long long N2c = 2 * Ncur, N2pc = round_up(N2c, 64);   // the last chunk may be shorter
            const bool acc = c0 > 0;
            if (chunked && half) {
                StageScope sc(e, ST_OPERANDS, st, lo ? 3 : 2);
                TD_TRY(freq_build_chunk_cols(ft, e->fhalf[fmt], e->N, c0, Ncur, e->Y, e->Xt, e->n, fmt, lo, e->chunk_ops.base, co, st));
            } else if (chunked) {
                StageScope sc(e, ST_OPERANDS, st, 3);
                const int n = e->n;
                TD_TRY(ensure_XGT(e, st));
                TD_TRY(freq_build_operands(ft, e->X + c0 * n, e->G + c0 * n, e->Y + c0 * n, e->Xt + c0 * n, e->XGT + c0, e->N, n,
                                           Ncur, fmt, lo, e->chunk_ops.base, co, st));
            }
            // rows of the row-major operands: the chunk's own (2 Ncur rows), or the resident operands'
            // two ranges [c0, c0 + Ncur) and [N + c0, N + c0 + Ncur)
            const bool two = chunked && half;
            const long long brows = two ? e->N2 : N2c;
            // per class: [a|b] and [c|d] in the character basis, (rows (comp, v, c), 2Nc columns)
            std::vector<tc::GemmGroup> gab, gcd, gz, gf;
            for (int g = 0; g < nC; ++g) {
                const int Mg = ft.cls_real[g] ? NR : 2 * NR;
                const long long hrow = (long long)g * 2 * NR;
                if (two) {
                    gab.push_back({Mg, (int)Ncur, ft.pcol_cnt[g], 0, ft.pcol_off[g], (int)c0, ft.pcol_off[g], hrow * L.ld1});
                    gab.push_back({Mg, (int)Ncur, ft.pcol_cnt[g], 0, ft.pcol_off[g], (int)(e->N + c0), ft.pcol_off[g],
                                   hrow * L.ld1 + Ncur});
                } else {
                    gab.push_back({Mg, (int)N2c, ft.pcol_cnt[g], 0, ft.pcol_off[g], 0, ft.pcol_off[g], hrow * L.ld1});
                }
                gz.push_back({Mg, ft.pcol_cnt[g], (int)N2pc, (int)hrow, 0, ft.pcol_off[g], 0, (long long)ft.pcol_off[g]});
                if (ft.mcol_cnt[g] > 0) {
                    if (two) {
                        gcd.push_back({Mg, (int)Ncur, ft.mcol_cnt[g], 0, ft.mcol_off[g], (int)c0, ft.mcol_off[g], hrow * L.ld1});
                        gcd.push_back({Mg, (int)Ncur, ft.mcol_cnt[g], 0, ft.mcol_off[g], (int)(e->N + c0), ft.mcol_off[g],
                                       hrow * L.ld1 + Ncur});
                    } else {
                        gcd.push_back({Mg, (int)N2c, ft.mcol_cnt[g], 0, ft.mcol_off[g], 0, ft.mcol_off[g], hrow * L.ld1});
                    }
                    gf.push_back({Mg, ft.mcol_cnt[g], (int)N2pc, (int)hrow, 0, ft.mcol_off[g], 0, (long long)ft.mcol_off[g]});
                } else if (!fused_cd) {
                    TD_CUDA(cudaMemsetAsync(static_cast<uint8_t *>(Ch) + hrow * L.ld1 * as, 0, (size_t)2 * NR * L.ld1 * as, st));
                }
            }
            {
                StageScope sc(e, ST_GEMM_AB, st);
                TD_TRY(gemm_groups(e, fmt, nprod, Lab_hi, Lab_lo, 2LL * NR, ft.Kq, co.V_hi, co.V_lo, brows, ft.Kq, gab, H, L.ld1, false,
                                   st, freq_ab_drain()));
            }
            if (fused_cd) {
                // [c|d] formed inside the weights kernel (the class's few mode columns)
                StageScope sc(e, ST_WEIGHTS, st);
                TD_TRY(freq_weights_cd(ft, (const float *)H, L.ld1, Lcd_hi, Lcd_lo, co.XG_hi, co.XG_lo, e->rho + c0, Ncur, NR, N2pc,
                                       apply_d4, fmt, Cw_hi, Cw_lo, AB_hi, AB_lo, st));
            } else {
                {
                    StageScope sc(e, ST_GEMM_CD, st);
                    TD_TRY(gemm_groups(e, fmt, nprod, Lcd_hi, Lcd_lo, 2LL * NR, Kmq1, co.XG_hi, co.XG_lo, brows, Kmq1, gcd, Ch, L.ld1,
                                       false, st));
                }
                StageScope sc(e, ST_WEIGHTS, st);
                if (f64)
                    TD_TRY(freq_weights<double>(ft, (const double *)H, (const double *)Ch, L.ld1, e->rho + c0, Ncur, NR, N2pc,
                                                apply_d4, fmt, Cw_hi, Cw_lo, AB_hi, AB_lo, st));
                else
                    TD_TRY(freq_weights<float>(ft, (const float *)H, (const float *)Ch, L.ld1, e->rho + c0, Ncur, NR, N2pc,
                                               apply_d4, fmt, Cw_hi, Cw_lo, AB_hi, AB_lo, st));
            }
            {
                StageScope sc(e, ST_GEMM_Z, st);
                TD_TRY(gemm_groups(e, fmt, nprod, Cw_hi, Cw_lo, (long long)nC * 2 * NR, N2pc, co.VT_hi, co.VT_lo, ft.Kq, N2pc,
                                   gz, O, ft.Kq, acc, st));
            }
            {
                StageScope sc(e, ST_GEMM_F, st);
                TD_TRY(gemm_groups(e, fmt, nprod, AB_hi, AB_lo, (long long)nC * 2 * NR, N2pc, co.YX_hi, co.YX_lo, Kmq1, N2pc,
                                   gf, OF, Kmq1, acc, st));
            }
        }
        {
            StageScope sc(e, ST_FOLD, st, n_classes + 2);
            if (f64) {
                TD_TRY(freq_reconstruct<double>(ft, NR, e->n, e->P, e->d_pair_mu, e->d_pair_nu, (const double *)O, (const double *)OF,
                                                (double *)U, L.ldz, (double *)r1, L.ldf, st));
                TD_TRY(sym_fold<double>(t64, e->pairs, e->d_blocks_ids, nb, nc, p0, Jf, nf_total, (const double *)U, L.ldz,
                                        (const double *)r1, L.ldf, e->ups, partD, partF, false, st));
            } else {
                TD_TRY(freq_reconstruct<float>(ft, NR, e->n, e->P, e->d_pair_mu, e->d_pair_nu, (const float *)O, (const float *)OF,
                                               (float *)U, L.ldz, (float *)r1, L.ldf, st));
                TD_TRY(sym_fold_tc(tr, e->pairs, nb, nc, p0, Jf, nf_total, (const float *)U, L.ldz, (const float *)r1, L.ldf, e->ups,
                                   partD, partF, st));
            }
        }
    }
    const double norm = 1.0 / (e->N_eff * (double)e->N_sym);
    StageScope sc(e, ST_OTHER, st, 4);
    fold_reduce_kernel<<<grid_for((long long)nb * e->n * e->n), 256, 0, st>>>(partD, partF, nf_total, e->n, nb, e->d_blocks_ids,
                                                                               norm, Ysr, R1r);
    TD_CUDA(cudaGetLastError());
    TD_TRY(rotate_mats(nb, e->n, e->dmax, e->Rrow, e->d_blocks_ids, e->d_blk_start, e->d_blk_dim, Ysr, rtmp, d_out, false, st));
    TD_TRY(rotate_rows_of(nb, e->n, e->dmax, e->Rrow, e->d_blocks_ids, e->d_blk_start, e->d_blk_dim, R1r, f_out, false, st));
    return 0;
}

int perturb_average_device(tdscha_ensemble *e, int nb, const double *R1, const double *Ys, int apply_d4, int precision,
                           double *f_out, double *d_out, cudaStream_t st) {
    TD_CHECK(e != nullptr, TDSCHA_EINVAL, "NULL ensemble");
    TD_CHECK(nb > 0, TDSCHA_EINVAL, "nb must be positive");
    TD_CHECK(apply_d4 == 0 || apply_d4 == 1, TDSCHA_EINVAL, "apply_D4 must be 0 or 1 (got %d)", apply_d4);
    TD_CHECK(precision >= TDSCHA_PREC_FP64 && precision <= TDSCHA_PREC_BF16, TDSCHA_EINVAL, "unknown precision %d", precision);
    const Format fmt = format_of(precision);
    const int nprod = products_of(precision);
    const bool lo = needs_lo(precision);
    if (use_freq_path(e, fmt)) return perturb_average_freq(e, nb, R1, Ys, apply_d4, fmt, nprod, lo, f_out, d_out, st);
    // factorised symmetry path (cosets.cuh) for the mixed formats, unless the tcgen05 symmetry
    // kernels are selected
    const bool use_cos = e->cosets && fmt != FMT_F64 && !(fmt == FMT_BF16 && sym_umma_enabled()) && cosets_enabled();
    const int sub = use_cos ? e->cosets->sub : 1;
    // fold chunking: Jf symmetries (cosets on the coset path) per partial, at most 64 partials;
    // symmetry chunks are multiples of `unit` rows
    const int n_units = use_cos ? e->cosets->n_cos : e->N_sym;
    const int Jf = use_cos ? ceil_div(n_units, 64) : std::max(16, ceil_div(e->N_sym, 64));
    const int nf_total = ceil_div(n_units, Jf);
    const int unit = use_cos ? sub * Jf : Jf;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    TD_CUDA(cudaStreamIsCapturing(st, &cap));
    long long Nc = e->N;
    int Jc = 0;
    OperandSet co;
    if (cap != cudaStreamCaptureStatusNone) {
        // inside a CUDA graph capture: the plan and buffers of the previous (eager) call, unchanged
        const AvgPlan &pl = e->plan;
        TD_CHECK(pl.valid && pl.nb == nb && pl.fmt == (int)fmt && pl.lo == lo && pl.cosets == use_cos && !pl.freq, TDSCHA_EINVAL,
                 "graph capture of the averages needs an earlier call with the same batch (%d) and precision", nb);
        Nc = pl.Nc;
        Jc = pl.Jc;
        if (Nc < e->N) {
            TD_CHECK(e->chunk_ops.bytes >= operand_bytes(e, Nc, fmt, lo), TDSCHA_EINVAL, "chunk buffer changed since the plan");
        } else {
            TD_CHECK(e->ops[fmt].built && (e->ops[fmt].has_lo || !lo), TDSCHA_EINVAL, "operands released since the plan");
            co = e->ops[fmt];
        }
    } else {
        // Configuration chunk: all configurations when their operands fit in half of the free memory
        // (then they stay resident between calls), else chunks of Nc whose operands are rebuilt from
        // the resident X, G, Y per (symmetry chunk, configuration chunk).  TDSCHA_CONFIG_CHUNK forces a
        // chunk size (tuning and tests).
        size_t free_b = 0, tot_b = 0;
        TD_CUDA(cudaMemGetInfo(&free_b, &tot_b));
        const char *env_chunk = getenv("TDSCHA_CONFIG_CHUNK");
        if (env_chunk && atoll(env_chunk) > 0 && atoll(env_chunk) < e->N) {
            Nc = atoll(env_chunk);
        } else if (!e->ops[fmt].built &&
                   operand_bytes(e, e->N, fmt, lo) > (free_b + e->ws.bytes + e->chunk_ops.bytes) / 2) {
            // memory this call may use: free + its own workspace and chunk buffer (so every call plans alike)
            const long long per_conf = 2 * (e->Kp + e->P + e->np + e->n) * (long long)format_bytes(fmt) * (lo ? 2 : 1);
            const long long fit = (long long)((free_b + e->ws.bytes + e->chunk_ops.bytes) * 0.4) / per_conf;
            Nc = std::min<long long>(e->N, std::max<long long>(32, fit / 32 * 32));
        }
        if (Nc < e->N) {
            const size_t need = operand_bytes(e, Nc, fmt, lo);
            if (e->chunk_ops.bytes < need) {
                if (e->chunk_ops.base) { TD_CUDA(cudaDeviceSynchronize()); cudaFree(e->chunk_ops.base); e->chunk_ops = Workspace(); }
                TD_CUDA(cudaMalloc(&e->chunk_ops.base, need));
                e->chunk_ops.bytes = need;
            }
            TD_CUDA(cudaMemGetInfo(&free_b, &tot_b));
        } else {
            TD_TRY(ensure_operands(e, fmt, lo, st));
            co = e->ops[fmt];
        }
        // GEMM chunk over symmetries: the largest multiple of Jf whose workspace fits in the budget
        // (fewer symmetry chunks = fewer rebuilds of chunked operands and fewer small launches)
        const size_t budget = std::max<size_t>((size_t)2 << 30, (size_t)((free_b + e->ws.bytes) * 0.6));
        Jc = (int)round_up(e->N_sym, unit);
        while (Jc > unit && layout(e, nb, Jc, nf_total, fmt, lo, Nc, use_cos ? Jc / sub : 0).total > budget) Jc -= unit;
        const char *env_sym = getenv("TDSCHA_SYM_CHUNK");   // forces a smaller chunk (tuning and tests)
        if (env_sym && atoi(env_sym) > 0) Jc = std::min(Jc, std::max(unit, atoi(env_sym) / unit * unit));
        e->plan.valid = true;
        e->plan.nb = nb;
        e->plan.fmt = (int)fmt;
        e->plan.lo = lo;
        e->plan.cosets = use_cos;
        e->plan.freq = false;
        e->plan.Nc = Nc;
        e->plan.Jc = Jc;
    }
    const bool chunked = Nc < e->N;
    const WsLayout L = layout(e, nb, Jc, nf_total, fmt, lo, Nc, use_cos ? Jc / sub : 0);
    if (cap != cudaStreamCaptureStatusNone)
        TD_CHECK(e->ws.bytes >= L.total, TDSCHA_EINVAL, "workspace changed since the plan");
    else
        TD_TRY(ensure_ws(e, L.total));
    uint8_t *W = static_cast<uint8_t *>(e->ws.base);
    void *B1_hi = W + L.B1_hi, *B1_lo = lo ? W + L.B1_lo : nullptr;
    void *r1_hi = W + L.r1_hi, *r1_lo = lo ? W + L.r1_lo : nullptr;
    void *D1 = W + L.D1, *Dcd = W + L.Dcd, *Z = W + L.Z, *F = W + L.F;
    void *Cw_hi = W + L.Cw_hi, *Cw_lo = lo ? W + L.Cw_lo : nullptr;
    void *AB_hi = W + L.AB_hi, *AB_lo = lo ? W + L.AB_lo : nullptr;
    double *partD = reinterpret_cast<double *>(W + L.partD);
    double *partF = reinterpret_cast<double *>(W + L.partF);
    float *Ucos = use_cos ? reinterpret_cast<float *>(W + L.Ucos) : nullptr;
    float *r1cos = use_cos ? reinterpret_cast<float *>(W + L.r1cos) : nullptr;
    // inputs into the ensemble's rotated basis
    double *Ysr = e->Rrow ? reinterpret_cast<double *>(W + L.Ysr) : nullptr;
    double *R1r = e->Rrow ? reinterpret_cast<double *>(W + L.R1r) : nullptr;
    double *rtmp = e->Rrow ? reinterpret_cast<double *>(W + L.rtmp) : nullptr;
    if (e->Rrow) {
        StageScope sc(e, ST_OTHER, st, 3);
        TD_TRY(rotate_mats(nb, e->n, e->dmax, e->Rrow, e->d_blocks_ids, e->d_blk_start, e->d_blk_dim, Ys, rtmp, Ysr, true, st));
        TD_TRY(rotate_rows_of(nb, e->n, e->dmax, e->Rrow, e->d_blocks_ids, e->d_blk_start, e->d_blk_dim, R1, R1r, true, st));
        Ys = Ysr;
        R1 = R1r;
    }

    SymTables t{e->sym, e->d_blk_sym_off, e->d_blk_start, e->d_blk_dim, e->n_blocks, e->n, e->dmax, e->symP, e->symPT, e->d_offP};
    SymTables tr = t;   // the coset representatives' tables
    if (use_cos) {
        tr.symP = e->cosets->repP;
        tr.symPT = e->cosets->repPT;
        tr.offP = e->cosets->d_offRep;
    }
    if (fmt == FMT_BF16 && sym_umma_enabled()) {
        // the bf16 formats run the symmetry transform and fold on tcgen05 (tables built on first use)
        if (!e->umma) {
            TD_CHECK(cap == cudaStreamCaptureStatusNone, TDSCHA_EINVAL,
                     "graph capture of the averages needs an earlier eager call in this precision");
            TD_TRY(sym_umma_create(t, e->N_sym, e->blk_dim, e->blk_sym_off, &e->umma));
        }
        t.umma = e->umma;
        t.blocks_ids = e->d_blocks_ids;
        t.err = e->d_err;
    }

    // kernels per transform / fold stage: one per non-empty block-pair class (+ the padding kernel of
    // the transform), or the tcgen05 kernel and its vector-part kernel
    int n_classes = 0;
    for (int m = 1; m <= SYM_MT_MAX; ++m) n_classes += e->pairs.count[m] > 0 ? 1 : 0;
    const int transform_launches = use_cos ? n_classes + 2 : (t.umma ? 3 : n_classes + 1);
    const int fold_launches = use_cos ? n_classes + 2 : (t.umma ? 2 : n_classes);
    const SymCosets *cs = e->cosets;
    for (int j0 = 0; j0 < e->N_sym; j0 += Jc) {
        const int nj = std::min(Jc, e->N_sym - j0);
        const long long M = (long long)nb * nj;
        const int ncj = nj / sub, p0 = j0 / sub;   // cosets of this chunk (coset path)
        // rows r = k * nj + jj (internal coset-major order of the symmetries on the coset path)
        {
            StageScope sc(e, ST_TRANSFORM, st, transform_launches);
            if (use_cos) {
                // U_p = S_p^T Ys S_p and r1 of the representatives (fp32), then the expansion D_j^T U_p D_j
                TD_TRY(sym_transform_tc(tr, e->pairs, nb, ncj, p0, Ys, R1, e->ups, e->Kp, e->np, FMT_F32, Ucos, nullptr, r1cos,
                                        nullptr, st));
                TD_TRY(coset_expand(nb, ncj, sub, j0, e->P, e->Kp, e->n, Ucos, e->d_pair_mu, e->d_pair_nu, cs->partner, cs->c0,
                                    cs->c1, fmt, B1_hi, B1_lo, st));
                TD_TRY(coset_expand_r1(nb, ncj, sub, j0, e->n, e->np, r1cos, cs->partner, cs->c0, cs->c1, fmt, r1_hi, r1_lo, st));
            } else {
                TD_TRY(sym_transform(t, e->pairs, nb, nj, j0, Ys, R1, e->ups, e->P, e->Kp, e->np, fmt, B1_hi, B1_lo, r1_hi,
                                     r1_lo, fmt != FMT_F64, st));
            }
        }
        for (long long c0 = 0; c0 < e->N; c0 += Nc) {
            const long long Ncur = std::min(Nc, e->N - c0);
            const long long N2c = 2 * Ncur, N2pc = round_up(N2c, 64);
            const bool acc = c0 > 0;
            if (chunked) {
                StageScope sc(e, ST_OPERANDS, st, 4);
                TD_TRY(build_chunk_operands(e, c0, Ncur, fmt, lo, e->chunk_ops.base, co, st));
            }
            // GEMM1: [a | b] = B1 . V^T      (M x 2Nc, K = Kp)
            {
                StageScope sc(e, ST_GEMM_AB, st);
                TD_TRY(gemm_abt(e, fmt, nprod, B1_hi, B1_lo, e->Kp, M, co.V_hi, co.V_lo, e->Kp, N2c, e->Kp, D1, L.ld1, st));
            }
            // [c | d] = r1 . [X; G]^T         (M x 2Nc, K = np)
            {
                StageScope sc(e, ST_GEMM_CD, st);
                TD_TRY(gemm_abt(e, fmt, nprod, r1_hi, r1_lo, e->np, M, co.XG_hi, co.XG_lo, e->np, N2c, e->np, Dcd, L.ld1, st));
            }
            // weights
            {
                StageScope sc(e, ST_WEIGHTS, st);
                const int Ni = (int)Ncur;
                if (fmt == FMT_F64)
                    weights_kernel<double><<<grid_for(M * (Ncur + N2pc - N2c)), 256, 0, st>>>(
                        (const double *)D1, (const double *)Dcd, L.ld1, e->rho + c0, Ni, (int)M, N2pc, apply_d4, fmt, Cw_hi,
                        Cw_lo, AB_hi, AB_lo);
                else
                    weights_kernel<float><<<grid_for(M * (Ncur + N2pc - N2c)), 256, 0, st>>>(
                        (const float *)D1, (const float *)Dcd, L.ld1, e->rho + c0, Ni, (int)M, N2pc, apply_d4, fmt, Cw_hi,
                        Cw_lo, AB_hi, AB_lo);
                TD_CUDA(cudaGetLastError());
            }
            // GEMM2: Z (+)= Cw . VT^T          (M x P, K = N2pc)
            {
                StageScope sc(e, ST_GEMM_Z, st);
                TD_TRY(gemm_abt(e, fmt, nprod, Cw_hi, Cw_lo, N2pc, M, co.VT_hi, co.VT_lo, N2pc, e->P, N2pc, Z, L.ldz, st, acc));
            }
            // F (+)= AB . YXt^T                (M x n, K = N2pc)
            {
                StageScope sc(e, ST_GEMM_F, st);
                TD_TRY(gemm_abt(e, fmt, nprod, AB_hi, AB_lo, N2pc, M, co.YXt_hi, co.YXt_lo, N2pc, e->n, N2pc, F, L.ldf, st, acc));
            }
        }
        // fold this chunk into the partials
        {
            StageScope sc(e, ST_FOLD, st, fold_launches);
            if (use_cos) {
                // sum over each coset of D_j W_j D_j^T, D_j F_j, then the representatives' dense fold
                TD_TRY(coset_fold_inner(nb, ncj, sub, j0, e->P, L.ldz, L.ldf, e->n, (const float *)Z, (const float *)F,
                                        e->d_pair_mu, e->d_pair_nu, cs->partner, cs->c0, cs->c1, Ucos, r1cos, st));
                TD_TRY(sym_fold_tc(tr, e->pairs, nb, ncj, p0, Jf, nf_total, Ucos, L.ldz, r1cos, L.ldf, e->ups, partD, partF, st));
            } else if (fmt == FMT_F64)
                TD_TRY(sym_fold<double>(t, e->pairs, e->d_blocks_ids, nb, nj, j0, Jf, nf_total, (const double *)Z, L.ldz,
                                        (const double *)F, L.ldf, e->ups, partD, partF, false, st));
            else
                TD_TRY(sym_fold<float>(t, e->pairs, e->d_blocks_ids, nb, nj, j0, Jf, nf_total, (const float *)Z, L.ldz,
                                       (const float *)F, L.ldf, e->ups, partD, partF, true, st));
        }
    }
    const double norm = 1.0 / (e->N_eff * (double)e->N_sym);
    StageScope sc(e, ST_OTHER, st, e->Rrow ? 4 : 1);
    // in the rotated basis: reduce into the input buffers (free now), then rotate into the outputs
    double *Dr = e->Rrow ? Ysr : d_out, *fr = e->Rrow ? R1r : f_out;
    fold_reduce_kernel<<<grid_for((long long)nb * e->n * e->n), 256, 0, st>>>(partD, partF, nf_total, e->n, nb, e->d_blocks_ids,
                                                                               norm, Dr, fr);
    TD_CUDA(cudaGetLastError());
    if (e->Rrow) {
        TD_TRY(rotate_mats(nb, e->n, e->dmax, e->Rrow, e->d_blocks_ids, e->d_blk_start, e->d_blk_dim, Dr, rtmp, d_out, false, st));
        TD_TRY(rotate_rows_of(nb, e->n, e->dmax, e->Rrow, e->d_blocks_ids, e->d_blk_start, e->d_blk_dim, fr, f_out, false, st));
    }
    return 0;
}

// ================================================================================================
// Vector-Jacobian product of the averages w.r.t. (Y, rho).
//
// With the forward quantities per (row r = (k, j), configuration i): a, b = [a|b], c, d = [c|d],
// weights gamma = rho (-c/3 + d4 a/8), delta = rho (-d/3 + d4 b/4), alpha = -rho a/6,
// beta = -rho b/3, the pairing <fbar, f_av> + <Dbar, D_av> equals
//   norm sum_{r,i} rho_i [ delta'/2 A' + gamma' B' + alpha' C' + beta' D' ]      (primes: rho_i = 1)
// where [A'|B'] = Q . V^T with Q_j[p] = 2 ups_mu ups_nu (S_j^T Dbar S_j)[mu nu] (packed) and
// [C'|D'] = phi . [Y; X~]^T with phi_j = S_j^T fbar; Q and phi come from the symmetry transform of
// (2 ups ups Dbar, fbar / ups) (ups is constant on a degenerate block).  Y enters through
// g = psi o y (second half of V, d = r1 . g) and directly through C' = phi . y:
//   Vbar[N+i, :] = sum_r K1_ri B1_r + K2_ri Q_r,  K1 = d4 A'/8 - D'/3, K2 = -c/3 + d4 a/8
//   gbar_i       = (d V[N+i] / d g_i)^T Vbar[N+i] + sum_r K3_ri r1_r,  K3 = -A'/6
//   Ybar_i       = norm rho_i (psi o gbar_i + sum_r K4_ri phi_r),  K4 = -a/6
//   rhobar_i     = norm sum_r BR_ri - Phi / N_eff,  Phi = norm sum_{r,i} rho_i BR_ri
// ================================================================================================
__global__ void vjp_cotangent_kernel(int nb, int n, const double *__restrict__ fbar, const double *__restrict__ Dbar,
                                     const double *__restrict__ ups, double *__restrict__ Rq, double *__restrict__ Dq) {
    const long long nn = (long long)n * n, total = (long long)nb * nn;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long e = idx % nn;
        const int mu = (int)(e / n), nu = (int)(e % n);
        Dq[idx] = 2.0 * ups[mu] * ups[nu] * Dbar[idx];
        if (e < n) Rq[(idx / nn) * n + e] = fbar[(idx / nn) * n + e] / ups[e];
    }
}

__global__ void build_YX_kernel(const double *Y, const double *Xt, int N, int n, long long np, double *YX) {
    const long long total = 2LL * N * np;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long k = idx / np, m = idx % np;
        YX[idx] = m < n ? ((k < N) ? Y[k * n + m] : Xt[(k - N) * n + m]) : 0.0;
    }
}

__global__ void vjp_coef_kernel(long long M, int N, long long ld, const double *__restrict__ D1, const double *__restrict__ Dcd,
                                const double *__restrict__ DA, const double *__restrict__ DC, int d4, double *__restrict__ K1,
                                double *__restrict__ K2, double *__restrict__ K3, double *__restrict__ K4, double *__restrict__ BR) {
    const long long total = M * N;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long r = idx / N, i = idx % N;
        const double a = D1[r * ld + i], b = D1[r * ld + N + i], c = Dcd[r * ld + i], d = Dcd[r * ld + N + i];
        const double Ap = DA[r * ld + i], Bp = DA[r * ld + N + i], Cp = DC[r * ld + i], Dp = DC[r * ld + N + i];
        const double k2 = -c / 3.0 + (d4 ? a / 8.0 : 0.0);
        K1[idx] = (d4 ? Ap / 8.0 : 0.0) - Dp / 3.0;
        K2[idx] = k2;
        K3[idx] = -Ap / 6.0;
        K4[idx] = -a / 6.0;
        BR[idx] = 0.5 * (-d / 3.0 + (d4 ? b / 4.0 : 0.0)) * Ap + k2 * Bp - a / 6.0 * Cp - b / 3.0 * Dp;
    }
}

// colsum[i] += sum_r BR[r][i]
__global__ void vjp_colsum_kernel(long long M, int N, const double *__restrict__ BR, double *__restrict__ colsum) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double s = 0.0;
    for (long long r = 0; r < M; ++r) s += BR[r * N + i];
    colsum[i] += s;
}

// gbar_i += d/dg_i sum_p Vbar[i][p] V[N+i][p] with V[N+i][(mu nu)] = x_mu g_nu + x_nu g_mu off the
// diagonal and x_mu g_mu on it; one CTA per i, one warp per row mu of the packed triangle
template <typename T>
__global__ void vjp_matvec_kernel(int N, int n, long long Kp, long long np, const T *__restrict__ Vbar,
                                  const double *__restrict__ X, T *__restrict__ gbar) {
    extern __shared__ double gs[];
    const int i = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const double *x = X + (long long)i * n;
    const T *vb = Vbar + (long long)i * Kp;
    for (int m = threadIdx.x; m < n; m += blockDim.x) gs[m] = 0.0;
    __syncthreads();
    for (int mu = warp; mu < n; mu += nw) {
        const long long row = (long long)mu * n - ((long long)mu * (mu - 1)) / 2 - mu;   // + nu gives pair(mu, nu)
        const double xm = x[mu];
        double own = 0.0;
        for (int nu = mu + lane; nu < n; nu += 32) {
            const double v = (double)vb[row + nu];
            if (nu == mu) {
                own += v * xm;   // V[N+i, (mu mu)] = x_mu g_mu
            } else {
                own += v * x[nu];
                atomicAdd(&gs[nu], v * xm);
            }
        }
        for (int o = 16; o > 0; o >>= 1) own += __shfl_down_sync(0xffffffffu, own, o);
        if (lane == 0) atomicAdd(&gs[mu], own);
    }
    __syncthreads();
    for (int m = threadIdx.x; m < n; m += blockDim.x) gbar[(long long)i * np + m] = (T)((double)gbar[(long long)i * np + m] + gs[m]);
}

template <typename T>
__global__ void vjp_final_kernel(int N, int n, long long np, double norm, const double *__restrict__ rho,
                                 const double *__restrict__ psi, const T *__restrict__ gbar, const T *__restrict__ ypart,
                                 double *__restrict__ Ybar) {
    const long long total = (long long)N * n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long i = idx / n, m = idx % n;
        Ybar[idx] = norm * rho[i] * (psi[m] * (double)gbar[i * np + m] + (double)ypart[i * np + m]);
    }
}

// Phi = norm sum_i rho_i colsum_i (one CTA, deterministic), rhobar_i = norm colsum_i - Phi / N_eff
__global__ void vjp_rho_kernel(int N, double norm, double N_eff, const double *__restrict__ rho,
                               const double *__restrict__ colsum, double *__restrict__ rhobar) {
    __shared__ double red[256];
    double s = 0.0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) s += rho[i] * colsum[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    const double Phi = norm * red[0];
    for (int i = threadIdx.x; i < N; i += blockDim.x) rhobar[i] = norm * colsum[i] - Phi / N_eff;
}

// row-major C (N x K) (+)= A^T B with A (M x N), B (M x K) row-major
static int gemm_atb(tdscha_ensemble *e, const double *A, long long lda, const double *B, long long ldb, long long M, long long N,
                    long long K, double *C, long long ldc, bool accumulate, cudaStream_t st) {
    const double one = 1.0, beta = accumulate ? 1.0 : 0.0;
    cublasSetStream(e->cublas, st);
    cublasStatus_t s = cublasDgemm(e->cublas, CUBLAS_OP_N, CUBLAS_OP_T, (int)K, (int)N, (int)M, &one, B, (int)ldb, A, (int)lda,
                                   &beta, C, (int)ldc);
    TD_CHECK(s == CUBLAS_STATUS_SUCCESS, TDSCHA_ECUDA, "cublasDgemm failed (%d)", (int)s);
    return 0;
}

// ---- the VJP with the contractions on the tensor cores (mixed storage formats) ----------------------
// K1..K4 of the FP64 path, written transposed (N x Mp, rows r contiguous, zero for r >= M) in the
// storage format, through 32 x 32 shared-memory tiles; BR (M x N, FP64) row-major as in the FP64 path.
__global__ void vjp_coef_mixed_kernel(long long M, int N, long long ld, long long Mp, const float *__restrict__ D1,
                                      const float *__restrict__ Dcd, const float *__restrict__ DA, const float *__restrict__ DC,
                                      int d4, Format fmt, void *K1h, void *K1l, void *K2h, void *K2l, void *K3h, void *K3l,
                                      void *K4h, void *K4l, double *__restrict__ BR) {
    __shared__ float tile[4][32][33];
    const long long r0 = (long long)blockIdx.y * 32;
    const int i0 = blockIdx.x * 32;
    for (int rr = threadIdx.y; rr < 32; rr += blockDim.y) {
        const long long r = r0 + rr;
        const int i = i0 + threadIdx.x;
        float k1 = 0.f, k2 = 0.f, k3 = 0.f, k4 = 0.f;
        if (r < M && i < N) {
            const double a = D1[r * ld + i], b = D1[r * ld + N + i], c = Dcd[r * ld + i], d = Dcd[r * ld + N + i];
            const double Ap = DA[r * ld + i], Bp = DA[r * ld + N + i], Cp = DC[r * ld + i], Dp = DC[r * ld + N + i];
            const double kk2 = -c / 3.0 + (d4 ? a / 8.0 : 0.0);
            k1 = (float)((d4 ? Ap / 8.0 : 0.0) - Dp / 3.0);
            k2 = (float)kk2;
            k3 = (float)(-Ap / 6.0);
            k4 = (float)(-a / 6.0);
            BR[r * N + i] = 0.5 * (-d / 3.0 + (d4 ? b / 4.0 : 0.0)) * Ap + kk2 * Bp - a / 6.0 * Cp - b / 3.0 * Dp;
        }
        tile[0][rr][threadIdx.x] = k1;
        tile[1][rr][threadIdx.x] = k2;
        tile[2][rr][threadIdx.x] = k3;
        tile[3][rr][threadIdx.x] = k4;
    }
    __syncthreads();
    for (int ii = threadIdx.y; ii < 32; ii += blockDim.y) {
        const int i = i0 + ii;
        const long long r = r0 + threadIdx.x;
        if (i < N && r < Mp) {
            const long long o = (long long)i * Mp + r;
            store_split(fmt, K1h, K1l, o, tile[0][threadIdx.x][ii]);
            store_split(fmt, K2h, K2l, o, tile[1][threadIdx.x][ii]);
            store_split(fmt, K3h, K3l, o, tile[2][threadIdx.x][ii]);
            store_split(fmt, K4h, K4l, o, tile[3][threadIdx.x][ii]);
        }
    }
}

// dst (C x Rp) = src^T for src (R x C, leading dimension lds), zero for rows r in [R, Rp); elements of
// 2 (bf16) or 4 (tf32) bytes moved as raw bits
template <typename E>
__global__ void transpose_pad_kernel(const E *__restrict__ src, long long R, long long C, long long lds, long long Rp,
                                     E *__restrict__ dst) {
    __shared__ E tile[32][33];
    const long long c0 = (long long)blockIdx.x * 32, r0 = (long long)blockIdx.y * 32;
    for (int rr = threadIdx.y; rr < 32; rr += blockDim.y) {
        const long long r = r0 + rr, c = c0 + threadIdx.x;
        tile[rr][threadIdx.x] = (r < R && c < C) ? src[r * lds + c] : E(0);
    }
    __syncthreads();
    for (int cc = threadIdx.y; cc < 32; cc += blockDim.y) {
        const long long c = c0 + cc, r = r0 + threadIdx.x;
        if (c < C && r < Rp) dst[c * Rp + r] = tile[threadIdx.x][cc];
    }
}

static int transpose_pad(Format fmt, const void *src, long long R, long long C, long long lds, long long Rp, void *dst,
                         cudaStream_t st) {
    if (!src) return 0;
    dim3 grid((unsigned)ceil_div(C, 32), (unsigned)ceil_div(Rp, 32)), block(32, 8);
    TD_CHECK(grid.y <= 65535, TDSCHA_EINVAL, "transpose of %lld rows exceeds the grid", Rp);
    if (fmt == FMT_BF16)
        transpose_pad_kernel<uint16_t><<<grid, block, 0, st>>>(static_cast<const uint16_t *>(src), R, C, lds, Rp,
                                                                static_cast<uint16_t *>(dst));
    else
        transpose_pad_kernel<float><<<grid, block, 0, st>>>(static_cast<const float *>(src), R, C, lds, Rp,
                                                             static_cast<float *>(dst));
    TD_CUDA(cudaGetLastError());
    return 0;
}

// [Y ; X~] (2N x np) in a storage format, built once per format
static int ensure_YX_fmt(tdscha_ensemble *e, Format fmt, bool lo, cudaStream_t st) {
    const int f = (int)fmt;
    if (e->YXm_hi[f] && (e->YXm_lo[f] || !lo)) return 0;
    const size_t es = format_bytes(fmt), cnt = (size_t)e->N2 * e->np;
    if (!e->YXm_hi[f]) TD_CUDA(cudaMalloc(&e->YXm_hi[f], cnt * es));
    if (lo && !e->YXm_lo[f]) TD_CUDA(cudaMalloc(&e->YXm_lo[f], cnt * es));
    // [Y ; X~] is [X ; G] with (X, G) -> (Y, X~)
    build_XG_kernel<<<grid_for((long long)cnt), 256, 0, st>>>(e->Y, e->Xt, e->N, e->n, e->np, fmt, e->YXm_hi[f],
                                                             lo ? e->YXm_lo[f] : nullptr);
    TD_CUDA(cudaGetLastError());
    return 0;
}

static int perturb_average_vjp_mixed(tdscha_ensemble *e, int nb, const double *R1, const double *Ys, int apply_d4,
                                     int precision, const double *fbar, const double *Dbar, double *Ybar, double *rhobar,
                                     cudaStream_t st) {
    const Format fmt = format_of(precision);
    const int nprod = products_of(precision);
    const bool lo = nprod == 3;
    const size_t es = format_bytes(fmt), nh = lo ? 2 : 1;
    TD_TRY(ensure_operands(e, fmt, lo, st));
    TD_TRY(ensure_YX_fmt(e, fmt, lo, st));
    OperandSet &o = e->ops[fmt];
    const int N = e->N, n = e->n;
    const long long Kp = e->Kp, np = e->np, ld1 = round_up(e->N2, 4);
    // memory plan: fixed buffers, then per symmetry row (M = nb * Jc rows, Mp = M rounded to 64)
    const size_t fixed = 4 * ((size_t)N * Kp + 2 * (size_t)N * np) + 8 * ((size_t)N + (size_t)nb * n + (size_t)nb * n * n) +
                         16 * 256;
    const size_t per_row = es * nh * (4 * (size_t)Kp + 4 * (size_t)np + 4 * (size_t)N) + 4 * 4 * (size_t)ld1 + 8 * (size_t)N;
    size_t free_b = 0, tot_b = 0;
    TD_CUDA(cudaMemGetInfo(&free_b, &tot_b));
    const size_t budget = std::max<size_t>((size_t)1 << 30, (size_t)((free_b + e->vjp_ws.bytes) * 0.5));
    TD_CHECK(budget > fixed + per_row * (nb + 64), TDSCHA_ENOMEM, "not enough device memory for the averages' VJP");
    int Jc = (int)std::min<long long>(e->N_sym, (long long)((budget - fixed) / per_row - 64) / nb);
    Jc = std::max(1, Jc);
    const long long Mmax = (long long)nb * Jc, Mpmax = round_up(Mmax, 64);
    const size_t need = fixed + per_row * (size_t)Mpmax + 64 * 256;
    if (e->vjp_ws.bytes < need) {
        if (e->vjp_ws.base) { TD_CUDA(cudaDeviceSynchronize()); cudaFree(e->vjp_ws.base); e->vjp_ws = Workspace(); }
        TD_CUDA(cudaMalloc(&e->vjp_ws.base, need));
        e->vjp_ws.bytes = need;
    }
    uint8_t *W = static_cast<uint8_t *>(e->vjp_ws.base);
    size_t off = 0;
    auto take = [&](size_t bytes) { void *p = W + off; off += (bytes + 255) / 256 * 256; return p; };
    float *Vbar = static_cast<float *>(take(4 * (size_t)N * Kp));
    float *gbar = static_cast<float *>(take(4 * (size_t)N * np)), *ypart = static_cast<float *>(take(4 * (size_t)N * np));
    double *colsum = static_cast<double *>(take(8 * (size_t)N));
    double *Rq = static_cast<double *>(take(8 * (size_t)nb * n)), *Dq = static_cast<double *>(take(8 * (size_t)nb * n * n));
    auto pair_of = [&](size_t count) {
        void *h = take(count * es);
        void *l = lo ? take(count * es) : nullptr;
        return std::make_pair(h, l);
    };
    auto B1 = pair_of(Mmax * Kp), Q = pair_of(Mmax * Kp), r1 = pair_of(Mmax * np), phi = pair_of(Mmax * np);
    auto B1T = pair_of(Kp * Mpmax), QT = pair_of(Kp * Mpmax), r1T = pair_of(np * Mpmax), phiT = pair_of(np * Mpmax);
    auto K1 = pair_of((size_t)N * Mpmax), K2 = pair_of((size_t)N * Mpmax), K3 = pair_of((size_t)N * Mpmax),
         K4 = pair_of((size_t)N * Mpmax);
    float *D1 = static_cast<float *>(take(4 * Mmax * ld1)), *Dcd = static_cast<float *>(take(4 * Mmax * ld1));
    float *DA = static_cast<float *>(take(4 * Mmax * ld1)), *DC = static_cast<float *>(take(4 * Mmax * ld1));
    double *BR = static_cast<double *>(take(8 * Mmax * (size_t)N));
    TD_CHECK(off <= e->vjp_ws.bytes, TDSCHA_EINVAL, "VJP workspace layout exceeds its allocation");
    TD_CUDA(cudaMemsetAsync(gbar, 0, 4 * (size_t)N * np, st));
    TD_CUDA(cudaMemsetAsync(ypart, 0, 4 * (size_t)N * np, st));
    TD_CUDA(cudaMemsetAsync(colsum, 0, 8 * (size_t)N, st));
    vjp_cotangent_kernel<<<grid_for((long long)nb * n * n), 256, 0, st>>>(nb, n, fbar, Dbar, e->ups, Rq, Dq);
    TD_CUDA(cudaGetLastError());

    SymTables t{e->sym, e->d_blk_sym_off, e->d_blk_start, e->d_blk_dim, e->n_blocks, e->n, e->dmax, e->symP, e->symPT, e->d_offP};
    bool first = true;
    for (int j0 = 0; j0 < e->N_sym; j0 += Jc) {
        const int nj = std::min(Jc, e->N_sym - j0);
        const long long M = (long long)nb * nj, Mp = round_up(M, 64);
        TD_TRY(sym_transform(t, e->pairs, nb, nj, j0, Ys, R1, e->ups, e->P, Kp, np, fmt, B1.first, B1.second, r1.first,
                             r1.second, true, st));
        TD_TRY(sym_transform(t, e->pairs, nb, nj, j0, Dq, Rq, e->ups, e->P, Kp, np, fmt, Q.first, Q.second, phi.first,
                             phi.second, true, st));
        // forward contractions: [a | b], [c | d], [A' | B'], [C' | D']   (M x 2N each)
        TD_TRY(gemm_abt(e, fmt, nprod, B1.first, B1.second, Kp, M, o.V_hi, o.V_lo, Kp, e->N2, Kp, D1, ld1, st));
        TD_TRY(gemm_abt(e, fmt, nprod, r1.first, r1.second, np, M, o.XG_hi, o.XG_lo, np, e->N2, np, Dcd, ld1, st));
        TD_TRY(gemm_abt(e, fmt, nprod, Q.first, Q.second, Kp, M, o.V_hi, o.V_lo, Kp, e->N2, Kp, DA, ld1, st));
        TD_TRY(gemm_abt(e, fmt, nprod, phi.first, phi.second, np, M, e->YXm_hi[fmt], lo ? e->YXm_lo[fmt] : nullptr, np,
                        e->N2, np, DC, ld1, st));
        {
            dim3 grid((unsigned)ceil_div(N, 32), (unsigned)ceil_div(Mp, 32)), block(32, 8);
            TD_CHECK(grid.y <= 65535, TDSCHA_EINVAL, "VJP coefficient grid too large");
            vjp_coef_mixed_kernel<<<grid, block, 0, st>>>(M, N, ld1, Mp, D1, Dcd, DA, DC, apply_d4, fmt, K1.first, K1.second,
                                                          K2.first, K2.second, K3.first, K3.second, K4.first, K4.second, BR);
            TD_CUDA(cudaGetLastError());
        }
        // the contraction index is the row r = (k, j): transpose the row-major left operands
        for (auto pr : {std::make_pair(B1, B1T), std::make_pair(Q, QT)}) {
            TD_TRY(transpose_pad(fmt, pr.first.first, M, Kp, Kp, Mp, pr.second.first, st));
            TD_TRY(transpose_pad(fmt, pr.first.second, M, Kp, Kp, Mp, pr.second.second, st));
        }
        for (auto pr : {std::make_pair(r1, r1T), std::make_pair(phi, phiT)}) {
            TD_TRY(transpose_pad(fmt, pr.first.first, M, np, np, Mp, pr.second.first, st));
            TD_TRY(transpose_pad(fmt, pr.first.second, M, np, np, Mp, pr.second.second, st));
        }
        // transposed contractions over the rows: Vbar (+)= K1^T B1 + K2^T Q, gbar += K3^T r1, ypart += K4^T phi
        TD_TRY(gemm_abt(e, fmt, nprod, K1.first, K1.second, Mp, N, B1T.first, B1T.second, Mp, Kp, Mp, Vbar, Kp, st, !first));
        TD_TRY(gemm_abt(e, fmt, nprod, K2.first, K2.second, Mp, N, QT.first, QT.second, Mp, Kp, Mp, Vbar, Kp, st, true));
        TD_TRY(gemm_abt(e, fmt, nprod, K3.first, K3.second, Mp, N, r1T.first, r1T.second, Mp, np, Mp, gbar, np, st, true));
        TD_TRY(gemm_abt(e, fmt, nprod, K4.first, K4.second, Mp, N, phiT.first, phiT.second, Mp, np, Mp, ypart, np, st, true));
        vjp_colsum_kernel<<<ceil_div(N, 256), 256, 0, st>>>(M, N, BR, colsum);
        TD_CUDA(cudaGetLastError());
        first = false;
    }
    const double norm = 1.0 / (e->N_eff * (double)e->N_sym);
    vjp_matvec_kernel<float><<<N, 256, (size_t)n * sizeof(double), st>>>(N, n, Kp, np, Vbar, e->X, gbar);
    vjp_final_kernel<float><<<grid_for((long long)N * n), 256, 0, st>>>(N, n, np, norm, e->rho, e->psi, gbar, ypart, Ybar);
    vjp_rho_kernel<<<1, 256, 0, st>>>(N, norm, e->N_eff, e->rho, colsum, rhobar);
    TD_CUDA(cudaGetLastError());
    return 0;
}

// TDSCHA_VJP_FREQ=0 keeps the averages' VJP on the rows over every symmetry (read at every call).
static bool vjp_freq_enabled() {
    const char *env = getenv("TDSCHA_VJP_FREQ");
    return !(env && atoi(env) == 0);
}

// ------------------------------------------------------------------------------------------------
// The averages' VJP on the character classes (freq.cuh): the forward quantities and the cotangent
// transforms class by class, coefficients in the character basis, transposed contractions over the
// class rows.  Inputs in the ensemble's rotated basis; resident class operands (no configuration
// chunks).
// ------------------------------------------------------------------------------------------------
static int ensure_freq_yx_rows(tdscha_ensemble *e, Format fmt, bool lo, cudaStream_t st) {
    const FreqTables &ft = *e->freq;
    if (ft.Kmq == 0) return 0;
    if (e->fyx_hi[fmt] && (!lo || e->fyx_lo[fmt])) return 0;
    const size_t bytes = (size_t)e->N2 * ft.Kmq * format_bytes(fmt);
    if (!e->fyx_hi[fmt]) TD_CUDA(cudaMalloc(&e->fyx_hi[fmt], bytes));
    if (lo && !e->fyx_lo[fmt]) TD_CUDA(cudaMalloc(&e->fyx_lo[fmt], bytes));
    return freq_build_mode_rows(ft, e->Y, e->Xt, e->n, e->N, fmt, e->fyx_hi[fmt], lo ? e->fyx_lo[fmt] : nullptr, st);
}

static int perturb_average_vjp_freq(tdscha_ensemble *e, int nb, const double *R1, const double *Ys, int apply_d4,
                                    const double *fbar, const double *Dbar, double *Ybar, double *rhobar, cudaStream_t st,
                                    Format fmt, int nprod, bool lo) {
    const FreqTables &ft = *e->freq;
    const SymCosets *cs = e->cosets;
    const int n_cos = cs->n_cos, sub = cs->sub, nC = ft.n_class, N = e->N, n = e->n;
    const bool f64 = fmt == FMT_F64;
    const size_t es = format_bytes(fmt), as = f64 ? 8 : 4, nh = lo ? 2 : 1;
    const long long Kq = ft.Kq, Kmq1 = std::max(ft.Kmq, 1), ld1 = round_up(e->N2, 4);
    TD_TRY(ensure_freq_operands(e, fmt, lo, st));
    TD_TRY(ensure_freq_yx_rows(e, fmt, lo, st));
    const FreqOps &co = e->fops[fmt];
    // workspace: fixed part, then per coset (NR = nb * cosets of the chunk, NRp = NR rounded to 64)
    const size_t fixed = as * ((size_t)N * Kq + 2 * (size_t)N * Kmq1 + (size_t)N * e->Kp + 2 * (size_t)N * e->np) +
                         8 * ((size_t)N + (size_t)nb * n + (size_t)nb * n * n) + 32 * 256;
    auto per_chunk = [&](int ncj) {
        const size_t NR = (size_t)nb * ncj, NRp = round_up(NR, 64), rows = (size_t)nC * 2 * NR;
        size_t b = 2 * as * (NR * e->Kp + NR * e->np);                      // U, r1, Q, phi
        b += 2 * es * nh * (2 * NR * Kq + 2 * NR * Kmq1);                    // Lab, LQ, Lcd, Lphi
        if (!f64) b += 2 * es * nh * ((size_t)Kq * 2 * NRp + (size_t)Kmq1 * 2 * NRp);   // their transposes
        b += 4 * as * rows * ld1;                                            // H, Ch, HQ, Cp
        b += f64 ? 4 * 8 * rows * ld1 : 4 * es * nh * (size_t)N * nC * 2 * NRp;   // K1..K4
        b += 8 * rows * (size_t)N;                                           // BR
        return b + 32 * 256;
    };
    size_t free_b = 0, tot_b = 0;
    TD_CUDA(cudaMemGetInfo(&free_b, &tot_b));
    const size_t budget = std::max<size_t>((size_t)1 << 30, (size_t)((free_b + e->vjp_ws.bytes) * 0.5));
    TD_CHECK(budget > fixed + per_chunk(1), TDSCHA_ENOMEM, "not enough device memory for the averages' VJP");
    int ncj = n_cos;
    while (ncj > 1 && fixed + per_chunk(ncj) > budget) ncj = (ncj + 1) / 2;
    const size_t need = fixed + per_chunk(ncj);
    if (e->vjp_ws.bytes < need) {
        if (e->vjp_ws.base) { TD_CUDA(cudaDeviceSynchronize()); cudaFree(e->vjp_ws.base); e->vjp_ws = Workspace(); }
        TD_CUDA(cudaMalloc(&e->vjp_ws.base, need));
        e->vjp_ws.bytes = need;
    }
    uint8_t *W = static_cast<uint8_t *>(e->vjp_ws.base);
    size_t off = 0;
    auto take = [&](size_t bytes) { void *p = W + off; off += (bytes + 255) / 256 * 256; return p; };
    const long long NRmax = (long long)nb * ncj, NRpmax = round_up(NRmax, 64), rowsmax = (long long)nC * 2 * NRmax;
    void *VbarQ = take(as * (size_t)N * Kq), *GQ = take(as * (size_t)N * Kmq1), *YQ = take(as * (size_t)N * Kmq1);
    void *Vbar = take(as * (size_t)N * e->Kp), *gbar = take(as * (size_t)N * e->np), *ypart = take(as * (size_t)N * e->np);
    double *colsum = static_cast<double *>(take(8 * (size_t)N));
    double *Rq = static_cast<double *>(take(8 * (size_t)nb * n)), *Dq = static_cast<double *>(take(8 * (size_t)nb * n * n));
    void *U = take(as * NRmax * e->Kp), *r1 = take(as * NRmax * e->np), *Q = take(as * NRmax * e->Kp), *phi = take(as * NRmax * e->np);
    auto pair_of = [&](size_t count) { void *h = take(count * es); void *l = lo ? take(count * es) : nullptr; return std::make_pair(h, l); };
    auto Lab = pair_of(2 * NRmax * Kq), LQ = pair_of(2 * NRmax * Kq), Lcd = pair_of(2 * NRmax * Kmq1), Lph = pair_of(2 * NRmax * Kmq1);
    std::pair<void *, void *> LabT{nullptr, nullptr}, LQT{nullptr, nullptr}, LcdT{nullptr, nullptr}, LphT{nullptr, nullptr};
    if (!f64) {
        LabT = pair_of((size_t)Kq * 2 * NRpmax);
        LQT = pair_of((size_t)Kq * 2 * NRpmax);
        LcdT = pair_of((size_t)Kmq1 * 2 * NRpmax);
        LphT = pair_of((size_t)Kmq1 * 2 * NRpmax);
    }
    void *H = take(as * rowsmax * ld1), *Ch = take(as * rowsmax * ld1), *HQ = take(as * rowsmax * ld1), *Cp = take(as * rowsmax * ld1);
    std::pair<void *, void *> Ks[4];
    for (auto &k : Ks) k = f64 ? std::make_pair(take(8 * rowsmax * ld1), (void *)nullptr) : pair_of((size_t)N * nC * 2 * NRpmax);
    double *BR = static_cast<double *>(take(8 * rowsmax * (size_t)N));
    TD_CHECK(off <= e->vjp_ws.bytes, TDSCHA_EINVAL, "VJP workspace layout exceeds its allocation");
    TD_CUDA(cudaMemsetAsync(colsum, 0, 8 * (size_t)N, st));
    vjp_cotangent_kernel<<<grid_for((long long)nb * n * n), 256, 0, st>>>(nb, n, fbar, Dbar, e->ups, Rq, Dq);
    TD_CUDA(cudaGetLastError());
    SymTables tr{e->sym, e->d_blk_sym_off, e->d_blk_start, e->d_blk_dim, e->n_blocks, e->n, e->dmax, cs->repP, cs->repPT, cs->d_offRep};
    SymTables t64{cs->repS, cs->d_offRepS, e->d_blk_start, e->d_blk_dim, e->n_blocks, e->n, e->dmax, nullptr, nullptr, nullptr};
    bool first = true;
    for (int p0 = 0; p0 < n_cos; p0 += ncj) {
        const int nc = std::min(ncj, n_cos - p0);
        const int NR = nb * nc, NRp = (int)round_up(NR, 64);
        const long long RT = (long long)nC * 2 * NRp, rows = (long long)nC * 2 * NR;
        // transforms over the representatives and left operands
        if (f64) {
            TD_TRY(sym_transform(t64, e->pairs, nb, nc, p0, Ys, R1, e->ups, e->P, e->Kp, e->np, FMT_F64, U, nullptr, r1, nullptr, false, st));
            TD_TRY(sym_transform(t64, e->pairs, nb, nc, p0, Dq, Rq, e->ups, e->P, e->Kp, e->np, FMT_F64, Q, nullptr, phi, nullptr, false, st));
            TD_TRY(freq_left<double>(ft, NR, n, (const double *)U, e->Kp, (const double *)r1, e->np, fmt, Lab.first, Lab.second,
                                     Lcd.first, Lcd.second, st));
            TD_TRY(freq_left<double>(ft, NR, n, (const double *)Q, e->Kp, (const double *)phi, e->np, fmt, LQ.first, LQ.second,
                                     Lph.first, Lph.second, st));
        } else {
            TD_TRY(sym_transform_tc(tr, e->pairs, nb, nc, p0, Ys, R1, e->ups, e->Kp, e->np, FMT_F32, U, nullptr, r1, nullptr, st));
            TD_TRY(sym_transform_tc(tr, e->pairs, nb, nc, p0, Dq, Rq, e->ups, e->Kp, e->np, FMT_F32, Q, nullptr, phi, nullptr, st));
            TD_TRY(freq_left<float>(ft, NR, n, (const float *)U, e->Kp, (const float *)r1, e->np, fmt, Lab.first, Lab.second,
                                    Lcd.first, Lcd.second, st));
            TD_TRY(freq_left<float>(ft, NR, n, (const float *)Q, e->Kp, (const float *)phi, e->np, fmt, LQ.first, LQ.second,
                                    Lph.first, Lph.second, st));
        }
        // forward class contractions: [a|b], [c|d] of (U, r1) and [A'|B'], [C'|D'] of (Q, phi)
        std::vector<tc::GemmGroup> gab, gcd;
        for (int g = 0; g < nC; ++g) {
            const int Mg = ft.cls_real[g] ? NR : 2 * NR;
            const long long hrow = (long long)g * 2 * NR;
            gab.push_back({Mg, (int)e->N2, ft.pcol_cnt[g], 0, ft.pcol_off[g], 0, ft.pcol_off[g], hrow * ld1});
            if (ft.mcol_cnt[g] > 0) {
                gcd.push_back({Mg, (int)e->N2, ft.mcol_cnt[g], 0, ft.mcol_off[g], 0, ft.mcol_off[g], hrow * ld1});
            } else {
                TD_CUDA(cudaMemsetAsync(static_cast<uint8_t *>(Ch) + hrow * ld1 * as, 0, (size_t)2 * NR * ld1 * as, st));
                TD_CUDA(cudaMemsetAsync(static_cast<uint8_t *>(Cp) + hrow * ld1 * as, 0, (size_t)2 * NR * ld1 * as, st));
            }
        }
        TD_TRY(gemm_groups(e, fmt, nprod, Lab.first, Lab.second, 2LL * NR, Kq, co.V_hi, co.V_lo, e->N2, Kq, gab, H, ld1, false, st));
        TD_TRY(gemm_groups(e, fmt, nprod, LQ.first, LQ.second, 2LL * NR, Kq, co.V_hi, co.V_lo, e->N2, Kq, gab, HQ, ld1, false, st));
        TD_TRY(gemm_groups(e, fmt, nprod, Lcd.first, Lcd.second, 2LL * NR, Kmq1, co.XG_hi, co.XG_lo, e->N2, Kmq1, gcd, Ch, ld1, false, st));
        TD_TRY(gemm_groups(e, fmt, nprod, Lph.first, Lph.second, 2LL * NR, Kmq1, e->fyx_hi[fmt], lo ? e->fyx_lo[fmt] : nullptr,
                           e->N2, Kmq1, gcd, Cp, ld1, false, st));
        // coefficients and the rho pairing
        void *Kh[4] = {Ks[0].first, Ks[1].first, Ks[2].first, Ks[3].first};
        void *Kl[4] = {Ks[0].second, Ks[1].second, Ks[2].second, Ks[3].second};
        if (f64) {
            TD_TRY(freq_vjp_coef<double>(ft, sub, (const double *)H, (const double *)Ch, (const double *)HQ, (const double *)Cp, ld1,
                                         N, NR, NRp, apply_d4, false, fmt, Kh, Kl, ld1, BR, st));
        } else {
            for (int q = 0; q < 4; ++q) {
                TD_CUDA(cudaMemsetAsync(Kh[q], 0, (size_t)N * RT * es, st));
                if (lo) TD_CUDA(cudaMemsetAsync(Kl[q], 0, (size_t)N * RT * es, st));
            }
            TD_TRY(freq_vjp_coef<float>(ft, sub, (const float *)H, (const float *)Ch, (const float *)HQ, (const float *)Cp, ld1, N,
                                        NR, NRp, apply_d4, true, fmt, Kh, Kl, RT, BR, st));
        }
        vjp_colsum_kernel<<<ceil_div(N, 256), 256, 0, st>>>(rows, N, BR, colsum);
        TD_CUDA(cudaGetLastError());
        // transposed contractions over the class rows
        if (f64) {
            std::vector<std::array<long long, 5>> gp, gm;
            for (int g = 0; g < nC; ++g) {
                const long long row0 = (long long)g * 2 * NR, nr = ft.cls_real[g] ? NR : 2 * NR;
                gp.push_back({row0, nr, ft.pcol_off[g], ft.pcol_cnt[g], 0});
                if (ft.mcol_cnt[g] > 0) gm.push_back({row0, nr, ft.mcol_off[g], ft.mcol_cnt[g], 0});
            }
            // the left operands' rows start at 0 for every class: offset K by the class block, R by 0
            auto run = [&](const std::vector<std::array<long long, 5>> &gs, const double *K, const void *R, long long ldr, void *C,
                           long long ldc, bool acc) {
                const double one = 1.0, beta = acc ? 1.0 : 0.0;
                cublasSetStream(e->cublas, st);
                for (const auto &g : gs) {
                    cublasStatus_t s2 = cublasDgemm(e->cublas, CUBLAS_OP_N, CUBLAS_OP_T, (int)g[3], N, (int)g[1], &one,
                                                    static_cast<const double *>(R) + g[2], (int)ldr, K + g[0] * ld1, (int)ld1, &beta,
                                                    static_cast<double *>(C) + g[2], (int)ldc);
                    TD_CHECK(s2 == CUBLAS_STATUS_SUCCESS, TDSCHA_ECUDA, "cublasDgemm failed (%d)", (int)s2);
                }
                return 0;
            };
            TD_TRY(run(gp, (const double *)Kh[0], Lab.first, Kq, VbarQ, Kq, !first));
            TD_TRY(run(gp, (const double *)Kh[1], LQ.first, Kq, VbarQ, Kq, true));
            TD_TRY(run(gm, (const double *)Kh[2], Lcd.first, Kmq1, GQ, Kmq1, !first));
            TD_TRY(run(gm, (const double *)Kh[3], Lph.first, Kmq1, YQ, Kmq1, !first));
        } else {
            TD_TRY(freq_transpose_left(fmt, Lab.first, NR, NRp, Kq, LabT.first, st));
            TD_TRY(freq_transpose_left(fmt, LQ.first, NR, NRp, Kq, LQT.first, st));
            TD_TRY(freq_transpose_left(fmt, Lcd.first, NR, NRp, Kmq1, LcdT.first, st));
            TD_TRY(freq_transpose_left(fmt, Lph.first, NR, NRp, Kmq1, LphT.first, st));
            if (lo) {
                TD_TRY(freq_transpose_left(fmt, Lab.second, NR, NRp, Kq, LabT.second, st));
                TD_TRY(freq_transpose_left(fmt, LQ.second, NR, NRp, Kq, LQT.second, st));
                TD_TRY(freq_transpose_left(fmt, Lcd.second, NR, NRp, Kmq1, LcdT.second, st));
                TD_TRY(freq_transpose_left(fmt, Lph.second, NR, NRp, Kmq1, LphT.second, st));
            }
            std::vector<tc::GemmGroup> gp, gm;
            for (int g = 0; g < nC; ++g) {
                const int Kg = ft.cls_real[g] ? NRp : 2 * NRp;
                const int a_k = g * 2 * NRp;
                gp.push_back({N, ft.pcol_cnt[g], Kg, 0, a_k, ft.pcol_off[g], 0, (long long)ft.pcol_off[g]});
                if (ft.mcol_cnt[g] > 0) gm.push_back({N, ft.mcol_cnt[g], Kg, 0, a_k, ft.mcol_off[g], 0, (long long)ft.mcol_off[g]});
            }
            TD_TRY(gemm_groups(e, fmt, nprod, Kh[0], Kl[0], N, RT, LabT.first, LabT.second, Kq, 2LL * NRp, gp, VbarQ, Kq, !first, st));
            TD_TRY(gemm_groups(e, fmt, nprod, Kh[1], Kl[1], N, RT, LQT.first, LQT.second, Kq, 2LL * NRp, gp, VbarQ, Kq, true, st));
            TD_TRY(gemm_groups(e, fmt, nprod, Kh[2], Kl[2], N, RT, LcdT.first, LcdT.second, Kmq1, 2LL * NRp, gm, GQ, Kmq1, !first, st));
            TD_TRY(gemm_groups(e, fmt, nprod, Kh[3], Kl[3], N, RT, LphT.first, LphT.second, Kmq1, 2LL * NRp, gm, YQ, Kmq1, !first, st));
        }
        first = false;
    }
    const double norm = 1.0 / (e->N_eff * (double)e->N_sym);
    if (f64) {
        TD_TRY(freq_vjp_reconstruct<double>(ft, N, n, e->P, (const double *)VbarQ, (const double *)GQ, (const double *)YQ,
                                            (double *)Vbar, e->Kp, (double *)gbar, (double *)ypart, e->np, st));
        vjp_matvec_kernel<double><<<N, 256, (size_t)n * sizeof(double), st>>>(N, n, e->Kp, e->np, (const double *)Vbar, e->X, (double *)gbar);
        vjp_final_kernel<double><<<grid_for((long long)N * n), 256, 0, st>>>(N, n, e->np, norm, e->rho, e->psi, (const double *)gbar,
                                                                             (const double *)ypart, Ybar);
    } else {
        TD_TRY(freq_vjp_reconstruct<float>(ft, N, n, e->P, (const float *)VbarQ, (const float *)GQ, (const float *)YQ,
                                           (float *)Vbar, e->Kp, (float *)gbar, (float *)ypart, e->np, st));
        vjp_matvec_kernel<float><<<N, 256, (size_t)n * sizeof(double), st>>>(N, n, e->Kp, e->np, (const float *)Vbar, e->X, (float *)gbar);
        vjp_final_kernel<float><<<grid_for((long long)N * n), 256, 0, st>>>(N, n, e->np, norm, e->rho, e->psi, (const float *)gbar,
                                                                            (const float *)ypart, Ybar);
    }
    vjp_rho_kernel<<<1, 256, 0, st>>>(N, norm, e->N_eff, e->rho, colsum, rhobar);
    TD_CUDA(cudaGetLastError());
    return 0;
}

static int vjp_in_ensemble_basis(tdscha_ensemble *e, int nb, const double *R1, const double *Ys, int apply_d4,
                                 const double *fbar, const double *Dbar, double *Ybar, double *rhobar, cudaStream_t st,
                                 int precision) {
    if (e->freq && use_freq_path(e, format_of(precision)) && vjp_freq_enabled()) {
        TD_CHECK(nb > 0, TDSCHA_EINVAL, "nb must be positive");
        TD_CHECK(apply_d4 == 0 || apply_d4 == 1, TDSCHA_EINVAL, "apply_D4 must be 0 or 1 (got %d)", apply_d4);
        TD_CHECK(R1 && Ys && fbar && Dbar && Ybar && rhobar, TDSCHA_EINVAL, "NULL argument");
        TD_CHECK(precision >= 0 && precision <= TDSCHA_PREC_BF16, TDSCHA_EINVAL, "unknown precision %d", precision);
        return perturb_average_vjp_freq(e, nb, R1, Ys, apply_d4, fbar, Dbar, Ybar, rhobar, st, format_of(precision),
                                        products_of(precision), needs_lo(precision));
    }
    if (precision != TDSCHA_PREC_FP64) {
        TD_CHECK(nb > 0, TDSCHA_EINVAL, "nb must be positive");
        TD_CHECK(apply_d4 == 0 || apply_d4 == 1, TDSCHA_EINVAL, "apply_D4 must be 0 or 1 (got %d)", apply_d4);
        TD_CHECK(R1 && Ys && fbar && Dbar && Ybar && rhobar, TDSCHA_EINVAL, "NULL argument");
        TD_CHECK(precision >= 0 && precision <= TDSCHA_PREC_BF16, TDSCHA_EINVAL, "unknown precision %d", precision);
        return perturb_average_vjp_mixed(e, nb, R1, Ys, apply_d4, precision, fbar, Dbar, Ybar, rhobar, st);
    }
    TD_CHECK(nb > 0, TDSCHA_EINVAL, "nb must be positive");
    TD_CHECK(apply_d4 == 0 || apply_d4 == 1, TDSCHA_EINVAL, "apply_D4 must be 0 or 1 (got %d)", apply_d4);
    TD_CHECK(R1 && Ys && fbar && Dbar && Ybar && rhobar, TDSCHA_EINVAL, "NULL argument");
    TD_TRY(ensure_operands(e, FMT_F64, false, st));
    OperandSet &o = e->ops[FMT_F64];
    const int N = e->N, n = e->n;
    if (!e->YX) {
        TD_CUDA(cudaMalloc(&e->YX, (size_t)e->N2 * e->np * sizeof(double)));
        build_YX_kernel<<<grid_for(e->N2 * e->np), 256, 0, st>>>(e->Y, e->Xt, N, n, e->np, e->YX);
        TD_CUDA(cudaGetLastError());
    }
    const long long ld1 = round_up(e->N2, 4);
    // persistent buffers, then per-chunk rows (M = nb * Jc)
    const size_t fixed = 8 * ((size_t)N * e->Kp + 2 * (size_t)N * e->np + N + (size_t)nb * n + (size_t)nb * n * n) + 8 * 256;
    const size_t per_row = 8 * (2 * (size_t)e->Kp + 2 * (size_t)e->np + 4 * (size_t)ld1 + 5 * (size_t)N);
    size_t free_b = 0, tot_b = 0;
    TD_CUDA(cudaMemGetInfo(&free_b, &tot_b));
    const size_t budget = std::max<size_t>((size_t)1 << 30, (size_t)((free_b + e->vjp_ws.bytes) * 0.5));
    TD_CHECK(budget > fixed + per_row * nb, TDSCHA_ENOMEM, "not enough device memory for the averages' VJP");
    int Jc = std::min<long long>(e->N_sym, (long long)((budget - fixed) / (per_row * nb)));
    Jc = std::max(1, Jc);
    const size_t need = fixed + per_row * (size_t)nb * Jc + 16 * 256;
    if (e->vjp_ws.bytes < need) {
        if (e->vjp_ws.base) { TD_CUDA(cudaDeviceSynchronize()); cudaFree(e->vjp_ws.base); e->vjp_ws = Workspace(); }
        TD_CUDA(cudaMalloc(&e->vjp_ws.base, need));
        e->vjp_ws.bytes = need;
    }
    uint8_t *W = static_cast<uint8_t *>(e->vjp_ws.base);
    size_t off = 0;
    auto take = [&](size_t count) { double *p = reinterpret_cast<double *>(W + off); off += (count * 8 + 255) / 256 * 256; return p; };
    double *Vbar = take((size_t)N * e->Kp), *gbar = take((size_t)N * e->np), *ypart = take((size_t)N * e->np);
    double *colsum = take(N), *Rq = take((size_t)nb * n), *Dq = take((size_t)nb * n * n);
    const long long Mmax = (long long)nb * Jc;
    double *B1 = take(Mmax * e->Kp), *Q = take(Mmax * e->Kp), *r1 = take(Mmax * e->np), *phi = take(Mmax * e->np);
    double *D1 = take(Mmax * ld1), *Dcd = take(Mmax * ld1), *DA = take(Mmax * ld1), *DC = take(Mmax * ld1);
    double *K1 = take(Mmax * N), *K2 = take(Mmax * N), *K3 = take(Mmax * N), *K4 = take(Mmax * N), *BR = take(Mmax * N);
    TD_CUDA(cudaMemsetAsync(gbar, 0, (size_t)N * e->np * 8, st));
    TD_CUDA(cudaMemsetAsync(ypart, 0, (size_t)N * e->np * 8, st));
    TD_CUDA(cudaMemsetAsync(colsum, 0, (size_t)N * 8, st));
    vjp_cotangent_kernel<<<grid_for((long long)nb * n * n), 256, 0, st>>>(nb, n, fbar, Dbar, e->ups, Rq, Dq);
    TD_CUDA(cudaGetLastError());

    SymTables t{e->sym, e->d_blk_sym_off, e->d_blk_start, e->d_blk_dim, e->n_blocks, e->n, e->dmax, e->symP, e->symPT, e->d_offP};
    bool first = true;
    for (int j0 = 0; j0 < e->N_sym; j0 += Jc) {
        const int nj = std::min(Jc, e->N_sym - j0);
        const long long M = (long long)nb * nj;
        TD_TRY(sym_transform(t, e->pairs, nb, nj, j0, Ys, R1, e->ups, e->P, e->Kp, e->np, FMT_F64, B1, nullptr, r1, nullptr,
                             false, st));
        TD_TRY(sym_transform(t, e->pairs, nb, nj, j0, Dq, Rq, e->ups, e->P, e->Kp, e->np, FMT_F64, Q, nullptr, phi, nullptr,
                             false, st));
        TD_TRY(gemm_abt(e, FMT_F64, 1, B1, nullptr, e->Kp, M, o.V_hi, nullptr, e->Kp, e->N2, e->Kp, D1, ld1, st));
        TD_TRY(gemm_abt(e, FMT_F64, 1, r1, nullptr, e->np, M, o.XG_hi, nullptr, e->np, e->N2, e->np, Dcd, ld1, st));
        TD_TRY(gemm_abt(e, FMT_F64, 1, Q, nullptr, e->Kp, M, o.V_hi, nullptr, e->Kp, e->N2, e->Kp, DA, ld1, st));
        TD_TRY(gemm_abt(e, FMT_F64, 1, phi, nullptr, e->np, M, e->YX, nullptr, e->np, e->N2, e->np, DC, ld1, st));
        vjp_coef_kernel<<<grid_for(M * N), 256, 0, st>>>(M, N, ld1, D1, Dcd, DA, DC, apply_d4, K1, K2, K3, K4, BR);
        TD_CUDA(cudaGetLastError());
        TD_TRY(gemm_atb(e, K1, N, B1, e->Kp, M, N, e->Kp, Vbar, e->Kp, !first, st));
        TD_TRY(gemm_atb(e, K2, N, Q, e->Kp, M, N, e->Kp, Vbar, e->Kp, true, st));
        TD_TRY(gemm_atb(e, K3, N, r1, e->np, M, N, e->np, gbar, e->np, true, st));
        TD_TRY(gemm_atb(e, K4, N, phi, e->np, M, N, e->np, ypart, e->np, true, st));
        vjp_colsum_kernel<<<ceil_div(N, 256), 256, 0, st>>>(M, N, BR, colsum);
        TD_CUDA(cudaGetLastError());
        first = false;
    }
    const double norm = 1.0 / (e->N_eff * (double)e->N_sym);
    vjp_matvec_kernel<double><<<N, 256, (size_t)n * sizeof(double), st>>>(N, n, e->Kp, e->np, Vbar, e->X, gbar);
    vjp_final_kernel<double><<<grid_for((long long)N * n), 256, 0, st>>>(N, n, e->np, norm, e->rho, e->psi, gbar, ypart, Ybar);
    vjp_rho_kernel<<<1, 256, 0, st>>>(N, norm, e->N_eff, e->rho, colsum, rhobar);
    TD_CUDA(cudaGetLastError());
    return 0;
}

// The ensemble's rotated basis (X' = X R, tables R^T S R): (R1, Ys, fbar, Dbar) are rotated in,
// d/dY = d/dY' . R^T rotated back; rho is unchanged.
int perturb_average_vjp_device(tdscha_ensemble *e, int nb, const double *R1, const double *Ys, int apply_d4,
                               const double *fbar, const double *Dbar, double *Ybar, double *rhobar, cudaStream_t st,
                               int precision) {
    TD_CHECK(e != nullptr, TDSCHA_EINVAL, "NULL ensemble");
    if (!e->Rrow) return vjp_in_ensemble_basis(e, nb, R1, Ys, apply_d4, fbar, Dbar, Ybar, rhobar, st, precision);
    TD_CHECK(nb > 0, TDSCHA_EINVAL, "nb must be positive");
    TD_CHECK(R1 && Ys && fbar && Dbar && Ybar && rhobar, TDSCHA_EINVAL, "NULL argument");
    const int n = e->n;
    const size_t vec = ((size_t)nb * n * 8 + 255) / 256 * 256, mat = ((size_t)nb * n * n * 8 + 255) / 256 * 256;
    const size_t yb = ((size_t)e->N * n * 8 + 255) / 256 * 256;
    const size_t need = 2 * vec + 3 * mat + yb;
    if (e->rot_ws.bytes < need) {
        if (e->rot_ws.base) { TD_CUDA(cudaDeviceSynchronize()); cudaFree(e->rot_ws.base); e->rot_ws = Workspace(); }
        TD_CUDA(cudaMalloc(&e->rot_ws.base, need));
        e->rot_ws.bytes = need;
    }
    uint8_t *W = static_cast<uint8_t *>(e->rot_ws.base);
    double *R1r = reinterpret_cast<double *>(W), *fr = reinterpret_cast<double *>(W + vec);
    double *Ysr = reinterpret_cast<double *>(W + 2 * vec), *Dr = reinterpret_cast<double *>(W + 2 * vec + mat);
    double *tmp = reinterpret_cast<double *>(W + 2 * vec + 2 * mat), *Yr = reinterpret_cast<double *>(W + 2 * vec + 3 * mat);
    const int dmax = e->dmax;
    TD_TRY(rotate_rows_of(nb, n, dmax, e->Rrow, e->d_blocks_ids, e->d_blk_start, e->d_blk_dim, R1, R1r, true, st));
    TD_TRY(rotate_rows_of(nb, n, dmax, e->Rrow, e->d_blocks_ids, e->d_blk_start, e->d_blk_dim, fbar, fr, true, st));
    TD_TRY(rotate_mats(nb, n, dmax, e->Rrow, e->d_blocks_ids, e->d_blk_start, e->d_blk_dim, Ys, tmp, Ysr, true, st));
    TD_TRY(rotate_mats(nb, n, dmax, e->Rrow, e->d_blocks_ids, e->d_blk_start, e->d_blk_dim, Dbar, tmp, Dr, true, st));
    TD_TRY(vjp_in_ensemble_basis(e, nb, R1r, Ysr, apply_d4, fr, Dr, Yr, rhobar, st, precision));
    return rotate_rows_of(e->N, n, dmax, e->Rrow, e->d_blocks_ids, e->d_blk_start, e->d_blk_dim, Yr, Ybar, false, st);
}

}  // namespace tdscha
