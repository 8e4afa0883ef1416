// apply.cu -- apply_full_L on the device (FP64 outside the two ensemble contractions), the
// bi-conjugate Lanczos step and the continued-fraction Green function.
//
// Follows Modules/DynamicalLanczos.py:
//   apply_L1_FT                :2227-2385   (harmonic 2x2 blocks per packed pair, w^2 on R)
//   get_Y1 / get_ReA1          :2827-2888   (unpacking, halved off-diagonals for the transpose)
//   get_alpha1_beta1_wigner    :2713-2822,  get_chi_minus/plus :2572-2627
//   apply_anharmonic_FT        :2891-3281   (prologue mixing, epilogue packing and signs)
//   apply_full_L               :3467-3570   (sum, reverse_L, shift)
//   run_FT step                :6026-6153   (n_rep_orth = 0)
//   get_green_function_continued_fraction :4951-5047
#include <cmath>
#include <cuComplex.h>
#include <cuda.h>
#include <mutex>

#include "apply.cuh"
#include "common.cuh"
#include "ensemble.cuh"

namespace tdscha {

constexpr double PY_EPSILON = 1e-12;   // DynamicalLanczos.py:121

__device__ __forceinline__ double bose_div(double w, double T) {   // 1/(exp(w / (T/RyToK)) - 1), as in L1
    return T > 0 ? 1.0 / (exp(w / (T / RY_TO_K)) - 1.0) : 0.0;
}
__device__ __forceinline__ double bose_mul(double w, double T) {   // 1/(exp(w*RyToK/T) - 1), as in the anharmonic part
    return T > PY_EPSILON ? 1.0 / (exp(w * RY_TO_K / T) - 1.0) : 0.0;
}

// row of packed pair p (row-major upper triangle): largest mu with mu*n - mu(mu-1)/2 <= p
__device__ __forceinline__ void unpair(long long p, int n, int &mu, int &nu) {
    // solve p = mu*n - mu(mu-1)/2 + (nu - mu) ; start from the float estimate and fix up
    double nn = 2.0 * n + 1.0;
    int m = (int)floor((nn - sqrt(nn * nn - 8.0 * (double)p)) / 2.0);
    if (m < 0) m = 0;
    if (m > n - 1) m = n - 1;
    while (m > 0 && (long long)m * n - ((long long)m * (m - 1)) / 2 > p) --m;
    while (m + 1 < n && (long long)(m + 1) * n - ((long long)(m + 1) * m) / 2 <= p) ++m;
    mu = m;
    nu = (int)(p - ((long long)m * n - ((long long)m * (m - 1)) / 2)) + m;
}

// ---- prologue: (R1, Upsilon^(1)) of each vector ----------------------------------------------
__global__ void prologue_kernel(int nb, int n, long long len, const double *__restrict__ psi, const int *__restrict__ transpose,
                                const double *__restrict__ w, double T, int use_wigner, double *R, double *Ys) {
    const long long P = (long long)n * (n + 1) / 2;
    const long long total = (long long)nb * P;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(idx / P);
        const long long p = idx % P;
        int mu, nu;
        unpair(p, n, mu, nu);
        const double *ps = psi + (long long)k * len;
        double y;
        if (!use_wigner) {
            const double pY = ps[n + p];
            if (!transpose[k]) {
                y = pY;
            } else {
                const double pA = ps[n + P + p];
                const double half = (mu == nu) ? 1.0 : 0.5;
                const double na = bose_mul(w[mu], T), nbb = bose_mul(w[nu], T);
                const double Ya = 2 * w[mu] / (2 * na + 1), Yb = 2 * w[nu] / (2 * nbb + 1);
                const double RAa = 2 * w[mu] * na * (na + 1) / (2 * na + 1), RAb = 2 * w[nu] * nbb * (nbb + 1) / (2 * nbb + 1);
                const double cY = 2 * (Ya * Yb * Yb + Ya * Ya * Yb);
                const double cR = 2 * (Ya * RAb * Yb + Ya * RAa * Yb);
                y = half * pY * cY + half * pA * cR;
            }
        } else {
            // alpha^(1) from a'^(1), b'^(1): w_a = w[col], w_b = w[row]
            const double wa = w[nu], wb = w[mu];
            const double na = bose_div(wa, T), nbb = bose_div(wb, T);
            const double Xf = (1 + 2 * na) * (1 + 2 * nbb) / 8;
            const double w2X = (wa * wb) / Xf;
            const double chim = ((wa - wb) * (na - nbb)) / (2 * wa * wb);
            const double chip = ((wa + wb) * (1 + na + nbb)) / (2 * wa * wb);
            y = w2X * sqrt(-0.5 * chim) * ps[n + p] - w2X * sqrt(0.5 * chip) * ps[n + P + p];
        }
        double *Yk = Ys + (long long)k * n * n;
        Yk[(long long)mu * n + nu] = y;
        Yk[(long long)nu * n + mu] = y;
        if (p < n) R[(long long)k * n + p] = ps[p];
    }
}

// ---- epilogue: L1 + anharmonic packing, reverse, shift -----------------------------------------
__global__ void epilogue_kernel(int nb, int n, long long len, const double *__restrict__ psi, const int *__restrict__ transpose,
                                const double *__restrict__ w, double T, tdscha_apply_opts o, const double *__restrict__ fav,
                                const double *__restrict__ dav, double *__restrict__ out) {
    const long long P = (long long)n * (n + 1) / 2;
    const long long total = (long long)nb * len;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(idx / len);
        const long long i = idx % len;
        const double *ps = psi + (long long)k * len;
        const int tr = transpose[k];
        double v = 0.0;
        if (i < n) {
            if (!o.ignore_harmonic) v = o.use_wigner ? -(ps[i] * w[i]) * w[i] : (ps[i] * w[i]) * w[i];
            if (!o.ignore_v3) v += o.use_wigner ? fav[(long long)k * n + i] : -fav[(long long)k * n + i];
        } else {
            const bool inY = i < n + P;
            const long long p = inY ? i - n : i - n - P;
            int mu, nu;
            unpair(p, n, mu, nu);
            const double wa = w[nu], wb = w[mu];   // w_a = column mode, w_b = row mode
            const double pY = ps[n + p], pA = ps[n + P + p];
            if (!o.ignore_harmonic) {
                if (!o.use_wigner) {
                    const double na = bose_div(wa, T), nbb = bose_div(wb, T);
                    const double den = (2 * na + 1) * (2 * nbb + 1);
                    const double Xab = -wa * wa - wb * wb - (2 * wa * wb) / den;
                    const double Yab = -(8 * wa * wb) / den;
                    const double X1ab = -(2 * na * nbb + na + nbb) * (2 * na * nbb + na + nbb + 1) * (2 * wa * wb) / den;
                    const double Y1ab = -wa * wa - wb * wb + (2 * wa * wb) / den;
                    if (inY) v = -Xab * pY + (tr ? -X1ab * pA : -Yab * pA);
                    else v = (tr ? -Yab * pY : -X1ab * pY) - Y1ab * pA;
                } else {
                    v = inY ? -(wa * wa + wb * wb - 2. * wa * wb) * pY : -(wa * wa + wb * wb + 2. * wa * wb) * pA;
                }
            }
            if (!o.ignore_v3) {
                const double d = dav[(long long)k * n * n + (long long)mu * n + nu];
                if (!o.use_wigner) {
                    const double na = bose_mul(w[mu], T), nbb = bose_mul(w[nu], T);
                    const double Ya = 2 * w[mu] / (2 * na + 1), Yb = 2 * w[nu] / (2 * nbb + 1);
                    if (!tr) {
                        if (inY) v += -(d * Ya + d * Yb);
                        else {
                            const double RAa = 2 * w[mu] * na * (na + 1) / (2 * na + 1);
                            const double RAb = 2 * w[nu] * nbb * (nbb + 1) / (2 * nbb + 1);
                            v += -(d * RAa + d * RAb);
                        }
                    } else if (inY) {
                        v += -(0.5 * (1.0 / Ya) * d * (1.0 / Yb)) * (mu == nu ? 1.0 : 2.0);
                    }
                } else {
                    const double na = bose_mul(w[mu], T), nbb = bose_mul(w[nu], T);
                    if (inY) {
                        const double chim = (w[mu] - w[nu]) * (na - nbb) / (2. * w[mu] * w[nu]);
                        v += sqrt(-0.5 * chim) * d;
                    } else {
                        const double chip = (w[mu] + w[nu]) * (1 + na + nbb) / (2. * w[mu] * w[nu]);
                        v += -sqrt(0.5 * chip) * d;
                    }
                }
            }
        }
        if (o.reverse_L) v *= -1;
        v += o.shift_value * ps[i];
        out[idx] = v;
    }
}

static int grid_for(long long total, int threads = 256) {
    long long g = (total + threads - 1) / threads;
    return (int)std::min<long long>(std::max<long long>(g, 1), 148LL * 32);
}

int apply_full_L_device(tdscha_ensemble *e, int nb, const double *psi, const int *transpose_h, const tdscha_apply_opts *opts,
                        int precision, double *out, cudaStream_t st, void *scratch, size_t scratch_bytes) {
    TD_CHECK(e && psi && out && transpose_h && scratch, TDSCHA_EINVAL, "NULL argument");
    TD_CHECK(nb > 0 && nb <= 64, TDSCHA_EINVAL, "1..64 vectors per apply call (got %d)", nb);
    TD_CHECK(scratch_bytes > 256, TDSCHA_EINVAL, "apply scratch too small");
    // scratch: transpose flags (nb ints, 256 bytes), then the work of apply_full_L_device_flags
    uint8_t *s = static_cast<uint8_t *>(scratch);
    int *tr_d = reinterpret_cast<int *>(s);
    TD_CUDA(cudaMemcpyAsync(tr_d, transpose_h, nb * sizeof(int), cudaMemcpyHostToDevice, st));
    return apply_full_L_device_flags(e, nb, psi, tr_d, opts, precision, out, st, reinterpret_cast<double *>(s + 256),
                                     scratch_bytes - 256);
}

// apply_full_L with the transpose flags already on the device (no host transfer: graph-capturable);
// work: R (nb n), Ys (nb n^2), f (nb n), D (nb n^2) doubles.
int apply_full_L_device_flags(tdscha_ensemble *e, int nb, const double *psi, const int *tr_d, const tdscha_apply_opts *opts,
                              int precision, double *out, cudaStream_t st, double *work, size_t work_bytes) {
    TD_CHECK(e && psi && out && tr_d && work, TDSCHA_EINVAL, "NULL argument");
    TD_CHECK(nb > 0 && nb <= 64, TDSCHA_EINVAL, "1..64 vectors per apply call (got %d)", nb);
    tdscha_apply_opts o{0, 0, 0, 0, 0, 0.0};
    if (opts) o = *opts;
    const int n = e->n;
    const long long P = (long long)n * (n + 1) / 2;
    const long long len = n + 2 * P;
    TD_CHECK(work_bytes >= (size_t)nb * (2 * n + 2 * (size_t)n * n) * sizeof(double), TDSCHA_EINVAL, "apply work too small");
    double *R = work;
    double *Ys = R + (size_t)nb * n;
    double *fav = Ys + (size_t)nb * n * n;
    double *dav = fav + (size_t)nb * n;
    e->prof.launches[ST_OTHER] += o.ignore_v3 ? 1 : 2;
    if (!o.ignore_v3) {
        prologue_kernel<<<grid_for((long long)nb * P), 256, 0, st>>>(nb, n, len, psi, tr_d, e->w, e->T, o.use_wigner, R, Ys);
        TD_CUDA(cudaGetLastError());
        TD_TRY(perturb_average_device(e, nb, R, Ys, o.ignore_v4 ? 0 : 1, precision, fav, dav, st));
    }
    epilogue_kernel<<<grid_for((long long)nb * len), 256, 0, st>>>(nb, n, len, psi, tr_d, e->w, e->T, o, fav, dav, out);
    TD_CUDA(cudaGetLastError());
    return 0;
}

// The two halves of apply_full_L around the averages, for callers that reduce the averages of
// configuration slices across devices themselves.  tr_d: device copy of the transpose flags.
int apply_prologue_device(tdscha_ensemble *e, int nb, const double *psi, const int *tr_d, const tdscha_apply_opts *opts,
                          double *R, double *Ys, cudaStream_t st) {
    TD_CHECK(e && psi && tr_d && R && Ys && nb > 0, TDSCHA_EINVAL, "bad prologue arguments");
    tdscha_apply_opts o{0, 0, 0, 0, 0, 0.0};
    if (opts) o = *opts;
    const int n = e->n;
    const long long P = (long long)n * (n + 1) / 2;
    e->prof.launches[ST_OTHER] += 1;
    prologue_kernel<<<grid_for((long long)nb * P), 256, 0, st>>>(nb, n, n + 2 * P, psi, tr_d, e->w, e->T, o.use_wigner, R, Ys);
    TD_CUDA(cudaGetLastError());
    return 0;
}

int apply_epilogue_device(tdscha_ensemble *e, int nb, const double *psi, const int *tr_d, const tdscha_apply_opts *opts,
                          const double *fav, const double *dav, double *out, cudaStream_t st) {
    TD_CHECK(e && psi && tr_d && out && nb > 0, TDSCHA_EINVAL, "bad epilogue arguments");
    tdscha_apply_opts o{0, 0, 0, 0, 0, 0.0};
    if (opts) o = *opts;
    TD_CHECK(o.ignore_v3 || (fav && dav), TDSCHA_EINVAL, "averages required unless ignore_v3");
    const int n = e->n;
    const long long len = n + (long long)n * (n + 1);
    e->prof.launches[ST_OTHER] += 1;
    epilogue_kernel<<<grid_for((long long)nb * len), 256, 0, st>>>(nb, n, len, psi, tr_d, e->w, e->T, o, fav, dav, out);
    TD_CUDA(cudaGetLastError());
    return 0;
}

size_t apply_scratch_bytes(const tdscha_ensemble *e, int nb) {
    const size_t n = e->n;
    return 256 + (size_t)nb * (2 * n + 2 * n * n) * sizeof(double);
}

// ---- bi-conjugate Lanczos step ----------------------------------------------------------------
constexpr int LZ_THREADS = 256;
constexpr int LZ_BLOCKS = 148 * 2;

__device__ double block_sum(double v, double *sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r += sh[i];
    return r;   // valid on thread 0
}

// partial[c][blk] = sum_{i in blk's strided range} p[i] * Lq[i] * mask[i]
__global__ void lz_dot_kernel(long long len, const double *p, const double *Lq, const double *mask, double *partial) {
    __shared__ double sh[32];
    const int c = blockIdx.y;
    const double *pc = p + (long long)c * len, *lc = Lq + (long long)c * len;
    double acc = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
        acc += pc[i] * lc[i] * (mask ? mask[i] : 1.0);
    double s = block_sum(acc, sh);
    if (threadIdx.x == 0) partial[c * gridDim.x + blockIdx.x] = s;
}

struct StepScalars {
    double a, p_norm, hist_q, hist_p;
};
__device__ StepScalars step_scalars(const double *sc_in, const double *partial_a, int nblk, int c) {
    const double *s = sc_in + 6 * c;
    const int k = (int)s[5];
    const double c_old = k >= 1 ? s[0] : 1.0;
    const double p_norm = s[2] / c_old;
    double dot = 0.0;
    for (int b = 0; b < nblk; ++b) dot += partial_a[c * nblk + b];
    StepScalars r;
    r.a = dot * p_norm;
    r.p_norm = p_norm;
    r.hist_q = k >= 1 ? s[0] : 0.0;                       // c_{k-1}
    const double old_p_norm = (k >= 2) ? s[3] / s[4] : s[3];
    r.hist_p = k >= 1 ? s[1] * (old_p_norm / p_norm) : 0.0;
    return r;
}

// r = Lq - a q - c_{k-1} q_prev ; s = pL - a p - b_{k-1} p_prev old/p ; partials of r.r, s.s, s.r
__global__ void lz_residual_kernel(long long len, const double *Lq, const double *pL, const double *q, const double *p,
                                   const double *q_prev, const double *p_prev, const double *sc_in, const double *partial_a,
                                   int nblk, const double *mask, double *rbuf, double *sbuf, double *partial3) {
    __shared__ double sh[32];
    const int c = blockIdx.y;
    const StepScalars S = step_scalars(sc_in, partial_a, nblk, c);
    const long long o = (long long)c * len;
    double rr = 0, ss = 0, sr = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x) {
        double r = Lq[o + i] - S.a * q[o + i];
        double s = pL[o + i] - S.a * p[o + i];
        if (S.hist_q != 0.0 || S.hist_p != 0.0) {
            r -= S.hist_q * q_prev[o + i];
            s -= S.hist_p * p_prev[o + i];
        }
        rbuf[o + i] = r;
        sbuf[o + i] = s;
        const double m = mask ? mask[i] : 1.0;
        rr += r * r * m;
        ss += s * s * m;
        sr += s * r * m;
    }
    double t;
    t = block_sum(rr, sh);
    if (threadIdx.x == 0) partial3[(c * 3 + 0) * gridDim.x + blockIdx.x] = t;
    t = block_sum(ss, sh);
    if (threadIdx.x == 0) partial3[(c * 3 + 1) * gridDim.x + blockIdx.x] = t;
    t = block_sum(sr, sh);
    if (threadIdx.x == 0) partial3[(c * 3 + 2) * gridDim.x + blockIdx.x] = t;
}

__global__ void lz_finish_kernel(long long len, const double *sc_in, const double *partial_a, const double *partial3, int nblk,
                                 double *q_next, double *p_next, double *sc_out) {
    const int c = blockIdx.y;
    const StepScalars S = step_scalars(sc_in, partial_a, nblk, c);
    double rr = 0, ss = 0, sr = 0;
    for (int b = 0; b < nblk; ++b) {
        rr += partial3[(c * 3 + 0) * nblk + b];
        ss += partial3[(c * 3 + 1) * nblk + b];
        sr += partial3[(c * 3 + 2) * nblk + b];
    }
    const double snorm = sqrt(ss);
    const double bcoef = sqrt(rr);
    // c = (s/|s|) . (r/b) * |s| p_norm ; evaluated as in run_FT
    double sdot = 0.0;
    sdot = sr / snorm / bcoef;
    const double s_norm_new = snorm * S.p_norm;
    const double ccoef = sdot * s_norm_new;
    const long long o = (long long)c * len;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x) {
        q_next[o + i] = q_next[o + i] / bcoef;
        p_next[o + i] = p_next[o + i] / snorm;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sc_out[4 * c + 0] = S.a;
        sc_out[4 * c + 1] = bcoef;
        sc_out[4 * c + 2] = ccoef;
        sc_out[4 * c + 3] = s_norm_new;
    }
}

int lanczos_step_device(int nc, long long len, const double *Lq, const double *pL, const double *q, const double *p,
                        const double *q_prev, const double *p_prev, const double *sc_in, const double *mask, double *q_next,
                        double *p_next, double *sc_out, cudaStream_t st, double *scratch, size_t scratch_bytes) {
    TD_CHECK(nc > 0 && len > 0, TDSCHA_EINVAL, "empty Lanczos step");
    TD_CHECK(Lq && pL && q && p && sc_in && q_next && p_next && sc_out, TDSCHA_EINVAL, "NULL argument");
    const int nblk = LZ_BLOCKS;
    const size_t need = (size_t)nc * nblk * 4 * sizeof(double);
    TD_CHECK(scratch_bytes >= need, TDSCHA_EINVAL, "Lanczos scratch too small");
    double *pa = scratch, *p3 = scratch + (size_t)nc * nblk;
    const double *qp = q_prev ? q_prev : q, *pp = p_prev ? p_prev : p;
    dim3 g(nblk, nc);
    lz_dot_kernel<<<g, LZ_THREADS, 0, st>>>(len, p, Lq, mask, pa);
    lz_residual_kernel<<<g, LZ_THREADS, 0, st>>>(len, Lq, pL, q, p, qp, pp, sc_in, pa, nblk, mask, q_next, p_next, p3);
    lz_finish_kernel<<<g, LZ_THREADS, 0, st>>>(len, sc_in, pa, p3, nblk, q_next, p_next, sc_out);
    TD_CUDA(cudaGetLastError());
    return 0;
}

size_t lanczos_scratch_bytes(int nc) { return (size_t)nc * LZ_BLOCKS * 4 * sizeof(double); }

// ---- Lanczos step without any allocation ---------------------------------------------------------
// The step's only temporaries are its per-block reduction partials (4 doubles per chain and block).
// For callers that cannot allocate device memory, they live in this fixed file-scope array, which
// every GPU that loads the library holds until the process exits.
constexpr int LZ_NOALLOC_MAX_CHAINS = 32;
static __device__ __align__(256) double g_lz_noalloc_scratch[(size_t)LZ_NOALLOC_MAX_CHAINS * LZ_BLOCKS * 4];

// Device address of the array, looked up once per device (with that device current) and again only
// when the device's context changed since (after a device reset the module is loaded anew and the
// array may sit elsewhere).  The context handle comes from the driver entry point cuCtxGetCurrent.
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
static std::mutex g_noalloc_mutex;
static void *g_noalloc_addr[128] = {nullptr};
static CUcontext g_noalloc_ctx[128] = {nullptr};

static int current_context(CUcontext *ctx) {
    static CtxGetCurrentFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        TD_CHECK(cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
                     q == cudaDriverEntryPointSuccess && p != nullptr,
                 TDSCHA_ECUDA, "cuCtxGetCurrent entry point unavailable");
        fn = reinterpret_cast<CtxGetCurrentFn>(p);
    }
    TD_CHECK(fn(ctx) == CUDA_SUCCESS, TDSCHA_ECUDA, "cuCtxGetCurrent failed");
    return 0;
}

static int noalloc_scratch_address(double **out) {
    int dev = 0;
    TD_CUDA(cudaGetDevice(&dev));
    TD_CHECK(dev >= 0 && dev < 128, TDSCHA_EINVAL, "device index %d out of range", dev);
    TD_CUDA(cudaSetDevice(dev));            // makes the device's primary context current (CUDA >= 12)
    CUcontext ctx = nullptr;
    TD_TRY(current_context(&ctx));
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev] || g_noalloc_ctx[dev] != ctx) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_lz_noalloc_scratch);
        TD_CHECK(e == cudaSuccess && p != nullptr, TDSCHA_ECUDA, "cudaGetSymbolAddress of the Lanczos scratch failed: %s",
                 cudaGetErrorString(e));
        g_noalloc_addr[dev] = p;
        g_noalloc_ctx[dev] = ctx;
    }
    *out = static_cast<double *>(g_noalloc_addr[dev]);
    return 0;
}

}  // namespace tdscha

extern "C" int tdscha_lanczos_step_device_noalloc(int nc, long long len, const double *Lq, const double *pL,
                                                  const double *q, const double *p, const double *q_prev,
                                                  const double *p_prev, const double *sc_in, const double *mask,
                                                  double *q_next, double *p_next, double *sc_out, void *stream) {
    using namespace tdscha;
    clear_error();
    TD_CHECK(nc > 0 && nc <= LZ_NOALLOC_MAX_CHAINS, TDSCHA_EINVAL,
             "tdscha_lanczos_step_device_noalloc: %d chains requested, its fixed scratch holds at most %d", nc,
             LZ_NOALLOC_MAX_CHAINS);
    double *scratch = nullptr;
    TD_TRY(noalloc_scratch_address(&scratch));
    // every partial the kernels read is written earlier in the same call: nothing needs clearing
    return lanczos_step_device(nc, len, Lq, pL, q, p, q_prev, p_prev, sc_in, mask, q_next, p_next, sc_out,
                               static_cast<cudaStream_t>(stream), scratch,
                               (size_t)LZ_NOALLOC_MAX_CHAINS * LZ_BLOCKS * 4 * sizeof(double));
}

namespace tdscha {

// ---- continued fraction -------------------------------------------------------------------------
struct CFParams {
    int n_iter, n_b, n_c, use_terminator, last_average, use_wigner;
    double sign, shift, smearing, modulus;
};

__global__ void cf_kernel(CFParams prm, const double *a, const double *b, const double *c, int n_w, const double *omega, double *gf) {
    const int iw = blockIdx.x * blockDim.x + threadIdx.x;
    if (iw >= n_w) return;
    const double w = omega[iw];
    const double wsgn = prm.use_wigner ? 1.0 : -1.0;     // a -/+ w^2
    const bool nonsym = (c != nullptr) && (prm.n_c == prm.n_b);
    cuDoubleComplex g;
    if (prm.use_terminator) {
        double a_av = 0, b_av = 0, c_av = 0;
        const int la = min(prm.last_average, prm.n_iter), lb = min(prm.last_average, prm.n_b);
        for (int i = prm.n_iter - la; i < prm.n_iter; ++i) a_av += a[i];
        a_av /= la;
        for (int i = prm.n_b - lb; i < prm.n_b; ++i) b_av += b[i];
        b_av /= lb;
        c_av = b_av;
        if (nonsym) {
            c_av = 0;
            for (int i = prm.n_c - lb; i < prm.n_c; ++i) c_av += c[i];
            c_av /= lb;
        }
        const double A = a_av * prm.sign - prm.sign * prm.shift, B = b_av * prm.sign, C = c_av * prm.sign;
        const double x = A + wsgn * w * w;
        // (x -/+ sqrt(x^2 - 4bc + 0j)) / (2bc): standard uses '-' , Wigner '+'
        const double disc = x * x - 4 * B * C;
        cuDoubleComplex sq = disc >= 0 ? make_cuDoubleComplex(sqrt(disc), 0.0) : make_cuDoubleComplex(0.0, sqrt(-disc));
        cuDoubleComplex num = prm.use_wigner ? cuCadd(make_cuDoubleComplex(x, 0), sq) : cuCsub(make_cuDoubleComplex(x, 0), sq);
        g = make_cuDoubleComplex(cuCreal(num) / (2 * B * C), cuCimag(num) / (2 * B * C));
    } else {
        const double A = a[prm.n_iter - 1] * prm.sign - prm.sign * prm.shift;
        g = cuCdiv(make_cuDoubleComplex(1.0, 0.0), make_cuDoubleComplex(A + wsgn * w * w, 2 * w * prm.smearing));
    }
    for (int i = prm.n_iter - 2; i >= 0; --i) {
        const double A = a[i] * prm.sign - prm.sign * prm.shift;
        const double B = b[i] * prm.sign;
        const double C = nonsym ? c[i] * prm.sign : B;
        cuDoubleComplex den = make_cuDoubleComplex(A + wsgn * w * w, 2 * w * prm.smearing);
        den = cuCsub(den, cuCmul(make_cuDoubleComplex(B * C, 0.0), g));
        g = cuCdiv(make_cuDoubleComplex(1.0, 0.0), den);
    }
    double re = cuCreal(g), im = cuCimag(g);
    if (prm.use_wigner) re = -re;
    gf[2 * iw] = re * prm.modulus;
    gf[2 * iw + 1] = im * prm.modulus;
}

int continued_fraction_device(int n_iter, const double *a, const double *b, const double *c, int n_b, int n_c, int n_w,
                              const double *omega, int use_terminator, int last_average, double smearing, int use_wigner,
                              int reverse_L, double shift_value, double modulus, double *gf_out, cudaStream_t st) {
    TD_CHECK(n_iter > 0 && n_w > 0 && a && omega && gf_out, TDSCHA_EINVAL, "bad continued-fraction arguments");
    TD_CHECK(n_iter == 1 || (b && n_b >= n_iter - 1), TDSCHA_EINVAL, "need at least n_iter - 1 b coefficients");
    TD_CHECK(!use_terminator || (b && n_b >= 1 && last_average >= 1), TDSCHA_EINVAL, "terminator needs b coefficients");
    CFParams prm{n_iter, n_b, c ? n_c : 0, use_terminator, last_average, use_wigner, reverse_L ? -1.0 : 1.0, shift_value, smearing, modulus};
    cf_kernel<<<ceil_div(n_w, 128), 128, 0, st>>>(prm, a, b, c, n_w, omega, gf_out);
    TD_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace tdscha
