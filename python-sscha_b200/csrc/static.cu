// static.cu -- the static (zero-frequency) L operator of the free-energy Hessian, on the device:
//
//   apply_L1_static        Modules/DynamicalLanczos.py:2502-2565
//   apply_anharmonic_static                       :3287-3354
//
// on batches of static vectors psi = (R (n), Upsilon packed upper row-major (P = n(n+1)/2)):
//   L1:   out_R = R w^(2 power),  out_Y = Y / Lambda^power
//         Lambda_ab = [(n_a + n_b + 1)/(w_a + w_b) - (n_a - n_b)/(w_a - w_b)] / (4 w_a w_b)
//   anh:  R1 = R, Upsilon1 = -2 Yw Y Yw (Y the symmetric unpacking, Yw = 2w/(2n+1)),
//         (f, D) = the symmetrised averages, out = (-f, D packed upper)
// The averages are the same device pipeline as the dynamical apply (perturb_average_device).
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "apply.cuh"
#include "common.cuh"
#include "ensemble.cuh"

namespace tdscha {
namespace {

constexpr double PY_EPS = 1e-12;   // DynamicalLanczos.py:121

__device__ __forceinline__ long long pair_of(int mu, int nu, int n) {   // mu <= nu, row-major upper
    return (long long)mu * n - ((long long)mu * (mu - 1)) / 2 + (nu - mu);
}

__device__ __forceinline__ void unpair_s(long long p, int n, int &mu, int &nu) {
    double nn = 2.0 * n + 1.0;
    int m = (int)floor((nn - sqrt(nn * nn - 8.0 * (double)p)) / 2.0);
    if (m < 0) m = 0;
    if (m > n - 1) m = n - 1;
    while (m > 0 && (long long)m * n - ((long long)m * (m - 1)) / 2 > p) --m;
    while (m + 1 < n && (long long)(m + 1) * n - ((long long)(m + 1) * m) / 2 <= p) ++m;
    mu = m;
    nu = (int)(p - ((long long)m * n - ((long long)m * (m - 1)) / 2)) + m;
}

__device__ __forceinline__ double l1_R(double w, double power) {
    if (power == 1.0) return w * w;
    if (power == -1.0) return 1.0 / (w * w);
    return pow(w, 2.0 * power);
}

__device__ __forceinline__ double l1_Y(double y, double lam, double power) {
    if (power == 1.0) return y / lam;
    if (power == -1.0) return y * lam;
    return y / pow(lam, power);
}

// out = [with_l1] L1_static(psi)^power  (+ the anharmonic part when f / D are given)
__global__ void static_out_kernel(int nb, int n, const double *__restrict__ psi, const double *__restrict__ w,
                                  const double *__restrict__ lam, int with_l1, double power, const double *__restrict__ f,
                                  const double *__restrict__ D, double *__restrict__ out) {
    const long long P = (long long)n * (n + 1) / 2, len = n + P;
    const long long total = (long long)nb * len;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long k = idx / len, e = idx % len;
        double v;
        if (e < n) {
            v = with_l1 ? psi[idx] * l1_R(w[e], power) : 0.0;
            if (f) v -= f[k * n + e];
        } else {
            const long long p = e - n;
            v = with_l1 ? l1_Y(psi[idx], lam[p], power) : 0.0;
            if (D) {
                int mu, nu;
                unpair_s(p, n, mu, nu);
                v += D[(k * n + mu) * n + nu];
            }
        }
        out[idx] = v;
    }
}

// R1 = psi_R; Upsilon1[mu][nu] = -2 Yw_mu Yw_nu Y[mu][nu] (Y the symmetric unpacking of psi_Y)
__global__ void static_prologue_kernel(int nb, int n, const double *__restrict__ psi, const double *__restrict__ w, double T,
                                       double *__restrict__ R1, double *__restrict__ Y1) {
    const long long P = (long long)n * (n + 1) / 2, len = n + P, nn = (long long)n * n;
    const long long total = (long long)nb * nn;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long k = idx / nn, e = idx % nn;
        const int mu = (int)(e / n), nu = (int)(e % n);
        const double *ps = psi + k * len;
        const double nm = T > PY_EPS ? 1.0 / (exp(w[mu] * RY_TO_K / T) - 1.0) : 0.0;
        const double nv = T > PY_EPS ? 1.0 / (exp(w[nu] * RY_TO_K / T) - 1.0) : 0.0;
        const double ym = 2 * w[mu] / (2 * nm + 1), yv = 2 * w[nu] / (2 * nv + 1);
        const double y = ps[n + (mu <= nu ? pair_of(mu, nu, n) : pair_of(nu, mu, n))];
        Y1[idx] = -2.0 * y * ym * yv;
        if (nu == 0) R1[k * n + mu] = ps[mu];
    }
}

int grid_of(long long total) {
    long long g = (total + 255) / 256;
    return (int)std::min<long long>(std::max<long long>(g, 1), 148LL * 32);
}

}  // namespace

// Lambda of the packed pairs, computed on the host in FP64 exactly as the reference does it,
// including its two quirks: both Bose factors are zeroed by the mask of w_a (:2535-2536), and
// the equal-frequency branch multiplies by the square of an all-zero array (:2539-2540, the
// array is taken before the factors are filled), so it contributes -beta e^(w beta) * 0.
int ensure_static_lambda(tdscha_ensemble *e) {
    if (e->d_static_lam) return 0;
    const int n = e->n;
    const long long P = (long long)n * (n + 1) / 2;
    std::vector<double> w(n), lam(P);
    TD_CUDA(cudaMemcpy(w.data(), e->w, n * sizeof(double), cudaMemcpyDeviceToHost));
    const double T = e->T;
    long long p = 0;
    for (int b = 0; b < n; ++b) {
        for (int a = b; a < n; ++a, ++p) {
            const double wa = w[a], wb = w[b];
            double na = 0, nb = 0, diff = 0;
            const bool equal = std::fabs(wa - wb) < 1e-8;
            if (T > 0) {
                const double beta = RY_TO_K / T;
                const bool masked = 0.01 * wa * RY_TO_K > T;
                na = masked ? 0.0 : 1.0 / (std::exp(wa * beta) - 1.0);
                nb = masked ? 0.0 : 1.0 / (std::exp(wb * beta) - 1.0);
                diff = equal ? -beta * std::exp(wa * beta) * (0.0 * 0.0) : (na - nb) / (wa - wb);
            }
            double L = (na + nb + 1) / (wa + wb) - diff;
            lam[p] = L / (4 * wa * wb);
        }
    }
    TD_CUDA(cudaMalloc(&e->d_static_lam, P * sizeof(double)));
    TD_CUDA(cudaMemcpy(e->d_static_lam, lam.data(), P * sizeof(double), cudaMemcpyHostToDevice));
    return 0;
}

size_t static_work_bytes(const tdscha_ensemble *e, int nb) {
    const size_t n = e->n;
    return (size_t)nb * (2 * n + 2 * n * n) * sizeof(double);
}

int apply_L1_static_device(tdscha_ensemble *e, int nb, const double *psi, double power, double *out, cudaStream_t st) {
    TD_CHECK(e && psi && out && nb > 0, TDSCHA_EINVAL, "bad L1_static arguments");
    TD_TRY(ensure_static_lambda(e));
    const long long len = e->n + (long long)e->n * (e->n + 1) / 2;
    static_out_kernel<<<grid_of((long long)nb * len), 256, 0, st>>>(nb, e->n, psi, e->w, e->d_static_lam, 1, power,
                                                                   nullptr, nullptr, out);
    TD_CUDA(cudaGetLastError());
    return 0;
}

int apply_static_L_device(tdscha_ensemble *e, int nb, const double *psi, int ignore_v4, int include_L1, int precision,
                          double *out, cudaStream_t st, double *work, size_t work_bytes) {
    TD_CHECK(e && psi && out && work, TDSCHA_EINVAL, "NULL argument");
    TD_CHECK(nb > 0 && nb <= 64, TDSCHA_EINVAL, "1..64 vectors per static apply (got %d)", nb);
    TD_CHECK(work_bytes >= static_work_bytes(e, nb), TDSCHA_EINVAL, "static apply work too small");
    TD_TRY(ensure_static_lambda(e));
    const int n = e->n;
    const long long len = n + (long long)n * (n + 1) / 2;
    double *R1 = work, *Y1 = R1 + (size_t)nb * n, *f = Y1 + (size_t)nb * n * n, *D = f + (size_t)nb * n;
    static_prologue_kernel<<<grid_of((long long)nb * n * n), 256, 0, st>>>(nb, n, psi, e->w, e->T, R1, Y1);
    TD_CUDA(cudaGetLastError());
    TD_TRY(perturb_average_device(e, nb, R1, Y1, ignore_v4 ? 0 : 1, precision, f, D, st));
    static_out_kernel<<<grid_of((long long)nb * len), 256, 0, st>>>(nb, n, psi, e->w, e->d_static_lam,
                                                                   include_L1 ? 1 : 0, 1.0, f, D, out);
    TD_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace tdscha
