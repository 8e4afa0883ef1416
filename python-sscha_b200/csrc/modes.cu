// modes.cu -- the inputs of the Lanczos built on the GPU from an ensemble and its symmetry group:
//
//   X = (u o sqrt(m)) . pols,  Y = (f / sqrt(m)) . pols        (Modules/DynamicalLanczos.py:376-442)
//   S_b^j = E_b^T P_j E_b  per degenerate block b              (what DynamicalLanczos.py:749 obtains
//                                                               from cellconstructor's
//                                                               GetSymmetriesOnModesDeg)
// with E = pols (3 nat x n, mass-weighted polarisation vectors) and P_j the Cartesian action of
// symmetry j on mass-weighted displacements: (P_j v)[perm_j(a)] = R_j v[a] (perm_j the image atom).
// Both are FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "modes.cuh"

namespace tdscha {
namespace {

constexpr int PT = 32;   // projection tile (outputs) and K chunk

// out[i][m] = sum_k in[i][k] * s_k * pols[k][m]   with s_k = sqrt(m_k) or 1 / sqrt(m_k)
__global__ void __launch_bounds__(PT * 8)
project_kernel(const double *__restrict__ in, const double *__restrict__ masses, int divide, const double *__restrict__ pols,
               int N, int K, int n, double *__restrict__ out) {
    __shared__ double A[PT][PT + 1], B[PT][PT + 1];
    const int tx = threadIdx.x % PT, ty = threadIdx.x / PT;   // 32 x 8 threads, 4 rows each
    const int i0 = blockIdx.y * PT, m0 = blockIdx.x * PT;
    double acc[4] = {0, 0, 0, 0};
    for (int k0 = 0; k0 < K; k0 += PT) {
        for (int r = ty; r < PT; r += 8) {
            const int i = i0 + r, k = k0 + tx;
            double v = 0;
            if (i < N && k < K) {
                const double s = sqrt(masses[k]);
                v = divide ? in[(long long)i * K + k] / s : in[(long long)i * K + k] * s;
            }
            A[r][tx] = v;
            const int kk = k0 + r, m = m0 + tx;
            B[r][tx] = (kk < K && m < n) ? pols[(long long)kk * n + m] : 0.0;
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < PT; ++kk) {
            const double b = B[kk][tx];
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[q] = fma(A[ty + 8 * q][kk], b, acc[q]);
        }
        __syncthreads();
    }
    for (int q = 0; q < 4; ++q) {
        const int i = i0 + ty + 8 * q, m = m0 + tx;
        if (i < N && m < n) out[(long long)i * n + m] = acc[q];
    }
}

constexpr int ST = 256;       // threads of the symmetry kernel
constexpr int SCH = 8;        // atoms per chunk
constexpr int SDMAX = 80;     // largest block
constexpr int SOUT = (SDMAX * SDMAX + ST - 1) / ST;

// one CTA per (symmetry j, block b): S[j][p][q] = sum_a sum_al E[3 perm_j(a) + al][c_p] (R_j E[3a..3a+2][c_q])_al
__global__ void __launch_bounds__(ST)
sym_modes_kernel(const double *__restrict__ pols, int nat, int n, const int *__restrict__ perm, const double *__restrict__ rot,
                 const int *__restrict__ cols, const int *__restrict__ col_off, const int *__restrict__ dims,
                 const long long *__restrict__ out_off, int N_sym, double *__restrict__ out) {
    __shared__ double Lh[3 * SCH][SDMAX], Rh[3 * SCH][SDMAX];
    __shared__ double R[9];
    const int j = blockIdx.x, b = blockIdx.y;
    const int d = dims[b];
    const int *c = cols + col_off[b];
    if (threadIdx.x < 9) R[threadIdx.x] = rot[(long long)j * 9 + threadIdx.x];
    const int *pj = perm + (long long)j * nat;
    double acc[SOUT];
#pragma unroll
    for (int o = 0; o < SOUT; ++o) acc[o] = 0;
    __syncthreads();
    for (int a0 = 0; a0 < nat; a0 += SCH) {
        const int na = min(SCH, nat - a0);
        for (int e = threadIdx.x; e < 3 * SCH * d; e += ST) {
            const int r = e / d, q = e % d, a = a0 + r / 3, al = r % 3;
            double lv = 0, rv = 0;
            if (r / 3 < na) {
                const int col = c[q];
                lv = pols[(long long)(3 * pj[a] + al) * n + col];
                rv = R[3 * al] * pols[(long long)(3 * a) * n + col] + R[3 * al + 1] * pols[(long long)(3 * a + 1) * n + col] +
                     R[3 * al + 2] * pols[(long long)(3 * a + 2) * n + col];
            }
            Lh[r][q] = lv;
            Rh[r][q] = rv;
        }
        __syncthreads();
#pragma unroll
        for (int o = 0; o < SOUT; ++o) {
            const int idx = threadIdx.x + o * ST;
            if (idx < d * d) {
                const int p = idx / d, q = idx % d;
                double s = acc[o];
                for (int r = 0; r < 3 * na; ++r) s = fma(Lh[r][p], Rh[r][q], s);
                acc[o] = s;
            }
        }
        __syncthreads();
    }
    double *S = out + out_off[b] + (long long)j * d * d;
#pragma unroll
    for (int o = 0; o < SOUT; ++o) {
        const int idx = threadIdx.x + o * ST;
        if (idx < d * d) S[idx] = acc[o];
    }
}

struct DeviceAlloc {
    std::vector<void *> ptrs;
    ~DeviceAlloc() {
        for (void *p : ptrs) cudaFree(p);
    }
    template <typename T>
    int get(T **p, size_t count) {
        void *v = nullptr;
        TD_CUDA(cudaMalloc(&v, std::max<size_t>(count, 1) * sizeof(T)));
        ptrs.push_back(v);
        *p = static_cast<T *>(v);
        return 0;
    }
};

}  // namespace

int project_ensemble(const double *u, const double *f, const double *masses, const double *pols, int N, int nat3, int n,
                     double *X_out, double *Y_out) {
    TD_CHECK(N > 0 && nat3 > 0 && n > 0 && n <= nat3, TDSCHA_EINVAL, "bad sizes N=%d 3nat=%d n=%d", N, nat3, n);
    TD_CHECK(u && f && masses && pols && X_out && Y_out, TDSCHA_EINVAL, "NULL argument");
    for (int k = 0; k < nat3; ++k) TD_CHECK(masses[k] > 0, TDSCHA_EINVAL, "non-positive mass at %d", k);
    DeviceAlloc al;
    double *du, *df, *dm, *dp, *dX, *dY;
    const size_t nu = (size_t)N * nat3, nx = (size_t)N * n;
    TD_TRY(al.get(&du, nu));
    TD_TRY(al.get(&df, nu));
    TD_TRY(al.get(&dm, nat3));
    TD_TRY(al.get(&dp, (size_t)nat3 * n));
    TD_TRY(al.get(&dX, nx));
    TD_TRY(al.get(&dY, nx));
    TD_CUDA(cudaMemcpy(du, u, nu * sizeof(double), cudaMemcpyHostToDevice));
    TD_CUDA(cudaMemcpy(df, f, nu * sizeof(double), cudaMemcpyHostToDevice));
    TD_CUDA(cudaMemcpy(dm, masses, nat3 * sizeof(double), cudaMemcpyHostToDevice));
    TD_CUDA(cudaMemcpy(dp, pols, (size_t)nat3 * n * sizeof(double), cudaMemcpyHostToDevice));
    dim3 grid((unsigned)ceil_div(n, PT), (unsigned)ceil_div(N, PT));
    project_kernel<<<grid, PT * 8>>>(du, dm, 0, dp, N, nat3, n, dX);
    project_kernel<<<grid, PT * 8>>>(df, dm, 1, dp, N, nat3, n, dY);
    TD_CUDA(cudaGetLastError());
    TD_CUDA(cudaMemcpy(X_out, dX, nx * sizeof(double), cudaMemcpyDeviceToHost));
    TD_CUDA(cudaMemcpy(Y_out, dY, nx * sizeof(double), cudaMemcpyDeviceToHost));
    return 0;
}

int symmetries_on_modes(const double *pols, int nat, int n, int N_sym, const int *perm, const double *rot, int n_blocks,
                        const int *n_deg, const int *const *deg_space, double *const *sym_out) {
    TD_CHECK(nat > 0 && n > 0 && n <= 3 * nat && N_sym > 0 && n_blocks > 0, TDSCHA_EINVAL,
             "bad sizes nat=%d n=%d N_sym=%d n_blocks=%d", nat, n, N_sym, n_blocks);
    TD_CHECK(pols && perm && rot && n_deg && deg_space && sym_out, TDSCHA_EINVAL, "NULL argument");
    std::vector<int> cols, col_off(n_blocks), dims(n_blocks);
    std::vector<long long> out_off(n_blocks);
    long long total = 0;
    for (int b = 0; b < n_blocks; ++b) {
        const int d = n_deg[b];
        TD_CHECK(d >= 1 && d <= SDMAX, TDSCHA_EINVAL, "block %d has %d modes (1..%d supported)", b, d, SDMAX);
        TD_CHECK(deg_space[b] && sym_out[b], TDSCHA_EINVAL, "NULL block %d", b);
        col_off[b] = (int)cols.size();
        dims[b] = d;
        out_off[b] = total;
        total += (long long)N_sym * d * d;
        for (int q = 0; q < d; ++q) {
            TD_CHECK(deg_space[b][q] >= 0 && deg_space[b][q] < n, TDSCHA_EINVAL, "mode index %d out of range", deg_space[b][q]);
            cols.push_back(deg_space[b][q]);
        }
    }
    for (long long k = 0; k < (long long)N_sym * nat; ++k)
        TD_CHECK(perm[k] >= 0 && perm[k] < nat, TDSCHA_EINVAL, "atom permutation entry %lld out of range", k);
    DeviceAlloc al;
    double *dp, *drot, *dout;
    int *dperm, *dcols, *dcoff, *ddims;
    long long *doff;
    TD_TRY(al.get(&dp, (size_t)3 * nat * n));
    TD_TRY(al.get(&drot, (size_t)N_sym * 9));
    TD_TRY(al.get(&dperm, (size_t)N_sym * nat));
    TD_TRY(al.get(&dcols, cols.size()));
    TD_TRY(al.get(&dcoff, n_blocks));
    TD_TRY(al.get(&ddims, n_blocks));
    TD_TRY(al.get(&doff, n_blocks));
    TD_TRY(al.get(&dout, (size_t)total));
    TD_CUDA(cudaMemcpy(dp, pols, (size_t)3 * nat * n * sizeof(double), cudaMemcpyHostToDevice));
    TD_CUDA(cudaMemcpy(drot, rot, (size_t)N_sym * 9 * sizeof(double), cudaMemcpyHostToDevice));
    TD_CUDA(cudaMemcpy(dperm, perm, (size_t)N_sym * nat * sizeof(int), cudaMemcpyHostToDevice));
    TD_CUDA(cudaMemcpy(dcols, cols.data(), cols.size() * sizeof(int), cudaMemcpyHostToDevice));
    TD_CUDA(cudaMemcpy(dcoff, col_off.data(), n_blocks * sizeof(int), cudaMemcpyHostToDevice));
    TD_CUDA(cudaMemcpy(ddims, dims.data(), n_blocks * sizeof(int), cudaMemcpyHostToDevice));
    TD_CUDA(cudaMemcpy(doff, out_off.data(), n_blocks * sizeof(long long), cudaMemcpyHostToDevice));
    sym_modes_kernel<<<dim3((unsigned)N_sym, (unsigned)n_blocks), ST>>>(dp, nat, n, dperm, drot, dcols, dcoff, ddims, doff, N_sym,
                                                                        dout);
    TD_CUDA(cudaGetLastError());
    for (int b = 0; b < n_blocks; ++b)
        TD_CUDA(cudaMemcpy(sym_out[b], dout + out_off[b], (size_t)N_sym * dims[b] * dims[b] * sizeof(double),
                           cudaMemcpyDeviceToHost));
    return 0;
}

}  // namespace tdscha
