// symmetry.cu -- block-pair kernels for the symmetry transform and fold (see symmetry.cuh).
#include <algorithm>
#include <type_traits>
#include <vector>

#include "symmetry.cuh"

namespace tdscha {

__device__ __forceinline__ long long sym_pair_index(int mu, int nu, int n) {   // mu <= nu, row-major upper triangle
    return (long long)mu * n - ((long long)mu * (mu - 1)) / 2 + (nu - mu);
}

// acc (+)= A (m x k) . B (k x n), shared-memory operands addressed with (row, col) strides; thread
// (ty, tx) of the 16 x 16 grid owns rows ty + 16 i and columns tx + 16 j (i, j < MT).
template <typename T, int MT>
__device__ __forceinline__ void mm_tile(T (&acc)[MT][MT], const T *A, int a_rs, int a_cs, const T *B, int b_rs, int b_cs,
                                        int m, int n, int k, int ty, int tx) {
#pragma unroll 2
    for (int kk = 0; kk < k; ++kk) {
        T a[MT], b[MT];
#pragma unroll
        for (int i = 0; i < MT; ++i) {
            const int r = ty + 16 * i;
            a[i] = r < m ? A[r * a_rs + kk * a_cs] : T(0);
        }
#pragma unroll
        for (int j = 0; j < MT; ++j) {
            const int c = tx + 16 * j;
            b[j] = c < n ? B[kk * b_rs + c * b_cs] : T(0);
        }
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < MT; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
}

template <typename T, int MT>
__device__ __forceinline__ void zero_tile(T (&acc)[MT][MT]) {
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < MT; ++j) acc[i][j] = T(0);
}

// ---- transform -------------------------------------------------------------------------------------
// grid (pairs of the class, j-chunks of JT symmetries, nb); Ys[b, c] is staged once per CTA.
template <typename T, int MT>
__global__ void __launch_bounds__(SYM_THREADS)
transform_kernel(SymTables t, const int *__restrict__ pb, const int *__restrict__ pc, int nj, int j0, int JT,
                 const double *__restrict__ Ys, const double *__restrict__ R1, const double *__restrict__ ups, long long Kp,
                 long long np, Format fmt, void *B1_hi, void *B1_lo, void *r1_hi, void *r1_lo) {
    constexpr int DM = 16 * MT;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    T *Yt = reinterpret_cast<T *>(sm_raw);     // d_b x d_c   Ys[b, c]
    T *Sb = Yt + DM * DM;                       // d_b x d_b   S_j block b (row-major S[p][mu])
    T *Sc = Sb + DM * DM;                       // d_c x d_c
    T *M1 = Sc + DM * DM;                       // d_b x d_c   Ys[b, c] S_c
    const int b = pb[blockIdx.x], c = pc[blockIdx.x];
    const int k = blockIdx.z;
    const int ja = j0 + blockIdx.y * JT, jb = min(ja + JT, j0 + nj);
    const int n = t.n;
    const int sb = t.start[b], db = t.dim[b], sc = t.start[c], dc = t.dim[c];
    const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
    const double *Yk = Ys + (long long)k * n * n;
    for (int e = threadIdx.x; e < db * dc; e += blockDim.x) Yt[e] = (T)Yk[(long long)(sb + e / dc) * n + sc + e % dc];
    for (int j = ja; j < jb; ++j) {
        const long long r = (long long)k * nj + (j - j0);
        const double *Sbg = t.sym + t.off[b] + (long long)j * db * db;
        const double *Scg = t.sym + t.off[c] + (long long)j * dc * dc;
        __syncthreads();
        for (int e = threadIdx.x; e < db * db; e += blockDim.x) Sb[e] = (T)Sbg[e];
        for (int e = threadIdx.x; e < dc * dc; e += blockDim.x) Sc[e] = (T)Scg[e];
        __syncthreads();
        T acc[MT][MT];
        zero_tile(acc);
        mm_tile(acc, Yt, dc, 1, Sc, dc, 1, db, dc, dc, ty, tx);          // M1 = Ys[b,c] S_c
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int jj = 0; jj < MT; ++jj) {
                const int rr = ty + 16 * i, cc = tx + 16 * jj;
                if (rr < db && cc < dc) M1[rr * dc + cc] = acc[i][jj];
            }
        if (b == c && threadIdx.x < db) {   // r1 for the modes of block b: ups o (S_b^T R)
            const double *Rk = R1 + (long long)k * n + sb;
            double s = 0.0;
            for (int p = 0; p < db; ++p) s += (double)Sb[p * db + threadIdx.x] * Rk[p];
            store_split(fmt, r1_hi, r1_lo, r * np + sb + threadIdx.x, ups[sb + threadIdx.x] * s);
        }
        __syncthreads();
        zero_tile(acc);
        mm_tile(acc, Sb, 1, db, M1, dc, 1, db, dc, db, ty, tx);          // S_b^T M1
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int jj = 0; jj < MT; ++jj) {
                const int mu = ty + 16 * i, nu = tx + 16 * jj;
                const int gm = sb + mu, gn = sc + nu;
                if (mu < db && nu < dc && gm <= gn)
                    store_split(fmt, B1_hi, B1_lo, r * Kp + sym_pair_index(gm, gn, n), (double)acc[i][jj]);
            }
    }
}

// zero the padding columns B1[:, P:Kp) and r1[:, n:np)
__global__ void pad_kernel(long long M, long long P, long long Kp, int n, long long np, Format fmt, void *B1_hi, void *B1_lo,
                           void *r1_hi, void *r1_lo) {
    const long long w1 = Kp - P, w2 = np - n;
    const long long total = M * (w1 + w2);
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long r = idx / (w1 + w2), q = idx % (w1 + w2);
        if (q < w1) store_split(fmt, B1_hi, B1_lo, r * Kp + P + q, 0.0);
        else store_split(fmt, r1_hi, r1_lo, r * np + n + (q - w1), 0.0);
    }
}

// ---- fold ------------------------------------------------------------------------------------------
// grid (pairs of the class, fold chunks of Jf symmetries, nb).  The two block products of one
// symmetry run in the compute type T over <= d terms; their result is summed over symmetries in FP64.
template <typename T, typename AccT, int MT>
__global__ void __launch_bounds__(SYM_THREADS, 2)
fold_kernel(SymTables t, const int *__restrict__ pb, const int *__restrict__ pc, const AccT *__restrict__ Z, long long ldz,
            const AccT *__restrict__ F, long long ldf, const double *__restrict__ ups, int nj, int j0, int Jf, int nf_total,
            double *__restrict__ partD, double *__restrict__ partF) {
    constexpr int DM = 16 * MT;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    T *Sb = reinterpret_cast<T *>(sm_raw);   // d_b x d_b  S_j block b, row-major S[mu][p]
    T *ScT = Sb + DM * DM;                   // d_c x d_c  transposed: ScT[q][nu] = S_c[nu][q]
    T *Wt = ScT + DM * DM;                   // d_b x d_c  W_j[b, c]
    T *U = Wt + DM * DM;                     // d_b x d_c  W_j[b, c] S_c^T
    const int b = pb[blockIdx.x], c = pc[blockIdx.x];
    const int fc = blockIdx.y, k = blockIdx.z;
    const int n = t.n;
    const int sb = t.start[b], db = t.dim[b], sc = t.start[c], dc = t.dim[c];
    const int fg = j0 / Jf + fc;
    const int ja = j0 + fc * Jf, jb = min(j0 + (fc + 1) * Jf, j0 + nj);
    const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
    double acc[MT][MT];
    zero_tile(acc);
    double facc = 0.0;   // f partial for mode sb + threadIdx.x (diagonal pairs only)
    for (int j = ja; j < jb; ++j) {
        const long long r = (long long)k * nj + (j - j0);
        const double *Sbg = t.sym + t.off[b] + (long long)j * db * db;
        const double *Scg = t.sym + t.off[c] + (long long)j * dc * dc;
        __syncthreads();
        for (int e = threadIdx.x; e < db * db; e += blockDim.x) Sb[e] = (T)Sbg[e];
        for (int e = threadIdx.x; e < dc * dc; e += blockDim.x) ScT[(e % dc) * dc + e / dc] = (T)Scg[e];
        for (int e = threadIdx.x; e < db * dc; e += blockDim.x) {
            const int p = e / dc, q = e % dc;
            int gm = sb + p, gn = sc + q;
            if (gm > gn) { const int s = gm; gm = gn; gn = s; }
            const double z = (double)Z[r * ldz + sym_pair_index(gm, gn, n)];
            Wt[e] = (T)((gm == gn ? 2.0 : 1.0) * ups[gm] * ups[gn] * z);
        }
        __syncthreads();
        T u[MT][MT];
        zero_tile(u);
        mm_tile(u, Wt, dc, 1, ScT, dc, 1, db, dc, dc, ty, tx);        // U = W S_c^T (<= d_c terms)
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int jj = 0; jj < MT; ++jj) {
                const int rr = ty + 16 * i, cc = tx + 16 * jj;
                if (rr < db && cc < dc) U[rr * dc + cc] = u[i][jj];
            }
        if (b == c && threadIdx.x < db) {
            const AccT *Fr = F + r * ldf + sb;
            double s = 0.0;
            for (int p = 0; p < db; ++p) s += (double)Sb[threadIdx.x * db + p] * (double)Fr[p];
            facc += s;
        }
        __syncthreads();
        zero_tile(u);
        mm_tile(u, Sb, db, 1, U, dc, 1, db, dc, db, ty, tx);          // S_b U (<= d_b terms) ...
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int jj = 0; jj < MT; ++jj) acc[i][jj] += (double)u[i][jj];   // ... then summed over j in FP64
    }
    double *out = partD + ((long long)k * nf_total + fg) * (long long)n * n;
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int jj = 0; jj < MT; ++jj) {
            const int mu = ty + 16 * i, nu = tx + 16 * jj;
            if (mu < db && nu < dc) out[(long long)(sb + mu) * n + sc + nu] = acc[i][jj];
        }
    if (b == c && threadIdx.x < db) partF[((long long)k * nf_total + fg) * n + sb + threadIdx.x] = facc;
}

// ---- host ------------------------------------------------------------------------------------------
int build_pair_classes(const std::vector<int> &dim, PairClasses &pc, size_t *bytes) {
    std::vector<int> lb[SYM_MT_MAX + 1], lc[SYM_MT_MAX + 1];
    const int nbk = (int)dim.size();
    for (int b = 0; b < nbk; ++b)
        for (int c = b; c < nbk; ++c) {
            const int mt = std::max(1, (std::max(dim[b], dim[c]) + 15) / 16);
            TD_CHECK(mt <= SYM_MT_MAX, TDSCHA_EINVAL, "degenerate block of %d modes exceeds the supported %d",
                     std::max(dim[b], dim[c]), DMAX_SUPPORTED);
            lb[mt].push_back(b);
            lc[mt].push_back(c);
        }
    for (int mt = 1; mt <= SYM_MT_MAX; ++mt) {
        pc.count[mt] = (int)lb[mt].size();
        if (!pc.count[mt]) continue;
        TD_CUDA(cudaMalloc(&pc.b[mt], lb[mt].size() * sizeof(int)));
        TD_CUDA(cudaMalloc(&pc.c[mt], lc[mt].size() * sizeof(int)));
        TD_CUDA(cudaMemcpy(pc.b[mt], lb[mt].data(), lb[mt].size() * sizeof(int), cudaMemcpyHostToDevice));
        TD_CUDA(cudaMemcpy(pc.c[mt], lc[mt].data(), lc[mt].size() * sizeof(int), cudaMemcpyHostToDevice));
        if (bytes) *bytes += 2 * lb[mt].size() * sizeof(int);
    }
    return 0;
}

void free_pair_classes(PairClasses &pc) {
    for (int mt = 0; mt <= SYM_MT_MAX; ++mt) {
        if (pc.b[mt]) cudaFree(pc.b[mt]);
        if (pc.c[mt]) cudaFree(pc.c[mt]);
        pc.b[mt] = pc.c[mt] = nullptr;
        pc.count[mt] = 0;
    }
}

template <typename T, int MT>
static int launch_transform(const SymTables &t, const PairClasses &pc, int nb, int nj, int j0, const double *Ys, const double *R1,
                            const double *ups, long long Kp, long long np, Format fmt, void *B1_hi, void *B1_lo, void *r1_hi,
                            void *r1_lo, cudaStream_t st) {
    if (!pc.count[MT]) return 0;
    constexpr int JT = 8;
    const size_t smem = 4 * (size_t)(16 * MT) * (16 * MT) * sizeof(T);
    auto kern = transform_kernel<T, MT>;
    TD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)pc.count[MT], (unsigned)ceil_div(nj, JT), (unsigned)nb);
    kern<<<grid, SYM_THREADS, smem, st>>>(t, pc.b[MT], pc.c[MT], nj, j0, JT, Ys, R1, ups, Kp, np, fmt, B1_hi, B1_lo, r1_hi, r1_lo);
    TD_CUDA(cudaGetLastError());
    return 0;
}

template <typename T>
static int transform_all(const SymTables &t, const PairClasses &pc, int nb, int nj, int j0, const double *Ys, const double *R1,
                         const double *ups, long long Kp, long long np, Format fmt, void *B1_hi, void *B1_lo, void *r1_hi,
                         void *r1_lo, cudaStream_t st) {
    TD_TRY((launch_transform<T, 1>(t, pc, nb, nj, j0, Ys, R1, ups, Kp, np, fmt, B1_hi, B1_lo, r1_hi, r1_lo, st)));
    TD_TRY((launch_transform<T, 2>(t, pc, nb, nj, j0, Ys, R1, ups, Kp, np, fmt, B1_hi, B1_lo, r1_hi, r1_lo, st)));
    TD_TRY((launch_transform<T, 3>(t, pc, nb, nj, j0, Ys, R1, ups, Kp, np, fmt, B1_hi, B1_lo, r1_hi, r1_lo, st)));
    TD_TRY((launch_transform<T, 4>(t, pc, nb, nj, j0, Ys, R1, ups, Kp, np, fmt, B1_hi, B1_lo, r1_hi, r1_lo, st)));
    TD_TRY((launch_transform<T, 5>(t, pc, nb, nj, j0, Ys, R1, ups, Kp, np, fmt, B1_hi, B1_lo, r1_hi, r1_lo, st)));
    return 0;
}

int sym_transform(const SymTables &t, const PairClasses &pc, int nb, int nj, int j0, const double *Ys, const double *R1,
                  const double *ups, long long P, long long Kp, long long np, Format fmt, void *B1_hi, void *B1_lo,
                  void *r1_hi, void *r1_lo, bool fp32_compute, cudaStream_t st) {
    const long long M = (long long)nb * nj;
    const long long pad = M * ((Kp - P) + (np - t.n));
    if (pad > 0) {
        const int g = (int)std::min<long long>((pad + 255) / 256, 148LL * 16);
        pad_kernel<<<g, 256, 0, st>>>(M, P, Kp, t.n, np, fmt, B1_hi, B1_lo, r1_hi, r1_lo);
        TD_CUDA(cudaGetLastError());
    }
    if (fp32_compute && fmt == FMT_BF16 && t.umma)
        return sym_transform_umma(t.umma, t, t.blocks_ids, nb, nj, j0, Ys, R1, ups, Kp, np, fmt, B1_hi, B1_lo, r1_hi, r1_lo,
                                  t.err, st);
    if (fp32_compute) return sym_transform_tc(t, pc, nb, nj, j0, Ys, R1, ups, Kp, np, fmt, B1_hi, B1_lo, r1_hi, r1_lo, st);
    return transform_all<double>(t, pc, nb, nj, j0, Ys, R1, ups, Kp, np, fmt, B1_hi, B1_lo, r1_hi, r1_lo, st);
}

template <typename T, typename AccT, int MT>
static int launch_fold(const SymTables &t, const PairClasses &pc, int nb, int nj, int j0, int Jf, int nf_total, const AccT *Z,
                       long long ldz, const AccT *F, long long ldf, const double *ups, double *partD, double *partF, cudaStream_t st) {
    if (!pc.count[MT]) return 0;
    const size_t smem = 4 * (size_t)(16 * MT) * (16 * MT) * sizeof(T);
    auto kern = fold_kernel<T, AccT, MT>;
    TD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)pc.count[MT], (unsigned)ceil_div(nj, Jf), (unsigned)nb);
    kern<<<grid, SYM_THREADS, smem, st>>>(t, pc.b[MT], pc.c[MT], Z, ldz, F, ldf, ups, nj, j0, Jf, nf_total, partD, partF);
    TD_CUDA(cudaGetLastError());
    return 0;
}

template <typename T, typename AccT>
static int fold_all(const SymTables &t, const PairClasses &pc, int nb, int nj, int j0, int Jf, int nf_total, const AccT *Z,
                    long long ldz, const AccT *F, long long ldf, const double *ups, double *partD, double *partF, cudaStream_t st) {
    TD_TRY((launch_fold<T, AccT, 1>(t, pc, nb, nj, j0, Jf, nf_total, Z, ldz, F, ldf, ups, partD, partF, st)));
    TD_TRY((launch_fold<T, AccT, 2>(t, pc, nb, nj, j0, Jf, nf_total, Z, ldz, F, ldf, ups, partD, partF, st)));
    TD_TRY((launch_fold<T, AccT, 3>(t, pc, nb, nj, j0, Jf, nf_total, Z, ldz, F, ldf, ups, partD, partF, st)));
    TD_TRY((launch_fold<T, AccT, 4>(t, pc, nb, nj, j0, Jf, nf_total, Z, ldz, F, ldf, ups, partD, partF, st)));
    TD_TRY((launch_fold<T, AccT, 5>(t, pc, nb, nj, j0, Jf, nf_total, Z, ldz, F, ldf, ups, partD, partF, st)));
    return 0;
}

template <typename AccT>
int sym_fold(const SymTables &t, const PairClasses &pc, const int *blocks_ids, int nb, int nj, int j0, int Jf, int nf_total,
             const AccT *Z, long long ldz, const AccT *F, long long ldf, const double *ups, double *partD, double *partF,
             bool fp32_compute, cudaStream_t st) {
    (void)blocks_ids;
    if constexpr (std::is_same<AccT, float>::value) {
        if (fp32_compute && t.umma)
            return sym_fold_umma(t.umma, t, t.blocks_ids, nb, nj, j0, Jf, nf_total, Z, ldz, F, ldf, ups, partD, partF, t.err, st);
        if (fp32_compute) return sym_fold_tc(t, pc, nb, nj, j0, Jf, nf_total, Z, ldz, F, ldf, ups, partD, partF, st);
    }
    if (fp32_compute) return fold_all<float, AccT>(t, pc, nb, nj, j0, Jf, nf_total, Z, ldz, F, ldf, ups, partD, partF, st);
    return fold_all<double, AccT>(t, pc, nb, nj, j0, Jf, nf_total, Z, ldz, F, ldf, ups, partD, partF, st);
}

template int sym_fold<float>(const SymTables &, const PairClasses &, const int *, int, int, int, int, int, const float *, long long,
                             const float *, long long, const double *, double *, double *, bool, cudaStream_t);
template int sym_fold<double>(const SymTables &, const PairClasses &, const int *, int, int, int, int, int, const double *,
                              long long, const double *, long long, const double *, double *, double *, bool, cudaStream_t);

}  // namespace tdscha
