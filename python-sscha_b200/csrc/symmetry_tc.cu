// symmetry_tc.cu -- the symmetry transform and fold of the mixed-precision modes on the tensor pipe.
//
// Same block-pair decomposition as symmetry.cu (S_j block diagonal over degenerate blocks), but the
// two d_b x d_c products per (vector k, symmetry j, block pair b <= c) run as warp-level
// mma.sync.m16n8k8 tf32 tiles with three-term splitting (hi.hi + hi.lo + lo.hi of tf32 halves,
// ~21 significant bits, fp32 accumulation per symmetry) instead of FP32 register micro-tiles on the
// CUDA cores.
//
//   * One warp task = one 16 x 8 output tile, so even a (72-mode, 3-mode) block pair keeps most of
//     the 16 warps busy.
//   * Operands reused across symmetries or tiles (the Ys block, the intermediate product) are kept
//     in shared memory already split, as (hi, lo) float2 pairs; the symmetry blocks are fp32 and
//     split while the fragments are loaded.
//   * Symmetry j + 1's blocks are copied (cp.async) into the second half of a double buffer while
//     symmetry j is computed.
//   * Block dimensions are zero-padded to 16 on the row side of an A operand and 8 elsewhere.
//     Leading dimensions make every fragment load free of bank conflicts: fp32 arrays read as
//     (row g, column t) use ld = 4 (mod 8), fp32 arrays read as (row t, column g) use ld = 8
//     (mod 16), float2 arrays use ld = 4 (mod 8) (in float2 units).
#include <algorithm>
#include <cstdint>
#include <cuda_bf16.h>

#include "symmetry.cuh"

namespace tdscha {
namespace {

constexpr int THREADS = 512;
constexpr int NW = THREADS / 32;

__host__ __device__ constexpr int ld_gt(int d) { return d + ((4 - d % 8) + 8) % 8; }     // ld = 4 (mod 8)
__host__ __device__ constexpr int ld_tg(int d) { return d + ((8 - d % 16) + 16) % 16; }  // ld = 8 (mod 16)

__device__ __forceinline__ long long pair_index(int mu, int nu, int n) {   // mu <= nu, row-major upper triangle
    return (long long)mu * n - ((long long)mu * (mu - 1)) / 2 + (nu - mu);
}

__device__ __forceinline__ uint32_t to_tf32(float v) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
    return r;
}
__device__ __forceinline__ void split_tf32(float v, uint32_t &hi, uint32_t &lo) {
    hi = to_tf32(v);
    lo = to_tf32(v - __uint_as_float(hi));
}
__device__ __forceinline__ float2 split2(float v) {
    uint32_t h, l;
    split_tf32(v, h, l);
    return make_float2(__uint_as_float(h), __uint_as_float(l));
}
__device__ __forceinline__ void mma_tf32(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// 4-byte asynchronous global -> shared copies; `valid` false writes a zero instead (src-size 0).
__device__ __forceinline__ void cp_async4(float *dst, const float *src, bool valid) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(valid ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(PENDING) : "memory"); }

// Operand views of one warp tile.  Element (r, c) of the logical operand:
//   F32   : p[r * ld + c]          fp32, split on load
//   F32T  : p[c * ld + r]          fp32 stored transposed, split on load
//   F2    : q[r * ld + c]          float2 (hi, lo), already split
enum OpKind { F32, F32T, F2 };
template <int KIND>
__device__ __forceinline__ void load_op(const void *p, int ld, int r, int c, uint32_t &hi, uint32_t &lo) {
    if constexpr (KIND == F2) {
        const float2 v = static_cast<const float2 *>(p)[r * ld + c];
        hi = __float_as_uint(v.x);
        lo = __float_as_uint(v.y);
    } else if constexpr (KIND == F32) {
        split_tf32(static_cast<const float *>(p)[r * ld + c], hi, lo);
    } else {
        split_tf32(static_cast<const float *>(p)[c * ld + r], hi, lo);
    }
}

// c += A[m0:m0+16, 0:8 kt] . B[0:8 kt, n0:n0+8], three-term tf32 split.  Fragment layouts of
// m16n8k8 (g = lane / 4, t = lane % 4): a0 (g, t), a1 (g + 8, t), a2 (g, t + 4), a3 (g + 8, t + 4);
// b0 (t, g), b1 (t + 4, g); c0/c1 (g, 2t / 2t + 1), c2/c3 (g + 8, 2t / 2t + 1).
template <int AK, int BK>
__device__ __forceinline__ void warp_tile(float (&c)[4], const void *A, int lda, const void *B, int ldb, int m0, int n0, int kt) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll 2
    for (int ks = 0; ks < kt; ++ks) {
        const int k0 = ks * 8;
        uint32_t ah[4], al[4], bh0, bl0, bh1, bl1;
        load_op<AK>(A, lda, m0 + g, k0 + t, ah[0], al[0]);
        load_op<AK>(A, lda, m0 + g + 8, k0 + t, ah[1], al[1]);
        load_op<AK>(A, lda, m0 + g, k0 + t + 4, ah[2], al[2]);
        load_op<AK>(A, lda, m0 + g + 8, k0 + t + 4, ah[3], al[3]);
        load_op<BK>(B, ldb, k0 + t, n0 + g, bh0, bl0);
        load_op<BK>(B, ldb, k0 + t + 4, n0 + g, bh1, bl1);
        mma_tf32(c, al, bh0, bh1);   // small terms first
        mma_tf32(c, ah, bl0, bl1);
        mma_tf32(c, ah, bh0, bh1);
    }
}

// store a warp tile's accumulators as split (hi, lo) pairs into a float2 array
__device__ __forceinline__ void store_tile_f2(float2 *X, int ld, int m0, int n0, const float (&c)[4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const float2 a0 = split2(c[0]), a1 = split2(c[1]), a2 = split2(c[2]), a3 = split2(c[3]);
    *reinterpret_cast<float4 *>(&X[(m0 + g) * ld + n0 + 2 * t]) = make_float4(a0.x, a0.y, a1.x, a1.y);
    *reinterpret_cast<float4 *>(&X[(m0 + g + 8) * ld + n0 + 2 * t]) = make_float4(a2.x, a2.y, a3.x, a3.y);
}

// bf16 / tf32 hi + lo of an fp32 value into the GEMM operand arrays
__device__ __forceinline__ void store_split_f(Format fmt, void *hi, void *lo, long long idx, float x) {
    if (fmt == FMT_BF16) {
        const __nv_bfloat16 h = __float2bfloat16_rn(x);
        static_cast<__nv_bfloat16 *>(hi)[idx] = h;
        if (lo) static_cast<__nv_bfloat16 *>(lo)[idx] = __float2bfloat16_rn(x - __bfloat162float(h));
    } else {
        const float h = __uint_as_float(to_tf32(x));
        static_cast<float *>(hi)[idx] = h;
        if (lo) static_cast<float *>(lo)[idx] = __uint_as_float(to_tf32(x - h));
    }
}

template <int MT>
struct TcShape {
    static constexpr int DM = 16 * MT;   // padded block size of the class
    static constexpr int L2 = ld_gt(DM);  // float2 arrays
    static constexpr int LG = ld_gt(DM);  // fp32 arrays read (row g, column t)
    static constexpr int LT = ld_tg(DM);  // fp32 arrays read (row t, column g)
    // transform: Yk2 + M12 (float2) + 2 x (S_b, S_c) fp32
    static constexpr size_t TRANSFORM_SMEM = (size_t)DM * (2 * L2 * 8 + 4 * LT * 4);
    // fold: 2 x (S_b, S_c, W) fp32 + U2 float2
    static constexpr size_t FOLD_SMEM = (size_t)DM * (6 * LG * 4 + L2 * 8);
    // fold step-2 tiles per warp (16 x 8 tiles of the largest block pair of the class)
    static constexpr int TILES_PER_WARP = ((DM / 16) * (DM / 8) + NW - 1) / NW;
};

// ---- transform ---------------------------------------------------------------------------------------
// grid (pairs of the class, j-chunks of JT symmetries, nb).  Per symmetry:
//   step 1  M1 (d_b x d_c) = Ys_k[b, c] . S_c        (A = Yk2, B = S_c)
//   step 2  T  (d_b x d_c) = S_b^T . M1               (A = S_b read transposed, B = M12)
// T is staged in shared memory and written row by row to B1 (packed pairs, format fmt) for
// global modes mu <= nu.
template <int MT>
__global__ void __launch_bounds__(THREADS)
transform_tc_kernel(SymTables tb, const int *__restrict__ pb, const int *__restrict__ pc, int nj, int j0, int JT,
                    const double *__restrict__ Ys, const double *__restrict__ R1, const double *__restrict__ ups, long long Kp,
                    long long np, Format fmt, void *B1_hi, void *B1_lo, void *r1_hi, void *r1_lo) {
    using S = TcShape<MT>;
    constexpr int DM = S::DM, L2 = S::L2, LT = S::LT;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    float2 *Yk2 = reinterpret_cast<float2 *>(sm_raw);    // [DM][L2]  Ys_k[b, c] (mu, nu), split
    float2 *M12 = Yk2 + DM * L2;                          // [DM][L2]  Ys_k[b, c] S_c (mu', nu'), split
    float *Sbuf = reinterpret_cast<float *>(M12 + DM * L2);   // 2 x ([DM][LT] S_b (p, mu), [DM][LT] S_c (nu, nu'))
    const int b = pb[blockIdx.x], c = pc[blockIdx.x];
    const int k = blockIdx.z;
    const int ja = j0 + blockIdx.y * JT, jb = min(ja + JT, j0 + nj);
    const int n = tb.n;
    const int sb = tb.start[b], db = tb.dim[b], sc = tb.start[c], dc = tb.dim[c];
    const int DB = (db + 15) & ~15, DC = (dc + 7) & ~7;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const float *Sb_base = tb.sym32 + tb.off[b], *Sc_base = tb.sym32 + tb.off[c];
    auto issue = [&](int j, int buf) {   // symmetry j's two blocks (zero padded) into buffer `buf`
        float *sbd = Sbuf + buf * 2 * DM * LT, *scd = sbd + DM * LT;
        const float *Sbg = Sb_base + (long long)j * db * db, *Scg = Sc_base + (long long)j * dc * dc;
        for (int p = warp; p < DB; p += NW)
            for (int q = lane; q < DB; q += 32) {
                const bool v = p < db && q < db;
                cp_async4(&sbd[p * LT + q], v ? Sbg + p * db + q : Sbg, v);
            }
        for (int p = warp; p < DC; p += NW)
            for (int q = lane; q < DC; q += 32) {
                const bool v = p < dc && q < dc;
                cp_async4(&scd[p * LT + q], v ? Scg + p * dc + q : Scg, v);
            }
        cp_async_commit();
    };
    if (ja < jb) issue(ja, 0);
    const double *Yg = Ys + (long long)k * n * n;
    for (int mu = warp; mu < DB; mu += NW)
        for (int nu = lane; nu < DC; nu += 32)
            Yk2[mu * L2 + nu] = split2((mu < db && nu < dc) ? (float)Yg[(long long)(sb + mu) * n + sc + nu] : 0.f);
    const int mt = DB / 16, nt = DC / 8, tiles = mt * nt;
    for (int j = ja; j < jb; ++j) {
        const int cur = (j - ja) & 1;
        float *Sb = Sbuf + cur * 2 * DM * LT, *Sc = Sb + DM * LT;
        const long long r = (long long)k * nj + (j - j0);
        if (j + 1 < jb) {            // prefetch the next symmetry, then wait for this one
            issue(j + 1, cur ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        for (int ti = warp; ti < tiles; ti += NW) {
            const int m0 = (ti / nt) * 16, n0 = (ti % nt) * 8;
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            warp_tile<F2, F32>(acc, Yk2, L2, Sc, LT, m0, n0, DC / 8);
            store_tile_f2(M12, L2, m0, n0, acc);
        }
        if (b == c && (int)threadIdx.x < db) {   // r1 for the modes of block b: ups o (S_b^T R)
            const double *Rk = R1 + (long long)k * n + sb;
            double s = 0.0;
            for (int p = 0; p < db; ++p) s += (double)Sb[p * LT + threadIdx.x] * Rk[p];
            store_split(fmt, r1_hi, r1_lo, r * np + sb + threadIdx.x, ups[sb + threadIdx.x] * s);
        }
        __syncthreads();             // M1 complete; S_c of this symmetry no longer needed
        float *Tb = Sc;              // step-2 result staged where S_c was
        for (int ti = warp; ti < tiles; ti += NW) {
            const int m0 = (ti / nt) * 16, n0 = (ti % nt) * 8;
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            warp_tile<F32T, F2>(acc, Sb, LT, M12, L2, m0, n0, DB / 8);
            const int g = lane >> 2, t = lane & 3;
            *reinterpret_cast<float2 *>(&Tb[(m0 + g) * LT + n0 + 2 * t]) = make_float2(acc[0], acc[1]);
            *reinterpret_cast<float2 *>(&Tb[(m0 + g + 8) * LT + n0 + 2 * t]) = make_float2(acc[2], acc[3]);
        }
        __syncthreads();
        // one row mu per warp: consecutive lanes write consecutive packed pairs
        for (int mu = warp; mu < db; mu += NW) {
            const int gm = sb + mu;
            const long long row = r * Kp + pair_index(gm, gm, n) - gm;   // + gn gives pair(gm, gn)
            for (int nu = lane; nu < dc; nu += 32) {
                const int gn = sc + nu;
                if (gm <= gn) store_split_f(fmt, B1_hi, B1_lo, row + gn, Tb[mu * LT + nu]);
            }
        }
        __syncthreads();             // buffers of this symmetry free for the prefetch two steps ahead
    }
}

// ---- fold ---------------------------------------------------------------------------------------------
// grid (pairs of the class, fold chunks of Jf symmetries, nb).  Per symmetry:
//   W  (d_b x d_c) = ups_mu ups_nu (2 on the diagonal) Z[r, pair(mu, nu)]
//   step 1  U = W . S_c^T                   (A = W, B = S_c read transposed)
//   step 2  D += S_b . U                    (A = S_b, B = U2); fp32 per symmetry, summed in fp64
template <int MT>
__global__ void __launch_bounds__(THREADS)
fold_tc_kernel(SymTables tb, const int *__restrict__ pb, const int *__restrict__ pc, const float *__restrict__ Z, long long ldz,
               const float *__restrict__ F, long long ldf, const double *__restrict__ ups, int nj, int j0, int Jf, int nf_total,
               double *__restrict__ partD, double *__restrict__ partF) {
    using S = TcShape<MT>;
    constexpr int DM = S::DM, L2 = S::L2, LG = S::LG;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    float2 *U2 = reinterpret_cast<float2 *>(sm_raw);        // [DM][L2]  W S_c^T (mu', nu'), split
    float *Sbuf = reinterpret_cast<float *>(U2 + DM * L2);  // 2 x ([DM][LG] S_b (mu, p), S_c (nu', nu), W (mu, nu))
    const int b = pb[blockIdx.x], c = pc[blockIdx.x];
    const int fc = blockIdx.y, k = blockIdx.z;
    const int n = tb.n;
    const int sb = tb.start[b], db = tb.dim[b], sc = tb.start[c], dc = tb.dim[c];
    const int DB = (db + 15) & ~15, DC = (dc + 7) & ~7;
    const int fg = j0 / Jf + fc;
    const int ja = j0 + fc * Jf, jb = min(j0 + (fc + 1) * Jf, j0 + nj);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int mt = DB / 16, nt = DC / 8, tiles = mt * nt;
    const float *Sb_base = tb.sym32 + tb.off[b], *Sc_base = tb.sym32 + tb.off[c];
    auto issue = [&](int j, int buf) {   // symmetry j's blocks and its raw Z block into buffer `buf`
        float *sbd = Sbuf + buf * 3 * DM * LG, *scd = sbd + DM * LG, *wd = scd + DM * LG;
        const float *Sbg = Sb_base + (long long)j * db * db, *Scg = Sc_base + (long long)j * dc * dc;
        const float *Zr = Z + ((long long)k * nj + (j - j0)) * ldz;
        for (int p = warp; p < DB; p += NW)
            for (int q = lane; q < DB; q += 32) {
                const bool v = p < db && q < db;
                cp_async4(&sbd[p * LG + q], v ? Sbg + p * db + q : Sbg, v);
            }
        for (int p = warp; p < DC; p += NW)
            for (int q = lane; q < DC; q += 32) {
                const bool v = p < dc && q < dc;
                cp_async4(&scd[p * LG + q], v ? Scg + p * dc + q : Scg, v);
            }
        for (int mu = warp; mu < DB; mu += NW)
            for (int nu = lane; nu < DC; nu += 32) {
                const bool v = mu < db && nu < dc;
                int gm = sb + mu, gn = sc + nu;
                if (gm > gn) { const int s2 = gm; gm = gn; gn = s2; }
                cp_async4(&wd[mu * LG + nu], v ? Zr + pair_index(gm, gn, n) : Zr, v);
            }
        cp_async_commit();
    };
    // W = ups_mu ups_nu (2 on the diagonal) Z: each thread scales the elements it copied itself
    auto scale_w = [&](float *wd) {
        for (int mu = warp; mu < db; mu += NW)
            for (int nu = lane; nu < dc; nu += 32) {
                const int gm = sb + mu, gn = sc + nu;
                wd[mu * LG + nu] *= (float)((gm == gn ? 2.0 : 1.0) * ups[gm] * ups[gn]);
            }
    };
    constexpr int TPW = S::TILES_PER_WARP;   // step-2 tiles warp, warp + NW, ...: fp64 sums in registers
    double accD[TPW][4];
#pragma unroll
    for (int i = 0; i < TPW; ++i)
#pragma unroll
        for (int e = 0; e < 4; ++e) accD[i][e] = 0.0;
    double facc = 0.0;
    if (ja < jb) issue(ja, 0);
    for (int j = ja; j < jb; ++j) {
        const int cur = (j - ja) & 1;
        float *Sb = Sbuf + cur * 3 * DM * LG, *Sc = Sb + DM * LG, *W = Sc + DM * LG;
        const long long r = (long long)k * nj + (j - j0);
        if (j + 1 < jb) {
            issue(j + 1, cur ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        scale_w(W);
        __syncthreads();
        for (int ti = warp; ti < tiles; ti += NW) {
            const int m0 = (ti / nt) * 16, n0 = (ti % nt) * 8;
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            warp_tile<F32, F32T>(acc, W, LG, Sc, LG, m0, n0, DC / 8);
            store_tile_f2(U2, L2, m0, n0, acc);
        }
        if (b == c && (int)threadIdx.x < db) {
            const float *Fr = F + r * ldf + sb;
            double s = 0.0;
            for (int p = 0; p < db; ++p) s += (double)Sb[threadIdx.x * LG + p] * (double)Fr[p];
            facc += s;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < TPW; ++i) {
            const int ti = warp + i * NW;
            if (ti < tiles) {
                const int m0 = (ti / nt) * 16, n0 = (ti % nt) * 8;
                float acc[4] = {0.f, 0.f, 0.f, 0.f};
                warp_tile<F32, F2>(acc, Sb, LG, U2, L2, m0, n0, DB / 8);
#pragma unroll
                for (int e = 0; e < 4; ++e) accD[i][e] += (double)acc[e];
            }
        }
        __syncthreads();   // U2 and this symmetry's buffers free
    }
    double *out = partD + ((long long)k * nf_total + fg) * (long long)n * n;
#pragma unroll
    for (int i = 0; i < TPW; ++i) {
        const int ti = warp + i * NW;
        if (ti >= tiles) continue;
        const int m0 = (ti / nt) * 16, n0 = (ti % nt) * 8;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int mu = m0 + g + 8 * (e >> 1), nu = n0 + 2 * t + (e & 1);
            if (mu < db && nu < dc) out[(long long)(sb + mu) * n + sc + nu] = accD[i][e];
        }
    }
    if (b == c && (int)threadIdx.x < db) partF[((long long)k * nf_total + fg) * n + sb + threadIdx.x] = facc;
}

template <int MT>
int launch_transform_tc(const SymTables &t, const PairClasses &pc, int nb, int nj, int j0, const double *Ys, const double *R1,
                        const double *ups, long long Kp, long long np, Format fmt, void *B1_hi, void *B1_lo, void *r1_hi,
                        void *r1_lo, cudaStream_t st) {
    if (!pc.count[MT]) return 0;
    using S = TcShape<MT>;
    static_assert(S::TRANSFORM_SMEM <= 227 * 1024, "transform shared memory");
    constexpr int JT = 16;
    auto kern = transform_tc_kernel<MT>;
    TD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::TRANSFORM_SMEM));
    dim3 grid((unsigned)pc.count[MT], (unsigned)ceil_div(nj, JT), (unsigned)nb);
    kern<<<grid, THREADS, S::TRANSFORM_SMEM, st>>>(t, pc.b[MT], pc.c[MT], nj, j0, JT, Ys, R1, ups, Kp, np, fmt, B1_hi, B1_lo,
                                                    r1_hi, r1_lo);
    TD_CUDA(cudaGetLastError());
    return 0;
}

template <int MT>
int launch_fold_tc(const SymTables &t, const PairClasses &pc, int nb, int nj, int j0, int Jf, int nf_total, const float *Z,
                   long long ldz, const float *F, long long ldf, const double *ups, double *partD, double *partF, cudaStream_t st) {
    if (!pc.count[MT]) return 0;
    using S = TcShape<MT>;
    static_assert(S::FOLD_SMEM <= 227 * 1024, "fold shared memory");
    auto kern = fold_tc_kernel<MT>;
    TD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::FOLD_SMEM));
    dim3 grid((unsigned)pc.count[MT], (unsigned)ceil_div(nj, Jf), (unsigned)nb);
    kern<<<grid, THREADS, S::FOLD_SMEM, st>>>(t, pc.b[MT], pc.c[MT], Z, ldz, F, ldf, ups, nj, j0, Jf, nf_total, partD, partF);
    TD_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace

int sym_transform_tc(const SymTables &t, const PairClasses &pc, int nb, int nj, int j0, const double *Ys, const double *R1,
                     const double *ups, long long Kp, long long np, Format fmt, void *B1_hi, void *B1_lo, void *r1_hi,
                     void *r1_lo, cudaStream_t st) {
    TD_CHECK(fmt == FMT_BF16 || fmt == FMT_TF32, TDSCHA_EINVAL, "tensor-core symmetry transform needs a split storage format");
    TD_TRY((launch_transform_tc<1>(t, pc, nb, nj, j0, Ys, R1, ups, Kp, np, fmt, B1_hi, B1_lo, r1_hi, r1_lo, st)));
    TD_TRY((launch_transform_tc<2>(t, pc, nb, nj, j0, Ys, R1, ups, Kp, np, fmt, B1_hi, B1_lo, r1_hi, r1_lo, st)));
    TD_TRY((launch_transform_tc<3>(t, pc, nb, nj, j0, Ys, R1, ups, Kp, np, fmt, B1_hi, B1_lo, r1_hi, r1_lo, st)));
    TD_TRY((launch_transform_tc<4>(t, pc, nb, nj, j0, Ys, R1, ups, Kp, np, fmt, B1_hi, B1_lo, r1_hi, r1_lo, st)));
    TD_TRY((launch_transform_tc<5>(t, pc, nb, nj, j0, Ys, R1, ups, Kp, np, fmt, B1_hi, B1_lo, r1_hi, r1_lo, st)));
    return 0;
}

int sym_fold_tc(const SymTables &t, const PairClasses &pc, int nb, int nj, int j0, int Jf, int nf_total, const float *Z,
                long long ldz, const float *F, long long ldf, const double *ups, double *partD, double *partF, cudaStream_t st) {
    TD_TRY((launch_fold_tc<1>(t, pc, nb, nj, j0, Jf, nf_total, Z, ldz, F, ldf, ups, partD, partF, st)));
    TD_TRY((launch_fold_tc<2>(t, pc, nb, nj, j0, Jf, nf_total, Z, ldz, F, ldf, ups, partD, partF, st)));
    TD_TRY((launch_fold_tc<3>(t, pc, nb, nj, j0, Jf, nf_total, Z, ldz, F, ldf, ups, partD, partF, st)));
    TD_TRY((launch_fold_tc<4>(t, pc, nb, nj, j0, Jf, nf_total, Z, ldz, F, ldf, ups, partD, partF, st)));
    TD_TRY((launch_fold_tc<5>(t, pc, nb, nj, j0, Jf, nf_total, Z, ldz, F, ldf, ups, partD, partF, st)));
    return 0;
}

}  // namespace tdscha
