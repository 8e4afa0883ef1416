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
//   * Fragments come from shared memory through ldmatrix (one instruction per four tf32 values of
//     a warp tile).  B operands are stored n-major ([n][k]), the layout ldmatrix hands out as the
//     "col" fragment, so the symmetry blocks come from a transposed copy where needed and the
//     intermediate products are written transposed.
//   * Operands reused across symmetries or tiles (the Ys block, the intermediate product) are kept
//     already split into tf32 hi / lo arrays; symmetry blocks and the fold's weights are fp32 and
//     split after the ldmatrix.
//   * Symmetry j + 1's blocks (16-byte cp.async from zero-padded fp32 tables) are copied into the
//     second half of a double buffer while symmetry j is computed.
//   * Block dimensions are zero-padded to 16 on the m side and 8 on the n and k sides.  Every
//     shared array has leading dimension ld = 4 (mod 8) floats, which makes the ldmatrix row
//     addresses and the transposed fragment stores free of bank conflicts.
#include <algorithm>
#include <cstdlib>
#include <cstdint>
#include <cuda_bf16.h>

#include "symmetry.cuh"

namespace tdscha {
namespace {

// threads of a CTA per block class: small classes get small CTAs (several per SM) so that the
// fixed per-symmetry cost (table copy, barriers) of their many small block pairs overlaps
__host__ __device__ constexpr int threads_for(int MT) { return MT <= 2 ? 128 : (MT == 3 ? 256 : 512); }

__host__ __device__ constexpr int ld_for(int d) { return d + ((4 - d % 8) + 8) % 8; }   // ld = 4 (mod 8)

__device__ __forceinline__ long long pair_index(int mu, int nu, int n) {   // mu <= nu, row-major upper triangle
    return (long long)mu * n - ((long long)mu * (mu - 1)) / 2 + (nu - mu);
}
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ uint32_t to_tf32(float v) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
    return r;
}
__device__ __forceinline__ void split_tf32(float v, uint32_t &hi, uint32_t &lo) {
    hi = to_tf32(v);
    lo = to_tf32(v - __uint_as_float(hi));
}
__device__ __forceinline__ void mma_tf32(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// ldmatrix of 8 x 8 b16 matrices = 8 rows x 4 fp32 words: thread 4g + t receives word t of row g.
__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], uint32_t addr) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(addr));
}
__device__ __forceinline__ void ldsm_x2(uint32_t (&r)[2], uint32_t addr) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];" : "=r"(r[0]), "=r"(r[1]) : "r"(addr));
}

// asynchronous global -> shared copies; `valid` false writes zeros instead (src-size 0)
__device__ __forceinline__ void cp_async4(float *dst, const float *src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(valid ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cp_async16(float *dst, const float *src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(PENDING) : "memory"); }

// rows x cols (cols a multiple of 4) of a (dp x dp) zero-padded fp32 table into shared memory with
// leading dimension ld; rows / chunks beyond the table are zero filled
template <int LD, int THREADS>
__device__ __forceinline__ void copy_table(float *dst, const float *src, int dp, int rows, int cols) {
    const int cpr = cols >> 2;
    for (int e = threadIdx.x; e < rows * cpr; e += THREADS) {
        const int r = e / cpr, ch = e - r * cpr;
        const bool v = r < dp && 4 * ch < dp;
        cp_async16(dst + r * LD + 4 * ch, v ? src + (long long)r * dp + 4 * ch : src, v);
    }
}

// c += A[m0:m0+16, 0:8 kt] . B[0:8 kt, n0:n0+8] with three-term tf32 splitting.  A is stored
// row-major [m][k], B n-major [n][k], both with leading dimension LD.  A_SPLIT / B_SPLIT: the
// operand is given as separate hi / lo arrays; otherwise it is one fp32 array split on load.
// Fragment layouts of m16n8k8 (g = lane / 4, t = lane % 4): a0 (g, t), a1 (g + 8, t),
// a2 (g, t + 4), a3 (g + 8, t + 4); b0 (k = t, n = g), b1 (k = t + 4, n = g).
template <int LD, bool A_SPLIT, bool B_SPLIT>
__device__ __forceinline__ void warp_tile(float (&c)[4], const float *Ahi, const float *Alo, const float *Bhi, const float *Blo,
                                          int m0, int n0, int kt) {
    const int lane = threadIdx.x & 31, q = lane >> 3, r8 = lane & 7;
    const uint32_t a_off = (uint32_t)(((m0 + r8 + 8 * (q & 1)) * LD + 4 * (q >> 1)) * 4);
    const uint32_t b_off = (uint32_t)(((n0 + r8) * LD + 4 * (q & 1)) * 4);
    const uint32_t ah_base = smem_u32(Ahi) + a_off, bh_base = smem_u32(Bhi) + b_off;
    const uint32_t al_base = A_SPLIT ? smem_u32(Alo) + a_off : 0u, bl_base = B_SPLIT ? smem_u32(Blo) + b_off : 0u;
    float c_lh[4] = {0.f, 0.f, 0.f, 0.f}, c_hl[4] = {0.f, 0.f, 0.f, 0.f}, c_hh[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 2
    for (int ks = 0; ks < kt; ++ks) {
        uint32_t ah[4], al[4], bh[2], bl[2];
        if constexpr (A_SPLIT) {
            ldsm_x4(ah, ah_base + ks * 32);
            ldsm_x4(al, al_base + ks * 32);
        } else {
            uint32_t raw[4];
            ldsm_x4(raw, ah_base + ks * 32);
#pragma unroll
            for (int i = 0; i < 4; ++i) split_tf32(__uint_as_float(raw[i]), ah[i], al[i]);
        }
        if constexpr (B_SPLIT) {
            ldsm_x2(bh, bh_base + ks * 32);
            ldsm_x2(bl, bl_base + ks * 32);
        } else {
            uint32_t raw[2];
            ldsm_x2(raw, bh_base + ks * 32);
#pragma unroll
            for (int i = 0; i < 2; ++i) split_tf32(__uint_as_float(raw[i]), bh[i], bl[i]);
        }
        mma_tf32(c_lh, al, bh[0], bh[1]);   // three independent accumulation chains: the tensor
        mma_tf32(c_hl, ah, bl[0], bl[1]);   // pipe overlaps them instead of waiting on one chain
        mma_tf32(c_hh, ah, bh[0], bh[1]);
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) c[e] += (c_lh[e] + c_hl[e]) + c_hh[e];   // small terms first
}

// a warp tile's accumulators, transposed ([n][m]) and split, into hi / lo arrays
template <int LD>
__device__ __forceinline__ void store_tile_t(float *Xhi, float *Xlo, int m0, int n0, const float (&c)[4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const int idx = (n0 + 2 * t + (e & 1)) * LD + m0 + g + 8 * (e >> 1);
        uint32_t h, l;
        split_tf32(c[e], h, l);
        Xhi[idx] = __uint_as_float(h);
        Xlo[idx] = __uint_as_float(l);
    }
}

// bf16 / tf32 hi + lo of an fp32 value into the GEMM operand arrays (FMT_F32: the value itself)
__device__ __forceinline__ void store_split_f(Format fmt, void *hi, void *lo, long long idx, float x) {
    if (fmt == FMT_F32) {
        static_cast<float *>(hi)[idx] = x;
    } else if (fmt == FMT_BF16) {
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
    static constexpr int LD = ld_for(DM);
    static constexpr int ARR = DM * LD;   // floats per shared array
    static constexpr size_t SMEM = (size_t)8 * ARR * sizeof(float);
    static constexpr int THREADS = threads_for(MT);
    static constexpr int NW = THREADS / 32;
    // fold step-2 tiles per warp (16 x 8 tiles of the largest block pair of the class)
    static constexpr int TILES_PER_WARP = ((DM / 16) * (DM / 8) + NW - 1) / NW;
};

// ---- transform ---------------------------------------------------------------------------------------
// grid (pairs of the class, j-chunks of JT symmetries, nb).  Per symmetry:
//   step 1  M1 (d_b x d_c) = Ys_k[b, c] . S_c       A = Y (split), B[n][k] = S_c^T (transposed table)
//   step 2  T  (d_b x d_c) = S_b^T . M1              A = S_b^T (transposed table), B[n][k] = M1^T (split)
// T is staged in shared memory and written row by row to B1 (packed pairs, format fmt) for
// global modes mu <= nu.
template <int MT>
__global__ void __launch_bounds__(threads_for(MT))
transform_tc_kernel(SymTables tb, const int *__restrict__ pb, const int *__restrict__ pc, int nj, int j0, int JT,
                    const double *__restrict__ Ys, const double *__restrict__ R1, const double *__restrict__ ups, long long Kp,
                    long long np, Format fmt, void *B1_hi, void *B1_lo, void *r1_hi, void *r1_lo) {
    using S = TcShape<MT>;
    constexpr int LD = S::LD, ARR = S::ARR, NW = S::NW;
    extern __shared__ __align__(16) float smf[];
    float *Yhi = smf, *Ylo = smf + ARR;               // Ys_k[b, c] (mu, nu)
    float *MThi = smf + 2 * ARR, *MTlo = smf + 3 * ARR;   // M1^T (nu', mu')
    float *Tab = smf + 4 * ARR;                       // buffers x {S_b^T (mu, p), S_c^T (nu', nu)}
    const int b = pb[blockIdx.x], c = pc[blockIdx.x];
    const int k = blockIdx.z;
    const int ja = j0 + blockIdx.y * JT, jb = min(ja + JT, j0 + nj);
    const int n = tb.n;
    const int sb = tb.start[b], db = tb.dim[b], sc = tb.start[c], dc = tb.dim[c];
    const int DB = (db + 15) & ~15, DB8 = (db + 7) & ~7, DC = (dc + 7) & ~7;
    const int dpb = (db + 3) & ~3, dpc = (dc + 3) & ~3;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const float *Tb_base = tb.symPT + tb.offP[b], *Tc_base = tb.symPT + tb.offP[c];
    auto issue = [&](int j, int buf) {
        float *stb = Tab + buf * 2 * ARR, *stc = stb + ARR;
        copy_table<LD, S::THREADS>(stb, Tb_base + (long long)j * dpb * dpb, dpb, DB, DB8);
        copy_table<LD, S::THREADS>(stc, Tc_base + (long long)j * dpc * dpc, dpc, DC, DC);
        cp_async_commit();
    };
    if (ja < jb) issue(ja, 0);
    const double *Yg = Ys + (long long)k * n * n;
    for (int mu = warp; mu < DB; mu += NW)
        for (int nu = lane; nu < DC; nu += 32) {
            uint32_t h, l;
            split_tf32((mu < db && nu < dc) ? (float)Yg[(long long)(sb + mu) * n + sc + nu] : 0.f, h, l);
            Yhi[mu * LD + nu] = __uint_as_float(h);
            Ylo[mu * LD + nu] = __uint_as_float(l);
        }
    const int mt = DB / 16, nt = DC / 8, tiles = mt * nt;
    for (int j = ja; j < jb; ++j) {
        const int cur = (j - ja) & 1;
        float *STb = Tab + cur * 2 * ARR, *STc = STb + ARR;
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
            warp_tile<LD, true, false>(acc, Yhi, Ylo, STc, nullptr, m0, n0, DC / 8);
            store_tile_t<LD>(MThi, MTlo, m0, n0, acc);
        }
        if (b == c && (int)threadIdx.x < db) {   // r1 for the modes of block b: ups o (S_b^T R)
            const double *Rk = R1 + (long long)k * n + sb;
            double s = 0.0;
            for (int p = 0; p < db; ++p) s += (double)STb[threadIdx.x * LD + p] * Rk[p];
            store_split(fmt, r1_hi, r1_lo, r * np + sb + threadIdx.x, ups[sb + threadIdx.x] * s);
        }
        __syncthreads();             // M1 complete; S_c of this symmetry no longer needed
        float *T = STc;              // step-2 result staged where S_c^T was
        for (int ti = warp; ti < tiles; ti += NW) {
            const int m0 = (ti / nt) * 16, n0 = (ti % nt) * 8;
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            warp_tile<LD, false, true>(acc, STb, nullptr, MThi, MTlo, m0, n0, DB8 / 8);
            const int g = lane >> 2, t = lane & 3;
            *reinterpret_cast<float2 *>(&T[(m0 + g) * LD + n0 + 2 * t]) = make_float2(acc[0], acc[1]);
            *reinterpret_cast<float2 *>(&T[(m0 + g + 8) * LD + n0 + 2 * t]) = make_float2(acc[2], acc[3]);
        }
        __syncthreads();
        // one row mu per warp: consecutive lanes write consecutive packed pairs
        for (int mu = warp; mu < db; mu += NW) {
            const int gm = sb + mu;
            const long long row = r * Kp + pair_index(gm, gm, n) - gm;   // + gn gives pair(gm, gn)
            for (int nu = lane; nu < dc; nu += 32) {
                const int gn = sc + nu;
                if (gm <= gn) store_split_f(fmt, B1_hi, B1_lo, row + gn, T[mu * LD + nu]);
            }
        }
        __syncthreads();             // buffers of this symmetry free for the prefetch two steps ahead
    }
}

// The same transform with a quarter of the shared memory (four arrays instead of eight), so that two
// CTAs share an SM and hide each other's per-symmetry latency: the Ys block and the intermediate
// product are kept as fp32 and split into tf32 hi / lo as they are loaded into fragments (the same
// values as the pre-split arrays, so the results are bit-identical), and the two symmetry tables
// have one buffer (the copy of symmetry j + 1 is issued after symmetry j is stored).
template <int MT>
__global__ void __launch_bounds__(threads_for(MT), 2)
transform_tc_lean_kernel(SymTables tb, const int *__restrict__ pb, const int *__restrict__ pc, int nj, int j0, int JT,
                         const double *__restrict__ Ys, const double *__restrict__ R1, const double *__restrict__ ups,
                         long long Kp, long long np, Format fmt, void *B1_hi, void *B1_lo, void *r1_hi, void *r1_lo) {
    using S = TcShape<MT>;
    constexpr int LD = S::LD, ARR = S::ARR, NW = S::NW;
    extern __shared__ __align__(16) float smf[];
    float *Yr = smf;                       // Ys_k[b, c] (mu, nu), fp32
    float *MTr = smf + ARR;                // M1^T (nu', mu'), fp32
    float *STb = smf + 2 * ARR, *STc = smf + 3 * ARR;   // S_b^T (mu, p), S_c^T (nu', nu) of the symmetry
    const int b = pb[blockIdx.x], c = pc[blockIdx.x];
    const int k = blockIdx.z;
    const int ja = j0 + blockIdx.y * JT, jb = min(ja + JT, j0 + nj);
    const int n = tb.n;
    const int sb = tb.start[b], db = tb.dim[b], sc = tb.start[c], dc = tb.dim[c];
    const int DB = (db + 15) & ~15, DB8 = (db + 7) & ~7, DC = (dc + 7) & ~7;
    const int dpb = (db + 3) & ~3, dpc = (dc + 3) & ~3;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const float *Tb_base = tb.symPT + tb.offP[b], *Tc_base = tb.symPT + tb.offP[c];
    const double *Yg = Ys + (long long)k * n * n;
    for (int mu = warp; mu < DB; mu += NW)
        for (int nu = lane; nu < DC; nu += 32)
            Yr[mu * LD + nu] = (mu < db && nu < dc) ? (float)Yg[(long long)(sb + mu) * n + sc + nu] : 0.f;
    const int mt = DB / 16, nt = DC / 8, tiles = mt * nt;
    for (int j = ja; j < jb; ++j) {
        const long long r = (long long)k * nj + (j - j0);
        copy_table<LD, S::THREADS>(STb, Tb_base + (long long)j * dpb * dpb, dpb, DB, DB8);
        copy_table<LD, S::THREADS>(STc, Tc_base + (long long)j * dpc * dpc, dpc, DC, DC);
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
        for (int ti = warp; ti < tiles; ti += NW) {
            const int m0 = (ti / nt) * 16, n0 = (ti % nt) * 8;
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            warp_tile<LD, false, false>(acc, Yr, nullptr, STc, nullptr, m0, n0, DC / 8);
            const int g = lane >> 2, t = lane & 3;
#pragma unroll
            for (int e = 0; e < 4; ++e) MTr[(n0 + 2 * t + (e & 1)) * LD + m0 + g + 8 * (e >> 1)] = acc[e];
        }
        if (b == c && (int)threadIdx.x < db) {   // r1 for the modes of block b: ups o (S_b^T R)
            const double *Rk = R1 + (long long)k * n + sb;
            double s = 0.0;
            for (int p = 0; p < db; ++p) s += (double)STb[threadIdx.x * LD + p] * Rk[p];
            store_split(fmt, r1_hi, r1_lo, r * np + sb + threadIdx.x, ups[sb + threadIdx.x] * s);
        }
        __syncthreads();             // M1 complete; S_c of this symmetry no longer needed
        float *T = STc;              // step-2 result staged where S_c^T was
        for (int ti = warp; ti < tiles; ti += NW) {
            const int m0 = (ti / nt) * 16, n0 = (ti % nt) * 8;
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            warp_tile<LD, false, false>(acc, STb, nullptr, MTr, nullptr, m0, n0, DB8 / 8);
            const int g = lane >> 2, t = lane & 3;
            *reinterpret_cast<float2 *>(&T[(m0 + g) * LD + n0 + 2 * t]) = make_float2(acc[0], acc[1]);
            *reinterpret_cast<float2 *>(&T[(m0 + g + 8) * LD + n0 + 2 * t]) = make_float2(acc[2], acc[3]);
        }
        __syncthreads();
        for (int mu = warp; mu < db; mu += NW) {
            const int gm = sb + mu;
            const long long row = r * Kp + pair_index(gm, gm, n) - gm;   // + gn gives pair(gm, gn)
            for (int nu = lane; nu < dc; nu += 32) {
                const int gn = sc + nu;
                if (gm <= gn) store_split_f(fmt, B1_hi, B1_lo, row + gn, T[mu * LD + nu]);
            }
        }
        __syncthreads();             // the tables' buffers are free for the next symmetry's copy
    }
}

// ---- fold ---------------------------------------------------------------------------------------------
// grid (pairs of the class, fold chunks of Jf symmetries, nb).  Per symmetry:
//   W  (d_b x d_c) = ups_mu ups_nu (2 on the diagonal) Z[r, pair(mu, nu)]
//   step 1  U = W . S_c^T          A = W (fp32), B[n][k] = S_c (table as given)
//   step 2  D += S_b . U           A = S_b (table as given), B[n][k] = U^T (split); fp32 per
//                                  symmetry, summed over symmetries in fp64
template <int MT>
__global__ void __launch_bounds__(threads_for(MT))
fold_tc_kernel(SymTables tb, const int *__restrict__ pb, const int *__restrict__ pc, const float *__restrict__ Z, long long ldz,
               const float *__restrict__ F, long long ldf, const double *__restrict__ ups, int nj, int j0, int Jf, int nf_total,
               double *__restrict__ partD, double *__restrict__ partF) {
    using S = TcShape<MT>;
    constexpr int LD = S::LD, ARR = S::ARR, NW = S::NW;
    extern __shared__ __align__(16) float smf[];
    float *UThi = smf, *UTlo = smf + ARR;   // U^T (nu', mu')
    float *Buf = smf + 2 * ARR;             // buffers x {S_b (mu, p), S_c (nu', nu), W (mu, nu)}
    const int b = pb[blockIdx.x], c = pc[blockIdx.x];
    const int fc = blockIdx.y, k = blockIdx.z;
    const int n = tb.n;
    const int sb = tb.start[b], db = tb.dim[b], sc = tb.start[c], dc = tb.dim[c];
    const int DB = (db + 15) & ~15, DB8 = (db + 7) & ~7, DC = (dc + 7) & ~7;
    const int dpb = (db + 3) & ~3, dpc = (dc + 3) & ~3;
    const int fg = j0 / Jf + fc;
    const int ja = j0 + fc * Jf, jb = min(j0 + (fc + 1) * Jf, j0 + nj);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int mt = DB / 16, nt = DC / 8, tiles = mt * nt;
    const float *Pb_base = tb.symP + tb.offP[b], *Pc_base = tb.symP + tb.offP[c];
    auto issue = [&](int j, int buf) {
        float *snb = Buf + buf * 3 * ARR, *snc = snb + ARR, *wd = snc + ARR;
        copy_table<LD, S::THREADS>(snb, Pb_base + (long long)j * dpb * dpb, dpb, DB, DB8);
        copy_table<LD, S::THREADS>(snc, Pc_base + (long long)j * dpc * dpc, dpc, DC, DC);
        const float *Zr = Z + ((long long)k * nj + (j - j0)) * ldz;
        for (int mu = warp; mu < DB; mu += NW)
            for (int nu = lane; nu < DC; nu += 32) {
                const bool v = mu < db && nu < dc;
                int gm = sb + mu, gn = sc + nu;
                if (gm > gn) { const int s2 = gm; gm = gn; gn = s2; }
                cp_async4(&wd[mu * LD + nu], v ? Zr + pair_index(gm, gn, n) : Zr, v);
            }
        cp_async_commit();
    };
    // W = ups_mu ups_nu (2 on the diagonal) Z: each thread scales the elements it copied itself
    auto scale_w = [&](float *wd) {
        for (int mu = warp; mu < db; mu += NW)
            for (int nu = lane; nu < dc; nu += 32) {
                const int gm = sb + mu, gn = sc + nu;
                wd[mu * LD + nu] *= (float)((gm == gn ? 2.0 : 1.0) * ups[gm] * ups[gn]);
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
        float *SNb = Buf + cur * 3 * ARR, *SNc = SNb + ARR, *W = SNc + ARR;
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
            warp_tile<LD, false, false>(acc, W, nullptr, SNc, nullptr, m0, n0, DC / 8);
            store_tile_t<LD>(UThi, UTlo, m0, n0, acc);
        }
        if (b == c && (int)threadIdx.x < db) {
            const float *Fr = F + r * ldf + sb;
            double s = 0.0;
            for (int p = 0; p < db; ++p) s += (double)SNb[threadIdx.x * LD + p] * (double)Fr[p];
            facc += s;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < TPW; ++i) {
            const int ti = warp + i * NW;
            if (ti < tiles) {
                const int m0 = (ti / nt) * 16, n0 = (ti % nt) * 8;
                float acc[4] = {0.f, 0.f, 0.f, 0.f};
                warp_tile<LD, false, true>(acc, SNb, nullptr, UThi, UTlo, m0, n0, DB8 / 8);
#pragma unroll
                for (int e = 0; e < 4; ++e) accD[i][e] += (double)acc[e];
            }
        }
        __syncthreads();   // U^T and this symmetry's buffers free
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

// The fold with four shared arrays (U^T as fp32 split into tf32 hi / lo on load, one buffer of the
// symmetry's S_b, S_c and W) and at most 256 threads, so that two CTAs share an SM: bit-identical to
// fold_tc_kernel (same split values, same product order, same fp64 sums).
__host__ __device__ constexpr int lean_fold_threads(int MT) { return threads_for(MT) < 256 ? threads_for(MT) : 256; }

template <int MT>
__global__ void __launch_bounds__(lean_fold_threads(MT), 2)
fold_tc_lean_kernel(SymTables tb, const int *__restrict__ pb, const int *__restrict__ pc, const float *__restrict__ Z,
                    long long ldz, const float *__restrict__ F, long long ldf, const double *__restrict__ ups, int nj, int j0,
                    int Jf, int nf_total, double *__restrict__ partD, double *__restrict__ partF) {
    using S = TcShape<MT>;
    constexpr int LD = S::LD, ARR = S::ARR;
    constexpr int THREADS = lean_fold_threads(MT), NW = THREADS / 32;
    constexpr int TPW = ((S::DM / 16) * (S::DM / 8) + NW - 1) / NW;
    extern __shared__ __align__(16) float smf[];
    float *UTr = smf;                                       // U^T (nu', mu'), fp32
    float *SNb = smf + ARR, *SNc = smf + 2 * ARR, *W = smf + 3 * ARR;
    const int b = pb[blockIdx.x], c = pc[blockIdx.x];
    const int fc = blockIdx.y, k = blockIdx.z;
    const int n = tb.n;
    const int sb = tb.start[b], db = tb.dim[b], sc = tb.start[c], dc = tb.dim[c];
    const int DB = (db + 15) & ~15, DB8 = (db + 7) & ~7, DC = (dc + 7) & ~7;
    const int dpb = (db + 3) & ~3, dpc = (dc + 3) & ~3;
    const int fg = j0 / Jf + fc;
    const int ja = j0 + fc * Jf, jb = min(j0 + (fc + 1) * Jf, j0 + nj);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int mt = DB / 16, nt = DC / 8, tiles = mt * nt;
    const float *Pb_base = tb.symP + tb.offP[b], *Pc_base = tb.symP + tb.offP[c];
    double accD[TPW][4];
#pragma unroll
    for (int i = 0; i < TPW; ++i)
#pragma unroll
        for (int e = 0; e < 4; ++e) accD[i][e] = 0.0;
    double facc = 0.0;
    for (int j = ja; j < jb; ++j) {
        const long long r = (long long)k * nj + (j - j0);
        copy_table<LD, THREADS>(SNb, Pb_base + (long long)j * dpb * dpb, dpb, DB, DB8);
        copy_table<LD, THREADS>(SNc, Pc_base + (long long)j * dpc * dpc, dpc, DC, DC);
        const float *Zr = Z + r * ldz;
        for (int mu = warp; mu < DB; mu += NW)
            for (int nu = lane; nu < DC; nu += 32) {
                const bool v = mu < db && nu < dc;
                int gm = sb + mu, gn = sc + nu;
                if (gm > gn) { const int s2 = gm; gm = gn; gn = s2; }
                cp_async4(&W[mu * LD + nu], v ? Zr + pair_index(gm, gn, n) : Zr, v);
            }
        cp_async_commit();
        cp_async_wait<0>();
        // W = ups_mu ups_nu (2 on the diagonal) Z: each thread scales the elements it copied itself
        for (int mu = warp; mu < db; mu += NW)
            for (int nu = lane; nu < dc; nu += 32) {
                const int gm = sb + mu, gn = sc + nu;
                W[mu * LD + nu] *= (float)((gm == gn ? 2.0 : 1.0) * ups[gm] * ups[gn]);
            }
        __syncthreads();
        for (int ti = warp; ti < tiles; ti += NW) {
            const int m0 = (ti / nt) * 16, n0 = (ti % nt) * 8;
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            warp_tile<LD, false, false>(acc, W, nullptr, SNc, nullptr, m0, n0, DC / 8);
#pragma unroll
            for (int e = 0; e < 4; ++e) UTr[(n0 + 2 * t + (e & 1)) * LD + m0 + g + 8 * (e >> 1)] = acc[e];
        }
        if (b == c && (int)threadIdx.x < db) {
            const float *Fr = F + r * ldf + sb;
            double sum = 0.0;
            for (int p = 0; p < db; ++p) sum += (double)SNb[threadIdx.x * LD + p] * (double)Fr[p];
            facc += sum;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < TPW; ++i) {
            const int ti = warp + i * NW;
            if (ti < tiles) {
                const int m0 = (ti / nt) * 16, n0 = (ti % nt) * 8;
                float acc[4] = {0.f, 0.f, 0.f, 0.f};
                warp_tile<LD, false, false>(acc, SNb, nullptr, UTr, nullptr, m0, n0, DB8 / 8);
#pragma unroll
                for (int e = 0; e < 4; ++e) accD[i][e] += (double)acc[e];
            }
        }
        __syncthreads();   // U^T and this symmetry's buffers free
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
    static_assert(S::SMEM <= 227 * 1024, "shared memory");
    constexpr int JT = 16;
    // the lean kernel (half the shared memory: two CTAs per SM) unless TDSCHA_SYM_LEAN=0
    const char *env = getenv("TDSCHA_SYM_LEAN");
    const bool lean = !(env && atoi(env) == 0);
    auto kern = lean ? transform_tc_lean_kernel<MT> : transform_tc_kernel<MT>;
    const size_t smem = lean ? S::SMEM / 2 : S::SMEM;
    TD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)pc.count[MT], (unsigned)ceil_div(nj, JT), (unsigned)nb);
    kern<<<grid, S::THREADS, smem, st>>>(t, pc.b[MT], pc.c[MT], nj, j0, JT, Ys, R1, ups, Kp, np, fmt, B1_hi, B1_lo, r1_hi, r1_lo);
    TD_CUDA(cudaGetLastError());
    return 0;
}

template <int MT>
int launch_fold_tc(const SymTables &t, const PairClasses &pc, int nb, int nj, int j0, int Jf, int nf_total, const float *Z,
                   long long ldz, const float *F, long long ldf, const double *ups, double *partD, double *partF, cudaStream_t st) {
    if (!pc.count[MT]) return 0;
    using S = TcShape<MT>;
    static_assert(S::SMEM <= 227 * 1024, "shared memory");
    // the lean kernel (half the shared memory, two CTAs per SM) unless TDSCHA_SYM_LEAN=0
    const char *env = getenv("TDSCHA_SYM_LEAN");
    const bool lean = !(env && atoi(env) == 0);
    auto kern = lean ? fold_tc_lean_kernel<MT> : fold_tc_kernel<MT>;
    const size_t smem = lean ? S::SMEM / 2 : S::SMEM;
    const int threads = lean ? lean_fold_threads(MT) : S::THREADS;
    TD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)pc.count[MT], (unsigned)ceil_div(nj, Jf), (unsigned)nb);
    kern<<<grid, threads, smem, st>>>(t, pc.b[MT], pc.c[MT], Z, ldz, F, ldf, ups, nj, j0, Jf, nf_total, partD, partF);
    TD_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace

int sym_transform_tc(const SymTables &t, const PairClasses &pc, int nb, int nj, int j0, const double *Ys, const double *R1,
                     const double *ups, long long Kp, long long np, Format fmt, void *B1_hi, void *B1_lo, void *r1_hi,
                     void *r1_lo, cudaStream_t st) {
    TD_CHECK(fmt == FMT_BF16 || fmt == FMT_TF32 || fmt == FMT_F32, TDSCHA_EINVAL,
             "tensor-core symmetry transform needs a split storage format or fp32");
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
