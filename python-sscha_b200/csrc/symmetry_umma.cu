// symmetry_umma.cu -- the symmetry transform and fold of the bf16 storage formats on the 5th-generation
// tensor cores: tcgen05.mma kind::f16 on bf16 hi / lo operands (hi.hi + hi.lo + lo.hi, FP32
// accumulation in tensor memory), symmetry tables brought in by TMA.
//
// Per block pair (b <= c) and symmetry j the two d_b x d_c products of the reference's block gather
// (CModules/LanczosFunctions.c:2158-2170, applied here to the n x n objects instead of the images):
//
//   transform   T_kj = S_b^T  Ys_k[b, c]  S_c          (the packed rows of B1, one per (k, j))
//   fold        D_k += S_b    W_kj        S_c^T        (summed over a chunk of symmetries)
//
// are arranged so that both products of one symmetry are tensor-core contractions whose operands are
// shared by g vectors k and never need a transpose:
//
//   MMA1   D1[nu'][(k, mu)] = sum_nu  A1[nu'][nu] . Bv[(k, mu)][nu]       M = 128 (nu' < d_c valid)
//            transform: A1 = S_c^T, Bv = Ys_k[b, c]  ->  D1 = (Ys_k S_c)^T per k
//            fold:      A1 = S_c,   Bv = W_kj        ->  D1 = (W_kj S_c^T)^T per k
//   MMA2   D2[mu'][(k, nu')] = sum_mu A2[mu'][mu] . B2[(k, nu')][mu]     M = 128 (mu' < d_b valid)
//            B2 = D1 read back row by row (thread nu' owns row nu' of every vector's product)
//            transform: A2 = S_b^T -> D2 = T_kj;   fold: A2 = S_b -> D2 accumulates S_b U_kj
//
// Operands are K-major with the 32-byte swizzle: K is cut into regions of 16 bf16 (one MMA K step),
// each region holds its rows at 32 bytes.  An A operand is read as 128 rows; the rows past the
// block's size are whatever follows in shared memory (their products land in accumulator rows that
// are never read), while every K column past the block's size is zero in both operands.
//
// Warp roles (448 threads): warp 0 TMA producer (tables), warp 1 TMEM allocation and MMA issue,
// warps 2-5 loaders (the Bv operand), warps 6-9 converters (D1 -> B2), warps 10-13 drainers (D2 ->
// B1 rows or FP64 partial sums).  Every mbarrier wait is bounded (the contraction kernel's budget);
// on expiry the CTA raises ERR_TIMEOUT, drains its copies in flight, retires its MMAs, frees its
// tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "symmetry.cuh"
#include "tc_gemm.cuh"

namespace tdscha {
namespace su {

constexpr int THREADS = 448;
constexpr int MAX_SMEM = 220 * 1024;
constexpr unsigned long long DRAIN_NS = 4000000000ull;

__host__ __device__ constexpr int kpad(int d) { return (d + 15) & ~15; }
__host__ __device__ constexpr int dpad(int d) { return (d + 7) & ~7; }

struct Item {
    int b, c, k0, g, ja, jb, fg, pad;
};

// shared-memory layout of one work item (bytes from the 1024-aligned base)
struct Lay {
    int nkb_b, nkb_c, Db, Dc, N1, N2;
    int A1h, A1l, A2h, A2l, slot, Vh, Vl, B2h, B2l, bars, total;
};
__host__ __device__ inline Lay layout_of(int db, int dc, int g) {
    Lay L;
    L.nkb_b = kpad(db) / 16;
    L.nkb_c = kpad(dc) / 16;
    L.Db = dpad(db);
    L.Dc = dpad(dc);
    L.N1 = g * kpad(db);
    L.N2 = g * kpad(dc);
    int off = 0;
    // two slots of the symmetry tables (slot x at + x * slot bytes), so that the next symmetry's
    // tables are copied while this one is computed
    L.A1h = off; off += L.nkb_c * L.Dc * 32;
    L.A1l = off; off += L.nkb_c * L.Dc * 32;
    L.A2h = off; off += L.nkb_b * L.Db * 32;
    L.A2l = off; off += L.nkb_b * L.Db * 32;
    L.slot = off;
    off *= 2;
    L.Vh = off; off += L.nkb_c * L.N1 * 32;
    L.Vl = off; off += L.nkb_c * L.N1 * 32;
    L.B2h = off; off += L.nkb_b * L.N2 * 32;
    L.B2l = off; off += L.nkb_b * L.N2 * 32;
    off += 128 * 32;              // an A operand's 128 rows read past its last region
    L.bars = off; off += 256;
    L.total = off + 1024;         // alignment slack
    return L;
}

struct Params {
    const CUtensorMap *maps;      // 4 per block: given hi, given lo, transposed hi, transposed lo
    const Item *items;
    const int *start, *dim;
    int n, nj, j0, nf_total;
    const double *Ys;             // transform: Ys (nb, n, n)
    void *B1_hi, *B1_lo;          // transform: packed rows (bf16)
    long long Kp;
    const float *Z;               // fold: Z rows (packed pairs), ldz
    long long ldz;
    const double *ups;
    double *partD;                // fold: (nb, nf_total, n, n) partial sums
    unsigned *err;
    unsigned long long wait_ns;
};

// ---- PTX wrappers ------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: true when the phase completed, false on timeout or when another role aborted.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort_flag, unsigned long long budget) {
    unsigned long long t0 = 0;
    for (uint32_t it = 0;; ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 255u) == 255u) {
            if (*abort_flag) return false;
            const unsigned long long t = globaltimer();
            if (t0 == 0) t0 = t;
            else if (t - t0 > budget) return false;
        }
    }
}
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, int c0, int c1, int c2, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}
// Shared-memory descriptor of a K-major operand region with the 32-byte swizzle: rows of 32 bytes,
// 8-row groups 256 bytes apart (stride byte offset), leading byte offset unused (16 B), descriptor
// version 1, layout type 6 (SWIZZLE_32B).
__device__ __forceinline__ uint64_t sw32_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1u << 16;
    d |= (uint64_t)(256u >> 4) << 32;
    d |= (uint64_t)1u << 46;
    d |= (uint64_t)6u << 61;
    return d;
}
// kind::f16 instruction descriptor: f32 accumulator, bf16 A and B, both K-major, N >> 3, M >> 4.
__device__ __forceinline__ uint32_t idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum));
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
// 16 columns of this thread's lane, without waiting (several loads share one tcgen05.wait::ld)
__device__ __forceinline__ void tmem_ld16_nw(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
constexpr int MAXKB = 5;   // K regions of a block of up to 80 modes

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// byte offset of element kk (0..15) of row R inside a 32-byte-swizzled region
__device__ __forceinline__ uint32_t sw32_off(int R, int kk) {
    return (uint32_t)(R * 32 + ((((kk >> 3) ^ ((R >> 2) & 1)) << 4) | ((kk & 7) * 2)));
}
// 8 consecutive K elements (one 16-byte chunk, kk0 = 0 or 8) of row R as bf16 hi and lo
__device__ __forceinline__ void put8(uint8_t *hi_region, uint8_t *lo_region, int R, int kk0, const float (&x)[8]) {
    uint32_t h[4], l[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const __nv_bfloat16 h0 = __float2bfloat16_rn(x[2 * i]), h1 = __float2bfloat16_rn(x[2 * i + 1]);
        const __nv_bfloat16 l0 = __float2bfloat16_rn(x[2 * i] - __bfloat162float(h0));
        const __nv_bfloat16 l1 = __float2bfloat16_rn(x[2 * i + 1] - __bfloat162float(h1));
        h[i] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
        l[i] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
    }
    const uint32_t off = sw32_off(R, kk0);
    *reinterpret_cast<uint4 *>(hi_region + off) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4 *>(lo_region + off) = make_uint4(l[0], l[1], l[2], l[3]);
}
__device__ __forceinline__ long long pair_index(int mu, int nu, int n) {   // mu <= nu
    return (long long)mu * n - ((long long)mu * (mu - 1)) / 2 + (nu - mu);
}

// barrier slots
// barrier slots; A1F..A2E and D1F, D1E come in pairs (slot 0, slot 1)
enum Bar : int { A1F = 0, A1E = 2, A2F = 4, A2E = 6, VF = 8, VE, D1F, D1E = 12, B2F = 14, B2E, D2F, D2E, DONE, NBARS };

template <bool FOLD>
__global__ void __launch_bounds__(THREADS, 1) sym_umma_kernel(const Params p) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *sm = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const Item it = p.items[blockIdx.x];
    const int b = it.b, c = it.c, g = it.g, k0 = it.k0;
    const int sb = p.start[b], db = p.dim[b], sc = p.start[c], dc = p.dim[c];
    const Lay L = layout_of(db, dc, g);
    const int nJ = it.jb - it.ja;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + L.bars);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(bars + NBARS);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + NBARS + 1);
    auto bar = [&](int i) { return smem_u32(&bars[i]); };
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int i = 0; i < NBARS; ++i) {
            const bool by_warps = (i == VF || i == D1E || i == D1E + 1 || i == B2F || i == D2E);
            mbar_init(bar(i), by_warps ? 4u : 1u);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)), "r"(512u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t tmem = *tmem_slot;
    // D1 double buffered when both copies and D2 fit the 512 columns (converters of symmetry j then
    // overlap the first product of j + 1)
    const int nd1 = (2 * L.N1 + L.N2 <= 512) ? 2 : 1;
    const uint32_t D2 = tmem + (uint32_t)(nd1 * L.N1);
    const unsigned long long W = p.wait_ns;

    int issued_a1 = 0, issued_a2 = 0;   // loads handed to TMA (abort drain)
    if (warp == 0 && lane == 0) {
        // ---------------- TMA producer: symmetry tables of blocks c (A1) and b (A2) ----------------
        const int var = FOLD ? 0 : 2;   // fold: tables as given; transform: transposed
        const CUtensorMap *mc_hi = p.maps + 4 * c + var, *mc_lo = mc_hi + 1;
        const CUtensorMap *mb_hi = p.maps + 4 * b + var, *mb_lo = mb_hi + 1;
        const uint32_t bytes_c = 2u * L.nkb_c * L.Dc * 32u, bytes_b = 2u * L.nkb_b * L.Db * 32u;
        for (int i = 0; i < nJ; ++i) {
            const int j = it.ja + i;
            const int x = i & 1;                                   // table slot
            const uint32_t ph = ((uint32_t)(i >> 1) & 1u) ^ 1u;    // its (use - 1) phase
            uint8_t *base = sm + x * L.slot;
            if (!mbar_wait(bar(A1E + x), ph, abort_flag, W)) { *abort_flag = 1; break; }
            mbar_expect_tx(bar(A1F + x), bytes_c);
            for (int s = 0; s < L.nkb_c; ++s) {
                tma_load_3d(smem_u32(base + L.A1h + s * L.Dc * 32), mc_hi, 16 * s, 0, j, bar(A1F + x));
                tma_load_3d(smem_u32(base + L.A1l + s * L.Dc * 32), mc_lo, 16 * s, 0, j, bar(A1F + x));
            }
            issued_a1 = i + 1;
            if (!mbar_wait(bar(A2E + x), ph, abort_flag, W)) { *abort_flag = 1; break; }
            mbar_expect_tx(bar(A2F + x), bytes_b);
            for (int s = 0; s < L.nkb_b; ++s) {
                tma_load_3d(smem_u32(base + L.A2h + s * L.Db * 32), mb_hi, 16 * s, 0, j, bar(A2F + x));
                tma_load_3d(smem_u32(base + L.A2l + s * L.Db * 32), mb_lo, 16 * s, 0, j, bar(A2F + x));
            }
            issued_a2 = i + 1;
        }
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer ----------------
        const uint32_t id1 = idesc_bf16(128, L.N1), id2 = idesc_bf16(128, L.N2);
        const uint32_t a1h0 = smem_u32(sm + L.A1h), a1l0 = smem_u32(sm + L.A1l);
        const uint32_t a2h0 = smem_u32(sm + L.A2h), a2l0 = smem_u32(sm + L.A2l);
        const uint32_t vh = smem_u32(sm + L.Vh), vl = smem_u32(sm + L.Vl);
        const uint32_t b2h = smem_u32(sm + L.B2h), b2l = smem_u32(sm + L.B2l);
        bool ok = true;
        if (!FOLD) ok = mbar_wait(bar(VF), 0u, abort_flag, W);   // the Ys operand, loaded once
        for (int i = 0; i < nJ && ok; ++i) {
            const uint32_t ph = (uint32_t)i & 1u;
            const int x = i & 1;                                    // table slot
            const uint32_t tph = (uint32_t)(i >> 1) & 1u;
            const int xd = i % nd1;                                 // D1 buffer
            const uint32_t dph = (uint32_t)(i / nd1) & 1u;
            const uint32_t D1 = tmem + (uint32_t)(xd * L.N1);
            const uint32_t a1h = a1h0 + x * L.slot, a1l = a1l0 + x * L.slot;
            const uint32_t a2h = a2h0 + x * L.slot, a2l = a2l0 + x * L.slot;
            if (FOLD && !mbar_wait(bar(VF), ph, abort_flag, W)) { ok = false; break; }
            if (!mbar_wait(bar(A1F + x), tph, abort_flag, W) || !mbar_wait(bar(D1E + xd), dph ^ 1u, abort_flag, W)) {
                ok = false;
                break;
            }
            tc_after();
            for (int s = 0; s < L.nkb_c; ++s) {
                const uint32_t ao = s * L.Dc * 32, bo = s * L.N1 * 32;
                umma_bf16(D1, sw32_desc(a1h + ao), sw32_desc(vh + bo), id1, s > 0 ? 1u : 0u);
                umma_bf16(D1, sw32_desc(a1h + ao), sw32_desc(vl + bo), id1, 1u);
                umma_bf16(D1, sw32_desc(a1l + ao), sw32_desc(vh + bo), id1, 1u);
            }
            umma_commit(bar(A1E + x));
            umma_commit(bar(D1F + xd));
            if (FOLD) umma_commit(bar(VE));
            if (!mbar_wait(bar(A2F + x), tph, abort_flag, W) || !mbar_wait(bar(B2F), ph, abort_flag, W)) { ok = false; break; }
            if ((!FOLD || i == 0) && !mbar_wait(bar(D2E), ph ^ 1u, abort_flag, W)) { ok = false; break; }
            tc_after();
            for (int s = 0; s < L.nkb_b; ++s) {
                const uint32_t ao = s * L.Db * 32, bo = s * L.N2 * 32;
                const uint32_t first = (FOLD ? (i > 0 || s > 0) : (s > 0)) ? 1u : 0u;
                umma_bf16(D2, sw32_desc(a2h + ao), sw32_desc(b2h + bo), id2, first);
                umma_bf16(D2, sw32_desc(a2h + ao), sw32_desc(b2l + bo), id2, 1u);
                umma_bf16(D2, sw32_desc(a2l + ao), sw32_desc(b2h + bo), id2, 1u);
            }
            umma_commit(bar(A2E + x));
            umma_commit(bar(B2E));
            if (!FOLD || i == nJ - 1) umma_commit(bar(D2F));
        }
        if (!ok) *abort_flag = 1;
    } else if (warp >= 2 && warp < 6) {
        // ---------------- loaders: the Bv operand (rows (k, mu), K = nu) ----------------
        const int t = threadIdx.x - 64;
        const int Kb = kpad(db), Kc = kpad(dc);
        const int rows = g * Kb, chunks = Kc / 8;
        bool ok = true;
        for (int i = 0; i < (FOLD ? nJ : 1) && ok; ++i) {
            const int j = it.ja + i;
            if (FOLD && !mbar_wait(bar(VE), ((uint32_t)i & 1u) ^ 1u, abort_flag, W)) { ok = false; break; }
            for (int task = t; task < rows * chunks; task += 128) {
                const int R = task / chunks, ch = task - R * chunks;
                const int k = R / Kb, mu = R - k * Kb;
                const int nu0 = 8 * ch;
                float x[8];
                if (mu < db) {
                    if (FOLD) {
                        const long long r = (long long)(k0 + k) * p.nj + (j - p.j0);
                        const float *Zr = p.Z + r * p.ldz;
                        const int gm = sb + mu;
#pragma unroll
                        for (int e = 0; e < 8; ++e) {
                            const int nu = nu0 + e;
                            float v = 0.f;
                            if (nu < dc) {
                                const int gn = sc + nu;
                                const long long pi = gm <= gn ? pair_index(gm, gn, p.n) : pair_index(gn, gm, p.n);
                                v = (float)((gm == gn ? 2.0 : 1.0) * p.ups[gm] * p.ups[gn]) * Zr[pi];
                            }
                            x[e] = v;
                        }
                    } else {
                        const double *Yr = p.Ys + ((long long)(k0 + k) * p.n + sb + mu) * p.n + sc;
#pragma unroll
                        for (int e = 0; e < 8; ++e) x[e] = (nu0 + e < dc) ? (float)Yr[nu0 + e] : 0.f;
                    }
                } else {
#pragma unroll
                    for (int e = 0; e < 8; ++e) x[e] = 0.f;
                }
                const int s = nu0 >> 4;
                put8(sm + L.Vh + s * L.N1 * 32, sm + L.Vl + s * L.N1 * 32, R, nu0 & 15, x);
            }
            fence_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(bar(VF));
        }
        if (!ok) *abort_flag = 1;
    } else if (warp >= 6 && warp < 10) {
        // ---------------- converters: D1 row nu' -> B2 rows (k, nu'), K = mu ----------------
        const int q = warp & 3;
        const int nup = q * 32 + lane;
        const int Kb = kpad(db), Kc = kpad(dc);
        bool ok = true;
        for (int i = 0; i < nJ && ok; ++i) {
            const uint32_t ph = (uint32_t)i & 1u;
            const int xd = i % nd1;
            const uint32_t dph = (uint32_t)(i / nd1) & 1u;
            const uint32_t D1 = tmem + (uint32_t)(xd * L.N1);
            if (!mbar_wait(bar(D1F + xd), dph, abort_flag, W) || !mbar_wait(bar(B2E), ph ^ 1u, abort_flag, W)) {
                ok = false;
                break;
            }
            tc_after();
            for (int k = 0; k < g; ++k) {
                uint32_t r[MAXKB][16];
#pragma unroll
                for (int s = 0; s < MAXKB; ++s)
                    if (s < L.nkb_b) tmem_ld16_nw(D1 + ((uint32_t)(q * 32) << 16) + (uint32_t)(k * Kb + 16 * s), r[s]);
                tmem_wait_ld();
                if (nup < dc) {
                    const int R = k * Kc + nup;
#pragma unroll
                    for (int s = 0; s < MAXKB; ++s) {
                        if (s >= L.nkb_b) break;
                        float x0[8], x1[8];
#pragma unroll
                        for (int e = 0; e < 8; ++e) {
                            x0[e] = (16 * s + e < db) ? __uint_as_float(r[s][e]) : 0.f;
                            x1[e] = (16 * s + 8 + e < db) ? __uint_as_float(r[s][8 + e]) : 0.f;
                        }
                        put8(sm + L.B2h + s * L.N2 * 32, sm + L.B2l + s * L.N2 * 32, R, 0, x0);
                        put8(sm + L.B2h + s * L.N2 * 32, sm + L.B2l + s * L.N2 * 32, R, 8, x1);
                    }
                }
            }
            fence_async_smem();
            tc_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(bar(B2F));
                mbar_arrive(bar(D1E + xd));
            }
        }
        if (!ok) *abort_flag = 1;
    } else if (warp >= 10) {
        // ---------------- drainers: D2 row mu' ----------------
        const int q = warp & 3;
        const int mup = q * 32 + lane;
        const int Kc = kpad(dc);
        bool ok = true;
        for (int i = (FOLD ? nJ - 1 : 0); i < nJ && ok; ++i) {
            const int j = it.ja + i;
            if (!mbar_wait(bar(D2F), FOLD ? 0u : ((uint32_t)i & 1u), abort_flag, W)) { ok = false; break; }
            tc_after();
            for (int k = 0; k < g; ++k) {
                uint32_t rr[MAXKB][16];
#pragma unroll
                for (int s = 0; s < MAXKB; ++s)
                    if (s < L.nkb_c) tmem_ld16_nw(D2 + ((uint32_t)(q * 32) << 16) + (uint32_t)(k * Kc + 16 * s), rr[s]);
                tmem_wait_ld();
#pragma unroll
                for (int s = 0; s < MAXKB; ++s) {
                    if (s >= L.nkb_c) break;
                    float v[16];
#pragma unroll
                    for (int e = 0; e < 16; ++e) v[e] = __uint_as_float(rr[s][e]);
                    if (mup >= db) continue;
                    const int gm = sb + mup;
                    if (FOLD) {
                        double *out = p.partD + ((long long)(k0 + k) * p.nf_total + it.fg) * (long long)p.n * p.n +
                                      (long long)gm * p.n + sc;
#pragma unroll
                        for (int e = 0; e < 16; ++e)
                            if (16 * s + e < dc) out[16 * s + e] = (double)v[e];
                    } else {
                        const long long r = (long long)(k0 + k) * p.nj + (j - p.j0);
                        const long long row = r * p.Kp + pair_index(gm, gm, p.n) - gm;   // + gn = pair(gm, gn)
                        __nv_bfloat16 *hi = static_cast<__nv_bfloat16 *>(p.B1_hi);
                        __nv_bfloat16 *lo = static_cast<__nv_bfloat16 *>(p.B1_lo);
#pragma unroll
                        for (int e = 0; e < 16; ++e) {
                            const int nu = 16 * s + e, gn = sc + nu;
                            if (nu < dc && gm <= gn) {
                                const __nv_bfloat16 h = __float2bfloat16_rn(v[e]);
                                hi[row + gn] = h;
                                if (lo) lo[row + gn] = __float2bfloat16_rn(v[e] - __bfloat162float(h));
                            }
                        }
                    }
                }
            }
            tc_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(bar(D2E));
        }
        if (!ok) *abort_flag = 1;
    }

    // ---------------- teardown ----------------
    tc_before();
    __syncthreads();
    if (*abort_flag) {
        if (threadIdx.x == 0) atomicOr(p.err, ERR_TIMEOUT);
        volatile int never = 0;
        if (warp == 0 && lane == 0) {
            // the last two loads of each table (one per slot) can still be in flight
            for (int i = std::max(0, issued_a1 - 2); i < issued_a1; ++i)
                mbar_wait(bar(A1F + (i & 1)), (uint32_t)(i >> 1) & 1u, &never, DRAIN_NS);
            for (int i = std::max(0, issued_a2 - 2); i < issued_a2; ++i)
                mbar_wait(bar(A2F + (i & 1)), (uint32_t)(i >> 1) & 1u, &never, DRAIN_NS);
        }
        if (warp == 1 && lane == 0) {
            umma_commit(bar(DONE));
            mbar_wait(bar(DONE), 0u, &never, DRAIN_NS);
        }
        __syncthreads();
    }
    if (warp == 1) {
        tc_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
    }
}

// ---- vector parts on the CUDA cores (FP64) ----------------------------------------------------------
// r1[r, mu] = ups_mu (S_j^T R1_k)_mu for the rows r = k * nj + (j - j0) of this call
__global__ void r1_kernel(const double *__restrict__ sym, const long long *__restrict__ off, const int *__restrict__ start,
                          const int *__restrict__ dim, const int *__restrict__ bid, int n, int nb, int nj, int j0,
                          const double *__restrict__ R1, const double *__restrict__ ups, long long np, Format fmt, void *r1_hi,
                          void *r1_lo) {
    const long long total = (long long)nb * nj * n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
        const int mu = (int)(idx % n);
        const long long rr = idx / n;          // = k * nj + jj
        const int k = (int)(rr / nj), jj = (int)(rr % nj);
        const int bb = bid[mu], s0 = start[bb], d = dim[bb], i = mu - s0;
        const double *S = sym + off[bb] + (long long)(j0 + jj) * d * d;
        const double *R = R1 + (long long)k * n + s0;
        double acc = 0.0;
        for (int q = 0; q < d; ++q) acc += S[q * d + i] * R[q];
        store_split(fmt, r1_hi, r1_lo, rr * np + mu, ups[mu] * acc);
    }
}

// partF[(k, fg), mu] = sum_{j in fold chunk fg} (S_j F_r)_mu
__global__ void partF_kernel(const double *__restrict__ sym, const long long *__restrict__ off, const int *__restrict__ start,
                             const int *__restrict__ dim, const int *__restrict__ bid, int n, int nb, int nj, int j0, int Jf,
                             int nf_total, const float *__restrict__ F, long long ldf, double *__restrict__ partF) {
    const int nfc = (nj + Jf - 1) / Jf;
    const long long total = (long long)nb * nfc * n;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
        const int mu = (int)(idx % n);
        const long long rest = idx / n;
        const int fc = (int)(rest % nfc), k = (int)(rest / nfc);
        const int bb = bid[mu], s0 = start[bb], d = dim[bb], i = mu - s0;
        const int ja = j0 + fc * Jf, jb = min(j0 + (fc + 1) * Jf, j0 + nj);
        double acc = 0.0;
        for (int j = ja; j < jb; ++j) {
            const double *S = sym + off[bb] + (long long)j * d * d + (long long)i * d;
            const float *Fr = F + ((long long)k * nj + (j - j0)) * ldf + s0;
            for (int q = 0; q < d; ++q) acc += S[q] * (double)Fr[q];
        }
        partF[((long long)k * nf_total + (j0 / Jf + fc)) * n + mu] = acc;
    }
}

// bf16 hi / lo tables of block b, zero padded to (N_sym, Dpad, Kpad): as given (trans = 0) or transposed
__global__ void table_kernel(const double *__restrict__ S, int N_sym, int d, int Dp, int Kq, int trans, __nv_bfloat16 *hi,
                             __nv_bfloat16 *lo) {
    const long long total = (long long)N_sym * Dp * Kq;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(idx % Kq);
        const long long rest = idx / Kq;
        const int r = (int)(rest % Dp);
        const long long j = rest / Dp;
        double v = 0.0;
        if (r < d && q < d) v = trans ? S[j * d * d + (long long)q * d + r] : S[j * d * d + (long long)r * d + q];
        const __nv_bfloat16 h = __float2bfloat16_rn((float)v);
        hi[idx] = h;
        lo[idx] = __float2bfloat16_rn((float)(v - (double)__bfloat162float(h)));
    }
}

}  // namespace su

// ---- host side --------------------------------------------------------------------------------------
struct SymUmma {
    int device = 0, N_sym = 0, n_blocks = 0;
    std::vector<int> dim;
    void *tables = nullptr;           // all bf16 tables
    CUtensorMap *d_maps = nullptr;    // 4 per block
    std::mutex mu;
    std::map<std::tuple<int, int, int, int, int>, std::pair<su::Item *, int>> items;   // (fold, nb, nj, j0, Jf)
    std::map<std::tuple<int, int, int, int, int>, int> smem;
};

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

int sym_umma_create(const SymTables &t, int N_sym, const std::vector<int> &dim, const std::vector<long long> &sym_off,
                    SymUmma **out) {
    *out = nullptr;
    for (int d : dim) TD_CHECK(d <= 80, TDSCHA_EINVAL, "tensor-core symmetry kernels: block of %d modes (max 80)", d);
    EncodeTiledFn enc = encode_fn();
    TD_CHECK(enc != nullptr, TDSCHA_ECUDA, "cuTensorMapEncodeTiled entry point unavailable");
    SymUmma *u = new SymUmma();
    TD_CUDA(cudaGetDevice(&u->device));
    u->N_sym = N_sym;
    u->n_blocks = (int)dim.size();
    u->dim = dim;
    std::vector<size_t> off(dim.size());
    size_t total = 0;
    for (size_t b = 0; b < dim.size(); ++b) {
        off[b] = total;
        total += 4 * (size_t)N_sym * su::dpad(dim[b]) * su::kpad(dim[b]) * sizeof(__nv_bfloat16);
        total = (total + 255) / 256 * 256;
    }
    cudaError_t ce = cudaMalloc(&u->tables, total);
    if (ce != cudaSuccess) { delete u; TD_CHECK(false, TDSCHA_ENOMEM, "tensor-core symmetry tables: %s", cudaGetErrorString(ce)); }
    ce = cudaMalloc(&u->d_maps, 4 * dim.size() * sizeof(CUtensorMap));
    if (ce != cudaSuccess) { cudaFree(u->tables); delete u; TD_CHECK(false, TDSCHA_ENOMEM, "tensor maps: %s", cudaGetErrorString(ce)); }
    std::vector<CUtensorMap> maps(4 * dim.size());
    for (size_t b = 0; b < dim.size(); ++b) {
        const int d = dim[b], Dp = su::dpad(d), Kq = su::kpad(d);
        const size_t one = (size_t)N_sym * Dp * Kq;
        __nv_bfloat16 *base = reinterpret_cast<__nv_bfloat16 *>(static_cast<uint8_t *>(u->tables) + off[b]);
        for (int tr = 0; tr < 2; ++tr) {
            __nv_bfloat16 *hi = base + (2 * tr) * one, *lo = base + (2 * tr + 1) * one;
            const int grid = (int)std::min<size_t>((one + 255) / 256, 148 * 64);
            su::table_kernel<<<grid, 256>>>(t.sym + sym_off[b], N_sym, d, Dp, Kq, tr, hi, lo);
            for (int part = 0; part < 2; ++part) {
                cuuint64_t gdim[3] = {(cuuint64_t)Kq, (cuuint64_t)Dp, (cuuint64_t)N_sym};
                cuuint64_t gstride[2] = {(cuuint64_t)Kq * 2, (cuuint64_t)Dp * Kq * 2};
                cuuint32_t box[3] = {16, (cuuint32_t)Dp, 1};
                cuuint32_t es[3] = {1, 1, 1};
                CUresult r = enc(&maps[4 * b + 2 * tr + part], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, part ? lo : hi, gdim,
                                 gstride, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
                if (r != CUDA_SUCCESS) {
                    cudaFree(u->tables);
                    cudaFree(u->d_maps);
                    delete u;
                    TD_CHECK(false, TDSCHA_ECUDA, "cuTensorMapEncodeTiled (symmetry tables) failed (%d)", (int)r);
                }
            }
        }
    }
    TD_CUDA(cudaGetLastError());
    TD_CUDA(cudaMemcpy(u->d_maps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
    TD_CUDA(cudaDeviceSynchronize());
    *out = u;
    return 0;
}

void sym_umma_destroy(SymUmma *u) {
    if (!u) return;
    if (u->tables) cudaFree(u->tables);
    if (u->d_maps) cudaFree(u->d_maps);
    for (auto &kv : u->items) cudaFree(kv.second.first);
    delete u;
}

// vectors per work item of a block pair: the accumulators (g x Kpad columns each) fit 256 TMEM
// columns and the operands fit the shared memory
static int group_of(int db, int dc, int nb) {
    int g = std::max(1, std::min(nb, 256 / std::max(su::kpad(db), su::kpad(dc))));
    while (g > 1 && su::layout_of(db, dc, g).total > su::MAX_SMEM) --g;
    return g;
}

// Work items of one call (cached; built outside any stream capture by the eager calls that precede it)
static int get_items(SymUmma *u, const SymTables &t, bool fold, int nb, int nj, int j0, int Jf, cudaStream_t st,
                     su::Item **items, int *count, int *smem) {
    const auto key = std::make_tuple(fold ? 1 : 0, nb, nj, j0, fold ? Jf : 0);
    std::lock_guard<std::mutex> lock(u->mu);
    auto itx = u->items.find(key);
    if (itx != u->items.end()) {
        *items = itx->second.first;
        *count = itx->second.second;
        *smem = u->smem[key];
        return 0;
    }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    TD_CUDA(cudaStreamIsCapturing(st, &cap));
    TD_CHECK(cap == cudaStreamCaptureStatusNone, TDSCHA_EINVAL,
             "tensor-core symmetry kernels: first call for this batch is being captured (make an eager call first)");
    const int nbk = u->n_blocks;
    std::vector<su::Item> v;
    int smax = 0;
    // cost of one symmetry of one item ~ fixed pipeline latency + the work of its products
    std::vector<std::tuple<int, int, int, int, double>> groups;   // b, c, k0, g, cost per symmetry
    double total = 0;
    for (int b = 0; b < nbk; ++b)
        for (int c = b; c < nbk; ++c) {
            const int db = u->dim[b], dc = u->dim[c];
            const int g = group_of(db, dc, nb);
            smax = std::max(smax, su::layout_of(db, dc, g).total);
            for (int k0 = 0; k0 < nb; k0 += g) {
                const int gk = std::min(g, nb - k0);
                const double cost = 1.0 + (double)gk * db * dc * (db + dc) / 2.0e5;
                groups.emplace_back(b, c, k0, gk, cost);
                total += cost * nj;
            }
        }
    if (fold) {
        const int nfc = (nj + Jf - 1) / Jf;
        for (auto &gr : groups)
            for (int fc = 0; fc < nfc; ++fc) {
                su::Item x{std::get<0>(gr), std::get<1>(gr), std::get<2>(gr), std::get<3>(gr), j0 + fc * Jf,
                           std::min(j0 + (fc + 1) * Jf, j0 + nj), j0 / Jf + fc, 0};
                v.push_back(x);
            }
    } else {
        const double target = std::max(1.0, total / (4.0 * 148));
        for (auto &gr : groups) {
            const int chunks = std::max(1, std::min(nj, (int)(std::get<4>(gr) * nj / target + 0.5)));
            for (int q = 0; q < chunks; ++q) {
                const int ja = j0 + (int)((long long)nj * q / chunks), jb = j0 + (int)((long long)nj * (q + 1) / chunks);
                if (jb > ja) v.push_back(su::Item{std::get<0>(gr), std::get<1>(gr), std::get<2>(gr), std::get<3>(gr), ja, jb, 0, 0});
            }
        }
    }
    // heaviest items first, so that the tail of the grid is made of short ones
    std::stable_sort(v.begin(), v.end(), [&](const su::Item &x, const su::Item &y) {
        auto w = [&](const su::Item &z) { return (double)(z.jb - z.ja) * (1.0 + (double)z.g * u->dim[z.b] * u->dim[z.c] *
                                                                              (u->dim[z.b] + u->dim[z.c]) / 2.0e5); };
        return w(x) > w(y);
    });
    su::Item *d = nullptr;
    TD_CUDA(cudaMalloc(&d, v.size() * sizeof(su::Item)));
    TD_CUDA(cudaMemcpy(d, v.data(), v.size() * sizeof(su::Item), cudaMemcpyHostToDevice));
    u->items[key] = {d, (int)v.size()};
    u->smem[key] = smax;
    *items = d;
    *count = (int)v.size();
    *smem = smax;
    (void)t;
    return 0;
}

template <bool FOLD>
static int launch_umma(const su::Params &prm, int count, int smem, cudaStream_t st) {
    // at least ~half of the shared memory per CTA: one CTA per SM, so that no two CTAs wait on each
    // other's tensor-memory columns
    smem = std::max(smem, 116 * 1024);
    auto kern = su::sym_umma_kernel<FOLD>;
    TD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    kern<<<count, su::THREADS, smem, st>>>(prm);
    TD_CUDA(cudaGetLastError());
    return 0;
}

int sym_transform_umma(SymUmma *u, const SymTables &t, const int *blocks_ids, int nb, int nj, int j0, const double *Ys,
                       const double *R1, const double *ups, long long Kp, long long np, Format fmt, void *B1_hi, void *B1_lo,
                       void *r1_hi, void *r1_lo, unsigned *err, cudaStream_t st) {
    TD_CHECK(u && fmt == FMT_BF16, TDSCHA_EINVAL, "tensor-core symmetry transform: bf16 storage only");
    su::Item *items = nullptr;
    int count = 0, smem = 0;
    TD_TRY(get_items(u, t, false, nb, nj, j0, 0, st, &items, &count, &smem));
    su::Params prm{};
    prm.maps = u->d_maps;
    prm.items = items;
    prm.start = t.start;
    prm.dim = t.dim;
    prm.n = t.n;
    prm.nj = nj;
    prm.j0 = j0;
    prm.Ys = Ys;
    prm.B1_hi = B1_hi;
    prm.B1_lo = B1_lo;
    prm.Kp = Kp;
    prm.ups = ups;
    prm.err = err;
    prm.wait_ns = tc::wait_budget_ns();
    TD_TRY(launch_umma<false>(prm, count, smem, st));
    const long long total = (long long)nb * nj * t.n;
    su::r1_kernel<<<(int)std::min<long long>((total + 255) / 256, 148 * 32), 256, 0, st>>>(
        t.sym, t.off, t.start, t.dim, blocks_ids, t.n, nb, nj, j0, R1, ups, np, fmt, r1_hi, r1_lo);
    TD_CUDA(cudaGetLastError());
    return 0;
}

int sym_fold_umma(SymUmma *u, const SymTables &t, const int *blocks_ids, int nb, int nj, int j0, int Jf, int nf_total,
                  const float *Z, long long ldz, const float *F, long long ldf, const double *ups, double *partD,
                  double *partF, unsigned *err, cudaStream_t st) {
    TD_CHECK(u != nullptr, TDSCHA_EINVAL, "tensor-core symmetry fold: tables not built");
    TD_CHECK(j0 % Jf == 0, TDSCHA_EINVAL, "symmetry chunk start %d not a multiple of the fold chunk %d", j0, Jf);
    su::Item *items = nullptr;
    int count = 0, smem = 0;
    TD_TRY(get_items(u, t, true, nb, nj, j0, Jf, st, &items, &count, &smem));
    su::Params prm{};
    prm.maps = u->d_maps;
    prm.items = items;
    prm.start = t.start;
    prm.dim = t.dim;
    prm.n = t.n;
    prm.nj = nj;
    prm.j0 = j0;
    prm.nf_total = nf_total;
    prm.Z = Z;
    prm.ldz = ldz;
    prm.ups = ups;
    prm.partD = partD;
    prm.err = err;
    prm.wait_ns = tc::wait_budget_ns();
    TD_TRY(launch_umma<true>(prm, count, smem, st));
    const int nfc = (nj + Jf - 1) / Jf;
    const long long total = (long long)nb * nfc * t.n;
    su::partF_kernel<<<(int)std::min<long long>((total + 255) / 256, 148 * 32), 256, 0, st>>>(
        t.sym, t.off, t.start, t.dim, blocks_ids, t.n, nb, nj, j0, Jf, nf_total, F, ldf, partF);
    TD_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace tdscha
