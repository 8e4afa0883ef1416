// tc_gemm.cu -- hand-written sm_100a tensor-core contraction D = A . B^T for the ensemble averages.
//
//   A (M x K), B (N x K): row-major, K contiguous ("K-major" for both UMMA operands), stored as
//   bf16 or tf32-rounded fp32; optionally as hi/lo splits so that three products
//   hi.hi + hi.lo + lo.hi recover ~16 (bf16) / ~21 (tf32) significant bits.
//   D (M x N): fp32, row-major, written with edge masking.
//
// Pipeline (persistent: one CTA per SM walks 128 x BN output tiles; BN = 256, 128 or 64; 10 warps):
//   warp 0      : TMA producer -- cp.async.bulk.tensor.2d into a STAGES-deep ring of 128B-swizzled
//                 tiles, completion tracked by mbarrier transaction counts;
//   warp 1      : allocates 2 x BN TMEM columns (two accumulator buffers); one elected thread issues
//                 tcgen05.mma (kind::f16 for bf16, kind::tf32) from shared-memory descriptors,
//                 accumulating in TMEM, and frees each ring slot with tcgen05.commit -> mbarrier;
//   warps 2..9  : epilogue -- tcgen05.ld 32x32b from TMEM (warp w reads lanes 32*(w%4)..+31, half of
//                 the columns), fp32 sums in registers, stores to global memory through a per-warp
//                 shared-memory block (full 128-byte lines per store instruction).
// Every mbarrier wait is bounded by a %globaltimer budget; on expiry the CTA raises ERR_TIMEOUT in
// the caller's error word, drains its own TMA copies (bounded), frees TMEM and returns.
#include <cuda.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <map>
#include <mutex>
#include <tuple>
#include <utility>
#include <vector>

#include "common.cuh"
#include "tc_gemm.cuh"

namespace tdscha {
namespace tc {

constexpr int BM = 128;
constexpr int NUM_THREADS = 320;   // producer, MMA, 8 epilogue warps
constexpr unsigned long long DEFAULT_WAIT_BUDGET_NS = 4000000000ull;   // 4 s per pipeline wait
constexpr unsigned long long DRAIN_BUDGET_NS = 4000000000ull;          // 4 s per wait of the abort path

// Budget of every pipeline wait of the next launches (tdscha_set_wait_budget), and a one-shot request
// that the next launch's producers issue no copy, so that the MMA warps' first wait can only end by
// running out (tdscha_debug_stall_next_contraction: a test of the abort path).
static std::atomic<unsigned long long> g_wait_budget_ns{DEFAULT_WAIT_BUDGET_NS};
static std::atomic<int> g_stall_next{0};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
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
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort_flag,
                                          unsigned long long budget_ns) {
    unsigned long long t0 = 0;
    for (uint32_t it = 0;; ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 255u) == 255u) {
            if (*abort_flag) return false;
            unsigned long long t = globaltimer();
            if (t0 == 0) t0 = t;
            else if (t - t0 > budget_ns) return false;
        }
    }
}

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Loose alignment of the CTAs' tile starts.  Each producer counts its tile starts in a global
// counter; before loading its i-th tile it waits (at most `budget_ns`, then goes on regardless)
// until every CTA that has an i-th tile has started it.  CTAs then walk the K range of concurrent
// tiles together and the A / B panels they share are read from HBM once and hit in L2 afterwards;
// without it they drift apart over the long K loops and most panel reads miss.  Purely a
// performance hint: results never depend on it.
__device__ __forceinline__ void tile_start_sync(unsigned *counter, unsigned target, unsigned long long budget_ns) {
    atomicAdd(counter, 1u);
    if (budget_ns == 0) return;
    const unsigned long long t0 = globaltimer();
    while (ld_acquire_gpu(counter) < target) {
        if (globaltimer() - t0 > budget_ns) break;
        __nanosleep(128);
    }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int c0, int c1, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(bar)
        : "memory");
}

// Shared-memory matrix descriptor of a K-major tile stored as rows of 128 bytes with the 128-byte
// swizzle (what TMA writes with CU_TENSOR_MAP_SWIZZLE_128B): start address >> 4 in bits 0-13,
// leading byte offset (unused for swizzled K-major, 16 B) in bits 16-29, stride byte offset = 1024
// (one 8-row swizzle atom) in bits 32-45, descriptor version 1 in bits 46-47, swizzle mode 2
// (128B) in bits 61-63.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)(16u >> 4) << 16;
    d |= (uint64_t)(1024u >> 4) << 32;
    d |= (uint64_t)1u << 46;
    d |= (uint64_t)2u << 61;
    return d;
}

// Instruction descriptor for kind::f16 / kind::tf32 with fp32 accumulation, both operands K-major:
// D format (bits 4-5) = 1 (f32); A/B format (bits 7-9, 10-12) = 1 (bf16) or 2 (tf32);
// N >> 3 in bits 17-22; M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t make_idesc(bool tf32, int m, int n) {
    return (1u << 4) | ((tf32 ? 2u : 1u) << 7) | ((tf32 ? 2u : 1u) << 10) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

template <bool TF32>
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accum) {
    if constexpr (TF32) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
            ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum));
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
            ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum));
    }
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Sub-problems of one launch (a single contraction is one group): tile0 = tiles of the groups before.
constexpr int MAX_GROUPS = 64;
struct DevGroup {
    int M, N, K, a_row, a_k, b_row, b_k, tile0, num_m, num_n;
    long long d_off;
};
struct GroupTable {
    int n, total_tiles;
    DevGroup g[MAX_GROUPS];
};

__device__ __forceinline__ const DevGroup &group_of(const GroupTable &gt, int t) {
    int g = 0;
    while (g + 1 < gt.n && gt.g[g + 1].tile0 <= t) ++g;
    return gt.g[g];
}

// Tile order of the persistent schedule: groups of `gm` M-tiles, N-tiles of a group in turn, M
// fastest inside a group.  The ~148 tiles in flight then form a gm x (148/gm) block that shares its
// A rows and B rows through L2, instead of one N column of tiles streaming all of A from HBM.
__device__ __forceinline__ void tile_coords(int t, int num_m, int num_n, int gm, int &m_blk, int &n_blk) {
    const int per_group = gm * num_n;
    const int g = t / per_group, rem = t % per_group;
    const int m_first = g * gm;
    const int rows = min(gm, num_m - m_first);
    n_blk = rem / rows;
    m_blk = m_first + rem % rows;
}

template <int BN, int STAGES, bool TF32, int NPROD>
struct Cfg {
    static constexpr int A_BYTES = BM * 128;                 // one 128 x (128 B) tile
    static constexpr int B_BYTES = BN * 128;
    static constexpr int NOPS = (NPROD == 3) ? 2 : 1;        // hi (+ lo)
    static constexpr int STAGE_BYTES = NOPS * (A_BYTES + B_BYTES);
    static constexpr int K_ELEMS = TF32 ? 32 : 64;            // K per stage (128 B of K)
    static constexpr int UMMA_K = TF32 ? 8 : 16;              // K per instruction (32 B)
    static constexpr uint32_t TMEM_COLS = 2 * BN;             // two accumulator buffers
    static constexpr int EPI_WARPS = 8;                       // 2 warps per TMEM lane quadrant
    static constexpr int EPI_COLS = BN / 2;                   // columns owned by one epilogue thread
    static constexpr int EPI_BUF_FLOATS = 32 * 32;            // one epilogue warp's 32 x 32 staging block
    static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/ +
                                      EPI_WARPS * EPI_BUF_FLOATS * 4 /*epilogue staging*/;
    static_assert(SMEM_BYTES <= 227 * 1024, "shared memory of the contraction kernel");
};

// Persistent: CTA c processes tiles c, c + gridDim.x, ... (m fastest).  Each tile's K loop is split
// into chunks of `drain` k-blocks; a chunk accumulates from zero in one of two TMEM buffers (the MMA
// warp moves on to the other buffer) and the epilogue warps add it into round-to-nearest fp32
// registers, which bounds the error of the tensor core's own fp32 accumulation to `drain` k-blocks.
template <int BN, int STAGES, bool TF32, int NPROD>
__global__ void __launch_bounds__(NUM_THREADS, 1)
tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA_hi, const __grid_constant__ CUtensorMap tmA_lo,
               const __grid_constant__ CUtensorMap tmB_hi, const __grid_constant__ CUtensorMap tmB_lo,
               const __grid_constant__ GroupTable gt, int drain, int group_m, float *__restrict__ D, long long ldd, unsigned *err,
               unsigned *tile_sync, unsigned sync_ns, int accumulate, unsigned long long wait_ns, int stall) {
    using C = Cfg<BN, STAGES, TF32, NPROD>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + STAGES * C::STAGE_BYTES);
    // bars[0..S) full, [S..2S) empty, [2S, 2S+2) accumulator full, [2S+2, 2S+4) accumulator empty
    uint64_t *acc_full = bars + 2 * STAGES;
    uint64_t *acc_empty = bars + 2 * STAGES + 2;
    volatile int *abort_flag = reinterpret_cast<volatile int *>(bars + 2 * STAGES + 4);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * STAGES + 5);
    uint64_t *done_bar = bars + 2 * STAGES + 6;   // abort path: completion of every MMA issued
    float *epi_buf = reinterpret_cast<float *>(smem + STAGES * C::STAGE_BYTES + 256);   // epilogue staging blocks

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int num_tiles = gt.total_tiles;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(smem_u32(&bars[s]), 1);
            mbar_init(smem_u32(&bars[STAGES + s]), 1);
        }
        for (int x = 0; x < 2; ++x) {
            mbar_init(smem_u32(&acc_full[x]), 1);
            mbar_init(smem_u32(&acc_empty[x]), C::EPI_WARPS);
        }
        mbar_init(smem_u32(done_bar), 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tmem_slot)), "r"(C::TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem_base = *tmem_slot;

    long long issued = 0;   // k-blocks handed to TMA by the producer (for the drain on abort)
    if (warp == 0 && lane == 0 && !stall) {
        // ---------------- TMA producer ----------------
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmA_hi)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmB_hi)) : "memory");
        long long g = 0;
        unsigned target = 0;   // tile starts of all CTAs up to and including this round
        for (int t = blockIdx.x, round = 0; t < num_tiles && !*abort_flag; t += gridDim.x, ++round) {
            target += (unsigned)min((int)gridDim.x, num_tiles - round * (int)gridDim.x);
            if (tile_sync) tile_start_sync(tile_sync, target, round > 0 ? sync_ns : 0ull);
            const DevGroup &G = group_of(gt, t);
            int mb, nbk;
            tile_coords(t - G.tile0, G.num_m, G.num_n, group_m, mb, nbk);
            const int m0 = G.a_row + mb * BM, n0 = G.b_row + nbk * BN;
            const int num_kb = G.K / C::K_ELEMS;
            for (int kb = 0; kb < num_kb; ++kb, ++g) {
                const int s = (int)(g % STAGES);
                const uint32_t ph = (uint32_t)(g / STAGES) & 1u;
                if (!mbar_wait(smem_u32(&bars[STAGES + s]), ph ^ 1u, abort_flag, wait_ns)) { *abort_flag = 1; break; }
                uint8_t *st = smem + s * C::STAGE_BYTES;
                const uint32_t full = smem_u32(&bars[s]);
                mbar_expect_tx(full, C::STAGE_BYTES);
                const int kc = kb * C::K_ELEMS;
                tma_load_2d(smem_u32(st), &tmA_hi, G.a_k + kc, m0, full);
                tma_load_2d(smem_u32(st + C::NOPS * C::A_BYTES), &tmB_hi, G.b_k + kc, n0, full);
                if constexpr (NPROD == 3) {
                    tma_load_2d(smem_u32(st + C::A_BYTES), &tmA_lo, G.a_k + kc, m0, full);
                    tma_load_2d(smem_u32(st + C::NOPS * C::A_BYTES + C::B_BYTES), &tmB_lo, G.b_k + kc, n0, full);
                }
                issued = g + 1;
            }
        }
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer ----------------
        constexpr uint32_t idesc = make_idesc(TF32, BM, BN);
        long long g = 0, ch = 0;
        bool ok = true;
        for (int t = blockIdx.x; t < num_tiles && ok; t += gridDim.x) {
            const int num_kb = group_of(gt, t).K / C::K_ELEMS;
            const int chunks_per_tile = (num_kb + drain - 1) / drain;
            for (int c = 0; c < chunks_per_tile && ok; ++c, ++ch) {
                const int X = (int)(ch & 1);
                const uint32_t use = (uint32_t)(ch >> 1);
                if (!mbar_wait(smem_u32(&acc_empty[X]), (use & 1u) ^ 1u, abort_flag, wait_ns)) { ok = false; break; }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t dtm = tmem_base + (uint32_t)(X * BN);
                const int kb_end = min(num_kb, (c + 1) * drain);
                for (int kb = c * drain; kb < kb_end; ++kb, ++g) {
                    const int s = (int)(g % STAGES);
                    const uint32_t ph = (uint32_t)(g / STAGES) & 1u;
                    if (!mbar_wait(smem_u32(&bars[s]), ph, abort_flag, wait_ns)) { ok = false; break; }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    uint8_t *st = smem + s * C::STAGE_BYTES;
                    const uint32_t a_hi = smem_u32(st);
                    const uint32_t b_hi = smem_u32(st + C::NOPS * C::A_BYTES);
#pragma unroll
                    for (int k = 0; k < C::K_ELEMS / C::UMMA_K; ++k) {
                        const uint32_t koff = k * 32;   // bytes inside the 128-byte swizzled row
                        const uint32_t acc = (kb > c * drain || k > 0) ? 1u : 0u;
                        umma<TF32>(dtm, sw128_desc(a_hi + koff), sw128_desc(b_hi + koff), idesc, acc);
                        if constexpr (NPROD == 3) {
                            const uint32_t a_lo = smem_u32(st + C::A_BYTES);
                            const uint32_t b_lo = smem_u32(st + C::NOPS * C::A_BYTES + C::B_BYTES);
                            umma<TF32>(dtm, sw128_desc(a_hi + koff), sw128_desc(b_lo + koff), idesc, 1u);
                            umma<TF32>(dtm, sw128_desc(a_lo + koff), sw128_desc(b_hi + koff), idesc, 1u);
                        }
                    }
                    umma_commit(smem_u32(&bars[STAGES + s]));   // slot s free once these MMAs retire
                }
                if (!ok) break;
                umma_commit(smem_u32(&acc_full[X]));             // chunk accumulated in buffer X
            }
        }
        if (!ok) *abort_flag = 1;
    } else if (warp >= 2) {
        // ---------------- epilogue: drain chunks into fp32 registers, store each tile ----------------
        const int ew = warp - 2;
        const int q = warp & 3;              // TMEM lane quadrant this warp may access
        const int half = ew >> 2;            // which half of the BN columns this warp owns
        long long ch = 0;
        bool ok = true;
        for (int t = blockIdx.x; t < num_tiles && ok; t += gridDim.x) {
            const DevGroup &G = group_of(gt, t);
            int mb, nbk;
            tile_coords(t - G.tile0, G.num_m, G.num_n, group_m, mb, nbk);
            const int m0 = mb * BM, n0 = nbk * BN;
            const int M = G.M, N = G.N;
            const int chunks_per_tile = (G.K / C::K_ELEMS + drain - 1) / drain;
            float acc[C::EPI_COLS];
#pragma unroll
            for (int i = 0; i < C::EPI_COLS; ++i) acc[i] = 0.f;
            for (int c = 0; c < chunks_per_tile; ++c, ++ch) {
                const int X = (int)(ch & 1);
                const uint32_t use = (uint32_t)(ch >> 1);
                if (!mbar_wait(smem_u32(&acc_full[X]), use & 1u, abort_flag, wait_ns)) { ok = false; break; }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t tbase = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(X * BN + half * C::EPI_COLS);
#pragma unroll
                for (int sub = 0; sub < C::EPI_COLS / 32; ++sub) {
                    uint32_t r[32];
                    tmem_ld32(tbase + (uint32_t)(sub * 32), r);
#pragma unroll
                    for (int i = 0; i < 32; ++i) acc[sub * 32 + i] += __uint_as_float(r[i]);
                }
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncwarp();
                if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_empty[X])) : "memory");
            }
            if (!ok) break;
            // Store through this warp's 32 x 32 staging block: each lane writes its row's 32 columns, then
            // lanes 8i..8i+7 store 128 contiguous bytes of one row each, so one store instruction covers
            // four full 128-byte lines instead of 16 bytes of 32 rows.  16-byte chunks are XOR-swizzled by
            // row (chunk j of row r at j ^ (r & 7)), which keeps both phases free of bank conflicts.
            float *wbuf = epi_buf + ew * C::EPI_BUF_FLOATS;
            const int cb0 = n0 + half * C::EPI_COLS;
            const bool vec = ((ldd & 3) == 0) && ((G.d_off & 3) == 0);
            const int rsub = lane >> 3, chk = lane & 7;
#pragma unroll
            for (int sub = 0; sub < C::EPI_COLS / 32; ++sub) {
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    *reinterpret_cast<float4 *>(wbuf + lane * 32 + 4 * (j ^ (lane & 7))) =
                        make_float4(acc[sub * 32 + 4 * j], acc[sub * 32 + 4 * j + 1], acc[sub * 32 + 4 * j + 2],
                                    acc[sub * 32 + 4 * j + 3]);
                __syncwarp();
                const int cb = cb0 + sub * 32 + 4 * chk;
#pragma unroll 1
                for (int i0 = 0; i0 < 32; i0 += 4) {
                    const int i = i0 + rsub;
                    const float4 v = *reinterpret_cast<const float4 *>(wbuf + i * 32 + 4 * (chk ^ (i & 7)));
                    const long long grow = (long long)m0 + q * 32 + i;
                    if (grow >= M) continue;
                    float *drow = D + G.d_off + grow * ldd;
                    if (vec && cb + 4 <= N) {
                        float4 o = v;
                        if (accumulate) {
                            const float4 old = *reinterpret_cast<const float4 *>(drow + cb);
                            o.x += old.x; o.y += old.y; o.z += old.z; o.w += old.w;
                        }
                        *reinterpret_cast<float4 *>(drow + cb) = o;
                    } else {
                        const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                        for (int e = 0; e < 4; ++e)
                            if (cb + e < N) drow[cb + e] = accumulate ? drow[cb + e] + vv[e] : vv[e];
                    }
                }
                __syncwarp();   // the block is rewritten by the next 32 columns
            }
        }
        if (!ok) *abort_flag = 1;
    }

    // ---------------- teardown ----------------
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (*abort_flag) {
        if (threadIdx.x == 0) atomicOr(err, ERR_TIMEOUT);
        volatile int never = 0;
        if (warp == 0 && lane == 0) {
            // drain the TMA copies this CTA still has in flight (bounded; copies older than the last
            // STAGES completed before their slots were handed back)
            for (long long g = (issued > STAGES ? issued - STAGES : 0); g < issued; ++g)
                mbar_wait(smem_u32(&bars[g % STAGES]), (uint32_t)(g / STAGES) & 1u, &never, DRAIN_BUDGET_NS);
        }
        if (warp == 1 && lane == 0) {
            // every MMA this thread issued has retired before the accumulator columns are released
            umma_commit(smem_u32(done_bar));
            mbar_wait(smem_u32(done_bar), 0u, &never, DRAIN_BUDGET_NS);
        }
        __syncthreads();
    }
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(C::TMEM_COLS) : "memory");
    }
}

// ------------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn get_encode() {
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

// rows x K operand, leading dimension ld (elements), box = box_rows x (128 bytes of K)
static int make_map(CUtensorMap *map, const void *base, bool tf32, long long rows, long long K, long long ld, int box_rows) {
    EncodeTiledFn enc = get_encode();
    TD_CHECK(enc != nullptr, TDSCHA_ECUDA, "cuTensorMapEncodeTiled entry point unavailable");
    const size_t es = tf32 ? 4 : 2;
    TD_CHECK((reinterpret_cast<uintptr_t>(base) & 15) == 0, TDSCHA_EINVAL, "operand base not 16-byte aligned");
    TD_CHECK(((ld * es) & 15) == 0, TDSCHA_EINVAL, "operand row stride not a multiple of 16 bytes");
    cuuint64_t gdim[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    cuuint64_t gstride[1] = {(cuuint64_t)(ld * es)};
    cuuint32_t box[2] = {(cuuint32_t)(128 / es), (cuuint32_t)box_rows};
    cuuint32_t estride[2] = {1, 1};
    CUresult r = enc(map, tf32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                     const_cast<void *>(base), gdim, gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    TD_CHECK(r == CUDA_SUCCESS, TDSCHA_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return 0;
}

// k-blocks accumulated in TMEM before the epilogue drains them.  Split modes drain every k-block:
// their error is otherwise dominated by the tensor core's own fp32 accumulation; single-product
// modes are limited by operand rounding and drain every 16.  TDSCHA_DRAIN_KB overrides (tuning).
static int default_drain(int nprod) {
    static int env_d = -2;
    if (env_d == -2) {
        const char *env = getenv("TDSCHA_DRAIN_KB");
        env_d = env ? std::max(1, atoi(env)) : -1;
    }
    if (env_d > 0) return env_d;
    return nprod == 3 ? 1 : 16;
}

// Autotuner key: one choice per (format, products, M, N, K, device).
struct TuneKey {
    int tf32, nprod, M, N, K, dev;
    unsigned long long shape;   // hash of the sub-problems' shapes of a grouped launch (0: one problem)
    bool operator<(const TuneKey &o) const {
        return std::tie(tf32, nprod, M, N, K, dev, shape) < std::tie(o.tf32, o.nprod, o.M, o.N, o.K, o.dev, o.shape);
    }
};
static std::mutex g_tune_mutex;

// One tile-start counter per (device, stream), zeroed on the stream before every launch, so that
// contractions running concurrently on different streams never share one.  A counter (256 bytes)
// is allocated on a stream's first launch outside graph capture and kept for the process.
static std::mutex g_sync_mutex;
static std::map<std::pair<int, cudaStream_t>, unsigned *> g_sync_counter;

static int tile_sync_counter(int dev, cudaStream_t st, bool capturing, unsigned **out) {
    std::lock_guard<std::mutex> lock(g_sync_mutex);
    TD_CHECK(dev >= 0 && dev < 64, TDSCHA_EINVAL, "device index %d out of range", dev);
    auto it = g_sync_counter.find({dev, st});
    if (it != g_sync_counter.end()) { *out = it->second; return 0; }
    if (capturing) { *out = nullptr; return 0; }   // no allocation inside a capture: no alignment
    void *slab = nullptr;
    TD_CUDA(cudaMalloc(&slab, 256));
    g_sync_counter[{dev, st}] = static_cast<unsigned *>(slab);
    *out = static_cast<unsigned *>(slab);
    return 0;
}

// Budget of one tile-start wait (TDSCHA_TILE_SYNC_US, 0 disables the alignment).
static unsigned tile_sync_budget_ns() {
    static long long v = -1;
    if (v < 0) {
        const char *env = getenv("TDSCHA_TILE_SYNC_US");
        v = env ? std::max(0, atoi(env)) * 1000LL : 50000LL;
    }
    return (unsigned)v;
}

// One tile configuration of a contraction, ready to launch with a tile-group size.
struct Prepared {
    std::function<void(int)> launch;
    int num_m = 0;
    int bn = 0;            // tile width (outputs per tile along N)
    long long tiles = 0;
};

// Extents of the two operand buffers and the sub-problems of one contraction.
struct Problem {
    long long a_rows, a_cols, b_rows, b_cols;
    std::vector<GemmGroup> groups;
};

template <int BN, int STAGES, bool TF32, int NPROD>
static int prepare_cfg(const GemmOperands &op, const Problem &pb, size_t g0, size_t g1, float *D, long long ldd,
                       cudaStream_t st, unsigned *err, unsigned *counter, int stall, Prepared *out) {
    using C = Cfg<BN, STAGES, TF32, NPROD>;
    CUtensorMap a_hi, a_lo, b_hi, b_lo;
    TD_TRY(make_map(&a_hi, op.A_hi, TF32, pb.a_rows, pb.a_cols, op.lda, BM));
    TD_TRY(make_map(&b_hi, op.B_hi, TF32, pb.b_rows, pb.b_cols, op.ldb, BN));
    if (NPROD == 3) {
        TD_TRY(make_map(&a_lo, op.A_lo, TF32, pb.a_rows, pb.a_cols, op.lda, BM));
        TD_TRY(make_map(&b_lo, op.B_lo, TF32, pb.b_rows, pb.b_cols, op.ldb, BN));
    } else {
        a_lo = a_hi;
        b_lo = b_hi;
    }
    GroupTable gt{};
    gt.n = (int)(g1 - g0);
    long long tiles = 0;
    int max_m = 1;
    for (size_t i = g0; i < g1; ++i) {
        const GemmGroup &q = pb.groups[i];
        DevGroup &d = gt.g[i - g0];
        d.M = q.M; d.N = q.N; d.K = q.K;
        d.a_row = q.a_row; d.a_k = q.a_k; d.b_row = q.b_row; d.b_k = q.b_k;
        d.d_off = q.d_off;
        d.num_m = ceil_div(q.M, BM);
        d.num_n = ceil_div(q.N, BN);
        d.tile0 = (int)tiles;
        tiles += (long long)d.num_m * d.num_n;
        max_m = std::max(max_m, d.num_m);
    }
    TD_CHECK(tiles < (1LL << 31), TDSCHA_EINVAL, "tc::gemm: %lld tiles exceed the schedule", tiles);
    gt.total_tiles = (int)tiles;
    auto kern = tc_gemm_kernel<BN, STAGES, TF32, NPROD>;
    TD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM_BYTES));
    int dev = 0, sms = 148;
    TD_CUDA(cudaGetDevice(&dev));
    TD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int drain = op.drain_kb > 0 ? op.drain_kb : default_drain(NPROD);
    const dim3 grid((unsigned)std::min<long long>(tiles, sms));
    const unsigned sync_ns = tile_sync_budget_ns();
    const int accumulate = op.accumulate ? 1 : 0;
    const unsigned long long wait_ns = g_wait_budget_ns.load();
    unsigned *cnt = (sync_ns > 0 && tiles > grid.x) ? counter : nullptr;
    out->num_m = max_m;
    out->bn = BN;
    out->tiles = tiles;
    out->launch = [=](int gm) {
        if (cnt) cudaMemsetAsync(cnt, 0, sizeof(unsigned), st);
        kern<<<grid, NUM_THREADS, C::SMEM_BYTES, st>>>(a_hi, a_lo, b_hi, b_lo, gt, drain, gm, D, ldd, err, cnt, sync_ns,
                                                        accumulate, wait_ns, stall);
    };
    return 0;
}

// ---- tile-shape and tile-order autotuner -----------------------------------------------------------
// On the first call for a (format, products, M, N, K) the launcher times every candidate (tile
// configuration, tile-group size) on the caller's stream and remembers the winner: the candidates run
// in turn, twice round (every run writes the same D), and each keeps its faster run, so that the clock
// drift of a power-capped GPU over the trials does not favour the candidates timed first.
// TDSCHA_AUTOTUNE_VERBOSE=1 prints every trial and the choice to stderr.  Tile configurations: 128 x 256 with the stage count that
// fits (2 for the split modes, 4 otherwise) and 128 x 128 with more stages (3 / 6): the wide tile
// reads each A panel half as often, the narrow one keeps a deeper copy pipeline.  Small problems,
// launches that accumulate or are being captured, and TDSCHA_AUTOTUNE=0 use the wide tile in the
// m-fastest order; TDSCHA_TILE_N (256 | 128) and TDSCHA_GROUP_M fix the choice.
static std::map<TuneKey, std::pair<int, int>> g_tune_cfg;

static int choose(int tf32, int nprod, int M, int N, int K, unsigned long long shape, const Prepared *cfgs, int ncfg,
                  cudaStream_t st, bool allow_trials, int *cfg_out, int *gm_out) {
    int dev = 0, sms = 148;
    TD_CUDA(cudaGetDevice(&dev));
    TD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    int forced_cfg = -1;
    if (const char *env = getenv("TDSCHA_TILE_N")) forced_cfg = atoi(env) == 128 ? 1 : 0;
    const char *env_gm = getenv("TDSCHA_GROUP_M");
    if (forced_cfg >= 0 || env_gm) {
        const int c = forced_cfg >= 0 ? std::min(forced_cfg, ncfg - 1) : 0;
        *cfg_out = c;
        *gm_out = env_gm ? std::max(1, std::min(cfgs[c].num_m, atoi(env_gm))) : cfgs[c].num_m;
        return 0;
    }
    const TuneKey key{tf32, nprod, M, N, K, dev, shape};
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tune_cfg.find(key);
        if (it != g_tune_cfg.end()) { *cfg_out = it->second.first; *gm_out = it->second.second; return 0; }
    }
    const char *env = getenv("TDSCHA_AUTOTUNE");
    const bool enabled = allow_trials && !(env && atoi(env) == 0);
    int best_c = 0, best_gm = cfgs[0].num_m;
    const char *env_v = getenv("TDSCHA_AUTOTUNE_VERBOSE");
    const bool verbose = env_v && atoi(env_v) == 1;
    if (enabled && cfgs[0].tiles >= 8LL * sms) {
        std::vector<std::pair<int, int>> cands;   // (configuration, tile-group size)
        for (int c = 0; c < ncfg; ++c) {
            const int num_m = cfgs[c].num_m;
            const int cand_all[] = {num_m, 48, 24, 12, 6};
            for (int ci = 0; ci < 5; ++ci) {
                const int cand = cand_all[ci];
                bool dup = cand > num_m;
                for (int cj = 0; cj < ci; ++cj) dup = dup || cand_all[cj] == cand;
                if (!dup) cands.push_back({c, cand});
            }
        }
        cudaEvent_t e0, e1;
        TD_CUDA(cudaEventCreate(&e0));
        TD_CUDA(cudaEventCreate(&e1));
        std::vector<float> t_min(cands.size(), 1e30f);
        for (int round = 0; round < 2; ++round)
            for (size_t i = 0; i < cands.size(); ++i) {
                TD_CUDA(cudaEventRecord(e0, st));
                cfgs[cands[i].first].launch(cands[i].second);
                TD_CUDA(cudaGetLastError());
                TD_CUDA(cudaEventRecord(e1, st));
                TD_CUDA(cudaEventSynchronize(e1));
                float ms = 0.f;
                TD_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                t_min[i] = std::min(t_min[i], ms);
                if (verbose)
                    fprintf(stderr, "[tc autotune] M=%d N=%d K=%d nprod=%d tile_n=%d group_m=%d round %d: %.3f ms\n", M, N, K,
                            nprod, cfgs[cands[i].first].bn, cands[i].second, round, ms);
            }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        size_t bi = 0;
        for (size_t i = 1; i < cands.size(); ++i)
            if (t_min[i] < t_min[bi]) bi = i;
        best_c = cands[bi].first;
        best_gm = cands[bi].second;
    }
    if (verbose)
        fprintf(stderr, "[tc autotune] M=%d N=%d K=%d nprod=%d -> tile_n=%d group_m=%d\n", M, N, K, nprod, cfgs[best_c].bn,
                best_gm);
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    if (allow_trials) g_tune_cfg[key] = {best_c, best_gm};
    *cfg_out = best_c;
    *gm_out = best_gm;
    return 0;
}

template <bool TF32, int NPROD>
static int launch_tuned(const GemmOperands &op, const Problem &pb, float *D, long long ldd, cudaStream_t st, unsigned *err) {
    constexpr int S_WIDE = NPROD == 3 ? 2 : 4, S_NARROW = NPROD == 3 ? 3 : 6, S_THIN = NPROD == 3 ? 4 : 8;
    int dev = 0;
    TD_CUDA(cudaGetDevice(&dev));
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    TD_CUDA(cudaStreamIsCapturing(st, &cap));
    const bool capturing = cap != cudaStreamCaptureStatusNone;
    unsigned *counter = nullptr;
    if (tile_sync_budget_ns() > 0) TD_TRY(tile_sync_counter(dev, st, capturing, &counter));
    const int stall = g_stall_next.exchange(0);
    for (size_t g0 = 0; g0 < pb.groups.size(); g0 += MAX_GROUPS) {
        const size_t g1 = std::min(pb.groups.size(), g0 + MAX_GROUPS);
        Prepared cfgs[3];
        TD_TRY((prepare_cfg<256, S_WIDE, TF32, NPROD>(op, pb, g0, g1, D, ldd, st, err, counter, stall, &cfgs[0])));
        TD_TRY((prepare_cfg<128, S_NARROW, TF32, NPROD>(op, pb, g0, g1, D, ldd, st, err, counter, stall, &cfgs[1])));
        // outputs at most 64 columns wide in every group (the per-class mode-column contractions): the
        // 128 x 64 tile, whose shorter B rows leave room for a deeper A stream, and no wasted MMA columns
        bool thin = true;
        for (size_t i = g0; i < g1; ++i) thin = thin && pb.groups[i].N <= 64;
        const char *env_tn = getenv("TDSCHA_TILE_N");
        if (env_tn) thin = thin && atoi(env_tn) == 64;
        if (thin) TD_TRY((prepare_cfg<64, S_THIN, TF32, NPROD>(op, pb, g0, g1, D, ldd, st, err, counter, stall, &cfgs[2])));
        // tuning key: the one problem's shape, or the groups' shapes hashed (FNV-1a)
        int kM = pb.groups[g0].M, kN = pb.groups[g0].N, kK = pb.groups[g0].K;
        unsigned long long shape = 0;
        if (g1 - g0 > 1) {
            shape = 1469598103934665603ull;
            for (size_t i = g0; i < g1; ++i)
                for (long long v : {(long long)pb.groups[i].M, (long long)pb.groups[i].N, (long long)pb.groups[i].K}) {
                    shape ^= (unsigned long long)v;
                    shape *= 1099511628211ull;
                }
            kM = (int)(g1 - g0);
        }
        int c = 0, gm = cfgs[0].num_m;
        if (thin && !stall) {
            c = 2;
            gm = cfgs[2].num_m;
        } else if (!stall) {   // abort-path test: one launch of the wide tile, no tuning trials
            // trial runs write D, so an accumulating launch only reuses a choice tuned earlier (and a
            // launch being captured into a CUDA graph runs nothing, so it cannot time trials)
            TD_TRY(choose(TF32 ? 1 : 0, NPROD, kM, kN, kK, shape, cfgs, 2, st, !op.accumulate && !capturing, &c, &gm));
        }
        cfgs[c].launch(gm);
        TD_CUDA(cudaGetLastError());
    }
    return 0;
}

void set_wait_budget_ns(unsigned long long ns) { g_wait_budget_ns.store(ns); }
unsigned long long wait_budget_ns() { return g_wait_budget_ns.load(); }
void stall_next_launch() { g_stall_next.store(1); }

static int dispatch(const GemmOperands &op, const Problem &pb, float *D, long long ldd, cudaStream_t st, unsigned *err) {
    if (op.fmt == FMT_TF32) {
        if (op.nprod == 3) return launch_tuned<true, 3>(op, pb, D, ldd, st, err);
        return launch_tuned<true, 1>(op, pb, D, ldd, st, err);
    }
    if (op.nprod == 3) return launch_tuned<false, 3>(op, pb, D, ldd, st, err);
    return launch_tuned<false, 1>(op, pb, D, ldd, st, err);
}

int gemm(const GemmOperands &op, int M, int N, int K, float *D, long long ldd, cudaStream_t st, unsigned *err) {
    TD_CHECK(M > 0 && N > 0 && K > 0, TDSCHA_EINVAL, "tc::gemm: empty problem %d x %d x %d", M, N, K);
    const bool tf32 = op.fmt == FMT_TF32;
    TD_CHECK(op.fmt == FMT_TF32 || op.fmt == FMT_BF16, TDSCHA_EINVAL, "tc::gemm: operand format must be bf16 or tf32");
    TD_CHECK(K % (tf32 ? 32 : 64) == 0, TDSCHA_EINVAL, "tc::gemm: K=%d not a multiple of the 128-byte K block", K);
    TD_CHECK(op.nprod == 1 || op.nprod == 3, TDSCHA_EINVAL, "tc::gemm: nprod must be 1 or 3");
    constexpr long long LD_MAX = 1LL << 31;
    TD_CHECK(op.lda >= K && op.ldb >= K && ldd >= N && op.lda < LD_MAX && op.ldb < LD_MAX && ldd < LD_MAX, TDSCHA_EINVAL,
             "tc::gemm: leading dimensions lda=%lld ldb=%lld ldd=%lld inconsistent with K=%d N=%d", op.lda, op.ldb, ldd, K, N);
    TD_CHECK(op.A_hi && op.B_hi && D && (op.nprod == 1 || (op.A_lo && op.B_lo)), TDSCHA_EINVAL, "tc::gemm: NULL operand");
    Problem pb{M, K, N, K, {GemmGroup{M, N, K, 0, 0, 0, 0, 0}}};
    return dispatch(op, pb, D, ldd, st, err);
}

int gemm_grouped(const GemmOperands &op, long long a_rows, long long a_cols, long long b_rows, long long b_cols,
                 const GemmGroup *groups, int n_groups, float *D, long long ldd, cudaStream_t st, unsigned *err) {
    TD_CHECK(n_groups > 0 && groups, TDSCHA_EINVAL, "tc::gemm_grouped: no groups");
    const bool tf32 = op.fmt == FMT_TF32;
    TD_CHECK(op.fmt == FMT_TF32 || op.fmt == FMT_BF16, TDSCHA_EINVAL, "tc::gemm_grouped: operand format must be bf16 or tf32");
    TD_CHECK(op.nprod == 1 || op.nprod == 3, TDSCHA_EINVAL, "tc::gemm_grouped: nprod must be 1 or 3");
    const int kblk = tf32 ? 32 : 64;
    constexpr long long LD_MAX = 1LL << 31;
    TD_CHECK(op.lda >= a_cols && op.ldb >= b_cols && op.lda < LD_MAX && op.ldb < LD_MAX && ldd < LD_MAX && a_rows < LD_MAX &&
                 b_rows < LD_MAX && a_cols < LD_MAX && b_cols < LD_MAX,
             TDSCHA_EINVAL, "tc::gemm_grouped: operand extents inconsistent with their leading dimensions");
    TD_CHECK(op.A_hi && op.B_hi && D && (op.nprod == 1 || (op.A_lo && op.B_lo)), TDSCHA_EINVAL, "tc::gemm_grouped: NULL operand");
    Problem pb{a_rows, a_cols, b_rows, b_cols, {}};
    for (int i = 0; i < n_groups; ++i) {
        const GemmGroup &g = groups[i];
        TD_CHECK(g.M > 0 && g.N > 0 && g.K > 0 && g.K % kblk == 0 && g.a_k % kblk == 0 && g.b_k % kblk == 0, TDSCHA_EINVAL,
                 "tc::gemm_grouped: group %d: M=%d N=%d K=%d a_k=%d b_k=%d (K and offsets multiples of %d)", i, g.M, g.N, g.K,
                 g.a_k, g.b_k, kblk);
        TD_CHECK(g.a_row >= 0 && g.b_row >= 0 && g.a_row < a_rows && g.b_row < b_rows && g.a_k + (long long)g.K <= a_cols &&
                     g.b_k + (long long)g.K <= b_cols && g.N <= ldd && g.d_off >= 0,
                 TDSCHA_EINVAL, "tc::gemm_grouped: group %d outside its operands", i);
        pb.groups.push_back(g);
    }
    return dispatch(op, pb, D, ldd, st, err);
}

}  // namespace tc
}  // namespace tdscha
