// tc_gemm.cuh -- interface of the tcgen05 contraction kernel (tc_gemm.cu).
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"

namespace tdscha {
namespace tc {

// D (M x N, fp32) = A (M x K) . B (N x K)^T, both operands row-major with K contiguous.
// fmt FMT_BF16: bf16 elements; FMT_TF32: fp32 elements already rounded to tf32.
// nprod 3 uses A_lo/B_lo (hi.hi + hi.lo + lo.hi); nprod 1 ignores them.
struct GemmOperands {
    Format fmt;
    int nprod;
    const void *A_hi, *A_lo;
    long long lda;   // elements; lda * element size must be a multiple of 16 bytes
    const void *B_hi, *B_lo;
    long long ldb;
    int drain_kb = 0;   // k-blocks per TMEM chunk drained to fp32 registers (0 = library default)
    bool accumulate = false;   // D += A . B^T instead of D = A . B^T
};

// K must be a multiple of 64 (bf16) or 32 (tf32); operands must be readable up to K columns.
int gemm(const GemmOperands &op, int M, int N, int K, float *D, long long ldd, cudaStream_t st, unsigned *err);

// One sub-problem of a grouped launch: D[d_off + m * ldd + n] (+)= sum_k A[a_row + m, a_k + k] B[b_row + n, b_k + k]
// for m < M, n < N, k < K (K a multiple of the 128-byte k-block; a_k, b_k multiples of it too).
struct GemmGroup {
    int M, N, K;
    int a_row, a_k, b_row, b_k;
    long long d_off;
};

// Several sub-problems over the same A (a_rows x a_cols) and B (b_rows x b_cols) buffers in one
// persistent launch (every 64 groups one launch): the tiles of all groups share the machine, so
// groups of a few tiles each leave no SM idle.
int gemm_grouped(const GemmOperands &op, long long a_rows, long long a_cols, long long b_rows, long long b_cols,
                 const GemmGroup *groups, int n_groups, float *D, long long ldd, cudaStream_t st, unsigned *err);

// Budget of every bounded wait of later launches (default 4 s), and a one-shot request that the next
// launch's producers issue no copy (its MMA warps' first wait then runs out): the abort-path test.
void set_wait_budget_ns(unsigned long long ns);
unsigned long long wait_budget_ns();
void stall_next_launch();

}  // namespace tc
}  // namespace tdscha
