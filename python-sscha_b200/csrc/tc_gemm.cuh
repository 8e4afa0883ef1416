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

// Budget of every bounded wait of later launches (default 4 s), and a one-shot request that the next
// launch's producers issue no copy (its MMA warps' first wait then runs out): the abort-path test.
void set_wait_budget_ns(unsigned long long ns);
unsigned long long wait_budget_ns();
void stall_next_launch();

}  // namespace tc
}  // namespace tdscha
