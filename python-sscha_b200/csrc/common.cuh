// common.cuh -- shared helpers of the tdscha_b200 CUDA library (sm_100a only).
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <cstdio>
#include <cstdarg>

#include "tdscha_b200.h"

namespace tdscha {

// Thread-local message of the last failure (tdscha_last_error).
void set_error(const char *fmt, ...);
void clear_error();

#define TD_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            ::tdscha::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
            return e_ == cudaErrorMemoryAllocation ? TDSCHA_ENOMEM : TDSCHA_ECUDA;             \
        }                                                                                      \
    } while (0)

#define TD_CHECK(cond, code, ...)                                                              \
    do {                                                                                       \
        if (!(cond)) {                                                                         \
            ::tdscha::set_error(__VA_ARGS__);                                                  \
            return (code);                                                                     \
        }                                                                                      \
    } while (0)

#define TD_TRY(expr)                                                                           \
    do {                                                                                       \
        int rc_ = (expr);                                                                      \
        if (rc_ != 0) return rc_;                                                              \
    } while (0)

constexpr double RY_TO_K = 157887.32400374097;  // CModules/LanczosFunctions.h:9

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }
inline long long round_up(long long a, long long b) { return (a + b - 1) / b * b; }

// Operand storage formats of the tensor-core contractions (FMT_F32: plain fp32, for intermediate
// products that are not contraction operands).
enum Format : int { FMT_F64 = 0, FMT_BF16 = 1, FMT_TF32 = 2, FMT_F32 = 3 };

inline Format format_of(int precision) {
    switch (precision) {
        case TDSCHA_PREC_TF32:
        case TDSCHA_PREC_TF32X3: return FMT_TF32;
        case TDSCHA_PREC_BF16X3:
        case TDSCHA_PREC_BF16: return FMT_BF16;
        default: return FMT_F64;
    }
}
inline int products_of(int precision) {
    return (precision == TDSCHA_PREC_BF16X3 || precision == TDSCHA_PREC_TF32X3) ? 3 : 1;
}
inline bool needs_lo(int precision) { return products_of(precision) == 3; }

// Device-side error word shared by all kernels of a call: bit 0 = a bounded wait expired.
constexpr unsigned ERR_TIMEOUT = 1u;

// ---- split helpers (device) -----------------------------------------------------------------
__device__ __forceinline__ uint16_t bf16_bits_rn(float f) {
    return __bfloat16_as_ushort(__float2bfloat16_rn(f));
}
__device__ __forceinline__ float bf16_bits_to_float(uint16_t b) { return __bfloat162float(__ushort_as_bfloat16(b)); }

__device__ __forceinline__ float tf32_round(float f) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(f));
    return __uint_as_float(r);
}

// Store x (FP64) into an operand slot of the given format: hi (and lo when lo != nullptr).
__device__ __forceinline__ void store_split(Format fmt, void *hi, void *lo, long long idx, double x) {
    if (fmt == FMT_F64) {
        static_cast<double *>(hi)[idx] = x;
    } else if (fmt == FMT_F32) {
        static_cast<float *>(hi)[idx] = (float)x;
    } else if (fmt == FMT_BF16) {
        uint16_t h = bf16_bits_rn((float)x);
        static_cast<uint16_t *>(hi)[idx] = h;
        if (lo) static_cast<uint16_t *>(lo)[idx] = bf16_bits_rn((float)(x - (double)bf16_bits_to_float(h)));
    } else {
        float h = tf32_round((float)x);
        static_cast<float *>(hi)[idx] = h;
        if (lo) static_cast<float *>(lo)[idx] = tf32_round((float)(x - (double)h));
    }
}

inline size_t format_bytes(Format f) { return f == FMT_F64 ? 8 : (f == FMT_BF16 ? 2 : 4); }   // FMT_F32: 4

}  // namespace tdscha
