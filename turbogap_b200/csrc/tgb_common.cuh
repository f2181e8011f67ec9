// tgb_common.cuh -- shared definitions of the B200 SOAP-GAP backend.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/tgb200.h"

namespace tgb {

// ---- error reporting ------------------------------------------------------
void set_error(const char *fmt, ...);
const char *last_error();

#define TGB_CUDA(call)                                                            \
    do {                                                                          \
        cudaError_t e__ = (call);                                                 \
        if (e__ != cudaSuccess) {                                                 \
            ::tgb::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #call,          \
                             cudaGetErrorString(e__));                            \
            return TG_ERR_CUDA;                                                   \
        }                                                                         \
    } while (0)

#define TGB_CHECK(cond, code, ...)                                                \
    do {                                                                          \
        if (!(cond)) {                                                            \
            ::tgb::set_error(__VA_ARGS__);                                        \
            return (code);                                                        \
        }                                                                         \
    } while (0)

#define TGB_TRY(call)                                                             \
    do {                                                                          \
        int r__ = (call);                                                         \
        if (r__ != TG_OK) return r__;                                             \
    } while (0)

// Device error word bits (read back after each step / call).
enum DevErr : unsigned {
    DEV_ERR_NEIGH_CAPACITY = 1u << 0,   // pair array too small
    DEV_ERR_TIMEOUT_TMA = 1u << 1,      // bounded mbarrier wait expired (producer)
    DEV_ERR_TIMEOUT_MMA = 1u << 2,      // bounded mbarrier wait expired (MMA issuer)
    DEV_ERR_TIMEOUT_EPI = 1u << 3,      // bounded mbarrier wait expired (epilogue)
    DEV_ERR_BAD_INDEX = 1u << 4,        // index outside its array (skipped)
    DEV_ERR_NONFINITE = 1u << 5,        // NaN/Inf in an energy or force
    DEV_ERR_CELL_CAPACITY = 1u << 6,    // too many atoms for the cell grid
};

// ---- small device helpers --------------------------------------------------
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Split a value into bf16 hi + bf16 lo with hi + lo ~= x to about 2^-16 relative.
__device__ __forceinline__ void bf16_split(float x, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
    hi = __float2bfloat16_rn(x);
    lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

constexpr double kPi = 3.14159265358979323846;

// Maximum sizes compiled into the kernels.
constexpr int kMaxSpecies = 4;
constexpr int kTableIntervals = 2048;   // cubic-Hermite intervals per species over [0, rcut_hard]

}  // namespace tgb
