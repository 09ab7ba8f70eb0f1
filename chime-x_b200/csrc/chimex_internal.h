// chimex_internal.h -- shared declarations of libchimex (not installed).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/chimex.h"

namespace chx {

// Value maps: how a packed byte becomes the int8 operands of the correlator.
// For a row element y the operand pair is (a0, a1); for a column element x
// the Re column is (b0, b1) and the Im column is (b2, b3), so that per sample
//   Re += a0*b0 + a1*b1,   Im += a0*b2 + a1*b3.
// MAP_EXACT   signed values s = nibble - 8: a = (yr, yi), Re = (xr, xi),
//             Im = (-xi, xr); exact visibilities, no corrections needed.
// MAP_CONF    offset nibbles n = s + 8: the partials of the conference corr
//             kernel (pairwise_correlator_UT.cl:107-201).
// MAP_PACKED  offset nibbles with the y imaginary nibble inverted (15 - n):
//             the partials of the packed corr kernel
//             (packed_correlator_overflow_protected_to_2272_iter_UT.cl:91-285):
//             a = (y'r, 15 - y'i), Re = (x'r, -x'i), Im = (-x'i, -x'r).
// The non-UT conventions negate Im in the epilogue.
enum ValueMap : int { MAP_EXACT = 0, MAP_CONF = 1, MAP_PACKED = 2 };

struct Shape {
    int E, F, T;
    int64_t NB1, NB;
};

}  // namespace chx

struct chx_plan {
    int E, F, T, TA, ut, kernel_batch, device;
    int64_t NB1, NB;
    int algo;     // CHX_ALGO_*
    int tsplit;   // 0 = auto
    int tile;     // 0 = auto
    int *d_err;   // device error word (bounded-wait timeouts)
    int sm_count;
};

namespace chx {

// Error helpers: set the thread-local message and return the code.
int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);
void clear_error();

#define CHX_CUDA(call)                                      \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return chx::cuda_fail(e_, #call); \
    } while (0)

// RAII: make `dev` current for the scope, restore the previous device.
struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) ok = (cudaSetDevice(dev) == cudaSuccess);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev)
            cudaSetDevice(prev);
    }
};

inline int64_t num_blocks_of(int E) {
    int64_t n = E / 32;
    return n * (n + 1) / 2;
}

// ---- SIMT kernels (simt_kernels.cu) ----
// Correlates samples [t_begin, t_end) of every channel with the CUDA-core
// dp4a kernel.  mode: 0 store, 1 add (plain RMW), 2 atomic add.
cudaError_t launch_correlate_simt(const uint8_t *packed, int32_t *blocks, int E, int F,
                                  int T, int map, int ut, int mode, int splits,
                                  cudaStream_t st);
cudaError_t launch_offset_accumulate(const uint8_t *packed, uint32_t *sums, int E, int F,
                                     int T, cudaStream_t st);
cudaError_t launch_preseed(const uint32_t *sums, int32_t *blocks, int E, int F, int T,
                           int packed_variant, int ut, cudaStream_t st);
cudaError_t launch_blocks_to_triangle(const int32_t *blocks, int32_t *tri, int E, int F,
                                      cudaStream_t st);
cudaError_t launch_blocks_to_full(const int32_t *blocks, int32_t *full, int E, int F,
                                  cudaStream_t st);

// ---- tensor-core kernels (tc_correlator.cu) ----
struct TcArgs {
    const uint8_t *packed;  // [T][F][E] (sample stride = in_stride bytes)
    int64_t in_stride;      // bytes between consecutive samples of a channel
    int64_t chan_stride;    // bytes between channels within a sample row
    int32_t *blocks;        // [F][NB][2048]
    int64_t out_chan_stride;  // int32 words between channels' block buffers
    int E, F, T;
    int map, ut;
    int mode;       // 0 store, 1 add, 2 atomic add
    int splits;     // sample-range splits
    int *err;       // device error word
};
bool tc_supported(int E, int T);
cudaError_t launch_correlate_tc(const TcArgs &a, int sm_count, cudaStream_t st);

}  // namespace chx
