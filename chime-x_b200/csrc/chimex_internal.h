// chimex_internal.h -- shared declarations of libchimex (not installed).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#include <functional>
#include <string>
#include <vector>

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
    void *d_chans;  // tensor-core channel table (ChanDesc[F])
    void *d_units;  // tensor-core work units (Unit[nunits]) then grid + 1 offsets
    int nunits;
    int grid;       // persistent CTAs (or CTA pairs) of a tensor-core launch
    int tile_built; // tile variant the tables were built for
    bool has_split_units;  // some output cells receive several units (TMA reduce-add)
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

// NVTX range around a public entry point: profilers (nsys, ncu) show each
// call by name; without a tool attached a push/pop is a cheap no-op.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
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

// ---- tensor-core kernel (tc_correlator.cu) ----
// A channel as the tensor-core kernel sees it: the TMA map of its packed
// samples (dims {E, channels, samples}), its block-buffer address and shape.
struct __align__(64) ChanDesc {
    CUtensorMap map;   // samples; used unless the launch passes one map for all channels
    CUtensorMap omap;  // block output as rows of 64 words (tc_encode_out_map); same rule
    uint64_t out;      // block buffer: absolute address, or byte offset added to
                       // the launch's out_base
    int E;             // elements
    int nb1;           // E / 32
    int fcoord;        // channel coordinate inside the TMA map
    int orow;          // first row of this channel's blocks inside omap
    int pad[10];
};
static_assert(sizeof(ChanDesc) == 320, "ChanDesc layout");

// One work unit: a 128-element y tile against one or two 128-element x tiles
// of one channel over samples [t0, t1).  tyx = ty | x0 << 10 | nx << 20.
struct Unit {
    int chan;
    int tyx;
    int t0, t1;
    long long out_off;  // int32 words added to the channel's block buffer
    int split;          // 1: other units add to the same cells (TMA reduce-add)
    int cost;           // samples x x-tiles, for scheduling
};
static_assert(sizeof(Unit) == 32, "Unit layout");

constexpr int kUnitMaxSamples = 1 << 18;  // int32-exact bound per unit
constexpr int kUnitStageSamples = 32;      // samples per pipeline stage of both kernels

// Scheduling cost of a unit over samples [t0, t1): its pipeline stages, times
// the x tiles it converts plus its y tile for the one-SM kernel (nx = 1 or 2
// x tiles of 128 elements); SM-pair units all convert one y and one x tile per
// SM, so their cost is their stage count.  Plans, batches, streams and the
// allocation-free entry point share it so that their schedules agree.
__host__ __device__ inline int unit_cost(bool pair, int t0, int t1, int nx) {
    const int stages = (t1 - t0 + kUnitStageSamples - 1) / kUnitStageSamples;
    return pair ? stages : stages * (2 * nx + 1);
}

struct TcLaunch {
    const ChanDesc *chans;  // device
    const Unit *units;      // device, grouped by CTA
    int nunits;
    const int *cta_offsets; // device, grid + 1 entries
    uint64_t out_base;      // added to ChanDesc::out
    int use_param_map;      // 1: every channel uses the kernel-parameter map
    int map;                // value map (MAP_*)
    int ut;
    int accumulate;
    int *err;
    int grid;               // persistent CTAs (<= SMs)
};

bool tc_supported(int E, int T);
// Appends the units of one channel's sample range [t_begin, t_end) to `out`.
void tc_append_units(std::vector<Unit> &out, int chan, int E, int t_begin, int t_end,
                     int tsplit, long long out_off);
// Assigns units to `grid` persistent CTAs (longest first, to the least
// loaded CTA) and reorders them CTA by CTA; offsets gets grid + 1 entries.
void tc_schedule(std::vector<Unit> &u, int grid, std::vector<int> &offsets);
// Makespan, in unit-cost units, of that assignment when every unit also pays
// `handoff_stages` of its stages for the accumulator hand-off.
long long tc_estimate_makespan(const std::vector<Unit> &u, int grid, int handoff_stages);
// Number of sample-range splits k (1-8) whose units, made by build(k, out),
// have the shortest estimated makespan on the tile variant.
int tc_choose_split(int tile, int sm_count,
                    const std::function<void(int, std::vector<Unit> &)> &build);
// The same for F channels of E elements and T samples.
int tc_auto_split(int tile, int E, int F, int T, int sm_count);
// Encodes the TMA map of packed samples: dims {E, channels, samples}.
int tc_encode_map(CUtensorMap *m, const void *base, int E, int channels, int64_t samples,
                  int64_t chan_stride, int64_t sample_stride);
// Encodes the TMA map of a block buffer seen as `rows` rows of 64 int32 words
// (one 32-cell block row of Re/Im pairs), tile {32 words, 32 rows}, 128-byte
// swizzle.  The epilogues store (or add) their tiles through it.  rows must
// stay below 2^31 (tc_out_rows_ok).
int tc_encode_out_map(CUtensorMap *m, void *base, int64_t rows);
inline bool tc_out_rows_ok(int64_t rows) { return rows > 0 && rows < (1LL << 31); }
// param_map / param_omap: the maps every channel uses when L.use_param_map.
cudaError_t tc_launch(const TcLaunch &L, const CUtensorMap *param_map,
                      const CUtensorMap *param_omap, cudaStream_t st);

// ---- 2-SM tensor-core kernel (tc_pair_correlator.cu) ----
// Units of 256 x 256 elements (tyx = ty2 | tx2 << 10, 128-element tile pairs),
// computed by a cluster of two CTAs with tcgen05.mma.cta_group::2.  In the
// launch, grid counts clusters and cta_offsets is indexed by cluster.
void tc_append_pair_units(std::vector<Unit> &out, int chan, int E, int t_begin, int t_end,
                          int tsplit, long long out_off);
cudaError_t tc_pair_launch(const TcLaunch &L, const CUtensorMap *param_map,
                           const CUtensorMap *param_omap, cudaStream_t st);

// Tensor-core tile variants (CHX_OPT_TILE).
constexpr int kTile1Sm = 1;  // 128 x 256 elements per CTA
constexpr int kTile2Sm = 2;  // 256 x 256 elements per CTA pair
constexpr int kTileMax = kTile2Sm;
int tc_default_tile(int E);
// Dispatch by tile variant: units of one channel's sample range, persistent
// CTAs (or clusters) for `sm_count` SMs, and the launch.
void tc_append_tile_units(int tile, std::vector<Unit> &out, int chan, int E, int t_begin,
                          int t_end, int tsplit, long long out_off);
int tc_tile_slots(int tile, int sm_count);
cudaError_t tc_tile_launch(int tile, const TcLaunch &L, const CUtensorMap *param_map,
                           const CUtensorMap *param_omap, cudaStream_t st);
// Device address of the error word of chx_correlate_noalloc on the current
// device (noalloc.cu); the bounded-wait self-test writes it in mode 2.
cudaError_t noalloc_error_word(int **out);
// The autotuner's cached choice for (device, E, T) (batch.cu): true and the
// tile variant and split count when an entry with the same E and a T within a
// factor 2 exists.
bool tc_tune_lookup(int device, int E, int T, int *tile, int *split);

}  // namespace chx
