// api.cu -- C ABI of libchimex: plans and the plain-path entry points.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>

#include "chimex_internal.h"

namespace chx {

static thread_local char g_err[512] = "";

int fail(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    return fail(e == cudaErrorMemoryAllocation ? CHX_E_NOMEM : CHX_E_CUDA, "%s: %s (%s)",
                what, cudaGetErrorString(e), cudaGetErrorName(e));
}

void clear_error() { g_err[0] = 0; }

}  // namespace chx

using namespace chx;

namespace {

// Device buffers passed to the plan entry points must be 16-byte aligned: the
// tensor-core kernels move them with TMA and the CUDA-core kernels with 8-
// and 16-byte vector accesses.  (Allocations from cudaMalloc and torch are
// 256-byte aligned.)
bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

void free_plan_device(chx_plan *p) {
    if (p->d_err) cudaFree(p->d_err);
    if (p->d_chans) cudaFree(p->d_chans);
    if (p->d_units) cudaFree(p->d_units);
    p->d_err = nullptr;
    p->d_chans = nullptr;
    p->d_units = nullptr;
}

// Channel table and work units of the tensor-core kernel for the plan's
// shape: F channels sharing one TMA map (passed per launch), units of every
// channel sorted by decreasing cost.
cudaError_t build_tc_tables(chx_plan *p) {
    std::vector<ChanDesc> chans(p->F);
    memset(chans.data(), 0, chans.size() * sizeof(ChanDesc));
    for (int f = 0; f < p->F; f++) {
        chans[f].out = (uint64_t)f * (uint64_t)p->NB * 2048u * 4u;
        chans[f].E = p->E;
        chans[f].nb1 = (int)p->NB1;
        chans[f].fcoord = f;
        chans[f].orow = (int)((int64_t)f * p->NB * 32);
    }
    std::vector<Unit> units;
    // Unset options: the tile is the autotuner's cached choice for this shape,
    // if any, else the default; the split comes from the makespan estimate,
    // which sees how many units this plan has (the tuner times a workload that
    // fills the GPU, where splitting only adds hand-offs).
    int tile = p->tile, split = p->tsplit;
    int tuned_tile = 0, tuned_split = 0;
    if (!tile && tc_tune_lookup(p->device, p->E, p->T, &tuned_tile, &tuned_split))
        tile = tuned_tile;
    if (!tile) tile = tc_default_tile(p->E);
    if (!split) split = tc_auto_split(tile, p->E, p->F, p->T, p->sm_count);
    for (int f = 0; f < p->F; f++) tc_append_tile_units(tile, units, f, p->E, 0, p->T, split, 0);
    const int slots = tc_tile_slots(tile, p->sm_count);
    const int grid = (int)std::min<size_t>(units.size(), (size_t)std::max(1, slots));
    std::vector<int> offsets;
    tc_schedule(units, grid, offsets);
    if (p->d_chans) cudaFree(p->d_chans);
    if (p->d_units) cudaFree(p->d_units);
    p->d_chans = p->d_units = nullptr;
    const size_t ubytes = units.size() * sizeof(Unit);
    cudaError_t e = cudaMalloc(&p->d_chans, chans.size() * sizeof(ChanDesc));
    if (e == cudaSuccess) e = cudaMalloc(&p->d_units, ubytes + offsets.size() * sizeof(int));
    if (e == cudaSuccess)
        e = cudaMemcpy(p->d_chans, chans.data(), chans.size() * sizeof(ChanDesc),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(p->d_units, units.data(), ubytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy((char *)p->d_units + ubytes, offsets.data(), offsets.size() * sizeof(int),
                       cudaMemcpyHostToDevice);
    p->nunits = (int)units.size();
    p->grid = grid;
    p->tile_built = tile;
    p->has_split_units = false;
    for (const Unit &u : units) p->has_split_units |= (u.split != 0);
    return e;
}

// The tensor-core path addresses the plan's blocks as F*NB*32 rows of a TMA map.
bool plan_tc_ok(const chx_plan *p) {
    return tc_supported(p->E, p->T) && tc_out_rows_ok((int64_t)p->F * p->NB * 32);
}

// Launches the tensor-core kernel on the plan's tables with `map`.
int run_tc(chx_plan *p, const uint8_t *d_packed, int32_t *d_blocks, int map, int accumulate,
           cudaStream_t st) {
    if ((reinterpret_cast<uintptr_t>(d_packed) & 15) != 0)
        return fail(CHX_E_INVALID, "packed input must be 16-byte aligned for TMA");
    if ((reinterpret_cast<uintptr_t>(d_blocks) & 15) != 0)
        return fail(CHX_E_INVALID, "block buffer must be 16-byte aligned for TMA");
    CUtensorMap tmap, omap;
    int r = tc_encode_map(&tmap, d_packed, p->E, p->F, p->T, p->E, (int64_t)p->F * p->E);
    if (r != 0) return fail(CHX_E_CUDA, "cuTensorMapEncodeTiled failed (%d)", r);
    r = tc_encode_out_map(&omap, d_blocks, (int64_t)p->F * p->NB * 32);
    if (r != 0) return fail(CHX_E_CUDA, "cuTensorMapEncodeTiled (blocks) failed (%d)", r);
    if (p->has_split_units && !accumulate)
        CHX_CUDA(cudaMemsetAsync(d_blocks, 0, (size_t)chx_plan_block_words(p) * 4, st));
    TcLaunch L;
    L.chans = (const ChanDesc *)p->d_chans;
    L.units = (const Unit *)p->d_units;
    L.nunits = p->nunits;
    L.cta_offsets = (const int *)((const char *)p->d_units + (size_t)p->nunits * sizeof(Unit));
    L.out_base = (uint64_t)d_blocks;
    L.use_param_map = 1;
    L.map = map;
    L.ut = p->ut;
    L.accumulate = accumulate;
    L.err = p->d_err;
    L.grid = p->grid;
    CHX_CUDA(tc_tile_launch(p->tile_built, L, &tmap, &omap, st));
    return CHX_OK;
}

}  // namespace

extern "C" {

const char *chx_version(void) { return "chimex-b200 0.1"; }

const char *chx_last_error(void) { return g_err; }

int chx_plan_create(chx_plan **plan, int E, int F, int T, int TA, int ut, int kernel_batch,
                    int device) {
    clear_error();
    NvtxRange nvtx_("chx_plan_create");
    if (!plan) return fail(CHX_E_INVALID, "plan pointer is NULL");
    *plan = nullptr;
    if (E < 32 || E % 32 != 0)
        return fail(CHX_E_INVALID, "num_elements=%d must be a positive multiple of 32", E);
    if (E > 65536) return fail(CHX_E_UNSUPPORTED, "num_elements=%d exceeds 65536", E);
    if (F < 1) return fail(CHX_E_INVALID, "num_frequencies=%d must be >= 1", F);
    if (T < 1 || T > 16777215)
        return fail(CHX_E_INVALID, "num_timesamples=%d outside [1, 16777215]", T);
    if (TA < 1) return fail(CHX_E_INVALID, "time_accum=%d must be >= 1", TA);
    if (ut != 0 && ut != 1)
        return fail(CHX_E_INVALID, "upper_triangle_convention=%d not in {0,1}", ut);
    if (kernel_batch != 0 && kernel_batch != 1)
        return fail(CHX_E_INVALID, "kernel_batch=%d not in {0,1}", kernel_batch);
    int ndev = 0;
    CHX_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev)
        return fail(CHX_E_INVALID, "device=%d outside [0,%d)", device, ndev);
    DeviceGuard g(device);
    if (!g.ok) return fail(CHX_E_CUDA, "cudaSetDevice(%d) failed", device);
    chx_plan *p = new (std::nothrow) chx_plan();
    if (!p) return fail(CHX_E_NOMEM, "host allocation failed");
    p->E = E;
    p->F = F;
    p->T = T;
    p->TA = TA;
    p->ut = ut;
    p->kernel_batch = kernel_batch;
    p->device = device;
    p->NB1 = E / 32;
    p->NB = num_blocks_of(E);
    p->algo = CHX_ALGO_AUTO;
    p->tsplit = 0;
    p->tile = 0;
    p->d_err = nullptr;
    p->d_chans = nullptr;
    p->d_units = nullptr;
    p->nunits = 0;
    cudaError_t e = cudaDeviceGetAttribute(&p->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(p->d_err, 0, sizeof(int));
    if (e == cudaSuccess) e = build_tc_tables(p);
    if (e != cudaSuccess) {
        free_plan_device(p);
        delete p;
        return cuda_fail(e, "plan device state");
    }
    *plan = p;
    return CHX_OK;
}

int chx_plan_destroy(chx_plan *p) {
    clear_error();
    if (!p) return CHX_OK;
    DeviceGuard g(p->device);
    free_plan_device(p);
    delete p;
    return CHX_OK;
}

int chx_plan_set_option(chx_plan *p, int option, int64_t value) {
    clear_error();
    if (!p) return fail(CHX_E_INVALID, "plan is NULL");
    switch (option) {
    case CHX_OPT_ALGO:
        if (value < CHX_ALGO_AUTO || value > CHX_ALGO_TC)
            return fail(CHX_E_INVALID, "unknown algorithm %lld", (long long)value);
        if (value == CHX_ALGO_TC && !plan_tc_ok(p))
            return fail(CHX_E_UNSUPPORTED, "tensor-core path does not take E=%d T=%d", p->E, p->T);
        p->algo = (int)value;
        return CHX_OK;
    case CHX_OPT_TSPLIT: {
        if (value < 0 || value > 4096) return fail(CHX_E_INVALID, "tsplit %lld", (long long)value);
        p->tsplit = (int)value;
        DeviceGuard g(p->device);
        CHX_CUDA(build_tc_tables(p));
        return CHX_OK;
    }
    case CHX_OPT_TILE: {
        if (value < 0 || value > kTileMax)
            return fail(CHX_E_INVALID,
                        "tile variant %lld (0 auto, 1 one SM, 2 SM pair)",
                        (long long)value);
        p->tile = (int)value;
        DeviceGuard g(p->device);
        CHX_CUDA(build_tc_tables(p));
        return CHX_OK;
    }
    default:
        return fail(CHX_E_INVALID, "unknown option %d", option);
    }
}

int64_t chx_plan_block_words(const chx_plan *p) { return p ? (int64_t)p->F * p->NB * 2048 : -1; }
int64_t chx_plan_input_bytes(const chx_plan *p) {
    return p ? (int64_t)p->T * p->F * p->E : -1;
}
int64_t chx_plan_sum_words(const chx_plan *p) { return p ? (int64_t)p->F * p->E * 2 : -1; }
int64_t chx_plan_triangle_words(const chx_plan *p) {
    return p ? (int64_t)p->F * p->E * (p->E + 1) : -1;
}

// Sample-range splits for a plain-path launch of `units` independent output
// tiles: enough CTAs to fill the SMs several times, never below 1.
static int auto_splits(int64_t units, int T, int sm_count, int min_chunk) {
    int64_t want = (int64_t)sm_count * 4;
    int s = 1;
    while (units * s < want && T / (2 * s) >= min_chunk) s *= 2;
    return s;
}

int chx_correlate(chx_plan *p, const uint8_t *d_packed, int32_t *d_blocks, void *stream,
                  int accumulate) {
    clear_error();
    NvtxRange nvtx_("chx_correlate");
    if (!p || !d_packed || !d_blocks) return fail(CHX_E_INVALID, "NULL argument");
    if (!aligned16(d_packed) || !aligned16(d_blocks))
        return fail(CHX_E_INVALID, "device buffers must be 16-byte aligned");
    DeviceGuard g(p->device);
    cudaStream_t st = (cudaStream_t)stream;
    const bool use_tc =
        (p->algo == CHX_ALGO_TC) || (p->algo == CHX_ALGO_AUTO && plan_tc_ok(p));
    if (use_tc) return run_tc(p, d_packed, d_blocks, MAP_EXACT, accumulate ? 1 : 0, st);
    const int splits =
        p->tsplit ? p->tsplit : auto_splits((int64_t)p->NB * p->F, p->T, p->sm_count, 256);
    int mode;
    if (splits > 1) {
        if (!accumulate)
            CHX_CUDA(cudaMemsetAsync(d_blocks, 0, (size_t)chx_plan_block_words(p) * 4, st));
        mode = 2;
    } else {
        mode = accumulate ? 1 : 0;
    }
    CHX_CUDA(launch_correlate_simt(d_packed, d_blocks, p->E, p->F, p->T, MAP_EXACT, p->ut,
                                   mode, splits, st));
    return CHX_OK;
}

int chx_offset_accumulate(chx_plan *p, const uint8_t *d_packed, uint32_t *d_sums,
                          void *stream, int accumulate) {
    clear_error();
    NvtxRange nvtx_("chx_offset_accumulate");
    if (!p || !d_packed || !d_sums) return fail(CHX_E_INVALID, "NULL argument");
    if (!aligned16(d_packed) || !aligned16(d_sums))
        return fail(CHX_E_INVALID, "device buffers must be 16-byte aligned");
    DeviceGuard g(p->device);
    cudaStream_t st = (cudaStream_t)stream;
    if (!accumulate)
        CHX_CUDA(cudaMemsetAsync(d_sums, 0, (size_t)chx_plan_sum_words(p) * 4, st));
    CHX_CUDA(launch_offset_accumulate(d_packed, d_sums, p->E, p->F, p->T, st));
    return CHX_OK;
}

int chx_preseed(chx_plan *p, const uint32_t *d_sums, int32_t *d_blocks, void *stream) {
    clear_error();
    NvtxRange nvtx_("chx_preseed");
    if (!p || !d_sums || !d_blocks) return fail(CHX_E_INVALID, "NULL argument");
    if (!aligned16(d_sums) || !aligned16(d_blocks))
        return fail(CHX_E_INVALID, "device buffers must be 16-byte aligned");
    DeviceGuard g(p->device);
    CHX_CUDA(launch_preseed(d_sums, d_blocks, p->E, p->F, p->T, p->kernel_batch, p->ut,
                            (cudaStream_t)stream));
    return CHX_OK;
}

int chx_corr_compat(chx_plan *p, const uint8_t *d_packed, int32_t *d_blocks, void *stream) {
    clear_error();
    NvtxRange nvtx_("chx_corr_compat");
    if (!p || !d_packed || !d_blocks) return fail(CHX_E_INVALID, "NULL argument");
    if (!aligned16(d_packed) || !aligned16(d_blocks))
        return fail(CHX_E_INVALID, "device buffers must be 16-byte aligned");
    // The reference kernels' own domain (main_wrapper.c:564-569,
    // pairwise_correlator_UT.cl:82, help text main_wrapper.c:57).
    if (p->T % p->TA != 0)
        return fail(CHX_E_INVALID, "T=%d is not a multiple of time_accum=%d", p->T, p->TA);
    if (p->TA % 8 != 0)
        return fail(CHX_E_INVALID, "time_accum=%d is not a multiple of 8", p->TA);
    if (p->T % 32 != 0) return fail(CHX_E_INVALID, "T=%d is not a multiple of 32", p->T);
    if (p->kernel_batch == CHX_KERNEL_CONFERENCE && p->TA > 291)
        return fail(CHX_E_INVALID, "time_accum=%d > 291 overflows the conference kernel", p->TA);
    if (p->kernel_batch == CHX_KERNEL_PACKED && p->TA > 2272)
        return fail(CHX_E_INVALID, "time_accum=%d > 2272 overflows the packed kernel", p->TA);
    if (p->kernel_batch == CHX_KERNEL_PACKED && p->F != 1)
        return fail(CHX_E_UNSUPPORTED,
                    "the packed reference kernel has no channel index: F must be 1 (F=%d)", p->F);
    DeviceGuard g(p->device);
    cudaStream_t st = (cudaStream_t)stream;
    const int map = p->kernel_batch == CHX_KERNEL_PACKED ? MAP_PACKED : MAP_CONF;
    if (p->algo != CHX_ALGO_SIMT && plan_tc_ok(p))
        return run_tc(p, d_packed, d_blocks, map, 1, st);
    const int splits =
        p->tsplit ? p->tsplit : auto_splits((int64_t)p->NB * p->F, p->T, p->sm_count, 256);
    CHX_CUDA(launch_correlate_simt(d_packed, d_blocks, p->E, p->F, p->T, map, p->ut,
                                   splits > 1 ? 2 : 1, splits, st));
    return CHX_OK;
}

int chx_blocks_to_triangle(chx_plan *p, const int32_t *d_blocks, int32_t *d_tri, void *stream) {
    clear_error();
    NvtxRange nvtx_("chx_blocks_to_triangle");
    if (!p || !d_blocks || !d_tri) return fail(CHX_E_INVALID, "NULL argument");
    if (!aligned16(d_blocks) || !aligned16(d_tri))
        return fail(CHX_E_INVALID, "device buffers must be 16-byte aligned");
    DeviceGuard g(p->device);
    CHX_CUDA(launch_blocks_to_triangle(d_blocks, d_tri, p->E, p->F, (cudaStream_t)stream));
    return CHX_OK;
}

int chx_blocks_to_full(chx_plan *p, const int32_t *d_blocks, int32_t *d_full, void *stream) {
    clear_error();
    NvtxRange nvtx_("chx_blocks_to_full");
    if (!p || !d_blocks || !d_full) return fail(CHX_E_INVALID, "NULL argument");
    if (!aligned16(d_blocks) || !aligned16(d_full))
        return fail(CHX_E_INVALID, "device buffers must be 16-byte aligned");
    DeviceGuard g(p->device);
    CHX_CUDA(launch_blocks_to_full(d_blocks, d_full, p->E, p->F, (cudaStream_t)stream));
    return CHX_OK;
}

int chx_plan_check(chx_plan *p, void *stream) {
    clear_error();
    if (!p) return fail(CHX_E_INVALID, "plan is NULL");
    DeviceGuard g(p->device);
    cudaStream_t st = (cudaStream_t)stream;
    int h = 0;
    CHX_CUDA(cudaMemcpyAsync(&h, p->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CHX_CUDA(cudaStreamSynchronize(st));
    if (h != 0) {
        CHX_CUDA(cudaMemsetAsync(p->d_err, 0, sizeof(int), st));
        CHX_CUDA(cudaStreamSynchronize(st));
        return fail(CHX_E_TIMEOUT, "a bounded device wait gave up (code 0x%x)", h);
    }
    return CHX_OK;
}

}  // extern "C"
