// noalloc.cu -- chx_correlate_noalloc: the fused tensor-core correlator for
// callers that must not allocate memory.
//
// Who needs it.  A real-time X-engine process reserves all of its device
// memory up front (input rings, resident accumulators) and then runs its
// per-frame loop for hours.  In that loop cudaMalloc/cudaFree are off limits:
// they can implicitly synchronise the whole device (stalling the copy and
// correlation streams that keep up with the telescope), they can fail once
// the pre-reserved pools have taken the memory, and host frameworks that own
// the device allocator (a caching allocator, an embedding runtime) forbid
// side allocations behind their back.  The plan-based chx_correlate needs a
// plan, and creating a plan allocates its work tables and error word.  This
// entry point needs no plan and allocates nothing: the kernel's scratch (the
// channel table, the work-unit table and the error word) lives in one
// file-scope __device__ array that every GPU loading the library holds until
// the process exits.
//
// Limits: at most kNoAllocMaxChannels channels and kNoAllocMaxUnits work
// units per call (for E = 2048 a channel needs 36 SM-pair units, so all 64
// channels fit; E = 4096 needs 136); larger requests are rejected with
// CHX_E_UNSUPPORTED.  The tile variant follows the plan path's default rule
// (SM pair for an even number of 128-element tiles); sample ranges are cut
// only where int32 exactness requires it.
//
// Sharing: every call, on every stream, uses the same array and leaves its
// contents there.  Two calls whose kernels overlap on the GPU race on the
// tables and give wrong results: order them (one stream, or events).
#include <algorithm>
#include <mutex>

#include "chimex_internal.h"

namespace chx {
namespace {

constexpr int kNoAllocMaxChannels = 64;
constexpr int kNoAllocMaxUnits = 4096;
constexpr size_t kOffErr = 0;
constexpr size_t kOffChans = 256;
constexpr size_t kOffUnits = kOffChans + sizeof(ChanDesc) * kNoAllocMaxChannels;
constexpr size_t kOffOffsets = kOffUnits + sizeof(Unit) * kNoAllocMaxUnits;
constexpr int kNoAllocMaxGrid = 1024;
constexpr size_t kScratchBytes = kOffOffsets + sizeof(int) * (kNoAllocMaxGrid + 1);  // ~162 KiB

// The scratch: error word, channel table, unit table.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch_addr[kMaxDevices] = {};  // device address of g_noalloc_scratch
// Host staging for the tables (copied to the device every call) and for the
// largest-first unit order before it is dealt to the CTAs.
alignas(64) unsigned char g_host_tables[kScratchBytes];
Unit g_host_sorted[kNoAllocMaxUnits];

// Device address of the scratch array on the current device, looked up once
// per device.  In host code the symbol itself is only a host-side stand-in.
cudaError_t scratch_address(int dev, void **out) {
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

}  // namespace
}  // namespace chx

using namespace chx;

extern "C" int chx_correlate_noalloc(const uint8_t *d_packed, int32_t *d_blocks, int E, int F,
                                     int T, int upper_triangle_convention, int accumulate,
                                     void *stream) {
    clear_error();
    if (!d_packed || !d_blocks) return fail(CHX_E_INVALID, "NULL argument");
    if (E < 32 || E % 32 != 0 || E > 65536)
        return fail(CHX_E_INVALID, "num_elements=%d must be a multiple of 32 in [32, 65536]", E);
    if (F < 1) return fail(CHX_E_INVALID, "num_frequencies=%d must be >= 1", F);
    if (T < 1 || T > 16777215)
        return fail(CHX_E_INVALID, "num_timesamples=%d outside [1, 16777215]", T);
    if (upper_triangle_convention != 0 && upper_triangle_convention != 1)
        return fail(CHX_E_INVALID, "upper_triangle_convention=%d not in {0,1}",
                    upper_triangle_convention);
    if ((reinterpret_cast<uintptr_t>(d_packed) & 15) != 0)
        return fail(CHX_E_INVALID, "packed input must be 16-byte aligned for TMA");
    if ((reinterpret_cast<uintptr_t>(d_blocks) & 15) != 0)
        return fail(CHX_E_INVALID, "block buffer must be 16-byte aligned for TMA");
    if (F > kNoAllocMaxChannels)
        return fail(CHX_E_UNSUPPORTED, "no-allocation entry point takes at most %d channels (F=%d)",
                    kNoAllocMaxChannels, F);
    // Work units of the same shape as the plan-based path's default tile:
    // SM pair: 256-element y and x tile pairs on and above the diagonal;
    // one SM: each 128-element y tile against 256-element x ranges; sample
    // ranges of at most kUnitMaxSamples.
    const int tile = tc_default_tile(E);
    const int nt = (E + 127) / 128, nt2 = (nt + 1) / 2;
    const int chunks = (T + kUnitMaxSamples - 1) / kUnitMaxSamples;
    int64_t per_chan = 0;
    if (tile == kTile2Sm)
        per_chan = (int64_t)nt2 * (nt2 + 1) / 2;
    else
        for (int ty = 0; ty < nt; ty++) per_chan += (nt - ty + 1) / 2;
    const int64_t nunits = per_chan * chunks * F;
    if (nunits > kNoAllocMaxUnits)
        return fail(CHX_E_UNSUPPORTED,
                    "no-allocation entry point takes at most %d work units; E=%d F=%d T=%d needs "
                    "%lld",
                    kNoAllocMaxUnits, E, F, T, (long long)nunits);

    std::lock_guard<std::mutex> lock(g_mu);
    int dev = 0;
    CHX_CUDA(cudaGetDevice(&dev));
    void *scratch = nullptr;
    CHX_CUDA(scratch_address(dev, &scratch));

    const int64_t nb = num_blocks_of(E);
    ChanDesc *chans = reinterpret_cast<ChanDesc *>(g_host_tables + kOffChans);
    memset(chans, 0, sizeof(ChanDesc) * F);
    for (int f = 0; f < F; f++) {
        chans[f].out = (uint64_t)f * (uint64_t)nb * 2048u * 4u;
        chans[f].E = E;
        chans[f].nb1 = E / 32;
        chans[f].fcoord = f;
        chans[f].orow = (int)((int64_t)f * nb * 32);
    }
    Unit *units = g_host_sorted;
    int n = 0;
    auto add_unit = [&](int f, int tyx, int c, int cost_per_stage) {
        Unit &u = units[n++];
        u.chan = f;
        u.tyx = tyx;
        u.t0 = c * kUnitMaxSamples;
        u.t1 = std::min(T, u.t0 + kUnitMaxSamples);
        u.out_off = 0;
        u.split = chunks > 1 ? 1 : 0;
        u.cost = ((u.t1 - u.t0 + 31) / 32) * cost_per_stage;
    };
    for (int f = 0; f < F; f++) {
        if (tile == kTile2Sm) {
            for (int ty2 = 0; ty2 < nt2; ty2++)
                for (int tx2 = ty2; tx2 < nt2; tx2++)
                    for (int c = 0; c < chunks; c++) add_unit(f, ty2 | (tx2 << 10), c, 1);
        } else {
            for (int ty = 0; ty < nt; ty++)
                for (int x0 = ty; x0 < nt; x0 += 2) {
                    const int nx = std::min(2, nt - x0);
                    for (int c = 0; c < chunks; c++)
                        add_unit(f, ty | (x0 << 10) | (nx << 20), c, 2 * nx + 1);
                }
        }
    }
    // Largest first, sorted in place (std::sort does not allocate), then dealt
    // round robin: CTA b takes sorted units b, b + grid, ... stored contiguously.
    std::sort(units, units + n, [](const Unit &a, const Unit &b) { return a.cost > b.cost; });
    int sm_count = 0;
    CHX_CUDA(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev));
    const int grid = std::min(std::min(n, tc_tile_slots(tile, sm_count)), kNoAllocMaxGrid);
    Unit *dealt = reinterpret_cast<Unit *>(g_host_tables + kOffUnits);
    int *offsets = reinterpret_cast<int *>(g_host_tables + kOffOffsets);
    int k = 0;
    for (int b = 0; b < grid; b++) {
        offsets[b] = k;
        for (int i = b; i < n; i += grid) dealt[k++] = units[i];
    }
    offsets[grid] = k;

    cudaStream_t st = (cudaStream_t)stream;
    unsigned char *dscr = static_cast<unsigned char *>(scratch);
    // The error word starts at zero for this call; the tables are replaced.
    CHX_CUDA(cudaMemsetAsync(dscr + kOffErr, 0, sizeof(int), st));
    CHX_CUDA(cudaMemcpyAsync(dscr + kOffChans, chans, sizeof(ChanDesc) * F,
                             cudaMemcpyHostToDevice, st));
    CHX_CUDA(cudaMemcpyAsync(dscr + kOffUnits, dealt, sizeof(Unit) * n, cudaMemcpyHostToDevice,
                             st));
    CHX_CUDA(cudaMemcpyAsync(dscr + kOffOffsets, offsets, sizeof(int) * (grid + 1),
                             cudaMemcpyHostToDevice, st));
    if (chunks > 1 && !accumulate)
        CHX_CUDA(cudaMemsetAsync(d_blocks, 0, (size_t)F * nb * 2048 * 4, st));

    CUtensorMap tmap, omap;
    int r = tc_encode_map(&tmap, d_packed, E, F, T, E, (int64_t)F * E);
    if (r != 0) return fail(CHX_E_CUDA, "cuTensorMapEncodeTiled failed (%d)", r);
    r = tc_encode_out_map(&omap, d_blocks, (int64_t)F * nb * 32);
    if (r != 0) return fail(CHX_E_CUDA, "cuTensorMapEncodeTiled (blocks) failed (%d)", r);
    TcLaunch L;
    L.chans = reinterpret_cast<const ChanDesc *>(dscr + kOffChans);
    L.units = reinterpret_cast<const Unit *>(dscr + kOffUnits);
    L.nunits = n;
    L.cta_offsets = reinterpret_cast<const int *>(dscr + kOffOffsets);
    L.out_base = (uint64_t)d_blocks;
    L.use_param_map = 1;
    L.map = MAP_EXACT;
    L.ut = upper_triangle_convention;
    L.accumulate = accumulate ? 1 : 0;
    L.err = reinterpret_cast<int *>(dscr + kOffErr);
    L.grid = grid;
    CHX_CUDA(tc_tile_launch(tile, L, &tmap, &omap, st));
    return CHX_OK;
}
