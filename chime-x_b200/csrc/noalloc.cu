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
// The tables are written on the device by a small kernel whose only inputs
// are its launch parameters (the shape, the tile variant and the unit
// classes), so a call reads no host memory after it returns and needs no
// host staging buffer.  The units are those of the plan path's default tile
// variant, sample ranges cut only where int32 exactness requires it, ordered
// by decreasing cost (unit_cost) and dealt round robin to the persistent CTAs.
//
// Limits: at most kNoAllocMaxChannels channels and kNoAllocMaxUnits work
// units per call (for E = 2048 a channel needs 36 SM-pair units, so all 64
// channels fit; E = 4096 needs 136); larger requests are rejected with
// CHX_E_UNSUPPORTED.
//
// Sharing: every call, on every stream, uses the same array and leaves its
// tables there.  Two calls whose kernels overlap on the GPU race on the tables
// and give wrong results: order them (one stream, or events).  The error word
// collects the bounded-wait timeouts of every call until chx_noalloc_check
// reads and clears it.
#include <algorithm>
#include <mutex>

#include "chimex_internal.h"

namespace chx {
namespace {

constexpr int kNoAllocMaxChannels = 64;
constexpr int kNoAllocMaxUnits = 4096;
constexpr int kNoAllocMaxGrid = 1024;
constexpr size_t kOffErr = 0;
constexpr size_t kOffChans = 256;
constexpr size_t kOffUnits = kOffChans + sizeof(ChanDesc) * kNoAllocMaxChannels;
constexpr size_t kOffOffsets = kOffUnits + sizeof(Unit) * kNoAllocMaxUnits;
constexpr size_t kScratchBytes = kOffOffsets + sizeof(int) * (kNoAllocMaxGrid + 1);  // ~162 KiB
static_assert(kOffChans % alignof(ChanDesc) == 0 && kOffUnits % 16 == 0, "table alignment");

// The scratch: error word, channel table, unit table, per-CTA unit offsets.
// Zero-initialised when the library's device code is loaded.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Units of equal cost: `per_chan` units per channel and chunk (all units of
// the SM-pair tile, or the one-SM tile's units with nx x tiles) over the
// sample chunks [chunk0, chunk0 + nchunks) of kUnitMaxSamples samples.
struct UnitClass {
    int count;
    int chunk0, nchunks;
    int nx;  // one-SM tile: 1 or 2 x tiles; SM-pair tile: 2
    int per_chan;
};

struct TableParams {
    int E, F, T;
    int pair;    // 1: SM-pair tile, 0: one-SM tile
    int nt;      // 128-element tiles per channel
    int chunks;  // sample chunks
    int n;       // units
    int grid;    // persistent CTAs (clusters for the SM pair)
    int nclass;
    long long nb;  // blocks per channel
    UnitClass cls[4];  // in decreasing cost
};

// tyx of the k-th unit of one channel among the units of its kind, in the
// order tc_append_pair_units / tc_append_units enumerate them.
__device__ int kth_tyx(const TableParams &P, int nx, int k) {
    if (P.pair) {
        const int nt2 = (P.nt + 1) / 2;
        int ty2 = 0;
        while (ty2 < nt2 - 1 && k >= nt2 - ty2) {
            k -= nt2 - ty2;
            ty2++;
        }
        return ty2 | ((ty2 + k) << 10);
    }
    for (int ty = 0; ty < P.nt; ty++) {
        const int rem = P.nt - ty;  // x tiles at and right of the diagonal
        const int c = nx == 2 ? rem / 2 : rem % 2;
        if (k < c) return ty | ((nx == 2 ? ty + 2 * k : P.nt - 1) << 10) | (nx << 20);
        k -= c;
    }
    return 0;  // not reached for k < per_chan
}

// One thread per unit (and per channel descriptor and CTA offset): writes the
// tables of one call into the scratch array.
__global__ void noalloc_tables_kernel(const TableParams P) {
    unsigned char *scr = g_noalloc_scratch;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    ChanDesc *chans = reinterpret_cast<ChanDesc *>(scr + kOffChans);
    Unit *units = reinterpret_cast<Unit *>(scr + kOffUnits);
    int *offs = reinterpret_cast<int *>(scr + kOffOffsets);
    const int per_cta = P.n / P.grid, extra = P.n % P.grid;
    if (i < P.F) {
        // every launch passes its TMA maps as parameters: the maps stay zero
        int4 *w = reinterpret_cast<int4 *>(chans + i);
        for (int k = 0; k < (int)(sizeof(ChanDesc) / sizeof(int4)); k++)
            w[k] = make_int4(0, 0, 0, 0);
        chans[i].out = (uint64_t)i * (uint64_t)P.nb * 2048u * 4u;
        chans[i].E = P.E;
        chans[i].nb1 = P.E / 32;
        chans[i].fcoord = i;
        chans[i].orow = (int)((long long)i * P.nb * 32);
    }
    if (i <= P.grid) offs[i] = i * per_cta + min(i, extra);
    if (i >= P.n) return;
    int j = i, k = 0;
    while (k < P.nclass - 1 && j >= P.cls[k].count) {
        j -= P.cls[k].count;
        k++;
    }
    const UnitClass &C = P.cls[k];
    const int c = C.chunk0 + j / (P.F * C.per_chan);
    const int r = j % (P.F * C.per_chan);
    Unit u;
    u.chan = r / C.per_chan;
    u.tyx = kth_tyx(P, C.nx, r % C.per_chan);
    u.t0 = c * kUnitMaxSamples;
    u.t1 = min(P.T, u.t0 + kUnitMaxSamples);
    u.out_off = 0;
    u.split = P.chunks > 1 ? 1 : 0;
    u.cost = unit_cost(P.pair != 0, u.t0, u.t1, C.nx);
    // round robin: sorted unit i is the (i / grid)-th unit of CTA i % grid
    const int b = i % P.grid;
    units[b * per_cta + min(b, extra) + i / P.grid] = u;
}

// Device address of the scratch array, looked up once per device and context.
// In host code the symbol itself is only a host-side stand-in, not a device
// address; the lookup must run with the device current.  A device reset
// destroys the context that owned the address, so the cache is keyed on the
// context as well as the ordinal.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
struct AddrCache {
    CUcontext ctx;
    void *addr;
};
AddrCache g_scratch_addr[kMaxDevices] = {};

using CtxGetCurrentFn = CUresult (*)(CUcontext *);

CUcontext current_context() {
    static CtxGetCurrentFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !p)
            return nullptr;
        fn = reinterpret_cast<CtxGetCurrentFn>(p);
    }
    CUcontext c = nullptr;
    return fn(&c) == CUDA_SUCCESS ? c : nullptr;
}

cudaError_t scratch_address(int dev, void **out) {
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mu);
    AddrCache &c = g_scratch_addr[dev];
    const CUcontext ctx = current_context();
    if (!c.addr || !ctx || ctx != c.ctx) {
        void *p = nullptr;
        // loads the library's device code into the context if it is not yet
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        c.addr = p;
        c.ctx = current_context();
    }
    *out = c.addr;
    return cudaSuccess;
}

// The unit classes of a call, in decreasing cost; returns the unit count.
int64_t unit_classes(int E, int F, int T, bool pair, TableParams *P) {
    const int nt = (E + 127) / 128;
    const int chunks = (T + kUnitMaxSamples - 1) / kUnitMaxSamples;
    P->nt = nt;
    P->chunks = chunks;
    P->pair = pair ? 1 : 0;
    P->nclass = 0;
    int64_t per[2];
    int kinds[2], nkinds;
    if (pair) {
        const int nt2 = (nt + 1) / 2;
        per[0] = (int64_t)nt2 * (nt2 + 1) / 2;
        kinds[0] = 2;
        nkinds = 1;
    } else {
        per[0] = per[1] = 0;
        for (int ty = 0; ty < nt; ty++) {
            per[0] += (nt - ty) / 2;  // units with two x tiles
            per[1] += (nt - ty) % 2;  // units with one
        }
        kinds[0] = 2;
        kinds[1] = 1;
        nkinds = 2;
    }
    int64_t total = 0;
    for (int part = 0; part < 2; part++) {  // full chunks, then the last chunk
        const int c0 = part == 0 ? 0 : chunks - 1;
        const int nc = part == 0 ? chunks - 1 : 1;
        if (nc <= 0) continue;
        for (int k = 0; k < nkinds; k++) {
            if (per[k] == 0) continue;
            UnitClass &C = P->cls[P->nclass++];
            const int64_t count = per[k] * F * nc;
            C.count = (int)std::min<int64_t>(count, kNoAllocMaxUnits + 1);
            C.chunk0 = c0;
            C.nchunks = nc;
            C.nx = kinds[k];
            C.per_chan = (int)per[k];
            total += count;
        }
    }
    // decreasing cost (at most four classes: insertion sort, no allocation)
    auto cost = [&](const UnitClass &C) {
        const int t0 = C.chunk0 * kUnitMaxSamples;
        return unit_cost(pair, t0, std::min(T, t0 + kUnitMaxSamples), C.nx);
    };
    for (int a = 1; a < P->nclass; a++)
        for (int b = a; b > 0 && cost(P->cls[b]) > cost(P->cls[b - 1]); b--) {
            const UnitClass t = P->cls[b];
            P->cls[b] = P->cls[b - 1];
            P->cls[b - 1] = t;
        }
    return total;
}

}  // namespace

cudaError_t noalloc_error_word(int **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    void *scratch = nullptr;
    if (e == cudaSuccess) e = scratch_address(dev, &scratch);
    if (e == cudaSuccess)
        *out = reinterpret_cast<int *>(static_cast<unsigned char *>(scratch) + kOffErr);
    return e;
}

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
    const int tile = tc_default_tile(E);
    TableParams P;
    P.E = E;
    P.F = F;
    P.T = T;
    P.nb = num_blocks_of(E);
    const int64_t nunits = unit_classes(E, F, T, tile == kTile2Sm, &P);
    if (nunits > kNoAllocMaxUnits)
        return fail(CHX_E_UNSUPPORTED,
                    "no-allocation entry point takes at most %d work units; E=%d F=%d T=%d needs "
                    "%lld",
                    kNoAllocMaxUnits, E, F, T, (long long)nunits);
    P.n = (int)nunits;

    int dev = 0;
    CHX_CUDA(cudaGetDevice(&dev));
    void *scratch = nullptr;
    CHX_CUDA(scratch_address(dev, &scratch));
    int sm_count = 0;
    CHX_CUDA(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev));
    P.grid = std::min(std::min(P.n, tc_tile_slots(tile, sm_count)), kNoAllocMaxGrid);

    cudaStream_t st = (cudaStream_t)stream;
    const int threads = std::max(std::max(P.n, P.grid + 1), F);
    noalloc_tables_kernel<<<(threads + 255) / 256, 256, 0, st>>>(P);
    CHX_CUDA(cudaGetLastError());
    if (P.chunks > 1 && !accumulate)
        CHX_CUDA(cudaMemsetAsync(d_blocks, 0, (size_t)F * P.nb * 2048 * 4, st));

    CUtensorMap tmap, omap;
    int r = tc_encode_map(&tmap, d_packed, E, F, T, E, (int64_t)F * E);
    if (r != 0) return fail(CHX_E_CUDA, "cuTensorMapEncodeTiled failed (%d)", r);
    r = tc_encode_out_map(&omap, d_blocks, (int64_t)F * P.nb * 32);
    if (r != 0) return fail(CHX_E_CUDA, "cuTensorMapEncodeTiled (blocks) failed (%d)", r);
    unsigned char *dscr = static_cast<unsigned char *>(scratch);
    TcLaunch L;
    L.chans = reinterpret_cast<const ChanDesc *>(dscr + kOffChans);
    L.units = reinterpret_cast<const Unit *>(dscr + kOffUnits);
    L.nunits = P.n;
    L.cta_offsets = reinterpret_cast<const int *>(dscr + kOffOffsets);
    L.out_base = (uint64_t)d_blocks;
    L.use_param_map = 1;
    L.map = MAP_EXACT;
    L.ut = upper_triangle_convention;
    L.accumulate = accumulate ? 1 : 0;
    L.err = reinterpret_cast<int *>(dscr + kOffErr);
    L.grid = P.grid;
    CHX_CUDA(tc_tile_launch(tile, L, &tmap, &omap, st));
    return CHX_OK;
}

extern "C" int chx_noalloc_check(void *stream) {
    clear_error();
    int *err = nullptr;
    CHX_CUDA(noalloc_error_word(&err));
    cudaStream_t st = (cudaStream_t)stream;
    int h = 0;
    CHX_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CHX_CUDA(cudaStreamSynchronize(st));
    if (h != 0) {
        CHX_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
        CHX_CUDA(cudaStreamSynchronize(st));
        return fail(CHX_E_TIMEOUT, "a bounded device wait gave up (code 0x%x)", h);
    }
    return CHX_OK;
}
