// batch.cu -- batched ragged launch and the tile autotuner.
//
// A batch is many channels with their own element counts, integration lengths
// and integration counts, correlated by one persistent tensor-core launch:
// every (channel, integration, tile pair, sample range) becomes a work unit,
// the units are assigned to the persistent CTAs (or CTA pairs) longest first,
// and the whole launch, with the zeroing of outputs that receive split units,
// is captured once in a CUDA graph per accumulate mode.  Each channel carries
// its own TMA map in the device-side channel table.
//
// The autotuner times the tile variants (one SM, SM pair) and sample splits
// for an (E, T) shape on the current device and caches the fastest; batches
// and AUTO plans consult the cache.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "chimex_internal.h"

namespace chx {
namespace {

struct TuneKey {
    int device, E, T;
    bool operator<(const TuneKey &o) const {
        if (device != o.device) return device < o.device;
        if (E != o.E) return E < o.E;
        return T < o.T;
    }
};
struct TuneVal {
    int tile, split;
    double ms;
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneVal> g_tune;

// Nearest cached entry for (E, T): same E, the closest T within a factor 2.
bool tune_lookup(int device, int E, int T, TuneVal *out) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    bool found = false;
    double best = 1e300;
    for (const auto &kv : g_tune) {
        if (kv.first.device != device || kv.first.E != E) continue;
        const double r = std::abs(std::log((double)kv.first.T / (double)T));
        if (r < best && r <= std::log(2.0)) {
            best = r;
            *out = kv.second;
            found = true;
        }
    }
    return found;
}

}  // namespace

bool tc_tune_lookup(int device, int E, int T, int *tile, int *split) {
    TuneVal tv;
    if (!tune_lookup(device, E, T, &tv)) return false;
    *tile = tv.tile;
    *split = tv.split;
    return true;
}

}  // namespace chx

struct chx_batch {
    int device = 0, ut = 1, n = 0, tile = 0, grid = 0, nunits = 0;
    std::vector<chx_channel_desc> descs;
    chx::ChanDesc *d_chans = nullptr;
    void *d_units = nullptr;  // units then grid + 1 offsets
    std::vector<std::pair<void *, size_t>> zero_regions;  // outputs with split units
    cudaGraph_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    double ops = 0.0;
    int *d_err = nullptr;
};

using namespace chx;

namespace {

void free_batch(chx_batch *b) {
    for (int a = 0; a < 2; a++) {
        if (b->exec[a]) cudaGraphExecDestroy(b->exec[a]);
        if (b->graph[a]) cudaGraphDestroy(b->graph[a]);
        b->exec[a] = nullptr;
        b->graph[a] = nullptr;
    }
    if (b->d_chans) cudaFree(b->d_chans);
    if (b->d_units) cudaFree(b->d_units);
    if (b->d_err) cudaFree(b->d_err);
    b->d_chans = nullptr;
    b->d_units = nullptr;
    b->d_err = nullptr;
}

// Records the batch's work (zeroing + one persistent launch) on `st`.
int record_batch(chx_batch *b, cudaStream_t st, int accumulate) {
    if (!accumulate)
        for (const auto &z : b->zero_regions) CHX_CUDA(cudaMemsetAsync(z.first, 0, z.second, st));
    TcLaunch L;
    L.chans = b->d_chans;
    L.units = (const Unit *)b->d_units;
    L.nunits = b->nunits;
    L.cta_offsets = (const int *)((const char *)b->d_units + (size_t)b->nunits * sizeof(Unit));
    L.out_base = 0;
    L.use_param_map = 0;
    L.map = MAP_EXACT;
    L.ut = b->ut;
    L.accumulate = accumulate;
    L.err = b->d_err;
    L.grid = b->grid;
    CHX_CUDA(tc_tile_launch(b->tile, L, nullptr, nullptr, st));
    return CHX_OK;
}

}  // namespace

extern "C" {

int chx_batch_create(chx_batch **out, int n, const chx_channel_desc *descs, int ut, int device) {
    clear_error();
    NvtxRange nvtx_("chx_batch_create");
    if (!out || !descs || n < 1) return fail(CHX_E_INVALID, "need at least one channel");
    *out = nullptr;
    if (ut != 0 && ut != 1) return fail(CHX_E_INVALID, "upper_triangle_convention=%d", ut);
    for (int c = 0; c < n; c++) {
        const chx_channel_desc &d = descs[c];
        if (d.num_elements < 32 || d.num_elements % 32 || d.num_elements > 65536)
            return fail(CHX_E_INVALID, "channel %d: num_elements=%d", c, d.num_elements);
        if (d.num_timesamples < 1 || d.num_integrations < 1)
            return fail(CHX_E_INVALID, "channel %d: T=%d integrations=%d", c, d.num_timesamples,
                        d.num_integrations);
        if ((int64_t)d.num_timesamples * d.num_integrations > 2147483647LL)
            return fail(CHX_E_INVALID, "channel %d: too many samples", c);
        if (!d.d_packed || !d.d_blocks) return fail(CHX_E_INVALID, "channel %d: NULL buffer", c);
        if (reinterpret_cast<uintptr_t>(d.d_blocks) & 15)
            return fail(CHX_E_INVALID, "channel %d: block buffer must be 16-byte aligned", c);
        if (!tc_out_rows_ok((int64_t)d.num_integrations * num_blocks_of(d.num_elements) * 32))
            return fail(CHX_E_UNSUPPORTED, "channel %d: block buffers too large", c);
        const int64_t stride = d.input_stride ? d.input_stride : d.num_elements;
        if (stride < d.num_elements || stride % 16 || (reinterpret_cast<uintptr_t>(d.d_packed) & 15))
            return fail(CHX_E_INVALID,
                        "channel %d: input stride %lld and address must be 16-byte multiples "
                        "and the stride >= E",
                        c, (long long)stride);
    }
    int ndev = 0;
    CHX_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(CHX_E_INVALID, "device=%d", device);
    DeviceGuard g(device);
    chx_batch *b = new (std::nothrow) chx_batch();
    if (!b) return fail(CHX_E_NOMEM, "host allocation failed");
    b->device = device;
    b->ut = ut;
    b->n = n;
    b->descs.assign(descs, descs + n);

    int sm_count = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) {
        delete b;
        return cuda_fail(e, "device attribute");
    }

    // Tile: the autotuned choice of the costliest channel, else the default.
    int heaviest = 0;
    double heaviest_ops = -1;
    for (int c = 0; c < n; c++) {
        const double E = descs[c].num_elements;
        const double ops = 8.0 * E * (E + 1) / 2 * descs[c].num_timesamples *
                           descs[c].num_integrations;
        b->ops += ops;
        if (ops > heaviest_ops) {
            heaviest_ops = ops;
            heaviest = c;
        }
    }
    TuneVal tv;
    b->tile = tune_lookup(device, descs[heaviest].num_elements, descs[heaviest].num_timesamples, &tv)
                  ? tv.tile
                  : tc_default_tile(descs[heaviest].num_elements);

    // Sample splits: one for every channel, chosen for the whole batch by the
    // makespan estimate (a few long channels are split to fill the GPU, many
    // short integrations are not).  The autotuner's split was timed on a lone
    // channel, where splitting fills idle SMs that a batch already fills, so
    // batches take only its tile.
    const int auto_split = tc_choose_split(b->tile, sm_count, [&](int k, std::vector<Unit> &u) {
        for (int c = 0; c < n; c++)
            for (int i = 0; i < descs[c].num_integrations; i++)
                tc_append_tile_units(b->tile, u, c, descs[c].num_elements,
                                     i * descs[c].num_timesamples,
                                     (i + 1) * descs[c].num_timesamples, k, 0);
    });

    std::vector<ChanDesc> chans(n);
    memset(chans.data(), 0, chans.size() * sizeof(ChanDesc));
    std::vector<Unit> units;
    for (int c = 0; c < n; c++) {
        const chx_channel_desc &d = descs[c];
        const int64_t stride = d.input_stride ? d.input_stride : d.num_elements;
        const int64_t samples = (int64_t)d.num_timesamples * d.num_integrations;
        const int r = tc_encode_map(&chans[c].map, d.d_packed, d.num_elements, 1, samples,
                                    ((int64_t)d.num_elements + 15) / 16 * 16, stride);
        if (r != 0) {
            delete b;
            return fail(CHX_E_CUDA, "channel %d: cuTensorMapEncodeTiled failed (%d)", c, r);
        }
        const int64_t nb_c = num_blocks_of(d.num_elements);
        const int r2 = tc_encode_out_map(&chans[c].omap, d.d_blocks, d.num_integrations * nb_c * 32);
        if (r2 != 0) {
            delete b;
            return fail(CHX_E_CUDA, "channel %d: cuTensorMapEncodeTiled (blocks) failed (%d)", c, r2);
        }
        chans[c].orow = 0;
        chans[c].out = (uint64_t)d.d_blocks;
        chans[c].E = d.num_elements;
        chans[c].nb1 = d.num_elements / 32;
        chans[c].fcoord = 0;
        const int split = auto_split;
        const int64_t nb = num_blocks_of(d.num_elements);
        for (int i = 0; i < d.num_integrations; i++) {
            const size_t before = units.size();
            const int t0 = i * d.num_timesamples, t1 = t0 + d.num_timesamples;
            tc_append_tile_units(b->tile, units, c, d.num_elements, t0, t1, split,
                                 (long long)i * nb * 2048);
            bool any_split = false;
            for (size_t k = before; k < units.size(); k++) any_split |= units[k].split != 0;
            if (any_split)
                b->zero_regions.push_back({d.d_blocks + (size_t)i * nb * 2048, (size_t)nb * 2048 * 4});
        }
    }
    const int slots = tc_tile_slots(b->tile, sm_count);
    b->grid = (int)std::min<size_t>(units.size(), (size_t)std::max(1, slots));
    std::vector<int> offsets;
    tc_schedule(units, b->grid, offsets);
    b->nunits = (int)units.size();

    const size_t ubytes = units.size() * sizeof(Unit);
    e = cudaMalloc(&b->d_chans, chans.size() * sizeof(ChanDesc));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_units, ubytes + offsets.size() * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(b->d_err, 0, sizeof(int));
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_chans, chans.data(), chans.size() * sizeof(ChanDesc),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_units, units.data(), ubytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy((char *)b->d_units + ubytes, offsets.data(), offsets.size() * sizeof(int),
                       cudaMemcpyHostToDevice);
    // Capture the launch once per accumulate mode.
    cudaStream_t cs = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    for (int a = 0; a < 2 && e == cudaSuccess; a++) {
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) break;
        const int rc = record_batch(b, cs, a);
        cudaGraph_t gr = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(cs, &gr);
        if (rc != CHX_OK) {
            if (gr) cudaGraphDestroy(gr);
            cudaStreamDestroy(cs);
            free_batch(b);
            delete b;
            return rc;
        }
        e = e2;
        if (e == cudaSuccess) {
            b->graph[a] = gr;
            e = cudaGraphInstantiate(&b->exec[a], gr, 0);
        }
    }
    if (cs) cudaStreamDestroy(cs);
    if (e != cudaSuccess) {
        free_batch(b);
        delete b;
        return cuda_fail(e, "batch set-up");
    }
    *out = b;
    return CHX_OK;
}

int chx_batch_run(chx_batch *b, void *stream, int accumulate) {
    clear_error();
    NvtxRange nvtx_("chx_batch_run");
    if (!b) return fail(CHX_E_INVALID, "batch is NULL");
    DeviceGuard g(b->device);
    CHX_CUDA(cudaGraphLaunch(b->exec[accumulate ? 1 : 0], (cudaStream_t)stream));
    return CHX_OK;
}

int64_t chx_batch_work_units(const chx_batch *b) { return b ? b->nunits : -1; }

double chx_batch_ops(const chx_batch *b) { return b ? b->ops : -1.0; }

int chx_batch_destroy(chx_batch *b) {
    clear_error();
    if (!b) return CHX_OK;
    DeviceGuard g(b->device);
    free_batch(b);
    delete b;
    return CHX_OK;
}

int chx_batch_check(chx_batch *b, void *stream) {
    clear_error();
    if (!b) return fail(CHX_E_INVALID, "batch is NULL");
    DeviceGuard g(b->device);
    cudaStream_t st = (cudaStream_t)stream;
    int h = 0;
    CHX_CUDA(cudaMemcpyAsync(&h, b->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CHX_CUDA(cudaStreamSynchronize(st));
    if (h) {
        CHX_CUDA(cudaMemsetAsync(b->d_err, 0, sizeof(int), st));
        CHX_CUDA(cudaStreamSynchronize(st));
        return fail(CHX_E_TIMEOUT, "a bounded device wait gave up (code 0x%x)", h);
    }
    return CHX_OK;
}

int chx_autotune(int E, int T, const uint8_t *d_in, int32_t *d_out, void *stream, int *best_tile,
                 int *best_split, double *best_ms) {
    clear_error();
    NvtxRange nvtx_("chx_autotune");
    if (!d_in || !d_out) return fail(CHX_E_INVALID, "NULL scratch buffer");
    int dev = 0;
    CHX_CUDA(cudaGetDevice(&dev));
    cudaStream_t st = (cudaStream_t)stream;
    // Channels timed together: enough for about two waves of SM-pair units,
    // so that the comparison measures each variant's speed per unit rather
    // than how many SMs a lone channel leaves idle (a lone E=2048 channel has
    // 36 SM-pair units for 74 clusters).  The caller's scratch holds one
    // channel; more come from a temporary allocation (at most 64 channels
    // and 2 GiB), without which the lone channel is timed.
    int sm_count = 0;
    CHX_CUDA(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev));
    if (E < 32 || E % 32 != 0 || T < 1) return fail(CHX_E_INVALID, "E=%d T=%d", E, T);
    const int64_t nt2 = ((E + 127) / 128 + 1) / 2;
    const int64_t pair_units = nt2 * (nt2 + 1) / 2;
    const int64_t nb = num_blocks_of(E);
    int64_t F = std::min<int64_t>(64, std::max<int64_t>(1, (sm_count + pair_units - 1) / pair_units));
    while (F > 1 && F * ((int64_t)T * E + nb * 2048 * 4) > (2LL << 30)) F--;
    const uint8_t *in = d_in;
    int32_t *out = d_out;
    void *own_in = nullptr, *own_out = nullptr;
    if (F > 1) {
        if (cudaMalloc(&own_in, (size_t)F * T * E) != cudaSuccess ||
            cudaMalloc(&own_out, (size_t)F * nb * 2048 * 4) != cudaSuccess) {
            cudaGetLastError();  // out of memory: time the lone channel instead
            if (own_in) cudaFree(own_in);
            own_in = own_out = nullptr;
            F = 1;
        } else {
            // The kernels' speed does not depend on the sample values.
            const cudaError_t me = cudaMemsetAsync(own_in, 0x5a, (size_t)F * T * E, st);
            if (me != cudaSuccess) {
                cudaFree(own_in);
                cudaFree(own_out);
                return cuda_fail(me, "autotune scratch");
            }
            in = static_cast<const uint8_t *>(own_in);
            out = static_cast<int32_t *>(own_out);
        }
    }
    chx_plan *p = nullptr;
    int rc = chx_plan_create(&p, E, (int)F, T, T, 1, 0, dev);
    if (rc != CHX_OK) {
        if (own_in) cudaFree(own_in);
        if (own_out) cudaFree(own_out);
        return rc;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t ce = cudaEventCreate(&e0);
    if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
    TuneVal best{0, 1, 1e300};
    const int tiles[2] = {kTile1Sm, kTile2Sm};
    const int splits[3] = {1, 2, 4};
    for (int ti = 0; ti < 2 && ce == cudaSuccess && rc == CHX_OK; ti++) {
        for (int si = 0; si < 3 && rc == CHX_OK; si++) {
            if (splits[si] > 1 && T / splits[si] < 256) continue;
            rc = chx_plan_set_option(p, CHX_OPT_TILE, tiles[ti]);
            if (rc == CHX_OK) rc = chx_plan_set_option(p, CHX_OPT_TSPLIT, splits[si]);
            if (rc != CHX_OK) break;
            for (int w = 0; w < 2 && rc == CHX_OK; w++) rc = chx_correlate(p, in, out, st, 0);
            const int reps = 5;
            ce = cudaEventRecord(e0, st);
            for (int r = 0; r < reps && rc == CHX_OK; r++) rc = chx_correlate(p, in, out, st, 0);
            if (ce == cudaSuccess) ce = cudaEventRecord(e1, st);
            if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
            float ms = 0;
            if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
            if (rc == CHX_OK && ce == cudaSuccess && ms / reps < best.ms)
                best = TuneVal{tiles[ti], splits[si], ms / reps};
        }
    }
    if (rc == CHX_OK && ce == cudaSuccess) rc = chx_plan_check(p, st);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    chx_plan_destroy(p);
    if (own_in) cudaFree(own_in);
    if (own_out) cudaFree(own_out);
    if (rc != CHX_OK) return rc;
    if (ce != cudaSuccess) return cuda_fail(ce, "autotune timing");
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune[TuneKey{dev, E, T}] = best;
    }
    if (best_tile) *best_tile = best.tile;
    if (best_split) *best_split = best.split;
    if (best_ms) *best_ms = best.ms;
    return CHX_OK;
}

}  // extern "C"
