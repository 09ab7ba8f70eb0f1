// stream.cu -- streaming correlation: frames of samples arrive per channel,
// integrations of time_accum samples are dumped as they complete.
//
// Memory per admitted channel (allocated at admission, resident until the
// stream is destroyed): an input ring of two integrations (2 * TA * E bytes)
// and two block buffers (2 * NB * 8 KiB), so one integration can be correlated
// and read while the next fills.  A channel is admitted only when these fit
// the HBM budget.
//
// Each submit appends one frame per listed channel to its ring (in place when
// the caller wrote it into the slot returned by chx_stream_frame_slot).  The
// channels whose integration completes are correlated by one persistent
// tensor-core launch over all their work units (per tile variant: each
// channel takes the plan path's default, the SM-pair kernel from E > 128 up
// and the one-SM kernel below): the integration's samples
// accumulate in TMEM and each dump buffer is written once, so the resident
// state never travels through HBM per frame.  An event recorded after each
// launch is waited for by the stream's completion thread, which records, per
// integration, the latency from its last frame's arrival to the moment the
// completed dump is visible to the host (the compute stream itself never waits
// on the host).
#include <time.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "chimex_internal.h"

namespace chx {
namespace {

int64_t now_ns() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (int64_t)ts.tv_sec * 1000000000LL + ts.tv_nsec;
}

struct StreamChan {
    int E = 0, TA = 0;
    int64_t NB = 0;
    uint8_t *ring = nullptr;     // [2][TA][E]
    int32_t *dumps = nullptr;    // [2][NB][2048]
    std::vector<Unit> units[2];  // work of ring half h -> dump h
    bool pair = true;            // units for the SM-pair kernel (else the one-SM kernel)
    int half = 0;                // half being filled
    int filled = 0;              // samples in that half
    int64_t seq = 0;             // integrations completed (dispatched)
    int64_t last_arrival = 0;
    // published by the completion thread
    int64_t done_seq = -1;
    int done_half = 0;
};

// One launch's unit table: pinned host staging, its device copy, and an event
// recorded after the launch that reads it.
struct Slot {
    void *host = nullptr;
    void *dev = nullptr;
    cudaEvent_t done = nullptr;
};
constexpr int kSlots = 8;

// One frame copied into a ring slot (device addresses, 16-byte aligned, bytes
// a multiple of 16).
struct FrameCopy {
    const uint8_t *src;
    uint8_t *dst;
    int64_t bytes;
};

// All frame copies of one submit in one launch: block y = copy, blocks x
// stride over its 16-byte words.
__global__ void frame_copy_kernel(const FrameCopy *copies) {
    const FrameCopy c = copies[blockIdx.y];
    const int64_t words = c.bytes >> 4;
    const uint4 *src = reinterpret_cast<const uint4 *>(c.src);
    uint4 *dst = reinterpret_cast<uint4 *>(c.dst);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words;
         i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = __ldg(src + i);
}

cudaError_t launch_frame_copies(const FrameCopy *d_copies, int n, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    if (n > 65535) return cudaErrorInvalidValue;
    frame_copy_kernel<<<dim3(8, n), 256, 0, st>>>(d_copies);
    return cudaGetLastError();
}

// The integrations one launch completes, and the event recorded after it.
struct Pending {
    struct Item {
        int chan, half;
        int64_t seq, arrival;
    };
    std::vector<Item> items;
    cudaEvent_t ev = nullptr;
};

}  // namespace
}  // namespace chx

using namespace chx;

struct chx_stream {
    int device = 0, max_channels = 0, frame_len = 0, ut = 1, tile = kTile2Sm, sm_count = 0;
    int64_t budget = 0, resident = 0;
    std::vector<StreamChan> chans;
    ChanDesc *d_chans = nullptr;
    std::vector<ChanDesc> h_chans;
    Slot slots[kSlots];
    size_t slot_cap = 0;  // bytes per slot: units, offsets, frame copies
    int next_slot = 0;
    int *d_err = nullptr;
    int64_t frames = 0, dumps = 0;
    std::mutex mu;  // guards latencies, dumps, done_* fields, queue and spare
    std::condition_variable cv;       // new launch queued, or stop
    std::condition_variable cv_done;  // a launch was published
    std::vector<double> latencies_ms;
    std::deque<Pending *> queue;   // launches in submission order
    std::vector<Pending *> spare;  // completed records for reuse
    std::thread poller;
    bool stop = false;
};

namespace {

// Completion thread: waits (polling with short sleeps, not spinning) for each
// launch in order and publishes its dumps with their latency.
void poll_loop(chx_stream *s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        s->cv.wait(lk, [s] { return s->stop || !s->queue.empty(); });
        if (s->queue.empty()) break;  // stopping with nothing left
        Pending *p = s->queue.front();
        lk.unlock();
        // Poll the event with 20 us sleeps in between: the thread takes a few
        // percent of a host core instead of spinning on one, and sees the
        // completion within ~20-70 us.  (A blocking-sync event waited on with
        // cudaEventSynchronize measured 0.96 ms p50 frame-to-dump latency on
        // B200, against 0.65 ms for polling: the wake-up comes late.)
        cudaError_t q;
        while ((q = cudaEventQuery(p->ev)) == cudaErrorNotReady) {
            timespec ts{0, 20000};
            nanosleep(&ts, nullptr);
        }
        const int64_t t = now_ns();
        lk.lock();
        s->queue.pop_front();
        if (q == cudaSuccess) {
            for (const auto &it : p->items) {
                s->latencies_ms.push_back((double)(t - it.arrival) * 1e-6);
                StreamChan &c = s->chans[it.chan];
                if (it.seq > c.done_seq) {
                    c.done_seq = it.seq;
                    c.done_half = it.half;
                }
                s->dumps++;
            }
        }
        p->items.clear();
        s->spare.push_back(p);
        s->cv_done.notify_all();
    }
}

// Waits until the completion thread has published every launch queued so far.
bool wait_published(chx_stream *s, int64_t timeout_ms) {
    std::unique_lock<std::mutex> lk(s->mu);
    return s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms),
                               [s] { return s->queue.empty(); });
}

void stop_poller(chx_stream *s) {
    if (!s->poller.joinable()) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    s->poller.join();
}

void free_stream(chx_stream *s) {
    for (auto &c : s->chans) {
        if (c.ring) cudaFree(c.ring);
        if (c.dumps) cudaFree(c.dumps);
    }
    if (s->d_chans) cudaFree(s->d_chans);
    for (auto &sl : s->slots) {
        if (sl.dev) cudaFree(sl.dev);
        if (sl.host) cudaFreeHost(sl.host);
        if (sl.done) cudaEventDestroy(sl.done);
        sl = Slot();
    }
    if (s->d_err) cudaFree(s->d_err);
    for (Pending *p : s->queue) {
        if (p->ev) cudaEventDestroy(p->ev);
        delete p;
    }
    for (Pending *p : s->spare) {
        if (p->ev) cudaEventDestroy(p->ev);
        delete p;
    }
    s->queue.clear();
    s->spare.clear();
}

}  // namespace

extern "C" {

int chx_stream_create(chx_stream **out, int max_channels, int frame_len, int ut, int64_t budget,
                      int device) {
    clear_error();
    if (!out) return fail(CHX_E_INVALID, "NULL output");
    *out = nullptr;
    if (max_channels < 1 || max_channels > 65536)
        return fail(CHX_E_INVALID, "max_channels=%d", max_channels);
    if (frame_len < 1 || frame_len % 32) return fail(CHX_E_INVALID, "frame_len=%d must be a multiple of 32", frame_len);
    if (ut != 0 && ut != 1) return fail(CHX_E_INVALID, "upper_triangle_convention=%d", ut);
    int ndev = 0;
    CHX_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(CHX_E_INVALID, "device=%d", device);
    DeviceGuard g(device);
    chx_stream *s = new (std::nothrow) chx_stream();
    if (!s) return fail(CHX_E_NOMEM, "host allocation failed");
    s->device = device;
    s->max_channels = max_channels;
    s->frame_len = frame_len;
    s->ut = ut;
    s->budget = budget;
    s->chans.reserve(max_channels);
    s->h_chans.resize(max_channels);
    memset(s->h_chans.data(), 0, s->h_chans.size() * sizeof(ChanDesc));
    cudaError_t e = cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_chans, (size_t)max_channels * sizeof(ChanDesc));
    if (e == cudaSuccess) e = cudaMalloc(&s->d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(s->d_err, 0, sizeof(int));
    for (int k = 0; k < kSlots && e == cudaSuccess; k++)
        e = cudaEventCreateWithFlags(&s->slots[k].done, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        free_stream(s);
        delete s;
        return cuda_fail(e, "stream set-up");
    }
    s->resident = (int64_t)max_channels * sizeof(ChanDesc);
    try {
        s->poller = std::thread(poll_loop, s);
    } catch (...) {
        free_stream(s);
        delete s;
        return fail(CHX_E_NOMEM, "cannot start the completion thread");
    }
    *out = s;
    return CHX_OK;
}

int chx_stream_admit(chx_stream *s, int E, int TA, int *channel_id) {
    clear_error();
    NvtxRange nvtx_("chx_stream_admit");
    if (!s || !channel_id) return fail(CHX_E_INVALID, "NULL argument");
    if ((int)s->chans.size() >= s->max_channels)
        return fail(CHX_E_ADMISSION, "stream already holds %d channels", s->max_channels);
    if (E < 32 || E % 32 || E > 65536) return fail(CHX_E_INVALID, "num_elements=%d", E);
    if (TA < s->frame_len || TA % s->frame_len)
        return fail(CHX_E_INVALID, "time_accum=%d must be a multiple of frame_len=%d", TA,
                    s->frame_len);
    if (TA > kUnitMaxSamples)
        return fail(CHX_E_UNSUPPORTED, "time_accum=%d above %d samples", TA, kUnitMaxSamples);
    DeviceGuard g(s->device);
    const int64_t NB = num_blocks_of(E);
    const int64_t ring_bytes = 2LL * TA * E;
    const int64_t dump_bytes = 2LL * NB * 2048 * 4;
    // units: both halves of this channel
    std::vector<Unit> u0, u1;
    const int cid = (int)s->chans.size();
    // The tile variant the plain path would choose for this E.
    const bool pair = tc_default_tile(E) == kTile2Sm;
    if (pair) {
        tc_append_pair_units(u0, cid, E, 0, TA, 1, 0);
        tc_append_pair_units(u1, cid, E, TA, 2 * TA, 1, NB * 2048);
    } else {
        tc_append_units(u0, cid, E, 0, TA, 1, 0);
        tc_append_units(u1, cid, E, TA, 2 * TA, 1, NB * 2048);
    }
    const int64_t need = ring_bytes + dump_bytes;
    if (s->budget > 0) {
        if (s->resident + need > s->budget)
            return fail(CHX_E_ADMISSION, "channel needs %lld bytes; %lld of %lld in use",
                        (long long)need, (long long)s->resident, (long long)s->budget);
    } else {
        size_t fr = 0, tot = 0;
        CHX_CUDA(cudaMemGetInfo(&fr, &tot));
        const int64_t headroom = 2LL << 30;
        if ((int64_t)fr < need + headroom)
            return fail(CHX_E_ADMISSION, "channel needs %lld bytes; %lld free", (long long)need,
                        (long long)fr);
    }
    StreamChan c;
    c.E = E;
    c.TA = TA;
    c.NB = NB;
    cudaError_t e = cudaMalloc(&c.ring, ring_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&c.dumps, dump_bytes);
    if (e == cudaSuccess) e = cudaMemset(c.dumps, 0, dump_bytes);
    if (e != cudaSuccess) {
        if (c.ring) cudaFree(c.ring);
        if (c.dumps) cudaFree(c.dumps);
        cudaGetLastError();
        return fail(CHX_E_ADMISSION, "allocation for the channel failed: %s", cudaGetErrorString(e));
    }
    ChanDesc &d = s->h_chans[cid];
    const int r = tc_encode_map(&d.map, c.ring, E, 1, 2LL * TA, E, E);
    if (r != 0) {
        cudaFree(c.ring);
        cudaFree(c.dumps);
        return fail(CHX_E_CUDA, "cuTensorMapEncodeTiled failed (%d)", r);
    }
    const int r2 = tc_encode_out_map(&d.omap, c.dumps, 2 * NB * 32);
    if (r2 != 0) {
        cudaFree(c.ring);
        cudaFree(c.dumps);
        return fail(CHX_E_CUDA, "cuTensorMapEncodeTiled (dumps) failed (%d)", r2);
    }
    d.orow = 0;
    d.out = (uint64_t)c.dumps;
    d.E = E;
    d.nb1 = E / 32;
    d.fcoord = 0;
    CHX_CUDA(cudaMemcpy(s->d_chans + cid, &d, sizeof(ChanDesc), cudaMemcpyHostToDevice));
    c.units[0] = std::move(u0);
    c.units[1] = std::move(u1);
    c.pair = pair;
    // Grow the per-launch unit tables to hold every channel completing at
    // once.  Growing waits for all launches that read the old tables.
    size_t total_units = c.units[0].size();
    for (const auto &x : s->chans) total_units += x.units[0].size();
    const size_t need_bytes = total_units * sizeof(Unit) +
                              2 * ((size_t)(s->sm_count + 1) * sizeof(int) + 16) +
                              (size_t)s->max_channels * sizeof(FrameCopy);
    if (need_bytes > s->slot_cap) {
        const size_t cap = std::max(need_bytes, s->slot_cap * 2);
        e = cudaDeviceSynchronize();
        for (int k = 0; k < kSlots && e == cudaSuccess; k++) {
            Slot &sl = s->slots[k];
            if (sl.dev) cudaFree(sl.dev);
            if (sl.host) cudaFreeHost(sl.host);
            sl.dev = sl.host = nullptr;
            e = cudaMalloc(&sl.dev, cap);
            if (e == cudaSuccess) e = cudaMallocHost(&sl.host, cap);
        }
        if (e != cudaSuccess) {
            cudaFree(c.ring);
            cudaFree(c.dumps);
            s->slot_cap = 0;  // the next admission reallocates every slot
            return cuda_fail(e, "unit table growth");
        }
        s->slot_cap = cap;
    }
    s->resident += need;
    s->chans.push_back(std::move(c));
    *channel_id = cid;
    return CHX_OK;
}

int chx_stream_frame_slot(chx_stream *s, int channel_id, uint8_t **d_slot) {
    clear_error();
    if (!s || !d_slot || channel_id < 0 || channel_id >= (int)s->chans.size())
        return fail(CHX_E_INVALID, "bad channel");
    StreamChan &c = s->chans[channel_id];
    *d_slot = c.ring + ((int64_t)c.half * c.TA + c.filled) * c.E;
    return CHX_OK;
}

int chx_stream_submit(chx_stream *s, int n, const int *ids, const uint8_t *const *d_frames,
                      const int64_t *arrival_ns, void *stream) {
    clear_error();
    NvtxRange nvtx_("chx_stream_submit");
    if (!s || n < 0 || (n > 0 && !ids)) return fail(CHX_E_INVALID, "NULL argument");
    // Validate everything before any channel state moves.
    for (int i = 0; i < n; i++) {
        if (ids[i] < 0 || ids[i] >= (int)s->chans.size())
            return fail(CHX_E_INVALID, "channel id %d", ids[i]);
        if (d_frames && d_frames[i] && (reinterpret_cast<uintptr_t>(d_frames[i]) & 15))
            return fail(CHX_E_INVALID, "frame %d is not 16-byte aligned", i);
    }
    DeviceGuard g(s->device);
    cudaStream_t st = (cudaStream_t)stream;
    Pending *pend = nullptr;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (!s->spare.empty()) {
            pend = s->spare.back();
            s->spare.pop_back();
        }
    }
    if (!pend) {
        pend = new (std::nothrow) Pending();
        if (!pend) return fail(CHX_E_NOMEM, "host allocation failed");
        const cudaError_t e = cudaEventCreateWithFlags(&pend->ev, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            delete pend;
            return cuda_fail(e, "completion event");
        }
    }
    // Returns an unused record to the spare list.
    auto drop = [s](Pending *p) {
        p->items.clear();
        std::lock_guard<std::mutex> lock(s->mu);
        s->spare.push_back(p);
    };
    std::vector<Unit> units, units1;  // SM-pair and one-SM kernel work
    std::vector<FrameCopy> copies;
    for (int i = 0; i < n; i++) {
        const int id = ids[i];
        StreamChan &c = s->chans[id];
        uint8_t *slot = c.ring + ((int64_t)c.half * c.TA + c.filled) * c.E;
        const uint8_t *src = d_frames ? d_frames[i] : nullptr;
        if (src && src != slot) copies.push_back({src, slot, (int64_t)s->frame_len * c.E});
        c.filled += s->frame_len;
        c.last_arrival = arrival_ns ? arrival_ns[i] : now_ns();
        s->frames++;
        if (c.filled == c.TA) {
            std::vector<Unit> &dst = c.pair ? units : units1;
            dst.insert(dst.end(), c.units[c.half].begin(), c.units[c.half].end());
            pend->items.push_back({id, c.half, c.seq, c.last_arrival});
            c.seq++;
            c.half ^= 1;
            c.filled = 0;
        }
    }
    if (units.empty() && units1.empty() && copies.empty()) {
        drop(pend);
        return CHX_OK;
    }
    // Each kernel's units go to its own persistent grid (clusters of two CTAs
    // for the SM-pair kernel, single CTAs for the other).
    const int grid = (int)std::max<size_t>(
        1, std::min<size_t>(units.size(), (size_t)std::max(1, s->sm_count / 2)));
    const int grid1 =
        (int)std::max<size_t>(1, std::min<size_t>(units1.size(), (size_t)std::max(1, s->sm_count)));
    std::vector<int> offsets, offsets1;
    if (!units.empty()) tc_schedule(units, grid, offsets);
    if (!units1.empty()) tc_schedule(units1, grid1, offsets1);
    // Slot table: pair units and their offsets, one-SM units and theirs, then
    // the frame copies; each part 16-byte aligned.
    auto up16 = [](size_t x) { return (x + 15) / 16 * 16; };
    const size_t ub = units.size() * sizeof(Unit);
    const size_t u1b0 = up16(ub + offsets.size() * sizeof(int));
    const size_t u1b = units1.size() * sizeof(Unit);
    const size_t cb0 = up16(u1b0 + u1b + offsets1.size() * sizeof(int));
    const size_t tb = cb0 + copies.size() * sizeof(FrameCopy);
    if (tb > s->slot_cap) {
        drop(pend);
        return fail(CHX_E_INVALID, "unit table overflow");
    }
    // Reuse the oldest slot once the launch that read it has finished.
    Slot &sl = s->slots[s->next_slot];
    s->next_slot = (s->next_slot + 1) % kSlots;
    cudaError_t e = cudaEventSynchronize(sl.done);
    if (e == cudaSuccess) {
        char *h = static_cast<char *>(sl.host);
        memcpy(h, units.data(), ub);
        memcpy(h + ub, offsets.data(), offsets.size() * sizeof(int));
        memcpy(h + u1b0, units1.data(), u1b);
        memcpy(h + u1b0 + u1b, offsets1.data(), offsets1.size() * sizeof(int));
        memcpy(h + cb0, copies.data(), copies.size() * sizeof(FrameCopy));
        e = cudaMemcpyAsync(sl.dev, sl.host, tb, cudaMemcpyHostToDevice, st);
    }
    if (e == cudaSuccess && !copies.empty())
        e = launch_frame_copies((const FrameCopy *)((const char *)sl.dev + cb0), (int)copies.size(),
                                st);
    TcLaunch L;
    L.chans = s->d_chans;
    L.out_base = 0;
    L.use_param_map = 0;
    L.map = MAP_EXACT;
    L.ut = s->ut;
    L.accumulate = 0;
    L.err = s->d_err;
    if (e == cudaSuccess && !units.empty()) {
        L.units = (const Unit *)sl.dev;
        L.nunits = (int)units.size();
        L.cta_offsets = (const int *)((const char *)sl.dev + ub);
        L.grid = grid;
        e = tc_pair_launch(L, nullptr, nullptr, st);
    }
    if (e == cudaSuccess && !units1.empty()) {
        L.units = (const Unit *)((const char *)sl.dev + u1b0);
        L.nunits = (int)units1.size();
        L.cta_offsets = (const int *)((const char *)sl.dev + u1b0 + u1b);
        L.grid = grid1;
        e = tc_launch(L, nullptr, nullptr, st);
    }
    if (e == cudaSuccess) e = cudaEventRecord(sl.done, st);
    if (e != cudaSuccess) {
        drop(pend);
        return cuda_fail(e, "stream launch");
    }
    if (pend->items.empty()) {  // frames copied, no integration completed
        drop(pend);
        return CHX_OK;
    }
    e = cudaEventRecord(pend->ev, st);
    if (e != cudaSuccess) {
        drop(pend);
        return cuda_fail(e, "completion event");
    }
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->queue.push_back(pend);
    }
    s->cv.notify_one();
    return CHX_OK;
}

int chx_stream_last_dump(chx_stream *s, int channel_id, const int32_t **d_blocks, int64_t *seq) {
    clear_error();
    if (!s || channel_id < 0 || channel_id >= (int)s->chans.size())
        return fail(CHX_E_INVALID, "bad channel");
    std::lock_guard<std::mutex> lock(s->mu);
    const StreamChan &c = s->chans[channel_id];
    if (c.done_seq < 0) {
        if (d_blocks) *d_blocks = nullptr;
        if (seq) *seq = -1;
        return CHX_OK;
    }
    if (d_blocks) *d_blocks = c.dumps + (size_t)c.done_half * c.NB * 2048;
    if (seq) *seq = c.done_seq;
    return CHX_OK;
}

int chx_stream_stats_get(chx_stream *s, chx_stream_stats *out) {
    clear_error();
    if (!s || !out) return fail(CHX_E_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lock(s->mu);
    out->frames = s->frames;
    out->dumps = s->dumps;
    out->resident_bytes = s->resident;
    std::vector<double> v = s->latencies_ms;
    if (v.empty()) {
        out->p50_ms = out->p99_ms = out->max_ms = 0.0;
        return CHX_OK;
    }
    std::sort(v.begin(), v.end());
    auto pct = [&](double q) {
        const size_t k = std::min(v.size() - 1, (size_t)(q * (double)(v.size() - 1) + 0.5));
        return v[k];
    };
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
    out->max_ms = v.back();
    return CHX_OK;
}

int chx_stream_reset_stats(chx_stream *s) {
    clear_error();
    if (!s) return fail(CHX_E_INVALID, "NULL stream");
    std::lock_guard<std::mutex> lock(s->mu);
    s->latencies_ms.clear();
    return CHX_OK;
}

int chx_stream_sync(chx_stream *s) {
    clear_error();
    if (!s) return fail(CHX_E_INVALID, "NULL stream");
    if (!wait_published(s, 60000))
        return fail(CHX_E_TIMEOUT, "launches still unpublished after 60 s");
    return CHX_OK;
}

int chx_stream_check(chx_stream *s) {
    clear_error();
    if (!s) return fail(CHX_E_INVALID, "NULL stream");
    DeviceGuard g(s->device);
    CHX_CUDA(cudaDeviceSynchronize());
    if (!wait_published(s, 60000))
        return fail(CHX_E_TIMEOUT, "launches still unpublished after 60 s");
    int h = 0;
    CHX_CUDA(cudaMemcpy(&h, s->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) {
        CHX_CUDA(cudaMemset(s->d_err, 0, sizeof(int)));
        return fail(CHX_E_TIMEOUT, "a bounded device wait gave up (code 0x%x)", h);
    }
    return CHX_OK;
}

int chx_stream_destroy(chx_stream *s) {
    clear_error();
    if (!s) return CHX_OK;
    DeviceGuard g(s->device);
    cudaDeviceSynchronize();
    stop_poller(s);
    free_stream(s);
    delete s;
    return CHX_OK;
}

}  // extern "C"
