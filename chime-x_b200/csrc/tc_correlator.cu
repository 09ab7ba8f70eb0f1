// tc_correlator.cu -- tcgen05 kind::i8 correlator for sm_100a.
//
// Formulation.  For one channel, a work unit is a pair of 128-element tiles
// (Ty <= Tx) over a range of samples.  Each sample contributes two k-rows:
//   A (M = 128 rows, the y elements of tile Ty):   k = 2t : a0(y),  2t+1 : a1(y)
//   B (N = 256 cols, the x elements of tile Tx):   k = 2t : [b0(x) | b2(x)]
//                                                  2t+1 : [b1(x) | b3(x)]
// so that D = A^T B (int32, in TMEM) holds Re(y, x) in columns 0..127 and
// Im(y, x) in columns 128..255 (value maps in chimex_internal.h).  Four int8
// MACs per complex visibility per sample, none wasted; every TMEM lane is one
// output row y, so the epilogue writes the reference block layout directly.
//
// Operands are MN-major (elements contiguous, as in the input bytes) with the
// 128-byte swizzle: a k-row is 128 bytes (128 elements); 8 k-rows form a
// 1 KiB swizzle atom.  A stage holds 64 samples = 128 k-rows:
//   A stage: 16 KiB  (one MN atom wide)
//   B stage: 32 KiB  (two MN atoms: Re columns then Im columns, LBO = 16 KiB)
//
// Roles (288 threads):
//   warps 0-7  unpack: load packed bytes from global memory (16 B per
//              thread-chunk), convert nibbles to int8 with SWAR arithmetic and
//              store the swizzled operand rows; then the epilogue.
//   warp 8     TMEM allocation and the single-thread MMA issue loop.
// Every mbarrier wait is bounded (globaltimer); on timeout the kernel records
// an error code in the caller's error word, drains its MMAs and returns.
#include "chimex_internal.h"

namespace chx {

namespace {

constexpr int kTile = 128;              // elements per tile side
constexpr int kStageSamples = 64;       // samples per pipeline stage
constexpr int kStages = 4;              // operand ring depth
constexpr int kABytes = 2 * kStageSamples * 128;   // 16 KiB
constexpr int kBBytes = 2 * kABytes;               // 32 KiB
constexpr int kUnpackWarps = 8;
constexpr int kUnpackThreads = kUnpackWarps * 32;
constexpr int kThreads = kUnpackThreads + 32;
constexpr int kTmemCols = 256;
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s

constexpr int kSmemBytes = kStages * (kABytes + kBBytes) + 1024 /*align*/ + 256 /*bars*/;

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: true when the phase completed, false on timeout or abort.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity,
                                          volatile int *abort_flag) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer();
    while (true) {
#pragma unroll 1
        for (int i = 0; i < 32; i++)
            if (mbar_try_wait(bar, parity)) return true;
        if (*abort_flag) return false;
        if (globaltimer() - t0 > kWaitLimitNs) return false;
    }
}
// Bounded wait that ignores the abort flag (used to drain in-flight MMAs).
__device__ __forceinline__ bool mbar_wait_timeout(uint64_t *bar, uint32_t parity) {
    const uint64_t t0 = globaltimer();
    while (!mbar_try_wait(bar, parity))
        if (globaltimer() - t0 > kWaitLimitNs) return false;
    return true;
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Shared-memory matrix descriptor (tcgen05): start, leading and stride byte
// offsets in 16-byte units, version 1, 128-byte swizzle (layout type 2).
__device__ __forceinline__ uint64_t make_sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// Instruction descriptor: kind::i8, D = s32, A = B = signed int8, both
// MN-major, N = 256, M = 128.
constexpr uint32_t kIdesc = (2u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
                            ((256u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ------------------------------------------------------------- SWAR unpack
// n: four offset-binary nibbles (0..15), one per byte.
__device__ __forceinline__ uint32_t sgn(uint32_t n) {  // n - 8 per byte
    return (n + 0x78787878u) ^ 0x80808080u;
}
__device__ __forceinline__ uint32_t neg_sgn(uint32_t n) {  // 8 - n per byte
    return (0x88888888u - n) ^ 0x80808080u;
}
__device__ __forceinline__ uint32_t neg(uint32_t n) {  // -n per byte
    return (0x80808080u - n) ^ 0x80808080u;
}

struct Conv {
    uint32_t a0, a1, b0, b1, b2, b3;
};

template <int MAP>
__device__ __forceinline__ Conv convert(uint32_t w) {
    const uint32_t lo = w & 0x0F0F0F0Fu;
    const uint32_t hi = (w >> 4) & 0x0F0F0F0Fu;
    Conv c;
    if (MAP == MAP_EXACT) {
        c.a0 = sgn(hi);
        c.a1 = sgn(lo);
        c.b0 = c.a0;
        c.b1 = c.a1;
        c.b2 = neg_sgn(lo);
        c.b3 = c.a0;
    } else if (MAP == MAP_CONF) {
        c.a0 = hi;
        c.a1 = lo;
        c.b0 = hi;
        c.b1 = lo;
        c.b2 = neg(lo);
        c.b3 = hi;
    } else {
        c.a0 = hi;
        c.a1 = lo ^ 0x0F0F0F0Fu;
        c.b0 = hi;
        c.b1 = neg(lo);
        c.b2 = c.b1;
        c.b3 = neg(hi);
    }
    return c;
}

// Byte offset of 16-byte chunk `g` (elements 16g..16g+15) of k-row `k` inside
// a 128-byte-wide MN-major swizzled operand block.
__device__ __forceinline__ uint32_t swz(int k, int g) {
    return (uint32_t)(k * 128 + ((g ^ (k & 7)) << 4));
}

__device__ __forceinline__ void sts128(uint32_t addr, uint4 v) {
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(v.x), "r"(v.y),
                 "r"(v.z), "r"(v.w)
                 : "memory");
}

__device__ __forceinline__ uint4 ldg_nc(const uint8_t *p) {
    uint4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}

// (Ty, Tx) of tile pair p in row-major upper-triangle order.
__device__ __forceinline__ void decode_pair(int p, int nt, int &ty, int &tx) {
    int r = p, y = 0;
    while (r >= nt - y) {
        r -= nt - y;
        y++;
    }
    ty = y;
    tx = y + r;
}

struct KParams {
    const uint8_t *packed;
    int64_t in_stride, chan_stride;
    int32_t *blocks;
    int64_t out_chan_stride;
    int E, F, T;
    int nt, npairs, splits, tchunk;
    int nb1;
    int ut, mode;
    int *err;
};

template <int MAP>
__global__ void __launch_bounds__(kThreads, 1) tc_correlate_kernel(const KParams P) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t *sA = smem;
    uint8_t *sB = smem + kStages * kABytes;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sB + kStages * kBBytes);
    uint64_t *full = bars;                 // [kStages]
    uint64_t *empty = bars + kStages;      // [kStages]
    uint64_t *accum_full = bars + 2 * kStages;
    uint64_t *drain = bars + 2 * kStages + 1;
    volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(bars + 2 * kStages + 2);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(bars + 2 * kStages + 3);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    // ---- work unit
    int u = blockIdx.x;
    const int split = u % P.splits;
    u /= P.splits;
    const int pair = u % P.npairs;
    const int f = u / P.npairs;
    int ty, tx;
    decode_pair(pair, P.nt, ty, tx);
    const int t_begin = split * P.tchunk;
    const int t_end = min(P.T, t_begin + P.tchunk);
    const int nstages = (t_end - t_begin + kStageSamples - 1) / kStageSamples;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; s++) {
            mbar_init(&full[s], kUnpackThreads);
            mbar_init(&empty[s], 1);
        }
        mbar_init(accum_full, 1);
        mbar_init(drain, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == kUnpackWarps) {
        asm volatile(
            "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                smem_u32((const void *)tmem_slot)),
            "r"(kTmemCols)
            : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == kUnpackWarps) {
        // ------------------------------------------------------ MMA issuer
        if (lane == 0) {
            bool ok = true;
            for (int it = 0; it < nstages; it++) {
                const int slot = it % kStages;
                const uint32_t phase = (it / kStages) & 1;
                if (!mbar_wait(&full[slot], phase, abort_flag)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t a0 = smem_u32(sA + slot * kABytes);
                const uint32_t b0 = smem_u32(sB + slot * kBBytes);
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const uint64_t ad = make_sdesc(a0 + i * 4096, kABytes, 1024);
                    const uint64_t bd = make_sdesc(b0 + i * 4096, kABytes, 1024);
                    mma_i8(tmem_base, ad, bd, kIdesc, (it > 0 || i > 0) ? 1u : 0u);
                }
                // Release the slot only if it will be refilled: no barrier
                // arrival may be left pending when the CTA retires.
                if (it + kStages < nstages) mma_commit(&empty[slot]);
            }
            if (ok) {
                mma_commit(accum_full);
            } else {
                atomicOr(P.err, 0x1);
                *abort_flag = 1;
                mma_commit(drain);  // completes once every issued MMA is done
                mbar_wait_timeout(drain, 0);
            }
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------ unpack
        const int tid = threadIdx.x;  // 0..255
        const uint8_t *chan = P.packed + (int64_t)f * P.chan_stride;
        const int ey = ty * kTile, ex = tx * kTile;
        bool ok = true;
        // Each thread converts chunks c = tid and tid + 256 of the 512 16-byte
        // chunks (64 samples x 8 chunks) of each tile per stage.
        uint4 vy[2], vx[2];
        auto load = [&](int it) {
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const int c = tid + j * kUnpackThreads;
                const int s = c >> 3, g = c & 7;
                const int t = t_begin + it * kStageSamples + s;
                const bool tv = t < t_end;
                const uint8_t *row = chan + (int64_t)t * P.in_stride;
                // samples outside the range are zeroed at the store
                vy[j] = (tv && ey + 16 * g < P.E) ? ldg_nc(row + ey + 16 * g) : make_uint4(0, 0, 0, 0);
                vx[j] = (tv && ex + 16 * g < P.E) ? ldg_nc(row + ex + 16 * g) : make_uint4(0, 0, 0, 0);
            }
        };
        if (nstages > 0) load(0);
        for (int it = 0; it < nstages && ok; it++) {
            const int slot = it % kStages;
            const uint32_t phase = (it / kStages) & 1;
            uint4 cy[2] = {vy[0], vy[1]}, cx[2] = {vx[0], vx[1]};
            if (it + 1 < nstages) load(it + 1);
            if (!mbar_wait(&empty[slot], phase ^ 1, abort_flag)) {
                ok = false;
                break;
            }
            const uint32_t a_base = smem_u32(sA + slot * kABytes);
            const uint32_t b_base = smem_u32(sB + slot * kBBytes);
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const int c = tid + j * kUnpackThreads;
                const int s = c >> 3, g = c & 7;
                const int t = t_begin + it * kStageSamples + s;
                Conv y0 = convert<MAP>(cy[j].x), y1 = convert<MAP>(cy[j].y),
                     y2 = convert<MAP>(cy[j].z), y3 = convert<MAP>(cy[j].w);
                Conv x0 = convert<MAP>(cx[j].x), x1 = convert<MAP>(cx[j].y),
                     x2 = convert<MAP>(cx[j].z), x3 = convert<MAP>(cx[j].w);
                uint4 A0 = make_uint4(y0.a0, y1.a0, y2.a0, y3.a0);
                uint4 A1 = make_uint4(y0.a1, y1.a1, y2.a1, y3.a1);
                uint4 B0 = make_uint4(x0.b0, x1.b0, x2.b0, x3.b0);
                uint4 B1 = make_uint4(x0.b1, x1.b1, x2.b1, x3.b1);
                uint4 B2 = make_uint4(x0.b2, x1.b2, x2.b2, x3.b2);
                uint4 B3 = make_uint4(x0.b3, x1.b3, x2.b3, x3.b3);
                if (t >= t_end) {  // exact zeros whatever the map
                    A0 = A1 = B0 = B1 = B2 = B3 = make_uint4(0, 0, 0, 0);
                }
                const int k0 = 2 * s, k1 = 2 * s + 1;
                sts128(a_base + swz(k0, g), A0);
                sts128(a_base + swz(k1, g), A1);
                sts128(b_base + swz(k0, g), B0);
                sts128(b_base + swz(k1, g), B1);
                sts128(b_base + kABytes + swz(k0, g), B2);
                sts128(b_base + kABytes + swz(k1, g), B3);
            }
            fence_proxy_async();
            mbar_arrive(&full[slot]);
        }
        if (!ok) {
            atomicOr(P.err, 0x2);
            *abort_flag = 1;
        }

        // ------------------------------------------------------ epilogue
        if (ok && mbar_wait(accum_full, 0, abort_flag)) {
            tc_fence_after();
            const int q = warp & 3;        // TMEM lane quarter = 32 output rows
            const int h = warp >> 2;       // which two 32-column x blocks
            const int by = ty * 4 + q;
            int32_t *out_chan = P.blocks + (int64_t)f * P.out_chan_stride;
#pragma unroll 1
            for (int jj = 0; jj < 2; jj++) {
                const int j = 2 * h + jj;
                const int bx = tx * 4 + j;
                uint32_t re[32], im[32];
                const uint32_t taddr = tmem_base + ((uint32_t)(32 * q) << 16);
                tmem_ld32(taddr + 32 * j, re);
                tmem_ld32(taddr + 128 + 32 * j, im);
                tmem_wait_ld();
                if (by >= P.nb1 || bx >= P.nb1 || bx < by) continue;
                const int64_t b = (int64_t)by * P.nb1 - (int64_t)by * (by - 1) / 2 + (bx - by);
                int32_t *dst = out_chan + (b * 32 + lane) * 64;
                if (!P.ut) {
#pragma unroll
                    for (int i = 0; i < 32; i++) im[i] = 0u - im[i];
                }
                if (P.mode == 0) {
#pragma unroll
                    for (int i = 0; i < 32; i += 2)
                        *reinterpret_cast<int4 *>(dst + 2 * i) =
                            make_int4((int)re[i], (int)im[i], (int)re[i + 1], (int)im[i + 1]);
                } else if (P.mode == 1) {
#pragma unroll
                    for (int i = 0; i < 32; i += 2) {
                        int4 o = *reinterpret_cast<int4 *>(dst + 2 * i);
                        o.x = (int)((uint32_t)o.x + re[i]);
                        o.y = (int)((uint32_t)o.y + im[i]);
                        o.z = (int)((uint32_t)o.z + re[i + 1]);
                        o.w = (int)((uint32_t)o.w + im[i + 1]);
                        *reinterpret_cast<int4 *>(dst + 2 * i) = o;
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < 32; i++) {
                        atomicAdd(dst + 2 * i, (int)re[i]);
                        atomicAdd(dst + 2 * i + 1, (int)im[i]);
                    }
                }
            }
        } else if (ok) {
            atomicOr(P.err, 0x4);
            *abort_flag = 1;
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == kUnpackWarps) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                     "r"(kTmemCols)
                     : "memory");
    }
}

}  // namespace

bool tc_supported(int E, int T) { return E >= 32 && E % 32 == 0 && T >= 1; }

cudaError_t launch_correlate_tc(const TcArgs &a, int sm_count, cudaStream_t st) {
    (void)sm_count;
    if ((reinterpret_cast<uintptr_t>(a.packed) & 15) || (a.in_stride & 15) || (a.chan_stride & 15))
        return cudaErrorMisalignedAddress;
    KParams P;
    P.packed = a.packed;
    P.in_stride = a.in_stride;
    P.chan_stride = a.chan_stride;
    P.blocks = a.blocks;
    P.out_chan_stride = a.out_chan_stride;
    P.E = a.E;
    P.F = a.F;
    P.T = a.T;
    P.nt = (a.E + kTile - 1) / kTile;
    P.npairs = P.nt * (P.nt + 1) / 2;
    int splits = a.splits < 1 ? 1 : a.splits;
    int tchunk = (a.T + splits - 1) / splits;
    tchunk = (tchunk + kStageSamples - 1) / kStageSamples * kStageSamples;
    splits = (a.T + tchunk - 1) / tchunk;
    P.splits = splits;
    P.tchunk = tchunk;
    P.nb1 = a.E / 32;
    P.ut = a.ut;
    P.mode = a.mode;
    P.err = a.err;
    const int64_t units = (int64_t)a.F * P.npairs * splits;
    if (units <= 0 || units > 0x7FFFFFFF) return cudaErrorInvalidValue;
    static bool attr_done[3] = {false, false, false};
    cudaError_t e = cudaSuccess;
    if (a.map == MAP_EXACT) {
        if (!attr_done[0]) {
            e = cudaFuncSetAttribute(tc_correlate_kernel<MAP_EXACT>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
            attr_done[0] = (e == cudaSuccess);
        }
        if (e == cudaSuccess)
            tc_correlate_kernel<MAP_EXACT><<<(unsigned)units, kThreads, kSmemBytes, st>>>(P);
    } else if (a.map == MAP_CONF) {
        if (!attr_done[1]) {
            e = cudaFuncSetAttribute(tc_correlate_kernel<MAP_CONF>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
            attr_done[1] = (e == cudaSuccess);
        }
        if (e == cudaSuccess)
            tc_correlate_kernel<MAP_CONF><<<(unsigned)units, kThreads, kSmemBytes, st>>>(P);
    } else {
        if (!attr_done[2]) {
            e = cudaFuncSetAttribute(tc_correlate_kernel<MAP_PACKED>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
            attr_done[2] = (e == cudaSuccess);
        }
        if (e == cudaSuccess)
            tc_correlate_kernel<MAP_PACKED><<<(unsigned)units, kThreads, kSmemBytes, st>>>(P);
    }
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace chx
