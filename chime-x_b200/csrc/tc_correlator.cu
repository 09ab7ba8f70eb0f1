// tc_correlator.cu -- tcgen05 kind::i8 correlator for sm_100a.
//
// Formulation.  A work unit is one 128-element y tile (M = 128 TMEM lanes)
// against W = 128 or 256 x elements (N = W) of one channel over a sample
// range.  Per sample the y tile provides three int8 k-row types and the x
// tile two:
//     R = yr, I = yi, N = -yr          X = 16*xr, Y = 16*xi
// and two int32 accumulators in TMEM receive
//     Re (cols 0..W)        += R*X + I*Y          = 16 * sum (yr xr + yi xi)
//     Im (cols 256..256+W)  += I*X + N*Y          = 16 * sum (yi xr - yr xi)
// which is V[y][x] = sum s_y conj(s_x) (cpu_corr_test.c:188-193) scaled by 16:
// four int8 MACs per complex visibility per sample, none wasted.  Scaling the
// x operand by 16 makes its conversion one or two logic ops per 4 bytes; the
// epilogue shifts the accumulators right by 4 (exact).  |Re|, |Im| <= 16*128*T
// stays below 2^31 for T < 2^20; units never exceed kUnitMaxSamples samples.
// The reference-compatibility value maps (offset nibbles, inverted imaginary
// nibble) use the same structure with other conversions and an unsigned x.
//
// Shared-memory operands are MN-major (elements contiguous, like the input
// bytes) with the 128-byte swizzle: an 8 k-row x 128-byte atom per 8 samples
// and component.  One stage covers 32 samples:
//   y: atoms [R0 I0 R1 I1 R2 I2 R3 I3 | I0 N0 I1 N1 I2 N2 I3 N3]   16 KiB
//   x: per 128-element slice [X0 Y0 X1 Y1 X2 Y2 X3 Y3]             8 KiB per slice
// (digit = 8-sample block; the I rows are stored twice so that every MMA
// reads four consecutive atoms).  Four MMAs per stage (K = 32 each),
// alternating accumulators so that consecutive MMAs are independent:
//   Re += [R0 I0 R1 I1].[X0 Y0 X1 Y1]    Im += [I0 N0 I1 N1].[X0 Y0 X1 Y1]
//   Re += [R2 I2 R3 I3].[X2 Y2 X3 Y3]    Im += [I2 N2 I3 N3].[X2 Y2 X3 Y3]
//
// Roles (320 threads, one persistent CTA per SM, units taken round-robin from
// a table sorted by decreasing cost):
//   warps 0-7  unpack: read packed bytes from the TMA ring, convert with SWAR
//              logic, store swizzled operand rows; then the epilogue (TMEM ->
//              reference block layout).
//   warp 8     TMA producer: packed y and x tiles, 32 samples per stage.
//   warp 9     TMEM allocation and the single-thread MMA issue loop.
// Every wait is bounded (globaltimer): on timeout the CTA records an error
// code in the caller's error word, drains its MMAs and TMA loads and returns.
#include "chimex_internal.h"

#include <cudaTypedefs.h>
#include <string.h>

#include <algorithm>

namespace chx {

namespace {

constexpr int kStageSamples = 32;
constexpr int kOpStages = 4;    // operand ring
constexpr int kPkStages = 6;    // packed-tile ring
constexpr int kYOpBytes = 16 * 1024;
constexpr int kXOpBytes = 16 * 1024;
constexpr int kPkYBytes = kStageSamples * 128;      // 4 KiB
constexpr int kPkXBytes = 2 * kPkYBytes;            // 8 KiB
constexpr int kUnpackWarps = 8;
constexpr int kUnpackThreads = kUnpackWarps * 32;
constexpr int kProducerWarp = 8;
constexpr int kMmaWarp = 9;
constexpr int kThreads = 320;
constexpr int kTmemCols = 512;
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s

constexpr int kOffOpY = 0;
constexpr int kOffOpX = kOffOpY + kOpStages * kYOpBytes;
constexpr int kOffPkY = kOffOpX + kOpStages * kXOpBytes;
constexpr int kOffPkX = kOffPkY + kPkStages * kPkYBytes;
constexpr int kOffBars = kOffPkX + kPkStages * kPkXBytes;
constexpr int kSmemBytes = kOffBars + 256 + 1024;

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: true when the phase completed, false on timeout or abort.
__device__ __noinline__ bool mbar_wait_slow(uint32_t bar, uint32_t parity,
                                            volatile int *abort_flag) {
    const uint64_t t0 = globaltimer();
    while (true) {
#pragma unroll 1
        for (int i = 0; i < 64; i++)
            if (mbar_try_wait(bar, parity)) return true;
        if (*abort_flag) return false;
        if (globaltimer() - t0 > kWaitLimitNs) return false;
    }
}
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity,
                                          volatile int *abort_flag) {
    if (mbar_try_wait(bar, parity)) return true;
    return mbar_wait_slow(bar, parity, abort_flag);
}
// Bounded wait ignoring the abort flag (draining in-flight asynchronous work).
__device__ __noinline__ bool mbar_wait_drain(uint32_t bar, uint32_t parity) {
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

// TMA: 3-D tile {128 elements, 1 channel, 32 samples} -> shared memory.
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, int x, int y,
                                            int z, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

// Shared-memory matrix descriptor: start, leading and stride byte offsets in
// 16-byte units, descriptor version 1, 128-byte swizzle (layout type 2).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46) |
           ((uint64_t)2 << 61);
}

// Instruction descriptor: kind::i8, D = s32, A = signed int8, B signed or
// unsigned int8, both MN-major, M = 128, N = n.
__device__ __forceinline__ uint32_t idesc_i8(int n, bool b_signed) {
    return (2u << 4) | (1u << 7) | ((b_signed ? 1u : 0u) << 10) | (1u << 15) | (1u << 16) |
           ((uint32_t)(n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
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

__device__ __forceinline__ uint4 lds128(uint32_t addr) {
    uint4 v;
    asm volatile("ld.shared.v4.b32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "r"(addr)
                 : "memory");
    return v;
}
__device__ __forceinline__ void sts128(uint32_t addr, uint32_t a, uint32_t b, uint32_t c,
                                       uint32_t d) {
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c),
                 "r"(d)
                 : "memory");
}

// ------------------------------------------------------------- SWAR unpack
// Per byte of n: an offset-binary nibble 0..15.
__device__ __forceinline__ uint32_t sgn(uint32_t n) { return (n + 0x78787878u) ^ 0x80808080u; }
__device__ __forceinline__ uint32_t neg_sgn(uint32_t n) {
    return (0x88888888u - n) ^ 0x80808080u;
}
__device__ __forceinline__ uint32_t neg(uint32_t n) { return (0x80808080u - n) ^ 0x80808080u; }

// y operand rows R, I, N from four packed bytes.
template <int MAP>
__device__ __forceinline__ void yconv(uint32_t w, uint32_t &r, uint32_t &i, uint32_t &n) {
    const uint32_t lo = w & 0x0F0F0F0Fu;
    const uint32_t hi = (w >> 4) & 0x0F0F0F0Fu;
    if (MAP == MAP_EXACT) {  // yr, yi, -yr
        r = sgn(hi);
        i = sgn(lo);
        n = neg_sgn(hi);
    } else if (MAP == MAP_CONF) {  // y'r, y'i, -y'r
        r = hi;
        i = lo;
        n = neg(hi);
    } else {  // y'r, -(15 - y'i), -y'r
        r = hi;
        i = neg(lo ^ 0x0F0F0F0Fu);
        n = neg(hi);
    }
}
// x operand rows X = 16*re, Y = 16*im (signed for MAP_EXACT, else unsigned).
template <int MAP>
__device__ __forceinline__ void xconv(uint32_t w, uint32_t &xr, uint32_t &xi) {
    if (MAP == MAP_EXACT) {
        xr = (w & 0xF0F0F0F0u) ^ 0x80808080u;
        xi = ((w << 4) & 0xF0F0F0F0u) ^ 0x80808080u;
    } else {
        xr = w & 0xF0F0F0F0u;
        xi = (w << 4) & 0xF0F0F0F0u;
    }
}

// Byte offset of 16-byte chunk g of row r (0..7) in a 128-byte-swizzled atom.
__device__ __forceinline__ uint32_t swz(int r, int g) {
    return (uint32_t)(r * 128 + ((g ^ r) << 4));
}

struct KParams {
    const ChanDesc *chans;
    const Unit *units;
    int nunits;
    uint64_t out_base;
    int use_param_map;
    int ut;
    int accumulate;
    int *err;
};

template <int MAP>
__global__ void __launch_bounds__(kThreads, 1)
tc_correlate_kernel(const __grid_constant__ CUtensorMap pmap, const KParams P) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const uint32_t sbase = smem_u32(smem);
    const uint32_t op_y = sbase + kOffOpY, op_x = sbase + kOffOpX;
    const uint32_t pk_y = sbase + kOffPkY, pk_x = sbase + kOffPkX;
    const uint32_t bars = sbase + kOffBars;
    auto full_pk = [&](int s) { return bars + 8 * s; };
    auto empty_pk = [&](int s) { return bars + 8 * (kPkStages + s); };
    auto full_op = [&](int s) { return bars + 8 * (2 * kPkStages + s); };
    auto empty_op = [&](int s) { return bars + 8 * (2 * kPkStages + kOpStages + s); };
    const uint32_t acc_full = bars + 8 * (2 * kPkStages + 2 * kOpStages);
    const uint32_t acc_empty = acc_full + 8;
    const uint32_t drain = acc_full + 16;
    uint8_t *bar_ptr = smem + kOffBars;
    volatile uint32_t *tmem_slot =
        reinterpret_cast<volatile uint32_t *>(bar_ptr + 8 * (2 * kPkStages + 2 * kOpStages + 3));
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kPkStages; s++) {
            mbar_init(full_pk(s), 1);
            mbar_init(empty_pk(s), kUnpackThreads);
        }
        for (int s = 0; s < kOpStages; s++) {
            mbar_init(full_op(s), kUnpackThreads);
            mbar_init(empty_op(s), 1);
        }
        mbar_init(acc_full, 1);
        mbar_init(acc_empty, kUnpackThreads);
        mbar_init(drain, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == kMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32((const void *)tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    const int nunits = P.nunits;
    const int first = blockIdx.x, stride = gridDim.x;

    if (warp == kProducerWarp) {
        // ------------------------------------------------------ TMA producer
        if (lane == 0) {
            uint32_t g = 0;  // global stage counter
            bool ok = true;
            for (int u = first; u < nunits && ok; u += stride) {
                const Unit U = P.units[u];
                const ChanDesc *cd = P.chans + U.chan;
                const CUtensorMap *map = P.use_param_map ? &pmap : &cd->map;
                const int fc = cd->fcoord;
                const int ty = U.tyx & 1023, x0 = (U.tyx >> 10) & 1023, nx = (U.tyx >> 20) & 3;
                const int nst = (U.t1 - U.t0 + kStageSamples - 1) / kStageSamples;
                const uint32_t bytes = (uint32_t)(kPkYBytes * (1 + nx));
                for (int it = 0; it < nst; it++, g++) {
                    const int s = g % kPkStages;
                    const uint32_t ph = (g / kPkStages) & 1;
                    if (!mbar_wait(empty_pk(s), ph ^ 1, abort_flag)) {
                        ok = false;
                        break;
                    }
                    const int t = U.t0 + it * kStageSamples;
                    mbar_expect_tx(full_pk(s), bytes);
                    tma_load_3d(pk_y + s * kPkYBytes, map, ty * 128, fc, t, full_pk(s));
                    for (int j = 0; j < nx; j++)
                        tma_load_3d(pk_x + s * kPkXBytes + j * kPkYBytes, map, (x0 + j) * 128, fc,
                                    t, full_pk(s));
                }
            }
            if (!ok) {
                atomicOr(P.err, 0x10);
                *abort_flag = 1;
            }
            // Drain: wait (bounded) for the last loads issued on every slot so
            // that no TMA write lands after the CTA retires.
            const uint32_t issued = g;
            for (uint32_t k = (issued > (uint32_t)kPkStages ? issued - kPkStages : 0); k < issued;
                 k++)
                mbar_wait_drain(full_pk(k % kPkStages), (k / kPkStages) & 1);
        }
        __syncwarp();
    } else if (warp == kMmaWarp) {
        // ------------------------------------------------------ MMA issuer
        if (lane == 0) {
            uint32_t g = 0, acc_phase = 0;
            bool ok = true;
            const bool b_signed = (MAP == MAP_EXACT);
            // Descriptors of operand slot 0; slot s adds its byte offset >> 4
            // to the start-address field (shared addresses stay < 256 KiB).
            const uint64_t dRe0 = sdesc(op_y, 1024, 1024), dRe1 = sdesc(op_y + 4096, 1024, 1024);
            const uint64_t dIm0 = sdesc(op_y + 8192, 1024, 1024);
            const uint64_t dIm1 = sdesc(op_y + 12288, 1024, 1024);
            const uint64_t dX0 = sdesc(op_x, 8192, 1024), dX1 = sdesc(op_x + 4096, 8192, 1024);
            for (int u = first; u < nunits && ok; u += stride) {
                const Unit U = P.units[u];
                const int nx = (U.tyx >> 20) & 3;
                const uint32_t idesc = idesc_i8(128 * nx, b_signed);
                const int nst = (U.t1 - U.t0 + kStageSamples - 1) / kStageSamples;
                const bool last_unit = (u + stride >= nunits);
                // the epilogue of the previous unit must have drained TMEM
                if (!mbar_wait(acc_empty, acc_phase ^ 1, abort_flag)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                for (int it = 0; it < nst; it++, g++) {
                    const int s = g % kOpStages;
                    const uint32_t ph = (g / kOpStages) & 1;
                    if (!mbar_wait(full_op(s), ph, abort_flag)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint64_t so_y = (uint64_t)((s * kYOpBytes) >> 4);
                    const uint64_t so_x = (uint64_t)((s * kXOpBytes) >> 4);
                    const uint32_t first_k = (it > 0) ? 1u : 0u;
                    mma_i8(tmem_base, dRe0 + so_y, dX0 + so_x, idesc, first_k);        // Re
                    mma_i8(tmem_base + 256, dIm0 + so_y, dX0 + so_x, idesc, first_k);  // Im
                    mma_i8(tmem_base, dRe1 + so_y, dX1 + so_x, idesc, 1u);             // Re
                    mma_i8(tmem_base + 256, dIm1 + so_y, dX1 + so_x, idesc, 1u);       // Im
                    // Release the operand slot unless nothing will refill it:
                    // no arrival may be left pending when the CTA retires.
                    if (!(last_unit && it + kOpStages >= nst)) mma_commit(empty_op(s));
                }
                if (!ok) break;
                mma_commit(acc_full);
                acc_phase ^= 1;
            }
            if (!ok) {
                atomicOr(P.err, 0x20);
                *abort_flag = 1;
                mma_commit(drain);
                mbar_wait_drain(drain, 0);
            }
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------ unpack + epilogue
        const int tid = threadIdx.x;  // 0..255
        // y chunk: sample sy = tid >> 3, 16-element group gy = tid & 7
        const int sy = tid >> 3, gy = tid & 7;
        const uint32_t ry = (uint32_t)(sy & 7), by8 = (uint32_t)(sy >> 3);
        const uint32_t ldy = (uint32_t)(sy * 128 + gy * 16);
        const uint32_t sty_r = (2 * by8) * 1024 + swz(ry, gy);  // R; I at +1K
        const uint32_t sty_i = 8192 + sty_r;                      // I; N at +1K
        // x chunks c = tid + 256 j (slice j): the same sample and group as y
        const uint32_t stx = (2 * by8) * 1024 + swz(ry, gy);
        uint32_t g = 0, acc_phase = 0;
        bool ok = true;
        for (int u = first; u < nunits && ok; u += stride) {
            const Unit U = P.units[u];
            const ChanDesc *cd = P.chans + U.chan;
            const int ty = U.tyx & 1023, x0 = (U.tyx >> 10) & 1023, nx = (U.tyx >> 20) & 3;
            const int nst = (U.t1 - U.t0 + kStageSamples - 1) / kStageSamples;
            for (int it = 0; it < nst; it++, g++) {
                const int ps = g % kPkStages;
                const uint32_t pph = (g / kPkStages) & 1;
                if (!mbar_wait(full_pk(ps), pph, abort_flag)) {
                    ok = false;
                    break;
                }
                const bool valid = (U.t0 + it * kStageSamples + sy) < U.t1;
                const uint4 wy = lds128(pk_y + ps * kPkYBytes + ldy);
                const uint4 wx0 = lds128(pk_x + ps * kPkXBytes + ldy);
                uint4 wx1 = make_uint4(0, 0, 0, 0);
                if (nx > 1) wx1 = lds128(pk_x + ps * kPkXBytes + kPkYBytes + ldy);
                // Convert before releasing the packed slot: the converted
                // registers depend on the loaded words, so the slot is free
                // once the arrive is visible.
                uint32_t r[4], i[4], n[4], xr0[4], xi0[4], xr1[4], xi1[4];
                yconv<MAP>(wy.x, r[0], i[0], n[0]);
                yconv<MAP>(wy.y, r[1], i[1], n[1]);
                yconv<MAP>(wy.z, r[2], i[2], n[2]);
                yconv<MAP>(wy.w, r[3], i[3], n[3]);
                xconv<MAP>(wx0.x, xr0[0], xi0[0]);
                xconv<MAP>(wx0.y, xr0[1], xi0[1]);
                xconv<MAP>(wx0.z, xr0[2], xi0[2]);
                xconv<MAP>(wx0.w, xr0[3], xi0[3]);
                xconv<MAP>(wx1.x, xr1[0], xi1[0]);
                xconv<MAP>(wx1.y, xr1[1], xi1[1]);
                xconv<MAP>(wx1.z, xr1[2], xi1[2]);
                xconv<MAP>(wx1.w, xr1[3], xi1[3]);
                if (!valid) {  // samples outside the unit contribute zero
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        r[k] = i[k] = n[k] = xr0[k] = xi0[k] = xr1[k] = xi1[k] = 0u;
                }
                mbar_arrive(empty_pk(ps));

                const int os = g % kOpStages;
                const uint32_t oph = (g / kOpStages) & 1;
                if (!mbar_wait(empty_op(os), oph ^ 1, abort_flag)) {
                    ok = false;
                    break;
                }
                const uint32_t ya = op_y + os * kYOpBytes, xa = op_x + os * kXOpBytes;
                sts128(ya + sty_r, r[0], r[1], r[2], r[3]);
                sts128(ya + sty_r + 1024, i[0], i[1], i[2], i[3]);
                sts128(ya + sty_i, i[0], i[1], i[2], i[3]);
                sts128(ya + sty_i + 1024, n[0], n[1], n[2], n[3]);
                sts128(xa + stx, xr0[0], xr0[1], xr0[2], xr0[3]);
                sts128(xa + stx + 1024, xi0[0], xi0[1], xi0[2], xi0[3]);
                if (nx > 1) {
                    sts128(xa + 8192 + stx, xr1[0], xr1[1], xr1[2], xr1[3]);
                    sts128(xa + 8192 + stx + 1024, xi1[0], xi1[1], xi1[2], xi1[3]);
                }
                fence_proxy_async();
                mbar_arrive(full_op(os));
            }
            if (!ok) break;

            // -------------------------------------------------- epilogue
            if (!mbar_wait(acc_full, acc_phase, abort_flag)) {
                ok = false;
                break;
            }
            acc_phase ^= 1;
            tc_fence_after();
            const int q = warp & 3, h = warp >> 2;
            const int nb1 = cd->nb1;
            const int by = ty * 4 + q;
            int32_t *out = reinterpret_cast<int32_t *>(P.out_base + cd->out) + U.out_off;
            const int mode = U.split ? 2 : (P.accumulate ? 1 : 0);
            const int nblk = 2 * nx;  // x blocks per warp
#pragma unroll 1
            for (int jj = 0; jj < nblk; jj++) {
                const int j = h * nblk + jj;
                uint32_t re[32], im[32];
                const uint32_t taddr = tmem_base + ((uint32_t)(32 * q) << 16) + 32 * j;
                tmem_ld32(taddr, re);
                tmem_ld32(taddr + 256, im);
                tmem_wait_ld();
                const int bx = x0 * 4 + j;
                if (by >= nb1 || bx >= nb1 || bx < by) continue;
                const int64_t b = (int64_t)by * nb1 - (int64_t)by * (by - 1) / 2 + (bx - by);
                int32_t *dst = out + (b * 32 + lane) * 64;
#pragma unroll
                for (int k = 0; k < 32; k++) {
                    re[k] = (uint32_t)((int32_t)re[k] >> 4);
                    im[k] = (uint32_t)((int32_t)im[k] >> 4);
                    if (!P.ut) im[k] = 0u - im[k];
                }
                if (mode == 0) {
#pragma unroll
                    for (int k = 0; k < 32; k += 2)
                        *reinterpret_cast<int4 *>(dst + 2 * k) =
                            make_int4((int)re[k], (int)im[k], (int)re[k + 1], (int)im[k + 1]);
                } else if (mode == 1) {
#pragma unroll
                    for (int k = 0; k < 32; k += 2) {
                        int4 o = *reinterpret_cast<int4 *>(dst + 2 * k);
                        o.x = (int)((uint32_t)o.x + re[k]);
                        o.y = (int)((uint32_t)o.y + im[k]);
                        o.z = (int)((uint32_t)o.z + re[k + 1]);
                        o.w = (int)((uint32_t)o.w + im[k + 1]);
                        *reinterpret_cast<int4 *>(dst + 2 * k) = o;
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < 32; k++) {
                        atomicAdd(dst + 2 * k, (int)re[k]);
                        atomicAdd(dst + 2 * k + 1, (int)im[k]);
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(acc_empty);
        }
        if (!ok) {
            atomicOr(P.err, 0x40);
            *abort_flag = 1;
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == kMmaWarp) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                     "r"(kTmemCols)
                     : "memory");
    }
}

template <int MAP>
cudaError_t launch_map(const TcLaunch &L, const CUtensorMap *pmap, cudaStream_t st) {
    static bool attr_done = false;
    if (!attr_done) {
        cudaError_t e = cudaFuncSetAttribute(tc_correlate_kernel<MAP>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
        if (e != cudaSuccess) return e;
        attr_done = true;
    }
    KParams P;
    P.chans = L.chans;
    P.units = L.units;
    P.nunits = L.nunits;
    P.out_base = L.out_base;
    P.use_param_map = L.use_param_map;
    P.ut = L.ut;
    P.accumulate = L.accumulate;
    P.err = L.err;
    CUtensorMap dummy;
    memset(&dummy, 0, sizeof(dummy));
    tc_correlate_kernel<MAP><<<L.grid, kThreads, kSmemBytes, st>>>(pmap ? *pmap : dummy, P);
    return cudaGetLastError();
}

}  // namespace

bool tc_supported(int E, int T) { return E >= 32 && E % 32 == 0 && E <= 65536 && T >= 1; }

void tc_append_units(std::vector<Unit> &out, int chan, int E, int t_begin, int t_end, int tsplit,
                     long long out_off) {
    const int nt = (E + 127) / 128;
    const int span = t_end - t_begin;
    if (span <= 0) return;
    int splits = tsplit < 1 ? 1 : tsplit;
    int chunk = (span + splits - 1) / splits;
    chunk = (chunk + kStageSamples - 1) / kStageSamples * kStageSamples;
    if (chunk > kUnitMaxSamples) chunk = kUnitMaxSamples;
    splits = (span + chunk - 1) / chunk;
    for (int ty = 0; ty < nt; ty++) {
        for (int x0 = ty; x0 < nt; x0 += 2) {
            const int nx = std::min(2, nt - x0);
            for (int s = 0; s < splits; s++) {
                Unit u;
                u.chan = chan;
                u.tyx = ty | (x0 << 10) | (nx << 20);
                u.t0 = t_begin + s * chunk;
                u.t1 = std::min(t_end, u.t0 + chunk);
                u.out_off = out_off;
                u.split = splits > 1 ? 1 : 0;
                u.cost = ((u.t1 - u.t0 + kStageSamples - 1) / kStageSamples) * (nx + 1);
                out.push_back(u);
            }
        }
    }
}

void tc_sort_units(std::vector<Unit> &u) {
    std::stable_sort(u.begin(), u.end(),
                     [](const Unit &a, const Unit &b) { return a.cost > b.cost; });
}

int tc_encode_map(CUtensorMap *m, const void *base, int E, int channels, int64_t samples,
                  int64_t chan_stride, int64_t sample_stride) {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !p)
            return -1;
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    cuuint64_t dims[3] = {(cuuint64_t)E, (cuuint64_t)channels, (cuuint64_t)samples};
    cuuint64_t strides[2] = {(cuuint64_t)chan_stride, (cuuint64_t)sample_stride};
    cuuint32_t box[3] = {128, 1, (cuuint32_t)kStageSamples};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void *>(base), dims, strides,
                    box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : (int)r;
}

cudaError_t tc_launch(const TcLaunch &L, const CUtensorMap *param_map, cudaStream_t st) {
    if (L.nunits <= 0) return cudaSuccess;
    if (L.grid <= 0) return cudaErrorInvalidValue;
    switch (L.map) {
    case MAP_EXACT: return launch_map<MAP_EXACT>(L, param_map, st);
    case MAP_CONF: return launch_map<MAP_CONF>(L, param_map, st);
    default: return launch_map<MAP_PACKED>(L, param_map, st);
    }
}

}  // namespace chx
