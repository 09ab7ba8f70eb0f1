// tc_common.cuh -- PTX helpers and nibble conversions shared by the
// tensor-core correlator kernels (tcgen05, TMA, mbarrier, SWAR unpack).
#pragma once

#include "chimex_internal.h"

namespace chx {
namespace tc {

constexpr uint64_t kWaitLimitNs = 2000000000ull;  // bounded waits: 2 s

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
static __device__ __noinline__ bool mbar_wait_slow(uint32_t bar, uint32_t parity,
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
static __device__ __noinline__ bool mbar_wait_drain(uint32_t bar, uint32_t parity) {
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

// TMA: 2-D tile {32 words, 32 rows} of the block output from shared memory
// (128-byte swizzled), stored or added (s32) into global memory.  One thread
// issues it; completion is tracked with the issuing thread's bulk groups.
__device__ __forceinline__ void tma_store_2d(const CUtensorMap *map, uint32_t src, int x, int y) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::
                     "l"(reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(src)
                 : "memory");
}
__device__ __forceinline__ void tma_add_2d(const CUtensorMap *map, uint32_t src, int x, int y) {
    asm volatile(
        "cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.tile.bulk_group"
        " [%0, {%1, %2}], [%3];" ::"l"(reinterpret_cast<uint64_t>(map)),
        "r"(x), "r"(y), "r"(src)
        : "memory");
}
__device__ __forceinline__ void bulk_commit() {
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// Waits until at most N of this thread's bulk groups still read shared memory.
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
// Waits until every bulk group of this thread has completed its writes.
__device__ __forceinline__ void bulk_wait_all() {
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
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

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7])
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

// Half of one row (lane) of a 32 x 32-word staging tile: (Re, Im) pairs
// 8*part .. 8*part+7 as the 16-byte chunks 4*part .. 4*part+3, chunk c at
// position c ^ (row & 7) (the 128-byte swizzle of the output tensor map), so
// the warp's stores spread over every bank.
__device__ __forceinline__ void stage_row_half(uint32_t tile, int row, int part,
                                               const uint32_t (&re)[8], const uint32_t (&im)[8]) {
    const uint32_t base = tile + (uint32_t)row * 128u;
    const uint32_t x = (uint32_t)(row & 7);
#pragma unroll
    for (int c = 0; c < 4; c++)
        sts128(base + ((((uint32_t)(4 * part + c)) ^ x) << 4), re[2 * c], im[2 * c],
               re[2 * c + 1], im[2 * c + 1]);
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


}  // namespace tc
}  // namespace chx
