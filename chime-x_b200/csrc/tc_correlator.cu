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
// and component.  One stage covers 32 samples, each component's four atoms
// contiguous (one MMA's K = 32 is one component over the stage's 32 samples):
//   y: atoms [R0 R1 R2 R3 | I0 I1 I2 I3 | N0 N1 N2 N3]   12 KiB
//   x: per 128-element slice [X0 X1 X2 X3 | Y0 Y1 Y2 Y3] 8 KiB per slice
// (digit = 8-sample block).  Four MMAs per stage, alternating accumulators so
// that consecutive MMAs are independent:
//   Re += R.X    Im += I.X    Re += I.Y    Im += N.Y
// Every operand row is stored once (a layout interleaving R and I per
// 8-sample block needed the I rows twice: 16 KiB of y per stage, measured
// 3-4 % slower on the SM-pair kernel, whose shared-memory traffic bounds it).
//
// Roles (576 threads, one persistent CTA per SM; each CTA works through its
// own contiguous range of the unit table, assigned on the host by cost):
//   warps 0-15 unpack: read packed bytes from the TMA ring, convert with SWAR
//              logic, store swizzled operand rows (warps 0-7 the y tile,
//              8-15 the x tile); then the epilogue (TMEM -> block layout).
//   warp 16    TMA producer: packed y and x tiles, 32 samples per stage.
//   warp 17    TMEM allocation and the single-thread MMA issue loop, which
//              consumes stages in pairs (eight MMAs alternating between the
//              Re and Im accumulators, one commit): committing after every
//              few MMAs stalls the tensor pipe, and back-to-back MMAs into one
//              accumulator wait for each other's TMEM update.
// Every wait is bounded (globaltimer): on timeout the CTA records an error
// code in the caller's error word, drains its MMAs and TMA loads and returns.
#include "tc_common.cuh"

#include <cudaTypedefs.h>
#include <string.h>

#include <algorithm>
#include <functional>
#include <queue>

namespace chx {

namespace {

using namespace tc;

constexpr int kStageSamples = kUnitStageSamples;
constexpr int kOpStages = 4;    // operand ring
constexpr int kPkStages = 6;    // packed-tile ring
constexpr int kYOpBytes = 16 * 1024;  // 12 KiB of operands; the slots also hold the epilogue staging
constexpr int kXOpBytes = 16 * 1024;
constexpr int kPkYBytes = kStageSamples * 128;      // 4 KiB
constexpr int kPkXBytes = 2 * kPkYBytes;            // 8 KiB
constexpr int kUnpackWarps = 16;
constexpr int kUnpackThreads = kUnpackWarps * 32;
constexpr int kProducerWarp = 16;
constexpr int kMmaWarp = 17;
constexpr int kThreads = 576;
constexpr int kTmemCols = 512;

constexpr int kOffOpY = 0;
constexpr int kOffOpX = kOffOpY + kOpStages * kYOpBytes;
constexpr int kOffPkY = kOffOpX + kOpStages * kXOpBytes;
constexpr int kOffPkX = kOffPkY + kPkStages * kPkYBytes;
constexpr int kOffBars = kOffPkX + kPkStages * kPkXBytes;
constexpr int kSmemBytes = kOffBars + 256 + 1024;
// Epilogue staging (two 4 KiB tiles per unpack warp) reuses the operand slots.
constexpr int kEpiTiles = 2;
static_assert(kUnpackWarps * 8192 <= kOffPkY - kOffOpY, "epilogue staging");

struct KParams {
    const ChanDesc *chans;
    const Unit *units;
    int nunits;
    const int *cta_offsets;  // CTA b takes units [cta_offsets[b], cta_offsets[b+1])
    uint64_t out_base;
    int use_param_map;
    int ut;
    int accumulate;
    int *err;
};

template <int MAP>
__global__ void __launch_bounds__(kThreads, 1)
tc_correlate_kernel(const __grid_constant__ CUtensorMap pmap,
                    const __grid_constant__ CUtensorMap pomap, const KParams P) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const uint32_t sbase = smem_u32(smem);
    const uint32_t op_y = sbase + kOffOpY, op_x = sbase + kOffOpX;
    const uint32_t pk_y = sbase + kOffPkY, pk_x = sbase + kOffPkX;
    const uint32_t bars = sbase + kOffBars;
    // barrier map (8 bytes each)
    auto full_pk = [&](int s) { return bars + 8 * s; };
    auto empty_pk = [&](int s) { return bars + 8 * (kPkStages + s); };
    auto full_op = [&](int s) { return bars + 8 * (2 * kPkStages + s); };
    auto empty_pair = [&](int s) { return bars + 8 * (2 * kPkStages + kOpStages + s); };
    const uint32_t acc_full = bars + 8 * (2 * kPkStages + kOpStages + 2);
    const uint32_t acc_empty = acc_full + 8;
    const uint32_t drain = acc_full + 16;
    volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(
        smem + kOffBars + 8 * (2 * kPkStages + kOpStages + 5));
    const uint32_t epi_done = bars + 8 * (2 * kPkStages + kOpStages + 6);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kPkStages; s++) {
            mbar_init(full_pk(s), 1);
            mbar_init(empty_pk(s), kUnpackWarps);
        }
        for (int s = 0; s < kOpStages; s++) mbar_init(full_op(s), kUnpackWarps);
        mbar_init(empty_pair(0), 1);
        mbar_init(empty_pair(1), 1);
        mbar_init(acc_full, 1);
        mbar_init(acc_empty, kUnpackThreads);
        mbar_init(drain, 1);
        mbar_init(epi_done, kUnpackWarps);
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

    // This CTA's units: a contiguous range of the table, balanced on the host.
    const int first = P.cta_offsets[blockIdx.x], last = P.cta_offsets[blockIdx.x + 1];

    if (warp == kProducerWarp) {
        // ------------------------------------------------------ TMA producer
        if (lane == 0) {
            uint32_t g = 0;  // stage counter (32 samples per stage)
            bool ok = true;
            for (int u = first; u < last && ok; u++) {
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
        // Stages are consumed in pairs (64 samples): eight MMAs alternating
        // between the Re and Im accumulators, then one commit releasing both
        // operand slots.
        if (lane == 0) {
            uint32_t gp = 0, acc_phase = 0;  // pair counter (pair gp uses slot gp & 1)
            bool ok = true;
            const bool b_signed = (MAP == MAP_EXACT);
            // per stage: y rows R, I, N and x rows X, Y (two 128-element
            // slices 8 KiB apart), 32 samples each
            const uint64_t dR = sdesc(op_y, 1024, 1024), dI = sdesc(op_y + 4096, 1024, 1024);
            const uint64_t dN = sdesc(op_y + 8192, 1024, 1024);
            const uint64_t dX = sdesc(op_x, 8192, 1024), dY = sdesc(op_x + 4096, 8192, 1024);
            for (int u = first; u < last && ok; u++) {
                const Unit U = P.units[u];
                const int nx = (U.tyx >> 20) & 3;
                const uint32_t idesc = idesc_i8(128 * nx, b_signed);
                const int nst = (U.t1 - U.t0 + kStageSamples - 1) / kStageSamples;
                const int npair = (nst + 1) / 2;
                // the epilogue of the previous unit must have drained TMEM
                if (!mbar_wait(acc_empty, acc_phase ^ 1, abort_flag)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                for (int ip = 0; ip < npair; ip++, gp++) {
                    const int ps = gp & 1;
                    const uint32_t ph = (gp >> 1) & 1;
                    const int nin = (2 * ip + 1 < nst) ? 2 : 1;  // stages in this pair
                    if (!mbar_wait(full_op(2 * ps), ph, abort_flag) ||
                        !mbar_wait(full_op(2 * ps + 1), ph, abort_flag)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t acc = (ip > 0) ? 1u : 0u;
                    // Re and Im MMAs alternate: consecutive MMAs then go to
                    // different accumulators and need not wait for each
                    // other's TMEM update.
                    for (int j = 0; j < nin; j++) {
                        const int s = 2 * ps + j;
                        const uint64_t so_y = (uint64_t)((s * kYOpBytes) >> 4);
                        const uint64_t so_x = (uint64_t)((s * kXOpBytes) >> 4);
                        const uint32_t a0 = (j > 0) ? 1u : acc;
                        mma_i8(tmem_base, dR + so_y, dX + so_x, idesc, a0);        // Re += R X
                        mma_i8(tmem_base + 256, dI + so_y, dX + so_x, idesc, a0);  // Im += I X
                        mma_i8(tmem_base, dI + so_y, dY + so_x, idesc, 1u);        // Re += I Y
                        mma_i8(tmem_base + 256, dN + so_y, dY + so_x, idesc, 1u);  // Im += N Y
                    }
                    mma_commit(empty_pair(ps));
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
            // No arrival may be pending when the CTA retires: wait for the
            // last phase committed on each pair barrier.
            for (uint32_t k = 0; k < 2; k++) {
                const uint32_t ncommit = gp > k ? (gp - 1 - k) / 2 + 1 : 0;  // commits on slot k
                if (ncommit) mbar_wait_drain(empty_pair(k), (ncommit - 1) & 1);
            }
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------ unpack + epilogue
        // Threads 0..255 convert the y tile (one 16-element chunk of one
        // sample each), threads 256..511 the x tile (the same chunk position
        // in each 128-element slice).
        const int tid = threadIdx.x;  // 0..511
        const bool is_y = tid < 256;
        const int c = tid & 255;
        const int sy = c >> 3, gy = c & 7;
        const uint32_t ry = (uint32_t)(sy & 7), by8 = (uint32_t)(sy >> 3);
        const uint32_t ldoff = (uint32_t)(sy * 128 + gy * 16);
        const uint32_t st_a = by8 * 1024 + swz(ry, gy);  // R (y) or X (x); I / Y at +4K, N at +8K
        uint32_t g = 0, gp_base = 0, acc_phase = 0, epi_phase = 0;
        bool ok = true;
        // Epilogue staging: 8 KiB per warp inside the operand slots, which
        // are idle from the accumulator commit until the next unit's unpack.
        const uint32_t stage = op_y + (uint32_t)warp * 8192u;
        for (int u = first; u < last && ok; u++) {
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
                uint32_t v0[4], v1[4], v2[4], v3[4];  // y: R, I, N; x: X0, Y0, X1, Y1
                if (is_y) {
                    const uint4 w = lds128(pk_y + ps * kPkYBytes + ldoff);
                    yconv<MAP>(w.x, v0[0], v1[0], v2[0]);
                    yconv<MAP>(w.y, v0[1], v1[1], v2[1]);
                    yconv<MAP>(w.z, v0[2], v1[2], v2[2]);
                    yconv<MAP>(w.w, v0[3], v1[3], v2[3]);
#pragma unroll
                    for (int k = 0; k < 4; k++) v3[k] = 0u;
                } else {
                    const uint4 w0 = lds128(pk_x + ps * kPkXBytes + ldoff);
                    uint4 w1 = make_uint4(0, 0, 0, 0);
                    if (nx > 1) w1 = lds128(pk_x + ps * kPkXBytes + kPkYBytes + ldoff);
                    xconv<MAP>(w0.x, v0[0], v1[0]);
                    xconv<MAP>(w0.y, v0[1], v1[1]);
                    xconv<MAP>(w0.z, v0[2], v1[2]);
                    xconv<MAP>(w0.w, v0[3], v1[3]);
                    xconv<MAP>(w1.x, v2[0], v3[0]);
                    xconv<MAP>(w1.y, v2[1], v3[1]);
                    xconv<MAP>(w1.z, v2[2], v3[2]);
                    xconv<MAP>(w1.w, v2[3], v3[3]);
                }
                if (!valid) {  // samples outside the unit contribute zero
#pragma unroll
                    for (int k = 0; k < 4; k++) v0[k] = v1[k] = v2[k] = v3[k] = 0u;
                }
                // The converted registers depend on the loaded words, and
                // __syncwarp orders every lane before lane 0's arrive: one
                // arrival per warp frees the packed slot.
                __syncwarp();
                if (lane == 0) mbar_arrive(empty_pk(ps));

                // operand slot of stage `it`: pair (gp_base + it/2), half it&1
                const uint32_t gpair = gp_base + (uint32_t)(it >> 1);
                const int os = 2 * (int)(gpair & 1) + (it & 1);
                if (!mbar_wait(empty_pair(gpair & 1), ((gpair >> 1) & 1) ^ 1, abort_flag)) {
                    ok = false;
                    break;
                }
                // a pair cut short by an odd stage count still completes a
                // phase on its second slot, keeping every slot's parity in step
                const bool lone = (it == nst - 1) && ((it & 1) == 0);
                if (is_y) {
                    const uint32_t ya = op_y + os * kYOpBytes + st_a;
                    sts128(ya, v0[0], v0[1], v0[2], v0[3]);                // R
                    sts128(ya + 4096, v1[0], v1[1], v1[2], v1[3]);  // I
                    sts128(ya + 8192, v2[0], v2[1], v2[2], v2[3]);  // N
                } else {
                    const uint32_t xa = op_x + os * kXOpBytes + st_a;
                    sts128(xa, v0[0], v0[1], v0[2], v0[3]);  // X slice 0
                    sts128(xa + 4096, v1[0], v1[1], v1[2], v1[3]);  // Y slice 0
                    if (nx > 1) {
                        sts128(xa + 8192, v2[0], v2[1], v2[2], v2[3]);         // X slice 1
                        sts128(xa + 8192 + 4096, v3[0], v3[1], v3[2], v3[3]);  // Y slice 1
                    }
                }
                fence_proxy_async();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(full_op(os));
                    if (lone) mbar_arrive(full_op(os + 1));
                }
            }
            if (!ok) break;
            gp_base += (uint32_t)((nst + 1) / 2);

            // -------------------------------------------------- epilogue
            if (!mbar_wait(acc_full, acc_phase, abort_flag)) {
                ok = false;
                break;
            }
            acc_phase ^= 1;
            tc_fence_after();
            const int q = warp & 3, h = warp >> 2;  // lane quarter, column group
            const int nb1 = cd->nb1;
            const int by = ty * 4 + q;
            // Split units (other units cover the same cells' other sample ranges)
            // add like accumulate mode: every element of a TMA reduce-add is an
            // individual relaxed reduction at gpu scope, so concurrent units meet
            // exactly in the zeroed (or accumulating) output.
            const bool add = U.split || P.accumulate;
            const CUtensorMap *omap = P.use_param_map ? &pomap : &cd->omap;
            const int row0 = cd->orow + (int)(U.out_off >> 6);
            uint32_t nchunk = 0;
#pragma unroll 1
            for (int jj = 0; jj < nx; jj++) {
                const int j = h * nx + jj;  // 32-column x block
                const int bx = x0 * 4 + j;
                if (by >= nb1 || bx >= nb1 || bx < by) continue;  // warp-uniform
                const int64_t b = (int64_t)by * nb1 - (int64_t)by * (by - 1) / 2 + (bx - by);
                const uint32_t taddr = tmem_base + ((uint32_t)(32 * q) << 16) + 32 * j;
#pragma unroll 1
                for (int half = 0; half < 2; half++) {
                    // Stage the 32 x 32-word tile (rows = lanes) in two
                    // 8-column parts, then hand it to TMA.
                    const uint32_t tile = stage + (nchunk % (uint32_t)kEpiTiles) * 4096u;
                    if (lane == 0) bulk_wait_read<kEpiTiles - 1>();
                    __syncwarp();
#pragma unroll
                    for (int part = 0; part < 2; part++) {
                        uint32_t re[8], im[8];
                        tmem_ld8(taddr + 16 * half + 8 * part, re);
                        tmem_ld8(taddr + 256 + 16 * half + 8 * part, im);
                        tmem_wait_ld();
#pragma unroll
                        for (int k = 0; k < 8; k++) {
                            re[k] = (uint32_t)((int32_t)re[k] >> 4);
                            im[k] = (uint32_t)((int32_t)im[k] >> 4);
                            if (!P.ut) im[k] = 0u - im[k];
                        }
                        stage_row_half(tile, lane, part, re, im);
                    }
                    fence_proxy_async();
                    __syncwarp();
                    if (lane == 0) {
                        const int y = row0 + (int)b * 32;
                        if (add)
                            tma_add_2d(omap, tile, 32 * half, y);
                        else
                            tma_store_2d(omap, tile, 32 * half, y);
                        bulk_commit();
                    }
                    nchunk++;
                }
            }
            if (lane == 0) bulk_wait_read<0>();  // staging read by TMA
            tc_fence_before();
            __syncwarp();
            mbar_arrive(acc_empty);
            if (lane == 0) mbar_arrive(epi_done);
            // The next unit's unpack overwrites the staging tiles: wait until
            // every warp's tiles have been read.
            if (!mbar_wait(epi_done, epi_phase, abort_flag)) {
                ok = false;
                break;
            }
            epi_phase ^= 1;
        }
        if (!ok) {
            atomicOr(P.err, 0x40);
            *abort_flag = 1;
        }
        if (lane == 0) bulk_wait_all();  // output tiles written
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
cudaError_t launch_map(const TcLaunch &L, const CUtensorMap *pmap, const CUtensorMap *pomap,
                       cudaStream_t st) {
    // The shared-memory opt-in is a per-device function attribute.
    static bool attr_done[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr_done[dev]) {
        e = cudaFuncSetAttribute(tc_correlate_kernel<MAP>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
        if (e != cudaSuccess) return e;
        attr_done[dev] = true;
    }
    KParams P;
    P.chans = L.chans;
    P.units = L.units;
    P.nunits = L.nunits;
    P.cta_offsets = L.cta_offsets;
    P.out_base = L.out_base;
    P.use_param_map = L.use_param_map;
    P.ut = L.ut;
    P.accumulate = L.accumulate;
    P.err = L.err;
    CUtensorMap dummy;
    memset(&dummy, 0, sizeof(dummy));
    tc_correlate_kernel<MAP><<<L.grid, kThreads, kSmemBytes, st>>>(
        pmap ? *pmap : dummy, pomap ? *pomap : dummy, P);
    return cudaGetLastError();
}

}  // namespace

// The SM-pair kernel's 256-element units cover an odd number of 128-element
// tiles with a half-empty row and column of units, whose missing tile's work
// is done in vain; the one-SM kernel wastes none but converts two x tiles per
// y tile on one SM.  Measured on B200 with the automatic split (T = 16384,
// F = 8, TOPS, SM pair / one SM): E = 1920 2427 / 2024, 1664 1998 / 1775,
// 1408 2051 / 1953, 1152 1903 / 1611, 896 1514 / 1473, 640 1418 / 1449,
// 384 953 / 732, and 2048 2741 / 2133.  The SM pair is the default from two
// tiles up; a single tile (E <= 128) would leave three quarters of its one
// pair unit empty, so it goes to the one-SM kernel.  Both stay available as a
// tile option and to the autotuner.
int tc_default_tile(int E) {
    const int nt = (E + 127) / 128;
    return nt >= 2 ? kTile2Sm : kTile1Sm;
}

void tc_append_tile_units(int tile, std::vector<Unit> &out, int chan, int E, int t_begin,
                          int t_end, int tsplit, long long out_off) {
    if (tile == kTile2Sm)
        tc_append_pair_units(out, chan, E, t_begin, t_end, tsplit, out_off);
    else
        tc_append_units(out, chan, E, t_begin, t_end, tsplit, out_off);
}

int tc_tile_slots(int tile, int sm_count) {
    return tile == kTile2Sm ? sm_count / 2 : sm_count;
}

cudaError_t tc_tile_launch(int tile, const TcLaunch &L, const CUtensorMap *param_map,
                           const CUtensorMap *param_omap, cudaStream_t st) {
    if (tile == kTile2Sm) return tc_pair_launch(L, param_map, param_omap, st);
    return tc_launch(L, param_map, param_omap, st);
}

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
                u.cost = unit_cost(false, u.t0, u.t1, nx);
                out.push_back(u);
            }
        }
    }
}

void tc_schedule(std::vector<Unit> &u, int grid, std::vector<int> &offsets) {
    // Longest-processing-time-first: hand each unit, largest first, to the
    // CTA with the least assigned cost, then store the units CTA by CTA.  For
    // the one-SM kernel this puts every channel's cheaper one-x-tile units at
    // the end, where they read the channels' samples from DRAM a second time
    // (E=1920, F=8: 2.4x the input).  Orders that keep a channel's units
    // together read less (1.65x by sample range, then enumeration order) but
    // balance the CTAs worse and measured slower (1825 vs 2033 TOPS), and
    // ordering each CTA's units by channel read more (2.5x).
    std::stable_sort(u.begin(), u.end(),
                     [](const Unit &a, const Unit &b) { return a.cost > b.cost; });
    if (grid < 1) grid = 1;
    std::vector<long long> load(grid, 0);
    std::vector<int> owner(u.size());
    std::vector<std::pair<long long, int>> heap;  // (load, cta), min-heap
    heap.reserve(grid);
    for (int b = 0; b < grid; b++) heap.push_back({0, b});
    auto cmp = [](const std::pair<long long, int> &a, const std::pair<long long, int> &b) {
        return a.first != b.first ? a.first > b.first : a.second > b.second;
    };
    std::make_heap(heap.begin(), heap.end(), cmp);
    for (size_t i = 0; i < u.size(); i++) {
        std::pop_heap(heap.begin(), heap.end(), cmp);
        auto &top = heap.back();
        owner[i] = top.second;
        top.first += u[i].cost;
        std::push_heap(heap.begin(), heap.end(), cmp);
    }
    offsets.assign(grid + 1, 0);
    for (size_t i = 0; i < u.size(); i++) offsets[owner[i] + 1]++;
    for (int b = 0; b < grid; b++) offsets[b + 1] += offsets[b];
    std::vector<int> fill(offsets.begin(), offsets.end() - 1);
    std::vector<Unit> out(u.size());
    for (size_t i = 0; i < u.size(); i++) out[fill[owner[i]]++] = u[i];
    u.swap(out);
}

long long tc_estimate_makespan(const std::vector<Unit> &u, int grid, int handoff_stages) {
    if (grid < 1) grid = 1;
    std::vector<long long> cost(u.size());
    for (size_t i = 0; i < u.size(); i++) {
        const long long st = std::max(1, (u[i].t1 - u[i].t0 + kStageSamples - 1) / kStageSamples);
        cost[i] = u[i].cost + (long long)handoff_stages * u[i].cost / st;
    }
    std::sort(cost.begin(), cost.end(), std::greater<long long>());
    std::priority_queue<long long, std::vector<long long>, std::greater<long long>> load;
    for (int b = 0; b < grid; b++) load.push(0);
    long long span = 0;
    for (long long c : cost) {
        const long long l = load.top() + c;
        load.pop();
        load.push(l);
        span = std::max(span, l);
    }
    return span;
}

int tc_choose_split(int tile, int sm_count,
                    const std::function<void(int, std::vector<Unit> &)> &build) {
    // A unit's accumulator hand-off costs about as much as 11 of its stages in
    // the SM-pair kernel (measured on B200: ~9,400 cycles against ~850 per
    // stage) and about 16 in the one-SM kernel, whose unpack warps run the
    // epilogue themselves.  Splitting a channel's samples therefore pays only
    // while it fills idle SMs.  With these overheads the estimate came within
    // 2 % of the best measured split of every shape tried (E = 256-2048,
    // F = 1-16, T = 16384; e.g. E = 1024, F = 2: 7 splits, 1551 vs 598 TOPS
    // unsplit; E = 2048, F = 8: no split).  A split must win by 3 % to pay for
    // zeroing the output and for the reduce-adds.
    const int handoff_stages = tile == kTile2Sm ? 11 : 16;
    const int grid_slots = tc_tile_slots(tile, sm_count);
    long long best = -1;
    int best_k = 1;
    size_t last_n = 0;
    for (int k = 1; k <= 8; k++) {
        std::vector<Unit> units;
        build(k, units);
        if (units.empty()) return 1;
        // Eight or more waves of unsplit units leave at most about an eighth
        // of a wave idle, less than the hand-offs that splitting adds.
        if (k == 1 && units.size() >= (size_t)8 * std::max(1, grid_slots)) return 1;
        // Ranges are rounded to whole stages: skip splits that cut the same way.
        if (units.size() == last_n) continue;
        last_n = units.size();
        const int grid = (int)std::min<size_t>(units.size(), (size_t)std::max(1, grid_slots));
        const long long span = tc_estimate_makespan(units, grid, handoff_stages);
        if (best < 0 || (k == 1 ? span < best : span * 100 < best * 97)) {
            best = span;
            best_k = k;
        }
    }
    return best_k;
}

int tc_auto_split(int tile, int E, int F, int T, int sm_count) {
    return tc_choose_split(tile, sm_count, [&](int k, std::vector<Unit> &units) {
        for (int f = 0; f < F; f++) tc_append_tile_units(tile, units, f, E, 0, T, k, 0);
    });
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

int tc_encode_out_map(CUtensorMap *m, void *base, int64_t rows) {
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
    if (!tc_out_rows_ok(rows) || (reinterpret_cast<uintptr_t>(base) & 15)) return -2;
    cuuint64_t dims[2] = {64, (cuuint64_t)rows};
    cuuint64_t strides[1] = {256};
    cuuint32_t box[2] = {32, 32};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_INT32, 2, base, dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : (int)r;
}

cudaError_t tc_launch(const TcLaunch &L, const CUtensorMap *param_map,
                      const CUtensorMap *param_omap, cudaStream_t st) {
    if (L.nunits <= 0) return cudaSuccess;
    if (L.grid <= 0) return cudaErrorInvalidValue;
    if (L.use_param_map && (!param_map || !param_omap)) return cudaErrorInvalidValue;
    switch (L.map) {
    case MAP_EXACT: return launch_map<MAP_EXACT>(L, param_map, param_omap, st);
    case MAP_CONF: return launch_map<MAP_CONF>(L, param_map, param_omap, st);
    default: return launch_map<MAP_PACKED>(L, param_map, param_omap, st);
    }
}

}  // namespace chx
