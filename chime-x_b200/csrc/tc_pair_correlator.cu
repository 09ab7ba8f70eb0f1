// tc_pair_correlator.cu -- 2-SM (cta_group::2) variant of the tcgen05
// kind::i8 correlator.
//
// A cluster of two CTAs computes a 256 x 256-element unit: CTA r holds y tile
// 2*ty2 + r (its 128 rows of A, M = 256 over the pair) and x tile 2*tx2 + r
// (its 128 columns of B, N = 256 over the pair).  One thread of CTA 0 issues
// tcgen05.mma.cta_group::2; each SM's tensor core reads only its own A rows
// and B half from its own shared memory, so per SM the unpack converts one
// 128-element x tile instead of two and the operand reads per MAC drop by a
// third, for the same tensor work per SM as the 1-SM kernel.  Each CTA's TMEM
// receives its 128 rows x 256 columns of Re (columns 0-255) and Im (256-511).
//
// Operand formulation, layout, value maps and the stage-pair MMA order are the
// 1-SM kernel's (tc_correlator.cu); per CTA a 32-sample stage holds y
// [R0 R1 R2 R3 | I0 I1 I2 I3 | N0 N1 N2 N3] (12 KiB) and x
// [X0 X1 X2 X3 | Y0 Y1 Y2 Y3] (8 KiB), each part an 8-sample atom.
//
// Warps: 0-15 unpack (0-7 y, 8-15 x), 16 TMA producer, 17 MMA issuer (CTA 0),
// 18-25 epilogue.  The epilogue warps drain the accumulators of one unit while
// the unpack warps convert the next; each 32 x 32-word output tile goes from
// TMEM through a swizzled staging tile in shared memory to a TMA store (or
// reduce-add) into the block buffer.
//
// Synchronisation across the pair:
//   full_pair[p] in CTA 0; every unpack warp of both CTAs arrives once per
//                stage pair (one lane, after its lanes' proxy fences) -> the
//                MMA thread waits.
//   empty_pair   in both CTAs; CTA 0's commit arrives on both (multicast).
//   acc_full     in both CTAs; CTA 0's commit arrives on both (multicast).
//   acc_empty    in CTA 0; every epilogue warp of both CTAs arrives.
// TMA loads, the packed ring and its barriers are local to each CTA.  Both
// CTAs meet at cluster barriers after set-up and before exit, so no remote
// arrival can land after a CTA retires.  Every wait is bounded.
#include "tc_cluster.cuh"

#include <cudaTypedefs.h>
#include <string.h>

#include <algorithm>

namespace chx {

namespace {

using namespace tc;

constexpr int kStageSamples = kUnitStageSamples;
constexpr int kOpSlots = 4;     // 2 stage pairs
constexpr int kPairs = kOpSlots / 2;
constexpr int kPkStages = 4;
constexpr int kYOpBytes = 12 * 1024;
constexpr int kXOpBytes = 8 * 1024;
constexpr int kPkBytes = kStageSamples * 128;  // one 128-element tile, 4 KiB
constexpr int kUnpackWarps = 16;
constexpr int kProducerWarp = 16;
constexpr int kMmaWarp = 17;
constexpr int kEpiWarp0 = 18;   // epilogue warps from here on, lane quarter = warp % 4
constexpr int kEpiWarps = 8;    // 4 or 8: each warp drains 8 / (kEpiWarps / 4) column blocks
constexpr int kEpiTiles = 3;    // 4 KiB output staging tiles per epilogue warp
constexpr int kEpiStageBytes = kEpiTiles * 4096;
constexpr int kEpiBlocks = 8 / (kEpiWarps / 4);
constexpr int kThreads = (kEpiWarp0 + kEpiWarps) * 32;
static_assert(kEpiWarps == 4 || kEpiWarps == 8, "epilogue warps");
constexpr int kTmemCols = 512;

constexpr int kOffOpY = 0;
constexpr int kOffOpX = kOffOpY + kOpSlots * kYOpBytes;
constexpr int kOffPkY = kOffOpX + kOpSlots * kXOpBytes;
constexpr int kOffPkX = kOffPkY + kPkStages * kPkBytes;
constexpr int kOffStage = kOffPkX + kPkStages * kPkBytes;
constexpr int kOffBars = kOffStage + kEpiWarps * kEpiStageBytes;
constexpr int kSmemBytes = kOffBars + 256 + 1024;
static_assert(kSmemBytes <= 232448, "shared memory per CTA");

// Barrier offsets inside the barrier block (8 bytes each).
constexpr int kBarFullPk = 0;
constexpr int kBarEmptyPk = kBarFullPk + kPkStages;
constexpr int kBarFullPair = kBarEmptyPk + kPkStages;
constexpr int kBarEmptyPair = kBarFullPair + kPairs;
constexpr int kBarAccFull = kBarEmptyPair + kPairs;
constexpr int kBarAccEmpty = kBarAccFull + 1;
constexpr int kBarDrain = kBarAccEmpty + 1;
constexpr int kBarCount = kBarDrain + 1;
static_assert(kBarCount * 8 + 8 <= 256, "barrier block");

struct KParams {
    const ChanDesc *chans;
    const Unit *units;
    const int *cluster_offsets;  // cluster c takes units [off[c], off[c+1])
    uint64_t out_base;
    int use_param_map;
    int ut;
    int accumulate;
    int *err;
};

template <int MAP>
__global__ void __launch_bounds__(kThreads, 1)
tc_pair_kernel(const __grid_constant__ CUtensorMap pmap, const __grid_constant__ CUtensorMap pomap,
               const KParams P) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const uint32_t sbase = smem_u32(smem);
    const uint32_t op_y = sbase + kOffOpY, op_x = sbase + kOffOpX;
    const uint32_t pk_y = sbase + kOffPkY, pk_x = sbase + kOffPkX;
    const uint32_t bars = sbase + kOffBars;
    auto bar = [&](int i) { return bars + 8 * i; };
    volatile uint32_t *tmem_slot =
        reinterpret_cast<volatile uint32_t *>(smem + kOffBars + 8 * kBarCount);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_rank();
    const int cluster = blockIdx.x >> 1;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kPkStages; s++) {
            mbar_init(bar(kBarFullPk + s), 1);
            mbar_init(bar(kBarEmptyPk + s), kUnpackWarps);
        }
        for (int s = 0; s < kPairs; s++) mbar_init(bar(kBarFullPair + s), 2 * kUnpackWarps);
        for (int s = 0; s < kPairs; s++) mbar_init(bar(kBarEmptyPair + s), 1);
        mbar_init(bar(kBarAccFull), 1);
        mbar_init(bar(kBarAccEmpty), 2 * kEpiWarps);
        mbar_init(bar(kBarDrain), 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == kMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32((const void *)tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync();  // barriers of both CTAs initialised, TMEM allocated
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    const int first = P.cluster_offsets[cluster], last = P.cluster_offsets[cluster + 1];

    if (warp == kProducerWarp) {
        // ------------------------------------------------- TMA producer (both CTAs)
        if (lane == 0) {
            uint32_t g = 0;
            bool ok = true;
            for (int u = first; u < last && ok; u++) {
                const Unit U = P.units[u];
                const ChanDesc *cd = P.chans + U.chan;
                const CUtensorMap *map = P.use_param_map ? &pmap : &cd->map;
                const int fc = cd->fcoord;
                const int ty = 2 * (U.tyx & 1023) + (int)rank;
                const int tx = 2 * ((U.tyx >> 10) & 1023) + (int)rank;
                const int nst = (U.t1 - U.t0 + kStageSamples - 1) / kStageSamples;
                for (int it = 0; it < nst; it++, g++) {
                    const int s = g % kPkStages;
                    const uint32_t ph = (g / kPkStages) & 1;
                    if (!mbar_wait(bar(kBarEmptyPk + s), ph ^ 1, abort_flag)) {
                        ok = false;
                        break;
                    }
                    const int t = U.t0 + it * kStageSamples;
                    mbar_expect_tx(bar(kBarFullPk + s), 2 * kPkBytes);
                    tma_load_3d(pk_y + s * kPkBytes, map, ty * 128, fc, t, bar(kBarFullPk + s));
                    tma_load_3d(pk_x + s * kPkBytes, map, tx * 128, fc, t, bar(kBarFullPk + s));
                }
            }
            if (!ok) {
                atomicOr(P.err, 0x100);
                *abort_flag = 1;
            }
            const uint32_t issued = g;
            for (uint32_t k = (issued > (uint32_t)kPkStages ? issued - kPkStages : 0); k < issued;
                 k++)
                mbar_wait_drain(bar(kBarFullPk + (int)(k % kPkStages)), (k / kPkStages) & 1);
        }
        __syncwarp();
    } else if (warp == kMmaWarp) {
        // ------------------------------------------------- MMA issuer (CTA 0 only)
        if (lane == 0) {
            if (rank == 0) {
                uint32_t gp = 0, acc_phase = 0;
                bool ok = true;
                const bool b_signed = (MAP == MAP_EXACT);
                // M = 256 over the pair, N = 256 over the pair.
                const uint32_t idesc = (2u << 4) | (1u << 7) | ((b_signed ? 1u : 0u) << 10) |
                                       (1u << 15) | (1u << 16) | ((256u >> 3) << 17) |
                                       ((256u >> 4) << 24);
                // per stage: y rows R, I, N and x rows X, Y, 32 samples each
                const uint64_t dR = sdesc(op_y, 1024, 1024);
                const uint64_t dI = sdesc(op_y + 4096, 1024, 1024);
                const uint64_t dN = sdesc(op_y + 8192, 1024, 1024);
                const uint64_t dX = sdesc(op_x, 1024, 1024), dY = sdesc(op_x + 4096, 1024, 1024);
                for (int u = first; u < last && ok; u++) {
                    const Unit U = P.units[u];
                    const int nst = (U.t1 - U.t0 + kStageSamples - 1) / kStageSamples;
                    const int npair = (nst + 1) / 2;
                    if (!mbar_wait_cluster(bar(kBarAccEmpty), acc_phase ^ 1, abort_flag)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    for (int ip = 0; ip < npair; ip++, gp++) {
                        const int ps = (int)(gp % kPairs);
                        const uint32_t ph = (gp / kPairs) & 1;
                        const int nin = (2 * ip + 1 < nst) ? 2 : 1;
                        if (!mbar_wait_cluster(bar(kBarFullPair + ps), ph, abort_flag)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t acc = (ip > 0) ? 1u : 0u;
                        // Re and Im MMAs alternate: consecutive MMAs then go
                        // to different accumulators and need not wait for
                        // each other's TMEM update (8-9 % faster than four
                        // Re MMAs followed by four Im MMAs).
                        for (int j = 0; j < nin; j++) {
                            const int s = 2 * ps + j;
                            const uint64_t so_y = (uint64_t)((s * kYOpBytes) >> 4);
                            const uint64_t so_x = (uint64_t)((s * kXOpBytes) >> 4);
                            const uint32_t a0 = (j > 0) ? 1u : acc;
                            mma_i8_pair(tmem_base, dR + so_y, dX + so_x, idesc, a0);        // Re += R X
                            mma_i8_pair(tmem_base + 256, dI + so_y, dX + so_x, idesc, a0);  // Im += I X
                            mma_i8_pair(tmem_base, dI + so_y, dY + so_x, idesc, 1u);        // Re += I Y
                            mma_i8_pair(tmem_base + 256, dN + so_y, dY + so_x, idesc, 1u);  // Im += N Y
                        }
                        mma_commit_pair(bar(kBarEmptyPair + ps));
                    }
                    if (!ok) break;
                    mma_commit_pair(bar(kBarAccFull));
                    acc_phase ^= 1;
                }
                if (!ok) {
                    atomicOr(P.err, 0x200);
                    *abort_flag = 1;
                    asm volatile(
                        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64"
                        " [%0];" ::"r"(bar(kBarDrain))
                        : "memory");
                    mbar_wait_drain(bar(kBarDrain), 0);
                }
            }
        }
        __syncwarp();
    } else if (warp < kUnpackWarps) {
        // ------------------------------------------------- unpack (both CTAs)
        const int tid = threadIdx.x;  // 0..511
        const bool is_y = tid < 256;
        const int c = tid & 255;
        const int sy = c >> 3, gy = c & 7;
        const uint32_t ry = (uint32_t)(sy & 7), by8 = (uint32_t)(sy >> 3);
        const uint32_t ldoff = (uint32_t)(sy * 128 + gy * 16);
        const uint32_t st_a = by8 * 1024 + swz(ry, gy);  // R or X; I / Y at +4K, N at +8K
        const uint32_t full_pair_leader = mapa(bar(kBarFullPair), 0);
        uint32_t g = 0, gp = 0;
        bool ok = true;
        for (int u = first; u < last && ok; u++) {
            const Unit U = P.units[u];
            const int nst = (U.t1 - U.t0 + kStageSamples - 1) / kStageSamples;
            // Stages are unpacked two at a time (one stage pair): both loads
            // and conversions first, then one wait for the operand slots, the
            // stores of both stages, one proxy fence and one arrive per warp.
            for (int it = 0; it < nst; it += 2, gp++) {
                const int nin = (it + 1 < nst) ? 2 : 1;
                uint32_t v0[2][4], v1[2][4], v2[2][4];
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    if (j >= nin) break;
                    const uint32_t gs = g + (uint32_t)j;
                    const int ps = (int)(gs % kPkStages);
                    if (!mbar_wait(bar(kBarFullPk + ps), (gs / kPkStages) & 1, abort_flag)) {
                        ok = false;
                        break;
                    }
                    const bool valid = (U.t0 + (it + j) * kStageSamples + sy) < U.t1;
                    if (is_y) {
                        const uint4 w = lds128(pk_y + ps * kPkBytes + ldoff);
                        yconv<MAP>(w.x, v0[j][0], v1[j][0], v2[j][0]);
                        yconv<MAP>(w.y, v0[j][1], v1[j][1], v2[j][1]);
                        yconv<MAP>(w.z, v0[j][2], v1[j][2], v2[j][2]);
                        yconv<MAP>(w.w, v0[j][3], v1[j][3], v2[j][3]);
                    } else {
                        const uint4 w = lds128(pk_x + ps * kPkBytes + ldoff);
                        xconv<MAP>(w.x, v0[j][0], v1[j][0]);
                        xconv<MAP>(w.y, v0[j][1], v1[j][1]);
                        xconv<MAP>(w.z, v0[j][2], v1[j][2]);
                        xconv<MAP>(w.w, v0[j][3], v1[j][3]);
#pragma unroll
                        for (int k = 0; k < 4; k++) v2[j][k] = 0u;
                    }
                    if (!valid) {
#pragma unroll
                        for (int k = 0; k < 4; k++) v0[j][k] = v1[j][k] = v2[j][k] = 0u;
                    }
                    // The converted registers depend on the loads, and
                    // __syncwarp orders every lane before lane 0's arrive:
                    // one arrival per warp frees the slot.
                    __syncwarp();
                    if (lane == 0) mbar_arrive(bar(kBarEmptyPk + ps));
                }
                if (!ok) break;
                g += (uint32_t)nin;

                const int pslot = (int)(gp % kPairs);
                if (!mbar_wait(bar(kBarEmptyPair + pslot), ((gp / kPairs) & 1) ^ 1, abort_flag)) {
                    ok = false;
                    break;
                }
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    if (j >= nin) break;
                    const int os = 2 * pslot + j;
                    if (is_y) {
                        const uint32_t ya = op_y + os * kYOpBytes + st_a;
                        sts128(ya, v0[j][0], v0[j][1], v0[j][2], v0[j][3]);                // R
                        sts128(ya + 4096, v1[j][0], v1[j][1], v1[j][2], v1[j][3]);  // I
                        sts128(ya + 8192, v2[j][0], v2[j][1], v2[j][2], v2[j][3]);  // N
                    } else {
                        const uint32_t xa = op_x + os * kXOpBytes + st_a;
                        sts128(xa, v0[j][0], v0[j][1], v0[j][2], v0[j][3]);         // X
                        sts128(xa + 4096, v1[j][0], v1[j][1], v1[j][2], v1[j][3]);  // Y
                    }
                }
                fence_proxy_async();
                __syncwarp();
                if (lane == 0) mbar_arrive_cluster(full_pair_leader + 8 * pslot);
            }
        }
        if (!ok) {
            atomicOr(P.err, 0x400);
            *abort_flag = 1;
        }
        // No multicast arrival may still be on its way to this CTA's pair
        // barriers when it retires: thread 0 waits for the last phase of each.
        if (tid == 0)
            for (int k = 0; k < kPairs; k++)
                if (gp > (uint32_t)k)  // pairs gp' < gp with slot k: their last phase
                    mbar_wait_drain(bar(kBarEmptyPair + k), ((gp - 1 - k) / kPairs) & 1);
    } else {
        // ------------------------------------------------- epilogue (both CTAs)
        // Epilogue warp w drains TMEM lanes 32 * (w % 4) .. +31 (its quarter of
        // the CTA's 128 y rows) over kEpiBlocks 32-column blocks of Re and Im,
        // hands the cells to TMA through its staging tiles, and releases the
        // accumulator as soon as its last TMEM load completes, while the unpack
        // warps are already converting the next unit.
        const int q = warp & 3;
        const int j0 = ((warp - kEpiWarp0) >> 2) * kEpiBlocks;
        const uint32_t acc_empty_leader = mapa(bar(kBarAccEmpty), 0);
        const uint32_t stage = sbase + kOffStage + (uint32_t)(warp - kEpiWarp0) * kEpiStageBytes;
        uint32_t acc_phase = 0, nchunk = 0;
        bool ok = true;
        for (int u = first; u < last && ok; u++) {
            const Unit U = P.units[u];
            const ChanDesc *cd = P.chans + U.chan;
            const int ty = 2 * (U.tyx & 1023) + (int)rank;
            const int tx2 = (U.tyx >> 10) & 1023;
            const int nb1 = cd->nb1;
            const int by = ty * 4 + q;
            // Split units (other units cover the same cells' other sample ranges)
            // add like accumulate mode: every element of a TMA reduce-add is an
            // individual relaxed reduction at gpu scope, so concurrent units meet
            // exactly in the zeroed (or accumulating) output.
            const bool add = U.split || P.accumulate;
            const CUtensorMap *omap = P.use_param_map ? &pomap : &cd->omap;
            const int row0 = cd->orow + (int)(U.out_off >> 6);
            if (!mbar_wait(bar(kBarAccFull), acc_phase, abort_flag)) {
                ok = false;
                break;
            }
            acc_phase ^= 1;
            tc_fence_after();
#pragma unroll 1
            for (int j = j0; j < j0 + kEpiBlocks; j++) {  // 32-column block of the 256 x columns
                const int bx = tx2 * 8 + j;
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
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive_cluster(acc_empty_leader);
        }
        if (!ok) {
            atomicOr(P.err, 0x800);
            *abort_flag = 1;
        }
        if (lane == 0) bulk_wait_all();  // output tiles written
    }

    tc_fence_before();
    __syncthreads();
    cluster_sync();  // no remote arrivals after this point
    if (warp == kMmaWarp) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                     "r"(kTmemCols)
                     : "memory");
    }
}

template <int MAP>
cudaError_t launch_pair_map(const TcLaunch &L, const CUtensorMap *pmap, const CUtensorMap *pomap,
                            cudaStream_t st) {
    static bool attr_done[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr_done[dev]) {
        e = cudaFuncSetAttribute(tc_pair_kernel<MAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kSmemBytes);
        if (e != cudaSuccess) return e;
        attr_done[dev] = true;
    }
    KParams P;
    P.chans = L.chans;
    P.units = L.units;
    P.cluster_offsets = L.cta_offsets;
    P.out_base = L.out_base;
    P.use_param_map = L.use_param_map;
    P.ut = L.ut;
    P.accumulate = L.accumulate;
    P.err = L.err;
    CUtensorMap dummy;
    memset(&dummy, 0, sizeof(dummy));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * L.grid);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = kSmemBytes;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, tc_pair_kernel<MAP>, pmap ? *pmap : dummy, pomap ? *pomap : dummy,
                           P);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace

void tc_append_pair_units(std::vector<Unit> &out, int chan, int E, int t_begin, int t_end,
                          int tsplit, long long out_off) {
    const int nt2 = ((E + 127) / 128 + 1) / 2;
    const int span = t_end - t_begin;
    if (span <= 0) return;
    int splits = tsplit < 1 ? 1 : tsplit;
    int chunk = (span + splits - 1) / splits;
    chunk = (chunk + kStageSamples - 1) / kStageSamples * kStageSamples;
    if (chunk > kUnitMaxSamples) chunk = kUnitMaxSamples;
    splits = (span + chunk - 1) / chunk;
    for (int ty2 = 0; ty2 < nt2; ty2++)
        for (int tx2 = ty2; tx2 < nt2; tx2++)
            for (int s = 0; s < splits; s++) {
                Unit u;
                u.chan = chan;
                u.tyx = ty2 | (tx2 << 10);
                u.t0 = t_begin + s * chunk;
                u.t1 = std::min(t_end, u.t0 + chunk);
                u.out_off = out_off;
                u.split = splits > 1 ? 1 : 0;
                u.cost = unit_cost(true, u.t0, u.t1, 2);
                out.push_back(u);
            }
}

cudaError_t tc_pair_launch(const TcLaunch &L, const CUtensorMap *param_map,
                           const CUtensorMap *param_omap, cudaStream_t st) {
    if (L.nunits <= 0) return cudaSuccess;
    if (L.grid <= 0) return cudaErrorInvalidValue;
    if (L.use_param_map && (!param_map || !param_omap)) return cudaErrorInvalidValue;
    switch (L.map) {
    case MAP_EXACT: return launch_pair_map<MAP_EXACT>(L, param_map, param_omap, st);
    case MAP_CONF: return launch_pair_map<MAP_CONF>(L, param_map, param_omap, st);
    default: return launch_pair_map<MAP_PACKED>(L, param_map, param_omap, st);
    }
}

}  // namespace chx
