// simt_kernels.cu -- CUDA-core kernels of libchimex:
//   * correlate_simt: dp4a correlator over 32x32 blocks (baseline path and the
//     fallback for shapes the tensor-core kernel does not take; also used by
//     chx_corr_compat with the offset-domain value maps),
//   * offset_accumulate: offsetAccumulateElements (offset_accumulator.cl:7-49),
//   * preseed: the four preseed variants (preseed_multifreq*_UT.cl),
//   * block -> triangle / full-matrix reorganisation (gpu_data_reorg.c:36-124).
#include <algorithm>

#include "chimex_internal.h"

namespace chx {

namespace {

// (by, bx) of block b in the row-major upper-triangle enumeration of
// main_wrapper.c:529-540.
__device__ __forceinline__ void decode_block(int b, int nb1, int &by, int &bx) {
    int r = b, y = 0;
    while (r >= nb1 - y) {
        r -= nb1 - y;
        y++;
    }
    by = y;
    bx = y + r;
}

// Operand bytes of one packed sample under a value map (see chimex_internal.h).
struct Ops {
    int a0, a1, b0, b1, b2, b3;
};

template <int MAP>
__device__ __forceinline__ Ops map_byte(uint32_t p) {
    const int hi = (p >> 4) & 15, lo = p & 15;
    Ops o;
    if (MAP == MAP_EXACT) {
        o.a0 = hi - 8; o.a1 = lo - 8;
        o.b0 = hi - 8; o.b1 = lo - 8; o.b2 = 8 - lo; o.b3 = hi - 8;
    } else if (MAP == MAP_CONF) {
        o.a0 = hi; o.a1 = lo;
        o.b0 = hi; o.b1 = lo; o.b2 = -lo; o.b3 = hi;
    } else {
        o.a0 = hi; o.a1 = 15 - lo;
        o.b0 = hi; o.b1 = -lo; o.b2 = -lo; o.b3 = -hi;
    }
    return o;
}

__device__ __forceinline__ uint32_t put_byte(uint32_t w, int v, int j) {
    return w | ((uint32_t)(v & 0xFF) << (8 * j));
}

// One CTA = one 32x32 output block of one channel over one sample range.
// Each of the 256 threads owns a 2x2 group of cells.  Samples are staged 32
// at a time: packed bytes -> shared memory -> int8x4 words per element
// ([component][word][element], conflict-free for the compute loop).
template <int MAP>
__global__ void __launch_bounds__(256)
correlate_simt_kernel(const uint8_t *__restrict__ packed, int32_t *__restrict__ blocks,
                      int E, int F, int T, int nb1, int64_t nb, int ut, int mode,
                      int tchunk) {
    __shared__ uint32_t py[32][8];  // [sample][element/4] packed bytes
    __shared__ uint32_t px[32][8];
    __shared__ int32_t A[2][8][32];  // [a0|a1][sample/4][element]
    __shared__ int32_t B[4][8][32];  // [b0..b3][sample/4][element]

    const int b = blockIdx.x, f = blockIdx.y;
    int by, bx;
    decode_block(b, nb1, by, bx);
    const int t_begin = blockIdx.z * tchunk;
    const int t_end = min(T, t_begin + tchunk);
    const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
    const int64_t row = (int64_t)F * E;
    const uint8_t *base = packed + (int64_t)f * E;

    int re[2][2] = {{0, 0}, {0, 0}}, im[2][2] = {{0, 0}, {0, 0}};

    for (int t0 = t_begin; t0 < t_end; t0 += 32) {
        {
            const int r = tid >> 3, c = tid & 7;
            const int t = t0 + r;
            uint32_t vy = 0, vx = 0;
            if (t < t_end) {
                vy = *reinterpret_cast<const uint32_t *>(base + t * row + by * 32 + c * 4);
                vx = *reinterpret_cast<const uint32_t *>(base + t * row + bx * 32 + c * 4);
            }
            py[r][c] = vy;
            px[r][c] = vx;
        }
        __syncthreads();
        {
            const int e = tid & 31, w = tid >> 5;
            uint32_t a0 = 0, a1 = 0, b0 = 0, b1 = 0, b2 = 0, b3 = 0;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int s = 4 * w + j;
                if (t0 + s < t_end) {
                    const uint32_t pyb = (py[s][e >> 2] >> (8 * (e & 3))) & 0xFF;
                    const uint32_t pxb = (px[s][e >> 2] >> (8 * (e & 3))) & 0xFF;
                    const Ops oy = map_byte<MAP>(pyb), ox = map_byte<MAP>(pxb);
                    a0 = put_byte(a0, oy.a0, j);
                    a1 = put_byte(a1, oy.a1, j);
                    b0 = put_byte(b0, ox.b0, j);
                    b1 = put_byte(b1, ox.b1, j);
                    b2 = put_byte(b2, ox.b2, j);
                    b3 = put_byte(b3, ox.b3, j);
                }
            }
            A[0][w][e] = (int32_t)a0;
            A[1][w][e] = (int32_t)a1;
            B[0][w][e] = (int32_t)b0;
            B[1][w][e] = (int32_t)b1;
            B[2][w][e] = (int32_t)b2;
            B[3][w][e] = (int32_t)b3;
        }
        __syncthreads();
#pragma unroll
        for (int w = 0; w < 8; w++) {
            int ya0[2], ya1[2], xb0[2], xb1[2], xb2[2], xb3[2];
#pragma unroll
            for (int i = 0; i < 2; i++) {
                ya0[i] = A[0][w][2 * ty + i];
                ya1[i] = A[1][w][2 * ty + i];
                xb0[i] = B[0][w][2 * tx + i];
                xb1[i] = B[1][w][2 * tx + i];
                xb2[i] = B[2][w][2 * tx + i];
                xb3[i] = B[3][w][2 * tx + i];
            }
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    re[i][j] = __dp4a(ya0[i], xb0[j], re[i][j]);
                    re[i][j] = __dp4a(ya1[i], xb1[j], re[i][j]);
                    im[i][j] = __dp4a(ya0[i], xb2[j], im[i][j]);
                    im[i][j] = __dp4a(ya1[i], xb3[j], im[i][j]);
                }
        }
        __syncthreads();
    }

    int32_t *blk = blocks + ((int64_t)f * nb + b) * 2048;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int y = 2 * ty + i, x = 2 * tx + j;
            const int vr = re[i][j];
            const int vi = ut ? im[i][j] : (int)(0u - (uint32_t)im[i][j]);
            int32_t *cell = blk + y * 64 + 2 * x;
            if (mode == 0) {
                *reinterpret_cast<int2 *>(cell) = make_int2(vr, vi);
            } else if (mode == 1) {
                int2 o = *reinterpret_cast<int2 *>(cell);
                o.x = (int)((uint32_t)o.x + (uint32_t)vr);
                o.y = (int)((uint32_t)o.y + (uint32_t)vi);
                *reinterpret_cast<int2 *>(cell) = o;
            } else {
                atomicAdd(cell, vr);
                atomicAdd(cell + 1, vi);
            }
        }
}

// offsetAccumulateElements (offset_accumulator.cl:18-47).  The work is the
// (vector block, 16-sample group) space: a vector block is 32 consecutive
// 16-byte vectors of a sample row (16 (f, e) bytes each), a group 16 samples.
// Each CTA takes an equal, contiguous share of that space (so every SM of the
// single wave streams the same number of bytes); inside a share, warp w
// streams the groups w, w + 8, ... of one vector block at a time (each lane
// one vector: coalesced 512-byte rows), loading a group's 16 vectors at once
// so that enough bytes are in flight to keep HBM busy.  The nibbles are summed
// four lanes at a time in byte-wide SWAR registers (15 * 16 < 256) and flushed
// to 32-bit sums after every group; the 8 warps' sums meet in shared memory,
// and the CTAs' in one atomic add per word for each vector block they touch.
constexpr int kOaWarps = 8;

__global__ void __launch_bounds__(kOaWarps * 32)
offset_accumulate_kernel(const uint8_t *__restrict__ packed, uint32_t *__restrict__ sums,
                         int64_t nvec, int T, int64_t ngroups, int64_t nwork) {
    __shared__ uint32_t part[kOaWarps][32][32];  // [warp][word][lane]
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint4 *p = reinterpret_cast<const uint4 *>(packed);
    const int64_t L1 = nwork * (blockIdx.x + 1) / gridDim.x;
    for (int64_t L = nwork * blockIdx.x / gridDim.x; L < L1;) {  // uniform across the CTA
        const int64_t vb = L / ngroups;
        const int64_t end = min(L1, (vb + 1) * ngroups);  // this vector block's part
        const int64_t g0 = L - vb * ngroups, g1 = end - vb * ngroups;
        const int64_t i = vb * 32 + lane;
        uint32_t s[32];  // element 4q + j: s[2 (4q + j)] re, s[2 (4q + j) + 1] im
#pragma unroll
        for (int k = 0; k < 32; k++) s[k] = 0u;
        if (i < nvec) {
            for (int64_t g = g0 + w; g < g1; g += kOaWarps) {
                const int t = (int)(16 * g);
                uint32_t lo[4] = {0u, 0u, 0u, 0u}, hi[4] = {0u, 0u, 0u, 0u};
                const uint4 *row = p + (int64_t)t * nvec + i;
                auto add = [&](const uint4 v) {
                    lo[0] += v.x & 0x0F0F0F0Fu;
                    hi[0] += (v.x >> 4) & 0x0F0F0F0Fu;
                    lo[1] += v.y & 0x0F0F0F0Fu;
                    hi[1] += (v.y >> 4) & 0x0F0F0F0Fu;
                    lo[2] += v.z & 0x0F0F0F0Fu;
                    hi[2] += (v.z >> 4) & 0x0F0F0F0Fu;
                    lo[3] += v.w & 0x0F0F0F0Fu;
                    hi[3] += (v.w >> 4) & 0x0F0F0F0Fu;
                };
                if (t + 16 <= T) {  // a full group: 16 independent loads in flight
                    uint4 v[16];
#pragma unroll
                    for (int k = 0; k < 16; k++) v[k] = __ldg(row + (int64_t)k * nvec);
#pragma unroll
                    for (int k = 0; k < 16; k++) add(v[k]);
                } else {
                    for (int k = 0; t + k < T; k++) add(__ldg(row + (int64_t)k * nvec));
                }
#pragma unroll
                for (int q = 0; q < 4; q++) {
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        s[2 * (4 * q + j)] += (hi[q] >> (8 * j)) & 0xFFu;
                        s[2 * (4 * q + j) + 1] += (lo[q] >> (8 * j)) & 0xFFu;
                    }
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 32; k++) part[w][k][lane] = s[k];
        __syncthreads();
        // Thread r handles (word, lane) pairs r, r + 256, ...: sum over the warps.
#pragma unroll
        for (int r = threadIdx.x; r < 32 * 32; r += kOaWarps * 32) {
            const int k = r >> 5, l = r & 31;
            const int64_t iv = vb * 32 + l;
            uint32_t acc = 0u;
#pragma unroll
            for (int ww = 0; ww < kOaWarps; ww++) acc += part[ww][k][l];
            if (iv < nvec && acc != 0u) atomicAdd(sums + 32 * iv + k, acc);
        }
        __syncthreads();  // part is rewritten for the next vector block
        L = end;
    }
}

// preseed: writes (=) the offset correction of every cell of one block.
// Formulas: preseed_multifreq_UT.cl:54-70 / preseed_multifreq.cl:54-70
// (conference) and preseed_multifreq_highly_packed_correlator_method{_UT,}.cl
// :54-70 (packed); x is the column element, y the row element.  sx / sy hold
// the (re, im) sums of the block's 32 columns / rows; 256 threads write two
// neighbouring cells (xl, xl + 1) per 16-byte store.
__device__ __forceinline__ void preseed_block(const uint32_t *sx, const uint32_t *sy,
                                              int32_t *blk, uint32_t t128,
                                              int packed_variant, int ut, int tid) {
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const int c2 = tid + 256 * k, yl = c2 >> 4, xl0 = (c2 & 15) * 2;
        const uint32_t yr = sy[2 * yl], yi = sy[2 * yl + 1];
        uint32_t v[4];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int xl = xl0 + h;
            const uint32_t xr = sx[2 * xl], xi = sx[2 * xl + 1];
            uint32_t re, imv;
            if (!packed_variant) {
                re = t128 - 8u * (xr + xi + yr + yi);
                imv = ut ? 8u * ((xi - xr) + (yr - yi)) : 8u * ((xr - xi) + (yi - yr));
            } else {
                re = t128 - 8u * xr + 7u * xi - 8u * (yr + yi);
                imv = ut ? 8u * xi + 7u * xr + 8u * (yr - yi)
                         : 0u - 8u * xi - 7u * xr - 8u * (yr - yi);
            }
            v[2 * h] = re;
            v[2 * h + 1] = imv;
        }
        *reinterpret_cast<int4 *>(blk + (yl * 32 + xl0) * 2) =
            make_int4((int)v[0], (int)v[1], (int)v[2], (int)v[3]);
    }
}

// One CTA per run of kPsBlocks consecutive blocks of one channel: every
// thread issues its 2 x kPsBlocks 16-byte stores back to back (no dependency
// between them), which keeps more bytes in flight per thread than one block
// per CTA.  The blocks' row and column sums are gathered into shared memory
// first.
constexpr int kPsBlocks = 4;

__global__ void __launch_bounds__(256)
preseed_kernel(const uint32_t *__restrict__ sums, int32_t *__restrict__ blocks, int E,
               int nb1, int64_t nb, uint32_t t128, int packed_variant, int ut) {
    __shared__ uint32_t sx[kPsBlocks][64], sy[kPsBlocks][64];
    const int f = blockIdx.y;
    const int64_t b0 = (int64_t)blockIdx.x * kPsBlocks;
    const int tid = threadIdx.x;
    for (int i = tid; i < kPsBlocks * 64; i += 256) {
        const int k = i >> 6, w = i & 63;
        if (b0 + k < nb) {
            int by, bx;
            decode_block((int)(b0 + k), nb1, by, bx);
            sx[k][w] = sums[((int64_t)f * E + bx * 32) * 2 + w];
            sy[k][w] = sums[((int64_t)f * E + by * 32) * 2 + w];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kPsBlocks; k++)
        if (b0 + k < nb)
            preseed_block(sx[k], sy[k], blocks + ((int64_t)f * nb + b0 + k) * 2048, t128,
                          packed_variant, ut, tid);
}

// Block layout -> packed triangle (gpu_data_reorg.c:76-124).  The block is
// read into shared memory with 16-byte loads; each of its rows is a
// contiguous run of cells in the triangle (x >= y only on the diagonal
// block) starting at any cell index, so every row is written as 16-byte
// stores of cell pairs, with a single 8-byte store for an odd first cell and
// for an odd last cell.  16 threads per row, two rows per thread.
__global__ void __launch_bounds__(256)
blocks_to_triangle_kernel(const int32_t *__restrict__ blocks, int32_t *__restrict__ tri,
                          int E, int nb1, int64_t nb) {
    __shared__ __align__(16) int2 cells[32 * 32];
    const int b = blockIdx.x, f = blockIdx.y;
    int by, bx;
    decode_block(b, nb1, by, bx);
    const int64_t ntri = (int64_t)E * (E + 1) / 2;
    const int4 *blk = reinterpret_cast<const int4 *>(blocks + ((int64_t)f * nb + b) * 2048);
    int4 *c4 = reinterpret_cast<int4 *>(cells);
#pragma unroll
    for (int k = 0; k < 2; k++) c4[threadIdx.x + 256 * k] = __ldg(blk + threadIdx.x + 256 * k);
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 2; r++) {
        const int slot = threadIdx.x + 256 * r, yl = slot >> 4, k = slot & 15;
        const int xs = (bx == by) ? yl : 0;  // first cell of the row written
        const int64_t y = by * 32 + yl;
        const int64_t a0 = f * ntri + y * E - (y - 1) * y / 2 + (bx * 32 + xs - y);
        const int head = (int)(a0 & 1);      // odd start: one 8-byte cell first
        const int n = 32 - xs - head;        // cells after the head
        const int2 *row = cells + yl * 32;
        if (k < n / 2) {
            const int x = xs + head + 2 * k;
            const int2 u = row[x], v = row[x + 1];
            *reinterpret_cast<int4 *>(tri + 2 * (a0 + head + 2 * k)) = make_int4(u.x, u.y, v.x, v.y);
        }
        if (k == 15 && head) *reinterpret_cast<int2 *>(tri + 2 * a0) = row[xs];
        if (k == 14 && (n & 1)) *reinterpret_cast<int2 *>(tri + 2 * (a0 + 31 - xs)) = row[31];
    }
}

// Block layout -> full Hermitian matrix (gpu_data_reorg.c:36-74).  The upper
// triangle is written row by row straight from the block; the mirrored lower
// triangle (conjugates) goes through a shared-memory transpose so that its
// rows are written contiguously too.
__global__ void __launch_bounds__(256)
blocks_to_full_kernel(const int32_t *__restrict__ blocks, int32_t *__restrict__ full,
                      int E, int nb1, int64_t nb) {
    __shared__ int2 tile[32][33];
    const int b = blockIdx.x, f = blockIdx.y;
    int by, bx;
    decode_block(b, nb1, by, bx);
    const int32_t *blk = blocks + ((int64_t)f * nb + b) * 2048;
    int32_t *m = full + (int64_t)f * E * E * 2;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int c = threadIdx.x + 256 * k, yl = c >> 5, xl = c & 31;
        const int64_t y = by * 32 + yl, x = bx * 32 + xl;
        const int2 v = *reinterpret_cast<const int2 *>(blk + 2 * c);
        tile[yl][xl] = v;
        if (x >= y) *reinterpret_cast<int2 *>(m + (y * E + x) * 2) = v;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int c = threadIdx.x + 256 * k, xl = c >> 5, yl = c & 31;
        const int64_t y = by * 32 + yl, x = bx * 32 + xl;
        if (x > y) {
            const int2 v = tile[yl][xl];
            *reinterpret_cast<int2 *>(m + (x * E + y) * 2) = make_int2(v.x, (int)(0u - (uint32_t)v.y));
        }
    }
}

}  // namespace

cudaError_t launch_correlate_simt(const uint8_t *packed, int32_t *blocks, int E, int F,
                                  int T, int map, int ut, int mode, int splits,
                                  cudaStream_t st) {
    const int nb1 = E / 32;
    const int64_t nb = num_blocks_of(E);
    if (splits < 1) splits = 1;
    int tchunk = (T + splits - 1) / splits;
    tchunk = (tchunk + 31) / 32 * 32;
    splits = (T + tchunk - 1) / tchunk;
    dim3 grid((unsigned)nb, (unsigned)F, (unsigned)splits);
    if (map == MAP_EXACT)
        correlate_simt_kernel<MAP_EXACT><<<grid, 256, 0, st>>>(packed, blocks, E, F, T, nb1, nb, ut, mode, tchunk);
    else if (map == MAP_CONF)
        correlate_simt_kernel<MAP_CONF><<<grid, 256, 0, st>>>(packed, blocks, E, F, T, nb1, nb, ut, mode, tchunk);
    else
        correlate_simt_kernel<MAP_PACKED><<<grid, 256, 0, st>>>(packed, blocks, E, F, T, nb1, nb, ut, mode, tchunk);
    return cudaGetLastError();
}

cudaError_t launch_offset_accumulate(const uint8_t *packed, uint32_t *sums, int E, int F,
                                     int T, cudaStream_t st) {
    const int64_t nvec = (int64_t)F * E / 16;  // E % 32 == 0
    const int64_t vblocks = (nvec + 31) / 32;
    const int64_t ngroups = (T + 15) / 16;
    const int64_t nwork = vblocks * ngroups;
    // One wave of three CTAs per SM (66 registers, 32 KiB shared memory), each
    // with an equal share of the work.
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>((int64_t)3 * sms, nwork));
    offset_accumulate_kernel<<<(unsigned)grid, kOaWarps * 32, 0, st>>>(packed, sums, nvec, T,
                                                                      ngroups, nwork);
    return cudaGetLastError();
}

cudaError_t launch_preseed(const uint32_t *sums, int32_t *blocks, int E, int F, int T,
                           int packed_variant, int ut, cudaStream_t st) {
    const int64_t nb = num_blocks_of(E);
    dim3 grid((unsigned)((nb + kPsBlocks - 1) / kPsBlocks), (unsigned)F);
    preseed_kernel<<<grid, 256, 0, st>>>(sums, blocks, E, E / 32, nb, (uint32_t)T * 128u,
                                         packed_variant, ut);
    return cudaGetLastError();
}

cudaError_t launch_blocks_to_triangle(const int32_t *blocks, int32_t *tri, int E, int F,
                                      cudaStream_t st) {
    dim3 grid((unsigned)num_blocks_of(E), (unsigned)F);
    blocks_to_triangle_kernel<<<grid, 256, 0, st>>>(blocks, tri, E, E / 32, num_blocks_of(E));
    return cudaGetLastError();
}

cudaError_t launch_blocks_to_full(const int32_t *blocks, int32_t *full, int E, int F,
                                  cudaStream_t st) {
    dim3 grid((unsigned)num_blocks_of(E), (unsigned)F);
    blocks_to_full_kernel<<<grid, 256, 0, st>>>(blocks, full, E, E / 32, num_blocks_of(E));
    return cudaGetLastError();
}

}  // namespace chx
