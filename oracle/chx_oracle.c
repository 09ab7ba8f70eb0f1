/*
 * chx_oracle.c -- CPU restatement of the CHIME-x correlator arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY (see chx_oracle.h).  Integer results are computed
 * in uint32 so that wrap-around matches the reference's 32-bit arithmetic
 * without relying on C signed overflow.
 */
#include "chx_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* input_generator.c:8-15: add the offset and clip into [lo, hi]. */
static int clip_offset(int v, int off, int lo, int hi) {
    int r = v + off;
    if (r > hi) return hi;
    if (r < lo) return lo;
    return r;
}

/* Restates generate_char_data_set (input_generator.c:17-103).  The random
 * stream is glibc srand()/rand(), the reference's only external dependency:
 * the generator reseeds once, and again at every time step unless
 * no_repeat_random is set; it draws re before im for every element of every
 * channel, including channels that are then overwritten with the default
 * value by the single-channel override. */
void orc_generate(int gen_type, int seed, int default_re, int default_im,
                  int initial_re, int initial_im, int single_freq, int T,
                  int F, int E, int no_repeat_random, uint8_t *out) {
    if (single_freq > F || single_freq < 0) single_freq = ORC_ALL_FREQUENCIES;
    const unsigned dre = (unsigned)clip_offset(default_re, 8, 0, 15);
    const unsigned dim = (unsigned)clip_offset(default_im, 8, 0, 15);
    const unsigned ire = (unsigned)clip_offset(initial_re, 8, 0, 15);
    const unsigned iim = (unsigned)clip_offset(initial_im, 8, 0, 15);
    const uint8_t default_byte = (uint8_t)(((dre << 4) & 0xF0) | (dim & 0x0F));

    if (gen_type == ORC_GEN_RANDOM_SEEDED) srand((unsigned)seed);
    for (int t = 0; t < T; t++) {
        if (gen_type == ORC_GEN_RANDOM_SEEDED && !no_repeat_random)
            srand((unsigned)seed);
        for (int f = 0; f < F; f++) {
            uint8_t *row = out + ((size_t)t * F + f) * E;
            for (int e = 0; e < E; e++) {
                unsigned re, im;
                switch (gen_type) {
                case ORC_GEN_CONSTANT:
                    re = ire;
                    im = iim;
                    break;
                case ORC_GEN_RAMP_UP:
                    re = (unsigned)(f + (int)ire + e) % 16u;
                    im = (unsigned)(f + (int)iim + e) % 16u;
                    break;
                case ORC_GEN_RAMP_DOWN:
                    re = 15u - (unsigned)(f + (int)ire + e) % 16u;
                    im = 15u - (unsigned)(f + (int)iim + e) % 16u;
                    break;
                case ORC_GEN_RANDOM_SEEDED:
                    re = (unsigned)(rand() % 16);
                    im = (unsigned)(rand() % 16);
                    break;
                default:
                    re = dre;
                    im = dim;
                    break;
                }
                /* The reference stores unsigned char values: truncate. */
                re &= 0xFFu;
                im &= 0xFFu;
                uint8_t b = (uint8_t)(((re << 4) & 0xF0) + (im & 0x0F));
                if (single_freq != ORC_ALL_FREQUENCIES && f != single_freq)
                    b = default_byte;
                row[e] = b;
            }
        }
    }
}

int64_t orc_num_blocks(int E) {
    int64_t n = E / 32;
    return n * (n + 1) / 2;
}

/* Block index of (by, bx), bx >= by, in the row-major upper-triangle order of
 * the id maps built at main_wrapper.c:529-540. */
static int64_t block_index(int64_t nb1, int64_t by, int64_t bx) {
    return by * nb1 - by * (by - 1) / 2 + (bx - by);
}

/* Accumulates, for one channel and a sample range, the (y, x) products over
 * every cell of every upper-triangle block, diagonal-block lower halves
 * included.  acc_re/acc_im are E x E row-major scratch (only the cells with
 * x >= 32*(y/32) are touched).  The visibility definition is
 * cpu_corr_test.c:188-193 (Re = xr*yr + xi*yi, Im = xr*yi - xi*yr). */
static void accumulate_channel(const uint8_t *packed, int F, int E, int f,
                               int t0, int t1, uint32_t *acc_re,
                               uint32_t *acc_im, int32_t *sr, int32_t *si) {
    for (int t = t0; t < t1; t++) {
        const uint8_t *row = packed + ((size_t)t * F + f) * E;
        for (int e = 0; e < E; e++) {
            sr[e] = (int32_t)((row[e] >> 4) & 0x0F) - 8;
            si[e] = (int32_t)(row[e] & 0x0F) - 8;
        }
        for (int y = 0; y < E; y++) {
            const int32_t yr = sr[y], yi = si[y];
            const int xs = (y / 32) * 32;
            uint32_t *pr = acc_re + (size_t)y * E;
            uint32_t *pi = acc_im + (size_t)y * E;
            for (int x = xs; x < E; x++) {
                pr[x] += (uint32_t)(sr[x] * yr + si[x] * yi);
                pi[x] += (uint32_t)(sr[x] * yi - si[x] * yr);
            }
        }
    }
}

void orc_correlate_blocks_range(const uint8_t *packed, int T, int F, int E,
                                int t0, int t1, int ut, int accumulate,
                                int32_t *blocks) {
    (void)T;
    const int64_t nb1 = E / 32;
    const int64_t nb = orc_num_blocks(E);
    uint32_t *acc_re = (uint32_t *)calloc((size_t)E * E, sizeof(uint32_t));
    uint32_t *acc_im = (uint32_t *)calloc((size_t)E * E, sizeof(uint32_t));
    int32_t *sr = (int32_t *)malloc((size_t)E * sizeof(int32_t));
    int32_t *si = (int32_t *)malloc((size_t)E * sizeof(int32_t));
    for (int f = 0; f < F; f++) {
        memset(acc_re, 0, (size_t)E * E * sizeof(uint32_t));
        memset(acc_im, 0, (size_t)E * E * sizeof(uint32_t));
        accumulate_channel(packed, F, E, f, t0, t1, acc_re, acc_im, sr, si);
        for (int64_t by = 0; by < nb1; by++) {
            for (int64_t bx = by; bx < nb1; bx++) {
                uint32_t *blk = (uint32_t *)blocks +
                    ((size_t)(f * nb + block_index(nb1, by, bx))) * 2048;
                for (int yl = 0; yl < 32; yl++) {
                    const size_t y = (size_t)(by * 32 + yl);
                    for (int xl = 0; xl < 32; xl++) {
                        const size_t x = (size_t)(bx * 32 + xl);
                        uint32_t re = acc_re[y * E + x];
                        uint32_t im = acc_im[y * E + x];
                        if (!ut) im = 0u - im;
                        uint32_t *cell = blk + (yl * 32 + xl) * 2;
                        if (accumulate) {
                            cell[0] += re;
                            cell[1] += im;
                        } else {
                            cell[0] = re;
                            cell[1] = im;
                        }
                    }
                }
            }
        }
    }
    free(acc_re);
    free(acc_im);
    free(sr);
    free(si);
}

void orc_correlate_blocks(const uint8_t *packed, int T, int F, int E, int ut,
                          int accumulate, int32_t *blocks) {
    orc_correlate_blocks_range(packed, T, F, E, 0, T, ut, accumulate, blocks);
}

/* cpu_corr_test.c:156-203 (ut=1) and :59-106 (ut=0): the triangle index
 * runs over f, y, x >= y; the first sample assigns, later samples add. */
void orc_correlate_triangle(const uint8_t *packed, int T, int F, int E, int ut,
                            int32_t *tri) {
    const size_t ntri = (size_t)E * (E + 1) / 2;
    uint32_t *out = (uint32_t *)tri;
    memset(out, 0, (size_t)F * ntri * 2 * sizeof(uint32_t));
    int32_t *sr = (int32_t *)malloc((size_t)E * sizeof(int32_t));
    int32_t *si = (int32_t *)malloc((size_t)E * sizeof(int32_t));
    for (int t = 0; t < T; t++) {
        for (int f = 0; f < F; f++) {
            const uint8_t *row = packed + ((size_t)t * F + f) * E;
            for (int e = 0; e < E; e++) {
                sr[e] = (int32_t)((row[e] >> 4) & 0x0F) - 8;
                si[e] = (int32_t)(row[e] & 0x0F) - 8;
            }
            uint32_t *o = out + (size_t)f * ntri * 2;
            for (int y = 0; y < E; y++) {
                for (int x = y; x < E; x++) {
                    int32_t im = ut ? (sr[x] * si[y] - si[x] * sr[y])
                                    : (si[x] * sr[y] - sr[x] * si[y]);
                    o[0] += (uint32_t)(sr[x] * sr[y] + si[x] * si[y]);
                    o[1] += (uint32_t)im;
                    o += 2;
                }
            }
        }
    }
    free(sr);
    free(si);
}

/* gpu_data_reorg.c:76-124: walk the block buffer in order; the triangle
 * address of (y, x) is f*E(E+1)/2 + y*E - y(y-1)/2 + (x - y) (:101); cells
 * below the diagonal of a diagonal block are skipped (:107-115). */
void orc_blocks_to_triangle(const int32_t *blocks, int F, int E, int32_t *tri) {
    const int64_t nb1 = E / 32;
    const int64_t nb = orc_num_blocks(E);
    const int64_t ntri = (int64_t)E * (E + 1) / 2;
    for (int f = 0; f < F; f++) {
        for (int64_t by = 0; by < nb1; by++) {
            for (int64_t bx = by; bx < nb1; bx++) {
                const int32_t *blk =
                    blocks + ((size_t)(f * nb + block_index(nb1, by, bx))) * 2048;
                for (int yl = 0; yl < 32; yl++) {
                    for (int xl = 0; xl < 32; xl++) {
                        if (bx == by && xl < yl) continue;
                        const int64_t y = by * 32 + yl, x = bx * 32 + xl;
                        const int64_t a =
                            f * ntri + y * E - (y - 1) * y / 2 + (x - y);
                        tri[2 * a] = blk[(yl * 32 + xl) * 2];
                        tri[2 * a + 1] = blk[(yl * 32 + xl) * 2 + 1];
                    }
                }
            }
        }
    }
}

/* gpu_data_reorg.c:36-74: full matrix; cells above the diagonal are copied
 * and mirrored as their conjugate below it. */
void orc_blocks_to_full(const int32_t *blocks, int F, int E, int32_t *full) {
    const int64_t nb1 = E / 32;
    const int64_t nb = orc_num_blocks(E);
    for (int f = 0; f < F; f++) {
        uint32_t *m = (uint32_t *)full + (size_t)f * E * E * 2;
        for (int64_t by = 0; by < nb1; by++) {
            for (int64_t bx = by; bx < nb1; bx++) {
                const uint32_t *blk = (const uint32_t *)blocks +
                    ((size_t)(f * nb + block_index(nb1, by, bx))) * 2048;
                for (int yl = 0; yl < 32; yl++) {
                    for (int xl = 0; xl < 32; xl++) {
                        const int64_t y = by * 32 + yl, x = bx * 32 + xl;
                        if (x < y) continue;
                        const uint32_t re = blk[(yl * 32 + xl) * 2];
                        const uint32_t im = blk[(yl * 32 + xl) * 2 + 1];
                        if (x > y) {
                            m[(x * E + y) * 2] = re;
                            m[(x * E + y) * 2 + 1] = 0u - im;
                        }
                        m[(y * E + x) * 2] = re;
                        m[(y * E + x) * 2 + 1] = im;
                    }
                }
            }
        }
    }
}

/* offset_accumulator.cl:18-47: per (f, e), the sum over samples of the
 * offset-binary high (re) and low (im) nibbles, output uint32[F*E][2]. */
void orc_offset_accumulate(const uint8_t *packed, int T, int F, int E,
                           int accumulate, uint32_t *sums) {
    const size_t n = (size_t)F * E;
    if (!accumulate) memset(sums, 0, n * 2 * sizeof(uint32_t));
    for (int t = 0; t < T; t++) {
        const uint8_t *row = packed + (size_t)t * n;
        for (size_t i = 0; i < n; i++) {
            sums[2 * i] += (row[i] >> 4) & 0x0F;
            sums[2 * i + 1] += row[i] & 0x0F;
        }
    }
}

/* Preseed correction per cell (y = row element, x = column element), from
 * the offset sums Sr, Si.  Conference kernels: preseed_multifreq_UT.cl:54-70
 * and :130-164 (UT), preseed_multifreq.cl:54-70 (non-UT).  Packed kernels:
 * preseed_multifreq_highly_packed_correlator_method_UT.cl:54-70 and the
 * non-UT file's :54-70. */
void orc_preseed(const uint32_t *sums, int T, int F, int E, int packed_variant,
                 int ut, int32_t *blocks) {
    const int64_t nb1 = E / 32;
    const int64_t nb = orc_num_blocks(E);
    const uint32_t c128 = (uint32_t)T * 128u;
    for (int f = 0; f < F; f++) {
        const uint32_t *s = sums + (size_t)f * E * 2;
        for (int64_t by = 0; by < nb1; by++) {
            for (int64_t bx = by; bx < nb1; bx++) {
                uint32_t *blk = (uint32_t *)blocks +
                    ((size_t)(f * nb + block_index(nb1, by, bx))) * 2048;
                for (int yl = 0; yl < 32; yl++) {
                    const size_t y = (size_t)(by * 32 + yl);
                    const uint32_t yr = s[2 * y], yi = s[2 * y + 1];
                    for (int xl = 0; xl < 32; xl++) {
                        const size_t x = (size_t)(bx * 32 + xl);
                        const uint32_t xr = s[2 * x], xi = s[2 * x + 1];
                        uint32_t re, im;
                        if (!packed_variant) {
                            re = c128 - 8u * (xr + xi + yr + yi);
                            im = ut ? 8u * ((xi - xr) + (yr - yi))
                                    : 8u * ((xr - xi) + (yi - yr));
                        } else {
                            re = c128 - 8u * xr + 7u * xi - 8u * (yr + yi);
                            im = ut ? 8u * xi + 7u * xr + 8u * (yr - yi)
                                    : 0u - 8u * xi - 7u * xr - 8u * (yr - yi);
                        }
                        uint32_t *cell = blk + (yl * 32 + xl) * 2;
                        cell[0] = re;
                        cell[1] = im;
                    }
                }
            }
        }
    }
}

/* The reference corr kernels add, per cell, partials built from the
 * offset-binary nibbles x' = x + 8:
 *   conference (pairwise_correlator_UT.cl:107-201):
 *     Re = sum x'r y'r + x'i y'i,  Im(UT) = sum x'r y'i - x'i y'r,
 *     Im(non-UT, pairwise_correlator.cl:167-201) = -Im(UT);
 *   packed (packed_correlator_overflow_protected_to_2272_iter_UT.cl:91-285):
 *     the y imaginary nibble is inverted (15 - y'i), giving
 *     Re = conference Re - 15 sum x'i,
 *     Im(UT) = conference Im(UT) - 15 sum x'r,
 *     Im(non-UT) = -conference Im(UT) + 15 sum x'r.
 * These equal the reference outputs wherever its 16-bit lanes (plus the
 * packed kernel's overflow counters) do not lose bits. */
void orc_corr_partials(const uint8_t *packed, int T, int F, int E,
                       int packed_variant, int ut, int32_t *blocks) {
    const int64_t nb1 = E / 32;
    const int64_t nb = orc_num_blocks(E);
    uint32_t *acc_re = (uint32_t *)malloc((size_t)E * E * sizeof(uint32_t));
    uint32_t *acc_im = (uint32_t *)malloc((size_t)E * E * sizeof(uint32_t));
    uint32_t *sxr = (uint32_t *)malloc((size_t)E * sizeof(uint32_t));
    uint32_t *sxi = (uint32_t *)malloc((size_t)E * sizeof(uint32_t));
    int32_t *pr = (int32_t *)malloc((size_t)E * sizeof(int32_t));
    int32_t *pi = (int32_t *)malloc((size_t)E * sizeof(int32_t));
    for (int f = 0; f < F; f++) {
        memset(acc_re, 0, (size_t)E * E * sizeof(uint32_t));
        memset(acc_im, 0, (size_t)E * E * sizeof(uint32_t));
        memset(sxr, 0, (size_t)E * sizeof(uint32_t));
        memset(sxi, 0, (size_t)E * sizeof(uint32_t));
        for (int t = 0; t < T; t++) {
            const uint8_t *row = packed + ((size_t)t * F + f) * E;
            for (int e = 0; e < E; e++) {
                pr[e] = (row[e] >> 4) & 0x0F;
                pi[e] = row[e] & 0x0F;
                sxr[e] += (uint32_t)pr[e];
                sxi[e] += (uint32_t)pi[e];
            }
            for (int y = 0; y < E; y++) {
                const int32_t yr = pr[y], yi = pi[y];
                const int xs = (y / 32) * 32;
                uint32_t *ar = acc_re + (size_t)y * E;
                uint32_t *ai = acc_im + (size_t)y * E;
                for (int x = xs; x < E; x++) {
                    ar[x] += (uint32_t)(pr[x] * yr + pi[x] * yi);
                    ai[x] += (uint32_t)(pr[x] * yi - pi[x] * yr);
                }
            }
        }
        for (int64_t by = 0; by < nb1; by++) {
            for (int64_t bx = by; bx < nb1; bx++) {
                uint32_t *blk = (uint32_t *)blocks +
                    ((size_t)(f * nb + block_index(nb1, by, bx))) * 2048;
                for (int yl = 0; yl < 32; yl++) {
                    const size_t y = (size_t)(by * 32 + yl);
                    for (int xl = 0; xl < 32; xl++) {
                        const size_t x = (size_t)(bx * 32 + xl);
                        uint32_t re = acc_re[y * E + x];
                        uint32_t im = acc_im[y * E + x];
                        if (packed_variant) {
                            re -= 15u * sxi[x];
                            im = ut ? im - 15u * sxr[x] : (0u - im) + 15u * sxr[x];
                        } else if (!ut) {
                            im = 0u - im;
                        }
                        uint32_t *cell = blk + (yl * 32 + xl) * 2;
                        cell[0] += re;
                        cell[1] += im;
                    }
                }
            }
        }
    }
    free(acc_re);
    free(acc_im);
    free(sxr);
    free(sxi);
    free(pr);
    free(pi);
}

uint64_t orc_fnv1a32(const int32_t *v, size_t n) {
    uint64_t h = 0xcbf29ce484222325ull;
    for (size_t i = 0; i < n; i++) {
        h ^= (uint64_t)(uint32_t)v[i];
        h *= 0x100000001b3ull;
    }
    return h;
}

int64_t orc_weighted_power(const uint8_t *packed, int T, int F, int E, int f,
                           const int32_t *w) {
    int64_t total = 0;
    for (int t = 0; t < T; t++) {
        const uint8_t *row = packed + ((size_t)t * F + f) * E;
        int64_t zr = 0, zi = 0;
        for (int e = 0; e < E; e++) {
            const int64_t sr = (int64_t)((row[e] >> 4) & 0x0F) - 8;
            const int64_t si = (int64_t)(row[e] & 0x0F) - 8;
            zr += w[2 * e] * sr - w[2 * e + 1] * si;
            zi += w[2 * e] * si + w[2 * e + 1] * sr;
        }
        total += zr * zr + zi * zi;
    }
    return total;
}

int64_t orc_weighted_from_blocks(const int32_t *blocks, int F, int E, int f,
                                 const int32_t *w) {
    (void)F;
    const int64_t nb1 = E / 32;
    const int64_t nb = orc_num_blocks(E);
    int64_t total = 0;
    for (int64_t by = 0; by < nb1; by++) {
        for (int64_t bx = by; bx < nb1; bx++) {
            const int32_t *blk =
                blocks + ((size_t)(f * nb + block_index(nb1, by, bx))) * 2048;
            for (int yl = 0; yl < 32; yl++) {
                for (int xl = 0; xl < 32; xl++) {
                    const int64_t y = by * 32 + yl, x = bx * 32 + xl;
                    if (x < y) continue;
                    const int64_t vr = blk[(yl * 32 + xl) * 2];
                    const int64_t vi = blk[(yl * 32 + xl) * 2 + 1];
                    const int64_t wyr = w[2 * y], wyi = w[2 * y + 1];
                    const int64_t wxr = w[2 * x], wxi = w[2 * x + 1];
                    /* c = w_y * conj(w_x) */
                    const int64_t cr = wyr * wxr + wyi * wxi;
                    const int64_t ci = wyi * wxr - wyr * wxi;
                    const int64_t re_cv = cr * vr - ci * vi;
                    total += (x == y) ? re_cv : 2 * re_cv;
                }
            }
        }
    }
    return total;
}

void orc_visibility(const uint8_t *packed, int T, int F, int E, int f, int y,
                    int x, int32_t *re, int32_t *im) {
    uint32_t r = 0, i = 0;
    for (int t = 0; t < T; t++) {
        const uint8_t *row = packed + ((size_t)t * F + f) * E;
        const int32_t yr = ((row[y] >> 4) & 0x0F) - 8, yi = (row[y] & 0x0F) - 8;
        const int32_t xr = ((row[x] >> 4) & 0x0F) - 8, xi = (row[x] & 0x0F) - 8;
        r += (uint32_t)(xr * yr + xi * yi);
        i += (uint32_t)(xr * yi - xi * yr);
    }
    *re = (int32_t)r;
    *im = (int32_t)i;
}

/* ------------------------------------------------------------------------
 * Threaded whole-channel correlation for word-for-word checks at full size.
 * Same visibility definition as accumulate_channel (cpu_corr_test.c:188-193,
 * Im negated for ut=0 as in cpu_corr_test.c:91-96) and the same block layout
 * (main_wrapper.c:529-540, preseed_multifreq_UT.cl:128), computed block by
 * block so that host threads can share the work: each thread takes the next
 * block from a shared counter and sums its 32 x 32 cells over the samples.
 */
struct mt_job {
    const int16_t *sr, *si; /* channel samples, [t][E], sign-extended */
    int E, nt, ut;
    int64_t nb1, nblocks;
    int64_t next;           /* next block to take (guarded by mu) */
    pthread_mutex_t mu;
    int32_t *blocks;
};

static void *mt_worker(void *arg) {
    struct mt_job *J = (struct mt_job *)arg;
    uint32_t acc_re[32][32], acc_im[32][32];
    const int E = J->E;
    for (;;) {
        pthread_mutex_lock(&J->mu);
        const int64_t b = J->next++;
        pthread_mutex_unlock(&J->mu);
        if (b >= J->nblocks) break;
        /* block b -> (by, bx): walk the rows of the upper triangle */
        int64_t by = 0, rem = b;
        while (rem >= J->nb1 - by) {
            rem -= J->nb1 - by;
            by++;
        }
        const int64_t bx = by + rem;
        memset(acc_re, 0, sizeof(acc_re));
        memset(acc_im, 0, sizeof(acc_im));
        for (int t = 0; t < J->nt; t++) {
            const int16_t *yr = J->sr + (size_t)t * E + by * 32;
            const int16_t *yi = J->si + (size_t)t * E + by * 32;
            const int16_t *xr = J->sr + (size_t)t * E + bx * 32;
            const int16_t *xi = J->si + (size_t)t * E + bx * 32;
            for (int yl = 0; yl < 32; yl++) {
                const int32_t a = yr[yl], c = yi[yl];
                uint32_t *pr = acc_re[yl], *pi = acc_im[yl];
                for (int xl = 0; xl < 32; xl++) {
                    pr[xl] += (uint32_t)(xr[xl] * a + xi[xl] * c);
                    pi[xl] += (uint32_t)(xr[xl] * c - xi[xl] * a);
                }
            }
        }
        uint32_t *blk = (uint32_t *)J->blocks + (size_t)b * 2048;
        for (int yl = 0; yl < 32; yl++)
            for (int xl = 0; xl < 32; xl++) {
                blk[(yl * 32 + xl) * 2] = acc_re[yl][xl];
                blk[(yl * 32 + xl) * 2 + 1] = J->ut ? acc_im[yl][xl] : 0u - acc_im[yl][xl];
            }
    }
    return NULL;
}

int orc_correlate_channel_mt(const uint8_t *packed, int T, int F, int E, int f,
                             int t0, int t1, int ut, int nthreads,
                             int32_t *blocks) {
    (void)T;
    if (t1 < t0 || E % 32 != 0 || f < 0 || f >= F) return -1;
    const int nt = t1 - t0;
    int16_t *sr = (int16_t *)malloc((size_t)(nt ? nt : 1) * E * sizeof(int16_t));
    int16_t *si = (int16_t *)malloc((size_t)(nt ? nt : 1) * E * sizeof(int16_t));
    if (!sr || !si) {
        free(sr);
        free(si);
        return -2;
    }
    for (int t = 0; t < nt; t++) {
        const uint8_t *row = packed + ((size_t)(t0 + t) * F + f) * E;
        for (int e = 0; e < E; e++) {
            sr[(size_t)t * E + e] = (int16_t)(((row[e] >> 4) & 0x0F) - 8);
            si[(size_t)t * E + e] = (int16_t)((row[e] & 0x0F) - 8);
        }
    }
    struct mt_job J;
    J.sr = sr;
    J.si = si;
    J.E = E;
    J.nt = nt;
    J.ut = ut;
    J.nb1 = E / 32;
    J.nblocks = orc_num_blocks(E);
    J.next = 0;
    J.blocks = blocks;
    pthread_mutex_init(&J.mu, NULL);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    int started = 0;
    for (int i = 1; i < nthreads; i++)
        if (pthread_create(&th[started], NULL, mt_worker, &J) == 0) started++;
    mt_worker(&J); /* the calling thread works too */
    for (int i = 0; i < started; i++) pthread_join(th[i], NULL);
    pthread_mutex_destroy(&J.mu);
    free(sr);
    free(si);
    return 0;
}
