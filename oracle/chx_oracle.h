/*
 * chx_oracle.h -- CPU restatement of the CHIME-x correlator arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * product path: only tests/, the smoke check and the CPU-baseline leg of
 * bench.py load it.  The product library (libchimex) never links it.
 *
 * Every routine restates the integer arithmetic of one reference routine
 * (cited per function, paths relative to the CHIME-x project root).  All
 * int32 arithmetic wraps modulo 2^32 exactly as the reference's C / OpenCL
 * integer arithmetic does (computed in uint32 to avoid C signed-overflow UB).
 *
 * Parity of this restatement is pinned against the reference's own CPU code
 * (cpu_corr_test.c, input_generator.c, gpu_data_reorg.c) compiled from its
 * sources into oracle/_ref/ by oracle/Makefile, and against the known-answer
 * hashes committed under tests/golden/.
 */
#ifndef CHX_ORACLE_H
#define CHX_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Generator types, as in generator_defs.h:5-8. */
#define ORC_GEN_CONSTANT 1
#define ORC_GEN_RAMP_UP 2
#define ORC_GEN_RAMP_DOWN 3
#define ORC_GEN_RANDOM_SEEDED 4
#define ORC_ALL_FREQUENCIES (-1)

/* Seeded 4-bit data generator with the semantics of
 * generate_char_data_set (input_generator.c:17-103).  Writes T*F*E bytes,
 * byte = (re+8)<<4 | (im+8), address t*F*E + f*E + e. */
void orc_generate(int gen_type, int seed, int default_re, int default_im,
                  int initial_re, int initial_im, int single_freq, int T,
                  int F, int E, int no_repeat_random, uint8_t *out);

/* Number of 32x32 blocks in the upper triangle of an E-element matrix
 * (main_wrapper.c:277-278). */
int64_t orc_num_blocks(int E);

/* Full correlation in the GPU block layout int32[F][NB][32][32][2]
 * (pairwise_correlator_UT.cl:161, preseed_multifreq_UT.cl:128), including the
 * lower halves of the diagonal blocks.  ut=1: V[y][x] = sum s_y conj(s_x)
 * (cpu_corr_test.c:188-193); ut=0: imaginary part negated
 * (cpu_corr_test.c:91-96).  accumulate=0 overwrites, 1 adds. */
void orc_correlate_blocks(const uint8_t *packed, int T, int F, int E, int ut,
                          int accumulate, int32_t *blocks);

/* Same visibilities restricted to a sample range [t0, t1). */
void orc_correlate_blocks_range(const uint8_t *packed, int T, int F, int E,
                                int t0, int t1, int ut, int accumulate,
                                int32_t *blocks);

/* One channel's blocks int32[NB][32][32][2] over samples [t0, t1), the same
 * values as orc_correlate_blocks_range for channel f, computed block by block
 * on nthreads host threads (word-for-word checks at full size).  Returns 0. */
int orc_correlate_channel_mt(const uint8_t *packed, int T, int F, int E, int f,
                             int t0, int t1, int ut, int nthreads,
                             int32_t *blocks);

/* Upper-triangle correlation int32[F][E(E+1)/2][2], the reference CPU
 * check (cpu_corr_test.c:156-203 for ut=1, :59-106 for ut=0). */
void orc_correlate_triangle(const uint8_t *packed, int T, int F, int E, int ut,
                            int32_t *tri);

/* Block layout -> packed upper triangle (gpu_data_reorg.c:76-124). */
void orc_blocks_to_triangle(const int32_t *blocks, int F, int E, int32_t *tri);

/* Block layout -> full Hermitian matrix int32[F][E][E][2]
 * (gpu_data_reorg.c:36-74). */
void orc_blocks_to_full(const int32_t *blocks, int F, int E, int32_t *full);

/* Offset-binary nibble sums S[f][e][re,im] over all T samples
 * (offset_accumulator.cl:7-49).  accumulate=1 adds into sums. */
void orc_offset_accumulate(const uint8_t *packed, int T, int F, int E,
                           int accumulate, uint32_t *sums);

/* Preseed: writes the offset correction into every block cell.
 * packed_variant=0: conference kernels (preseed_multifreq_UT.cl:43-115,
 * preseed_multifreq.cl); 1: highly-packed kernels
 * (preseed_multifreq_highly_packed_correlator_method_UT.cl:43-117 and the
 * non-UT file).  T is the NUM_TIMESAMPLES term of the 128*T constant. */
void orc_preseed(const uint32_t *sums, int T, int F, int E, int packed_variant,
                 int ut, int32_t *blocks);

/* The partial the reference corr kernel adds into the block buffer for all
 * T/TA chunks, in its exact domain: offset-domain products for the
 * conference kernel (pairwise_correlator_UT.cl:82-201), inverted-imaginary
 * products for the packed kernel
 * (packed_correlator_overflow_protected_to_2272_iter_UT.cl:84-285).
 * Adds into blocks. */
void orc_corr_partials(const uint8_t *packed, int T, int F, int E,
                       int packed_variant, int ut, int32_t *blocks);

/* 64-bit FNV-1a over int32 words taken as uint32. */
uint64_t orc_fnv1a32(const int32_t *v, size_t n);

/* Checksum identity used at full sizes: for integer weights w (E of them,
 * complex, re/im interleaved), returns sum_t |sum_e w_e s_e(t)|^2 for one
 * channel as an int64 (the exact value of sum_{y,x} conj(w_y) w_x V*... see
 * orc_weighted_from_blocks). */
int64_t orc_weighted_power(const uint8_t *packed, int T, int F, int E, int f,
                           const int32_t *w);

/* The same quantity evaluated from a block buffer (ut=1 convention):
 * sum_y |w_y|^2 V[y][y] + 2 Re sum_{x>y} w_y conj(w_x) V[y][x]. */
int64_t orc_weighted_from_blocks(const int32_t *blocks, int F, int E, int f,
                                 const int32_t *w);

/* One visibility computed directly in O(T) (ut=1), for spot checks. */
void orc_visibility(const uint8_t *packed, int T, int F, int E, int f, int y,
                    int x, int32_t *re, int32_t *im);

#ifdef __cplusplus
}
#endif

#endif
