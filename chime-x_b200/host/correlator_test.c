/* correlator_test -- C host program for libchimex with the command line of the
 * reference's correlator harness (main_wrapper.c:52-231): it generates the
 * reference's synthetic 4-bit input, runs the correlator for a number of
 * iterations with the input copied from pinned host memory every iteration
 * (or once, with --timer_without_copies), reports the time and the rate, and
 * with --check_results compares every visibility with a direct CPU sum.
 *
 * Paths (all through include/chimex.h):
 *   default          chx_correlate: the fused exact tensor-core correlator
 *   --pipeline (-P)  the reference's three-kernel pipeline,
 *                    chx_offset_accumulate -> chx_preseed -> chx_corr_compat
 *                    (main_wrapper.c:693-777), family chosen by --kernel_batch
 *   --noalloc (-n)   chx_correlate_noalloc (no plan, no allocation per call)
 * Exit status 0 on success (and, with -c, a matching check), 1 otherwise.
 */
#define _GNU_SOURCE
#include <getopt.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <cuda_runtime.h>

#include "chimex.h"

enum { GEN_CONSTANT = 1, GEN_RAMP_UP = 2, GEN_RAMP_DOWN = 3, GEN_RANDOM = 4 };
#define ALL_FREQUENCIES (-1)

static void print_help(void) {
    printf("Usage: ./correlator_test [opts]\n\n");
    printf("Options:\n");
    printf("  --help (-h)                               Display the available run options.\n");
    printf("  --device (-d) [device_number]             Default: 0.\n");
    printf("  --iterations (-i) [number]                Default: 100. Number of iterations.\n");
    printf("  --time_accum (-t) [number]                Default: 256. Reference kernels: [8,291] conference, [8,2272] packed.\n");
    printf("  --time_steps (-T) [number]                Default: 128 * time_accum.\n");
    printf("  --num_freq (-f) [number]                  Default: 1. Frequency channels per run.\n");
    printf("  --num_elements (-e) [number]              Default: 2048. Elements (multiple of 32).\n");
    printf("  --timer_without_copies (-w)               Default: off. Copy the input once, time the kernels only.\n");
    printf("  --upper_triangle_convention (-U) [0|1]    Default: 1.\n");
    printf("  --check_results (-c)                      Default: off. Compare every visibility with a CPU sum.\n");
    printf("  --verbose (-v)                            Default: off. Print the products (implies -c).\n");
    printf("  --gen_type (-g) [1-4]                     Default: 4 (1 constant, 2 ramp up, 3 ramp down, 4 random).\n");
    printf("  --random_seed (-r) [number]               Default: 42.\n");
    printf("  --no_repeat_random (-p)                   Default: off. A new random sequence every time step.\n");
    printf("  --generate_frequency (-q) [number]        Default: -1 (all). Other channels take the default values.\n");
    printf("  --default_real (-x) [-8..7]               Default: 0.\n");
    printf("  --default_imaginary (-y) [-8..7]          Default: 0.\n");
    printf("  --initial_real (-X) [-8..7]               Default: 0.\n");
    printf("  --initial_imaginary (-Y) [-8..7]          Default: 0.\n");
    printf("  --kernel_batch (-k) [0|1]                 Default: 0 (conference kernels), 1 (packed kernels; -P only).\n");
    printf("  --pipeline (-P)                           Run offset_accumulate -> preseed -> corr_compat.\n");
    printf("  --noalloc (-n)                            Run chx_correlate_noalloc.\n");
}

static int clip_nibble(int v) {
    v += 8;
    return v < 0 ? 0 : (v > 15 ? 15 : v);
}

/* The reference's synthetic input (input_generator.c:17-103): bytes
 * (re+8)<<4 | (im+8), time-major [T][F][E]; the random mode draws two glibc
 * rand() values per element, reseeding every time step unless no_repeat. */
static void generate(int gen, int seed, int dre, int dim, int ire, int iim, int single_freq,
                     int T, int F, int E, int no_repeat, uint8_t *out) {
    if (single_freq > F || single_freq < 0) single_freq = ALL_FREQUENCIES;
    const unsigned d_re = (unsigned)clip_nibble(dre), d_im = (unsigned)clip_nibble(dim);
    const unsigned i_re = (unsigned)clip_nibble(ire), i_im = (unsigned)clip_nibble(iim);
    const uint8_t fill = (uint8_t)((d_re << 4) | d_im);
    if (gen == GEN_RANDOM) srand((unsigned)seed);
    for (int t = 0; t < T; t++) {
        if (gen == GEN_RANDOM && !no_repeat) srand((unsigned)seed);
        for (int f = 0; f < F; f++) {
            uint8_t *row = out + ((size_t)t * F + f) * E;
            for (int e = 0; e < E; e++) {
                unsigned re = d_re, im = d_im;
                if (gen == GEN_CONSTANT) {
                    re = i_re;
                    im = i_im;
                } else if (gen == GEN_RAMP_UP) {
                    re = (unsigned)(f + (int)i_re + e) % 16u;
                    im = (unsigned)(f + (int)i_im + e) % 16u;
                } else if (gen == GEN_RAMP_DOWN) {
                    re = 15u - (unsigned)(f + (int)i_re + e) % 16u;
                    im = 15u - (unsigned)(f + (int)i_im + e) % 16u;
                } else if (gen == GEN_RANDOM) {
                    re = (unsigned)(rand() % 16);
                    im = (unsigned)(rand() % 16);
                }
                uint8_t b = (uint8_t)(((re & 15u) << 4) | (im & 15u));
                if (single_freq != ALL_FREQUENCIES && f != single_freq) b = fill;
                row[e] = b;
            }
        }
    }
}

/* Checks the triangle [F][E(E+1)/2][2] against direct sums
 * V[y][x] = sum_t s_y conj(s_x) (Im negated for the non-UT convention).
 * Rows are split over OpenMP threads; returns the number of mismatches. */
static long long check_triangle(const uint8_t *in, const int32_t *tri, int T, int F, int E,
                                int ut, int verbose) {
    long long errors = 0;
    const int64_t per_chan = (int64_t)E * (E + 1) / 2;
    for (int f = 0; f < F; f++) {
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : errors)
        for (int y = 0; y < E; y++) {
            int64_t *re = (int64_t *)calloc((size_t)(E - y), sizeof(int64_t));
            int64_t *im = (int64_t *)calloc((size_t)(E - y), sizeof(int64_t));
            for (int t = 0; t < T; t++) {
                const uint8_t *row = in + ((size_t)t * F + f) * E;
                const int yr = (row[y] >> 4) - 8, yi = (row[y] & 15) - 8;
                for (int x = y; x < E; x++) {
                    const int xr = (row[x] >> 4) - 8, xi = (row[x] & 15) - 8;
                    re[x - y] += yr * xr + yi * xi;
                    im[x - y] += yi * xr - yr * xi;
                }
            }
            const int64_t base = (int64_t)f * per_chan + (int64_t)y * E - (int64_t)y * (y - 1) / 2;
            for (int x = y; x < E; x++) {
                const int32_t gr = tri[2 * (base + x - y)], gi = tri[2 * (base + x - y) + 1];
                const int32_t cr = (int32_t)re[x - y], ci = (int32_t)(ut ? im[x - y] : -im[x - y]);
                if (gr != cr || gi != ci) {
                    if (errors < 10)
                        printf("  mismatch f=%d y=%d x=%d: GPU (%d, %d) CPU (%d, %d)\n", f, y, x,
                               gr, gi, cr, ci);
                    errors++;
                } else if (verbose && E <= 64) {
                    printf("  f=%d y=%d x=%d: (%d, %d)\n", f, y, x, gr, gi);
                }
            }
            free(re);
            free(im);
        }
    }
    return errors;
}

#define CK(call)                                                                        \
    do {                                                                                \
        int rc_ = (call);                                                               \
        if (rc_ != CHX_OK) {                                                            \
            fprintf(stderr, "%s failed (%d): %s\n", #call, rc_, chx_last_error());      \
            return 1;                                                                   \
        }                                                                               \
    } while (0)
#define CU(call)                                                                        \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            fprintf(stderr, "%s failed: %s\n", #call, cudaGetErrorString(e_));          \
            return 1;                                                                   \
        }                                                                               \
    } while (0)

int main(int argc, char **argv) {
    int device = 0, iterations = 100, num_freq = 1, num_elem = 2048, time_accum = 256;
    int time_steps = 256 * 128, t_set = 0, no_copies = 0, check = 0, verbose = 0;
    int gen = GEN_RANDOM, seed = 42, no_repeat = 0, gen_freq = ALL_FREQUENCIES;
    int dre = 0, dim = 0, ire = 0, iim = 0, kernel_batch = 0, ut = 1, pipeline = 0,
        noalloc = 0;
    static struct option opts[] = {
        {"device", required_argument, 0, 'd'},
        {"iterations", required_argument, 0, 'i'},
        {"num_freq", required_argument, 0, 'f'},
        {"num_elements", required_argument, 0, 'e'},
        {"num_elem", required_argument, 0, 'e'},
        {"time_accum", required_argument, 0, 't'},
        {"time_steps", required_argument, 0, 'T'},
        {"timer_without_copies", no_argument, 0, 'w'},
        {"upper_triangle_convention", required_argument, 0, 'U'},
        {"check_results", no_argument, 0, 'c'},
        {"verbose", no_argument, 0, 'v'},
        {"gen_type", required_argument, 0, 'g'},
        {"random_seed", required_argument, 0, 'r'},
        {"no_repeat_random", no_argument, 0, 'p'},
        {"generate_frequency", required_argument, 0, 'q'},
        {"default_real", required_argument, 0, 'x'},
        {"default_imaginary", required_argument, 0, 'y'},
        {"initial_real", required_argument, 0, 'X'},
        {"initial_imaginary", required_argument, 0, 'Y'},
        {"kernel_batch", required_argument, 0, 'k'},
        {"pipeline", no_argument, 0, 'P'},
        {"noalloc", no_argument, 0, 'n'},
        {"help", no_argument, 0, 'h'},
        {0, 0, 0, 0}};
    for (;;) {
        int idx = 0;
        const int o = getopt_long(argc, argv, "d:i:f:e:t:T:wcvg:r:pq:x:y:X:Y:hk:U:Pn", opts, &idx);
        if (o == -1) break;
        switch (o) {
        case 'h': print_help(); return 0;
        case 'd': device = atoi(optarg); break;
        case 'i': iterations = atoi(optarg); break;
        case 'f': num_freq = atoi(optarg); break;
        case 'e': num_elem = atoi(optarg); break;
        case 't':
            time_accum = atoi(optarg);
            if (!t_set) time_steps = 128 * time_accum;
            break;
        case 'T':
            time_steps = atoi(optarg);
            t_set = 1;
            break;
        case 'w': no_copies = 1; break;
        case 'c': check = 1; break;
        case 'v': verbose = check = 1; break;
        case 'g':
            gen = atoi(optarg);
            if (gen < 1 || gen > 4) {
                printf("Invalid parameter for gen_type.  See help for options\n");
                print_help();
                return 1;
            }
            break;
        case 'r': seed = atoi(optarg); break;
        case 'p': no_repeat = 1; break;
        case 'q': gen_freq = atoi(optarg); break;
        case 'x': dre = atoi(optarg); break;
        case 'y': dim = atoi(optarg); break;
        case 'X': ire = atoi(optarg); break;
        case 'Y': iim = atoi(optarg); break;
        case 'k':
            kernel_batch = atoi(optarg);
            if (kernel_batch < 0 || kernel_batch > 1) {
                printf("Invalid parameter for kernel_batch.  See help for options\n");
                print_help();
                return 1;
            }
            break;
        case 'U':
            ut = atoi(optarg);
            if (ut < 0 || ut > 1) {
                printf("Invalid parameter for upper_triangle_convention.  See help for options\n");
                print_help();
                return 1;
            }
            break;
        case 'P': pipeline = 1; break;
        case 'n': noalloc = 1; break;
        default: print_help(); return 1;
        }
    }
    if (iterations < 1) {
        printf("iterations must be >= 1\n");
        return 1;
    }

    chx_plan *plan = NULL;
    CK(chx_plan_create(&plan, num_elem, num_freq, time_steps, time_accum, ut, kernel_batch,
                       device));
    CU(cudaSetDevice(device));
    const size_t in_bytes = (size_t)chx_plan_input_bytes(plan);
    const size_t out_words = (size_t)chx_plan_block_words(plan);
    const size_t tri_words = (size_t)chx_plan_triangle_words(plan);
    printf("Num_blocks %lld Output Length %zu and size %zu B\n",
           (long long)(num_elem / 32) * (num_elem / 32 + 1) / 2, out_words, out_words * 4);
    printf("Size of Data block = %zu B\n", in_bytes);

    uint8_t *h_in = NULL, *d_in = NULL;
    int32_t *d_blocks = NULL, *d_tri = NULL;
    uint32_t *d_sums = NULL;
    CU(cudaMallocHost((void **)&h_in, in_bytes));
    CU(cudaMalloc((void **)&d_in, in_bytes));
    CU(cudaMalloc((void **)&d_blocks, out_words * 4));
    if (pipeline) CU(cudaMalloc((void **)&d_sums, (size_t)chx_plan_sum_words(plan) * 4));
    generate(gen, seed, dre, dim, ire, iim, gen_freq, time_steps, num_freq, num_elem, no_repeat,
             h_in);

    cudaStream_t st;
    CU(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    cudaEvent_t e0, e1;
    CU(cudaEventCreate(&e0));
    CU(cudaEventCreate(&e1));
    if (no_copies) CU(cudaMemcpyAsync(d_in, h_in, in_bytes, cudaMemcpyHostToDevice, st));
    printf("Running %i iterations of full corr (%i time samples (%i Ki time samples), %i elements, "
           "%i frequencies)\n",
           iterations, time_steps, time_steps / 1024, num_elem, num_freq);
    CU(cudaEventRecord(e0, st));
    for (int it = 0; it < iterations; it++) {
        if (!no_copies) CU(cudaMemcpyAsync(d_in, h_in, in_bytes, cudaMemcpyHostToDevice, st));
        if (pipeline) {
            CK(chx_offset_accumulate(plan, d_in, d_sums, st, 0));
            CK(chx_preseed(plan, d_sums, d_blocks, st));
            CK(chx_corr_compat(plan, d_in, d_blocks, st));
        } else if (noalloc) {
            CK(chx_correlate_noalloc(d_in, d_blocks, num_elem, num_freq, time_steps, ut, 0, st));
        } else {
            CK(chx_correlate(plan, d_in, d_blocks, st, 0));
        }
    }
    CU(cudaEventRecord(e1, st));
    CU(cudaEventSynchronize(e1));
    if (!noalloc) CK(chx_plan_check(plan, st));
    else CK(chx_noalloc_check(st));
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, e0, e1));
    const double secs = ms * 1e-3;
    const double ops = 8.0 * num_elem * (num_elem + 1.0) / 2.0 * time_steps * num_freq * iterations;
    printf("Correlation matrices computation time: %6.4fs on GPU (%.1f kHz of 400 MHz band, or "
           "%.1fx10^3 correlation matrices/s)\n",
           secs, (double)time_steps * num_freq / secs / 1000 * iterations,
           (double)time_steps * num_freq / secs / 1000 * iterations);
    printf("    [%.1f TOPS exact int8 (8*E(E+1)/2*T*F per iteration), %s]\n", ops / secs / 1e12,
           no_copies ? "kernels only" : "host copies included");

    int status = 0;
    if (check) {
        printf("Checking results. Please wait...\n");
        int32_t *h_tri = (int32_t *)malloc(tri_words * 4);
        if (!h_tri) {
            printf("failed to allocate memory\n");
            return 1;
        }
        CU(cudaMalloc((void **)&d_tri, tri_words * 4));
        CK(chx_blocks_to_triangle(plan, d_blocks, d_tri, st));
        CU(cudaMemcpyAsync(h_tri, d_tri, tri_words * 4, cudaMemcpyDeviceToHost, st));
        CU(cudaStreamSynchronize(st));
        const clock_t c0 = clock();
        const long long errors =
            check_triangle(h_in, h_tri, time_steps, num_freq, num_elem, ut, verbose);
        const double cpu_s = (double)(clock() - c0) / CLOCKS_PER_SEC;
        if (errors) {
            printf("Error with correlation/accumulation! Num Err: %lld and length of correlated "
                   "data: %zu\n",
                   errors, tri_words / 2);
            status = 1;
        } else {
            printf("Correlation/accumulation successful! CPU matches GPU.\n");
        }
        printf("Full Corr: %4.2fs CPU time\n", cpu_s);
        free(h_tri);
        cudaFree(d_tri);
    } else {
        printf("\nGPU calculations have not been verified (use -c).\n\n");
    }
    cudaFree(d_in);
    cudaFree(d_blocks);
    if (d_sums) cudaFree(d_sums);
    cudaFreeHost(h_in);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(st);
    chx_plan_destroy(plan);
    return status;
}
