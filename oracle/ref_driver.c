/*
 * ref_driver.c -- test/baseline driver linked against the reference's own CPU
 * correlator (cpu_corr_test.c:156-203 and :59-106) built from its sources.
 *
 * Usage: cpu_corr_ref T F E gen_type seed no_repeat ut
 * Runs the reference's generate-and-correlate routine once and prints one
 * JSON line with the wall time and the FNV-1a hash of the triangle.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <time.h>

#include "cpu_corr_test.h"

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + ts.tv_nsec * 1e-9;
}

int main(int argc, char **argv) {
    if (argc < 8) {
        fprintf(stderr, "usage: %s T F E gen_type seed no_repeat ut\n", argv[0]);
        return 2;
    }
    const int T = atoi(argv[1]), F = atoi(argv[2]), E = atoi(argv[3]);
    const int gen = atoi(argv[4]), seed = atoi(argv[5]);
    const int no_repeat = atoi(argv[6]), ut = atoi(argv[7]);
    const size_t n = (size_t)F * E * (E + 1);
    int *tri = (int *)calloc(n, sizeof(int));
    if (!tri) return 1;
    const double t0 = now_s();
    int err;
    if (ut)
        err = cpu_data_generate_and_correlate_upper_triangle_only(
            T, F, E, tri, gen, seed, 0, 0, 0, 0, -1, no_repeat, 0);
    else
        err = cpu_data_generate_and_correlate_upper_triangle_only_nonstandard_convention(
            T, F, E, tri, gen, seed, 0, 0, 0, 0, -1, no_repeat, 0);
    const double dt = now_s() - t0;
    uint64_t h = 0xcbf29ce484222325ull;
    for (size_t i = 0; i < n; i++) {
        h ^= (uint64_t)(uint32_t)tri[i];
        h *= 0x100000001b3ull;
    }
    printf("{\"seconds\": %.6f, \"hash\": \"%016llx\", \"updates\": %.0f, \"err\": %d}\n",
           dt, (unsigned long long)h, (double)E * (E + 1) / 2.0 * T * F, err);
    free(tri);
    return err ? 1 : 0;
}
