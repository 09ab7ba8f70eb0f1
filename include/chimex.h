/*
 * chimex.h -- C ABI of libchimex, the B200 (sm_100a) CHIME X-engine.
 *
 * Drop-in replacement for the device side of CHIME-x's correlator_test: the
 * reference builds three OpenCL kernels (corr, offsetAccumulateElements,
 * preseed) with the problem size baked in as -D macros
 * (main_wrapper.c:309-372) and launches them on an event-chained queue
 * (main_wrapper.c:693-777).  Here the problem size lives in a plan, every
 * kernel takes plain device pointers, and the fused chx_correlate replaces the
 * whole accumulate -> preseed -> corr chain.
 *
 * Data contract (identical to the reference):
 *   input   uint8 [T][F][E]: byte = (re+8)<<4 | (im+8), re, im in [-8, 7]
 *           (four_bit_macros.h:8-9, input_generator.c:58,85)
 *   output  int32 [F][NB][32][32][2] (re, im) with NB = (E/32)(E/32+1)/2
 *           blocks enumerated row-major over the upper triangle
 *           (main_wrapper.c:529-540), cell (y, x) = V[y][x] with y the row
 *           element, x >= y's block column; diagonal blocks hold all 32x32
 *           cells (pairwise_correlator_UT.cl:161, gpu_data_reorg.c:76-124).
 *   V[y][x] = sum_t s_y conj(s_x) for upper_triangle_convention = 1
 *           (cpu_corr_test.c:188-193); the imaginary part is negated for 0
 *           (cpu_corr_test.c:91-96).
 *
 * Conventions: every function returns CHX_OK (0) or a negative CHX_E_* code
 * and sets a thread-local message readable with chx_last_error().  Device
 * pointers must be 16-byte aligned (TMA and vector accesses; cudaMalloc and
 * torch allocations are 256-byte aligned) and are refused with CHX_E_INVALID
 * otherwise.  Device pointers and streams are owned by the caller; the library owns its plans,
 * their small device-side tables and any scratch a plan allocates at
 * creation.  Work is enqueued asynchronously on the given stream (a
 * cudaStream_t passed as void*; NULL = the legacy default stream).  A plan is
 * thread-compatible: one thread at a time per plan.
 */
#ifndef CHIMEX_H
#define CHIMEX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CHX_OK 0
#define CHX_E_INVALID (-1)     /* bad argument or shape */
#define CHX_E_UNSUPPORTED (-2) /* valid, but outside what this library handles */
#define CHX_E_CUDA (-3)        /* a CUDA runtime call failed */
#define CHX_E_NOMEM (-4)       /* device or host allocation failed */
#define CHX_E_TIMEOUT (-5)     /* a bounded device-side wait gave up */
#define CHX_E_NOT_READY (-6)   /* asynchronous result not available yet */
#define CHX_E_ADMISSION (-7)   /* streaming admission refused (HBM budget) */

/* Kernel families of the reference (main_wrapper.c:282-305, -k flag). */
#define CHX_KERNEL_CONFERENCE 0 /* pairwise_correlator*.cl + preseed_multifreq*.cl */
#define CHX_KERNEL_PACKED 1     /* packed_correlator_overflow_protected_to_2272_iter*.cl */

/* Algorithms for the fused plain path (chx_plan_set_option CHX_OPT_ALGO). */
#define CHX_ALGO_AUTO 0 /* tensor-core path when the shape allows it */
#define CHX_ALGO_SIMT 1 /* CUDA-core dp4a kernel (baseline / small shapes) */
#define CHX_ALGO_TC 2   /* tcgen05 kind::i8 kernel */

/* Plan options. */
#define CHX_OPT_ALGO 1      /* one of CHX_ALGO_* */
#define CHX_OPT_TSPLIT 2    /* number of sample-range splits: 0 auto (the
                               autotuned value, else the split with the
                               shortest estimated makespan, so that few
                               channels still fill the GPU), n >= 1 fixed */
#define CHX_OPT_TILE 3      /* tensor-core tile variant: 0 auto (the
                               autotuned variant, else the SM pair from
                               E > 128 up and one SM below), 1 one SM
                               (128 x 256 elements), 2 SM pair (256 x 256) */

typedef struct chx_plan chx_plan;

/* Library version, e.g. "chimex-b200 0.1". */
const char *chx_version(void);

/* Message describing the last failure on this thread ("" if none). */
const char *chx_last_error(void);

/* Creates a plan for E elements, F channels, T samples per call.
 * Replaces the -D NUM_ELEMENTS/NUM_FREQUENCIES/NUM_BLOCKS/NUM_TIMESAMPLES/
 * NUM_TIME_ACCUM build of main_wrapper.c:277-312.  Requires E % 32 == 0
 * (32-element blocks, main_wrapper.c:277-278), F >= 1, 1 <= T <= 16777215
 * (int32 exactness: |Re|, |Im| <= 128 T), upper_triangle_convention in
 * {0, 1}, kernel_batch in {0, 1}.  time_accum only constrains the reference
 * compatibility kernels (chx_corr_compat); the fused path is exact for any
 * T and time_accum.  device = CUDA ordinal. */
int chx_plan_create(chx_plan **plan, int num_elements, int num_frequencies,
                    int num_timesamples, int time_accum,
                    int upper_triangle_convention, int kernel_batch, int device);
int chx_plan_destroy(chx_plan *plan);

/* Sets an option (CHX_OPT_*) on a plan. */
int chx_plan_set_option(chx_plan *plan, int option, int64_t value);

/* Sizes in elements: output block buffer (F*NB*2048 int32), packed input
 * (T*F*E bytes), offset sums (F*E*2 uint32), triangle (F*E*(E+1) int32). */
int64_t chx_plan_block_words(const chx_plan *plan);
int64_t chx_plan_input_bytes(const chx_plan *plan);
int64_t chx_plan_sum_words(const chx_plan *plan);
int64_t chx_plan_triangle_words(const chx_plan *plan);

/* Fused correlator: exact visibilities of d_packed written into d_blocks in
 * the reference block layout.  accumulate = 0 overwrites d_blocks, 1 adds
 * to it.  Replaces the offsetAccumulateElements -> preseed -> corr chain of
 * main_wrapper.c:693-777 (whose net result is the same buffer).  The
 * tensor-core path needs d_packed and d_blocks 16-byte aligned (TMA) and
 * returns CHX_E_INVALID otherwise. */
int chx_correlate(chx_plan *plan, const uint8_t *d_packed, int32_t *d_blocks,
                  void *stream, int accumulate);

/* Offset-binary nibble sums, uint32 [F][E][re, im] over T samples.
 * Replaces offsetAccumulateElements (offset_accumulator.cl:7-49).
 * accumulate = 0 zeroes d_sums first (main_wrapper.c:671-679 zeroes the
 * buffer before every run); 1 adds like the reference's atomic_add. */
int chx_offset_accumulate(chx_plan *plan, const uint8_t *d_packed,
                          uint32_t *d_sums, void *stream, int accumulate);

/* Writes (=) the offset correction into every block cell from the sums, for
 * the plan's kernel_batch and convention.  Replaces preseed
 * (preseed_multifreq_UT.cl:20-25, preseed_multifreq.cl,
 * preseed_multifreq_highly_packed_correlator_method{_UT,}.cl). */
int chx_preseed(chx_plan *plan, const uint32_t *d_sums, int32_t *d_blocks,
                void *stream);

/* Adds the reference corr kernel's partials (offset-domain products for the
 * conference family, inverted-imaginary products for the packed family) to
 * d_blocks, so that accumulate -> preseed -> corr_compat reproduces the
 * reference pipeline bit for bit.  Replaces corr
 * (pairwise_correlator_UT.cl:23-27,
 * packed_correlator_overflow_protected_to_2272_iter_UT.cl:16-20).  Enforces
 * the reference's own domain: T % time_accum == 0, time_accum % 8 == 0,
 * T % 32 == 0, time_accum <= 291 (conference) or <= 2272 (packed), and
 * F == 1 for the packed family (its kernel has no channel index). */
int chx_corr_compat(chx_plan *plan, const uint8_t *d_packed, int32_t *d_blocks,
                    void *stream);

/* Block layout -> packed upper triangle int32 [F][E(E+1)/2][2], on the
 * device.  Replaces the host reorganize_GPU_to_upper_triangle
 * (gpu_data_reorg.c:76-124). */
int chx_blocks_to_triangle(chx_plan *plan, const int32_t *d_blocks,
                           int32_t *d_triangle, void *stream);

/* Block layout -> full Hermitian matrix int32 [F][E][E][2] on the device.
 * Replaces reorganize_GPU_to_full_Matrix_for_comparison
 * (gpu_data_reorg.c:36-74). */
int chx_blocks_to_full(chx_plan *plan, const int32_t *d_blocks, int32_t *d_full,
                       void *stream);

/* Fused correlator for callers that cannot allocate memory.  It has no
 * counterpart in the reference.  It is meant for the per-frame loop of a
 * real-time correlator that reserves all of its device memory at start-up:
 * inside that loop cudaMalloc/cudaFree may stall every stream of the device
 * (they can synchronise it), may fail once the reserved pools hold the
 * memory, and are forbidden outright when another runtime owns the device
 * allocator.  chx_correlate needs a plan, and creating a plan allocates.
 * This entry point computes exactly what chx_correlate computes for a plan
 * of (E, F, T, upper_triangle_convention), needs no plan and calls no
 * allocator: its work tables live in a fixed-size array inside the library
 * (about 162 KiB on every GPU that loads it, kept until exit), written on the
 * device by a small kernel from its launch parameters.  It uses the plan
 * path's default tile variant and cuts sample ranges only where int32
 * exactness requires it (no automatic split).  Limits: F <= 64 channels and
 * at most 4096 work units (36 per E=2048 channel per 262144 samples); larger
 * calls return CHX_E_UNSUPPORTED.  The first call on each device (and again
 * after a device reset) looks the array up, which loads the library's device
 * code; make that first call before any stream capture.  All calls share the
 * array: calls whose kernels overlap on the GPU race, so order them on one
 * stream or with events.  Device-side wait timeouts are recorded in the
 * array and reported by chx_noalloc_check. */
int chx_correlate_noalloc(const uint8_t *d_packed, int32_t *d_blocks, int num_elements,
                          int num_frequencies, int num_timesamples,
                          int upper_triangle_convention, int accumulate, void *stream);

/* Reads and clears the error word of chx_correlate_noalloc on the current
 * device: the bounded-wait timeouts of every call made since the last check.
 * Synchronises the stream; allocates nothing.  Returns CHX_OK or
 * CHX_E_TIMEOUT.  No counterpart in the reference. */
int chx_noalloc_check(void *stream);

/* Reads and clears the plan's device error word (bounded-wait timeouts).
 * Synchronises the stream.  Returns CHX_OK or CHX_E_TIMEOUT. */
int chx_plan_check(chx_plan *plan, void *stream);

/* Self-test of the bounded device-side waits (no counterpart in the
 * reference, whose kernels spin without a bound).  Runs one CTA on `device`
 * that waits, with the same helper and 2 s limit as the correlator kernels,
 * on a barrier phase that nothing completes: mode 0 lets the limit run out,
 * mode 1 raises the CTA's abort flag after ~10 ms, mode 2 does as mode 1 and
 * then records the give-up in chx_correlate_noalloc's error word (read by
 * chx_noalloc_check) as a correlator kernel would.  Returns CHX_E_TIMEOUT when
 * the wait gave up as designed (elapsed_ms: how long it waited), CHX_E_INVALID
 * if it claimed completion, CHX_E_CUDA on a CUDA error.  The context stays
 * usable afterwards. */
int chx_selftest_bounded_wait(int device, int mode, int *elapsed_ms);

/* ---------------------------------------------------------------------
 * Batched ragged launch: many channels with their own element counts and
 * sample counts in one persistent launch (captured in a CUDA graph).
 * ------------------------------------------------------------------- */
typedef struct chx_channel_desc {
    int num_elements;      /* E_c, multiple of 32 */
    int num_timesamples;   /* samples per integration, T_c */
    int num_integrations;  /* integrations, each dumped to its own buffer */
    int64_t input_stride;  /* bytes between consecutive samples (0 = E_c) */
    const uint8_t *d_packed; /* [num_integrations * T_c] samples of E_c bytes */
    int32_t *d_blocks;     /* num_integrations block buffers of NB_c*2048 */
} chx_channel_desc;

/* A batch is thread-compatible like a plan: one thread at a time per batch.
 * Its channels' buffers stay owned by the caller and must outlive it. */
typedef struct chx_batch chx_batch;

/* Builds the tile queue for n channels.  The descriptors are copied.  The
 * channel work is ordered by a cost model.  The tile variant is the
 * autotuner's (chx_autotune) for the costliest channel when cached, else the
 * default; the sample split is one for the whole batch, chosen by a makespan
 * estimate so that a few long channels still fill the GPU. */
int chx_batch_create(chx_batch **batch, int n, const chx_channel_desc *descs,
                     int upper_triangle_convention, int device);
/* Enqueues the whole batch (one graph launch).  accumulate as chx_correlate. */
int chx_batch_run(chx_batch *batch, void *stream, int accumulate);
/* Work units (tile pairs x splits) in the queue, and exact ops per run. */
int64_t chx_batch_work_units(const chx_batch *batch);
double chx_batch_ops(const chx_batch *batch);
/* Reads and clears the batch's device error word (bounded-wait timeouts).
 * Synchronises the stream.  Returns CHX_OK or CHX_E_TIMEOUT. */
int chx_batch_check(chx_batch *batch, void *stream);
int chx_batch_destroy(chx_batch *batch);

/* Times the tensor-core tile variants and split counts for channels of
 * (E, T) on the current device and caches the winner.  It times enough
 * channels to fill the GPU (about two waves of SM-pair units; beyond the one
 * channel the caller's scratch holds it allocates temporary buffers, up to 64
 * channels and 2 GiB), so the choice reflects each variant's speed rather
 * than how many SMs a lone channel leaves idle.  Batches and plans created
 * afterwards with CHX_OPT_TILE left at 0 take its tile for channels of the
 * same E and a T within a factor 2.  Their sample split comes from their own
 * makespan estimate, which sees how many units the whole launch has.
 * d_scratch_in/d_scratch_out must hold T*E bytes and NB*2048 int32. */
int chx_autotune(int num_elements, int num_timesamples, const uint8_t *d_scratch_in,
                 int32_t *d_scratch_out, void *stream, int *best_tile,
                 int *best_split, double *best_ms);

/* ---------------------------------------------------------------------
 * Streaming: frames of samples arrive per channel and every time_accum
 * samples the channel's integration is correlated and dumped.  The reference
 * has no streaming layer: its host loop (main_wrapper.c) correlates whole
 * buffers; this is the serving form of the same correlation.
 *
 * Each admitted channel holds, until chx_stream_destroy, an input ring of two
 * integrations (2*time_accum*E bytes) and two dump buffers (2*NB*8 KiB), all
 * in HBM.  A submit appends one frame per listed channel; the channels whose
 * integration completes are correlated by one tensor-core launch on the given
 * stream (the integration accumulates in tensor memory and is written to its
 * dump buffer once).
 * ------------------------------------------------------------------- */
/* A stream is driven by one host thread at a time (admit, submit, stats);
 * its completion thread only publishes finished dumps. */
typedef struct chx_stream chx_stream;

typedef struct chx_stream_stats {
    int64_t frames;         /* frames submitted */
    int64_t dumps;          /* integrations completed on the device */
    double p50_ms, p99_ms;  /* last-frame-arrival to dump-complete latency */
    double max_ms;
    int64_t resident_bytes; /* HBM held by rings, dump buffers, channel table */
} chx_stream_stats;

/* frame_len: samples per frame (multiple of 32).  hbm_budget_bytes > 0 caps
 * the resident bytes; 0 admits while cudaMemGetInfo leaves 2 GiB free. */
int chx_stream_create(chx_stream **s, int max_channels, int frame_len,
                      int upper_triangle_convention, int64_t hbm_budget_bytes,
                      int device);
/* Admits a channel with E elements dumping every time_accum samples (a
 * multiple of frame_len, at most 262144).  Returns CHX_E_ADMISSION, admitting
 * nothing, when its ring and dump buffers do not fit. */
int chx_stream_admit(chx_stream *s, int num_elements, int time_accum,
                     int *channel_id);
/* Device address where channel c's next frame (frame_len*E bytes) belongs.
 * A producer that writes frames there itself (then submits with d_frames
 * NULL) must not write into a ring half whose integration is still being
 * correlated: wait for the dump of that integration first. */
int chx_stream_frame_slot(chx_stream *s, int channel_id, uint8_t **d_slot);
/* Appends one frame per listed channel.  d_frames NULL, or an entry equal to
 * the channel's frame slot: the frame is already in place; otherwise
 * d_frames[i] (device memory) is copied into the ring on `stream`.
 * arrival_ns: CLOCK_MONOTONIC arrival time of each frame (NULL = now).  Host
 * tables are reused after 8 launches, so a submit may wait for the launch
 * 8 submits back. */
int chx_stream_submit(chx_stream *s, int n, const int *channel_ids,
                      const uint8_t *const *d_frames, const int64_t *arrival_ns,
                      void *stream);
/* Channel c's last integration whose dump has completed on the device and
 * been published by the stream's completion thread (NULL, seq -1 if none),
 * and its sequence number.  The buffer is overwritten when integration seq+2
 * completes.  Completion is observed by a host thread that polls, with
 * 20 us sleeps in between, an event recorded after each launch;
 * chx_stream_sync waits for it. */
int chx_stream_last_dump(chx_stream *s, int channel_id, const int32_t **d_blocks,
                         int64_t *seq);
/* Counters and latency percentiles over the dumps completed so far. */
int chx_stream_stats_get(chx_stream *s, chx_stream_stats *out);
/* Forgets the latency samples (counters stay). */
int chx_stream_reset_stats(chx_stream *s);
/* Waits until every launch submitted so far has completed on the device and
 * its dumps are published (chx_stream_last_dump, statistics). */
int chx_stream_sync(chx_stream *s);
/* Synchronises the device and the published dumps, reads and clears the
 * device error word.  Returns CHX_OK or CHX_E_TIMEOUT. */
int chx_stream_check(chx_stream *s);
int chx_stream_destroy(chx_stream *s);

#ifdef __cplusplus
}
#endif

#endif /* CHIMEX_H */
