/*
 * h261b.h -- native API of the B200 H.261 encode core (libh261b.so).
 *
 * Two ways in:
 *   1. the reference's own boundary, h261b_abi.h (sixteen gpu_device.h entry
 *      points, one process-global encoder, synchronous calls);
 *   2. this batched engine: many independent encode sessions of mixed size
 *      and QUANT share one device; each h261b_engine_step() encodes the next
 *      picture of every session that has one queued, in one launch over a
 *      flat macroblock work list.  Source pictures go up
 *      in one host-to-device copy per step, compact results come back in one
 *      copy, reconstructions stay in HBM as the next reference.  Steps
 *      alternate between two streams so that one step's copies overlap the
 *      neighbouring steps' kernels.
 *
 * All functions return H261B_OK (0) or a negative status; the text of the
 * last failure on the calling thread is available from h261b_last_error().
 * Nothing here takes or returns framework types: plain pointers and sizes.
 * An engine is used from one host thread at a time.
 */
#ifndef H261B_H
#define H261B_H

#include <stdint.h>
#include "h261b_abi.h"

#ifdef __cplusplus
extern "C" {
#endif

#define H261B_OK              0
#define H261B_ERR_ARG        -1   /* bad argument or unsupported size       */
#define H261B_ERR_CUDA       -2   /* CUDA runtime error (message has it)    */
#define H261B_ERR_NOMEM      -3   /* host or device allocation failed       */
#define H261B_ERR_BUDGET     -4   /* admission refused: HBM budget exceeded */
#define H261B_ERR_STATE      -5   /* call out of order                      */
#define H261B_ERR_NO_DEVICE  -6   /* no CUDA device / library not usable    */

#define H261B_ME_REFERENCE 0      /* the reference's two-stage search       */
#define H261B_ME_FULL      1      /* exhaustive +-15 (not bit-exact to it)  */

/* text of the last error on this thread ("" if none) */
const char *h261b_last_error(void);
/* last status recorded by a call of the reference-compatible boundary */
int h261b_abi_last_status(void);
/* library version string */
const char *h261b_version(void);

typedef struct h261b_engine_s h261b_engine_t;

typedef struct {
    int32_t device;           /* CUDA device ordinal                         */
    int32_t max_sessions;     /* session slots (<= 65536)                    */
    int64_t hbm_budget_bytes; /* admission limit for session pictures, 0 = none */
    int32_t me_mode;          /* H261B_ME_REFERENCE / H261B_ME_FULL          */
    int32_t fmad;             /* 1: fused double multiply-add in the DCTs
                                 (bit-exact to the reference built with nvcc
                                 defaults), 0: separately rounded            */
    int32_t warps_per_cta;    /* 1..8, 0 = tuned                              */
    int32_t max_ctas;         /* grid cap, 0 = one wave of resident CTAs     */
    int32_t copy_threads;     /* host threads copying batched submissions
                                 into the staging arena (the caller's thread
                                 included); 0 = min(8, cores / 2), 1 = none  */
    int32_t levels_to_host;   /* 1: copy every step's quantised levels back
                                 (h261b_frame_result_t.levels); 0: keep them
                                 on the device (sessions that write their
                                 bitstream on the device need no levels)    */
    int64_t bits_host_bytes;  /* initial size of each of the two host
                                 bitstream arenas, 0 = 8 MiB; grows when a
                                 step's pictures do not fit                 */
    int32_t use_graphs;       /* 1 (default): a step whose launches look like
                                 an earlier one's (sizes, arenas, launch
                                 shape) replays that step's CUDA graph      */
    /* Encode-kernel knobs.  0 (the default) leaves a knob to the tuner,
     * which tries the candidates on the engine's first mostly-inter steps
     * and keeps the fastest by CUDA-event time (per device, for the rest of
     * the process); the output never depends on them. */
    int32_t kernel_split;     /* 1: one kernel per step (search, mode
                                 decision and encode fused); 2: a search
                                 kernel (more warps per SM) and an encode
                                 kernel chained by a programmatic dependent
                                 launch                                      */
    int32_t tail_items;       /* n > 0: each warp takes all but n - 1 of its
                                 share of the work list in one static run and
                                 draws the rest one MB at a time            */
    int32_t staging;          /* 1: 16-byte cp.async copies of the search
                                 window; 2: one bulk copy per window row
                                 completed on a shared-memory barrier        */
    int32_t reserved;
} h261b_engine_config_t;

void h261b_engine_config_default(h261b_engine_config_t *cfg);
int h261b_engine_create(const h261b_engine_config_t *cfg, h261b_engine_t **out);
int h261b_engine_destroy(h261b_engine_t *e);

typedef struct {
    int32_t width, height;    /* multiples of 16, e.g. 176x144 or 352x288    */
    int32_t quant;            /* fixed picture QUANT 1..31                   */
    int32_t intra_period;     /* 0: only the first picture is intra          */
    int32_t denoise;          /* DCT-domain denoise strength (reference: 5)  */
    int32_t bitstream;        /* 1: write each picture's H.261 bitstream on
                                 the device (QCIF and CIF only), the bytes
                                 the reference's writers produce             */
    int32_t rate_control;     /* 0: fixed QUANT; 1: the reference's CBR rate
                                 control on the device (needs bitstream = 1;
                                 `quant` is its starting QUANT, the
                                 reference uses 10)                          */
    int32_t bitrate;          /* bit/s for rate_control = 1 (VBV = 1 s)      */
    int32_t psnr;             /* 1: measure each picture's PSNR (the
                                 reference's get_frame_psnr, h261_main.c:38-91)
                                 from squared errors summed on the device    */
} h261b_session_config_t;

/* Device bytes one session of this size holds (pictures + state), and the
 * bytes a session that writes its bitstream holds in addition (0 for a
 * size the H.261 syntax has no source format for). */
int64_t h261b_session_bytes(int32_t width, int32_t height);
int64_t h261b_session_bits_bytes(int32_t width, int32_t height);
/* all device bytes a session of this configuration holds (the admission
 * charge), or a negative status for an invalid configuration */
int64_t h261b_session_config_bytes(const h261b_session_config_t *cfg);

int h261b_session_open(h261b_engine_t *e, const h261b_session_config_t *cfg, int32_t *session_id);
int h261b_session_close(h261b_engine_t *e, int32_t session_id);
/* Allocate the device blocks of `count` sessions of this configuration
 * ahead of their opening (capacity planning for a server: opens then take
 * a block from the pool without allocating).  The blocks count against no
 * budget until a session holds them. */
int h261b_engine_reserve(h261b_engine_t *e, const h261b_session_config_t *cfg, int32_t count);
/* Size both step arenas (upload, results, descriptors) for `pictures`
 * pictures of this configuration in one step, on top of what earlier calls
 * reserved: steps up to that size never reallocate an arena. */
int h261b_engine_reserve_step(h261b_engine_t *e, const h261b_session_config_t *cfg, int32_t pictures);

/* Queue the session's next source picture (packed planes: Y stride W,
 * chroma stride W/2); the bytes are copied before the call returns.
 * quant > 0 replaces the session's QUANT from this picture on. */
int h261b_session_submit(h261b_engine_t *e, int32_t session_id, const uint8_t *y, const uint8_t *cb,
                         const uint8_t *cr, int32_t quant);

/* Queue the session's next picture by writing it in place: on return *y,
 * *cb and *cr point into the pinned staging arena (packed planes, strides
 * W and W/2); fill them before the next h261b_engine_step().  Saves the
 * copy h261b_session_submit makes. */
int h261b_session_input(h261b_engine_t *e, int32_t session_id, int32_t quant, uint8_t **y, uint8_t **cb,
                        uint8_t **cr);

/* h261b_session_input for n sessions in one call.  On return *staging is the
 * pinned arena the pictures go into and offsets[3i], [3i+1], [3i+2] the byte
 * offsets of session ids[i]'s Y, Cb and Cr planes in it.  quants may be NULL
 * (every session keeps its QUANT).  All or nothing: on an error no session
 * of the call is queued. */
int h261b_engine_inputs(h261b_engine_t *e, int32_t n, const int32_t *ids, const int32_t *quants,
                        uint8_t **staging, int64_t *offsets);

/* h261b_session_submit for n sessions in one call: session ids[i] gets the
 * picture y[i], cb[i], cr[i] (packed planes) and QUANT quants[i] (quants may
 * be NULL).  The pictures are copied into the staging arena by the engine's
 * copy threads before the call returns.  All or nothing, as
 * h261b_engine_inputs. */
int h261b_engine_submit_batch(h261b_engine_t *e, int32_t n, const int32_t *ids, const uint8_t *const *y,
                              const uint8_t *const *cb, const uint8_t *const *cr, const int32_t *quants);

/* h261b_engine_submit_batch that returns as soon as the copies have started:
 * the engine's copy threads move the pictures while the caller does other
 * work (reading the previous step, for one); the next h261b_engine_step()
 * waits for them.  The source planes must stay unchanged until that step
 * has been issued. */
int h261b_engine_submit_batch_async(h261b_engine_t *e, int32_t n, const int32_t *ids, const uint8_t *const *y,
                                    const uint8_t *const *cb, const uint8_t *const *cr, const int32_t *quants);

/* Queue a picture that is already in device memory (packed planes, pitch W
 * and W/2; Y 16-byte and Cb/Cr 8-byte aligned).  It must stay unchanged
 * until the step that reads it has completed. */
int h261b_session_submit_device(h261b_engine_t *e, int32_t session_id, const uint8_t *y, const uint8_t *cb,
                                const uint8_t *cr, int32_t quant);

/* h261b_session_submit_device for n sessions in one call: picture i of
 * session ids[i] at device planes y[i], cb[i], cr[i] with QUANT quants[i]
 * (quants may be NULL).  All or nothing: nothing is queued when any picture
 * is refused (a session named twice, not open or already queued, a NULL or
 * misaligned plane, QUANT above 31). */
int h261b_engine_submit_device_batch(h261b_engine_t *e, int32_t n, const int32_t *ids, const uint8_t *const *y,
                                     const uint8_t *const *cb, const uint8_t *const *cr, const int32_t *quants);

/* Encode the queued picture of every session that has one (one frame-step).
 * Returns the number of pictures encoded (>= 0) or a negative status.  The
 * call is asynchronous; results become readable after h261b_engine_sync(). */
int h261b_engine_step(h261b_engine_t *e);
/* Wait for the last step issued / for the one before it (so the host can
 * read step k's results while step k+1 runs).  A step's results stay
 * readable until the third step after it is issued. */
int h261b_engine_sync(h261b_engine_t *e);
int h261b_engine_wait_previous(h261b_engine_t *e);
/* Wait for step number `step` (steps are numbered 0, 1, ... in issue order)
 * to complete; its results are then the latest readable ones.  With two
 * steps issued ahead, a caller reads step k-2 while k-1 and k run.  Only
 * the steps still in flight (the last three issued) can be waited for. */
int h261b_engine_wait_step(h261b_engine_t *e, int64_t step);

/* per-macroblock result of a step (16 bytes) */
typedef struct {
    int16_t type;             /* 0 intra, 2 inter                             */
    int16_t flags;            /* 1 MC | 2 FILTER | 4 COEFF                    */
    int8_t quant;
    int8_t cbp;               /* bit 32>>b set when block b is coded          */
    int8_t mvx, mvy;
    int32_t cost;             /* mode-decision SATD cost                      */
    int32_t coef_bits;        /* bits of its blocks in the bitstream (TCOEFF,
                                 intra DC, EOB); 0 without a bitstream       */
} h261b_mb_result_t;

typedef struct {
    int32_t frame_index;      /* picture number within the session           */
    int32_t frame_type;       /* 0 intra, 1 inter                             */
    int32_t quant;            /* picture QUANT used                           */
    int32_t num_mb;
    const h261b_mb_result_t *mbs;  /* num_mb entries                          */
    const int8_t *levels;     /* num_mb x 6 x 64 quantised levels, each
                                 block column-major (index u * 8 + v for
                                 horizontal frequency u, vertical v); an
                                 intra DC is stored as uint8 1..255; NULL
                                 when levels_to_host is 0                    */
    const uint8_t *bits;      /* the picture's H.261 bytes (sessions with
                                 bitstream = 1), else NULL                   */
    int32_t bits_bytes;
    int32_t bits_status;      /* 0, or negative: the picture has no
                                 bitstream (H261B_ERR_STATE: a record the
                                 syntax cannot express)                      */
    uint64_t ssd[3];          /* psnr = 1: squared error of Y, Cb, Cr         */
    double psnr[3];           /* psnr = 1: 10 log10(255^2 N / ssd), 100 when
                                 ssd = 0, as the reference computes it       */
} h261b_frame_result_t;

/* Results of the latest completed step that encoded this session (pointers
 * stay valid until the third step after that one is issued). */
int h261b_session_result(h261b_engine_t *e, int32_t session_id, h261b_frame_result_t *out);

/* The macroblock records of the latest completed step as one array: the
 * records of every session the step encoded, session after session in
 * ascending session id (each session's h261b_session_result().mbs points
 * into it).  *step receives the step's number (0, 1, ...), -1 and *count 0
 * when no step has completed.  Valid until the third step after it is
 * issued. */
int h261b_engine_step_records(h261b_engine_t *e, const h261b_mb_result_t **records, int64_t *count,
                              int64_t *step);

/* Bitstream bytes and pictures the latest completed step wrote, over its
 * open sessions that write one. */
int h261b_engine_step_bits(h261b_engine_t *e, int64_t *bytes, int32_t *pictures);

/* one picture of a step's bitstream output */
typedef struct {
    int32_t session_id;
    int32_t frame_index;
    int32_t bytes;
    int32_t status;           /* 0: bits points into the host arena; 1: the
                                 arena was full, h261b_session_result() reads
                                 it from the device; < 0: no bitstream        */
    const uint8_t *bits;
} h261b_picture_t;

/* Every picture the latest completed step wrote as a bitstream, in
 * ascending session id: up to cap entries into out, *count = all of them.
 * *arena / *arena_bytes: the host arena holding them (each picture on a
 * 16-byte boundary) and the bytes of it in use, for callers that move a
 * step's output in one copy.  Valid until the third step after it is
 * issued. */
int h261b_engine_step_pictures(h261b_engine_t *e, int32_t cap, h261b_picture_t *out, int32_t *count,
                               const uint8_t **arena, int64_t *arena_bytes);

/* Copy the session's latest reconstruction (packed planes) to the host. */
int h261b_session_recon(h261b_engine_t *e, int32_t session_id, uint8_t *y, uint8_t *cb, uint8_t *cr);

/* Expand one result into the reference's h261_macroblock_t array (what the
 * reference's GOB / macroblock writers read); mbs[] gets num_mb entries. */
int h261b_result_to_abi(const h261b_frame_result_t *r, int32_t width, h261_macroblock_t *mbs);

/* Device timeline of the latest completed step (CUDA events on its
 * stream): uploads, waiting for the previous step's encode kernel, the
 * encode kernel, the bitstream kernels, and begin to end. */
typedef struct {
    int64_t step;
    float upload_ms, wait_ms, encode_ms, bitstream_ms, total_ms;
    float reserved;
} h261b_step_timing_t;
int h261b_engine_step_timing(h261b_engine_t *e, h261b_step_timing_t *t);

/* Steps captured as CUDA graphs and steps that replayed one. */
int h261b_engine_graph_stats(h261b_engine_t *e, int64_t *captures, int64_t *replays);
/* The launch shape of the encode kernel (warps per CTA, CTA cap; 0 = one
 * wave) and whether it came from tuning (1), from a tuning of an earlier
 * engine on the same device in this process (2) or from the configuration
 * (0). */
int h261b_engine_launch_shape(h261b_engine_t *e, int32_t *warps_per_cta, int32_t *max_ctas, int32_t *source);

/* Every knob of the encode kernel's launch, in h261b_engine_config_t's
 * encoding (kernel_split 1 fused / 2 search + encode, tail_items n + 1,
 * staging 1 cp.async / 2 bulk rows). */
typedef struct {
    int32_t warps_per_cta, max_ctas, kernel_split, tail_items, staging;
    int32_t source;           /* 0 configured, 1 tuned by this engine, 2 tuned
                                 earlier in this process on this device      */
    int32_t tuning;           /* 1 while this engine still tries candidates  */
    int32_t reserved;
} h261b_launch_plan_t;
/* The engine's launch plan, and the candidates its tuner measured so far
 * (each with its encode time in ms, in the order run; up to log_cap of them
 * into log / log_ms, the total in *log_count). */
int h261b_engine_plan(h261b_engine_t *e, h261b_launch_plan_t *plan, int32_t log_cap, h261b_launch_plan_t *log,
                      float *log_ms, int32_t *log_count);

/* Device time of the last step's encode kernel, and of its bitstream
 * kernel (0 without bitstream sessions), in milliseconds (CUDA events). */
int h261b_engine_last_kernel_ms(h261b_engine_t *e, float *ms);
int h261b_engine_last_bits_ms(h261b_engine_t *e, float *ms);
/* Bytes the last step copied host->device (descriptors, work list,
 * pictures) and device->host (records, picture records, levels when copied;
 * the bitstream bytes, which the device writes into mapped host memory,
 * are h261b_engine_step_bits()). */
int h261b_engine_last_copy_bytes(h261b_engine_t *e, int64_t *h2d, int64_t *d2h);
/* Throughput of the 4-pixel SAD primitive the motion search uses, measured
 * on the device with every SM busy: absolute differences per second. */
int h261b_measure_sad_peak(int32_t device, double *absdiff_per_s);
/* Bounds checks of the checking build (lib/libh261b_check.so, `make check`,
 * compiled with H261B_DEBUG_CHECKS): every global access of the encode
 * kernel whose address depends on a vector, a work item or a picture size,
 * and the motion compensation's window reads, test their index first and a
 * failing test is counted, its access skipped or clamped.  Reports whether
 * the loaded library checks (enabled), the failures since the last call
 * (then resets the count) and the first failure's site and index.  The
 * normal build reports enabled = 0 and no failures. */
int h261b_debug_check_status(int32_t *enabled, int64_t *violations, int32_t *first_site, int32_t *first_value);
/* Waits of the bulk-copy staging (staging = 2) that gave up on the current
 * device since the last call (then resets the count).  Every wait of the
 * encode kernel is bounded; a wait that gives up leaves that MB's window
 * incomplete, so a non-zero count means the step's output is wrong.  0 in
 * every correct run. */
int h261b_stage_status(int64_t *timeouts);

/* ---- one picture, no allocation ------------------------------------------
 * No counterpart in the reference: this entry point exists for callers that
 * cannot call cudaMalloc (their device memory belongs to another allocator
 * or pool, or an allocation is not allowed where they run).  The caller
 * passes every input, output and state buffer as device memory; the small
 * scratch the kernel needs (descriptor and work list) is a fixed static
 * device array inside the library, so the call allocates nothing.  Limits:
 * pictures of at most H261B_NOALLOC_MAX_MB macroblocks (larger ones are
 * refused with H261B_ERR_ARG); the first call on a device sets up the
 * scratch address and should come before any stream capture; calls whose
 * work overlaps on the GPU race on the shared scratch (use one stream). */
#define H261B_NOALLOC_MAX_MB      4096
#define H261B_NOALLOC_STATE_BYTES 1040   /* per-stream denoise state          */

typedef struct {
    int32_t width, height;    /* multiples of 16                              */
    int32_t frame_type;       /* H261B_FRAME_TYPE_INTRA / _INTER              */
    int32_t quant;            /* picture QUANT 1..31                          */
    int32_t me_mode;          /* H261B_ME_REFERENCE / H261B_ME_FULL           */
    int32_t fmad;             /* 1: the reference's default-build arithmetic  */
    int32_t denoise;          /* denoise strength; read only when reset_state
                                 is 1 (later calls keep the strength the
                                 stream started with and ignore this field) */
    int32_t reset_state;      /* 1: first picture of a stream, clear state    */
    const uint8_t *cur_y, *cur_cb, *cur_cr;  /* device: source, pitch W / W/2 */
    const uint8_t *ref_y, *ref_cb, *ref_cr;  /* device: previous reconstruction */
    uint8_t *rec_y, *rec_cb, *rec_cr;        /* device: reconstruction (out)  */
    void *state;              /* device: H261B_NOALLOC_STATE_BYTES, in/out     */
    h261b_mb_result_t *mbs;   /* device: num_mb results (out)                 */
    int8_t *levels;           /* device: num_mb x 384 levels (out)            */
} h261b_noalloc_picture_t;

/* Queue the encode of one picture on `stream` (a cudaStream_t, may be 0).
 * Luma planes, state and mbs 16-byte aligned; chroma planes and levels
 * 8-byte aligned. */
int h261b_encode_picture_noalloc(const h261b_noalloc_picture_t *pic, void *stream);

/* Number of sessions open / queued, device bytes held. */
int h261b_engine_stats(h261b_engine_t *e, int32_t *open_sessions, int32_t *queued, int64_t *device_bytes);

#ifdef __cplusplus
}
#endif
#endif
