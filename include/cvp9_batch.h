/*
 * cvp9_batch.h — multi-stream reconstruction engine (added beside the
 * drop-in backend; no counterpart in the reference, which decodes one
 * stream per context, src/decoder/vp9_decoder.c:21-46).
 *
 * One step reconstructs one frame of each listed stream through a single
 * launch chain (block scan, SB-diagonal wavefront recon across all streams,
 * loop filter + NV12), optionally replayed from a CUDA graph per shape
 * bucket. Every stream keeps its reference pool on the device. Streams are
 * admitted against an HBM budget. The arithmetic per stream is exactly the
 * per-stream backend's (include/cuda_backend.h): a frame decodes to the same
 * bytes alone or inside any batch.
 *
 * Lifetime rules:
 *  - host inputs: parsed frames are read during cvp9_batch_submit; arrays in
 *    page-locked memory (cudaHostAlloc / cudaHostRegister) are DMA'd directly
 *    and must stay unchanged until the step completes (cvp9_batch_wait or
 *    cvp9_batch_poll returning 1); other arrays are copied before submit
 *    returns.
 *  - CVP9_BATCH_DEVICE_INPUTS: pf->blocks and pf->coeffs are device pointers
 *    on the engine's GPU, read by the step's kernels.
 *  - outputs: a step's frames leave the device in one copy, into one of
 *    five page-locked output areas used in turn. cvp9_batch_get_frame returns
 *    planes of the stream's most recent frame, valid until the fifth step
 *    after the one that produced it is submitted; after that the call
 *    answers CVP9_ERR_INVALID_DATA. With CVP9_BATCH_NO_OUTPUT the frame stays
 *    on the device only (it still becomes the stream's reference).
 */
#ifndef CVP9_BATCH_H
#define CVP9_BATCH_H

#include "cvp9_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cvp9_batch cvp9_batch_t;

typedef struct {
    int      device;         /* CUDA ordinal; -1: $CVP9_CUDA_DEVICE or 0         */
    int      arith;          /* 0 REFCPU, 1 SPEC, 2 FULL; -1: $CVP9_ARITH or REFCPU */
    uint64_t hbm_budget;     /* bytes of stream state to admit; 0: 150 GB         */
    int      max_streams;    /* 0: 1024                                          */
    int      use_graphs;     /* replay the kernel chain from per-bucket graphs    */
    int      autotune;       /* choose the kernel configuration per shape bucket
                              * by timing its first steps ($CVP9_AUTOTUNE=0
                              * overrides); 0: fixed defaults                    */
    int      pack;           /* pack dense host coefficient arrays before the
                              * upload (cvp9_pack_coeffs). 0: steps that move at
                              * least 64 MB of them pack a share of their frames,
                              * raised while submits wait for the link and
                              * lowered while they do not; 1 always; -1 never
                              * ($CVP9_PACK=0|1 overrides)                       */
} cvp9_batch_config_t;

/* The tuner's record of one shape bucket (a step's arithmetic, frame count
 * and superblock count, each rounded up to a power of two). */
typedef struct {
    uint64_t key;
    int      frames;         /* frames per step when the bucket was opened       */
    int      settled;        /* 1: every knob measured, the fields below hold     */
    int      inter_path;     /* 0 general kernel only, 1 warp-per-SB inter kernel
                              * (96 registers), 2 the same at 80 registers,
                              * 3 prediction and residual as two kernels (64
                              * registers for the residual), 4 (REFCPU) the
                              * same with 8x8 TXs walked TX by TX                */
    int      lf_tile_h;      /* loop filter: 16 register strips (8x16 per thread),
                              * 32 shared-memory tiles (64x32 per CTA)           */
    int      half_width;     /* 1: wavefront kernel on half the resident CTAs    */
    int      trials;         /* configurations measured                          */
    float    best_ms;        /* kernel time of the best configuration            */
} cvp9_batch_tune_t;

enum {
    CVP9_BATCH_DEVICE_INPUTS = 1u << 0,
    CVP9_BATCH_NO_OUTPUT     = 1u << 1,
};

typedef struct {
    float    step_ms;        /* device time of the last completed step          */
    float    kernels_ms;     /* its scan + recon + filter kernels                */
    float    h2d_ms;         /* its input upload                                 */
    uint64_t h2d_bytes;      /* bytes uploaded by that step                      */
    uint64_t d2h_bytes;      /* bytes downloaded by that step                    */
    uint64_t reserved_bytes; /* HBM reserved by the open streams                 */
    int      open_streams;
    int      graph_replays;  /* steps launched from a cached graph (cumulative)  */
    uint32_t kernel_launches;/* kernels launched by that step                    */
    float    scan_ms;        /* per-kernel device times of that step             */
    float    recon_ms;
    float    filter_ms;
    uint32_t packed_frames;  /* frames of that step uploaded packed              */
    float    submit_pack_ms; /* host time the last submit spent packing          */
    float    submit_wait_ms; /* and waiting for a free step slot                 */
    float    submit_stage_ms;/* and copying inputs into the staging buffer       */
    uint64_t dev_held_bytes; /* device memory the engine holds from the driver   */
    uint64_t host_held_bytes;/* page-locked host memory it holds                 */
} cvp9_batch_stats_t;

cvp9_err_t  cvp9_batch_create(const cvp9_batch_config_t *cfg, cvp9_batch_t **out);
void        cvp9_batch_destroy(cvp9_batch_t *b);

/* HBM the engine reserves for one stream of this size (admission unit). */
uint64_t    cvp9_batch_stream_bytes(uint32_t width, uint32_t height);

/* Admit a stream: returns its id (>= 0), or CVP9_ERR_NOMEM when the HBM
 * budget or the stream limit would be exceeded (retry after a close). */
int         cvp9_batch_open_stream(cvp9_batch_t *b, uint32_t width, uint32_t height);

/* Take device and page-locked memory from the driver now for `nstreams`
 * streams of width x height (their frames, output areas and step buffers),
 * so that opening and decoding that many streams later allocates nothing
 * from the driver: pinning host memory costs about 0.4 ms per MB and
 * device allocations can wait for the device, both on a serving loop's
 * critical path. The step output areas and staging buffers are sized for a
 * step holding every reserved stream at once (steps in flight are waited
 * for first). Admission (the HBM budget) is unchanged. Calls add up. */
cvp9_err_t  cvp9_batch_reserve(cvp9_batch_t *b, uint32_t width, uint32_t height, int nstreams);
cvp9_err_t  cvp9_batch_close_stream(cvp9_batch_t *b, int sid);

/* Enqueue one step: frame pfs[i] for stream sids[i] (each stream at most
 * once). Returns once inputs are staged; up to three steps are in flight. */
cvp9_err_t  cvp9_batch_submit(cvp9_batch_t *b, int n, const int *sids,
                              const vp9_parsed_frame_t *const *pfs, const int64_t *pts,
                              uint32_t flags);

/* Sparse coefficients of one frame: the nonzero entries of the dense int16
 * coefficient array the parser would have written (same layout, same
 * indices), as parallel arrays. A parser that emits coefficients as it
 * decodes tokens can fill these instead of a mostly-zero dense array;
 * indices must be distinct. */
typedef struct {
    uint32_t        n;       /* nonzero coefficients                            */
    const uint32_t *pos;     /* index into the dense array (< num_coeffs)       */
    const int16_t  *val;     /* their values                                    */
} cvp9_coeff_list_t;

/* As cvp9_batch_submit, with coefficients given as lists[i] instead of
 * pfs[i]->coeffs (ignored; pfs[i]->num_coeffs still gives the dense size).
 * Only the lists cross the bus: the engine zeroes each frame's dense array
 * on the device and scatters the list into it, so every output byte is the
 * one the dense submit gives. Host inputs only (no CVP9_BATCH_DEVICE_INPUTS);
 * lists in page-locked memory are read after the call returns and must stay
 * unchanged until the step completes, like page-locked dense inputs.
 * No counterpart in the reference, whose parser writes the dense array. */
cvp9_err_t  cvp9_batch_submit_sparse(cvp9_batch_t *b, int n, const int *sids,
                                     const vp9_parsed_frame_t *const *pfs,
                                     const cvp9_coeff_list_t *lists, const int64_t *pts,
                                     uint32_t flags);

/* Coefficient packing. Dense coefficient arrays are mostly zeros, and a
 * large step's upload is bound by the PCIe link, so the engine packs the
 * coefficients the reconstruction reads on its host worker threads, uploads
 * the packed frames and rebuilds the dense arrays on the device. Exposed so
 * that the format can be checked on its own.
 *
 * A packed frame is 32-bit words: [0] P, the number of 65536-coefficient
 * pages (ceil(num_coeffs / 65536)); for page p, [1 + 2p] the first word of
 * its data (a multiple of 4; bit 31 set: dense page) and [2 + 2p] its count.
 * An entry page holds `count` words (offset in the page) | (value << 16) and
 * is zero everywhere else; a dense page holds its `count` coefficients as
 * int16, two per word. A page becomes dense when its entries would outgrow
 * the dense form. Coefficients read: SPEC every one; REFCPU each non-skip
 * block's luma TXs, [coeff_offset, + (cw/n)(ch/n) n^2) with the block
 * clipped to the frame (cw x ch) and n the TX size; the others come out as
 * zeros.
 *
 * cvp9_pack_bound_words: words that packing a frame may need.
 * cvp9_pack_coeffs: packs pf's coefficients into out, returns the words
 * used; -1 when cap_words is short, the arrays are missing, or (REFCPU) the
 * blocks' spans are not in ascending order (the engine then uploads that
 * frame's coefficients as it would without packing). */
size_t      cvp9_pack_bound_words(uint32_t num_coeffs);
int64_t     cvp9_pack_coeffs(int arith, const vp9_parsed_frame_t *pf, uint32_t *out, size_t cap_words);

/* Block (bounded) until every submitted step is complete. Returns the first
 * per-stream error of those steps (CVP9_ERR_INVALID_DATA for a rejected
 * block layout, CVP9_ERR_GPU for an expired device wait), else CVP9_OK. */
cvp9_err_t  cvp9_batch_wait(cvp9_batch_t *b);

/* 1 if every submitted step is complete, 0 if not, <0 on error. */
int         cvp9_batch_poll(cvp9_batch_t *b);

/* Latest completed frame of a stream (CVP9_ERR_AGAIN if its last step is
 * still running, CVP9_ERR_UNSUPPORTED if it has none on the host). */
cvp9_err_t  cvp9_batch_get_frame(cvp9_batch_t *b, int sid, cvp9_frame_info_t *info);

/* The frame stream `sid` got from step `seq` (a value of
 * cvp9_batch_last_seq after the submit that held it): AGAIN while that step
 * runs, INVALID_DATA if the stream was not in it, the step produced no
 * output for it, or its output area has since been given to a newer step
 * (five steps later). A stream may sit in several steps in flight at once;
 * this reads each of their frames in turn. */
cvp9_err_t  cvp9_batch_get_frame_at(cvp9_batch_t *b, int sid, uint64_t seq, cvp9_frame_info_t *info);

cvp9_err_t  cvp9_batch_stats(cvp9_batch_t *b, cvp9_batch_stats_t *st);

/* Device timer over whole steps: start records an event ahead of the next
 * step's upload; stop records one after the last submitted step's download,
 * waits for it (bounded) and returns the elapsed device milliseconds. */
cvp9_err_t  cvp9_batch_timer_start(cvp9_batch_t *b);
cvp9_err_t  cvp9_batch_timer_stop(cvp9_batch_t *b, float *ms);
const char *cvp9_batch_last_error(cvp9_batch_t *b);

/* Sequence number of the most recently submitted step (steps count from 1). */
uint64_t    cvp9_batch_last_seq(cvp9_batch_t *b);

/* Host-clock latency of step `seq`: from cvp9_batch_submit to its outputs
 * landing in host memory (CVP9_ERR_AGAIN while it runs; the most recent
 * 4096 steps are kept). */
cvp9_err_t  cvp9_batch_step_latency(cvp9_batch_t *b, uint64_t seq, double *ms);

/* Device timeline of a completed step `seq` (recent 4096 steps, after a
 * cvp9_batch_timer_start): milliseconds from the timer's start event to its
 * upload start, upload end, kernels start, kernels end and download end
 * (negative for events recorded before the start event). AGAIN while it
 * runs. Shows how consecutive steps overlap on the copy and compute
 * streams. */
cvp9_err_t  cvp9_batch_step_timeline(cvp9_batch_t *b, uint64_t seq, float t[5]);

/* Tuner buckets in use, and a copy of bucket i (0 <= i < count). */
int         cvp9_batch_tune_count(cvp9_batch_t *b);
cvp9_err_t  cvp9_batch_tune_entry(cvp9_batch_t *b, int i, cvp9_batch_tune_t *out);

#ifdef __cplusplus
}
#endif

#endif /* CVP9_BATCH_H */
