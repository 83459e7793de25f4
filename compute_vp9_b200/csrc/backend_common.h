/*
 * backend_common.h — host helpers shared by the per-stream backend
 * (cuda_backend.c) and the multi-stream batch engine (batch.c).
 */
#ifndef CVP9_BACKEND_COMMON_H
#define CVP9_BACKEND_COMMON_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>
#include "recon_job.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Make `device` current and, once per device per process, upload the
 * float64 DCT basis and set the kernels' shared-memory limits. 0 on success. */
int cvp9_device_setup(int device);

/* Resident reconstruction CTAs per SM for the profile (after setup). */
int cvp9_recon_ctas_per_sm(int device, int arith);
/* The same for the VP9 loop filter kernel (superblock-row tickets). */
int  cvp9_lf_full_ctas_per_sm(int device);

/* The basis of the reference's float64 inverse DCT, N = 4, 8, 16, 32
 * concatenated (16 + 64 + 256 + 1024 doubles), built with the expression of
 * src/decoder/vp9_reconstruct.c:19-29 so libm produces the same doubles. */
void cvp9_build_dct_basis(double *out);

/* SB-diagonal ticket order: append the SBs of a sb_cols x sb_rows grid of
 * job `job` that lie on anti-diagonal d (row + col == d) to out. Returns
 * the number written. */
int cvp9_tickets_on_diagonal(int sb_cols, int sb_rows, int job, int d, uint32_t *out);

/* Quantiser steps for a qindex (vp9_dequant.h:67-75 with delta 0). */
int cvp9_dc_q(int qindex);
int cvp9_ac_q(int qindex);

/* Environment knobs: $CVP9_CUDA_DEVICE, $CVP9_ARITH (refcpu|spec|full),
 * $CVP9_INTER_FAST (warp-per-superblock inter path: 0 off, 1 the
 * 96-register kernel, 2 the 80-register kernel, 3 the two-kernel split,
 * k_pred + k_resid, 4 (REFCPU) the split with 8x8 TXs walked per TX,
 * 5 (REFCPU) path 4 with 8x8-only superblocks in a residual kernel of
 * their own; default 1). */
int cvp9_env_device(void);
int cvp9_env_arith(void);
int cvp9_env_inter_fast(void);
int cvp9_env_autotune(void);        /* $CVP9_AUTOTUNE: 0 turns tuning off */
int cvp9_env_recon_warp(void);      /* $CVP9_RECON_WARP: 0 keeps every k_recon level CTA-wide */
int cvp9_env_gather(void);          /* $CVP9_GATHER: 0 uploads whole coefficient arrays */
/* coefficient packing: -1 never, 0 large steps, 1 always ($CVP9_PACK=0|1
 * overrides the configured value) */
int cvp9_env_pack(int configured);

/* Whether the profile can reconstruct a frame with this header's
 * interpolation filter, as the frame's bitstream defines it. REFCPU: every
 * value (the CPU path, src/decoder/vp9_reconstruct.c:94-131, always
 * predicts bilinearly and never reads the field). SPEC: EIGHTTAP only (the
 * shaders hold the regular table alone, shaders/vp9_mc.comp.glsl:40-57).
 * On 0, *why names the reason for the caller's error text. */
int cvp9_filter_supported(int arith, int interp_filter, const char **why);

/* Whether the profile takes this frame: the filter rule above on inter
 * frames; FULL also wants both sizes multiples of 8 (its transform and
 * loop-filter edges then end inside the frame, as the MI grid does). */
int cvp9_frame_supported(int arith, const vp9_parsed_frame_t *pf, const char **why);

/* The FULL profile's fields of a job: per-plane quantiser steps with the
 * header's delta_q values, lossless, the frame's filter, the tile columns. */
void cvp9_job_full(cvp9_job_t *job, const vp9_parsed_frame_t *pf);

/* Fill the frame-geometry and parameter fields of a job from a parsed
 * frame (inputs, output, refs and scratch pointers are set by the caller). */
void cvp9_job_geometry(cvp9_job_t *job, const vp9_parsed_frame_t *pf);

/* Monotonic clock in seconds. */
double cvp9_now(void);

#ifdef __cplusplus
}
#endif

#endif /* CVP9_BACKEND_COMMON_H */

/* ── Autotuner ──────────────────────────────────────────────────────────────
 * Per shape bucket, the kernel configuration is chosen by timing: each
 * candidate runs on two steps of that bucket (the faster counts) and
 * replaces the best so far only if it is more than 2% faster; knobs are
 * settled one at a time (coordinate descent): the inter path, then the
 * loop-filter layout, then the wavefront width. Every configuration
 * produces the same bytes; only the speed differs. Pure host logic. */

#define CVP9_TUNE_BUCKETS 64

typedef struct {
    int8_t inter;      /* 0 general kernel only, 1 k_inter (96 registers), 2 k_inter (80),
                        * 3 k_pred + k_resid, 4 REFCPU: the same, 8x8 TXs walked per TX,
                        * 5 REFCPU: 4 with 8x8-only superblocks in their own residual kernel */
    int8_t lf32;       /* loop filter in 64x32 shared-memory tiles instead of
                        * 8x16 register strips */
    int8_t half;       /* wavefront kernel on half the resident CTAs */
} cvp9_tcfg_t;

typedef struct {
    uint64_t    key;
    int         frames;
    int         state;         /* 0 free, 1 measuring, 2 settled */
    int         stage, idx;    /* knob being settled, candidate within it */
    int         trials;        /* candidates measured */
    int         cur_n;         /* samples of the current candidate */
    cvp9_tcfg_t best, cur;
    float       best_ms, cur_ms;
    uint64_t    last_use;
} cvp9_tbucket_t;

typedef struct {
    cvp9_tbucket_t b[CVP9_TUNE_BUCKETS];
    int         arith;
    int         enabled;
    cvp9_tcfg_t fixed;         /* configuration when tuning is off */
    uint64_t    clock;
} cvp9_tuner_t;

void cvp9_tuner_init(cvp9_tuner_t *t, int arith, int enabled, cvp9_tcfg_t fixed);
/* Configuration for a step of bucket `key`; returns the bucket index whose
 * measurement this step feeds, or -1 (settled bucket or tuning off). */
int  cvp9_tuner_pick(cvp9_tuner_t *t, uint64_t key, int frames, cvp9_tcfg_t *cfg);
/* Kernel time of a completed step that ran `cfg` for bucket `idx`. */
void cvp9_tuner_report(cvp9_tuner_t *t, int idx, cvp9_tcfg_t cfg, float ms);
/* Coarse bucket of a step: arithmetic, frame count and superblock count,
 * each rounded up to a power of two, so serving steps share buckets. */
uint64_t cvp9_tune_key(int arith, int frames, uint64_t superblocks);

/* Share of a large step's frames the batch engine packs, in 16ths: one
 * more after a pipelined submit that waited over 0.05 ms for its step slot
 * (the link is behind), one fewer after one that did not (the host is);
 * unchanged when no step was in flight. Clamped to 0..16. */
int cvp9_pack_share_update(int q, int pipelined, double waited_ms);

/* Host worker threads. cvp9_parallel_for runs fn(ctx, k) for k in
 * [0, ntasks) on a pool of one thread per online CPU up to 16, the caller
 * included ($CVP9_HOST_THREADS overrides), taking tasks itself, and returns
 * when all are done; one job holds the pool at a time (a second caller runs
 * its tasks alone). */
int  cvp9_pool_threads(void);
void cvp9_parallel_for(int ntasks, void (*fn)(void *ctx, int task), void *ctx);

/* memcpy split across a pool of its own, 4 threads with the caller
 * ($CVP9_COPY_THREADS overrides); plain memcpy below 1 MB. The per-stream
 * backend stages the parser's arrays with it: one thread moves ~12 GB/s,
 * slower than the PCIe link. */
void cvp9_parallel_memcpy(void *dst, const void *src, size_t n);
