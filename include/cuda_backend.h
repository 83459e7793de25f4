/*
 * cuda_backend.h — CUDA reconstruction backend for compute-vp9 (B200,
 * sm_100a). Drop-in for the Vulkan backend: the eight entry points below
 * have the signatures and return-code contract of
 * src/backend/vulkan/vulkan_backend.h:141-163 and are called from the same
 * places in src/decoder/vp9_decoder.c (init 110-119, decode 203-207 and
 * 448-452, get 256-259, dmabuf 286-293, export 295-317, render target
 * 319-325, destroy 131-134).
 *
 * Contract (mirrors the Vulkan backend):
 *  - cuda_decode_frame copies everything it needs out of *pf before it
 *    returns (the caller reuses the parsed frame), enqueues the frame and
 *    returns CVP9_OK; CVP9_ERR_AGAIN when all CVP9_CUDA_INFLIGHT slots hold
 *    undelivered frames.
 *  - cuda_get_frame(wait=0) returns CVP9_ERR_AGAIN while the oldest frame is
 *    still on the GPU unless every slot is busy, in which case it blocks;
 *    wait=1 always blocks. CVP9_ERR_UNSUPPORTED when nothing is queued.
 *    Frames come back in submission order. Plane pointers point into
 *    backend-owned pinned memory and stay valid for the next two
 *    cuda_decode_frame calls (include/compute_vp9/decoder.h:100-104),
 *    however many frames the ring holds when the frame is delivered.
 *  - Errors found on the device (invalid block layout, an expired bounded
 *    wait) are reported by the cuda_get_frame call that delivers the frame:
 *    CVP9_ERR_INVALID_DATA or CVP9_ERR_GPU.
 *  - cuda_get_frame_dmabuf returns CVP9_ERR_UNSUPPORTED (no DMA-BUF export
 *    on a headless compute box). cuda_export_buffer_alloc returns a
 *    host-mapped pinned buffer (fd = -1, mapped = host pointer) that the GPU
 *    writes directly; cuda_set_render_target arms it as the one-shot NV12
 *    target of the next decode.
 *
 * Arithmetic: CVP9_CUDA_ARITH_REFCPU (default) reproduces the library's CPU
 * reconstruction (src/decoder/vp9_reconstruct.c) and reference-pool rules
 * (src/decoder/vp9_decoder.c:224-231) bit for bit; CVP9_CUDA_ARITH_SPEC runs
 * the shader arithmetic (integer butterflies with dequantisation, 8-tap MC
 * on all planes, shader intra rules) with the Vulkan pool rules
 * (refresh_frame_flags, ref_frame_idx); the shaders hold only the regular
 * 8-tap filter, so SPEC returns CVP9_ERR_UNSUPPORTED (from decode) for an
 * inter frame whose header asks for another filter. CVP9_CUDA_ARITH_FULL is
 * SPEC completed to the VP9 specification where the reference is a
 * skeleton: compound prediction, the smooth/sharp/bilinear filters, intra
 * prediction per transform block with the directional modes, ADST (and the
 * Walsh-Hadamard transform of lossless frames), the header's delta_q values,
 * and the VP9 loop filter; it returns CVP9_ERR_UNSUPPORTED for sizes that
 * are not multiples of 8, a SWITCHABLE filter on an inter frame (the parsed
 * block record has no per-block filter) and references of another size.
 * The environment variable CVP9_ARITH=refcpu|spec|full picks the profile for
 * cuda_backend_init; CVP9_CUDA_DEVICE picks the GPU.
 */
#ifndef CVP9_CUDA_BACKEND_H
#define CVP9_CUDA_BACKEND_H

#include "cvp9_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define CVP9_CUDA_INFLIGHT 3

typedef enum {
    CVP9_CUDA_ARITH_REFCPU = 0,
    CVP9_CUDA_ARITH_SPEC   = 1,
    CVP9_CUDA_ARITH_FULL   = 2,
} cvp9_cuda_arith_t;

typedef struct {
    int device;     /* CUDA ordinal; -1: $CVP9_CUDA_DEVICE or 0        */
    int arith;      /* cvp9_cuda_arith_t; -1: $CVP9_ARITH or REFCPU     */
    int autotune;   /* >= 0: time the kernel configurations on the first
                     * frames of each size and keep the fastest (unless
                     * $CVP9_AUTOTUNE=0); -1: fixed defaults              */
} cuda_backend_options_t;

/* ── Drop-in entry points (vulkan_backend.h:141-163) ────────────────────── */

cvp9_err_t cuda_backend_init(void **ctx);
void       cuda_backend_destroy(void *ctx);
cvp9_err_t cuda_decode_frame(void *ctx, const vp9_parsed_frame_t *pf, int64_t pts);
cvp9_err_t cuda_get_frame(void *ctx, cvp9_frame_info_t *info, int wait);
cvp9_err_t cuda_get_frame_dmabuf(void *ctx, cvp9_dmabuf_frame_t *out);
cvp9_err_t cuda_export_buffer_alloc(void *ctx, uint64_t size, cvp9_export_buffer_t *out);
void       cuda_export_buffer_free(void *ctx, cvp9_export_buffer_t *buf);
cvp9_err_t cuda_set_render_target(void *ctx, const cvp9_export_buffer_t *target);

/* ── Additions beside the drop-in set ───────────────────────────────────── */

/* init with explicit options (NULL = defaults above) */
cvp9_err_t cuda_backend_init_ex(void **ctx, const cuda_backend_options_t *opt);

/* Device timing of the most recently delivered frame: milliseconds from the
 * start of its input upload to the end of its output copy, and of the GPU
 * kernels alone. */
cvp9_err_t cuda_backend_last_timing(void *ctx, float *total_ms, float *kernels_ms);

/* Text of the last CUDA error seen by this context ("" if none). */
const char *cuda_backend_last_error(void *ctx);

/* Diagnostic, no counterpart in the reference: exercises the bounded
 * neighbour wait of the wavefront kernel. A 128x64 frame whose right
 * superblock holds an intra block is reconstructed with only that superblock
 * scheduled, so its wait for the left neighbour can never be satisfied; the
 * wait gives up after its iteration limit and the kernel returns. *status
 * receives the frame's CVP9_JOB_* word (CVP9_JOB_TIMEOUT set when the limit
 * worked), *ms the kernel's device time. Returns CVP9_OK when the launch
 * completed and the device stayed usable. Allocates and frees its own small
 * buffers on `device` (-1: $CVP9_CUDA_DEVICE or 0). */
cvp9_err_t cuda_backend_selftest_wait_limit(int device, uint32_t *status, float *ms);

/* ── Allocation-free reconstruction of one frame ────────────────────────── *
 * No counterpart in the reference. For callers that must not allocate GPU
 * memory while decoding — a media framework or inference server that owns
 * all device memory through its own pools, or a real-time thread where
 * cudaMalloc/cudaFree could stall on device-wide synchronisation. The caller
 * owns every buffer: pf->blocks and pf->coeffs are DEVICE pointers,
 * ref_planes[i] are device I420 frames (NULL = empty slot) of size
 * ref_width[i] x ref_height[i], out_i420 receives the frame
 * (W*H + 2*ceil(W/2)*ceil(H/2) bytes), status_dev (optional, device) receives
 * the CVP9_JOB_* status word. Work is enqueued on `stream` (a cudaStream_t,
 * NULL = legacy default stream); nothing is allocated or freed.
 * The kernels' scratch is a fixed ~200 KB __device__ array in the library:
 *  - frames above CVP9_NOALLOC_MAX_SB superblocks (7680x4320) are rejected
 *    with CVP9_ERR_INVALID_DATA and a message on stderr;
 *  - every GPU the library is used on keeps that array until process exit;
 *  - all calls share it, so calls that overlap on the GPU race: serialise
 *    them on one stream;
 *  - the first call on a device performs that device's one-time set-up,
 *    so make it before any stream capture. */
#define CVP9_NOALLOC_MAX_SB 8160
cvp9_err_t cuda_reconstruct_noalloc(const vp9_parsed_frame_t *pf,
                                    const uint8_t *const ref_planes[8],
                                    const uint32_t ref_width[8],
                                    const uint32_t ref_height[8],
                                    uint8_t *out_i420, int arith,
                                    uint32_t *status_dev, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CVP9_CUDA_BACKEND_H */
