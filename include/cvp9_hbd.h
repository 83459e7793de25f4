/*
 * cvp9_hbd.h — profile 2 (10-bit 4:2:0) reconstruction, many streams per
 * step. Added beside the 8-bit paths: the reference reads bit_depth from
 * the uncompressed header (src/decoder/vp9_bitstream.c:49-52) but its
 * parsed frame stores int16 coefficients (src/decoder/vp9_parsed_frame.h:45),
 * its quantiser tables are the 8-bit ones (src/decoder/vp9_dequant.h:12-60)
 * and it reconstructs into uint8 planes (src/decoder/vp9_reconstruct.c), so
 * it has no 10-bit path to replace. This one takes what a 10-bit parser
 * produces: the same header and block records (vp9_parsed_frame_t, with
 * hdr.bit_depth = 10) and the dequantised coefficients as int32 in the dense
 * layout of pf->coeffs (the 32x32 halving applied; a 10-bit stream's
 * dequantised values reach +-2^17, past int16).
 *
 * Arithmetic: the VP9 profile of the 8-bit FULL path (compound prediction,
 * every frame filter, per-TX intra with all ten modes and the VP9 edge
 * rules, DCT/ADST/WHT, the VP9 loop filter) at 10 bits — transforms in
 * 64-bit integers with 32-bit values between the row and column pass, both
 * 8-tap passes rounded and clipped to [0, 1023], missing intra edges 511
 * (above) and 513 (left), loop-filter thresholds and flatness tests scaled
 * by 4. No 10-bit VP9 conformance data exists here: parity is against the
 * scalar restatement in oracle/ only (unpinned).
 *
 * Frames: I420 with uint16 samples, luma W x H, chroma ceil(W/2) x
 * ceil(H/2); sizes multiples of 8; references of the frame's size; the
 * header's filter not SWITCHABLE (else CVP9_ERR_UNSUPPORTED). Reference
 * pool per stream on the device, slots refreshed by refresh_frame_flags
 * (0 means slot 0), as the 8-bit FULL path.
 *
 * Lifetime: host inputs are read while cvp9_hbd_submit runs (arrays in
 * page-locked memory until the step completes); with CVP9_HBD_DEVICE_INPUTS
 * the block records and coefficients are device pointers. Two steps are in
 * flight at most: a submit completes the step two before it first, so the
 * upload of one step, the kernels of the one before and the download of
 * the one before that overlap. cvp9_hbd_get_frame completes every step in
 * flight and returns the stream's latest frame; its planes stay valid until
 * the stream's second next step is submitted. An engine is used from one
 * thread at a time (as a reference decoder context is); separate engines
 * are independent.
 */
#ifndef CVP9_HBD_H
#define CVP9_HBD_H

#include "cvp9_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cvp9_hbd cvp9_hbd_t;

typedef struct {
    const vp9_parsed_frame_t *pf;   /* header and block records; pf->coeffs unused */
    const int32_t            *coeffs;   /* pf->num_coeffs dequantised coefficients */
} cvp9_hbd_frame_t;

typedef struct {
    uint32_t  width, height;
    uint32_t  stride_y, stride_uv;  /* in samples */
    uint16_t *plane_y, *plane_u, *plane_v;
    int64_t   pts;
} cvp9_hbd_frame_info_t;

enum {
    CVP9_HBD_DEVICE_INPUTS = 1u << 0,   /* pf->blocks and coeffs are device pointers   */
    CVP9_HBD_NO_OUTPUT     = 1u << 1,   /* frames stay on the device (references only) */
};

/* device < 0: $CVP9_CUDA_DEVICE or 0. */
int  cvp9_hbd_create(int device, cvp9_hbd_t **out);
void cvp9_hbd_destroy(cvp9_hbd_t *h);

/* A stream of width x height frames; returns its id (>= 0) or a cvp9_err_t. */
int  cvp9_hbd_open_stream(cvp9_hbd_t *h, uint32_t width, uint32_t height);
int  cvp9_hbd_close_stream(cvp9_hbd_t *h, int sid);

/* One frame of each of n distinct streams through one launch chain. */
int  cvp9_hbd_submit(cvp9_hbd_t *h, int n, const int *sids, const cvp9_hbd_frame_t *frames,
                     const int64_t *pts, unsigned flags);
/* The same with each frame's coefficients as (index, value) lists: the
 * nonzero dequantised coefficients, indices into the dense layout,
 * distinct. The engine zeroes the dense array on the device and scatters
 * the lists into it, so the frames are those of cvp9_hbd_submit; 8 bytes per
 * nonzero coefficient cross the bus instead of 4 per coefficient. frames[i]
 * .coeffs is not read. */
typedef struct {
    uint32_t        n;
    const uint32_t *pos;
    const int32_t  *val;
} cvp9_hbd_coeff_list_t;
int  cvp9_hbd_submit_sparse(cvp9_hbd_t *h, int n, const int *sids, const cvp9_hbd_frame_t *frames,
                            const cvp9_hbd_coeff_list_t *lists, const int64_t *pts, unsigned flags);
/* Wait for the last step; CVP9_OK, CVP9_ERR_INVALID_DATA (a frame's blocks
 * were outside the supported domain; that frame is not delivered) or
 * CVP9_ERR_GPU. */
int  cvp9_hbd_wait(cvp9_hbd_t *h);
/* The stream's most recent delivered frame (host planes). */
int  cvp9_hbd_get_frame(cvp9_hbd_t *h, int sid, cvp9_hbd_frame_info_t *info);
/* Device times of the last completed step in ms: upload, scan, recon,
 * loop filter, download (with steps in flight the spans overlap the
 * neighbouring steps'). */
int  cvp9_hbd_step_times(cvp9_hbd_t *h, float ms[5]);
/* Device time from timer_start (recorded behind all queued work) to
 * timer_stop (behind the last submitted step's download), in ms. */
int  cvp9_hbd_timer_start(cvp9_hbd_t *h);
int  cvp9_hbd_timer_stop(cvp9_hbd_t *h, float *ms);

#ifdef __cplusplus
}
#endif

#endif /* CVP9_HBD_H */
