/*
 * ref_harness.c — drives the reference's own compiled CPU reconstruction
 * (vp9_reconstruct_frame from src/decoder/vp9_reconstruct.c, built from the
 * reference sources by oracle/Makefile into oracle/_ref/). TEST
 * INFRASTRUCTURE ONLY: it pins the restatement in oracle_refcpu.c and serves
 * as bench.py's "reference" CPU baseline.
 *
 * The reference-pool and output handling around the call restates
 * src/decoder/vp9_decoder.c:209-247 (that code sits inside cvp9_decode,
 * behind the bitstream parser, so it cannot be called on its own).
 */
#include "compute_vp9/decoder.h"
#include "vp9_parsed_frame.h"
#include "vp9_reconstruct.h"
#include "vp9_frame.h"

#include <stdlib.h>
#include <string.h>

typedef struct {
    cvp9_frame_info_t ref_frames[8];
} ref_stream_t;

void *ref_stream_create(void)
{
    return calloc(1, sizeof(ref_stream_t));
}

void ref_stream_destroy(void *p)
{
    ref_stream_t *s = (ref_stream_t *)p;
    if (!s) return;
    for (int i = 0; i < 8; i++) cvp9_frame_free(&s->ref_frames[i]);
    free(s);
}

/* One cvp9_decode worth of reconstruction: returns 1 on success and copies
 * the I420 frame into out_i420 (w*h + 2*cw*ch bytes) when non-NULL. */
int ref_stream_decode(void *p, const vp9_parsed_frame_t *pf, uint8_t *out_i420)
{
    ref_stream_t *s = (ref_stream_t *)p;
    cvp9_frame_info_t rec;
    memset(&rec, 0, sizeof(rec));
    const cvp9_frame_info_t *refs[8];
    for (int i = 0; i < 8; i++) refs[i] = &s->ref_frames[i];
    if (!vp9_reconstruct_frame(pf, refs, &rec)) return 0;

    if (out_i420) {
        size_t ny = (size_t)rec.stride_y * rec.height;
        size_t nc = (size_t)rec.stride_uv * ((rec.height + 1) / 2);
        memcpy(out_i420, rec.plane_y, ny);
        memcpy(out_i420 + ny, rec.plane_u, nc);
        memcpy(out_i420 + ny + nc, rec.plane_v, nc);
    }
    if (pf->hdr.frame_type == VP9_FRAME_KEY) {
        for (int i = 0; i < 8; i++) cvp9_frame_copy(&s->ref_frames[i], &rec);
    } else {
        cvp9_frame_copy(&s->ref_frames[0], &rec);
    }
    cvp9_frame_free(&rec);
    return 1;
}

/* Byte offsets of the boundary structs as the reference compiles them
 * (pins include/cvp9_types.h). Returns the number of values written. */
int ref_layout(uint32_t *out, int cap)
{
    uint32_t v[] = {
        (uint32_t)sizeof(vp9_frame_header_t),
        (uint32_t)offsetof(vp9_frame_header_t, width),
        (uint32_t)offsetof(vp9_frame_header_t, base_qindex),
        (uint32_t)offsetof(vp9_frame_header_t, filter_level),
        (uint32_t)offsetof(vp9_frame_header_t, sharpness_level),
        (uint32_t)offsetof(vp9_frame_header_t, refresh_frame_flags),
        (uint32_t)offsetof(vp9_frame_header_t, ref_frame_idx),
        (uint32_t)offsetof(vp9_frame_header_t, segmentation_enabled),
        (uint32_t)sizeof(vp9_macroblock_info_t),
        (uint32_t)offsetof(vp9_macroblock_info_t, tx_size),
        (uint32_t)offsetof(vp9_macroblock_info_t, mv),
        (uint32_t)offsetof(vp9_macroblock_info_t, skip),
        (uint32_t)offsetof(vp9_macroblock_info_t, coeff_offset),
        (uint32_t)offsetof(vp9_macroblock_info_t, eob),
        (uint32_t)sizeof(cvp9_mv_t),
        (uint32_t)sizeof(vp9_parsed_frame_t),
        (uint32_t)offsetof(vp9_parsed_frame_t, blocks),
        (uint32_t)offsetof(vp9_parsed_frame_t, num_blocks),
        (uint32_t)offsetof(vp9_parsed_frame_t, coeffs),
        (uint32_t)offsetof(vp9_parsed_frame_t, num_coeffs),
        (uint32_t)offsetof(vp9_parsed_frame_t, mv_grid),
        (uint32_t)offsetof(vp9_parsed_frame_t, mv_grid_width),
        (uint32_t)offsetof(vp9_parsed_frame_t, mi_block_grid),
        (uint32_t)sizeof(cvp9_frame_info_t),
        (uint32_t)offsetof(cvp9_frame_info_t, plane_y),
        (uint32_t)offsetof(cvp9_frame_info_t, pts),
        (uint32_t)sizeof(cvp9_export_buffer_t),
        (uint32_t)sizeof(cvp9_dmabuf_frame_t),
    };
    int n = (int)(sizeof(v) / sizeof(v[0]));
    for (int i = 0; i < n && i < cap; i++) out[i] = v[i];
    return n;
}
