/*
 * oracle_stream.c — per-stream decode harness around the oracle profiles.
 * TEST INFRASTRUCTURE ONLY.
 *
 * Pool rules:
 *   REFCPU — src/decoder/vp9_decoder.c:224-231: a key frame is copied into
 *            all 8 slots, any other frame into slot 0 only.
 *   SPEC, FULL — src/backend/vulkan/vulkan_backend.c:1312-1354: the slots set in
 *            refresh_frame_flags (0 means 0x01) take the new frame; here all
 *            three planes, where the Vulkan skeleton copies luma only.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>

struct oracle_stream {
    int            profile;
    oracle_frame_t slot[8];
};

oracle_stream_t *oracle_stream_create(int profile)
{
    oracle_stream_t *s = calloc(1, sizeof(*s));
    if (s) s->profile = profile;
    return s;
}

void oracle_stream_destroy(oracle_stream_t *s)
{
    if (!s) return;
    for (int i = 0; i < 8; i++) oracle_frame_free(&s->slot[i]);
    free(s);
}

static int copy_frame(oracle_frame_t *dst, const oracle_frame_t *src)
{
    oracle_frame_free(dst);
    *dst = *src;
    size_t ny = (size_t)src->stride_y * src->height;
    size_t nc = (size_t)src->stride_uv * ((src->height + 1) / 2);
    dst->y = malloc(ny ? ny : 1); dst->u = malloc(nc ? nc : 1); dst->v = malloc(nc ? nc : 1);
    if (!dst->y || !dst->u || !dst->v) { oracle_frame_free(dst); return 0; }
    memcpy(dst->y, src->y, ny); memcpy(dst->u, src->u, nc); memcpy(dst->v, src->v, nc);
    return 1;
}

int oracle_stream_decode(oracle_stream_t *s, const vp9_parsed_frame_t *pf, uint8_t *out_i420)
{
    if (!s || !pf) return 0;
    const oracle_frame_t *refs[8];
    for (int i = 0; i < 8; i++) refs[i] = s->slot[i].y ? &s->slot[i] : NULL;

    oracle_frame_t out = {0};
    int ok = s->profile == ORACLE_SPEC ? oracle_spec_reconstruct(pf, refs, &out)
           : s->profile == ORACLE_FULL ? oracle_full_reconstruct(pf, refs, &out)
                                       : oracle_refcpu_reconstruct(pf, refs, &out);
    if (!ok) return 0;

    if (out_i420) {
        size_t ny = (size_t)out.stride_y * out.height;
        size_t nc = (size_t)out.stride_uv * ((out.height + 1) / 2);
        memcpy(out_i420, out.y, ny);
        memcpy(out_i420 + ny, out.u, nc);
        memcpy(out_i420 + ny + nc, out.v, nc);
    }

    if (s->profile != ORACLE_REFCPU) {
        unsigned refresh = pf->hdr.refresh_frame_flags ? pf->hdr.refresh_frame_flags : 0x01u;
        for (int i = 0; i < 8; i++)
            if (refresh & (1u << i)) copy_frame(&s->slot[i], &out);
    } else if (pf->hdr.frame_type == VP9_FRAME_KEY) {
        for (int i = 0; i < 8; i++) copy_frame(&s->slot[i], &out);
    } else {
        copy_frame(&s->slot[0], &out);
    }
    oracle_frame_free(&out);
    return 1;
}
