/*
 * dropin_harness.c — the CUDA backend seen from the reference's side.
 *
 * Linked into the reference library built with the CUDA branch of
 * integration/vp9_decoder_cuda.patch (ENABLE_CUDA), this program decodes the
 * same packet stream twice through the reference's public API
 * (include/compute_vp9/decoder.h): once with CVP9_BACKEND_CPU (the
 * reference's own reconstruction) and once with CVP9_BACKEND_CUDA, and
 * compares every delivered frame byte for byte.
 *
 * Packets come from the reference's synthetic packet writer
 * (tests/vp9_synth.h: spec-conformant headers, zero-filled tile payloads),
 * a key frame every `gop` frames. The CUDA context is driven the way the
 * reference's VA-API entry point drives a GPU backend
 * (src/vaapi/vaapi_entrypoint.c:457-471): submit until cvp9_decode answers
 * CVP9_ERR_AGAIN, then take the oldest frame and submit again; a
 * non-blocking cvp9_get_frame is polled along the way.
 *
 *     dropin_harness WIDTH HEIGHT FRAMES GOP
 *
 * Prints one JSON line; exits 0 when the CUDA backend was active, every
 * frame matched, frames came back in submission order and back-pressure was
 * seen.
 */
#include "compute_vp9/decoder.h"
#include "vp9_synth.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static size_t frame_bytes(const cvp9_frame_info_t *f)
{
    return (size_t)f->width * f->height + 2 * (size_t)((f->width + 1) / 2) * ((f->height + 1) / 2);
}

/* Copy a delivered I420 frame into one contiguous buffer. */
static void take(const cvp9_frame_info_t *f, uint8_t *dst)
{
    const uint32_t cw = (f->width + 1) / 2, ch = (f->height + 1) / 2;
    for (uint32_t y = 0; y < f->height; y++) memcpy(dst + (size_t)y * f->width, f->plane_y + (size_t)y * f->stride_y, f->width);
    uint8_t *u = dst + (size_t)f->width * f->height, *v = u + (size_t)cw * ch;
    for (uint32_t y = 0; y < ch; y++) {
        memcpy(u + (size_t)y * cw, f->plane_u + (size_t)y * f->stride_uv, cw);
        memcpy(v + (size_t)y * cw, f->plane_v + (size_t)y * f->stride_uv, cw);
    }
}

int main(int argc, char **argv)
{
    if (argc < 5) {
        fprintf(stderr, "usage: %s WIDTH HEIGHT FRAMES GOP\n", argv[0]);
        return 2;
    }
    const uint32_t w = (uint32_t)atoi(argv[1]), h = (uint32_t)atoi(argv[2]);
    const int frames = atoi(argv[3]), gop = atoi(argv[4]) > 0 ? atoi(argv[4]) : frames;
    const size_t fb = (size_t)w * h + 2 * (size_t)((w + 1) / 2) * ((h + 1) / 2);
    uint8_t *pkt = malloc(vp9_synth_bufsize(w, h));
    uint8_t *want = malloc(fb * (size_t)frames), *got = malloc(fb);
    if (!pkt || !want || !got) return 2;

    cvp9_config_t cpu_cfg = { CVP9_BACKEND_CPU, 0, 0 }, gpu_cfg = { CVP9_BACKEND_CUDA, 0, 0 };
    cvp9_ctx_t *cpu = NULL, *gpu = NULL;
    if (cvp9_create(&cpu_cfg, &cpu) != CVP9_OK || cvp9_create(&gpu_cfg, &gpu) != CVP9_OK) return 2;
    const int cuda_active = cvp9_active_backend(gpu) == CVP9_BACKEND_CUDA;

    int mismatched = 0, compared = 0, again = 0, polled_again = 0, out_of_order = 0, errors = 0;
    int next_out = 0;

    /* deliver (and check) the CUDA context's oldest frame; wait=0 polls */
    #define DELIVER(wait_)                                                                  \
        do {                                                                                \
            cvp9_frame_info_t fi;                                                           \
            cvp9_err_t r_ = (wait_) ? cvp9_get_frame_sync(gpu, &fi) : cvp9_get_frame(gpu, &fi); \
            if (r_ == CVP9_ERR_AGAIN) { polled_again++; break; }                            \
            if (r_ != CVP9_OK) { errors++; break; }                                         \
            if (fi.pts != next_out) out_of_order++;                                         \
            if (frame_bytes(&fi) != fb) { errors++; next_out++; break; }                    \
            take(&fi, got);                                                                 \
            if (memcmp(got, want + fb * (size_t)fi.pts, fb) != 0) mismatched++;             \
            compared++;                                                                     \
            next_out++;                                                                     \
        } while (0)

    for (int f = 0; f < frames; f++) {
        size_t n = (f % gop == 0) ? vp9_synth_keyframe(pkt, w, h, 0) : vp9_synth_interframe(pkt, w, h, 0);
        /* the reference's CPU reconstruction of this packet */
        cvp9_frame_info_t ci;
        if (cvp9_decode(cpu, pkt, n, f) != CVP9_OK || cvp9_get_frame_sync(cpu, &ci) != CVP9_OK) { errors++; continue; }
        take(&ci, want + fb * (size_t)f);
        /* the CUDA backend, with back-pressure */
        cvp9_err_t rc = cvp9_decode(gpu, pkt, n, f);
        while (rc == CVP9_ERR_AGAIN) {
            again++;
            DELIVER(1);
            rc = cvp9_decode(gpu, pkt, n, f);
        }
        if (rc != CVP9_OK) { errors++; continue; }
        if (f % 3 == 2) DELIVER(0);        /* a non-blocking poll now and then */
    }
    for (;;) {
        cvp9_frame_info_t fi;
        cvp9_err_t r = cvp9_get_frame_sync(gpu, &fi);
        if (r == CVP9_ERR_UNSUPPORTED) break;                /* nothing queued */
        if (r != CVP9_OK) { errors++; break; }
        if (fi.pts != next_out) out_of_order++;
        take(&fi, got);
        if (memcmp(got, want + fb * (size_t)fi.pts, fb) != 0) mismatched++;
        compared++;
        next_out++;
    }
    cvp9_destroy(gpu);
    cvp9_destroy(cpu);
    const int ok = cuda_active && !errors && !mismatched && !out_of_order && compared == frames && again > 0;
    printf("{\"cuda_active\": %d, \"frames\": %d, \"compared\": %d, \"mismatched\": %d, \"again\": %d, "
           "\"polled_again\": %d, \"out_of_order\": %d, \"errors\": %d, \"ok\": %d}\n",
           cuda_active, frames, compared, mismatched, again, polled_again, out_of_order, errors, ok);
    free(pkt);
    free(want);
    free(got);
    return ok ? 0 : 1;
}
