/*
 * oracle_refcpu.c — scalar restatement of the reference CPU reconstruction
 * (src/decoder/vp9_reconstruct.c). TEST INFRASTRUCTURE ONLY: the checker for
 * the CUDA REFCPU profile; never linked into the product.
 *
 * Must be built with -ffp-contract=off (no fused multiply-add), like the
 * reference's default x86-64 build, so every float64 product and sum rounds
 * separately in the same order.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

void oracle_frame_free(oracle_frame_t *f)
{
    if (!f) return;
    free(f->y); free(f->u); free(f->v);
    f->y = f->u = f->v = NULL;
}

/* vp9_frame.c:8-34: planes with stride = width, filled with 128. */
static int frame_alloc(oracle_frame_t *f, uint32_t w, uint32_t h)
{
    oracle_frame_free(f);
    f->width = w; f->height = h;
    f->stride_y = w;
    f->stride_uv = (w + 1) / 2;
    size_t ny = (size_t)w * h, nc = (size_t)f->stride_uv * ((h + 1) / 2);
    f->y = malloc(ny ? ny : 1);
    f->u = malloc(nc ? nc : 1);
    f->v = malloc(nc ? nc : 1);
    if (!f->y || !f->u || !f->v) { oracle_frame_free(f); return 0; }
    memset(f->y, 128, ny);
    memset(f->u, 128, nc);
    memset(f->v, 128, nc);
    return 1;
}

/* ── float64 inverse DCT (vp9_reconstruct.c:13-60) ─────────────────────── */

/* Basis M[i][j] = s_i * cos((2j+1) i pi / 2N), same expression and operand
 * order as the reference (:19-29), so libm gives identical doubles. */
static void dct_basis(double M[32][32], int n)
{
    double s0 = sqrt(1.0 / n);
    double s1 = sqrt(2.0 / n);
    for (int i = 0; i < n; i++) {
        double s = (i == 0) ? s0 : s1;
        for (int j = 0; j < n; j++)
            M[i][j] = s * cos(((2.0 * j + 1.0) * i * 3.141592653589793) / (2.0 * n));
    }
}

void oracle_refcpu_basis(double *out)
{
    double M[32][32];
    int base = 0;
    for (int n = 4; n <= 32; n *= 2) {
        dct_basis(M, n);
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) out[base + i * n + j] = M[i][j];
        base += n * n;
    }
}

void oracle_refcpu_idct2d(const int16_t *in, int16_t *out, int n)
{
    double M[32][32], T[32][32];
    dct_basis(M, n);
    /* T = M^T * X, k ascending (:31-40) */
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            double acc = 0.0;
            for (int k = 0; k < n; k++) acc += M[k][i] * in[k * n + j];
            T[i][j] = acc;
        }
    /* O = T * M, k ascending (:42-51); round half away from zero, saturate
     * to int16 (:53-59) */
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            double acc = 0.0;
            for (int k = 0; k < n; k++) acc += T[i][k] * M[k][j];
            int32_t r = (int32_t)(acc + (acc >= 0 ? 0.5 : -0.5));
            out[i * n + j] = (int16_t)clampi(r, -32768, 32767);
        }
}

/* ── Prediction (vp9_reconstruct.c:63-131) ─────────────────────────────── */

/* mode 0 DC, 1 V, 2 H, anything else TM (:63-91). */
static void predict_intra(uint8_t *dst, int stride, int w, int h,
                          const uint8_t *above, const uint8_t *left, int top_left, int mode)
{
    if (mode == 0) {
        uint32_t sum = 0;
        for (int i = 0; i < w; i++) sum += above[i];
        for (int i = 0; i < h; i++) sum += left[i];
        uint8_t dc = (uint8_t)((sum + (uint32_t)((w + h) >> 1)) / (uint32_t)(w + h));
        for (int r = 0; r < h; r++) memset(dst + (size_t)r * stride, dc, (size_t)w);
    } else if (mode == 1) {
        for (int r = 0; r < h; r++) memcpy(dst + (size_t)r * stride, above, (size_t)w);
    } else if (mode == 2) {
        for (int r = 0; r < h; r++) memset(dst + (size_t)r * stride, left[r], (size_t)w);
    } else {
        for (int r = 0; r < h; r++)
            for (int c = 0; c < w; c++)
                dst[(size_t)r * stride + c] = (uint8_t)clampi(above[c] + left[r] - top_left, 0, 255);
    }
}

/* Bilinear 1/8-pel MC with a per-sample clamp into [0,rw-1]x[0,rh-1]; two
 * rounded 3-bit stages, horizontal first (:94-131). */
static void predict_bilinear(uint8_t *dst, int dst_stride, const uint8_t *ref, int ref_stride,
                             int w, int h, int bx, int by, int mvx, int mvy, int rw, int rh)
{
    int px8 = bx * 8 + mvx, py8 = by * 8 + mvy;
    int ix = px8 >> 3, iy = py8 >> 3;
    int fx = px8 & 7, fy = py8 & 7;
    for (int r = 0; r < h; r++) {
        int y0 = clampi(iy + r, 0, rh - 1), y1 = clampi(iy + r + 1, 0, rh - 1);
        for (int c = 0; c < w; c++) {
            int x0 = clampi(ix + c, 0, rw - 1), x1 = clampi(ix + c + 1, 0, rw - 1);
            uint32_t a = ref[(size_t)y0 * ref_stride + x0], b = ref[(size_t)y0 * ref_stride + x1];
            uint32_t d = ref[(size_t)y1 * ref_stride + x0], e = ref[(size_t)y1 * ref_stride + x1];
            uint32_t top = (a * (uint32_t)(8 - fx) + b * (uint32_t)fx + 4) >> 3;
            uint32_t bot = (d * (uint32_t)(8 - fx) + e * (uint32_t)fx + 4) >> 3;
            dst[(size_t)r * dst_stride + c] = (uint8_t)((top * (uint32_t)(8 - fy) + bot * (uint32_t)fy + 4) >> 3);
        }
    }
}

/* Gather intra edges for one plane at (x, y) of size w x h: 127 where the
 * frame edge is reached; the corner is 127 unless both x > 0 and y > 0
 * (:200-245). */
static void gather_edges(const uint8_t *plane, int stride, int x, int y, int w, int h,
                         uint8_t *above, uint8_t *left, int *top_left)
{
    *top_left = 127;
    if (y > 0) {
        for (int i = 0; i < w; i++) above[i] = plane[(size_t)(y - 1) * stride + x + i];
        if (x > 0) *top_left = plane[(size_t)(y - 1) * stride + x - 1];
    } else {
        memset(above, 127, (size_t)w);
    }
    if (x > 0) {
        for (int i = 0; i < h; i++) left[i] = plane[(size_t)(y + i) * stride + x - 1];
    } else {
        memset(left, 127, (size_t)h);
    }
}

/* ── Loop filter (vp9_reconstruct.c:134-191 ≡ vp9_loopfilter.comp.glsl) ── */

static inline void filter4_at(uint8_t *p, size_t o1, size_t o0, size_t q0o, size_t q1o, int thr)
{
    int p1 = p[o1], p0 = p[o0], q0 = p[q0o], q1 = p[q1o];
    if (abs(p0 - q0) * 2 + abs(p1 - q1) / 2 > thr) return;
    int delta = clampi((3 * (q0 - p0) + 4) >> 3, -thr, thr);
    p[o0]  = (uint8_t)clampi(p0 + delta, 0, 255);
    p[q0o] = (uint8_t)clampi(q0 - delta, 0, 255);
    p[o1]  = (uint8_t)clampi(p1 + delta / 2, 0, 255);
    p[q1o] = (uint8_t)clampi(q1 - delta / 2, 0, 255);
}

void oracle_loopfilter(uint8_t *y, uint32_t w, uint32_t h, uint32_t stride,
                       int level, int sharpness, int profile)
{
    if (profile == ORACLE_REFCPU && level == 0) return;   /* :136 */
    int thr = level;
    if (sharpness > 0) {
        thr >>= (sharpness > 4) ? 2 : 1;
        if (thr > 9 - sharpness) thr = 9 - sharpness;
    }
    if (thr < 1) thr = 1;
    /* Horizontal edges first (rows 8, 16, ...), then vertical edges; each
     * filter touches rows/cols edge-2 .. edge+1. Accesses that would leave
     * the plane (heights/widths of 8k+1, where the reference reads past its
     * allocation) are skipped. */
    size_t plane_bytes = (size_t)stride * h;
    for (uint32_t e = 8; e < h; e += 8) {
        if (e + 1 >= h) continue;
        for (uint32_t x = 0; x < w; x++)
            filter4_at(y, (size_t)(e - 2) * stride + x, (size_t)(e - 1) * stride + x,
                       (size_t)e * stride + x, (size_t)(e + 1) * stride + x, thr);
    }
    for (uint32_t e = 8; e < w; e += 8) {
        for (uint32_t r = 0; r < h; r++) {
            size_t q1o = (size_t)r * stride + e + 1;
            if (q1o >= plane_bytes) continue;
            filter4_at(y, (size_t)r * stride + e - 2, (size_t)r * stride + e - 1,
                       (size_t)r * stride + e, q1o, thr);
        }
    }
}

/* ── Whole frame (vp9_reconstruct.c:194-370) ───────────────────────────── */

int oracle_refcpu_reconstruct(const vp9_parsed_frame_t *pf,
                              const oracle_frame_t *const refs[8],
                              oracle_frame_t *out)
{
    int W = (int)pf->hdr.width, H = (int)pf->hdr.height;
    if (!frame_alloc(out, (uint32_t)W, (uint32_t)H)) return 0;
    uint8_t above[4096], left[4096];
    int16_t res[1024];

    for (uint32_t bi = 0; bi < pf->num_blocks; bi++) {
        const vp9_macroblock_info_t *b = &pf->blocks[bi];
        int bx = b->x, by = b->y, bw = b->width, bh = b->height;
        if (bx + bw > W) bw = W - bx;
        if (by + bh > H) bh = H - by;
        if (bw <= 0 || bh <= 0) continue;

        int cbx = bx / 2, cby = by / 2, cbw = (bw + 1) / 2, cbh = (bh + 1) / 2;
        int ys = (int)out->stride_y, cs = (int)out->stride_uv;
        uint8_t *dy = out->y + (size_t)by * ys + bx;
        uint8_t *du = out->u + (size_t)cby * cs + cbx;
        uint8_t *dv = out->v + (size_t)cby * cs + cbx;

        if (b->is_intra) {
            int tl;
            gather_edges(out->y, ys, bx, by, bw, bh, above, left, &tl);
            predict_intra(dy, ys, bw, bh, above, left, tl, b->y_mode);
            gather_edges(out->u, cs, cbx, cby, cbw, cbh, above, left, &tl);
            predict_intra(du, cs, cbw, cbh, above, left, tl, b->uv_mode);
            gather_edges(out->v, cs, cbx, cby, cbw, cbh, above, left, &tl);
            predict_intra(dv, cs, cbw, cbh, above, left, tl, b->uv_mode);
        } else {
            /* ref_frame[0]-1 indexes the pool slot directly (:250-263) */
            int slot = b->ref_frame[0] - 1;
            const oracle_frame_t *ref = (slot >= 0 && slot < 8) ? refs[slot] : NULL;
            if (ref && ref->y) {
                predict_bilinear(dy, ys, ref->y, (int)ref->stride_y, bw, bh, bx, by,
                                 b->mv[0][0], b->mv[0][1], (int)ref->width, (int)ref->height);
            } else {
                for (int r = 0; r < bh; r++) memset(dy + (size_t)r * ys, 127, (size_t)bw);
            }
            if (ref && ref->u && ref->v) {
                /* chroma MV halves with C truncation; chroma extent is the
                 * floor half of the reference size (:313-327) */
                int cmx = b->mv[0][0] / 2, cmy = b->mv[0][1] / 2;
                int rw = (int)ref->width / 2, rh = (int)ref->height / 2;
                predict_bilinear(du, cs, ref->u, (int)ref->stride_uv, cbw, cbh, cbx, cby, cmx, cmy, rw, rh);
                predict_bilinear(dv, cs, ref->v, (int)ref->stride_uv, cbw, cbh, cbx, cby, cmx, cmy, rw, rh);
            } else {
                for (int r = 0; r < cbh; r++) {
                    memset(du + (size_t)r * cs, 127, (size_t)cbw);
                    memset(dv + (size_t)r * cs, 127, (size_t)cbw);
                }
            }
        }

        /* Luma residual only; TX count from the clamped size, so TXs that
         * straddle the frame edge are dropped and the coefficient stride
         * follows the clamped count (:336-363). */
        if (!b->skip) {
            if (b->tx_size > 3) continue;   /* larger sizes overrun the reference's buffers */
            int n = 1 << (b->tx_size + 2);
            int ntx = bw / n, nty = bh / n;
            for (int ty = 0; ty < nty; ty++)
                for (int tx = 0; tx < ntx; tx++) {
                    uint32_t off = b->coeff_offset + (uint32_t)((ty * ntx + tx) * n * n);
                    oracle_refcpu_idct2d(&pf->coeffs[off], res, n);
                    for (int r = 0; r < n; r++)
                        for (int c = 0; c < n; c++) {
                            uint8_t *p = out->y + (size_t)(by + ty * n + r) * ys + (bx + tx * n + c);
                            *p = (uint8_t)clampi((int)*p + res[r * n + c], 0, 255);
                        }
                }
        }
    }

    oracle_loopfilter(out->y, (uint32_t)W, (uint32_t)H, out->stride_y,
                      pf->hdr.filter_level, pf->hdr.sharpness_level, ORACLE_REFCPU);
    return 1;
}
