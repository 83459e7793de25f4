/*
 * oracle_hbd.c — scalar restatement of the profile 2 (10-bit 4:2:0) path.
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine of
 * include/cvp9_hbd.h (k_hbd_recon, k_lf_full<uint16_t>).
 *
 * The FULL profile (oracle_full.c; the same prediction, loop-filter and
 * frame code, oracle_full_body.inc) on uint16 samples in [0, 1023]:
 *   - coefficients arrive dequantised as int32 (the 32x32 halving applied);
 *   - the 1-D inverse DCT / ADST / WHT run in 64-bit integers (the same
 *     butterflies as the 8-bit oracles, oracle_txfm_*.inc) and the row
 *     pass's outputs are kept as 32-bit values for the column pass, the way
 *     a 10-bit VP9 decoder keeps its transform coefficients in 32 bits;
 *   - both 8-tap passes round and clip to 10 bits; missing intra edges are
 *     511 above and 513 on the left, a DC with neither 512, a missing first
 *     reference predicts 512;
 *   - the loop filter's limits and flatness thresholds are scaled by 4 and
 *     its 4-tap filter clamps to [-512, 511] around 512.
 * No 10-bit VP9 decoder or conformance stream is present here, so this is
 * restated from the published algorithm and its parity is unpinned; the
 * 64-bit transforms are checked against the 32-bit ones on inputs where
 * neither overflows (tests/test_hbd_oracle.py).
 */
#include "oracle.h"
#include "oracle_vp9_common.h"
#include "../compute_vp9_b200/csrc/vp9_tables.h"

#include <stdlib.h>
#include <string.h>

static const int16_t k_dc_q[256] = CVP9_QTABLE_DC_INIT;
static const int16_t k_ac_q[256] = CVP9_QTABLE_AC_INIT;
static const int k_filters[4][16][8] = {
    CVP9_SUBPEL_REGULAR_INIT, CVP9_SUBPEL_SMOOTH_INIT, CVP9_SUBPEL_SHARP_INIT, CVP9_SUBPEL_BILINEAR_INIT
};
static const uint8_t k_tx_type[10] = CVP9_INTRA_TX_TYPE_INIT;

/* ── 64-bit 1-D inverse transforms ─────────────────────────────────────── */

#define RS(x) (((x) + 8192) >> 14)
enum {
    C1 = 16364, C2 = 16305, C3 = 16207, C4 = 16069, C5 = 15893, C6 = 15679,
    C7 = 15426, C8 = 15137, C9 = 14811, C10 = 14449, C11 = 14053, C12 = 13623,
    C13 = 13160, C14 = 12665, C15 = 12140, C16 = 11585, C17 = 11003, C18 = 10394,
    C19 = 9760, C20 = 9102, C21 = 8423, C22 = 7723, C23 = 7005, C24 = 6270,
    C25 = 5520, C26 = 4756, C27 = 3981, C28 = 3196, C29 = 2404, C30 = 1606,
    C31 = 804
};
enum { S1 = 5283, S2 = 9929, S3 = 13377, S4 = 15212 };

#define TXI int64_t
#define TXN(name) name##_64
#include "oracle_txfm_dct.inc"
#include "oracle_txfm_adst.inc"
#undef TXI
#undef TXN

/* One 1-D inverse of n points, in place semantics through out. */
void oracle_hbd_itx1d(int n, int adst, const int64_t *in, int64_t *out)
{
    int64_t tmp[32];
    memcpy(tmp, in, (size_t)n * sizeof(int64_t));
    if (adst && n == 4) iadst4_64(tmp, out);
    else if (adst && n == 8) iadst8_64(tmp, out);
    else if (adst && n == 16) iadst16_64(tmp, out);
    else if (n == 4) idct4_64(tmp, out);
    else if (n == 8) idct8_64(tmp, out);
    else if (n == 16) idct16_64(tmp, out);
    else idct32_64(tmp, out);
}

/* 4-point inverse Walsh-Hadamard of one row (rows: the quantiser step 4
 * undone first) or column. */
static void iwht4_64(int64_t *x, int rows)
{
    int64_t a = x[0], c = x[1], d = x[2], b = x[3];
    if (rows) { a >>= 2; c >>= 2; d >>= 2; b >>= 2; }
    a += c; d -= b;
    int64_t e = (a - d) >> 1;
    b = e - b; c = e - c;
    a -= b; d += c;
    x[0] = a; x[1] = b; x[2] = c; x[3] = d;
}

/* Residual of one n x n TX from dequantised coefficients: rows (ADST
 * along them when tx_type is 2 or 3), the row outputs kept as int32, then
 * columns (ADST when 1 or 3), final rounding shift 4/5/6/6; lossless 4x4:
 * the Walsh-Hadamard rows and columns, no final shift. */
void oracle_hbd_itx2d(const int32_t *in, int64_t *out, int n, int tx_type, int lossless)
{
    const int row_adst = tx_type == 2 || tx_type == 3, col_adst = tx_type == 1 || tx_type == 3;
    const int wht = lossless && n == 4;
    int32_t buf[32][32];
    int64_t v[32];
    for (int r = 0; r < n; r++) {
        for (int c = 0; c < n; c++) v[c] = in[r * n + c];
        if (wht) iwht4_64(v, 1);
        else oracle_hbd_itx1d(n, row_adst, v, v);
        for (int c = 0; c < n; c++) buf[r][c] = (int32_t)v[c];
    }
    const int sh = n == 4 ? 4 : (n == 8 ? 5 : 6);
    for (int c = 0; c < n; c++) {
        for (int r = 0; r < n; r++) v[r] = buf[r][c];
        if (wht) iwht4_64(v, 0);
        else oracle_hbd_itx1d(n, col_adst, v, v);
        for (int r = 0; r < n; r++) out[r * n + c] = wht ? v[r] : (v[r] + (1 << (sh - 1))) >> sh;
    }
}

/* ── Prediction, loop filter and frame loop, 10-bit ─────────────────────── */

#define PIX uint16_t
#define PIX_MAX 1023
#define PIX_MID 512
#define LF_SH 2
#define COEF int32_t
#define RES_T int64_t
#define RESIDUAL(src, res, n, tx_type, lossless, q_dc, q_ac) \
    ((void)(q_dc), (void)(q_ac), oracle_hbd_itx2d((src), (res), (n), (tx_type), (lossless)))
#define FULL_PUBLIC(name) oracle_hbd_##name
#include "oracle_full_body.inc"

int oracle_hbd_reconstruct(const vp9_parsed_frame_t *pf, const int32_t *coeffs,
                           const oracle_frame_t *const pool[8], oracle_frame_t *out)
{
    if (pf->hdr.bit_depth != 10) return 0;
    /* blocks the CUDA path rejects (CVP9_JOB_BAD_BLOCK): a transform larger
     * than the block (a sub-8x8 block counts as its 8x8) */
    for (uint32_t i = 0; i < pf->num_blocks; i++) {
        const vp9_macroblock_info_t *b = &pf->blocks[i];
        const int sub8 = b->width < 8 || b->height < 8;
        const int m = sub8 ? 8 : mini(b->width, b->height);
        if (b->tx_size > 3 || (4 << b->tx_size) > m) return 0;
    }
    return full_reconstruct(pf, coeffs, pool, out);
}

/* ── Stream: the reference pool of the FULL profile ─────────────────────── */

struct oracle_hbd_stream {
    oracle_frame_t slot[8];
};

oracle_hbd_stream_t *oracle_hbd_stream_create(void)
{
    return calloc(1, sizeof(oracle_hbd_stream_t));
}

void oracle_hbd_stream_destroy(oracle_hbd_stream_t *s)
{
    if (!s) return;
    for (int i = 0; i < 8; i++) oracle_frame_free(&s->slot[i]);
    free(s);
}

static size_t frame_samples(const oracle_frame_t *f, size_t *nc)
{
    *nc = (size_t)f->stride_uv * ((f->height + 1) / 2);
    return (size_t)f->stride_y * f->height;
}

static int copy_frame16(oracle_frame_t *dst, const oracle_frame_t *src)
{
    oracle_frame_free(dst);
    *dst = *src;
    size_t nc, ny = frame_samples(src, &nc);
    dst->y = malloc(ny ? 2 * ny : 1); dst->u = malloc(nc ? 2 * nc : 1); dst->v = malloc(nc ? 2 * nc : 1);
    if (!dst->y || !dst->u || !dst->v) { oracle_frame_free(dst); return 0; }
    memcpy(dst->y, src->y, 2 * ny); memcpy(dst->u, src->u, 2 * nc); memcpy(dst->v, src->v, 2 * nc);
    return 1;
}

int oracle_hbd_stream_decode(oracle_hbd_stream_t *s, const vp9_parsed_frame_t *pf, const int32_t *coeffs,
                             uint16_t *out_i420)
{
    if (!s || !pf) return 0;
    const oracle_frame_t *refs[8];
    for (int i = 0; i < 8; i++) refs[i] = s->slot[i].y ? &s->slot[i] : NULL;
    oracle_frame_t out = {0};
    if (!oracle_hbd_reconstruct(pf, coeffs, refs, &out)) return 0;
    if (out_i420) {
        size_t nc, ny = frame_samples(&out, &nc);
        memcpy(out_i420, out.y, 2 * ny);
        memcpy(out_i420 + ny, out.u, 2 * nc);
        memcpy(out_i420 + ny + nc, out.v, 2 * nc);
    }
    const unsigned refresh = pf->hdr.refresh_frame_flags ? pf->hdr.refresh_frame_flags : 0x01u;
    for (int i = 0; i < 8; i++)
        if (refresh & (1u << i)) copy_frame16(&s->slot[i], &out);
    oracle_frame_free(&out);
    return 1;
}
