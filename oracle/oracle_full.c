/*
 * oracle_full.c — scalar restatement of the FULL profile. TEST
 * INFRASTRUCTURE ONLY: the checker for the CUDA FULL profile.
 *
 * FULL is the shader profile (oracle_spec.c) completed to the VP9
 * specification where the reference is a skeleton:
 *   - inter: the frame header's filter (regular = the shader's table;
 *     smooth, sharp, bilinear = the VP9 tables, which the reference lacks)
 *     and compound prediction (ref_frame[1], mv[1]; the two 8-bit
 *     predictions averaged with rounding), which the parser emits
 *     (src/decoder/vp9_kf_tile.c:1160-1165) and the reference's recon drops;
 *   - intra: prediction per transform block in raster order, with the VP9
 *     edge rules (127 above / 129 left fills, above-right only for 4x4
 *     transforms inside their block, replication past the frame edge, left
 *     availability ending at tile columns) and all ten modes, including the
 *     directional D45..D63 the shader leaves as TODO
 *     (shaders/vp9_intra_pred.comp.glsl:102-105);
 *   - residual: dequantisation with the header's delta_q values and the
 *     32x32 halving, rows then columns, ADST on intra luma transforms below
 *     32x32 by the tile parser's mode -> type map (vp9_kf_tile.c:361-372,
 *     vp9_default_probs.h:1728), the Walsh-Hadamard transform when the frame
 *     is lossless;
 *   - the VP9 loop filter: 4-, 8- and 16-wide filters chosen per edge from
 *     the transform size, block and transform edges, skipped inner edges of
 *     skipped inter blocks, superblock order (all vertical edges of a
 *     superblock, then its horizontal edges), replacing the 4-tap skeleton
 *     (shaders/vp9_loopfilter.comp.glsl:42-89).
 * Integer arithmetic is 32-bit with wrap-around (built with -fwrapv), as in
 * the shader transforms. Limits of the parsed-frame boundary (the block
 * record keeps one MV and one mode per sub-8x8 block, no per-block filter
 * and no segment or loop-filter delta data): a sub-8x8 block predicts its
 * whole 8x8 with that MV or mode; every block filters at filter_level.
 * Frames must be multiples of 8 in both dimensions, references must have the
 * frame's size, and the header's filter must not be SWITCHABLE; otherwise
 * oracle_full_reconstruct returns 0 (the CUDA backend returns
 * CVP9_ERR_UNSUPPORTED).
 *
 * No VP9 conformance streams or decoder are present here, so this profile is
 * restated from the published algorithm and its parity is unpinned.
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

/* ── 1-D inverse ADSTs (32-bit wrap, Q14 rounding as the DCTs) ──────────── */

#define RS(x) (((x) + 8192) >> 14)
enum {
    C1 = 16364, C2 = 16305, C3 = 16207, C4 = 16069, C5 = 15893, C6 = 15679,
    C7 = 15426, C8 = 15137, C9 = 14811, C10 = 14449, C11 = 14053, C12 = 13623,
    C13 = 13160, C14 = 12665, C15 = 12140, C16 = 11585, C17 = 11003, C18 = 10394,
    C19 = 9760, C20 = 9102, C21 = 8423, C22 = 7723, C23 = 7005, C24 = 6270,
    C25 = 5520, C26 = 4756, C27 = 3981, C28 = 3196, C29 = 2404, C30 = 1606,
    C31 = 804
};
/* sin(k*pi/9) * 2/3 * sqrt(2) in Q14, the 4-point ADST multipliers */
enum { S1 = 5283, S2 = 9929, S3 = 13377, S4 = 15212 };

#define TXI int
#define TXN(name) name
#include "oracle_txfm_adst.inc"
#undef TXI
#undef TXN

static void itx1d(int n, int adst, const int *in, int *out)
{
    if (!adst) { oracle_idct1d(n, in, out); return; }
    if (n == 4) iadst4(in, out);
    else if (n == 8) iadst8(in, out);
    else iadst16(in, out);
}

/* 4x4 inverse Walsh-Hadamard of a lossless frame (quantiser step 4, undone
 * by the first shift), added without a final rounding shift. */
static void iwht4(const int32_t *in, int32_t *out)
{
    int t[16];
    for (int r = 0; r < 4; r++) {
        int a = in[r * 4 + 0] >> 2, c = in[r * 4 + 1] >> 2, d = in[r * 4 + 2] >> 2, b = in[r * 4 + 3] >> 2;
        a += c; d -= b;
        int e = (a - d) >> 1;
        b = e - b; c = e - c;
        a -= b; d += c;
        t[r * 4 + 0] = a; t[r * 4 + 1] = b; t[r * 4 + 2] = c; t[r * 4 + 3] = d;
    }
    for (int col = 0; col < 4; col++) {
        int a = t[0 * 4 + col], c = t[1 * 4 + col], d = t[2 * 4 + col], b = t[3 * 4 + col];
        a += c; d -= b;
        int e = (a - d) >> 1;
        b = e - b; c = e - c;
        a -= b; d += c;
        out[0 * 4 + col] = a; out[1 * 4 + col] = b; out[2 * 4 + col] = c; out[3 * 4 + col] = d;
    }
}

/* Residual of one n x n TX: dequantise (DC step at [0][0]; 32x32 values
 * halved toward zero), rows then columns (ADST where tx_type asks: 1 down
 * the columns, 2 along the rows, 3 both), final rounding shift 4/5/6/6. */
void oracle_full_itx2d(const int16_t *in, int32_t *out, int n, int tx_type, int lossless,
                       int q_dc, int q_ac)
{
    int32_t dq[1024];
    for (int i = 0; i < n * n; i++) {
        int v = (int)in[i] * (i == 0 ? q_dc : q_ac);
        dq[i] = n == 32 ? v / 2 : v;
    }
    if (lossless && n == 4) { iwht4(dq, out); return; }
    const int row_adst = tx_type == 2 || tx_type == 3, col_adst = tx_type == 1 || tx_type == 3;
    int buf[32][32], tmp[32], res[32];
    for (int r = 0; r < n; r++) {
        for (int c = 0; c < n; c++) tmp[c] = dq[r * n + c];
        itx1d(n, row_adst, tmp, res);
        for (int c = 0; c < n; c++) buf[r][c] = res[c];
    }
    const int sh = n == 4 ? 4 : (n == 8 ? 5 : 6);
    for (int c = 0; c < n; c++) {
        for (int r = 0; r < n; r++) tmp[r] = buf[r][c];
        itx1d(n, col_adst, tmp, res);
        for (int r = 0; r < n; r++) out[r * n + c] = (res[r] + (1 << (sh - 1))) >> sh;
    }
}

/* ── Prediction, loop filter and frame loop, 8-bit ────────────────────── */

#define PIX uint8_t
#define PIX_MAX 255
#define PIX_MID 128
#define LF_SH 0
#define COEF int16_t
#define RES_T int32_t
#define RESIDUAL(src, res, n, tx_type, lossless, q_dc, q_ac) \
    oracle_full_itx2d((src), (res), (n), (tx_type), (lossless), (q_dc), (q_ac))
#define FULL_PUBLIC(name) oracle_full_##name
#include "oracle_full_body.inc"

int oracle_full_reconstruct(const vp9_parsed_frame_t *pf, const oracle_frame_t *const pool[8],
                            oracle_frame_t *out)
{
    return full_reconstruct(pf, pf->coeffs, pool, out);
}
