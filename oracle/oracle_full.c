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
#include "../compute_vp9_b200/csrc/vp9_tables.h"

#include <stdlib.h>
#include <string.h>

static const int16_t k_dc_q[256] = CVP9_QTABLE_DC_INIT;
static const int16_t k_ac_q[256] = CVP9_QTABLE_AC_INIT;
static const int k_filters[4][16][8] = {
    CVP9_SUBPEL_REGULAR_INIT, CVP9_SUBPEL_SMOOTH_INIT, CVP9_SUBPEL_SHARP_INIT, CVP9_SUBPEL_BILINEAR_INIT
};
static const uint8_t k_tx_type[10] = CVP9_INTRA_TX_TYPE_INIT;

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int mini(int a, int b) { return a < b ? a : b; }
static inline int absi(int v) { return v < 0 ? -v : v; }

typedef struct {
    uint8_t *p;
    int w, h, stride;
} plane_t;

static plane_t fplane(const oracle_frame_t *f, int idx)
{
    plane_t pl;
    if (idx == 0) { pl.p = f->y; pl.w = (int)f->width; pl.h = (int)f->height; pl.stride = (int)f->stride_y; }
    else {
        pl.p = idx == 1 ? f->u : f->v;
        pl.w = (int)(f->width + 1) / 2; pl.h = (int)(f->height + 1) / 2; pl.stride = (int)f->stride_uv;
    }
    return pl;
}

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

static void iadst4(const int *in, int *out)
{
    int x0 = in[0], x1 = in[1], x2 = in[2], x3 = in[3];
    int a = S1 * x0 + S4 * x2 + S2 * x3;
    int b = S2 * x0 - S1 * x2 - S4 * x3;
    int c = S3 * (x0 - x2 + x3);
    int d = S3 * x1;
    out[0] = RS(a + d);
    out[1] = RS(b + d);
    out[2] = RS(c);
    out[3] = RS(a + b - d);
}

/* butterfly pair: (x*ca + y*cb, x*cb - y*ca) */
#define ROT(x, y, ca, cb, o0, o1) do { o0 = (x) * (ca) + (y) * (cb); o1 = (x) * (cb) - (y) * (ca); } while (0)

static void iadst8(const int *in, int *out)
{
    int x0 = in[7], x1 = in[0], x2 = in[5], x3 = in[2], x4 = in[3], x5 = in[4], x6 = in[1], x7 = in[6];
    int s0, s1, s2, s3, s4, s5, s6, s7;
    ROT(x0, x1, C2, C30, s0, s1);
    ROT(x2, x3, C10, C22, s2, s3);
    ROT(x4, x5, C18, C14, s4, s5);
    ROT(x6, x7, C26, C6, s6, s7);
    x0 = RS(s0 + s4); x1 = RS(s1 + s5); x2 = RS(s2 + s6); x3 = RS(s3 + s7);
    x4 = RS(s0 - s4); x5 = RS(s1 - s5); x6 = RS(s2 - s6); x7 = RS(s3 - s7);
    s4 = C8 * x4 + C24 * x5;
    s5 = C24 * x4 - C8 * x5;
    s6 = -C24 * x6 + C8 * x7;
    s7 = C8 * x6 + C24 * x7;
    s0 = x0 + x2; s1 = x1 + x3; s2 = x0 - x2; s3 = x1 - x3;
    x4 = RS(s4 + s6); x5 = RS(s5 + s7); x6 = RS(s4 - s6); x7 = RS(s5 - s7);
    x2 = RS(C16 * (s2 + s3));
    x3 = RS(C16 * (s2 - s3));
    int y6 = RS(C16 * (x6 + x7)), y7 = RS(C16 * (x6 - x7));
    out[0] = s0; out[1] = -x4; out[2] = y6; out[3] = -x2;
    out[4] = x3; out[5] = -y7; out[6] = x5; out[7] = -s1;
}

static void iadst16(const int *in, int *out)
{
    int x[16], s[16];
    static const int perm[16] = { 15, 0, 13, 2, 11, 4, 9, 6, 7, 8, 5, 10, 3, 12, 1, 14 };
    for (int i = 0; i < 16; i++) x[i] = in[perm[i]];
    /* stage 1: eight rotations by odd multiples of pi/64 */
    static const int ca[8] = { C1, C5, C9, C13, C17, C21, C25, C29 };
    static const int cb[8] = { C31, C27, C23, C19, C15, C11, C7, C3 };
    for (int k = 0; k < 8; k++) ROT(x[2 * k], x[2 * k + 1], ca[k], cb[k], s[2 * k], s[2 * k + 1]);
    for (int k = 0; k < 8; k++) {
        x[k] = RS(s[k] + s[k + 8]);
        x[k + 8] = RS(s[k] - s[k + 8]);
    }
    /* stage 2 */
    for (int k = 0; k < 8; k++) s[k] = x[k];
    s[8] = x[8] * C4 + x[9] * C28;
    s[9] = x[8] * C28 - x[9] * C4;
    s[10] = x[10] * C20 + x[11] * C12;
    s[11] = x[10] * C12 - x[11] * C20;
    s[12] = -x[12] * C28 + x[13] * C4;
    s[13] = x[12] * C4 + x[13] * C28;
    s[14] = -x[14] * C12 + x[15] * C20;
    s[15] = x[14] * C20 + x[15] * C12;
    for (int k = 0; k < 4; k++) {
        x[k] = s[k] + s[k + 4];
        x[k + 4] = s[k] - s[k + 4];
        x[k + 8] = RS(s[k + 8] + s[k + 12]);
        x[k + 12] = RS(s[k + 8] - s[k + 12]);
    }
    /* stage 3 */
    for (int g = 0; g < 16; g += 8) {
        s[g + 0] = x[g + 0];
        s[g + 1] = x[g + 1];
        s[g + 2] = x[g + 2];
        s[g + 3] = x[g + 3];
        s[g + 4] = x[g + 4] * C8 + x[g + 5] * C24;
        s[g + 5] = x[g + 4] * C24 - x[g + 5] * C8;
        s[g + 6] = -x[g + 6] * C24 + x[g + 7] * C8;
        s[g + 7] = x[g + 6] * C8 + x[g + 7] * C24;
        x[g + 0] = s[g + 0] + s[g + 2];
        x[g + 1] = s[g + 1] + s[g + 3];
        x[g + 2] = s[g + 0] - s[g + 2];
        x[g + 3] = s[g + 1] - s[g + 3];
        x[g + 4] = RS(s[g + 4] + s[g + 6]);
        x[g + 5] = RS(s[g + 5] + s[g + 7]);
        x[g + 6] = RS(s[g + 4] - s[g + 6]);
        x[g + 7] = RS(s[g + 5] - s[g + 7]);
    }
    /* stage 4 */
    int t2 = RS(-C16 * (x[2] + x[3])), t3 = RS(C16 * (x[2] - x[3]));
    int t6 = RS(C16 * (x[6] + x[7])), t7 = RS(C16 * (-x[6] + x[7]));
    int t10 = RS(C16 * (x[10] + x[11])), t11 = RS(C16 * (-x[10] + x[11]));
    int t14 = RS(-C16 * (x[14] + x[15])), t15 = RS(C16 * (x[14] - x[15]));
    out[0] = x[0];   out[1] = -x[8];  out[2] = x[12];  out[3] = -x[4];
    out[4] = t6;     out[5] = t14;    out[6] = t10;    out[7] = t2;
    out[8] = t3;     out[9] = t11;    out[10] = t15;   out[11] = t7;
    out[12] = x[5];  out[13] = -x[13]; out[14] = x[9]; out[15] = -x[1];
}

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

/* ── Intra prediction of one transform block ───────────────────────────── */

#define AVG2(a, b) (((a) + (b) + 1) >> 1)
#define AVG3(a, b, c) (((a) + 2 * (b) + (c) + 2) >> 2)

/* Predict the n x n TX at (x0, y0) of plane pl in place. have_top/left:
 * neighbours available; have_right: the above-right n samples may be read
 * (4x4 TXs not in the last TX column of their block). Above samples past
 * the plane's right edge repeat the last one inside; left samples past the
 * bottom edge repeat the last one inside. */
void oracle_full_intra_tx(uint8_t *plane, int pw, int ph, int stride, int x0, int y0, int n,
                          int mode, int have_top, int have_left, int have_right)
{
    uint8_t abuf[65], left[32];
    uint8_t *above = abuf + 1;
    if (have_top) {
        const uint8_t *ar = plane + (size_t)(y0 - 1) * stride;
        int want = n + ((n == 4 && have_right) ? 4 : 0);
        int cnt = mini(want, pw - x0);
        for (int i = 0; i < 2 * n; i++) above[i] = ar[x0 + (i < cnt ? i : cnt - 1)];
        above[-1] = have_left ? ar[x0 - 1] : 129;
    } else {
        memset(abuf, 127, (size_t)(2 * n + 1));
    }
    if (have_left) {
        for (int i = 0; i < n; i++) left[i] = plane[(size_t)(y0 + mini(i, ph - 1 - y0)) * stride + x0 - 1];
    } else {
        memset(left, 129, (size_t)n);
    }
    int dc = 128;
    if (mode == 0) {
        int sa = 0, sl = 0;
        for (int i = 0; i < n; i++) { sa += above[i]; sl += left[i]; }
        if (have_top && have_left) dc = (sa + sl + n) / (2 * n);
        else if (have_top) dc = (sa + n / 2) / n;
        else if (have_left) dc = (sl + n / 2) / n;
    }
    for (int r = 0; r < n; r++)
        for (int c = 0; c < n; c++) {
            int v;
            switch (mode) {
            case 1: v = above[c]; break;                                    /* V    */
            case 2: v = left[r]; break;                                     /* H    */
            case 3: {                                                       /* D45  */
                int k = r + c;
                v = k + 2 < 2 * n ? AVG3(above[k], above[k + 1], above[k + 2]) : above[2 * n - 1];
                break;
            }
            case 4: {                                                       /* D135 */
                /* edge from the bottom of the left column over the corner
                 * to the end of the above row: e(t), t = c - r */
                int t = c - r;
#define EDGE(u) ((u) >= 0 ? above[(u)] : ((u) == -1 ? above[-1] : left[-(u) - 2]))
                v = AVG3(EDGE(t - 2), EDGE(t - 1), EDGE(t));
                break;
            }
            case 5:                                                         /* D117 */
                if (r == 0) v = AVG2(above[c - 1], above[c]);
                else if (r == 1) v = c == 0 ? AVG3(left[0], above[-1], above[0])
                                            : AVG3(above[c - 2], above[c - 1], above[c]);
                else if (c == 0) v = r == 2 ? AVG3(above[-1], left[0], left[1])
                                            : AVG3(left[r - 3], left[r - 2], left[r - 1]);
                else {
                    /* two rows up, one column left, until row 0 or 1 or column 0 */
                    int rr = r, cc = c;
                    while (rr >= 2 && cc >= 1) { rr -= 2; cc -= 1; }
                    if (rr == 0) v = AVG2(above[cc - 1], above[cc]);
                    else if (rr == 1) v = cc == 0 ? AVG3(left[0], above[-1], above[0])
                                                  : AVG3(above[cc - 2], above[cc - 1], above[cc]);
                    else v = rr == 2 ? AVG3(above[-1], left[0], left[1])
                                     : AVG3(left[rr - 3], left[rr - 2], left[rr - 1]);
                }
                break;
            case 6: {                                                       /* D153 */
                int rr = r, cc = c;
                while (rr >= 1 && cc >= 2) { rr -= 1; cc -= 2; }
                if (cc == 0) v = rr == 0 ? AVG2(above[-1], left[0]) : AVG2(left[rr - 1], left[rr]);
                else if (cc == 1) v = rr == 0 ? AVG3(left[0], above[-1], above[0])
                                             : rr == 1 ? AVG3(above[-1], left[0], left[1])
                                                       : AVG3(left[rr - 2], left[rr - 1], left[rr]);
                else v = AVG3(above[cc - 3], above[cc - 2], above[cc - 1]);   /* row 0 */
                break;
            }
            case 7: {                                                       /* D207 */
                int k = r + (c >> 1);
#define LFT(i) left[(i) < n ? (i) : n - 1]
                v = (c & 1) ? AVG3(LFT(k), LFT(k + 1), LFT(k + 2)) : AVG2(LFT(k), LFT(k + 1));
                break;
            }
            case 8: {                                                       /* D63  */
                int k = (r >> 1) + c;
                v = (r & 1) ? AVG3(above[k], above[k + 1], above[k + 2]) : AVG2(above[k], above[k + 1]);
                break;
            }
            case 9: v = clampi(left[r] + above[c] - above[-1], 0, 255); break;   /* TM */
            default: v = dc; break;                                         /* DC   */
            }
            int X = x0 + c, Y = y0 + r;
            if (X < pw && Y < ph) plane[(size_t)Y * stride + X] = (uint8_t)v;
        }
#undef EDGE
#undef LFT
}

/* ── Inter prediction ──────────────────────────────────────────────────── */

static int interp(plane_t ref, const int (*f)[8], int bx, int by, int fx, int fy)
{
#define FETCH(xx, yy) ((int)ref.p[(size_t)clampi((yy), 0, ref.h - 1) * ref.stride + clampi((xx), 0, ref.w - 1)])
    if (fx == 0 && fy == 0) return FETCH(bx, by);
    int rows[8];
    for (int r = 0; r < 8; r++) {
        int acc = 0;
        for (int t = 0; t < 8; t++) acc += f[fx][t] * FETCH(bx + t - 3, by + r - 3);
        rows[r] = clampi((acc + 64) >> 7, 0, 255);
    }
    int acc = 0;
    for (int t = 0; t < 8; t++) acc += f[fy][t] * rows[t];
    return clampi((acc + 64) >> 7, 0, 255);
#undef FETCH
}

/* One prediction of a region; avg: round-average into what is there (the
 * second prediction of a compound block). */
static void inter_region(plane_t dst, plane_t ref, const int (*f)[8], int x, int y, int w, int h,
                         int mvx, int mvy, int chroma, int avg)
{
    for (int r = 0; r < h; r++)
        for (int c = 0; c < w; c++) {
            int px = x + c, py = y + r, v;
            if (!chroma) v = interp(ref, f, px + (mvx >> 3), py + (mvy >> 3), (mvx & 7) << 1, (mvy & 7) << 1);
            else v = interp(ref, f, px + (mvx >> 4), py + (mvy >> 4), mvx & 15, mvy & 15);
            uint8_t *d = dst.p + (size_t)py * dst.stride + px;
            *d = (uint8_t)(avg ? (*d + v + 1) >> 1 : v);
        }
}

/* Stage entry point: one block's prediction from ref0 (and, when compound,
 * averaged with the prediction from ref1), filter = interp_filter 0..3. */
void oracle_full_mc_block(const uint8_t *ref0, const uint8_t *ref1, int rw, int rh, int rstride,
                          uint8_t *dst, int dw, int dh, int dstride, int x, int y, int bw, int bh,
                          int mv0x, int mv0y, int mv1x, int mv1y, int compound, int filter, int chroma)
{
    plane_t d = { dst, dw, dh, dstride };
    plane_t r0 = { (uint8_t *)ref0, rw, rh, rstride }, r1 = { (uint8_t *)ref1, rw, rh, rstride };
    inter_region(d, r0, k_filters[filter & 3], x, y, bw, bh, mv0x, mv0y, chroma, 0);
    if (compound) inter_region(d, r1, k_filters[filter & 3], x, y, bw, bh, mv1x, mv1y, chroma, 1);
}

static int max_tx_for(int w, int h)
{
    int m = w < h ? w : h;
    return m >= 32 ? 3 : (m >= 16 ? 2 : (m >= 8 ? 1 : 0));
}

/* First MI column of the tile column holding mi_col. */
static int tile_start(int mi_col, int mi_cols, int log2_tile_cols)
{
    int sb_cols = (mi_cols + 7) >> 3, start = 0;
    for (int t = 1; t < (1 << log2_tile_cols); t++) {
        int o = ((t * sb_cols) >> log2_tile_cols) << 3;
        if (o > mi_cols) o = mi_cols;
        if (o <= mi_col) start = o;
    }
    return start;
}

/* Plane TX layout of a block (the tile parser's, vp9_kf_tile.c:320-396). */
typedef struct { int tx, n, nx4, ny4, pbw, pbh, px0, py0; } ptx_t;

static ptx_t plane_tx(const vp9_macroblock_info_t *b, int plane, int mi_cols, int mi_rows)
{
    ptx_t t;
    int ss = plane > 0;
    int sub8 = b->width < 8 || b->height < 8;
    int ew = sub8 ? 8 : b->width, eh = sub8 ? 8 : b->height;
    int pw = ss ? ew / 2 : ew, ph = ss ? eh / 2 : eh;
    if (pw < 4) pw = 4;
    if (ph < 4) ph = 4;
    int tx = b->tx_size;
    if (ss) { int mt = max_tx_for(pw, ph); tx = sub8 ? 0 : (tx > mt ? mt : tx); }
    int mi_col = b->x >> 3, mi_row = b->y >> 3;
    int o4x = (mi_col * 2) >> ss, o4y = (mi_row * 2) >> ss;
    int mw = pw / 4, mh = ph / 4;
    if (o4x + mw > ((mi_cols * 2) >> ss)) mw = ((mi_cols * 2) >> ss) - o4x;
    if (o4y + mh > ((mi_rows * 2) >> ss)) mh = ((mi_rows * 2) >> ss) - o4y;
    t.tx = tx;
    t.n = 4 << tx;
    t.nx4 = mw;
    t.ny4 = mh;
    t.pbw = pw;
    t.pbh = ph;
    t.px0 = ss ? b->x / 2 : b->x;
    t.py0 = ss ? b->y / 2 : b->y;
    return t;
}

static int full_frame_alloc(oracle_frame_t *f, uint32_t w, uint32_t h)
{
    oracle_frame_free(f);
    f->width = w; f->height = h; f->stride_y = w; f->stride_uv = (w + 1) / 2;
    size_t ny = (size_t)w * h, nc = (size_t)f->stride_uv * ((h + 1) / 2);
    f->y = malloc(ny ? ny : 1); f->u = malloc(nc ? nc : 1); f->v = malloc(nc ? nc : 1);
    if (!f->y || !f->u || !f->v) { oracle_frame_free(f); return 0; }
    memset(f->y, 128, ny); memset(f->u, 128, nc); memset(f->v, 128, nc);
    return 1;
}

static void add_residual(plane_t pl, int x0, int y0, int n, const int32_t *res)
{
    for (int r = 0; r < n; r++)
        for (int c = 0; c < n; c++) {
            int X = x0 + c, Y = y0 + r;
            if (X >= pl.w || Y >= pl.h) continue;
            uint8_t *p = pl.p + (size_t)Y * pl.stride + X;
            *p = (uint8_t)clampi((int)*p + res[r * n + c], 0, 255);
        }
}

static int any_nonzero(const int16_t *c, int n)
{
    for (int i = 0; i < n; i++) if (c[i]) return 1;
    return 0;
}

/* ── Loop filter ───────────────────────────────────────────────────────── */

typedef struct { uint8_t txy, txuv, skipi, xin, yin; } mi_info_t;

typedef struct { int lim, mblim, hev; } lf_thr_t;

static lf_thr_t lf_thresholds(int level, int sharp)
{
    lf_thr_t t;
    int bil = level >> ((sharp > 0) + (sharp > 4));
    if (sharp > 0 && bil > 9 - sharp) bil = 9 - sharp;
    if (bil < 1) bil = 1;
    t.lim = bil;
    t.mblim = 2 * (level + 2) + bil;
    t.hev = level >> 4;
    return t;
}

static inline int sc8(int v) { return v < -128 ? -128 : (v > 127 ? 127 : v); }

/* Filter across one edge at sample s[0] (q0), s[-1] (p0), step between
 * taps `st`; fs = 4, 8 or 16 (the widest filter allowed there). */
static void lf_edge(uint8_t *s, int st, int fs, lf_thr_t th)
{
#define P(i) ((int)s[(-(i) - 1) * st])
#define Q(i) ((int)s[(i) * st])
    const int p3 = P(3), p2 = P(2), p1 = P(1), p0 = P(0), q0 = Q(0), q1 = Q(1), q2 = Q(2), q3 = Q(3);
    const int mask = absi(p3 - p2) <= th.lim && absi(p2 - p1) <= th.lim && absi(p1 - p0) <= th.lim &&
                     absi(q1 - q0) <= th.lim && absi(q2 - q1) <= th.lim && absi(q3 - q2) <= th.lim &&
                     absi(p0 - q0) * 2 + absi(p1 - q1) / 2 <= th.mblim;
    if (!mask) return;
    const int flat = fs >= 8 && absi(p1 - p0) <= 1 && absi(q1 - q0) <= 1 && absi(p2 - p0) <= 1 &&
                     absi(q2 - q0) <= 1 && absi(p3 - p0) <= 1 && absi(q3 - q0) <= 1;
    int flat2 = 0;
    if (fs == 16 && flat) {
        flat2 = 1;
        for (int i = 4; i < 8; i++) flat2 &= absi(P(i) - p0) <= 1 && absi(Q(i) - q0) <= 1;
    }
    if (flat2) {
        /* 15-tap: window of 15 around each of p6..q6, centre weighted 2,
         * samples beyond p7/q7 repeating them */
        int v[16], o[16];
        for (int i = 0; i < 8; i++) { v[7 - i] = P(i); v[8 + i] = Q(i); }
        for (int k = 1; k < 15; k++) {
            int acc = v[k];
            for (int t = k - 7; t <= k + 7; t++) acc += v[clampi(t, 0, 15)];
            o[k] = (acc + 8) >> 4;
        }
        for (int k = 1; k < 15; k++) s[(k - 8) * st] = (uint8_t)o[k];
    } else if (flat) {
        /* 7-tap on p2..q2 over p3..q3, the same window rule */
        int v[8], o[8];
        for (int i = 0; i < 4; i++) { v[3 - i] = P(i); v[4 + i] = Q(i); }
        for (int k = 1; k < 7; k++) {
            int acc = v[k];
            for (int t = k - 3; t <= k + 3; t++) acc += v[clampi(t, 0, 7)];
            o[k] = (acc + 4) >> 3;
        }
        for (int k = 1; k < 7; k++) s[(k - 4) * st] = (uint8_t)o[k];
    } else {
        const int ps1 = p1 - 128, ps0 = p0 - 128, qs0 = q0 - 128, qs1 = q1 - 128;
        const int hev = absi(p1 - p0) > th.hev || absi(q1 - q0) > th.hev;
        int f = hev ? sc8(ps1 - qs1) : 0;
        f = sc8(f + 3 * (qs0 - ps0));
        const int f1 = sc8(f + 4) >> 3, f2 = sc8(f + 3) >> 3;
        s[0] = (uint8_t)(sc8(qs0 - f1) + 128);
        s[-st] = (uint8_t)(sc8(ps0 + f2) + 128);
        if (!hev) {
            const int f3 = (f1 + 1) >> 1;
            s[st] = (uint8_t)(sc8(qs1 - f3) + 128);
            s[-2 * st] = (uint8_t)(sc8(ps1 + f3) + 128);
        }
    }
#undef P
#undef Q
}

/* Filter size of the edge on the left (dir 0) or top (dir 1) side of 8x8
 * unit (ux, uy) of a plane, 0 for none; *inner: the 4x4 edge 4 samples in
 * is filtered too. Chroma units take the block at their top-left MI. */
static int lf_unit_edge(const mi_info_t *mi, int mi_cols, int mi_rows, int plane, int ux, int uy, int dir,
                        int *inner)
{
    const int ss = plane > 0;
    const mi_info_t *m = &mi[(size_t)(uy << ss) * mi_cols + (ux << ss)];
    const int tx = ss ? m->txuv : m->txy;
    const int pos = (dir ? m->yin : m->xin) * (ss ? 4 : 8);     /* samples into the block */
    const int e = (dir ? uy : ux) * 8;                          /* edge in plane samples  */
    /* a chroma unit whose second half lies past the frame edge */
    const int half = ss && (((dir ? uy : ux) << 1) + 1 >= (dir ? mi_rows : mi_cols));
    *inner = tx == 0 && !m->skipi && !half;
    if (e == 0) return 0;
    const int block_edge = pos == 0, tx_edge = pos % (4 << tx) == 0;
    if (!block_edge && !(tx_edge && !m->skipi)) return 0;
    int fs = tx == 0 ? 4 : (tx == 1 ? 8 : 16);
    if (fs == 4 && e % 32 == 0) fs = 8;
    if (fs == 16 && half) fs = 8;
    return fs;
}

static void full_loopfilter(oracle_frame_t *out, const mi_info_t *mi, int mi_cols, int mi_rows,
                            int level, int sharp)
{
    if (level == 0) return;
    const lf_thr_t th = lf_thresholds(level, sharp);
    const int sb_cols = (mi_cols + 7) >> 3, sb_rows = (mi_rows + 7) >> 3;
    for (int sr = 0; sr < sb_rows; sr++)
        for (int sc = 0; sc < sb_cols; sc++)
            for (int p = 0; p < 3; p++) {
                plane_t pl = fplane(out, p);
                const int ss = p > 0, sz = 64 >> ss;
                const int x0 = sc * sz, y0 = sr * sz;
                const int x1 = mini(x0 + sz, pl.w), y1 = mini(y0 + sz, pl.h);
                /* vertical edges: each row left to right */
                for (int y = y0; y < y1; y++)
                    for (int x = x0; x < x1; x += 8) {
                        int inner, fs = lf_unit_edge(mi, mi_cols, mi_rows, p, x >> 3, y >> 3, 0, &inner);
                        uint8_t *s = pl.p + (size_t)y * pl.stride + x;
                        if (fs) lf_edge(s, 1, fs, th);
                        if (inner && x + 4 < pl.w) lf_edge(s + 4, 1, 4, th);
                    }
                /* horizontal edges: each column top to bottom */
                for (int x = x0; x < x1; x++)
                    for (int y = y0; y < y1; y += 8) {
                        int inner, fs = lf_unit_edge(mi, mi_cols, mi_rows, p, x >> 3, y >> 3, 1, &inner);
                        uint8_t *s = pl.p + (size_t)y * pl.stride + x;
                        if (fs) lf_edge(s, pl.stride, fs, th);
                        if (inner && y + 4 < pl.h) lf_edge(s + 4 * (size_t)pl.stride, pl.stride, 4, th);
                    }
            }
}

/* ── Frame ─────────────────────────────────────────────────────────────── */

int oracle_full_reconstruct(const vp9_parsed_frame_t *pf, const oracle_frame_t *const pool[8],
                            oracle_frame_t *out)
{
    const int W = (int)pf->hdr.width, H = (int)pf->hdr.height;
    const int inter_frame = pf->hdr.frame_type != VP9_FRAME_KEY && !pf->hdr.intra_only;
    if ((W & 7) || (H & 7) || (inter_frame && (int)pf->hdr.interp_filter > 3)) return 0;
    for (int k = 0; k < 3; k++) {
        const oracle_frame_t *r = pool[pf->hdr.ref_frame_idx[k] & 7];
        if (inter_frame && r && r->y && ((int)r->width != W || (int)r->height != H))
            return 0;
    }
    if (!full_frame_alloc(out, (uint32_t)W, (uint32_t)H)) return 0;
    const int mi_cols = W >> 3, mi_rows = H >> 3;
    const int base = pf->hdr.base_qindex;
    const int lossless = base == 0 && pf->hdr.y_dc_delta_q == 0 && pf->hdr.uv_dc_delta_q == 0 &&
                         pf->hdr.uv_ac_delta_q == 0;
    const int qdc[2] = { k_dc_q[CVP9_QINDEX_CLAMP(base + pf->hdr.y_dc_delta_q)],
                         k_dc_q[CVP9_QINDEX_CLAMP(base + pf->hdr.uv_dc_delta_q)] };
    const int qac[2] = { k_ac_q[CVP9_QINDEX_CLAMP(base)],
                         k_ac_q[CVP9_QINDEX_CLAMP(base + pf->hdr.uv_ac_delta_q)] };
    const int (*filt)[8] = k_filters[inter_frame ? pf->hdr.interp_filter : 0];
    plane_t dp[3] = { fplane(out, 0), fplane(out, 1), fplane(out, 2) };
    mi_info_t *mi = calloc((size_t)mi_cols * mi_rows, sizeof(mi_info_t));
    if (!mi) return 0;
    int32_t res[1024];

    for (uint32_t bi = 0; bi < pf->num_blocks; bi++) {
        const vp9_macroblock_info_t *b = &pf->blocks[bi];
        const int sub8 = b->width < 8 || b->height < 8;
        const int bw = sub8 ? 8 : b->width, bh = sub8 ? 8 : b->height;
        const int bx = b->x, by = b->y;
        const int mi_col = bx >> 3, mi_row = by >> 3;
        if (bx >= W || by >= H) continue;
        const int cw = mini(bw, W - bx), ch = mini(bh, H - by);
        const int ccw = mini(bw / 2 > 4 ? bw / 2 : 4, dp[1].w - bx / 2), cch = mini(bh / 2 > 4 ? bh / 2 : 4, dp[1].h - by / 2);

        /* mode info for the loop filter */
        {
            int uvpw = bw / 2 < 4 ? 4 : bw / 2, uvph = bh / 2 < 4 ? 4 : bh / 2;
            int txuv = sub8 ? 0 : mini(b->tx_size, max_tx_for(uvpw, uvph));
            for (int r = 0; r < (ch + 7) / 8; r++)
                for (int c = 0; c < (cw + 7) / 8; c++) {
                    mi_info_t *m = &mi[(size_t)(mi_row + r) * mi_cols + mi_col + c];
                    m->txy = b->tx_size & 3;
                    m->txuv = (uint8_t)txuv;
                    m->skipi = b->skip && !b->is_intra;
                    m->xin = (uint8_t)c;
                    m->yin = (uint8_t)r;
                }
        }

        uint32_t off = b->coeff_offset;
        if (!b->is_intra) {
            for (int k = 0; k < 2; k++) {
                if (k == 1 && b->ref_frame[1] == 0) break;
                int sel = clampi((int)b->ref_frame[k] - 1, 0, 2);
                const oracle_frame_t *ref = pool[pf->hdr.ref_frame_idx[sel] & 7];
                if (!ref || !ref->y) {
                    if (k == 0)
                        for (int p = 0; p < 3; p++) {
                            int x0 = p ? bx / 2 : bx, y0 = p ? by / 2 : by, ww = p ? ccw : cw, hh = p ? cch : ch;
                            for (int r = 0; r < hh; r++)
                                memset(dp[p].p + (size_t)(y0 + r) * dp[p].stride + x0, 128, (size_t)ww);
                        }
                    break;
                }
                int mvx = b->mv[k][0], mvy = b->mv[k][1];
                inter_region(dp[0], fplane(ref, 0), filt, bx, by, cw, ch, mvx, mvy, 0, k);
                inter_region(dp[1], fplane(ref, 1), filt, bx / 2, by / 2, ccw, cch, mvx, mvy, 1, k);
                inter_region(dp[2], fplane(ref, 2), filt, bx / 2, by / 2, ccw, cch, mvx, mvy, 1, k);
            }
            if (!b->skip && b->tx_size <= 3)
                for (int p = 0; p < 3; p++) {
                    ptx_t t = plane_tx(b, p, mi_cols, mi_rows);
                    const int pl = p > 0;
                    for (int y4 = 0; y4 < t.ny4; y4 += 1 << t.tx)
                        for (int x4 = 0; x4 < t.nx4; x4 += 1 << t.tx) {
                            if (off + (uint32_t)(t.n * t.n) > pf->num_coeffs) { off = pf->num_coeffs; continue; }
                            const int16_t *src = pf->coeffs + off;
                            off += (uint32_t)(t.n * t.n);
                            if (!any_nonzero(src, t.n * t.n)) continue;
                            oracle_full_itx2d(src, res, t.n, 0, lossless, qdc[pl], qac[pl]);
                            add_residual(dp[p], t.px0 + x4 * 4, t.py0 + y4 * 4, t.n, res);
                        }
                }
        } else {
            const int left_ok = mi_col > tile_start(mi_col, mi_cols, pf->hdr.log2_tile_cols);
            for (int p = 0; p < 3; p++) {
                ptx_t t = plane_tx(b, p, mi_cols, mi_rows);
                const int pl = p > 0;
                const int mode = p ? b->uv_mode : b->y_mode;
                const int tx_type = (p == 0 && !lossless && t.tx < 3 && b->y_mode < 10) ? k_tx_type[b->y_mode] : 0;
                const int step = 1 << t.tx, pbw4 = t.pbw / 4;
                for (int y4 = 0; y4 < t.ny4; y4 += step)
                    for (int x4 = 0; x4 < t.nx4; x4 += step) {
                        const int x0 = t.px0 + x4 * 4, y0 = t.py0 + y4 * 4;
                        oracle_full_intra_tx(dp[p].p, dp[p].w, dp[p].h, dp[p].stride, x0, y0, t.n,
                                             mode > 9 ? 0 : mode, y4 > 0 || mi_row > 0, x4 > 0 || left_ok,
                                             x4 + step < pbw4);
                        if (b->skip || b->tx_size > 3) continue;
                        if (off + (uint32_t)(t.n * t.n) > pf->num_coeffs) { off = pf->num_coeffs; continue; }
                        const int16_t *src = pf->coeffs + off;
                        off += (uint32_t)(t.n * t.n);
                        if (!any_nonzero(src, t.n * t.n)) continue;
                        oracle_full_itx2d(src, res, t.n, tx_type, lossless, qdc[pl], qac[pl]);
                        add_residual(dp[p], x0, y0, t.n, res);
                    }
            }
        }
    }

    full_loopfilter(out, mi, mi_cols, mi_rows, pf->hdr.filter_level, pf->hdr.sharpness_level);
    free(mi);
    return 1;
}
