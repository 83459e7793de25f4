/*
 * oracle_spec.c — scalar restatement of the shader arithmetic (SPEC
 * profile). TEST INFRASTRUCTURE ONLY: the checker for the CUDA SPEC profile.
 *
 * Built with -fwrapv: the shader integer math is 32-bit two's complement with
 * no intermediate clamp (vp9_idct.comp.glsl), and right shifts of negative
 * values are arithmetic.
 */
#include "oracle.h"
#include "../compute_vp9_b200/csrc/vp9_tables.h"

#include <stdlib.h>
#include <string.h>

static const int16_t k_dc_q[256] = CVP9_QTABLE_DC_INIT;
static const int16_t k_ac_q[256] = CVP9_QTABLE_AC_INIT;
static const int k_subpel[16][8] = CVP9_SUBPEL_REGULAR_INIT;

int oracle_dc_quant(int q) { return k_dc_q[CVP9_QINDEX_CLAMP(q)]; }
int oracle_ac_quant(int q) { return k_ac_q[CVP9_QINDEX_CLAMP(q)]; }

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* cos(k*pi/64) in Q14, the butterfly multipliers. */
enum {
    C1 = 16364, C2 = 16305, C3 = 16207, C4 = 16069, C5 = 15893, C6 = 15679,
    C7 = 15426, C8 = 15137, C9 = 14811, C10 = 14449, C11 = 14053, C12 = 13623,
    C13 = 13160, C14 = 12665, C15 = 12140, C16 = 11585, C17 = 11003, C18 = 10394,
    C19 = 9760, C20 = 9102, C21 = 8423, C22 = 7723, C23 = 7005, C24 = 6270,
    C25 = 5520, C26 = 4756, C27 = 3981, C28 = 3196, C29 = 2404, C30 = 1606,
    C31 = 804
};

/* Q14 rounding shift after every multiply (vp9_idct.comp.glsl:42). */
#define RS(x) (((x) + 8192) >> 14)

/* ── 1-D inverse DCTs (vp9_idct.comp.glsl:47-649) ──────────────────────── */

static void idct4(const int *in, int *out)
{
    int s0 = RS((in[0] + in[2]) * C16);
    int s1 = RS((in[0] - in[2]) * C16);
    int s2 = RS(in[1] * C24 - in[3] * C8);
    int s3 = RS(in[1] * C8 + in[3] * C24);
    out[0] = s0 + s3;
    out[1] = s1 + s2;
    out[2] = s1 - s2;
    out[3] = s0 - s3;
}

static void idct8(const int *in, int *out)
{
    int a[8], b[8];
    a[0] = in[0]; a[1] = in[2]; a[2] = in[4]; a[3] = in[6];
    a[4] = RS(in[1] * C28 - in[7] * C4);
    a[7] = RS(in[1] * C4 + in[7] * C28);
    a[5] = RS(in[5] * C12 - in[3] * C20);
    a[6] = RS(in[5] * C20 + in[3] * C12);

    b[0] = RS((a[0] + a[2]) * C16);
    b[1] = RS((a[0] - a[2]) * C16);
    b[2] = RS(a[1] * C24 - a[3] * C8);
    b[3] = RS(a[1] * C8 + a[3] * C24);
    b[4] = a[4] + a[5];
    b[5] = a[4] - a[5];
    b[6] = -a[6] + a[7];
    b[7] = a[6] + a[7];

    a[0] = b[0] + b[3];
    a[1] = b[1] + b[2];
    a[2] = b[1] - b[2];
    a[3] = b[0] - b[3];
    a[4] = b[4];
    a[5] = RS((b[6] - b[5]) * C16);
    a[6] = RS((b[5] + b[6]) * C16);
    a[7] = b[7];

    for (int i = 0; i < 4; i++) {
        out[i] = a[i] + a[7 - i];
        out[7 - i] = a[i] - a[7 - i];
    }
}

static void idct16(const int *in, int *out)
{
    int a[16], b[16];
    /* even/odd reordering of the inputs */
    static const int perm[16] = { 0, 8, 4, 12, 2, 10, 6, 14, 1, 9, 5, 13, 3, 11, 7, 15 };
    for (int i = 0; i < 16; i++) a[i] = in[perm[i]];

    for (int i = 0; i < 8; i++) b[i] = a[i];
    b[8]  = RS(a[8] * C30 - a[15] * C2);
    b[15] = RS(a[8] * C2 + a[15] * C30);
    b[9]  = RS(a[9] * C14 - a[14] * C18);
    b[14] = RS(a[9] * C18 + a[14] * C14);
    b[10] = RS(a[10] * C22 - a[13] * C10);
    b[13] = RS(a[10] * C10 + a[13] * C22);
    b[11] = RS(a[11] * C6 - a[12] * C26);
    b[12] = RS(a[11] * C26 + a[12] * C6);

    for (int i = 0; i < 4; i++) a[i] = b[i];
    a[4] = RS(b[4] * C28 - b[7] * C4);
    a[7] = RS(b[4] * C4 + b[7] * C28);
    a[5] = RS(b[5] * C12 - b[6] * C20);
    a[6] = RS(b[5] * C20 + b[6] * C12);
    a[8]  = b[8] + b[9];
    a[9]  = b[8] - b[9];
    a[10] = -b[10] + b[11];
    a[11] = b[10] + b[11];
    a[12] = b[12] + b[13];
    a[13] = b[12] - b[13];
    a[14] = -b[14] + b[15];
    a[15] = b[14] + b[15];

    b[0] = RS((a[0] + a[1]) * C16);
    b[1] = RS((a[0] - a[1]) * C16);
    b[2] = RS(a[2] * C24 - a[3] * C8);
    b[3] = RS(a[2] * C8 + a[3] * C24);
    b[4] = a[4] + a[5];
    b[5] = a[4] - a[5];
    b[6] = -a[6] + a[7];
    b[7] = a[6] + a[7];
    b[8] = a[8];
    b[15] = a[15];
    b[9]  = RS(-a[9] * C8 + a[14] * C24);
    b[14] = RS(a[9] * C24 + a[14] * C8);
    b[10] = RS(-a[10] * C24 - a[13] * C8);
    b[13] = RS(-a[10] * C8 + a[13] * C24);
    b[11] = a[11];
    b[12] = a[12];

    a[0] = b[0] + b[3];
    a[1] = b[1] + b[2];
    a[2] = b[1] - b[2];
    a[3] = b[0] - b[3];
    a[4] = b[4];
    a[5] = RS((b[6] - b[5]) * C16);
    a[6] = RS((b[5] + b[6]) * C16);
    a[7] = b[7];
    a[8]  = b[8] + b[11];
    a[9]  = b[9] + b[10];
    a[10] = b[9] - b[10];
    a[11] = b[8] - b[11];
    a[12] = -b[12] + b[15];
    a[13] = -b[13] + b[14];
    a[14] = b[13] + b[14];
    a[15] = b[12] + b[15];

    for (int i = 0; i < 4; i++) {
        b[i] = a[i] + a[7 - i];
        b[7 - i] = a[i] - a[7 - i];
    }
    b[8] = a[8];
    b[9] = a[9];
    b[10] = RS((-a[10] + a[13]) * C16);
    b[13] = RS((a[10] + a[13]) * C16);
    b[11] = RS((-a[11] + a[12]) * C16);
    b[12] = RS((a[11] + a[12]) * C16);
    b[14] = a[14];
    b[15] = a[15];

    for (int i = 0; i < 8; i++) {
        out[i] = b[i] + b[15 - i];
        out[15 - i] = b[i] - b[15 - i];
    }
}

static void idct32(const int *in, int *out)
{
    int a[32], b[32];
    /* stage 1: even inputs in bit-reversed order, odd inputs rotated */
    static const int perm[16] = { 0, 16, 8, 24, 4, 20, 12, 28, 2, 18, 10, 26, 6, 22, 14, 30 };
    for (int i = 0; i < 16; i++) a[i] = in[perm[i]];
    a[16] = RS(in[1] * C31 - in[31] * C1);
    a[31] = RS(in[1] * C1 + in[31] * C31);
    a[17] = RS(in[17] * C15 - in[15] * C17);
    a[30] = RS(in[17] * C17 + in[15] * C15);
    a[18] = RS(in[9] * C23 - in[23] * C9);
    a[29] = RS(in[9] * C9 + in[23] * C23);
    a[19] = RS(in[25] * C7 - in[7] * C25);
    a[28] = RS(in[25] * C25 + in[7] * C7);
    a[20] = RS(in[5] * C27 - in[27] * C5);
    a[27] = RS(in[5] * C5 + in[27] * C27);
    a[21] = RS(in[21] * C11 - in[11] * C21);
    a[26] = RS(in[21] * C21 + in[11] * C11);
    a[22] = RS(in[13] * C19 - in[19] * C13);
    a[25] = RS(in[13] * C13 + in[19] * C19);
    a[23] = RS(in[29] * C3 - in[3] * C29);
    a[24] = RS(in[29] * C29 + in[3] * C3);

    /* stage 2 */
    for (int i = 0; i < 8; i++) b[i] = a[i];
    b[8]  = RS(a[8] * C30 - a[15] * C2);
    b[15] = RS(a[8] * C2 + a[15] * C30);
    b[9]  = RS(a[9] * C14 - a[14] * C18);
    b[14] = RS(a[9] * C18 + a[14] * C14);
    b[10] = RS(a[10] * C22 - a[13] * C10);
    b[13] = RS(a[10] * C10 + a[13] * C22);
    b[11] = RS(a[11] * C6 - a[12] * C26);
    b[12] = RS(a[11] * C26 + a[12] * C6);
    for (int i = 16; i < 32; i += 4) {
        b[i]     = a[i] + a[i + 1];
        b[i + 1] = a[i] - a[i + 1];
        b[i + 2] = -a[i + 2] + a[i + 3];
        b[i + 3] = a[i + 2] + a[i + 3];
    }

    /* stage 3 */
    for (int i = 0; i < 4; i++) a[i] = b[i];
    a[4] = RS(b[4] * C28 - b[7] * C4);
    a[7] = RS(b[4] * C4 + b[7] * C28);
    a[5] = RS(b[5] * C12 - b[6] * C20);
    a[6] = RS(b[5] * C20 + b[6] * C12);
    for (int i = 8; i < 16; i += 4) {
        a[i]     = b[i] + b[i + 1];
        a[i + 1] = b[i] - b[i + 1];
        a[i + 2] = -b[i + 2] + b[i + 3];
        a[i + 3] = b[i + 2] + b[i + 3];
    }
    a[16] = b[16];
    a[31] = b[31];
    a[17] = RS(-b[17] * C4 + b[30] * C28);
    a[30] = RS(b[17] * C28 + b[30] * C4);
    a[18] = RS(-b[18] * C28 - b[29] * C4);
    a[29] = RS(-b[18] * C4 + b[29] * C28);
    a[19] = b[19];
    a[20] = b[20];
    a[21] = RS(-b[21] * C20 + b[26] * C12);
    a[26] = RS(b[21] * C12 + b[26] * C20);
    a[22] = RS(-b[22] * C12 - b[25] * C20);
    a[25] = RS(-b[22] * C20 + b[25] * C12);
    a[23] = b[23];
    a[24] = b[24];
    a[27] = b[27];
    a[28] = b[28];

    /* stage 4 */
    b[0] = RS((a[0] + a[1]) * C16);
    b[1] = RS((a[0] - a[1]) * C16);
    b[2] = RS(a[2] * C24 - a[3] * C8);
    b[3] = RS(a[2] * C8 + a[3] * C24);
    b[4] = a[4] + a[5];
    b[5] = a[4] - a[5];
    b[6] = -a[6] + a[7];
    b[7] = a[6] + a[7];
    b[8] = a[8];
    b[15] = a[15];
    b[9]  = RS(-a[9] * C8 + a[14] * C24);
    b[14] = RS(a[9] * C24 + a[14] * C8);
    b[10] = RS(-a[10] * C24 - a[13] * C8);
    b[13] = RS(-a[10] * C8 + a[13] * C24);
    b[11] = a[11];
    b[12] = a[12];
    for (int i = 16; i < 32; i += 8) {
        b[i]     = a[i] + a[i + 3];
        b[i + 1] = a[i + 1] + a[i + 2];
        b[i + 2] = a[i + 1] - a[i + 2];
        b[i + 3] = a[i] - a[i + 3];
        b[i + 4] = -a[i + 4] + a[i + 7];
        b[i + 5] = -a[i + 5] + a[i + 6];
        b[i + 6] = a[i + 5] + a[i + 6];
        b[i + 7] = a[i + 4] + a[i + 7];
    }

    /* stage 5 */
    a[0] = b[0] + b[3];
    a[1] = b[1] + b[2];
    a[2] = b[1] - b[2];
    a[3] = b[0] - b[3];
    a[4] = b[4];
    a[5] = RS((b[6] - b[5]) * C16);
    a[6] = RS((b[5] + b[6]) * C16);
    a[7] = b[7];
    a[8]  = b[8] + b[11];
    a[9]  = b[9] + b[10];
    a[10] = b[9] - b[10];
    a[11] = b[8] - b[11];
    a[12] = -b[12] + b[15];
    a[13] = -b[13] + b[14];
    a[14] = b[13] + b[14];
    a[15] = b[12] + b[15];
    a[16] = b[16];
    a[17] = b[17];
    a[18] = RS(-b[18] * C8 + b[29] * C24);
    a[29] = RS(b[18] * C24 + b[29] * C8);
    a[19] = RS(-b[19] * C8 + b[28] * C24);
    a[28] = RS(b[19] * C24 + b[28] * C8);
    a[20] = RS(-b[20] * C24 - b[27] * C8);
    a[27] = RS(-b[20] * C8 + b[27] * C24);
    a[21] = RS(-b[21] * C24 - b[26] * C8);
    a[26] = RS(-b[21] * C8 + b[26] * C24);
    a[22] = b[22];
    a[23] = b[23];
    a[24] = b[24];
    a[25] = b[25];
    a[30] = b[30];
    a[31] = b[31];

    /* stage 6 */
    for (int i = 0; i < 4; i++) {
        b[i] = a[i] + a[7 - i];
        b[7 - i] = a[i] - a[7 - i];
    }
    b[8] = a[8];
    b[9] = a[9];
    b[10] = RS((-a[10] + a[13]) * C16);
    b[13] = RS((a[10] + a[13]) * C16);
    b[11] = RS((-a[11] + a[12]) * C16);
    b[12] = RS((a[11] + a[12]) * C16);
    b[14] = a[14];
    b[15] = a[15];
    for (int i = 0; i < 4; i++) {
        b[16 + i] = a[16 + i] + a[23 - i];
        b[23 - i] = a[16 + i] - a[23 - i];
        b[24 + i] = -a[24 + i] + a[31 - i];
        b[31 - i] = a[24 + i] + a[31 - i];
    }

    /* stage 7 */
    for (int i = 0; i < 8; i++) {
        a[i] = b[i] + b[15 - i];
        a[15 - i] = b[i] - b[15 - i];
    }
    for (int i = 16; i < 20; i++) a[i] = b[i];
    for (int i = 0; i < 4; i++) {
        int lo = 20 + i, hi = 27 - i;
        a[lo] = RS((-b[lo] + b[hi]) * C16);
        a[hi] = RS((b[lo] + b[hi]) * C16);
    }
    for (int i = 28; i < 32; i++) a[i] = b[i];

    /* final stage */
    for (int i = 0; i < 16; i++) {
        out[i] = a[i] + a[31 - i];
        out[31 - i] = a[i] - a[31 - i];
    }
}

void oracle_idct1d(int n, const int *in, int *out)
{
    int tmp[32];
    memcpy(tmp, in, (size_t)n * sizeof(int));
    switch (n) {
    case 4: idct4(tmp, out); break;
    case 8: idct8(tmp, out); break;
    case 16: idct16(tmp, out); break;
    default: idct32(tmp, out); break;
    }
}

/* Dequantise (DC step at [0][0] only, no 32x32 halving), columns then rows,
 * final rounding shift 4/5/6/6 for N = 4/8/16/32 (vp9_idct.comp.glsl:654-789). */
void oracle_spec_idct2d(const int16_t *in, int32_t *out, int n, int q_dc, int q_ac)
{
    int buf[32][32];
    int col[32], res[32];
    for (int c = 0; c < n; c++) {
        for (int r = 0; r < n; r++) col[r] = (int)in[r * n + c] * ((r == 0 && c == 0) ? q_dc : q_ac);
        oracle_idct1d(n, col, res);
        for (int r = 0; r < n; r++) buf[r][c] = res[r];
    }
    for (int r = 0; r < n; r++) {
        oracle_idct1d(n, buf[r], res);
        for (int c = 0; c < n; c++) buf[r][c] = res[c];
    }
    int sh = n == 4 ? 4 : (n == 8 ? 5 : 6);
    for (int r = 0; r < n; r++)
        for (int c = 0; c < n; c++)
            out[r * n + c] = (buf[r][c] + (1 << (sh - 1))) >> sh;
}

/* ── Plane helpers ─────────────────────────────────────────────────────── */

typedef struct {
    uint8_t *p;
    int w, h, stride;
} plane_t;

static plane_t frame_plane(const oracle_frame_t *f, int idx)
{
    plane_t pl;
    if (idx == 0) { pl.p = f->y; pl.w = (int)f->width; pl.h = (int)f->height; pl.stride = (int)f->stride_y; }
    else {
        pl.p = idx == 1 ? f->u : f->v;
        pl.w = (int)(f->width + 1) / 2; pl.h = (int)(f->height + 1) / 2; pl.stride = (int)f->stride_uv;
    }
    return pl;
}

/* Intra prediction with the shader's availability rules
 * (vp9_intra_pred.comp.glsl:54-109), generalised to w x h: above samples
 * span the block width, left samples the block height, unavailable edges
 * read 128; modes other than DC/V/H/TM(9) fall back to V. */
static void spec_intra(plane_t pl, int x, int y, int w, int h, int mode)
{
    int has_above = y > 0, has_left = x > 0;
    const uint8_t *P = pl.p;
    int S = pl.stride;
    int dc = 128;
    if (mode == 0) {
        uint32_t sa = 0, sl = 0;
        if (has_above) for (int i = 0; i < w; i++) sa += P[(size_t)(y - 1) * S + x + i];
        if (has_left) for (int i = 0; i < h; i++) sl += P[(size_t)(y + i) * S + x - 1];
        if (has_above && has_left) dc = (int)((sa + sl + (uint32_t)(w + h) / 2) / (uint32_t)(w + h));
        else if (has_above) dc = (int)((sa + (uint32_t)w / 2) / (uint32_t)w);
        else if (has_left) dc = (int)((sl + (uint32_t)h / 2) / (uint32_t)h);
    }
    int tl = (has_above && has_left) ? P[(size_t)(y - 1) * S + x - 1] : 128;
    uint8_t abv[256], lft[256];
    for (int i = 0; i < w; i++) abv[i] = has_above ? P[(size_t)(y - 1) * S + x + i] : 128;
    for (int i = 0; i < h; i++) lft[i] = has_left ? P[(size_t)(y + i) * S + x - 1] : 128;
    for (int r = 0; r < h; r++)
        for (int c = 0; c < w; c++) {
            int v;
            if (mode == 0) v = dc;
            else if (mode == 2) v = lft[r];
            else if (mode == 9) v = clampi(abv[c] + lft[r] - tl, 0, 255);
            else v = abv[c];
            pl.p[(size_t)(y + r) * S + x + c] = (uint8_t)v;
        }
}

/* Separable 8-tap regular interpolation of one sample at integer base
 * (bx, by) and phases (fx, fy) in 1/16 units, every fetch clamped into the
 * reference plane; horizontal pass rounds and clips to 8 bits before the
 * vertical pass (vp9_mc.comp.glsl:61-110). */
static int spec_interp(plane_t ref, int bx, int by, int fx, int fy)
{
    #define FETCH(xx, yy) ((int)ref.p[(size_t)clampi((yy), 0, ref.h - 1) * ref.stride + clampi((xx), 0, ref.w - 1)])
    if (fx == 0 && fy == 0) return FETCH(bx, by);
    int rows[8];
    for (int r = 0; r < 8; r++) {
        int acc = 0;
        for (int t = 0; t < 8; t++) acc += k_subpel[fx][t] * FETCH(bx + t - 3, by + r - 3);
        rows[r] = clampi((acc + 64) >> 7, 0, 255);
    }
    int acc = 0;
    for (int t = 0; t < 8; t++) acc += k_subpel[fy][t] * rows[t];
    return clampi((acc + 64) >> 7, 0, 255);
    #undef FETCH
}

/* Inter prediction of one plane region: luma uses the 1/8-pel MV on even
 * phases ((mv & 7) << 1, integer mv >> 3); 4:2:0 chroma reads the same MV as
 * 1/16 chroma pel (phase mv & 15, integer mv >> 4). */
static void spec_inter(plane_t dst, plane_t ref, int x, int y, int w, int h,
                       int mvx, int mvy, int chroma)
{
    for (int r = 0; r < h; r++)
        for (int c = 0; c < w; c++) {
            int px = x + c, py = y + r, v;
            if (!chroma) {
                v = spec_interp(ref, px + (mvx >> 3), py + (mvy >> 3), (mvx & 7) << 1, (mvy & 7) << 1);
            } else {
                v = spec_interp(ref, px + (mvx >> 4), py + (mvy >> 4), mvx & 15, mvy & 15);
            }
            dst.p[(size_t)py * dst.stride + px] = (uint8_t)v;
        }
}

/* Stage-level entry points (unit tests against the shader translations). */
void oracle_spec_intra_block(uint8_t *plane, int w, int h, int stride, int x, int y,
                             int bw, int bh, int mode)
{
    plane_t pl = { plane, w, h, stride };
    spec_intra(pl, x, y, bw, bh, mode);
}

void oracle_spec_mc_block(const uint8_t *ref, int rw, int rh, int rstride,
                          uint8_t *dst, int dw, int dh, int dstride,
                          int x, int y, int bw, int bh, int mvx, int mvy, int chroma)
{
    plane_t r = { (uint8_t *)ref, rw, rh, rstride }, d = { dst, dw, dh, dstride };
    spec_inter(d, r, x, y, bw, bh, mvx, mvy, chroma);
}

static int max_tx_for(int w, int h)
{
    int m = w < h ? w : h;
    return m >= 32 ? 3 : (m >= 16 ? 2 : (m >= 8 ? 1 : 0));
}

/* Residual of every TX of one plane in the tile parser's coefficient order
 * (vp9_kf_tile.c:320-396); samples outside the frame are not written.
 * Returns the number of coefficients consumed. */
static uint32_t spec_residual_plane(plane_t pl, const int16_t *coeffs, uint32_t avail,
                                    const vp9_macroblock_info_t *b, int plane,
                                    int mi_cols, int mi_rows, int q_dc, int q_ac)
{
    int ss = plane > 0;
    int sub8 = b->width < 8 || b->height < 8;
    int ew = sub8 ? 8 : b->width, eh = sub8 ? 8 : b->height;
    int pw = ss ? ew / 2 : ew, ph = ss ? eh / 2 : eh;
    if (pw < 4) pw = 4;
    if (ph < 4) ph = 4;
    int tx = b->tx_size;
    if (ss) { int mt = max_tx_for(pw, ph); tx = sub8 ? 0 : (tx > mt ? mt : tx); }
    int n = 4 << tx, txs4 = 1 << tx, area = n * n;
    int mi_col = b->x >> 3, mi_row = b->y >> 3;
    int o4x = (mi_col * 2) >> ss, o4y = (mi_row * 2) >> ss;
    int max_w = pw / 4, max_h = ph / 4;
    if (o4x + max_w > ((mi_cols * 2) >> ss)) max_w = ((mi_cols * 2) >> ss) - o4x;
    if (o4y + max_h > ((mi_rows * 2) >> ss)) max_h = ((mi_rows * 2) >> ss) - o4y;
    int px0 = ss ? b->x / 2 : b->x, py0 = ss ? b->y / 2 : b->y;
    int32_t res[1024];
    uint32_t used = 0;
    for (int y4 = 0; y4 < max_h; y4 += txs4)
        for (int x4 = 0; x4 < max_w; x4 += txs4) {
            if (used + (uint32_t)area > avail) return used;
            const int16_t *src = coeffs + used;
            used += (uint32_t)area;
            int nz = 0;
            for (int i = 0; i < area && !nz; i++) nz = src[i] != 0;
            if (!nz) continue;
            oracle_spec_idct2d(src, res, n, q_dc, q_ac);
            for (int r = 0; r < n; r++)
                for (int c = 0; c < n; c++) {
                    int X = px0 + x4 * 4 + c, Y = py0 + y4 * 4 + r;
                    if (X >= pl.w || Y >= pl.h) continue;
                    uint8_t *p = pl.p + (size_t)Y * pl.stride + X;
                    *p = (uint8_t)clampi((int)*p + res[r * n + c], 0, 255);
                }
        }
    return used;
}

static int spec_frame_alloc(oracle_frame_t *f, uint32_t w, uint32_t h)
{
    oracle_frame_free(f);
    f->width = w; f->height = h; f->stride_y = w; f->stride_uv = (w + 1) / 2;
    size_t ny = (size_t)w * h, nc = (size_t)f->stride_uv * ((h + 1) / 2);
    f->y = malloc(ny ? ny : 1); f->u = malloc(nc ? nc : 1); f->v = malloc(nc ? nc : 1);
    if (!f->y || !f->u || !f->v) { oracle_frame_free(f); return 0; }
    memset(f->y, 128, ny); memset(f->u, 128, nc); memset(f->v, 128, nc);
    return 1;
}

int oracle_spec_reconstruct(const vp9_parsed_frame_t *pf,
                            const oracle_frame_t *const pool[8],
                            oracle_frame_t *out)
{
    int W = (int)pf->hdr.width, H = (int)pf->hdr.height;
    if (!spec_frame_alloc(out, (uint32_t)W, (uint32_t)H)) return 0;
    int mi_cols = (W + 7) >> 3, mi_rows = (H + 7) >> 3;
    int q_dc = oracle_dc_quant(pf->hdr.base_qindex);
    int q_ac = oracle_ac_quant(pf->hdr.base_qindex);
    plane_t dp[3] = { frame_plane(out, 0), frame_plane(out, 1), frame_plane(out, 2) };

    for (uint32_t bi = 0; bi < pf->num_blocks; bi++) {
        const vp9_macroblock_info_t *b = &pf->blocks[bi];
        int bx = b->x, by = b->y, bw = b->width, bh = b->height;
        if (bx + bw > W) bw = W - bx;
        if (by + bh > H) bh = H - by;
        if (bw <= 0 || bh <= 0) continue;
        int cbx = bx / 2, cby = by / 2, cbw = (bw + 1) / 2, cbh = (bh + 1) / 2;

        if (b->is_intra) {
            spec_intra(dp[0], bx, by, bw, bh, b->y_mode);
            spec_intra(dp[1], cbx, cby, cbw, cbh, b->uv_mode);
            spec_intra(dp[2], cbx, cby, cbw, cbh, b->uv_mode);
        } else {
            /* reference selector 0..2 through the header's slot indices */
            int sel = clampi((int)b->ref_frame[0] - 1, 0, 2);
            const oracle_frame_t *ref = pool[pf->hdr.ref_frame_idx[sel] & 7];
            if (ref && ref->y) {
                spec_inter(dp[0], frame_plane(ref, 0), bx, by, bw, bh, b->mv[0][0], b->mv[0][1], 0);
                spec_inter(dp[1], frame_plane(ref, 1), cbx, cby, cbw, cbh, b->mv[0][0], b->mv[0][1], 1);
                spec_inter(dp[2], frame_plane(ref, 2), cbx, cby, cbw, cbh, b->mv[0][0], b->mv[0][1], 1);
            } else {
                for (int p = 0; p < 3; p++) {
                    int x0 = p ? cbx : bx, y0 = p ? cby : by, ww = p ? cbw : bw, hh = p ? cbh : bh;
                    for (int r = 0; r < hh; r++)
                        memset(dp[p].p + (size_t)(y0 + r) * dp[p].stride + x0, 128, (size_t)ww);
                }
            }
        }

        if (!b->skip && b->tx_size <= 3) {
            uint32_t off = b->coeff_offset;
            for (int p = 0; p < 3; p++) {
                uint32_t avail = off < pf->num_coeffs ? pf->num_coeffs - off : 0;
                off += spec_residual_plane(dp[p], pf->coeffs + off, avail, b, p,
                                           mi_cols, mi_rows, q_dc, q_ac);
            }
        }
    }

    oracle_loopfilter(out->y, (uint32_t)W, (uint32_t)H, out->stride_y,
                      pf->hdr.filter_level, pf->hdr.sharpness_level, ORACLE_SPEC);
    return 1;
}

void oracle_nv12_pack(const uint8_t *i420, uint8_t *dst, uint32_t w, uint32_t h)
{
    uint32_t cw = (w + 1) / 2, ch = (h + 1) / 2;
    size_t ly = (size_t)w * h, lc = (size_t)cw * ch;
    memcpy(dst, i420, ly);
    for (uint32_t y = 0; y < ch; y++)
        for (uint32_t x = 0; x < cw; x++) {
            dst[ly + (size_t)y * 2 * cw + 2 * x]     = i420[ly + (size_t)y * cw + x];
            dst[ly + (size_t)y * 2 * cw + 2 * x + 1] = i420[ly + lc + (size_t)y * cw + x];
        }
}
