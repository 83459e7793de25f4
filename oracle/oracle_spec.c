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

#define TXI int
#define TXN(name) name
#include "oracle_txfm_dct.inc"
#undef TXI
#undef TXN

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
