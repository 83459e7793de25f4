/*
 * oracle_vp9_common.h — the parts of the FULL oracle that do not depend on
 * the sample type, shared by oracle_full.c (8-bit) and oracle_hbd.c (10-bit):
 * the tile parser's TX layout, tile-column starts and the loop filter's
 * edge selection and thresholds. TEST INFRASTRUCTURE ONLY.
 */
#ifndef ORACLE_VP9_COMMON_H
#define ORACLE_VP9_COMMON_H

#include "oracle.h"

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int mini(int a, int b) { return a < b ? a : b; }
static inline int absi(int v) { return v < 0 ? -v : v; }

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

#endif /* ORACLE_VP9_COMMON_H */
