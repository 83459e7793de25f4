/*
 * synth.c — seeded synthetic parsed-frame generator (host C).
 *
 * Layout conventions reproduced from the CPU tile parser:
 *   - block fields: src/decoder/vp9_kf_tile.c:980-983 (x, y, width, height
 *     from the MI position and block size) and :1153-1165 (modes, refs,
 *     mv[i] = {col,row}, coeff_offset taken before the tokens are appended);
 *   - coefficients: vp9_kf_tile.c:320-396 — per block, plane 0 then 1 then 2;
 *     per plane a raster of TXs clipped at the MI-aligned frame edge, each TX
 *     a dense row-major N*N int16 run; skip blocks append nothing; sub-8x8
 *     blocks code a full 8x8 of luma and a 4x4 per chroma plane;
 *   - MV grid: vp9_kf_tile.c:1167-1182 — one cell per 4x4, covering the
 *     block's MI footprint (at least 8x8), ref selector = ref_frame[0] - 1.
 * Partition shapes follow VP9's rule that a square block whose lower or right
 * half starts outside the frame must be split (HORZ/VERT/SPLIT).
 */
#include "cvp9_synth.h"

#include <stdlib.h>
#include <string.h>

/* ── RNG: splitmix64 seeding a xoshiro256** generator ───────────────────── */

typedef struct { uint64_t s[4]; } rng_t;

static uint64_t splitmix64(uint64_t *x)
{
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static void rng_seed(rng_t *r, uint64_t seed, uint64_t stream)
{
    uint64_t x = seed ^ (stream * 0xD1342543DE82EF95ull);
    for (int i = 0; i < 4; i++) r->s[i] = splitmix64(&x);
}

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static inline uint64_t rng_next(rng_t *r)
{
    uint64_t *s = r->s;
    uint64_t result = rotl(s[1] * 5, 7) * 9;
    uint64_t t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return result;
}

static inline uint32_t rng_u32(rng_t *r) { return (uint32_t)(rng_next(r) >> 32); }

/* uniform integer in [lo, hi] */
static inline int rng_range(rng_t *r, int lo, int hi)
{
    uint64_t span = (uint64_t)(hi - lo) + 1;
    return lo + (int)((rng_next(r) >> 11) % span);
}

/* uniform double in [0, 1) */
static inline double rng_unit(rng_t *r) { return (double)(rng_next(r) >> 11) * (1.0 / 9007199254740992.0); }

/* Exponential(1)-like magnitude without libm: -log2(U) split into the count
 * of leading zero bits plus a linear estimate of the mantissa's log. */
static double rng_exp(rng_t *r)
{
    uint64_t x = rng_next(r) | 1ull;
    int lz = __builtin_clzll(x);
    uint64_t m = x << lz;                       /* top bit set */
    double mant = (double)(m >> 11) * (1.0 / 9007199254740992.0);  /* [0.5,1) */
    return 0.69314718055994530942 * ((double)lz + 2.0 * (1.0 - mant));
}

/* ── Generator state ────────────────────────────────────────────────────── */

struct cvp9_synth {
    cvp9_synth_config_t cfg;
    vp9_parsed_frame_t  pf;
    uint32_t            blocks_cap;
    uint32_t            coeffs_cap;
    /* per-frame scratch used to emit blocks tile-column major */
    vp9_macroblock_info_t *tmp_blocks;
    uint32_t            tmp_cap;
};

void cvp9_synth_preset(cvp9_synth_config_t *c, int preset,
                       uint32_t width, uint32_t height, uint64_t seed)
{
    memset(c, 0, sizeof(*c));
    c->seed = seed;
    c->coeff_max = 512;
    c->coeff_scale = 24.0;
    c->golden_every = 16;
    c->altref_every = 32;
    c->sharpness = 0;
    c->interp_filter = VP9_FILTER_EIGHTTAP;
    c->min_bsize = 8;
    c->max_bsize = 64;
    c->rect_partitions = 0;
    if (preset == 2) {
        c->width = 1920; c->height = 1080;
        c->gop = 60;
        c->fixed_bsize = 0;
        c->rect_partitions = 1;
        c->fixed_tx = -1;
        c->tx_weights[0] = 30; c->tx_weights[1] = 30;
        c->tx_weights[2] = 25; c->tx_weights[3] = 15;
        c->density_min = 0.02; c->density_max = 0.20;
        c->mv_range_px = 128;
        c->nrefs = 3;
        c->qindex = 60;
        c->lf_level = -1;
        c->interp_filter = -1;
        c->intra_in_inter = 0.05;
        c->skip_prob = 0.0;
    } else {
        c->width = 1280; c->height = 720;
        c->gop = 0;
        c->fixed_bsize = 8;
        c->fixed_tx = 1;
        c->density_min = 0.05; c->density_max = 0.05;
        c->mv_range_px = 64;
        c->nrefs = 1;
        c->qindex = 60;
        c->lf_level = 32;
        c->intra_in_inter = 0.0;
        c->skip_prob = 0.0;
    }
    if (width) c->width = width;
    if (height) c->height = height;
}

uint64_t cvp9_fnv1a64(const void *data, size_t n, uint64_t h)
{
    const uint8_t *p = (const uint8_t *)data;
    if (h == 0) h = 0xcbf29ce484222325ull;
    for (size_t i = 0; i < n; i++) {
        h ^= p[i];
        h *= 0x100000001b3ull;
    }
    return h;
}

cvp9_synth_t *cvp9_synth_create(const cvp9_synth_config_t *cfg)
{
    if (!cfg || cfg->width == 0 || cfg->height == 0 ||
        cfg->width > 16384 || cfg->height > 16384) return NULL;
    cvp9_synth_t *s = calloc(1, sizeof(*s));
    if (!s) return NULL;
    s->cfg = *cfg;
    vp9_parsed_frame_t *pf = &s->pf;
    pf->mv_grid_width  = (cfg->width + 3) / 4;
    pf->mv_grid_height = (cfg->height + 3) / 4;
    pf->mv_grid = calloc((size_t)pf->mv_grid_width * pf->mv_grid_height, sizeof(cvp9_mv_t));
    pf->mi_grid_width  = (cfg->width + 7) / 8;
    pf->mi_grid_height = (cfg->height + 7) / 8;
    size_t mi = (size_t)pf->mi_grid_width * pf->mi_grid_height;
    pf->mi_width_grid  = calloc(mi, 1);
    pf->mi_height_grid = calloc(mi, 1);
    pf->mi_block_grid  = calloc(mi, sizeof(uint32_t));
    s->blocks_cap = 1024;
    s->coeffs_cap = 1u << 16;
    pf->blocks = malloc(s->blocks_cap * sizeof(vp9_macroblock_info_t));
    pf->coeffs = malloc(s->coeffs_cap * sizeof(int16_t));
    pf->blocks_capacity = s->blocks_cap;
    pf->coeffs_capacity = s->coeffs_cap;
    if (!pf->mv_grid || !pf->mi_width_grid || !pf->mi_height_grid ||
        !pf->mi_block_grid || !pf->blocks || !pf->coeffs) {
        cvp9_synth_destroy(s);
        return NULL;
    }
    return s;
}

void cvp9_synth_destroy(cvp9_synth_t *s)
{
    if (!s) return;
    free(s->pf.blocks);
    free(s->pf.coeffs);
    free(s->pf.mv_grid);
    free(s->pf.mi_width_grid);
    free(s->pf.mi_height_grid);
    free(s->pf.mi_block_grid);
    free(s->tmp_blocks);
    free(s);
}

static int grow_blocks(cvp9_synth_t *s, uint32_t need)
{
    if (need <= s->blocks_cap) return 1;
    uint32_t cap = s->blocks_cap;
    while (cap < need) cap *= 2;
    void *p = realloc(s->pf.blocks, (size_t)cap * sizeof(vp9_macroblock_info_t));
    if (!p) return 0;
    s->pf.blocks = p;
    s->blocks_cap = cap;
    s->pf.blocks_capacity = cap;
    return 1;
}

static int grow_coeffs(cvp9_synth_t *s, uint32_t need)
{
    if (need <= s->coeffs_cap) return 1;
    uint32_t cap = s->coeffs_cap;
    while (cap < need) cap *= 2;
    void *p = realloc(s->pf.coeffs, (size_t)cap * sizeof(int16_t));
    if (!p) return 0;
    s->pf.coeffs = p;
    s->coeffs_cap = cap;
    s->pf.coeffs_capacity = cap;
    return 1;
}

static int max_tx_for(int w, int h)
{
    int m = w < h ? w : h;
    if (m >= 32) return 3;
    if (m >= 16) return 2;
    if (m >= 8) return 1;
    return 0;
}

typedef struct {
    cvp9_synth_t *s;
    rng_t        *r;
    int           is_key;
    int           ok;
} emit_ctx_t;

/* Append the dense coefficients of one block (parser order). */
static void emit_coeffs(emit_ctx_t *e, vp9_macroblock_info_t *b)
{
    cvp9_synth_t *s = e->s;
    const cvp9_synth_config_t *c = &s->cfg;
    vp9_parsed_frame_t *pf = &s->pf;
    rng_t *r = e->r;

    int mi_cols = (int)(c->width + 7) >> 3;
    int mi_rows = (int)(c->height + 7) >> 3;
    int mi_col = b->x >> 3, mi_row = b->y >> 3;
    int sub8 = b->width < 8 || b->height < 8;
    int ew = sub8 ? 8 : b->width, eh = sub8 ? 8 : b->height;

    double density = c->density_min;
    if (c->density_max > c->density_min)
        density += (c->density_max - c->density_min) * rng_unit(r);
    uint32_t thresh = (uint32_t)(density * 4294967296.0 > 4294967295.0 ? 4294967295.0
                                                                         : density * 4294967296.0);
    int max_eob = 0;

    for (int plane = 0; plane < 3; plane++) {
        int ss = plane > 0;
        int pw = ss ? ew / 2 : ew, ph = ss ? eh / 2 : eh;
        if (pw < 4) pw = 4;
        if (ph < 4) ph = 4;
        int tx = b->tx_size;
        if (ss) {
            int mt = max_tx_for(pw, ph);
            tx = sub8 ? 0 : (tx > mt ? mt : tx);
        }
        int n4w = pw / 4, n4h = ph / 4;
        int txs4 = 1 << tx;
        int origin4x = (mi_col * 2) >> ss, origin4y = (mi_row * 2) >> ss;
        int plane_w4 = (mi_cols * 2) >> ss, plane_h4 = (mi_rows * 2) >> ss;
        int max_w = n4w, max_h = n4h;
        if (origin4x + max_w > plane_w4) max_w = plane_w4 - origin4x;
        if (origin4y + max_h > plane_h4) max_h = plane_h4 - origin4y;
        int n = 4 << tx;
        int area = n * n;
        for (int y4 = 0; y4 < max_h; y4 += txs4) {
            for (int x4 = 0; x4 < max_w; x4 += txs4) {
                if (!grow_coeffs(s, pf->num_coeffs + (uint32_t)area)) { e->ok = 0; return; }
                int16_t *dst = &pf->coeffs[pf->num_coeffs];
                memset(dst, 0, (size_t)area * sizeof(int16_t));
                int last = -1;
                for (int i = 0; i < area; i++) {
                    if (rng_u32(r) >= thresh) continue;
                    int mag = 1 + (int)(c->coeff_scale * rng_exp(r));
                    if (mag > c->coeff_max) mag = c->coeff_max;
                    dst[i] = (int16_t)((rng_next(r) & 1) ? -mag : mag);
                    last = i;
                }
                if (plane == 0 && last + 1 > max_eob) max_eob = last + 1;
                pf->num_coeffs += (uint32_t)area;
            }
        }
    }
    b->eob = (uint16_t)max_eob;
}

static const uint8_t k_modes4[4] = { 0, 1, 2, 9 };

static void emit_block(emit_ctx_t *e, int x, int y, int w, int h)
{
    if (!e->ok) return;
    cvp9_synth_t *s = e->s;
    const cvp9_synth_config_t *c = &s->cfg;
    vp9_parsed_frame_t *pf = &s->pf;
    rng_t *r = e->r;

    if (!grow_blocks(s, pf->num_blocks + 1)) { e->ok = 0; return; }
    vp9_macroblock_info_t *b = &pf->blocks[pf->num_blocks];
    memset(b, 0, sizeof(*b));
    b->x = (uint16_t)x;
    b->y = (uint16_t)y;
    b->width = (uint8_t)w;
    b->height = (uint8_t)h;

    int mt = max_tx_for(w < 8 ? 8 : w, h < 8 ? 8 : h);
    if (w < 8 || h < 8) mt = 0;
    int tx;
    if (c->fixed_tx >= 0) {
        tx = c->fixed_tx > mt ? mt : c->fixed_tx;
    } else {
        int tot = 0;
        for (int i = 0; i <= mt; i++) tot += c->tx_weights[i];
        int pick = tot > 0 ? rng_range(r, 0, tot - 1) : 0;
        tx = 0;
        for (int i = 0; i <= mt; i++) {
            if (pick < c->tx_weights[i]) { tx = i; break; }
            pick -= c->tx_weights[i];
            tx = i;
        }
    }
    b->tx_size = (uint8_t)tx;

    int intra = e->is_key || (c->intra_in_inter > 0 && rng_unit(r) < c->intra_in_inter);
    b->is_intra = (uint8_t)intra;
    if (intra) {
        if (c->all_intra_modes) {
            b->y_mode = (uint8_t)rng_range(r, 0, 9);
            b->uv_mode = (uint8_t)rng_range(r, 0, 9);
        } else {
            b->y_mode = k_modes4[rng_range(r, 0, 3)];
            b->uv_mode = k_modes4[rng_range(r, 0, 3)];
        }
        b->ref_frame[0] = 0;
    } else {
        b->y_mode = 13;  /* NEWMV-style inter mode index, unused by recon */
        b->uv_mode = 0;
        int nrefs = c->nrefs < 1 ? 1 : (c->nrefs > 3 ? 3 : c->nrefs);
        b->ref_frame[0] = (uint8_t)rng_range(r, 1, nrefs);
        int range8 = c->mv_range_px * 8;
        b->mv[0][0] = (int16_t)rng_range(r, -range8, range8);
        b->mv[0][1] = (int16_t)rng_range(r, -range8, range8);
    }
    b->ref_frame[1] = 0;
    if (!intra && c->compound_prob > 0 && rng_unit(r) < c->compound_prob) {
        /* second reference: another of LAST/GOLDEN/ALTREF, its own MV */
        int second = rng_range(r, 1, 2);
        b->ref_frame[1] = (uint8_t)(1 + (b->ref_frame[0] - 1 + second) % 3);
        int range8 = c->mv_range_px * 8;
        b->mv[1][0] = (int16_t)rng_range(r, -range8, range8);
        b->mv[1][1] = (int16_t)rng_range(r, -range8, range8);
    }
    b->skip = (uint8_t)(c->skip_prob > 0 && rng_unit(r) < c->skip_prob);
    b->coeff_offset = pf->num_coeffs;

    if (!intra) {
        int gx0 = x / 4, gy0 = y / 4;
        int bw_mi = w / 8 ? w / 8 : 1, bh_mi = h / 8 ? h / 8 : 1;
        int gx1 = gx0 + bw_mi * 2, gy1 = gy0 + bh_mi * 2;
        if (gx1 > (int)pf->mv_grid_width) gx1 = (int)pf->mv_grid_width;
        if (gy1 > (int)pf->mv_grid_height) gy1 = (int)pf->mv_grid_height;
        for (int gy = gy0; gy < gy1; gy++)
            for (int gx = gx0; gx < gx1; gx++) {
                cvp9_mv_t *g = &pf->mv_grid[(size_t)gy * pf->mv_grid_width + gx];
                g->x = b->mv[0][0];
                g->y = b->mv[0][1];
                g->ref = b->ref_frame[0] - 1;
                g->pad = 0;
            }
    }

    if (!b->skip) emit_coeffs(e, b);
    pf->num_blocks++;
}

/* Recursive VP9-style partition of the square at (x, y) of size sz. */
static void partition(emit_ctx_t *e, int x, int y, int sz)
{
    if (!e->ok) return;
    const cvp9_synth_config_t *c = &e->s->cfg;
    int W = (int)c->width, H = (int)c->height;
    if (x >= W || y >= H) return;
    rng_t *r = e->r;

    int half = sz / 2;
    int has_rows = (y + half) < H;
    int has_cols = (x + half) < W;

    if (sz == 8) {
        if (c->min_bsize <= 4 && rng_range(r, 0, 3) == 0) {
            /* sub-8x8: the parser emits one block per MI, width/height 4..8 */
            int kind = rng_range(r, 0, 2);
            emit_block(e, x, y, kind == 2 ? 8 : 4, kind == 1 ? 8 : 4);
        } else {
            emit_block(e, x, y, 8, 8);
        }
        return;
    }

    /* choose NONE / HORZ / VERT / SPLIT */
    int choice;  /* 0 none, 1 horz, 2 vert, 3 split */
    if (c->fixed_bsize) {
        choice = sz > c->fixed_bsize ? 3 : 0;
        if (choice == 0 && (!has_rows || !has_cols)) choice = 3;
    } else if (sz > c->max_bsize) {
        choice = 3;
    } else {
        /* levels left below this size down to min leaf 8 */
        int levels = 0;
        for (int t = sz; t > 8; t >>= 1) levels++;
        /* stop here with prob 1/(levels+1): leaf depth uniform over sizes */
        if (rng_range(r, 0, levels) == 0) {
            choice = 0;
            if (c->rect_partitions) {
                int k = rng_range(r, 0, 2);
                choice = k;  /* none, horz or vert */
            }
        } else {
            choice = 3;
        }
        if (!has_rows && !has_cols) choice = 3;
        else if (!has_rows && choice != 3) choice = c->rect_partitions ? 1 : 3;
        else if (!has_cols && choice != 3) choice = c->rect_partitions ? 2 : 3;
    }

    switch (choice) {
    case 0:
        emit_block(e, x, y, sz, sz);
        break;
    case 1:
        emit_block(e, x, y, sz, half);
        if (has_rows) emit_block(e, x, y + half, sz, half);
        break;
    case 2:
        emit_block(e, x, y, half, sz);
        if (has_cols) emit_block(e, x + half, y, half, sz);
        break;
    default:
        partition(e, x, y, half);
        partition(e, x + half, y, half);
        partition(e, x, y + half, half);
        partition(e, x + half, y + half, half);
        break;
    }
}

const vp9_parsed_frame_t *cvp9_synth_frame(cvp9_synth_t *s, int index)
{
    if (!s || index < 0) return NULL;
    const cvp9_synth_config_t *c = &s->cfg;
    vp9_parsed_frame_t *pf = &s->pf;

    rng_t r;
    rng_seed(&r, c->seed, (uint64_t)index + 1);

    int is_key = (index == 0) || (c->gop > 0 && index % c->gop == 0);

    pf->num_blocks = 0;
    pf->num_coeffs = 0;
    memset(pf->mv_grid, 0, (size_t)pf->mv_grid_width * pf->mv_grid_height * sizeof(cvp9_mv_t));

    vp9_frame_header_t *h = &pf->hdr;
    memset(h, 0, sizeof(*h));
    h->frame_type = is_key ? VP9_FRAME_KEY : VP9_FRAME_NON_KEY;
    h->width = c->width;
    h->height = c->height;
    h->render_width = c->width;
    h->render_height = c->height;
    h->profile = 0;
    h->bit_depth = 8;
    h->subsampling_x = 1;
    h->subsampling_y = 1;
    h->show_frame = true;
    h->refresh_frame_context = true;
    h->log2_tile_cols = (uint8_t)(c->log2_tile_cols > 0 ? c->log2_tile_cols : 0);
    h->base_qindex = (int16_t)c->qindex;
    h->filter_level = (uint8_t)(c->lf_level >= 0 ? c->lf_level : rng_range(&r, 0, 63));
    h->sharpness_level = (uint8_t)c->sharpness;
    h->interp_filter = (vp9_interp_filter_t)(c->interp_filter >= 0 ? c->interp_filter
                                                                    : rng_range(&r, 0, 2));
    if (is_key) {
        h->refresh_frame_flags = 0xFF;
    } else {
        uint8_t f = 0x01;
        int rel = c->gop > 0 ? index % c->gop : index;
        if (c->golden_every > 0 && rel % c->golden_every == 0) f |= 0x02;
        if (c->altref_every > 0 && rel % c->altref_every == 0) f |= 0x04;
        h->refresh_frame_flags = f;
    }
    h->ref_frame_idx[0] = 0;
    h->ref_frame_idx[1] = 1;
    h->ref_frame_idx[2] = 2;

    emit_ctx_t e = { s, &r, is_key, 1 };
    int sb_cols = (int)(c->width + 63) / 64;
    int sb_rows = (int)(c->height + 63) / 64;
    int tile_cols = 1 << (c->log2_tile_cols > 0 ? c->log2_tile_cols : 0);
    if (tile_cols > sb_cols) tile_cols = sb_cols;

    /* Tile columns are emitted one after another (each tile's SBs in raster
     * order), which is the order the tile merge produces. */
    for (int t = 0; t < tile_cols && e.ok; t++) {
        int c0 = (t * sb_cols) / tile_cols;
        int c1 = ((t + 1) * sb_cols) / tile_cols;
        for (int row = 0; row < sb_rows && e.ok; row++)
            for (int col = c0; col < c1 && e.ok; col++)
                partition(&e, col * 64, row * 64, 64);
    }
    return e.ok ? pf : NULL;
}
