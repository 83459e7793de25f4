/*
 * batch.c — multi-stream reconstruction engine (include/cvp9_batch.h).
 *
 * Three CUDA streams: inputs go up on `hs`, kernels run on `cs`, outputs
 * come down on `ds`, so step n+1's upload and step n-1's download overlap
 * step n's kernels. Two step slots hold the per-step staging (pinned
 * inputs, device inputs, job table, SB scratch, tickets, statuses, cached
 * graph); a slot is reused only after the step that last used it is done.
 *
 * Per stream the engine keeps the reference pool on the device (up to 12
 * frame buffers; refs are pointer swaps) and its SB done flags, whose epoch
 * advances every frame so they never need clearing.
 *
 * Nothing on the submit or admission path calls the driver's allocator:
 * device and pinned host buffers are carved from two chunked arenas
 * (arena.h). A stream's buffers are released when a closed slot is recycled
 * (its last step is complete by then) and a step slot's when they are
 * outgrown (after the slot's previous step completed).
 */
#include "cvp9_batch.h"
#include "backend_common.h"
#include "recon_launch.h"
#include "arena.h"

#include <cuda_runtime_api.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define BSLOTS 3
#define MAXF 12
/* steps of at least this many frames send their inputs as one staged copy
 * (smaller steps have few copies, and a serving step's submit latency
 * counts: staging took a 9-frame step's submit from 0.3 to 1.1 ms) */
#define COALESCE_MIN_FRAMES 32
/* Page-locked output areas (step q downloads into area q % OUTR), and the
 * records each stream keeps of where its recent frames landed: up to two
 * other steps in flight holding the stream, the two newest completed
 * frames, and the new one. */
#define OUTR (BSLOTS + 2)
#define WAIT_LIMIT_S 60.0
#define ALIGN_UP(x, a) (((x) + (a) - 1) / (a) * (a))
#define LAT_RING 4096
#define PACK_AUTO_BYTES (64ull << 20)   /* dense coefficient bytes from which a step packs */

typedef struct {
    uint8_t *dev;
    size_t   cap;
    int32_t  w, h;
    int      users;
    uint64_t d2h_seq;          /* last step whose download reads this frame */
} bframe_t;

typedef struct {
    int       open;
    int32_t   W, H;
    int       n_sb;
    uint32_t *d_sb_done;
    uint32_t *d_mi_map;         /* FULL loop filter: mode info per 8x8 MI   */
    size_t    mi_cap;           /* its entries                              */
    uint32_t  epoch;
    bframe_t  f[MAXF];
    int       ref_slot[8];
    uint64_t  reserved;
    /* the stream's frames of its recent steps: where each landed in the
     * engine's per-step output areas */
    uint8_t  *h_out[OUTR];        /* planes in output area out_area[k]         */
    int       out_area[OUTR];
    int32_t   out_w[OUTR], out_h[OUTR];
    int64_t   out_pts[OUTR];
    uint64_t  out_seq[OUTR];      /* step that downloads into it, 0 none       */
    uint32_t  out_status[OUTR];   /* that step's status word for this stream   */
    int       latest;           /* output buffer of the newest step, -1 none */
    uint64_t  last_seq;         /* newest step that included this stream     */
    uint32_t  last_status;
    int       sb_cap;           /* capacity of d_sb_done (SBs)               */
} bstream_t;

struct cvp9_batch;
typedef struct { struct cvp9_batch *b; uint64_t seq; } lat_arg_t;

/* A frame's host inputs in the step's device buffer: arrays k = blocks,
 * dense coefficients, list positions, list values, packed coefficients. */
enum { IN_BLOCKS, IN_COEFFS, IN_POS, IN_VAL, IN_PACKED, IN_N };
typedef struct {
    size_t      at[IN_N];  /* byte offsets in d_in */
    const void *gsrc;      /* REFCPU gather source: device view of page-locked coefficients */
    unsigned    staged;    /* bit k: array k goes through the pinned staging buffer */
    int         outk;      /* output record of the frame's stream, -1 none */
    size_t      out_off;   /* the frame's offset in the step's output staging and area */
} bfin_t;
typedef struct { const void *src; size_t off, n; } bdirect_t;

typedef struct {
    uint64_t        seq;
    int             busy;
    lat_arg_t       lat_arg;     /* completion-callback argument of this slot */
    cudaEvent_t     ev_start, ev_h2d, ev_k0, ev_k1, ev_end;
    cudaEvent_t     ev_cb;       /* after the completion callback: slot reuse waits on it */
    cudaEvent_t     ev_kern[4];
    uint8_t        *h_in;   size_t h_in_cap;
    uint32_t       *h_pack; size_t h_pack_cap;     /* packed coefficients (pinned) */
    bfin_t         *fin; bdirect_t *direct;        /* per frame / per array of the step */
    bdirect_t      *stg; int stg_cap;              /* pieces copied into h_in on the host pool */
    uint8_t        *d_out; size_t d_out_cap;       /* the step's frames side by side (device) */
    size_t          out_total;                     /* their bytes, 256-aligned each */
    int64_t        *pk_words; size_t *pk_off;     /* packed words (-1: not packed), offset in h_pack */
    int             fin_cap;
    uint32_t        packed;                     /* frames uploaded packed */
    uint8_t        *d_in;   size_t d_in_cap;
    cvp9_job_t     *h_jobs; cvp9_job_t *d_jobs; int jobs_cap;
    uint32_t       *d_sb_range; size_t sb_cap;      /* uint32 entries */
    uint32_t       *d_misc; uint32_t *h_misc; int misc_cap;  /* [0] tickets, [1+i] status, [n+1] gathered
                                                     * bytes, [n+2+i] malformed packed frame i */
    uint32_t       *d_tickets; size_t tickets_cap; uint32_t n_tickets; uint64_t tickets_key;
    uint32_t       *h_tickets; size_t h_tickets_cap;
    uint32_t       *d_fast; size_t fast_cap;    /* inter fast path: flags, tickets, count */
    int             tune_idx;                   /* tuner bucket this step measures, -1 none */
    cvp9_tcfg_t     tune_cfg;
    size_t          h_jobs_bytes, d_jobs_bytes, h_misc_bytes, d_misc_bytes;
    cudaGraphExec_t graph; uint64_t graph_key;
    int             n;
    int            *sids;  int sids_cap;
    uint64_t        h2d_bytes, d2h_bytes;
    uint32_t        launches;
    uint32_t        launches_extra;  /* upload-stream kernels of the step */
} bslot_t;

struct cvp9_batch {
    int          device, arith, use_graphs, max_streams;
    int          gather;     /* REFCPU: luma-only coefficient upload by kernel */
    int          pack;       /* host coefficient packing: -1 never, 0 large steps, 1 always */
    int          pack_q;     /* large steps: frames packed, in 16ths of the step (0..16) */
    int          pack_fixed; /* $CVP9_PACK_SHARE=0..16 pins pack_q (-1: the feedback sets it) */
    cvp9_tuner_t tuner;      /* kernel configuration per shape bucket */
    uint64_t     budget, reserved;
    cudaStream_t cs, hs, ds;
    bstream_t   *st;
    int          nst;
    bslot_t      slot[BSLOTS];
    uint64_t     seq;        /* steps submitted */
    uint64_t     done_seq;   /* every step <= done_seq is complete */
    int          graph_replays;
    int          coalesce;   /* stage page-locked inputs of large steps: 1 always, 0 never,
                              * -1 when the step packs nothing ($CVP9_COALESCE) */
    int          collect;    /* download a step's frames in one copy ($CVP9_DL_COLLECT=0: one each) */
    int          resident_ctas;
    int          lf_full_ctas;   /* k_lf_full CTAs resident on the device */
    cudaEvent_t  ev_t0, ev_t1;
    /* host-clock submit and completion time of recent steps */
    double       lat_submit[LAT_RING];
    volatile double lat_done[LAT_RING];
    uint64_t     lat_seq[LAT_RING];
    /* device timeline of recent steps, ms after the timer's start event:
     * upload start, upload end, kernels start, kernels end, download end */
    float        tl[LAT_RING][5];
    /* per-step output areas (page-locked): step q downloads its frames into
     * area q % OUTR in one copy; area_seq says which step's frames it holds */
    uint8_t     *h_area[OUTR];
    size_t       h_area_cap[OUTR];
    uint64_t     area_seq[OUTR];
    size_t       out_reserve;  /* output bytes of one step the reservations cover */
    uint64_t     tl_seq[LAT_RING];
    int          t0_set;
    float        submit_pack_ms, submit_wait_ms;   /* the last submit's host time */
    float        submit_stage_ms;
    cvp9_batch_stats_t last;
    arena_t      dev;        /* device buffers: frames, flags, step inputs      */
    arena_t      pin;        /* pinned host buffers: downloads, job tables      */
    char         err[192];
};

static cvp9_err_t bfail(cvp9_batch_t *b, cudaError_t e, const char *what)
{
    snprintf(b->err, sizeof(b->err), "%s: %s", what, cudaGetErrorString(e));
    return CVP9_ERR_GPU;
}

#define BCK(call, what) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) return bfail(b, e_, what); } while (0)

static size_t frame_bytes(int32_t w, int32_t h)
{
    return (size_t)w * h + 2 * (size_t)((w + 1) / 2) * ((h + 1) / 2);
}

uint64_t cvp9_batch_stream_bytes(uint32_t w, uint32_t h)
{
    /* reference frames (LAST, GOLDEN, ALTREF, a stale key frame), the frame
     * being written, two whose downloads are in flight; SB flags; per-step
     * buffers x BSLOTS: the dense coefficient array (2 bytes per sample), its
     * packed form (at most as large), the blocks and the output staging */
    uint64_t fb = frame_bytes((int32_t)w, (int32_t)h);
    uint64_t nsb = (uint64_t)((w + 63) / 64) * ((h + 63) / 64);
    return 7 * fb + nsb * 20 + BSLOTS * (5 * fb + (uint64_t)((w + 7) / 8) * ((h + 7) / 8) * 32);
}

cvp9_err_t cvp9_batch_create(const cvp9_batch_config_t *cfg, cvp9_batch_t **out)
{
    if (!out) return CVP9_ERR_INVALID_DATA;
    *out = NULL;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return CVP9_ERR_NO_BACKEND;
    cvp9_batch_t *b = calloc(1, sizeof(*b));
    if (!b) return CVP9_ERR_NOMEM;
    b->device = (cfg && cfg->device >= 0) ? cfg->device : cvp9_env_device();
    b->arith = (cfg && cfg->arith >= 0) ? (cfg->arith == 2 ? CVP9_ARITH_FULL : cfg->arith ? CVP9_ARITH_SPEC
                                                                                : CVP9_ARITH_REFCPU)
                                        : cvp9_env_arith();
    b->budget = (cfg && cfg->hbm_budget) ? cfg->hbm_budget : 150ull * 1000 * 1000 * 1000;
    b->max_streams = (cfg && cfg->max_streams > 0) ? cfg->max_streams : 1024;
    b->use_graphs = cfg ? cfg->use_graphs : 1;
    b->gather = b->arith == CVP9_ARITH_REFCPU && cvp9_env_gather();
    {
        const char *e = getenv("CVP9_COALESCE");
        b->coalesce = (e && e[0] == '1') ? 1 : (e && e[0] == '0') ? 0 : -1;
        e = getenv("CVP9_DL_COLLECT");
        b->collect = !(e && e[0] == '0');
    }
    b->pack = cvp9_env_pack(cfg ? cfg->pack : 0);
    b->pack_q = 16;
    {
        const char *e = getenv("CVP9_PACK_SHARE");
        b->pack_fixed = (e && *e) ? atoi(e) : -1;
        if (b->pack_fixed > 16) b->pack_fixed = 16;
        if (b->pack_fixed >= 0) b->pack_q = b->pack_fixed;
    }
    {
        cvp9_tcfg_t fixed = { (int8_t)cvp9_env_inter_fast(), 0, 0 };
        cvp9_tuner_init(&b->tuner, b->arith, cfg && cfg->autotune && cvp9_env_autotune(), fixed);
    }
    if (b->device >= ndev || cvp9_device_setup(b->device) != 0) { free(b); return CVP9_ERR_NO_BACKEND; }
    b->st = calloc((size_t)b->max_streams, sizeof(bstream_t));
    if (!b->st) { free(b); return CVP9_ERR_NOMEM; }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    b->resident_ctas = sms * cvp9_recon_ctas_per_sm(b->device, b->arith);
    b->lf_full_ctas = sms * cvp9_lf_full_ctas_per_sm(b->device);
    {
        /* chunk sizes scale with the budget: 2 GB device / 256 MB pinned at
         * the 150 GB default; the first chunk of each is taken now */
        uint64_t dc = b->budget / 64, hc = b->budget / 512;
        b->dev.host = 0;
        b->dev.chunk_min = dc < (64ull << 20) ? (64ull << 20) : dc > (2ull << 30) ? (2ull << 30) : dc;
        b->pin.host = 1;
        b->pin.chunk_min = hc < (16ull << 20) ? (16ull << 20) : hc > (256ull << 20) ? (256ull << 20) : hc;
        void *p0 = arena_alloc(&b->dev, 1), *p1 = arena_alloc(&b->pin, 1);
        if (!p0 || !p1) {
            cvp9_batch_destroy(b);
            return CVP9_ERR_NOMEM;
        }
        arena_free(&b->dev, p0, 1);
        arena_free(&b->pin, p1, 1);
    }
    if (cudaStreamCreateWithFlags(&b->cs, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->hs, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->ds, cudaStreamNonBlocking) != cudaSuccess) {
        cvp9_batch_destroy(b);
        return CVP9_ERR_GPU;
    }
    for (int i = 0; i < BSLOTS; i++) {
        bslot_t *s = &b->slot[i];
        if (cudaEventCreate(&s->ev_start) != cudaSuccess || cudaEventCreate(&s->ev_h2d) != cudaSuccess ||
            cudaEventCreate(&s->ev_k0) != cudaSuccess || cudaEventCreate(&s->ev_k1) != cudaSuccess ||
            cudaEventCreate(&s->ev_end) != cudaSuccess || cudaEventCreate(&s->ev_kern[0]) != cudaSuccess ||
            cudaEventCreate(&s->ev_kern[1]) != cudaSuccess || cudaEventCreate(&s->ev_kern[2]) != cudaSuccess ||
            cudaEventCreate(&s->ev_kern[3]) != cudaSuccess || cudaEventCreate(&s->ev_cb) != cudaSuccess) {
            cvp9_batch_destroy(b);
            return CVP9_ERR_GPU;
        }
    }
    if (cudaEventCreate(&b->ev_t0) != cudaSuccess || cudaEventCreate(&b->ev_t1) != cudaSuccess) {
        cvp9_batch_destroy(b);
        return CVP9_ERR_GPU;
    }
    *out = b;
    return CVP9_OK;
}

/* Release a stream slot's buffers (its last step is complete). */
static void free_stream(cvp9_batch_t *b, bstream_t *s)
{
    for (int i = 0; i < MAXF; i++) arena_free(&b->dev, s->f[i].dev, s->f[i].cap);
    arena_free(&b->dev, s->d_sb_done, (size_t)s->sb_cap * 4);
    arena_free(&b->dev, s->d_mi_map, s->mi_cap * 4);
    memset(s, 0, sizeof(*s));
}

void cvp9_batch_destroy(cvp9_batch_t *b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->cs) cudaStreamSynchronize(b->cs);
    if (b->hs) cudaStreamSynchronize(b->hs);
    if (b->ds) cudaStreamSynchronize(b->ds);
    for (int i = 0; i < BSLOTS; i++) {
        bslot_t *s = &b->slot[i];
        if (s->graph) cudaGraphExecDestroy(s->graph);
        if (s->ev_start) cudaEventDestroy(s->ev_start);
        if (s->ev_h2d) cudaEventDestroy(s->ev_h2d);
        if (s->ev_k0) cudaEventDestroy(s->ev_k0);
        if (s->ev_k1) cudaEventDestroy(s->ev_k1);
        if (s->ev_end) cudaEventDestroy(s->ev_end);
        if (s->ev_cb) cudaEventDestroy(s->ev_cb);
        for (int k = 0; k < 4; k++) if (s->ev_kern[k]) cudaEventDestroy(s->ev_kern[k]);
        free(s->sids);
        free(s->fin);
        free(s->direct);
        free(s->stg);
        free(s->pk_words);
        free(s->pk_off);
    }
    /* every stream and slot buffer lives in the arenas; the streams were
     * synchronised above */
    arena_destroy(&b->dev);
    arena_destroy(&b->pin);
    free(b->st);
    if (b->ev_t0) cudaEventDestroy(b->ev_t0);
    if (b->ev_t1) cudaEventDestroy(b->ev_t1);
    if (b->cs) cudaStreamDestroy(b->cs);
    if (b->hs) cudaStreamDestroy(b->hs);
    if (b->ds) cudaStreamDestroy(b->ds);
    free(b);
}

int cvp9_batch_open_stream(cvp9_batch_t *b, uint32_t w, uint32_t h)
{
    if (!b || w == 0 || h == 0 || w > 65535 || h > 65535) return CVP9_ERR_INVALID_DATA;
    uint64_t need = cvp9_batch_stream_bytes(w, h);
    if (b->reserved + need > b->budget) return CVP9_ERR_NOMEM;
    /* prefer a closed slot whose buffers can be reused as they are */
    int sid = -1, fresh = -1;
    const int n_sb = (int)(((w + 63) / 64) * ((h + 63) / 64));
    const size_t fb_need = frame_bytes((int32_t)w, (int32_t)h);
    for (int i = 0; i < b->max_streams; i++) {
        bstream_t *c = &b->st[i];
        if (c->open) continue;
        /* smallest closed slot whose buffers fit */
        if (c->d_sb_done && c->sb_cap >= n_sb && (sid < 0 || c->sb_cap < b->st[sid].sb_cap)) sid = i;
        if (fresh < 0 && !c->d_sb_done) fresh = i;
    }
    if (sid < 0) sid = fresh;
    if (sid < 0) {   /* every free slot holds buffers of another size: recycle one */
        for (int i = 0; i < b->max_streams; i++) if (!b->st[i].open) { sid = i; break; }
        if (sid < 0) return CVP9_ERR_NOMEM;
        free_stream(b, &b->st[sid]);
    }
    bstream_t *s = &b->st[sid];
    if (cudaSetDevice(b->device) != cudaSuccess) return CVP9_ERR_GPU;
    /* frames too small for this stream are released now, while idle, so
     * that acquire_frame only ever fills empty entries */
    for (int i = 0; i < MAXF; i++)
        if (s->f[i].dev && s->f[i].cap < fb_need) {
            arena_free(&b->dev, s->f[i].dev, s->f[i].cap);
            s->f[i].dev = NULL;
            s->f[i].cap = 0;
        }
    if (!s->d_sb_done || s->sb_cap < n_sb) {
        arena_free(&b->dev, s->d_sb_done, (size_t)s->sb_cap * 4);
        s->d_sb_done = (uint32_t *)arena_alloc(&b->dev, (size_t)n_sb * 4);
        s->sb_cap = s->d_sb_done ? n_sb : 0;
        if (!s->d_sb_done) {
            free_stream(b, s);
            return CVP9_ERR_NOMEM;
        }
    }
    /* flags are compared against a per-stream epoch: start from zero */
    if (cudaMemsetAsync(s->d_sb_done, 0, (size_t)n_sb * 4, b->cs) != cudaSuccess) {
        free_stream(b, s);
        return CVP9_ERR_NOMEM;
    }
    if (b->arith == CVP9_ARITH_FULL) {
        const size_t nmi = (size_t)((w + 7) / 8) * ((h + 7) / 8);
        if (s->mi_cap < nmi) {
            arena_free(&b->dev, s->d_mi_map, s->mi_cap * 4);
            s->d_mi_map = (uint32_t *)arena_alloc(&b->dev, nmi * 4);
            s->mi_cap = s->d_mi_map ? nmi : 0;
            if (!s->d_mi_map) {
                free_stream(b, s);
                return CVP9_ERR_NOMEM;
            }
        }
        /* entries carry the frame epoch, which restarts with the stream */
        if (cudaMemsetAsync(s->d_mi_map, 0, nmi * 4, b->cs) != cudaSuccess) {
            free_stream(b, s);
            return CVP9_ERR_NOMEM;
        }
    }
    s->W = (int32_t)w;
    s->H = (int32_t)h;
    s->n_sb = n_sb;
    s->epoch = 0;
    for (int i = 0; i < MAXF; i++) { s->f[i].users = 0; s->f[i].d2h_seq = 0; }
    for (int k = 0; k < OUTR; k++) { s->out_seq[k] = 0; s->out_status[k] = 0; }
    s->latest = -1;
    s->last_seq = 0;
    s->last_status = 0;
    for (int i = 0; i < 8; i++) s->ref_slot[i] = -1;
    s->latest = -1;
    s->reserved = need;
    s->open = 1;
    b->reserved += need;
    if (sid + 1 > b->nst) b->nst = sid + 1;
    return sid;
}

static int stream_busy(cvp9_batch_t *b, const bstream_t *s)
{
    return s->last_seq > b->done_seq;
}

static cvp9_err_t wait_slot(cvp9_batch_t *b, bslot_t *s);

cvp9_err_t cvp9_batch_close_stream(cvp9_batch_t *b, int sid)
{
    if (!b || sid < 0 || sid >= b->max_streams || !b->st[sid].open) return CVP9_ERR_INVALID_DATA;
    bstream_t *s = &b->st[sid];
    /* wait for the steps up to this stream's last one only; later steps
     * keep running */
    for (uint64_t q = b->done_seq + 1; stream_busy(b, s) && q <= s->last_seq; q++) {
        bslot_t *o = &b->slot[q % BSLOTS];
        if (o->seq != q) continue;
        cvp9_err_t e = wait_slot(b, o);
        if (e == CVP9_ERR_GPU) return e;
    }
    b->reserved -= s->reserved;
    /* keep the device buffers for the next admitted stream */
    s->open = 0;
    s->reserved = 0;
    for (int i = 0; i < 8; i++) s->ref_slot[i] = -1;
    for (int i = 0; i < MAXF; i++) s->f[i].users = 0;
    return CVP9_OK;
}

/* Per-slot buffers grow with 50% headroom; the slot's previous step is
 * complete when they do, so the old range is idle. */
static cvp9_err_t grow_dev(cvp9_batch_t *b, void **p, size_t *cap, size_t need)
{
    if (arena_grow(&b->dev, p, cap, need) != 0) {
        snprintf(b->err, sizeof(b->err), "device arena: no memory for %zu bytes", need);
        return CVP9_ERR_NOMEM;
    }
    return CVP9_OK;
}

static cvp9_err_t grow_host(cvp9_batch_t *b, void **p, size_t *cap, size_t need)
{
    if (arena_grow(&b->pin, p, cap, need) != 0) {
        snprintf(b->err, sizeof(b->err), "pinned arena: no memory for %zu bytes", need);
        return CVP9_ERR_NOMEM;
    }
    return CVP9_OK;
}

/* A frame buffer of stream s with no reference user; if its last download
 * may still be running, the compute stream waits for it. */
static int acquire_frame(cvp9_batch_t *b, bstream_t *s)
{
    size_t need = frame_bytes(s->W, s->H);
    /* an allocated frame whose download is done, else one still being
     * downloaded (the kernels then wait for that download), else a new one */
    int pick = -1, busy = -1, fresh = -1;
    for (int i = 0; i < MAXF; i++) {
        if (s->f[i].users) continue;
        if (s->f[i].dev && s->f[i].cap >= need) {
            if (s->f[i].d2h_seq <= b->done_seq) { pick = i; break; }
            if (busy < 0) busy = i;
        } else if (!s->f[i].dev && fresh < 0) {
            fresh = i;
        }
    }
    if (pick < 0) pick = fresh >= 0 ? fresh : busy;
    if (pick < 0) return -1;
    bframe_t *f = &s->f[pick];
    if (f->d2h_seq > b->done_seq) {
        /* a step still in flight downloads it */
        bslot_t *o = &b->slot[f->d2h_seq % BSLOTS];
        if (o->seq == f->d2h_seq) cudaStreamWaitEvent(b->cs, o->ev_end, 0);
    }
    if (!f->dev) {
        /* open_stream released every entry smaller than this stream's frames */
        f->dev = (uint8_t *)arena_alloc(&b->dev, need);
        if (!f->dev) return -1;
        f->cap = need;
    }
    f->w = s->W;
    f->h = s->H;
    return pick;
}

static void set_ref(bstream_t *s, int slot, int frame)
{
    if (s->ref_slot[slot] >= 0) s->f[s->ref_slot[slot]].users--;
    s->ref_slot[slot] = frame;
    if (frame >= 0) s->f[frame].users++;
}

static uint64_t mix64(uint64_t h, uint64_t v)
{
    h ^= v + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
    return h * 0xBF58476D1CE4E5B9ull;
}

/* Status word of job i of a completed slot; a malformed packed upload
 * (job i's own unpack error word) reads as a bad block. */
static uint32_t slot_status(const bslot_t *s, int i)
{
    uint32_t st = s->h_misc[1 + i];
    if (s->h_misc[s->n + 2 + i]) st |= CVP9_JOB_BAD_BLOCK;
    return st;
}

static void complete_slot(cvp9_batch_t *b, bslot_t *s)
{
    float t = 0.f, k = 0.f, u = 0.f;
    cudaEventElapsedTime(&t, s->ev_start, s->ev_end);
    cudaEventElapsedTime(&k, s->ev_k0, s->ev_k1);
    cudaEventElapsedTime(&u, s->ev_start, s->ev_h2d);
    b->last.step_ms = t;
    b->last.kernels_ms = k;
    b->last.h2d_ms = u;
    b->last.h2d_bytes = s->h2d_bytes + s->h_misc[s->n + 1];
    b->last.d2h_bytes = s->d2h_bytes;
    b->last.kernel_launches = s->launches + s->launches_extra;
    b->last.packed_frames = s->packed;
    float a = 0.f, r = 0.f, f = 0.f;
    cudaEventElapsedTime(&a, s->ev_kern[0], s->ev_kern[1]);
    cudaEventElapsedTime(&r, s->ev_kern[1], s->ev_kern[2]);
    cudaEventElapsedTime(&f, s->ev_kern[2], s->ev_kern[3]);
    b->last.scan_ms = a;
    b->last.recon_ms = r;
    b->last.filter_ms = f;
    cvp9_tuner_report(&b->tuner, s->tune_idx, s->tune_cfg, k);
    if (b->t0_set) {
        cudaEvent_t ev[5] = { s->ev_start, s->ev_h2d, s->ev_k0, s->ev_k1, s->ev_end };
        float *tl = b->tl[s->seq % LAT_RING];
        for (int i = 0; i < 5; i++)
            if (cudaEventElapsedTime(&tl[i], b->ev_t0, ev[i]) != cudaSuccess) tl[i] = 0.f;
        b->tl_seq[s->seq % LAT_RING] = s->seq;
    }
    for (int i = 0; i < s->n; i++) {
        bstream_t *st = &b->st[s->sids[i]];
        if (!st->open) continue;
        const uint32_t w = slot_status(s, i);
        if (st->last_seq == s->seq) st->last_status = w;
        for (int k = 0; k < OUTR; k++)
            if (st->out_seq[k] == s->seq) st->out_status[k] = w;
    }
    if (s->seq > b->done_seq) b->done_seq = s->seq;
    s->busy = 0;
}

static cvp9_err_t wait_slot(cvp9_batch_t *b, bslot_t *s)
{
    if (!s->busy) return CVP9_OK;
    double t0 = cvp9_now();
    for (;;) {
        cudaError_t e = cudaEventQuery(s->ev_cb);
        if (e == cudaSuccess) break;
        if (e != cudaErrorNotReady) return bfail(b, e, "step completion");
        if (cvp9_now() - t0 > WAIT_LIMIT_S) {
            snprintf(b->err, sizeof(b->err), "step did not complete within %.0f s", WAIT_LIMIT_S);
            return CVP9_ERR_GPU;
        }
        struct timespec ts = { 0, 20000 };
        nanosleep(&ts, NULL);
    }
    complete_slot(b, s);
    return CVP9_OK;
}

static int is_pinned(const void *p)
{
    struct cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return 0; }
    return a.type == cudaMemoryTypeHost;
}

/* Device address of page-locked host memory (NULL if it is not mapped). */
static const void *mapped_ptr(const void *p)
{
    struct cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return NULL; }
    return a.type == cudaMemoryTypeHost ? a.devicePointer : NULL;
}

/* Entry of the stream's output record for the step being submitted: not
 * one of a step still in flight, and not one of the two newest completed
 * frames. With at most two other steps in flight (the slot being reused has
 * completed) one of the OUTR entries is always free. */
static int pick_out(const cvp9_batch_t *b, const bstream_t *st)
{
    uint64_t n1 = 0, n2 = 0;
    for (int k = 0; k < OUTR; k++) {
        uint64_t q = st->out_seq[k];
        if (!q || q > b->done_seq) continue;
        if (q > n1) { n2 = n1; n1 = q; } else if (q > n2) n2 = q;
    }
    for (int k = 0; k < OUTR; k++) {
        uint64_t q = st->out_seq[k];
        if (q && (q > b->done_seq || q == n1 || q == n2)) continue;
        return k;
    }
    return -1;
}

/* Per-frame bookkeeping of a slot for steps of up to n frames. */
static cvp9_err_t slot_frames(bslot_t *s, int n)
{
    if (s->fin_cap >= n) return CVP9_OK;
    free(s->fin);
    free(s->direct);
    free(s->pk_words);
    free(s->pk_off);
    s->fin = malloc((size_t)n * sizeof(bfin_t));
    s->direct = malloc((size_t)n * IN_N * sizeof(bdirect_t));
    s->pk_words = malloc((size_t)n * sizeof(int64_t));
    s->pk_off = malloc((size_t)n * sizeof(size_t));
    s->fin_cap = (s->fin && s->direct && s->pk_words && s->pk_off) ? n : 0;
    return s->fin_cap ? CVP9_OK : CVP9_ERR_NOMEM;
}

/* Packing runs on the host pool, a task per frame. */
typedef struct {
    int                              arith;
    const vp9_parsed_frame_t *const *pfs;
    uint32_t                        *base;
    const size_t                    *off;
    int64_t                         *words;
} pack_job_t;

static void pack_task(void *ctx, int i)
{
    pack_job_t *j = (pack_job_t *)ctx;
    const vp9_parsed_frame_t *pf = j->pfs[i];
    j->words[i] = pf->num_coeffs ? cvp9_pack_coeffs(j->arith, pf, j->base + j->off[i],
                                                    cvp9_pack_bound_words(pf->num_coeffs))
                                 : -1;
}

/* Staging runs on the host pool too: piece k of the step's staged arrays
 * (src -> h_in + off, at most STAGE_PIECE bytes). */
#define STAGE_PIECE (4u << 20)
typedef struct { uint8_t *h_in; const bdirect_t *pc; } stage_job_t;

static void stage_task(void *ctx, int k)
{
    const stage_job_t *j = (const stage_job_t *)ctx;
    memcpy(j->h_in + j->pc[k].off, j->pc[k].src, j->pc[k].n);
}

static void CUDART_CB step_done_cb(void *p)
{
    lat_arg_t *a = (lat_arg_t *)p;
    a->b->lat_done[a->seq % LAT_RING] = cvp9_now();
}

static cvp9_err_t submit_impl(cvp9_batch_t *b, int n, const int *sids, const vp9_parsed_frame_t *const *pfs,
                              const cvp9_coeff_list_t *lists, const int64_t *pts, uint32_t flags);

cvp9_err_t cvp9_batch_submit(cvp9_batch_t *b, int n, const int *sids,
                             const vp9_parsed_frame_t *const *pfs, const int64_t *pts, uint32_t flags)
{
    return submit_impl(b, n, sids, pfs, NULL, pts, flags);
}

cvp9_err_t cvp9_batch_submit_sparse(cvp9_batch_t *b, int n, const int *sids,
                                    const vp9_parsed_frame_t *const *pfs, const cvp9_coeff_list_t *lists,
                                    const int64_t *pts, uint32_t flags)
{
    if (!lists || (flags & CVP9_BATCH_DEVICE_INPUTS)) return CVP9_ERR_INVALID_DATA;
    return submit_impl(b, n, sids, pfs, lists, pts, flags);
}

static cvp9_err_t submit_impl(cvp9_batch_t *b, int n, const int *sids, const vp9_parsed_frame_t *const *pfs,
                              const cvp9_coeff_list_t *lists, const int64_t *pts, uint32_t flags)
{
    if (!b || n <= 0 || !sids || !pfs) return CVP9_ERR_INVALID_DATA;
    if (cudaSetDevice(b->device) != cudaSuccess) return CVP9_ERR_GPU;
    const int dev_in = (flags & CVP9_BATCH_DEVICE_INPUTS) != 0;
    const int want_out = !(flags & CVP9_BATCH_NO_OUTPUT);

    /* validate */
    for (int i = 0; i < n; i++) {
        int sid = sids[i];
        if (sid < 0 || sid >= b->max_streams || !b->st[sid].open || !pfs[i]) return CVP9_ERR_INVALID_DATA;
        const vp9_parsed_frame_t *pf = pfs[i];
        if ((int32_t)pf->hdr.width != b->st[sid].W || (int32_t)pf->hdr.height != b->st[sid].H)
            return CVP9_ERR_INVALID_DATA;
        if (pf->num_blocks && !pf->blocks) return CVP9_ERR_INVALID_DATA;
        if (lists ? (lists[i].n && (!lists[i].pos || !lists[i].val)) : (pf->num_coeffs && !pf->coeffs))
            return CVP9_ERR_INVALID_DATA;
        for (int j = 0; j < i; j++) if (sids[j] == sid) return CVP9_ERR_INVALID_DATA;
        const char *why = NULL;
        if (!cvp9_frame_supported(b->arith, pf, &why)) {
            snprintf(b->err, sizeof(b->err), "stream %d: %s", sid, why);
            return CVP9_ERR_UNSUPPORTED;
        }
        if (b->arith == CVP9_ARITH_FULL && pf->hdr.frame_type != VP9_FRAME_KEY && !pf->hdr.intra_only)
            for (int k = 0; k < 3; k++) {
                const bstream_t *st = &b->st[sid];
                int f = st->ref_slot[pf->hdr.ref_frame_idx[k] & 7];
                if (f >= 0 && (st->f[f].w != st->W || st->f[f].h != st->H)) {
                    snprintf(b->err, sizeof(b->err), "stream %d: reference of another size "
                             "(scaled motion compensation is not built)", sid);
                    return CVP9_ERR_UNSUPPORTED;
                }
            }
    }

    const uint64_t seq = b->seq + 1;
    bslot_t *s = &b->slot[seq % BSLOTS];
    const double tw0 = cvp9_now();
    const int pipelined = b->seq > b->done_seq;    /* an earlier step still in flight */
    cvp9_err_t err = wait_slot(b, s);
    if (err != CVP9_OK) return err;
    b->lat_submit[seq % LAT_RING] = cvp9_now();
    const double waited_ms = (b->lat_submit[seq % LAT_RING] - tw0) * 1e3;
    b->submit_wait_ms = (float)waited_ms;
    b->submit_pack_ms = 0.f;
    b->submit_stage_ms = 0.f;

    /* sizes */
    const int full = b->arith == CVP9_ARITH_FULL;
    size_t in_bytes = 0, n_sb = 0;
    int max_sbr = 0;
    int max_blocks = 0, max_mi = 0, lf_tx = 0, lf_ty = 0, lf_sx = 0, lf_sy = 0;
    int flat_w = 0, flat_h = 0, flat_nv = 0;
    int maxd = 0, wave = 0;      /* wave: superblocks on the step's widest diagonals */
    uint64_t key = mix64(0, (uint64_t)n);
    for (int i = 0; i < n; i++) {
        const vp9_parsed_frame_t *pf = pfs[i];
        bstream_t *st = &b->st[sids[i]];
        if (!dev_in) {
            in_bytes += ALIGN_UP((size_t)pf->num_blocks * sizeof(vp9_macroblock_info_t), 256);
            in_bytes += ALIGN_UP((size_t)pf->num_coeffs * sizeof(int16_t), 256);
            if (lists)
                in_bytes += ALIGN_UP((size_t)lists[i].n * 4, 256) + ALIGN_UP((size_t)lists[i].n * 2, 256);
        }
        n_sb += (size_t)st->n_sb;
        if ((int)pf->num_blocks > max_blocks) max_blocks = (int)pf->num_blocks;
        int mi = ((st->W + 7) / 8) * ((st->H + 7) / 8);
        if (mi > max_mi) max_mi = mi;
        int tiled = (st->W % 8) != 1 && (st->H % 8) != 1;
        if (tiled) {
            /* both grids; the tuned configuration picks one per step below */
            int tx = (st->W + 4 + 63) / 64, ty = (st->H + 4 + 63) / 64;
            if (tx > lf_tx) lf_tx = tx;
            if (ty > lf_ty) lf_ty = ty;
            if (!(st->W & 3)) {
                int sx = ((st->W + 4 + 7) / 8 + 127) / 128, sy = (st->H + 4 + 15) / 16;
                if (sx > lf_sx) lf_sx = sx;
                if (sy > lf_sy) lf_sy = sy;
            }
        } else {
            if (st->W > flat_w) flat_w = st->W;
            if (st->H > flat_h) flat_h = st->H;
        }
        int d = (st->W + 63) / 64 + (st->H + 63) / 64 - 1;
        if (d > maxd) maxd = d;
        {
            const int sc = (st->W + 63) / 64, sr = (st->H + 63) / 64;
            wave += sc < sr ? sc : sr;
        }
        if ((st->H + 63) / 64 > max_sbr) max_sbr = (st->H + 63) / 64;
        key = mix64(key, ((uint64_t)st->W << 32) | (uint64_t)st->H);
    }

    /* kernel configuration of this step (tuner) */
    cvp9_tcfg_t tc;
    s->tune_idx = cvp9_tuner_pick(&b->tuner, cvp9_tune_key(b->arith, n, (uint64_t)n_sb), n, &tc);
    s->tune_cfg = tc;
    int any_tile = 0, any_strip = 0;

    if ((err = slot_frames(s, n))) return err;

    /* outputs: each frame's place in the step's staging buffer and in the
     * step's output area (taken from the arenas before anything of the step
     * is queued); the area last held step seq - OUTR, long complete */
    s->out_total = 0;
    for (int i = 0; i < n; i++) {
        bstream_t *st = &b->st[sids[i]];
        s->fin[i].outk = -1;
        if (!want_out) continue;
        const int k = pick_out(b, st);
        if (k < 0) {
            snprintf(b->err, sizeof(b->err), "stream %d: no free output record", sids[i]);
            return CVP9_ERR_NOMEM;
        }
        s->fin[i].outk = k;
        s->fin[i].out_off = s->out_total;
        s->out_total += ALIGN_UP(frame_bytes(st->W, st->H), 256);
    }
    if (s->out_total) {
        const int a = (int)(seq % OUTR);
        if ((b->collect && (err = grow_dev(b, (void **)&s->d_out, &s->d_out_cap, s->out_total))) ||
            (err = grow_host(b, (void **)&b->h_area[a], &b->h_area_cap[a], s->out_total)))
            return err;
        b->area_seq[a] = seq;
    }

    /* Large steps of dense host arrays: pack the coefficients on the host
     * pool (the PCIe link, not the host, bounds such a step) */
    int any_packed = 0;
    uint32_t max_pages = 0;
    s->packed = 0;
    for (int i = 0; i < n; i++) s->pk_words[i] = -1;
    if (!dev_in && !lists && b->pack >= 0) {
        size_t cb = 0, tot = 0;
        for (int i = 0; i < n; i++) cb += (size_t)pfs[i]->num_coeffs * 2;
        int npack = 0;
        if (b->pack == 1) {
            npack = n;
        } else if (cb >= PACK_AUTO_BYTES) {
            if (b->pack_fixed < 0) b->pack_q = cvp9_pack_share_update(b->pack_q, pipelined, waited_ms);
            npack = (b->pack_q * n + 8) / 16;
        }
        if (npack) {
            for (int i = 0; i < npack; i++) {
                s->pk_off[i] = tot;
                if (pfs[i]->num_coeffs) tot += ALIGN_UP(cvp9_pack_bound_words(pfs[i]->num_coeffs), 64);
            }
            /* no page-locked room for the packed frames: they go up dense */
            if (tot && grow_host(b, (void **)&s->h_pack, &s->h_pack_cap, tot * 4) == CVP9_OK) {
                pack_job_t pj = { b->arith, pfs, s->h_pack, s->pk_off, s->pk_words };
                const double tp0 = cvp9_now();
                cvp9_parallel_for(npack, pack_task, &pj);
                b->submit_pack_ms = (float)((cvp9_now() - tp0) * 1e3);
            }
            for (int i = 0; i < n; i++) {
                if (s->pk_words[i] < 0) continue;
                any_packed = 1;
                s->packed++;
                in_bytes += ALIGN_UP((size_t)s->pk_words[i] * 4, 256);
                uint32_t np = (uint32_t)(((uint64_t)pfs[i]->num_coeffs + 65535) >> 16);
                if (np > max_pages) max_pages = np;
            }
        }
    }

    /* how each host array travels: the gather kernel (REFCPU coefficients in
     * page-locked memory), direct DMA (page-locked), or the pinned staging
     * buffer (pageable); coefficient regions the device fills get no copy.
     * A step of many frames (COALESCE_MIN_FRAMES) that packed nothing also stages its page-locked
     * block records and list arrays, so that its upload is one large copy:
     * the PCIe link runs both directions at once best for large copies (two
     * of ~100 MB each way move in 3.8 ms together, as 0.8 MB and 3.1 MB
     * pieces in 5.1 ms; a 64x1080p step of coefficient lists 6.4 -> 5.2 ms).
     * A step that packs does not: its host threads already use the host
     * memory bandwidth that the staging copy would take (packed 64x1080p:
     * 6.7 ms unstaged, 8.1 ms staged). $CVP9_COALESCE=0|1 forces either. */
    int any_staged = 0;
    size_t stage_bytes = 0;
    const int coalesce = !dev_in && n >= COALESCE_MIN_FRAMES &&
                         (b->coalesce > 0 || (b->coalesce < 0 && !any_packed));
    for (int i = 0; i < n && !dev_in; i++) {
        const vp9_parsed_frame_t *pf = pfs[i];
        bfin_t *f = &s->fin[i];
        const int packed = s->pk_words[i] >= 0;
        f->gsrc = NULL;
        f->staged = 0;
        if (b->gather && !lists && !packed && pf->num_coeffs && pf->num_blocks) f->gsrc = mapped_ptr(pf->coeffs);
        if (pf->num_blocks && (coalesce || !is_pinned(pf->blocks))) f->staged |= 1u << IN_BLOCKS;
        if (!lists && !packed && !f->gsrc && pf->num_coeffs && !is_pinned(pf->coeffs)) f->staged |= 1u << IN_COEFFS;
        if (lists && lists[i].n && (coalesce || !is_pinned(lists[i].pos))) f->staged |= 1u << IN_POS;
        if (lists && lists[i].n && (coalesce || !is_pinned(lists[i].val))) f->staged |= 1u << IN_VAL;
        if (packed && coalesce) f->staged |= 1u << IN_PACKED;
        any_staged |= f->staged != 0;
        /* the staging buffer holds the staged arrays only (the regions the
         * device fills, and the directly copied arrays, live on the device) */
        const size_t len[IN_N] = { (size_t)pf->num_blocks * sizeof(vp9_macroblock_info_t),
                                   (size_t)pf->num_coeffs * sizeof(int16_t),
                                   lists ? (size_t)lists[i].n * 4 : 0, lists ? (size_t)lists[i].n * 2 : 0,
                                   packed ? (size_t)s->pk_words[i] * 4 : 0 };
        for (int k = 0; k < IN_N; k++)
            if ((f->staged >> k) & 1) stage_bytes += ALIGN_UP(len[k], 256);
    }
    if (!dev_in && in_bytes) {
        if ((any_staged && (err = grow_host(b, (void **)&s->h_in, &s->h_in_cap, stage_bytes))) ||
            (err = grow_dev(b, (void **)&s->d_in, &s->d_in_cap, in_bytes)))
            return err;
    }
    if (s->jobs_cap < n) {
        /* sized for every admitted stream at once, so this happens at most
         * a few times */
        int cap = n > b->nst ? n : b->nst;
        s->jobs_cap = 0;
        if ((err = grow_host(b, (void **)&s->h_jobs, &s->h_jobs_bytes, (size_t)cap * sizeof(cvp9_job_t))) ||
            (err = grow_dev(b, (void **)&s->d_jobs, &s->d_jobs_bytes, (size_t)cap * sizeof(cvp9_job_t))))
            return err;
        s->jobs_cap = cap;
    }
    if (s->misc_cap < 2 * n + 3) {
        int cap = 2 * (n > b->nst ? n : b->nst) + 3;
        s->misc_cap = 0;
        if ((err = grow_host(b, (void **)&s->h_misc, &s->h_misc_bytes, (size_t)cap * 4)) ||
            (err = grow_dev(b, (void **)&s->d_misc, &s->d_misc_bytes, (size_t)cap * 4)))
            return err;
        s->misc_cap = cap;
    }
    if ((err = grow_dev(b, (void **)&s->d_sb_range, &s->sb_cap, n_sb * 16))) return err;
    if ((err = grow_dev(b, (void **)&s->d_fast, &s->fast_cap, (2 * n_sb + 2) * 4))) return err;
    if (s->sids_cap < n) {
        free(s->sids);
        s->sids = malloc((size_t)n * sizeof(int));
        if (!s->sids) return CVP9_ERR_NOMEM;
        s->sids_cap = n;
    }

    /* tickets: SB-diagonal order, streams interleaved on each diagonal */
    if (s->tickets_key != key || !s->d_tickets) {
        size_t need = n_sb * 4;
        if ((err = grow_dev(b, (void **)&s->d_tickets, &s->tickets_cap, need))) return err;
        if ((err = grow_host(b, (void **)&s->h_tickets, &s->h_tickets_cap, need ? need : 4))) return err;
        uint32_t *t = s->h_tickets;
        uint32_t cnt = 0;
        for (int d = 0; d < maxd; d++)
            for (int i = 0; i < n; i++) {
                bstream_t *st = &b->st[sids[i]];
                cnt += (uint32_t)cvp9_tickets_on_diagonal((st->W + 63) / 64, (st->H + 63) / 64, i, d, t + cnt);
            }
        cudaError_t e = cudaMemcpyAsync(s->d_tickets, t, (size_t)cnt * 4, cudaMemcpyHostToDevice, b->hs);
        if (e != cudaSuccess) return bfail(b, e, "tickets");
        s->n_tickets = cnt;
        s->tickets_key = key;
    }

    /* inputs: the staged arrays first, side by side in h_in and up in one
     * copy; then direct DMA of page-locked arrays (the caller's, and the
     * packed frames); regions the device fills (gathered, scattered or
     * unpacked coefficients) get space only */
    s->h2d_bytes = 0;
    BCK(cudaEventRecord(s->ev_start, b->hs), "event");
    int any_gather = 0, ndirect = 0, npieces = 0;
    size_t off = 0, staged_end = 0;
    for (int phase = 0; phase < 2 && !dev_in; phase++) {
        for (int i = 0; i < n; i++) {
            const vp9_parsed_frame_t *pf = pfs[i];
            bfin_t *f = &s->fin[i];
            const int packed = s->pk_words[i] >= 0;
            const void *src[IN_N] = { pf->blocks, pf->coeffs, lists ? lists[i].pos : NULL,
                                      lists ? lists[i].val : NULL, packed ? s->h_pack + s->pk_off[i] : NULL };
            const size_t len[IN_N] = { (size_t)pf->num_blocks * sizeof(vp9_macroblock_info_t),
                                       (size_t)pf->num_coeffs * sizeof(int16_t),
                                       lists ? (size_t)lists[i].n * 4 : 0, lists ? (size_t)lists[i].n * 2 : 0,
                                       packed ? (size_t)s->pk_words[i] * 4 : 0 };
            const int copied[IN_N] = { 1, !(f->gsrc || lists || packed), 1, 1, 1 };
            for (int k = 0; k < IN_N; k++) {
                const int stg = (f->staged >> k) & 1;
                if (stg != (phase == 0)) continue;
                f->at[k] = off;
                if (len[k] && copied[k]) {
                    if (stg) {
                        /* pieces of at most STAGE_PIECE bytes, copied below */
                        const int np = (int)((len[k] + STAGE_PIECE - 1) / STAGE_PIECE);
                        if (npieces + np > s->stg_cap) {
                            int cap = 2 * (npieces + np) + 64;
                            bdirect_t *q = (bdirect_t *)realloc(s->stg, (size_t)cap * sizeof(bdirect_t));
                            if (!q) return CVP9_ERR_NOMEM;
                            s->stg = q;
                            s->stg_cap = cap;
                        }
                        for (size_t o = 0; o < len[k]; o += STAGE_PIECE) {
                            s->stg[npieces].src = (const uint8_t *)src[k] + o;
                            s->stg[npieces].off = off + o;
                            s->stg[npieces].n = len[k] - o < STAGE_PIECE ? len[k] - o : STAGE_PIECE;
                            npieces++;
                        }
                    } else {
                        s->direct[ndirect].src = src[k];
                        s->direct[ndirect].off = off;
                        s->direct[ndirect].n = len[k];
                        ndirect++;
                    }
                }
                off += ALIGN_UP(len[k], 256);
            }
            any_gather |= phase == 1 && f->gsrc != NULL;
        }
        if (phase == 0) staged_end = off;
    }
    if (npieces) {
        stage_job_t sj = { s->h_in, s->stg };
        const double ts0 = cvp9_now();
        cvp9_parallel_for(npieces, stage_task, &sj);
        b->submit_stage_ms = (float)((cvp9_now() - ts0) * 1e3);
    }
    cudaError_t ue = cudaSuccess;
    if (staged_end) {
        ue = cudaMemcpyAsync(s->d_in, s->h_in, staged_end, cudaMemcpyHostToDevice, b->hs);
        s->h2d_bytes += staged_end;
    }
    for (int k = 0; k < ndirect && ue == cudaSuccess; k++) {
        ue = cudaMemcpyAsync(s->d_in + s->direct[k].off, s->direct[k].src, s->direct[k].n,
                             cudaMemcpyHostToDevice, b->hs);
        s->h2d_bytes += s->direct[k].n;
    }
    /* sparse frames: their dense coefficient regions start at zero */
    for (int i = 0; lists && i < n && ue == cudaSuccess; i++)
        if (pfs[i]->num_coeffs)
            ue = cudaMemsetAsync(s->d_in + s->fin[i].at[IN_COEFFS], 0, (size_t)pfs[i]->num_coeffs * 2, b->hs);
    if (ue != cudaSuccess) return bfail(b, ue, "upload inputs");

    /* jobs, outputs, reference pools */
    uint32_t sb_base = 0;
    int out_frame[1024];
    int *ofr = n <= 1024 ? out_frame : malloc((size_t)n * sizeof(int));
    if (!ofr) return CVP9_ERR_NOMEM;
    for (int i = 0; i < n; i++) {
        const vp9_parsed_frame_t *pf = pfs[i];
        bstream_t *st = &b->st[sids[i]];
        int of = acquire_frame(b, st);
        if (of < 0) {
            if (ofr != out_frame) free(ofr);
            return bfail(b, cudaErrorMemoryAllocation, "frame pool");
        }
        ofr[i] = of;
        cvp9_job_t *job = &s->h_jobs[i];
        memset(job, 0, sizeof(*job));
        cvp9_job_geometry(job, pf);
        if (full) {
            cvp9_job_full(job, pf);
            job->mi_map = st->d_mi_map;
            job->lf_tiled = 0;                  /* the VP9 filter replaces the others */
        }
        if (job->lf_tiled && !tc.lf32 && !(st->W & 3)) job->lf_tiled = 2;   /* register strips */
        any_tile |= job->lf_tiled == 1;
        any_strip |= job->lf_tiled == 2;
        const bfin_t *f = &s->fin[i];
        job->blocks = dev_in ? pf->blocks : (const vp9_macroblock_info_t *)(s->d_in + f->at[IN_BLOCKS]);
        job->coeffs = dev_in ? pf->coeffs : (const int16_t *)(s->d_in + f->at[IN_COEFFS]);
        job->out = st->f[of].dev;
        job->nv12 = NULL;
        job->dl = (s->fin[i].outk >= 0 && b->collect) ? s->d_out + s->fin[i].out_off : NULL;
        for (int r = 0; r < 8; r++) {
            int f = st->ref_slot[r];
            if (f >= 0) {
                job->ref[r].plane = st->f[f].dev;
                job->ref[r].w = st->f[f].w;
                job->ref[r].h = st->f[f].h;
            }
        }
        job->coeffs_src = dev_in ? NULL : (const int16_t *)f->gsrc;
        if (lists && lists[i].n) {
            job->sp_pos = (const uint32_t *)(s->d_in + f->at[IN_POS]);
            job->sp_val = (const int16_t *)(s->d_in + f->at[IN_VAL]);
            job->sp_n = lists[i].n;
        }
        if (!dev_in && s->pk_words[i] >= 0) {
            job->packed = (const uint32_t *)(s->d_in + f->at[IN_PACKED]);
            job->packed_words = (uint32_t)s->pk_words[i];
        }
        job->epoch = ++st->epoch;
        job->sb_range = s->d_sb_range + 4 * (size_t)sb_base;
        job->sb_done = st->d_sb_done;
        job->status = s->d_misc + 1 + i;
        sb_base += (uint32_t)st->n_sb;
        s->sids[i] = sids[i];
    }
    BCK(cudaMemcpyAsync(s->d_jobs, s->h_jobs, (size_t)n * sizeof(cvp9_job_t), cudaMemcpyHostToDevice, b->hs),
        "upload jobs");
    s->h2d_bytes += (size_t)n * sizeof(cvp9_job_t);
    /* the counter of gathered bytes and the per-job unpack error words are
     * cleared here, on the upload stream; the compute stream's clear of the
     * status words stops before them */
    BCK(cudaMemsetAsync(s->d_misc + n + 1, 0, (size_t)(n + 1) * 4, b->hs), "clear upload words");
    s->launches_extra = 0;
    if (any_gather) {
        int grc = cvp9k_launch_gather(s->d_jobs, n, max_blocks, s->d_misc + n + 1, b->hs);
        if (grc != 0) return bfail(b, (cudaError_t)grc, "coefficient gather");
        s->launches_extra++;
    }
    if (lists) {
        uint32_t max_n = 0;
        for (int i = 0; i < n; i++) if (lists[i].n > max_n) max_n = lists[i].n;
        int src = cvp9k_launch_scatter(s->d_jobs, n, max_n, b->hs);
        if (src != 0) return bfail(b, (cudaError_t)src, "coefficient scatter");
        s->launches_extra++;
    }
    if (any_packed) {
        int urc = cvp9k_launch_unpack(s->d_jobs, n, max_pages, s->d_misc + n + 2, b->hs);
        if (urc != 0) return bfail(b, (cudaError_t)urc, "coefficient unpack");
        s->launches_extra++;
    }
    BCK(cudaEventRecord(s->ev_h2d, b->hs), "event");

    /* kernels */
    BCK(cudaStreamWaitEvent(b->cs, s->ev_h2d, 0), "wait inputs");
    BCK(cudaEventRecord(s->ev_k0, b->cs), "event");
    cvp9k_launch_t L;
    memset(&L, 0, sizeof(L));
    L.jobs = s->d_jobs;
    L.njobs = n;
    L.arith = full ? CVP9_ARITH_SPEC : b->arith;
    L.max_blocks = max_blocks;
    L.scan_ctas = (max_mi + 255) / 256;
    L.tickets = s->d_tickets;
    L.n_tickets = s->n_tickets;
    L.ticket_counter = s->d_misc;
    {
        int width = tc.half ? (b->resident_ctas + 1) / 2 : b->resident_ctas;
        /* at most twice the wavefront's width: a CTA beyond that only holds
         * a ticket whose neighbours are not done and spins on them, keeping
         * SM slots from work that could run beside this step (a 2160p key
         * frame is 34 superblocks wide; 64 1080p frames are 1088) */
        const int cap = 2 * wave > 32 ? 2 * wave : 32;
        if (width > cap) width = cap;
        L.recon_ctas = (int)s->n_tickets < width ? (int)s->n_tickets : width;
    }
    L.lf_tile_h = tc.lf32 ? 32 : 64;
    L.warp_levels = cvp9_env_recon_warp();
    if (tc.inter) {
        L.general = s->d_fast;
        L.general_tickets = s->d_fast + s->n_tickets;
        L.n_general = s->d_fast + 2 * (size_t)s->n_tickets;
        L.inter_variant = tc.inter;
    }
    L.lf_tiles_x = any_tile ? lf_tx : 0;
    L.lf_tiles_y = any_tile ? lf_ty : 0;
    L.lf_strips_x = any_strip ? lf_sx : 0;
    L.lf_strips_y = any_strip ? lf_sy : 0;
    L.flat_lf_max_w = flat_w;
    L.flat_lf_max_h = flat_h;
    L.flat_nv12 = flat_nv;
    if (full) {
        L.full = 1;
        L.lf_counter = s->d_misc + 2 * (size_t)n + 2;
        L.lf_tickets = (uint32_t)(n * max_sbr);
        L.lf_ctas = b->lf_full_ctas;   /* as many as fit: rows wait only on rows taken earlier */
    }
    for (int k = 0; k < 4; k++) L.ev[k] = s->ev_kern[k];
    uint64_t gkey = mix64(mix64(mix64(key, (uint64_t)(uintptr_t)s->d_jobs), (uint64_t)(uintptr_t)s->d_sb_range),
                          mix64((uint64_t)(uintptr_t)s->d_misc, (uint64_t)(uintptr_t)s->d_tickets));
    gkey = mix64(gkey, ((uint64_t)L.scan_ctas << 32) | (uint64_t)L.recon_ctas);
    gkey = mix64(gkey, (uint64_t)(uintptr_t)L.general);
    gkey = mix64(gkey, ((uint64_t)L.inter_variant << 16) | (uint64_t)L.lf_tile_h);
    gkey = mix64(gkey, ((uint64_t)L.full << 32) | (uint64_t)L.lf_tickets);
    gkey = mix64(gkey, (uint64_t)L.warp_levels);
    /* k_inter + k_compact, or k_pred + k_resid + k_compact (the split, both
     * profiles: cvp9k_launch_frame dispatches inter paths 3 and 4 to it) */
    const int split = L.inter_variant >= 3;     /* path 5: one more residual kernel */
    s->launches = full ? (uint32_t)(2 * (L.scan_ctas > 0) + 1 + 1)     /* scan, mode info, recon, VP9 filter */
                       : (uint32_t)((L.scan_ctas > 0) + 1 + any_tile + any_strip + (flat_w > 0 ? 2 : 0) +
                                    (L.general ? (split ? 3 + (L.inter_variant == 5 && L.arith == CVP9_ARITH_REFCPU) : 2) : 0));
    if (b->use_graphs) {
        if (!s->graph || s->graph_key != gkey) {
            if (s->graph) { cudaGraphExecDestroy(s->graph); s->graph = NULL; }
            cudaGraph_t g;
            BCK(cudaStreamBeginCapture(b->cs, cudaStreamCaptureModeThreadLocal), "graph capture");
            cudaMemsetAsync(s->d_sb_range, 0, n_sb * 16, b->cs);
            cudaMemsetAsync(s->d_misc, 0, (size_t)(n + 1) * 4, b->cs);
            if (full) cudaMemsetAsync(L.lf_counter, 0, 4, b->cs);
            int lrc = cvp9k_launch_frame(&L, b->cs);
            cudaError_t ce = cudaStreamEndCapture(b->cs, &g);
            if (lrc != 0 || ce != cudaSuccess) {
                if (ce == cudaSuccess) cudaGraphDestroy(g);
                cudaGetLastError();
                return bfail(b, lrc != 0 ? (cudaError_t)lrc : ce, "graph capture");
            }
            ce = cudaGraphInstantiate(&s->graph, g, 0);
            cudaGraphDestroy(g);
            if (ce != cudaSuccess) { s->graph = NULL; return bfail(b, ce, "graph instantiate"); }
            s->graph_key = gkey;
        } else {
            b->graph_replays++;
        }
        BCK(cudaGraphLaunch(s->graph, b->cs), "graph launch");
    } else {
        BCK(cudaMemsetAsync(s->d_sb_range, 0, n_sb * 16, b->cs), "clear sb_range");
        BCK(cudaMemsetAsync(s->d_misc, 0, (size_t)(n + 1) * 4, b->cs), "clear status");
        if (full) BCK(cudaMemsetAsync(L.lf_counter, 0, 4, b->cs), "clear filter tickets");
        int lrc = cvp9k_launch_frame(&L, b->cs);
        if (lrc != 0) return bfail(b, (cudaError_t)lrc, "launch");
    }
    BCK(cudaEventRecord(s->ev_k1, b->cs), "event");

    /* downloads: the frames side by side in the staging buffer (one kernel),
     * then one copy into the step's output area */
    BCK(cudaStreamWaitEvent(b->ds, s->ev_k1, 0), "wait kernels");
    s->d2h_bytes = 0;
    const int area = (int)(seq % OUTR);
    if (s->out_total && !b->collect) {
        for (int i = 0; i < n; i++) {
            const bstream_t *st = &b->st[sids[i]];
            BCK(cudaMemcpyAsync(b->h_area[area] + s->fin[i].out_off, st->f[ofr[i]].dev, frame_bytes(st->W, st->H),
                                cudaMemcpyDeviceToHost, b->ds), "download");
            s->d2h_bytes += frame_bytes(st->W, st->H);
        }
    } else if (s->out_total) {
        size_t max_fb = 0;
        for (int i = 0; i < n; i++) {
            const size_t fb = frame_bytes(b->st[sids[i]].W, b->st[sids[i]].H);
            if (fb > max_fb) max_fb = fb;
        }
        int crc = cvp9k_launch_collect(s->d_jobs, n, max_fb, b->ds);
        if (crc != 0) {
            if (ofr != out_frame) free(ofr);
            return bfail(b, (cudaError_t)crc, "output collection");
        }
        s->launches_extra++;
        BCK(cudaMemcpyAsync(b->h_area[area], s->d_out, s->out_total, cudaMemcpyDeviceToHost, b->ds), "download");
        s->d2h_bytes += s->out_total;
    }
    for (int i = 0; i < n; i++) {
        bstream_t *st = &b->st[sids[i]];
        if (want_out) {
            const int par = s->fin[i].outk;
            st->h_out[par] = b->h_area[area] + s->fin[i].out_off;
            st->out_area[par] = area;
            st->f[ofr[i]].d2h_seq = seq;
            st->out_w[par] = st->W;
            st->out_h[par] = st->H;
            st->out_pts[par] = pts ? pts[i] : 0;
            st->out_seq[par] = seq;
            st->out_status[par] = 0;
            st->latest = par;
        }
        st->last_seq = seq;
        /* pool update, as the per-stream backend does */
        const vp9_parsed_frame_t *pf = pfs[i];
        if (b->arith != CVP9_ARITH_REFCPU) {
            unsigned refresh = pf->hdr.refresh_frame_flags ? pf->hdr.refresh_frame_flags : 0x01u;
            for (int r = 0; r < 8; r++) if (refresh & (1u << r)) set_ref(st, r, ofr[i]);
        } else if (pf->hdr.frame_type == VP9_FRAME_KEY) {
            for (int r = 0; r < 8; r++) set_ref(st, r, ofr[i]);
        } else {
            set_ref(st, 0, ofr[i]);
        }
    }
    if (ofr != out_frame) free(ofr);
    BCK(cudaMemcpyAsync(s->h_misc, s->d_misc, (size_t)(2 * n + 2) * 4, cudaMemcpyDeviceToHost, b->ds), "status");
    s->d2h_bytes += (size_t)(n + 3) * 4;
    /* ev_end, then the completion callback (so a stamped step is complete
     * for every other query), then ev_cb, which slot reuse waits on so the
     * callback's argument is never overwritten while pending */
    BCK(cudaEventRecord(s->ev_end, b->ds), "event");
    s->lat_arg.b = b;
    s->lat_arg.seq = seq;
    b->lat_seq[seq % LAT_RING] = seq;
    b->lat_done[seq % LAT_RING] = 0.0;
    BCK(cudaLaunchHostFunc(b->ds, step_done_cb, &s->lat_arg), "completion callback");
    BCK(cudaEventRecord(s->ev_cb, b->ds), "event");

    s->seq = seq;
    s->n = n;
    s->busy = 1;
    b->seq = seq;
    return CVP9_OK;
}

cvp9_err_t cvp9_batch_wait(cvp9_batch_t *b)
{
    if (!b) return CVP9_ERR_INVALID_DATA;
    cvp9_err_t first = CVP9_OK;
    for (uint64_t q = b->done_seq + 1; q <= b->seq; q++) {
        bslot_t *s = &b->slot[q % BSLOTS];
        if (s->seq != q) continue;
        cvp9_err_t e = wait_slot(b, s);
        if (e != CVP9_OK) return e;
        for (int i = 0; i < s->n && first == CVP9_OK; i++) {
            uint32_t stt = slot_status(s, i);
            if (stt & (CVP9_JOB_BAD_BLOCK | CVP9_JOB_BAD_ORDER | CVP9_JOB_TOO_MANY)) first = CVP9_ERR_INVALID_DATA;
            else if (stt & CVP9_JOB_TIMEOUT) first = CVP9_ERR_GPU;
        }
    }
    b->done_seq = b->seq;
    return first;
}

int cvp9_batch_poll(cvp9_batch_t *b)
{
    if (!b) return CVP9_ERR_INVALID_DATA;
    for (uint64_t q = b->done_seq + 1; q <= b->seq; q++) {
        bslot_t *s = &b->slot[q % BSLOTS];
        if (s->seq != q || !s->busy) continue;
        cudaError_t e = cudaEventQuery(s->ev_cb);
        if (e == cudaErrorNotReady) return 0;
        if (e != cudaSuccess) return CVP9_ERR_GPU;
        complete_slot(b, s);
    }
    b->done_seq = b->seq;
    return 1;
}

/* Planes of output buffer k of stream sid, once the step downloading into
 * it has completed (AGAIN while it runs). */
static cvp9_err_t deliver(cvp9_batch_t *b, int sid, int k, cvp9_frame_info_t *info)
{
    bstream_t *st = &b->st[sid];
    if (st->out_seq[k] > b->done_seq) {
        bslot_t *s = &b->slot[st->out_seq[k] % BSLOTS];
        if (s->busy && s->seq == st->out_seq[k]) {
            /* the frame and the status words have landed once ev_end is done */
            cudaError_t e = cudaEventQuery(s->ev_end);
            if (e == cudaErrorNotReady) return CVP9_ERR_AGAIN;
            if (e != cudaSuccess) return bfail(b, e, "step completion");
            for (int i = 0; i < s->n; i++)
                if (s->sids[i] == sid) {
                    st->out_status[k] = slot_status(s, i);
                    if (st->last_seq == s->seq) st->last_status = st->out_status[k];
                }
            if (cudaEventQuery(s->ev_cb) == cudaSuccess) complete_slot(b, s);
        }
    }
    /* the output area has since taken a newer step's frames */
    if (b->area_seq[st->out_area[k]] != st->out_seq[k]) return CVP9_ERR_INVALID_DATA;
    const uint32_t status = st->out_status[k];
    if (status & (CVP9_JOB_BAD_BLOCK | CVP9_JOB_BAD_ORDER | CVP9_JOB_TOO_MANY)) return CVP9_ERR_INVALID_DATA;
    if (status & CVP9_JOB_TIMEOUT) return CVP9_ERR_GPU;
    uint32_t w = (uint32_t)st->out_w[k], h = (uint32_t)st->out_h[k];
    uint32_t cw = (w + 1) / 2, ch = (h + 1) / 2;
    info->width = w;
    info->height = h;
    info->stride_y = w;
    info->stride_uv = cw;
    info->plane_y = st->h_out[k];
    info->plane_u = st->h_out[k] + (size_t)w * h;
    info->plane_v = st->h_out[k] + (size_t)w * h + (size_t)cw * ch;
    info->pts = st->out_pts[k];
    return CVP9_OK;
}

cvp9_err_t cvp9_batch_get_frame(cvp9_batch_t *b, int sid, cvp9_frame_info_t *info)
{
    if (!b || !info || sid < 0 || sid >= b->max_streams || !b->st[sid].open) return CVP9_ERR_INVALID_DATA;
    if (b->st[sid].latest < 0) return CVP9_ERR_UNSUPPORTED;
    return deliver(b, sid, b->st[sid].latest, info);
}

cvp9_err_t cvp9_batch_get_frame_at(cvp9_batch_t *b, int sid, uint64_t seq, cvp9_frame_info_t *info)
{
    if (!b || !info || sid < 0 || sid >= b->max_streams || !b->st[sid].open || seq == 0) return CVP9_ERR_INVALID_DATA;
    const bstream_t *st = &b->st[sid];
    for (int k = 0; k < OUTR; k++)
        if (st->out_seq[k] == seq) return deliver(b, sid, k, info);
    return CVP9_ERR_INVALID_DATA;
}

cvp9_err_t cvp9_batch_reserve(cvp9_batch_t *b, uint32_t w, uint32_t h, int nstreams)
{
    if (!b || w == 0 || h == 0 || w > 65535 || h > 65535 || nstreams <= 0) return CVP9_ERR_INVALID_DATA;
    if (cudaSetDevice(b->device) != cudaSuccess) return CVP9_ERR_GPU;
    const uint64_t fb = frame_bytes((int32_t)w, (int32_t)h);
    /* the output areas and staging buffers are resized below: no step may
     * still use them */
    for (int k = 0; k < BSLOTS; k++) {
        cvp9_err_t e = wait_slot(b, &b->slot[k]);
        if (e != CVP9_OK) return e;
    }
    /* device: the admission unit per stream covers its frames and its share
     * of the step buffers (the output staging with the arena's headroom on
     * top); host: one frame per stream of slack for the step's staging and
     * packing buffers; then every output area and staging buffer sized for
     * a step holding all reserved streams at once */
    const uint64_t dev = (uint64_t)nstreams * (cvp9_batch_stream_bytes(w, h) + 2 * fb);
    const uint64_t pin = (uint64_t)nstreams * fb;
    if (arena_reserve(&b->dev, (size_t)(b->dev.held - b->dev.used + dev)) != 0) {
        snprintf(b->err, sizeof(b->err), "device arena: no memory to reserve %llu bytes", (unsigned long long)dev);
        return CVP9_ERR_NOMEM;
    }
    if (arena_reserve(&b->pin, (size_t)(b->pin.held - b->pin.used + pin)) != 0) {
        snprintf(b->err, sizeof(b->err), "pinned arena: no memory to reserve %llu bytes", (unsigned long long)pin);
        return CVP9_ERR_NOMEM;
    }
    b->out_reserve += (size_t)nstreams * ALIGN_UP(fb, 256);
    cvp9_err_t err;
    for (int a = 0; a < OUTR; a++) {
        if (b->h_area[a] && b->h_area_cap[a] >= b->out_reserve) continue;
        b->area_seq[a] = 0;                    /* its frames, if any, are gone */
        if ((err = grow_host(b, (void **)&b->h_area[a], &b->h_area_cap[a], b->out_reserve))) return err;
    }
    for (int k = 0; k < BSLOTS && b->collect; k++)
        if ((err = grow_dev(b, (void **)&b->slot[k].d_out, &b->slot[k].d_out_cap, b->out_reserve))) return err;
    return CVP9_OK;
}

cvp9_err_t cvp9_batch_stats(cvp9_batch_t *b, cvp9_batch_stats_t *out)
{
    if (!b || !out) return CVP9_ERR_INVALID_DATA;
    *out = b->last;
    out->reserved_bytes = b->reserved;
    int open = 0;
    for (int i = 0; i < b->nst; i++) open += b->st[i].open;
    out->open_streams = open;
    out->graph_replays = b->graph_replays;
    out->submit_pack_ms = b->submit_pack_ms;
    out->submit_wait_ms = b->submit_wait_ms;
    out->submit_stage_ms = b->submit_stage_ms;
    out->dev_held_bytes = b->dev.held;
    out->host_held_bytes = b->pin.held;
    return CVP9_OK;
}

const char *cvp9_batch_last_error(cvp9_batch_t *b)
{
    return b ? b->err : "";
}

cvp9_err_t cvp9_batch_timer_start(cvp9_batch_t *b)
{
    if (!b) return CVP9_ERR_INVALID_DATA;
    if (cudaSetDevice(b->device) != cudaSuccess) return CVP9_ERR_GPU;
    /* the next step's upload (hs) starts after this event */
    BCK(cudaEventRecord(b->ev_t0, b->hs), "timer");
    b->t0_set = 1;
    return CVP9_OK;
}

cvp9_err_t cvp9_batch_timer_stop(cvp9_batch_t *b, float *ms)
{
    if (!b || !ms) return CVP9_ERR_INVALID_DATA;
    if (cudaSetDevice(b->device) != cudaSuccess) return CVP9_ERR_GPU;
    /* ds holds the last step's download, which follows its kernels */
    BCK(cudaEventRecord(b->ev_t1, b->ds), "timer");
    double t0 = cvp9_now();
    for (;;) {
        cudaError_t e = cudaEventQuery(b->ev_t1);
        if (e == cudaSuccess) break;
        if (e != cudaErrorNotReady) return bfail(b, e, "timer");
        if (cvp9_now() - t0 > WAIT_LIMIT_S) return CVP9_ERR_GPU;
        struct timespec ts = { 0, 20000 };
        nanosleep(&ts, NULL);
    }
    BCK(cudaEventElapsedTime(ms, b->ev_t0, b->ev_t1), "timer");
    return CVP9_OK;
}

uint64_t cvp9_batch_last_seq(cvp9_batch_t *b)
{
    return b ? b->seq : 0;
}

cvp9_err_t cvp9_batch_step_latency(cvp9_batch_t *b, uint64_t seq, double *ms)
{
    if (!b || !ms || seq == 0 || seq > b->seq || b->seq - seq >= LAT_RING) return CVP9_ERR_INVALID_DATA;
    if (b->lat_seq[seq % LAT_RING] != seq) return CVP9_ERR_INVALID_DATA;
    double d = b->lat_done[seq % LAT_RING];
    if (d == 0.0) return CVP9_ERR_AGAIN;
    *ms = 1000.0 * (d - b->lat_submit[seq % LAT_RING]);
    return CVP9_OK;
}

cvp9_err_t cvp9_batch_step_timeline(cvp9_batch_t *b, uint64_t seq, float t[5])
{
    if (!b || !t || seq == 0 || seq > b->seq || b->seq - seq >= LAT_RING || !b->t0_set) return CVP9_ERR_INVALID_DATA;
    if (seq > b->done_seq) return CVP9_ERR_AGAIN;
    if (b->tl_seq[seq % LAT_RING] != seq) return CVP9_ERR_INVALID_DATA;
    memcpy(t, b->tl[seq % LAT_RING], 5 * sizeof(float));
    return CVP9_OK;
}

int cvp9_batch_tune_count(cvp9_batch_t *b)
{
    if (!b) return 0;
    int n = 0;
    for (int i = 0; i < CVP9_TUNE_BUCKETS; i++) n += b->tuner.b[i].state != 0;
    return n;
}

cvp9_err_t cvp9_batch_tune_entry(cvp9_batch_t *b, int i, cvp9_batch_tune_t *out)
{
    if (!b || !out || i < 0) return CVP9_ERR_INVALID_DATA;
    for (int k = 0; k < CVP9_TUNE_BUCKETS; k++) {
        const cvp9_tbucket_t *e = &b->tuner.b[k];
        if (!e->state || i--) continue;
        memset(out, 0, sizeof(*out));
        out->key = e->key;
        out->frames = e->frames;
        out->settled = e->state == 2;
        out->inter_path = e->best.inter;
        out->lf_tile_h = e->best.lf32 ? 32 : 16;
        out->half_width = e->best.half;
        out->trials = e->trials;
        out->best_ms = e->trials ? e->best_ms : 0.f;
        return CVP9_OK;
    }
    return CVP9_ERR_INVALID_DATA;
}
