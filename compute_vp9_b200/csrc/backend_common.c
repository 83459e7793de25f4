/*
 * backend_common.c — device setup, DCT basis, ticket order, job geometry.
 * Compiled with -ffp-contract=off so the basis matches the reference's
 * separately rounded float64 arithmetic.
 */
#include "backend_common.h"
#include "recon_launch.h"
#include "vp9_tables.h"

#include <math.h>
#include <pthread.h>
#include <unistd.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static const int16_t k_dc_q[256] = CVP9_QTABLE_DC_INIT;
static const int16_t k_ac_q[256] = CVP9_QTABLE_AC_INIT;

int cvp9_dc_q(int q) { return k_dc_q[CVP9_QINDEX_CLAMP(q)]; }
int cvp9_ac_q(int q) { return k_ac_q[CVP9_QINDEX_CLAMP(q)]; }

void cvp9_build_dct_basis(double *out)
{
    int base = 0;
    for (int n = 4; n <= 32; n *= 2) {
        double scale_zero = sqrt(1.0 / n);
        double scale_other = sqrt(2.0 / n);
        for (int i = 0; i < n; i++) {
            double scale = (i == 0) ? scale_zero : scale_other;
            for (int j = 0; j < n; j++)
                out[base + i * n + j] = scale * cos(((2.0 * j + 1.0) * i * 3.141592653589793) / (2.0 * n));
        }
        base += n * n;
    }
}

#define MAX_DEVICES 64
static pthread_mutex_t g_setup_lock = PTHREAD_MUTEX_INITIALIZER;
static int g_setup_done[MAX_DEVICES];
static int g_ctas[MAX_DEVICES][2];
static int g_lf_ctas[MAX_DEVICES];

int cvp9_device_setup(int device)
{
    if (device < 0 || device >= MAX_DEVICES) return -1;
    if (cudaSetDevice(device) != cudaSuccess) return -1;
    pthread_mutex_lock(&g_setup_lock);
    int rc = 0;
    if (!g_setup_done[device]) {
        double basis[16 + 64 + 256 + 1024];
        cvp9_build_dct_basis(basis);
        if (cvp9k_upload_dct_basis(basis, 16 + 64 + 256 + 1024) != 0 || cvp9k_configure() != 0) {
            rc = -1;
        } else {
            g_ctas[device][0] = cvp9k_recon_ctas_per_sm(CVP9_ARITH_REFCPU);
            g_ctas[device][1] = cvp9k_recon_ctas_per_sm(CVP9_ARITH_SPEC);
            g_lf_ctas[device] = cvp9k_lf_full_ctas_per_sm();
            g_setup_done[device] = 1;
        }
    }
    pthread_mutex_unlock(&g_setup_lock);
    return rc;
}

int cvp9_recon_ctas_per_sm(int device, int arith)
{
    if (device < 0 || device >= MAX_DEVICES) return 1;
    int v = g_ctas[device][arith != CVP9_ARITH_REFCPU ? 1 : 0];    /* FULL runs the SPEC kernel */
    return v > 0 ? v : 1;
}

int cvp9_lf_full_ctas_per_sm(int device)
{
    if (device < 0 || device >= MAX_DEVICES) return 1;
    return g_lf_ctas[device] > 0 ? g_lf_ctas[device] : 1;
}

int cvp9_tickets_on_diagonal(int sb_cols, int sb_rows, int job, int d, uint32_t *out)
{
    int n = 0;
    int r0 = d - (sb_cols - 1);
    if (r0 < 0) r0 = 0;
    int r1 = d < sb_rows - 1 ? d : sb_rows - 1;
    for (int r = r0; r <= r1; r++) {
        int c = d - r;
        out[n++] = ((uint32_t)job << 20) | (uint32_t)(r * sb_cols + c);
    }
    return n;
}

int cvp9_env_device(void)
{
    const char *e = getenv("CVP9_CUDA_DEVICE");
    return e && *e ? atoi(e) : 0;
}

int cvp9_env_gather(void)
{
    const char *e = getenv("CVP9_GATHER");
    return !(e && *e == '0');
}

int cvp9_env_pack(int configured)
{
    const char *e = getenv("CVP9_PACK");
    if (e && *e == '0') return -1;
    if (e && *e == '1') return 1;
    return configured < 0 ? -1 : configured > 0 ? 1 : 0;
}

int cvp9_env_autotune(void)
{
    const char *e = getenv("CVP9_AUTOTUNE");
    return !(e && *e == '0');
}

int cvp9_env_inter_fast(void)
{
    const char *e = getenv("CVP9_INTER_FAST");
    if (e && *e >= '0' && *e <= '5' && !e[1]) return *e - '0';
    return 1;
}

int cvp9_env_recon_warp(void)
{
    const char *e = getenv("CVP9_RECON_WARP");
    return !(e && e[0] == '0' && !e[1]);
}

int cvp9_env_arith(void)
{
    const char *e = getenv("CVP9_ARITH");
    if (e && (strcmp(e, "spec") == 0 || strcmp(e, "SPEC") == 0)) return CVP9_ARITH_SPEC;
    if (e && (strcmp(e, "full") == 0 || strcmp(e, "FULL") == 0)) return CVP9_ARITH_FULL;
    return CVP9_ARITH_REFCPU;
}

int cvp9_filter_supported(int arith, int interp_filter, const char **why)
{
    if (arith == CVP9_ARITH_REFCPU || interp_filter == VP9_FILTER_EIGHTTAP) return 1;
    if (arith == CVP9_ARITH_FULL && interp_filter >= 0 && interp_filter <= VP9_FILTER_BILINEAR) return 1;
    if (why) *why = arith == CVP9_ARITH_FULL
        ? "SWITCHABLE interpolation filter: the parsed block record carries no per-block filter"
        : "interpolation filter other than EIGHTTAP: the shader profile holds the regular 8-tap table only";
    return 0;
}

int cvp9_frame_supported(int arith, const vp9_parsed_frame_t *pf, const char **why)
{
    const int inter = pf->hdr.frame_type != VP9_FRAME_KEY && !pf->hdr.intra_only;
    if (arith == CVP9_ARITH_FULL && ((pf->hdr.width & 7) || (pf->hdr.height & 7))) {
        if (why) *why = "the VP9 profile takes frames whose sizes are multiples of 8";
        return 0;
    }
    /* intra frames carry no filter; only inter frames are held to it */
    return inter ? cvp9_filter_supported(arith, (int)pf->hdr.interp_filter, why) : 1;
}

void cvp9_job_full(cvp9_job_t *job, const vp9_parsed_frame_t *pf)
{
    const vp9_frame_header_t *h = &pf->hdr;
    const int q = h->base_qindex;
    const int inter = h->frame_type != VP9_FRAME_KEY && !h->intra_only;
    job->full = 1;
    job->q_dc = cvp9_dc_q(q + h->y_dc_delta_q);
    job->q_ac = cvp9_ac_q(q);
    job->q_dc_uv = cvp9_dc_q(q + h->uv_dc_delta_q);
    job->q_ac_uv = cvp9_ac_q(q + h->uv_ac_delta_q);
    job->lossless = (uint8_t)(q == 0 && h->y_dc_delta_q == 0 && h->uv_dc_delta_q == 0 && h->uv_ac_delta_q == 0);
    job->interp_filter = (uint8_t)(inter ? (h->interp_filter & 3) : 0);
    job->log2_tile_cols = h->log2_tile_cols;
}

void cvp9_job_geometry(cvp9_job_t *job, const vp9_parsed_frame_t *pf)
{
    int W = (int)pf->hdr.width, H = (int)pf->hdr.height;
    job->W = W;
    job->H = H;
    job->CW = (W + 1) / 2;
    job->CH = (H + 1) / 2;
    job->sb_cols = (W + 63) / 64;
    job->sb_rows = (H + 63) / 64;
    job->mi_cols = (W + 7) / 8;
    job->mi_rows = (H + 7) / 8;
    job->num_blocks = pf->num_blocks;
    job->num_coeffs = pf->num_coeffs;
    job->q_dc = cvp9_dc_q(pf->hdr.base_qindex);
    job->q_ac = cvp9_ac_q(pf->hdr.base_qindex);
    job->lf_level = pf->hdr.filter_level;
    job->lf_sharpness = pf->hdr.sharpness_level;
    for (int i = 0; i < 3; i++) job->ref_slot_of[i] = pf->hdr.ref_frame_idx[i] & 7;
    job->lf_tiled = (uint8_t)((W % 8) != 1 && (H % 8) != 1);
}

double cvp9_now(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* ── Autotuner ─────────────────────────────────────────────────────────── */

static int ceil_log2_u64(uint64_t v)
{
    int l = 0;
    while (l < 63 && (1ull << l) < v) l++;
    return l;
}

uint64_t cvp9_tune_key(int arith, int frames, uint64_t superblocks)
{
    return ((uint64_t)(arith & 0xff) << 16) | ((uint64_t)ceil_log2_u64((uint64_t)(frames > 0 ? frames : 1)) << 8) |
           (uint64_t)ceil_log2_u64(superblocks ? superblocks : 1);
}

void cvp9_tuner_init(cvp9_tuner_t *t, int arith, int enabled, cvp9_tcfg_t fixed)
{
    memset(t, 0, sizeof(*t));
    t->arith = arith;
    t->enabled = enabled;
    t->fixed = fixed;
    /* FULL: every superblock goes through the general kernel and the VP9
     * loop filter has one layout; only the wavefront width is tuned */
    if (arith == CVP9_ARITH_FULL) { t->fixed.inter = 0; t->fixed.lf32 = 0; }
}

static int same_cfg(cvp9_tcfg_t a, cvp9_tcfg_t b)
{
    return a.inter == b.inter && a.lf32 == b.lf32 && a.half == b.half;
}

/* Move to the next candidate; settle when every knob is done. */
static void tune_advance(cvp9_tuner_t *t, cvp9_tbucket_t *e)
{
    for (;;) {
        e->idx++;
        if (e->stage == 0) {
            /* inter path: the default was candidate 0; then the general
             * kernel alone, k_inter at 80 registers, the two-kernel split
             * and (REFCPU) the split walking 8x8 TXs per TX, and that split
             * with superblocks of 8x8 TXs only in a residual kernel of their
             * own */
            static const int8_t alts[5] = { 0, 2, 3, 4, 5 };
            if (t->arith != CVP9_ARITH_FULL && e->idx <= (t->arith == CVP9_ARITH_REFCPU ? 5 : 3)) {
                e->cur = e->best;
                e->cur.inter = alts[e->idx - 1];
                break;
            }
            e->stage = 1;
            e->idx = 0;
        } else if (e->stage == 1) {
            if (e->idx == 1 && t->arith != CVP9_ARITH_FULL) { e->cur = e->best; e->cur.lf32 = 1; break; }
            e->stage = 2;
            e->idx = 0;
        } else if (e->stage == 2) {
            if (e->idx == 1) { e->cur = e->best; e->cur.half = 1; break; }
            e->state = 2;
            return;
        } else {
            e->state = 2;
            return;
        }
    }
    e->cur_n = 0;
    e->cur_ms = 0.f;
}

int cvp9_tuner_pick(cvp9_tuner_t *t, uint64_t key, int frames, cvp9_tcfg_t *cfg)
{
    *cfg = t->fixed;
    if (!t->enabled) return -1;
    t->clock++;
    int free_i = -1, lru = 0;
    for (int i = 0; i < CVP9_TUNE_BUCKETS; i++) {
        cvp9_tbucket_t *e = &t->b[i];
        if (e->state && e->key == key) {
            e->last_use = t->clock;
            if (e->state == 2) { *cfg = e->best; return -1; }
            *cfg = e->cur;
            return i;
        }
        if (!e->state && free_i < 0) free_i = i;
        if (e->last_use < t->b[lru].last_use) lru = i;
    }
    int i = free_i >= 0 ? free_i : lru;
    cvp9_tbucket_t *e = &t->b[i];
    memset(e, 0, sizeof(*e));
    e->key = key;
    e->frames = frames;
    e->state = 1;
    e->cur = t->fixed;
    e->best = t->fixed;
    e->best_ms = 3.4e38f;
    e->last_use = t->clock;
    *cfg = e->cur;
    return i;
}

void cvp9_tuner_report(cvp9_tuner_t *t, int idx, cvp9_tcfg_t cfg, float ms)
{
    if (idx < 0 || idx >= CVP9_TUNE_BUCKETS) return;
    cvp9_tbucket_t *e = &t->b[idx];
    if (e->state != 1 || !same_cfg(cfg, e->cur) || !(ms > 0.f)) return;   /* a stale sample */
    e->cur_ms = e->cur_n ? (ms < e->cur_ms ? ms : e->cur_ms) : ms;
    if (++e->cur_n < 2) return;
    e->trials++;
    /* a challenger must win by more than 2% (timing noise keeps the
     * incumbent) */
    if (e->cur_ms < (e->trials == 1 ? 3.4e38f : 0.98f * e->best_ms)) {
        e->best_ms = e->cur_ms;
        e->best = e->cur;
    }
    tune_advance(t, e);
}

/* ── Share of a large step's frames that are packed ─────────────────────── */

int cvp9_pack_share_update(int q, int pipelined, double waited_ms)
{
    /* Packing trades host time (reading every dense array) for link time.
     * Balance the two while steps are pipelined: a submit that had to wait
     * for its slot found the link (or the GPU) behind, so the host can pack
     * more; one that did not wait found the host behind, so it packs less.
     * A caller that waits for each step first gives no signal. */
    if (pipelined) q += waited_ms > 0.05 ? 1 : -1;
    return q < 0 ? 0 : q > 16 ? 16 : q;
}

/* ── Host worker pools ────────────────────────────────────────────────── */

/* Two pools: a small one for staging copies (the per-stream backend, on
 * every frame) and a large one for packing (large batch steps). Copies
 * measured slower on the GPU hosts whenever their tasks could land on any
 * of 16 workers, so they keep a pool of their own. */
#define POOL_MAX_THREADS 16

typedef struct {
    pthread_mutex_t mu;
    pthread_cond_t  work, done;
    pthread_mutex_t busy;            /* one parallel job at a time */
    pthread_once_t  once;
    void          (*fn)(void *, int);
    void           *ctx;
    int             ntasks, next, pending;
    int             nthreads;        /* workers (the caller is one more) */
    const char     *env;             /* total threads override */
    int             deflt;           /* total threads by default; 0: one per CPU up to 16 */
} pool_t;

#define POOL_INIT(env, deflt) { PTHREAD_MUTEX_INITIALIZER, PTHREAD_COND_INITIALIZER, PTHREAD_COND_INITIALIZER, \
                                PTHREAD_MUTEX_INITIALIZER, PTHREAD_ONCE_INIT, NULL, NULL, 0, 0, 0, -1, env, deflt }
static pool_t g_copy_pool = POOL_INIT("CVP9_COPY_THREADS", 4);
static pool_t g_work_pool = POOL_INIT("CVP9_HOST_THREADS", 0);

/* takes tasks until none is left; called with p->mu held */
static void pool_drain(pool_t *p)
{
    while (p->next < p->ntasks) {
        int k = p->next++;
        void (*fn)(void *, int) = p->fn;
        void *ctx = p->ctx;
        pthread_mutex_unlock(&p->mu);
        fn(ctx, k);
        pthread_mutex_lock(&p->mu);
        if (--p->pending == 0) pthread_cond_broadcast(&p->done);
    }
}

static void *pool_worker(void *arg)
{
    pool_t *p = (pool_t *)arg;
    pthread_mutex_lock(&p->mu);
    for (;;) {
        while (p->next >= p->ntasks) pthread_cond_wait(&p->work, &p->mu);
        pool_drain(p);
    }
    return NULL;
}

static void pool_start(pool_t *p)
{
    long cpus = sysconf(_SC_NPROCESSORS_ONLN);
    int total = p->deflt ? p->deflt : (int)(cpus < POOL_MAX_THREADS ? cpus : POOL_MAX_THREADS);
    const char *e = getenv(p->env);
    if (e && *e) total = atoi(e);
    if (total > POOL_MAX_THREADS) total = POOL_MAX_THREADS;
    int started = 0;
    for (int i = 0; i < total - 1; i++) {
        pthread_t t;
        pthread_attr_t at;
        pthread_attr_init(&at);
        pthread_attr_setdetachstate(&at, PTHREAD_CREATE_DETACHED);
        if (pthread_create(&t, &at, pool_worker, p) == 0) started++;
        pthread_attr_destroy(&at);
    }
    p->nthreads = started;
}

static void copy_pool_start(void) { pool_start(&g_copy_pool); }
static void work_pool_start(void) { pool_start(&g_work_pool); }

static int pool_threads(pool_t *p)
{
    pthread_once(&p->once, p == &g_copy_pool ? copy_pool_start : work_pool_start);
    return p->nthreads + 1;
}

static void pool_run(pool_t *p, int ntasks, void (*fn)(void *ctx, int task), void *ctx)
{
    if (ntasks <= 0) return;
    pool_threads(p);
    if (ntasks == 1 || p->nthreads <= 0 || pthread_mutex_trylock(&p->busy) != 0) {
        for (int k = 0; k < ntasks; k++) fn(ctx, k);
        return;
    }
    pthread_mutex_lock(&p->mu);
    p->fn = fn;
    p->ctx = ctx;
    p->ntasks = ntasks;
    p->next = 0;
    p->pending = ntasks;
    /* wake only as many workers as there are tasks besides the caller's */
    for (int k = 1; k < ntasks && k <= p->nthreads; k++) pthread_cond_signal(&p->work);
    pool_drain(p);                                   /* the caller works too */
    while (p->pending > 0) pthread_cond_wait(&p->done, &p->mu);
    p->ntasks = 0;
    p->next = 0;
    pthread_mutex_unlock(&p->mu);
    pthread_mutex_unlock(&p->busy);
}

int cvp9_pool_threads(void) { return pool_threads(&g_work_pool); }

void cvp9_parallel_for(int ntasks, void (*fn)(void *ctx, int task), void *ctx)
{
    pool_run(&g_work_pool, ntasks, fn, ctx);
}

typedef struct { char *dst; const char *src; size_t n, chunk; } copy_job_t;

static void copy_task(void *ctx, int k)
{
    const copy_job_t *j = (const copy_job_t *)ctx;
    size_t off = (size_t)k * j->chunk;
    if (off < j->n) memcpy(j->dst + off, j->src + off, off + j->chunk <= j->n ? j->chunk : j->n - off);
}

void cvp9_parallel_memcpy(void *dst, const void *src, size_t n)
{
    if (n < (1u << 20)) { memcpy(dst, src, n); return; }
    const int parts = pool_threads(&g_copy_pool);
    copy_job_t j = { (char *)dst, (const char *)src, n, (n / parts + 4095) & ~(size_t)4095 };
    pool_run(&g_copy_pool, (int)((n + j.chunk - 1) / j.chunk), copy_task, &j);
}
