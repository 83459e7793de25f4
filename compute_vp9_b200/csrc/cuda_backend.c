/*
 * cuda_backend.c — per-stream CUDA backend behind the compute-vp9 backend
 * ABI (include/cuda_backend.h). Host code in C over the CUDA runtime; the
 * kernels are reached through the launch shim in recon.cu.
 *
 * Per context:
 *   - one CUDA stream; every frame is upload -> scan/recon/filter -> output
 *     copy on it, so stream order carries all cross-frame hazards;
 *   - a device-resident reference pool: up to 8 slots pointing at device
 *     I420 frames (pointer swaps, no copies — the Vulkan backend copies
 *     luma into images, vulkan_backend.c:1310-1354);
 *   - CVP9_CUDA_INFLIGHT slots of pinned staging (inputs, job descriptor,
 *     status word) so the CPU parse of the next frame overlaps the GPU work
 *     of this one (vulkan_backend.h:36-81);
 *   - OUTBUFS pinned output frames, apart from the slots. A delivered
 *     frame's planes stay untouched for the next two decode calls whatever
 *     the ring holds, as include/compute_vp9/decoder.h:100-104 promises (the
 *     Vulkan backend keeps its output in the ring slot, which the very next
 *     decode reuses when two other frames are still in flight).
 */
#include "cuda_backend.h"
#include "backend_common.h"
#include "recon_launch.h"

#include <cuda_runtime_api.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define MAX_DFRAMES 12
#define WAIT_LIMIT_S 30.0
/* Output frames needed so that a delivered frame survives two decodes: at a
 * decode at most two frames are pending, at most four frames entered the
 * ring since the decode two calls back (two pending then, two decoded since),
 * plus the new one. */
#define OUTBUFS (CVP9_CUDA_INFLIGHT + 2)

typedef struct {
    uint8_t *h;
    size_t   cap;
    int      busy;         /* holds a frame still in the ring               */
    uint64_t free_after;   /* may be reused once this many decodes were made */
} outbuf_t;

typedef struct {
    uint8_t *dev;
    size_t   cap;
    int32_t  w, h;
    int      users;       /* reference slots pointing here */
} dframe_t;

typedef struct {
    int          pending;
    int64_t      pts;
    int32_t      w, h;
    cudaEvent_t  ev_start, ev_k0, ev_k1, ev_end;
    int          tune_idx;             /* tuner bucket this frame measures, -1 none */
    cvp9_tcfg_t  tune_cfg;
    /* pinned staging */
    void        *h_blocks;  size_t h_blocks_cap;
    void        *h_coeffs;  size_t h_coeffs_cap;
    cvp9_job_t  *h_job;
    uint32_t    *h_status;
    int          out;                  /* output buffer of this frame */
    /* device inputs */
    void        *d_blocks;  size_t d_blocks_cap;
    void        *d_coeffs;  size_t d_coeffs_cap;
    cvp9_job_t  *d_job;
} slot_t;

typedef struct {
    int          device;
    int          arith;
    cudaStream_t stream;
    int32_t      W, H;                 /* current geometry */
    int          sb_cols, sb_rows, n_sb;
    dframe_t     frames[MAX_DFRAMES];
    int          ref_slot[8];          /* index into frames, -1 = empty */
    uint32_t     epoch;
    /* per-geometry scratch */
    uint32_t    *d_sb_range;           /* 4 * n_sb, zeroed per frame    */
    uint32_t    *d_sb_done;            /* n_sb                          */
    uint32_t    *d_misc;               /* [0] status, [1] ticket counter, [2] filter tickets */
    uint32_t    *d_tickets;
    uint32_t    *d_fast;               /* inter fast path: general flags, tickets, count */
    uint32_t    *d_mi_map;             /* FULL loop filter: mode info per 8x8 MI          */
    cvp9_tuner_t tuner;                /* kernel configuration per frame size */
    int          resident_ctas;
    uint32_t     n_tickets;
    int          recon_ctas;
    slot_t       slots[CVP9_CUDA_INFLIGHT];
    int          ring_head, ring_count;
    outbuf_t     outs[OUTBUFS];
    uint64_t     decodes;              /* successful decode calls */
    void        *pending_target;       /* device pointer of armed NV12 target */
    uint64_t     pending_target_size;
    float        last_total_ms, last_kernel_ms;
    char         last_error[160];
} cuctx_t;

static cvp9_err_t fail(cuctx_t *c, cudaError_t e, const char *what)
{
    if (c) snprintf(c->last_error, sizeof(c->last_error), "%s: %s", what, cudaGetErrorString(e));
    return CVP9_ERR_GPU;
}

#define CK(call, what) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) return fail(c, e_, what); } while (0)

static void free_slot(slot_t *s)
{
    if (s->ev_start) cudaEventDestroy(s->ev_start);
    if (s->ev_k0) cudaEventDestroy(s->ev_k0);
    if (s->ev_k1) cudaEventDestroy(s->ev_k1);
    if (s->ev_end) cudaEventDestroy(s->ev_end);
    cudaFreeHost(s->h_blocks);
    cudaFreeHost(s->h_coeffs);
    cudaFreeHost(s->h_job);
    cudaFreeHost(s->h_status);
    cudaFree(s->d_blocks);
    cudaFree(s->d_coeffs);
    cudaFree(s->d_job);
    memset(s, 0, sizeof(*s));
}

static void free_geometry(cuctx_t *c)
{
    cudaFree(c->d_sb_range);
    cudaFree(c->d_sb_done);
    cudaFree(c->d_tickets);
    cudaFree(c->d_fast);
    cudaFree(c->d_mi_map);
    c->d_sb_range = c->d_sb_done = c->d_tickets = c->d_fast = c->d_mi_map = NULL;
    c->n_tickets = 0;
}

cvp9_err_t cuda_backend_init_ex(void **out, const cuda_backend_options_t *opt)
{
    if (!out) return CVP9_ERR_INVALID_DATA;
    *out = NULL;
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count <= 0) return CVP9_ERR_NO_BACKEND;
    cuctx_t *c = calloc(1, sizeof(*c));
    if (!c) return CVP9_ERR_NOMEM;
    c->device = (opt && opt->device >= 0) ? opt->device : cvp9_env_device();
    c->arith = (opt && opt->arith >= 0) ? (opt->arith == CVP9_CUDA_ARITH_SPEC ? CVP9_ARITH_SPEC
                                           : opt->arith == CVP9_CUDA_ARITH_FULL ? CVP9_ARITH_FULL : CVP9_ARITH_REFCPU)
                                        : cvp9_env_arith();
    {
        cvp9_tcfg_t fixed = { (int8_t)cvp9_env_inter_fast(), 0, 0 };
        cvp9_tuner_init(&c->tuner, c->arith, !(opt && opt->autotune < 0) && cvp9_env_autotune(), fixed);
    }
    if (c->device >= dev_count || cvp9_device_setup(c->device) != 0) { free(c); return CVP9_ERR_NO_BACKEND; }
    for (int i = 0; i < 8; i++) c->ref_slot[i] = -1;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc((void **)&c->d_misc, 64) != cudaSuccess) {
        cuda_backend_destroy(c);
        return CVP9_ERR_GPU;
    }
    for (int i = 0; i < CVP9_CUDA_INFLIGHT; i++) {
        slot_t *s = &c->slots[i];
        if (cudaEventCreate(&s->ev_start) != cudaSuccess || cudaEventCreate(&s->ev_k0) != cudaSuccess ||
            cudaEventCreate(&s->ev_k1) != cudaSuccess || cudaEventCreate(&s->ev_end) != cudaSuccess ||
            cudaMallocHost((void **)&s->h_job, sizeof(cvp9_job_t)) != cudaSuccess ||
            cudaMallocHost((void **)&s->h_status, 64) != cudaSuccess ||
            cudaMalloc((void **)&s->d_job, sizeof(cvp9_job_t)) != cudaSuccess) {
            cuda_backend_destroy(c);
            return CVP9_ERR_GPU;
        }
    }
    c->epoch = 0;
    *out = c;
    return CVP9_OK;
}

cvp9_err_t cuda_backend_init(void **ctx)
{
    return cuda_backend_init_ex(ctx, NULL);
}

void cuda_backend_destroy(void *ctx)
{
    cuctx_t *c = (cuctx_t *)ctx;
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (int i = 0; i < CVP9_CUDA_INFLIGHT; i++) free_slot(&c->slots[i]);
    for (int i = 0; i < OUTBUFS; i++) cudaFreeHost(c->outs[i].h);
    for (int i = 0; i < MAX_DFRAMES; i++) cudaFree(c->frames[i].dev);
    free_geometry(c);
    cudaFree(c->d_misc);
    if (c->stream) cudaStreamDestroy(c->stream);
    free(c);
}

/* (Re)build the per-geometry scratch. Frames in flight finish first; the
 * reference pool keeps its frames (they carry their own size, and MC clamps
 * into each reference's own extent as the CPU path does). */
static cvp9_err_t set_geometry(cuctx_t *c, int32_t W, int32_t H)
{
    CK(cudaStreamSynchronize(c->stream), "sync before resize");
    free_geometry(c);
    c->W = W;
    c->H = H;
    c->sb_cols = (W + 63) / 64;
    c->sb_rows = (H + 63) / 64;
    c->n_sb = c->sb_cols * c->sb_rows;
    CK(cudaMalloc((void **)&c->d_sb_range, (size_t)c->n_sb * 16), "alloc sb_range");
    CK(cudaMalloc((void **)&c->d_sb_done, (size_t)c->n_sb * 4), "alloc sb_done");
    CK(cudaMemset(c->d_sb_done, 0, (size_t)c->n_sb * 4), "clear sb_done");
    CK(cudaMalloc((void **)&c->d_tickets, (size_t)c->n_sb * 4), "alloc tickets");
    CK(cudaMalloc((void **)&c->d_fast, (size_t)(2 * c->n_sb + 2) * 4), "alloc fast-path scratch");
    if (c->arith == CVP9_ARITH_FULL) {
        size_t nmi = (size_t)((W + 7) / 8) * ((H + 7) / 8);
        CK(cudaMalloc((void **)&c->d_mi_map, nmi * 4), "alloc mode-info map");
        CK(cudaMemset(c->d_mi_map, 0, nmi * 4), "clear mode-info map");
    }
    uint32_t *t = malloc((size_t)c->n_sb * 4);
    if (!t) return CVP9_ERR_NOMEM;
    uint32_t n = 0;
    for (int d = 0; d < c->sb_cols + c->sb_rows - 1; d++)
        n += (uint32_t)cvp9_tickets_on_diagonal(c->sb_cols, c->sb_rows, 0, d, t + n);
    cudaError_t e = cudaMemcpy(c->d_tickets, t, (size_t)n * 4, cudaMemcpyHostToDevice);
    free(t);
    if (e != cudaSuccess) return fail(c, e, "upload tickets");
    c->n_tickets = n;
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c->device);
    int resident = dev_sms * cvp9_recon_ctas_per_sm(c->device, c->arith);
    c->resident_ctas = resident;
    c->recon_ctas = (int)n < resident ? (int)n : resident;
    c->epoch = 0;
    return CVP9_OK;
}

static cvp9_err_t grow_pinned(cuctx_t *c, void **p, size_t *cap, size_t need)
{
    if (*cap >= need) return CVP9_OK;
    cudaFreeHost(*p);
    *p = NULL;
    *cap = 0;
    size_t n = need + need / 4 + 4096;
    CK(cudaMallocHost(p, n), "pinned staging");
    *cap = n;
    return CVP9_OK;
}

static cvp9_err_t grow_device(cuctx_t *c, void **p, size_t *cap, size_t need)
{
    if (*cap >= need) return CVP9_OK;
    /* the previous user of this slot's buffer finished (slot not pending
     * and stream-ordered), so free is safe */
    cudaFree(*p);
    *p = NULL;
    *cap = 0;
    size_t n = need + need / 4 + 4096;
    CK(cudaMalloc(p, n), "device staging");
    *cap = n;
    return CVP9_OK;
}

/* A device frame no reference slot uses (stream order makes reuse safe). */
static int acquire_dframe(cuctx_t *c, int32_t W, int32_t H)
{
    size_t need = (size_t)W * H + 2 * (size_t)((W + 1) / 2) * ((H + 1) / 2);
    int pick = -1;
    for (int i = 0; i < MAX_DFRAMES; i++) {
        if (c->frames[i].users) continue;
        if (c->frames[i].dev && c->frames[i].cap >= need) { pick = i; break; }
        if (pick < 0) pick = i;
    }
    if (pick < 0) return -1;
    dframe_t *f = &c->frames[pick];
    if (!f->dev || f->cap < need) {
        if (f->dev) { cudaStreamSynchronize(c->stream); cudaFree(f->dev); }
        f->dev = NULL;
        f->cap = 0;
        if (cudaMalloc((void **)&f->dev, need) != cudaSuccess) return -1;
        f->cap = need;
    }
    f->w = W;
    f->h = H;
    return pick;
}

static void set_ref(cuctx_t *c, int slot, int frame)
{
    if (c->ref_slot[slot] >= 0) c->frames[c->ref_slot[slot]].users--;
    c->ref_slot[slot] = frame;
    if (frame >= 0) c->frames[frame].users++;
}

cvp9_err_t cuda_decode_frame(void *ctx, const vp9_parsed_frame_t *pf, int64_t pts)
{
    cuctx_t *c = (cuctx_t *)ctx;
    if (!c || !pf) return CVP9_ERR_INVALID_DATA;
    if (c->ring_count == CVP9_CUDA_INFLIGHT) return CVP9_ERR_AGAIN;
    int32_t W = (int32_t)pf->hdr.width, H = (int32_t)pf->hdr.height;
    if (W <= 0 || H <= 0 || W > 65535 || H > 65535) return CVP9_ERR_INVALID_DATA;
    if (pf->num_blocks && !pf->blocks) return CVP9_ERR_INVALID_DATA;
    if (pf->num_coeffs && !pf->coeffs) return CVP9_ERR_INVALID_DATA;
    const char *why = NULL;
    if (!cvp9_frame_supported(c->arith, pf, &why)) {
        snprintf(c->last_error, sizeof(c->last_error), "%s", why);
        return CVP9_ERR_UNSUPPORTED;
    }
    if (c->arith == CVP9_ARITH_FULL && pf->hdr.frame_type != VP9_FRAME_KEY && !pf->hdr.intra_only)
        for (int k = 0; k < 3; k++) {
            int f = c->ref_slot[pf->hdr.ref_frame_idx[k] & 7];
            if (f >= 0 && (c->frames[f].w != W || c->frames[f].h != H)) {
                snprintf(c->last_error, sizeof(c->last_error),
                         "reference %d is %dx%d: scaled motion compensation is not built", k,
                         (int)c->frames[f].w, (int)c->frames[f].h);
                return CVP9_ERR_UNSUPPORTED;
            }
        }
    if (cudaSetDevice(c->device) != cudaSuccess) return CVP9_ERR_GPU;

    cvp9_err_t err;
    if (W != c->W || H != c->H || !c->d_tickets) {
        if ((err = set_geometry(c, W, H)) != CVP9_OK) return err;
    }
    size_t nv12_need = (size_t)W * H + 2 * (size_t)((W + 1) / 2) * ((H + 1) / 2);
    if (c->pending_target && c->pending_target_size < nv12_need) return CVP9_ERR_INVALID_DATA;

    slot_t *s = &c->slots[(c->ring_head + c->ring_count) % CVP9_CUDA_INFLIGHT];
    size_t nbb = (size_t)pf->num_blocks * sizeof(vp9_macroblock_info_t);
    size_t ncb = (size_t)pf->num_coeffs * sizeof(int16_t);
    size_t outb = nv12_need;
    int ob = -1;
    for (int i = 0; i < OUTBUFS && ob < 0; i++)
        if (!c->outs[i].busy && c->outs[i].free_after <= c->decodes) ob = i;
    if (ob < 0) return fail(c, cudaErrorMemoryAllocation, "output buffers");
    outbuf_t *o = &c->outs[ob];
    if ((err = grow_pinned(c, &s->h_blocks, &s->h_blocks_cap, nbb ? nbb : 64)) ||
        (err = grow_pinned(c, &s->h_coeffs, &s->h_coeffs_cap, ncb ? ncb : 64)) ||
        (err = grow_pinned(c, (void **)&o->h, &o->cap, outb)) ||
        (err = grow_device(c, &s->d_blocks, &s->d_blocks_cap, nbb ? nbb : 64)) ||
        (err = grow_device(c, &s->d_coeffs, &s->d_coeffs_cap, ncb ? ncb : 64)))
        return err;
    /* the parser's arrays are borrowed for this call only: stage them now */
    if (nbb) cvp9_parallel_memcpy(s->h_blocks, pf->blocks, nbb);
    if (ncb) cvp9_parallel_memcpy(s->h_coeffs, pf->coeffs, ncb);

    int of = acquire_dframe(c, W, H);
    if (of < 0) return fail(c, cudaErrorMemoryAllocation, "frame pool");

    cvp9_job_t *job = s->h_job;
    memset(job, 0, sizeof(*job));
    cvp9_job_geometry(job, pf);
    const int full = c->arith == CVP9_ARITH_FULL;
    if (full) {
        cvp9_job_full(job, pf);
        job->mi_map = c->d_mi_map;
    }
    cvp9_tcfg_t tc;
    s->tune_idx = cvp9_tuner_pick(&c->tuner, cvp9_tune_key(c->arith, 1, (uint64_t)c->n_sb), 1, &tc);
    s->tune_cfg = tc;
    job->blocks = (const vp9_macroblock_info_t *)s->d_blocks;
    job->coeffs = (const int16_t *)s->d_coeffs;
    job->out = c->frames[of].dev;
    job->nv12 = (uint8_t *)c->pending_target;
    if (job->lf_tiled && !tc.lf32 && !(W & 3) && !job->nv12) job->lf_tiled = 2;   /* register strips */
    for (int i = 0; i < 8; i++) {
        int f = c->ref_slot[i];
        if (f >= 0) {
            job->ref[i].plane = c->frames[f].dev;
            job->ref[i].w = c->frames[f].w;
            job->ref[i].h = c->frames[f].h;
        }
    }
    job->epoch = ++c->epoch;
    job->sb_range = c->d_sb_range;
    job->sb_done = c->d_sb_done;
    job->status = c->d_misc;

    cudaStream_t st = c->stream;
    CK(cudaEventRecord(s->ev_start, st), "event");
    if (nbb) CK(cudaMemcpyAsync(s->d_blocks, s->h_blocks, nbb, cudaMemcpyHostToDevice, st), "upload blocks");
    if (ncb) CK(cudaMemcpyAsync(s->d_coeffs, s->h_coeffs, ncb, cudaMemcpyHostToDevice, st), "upload coeffs");
    CK(cudaMemcpyAsync(s->d_job, job, sizeof(*job), cudaMemcpyHostToDevice, st), "upload job");
    CK(cudaMemsetAsync(c->d_sb_range, 0, (size_t)c->n_sb * 16, st), "clear sb_range");
    CK(cudaMemsetAsync(c->d_misc, 0, 12, st), "clear status");
    CK(cudaEventRecord(s->ev_k0, st), "event");

    cvp9k_launch_t L;
    memset(&L, 0, sizeof(L));
    L.jobs = s->d_job;
    L.njobs = 1;
    L.arith = full ? CVP9_ARITH_SPEC : c->arith;
    L.max_blocks = (int)pf->num_blocks;
    L.tickets = c->d_tickets;
    L.n_tickets = c->n_tickets;
    L.ticket_counter = c->d_misc + 1;
    L.recon_ctas = tc.half ? (c->recon_ctas + 1) / 2 : c->recon_ctas;
    L.lf_tile_h = tc.lf32 ? 32 : 64;
    L.warp_levels = cvp9_env_recon_warp();
    if (tc.inter) {
        L.general = c->d_fast;
        L.general_tickets = c->d_fast + c->n_sb;
        L.n_general = c->d_fast + 2 * c->n_sb;
        L.inter_variant = tc.inter;
    }
    if (full) {
        L.full = 1;
        L.lf_counter = c->d_misc + 2;
        L.lf_tickets = (uint32_t)c->sb_rows;
        L.lf_ctas = c->sb_rows;
        L.full_nv12_max_px = job->nv12 ? W * H : 0;
    } else if (job->lf_tiled == 2) {
        L.lf_strips_x = ((W + 4 + 7) / 8 + 127) / 128;
        L.lf_strips_y = (H + 4 + 15) / 16;
    } else if (job->lf_tiled) {
        L.lf_tiles_x = (W + 4 + 63) / 64;
        L.lf_tiles_y = (H + 4 + 63) / 64;
    } else {
        L.flat_lf_max_w = W;
        L.flat_lf_max_h = H;
        L.flat_nv12 = job->nv12 != NULL;
    }
    int lrc = cvp9k_launch_frame(&L, st);
    if (lrc != 0) return fail(c, (cudaError_t)lrc, "launch");
    CK(cudaEventRecord(s->ev_k1, st), "event");
    CK(cudaMemcpyAsync(o->h, c->frames[of].dev, outb, cudaMemcpyDeviceToHost, st), "download frame");
    CK(cudaMemcpyAsync(s->h_status, c->d_misc, 4, cudaMemcpyDeviceToHost, st), "download status");
    CK(cudaEventRecord(s->ev_end, st), "event");

    /* reference pool update (host bookkeeping; stream order protects reuse) */
    if (c->arith != CVP9_ARITH_REFCPU) {
        unsigned refresh = pf->hdr.refresh_frame_flags ? pf->hdr.refresh_frame_flags : 0x01u;
        for (int i = 0; i < 8; i++) if (refresh & (1u << i)) set_ref(c, i, of);
    } else if (pf->hdr.frame_type == VP9_FRAME_KEY) {
        for (int i = 0; i < 8; i++) set_ref(c, i, of);
    } else {
        set_ref(c, 0, of);
    }

    c->pending_target = NULL;
    c->pending_target_size = 0;
    s->pending = 1;
    s->out = ob;
    o->busy = 1;
    c->decodes++;
    s->pts = pts;
    s->w = W;
    s->h = H;
    c->ring_count++;
    return CVP9_OK;
}

static cvp9_err_t wait_event(cuctx_t *c, cudaEvent_t ev)
{
    double t0 = cvp9_now();
    for (;;) {
        cudaError_t e = cudaEventQuery(ev);
        if (e == cudaSuccess) return CVP9_OK;
        if (e != cudaErrorNotReady) return fail(c, e, "frame completion");
        if (cvp9_now() - t0 > WAIT_LIMIT_S) {
            snprintf(c->last_error, sizeof(c->last_error), "frame did not complete within %.0f s", WAIT_LIMIT_S);
            return CVP9_ERR_GPU;
        }
        struct timespec ts = { 0, 20000 };
        nanosleep(&ts, NULL);
    }
}

cvp9_err_t cuda_get_frame(void *ctx, cvp9_frame_info_t *info, int wait)
{
    cuctx_t *c = (cuctx_t *)ctx;
    if (!c || !info) return CVP9_ERR_INVALID_DATA;
    if (c->ring_count == 0) return CVP9_ERR_UNSUPPORTED;
    slot_t *s = &c->slots[c->ring_head];
    if (!wait && c->ring_count < CVP9_CUDA_INFLIGHT) {
        cudaError_t e = cudaEventQuery(s->ev_end);
        if (e == cudaErrorNotReady) return CVP9_ERR_AGAIN;
        if (e != cudaSuccess) return fail(c, e, "frame completion");
    } else {
        cvp9_err_t err = wait_event(c, s->ev_end);
        if (err != CVP9_OK) return err;
    }
    s->pending = 0;
    c->ring_head = (c->ring_head + 1) % CVP9_CUDA_INFLIGHT;
    c->ring_count--;
    outbuf_t *o = &c->outs[s->out];
    o->busy = 0;
    o->free_after = c->decodes + 2;     /* untouched by the next two decodes */

    float t = 0.f, k = 0.f;
    cudaEventElapsedTime(&t, s->ev_start, s->ev_end);
    cudaEventElapsedTime(&k, s->ev_k0, s->ev_k1);
    c->last_total_ms = t;
    c->last_kernel_ms = k;
    cvp9_tuner_report(&c->tuner, s->tune_idx, s->tune_cfg, k);

    uint32_t status = *s->h_status;
    if (status & (CVP9_JOB_BAD_BLOCK | CVP9_JOB_BAD_ORDER | CVP9_JOB_TOO_MANY)) {
        snprintf(c->last_error, sizeof(c->last_error), "block layout rejected on device (status 0x%x)", status);
        return CVP9_ERR_INVALID_DATA;
    }
    if (status & CVP9_JOB_TIMEOUT) {
        snprintf(c->last_error, sizeof(c->last_error), "wavefront wait expired on device");
        return CVP9_ERR_GPU;
    }

    uint32_t w = (uint32_t)s->w, h = (uint32_t)s->h, cw = (w + 1) / 2, ch = (h + 1) / 2;
    info->width = w;
    info->height = h;
    info->stride_y = w;
    info->stride_uv = cw;
    info->plane_y = o->h;
    info->plane_u = o->h + (size_t)w * h;
    info->plane_v = o->h + (size_t)w * h + (size_t)cw * ch;
    info->pts = s->pts;
    return CVP9_OK;
}

cvp9_err_t cuda_get_frame_dmabuf(void *ctx, cvp9_dmabuf_frame_t *out)
{
    (void)ctx;
    (void)out;
    return CVP9_ERR_UNSUPPORTED;
}

cvp9_err_t cuda_export_buffer_alloc(void *ctx, uint64_t size, cvp9_export_buffer_t *out)
{
    cuctx_t *c = (cuctx_t *)ctx;
    if (!c || !out || size == 0) return CVP9_ERR_INVALID_DATA;
    if (cudaSetDevice(c->device) != cudaSuccess) return CVP9_ERR_GPU;
    void *h = NULL, *d = NULL;
    cudaError_t e = cudaHostAlloc(&h, (size_t)size, cudaHostAllocMapped | cudaHostAllocPortable);
    if (e != cudaSuccess) return fail(c, e, "export buffer");
    e = cudaHostGetDevicePointer(&d, h, 0);
    if (e != cudaSuccess) { cudaFreeHost(h); return fail(c, e, "export buffer mapping"); }
    memset(out, 0, sizeof(*out));
    out->fd = -1;
    out->mapped = h;
    out->size = size;
    out->priv_buf = d;
    out->priv_mem = h;
    return CVP9_OK;
}

void cuda_export_buffer_free(void *ctx, cvp9_export_buffer_t *buf)
{
    cuctx_t *c = (cuctx_t *)ctx;
    if (!c || !buf || !buf->priv_mem) return;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    if (c->pending_target == buf->priv_buf) c->pending_target = NULL;
    cudaFreeHost(buf->priv_mem);
    memset(buf, 0, sizeof(*buf));
    buf->fd = -1;
}

cvp9_err_t cuda_set_render_target(void *ctx, const cvp9_export_buffer_t *target)
{
    cuctx_t *c = (cuctx_t *)ctx;
    if (!c) return CVP9_ERR_INVALID_DATA;
    if (!target) {
        c->pending_target = NULL;
        c->pending_target_size = 0;
        return CVP9_OK;
    }
    if (!target->priv_buf) return CVP9_ERR_UNSUPPORTED;
    c->pending_target = target->priv_buf;
    c->pending_target_size = target->size;
    return CVP9_OK;
}

cvp9_err_t cuda_backend_last_timing(void *ctx, float *total_ms, float *kernels_ms)
{
    cuctx_t *c = (cuctx_t *)ctx;
    if (!c) return CVP9_ERR_INVALID_DATA;
    if (total_ms) *total_ms = c->last_total_ms;
    if (kernels_ms) *kernels_ms = c->last_kernel_ms;
    return CVP9_OK;
}

const char *cuda_backend_last_error(void *ctx)
{
    cuctx_t *c = (cuctx_t *)ctx;
    return c ? c->last_error : "";
}

cvp9_err_t cuda_backend_selftest_wait_limit(int device, uint32_t *status, float *ms)
{
    if (!status || !ms) return CVP9_ERR_INVALID_DATA;
    *status = 0;
    *ms = 0.f;
    if (device < 0) device = cvp9_env_device();
    if (cudaSetDevice(device) != cudaSuccess || cvp9_device_setup(device) != 0) return CVP9_ERR_NO_BACKEND;
    const int W = 128, H = 64;
    vp9_macroblock_info_t blk[2];
    memset(blk, 0, sizeof(blk));
    blk[0].x = 0;  blk[0].width = 64; blk[0].height = 64; blk[0].tx_size = 3;
    blk[0].ref_frame[0] = 1; blk[0].skip = 1;            /* inter, left SB   */
    blk[1].x = 64; blk[1].width = 64; blk[1].height = 64; blk[1].tx_size = 3;
    blk[1].is_intra = 1; blk[1].skip = 1;                /* intra, right SB  */
    const size_t fb = (size_t)W * H + 2 * (size_t)(W / 2) * (H / 2);
    const uint32_t ticket = 1u;                          /* job 0, SB 1 only */
    vp9_macroblock_info_t *d_blk = NULL;
    uint8_t *d_out = NULL;
    uint32_t *d_u32 = NULL;                              /* sb_range 8, sb_done 2, status 1, counter 1, ticket 1 */
    cvp9_job_t *d_job = NULL;
    cudaEvent_t e0 = NULL, e1 = NULL;
    cvp9_err_t rc = CVP9_ERR_GPU;
    if (cudaMalloc((void **)&d_blk, sizeof(blk)) != cudaSuccess ||
        cudaMalloc((void **)&d_out, fb) != cudaSuccess ||
        cudaMalloc((void **)&d_u32, 13 * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc((void **)&d_job, sizeof(cvp9_job_t)) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        goto done;
    {
        cvp9_job_t job;
        memset(&job, 0, sizeof(job));
        job.W = W; job.H = H; job.CW = W / 2; job.CH = H / 2;
        job.sb_cols = 2; job.sb_rows = 1; job.mi_cols = W / 8; job.mi_rows = H / 8;
        job.blocks = d_blk; job.num_blocks = 2;
        job.coeffs = NULL; job.num_coeffs = 0;
        job.out = d_out;
        job.lf_level = 0; job.lf_tiled = 1;
        job.epoch = 1;
        job.sb_range = d_u32;
        job.sb_done = d_u32 + 8;
        job.status = d_u32 + 10;
        if (cudaMemcpy(d_blk, blk, sizeof(blk), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemset(d_u32, 0, 13 * sizeof(uint32_t)) != cudaSuccess ||
            cudaMemcpy(d_u32 + 12, &ticket, 4, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(d_job, &job, sizeof(job), cudaMemcpyHostToDevice) != cudaSuccess)
            goto done;
        cvp9k_launch_t L;
        memset(&L, 0, sizeof(L));
        L.jobs = d_job;
        L.njobs = 1;
        L.arith = CVP9_ARITH_REFCPU;
        L.max_blocks = 2;
        L.tickets = d_u32 + 12;
        L.n_tickets = 1;
        L.ticket_counter = d_u32 + 11;
        L.recon_ctas = 1;
        if (cudaEventRecord(e0, 0) != cudaSuccess || cvp9k_launch_frame(&L, 0) != 0 ||
            cudaEventRecord(e1, 0) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess)
            goto done;
        cudaEventElapsedTime(ms, e0, e1);
        if (cudaMemcpy(status, d_u32 + 10, 4, cudaMemcpyDeviceToHost) != cudaSuccess) goto done;
        rc = CVP9_OK;
    }
done:
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(d_blk);
    cudaFree(d_out);
    cudaFree(d_u32);
    cudaFree(d_job);
    return rc;
}
