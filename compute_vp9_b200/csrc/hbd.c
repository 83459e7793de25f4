/*
 * hbd.c — the profile 2 (10-bit) engine of include/cvp9_hbd.h.
 *
 * Per stream: nine device frame buffers (the eight reference slots can hold
 * at most eight distinct frames, so one is always free for the next
 * output), the superblock done flags and ranges, the loop filter's
 * mode-info map and a page-locked host frame for the download. Per step:
 * the block records and coefficients are uploaded (or taken as device
 * pointers), the jobs and the SB-diagonal ticket list go up, and one launch
 * chain runs k_scan_blocks, k_lf_mimap, k_hbd_recon and
 * k_lf_full<uint16_t> over every frame of the step; the frames come back
 * one copy each.
 */
#include "cvp9_hbd.h"
#include "backend_common.h"
#include "recon_launch.h"

#include <cuda_runtime_api.h>
#include <stdlib.h>
#include <string.h>

#define HBD_NBUF 9

typedef struct {
    int       open;
    uint32_t  W, H;
    size_t    frame_bytes;             /* 2 * (W*H + 2*CW*CH)                     */
    int       n_sb, n_mi;
    uint8_t  *buf[HBD_NBUF];           /* device frames                           */
    int       slot[8];                 /* reference slot -> buffer, -1 empty      */
    int       latest;                  /* buffer of the last delivered frame      */
    uint32_t *d_sb_range, *d_sb_done, *d_mi_map;
    uint32_t  epoch;
    uint16_t *h_out;                   /* page-locked copy of the latest frame    */
    int       have_out;
    int64_t   pts;
} hbd_stream_t;

struct cvp9_hbd {
    int            device, sms, recon_ctas, lf_ctas;
    cudaStream_t   st;
    cudaEvent_t    ev[6];
    hbd_stream_t  *s;
    int            ns, cap;
    /* step buffers (grow only) */
    cvp9_job_t    *h_jobs, *d_jobs;
    int            jobs_cap;
    uint32_t      *h_tickets, *d_tickets;
    size_t         tickets_cap;
    uint32_t      *d_words;            /* ticket counter, lf counter, status per job */
    uint32_t      *h_status;
    int            words_cap;
    uint8_t       *d_in;               /* uploaded blocks and coefficients          */
    size_t         in_cap;
    int            pending, pending_n, step_flags;
    int            err;                /* status of a step that completed inside a submit */
    int            pending_sid[1024];
    int64_t        pending_pts[1024];
    float          ms[5];
};

static int grow_dev(void **p, size_t *cap, size_t need)
{
    if (*cap >= need) return 0;
    if (*p) cudaFree(*p);
    *p = NULL;
    *cap = 0;
    if (cudaMalloc(p, need) != cudaSuccess) { *p = NULL; return -1; }
    *cap = need;
    return 0;
}

int cvp9_hbd_create(int device, cvp9_hbd_t **out)
{
    if (!out) return CVP9_ERR_INVALID_DATA;
    *out = NULL;
    if (device < 0) device = cvp9_env_device();
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device >= ndev || cvp9_device_setup(device) != 0)
        return CVP9_ERR_NO_BACKEND;
    cvp9_hbd_t *h = calloc(1, sizeof(*h));
    if (!h) return CVP9_ERR_NOMEM;
    h->device = device;
    cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, device);
    int per = cvp9k_hbd_ctas_per_sm();
    h->recon_ctas = h->sms * (per > 0 ? per : 1);
    h->lf_ctas = h->sms * cvp9_lf_full_ctas_per_sm(device);
    if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) { free(h); return CVP9_ERR_GPU; }
    for (int i = 0; i < 6; i++)
        if (cudaEventCreate(&h->ev[i]) != cudaSuccess) { cvp9_hbd_destroy(h); return CVP9_ERR_GPU; }
    *out = h;
    return CVP9_OK;
}

static void stream_free(hbd_stream_t *s)
{
    for (int i = 0; i < HBD_NBUF; i++) if (s->buf[i]) cudaFree(s->buf[i]);
    if (s->d_sb_range) cudaFree(s->d_sb_range);
    if (s->d_sb_done) cudaFree(s->d_sb_done);
    if (s->d_mi_map) cudaFree(s->d_mi_map);
    if (s->h_out) cudaFreeHost(s->h_out);
    memset(s, 0, sizeof(*s));
}

void cvp9_hbd_destroy(cvp9_hbd_t *h)
{
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->st) cudaStreamSynchronize(h->st);
    for (int i = 0; i < h->ns; i++) stream_free(&h->s[i]);
    free(h->s);
    if (h->d_jobs) cudaFree(h->d_jobs);
    if (h->h_jobs) cudaFreeHost(h->h_jobs);
    if (h->d_tickets) cudaFree(h->d_tickets);
    if (h->h_tickets) cudaFreeHost(h->h_tickets);
    if (h->d_words) cudaFree(h->d_words);
    if (h->h_status) cudaFreeHost(h->h_status);
    if (h->d_in) cudaFree(h->d_in);
    for (int i = 0; i < 6; i++) if (h->ev[i]) cudaEventDestroy(h->ev[i]);
    if (h->st) cudaStreamDestroy(h->st);
    free(h);
}

int cvp9_hbd_open_stream(cvp9_hbd_t *h, uint32_t width, uint32_t height)
{
    if (!h || width == 0 || height == 0 || (width & 7) || (height & 7) || width > 16384 || height > 16384)
        return CVP9_ERR_UNSUPPORTED;
    cudaSetDevice(h->device);
    int sid = -1;
    for (int i = 0; i < h->ns; i++) if (!h->s[i].open) { sid = i; break; }
    if (sid < 0) {
        if (h->ns == h->cap) {
            int nc = h->cap ? 2 * h->cap : 16;
            hbd_stream_t *ns = realloc(h->s, (size_t)nc * sizeof(*ns));
            if (!ns) return CVP9_ERR_NOMEM;
            memset(ns + h->cap, 0, (size_t)(nc - h->cap) * sizeof(*ns));
            h->s = ns;
            h->cap = nc;
        }
        sid = h->ns++;
    }
    hbd_stream_t *s = &h->s[sid];
    memset(s, 0, sizeof(*s));
    s->W = width;
    s->H = height;
    const size_t cw = (width + 1) / 2, ch = (height + 1) / 2;
    s->frame_bytes = 2 * ((size_t)width * height + 2 * cw * ch);
    s->n_sb = (int)(((width + 63) / 64) * ((height + 63) / 64));
    s->n_mi = (int)((width / 8) * (height / 8));
    int ok = 1;
    for (int i = 0; i < HBD_NBUF && ok; i++) ok = cudaMalloc((void **)&s->buf[i], s->frame_bytes) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&s->d_sb_range, (size_t)s->n_sb * 16) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&s->d_sb_done, (size_t)s->n_sb * 4) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&s->d_mi_map, (size_t)s->n_mi * 4) == cudaSuccess;
    ok = ok && cudaHostAlloc((void **)&s->h_out, s->frame_bytes, cudaHostAllocDefault) == cudaSuccess;
    /* done flags and mode-info tags compare against the stream's epoch */
    ok = ok && cudaMemset(s->d_sb_done, 0, (size_t)s->n_sb * 4) == cudaSuccess;
    ok = ok && cudaMemset(s->d_mi_map, 0, (size_t)s->n_mi * 4) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        stream_free(s);
        return CVP9_ERR_NOMEM;
    }
    for (int i = 0; i < 8; i++) s->slot[i] = -1;
    s->latest = -1;
    s->open = 1;
    return sid;
}

int cvp9_hbd_close_stream(cvp9_hbd_t *h, int sid)
{
    if (!h || sid < 0 || sid >= h->ns || !h->s[sid].open) return CVP9_ERR_INVALID_DATA;
    cudaSetDevice(h->device);
    cvp9_hbd_wait(h);
    stream_free(&h->s[sid]);
    return CVP9_OK;
}

static int frame_check(const hbd_stream_t *s, const vp9_parsed_frame_t *pf)
{
    const vp9_frame_header_t *hd = &pf->hdr;
    if (hd->bit_depth != 10 || hd->width != s->W || hd->height != s->H) return CVP9_ERR_UNSUPPORTED;
    const int inter = hd->frame_type != VP9_FRAME_KEY && !hd->intra_only;
    if (inter && (int)hd->interp_filter > VP9_FILTER_BILINEAR) return CVP9_ERR_UNSUPPORTED;
    return CVP9_OK;
}

/* Complete the step in flight: status, deliveries, times. */
static int finish_step(cvp9_hbd_t *h)
{
    if (!h->pending) return CVP9_OK;
    h->pending = 0;
    if (cudaStreamSynchronize(h->st) != cudaSuccess) return CVP9_ERR_GPU;
    int rc = CVP9_OK;
    for (int i = 0; i < h->pending_n; i++) {
        hbd_stream_t *s = &h->s[h->pending_sid[i]];
        const uint32_t st = h->h_status[i];
        if (st & CVP9_JOB_TIMEOUT) rc = CVP9_ERR_GPU;
        else if (st && rc == CVP9_OK) rc = CVP9_ERR_INVALID_DATA;
        s->have_out = !st && !(h->step_flags & CVP9_HBD_NO_OUTPUT);
        s->pts = h->pending_pts[i];
    }
    float t[5] = {0};
    cudaEventElapsedTime(&t[0], h->ev[0], h->ev[1]);
    cudaEventElapsedTime(&t[1], h->ev[1], h->ev[2]);
    cudaEventElapsedTime(&t[2], h->ev[2], h->ev[3]);
    cudaEventElapsedTime(&t[3], h->ev[3], h->ev[4]);
    cudaEventElapsedTime(&t[4], h->ev[4], h->ev[5]);
    memcpy(h->ms, t, sizeof(t));
    return rc;
}

int cvp9_hbd_wait(cvp9_hbd_t *h)
{
    if (!h) return CVP9_ERR_INVALID_DATA;
    cudaSetDevice(h->device);
    int rc = finish_step(h);
    if (rc == CVP9_OK) rc = h->err;
    h->err = CVP9_OK;
    return rc;
}

static int submit_step(cvp9_hbd_t *h, int n, const int *sids, const cvp9_hbd_frame_t *frames,
                       const cvp9_hbd_coeff_list_t *lists, const int64_t *pts, unsigned flags)
{
    if (!h || n <= 0 || n > 1024 || !sids || !frames) return CVP9_ERR_INVALID_DATA;
    cudaSetDevice(h->device);
    const int prev = finish_step(h);
    if (prev != CVP9_OK && h->err == CVP9_OK) h->err = prev;
    for (int i = 0; i < n; i++) {
        const int sid = sids[i];
        if (sid < 0 || sid >= h->ns || !h->s[sid].open || !frames[i].pf) return CVP9_ERR_INVALID_DATA;
        for (int k = 0; k < i; k++) if (sids[k] == sid) return CVP9_ERR_INVALID_DATA;
        const vp9_parsed_frame_t *pf = frames[i].pf;
        int c = frame_check(&h->s[sid], pf);
        if (c != CVP9_OK) return c;
        if (pf->num_blocks && !pf->blocks) return CVP9_ERR_INVALID_DATA;
        if (!lists && pf->num_coeffs && !frames[i].coeffs) return CVP9_ERR_INVALID_DATA;
        if (lists && lists[i].n && (!lists[i].pos || !lists[i].val)) return CVP9_ERR_INVALID_DATA;
    }
    /* step buffers */
    size_t in_bytes = 0;
    size_t ntk = 0;
    int max_blocks = 0, max_sb_rows = 0;
    uint32_t max_n = 0;
    for (int i = 0; i < n; i++) {
        const vp9_parsed_frame_t *pf = frames[i].pf;
        if (!(flags & CVP9_HBD_DEVICE_INPUTS))
            in_bytes += (((size_t)pf->num_blocks * sizeof(vp9_macroblock_info_t) + 255) & ~(size_t)255) +
                        (((size_t)pf->num_coeffs * 4 + 255) & ~(size_t)255);
        if (lists) {
            /* the lists, and the dense array they are scattered into */
            in_bytes += 2 * (((size_t)lists[i].n * 4 + 255) & ~(size_t)255);
            if (flags & CVP9_HBD_DEVICE_INPUTS) in_bytes += ((size_t)pf->num_coeffs * 4 + 255) & ~(size_t)255;
            if (lists[i].n > max_n) max_n = lists[i].n;
        }
        const hbd_stream_t *s = &h->s[sids[i]];
        ntk += (size_t)s->n_sb;
        if ((int)pf->num_blocks > max_blocks) max_blocks = (int)pf->num_blocks;
        const int rows = (int)((s->H + 63) / 64);
        if (rows > max_sb_rows) max_sb_rows = rows;
    }
    if (n > h->jobs_cap) {
        if (h->d_jobs) cudaFree(h->d_jobs);
        if (h->h_jobs) cudaFreeHost(h->h_jobs);
        h->d_jobs = NULL;
        h->h_jobs = NULL;
        h->jobs_cap = 0;
        if (cudaMalloc((void **)&h->d_jobs, (size_t)n * sizeof(cvp9_job_t)) != cudaSuccess ||
            cudaHostAlloc((void **)&h->h_jobs, (size_t)n * sizeof(cvp9_job_t), cudaHostAllocDefault) != cudaSuccess)
            return CVP9_ERR_NOMEM;
        h->jobs_cap = n;
    }
    if (ntk > h->tickets_cap) {
        if (h->d_tickets) cudaFree(h->d_tickets);
        if (h->h_tickets) cudaFreeHost(h->h_tickets);
        h->d_tickets = NULL;
        h->h_tickets = NULL;
        h->tickets_cap = 0;
        if (cudaMalloc((void **)&h->d_tickets, ntk * 4) != cudaSuccess ||
            cudaHostAlloc((void **)&h->h_tickets, ntk * 4, cudaHostAllocDefault) != cudaSuccess)
            return CVP9_ERR_NOMEM;
        h->tickets_cap = ntk;
    }
    if (n + 2 > h->words_cap) {
        if (h->d_words) cudaFree(h->d_words);
        if (h->h_status) cudaFreeHost(h->h_status);
        h->d_words = NULL;
        h->h_status = NULL;
        h->words_cap = 0;
        if (cudaMalloc((void **)&h->d_words, (size_t)(n + 2) * 4) != cudaSuccess ||
            cudaHostAlloc((void **)&h->h_status, (size_t)n * 4, cudaHostAllocDefault) != cudaSuccess)
            return CVP9_ERR_NOMEM;
        h->words_cap = n + 2;
    }
    if (in_bytes && grow_dev((void **)&h->d_in, &h->in_cap, in_bytes) != 0) return CVP9_ERR_NOMEM;

    cudaEventRecord(h->ev[0], h->st);
    /* uploads and jobs */
    size_t at = 0;
    for (int i = 0; i < n; i++) {
        hbd_stream_t *s = &h->s[sids[i]];
        const vp9_parsed_frame_t *pf = frames[i].pf;
        cvp9_job_t *job = &h->h_jobs[i];
        memset(job, 0, sizeof(*job));
        cvp9_job_geometry(job, pf);
        cvp9_job_full(job, pf);
        const vp9_macroblock_info_t *blocks = pf->blocks;
        const int32_t *coeffs = frames[i].coeffs;
        if (!(flags & CVP9_HBD_DEVICE_INPUTS)) {
            const size_t bb = (size_t)pf->num_blocks * sizeof(vp9_macroblock_info_t);
            const size_t cb = (size_t)pf->num_coeffs * 4;
            uint8_t *db = h->d_in + at;
            at += (bb + 255) & ~(size_t)255;
            uint8_t *dc = h->d_in + at;
            at += (cb + 255) & ~(size_t)255;
            if (bb && cudaMemcpyAsync(db, pf->blocks, bb, cudaMemcpyHostToDevice, h->st) != cudaSuccess)
                return CVP9_ERR_GPU;
            if (!lists && cb &&
                cudaMemcpyAsync(dc, frames[i].coeffs, cb, cudaMemcpyHostToDevice, h->st) != cudaSuccess)
                return CVP9_ERR_GPU;
            blocks = (const vp9_macroblock_info_t *)db;
            coeffs = (const int32_t *)dc;
        }
        if (lists) {
            const size_t cb = (size_t)pf->num_coeffs * 4, lb = (size_t)lists[i].n * 4;
            uint8_t *dc = (uint8_t *)coeffs;
            if (flags & CVP9_HBD_DEVICE_INPUTS) {
                dc = h->d_in + at;
                at += (cb + 255) & ~(size_t)255;
                coeffs = (const int32_t *)dc;
            }
            uint8_t *dp = h->d_in + at;
            at += (lb + 255) & ~(size_t)255;
            uint8_t *dv = h->d_in + at;
            at += (lb + 255) & ~(size_t)255;
            const int dev = (flags & CVP9_HBD_DEVICE_INPUTS) != 0;
            if ((cb && cudaMemsetAsync(dc, 0, cb, h->st) != cudaSuccess) ||
                (lb && cudaMemcpyAsync(dp, lists[i].pos, lb, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                       h->st) != cudaSuccess) ||
                (lb && cudaMemcpyAsync(dv, lists[i].val, lb, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                       h->st) != cudaSuccess))
                return CVP9_ERR_GPU;
            job->sp_pos = (const uint32_t *)dp;
            job->sp_val32 = (const int32_t *)dv;
            job->sp_n = lists[i].n;
        }
        job->blocks = blocks;
        job->coeffs = NULL;
        job->coeffs32 = coeffs;
        /* the output goes to a buffer no slot holds */
        int ob = -1;
        for (int b = 0; b < HBD_NBUF && ob < 0; b++) {
            int held = 0;
            for (int k = 0; k < 8; k++) held |= s->slot[k] == b;
            if (!held) ob = b;
        }
        job->out = s->buf[ob];
        for (int k = 0; k < 8; k++)
            if (s->slot[k] >= 0) {
                job->ref[k].plane = s->buf[s->slot[k]];
                job->ref[k].w = (int32_t)s->W;
                job->ref[k].h = (int32_t)s->H;
            }
        job->epoch = ++s->epoch;
        job->sb_range = s->d_sb_range;
        job->sb_done = s->d_sb_done;
        job->mi_map = s->d_mi_map;
        job->status = h->d_words + 2 + i;
        if (cudaMemsetAsync(s->d_sb_range, 0, (size_t)s->n_sb * 16, h->st) != cudaSuccess) return CVP9_ERR_GPU;
        /* pool: the slots refresh_frame_flags names take the new frame */
        const unsigned refresh = pf->hdr.refresh_frame_flags ? pf->hdr.refresh_frame_flags : 0x01u;
        for (int k = 0; k < 8; k++) if (refresh & (1u << k)) s->slot[k] = ob;
        s->latest = ob;
        h->pending_sid[i] = sids[i];
        h->pending_pts[i] = pts ? pts[i] : 0;
    }
    /* tickets: superblock diagonals, the step's frames interleaved */
    uint32_t nt = 0;
    int maxd = 0;
    for (int i = 0; i < n; i++) {
        const hbd_stream_t *s = &h->s[sids[i]];
        const int d = (int)((s->W + 63) / 64 + (s->H + 63) / 64 - 2);
        if (d > maxd) maxd = d;
    }
    for (int d = 0; d <= maxd; d++)
        for (int i = 0; i < n; i++) {
            const hbd_stream_t *s = &h->s[sids[i]];
            nt += (uint32_t)cvp9_tickets_on_diagonal((int)((s->W + 63) / 64), (int)((s->H + 63) / 64), i, d,
                                                     h->h_tickets + nt);
        }
    if (cudaMemcpyAsync(h->d_jobs, h->h_jobs, (size_t)n * sizeof(cvp9_job_t), cudaMemcpyHostToDevice, h->st) !=
            cudaSuccess ||
        cudaMemcpyAsync(h->d_tickets, h->h_tickets, (size_t)nt * 4, cudaMemcpyHostToDevice, h->st) != cudaSuccess ||
        cudaMemsetAsync(h->d_words, 0, (size_t)(n + 2) * 4, h->st) != cudaSuccess)
        return CVP9_ERR_GPU;
    if (lists && cvp9k_launch_scatter(h->d_jobs, n, max_n, h->st) != 0) return CVP9_ERR_GPU;

    cvp9k_launch_t L;
    memset(&L, 0, sizeof(L));
    L.jobs = h->d_jobs;
    L.njobs = n;
    L.arith = CVP9_ARITH_FULL;
    L.full = 1;
    L.hbd = 1;
    L.max_blocks = max_blocks;
    L.tickets = h->d_tickets;
    L.n_tickets = nt;
    L.ticket_counter = h->d_words;
    L.recon_ctas = h->recon_ctas;
    L.lf_counter = h->d_words + 1;
    L.lf_tickets = (uint32_t)(n * max_sb_rows);
    L.lf_ctas = h->lf_ctas;
    L.ev[0] = h->ev[1];
    L.ev[1] = h->ev[2];
    L.ev[2] = h->ev[3];
    L.ev[3] = h->ev[4];
    if (cvp9k_launch_frame(&L, h->st) != 0) return CVP9_ERR_GPU;
    if (cudaMemcpyAsync(h->h_status, h->d_words + 2, (size_t)n * 4, cudaMemcpyDeviceToHost, h->st) != cudaSuccess)
        return CVP9_ERR_GPU;
    if (!(flags & CVP9_HBD_NO_OUTPUT))
        for (int i = 0; i < n; i++) {
            hbd_stream_t *s = &h->s[sids[i]];
            if (cudaMemcpyAsync(s->h_out, s->buf[s->latest], s->frame_bytes, cudaMemcpyDeviceToHost, h->st) !=
                cudaSuccess)
                return CVP9_ERR_GPU;
        }
    cudaEventRecord(h->ev[5], h->st);
    h->pending = 1;
    h->pending_n = n;
    h->step_flags = (int)flags;
    return CVP9_OK;
}

int cvp9_hbd_submit(cvp9_hbd_t *h, int n, const int *sids, const cvp9_hbd_frame_t *frames,
                    const int64_t *pts, unsigned flags)
{
    return submit_step(h, n, sids, frames, NULL, pts, flags);
}

int cvp9_hbd_submit_sparse(cvp9_hbd_t *h, int n, const int *sids, const cvp9_hbd_frame_t *frames,
                           const cvp9_hbd_coeff_list_t *lists, const int64_t *pts, unsigned flags)
{
    if (!lists) return CVP9_ERR_INVALID_DATA;
    return submit_step(h, n, sids, frames, lists, pts, flags);
}

int cvp9_hbd_get_frame(cvp9_hbd_t *h, int sid, cvp9_hbd_frame_info_t *info)
{
    if (!h || !info || sid < 0 || sid >= h->ns || !h->s[sid].open) return CVP9_ERR_INVALID_DATA;
    cudaSetDevice(h->device);
    const int rc = finish_step(h);
    if (rc != CVP9_OK && h->err == CVP9_OK) h->err = rc;
    hbd_stream_t *s = &h->s[sid];
    if (!s->have_out) return CVP9_ERR_UNSUPPORTED;
    const uint32_t cw = (s->W + 1) / 2, ch = (s->H + 1) / 2;
    info->width = s->W;
    info->height = s->H;
    info->stride_y = s->W;
    info->stride_uv = cw;
    info->plane_y = s->h_out;
    info->plane_u = s->h_out + (size_t)s->W * s->H;
    info->plane_v = info->plane_u + (size_t)cw * ch;
    info->pts = s->pts;
    return CVP9_OK;
}

int cvp9_hbd_step_times(cvp9_hbd_t *h, float ms[5])
{
    if (!h || !ms) return CVP9_ERR_INVALID_DATA;
    memcpy(ms, h->ms, sizeof(h->ms));
    return CVP9_OK;
}
