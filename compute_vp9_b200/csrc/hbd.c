/*
 * hbd.c — the profile 2 (10-bit) engine of include/cvp9_hbd.h.
 *
 * Per stream: ten device frame buffers (the eight reference slots hold at
 * most eight distinct frames and at most one more can still be on its way
 * to the host, so one is always free for the next output), the superblock
 * done flags and ranges, the loop filter's mode-info map and two
 * page-locked host frames (one per step slot) for the downloads.
 *
 * Two step slots keep two steps in flight on three CUDA streams: a step's
 * inputs go up on the upload stream, its launch chain (k_scan_blocks,
 * k_lf_mimap, k_hbd_recon, k_lf_full<uint16_t>) runs on the kernel stream
 * in submission order — a stream's next frame reads this one as a
 * reference and reuses its per-stream scratch — and its frames come down on
 * the download stream, so the download of one step, the kernels of the
 * next and the upload of the one after can overlap. A slot is reused once
 * its previous step has completed.
 */
#include "cvp9_hbd.h"
#include "backend_common.h"
#include "recon_launch.h"

#include <cuda_runtime_api.h>
#include <stdlib.h>
#include <string.h>

#define HBD_NBUF 10
#define HBD_SLOTS 2
#define HBD_MAX_STEP 1024

typedef struct {
    int       open;
    uint32_t  W, H;
    size_t    frame_bytes;             /* 2 * (W*H + 2*CW*CH)                        */
    int       n_sb, n_mi;
    uint8_t  *buf[HBD_NBUF];           /* device frames                              */
    int       slot[8];                 /* reference slot -> buffer, -1 empty         */
    int       dl_buf[HBD_SLOTS];       /* buffer each step slot downloads, -1 none   */
    uint32_t *d_sb_range, *d_sb_done, *d_mi_map;
    uint32_t  epoch;
    uint16_t *h_out[HBD_SLOTS];        /* page-locked frames, one per step slot      */
    int       out_slot;                /* step slot holding the latest delivered frame, -1 none */
    int64_t   pts;
} hbd_stream_t;

typedef struct {
    cvp9_job_t *h_jobs, *d_jobs;
    size_t      jobs_cap;              /* bytes                                      */
    uint32_t   *h_tickets, *d_tickets;
    size_t      tickets_cap;           /* bytes                                      */
    uint32_t   *d_words;               /* ticket counter, lf counter, status per job */
    uint32_t   *h_status;
    size_t      words_cap;             /* bytes                                      */
    uint8_t    *d_in;                  /* uploaded blocks, coefficients and lists    */
    size_t      in_cap;
    cudaEvent_t ev[6];                 /* start, scan, recon, filter, kernels done, downloaded */
    cudaEvent_t ev_up;                 /* inputs on the device                       */
    int         pending, n, flags;
    int         sid[HBD_MAX_STEP];
    int64_t     pts[HBD_MAX_STEP];
} hbd_slot_t;

struct cvp9_hbd {
    int            device, sms, recon_ctas, lf_ctas;
    cudaStream_t   st_up, st_k, st_dn;
    hbd_slot_t     slot[HBD_SLOTS];
    uint64_t       next_seq;           /* steps submitted                            */
    hbd_stream_t  *s;
    int            ns, cap;
    int            err;                /* first failure of a step completed inside a submit */
    float          ms[5];
    cudaEvent_t    t_start, t_stop;
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

/* A device buffer and its page-locked host twin, grown together. */
static int grow_pair(void **d, void **hst, size_t *cap, size_t need)
{
    if (*cap >= need) return 0;
    if (*d) cudaFree(*d);
    if (*hst) cudaFreeHost(*hst);
    *d = *hst = NULL;
    *cap = 0;
    if (cudaMalloc(d, need) != cudaSuccess || cudaHostAlloc(hst, need, cudaHostAllocDefault) != cudaSuccess) return -1;
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
    int ok = cudaStreamCreateWithFlags(&h->st_up, cudaStreamNonBlocking) == cudaSuccess &&
             cudaStreamCreateWithFlags(&h->st_k, cudaStreamNonBlocking) == cudaSuccess &&
             cudaStreamCreateWithFlags(&h->st_dn, cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreate(&h->t_start) == cudaSuccess && cudaEventCreate(&h->t_stop) == cudaSuccess;
    for (int k = 0; k < HBD_SLOTS && ok; k++) {
        for (int i = 0; i < 6 && ok; i++) ok = cudaEventCreate(&h->slot[k].ev[i]) == cudaSuccess;
        ok = ok && cudaEventCreateWithFlags(&h->slot[k].ev_up, cudaEventDisableTiming) == cudaSuccess;
    }
    if (!ok) {
        cvp9_hbd_destroy(h);
        return CVP9_ERR_GPU;
    }
    *out = h;
    return CVP9_OK;
}

static void stream_free(hbd_stream_t *s)
{
    for (int i = 0; i < HBD_NBUF; i++) if (s->buf[i]) cudaFree(s->buf[i]);
    if (s->d_sb_range) cudaFree(s->d_sb_range);
    if (s->d_sb_done) cudaFree(s->d_sb_done);
    if (s->d_mi_map) cudaFree(s->d_mi_map);
    for (int k = 0; k < HBD_SLOTS; k++) if (s->h_out[k]) cudaFreeHost(s->h_out[k]);
    memset(s, 0, sizeof(*s));
}

void cvp9_hbd_destroy(cvp9_hbd_t *h)
{
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->st_up) cudaStreamSynchronize(h->st_up);
    if (h->st_k) cudaStreamSynchronize(h->st_k);
    if (h->st_dn) cudaStreamSynchronize(h->st_dn);
    for (int i = 0; i < h->ns; i++) stream_free(&h->s[i]);
    free(h->s);
    for (int k = 0; k < HBD_SLOTS; k++) {
        hbd_slot_t *sl = &h->slot[k];
        if (sl->d_jobs) cudaFree(sl->d_jobs);
        if (sl->h_jobs) cudaFreeHost(sl->h_jobs);
        if (sl->d_tickets) cudaFree(sl->d_tickets);
        if (sl->h_tickets) cudaFreeHost(sl->h_tickets);
        if (sl->d_words) cudaFree(sl->d_words);
        if (sl->h_status) cudaFreeHost(sl->h_status);
        if (sl->d_in) cudaFree(sl->d_in);
        for (int i = 0; i < 6; i++) if (sl->ev[i]) cudaEventDestroy(sl->ev[i]);
        if (sl->ev_up) cudaEventDestroy(sl->ev_up);
    }
    if (h->t_start) cudaEventDestroy(h->t_start);
    if (h->t_stop) cudaEventDestroy(h->t_stop);
    if (h->st_up) cudaStreamDestroy(h->st_up);
    if (h->st_k) cudaStreamDestroy(h->st_k);
    if (h->st_dn) cudaStreamDestroy(h->st_dn);
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
    for (int k = 0; k < HBD_SLOTS && ok; k++)
        ok = cudaHostAlloc((void **)&s->h_out[k], s->frame_bytes, cudaHostAllocDefault) == cudaSuccess;
    /* done flags and mode-info tags compare against the stream's epoch */
    ok = ok && cudaMemset(s->d_sb_done, 0, (size_t)s->n_sb * 4) == cudaSuccess;
    ok = ok && cudaMemset(s->d_mi_map, 0, (size_t)s->n_mi * 4) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        stream_free(s);
        return CVP9_ERR_NOMEM;
    }
    for (int i = 0; i < 8; i++) s->slot[i] = -1;
    for (int k = 0; k < HBD_SLOTS; k++) s->dl_buf[k] = -1;
    s->out_slot = -1;
    s->open = 1;
    return sid;
}

static int frame_check(const hbd_stream_t *s, const vp9_parsed_frame_t *pf)
{
    const vp9_frame_header_t *hd = &pf->hdr;
    if (hd->bit_depth != 10 || hd->width != s->W || hd->height != s->H) return CVP9_ERR_UNSUPPORTED;
    const int inter = hd->frame_type != VP9_FRAME_KEY && !hd->intra_only;
    if (inter && (int)hd->interp_filter > VP9_FILTER_BILINEAR) return CVP9_ERR_UNSUPPORTED;
    return CVP9_OK;
}

/* Complete the step a slot holds: its status, deliveries, times. */
static int finish_slot(cvp9_hbd_t *h, int k)
{
    hbd_slot_t *sl = &h->slot[k];
    if (!sl->pending) return CVP9_OK;
    sl->pending = 0;
    if (cudaEventSynchronize(sl->ev[5]) != cudaSuccess) return CVP9_ERR_GPU;
    int rc = CVP9_OK;
    for (int i = 0; i < sl->n; i++) {
        hbd_stream_t *s = &h->s[sl->sid[i]];
        if (!s->open) continue;
        s->dl_buf[k] = -1;
        const uint32_t st = sl->h_status[i];
        if (st & CVP9_JOB_TIMEOUT) rc = CVP9_ERR_GPU;
        else if (st && rc == CVP9_OK) rc = CVP9_ERR_INVALID_DATA;
        s->out_slot = (!st && !(sl->flags & CVP9_HBD_NO_OUTPUT)) ? k : -1;
        s->pts = sl->pts[i];
    }
    float t[5] = {0};
    for (int i = 0; i < 5; i++) cudaEventElapsedTime(&t[i], sl->ev[i], sl->ev[i + 1]);
    memcpy(h->ms, t, sizeof(t));
    return rc;
}

/* Complete every step in flight, oldest first. */
static int finish_all(cvp9_hbd_t *h)
{
    int rc = CVP9_OK;
    for (uint64_t d = HBD_SLOTS; d >= 1; d--) {
        if (h->next_seq < d) continue;
        const int r = finish_slot(h, (int)((h->next_seq - d) % HBD_SLOTS));
        if (r != CVP9_OK && rc == CVP9_OK) rc = r;
    }
    return rc;
}

int cvp9_hbd_wait(cvp9_hbd_t *h)
{
    if (!h) return CVP9_ERR_INVALID_DATA;
    cudaSetDevice(h->device);
    int rc = finish_all(h);
    if (rc == CVP9_OK) rc = h->err;
    h->err = CVP9_OK;
    return rc;
}

int cvp9_hbd_close_stream(cvp9_hbd_t *h, int sid)
{
    if (!h || sid < 0 || sid >= h->ns || !h->s[sid].open) return CVP9_ERR_INVALID_DATA;
    cudaSetDevice(h->device);
    const int rc = finish_all(h);
    if (rc != CVP9_OK && h->err == CVP9_OK) h->err = rc;
    stream_free(&h->s[sid]);
    return CVP9_OK;
}

static int submit_step(cvp9_hbd_t *h, int n, const int *sids, const cvp9_hbd_frame_t *frames,
                       const cvp9_hbd_coeff_list_t *lists, const int64_t *pts, unsigned flags)
{
    if (!h || n <= 0 || n > HBD_MAX_STEP || !sids || !frames) return CVP9_ERR_INVALID_DATA;
    cudaSetDevice(h->device);
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
    /* the slot this step takes: its previous step completes first */
    const int k = (int)(h->next_seq % HBD_SLOTS);
    hbd_slot_t *sl = &h->slot[k];
    const int prev = finish_slot(h, k);
    if (prev != CVP9_OK && h->err == CVP9_OK) h->err = prev;

    size_t in_bytes = 0, ntk = 0;
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
    if (grow_pair((void **)&sl->d_jobs, (void **)&sl->h_jobs, &sl->jobs_cap, (size_t)n * sizeof(cvp9_job_t)) != 0 ||
        grow_pair((void **)&sl->d_tickets, (void **)&sl->h_tickets, &sl->tickets_cap, ntk * 4) != 0 ||
        grow_pair((void **)&sl->d_words, (void **)&sl->h_status, &sl->words_cap, (size_t)(n + 2) * 4) != 0 ||
        (in_bytes && grow_dev((void **)&sl->d_in, &sl->in_cap, in_bytes) != 0))
        return CVP9_ERR_NOMEM;

    /* uploads (upload stream); the per-stream scratch is cleared on the
     * kernel stream, behind the previous step's kernels that use it */
    cudaEventRecord(sl->ev[0], h->st_up);
    size_t at = 0;
    for (int i = 0; i < n; i++) {
        hbd_stream_t *s = &h->s[sids[i]];
        const vp9_parsed_frame_t *pf = frames[i].pf;
        cvp9_job_t *job = &sl->h_jobs[i];
        memset(job, 0, sizeof(*job));
        cvp9_job_geometry(job, pf);
        cvp9_job_full(job, pf);
        const vp9_macroblock_info_t *blocks = pf->blocks;
        const int32_t *coeffs = frames[i].coeffs;
        if (!(flags & CVP9_HBD_DEVICE_INPUTS)) {
            const size_t bb = (size_t)pf->num_blocks * sizeof(vp9_macroblock_info_t);
            const size_t cb = (size_t)pf->num_coeffs * 4;
            uint8_t *db = sl->d_in + at;
            at += (bb + 255) & ~(size_t)255;
            uint8_t *dc = sl->d_in + at;
            at += (cb + 255) & ~(size_t)255;
            if (bb && cudaMemcpyAsync(db, pf->blocks, bb, cudaMemcpyHostToDevice, h->st_up) != cudaSuccess)
                return CVP9_ERR_GPU;
            if (!lists && cb &&
                cudaMemcpyAsync(dc, frames[i].coeffs, cb, cudaMemcpyHostToDevice, h->st_up) != cudaSuccess)
                return CVP9_ERR_GPU;
            blocks = (const vp9_macroblock_info_t *)db;
            coeffs = (const int32_t *)dc;
        }
        if (lists) {
            const size_t cb = (size_t)pf->num_coeffs * 4, lb = (size_t)lists[i].n * 4;
            uint8_t *dc = (uint8_t *)coeffs;
            if (flags & CVP9_HBD_DEVICE_INPUTS) {
                dc = sl->d_in + at;
                at += (cb + 255) & ~(size_t)255;
                coeffs = (const int32_t *)dc;
            }
            uint8_t *dp = sl->d_in + at;
            at += (lb + 255) & ~(size_t)255;
            uint8_t *dv = sl->d_in + at;
            at += (lb + 255) & ~(size_t)255;
            const enum cudaMemcpyKind kind =
                (flags & CVP9_HBD_DEVICE_INPUTS) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
            if ((cb && cudaMemsetAsync(dc, 0, cb, h->st_up) != cudaSuccess) ||
                (lb && cudaMemcpyAsync(dp, lists[i].pos, lb, kind, h->st_up) != cudaSuccess) ||
                (lb && cudaMemcpyAsync(dv, lists[i].val, lb, kind, h->st_up) != cudaSuccess))
                return CVP9_ERR_GPU;
            job->sp_pos = (const uint32_t *)dp;
            job->sp_val32 = (const int32_t *)dv;
            job->sp_n = lists[i].n;
        }
        job->blocks = blocks;
        job->coeffs = NULL;
        job->coeffs32 = coeffs;
        /* the output goes to a buffer no slot holds and no download reads */
        int ob = -1;
        for (int b = 0; b < HBD_NBUF && ob < 0; b++) {
            int held = 0;
            for (int r = 0; r < 8; r++) held |= s->slot[r] == b;
            for (int q = 0; q < HBD_SLOTS; q++) held |= s->dl_buf[q] == b;
            if (!held) ob = b;
        }
        job->out = s->buf[ob];
        for (int r = 0; r < 8; r++)
            if (s->slot[r] >= 0) {
                job->ref[r].plane = s->buf[s->slot[r]];
                job->ref[r].w = (int32_t)s->W;
                job->ref[r].h = (int32_t)s->H;
            }
        job->epoch = ++s->epoch;
        job->sb_range = s->d_sb_range;
        job->sb_done = s->d_sb_done;
        job->mi_map = s->d_mi_map;
        job->status = sl->d_words + 2 + i;
        /* pool: the slots refresh_frame_flags names take the new frame */
        const unsigned refresh = pf->hdr.refresh_frame_flags ? pf->hdr.refresh_frame_flags : 0x01u;
        for (int r = 0; r < 8; r++) if (refresh & (1u << r)) s->slot[r] = ob;
        s->dl_buf[k] = ob;
        sl->sid[i] = sids[i];
        sl->pts[i] = pts ? pts[i] : 0;
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
                                                     sl->h_tickets + nt);
        }
    if (cudaMemcpyAsync(sl->d_jobs, sl->h_jobs, (size_t)n * sizeof(cvp9_job_t), cudaMemcpyHostToDevice, h->st_up) !=
            cudaSuccess ||
        cudaMemcpyAsync(sl->d_tickets, sl->h_tickets, (size_t)nt * 4, cudaMemcpyHostToDevice, h->st_up) !=
            cudaSuccess ||
        cudaEventRecord(sl->ev_up, h->st_up) != cudaSuccess)
        return CVP9_ERR_GPU;

    /* kernels (kernel stream, in submission order) */
    if (cudaStreamWaitEvent(h->st_k, sl->ev_up, 0) != cudaSuccess ||
        cudaMemsetAsync(sl->d_words, 0, (size_t)(n + 2) * 4, h->st_k) != cudaSuccess)
        return CVP9_ERR_GPU;
    for (int i = 0; i < n; i++) {
        const hbd_stream_t *s = &h->s[sids[i]];
        if (cudaMemsetAsync(s->d_sb_range, 0, (size_t)s->n_sb * 16, h->st_k) != cudaSuccess) return CVP9_ERR_GPU;
    }
    if (lists && cvp9k_launch_scatter(sl->d_jobs, n, max_n, h->st_k) != 0) return CVP9_ERR_GPU;
    cvp9k_launch_t L;
    memset(&L, 0, sizeof(L));
    L.jobs = sl->d_jobs;
    L.njobs = n;
    L.arith = CVP9_ARITH_FULL;
    L.full = 1;
    L.hbd = 1;
    L.max_blocks = max_blocks;
    L.tickets = sl->d_tickets;
    L.n_tickets = nt;
    L.ticket_counter = sl->d_words;
    L.recon_ctas = h->recon_ctas;
    L.lf_counter = sl->d_words + 1;
    L.lf_tickets = (uint32_t)(n * max_sb_rows);
    L.lf_ctas = h->lf_ctas;
    L.ev[0] = sl->ev[1];
    L.ev[1] = sl->ev[2];
    L.ev[2] = sl->ev[3];
    L.ev[3] = sl->ev[4];
    if (cvp9k_launch_frame(&L, h->st_k) != 0) return CVP9_ERR_GPU;

    /* downloads (download stream), behind the kernels */
    if (cudaStreamWaitEvent(h->st_dn, sl->ev[4], 0) != cudaSuccess ||
        cudaMemcpyAsync(sl->h_status, sl->d_words + 2, (size_t)n * 4, cudaMemcpyDeviceToHost, h->st_dn) !=
            cudaSuccess)
        return CVP9_ERR_GPU;
    if (!(flags & CVP9_HBD_NO_OUTPUT))
        for (int i = 0; i < n; i++) {
            hbd_stream_t *s = &h->s[sids[i]];
            if (cudaMemcpyAsync(s->h_out[k], s->buf[s->dl_buf[k]], s->frame_bytes, cudaMemcpyDeviceToHost,
                                h->st_dn) != cudaSuccess)
                return CVP9_ERR_GPU;
        }
    cudaEventRecord(sl->ev[5], h->st_dn);
    sl->pending = 1;
    sl->n = n;
    sl->flags = (int)flags;
    h->next_seq++;
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
    const int rc = finish_all(h);
    if (rc != CVP9_OK && h->err == CVP9_OK) h->err = rc;
    hbd_stream_t *s = &h->s[sid];
    if (s->out_slot < 0) return CVP9_ERR_UNSUPPORTED;
    const uint32_t cw = (s->W + 1) / 2, ch = (s->H + 1) / 2;
    info->width = s->W;
    info->height = s->H;
    info->stride_y = s->W;
    info->stride_uv = cw;
    info->plane_y = s->h_out[s->out_slot];
    info->plane_u = info->plane_y + (size_t)s->W * s->H;
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

int cvp9_hbd_timer_start(cvp9_hbd_t *h)
{
    if (!h) return CVP9_ERR_INVALID_DATA;
    cudaSetDevice(h->device);
    /* behind everything queued so far: the next step's uploads follow it */
    if (cudaStreamSynchronize(h->st_up) != cudaSuccess || cudaStreamSynchronize(h->st_k) != cudaSuccess ||
        cudaStreamSynchronize(h->st_dn) != cudaSuccess || cudaEventRecord(h->t_start, h->st_up) != cudaSuccess)
        return CVP9_ERR_GPU;
    return CVP9_OK;
}

int cvp9_hbd_timer_stop(cvp9_hbd_t *h, float *ms)
{
    if (!h || !ms) return CVP9_ERR_INVALID_DATA;
    cudaSetDevice(h->device);
    /* the last step's download follows its kernels, which follow its uploads */
    if (cudaEventRecord(h->t_stop, h->st_dn) != cudaSuccess || cudaEventSynchronize(h->t_stop) != cudaSuccess ||
        cudaEventElapsedTime(ms, h->t_start, h->t_stop) != cudaSuccess)
        return CVP9_ERR_GPU;
    return CVP9_OK;
}
