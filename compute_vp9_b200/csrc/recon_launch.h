/*
 * recon_launch.h — C-ABI launch shims exported by recon.cu (internal: the
 * public entry points are in include/cuda_backend.h and include/cvp9_batch.h).
 */
#ifndef CVP9_RECON_LAUNCH_H
#define CVP9_RECON_LAUNCH_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>
#include "recon_job.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One batch step: J jobs (one frame each) through scan -> recon -> filter. */
typedef struct {
    const cvp9_job_t *jobs;        /* device array of njobs descriptors          */
    int              njobs;
    int              arith;        /* CVP9_ARITH_*                               */
    int              max_blocks;   /* largest num_blocks over the jobs           */
    int              scan_ctas;    /* >0: fixed scan grid (grid-stride), else from max_blocks */
    const uint32_t  *tickets;      /* device: (job << 20 | sb) in SB-diagonal order */
    uint32_t         n_tickets;
    uint32_t        *ticket_counter;  /* device, zeroed before the launch        */
    int              recon_ctas;   /* grid of the persistent recon kernel        */
    int              lf_tiles_x, lf_tiles_y;   /* tiled filter grid in 64x64 tiles (max over jobs) */
    int              lf_tile_h;    /* 64 (default) or 32: filter tile height */
    int              lf_strips_x, lf_strips_y;  /* register-strip filter grid (jobs with lf_tiled == 2) */
    int              flat_lf_max_w, flat_lf_max_h; /* >0: run the frame-wide filter */
    int              flat_nv12;
    /* Inter fast path: when `general` is set, k_inter takes the
     * superblocks that hold inter blocks only, one warp each, and k_recon
     * runs on the rest. One device buffer of 2 n_tickets + 2 words:
     * general = its start (flags), general_tickets = + n_tickets,
     * n_general = + 2 n_tickets (count, then a scratch counter). */
    uint32_t        *general;
    uint32_t        *general_tickets;
    uint32_t        *n_general;
    int              inter_variant;  /* 0: default, 1: 96-register k_inter, 2: 80-register */
    int              warp_levels;    /* k_recon: levels of small intra blocks a warp per block */
    /* FULL profile (jobs with full set; arith SPEC): k_lf_mimap after the
     * scan, the VP9 loop filter k_lf_full after the reconstruction instead
     * of the other filters, then the NV12 pack of armed targets. */
    int              full;
    uint32_t        *lf_counter;   /* device word, zeroed before the launch      */
    uint32_t         lf_tickets;   /* njobs * (most superblock rows of a job)    */
    int              lf_ctas;      /* grid of k_lf_full                          */
    int              full_nv12_max_px;  /* > 0: largest W*H of a job with a target */
    /* Profile 2 (10-bit): jobs with coeffs32 and 16-bit planes through
     * k_scan_blocks, k_lf_mimap, k_hbd_recon (tickets, recon_ctas) and
     * k_lf_full<uint16_t> (lf_* as for FULL); nothing else runs. */
    int              hbd;
    cudaEvent_t      ev[4];        /* optional: before scan, recon, filter; after */
} cvp9k_launch_t;

size_t cvp9k_recon_smem_bytes(void);
int    cvp9k_upload_dct_basis(const double *basis, int count);
int    cvp9k_configure(void);
int    cvp9k_recon_ctas_per_sm(int arith);
/* CTAs of k_lf_full (128 threads, static shared memory) resident per SM. */
int    cvp9k_lf_full_ctas_per_sm(void);
/* CTAs of k_hbd_recon resident per SM. */
int    cvp9k_hbd_ctas_per_sm(void);
/* REFCPU upload of the coefficients the reconstruction reads — each block's
 * luma TXs — straight from page-locked host memory into jobs[j].coeffs, for
 * every job with coeffs_src set; adds the bytes moved to *bytes (device).
 * Blocks must already be on the device. */
int    cvp9k_launch_gather(const cvp9_job_t *jobs, int njobs, int max_blocks, uint32_t *bytes,
                           cudaStream_t stream);

/* Sparse coefficient upload: jobs[j].coeffs[sp_pos[k]] = sp_val[k] for
 * every job with sp_n > 0 (indices past num_coeffs are ignored); jobs with
 * sp_val32 set write coeffs32[sp_pos[k]] = sp_val32[k] instead. */
int    cvp9k_launch_scatter(const cvp9_job_t *jobs, int njobs, uint32_t max_n, cudaStream_t stream);

/* Packed coefficient upload: every job with `packed` set gets its dense
 * coeffs array rebuilt from the pages (entry pages zero-filled, then
 * scattered; dense pages copied). max_pages: most pages of any job; a
 * malformed page of job j sets err[j] to 1 (device, one word per job). */
int    cvp9k_launch_unpack(const cvp9_job_t *jobs, int njobs, uint32_t max_pages, uint32_t *err,
                           cudaStream_t stream);

/* Output collection of a batch step: every job with `dl` set gets its
 * I420 frame (`out`, W*H + 2*CW*CH bytes) copied to `dl`, so that the step's
 * frames leave the device in one copy. max_bytes: the largest frame. */
int    cvp9k_launch_collect(const cvp9_job_t *jobs, int njobs, size_t max_bytes, cudaStream_t stream);

/* Enqueue the chain on `stream`; returns the cudaError_t of the first
 * failing call (0 on success). */
int    cvp9k_launch_frame(const cvp9k_launch_t *launch, cudaStream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* CVP9_RECON_LAUNCH_H */
