/*
 * recon_job.h — one frame of one stream as the reconstruction kernels see
 * it. Shared by the C host (cuda_backend.c, batch.c) and the CUDA kernels
 * (recon.cu); plain C, no CUDA types.
 *
 * Device memory layout of a frame: one I420 buffer, luma W x H at stride W,
 * then U and V at ceil(W/2) x ceil(H/2), stride ceil(W/2) — the same layout
 * the reference hands out (src/decoder/vp9_frame.c:8-34), so a frame leaves
 * the device in one copy and reference frames need no repacking.
 */
#ifndef CVP9_RECON_JOB_H
#define CVP9_RECON_JOB_H

#include <stdint.h>
#include "cvp9_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Arithmetic profiles. FULL runs the SPEC kernels with job.full set: the
 * shader arithmetic completed to the VP9 specification where the reference
 * is a skeleton (compound prediction, every frame-level filter, per-TX
 * directional intra with ADST, the VP9 loop filter). */
enum { CVP9_ARITH_REFCPU = 0, CVP9_ARITH_SPEC = 1, CVP9_ARITH_FULL = 2 };

/* Job status bits, written by the kernels, read back with the frame. */
enum {
    CVP9_JOB_BAD_BLOCK   = 1u << 0,  /* block outside the supported domain    */
    CVP9_JOB_BAD_ORDER   = 1u << 1,  /* SB's blocks not contiguous in the list */
    CVP9_JOB_TIMEOUT     = 1u << 2,  /* a bounded wait on a neighbour expired  */
    CVP9_JOB_TOO_MANY    = 1u << 3,  /* more than 256 blocks in one SB         */
};

typedef struct {
    const uint8_t *plane;   /* I420 base of the reference, NULL when empty */
    int32_t        w, h;    /* its luma size                               */
} cvp9_ref_t;

typedef struct {
    int32_t  W, H, CW, CH;          /* luma and chroma sizes                     */
    int32_t  sb_cols, sb_rows;      /* 64x64 superblock grid                     */
    int32_t  mi_cols, mi_rows;      /* 8x8 mode-info grid                        */
    const vp9_macroblock_info_t *blocks;
    const int16_t *coeffs;
    uint32_t num_blocks, num_coeffs;
    uint8_t *out;                   /* I420 frame being reconstructed            */
    uint8_t *nv12;                  /* optional NV12 target (W*H + 2*CW*CH)      */
    cvp9_ref_t ref[8];              /* reference pool slots                      */
    int32_t  q_dc, q_ac;            /* frame quantiser steps (SPEC residual)      */
    int32_t  lf_level, lf_sharpness;
    uint8_t  ref_slot_of[3];        /* SPEC: LAST/GOLDEN/ALTREF -> pool slot      */
    uint8_t  lf_tiled;              /* 0: frame-wide filter (W or H = 8k+1);
                                     * 1: shared-memory tiles; 2: register strips */
    uint32_t epoch;                 /* frame sequence number for sb_done flags    */
    uint32_t *sb_range;             /* per SB {start, end, groups, spare}         */
    uint32_t *sb_done;              /* per SB: epoch of the last finished frame   */
    uint32_t *status;               /* CVP9_JOB_* bits                            */
    const int16_t *coeffs_src;      /* REFCPU upload: the parser's coefficient array
                                     * in page-locked host memory, read by
                                     * k_gather_luma (NULL: coeffs already on device) */
    const uint32_t *sp_pos;         /* sparse upload: indices into coeffs (device)  */
    const int16_t  *sp_val;         /* and their values; coeffs zeroed beforehand   */
    uint32_t        sp_n;           /* k_scatter_coeffs writes them; 0: none        */
    uint32_t        packed_words;   /* packed upload (cvp9_pack_coeffs): its words  */
    const uint32_t *packed;         /* (device), expanded into coeffs by
                                     * k_unpack_coeffs; NULL: none                  */
    /* FULL profile (full != 0) */
    uint32_t *mi_map;               /* per 8x8 MI: loop-filter mode info, tagged
                                     * with the frame's epoch (k_lf_mimap)          */
    int32_t  q_dc_uv, q_ac_uv;      /* chroma quantiser steps (q_dc, q_ac: luma)     */
    uint8_t  full;
    uint8_t  interp_filter;         /* 0 regular, 1 smooth, 2 sharp, 3 bilinear      */
    uint8_t  lossless;              /* 4x4 Walsh-Hadamard residual                  */
    uint8_t  log2_tile_cols;        /* intra left edges end at tile columns         */
    /* batch engine download */
    uint8_t *dl;                    /* the step's contiguous output staging
                                     * (device): k_collect copies `out` here;
                                     * NULL: no download                           */
    /* profile 2 (10-bit, k_hbd_recon): out and the reference planes hold
     * uint16 samples in the same I420 layout; coeffs32 the dequantised
     * coefficients (num_coeffs of them, the dense layout of coeffs) */
    const int32_t *coeffs32;
    const int32_t *sp_val32;        /* sparse upload of coeffs32 (with sp_pos, sp_n) */
} cvp9_job_t;

#ifdef __cplusplus
}
#endif

#endif /* CVP9_RECON_JOB_H */
