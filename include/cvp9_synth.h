/*
 * cvp9_synth.h — seeded synthetic parsed-frame streams.
 *
 * Produces vp9_parsed_frame_t contents the way the CPU tile parser lays them
 * out (src/decoder/vp9_kf_tile.c:320-396 coefficient order, :1153-1182 block
 * and MV-grid fields), so the reconstruction path can be driven with
 * content-bearing frames without a real bitstream. Frames are a pure function
 * of (config, frame index): any frame can be regenerated independently.
 */
#ifndef CVP9_SYNTH_H
#define CVP9_SYNTH_H

#include "cvp9_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    uint32_t width, height;
    uint64_t seed;
    int      gop;              /* key frame every gop frames; <=0: frame 0 only  */
    int      fixed_bsize;      /* >0: every block this square size (4..64)       */
    int      min_bsize;        /* smallest partition leaf (4 or 8)               */
    int      max_bsize;        /* largest leaf (8..64)                           */
    int      rect_partitions;  /* allow HORZ / VERT partitions                  */
    int      fixed_tx;         /* >=0: this tx_size everywhere (capped by block) */
    int      tx_weights[4];    /* weights of TX 4/8/16/32 when fixed_tx < 0      */
    double   density_min;      /* per-block nonzero-coefficient fraction range   */
    double   density_max;
    int      coeff_max;        /* |coeff| clip                                   */
    double   coeff_scale;      /* Laplacian scale of |coeff|                     */
    int      mv_range_px;      /* MVs uniform in +-range px (1/8-pel units)      */
    int      nrefs;            /* 1: LAST only, 3: LAST/GOLDEN/ALTREF            */
    int      golden_every;     /* refresh_frame_flags bit 1 period               */
    int      altref_every;     /* refresh_frame_flags bit 2 period               */
    int      qindex;
    int      lf_level;         /* <0: uniform 0..63 per frame                    */
    int      sharpness;
    int      interp_filter;    /* <0: uniform over regular/smooth/sharp          */
    int      all_intra_modes;  /* modes 0..9 instead of {DC,V,H,TM}              */
    double   intra_in_inter;   /* share of intra blocks inside inter frames      */
    double   skip_prob;        /* share of skip blocks                           */
    int      log2_tile_cols;   /* >0: blocks emitted tile-column major           */
    double   compound_prob;    /* share of inter blocks with a second reference  */
} cvp9_synth_config_t;

/* Workload presets: 1 = plain 720p stream (every SB split to 8x8, TX 8x8,
 * q60, 5% density, +-64 px MVs, LAST only, LF 32), 2 = 1080p GOP-60 stream
 * (partition depth uniform 8..64, TX 4/8/16/32 at 30/30/25/15, 2-20%
 * density, +-128 px, three references, LF level per frame). width/height
 * override the preset's size when non-zero. */
void cvp9_synth_preset(cvp9_synth_config_t *cfg, int preset,
                       uint32_t width, uint32_t height, uint64_t seed);

typedef struct cvp9_synth cvp9_synth_t;

cvp9_synth_t *cvp9_synth_create(const cvp9_synth_config_t *cfg);
void          cvp9_synth_destroy(cvp9_synth_t *s);

/* Fill frame `index` of the stream. The returned parsed frame and all its
 * arrays are owned by the generator and stay valid until the next call. */
const vp9_parsed_frame_t *cvp9_synth_frame(cvp9_synth_t *s, int index);

/* FNV-1a 64-bit over a byte range (used for golden frame hashes). */
uint64_t cvp9_fnv1a64(const void *data, size_t n, uint64_t h);

#ifdef __cplusplus
}
#endif

#endif /* CVP9_SYNTH_H */
