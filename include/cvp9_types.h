/*
 * cvp9_types.h — the data model at the reconstruction boundary.
 *
 * These declarations are layout-identical to the compute-vp9 library's own
 * public and internal headers, because the CUDA backend receives the very
 * objects the CPU tile parser fills in:
 *   - cvp9_err_t, cvp9_frame_info_t, cvp9_dmabuf_frame_t,
 *     cvp9_export_buffer_t      ↔ include/compute_vp9/decoder.h:27-36, 47-56,
 *                                  124-132, 151-157
 *   - vp9_frame_header_t        ↔ src/decoder/vp9_bitstream.h:40-92
 *   - cvp9_mv_t                 ↔ src/decoder/vp9_parsed_frame.h:11-16
 *   - vp9_macroblock_info_t     ↔ src/decoder/vp9_parsed_frame.h:19-33
 *   - vp9_parsed_frame_t        ↔ src/decoder/vp9_parsed_frame.h:36-63
 * Field order, widths and names follow those headers exactly so a pointer
 * from the reference decoder can be handed to this library unchanged; the
 * byte offsets are pinned by tests/golden/layout.json.
 *
 * When this header is compiled inside the reference tree (which already
 * declares all of these types), define CVP9_HAVE_REFERENCE_TYPES before
 * including it and only the backend prototypes are used.
 */
#ifndef CVP9_TYPES_H
#define CVP9_TYPES_H

#include <stdint.h>
#include <stddef.h>
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef CVP9_HAVE_REFERENCE_TYPES

/* ── Public API types ───────────────────────────────────────────────────── */

typedef enum {
    CVP9_BACKEND_AUTO   = 0,
    CVP9_BACKEND_VULKAN = 1,
    CVP9_BACKEND_OPENCL = 2,
    CVP9_BACKEND_CPU    = 3,
    CVP9_BACKEND_CUDA   = 4,   /* appended: keeps every existing value */
} cvp9_backend_t;

typedef enum {
    CVP9_OK               =  0,
    CVP9_ERR_NOMEM        = -1,
    CVP9_ERR_NO_BACKEND   = -2,
    CVP9_ERR_INVALID_DATA = -3,
    CVP9_ERR_UNSUPPORTED  = -4,
    CVP9_ERR_GPU          = -5,
    CVP9_ERR_AGAIN        = -6,
} cvp9_err_t;

/* One decoded I420 frame. Strides are in bytes; chroma is ceil(w/2) x ceil(h/2). */
typedef struct {
    uint32_t  width;
    uint32_t  height;
    uint32_t  stride_y;
    uint32_t  stride_uv;
    uint8_t  *plane_y;
    uint8_t  *plane_u;
    uint8_t  *plane_v;
    int64_t   pts;
} cvp9_frame_info_t;

typedef struct {
    int       fd;
    uint64_t  size;
    uint32_t  width;
    uint32_t  height;
    uint32_t  offsets[3];
    uint32_t  pitches[3];
    int64_t   pts;
} cvp9_dmabuf_frame_t;

typedef struct {
    int       fd;
    void     *mapped;
    uint64_t  size;
    void     *priv_buf;
    void     *priv_mem;
} cvp9_export_buffer_t;

/* ── Uncompressed frame header (fields the reconstruction reads) ────────── */

typedef enum {
    VP9_FRAME_KEY        = 0,
    VP9_FRAME_NON_KEY    = 1,
    VP9_FRAME_INTRA_ONLY = 2,
    VP9_FRAME_S          = 3,
} vp9_frame_type_t;

typedef enum {
    VP9_CS_UNKNOWN  = 0,
    VP9_CS_BT601    = 1,
    VP9_CS_BT709    = 2,
    VP9_CS_SMPTE170 = 3,
    VP9_CS_SMPTE240 = 4,
    VP9_CS_BT2020   = 5,
    VP9_CS_SRGB     = 7,
} vp9_color_space_t;

typedef enum {
    VP9_FILTER_EIGHTTAP        = 0,
    VP9_FILTER_EIGHTTAP_SMOOTH = 1,
    VP9_FILTER_EIGHTTAP_SHARP  = 2,
    VP9_FILTER_BILINEAR        = 3,
    VP9_FILTER_SWITCHABLE      = 4,
} vp9_interp_filter_t;

typedef struct {
    vp9_frame_type_t    frame_type;
    uint32_t            width;
    uint32_t            height;
    uint32_t            render_width;
    uint32_t            render_height;
    uint8_t             profile;
    uint8_t             bit_depth;
    vp9_color_space_t   color_space;
    bool                color_range;
    uint8_t             subsampling_x;
    uint8_t             subsampling_y;
    bool                show_frame;
    bool                show_existing_frame;
    uint8_t             frame_to_show_map_idx;
    bool                intra_only;
    uint8_t             reset_frame_context;
    bool                error_resilient;
    bool                allow_high_precision_mv;
    vp9_interp_filter_t interp_filter;
    bool                refresh_frame_context;
    bool                frame_parallel;
    uint8_t             frame_context_idx;
    uint8_t             log2_tile_cols;
    uint8_t             log2_tile_rows;
    uint32_t            uncompressed_header_bytes;
    uint16_t            first_partition_size;
    int16_t             base_qindex;
    int8_t              y_dc_delta_q;
    int8_t              uv_dc_delta_q;
    int8_t              uv_ac_delta_q;
    uint8_t             filter_level;
    uint8_t             sharpness_level;
    uint8_t             refresh_frame_flags;
    uint8_t             ref_frame_idx[3];
    uint8_t             ref_frame_sign_bias[4];
    bool                segmentation_enabled;
} vp9_frame_header_t;

/* ── Parsed-frame model: what the CPU parse hands to reconstruction ─────── */

/* Per-4x4 motion vector cell (1/8 pel) and reference selector 0..2. */
typedef struct {
    int32_t x;
    int32_t y;
    int32_t ref;
    int32_t pad;
} cvp9_mv_t;

/* Per-block descriptor, 32 bytes. tx_size is the VP9 index 0..3
 * (4, 8, 16, 32 px); mv[i] = {col, row} in 1/8 pel; coeff_offset points at
 * the block's first int16 coefficient (luma TXs, then U, then V). */
typedef struct {
    uint16_t x;
    uint16_t y;
    uint8_t  width;
    uint8_t  height;
    uint8_t  tx_size;
    uint8_t  is_intra;
    uint8_t  y_mode;
    uint8_t  uv_mode;
    uint8_t  ref_frame[2];
    int16_t  mv[2][2];
    uint8_t  skip;
    uint32_t coeff_offset;
    uint16_t eob;
} vp9_macroblock_info_t;

typedef struct {
    vp9_frame_header_t      hdr;
    vp9_macroblock_info_t  *blocks;
    uint32_t                num_blocks;
    uint32_t                blocks_capacity;
    int16_t                *coeffs;
    uint32_t                num_coeffs;
    uint32_t                coeffs_capacity;
    cvp9_mv_t              *mv_grid;
    uint32_t                mv_grid_width;
    uint32_t                mv_grid_height;
    uint8_t                *mi_width_grid;
    uint8_t                *mi_height_grid;
    uint32_t                mi_grid_width;
    uint32_t                mi_grid_height;
    uint32_t               *mi_block_grid;
} vp9_parsed_frame_t;

#endif /* CVP9_HAVE_REFERENCE_TYPES */

#ifdef __cplusplus
}
#endif

#endif /* CVP9_TYPES_H */
