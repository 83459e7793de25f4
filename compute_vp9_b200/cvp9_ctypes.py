"""ctypes mirrors of the boundary types in include/cvp9_types.h.

Field order and widths follow the reference decoder's structs
(src/decoder/vp9_parsed_frame.h:11-63, src/decoder/vp9_bitstream.h:40-92,
include/compute_vp9/decoder.h:27-157) so Python tests can build and read the
exact objects the C ABI exchanges.
"""
import ctypes as C

# cvp9_err_t (include/compute_vp9/decoder.h:27-36)
CVP9_OK = 0
CVP9_ERR_NOMEM = -1
CVP9_ERR_NO_BACKEND = -2
CVP9_ERR_INVALID_DATA = -3
CVP9_ERR_UNSUPPORTED = -4
CVP9_ERR_GPU = -5
CVP9_ERR_AGAIN = -6

ERR_NAMES = {
    CVP9_OK: "OK",
    CVP9_ERR_NOMEM: "Out of memory",
    CVP9_ERR_NO_BACKEND: "No compute backend available",
    CVP9_ERR_INVALID_DATA: "Invalid bitstream data",
    CVP9_ERR_UNSUPPORTED: "Unsupported operation",
    CVP9_ERR_GPU: "GPU error",
    CVP9_ERR_AGAIN: "Frame not ready yet (try again)",
}

VP9_FRAME_KEY = 0
VP9_FRAME_NON_KEY = 1

ARITH_REFCPU = 0
ARITH_SPEC = 1
ARITH_FULL = 2


class FrameHeader(C.Structure):
    _fields_ = [
        ("frame_type", C.c_int),
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("render_width", C.c_uint32),
        ("render_height", C.c_uint32),
        ("profile", C.c_uint8),
        ("bit_depth", C.c_uint8),
        ("color_space", C.c_int),
        ("color_range", C.c_bool),
        ("subsampling_x", C.c_uint8),
        ("subsampling_y", C.c_uint8),
        ("show_frame", C.c_bool),
        ("show_existing_frame", C.c_bool),
        ("frame_to_show_map_idx", C.c_uint8),
        ("intra_only", C.c_bool),
        ("reset_frame_context", C.c_uint8),
        ("error_resilient", C.c_bool),
        ("allow_high_precision_mv", C.c_bool),
        ("interp_filter", C.c_int),
        ("refresh_frame_context", C.c_bool),
        ("frame_parallel", C.c_bool),
        ("frame_context_idx", C.c_uint8),
        ("log2_tile_cols", C.c_uint8),
        ("log2_tile_rows", C.c_uint8),
        ("uncompressed_header_bytes", C.c_uint32),
        ("first_partition_size", C.c_uint16),
        ("base_qindex", C.c_int16),
        ("y_dc_delta_q", C.c_int8),
        ("uv_dc_delta_q", C.c_int8),
        ("uv_ac_delta_q", C.c_int8),
        ("filter_level", C.c_uint8),
        ("sharpness_level", C.c_uint8),
        ("refresh_frame_flags", C.c_uint8),
        ("ref_frame_idx", C.c_uint8 * 3),
        ("ref_frame_sign_bias", C.c_uint8 * 4),
        ("segmentation_enabled", C.c_bool),
    ]


class MV(C.Structure):
    _fields_ = [("x", C.c_int32), ("y", C.c_int32), ("ref", C.c_int32), ("pad", C.c_int32)]


class BlockInfo(C.Structure):
    _fields_ = [
        ("x", C.c_uint16),
        ("y", C.c_uint16),
        ("width", C.c_uint8),
        ("height", C.c_uint8),
        ("tx_size", C.c_uint8),
        ("is_intra", C.c_uint8),
        ("y_mode", C.c_uint8),
        ("uv_mode", C.c_uint8),
        ("ref_frame", C.c_uint8 * 2),
        ("mv", (C.c_int16 * 2) * 2),
        ("skip", C.c_uint8),
        ("coeff_offset", C.c_uint32),
        ("eob", C.c_uint16),
    ]


class ParsedFrame(C.Structure):
    _fields_ = [
        ("hdr", FrameHeader),
        ("blocks", C.POINTER(BlockInfo)),
        ("num_blocks", C.c_uint32),
        ("blocks_capacity", C.c_uint32),
        ("coeffs", C.POINTER(C.c_int16)),
        ("num_coeffs", C.c_uint32),
        ("coeffs_capacity", C.c_uint32),
        ("mv_grid", C.POINTER(MV)),
        ("mv_grid_width", C.c_uint32),
        ("mv_grid_height", C.c_uint32),
        ("mi_width_grid", C.POINTER(C.c_uint8)),
        ("mi_height_grid", C.POINTER(C.c_uint8)),
        ("mi_grid_width", C.c_uint32),
        ("mi_grid_height", C.c_uint32),
        ("mi_block_grid", C.POINTER(C.c_uint32)),
    ]


class FrameInfo(C.Structure):
    _fields_ = [
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("stride_y", C.c_uint32),
        ("stride_uv", C.c_uint32),
        ("plane_y", C.POINTER(C.c_uint8)),
        ("plane_u", C.POINTER(C.c_uint8)),
        ("plane_v", C.POINTER(C.c_uint8)),
        ("pts", C.c_int64),
    ]


class DmabufFrame(C.Structure):
    _fields_ = [
        ("fd", C.c_int),
        ("size", C.c_uint64),
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("offsets", C.c_uint32 * 3),
        ("pitches", C.c_uint32 * 3),
        ("pts", C.c_int64),
    ]


class ExportBuffer(C.Structure):
    _fields_ = [
        ("fd", C.c_int),
        ("mapped", C.c_void_p),
        ("size", C.c_uint64),
        ("priv_buf", C.c_void_p),
        ("priv_mem", C.c_void_p),
    ]


class SynthConfig(C.Structure):
    """Mirror of cvp9_synth_config_t (include/cvp9_synth.h)."""
    _fields_ = [
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("seed", C.c_uint64),
        ("gop", C.c_int),
        ("fixed_bsize", C.c_int),
        ("min_bsize", C.c_int),
        ("max_bsize", C.c_int),
        ("rect_partitions", C.c_int),
        ("fixed_tx", C.c_int),
        ("tx_weights", C.c_int * 4),
        ("density_min", C.c_double),
        ("density_max", C.c_double),
        ("coeff_max", C.c_int),
        ("coeff_scale", C.c_double),
        ("mv_range_px", C.c_int),
        ("nrefs", C.c_int),
        ("golden_every", C.c_int),
        ("altref_every", C.c_int),
        ("qindex", C.c_int),
        ("lf_level", C.c_int),
        ("sharpness", C.c_int),
        ("interp_filter", C.c_int),
        ("all_intra_modes", C.c_int),
        ("intra_in_inter", C.c_double),
        ("skip_prob", C.c_double),
        ("log2_tile_cols", C.c_int),
        ("compound_prob", C.c_double),
    ]


def layout_offsets():
    """The same offsets ref_harness.c:ref_layout reports for the reference."""
    o = C.sizeof
    return [
        o(FrameHeader), FrameHeader.width.offset, FrameHeader.base_qindex.offset,
        FrameHeader.filter_level.offset, FrameHeader.sharpness_level.offset,
        FrameHeader.refresh_frame_flags.offset, FrameHeader.ref_frame_idx.offset,
        FrameHeader.segmentation_enabled.offset,
        o(BlockInfo), BlockInfo.tx_size.offset, BlockInfo.mv.offset, BlockInfo.skip.offset,
        BlockInfo.coeff_offset.offset, BlockInfo.eob.offset,
        o(MV),
        o(ParsedFrame), ParsedFrame.blocks.offset, ParsedFrame.num_blocks.offset,
        ParsedFrame.coeffs.offset, ParsedFrame.num_coeffs.offset, ParsedFrame.mv_grid.offset,
        ParsedFrame.mv_grid_width.offset, ParsedFrame.mi_block_grid.offset,
        o(FrameInfo), FrameInfo.plane_y.offset, FrameInfo.pts.offset,
        o(ExportBuffer), o(DmabufFrame),
    ]


def i420_size(w, h):
    cw, ch = (w + 1) // 2, (h + 1) // 2
    return w * h + 2 * cw * ch
