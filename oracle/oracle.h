/*
 * oracle.h — CPU restatement of compute-vp9's reconstruction, used ONLY as
 * the checker by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg. Nothing in the product links or calls it.
 *
 * Two arithmetic profiles:
 *   REFCPU — src/decoder/vp9_reconstruct.c:13-370 plus the reference-pool and
 *            output handling of src/decoder/vp9_decoder.c:209-247. Pinned
 *            against the reference compiled from source (oracle/_ref) and the
 *            committed golden hashes in tests/golden/.
 *   SPEC   — the arithmetic of shaders/vp9_idct.comp.glsl, vp9_mc.comp.glsl,
 *            vp9_intra_pred.comp.glsl, vp9_loopfilter.comp.glsl and
 *            vp9_nv12_pack.comp.glsl, applied block by block in parse order,
 *            with chroma MC and the all-plane residual written from the VP9
 *            design. The shaders cannot run here (no graphics stack); the
 *            profile is pinned stage by stage to mechanical Python
 *            translations of the shaders' own functions (inverse transforms,
 *            luma MC, intra: tests/golden/spec_*.json) and, for the loop
 *            filter, to the REFCPU one it equals. Chroma MC and the all-plane
 *            residual have no shader counterpart: unpinned.
 *   FULL   — SPEC completed to the VP9 specification where the reference is
 *            a skeleton (oracle_full.c): unpinned, no VP9 decoder or
 *            conformance stream is present to pin it.
 */
#ifndef CVP9_ORACLE_H
#define CVP9_ORACLE_H

#include "cvp9_types.h"

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_REFCPU = 0, ORACLE_SPEC = 1, ORACLE_FULL = 2 };

/* A frame owned by the oracle: I420, stride = width (vp9_frame.c:8-34). */
typedef struct {
    uint32_t width, height, stride_y, stride_uv;
    uint8_t *y, *u, *v;
} oracle_frame_t;

/* REFCPU: whole-frame reconstruction. refs[i] may be NULL or have NULL planes
 * (the "reference missing" path). out is (re)allocated and filled. */
int  oracle_refcpu_reconstruct(const vp9_parsed_frame_t *pf,
                               const oracle_frame_t *const refs[8],
                               oracle_frame_t *out);

/* SPEC: whole-frame reconstruction from the pool slots (8). */
int  oracle_spec_reconstruct(const vp9_parsed_frame_t *pf,
                             const oracle_frame_t *const pool[8],
                             oracle_frame_t *out);

/* FULL: the shader profile completed to the VP9 specification where the
 * reference is a skeleton (oracle_full.c). Returns 0 for frames the profile
 * does not take (sizes not multiples of 8, a SWITCHABLE filter on an inter
 * frame, references of another size). */
int  oracle_full_reconstruct(const vp9_parsed_frame_t *pf,
                             const oracle_frame_t *const pool[8],
                             oracle_frame_t *out);

void oracle_frame_free(oracle_frame_t *f);

/* ── Stage-level entry points (unit tests) ─────────────────────────────── */

/* REFCPU float64 DCT basis for N = 4, 8, 16, 32 concatenated (1360 doubles). */
void oracle_refcpu_basis(double *out);

/* REFCPU float64 inverse DCT of raw coefficients (vp9_reconstruct.c:13-60). */
void oracle_refcpu_idct2d(const int16_t *in, int16_t *out, int n);

/* SPEC integer inverse DCT with dequantisation (vp9_idct.comp.glsl:654-789):
 * returns the rounded residual (before the add/clamp). */
void oracle_spec_idct2d(const int16_t *in, int32_t *out, int n, int q_dc, int q_ac);

/* SPEC intra prediction of one w x h block in place (neighbours read from
 * the same plane; vp9_intra_pred.comp.glsl:54-109 generalised to w x h). */
void oracle_spec_intra_block(uint8_t *plane, int w, int h, int stride, int x, int y,
                             int bw, int bh, int mode);

/* SPEC inter prediction of one block of dst from ref (luma: 1/8-pel MV on
 * even phases, vp9_mc.comp.glsl:61-110; chroma: the MV as 1/16 chroma pel). */
void oracle_spec_mc_block(const uint8_t *ref, int rw, int rh, int rstride,
                          uint8_t *dst, int dw, int dh, int dstride,
                          int x, int y, int bw, int bh, int mvx, int mvy, int chroma);

/* The shader 1-D inverse DCT, n = 4, 8, 16 or 32 (32-bit wrap). */
void oracle_idct1d(int n, const int *in, int *out);

/* FULL residual of one n x n TX: dequantised (32x32 halved toward zero),
 * rows then columns, tx_type 0 DCT, 1 ADST down the columns, 2 ADST along
 * the rows, 3 both; Walsh-Hadamard for 4x4 when lossless. */
void oracle_full_itx2d(const int16_t *in, int32_t *out, int n, int tx_type, int lossless,
                       int q_dc, int q_ac);

/* FULL inter prediction of one block (compound: averaged with ref1). */
void oracle_full_mc_block(const uint8_t *ref0, const uint8_t *ref1, int rw, int rh, int rstride,
                          uint8_t *dst, int dw, int dh, int dstride, int x, int y, int bw, int bh,
                          int mv0x, int mv0y, int mv1x, int mv1y, int compound, int filter, int chroma);

/* FULL intra prediction of one n x n TX in place (VP9 edge rules). */
void oracle_full_intra_tx(uint8_t *plane, int pw, int ph, int stride, int x0, int y0, int n,
                          int mode, int have_top, int have_left, int have_right);

/* Loop filter in place on a luma plane: REFCPU (level 0 = off) or SPEC
 * (threshold floored at 1, always on). */
void oracle_loopfilter(uint8_t *y, uint32_t w, uint32_t h, uint32_t stride,
                       int level, int sharpness, int profile);

/* I420 -> NV12 (vp9_nv12_pack.comp.glsl:33-59); dst holds w*h + 2*cw*ch bytes. */
void oracle_nv12_pack(const uint8_t *i420, uint8_t *dst, uint32_t w, uint32_t h);

/* ── Stream harness: recon + reference pool + delivery ─────────────────── */

typedef struct oracle_stream oracle_stream_t;

oracle_stream_t *oracle_stream_create(int profile);
void             oracle_stream_destroy(oracle_stream_t *s);

/* Reconstruct one frame and apply the profile's pool update. The decoded
 * I420 frame (w*h + 2*cw*ch bytes) is copied to out_i420 if non-NULL. */
int              oracle_stream_decode(oracle_stream_t *s, const vp9_parsed_frame_t *pf,
                                      uint8_t *out_i420);

/* ── Profile 2 (10-bit, oracle_hbd.c): frames of uint16 samples held in
 * oracle_frame_t (plane pointers cast), coefficients dequantised int32 ── */

int  oracle_hbd_reconstruct(const vp9_parsed_frame_t *pf, const int32_t *coeffs,
                            const oracle_frame_t *const pool[8], oracle_frame_t *out);
/* one 1-D inverse (DCT, or ADST for n < 32 when adst), 64-bit */
void oracle_hbd_itx1d(int n, int adst, const int64_t *in, int64_t *out);
/* residual of one n x n TX (tx_type as oracle_full_itx2d) */
void oracle_hbd_itx2d(const int32_t *in, int64_t *out, int n, int tx_type, int lossless);
void oracle_hbd_mc_block(const uint16_t *ref0, const uint16_t *ref1, int rw, int rh, int rstride,
                         uint16_t *dst, int dw, int dh, int dstride, int x, int y, int bw, int bh,
                         int mv0x, int mv0y, int mv1x, int mv1y, int compound, int filter, int chroma);
void oracle_hbd_intra_tx(uint16_t *plane, int pw, int ph, int stride, int x0, int y0, int n,
                         int mode, int have_top, int have_left, int have_right);

typedef struct oracle_hbd_stream oracle_hbd_stream_t;
oracle_hbd_stream_t *oracle_hbd_stream_create(void);
void                 oracle_hbd_stream_destroy(oracle_hbd_stream_t *s);
/* One frame and the pool update (refresh_frame_flags, 0 meaning slot 0);
 * the frame (w*h + 2*cw*ch samples) to out_i420 when non-NULL. */
int                  oracle_hbd_stream_decode(oracle_hbd_stream_t *s, const vp9_parsed_frame_t *pf,
                                              const int32_t *coeffs, uint16_t *out_i420);

/* 8-bit DC/AC quantiser lookups (src/decoder/vp9_dequant.h:12-75). */
int oracle_dc_quant(int qindex);
int oracle_ac_quant(int qindex);

#ifdef __cplusplus
}
#endif

#endif /* CVP9_ORACLE_H */
