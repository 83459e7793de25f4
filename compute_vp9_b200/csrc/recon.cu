/*
 * recon.cu — VP9 reconstruction kernels for sm_100a.
 *
 * Three launches per batch of frames (one frame from each of J streams):
 *
 *   k_scan_blocks   one thread per block: superblock (SB) membership, the
 *                   contiguous block range of every SB, layout checks.
 *   k_recon<A>      one CTA per SB ticket, tickets handed out in
 *                   SB-diagonal order across all streams of the batch. A CTA
 *                   builds its SB's dependency levels in shared memory, waits
 *                   (bounded) for the left / above / above-left SBs only when
 *                   the SB holds intra blocks, then runs the levels:
 *                   prediction + first transform pass, barrier, second pass +
 *                   residual add, barrier. The SB tile (with a one-pixel
 *                   halo) lives in shared memory; the finished tile is
 *                   written once and the SB's done flag released.
 *   k_loopfilter<A> the 4-tap deblock on 64x64 luma tiles shifted by 4 px so
 *                   every filter tap of every 8-px edge falls inside one tile
 *                   (horizontal pass then vertical pass, in place), with the
 *                   NV12 pack fused into the same tile pass.
 *
 * Arithmetic profiles (template A):
 *   CVP9_ARITH_REFCPU reproduces src/decoder/vp9_reconstruct.c:194-370
 *     bit for bit: float64 inverse DCT of the raw coefficients with the
 *     host-built basis (separately rounded products and sums, k ascending),
 *     bilinear MC, the CPU's 127 edge rules, luma-only residual.
 *   CVP9_ARITH_SPEC reproduces the shader arithmetic: dequantised integer
 *     butterflies (vp9_idct.comp.glsl), regular 8-tap MC (vp9_mc.comp.glsl)
 *     on luma and chroma, intra with the shader's availability rules
 *     (vp9_intra_pred.comp.glsl), the residual of every TX of every plane.
 *
 * No tensor cores: every sample is integer-exact and nothing here is a dense
 * contraction; the kernels are bound by memory traffic and dependency
 * latency.
 */
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "recon_job.h"
#include "vp9_tables.h"
#include "recon_launch.h"

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxBlocks = 128;      /* blocks per SB (the tile parser emits at most 64) */
constexpr int kCoefStage = 6144;     /* int16 coefficients staged per SB (64x64 luma + chroma) */
constexpr int kMaxItems = 1536;      /* TX columns per SB: 4x4 TXs on all three planes */
constexpr int kYPitch = 72;          /* luma tile row pitch; x = 0 at byte 4 */
constexpr int kCPitch = 40;          /* chroma tile row pitch; x = 0 at byte 4 */
constexpr int kTempPitch = 65;       /* doubles per REFCPU temp row */
constexpr int kStagePerWarp = 768;   /* bytes of MC staging per warp */
constexpr int kTyBytes = (65 * kYPitch + 15) / 16 * 16;
constexpr int kTcBytes = (33 * kCPitch + 15) / 16 * 16;
constexpr long long kSpinLimit = 1ll << 20;   /* ~0.25 s of polling */

__constant__ double c_dct[16 + 64 + 256 + 1024];      /* N = 4, 8, 16, 32 */
__constant__ int c_subpel[16][8] = CVP9_SUBPEL_REGULAR_INIT;
/* FULL: the frame header's filter, interp_filter 0..3 */
__constant__ int c_subpel4[4][16][8] = { CVP9_SUBPEL_REGULAR_INIT, CVP9_SUBPEL_SMOOTH_INIT,
                                         CVP9_SUBPEL_SHARP_INIT, CVP9_SUBPEL_BILINEAR_INIT };
__constant__ uint8_t c_tx_type[10] = CVP9_INTRA_TX_TYPE_INIT;
/* the same taps as signed bytes, taps 0-3 and 4-7 in two words, for dp4a
 * (phase 0's 128 does not fit a byte: callers take the centre sample for
 * it, which is what its filter computes); uploaded by cvp9k_configure */
__constant__ uint32_t c_subpel_pk[16][2];
/* the four VP9 filters (c_subpel4) packed the same way, for the FULL profile */
__constant__ uint32_t c_subpel4_pk[4][16][2];

__device__ __forceinline__ const double *dct_basis(int txl)
{
    return c_dct + (txl == 0 ? 0 : txl == 1 ? 16 : txl == 2 ? 80 : 336);
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ uint32_t tap_round(int acc) { return (uint32_t)clampi((acc + 64) >> 7, 0, 255); }

__device__ __forceinline__ int dp4a_su(uint32_t taps, uint32_t px, int c)
{
    int d;
    asm("dp4a.s32.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(taps), "r"(px), "r"(c));
    return d;
}

/* One 8-tap output from samples s0 (samples 0-3 of the window) and s1
 * (4-7): phase 0 is the centre sample itself. */
__device__ __forceinline__ uint32_t tap8(uint32_t ta, uint32_t tb, int phase, uint32_t s0, uint32_t s1)
{
    return phase ? tap_round(dp4a_su(tb, s1, dp4a_su(ta, s0, 0))) : (s0 >> 24);
}

/* t / d for 0 <= t < 4096 and 1 <= d <= 16 without an integer divide:
 * (t * ceil(2^16 / d)) >> 16 is exact in that range. */
__device__ __forceinline__ int div_small(int t, int d)
{
    return (int)(((unsigned)t * ((65536u + (unsigned)d - 1u) / (unsigned)d)) >> 16);
}

/* ── Asynchronous global -> shared copies (16 bytes, both sides aligned) ── */

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

/* 8 and 4 bytes (both sides aligned to the size) */
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" :: "r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem)
{
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" :: "r"(sa), "l"(gmem) : "memory");
}
/* all but the newest group have landed */
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }


/* ── 32-bit wrap-around integer for the shader butterflies ───────────────── */
struct wi {
    int v;
    __device__ __forceinline__ wi() : v(0) {}
    __device__ __forceinline__ wi(int x) : v(x) {}
};
__device__ __forceinline__ wi operator+(wi a, wi b) { return wi((int)((unsigned)a.v + (unsigned)b.v)); }
__device__ __forceinline__ wi operator-(wi a, wi b) { return wi((int)((unsigned)a.v - (unsigned)b.v)); }
__device__ __forceinline__ wi operator-(wi a) { return wi((int)(0u - (unsigned)a.v)); }
__device__ __forceinline__ wi operator*(wi a, int k) { return wi((int)((unsigned)a.v * (unsigned)k)); }
__device__ __forceinline__ wi RS(wi x) { return wi(((int)((unsigned)x.v + 8192u)) >> 14); }
__device__ __forceinline__ wi shr(wi x, int k) { return wi(x.v >> k); }

/* 64-bit integer for the same butterflies at 10 bits (profile 2): products
 * of the +-2^17 dequantised range and the Q14 multipliers need 64 bits. */
struct wl {
    long long v;
    __device__ __forceinline__ wl() : v(0) {}
    __device__ __forceinline__ wl(long long x) : v(x) {}
};
__device__ __forceinline__ wl operator+(wl a, wl b) { return wl(a.v + b.v); }
__device__ __forceinline__ wl operator-(wl a, wl b) { return wl(a.v - b.v); }
__device__ __forceinline__ wl operator-(wl a) { return wl(-a.v); }
__device__ __forceinline__ wl operator*(wl a, int k) { return wl(a.v * (long long)k); }
__device__ __forceinline__ wl RS(wl x) { return wl((x.v + 8192) >> 14); }
__device__ __forceinline__ wl shr(wl x, int k) { return wl(x.v >> k); }

/* cos(k*pi/64) in Q14 */
enum : int {
    K1 = 16364, K2 = 16305, K3 = 16207, K4 = 16069, K5 = 15893, K6 = 15679,
    K7 = 15426, K8 = 15137, K9 = 14811, K10 = 14449, K11 = 14053, K12 = 13623,
    K13 = 13160, K14 = 12665, K15 = 12140, K16 = 11585, K17 = 11003, K18 = 10394,
    K19 = 9760, K20 = 9102, K21 = 8423, K22 = 7723, K23 = 7005, K24 = 6270,
    K25 = 5520, K26 = 4756, K27 = 3981, K28 = 3196, K29 = 2404, K30 = 1606,
    K31 = 804
};

/* 1-D inverse DCTs, in place on x[0..N). Same stage structure and rounding
 * as vp9_idct.comp.glsl:47-649. */
template <class T>
__device__ __forceinline__ void idct4(T *x)
{
    T s0 = RS((x[0] + x[2]) * K16), s1 = RS((x[0] - x[2]) * K16);
    T s2 = RS(x[1] * K24 - x[3] * K8), s3 = RS(x[1] * K8 + x[3] * K24);
    x[0] = s0 + s3; x[1] = s1 + s2; x[2] = s1 - s2; x[3] = s0 - s3;
}

template <class T>
__device__ __forceinline__ void idct8(T *x)
{
    T a[8], b[8];
    a[0] = x[0]; a[1] = x[2]; a[2] = x[4]; a[3] = x[6];
    a[4] = RS(x[1] * K28 - x[7] * K4); a[7] = RS(x[1] * K4 + x[7] * K28);
    a[5] = RS(x[5] * K12 - x[3] * K20); a[6] = RS(x[5] * K20 + x[3] * K12);
    b[0] = RS((a[0] + a[2]) * K16); b[1] = RS((a[0] - a[2]) * K16);
    b[2] = RS(a[1] * K24 - a[3] * K8); b[3] = RS(a[1] * K8 + a[3] * K24);
    b[4] = a[4] + a[5]; b[5] = a[4] - a[5]; b[6] = -a[6] + a[7]; b[7] = a[6] + a[7];
    a[0] = b[0] + b[3]; a[1] = b[1] + b[2]; a[2] = b[1] - b[2]; a[3] = b[0] - b[3];
    a[4] = b[4]; a[5] = RS((b[6] - b[5]) * K16); a[6] = RS((b[5] + b[6]) * K16); a[7] = b[7];
#pragma unroll
    for (int i = 0; i < 4; i++) { x[i] = a[i] + a[7 - i]; x[7 - i] = a[i] - a[7 - i]; }
}

template <class T>
__device__ __forceinline__ void idct16(T *x)
{
    T a[16], b[16];
    a[0] = x[0]; a[1] = x[8]; a[2] = x[4]; a[3] = x[12]; a[4] = x[2]; a[5] = x[10];
    a[6] = x[6]; a[7] = x[14]; a[8] = x[1]; a[9] = x[9]; a[10] = x[5]; a[11] = x[13];
    a[12] = x[3]; a[13] = x[11]; a[14] = x[7]; a[15] = x[15];
#pragma unroll
    for (int i = 0; i < 8; i++) b[i] = a[i];
    b[8] = RS(a[8] * K30 - a[15] * K2);   b[15] = RS(a[8] * K2 + a[15] * K30);
    b[9] = RS(a[9] * K14 - a[14] * K18);  b[14] = RS(a[9] * K18 + a[14] * K14);
    b[10] = RS(a[10] * K22 - a[13] * K10); b[13] = RS(a[10] * K10 + a[13] * K22);
    b[11] = RS(a[11] * K6 - a[12] * K26);  b[12] = RS(a[11] * K26 + a[12] * K6);
#pragma unroll
    for (int i = 0; i < 4; i++) a[i] = b[i];
    a[4] = RS(b[4] * K28 - b[7] * K4); a[7] = RS(b[4] * K4 + b[7] * K28);
    a[5] = RS(b[5] * K12 - b[6] * K20); a[6] = RS(b[5] * K20 + b[6] * K12);
    a[8] = b[8] + b[9]; a[9] = b[8] - b[9]; a[10] = -b[10] + b[11]; a[11] = b[10] + b[11];
    a[12] = b[12] + b[13]; a[13] = b[12] - b[13]; a[14] = -b[14] + b[15]; a[15] = b[14] + b[15];
    b[0] = RS((a[0] + a[1]) * K16); b[1] = RS((a[0] - a[1]) * K16);
    b[2] = RS(a[2] * K24 - a[3] * K8); b[3] = RS(a[2] * K8 + a[3] * K24);
    b[4] = a[4] + a[5]; b[5] = a[4] - a[5]; b[6] = -a[6] + a[7]; b[7] = a[6] + a[7];
    b[8] = a[8]; b[15] = a[15];
    b[9] = RS(-a[9] * K8 + a[14] * K24);   b[14] = RS(a[9] * K24 + a[14] * K8);
    b[10] = RS(-a[10] * K24 - a[13] * K8); b[13] = RS(-a[10] * K8 + a[13] * K24);
    b[11] = a[11]; b[12] = a[12];
    a[0] = b[0] + b[3]; a[1] = b[1] + b[2]; a[2] = b[1] - b[2]; a[3] = b[0] - b[3];
    a[4] = b[4]; a[5] = RS((b[6] - b[5]) * K16); a[6] = RS((b[5] + b[6]) * K16); a[7] = b[7];
    a[8] = b[8] + b[11]; a[9] = b[9] + b[10]; a[10] = b[9] - b[10]; a[11] = b[8] - b[11];
    a[12] = -b[12] + b[15]; a[13] = -b[13] + b[14]; a[14] = b[13] + b[14]; a[15] = b[12] + b[15];
#pragma unroll
    for (int i = 0; i < 4; i++) { b[i] = a[i] + a[7 - i]; b[7 - i] = a[i] - a[7 - i]; }
    b[8] = a[8]; b[9] = a[9];
    b[10] = RS((-a[10] + a[13]) * K16); b[13] = RS((a[10] + a[13]) * K16);
    b[11] = RS((-a[11] + a[12]) * K16); b[12] = RS((a[11] + a[12]) * K16);
    b[14] = a[14]; b[15] = a[15];
#pragma unroll
    for (int i = 0; i < 8; i++) { x[i] = b[i] + b[15 - i]; x[15 - i] = b[i] - b[15 - i]; }
}

template <class T>
__device__ __forceinline__ void idct32(T *x)
{
    T a[32], b[32];
    a[0] = x[0]; a[1] = x[16]; a[2] = x[8]; a[3] = x[24]; a[4] = x[4]; a[5] = x[20];
    a[6] = x[12]; a[7] = x[28]; a[8] = x[2]; a[9] = x[18]; a[10] = x[10]; a[11] = x[26];
    a[12] = x[6]; a[13] = x[22]; a[14] = x[14]; a[15] = x[30];
    a[16] = RS(x[1] * K31 - x[31] * K1);  a[31] = RS(x[1] * K1 + x[31] * K31);
    a[17] = RS(x[17] * K15 - x[15] * K17); a[30] = RS(x[17] * K17 + x[15] * K15);
    a[18] = RS(x[9] * K23 - x[23] * K9);  a[29] = RS(x[9] * K9 + x[23] * K23);
    a[19] = RS(x[25] * K7 - x[7] * K25);  a[28] = RS(x[25] * K25 + x[7] * K7);
    a[20] = RS(x[5] * K27 - x[27] * K5);  a[27] = RS(x[5] * K5 + x[27] * K27);
    a[21] = RS(x[21] * K11 - x[11] * K21); a[26] = RS(x[21] * K21 + x[11] * K11);
    a[22] = RS(x[13] * K19 - x[19] * K13); a[25] = RS(x[13] * K13 + x[19] * K19);
    a[23] = RS(x[29] * K3 - x[3] * K29);  a[24] = RS(x[29] * K29 + x[3] * K3);
    /* stage 2 */
#pragma unroll
    for (int i = 0; i < 8; i++) b[i] = a[i];
    b[8] = RS(a[8] * K30 - a[15] * K2);   b[15] = RS(a[8] * K2 + a[15] * K30);
    b[9] = RS(a[9] * K14 - a[14] * K18);  b[14] = RS(a[9] * K18 + a[14] * K14);
    b[10] = RS(a[10] * K22 - a[13] * K10); b[13] = RS(a[10] * K10 + a[13] * K22);
    b[11] = RS(a[11] * K6 - a[12] * K26);  b[12] = RS(a[11] * K26 + a[12] * K6);
#pragma unroll
    for (int i = 16; i < 32; i += 4) {
        b[i] = a[i] + a[i + 1]; b[i + 1] = a[i] - a[i + 1];
        b[i + 2] = -a[i + 2] + a[i + 3]; b[i + 3] = a[i + 2] + a[i + 3];
    }
    /* stage 3 */
#pragma unroll
    for (int i = 0; i < 4; i++) a[i] = b[i];
    a[4] = RS(b[4] * K28 - b[7] * K4); a[7] = RS(b[4] * K4 + b[7] * K28);
    a[5] = RS(b[5] * K12 - b[6] * K20); a[6] = RS(b[5] * K20 + b[6] * K12);
#pragma unroll
    for (int i = 8; i < 16; i += 4) {
        a[i] = b[i] + b[i + 1]; a[i + 1] = b[i] - b[i + 1];
        a[i + 2] = -b[i + 2] + b[i + 3]; a[i + 3] = b[i + 2] + b[i + 3];
    }
    a[16] = b[16]; a[31] = b[31];
    a[17] = RS(-b[17] * K4 + b[30] * K28);  a[30] = RS(b[17] * K28 + b[30] * K4);
    a[18] = RS(-b[18] * K28 - b[29] * K4);  a[29] = RS(-b[18] * K4 + b[29] * K28);
    a[19] = b[19]; a[20] = b[20];
    a[21] = RS(-b[21] * K20 + b[26] * K12); a[26] = RS(b[21] * K12 + b[26] * K20);
    a[22] = RS(-b[22] * K12 - b[25] * K20); a[25] = RS(-b[22] * K20 + b[25] * K12);
    a[23] = b[23]; a[24] = b[24]; a[27] = b[27]; a[28] = b[28];
    /* stage 4 */
    b[0] = RS((a[0] + a[1]) * K16); b[1] = RS((a[0] - a[1]) * K16);
    b[2] = RS(a[2] * K24 - a[3] * K8); b[3] = RS(a[2] * K8 + a[3] * K24);
    b[4] = a[4] + a[5]; b[5] = a[4] - a[5]; b[6] = -a[6] + a[7]; b[7] = a[6] + a[7];
    b[8] = a[8]; b[15] = a[15];
    b[9] = RS(-a[9] * K8 + a[14] * K24);   b[14] = RS(a[9] * K24 + a[14] * K8);
    b[10] = RS(-a[10] * K24 - a[13] * K8); b[13] = RS(-a[10] * K8 + a[13] * K24);
    b[11] = a[11]; b[12] = a[12];
#pragma unroll
    for (int i = 16; i < 32; i += 8) {
        b[i] = a[i] + a[i + 3]; b[i + 1] = a[i + 1] + a[i + 2];
        b[i + 2] = a[i + 1] - a[i + 2]; b[i + 3] = a[i] - a[i + 3];
        b[i + 4] = -a[i + 4] + a[i + 7]; b[i + 5] = -a[i + 5] + a[i + 6];
        b[i + 6] = a[i + 5] + a[i + 6]; b[i + 7] = a[i + 4] + a[i + 7];
    }
    /* stage 5 */
    a[0] = b[0] + b[3]; a[1] = b[1] + b[2]; a[2] = b[1] - b[2]; a[3] = b[0] - b[3];
    a[4] = b[4]; a[5] = RS((b[6] - b[5]) * K16); a[6] = RS((b[5] + b[6]) * K16); a[7] = b[7];
    a[8] = b[8] + b[11]; a[9] = b[9] + b[10]; a[10] = b[9] - b[10]; a[11] = b[8] - b[11];
    a[12] = -b[12] + b[15]; a[13] = -b[13] + b[14]; a[14] = b[13] + b[14]; a[15] = b[12] + b[15];
    a[16] = b[16]; a[17] = b[17];
    a[18] = RS(-b[18] * K8 + b[29] * K24);  a[29] = RS(b[18] * K24 + b[29] * K8);
    a[19] = RS(-b[19] * K8 + b[28] * K24);  a[28] = RS(b[19] * K24 + b[28] * K8);
    a[20] = RS(-b[20] * K24 - b[27] * K8);  a[27] = RS(-b[20] * K8 + b[27] * K24);
    a[21] = RS(-b[21] * K24 - b[26] * K8);  a[26] = RS(-b[21] * K8 + b[26] * K24);
    a[22] = b[22]; a[23] = b[23]; a[24] = b[24]; a[25] = b[25]; a[30] = b[30]; a[31] = b[31];
    /* stage 6 */
#pragma unroll
    for (int i = 0; i < 4; i++) { b[i] = a[i] + a[7 - i]; b[7 - i] = a[i] - a[7 - i]; }
    b[8] = a[8]; b[9] = a[9];
    b[10] = RS((-a[10] + a[13]) * K16); b[13] = RS((a[10] + a[13]) * K16);
    b[11] = RS((-a[11] + a[12]) * K16); b[12] = RS((a[11] + a[12]) * K16);
    b[14] = a[14]; b[15] = a[15];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        b[16 + i] = a[16 + i] + a[23 - i]; b[23 - i] = a[16 + i] - a[23 - i];
        b[24 + i] = -a[24 + i] + a[31 - i]; b[31 - i] = a[24 + i] + a[31 - i];
    }
    /* stage 7 */
#pragma unroll
    for (int i = 0; i < 8; i++) { a[i] = b[i] + b[15 - i]; a[15 - i] = b[i] - b[15 - i]; }
#pragma unroll
    for (int i = 16; i < 20; i++) a[i] = b[i];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        a[20 + i] = RS((-b[20 + i] + b[27 - i]) * K16);
        a[27 - i] = RS((b[20 + i] + b[27 - i]) * K16);
    }
#pragma unroll
    for (int i = 28; i < 32; i++) a[i] = b[i];
    /* output */
#pragma unroll
    for (int i = 0; i < 16; i++) { x[i] = a[i] + a[31 - i]; x[31 - i] = a[i] - a[31 - i]; }
}

/* ── Shared-memory layout of one reconstruction CTA ─────────────────────── */

struct BlkS {
    uint8_t  x, y;          /* local luma position in the SB               */
    uint8_t  w, h;          /* coded size                                  */
    uint8_t  cw, ch;        /* size clamped to the frame                   */
    uint8_t  txl;           /* luma tx_size 0..3                           */
    uint8_t  flags;         /* 1 intra, 2 skip                             */
    uint8_t  ymode, uvmode;
    uint8_t  ref0;
    uint8_t  ptxl[3];       /* residual TX log2-4 per plane                */
    uint8_t  pnx[3];        /* residual TXs per row per plane              */
    uint8_t  ref1;          /* FULL: second reference of a compound block  */
    uint16_t pnt[3];        /* residual TX count per plane                 */
    int16_t  mvx, mvy;
    int16_t  mv1x, mv1y;    /* FULL: its MV                                */
    uint32_t coeff;
};
/* BlkS.flags: 1 intra, 2 skip, 4 FULL intra (one warp predicts and
 * reconstructs the block TX by TX; no residual items) */

struct ReconSmem {
    union {
        double  d[64 * kTempPitch];              /* REFCPU first-pass output    */
        int32_t i[64 * 64 + 2 * 32 * 32];        /* SPEC column-pass output     */
    } temp;
    /* tiles, contiguous and 16-byte sized so they fill with vector stores */
    uint8_t  ty[kTyBytes];                       /* luma tile, row 0 = halo     */
    uint8_t  tu[kTcBytes];
    uint8_t  tv[kTcBytes];
    int16_t  coef[kCoefStage];                   /* the SB's coefficient span   */
    cvp9_job_t jc;                               /* this ticket's job           */
    BlkS     blk[kMaxBlocks];
    unsigned long long lvl_cnt[kMaxBlocks + 1];
    uint8_t  lvl_big[kMaxBlocks + 1];            /* level holds a block that is
                                                  * not a small intra block    */
    uint32_t txmask[256 + 64 + 64];              /* per-TX column-nonzero bits  */
    uint16_t cell[256];                          /* owner block + 1 per 4x4     */
    uint16_t lvl[kMaxBlocks];
    uint16_t order[kMaxBlocks];
    uint16_t chunk_off[kMaxBlocks + 1];
    uint16_t item_off[kMaxBlocks + 1];
    uint16_t base_blk[kMaxBlocks + 1];
    uint16_t base_chunk[kMaxBlocks + 1];
    uint16_t base_item[kMaxBlocks + 1];
    uint8_t  chunk_blk[256];                     /* chunk -> block position     */
    uint8_t  item_blk[kMaxItems];                /* TX column/row -> position   */
    alignas(16) uint8_t stage[kWarps][kStagePerWarp];
    int      scan_tmp[2 * kWarps];
    unsigned c_lo, c_hi;                         /* coefficient span of the SB  */
    int      ticket;
    int      nlev;
    int      nb;
};

__device__ __forceinline__ uint8_t &TY(ReconSmem &s, int x, int y) { return s.ty[(y + 1) * kYPitch + x + 4]; }
__device__ __forceinline__ uint8_t &TC(ReconSmem &s, int p, int x, int y)
{
    return (p == 1 ? s.tu : s.tv)[(y + 1) * kCPitch + x + 4];
}

__device__ __forceinline__ int max_tx_for(int w, int h)
{
    int m = w < h ? w : h;
    return m >= 32 ? 3 : (m >= 16 ? 2 : (m >= 8 ? 1 : 0));
}

/* Residual TX layout of one block (plane TX size, TXs per row, TX count).
 * REFCPU: luma only, counts from the frame-clamped size
 * (vp9_reconstruct.c:336-347). SPEC: every plane in the tile parser's layout
 * (vp9_kf_tile.c:320-396): coded area clipped at the MI-aligned frame edge. */
/* The tile parser's TX layout of one plane of a block (vp9_kf_tile.c:
 * 320-396): TX size, TXs per row and per column over the coded area clipped
 * at the MI-aligned frame edge, and the plane block width (sub-8x8 blocks
 * code a whole 8x8, chroma at least 4x4). */
__device__ __forceinline__ void plane_layout(const BlkS &b, const cvp9_job_t &job, int gx, int gy, int p,
                                             int &tx, int &nx, int &ny, int &pbw)
{
    int sub8 = b.w < 8 || b.h < 8;
    int ew = sub8 ? 8 : b.w, eh = sub8 ? 8 : b.h;
    int mi_col = gx >> 3, mi_row = gy >> 3;
    int ss = p > 0;
    int pw = ss ? ew / 2 : ew, ph = ss ? eh / 2 : eh;
    pw = pw < 4 ? 4 : pw;
    ph = ph < 4 ? 4 : ph;
    tx = b.txl;
    if (ss) { int mt = max_tx_for(pw, ph); tx = sub8 ? 0 : (tx > mt ? mt : tx); }
    int t4 = 1 << tx;
    int o4x = (mi_col * 2) >> ss, o4y = (mi_row * 2) >> ss;
    int mw = pw / 4, mh = ph / 4;
    int lim_w = ((job.mi_cols * 2) >> ss) - o4x, lim_h = ((job.mi_rows * 2) >> ss) - o4y;
    if (mw > lim_w) mw = lim_w;
    if (mh > lim_h) mh = lim_h;
    nx = mw > 0 ? (mw + t4 - 1) / t4 : 0;
    ny = mh > 0 ? (mh + t4 - 1) / t4 : 0;
    pbw = pw;
}

template <int A>
__device__ void residual_layout(BlkS &b, const cvp9_job_t &job, int gx, int gy)
{
    b.pnt[0] = b.pnt[1] = b.pnt[2] = 0;
    b.pnx[0] = b.pnx[1] = b.pnx[2] = 0;
    b.ptxl[0] = b.ptxl[1] = b.ptxl[2] = 0;
    if (b.flags & 2) return;
    if (A == CVP9_ARITH_REFCPU) {
        int n = 4 << b.txl;
        int nx = b.cw / n, ny = b.ch / n;
        b.ptxl[0] = b.txl;
        b.pnx[0] = (uint8_t)nx;
        b.pnt[0] = (uint16_t)(nx * ny);
    } else {
        for (int p = 0; p < 3; p++) {
            int tx, nx, ny, pbw;
            plane_layout(b, job, gx, gy, p, tx, nx, ny, pbw);
            b.ptxl[p] = (uint8_t)tx;
            b.pnx[p] = (uint8_t)nx;
            b.pnt[p] = (uint16_t)(nx * ny);
        }
    }
}

__device__ __forceinline__ int block_items(const BlkS &b)
{
    if (b.flags & 4) return 0;      /* FULL intra: reconstructed by its prediction warp */
    return b.pnt[0] * (4 << b.ptxl[0]) + b.pnt[1] * (4 << b.ptxl[1]) + b.pnt[2] * (4 << b.ptxl[2]);
}

__device__ __forceinline__ int block_chunks(const BlkS &b)
{
    return ((b.cw + 7) >> 3) * ((b.ch + 7) >> 3);
}

/* ── Prediction of one 8x8 luma chunk (+ its 4x4 chroma) by one warp ───── */

template <int A>
__device__ void predict_intra_chunk(ReconSmem &s, const BlkS &b, int gbx, int gby,
                                    int lx0, int ly0, int lw, int lh,
                                    int cx0, int cy0, int clw, int clh, int lane)
{
    const int fill = A == CVP9_ARITH_REFCPU ? 127 : 128;
    /* luma */
    {
        int has_a = gby > 0, has_l = gbx > 0;
        int dc = 128;
        if (b.ymode == 0) {
            unsigned sa = 0, sl = 0;
            for (int i = lane; i < b.cw; i += 32) sa += has_a ? TY(s, b.x + i, b.y - 1) : (unsigned)fill;
            for (int i = lane; i < b.ch; i += 32) sl += has_l ? TY(s, b.x - 1, b.y + i) : (unsigned)fill;
            sa = __reduce_add_sync(0xffffffffu, sa);
            sl = __reduce_add_sync(0xffffffffu, sl);
            if (A == CVP9_ARITH_REFCPU) {
                unsigned n = b.cw + b.ch;
                dc = (int)((sa + sl + (n >> 1)) / n);
            } else {
                if (has_a && has_l) dc = (int)((sa + sl + (unsigned)(b.cw + b.ch) / 2) / (unsigned)(b.cw + b.ch));
                else if (has_a) dc = (int)((sa + (unsigned)b.cw / 2) / (unsigned)b.cw);
                else if (has_l) dc = (int)((sl + (unsigned)b.ch / 2) / (unsigned)b.ch);
            }
        }
        int tl = (has_a && has_l) ? TY(s, b.x - 1, b.y - 1) : fill;
        for (int idx = lane; idx < 64; idx += 32) {
            int r = idx >> 3, c = idx & 7;
            if (r >= lh || c >= lw) continue;
            int X = lx0 + c, Y = ly0 + r;
            int av = has_a ? TY(s, X, b.y - 1) : fill;
            int lv = has_l ? TY(s, b.x - 1, Y) : fill;
            int v;
            if (A == CVP9_ARITH_REFCPU) {
                v = b.ymode == 0 ? dc : b.ymode == 1 ? av : b.ymode == 2 ? lv : clampi(av + lv - tl, 0, 255);
            } else {
                v = b.ymode == 0 ? dc : b.ymode == 2 ? lv : b.ymode == 9 ? clampi(av + lv - tl, 0, 255) : av;
            }
            TY(s, X, Y) = (uint8_t)v;
        }
    }
    /* chroma: both planes, uv_mode */
    {
        int gcx = gbx >> 1, gcy = gby >> 1;
        int bcx = b.x >> 1, bcy = b.y >> 1;
        int cbw = (b.cw + 1) >> 1, cbh = (b.ch + 1) >> 1;
        int has_a = gcy > 0, has_l = gcx > 0;
        int dcs[2] = { 128, 128 };
        if (b.uvmode == 0) {
#pragma unroll
            for (int p = 1; p <= 2; p++) {
                unsigned sa = 0, sl = 0;
                for (int i = lane; i < cbw; i += 32) sa += has_a ? TC(s, p, bcx + i, bcy - 1) : (unsigned)fill;
                for (int i = lane; i < cbh; i += 32) sl += has_l ? TC(s, p, bcx - 1, bcy + i) : (unsigned)fill;
                sa = __reduce_add_sync(0xffffffffu, sa);
                sl = __reduce_add_sync(0xffffffffu, sl);
                int dc = 128;
                if (A == CVP9_ARITH_REFCPU) {
                    unsigned n = cbw + cbh;
                    dc = (int)((sa + sl + (n >> 1)) / n);
                } else {
                    if (has_a && has_l) dc = (int)((sa + sl + (unsigned)(cbw + cbh) / 2) / (unsigned)(cbw + cbh));
                    else if (has_a) dc = (int)((sa + (unsigned)cbw / 2) / (unsigned)cbw);
                    else if (has_l) dc = (int)((sl + (unsigned)cbh / 2) / (unsigned)cbh);
                }
                dcs[p - 1] = dc;
            }
        }
        int p = 1 + (lane >> 4);
        int r = (lane >> 2) & 3, c = lane & 3;
        if (r < clh && c < clw) {
            int X = cx0 + c, Y = cy0 + r;
            int av = has_a ? TC(s, p, X, bcy - 1) : fill;
            int lv = has_l ? TC(s, p, bcx - 1, Y) : fill;
            int tl = (has_a && has_l) ? TC(s, p, bcx - 1, bcy - 1) : fill;
            int m = b.uvmode, v;
            int dc = p == 1 ? dcs[0] : dcs[1];
            if (A == CVP9_ARITH_REFCPU) {
                v = m == 0 ? dc : m == 1 ? av : m == 2 ? lv : clampi(av + lv - tl, 0, 255);
            } else {
                v = m == 0 ? dc : m == 2 ? lv : m == 9 ? clampi(av + lv - tl, 0, 255) : av;
            }
            TC(s, p, X, Y) = (uint8_t)v;
        }
    }
}

/* Stage a (sw x sh) window of a reference plane starting at (x0, y0), at
 * most 16 wide and 2*MAXI high, every sample clamped into [0, pw-1] x
 * [0, ph-1], in two steps: every lane's loads first, then its shared-memory
 * stores. (Loaded and stored one by one, each load waits for the store
 * before it, which may alias: a round trip to L2 per row.) */
template <int MAXI>
struct WinRows {
    uint32_t v[MAXI];
    __device__ __forceinline__ void load(const uint8_t *__restrict__ plane, int stride, int pw, int ph,
                                         int x0, int y0, int sw, int sh, int lane)
    {
        const int xm = pw > 0 ? pw - 1 : 0, ym = ph > 0 ? ph - 1 : 0;
        const int sx = lane & 15;
        const int xx = clampi(x0 + sx, 0, xm);
#pragma unroll
        for (int k = 0; k < MAXI; k++) {
            const int sy = (lane >> 4) + 2 * k;
            v[k] = (sx < sw && sy < sh) ? (uint32_t)__ldg(plane + (size_t)clampi(y0 + sy, 0, ym) * stride + xx) : 0u;
        }
    }
    __device__ __forceinline__ void store(uint8_t *st, int sp, int sw, int sh, int lane) const
    {
        const int sx = lane & 15;
        if (sx >= sw) return;
#pragma unroll
        for (int k = 0; k < MAXI; k++) {
            const int sy = (lane >> 4) + 2 * k;
            if (sy < sh) st[sy * sp + sx] = (uint8_t)v[k];
        }
    }
};

/* Geometry of one chunk's REFCPU bilinear prediction: integer positions and
 * fractions of the luma and chroma windows (vp9_reconstruct.c:94-131,
 * :313-327) and whether each window can be staged with aligned 16-byte
 * copies (inside its plane, rows 16-byte aligned). */
struct McGeo {
    const uint8_t *rp, *ru, *rv;
    int rw, rh, rcs;
    int ix, iy, fx, fy, cix, ciy, cfx, cfy, la, ca;
    bool lfast, cfast;
};

__device__ __forceinline__ bool refcpu_geo(const ReconSmem &s, const BlkS &b, int sbx, int sby,
                                           int lx0, int ly0, int lw, int lh, int cx0, int cy0,
                                           int clw, int clh, McGeo &g)
{
    const int slot = (int)b.ref0 - 1;
    if (slot < 0 || slot >= 8 || !s.jc.ref[slot].plane) return false;
    const cvp9_ref_t &R = s.jc.ref[slot];
    g.rp = R.plane;
    g.rw = R.w;
    g.rh = R.h;
    g.rcs = (g.rw + 1) >> 1;
    g.ru = g.rp + (size_t)g.rw * g.rh;
    g.rv = g.ru + (size_t)g.rcs * ((g.rh + 1) >> 1);
    const int px8 = (sbx + lx0) * 8 + b.mvx, py8 = (sby + ly0) * 8 + b.mvy;
    g.ix = px8 >> 3; g.iy = py8 >> 3; g.fx = px8 & 7; g.fy = py8 & 7;
    const int cmx = b.mvx / 2, cmy = b.mvy / 2;            /* halves toward zero */
    const int cpx8 = ((sbx >> 1) + cx0) * 8 + cmx, cpy8 = ((sby >> 1) + cy0) * 8 + cmy;
    g.cix = cpx8 >> 3; g.ciy = cpy8 >> 3; g.cfx = cpx8 & 7; g.cfy = cpy8 & 7;
    const int crw = g.rw >> 1, crh = g.rh >> 1;            /* floor half of the ref size */
    const bool aligned = !(g.rw & 15) && !(g.rcs & 15) && !((uintptr_t)g.rp & 15) &&
                         !((uintptr_t)g.ru & 15) && !((uintptr_t)g.rv & 15);
    g.lfast = aligned && g.ix >= 0 && g.iy >= 0 && g.ix + lw < g.rw && g.iy + lh < g.rh;
    g.cfast = aligned && g.cix >= 0 && g.ciy >= 0 && g.cix + clw < crw && g.ciy + clh < crh;
    g.la = g.ix & ~15;
    g.ca = g.cix & ~15;
    return true;
}

/* Stage layout of one chunk (608 bytes): luma rows at 32-byte pitch, then U
 * and V rows. Rows needing bytes past the first 16 take a second copy. */
constexpr int kChunkStage = 608;

/* Lane-group variants: 8 lanes per chunk (k = lane & 7). Issue: the group's
 * lanes share the chunk's window copies. Compute: lane k produces luma row k
 * (up to 8 samples) and, for k < 4 / k >= 4, row k&3 of U / V. */
__device__ __forceinline__ void refcpu_issue8(uint8_t *st, const McGeo &g, int lw, int lh,
                                              int clw, int clh, int k)
{
    if (g.lfast) {
        const int two = (g.ix - g.la) + lw >= 16;
        for (int j = k; j < 2 * (lh + 1); j += 8) {
            const int row = j >> 1, half = j & 1;
            if (half == 0 || two)
                cp_async16(st + row * 32 + half * 16, g.rp + (size_t)(g.iy + row) * g.rw + g.la + half * 16);
        }
    }
    if (g.cfast) {
        const int two = (g.cix - g.ca) + clw >= 16;
        const int per = 2 * (clh + 1);
        for (int j = k; j < 2 * per; j += 8) {
            const int pl = j >= per, jj = j - pl * per, row = jj >> 1, half = jj & 1;
            if (half == 0 || two)
                cp_async16(st + 288 + pl * 160 + row * 32 + half * 16,
                           (pl ? g.rv : g.ru) + (size_t)(g.ciy + row) * g.rcs + g.ca + half * 16);
        }
    }
}

/* nine consecutive bytes of a staged row starting at byte `off`, from three
 * aligned 32-bit shared-memory words */
__device__ __forceinline__ void row9(const uint8_t *row, int off, unsigned v[9])
{
    const uint32_t *w = reinterpret_cast<const uint32_t *>(row) + (off >> 2);
    const unsigned sh = 8u * (unsigned)(off & 3);
    const unsigned w0 = w[0], w1 = w[1], w2 = w[2];
    const unsigned lo = __funnelshift_r(w0, w1, sh), mid = __funnelshift_r(w1, w2, sh), hi = w2 >> sh;
#pragma unroll
    for (int i = 0; i < 4; i++) { v[i] = (lo >> (8 * i)) & 0xffu; v[4 + i] = (mid >> (8 * i)) & 0xffu; }
    v[8] = hi & 0xffu;
}

__device__ __forceinline__ void refcpu_compute8(ReconSmem &s, const uint8_t *st, const McGeo &g,
                                                int lx0, int ly0, int lw, int lh,
                                                int cx0, int cy0, int clw, int clh, int k)
{
    if (k < lh) {
        unsigned a[9], b[9];
        if (g.lfast) {
            row9(st + k * 32, g.ix - g.la, a);
            row9(st + (k + 1) * 32, g.ix - g.la, b);
        } else {
            const int y0 = clampi(g.iy + k, 0, g.rh - 1), y1 = clampi(g.iy + k + 1, 0, g.rh - 1);
            const uint8_t *r0 = g.rp + (size_t)y0 * g.rw, *r1 = g.rp + (size_t)y1 * g.rw;
#pragma unroll
            for (int c = 0; c < 9; c++) {
                const int x = clampi(g.ix + c, 0, g.rw - 1);
                a[c] = __ldg(r0 + x);
                b[c] = __ldg(r1 + x);
            }
        }
        const unsigned wx = 8 - g.fx, wy = 8 - g.fy;
        unsigned out[8];
#pragma unroll
        for (int c = 0; c < 8; c++) {
            const unsigned t = (a[c] * wx + a[c + 1] * g.fx + 4) >> 3;
            const unsigned u = (b[c] * wx + b[c + 1] * g.fx + 4) >> 3;
            out[c] = (t * wy + u * g.fy + 4) >> 3;
        }
        uint8_t *d = &TY(s, lx0, ly0 + k);
        if (lw == 8) {
            uint32_t *d4 = reinterpret_cast<uint32_t *>(d);
            d4[0] = out[0] | out[1] << 8 | out[2] << 16 | out[3] << 24;
            d4[1] = out[4] | out[5] << 8 | out[6] << 16 | out[7] << 24;
        } else {
#pragma unroll
            for (int c = 0; c < 8; c++) if (c < lw) d[c] = (uint8_t)out[c];
        }
    }
    {
        const int p = 1 + (k >> 2), r = k & 3;
        if (r < clh) {
            unsigned a[5], b[5];
            if (g.cfast) {
                const uint8_t *s0 = st + 288 + (p - 1) * 160 + r * 32 + (g.cix - g.ca), *s1 = s0 + 32;
#pragma unroll
                for (int c = 0; c < 5; c++) { a[c] = s0[c]; b[c] = s1[c]; }
            } else {
                const int crw = g.rw >> 1, crh = g.rh >> 1;
                const int xm = crw > 0 ? crw - 1 : 0, ym = crh > 0 ? crh - 1 : 0;
                const uint8_t *pl = p == 1 ? g.ru : g.rv;
                const uint8_t *r0 = pl + (size_t)clampi(g.ciy + r, 0, ym) * g.rcs;
                const uint8_t *r1 = pl + (size_t)clampi(g.ciy + r + 1, 0, ym) * g.rcs;
#pragma unroll
                for (int c = 0; c < 5; c++) {
                    const int x = clampi(g.cix + c, 0, xm);
                    a[c] = __ldg(r0 + x);
                    b[c] = __ldg(r1 + x);
                }
            }
            uint8_t *d = &TC(s, p, cx0, cy0 + r);
#pragma unroll
            for (int c = 0; c < 4; c++) {
                if (c >= clw) break;
                const unsigned t = (a[c] * (8 - g.cfx) + a[c + 1] * g.cfx + 4) >> 3;
                const unsigned u = (b[c] * (8 - g.cfx) + b[c + 1] * g.cfx + 4) >> 3;
                d[c] = (uint8_t)((t * (8 - g.cfy) + u * g.cfy + 4) >> 3);
            }
        }
    }
}

/* Lane-group flat fill (missing reference): lane k fills luma row k and one
 * chroma row, like refcpu_compute8. */
__device__ __forceinline__ void refcpu_fill8(ReconSmem &s, int v, int lx0, int ly0, int lw, int lh,
                                             int cx0, int cy0, int clw, int clh, int k)
{
    if (k < lh)
        for (int c = 0; c < lw; c++) TY(s, lx0 + c, ly0 + k) = (uint8_t)v;
    const int p = 1 + (k >> 2), r = k & 3;
    if (r < clh)
        for (int c = 0; c < clw; c++) TC(s, p, cx0 + c, cy0 + r) = (uint8_t)v;
}

/* A reference that is absent predicts as a flat value (127 REFCPU, 128 SPEC). */
__device__ __forceinline__ void fill_chunk(ReconSmem &s, int v, int lx0, int ly0, int lw, int lh,
                                          int cx0, int cy0, int clw, int clh, int lane)
{
    for (int idx = lane; idx < 64; idx += 32) {
        int r = idx >> 3, c = idx & 7;
        if (r < lh && c < lw) TY(s, lx0 + c, ly0 + r) = (uint8_t)v;
    }
    int p = 1 + (lane >> 4), r = (lane >> 2) & 3, c = lane & 3;
    if (r < clh && c < clw) TC(s, p, cx0 + c, cy0 + r) = (uint8_t)v;
}

/* SPEC inter prediction of one chunk from one reference: 8-tap on luma
 * (even phases of the 1/8-pel MV) and chroma (1/16 chroma pel), every fetch
 * clamped into the reference plane, horizontal pass rounded and clipped to 8
 * bits before the vertical pass (vp9_mc.comp.glsl:61-110). F: the filter
 * (the regular one under SPEC). avg: round-average into the tile (the
 * second prediction of a FULL compound block). */
/* One 8-tap output of a staged row (4-byte aligned in shared memory) at
 * column c: samples c..c+7 as two words, two dp4a (tap8). The same value as
 * the scalar sum: clamp((sum + 64) >> 7, 0, 255). */
__device__ __forceinline__ uint32_t htap8(const uint8_t *row, int c, const uint32_t *pk, int phase)
{
    const uint32_t *w = reinterpret_cast<const uint32_t *>(row) + (c >> 2);
    const unsigned sh = 8u * (unsigned)(c & 3);
    const uint32_t w0 = w[0], w1 = w[1], w2 = w[2];
    return tap8(pk[0], pk[1], phase, __funnelshift_r(w0, w1, sh), __funnelshift_r(w1, w2, sh));
}

__device__ void spec_inter_pass(ReconSmem &s, const cvp9_ref_t &R, int mvx, int mvy, const int (*F)[8],
                                const uint32_t (*P)[2], bool avg,
                                int sbx, int sby, int lx0, int ly0, int lw, int lh,
                                int cx0, int cy0, int clw, int clh, int warp, int lane)
{
    const uint8_t *rp = R.plane;
    const int rw = R.w, rh = R.h;
    const int rcs = (rw + 1) >> 1;
    const uint8_t *ru = rp + (size_t)rw * rh;
    const uint8_t *rv = ru + (size_t)rcs * ((rh + 1) >> 1);
    uint8_t *st = s.stage[warp];
        /* luma: (lw+7) x (lh+7) window at pitch 16; H pass into 15 x 8 */
        int bx = sbx + lx0 + (mvx >> 3), by = sby + ly0 + (mvy >> 3);
        int fx = (mvx & 7) << 1, fy = (mvy & 7) << 1;
        int gcx = (sbx >> 1) + cx0, gcy = (sby >> 1) + cy0;
        int cbx = gcx + (mvx >> 4), cby = gcy + (mvy >> 4);
        int cfx = mvx & 15, cfy = mvy & 15;
        int cw2 = (rw + 1) >> 1, ch2 = (rh + 1) >> 1;
        uint8_t *sy_ = st;              /* 15 x 16 */
        uint8_t *hy = st + 240;         /* 15 x 8  */
        uint8_t *su = st + 360;         /* 11 x 12 */
        uint8_t *sv = st + 492;         /* 11 x 12 */
        uint8_t *hu = st + 624;         /* 11 x 4  */
        uint8_t *hv = st + 668;         /* 11 x 4  */
        {
            /* all three windows' reads in flight at once */
            WinRows<8> wl;
            WinRows<6> wu, wv;
            wl.load(rp, rw, rw, rh, bx - 3, by - 3, lw + 7, lh + 7, lane);
            wu.load(ru, rcs, cw2, ch2, cbx - 3, cby - 3, clw + 7, clh + 7, lane);
            wv.load(rv, rcs, cw2, ch2, cbx - 3, cby - 3, clw + 7, clh + 7, lane);
            wl.store(sy_, 16, lw + 7, lh + 7, lane);
            wu.store(su, 12, clw + 7, clh + 7, lane);
            wv.store(sv, 12, clw + 7, clh + 7, lane);
        }
        __syncwarp();
        /* horizontal pass (rounded, clipped to 8 bits) */
        for (int i = lane; i < (lh + 7) * lw; i += 32) {
            int r = lw == 8 ? i >> 3 : i / lw, c = i - r * lw;
            hy[r * 8 + c] = (uint8_t)htap8(sy_ + r * 16, c, P[fx], fx);
        }
        for (int i = lane; i < 2 * (clh + 7) * clw; i += 32) {
            int pl = i >= (clh + 7) * clw;
            int j = pl ? i - (clh + 7) * clw : i;
            int r = clw == 4 ? j >> 2 : j / clw, c = j - r * clw;
            const uint8_t *src = pl ? sv : su;
            (pl ? hv : hu)[r * 4 + c] = (uint8_t)htap8(src + r * 12, c, P[cfx], cfx);
        }
        __syncwarp();
        for (int idx = lane; idx < 64; idx += 32) {
            int r = idx >> 3, c = idx & 7;
            if (r >= lh || c >= lw) continue;
            int v;
            if (fx == 0 && fy == 0) {
                v = sy_[(r + 3) * 16 + c + 3];
            } else {
                int acc = 0;
#pragma unroll
                for (int t = 0; t < 8; t++) acc += F[fy][t] * hy[(r + t) * 8 + c];
                v = clampi((acc + 64) >> 7, 0, 255);
            }
            uint8_t &d = TY(s, lx0 + c, ly0 + r);
            d = (uint8_t)(avg ? ((int)d + v + 1) >> 1 : v);
        }
        {
            int p = 1 + (lane >> 4), r = (lane >> 2) & 3, c = lane & 3;
            if (r < clh && c < clw) {
                int v;
                if (cfx == 0 && cfy == 0) {
                    v = (p == 1 ? su : sv)[(r + 3) * 12 + c + 3];
                } else {
                    const uint8_t *h = p == 1 ? hu : hv;
                    int acc = 0;
#pragma unroll
                    for (int t = 0; t < 8; t++) acc += F[cfy][t] * h[(r + t) * 4 + c];
                    v = clampi((acc + 64) >> 7, 0, 255);
                }
                uint8_t &d = TC(s, p, cx0 + c, cy0 + r);
                d = (uint8_t)(avg ? ((int)d + v + 1) >> 1 : v);
            }
        }
        __syncwarp();
}

/* SPEC inter prediction of one chunk; FULL also takes the header's filter
 * and averages in a second reference's prediction (compound blocks). A
 * missing first reference predicts flat 128; a missing second one leaves
 * the single prediction. */
__device__ void spec_inter_chunk(ReconSmem &s, const BlkS &b, int sbx, int sby,
                                 int lx0, int ly0, int lw, int lh,
                                 int cx0, int cy0, int clw, int clh, int warp, int lane)
{
    const cvp9_job_t &job = s.jc;
    const cvp9_ref_t &R = job.ref[job.ref_slot_of[clampi((int)b.ref0 - 1, 0, 2)] & 7];
    if (!R.plane) { fill_chunk(s, 128, lx0, ly0, lw, lh, cx0, cy0, clw, clh, lane); return; }
    const int (*F)[8] = job.full ? c_subpel4[job.interp_filter & 3] : c_subpel;
    const uint32_t (*P)[2] = job.full ? c_subpel4_pk[job.interp_filter & 3] : c_subpel_pk;
    spec_inter_pass(s, R, b.mvx, b.mvy, F, P, false, sbx, sby, lx0, ly0, lw, lh, cx0, cy0, clw, clh, warp, lane);
    if (b.ref1) {
        const cvp9_ref_t &R1 = job.ref[job.ref_slot_of[clampi((int)b.ref1 - 1, 0, 2)] & 7];
        if (R1.plane)
            spec_inter_pass(s, R1, b.mv1x, b.mv1y, F, P, true, sbx, sby, lx0, ly0, lw, lh, cx0, cy0, clw, clh,
                            warp, lane);
    }
}

/* ── Residual: one item = one TX column (pass 1) or one TX row (pass 2) ── */

struct TxRef {
    int plane, txl, n;
    int px0, py0;      /* TX origin in the SB tile of its plane */
    uint64_t coeff;    /* first coefficient of the TX            */
    int mask_idx;
};

__device__ __forceinline__ TxRef locate_item(const BlkS &b, int item, int *lane_idx)
{
    TxRef t;
    uint64_t off = b.coeff;
    int p = 0;
    for (; p < 2; p++) {
        int cnt = b.pnt[p] * (4 << b.ptxl[p]);
        if (item < cnt) break;
        item -= cnt;
        off += (uint64_t)b.pnt[p] * (uint64_t)(16 << (2 * b.ptxl[p]));
    }
    int txl = b.ptxl[p], n = 4 << txl;
    int tx = item >> (2 + txl);
    *lane_idx = item & (n - 1);
    int nx = b.pnx[p];
    int tx_y = nx == 1 ? tx : div_small(tx, nx), tx_x = tx - tx_y * nx;
    t.plane = p;
    t.txl = txl;
    t.n = n;
    int ox = p ? (b.x >> 1) : b.x, oy = p ? (b.y >> 1) : b.y;
    t.px0 = ox + tx_x * n;
    t.py0 = oy + tx_y * n;
    t.coeff = off + (uint64_t)tx * (uint64_t)(n * n);
    t.mask_idx = p == 0 ? (t.py0 >> 2) * 16 + (t.px0 >> 2)
                        : 256 + (p - 1) * 64 + (t.py0 >> 2) * 8 + (t.px0 >> 2);
    return t;
}

/* REFCPU pass 1: T[:, j] = M^T X[:, j] over the nonzero X[k][j], k ascending
 * (vp9_reconstruct.c:31-40). Skipped zero terms add +-0 to a sum that is
 * never -0, so the result is bit-identical to the full sum. */
template <int N>
__device__ __forceinline__ void refcpu_col(ReconSmem &s, const int16_t *X, int j,
                                           int px0, int py0, int mask_idx, const double *M)
{
    unsigned nzm = 0;
#pragma unroll
    for (int k = 0; k < N; k++) nzm |= (X[k * N + j] != 0 ? 1u : 0u) << k;
    if (!nzm) return;
    double acc[N];
#pragma unroll
    for (int i = 0; i < N; i++) acc[i] = 0.0;
    while (nzm) {
        const int k = __ffs(nzm) - 1;
        nzm &= nzm - 1;
        const double xd = (double)X[k * N + j];
#pragma unroll
        for (int i = 0; i < N; i++) acc[i] = __dadd_rn(acc[i], __dmul_rn(M[k * N + i], xd));
    }
#pragma unroll
    for (int i = 0; i < N; i++) s.temp.d[(py0 + i) * kTempPitch + px0 + j] = acc[i];
    atomicOr(&s.txmask[mask_idx], 1u << j);
}

/* REFCPU pass 2: O[i, :] = T[i, :] M over the nonzero columns, round half
 * away from zero, saturate to int16, add and clamp (:42-59, :351-360). */
template <int N>
__device__ __forceinline__ void refcpu_row(ReconSmem &s, int i, int px0, int py0, unsigned mask,
                                           const double *M)
{
    double acc[N];
#pragma unroll
    for (int j = 0; j < N; j++) acc[j] = 0.0;
    while (mask) {
        const int k = __ffs(mask) - 1;
        mask &= mask - 1;
        double t = s.temp.d[(py0 + i) * kTempPitch + px0 + k];
#pragma unroll
        for (int j = 0; j < N; j++) acc[j] = __dadd_rn(acc[j], __dmul_rn(t, M[k * N + j]));
    }
#pragma unroll
    for (int j = 0; j < N; j++) {
        double v = acc[j];
        int r = __double2int_rz(__dadd_rn(v, v >= 0.0 ? 0.5 : -0.5));
        r = clampi(r, -32768, 32767);
        uint8_t &px = TY(s, px0 + j, py0 + i);
        px = (uint8_t)clampi((int)px + r, 0, 255);
    }
}

/* REFCPU pass 2 without the add: row i's rounded, saturated residual
 * (the same operations as refcpu_row) into res, the SB's 64x64 luma grid,
 * for the level that predicts the TX's block to add. */
template <int N>
__device__ __forceinline__ void refcpu_row_res(ReconSmem &s, int i, int px0, int py0, unsigned mask,
                                               const double *M, int16_t *res)
{
    double acc[N];
#pragma unroll
    for (int j = 0; j < N; j++) acc[j] = 0.0;
    while (mask) {
        const int k = __ffs(mask) - 1;
        mask &= mask - 1;
        double t = s.temp.d[(py0 + i) * kTempPitch + px0 + k];
#pragma unroll
        for (int j = 0; j < N; j++) acc[j] = __dadd_rn(acc[j], __dmul_rn(t, M[k * N + j]));
    }
#pragma unroll
    for (int j = 0; j < N; j++) {
        double v = acc[j];
        int r = __double2int_rz(__dadd_rn(v, v >= 0.0 ? 0.5 : -0.5));
        res[(py0 + i) * 64 + px0 + j] = (int16_t)clampi(r, -32768, 32767);
    }
}

/* The add and clamp of refcpu_row, from res. */
template <int N>
__device__ __forceinline__ void refcpu_add_res(ReconSmem &s, int i, int px0, int py0, const int16_t *res)
{
#pragma unroll
    for (int j = 0; j < N; j++) {
        uint8_t &px = TY(s, px0 + j, py0 + i);
        px = (uint8_t)clampi((int)px + res[(py0 + i) * 64 + px0 + j], 0, 255);
    }
}

template <class T>
__device__ __forceinline__ void idct_n(T *x, int n)
{
    if (n == 4) idct4(x);
    else if (n == 8) idct8(x);
    else if (n == 16) idct16(x);
    else idct32(x);
}

__device__ __forceinline__ int32_t *spec_temp(ReconSmem &s, int plane, int x, int y)
{
    if (plane == 0) return &s.temp.i[y * 64 + x];
    return &s.temp.i[4096 + (plane - 1) * 1024 + y * 32 + x];
}

/* SPEC pass 1: dequantise column j (DC step at [0][0] only) and run the
 * 1-D transform down the column (vp9_idct.comp.glsl:666-679). */
template <int N>
__device__ __forceinline__ void spec_col(ReconSmem &s, const int16_t *X, int j,
                                         const TxRef &t, int q_dc, int q_ac)
{
    wi v[N];
    bool any = false;
#pragma unroll
    for (int k = 0; k < N; k++) {
        int c = X[k * N + j];
        any |= c != 0;
        v[k] = wi(c) * ((k == 0 && j == 0) ? q_dc : q_ac);
    }
    if (any) {
        idct_n(v, N);
        atomicOr(&s.txmask[t.mask_idx], 1u);
    }
#pragma unroll
    for (int k = 0; k < N; k++) *spec_temp(s, t.plane, t.px0 + j, t.py0 + k) = any ? v[k].v : 0;
}

/* SPEC pass 2: row transform, final rounding shift 4/5/6/6, add and clamp;
 * samples outside the frame are left alone (tile write-back clips them). */
template <int N>
__device__ __forceinline__ void spec_row(ReconSmem &s, int i, const TxRef &t)
{
    wi v[N];
#pragma unroll
    for (int k = 0; k < N; k++) v[k] = wi(*spec_temp(s, t.plane, t.px0 + k, t.py0 + i));
    idct_n(v, N);
    const int sh = N == 4 ? 4 : (N == 8 ? 5 : 6);
#pragma unroll
    for (int j = 0; j < N; j++) {
        int r = ((int)((unsigned)v[j].v + (1u << (sh - 1)))) >> sh;
        uint8_t &px = t.plane == 0 ? TY(s, t.px0 + j, t.py0 + i) : TC(s, t.plane, t.px0 + j, t.py0 + i);
        px = (uint8_t)clampi((int)px + r, 0, 255);
    }
}

/* ── FULL profile: ADST and WHT, rows-then-columns residual, per-TX intra ── */

/* sin(k*pi/9) * 2/3 * sqrt(2) in Q14, the 4-point ADST multipliers */
enum : int { KS1 = 5283, KS2 = 9929, KS3 = 13377, KS4 = 15212 };

/* 1-D inverse ADSTs in place, 32-bit wrap and Q14 rounding as the DCTs. */
template <class T>
__device__ __forceinline__ void iadst4(T *x)
{
    T a = x[0] * KS1 + x[2] * KS4 + x[3] * KS2;
    T b = x[0] * KS2 - x[2] * KS1 - x[3] * KS4;
    T c = (x[0] - x[2] + x[3]) * KS3;
    T d = x[1] * KS3;
    x[0] = RS(a + d); x[1] = RS(b + d); x[2] = RS(c); x[3] = RS(a + b - d);
}

template <class T>
__device__ __forceinline__ void rot(T x, T y, int ca, int cb, T &o0, T &o1)
{
    o0 = x * ca + y * cb;
    o1 = x * cb - y * ca;
}

template <class T>
__device__ __forceinline__ void iadst8(T *in)
{
    T x0 = in[7], x1 = in[0], x2 = in[5], x3 = in[2], x4 = in[3], x5 = in[4], x6 = in[1], x7 = in[6];
    T s0, s1, s2, s3, s4, s5, s6, s7;
    rot(x0, x1, K2, K30, s0, s1);
    rot(x2, x3, K10, K22, s2, s3);
    rot(x4, x5, K18, K14, s4, s5);
    rot(x6, x7, K26, K6, s6, s7);
    x0 = RS(s0 + s4); x1 = RS(s1 + s5); x2 = RS(s2 + s6); x3 = RS(s3 + s7);
    x4 = RS(s0 - s4); x5 = RS(s1 - s5); x6 = RS(s2 - s6); x7 = RS(s3 - s7);
    s4 = x4 * K8 + x5 * K24;
    s5 = x4 * K24 - x5 * K8;
    s6 = x7 * K8 - x6 * K24;
    s7 = x6 * K8 + x7 * K24;
    s0 = x0 + x2; s1 = x1 + x3; s2 = x0 - x2; s3 = x1 - x3;
    x4 = RS(s4 + s6); x5 = RS(s5 + s7); x6 = RS(s4 - s6); x7 = RS(s5 - s7);
    x2 = RS((s2 + s3) * K16);
    x3 = RS((s2 - s3) * K16);
    T y6 = RS((x6 + x7) * K16), y7 = RS((x6 - x7) * K16);
    in[0] = s0; in[1] = -x4; in[2] = y6; in[3] = -x2;
    in[4] = x3; in[5] = -y7; in[6] = x5; in[7] = -s1;
}

template <class T>
__device__ __forceinline__ void iadst16(T *in)
{
    T x[16], s[16];
    x[0] = in[15]; x[1] = in[0]; x[2] = in[13]; x[3] = in[2]; x[4] = in[11]; x[5] = in[4];
    x[6] = in[9]; x[7] = in[6]; x[8] = in[7]; x[9] = in[8]; x[10] = in[5]; x[11] = in[10];
    x[12] = in[3]; x[13] = in[12]; x[14] = in[1]; x[15] = in[14];
    rot(x[0], x[1], K1, K31, s[0], s[1]);
    rot(x[2], x[3], K5, K27, s[2], s[3]);
    rot(x[4], x[5], K9, K23, s[4], s[5]);
    rot(x[6], x[7], K13, K19, s[6], s[7]);
    rot(x[8], x[9], K17, K15, s[8], s[9]);
    rot(x[10], x[11], K21, K11, s[10], s[11]);
    rot(x[12], x[13], K25, K7, s[12], s[13]);
    rot(x[14], x[15], K29, K3, s[14], s[15]);
#pragma unroll
    for (int k = 0; k < 8; k++) { x[k] = RS(s[k] + s[k + 8]); x[k + 8] = RS(s[k] - s[k + 8]); }
#pragma unroll
    for (int k = 0; k < 8; k++) s[k] = x[k];
    s[8] = x[8] * K4 + x[9] * K28;
    s[9] = x[8] * K28 - x[9] * K4;
    s[10] = x[10] * K20 + x[11] * K12;
    s[11] = x[10] * K12 - x[11] * K20;
    s[12] = x[13] * K4 - x[12] * K28;
    s[13] = x[12] * K4 + x[13] * K28;
    s[14] = x[15] * K20 - x[14] * K12;
    s[15] = x[14] * K20 + x[15] * K12;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        x[k] = s[k] + s[k + 4];
        x[k + 4] = s[k] - s[k + 4];
        x[k + 8] = RS(s[k + 8] + s[k + 12]);
        x[k + 12] = RS(s[k + 8] - s[k + 12]);
    }
#pragma unroll
    for (int g = 0; g < 16; g += 8) {
        s[g + 0] = x[g + 0]; s[g + 1] = x[g + 1]; s[g + 2] = x[g + 2]; s[g + 3] = x[g + 3];
        s[g + 4] = x[g + 4] * K8 + x[g + 5] * K24;
        s[g + 5] = x[g + 4] * K24 - x[g + 5] * K8;
        s[g + 6] = x[g + 7] * K8 - x[g + 6] * K24;
        s[g + 7] = x[g + 6] * K8 + x[g + 7] * K24;
        x[g + 0] = s[g + 0] + s[g + 2];
        x[g + 1] = s[g + 1] + s[g + 3];
        x[g + 2] = s[g + 0] - s[g + 2];
        x[g + 3] = s[g + 1] - s[g + 3];
        x[g + 4] = RS(s[g + 4] + s[g + 6]);
        x[g + 5] = RS(s[g + 5] + s[g + 7]);
        x[g + 6] = RS(s[g + 4] - s[g + 6]);
        x[g + 7] = RS(s[g + 5] - s[g + 7]);
    }
    T t2 = RS(-((x[2] + x[3]) * K16)), t3 = RS((x[2] - x[3]) * K16);
    T t6 = RS((x[6] + x[7]) * K16), t7 = RS((x[7] - x[6]) * K16);
    T t10 = RS((x[10] + x[11]) * K16), t11 = RS((x[11] - x[10]) * K16);
    T t14 = RS(-((x[14] + x[15]) * K16)), t15 = RS((x[14] - x[15]) * K16);
    in[0] = x[0];  in[1] = -x[8];  in[2] = x[12];  in[3] = -x[4];
    in[4] = t6;    in[5] = t14;    in[6] = t10;    in[7] = t2;
    in[8] = t3;    in[9] = t11;    in[10] = t15;   in[11] = t7;
    in[12] = x[5]; in[13] = -x[13]; in[14] = x[9]; in[15] = -x[1];
}

/* 4-point inverse Walsh-Hadamard (lossless frames); the row pass first
 * undoes the quantiser step 4 with a shift. */
template <class T>
__device__ __forceinline__ void iwht4(T *x, bool rows)
{
    T a = x[0], c = x[1], d = x[2], b = x[3];
    if (rows) { a = shr(a, 2); c = shr(c, 2); d = shr(d, 2); b = shr(b, 2); }
    a = a + c; d = d - b;
    T e = shr(a - d, 1);
    b = e - b; c = e - c;
    a = a - b; d = d + c;
    x[0] = a; x[1] = b; x[2] = c; x[3] = d;
}

template <int N, class T>
__device__ __forceinline__ void itx1(T *v, bool adst)
{
    if (N == 4 && adst) iadst4(v);
    else if (N == 8 && adst) iadst8(v);
    else if (N == 16 && adst) iadst16(v);
    else idct_n(v, N);
}

/* FULL pass 1 on TX row i: dequantise (the plane's steps, DC at [0][0];
 * 32x32 values halved toward zero) and transform along the row (DCT, or
 * ADST when row_adst; WHT when lossless) into the temp rows. Returns
 * whether the row had a nonzero coefficient. */
template <int N>
__device__ __forceinline__ bool full_row(ReconSmem &s, const int16_t *X, int i, int plane, int px0, int py0,
                                         int qdc, int qac, bool lossless, bool row_adst)
{
    wi v[N];
    bool any = false;
#pragma unroll
    for (int k = 0; k < N; k++) {
        int c = X[i * N + k];
        any |= c != 0;
        int d = c * ((i == 0 && k == 0) ? qdc : qac);
        v[k] = wi(N == 32 ? d / 2 : d);
    }
    if (any) {
        if (N == 4 && lossless) iwht4(v, true);
        else itx1<N>(v, row_adst);
    }
#pragma unroll
    for (int k = 0; k < N; k++) *spec_temp(s, plane, px0 + k, py0 + i) = any ? v[k].v : 0;
    return any;
}

/* FULL pass 2 on TX column j: transform down the column, final rounding
 * shift 4/5/6/6 (none after the WHT), add and clamp into the tile. */
template <int N>
__device__ __forceinline__ void full_col(ReconSmem &s, int j, int plane, int px0, int py0, bool lossless,
                                         bool col_adst)
{
    wi v[N];
#pragma unroll
    for (int k = 0; k < N; k++) v[k] = wi(*spec_temp(s, plane, px0 + j, py0 + k));
    const bool wht = N == 4 && lossless;
    if (wht) iwht4(v, false);
    else itx1<N>(v, col_adst);
    const int sh = N == 4 ? 4 : (N == 8 ? 5 : 6);
#pragma unroll
    for (int k = 0; k < N; k++) {
        int r = wht ? v[k].v : ((int)((unsigned)v[k].v + (1u << (sh - 1)))) >> sh;
        uint8_t &px = plane == 0 ? TY(s, px0 + j, py0 + k) : TC(s, plane, px0 + j, py0 + k);
        px = (uint8_t)clampi((int)px + r, 0, 255);
    }
}

/* First MI column of the tile column holding mi_col (VP9 tile offsets). */
__device__ __forceinline__ int full_tile_start(int mi_col, int mi_cols, int log2_tile_cols)
{
    const int sb_cols = (mi_cols + 7) >> 3;
    int start = 0;
    for (int t = 1; t < (1 << log2_tile_cols); t++) {
        int o = ((t * sb_cols) >> log2_tile_cols) << 3;
        if (o > mi_cols) o = mi_cols;
        if (o <= mi_col) start = o;
    }
    return start;
}

__device__ __forceinline__ uint8_t &TP(ReconSmem &s, int p, int x, int y)
{
    return p == 0 ? TY(s, x, y) : TC(s, p, x, y);
}

#define FAVG2(a, b) (((a) + (b) + 1) >> 1)
#define FAVG3(a, b, c) (((a) + 2 * (b) + (c) + 2) >> 2)

/* One sample of a VP9 intra predictor from the TX's edges: above[-1..2n-1]
 * (above[-1] the corner), left[0..n-1]; MAXV: the largest sample value (TM
 * clips to it). */
template <int MAXV = 255, class E>
__device__ __forceinline__ int full_pred(int mode, int r, int c, int n, const E *above, const E *left, int dc)
{
    switch (mode) {
    case 1: return above[c];
    case 2: return left[r];
    case 3: {
        const int k = r + c;
        return k + 2 < 2 * n ? FAVG3(above[k], above[k + 1], above[k + 2]) : above[2 * n - 1];
    }
    case 4: {
        const int t = c - r;
        auto e = [&](int u) -> int { return u >= 0 ? above[u] : (u == -1 ? above[-1] : left[-u - 2]); };
        return FAVG3(e(t - 2), e(t - 1), e(t));
    }
    case 5: {
        const int k = min(r >> 1, c), rr = r - 2 * k, cc = c - k;
        if (rr == 0) return FAVG2(above[cc - 1], above[cc]);
        if (rr == 1) return cc == 0 ? FAVG3(left[0], above[-1], above[0]) : FAVG3(above[cc - 2], above[cc - 1], above[cc]);
        return rr == 2 ? FAVG3(above[-1], left[0], left[1]) : FAVG3(left[rr - 3], left[rr - 2], left[rr - 1]);
    }
    case 6: {
        const int k = min(r, c >> 1), rr = r - k, cc = c - 2 * k;
        if (cc == 0) return rr == 0 ? FAVG2(above[-1], left[0]) : FAVG2(left[rr - 1], left[rr]);
        if (cc == 1) return rr == 0 ? FAVG3(left[0], above[-1], above[0])
                          : rr == 1 ? FAVG3(above[-1], left[0], left[1]) : FAVG3(left[rr - 2], left[rr - 1], left[rr]);
        return FAVG3(above[cc - 3], above[cc - 2], above[cc - 1]);
    }
    case 7: {
        const int k = r + (c >> 1);
        auto L = [&](int i) -> int { return left[i < n ? i : n - 1]; };
        return (c & 1) ? FAVG3(L(k), L(k + 1), L(k + 2)) : FAVG2(L(k), L(k + 1));
    }
    case 8: {
        const int k = (r >> 1) + c;
        return (r & 1) ? FAVG3(above[k], above[k + 1], above[k + 2]) : FAVG2(above[k], above[k + 1]);
    }
    case 9: return clampi((int)left[r] + (int)above[c] - (int)above[-1], 0, MAXV);
    default: return dc;
    }
}

/* FULL intra prediction of one n x n TX at tile position (lx, ly) of plane
 * p, plane position (X0, Y0) in a plane of pw x ph samples: VP9 edge rules
 * (127 above / 129 left when unavailable, above-right only for a 4x4 TX
 * with have_right, samples past the plane's right or bottom edge repeating
 * the last one inside). One warp; `edge` is the warp's scratch. */
__device__ void full_intra_tx(ReconSmem &s, int p, int lx, int ly, int X0, int Y0, int pw, int ph, int n,
                              int mode, bool have_top, bool have_left, bool have_right, uint8_t *edge, int lane)
{
    uint8_t *above = edge + 1, *left = edge + 80;
    if (have_top) {
        const int want = n + ((n == 4 && have_right) ? 4 : 0);
        const int cnt = min(want, pw - X0);
        for (int i = lane; i < 2 * n; i += 32) above[i] = TP(s, p, lx + (i < cnt ? i : cnt - 1), ly - 1);
        if (lane == 0) above[-1] = have_left ? TP(s, p, lx - 1, ly - 1) : (uint8_t)129;
    } else {
        for (int i = lane; i < 2 * n + 1; i += 32) edge[i] = 127;
    }
    for (int i = lane; i < n; i += 32) left[i] = have_left ? TP(s, p, lx - 1, ly + min(i, ph - 1 - Y0)) : (uint8_t)129;
    __syncwarp();
    int dc = 128;
    if (mode == 0) {
        const unsigned sa = __reduce_add_sync(0xffffffffu, lane < n ? (unsigned)above[lane] : 0u);
        const unsigned sl = __reduce_add_sync(0xffffffffu, lane < n ? (unsigned)left[lane] : 0u);
        if (have_top && have_left) dc = (int)((sa + sl + (unsigned)n) / (unsigned)(2 * n));
        else if (have_top) dc = (int)((sa + (unsigned)n / 2) / (unsigned)n);
        else if (have_left) dc = (int)((sl + (unsigned)n / 2) / (unsigned)n);
    }
    const int lg = n == 4 ? 2 : n == 8 ? 3 : n == 16 ? 4 : 5;
    for (int idx = lane; idx < n * n; idx += 32) {
        const int r = idx >> lg, c = idx & (n - 1);
        TP(s, p, lx + c, ly + r) = (uint8_t)full_pred(mode, r, c, n, above, left, dc);
    }
    __syncwarp();
}

/* FULL residual of one n x n TX by one warp (lane = row, then column). */
template <int N>
__device__ void full_tx_warp(ReconSmem &s, const int16_t *X, int p, int lx, int ly, int qdc, int qac,
                             bool lossless, int tx_type, int lane)
{
    bool any = false;
    if (lane < N) any = full_row<N>(s, X, lane, p, lx, ly, qdc, qac, lossless, tx_type == 2 || tx_type == 3);
    any = __any_sync(0xffffffffu, any);
    __syncwarp();
    if (any && lane < N) full_col<N>(s, lane, p, lx, ly, lossless, tx_type == 1 || tx_type == 3);
    __syncwarp();
}

/* FULL intra block, one warp: for each plane, each TX in raster order is
 * predicted from the reconstructed samples around it and gets its residual
 * before the next TX is predicted (the VP9 decoding order). */
__device__ void full_intra_block(ReconSmem &s, const BlkS &b, int sbx, int sby, bool staged, unsigned c_base,
                                 int warp, int lane)
{
    const cvp9_job_t &job = s.jc;
    const int gx = sbx + b.x, gy = sby + b.y;
    const int mi_col = gx >> 3, mi_row = gy >> 3;
    const bool left_ok = mi_col > full_tile_start(mi_col, job.mi_cols, job.log2_tile_cols);
    uint8_t *edge = s.stage[warp];
    uint64_t off = b.coeff;
    for (int p = 0; p < 3; p++) {
        int txl, nx, ny, pbw;
        plane_layout(b, job, gx, gy, p, txl, nx, ny, pbw);
        const int n = 4 << txl;
        const int mode = p ? (b.uvmode > 9 ? 0 : b.uvmode) : (b.ymode > 9 ? 0 : b.ymode);
        const int tx_type = (p == 0 && !job.lossless && txl < 3 && b.ymode < 10) ? c_tx_type[b.ymode] : 0;
        const int pw = p ? job.CW : job.W, ph = p ? job.CH : job.H;
        const int ox = p ? (b.x >> 1) : b.x, oy = p ? (b.y >> 1) : b.y;
        const int gox = p ? (gx >> 1) : gx, goy = p ? (gy >> 1) : gy;
        const int qdc = p ? job.q_dc_uv : job.q_dc, qac = p ? job.q_ac_uv : job.q_ac;
        for (int ty = 0; ty < ny; ty++)
            for (int tx = 0; tx < nx; tx++) {
                const int lx = ox + tx * n, ly = oy + ty * n;
                full_intra_tx(s, p, lx, ly, gox + tx * n, goy + ty * n, pw, ph, n, mode,
                              ty > 0 || mi_row > 0, tx > 0 || left_ok, (tx + 1) * n < pbw, edge, lane);
                if (b.flags & 2) continue;
                const uint64_t co = off + (uint64_t)(ty * nx + tx) * (uint64_t)(n * n);
                if (co + (uint64_t)(n * n) > (uint64_t)job.num_coeffs) continue;
                const int16_t *X = staged ? s.coef + (co - c_base) : job.coeffs + co;
                switch (txl) {
                case 0: full_tx_warp<4>(s, X, p, lx, ly, qdc, qac, job.lossless, tx_type, lane); break;
                case 1: full_tx_warp<8>(s, X, p, lx, ly, qdc, qac, job.lossless, tx_type, lane); break;
                case 2: full_tx_warp<16>(s, X, p, lx, ly, qdc, qac, job.lossless, tx_type, lane); break;
                default: full_tx_warp<32>(s, X, p, lx, ly, qdc, qac, job.lossless, 0, lane); break;
                }
            }
        if (!(b.flags & 2)) off += (uint64_t)(nx * ny) * (uint64_t)(n * n);
    }
}

/* The two transform passes of one residual item (a TX column, then a TX
 * row; FULL: a row, then a column) of block b, item index `item` inside the
 * block. Pass 1 reads the coefficients (staged span or global), pass 2 adds
 * the residual into the tile. */
template <int A>
__device__ __forceinline__ void item_pass1(ReconSmem &s, const BlkS &b, int item, bool staged, unsigned c_base)
{
    const cvp9_job_t &job = s.jc;
    int j;
    TxRef t = locate_item(b, item, &j);
    if (t.coeff + (uint64_t)(t.n * t.n) > (uint64_t)job.num_coeffs) return;
    const int16_t *X = staged ? s.coef + (t.coeff - c_base) : job.coeffs + t.coeff;
    if (A == CVP9_ARITH_REFCPU) {
        const double *M = dct_basis(t.txl);
        switch (t.txl) {
        case 0: refcpu_col<4>(s, X, j, t.px0, t.py0, t.mask_idx, M); break;
        case 1: refcpu_col<8>(s, X, j, t.px0, t.py0, t.mask_idx, M); break;
        case 2: refcpu_col<16>(s, X, j, t.px0, t.py0, t.mask_idx, M); break;
        default: refcpu_col<32>(s, X, j, t.px0, t.py0, t.mask_idx, M); break;
        }
    } else if (job.full) {
        /* FULL inter residual (DCT): rows first, item j = row j */
        const int qdc = t.plane ? job.q_dc_uv : job.q_dc, qac = t.plane ? job.q_ac_uv : job.q_ac;
        bool any;
        switch (t.txl) {
        case 0: any = full_row<4>(s, X, j, t.plane, t.px0, t.py0, qdc, qac, job.lossless, false); break;
        case 1: any = full_row<8>(s, X, j, t.plane, t.px0, t.py0, qdc, qac, job.lossless, false); break;
        case 2: any = full_row<16>(s, X, j, t.plane, t.px0, t.py0, qdc, qac, job.lossless, false); break;
        default: any = full_row<32>(s, X, j, t.plane, t.px0, t.py0, qdc, qac, job.lossless, false); break;
        }
        if (any) atomicOr(&s.txmask[t.mask_idx], 1u);
    } else {
        switch (t.txl) {
        case 0: spec_col<4>(s, X, j, t, job.q_dc, job.q_ac); break;
        case 1: spec_col<8>(s, X, j, t, job.q_dc, job.q_ac); break;
        case 2: spec_col<16>(s, X, j, t, job.q_dc, job.q_ac); break;
        default: spec_col<32>(s, X, j, t, job.q_dc, job.q_ac); break;
        }
    }
}

template <int A>
__device__ __forceinline__ void item_pass2(ReconSmem &s, const BlkS &b, int item)
{
    const cvp9_job_t &job = s.jc;
    int i;
    TxRef t = locate_item(b, item, &i);
    unsigned mask = s.txmask[t.mask_idx];
    if (!mask) return;
    if (A == CVP9_ARITH_REFCPU) {
        const double *M = dct_basis(t.txl);
        switch (t.txl) {
        case 0: refcpu_row<4>(s, i, t.px0, t.py0, mask, M); break;
        case 1: refcpu_row<8>(s, i, t.px0, t.py0, mask, M); break;
        case 2: refcpu_row<16>(s, i, t.px0, t.py0, mask, M); break;
        default: refcpu_row<32>(s, i, t.px0, t.py0, mask, M); break;
        }
    } else if (job.full) {
        /* item i = column i */
        switch (t.txl) {
        case 0: full_col<4>(s, i, t.plane, t.px0, t.py0, job.lossless, false); break;
        case 1: full_col<8>(s, i, t.plane, t.px0, t.py0, job.lossless, false); break;
        case 2: full_col<16>(s, i, t.plane, t.px0, t.py0, job.lossless, false); break;
        default: full_col<32>(s, i, t.plane, t.px0, t.py0, job.lossless, false); break;
        }
    } else {
        switch (t.txl) {
        case 0: spec_row<4>(s, i, t); break;
        case 1: spec_row<8>(s, i, t); break;
        case 2: spec_row<16>(s, i, t); break;
        default: spec_row<32>(s, i, t); break;
        }
    }
}

/* REFCPU item passes that keep the residual apart from the prediction:
 * item_pass2_res computes row `item` of its TX into res, item_add_res adds
 * it to the predicted pixels (TXs without coefficients have neither). */
template <int A>
__device__ __forceinline__ void item_pass2_res(ReconSmem &s, const BlkS &b, int item, int16_t *res)
{
    int i;
    TxRef t = locate_item(b, item, &i);
    unsigned mask = s.txmask[t.mask_idx];
    if (!mask) return;
    const double *M = dct_basis(t.txl);
    switch (t.txl) {
    case 0: refcpu_row_res<4>(s, i, t.px0, t.py0, mask, M, res); break;
    case 1: refcpu_row_res<8>(s, i, t.px0, t.py0, mask, M, res); break;
    case 2: refcpu_row_res<16>(s, i, t.px0, t.py0, mask, M, res); break;
    default: refcpu_row_res<32>(s, i, t.px0, t.py0, mask, M, res); break;
    }
}

template <int A>
__device__ __forceinline__ void item_add_res(ReconSmem &s, const BlkS &b, int item, const int16_t *res)
{
    int i;
    TxRef t = locate_item(b, item, &i);
    if (!s.txmask[t.mask_idx]) return;
    switch (t.txl) {
    case 0: refcpu_add_res<4>(s, i, t.px0, t.py0, res); break;
    case 1: refcpu_add_res<8>(s, i, t.px0, t.py0, res); break;
    case 2: refcpu_add_res<16>(s, i, t.px0, t.py0, res); break;
    default: refcpu_add_res<32>(s, i, t.px0, t.py0, res); break;
    }
}

/* ── Synchronisation helpers ────────────────────────────────────────────── */

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(unsigned *p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

/* Bounded wait until flag == epoch; returns false on timeout. */
__device__ bool wait_flag(const unsigned *flag, unsigned epoch)
{
    for (long long it = 0; it < kSpinLimit; it++) {
        if (ld_acquire(flag) == epoch) return true;
        __nanosleep(it < 64 ? 32 : 256);
    }
    return false;
}

__device__ __forceinline__ void pf_l2(const void *p)
{
    asm volatile("prefetch.global.L2 [%0];" :: "l"(p));
}

/* Prefetch into L2 the rows of a reference window (clamped like the
 * prediction reads) — first and last 128-byte line of each row. */
__device__ __forceinline__ void pf_window(const uint8_t *plane, int stride, int pw, int ph,
                                          int x0, int y0, int w, int h)
{
    int xm = pw > 0 ? pw - 1 : 0, ym = ph > 0 ? ph - 1 : 0;
    int xa = clampi(x0, 0, xm), xb = clampi(x0 + w - 1, 0, xm);
    for (int r = 0; r < h; r++) {
        const uint8_t *row = plane + (size_t)clampi(y0 + r, 0, ym) * stride;
        pf_l2(row + xa);
        if ((xb >> 7) != (xa >> 7)) pf_l2(row + xb);
    }
}

/* One thread per block, right after the descriptors are read: pull the
 * block's reference windows towards L2 so the prediction phase finds them
 * there. Addresses are clamped into the buffers exactly as the later reads
 * are. */
template <int A>
__device__ void prefetch_block(const BlkS &b, const cvp9_job_t &job, int sbx, int sby)
{
    if (b.flags & 1) return;
    const cvp9_ref_t *R;
    if (A == CVP9_ARITH_REFCPU) {
        int slot = (int)b.ref0 - 1;
        R = (slot >= 0 && slot < 8) ? &job.ref[slot] : nullptr;
    } else {
        R = &job.ref[job.ref_slot_of[clampi((int)b.ref0 - 1, 0, 2)] & 7];
    }
    if (!R || !R->plane) return;
    const int rw = R->w, rh = R->h, rcs = (rw + 1) >> 1;
    const uint8_t *ru = R->plane + (size_t)rw * rh;
    const uint8_t *rv = ru + (size_t)rcs * ((rh + 1) >> 1);
    const int gx = sbx + b.x, gy = sby + b.y, cbw = (b.cw + 1) >> 1, cbh = (b.ch + 1) >> 1;
    if (A == CVP9_ARITH_REFCPU) {
        int px8 = gx * 8 + b.mvx, py8 = gy * 8 + b.mvy;
        pf_window(R->plane, rw, rw, rh, px8 >> 3, py8 >> 3, b.cw + 1, b.ch + 1);
        int cx8 = (gx >> 1) * 8 + b.mvx / 2, cy8 = (gy >> 1) * 8 + b.mvy / 2;
        pf_window(ru, rcs, rw >> 1, rh >> 1, cx8 >> 3, cy8 >> 3, cbw + 1, cbh + 1);
        pf_window(rv, rcs, rw >> 1, rh >> 1, cx8 >> 3, cy8 >> 3, cbw + 1, cbh + 1);
    } else {
        pf_window(R->plane, rw, rw, rh, gx + (b.mvx >> 3) - 3, gy + (b.mvy >> 3) - 3, b.cw + 7, b.ch + 7);
        int cx = (gx >> 1) + (b.mvx >> 4) - 3, cy = (gy >> 1) + (b.mvy >> 4) - 3;
        pf_window(ru, rcs, rcs, (rh + 1) >> 1, cx, cy, cbw + 7, cbh + 7);
        pf_window(rv, rcs, rcs, (rh + 1) >> 1, cx, cy, cbw + 7, cbh + 7);
    }
}

/* Exclusive prefix sums of two per-thread counts over the CTA (thread order).
 * Returns the totals; uses s_tmp[2 * kWarps]. Must be called by all threads. */
__device__ __forceinline__ void cta_scan2(int a, int b, int *ea, int *eb, int *ta, int *tb, int *s_tmp)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int xa = a, xb = b;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int ya = __shfl_up_sync(0xffffffffu, xa, o), yb = __shfl_up_sync(0xffffffffu, xb, o);
        if (lane >= o) { xa += ya; xb += yb; }
    }
    if (lane == 31) { s_tmp[warp] = xa; s_tmp[kWarps + warp] = xb; }
    __syncthreads();
    int pa = 0, pb = 0, sa = 0, sb = 0;
#pragma unroll
    for (int w = 0; w < kWarps; w++) {
        int va = s_tmp[w], vb = s_tmp[kWarps + w];
        if (w < warp) { pa += va; pb += vb; }
        sa += va; sb += vb;
    }
    *ea = pa + xa - a;
    *eb = pb + xb - b;
    *ta = sa;
    *tb = sb;
}

/* Position and extent of chunk `chk` (level order): an 8x8 luma region of
 * its block clipped to the frame, and the matching 4x4 chroma region. */
struct ChunkP {
    const BlkS *b;
    int lx0, ly0, lw, lh, cx0, cy0, clw, clh;
};

__device__ __forceinline__ ChunkP chunk_params(const ReconSmem &s, int chk)
{
    ChunkP c;
    const int lo = s.chunk_blk[chk];
    const BlkS &b = s.blk[s.order[lo]];
    c.b = &b;
    const int k = chk - s.chunk_off[lo];
    const int nx = (b.cw + 7) >> 3;
    const int ccy = nx == 1 ? k : div_small(k, nx), ccx = k - ccy * nx;
    c.lx0 = b.x + ccx * 8;
    c.ly0 = b.y + ccy * 8;
    c.lw = min(8, b.cw - ccx * 8);
    c.lh = min(8, b.ch - ccy * 8);
    const int cbw = (b.cw + 1) >> 1, cbh = (b.ch + 1) >> 1;
    c.cx0 = (b.x >> 1) + ccx * 4;
    c.cy0 = (b.y >> 1) + ccy * 4;
    c.clw = min(4, cbw - ccx * 4);
    c.clh = min(4, cbh - ccy * 4);
    return c;
}

} /* namespace */

/* ── Kernels ─────────────────────────────────────────────────────────────── */

/* Per block: SB membership and the contiguous range of each SB. The
 * per-frame scratch (sb_range, status) is zeroed before this launch. */
__global__ void __launch_bounds__(256) k_scan_blocks(const cvp9_job_t *__restrict__ jobs)
{
    const cvp9_job_t &job = jobs[blockIdx.y];
    const vp9_macroblock_info_t *B = job.blocks;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < job.num_blocks; i += gridDim.x * blockDim.x) {
    auto sb_of = [&](uint32_t k, bool *ok) -> int {
        vp9_macroblock_info_t b = B[k];
        int x = b.x, y = b.y, w = b.width, h = b.height;
        bool good = x < job.W && y < job.H && w >= 4 && h >= 4 && w <= 64 && h <= 64 &&
                    !(x & 3) && !(y & 3) && !(w & 3) && !(h & 3) &&
                    (x & 63) + w <= 64 && (y & 63) + h <= 64 && b.tx_size <= 3;
        *ok = good;
        return (y >> 6) * job.sb_cols + (x >> 6);
    };
    bool ok;
    int sb = sb_of(i, &ok);
    if (!ok) { atomicOr(job.status, (unsigned)CVP9_JOB_BAD_BLOCK); continue; }
    bool okp = true, okn = true;
    int prev = i > 0 ? sb_of(i - 1, &okp) : -1;
    int next = i + 1 < job.num_blocks ? sb_of(i + 1, &okn) : -1;
    uint32_t *r = job.sb_range + 4 * sb;
    if (prev != sb) { r[0] = i; atomicAdd(&r[2], 1u); }
    if (next != sb) r[1] = i + 1;
    }
}

template <int A>
__global__ void __launch_bounds__(kThreads, 3) k_recon(const cvp9_job_t *__restrict__ jobs,
                                                   const uint32_t *__restrict__ tickets,
                                                   uint32_t n_tickets, uint32_t *ticket_counter,
                                                   const uint32_t *__restrict__ n_dev, int warp_levels)
{
    /* with the inter fast path the general ticket count is known on the device */
    if (n_dev) n_tickets = *n_dev;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ReconSmem &s = *reinterpret_cast<ReconSmem *>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const cvp9_job_t &job = s.jc;     /* valid after the reset barrier */

    for (;;) {
        __syncthreads();
        if (tid == 0) s.ticket = (int)atomicAdd(ticket_counter, 1u);
        __syncthreads();
        const int ticket = s.ticket;
        if (ticket >= (int)n_tickets) return;
        const uint32_t code = tickets[ticket];
        const cvp9_job_t *gj = jobs + (code >> 20);
        {
            const uint32_t *src = reinterpret_cast<const uint32_t *>(gj);
            uint32_t *dst = reinterpret_cast<uint32_t *>(&s.jc);
            for (int i = tid; i < (int)(sizeof(cvp9_job_t) / 4); i += kThreads) dst[i] = src[i];
        }
        const int sb = (int)(code & 0xFFFFFu);
        const int g_sb_cols = gj->sb_cols;
        const int sbr = sb / g_sb_cols, sbc = sb - sbr * g_sb_cols;
        const int sbx = sbc * 64, sby = sbr * 64;
        const uint32_t *rg = gj->sb_range + 4 * sb;
        const uint32_t start = rg[0], end = rg[1], groups = rg[2];
        const uint32_t g_nblocks = gj->num_blocks;
        const bool layout_bad = (*(volatile uint32_t *)gj->status & CVP9_JOB_BAD_BLOCK) != 0;
        bool bad = groups > 1 || end < start || end > g_nblocks ||
                   (groups && end - start > (uint32_t)kMaxBlocks);
        int nb = (groups && !bad && !layout_bad) ? (int)(end - start) : 0;

        /* reset per-SB state, tile = 128 */
        {
            uint4 *t4 = reinterpret_cast<uint4 *>(s.ty);
            const uint4 fill = make_uint4(0x80808080u, 0x80808080u, 0x80808080u, 0x80808080u);
            for (int i = tid; i < (kTyBytes + 2 * kTcBytes) / 16; i += kThreads) t4[i] = fill;
        }
        for (int i = tid; i < 256 + 128; i += kThreads) s.txmask[i] = 0;
        for (int i = tid; i < 256; i += kThreads) s.cell[i] = 0;
        for (int i = tid; i <= kMaxBlocks; i += kThreads) { s.lvl_cnt[i] = 0ull; s.lvl_big[i] = 0; }
        if (tid == 0) { s.nlev = 1; s.nb = nb; s.c_lo = 0xFFFFFFFFu; s.c_hi = 0u; }
        __syncthreads();

        /* 1. load and re-check blocks (a block must sit inside this SB,
         * 4-aligned, 4..64 px, tx_size <= 3; sub-8x8 blocks on the 8x8 MI
         * grid), then mark the 4x4 cells each one covers */
        bool my_intra = false, overlap = false, my_bad = false;
        BlkS mb;
        int nch = 0, nit = 0;
        if (tid < nb) {
            vp9_macroblock_info_t g = job.blocks[start + tid];
            int lx = (int)g.x - sbx, ly = (int)g.y - sby;
            my_bad = lx < 0 || ly < 0 || (lx & 3) || (ly & 3) || (g.width & 3) || (g.height & 3) ||
                     g.width < 4 || g.height < 4 || lx + g.width > 64 || ly + g.height > 64 ||
                     g.x >= job.W || g.y >= job.H || g.tx_size > 3 ||
                     ((g.width < 8 || g.height < 8) && ((lx & 7) || (ly & 7)));
            if (my_bad) { lx = 0; ly = 0; g.width = 4; g.height = 4; g.tx_size = 0; }
            mb.x = (uint8_t)lx;
            mb.y = (uint8_t)ly;
            mb.w = g.width;
            mb.h = g.height;
            int cw = g.width, ch = g.height;
            if (g.x + cw > job.W) cw = job.W - g.x;
            if (g.y + ch > job.H) ch = job.H - g.y;
            mb.cw = (uint8_t)cw;
            mb.ch = (uint8_t)ch;
            mb.txl = g.tx_size;
            mb.flags = (uint8_t)((g.is_intra ? 1 : 0) | (g.skip ? 2 : 0));
            mb.ymode = g.y_mode;
            mb.uvmode = g.uv_mode;
            mb.ref0 = g.ref_frame[0];
            mb.mvx = g.mv[0][0];
            mb.mvy = g.mv[0][1];
            mb.ref1 = 0;
            mb.mv1x = g.mv[1][0];
            mb.mv1y = g.mv[1][1];
            mb.coeff = g.coeff_offset;
            if (A == CVP9_ARITH_SPEC && job.full) {
                /* the block's whole MI for a sub-8x8 block (one MV, one
                 * mode); a second reference; intra blocks TX by TX */
                if (g.width < 8 || g.height < 8) {
                    mb.cw = (uint8_t)min(8, job.W - (int)g.x);
                    mb.ch = (uint8_t)min(8, job.H - (int)g.y);
                }
                if (!g.is_intra) mb.ref1 = g.ref_frame[1];
                else mb.flags |= 4;
            }
            residual_layout<A>(mb, job, g.x, g.y);
            s.blk[tid] = mb;
            my_intra = g.is_intra != 0;
            nch = block_chunks(mb);
            nit = block_items(mb);
        }
        if (__syncthreads_or(my_bad)) {
            /* leave the tile at 128 and flag the frame */
            if (tid == 0) atomicOr(job.status, (unsigned)CVP9_JOB_BAD_BLOCK);
            nb = 0;
            my_intra = false;
            if (tid == 0) s.nb = 0;
        }
        if (tid < nb) prefetch_block<A>(mb, job, sbx, sby);
        {
            /* span of coefficients the residual pass reads */
            unsigned lo = 0xFFFFFFFFu, hi = 0u;
            if (tid < nb) {
                uint64_t n = 0;
#pragma unroll
                for (int q = 0; q < 3; q++) n += (uint64_t)mb.pnt[q] * (uint64_t)(16 << (2 * mb.ptxl[q]));
                uint64_t e = (uint64_t)mb.coeff + n;
                if (n) { lo = mb.coeff; hi = e > 0xFFFFFFFFull ? 0xFFFFFFFFu : (unsigned)e; }
            }
            lo = __reduce_min_sync(0xffffffffu, lo);
            hi = __reduce_max_sync(0xffffffffu, hi);
            if (lane == 0) { atomicMin(&s.c_lo, lo); atomicMax(&s.c_hi, hi); }
        }
        if (tid < nb) {
            /* cells a block writes: its prediction area; under SPEC a
             * sub-8x8 block's residual spans the whole 8x8 MI
             * (vp9_kf_tile.c:327-330), so it owns that area too */
            int ow = mb.cw, oh = mb.ch;
            if (A == CVP9_ARITH_SPEC && (mb.w < 8 || mb.h < 8)) {
                ow = min(8, job.W - (sbx + mb.x));
                oh = min(8, job.H - (sby + mb.y));
            }
            int c0x = mb.x >> 2, c0y = mb.y >> 2;
            int c1x = (mb.x + ow - 1) >> 2, c1y = (mb.y + oh - 1) >> 2;
            for (int cy = c0y; cy <= c1y; cy++)
                for (int cx = c0x; cx <= c1x; cx++)
                    if (atomicCAS(&s.cell[cy * 16 + cx], (uint16_t)0, (uint16_t)(tid + 1)) != 0) overlap = true;
        }
        const int any_intra = __syncthreads_or(my_intra);
        const int any_inter = __syncthreads_or(tid < nb && !my_intra);
        const int any_overlap = __syncthreads_or(overlap);

        /* stage the SB's coefficient span in shared memory with 16-byte loads
         * (issued now, stored after the dependency analysis) */
        const unsigned c_lo = s.c_lo, c_hi = s.c_hi;
        const unsigned c_base = c_lo & ~7u;
        const bool staged = c_hi > c_lo && c_hi <= job.num_coeffs && c_hi - c_base <= (unsigned)kCoefStage;
        const bool c_vec = !((uintptr_t)job.coeffs & 15);
        constexpr int kStageIt = kCoefStage / 8 / kThreads;
#pragma unroll
        for (int k = 0; k < kStageIt; k++) {
            unsigned e = c_base + 8u * (unsigned)(tid + k * kThreads);
            if (staged && c_vec && e < c_hi && e + 8 <= job.num_coeffs)
                cp_async16(&s.coef[e - c_base], job.coeffs + e);
        }
        cp_async_commit();

        /* 2. dependency levels. An intra block depends on the blocks that own
         * its above row, left column and above-left corner inside the SB. */
        bool seq = any_overlap != 0;
        int deps[33];
        int ndeps = 0;
        if (any_intra && !seq) {
            bool late = false;
            if (tid < nb && my_intra) {
                const BlkS &b = s.blk[tid];
                int c0x = b.x >> 2, c0y = b.y >> 2;
                int c1x = (b.x + b.cw - 1) >> 2, c1y = (b.y + b.ch - 1) >> 2;
                auto add = [&](int cx, int cy) {
                    int o = s.cell[cy * 16 + cx];
                    if (!o) return;
                    o -= 1;
                    if (o >= tid) { late = true; return; }
                    for (int k = 0; k < ndeps; k++) if (deps[k] == o) return;
                    if (ndeps < 33) deps[ndeps++] = o;
                };
                if (c0y > 0) for (int cx = c0x; cx <= c1x; cx++) add(cx, c0y - 1);
                if (c0x > 0) for (int cy = c0y; cy <= c1y; cy++) add(c0x - 1, cy);
                if (c0x > 0 && c0y > 0) add(c0x - 1, c0y - 1);
            }
            seq = __syncthreads_or(late) != 0;
        }
        if (tid < kMaxBlocks) s.lvl[tid] = 0;
        __syncthreads();
        if (seq) {
            if (tid < nb) s.lvl[tid] = (uint16_t)tid;
        } else if (any_intra) {
            /* longest-path levels. A block's dependencies all have lower
             * indices, so the warps settle their 32 blocks in index order:
             * warp w relaxes its blocks (warp syncs only) until none
             * changes, the earlier warps' levels being final, then one CTA
             * barrier hands over to warp w + 1 */
            volatile uint16_t *vl = s.lvl;
            const int nw = (nb + 31) >> 5;
            for (int w = 0; w < nw; w++) {
                if (warp == w) {
                    for (int it = 0; it <= 32; it++) {   /* settles in at most 32 passes: a DAG in index order */
                        bool changed = false;
                        if (tid < nb && ndeps) {
                            int L = 0;
                            for (int k = 0; k < ndeps; k++) { int v = vl[deps[k]] + 1; L = v > L ? v : L; }
                            if (L != vl[tid]) { vl[tid] = (uint16_t)L; changed = true; }
                        }
                        __syncwarp();
                        if (!__any_sync(0xffffffffu, changed)) break;
                    }
                }
                __syncthreads();
            }
        }
        __syncthreads();

        /* 3. order blocks by level. One level (no intra dependency inside the
         * SB): list order, offsets from a CTA-wide prefix sum. Otherwise a
         * counting sort: each level's blocks, chunks and items get contiguous
         * ranges (one packed 64-bit atomic keeps a block's three offsets
         * consistent with each other). */
        if (!any_intra && !seq) {
            int ec, ei, tc, ti;
            cta_scan2(tid < nb ? nch : 0, tid < nb ? nit : 0, &ec, &ei, &tc, &ti, s.scan_tmp);
            if (tid < nb) {
                s.order[tid] = (uint16_t)tid;
                s.chunk_off[tid] = (uint16_t)ec;
                s.item_off[tid] = (uint16_t)ei;
            }
            if (tid == 0) {
                s.nlev = 1;
                s.base_blk[0] = 0; s.base_blk[1] = (uint16_t)nb;
                s.base_chunk[0] = 0; s.base_chunk[1] = (uint16_t)tc;
                s.base_item[0] = 0; s.base_item[1] = (uint16_t)ti;
                if (nb > 0) { s.chunk_off[nb] = (uint16_t)tc; s.item_off[nb] = (uint16_t)ti; }
            }
        } else {
        unsigned long long old = 0;
        int my_lvl = 0;
        if (tid < nb) {
            my_lvl = s.lvl[tid];
            atomicMax(&s.nlev, my_lvl + 1);
            /* small intra block: a warp predicts and transforms it alone */
            if (!my_intra || nit > 32 || nch > 4) s.lvl_big[my_lvl] = 1;
            old = atomicAdd(&s.lvl_cnt[my_lvl], (1ull << 40) | ((unsigned long long)nch << 20) |
                                                    (unsigned long long)nit);
        }
        __syncthreads();
        const int nlev_s = s.nlev;
        if (warp == 0) {
            /* exclusive scan over levels, 8 levels per lane */
            int per = (nlev_s + 31) / 32;
            int b0 = lane * per;
            unsigned sb_ = 0, sc = 0, si = 0;
            for (int l = b0; l < b0 + per && l < nlev_s; l++) {
                unsigned long long v = s.lvl_cnt[l];
                sb_ += (unsigned)(v >> 40); sc += (unsigned)((v >> 20) & 0xFFFFF); si += (unsigned)(v & 0xFFFFF);
            }
            unsigned xb = sb_, xc = sc, xi = si;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                unsigned yb = __shfl_up_sync(0xffffffffu, xb, o);
                unsigned yc = __shfl_up_sync(0xffffffffu, xc, o);
                unsigned yi = __shfl_up_sync(0xffffffffu, xi, o);
                if (lane >= o) { xb += yb; xc += yc; xi += yi; }
            }
            unsigned eb = xb - sb_, ec = xc - sc, ei = xi - si;
            for (int l = b0; l < b0 + per && l < nlev_s; l++) {
                s.base_blk[l] = (uint16_t)eb; s.base_chunk[l] = (uint16_t)ec; s.base_item[l] = (uint16_t)ei;
                unsigned long long v = s.lvl_cnt[l];
                eb += (unsigned)(v >> 40); ec += (unsigned)((v >> 20) & 0xFFFFF); ei += (unsigned)(v & 0xFFFFF);
            }
            if (lane == 31) { s.base_blk[nlev_s] = (uint16_t)eb; s.base_chunk[nlev_s] = (uint16_t)ec; s.base_item[nlev_s] = (uint16_t)ei; }
        }
        __syncthreads();
        if (tid < nb) {
            int p = s.base_blk[my_lvl] + (int)(old >> 40);
            s.order[p] = (uint16_t)tid;
            s.chunk_off[p] = (uint16_t)(s.base_chunk[my_lvl] + (int)((old >> 20) & 0xFFFFF));
            s.item_off[p] = (uint16_t)(s.base_item[my_lvl] + (int)(old & 0xFFFFF));
        }
        if (tid == 0 && nb > 0) { s.chunk_off[nb] = s.base_chunk[nlev_s]; s.item_off[nb] = s.base_item[nlev_s]; }
        }
        __syncthreads();
        const int nlev = s.nlev;
#pragma unroll
        for (int k = 0; k < kStageIt; k++) {
            unsigned e = c_base + 8u * (unsigned)(tid + k * kThreads);
            if (!staged || e >= c_hi) continue;
            if (!(c_vec && e + 8 <= job.num_coeffs))
                for (unsigned q = e; q < e + 8 && q < c_hi; q++) s.coef[q - c_base] = job.coeffs[q];
        }
        /* chunk -> block and TX item -> block maps, a warp per block */
        for (int p = warp; p < nb; p += kWarps) {
            int c0 = s.chunk_off[p], c1 = s.chunk_off[p + 1];
            for (int c = c0 + lane; c < c1; c += 32) s.chunk_blk[c] = (uint8_t)p;
            int i0 = s.item_off[p], i1 = s.item_off[p + 1];
            for (int i = i0 + lane; i < i1 && i < kMaxItems; i += 32) s.item_blk[i] = (uint8_t)p;
        }

        /* 4. wait for the neighbour SBs when intra blocks read their edges */
        if (any_intra) {
            if (tid == 0) {
                bool ok = true;
                if (sbc > 0) ok &= wait_flag(job.sb_done + sb - 1, job.epoch);
                if (sbr > 0) ok &= wait_flag(job.sb_done + sb - job.sb_cols, job.epoch);
                if (sbr > 0 && sbc > 0) ok &= wait_flag(job.sb_done + sb - job.sb_cols - 1, job.epoch);
                if (!ok) atomicOr(job.status, (unsigned)CVP9_JOB_TIMEOUT);
            }
            __syncthreads();
            /* halo: row above (x = -1..63) and column to the left */
            const uint8_t *Y = job.out;
            const uint8_t *U = job.out + (size_t)job.W * job.H;
            const uint8_t *V = U + (size_t)job.CW * job.CH;
            if (sby > 0) {
                for (int i = tid - 1; i < 64; i += kThreads) {
                    int gx = sbx + i;
                    if (gx >= 0 && gx < job.W) TY(s, i, -1) = Y[(size_t)(sby - 1) * job.W + gx];
                }
                for (int i = tid - 1; i < 32; i += kThreads) {
                    int gx = (sbx >> 1) + i;
                    if (gx >= 0 && gx < job.CW) {
                        TC(s, 1, i, -1) = U[(size_t)((sby >> 1) - 1) * job.CW + gx];
                        TC(s, 2, i, -1) = V[(size_t)((sby >> 1) - 1) * job.CW + gx];
                    }
                }
            }
            if (sbx > 0) {
                for (int i = tid; i < 64; i += kThreads) {
                    int gy = sby + i;
                    if (gy < job.H) TY(s, -1, i) = Y[(size_t)gy * job.W + sbx - 1];
                }
                for (int i = tid; i < 32; i += kThreads) {
                    int gy = (sby >> 1) + i;
                    if (gy < job.CH) {
                        TC(s, 1, -1, i) = U[(size_t)gy * job.CW + (sbx >> 1) - 1];
                        TC(s, 2, -1, i) = V[(size_t)gy * job.CW + (sbx >> 1) - 1];
                    }
                }
            }
        }
        /* FULL intra blocks, and the warp-per-block levels, read their
         * coefficients during the prediction phase */
        const bool warp_lv = warp_levels && any_intra;
        if ((A == CVP9_ARITH_SPEC && job.full) || warp_lv) cp_async_wait_all();
        __syncthreads();
        /* Every block intra and no two blocks overlapping (REFCPU, or SPEC
         * without the FULL completion, whose intra blocks reconstruct TX by
         * TX in their prediction warp): the first transform pass reads
         * coefficients only, so every TX's runs here at once, on all
         * threads, into its own place of the SB-wide temp (no inter
         * prediction stages reference windows there); the levels then
         * predict and run the second pass only */
        const bool pre1 = (A == CVP9_ARITH_REFCPU || !job.full) && warp_lv && !any_inter && !seq;
        /* REFCPU goes further: the second pass does not read the prediction
         * either (the residual is rounded and saturated on its own before
         * the add), so it runs here too, into a 64x64 int16 grid over the
         * coefficient staging (spent once the first pass has read it); a
         * level then predicts its blocks and adds their residual */
        const bool pre2 = A == CVP9_ARITH_REFCPU && pre1;
        int16_t *const res = s.coef;
        if (pre1) {
            const int n_items = min((int)s.base_item[nlev], kMaxItems);   /* <= 1024: disjoint luma TXs */
            for (int it = tid; it < n_items; it += kThreads) {
                const int lo = s.item_blk[it];
                item_pass1<A>(s, s.blk[s.order[lo]], it - s.item_off[lo], staged, c_base);
            }
            __syncthreads();
            if (pre2) {
                for (int it = tid; it < n_items; it += kThreads) {
                    const int lo = s.item_blk[it];
                    item_pass2_res<A>(s, s.blk[s.order[lo]], it - s.item_off[lo], res);
                }
                __syncthreads();
            }
        }

        /* 5. levels */
        for (int L = 0; L < nlev && nb > 0; L++) {
            if (warp_lv && !s.lvl_big[L]) {
                /* every block of the level is a small intra block: a warp
                 * per block predicts it and runs both transform passes on its
                 * lanes; one CTA barrier for the level instead of three */
                for (int pos = s.base_blk[L] + warp; pos < s.base_blk[L + 1]; pos += kWarps) {
                    const BlkS &b = s.blk[s.order[pos]];
                    if (b.flags & 4) {
                        full_intra_block(s, b, sbx, sby, staged, c_base, warp, lane);
                        continue;
                    }
                    for (int chk = s.chunk_off[pos]; chk < s.chunk_off[pos + 1]; chk++) {
                        const ChunkP c = chunk_params(s, chk);
                        predict_intra_chunk<A>(s, b, sbx + b.x, sby + b.y, c.lx0, c.ly0, c.lw, c.lh,
                                               c.cx0, c.cy0, c.clw, c.clh, lane);
                    }
                    __syncwarp();
                    const int n_it = s.item_off[pos + 1] - s.item_off[pos];
                    if (!pre1) {
                        for (int k = lane; k < n_it; k += 32) item_pass1<A>(s, b, k, staged, c_base);
                        __syncwarp();
                    }
                    if (pre2) {
                        for (int k = lane; k < n_it; k += 32) item_add_res<A>(s, b, k, res);
                    } else {
                        for (int k = lane; k < n_it; k += 32) item_pass2<A>(s, b, k);
                    }
                    __syncwarp();
                }
                __syncthreads();
                if (seq) {
                    for (int i = tid; i < 256 + 128; i += kThreads) s.txmask[i] = 0;
                    __syncthreads();
                }
                continue;
            }
            /* phase P: prediction, warp per 8x8 chunk. REFCPU stages the
             * windows of up to kRound chunks per warp with async copies into
             * the (idle) transform buffer, waits once, then computes them. */
            const int chk0 = s.base_chunk[L], chk1 = s.base_chunk[L + 1];
            if (A == CVP9_ARITH_REFCPU) {
                constexpr int kRound = 4;
                uint8_t *wst = reinterpret_cast<uint8_t *>(s.temp.d) + warp * (kRound * kChunkStage);
                const int q = lane >> 3, k = lane & 7;
                for (int base = chk0 + warp; base < chk1; base += kRound * kWarps) {
                    /* lane group q works on chunk base + q * kWarps */
                    const int chk = base + q * kWarps;
                    const bool have = chk < chk1;
                    ChunkP c;
                    McGeo g;
                    bool inter = false, has_ref = false;
                    if (have) {
                        c = chunk_params(s, chk);
                        inter = !(c.b->flags & 1);
                        if (inter) {
                            has_ref = refcpu_geo(s, *c.b, sbx, sby, c.lx0, c.ly0, c.lw, c.lh,
                                                 c.cx0, c.cy0, c.clw, c.clh, g);
                            if (has_ref) refcpu_issue8(wst + q * kChunkStage, g, c.lw, c.lh, c.clw, c.clh, k);
                        }
                    }
                    cp_async_commit();
                    cp_async_wait_all();
                    __syncwarp();
                    if (have && inter) {
                        if (has_ref)
                            refcpu_compute8(s, wst + q * kChunkStage, g, c.lx0, c.ly0, c.lw, c.lh,
                                            c.cx0, c.cy0, c.clw, c.clh, k);
                        else
                            refcpu_fill8(s, 127, c.lx0, c.ly0, c.lw, c.lh, c.cx0, c.cy0, c.clw, c.clh, k);
                    }
                    /* intra chunks of this round, one at a time with the whole warp */
                    const unsigned intra_mask = __ballot_sync(0xffffffffu, have && !inter && k == 0);
                    for (unsigned m = intra_mask; m; m &= m - 1) {
                        const int qq = (__ffs(m) - 1) >> 3;
                        ChunkP ci = chunk_params(s, base + qq * kWarps);
                        const BlkS &bi = *ci.b;
                        predict_intra_chunk<A>(s, bi, sbx + bi.x, sby + bi.y, ci.lx0, ci.ly0, ci.lw, ci.lh,
                                               ci.cx0, ci.cy0, ci.clw, ci.clh, lane);
                    }
                    __syncwarp();
                }
            } else {
                for (int chk = chk0 + warp; chk < chk1; chk += kWarps) {
                    ChunkP c = chunk_params(s, chk);
                    const BlkS &b = *c.b;
                    if (b.flags & 4) {
                        /* FULL intra: the warp of the block's first chunk
                         * does the whole block, TX by TX */
                        if (c.lx0 == b.x && c.ly0 == b.y) full_intra_block(s, b, sbx, sby, staged, c_base, warp, lane);
                    } else if (b.flags & 1)
                        predict_intra_chunk<A>(s, b, sbx + b.x, sby + b.y, c.lx0, c.ly0, c.lw, c.lh,
                                               c.cx0, c.cy0, c.clw, c.clh, lane);
                    else
                        spec_inter_chunk(s, b, sbx, sby, c.lx0, c.ly0, c.lw, c.lh, c.cx0, c.cy0,
                                         c.clw, c.clh, warp, lane);
                }
            }
            cp_async_wait_all();     /* the SB's coefficient span */
            __syncthreads();
            /* phase P': first transform pass, thread per TX column */
            if (!pre1) {
                for (int it = s.base_item[L] + tid; it < s.base_item[L + 1]; it += kThreads) {
                    const int lo = s.item_blk[it];
                    item_pass1<A>(s, s.blk[s.order[lo]], it - s.item_off[lo], staged, c_base);
                }
                __syncthreads();
            }
            /* phase Q: second pass + residual add, thread per TX row */
            for (int it = s.base_item[L] + tid; it < s.base_item[L + 1]; it += kThreads) {
                const int lo = s.item_blk[it];
                if (pre2) item_add_res<A>(s, s.blk[s.order[lo]], it - s.item_off[lo], res);
                else item_pass2<A>(s, s.blk[s.order[lo]], it - s.item_off[lo]);
            }
            __syncthreads();
            if (seq) {
                /* overlapping blocks may reuse a TX position at a later level */
                for (int i = tid; i < 256 + 128; i += kThreads) s.txmask[i] = 0;
                __syncthreads();
            }
        }

        /* 6. write the tile (clipped to the frame) and release the SB */
        {
            const int vw = min(64, job.W - sbx), vh = min(64, job.H - sby);
            uint8_t *Y = job.out;
            if ((job.W & 3) == 0) {
                for (int i = tid; i < vh * 16; i += kThreads) {
                    int r = i >> 4, c4 = (i & 15) * 4;
                    if (c4 >= vw) continue;
                    *reinterpret_cast<uint32_t *>(Y + (size_t)(sby + r) * job.W + sbx + c4) =
                        *reinterpret_cast<const uint32_t *>(&TY(s, c4, r));
                }
            } else {
                for (int i = tid; i < vh * 64; i += kThreads) {
                    int r = i >> 6, c = i & 63;
                    if (c < vw) Y[(size_t)(sby + r) * job.W + sbx + c] = TY(s, c, r);
                }
            }
            const int cvw = min(32, job.CW - (sbx >> 1)), cvh = min(32, job.CH - (sby >> 1));
            uint8_t *U = job.out + (size_t)job.W * job.H;
            uint8_t *V = U + (size_t)job.CW * job.CH;
            if ((job.CW & 3) == 0 && ((size_t)job.W * job.H & 3) == 0) {
                for (int i = tid; i < 2 * cvh * 8; i += kThreads) {
                    int p = i >= cvh * 8;
                    int k = p ? i - cvh * 8 : i;
                    int r = k >> 3, c4 = (k & 7) * 4;
                    if (c4 >= cvw) continue;
                    *reinterpret_cast<uint32_t *>((p ? V : U) + (size_t)((sby >> 1) + r) * job.CW + (sbx >> 1) + c4) =
                        *reinterpret_cast<const uint32_t *>(&TC(s, 1 + p, c4, r));
                }
            } else
            for (int i = tid; i < 2 * cvh * 32; i += kThreads) {
                int p = i >= cvh * 32;
                int k = p ? i - cvh * 32 : i;
                int r = k >> 5, c = k & 31;
                if (c >= cvw) continue;
                (p ? V : U)[(size_t)((sby >> 1) + r) * job.CW + (sbx >> 1) + c] = TC(s, 1 + p, c, r);
            }
        }
        if (tid == 0 && bad)
            atomicOr(job.status, (unsigned)CVP9_JOB_BAD_ORDER |
                                 ((groups && end >= start && end - start > (uint32_t)kMaxBlocks) ? (unsigned)CVP9_JOB_TOO_MANY : 0u));
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            st_release(job.sb_done + sb, job.epoch);
        }
    }
}

/* ── Inter-only superblocks: one warp per SB ─────────────────────────────
 *
 * Most superblocks of an inter frame hold inter blocks only; nothing in them
 * depends on another superblock of the same frame. k_inter gives each such
 * SB to one warp, which predicts and adds the residual in a per-warp tile
 * and writes the tile once, with no CTA barriers and no dependency analysis.
 * An SB the warp cannot take (an intra block, a block outside the supported
 * domain, overlapping blocks, uncovered 4x4 cells, more than 64 blocks) is
 * marked general and left to k_recon, which k_compact feeds with the general
 * tickets in their original SB-diagonal order. k_inter releases the done
 * flag of every SB it finishes, so general SBs that wait on a neighbour see
 * it done. The arithmetic is the REFCPU profile of k_recon, term for term. */

namespace {

constexpr int kFastWarps = 4;                     /* SBs per CTA */

/* One block, 16 bytes. geo: x/4 | y/4 << 4 | clamped cw << 8 | ch << 15 |
 * reference slot << 22 (REFCPU: pool slot, 15 none; SPEC: LAST/GOLDEN/ALTREF
 * 0..2) | tx_size << 26 | skip << 28. ext (SPEC): luma TXs per row | per
 * column << 5 | chroma TXs per row << 10 | per column << 14 | chroma
 * tx_size << 18. */
struct FastBlk {
    uint32_t geo;
    uint32_t mv;      /* mv[0]: col in the low half, row in the high half (1/8 pel) */
    uint32_t coeff;   /* first coefficient of the block */
    uint32_t ext;
};

__device__ __forceinline__ int fb_x(const FastBlk &b) { return (int)(b.geo & 0xfu) << 2; }
__device__ __forceinline__ int fb_y(const FastBlk &b) { return (int)((b.geo >> 4) & 0xfu) << 2; }
__device__ __forceinline__ int fb_cw(const FastBlk &b) { return (int)((b.geo >> 8) & 0x7fu); }
__device__ __forceinline__ int fb_ch(const FastBlk &b) { return (int)((b.geo >> 15) & 0x7fu); }
__device__ __forceinline__ int fb_slot(const FastBlk &b) { return (int)((b.geo >> 22) & 0xfu); }
__device__ __forceinline__ int fb_txl(const FastBlk &b) { return (int)((b.geo >> 26) & 3u); }
__device__ __forceinline__ bool fb_skip(const FastBlk &b) { return (b.geo >> 28) & 1u; }

/* Tile pitches: 72 and 40 bytes put eight consecutive rows in eight
 * different bank groups (a 64-byte pitch maps rows r and r+2 together). */
constexpr int kFY = 72, kFC = 40;

struct __align__(16) FastSmem {                   /* one per warp; 16-byte vector access */
    uint8_t  ty[64 * kFY];                        /* luma tile */
    uint8_t  tu[32 * kFC];
    uint8_t  tv[32 * kFC];
    union {
        int16_t  coef[1056];                      /* residual: the TXs in flight, (N*N + 2) apart */
        uint32_t cells[8];                        /* set-up: 4x4-cell occupancy, 2 cell rows per word */
    };
    FastBlk  blk[64];
    union {
        struct {                                  /* prediction */
            uint16_t choff[65];                   /* first chunk of each block */
            uint8_t  chblk[128];                  /* chunk -> block */
        };
        struct {                                  /* residual, per TX size */
            uint16_t txoff[65];                   /* first TX of each block */
            uint8_t  txblk[256];                  /* TX -> block */
        };
    };
};

/* The basis again in global memory: lane-varying reads are served by L1
 * instead of being serialised by the constant cache. */
__device__ __align__(16) double g_dct[16 + 64 + 256 + 1024];

static_assert(sizeof(FastSmem) % 16 == 0, "per-warp tiles must stay 16-byte aligned");
static_assert(sizeof(FastSmem) * kFastWarps + 1024 <= 233472 / 5, "five CTAs of k_inter per SM");
static_assert(offsetof(FastSmem, coef) % 16 == 0 && offsetof(FastSmem, tu) % 16 == 0 &&
              offsetof(FastSmem, tv) % 16 == 0, "vector-accessed members must be 16-byte aligned");

/* 16 bytes from an 8-byte-aligned shared-memory address */
__device__ __forceinline__ uint4 ld_smem16(const uint8_t *p)
{
    const uint2 a = reinterpret_cast<const uint2 *>(p)[0], b = reinterpret_cast<const uint2 *>(p)[1];
    return make_uint4(a.x, a.y, b.x, b.y);
}

__device__ __forceinline__ int warp_incl_scan(int x, int lane)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

/* The same nine bytes from two 8-byte reads of the aligned 16 bytes around
 * them (p & 7 <= 7, so r[0..8] always lie inside; callers keep the span
 * inside the buffer): fewer L1 requests than three word reads. */
__device__ __forceinline__ void ld9d(const uint8_t *p, uint32_t &lo, uint32_t &mid, uint32_t &hi)
{
    const uintptr_t a = (uintptr_t)p;
    const uint2 *q = reinterpret_cast<const uint2 *>(a & ~(uintptr_t)7);
    const uint2 v0 = __ldg(q), v1 = __ldg(q + 1);
    const unsigned o = (unsigned)(a & 7), sh = 8u * (o & 3u);
    /* words w[o/4 .. o/4 + 2] of the four, by whether o >= 4 */
    const bool up = o >= 4;
    const uint32_t w0 = up ? v0.y : v0.x, w1 = up ? v1.x : v0.y, w2 = up ? v1.y : v1.x;
    lo = __funnelshift_r(w0, w1, sh);
    mid = __funnelshift_r(w1, w2, sh);
    hi = w2 >> sh;
}

/* The same nine bytes with every sample clamped into [0, pw-1] x [0, ph-1]. */
__device__ __forceinline__ void ld9c(const uint8_t *plane, int pw, int ph, int x0, int y,
                                     uint32_t &lo, uint32_t &mid, uint32_t &hi)
{
    const uint8_t *row = plane + (size_t)clampi(y, 0, ph - 1) * pw;
    uint32_t v[3] = { 0, 0, 0 };
#pragma unroll
    for (int x = 0; x < 9; x++) v[x >> 2] |= (uint32_t)__ldg(row + clampi(x0 + x, 0, pw - 1)) << (8 * (x & 3));
    lo = v[0]; mid = v[1]; hi = v[2];
}

__device__ __forceinline__ void ld5w(const uint8_t *p, uint32_t &lo, uint32_t &hi)
{
    const uintptr_t a = (uintptr_t)p;
    const uint32_t *w = reinterpret_cast<const uint32_t *>(a & ~(uintptr_t)3);
    const unsigned sh = 8u * (unsigned)(a & 3);
    const uint32_t w0 = __ldg(w), w1 = __ldg(w + 1);
    lo = __funnelshift_r(w0, w1, sh);
    hi = w1 >> sh;
}

/* five chroma bytes, clamped into [0, cw-1] x [0, ch-1] (cw, ch may be 0) */
__device__ __forceinline__ void ld5c(const uint8_t *plane, int stride, int cw, int ch, int x0, int y,
                                     uint32_t &lo, uint32_t &hi)
{
    const int xm = cw > 0 ? cw - 1 : 0, ym = ch > 0 ? ch - 1 : 0;
    const uint8_t *row = plane + (size_t)clampi(y, 0, ym) * stride;
    uint32_t v[2] = { 0, 0 };
#pragma unroll
    for (int x = 0; x < 5; x++) v[x >> 2] |= (uint32_t)__ldg(row + clampi(x0 + x, 0, xm)) << (8 * (x & 3));
    lo = v[0]; hi = v[1];
}

/* Two-stage bilinear of vp9_reconstruct.c:105-128 on two samples at once:
 * (a (8-f) + b f + 4) >> 3 per 16-bit field; every intermediate is below
 * 2^11, so fields never carry into each other. */
__device__ __forceinline__ uint32_t bil2(uint32_t a, uint32_t b, uint32_t wa, uint32_t wb)
{
    return ((a * wa + b * wb + 0x00040004u) >> 3) & 0x00ff00ffu;
}

/* Eight luma samples of one row from rows r (lo0 mid0 hi0) and r+1. */
__device__ __forceinline__ void bilinear8(uint32_t lo0, uint32_t mid0, uint32_t hi0,
                                          uint32_t lo1, uint32_t mid1, uint32_t hi1,
                                          int fx, int fy, uint32_t &o0, uint32_t &o1)
{
    const uint32_t wx = 8u - (uint32_t)fx, ux = (uint32_t)fx, wy = 8u - (uint32_t)fy, uy = (uint32_t)fy;
    /* fields (r[2k], r[2k+1]) and (r[2k+1], r[2k+2]) */
    const uint32_t s0 = __funnelshift_r(lo0, mid0, 8), t0 = __funnelshift_r(mid0, hi0, 8);
    const uint32_t s1 = __funnelshift_r(lo1, mid1, 8), t1 = __funnelshift_r(mid1, hi1, 8);
    const uint32_t h00 = bil2(__byte_perm(lo0, 0, 0x4140), __byte_perm(s0, 0, 0x4140), wx, ux);
    const uint32_t h01 = bil2(__byte_perm(lo0, 0, 0x4342), __byte_perm(s0, 0, 0x4342), wx, ux);
    const uint32_t h02 = bil2(__byte_perm(mid0, 0, 0x4140), __byte_perm(t0, 0, 0x4140), wx, ux);
    const uint32_t h03 = bil2(__byte_perm(mid0, 0, 0x4342), __byte_perm(t0, 0, 0x4342), wx, ux);
    const uint32_t h10 = bil2(__byte_perm(lo1, 0, 0x4140), __byte_perm(s1, 0, 0x4140), wx, ux);
    const uint32_t h11 = bil2(__byte_perm(lo1, 0, 0x4342), __byte_perm(s1, 0, 0x4342), wx, ux);
    const uint32_t h12 = bil2(__byte_perm(mid1, 0, 0x4140), __byte_perm(t1, 0, 0x4140), wx, ux);
    const uint32_t h13 = bil2(__byte_perm(mid1, 0, 0x4342), __byte_perm(t1, 0, 0x4342), wx, ux);
    const uint32_t v0 = bil2(h00, h10, wy, uy), v1 = bil2(h01, h11, wy, uy);
    const uint32_t v2 = bil2(h02, h12, wy, uy), v3 = bil2(h03, h13, wy, uy);
    o0 = __byte_perm(v0, v1, 0x6420);
    o1 = __byte_perm(v2, v3, 0x6420);
}

/* Four chroma samples from rows r (lo0 hi0: bytes 0..4) and r+1. */
__device__ __forceinline__ uint32_t bilinear4(uint32_t lo0, uint32_t hi0, uint32_t lo1, uint32_t hi1,
                                              int fx, int fy)
{
    const uint32_t wx = 8u - (uint32_t)fx, ux = (uint32_t)fx, wy = 8u - (uint32_t)fy, uy = (uint32_t)fy;
    const uint32_t s0 = __funnelshift_r(lo0, hi0, 8), s1 = __funnelshift_r(lo1, hi1, 8);
    const uint32_t h00 = bil2(__byte_perm(lo0, 0, 0x4140), __byte_perm(s0, 0, 0x4140), wx, ux);
    const uint32_t h01 = bil2(__byte_perm(lo0, 0, 0x4342), __byte_perm(s0, 0, 0x4342), wx, ux);
    const uint32_t h10 = bil2(__byte_perm(lo1, 0, 0x4140), __byte_perm(s1, 0, 0x4140), wx, ux);
    const uint32_t h11 = bil2(__byte_perm(lo1, 0, 0x4342), __byte_perm(s1, 0, 0x4342), wx, ux);
    return __byte_perm(bil2(h00, h10, wy, uy), bil2(h01, h11, wy, uy), 0x6420);
}

/* One lane's share of a prediction pass, split so that a warp can issue the
 * reads of two passes before computing either. */
struct FastLuma {
    uint8_t *d;
    int lw, fx, fy;
    bool act, ref;
    uint32_t lo0, mid0, hi0, lo1, mid1, hi1;
};

struct FastChroma {
    uint8_t *d;
    int clw, fx, fy;
    bool act, ref;
    uint32_t lo0, hi0, lo1, hi1;
};

/* Chunk k of block b: its 8x8 luma and 4x4 chroma regions (clipped). */
template <class S>
__device__ __forceinline__ void fast_chunk(const S &w, int c, FastBlk &fb, int &lx0, int &ly0, int &lw,
                                           int &lh, int &cx0, int &cy0, int &clw, int &clh)
{
    const int b = w.chblk[c];
    fb = w.blk[b];
    const int bx = fb_x(fb), by = fb_y(fb), cw = fb_cw(fb), ch = fb_ch(fb);
    const int k = c - w.choff[b];
    const int nx = (cw + 7) >> 3;
    const int ccy = nx == 1 ? k : div_small(k, nx), ccx = k - ccy * nx;
    lx0 = bx + ccx * 8;
    ly0 = by + ccy * 8;
    lw = min(8, cw - ccx * 8);
    lh = min(8, ch - ccy * 8);
    cx0 = (bx >> 1) + ccx * 4;
    cy0 = (by >> 1) + ccy * 4;
    clw = min(4, ((cw + 1) >> 1) - ccx * 4);
    clh = min(4, ((ch + 1) >> 1) - ccy * 4);
}

/* Where a superblock's prediction lands: its luma and chroma origins and
 * pitches (the warp's shared tiles, or the frame itself), and the extent
 * inside the frame from those origins (luma vw x vh, chroma cvw x cvh):
 * SPEC TXs follow the MI grid and can reach past the frame edge, where
 * nothing is written. */
struct PredDst {
    uint8_t *y, *u, *v;
    int      py, pc;
    int      vw, vh, cvw, cvh;
};

/* One lane's luma row (chunk c, row lane%8) and chroma row (plane
 * (lane/4)%2, row lane%4) of chunk c: geometry, reference and MV decoded
 * once for both, reads issued, nothing computed yet. */
template <class S>
__device__ __forceinline__ void fast_pred_issue(const S &w, const PredDst &D, const cvp9_job_t &job, int c, int lane,
                                                int nchunks, int sbx, int sby, FastLuma &J, FastChroma &K)
{
    /* Each lane reads one reference row of its chunk (luma row kk, chroma
     * row r of its plane) and takes the row below from the next lane; the
     * last lane of a chunk (plane) reads its second row itself. Lanes below
     * the chunk's clipped height still read, for their upper neighbours.
     * A row is read as aligned words when its needed bytes are inside the
     * reference and the words past its end stay inside the frame, else byte
     * by byte with every sample clamped — the same bytes wherever used. */
    J.act = J.ref = false;
    K.act = K.ref = false;
    const int kk = lane & 7, p = (lane >> 2) & 1, r = lane & 3;
    uint32_t l0 = 0, m0 = 0, h0 = 0, cl0 = 0, ch0 = 0;
    if (c < nchunks) {
        FastBlk fb;
        int lx0, ly0, lw, lh, cx0, cy0, clw, clh;
        fast_chunk(w, c, fb, lx0, ly0, lw, lh, cx0, cy0, clw, clh);
        const int slot = fb_slot(fb);
        const uint8_t *rp = nullptr;
        int rw = 0, rh = 0;
        if (slot < 8) {
            const cvp9_ref_t &R = job.ref[slot];
            rp = R.plane;
            rw = R.w;
            rh = R.h;
        }
        const int mvx = (int16_t)(fb.mv & 0xffffu), mvy = (int16_t)(fb.mv >> 16);
        J.act = kk < lh;
        J.d = D.y + (ly0 + kk) * D.py + lx0;
        J.lw = lw;
        K.act = r < clh && clw > 0;
        K.d = (p ? D.v : D.u) + (cy0 + r) * D.pc + cx0;
        K.clw = clw;
        if (rp) {
            J.ref = true;
            const int px8 = (sbx + lx0) * 8 + mvx, py8 = (sby + ly0) * 8 + mvy;
            const int ix = px8 >> 3, y0 = (py8 >> 3) + kk;
            J.fx = px8 & 7;
            J.fy = py8 & 7;
            /* luma rows are followed by the chroma planes: reads past a row
             * end stay inside the frame; the plane starts 8-byte aligned, so
             * with ix >= 0 they never start before it */
            const bool hin = ix >= 0 && ix + lw < rw && rw >= 16;   /* 16-byte reads stay in the frame */
            if (hin && y0 >= 0 && y0 < rh) ld9d(rp + (size_t)y0 * rw + ix, l0, m0, h0);
            else ld9c(rp, rw, rh, ix, y0, l0, m0, h0);
            if (kk == 7) {
                if (hin && y0 + 1 >= 0 && y0 + 1 < rh) ld9d(rp + (size_t)(y0 + 1) * rw + ix, J.lo1, J.mid1, J.hi1);
                else ld9c(rp, rw, rh, ix, y0 + 1, J.lo1, J.mid1, J.hi1);
            }
            if (clw > 0) {
                K.ref = true;
                const int rcs = (rw + 1) >> 1, crw = rw >> 1, crh = rh >> 1;
                const uint8_t *pl = rp + (size_t)rw * rh + (p ? (size_t)rcs * ((rh + 1) >> 1) : 0);
                const int cpx8 = ((sbx >> 1) + cx0) * 8 + mvx / 2, cpy8 = ((sby >> 1) + cy0) * 8 + mvy / 2;
                const int cix = cpx8 >> 3, y1 = (cpy8 >> 3) + r;
                K.fx = cpx8 & 7;
                K.fy = cpy8 & 7;
                /* a further chroma row below the one read: word reads stay inside */
                const bool chin = cix >= 0 && cix + clw < crw && rcs >= 8;   /* 8-byte reads stay in the plane */
                if (chin && y1 >= 0 && y1 + 1 < crh) ld5w(pl + (size_t)y1 * rcs + cix, cl0, ch0);
                else ld5c(pl, rcs, crw, crh, cix, y1, cl0, ch0);
                if (r == 3) {
                    if (chin && y1 + 1 >= 0 && y1 + 2 < crh) ld5w(pl + (size_t)(y1 + 1) * rcs + cix, K.lo1, K.hi1);
                    else ld5c(pl, rcs, crw, crh, cix, y1 + 1, K.lo1, K.hi1);
                }
            }
        }
    }
    const uint32_t nl = __shfl_down_sync(0xffffffffu, l0, 1), nm = __shfl_down_sync(0xffffffffu, m0, 1);
    const uint32_t nh = __shfl_down_sync(0xffffffffu, h0, 1);
    const uint32_t ncl = __shfl_down_sync(0xffffffffu, cl0, 1), nch = __shfl_down_sync(0xffffffffu, ch0, 1);
    J.lo0 = l0;
    J.mid0 = m0;
    J.hi0 = h0;
    if (kk != 7) {
        J.lo1 = nl;
        J.mid1 = nm;
        J.hi1 = nh;
    }
    K.lo0 = cl0;
    K.hi0 = ch0;
    if (r != 3) {
        K.lo1 = ncl;
        K.hi1 = nch;
    }
}

__device__ __forceinline__ void fast_luma_finish(const FastLuma &J)
{
    if (!J.act) return;
    uint32_t o0 = 0x7f7f7f7fu, o1 = 0x7f7f7f7fu;     /* missing reference: 127 */
    if (J.ref) bilinear8(J.lo0, J.mid0, J.hi0, J.lo1, J.mid1, J.hi1, J.fx, J.fy, o0, o1);
    if (J.lw == 8 && !((uintptr_t)J.d & 3)) {
        reinterpret_cast<uint32_t *>(J.d)[0] = o0;
        reinterpret_cast<uint32_t *>(J.d)[1] = o1;
    } else {
#pragma unroll
        for (int x = 0; x < 8; x++) if (x < J.lw) J.d[x] = (uint8_t)((x < 4 ? o0 : o1) >> (8 * (x & 3)));
    }
}

__device__ __forceinline__ void fast_chroma_finish(const FastChroma &J)
{
    if (!J.act) return;
    const uint32_t o = J.ref ? bilinear4(J.lo0, J.hi0, J.lo1, J.hi1, J.fx, J.fy) : 0x7f7f7f7fu;
    if (J.clw == 4 && !((uintptr_t)J.d & 3)) {
        *reinterpret_cast<uint32_t *>(J.d) = o;
    } else {
#pragma unroll
        for (int x = 0; x < 4; x++) if (x < J.clw) J.d[x] = (uint8_t)(o >> (8 * x));
    }
}

/* Where the q-th TX of size N in the SB sits; `ok` is false past the last
 * TX or when the TX's coefficients run past the array. */
template <int N, class S>
__device__ __forceinline__ const int16_t *fast_tx_locate(const S &w, const cvp9_job_t &job, int q, int ntx,
                                                        int i, int &px0, int &py0, bool &ok)
{
    ok = false;
    px0 = py0 = 0;
    if (q >= ntx) return nullptr;
    const int b = w.txblk[q];
    const FastBlk fb = w.blk[b];
    const int bx = fb_x(fb), by = fb_y(fb), cw = fb_cw(fb);
    const int nx = cw / N;
    const int tq = q - w.txoff[b];
    const int tyy = nx == 1 ? tq : tq / nx, txx = tq - tyy * nx;
    px0 = bx + txx * N;
    py0 = by + tyy * N;
    const uint64_t c0 = (uint64_t)fb.coeff + (uint64_t)tq * (N * N);
    if (c0 + N * N > (uint64_t)job.num_coeffs) return nullptr;
    ok = true;
    return job.coeffs + c0 + (uint64_t)i * N;
}

/* one TX row (N int16) into registers, widest loads the alignment allows */
template <int N>
__device__ __forceinline__ void fast_row_load(uint32_t (&v)[N / 2], const int16_t *src)
{
    const uintptr_t a = (uintptr_t)src;
    if (N >= 8 && !(a & 15)) {
#pragma unroll
        for (int k = 0; k < N / 8; k++) {
            const uint4 q = __ldg(reinterpret_cast<const uint4 *>(src) + k);
            v[4 * k] = q.x; v[4 * k + 1] = q.y; v[4 * k + 2] = q.z; v[4 * k + 3] = q.w;
        }
    } else if (!(a & 3)) {
#pragma unroll
        for (int k = 0; k < N / 2; k++) v[k] = __ldg(reinterpret_cast<const uint32_t *>(src) + k);
    } else {
#pragma unroll
        for (int k = 0; k < N / 2; k++)
            v[k] = (uint32_t)(uint16_t)__ldg(src + 2 * k) | (uint32_t)(uint16_t)__ldg(src + 2 * k + 1) << 16;
    }
}

/* REFCPU residual of every luma TX of size N in the SB. 32/N TXs at a time,
 * lane = (TX, row i). A lane forms T[i][k] = sum_l M[l][i] X[l][k] (l
 * ascending) for each nonzero column k and accumulates O[i][j] += T[i][k]
 * M[k][j] (k ascending) — the two passes of vp9_reconstruct.c:31-50 fused
 * per row. The loops run over the union of the group's nonzero rows and
 * columns so they stay warp-uniform; a term whose coefficient is zero in a
 * lane's own TX adds +-0 to a sum that is never -0, leaving it unchanged.
 * The next group's coefficients are loaded while the current one computes.
 * The predicted rows are read from, and the results written to, dst (the
 * warp's luma tile or the frame: row r of the superblock at dst + r *
 * pitch); frame rows (GLOBAL) are read before the transform, so that they
 * arrive while it computes. */
template <int N, bool GLOBAL, class S>
__device__ void fast_residual(S &w, uint8_t *dst, int pitch, const cvp9_job_t &job, int ntx, int lane)
{
    constexpr int G = 32 / N, NN = N * N;
    constexpr int NH = N == 32 ? 2 : 1, NJ = N / NH;
    constexpr unsigned kSeg = N == 32 ? 0xffffffffu : ((1u << N) - 1u);
    const int g = lane / N, i = lane % N;
    const int boff = N == 4 ? 0 : N == 8 ? 16 : N == 16 ? 80 : 336;
    const double *Mg = g_dct + boff;     /* lane-varying reads */
    const double *Mc = c_dct + boff;     /* warp-uniform reads */
    int16_t *X = w.coef + g * (NN + 2);      /* padded: the groups' rows fall in different banks */
    uint32_t rv[N / 2];
    int px0, py0;
    bool have;
    {
        const int16_t *src = fast_tx_locate<N>(w, job, g, ntx, i, px0, py0, have);
        if (have) fast_row_load<N>(rv, src);
    }
    for (int q0 = 0; q0 < ntx; q0 += G) {
        if (have) {
            uint32_t *dst = reinterpret_cast<uint32_t *>(X + i * N);
#pragma unroll
            for (int k = 0; k < N / 2; k++) dst[k] = rv[k];
        }
        __syncwarp();
        int npx0, npy0;
        bool nhave;
        {
            const int16_t *src = fast_tx_locate<N>(w, job, q0 + G + g, ntx, i, npx0, npy0, nhave);
            if (nhave) fast_row_load<N>(rv, src);
        }
        uint32_t cm = 0;                     /* nonzero rows of column i of this lane's TX */
        if (have) {
#pragma unroll
            for (int l = 0; l < N; l++) cm |= (X[l * N + i] != 0 ? 1u : 0u) << l;
        }
        const unsigned nzl = __ballot_sync(0xffffffffu, cm != 0);
        unsigned U = 0;
#pragma unroll
        for (int s = 0; s < G; s++) U |= nzl >> (s * N);
        U &= kSeg;
        if (U) {
#pragma unroll
            for (int h = 0; h < NH; h++) {
                uint8_t *rowp = dst + (py0 + i) * pitch + px0 + h * NJ;
                const bool words = !GLOBAL || !((uintptr_t)rowp & 3);
                uint32_t pix[NJ / 4];
#pragma unroll
                for (int j4 = 0; j4 < NJ / 4; j4++) pix[j4] = 0u;
                if (GLOBAL && have) {
                    if (words) {
#pragma unroll
                        for (int j4 = 0; j4 < NJ / 4; j4++) pix[j4] = reinterpret_cast<const uint32_t *>(rowp)[j4];
                    } else {
#pragma unroll
                        for (int j = 0; j < NJ; j++) pix[j >> 2] |= (uint32_t)rowp[j] << (8 * (j & 3));
                    }
                }
                double acc[NJ];
#pragma unroll
                for (int j = 0; j < NJ; j++) acc[j] = 0.0;
                for (unsigned u = U; u; u &= u - 1) {
                    const int k = __ffs(u) - 1;
                    const uint32_t cmk = __shfl_sync(0xffffffffu, cm, g * N + k);
                    const uint32_t cmu = __reduce_or_sync(0xffffffffu, cmk);
                    double t = 0.0;
                    for (uint32_t v = cmu; v; v &= v - 1) {
                        const int l = __ffs(v) - 1;
                        t = __dadd_rn(t, __dmul_rn(__ldg(Mg + l * N + i), (double)X[l * N + k]));
                    }
#pragma unroll
                    for (int j = 0; j < NJ; j++) acc[j] = __dadd_rn(acc[j], __dmul_rn(t, Mc[k * N + h * NJ + j]));
                }
                if (have) {
#pragma unroll
                    for (int j4 = 0; j4 < NJ / 4; j4++) {
                        uint32_t word = GLOBAL ? pix[j4] : reinterpret_cast<const uint32_t *>(rowp)[j4], outw = 0;
#pragma unroll
                        for (int e = 0; e < 4; e++) {
                            /* round half away from zero; the int16 saturation of
                             * vp9_reconstruct.c:52-59 cannot change the result of
                             * the 0..255 clamp that follows, so it is folded in */
                            const int r = __double2int_rz(__dadd_rn(acc[j4 * 4 + e], copysign(0.5, acc[j4 * 4 + e])));
                            const int px = (int)((word >> (8 * e)) & 0xffu);
                            outw |= (uint32_t)clampi(px + r, 0, 255) << (8 * e);
                        }
                        if (words) {
                            reinterpret_cast<uint32_t *>(rowp)[j4] = outw;
                        } else {
#pragma unroll
                            for (int e = 0; e < 4; e++) rowp[4 * j4 + e] = (uint8_t)(outw >> (8 * e));
                        }
                    }
                }
            }
        }
        __syncwarp();
        have = nhave;
        px0 = npx0;
        py0 = npy0;
    }
}

/* fast_residual with each group walking its own TX's nonzero columns
 * (ascending) instead of the union over the warp's groups: the warp loops
 * as long as its busiest group. Column k differs between groups, so the
 * basis row M[k][.] is read from the global copy (four 16-byte loads, L1
 * hits). Same operations and order per TX as fast_residual — the terms the
 * union adds are exact zeros. */
template <int N, bool GLOBAL, class S>
__device__ void fast_residual_d(S &w, uint8_t *dst, int pitch, const cvp9_job_t &job, int ntx, int lane)
{
    static_assert(N == 8, "the 8x8 transform");
    constexpr int G = 32 / N, NN = N * N;
    constexpr int boff = 16;
    const int g = lane / N, i = lane % N;
    const double *Mg = g_dct + boff;
    int16_t *X = w.coef + g * (NN + 2);
    uint32_t rv[N / 2];
    int px0, py0;
    bool have;
    {
        const int16_t *src = fast_tx_locate<N>(w, job, g, ntx, i, px0, py0, have);
        if (have) fast_row_load<N>(rv, src);
    }
    for (int q0 = 0; q0 < ntx; q0 += G) {
        uint32_t rm = 0;                     /* nonzero columns of this lane's row */
        if (have) {
            uint32_t *xs = reinterpret_cast<uint32_t *>(X + i * N);
#pragma unroll
            for (int k = 0; k < N / 2; k++) {
                xs[k] = rv[k];
                const uint32_t m = __vcmpne2(rv[k], 0u);
                rm |= ((m & 1u) | ((m >> 15) & 2u)) << (2 * k);
            }
        }
        /* nonzero columns of this lane's TX: OR over its group's lanes */
        uint32_t cols = rm;
#pragma unroll
        for (int o = 1; o < N; o <<= 1) cols |= __shfl_xor_sync(0xffffffffu, cols, o);
        __syncwarp();
        uint8_t *rowp = dst + (py0 + i) * pitch + px0;
        const bool words = !GLOBAL || !((uintptr_t)rowp & 3);
        uint32_t pix[N / 4];
#pragma unroll
        for (int j4 = 0; j4 < N / 4; j4++) pix[j4] = 0u;
        if (GLOBAL && have && cols) {
            if (words) {
#pragma unroll
                for (int j4 = 0; j4 < N / 4; j4++) pix[j4] = reinterpret_cast<const uint32_t *>(rowp)[j4];
            } else {
#pragma unroll
                for (int j = 0; j < N; j++) pix[j >> 2] |= (uint32_t)rowp[j] << (8 * (j & 3));
            }
        }
        int npx0, npy0;
        bool nhave;
        {
            const int16_t *src = fast_tx_locate<N>(w, job, q0 + G + g, ntx, i, npx0, npy0, nhave);
            if (nhave) fast_row_load<N>(rv, src);
        }
        double acc[N];
#pragma unroll
        for (int j = 0; j < N; j++) acc[j] = 0.0;
        const bool any = cols != 0;
        uint32_t left = cols;
        while (__any_sync(0xffffffffu, left != 0)) {
            const bool act = left != 0;
            const int k = act ? __ffs(left) - 1 : 0;
            left &= left - 1;
            /* rows of column k of this lane's TX: bit (group, row) of the ballot */
            const unsigned B = __ballot_sync(0xffffffffu, act && ((rm >> k) & 1u));
            if (act) {
                const unsigned rows = (B >> (g * N)) & ((1u << N) - 1u);
                double t = 0.0;
                for (unsigned v = rows; v; v &= v - 1) {
                    const int l = __ffs(v) - 1;
                    t = __dadd_rn(t, __dmul_rn(__ldg(Mg + l * N + i), (double)X[l * N + k]));
                }
                const double2 *Mr = reinterpret_cast<const double2 *>(Mg + k * N);
#pragma unroll
                for (int j2 = 0; j2 < N / 2; j2++) {
                    const double2 m = __ldg(Mr + j2);
                    acc[2 * j2] = __dadd_rn(acc[2 * j2], __dmul_rn(t, m.x));
                    acc[2 * j2 + 1] = __dadd_rn(acc[2 * j2 + 1], __dmul_rn(t, m.y));
                }
            }
        }
        if (any && have) {
#pragma unroll
            for (int j4 = 0; j4 < N / 4; j4++) {
                const uint32_t word = GLOBAL ? pix[j4] : reinterpret_cast<const uint32_t *>(rowp)[j4];
                uint32_t outw = 0;
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    /* round half away from zero; the int16 saturation of
                     * vp9_reconstruct.c:52-59 cannot change the result of
                     * the 0..255 clamp that follows, so it is folded in */
                    const int r = __double2int_rz(__dadd_rn(acc[j4 * 4 + e], copysign(0.5, acc[j4 * 4 + e])));
                    const int px = (int)((word >> (8 * e)) & 0xffu);
                    outw |= (uint32_t)clampi(px + r, 0, 255) << (8 * e);
                }
                if (words) {
                    reinterpret_cast<uint32_t *>(rowp)[j4] = outw;
                } else {
#pragma unroll
                    for (int e = 0; e < 4; e++) rowp[4 * j4 + e] = (uint8_t)(outw >> (8 * e));
                }
            }
        }
        __syncwarp();
        have = nhave;
        px0 = npx0;
        py0 = npy0;
    }
}

/* ── SPEC arithmetic in k_inter ─────────────────────────────────────────── */

/* 16 consecutive bytes of a row at p as four words (aligned word reads;
 * callers keep the aligned span inside the buffer) */
__device__ __forceinline__ void ld16w(const uint8_t *p, uint32_t o[4])
{
    const uintptr_t a = (uintptr_t)p;
    const uint32_t *w = reinterpret_cast<const uint32_t *>(a & ~(uintptr_t)3);
    const unsigned sh = 8u * (unsigned)(a & 3);
    const uint32_t w0 = __ldg(w), w1 = __ldg(w + 1), w2 = __ldg(w + 2), w3 = __ldg(w + 3), w4 = __ldg(w + 4);
    o[0] = __funnelshift_r(w0, w1, sh);
    o[1] = __funnelshift_r(w1, w2, sh);
    o[2] = __funnelshift_r(w2, w3, sh);
    o[3] = __funnelshift_r(w3, w4, sh);
}

/* the same 16 bytes, every sample clamped into [0, pw-1] x [0, ph-1] */
__device__ __forceinline__ void ld16c(const uint8_t *plane, int stride, int pw, int ph, int x0, int y, uint32_t o[4])
{
    const int xm = pw > 0 ? pw - 1 : 0, ym = ph > 0 ? ph - 1 : 0;
    const uint8_t *row = plane + (size_t)clampi(y, 0, ym) * stride;
    o[0] = o[1] = o[2] = o[3] = 0u;
#pragma unroll
    for (int x = 0; x < 16; x++) o[x >> 2] |= (uint32_t)__ldg(row + clampi(x0 + x, 0, xm)) << (8 * (x & 3));
}


/* shader rounding of one 8-tap sum: (acc + 64) >> 7 clipped to 8 bits */

/* bytes k..k+3 of o[] as one word (k a compile-time index) */
__device__ __forceinline__ uint32_t win4(const uint32_t o[4], int k)
{
    return (k & 3) ? __funnelshift_r(o[k >> 2], o[(k >> 2) + 1], 8 * (k & 3)) : o[k >> 2];
}

/* c + the dot product of four signed taps with four unsigned samples */


/* 4x4 byte transpose: rows a..d (one word of four columns each) to four
 * words, one column each (its bytes in row order) */
__device__ __forceinline__ void tr4(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t col[4])
{
    const uint32_t x0 = __byte_perm(a, b, 0x5140), x1 = __byte_perm(a, b, 0x7362);
    const uint32_t y0 = __byte_perm(c, d, 0x5140), y1 = __byte_perm(c, d, 0x7362);
    col[0] = __byte_perm(x0, y0, 0x5410);
    col[1] = __byte_perm(x0, y0, 0x7632);
    col[2] = __byte_perm(x1, y1, 0x5410);
    col[3] = __byte_perm(x1, y1, 0x7632);
}

/* Luma prediction of four chunks (vp9_mc.comp.glsl:61-110): lane = (chunk
 * c0 + lane/8, k = lane%8). Horizontal 8-tap rows k and k+8 of each chunk's
 * 15-row window go to shared rows (rounded, clipped to 8 bits), then lane k
 * filters output row k vertically. Fetches clamp into the reference. */
template <class S>
__device__ void spec_luma_pass(S &w, const PredDst &D, const cvp9_job_t &job, int c0, int nchunks, int sbx, int sby,
                               int lane)
{
    uint8_t *hb = reinterpret_cast<uint8_t *>(w.coef);        /* 4 chunks x 15 rows x 8 */
    const int q = lane >> 3, k = lane & 7, c = c0 + q;
    FastBlk fb;
    int lx0 = 0, ly0 = 0, lw = 0, lh = 0, cx0, cy0, clw, clh;
    const uint8_t *rp = nullptr;
    int rw = 0, rh = 0, fx = 0, fy = 0, bx = 0, by = 0;
    if (c < nchunks) {
        fast_chunk(w, c, fb, lx0, ly0, lw, lh, cx0, cy0, clw, clh);
        const cvp9_ref_t &R = job.ref[job.ref_slot_of[fb_slot(fb) & 3] & 7];
        rp = R.plane; rw = R.w; rh = R.h;
        const int mvx = (int16_t)(fb.mv & 0xffffu), mvy = (int16_t)(fb.mv >> 16);
        bx = sbx + lx0 + (mvx >> 3);
        by = sby + ly0 + (mvy >> 3);
        fx = (mvx & 7) << 1;
        fy = (mvy & 7) << 1;
        if (rp) {
            const uint32_t ta = c_subpel_pk[fx][0], tb = c_subpel_pk[fx][1];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int hr = k + 8 * h;
                if (hr >= lh + 7) continue;
                const int y = by - 3 + hr, x0 = bx - 3;
                uint32_t o[4];
                if (x0 >= 0 && x0 + lw + 6 < rw && y >= 0 && y < rh) ld16w(rp + (size_t)y * rw + x0, o);
                else ld16c(rp, rw, rw, rh, x0, y, o);
                uint32_t out0 = 0, out1 = 0;
#pragma unroll
                for (int cc = 0; cc < 8; cc++) {
                    const uint32_t v = tap8(ta, tb, fx, win4(o, cc), win4(o, cc + 4));
                    if (cc < 4) out0 |= v << (8 * cc); else out1 |= v << (8 * (cc - 4));
                }
                uint32_t *hrow = reinterpret_cast<uint32_t *>(hb + (q * 15 + hr) * 8);
                hrow[0] = out0;
                hrow[1] = out1;
            }
        }
    }
    __syncwarp();
    if (c < nchunks && k < lh) {
        uint32_t o0 = 0x80808080u, o1 = 0x80808080u;           /* missing reference: 128 */
        if (rp) {
            o0 = o1 = 0;
            /* rows k..k+7 of the filtered window, transposed four by four
             * so that a column's taps meet as one word */
            const uint2 *hrows = reinterpret_cast<const uint2 *>(hb + (q * 15 + k) * 8);
            uint32_t lo[8], hi[8];
#pragma unroll
            for (int tt = 0; tt < 8; tt++) {
                const uint2 v = hrows[tt];
                lo[tt] = v.x;
                hi[tt] = v.y;
            }
            const uint32_t va = c_subpel_pk[fy][0], vb = c_subpel_pk[fy][1];
#pragma unroll
            for (int half = 0; half < 2; half++) {
                const uint32_t *rw8 = half ? hi : lo;
                uint32_t ca[4], cb[4];
                tr4(rw8[0], rw8[1], rw8[2], rw8[3], ca);
                tr4(rw8[4], rw8[5], rw8[6], rw8[7], cb);
                uint32_t word = 0;
#pragma unroll
                for (int j = 0; j < 4; j++) word |= tap8(va, vb, fy, ca[j], cb[j]) << (8 * j);
                if (half) o1 = word; else o0 = word;
            }
        }
        uint8_t *d = D.y + (ly0 + k) * D.py + lx0;
        if (lw == 8 && !((uintptr_t)d & 3)) {
            reinterpret_cast<uint32_t *>(d)[0] = o0;
            reinterpret_cast<uint32_t *>(d)[1] = o1;
        } else {
#pragma unroll
            for (int x = 0; x < 8; x++) if (x < lw) d[x] = (uint8_t)((x < 4 ? o0 : o1) >> (8 * (x & 3)));
        }
    }
    __syncwarp();
}

/* Chroma prediction of four chunks, both planes: lane = (chunk c0 + lane/8,
 * plane, r = lane%4); the chroma MV is read as 1/16 chroma pel (16 phases),
 * fetches clamp into the ceil-half planes. */
template <class S>
__device__ void spec_chroma_pass(S &w, const PredDst &D, const cvp9_job_t &job, int c0, int nchunks, int sbx, int sby,
                                 int lane)
{
    uint8_t *hb = reinterpret_cast<uint8_t *>(w.coef) + 480;  /* 4 chunks x 2 planes x 11 rows x 4 */
    const int q = lane >> 3, p = (lane >> 2) & 1, r = lane & 3, c = c0 + q;
    FastBlk fb;
    int lx0, ly0, lw, lh, cx0 = 0, cy0 = 0, clw = 0, clh = 0;
    const uint8_t *pl = nullptr;
    int cw2 = 0, ch2 = 0, rcs = 0, fx = 0, fy = 0, bx = 0, by = 0;
    if (c < nchunks) {
        fast_chunk(w, c, fb, lx0, ly0, lw, lh, cx0, cy0, clw, clh);
        const cvp9_ref_t &R = job.ref[job.ref_slot_of[fb_slot(fb) & 3] & 7];
        if (R.plane && clw > 0) {
            const int rw = R.w, rh = R.h;
            rcs = (rw + 1) >> 1;
            cw2 = rcs;
            ch2 = (rh + 1) >> 1;
            pl = R.plane + (size_t)rw * rh + (p ? (size_t)rcs * ch2 : 0);
            const int mvx = (int16_t)(fb.mv & 0xffffu), mvy = (int16_t)(fb.mv >> 16);
            bx = (sbx >> 1) + cx0 + (mvx >> 4);
            by = (sby >> 1) + cy0 + (mvy >> 4);
            fx = mvx & 15;
            fy = mvy & 15;
            const uint32_t ta = c_subpel_pk[fx][0], tb = c_subpel_pk[fx][1];
#pragma unroll
            for (int h = 0; h < 3; h++) {
                const int hr = r + 4 * h;
                if (hr >= clh + 7) continue;
                const int y = by - 3 + hr, x0 = bx - 3;
                uint32_t o[4];
                /* a further chroma row exists below: word reads stay inside */
                if (x0 >= 0 && x0 + clw + 6 < cw2 && y >= 0 && y + 1 < ch2) ld16w(pl + (size_t)y * rcs + x0, o);
                else ld16c(pl, rcs, cw2, ch2, x0, y, o);
                uint32_t out = 0;
#pragma unroll
                for (int cc = 0; cc < 4; cc++) out |= tap8(ta, tb, fx, win4(o, cc), win4(o, cc + 4)) << (8 * cc);
                *reinterpret_cast<uint32_t *>(hb + ((q * 2 + p) * 11 + hr) * 4) = out;
            }
        }
    }
    __syncwarp();
    if (c < nchunks && clw > 0 && r < clh) {
        uint32_t o = 0x80808080u;                             /* missing reference: 128 */
        if (pl) {
            o = 0;
            const uint32_t *hrows = reinterpret_cast<const uint32_t *>(hb + ((q * 2 + p) * 11 + r) * 4);
            uint32_t ca[4], cb[4];
            tr4(hrows[0], hrows[1], hrows[2], hrows[3], ca);
            tr4(hrows[4], hrows[5], hrows[6], hrows[7], cb);
            const uint32_t va = c_subpel_pk[fy][0], vb = c_subpel_pk[fy][1];
#pragma unroll
            for (int j = 0; j < 4; j++) o |= tap8(va, vb, fy, ca[j], cb[j]) << (8 * j);
        }
        uint8_t *d = (p ? D.v : D.u) + (cy0 + r) * D.pc + cx0;
        if (clw == 4 && !((uintptr_t)d & 3)) {
            *reinterpret_cast<uint32_t *>(d) = o;
        } else {
#pragma unroll
            for (int x = 0; x < 4; x++) if (x < clw) d[x] = (uint8_t)(o >> (8 * x));
        }
    }
    __syncwarp();
}

/* SPEC TX layout of a block in plane p (vp9_kf_tile.c:320-396 for blocks of
 * 8x8 and up): TX log2 size, TXs per row and column (MI-clipped), plane
 * origin in the SB tile, coefficients before this plane. */
struct SpecTx {
    int txl, nx, ny, ox, oy;
    uint64_t base;
};

__device__ __forceinline__ SpecTx spec_tx_layout(const FastBlk &b, int p)
{
    SpecTx s;
    const int l_nx = (int)(b.ext & 0x1fu), l_ny = (int)((b.ext >> 5) & 0x1fu);
    const int c_nx = (int)((b.ext >> 10) & 0xfu), c_ny = (int)((b.ext >> 14) & 0xfu);
    const int ltx = fb_txl(b), ctx = (int)((b.ext >> 18) & 3u);
    const int lc = l_nx * l_ny * (16 << (2 * ltx)), cc = c_nx * c_ny * (16 << (2 * ctx));
    if (p == 0) { s.txl = ltx; s.nx = l_nx; s.ny = l_ny; s.ox = fb_x(b); s.oy = fb_y(b); s.base = 0; }
    else { s.txl = ctx; s.nx = c_nx; s.ny = c_ny; s.ox = fb_x(b) >> 1; s.oy = fb_y(b) >> 1;
           s.base = (uint64_t)lc + (p == 2 ? (uint64_t)cc : 0); }
    return s;
}

/* SPEC residual of every TX of size N in plane P: 32/N TXs at a time.
 * Column pass, lane = (TX, column j): dequantise (DC step at [0][0] only),
 * 1-D butterfly down the column (vp9_idct.comp.glsl:666-679); the group's
 * int32 column results replace its staged coefficients in shared memory;
 * row pass, lane = (TX, row i): butterfly along the row, final shift 4/5/6,
 * add and clamp into the tile (:680-789). A group with no nonzero
 * coefficient adds nothing and is skipped. */
template <int N, bool GLOBAL, class S>
__device__ void spec_fast_residual(S &w, const PredDst &D, const cvp9_job_t &job, int P, int ntx, int lane)
{
    constexpr int G = 32 / N, NN = N * N;
    const int g = lane / N, i = lane % N;
    int16_t *X = w.coef + g * NN;
    int32_t *T = reinterpret_cast<int32_t *>(w.coef) + g * NN;
    uint8_t *tile = P == 0 ? D.y : (P == 1 ? D.u : D.v);
    const int pitch = P == 0 ? D.py : D.pc;
    const int sh = N == 4 ? 4 : (N == 8 ? 5 : 6);
    for (int q0 = 0; q0 < ntx; q0 += G) {
        const int q = q0 + g;
        bool have = q < ntx;
        int px0 = 0, py0 = 0;
        if (have) {
            const int b = w.txblk[q];
            const FastBlk fb = w.blk[b];
            const SpecTx L = spec_tx_layout(fb, P);
            const int tq = q - w.txoff[b];
            const int tyy = L.nx == 1 ? tq : tq / L.nx, txx = tq - tyy * L.nx;
            px0 = L.ox + txx * N;
            py0 = L.oy + tyy * N;
            const uint64_t c0 = (uint64_t)fb.coeff + L.base + (uint64_t)tq * NN;
            if (c0 + NN > (uint64_t)job.num_coeffs) have = false;
            else {
                uint32_t rv[N / 2];
                fast_row_load<N>(rv, job.coeffs + c0 + (uint64_t)i * N);
                uint32_t *dst = reinterpret_cast<uint32_t *>(X + i * N);
#pragma unroll
                for (int k = 0; k < N / 2; k++) dst[k] = rv[k];
            }
        }
        __syncwarp();
        wi v[N];
        bool any = false;
        if (have) {
#pragma unroll
            for (int k = 0; k < N; k++) {
                const int cf = X[k * N + i];
                any |= cf != 0;
                v[k] = wi(cf) * ((k == 0 && i == 0) ? job.q_dc : job.q_ac);
            }
            if (any) idct_n(v, N);
        }
        const bool grp_any = __any_sync(0xffffffffu, any);
        __syncwarp();                          /* every lane has read its column */
        if (grp_any) {
            if (have) {
#pragma unroll
                for (int k = 0; k < N; k++) T[k * N + i] = any ? v[k].v : 0;
            }
            __syncwarp();
            if (have) {
#pragma unroll
                for (int k = 0; k < N; k++) v[k] = wi(T[i * N + k]);
                idct_n(v, N);
                uint8_t *rowp = tile + (py0 + i) * pitch + px0;
                const int vw = P == 0 ? D.vw : D.cvw, vh = P == 0 ? D.vh : D.cvh;
                const int xin = vw - px0;            /* samples of the row inside the frame */
                const bool rowin = py0 + i < vh;
                const bool words = (!GLOBAL || !((uintptr_t)rowp & 3)) && xin >= N;
#pragma unroll
                for (int j4 = 0; j4 < N / 4; j4++) {
                    if (!rowin || 4 * j4 >= xin) continue;
                    uint32_t word;
                    if (words) {
                        word = reinterpret_cast<const uint32_t *>(rowp)[j4];
                    } else {
                        word = 0;
#pragma unroll
                        for (int e = 0; e < 4; e++)
                            if (4 * j4 + e < xin) word |= (uint32_t)rowp[4 * j4 + e] << (8 * e);
                    }
                    uint32_t outw = 0;
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const int r = ((int)((unsigned)v[j4 * 4 + e].v + (1u << (sh - 1)))) >> sh;
                        outw |= (uint32_t)clampi((int)((word >> (8 * e)) & 0xffu) + r, 0, 255) << (8 * e);
                    }
                    if (words) {
                        reinterpret_cast<uint32_t *>(rowp)[j4] = outw;
                    } else {
#pragma unroll
                        for (int e = 0; e < 4; e++)
                            if (4 * j4 + e < xin) rowp[4 * j4 + e] = (uint8_t)(outw >> (8 * e));
                    }
                }
            }
        }
        __syncwarp();
    }
}

} /* namespace */

/* Steps 1-2 of a superblock on the warp-per-SB paths: load, check and pack
 * its block descriptors (w.blk), check that they tile the visible SB exactly
 * (4x4-cell occupancy in w.cells), and map its 8x8 prediction chunks
 * (w.choff, w.chblk). Returns the number of chunks, or -1 when the SB
 * belongs to the general kernel (intra, malformed, odd layouts). nb_out: the
 * SB's block count. CHECK = false: only load and pack the descriptors (a
 * second kernel on an SB the first one already took; returns 0). */
template <int A, bool CHECK = true, class S>
__device__ int fast_sb_setup(S &w, const cvp9_job_t &job, int sb, int sbx, int sby, int lane, int &nb_out)
{
    const int W = job.W, H = job.H;
    const uint32_t *rg = job.sb_range + 4 * sb;
    const uint32_t start = rg[0], end = rg[1], groups = rg[2];
    bool gen = groups != 1 || end < start || end > job.num_blocks || end - start > 64u ||
               (*job.status & CVP9_JOB_BAD_BLOCK) != 0;
    const int nb = gen ? 0 : (int)(end - start);
    nb_out = nb;

    /* 1. blocks: load, check, pack; 4x4-cell occupancy */
    if (CHECK) {
        if (lane < 8) w.cells[lane] = 0u;
        __syncwarp();
    }
    bool bad = false, ovl = false;
    int nch[2] = { 0, 0 };
#pragma unroll
    for (int r = 0; r < 2; r++) {
        const int i = lane + 32 * r;
        if (i >= nb) continue;
        const uint32_t *g = reinterpret_cast<const uint32_t *>(job.blocks + start + i);
        const uint32_t g0 = __ldg(g), g1 = __ldg(g + 1), g2 = __ldg(g + 2), g3 = __ldg(g + 3);
        const uint32_t g5 = __ldg(g + 5), g6 = __ldg(g + 6);
        const int gx = (int)(g0 & 0xffffu), gy = (int)(g0 >> 16);
        const int bw = (int)(g1 & 0xffu), bh = (int)((g1 >> 8) & 0xffu);
        const int txl = (int)((g1 >> 16) & 0xffu), intra = (int)(g1 >> 24);
        const int ref0 = (int)((g2 >> 16) & 0xffu), skip = (int)(g5 & 0xffu);
        const int lx = gx - sbx, ly = gy - sby;
        const bool mb = lx < 0 || ly < 0 || (lx & 3) || (ly & 3) || (bw & 3) || (bh & 3) ||
                        bw < 4 || bh < 4 || lx + bw > 64 || ly + bh > 64 || gx >= W || gy >= H || txl > 3 ||
                        ((bw < 8 || bh < 8) && ((lx & 7) || (ly & 7)));
        bad |= mb || intra;
        if (mb) continue;
        const int cw = min(bw, W - gx), ch = min(bh, H - gy);
        FastBlk fb;
        uint32_t slot4 = (ref0 >= 1 && ref0 <= 8) ? (uint32_t)(ref0 - 1) : 15u;
        fb.ext = 0u;
        if (A == CVP9_ARITH_SPEC) {
            /* sub-8x8 residuals span their whole 8x8 MI (they overlap), and
             * 32x32 TXs need more staging than a warp has: general path */
            slot4 = (uint32_t)clampi(ref0 - 1, 0, 2);
            int uvtx = min(txl, max_tx_for(max(bw / 2, 4), max(bh / 2, 4)));
            /* the fast path keeps every TX inside its block and its rows
             * word-aligned: MI-aligned power-of-two blocks, TX <= block */
            bad |= bw < 8 || bh < 8 || txl == 3 || uvtx == 3 || (lx & 7) || (ly & 7) ||
                   (bw & (bw - 1)) || (bh & (bh - 1)) || (4 << txl) > min(bw, bh);
            if (!skip) {
                int nxy[2][2];
#pragma unroll
                for (int pp = 0; pp < 2; pp++) {
                    const int t4 = 1 << (pp ? uvtx : txl);
                    const int pw = max(pp ? bw / 2 : bw, 4), ph = max(pp ? bh / 2 : bh, 4);
                    const int o4x = ((gx >> 3) * 2) >> pp, o4y = ((gy >> 3) * 2) >> pp;
                    const int mw = min(pw / 4, ((job.mi_cols * 2) >> pp) - o4x);
                    const int mh = min(ph / 4, ((job.mi_rows * 2) >> pp) - o4y);
                    nxy[pp][0] = mw > 0 ? (mw + t4 - 1) / t4 : 0;
                    nxy[pp][1] = mh > 0 ? (mh + t4 - 1) / t4 : 0;
                }
                fb.ext = (uint32_t)nxy[0][0] | (uint32_t)nxy[0][1] << 5 | (uint32_t)nxy[1][0] << 10 |
                         (uint32_t)nxy[1][1] << 14 | (uint32_t)uvtx << 18;
            }
        }
        fb.geo = (uint32_t)(lx >> 2) | (uint32_t)(ly >> 2) << 4 | (uint32_t)cw << 8 | (uint32_t)ch << 15 |
                 slot4 << 22 | (uint32_t)txl << 26 | (skip ? 1u : 0u) << 28;
        fb.mv = g3;
        fb.coeff = g6;
        w.blk[i] = fb;
        if (!CHECK) continue;
        nch[r] = ((cw + 7) >> 3) * ((ch + 7) >> 3);
        const int c0x = lx >> 2, c1x = (lx + cw - 1) >> 2, c0y = ly >> 2, c1y = (ly + ch - 1) >> 2;
        const uint32_t m = (2u << c1x) - (1u << c0x);
        for (int cy = c0y; cy <= c1y; cy++) {
            const uint32_t mm = m << (16 * (cy & 1));
            ovl |= (atomicOr(&w.cells[cy >> 1], mm) & mm) != 0u;
        }
    }
    __syncwarp();
    if (!CHECK) return 0;
    const int vw = min(64, W - sbx), vh = min(64, H - sby);
    bool gap = false;
    if (lane < 8) {
        const int ncx = (vw + 3) >> 2, ncy = (vh + 3) >> 2;
        const uint32_t rowm = ncx >= 16 ? 0xffffu : ((1u << ncx) - 1u);
        const uint32_t expect = (2 * lane < ncy ? rowm : 0u) | (2 * lane + 1 < ncy ? rowm << 16 : 0u);
        gap = w.cells[lane] != expect;
    }
    gen = __any_sync(0xffffffffu, gen || bad || ovl || gap) != 0;
    if (gen) return -1;

    /* 2. chunk (8x8 luma + 4x4 chroma) offsets and map */
    int nchunks;
    {
        const int x0 = warp_incl_scan(nch[0], lane), x1 = warp_incl_scan(nch[1], lane);
        const int tot0 = __shfl_sync(0xffffffffu, x0, 31), tot1 = __shfl_sync(0xffffffffu, x1, 31);
        nchunks = tot0 + tot1;
        if (nchunks > 128) return -1;   /* more chunks than the map holds (odd block sizes) */
        const int e0 = x0 - nch[0], e1 = tot0 + x1 - nch[1];
        if (lane < nb) { w.choff[lane] = (uint16_t)e0; for (int c = 0; c < nch[0]; c++) w.chblk[e0 + c] = (uint8_t)lane; }
        if (lane + 32 < nb) { w.choff[lane + 32] = (uint16_t)e1; for (int c = 0; c < nch[1]; c++) w.chblk[e1 + c] = (uint8_t)(lane + 32); }
    }
    __syncwarp();
    return nchunks;
}

/* REFCPU luma residual of a set-up superblock (fast_sb_setup): one pass
 * per TX size present, TXs counted on the frame-clamped block
 * (vp9_reconstruct.c:338-340), added to the predicted rows at dst. U8: 8x8
 * TXs through fast_residual_d, each TX walking its own nonzero columns
 * (measured faster on both 8x8-only and mixed content; an unrolled
 * union-of-columns form, tried before it, cut instructions on 8x8 content
 * but its code size cost more on mixed TX sizes). */
template <bool GLOBAL, bool U8, class S, bool ONLY8 = false>
__device__ void fast_refcpu_residual(S &w, uint8_t *dst, int pitch, const cvp9_job_t &job, int nb, int lane)
{
    unsigned sizes = 0;
#pragma unroll
    for (int r = 0; r < 2; r++) {
        const int i = lane + 32 * r;
        if (i < nb && !fb_skip(w.blk[i])) sizes |= 1u << fb_txl(w.blk[i]);
    }
    sizes = __reduce_or_sync(0xffffffffu, sizes);
    for (unsigned sz = sizes; sz; sz &= sz - 1) {
        const int txl = __ffs(sz) - 1, n = 4 << txl;
        int cnt[2] = { 0, 0 };
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const int i = lane + 32 * r;
            if (i < nb) {
                const FastBlk fb = w.blk[i];
                if (!fb_skip(fb) && fb_txl(fb) == txl) cnt[r] = (fb_cw(fb) / n) * (fb_ch(fb) / n);
            }
        }
        const int x0 = warp_incl_scan(cnt[0], lane), x1 = warp_incl_scan(cnt[1], lane);
        const int tot0 = __shfl_sync(0xffffffffu, x0, 31), tot1 = __shfl_sync(0xffffffffu, x1, 31);
        const int e0 = x0 - cnt[0], e1 = tot0 + x1 - cnt[1];
        const int ntx = tot0 + tot1;        /* at most 256: the TXs tile the SB's luma */
        if (lane < nb) { w.txoff[lane] = (uint16_t)e0; for (int c = 0; c < cnt[0]; c++) w.txblk[e0 + c] = (uint8_t)lane; }
        if (lane + 32 < nb) { w.txoff[lane + 32] = (uint16_t)e1; for (int c = 0; c < cnt[1]; c++) w.txblk[e1 + c] = (uint8_t)(lane + 32); }
        __syncwarp();
        if (ONLY8) {
            /* the caller took superblocks whose TXs are all 8x8 */
            fast_residual_d<8, GLOBAL>(w, dst, pitch, job, ntx, lane);
        } else {
            switch (txl) {
            case 0: fast_residual<4, GLOBAL>(w, dst, pitch, job, ntx, lane); break;
            case 1:
                if (U8) fast_residual_d<8, GLOBAL>(w, dst, pitch, job, ntx, lane);
                else fast_residual<8, GLOBAL>(w, dst, pitch, job, ntx, lane);
                break;
            case 2: fast_residual<16, GLOBAL>(w, dst, pitch, job, ntx, lane); break;
            default: fast_residual<32, GLOBAL>(w, dst, pitch, job, ntx, lane); break;
            }
        }
        __syncwarp();
    }
}

/* SPEC residual of a set-up superblock: one pass per (plane, TX size)
 * present, every plane in the tile parser's MI-clipped layout, added to the
 * predicted planes at D. */
template <bool GLOBAL, class S>
__device__ void fast_spec_residual(S &w, const PredDst &D, const cvp9_job_t &job, int nb, int lane)
{
    for (int P = 0; P < 3; P++) {
        unsigned sizes = 0;
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const int i = lane + 32 * r;
            if (i < nb && !fb_skip(w.blk[i])) sizes |= 1u << spec_tx_layout(w.blk[i], P).txl;
        }
        sizes = __reduce_or_sync(0xffffffffu, sizes);
        for (unsigned sz = sizes; sz; sz &= sz - 1) {
            const int txl = __ffs(sz) - 1;
            int cnt[2] = { 0, 0 };
#pragma unroll
            for (int r = 0; r < 2; r++) {
                const int i = lane + 32 * r;
                if (i < nb) {
                    const FastBlk fb = w.blk[i];
                    if (fb_skip(fb)) continue;
                    const SpecTx L = spec_tx_layout(fb, P);
                    if (L.txl == txl) cnt[r] = L.nx * L.ny;
                }
            }
            const int x0 = warp_incl_scan(cnt[0], lane), x1 = warp_incl_scan(cnt[1], lane);
            const int tot0 = __shfl_sync(0xffffffffu, x0, 31), tot1 = __shfl_sync(0xffffffffu, x1, 31);
            const int e0 = x0 - cnt[0], e1 = tot0 + x1 - cnt[1];
            const int ntx = tot0 + tot1;    /* at most 256: the TXs tile the SB's plane */
            if (lane < nb) { w.txoff[lane] = (uint16_t)e0; for (int c = 0; c < cnt[0]; c++) w.txblk[e0 + c] = (uint8_t)lane; }
            if (lane + 32 < nb) { w.txoff[lane + 32] = (uint16_t)e1; for (int c = 0; c < cnt[1]; c++) w.txblk[e1 + c] = (uint8_t)(lane + 32); }
            __syncwarp();
            switch (txl) {
            case 0: spec_fast_residual<4, GLOBAL>(w, D, job, P, ntx, lane); break;
            case 1: spec_fast_residual<8, GLOBAL>(w, D, job, P, ntx, lane); break;
            default: spec_fast_residual<16, GLOBAL>(w, D, job, P, ntx, lane); break;   /* 32 went general */
            }
            __syncwarp();
        }
    }
}

/* MINB: CTAs per SM the register allocation is sized for (5: up to 96
 * registers, no spills; 6: 80 registers, a few spilled). */
template <int A, int MINB>
__global__ void __launch_bounds__(kFastWarps * 32, MINB) k_inter(const cvp9_job_t *__restrict__ jobs,
                                                            const uint32_t *__restrict__ tickets,
                                                            uint32_t n_tickets, uint32_t *__restrict__ general)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    FastSmem &w = reinterpret_cast<FastSmem *>(smem_raw)[warp];
    const uint32_t t = blockIdx.x * kFastWarps + warp;
    if (t >= n_tickets) return;
    const uint32_t code = __ldg(tickets + t);
    const cvp9_job_t &job = jobs[code >> 20];
    const int sb = (int)(code & 0xFFFFFu);
    const int sb_cols = job.sb_cols;
    const int sbr = sb / sb_cols, sbc = sb - sbr * sb_cols;
    const int sbx = sbc * 64, sby = sbr * 64;
    const int W = job.W, H = job.H;
    int nb;
    int nchunks = fast_sb_setup<A>(w, job, sb, sbx, sby, lane, nb);
    if (lane == 0) general[t] = nchunks < 0 ? 1u : 0u;
    if (nchunks < 0) {
        if (lane == 0) atomicAdd(general + 2 * n_tickets + 1, 1u);   /* k_compact skips when 0 */
        return;
    }

    /* 3. prediction (vp9_reconstruct.c:94-131). Luma passes: lane = (chunk
     * c0 + lane/8, row lane%8); chroma passes: lane = (chunk c0 + lane/8,
     * plane, row). Two luma and two chroma passes are in flight: all four
     * issue their loads before any computes. */
    if (A == CVP9_ARITH_SPEC) {
        const PredDst DS = { w.ty, w.tu, w.tv, kFY, kFC, 64, 64, 32, 32 };
        for (int c0 = 0; c0 < nchunks; c0 += 4) spec_luma_pass(w, DS, job, c0, nchunks, sbx, sby, lane);
        for (int c0 = 0; c0 < nchunks; c0 += 4) spec_chroma_pass(w, DS, job, c0, nchunks, sbx, sby, lane);
        nchunks = 0;                      /* the REFCPU passes below do nothing */
    }
    for (int c0 = 0; c0 < nchunks; c0 += 8) {
        FastLuma a, b;
        FastChroma ca, cb;
        const PredDst D = { w.ty, w.tu, w.tv, kFY, kFC, 64, 64, 32, 32 };
        fast_pred_issue(w, D, job, c0 + (lane >> 3), lane, nchunks, sbx, sby, a, ca);
        fast_pred_issue(w, D, job, c0 + 4 + (lane >> 3), lane, nchunks, sbx, sby, b, cb);
        fast_luma_finish(a);
        fast_luma_finish(b);
        fast_chroma_finish(ca);
        fast_chroma_finish(cb);
    }
    __syncwarp();

    /* 4. residual, one pass per (plane, TX size) present: REFCPU luma only
     * with TXs counted on the frame-clamped block; SPEC every plane in the
     * tile parser's MI-clipped layout */
    if (A == CVP9_ARITH_REFCPU) fast_refcpu_residual<false, false>(w, w.ty, kFY, job, nb, lane);
    if (A == CVP9_ARITH_SPEC) {
        const PredDst D = { w.ty, w.tu, w.tv, kFY, kFC, 64, 64, 32, 32 };
        fast_spec_residual<false>(w, D, job, nb, lane);
    }

    /* 5. write the tile (clipped to the frame) and release the SB */
    {
        const int vw = min(64, W - sbx), vh = min(64, H - sby);
        uint8_t *Y = job.out;
        if (!(W & 15) && !((uintptr_t)Y & 15)) {
            for (int i = lane; i < vh * 4; i += 32) {
                const int r = i >> 2, c16 = (i & 3) * 16;
                if (c16 < vw)
                    *reinterpret_cast<uint4 *>(Y + (size_t)(sby + r) * W + sbx + c16) =
                        ld_smem16(w.ty + r * kFY + c16);
            }
        } else if (!(W & 3) && !((uintptr_t)Y & 3)) {
            for (int i = lane; i < vh * 16; i += 32) {
                const int r = i >> 4, c4 = (i & 15) * 4;
                if (c4 < vw)
                    *reinterpret_cast<uint32_t *>(Y + (size_t)(sby + r) * W + sbx + c4) =
                        *reinterpret_cast<const uint32_t *>(w.ty + r * kFY + c4);
            }
        } else {
            for (int i = lane; i < vh * 64; i += 32) {
                const int r = i >> 6, c = i & 63;
                if (c < vw) Y[(size_t)(sby + r) * W + sbx + c] = w.ty[r * kFY + c];
            }
        }
        const int CW = job.CW, CH = job.CH;
        const int cvw = min(32, CW - (sbx >> 1)), cvh = min(32, CH - (sby >> 1));
        uint8_t *U = Y + (size_t)W * H;
        uint8_t *V = U + (size_t)CW * CH;
        if (!(CW & 15) && !((uintptr_t)U & 15) && !((uintptr_t)V & 15)) {
            for (int i = lane; i < 2 * cvh * 2; i += 32) {
                const int p = i >= cvh * 2, k = p ? i - cvh * 2 : i;
                const int r = k >> 1, c16 = (k & 1) * 16;
                if (c16 < cvw)
                    *reinterpret_cast<uint4 *>((p ? V : U) + (size_t)((sby >> 1) + r) * CW + (sbx >> 1) + c16) =
                        ld_smem16((p ? w.tv : w.tu) + r * kFC + c16);
            }
        } else if (!(CW & 3) && !((uintptr_t)U & 3) && !((uintptr_t)V & 3)) {
            for (int i = lane; i < 2 * cvh * 8; i += 32) {
                const int p = i >= cvh * 8, k = p ? i - cvh * 8 : i;
                const int r = k >> 3, c4 = (k & 7) * 4;
                if (c4 < cvw)
                    *reinterpret_cast<uint32_t *>((p ? V : U) + (size_t)((sby >> 1) + r) * CW + (sbx >> 1) + c4) =
                        *reinterpret_cast<const uint32_t *>((p ? w.tv : w.tu) + r * kFC + c4);
            }
        } else {
            for (int i = lane; i < 2 * cvh * 32; i += 32) {
                const int p = i >= cvh * 32, k = p ? i - cvh * 32 : i;
                const int r = k >> 5, c = k & 31;
                if (c < cvw) (p ? V : U)[(size_t)((sby >> 1) + r) * CW + (sbx >> 1) + c] = (p ? w.tv : w.tu)[r * kFC + c];
            }
        }
    }
    __syncwarp();
    if (lane == 0) {
        __threadfence();
        st_release(job.sb_done + sb, job.epoch);
    }
}

/* ── Prediction with its reads one pass ahead (k_pred) ──────────────────
 * The passes of fast_pred_issue / fast_*_finish, but each lane's reference
 * rows go to a shared-memory slot by cp.async, and the next iteration's
 * rows are requested before the current one is filtered, so a warp has two
 * iterations' reads in flight instead of waiting on each. A lane's slot:
 * its luma row (16 bytes around the 9 it needs), the row below (the chunk's
 * last lane only), its chroma row (8 bytes around 5) and the row below
 * (the plane's last lane only). The rows below of the other lanes are their
 * neighbours' rows, read from the neighbour's slot. Rows that need clamped
 * samples are read at once, byte by byte, and stored already extracted. */
constexpr int kSlot = 48, kSlotLB = 16, kSlotCA = 32, kSlotCB = 40;

struct PredGeo {                 /* one lane's pass: what the filter step needs */
    uint8_t *dl, *dc;            /* luma / chroma destination (frame) */
    uint32_t fl;                 /* lw | fx << 4 | fy << 7 | act << 10 | ref << 11 | o0 << 12 | o1 << 15 */
    uint32_t fc;                 /* clw | fx << 3 | fy << 6 | act << 9 | ref << 10 | o0 << 11 | o1 << 13 */
};

/* 9 bytes at offset o (0..7) of the 16 at q (shared memory, 16-byte aligned) */
__device__ __forceinline__ void slot9(const uint8_t *q, unsigned o, uint32_t &lo, uint32_t &mid, uint32_t &hi)
{
    const uint4 v = *reinterpret_cast<const uint4 *>(q);
    const bool up = o >= 4;
    const unsigned sh = 8u * (o & 3u);
    const uint32_t w0 = up ? v.y : v.x, w1 = up ? v.z : v.y, w2 = up ? v.w : v.z;
    lo = __funnelshift_r(w0, w1, sh);
    mid = __funnelshift_r(w1, w2, sh);
    hi = w2 >> sh;
}

/* 5 bytes at offset o (0..3) of the 8 at q (shared memory, 8-byte aligned) */
__device__ __forceinline__ void slot5(const uint8_t *q, unsigned o, uint32_t &lo, uint32_t &hi)
{
    const uint2 v = *reinterpret_cast<const uint2 *>(q);
    const unsigned sh = 8u * o;
    lo = __funnelshift_r(v.x, v.y, sh);
    hi = v.y >> sh;
}

/* Geometry of chunk c for this lane (as fast_pred_issue) and its row reads,
 * into slot (this lane's, this pass's). */
template <class S>
__device__ __forceinline__ void pred_request(const S &w, const PredDst &D, const cvp9_job_t &job, int c, int lane,
                                             int nchunks, int sbx, int sby, uint8_t *slot, PredGeo &G)
{
    G.fl = 0u;
    G.fc = 0u;
    if (c >= nchunks) return;
    const int kk = lane & 7, p = (lane >> 2) & 1, r = lane & 3;
    FastBlk fb;
    int lx0, ly0, lw, lh, cx0, cy0, clw, clh;
    fast_chunk(w, c, fb, lx0, ly0, lw, lh, cx0, cy0, clw, clh);
    const int slotr = fb_slot(fb);
    const uint8_t *rp = nullptr;
    int rw = 0, rh = 0;
    if (slotr < 8) {
        const cvp9_ref_t &R = job.ref[slotr];
        rp = R.plane;
        rw = R.w;
        rh = R.h;
    }
    const int mvx = (int16_t)(fb.mv & 0xffffu), mvy = (int16_t)(fb.mv >> 16);
    G.dl = D.y + (ly0 + kk) * D.py + lx0;
    G.dc = (p ? D.v : D.u) + (cy0 + r) * D.pc + cx0;
    uint32_t fl = (uint32_t)lw | (kk < lh ? 1u << 10 : 0u);
    uint32_t fc = (uint32_t)max(clw, 0) | (r < clh && clw > 0 ? 1u << 9 : 0u);
    if (rp) {
        const int px8 = (sbx + lx0) * 8 + mvx, py8 = (sby + ly0) * 8 + mvy;
        const int ix = px8 >> 3, y0 = (py8 >> 3) + kk;
        fl |= (uint32_t)(px8 & 7) << 4 | (uint32_t)(py8 & 7) << 7 | 1u << 11;
        /* luma rows are followed by the chroma planes: 16-byte reads past a
         * row end stay inside the frame; the plane starts 8-byte aligned */
        const bool hin = ix >= 0 && ix + lw < rw && rw >= 16;   /* 16-byte reads stay in the frame */
#pragma unroll
        for (int e = 0; e < 2; e++) {
            if (e == 1 && kk != 7) break;            /* the row below: the chunk's last lane */
            const int y = y0 + e;
            uint8_t *dst = slot + (e ? kSlotLB : 0);
            if (hin && y >= 0 && y < rh) {
                const uint8_t *a = rp + (size_t)y * rw + ix;
                const uint8_t *a8 = reinterpret_cast<const uint8_t *>((uintptr_t)a & ~(uintptr_t)7);
                cp_async8(dst, a8);
                cp_async8(dst + 8, a8 + 8);
                fl |= (uint32_t)((uintptr_t)a & 7) << (12 + 3 * e);
            } else {
                uint32_t lo, mid, hi;
                ld9c(rp, rw, rh, ix, y, lo, mid, hi);
                *reinterpret_cast<uint4 *>(dst) = make_uint4(lo, mid, hi, 0u);
            }
        }
        /* the row below of the other lanes is their neighbour's row: the
         * filter step needs its offset, from the same column and y0 + 1 */
        if (kk != 7 && hin && y0 + 1 >= 0 && y0 + 1 < rh)
            fl |= (uint32_t)(((uintptr_t)rp + (size_t)(y0 + 1) * rw + ix) & 7) << 15;
        if (clw > 0) {
            const int rcs = (rw + 1) >> 1, crw = rw >> 1, crh = rh >> 1;
            const uint8_t *pl = rp + (size_t)rw * rh + (p ? (size_t)rcs * ((rh + 1) >> 1) : 0);
            const int cpx8 = ((sbx >> 1) + cx0) * 8 + mvx / 2, cpy8 = ((sby >> 1) + cy0) * 8 + mvy / 2;
            const int cix = cpx8 >> 3, y1 = (cpy8 >> 3) + r;
            fc |= (uint32_t)(cpx8 & 7) << 3 | (uint32_t)(cpy8 & 7) << 6 | 1u << 10;
            /* a further chroma row below the one read: reads stay inside */
            const bool chin = cix >= 0 && cix + clw < crw && rcs >= 8;   /* 8-byte reads stay in the plane */
#pragma unroll
            for (int e = 0; e < 2; e++) {
                if (e == 1 && r != 3) break;         /* the row below: the plane's last lane */
                const int y = y1 + e;
                uint8_t *dst = slot + (e ? kSlotCB : kSlotCA);
                if (chin && y >= 0 && y + 1 < crh) {
                    const uint8_t *a = pl + (size_t)y * rcs + cix;
                    const uint8_t *a4 = reinterpret_cast<const uint8_t *>((uintptr_t)a & ~(uintptr_t)3);
                    cp_async4(dst, a4);
                    cp_async4(dst + 4, a4 + 4);
                    fc |= (uint32_t)((uintptr_t)a & 3) << (11 + 2 * e);
                } else {
                    uint32_t lo, hi;
                    ld5c(pl, rcs, crw, crh, cix, y, lo, hi);
                    *reinterpret_cast<uint2 *>(dst) = make_uint2(lo, hi);
                }
            }
            if (r != 3 && chin && y1 + 1 >= 0 && y1 + 2 < crh)
                fc |= (uint32_t)(((uintptr_t)pl + (size_t)(y1 + 1) * rcs + cix) & 3) << 13;
        }
    }
    G.fl = fl;
    G.fc = fc;
}

/* The filter step of a pass whose rows have landed: base is the warp's
 * slots for this pass (lane i at base + i * kSlot). */
__device__ __forceinline__ void pred_filter(const PredGeo &G, const uint8_t *base, int lane)
{
    const int kk = lane & 7, r = lane & 3;
    const uint8_t *own = base + lane * kSlot;
    if (G.fl & (1u << 10)) {
        uint32_t o0 = 0x7f7f7f7fu, o1 = 0x7f7f7f7fu;     /* missing reference: 127 */
        if (G.fl & (1u << 11)) {
            uint32_t lo0, mid0, hi0, lo1, mid1, hi1;
            slot9(own, (G.fl >> 12) & 7u, lo0, mid0, hi0);
            slot9(kk == 7 ? own + kSlotLB : own + kSlot, (G.fl >> 15) & 7u, lo1, mid1, hi1);
            bilinear8(lo0, mid0, hi0, lo1, mid1, hi1, (G.fl >> 4) & 7, (G.fl >> 7) & 7, o0, o1);
        }
        const int lw = G.fl & 15u;
        if (lw == 8 && !((uintptr_t)G.dl & 3)) {
            reinterpret_cast<uint32_t *>(G.dl)[0] = o0;
            reinterpret_cast<uint32_t *>(G.dl)[1] = o1;
        } else {
#pragma unroll
            for (int x = 0; x < 8; x++) if (x < lw) G.dl[x] = (uint8_t)((x < 4 ? o0 : o1) >> (8 * (x & 3)));
        }
    }
    if (G.fc & (1u << 9)) {
        uint32_t o = 0x7f7f7f7fu;
        if (G.fc & (1u << 10)) {
            uint32_t lo0, hi0, lo1, hi1;
            slot5(own + kSlotCA, (G.fc >> 11) & 3u, lo0, hi0);
            slot5(r == 3 ? own + kSlotCB : own + kSlot + kSlotCA, (G.fc >> 13) & 3u, lo1, hi1);
            o = bilinear4(lo0, hi0, lo1, hi1, (G.fc >> 3) & 7, (G.fc >> 6) & 7);
        }
        const int clw = G.fc & 7u;
        if (clw == 4 && !((uintptr_t)G.dc & 3)) {
            *reinterpret_cast<uint32_t *>(G.dc) = o;
        } else {
#pragma unroll
            for (int x = 0; x < 4; x++) if (x < clw) G.dc[x] = (uint8_t)(o >> (8 * x));
        }
    }
}

/* ── REFCPU superblocks in two kernels ──────────────────────────────────
 * k_inter's REFCPU work split in two leaner kernels. k_inter holds a
 * superblock's tiles, its coefficient staging and the transform's registers
 * at once, which caps it at 20 warps per SM; its time follows the warps it
 * keeps resident. k_pred predicts straight into the output frame and marks
 * the general superblocks; k_resid adds the luma residual to the frame in
 * place and releases the superblock. Same operations in the same order as
 * k_inter, so the same bytes; the frame's luma makes one more round trip
 * through L2/HBM. */
struct __align__(16) PredSmem {                   /* k_pred, one per warp */
    union {
        uint8_t stage[2 * 2 * 32 * kSlot];        /* REFCPU: 2 iterations x 2 passes x 32 lane slots */
        int16_t coef[2 * 32 * kSlot];             /* SPEC: the filtered rows of the 8-tap passes */
    };
    FastBlk  blk[64];
    uint32_t cells[8];
    uint16_t choff[65];
    uint8_t  chblk[128];
};

struct __align__(16) ResidSmem {                  /* k_resid, one per warp */
    union {
        int16_t  coef[1056];
        uint32_t cells[8];
    };
    FastBlk  blk[64];
    union {
        struct {
            uint16_t choff[65];
            uint8_t  chblk[128];
        };
        struct {
            uint16_t txoff[65];
            uint8_t  txblk[256];
        };
    };
};

static_assert(sizeof(PredSmem) % 16 == 0 && sizeof(ResidSmem) % 16 == 0, "per-warp areas stay 16-byte aligned");
static_assert(offsetof(ResidSmem, coef) % 16 == 0, "coefficient rows are written as words");

/* CTAs of 4 warps per SM the registers are sized for: prediction at 96
 * registers (20 warps), residual at 64 (32 warps, some spilled); measured
 * best of 5..8 each on 64 x 1080p steps (1.016 ms against 1.028 for 80/64
 * and 1.10 for 80/80). */
constexpr int kPredMinB = 5, kResidMinB = 8, kResid8MinB = 8;

/* MARK (REFCPU inter path 5): a taken superblock with a TX other than 8x8
 * is marked 2 instead of 0, for k_resid's PART 2. */
template <int A, int MINB, bool MARK = false>
__global__ void __launch_bounds__(kFastWarps * 32, MINB) k_pred(const cvp9_job_t *__restrict__ jobs,
                                                           const uint32_t *__restrict__ tickets,
                                                           uint32_t n_tickets, uint32_t *__restrict__ general)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    PredSmem &w = reinterpret_cast<PredSmem *>(smem_raw)[warp];
    const uint32_t t = blockIdx.x * kFastWarps + warp;
    if (t >= n_tickets) return;
    const uint32_t code = __ldg(tickets + t);
    const cvp9_job_t &job = jobs[code >> 20];
    const int sb = (int)(code & 0xFFFFFu);
    const int sbr = sb / job.sb_cols, sbc = sb - sbr * job.sb_cols;
    const int sbx = sbc * 64, sby = sbr * 64;
    int nb;
    const int nchunks = fast_sb_setup<A>(w, job, sb, sbx, sby, lane, nb);
    unsigned mark = 0u;
    if (MARK && nchunks >= 0) {
        unsigned sizes = 0u;
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const int i = lane + 32 * r;
            if (i < nb && !fb_skip(w.blk[i])) sizes |= 1u << fb_txl(w.blk[i]);
        }
        mark = (__reduce_or_sync(0xffffffffu, sizes) & ~2u) ? 2u : 0u;
    }
    if (lane == 0) general[t] = nchunks < 0 ? 1u : mark;
    if (nchunks < 0) {
        if (lane == 0) atomicAdd(general + 2 * n_tickets + 1, 1u);   /* k_compact skips when 0 */
        return;
    }
    const int W = job.W, H = job.H, CW = job.CW, CH = job.CH;
    uint8_t *Y = job.out;
    uint8_t *U = Y + (size_t)W * H;
    uint8_t *V = U + (size_t)CW * CH;
    const size_t coff = (size_t)(sby >> 1) * CW + (sbx >> 1);
    const PredDst D = { Y + (size_t)sby * W + sbx, U + coff, V + coff, W, CW,
                        min(64, W - sbx), min(64, H - sby), min(32, CW - (sbx >> 1)), min(32, CH - (sby >> 1)) };
    if (A == CVP9_ARITH_SPEC) {
        for (int c0 = 0; c0 < nchunks; c0 += 4) spec_luma_pass(w, D, job, c0, nchunks, sbx, sby, lane);
        for (int c0 = 0; c0 < nchunks; c0 += 4) spec_chroma_pass(w, D, job, c0, nchunks, sbx, sby, lane);
        return;
    }
    /* two passes of four chunks per iteration; the next iteration's rows
     * are requested before this one's are filtered */
    const int nit = (nchunks + 7) >> 3;
    auto slots = [&](int st, int pass) { return w.stage + (st * 2 + pass) * 32 * kSlot; };
    PredGeo a, b, na, nx;
    na.fl = na.fc = nx.fl = nx.fc = 0u;
    na.dl = na.dc = nx.dl = nx.dc = nullptr;
    pred_request(w, D, job, lane >> 3, lane, nchunks, sbx, sby, slots(0, 0) + lane * kSlot, a);
    pred_request(w, D, job, 4 + (lane >> 3), lane, nchunks, sbx, sby, slots(0, 1) + lane * kSlot, b);
    cp_async_commit();
    for (int it = 0; it < nit; it++) {
        const int cur = it & 1;
        if (it + 1 < nit) {
            const int c1 = (it + 1) * 8;
            pred_request(w, D, job, c1 + (lane >> 3), lane, nchunks, sbx, sby, slots(cur ^ 1, 0) + lane * kSlot, na);
            pred_request(w, D, job, c1 + 4 + (lane >> 3), lane, nchunks, sbx, sby, slots(cur ^ 1, 1) + lane * kSlot, nx);
            cp_async_commit();
            cp_async_wait_prev();
        } else {
            cp_async_wait_all();
        }
        __syncwarp();
        pred_filter(a, slots(cur, 0), lane);
        pred_filter(b, slots(cur, 1), lane);
        __syncwarp();                    /* the stage is refilled next iteration */
        a = na;
        b = nx;
    }
}

/* U8: the REFCPU 8x8 transform through fast_residual_d (inter path 4) */
/* PART 0: every superblock k_pred took (general[t] == 0); with k_pred
 * marking TX sizes (inter path 5, REFCPU), PART 1 takes the superblocks
 * whose TXs are all 8x8 (general[t] == 0) with only the 8x8 transform in its
 * code, PART 2 the others (general[t] == 2). */
template <int A, int MINB, bool U8, int PART = 0>
__global__ void __launch_bounds__(kFastWarps * 32, MINB) k_resid(const cvp9_job_t *__restrict__ jobs,
                                                            const uint32_t *__restrict__ tickets,
                                                            uint32_t n_tickets, const uint32_t *__restrict__ general)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    ResidSmem &w = reinterpret_cast<ResidSmem *>(smem_raw)[warp];
    const uint32_t t = blockIdx.x * kFastWarps + warp;
    if (t >= n_tickets || general[t] != (PART == 2 ? 2u : 0u)) return;    /* general superblocks: k_recon */
    const uint32_t code = __ldg(tickets + t);
    const cvp9_job_t &job = jobs[code >> 20];
    const int sb = (int)(code & 0xFFFFFu);
    const int sbr = sb / job.sb_cols, sbc = sb - sbr * job.sb_cols;
    const int sbx = sbc * 64, sby = sbr * 64;
    int nb;
    /* the same descriptors k_pred checked and packed: packing alone */
    fast_sb_setup<A, false>(w, job, sb, sbx, sby, lane, nb);
    __syncwarp();
    if (A == CVP9_ARITH_SPEC) {
        const int W = job.W, H = job.H, CW = job.CW, CH = job.CH;
        uint8_t *Y = job.out;
        uint8_t *U = Y + (size_t)W * H;
        uint8_t *V = U + (size_t)CW * CH;
        const size_t coff = (size_t)(sby >> 1) * CW + (sbx >> 1);
        const PredDst D = { Y + (size_t)sby * W + sbx, U + coff, V + coff, W, CW,
                        min(64, W - sbx), min(64, H - sby), min(32, CW - (sbx >> 1)), min(32, CH - (sby >> 1)) };
        fast_spec_residual<true>(w, D, job, nb, lane);
    } else {
        fast_refcpu_residual<true, U8, ResidSmem, PART == 1>(w, job.out + (size_t)sby * job.W + sbx, job.W, job,
                                                             nb, lane);
    }
    __syncwarp();
    if (lane == 0) {
        __threadfence();
        st_release(job.sb_done + sb, job.epoch);
    }
}

/* Order-preserving compaction of the tickets k_inter marked general, one
 * CTA: each thread counts a contiguous segment, a CTA-wide scan places the
 * segments, the thread copies its general tickets. */
__global__ void __launch_bounds__(1024) k_compact(const uint32_t *__restrict__ tickets,
                                                  const uint32_t *__restrict__ general, uint32_t n,
                                                  uint32_t *__restrict__ out, uint32_t *__restrict__ count)
{
    __shared__ uint32_t wsum[32];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (count[1] == 0u) {                /* k_inter took every superblock */
        if (tid == 0) *count = 0u;
        return;
    }
    const uint32_t per = (n + 1023u) / 1024u;
    const uint32_t b = min(n, (uint32_t)tid * per), e = min(n, b + per);
    uint32_t c = 0;
    for (uint32_t i = b; i < e; i++) c += general[i] == 1u;
    uint32_t x = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t v = wsum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += y;
        }
        wsum[lane] = v;
    }
    __syncthreads();
    uint32_t pos = x - c + (wid ? wsum[wid - 1] : 0u);
    for (uint32_t i = b; i < e; i++)
        if (general[i] == 1u) out[pos++] = tickets[i];
    if (tid == 1023) *count = pos;
}

/* ── Loop filter ─────────────────────────────────────────────────────────── */

__device__ __forceinline__ void filter4(uint8_t *p1, uint8_t *p0, uint8_t *q0, uint8_t *q1, int thr)
{
    int P1 = *p1, P0 = *p0, Q0 = *q0, Q1 = *q1;
    int d0 = P0 - Q0, d1 = P1 - Q1;
    if ((d0 < 0 ? -d0 : d0) * 2 + (d1 < 0 ? -d1 : d1) / 2 > thr) return;
    int delta = clampi((3 * (Q0 - P0) + 4) >> 3, -thr, thr);
    *p0 = (uint8_t)clampi(P0 + delta, 0, 255);
    *q0 = (uint8_t)clampi(Q0 - delta, 0, 255);
    *p1 = (uint8_t)clampi(P1 + delta / 2, 0, 255);
    *q1 = (uint8_t)clampi(Q1 - delta / 2, 0, 255);
}

__device__ __forceinline__ int lf_threshold(int level, int sharp)
{
    int t = level;
    if (sharp > 0) {
        t >>= (sharp > 4) ? 2 : 1;
        if (t > 9 - sharp) t = 9 - sharp;
    }
    return t < 1 ? 1 : t;
}

/* Tile (tx, ty) covers luma [64tx-4, 64tx+60) x [TH ty-4, TH ty+TH-4): every
 * tap of every 8-px edge (rows/cols e-2..e+1) lies in one tile and every
 * row in one tile, so the horizontal pass then the vertical pass run
 * tile-locally and in place with the same result as the frame-wide passes
 * (vp9_reconstruct.c:146-190). TH is 64 or 32 (tile height, chosen per shape
 * by the engine's tuner). Requires W and H not of the form 8k+1 (lf_tiled).
 * Rows move as 32-bit words when the frame width allows. */
template <int A, int TH>
__global__ void __launch_bounds__(256) k_loopfilter(const cvp9_job_t *__restrict__ jobs)
{
    __shared__ __align__(16) uint8_t t[TH * 68];
    const cvp9_job_t &job = jobs[blockIdx.z];
    const int tx = blockIdx.x, ty = blockIdx.y;
    const int x0 = tx * 64 - 4, y0 = ty * TH - 4;
    if (job.lf_tiled != 1 || x0 >= job.W || y0 >= job.H) return;
    const bool filt = !(A == CVP9_ARITH_REFCPU && job.lf_level == 0);
    if (!filt && !job.nv12) return;
    const int tid = threadIdx.x;
    const int xa = max(x0, 0), xb = min(x0 + 64, job.W);
    const int ya = max(y0, 0), yb = min(y0 + TH, job.H);
    uint8_t *Y = job.out;
    const int W = job.W;
    const bool words = !(W & 3) && !((uintptr_t)Y & 3);
    /* tile byte (x - x0, y - y0) at t[(y - y0) * 68 + (x - x0)] */
    if (words) {
        const int w0 = (xa - x0) >> 2, nw = (xb - xa) >> 2;
        for (int i = tid; i < (yb - ya) * 16; i += 256) {
            const int r = i >> 4, c = i & 15;
            if (c < nw)
                *reinterpret_cast<uint32_t *>(&t[(ya - y0 + r) * 68 + 4 * (w0 + c)]) =
                    *reinterpret_cast<const uint32_t *>(Y + (size_t)(ya + r) * W + xa + 4 * c);
        }
    } else {
        for (int i = tid; i < (yb - ya) * 64; i += 256) {
            const int r = i >> 6, c = i & 63;
            const int gx = xa + c;
            if (gx < xb) t[(ya - y0 + r) * 68 + (gx - x0)] = Y[(size_t)(ya + r) * W + gx];
        }
    }
    __syncthreads();
    if (filt) {
        const int thr = lf_threshold(job.lf_level, job.lf_sharpness);
        /* horizontal edges e = y0 + 4 + 8k */
        for (int i = tid; i < (TH / 8) * 64; i += 256) {
            const int k = i >> 6, c = i & 63;
            const int e = y0 + 4 + 8 * k, gx = x0 + c;
            if (e < 8 || e >= job.H || gx < xa || gx >= xb) continue;
            const int r = e - y0;
            filter4(&t[(r - 2) * 68 + c], &t[(r - 1) * 68 + c], &t[r * 68 + c], &t[(r + 1) * 68 + c], thr);
        }
        __syncthreads();
        for (int i = tid; i < 8 * TH; i += 256) {
            const int k = i / TH, r = i % TH;
            const int e = x0 + 4 + 8 * k, gy = y0 + r;
            if (e < 8 || e >= job.W || gy < ya || gy >= yb) continue;
            const int c = e - x0;
            uint8_t *row = &t[r * 68];
            filter4(&row[c - 2], &row[c - 1], &row[c], &row[c + 1], thr);
        }
        __syncthreads();
        if (words) {
            const int w0 = (xa - x0) >> 2, nw = (xb - xa) >> 2;
            for (int i = tid; i < (yb - ya) * 16; i += 256) {
                const int r = i >> 4, c = i & 15;
                if (c < nw)
                    *reinterpret_cast<uint32_t *>(Y + (size_t)(ya + r) * W + xa + 4 * c) =
                        *reinterpret_cast<const uint32_t *>(&t[(ya - y0 + r) * 68 + 4 * (w0 + c)]);
            }
        } else {
            for (int i = tid; i < (yb - ya) * 64; i += 256) {
                const int r = i >> 6, c = i & 63;
                const int gx = xa + c;
                if (gx < xb) Y[(size_t)(ya + r) * W + gx] = t[(ya - y0 + r) * 68 + (gx - x0)];
            }
        }
    }
    if (job.nv12) {
        uint8_t *D = job.nv12;
        for (int i = tid; i < (yb - ya) * 64; i += 256) {
            const int r = i >> 6, c = i & 63;
            const int gx = xa + c;
            if (gx < xb) D[(size_t)(ya + r) * W + gx] = t[(ya - y0 + r) * 68 + (gx - x0)];
        }
        /* chroma [32tx-2, 32tx+30) x [TH/2 ty-2, TH/2 ty+TH/2-2) interleaved */
        const int cxa = max(tx * 32 - 2, 0), cxb = min(tx * 32 + 30, job.CW);
        const int cya = max(ty * (TH / 2) - 2, 0), cyb = min(ty * (TH / 2) + TH / 2 - 2, job.CH);
        const uint8_t *U = job.out + (size_t)W * job.H;
        const uint8_t *V = U + (size_t)job.CW * job.CH;
        uint8_t *UV = D + (size_t)W * job.H;
        for (int i = tid; i < (cyb - cya) * 32; i += 256) {
            const int r = i >> 5, c = i & 31;
            const int gx = cxa + c, gy = cya + r;
            if (gx >= cxb) continue;
            const size_t so = (size_t)gy * job.CW + gx;
            const size_t d = (size_t)gy * 2 * job.CW + 2 * gx;
            UV[d] = U[so];
            UV[d + 1] = V[so];
        }
    }
}

/* Register strips: thread (k, j) owns luma columns [8k-4, 8k+4) and rows
 * [16j-4, 16j+12) as two 32-bit words per row. Its two horizontal edges
 * (rows 16j, 16j+8) have every tap inside the strip's rows, and its one
 * vertical edge (column 8k) every tap inside its columns; every pixel lies in
 * one strip. So the horizontal pass then the vertical pass run in registers,
 * with the frame-wide result (vp9_reconstruct.c:146-190) and no shared
 * memory or barriers. Jobs with lf_tiled == 2: W a multiple of 4 (whole
 * words), W and H not of the form 8k+1, no NV12 target. */
__device__ __forceinline__ uint32_t lf_byte(uint32_t w, int i) { return (w >> (8 * i)) & 0xffu; }
__device__ __forceinline__ uint32_t lf_put(uint32_t w, int i, int v)
{
    return (w & ~(0xffu << (8 * i))) | ((uint32_t)v << (8 * i));
}

__device__ __forceinline__ void lf_filter_vals(int &P1, int &P0, int &Q0, int &Q1, int thr)
{
    const int d0 = P0 - Q0, d1 = P1 - Q1;
    if (abs(d0) * 2 + abs(d1) / 2 > thr) return;
    const int delta = clampi((3 * (Q0 - P0) + 4) >> 3, -thr, thr);
    P0 = clampi(P0 + delta, 0, 255);
    Q0 = clampi(Q0 - delta, 0, 255);
    P1 = clampi(P1 + delta / 2, 0, 255);
    Q1 = clampi(Q1 - delta / 2, 0, 255);
}

template <int A>
__global__ void __launch_bounds__(128) k_lf_strip(const cvp9_job_t *__restrict__ jobs)
{
    const cvp9_job_t &job = jobs[blockIdx.z];
    const int k = blockIdx.x * 128 + threadIdx.x;
    const int xs = 8 * k - 4, y0 = 16 * (int)blockIdx.y - 4;
    if (job.lf_tiled != 2 || xs >= job.W || y0 >= job.H) return;
    if (A == CVP9_ARITH_REFCPU && job.lf_level == 0) return;
    const int W = job.W, H = job.H;
    uint8_t *Y = job.out;
    const bool hasA = xs >= 0, hasB = xs + 4 < W;     /* word A: xs..xs+3, word B: xs+4..xs+7 */
    uint32_t a[16], b[16];
#pragma unroll
    for (int r = 0; r < 16; r++) {
        const int gy = y0 + r;
        a[r] = 0u;
        b[r] = 0u;
        if (gy >= 0 && gy < H) {
            const uint8_t *row = Y + (size_t)gy * W;
            if (hasA) a[r] = *reinterpret_cast<const uint32_t *>(row + xs);
            if (hasB) b[r] = *reinterpret_cast<const uint32_t *>(row + xs + 4);
        }
    }
    const int thr = lf_threshold(job.lf_level, job.lf_sharpness);
    /* horizontal edges at strip rows 4 and 12 */
#pragma unroll
    for (int m = 4; m <= 12; m += 8) {
        const int e = y0 + m;
        if (e < 8 || e >= H) continue;
#pragma unroll
        for (int c = 0; c < 8; c++) {
            if (c < 4 ? !hasA : !hasB) continue;
            uint32_t *wv = c < 4 ? a : b;
            const int bi = c & 3;
            int P1 = (int)lf_byte(wv[m - 2], bi), P0 = (int)lf_byte(wv[m - 1], bi);
            int Q0 = (int)lf_byte(wv[m], bi), Q1 = (int)lf_byte(wv[m + 1], bi);
            lf_filter_vals(P1, P0, Q0, Q1, thr);
            wv[m - 2] = lf_put(wv[m - 2], bi, P1);
            wv[m - 1] = lf_put(wv[m - 1], bi, P0);
            wv[m] = lf_put(wv[m], bi, Q0);
            wv[m + 1] = lf_put(wv[m + 1], bi, Q1);
        }
    }
    /* vertical edge at column xs + 4 = 8k: bytes 2, 3 of A and 0, 1 of B */
    const int ev = xs + 4;
    if (ev >= 8 && ev < W) {
#pragma unroll
        for (int r = 0; r < 16; r++) {
            const int gy = y0 + r;
            if (gy < 0 || gy >= H) continue;
            int P1 = (int)lf_byte(a[r], 2), P0 = (int)lf_byte(a[r], 3);
            int Q0 = (int)lf_byte(b[r], 0), Q1 = (int)lf_byte(b[r], 1);
            lf_filter_vals(P1, P0, Q0, Q1, thr);
            a[r] = (a[r] & 0x0000ffffu) | (uint32_t)P1 << 16 | (uint32_t)P0 << 24;
            b[r] = (b[r] & 0xffff0000u) | (uint32_t)Q0 | (uint32_t)Q1 << 8;
        }
    }
#pragma unroll
    for (int r = 0; r < 16; r++) {
        const int gy = y0 + r;
        if (gy < 0 || gy >= H) continue;
        uint8_t *row = Y + (size_t)gy * W;
        if (hasA) *reinterpret_cast<uint32_t *>(row + xs) = a[r];
        if (hasB) *reinterpret_cast<uint32_t *>(row + xs + 4) = b[r];
    }
}

/* Frame-wide loop filter for widths/heights of the form 8k+1, with the
 * reference's flat addressing (vertical edges at the last column read the
 * next row's first sample) and out-of-plane accesses skipped. */
__global__ void k_lf_flat_h(const cvp9_job_t *__restrict__ jobs, int refcpu)
{
    const cvp9_job_t &job = jobs[blockIdx.y];
    if (job.lf_tiled || (refcpu && job.lf_level == 0)) return;
    int thr = lf_threshold(job.lf_level, job.lf_sharpness);
    int nedge = job.H > 8 ? (job.H - 1) / 8 : 0;
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)nedge * job.W) return;
    int e = 8 * (int)(i / job.W + 1), x = (int)(i % job.W);
    if (e + 1 >= job.H) return;
    uint8_t *Y = job.out;
    size_t S = (size_t)job.W;
    filter4(Y + (e - 2) * S + x, Y + (e - 1) * S + x, Y + e * S + x, Y + (e + 1) * S + x, thr);
}

__global__ void k_lf_flat_v(const cvp9_job_t *__restrict__ jobs, int refcpu)
{
    const cvp9_job_t &job = jobs[blockIdx.y];
    if (job.lf_tiled || (refcpu && job.lf_level == 0)) return;
    int thr = lf_threshold(job.lf_level, job.lf_sharpness);
    int nedge = job.W > 8 ? (job.W - 1) / 8 : 0;
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)nedge * job.H) return;
    int e = 8 * (int)(i / job.H + 1), r = (int)(i % job.H);
    uint8_t *Y = job.out;
    size_t S = (size_t)job.W, plane = S * job.H;
    size_t base = (size_t)r * S + e;
    if (base + 1 >= plane) return;
    filter4(Y + base - 2, Y + base - 1, Y + base, Y + base + 1, thr);
}

/* ── FULL profile: the VP9 loop filter ───────────────────────────────────
 *
 * k_lf_mimap records, per 8x8 MI, what the filter needs of the block that
 * covers it: luma and chroma TX size, whether it is a skipped inter block,
 * and the MI's offset inside the block (bits 0-1, 2-3, 4, 5-7, 8-10), tagged
 * with the frame's epoch in the high half so that entries of earlier frames
 * read as "no block". k_lf_full then filters superblock by superblock in the
 * VP9 order: every vertical edge of a superblock (each row left to right),
 * then its horizontal edges (each column top to bottom), superblocks in
 * raster order. A CTA takes a superblock row (ticket) and walks it left to
 * right; superblock (r, c) starts once row r-1 has finished (r-1, c+1), the
 * last one whose filtering reaches the samples (r, c) reads. Each
 * superblock is filtered in shared memory with an 8-sample halo above and
 * to the left, which its first edges modify. */
__global__ void __launch_bounds__(256) k_lf_mimap(const cvp9_job_t *__restrict__ jobs)
{
    const cvp9_job_t &job = jobs[blockIdx.y];
    if (!job.full || !job.mi_map) return;
    const uint32_t tag = (job.epoch & 0xFFFFu) << 16;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < job.num_blocks; i += gridDim.x * blockDim.x) {
        const vp9_macroblock_info_t b = job.blocks[i];
        if (b.x >= job.W || b.y >= job.H || b.tx_size > 3 || b.width < 4 || b.height < 4) continue;
        const bool sub8 = b.width < 8 || b.height < 8;
        const int bw = sub8 ? 8 : b.width, bh = sub8 ? 8 : b.height;
        const int uvw = bw / 2 < 4 ? 4 : bw / 2, uvh = bh / 2 < 4 ? 4 : bh / 2;
        const int txuv = sub8 ? 0 : min((int)b.tx_size, max_tx_for(uvw, uvh));
        const uint32_t info = tag | (uint32_t)b.tx_size | ((uint32_t)txuv << 2) |
                              ((uint32_t)(b.skip && !b.is_intra) << 4);
        const int mc = b.x >> 3, mr = b.y >> 3;
        const int nc = min((bw + 7) >> 3, job.mi_cols - mc), nr = min((bh + 7) >> 3, job.mi_rows - mr);
        for (int r = 0; r < nr; r++)
            for (int c = 0; c < nc; c++)
                job.mi_map[(size_t)(mr + r) * job.mi_cols + mc + c] = info | ((uint32_t)c << 5) | ((uint32_t)r << 8);
    }
}

struct LfThr { int lim, mblim, hev; };

/* Filter across one edge: q0 at s[0], p0 at s[-st]; fs = widest filter
 * allowed there (4, 8 or 16), narrowed by the flatness tests. T, SH: the
 * sample type and bit depth - 8; at 10 bits (profile 2) the flatness test
 * compares against 1 << SH, the 4-tap filter clamps to the signed range of
 * the bit depth around 128 << SH, and th arrives shifted by SH. */
template <class T, int SH>
__device__ __forceinline__ void lf_edge_full(T *s, int st, int fs, LfThr th)
{
    constexpr int kFlat = 1 << SH, kMid = 128 << SH;
    auto P = [&](int i) -> int { return s[(-i - 1) * st]; };
    auto Q = [&](int i) -> int { return s[i * st]; };
    const int p3 = P(3), p2 = P(2), p1 = P(1), p0 = P(0), q0 = Q(0), q1 = Q(1), q2 = Q(2), q3 = Q(3);
    const bool mask = abs(p3 - p2) <= th.lim && abs(p2 - p1) <= th.lim && abs(p1 - p0) <= th.lim &&
                      abs(q1 - q0) <= th.lim && abs(q2 - q1) <= th.lim && abs(q3 - q2) <= th.lim &&
                      abs(p0 - q0) * 2 + abs(p1 - q1) / 2 <= th.mblim;
    if (!mask) return;
    const bool flat = fs >= 8 && abs(p1 - p0) <= kFlat && abs(q1 - q0) <= kFlat && abs(p2 - p0) <= kFlat &&
                      abs(q2 - q0) <= kFlat && abs(p3 - p0) <= kFlat && abs(q3 - q0) <= kFlat;
    bool flat2 = false;
    if (fs == 16 && flat) {
        flat2 = true;
#pragma unroll
        for (int i = 4; i < 8; i++) flat2 &= abs(P(i) - p0) <= kFlat && abs(Q(i) - q0) <= kFlat;
    }
    if (flat2) {
        int v[16], o[16];
#pragma unroll
        for (int i = 0; i < 8; i++) { v[7 - i] = P(i); v[8 + i] = Q(i); }
#pragma unroll
        for (int k = 1; k < 15; k++) {
            int acc = v[k];
#pragma unroll
            for (int t = k - 7; t <= k + 7; t++) acc += v[t < 0 ? 0 : (t > 15 ? 15 : t)];
            o[k] = (acc + 8) >> 4;
        }
#pragma unroll
        for (int k = 1; k < 15; k++) s[(k - 8) * st] = (T)o[k];
    } else if (flat) {
        int v[8], o[8];
#pragma unroll
        for (int i = 0; i < 4; i++) { v[3 - i] = P(i); v[4 + i] = Q(i); }
#pragma unroll
        for (int k = 1; k < 7; k++) {
            int acc = v[k];
#pragma unroll
            for (int t = k - 3; t <= k + 3; t++) acc += v[t < 0 ? 0 : (t > 7 ? 7 : t)];
            o[k] = (acc + 4) >> 3;
        }
#pragma unroll
        for (int k = 1; k < 7; k++) s[(k - 4) * st] = (T)o[k];
    } else {
        auto sc8 = [](int v) { return v < -kMid ? -kMid : (v > kMid - 1 ? kMid - 1 : v); };
        const int ps1 = p1 - kMid, ps0 = p0 - kMid, qs0 = q0 - kMid, qs1 = q1 - kMid;
        const bool hev = abs(p1 - p0) > th.hev || abs(q1 - q0) > th.hev;
        int f = hev ? sc8(ps1 - qs1) : 0;
        f = sc8(f + 3 * (qs0 - ps0));
        const int f1 = sc8(f + 4) >> 3, f2 = sc8(f + 3) >> 3;
        s[0] = (T)(sc8(qs0 - f1) + kMid);
        s[-st] = (T)(sc8(ps0 + f2) + kMid);
        if (!hev) {
            const int f3 = (f1 + 1) >> 1;
            s[st] = (T)(sc8(qs1 - f3) + kMid);
            s[-2 * st] = (T)(sc8(ps1 + f3) + kMid);
        }
    }
}

/* Filter size of the edge on the left (dir 0) or top (dir 1) of 8x8 unit
 * (ux, uy) of a plane, 0 for none; inner: the 4x4 edge 4 samples in is
 * filtered too. Chroma units take the block at their top-left MI. */
/* e: the mode-info word of the unit's top-left MI (k_lf_mimap). */
__device__ __forceinline__ int lf_unit_edge(const cvp9_job_t &job, int plane, int ux, int uy, int dir, bool &inner,
                                            uint32_t e)
{
    const int ss = plane > 0;
    const uint32_t info = (e >> 16) == (job.epoch & 0xFFFFu) ? (e & 0xFFFFu) : 0u;
    const int tx = ss ? (int)((info >> 2) & 3u) : (int)(info & 3u);
    const bool skipi = (info >> 4) & 1u;
    const int pos = (int)(dir ? (info >> 8) & 7u : (info >> 5) & 7u) * (ss ? 4 : 8);
    const int u = dir ? uy : ux, edge = u * 8;
    const bool half = ss && ((u << 1) + 1 >= (dir ? job.mi_rows : job.mi_cols));
    inner = tx == 0 && !skipi && !half;
    if (edge == 0) return 0;
    const bool block_edge = pos == 0, tx_edge = (pos & ((4 << tx) - 1)) == 0;
    if (!block_edge && !(tx_edge && !skipi)) return 0;
    int fs = tx == 0 ? 4 : (tx == 1 ? 8 : 16);
    if (fs == 4 && (edge & 31) == 0) fs = 8;
    if (fs == 16 && half) fs = 8;
    return fs;
}

constexpr int kLfY = 72, kLfC = 40;      /* window pitches: 8-sample halo + superblock */

__device__ bool wait_at_least(const unsigned *flag, unsigned v)
{
    for (long long it = 0; it < kSpinLimit; it++) {
        if (ld_acquire(flag) >= v) return true;
        __nanosleep(it < 64 ? 32 : 256);
    }
    return false;
}

/* 4 samples as one load or store: a 32-bit word of 8-bit samples, two of
 * 16-bit ones. */
template <class T> struct Quad;
template <> struct Quad<uint8_t> { using type = unsigned int; };
template <> struct Quad<uint16_t> { using type = uint2; };

template <class T, int SH>
__global__ void __launch_bounds__(128) k_lf_full(const cvp9_job_t *__restrict__ jobs, int njobs,
                                                uint32_t n_tickets, uint32_t *counter)
{
    using Q4 = typename Quad<T>::type;
    __shared__ __align__(16) T wy[kLfY * kLfY];
    __shared__ __align__(16) T wc[2][kLfC * kLfC];
    __shared__ uint32_t mi_s[64];          /* the superblock's 8x8 mode-info words */
    __shared__ int s_ticket;
    const int tid = threadIdx.x;
    for (;;) {
        __syncthreads();
        if (tid == 0) s_ticket = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int t = s_ticket;
        if (t >= (int)n_tickets) return;
        const cvp9_job_t &job = jobs[t % njobs];
        const int row = t / njobs;
        if (!job.full || row >= job.sb_rows || job.lf_level == 0) continue;
        LfThr th;
        {
            const int level = job.lf_level, sharp = job.lf_sharpness;
            int bil = level >> ((sharp > 0) + (sharp > 4));
            if (sharp > 0 && bil > 9 - sharp) bil = 9 - sharp;
            if (bil < 1) bil = 1;
            th.lim = bil << SH;
            th.mblim = (2 * (level + 2) + bil) << SH;
            th.hev = (level >> 4) << SH;
        }
        const int W = job.W, H = job.H, CW = job.CW, CH = job.CH;
        T *Y = reinterpret_cast<T *>(job.out);
        T *U = Y + (size_t)W * H;
        T *V = U + (size_t)CW * CH;
        unsigned *prog_prev = row > 0 ? job.sb_range + 4 * (size_t)(row - 1) * job.sb_cols + 3 : nullptr;
        unsigned *prog = job.sb_range + 4 * (size_t)row * job.sb_cols + 3;
        for (int c = 0; c < job.sb_cols; c++) {
            if (prog_prev && tid == 0) {
                const unsigned need = (unsigned)min(c + 2, job.sb_cols);
                if (!wait_at_least(prog_prev, need)) atomicOr(job.status, (unsigned)CVP9_JOB_TIMEOUT);
            }
            __syncthreads();
            const int X0 = c * 64, Y0 = row * 64, XC = c * 32, YC = row * 32;
            /* the superblock's mode info, once: each edge decision reads it */
            if (tid < 64) {
                const int mr = row * 8 + (tid >> 3), mc = c * 8 + (tid & 7);
                mi_s[tid] = (mr < job.mi_rows && mc < job.mi_cols) ? job.mi_map[(size_t)mr * job.mi_cols + mc] : 0u;
            }
            /* load the windows (4-byte words: W and the window origins are
             * multiples of 8, so every word is inside one row) */
            for (int i = tid; i < kLfY * (kLfY / 4); i += 128) {
                const int r = i / (kLfY / 4), w4 = i - r * (kLfY / 4);
                const int gy = Y0 - 8 + r, gx = X0 - 8 + 4 * w4;
                if (gy >= 0 && gy < H && gx >= 0 && gx < W)
                    *reinterpret_cast<Q4 *>(&wy[r * kLfY + 4 * w4]) =
                        __ldcg(reinterpret_cast<const Q4 *>(Y + (size_t)gy * W + gx));
            }
            for (int i = tid; i < 2 * kLfC * (kLfC / 4); i += 128) {
                const int pl = i >= kLfC * (kLfC / 4);
                const int k = pl ? i - kLfC * (kLfC / 4) : i;
                const int r = k / (kLfC / 4), w4 = k - r * (kLfC / 4);
                const int gy = YC - 8 + r, gx = XC - 8 + 4 * w4;
                if (gy >= 0 && gy < CH && gx >= 0 && gx < CW)
                    *reinterpret_cast<Q4 *>(&wc[pl][r * kLfC + 4 * w4]) =
                        __ldcg(reinterpret_cast<const Q4 *>((pl ? V : U) + (size_t)gy * CW + gx));
            }
            __syncthreads();
            /* vertical edges: a thread per row (64 luma, 32 + 32 chroma) */
            {
                const int p = tid < 64 ? 0 : (tid < 96 ? 1 : 2);
                const int r = p == 0 ? tid : (tid - 32 - 32 * p);
                const int sz = p ? 32 : 64, pw = p ? CW : W, ph = p ? CH : H;
                const int gy = (p ? YC : Y0) + r, gx0 = p ? XC : X0;
                T *row_p = p == 0 ? &wy[(8 + r) * kLfY + 8] : &wc[p - 1][(8 + r) * kLfC + 8];
                if (gy < ph)
                    for (int x = 0; x < sz && gx0 + x < pw; x += 8) {
                        bool inner;
                        const int ux = (gx0 + x) >> 3, uy = gy >> 3, ss = p > 0;
                        const int fs = lf_unit_edge(job, p, ux, uy, 0, inner,
                                                    mi_s[((uy << ss) - row * 8) * 8 + (ux << ss) - c * 8]);
                        if (fs) lf_edge_full<T, SH>(row_p + x, 1, fs, th);
                        if (inner && gx0 + x + 4 < pw) lf_edge_full<T, SH>(row_p + x + 4, 1, 4, th);
                    }
            }
            __syncthreads();
            /* horizontal edges: a thread per column */
            {
                const int p = tid < 64 ? 0 : (tid < 96 ? 1 : 2);
                const int x = p == 0 ? tid : (tid - 32 - 32 * p);
                const int sz = p ? 32 : 64, pw = p ? CW : W, ph = p ? CH : H;
                const int gx = (p ? XC : X0) + x, gy0 = p ? YC : Y0;
                const int pitch = p ? kLfC : kLfY;
                T *col_p = p == 0 ? &wy[8 * kLfY + 8 + x] : &wc[p - 1][8 * kLfC + 8 + x];
                if (gx < pw)
                    for (int y = 0; y < sz && gy0 + y < ph; y += 8) {
                        bool inner;
                        const int ux = gx >> 3, uy = (gy0 + y) >> 3, ss = p > 0;
                        const int fs = lf_unit_edge(job, p, ux, uy, 1, inner,
                                                    mi_s[((uy << ss) - row * 8) * 8 + (ux << ss) - c * 8]);
                        if (fs) lf_edge_full<T, SH>(col_p + y * pitch, pitch, fs, th);
                        if (inner && gy0 + y + 4 < ph) lf_edge_full<T, SH>(col_p + (y + 4) * pitch, pitch, 4, th);
                    }
            }
            __syncthreads();
            /* write back: the superblock's rows with the left halo, and the
             * halo rows above over the superblock's columns */
            for (int i = tid; i < kLfY * (kLfY / 4); i += 128) {
                const int r = i / (kLfY / 4), w4 = i - r * (kLfY / 4);
                if (r < 8 && w4 < 2) continue;                  /* the corner: untouched */
                const int gy = Y0 - 8 + r, gx = X0 - 8 + 4 * w4;
                if (gy >= 0 && gy < H && gx >= 0 && gx < W)
                    *reinterpret_cast<Q4 *>(Y + (size_t)gy * W + gx) =
                        *reinterpret_cast<const Q4 *>(&wy[r * kLfY + 4 * w4]);
            }
            for (int i = tid; i < 2 * kLfC * (kLfC / 4); i += 128) {
                const int pl = i >= kLfC * (kLfC / 4);
                const int k = pl ? i - kLfC * (kLfC / 4) : i;
                const int r = k / (kLfC / 4), w4 = k - r * (kLfC / 4);
                if (r < 8 && w4 < 2) continue;
                const int gy = YC - 8 + r, gx = XC - 8 + 4 * w4;
                if (gy >= 0 && gy < CH && gx >= 0 && gx < CW)
                    *reinterpret_cast<Q4 *>((pl ? V : U) + (size_t)gy * CW + gx) =
                        *reinterpret_cast<const Q4 *>(&wc[pl][r * kLfC + 4 * w4]);
            }
            __syncthreads();
            if (tid == 0) {
                __threadfence();
                st_release(prog, (unsigned)(c + 1));
            }
        }
    }
}

/* ── Profile 2 (10-bit 4:2:0): k_hbd_recon ─────────────────────────────
 *
 * The FULL profile's reconstruction on 16-bit samples in [0, 1023]. The
 * frame brings its coefficients dequantised, as int32 (coeffs32, the dense
 * layout of coeffs; the 32x32 halving already applied): the butterflies run
 * in 64-bit integers (wl) with 32-bit values between the row and the column
 * pass, both 8-tap passes of a prediction round and clip to 10 bits, intra
 * edges that are missing read 511 above and 513 on the left (512 for a DC
 * with neither), and every residual add clips to [0, 1023]. The loop filter
 * is k_lf_full<uint16_t, 2>.
 *
 * One CTA per superblock ticket (SB-diagonal order over the step's jobs,
 * persistent, as k_recon). Its inter blocks do not depend on one another or
 * on other superblocks, so they go first and together: prediction a thread
 * per column strip of up to 8 rows, then a thread per TX row, then per TX
 * column. The intra blocks follow by dependency level, the blocks of a
 * level on different warps, each block TX by TX (each TX predicted from the
 * reconstructed samples around it). A superblock whose blocks overlap, or
 * whose intra blocks read samples of blocks later in the list, runs block by
 * block in list order, so every sample is what the list order makes it. */
namespace {

constexpr int kHbdThreads = 256, kHbdWarps = kHbdThreads / 32;
constexpr int kHbdMaxBlocks = 256, kHbdMaxTx = 384;
constexpr int kHYP = 72, kHCP = 40;      /* tile pitches in samples; column -1 at index 3 */
constexpr int kHbdMax = 1023, kHbdMid = 512;

struct HbdBlk {
    uint8_t  x, y;            /* local luma origin in the SB                 */
    uint8_t  w, h;            /* coded size                                  */
    uint8_t  cw, ch;          /* luma region (a sub-8x8 block's whole 8x8)
                               * clamped to the frame                        */
    uint8_t  ccw, cch;        /* chroma region, clamped                      */
    uint8_t  txl, flags;      /* tx_size; 1 intra, 2 skip                    */
    uint8_t  ymode, uvmode;
    uint8_t  ref0, ref1;
    int16_t  mvx, mvy, mv1x, mv1y;
    uint32_t coeff;
};

struct HbdTx {
    uint32_t coeff;
    uint8_t  plane, txl, x, y;   /* plane-local tile position */
};

struct HbdSmem {
    uint16_t ty[65 * kHYP];                /* luma tile, row 0 = the row above */
    uint16_t tc[2][33 * kHCP];
    int32_t  tmp[64 * 64 + 2 * 32 * 32];   /* row-pass output at tile positions */
    HbdBlk   blk[kHbdMaxBlocks];
    HbdTx    tx[kHbdMaxTx];
    uint16_t tx_base[kHbdMaxTx + 1];       /* prefix over TXs of their sizes   */
    uint16_t it_base[kHbdMaxBlocks + 1];   /* prefix over blocks of their items */
    unsigned cell[256];                    /* claims of each 4x4 cell          */
    uint8_t  owner[256];                   /* the block claiming it (one claim) */
    uint8_t  lvl[kHbdMaxBlocks];           /* intra blocks: dependency level   */
    uint8_t  txnz[kHbdMaxTx];
    int32_t  edge[kHbdWarps][1 + 64 + 32]; /* intra, per warp: above[-1..2n-1], left */
    int      scan[kHbdWarps];
    cvp9_job_t jc;
    int      ticket, ntx, nlev, order_bad;
};

__device__ __forceinline__ uint16_t &HT(HbdSmem &s, int p, int x, int y)
{
    return p == 0 ? s.ty[(y + 1) * kHYP + x + 4] : s.tc[p - 1][(y + 1) * kHCP + x + 4];
}

__device__ __forceinline__ int32_t *hbd_tmp(HbdSmem &s, int p, int x, int y)
{
    return p == 0 ? &s.tmp[y * 64 + x] : &s.tmp[4096 + (p - 1) * 1024 + y * 32 + x];
}

__device__ __forceinline__ long long clampll(long long v, long long lo, long long hi)
{
    return v < lo ? lo : (v > hi ? hi : v);
}

/* Exclusive prefix of v over the CTA's threads (thread order); *total: the
 * sum. Every thread calls it. */
__device__ int hbd_scan(HbdSmem &s, int v, int *total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s.scan[warp] = x;
    __syncthreads();
    int off = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < kHbdWarps; w++) {
        const int t = s.scan[w];
        off += w < warp ? t : 0;
        tot += t;
    }
    *total = tot;
    __syncthreads();
    return off + x - v;
}

/* Largest k in [0, n) with base[k] <= v (base ascending, base[0] = 0). */
__device__ __forceinline__ int hbd_find(const uint16_t *base, int n, int v)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (base[mid] <= v) lo = mid; else hi = mid - 1;
    }
    return lo;
}

/* Prediction items of an inter block: a column strip of up to 8 rows of
 * one plane. */
__device__ __forceinline__ int hbd_pred_items(const HbdBlk &b)
{
    return (int)b.cw * (((int)b.ch + 7) >> 3) + 2 * (int)b.ccw * (((int)b.cch + 7) >> 3);
}

/* One column strip of one plane of an inter block: both 8-tap passes (the
 * frame's filter), each rounded and clipped to 10 bits, every fetch clamped
 * into the reference plane; a compound block averages its second
 * prediction in with rounding. A missing first reference predicts 512. */
__device__ void hbd_pred_strip(HbdSmem &s, const HbdBlk &b, int item, int sbx, int sby)
{
    const cvp9_job_t &job = s.jc;
    const int nl = (int)b.cw * (((int)b.ch + 7) >> 3), nc = (int)b.ccw * (((int)b.cch + 7) >> 3);
    int p, k;
    if (item < nl) { p = 0; k = item; }
    else { p = 1 + (item - nl >= nc); k = item - nl - (p - 1) * nc; }
    const int cols = p ? b.ccw : b.cw, rows = p ? b.cch : b.ch;
    const int grp = k / cols, c = k - grp * cols;
    const int r0 = grp * 8, nr = min(8, rows - r0);
    const int lx = (p ? (b.x >> 1) : b.x) + c, ly0 = (p ? (b.y >> 1) : b.y) + r0;
    const int gx = (p ? (sbx >> 1) : sbx) + lx, gy0 = (p ? (sby >> 1) : sby) + ly0;
    const int (*F)[8] = c_subpel4[job.interp_filter & 3];
    int out[8];
#pragma unroll
    for (int i = 0; i < 8; i++) out[i] = kHbdMid;
    for (int q = 0; q < 2; q++) {
        const int rf = q ? b.ref1 : b.ref0;
        if (q == 1 && rf == 0) break;
        const cvp9_ref_t &R = job.ref[job.ref_slot_of[clampi(rf - 1, 0, 2)] & 7];
        if (!R.plane) break;
        const uint16_t *rp = reinterpret_cast<const uint16_t *>(R.plane);
        int pw = R.w, ph = R.h;
        if (p) {
            rp += (size_t)R.w * R.h;
            pw = (R.w + 1) >> 1;
            ph = (R.h + 1) >> 1;
            if (p == 2) rp += (size_t)pw * ph;
        }
        const int mvx = q ? b.mv1x : b.mvx, mvy = q ? b.mv1y : b.mvy;
        const int X = gx + (p ? (mvx >> 4) : (mvx >> 3)), Y0 = gy0 + (p ? (mvy >> 4) : (mvy >> 3));
        const int fx = p ? (mvx & 15) : ((mvx & 7) << 1), fy = p ? (mvy & 15) : ((mvy & 7) << 1);
        int cx[8];
#pragma unroll
        for (int t = 0; t < 8; t++) cx[t] = clampi(X + t - 3, 0, pw - 1);
        int h[15];
#pragma unroll
        for (int j = 0; j < 15; j++) {
            h[j] = 0;
            if (j >= nr + 7) continue;
            const uint16_t *row = rp + (size_t)clampi(Y0 - 3 + j, 0, ph - 1) * pw;
            if (fx == 0) {
                h[j] = __ldg(row + cx[3]);
            } else {
                int a = 0;
#pragma unroll
                for (int t = 0; t < 8; t++) a += F[fx][t] * (int)__ldg(row + cx[t]);
                h[j] = clampi((a + 64) >> 7, 0, kHbdMax);
            }
        }
#pragma unroll
        for (int i = 0; i < 8; i++) {
            int v = h[i + 3];
            if (fy != 0) {
                int a = 0;
#pragma unroll
                for (int t = 0; t < 8; t++) a += F[fy][t] * h[i + t];
                v = clampi((a + 64) >> 7, 0, kHbdMax);
            }
            out[i] = q ? (out[i] + v + 1) >> 1 : v;
        }
    }
#pragma unroll
    for (int i = 0; i < 8; i++)
        if (i < nr) HT(s, p, lx, ly0 + i) = (uint16_t)out[i];
}

/* The TX layout of one plane of a block (as plane_layout). */
__device__ __forceinline__ void hbd_plane_layout(const HbdBlk &b, const cvp9_job_t &job, int gx, int gy, int p,
                                                 int &tx, int &nx, int &ny, int &pbw)
{
    const int sub8 = b.w < 8 || b.h < 8;
    const int ew = sub8 ? 8 : b.w, eh = sub8 ? 8 : b.h;
    const int ss = p > 0;
    int pw = ss ? ew / 2 : ew, ph = ss ? eh / 2 : eh;
    pw = pw < 4 ? 4 : pw;
    ph = ph < 4 ? 4 : ph;
    tx = b.txl;
    if (ss) { const int mt = max_tx_for(pw, ph); tx = sub8 ? 0 : (tx > mt ? mt : tx); }
    const int t4 = 1 << tx;
    const int o4x = ((gx >> 3) * 2) >> ss, o4y = ((gy >> 3) * 2) >> ss;
    int mw = pw / 4, mh = ph / 4;
    const int lim_w = ((job.mi_cols * 2) >> ss) - o4x, lim_h = ((job.mi_rows * 2) >> ss) - o4y;
    if (mw > lim_w) mw = lim_w;
    if (mh > lim_h) mh = lim_h;
    nx = mw > 0 ? (mw + t4 - 1) / t4 : 0;
    ny = mh > 0 ? (mh + t4 - 1) / t4 : 0;
    pbw = pw;
}

/* Residual TXs of an inter block in coefficient order (planes, then raster),
 * written from s.tx[at] when `at` >= 0; returns their count. The running
 * offset stops at num_coeffs: a TX that does not fit and every later one of
 * the block are dropped. */
__device__ int hbd_block_txs(HbdSmem &s, const HbdBlk &b, int sbx, int sby, int at)
{
    if ((b.flags & 2) || b.txl > 3) return 0;
    const cvp9_job_t &job = s.jc;
    const int gx = sbx + b.x, gy = sby + b.y;
    uint64_t off = b.coeff;
    int n = 0;
    for (int p = 0; p < 3; p++) {
        int txl, nx, ny, pbw;
        hbd_plane_layout(b, job, gx, gy, p, txl, nx, ny, pbw);
        const int sz = 16 << (2 * txl), ts = 4 << txl;
        const int ox = p ? (b.x >> 1) : b.x, oy = p ? (b.y >> 1) : b.y;
        for (int ty = 0; ty < ny; ty++)
            for (int tx = 0; tx < nx; tx++) {
                if (off + (uint64_t)sz > (uint64_t)job.num_coeffs) { off = job.num_coeffs; continue; }
                if (at >= 0 && at + n < kHbdMaxTx) {
                    HbdTx &t = s.tx[at + n];
                    t.coeff = (uint32_t)off;
                    t.plane = (uint8_t)p;
                    t.txl = (uint8_t)txl;
                    t.x = (uint8_t)(ox + tx * ts);
                    t.y = (uint8_t)(oy + ty * ts);
                }
                off += (uint64_t)sz;
                n++;
            }
    }
    return n;
}

/* Row pass of TX row i: the frame's dequantised coefficients through the
 * 1-D inverse (DCT, ADST along the row when row_adst, WHT when lossless),
 * 64-bit inside, 32-bit out into the temp rows. Returns whether the row had
 * a nonzero coefficient. */
template <int N>
__device__ __forceinline__ bool hbd_row(HbdSmem &s, const int32_t *X, int i, int p, int px0, int py0,
                                        bool lossless, bool row_adst)
{
    wl v[N];
    bool any = false;
#pragma unroll
    for (int k = 0; k < N; k++) {
        const int c = __ldg(X + i * N + k);
        any |= c != 0;
        v[k] = wl(c);
    }
    if (any) {
        if (N == 4 && lossless) iwht4(v, true);
        else itx1<N>(v, row_adst);
    }
    int32_t *d = hbd_tmp(s, p, px0, py0 + i);
#pragma unroll
    for (int k = 0; k < N; k++) d[k] = any ? (int32_t)v[k].v : 0;
    return any;
}

/* Column pass of TX column j: the 1-D inverse down the column (64-bit),
 * rounding shift 4/5/6/6 (none after the WHT), add and clip to 10 bits. */
template <int N>
__device__ __forceinline__ void hbd_col(HbdSmem &s, int j, int p, int px0, int py0, bool lossless, bool col_adst)
{
    wl v[N];
#pragma unroll
    for (int k = 0; k < N; k++) v[k] = wl(*hbd_tmp(s, p, px0 + j, py0 + k));
    const bool wht = N == 4 && lossless;
    if (wht) iwht4(v, false);
    else itx1<N>(v, col_adst);
    const int sh = N == 4 ? 4 : (N == 8 ? 5 : 6);
#pragma unroll
    for (int k = 0; k < N; k++) {
        const long long r = wht ? v[k].v : (v[k].v + (1ll << (sh - 1))) >> sh;
        uint16_t &px = HT(s, p, px0 + j, py0 + k);
        px = (uint16_t)clampll((long long)px + r, 0, kHbdMax);
    }
}

__device__ __forceinline__ void hbd_row_n(HbdSmem &s, int txl, const int32_t *X, int i, int p, int x, int y,
                                          bool lossless, bool row_adst, bool &any)
{
    switch (txl) {
    case 0: any = hbd_row<4>(s, X, i, p, x, y, lossless, row_adst); break;
    case 1: any = hbd_row<8>(s, X, i, p, x, y, lossless, row_adst); break;
    case 2: any = hbd_row<16>(s, X, i, p, x, y, lossless, row_adst); break;
    default: any = hbd_row<32>(s, X, i, p, x, y, lossless, false); break;
    }
}

__device__ __forceinline__ void hbd_col_n(HbdSmem &s, int txl, int j, int p, int x, int y, bool lossless,
                                          bool col_adst)
{
    switch (txl) {
    case 0: hbd_col<4>(s, j, p, x, y, lossless, col_adst); break;
    case 1: hbd_col<8>(s, j, p, x, y, lossless, col_adst); break;
    case 2: hbd_col<16>(s, j, p, x, y, lossless, col_adst); break;
    default: hbd_col<32>(s, j, p, x, y, lossless, false); break;
    }
}

/* Inter blocks [lo, hi) of the SB, whole CTA: predictions, then the TX rows,
 * then the TX columns of their residuals. */
__device__ void hbd_inter_blocks(HbdSmem &s, int lo, int hi, int nb, int sbx, int sby)
{
    const int tid = threadIdx.x;
    const cvp9_job_t &job = s.jc;
    const bool mine = tid >= lo && tid < hi && tid < nb && !(s.blk[tid].flags & 1);
    int total;
    /* 1. predictions */
    int cnt = mine ? hbd_pred_items(s.blk[tid]) : 0;
    int base = hbd_scan(s, cnt, &total);
    if (tid < kHbdMaxBlocks) s.it_base[tid] = (uint16_t)min(base, 0xFFFF);
    __syncthreads();
    for (int it = tid; it < total; it += kHbdThreads) {
        const int bi = hbd_find(s.it_base, nb, it);
        hbd_pred_strip(s, s.blk[bi], it - s.it_base[bi], sbx, sby);
    }
    /* 2. the residual TXs, a thread per block listing its own */
    cnt = mine ? hbd_block_txs(s, s.blk[tid], sbx, sby, -1) : 0;
    base = hbd_scan(s, cnt, &total);
    if (total > kHbdMaxTx) {
        if (tid == 0) atomicOr(job.status, (unsigned)CVP9_JOB_TOO_MANY);
        total = kHbdMaxTx;
    }
    if (mine && cnt) hbd_block_txs(s, s.blk[tid], sbx, sby, base);
    __syncthreads();
    const int ntx = total;
    /* prefix over TXs of their edge length (their rows, and columns), two
     * consecutive TXs a thread */
    {
        const int t0 = 2 * tid, t1 = 2 * tid + 1;
        const int a = t0 < ntx ? 4 << s.tx[t0].txl : 0, c = t1 < ntx ? 4 << s.tx[t1].txl : 0;
        int nrow_all;
        const int b0 = hbd_scan(s, a + c, &nrow_all);
        if (t0 <= ntx) s.tx_base[t0] = (uint16_t)b0;
        if (t1 <= ntx) s.tx_base[t1] = (uint16_t)(b0 + a);
        if (t0 < ntx) s.txnz[t0] = 0;
        if (t1 < ntx) s.txnz[t1] = 0;
    }
    if (ntx > 0) {
        __syncthreads();
        const int nrow = s.tx_base[ntx];
        for (int it = tid; it < nrow; it += kHbdThreads) {
            const int t = hbd_find(s.tx_base, ntx, it);
            const HbdTx &x = s.tx[t];
            bool any;
            hbd_row_n(s, x.txl, job.coeffs32 + x.coeff, it - s.tx_base[t], x.plane, x.x, x.y, job.lossless, false,
                      any);
            if (any) s.txnz[t] = 1;
        }
        __syncthreads();
        for (int it = tid; it < nrow; it += kHbdThreads) {
            const int t = hbd_find(s.tx_base, ntx, it);
            const HbdTx &x = s.tx[t];
            if (s.txnz[t]) hbd_col_n(s, x.txl, it - s.tx_base[t], x.plane, x.x, x.y, job.lossless, false);
        }
    }
    __syncthreads();
}

/* Intra prediction of one n x n TX of plane p (tile position lx, ly; plane
 * position X0, Y0 in a pw x ph plane) by one warp, the FULL edge rules at 10
 * bits: 511 above and 513 on the left when unavailable, above-right only for
 * a 4x4 TX with have_right, samples past the plane's edge repeating the
 * last one inside. */
__device__ void hbd_intra_tx(HbdSmem &s, int p, int lx, int ly, int X0, int Y0, int pw, int ph, int n, int mode,
                             bool have_top, bool have_left, bool have_right, int lane, int warp)
{
    int32_t *edge = s.edge[warp];
    int32_t *above = edge + 1, *left = edge + 65;
    if (have_top) {
        const int want = n + ((n == 4 && have_right) ? 4 : 0);
        const int cnt = min(want, pw - X0);
        for (int i = lane; i < 2 * n; i += 32) above[i] = HT(s, p, lx + (i < cnt ? i : cnt - 1), ly - 1);
        if (lane == 0) above[-1] = have_left ? HT(s, p, lx - 1, ly - 1) : kHbdMid + 1;
    } else {
        for (int i = lane; i < 2 * n + 1; i += 32) edge[i] = kHbdMid - 1;
    }
    for (int i = lane; i < n; i += 32) left[i] = have_left ? HT(s, p, lx - 1, ly + min(i, ph - 1 - Y0)) : kHbdMid + 1;
    __syncwarp();
    int dc = kHbdMid;
    if (mode == 0) {
        const unsigned sa = __reduce_add_sync(0xffffffffu, lane < n ? (unsigned)above[lane] : 0u);
        const unsigned sl = __reduce_add_sync(0xffffffffu, lane < n ? (unsigned)left[lane] : 0u);
        if (have_top && have_left) dc = (int)((sa + sl + (unsigned)n) / (unsigned)(2 * n));
        else if (have_top) dc = (int)((sa + (unsigned)n / 2) / (unsigned)n);
        else if (have_left) dc = (int)((sl + (unsigned)n / 2) / (unsigned)n);
    }
    const int lg = n == 4 ? 2 : n == 8 ? 3 : n == 16 ? 4 : 5;
    for (int idx = lane; idx < n * n; idx += 32) {
        const int r = idx >> lg, c = idx & (n - 1);
        HT(s, p, lx + c, ly + r) = (uint16_t)full_pred<kHbdMax>(mode, r, c, n, above, left, dc);
    }
    __syncwarp();
}

/* One intra block by one warp: each plane's TXs in raster order, each
 * predicted and given its residual before the next. */
__device__ void hbd_intra_block(HbdSmem &s, const HbdBlk &b, int sbx, int sby, int lane, int warp)
{
    const cvp9_job_t &job = s.jc;
    const int gx = sbx + b.x, gy = sby + b.y;
    const int mi_col = gx >> 3, mi_row = gy >> 3;
    const bool left_ok = mi_col > full_tile_start(mi_col, job.mi_cols, job.log2_tile_cols);
    const bool resid = !(b.flags & 2) && b.txl <= 3;
    uint64_t off = b.coeff;
    for (int p = 0; p < 3; p++) {
        int txl, nx, ny, pbw;
        hbd_plane_layout(b, job, gx, gy, p, txl, nx, ny, pbw);
        const int n = 4 << txl, sz = n * n;
        const int mode = p ? (b.uvmode > 9 ? 0 : b.uvmode) : (b.ymode > 9 ? 0 : b.ymode);
        const int tx_type = (p == 0 && !job.lossless && txl < 3 && b.ymode < 10) ? c_tx_type[b.ymode] : 0;
        const int pw = p ? job.CW : job.W, ph = p ? job.CH : job.H;
        const int ox = p ? (b.x >> 1) : b.x, oy = p ? (b.y >> 1) : b.y;
        const int gox = p ? (gx >> 1) : gx, goy = p ? (gy >> 1) : gy;
        for (int ty = 0; ty < ny; ty++)
            for (int tx = 0; tx < nx; tx++) {
                const int lx = ox + tx * n, ly = oy + ty * n;
                hbd_intra_tx(s, p, lx, ly, gox + tx * n, goy + ty * n, pw, ph, n, mode, ty > 0 || mi_row > 0,
                             tx > 0 || left_ok, (tx + 1) * n < pbw, lane, warp);
                if (!resid) continue;
                if (off + (uint64_t)sz > (uint64_t)job.num_coeffs) { off = job.num_coeffs; continue; }
                const int32_t *X = job.coeffs32 + off;
                off += (uint64_t)sz;
                bool any = false;
                if (lane < n) hbd_row_n(s, txl, X, lane, p, lx, ly, job.lossless, tx_type == 2 || tx_type == 3, any);
                any = __any_sync(0xffffffffu, any);
                __syncwarp();
                if (any && lane < n) hbd_col_n(s, txl, lane, p, lx, ly, job.lossless, tx_type == 1 || tx_type == 3);
                __syncwarp();
            }
    }
}

} /* namespace */

__global__ void __launch_bounds__(kHbdThreads, 3) k_hbd_recon(const cvp9_job_t *__restrict__ jobs,
                                                              const uint32_t *__restrict__ tickets,
                                                              uint32_t n_tickets, uint32_t *ticket_counter)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    HbdSmem &s = *reinterpret_cast<HbdSmem *>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const cvp9_job_t &job = s.jc;
    for (;;) {
        __syncthreads();
        if (tid == 0) s.ticket = (int)atomicAdd(ticket_counter, 1u);
        __syncthreads();
        const int ticket = s.ticket;
        if (ticket >= (int)n_tickets) return;
        const uint32_t code = tickets[ticket];
        const cvp9_job_t *gj = jobs + (code >> 20);
        {
            const uint32_t *src = reinterpret_cast<const uint32_t *>(gj);
            uint32_t *dst = reinterpret_cast<uint32_t *>(&s.jc);
            for (int i = tid; i < (int)(sizeof(cvp9_job_t) / 4); i += kHbdThreads) dst[i] = src[i];
        }
        const int sb = (int)(code & 0xFFFFFu);
        const int g_sb_cols = gj->sb_cols;
        const int sbr = sb / g_sb_cols, sbc = sb - sbr * g_sb_cols;
        const int sbx = sbc * 64, sby = sbr * 64;
        const uint32_t *rg = gj->sb_range + 4 * sb;
        const uint32_t start = rg[0], end = rg[1], groups = rg[2];
        const bool layout_bad = (*(volatile uint32_t *)gj->status & CVP9_JOB_BAD_BLOCK) != 0;
        const bool bad = groups > 1 || end < start || end > gj->num_blocks ||
                         (groups && end - start > (uint32_t)kHbdMaxBlocks);
        int nb = (groups && !bad && !layout_bad) ? (int)(end - start) : 0;
        /* the tile at 512, no cell claimed */
        for (int i = tid; i < 65 * kHYP; i += kHbdThreads) s.ty[i] = kHbdMid;
        for (int i = tid; i < 2 * 33 * kHCP; i += kHbdThreads) (&s.tc[0][0])[i] = kHbdMid;
        for (int i = tid; i < 256; i += kHbdThreads) s.cell[i] = 0;
        __syncthreads();

        /* 1. blocks (each inside this SB, 4-aligned, 4..64 px, tx_size <= 3,
         * sub-8x8 ones on the 8x8 grid), and the 4x4 cells they write */
        bool my_intra = false, my_bad = false;
        if (tid < nb) {
            const vp9_macroblock_info_t g = job.blocks[start + tid];
            const int lx = (int)g.x - sbx, ly = (int)g.y - sby;
            const bool sub8 = g.width < 8 || g.height < 8;
            const int bw = sub8 ? 8 : g.width, bh = sub8 ? 8 : g.height;
            /* ... and a transform no larger than the block */
            my_bad = lx < 0 || ly < 0 || (lx & 3) || (ly & 3) || (g.width & 3) || (g.height & 3) || g.width < 4 ||
                     g.height < 4 || lx + g.width > 64 || ly + g.height > 64 || g.x >= job.W || g.y >= job.H ||
                     g.tx_size > 3 || (sub8 && ((lx & 7) || (ly & 7))) || (4 << g.tx_size) > min(bw, bh);
            HbdBlk b;
            b.x = (uint8_t)(my_bad ? 0 : lx);
            b.y = (uint8_t)(my_bad ? 0 : ly);
            b.w = g.width;
            b.h = g.height;
            b.cw = (uint8_t)max(0, min(bw, job.W - (int)g.x));
            b.ch = (uint8_t)max(0, min(bh, job.H - (int)g.y));
            b.ccw = (uint8_t)max(0, min(max(bw / 2, 4), job.CW - (int)g.x / 2));
            b.cch = (uint8_t)max(0, min(max(bh / 2, 4), job.CH - (int)g.y / 2));
            b.txl = g.tx_size;
            b.flags = (uint8_t)((g.is_intra ? 1 : 0) | (g.skip ? 2 : 0));
            b.ymode = g.y_mode;
            b.uvmode = g.uv_mode;
            b.ref0 = g.ref_frame[0];
            b.ref1 = g.is_intra ? 0 : g.ref_frame[1];
            b.mvx = g.mv[0][0];
            b.mvy = g.mv[0][1];
            b.mv1x = g.mv[1][0];
            b.mv1y = g.mv[1][1];
            b.coeff = g.coeff_offset;
            s.blk[tid] = b;
            my_intra = g.is_intra != 0;
        }
        if (__syncthreads_or(my_bad)) {
            if (tid == 0) atomicOr(job.status, (unsigned)CVP9_JOB_BAD_BLOCK);
            nb = 0;
            my_intra = false;
        }
        if (tid < nb) {
            /* cells of the luma region a block writes (a sub-8x8 block its 8x8) */
            const HbdBlk &b = s.blk[tid];
            for (int cy = b.y >> 2; cy < min(16, (b.y + b.ch + 3) >> 2); cy++)
                for (int cx = b.x >> 2; cx < min(16, (b.x + b.cw + 3) >> 2); cx++) {
                    atomicAdd(&s.cell[cy * 16 + cx], 1u);
                    s.owner[cy * 16 + cx] = (uint8_t)tid;
                }
        }
        __syncthreads();
        bool my_over = false;
        for (int i = tid; i < 256; i += kHbdThreads) my_over |= s.cell[i] > 1;
        bool overlap = __syncthreads_or(my_over) != 0;
        const bool any_intra = __syncthreads_or(my_intra) != 0;
        if (any_intra && !overlap) {
            /* dependency levels of the intra blocks: 1 + the deepest intra
             * block owning a sample of the row above, the column to the
             * left or the corner (inter blocks, reconstructed first, count
             * 0). A block reading samples of a block later in the list runs
             * the superblock in list order instead. */
            if (tid == 0) {
                int nlev = 0, bad = 0;
                for (int i = 0; i < nb; i++) {
                    const HbdBlk &b = s.blk[i];
                    s.lvl[i] = 0;
                    if (!(b.flags & 1)) continue;
                    int lv = 0;
                    const int cx0 = b.x >> 2, cy0 = b.y >> 2;
                    const int cx1 = (b.x + b.cw - 1) >> 2, cy1 = (b.y + b.ch - 1) >> 2;
                    auto dep = [&](int cx, int cy) {
                        if (cx < 0 || cy < 0 || cx > 15 || cy > 15) return;
                        const int c = cy * 16 + cx;
                        if (!s.cell[c]) return;
                        const int j = s.owner[c];
                        if (j > i) bad = 1;
                        else if (j < i) lv = max(lv, (int)s.lvl[j]);
                    };
                    for (int cx = cx0 - 1; cx <= cx1; cx++) dep(cx, cy0 - 1);
                    for (int cy = cy0; cy <= cy1; cy++) dep(cx0 - 1, cy);
                    s.lvl[i] = (uint8_t)(lv + 1);
                    nlev = max(nlev, lv + 1);
                }
                s.nlev = nlev;
                s.order_bad = bad;
            }
            __syncthreads();
            overlap = s.order_bad != 0;
        }

        /* 2. intra blocks read the neighbour SBs' samples: wait for them,
         * then load the row above (x = -1..63) and the column to the left */
        if (any_intra) {
            if (tid == 0) {
                bool ok = true;
                if (sbc > 0) ok &= wait_flag(job.sb_done + sb - 1, job.epoch);
                if (sbr > 0) ok &= wait_flag(job.sb_done + sb - job.sb_cols, job.epoch);
                if (sbr > 0 && sbc > 0) ok &= wait_flag(job.sb_done + sb - job.sb_cols - 1, job.epoch);
                if (!ok) atomicOr(job.status, (unsigned)CVP9_JOB_TIMEOUT);
            }
            __syncthreads();
            const uint16_t *Y = reinterpret_cast<const uint16_t *>(job.out);
            const uint16_t *U = Y + (size_t)job.W * job.H;
            const uint16_t *V = U + (size_t)job.CW * job.CH;
            if (sby > 0) {
                for (int i = tid - 1; i < 64; i += kHbdThreads) {
                    const int gx = sbx + i;
                    if (gx >= 0 && gx < job.W) HT(s, 0, i, -1) = __ldcg(Y + (size_t)(sby - 1) * job.W + gx);
                }
                for (int i = tid - 1; i < 32; i += kHbdThreads) {
                    const int gx = (sbx >> 1) + i;
                    if (gx >= 0 && gx < job.CW) {
                        HT(s, 1, i, -1) = __ldcg(U + (size_t)((sby >> 1) - 1) * job.CW + gx);
                        HT(s, 2, i, -1) = __ldcg(V + (size_t)((sby >> 1) - 1) * job.CW + gx);
                    }
                }
            }
            if (sbx > 0) {
                for (int i = tid; i < 64; i += kHbdThreads) {
                    const int gy = sby + i;
                    if (gy < job.H) HT(s, 0, -1, i) = __ldcg(Y + (size_t)gy * job.W + sbx - 1);
                }
                for (int i = tid; i < 32; i += kHbdThreads) {
                    const int gy = (sby >> 1) + i;
                    if (gy < job.CH) {
                        HT(s, 1, -1, i) = __ldcg(U + (size_t)gy * job.CW + (sbx >> 1) - 1);
                        HT(s, 2, -1, i) = __ldcg(V + (size_t)gy * job.CW + (sbx >> 1) - 1);
                    }
                }
            }
        }
        __syncthreads();

        /* 3. reconstruct: inter blocks together, then intra blocks in order;
         * overlapping blocks one by one in list order */
        if (!overlap) {
            hbd_inter_blocks(s, 0, nb, nb, sbx, sby);
            /* intra blocks level by level, the blocks of a level one warp each */
            const int nlev = any_intra ? s.nlev : 0;
            for (int L = 1; L <= nlev; L++) {
                int k = 0;
                for (int i = 0; i < nb; i++) {
                    if (s.lvl[i] != L) continue;
                    if (k++ % kHbdWarps == warp) hbd_intra_block(s, s.blk[i], sbx, sby, lane, warp);
                }
                __syncthreads();
            }
        } else {
            for (int i = 0; i < nb; i++) {
                if (s.blk[i].flags & 1) {
                    if (warp == 0) hbd_intra_block(s, s.blk[i], sbx, sby, lane, warp);
                    __syncthreads();
                } else {
                    hbd_inter_blocks(s, i, i + 1, nb, sbx, sby);
                }
            }
        }

        /* 4. write the tile (clipped to the frame) and release the SB */
        {
            uint16_t *Y = reinterpret_cast<uint16_t *>(job.out);
            uint16_t *U = Y + (size_t)job.W * job.H;
            uint16_t *V = U + (size_t)job.CW * job.CH;
            const int vw = min(64, job.W - sbx), vh = min(64, job.H - sby);
            for (int i = tid; i < 64 * 64; i += kHbdThreads) {
                const int r = i >> 6, c = i & 63;
                if (r < vh && c < vw) Y[(size_t)(sby + r) * job.W + sbx + c] = HT(s, 0, c, r);
            }
            const int cvw = min(32, job.CW - (sbx >> 1)), cvh = min(32, job.CH - (sby >> 1));
            for (int i = tid; i < 2 * 32 * 32; i += kHbdThreads) {
                const int p = i >> 10, k = i & 1023, r = k >> 5, c = k & 31;
                if (r < cvh && c < cvw) (p ? V : U)[(size_t)((sby >> 1) + r) * job.CW + (sbx >> 1) + c] = HT(s, 1 + p, c, r);
            }
        }
        if (tid == 0 && bad)
            atomicOr(job.status, (unsigned)CVP9_JOB_BAD_ORDER |
                                 ((groups && end >= start && end - start > (uint32_t)kHbdMaxBlocks) ? (unsigned)CVP9_JOB_TOO_MANY : 0u));
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            st_release(job.sb_done + sb, job.epoch);
        }
    }
}

__global__ void k_nv12_pack(const cvp9_job_t *__restrict__ jobs)
{
    const cvp9_job_t &job = jobs[blockIdx.y];
    if ((job.lf_tiled && !job.full) || !job.nv12) return;
    size_t ny = (size_t)job.W * job.H, nc = (size_t)job.CW * job.CH;
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ny) job.nv12[i] = job.out[i];
    if (i < nc) {
        size_t gy = i / job.CW, gx = i % job.CW;
        job.nv12[ny + gy * 2 * job.CW + 2 * gx] = job.out[ny + i];
        job.nv12[ny + gy * 2 * job.CW + 2 * gx + 1] = job.out[ny + nc + i];
    }
}

/* ── Coefficient upload over PCIe, REFCPU ────────────────────────────────
 * The dense coefficient array interleaves each block's luma TXs with its
 * chroma TXs; REFCPU reads only the luma ones (vp9_reconstruct.c:336-360).
 * A warp per block copies that span, [coeff_offset, + (cw/n)(ch/n) n^2),
 * from the page-locked host array to the same offset of the device array
 * with 16-byte reads when both sides share their alignment; the chroma
 * coefficients never cross the bus. */
__global__ void __launch_bounds__(256) k_gather_luma(const cvp9_job_t *__restrict__ jobs, uint32_t *bytes)
{
    const cvp9_job_t &job = jobs[blockIdx.y];
    const int16_t *src = job.coeffs_src;
    if (!src) return;
    int16_t *dst = const_cast<int16_t *>(job.coeffs);
    const int lane = threadIdx.x & 31;
    uint32_t moved = 0;
    for (uint32_t bi = blockIdx.x * 8u + (threadIdx.x >> 5); bi < job.num_blocks; bi += gridDim.x * 8u) {
        const uint32_t *g = reinterpret_cast<const uint32_t *>(job.blocks + bi);
        const uint32_t g0 = g[0], g1 = g[1], g5 = g[5], g6 = g[6];
        const int x = (int)(g0 & 0xffffu), y = (int)(g0 >> 16);
        const int w = (int)(g1 & 0xffu), h = (int)((g1 >> 8) & 0xffu), tx = (int)((g1 >> 16) & 0xffu);
        if ((g5 & 0xffu) || tx > 3 || x >= job.W || y >= job.H) continue;
        const int n = 4 << tx;
        const int cw = min(w, job.W - x), ch = min(h, job.H - y);
        const uint64_t a = g6;
        uint64_t e = a + (uint64_t)((cw / n) * (ch / n)) * (uint64_t)(n * n);
        if (e > job.num_coeffs) e = job.num_coeffs;
        if (a >= e) continue;
        const char *s = reinterpret_cast<const char *>(src + a);
        char *d = reinterpret_cast<char *>(dst + a);
        const uint64_t len = (e - a) * 2;
        if ((((uintptr_t)s ^ (uintptr_t)d) & 15) == 0) {
            const uint64_t head = (16 - ((uintptr_t)s & 15)) & 15;
            const uint64_t h2 = head < len ? head : len;
            for (uint64_t o = 2 * lane; o < h2; o += 64)
                *reinterpret_cast<int16_t *>(d + o) = *reinterpret_cast<const int16_t *>(s + o);
            const uint64_t nv = (len - h2) / 16;
            const uint4 *sv = reinterpret_cast<const uint4 *>(s + h2);
            uint4 *dv = reinterpret_cast<uint4 *>(d + h2);
            for (uint64_t v = lane; v < nv; v += 32) dv[v] = sv[v];
            for (uint64_t o = h2 + nv * 16 + 2 * lane; o < len; o += 64)
                *reinterpret_cast<int16_t *>(d + o) = *reinterpret_cast<const int16_t *>(s + o);
        } else {
            for (uint64_t o = 2 * lane; o < len; o += 64)
                *reinterpret_cast<int16_t *>(d + o) = *reinterpret_cast<const int16_t *>(s + o);
        }
        moved += (uint32_t)len;
    }
    if (lane == 0 && moved) atomicAdd(bytes, moved);
}

/* Sparse coefficient upload: the caller's (index, value) list of a frame
 * is scattered into its zeroed dense array, which the reconstruction then
 * reads exactly as if the dense array had been uploaded. */
__global__ void __launch_bounds__(256) k_scatter_coeffs(const cvp9_job_t *__restrict__ jobs)
{
    const cvp9_job_t &job = jobs[blockIdx.y];
    const uint32_t n = job.sp_n;
    if (job.sp_val32) {
        /* profile 2: int32 dequantised values into coeffs32 */
        int32_t *dst = const_cast<int32_t *>(job.coeffs32);
        for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
            const uint32_t p = job.sp_pos[k];
            if (p < job.num_coeffs) dst[p] = job.sp_val32[k];
        }
        return;
    }
    int16_t *dst = const_cast<int16_t *>(job.coeffs);
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t p = job.sp_pos[k];
        if (p < job.num_coeffs) dst[p] = job.sp_val[k];
    }
}

/* Packed coefficient upload (format of cvp9_pack_coeffs): a CTA per (page,
 * frame) rebuilds 65536 coefficients of the dense array — a dense page is
 * copied, an entry page is zero-filled and then scattered. A malformed
 * page (data past the buffer, counts out of range) is left alone and sets
 * bit (job index) % 32 of *err, which the host reads with the step. */
__global__ void __launch_bounds__(256) k_unpack_coeffs(const cvp9_job_t *__restrict__ jobs, uint32_t *err)
{
    const cvp9_job_t &job = jobs[blockIdx.y];
    const uint32_t *pk = job.packed;
    if (!pk) return;
    const uint32_t nw = job.packed_words, np = nw ? pk[0] : 0u;
    if (1u + 2u * (uint64_t)np > nw) {
        if (threadIdx.x == 0 && blockIdx.x == 0) atomicOr(err + blockIdx.y, 1u);
        return;
    }
    for (uint32_t p = blockIdx.x; p < np; p += gridDim.x) {
        const uint32_t base = p << 16;
        if (p >= 65536u || base >= job.num_coeffs) break;
        const uint32_t st = pk[1 + 2 * p], cnt = pk[2 + 2 * p];
        const uint32_t s0 = st & 0x7fffffffu;
        const uint32_t len = min(65536u, job.num_coeffs - base);
        const bool dense = st >> 31;
        const uint64_t words = dense ? ((uint64_t)len + 1) / 2 : cnt;
        if ((s0 & 3u) || (dense && cnt != len) || (!dense && cnt > (len + 1) / 2) || s0 + words > nw) {
            if (threadIdx.x == 0) atomicOr(err + blockIdx.y, 1u);
            continue;
        }
        int16_t *dst = const_cast<int16_t *>(job.coeffs) + base;     /* 16-byte aligned */
        const uint32_t *src = pk + s0;                               /* 16-byte aligned */
        uint4 *d4 = reinterpret_cast<uint4 *>(dst);
        const uint32_t nv = len >> 3;
        if (dense) {
            const uint4 *s4 = reinterpret_cast<const uint4 *>(src);
            for (uint32_t v = threadIdx.x; v < nv; v += blockDim.x) d4[v] = __ldg(s4 + v);
            const int16_t *s16 = reinterpret_cast<const int16_t *>(src);
            for (uint32_t k = nv * 8 + threadIdx.x; k < len; k += blockDim.x) dst[k] = s16[k];
        } else {
            for (uint32_t v = threadIdx.x; v < nv; v += blockDim.x) d4[v] = make_uint4(0u, 0u, 0u, 0u);
            for (uint32_t k = nv * 8 + threadIdx.x; k < len; k += blockDim.x) dst[k] = 0;
            __syncthreads();
            for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x) {
                const uint32_t e = __ldg(src + k), o = e & 0xffffu;
                if (o < len) dst[o] = (int16_t)(e >> 16);
            }
        }
        __syncthreads();
    }
}

/* ── C-ABI launch shims ─────────────────────────────────────────────────── */

extern "C" {

size_t cvp9k_recon_smem_bytes(void) { return sizeof(ReconSmem); }

int cvp9k_launch_scatter(const cvp9_job_t *jobs, int njobs, uint32_t max_n, cudaStream_t st)
{
    if (njobs <= 0 || max_n == 0) return 0;
    unsigned gx = (max_n + 255u) / 256u;
    if (gx > 4096u) gx = 4096u;
    k_scatter_coeffs<<<dim3(gx, (unsigned)njobs), 256, 0, st>>>(jobs);
    return (int)cudaGetLastError();
}

int cvp9k_launch_unpack(const cvp9_job_t *jobs, int njobs, uint32_t max_pages, uint32_t *err, cudaStream_t st)
{
    if (njobs <= 0 || max_pages == 0) return 0;
    const unsigned gx = max_pages < 65535u ? max_pages : 65535u;
    k_unpack_coeffs<<<dim3(gx, (unsigned)njobs), 256, 0, st>>>(jobs, err);
    return (int)cudaGetLastError();
}

/* One job per blockIdx.y; 16-byte streaming copies (both ends are
 * 256-byte aligned arena ranges), the tail bytewise. */
__global__ void __launch_bounds__(256) k_collect(const cvp9_job_t *__restrict__ jobs)
{
    const cvp9_job_t &job = jobs[blockIdx.y];
    uint8_t *dst = job.dl;
    if (!dst) return;
    const uint8_t *src = job.out;
    const size_t n = (size_t)job.W * job.H + 2 * (size_t)job.CW * job.CH;
    const size_t n16 = n >> 4;
    const uint4 *s4 = reinterpret_cast<const uint4 *>(src);
    uint4 *d4 = reinterpret_cast<uint4 *>(dst);
    for (size_t i = (size_t)blockIdx.x * 256 + threadIdx.x; i < n16; i += (size_t)gridDim.x * 256)
        __stcs(d4 + i, __ldcs(s4 + i));
    if (blockIdx.x == 0)
        for (size_t i = (n16 << 4) + threadIdx.x; i < n; i += 256) dst[i] = src[i];
}

int cvp9k_launch_collect(const cvp9_job_t *jobs, int njobs, size_t max_bytes, cudaStream_t st)
{
    if (njobs <= 0 || !max_bytes) return 0;
    /* about four CTAs per SM in all, at least one per 256 KB of a frame */
    size_t gx = (max_bytes + (256u << 10) - 1) >> 18;
    const size_t want = (size_t)(4 * 148 + njobs - 1) / (size_t)njobs;
    if (gx > want) gx = want;
    if (gx < 1) gx = 1;
    k_collect<<<dim3((unsigned)gx, (unsigned)njobs), 256, 0, st>>>(jobs);
    return (int)cudaGetLastError();
}

int cvp9k_launch_gather(const cvp9_job_t *jobs, int njobs, int max_blocks, uint32_t *bytes, cudaStream_t st)
{
    if (njobs <= 0 || max_blocks <= 0) return 0;
    int gx = (max_blocks + 7) / 8;
    if (gx > 2048) gx = 2048;
    k_gather_luma<<<dim3((unsigned)gx, (unsigned)njobs), 256, 0, st>>>(jobs, bytes);
    return (int)cudaGetLastError();
}

int cvp9k_upload_dct_basis(const double *basis, int count)
{
    if (count != 16 + 64 + 256 + 1024) return -1;
    if (cudaMemcpyToSymbol(c_dct, basis, sizeof(double) * (size_t)count) != cudaSuccess) return -1;
    return cudaMemcpyToSymbol(g_dct, basis, sizeof(double) * (size_t)count) == cudaSuccess ? 0 : -1;
}

int cvp9k_configure(void)
{
    {
        static const int taps[16][8] = CVP9_SUBPEL_REGULAR_INIT;
        uint32_t pk[16][2];
        for (int f = 0; f < 16; f++)
            for (int h = 0; h < 2; h++) {
                uint32_t w = 0;
                for (int t = 0; t < 4; t++) w |= (uint32_t)(uint8_t)(int8_t)taps[f][4 * h + t] << (8 * t);
                pk[f][h] = w;
            }
        if (cudaMemcpyToSymbol(c_subpel_pk, pk, sizeof(pk)) != cudaSuccess) return -1;
    }
    {
        static const int taps4[4][16][8] = { CVP9_SUBPEL_REGULAR_INIT, CVP9_SUBPEL_SMOOTH_INIT,
                                             CVP9_SUBPEL_SHARP_INIT, CVP9_SUBPEL_BILINEAR_INIT };
        uint32_t pk[4][16][2];
        for (int k = 0; k < 4; k++)
            for (int f = 0; f < 16; f++)
                for (int h = 0; h < 2; h++) {
                    uint32_t w = 0;
                    for (int t = 0; t < 4; t++) {
                        const int v = taps4[k][f][4 * h + t];
                        /* phase 0 (the centre tap alone, 128) is not packed:
                         * tap8 takes the centre sample for it */
                        if (f && (v < -128 || v > 127)) return -1;
                        w |= (uint32_t)(uint8_t)(int8_t)v << (8 * t);
                    }
                    pk[k][f][h] = w;
                }
        if (cudaMemcpyToSymbol(c_subpel4_pk, pk, sizeof(pk)) != cudaSuccess) return -1;
    }
    size_t smem = sizeof(ReconSmem);
    if (cudaFuncSetAttribute(k_recon<CVP9_ARITH_REFCPU>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return -1;
    if (cudaFuncSetAttribute(k_recon<CVP9_ARITH_SPEC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return -1;
    /* all of the unified L1/shared storage as shared memory: three CTAs per SM */
    cudaFuncSetAttribute(k_recon<CVP9_ARITH_REFCPU>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaFuncSetAttribute(k_recon<CVP9_ARITH_SPEC>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaFuncSetAttribute(k_inter<CVP9_ARITH_REFCPU, 5>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaFuncSetAttribute(k_inter<CVP9_ARITH_REFCPU, 6>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaFuncSetAttribute(k_inter<CVP9_ARITH_SPEC, 5>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaFuncSetAttribute(k_inter<CVP9_ARITH_SPEC, 6>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (cudaFuncSetAttribute(k_hbd_recon, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(HbdSmem)) != cudaSuccess)
        return -1;
    cudaFuncSetAttribute(k_hbd_recon, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    /* Load every kernel the launcher can pick now. With lazy module loading
     * (the CUDA 12 default) a kernel's code is loaded at its first launch,
     * which stalls the device for tens of milliseconds; the tuner's first
     * trial of an inter path would otherwise take that stall inside a
     * serving step. */
    const void *fns[] = {
        (const void *)k_scan_blocks, (const void *)k_lf_mimap, (const void *)k_compact,
        (const void *)k_recon<CVP9_ARITH_REFCPU>, (const void *)k_recon<CVP9_ARITH_SPEC>,
        (const void *)k_inter<CVP9_ARITH_REFCPU, 5>, (const void *)k_inter<CVP9_ARITH_REFCPU, 6>,
        (const void *)k_inter<CVP9_ARITH_SPEC, 5>, (const void *)k_inter<CVP9_ARITH_SPEC, 6>,
        (const void *)k_pred<CVP9_ARITH_SPEC, kPredMinB>, (const void *)k_pred<CVP9_ARITH_REFCPU, kPredMinB>,
        (const void *)k_pred<CVP9_ARITH_REFCPU, kPredMinB, true>,
        (const void *)k_resid<CVP9_ARITH_SPEC, kResidMinB, false>,
        (const void *)k_resid<CVP9_ARITH_REFCPU, kResidMinB, true>,
        (const void *)k_resid<CVP9_ARITH_REFCPU, kResidMinB, false>,
        (const void *)k_resid<CVP9_ARITH_REFCPU, kResid8MinB, true, 1>,
        (const void *)k_resid<CVP9_ARITH_REFCPU, kResidMinB, true, 2>,
        (const void *)k_lf_full<uint8_t, 0>, (const void *)k_nv12_pack,
        (const void *)k_loopfilter<CVP9_ARITH_SPEC, 32>, (const void *)k_loopfilter<CVP9_ARITH_REFCPU, 32>,
        (const void *)k_loopfilter<CVP9_ARITH_SPEC, 64>, (const void *)k_loopfilter<CVP9_ARITH_REFCPU, 64>,
        (const void *)k_lf_strip<CVP9_ARITH_SPEC>, (const void *)k_lf_strip<CVP9_ARITH_REFCPU>,
        (const void *)k_lf_flat_h, (const void *)k_lf_flat_v,
        (const void *)k_gather_luma, (const void *)k_scatter_coeffs, (const void *)k_unpack_coeffs,
        (const void *)k_collect, (const void *)k_hbd_recon, (const void *)k_lf_full<uint16_t, 2>,
    };
    for (size_t i = 0; i < sizeof(fns) / sizeof(fns[0]); i++) {
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, fns[i]) != cudaSuccess) return -1;
    }
    return 0;
}

int cvp9k_hbd_ctas_per_sm(void)
{
    int n = 0;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_hbd_recon, kHbdThreads, sizeof(HbdSmem)) == cudaSuccess
        ? n : -1;
}

int cvp9k_lf_full_ctas_per_sm(void)
{
    int n = 0;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_lf_full<uint8_t, 0>, 128, 0) == cudaSuccess ? n : -1;
}

int cvp9k_recon_ctas_per_sm(int arith)
{
    int n = 0;
    cudaError_t e = arith == CVP9_ARITH_SPEC
        ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_recon<CVP9_ARITH_SPEC>, kThreads, sizeof(ReconSmem))
        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_recon<CVP9_ARITH_REFCPU>, kThreads, sizeof(ReconSmem));
    return e == cudaSuccess ? n : -1;
}

/* Timing events become event-record nodes when the stream is being captured. */
static cudaError_t mark(cudaEvent_t ev, cudaStream_t st, bool capturing)
{
    if (!ev) return cudaSuccess;
    return capturing ? cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal) : cudaEventRecord(ev, st);
}

int cvp9k_launch_frame(const cvp9k_launch_t *L, cudaStream_t st)
{
    if (!L || L->njobs <= 0) return (int)cudaErrorInvalidValue;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(st, &cap);
    if (e != cudaSuccess) return (int)e;
    const bool capturing = cap == cudaStreamCaptureStatusActive;
    if ((e = mark(L->ev[0], st, capturing)) != cudaSuccess) return (int)e;
    if (L->hbd) {
        /* profile 2: scan, mode-info map, k_hbd_recon, the 10-bit VP9 filter */
        if (L->max_blocks > 0) {
            dim3 g((unsigned)((L->max_blocks + 255) / 256), (unsigned)L->njobs);
            k_scan_blocks<<<g, 256, 0, st>>>(L->jobs);
            k_lf_mimap<<<g, 256, 0, st>>>(L->jobs);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
        if ((e = mark(L->ev[1], st, capturing)) != cudaSuccess) return (int)e;
        if (L->n_tickets > 0) {
            int grid = L->recon_ctas > 0 ? L->recon_ctas : (int)L->n_tickets;
            if (grid > (int)L->n_tickets) grid = (int)L->n_tickets;
            k_hbd_recon<<<grid, kHbdThreads, sizeof(HbdSmem), st>>>(L->jobs, L->tickets, L->n_tickets,
                                                                    L->ticket_counter);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
        if ((e = mark(L->ev[2], st, capturing)) != cudaSuccess) return (int)e;
        if (L->lf_tickets > 0 && L->lf_counter) {
            const int grid = L->lf_ctas > 0 && L->lf_ctas < (int)L->lf_tickets ? L->lf_ctas : (int)L->lf_tickets;
            k_lf_full<uint16_t, 2><<<grid, 128, 0, st>>>(L->jobs, L->njobs, L->lf_tickets, L->lf_counter);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
        return (int)mark(L->ev[3], st, capturing);
    }
    if (L->max_blocks > 0 || L->scan_ctas > 0) {
        int gx = L->scan_ctas > 0 ? L->scan_ctas : (L->max_blocks + 255) / 256;
        dim3 g((unsigned)gx, (unsigned)L->njobs);
        k_scan_blocks<<<g, 256, 0, st>>>(L->jobs);
        if (L->full) k_lf_mimap<<<g, 256, 0, st>>>(L->jobs);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
    if ((e = mark(L->ev[1], st, capturing)) != cudaSuccess) return (int)e;
    if (L->n_tickets > 0) {
        int grid = L->recon_ctas > 0 ? L->recon_ctas : (int)L->n_tickets;
        if (grid > (int)L->n_tickets) grid = (int)L->n_tickets;
        size_t smem = sizeof(ReconSmem);
        const bool fast = L->general && L->general_tickets && L->n_general;
        if (fast) {
            const unsigned fg = (L->n_tickets + kFastWarps - 1) / kFastWarps;
            /* the count of general superblocks that k_inter raises */
            if ((e = cudaMemsetAsync(L->n_general + 1, 0, 4, st)) != cudaSuccess) return (int)e;
            const size_t fs = kFastWarps * sizeof(FastSmem);
            const bool spec = L->arith == CVP9_ARITH_SPEC;
            if (L->inter_variant >= 3 && spec) {       /* SPEC has one split (3; 4 and 5 are REFCPU forms) */
                k_pred<CVP9_ARITH_SPEC, kPredMinB><<<fg, kFastWarps * 32, kFastWarps * sizeof(PredSmem), st>>>(
                    L->jobs, L->tickets, L->n_tickets, L->general);
                k_resid<CVP9_ARITH_SPEC, kResidMinB, false><<<fg, kFastWarps * 32, kFastWarps * sizeof(ResidSmem), st>>>(
                    L->jobs, L->tickets, L->n_tickets, L->general);
            } else if (L->inter_variant == 5) {
                /* REFCPU: k_pred marks superblocks with TXs other than 8x8;
                 * the 8x8-only residual kernel carries no larger transform */
                k_pred<CVP9_ARITH_REFCPU, kPredMinB, true><<<fg, kFastWarps * 32, kFastWarps * sizeof(PredSmem), st>>>(
                    L->jobs, L->tickets, L->n_tickets, L->general);
                k_resid<CVP9_ARITH_REFCPU, kResid8MinB, true, 1>
                    <<<fg, kFastWarps * 32, kFastWarps * sizeof(ResidSmem), st>>>(L->jobs, L->tickets, L->n_tickets,
                                                                               L->general);
                k_resid<CVP9_ARITH_REFCPU, kResidMinB, true, 2>
                    <<<fg, kFastWarps * 32, kFastWarps * sizeof(ResidSmem), st>>>(L->jobs, L->tickets, L->n_tickets,
                                                                               L->general);
            } else if (L->inter_variant == 3 || L->inter_variant == 4) {
                k_pred<CVP9_ARITH_REFCPU, kPredMinB><<<fg, kFastWarps * 32, kFastWarps * sizeof(PredSmem), st>>>(
                    L->jobs, L->tickets, L->n_tickets, L->general);
                if (L->inter_variant == 4)
                    k_resid<CVP9_ARITH_REFCPU, kResidMinB, true><<<fg, kFastWarps * 32, kFastWarps * sizeof(ResidSmem), st>>>(
                        L->jobs, L->tickets, L->n_tickets, L->general);
                else
                    k_resid<CVP9_ARITH_REFCPU, kResidMinB, false><<<fg, kFastWarps * 32, kFastWarps * sizeof(ResidSmem), st>>>(
                        L->jobs, L->tickets, L->n_tickets, L->general);
            } else if (L->inter_variant == 2) {
                if (spec) k_inter<CVP9_ARITH_SPEC, 6><<<fg, kFastWarps * 32, fs, st>>>(L->jobs, L->tickets, L->n_tickets, L->general);
                else k_inter<CVP9_ARITH_REFCPU, 6><<<fg, kFastWarps * 32, fs, st>>>(L->jobs, L->tickets, L->n_tickets, L->general);
            } else {
                if (spec) k_inter<CVP9_ARITH_SPEC, 5><<<fg, kFastWarps * 32, fs, st>>>(L->jobs, L->tickets, L->n_tickets, L->general);
                else k_inter<CVP9_ARITH_REFCPU, 5><<<fg, kFastWarps * 32, fs, st>>>(L->jobs, L->tickets, L->n_tickets, L->general);
            }
            k_compact<<<1, 1024, 0, st>>>(L->tickets, L->general, L->n_tickets, L->general_tickets, L->n_general);
            if (spec)
                k_recon<CVP9_ARITH_SPEC><<<grid, kThreads, smem, st>>>(L->jobs, L->general_tickets, L->n_tickets,
                                                                        L->ticket_counter, L->n_general,
                                                                        L->warp_levels);
            else
                k_recon<CVP9_ARITH_REFCPU><<<grid, kThreads, smem, st>>>(L->jobs, L->general_tickets, L->n_tickets,
                                                                          L->ticket_counter, L->n_general,
                                                                          L->warp_levels);
        } else if (L->arith == CVP9_ARITH_SPEC) {
            k_recon<CVP9_ARITH_SPEC><<<grid, kThreads, smem, st>>>(L->jobs, L->tickets, L->n_tickets, L->ticket_counter,
                                                                    nullptr, L->warp_levels);
        } else {
            k_recon<CVP9_ARITH_REFCPU><<<grid, kThreads, smem, st>>>(L->jobs, L->tickets, L->n_tickets, L->ticket_counter,
                                                                      nullptr, L->warp_levels);
        }
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
    if ((e = mark(L->ev[2], st, capturing)) != cudaSuccess) return (int)e;
    if (L->full) {
        if (L->lf_tickets > 0 && L->lf_counter) {
            const int grid = L->lf_ctas > 0 && L->lf_ctas < (int)L->lf_tickets ? L->lf_ctas : (int)L->lf_tickets;
            k_lf_full<uint8_t, 0><<<grid, 128, 0, st>>>(L->jobs, L->njobs, L->lf_tickets, L->lf_counter);
        }
        if (L->full_nv12_max_px > 0) {
            long long n = L->full_nv12_max_px;
            k_nv12_pack<<<dim3((unsigned)((n + 255) / 256), (unsigned)L->njobs), 256, 0, st>>>(L->jobs);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
        return (int)mark(L->ev[3], st, capturing);
    }
    if (L->lf_tiles_x > 0 && L->lf_tiles_y > 0) {
        /* lf_tiles_y counts 64-row tiles; 32-row tiles need twice as many
         * (one more covers the 4-row shift) */
        if (L->lf_tile_h == 32) {
            dim3 g((unsigned)L->lf_tiles_x, (unsigned)(2 * L->lf_tiles_y), (unsigned)L->njobs);
            if (L->arith == CVP9_ARITH_SPEC) k_loopfilter<CVP9_ARITH_SPEC, 32><<<g, 256, 0, st>>>(L->jobs);
            else k_loopfilter<CVP9_ARITH_REFCPU, 32><<<g, 256, 0, st>>>(L->jobs);
        } else {
            dim3 g((unsigned)L->lf_tiles_x, (unsigned)L->lf_tiles_y, (unsigned)L->njobs);
            if (L->arith == CVP9_ARITH_SPEC) k_loopfilter<CVP9_ARITH_SPEC, 64><<<g, 256, 0, st>>>(L->jobs);
            else k_loopfilter<CVP9_ARITH_REFCPU, 64><<<g, 256, 0, st>>>(L->jobs);
        }
    }
    if (L->lf_strips_x > 0 && L->lf_strips_y > 0) {
        dim3 g((unsigned)L->lf_strips_x, (unsigned)L->lf_strips_y, (unsigned)L->njobs);
        if (L->arith == CVP9_ARITH_SPEC) k_lf_strip<CVP9_ARITH_SPEC><<<g, 128, 0, st>>>(L->jobs);
        else k_lf_strip<CVP9_ARITH_REFCPU><<<g, 128, 0, st>>>(L->jobs);
    }
    if (L->flat_lf_max_w > 0) {
        long long nh = (long long)((L->flat_lf_max_h + 7) / 8) * L->flat_lf_max_w;
        long long nv = (long long)((L->flat_lf_max_w + 7) / 8) * L->flat_lf_max_h;
        int refcpu = L->arith == CVP9_ARITH_REFCPU;
        k_lf_flat_h<<<dim3((unsigned)((nh + 255) / 256), (unsigned)L->njobs), 256, 0, st>>>(L->jobs, refcpu);
        k_lf_flat_v<<<dim3((unsigned)((nv + 255) / 256), (unsigned)L->njobs), 256, 0, st>>>(L->jobs, refcpu);
        if (L->flat_nv12) {
            long long n = (long long)L->flat_lf_max_w * L->flat_lf_max_h;
            k_nv12_pack<<<dim3((unsigned)((n + 255) / 256), (unsigned)L->njobs), 256, 0, st>>>(L->jobs);
        }
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
    return (int)mark(L->ev[3], st, capturing);
}

} /* extern "C" */
