/* Host-side packing of dense coefficient arrays before the upload (format
 * and contract in cvp9_batch.h; k_unpack_coeffs in recon.cu rebuilds the
 * dense array on the device).
 *
 * The parser's arrays are dense int16, mostly zeros, and a large step's
 * upload is bound by the PCIe link. Packing keeps the nonzero coefficients
 * the reconstruction reads, as 32-bit (offset in page) | (value << 16)
 * entries per 65536-coefficient page; a page whose entries would outgrow
 * its dense form is sent dense. The scan is the host cost: 16 or 8
 * coefficients per step with AVX-512 / AVX2 compress, or a scalar loop that
 * skips zero 64-bit words; $CVP9_PACK_ISA=scalar|avx2|avx512 pins one (the
 * tests compare them). */
#include "cvp9_batch.h"
#include "recon_job.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define PAGE_SHIFT 16
#define PAGE_LEN   (1u << PAGE_SHIFT)
#define TAIL_SLACK 16u   /* vector stores may write 15 words past the data */

static inline uint32_t align4(uint32_t x) { return (x + 3u) & ~3u; }

size_t cvp9_pack_bound_words(uint32_t n)
{
    const uint32_t np = (uint32_t)(((uint64_t)n + PAGE_LEN - 1) >> PAGE_SHIFT);
    size_t w = align4(1u + 2u * np);
    if (np) {
        const uint32_t last = n - ((np - 1) << PAGE_SHIFT);
        w += (size_t)(np - 1) * align4(PAGE_LEN / 2) + align4((last + 1) / 2);
    }
    return w + TAIL_SLACK;
}

/* entries (off + k) | (v << 16) for the nonzero src[k], k in [0, m);
 * returns the new end of out */
typedef uint32_t *(*scan_fn)(const int16_t *src, uint32_t m, uint32_t off, uint32_t *out);

static inline uint32_t entry(uint32_t off, int16_t v) { return off | (uint32_t)(uint16_t)v << 16; }

static uint32_t *scan_scalar(const int16_t *src, uint32_t m, uint32_t off, uint32_t *out)
{
    uint32_t k = 0;
    for (; k < m && ((uintptr_t)(src + k) & 7); k++)
        if (src[k]) *out++ = entry(off + k, src[k]);
    for (; k + 4 <= m; k += 4) {
        uint64_t v;
        memcpy(&v, src + k, 8);
        if (!v) continue;
        for (uint32_t j = 0; j < 4; j++)
            if (src[k + j]) *out++ = entry(off + k + j, src[k + j]);
    }
    for (; k < m; k++)
        if (src[k]) *out++ = entry(off + k, src[k]);
    return out;
}

#if defined(__x86_64__)
#include <immintrin.h>

/* g_lut[m]: the positions of m's set bits, in order (permute indices) */
static uint8_t g_lut[256][8];

__attribute__((target("avx2,popcnt")))
static uint32_t *scan_avx2(const int16_t *src, uint32_t m, uint32_t off, uint32_t *out)
{
    const __m256i lane = _mm256_setr_epi32(0, 1, 2, 3, 4, 5, 6, 7);
    const __m128i zero = _mm_setzero_si128();
    uint32_t k = 0;
    for (; k + 32 <= m; k += 32) {
        const __m256i a = _mm256_loadu_si256((const __m256i *)(src + k));
        const __m256i b = _mm256_loadu_si256((const __m256i *)(src + k + 16));
        const __m256i ab = _mm256_or_si256(a, b);
        if (_mm256_testz_si256(ab, ab)) continue;
        for (uint32_t h = 0; h < 32; h += 8) {
            const __m128i v = _mm_loadu_si128((const __m128i *)(src + k + h));
            const __m128i z = _mm_cmpeq_epi16(v, zero);
            const unsigned nz = ~(unsigned)_mm_movemask_epi8(_mm_packs_epi16(z, zero)) & 0xffu;
            const __m256i ent = _mm256_or_si256(_mm256_slli_epi32(_mm256_cvtepi16_epi32(v), 16),
                                                _mm256_add_epi32(_mm256_set1_epi32((int)(off + k + h)), lane));
            const __m256i idx = _mm256_cvtepu8_epi32(_mm_loadl_epi64((const __m128i *)g_lut[nz]));
            _mm256_storeu_si256((__m256i *)out, _mm256_permutevar8x32_epi32(ent, idx));
            out += __builtin_popcount(nz);
        }
    }
    return k < m ? scan_scalar(src + k, m - k, off + k, out) : out;
}

__attribute__((target("avx512f,avx512bw,avx512vl,popcnt")))
static uint32_t *scan_avx512(const int16_t *src, uint32_t m, uint32_t off, uint32_t *out)
{
    const __m512i lane = _mm512_setr_epi32(0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15);
    uint32_t k = 0;
    for (; k + 32 <= m; k += 32) {
        const __m512i v = _mm512_loadu_si512((const void *)(src + k));
        const __mmask32 nz = _mm512_test_epi16_mask(v, v);
        if (!nz) continue;
        const __m512i e0 = _mm512_or_si512(_mm512_slli_epi32(_mm512_cvtepi16_epi32(_mm512_castsi512_si256(v)), 16),
                                           _mm512_add_epi32(_mm512_set1_epi32((int)(off + k)), lane));
        _mm512_storeu_si512((void *)out, _mm512_maskz_compress_epi32((__mmask16)nz, e0));
        out += __builtin_popcount((unsigned)(nz & 0xffffu));
        const __m512i e1 = _mm512_or_si512(_mm512_slli_epi32(_mm512_cvtepi16_epi32(_mm512_extracti64x4_epi64(v, 1)), 16),
                                           _mm512_add_epi32(_mm512_set1_epi32((int)(off + k + 16)), lane));
        _mm512_storeu_si512((void *)out, _mm512_maskz_compress_epi32((__mmask16)(nz >> 16), e1));
        out += __builtin_popcount((unsigned)(nz >> 16));
    }
    return k < m ? scan_scalar(src + k, m - k, off + k, out) : out;
}
#endif

static scan_fn g_scan = scan_scalar;
static pthread_once_t g_scan_once = PTHREAD_ONCE_INIT;

static void scan_init(void)
{
    const char *isa = getenv("CVP9_PACK_ISA");
    g_scan = scan_scalar;
#if defined(__x86_64__)
    for (int mk = 0; mk < 256; mk++) {
        int j = 0;
        for (int b = 0; b < 8; b++) if (mk >> b & 1) g_lut[mk][j++] = (uint8_t)b;
        for (; j < 8; j++) g_lut[mk][j] = 0;
    }
    __builtin_cpu_init();
    const int has512 = __builtin_cpu_supports("avx512f") && __builtin_cpu_supports("avx512bw") &&
                       __builtin_cpu_supports("avx512vl");
    const int has2 = __builtin_cpu_supports("avx2");
    if (isa && !strcmp(isa, "scalar")) return;
    if (isa && !strcmp(isa, "avx2")) { if (has2) g_scan = scan_avx2; return; }
    if (has512) g_scan = scan_avx512;
    else if (has2) g_scan = scan_avx2;
#else
    (void)isa;
#endif
}

typedef struct {
    const int16_t *src;
    uint32_t      *out;
    uint32_t       n, np;
    uint32_t       p;       /* page being filled */
    uint32_t       start;   /* its first data word */
    uint32_t       count;   /* its entries (its coefficients once dense) */
    int            dense;
} packer_t;

static inline uint32_t page_len(const packer_t *k, uint32_t p)
{
    const uint32_t base = p << PAGE_SHIFT;
    return k->n - base < PAGE_LEN ? k->n - base : PAGE_LEN;
}

static void close_page(packer_t *k)
{
    k->out[1 + 2 * k->p] = k->start | (k->dense ? 0x80000000u : 0u);
    k->out[2 + 2 * k->p] = k->count;
    const uint32_t end = k->start + (k->dense ? (k->count + 1) / 2 : k->count);
    k->start = align4(end);
    for (uint32_t w = end; w < k->start; w++) k->out[w] = 0;   /* padding: the same bytes from every scan */
    k->p++;
    k->count = 0;
    k->dense = 0;
}

/* the whole page as int16 (what the entries so far stood for, and more) */
static void make_dense(packer_t *k)
{
    const uint32_t len = page_len(k, k->p);
    uint32_t *d = k->out + k->start;
    memcpy(d, k->src + ((size_t)k->p << PAGE_SHIFT), (size_t)len * 2);
    if (len & 1) ((uint16_t *)d)[len] = 0;
    k->dense = 1;
    k->count = len;
}

/* coefficients [a, e) of the current page */
static void pack_span(packer_t *k, uint32_t a, uint32_t e)
{
    const uint32_t base = k->p << PAGE_SHIFT, cap = (page_len(k, k->p) + 1) / 2;
    while (a < e && !k->dense) {
        const uint32_t left = cap - k->count;
        if (!left) { make_dense(k); break; }
        const uint32_t m = e - a < left ? e - a : left;     /* at most one entry each */
        uint32_t *o = g_scan(k->src + a, m, a - base, k->out + k->start + k->count);
        k->count = (uint32_t)(o - (k->out + k->start));
        a += m;
    }
}

/* [a, e), after every earlier range */
static void pack_range(packer_t *k, uint64_t a, uint64_t e)
{
    while (a < e) {
        const uint32_t p = (uint32_t)(a >> PAGE_SHIFT);
        while (k->p < p) close_page(k);
        uint64_t pe = ((uint64_t)p + 1) << PAGE_SHIFT;
        if (pe > e) pe = e;
        pack_span(k, (uint32_t)a, (uint32_t)pe);
        a = pe;
    }
}

#if defined(__x86_64__)
/* The REFCPU block walk with the AVX-512 scan inlined: every luma span the
 * reconstruction reads is a whole number of 4x4 TXs (16 coefficients), so
 * it goes in vectors of 32 and at most one of 16, each stored whole and
 * advanced by its mask's popcount (no branch on the data; a store past the
 * entries is overwritten by later entries or the page padding, as in
 * scan_avx512). Spans that cross a page, would outgrow it or end at a
 * clipped array take the general path. Same words as the general walk. */
__attribute__((target("avx512f,avx512bw,avx512vl,popcnt")))
static int pack_refcpu_avx512(packer_t *k, const vp9_parsed_frame_t *pf)
{
    const __m512i lane = _mm512_setr_epi32(0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15);
    const int W = (int)pf->hdr.width, H = (int)pf->hdr.height;
    const uint32_t n = k->n;
    uint64_t last = 0;
    for (uint32_t i = 0; i < pf->num_blocks; i++) {
        const vp9_macroblock_info_t *b = &pf->blocks[i];
        if (b->skip || b->tx_size > 3 || (int)b->x >= W || (int)b->y >= H) continue;
        const int sh = 2 + b->tx_size;
        const int cw = b->width < W - b->x ? b->width : W - b->x;
        const int ch = b->height < H - b->y ? b->height : H - b->y;
        const uint64_t a = b->coeff_offset;
        uint64_t e = a + ((uint64_t)((cw >> sh) * (ch >> sh)) << (2 * sh));
        if (e > n) e = n;
        if (a >= e) continue;
        if (a < last) return -1;
        last = e;
        const uint32_t m = (uint32_t)(e - a);
        if ((a >> PAGE_SHIFT) != k->p || ((e - 1) >> PAGE_SHIFT) != k->p || k->dense || (m & 15) ||
            m > (page_len(k, k->p) + 1) / 2 - k->count) {
            pack_range(k, a, e);
            continue;
        }
        const int16_t *src = k->src + a;
        uint32_t off = (uint32_t)(a - ((uint64_t)k->p << PAGE_SHIFT));
        uint32_t *o = k->out + k->start + k->count;
        uint32_t j = 0;
        for (; j + 32 <= m; j += 32) {
            const __m512i v = _mm512_loadu_si512((const void *)(src + j));
            const __mmask32 nz = _mm512_test_epi16_mask(v, v);
            const __m512i base = _mm512_add_epi32(_mm512_set1_epi32((int)(off + j)), lane);
            const __m512i e0 = _mm512_or_si512(_mm512_slli_epi32(_mm512_cvtepi16_epi32(_mm512_castsi512_si256(v)), 16), base);
            const __m512i e1 = _mm512_or_si512(_mm512_slli_epi32(_mm512_cvtepi16_epi32(_mm512_extracti64x4_epi64(v, 1)), 16),
                                               _mm512_add_epi32(base, _mm512_set1_epi32(16)));
            _mm512_storeu_si512((void *)o, _mm512_maskz_compress_epi32((__mmask16)nz, e0));
            o += __builtin_popcount((unsigned)(nz & 0xffffu));
            _mm512_storeu_si512((void *)o, _mm512_maskz_compress_epi32((__mmask16)(nz >> 16), e1));
            o += __builtin_popcount((unsigned)(nz >> 16));
        }
        if (j < m) {
            const __m256i v = _mm256_loadu_si256((const __m256i *)(src + j));
            const __mmask16 nz = _mm256_test_epi16_mask(v, v);
            const __m512i e0 = _mm512_or_si512(_mm512_slli_epi32(_mm512_cvtepi16_epi32(v), 16),
                                               _mm512_add_epi32(_mm512_set1_epi32((int)(off + j)), lane));
            _mm512_storeu_si512((void *)o, _mm512_maskz_compress_epi32(nz, e0));
            o += __builtin_popcount((unsigned)nz);
        }
        k->count = (uint32_t)(o - (k->out + k->start));
    }
    return 0;
}
#endif

int64_t cvp9_pack_coeffs(int arith, const vp9_parsed_frame_t *pf, uint32_t *out, size_t cap_words)
{
    if (!pf || !out) return -1;
    const uint32_t n = pf->num_coeffs;
    if (cap_words < cvp9_pack_bound_words(n) || (n && !pf->coeffs)) return -1;
    pthread_once(&g_scan_once, scan_init);
    packer_t k;
    memset(&k, 0, sizeof(k));
    k.src = pf->coeffs;
    k.out = out;
    k.n = n;
    k.np = (uint32_t)(((uint64_t)n + PAGE_LEN - 1) >> PAGE_SHIFT);
    k.start = align4(1u + 2u * k.np);
    out[0] = k.np;
    if (arith != CVP9_ARITH_REFCPU) {     /* SPEC and FULL read every plane */
        pack_range(&k, 0, n);
    } else if (pf->num_blocks && !pf->blocks) {
        return -1;
#if defined(__x86_64__)
    } else if (g_scan == scan_avx512) {
        if (pack_refcpu_avx512(&k, pf) != 0) return -1;
#endif
    } else {
        /* each block's luma TX span, as k_gather_luma moves it */
        const int W = (int)pf->hdr.width, H = (int)pf->hdr.height;
        uint64_t last = 0;
        for (uint32_t i = 0; i < pf->num_blocks; i++) {
            const vp9_macroblock_info_t *b = &pf->blocks[i];
            if (b->skip || b->tx_size > 3 || (int)b->x >= W || (int)b->y >= H) continue;
            const int sh = 2 + b->tx_size;             /* TX side 4 << tx_size */
            const int cw = b->width < W - b->x ? b->width : W - b->x;
            const int ch = b->height < H - b->y ? b->height : H - b->y;
            const uint64_t a = b->coeff_offset;
            uint64_t e = a + ((uint64_t)((cw >> sh) * (ch >> sh)) << (2 * sh));
            if (e > n) e = n;
            if (a >= e) continue;
            if (a < last) return -1;
            if ((a >> PAGE_SHIFT) == k.p && ((e - 1) >> PAGE_SHIFT) == k.p && !k.dense &&
                e - a <= (page_len(&k, k.p) + 1) / 2 - k.count) {
                /* the common case: inside the page being filled, room left */
                uint32_t *o = g_scan(k.src + a, (uint32_t)(e - a), (uint32_t)(a - ((uint64_t)k.p << PAGE_SHIFT)),
                                     k.out + k.start + k.count);
                k.count = (uint32_t)(o - (k.out + k.start));
            } else {
                pack_range(&k, a, e);
            }
            last = e;
        }
    }
    while (k.p < k.np) close_page(&k);
    return (int64_t)k.start;
}
