/*
 * arena.h — chunked sub-allocator for the batch engine's device and pinned
 * host buffers.
 *
 * Driver allocation calls are slow and unpredictable on the decode path:
 * cudaFree and cudaFreeHost wait for all work on the device, pinning host
 * memory costs about 0.4 ms per MB, and stream-ordered allocations were seen
 * to block for up to a second while the pool grew. The engine therefore takes
 * large chunks from the driver (a few per run) and carves stream and step
 * buffers out of them with a first-fit free list kept in address order.
 * Freed ranges coalesce with their neighbours inside a chunk; chunks go back
 * to the driver only when the arena is destroyed.
 *
 * A range may be freed only when no queued device work still uses it; the
 * engine frees a stream's buffers after its last step completed and a step
 * slot's buffers after that slot's previous step completed.
 */
#ifndef CVP9_ARENA_H
#define CVP9_ARENA_H

#include <cuda_runtime_api.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ARENA_ALIGN 256

typedef struct { uint8_t *p; size_t n; int chunk; } arena_block_t;

typedef struct {
    int            host;        /* 1: pinned host memory, 0: device memory */
    size_t         chunk_min;   /* smallest chunk taken from the driver    */
    uint8_t      **chunk;
    size_t        *chunk_n;
    int            nchunks, chunks_cap;
    arena_block_t *fl;          /* free ranges, ascending address          */
    int            nfl, fl_cap;
    size_t         held;        /* bytes taken from the driver             */
    size_t         used;        /* bytes handed out                        */
} arena_t;

static size_t arena_round(size_t n)
{
    return (n + ARENA_ALIGN - 1) / ARENA_ALIGN * ARENA_ALIGN;
}

static int arena_fl_insert(arena_t *a, int at, arena_block_t blk)
{
    if (a->nfl == a->fl_cap) {
        int nc = a->fl_cap ? 2 * a->fl_cap : 64;
        arena_block_t *f = (arena_block_t *)realloc(a->fl, (size_t)nc * sizeof(*f));
        if (!f) return -1;
        a->fl = f;
        a->fl_cap = nc;
    }
    memmove(a->fl + at + 1, a->fl + at, (size_t)(a->nfl - at) * sizeof(*a->fl));
    a->fl[at] = blk;
    a->nfl++;
    return 0;
}

static void arena_fl_remove(arena_t *a, int at)
{
    memmove(a->fl + at, a->fl + at + 1, (size_t)(a->nfl - at - 1) * sizeof(*a->fl));
    a->nfl--;
}

/* Return a range to the free list, merging it with free neighbours of the
 * same chunk. */
static void arena_free(arena_t *a, void *p, size_t n)
{
    if (!p || !n) return;
    n = arena_round(n);
    uint8_t *q = (uint8_t *)p;
    int c = -1;
    for (int i = 0; i < a->nchunks; i++)
        if (q >= a->chunk[i] && q + n <= a->chunk[i] + a->chunk_n[i]) { c = i; break; }
    if (c < 0) return;                       /* not ours: ignore */
    int at = 0;
    while (at < a->nfl && a->fl[at].p < q) at++;
    a->used -= n;
    int merged = 0;
    if (at > 0 && a->fl[at - 1].chunk == c && a->fl[at - 1].p + a->fl[at - 1].n == q) {
        a->fl[at - 1].n += n;
        merged = 1;
        at--;
    }
    if (!merged) {
        arena_block_t blk = { q, n, c };
        if (arena_fl_insert(a, at, blk) != 0) return;   /* range is lost, not reused */
    }
    if (at + 1 < a->nfl && a->fl[at + 1].chunk == c && a->fl[at].p + a->fl[at].n == a->fl[at + 1].p) {
        a->fl[at].n += a->fl[at + 1].n;
        arena_fl_remove(a, at + 1);
    }
}

/* First fit; a new chunk of max(n, chunk_min) bytes when nothing fits.
 * Returns NULL when the driver refuses the chunk. */
static void *arena_alloc(arena_t *a, size_t n)
{
    n = arena_round(n ? n : 1);
    for (int i = 0; i < a->nfl; i++) {
        if (a->fl[i].n < n) continue;
        uint8_t *p = a->fl[i].p;
        a->fl[i].p += n;
        a->fl[i].n -= n;
        if (!a->fl[i].n) arena_fl_remove(a, i);
        a->used += n;
        return p;
    }
    size_t cs = n > a->chunk_min ? n : a->chunk_min;
    if (a->nchunks == a->chunks_cap) {
        int nc = a->chunks_cap ? 2 * a->chunks_cap : 16;
        uint8_t **ch = (uint8_t **)realloc(a->chunk, (size_t)nc * sizeof(*ch));
        if (!ch) return NULL;
        a->chunk = ch;
        size_t *cn = (size_t *)realloc(a->chunk_n, (size_t)nc * sizeof(*cn));
        if (!cn) return NULL;
        a->chunk_n = cn;
        a->chunks_cap = nc;
    }
    void *c = NULL;
    cudaError_t e = a->host ? cudaMallocHost(&c, cs) : cudaMalloc(&c, cs);
    if (e != cudaSuccess || !c) {
        cudaGetLastError();
        return NULL;
    }
    int ci = a->nchunks++;
    a->chunk[ci] = (uint8_t *)c;
    a->chunk_n[ci] = cs;
    a->held += cs;
    a->used += n;
    if (cs > n) {
        arena_block_t blk = { (uint8_t *)c + n, cs - n, ci };
        int at = 0;
        while (at < a->nfl && a->fl[at].p < blk.p) at++;
        if (arena_fl_insert(a, at, blk) != 0) { /* tail stays unused */ }
    }
    return c;
}

/* Replace *p (capacity *cap) by a range of at least `need` bytes, with 50%
 * headroom; the old range must be idle. */
static int arena_grow(arena_t *a, void **p, size_t *cap, size_t need)
{
    if (*p && *cap >= need) return 0;
    if (*p) arena_free(a, *p, *cap);
    *p = NULL;
    *cap = 0;
    size_t n = arena_round(need + need / 2 + ARENA_ALIGN);
    void *q = arena_alloc(a, n);
    if (!q) return -1;
    *p = q;
    *cap = n;
    return 0;
}

static void arena_destroy(arena_t *a)
{
    for (int i = 0; i < a->nchunks; i++) {
        if (a->host) cudaFreeHost(a->chunk[i]);
        else cudaFree(a->chunk[i]);
    }
    free(a->chunk);
    free(a->chunk_n);
    free(a->fl);
    memset(a, 0, sizeof(*a));
}

/* Make at least n bytes free (one new chunk for what is missing); the
 * chunk is then carved like any other. Returns -1 when the driver refuses. */
static int arena_reserve(arena_t *a, size_t n)
{
    const size_t free_b = a->held - a->used;
    if (free_b >= n) return 0;
    const size_t need = arena_round(n - free_b);
    void *p = arena_alloc(a, need);
    if (!p) return -1;
    arena_free(a, p, need);
    return 0;
}

#endif /* CVP9_ARENA_H */
