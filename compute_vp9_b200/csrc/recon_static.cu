/*
 * recon_static.cu — reconstruct one frame without allocating anything.
 *
 * Some callers cannot allocate device memory at decode time: a media
 * framework or inference server that owns every byte of the GPU through its
 * own pools and forbids cudaMalloc on the decode thread, or a real-time
 * thread where cudaMalloc/cudaFree may wait on device-wide synchronisation.
 * cuda_reconstruct_noalloc serves them. The caller passes device inputs
 * (blocks, coefficients), the reference frames and the output frame; the
 * per-frame scratch the kernels need (superblock ranges and done flags, the
 * wavefront ticket order, the ticket counter, the status word and the job
 * descriptor) lives in one file-scope __device__ array of fixed size instead
 * of in allocations.
 *
 * Limits and sharing rules:
 *  - at most CVP9_NOALLOC_MAX_SB superblocks (8160 = 7680x4320); larger
 *    frames are rejected with CVP9_ERR_INVALID_DATA and a message on stderr;
 *  - every process that loads the library holds the array (~200 KB) on every
 *    GPU it uses until exit;
 *  - all calls share the array: everything that must start at zero is
 *    cleared at the start of each call, and calls whose work overlaps on the
 *    GPU (different streams, or different host threads) race with each
 *    other — serialise them on one stream;
 *  - the first call on a device does the one-time set-up for that device
 *    (kernel attributes, the float64 DCT basis, and the device address of
 *    the array), so make that first call before any stream capture.
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "recon_job.h"
#include "recon_launch.h"
#include "backend_common.h"
#include "cuda_backend.h"

namespace {

constexpr int kMaxSb = CVP9_NOALLOC_MAX_SB;

/* layout of the scratch array (byte offsets) */
constexpr size_t kOffJob     = 0;                                   /* cvp9_job_t       */
constexpr size_t kOffMisc    = 1024;                                /* [0] tickets ctr, [1] status */
constexpr size_t kOffRange   = 2048;                                /* 4 x u32 per SB   */
constexpr size_t kOffDone    = kOffRange + (size_t)kMaxSb * 16;     /* u32 per SB       */
constexpr size_t kOffTickets = kOffDone + (size_t)kMaxSb * 4;       /* u32 per SB       */
constexpr size_t kScratchBytes = kOffTickets + (size_t)kMaxSb * 4;

static_assert(sizeof(cvp9_job_t) <= 1024, "job descriptor must fit its scratch slot");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

/* device address of the array per device, fetched once with that device current */
constexpr int kMaxDev = 64;
static unsigned char *g_scratch_ptr[kMaxDev];

__global__ void k_put_job(cvp9_job_t job, cvp9_job_t *dst)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) *dst = job;
}

/* SB-diagonal ticket order computed on the device: SB (r, c) goes after
 * every SB of a smaller anti-diagonal, in row order within its diagonal. */
__global__ void k_diag_tickets(int sb_cols, int sb_rows, uint32_t *tickets)
{
    int sb = blockIdx.x * blockDim.x + threadIdx.x;
    if (sb >= sb_cols * sb_rows) return;
    int r = sb / sb_cols, c = sb - r * sb_cols, d = r + c;
    int before = 0;
    for (int e = 0; e < d; e++) {
        int lo = e - (sb_cols - 1) > 0 ? e - (sb_cols - 1) : 0;
        int hi = e < sb_rows - 1 ? e : sb_rows - 1;
        before += hi - lo + 1;
    }
    int lo = d - (sb_cols - 1) > 0 ? d - (sb_cols - 1) : 0;
    tickets[before + (r - lo)] = (uint32_t)sb;
}

static int setup_device(int dev)
{
    if (dev < 0 || dev >= kMaxDev) return -1;
    if (g_scratch_ptr[dev]) return 0;
    if (cvp9_device_setup(dev) != 0) return -1;   /* cudaSetDevice(dev) inside */
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        fprintf(stderr, "[compute-vp9] cudaGetSymbolAddress: %s\n", cudaGetErrorString(e));
        return -1;
    }
    g_scratch_ptr[dev] = (unsigned char *)p;
    return 0;
}

} /* namespace */

extern "C" cvp9_err_t cuda_reconstruct_noalloc(const vp9_parsed_frame_t *pf,
                                               const uint8_t *const ref_planes[8],
                                               const uint32_t ref_width[8],
                                               const uint32_t ref_height[8],
                                               uint8_t *out_i420, int arith,
                                               uint32_t *status_dev, void *stream)
{
    if (!pf || !out_i420) return CVP9_ERR_INVALID_DATA;
    const int32_t W = (int32_t)pf->hdr.width, H = (int32_t)pf->hdr.height;
    if (W <= 0 || H <= 0 || W > 65535 || H > 65535) return CVP9_ERR_INVALID_DATA;
    const int sb_cols = (W + 63) / 64, sb_rows = (H + 63) / 64;
    if ((long long)sb_cols * sb_rows > kMaxSb) {
        fprintf(stderr, "[compute-vp9] cuda_reconstruct_noalloc: %dx%d needs %d superblocks, "
                        "the static scratch holds %d (7680x4320)\n", W, H, sb_cols * sb_rows, kMaxSb);
        return CVP9_ERR_INVALID_DATA;
    }
    if ((pf->num_blocks && !pf->blocks) || (pf->num_coeffs && !pf->coeffs)) return CVP9_ERR_INVALID_DATA;
    if (arith == CVP9_CUDA_ARITH_FULL) {
        fprintf(stderr, "[compute-vp9] cuda_reconstruct_noalloc: takes the REFCPU and SPEC profiles\n");
        return CVP9_ERR_UNSUPPORTED;
    }
    const int a = arith == CVP9_CUDA_ARITH_SPEC ? CVP9_ARITH_SPEC : CVP9_ARITH_REFCPU;
    const char *why = nullptr;
    if (!cvp9_frame_supported(a, pf, &why)) {
        fprintf(stderr, "[compute-vp9] cuda_reconstruct_noalloc: %s\n", why);
        return CVP9_ERR_UNSUPPORTED;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || setup_device(dev) != 0) return CVP9_ERR_GPU;
    unsigned char *base = g_scratch_ptr[dev];
    cudaStream_t st = (cudaStream_t)stream;
    const int n_sb = sb_cols * sb_rows;

    cvp9_job_t job;
    memset(&job, 0, sizeof(job));
    cvp9_job_geometry(&job, pf);
    job.blocks = pf->blocks;
    job.coeffs = pf->coeffs;
    job.out = out_i420;
    job.nv12 = nullptr;
    for (int i = 0; i < 8; i++) {
        if (ref_planes && ref_planes[i]) {
            job.ref[i].plane = ref_planes[i];
            job.ref[i].w = (int32_t)(ref_width ? ref_width[i] : 0);
            job.ref[i].h = (int32_t)(ref_height ? ref_height[i] : 0);
            if (job.ref[i].w <= 0 || job.ref[i].h <= 0) job.ref[i].plane = nullptr;
        }
    }
    job.epoch = 1;
    job.sb_range = (uint32_t *)(base + kOffRange);
    job.sb_done = (uint32_t *)(base + kOffDone);
    job.status = (uint32_t *)(base + kOffMisc) + 1;

    /* the array keeps the previous call's contents: clear what starts at 0 */
    if (cudaMemsetAsync(base + kOffMisc, 0, 64, st) != cudaSuccess ||
        cudaMemsetAsync(base + kOffRange, 0, (size_t)n_sb * 16, st) != cudaSuccess ||
        cudaMemsetAsync(base + kOffDone, 0, (size_t)n_sb * 4, st) != cudaSuccess)
        return CVP9_ERR_GPU;
    k_put_job<<<1, 1, 0, st>>>(job, (cvp9_job_t *)(base + kOffJob));
    k_diag_tickets<<<(n_sb + 255) / 256, 256, 0, st>>>(sb_cols, sb_rows, (uint32_t *)(base + kOffTickets));
    if (cudaGetLastError() != cudaSuccess) return CVP9_ERR_GPU;

    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cvp9k_launch_t L;
    memset(&L, 0, sizeof(L));
    L.jobs = (const cvp9_job_t *)(base + kOffJob);
    L.njobs = 1;
    L.arith = a;
    L.max_blocks = (int)pf->num_blocks;
    L.tickets = (const uint32_t *)(base + kOffTickets);
    L.n_tickets = (uint32_t)n_sb;
    L.ticket_counter = (uint32_t *)(base + kOffMisc);
    int resident = sms * cvp9_recon_ctas_per_sm(dev, a);
    L.recon_ctas = n_sb < resident ? n_sb : resident;
    if (job.lf_tiled) {
        L.lf_tiles_x = (W + 4 + 63) / 64;
        L.lf_tiles_y = (H + 4 + 63) / 64;
    } else {
        L.flat_lf_max_w = W;
        L.flat_lf_max_h = H;
    }
    if (cvp9k_launch_frame(&L, st) != 0) return CVP9_ERR_GPU;
    if (status_dev &&
        cudaMemcpyAsync(status_dev, base + kOffMisc + 4, 4, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return CVP9_ERR_GPU;
    return CVP9_OK;
}
