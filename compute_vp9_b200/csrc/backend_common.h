/*
 * backend_common.h — host helpers shared by the per-stream backend
 * (cuda_backend.c) and the multi-stream batch engine (batch.c).
 */
#ifndef CVP9_BACKEND_COMMON_H
#define CVP9_BACKEND_COMMON_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>
#include "recon_job.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Make `device` current and, once per device per process, upload the
 * float64 DCT basis and set the kernels' shared-memory limits. 0 on success. */
int cvp9_device_setup(int device);

/* Resident reconstruction CTAs per SM for the profile (after setup). */
int cvp9_recon_ctas_per_sm(int device, int arith);

/* The basis of the reference's float64 inverse DCT, N = 4, 8, 16, 32
 * concatenated (16 + 64 + 256 + 1024 doubles), built with the expression of
 * src/decoder/vp9_reconstruct.c:19-29 so libm produces the same doubles. */
void cvp9_build_dct_basis(double *out);

/* SB-diagonal ticket order: append the SBs of a sb_cols x sb_rows grid of
 * job `job` that lie on anti-diagonal d (row + col == d) to out. Returns
 * the number written. */
int cvp9_tickets_on_diagonal(int sb_cols, int sb_rows, int job, int d, uint32_t *out);

/* Quantiser steps for a qindex (vp9_dequant.h:67-75 with delta 0). */
int cvp9_dc_q(int qindex);
int cvp9_ac_q(int qindex);

/* Environment knobs: $CVP9_CUDA_DEVICE, $CVP9_ARITH (refcpu|spec),
 * $CVP9_INTER_FAST (warp-per-superblock inter path: 0 off, 1 the
 * 96-register kernel, 2 the 80-register kernel; default 1). */
int cvp9_env_device(void);
int cvp9_env_arith(void);
int cvp9_env_inter_fast(void);

/* Fill the frame-geometry and parameter fields of a job from a parsed
 * frame (inputs, output, refs and scratch pointers are set by the caller). */
void cvp9_job_geometry(cvp9_job_t *job, const vp9_parsed_frame_t *pf);

/* Monotonic clock in seconds. */
double cvp9_now(void);

#ifdef __cplusplus
}
#endif

#endif /* CVP9_BACKEND_COMMON_H */
