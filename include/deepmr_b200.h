/*
 * deepmr_b200 — C ABI of the B200 (sm_100a) non-Cartesian NUFFT library.
 *
 * The entry points replace the kernel seam of the reference NUFFT
 * (deepmr, src/deepmr/fft/...): the plan builder, the interpolation and
 * gridding launchers, and the FFT/apodisation/pad/crop steps around them.
 * Each declaration cites the reference interface it replaces
 * (paths relative to the reference project).
 *
 * Conventions
 *  - All data pointers are device pointers unless a parameter says "host".
 *  - complex64 data is interleaved (re, im) float32, i.e. torch.complex64.
 *  - Spatial shapes and per-axis parameters are given in (z, y, x) order for
 *    the last `ndim` axes (ndim = 1, 2 or 3); coordinates are (x, y, z)
 *    along their last axis, in grid units, like the reference.
 *  - Sample data is laid out (batch, total_samples) where total_samples is
 *    the sum of the per-frame sample counts (frame f occupies
 *    [frame_offsets[f], frame_offsets[f+1])). For equal-length frames this is
 *    exactly the reference's (..., ncontrasts, nviews, nsamples) layout.
 *  - Images / grids are laid out (batch, nframes, *shape).
 *  - Every call is ordered on the given CUDA stream (cudaStream_t passed as
 *    void*); none synchronises the device except dmr_plan_create (which
 *    reads bin counts back to the host) and dmr_plan_destroy.
 *  - Return value: 0 on success, a negative DMR_ERR_* code otherwise;
 *    dmr_last_error() gives a message for the calling host thread.
 *  - Host-thread safety: distinct plans may be used concurrently; one plan
 *    may be used from several threads (its FFT handles are locked per call).
 */
#ifndef DEEPMR_B200_H
#define DEEPMR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DMR_OK 0
#define DMR_ERR_INVALID -1     /* bad argument / shape */
#define DMR_ERR_CUDA -2        /* CUDA runtime error */
#define DMR_ERR_OOM -3         /* device allocation failed */
#define DMR_ERR_COORD -4       /* non-finite coordinate */
#define DMR_ERR_CUFFT -5       /* cuFFT error */
#define DMR_ERR_UNSUPPORTED -6 /* configuration not supported */
#define DMR_ERR_WORKSPACE -7   /* workspace too small */
#define DMR_ERR_TIMEOUT -8     /* a bounded device-side wait ran out: results not valid */

typedef struct dmr_plan dmr_plan;

/* Library version (major*10000 + minor*100 + patch). */
int dmr_version(void);

/* Message for the last error raised on this host thread. */
const char *dmr_last_error(void);

/* Number of kernels this library has launched since load (all threads). */
int64_t dmr_launch_count(void);

/*
 * Blocks of the tensor-core gridding kernel, over all plans on the current
 * device since load, that stopped because a bounded wait ran out (each such
 * block stops issuing work, waits for its MMAs in flight and frees its tensor
 * memory; the count should stay 0). Reads after a device synchronisation;
 * reset != 0 zeroes the counter. No reference counterpart (device health).
 */
int dmr_tc_timeouts(int64_t *count, int reset);

/*
 * Device status of a plan: `failed` (host, may be NULL) receives the number of
 * gridding blocks of this plan's calls that stopped on a bounded wait since
 * the last reset. Synchronises `stream`; returns DMR_ERR_TIMEOUT when that
 * number is non-zero (the outputs of the calls since the last reset are then
 * partial and must not be used), DMR_OK otherwise; reset != 0 zeroes it.
 * Calls on one plan from several streams share the word. No reference
 * counterpart (the reference's kernels have no device-side waits).
 */
int dmr_plan_status(dmr_plan *plan, int32_t *failed, int reset, void *stream);

/*
 * Test hook, no reference counterpart: enable != 0 makes every block of the
 * following tensor-core gridding launches (all plans) wait, before it reuses
 * an operand buffer, on an mbarrier that nothing signals, so that the bounded
 * wait (1 ms) runs out and the block stops; enable = 0 restores normal runs.
 * Exercises the timeout path without a GPU fault.
 */
int dmr_tc_test_stall(int enable);

/*
 * Query, no reference counterpart: 1 if the plan's forward / adjoint NUFFT
 * run their 3D FFT as the library's fused passes (apodise + zero-pad + FFT,
 * inverse FFT + crop + 1/G + apodisation, pruned to the lines with data),
 * 0 if they use cuFFT with separate pad / crop kernels (grid extents without
 * a compiled transform, 1D / 2D plans, or DMR_CUFFT=1 in the environment).
 * Replaces the FFT step of src/deepmr/fft/nufft.py:502-505 and 583-590.
 */
int dmr_fft3_fused(dmr_plan *plan);

/*
 * Tuning knob, no reference counterpart: atomic gridding of a 3D plan runs on
 * the tensor cores for batches of at least `coils` coils (default 20; below,
 * the CUDA-core kernel, whose cost scales with the coil count, is faster) and
 * on the CUDA cores otherwise. coils <= 0 only queries. Returns the previous
 * value. Process-wide; deterministic gridding is not affected.
 */
int dmr_tc_min_coils(int coils);

/*
 * Housekeeping, no reference counterpart: gives back to `device` the memory
 * that the library's scratch pool holds beyond what is in use. Calls without
 * a large enough workspace take their gridding scratch from this pool, which
 * keeps it for the next call; deterministic 3D gridding keeps every work
 * item's partial sums there (2 KB per gridding work item and coil: 13.6 GB
 * for 32 coils of the 192^3, 19.2 M-sample kooshball). Synchronises the
 * device first. Returns 0 or a DMR_ERR_* code.
 */
int dmr_scratch_release(int device);

/*
 * Memory control, no reference counterpart: the largest scratch, in bytes,
 * that deterministic 3D tensor-core gridding may take (its per-item partial
 * sums, 2 KB per gridding work item and coil). A call that would need more,
 * or for which the pool has no memory, runs on the register-tile kernel (or
 * the colour passes) instead: deterministic as well, slower, with a small
 * scratch. bytes > 0 sets the limit, 0 removes it (the default), < 0 only
 * queries. Returns the previous limit. Process-wide.
 */
int64_t dmr_det_scratch_limit(int64_t bytes);

/*
 * Cartesian-axis test of plan_nufft (src/deepmr/fft/nufft.py:104-109):
 * for coordinate axis a (x, y, z order), all(|s - round(s)| <= 1e-8 + 1e-5|round(s)|)
 * in float32 with s = shape_zyx[a] * coord[..., a] (the reference pairs the
 * coordinate axis with the shape entry of the same position). Writes one
 * flag per coordinate axis to host `is_cart_xyz` (synchronises the stream).
 */
int dmr_detect_cartesian(const float *coord, int64_t npts, int ndim,
                         const int32_t *shape_zyx, int32_t *is_cart_xyz,
                         void *stream);

/*
 * Build a device-resident NUFFT plan.
 * Replaces plan_nufft's interpolator precompute
 * (src/deepmr/fft/nufft.py:116-122 and src/deepmr/fft/_interp/plan.py:14-143):
 * instead of materialising (F, M, W) index/value tables per axis, the plan
 * rescales the coordinates (nufft.py:411-420, float32 multiply then add),
 * sorts the samples by spatial bin (stable) and keeps the sorted rescaled
 * coordinates; kernel weights are evaluated inside the gather/scatter kernels.
 *
 *  shape, os_shape, width, beta, oversamp: host arrays, (z, y, x) order, the
 *     values plan_nufft derives (after the Cartesian-axis override: width 1
 *     and oversamp 1 on Cartesian axes).
 *  coord: device, (total, ndim) float32, NOT rescaled (grid units).
 *  frame_offsets: host, nframes+1 int64 CSR offsets into the samples.
 *  tile: host, (z, y, x) bin size or NULL for the tuned default.
 */
int dmr_plan_create(int ndim, const int32_t *shape, const int32_t *os_shape,
                    const int32_t *width, const float *beta,
                    const float *oversamp, const float *coord,
                    const int64_t *frame_offsets, int64_t nframes,
                    const int32_t *tile, void *stream, dmr_plan **out);

/* Free a plan (synchronises the device). */
int dmr_plan_destroy(dmr_plan *plan);

/* Kernel-sum normalisation of the plan (src/deepmr/fft/_interp/plan.py:190-213). */
int dmr_plan_scale(const dmr_plan *plan, double *scale);

/* Total samples, frames and the bin tile (z, y, x) chosen by the plan. */
int dmr_plan_info(const dmr_plan *plan, int64_t *total, int64_t *nframes,
                  int32_t *tile_zyx);

/*
 * Interpolation, oversampled grid -> samples, scaled by 1/scale and
 * multiplied by `weight`.
 * Replaces do_interpolation[_cuda] + the /scale of apply_interpolation
 * (src/deepmr/fft/_interp/interp.py:14-120, 651-749) and the weight product
 * of _apply_nufft (src/deepmr/fft/nufft.py:513-515).
 *  grid: (batch, nframes, *os_shape) complex64 in FFT order (ifftshifted:
 *        centred index c is stored at (c - G//2) mod G on every axis),
 *        i.e. exactly the output of an unshifted cuFFT forward transform.
 *  kspace: (batch, total) complex64, fully written.
 *  weight: NULL, (total) float32 if weight_per_batch == 0, or
 *          (batch, total) float32 if weight_per_batch == 1.
 */
int dmr_interp(const dmr_plan *plan, const void *grid, void *kspace,
               int64_t batch, const float *weight, int weight_per_batch,
               void *stream);

/*
 * Gridding, samples -> oversampled grid (FFT order as above), scaled by
 * 1/scale, after multiplying the samples by `weight`.
 * Replaces do_gridding[_cuda] + the /scale of apply_gridding
 * (src/deepmr/fft/_interp/grid.py:14-125, 1026-1168) and the weight product
 * of _apply_nufft_adj (src/deepmr/fft/nufft.py:577-579).
 *  kspace: (batch, total) complex64, or float32 if kspace_real == 1.
 *  grid: (batch, nframes, *os_shape) complex64, fully written.
 *  deterministic: 0 = shared-memory tiles flushed with global atomics
 *     (summation order may vary between runs);
 *     1 = every grid point is summed by one owner in a fixed order (bitwise
 *     reproducible, no float atomics): 3D grids of 8 or more coils keep
 *     8^3-point block regions in registers (regions too dense for one block
 *     are split into partial sums added in a fixed order; without a caller
 *     workspace this call takes their scratch from a library-owned
 *     stream-ordered memory pool); other grids run the bins in colour passes
 *     of disjoint tiles.
 */
int dmr_grid(const dmr_plan *plan, const void *kspace, int kspace_real,
             void *grid, int64_t batch, const float *weight,
             int weight_per_batch, int deterministic, void *stream);

/* Bytes of workspace the forward/adjoint pipelines need for `batch`. */
int dmr_nufft_workspace_bytes(dmr_plan *plan, int64_t batch, size_t *bytes);

/*
 * Forward NUFFT: apodise + zero-pad + ifftshift (one kernel), cuFFT forward,
 * interpolation (fftshift folded into its indexing) with 1/scale and weight.
 * Replaces _apply_nufft (src/deepmr/fft/nufft.py:450-528).
 *  image: (batch, nframes, *shape) complex64, or float32 if image_real == 1.
 *  kspace: (batch, total) complex64.
 */
int dmr_nufft_forward(dmr_plan *plan, const void *image, int image_real,
                      void *kspace, int64_t batch, const float *weight,
                      int weight_per_batch, void *workspace,
                      size_t workspace_bytes, void *stream);

/*
 * Adjoint NUFFT: gridding (weight, 1/scale, ifftshift folded), cuFFT inverse,
 * fftshift + crop + 1/G + apodisation (one kernel).
 * Replaces _apply_nufft_adj (src/deepmr/fft/nufft.py:531-606).
 *  kspace: (batch, total) complex64, or float32 if kspace_real == 1.
 *  image: (batch, nframes, *shape) complex64.
 */
int dmr_nufft_adjoint(dmr_plan *plan, const void *kspace, int kspace_real,
                      void *image, int64_t batch, const float *weight,
                      int weight_per_batch, int deterministic,
                      void *workspace, size_t workspace_bytes, void *stream);

/*
 * Low-rank subspace NUFFT. Replaces the basis branches of the reference's
 * interpolation and gridding (_interpolate_lowrank{1,2,3} /
 * _gridding_lowrank{1,2,3}, src/deepmr/fft/_interp/interp.py:230-357 and
 * src/deepmr/fft/_interp/grid.py:287-417, selected by apply_nufft's
 * basis_adjoint / apply_nufft_adj's basis, src/deepmr/fft/nufft.py:450-606).
 * Forward: frame f interpolates sum_c basis_adjoint[f, c] * FFT(image[c]);
 * adjoint: image[c] = crop/apodise(IFFT(sum_f basis[c, f] * grid_f)). The
 * reference runs only when ncoeff equals the frame count; here any
 * 1 <= ncoeff <= 32 is accepted.
 *  image: (batch, ncoeff, *shape); kspace: (batch, total) as above.
 *  basis_adjoint: device (nframes, ncoeff) complex64; basis: device
 *  (ncoeff, nframes) complex64 (row-major).
 */
int dmr_nufft_lowrank_workspace_bytes(dmr_plan *plan, int64_t batch, int64_t ncoeff,
                                      size_t *bytes);
int dmr_nufft_forward_lowrank(dmr_plan *plan, const void *image, int image_real,
                              int64_t ncoeff, const void *basis_adjoint, void *kspace,
                              int64_t batch, const float *weight, int weight_per_batch,
                              void *workspace, size_t workspace_bytes, void *stream);
int dmr_nufft_adjoint_lowrank(dmr_plan *plan, const void *kspace, int kspace_real,
                              int64_t ncoeff, const void *basis, void *image,
                              int64_t batch, const float *weight, int weight_per_batch,
                              int deterministic, void *workspace, size_t workspace_bytes,
                              void *stream);

/*
 * Trajectory gradient of the NUFFT. No counterpart in the reference: its
 * autograd returns no coordinate gradient (src/deepmr/fft/nufft.py:188-209).
 *   grad[p, a] = post_scale * sum_b Re(conj(v_b[p]) * dy_b[p] / dcoord[p, a])
 * where y = dmr_nufft_forward(image) with `weight` (derivative of the
 * Kaiser-Bessel weights with the tap set held fixed; 0 on Cartesian axes).
 *  image: (batch, nframes, *shape) complex64 (float32 if image_real);
 *  v: (batch, total) complex64; grad: (total, ndim) float32 in the original
 *  sample order, coordinate axes (x, y, z), fully written (deterministic).
 * Forward operator y = A x: image = x, v = dL/dy, post_scale = 1.
 * Adjoint operator x = A^H y: image = dL/dx, v = y, post_scale = 1/prod(os_shape).
 * Uses the forward NUFFT workspace (dmr_nufft_workspace_bytes). Widths <= 8.
 */
int dmr_nufft_traj_grad(dmr_plan *plan, const void *image, int image_real,
                        const void *v, int64_t batch, const float *weight,
                        int weight_per_batch, double post_scale, float *grad,
                        void *workspace, size_t workspace_bytes, void *stream);

/* Bytes of workspace dmr_toeplitz_apply / dmr_toeplitz_finalize need. */
int dmr_toeplitz_workspace_bytes(int ndim, const int32_t *kshape,
                                 int64_t batch, size_t *bytes);

/*
 * Toeplitz kernel finalisation of plan_toeplitz
 * (src/deepmr/fft/toeplitz.py:131-155, plain case): from the point-spread
 * function psf (nk, *kshape) complex64 computes
 *   k = ifftshift(fftshift(fftn_ortho(ifftshift(psf)))) / mean(|k| over k != 0)
 * with NaN replaced by 0, into `kernel` (nk, *kshape).
 */
int dmr_toeplitz_finalize(int ndim, const int32_t *kshape, int64_t nk,
                          const void *psf, void *kernel, void *workspace,
                          size_t workspace_bytes, void *stream);

/*
 * Toeplitz self-adjoint: centred zero-pad to kshape, unshifted FFT,
 * multiply by kernel frame (i mod nk) and by 1/prod(kshape) (the two
 * orthonormal scalings), unshifted inverse FFT, centred crop.
 * Replaces _apply_nufft_selfadj (src/deepmr/fft/nufft.py:609-669) with the
 * plain branch of apply_toeplitz (src/deepmr/fft/_interp/toeplitz.py:84-87).
 *  image, out: (batch, *ishape) complex64 (or float32 image if image_real);
 *  batch element i uses kernel frame i mod nk.
 */
int dmr_toeplitz_apply(int ndim, const int32_t *kshape, const int32_t *ishape,
                       const void *kernel, int64_t nk, const void *image,
                       int image_real, void *out, int64_t batch,
                       void *workspace, size_t workspace_bytes, void *stream);

/*
 * SENSE + Toeplitz normal operator of a CG-SENSE reconstruction:
 *   out = sum_c conj(S_c) * T(S_c * x) + lamda * x
 * with T the Toeplitz self-adjoint of dmr_toeplitz_apply (single kernel
 * frame). Replaces C.H * NUFFTGramOp * C (+ lamda * Identity) of
 * src/deepmr/recon/alg/linop.py:145-146 and src/deepmr/optim/cg.py:86-94:
 * coil expansion is fused into the zero-pad kernel and the coil sum (in coil
 * order, deterministic) + lamda * x into the crop kernel.
 *  kernel: (*kshape) complex64; maps: (ncoils, *ishape); x, out: (*ishape),
 *  not aliased. Workspace: dmr_toeplitz_workspace_bytes(ndim, kshape, ncoils).
 */
int dmr_sense_normal(int ndim, const int32_t *kshape, const int32_t *ishape,
                     const void *kernel, const void *maps, int64_t ncoils,
                     const void *x, void *out, float lamda, void *workspace,
                     size_t workspace_bytes, void *stream);

/*
 * Conjugate gradient of cg_solve / CGStep (src/deepmr/optim/cg.py:16-221)
 * with every scalar kept on the device (no host synchronisation per step) and
 * float64 inner products reduced in a fixed order. `state` is a device buffer
 * of dmr_cg_state_bytes bytes. dmr_cg_init: x = 0, r = p = ahy,
 * rsold = <r, r>. dmr_cg_step, given q = AHA(p): alpha = rsold / <p, q>,
 * x += alpha p, r -= alpha q, rsnew = Re<r, r>, p = r + (rsnew / rsold) p.
 * dmr_cg_residual copies rsnew to the host (synchronises the stream).
 * All vectors are complex64 of n elements.
 */
int dmr_cg_state_bytes(size_t *bytes);
int dmr_cg_init(const void *ahy, void *x, void *r, void *p, int64_t n,
                void *state, void *stream);
int dmr_cg_step(void *x, void *r, void *p, const void *q, int64_t n,
                void *state, void *stream);
int dmr_cg_residual(const void *state, double *rsnew, void *stream);

/*
 * Allocation-free variant of the Toeplitz kernel normalisation step.
 * No counterpart in the reference. For callers that must not allocate device
 * memory (an application that hands the GPU a fixed memory pool at start-up,
 * a real-time reconstruction loop that forbids allocator calls once running,
 * or a host without a CUDA allocator of its own): scales the complex64 array
 * `kernel` (n elements) in place by 1 / mean(|k| over k != 0) and replaces
 * NaN by 0 and +-inf by +-FLT_MAX — the normalisation of dmr_toeplitz_finalize
 * — with the reduction's partial sums in a 64 KB static device array owned by
 * the library (kept by every device that loads it until the process exits)
 * instead of a caller workspace. Calls no allocator.
 *  - n must not exceed 67,108,864 elements (4096 partial sums x 16384
 *    elements); larger n returns DMR_ERR_INVALID.
 *  - The first call on a device looks up the array's device address
 *    (cudaGetSymbolAddress) with that device current; make that first call
 *    before any stream capture.
 *  - All calls share the array: calls that overlap on the GPU (different
 *    streams, or different host threads) race and give wrong results.
 */
int dmr_toeplitz_normalize_noalloc(void *kernel, int64_t n, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* DEEPMR_B200_H */
