// Device-resident NUFFT plan: geometry, bin structure and the sorted samples.
#pragma once

#include <cufft.h>

#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace dmr {

// Geometry passed by value to every kernel. Axis index 0 = x (fastest),
// 1 = y, 2 = z; unused axes have G = N = W = T = nb = 1.
struct Geom {
    int ndim;
    int G[3];       // oversampled grid extent
    int N[3];       // image extent
    int W[3];       // kernel width (1: Cartesian axis, nearest node by truncation)
    int half[3];    // G // 2 (fftshift offset)
    int T[3];       // bin / tile extent
    int nb[3];      // bins per axis
    float beta[3];  // Kaiser-Bessel beta
    double inv_hw[3];  // 1 / (W / 2)
    int nbins;      // bins per frame
    int nframes;
    int64_t gsize;  // grid points per (batch, frame)
    int64_t isize;  // image points per (batch, frame)
    int64_t total;  // samples over all frames
    int nr[3];      // register-tile gridding: block regions per axis (0: not planned)
    int nregions;   // block regions per frame
};

// One block-level unit of interpolation / atomic-gridding work: a chunk of
// the samples of one bin (bin id includes the frame: f * nbins + local).
struct WorkItem {
    int bin;
    int begin;
    int end;
};

// Samples of a tensor-core gridding work item, at most: the MMA's fp32 sums in
// tensor memory lose accuracy over longer chains, and longer items would
// unbalance the blocks.
constexpr int kTgSegment = 2048;

// One block of register-tile gridding: part `begin` of `end` equal fractions
// of every window bin of block region `region` (frame included). slot < 0:
// the block writes the grid; otherwise it writes partial sums to scratch slot
// `slot`. A reduction item (region, first slot, end slot) sums the slots of a
// split region in order.
struct RtItem {
    int region;
    int begin;
    int end;
    int slot;
};

struct FftPlan {
    cufftHandle handle = 0;
    size_t work_bytes = 0;
    std::mutex mu;
};

// Process-wide cache of cuFFT plans keyed by (device, rank, dims, batch).
std::shared_ptr<FftPlan> get_fft_plan(int ndim, const int *dims_zyx, int64_t batch, int *err);

// Register-tile gridding: whether the geometry admits it (3D, grid at least
// a block region plus the kernel support on every axis); plan the block items after the bin sort (host
// bin offsets h_start, nframes * nbins + 1 entries); scratch bytes a call of
// `batch` coils needs (0 when the kernel does not apply).
bool rt_geometry_ok(const Geom &g);
int rt_build(::dmr_plan *p, const std::vector<int32_t> &h_start, cudaStream_t st);
size_t rt_scratch_bytes(const ::dmr_plan *p, int64_t batch);
// scratch bytes of deterministic tensor-core gridding (every work item's
// region partial sums, 2 KB per item and coil)
size_t tm_scratch_bytes(const ::dmr_plan *p, int64_t batch);
// scratch bytes a gridding call of `batch` coils may need (either kernel)
size_t grid_scratch_bytes(const ::dmr_plan *p, int64_t batch);
// library-owned stream-ordered pool for the scratch of calls without a workspace
cudaMemPool_t scratch_pool(int dev);
// fused, pruned 3D FFT passes of the NUFFT pipelines (fftpass.cu): whether they
// apply to the plan (3D, every grid extent at least the image's, at most 512
// and a product of 2, 3 and 5; DMR_CUFFT=1 turns them off), the forward
// (apodise + pad + FFT into the grid) and the adjoint (inverse FFT of the grid,
// which it overwrites, + crop + 1/G + apodisation into the image)
bool fft3_applies(const ::dmr_plan *p);
int fft3_forward(const ::dmr_plan *p, const void *image, int image_real, int64_t batch, float2 *grid,
                 cudaStream_t st);
int fft3_adjoint(const ::dmr_plan *p, float2 *grid, int64_t batch, float2 *image, cudaStream_t st);
// the same passes for the 3D Toeplitz self-adjoint: whether they apply
// (kernel extents at least the image's and with a compiled transform), and
// pad + FFT + kernel multiply + inverse FFT + crop (data: batch kernel grids)
bool toep3_applies(int ndim, const int32_t *kshape, const int32_t *ishape);
int fft3_toeplitz(int ndim, const int32_t *kshape_zyx, const int32_t *ishape_zyx, const float2 *kernel, int64_t nk,
                  const void *image, int image_real, float2 *out, int64_t batch, float2 *data, cudaStream_t st);
// tensor-core gridding of 3D plans (tcgrid.cu: dispatch and health state,
// tmgrid.cu: the kernel); DMR_ERR_UNSUPPORTED when the plan has no gridding bins
int grid_tc_dispatch(const ::dmr_plan *p, const void *ksp, int kreal, float2 *grid, int64_t batch,
                     const float *weight, int wpb, int det, void *scratch, size_t scratch_bytes,
                     cudaStream_t st);
// tensor-core gridding with the plan's gridding bins (tmgrid.cu), atomic or
// deterministic (partial sums per work item, then a gather per grid point;
// scratch from the caller when it holds tm_scratch_bytes, else from the
// library pool; DMR_ERR_UNSUPPORTED, before any launch, when it needs more
// than `det_limit` bytes (> 0) or the pool has no memory for it, so that the
// caller takes another deterministic kernel); `timeouts` is the device
// address of the process-wide counter of blocks that stopped on a bounded wait
int grid_tm_dispatch(const ::dmr_plan *p, const void *ksp, int kreal, float2 *grid, int64_t batch,
                     const float *weight, int wpb, int det, void *scratch, size_t scratch_bytes, int *timeouts,
                     int stall, int64_t det_limit, cudaStream_t st);

}  // namespace dmr

struct dmr_plan {
    dmr::Geom g;
    int device;
    double scale;                       // kernel-sum normalisation
    std::vector<int64_t> frame_offsets;  // host CSR
    float os[3];
    // device buffers
    float *scoord[3] = {nullptr, nullptr, nullptr};  // sorted rescaled coordinates
    int32_t *sidx = nullptr;            // sorted position -> global sample index
    // 3D tensor-core gridding: bins of its own (tile tg_T, x y z) whose region
    // (tile + W - 1 per axis) is at most 7 x 6 x 6 = 252 points, one N = 256
    // MMA; the samples of a bin in acquisition order (consecutive samples of a
    // spoke, which share 32-byte sectors of k-space, are read together);
    // work items of at most 2048 samples, visited in 4 x 4 x 4-bin tiles.
    // tg_T[0] == 0: not planned.
    int tg_T[3] = {0, 0, 0};
    int tg_nb[3] = {1, 1, 1};
    int tg_nbins = 0;
    float *tg_scoord[3] = {nullptr, nullptr, nullptr};
    int32_t *tg_sidx = nullptr;
    // per sample (gridding order): the Kaiser-Bessel weights of its W taps on
    // each axis, [sample][axis][tg_wp] (tg_wp = 4 for W <= 4, else 8), and the
    // offsets of its first taps inside its bin, x | y << 8 | z << 16
    float *tg_w = nullptr;
    int32_t *tg_l = nullptr;
    int tg_wp = 0;
    dmr::WorkItem *tg_work = nullptr;
    int tg_nwork = 0;
    int32_t *tg_order = nullptr;
    // deterministic mode: the items of each bin, [tg_item_start[k],
    // tg_item_start[k + 1]) of tg_work for bin key k (frame * tg_nbins + bin;
    // items are numbered in key order, a bin's segments in sample order)
    int32_t *tg_item_start = nullptr;
    int32_t *bin_start = nullptr;       // (nframes * nbins + 1)
    dmr::WorkItem *work = nullptr;      // interpolation / atomic gridding items
    int nwork = 0;
    int32_t *work_order = nullptr;      // item order in 4x4x4-bin tiles (L2 reuse of halos and spokes)
    int32_t *tiles = nullptr;           // owner-gridding tile order (heavy first)
    int ntiles = 0;
    // deterministic gridding: whole non-empty bins grouped by colour; bins of
    // one colour have disjoint tile + halo regions
    dmr::WorkItem *det_work = nullptr;
    std::vector<int> det_color_start;   // host, ncolors + 1
    float *apod[3] = {nullptr, nullptr, nullptr};  // per-axis apodisation (image index)
    int64_t *foff_dev = nullptr;        // frame offsets on the device (nframes + 1)
    // register-tile gridding (3D): block items, reduction items for regions
    // split over several blocks, and the number of partial-sum slots
    dmr::RtItem *rt_items = nullptr;
    int nrt = 0;
    dmr::RtItem *rt_reduce = nullptr;
    int nrt_reduce = 0;
    int rt_slots = 0;
    // device status word: blocks of this plan's calls whose bounded wait ran out
    // (dmr_plan_status; 0 while every result is valid)
    int32_t *status = nullptr;

    ~dmr_plan()
    {
        for (int a = 0; a < 3; a++) {
            cudaFree(scoord[a]);
            cudaFree(apod[a]);
        }
        cudaFree(sidx);
        for (int a = 0; a < 3; a++) cudaFree(tg_scoord[a]);
        cudaFree(tg_sidx);
        cudaFree(tg_w);
        cudaFree(tg_l);
        cudaFree(tg_work);
        cudaFree(tg_order);
        cudaFree(tg_item_start);
        cudaFree(bin_start);
        cudaFree(work);
        cudaFree(work_order);
        cudaFree(tiles);
        cudaFree(det_work);
        cudaFree(foff_dev);
        cudaFree(rt_items);
        cudaFree(rt_reduce);
        cudaFree(status);
    }
};
