// Tensor-core gridding for 3D: dispatch, and the health state shared by the
// tensor-core kernels (tmgrid.cu).
//
// Reference: apply_gridding and its 3D kernel
// (src/deepmr/fft/_interp/grid.py:14-125, 253-284):
//   grid[f, b, iz, iy, ix] += value_z * value_y * value_x * y[f, b, p]   (then / scale)
//
// Every wait in the tensor-core kernels is bounded in time (%globaltimer): a
// wait that runs out makes the block stop issuing work, wait (again bounded)
// for its own MMAs in flight, free its tensor memory and count itself in the
// plan's status word and in a process-wide counter. The host reads the status
// with dmr_plan_status (the calls' results are then not valid) and the
// counter with dmr_tc_timeouts; dmr_tc_test_stall makes the waits run out on
// purpose (a barrier that nothing signals) to test that path without a fault.
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <mutex>

#include "plan.cuh"

namespace dmr {

__device__ int g_tc_timeouts = 0;  // blocks whose wait ran out, all plans (should stay 0)

static int tc_disabled()
{
    static const int v = [] {
        const char *e = getenv("DMR_NO_TC");
        return e && atoi(e) ? 1 : 0;
    }();
    return v;
}

static std::atomic<int> g_tc_stall{0};  // test hook (dmr_tc_test_stall)
// largest scratch (bytes) deterministic tensor-core gridding may take, 0: no
// limit (dmr_det_scratch_limit)
static std::atomic<int64_t> g_det_scratch_max{0};

// device address of g_tc_timeouts, looked up once per device (that device current)
static int timeouts_ptr(int dev, int **out)
{
    static std::mutex mu;
    static int *ptrs[64] = {};
    DMR_CHECK(dev >= 0 && dev < 64, DMR_ERR_UNSUPPORTED, "device index %d", dev);
    std::lock_guard<std::mutex> lock(mu);
    if (!ptrs[dev]) DMR_CUDA(cudaGetSymbolAddress((void **)&ptrs[dev], g_tc_timeouts));
    *out = ptrs[dev];
    return DMR_OK;
}

// Tensor-core gridding of a 3D plan with the kernel of tmgrid.cu (atomic, or
// deterministic through per-item partial sums); DMR_ERR_UNSUPPORTED when it does not
// apply or DMR_NO_TC=1 (then the caller uses the CUDA-core kernels).
int grid_tc_dispatch(const dmr_plan *p, const void *ksp, int kreal, float2 *grid, int64_t batch,
                     const float *weight, int wpb, int det, void *scratch, size_t scratch_bytes,
                     cudaStream_t st)
{
    if (tc_disabled()) return DMR_ERR_UNSUPPORTED;
    int dev = 0;
    DMR_CUDA(cudaGetDevice(&dev));
    int *timeouts = nullptr;
    DMR_TRY(timeouts_ptr(dev, &timeouts));
    return grid_tm_dispatch(p, ksp, kreal, grid, batch, weight, wpb, det, scratch, scratch_bytes, timeouts,
                            g_tc_stall.load(), g_det_scratch_max.load(), st);
}

}  // namespace dmr

using namespace dmr;

extern "C" int dmr_tc_timeouts(int64_t *count, int reset)
{
    DMR_CHECK(count, DMR_ERR_INVALID, "count is NULL");
    int v = 0;
    DMR_CUDA(cudaDeviceSynchronize());
    DMR_CUDA(cudaMemcpyFromSymbol(&v, g_tc_timeouts, sizeof(int)));
    *count = v;
    if (reset) {
        const int zero = 0;
        DMR_CUDA(cudaMemcpyToSymbol(g_tc_timeouts, &zero, sizeof(int)));
    }
    return DMR_OK;
}

extern "C" int64_t dmr_det_scratch_limit(int64_t bytes)
{
    return bytes >= 0 ? g_det_scratch_max.exchange(bytes) : g_det_scratch_max.load();
}

extern "C" int dmr_tc_test_stall(int enable)
{
    g_tc_stall.store(enable ? 1 : 0);
    return DMR_OK;
}

extern "C" int dmr_plan_status(dmr_plan *p, int32_t *failed, int reset, void *stream)
{
    DMR_CHECK(p, DMR_ERR_INVALID, "NULL plan");
    cudaStream_t st = (cudaStream_t)stream;
    int32_t v = 0;
    DMR_CUDA(cudaMemcpyAsync(&v, p->status, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    DMR_CUDA(cudaStreamSynchronize(st));
    if (failed) *failed = v;
    if (reset && v) {
        DMR_CUDA(cudaMemsetAsync(p->status, 0, sizeof(int32_t), st));
        DMR_CUDA(cudaStreamSynchronize(st));
    }
    DMR_CHECK(v == 0, DMR_ERR_TIMEOUT,
              "%d tensor-core gridding block(s) of this plan stopped on a bounded wait that ran out: "
              "the results of the calls since the last reset are not valid", (int)v);
    return DMR_OK;
}
