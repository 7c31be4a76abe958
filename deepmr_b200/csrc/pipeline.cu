// NUFFT pipelines around cuFFT: apodisation + zero-pad + ifftshift fused into
// one kernel before the forward transform, fftshift + crop + 1/G +
// apodisation fused into one kernel after the inverse transform, and the
// Toeplitz self-adjoint (pad, FFT, kernel multiply, inverse FFT, crop).
//
// Reference: _apply_nufft / _apply_nufft_adj / _apply_nufft_selfadj
// (src/deepmr/fft/nufft.py:423-669), resize (src/deepmr/_signal/resize.py:11-102),
// centred fft/ifft (src/deepmr/fft/fft.py:9-167), plan_toeplitz
// (src/deepmr/fft/toeplitz.py:131-155).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>

#include "plan.cuh"

namespace dmr {

int interp_dispatch(const dmr_plan *p, const float2 *grid, float2 *ksp, int64_t batch,
                    const float *weight, int wpb, cudaStream_t st);
int grid_dispatch(const dmr_plan *p, const void *ksp, int kreal, float2 *grid, int64_t batch,
                  const float *weight, int wpb, int det, void *scratch, size_t scratch_bytes,
                  cudaStream_t st);

// ---------------------------------------------------------------------------
// Generic centred resize with index rolls and per-axis apodisation:
//   output physical q -> logical lo = (q + oroll) mod O
//   input logical li = lo - so + si, valid for so <= lo < so + cp (resize.py:86-97)
//   input physical = (li + iroll) mod I
//   out = in * scale * apod_x * apod_y * apod_z (apodisation of the image side,
//   applied axis by axis from the last like _apodize, nufft.py:425-445)
// ---------------------------------------------------------------------------
struct ResizeArgs {
    int O[3], I[3];
    int oroll[3], iroll[3];
    int so[3], si[3], cp[3];
    const float *apod[3];
    int apod_on_output;
    float scale;
    int64_t nbatch;
    int64_t osize, isize;
    int in_real;
};

__global__ void __launch_bounds__(128) resize_kernel(ResizeArgs r, const void *__restrict__ in,
                                                     float2 *__restrict__ out)
{
    // one output row (fixed y, z, batch) per block step: the row's y/z index
    // arithmetic and apodisation are computed once, threads run along x
    const int64_t rows_per_batch = (int64_t)r.O[1] * r.O[2];
    const int64_t nrows = rows_per_batch * r.nbatch;
    for (int64_t row = blockIdx.x; row < nrows; row += gridDim.x) {
        const int64_t bi = row / rows_per_batch;
        const int rr = (int)(row - bi * rows_per_batch);
        const int qq[3] = {0, rr % r.O[1], rr / r.O[1]};
        bool rvalid = true;
        int li[3], lo[3], pi[3];
        float rs = r.scale;
#pragma unroll
        for (int a = 1; a < 3; a++) {
            lo[a] = qq[a] + r.oroll[a];
            if (lo[a] >= r.O[a]) lo[a] -= r.O[a];
            rvalid = rvalid && lo[a] >= r.so[a] && lo[a] < r.so[a] + r.cp[a];
            li[a] = lo[a] - r.so[a] + r.si[a];
            pi[a] = li[a] + r.iroll[a];
            if (pi[a] >= r.I[a]) pi[a] -= r.I[a];
            if (rvalid && r.apod[a]) rs *= r.apod[a][r.apod_on_output ? lo[a] : li[a]];
        }
        float2 *orow = out + bi * r.osize + (int64_t)rr * r.O[0];
        if (!rvalid) {
            for (int qx = threadIdx.x; qx < r.O[0]; qx += blockDim.x) orow[qx] = make_float2(0.0f, 0.0f);
            continue;
        }
        const int64_t irow = bi * r.isize + ((int64_t)pi[2] * r.I[1] + pi[1]) * r.I[0];
        for (int qx = threadIdx.x; qx < r.O[0]; qx += blockDim.x) {
            int lx = qx + r.oroll[0];
            if (lx >= r.O[0]) lx -= r.O[0];
            float2 v = make_float2(0.0f, 0.0f);
            if (lx >= r.so[0] && lx < r.so[0] + r.cp[0]) {
                const int ix = lx - r.so[0] + r.si[0];
                int px = ix + r.iroll[0];
                if (px >= r.I[0]) px -= r.I[0];
                if (r.in_real) v.x = reinterpret_cast<const float *>(in)[irow + px];
                else v = reinterpret_cast<const float2 *>(in)[irow + px];
                float sc = rs;
                if (r.apod[0]) sc *= r.apod[0][r.apod_on_output ? lx : ix];
                v.x *= sc;
                v.y *= sc;
            }
            orow[qx] = v;
        }
    }
}

// resize offsets of resize.py:86-91 for one axis of extent i -> o
static void resize_offsets(int i, int o, int &si, int &so, int &cp)
{
    si = std::max(i / 2 - o / 2, 0);
    so = std::max(o / 2 - i / 2, 0);
    cp = std::min(i - si, o - so);
}

static int launch_resize(const ResizeArgs &r, const void *in, float2 *out, cudaStream_t st)
{
    if (r.nbatch == 0 || r.osize == 0) return DMR_OK;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t nrows = (int64_t)r.O[1] * r.O[2] * r.nbatch;
    const unsigned blocks = (unsigned)std::min<int64_t>(nrows, (int64_t)sms * 64);
    resize_kernel<<<blocks, 128, 0, st>>>(r, in, out);
    DMR_LAUNCHED("resize_kernel");
    return DMR_OK;
}

// ---------------------------------------------------------------------------
// cuFFT plan cache (process-wide), work area supplied by the caller
// ---------------------------------------------------------------------------
static std::mutex g_fft_mu;
static std::map<std::tuple<int, int, int, int, int, int64_t>, std::shared_ptr<FftPlan>> g_fft;

std::shared_ptr<FftPlan> get_fft_plan(int ndim, const int *dims_zyx, int64_t batch, int *err)
{
    int dev = 0;
    cudaGetDevice(&dev);
    int d[3] = {1, 1, 1};
    for (int i = 0; i < ndim; i++) d[i] = dims_zyx[i];
    auto key = std::make_tuple(dev, ndim, d[0], d[1], d[2], batch);
    std::lock_guard<std::mutex> lk(g_fft_mu);
    auto it = g_fft.find(key);
    if (it != g_fft.end()) return it->second;
    auto fp = std::make_shared<FftPlan>();
    long long n[3];
    long long dist = 1;
    for (int i = 0; i < ndim; i++) {
        n[i] = dims_zyx[i];
        dist *= n[i];
    }
    cufftResult r = cufftCreate(&fp->handle);
    if (r == CUFFT_SUCCESS) r = cufftSetAutoAllocation(fp->handle, 0);
    size_t ws = 0;
    if (r == CUFFT_SUCCESS)
        r = cufftMakePlanMany64(fp->handle, ndim, n, nullptr, 1, dist, nullptr, 1, dist, CUFFT_C2C,
                                batch, &ws);
    if (r != CUFFT_SUCCESS) {
        set_error("cuFFT plan creation failed (code %d) for batch %lld", (int)r, (long long)batch);
        *err = DMR_ERR_CUFFT;
        if (fp->handle) cufftDestroy(fp->handle);
        return nullptr;
    }
    fp->work_bytes = ws;
    g_fft[key] = fp;
    *err = DMR_OK;
    return fp;
}

static int fft_exec(FftPlan &fp, float2 *data, int direction, void *work, cudaStream_t st)
{
    std::lock_guard<std::mutex> lk(fp.mu);
    cufftResult r = cufftSetStream(fp.handle, st);
    if (r == CUFFT_SUCCESS) r = cufftSetWorkArea(fp.handle, work);
    if (r == CUFFT_SUCCESS)
        r = cufftExecC2C(fp.handle, (cufftComplex *)data, (cufftComplex *)data, direction);
    DMR_CHECK(r == CUFFT_SUCCESS, DMR_ERR_CUFFT, "cufftExecC2C failed (code %d)", (int)r);
    return DMR_OK;
}

static void zyx_dims(const Geom &g, const int *ext, int out[3])
{
    for (int i = 0; i < g.ndim; i++) out[i] = ext[g.ndim - 1 - i];
}

struct NufftWs {
    float2 *grid;
    void *fft_work;
    void *rt_scratch;  // register-tile gridding partial sums (split regions)
    size_t rt_bytes;
    std::shared_ptr<FftPlan> fft;
};

static int nufft_ws(dmr_plan *p, int64_t batch, void *ws, size_t ws_bytes, NufftWs &out, size_t *need)
{
    const Geom &g = p->g;
    // the fused FFT passes need no cuFFT plan or work area
    std::shared_ptr<FftPlan> fp;
    if (!fft3_applies(p)) {
        int dims[3];
        zyx_dims(g, g.G, dims);
        int err = DMR_OK;
        fp = get_fft_plan(g.ndim, dims, batch * g.nframes, &err);
        if (!fp) return err;
    }
    const size_t grid_bytes = align_up((size_t)batch * g.nframes * g.gsize * sizeof(float2), 256);
    const size_t fft_bytes = fp ? align_up(fp->work_bytes, 256) : 0;
    const size_t rt_bytes = align_up(grid_scratch_bytes(p, batch), 256);
    const size_t total = grid_bytes + fft_bytes + rt_bytes;
    if (need) *need = total;
    if (!ws) return DMR_OK;
    DMR_CHECK(ws_bytes >= total, DMR_ERR_WORKSPACE, "workspace too small: %zu < %zu", ws_bytes, total);
    DMR_CHECK(((uintptr_t)ws & 255) == 0, DMR_ERR_INVALID, "workspace must be 256-byte aligned");
    out.grid = (float2 *)ws;
    out.fft_work = fp && fp->work_bytes ? (char *)ws + grid_bytes : nullptr;
    out.rt_scratch = rt_bytes ? (char *)ws + grid_bytes + fft_bytes : nullptr;
    out.rt_bytes = rt_bytes;
    out.fft = fp;
    return DMR_OK;
}

__device__ __forceinline__ float2 cmul_scaled(float2 k, float2 d, float s)
{
    // kernel value times spectrum (toeplitz.py:86), then the two orthonormal 1/sqrt(K)
    float2 o = make_float2(k.x * d.x - k.y * d.y, k.x * d.y + k.y * d.x);
    o.x *= s;
    o.y *= s;
    return o;
}

// data[b] *= kern[b mod nk] * s, per batch row (blockIdx.y); two complex values
// per thread with 16-byte accesses when vec (even row length, 16-byte aligned
// data and kernel)
__global__ void __launch_bounds__(256) cmul_kernel(float2 *__restrict__ data, const float2 *__restrict__ kern,
                                                   int64_t ksize, int64_t nk, int64_t nbatch, float s, int vec)
{
    for (int64_t bi = blockIdx.y; bi < nbatch; bi += gridDim.y) {
        float2 *d = data + bi * ksize;
        const float2 *k = kern + (bi % nk) * ksize;
        const int64_t step = (int64_t)gridDim.x * blockDim.x;
        if (vec) {
            float4 *d4 = reinterpret_cast<float4 *>(d);
            const float4 *k4 = reinterpret_cast<const float4 *>(k);
            for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ksize / 2; e += step) {
                const float4 dv = d4[e], kv = __ldg(k4 + e);
                const float2 a = cmul_scaled(make_float2(kv.x, kv.y), make_float2(dv.x, dv.y), s);
                const float2 c = cmul_scaled(make_float2(kv.z, kv.w), make_float2(dv.z, dv.w), s);
                d4[e] = make_float4(a.x, a.y, c.x, c.y);
            }
        } else {
            for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ksize; e += step)
                d[e] = cmul_scaled(k[e], d[e], s);
        }
    }
}

// mean of |k| over the non-zero entries (toeplitz.py:152), two-stage in float64
__global__ void absmean_partial_kernel(const float2 *__restrict__ k, int64_t n, double *__restrict__ sums,
                                       unsigned long long *__restrict__ counts)
{
    double s = 0.0;
    unsigned long long c = 0;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x) {
        const float2 v = k[e];
        if (v.x != 0.0f || v.y != 0.0f) {
            s += (double)hypotf(v.x, v.y);
            c++;
        }
    }
    __shared__ double ss[256];
    __shared__ unsigned long long sc[256];
    ss[threadIdx.x] = s;
    sc[threadIdx.x] = c;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            ss[threadIdx.x] += ss[threadIdx.x + h];
            sc[threadIdx.x] += sc[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        sums[blockIdx.x] = ss[0];
        counts[blockIdx.x] = sc[0];
    }
}

__global__ void normalise_kernel(float2 *__restrict__ k, int64_t n, const double *__restrict__ sums,
                                 const unsigned long long *__restrict__ counts, int nparts)
{
    __shared__ float inv_mean;
    if (threadIdx.x == 0) {
        double s = 0.0;
        unsigned long long c = 0;
        for (int i = 0; i < nparts; i++) {
            s += sums[i];
            c += counts[i];
        }
        // mean of an empty selection is NaN in the reference; keep that
        const float mean = c ? (float)(s / (double)c) : __int_as_float(0x7fc00000);
        inv_mean = mean;
    }
    __syncthreads();
    const float m = inv_mean;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x) {
        float2 v = k[e];
        v.x = v.x / m;
        v.y = v.y / m;
        // torch.nan_to_num: NaN -> 0, +-inf -> +-FLT_MAX
        if (isnan(v.x)) v.x = 0.0f; else if (isinf(v.x)) v.x = v.x > 0 ? 3.402823466e38f : -3.402823466e38f;
        if (isnan(v.y)) v.y = 0.0f; else if (isinf(v.y)) v.y = v.y > 0 ? 3.402823466e38f : -3.402823466e38f;
        k[e] = v;
    }
}

constexpr int kReduceBlocks = 296;

static int elem_blocks(int64_t n)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 256), (int64_t)sms * 8));
}

}  // namespace dmr

using namespace dmr;

extern "C" int dmr_nufft_workspace_bytes(dmr_plan *p, int64_t batch, size_t *bytes)
{
    DMR_CHECK(p && bytes && batch >= 1, DMR_ERR_INVALID, "bad argument");
    NufftWs w;
    return nufft_ws(p, batch, nullptr, 0, w, bytes);
}

namespace dmr {

// workspace carve + apodise/zero-pad/ifftshift + forward cuFFT: the grid of
// the forward NUFFT (FFT order), shared by the forward and the trajectory
// gradient
int forward_grid(dmr_plan *p, const void *image, int image_real, int64_t batch, void *workspace,
                 size_t workspace_bytes, cudaStream_t st, float2 **grid_out)
{
    const Geom &g = p->g;
    NufftWs w;
    DMR_TRY(nufft_ws(p, batch, workspace, workspace_bytes, w, nullptr));
    if (!w.fft) {
        DMR_TRY(fft3_forward(p, image, image_real, batch, w.grid, st));
        *grid_out = w.grid;
        return DMR_OK;
    }
    ResizeArgs r;
    memset(&r, 0, sizeof(r));
    for (int a = 0; a < 3; a++) {
        r.O[a] = g.G[a];
        r.I[a] = g.N[a];
        r.oroll[a] = g.half[a];  // X[q] = P[(q + G//2) mod G]: ifftshift folded in
        r.iroll[a] = 0;
        resize_offsets(g.N[a], g.G[a], r.si[a], r.so[a], r.cp[a]);
        r.apod[a] = (a < g.ndim && g.W[a] != 1) ? p->apod[a] : nullptr;
    }
    r.apod_on_output = 0;
    r.scale = 1.0f;
    r.nbatch = batch * g.nframes;
    r.osize = g.gsize;
    r.isize = g.isize;
    r.in_real = image_real;
    DMR_TRY(launch_resize(r, image, w.grid, st));
    DMR_TRY(fft_exec(*w.fft, w.grid, CUFFT_FORWARD, w.fft_work, st));
    *grid_out = w.grid;
    return DMR_OK;
}

}  // namespace dmr

extern "C" int dmr_nufft_forward(dmr_plan *p, const void *image, int image_real, void *kspace,
                                 int64_t batch, const float *weight, int weight_per_batch,
                                 void *workspace, size_t workspace_bytes, void *stream)
{
    DMR_CHECK(p && image && kspace && batch >= 1, DMR_ERR_INVALID, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    float2 *grid = nullptr;
    DMR_TRY(forward_grid(p, image, image_real, batch, workspace, workspace_bytes, st, &grid));
    return interp_dispatch(p, grid, (float2 *)kspace, batch, weight, weight_per_batch, st);
}

extern "C" int dmr_nufft_adjoint(dmr_plan *p, const void *kspace, int kspace_real, void *image,
                                 int64_t batch, const float *weight, int weight_per_batch,
                                 int deterministic, void *workspace, size_t workspace_bytes,
                                 void *stream)
{
    DMR_CHECK(p && image && kspace && batch >= 1, DMR_ERR_INVALID, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    const Geom &g = p->g;
    NufftWs w;
    DMR_TRY(nufft_ws(p, batch, workspace, workspace_bytes, w, nullptr));
    DMR_TRY(grid_dispatch(p, kspace, kspace_real, w.grid, batch, weight, weight_per_batch,
                          deterministic, w.rt_scratch, w.rt_bytes, st));
    if (!w.fft) return fft3_adjoint(p, w.grid, batch, (float2 *)image, st);
    DMR_TRY(fft_exec(*w.fft, w.grid, CUFFT_INVERSE, w.fft_work, st));
    ResizeArgs r;
    memset(&r, 0, sizeof(r));
    for (int a = 0; a < 3; a++) {
        r.O[a] = g.N[a];
        r.I[a] = g.G[a];
        r.oroll[a] = 0;
        r.iroll[a] = g.G[a] - g.half[a];  // fftshift folded in: centred li at (li - G//2) mod G
        if (r.iroll[a] == g.G[a]) r.iroll[a] = 0;
        resize_offsets(g.G[a], g.N[a], r.si[a], r.so[a], r.cp[a]);
        r.apod[a] = (a < g.ndim && g.W[a] != 1) ? p->apod[a] : nullptr;
    }
    r.apod_on_output = 1;
    r.scale = (float)(1.0 / (double)g.gsize);  // ifftn norm="backward" (nufft.py:587)
    r.nbatch = batch * g.nframes;
    r.osize = g.isize;
    r.isize = g.gsize;
    r.in_real = 0;
    return launch_resize(r, w.grid, (float2 *)image, st);
}

static int toep_dims(int ndim, const int32_t *kshape, int dims[3], int64_t &ksize)
{
    DMR_CHECK(ndim >= 1 && ndim <= 3 && kshape, DMR_ERR_INVALID, "bad Toeplitz shape");
    ksize = 1;
    for (int i = 0; i < ndim; i++) {
        DMR_CHECK(kshape[i] >= 1, DMR_ERR_INVALID, "bad Toeplitz shape");
        dims[i] = kshape[i];
        ksize *= kshape[i];
    }
    return DMR_OK;
}

// ---------------------------------------------------------------------------
// Low-rank subspace NUFFT (reference: _interpolate_lowrank* / _gridding_lowrank*,
// src/deepmr/fft/_interp/interp.py:230-357 and grid.py:287-417): frame f of
// the forward transform interpolates sum_c basis_adjoint[f, c] * FFT(coefficient
// image c); the adjoint grids every frame and projects with basis[c, f]. The
// subspace projection commutes with apodisation, padding and the FFT, so the
// pipelines transform the ncoeff coefficient images and combine grids.
// ---------------------------------------------------------------------------
namespace dmr {

constexpr int kMaxCoeff = 32;

// out[b, i, p] = sum_j M[i, j] in[b, j, p] with few inputs (nin <= kMaxCoeff):
// a thread holds the nin input values of one grid point
__global__ void __launch_bounds__(256) combine_few_in_kernel(const float2 *__restrict__ in, float2 *__restrict__ out,
                                                            const float2 *__restrict__ M, int nin, int nout,
                                                            int64_t npts, int64_t nbatch)
{
    for (int64_t b = blockIdx.y; b < nbatch; b += gridDim.y) {
        for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npts;
             p += (int64_t)gridDim.x * blockDim.x) {
            float2 v[kMaxCoeff];
#pragma unroll
            for (int j = 0; j < kMaxCoeff; j++)
                v[j] = j < nin ? in[(b * nin + j) * npts + p] : make_float2(0.0f, 0.0f);
            for (int i = 0; i < nout; i++) {
                float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
                for (int j = 0; j < kMaxCoeff; j++) {
                    if (j < nin) {
                        const float2 m = __ldg(M + (int64_t)i * nin + j);
                        acc.x += m.x * v[j].x - m.y * v[j].y;
                        acc.y += m.x * v[j].y + m.y * v[j].x;
                    }
                }
                out[(b * nout + i) * npts + p] = acc;
            }
        }
    }
}

// the same with few outputs (nout <= kMaxCoeff): a thread streams the inputs
// of one grid point and keeps the nout sums
__global__ void __launch_bounds__(256) combine_few_out_kernel(const float2 *__restrict__ in, float2 *__restrict__ out,
                                                             const float2 *__restrict__ M, int nin, int nout,
                                                             int64_t npts, int64_t nbatch)
{
    for (int64_t b = blockIdx.y; b < nbatch; b += gridDim.y) {
        for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npts;
             p += (int64_t)gridDim.x * blockDim.x) {
            float2 acc[kMaxCoeff];
#pragma unroll
            for (int i = 0; i < kMaxCoeff; i++) acc[i] = make_float2(0.0f, 0.0f);
            for (int j = 0; j < nin; j++) {
                const float2 v = in[(b * nin + j) * npts + p];
#pragma unroll
                for (int i = 0; i < kMaxCoeff; i++) {
                    if (i < nout) {
                        const float2 m = __ldg(M + (int64_t)i * nin + j);
                        acc[i].x += m.x * v.x - m.y * v.y;
                        acc[i].y += m.x * v.y + m.y * v.x;
                    }
                }
            }
#pragma unroll
            for (int i = 0; i < kMaxCoeff; i++)
                if (i < nout) out[(b * nout + i) * npts + p] = acc[i];
        }
    }
}

static int launch_combine(const float2 *in, float2 *out, const float2 *M, int nin, int nout, int64_t npts,
                          int64_t nbatch, cudaStream_t st)
{
    DMR_CHECK(nin <= kMaxCoeff || nout <= kMaxCoeff, DMR_ERR_UNSUPPORTED,
              "subspace projection with more than %d coefficients", kMaxCoeff);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned gy = (unsigned)std::min<int64_t>(nbatch, 65535);
    const unsigned gx = (unsigned)std::max<int64_t>(
        1, std::min<int64_t>(ceil_div(npts, 256), ceil_div((int64_t)sms * 8, gy)));
    if (nin <= kMaxCoeff && (nin <= nout || nout > kMaxCoeff))
        combine_few_in_kernel<<<dim3(gx, gy), 256, 0, st>>>(in, out, M, nin, nout, npts, nbatch);
    else
        combine_few_out_kernel<<<dim3(gx, gy), 256, 0, st>>>(in, out, M, nin, nout, npts, nbatch);
    DMR_LAUNCHED("combine_kernel");
    return DMR_OK;
}

struct LowrankWs {
    float2 *coef;   // (batch, ncoeff, *G)
    float2 *frame;  // (batch, nframes, *G)
    void *fft_work;
    void *rt_scratch;
    size_t rt_bytes;
    std::shared_ptr<FftPlan> fft;
};

static int lowrank_ws(dmr_plan *p, int64_t batch, int64_t ncoeff, void *ws, size_t ws_bytes, LowrankWs &out,
                      size_t *need)
{
    const Geom &g = p->g;
    DMR_CHECK(ncoeff >= 1 && ncoeff <= kMaxCoeff, DMR_ERR_UNSUPPORTED,
              "ncoeff must be in [1, %d] (got %lld)", kMaxCoeff, (long long)ncoeff);
    int dims[3];
    zyx_dims(g, g.G, dims);
    int err = DMR_OK;
    auto fp = get_fft_plan(g.ndim, dims, batch * ncoeff, &err);
    if (!fp) return err;
    const size_t coef_bytes = align_up((size_t)batch * ncoeff * g.gsize * sizeof(float2), 256);
    const size_t frame_bytes = align_up((size_t)batch * g.nframes * g.gsize * sizeof(float2), 256);
    const size_t fft_bytes = align_up(fp->work_bytes, 256);
    const size_t rt_bytes = align_up(grid_scratch_bytes(p, batch), 256);
    const size_t total = coef_bytes + frame_bytes + fft_bytes + rt_bytes;
    if (need) *need = total;
    if (!ws) return DMR_OK;
    DMR_CHECK(ws_bytes >= total, DMR_ERR_WORKSPACE, "workspace too small: %zu < %zu", ws_bytes, total);
    DMR_CHECK(((uintptr_t)ws & 255) == 0, DMR_ERR_INVALID, "workspace must be 256-byte aligned");
    char *c = (char *)ws;
    out.coef = (float2 *)c;
    out.frame = (float2 *)(c + coef_bytes);
    out.fft_work = fp->work_bytes ? c + coef_bytes + frame_bytes : nullptr;
    out.rt_scratch = rt_bytes ? c + coef_bytes + frame_bytes + fft_bytes : nullptr;
    out.rt_bytes = rt_bytes;
    out.fft = fp;
    return DMR_OK;
}

}  // namespace dmr

extern "C" int dmr_nufft_lowrank_workspace_bytes(dmr_plan *p, int64_t batch, int64_t ncoeff, size_t *bytes)
{
    DMR_CHECK(p && bytes && batch >= 1, DMR_ERR_INVALID, "bad argument");
    LowrankWs w;
    return lowrank_ws(p, batch, ncoeff, nullptr, 0, w, bytes);
}

extern "C" int dmr_nufft_forward_lowrank(dmr_plan *p, const void *image, int image_real, int64_t ncoeff,
                                         const void *basis_adjoint, void *kspace, int64_t batch,
                                         const float *weight, int weight_per_batch, void *workspace,
                                         size_t workspace_bytes, void *stream)
{
    DMR_CHECK(p && image && kspace && basis_adjoint && batch >= 1, DMR_ERR_INVALID, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    const Geom &g = p->g;
    LowrankWs w;
    DMR_TRY(lowrank_ws(p, batch, ncoeff, workspace, workspace_bytes, w, nullptr));
    ResizeArgs r;
    memset(&r, 0, sizeof(r));
    for (int a = 0; a < 3; a++) {
        r.O[a] = g.G[a];
        r.I[a] = g.N[a];
        r.oroll[a] = g.half[a];  // ifftshift folded in
        r.iroll[a] = 0;
        resize_offsets(g.N[a], g.G[a], r.si[a], r.so[a], r.cp[a]);
        r.apod[a] = (a < g.ndim && g.W[a] != 1) ? p->apod[a] : nullptr;
    }
    r.apod_on_output = 0;
    r.scale = 1.0f;
    r.nbatch = batch * ncoeff;
    r.osize = g.gsize;
    r.isize = g.isize;
    r.in_real = image_real;
    DMR_TRY(launch_resize(r, image, w.coef, st));
    DMR_TRY(fft_exec(*w.fft, w.coef, CUFFT_FORWARD, w.fft_work, st));
    DMR_TRY(launch_combine(w.coef, w.frame, (const float2 *)basis_adjoint, (int)ncoeff, g.nframes, g.gsize,
                           batch, st));
    return interp_dispatch(p, w.frame, (float2 *)kspace, batch, weight, weight_per_batch, st);
}

extern "C" int dmr_nufft_adjoint_lowrank(dmr_plan *p, const void *kspace, int kspace_real, int64_t ncoeff,
                                         const void *basis, void *image, int64_t batch, const float *weight,
                                         int weight_per_batch, int deterministic, void *workspace,
                                         size_t workspace_bytes, void *stream)
{
    DMR_CHECK(p && image && kspace && basis && batch >= 1, DMR_ERR_INVALID, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    const Geom &g = p->g;
    LowrankWs w;
    DMR_TRY(lowrank_ws(p, batch, ncoeff, workspace, workspace_bytes, w, nullptr));
    DMR_TRY(grid_dispatch(p, kspace, kspace_real, w.frame, batch, weight, weight_per_batch, deterministic,
                          w.rt_scratch, w.rt_bytes, st));
    DMR_TRY(launch_combine(w.frame, w.coef, (const float2 *)basis, g.nframes, (int)ncoeff, g.gsize, batch, st));
    DMR_TRY(fft_exec(*w.fft, w.coef, CUFFT_INVERSE, w.fft_work, st));
    ResizeArgs r;
    memset(&r, 0, sizeof(r));
    for (int a = 0; a < 3; a++) {
        r.O[a] = g.N[a];
        r.I[a] = g.G[a];
        r.oroll[a] = 0;
        r.iroll[a] = g.G[a] - g.half[a];  // fftshift folded in
        if (r.iroll[a] == g.G[a]) r.iroll[a] = 0;
        resize_offsets(g.G[a], g.N[a], r.si[a], r.so[a], r.cp[a]);
        r.apod[a] = (a < g.ndim && g.W[a] != 1) ? p->apod[a] : nullptr;
    }
    r.apod_on_output = 1;
    r.scale = (float)(1.0 / (double)g.gsize);  // ifftn norm="backward"
    r.nbatch = batch * ncoeff;
    r.osize = g.isize;
    r.isize = g.gsize;
    r.in_real = 0;
    return launch_resize(r, w.coef, (float2 *)image, st);
}

extern "C" int dmr_toeplitz_workspace_bytes(int ndim, const int32_t *kshape, int64_t batch, size_t *bytes)
{
    DMR_CHECK(bytes && batch >= 1, DMR_ERR_INVALID, "bad argument");
    int dims[3];
    int64_t ksize;
    DMR_TRY(toep_dims(ndim, kshape, dims, ksize));
    int err = DMR_OK;
    auto fp = get_fft_plan(ndim, dims, batch, &err);
    if (!fp) return err;
    *bytes = align_up((size_t)batch * ksize * sizeof(float2), 256) + align_up(fp->work_bytes, 256) +
             align_up(kReduceBlocks * (sizeof(double) + sizeof(unsigned long long)), 256);
    return DMR_OK;
}

// carve the Toeplitz workspace: data | cuFFT work | reduction scratch
static int toep_ws(int ndim, const int32_t *kshape, int64_t batch, void *ws, size_t ws_bytes,
                   float2 **data, void **work, double **sums, unsigned long long **counts,
                   std::shared_ptr<FftPlan> &fp)
{
    int dims[3];
    int64_t ksize;
    DMR_TRY(toep_dims(ndim, kshape, dims, ksize));
    int err = DMR_OK;
    fp = get_fft_plan(ndim, dims, batch, &err);
    if (!fp) return err;
    const size_t a = align_up((size_t)batch * ksize * sizeof(float2), 256);
    const size_t b = align_up(fp->work_bytes, 256);
    const size_t c = align_up(kReduceBlocks * (sizeof(double) + sizeof(unsigned long long)), 256);
    DMR_CHECK(ws && ws_bytes >= a + b + c, DMR_ERR_WORKSPACE, "workspace too small: %zu < %zu",
              ws_bytes, a + b + c);
    DMR_CHECK(((uintptr_t)ws & 255) == 0, DMR_ERR_INVALID, "workspace must be 256-byte aligned");
    *data = (float2 *)ws;
    *work = fp->work_bytes ? (char *)ws + a : nullptr;
    *sums = (double *)((char *)ws + a + b);
    *counts = (unsigned long long *)(*sums + kReduceBlocks);
    return DMR_OK;
}

extern "C" int dmr_toeplitz_finalize(int ndim, const int32_t *kshape, int64_t nk, const void *psf,
                                     void *kernel, void *workspace, size_t workspace_bytes,
                                     void *stream)
{
    DMR_CHECK(psf && kernel && nk >= 1, DMR_ERR_INVALID, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    float2 *data;
    void *work;
    double *sums;
    unsigned long long *counts;
    std::shared_ptr<FftPlan> fp;
    DMR_TRY(toep_ws(ndim, kshape, nk, workspace, workspace_bytes, &data, &work, &sums, &counts, fp));
    ResizeArgs r;
    memset(&r, 0, sizeof(r));
    int64_t ksize = 1;
    for (int a = 0; a < 3; a++) {
        const int ext = a < ndim ? kshape[ndim - 1 - a] : 1;
        r.O[a] = r.I[a] = r.cp[a] = ext;
        r.iroll[a] = ext / 2;  // ifftshift: out[q] = in[(q + n//2) mod n]
        if (r.iroll[a] == ext) r.iroll[a] = 0;
        ksize *= ext;
    }
    r.scale = 1.0f;
    r.nbatch = nk;
    r.osize = r.isize = ksize;
    DMR_TRY(launch_resize(r, psf, data, st));
    DMR_TRY(fft_exec(*fp, data, CUFFT_FORWARD, work, st));
    // fftshift then ifftshift cancel; the orthonormal 1/sqrt(K) cancels in the
    // normalisation but is applied so zero tests see the same values
    const float ortho = (float)(1.0 / std::sqrt((double)ksize));
    const int64_t n = nk * ksize;
    ResizeArgs s;
    memset(&s, 0, sizeof(s));
    for (int a = 0; a < 3; a++) {
        s.O[a] = s.I[a] = s.cp[a] = r.O[a];
    }
    s.scale = ortho;
    s.nbatch = nk;
    s.osize = s.isize = ksize;
    DMR_TRY(launch_resize(s, data, (float2 *)kernel, st));
    absmean_partial_kernel<<<kReduceBlocks, 256, 0, st>>>((const float2 *)kernel, n, sums, counts);
    DMR_LAUNCHED("absmean_partial_kernel");
    normalise_kernel<<<elem_blocks(n), 256, 0, st>>>((float2 *)kernel, n, sums, counts, kReduceBlocks);
    DMR_LAUNCHED("normalise_kernel");
    return DMR_OK;
}

extern "C" int dmr_toeplitz_apply(int ndim, const int32_t *kshape, const int32_t *ishape,
                                  const void *kernel, int64_t nk, const void *image, int image_real,
                                  void *out, int64_t batch, void *workspace, size_t workspace_bytes,
                                  void *stream)
{
    DMR_CHECK(kernel && image && out && ishape && nk >= 1 && batch >= 1, DMR_ERR_INVALID,
              "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    float2 *data;
    void *work;
    double *sums;
    unsigned long long *counts;
    std::shared_ptr<FftPlan> fp;
    DMR_TRY(toep_ws(ndim, kshape, batch, workspace, workspace_bytes, &data, &work, &sums, &counts, fp));
    if (toep3_applies(ndim, kshape, ishape))
        return fft3_toeplitz(ndim, kshape, ishape, (const float2 *)kernel, nk, image, image_real, (float2 *)out,
                             batch, data, st);
    ResizeArgs r;
    memset(&r, 0, sizeof(r));
    int64_t ksize = 1, isize = 1;
    for (int a = 0; a < 3; a++) {
        const int K = a < ndim ? kshape[ndim - 1 - a] : 1;
        const int N = a < ndim ? ishape[ndim - 1 - a] : 1;
        r.O[a] = K;
        r.I[a] = N;
        resize_offsets(N, K, r.si[a], r.so[a], r.cp[a]);
        ksize *= K;
        isize *= N;
    }
    r.scale = 1.0f;
    r.nbatch = batch;
    r.osize = ksize;
    r.isize = isize;
    r.in_real = image_real;
    DMR_TRY(launch_resize(r, image, data, st));
    DMR_TRY(fft_exec(*fp, data, CUFFT_FORWARD, work, st));
    {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const unsigned gy = (unsigned)std::min<int64_t>(batch, 65535);
        const int64_t per_row = ceil_div(ksize / 2 + 1, 256);
        const unsigned gx = (unsigned)std::max<int64_t>(1, std::min<int64_t>(per_row, ceil_div((int64_t)sms * 16, gy)));
        const int vec = (ksize % 2 == 0) && ((uintptr_t)data % 16 == 0) && ((uintptr_t)kernel % 16 == 0);
        cmul_kernel<<<dim3(gx, gy), 256, 0, st>>>(data, (const float2 *)kernel, ksize, nk, batch,
                                                  (float)(1.0 / (double)ksize), vec);
    }
    DMR_LAUNCHED("cmul_kernel");
    DMR_TRY(fft_exec(*fp, data, CUFFT_INVERSE, work, st));
    ResizeArgs c;
    memset(&c, 0, sizeof(c));
    for (int a = 0; a < 3; a++) {
        c.O[a] = r.I[a];
        c.I[a] = r.O[a];
        resize_offsets(c.I[a], c.O[a], c.si[a], c.so[a], c.cp[a]);
    }
    c.scale = 1.0f;
    c.nbatch = batch;
    c.osize = isize;
    c.isize = ksize;
    return launch_resize(c, data, (float2 *)out, st);
}

// ---------------------------------------------------------------------------
// Allocation-free Toeplitz kernel normalisation (dmr_toeplitz_normalize_noalloc).
//
// For callers that may not allocate device memory: the partial sums of the
// |k| reduction live in a file-scope static device array instead of a caller
// workspace. The array is a fixed 64 KB that every device loading this
// library keeps until process exit; it holds kNoAllocParts partial results of
// kNoAllocPerPart elements each, which bounds the input size.
// ---------------------------------------------------------------------------
namespace dmr {

constexpr int kNoAllocParts = 4096;
constexpr int64_t kNoAllocPerPart = 16384;
constexpr int64_t kNoAllocMaxElems = (int64_t)kNoAllocParts * kNoAllocPerPart;  // 67,108,864

// partial sums in [0, kNoAllocParts), partial counts (as 64-bit integers) after
static __device__ __align__(256) double g_norm_scratch[2 * kNoAllocParts];

// one contiguous slice of kNoAllocPerPart elements per block
__global__ void absmean_slice_kernel(const float2 *__restrict__ k, int64_t n, int64_t per_part,
                                     double *__restrict__ sums, unsigned long long *__restrict__ counts)
{
    const int64_t lo = blockIdx.x * per_part;
    const int64_t hi = min(n, lo + per_part);
    double s = 0.0;
    unsigned long long c = 0;
    for (int64_t e = lo + threadIdx.x; e < hi; e += blockDim.x) {
        const float2 v = k[e];
        if (v.x != 0.0f || v.y != 0.0f) {
            s += (double)hypotf(v.x, v.y);
            c++;
        }
    }
    __shared__ double ss[256];
    __shared__ unsigned long long sc[256];
    ss[threadIdx.x] = s;
    sc[threadIdx.x] = c;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            ss[threadIdx.x] += ss[threadIdx.x + h];
            sc[threadIdx.x] += sc[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {  // every partial is overwritten: nothing needs clearing
        sums[blockIdx.x] = ss[0];
        counts[blockIdx.x] = sc[0];
    }
}

// Device address of g_norm_scratch for the current device, looked up once per
// device with that device current (the host-side name is only a stand-in).
static int norm_scratch(double **out)
{
    static std::mutex mu;
    static double *addr[128] = {};
    int dev = 0;
    DMR_CUDA(cudaGetDevice(&dev));
    DMR_CHECK(dev >= 0 && dev < 128, DMR_ERR_UNSUPPORTED, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lk(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        DMR_CUDA(cudaGetSymbolAddress(&p, g_norm_scratch));
        addr[dev] = (double *)p;
    }
    *out = addr[dev];
    return DMR_OK;
}

}  // namespace dmr

extern "C" int dmr_toeplitz_normalize_noalloc(void *kernel, int64_t n, void *stream)
{
    DMR_CHECK(kernel && n >= 1, DMR_ERR_INVALID, "bad argument");
    DMR_CHECK(n <= kNoAllocMaxElems, DMR_ERR_INVALID,
              "n = %lld exceeds the %lld-element maximum of the allocation-free normalisation "
              "(use dmr_toeplitz_finalize with a workspace)",
              (long long)n, (long long)kNoAllocMaxElems);
    cudaStream_t st = (cudaStream_t)stream;
    double *sums = nullptr;
    DMR_TRY(norm_scratch(&sums));
    unsigned long long *counts = reinterpret_cast<unsigned long long *>(sums + kNoAllocParts);
    const int nparts = (int)ceil_div(n, kNoAllocPerPart);
    absmean_slice_kernel<<<nparts, 256, 0, st>>>((const float2 *)kernel, n, kNoAllocPerPart, sums, counts);
    DMR_LAUNCHED("absmean_slice_kernel");
    normalise_kernel<<<elem_blocks(n), 256, 0, st>>>((float2 *)kernel, n, sums, counts, nparts);
    DMR_LAUNCHED("normalise_kernel");
    return DMR_OK;
}
