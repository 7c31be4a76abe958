// NUFFT plan construction on the device: Cartesian-axis test, coordinate
// rescale, spatial binning and a stable sort of the samples by (bin, cell).
//
// Reference: plan_nufft (src/deepmr/fft/nufft.py:27-132) and
// plan_interpolator (src/deepmr/fft/_interp/plan.py:14-143). The reference
// materialises per-axis (F, M, W) index/value tables on the CPU; this plan
// keeps only the rescaled coordinates, sorted by bin, and the kernels
// evaluate the Kaiser-Bessel weights on the fly.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>

#include "kb.cuh"
#include "plan.cuh"

namespace dmr {

std::atomic<int64_t> g_launches{0};
static thread_local char t_err[1024] = "";

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_err, sizeof(t_err), fmt, ap);
    va_end(ap);
}

// ---------------------------------------------------------------------------
// Cartesian-axis test (src/deepmr/fft/nufft.py:104-109): numpy.allclose of
// s = N * c against round(s), evaluated in float32 like numpy does for a
// float32 array with Python-float tolerances.
// ---------------------------------------------------------------------------
__global__ void cartesian_kernel(const float *__restrict__ coord, int64_t npts, int ndim,
                                 float n0, float n1, float n2, int *__restrict__ flags)
{
    const float nn[3] = {n0, n1, n2};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npts;
         i += (int64_t)gridDim.x * blockDim.x) {
        for (int a = 0; a < ndim; a++) {
            const float s = __fmul_rn(nn[a], coord[i * ndim + a]);
            const float r = rintf(s);
            const float tol = __fadd_rn(1e-8f, __fmul_rn(1e-5f, fabsf(r)));
            const bool close = ((fabsf(__fsub_rn(s, r)) <= tol) && isfinite(r)) || (s == r);
            if (!close) flags[a] = 0;
        }
    }
}

// ---------------------------------------------------------------------------
// Rescale (nufft.py:411-420: float32 multiply, then float32 add), first tap
// x0 = ceil(k - W/2) in float64 like the reference (plan.py:260), wrap, bin.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int first_tap(float k, int W)
{
    if (W == 1) return (int)k;  // Cartesian axis: truncation (plan.py:117-121)
    return (int)ceil((double)k - 0.5 * (double)W);
}

__global__ void preprocess_kernel(Geom g, const float *__restrict__ coord,
                                  const int64_t *__restrict__ foff, float s0, float s1, float s2,
                                  float h0, float h1, float h2, float *__restrict__ rk0,
                                  float *__restrict__ rk1, float *__restrict__ rk2,
                                  int32_t *__restrict__ keys, int32_t *__restrict__ vals,
                                  int32_t *__restrict__ counts, int *__restrict__ err, int cell_order)
{
    const float sc[3] = {s0, s1, s2};
    const float sh[3] = {h0, h1, h2};
    float *rk[3] = {rk0, rk1, rk2};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < g.total;
         i += (int64_t)gridDim.x * blockDim.x) {
        // frame of sample i: last f with foff[f] <= i
        int lo = 0, hi = g.nframes;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (foff[mid] <= i) lo = mid; else hi = mid;
        }
        int b[3] = {0, 0, 0}, l[3] = {0, 0, 0};
        for (int a = 0; a < g.ndim; a++) {
            float k = __fadd_rn(__fmul_rn(coord[i * g.ndim + a], sc[a]), sh[a]);
            if (!(fabsf(k) < 1.0e8f)) {  // non-finite or absurd coordinate
                atomicOr(err, 1);
                k = 0.0f;
            }
            rk[a][i] = k;
            const int x0m = pmod(first_tap(k, g.W[a]), g.G[a]);
            b[a] = x0m / g.T[a];
            l[a] = x0m - b[a] * g.T[a];
        }
        // sort key: (frame, bin, cell of the first tap inside the bin), or
        // (frame, bin) with the samples of a bin in acquisition order
        const int bin = lo * g.nbins + (b[2] * g.nb[1] + b[1]) * g.nb[0] + b[0];
        const int cell = (l[2] * g.T[1] + l[1]) * g.T[0] + l[0];
        keys[i] = cell_order ? bin * (g.T[0] * g.T[1] * g.T[2]) + cell : bin;
        vals[i] = (int32_t)i;
        atomicAdd(&counts[bin], 1);
    }
}

__global__ void gather_sorted_kernel(int64_t total, int ndim, const int32_t *__restrict__ sidx,
                                     const float *__restrict__ rk0, const float *__restrict__ rk1,
                                     const float *__restrict__ rk2, float *__restrict__ sc0,
                                     float *__restrict__ sc1, float *__restrict__ sc2)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < total;
         j += (int64_t)gridDim.x * blockDim.x) {
        const int32_t i = sidx[j];
        sc0[j] = rk0[i];
        if (ndim > 1) sc1[j] = rk1[i];
        if (ndim > 2) sc2[j] = rk2[i];
    }
}

// sort key of the tensor-core gridding bins: (frame, bin) with tile tg_T
__global__ void tg_key_kernel(Geom g, int t0, int t1, int t2, int n0, int n1, int n2, int nbins,
                              const int64_t *__restrict__ foff, const float *__restrict__ rk0,
                              const float *__restrict__ rk1, const float *__restrict__ rk2,
                              int32_t *__restrict__ keys, int32_t *__restrict__ counts)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < g.total;
         i += (int64_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = g.nframes;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (foff[mid] <= i) lo = mid; else hi = mid;
        }
        const int bx = pmod(first_tap(rk0[i], g.W[0]), g.G[0]) / t0;
        const int by = pmod(first_tap(rk1[i], g.W[1]), g.G[1]) / t1;
        const int bz = pmod(first_tap(rk2[i], g.W[2]), g.G[2]) / t2;
        const int key = lo * nbins + (bz * n1 + by) * n0 + bx;
        keys[i] = key;
        atomicAdd(&counts[key], 1);
    }
}

// Per sample of the tensor-core gridding order: the Kaiser-Bessel weights of
// its W taps on each axis (the same arithmetic as tap_weight in the kernels)
// and the offsets of its first taps inside its bin (tile t).
__global__ void tg_weights_kernel(Geom g, int t0, int t1, int t2, int wp, const float *__restrict__ sc0,
                                  const float *__restrict__ sc1, const float *__restrict__ sc2,
                                  float *__restrict__ w, int32_t *__restrict__ l)
{
    const int tt[3] = {t0, t1, t2};
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < g.total;
         j += (int64_t)gridDim.x * blockDim.x) {
        const float k[3] = {sc0[j], sc1[j], sc2[j]};
        int pack = 0;
        for (int a = 0; a < 3; a++) {
            const int x0 = first_tap(k[a], g.W[a]);
            pack |= (pmod(x0, g.G[a]) % tt[a]) << (8 * a);
            for (int i = 0; i < wp; i++)
                w[(j * 3 + a) * wp + i] = i < g.W[a] ? tap_weight(x0, i, k[a], g.W[a], g.inv_hw[a], g.beta[a]) : 0.0f;
        }
        l[j] = pack;
    }
}

// Work items of at most `chunk` samples per non-empty bin, and their visiting
// order in 4 x 4 x 4-bin tiles (frame, tile z, y, x, bin z, y, x), so that
// bins sharing halo points or spokes run close together.
static void make_items(const std::vector<int32_t> &start, int nbins, const int nb[3], int chunk,
                       std::vector<WorkItem> &items, std::vector<int32_t> &order)
{
    items.clear();
    const int64_t nkeys = (int64_t)start.size() - 1;
    for (int64_t b = 0; b < nkeys; b++)
        for (int s = start[b]; s < start[b + 1]; s += chunk)
            items.push_back({(int)b, s, std::min(s + chunk, start[b + 1])});
    order.resize(items.size());
    for (size_t i = 0; i < items.size(); i++) order[i] = (int32_t)i;
    auto tkey = [&](const WorkItem &w) {
        const int64_t f = w.bin / nbins, lb = w.bin % nbins;
        const int64_t bx = lb % nb[0], by = (lb / nb[0]) % nb[1], bz = lb / ((int64_t)nb[0] * nb[1]);
        const int64_t ntx = (nb[0] + 3) >> 2, nty = (nb[1] + 3) >> 2, ntz = (nb[2] + 3) >> 2;
        const int64_t tile = ((f * ntz + (bz >> 2)) * nty + (by >> 2)) * ntx + (bx >> 2);
        return tile * 64 + (((bz & 3) * 4 + (by & 3)) * 4 + (bx & 3));
    };
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t a, int32_t b) { return tkey(items[a]) < tkey(items[b]); });
}

static int grid_blocks(int64_t n, int threads)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int64_t b = ceil_div(n, threads);
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)sms * 16));
}

// Host float32 apodisation of one axis, following _apodize
// (src/deepmr/fft/nufft.py:423-447) operation by operation in float32.
static std::vector<float> apod_table(int n, int w, float os, float beta)
{
    std::vector<float> ap(n, 1.0f);
    if (w == 1) return ap;
    const float os_i = std::ceil(os * (float)n);
    const float piw = (float)(M_PI * (double)w);
    const float b2 = beta * beta;
    for (int i = 0; i < n; i++) {
        const float x = (piw * (float)(i - n / 2)) / os_i;
        ap[i] = std::sqrt(b2 - x * x);
    }
    for (int i = 0; i < n; i++) ap[i] = ap[i] / std::sinh(ap[i]);
    const float dc = ap[n / 2];
    for (int i = 0; i < n; i++) {
        const float v = ap[i] / dc;
        ap[i] = std::isnan(v) ? 1.0f : v;
    }
    return ap;
}

// Kernel-sum normalisation (src/deepmr/fft/_interp/plan.py:190-213):
// product over axes of the kernel sampled at ceil(-W/2) + i, summed.
static double kernel_scale(const Geom &g)
{
    double s = 1.0;
    for (int a = 0; a < g.ndim; a++) {
        if (g.W[a] == 1) continue;
        const double start = std::ceil(-g.W[a] / 2.0);
        double acc = 0.0;
        for (int i = 0; i < g.W[a]; i++) acc += kb_f64((start + i) / (g.W[a] / 2.0), (double)g.beta[a]);
        s *= acc;
    }
    return s;
}

static void default_tile(int ndim, int T[3])
{
    // bins = shared-memory tiles: a 32-coil tile + width-4 halo stays under
    // ~100 KB (3D: 7^3 points, 2D: 19^2 points per coil)
    if (ndim == 1) { T[0] = 256; T[1] = T[2] = 1; }
    else if (ndim == 2) { T[0] = 16; T[1] = 16; T[2] = 1; }
    else { T[0] = 4; T[1] = 4; T[2] = 4; }
}

template <typename T>
static int dev_alloc(T **p, size_t n)
{
    if (n == 0) n = 1;
    DMR_CUDA(cudaMalloc((void **)p, n * sizeof(T)));
    return DMR_OK;
}

}  // namespace dmr

using namespace dmr;

extern "C" int dmr_version(void) { return 100; }

extern "C" const char *dmr_last_error(void) { return t_err; }

extern "C" int64_t dmr_launch_count(void) { return g_launches.load(); }

extern "C" int dmr_detect_cartesian(const float *coord, int64_t npts, int ndim,
                                    const int32_t *shape_zyx, int32_t *is_cart_xyz, void *stream)
{
    DMR_CHECK(ndim >= 1 && ndim <= 3, DMR_ERR_INVALID, "ndim must be 1, 2 or 3 (got %d)", ndim);
    DMR_CHECK(npts >= 0 && (coord || npts == 0), DMR_ERR_INVALID, "bad coordinate buffer");
    cudaStream_t st = (cudaStream_t)stream;
    int *d_flags = nullptr;
    DMR_CUDA(cudaMallocAsync((void **)&d_flags, 3 * sizeof(int), st));
    const int ones[3] = {1, 1, 1};
    int h[3] = {1, 1, 1};
    int rc = DMR_OK;
    do {
        cudaError_t e = cudaMemcpyAsync(d_flags, ones, sizeof(ones), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) { rc = cuda_fail(e, "memcpy", __FILE__, __LINE__); break; }
        if (npts > 0) {
            // the reference pairs coordinate axis a with shape entry a (z, y, x order)
            float n[3] = {0, 0, 0};
            for (int a = 0; a < ndim; a++) n[a] = (float)shape_zyx[a];
            cartesian_kernel<<<grid_blocks(npts, 256), 256, 0, st>>>(coord, npts, ndim, n[0], n[1],
                                                                    n[2], d_flags);
            g_launches.fetch_add(1);
            e = cudaGetLastError();
            if (e != cudaSuccess) { rc = cuda_fail(e, "cartesian_kernel", __FILE__, __LINE__); break; }
        }
        e = cudaMemcpyAsync(h, d_flags, sizeof(h), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) { rc = cuda_fail(e, "readback", __FILE__, __LINE__); break; }
    } while (0);
    cudaFreeAsync(d_flags, st);
    if (rc == DMR_OK)
        for (int a = 0; a < ndim; a++) is_cart_xyz[a] = h[a];
    return rc;
}

extern "C" int dmr_plan_destroy(dmr_plan *p)
{
    if (!p) return DMR_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(p->device);
    cudaDeviceSynchronize();
    delete p;  // the destructor frees the device buffers
    cudaSetDevice(cur);
    return DMR_OK;
}

namespace {

struct TempBuffers {
    void *ptr[12] = {};
    ~TempBuffers()
    {
        for (void *p : ptr) cudaFree(p);
    }
};

}  // namespace

extern "C" int dmr_plan_create(int ndim, const int32_t *shape, const int32_t *os_shape,
                               const int32_t *width, const float *beta, const float *oversamp,
                               const float *coord, const int64_t *frame_offsets, int64_t nframes,
                               const int32_t *tile, void *stream, dmr_plan **out)
{
    DMR_CHECK(out, DMR_ERR_INVALID, "out is NULL");
    *out = nullptr;
    DMR_CHECK(ndim >= 1 && ndim <= 3, DMR_ERR_INVALID, "ndim must be 1, 2 or 3 (got %d)", ndim);
    DMR_CHECK(shape && os_shape && width && beta && oversamp && frame_offsets, DMR_ERR_INVALID,
              "NULL parameter array");
    DMR_CHECK(nframes >= 1 && nframes < (1 << 20), DMR_ERR_INVALID, "bad nframes %lld",
              (long long)nframes);
    const int64_t total = frame_offsets[nframes];
    DMR_CHECK(frame_offsets[0] == 0 && total >= 0 && total < INT32_MAX, DMR_ERR_INVALID,
              "frame offsets must start at 0 and total samples must fit in int32");
    for (int64_t f = 0; f < nframes; f++)
        DMR_CHECK(frame_offsets[f + 1] >= frame_offsets[f], DMR_ERR_INVALID,
                  "frame offsets must be non-decreasing");
    DMR_CHECK(coord || total == 0, DMR_ERR_INVALID, "coord is NULL");

    cudaStream_t st = (cudaStream_t)stream;
    std::unique_ptr<dmr_plan> p(new dmr_plan());
    DMR_CUDA(cudaGetDevice(&p->device));
    Geom &g = p->g;
    memset(&g, 0, sizeof(g));
    g.ndim = ndim;
    g.nframes = (int)nframes;
    g.total = total;
    int T[3];
    default_tile(ndim, T);
    for (int a = 0; a < 3; a++) {
        g.G[a] = g.N[a] = g.W[a] = g.T[a] = g.nb[a] = 1;
        g.half[a] = 0;
        g.beta[a] = 0.0f;
        g.inv_hw[a] = 1.0;
        p->os[a] = 1.0f;
    }
    for (int i = 0; i < ndim; i++) {
        const int a = ndim - 1 - i;  // (z, y, x) input -> x = 0
        g.N[a] = shape[i];
        g.G[a] = os_shape[i];
        g.W[a] = width[i];
        g.beta[a] = beta[i];
        p->os[a] = oversamp[i];
        DMR_CHECK(g.N[a] >= 1 && g.G[a] >= 1 && g.W[a] >= 1 && g.W[a] <= 16, DMR_ERR_INVALID,
                  "bad axis %d: shape %d os_shape %d width %d (widths up to 16)", i, g.N[a],
                  g.G[a], g.W[a]);
        DMR_CHECK(g.W[a] == 1 || g.G[a] >= g.W[a], DMR_ERR_UNSUPPORTED,
                  "oversampled grid %d smaller than kernel width %d on axis %d", g.G[a], g.W[a], i);
        g.half[a] = g.G[a] / 2;
        g.inv_hw[a] = 1.0 / (g.W[a] / 2.0);
        const int t = tile ? tile[i] : T[a];
        DMR_CHECK(t >= 1, DMR_ERR_INVALID, "bad tile");
        g.T[a] = std::min(t, g.G[a]);
        g.nb[a] = (int)ceil_div(g.G[a], g.T[a]);
    }
    g.nbins = g.nb[0] * g.nb[1] * g.nb[2];
    g.gsize = (int64_t)g.G[0] * g.G[1] * g.G[2];
    g.isize = (int64_t)g.N[0] * g.N[1] * g.N[2];
    DMR_CHECK((int64_t)g.nbins * nframes * g.T[0] * g.T[1] * g.T[2] < INT32_MAX, DMR_ERR_UNSUPPORTED,
              "too many bins x cells for 32-bit sort keys");
    p->scale = kernel_scale(g);
    p->frame_offsets.assign(frame_offsets, frame_offsets + nframes + 1);

    // apodisation tables (image index), per axis
    for (int a = 0; a < 3; a++) {
        std::vector<float> ap = apod_table(g.N[a], a < ndim ? g.W[a] : 1, p->os[a], g.beta[a]);
        DMR_TRY(dev_alloc(&p->apod[a], ap.size()));
        DMR_CUDA(cudaMemcpyAsync(p->apod[a], ap.data(), ap.size() * sizeof(float),
                                 cudaMemcpyHostToDevice, st));
        DMR_CUDA(cudaStreamSynchronize(st));
    }

    // rescale constants (nufft.py:415-418), float32 like numpy
    float sc[3] = {1, 1, 1}, sh[3] = {0, 0, 0};
    for (int a = 0; a < ndim; a++) {
        const float gos = std::ceil(p->os[a] * (float)g.N[a]);
        sc[a] = gos / (float)g.N[a];
        sh[a] = std::floor(gos / 2.0f);
    }

    const int64_t nkeys = (int64_t)nframes * g.nbins;
    TempBuffers tmp;
    int32_t *keys = nullptr, *keys_s = nullptr, *vals = nullptr, *counts = nullptr;
    int64_t *d_foff = nullptr;
    int *d_err = nullptr;
    float *rk[3] = {nullptr, nullptr, nullptr};
    DMR_TRY(dev_alloc(&keys, total));
    tmp.ptr[0] = keys;
    DMR_TRY(dev_alloc(&keys_s, total));
    tmp.ptr[1] = keys_s;
    DMR_TRY(dev_alloc(&vals, total));
    tmp.ptr[2] = vals;
    DMR_TRY(dev_alloc(&counts, nkeys));
    tmp.ptr[3] = counts;
    DMR_TRY(dev_alloc(&d_foff, nframes + 1));
    p->foff_dev = d_foff;  // kept by the plan
    DMR_TRY(dev_alloc(&d_err, 1));
    tmp.ptr[5] = d_err;
    for (int a = 0; a < ndim; a++) {
        DMR_TRY(dev_alloc(&rk[a], total));
        tmp.ptr[6 + a] = rk[a];
        DMR_TRY(dev_alloc(&p->scoord[a], total));
    }
    DMR_TRY(dev_alloc(&p->sidx, total));
    DMR_TRY(dev_alloc(&p->status, 1));
    DMR_CUDA(cudaMemsetAsync(p->status, 0, sizeof(int32_t), st));
    DMR_CUDA(cudaMemsetAsync(counts, 0, nkeys * sizeof(int32_t), st));
    DMR_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    DMR_CUDA(cudaMemcpyAsync(d_foff, frame_offsets, (nframes + 1) * sizeof(int64_t),
                             cudaMemcpyHostToDevice, st));

    // Within a bin, samples are sorted by the cell of their first tap (register
    // reuse of the cube kernels); DMR_SORT_CELL=0 keeps them in acquisition
    // order instead (tuning).
    const char *env_order = getenv("DMR_SORT_CELL");
    const int cell_order = env_order ? atoi(env_order) != 0 : 1;
    if (total > 0) {
        preprocess_kernel<<<grid_blocks(total, 256), 256, 0, st>>>(
            g, coord, d_foff, sc[0], sc[1], sc[2], sh[0], sh[1], sh[2], rk[0], rk[1], rk[2],
            keys, vals, counts, d_err, cell_order);
        DMR_LAUNCHED("preprocess_kernel");
        const int64_t nsort = nkeys * (cell_order ? (int64_t)g.T[0] * g.T[1] * g.T[2] : 1);
        int end_bit = 1;
        while ((1ll << end_bit) < nsort) end_bit++;
        size_t temp_bytes = 0;
        DMR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys, keys_s, vals, p->sidx,
                                                 (int)total, 0, end_bit, st));
        void *temp = nullptr;
        DMR_CUDA(cudaMalloc(&temp, std::max<size_t>(temp_bytes, 1)));
        tmp.ptr[9] = temp;
        DMR_CUDA(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys, keys_s, vals, p->sidx,
                                                 (int)total, 0, end_bit, st));
        g_launches.fetch_add(1);
        gather_sorted_kernel<<<grid_blocks(total, 256), 256, 0, st>>>(
            total, ndim, p->sidx, rk[0], rk[1], rk[2], p->scoord[0], p->scoord[1], p->scoord[2]);
        DMR_LAUNCHED("gather_sorted_kernel");
    }
    std::vector<int32_t> h_counts(nkeys);
    int h_err = 0;
    DMR_CUDA(cudaMemcpyAsync(h_counts.data(), counts, nkeys * sizeof(int32_t),
                             cudaMemcpyDeviceToHost, st));
    DMR_CUDA(cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    DMR_CUDA(cudaStreamSynchronize(st));
    DMR_CHECK(h_err == 0, DMR_ERR_COORD, "non-finite (or |k| >= 1e8) k-space coordinate");

    // bin offsets
    std::vector<int32_t> h_start(nkeys + 1, 0);
    for (int64_t i = 0; i < nkeys; i++) h_start[i + 1] = h_start[i] + h_counts[i];

    // bins of the 3D tensor-core gridding: region (T + W - 1) of 7 x 6 x 6
    // points (x, y, z), i.e. T = (8 - W, 7 - W, 7 - W), for widths 2..5
    if (ndim == 3 && total > 0 && g.W[0] == g.W[1] && g.W[1] == g.W[2] && g.W[0] >= 2 && g.W[0] <= 5) {
        const int W = g.W[0];
        int tT[3] = {8 - W, 7 - W, 7 - W}, tnb[3];
        for (int a = 0; a < 3; a++) {
            tT[a] = std::min(tT[a], g.G[a]);
            tnb[a] = (int)ceil_div(g.G[a], tT[a]);
        }
        const int tbins = tnb[0] * tnb[1] * tnb[2];
        const int64_t tkeys = (int64_t)nframes * tbins;
        if (tkeys < INT32_MAX) {
            int32_t *tcounts = nullptr;
            DMR_TRY(dev_alloc(&tcounts, tkeys));
            tmp.ptr[10] = tcounts;
            DMR_CUDA(cudaMemsetAsync(tcounts, 0, tkeys * sizeof(int32_t), st));
            tg_key_kernel<<<grid_blocks(total, 256), 256, 0, st>>>(g, tT[0], tT[1], tT[2], tnb[0], tnb[1], tnb[2],
                                                                   tbins, d_foff, rk[0], rk[1], rk[2], keys, tcounts);
            DMR_LAUNCHED("tg_key_kernel");
            int tbit = 1;
            while ((1ll << tbit) < tkeys) tbit++;
            for (int a = 0; a < 3; a++) DMR_TRY(dev_alloc(&p->tg_scoord[a], total));
            DMR_TRY(dev_alloc(&p->tg_sidx, total));
            size_t tb = 0;
            DMR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys, keys_s, vals, p->tg_sidx, (int)total, 0,
                                                     tbit, st));
            void *ttemp = nullptr;
            DMR_CUDA(cudaMalloc(&ttemp, std::max<size_t>(tb, 1)));
            tmp.ptr[11] = ttemp;
            DMR_CUDA(cub::DeviceRadixSort::SortPairs(ttemp, tb, keys, keys_s, vals, p->tg_sidx, (int)total, 0,
                                                     tbit, st));
            g_launches.fetch_add(1);
            gather_sorted_kernel<<<grid_blocks(total, 256), 256, 0, st>>>(
                total, ndim, p->tg_sidx, rk[0], rk[1], rk[2], p->tg_scoord[0], p->tg_scoord[1], p->tg_scoord[2]);
            DMR_LAUNCHED("gather_sorted_kernel");
            p->tg_wp = W <= 4 ? 4 : 8;
            DMR_TRY(dev_alloc(&p->tg_w, (size_t)total * 3 * p->tg_wp));
            DMR_TRY(dev_alloc(&p->tg_l, total));
            tg_weights_kernel<<<grid_blocks(total, 256), 256, 0, st>>>(g, tT[0], tT[1], tT[2], p->tg_wp,
                                                                       p->tg_scoord[0], p->tg_scoord[1],
                                                                       p->tg_scoord[2], p->tg_w, p->tg_l);
            DMR_LAUNCHED("tg_weights_kernel");
            std::vector<int32_t> hc(tkeys);
            DMR_CUDA(cudaMemcpyAsync(hc.data(), tcounts, tkeys * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            DMR_CUDA(cudaStreamSynchronize(st));
            std::vector<int32_t> ts(tkeys + 1, 0);
            for (int64_t i = 0; i < tkeys; i++) ts[i + 1] = ts[i] + hc[i];
            std::vector<WorkItem> titems;
            std::vector<int32_t> torder;
            make_items(ts, tbins, tnb, kTgSegment, titems, torder);
            DMR_TRY(dev_alloc(&p->tg_work, titems.size()));
            DMR_TRY(dev_alloc(&p->tg_order, torder.size()));
            if (!titems.empty()) {
                DMR_CUDA(cudaMemcpyAsync(p->tg_work, titems.data(), titems.size() * sizeof(WorkItem),
                                         cudaMemcpyHostToDevice, st));
                DMR_CUDA(cudaMemcpyAsync(p->tg_order, torder.data(), torder.size() * sizeof(int32_t),
                                         cudaMemcpyHostToDevice, st));
            }
            // deterministic mode: the items of each bin (make_items numbers
            // them in key order, kTgSegment samples each)
            std::vector<int32_t> istart(tkeys + 1, 0);
            for (int64_t k = 0; k < tkeys; k++)
                istart[k + 1] = istart[k] + (int32_t)ceil_div(ts[k + 1] - ts[k], kTgSegment);
            DMR_CHECK(istart[tkeys] == (int64_t)titems.size(), DMR_ERR_UNSUPPORTED, "gridding item count mismatch");
            DMR_TRY(dev_alloc(&p->tg_item_start, istart.size()));
            DMR_CUDA(cudaMemcpyAsync(p->tg_item_start, istart.data(), istart.size() * sizeof(int32_t),
                                     cudaMemcpyHostToDevice, st));
            DMR_CUDA(cudaStreamSynchronize(st));
            p->tg_nwork = (int)titems.size();
            p->tg_nbins = tbins;
            for (int a = 0; a < 3; a++) {
                p->tg_T[a] = tT[a];
                p->tg_nb[a] = tnb[a];
            }
        }
    }

    // interpolation / atomic-gridding items: non-empty bins in chunks of at most
    // kChunk samples (bounded work per block), in spatial order so that blocks
    // running together share tile halos in L2
    const int kChunk = 2048;
    std::vector<WorkItem> items;
    for (int64_t b = 0; b < nkeys; b++) {
        for (int s = h_start[b]; s < h_start[b + 1]; s += kChunk)
            items.push_back({(int)b, s, std::min(s + kChunk, h_start[b + 1])});
    }

    // owner-gridding tiles: every tile of every frame, ordered by the samples
    // of the bins that can reach it (the bin itself and its lower neighbours)
    std::vector<std::pair<int64_t, int32_t>> tc;
    tc.reserve(nkeys);
    for (int64_t key = 0; key < nkeys; key++) {
        const int f = (int)(key / g.nbins);
        const int lb = (int)(key % g.nbins);
        const int bx = lb % g.nb[0], by = (lb / g.nb[0]) % g.nb[1], bz = lb / (g.nb[0] * g.nb[1]);
        const int bb[3] = {bx, by, bz};
        int lo[3], cnt[3];
        for (int a = 0; a < 3; a++) {
            const int first = pmod(bb[a] * g.T[a] - g.W[a] + 1, g.G[a]) / g.T[a];
            lo[a] = first;
            cnt[a] = pmod(bb[a] - first, g.nb[a]) + 1;
        }
        int64_t cost = 0;
        for (int iz = 0; iz < cnt[2]; iz++)
            for (int iy = 0; iy < cnt[1]; iy++)
                for (int ix = 0; ix < cnt[0]; ix++) {
                    const int sb = (((lo[2] + iz) % g.nb[2]) * g.nb[1] + (lo[1] + iy) % g.nb[1]) *
                                       g.nb[0] + (lo[0] + ix) % g.nb[0];
                    cost += h_counts[(int64_t)f * g.nbins + sb];
                }
        tc.push_back({cost, (int32_t)key});
    }
    std::stable_sort(tc.begin(), tc.end(),
                     [](const std::pair<int64_t, int32_t> &x, const std::pair<int64_t, int32_t> &y) {
                         return x.first > y.first;
                     });
    std::vector<int32_t> order(tc.size());
    for (size_t i = 0; i < tc.size(); i++) order[i] = tc[i].second;

    // deterministic gridding: colour bins so that same-colour tile + halo
    // regions [b*T, b*T + T + Wmax - 1) (mod G) are disjoint on some axis;
    // along each axis colour = b mod C with the smallest conflict-free C
    int wmax = 1;
    for (int a = 0; a < ndim; a++) wmax = std::max(wmax, g.W[a]);
    int C[3] = {1, 1, 1};
    for (int a = 0; a < 3; a++) {
        const int nb = g.nb[a];
        const int ext = g.T[a] + (a < ndim ? wmax : 1) - 1;
        for (C[a] = std::max(1, (int)ceil_div(ext, g.T[a])); C[a] < nb; C[a]++) {
            bool ok = true;
            for (int b1 = 0; b1 < nb && ok; b1++)
                for (int b2 = b1 + 1; b2 < nb && ok; b2++) {
                    if (b1 % C[a] != b2 % C[a]) continue;
                    // regions as sets of grid indices mod G
                    for (int i = 0; i < ext && ok; i++) {
                        const int x = (b1 * g.T[a] + i) % g.G[a];
                        const int d = pmod(x - b2 * g.T[a], g.G[a]);
                        if (d < ext) ok = false;
                    }
                }
            if (ok) break;
        }
        C[a] = std::min(C[a], nb);
    }
    const int ncolors = C[0] * C[1] * C[2];
    std::vector<std::vector<WorkItem>> by_color(ncolors);
    for (int64_t key = 0; key < nkeys; key++) {
        if (h_start[key + 1] == h_start[key]) continue;
        const int lb = (int)(key % g.nbins);
        const int bx = lb % g.nb[0], by = (lb / g.nb[0]) % g.nb[1], bz = lb / (g.nb[0] * g.nb[1]);
        const int col = (bz % C[2] * C[1] + by % C[1]) * C[0] + bx % C[0];
        by_color[col].push_back({(int)key, h_start[key], h_start[key + 1]});
    }
    std::vector<WorkItem> det;
    p->det_color_start.assign(1, 0);
    for (int c = 0; c < ncolors; c++) {
        // heaviest bins first inside a pass (shorter tail)
        std::stable_sort(by_color[c].begin(), by_color[c].end(), [](const WorkItem &x, const WorkItem &y) {
            return (x.end - x.begin) > (y.end - y.begin);
        });
        det.insert(det.end(), by_color[c].begin(), by_color[c].end());
        p->det_color_start.push_back((int)det.size());
    }
    DMR_TRY(dev_alloc(&p->det_work, det.size()));
    if (!det.empty())
        DMR_CUDA(cudaMemcpyAsync(p->det_work, det.data(), det.size() * sizeof(WorkItem),
                                 cudaMemcpyHostToDevice, st));

    // the same items visited in 4x4x4-bin tiles (frame, tile z, y, x, bin z, y, x):
    // bins that share halo points or spokes run close together, so their grid
    // lines and k-space sectors are still in L2 (DMR_NO_TILED_ORDER=1: key order)
    std::vector<int32_t> worder(items.size());
    for (size_t i = 0; i < items.size(); i++) worder[i] = (int32_t)i;
    static const bool tiled_order = [] {
        const char *e = getenv("DMR_NO_TILED_ORDER");
        return !(e && atoi(e));
    }();
    if (tiled_order) {
        auto tkey = [&](const WorkItem &w) {
            const int64_t f = w.bin / g.nbins, lb = w.bin % g.nbins;
            const int64_t bx = lb % g.nb[0], by = (lb / g.nb[0]) % g.nb[1], bz = lb / ((int64_t)g.nb[0] * g.nb[1]);
            const int64_t tx = bx >> 2, ty = by >> 2, tz = bz >> 2;
            const int64_t ntx = (g.nb[0] + 3) >> 2, nty = (g.nb[1] + 3) >> 2, ntz = (g.nb[2] + 3) >> 2;
            const int64_t tile = ((f * ntz + tz) * nty + ty) * ntx + tx;
            return tile * 64 + (((bz & 3) * 4 + (by & 3)) * 4 + (bx & 3));
        };
        std::stable_sort(worder.begin(), worder.end(),
                         [&](int32_t a, int32_t b) { return tkey(items[a]) < tkey(items[b]); });
    }
    p->nwork = (int)items.size();
    p->ntiles = (int)order.size();
    DMR_TRY(dev_alloc(&p->bin_start, nkeys + 1));
    DMR_TRY(dev_alloc(&p->work, items.size()));
    DMR_TRY(dev_alloc(&p->tiles, order.size()));
    DMR_CUDA(cudaMemcpyAsync(p->bin_start, h_start.data(), (nkeys + 1) * sizeof(int32_t),
                             cudaMemcpyHostToDevice, st));
    DMR_TRY(dev_alloc(&p->work_order, items.size()));
    if (!items.empty()) {
        DMR_CUDA(cudaMemcpyAsync(p->work, items.data(), items.size() * sizeof(WorkItem),
                                 cudaMemcpyHostToDevice, st));
        DMR_CUDA(cudaMemcpyAsync(p->work_order, worder.data(), worder.size() * sizeof(int32_t),
                                 cudaMemcpyHostToDevice, st));
    }
    DMR_CUDA(cudaMemcpyAsync(p->tiles, order.data(), order.size() * sizeof(int32_t),
                             cudaMemcpyHostToDevice, st));
    DMR_CUDA(cudaStreamSynchronize(st));
    DMR_TRY(rt_build(p.get(), h_start, st));
    *out = p.release();
    return DMR_OK;
}

extern "C" int dmr_plan_scale(const dmr_plan *p, double *scale)
{
    DMR_CHECK(p && scale, DMR_ERR_INVALID, "NULL argument");
    *scale = p->scale;
    return DMR_OK;
}

extern "C" int dmr_plan_info(const dmr_plan *p, int64_t *total, int64_t *nframes, int32_t *tile_zyx)
{
    DMR_CHECK(p, DMR_ERR_INVALID, "NULL plan");
    if (total) *total = p->g.total;
    if (nframes) *nframes = p->g.nframes;
    if (tile_zyx)
        for (int i = 0; i < p->g.ndim; i++) tile_zyx[i] = p->g.T[p->g.ndim - 1 - i];
    return DMR_OK;
}
