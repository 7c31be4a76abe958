// Interpolation (oversampled grid -> samples) and gridding (samples -> grid)
// with Kaiser-Bessel weights evaluated on the fly.
//
// Reference: apply_interpolation / apply_gridding and their Numba kernels
// (src/deepmr/fft/_interp/interp.py:14-227, 415-749;
//  src/deepmr/fft/_interp/grid.py:14-284, 424-1168). The reference launches
// one thread per (frame, batch, sample) over precomputed (F, M, W) tables and
// grids with two global float atomics per complex tap. Here samples are
// sorted by spatial bin (the plan), one thread block stages the bin's grid
// tile (plus the kernel halo) in shared memory for a chunk of coils, and a
// warp processes 32/CC samples x CC coils at a time, so each sample's weights
// are computed once per coil chunk and the grid is read coalesced.
//
// Grid layout everywhere: (batch, nframes, *G) complex64 in FFT order — the
// centred index c of an axis is stored at (c - G//2) mod G — so the fftshift
// of the reference's centred FFT (src/deepmr/fft/fft.py:77-80) costs nothing.
#include <algorithm>
#include <cstdlib>

#include "kb.cuh"
#include "plan.cuh"

namespace dmr {

template <int NDIM, int WMAX>
struct Meta {
    // samples staged per batch (sized so the weight table stays ~12 KB)
    static constexpr int SB = (NDIM * WMAX <= 16) ? 256 : (NDIM * WMAX <= 32 ? 128 : 64);
    static constexpr int NW = NDIM * WMAX;
    static size_t bytes() { return (size_t)SB * (NW * sizeof(float) + 2 * sizeof(int)); }
};

__device__ __forceinline__ void tile_origin(const Geom &g, int lb, int org[3])
{
    org[0] = (lb % g.nb[0]) * g.T[0];
    org[1] = ((lb / g.nb[0]) % g.nb[1]) * g.T[1];
    org[2] = (lb / (g.nb[0] * g.nb[1])) * g.T[2];
}

// Stage per-sample data of samples [base, base+n) of a bin whose tile starts
// at org: weights (NDIM x WMAX), linear offset of the first tap inside the
// (T + W - 1)^NDIM region, and the global sample index.
template <int NDIM, int WMAX>
__device__ __forceinline__ void stage_samples(const Geom &g, const int org[3], int base, int n,
                                              const float *__restrict__ sc0,
                                              const float *__restrict__ sc1,
                                              const float *__restrict__ sc2,
                                              const int32_t *__restrict__ sidx, int R0, int R1,
                                              float *wts, int *off, int *gi)
{
    constexpr int NW = NDIM * WMAX;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const int j = base + t;
        const float k[3] = {sc0[j], NDIM > 1 ? sc1[j] : 0.0f, NDIM > 2 ? sc2[j] : 0.0f};
        int l[3] = {0, 0, 0};
#pragma unroll
        for (int a = 0; a < NDIM; a++) {
            const int x0 = first_tap_dev(k[a], g.W[a]);
            l[a] = pmod(x0, g.G[a]) - org[a];
#pragma unroll
            for (int i = 0; i < WMAX; i++)
                if (i < g.W[a]) wts[t * NW + a * WMAX + i] = tap_weight(x0, i, k[a], g.W[a], g.inv_hw[a], g.beta[a]);
        }
        off[t] = (l[2] * R1 + l[1]) * R0 + l[0];
        gi[t] = sidx[j];
    }
}

// Sum over the taps of one sample: sum_z w_z sum_y w_y sum_x w_x tile[z][y][x].
// Weights come from the staged table `w` (NDIM x WMAX); the x loop is fully
// unrolled with x weights in registers, outer loops are unrolled for WMAX <= 4.
template <int NDIM, int WMAX>
__device__ __forceinline__ float2 gather_taps(const float2 *tp, const float *w, int Wx, int Wy, int Wz,
                                              int R0, int R1)
{
    constexpr int UO = WMAX <= 4 ? WMAX : 1;
    float wx[WMAX];
#pragma unroll
    for (int i = 0; i < WMAX; i++) wx[i] = i < Wx ? w[i] : 0.0f;
    float ar = 0.0f, ai = 0.0f;
    auto row_sum = [&](const float2 *row, float &rr, float &ri) {
#pragma unroll
        for (int ix = 0; ix < WMAX; ix++)
            if (ix < Wx) {
                const float2 v = row[ix];
                rr += wx[ix] * v.x;
                ri += wx[ix] * v.y;
            }
    };
    if (NDIM == 1) {
        row_sum(tp, ar, ai);
    } else if (NDIM == 2) {
#pragma unroll UO
        for (int iy = 0; iy < WMAX; iy++) {
            if (iy >= Wy) break;
            float rr = 0.0f, ri = 0.0f;
            row_sum(tp + iy * R0, rr, ri);
            const float wy = w[WMAX + iy];
            ar += wy * rr;
            ai += wy * ri;
        }
    } else {
#pragma unroll UO
        for (int iz = 0; iz < WMAX; iz++) {
            if (iz >= Wz) break;
            const float wz = w[2 * WMAX + iz];
#pragma unroll UO
            for (int iy = 0; iy < WMAX; iy++) {
                if (iy >= Wy) break;
                float rr = 0.0f, ri = 0.0f;
                row_sum(tp + (iz * R1 + iy) * R0, rr, ri);
                const float wzy = wz * w[WMAX + iy];
                ar += wzy * rr;
                ai += wzy * ri;
            }
        }
    }
    return make_float2(ar, ai);
}

// Spread one sample value v over its taps with shared-memory atomics; the tap
// weight is formed like the reference ((w_z * w_y) * w_x, grid.py:262-280).
template <int NDIM, int WMAX>
__device__ __forceinline__ void scatter_taps(float2 *tp, const float *w, float2 v, int Wx, int Wy, int Wz,
                                             int R0, int R1)
{
    constexpr int UO = WMAX <= 4 ? WMAX : 1;
    float wx[WMAX];
#pragma unroll
    for (int i = 0; i < WMAX; i++) wx[i] = i < Wx ? w[i] : 0.0f;
    auto row_add = [&](float2 *row, float wo) {
#pragma unroll
        for (int ix = 0; ix < WMAX; ix++)
            if (ix < Wx) {
                const float wv = NDIM == 1 ? wx[ix] : wo * wx[ix];
                atomicAdd(&row[ix].x, wv * v.x);
                atomicAdd(&row[ix].y, wv * v.y);
            }
    };
    if (NDIM == 1) {
        row_add(tp, 1.0f);
    } else if (NDIM == 2) {
#pragma unroll UO
        for (int iy = 0; iy < WMAX; iy++) {
            if (iy >= Wy) break;
            row_add(tp + iy * R0, w[WMAX + iy]);
        }
    } else {
#pragma unroll UO
        for (int iz = 0; iz < WMAX; iz++) {
            if (iz >= Wz) break;
            const float wz = w[2 * WMAX + iz];
#pragma unroll UO
            for (int iy = 0; iy < WMAX; iy++) {
                if (iy >= Wy) break;
                row_add(tp + (iz * R1 + iy) * R0, wz * w[WMAX + iy]);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Interpolation: grid -> samples, y = (sum_taps w * grid) / scale * weight.
// Block = 256 threads; blockIdx.x = work item (bin chunk), blockIdx.y = coil chunk.
// ---------------------------------------------------------------------------
template <int NDIM, int WMAX>
__global__ void __launch_bounds__(256) interp_kernel(
    Geom g, const WorkItem *__restrict__ work, const float *__restrict__ sc0,
    const float *__restrict__ sc1, const float *__restrict__ sc2, const int32_t *__restrict__ sidx,
    const float2 *__restrict__ grid, float2 *__restrict__ ksp, int64_t batch,
    const float *__restrict__ weight, int wpb, float scale, int cc_log2)
{
    extern __shared__ __align__(16) unsigned char smem[];
    using M = Meta<NDIM, WMAX>;
    const int CC = 1 << cc_log2;
    const WorkItem it = work[blockIdx.x];
    const int f = it.bin / g.nbins;
    int org[3];
    tile_origin(g, it.bin - f * g.nbins, org);
    const int R0 = g.T[0] + g.W[0] - 1;
    const int R1 = NDIM > 1 ? g.T[1] + g.W[1] - 1 : 1;
    const int R2 = NDIM > 2 ? g.T[2] + g.W[2] - 1 : 1;
    const int P = R0 * R1 * R2;
    const int PP = P | 1;
    float2 *tile = reinterpret_cast<float2 *>(smem);
    float *wts = reinterpret_cast<float *>(tile + (size_t)CC * PP);
    int *off = reinterpret_cast<int *>(wts + M::SB * M::NW);
    int *gi = off + M::SB;

    const int64_t b0 = (int64_t)blockIdx.y * CC;
    // stage the tile + halo of CC coils (coalesced along x; FFT-order wrap)
    for (int idx = threadIdx.x; idx < CC * P; idx += blockDim.x) {
        const int c = idx / P;
        const int r = idx - c * P;
        const int rx = r % R0;
        const int t = r / R0;
        const int ry = t % R1;
        const int rz = t / R1;
        const int64_t b = b0 + c;
        float2 v = make_float2(0.0f, 0.0f);
        if (b < batch) {
            const int px = (org[0] + rx + g.G[0] - g.half[0]) % g.G[0];
            const int py = (org[1] + ry + g.G[1] - g.half[1]) % g.G[1];
            const int pz = (org[2] + rz + g.G[2] - g.half[2]) % g.G[2];
            v = grid[(b * g.nframes + f) * g.gsize + ((int64_t)pz * g.G[1] + py) * g.G[0] + px];
        }
        tile[c * PP + r] = v;
    }

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    const int spw = 32 >> cc_log2;
    const int s = lane >> cc_log2;
    const int c = lane & (CC - 1);
    const int64_t b = b0 + c;
    const int Wx = g.W[0], Wy = g.W[1], Wz = g.W[2];
    
    for (int base = it.begin; base < it.end; base += M::SB) {
        const int n = min(M::SB, it.end - base);
        __syncthreads();  // tile staged / previous batch consumed
        stage_samples<NDIM, WMAX>(g, org, base, n, sc0, sc1, sc2, sidx, R0, R1, wts, off, gi);
        __syncthreads();
        for (int q = warp * spw + s; q < n; q += nwarps * spw) {
            const float2 acc = gather_taps<NDIM, WMAX>(tile + c * PP + off[q], wts + q * M::NW, Wx, Wy, Wz, R0, R1);
            const float ar = acc.x, ai = acc.y;
            if (b < batch) {
                const int64_t o = b * g.total + gi[q];
                float2 y = make_float2(ar / scale, ai / scale);
                if (weight) {
                    const float wv = weight[wpb ? o : (int64_t)gi[q]];
                    y.x *= wv;
                    y.y *= wv;
                }
                ksp[o] = y;
            }
        }
    }
}

__device__ __forceinline__ float2 load_sample(const void *ksp, int kreal, int64_t o)
{
    if (kreal) return make_float2(reinterpret_cast<const float *>(ksp)[o], 0.0f);
    return reinterpret_cast<const float2 *>(ksp)[o];
}

// ---------------------------------------------------------------------------
// Gridding, atomic mode: each block accumulates its bin's samples into a
// shared-memory tile + halo (shared atomics; lanes of a warp hold distinct
// coils) and flushes it to the grid with global atomics. The grid must be
// zeroed first. Summation order across blocks is not fixed.
// ---------------------------------------------------------------------------
template <int NDIM, int WMAX>
__global__ void __launch_bounds__(256) grid_atomic_kernel(
    Geom g, const WorkItem *__restrict__ work, const float *__restrict__ sc0,
    const float *__restrict__ sc1, const float *__restrict__ sc2, const int32_t *__restrict__ sidx,
    const void *__restrict__ ksp, int kreal, float2 *__restrict__ grid, int64_t batch,
    const float *__restrict__ weight, int wpb, float scale, int cc_log2)
{
    extern __shared__ __align__(16) unsigned char smem[];
    using M = Meta<NDIM, WMAX>;
    const int CC = 1 << cc_log2;
    const WorkItem it = work[blockIdx.x];
    const int f = it.bin / g.nbins;
    int org[3];
    tile_origin(g, it.bin - f * g.nbins, org);
    const int R0 = g.T[0] + g.W[0] - 1;
    const int R1 = NDIM > 1 ? g.T[1] + g.W[1] - 1 : 1;
    const int R2 = NDIM > 2 ? g.T[2] + g.W[2] - 1 : 1;
    const int P = R0 * R1 * R2;
    const int PP = P | 1;
    float2 *tile = reinterpret_cast<float2 *>(smem);
    float *wts = reinterpret_cast<float *>(tile + (size_t)CC * PP);
    int *off = reinterpret_cast<int *>(wts + M::SB * M::NW);
    int *gi = off + M::SB;

    for (int idx = threadIdx.x; idx < CC * PP; idx += blockDim.x) tile[idx] = make_float2(0.0f, 0.0f);

    const int64_t b0 = (int64_t)blockIdx.y * CC;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    const int spw = 32 >> cc_log2;
    const int s = lane >> cc_log2;
    const int c = lane & (CC - 1);
    const int64_t b = b0 + c;
    const int Wx = g.W[0], Wy = g.W[1], Wz = g.W[2];

    for (int base = it.begin; base < it.end; base += M::SB) {
        const int n = min(M::SB, it.end - base);
        __syncthreads();
        stage_samples<NDIM, WMAX>(g, org, base, n, sc0, sc1, sc2, sidx, R0, R1, wts, off, gi);
        __syncthreads();
        for (int q = warp * spw + s; q < n; q += nwarps * spw) {
            if (b >= batch) continue;
            const int64_t o = b * g.total + gi[q];
            float2 v = load_sample(ksp, kreal, o);
            if (weight) {
                const float wv = weight[wpb ? o : (int64_t)gi[q]];
                v.x *= wv;
                v.y *= wv;
            }
            scatter_taps<NDIM, WMAX>(tile + c * PP + off[q], wts + q * M::NW, v, Wx, Wy, Wz, R0, R1);
        }
    }
    __syncthreads();
    // flush tile + halo with global atomics (FFT-order wrap)
    for (int idx = threadIdx.x; idx < CC * P; idx += blockDim.x) {
        const int cc = idx / P;
        const int r = idx - cc * P;
        const int64_t bb = b0 + cc;
        if (bb >= batch) continue;
        const float2 v = tile[cc * PP + r];
        if (v.x == 0.0f && v.y == 0.0f) continue;
        const int rx = r % R0;
        const int t = r / R0;
        const int ry = t % R1;
        const int rz = t / R1;
        const int px = (org[0] + rx + g.G[0] - g.half[0]) % g.G[0];
        const int py = (org[1] + ry + g.G[1] - g.half[1]) % g.G[1];
        const int pz = (org[2] + rz + g.G[2] - g.half[2]) % g.G[2];
        float2 *dst = grid + (bb * g.nframes + f) * g.gsize + ((int64_t)pz * g.G[1] + py) * g.G[0] + px;
        atomicAdd(&dst->x, v.x / scale);
        atomicAdd(&dst->y, v.y / scale);
    }
}

// ---------------------------------------------------------------------------
// Cell-cube kernels. Samples are sorted by (bin, cell of their first tap), and
// in the kooshball / radial centre thousands of samples share a cell, so the
// W^NDIM taps of a cell are held in registers and reused across the cell's
// samples: interpolation reads the cube from the shared tile once per cell,
// gridding accumulates into the cube and flushes it (shared atomics) once per
// cell.
//
// Lane layout: lane = (stream s, slice group g, coil c). A lane owns SPL
// consecutive slices of the cube (tap indices along the outermost axis: z in
// 3D, y in 2D, x in 1D) for coil c: the whole cube (NG = 1) whenever it fits
// in 64 complex registers, else NG groups of slices whose partial sums are
// reduced with warp shuffles. CC coils and NS = 32/(NG*CC) independent sample
// streams per warp. Complex arithmetic uses the packed FP32 instructions
// (__ffma2_rn / __fmul2_rn).
// ---------------------------------------------------------------------------
template <int NDIM, int W, int CR = 64>
struct CubeShape {
    static constexpr int INS = NDIM == 3 ? W * W : (NDIM == 2 ? W : 1);  // taps per slice
    static constexpr int SPL0 = CR / INS;                                 // slices that fit in CR complex regs
    static constexpr int SPL = SPL0 >= W ? W : (SPL0 < 1 ? 1 : SPL0);     // slices per lane
    static constexpr int NGR = (W + SPL - 1) / SPL;                       // groups needed
    static constexpr int NG = NGR <= 1 ? 1 : (NGR <= 2 ? 2 : (NGR <= 4 ? 4 : (NGR <= 8 ? 8 : 16)));
    static constexpr int CUBE = SPL * INS;                                // complex registers
    static constexpr int NW = NDIM * W;                                   // staged weights
    // staging stride of a sample's weights: odd, so that the two samples a warp
    // reads at once (16 apart) fall on different banks
    static constexpr int NWP = NW | 1;
    static constexpr int SB = 128;                                        // staged samples (128: 24.3 vs 26.5 ms 3D gridding, 192^3 kooshball)
    static size_t meta_bytes() { return (size_t)SB * (NWP * sizeof(float) + 2 * sizeof(int)); }
};

// shared-memory geometry of the staged tile + halo for one coil chunk
struct Region {
    int R0, R1, R2;  // extents with halo (T + W - 1 on used axes)
    int SP;          // slice pitch of the outermost axis (padded against bank conflicts)
    int PP;          // coil pitch (padded)
};

// offset of tap j of a slice (row-major over the inner axes)
template <int NDIM, int W>
__device__ __forceinline__ int inner_off(int j, int R0)
{
    if (NDIM == 3) return (j / W) * R0 + (j % W);
    if (NDIM == 2) return j;
    return 0;
}

__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }

// stage weights (zero beyond an axis' own width), first-tap offset in the
// region, and global index of samples [base, base + n)
template <int NDIM, int W>
__device__ __forceinline__ void stage_cube_samples(const Geom &g, const int org[3], const Region &rg,
                                                   int base, int n, const float *__restrict__ sc0,
                                                   const float *__restrict__ sc1,
                                                   const float *__restrict__ sc2,
                                                   const int32_t *__restrict__ sidx, float *wts,
                                                   int *off, int *gi)
{
    constexpr int NW = (NDIM * W) | 1;  // staging stride (CubeShape::NWP)
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const int j = base + t;
        const float k[3] = {sc0[j], NDIM > 1 ? sc1[j] : 0.0f, NDIM > 2 ? sc2[j] : 0.0f};
        int l[3] = {0, 0, 0};
#pragma unroll
        for (int a = 0; a < NDIM; a++) {
            const int x0 = first_tap_dev(k[a], g.W[a]);
            l[a] = pmod(x0, g.G[a]) - org[a];
#pragma unroll
            for (int i = 0; i < W; i++)
                wts[t * NW + a * W + i] =
                    i < g.W[a] ? tap_weight(x0, i, k[a], g.W[a], g.inv_hw[a], g.beta[a]) : 0.0f;
        }
        off[t] = NDIM == 3 ? l[2] * rg.SP + l[1] * rg.R0 + l[0] : (NDIM == 2 ? l[1] * rg.SP + l[0] : l[0]);
        gi[t] = sidx[j];
    }
}

// Stage (or, with `flush`, atomically add back scaled by inv_scale) the
// tile + halo of CC coils, one grid row (R0 contiguous x) per thread step.
template <int NDIM>
__device__ __forceinline__ void region_io(const Geom &g, const Region &rg, const int org[3], int f,
                                          int64_t b0, int CC, int64_t batch, float2 *tile,
                                          float2 *__restrict__ grid, bool flush, float inv_scale)
{
    const int rpc = rg.R1 * rg.R2;  // rows per coil
    const int x_start = (org[0] + g.G[0] - g.half[0]) % g.G[0];
    for (int row = threadIdx.x; row < CC * rpc; row += blockDim.x) {
        const int c = row / rpc;
        const int rr = row - c * rpc;
        const int ry = rr % rg.R1;
        const int rz = rr / rg.R1;
        float2 *trow = tile + c * rg.PP + (NDIM == 3 ? rz * rg.SP + ry * rg.R0 : (NDIM == 2 ? ry * rg.SP : 0));
        const int64_t b = b0 + c;
        if (b >= batch) {
            if (!flush)
                for (int rx = 0; rx < rg.R0; rx++) trow[rx] = make_float2(0.0f, 0.0f);
            continue;
        }
        const int py = (org[1] + ry + g.G[1] - g.half[1]) % g.G[1];
        const int pz = (org[2] + rz + g.G[2] - g.half[2]) % g.G[2];
        float2 *grow = grid + (b * g.nframes + f) * g.gsize + ((int64_t)pz * g.G[1] + py) * g.G[0];
        int px = x_start;
        if (!flush) {
            for (int rx = 0; rx < rg.R0; rx++) {
                trow[rx] = grow[px];
                px = (px + 1 == g.G[0]) ? 0 : px + 1;
            }
        } else {
            for (int rx = 0; rx < rg.R0; rx++) {
                const float2 v = trow[rx];
                if (v.x != 0.0f || v.y != 0.0f) atomicAdd(grow + px, __fmul2_rn(v, f2(inv_scale)));
                px = (px + 1 == g.G[0]) ? 0 : px + 1;
            }
        }
    }
}

// Asynchronous 8-byte global -> shared copies (cp.async), so a block can stage
// its tile + halo while it computes sample weights.
__device__ __forceinline__ void cp_async8(void *sdst, const void *gsrc)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

template <int NDIM>
__device__ __forceinline__ void region_load_async(const Geom &g, const Region &rg, const int org[3], int f,
                                                  int64_t b0, int CC, int64_t batch, float2 *tile,
                                                  const float2 *__restrict__ grid)
{
    const int rpc = rg.R1 * rg.R2;
    const int x_start = (org[0] + g.G[0] - g.half[0]) % g.G[0];
    for (int row = threadIdx.x; row < CC * rpc; row += blockDim.x) {
        const int c = row / rpc;
        const int rr = row - c * rpc;
        const int ry = rr % rg.R1;
        const int rz = rr / rg.R1;
        float2 *trow = tile + c * rg.PP + (NDIM == 3 ? rz * rg.SP + ry * rg.R0 : (NDIM == 2 ? ry * rg.SP : 0));
        const int64_t b = b0 + c;
        if (b >= batch) {
            for (int rx = 0; rx < rg.R0; rx++) trow[rx] = make_float2(0.0f, 0.0f);
            continue;
        }
        const int py = (org[1] + ry + g.G[1] - g.half[1]) % g.G[1];
        const int pz = (org[2] + rz + g.G[2] - g.half[2]) % g.G[2];
        const float2 *grow = grid + (b * g.nframes + f) * g.gsize + ((int64_t)pz * g.G[1] + py) * g.G[0];
        int px = x_start;
        for (int rx = 0; rx < rg.R0; rx++) {
            cp_async8(trow + rx, grow + px);
            px = (px + 1 == g.G[0]) ? 0 : px + 1;
        }
    }
}

struct LaneMap {
    int c, gs, s, ns, stream, nstreams;
    unsigned smask;
};

template <int NG>
__device__ __forceinline__ LaneMap lane_map(int cc_log2)
{
    LaneMap m;
    const int CC = 1 << cc_log2;
    const int lane = threadIdx.x & 31;
    m.c = lane & (CC - 1);
    m.gs = (lane >> cc_log2) & (NG - 1);
    m.s = lane / (CC * NG);
    m.ns = 32 / (CC * NG);
    m.stream = (threadIdx.x >> 5) * m.ns + m.s;
    m.nstreams = (blockDim.x >> 5) * m.ns;
    m.smask = (CC * NG == 32) ? 0xffffffffu : (((1u << (CC * NG)) - 1u) << (m.s * CC * NG));
    return m;
}

constexpr int kCubeThreads = 128;
constexpr int kPf = 4;  // samples whose k-space values a gridding lane loads ahead
#ifndef DMR_INTERP_CUBE_REGS
#define DMR_INTERP_CUBE_REGS 64
#endif
#ifndef DMR_INTERP_COILS_3D
#define DMR_INTERP_COILS_3D 16
#endif
constexpr int kInterpCubeRegs = DMR_INTERP_CUBE_REGS;  // complex registers of an interpolation lane's cube

template <int NDIM, int W, int CR>
__global__ void __launch_bounds__(kCubeThreads) interp_cube_kernel(
    Geom g, Region rg, const WorkItem *__restrict__ work, const float *__restrict__ sc0,
    const float *__restrict__ sc1, const float *__restrict__ sc2, const int32_t *__restrict__ sidx,
    const float2 *__restrict__ grid, float2 *__restrict__ ksp, int64_t batch,
    const float *__restrict__ weight, int wpb, float inv_scale, int cc_log2)
{
    using S = CubeShape<NDIM, W, CR>;
    constexpr int NG = S::NG, SPL = S::SPL, INS = S::INS, NW = S::NW;
    extern __shared__ __align__(16) unsigned char smem[];
    const int CC = 1 << cc_log2;
    const WorkItem it = work[blockIdx.x];  // key order (16.2 vs 15.7 ms in 4x4x4-bin tiles)
    const int f = it.bin / g.nbins;
    int org[3];
    tile_origin(g, it.bin - f * g.nbins, org);
    float2 *tile = reinterpret_cast<float2 *>(smem);
    float *wts = reinterpret_cast<float *>(tile + (size_t)CC * rg.PP);
    int *off = reinterpret_cast<int *>(wts + S::SB * S::NWP);
    int *gi = off + S::SB;
    const int64_t b0 = (int64_t)blockIdx.y * CC;
    // tile copies in flight while the first batch of weights is computed
    region_load_async<NDIM>(g, rg, org, f, b0, CC, batch, tile, grid);

    const LaneMap m = lane_map<NG>(cc_log2);
    const int64_t b = b0 + m.c;
    const int z0 = m.gs * SPL;  // first slice of this lane
    const float2 *ctile = tile + m.c * rg.PP + z0 * rg.SP;

    for (int base = it.begin; base < it.end; base += S::SB) {
        const int n = min(S::SB, it.end - base);
        if (base != it.begin) __syncthreads();
        stage_cube_samples<NDIM, W>(g, org, rg, base, n, sc0, sc1, sc2, sidx, wts, off, gi);
        if (base == it.begin) cp_async_wait_all();
        __syncthreads();
        const int q0 = (int)((int64_t)n * m.stream / m.nstreams);
        const int q1 = (int)((int64_t)n * (m.stream + 1) / m.nstreams);
        int cur = -1;
        float2 cube[SPL][INS];
        for (int q = q0; q < q1; q++) {
            const int o = off[q];
            if (o != cur) {
                cur = o;
#pragma unroll
                for (int sl = 0; sl < SPL; sl++)
                    if (z0 + sl < W) {
#pragma unroll
                        for (int j = 0; j < INS; j++) cube[sl][j] = ctile[o + sl * rg.SP + inner_off<NDIM, W>(j, rg.R0)];
                    }
            }
            const float *w = wts + q * S::NWP;
            float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
            for (int sl = 0; sl < SPL; sl++) {
                if (z0 + sl >= W) continue;
                float2 t = make_float2(0.0f, 0.0f);
                if (NDIM == 3) {
#pragma unroll
                    for (int jy = 0; jy < W; jy++) {
                        float2 r = make_float2(0.0f, 0.0f);
#pragma unroll
                        for (int ix = 0; ix < W; ix++) r = __ffma2_rn(f2(w[ix]), cube[sl][jy * W + ix], r);
                        t = __ffma2_rn(f2(w[W + jy]), r, t);
                    }
                } else if (NDIM == 2) {
#pragma unroll
                    for (int ix = 0; ix < W; ix++) t = __ffma2_rn(f2(w[ix]), cube[sl][ix], t);
                } else {
                    t = cube[sl][0];
                }
                acc = __ffma2_rn(f2(w[(NDIM - 1) * W + z0 + sl]), t, acc);
            }
            if (NG > 1) {
#pragma unroll
                for (int k = 1; k < NG; k <<= 1) {
                    acc.x += __shfl_xor_sync(m.smask, acc.x, k * CC);
                    acc.y += __shfl_xor_sync(m.smask, acc.y, k * CC);
                }
            }
            if (m.gs == 0 && b < batch) {
                const int64_t o2 = b * g.total + gi[q];
                float sw = inv_scale;
                if (weight) sw *= weight[wpb ? o2 : (int64_t)gi[q]];
                ksp[o2] = __fmul2_rn(acc, f2(sw));
            }
        }
    }
}

template <int NDIM, int W, int CR>
__global__ void __launch_bounds__(kCubeThreads) grid_cube_kernel(
    Geom g, Region rg, const WorkItem *__restrict__ work, const float *__restrict__ sc0,
    const float *__restrict__ sc1, const float *__restrict__ sc2, const int32_t *__restrict__ sidx,
    const void *__restrict__ ksp, int kreal, float2 *__restrict__ grid, int64_t batch,
    const float *__restrict__ weight, int wpb, float inv_scale, int cc_log2)
{
    using S = CubeShape<NDIM, W, CR>;
    constexpr int NG = S::NG, SPL = S::SPL, INS = S::INS, NW = S::NW;
    extern __shared__ __align__(16) unsigned char smem[];
    const int CC = 1 << cc_log2;
    const WorkItem it = work[blockIdx.x];
    const int f = it.bin / g.nbins;
    int org[3];
    tile_origin(g, it.bin - f * g.nbins, org);
    float2 *tile = reinterpret_cast<float2 *>(smem);
    float *wts = reinterpret_cast<float *>(tile + (size_t)CC * rg.PP);
    int *off = reinterpret_cast<int *>(wts + S::SB * S::NWP);
    int *gi = off + S::SB;
    for (int e = threadIdx.x; e < CC * rg.PP; e += blockDim.x) tile[e] = make_float2(0.0f, 0.0f);
    const int64_t b0 = (int64_t)blockIdx.y * CC;

    const LaneMap m = lane_map<NG>(cc_log2);
    const int64_t b = b0 + m.c;
    const int z0 = m.gs * SPL;
    const bool active = z0 < W && b < batch;
    float2 *ctile = tile + m.c * rg.PP + z0 * rg.SP;

    for (int base = it.begin; base < it.end; base += S::SB) {
        const int n = min(S::SB, it.end - base);
        __syncthreads();
        stage_cube_samples<NDIM, W>(g, org, rg, base, n, sc0, sc1, sc2, sidx, wts, off, gi);
        __syncthreads();
        if (!active) continue;
        const int q0 = (int)((int64_t)n * m.stream / m.nstreams);
        const int q1 = (int)((int64_t)n * (m.stream + 1) / m.nstreams);
        int cur = -1;
        float2 cube[SPL][INS];
#pragma unroll
        for (int sl = 0; sl < SPL; sl++)
#pragma unroll
            for (int j = 0; j < INS; j++) cube[sl][j] = make_float2(0.0f, 0.0f);
        const int flip = (threadIdx.x >> 4) & 1;
        auto flush = [&](int o) {
#pragma unroll
            for (int sl = 0; sl < SPL; sl++)
                if (z0 + sl < W) {
#pragma unroll
                    for (int j = 0; j < INS; j++) {
                        // the upper half-warp adds the imaginary part first: the two
                        // halves then hit odd and even words, all 32 banks
                        float *p = reinterpret_cast<float *>(ctile + o + sl * rg.SP + inner_off<NDIM, W>(j, rg.R0));
                        const float a = flip ? cube[sl][j].y : cube[sl][j].x;
                        const float c = flip ? cube[sl][j].x : cube[sl][j].y;
                        atomicAdd(p + flip, a);
                        atomicAdd(p + 1 - flip, c);
                        cube[sl][j] = make_float2(0.0f, 0.0f);
                    }
                }
        };
        // the k-space values (and density weights) of the next kPf samples are
        // loaded ahead: a warp otherwise waits a full global-load latency per sample
        float2 pv[kPf];
        float pw[kPf];
        auto fetch = [&](int q, float2 &v, float &wt) {
            v = make_float2(0.0f, 0.0f);
            wt = 1.0f;
            if (q < q1) {
                const int64_t o2 = b * g.total + gi[q];
                v = load_sample(ksp, kreal, o2);
                if (weight) wt = weight[wpb ? o2 : (int64_t)gi[q]];
            }
        };
#pragma unroll
        for (int k = 0; k < kPf; k++) fetch(q0 + k, pv[k], pw[k]);
        for (int q = q0; q < q1; q++) {
            const int o = off[q];
            if (o != cur) {
                if (cur >= 0) flush(cur);
                cur = o;
            }
            float2 v = pv[0];
            if (weight) v = __fmul2_rn(v, f2(pw[0]));
#pragma unroll
            for (int k = 0; k + 1 < kPf; k++) {
                pv[k] = pv[k + 1];
                pw[k] = pw[k + 1];
            }
            fetch(q + kPf, pv[kPf - 1], pw[kPf - 1]);
            const float *w = wts + q * S::NWP;
#pragma unroll
            for (int sl = 0; sl < SPL; sl++) {
                if (z0 + sl >= W) continue;
                const float2 u = __fmul2_rn(f2(w[(NDIM - 1) * W + z0 + sl]), v);
                if (NDIM == 3) {
#pragma unroll
                    for (int jy = 0; jy < W; jy++) {
                        const float2 t = __fmul2_rn(f2(w[W + jy]), u);
#pragma unroll
                        for (int ix = 0; ix < W; ix++)
                            cube[sl][jy * W + ix] = __ffma2_rn(f2(w[ix]), t, cube[sl][jy * W + ix]);
                    }
                } else if (NDIM == 2) {
#pragma unroll
                    for (int ix = 0; ix < W; ix++) cube[sl][ix] = __ffma2_rn(f2(w[ix]), u, cube[sl][ix]);
                } else {
                    cube[sl][0] = __fadd2_rn(cube[sl][0], u);
                }
            }
        }
        if (cur >= 0) flush(cur);
    }
    __syncthreads();
    region_io<NDIM>(g, rg, org, f, b0, CC, batch, tile, grid, true, inv_scale);
}

// ---------------------------------------------------------------------------
// Gridding by slab ownership. Block = W warps; warp w owns the tile slices
// (outermost axis: z in 3D, y in 2D, x in 1D) congruent to w modulo W, so of
// every sample's W^NDIM taps it handles the one slice that falls in its own.
// All warps walk all samples of the bin in sorted (cell) order; lane (group
// rr, coil c) owns the taps of that slice whose next-axis offset (y in 3D, x
// in 2D) is congruent to rr modulo NR, for coil c, and accumulates them in
// registers while the cell does not change, then adds them to the shared tile
// with plain read-modify-writes. Every (point, coil) has exactly one owner
// lane, so there are no shared-memory atomics and each tile sums in a fixed
// order. The tile + halo is then added to the grid: with global atomics, or
// (deterministic mode) with plain read-modify-writes, the launcher running
// the bins in colour passes whose tile + halo regions are disjoint.
// ---------------------------------------------------------------------------
template <int NDIM, int W, int NR, bool ATOMIC_FLUSH>
__global__ void __launch_bounds__(32 * W) grid_slab_kernel(
    Geom g, Region rg, const WorkItem *__restrict__ work, const float *__restrict__ sc0,
    const float *__restrict__ sc1, const float *__restrict__ sc2, const int32_t *__restrict__ sidx,
    const void *__restrict__ ksp, int kreal, float2 *__restrict__ grid, int64_t batch,
    const float *__restrict__ weight, int wpb, float inv_scale, int cc_log2)
{
    using S = CubeShape<NDIM, W>;
    constexpr int NW = S::NW;
    constexpr int RL = NDIM == 1 ? 1 : (W + NR - 1) / NR;  // owned next-axis taps per lane
    constexpr int CL = NDIM == 3 ? W : 1;                  // x taps per owned row (3D)
    extern __shared__ __align__(16) unsigned char smem[];
    const int CC = 1 << cc_log2;
    const WorkItem it = work[blockIdx.x];
    const int f = it.bin / g.nbins;
    int org[3];
    tile_origin(g, it.bin - f * g.nbins, org);
    float2 *tile = reinterpret_cast<float2 *>(smem);
    float *wts = reinterpret_cast<float *>(tile + (size_t)CC * rg.PP);
    int *off = reinterpret_cast<int *>(wts + S::SB * S::NWP);
    int *gi = off + S::SB;
    for (int e = threadIdx.x; e < CC * rg.PP; e += blockDim.x) tile[e] = make_float2(0.0f, 0.0f);
    const int64_t b0 = (int64_t)blockIdx.y * CC;

    const int lane = threadIdx.x & 31;
    const int wz = threadIdx.x >> 5;  // owned slices: wz (mod W)
    const int c = lane & (CC - 1);
    const int rr = lane >> cc_log2;  // tap group on the next axis
    const int64_t b = b0 + c;
    const bool active = b < batch && (NDIM == 1 ? rr == 0 : (rr < NR && rr < W));
    float2 *ctile = tile + c * rg.PP;
    const int nstride = NDIM == 3 ? rg.R0 : 1;  // pitch of the next axis

    for (int base = it.begin; base < it.end; base += S::SB) {
        const int n = min(S::SB, it.end - base);
        __syncthreads();
        stage_cube_samples<NDIM, W>(g, org, rg, base, n, sc0, sc1, sc2, sidx, wts, off, gi);
        __syncthreads();
        if (!active) continue;
        int cur = -1, dz = 0;
        float2 acc[RL][CL];
#pragma unroll
        for (int k = 0; k < RL; k++)
#pragma unroll
            for (int i = 0; i < CL; i++) acc[k][i] = make_float2(0.0f, 0.0f);
        auto flush = [&](int o) {
            float2 *pl = ctile + o + dz * rg.SP;
#pragma unroll
            for (int k = 0; k < RL; k++) {
                const int dy = rr + NR * k;
                if (NDIM > 1 && dy >= W) continue;
                float2 *row = pl + (NDIM == 1 ? 0 : dy * nstride);
#pragma unroll
                for (int i = 0; i < CL; i++) {
                    row[i] = __fadd2_rn(row[i], acc[k][i]);
                    acc[k][i] = make_float2(0.0f, 0.0f);
                }
            }
        };
        for (int q = 0; q < n; q++) {
            const int o = off[q];
            if (o != cur) {
                if (cur >= 0) flush(cur);
                cur = o;
                const int lz = o / rg.SP;  // outermost index of the first tap
                dz = wz - lz % W;
                if (dz < 0) dz += W;
            }
            const int64_t o2 = b * g.total + gi[q];
            float2 v = load_sample(ksp, kreal, o2);
            if (weight) v = __fmul2_rn(v, f2(weight[wpb ? o2 : (int64_t)gi[q]]));
            const float *w = wts + q * S::NWP;
            const float2 u = __fmul2_rn(f2(w[(NDIM - 1) * W + dz]), v);
#pragma unroll
            for (int k = 0; k < RL; k++) {
                const int dy = rr + NR * k;
                if (NDIM > 1 && dy >= W) continue;
                if (NDIM == 3) {
                    const float2 t = __fmul2_rn(f2(w[W + dy]), u);
#pragma unroll
                    for (int i = 0; i < CL; i++) acc[k][i] = __ffma2_rn(f2(w[i]), t, acc[k][i]);
                } else if (NDIM == 2) {
                    acc[k][0] = __ffma2_rn(f2(w[dy]), u, acc[k][0]);
                } else {
                    acc[k][0] = __fadd2_rn(acc[k][0], u);
                }
            }
        }
        if (cur >= 0) flush(cur);
    }
    __syncthreads();
    if (ATOMIC_FLUSH) {
        region_io<NDIM>(g, rg, org, f, b0, CC, batch, tile, grid, true, inv_scale);
        return;
    }
    // deterministic: this bin's region is disjoint from every other bin of the
    // pass. A region longer than the grid on some axis (tiny grids) wraps onto
    // itself: then a single thread adds it, in a fixed order.
    const bool self_alias = rg.R0 > g.G[0] || (NDIM > 1 && rg.R1 > g.G[1]) || (NDIM > 2 && rg.R2 > g.G[2]);
    if (self_alias && threadIdx.x != 0) return;
    const int rpc = rg.R1 * rg.R2;
    const int x_start = (org[0] + g.G[0] - g.half[0]) % g.G[0];
    const int rstart = self_alias ? 0 : threadIdx.x;
    const int rstep = self_alias ? 1 : blockDim.x;
    for (int row = rstart; row < CC * rpc; row += rstep) {
        const int cc = row / rpc;
        const int r2 = row - cc * rpc;
        const int ry = r2 % rg.R1;
        const int rz = r2 / rg.R1;
        const int64_t bb = b0 + cc;
        if (bb >= batch) continue;
        const float2 *trow = tile + cc * rg.PP + (NDIM == 3 ? rz * rg.SP + ry * rg.R0 : (NDIM == 2 ? ry * rg.SP : 0));
        const int py = (org[1] + ry + g.G[1] - g.half[1]) % g.G[1];
        const int pz = (org[2] + rz + g.G[2] - g.half[2]) % g.G[2];
        float2 *grow = grid + (bb * g.nframes + f) * g.gsize + ((int64_t)pz * g.G[1] + py) * g.G[0];
        int px = x_start;
        for (int rx = 0; rx < rg.R0; rx++) {
            const float2 v = trow[rx];
            if (v.x != 0.0f || v.y != 0.0f) grow[px] = __ffma2_rn(v, f2(inv_scale), grow[px]);
            px = (px + 1 == g.G[0]) ? 0 : px + 1;
        }
    }
}

// ---------------------------------------------------------------------------
// Gridding, deterministic mode: one warp owns one tile (no halo) for CC coils
// and visits, in a fixed order, every sample of the bins that can reach the
// tile (the tile's own bin and its lower neighbours on each axis). Lane
// (group gr, coil c) owns the tile slices (outermost axis) congruent to gr
// modulo 32/CC, so every grid value is summed by one lane in sample order:
// bitwise reproducible, no atomics, and the grid is written exactly once
// (no zero-fill needed).
// ---------------------------------------------------------------------------
constexpr int kOwnerWarps = 2;

template <int NDIM>
__host__ __device__ inline void owner_dims(const Geom &g, int &slices, int &inner, int &SP, int &CP)
{
    slices = g.T[NDIM - 1];
    inner = 1;
    for (int a = 0; a < NDIM - 1; a++) inner *= g.T[a];
    SP = inner | 1;
    CP = (slices * SP) | 1;
}

template <int NDIM, int WMAX>
__global__ void __launch_bounds__(32 * kOwnerWarps) grid_owner_kernel(
    Geom g, const int32_t *__restrict__ tiles, int ntiles, const int32_t *__restrict__ bin_start,
    const float *__restrict__ sc0, const float *__restrict__ sc1, const float *__restrict__ sc2,
    const int32_t *__restrict__ sidx, const void *__restrict__ ksp, int kreal,
    float2 *__restrict__ grid, int64_t batch, const float *__restrict__ weight, int wpb,
    float scale, int cc_log2)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int CC = 1 << cc_log2;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int u = blockIdx.x * kOwnerWarps + warp;
    if (u >= ntiles) return;  // warp-uniform; no block-level barriers below
    int slices, inner, SP, CP;
    owner_dims<NDIM>(g, slices, inner, SP, CP);
    constexpr int NW = NDIM * WMAX;
    float2 *acc = reinterpret_cast<float2 *>(smem) + (size_t)warp * CC * CP;
    float *wbuf = reinterpret_cast<float *>(reinterpret_cast<float2 *>(smem) + (size_t)kOwnerWarps * CC * CP) +
                  warp * NW;

    const int key = tiles[u];
    const int f = key / g.nbins;
    const int lb = key - f * g.nbins;
    int org[3], bb[3], Te[3], lo[3], cnt[3];
    tile_origin(g, lb, org);
    bb[0] = lb % g.nb[0];
    bb[1] = (lb / g.nb[0]) % g.nb[1];
    bb[2] = lb / (g.nb[0] * g.nb[1]);
    for (int a = 0; a < 3; a++) {
        Te[a] = min(g.T[a], g.G[a] - org[a]);
        const int first = pmod(org[a] - g.W[a] + 1, g.G[a]) / g.T[a];
        lo[a] = first;
        cnt[a] = pmod(bb[a] - first, g.nb[a]) + 1;
    }
    for (int i = lane; i < CC * CP; i += 32) acc[i] = make_float2(0.0f, 0.0f);
    __syncwarp();

    const int gmask = (1 << (5 - cc_log2)) - 1;  // 32/CC slice groups
    const int gr = lane >> cc_log2;
    const int c = lane & (CC - 1);
    const int64_t b = (int64_t)blockIdx.y * CC + c;
    const int Wo = g.W[NDIM - 1];

    for (int iz = 0; iz < cnt[2]; iz++)
        for (int iy = 0; iy < cnt[1]; iy++)
            for (int ix = 0; ix < cnt[0]; ix++) {
                const int sb = (((lo[2] + iz) % g.nb[2]) * g.nb[1] + (lo[1] + iy) % g.nb[1]) * g.nb[0] +
                               (lo[0] + ix) % g.nb[0];
                const int s0 = bin_start[f * g.nbins + sb];
                const int s1 = bin_start[f * g.nbins + sb + 1];
                for (int j = s0; j < s1; j++) {
                    const float k[3] = {sc0[j], NDIM > 1 ? sc1[j] : 0.0f, NDIM > 2 ? sc2[j] : 0.0f};
                    int x0[3] = {0, 0, 0}, d[3] = {0, 0, 0};
                    bool hit = true;
#pragma unroll
                    for (int a = 0; a < NDIM; a++) {
                        x0[a] = first_tap_dev(k[a], g.W[a]);
                        d[a] = pmod(x0[a], g.G[a]) - org[a];
                        if (d[a] < 0) d[a] += g.G[a];
                        hit = hit && (d[a] < Te[a] || d[a] + g.W[a] - 1 >= g.G[a]);
                    }
                    if (!hit) continue;  // uniform across the warp
                    // weights: lane l computes table entries l, l + 32, ...
                    __syncwarp();  // previous sample's weights fully consumed
                    for (int e = lane; e < NW; e += 32) {
                        const int a = e / WMAX, i = e - a * WMAX;
                        wbuf[e] = i < g.W[a] ? tap_weight(x0[a], i, k[a], g.W[a], g.inv_hw[a], g.beta[a]) : 0.0f;
                    }
                    __syncwarp();
                    if (b >= batch) continue;
                    const int64_t o = b * g.total + sidx[j];
                    float2 v = load_sample(ksp, kreal, o);
                    if (weight) {
                        const float wv = weight[wpb ? o : (int64_t)sidx[j]];
                        v.x *= wv;
                        v.y *= wv;
                    }
                    float wx[WMAX];
#pragma unroll
                    for (int i = 0; i < WMAX; i++) wx[i] = wbuf[i];
                    float2 *basep = acc + c * CP;
                    const int Go = g.G[NDIM - 1];
                    for (int io = 0; io < Wo; io++) {
                        int uo = d[NDIM - 1] + io;
                        if (uo >= Go) uo -= Go;
                        if (uo >= Te[NDIM - 1] || (uo & gmask) != gr) continue;
                        float2 *sl = basep + uo * SP;
                        const float wo = wbuf[(NDIM - 1) * WMAX + io];
                        if (NDIM == 1) {
                            sl[0].x += wo * v.x;
                            sl[0].y += wo * v.y;
                        } else if (NDIM == 2) {
#pragma unroll
                            for (int i = 0; i < WMAX; i++) {
                                if (i >= g.W[0]) continue;
                                int ux = d[0] + i;
                                if (ux >= g.G[0]) ux -= g.G[0];
                                if (ux >= Te[0]) continue;
                                const float wv = wo * wx[i];
                                sl[ux].x += wv * v.x;
                                sl[ux].y += wv * v.y;
                            }
                        } else {
                            for (int iy2 = 0; iy2 < g.W[1]; iy2++) {
                                int uy = d[1] + iy2;
                                if (uy >= g.G[1]) uy -= g.G[1];
                                if (uy >= Te[1]) continue;
                                const float wzy = wo * wbuf[WMAX + iy2];
                                float2 *row = sl + uy * g.T[0];
#pragma unroll
                                for (int i = 0; i < WMAX; i++) {
                                    if (i >= g.W[0]) continue;
                                    int ux = d[0] + i;
                                    if (ux >= g.G[0]) ux -= g.G[0];
                                    if (ux >= Te[0]) continue;
                                    const float wv = wzy * wx[i];
                                    row[ux].x += wv * v.x;
                                    row[ux].y += wv * v.y;
                                }
                            }
                        }
                    }
                }
            }
    __syncwarp();
    // write the tile interior once, FFT order
    const int npts = slices * inner;
    for (int idx = lane; idx < CC * npts; idx += 32) {
        const int cc = idx / npts;
        const int r = idx - cc * npts;
        const int64_t bb2 = (int64_t)blockIdx.y * CC + cc;
        if (bb2 >= batch) continue;
        const int so = r / inner;
        const int ri = r - so * inner;
        int l[3] = {0, 0, 0};
        l[NDIM - 1] = so;
        if (NDIM == 2) l[0] = ri;
        if (NDIM == 3) {
            l[0] = ri % g.T[0];
            l[1] = ri / g.T[0];
        }
        if (l[0] >= Te[0] || l[1] >= Te[1] || l[2] >= Te[2]) continue;
        const float2 v = acc[cc * CP + so * SP + ri];
        const int px = (org[0] + l[0] + g.G[0] - g.half[0]) % g.G[0];
        const int py = (org[1] + l[1] + g.G[1] - g.half[1]) % g.G[1];
        const int pz = (org[2] + l[2] + g.G[2] - g.half[2]) % g.G[2];
        grid[(bb2 * g.nframes + f) * g.gsize + ((int64_t)pz * g.G[1] + py) * g.G[0] + px] =
            make_float2(v.x / scale, v.y / scale);
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static int wmax_for(const Geom &g)
{
    int w = 1;
    for (int a = 0; a < g.ndim; a++) w = std::max(w, g.W[a]);
    if (w <= 2) return 2;
    if (w <= 4) return 4;
    if (w <= 8) return 8;
    return 16;
}

static size_t region_points(const Geom &g)
{
    size_t p = 1;
    for (int a = 0; a < g.ndim; a++) p *= (size_t)(g.T[a] + g.W[a] - 1);
    return p | 1;
}

static int max_smem()
{
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v;
}

// Coils per block: a power of two <= 8 covering the batch, reduced until the
// tile + metadata fit in shared memory.
static int pick_cc_log2(int64_t batch, size_t per_coil, size_t fixed, size_t limit, int max_log2)
{
    int l = 0;
    while ((1ll << l) < batch && l < max_log2) l++;
    while (l > 0 && fixed + (per_coil << l) > limit) l--;
    return l;
}

template <int NDIM, int WMAX>
static int launch_interp(const dmr_plan *p, const float2 *grid, float2 *ksp, int64_t batch,
                         const float *weight, int wpb, cudaStream_t st)
{
    const Geom &g = p->g;
    using M = Meta<NDIM, WMAX>;
    const size_t per_coil = region_points(g) * sizeof(float2);
    const size_t limit = (size_t)max_smem();
    const int l = pick_cc_log2(batch, per_coil, M::bytes(), limit, 3);
    const size_t smem = M::bytes() + (per_coil << l);
    DMR_CHECK(smem <= limit, DMR_ERR_UNSUPPORTED, "interpolation tile needs %zu B of shared memory", smem);
    auto kern = interp_kernel<NDIM, WMAX>;
    DMR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t chunks = ceil_div(batch, 1ll << l);
    DMR_CHECK(chunks < 65536, DMR_ERR_UNSUPPORTED, "batch too large");
    dim3 grd(p->nwork, (unsigned)chunks);
    kern<<<grd, 256, smem, st>>>(g, p->work, p->scoord[0], p->scoord[1], p->scoord[2], p->sidx,
                                 grid, ksp, batch, weight, wpb, (float)p->scale, l);
    DMR_LAUNCHED("interp_kernel");
    return DMR_OK;
}

template <int NDIM, int WMAX>
static int launch_grid(const dmr_plan *p, const void *ksp, int kreal, float2 *grid, int64_t batch,
                       const float *weight, int wpb, int deterministic, cudaStream_t st)
{
    const Geom &g = p->g;
    const size_t limit = (size_t)max_smem();
    if (!deterministic) {
        using M = Meta<NDIM, WMAX>;
        const size_t per_coil = region_points(g) * sizeof(float2);
        const int l = pick_cc_log2(batch, per_coil, M::bytes(), limit, 3);
        const size_t smem = M::bytes() + (per_coil << l);
        DMR_CHECK(smem <= limit, DMR_ERR_UNSUPPORTED, "gridding tile needs %zu B of shared memory", smem);
        DMR_CUDA(cudaMemsetAsync(grid, 0, (size_t)batch * g.nframes * g.gsize * sizeof(float2), st));
        auto kern = grid_atomic_kernel<NDIM, WMAX>;
        DMR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const int64_t chunks = ceil_div(batch, 1ll << l);
        DMR_CHECK(chunks < 65536, DMR_ERR_UNSUPPORTED, "batch too large");
        if (p->nwork == 0) return DMR_OK;
        dim3 grd(p->nwork, (unsigned)chunks);
        kern<<<grd, 256, smem, st>>>(g, p->work, p->scoord[0], p->scoord[1], p->scoord[2], p->sidx,
                                     ksp, kreal, grid, batch, weight, wpb, (float)p->scale, l);
        DMR_LAUNCHED("grid_atomic_kernel");
        return DMR_OK;
    }
    int slices, inner, SP, CP;
    owner_dims<NDIM>(g, slices, inner, SP, CP);
    const size_t per_coil = (size_t)CP * sizeof(float2) * kOwnerWarps;
    const size_t wbytes = (size_t)kOwnerWarps * NDIM * WMAX * sizeof(float);
    const int l = pick_cc_log2(batch, per_coil, wbytes, limit, 2);
    const size_t smem = (per_coil << l) + wbytes;
    DMR_CHECK(smem <= limit, DMR_ERR_UNSUPPORTED, "owner tile needs %zu B of shared memory", smem);
    auto kern = grid_owner_kernel<NDIM, WMAX>;
    DMR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t chunks = ceil_div(batch, 1ll << l);
    DMR_CHECK(chunks < 65536, DMR_ERR_UNSUPPORTED, "batch too large");
    dim3 grd((unsigned)ceil_div(p->ntiles, kOwnerWarps), (unsigned)chunks);
    kern<<<grd, 32 * kOwnerWarps, smem, st>>>(g, p->tiles, p->ntiles, p->bin_start, p->scoord[0],
                                              p->scoord[1], p->scoord[2], p->sidx, ksp, kreal, grid,
                                              batch, weight, wpb, (float)p->scale, l);
    DMR_LAUNCHED("grid_owner_kernel");
    return DMR_OK;
}

// ---- cell-cube launchers ----------------------------------------------------
static int pad_mod16(int x, int m)
{
    m &= 15;
    return x + (((m - x) % 16) + 16) % 16;
}

template <int NDIM, int W, int CR = 64>
static Region cube_region(const Geom &g, int CC)
{
    using S = CubeShape<NDIM, W, CR>;
    Region r;
    r.R0 = g.T[0] + W - 1;
    r.R1 = NDIM > 1 ? g.T[1] + W - 1 : 1;
    r.R2 = NDIM > 2 ? g.T[2] + W - 1 : 1;
    // lanes of one half-warp differ in coil (pitch PP = 1 mod 16) and, with NG > 1,
    // in slice group (pitch SPL * SP = CC mod 16), so 8-byte accesses spread over banks
    // (the congruence may have no solution, e.g. SPL even and CC odd: then keep
    // the unpadded pitch; the search is bounded to one period)
    auto pad_slice = [&](int sp) {
        if (S::NG == 1) return sp;
        for (int d = 0; d < 16; d++)
            if (((S::SPL * (sp + d)) & 15) == (CC & 15)) return sp + d;
        return sp;
    };
    int P;
    if (NDIM == 3) {
        r.SP = pad_slice(r.R0 * r.R1);
        P = r.SP * r.R2;
    } else if (NDIM == 2) {
        r.SP = pad_slice(r.R0);
        P = r.SP * r.R1;
    } else {
        r.SP = 1;
        P = r.R0;
    }
    r.PP = pad_mod16(P, 1);
    return r;
}

// coils per block: power of two covering the batch, at most 32 / NG and
// max_coils, reduced until the tile + staged samples fit in shared memory.
// 3D interpolation caps at 16 coils (smaller tiles, more resident blocks:
// 15.6 vs 17.4 ms on the 192^3 kooshball with 32 coils); gridding keeps 32 (its
// per-sample weights are shared by more coils: 34.1 vs 35.2 ms).
template <int NDIM, int W, int CR = 64>
static int cube_config(const Geom &g, int64_t batch, Region &rg, size_t &smem, int max_coils)
{
    using S = CubeShape<NDIM, W, CR>;
    const size_t limit = (size_t)max_smem();
    // DMR_CUBE_MAX_COILS overrides the cap on coils per block (tuning)
    static const int env_cap = [] {
        const char *e = getenv("DMR_CUBE_MAX_COILS");
        return e ? std::max(1, atoi(e)) : 0;
    }();
    const int cap = env_cap ? env_cap : max_coils;
    int l = 0;
    while ((1ll << l) < batch && (1 << l) * S::NG < 32 && (2 << l) <= cap) l++;
    for (; l >= 0; l--) {
        rg = cube_region<NDIM, W, CR>(g, 1 << l);
        smem = S::meta_bytes() + (size_t)(1 << l) * rg.PP * sizeof(float2);
        if (smem <= limit) return l;
    }
    return -1;
}

template <int NDIM, int W>
static int launch_interp_cube(const dmr_plan *p, const float2 *grid, float2 *ksp, int64_t batch,
                              const float *weight, int wpb, cudaStream_t st)
{
    Region rg;
    size_t smem = 0;
    constexpr int CR = kInterpCubeRegs;
    const int l = cube_config<NDIM, W, CR>(p->g, batch, rg, smem, NDIM == 3 ? DMR_INTERP_COILS_3D : 32);
    DMR_CHECK(l >= 0, DMR_ERR_UNSUPPORTED, "interpolation tile does not fit in shared memory");
    auto kern = interp_cube_kernel<NDIM, W, CR>;
    DMR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t chunks = ceil_div(batch, 1ll << l);
    DMR_CHECK(chunks < 65536, DMR_ERR_UNSUPPORTED, "batch too large");
    kern<<<dim3(p->nwork, (unsigned)chunks), kCubeThreads, smem, st>>>(
        p->g, rg, p->work, p->scoord[0], p->scoord[1], p->scoord[2], p->sidx, grid, ksp, batch, weight,
        wpb, (float)(1.0 / p->scale), l);
    DMR_LAUNCHED("interp_cube_kernel");
    return DMR_OK;
}

template <int NDIM, int W>
static int launch_grid_cube(const dmr_plan *p, const void *ksp, int kreal, float2 *grid, int64_t batch,
                            const float *weight, int wpb, cudaStream_t st)
{
    Region rg;
    size_t smem = 0;
    // 3D: one 16-tap slice per lane (4 lanes per coil, 8 coils per warp): 27.1
    // vs 32.9 ms with the whole 64-tap cube per lane on the 192^3 kooshball
    // (fewer registers, more resident warps)
    constexpr int CR = NDIM == 3 ? 16 : 64;
    const int l = cube_config<NDIM, W, CR>(p->g, batch, rg, smem, 32);
    DMR_CHECK(l >= 0, DMR_ERR_UNSUPPORTED, "gridding tile does not fit in shared memory");
    DMR_CUDA(cudaMemsetAsync(grid, 0, (size_t)batch * p->g.nframes * p->g.gsize * sizeof(float2), st));
    if (p->nwork == 0) return DMR_OK;
    auto kern = grid_cube_kernel<NDIM, W, CR>;
    DMR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t chunks = ceil_div(batch, 1ll << l);
    DMR_CHECK(chunks < 65536, DMR_ERR_UNSUPPORTED, "batch too large");
    kern<<<dim3(p->nwork, (unsigned)chunks), kCubeThreads, smem, st>>>(
        p->g, rg, p->work, p->scoord[0], p->scoord[1], p->scoord[2], p->sidx, ksp, kreal, grid, batch,
        weight, wpb, (float)(1.0 / p->scale), l);
    DMR_LAUNCHED("grid_cube_kernel");
    return DMR_OK;
}

// Gridding with the slab kernel: CC = pow2 >= batch (at most 32) coils per
// block, NR = 32 / CC tap groups (extra lanes idle). Atomic mode launches all
// (chunked) work items at once; deterministic mode launches whole bins one
// colour pass at a time.
template <int NDIM, int W, int NR, bool ATOMIC>
static int launch_grid_slab_nr(const dmr_plan *p, const void *ksp, int kreal, float2 *grid, int64_t batch,
                               const float *weight, int wpb, int l, const Region &rg, size_t smem,
                               cudaStream_t st)
{
    auto kern = grid_slab_kernel<NDIM, W, NR, ATOMIC>;
    DMR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t chunks = ceil_div(batch, 1ll << l);
    DMR_CHECK(chunks < 65536, DMR_ERR_UNSUPPORTED, "batch too large");
    const float inv = (float)(1.0 / p->scale);
    if (ATOMIC) {
        kern<<<dim3(p->nwork, (unsigned)chunks), 32 * W, smem, st>>>(
            p->g, rg, p->work, p->scoord[0], p->scoord[1], p->scoord[2], p->sidx, ksp, kreal, grid, batch,
            weight, wpb, inv, l);
        DMR_LAUNCHED("grid_slab_kernel");
        return DMR_OK;
    }
    for (size_t c = 0; c + 1 < p->det_color_start.size(); c++) {
        const int n = p->det_color_start[c + 1] - p->det_color_start[c];
        if (n == 0) continue;
        kern<<<dim3(n, (unsigned)chunks), 32 * W, smem, st>>>(
            p->g, rg, p->det_work + p->det_color_start[c], p->scoord[0], p->scoord[1], p->scoord[2], p->sidx,
            ksp, kreal, grid, batch, weight, wpb, inv, l);
        DMR_LAUNCHED("grid_slab_kernel");
    }
    return DMR_OK;
}

template <int NDIM, int W, bool ATOMIC>
static int launch_grid_slab(const dmr_plan *p, const void *ksp, int kreal, float2 *grid, int64_t batch,
                            const float *weight, int wpb, cudaStream_t st)
{
    using S = CubeShape<NDIM, W>;
    const size_t limit = (size_t)max_smem();
    int l = 0;
    // deterministic passes run whole (unsplit) bins: at most 8 coils per block
    // so a dense bin is shared by several blocks (one per coil chunk)
    while ((1ll << l) < batch && l < (ATOMIC ? 5 : 3)) l++;
    Region rg;
    size_t smem = 0;
    for (; l >= 0; l--) {
        rg = cube_region<NDIM, W>(p->g, 1 << l);
        smem = S::meta_bytes() + (size_t)(1 << l) * rg.PP * sizeof(float2);
        if (smem <= limit) break;
    }
    DMR_CHECK(l >= 0, DMR_ERR_UNSUPPORTED, "gridding tile does not fit in shared memory");
    DMR_CUDA(cudaMemsetAsync(grid, 0, (size_t)batch * p->g.nframes * p->g.gsize * sizeof(float2), st));
    if (p->nwork == 0) return DMR_OK;
    switch (l) {
    case 5: return launch_grid_slab_nr<NDIM, W, 1, ATOMIC>(p, ksp, kreal, grid, batch, weight, wpb, l, rg, smem, st);
    case 4: return launch_grid_slab_nr<NDIM, W, 2, ATOMIC>(p, ksp, kreal, grid, batch, weight, wpb, l, rg, smem, st);
    case 3: return launch_grid_slab_nr<NDIM, W, 4, ATOMIC>(p, ksp, kreal, grid, batch, weight, wpb, l, rg, smem, st);
    case 2: return launch_grid_slab_nr<NDIM, W, 8, ATOMIC>(p, ksp, kreal, grid, batch, weight, wpb, l, rg, smem, st);
    case 1: return launch_grid_slab_nr<NDIM, W, 16, ATOMIC>(p, ksp, kreal, grid, batch, weight, wpb, l, rg, smem, st);
    default: return launch_grid_slab_nr<NDIM, W, 32, ATOMIC>(p, ksp, kreal, grid, batch, weight, wpb, l, rg, smem, st);
    }
}

// 3D gridding kernel choice: 0 = cell-cube kernel (shared atomics per cell),
// 1 = z-slab kernel; DMR_GRID_VARIANT overrides the default (tuning only)
static int grid_variant()
{
    static int v = [] {
        const char *e = getenv("DMR_GRID_VARIANT");
        return e ? atoi(e) : 0;
    }();
    return v;
}

// exact cube width instance for a plan: the widest axis, rounded up to an
// instantiated width (1..8, 12, 16; 3D only up to 8); 0 = use the generic kernels
static int cube_width(const Geom &g)
{
    int w = 1;
    for (int a = 0; a < g.ndim; a++) w = std::max(w, g.W[a]);
    if (w <= 8) return w;
    if (g.ndim == 3) return 0;
    return w <= 12 ? 12 : 16;
}

#define DMR_CUBE_CASES(F, ...)                                   \
    case 101: return F<1, 1>(__VA_ARGS__);                       \
    case 102: return F<1, 2>(__VA_ARGS__);                       \
    case 103: return F<1, 3>(__VA_ARGS__);                       \
    case 104: return F<1, 4>(__VA_ARGS__);                       \
    case 105: return F<1, 5>(__VA_ARGS__);                       \
    case 106: return F<1, 6>(__VA_ARGS__);                       \
    case 107: return F<1, 7>(__VA_ARGS__);                       \
    case 108: return F<1, 8>(__VA_ARGS__);                       \
    case 112: return F<1, 12>(__VA_ARGS__);                      \
    case 116: return F<1, 16>(__VA_ARGS__);                      \
    case 201: return F<2, 1>(__VA_ARGS__);                       \
    case 202: return F<2, 2>(__VA_ARGS__);                       \
    case 203: return F<2, 3>(__VA_ARGS__);                       \
    case 204: return F<2, 4>(__VA_ARGS__);                       \
    case 205: return F<2, 5>(__VA_ARGS__);                       \
    case 206: return F<2, 6>(__VA_ARGS__);                       \
    case 207: return F<2, 7>(__VA_ARGS__);                       \
    case 208: return F<2, 8>(__VA_ARGS__);                       \
    case 212: return F<2, 12>(__VA_ARGS__);                      \
    case 216: return F<2, 16>(__VA_ARGS__);                      \
    case 301: return F<3, 1>(__VA_ARGS__);                       \
    case 302: return F<3, 2>(__VA_ARGS__);                       \
    case 303: return F<3, 3>(__VA_ARGS__);                       \
    case 304: return F<3, 4>(__VA_ARGS__);                       \
    case 305: return F<3, 5>(__VA_ARGS__);                       \
    case 306: return F<3, 6>(__VA_ARGS__);                       \
    case 307: return F<3, 7>(__VA_ARGS__);                       \
    case 308: return F<3, 8>(__VA_ARGS__);

int interp_dispatch(const dmr_plan *p, const float2 *grid, float2 *ksp, int64_t batch,
                    const float *weight, int wpb, cudaStream_t st)
{
    if (p->nwork == 0) return DMR_OK;
    const int cw = cube_width(p->g);
    if (cw > 0) {
        switch (p->g.ndim * 100 + cw) {
            DMR_CUBE_CASES(launch_interp_cube, p, grid, ksp, batch, weight, wpb, st)
        default: break;
        }
    }
    const int wm = wmax_for(p->g);
    switch (p->g.ndim * 100 + wm) {
    case 102: return launch_interp<1, 2>(p, grid, ksp, batch, weight, wpb, st);
    case 104: return launch_interp<1, 4>(p, grid, ksp, batch, weight, wpb, st);
    case 108: return launch_interp<1, 8>(p, grid, ksp, batch, weight, wpb, st);
    case 116: return launch_interp<1, 16>(p, grid, ksp, batch, weight, wpb, st);
    case 202: return launch_interp<2, 2>(p, grid, ksp, batch, weight, wpb, st);
    case 204: return launch_interp<2, 4>(p, grid, ksp, batch, weight, wpb, st);
    case 208: return launch_interp<2, 8>(p, grid, ksp, batch, weight, wpb, st);
    case 216: return launch_interp<2, 16>(p, grid, ksp, batch, weight, wpb, st);
    case 302: return launch_interp<3, 2>(p, grid, ksp, batch, weight, wpb, st);
    case 304: return launch_interp<3, 4>(p, grid, ksp, batch, weight, wpb, st);
    case 308: return launch_interp<3, 8>(p, grid, ksp, batch, weight, wpb, st);
    case 316: return launch_interp<3, 16>(p, grid, ksp, batch, weight, wpb, st);
    default: break;
    }
    set_error("unsupported ndim/width");
    return DMR_ERR_UNSUPPORTED;
}

int grid_rt_dispatch(const dmr_plan *p, const void *ksp, int kreal, float2 *grid, int64_t batch,
                     const float *weight, int wpb, void *scratch, size_t scratch_bytes, cudaStream_t st);

// (the deterministic tensor-core gridding takes its larger scratch from the
// library pool, so that callers' workspaces do not hold it in atomic mode)
size_t grid_scratch_bytes(const dmr_plan *p, int64_t batch)
{
    return rt_scratch_bytes(p, batch);
}

// minimum coil count of atomic tensor-core gridding (dmr_tc_min_coils)
static std::atomic<int> g_tc_min_coils{20};

int grid_dispatch(const dmr_plan *p, const void *ksp, int kreal, float2 *grid, int64_t batch,
                  const float *weight, int wpb, int det, void *scratch, size_t scratch_bytes,
                  cudaStream_t st)
{
    // 3D gridding on the tensor cores: atomic, or deterministic (per-item
    // partial sums gathered per grid point in a fixed order, bitwise
    // reproducible), when the plan's gridding bins apply.
    // Its cost is mostly per sample (the spreading operand and the region
    // read-back are built for all 32 coil slots), so atomic gridding of fewer
    // coils runs on the CUDA cores, whose cost scales with the coil count
    // (192^3 kooshball: 12.1 vs 13.6 ms for 16 coils, 6.0 vs 13.0 for 8,
    // 24.1 vs 16.8 for 32).
    if (p->g.ndim == 3 && grid_variant() == 0 && (det || batch >= g_tc_min_coils.load())) {
        const int rc = grid_tc_dispatch(p, ksp, kreal, grid, batch, weight, wpb, det, scratch, scratch_bytes, st);
        if (rc != DMR_ERR_UNSUPPORTED) return rc;
    }
    // deterministic 3D gridding of 8+ coils otherwise: register tiles (one owner
    // per grid point, no colour passes) when the plan has them
    if (det) {
        const int rc = grid_rt_dispatch(p, ksp, kreal, grid, batch, weight, wpb, scratch, scratch_bytes, st);
        if (rc != DMR_ERR_UNSUPPORTED) return rc;
    }
    const int cw = cube_width(p->g);
    if (cw > 0 && (det || (p->g.ndim == 3 && grid_variant() == 1))) {
        switch (p->g.ndim * 100 + cw) {
#define SLAB(N, W)                                                                                  \
    case N * 100 + W:                                                                               \
        return det ? launch_grid_slab<N, W, false>(p, ksp, kreal, grid, batch, weight, wpb, st)     \
                   : launch_grid_slab<N, W, true>(p, ksp, kreal, grid, batch, weight, wpb, st);
            SLAB(1, 1) SLAB(1, 2) SLAB(1, 3) SLAB(1, 4) SLAB(1, 5) SLAB(1, 6) SLAB(1, 7) SLAB(1, 8)
            SLAB(2, 1) SLAB(2, 2) SLAB(2, 3) SLAB(2, 4) SLAB(2, 5) SLAB(2, 6) SLAB(2, 7) SLAB(2, 8)
            SLAB(3, 1) SLAB(3, 2) SLAB(3, 3) SLAB(3, 4) SLAB(3, 5) SLAB(3, 6) SLAB(3, 7) SLAB(3, 8)
#undef SLAB
        default: break;
        }
    }
    if (!det && cw > 0) {
        switch (p->g.ndim * 100 + cw) {
            DMR_CUBE_CASES(launch_grid_cube, p, ksp, kreal, grid, batch, weight, wpb, st)
        default: break;
        }
    }
    const int wm = wmax_for(p->g);
    switch (p->g.ndim * 100 + wm) {
    case 102: return launch_grid<1, 2>(p, ksp, kreal, grid, batch, weight, wpb, det, st);
    case 104: return launch_grid<1, 4>(p, ksp, kreal, grid, batch, weight, wpb, det, st);
    case 108: return launch_grid<1, 8>(p, ksp, kreal, grid, batch, weight, wpb, det, st);
    case 116: return launch_grid<1, 16>(p, ksp, kreal, grid, batch, weight, wpb, det, st);
    case 202: return launch_grid<2, 2>(p, ksp, kreal, grid, batch, weight, wpb, det, st);
    case 204: return launch_grid<2, 4>(p, ksp, kreal, grid, batch, weight, wpb, det, st);
    case 208: return launch_grid<2, 8>(p, ksp, kreal, grid, batch, weight, wpb, det, st);
    case 216: return launch_grid<2, 16>(p, ksp, kreal, grid, batch, weight, wpb, det, st);
    case 302: return launch_grid<3, 2>(p, ksp, kreal, grid, batch, weight, wpb, det, st);
    case 304: return launch_grid<3, 4>(p, ksp, kreal, grid, batch, weight, wpb, det, st);
    case 308: return launch_grid<3, 8>(p, ksp, kreal, grid, batch, weight, wpb, det, st);
    case 316: return launch_grid<3, 16>(p, ksp, kreal, grid, batch, weight, wpb, det, st);
    default: break;
    }
    set_error("unsupported ndim/width");
    return DMR_ERR_UNSUPPORTED;
}

}  // namespace dmr

using namespace dmr;

extern "C" int dmr_interp(const dmr_plan *p, const void *grid, void *kspace, int64_t batch,
                          const float *weight, int weight_per_batch, void *stream)
{
    DMR_CHECK(p && (grid || batch == 0) && (kspace || batch == 0), DMR_ERR_INVALID, "NULL argument");
    DMR_CHECK(batch >= 0, DMR_ERR_INVALID, "negative batch");
    if (batch == 0 || p->g.total == 0) return DMR_OK;
    return interp_dispatch(p, (const float2 *)grid, (float2 *)kspace, batch, weight,
                           weight_per_batch, (cudaStream_t)stream);
}

extern "C" int dmr_grid(const dmr_plan *p, const void *kspace, int kspace_real, void *grid,
                        int64_t batch, const float *weight, int weight_per_batch, int deterministic,
                        void *stream)
{
    DMR_CHECK(p && (grid || batch == 0) && (kspace || batch == 0), DMR_ERR_INVALID, "NULL argument");
    DMR_CHECK(batch >= 0, DMR_ERR_INVALID, "negative batch");
    if (batch == 0) return DMR_OK;
    return grid_dispatch(p, kspace, kspace_real, (float2 *)grid, batch, weight, weight_per_batch,
                         deterministic, nullptr, 0, (cudaStream_t)stream);
}

extern "C" int dmr_tc_min_coils(int coils)
{
    return coils > 0 ? dmr::g_tc_min_coils.exchange(coils) : dmr::g_tc_min_coils.load();
}
