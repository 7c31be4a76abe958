// Register-tile gridding for 3D: an output-stationary scatter.
//
// Reference: apply_gridding and its 3D kernel
// (src/deepmr/fft/_interp/grid.py:14-125, 253-284):
//   grid[f, b, iz, iy, ix] += value_z * value_y * value_x * y[f, b, p]   (then / scale)
//
// The oversampled grid of every frame is cut into 8^3 block regions. A block
// owns one region for 32 coils; each of its 8 warps owns a 4^3 sub-region and
// keeps it in registers (lane = coil: 64 complex accumulators per lane). The
// block walks the samples that can reach its region — those of the bins that
// cover first taps [org - W + 1, org + 7] on every axis — staging for each
// sample its x weights at the region's 8 positions (zero outside the kernel
// support), its y and z weights by tap with the y and z offsets of its first
// tap, and its 32 coil values in shared memory. Each warp then adds the
// samples whose support meets its sub-region: a warp-uniform two-level switch
// on the (z, y) offsets selects a branch-free body that touches exactly the
// (z, y) rows inside the support, with compile-time accumulator indices (the
// accumulators stay in registers); the only waste is the x positions of a
// 4-wide row that the support misses.
//
// There are no atomics: every grid point has one owner, which sums its
// contributions in the plan's fixed sample order, so the result is bitwise
// reproducible, and each grid point is written once with a plain store (no
// zero fill). A region whose window holds more than kRtChunk samples is split
// over several blocks (each takes the same fraction of every window bin) that
// write partial sums to scratch slots; a reduction kernel adds the slots of
// the region in slot order.
#include <algorithm>
#include <cstddef>
#include <cstdlib>
#include <vector>

#include "kb.cuh"
#include "plan.cuh"

namespace dmr {

constexpr int kRtX = 8, kRtY = 8, kRtZ = 8;   // block region (grid points)
constexpr int kRtPts = kRtX * kRtY * kRtZ;    // 512
constexpr int kRtWarps = 8;                   // 2 x 2 x 2 sub-regions of 4^3
constexpr int kRtThreads = 32 * kRtWarps;
constexpr int kRtCoils = 32;                  // coils per block (one per lane)
constexpr int kRtSB = 256;                    // samples staged per pass (one per thread)
constexpr int kRtMaxWB = 8;                   // window bins per axis
constexpr int kRtMaxBins = 128;               // window bins per region
constexpr int kRtChunk = 16384;               // window samples per block item
constexpr int kRtMinBatch = 8;                // below this, the cell-cube kernels are used
constexpr int kRtMaxW = 8;                    // kernel widths handled (offset cases -7..3)

__host__ __device__ constexpr int rt_extent(int a) { return a == 0 ? kRtX : (a == 1 ? kRtY : kRtZ); }

struct __align__(16) RtMeta {
    float qx[kRtSB][kRtX];               // x weights at region positions 0..7
    float wy[kRtSB][kRtMaxW];            // y weights of taps 0..W-1
    float wz[kRtSB][kRtMaxW];            // z weights of taps 0..W-1
    int fy[kRtSB];                       // y offset of the first tap from the region origin
    int fz[kRtSB];                       // z offset of the first tap from the region origin
    int gi[kRtSB];                       // global sample index
    unsigned mask[kRtSB];                // bit w: meets the column of warp w
    int n;                               // samples in this pass
    int pad[3];
};

// Double-buffered staging: the coil values of pass k+1 are copied (cp.async)
// while the warps accumulate pass k. A pass takes the same fraction of every
// window bin, so its samples spread over the whole region and the warps get
// similar shares of work between two barriers; inside a bin, samples keep
// the plan's sorted order.
struct RtShared {
    RtMeta meta[2];
    float2 v[2][kRtSB][kRtCoils + 1];    // sample values (padded rows: conflict-free staging)
    int wb_lo[kRtMaxBins];               // this item's slice of each window bin
    int wb_n[kRtMaxBins];
    int ps_start[kRtMaxBins];            // the current pass's slice of each window bin
    int ps_pre[kRtMaxBins + 1];          // exclusive prefix of the pass slice lengths
    int scan[kRtMaxBins + 1];
    int nwb;
};

// weights are read as float4 (qx) and values written by 8-byte cp.async
static_assert(sizeof(RtMeta) % 16 == 0, "RtMeta must stay 16-byte aligned in both buffers");
static_assert(offsetof(RtMeta, wy) % 16 == 0 && offsetof(RtMeta, wz) % 16 == 0, "aligned rows");
static_assert(offsetof(RtShared, v) % 16 == 0, "value buffers must be 16-byte aligned");
static_assert(sizeof(RtShared) <= 227 * 1024, "shared memory of a block");

__device__ __forceinline__ float2 rt_f2(float v) { return make_float2(v, v); }

// Bins of the window of a block region at org on one axis: the bins holding
// first taps [org - W + 1, min(org + extent - 1, G - 1)] taken modulo G (the
// part below 0 wraps to the top of the axis). Writes at most kRtMaxWB bins;
// returns the count, which the plan checks.
__host__ __device__ __forceinline__ int rt_axis_bins(int org, int ext, int G, int W, int T, int *bins)
{
    int n = 0;
    const int a = org - (W - 1);
    const int b = (org + ext - 1 < G - 1) ? org + ext - 1 : G - 1;
    if (a < 0)
        for (int bb = (G + a) / T; bb <= (G - 1) / T; bb++) {
            if (n < kRtMaxWB) bins[n] = bb;
            n++;
        }
    for (int bb = (a > 0 ? a : 0) / T; bb <= b / T; bb++) {
        if (n < kRtMaxWB) bins[n] = bb;
        n++;
    }
    return n;
}

__device__ __forceinline__ void rt_region(const Geom &g, int region, int &f, int org[3])
{
    f = region / g.nregions;
    const int lr = region - f * g.nregions;
    org[0] = (lr % g.nr[0]) * kRtX;
    org[1] = ((lr / g.nr[0]) % g.nr[1]) * kRtY;
    org[2] = (lr / (g.nr[0] * g.nr[1])) * kRtZ;
}

// Exclusive prefix of c over threads 0..127 into pre[0..128]; warp_tot is
// 4 ints of scratch. All threads call.
__device__ __forceinline__ void rt_scan128(int c, int *pre, int *warp_tot)
{
    const int lane = threadIdx.x & 31;
    int incl = c;
    if (threadIdx.x < 128) {
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += t;
        }
        if (lane == 31) warp_tot[threadIdx.x >> 5] = incl;
    }
    __syncthreads();
    if (threadIdx.x < 128) {
        int carry = 0;
        for (int w = 0; w < (int)(threadIdx.x >> 5); w++) carry += warp_tot[w];
        pre[threadIdx.x + 1] = incl + carry;
        if (threadIdx.x == 0) pre[0] = 0;
    }
    __syncthreads();
}

// Window bins of a region and this item's slice of each: part `part` of
// `nparts` equal fractions. Returns the item's sample count.
__device__ int rt_window_setup(const Geom &g, int f, const int org[3], int part, int nparts,
                               const int32_t *__restrict__ bin_start, RtShared &S)
{
    int bins[3][kRtMaxWB], cnt[3];
#pragma unroll
    for (int a = 0; a < 3; a++) cnt[a] = rt_axis_bins(org[a], rt_extent(a), g.G[a], g.W[a], g.T[a], bins[a]);
    const int nw = cnt[0] * cnt[1] * cnt[2];
    int c = 0;
    if ((int)threadIdx.x < nw) {
        const int ix = threadIdx.x % cnt[0];
        const int iy = (threadIdx.x / cnt[0]) % cnt[1];
        const int iz = threadIdx.x / (cnt[0] * cnt[1]);
        const int key = f * g.nbins + (bins[2][iz] * g.nb[1] + bins[1][iy]) * g.nb[0] + bins[0][ix];
        const int s0 = bin_start[key];
        const int64_t nb = bin_start[key + 1] - s0;
        const int lo = s0 + (int)(nb * part / nparts);
        const int hi = s0 + (int)(nb * (part + 1) / nparts);
        S.wb_lo[threadIdx.x] = lo;
        S.wb_n[threadIdx.x] = hi - lo;
        c = hi - lo;
    }
    if (threadIdx.x == 0) S.nwb = nw;
    rt_scan128(c, S.scan, S.ps_start);
    return S.scan[kRtMaxBins];
}

// Slice of every window bin for pass p of P (ps_start, ps_pre); returns its size.
__device__ __forceinline__ int rt_pass_layout(int p, int P, RtShared &S)
{
    int c = 0, start = 0;
    if ((int)threadIdx.x < S.nwb) {
        const int64_t nb = S.wb_n[threadIdx.x];
        const int a = (int)(nb * p / P), b = (int)(nb * (p + 1) / P);
        start = S.wb_lo[threadIdx.x] + a;
        c = b - a;
    }
    rt_scan128(c, S.ps_pre, S.scan);
    if ((int)threadIdx.x < S.nwb) S.ps_start[threadIdx.x] = start;
    __syncthreads();
    return S.ps_pre[kRtMaxBins];
}

// Stage the samples of the current pass layout: weights, offsets, masks, indices.
__device__ __forceinline__ void rt_stage_meta(const Geom &g, const int org[3], int n,
                                              const float *__restrict__ sc0,
                                              const float *__restrict__ sc1,
                                              const float *__restrict__ sc2,
                                              const int32_t *__restrict__ sidx,
                                              const float *__restrict__ wsample, const RtShared &S,
                                              RtMeta &M)
{
    const int nw = S.nwb;
    if (threadIdx.x == 0) M.n = n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        int lo = 0, hi = nw;  // ps_pre[lo] <= i < ps_pre[hi]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (S.ps_pre[mid] <= i) lo = mid; else hi = mid;
        }
        const int j = S.ps_start[lo] + (i - S.ps_pre[lo]);
        const int gi = sidx[j];
        const float dw = wsample ? wsample[gi] : 1.0f;
        const float k[3] = {sc0[j], sc1[j], sc2[j]};
        int fo[3], x0[3];
        bool rel = true;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const int W = g.W[a];
            x0[a] = first_tap_dev(k[a], W);
            int d = pmod(x0[a] - org[a], g.G[a]);
            if (d >= g.G[a] - (W - 1)) d -= g.G[a];
            fo[a] = d;
            rel = rel && d >= -(W - 1) && d <= rt_extent(a) - 1;
        }
        // x weights at region positions, y and z weights by tap
#pragma unroll
        for (int p = 0; p < kRtX; p++) M.qx[i][p] = 0.0f;
#pragma unroll
        for (int t = 0; t < kRtMaxW; t++) {
            if (t < g.W[0]) {
                const int p = fo[0] + t;
                if (p >= 0 && p < kRtX) M.qx[i][p] = dw * tap_weight(x0[0], t, k[0], g.W[0], g.inv_hw[0], g.beta[0]);
            }
            M.wy[i][t] = t < g.W[1] ? tap_weight(x0[1], t, k[1], g.W[1], g.inv_hw[1], g.beta[1]) : 0.0f;
            M.wz[i][t] = t < g.W[2] ? tap_weight(x0[2], t, k[2], g.W[2], g.inv_hw[2], g.beta[2]) : 0.0f;
        }
        // warp w = xw + 2 yw + 4 zw owns [4 xw, 4 xw + 4) x [4 yw, ...) x [4 zw, ...)
        unsigned m = 0;
#pragma unroll
        for (int w = 0; w < kRtWarps; w++) {
            const int o[3] = {(w & 1) * 4, ((w >> 1) & 1) * 4, (w >> 2) * 4};
            bool h = true;
#pragma unroll
            for (int a = 0; a < 3; a++) h = h && fo[a] <= o[a] + 3 && fo[a] + g.W[a] - 1 >= o[a];
            if (h) m |= 1u << w;
        }
        M.mask[i] = rel ? m : 0u;
        M.fy[i] = fo[1];
        M.fz[i] = fo[2];
        M.gi[i] = gi;
    }
}

__device__ __forceinline__ void rt_cp_async8(void *sdst, const void *gsrc)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}

// Stage the coil values of the staged samples (coil c of the block = batch
// b0 + c): asynchronous 8-byte copies for complex k-space without per-batch
// weights, plain loads otherwise. The caller waits (cp.async.wait_all).
__device__ __forceinline__ void rt_stage_values(const Geom &g, int n, int64_t b0, int64_t batch,
                                                const void *__restrict__ ksp, int kreal,
                                                const float *__restrict__ weight, int wpb,
                                                const RtMeta &M, float2 (*V)[kRtCoils + 1])
{
    const bool fast = !kreal && !(weight && wpb);
    for (int e = threadIdx.x; e < kRtCoils * kRtSB; e += blockDim.x) {
        const int c = e / kRtSB;
        const int s = e - c * kRtSB;
        if (s >= n) continue;
        const int64_t b = b0 + c;
        if (b >= batch || M.mask[s] == 0u) {
            V[s][c] = make_float2(0.0f, 0.0f);
            continue;
        }
        const int64_t o = b * g.total + M.gi[s];
        if (fast) {
            rt_cp_async8(&V[s][c], reinterpret_cast<const float2 *>(ksp) + o);
        } else {
            float2 v = kreal ? make_float2(reinterpret_cast<const float *>(ksp)[o], 0.0f)
                             : reinterpret_cast<const float2 *>(ksp)[o];
            if (weight && wpb) {
                const float w = weight[o];
                v.x *= w;
                v.y *= w;
            }
            V[s][c] = v;
        }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

__device__ __forceinline__ void rt_wait_values() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Add the taps (ty, tz) of one sample whose rows (DY + ty, DZ + tz) lie in the
// sub-region: acc[z][y][x] += wz[tz] wy[ty] px[x], px = v * qx. Row indices
// are compile-time constants.
template <int DY, int DZ, int W>
__device__ __forceinline__ void rt_add(float2 (&acc)[4][4][4], const float *wy, const float *wz,
                                       const float2 (&px)[4])
{
#pragma unroll
    for (int tz = 0; tz < W; tz++) {
        const int z = DZ + tz;
        if (z < 0 || z >= 4) continue;
        const float cz = wz[tz];
#pragma unroll
        for (int ty = 0; ty < W; ty++) {
            const int y = DY + ty;
            if (y < 0 || y >= 4) continue;
            const float c = cz * wy[ty];
#pragma unroll
            for (int x = 0; x < 4; x++) acc[z][y][x] = __ffma2_rn(rt_f2(c), px[x], acc[z][y][x]);
        }
    }
}

#define RT_OFFSETS(M) M(-7) M(-6) M(-5) M(-4) M(-3) M(-2) M(-1) M(0) M(1) M(2) M(3)

template <int DZ, int W>
__device__ __forceinline__ void rt_visit_y(float2 (&acc)[4][4][4], int dy, const float *wy, const float *wz,
                                           const float2 (&px)[4])
{
    switch (dy) {
#define RT_CASE_Y(D) \
    case D:          \
        if (D > -W) rt_add<D, DZ, W>(acc, wy, wz, px); \
        break;
        RT_OFFSETS(RT_CASE_Y)
#undef RT_CASE_Y
    default: break;
    }
}

// Visit: the offsets dy, dz in [-(W-1), 3] of the first tap from the
// sub-region origin select a branch-free body.
template <int W>
__device__ __forceinline__ void rt_visit(float2 (&acc)[4][4][4], int dy, int dz, const float *wy,
                                         const float *wz, const float2 (&px)[4])
{
    switch (dz) {
#define RT_CASE_Z(D) \
    case D:          \
        if (D > -W) rt_visit_y<D, W>(acc, dy, wy, wz, px); \
        break;
        RT_OFFSETS(RT_CASE_Z)
#undef RT_CASE_Z
    default: break;
    }
}

template <int W>
__global__ void __launch_bounds__(kRtThreads, 1) grid_rt_kernel(
    Geom g, const RtItem *__restrict__ items, const int32_t *__restrict__ bin_start,
    const float *__restrict__ sc0, const float *__restrict__ sc1, const float *__restrict__ sc2,
    const int32_t *__restrict__ sidx, const void *__restrict__ ksp, int kreal,
    float2 *__restrict__ grid, float2 *__restrict__ scratch, int64_t batch,
    const float *__restrict__ weight, int wpb, float inv_scale)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    RtShared &S = *reinterpret_cast<RtShared *>(smem_raw);
    const RtItem it = items[blockIdx.x];  // begin = part, end = nparts
    int f, org[3];
    rt_region(g, it.region, f, org);
    const int nall = rt_window_setup(g, f, org, it.begin, it.end, bin_start, S);

    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int ox = (w & 1) * 4, oy = ((w >> 1) & 1) * 4, oz = (w >> 2) * 4;
    const int64_t b0 = (int64_t)blockIdx.y * kRtCoils;
    const float *wsample = (weight && !wpb) ? weight : nullptr;

    float2 acc[4][4][4];
#pragma unroll
    for (int z = 0; z < 4; z++)
#pragma unroll
        for (int y = 0; y < 4; y++)
#pragma unroll
            for (int x = 0; x < 4; x++) acc[z][y][x] = make_float2(0.0f, 0.0f);

    // passes of at most kRtSB samples: each bin contributes ceil(share) at most
    const int npass = nall == 0 ? 0 : (nall + (kRtSB - S.nwb) - 1) / (kRtSB - S.nwb);
    if (npass > 0) {
        rt_stage_meta(g, org, rt_pass_layout(0, npass, S), sc0, sc1, sc2, sidx, wsample, S, S.meta[0]);
        __syncthreads();
        rt_stage_values(g, S.meta[0].n, b0, batch, ksp, kreal, weight, wpb, S.meta[0], S.v[0]);
        if (npass > 1)
            rt_stage_meta(g, org, rt_pass_layout(1, npass, S), sc0, sc1, sc2, sidx, wsample, S, S.meta[1]);
        rt_wait_values();
        __syncthreads();
    }
    for (int k = 0; k < npass; k++) {
        const int cur = k & 1;
        const int n = S.meta[cur].n;
        // copies of the next pass in flight during this one
        if (k + 1 < npass)
            rt_stage_values(g, S.meta[cur ^ 1].n, b0, batch, ksp, kreal, weight, wpb, S.meta[cur ^ 1],
                            S.v[cur ^ 1]);
        const RtMeta &M = S.meta[cur];
        const float2(*V)[kRtCoils + 1] = S.v[cur];
        for (int s0 = 0; s0 < n; s0 += 32) {
            const int s = s0 + lane;
            const unsigned m = s < n ? M.mask[s] : 0u;
            unsigned bits = __ballot_sync(0xffffffffu, (m >> w) & 1u);
            while (bits) {
                const int j = s0 + __ffs(bits) - 1;
                bits &= bits - 1;
                const float4 qx = *reinterpret_cast<const float4 *>(&M.qx[j][ox]);
                const float2 v = V[j][lane];
                const float2 px[4] = {__fmul2_rn(rt_f2(qx.x), v), __fmul2_rn(rt_f2(qx.y), v),
                                      __fmul2_rn(rt_f2(qx.z), v), __fmul2_rn(rt_f2(qx.w), v)};
                rt_visit<W>(acc, M.fy[j] - oy, M.fz[j] - oz, M.wy[j], M.wz[j], px);
            }
        }
        __syncthreads();  // pass k consumed: its buffers may be refilled
        if (k + 2 < npass)
            rt_stage_meta(g, org, rt_pass_layout(k + 2, npass, S), sc0, sc1, sc2, sidx, wsample, S,
                          S.meta[cur]);
        rt_wait_values();
        __syncthreads();
    }

    const int64_t b = b0 + lane;
    if (b >= batch) return;
    if (it.slot < 0) {
        float2 *gb = grid + (b * g.nframes + f) * g.gsize;
        const int px0 = org[0] + ox;
#pragma unroll
        for (int z = 0; z < 4; z++) {
            const int pz = org[2] + oz + z;
            if (pz >= g.G[2]) continue;
            const int gz = pmod(pz - g.half[2], g.G[2]);
#pragma unroll
            for (int y = 0; y < 4; y++) {
                const int py = org[1] + oy + y;
                if (py >= g.G[1]) continue;
                float2 *row = gb + ((int64_t)gz * g.G[1] + pmod(py - g.half[1], g.G[1])) * g.G[0];
#pragma unroll
                for (int x = 0; x < 4; x++) {
                    const int pxx = px0 + x;
                    if (pxx < g.G[0]) row[pmod(pxx - g.half[0], g.G[0])] = __fmul2_rn(acc[z][y][x], rt_f2(inv_scale));
                }
            }
        }
    } else {
        float2 *P = scratch + ((size_t)it.slot * gridDim.y + blockIdx.y) * kRtPts * kRtCoils;
#pragma unroll
        for (int z = 0; z < 4; z++)
#pragma unroll
            for (int y = 0; y < 4; y++)
#pragma unroll
                for (int x = 0; x < 4; x++) {
                    const int pt = ((oz + z) * kRtY + oy + y) * kRtX + ox + x;
                    P[pt * kRtCoils + lane] = acc[z][y][x];
                }
    }
}

// Sum the partial slots [begin, end) of a split region in slot order and write the grid.
__global__ void __launch_bounds__(256) grid_rt_reduce_kernel(Geom g, const RtItem *__restrict__ red,
                                                             const float2 *__restrict__ scratch,
                                                             float2 *__restrict__ grid, int64_t batch,
                                                             float inv_scale)
{
    const RtItem r = red[blockIdx.x];
    int f, org[3];
    rt_region(g, r.region, f, org);
    const int64_t b0 = (int64_t)blockIdx.y * kRtCoils;
    for (int e = threadIdx.x; e < kRtPts * kRtCoils; e += blockDim.x) {
        const int pt = e / kRtCoils;
        const int lane = e - pt * kRtCoils;
        const int64_t b = b0 + lane;
        const int x = pt % kRtX, y = (pt / kRtX) % kRtY, z = pt / (kRtX * kRtY);
        const int px = org[0] + x, py = org[1] + y, pz = org[2] + z;
        if (b >= batch || px >= g.G[0] || py >= g.G[1] || pz >= g.G[2]) continue;
        float2 s = make_float2(0.0f, 0.0f);
        for (int slot = r.begin; slot < r.end; slot++) {
            const float2 v = scratch[(((size_t)slot * gridDim.y + blockIdx.y) * kRtPts + pt) * kRtCoils + lane];
            s.x += v.x;
            s.y += v.y;
        }
        const int64_t o = (b * g.nframes + f) * g.gsize +
                          ((int64_t)pmod(pz - g.half[2], g.G[2]) * g.G[1] + pmod(py - g.half[1], g.G[1])) *
                              g.G[0] + pmod(px - g.half[0], g.G[0]);
        grid[o] = __fmul2_rn(s, rt_f2(inv_scale));
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
bool rt_geometry_ok(const Geom &g)
{
    if (g.ndim != 3) return false;
    for (int a = 0; a < 3; a++)
        if (g.G[a] < rt_extent(a) + g.W[a] - 1 || g.W[a] > kRtMaxW) return false;
    return true;
}

int rt_build(dmr_plan *p, const std::vector<int32_t> &h_start, cudaStream_t st)
{
    Geom &g = p->g;
    g.nr[0] = g.nr[1] = g.nr[2] = 0;
    g.nregions = 0;
    if (!rt_geometry_ok(g)) return DMR_OK;
    int nr[3];
    for (int a = 0; a < 3; a++) nr[a] = (int)ceil_div(g.G[a], rt_extent(a));
    // window bins: at most kRtMaxWB per axis, kRtMaxBins per region, and no bin twice
    std::vector<std::vector<int>> abins[3];
    int maxcnt[3] = {0, 0, 0};
    for (int a = 0; a < 3; a++)
        for (int r = 0; r < nr[a]; r++) {
            int bins[kRtMaxWB];
            const int n = rt_axis_bins(r * rt_extent(a), rt_extent(a), g.G[a], g.W[a], g.T[a], bins);
            if (n > kRtMaxWB) return DMR_OK;
            std::vector<int> v(bins, bins + n);
            std::vector<int> u(v);
            std::sort(u.begin(), u.end());
            if (std::unique(u.begin(), u.end()) != u.end() || u.back() >= g.nb[a]) return DMR_OK;
            abins[a].push_back(v);
            maxcnt[a] = std::max(maxcnt[a], n);
        }
    if (maxcnt[0] * maxcnt[1] * maxcnt[2] > kRtMaxBins) return DMR_OK;
    const int nregions = nr[0] * nr[1] * nr[2];
    if ((int64_t)nregions * g.nframes >= INT32_MAX / 2) return DMR_OK;

    // window sample count of every region (per frame)
    struct Reg {
        int region;
        int64_t count;
    };
    std::vector<Reg> regs;
    regs.reserve((size_t)nregions * g.nframes);
    for (int f = 0; f < g.nframes; f++) {
        for (int rz = 0; rz < nr[2]; rz++)
            for (int ry = 0; ry < nr[1]; ry++)
                for (int rx = 0; rx < nr[0]; rx++) {
                    int64_t c = 0;
                    for (int bz : abins[2][rz])
                        for (int by : abins[1][ry])
                            for (int bx : abins[0][rx]) {
                                const int key = f * g.nbins + (bz * g.nb[1] + by) * g.nb[0] + bx;
                                c += h_start[key + 1] - h_start[key];
                            }
                    regs.push_back({f * nregions + (rz * nr[1] + ry) * nr[0] + rx, c});
                }
    }
    // split regions first (heaviest first), then the others tile by tile, so
    // that the blocks running together share the bins of their windows in L2
    std::vector<RtItem> items, red;
    std::vector<Reg> heavy, light;
    for (const Reg &r : regs) (r.count > kRtChunk ? heavy : light).push_back(r);
    std::stable_sort(heavy.begin(), heavy.end(), [](const Reg &x, const Reg &y) { return x.count > y.count; });
    int slots = 0;
    for (const Reg &r : heavy) {
        const int n = (int)ceil_div(r.count, kRtChunk);
        red.push_back({r.region, slots, slots + n, 0});
        for (int k = 0; k < n; k++) items.push_back({r.region, k, n, slots + k});
        slots += n;
    }
    const int tile[3] = {4, 4, 4};  // regions per tile (x, y, z): a cube of 32 grid points
    auto tile_key = [&](int region) {
        const int f = region / nregions, lr = region % nregions;
        const int rx = lr % nr[0], ry = (lr / nr[0]) % nr[1], rz = lr / (nr[0] * nr[1]);
        const int64_t tx = rx / tile[0], ty = ry / tile[1], tz = rz / tile[2];
        const int64_t ntx = ceil_div(nr[0], tile[0]), nty = ceil_div(nr[1], tile[1]);
        return (((int64_t)f * ceil_div(nr[2], tile[2]) + tz) * nty + ty) * ntx + tx;
    };
    std::stable_sort(light.begin(), light.end(),
                     [&](const Reg &x, const Reg &y) { return tile_key(x.region) < tile_key(y.region); });
    for (const Reg &r : light) items.push_back({r.region, 0, 1, -1});

    cudaFree(p->rt_items);
    cudaFree(p->rt_reduce);
    p->rt_items = nullptr;
    p->rt_reduce = nullptr;
    DMR_CUDA(cudaMalloc(&p->rt_items, std::max<size_t>(1, items.size()) * sizeof(RtItem)));
    DMR_CUDA(cudaMalloc(&p->rt_reduce, std::max<size_t>(1, red.size()) * sizeof(RtItem)));
    DMR_CUDA(cudaMemcpyAsync(p->rt_items, items.data(), items.size() * sizeof(RtItem),
                             cudaMemcpyHostToDevice, st));
    if (!red.empty())
        DMR_CUDA(cudaMemcpyAsync(p->rt_reduce, red.data(), red.size() * sizeof(RtItem),
                                 cudaMemcpyHostToDevice, st));
    DMR_CUDA(cudaStreamSynchronize(st));
    p->nrt = (int)items.size();
    p->nrt_reduce = (int)red.size();
    p->rt_slots = slots;
    for (int a = 0; a < 3; a++) g.nr[a] = nr[a];
    g.nregions = nregions;
    return DMR_OK;
}

static bool rt_applies(const dmr_plan *p, int64_t batch)
{
    return p->g.nregions > 0 && p->nrt > 0 && batch >= kRtMinBatch && getenv("DMR_NO_RT") == nullptr;
}

size_t rt_scratch_bytes(const dmr_plan *p, int64_t batch)
{
    if (!rt_applies(p, batch) || p->rt_slots == 0) return 0;
    const int64_t ncc = ceil_div(batch, kRtCoils);
    return (size_t)p->rt_slots * ncc * kRtPts * kRtCoils * sizeof(float2);
}

// Library-owned stream-ordered pool for the scratch of calls without a
// workspace (created on first use unless `create` is false; nullptr then).
static std::mutex g_pool_mu;
static std::map<int, cudaMemPool_t> g_pools;

static cudaMemPool_t find_pool(int dev, bool create)
{
    std::lock_guard<std::mutex> lk(g_pool_mu);
    auto it = g_pools.find(dev);
    if (it != g_pools.end()) return it->second;
    if (!create) return nullptr;
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    g_pools[dev] = pool;
    return pool;
}

cudaMemPool_t scratch_pool(int dev) { return find_pool(dev, true); }

template <int W>
static int rt_launch(const dmr_plan *p, const void *ksp, int kreal, float2 *grid, int64_t batch,
                     const float *weight, int wpb, float2 *scratch, int ncc, float inv_scale, cudaStream_t st)
{
    auto kern = grid_rt_kernel<W>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(RtShared));
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute", __FILE__, __LINE__);
    kern<<<dim3(p->nrt, ncc), kRtThreads, sizeof(RtShared), st>>>(
        p->g, p->rt_items, p->bin_start, p->scoord[0], p->scoord[1], p->scoord[2], p->sidx, ksp, kreal,
        grid, scratch, batch, weight, wpb, inv_scale);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "grid_rt_kernel", __FILE__, __LINE__);
    return DMR_OK;
}

// Returns DMR_ERR_UNSUPPORTED when the register-tile kernel does not apply.
int grid_rt_dispatch(const dmr_plan *p, const void *ksp, int kreal, float2 *grid, int64_t batch,
                     const float *weight, int wpb, void *scratch, size_t scratch_bytes, cudaStream_t st)
{
    if (!rt_applies(p, batch)) return DMR_ERR_UNSUPPORTED;
    const size_t need = rt_scratch_bytes(p, batch);
    void *owned = nullptr;
    if (need > 0 && (scratch == nullptr || scratch_bytes < need)) {
        cudaMemPool_t pool = scratch_pool(p->device);
        if (!pool || cudaMallocFromPoolAsync(&owned, need, pool, st) != cudaSuccess) {
            cudaGetLastError();
            return DMR_ERR_UNSUPPORTED;
        }
        scratch = owned;
    }
    const int ncc = (int)ceil_div(batch, kRtCoils);
    const float inv_scale = (float)(1.0 / p->scale);
    float2 *sp = (float2 *)scratch;
    int rc;
    switch (p->g.W[2]) {
    case 1: rc = rt_launch<1>(p, ksp, kreal, grid, batch, weight, wpb, sp, ncc, inv_scale, st); break;
    case 2: rc = rt_launch<2>(p, ksp, kreal, grid, batch, weight, wpb, sp, ncc, inv_scale, st); break;
    case 3: rc = rt_launch<3>(p, ksp, kreal, grid, batch, weight, wpb, sp, ncc, inv_scale, st); break;
    case 4: rc = rt_launch<4>(p, ksp, kreal, grid, batch, weight, wpb, sp, ncc, inv_scale, st); break;
    case 5: rc = rt_launch<5>(p, ksp, kreal, grid, batch, weight, wpb, sp, ncc, inv_scale, st); break;
    case 6: rc = rt_launch<6>(p, ksp, kreal, grid, batch, weight, wpb, sp, ncc, inv_scale, st); break;
    case 7: rc = rt_launch<7>(p, ksp, kreal, grid, batch, weight, wpb, sp, ncc, inv_scale, st); break;
    default: rc = rt_launch<8>(p, ksp, kreal, grid, batch, weight, wpb, sp, ncc, inv_scale, st); break;
    }
    if (rc == DMR_OK && p->nrt_reduce > 0) {
        grid_rt_reduce_kernel<<<dim3(p->nrt_reduce, ncc), 256, 0, st>>>(p->g, p->rt_reduce,
                                                                        (const float2 *)scratch, grid,
                                                                        batch, inv_scale);
        g_launches.fetch_add(1, std::memory_order_relaxed);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_fail(e, "grid_rt_reduce_kernel", __FILE__, __LINE__);
    }
    if (owned) cudaFreeAsync(owned, st);
    return rc;
}

}  // namespace dmr

// Return the scratch pool's free memory on `device` to the device.
extern "C" int dmr_scratch_release(int device)
{
    cudaMemPool_t pool = dmr::find_pool(device, false);
    if (!pool) return DMR_OK;
    int old = 0;
    DMR_CUDA(cudaGetDevice(&old));
    DMR_CUDA(cudaSetDevice(device));
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemPoolTrimTo(pool, 0);
    cudaSetDevice(old);
    if (e != cudaSuccess) return dmr::cuda_fail(e, "dmr_scratch_release", __FILE__, __LINE__);
    return DMR_OK;
}
