// Tensor-core gridding for 3D with the spreading matrix in tensor memory.
//
// Reference: apply_gridding and its 3D kernel
// (src/deepmr/fft/_interp/grid.py:14-125, 253-284):
//   grid[f, b, iz, iy, ix] += value_z * value_y * value_x * y[f, b, p]   (then / scale)
//
// As in tcgrid.cu, what one bin's samples add to its tile + halo (P points,
// P <= 384) for a chunk of up to 32 coils is the matrix product
//     D[p, n] = sum_s A[p, s] B[n, s]
// (A: spreading weights wx * wy * wz of sample s at point p, B: real and
// imaginary parts of the coil values), computed by tcgen05 TF32 MMAs with a
// three-term hi / lo split for float32 accuracy (hi*hi + hi*lo + lo*hi). Here
// the operand A is written by the threads straight into tensor memory
// (tcgen05.st; one thread per region point, eight samples per MMA), which the
// MMA reads as its A operand, so A never passes through shared memory; only
// B (64 x 16 floats per chunk) does.
//
// Roles (one block per SM, warp-specialised, all hand-offs through mbarriers):
//  - warps 0-11, builders: per 8-sample chunk, the A operand of their point in
//    one of the (up to 3) 128-point tiles and the B operand (one (coil, sample)
//    pair per thread); per finished work item, the accumulator read-back
//    (tcgen05.ld) and the float2 atomics into the grid;
//  - warp 12, one thread: the MMAs and tcgen05.commit;
//  - warps 13-16: per-axis Kaiser-Bessel weight vectors of each 128-sample
//    pass (one sample per thread);
//  - warp 17: cp.async of each pass's coil values (and density weights).
// Passes go through a ring of 3 shared-memory slots, operands through 2
// stages (A in tensor memory, B in shared memory), and each work item's
// accumulator alternates between two tensor-memory buffers, so the read-back
// of one item overlaps the MMAs of the next.
//
// Samples are visited in acquisition order within each bin (the plan's
// acq_sidx / acq_scoord), so consecutive samples of a spoke, which share
// 32-byte sectors of k-space, are read together.
//
// Every wait is bounded in global time; a wait that runs out sets a block-wide
// abort flag that makes every role leave its loop, the MMA thread waits
// (bounded) for its last MMAs, and the block frees its tensor memory and
// counts itself in the plan's status word (dmr_plan_status).
#include <algorithm>
#include <cstdint>

#include "kb.cuh"
#include "plan.cuh"
#include "tcgen05.cuh"

namespace dmr {

namespace {

constexpr int kTmBuilders = 384;           // 12 warps: 3 tiles x 4 lane quarters
constexpr int kTmMmaWarp = 12;
constexpr int kTmWeightWarp = 13;          // warps 13-16: one sample of the pass per thread
constexpr int kTmValueWarp = 17;
constexpr int kTmThreads = 18 * 32;
constexpr int kTmPassArrivals = 128 + 32 + 1;  // weight threads, value lanes (cp.async), meta
constexpr int kTmSC = 8;                   // samples per chunk (K of one tf32 MMA)
constexpr int kTmSB = 128;                 // samples per pass
constexpr int kTmSBP = kTmSB + 4;          // padded row (bank spread)
constexpr int kTmSlots = 3;                // pass ring
constexpr int kTmMaxMT = 3;                // 128-point tiles
constexpr int kTmMaxCC = 32;               // coils per block
constexpr uint64_t kTmWaitNs = 200000000ull;    // bound on a hand-off wait (200 ms)
constexpr uint64_t kTmDrainNs = 2000000000ull;  // bound on the wait for the last MMAs (2 s)
constexpr uint64_t kTmStallNs = 1000000ull;     // test stall (1 ms)

// pass metadata flags (slot meta[1]) and chunk flags for the MMA thread
constexpr int kPassFirst = 1, kPassLast = 2, kPassEnd = 4;
constexpr uint32_t kChunkFirst = 1, kChunkLast = 2, kChunkAcc = 4, kChunkEnd = 8;

// barriers: pass full / empty per slot, operand full / empty per stage,
// accumulator full / empty per buffer, final commit, never signalled (test)
enum { kBarPassFull = 0, kBarPassEmpty = 3, kBarAbFull = 6, kBarAbEmpty = 8, kBarAccFull = 10,
       kBarAccEmpty = 12, kBarFinal = 14, kBarNever = 15, kBarCount = 16 };

struct TmShape {
    int R[3];        // region extents (T + W - 1)
    int P;           // region points
    int MT;          // 128-point tiles
    int N;           // accumulator columns per tile (2 x coils, multiple of 16)
    int CC;          // coils per block
    int ncols;       // tensor-memory columns allocated
    int acol;        // first column of the A stages (after the two accumulators)
    int vrows;       // R[0] + R[1] + R[2]
    int slot_bytes;  // one pass slot
    int vals_off;    // offsets inside a slot: coil values, density weights, meta
    int wts_off;
    int meta_off;
    int bst_bytes;   // one B stage
};

__device__ __forceinline__ uint32_t bar_addr(uint64_t *bars, int i) { return tc_smem(&bars[i]); }

__device__ __forceinline__ void bar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// bounded wait for completion number k of an mbarrier; gives up (and raises the
// block's abort flag) after limit_ns, or as soon as another role raised it
__device__ __forceinline__ bool tm_wait(uint32_t bar, uint32_t k, uint64_t limit_ns, volatile int *abort)
{
    for (int i = 0; i < 64; i++)
        if (tc_try_wait(bar, k & 1)) return true;
    const uint64_t t0 = tc_now();
    for (;;) {
        for (int i = 0; i < 256; i++)
            if (tc_try_wait(bar, k & 1)) return true;
        if (*abort) return false;
        if (tc_now() - t0 > limit_ns) {
            *abort = 1;
            return false;
        }
    }
}

// tm_wait for all 32 lanes of a warp with a warp-uniform result (the callers
// go on to .sync.aligned tcgen05 instructions)
__device__ __forceinline__ bool tm_wait_warp(uint32_t bar, uint32_t k, uint64_t limit_ns, volatile int *abort)
{
    return __all_sync(0xffffffffu, tm_wait(bar, k, limit_ns, abort));
}

__device__ __forceinline__ void tm_st16(uint32_t taddr, const float (&v)[16])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
            taddr),
        "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]), "f"(v[8]), "f"(v[9]),
        "f"(v[10]), "f"(v[11]), "f"(v[12]), "f"(v[13]), "f"(v[14]), "f"(v[15])
        : "memory");
}

__device__ __forceinline__ void tm_mma(uint32_t d, uint32_t a, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(d),
        "r"(a), "l"(bdesc), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void tm_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// the pass sequence of a block: work items (bin, sample range) x coil chunks,
// tasks blockIdx.x, blockIdx.x + gridDim.x, ..., each cut into 128-sample passes
struct PassSeq {
    int task, ntasks, nchunks, base;
    WorkItem it;
    __device__ void start(const WorkItem *work, const int32_t *order, int nwork, int nch)
    {
        nchunks = nch;
        ntasks = nwork * nch;
        task = blockIdx.x;
        if (task < ntasks) {
            it = work[order[task / nchunks]];
            base = it.begin;
        }
    }
    __device__ bool done() const { return task >= ntasks; }
    __device__ void next(const WorkItem *work, const int32_t *order)
    {
        base += kTmSB;
        if (base >= it.end) {
            task += gridDim.x;
            if (task < ntasks) {
                it = work[order[task / nchunks]];
                base = it.begin;
            }
        }
    }
};

__global__ void __launch_bounds__(kTmThreads, 1) grid_tmem_kernel(
    Geom g, TmShape sh, const WorkItem *__restrict__ work, const int32_t *__restrict__ order, int nwork,
    int nchunks, const float *__restrict__ sc0, const float *__restrict__ sc1, const float *__restrict__ sc2,
    const int32_t *__restrict__ sidx, const void *__restrict__ ksp, int kreal, float2 *__restrict__ grid,
    int64_t batch, const float *__restrict__ weight, int wpb, float inv_scale, int *__restrict__ status,
    int *__restrict__ timeouts, int stall)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[kBarCount];
    __shared__ uint32_t tslot;
    __shared__ volatile int s_abort;
    __shared__ uint32_t stage_meta[2];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int W = g.W[0];
    unsigned char *bst = smem;                              // B stages
    unsigned char *slots = smem + 2 * sh.bst_bytes;          // pass ring

    // B stages start zeroed: rows of absent coils (N > 2 x coils) stay zero
    for (int e = tid; e < 2 * sh.bst_bytes / 16; e += kTmThreads)
        reinterpret_cast<float4 *>(bst)[e] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem(&tslot)),
                     "r"(sh.ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        const int counts[kBarCount] = {kTmPassArrivals, kTmPassArrivals, kTmPassArrivals, kTmBuilders, kTmBuilders,
                                       kTmBuilders, kTmBuilders, kTmBuilders, 1, 1, 1, 1, kTmBuilders, kTmBuilders,
                                       1, 1};
        for (int i = 0; i < kBarCount; i++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_addr(bars, i)), "r"(counts[i]));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tbase = tslot;
    const int RXY = sh.R[0] * sh.R[1];
    bool mma_issued = false;

    if (warp < kTmMmaWarp) {
        // ------------------------------------------------------------------ builders
        const int tile = warp >> 2, quarter = warp & 3;
        const bool has_tile = tile < sh.MT;  // warp-uniform
        const int p = tile * 128 + quarter * 32 + lane;
        const int pc = min(p, sh.P - 1);
        const int rz = pc / RXY, rem = pc - rz * RXY;
        const int ry = rem / sh.R[0], rx = rem - ry * sh.R[0];
        const uint32_t vx = (uint32_t)rx * kTmSBP * 4, vy = (uint32_t)(sh.R[0] + ry) * kTmSBP * 4,
                       vz = (uint32_t)(sh.R[0] + sh.R[1] + rz) * kTmSBP * 4;
        const uint32_t lanebase = (uint32_t)(quarter * 32) << 16;
        const int bc = tid >> 3, bs = tid & 7;  // B operand: coil and sample of this thread
        // B rows 2c (real) and 2c + 1 (imaginary) of coil bc; K: hi at s, lo at 8 + s
        const uint32_t boff = (uint32_t)(((2 * bc) >> 3) * kTcRowBytes + ((2 * bc) & 7) * 16 + (bs >> 2) * 128 +
                                         (bs & 3) * 4);
        uint32_t chunk_no = 0;
        int task_no = 0, drains[2] = {0, 0};
        // current and pending (finished, not yet read back) work items
        int cur_org[3] = {0, 0, 0}, cur_f = 0, cur_cact = 0;
        int64_t cur_b0 = 0;
        bool pend = false;
        int pend_org[3] = {0, 0, 0}, pend_f = 0, pend_cact = 0, pend_acc = 0, pend_since = 0;
        int64_t pend_b0 = 0;

        // read back the accumulator of the pending item and add it to the grid
        auto drain = [&]() -> bool {
            if (!tm_wait_warp(bar_addr(bars, kBarAccFull + pend_acc), drains[pend_acc], kTmWaitNs, &s_abort))
                return false;
            drains[pend_acc]++;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (has_tile) {
                int64_t gp = -1;
                if (p < sh.P) {
                    const int qx = (pend_org[0] + rx + g.G[0] - g.half[0]) % g.G[0];
                    const int qy = (pend_org[1] + ry + g.G[1] - g.half[1]) % g.G[1];
                    const int qz = (pend_org[2] + rz + g.G[2] - g.half[2]) % g.G[2];
                    gp = ((int64_t)qz * g.G[1] + qy) * g.G[0] + qx;
                }
                const uint32_t acc0 = tbase + lanebase + (uint32_t)((pend_acc * sh.MT + tile) * sh.N);
                for (int c0 = 0; c0 < sh.N; c0 += 16) {
                    uint32_t r[16];
                    tc_ld16(acc0 + (uint32_t)c0, r);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    if (gp >= 0) {
#pragma unroll
                        for (int i = 0; i < 8; i++) {
                            const int c = c0 / 2 + i;
                            const float2 v = make_float2(__uint_as_float(r[2 * i]) * inv_scale,
                                                         __uint_as_float(r[2 * i + 1]) * inv_scale);
                            if (c < pend_cact && (v.x != 0.0f || v.y != 0.0f))
                                atomicAdd(grid + ((pend_b0 + c) * g.nframes + pend_f) * g.gsize + gp, v);
                        }
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            bar_arrive(bar_addr(bars, kBarAccEmpty + pend_acc));
            pend = false;
            return true;
        };

        bool ok = true;
        for (uint32_t pass_no = 0; ok; pass_no++) {
            const int slot = pass_no % kTmSlots;
            if (!tm_wait_warp(bar_addr(bars, kBarPassFull + slot), pass_no / kTmSlots, kTmWaitNs, &s_abort)) {
                ok = false;
                break;
            }
            unsigned char *sl = slots + slot * sh.slot_bytes;
            const int *meta = reinterpret_cast<const int *>(sl + sh.meta_off);
            const int flags = meta[1];
            if (flags & kPassEnd) break;
            const int n = meta[2];
            if (flags & kPassFirst) {
                const int bin = meta[0];
                cur_f = bin / g.nbins;
                const int lb = bin - cur_f * g.nbins;
                cur_org[0] = (lb % g.nb[0]) * g.T[0];
                cur_org[1] = ((lb / g.nb[0]) % g.nb[1]) * g.T[1];
                cur_org[2] = (lb / (g.nb[0] * g.nb[1])) * g.T[2];
                cur_b0 = (int64_t)meta[3];
                cur_cact = meta[4];
            }
            const uint32_t vbase = tc_smem(sl);
            const float2 *vals = reinterpret_cast<const float2 *>(sl + sh.vals_off);
            const float *wts = reinterpret_cast<const float *>(sl + sh.wts_off);
            const int nch = (n + kTmSC - 1) / kTmSC;
            for (int ch = 0; ch < nch; ch++) {
                const int stage = chunk_no & 1;
                if (chunk_no >= 2 &&
                    !tm_wait_warp(bar_addr(bars, kBarAbEmpty + stage), (chunk_no >> 1) - 1, kTmWaitNs, &s_abort)) {
                    ok = false;
                    break;
                }
                // test hook: a barrier that nothing signals, so the wait runs out
                if (stall && chunk_no >= 2 && !tm_wait_warp(bar_addr(bars, kBarNever), 0, kTmStallNs, &s_abort)) {
                    ok = false;
                    break;
                }
                const bool first = (flags & kPassFirst) && ch == 0;
                const bool last = (flags & kPassLast) && ch == nch - 1;
                // A: weights of this thread's point for the chunk's 8 samples, hi | lo
                if (has_tile) {
                    const uint32_t so = (uint32_t)(ch * kTmSC) * 4;
                    const float4 x0 = tc_lds4(vbase + vx + so), x1 = tc_lds4(vbase + vx + so + 16);
                    const float4 y0 = tc_lds4(vbase + vy + so), y1 = tc_lds4(vbase + vy + so + 16);
                    const float4 z0 = tc_lds4(vbase + vz + so), z1 = tc_lds4(vbase + vz + so + 16);
                    const float w[8] = {x0.x * y0.x * z0.x, x0.y * y0.y * z0.y, x0.z * y0.z * z0.z,
                                        x0.w * y0.w * z0.w, x1.x * y1.x * z1.x, x1.y * y1.y * z1.y,
                                        x1.z * y1.z * z1.z, x1.w * y1.w * z1.w};
                    float v[16];
#pragma unroll
                    for (int s = 0; s < 8; s++) {
                        v[s] = tc_hi(w[s]);
                        v[8 + s] = w[s] - v[s];
                    }
                    tm_st16(tbase + lanebase + (uint32_t)(sh.acol + (stage * sh.MT + tile) * 16), v);
                }
                // B: coil bc, sample bs of the chunk (zero for absent coils / samples)
                if (bc < sh.CC) {
                    const int s = ch * kTmSC + bs;
                    float2 v = make_float2(0.0f, 0.0f);
                    if (bc < cur_cact && s < n) {
                        v = vals[bc * kTmSBP + s];
                        if (kreal) v.y = 0.0f;
                        if (weight) {
                            const float wt = wts[(wpb ? bc * kTmSBP : 0) + s];
                            v.x *= wt;
                            v.y *= wt;
                        }
                    }
                    unsigned char *b = bst + stage * sh.bst_bytes + boff;
                    const float hx = tc_hi(v.x), hy = tc_hi(v.y);
                    *reinterpret_cast<float *>(b) = hx;
                    *reinterpret_cast<float *>(b + 256) = v.x - hx;
                    *reinterpret_cast<float *>(b + 16) = hy;
                    *reinterpret_cast<float *>(b + 16 + 256) = v.y - hy;
                }
                if (tid == 0)
                    stage_meta[stage] = (first ? kChunkFirst : 0u) | (last ? kChunkLast : 0u) |
                                        ((task_no & 1) ? kChunkAcc : 0u);
                if (has_tile) asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                bar_arrive(bar_addr(bars, kBarAbFull + stage));
                chunk_no++;
                if (last) {
                    // the item is complete: read back the previous one, keep this one pending
                    if (pend && !drain()) {
                        ok = false;
                        break;
                    }
                    pend = true;
                    pend_acc = task_no & 1;
                    pend_since = 0;
                    pend_f = cur_f;
                    pend_b0 = cur_b0;
                    pend_cact = cur_cact;
                    for (int a = 0; a < 3; a++) pend_org[a] = cur_org[a];
                    task_no++;
                } else if (pend && ++pend_since >= 2) {
                    // two chunks of the next item are queued: read back meanwhile
                    if (!drain()) {
                        ok = false;
                        break;
                    }
                }
            }
            if (!ok) break;
            bar_arrive(bar_addr(bars, kBarPassEmpty + slot));
        }
        if (ok) {
            // end marker for the MMA thread, then the last read-back
            const int stage = chunk_no & 1;
            if (chunk_no < 2 ||
                tm_wait_warp(bar_addr(bars, kBarAbEmpty + stage), (chunk_no >> 1) - 1, kTmWaitNs, &s_abort)) {
                if (tid == 0) stage_meta[stage] = kChunkEnd;
                bar_arrive(bar_addr(bars, kBarAbFull + stage));
                if (pend) drain();
            }
        }
    } else if (warp == kTmMmaWarp) {
        // ------------------------------------------------------------------ MMA issue
        if (lane == 0) {
            // D f32, A / B tf32, both K-major, N, M = 128
            const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(sh.N >> 3) << 17) | (8u << 24);
            const uint64_t bdesc0 = tc_desc(tc_smem(bst));
            int acc_uses[2] = {0, 0};
            for (uint32_t chunk = 0;; chunk++) {
                const int stage = chunk & 1;
                if (!tm_wait(bar_addr(bars, kBarAbFull + stage), chunk >> 1, kTmWaitNs, &s_abort)) break;
                const uint32_t m = stage_meta[stage];
                if (m & kChunkEnd) break;
                const int acc = (m & kChunkAcc) ? 1 : 0;
                if ((m & kChunkFirst) && acc_uses[acc] > 0 &&
                    !tm_wait(bar_addr(bars, kBarAccEmpty + acc), acc_uses[acc] - 1, kTmWaitNs, &s_abort))
                    break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint64_t bh = bdesc0 + (uint64_t)((stage * sh.bst_bytes) >> 4), bl = bh + (256 >> 4);
                for (int t = 0; t < sh.MT; t++) {
                    const uint32_t d = tbase + (uint32_t)((acc * sh.MT + t) * sh.N);
                    const uint32_t ah = tbase + (uint32_t)(sh.acol + (stage * sh.MT + t) * 16), al = ah + 8;
                    tm_mma(d, ah, bh, idesc, (m & kChunkFirst) ? 0u : 1u);  // hi * hi
                    tm_mma(d, ah, bl, idesc, 1u);                            // hi * lo
                    tm_mma(d, al, bh, idesc, 1u);                            // lo * hi
                }
                mma_issued = true;
                tm_commit(bar_addr(bars, kBarAbEmpty + stage));
                if (m & kChunkLast) {
                    tm_commit(bar_addr(bars, kBarAccFull + acc));
                    acc_uses[acc]++;
                }
            }
        }
    } else {
        // ------------------------------------------------------------------ producers
        const bool wprod = warp < kTmValueWarp;
        const int wst = tid - kTmWeightWarp * 32;  // weight producers: sample of the pass
        PassSeq ps;
        ps.start(work, order, nwork, nchunks);
        // per-pass global inputs of this thread, loaded one pass ahead: the
        // coordinates of its sample (weight producers) or the sample indices of
        // its four samples (value producer)
        float kv[3] = {0.0f, 0.0f, 0.0f};
        int gi[4] = {-1, -1, -1, -1};
        auto load = [&](const PassSeq &q) {
            if (q.done()) return;
            const int nq = min(kTmSB, q.it.end - q.base);
            if (wprod) {
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    const float *sc = a == 0 ? sc0 : (a == 1 ? sc1 : sc2);
                    kv[a] = wst < nq ? sc[q.base + wst] : 0.0f;
                }
            } else {
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int st = lane + 32 * j;
                    gi[j] = st < nq ? sidx[q.base + st] : -1;
                }
            }
        };
        load(ps);
        for (uint32_t pass_no = 0;; pass_no++) {
            const int slot = pass_no % kTmSlots;
            if (pass_no >= kTmSlots &&
                !tm_wait_warp(bar_addr(bars, kBarPassEmpty + slot), pass_no / kTmSlots - 1, kTmWaitNs, &s_abort))
                break;
            unsigned char *sl = slots + slot * sh.slot_bytes;
            const uint32_t full = bar_addr(bars, kBarPassFull + slot);
            if (ps.done()) {
                // end marker
                if (wprod) {
                    bar_arrive(full);
                } else {
                    if (lane == 0) reinterpret_cast<int *>(sl + sh.meta_off)[1] = kPassEnd;
                    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(full) : "memory");
                    if (lane == 0) bar_arrive(full);
                }
                break;
            }
            const WorkItem it = ps.it;
            const int base = ps.base;
            const int n = min(kTmSB, it.end - base);
            const int64_t b0 = (int64_t)(ps.task % nchunks) * sh.CC;
            const int cact = (int)(batch - b0 < (int64_t)sh.CC ? batch - b0 : (int64_t)sh.CC);
            if (wprod) {
                // per-axis weight vectors over the region rows (zero off the support)
                const int f = it.bin / g.nbins, lb = it.bin - f * g.nbins;
                const int org[3] = {(lb % g.nb[0]) * g.T[0], ((lb / g.nb[0]) % g.nb[1]) * g.T[1],
                                    (lb / (g.nb[0] * g.nb[1])) * g.T[2]};
                const bool live = wst < n;
                float *vec = reinterpret_cast<float *>(sl);
                int row0 = 0;
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    int x0 = 0, l = -1000;
                    if (live) {
                        x0 = first_tap_dev(kv[a], W);
                        l = pmod(x0, g.G[a]) - org[a];  // in [0, T): the sample lies in this bin
                    }
                    for (int r = 0; r < sh.R[a]; r++) {
                        const int i = r - l;
                        vec[(row0 + r) * kTmSBP + wst] =
                            (i >= 0 && i < W) ? tap_weight(x0, i, kv[a], W, g.inv_hw[a], g.beta[a]) : 0.0f;
                    }
                    row0 += sh.R[a];
                }
                bar_arrive(full);
            } else {
                // coil values (and density weights) of the pass, cp.async
                if (lane == 0) {
                    int *meta = reinterpret_cast<int *>(sl + sh.meta_off);
                    meta[0] = it.bin;
                    meta[1] = (base == it.begin ? kPassFirst : 0) | (base + kTmSB >= it.end ? kPassLast : 0);
                    meta[2] = n;
                    meta[3] = (int)b0;
                    meta[4] = cact;
                }
                const uint32_t vdst = tc_smem(sl + sh.vals_off), wdst = tc_smem(sl + sh.wts_off);
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int st = lane + 32 * j;
                    if (gi[j] < 0) continue;
                    for (int c = 0; c < cact; c++) {
                        const int64_t e = (b0 + c) * g.total + gi[j];
                        const uint32_t d = vdst + (uint32_t)(c * kTmSBP + st) * 8;
                        if (kreal)
                            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d),
                                         "l"(reinterpret_cast<const float *>(ksp) + e)
                                         : "memory");
                        else
                            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d),
                                         "l"(reinterpret_cast<const float2 *>(ksp) + e)
                                         : "memory");
                    }
                    if (weight) {
                        if (wpb) {
                            for (int c = 0; c < cact; c++)
                                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                                                 wdst + (uint32_t)(c * kTmSBP + st) * 4),
                                             "l"(weight + (b0 + c) * g.total + gi[j])
                                             : "memory");
                        } else {
                            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(wdst + (uint32_t)st * 4),
                                         "l"(weight + gi[j])
                                         : "memory");
                        }
                    }
                }
                asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(full) : "memory");
                if (lane == 0) bar_arrive(full);
            }
            ps.next(work, order);
            load(ps);
        }
        if (!wprod) asm volatile("cp.async.wait_all;" ::: "memory");
    }

    // teardown: no MMA may still write tensor memory when it is freed
    if (warp == kTmMmaWarp && lane == 0 && mma_issued) {
        tm_commit(bar_addr(bars, kBarFinal));
        if (!tc_wait(bar_addr(bars, kBarFinal), 0, kTmDrainNs)) s_abort = 1;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(sh.ncols));
    if (tid == 0 && s_abort) {
        atomicAdd(timeouts, 1);
        atomicAdd(status, 1);
    }
}

bool tm_shape(const Geom &g, int64_t batch, int wpb, TmShape &s)
{
    if (g.ndim != 3 || batch < 1) return false;
    const int W = g.W[0];
    if (W < 2 || g.W[1] != W || g.W[2] != W) return false;
    for (int a = 0; a < 3; a++) s.R[a] = g.T[a] + W - 1;
    s.P = s.R[0] * s.R[1] * s.R[2];
    s.MT = (s.P + 127) / 128;
    if (s.MT > kTmMaxMT) return false;
    s.vrows = s.R[0] + s.R[1] + s.R[2];
    s.CC = (int)std::min<int64_t>(batch, kTmMaxCC);
    s.N = std::max(16, (2 * s.CC + 15) / 16 * 16);
    s.acol = 2 * s.MT * s.N;
    const int need = s.acol + 2 * s.MT * 16;
    s.ncols = 32;
    while (s.ncols < need) s.ncols <<= 1;
    if (s.ncols > 512) return false;
    s.bst_bytes = s.N * 64;
    int off = s.vrows * kTmSBP * 4;
    off = (off + 15) / 16 * 16;
    s.vals_off = off;
    off += s.CC * kTmSBP * 8;
    s.wts_off = off;
    off += (wpb ? s.CC : 1) * kTmSBP * 4;
    off = (off + 15) / 16 * 16;
    s.meta_off = off;
    off += 32;
    s.slot_bytes = (off + 127) / 128 * 128;
    return true;
}

}  // namespace

// Tensor-core gridding with the spreading operand in tensor memory;
// DMR_ERR_UNSUPPORTED when the geometry does not fit (the caller then uses
// the shared-memory-operand kernel of tcgrid.cu).
int grid_tm_dispatch(const dmr_plan *p, const void *ksp, int kreal, float2 *grid, int64_t batch,
                     const float *weight, int wpb, int *timeouts, int stall, cudaStream_t st)
{
    TmShape sh;
    if (!tm_shape(p->g, batch, wpb, sh)) return DMR_ERR_UNSUPPORTED;
    int dev = 0, sms = 0, smem_sm = 0, smem_blk = 0, reserved = 0;
    DMR_CUDA(cudaGetDevice(&dev));
    DMR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    DMR_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    DMR_CUDA(cudaDeviceGetAttribute(&smem_blk, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    DMR_CUDA(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev));
    size_t smem = (size_t)2 * sh.bst_bytes + (size_t)kTmSlots * sh.slot_bytes;
    if (smem > (size_t)smem_blk) return DMR_ERR_UNSUPPORTED;
    {
        // the dynamic maximum leaves room for the kernel's static shared memory
        cudaFuncAttributes fa;
        DMR_CUDA(cudaFuncGetAttributes(&fa, grid_tmem_kernel));
        smem_blk -= (int)fa.sharedSizeBytes;
        if (smem > (size_t)smem_blk) return DMR_ERR_UNSUPPORTED;
        DMR_CUDA(cudaFuncSetAttribute(grid_tmem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_blk));
    }
    // (set back to the size launched below: a larger maximum can make the
    // driver reserve more shared memory and leave less L1 cache)
    // co-resident blocks must not ask for more than the SM's 512 tensor-memory
    // columns: pad the shared memory until at most 512 / ncols blocks fit
    const int maxb = 512 / sh.ncols;
    int per_sm = 0;
    DMR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grid_tmem_kernel, kTmThreads, smem));
    if (per_sm > maxb) {
        const size_t fit = (size_t)smem_sm / (maxb + 1);
        if (fit > (size_t)reserved) smem = std::max(smem, fit - (size_t)reserved);
        DMR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grid_tmem_kernel, kTmThreads, smem));
        while (per_sm > maxb && smem + 1024 <= (size_t)smem_blk) {
            smem += 1024;
            DMR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grid_tmem_kernel, kTmThreads, smem));
        }
        if (per_sm > maxb) return DMR_ERR_UNSUPPORTED;
    }
    if (per_sm < 1) return DMR_ERR_UNSUPPORTED;
    DMR_CUDA(cudaFuncSetAttribute(grid_tmem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    DMR_CUDA(cudaMemsetAsync(grid, 0, (size_t)batch * p->g.nframes * p->g.gsize * sizeof(float2), st));
    if (p->nwork == 0) return DMR_OK;
    const int64_t nchunks = ceil_div(batch, sh.CC);
    const int64_t tasks = (int64_t)p->nwork * nchunks;
    DMR_CHECK(tasks < (1ll << 31), DMR_ERR_UNSUPPORTED, "too many gridding tasks");
    DMR_CHECK(nchunks * sh.CC < (1ll << 31), DMR_ERR_UNSUPPORTED, "batch too large");
    const int blocks = (int)std::min<int64_t>(tasks, (int64_t)sms * per_sm);
    grid_tmem_kernel<<<blocks, kTmThreads, smem, st>>>(
        p->g, sh, p->work, p->work_order, p->nwork, (int)nchunks, p->acq_scoord[0], p->acq_scoord[1],
        p->acq_scoord[2], p->acq_sidx, ksp, kreal, grid, batch, weight, wpb, (float)(1.0 / p->scale), p->status,
        timeouts, stall);
    DMR_LAUNCHED("grid_tmem_kernel");
    return DMR_OK;
}

}  // namespace dmr
