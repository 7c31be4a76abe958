// Tensor-core gridding for 3D: coil values x spreading weights, one N = 256
// MMA per term.
//
// Reference: apply_gridding and its 3D kernel
// (src/deepmr/fft/_interp/grid.py:14-125, 253-284):
//   grid[f, b, iz, iy, ix] += value_z * value_y * value_x * y[f, b, p]   (then / scale)
//
// What the samples of one bin add to its region (the bin's tile + the kernel
// halo, at most 7 x 6 x 6 = 252 points for the plan's gridding bins) for a
// chunk of up to 32 coils is a matrix product over the samples s:
//     D[r, p] = sum_s V[r, s] Wt[p, s]
// with V the coil values (row r < 64: tf32 "hi" part of coil component r,
// r = 2c + {0 real, 1 imaginary}; row 64 + r: the "lo" remainder) and Wt the
// spreading weights wx * wy * wz of sample s at region point p, split into
// hi and lo as well. Two tcgen05 TF32 MMAs per 8-sample chunk (M = 128
// value rows, N = 256 points, K = 8 samples), one with Wt_hi and one with
// Wt_lo, accumulate all four products hi*hi + hi*lo + lo*hi + lo*lo in tensor
// memory; the coil component's value at point p is D[r, p] + D[64 + r, p].
// (A tcgen05.mma of M = 128, K = 8 takes about the same time on the tensor
// core for any N up to 256, so the points go on N and a chunk costs two MMAs.)
//
// Precision: hi is x with the 13 mantissa bits that tf32 drops cleared, lo =
// x - hi; the tensor core reads lo to tf32 as well, so each product keeps a
// relative error of about 2^-21, and the accumulation is float32.
//
// Roles (one block per SM, warp-specialised, hand-offs through mbarriers):
//  - warps 0-7, builders, two groups of four warps building alternate chunks
//    (so consecutive chunks are built at the same time): per chunk, the
//    per-axis Kaiser-Bessel weights of its 8 samples placed on the region
//    rows (a table of about one entry per thread, from the plan's per-sample
//    tap weights), then the weight operand (two region points per thread:
//    8 samples, hi and lo) and the value operand (two (coil, sample) pairs per
//    thread) in shared memory, in a ring of operand stages;
//  - warps 8-15, read-back: per finished work item, the accumulator
//    (tcgen05.ld; lane quarter = warp mod 4, two warps per quarter), transposed
//    through shared memory to (point, coil) order, hi + lo rows summed, one
//    float2 atomic per point and coil into the grid (32 neighbouring points
//    per instruction, 8 warps issuing);
//  - warp 16, one thread: the two MMAs per chunk and tcgen05.commit;
//  - warp 17: cp.async of each 128-sample pass's tap weights and offsets
//    (the plan's), coil values (and density weights).
// Passes go through a ring of shared-memory slots; each work item's
// accumulator alternates between the two 256-column halves of tensor memory,
// so the read-back of one item overlaps the MMAs of the next.
//
// Every wait is bounded in global time; a wait that runs out raises a
// block-wide abort flag that makes every role leave its loop; the MMA thread
// waits (bounded) for its last MMAs, and the block frees its tensor memory and
// counts itself in the plan's status word (dmr_plan_status).
#include <algorithm>
#include <cstdint>

#include "kb.cuh"
#include "plan.cuh"
#include "tcgen05.cuh"

namespace dmr {

namespace {

#ifndef DMR_TM_BUILDER_GROUPS
#define DMR_TM_BUILDER_GROUPS 3
#endif
constexpr int kTmGroups = DMR_TM_BUILDER_GROUPS;  // builder groups of 128 threads, chunks in turn
constexpr int kTmGroup = 128;
constexpr int kTmBuilders = kTmGroups * kTmGroup;  // warps 0 .. 4 groups - 1
constexpr int kTmEpiWarp = 4 * kTmGroups;          // 8 read-back warps (two per tensor-memory lane quarter)
constexpr int kTmMmaWarp = kTmEpiWarp + 8;
constexpr int kTmValueWarp = kTmMmaWarp + 1;
constexpr int kTmThreads = (kTmValueWarp + 1) * 32;
constexpr int kTmEpi = 256;
constexpr int kTmMaxRows = 24;             // region rows over the three axes (7 + 6 + 6 = 19 used)
// a chunk's weight table: rows of 8 samples, 12 floats apart (48 bytes: the
// 16-byte reads of up to 8 consecutive rows fall on disjoint banks)
constexpr int kTmTableRow = 12;
constexpr int kTmTable = kTmMaxRows * kTmTableRow;
constexpr int kTmSC = 8;                   // samples per chunk (K of one tf32 MMA)
constexpr int kTmSB = 128;                 // samples per pass
// samples accumulated in tensor memory before a read-back: the fp32 sums of
// the MMA lose accuracy over long chains, so a longer work item is read back
// in segments of this many samples (a multiple of kTmSB)
constexpr int kTmSeg = kTgSegment;
static_assert(kTmSeg % kTmSB == 0, "segments of whole passes");
constexpr int kTmSBP = kTmSB + 4;          // padded row (bank spread)
constexpr int kTmMaxSlots = 3;             // pass ring
constexpr int kTmMaxStages = 4;            // operand stages
constexpr int kTmN = 256;                  // MMA N (region points, padded)
constexpr int kTmCC = 32;                  // coils per block (64 value rows + 64 remainder rows)
constexpr int kTmPassArrivals = 32 + 1;    // value lanes (cp.async), meta
constexpr int kTmVBytes = 16 * 256;        // value operand: 16 row groups x 256 B
constexpr int kTmWBytes = (kTmN / 8) * 256;  // weight operand (hi or lo): 32 row groups x 256 B
constexpr int kTmStageBytes = kTmVBytes + 2 * kTmWBytes;
constexpr int kTmXS = 32 + 4;              // read-back exchange: one value row's 32 points (+ pad: the
                                           // 16-byte stores of 8 consecutive rows cover all banks)
constexpr int kTmXBytes = 2 * 128 * kTmXS * 4;  // 2 buffers x 128 rows
constexpr uint64_t kTmWaitNs = 200000000ull;    // bound on a hand-off wait (200 ms)
constexpr uint64_t kTmDrainNs = 2000000000ull;  // bound on the wait for the last MMAs (2 s)
constexpr uint64_t kTmStallNs = 1000000ull;     // test stall (1 ms)

// pass metadata flags (slot meta[1]) and chunk flags for the MMA thread
constexpr int kPassFirst = 1, kPassLast = 2, kPassEnd = 4;
constexpr uint32_t kChunkFirst = 1, kChunkLast = 2, kChunkAcc = 4, kChunkEnd = 8;

// barriers: pass full / empty per slot, stage full / empty per operand stage,
// accumulator full / empty per half, final commit, never signalled (test)
enum { kBarPassFull = 0, kBarPassEmpty = 3, kBarStFull = 6, kBarStEmpty = 10, kBarAccFull = 14,
       kBarAccEmpty = 16, kBarFinal = 18, kBarNever = 19, kBarCount = 20 };

struct TmShape {
    int R[3];        // region extents (tile + W - 1)
    int P;           // region points (<= 256)
    int CC;          // coils per block (<= 32)
    int ccp;         // deterministic scratch: coil stride of a region point (CC rounded up to the gather's group)
    int vrows;       // R[0] + R[1] + R[2]
    int table_off;   // per builder group two chunk weight tables (offset in dynamic shared memory)
    int goff_off;    // read-back: grid offsets of the current item's region points
    int wp;          // tap weights per sample and axis in the plan (4 or 8)
    int l_off;       // offset inside a slot: the packed first-tap offsets
    int nslots;      // pass ring depth
    int nstages;     // operand stages
    int slot_bytes;  // one pass slot
    int vals_off;    // offsets inside a slot: coil values, density weights, meta
    int wts_off;
    int meta_off;
    int stages_off;  // offsets in dynamic shared memory
    int x_off;
};

__device__ __forceinline__ uint32_t bar_addr(uint64_t *bars, int i) { return tc_smem(&bars[i]); }

__device__ __forceinline__ void bar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// bounded wait for completion number k of an mbarrier; gives up (and raises the
// block's abort flag) after limit_ns, or as soon as another role raised it. The
// global timer is read only after 64 polls, then once per 256 polls.
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

// tm_wait for all 32 lanes of a warp with a warp-uniform result
__device__ __forceinline__ bool tm_wait_warp(uint32_t bar, uint32_t k, uint64_t limit_ns, volatile int *abort)
{
    return __all_sync(0xffffffffu, tm_wait(bar, k, limit_ns, abort));
}

// K-major, no swizzle: 8-row x 16-byte core matrices, 128 bytes apart along K,
// 256 bytes apart along M / N (an operand of K = 8)
__device__ __forceinline__ uint64_t tm_desc(uint32_t addr)
{
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(256 >> 4) << 32) |
           (1ull << 46);
}

__device__ __forceinline__ uint32_t tm_off(int row, int k)
{
    return (uint32_t)((row >> 3) * 256 + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

__device__ __forceinline__ void tm_mma(uint32_t d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}

// tcgen05.wait::ld, with the loaded registers as operands so that no read of
// them is moved before the wait
__device__ __forceinline__ void tm_wait_ld(uint32_t (&r)[16])
{
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :
                 : "memory");
}

__device__ __forceinline__ void tm_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tm_named_sync(int id, int n)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// named barrier `id` over n threads that also returns whether every thread
// passed `ok` (the read-back warps leave their loop together, so none is left
// waiting at a named barrier when a bounded wait runs out)
__device__ __forceinline__ bool tm_named_all(int id, int n, bool ok)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, %2, %3, p;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)ok), "r"(id), "r"(n)
        : "memory");
    return r != 0;
}

// the work of a block: work items (bin, sample range) x coil chunks, tasks
// blockIdx.x, blockIdx.x + gridDim.x, ... (neighbouring items run at the same
// time on different SMs, so their halos meet in L2), each cut into 128-sample
// passes
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
    __device__ void next_task(const WorkItem *work, const int32_t *order)
    {
        task += gridDim.x;
        if (task < ntasks) {
            it = work[order[task / nchunks]];
            base = it.begin;
        }
    }
    __device__ void next(const WorkItem *work, const int32_t *order)
    {
        base += kTmSB;
        if (base >= it.end) next_task(work, order);
    }
    __device__ void next_segment(const WorkItem *work, const int32_t *order)
    {
        base += kTmSeg;
        if (base >= it.end) next_task(work, order);
    }
};

__device__ __forceinline__ void bin_origin(const Geom &g, int bin, int &f, int org[3])
{
    f = bin / g.nbins;
    const int lb = bin - f * g.nbins;
    org[0] = (lb % g.nb[0]) * g.T[0];
    org[1] = ((lb / g.nb[0]) % g.nb[1]) * g.T[1];
    org[2] = (lb / (g.nb[0] * g.nb[1])) * g.T[2];
}

// g: the plan's geometry with the tensor-core gridding bins (T, nb, nbins)
__global__ void __launch_bounds__(kTmThreads, 1) grid_tmem_kernel(
    Geom g, TmShape sh, const WorkItem *__restrict__ work, const int32_t *__restrict__ order, int nwork,
    int nchunks, const float *__restrict__ tw, const int32_t *__restrict__ tl, const int32_t *__restrict__ sidx, const void *__restrict__ ksp, int kreal, float2 *__restrict__ grid,
    int64_t batch, const float *__restrict__ weight, int wpb, float inv_scale, float2 *__restrict__ scratch,
    int *__restrict__ status, int *__restrict__ timeouts, int stall)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[kBarCount];
    __shared__ uint32_t tslot;
    __shared__ volatile int s_abort;
    __shared__ uint32_t stage_meta[kTmMaxStages];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int W = g.W[0];
    unsigned char *slots = smem;
    unsigned char *stages = smem + sh.stages_off;
    float *xbuf = reinterpret_cast<float *>(smem + sh.x_off);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(tc_smem(&tslot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int i = 0; i < kBarCount; i++) {
            int c = 1;  // commits and the final / test barriers
            if (i < kBarPassEmpty) c = kTmPassArrivals;
            else if (i < kBarStFull) c = kTmBuilders;   // pass empty: every builder group
            else if (i < kBarStEmpty) c = kTmGroup;     // stage full: the group that built the chunk
            else if (i >= kBarAccEmpty && i < kBarFinal) c = kTmEpi;
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_addr(bars, i)), "r"(c));
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tbase = tslot;
    const int RXY = sh.R[0] * sh.R[1];
    bool mma_issued = false;

    if (warp < kTmEpiWarp) {
        // ------------------------------------------------------------------ builders
        // region points tid and tid + 128 (weight operand rows), value pairs
        // (coil, sample) = (tid >> 3, tid & 7) and (16 + (tid >> 3), tid & 7)
        const int bg = tid >> 7, btid = tid & (kTmGroup - 1);  // builder group, thread in group
        uint32_t vxyz[2][3], woff[2];
        bool has_point[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int p = btid + 128 * h;
            has_point[h] = p < sh.P;
            const int pc = min(p, sh.P - 1);
            const int rz = pc / RXY, rem = pc - rz * RXY;
            const int ry = rem / sh.R[0], rx = rem - ry * sh.R[0];
            vxyz[h][0] = (uint32_t)rx * (4 * kTmTableRow);  // table rows
            vxyz[h][1] = (uint32_t)(sh.R[0] + ry) * (4 * kTmTableRow);
            vxyz[h][2] = (uint32_t)(sh.R[0] + sh.R[1] + rz) * (4 * kTmTableRow);
            woff[h] = tm_off(p, 0);  // and + 128 for samples 4..7
        }
        const int bs = btid & 7;
        // the table entries of this thread: (region row, sample) = (e / 8, e % 8)
        // for e = btid and btid + 128 (rows of x, then y, then z)
        int trow_axis[2], trow_r[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int row = (btid + 128 * h) >> 3;
            trow_axis[h] = row < sh.R[0] ? 0 : (row < sh.R[0] + sh.R[1] ? 1 : 2);
            trow_r[h] = row - (trow_axis[h] == 0 ? 0 : (trow_axis[h] == 1 ? sh.R[0] : sh.R[0] + sh.R[1]));
        }
        float *tables = reinterpret_cast<float *>(smem + sh.table_off) + bg * 2 * kTmTable;
        uint32_t chunk_no = 0;
        int task_no = 0, cur_cact = 0;
        bool ok = true;
        for (uint32_t pass_no = 0; ok; pass_no++) {
            const int slot = pass_no % sh.nslots;
            // every decision to leave is taken by the whole group (named barrier
            // with reduction), so no warp of it is left at a named barrier
            const bool okp = tm_wait_warp(bar_addr(bars, kBarPassFull + slot), pass_no / sh.nslots, kTmWaitNs, &s_abort);
            if (!tm_named_all(2 + bg, kTmGroup, okp)) {
                ok = false;
                break;
            }
            unsigned char *sl = slots + slot * sh.slot_bytes;
            const int *meta = reinterpret_cast<const int *>(sl + sh.meta_off);
            const int flags = meta[1];
            if (flags & kPassEnd) break;
            const int n = meta[2];
            if (flags & kPassFirst) cur_cact = meta[4];
            const float *pw = reinterpret_cast<const float *>(sl);
            const int32_t *pl = reinterpret_cast<const int32_t *>(sl + sh.l_off);
            const float2 *vals = reinterpret_cast<const float2 *>(sl + sh.vals_off);
            const float *wts = reinterpret_cast<const float *>(sl + sh.wts_off);
            const int nch = (n + kTmSC - 1) / kTmSC;
            for (int ch = 0; ch < nch; ch++) {
                const bool first = (flags & kPassFirst) && ch == 0;
                const bool last = (flags & kPassLast) && ch == nch - 1;
                if ((int)(chunk_no % kTmGroups) != bg) {
                    // the other group builds this chunk
                    chunk_no++;
                    if (last) task_no++;
                    continue;
                }
                const int stage = chunk_no % sh.nstages;
                bool okc = chunk_no < (uint32_t)sh.nstages ||
                           tm_wait_warp(bar_addr(bars, kBarStEmpty + stage), chunk_no / sh.nstages - 1, kTmWaitNs,
                                        &s_abort);
                // test hook: a barrier that nothing signals, so the wait runs out
                if (stall && chunk_no >= (uint32_t)sh.nstages)
                    okc = tm_wait_warp(bar_addr(bars, kBarNever), 0, kTmStallNs, &s_abort) && okc;
                const uint32_t sbase = tc_smem(stages + stage * kTmStageBytes);
                // the chunk's weight table: Kaiser-Bessel weight of sample s at region
                // row r of each axis (zero off its taps); two per group, alternating
                // (a table is written again only after the group's next barrier)
                float *table = tables + ((chunk_no / kTmGroups) & 1) * kTmTable;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int e = btid + 128 * h;
                    if (e >= sh.vrows * 8) break;
                    const int a = trow_axis[h], si = ch * kTmSC + (e & 7);
                    float v = 0.0f;
                    if (si < n) {
                        const int i = trow_r[h] - ((pl[si] >> (8 * a)) & 255);
                        if (i >= 0 && i < W) v = pw[(si * 3 + a) * sh.wp + i];
                    }
                    table[(e >> 3) * kTmTableRow + (e & 7)] = v;
                }
                // the group's barrier: the table is complete, and the group leaves
                // together if a wait ran out (nothing asynchronous was written yet)
                if (!tm_named_all(2 + bg, kTmGroup, okc)) {
                    ok = false;
                    break;
                }
                // weight operand: rows p, samples 0..7, hi and lo (rows >= P are not read back)
                const uint32_t tb = tc_smem(table);
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    if (!has_point[h]) continue;
                    const uint32_t ax = tb + vxyz[h][0], ay = tb + vxyz[h][1], az = tb + vxyz[h][2];
                    const float4 x0 = tc_lds4(ax), x1 = tc_lds4(ax + 16);
                    const float4 y0 = tc_lds4(ay), y1 = tc_lds4(ay + 16);
                    const float4 z0 = tc_lds4(az), z1 = tc_lds4(az + 16);
                    const float4 w0 = make_float4(x0.x * y0.x * z0.x, x0.y * y0.y * z0.y, x0.z * y0.z * z0.z,
                                                  x0.w * y0.w * z0.w);
                    const float4 w1 = make_float4(x1.x * y1.x * z1.x, x1.y * y1.y * z1.y, x1.z * y1.z * z1.z,
                                                  x1.w * y1.w * z1.w);
                    const float4 h0 = make_float4(tc_hi(w0.x), tc_hi(w0.y), tc_hi(w0.z), tc_hi(w0.w));
                    const float4 h1 = make_float4(tc_hi(w1.x), tc_hi(w1.y), tc_hi(w1.z), tc_hi(w1.w));
                    const uint32_t wh = sbase + kTmVBytes + woff[h], wl = wh + kTmWBytes;
                    tc_sts4(wh, h0);
                    tc_sts4(wh + 128, h1);
                    tc_sts4(wl, make_float4(w0.x - h0.x, w0.y - h0.y, w0.z - h0.z, w0.w - h0.w));
                    tc_sts4(wl + 128, make_float4(w1.x - h1.x, w1.y - h1.y, w1.z - h1.z, w1.w - h1.w));
                }
                // value operand: coils bc, bc + 16 at sample bs (zero for absent coils / samples)
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int bc = (btid >> 3) + 16 * h;
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
                    const float hx = tc_hi(v.x), hy = tc_hi(v.y);
                    // samples 4..7 (128 bytes further, the same banks) store the
                    // imaginary row first, so that each store of the warp
                    // covers all 32 banks once
                    const int sw = bs >> 2;
                    tc_sts(sbase + tm_off(2 * bc + sw, bs), sw ? hy : hx);
                    tc_sts(sbase + tm_off(2 * bc + 1 - sw, bs), sw ? hx : hy);
                    tc_sts(sbase + tm_off(64 + 2 * bc + sw, bs), sw ? v.y - hy : v.x - hx);
                    tc_sts(sbase + tm_off(65 + 2 * bc - sw, bs), sw ? v.x - hx : v.y - hy);
                }
                if (btid == 0)
                    stage_meta[stage] = (first ? kChunkFirst : 0u) | (last ? kChunkLast : 0u) |
                                        ((task_no & 1) ? kChunkAcc : 0u);
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                bar_arrive(bar_addr(bars, kBarStFull + stage));
                chunk_no++;
                if (last) task_no++;
            }
            if (!ok) break;
            bar_arrive(bar_addr(bars, kBarPassEmpty + slot));
        }
        if (ok && (int)(chunk_no % kTmGroups) == bg) {
            // end marker for the MMA thread, from the group whose turn it is
            const int stage = chunk_no % sh.nstages;
            if (chunk_no < (uint32_t)sh.nstages ||
                tm_wait_warp(bar_addr(bars, kBarStEmpty + stage), chunk_no / sh.nstages - 1, kTmWaitNs, &s_abort)) {
                if (btid == 0) stage_meta[stage] = kChunkEnd;
                bar_arrive(bar_addr(bars, kBarStFull + stage));
            }
        }
    } else if (warp < kTmMmaWarp) {
        // ------------------------------------------------------------------ read-back
        // Per work item: the grid offsets of the region points (one per thread)
        // into shared memory; then per group of 32 points, the two warps of each
        // lane quarter load 16 columns each of its 32 value rows (tcgen05.ld, the
        // next group's load issued before this group is flushed) and store them
        // into X[row][point]; warp e then takes coils 4e .. 4e + 3 with lane =
        // point: value = X[2c][p] + X[64 + 2c][p] (real; hi + lo rows) and
        // X[2c + 1][p] + X[65 + 2c][p] (imaginary), one float2 atomic per
        // (point, coil): 32 neighbouring points per instruction, a few grid rows
        const int e = warp - kTmEpiWarp, et = tid - kTmEpiWarp * 32;
        const int q = warp & 3, hcol = e >> 2;
        const uint32_t lanebase = (uint32_t)(q * 32) << 16;
        const int row = q * 32 + lane;
        int *goff = reinterpret_cast<int *>(smem + sh.goff_off);
        PassSeq ps;
        ps.start(work, order, nwork, nchunks);
        uint32_t xg = 0;  // point groups read back so far (exchange buffer xg & 1)
        for (int k = 0; !ps.done(); k++) {
            int f, org[3];
            bin_origin(g, ps.it.bin, f, org);
            const int64_t b0 = (int64_t)(ps.task % nchunks) * sh.CC;
            const int cact = (int)(batch - b0 < (int64_t)sh.CC ? batch - b0 : (int64_t)sh.CC);
            const int acc = k & 1;
            const bool okw = tm_wait_warp(bar_addr(bars, kBarAccFull + acc), k >> 1, kTmWaitNs, &s_abort);
            // (also: every read-back thread is done with the previous item's offsets)
            if (!tm_named_all(1, kTmEpi, okw)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (et < sh.P) {
                const int pz = et / RXY, pr = et - pz * RXY;
                const int py = pr / sh.R[0], px = pr - py * sh.R[0];
                const int gx = (org[0] + px + g.G[0] - g.half[0]) % g.G[0];
                const int gy = (org[1] + py + g.G[1] - g.half[1]) % g.G[1];
                const int gz = (org[2] + pz + g.G[2] - g.half[2]) % g.G[2];
                goff[et] = (gz * g.G[1] + gy) * g.G[0] + gx;
            }
            const float2 *gitem = grid + (b0 * g.nframes + f) * g.gsize;
            // deterministic mode: the item stores its partial sums into its
            // scratch slot (the item's index), [region point][coil]
            float2 *part = scratch ? scratch + ((int64_t)order[ps.task / nchunks] * nchunks + ps.task % nchunks) *
                                                   kTmN * sh.ccp
                                   : nullptr;
            const int64_t cstride = (int64_t)g.nframes * g.gsize;
            uint32_t r[16], rn[16];
            tc_ld16(tbase + lanebase + (uint32_t)(acc * kTmN + 16 * hcol), r);
            tm_wait_ld(r);
            for (int c0 = 0; c0 < sh.P; c0 += 32, xg++) {
                // two exchange buffers, alternating over all groups of all items: a
                // buffer is written again only after the next group's barrier, which
                // its readers reach after reading it
                float *xb = xbuf + (xg & 1) * (128 * kTmXS);
                float4 *xw = reinterpret_cast<float4 *>(xb + row * kTmXS + 16 * hcol);
#pragma unroll
                for (int j = 0; j < 4; j++)
                    xw[j] = make_float4(__uint_as_float(r[4 * j]), __uint_as_float(r[4 * j + 1]),
                                        __uint_as_float(r[4 * j + 2]), __uint_as_float(r[4 * j + 3]));
                tm_named_sync(1, kTmEpi);
                const bool more = c0 + 32 < sh.P;
                if (more) tc_ld16(tbase + lanebase + (uint32_t)(acc * kTmN + c0 + 32 + 16 * hcol), rn);
                const int pp = c0 + lane;
                if (pp < sh.P) {
                    const float2 *gp = gitem + goff[pp];
                    float2 v[4];
#pragma unroll
                    for (int cc = 0; cc < 4; cc++) {
                        const int c = e * 4 + cc;
                        v[cc] = make_float2((xb[(2 * c) * kTmXS + lane] + xb[(64 + 2 * c) * kTmXS + lane]) * inv_scale,
                                            (xb[(2 * c + 1) * kTmXS + lane] + xb[(65 + 2 * c) * kTmXS + lane]) *
                                                inv_scale);
                    }
                    if (part) {
                        // coils 4e .. 4e + 3 of the point: one 32-byte sector in
                        // one 256-bit store (coils past the batch hold the zero
                        // rows of V)
                        if (e * 4 < cact)
                            asm volatile("st.global.cs.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(
                                             part + pp * sh.ccp + e * 4),
                                         "f"(v[0].x), "f"(v[0].y), "f"(v[1].x), "f"(v[1].y), "f"(v[2].x), "f"(v[2].y),
                                         "f"(v[3].x), "f"(v[3].y)
                                         : "memory");
                    } else {
#pragma unroll
                        for (int cc = 0; cc < 4; cc++) {
                            const int c = e * 4 + cc;
                            if (c < cact && (v[cc].x != 0.0f || v[cc].y != 0.0f))
                                atomicAdd(const_cast<float2 *>(gp) + c * cstride, v[cc]);
                        }
                    }
                }
                if (more) {
                    tm_wait_ld(rn);
#pragma unroll
                    for (int j = 0; j < 16; j++) r[j] = rn[j];
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            bar_arrive(bar_addr(bars, kBarAccEmpty + acc));
            ps.next_segment(work, order);
        }
    } else if (warp == kTmMmaWarp) {
        // ------------------------------------------------------------------ MMA issue
        if (lane == 0) {
            // D f32, A / B tf32, both K-major, N = 256, M = 128
            const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTmN >> 3) << 17) | (8u << 24);
            const uint32_t s0 = tc_smem(stages);
            int acc_uses[2] = {0, 0};
            for (uint32_t chunk = 0;; chunk++) {
                const int stage = chunk % sh.nstages;
                if (!tm_wait(bar_addr(bars, kBarStFull + stage), chunk / sh.nstages, kTmWaitNs, &s_abort)) break;
                const uint32_t m = stage_meta[stage];
                if (m & kChunkEnd) break;
                const int acc = (m & kChunkAcc) ? 1 : 0;
                if ((m & kChunkFirst) && acc_uses[acc] > 0 &&
                    !tm_wait(bar_addr(bars, kBarAccEmpty + acc), acc_uses[acc] - 1, kTmWaitNs, &s_abort))
                    break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t sb = s0 + (uint32_t)(stage * kTmStageBytes);
                const uint64_t vd = tm_desc(sb), wh = tm_desc(sb + kTmVBytes),
                               wl = tm_desc(sb + kTmVBytes + kTmWBytes);
                const uint32_t d = tbase + (uint32_t)(acc * kTmN);
                tm_mma(d, vd, wh, idesc, (m & kChunkFirst) ? 0u : 1u);
                tm_mma(d, vd, wl, idesc, 1u);
                mma_issued = true;
                tm_commit(bar_addr(bars, kBarStEmpty + stage));
                if (m & kChunkLast) {
                    tm_commit(bar_addr(bars, kBarAccFull + acc));
                    acc_uses[acc]++;
                }
            }
        }
    } else {
        // ------------------------------------------------------------------ producer
        // (warp 17) coordinates, coil values and density weights of each pass,
        // cp.async into the ring slot; sample indices loaded one pass ahead
        PassSeq ps;
        ps.start(work, order, nwork, nchunks);
        int gi[4] = {-1, -1, -1, -1};
        auto load = [&](const PassSeq &q) {
            if (q.done()) return;
            const int nq = min(kTmSB, q.it.end - q.base);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int st = lane + 32 * j;
                gi[j] = st < nq ? sidx[q.base + st] : -1;
            }
        };
        load(ps);
        for (uint32_t pass_no = 0;; pass_no++) {
            const int slot = pass_no % sh.nslots;
            if (pass_no >= (uint32_t)sh.nslots &&
                !tm_wait_warp(bar_addr(bars, kBarPassEmpty + slot), pass_no / sh.nslots - 1, kTmWaitNs, &s_abort))
                break;
            unsigned char *sl = slots + slot * sh.slot_bytes;
            const uint32_t full = bar_addr(bars, kBarPassFull + slot);
            if (ps.done()) {
                // end marker
                if (lane == 0) reinterpret_cast<int *>(sl + sh.meta_off)[1] = kPassEnd;
                asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(full) : "memory");
                if (lane == 0) bar_arrive(full);
                break;
            }
            const WorkItem it = ps.it;
            const int base = ps.base;
            const int n = min(kTmSB, it.end - base);
            const int64_t b0 = (int64_t)(ps.task % nchunks) * sh.CC;
            const int cact = (int)(batch - b0 < (int64_t)sh.CC ? batch - b0 : (int64_t)sh.CC);
            if (lane == 0) {
                int *meta = reinterpret_cast<int *>(sl + sh.meta_off);
                meta[0] = it.bin;
                meta[1] = ((base - it.begin) % kTmSeg == 0 ? kPassFirst : 0) |
                          (base + kTmSB >= it.end || (base + kTmSB - it.begin) % kTmSeg == 0 ? kPassLast : 0);
                meta[2] = n;
                meta[3] = (int)b0;
                meta[4] = cact;
            }
            const uint32_t tdst = tc_smem(sl), ldst = tc_smem(sl + sh.l_off), vdst = tc_smem(sl + sh.vals_off),
                           wdst = tc_smem(sl + sh.wts_off);
            {
                // tap weights: 3 wp floats per sample, in 16-byte pieces (sample-major,
                // so one pass's are contiguous in the plan and in the slot)
                const int pieces = n * 3 * sh.wp / 4;
                const float *src = tw + (int64_t)base * 3 * sh.wp;
                for (int q = lane; q < pieces; q += 32)
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(tdst + (uint32_t)q * 16),
                                 "l"(src + 4 * q)
                                 : "memory");
                for (int q = lane; q < n; q += 32)
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(ldst + (uint32_t)q * 4),
                                 "l"(tl + base + q)
                                 : "memory");
            }
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
            ps.next(work, order);
            load(ps);
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    }

    // teardown: no MMA may still write tensor memory when it is freed
    if (warp == kTmMmaWarp && lane == 0 && mma_issued) {
        tm_commit(bar_addr(bars, kBarFinal));
        if (!tc_wait(bar_addr(bars, kBarFinal), 0, kTmDrainNs)) s_abort = 1;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tbase));
    if (tid == 0 && s_abort) {
        atomicAdd(timeouts, 1);
        atomicAdd(status, 1);
    }
}

// The regions that cover grid position `pos` along one axis: bins b with
// offsets u in their region, (b T + u - half) = pos (mod G), 0 <= u < R <= 8,
// as 16-bit entries (b << 3 | u) + 1 in increasing u, 0 after the last. With
// R <= G a bin covers a position at most once; b T = (pos + half - u) mod G
// < G implies b < nb. Increasing u puts neighbouring positions of one bin at
// the same index.
__device__ __forceinline__ uint4 tm_cover(int pos, int G, int T, int R, int half)
{
    uint32_t e[4] = {0, 0, 0, 0};
    int n = 0;
    const int t = (pos + half) % G;
    for (int u = 0; u < R; u++) {
        int o = t - u;
        if (o < 0) o += G;
        if (o % T == 0) {
            e[n >> 1] |= (uint32_t)((o / T) << 3 | u) + 1u << (16 * (n & 1));
            n++;
        }
    }
    return make_uint4(e[0], e[1], e[2], e[3]);
}

__device__ __forceinline__ int tm_cover_count(const uint4 &c)
{
    const uint32_t w[4] = {c.x, c.y, c.z, c.w};
    int n = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) n += ((w[q] & 0xffffu) != 0) + ((w[q] >> 16) != 0);
    return n;
}

// G coils of one region point of a deterministic scratch slot (8 G
// contiguous bytes, 256-bit loads), and their addition to the accumulators
template <int G>
__device__ __forceinline__ void tm_ldg(const float2 *src, float (&v)[2 * G])
{
#pragma unroll
    for (int j = 0; j < G / 4; j++)
        asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
            : "=f"(v[8 * j]), "=f"(v[8 * j + 1]), "=f"(v[8 * j + 2]), "=f"(v[8 * j + 3]), "=f"(v[8 * j + 4]),
              "=f"(v[8 * j + 5]), "=f"(v[8 * j + 6]), "=f"(v[8 * j + 7])
            : "l"(src + 4 * j));
}

template <int G>
__device__ __forceinline__ void tm_addg(float2 (&acc)[G], const float (&v)[2 * G])
{
#pragma unroll
    for (int c = 0; c < G; c++) {
        acc[c].x += v[2 * c];
        acc[c].y += v[2 * c + 1];
    }
}

__device__ __forceinline__ int tm_cover_at(const uint4 &c, int k)
{
    const int q = k >> 1;  // entries 2q and 2q + 1 share a word
    const uint32_t w = q < 2 ? (q < 1 ? c.x : c.y) : (q < 3 ? c.z : c.w);
    return (int)((w >> (16 * (k & 1))) & 0xffff) - 1;
}

// Deterministic mode: every grid point adds, for kTmGatherCoils coils of one
// coil chunk, in a fixed order (covering bins by z, y, x offset, then each
// bin's items in sample order) the partial sums that the covering items
// stored in their scratch slots ([region point][coil]), and writes the grid
// once (0 where no item covers it). A thread reads its coils of a region
// point as 8 kTmGatherCoils contiguous bytes; lanes run along x, so a warp writes 32
// neighbouring grid points per coil. The coil groups of the same points are
// neighbouring blocks (blockIdx.x = point block * groups + group, blockIdx.y
// = chunk), so each point's coils (256 bytes of a slot) come from DRAM once.
// The cover lists of all positions (two entries per 32-bit word, up to 8 per
// position) are built per block in shared memory (G[0] + G[1] + G[2] uint4).
constexpr int kTmGatherCoils = 8;

__global__ void __launch_bounds__(256, 2) grid_tm_gather_kernel(Geom g, TmShape sh, const int32_t *__restrict__ istart,
                                                            const float2 *__restrict__ scratch,
                                                            float2 *__restrict__ grid, int64_t batch, int nchunks)
{
    extern __shared__ uint4 s_cover[];
    uint4 *cov[3] = {s_cover, s_cover + g.G[0], s_cover + g.G[0] + g.G[1]};
    for (int a = 0; a < 3; a++)
        for (int pos = threadIdx.x; pos < g.G[a]; pos += blockDim.x)
            cov[a][pos] = tm_cover(pos, g.G[a], g.T[a], sh.R[a], g.half[a]);
    __syncthreads();
    const int ngrp = (sh.CC + kTmGatherCoils - 1) / kTmGatherCoils;
    const int cch = blockIdx.y, c0 = (blockIdx.x % ngrp) * kTmGatherCoils;
    const int pblock = blockIdx.x / ngrp, pblocks = gridDim.x / ngrp;
    const int64_t b0 = (int64_t)cch * sh.CC + c0;
    // coils of this chunk (the last chunk may hold fewer than CC), of this group
    const int ccoils = (int)min((int64_t)sh.CC, batch - (int64_t)cch * sh.CC);
    const int cact = min(kTmGatherCoils, ccoils - c0);
    const int64_t npts = (int64_t)g.nframes * g.gsize;
    const int gxy = g.G[0] * g.G[1];
    for (int64_t i = (int64_t)pblock * blockDim.x + threadIdx.x; i < npts; i += (int64_t)pblocks * blockDim.x) {
        const int f = (int)(i / g.gsize), r = (int)(i - (int64_t)f * g.gsize);
        const int z = r / gxy, y = (r - z * gxy) / g.G[0], x = r - z * gxy - y * g.G[0];
        const uint4 cz = cov[2][z], cy = cov[1][y], cx = cov[0][x];
        float2 acc[kTmGatherCoils];
#pragma unroll
        for (int c = 0; c < kTmGatherCoils; c++) acc[c] = make_float2(0.0f, 0.0f);
        const int ncz = tm_cover_count(cz), ncy = tm_cover_count(cy), ncx = tm_cover_count(cx);
        auto slot = [&](int s, int pt) {
            return scratch + (((int64_t)s * nchunks + cch) * kTmN + pt) * sh.ccp + c0;
        };
        if (ncz <= 2 && ncy <= 2 && ncx <= 2) {
            // at most two covering bins per axis (every position of the usual
            // geometries): the item ranges of all 8 candidates first, then the
            // first items of 4 candidates at a time, so that their loads are
            // in flight together; the additions keep the general order
            int beg[8], cnt[8], pts[8];
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const int kz = q >> 2, ky = (q >> 1) & 1, kx = q & 1;
                beg[q] = cnt[q] = pts[q] = 0;
                if (kz < ncz && ky < ncy && kx < ncx) {
                    const int vz = tm_cover_at(cz, kz), vy = tm_cover_at(cy, ky), vx = tm_cover_at(cx, kx);
                    const int key = f * g.nbins + ((vz >> 3) * g.nb[1] + (vy >> 3)) * g.nb[0] + (vx >> 3);
                    beg[q] = __ldg(istart + key);
                    cnt[q] = __ldg(istart + key + 1) - beg[q];
                    pts[q] = ((vz & 7) * sh.R[1] + (vy & 7)) * sh.R[0] + (vx & 7);
                }
            }
#pragma unroll
            for (int h = 0; h < 4; h++) {
                float v[2][2 * kTmGatherCoils];
#pragma unroll
                for (int j = 0; j < 2; j++)
                    if (cnt[2 * h + j] > 0) tm_ldg<kTmGatherCoils>(slot(beg[2 * h + j], pts[2 * h + j]), v[j]);
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const int q = 2 * h + j;
                    if (cnt[q] > 0) {
                        tm_addg<kTmGatherCoils>(acc, v[j]);
                        for (int s = beg[q] + 1; s < beg[q] + cnt[q]; s++) {
                            float w[2 * kTmGatherCoils];
                            tm_ldg<kTmGatherCoils>(slot(s, pts[q]), w);
                            tm_addg<kTmGatherCoils>(acc, w);
                        }
                    }
                }
            }
        } else {
            for (int kz = 0; kz < ncz; kz++) {
                const int vz = tm_cover_at(cz, kz);
                for (int ky = 0; ky < ncy; ky++) {
                    const int vy = tm_cover_at(cy, ky);
                    const int kyz = f * g.nbins + ((vz >> 3) * g.nb[1] + (vy >> 3)) * g.nb[0];
                    const int pyz = ((vz & 7) * sh.R[1] + (vy & 7)) * sh.R[0];
                    for (int kx = 0; kx < ncx; kx++) {
                        const int vx = tm_cover_at(cx, kx);
                        const int key = kyz + (vx >> 3);
                        const int s1 = istart[key + 1];
                        for (int s = istart[key]; s < s1; s++) {
                            float w[2 * kTmGatherCoils];
                            tm_ldg<kTmGatherCoils>(slot(s, pyz + (vx & 7)), w);
                            tm_addg<kTmGatherCoils>(acc, w);
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int c = 0; c < kTmGatherCoils; c++)
            if (c < cact) grid[(b0 + c) * npts + i] = acc[c];
    }
}

bool tm_shape(const dmr_plan *p, int64_t batch, int wpb, int smem_limit, TmShape &s)
{
    const Geom &g = p->g;
    if (g.ndim != 3 || batch < 1 || p->tg_T[0] == 0) return false;
    const int W = g.W[0];
    for (int a = 0; a < 3; a++) s.R[a] = p->tg_T[a] + W - 1;
    s.P = s.R[0] * s.R[1] * s.R[2];
    if (s.P > kTmN) return false;
    s.vrows = s.R[0] + s.R[1] + s.R[2];
    if (s.vrows > kTmMaxRows) return false;
    s.CC = (int)std::min<int64_t>(batch, kTmCC);
    s.ccp = (s.CC + kTmGatherCoils - 1) / kTmGatherCoils * kTmGatherCoils;
    s.wp = p->tg_wp;
    int off = kTmSB * 3 * s.wp * 4;  // tap weights of the pass, [sample][axis][wp]
    s.l_off = off;
    off += kTmSB * 4;
    off = (off + 15) / 16 * 16;
    s.vals_off = off;
    off += s.CC * kTmSBP * 8;
    s.wts_off = off;
    off += (wpb ? s.CC : 1) * kTmSBP * 4;
    off = (off + 15) / 16 * 16;
    s.meta_off = off;
    off += 32;
    s.slot_bytes = (off + 127) / 128 * 128;
    // deepest ring that fits: 3 pass slots and 4 operand stages, else fewer
    for (int ns = kTmMaxSlots; ns >= 2; ns--)
        for (int nst = kTmMaxStages; nst >= 2; nst--) {
            const int stages_off = (ns * s.slot_bytes + 1023) / 1024 * 1024;
            const int x_off = stages_off + nst * kTmStageBytes;
            const int table_off = x_off + kTmXBytes;
            const int goff_off = table_off + 2 * kTmGroups * kTmTable * 4;
            if (goff_off + kTmN * 4 <= smem_limit) {
                s.nslots = ns;
                s.nstages = nst;
                s.stages_off = stages_off;
                s.x_off = x_off;
                s.table_off = table_off;
                s.goff_off = goff_off;
                return true;
            }
        }
    return false;
}

}  // namespace

// Tensor-core gridding of a 3D plan with its gridding bins; DMR_ERR_UNSUPPORTED
// when the plan has none or the geometry does not fit (the caller then uses
// the other kernels).
// scratch of deterministic tensor-core gridding: one slot of kTmN region
// points per (work item, coil chunk), each point the chunk's coils rounded up
// to the gather's coil group
size_t tm_scratch_bytes(const dmr_plan *p, int64_t batch)
{
    if (p->g.ndim != 3 || p->tg_T[0] == 0 || p->tg_nwork == 0 || batch < 1) return 0;
    const int64_t cc = std::min<int64_t>(batch, kTmCC);
    return (size_t)p->tg_nwork * ceil_div(batch, cc) * kTmN * ((cc + kTmGatherCoils - 1) / kTmGatherCoils * kTmGatherCoils) *
           sizeof(float2);
}

int grid_tm_dispatch(const dmr_plan *p, const void *ksp, int kreal, float2 *grid, int64_t batch,
                     const float *weight, int wpb, int det, void *scratch, size_t scratch_bytes, int *timeouts,
                     int stall, int64_t det_limit, cudaStream_t st)
{
    int dev = 0, sms = 0, smem_blk = 0;
    DMR_CUDA(cudaGetDevice(&dev));
    DMR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    DMR_CUDA(cudaDeviceGetAttribute(&smem_blk, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa;
    DMR_CUDA(cudaFuncGetAttributes(&fa, grid_tmem_kernel));
    TmShape sh;
    if (!tm_shape(p, batch, wpb, smem_blk - (int)fa.sharedSizeBytes, sh)) return DMR_ERR_UNSUPPORTED;
    const size_t smem = (size_t)sh.goff_off + kTmN * 4;
    // one block per SM: it allocates all 512 tensor-memory columns
    DMR_CUDA(cudaFuncSetAttribute(grid_tmem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    DMR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grid_tmem_kernel, kTmThreads, smem));
    if (per_sm != 1) return DMR_ERR_UNSUPPORTED;
    // deterministic mode needs the points of one region on distinct grid
    // points and at most 8 region points per axis (the gather's cover lists)
    if (det)
        for (int a = 0; a < 3; a++)
            if (sh.R[a] > p->g.G[a] || sh.R[a] > 8) return DMR_ERR_UNSUPPORTED;
    // the deterministic gather writes every grid point
    if (!det || p->tg_nwork == 0)
        DMR_CUDA(cudaMemsetAsync(grid, 0, (size_t)batch * p->g.nframes * p->g.gsize * sizeof(float2), st));
    if (p->tg_nwork == 0) return DMR_OK;
    const int64_t nchunks = ceil_div(batch, sh.CC);
    DMR_CHECK((int64_t)p->tg_nwork * nchunks < (1ll << 31), DMR_ERR_UNSUPPORTED, "too many gridding tasks");
    DMR_CHECK(nchunks * sh.CC < (1ll << 31), DMR_ERR_UNSUPPORTED, "batch too large");
    Geom g = p->g;
    for (int a = 0; a < 3; a++) {
        g.T[a] = p->tg_T[a];
        g.nb[a] = p->tg_nb[a];
    }
    g.nbins = p->tg_nbins;
    const float inv_scale = (float)(1.0 / p->scale);
    if (!det) {
        const int blocks = (int)std::min<int64_t>((int64_t)p->tg_nwork * nchunks, (int64_t)sms);
        grid_tmem_kernel<<<blocks, kTmThreads, smem, st>>>(
            g, sh, p->tg_work, p->tg_order, p->tg_nwork, (int)nchunks, p->tg_w, p->tg_l, p->tg_sidx, ksp, kreal,
            grid, batch, weight, wpb, inv_scale, nullptr, p->status, timeouts, stall);
        DMR_LAUNCHED("grid_tmem_kernel");
        return DMR_OK;
    }
    // deterministic: the items store their partial sums into scratch slots
    // (no grid writes), then the gather sums them per grid point in a fixed
    // order: every run adds the same values in the same order
    const int ngrp = (sh.CC + kTmGatherCoils - 1) / kTmGatherCoils;
    DMR_CHECK(nchunks <= 65535, DMR_ERR_UNSUPPORTED, "batch too large");
    // the gather's cover lists: one uint4 per grid position of each axis
    const size_t gsmem = (size_t)(p->g.G[0] + p->g.G[1] + p->g.G[2]) * sizeof(uint4);
    if (gsmem > 48 * 1024) {
        DMR_CHECK(gsmem <= (size_t)smem_blk, DMR_ERR_UNSUPPORTED, "grid too large for the gather");
        DMR_CUDA(cudaFuncSetAttribute(grid_tm_gather_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gsmem));
    }
    const size_t need = tm_scratch_bytes(p, batch);
    // over the caller's limit, or no memory for it: another deterministic
    // kernel takes the call (nothing has been launched yet)
    if (det_limit > 0 && need > (size_t)det_limit) return DMR_ERR_UNSUPPORTED;
    void *owned = nullptr;
    if (scratch == nullptr || scratch_bytes < need) {
        cudaMemPool_t pool = scratch_pool(p->device);
        if (pool == nullptr) return DMR_ERR_UNSUPPORTED;
        const cudaError_t e = cudaMallocFromPoolAsync(&owned, need, pool, st);
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            return DMR_ERR_UNSUPPORTED;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaMallocFromPoolAsync", __FILE__, __LINE__);
        scratch = owned;
    }
    int rc = DMR_OK;
    const int blocks = (int)std::min<int64_t>((int64_t)p->tg_nwork * nchunks, (int64_t)sms);
    grid_tmem_kernel<<<blocks, kTmThreads, smem, st>>>(
        g, sh, p->tg_work, p->tg_order, p->tg_nwork, (int)nchunks, p->tg_w, p->tg_l, p->tg_sidx, ksp, kreal, grid,
        batch, weight, wpb, inv_scale, (float2 *)scratch, p->status, timeouts, stall);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) rc = cuda_fail(e, "grid_tmem_kernel", __FILE__, __LINE__);
    if (rc == DMR_OK) {
        const int64_t npts = (int64_t)g.nframes * g.gsize;
        const int gblocks = (int)std::min<int64_t>(ceil_div(npts, 256), (int64_t)sms * 16);
        grid_tm_gather_kernel<<<dim3(gblocks * ngrp, (unsigned)nchunks), 256, gsmem, st>>>(
            g, sh, p->tg_item_start, (const float2 *)scratch, grid, batch, (int)nchunks);
        g_launches.fetch_add(1, std::memory_order_relaxed);
        e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_fail(e, "grid_tm_gather_kernel", __FILE__, __LINE__);
    }
    if (owned) cudaFreeAsync(owned, st);
    return rc;
}

}  // namespace dmr
