// Tensor-core gridding for 3D (tcgen05, TF32 operands with a three-term split).
//
// Reference: apply_gridding and its 3D kernel
// (src/deepmr/fft/_interp/grid.py:14-125, 253-284):
//   grid[f, b, iz, iy, ix] += value_z * value_y * value_x * y[f, b, p]   (then / scale)
//
// For one bin and a chunk of up to 32 coils, what the bin's samples add to its
// tile + halo (P = R0 R1 R2 points, R = T + W - 1 per axis) is a matrix product
//     D[p, n] = sum_s A[p, s] B[n, s]
// with A[p, s] = wx * wy * wz of sample s at point p (zero outside its W^3
// support) and B[n, s] the real (n = 2c) or imaginary (n = 2c + 1) part of the
// value of sample s for coil c. A block builds A and B in shared memory for
// eight samples at a time and one thread issues tcgen05.mma into a tensor-memory
// accumulator of M = 128 points x N = 2 x coils per 128-point tile; the
// accumulator stays in tensor memory for all the samples of the bin, and is
// then read back (tcgen05.ld) and added to the grid with global float2 atomics.
// The spreading weights are built once per sample for all coils of the chunk,
// and the zeros of A cost tensor-core cycles instead of scalar instructions.
//
// Precision: each float32 operand x is split into hi (x with the mantissa
// bits below tf32 cleared) and lo = x - hi, stored as two K blocks [hi | lo];
// three MMAs per 128-point tile add hi*hi, hi*lo and lo*hi, which leaves a
// relative error of about 2^-20 per product (the dropped lo*lo term and the
// tf32 reading of lo), and the accumulation is float32 in tensor memory.
//
// Operand layout (K-major, no swizzle): element (r, k) of an operand with K
// extent 16 is at byte (r / 8) * 512 + (k / 4) * 128 + (r % 8) * 16 + (k % 4) * 4,
// i.e. 8-row x 16-byte core matrices, adjacent along K (leading byte offset
// 128) and 512 bytes apart along M / N (stride byte offset 512); k < 8 holds
// the hi parts of the chunk's eight samples, k >= 8 the lo parts. One MMA takes
// K = 8 (two core matrices along K).
//
// Pipeline: A and B are double-buffered; the MMAs of one chunk run while the
// threads build the next, and a buffer is rebuilt only after the mbarrier
// signalled by tcgen05.commit for the chunk that last read it. Every wait is
// bounded in time (%globaltimer): a wait that runs out makes the block stop
// issuing work, wait (again bounded) for its own MMAs in flight, free its
// tensor memory and count itself in the plan's status word, which the host
// reads with dmr_plan_status (the call's result is then not valid).
#include <algorithm>
#include <atomic>
#include <mutex>
#include <cstdint>
#include <cstdlib>

#include "kb.cuh"
#include "plan.cuh"
#include "tcgen05.cuh"

namespace dmr {

constexpr int kTcThreads = 384;       // 12 warps (384: 20.0 ms vs 21.2 with 512 and 23.2 with 256, 192^3 kooshball)
constexpr int kTcSC = 8;              // samples per MMA chunk
constexpr int kTcK = 2 * kTcSC;       // K extent of a chunk in shared memory ([hi | lo])
constexpr int kTcSB = 128;            // samples staged per pass
constexpr int kTcSBP = kTcSB + 4;     // padded row of a staged weight vector (bank spread)
constexpr int kTcMaxMT = 4;           // 128-point tiles (P <= 512)
constexpr int kTcMaxCC = 32;          // coils per block (N <= 64)
static_assert(kTcMaxCC * kTcSC <= kTcThreads, "one (coil, sample) of a chunk per thread");
constexpr int kTcPairs = (2 * kTcMaxMT * 128 + kTcThreads - 1) / kTcThreads;  // A-build pairs per thread
static_assert(kTcRowBytes == kTcK * 32, "stride between 8-row core-matrix groups");
constexpr int kTcTileBytes = 16 * kTcRowBytes;  // 8192: one 128-row operand tile
constexpr uint64_t kTcWaitNs = 200000000ull;   // bound on an operand-buffer wait (200 ms)
constexpr uint64_t kTcDrainNs = 2000000000ull; // bound on the wait before tensor memory is freed (2 s)
constexpr uint64_t kTcStallNs = 1000000ull;    // test stall: wait on a barrier nothing signals (1 ms)

__device__ int g_tc_timeouts = 0;  // blocks whose wait ran out, all plans (should stay 0)

struct TcShape {
    int R[3];    // region extents (T + W - 1)
    int P;       // points of the region
    int MT;      // 128-point tiles
    int N;       // accumulator columns per tile (2 x coils, multiple of 32)
    int ncols;   // tensor-memory columns allocated (power of two >= MT * N)
    int CC;      // coils per block
};

// dynamic shared memory: A[2] | B[2] | staged weight vectors | global sample indices
__host__ __device__ inline size_t tc_smem_bytes(const TcShape &s)
{
    return (size_t)2 * s.MT * kTcTileBytes + (size_t)2 * s.N * (kTcK * 4) +
           (size_t)(s.R[0] + s.R[1] + s.R[2]) * kTcSBP * 4 + (size_t)kTcSB * 4;
}

__global__ void __launch_bounds__(kTcThreads, 2) grid_tc_kernel(
    Geom g, TcShape sh, const WorkItem *__restrict__ work, const int32_t *__restrict__ order, int nwork, int nchunks,
    const float *__restrict__ sc0, const float *__restrict__ sc1, const float *__restrict__ sc2,
    const int32_t *__restrict__ sidx, const void *__restrict__ ksp, int kreal, float2 *__restrict__ grid,
    int64_t batch, const float *__restrict__ weight, int wpb, float inv_scale, int *__restrict__ status,
    int stall)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    // mbar[0..1]: operand buffers; mbar[2]: never signalled (test stall)
    __shared__ __align__(8) uint64_t mbar[3];
    __shared__ uint32_t tslot;
    __shared__ int s_abort;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int W = g.W[0];
    // buffer b of A at smem + b * MT * 8192, of B at bbase + b * N * 64
    unsigned char *bbase = smem + 2 * sh.MT * kTcTileBytes;
    float *vec = reinterpret_cast<float *>(bbase + 2 * sh.N * (kTcK * 4));
    float *vx = vec, *vy = vx + sh.R[0] * kTcSBP, *vz = vy + sh.R[1] * kTcSBP;
    int *gi = reinterpret_cast<int *>(vz + sh.R[2] * kTcSBP);

    // zero both operand buffers once: A rows >= P and B rows of absent coils stay zero
    {
        float4 *z = reinterpret_cast<float4 *>(smem);
        const int n16 = (2 * sh.MT * kTcTileBytes + 2 * sh.N * kTcK * 4) / 16;
        for (int e = tid; e < n16; e += kTcThreads) z[e] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem(&tslot)),
                     "r"(sh.ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&mbar[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&mbar[1])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&mbar[2])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tbase = tslot;
    const uint32_t bar0 = tc_smem(&mbar[0]);  // mbarrier of buffer b at bar0 + 8 b
    // instruction descriptor: D f32, A / B tf32, both K-major, N, M = 128
    const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(sh.N >> 3) << 17) | (8u << 24);

    const int RXY = sh.R[0] * sh.R[1];
    const int bc = tid >> 3, bs = tid & 7;  // B build: coil and sample of this thread (CC <= 32)
    // A build: pairs e = tid + 256 j of (point p = e / 2, sample quad q = e % 2); per
    // pair the byte offset of its 16-byte row slot in an A buffer and the shared
    // addresses of its x / y / z weight-vector rows (+ 16 q bytes)
    const uint32_t s0a = tc_smem(smem);
    uint32_t pa[kTcPairs], px[kTcPairs], py[kTcPairs], pz[kTcPairs];
#pragma unroll
    for (int j = 0; j < kTcPairs; j++) {
        const int e = tid + j * kTcThreads;
        const int p = min(e >> 1, sh.P - 1), q = e & 1;
        const int rz = p / RXY, rem = p - rz * RXY;
        const int ry = rem / sh.R[0], rx = rem - ry * sh.R[0];
        pa[j] = (uint32_t)((p >> 3) * kTcRowBytes + (p & 7) * 16 + q * 128);
        px[j] = tc_smem(vx) + (uint32_t)(rx * kTcSBP + 4 * q) * 4;
        py[j] = tc_smem(vy) + (uint32_t)(ry * kTcSBP + 4 * q) * 4;
        pz[j] = tc_smem(vz) + (uint32_t)(rz * kTcSBP + 4 * q) * 4;
    }
    const int npairs = 2 * sh.P;
    const uint64_t dbase = tc_desc(s0a);
    uint32_t chunk_no = 0;  // chunks issued by this block (buffer = chunk_no & 1)
    uint32_t uses0 = 0, uses1 = 0;  // commits issued per buffer

    // staging role of this thread: axis sa of sample st of a pass (384 = 3 x 128)
    static_assert(kTcThreads == 3 * kTcSB, "one (axis, sample) per thread in the staging");
    const int sa = tid / kTcSB, st = tid - sa * kTcSB;
    const float *ssc = sa == 0 ? sc0 : (sa == 1 ? sc1 : sc2);
    float *sv = sa == 0 ? vx : (sa == 1 ? vy : vz);
    const int sR = sa == 0 ? sh.R[0] : (sa == 1 ? sh.R[1] : sh.R[2]);
    const int sG = sa == 0 ? g.G[0] : (sa == 1 ? g.G[1] : g.G[2]);
    const double sihw = sa == 0 ? g.inv_hw[0] : (sa == 1 ? g.inv_hw[1] : g.inv_hw[2]);
    const float sbeta = sa == 0 ? g.beta[0] : (sa == 1 ? g.beta[1] : g.beta[2]);
    // inputs of the first pass of the next task, loaded while the current one runs
    const int ntasks = nwork * nchunks;
    WorkItem nxt = {0, 0, 0};
    float pk = 0.0f;
    int psid = -1;
    if (blockIdx.x < ntasks) {
        nxt = work[order[blockIdx.x / nchunks]];
        if (st < nxt.end - nxt.begin) {
            pk = ssc[nxt.begin + st];
            psid = sa == 0 ? sidx[nxt.begin + st] : 0;
        }
    }

    for (int task = blockIdx.x; task < ntasks; task += gridDim.x) {
        const WorkItem it = nxt;
        const float k_first = pk;
        const int sid_first = psid;
        const int ntask = task + gridDim.x;
        if (ntask < ntasks) nxt = work[order[ntask / nchunks]];
        const int64_t b0 = (int64_t)(task % nchunks) * sh.CC;
        const int cact = (int)(batch - b0 < (int64_t)sh.CC ? batch - b0 : (int64_t)sh.CC);
        const int f = it.bin / g.nbins;
        int org[3];
        {
            const int lb = it.bin - f * g.nbins;
            org[0] = (lb % g.nb[0]) * g.T[0];
            org[1] = ((lb / g.nb[0]) % g.nb[1]) * g.T[1];
            org[2] = (lb / (g.nb[0] * g.nb[1])) * g.T[2];
        }
        const int soa = sa == 0 ? org[0] : (sa == 1 ? org[1] : org[2]);
        int first = 1;  // next MMA overwrites the accumulator
        // k-space row and density-weight row of this thread's coil (B build)
        const int64_t brow = (b0 + min(bc, max(cact - 1, 0))) * g.total;
        const float2 *kc = reinterpret_cast<const float2 *>(ksp) + brow;
        const float *kr = reinterpret_cast<const float *>(ksp) + brow;
        const float *wrow = weight ? (wpb ? weight + brow : weight) : nullptr;
        for (int base = it.begin; base < it.end; base += kTcSB) {
            const int n = min(kTcSB, it.end - base);
            __syncthreads();  // previous pass done with vx / vy / vz / gi
            // stage per-axis weight vectors over the region (zero off the support)
            {
                for (int r = 0; r < sR; r++) sv[r * kTcSBP + st] = 0.0f;
                int sid = -1;
                if (st < n) {
                    const float k = base == it.begin ? k_first : ssc[base + st];
                    sid = sa == 0 ? (base == it.begin ? sid_first : sidx[base + st]) : 0;
                    const int x0 = first_tap_dev(k, W);
                    const int l = pmod(x0, sG) - soa;  // in [0, T): the sample lies in this bin
                    if (l >= 0 && l + W <= sR)
                        for (int i = 0; i < W; i++) sv[(l + i) * kTcSBP + st] = tap_weight(x0, i, k, W, sihw, sbeta);
                }
                if (sa == 0) gi[st] = sid;
            }
            // last pass of the task: fetch the next task's first-pass inputs now
            if (base + kTcSB >= it.end && ntask < ntasks && st < nxt.end - nxt.begin) {
                pk = ssc[nxt.begin + st];
                psid = sa == 0 ? sidx[nxt.begin + st] : 0;
            }
            __syncthreads();
            const int nch = (n + kTcSC - 1) / kTcSC;
            // coil-sample value of this thread for chunk ch of the pass (density-weighted)
            // (the weight is applied at use: no wait on the loads here)
            auto fetch = [&](int ch, float2 &v, float &wt) {
                v = make_float2(0.0f, 0.0f);
                wt = 1.0f;
                if (ch < nch && bc < cact) {
                    const int gidx = gi[ch * kTcSC + bs];
                    if (gidx >= 0) {
                        v = kreal ? make_float2(kr[gidx], 0.0f) : kc[gidx];
                        if (wrow) wt = wrow[gidx];
                    }
                }
            };
            float2 pv0, pv1;
            float pw0, pw1;
            fetch(0, pv0, pw0);
            fetch(1, pv1, pw1);
            for (int ch = 0; ch < nch; ch++) {
                const int buf = chunk_no & 1;
                unsigned char *abuf = smem + buf * sh.MT * kTcTileBytes;
                unsigned char *bbuf = bbase + buf * sh.N * (kTcK * 4);
                const uint32_t bar = bar0 + 8 * buf;
                const uint32_t nuse = buf ? uses1 : uses0;
                if (chunk_no >= 2) {
                    // the MMAs of chunk chunk_no - 2 read this buffer
                    if (!tc_wait(bar, nuse - 1, kTcWaitNs)) s_abort = 1;
                    // test hook: a barrier that no commit signals, so this wait runs out
                    if (stall && !tc_wait(tc_smem(&mbar[2]), 0, kTcStallNs)) s_abort = 1;
                }
                const int s0 = ch * kTcSC;
                // A: thread per (point, sample quad), addresses precomputed
                {
                    const uint32_t ab = tc_smem(abuf), vo = (uint32_t)s0 * 4;
#pragma unroll
                    for (int j = 0; j < kTcPairs; j++) {
                        if (tid + j * kTcThreads >= npairs) break;
                        const float4 x = tc_lds4(px[j] + vo);
                        const float4 y = tc_lds4(py[j] + vo);
                        const float4 z = tc_lds4(pz[j] + vo);
                        const float4 w =
                            make_float4(x.x * y.x * z.x, x.y * y.y * z.y, x.z * y.z * z.z, x.w * y.w * z.w);
                        const float4 h = make_float4(tc_hi(w.x), tc_hi(w.y), tc_hi(w.z), tc_hi(w.w));
                        tc_sts4(ab + pa[j], h);
                        tc_sts4(ab + pa[j] + 256, make_float4(w.x - h.x, w.y - h.y, w.z - h.z, w.w - h.w));
                    }
                }
                // B: thread (coil c, sample s) of the chunk; absent coils / samples are zeros
                if (tid < sh.CC * kTcSC) {
                    const float2 v = make_float2(pv0.x * pw0, pv0.y * pw0);
                    const float hx = tc_hi(v.x), hy = tc_hi(v.y);
                    // rows 2c (real) and 2c + 1 (imaginary); K: hi at s, lo at 8 + s
                    unsigned char *r0 = bbuf + ((2 * bc) >> 3) * kTcRowBytes + ((2 * bc) & 7) * 16;
                    unsigned char *r1 = r0 + 16;
                    const int ko = (bs >> 2) * 128 + (bs & 3) * 4;
                    *reinterpret_cast<float *>(r0 + ko) = hx;
                    *reinterpret_cast<float *>(r0 + ko + 256) = v.x - hx;
                    *reinterpret_cast<float *>(r1 + ko) = hy;
                    *reinterpret_cast<float *>(r1 + ko + 256) = v.y - hy;
                }
                // values of chunk ch + 2 are loaded two chunks ahead of their use
                pv0 = pv1;
                pw0 = pw1;
                fetch(ch + 2, pv1, pw1);
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncthreads();
                if (s_abort) goto done;
                if (tid == 0) {
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    // descriptors differ from the one of the smem base only in the start address
                    const uint64_t da0 = dbase + ((tc_smem(abuf) - s0a) >> 4), db0 = dbase + ((tc_smem(bbuf) - s0a) >> 4);
                    for (int mt = 0; mt < sh.MT; mt++)
#pragma unroll
                        for (int ks = 0; ks < 3; ks++) {
                            // hi*hi, hi*lo, lo*hi: K blocks at byte 0 (hi) and 256 (lo)
                            const uint64_t da = da0 + ((mt * kTcTileBytes + (ks == 2 ? 256 : 0)) >> 4);
                            const uint64_t db = db0 + (ks == 1 ? 16 : 0);
                            const uint32_t acc = (first && ks == 0) ? 0u : 1u;
                            asm volatile(
                                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(
                                    tbase + (uint32_t)(mt * sh.N)),
                                "l"(da), "l"(db), "r"(idesc), "r"(acc));
                        }
                    asm volatile(
                        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                        : "memory");
                }
                first = 0;
                if (buf) uses1++; else uses0++;
                chunk_no++;
            }
        }
        if (first) continue;  // no samples (cannot happen for a planned item)
        // epilogue: wait for the last chunk, read the accumulators, add to the grid
        {
            const int lb = (chunk_no - 1) & 1;
            if (!tc_wait(bar0 + 8 * lb, (lb ? uses1 : uses0) - 1, kTcWaitNs)) s_abort = 1;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        __syncthreads();
        if (s_abort) goto done;
        // warps (quarter, part): the accumulator columns split in nparts ranges of 16+
        int nparts = min(kTcThreads / 128, sh.N / 16);
        while ((sh.N / 16) % nparts) nparts--;
        if ((warp >> 2) < nparts) {
            const int quarter = warp & 3, half = warp >> 2;
            const int ncol = sh.N / nparts;  // columns of this warp
            for (int mt = 0; mt < sh.MT; mt++) {
                const int p = mt * 128 + quarter * 32 + lane;
                int64_t gp = -1;
                if (p < sh.P) {
                    const int rz = p / RXY, rem = p - rz * RXY;
                    const int ry = rem / sh.R[0], rx = rem - ry * sh.R[0];
                    const int px = (org[0] + rx + g.G[0] - g.half[0]) % g.G[0];
                    const int py = (org[1] + ry + g.G[1] - g.half[1]) % g.G[1];
                    const int pz = (org[2] + rz + g.G[2] - g.half[2]) % g.G[2];
                    gp = ((int64_t)pz * g.G[1] + py) * g.G[0] + px;
                }
                for (int c0 = half * ncol; c0 < (half + 1) * ncol; c0 += 16) {
                    uint32_t r[16];
                    tc_ld16(tbase + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(mt * sh.N + c0), r);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    if (gp >= 0) {
#pragma unroll
                        for (int i = 0; i < 8; i++) {
                            const int c = c0 / 2 + i;
                            const float2 v = make_float2(__uint_as_float(r[2 * i]) * inv_scale,
                                                         __uint_as_float(r[2 * i + 1]) * inv_scale);
                            if (c < cact && (v.x != 0.0f || v.y != 0.0f))
                                atomicAdd(grid + ((b0 + c) * g.nframes + f) * g.gsize + gp, v);
                        }
                    }
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        // the next task's first MMAs overwrite the accumulator after its build barrier
    }
done:
    // let the last commit land before the tensor memory is released (bounded;
    // if even this wait runs out the block is counted as failed, since its
    // MMAs may still write the columns it frees)
    if (tid == 0) {
        bool fail = s_abort != 0;
        if (chunk_no > 0) {
            const int lb = (chunk_no - 1) & 1;
            if (!tc_wait(bar0 + 8 * lb, (lb ? uses1 : uses0) - 1, kTcDrainNs)) fail = true;
        }
        if (fail) {
            atomicAdd(&g_tc_timeouts, 1);
            atomicAdd(status, 1);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(sh.ncols));
}

static int tc_disabled()
{
    static const int v = [] {
        const char *e = getenv("DMR_NO_TC");
        return e && atoi(e) ? 1 : 0;
    }();
    return v;
}

static std::atomic<int> g_tc_stall{0};  // test hook (dmr_tc_test_stall)

static int tm_disabled()
{
    static const int v = [] {
        const char *e = getenv("DMR_NO_TMEM_A");
        return e && atoi(e) ? 1 : 0;
    }();
    return v;
}

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

static bool tc_shape(const Geom &g, int64_t batch, TcShape &s)
{
    if (g.ndim != 3 || batch < 1) return false;
    const int W = g.W[0];
    if (W < 2 || g.W[1] != W || g.W[2] != W) return false;
    for (int a = 0; a < 3; a++) s.R[a] = g.T[a] + W - 1;
    s.P = s.R[0] * s.R[1] * s.R[2];
    if (s.P > kTcMaxMT * 128 || s.R[0] + s.R[1] + s.R[2] > 64) return false;
    s.MT = (s.P + 127) / 128;
    s.CC = (int)std::min<int64_t>(batch, kTcMaxCC);
    s.N = std::max(32, (2 * s.CC + 31) / 32 * 32);  // two warps split a tile's columns in 16s
    const int need = s.MT * s.N;
    s.ncols = 32;
    while (s.ncols < need) s.ncols <<= 1;
    return s.ncols <= 512;
}

// Tensor-core gridding of a 3D plan: the kernel of tmgrid.cu (atomic, or
// deterministic in colour launches), else, in atomic mode, the kernel above;
// DMR_ERR_UNSUPPORTED when neither applies (then the caller uses the
// CUDA-core kernels).
int grid_tc_dispatch(const dmr_plan *p, const void *ksp, int kreal, float2 *grid, int64_t batch,
                     const float *weight, int wpb, int det, void *scratch, size_t scratch_bytes,
                     cudaStream_t st)
{
    if (tc_disabled()) return DMR_ERR_UNSUPPORTED;
    int dev = 0;
    DMR_CUDA(cudaGetDevice(&dev));
    if (!tm_disabled()) {
        int *timeouts = nullptr;
        DMR_TRY(timeouts_ptr(dev, &timeouts));
        const int rc =
            grid_tm_dispatch(p, ksp, kreal, grid, batch, weight, wpb, det, scratch, scratch_bytes, timeouts,
                             g_tc_stall.load(), st);
        if (rc != DMR_ERR_UNSUPPORTED) return rc;
    }
    if (det) return DMR_ERR_UNSUPPORTED;  // the kernel above adds with atomics in any order
    TcShape sh;
    if (!tc_shape(p->g, batch, sh)) return DMR_ERR_UNSUPPORTED;
    int sms = 0, smem_sm = 0, smem_blk = 0, reserved = 0;
    DMR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    DMR_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    DMR_CUDA(cudaDeviceGetAttribute(&smem_blk, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    DMR_CUDA(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev));
    size_t smem = tc_smem_bytes(sh);
    DMR_CHECK(smem <= (size_t)smem_blk, DMR_ERR_UNSUPPORTED, "tensor-core gridding needs %zu B of shared memory", smem);
    {
        // the dynamic maximum leaves room for the kernel's static shared memory
        cudaFuncAttributes fa;
        DMR_CUDA(cudaFuncGetAttributes(&fa, grid_tc_kernel));
        smem_blk -= (int)fa.sharedSizeBytes;
        if (smem > (size_t)smem_blk) return DMR_ERR_UNSUPPORTED;
        DMR_CUDA(cudaFuncSetAttribute(grid_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_blk));
    }
    // (set back to the size launched below: a larger maximum can make the
    // driver reserve more shared memory and leave less L1 cache)
    // resident blocks of one SM must not ask for more than its 512 tensor-memory
    // columns (a block that found none free would wait in tcgen05.alloc until a
    // co-resident block exits): pad the dynamic shared memory until the
    // occupancy calculator admits at most 512 / ncols blocks per SM
    const int maxb = 512 / sh.ncols;
    int per_sm = 0;
    DMR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grid_tc_kernel, kTcThreads, smem));
    if (per_sm > maxb) {
        const size_t fit = (size_t)smem_sm / (maxb + 1);  // per-block share if maxb + 1 blocks fit
        smem = std::max(smem, fit > (size_t)reserved ? fit - (size_t)reserved : smem);
        DMR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grid_tc_kernel, kTcThreads, smem));
        while (per_sm > maxb && smem + 1024 <= (size_t)smem_blk) {
            smem += 1024;
            DMR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grid_tc_kernel, kTcThreads, smem));
        }
        if (per_sm > maxb) return DMR_ERR_UNSUPPORTED;
    }
    DMR_CHECK(per_sm >= 1, DMR_ERR_UNSUPPORTED, "tensor-core gridding: no resident block");
    DMR_CUDA(cudaFuncSetAttribute(grid_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    DMR_CUDA(cudaMemsetAsync(grid, 0, (size_t)batch * p->g.nframes * p->g.gsize * sizeof(float2), st));
    if (p->nwork == 0) return DMR_OK;
    const int64_t nchunks = ceil_div(batch, sh.CC);
    const int64_t tasks = (int64_t)p->nwork * nchunks;
    DMR_CHECK(tasks < (1ll << 31), DMR_ERR_UNSUPPORTED, "too many gridding tasks");
    const int blocks = (int)std::min<int64_t>(tasks, (int64_t)sms * per_sm);
    grid_tc_kernel<<<blocks, kTcThreads, smem, st>>>(p->g, sh, p->work, p->work_order, p->nwork, (int)nchunks, p->scoord[0],
                                                      p->scoord[1], p->scoord[2], p->sidx, ksp, kreal, grid,
                                                      batch, weight, wpb, (float)(1.0 / p->scale), p->status,
                                                      g_tc_stall.load());
    DMR_LAUNCHED("grid_tc_kernel");
    return DMR_OK;
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
