// 3D FFT passes of the NUFFT pipelines, fused with the zero-padding /
// cropping and the apodisation, and pruned to the lines that hold data.
//
// The forward NUFFT (src/deepmr/fft/nufft.py:450-528) apodises the image,
// zero-pads it to the oversampled grid (src/deepmr/_signal/resize.py:11-102),
// and takes a centred FFT (src/deepmr/fft/fft.py:9-87); the adjoint
// (nufft.py:531-606) takes a centred inverse FFT (norm "backward", 1/G), crops
// and apodises. The grid lives in FFT order (centred index c at
// (c - G//2) mod G), so image index i of an axis sits at grid index
// (i - N//2) mod G, and only N of the G positions of an axis hold image data.
// A 3D transform is three passes of 1D transforms, and each pass touches only
// the lines that matter:
//   forward: x rows of the N1*N2 image rows (reading the image, apodising and
//   padding on the fly), y columns of the N2 planes with data (reading only
//   the N1 valid y), z columns everywhere (reading only the N2 valid z);
//   adjoint: z columns everywhere (writing only the N2 kept z), y columns of
//   the N2 kept planes (writing only the N1 kept y), x rows of the N1*N2 kept
//   rows (writing the cropped, scaled, apodised image directly).
// With G = 1.25 N that is 15.5 GB of DRAM traffic per 240^3 x 32 transform
// against 26.6 GB for a full-grid pad kernel plus three full passes.
//
// Each block transforms 16 lines at once in one shared-memory buffer
// ([position][line], line pitch 17 so that 8-byte accesses of a half-warp hit
// distinct banks): a Stockham autosort FFT (Govindaraju et al., "High performance discrete
// Fourier transforms on graphics processors", SC 2008) with radix-4, 2, 3 and
// 5 stages, twiddles from a per-length table computed in double precision on
// the host.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "plan.cuh"

namespace dmr {

namespace {

#ifndef DMR_FFT_LINES
#define DMR_FFT_LINES 16
#endif
// resident blocks per SM the compiler plans registers for: the row and column
// passes of blocks of at most 256 threads at 3 (about 80 registers; 39.5 vs
// 39.9 ms per 240^3 x 32 forward + adjoint pair at 2), larger blocks (a factor
// above 16: 320 or 384 threads) at 2, where 3 would cap them at 56-64
// registers and spill; the fused Toeplitz z pass at 2 (its forward transform,
// kernel multiply and inverse transform need the registers)
#ifndef DMR_FFT_MINB
#define DMR_FFT_MINB 3
#endif
#ifndef DMR_FFT_TOEP_MINB
#define DMR_FFT_TOEP_MINB 2
#endif
constexpr int kFftLines = DMR_FFT_LINES;  // lines per block (16 or 32)
constexpr int kFftLP = kFftLines + 2;     // shared-memory pitch of a position (16-byte rows)
constexpr int kFftShift = kFftLines == 32 ? 5 : 4;

__device__ __forceinline__ float2 cmulf(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// complex add / subtract as packed FP32 (one instruction each)
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }

// R-point DFT of v in place, V[m] = sum_q v[q] w^(q m), w = exp(-+2 pi i / R),
// for R = 2, 4 (no multiplications), 3 and 5 (roots of unity from the table
// of the transform length L)
template <int R, int L>
__device__ __forceinline__ void small_dft(float2 *v, const float2 *tw, bool inv)
{
    if constexpr (R == 2) {
        const float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 4) {
        const float2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
        const float2 s13 = cadd(v[1], v[3]), d13 = csub(v[1], v[3]);
        // w d13 with w = -i (forward) or +i (inverse)
        const float2 jd = inv ? make_float2(-d13.y, d13.x) : make_float2(d13.y, -d13.x);
        v[0] = cadd(s02, s13);
        v[1] = cadd(d02, jd);
        v[2] = csub(s02, s13);
        v[3] = csub(d02, jd);
    } else if constexpr (R == 3) {
        // w^2 = conj(w): V1,2 = v0 + Re(w) (v1 + v2) +- i Im(w) (v1 - v2)
        float2 w = tw[L / 3];
        if (inv) w.y = -w.y;
        const float2 a = make_float2(v[1].x + v[2].x, v[1].y + v[2].y);
        const float2 b = make_float2(v[1].x - v[2].x, v[1].y - v[2].y);
        const float2 m = make_float2(v[0].x + w.x * a.x, v[0].y + w.x * a.y);
        const float2 ib = make_float2(-w.y * b.y, w.y * b.x);
        v[0] = make_float2(v[0].x + a.x, v[0].y + a.y);
        v[1] = make_float2(m.x + ib.x, m.y + ib.y);
        v[2] = make_float2(m.x - ib.x, m.y - ib.y);
    } else if constexpr (R == 7) {
        // odd R: w^(R-j) = conj(w^j); a_k = v_k + v_(R-k), b_k = v_k - v_(R-k):
        // V_m, V_(R-m) = v0 + sum_k Re(w^(k m)) a_k +- i sum_k Im(w^(k m)) b_k
        constexpr int H = R / 2;
        float2 w[H + 1];
#pragma unroll
        for (int j = 1; j <= H; j++) {
            w[j] = tw[j * (L / R)];
            if (inv) w[j].y = -w[j].y;
        }
        float2 a[H + 1], b[H + 1];
#pragma unroll
        for (int k = 1; k <= H; k++) {
            a[k] = cadd(v[k], v[R - k]);
            b[k] = csub(v[k], v[R - k]);
        }
        float2 o[R];
        o[0] = v[0];
#pragma unroll
        for (int k = 1; k <= H; k++) o[0] = cadd(o[0], a[k]);
#pragma unroll
        for (int m = 1; m <= H; m++) {
            float2 re = v[0], im = make_float2(0.0f, 0.0f);
#pragma unroll
            for (int k = 1; k <= H; k++) {
                const int j = (k * m) % R;
                const float c = j <= H ? w[j].x : w[R - j].x;
                const float sn = j <= H ? w[j].y : -w[R - j].y;
                re = make_float2(re.x + c * a[k].x, re.y + c * a[k].y);
                im = make_float2(im.x + sn * b[k].x, im.y + sn * b[k].y);
            }
            // i * im = (-im.y, im.x)
            o[m] = make_float2(re.x - im.y, re.y + im.x);
            o[R - m] = make_float2(re.x + im.y, re.y - im.x);
        }
#pragma unroll
        for (int m = 0; m < R; m++) v[m] = o[m];
    } else {
        static_assert(R == 5, "radix");
        // w^4 = conj(w), w^3 = conj(w^2); a1 = v1 + v4, b1 = v1 - v4,
        // a2 = v2 + v3, b2 = v2 - v3:
        // V1,4 = v0 + Re(w) a1 + Re(w2) a2 +- i (Im(w) b1 + Im(w2) b2)
        // V2,3 = v0 + Re(w2) a1 + Re(w) a2 +- i (Im(w2) b1 - Im(w) b2)
        float2 w1 = tw[L / 5], w2 = tw[2 * (L / 5)];
        if (inv) {
            w1.y = -w1.y;
            w2.y = -w2.y;
        }
        const float2 a1 = make_float2(v[1].x + v[4].x, v[1].y + v[4].y);
        const float2 b1 = make_float2(v[1].x - v[4].x, v[1].y - v[4].y);
        const float2 a2 = make_float2(v[2].x + v[3].x, v[2].y + v[3].y);
        const float2 b2 = make_float2(v[2].x - v[3].x, v[2].y - v[3].y);
        const float2 m1 = make_float2(v[0].x + w1.x * a1.x + w2.x * a2.x, v[0].y + w1.x * a1.y + w2.x * a2.y);
        const float2 m2 = make_float2(v[0].x + w2.x * a1.x + w1.x * a2.x, v[0].y + w2.x * a1.y + w1.x * a2.y);
        const float2 s1 = make_float2(w1.y * b1.x + w2.y * b2.x, w1.y * b1.y + w2.y * b2.y);
        const float2 s2 = make_float2(w2.y * b1.x - w1.y * b2.x, w2.y * b1.y - w1.y * b2.y);
        v[0] = make_float2(v[0].x + a1.x + a2.x, v[0].y + a1.y + a2.y);
        v[1] = make_float2(m1.x - s1.y, m1.y + s1.x);
        v[4] = make_float2(m1.x + s1.y, m1.y - s1.x);
        v[2] = make_float2(m2.x - s2.y, m2.y + s2.x);
        v[3] = make_float2(m2.x + s2.y, m2.y - s2.x);
    }
}

template <int M>
struct Split {
    static constexpr int A = M % 4 == 0 ? 4 : (M % 2 == 0 ? 2 : (M % 3 == 0 ? 3 : (M % 5 == 0 ? 5 : 7)));
    static constexpr int B = M / A;
};

// M-point DFT of registers v (M divides L), natural order in and out: radix
// 2 / 3 / 4 / 5 directly, else M = A B in registers (index n = B n1 + n2):
// A-point DFTs over n1, twiddles w_M^(n2 k1), B-point DFTs over n2, output
// k1 + A k2. Every index is a compile-time constant once unrolled.
template <int M, int L>
__device__ __forceinline__ void reg_dft(float2 *v, const float2 *tw, bool inv)
{
    if constexpr (M == 2 || M == 3 || M == 4 || M == 5 || M == 7) {
        small_dft<M, L>(v, tw, inv);
    } else {
        constexpr int A = Split<M>::A, B = Split<M>::B;
        float2 y[M];
#pragma unroll
        for (int n2 = 0; n2 < B; n2++) {
            float2 a[A];
#pragma unroll
            for (int n1 = 0; n1 < A; n1++) a[n1] = v[B * n1 + n2];
            reg_dft<A, L>(a, tw, inv);
#pragma unroll
            for (int k1 = 0; k1 < A; k1++) {
                if ((n2 * k1) % M != 0) {
                    float2 w = tw[((n2 * k1) % M) * (L / M)];
                    if (inv) w.y = -w.y;
                    a[k1] = cmulf(a[k1], w);
                }
                y[n2 * A + k1] = a[k1];
            }
        }
#pragma unroll
        for (int k1 = 0; k1 < A; k1++) {
            float2 b[B];
#pragma unroll
            for (int n2 = 0; n2 < B; n2++) b[n2] = y[n2 * A + k1];
            reg_dft<B, L>(b, tw, inv);
#pragma unroll
            for (int k2 = 0; k2 < B; k2++) v[k1 + A * k2] = b[k2];
        }
    }
}

// A transform length L = L1 L2 (both at most 24, products of 2, 3, 4, 5, 7).
template <int L_, int L1_, int L2_>
struct Len {
    static constexpr int L = L_, L1 = L1_, L2 = L2_;
    // one thread per (line, column) of step A and per (line, row) of step B
    static constexpr int T = kFftLines * (L1 > L2 ? L1 : L2);
    static constexpr int MINB = T <= 256 ? DMR_FFT_MINB : 2;
    static_assert(L1 * L2 == L, "factors");
};

// Step A of the four-step transform of the block's 16 lines in buf
// ([position][line]): line c, column n2 takes positions L2 n1 + n2, an
// L1-point DFT, twiddles w_L^(n2 k1), back to positions L2 k1 + n2 (the
// positions it read: no barrier needed between its reads and writes).
// With `scale` the inputs are first multiplied by scale_line[c] * scale[position].
template <class F>
__device__ __forceinline__ void step_a(float2 *buf, const float2 *tw, bool inv, const float *scale = nullptr,
                                       const float *scale_line = nullptr)
{
    constexpr int L = F::L, L1 = F::L1, L2 = F::L2;
    const int w = threadIdx.x;
    if (w < kFftLines * L2) {
        const int c = w & (kFftLines - 1), n2 = w >> kFftShift;
        float2 a[L1];
#pragma unroll
        for (int n1 = 0; n1 < L1; n1++) a[n1] = buf[(L2 * n1 + n2) * kFftLP + c];
        if (scale) {
            const float sl = scale_line[c];
#pragma unroll
            for (int n1 = 0; n1 < L1; n1++) {
                const float sc = sl * scale[L2 * n1 + n2];
                a[n1].x *= sc;
                a[n1].y *= sc;
            }
        }
        reg_dft<L1, L>(a, tw, inv);
        // twiddles w_L^(n2 k1), index n2 k1 mod L kept incrementally
        int ti = 0;
#pragma unroll
        for (int k1 = 1; k1 < L1; k1++) {
            ti += n2;
            if (ti >= L) ti -= L;
            float2 t = tw[ti];
            if (inv) t.y = -t.y;
            a[k1] = cmulf(a[k1], t);
        }
#pragma unroll
        for (int k1 = 0; k1 < L1; k1++) buf[(L2 * k1 + n2) * kFftLP + c] = a[k1];
    }
}

// Step B for line c, row k1: positions L2 k1 + n2 (n2 < L2), an L2-point DFT;
// b[k2] is the transform at position k1 + L1 k2.
template <class F>
__device__ __forceinline__ void step_b(const float2 *buf, const float2 *tw, bool inv, int c, int k1, float2 *b)
{
    constexpr int L = F::L, L2 = F::L2;
#pragma unroll
    for (int n2 = 0; n2 < L2; n2++) b[n2] = buf[(L2 * k1 + n2) * kFftLP + c];
    reg_dft<L2, L>(b, tw, inv);
}

// the lengths with a compiled transform (grid extents of common matrix sizes
// at oversampling 1.25 and 2), as (L, L1, L2); other lengths use cuFFT
#define DMR_FFT_LENGTHS(X)                                                                            \
    X(32, 8, 4) X(40, 8, 5) X(48, 16, 3) X(56, 8, 7) X(64, 8, 8) X(80, 16, 5) X(96, 16, 6)              \
    X(112, 16, 7) X(120, 12, 10) X(128, 16, 8) X(140, 20, 7) X(144, 12, 12) X(160, 16, 10)               \
    X(168, 12, 14) X(192, 16, 12) X(200, 20, 10) X(224, 16, 14) X(240, 16, 15) X(256, 16, 16)            \
    X(280, 20, 14) X(288, 18, 16) X(320, 20, 16) X(336, 24, 14) X(384, 24, 16) X(400, 20, 20)            \
    X(480, 24, 20)

bool has_len(int L)
{
    switch (L) {
#define DMR_FFT_CASE(L, L1, L2) case L: return true;
        DMR_FFT_LENGTHS(DMR_FFT_CASE)
#undef DMR_FFT_CASE
    default: return false;
    }
}

struct FftGeom {
    int N[3], G[3];       // image / grid extents (x, y, z)
    int off[3];           // image index i sits at grid position (i + off) mod G
    int64_t nbf;          // batch * frames
    int64_t gsize, isize; // points per grid / image
    const float *apod[3]; // per-axis apodisation by image index (nullptr: 1)
    float scale;
};

__host__ __device__ __forceinline__ int wrapi(int v, int n)
{
    v %= n;
    return v < 0 ? v + n : v;
}

// whether position l of a length-L line lies in the cyclic range [q0, q0 + n)
__device__ __forceinline__ bool in_range(int l, int q0, int n, int L)
{
    int d = l - q0;
    if (d < 0) d += L;
    return d < n;
}

// asynchronous copy of `bytes` (4 or 8) into shared memory; when !valid the
// destination is zero-filled and nothing is read (src must still be mapped)
__device__ __forceinline__ void cp_async_fill(void *sdst, const void *src, int bytes, bool valid)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
    const int n = valid ? bytes : 0;
    if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Per-line data of a row tile, computed once by the first 16 threads: the
// image row offset, the grid row offset and the apodisation of the row's
// (y, z) times the scale; rows past the end get offset -1.
struct RowLine {
    int64_t img, grid;
    float s;
};

__device__ __forceinline__ void row_lines(const FftGeom &g, int64_t row0, int64_t nrows, RowLine *lines)
{
    const int c = threadIdx.x;
    if (c >= kFftLines) return;
    const int64_t row = row0 + c;
    RowLine ln;
    ln.img = -1;
    ln.grid = -1;
    ln.s = 0.0f;
    if (row < nrows) {
        const int N1 = g.N[1], N2 = g.N[2];
        const int64_t plane = (int64_t)N2 * N1;
        const int64_t bf = row / plane;
        const int rr = (int)(row - bf * plane);
        const int y = rr % N1, z = rr / N1;
        const int qy = wrapi(y + g.off[1], g.G[1]), qz = wrapi(z + g.off[2], g.G[2]);
        ln.img = bf * g.isize + (int64_t)rr * g.N[0];
        ln.grid = bf * g.gsize + ((int64_t)qz * g.G[1] + qy) * g.G[0];
        float s = g.scale;
        if (g.apod[1]) s *= g.apod[1][y];
        if (g.apod[2]) s *= g.apod[2][z];
        ln.s = s;
    }
    lines[c] = ln;
}

// Row passes (x): tiles of 16 rows, double-buffered (the next tile's loads
// are in flight while the current one is transformed); shared memory holds
// two [L][17] tiles, the twiddle table and the x apodisation.
//   forward (CROP false): image rows (real or complex) are placed at their
//   FFT-order positions (zero elsewhere), apodised, transformed and written
//   as full grid rows;
//   adjoint (CROP true): grid rows are inverse-transformed and the kept x,
//   scaled and apodised, written to the image.
template <class F, bool CROP>
__global__ void __launch_bounds__(F::T, F::MINB) fft_rows_kernel(FftGeom g, const float2 *__restrict__ tw,
                                                        const void *__restrict__ src, int src_real,
                                                        float2 *__restrict__ dst)
{
    constexpr int L = F::L, L1 = F::L1, L2 = F::L2, T = F::T;
    extern __shared__ __align__(16) float2 fsm[];
    float2 *bufs = fsm;                               // 2 x L * 17
    float2 *tws = fsm + 2 * L * kFftLP;               // L
    // L floats: the forward pass's x apodisation by grid position q (zero
    // outside the image), the adjoint's by image index i
    float *apx = reinterpret_cast<float *>(tws + L);
    __shared__ RowLine lines[2][kFftLines];
    __shared__ float line_s[2][kFftLines];
    // h0: grid position q holds image index (q + h0) mod L (when below N0)
    const int N0 = g.N[0], h0 = wrapi(-g.off[0], L);
    for (int i = threadIdx.x; i < L; i += T) {
        tws[i] = tw[i];
        if (CROP) {
            apx[i] = (g.apod[0] && i < N0) ? g.apod[0][i] : 1.0f;
        } else {
            int ii = i + h0;
            if (ii >= L) ii -= L;
            apx[i] = ii < N0 ? (g.apod[0] ? g.apod[0][ii] : 1.0f) : 0.0f;
        }
    }
    const int64_t nrows = g.nbf * g.N[2] * g.N[1];
    const int64_t ntiles = (nrows + kFftLines - 1) / kFftLines;
    // loads of tile t into buffer `slot` (line data first, so a barrier)
    auto prefetch = [&](int64_t t, int slot) {
        row_lines(g, t * kFftLines, nrows, lines[slot]);
        __syncthreads();
        if (threadIdx.x < kFftLines) line_s[slot][threadIdx.x] = lines[slot][threadIdx.x].s;
        float2 *buf = bufs + slot * L * kFftLP;
        for (int e = threadIdx.x; e < kFftLines * L; e += T) {
            const int c = e / L, q = e - c * L;
            const RowLine ln = lines[slot][c];
            float2 *d = buf + q * kFftLP + c;
            if (!CROP) {
                int i = q + h0;
                if (i >= L) i -= L;
                const bool ok = ln.img >= 0 && i < N0;
                if (src_real) {
                    const float *sp = reinterpret_cast<const float *>(src) + (ok ? ln.img + i : 0);
                    cp_async_fill(d, sp, 4, ok);
                    cp_async_fill(reinterpret_cast<float *>(d) + 1, sp, 4, false);
                } else {
                    cp_async_fill(d, reinterpret_cast<const float2 *>(src) + (ok ? ln.img + i : 0), 8, ok);
                }
            } else {
                const bool ok = ln.grid >= 0;
                cp_async_fill(d, reinterpret_cast<const float2 *>(src) + (ok ? ln.grid + q : 0), 8, ok);
            }
        }
        cp_async_commit();
    };
    int64_t t = blockIdx.x;
    if (t < ntiles) prefetch(t, 0);
    for (int it = 0; t < ntiles; t += gridDim.x, it++) {
        const int cur = it & 1;
        float2 *buf = bufs + cur * L * kFftLP;
        if (t + gridDim.x < ntiles) prefetch(t + gridDim.x, cur ^ 1);
        else cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        // forward: apodisation (position q of line c holds image index
        // (q + N0/2) mod L, or zero) applied as step A reads its inputs
        if (CROP) step_a<F>(buf, tws, true);
        else step_a<F>(buf, tws, false, apx, line_s[cur]);
        __syncthreads();
        // step B into registers, then (after every thread has read its
        // inputs) back into the tile in transform order
        const int w = threadIdx.x;
        const int c = w & (kFftLines - 1), k1 = w >> kFftShift;
        float2 b[L2];
        if (k1 < L1) step_b<F>(buf, tws, CROP, c, k1, b);
        __syncthreads();
        if (k1 < L1) {
#pragma unroll
            for (int k2 = 0; k2 < L2; k2++) buf[(k1 + L1 * k2) * kFftLP + c] = b[k2];
        }
        __syncthreads();
        if (!CROP) {
            for (int e = threadIdx.x; e < kFftLines * L; e += T) {
                const int cc = e / L, l = e - cc * L;
                const int64_t go = lines[cur][cc].grid;
                if (go >= 0) dst[go + l] = buf[l * kFftLP + cc];
            }
        } else {
            for (int e = threadIdx.x; e < kFftLines * N0; e += T) {
                const int cc = e / N0, i = e - cc * N0;
                const RowLine ln = lines[cur][cc];
                if (ln.img < 0) continue;
                int q = i - h0;
                if (q < 0) q += L;
                float2 v = buf[q * kFftLP + cc];
                const float sc = ln.s * apx[i];
                v.x *= sc;
                v.y *= sc;
                dst[ln.img + i] = v;
            }
        }
        // the tile's buffer is loaded again two iterations on
        __syncthreads();
    }
    cp_async_wait<0>();
}

// Column pass along y or z, in place on the grid: tiles of 16 consecutive x
// of one line set (batch*frame, outer index), the line running along the axis
// with element stride S. Input positions outside [in_q0, in_q0 + in_n)
// (cyclic) are zero and not read; outputs outside [out_q0, out_q0 + out_n)
// are not written. Outer index k in [0, nouter) selects plane / row
// (outer_q0 + k) mod outer_G with stride outer_stride. Double-buffered like
// the row passes; step B writes straight to the grid (16 consecutive x per
// half-warp).
struct ColArgs {
    int64_t S, outer_stride;
    int nouter, outer_q0, outer_G;
    int in_q0, in_n, out_q0, out_n;
    int inv;
};

template <class F, bool IN_ALL, bool OUT_ALL>
__global__ void __launch_bounds__(F::T, F::MINB) fft_cols_kernel(FftGeom g, ColArgs a, const float2 *__restrict__ tw,
                                                        float2 *grid)
{
    constexpr int L = F::L, L1 = F::L1, L2 = F::L2, T = F::T;
    extern __shared__ __align__(16) float2 fsm[];
    float2 *bufs = fsm, *tws = fsm + 2 * L * kFftLP;
    for (int i = threadIdx.x; i < L; i += T) tws[i] = tw[i];
    const int G0 = g.G[0];
    const int ntx = (G0 + kFftLines - 1) / kFftLines;
    const int64_t ntiles = g.nbf * a.nouter * ntx;
    const bool inv = a.inv != 0;
    // first x and base pointer of tile t
    auto tile = [&](int64_t t, int &x0) -> float2 * {
        const int tx = (int)(t % ntx);
        const int64_t rest = t / ntx;
        const int k = (int)(rest % a.nouter);
        const int64_t bf = rest / a.nouter;
        int qo = a.outer_q0 + k;
        if (qo >= a.outer_G) qo -= a.outer_G;
        x0 = tx * kFftLines;
        return grid + bf * g.gsize + (int64_t)qo * a.outer_stride + x0;
    };
    auto prefetch = [&](int64_t t, int slot) {
        int x0;
        const float2 *base = tile(t, x0);
        float2 *buf = bufs + slot * L * kFftLP;
        // pairs of x (16 bytes; grid extents are even, so a pair never
        // straddles the end of a row)
        constexpr int P = kFftLines / 2;
        for (int e = threadIdx.x; e < P * L; e += T) {
            const int l = e / P, c = 2 * (e - l * P);
            const bool ok = x0 + c < G0 && (IN_ALL || in_range(l, a.in_q0, a.in_n, L));
            const unsigned d = (unsigned)__cvta_generic_to_shared(buf + l * kFftLP + c);
            const float2 *sp = ok ? base + (int64_t)l * a.S + c : base;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(sp), "r"(ok ? 16 : 0)
                         : "memory");
        }
        cp_async_commit();
    };
    int64_t t = blockIdx.x;
    if (t < ntiles) prefetch(t, 0);
    for (int it = 0; t < ntiles; t += gridDim.x, it++) {
        const int cur = it & 1;
        float2 *buf = bufs + cur * L * kFftLP;
        if (t + gridDim.x < ntiles) prefetch(t + gridDim.x, cur ^ 1);
        else cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        step_a<F>(buf, tws, inv);
        __syncthreads();
        const int w = threadIdx.x;
        const int c = w & (kFftLines - 1), k1 = w >> kFftShift;
        int x0;
        float2 *base = tile(t, x0);
        if (k1 < L1 && x0 + c < G0) {
            float2 b[L2];
            step_b<F>(buf, tws, inv, c, k1, b);
#pragma unroll
            for (int k2 = 0; k2 < L2; k2++) {
                const int l = k1 + L1 * k2;
                if (OUT_ALL || in_range(l, a.out_q0, a.out_n, L)) base[(int64_t)l * a.S + c] = b[k2];
            }
        }
        // the tile's buffer is loaded again two iterations on
        __syncthreads();
    }
    cp_async_wait<0>();
}

// Toeplitz z pass: per tile of 16 x of one (batch, y), the z columns (reading
// the N2 z with data only), forward FFT, times kernel[b mod nk][z][y][x] *
// kscale, inverse FFT, and the N2 kept z written back; nothing leaves shared
// memory between the two transforms. Tiles run batch-fastest, so the blocks
// that read one kernel tile run together and share it in L2.
template <class F>
__global__ void __launch_bounds__(F::T, DMR_FFT_TOEP_MINB) fft_toep_z_kernel(FftGeom g, ColArgs a, int64_t nk,
                                                          const float2 *__restrict__ kern, float kscale,
                                                          const float2 *__restrict__ tw, float2 *grid)
{
    constexpr int L = F::L, L1 = F::L1, L2 = F::L2, T = F::T;
    extern __shared__ __align__(16) float2 fsm[];
    float2 *bufs = fsm, *tws = fsm + 2 * L * kFftLP;
    for (int i = threadIdx.x; i < L; i += T) tws[i] = tw[i];
    const int G0 = g.G[0];
    const int ntx = (G0 + kFftLines - 1) / kFftLines;
    const int64_t ntiles = g.nbf * a.nouter * ntx;
    // batch index, first x, and the tile's offset in a grid (y row a.outer)
    auto tile = [&](int64_t t, int64_t &bf, int &x0) -> int64_t {
        bf = t % g.nbf;
        const int64_t rest = t / g.nbf;
        const int tx = (int)(rest % ntx);
        const int k = (int)(rest / ntx);
        x0 = tx * kFftLines;
        return (int64_t)k * a.outer_stride + x0;
    };
    auto prefetch = [&](int64_t t, int slot) {
        int64_t bf;
        int x0;
        const float2 *base = grid + tile(t, bf, x0) + bf * g.gsize;
        float2 *buf = bufs + slot * L * kFftLP;
        constexpr int P = kFftLines / 2;
        for (int e = threadIdx.x; e < P * L; e += T) {
            const int l = e / P, c = 2 * (e - l * P);
            const bool ok = x0 + c < G0 && in_range(l, a.in_q0, a.in_n, L);
            const unsigned d = (unsigned)__cvta_generic_to_shared(buf + l * kFftLP + c);
            const float2 *sp = ok ? base + (int64_t)l * a.S + c : base;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(sp), "r"(ok ? 16 : 0)
                         : "memory");
        }
        cp_async_commit();
    };
    int64_t t = blockIdx.x;
    if (t < ntiles) prefetch(t, 0);
    for (int it = 0; t < ntiles; t += gridDim.x, it++) {
        const int cur = it & 1;
        float2 *buf = bufs + cur * L * kFftLP;
        if (t + gridDim.x < ntiles) prefetch(t + gridDim.x, cur ^ 1);
        else cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        int64_t bf;
        int x0;
        const int64_t to = tile(t, bf, x0);
        const int w = threadIdx.x;
        const int c = w & (kFftLines - 1), k1 = w >> kFftShift;
        // forward transform back into the tile (transform order)
        step_a<F>(buf, tws, false);
        __syncthreads();
        float2 b[L2];
        if (k1 < L1) step_b<F>(buf, tws, false, c, k1, b);
        __syncthreads();
        if (k1 < L1) {
#pragma unroll
            for (int k2 = 0; k2 < L2; k2++) buf[(k1 + L1 * k2) * kFftLP + c] = b[k2];
        }
        __syncthreads();
        // kernel multiply
        const float2 *kb = kern + (bf % nk) * g.gsize + to;
        for (int e = threadIdx.x; e < kFftLines * L; e += T) {
            const int l = e >> kFftShift, cc = e & (kFftLines - 1);
            if (x0 + cc < G0) {
                const float2 kv = kb[(int64_t)l * a.S + cc];
                float2 &v = buf[l * kFftLP + cc];
                const float2 m = cmulf(kv, v);
                v = make_float2(m.x * kscale, m.y * kscale);
            }
        }
        __syncthreads();
        // inverse transform, kept z to the grid
        step_a<F>(buf, tws, true);
        __syncthreads();
        if (k1 < L1 && x0 + c < G0) {
            step_b<F>(buf, tws, true, c, k1, b);
            float2 *base = grid + bf * g.gsize + to;
#pragma unroll
            for (int k2 = 0; k2 < L2; k2++) {
                const int l = k1 + L1 * k2;
                if (in_range(l, a.out_q0, a.out_n, L)) base[(int64_t)l * a.S + c] = b[k2];
            }
        }
        // the tile's buffer is loaded again two iterations on
        __syncthreads();
    }
    cp_async_wait<0>();
}

// per-device twiddle tables exp(-2 pi i t / L), t in [0, L), from double precision
std::mutex g_tw_mu;
std::map<std::pair<int, int>, float2 *> g_tw;

int twiddles(int L, const float2 **out)
{
    int dev = 0;
    DMR_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_tw_mu);
    auto key = std::make_pair(dev, L);
    auto it = g_tw.find(key);
    if (it != g_tw.end()) {
        *out = it->second;
        return DMR_OK;
    }
    std::vector<float2> h(L);
    const double two_pi = 6.283185307179586476925286766559;
    for (int t = 0; t < L; t++) {
        const double ang = two_pi * (double)t / (double)L;
        h[t] = make_float2((float)std::cos(ang), (float)-std::sin(ang));
    }
    float2 *d = nullptr;
    DMR_CUDA(cudaMalloc(&d, L * sizeof(float2)));
    DMR_CUDA(cudaMemcpy(d, h.data(), L * sizeof(float2), cudaMemcpyHostToDevice));
    g_tw[key] = d;
    *out = d;
    return DMR_OK;
}

int fft_disabled()
{
    static const int v = [] {
        const char *e = getenv("DMR_CUFFT");
        return e && atoi(e) ? 1 : 0;
    }();
    return v;
}

// two tiles, the twiddle table and the x apodisation (row passes)
size_t smem_bytes(int L) { return (size_t)(2 * L * kFftLP + L) * sizeof(float2) + L * sizeof(float); }

// grid size for a kernel looping over `ntiles` tiles: a few waves of resident blocks
int blocks_for(const void *kern, int threads, size_t smem, int64_t ntiles, int *blocks)
{
    int dev = 0, sms = 0, per_sm = 0;
    DMR_CUDA(cudaGetDevice(&dev));
    DMR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    DMR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    DMR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
    DMR_CHECK(per_sm >= 1, DMR_ERR_UNSUPPORTED, "FFT pass does not fit on an SM");
    const int64_t cap = (int64_t)sms * per_sm;
    *blocks = (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, cap));
    return DMR_OK;
}

template <class F, bool IN_ALL, bool OUT_ALL>
int launch_cols_tt(const FftGeom &g, const ColArgs &a, const float2 *tw, float2 *grid, cudaStream_t st)
{
    const size_t smem = smem_bytes(F::L);
    const int64_t ntiles = g.nbf * a.nouter * ((g.G[0] + kFftLines - 1) / kFftLines);
    if (ntiles == 0) return DMR_OK;
    int blocks = 0;
    DMR_TRY(blocks_for((const void *)fft_cols_kernel<F, IN_ALL, OUT_ALL>, F::T, smem, ntiles, &blocks));
    fft_cols_kernel<F, IN_ALL, OUT_ALL><<<blocks, F::T, smem, st>>>(g, a, tw, grid);
    DMR_LAUNCHED("fft_cols_kernel");
    return DMR_OK;
}

// the forward passes read part of each line and write all of it, the
// adjoint passes the other way round
template <class F>
int launch_cols_t(const FftGeom &g, const ColArgs &a, const float2 *tw, float2 *grid, cudaStream_t st)
{
    const int L = F::L;
    if (a.out_n == L) return launch_cols_tt<F, false, true>(g, a, tw, grid, st);
    if (a.in_n == L) return launch_cols_tt<F, true, false>(g, a, tw, grid, st);
    return launch_cols_tt<F, false, false>(g, a, tw, grid, st);
}

template <class F, bool CROP>
int launch_rows_t(const FftGeom &g, const float2 *tw, const void *src, int src_real, float2 *dst, cudaStream_t st)
{
    const size_t smem = smem_bytes(F::L);
    const int64_t ntiles = (g.nbf * g.N[2] * g.N[1] + kFftLines - 1) / kFftLines;
    if (ntiles == 0) return DMR_OK;
    int blocks = 0;
    DMR_TRY(blocks_for((const void *)fft_rows_kernel<F, CROP>, F::T, smem, ntiles, &blocks));
    fft_rows_kernel<F, CROP><<<blocks, F::T, smem, st>>>(g, tw, src, src_real, dst);
    DMR_LAUNCHED(CROP ? "fft_crop_rows_kernel" : "fft_pad_rows_kernel");
    return DMR_OK;
}

template <class F>
int launch_toep_z_t(const FftGeom &g, const ColArgs &a, int64_t nk, const float2 *kern, float kscale,
                    const float2 *tw, float2 *grid, cudaStream_t st)
{
    const size_t smem = smem_bytes(F::L);
    const int64_t ntiles = g.nbf * a.nouter * ((g.G[0] + kFftLines - 1) / kFftLines);
    if (ntiles == 0) return DMR_OK;
    int blocks = 0;
    DMR_TRY(blocks_for((const void *)fft_toep_z_kernel<F>, F::T, smem, ntiles, &blocks));
    fft_toep_z_kernel<F><<<blocks, F::T, smem, st>>>(g, a, nk, kern, kscale, tw, grid);
    DMR_LAUNCHED("fft_toep_z_kernel");
    return DMR_OK;
}

int launch_toep_z(int L, const FftGeom &g, const ColArgs &a, int64_t nk, const float2 *kern, float kscale,
                  const float2 *tw, float2 *grid, cudaStream_t st)
{
    switch (L) {
#define DMR_FFT_CASE(L, L1, L2) case L: return launch_toep_z_t<Len<L, L1, L2>>(g, a, nk, kern, kscale, tw, grid, st);
        DMR_FFT_LENGTHS(DMR_FFT_CASE)
#undef DMR_FFT_CASE
    default: return DMR_ERR_UNSUPPORTED;
    }
}

int launch_cols(int L, const FftGeom &g, const ColArgs &a, const float2 *tw, float2 *grid, cudaStream_t st)
{
    switch (L) {
#define DMR_FFT_CASE(L, L1, L2) case L: return launch_cols_t<Len<L, L1, L2>>(g, a, tw, grid, st);
        DMR_FFT_LENGTHS(DMR_FFT_CASE)
#undef DMR_FFT_CASE
    default: return DMR_ERR_UNSUPPORTED;
    }
}

int launch_rows(int L, bool crop, const FftGeom &g, const float2 *tw, const void *src, int src_real, float2 *dst,
                cudaStream_t st)
{
    switch (L) {
#define DMR_FFT_CASE(L, L1, L2)                                                                     \
    case L:                                                                                         \
        return crop ? launch_rows_t<Len<L, L1, L2>, true>(g, tw, src, src_real, dst, st)            \
                    : launch_rows_t<Len<L, L1, L2>, false>(g, tw, src, src_real, dst, st);
        DMR_FFT_LENGTHS(DMR_FFT_CASE)
#undef DMR_FFT_CASE
    default: return DMR_ERR_UNSUPPORTED;
    }
}

FftGeom make_geom(const dmr_plan *p, int64_t batch, float scale)
{
    const Geom &gg = p->g;
    FftGeom g;
    for (int a = 0; a < 3; a++) {
        g.N[a] = gg.N[a];
        g.G[a] = gg.G[a];
        g.apod[a] = gg.W[a] != 1 ? p->apod[a] : nullptr;
        g.off[a] = -(gg.N[a] / 2);  // FFT order: centred index N/2 at 0
    }
    g.nbf = batch * gg.nframes;
    g.gsize = gg.gsize;
    g.isize = gg.isize;
    g.scale = scale;
    return g;
}

ColArgs y_pass(const FftGeom &g, bool inv)
{
    // y columns of the N2 planes that hold data; the forward reads the N1
    // valid y only, the adjoint writes the N1 kept y only
    ColArgs a;
    a.S = g.G[0];
    a.outer_stride = (int64_t)g.G[0] * g.G[1];
    a.nouter = g.N[2];
    a.outer_q0 = wrapi(g.off[2], g.G[2]);
    a.outer_G = g.G[2];
    const int q0 = wrapi(g.off[1], g.G[1]);
    a.in_q0 = inv ? 0 : q0;
    a.in_n = inv ? g.G[1] : g.N[1];
    a.out_q0 = inv ? q0 : 0;
    a.out_n = inv ? g.N[1] : g.G[1];
    a.inv = inv;
    return a;
}

ColArgs z_pass(const FftGeom &g, bool inv)
{
    // z columns of every (y, x); the forward reads the N2 valid z only, the
    // adjoint writes the N2 kept z only
    ColArgs a;
    a.S = (int64_t)g.G[0] * g.G[1];
    a.outer_stride = g.G[0];
    a.nouter = g.G[1];
    a.outer_q0 = 0;
    a.outer_G = g.G[1];
    const int q0 = wrapi(g.off[2], g.G[2]);
    a.in_q0 = inv ? 0 : q0;
    a.in_n = inv ? g.G[2] : g.N[2];
    a.out_q0 = inv ? q0 : 0;
    a.out_n = inv ? g.N[2] : g.G[2];
    a.inv = inv;
    return a;
}

}  // namespace

bool fft3_applies(const dmr_plan *p)
{
    const Geom &g = p->g;
    if (fft_disabled() || (g.ndim != 2 && g.ndim != 3)) return false;
    for (int a = 0; a < g.ndim; a++)
        if (g.G[a] < g.N[a] || !has_len(g.G[a])) return false;
    return true;
}

// apodise + zero-pad + forward 3D FFT of `image` into `grid` (FFT order)
int fft3_forward(const dmr_plan *p, const void *image, int image_real, int64_t batch, float2 *grid,
                 cudaStream_t st)
{
    const FftGeom g = make_geom(p, batch, 1.0f);
    const float2 *tw[3] = {nullptr, nullptr, nullptr};
    for (int a = 0; a < p->g.ndim; a++) DMR_TRY(twiddles(g.G[a], &tw[a]));
    if (g.nbf == 0) return DMR_OK;
    DMR_TRY(launch_rows(g.G[0], false, g, tw[0], image, image_real, grid, st));
    DMR_TRY(launch_cols(g.G[1], g, y_pass(g, false), tw[1], grid, st));
    if (g.G[2] == 1) return DMR_OK;  // 2D
    return launch_cols(g.G[2], g, z_pass(g, false), tw[2], grid, st);
}

// inverse 3D FFT of `grid` (FFT order, overwritten) + crop + 1/G + apodisation into `image`
int fft3_adjoint(const dmr_plan *p, float2 *grid, int64_t batch, float2 *image, cudaStream_t st)
{
    const FftGeom g = make_geom(p, batch, (float)(1.0 / (double)p->g.gsize));
    const float2 *tw[3] = {nullptr, nullptr, nullptr};
    for (int a = 0; a < p->g.ndim; a++) DMR_TRY(twiddles(g.G[a], &tw[a]));
    if (g.nbf == 0) return DMR_OK;
    if (g.G[2] > 1) DMR_TRY(launch_cols(g.G[2], g, z_pass(g, true), tw[2], grid, st));
    DMR_TRY(launch_cols(g.G[1], g, y_pass(g, true), tw[1], grid, st));
    return launch_rows(g.G[0], true, g, tw[0], grid, 0, image, st);
}

bool toep3_applies(int ndim, const int32_t *kshape, const int32_t *ishape)
{
    if (fft_disabled() || (ndim != 2 && ndim != 3) || !kshape || !ishape) return false;
    for (int a = 0; a < ndim; a++)
        if (kshape[a] < ishape[a] || !has_len(kshape[a])) return false;
    return true;
}

// Toeplitz self-adjoint of a 3D image batch (src/deepmr/fft/nufft.py:609-669,
// _interp/toeplitz.py:84-87): zero-pad to the kernel grid (resize offsets
// K/2 - N/2, no shift), FFT, times kernel[b mod nk] / K (the two orthonormal
// 1/sqrt(K)), inverse FFT, crop; `data` is a workspace of batch kernel grids.
int fft3_toeplitz(int ndim, const int32_t *kshape_zyx, const int32_t *ishape_zyx, const float2 *kernel, int64_t nk,
                  const void *image, int image_real, float2 *out, int64_t batch, float2 *data, cudaStream_t st)
{
    FftGeom g;
    g.gsize = g.isize = 1;
    for (int a = 0; a < 3; a++) {
        g.G[a] = a < ndim ? kshape_zyx[ndim - 1 - a] : 1;
        g.N[a] = a < ndim ? ishape_zyx[ndim - 1 - a] : 1;
        g.off[a] = g.G[a] / 2 - g.N[a] / 2;
        g.apod[a] = nullptr;
        g.gsize *= g.G[a];
        g.isize *= g.N[a];
    }
    g.nbf = batch;
    g.scale = 1.0f;
    const float2 *tw[3] = {nullptr, nullptr, nullptr};
    for (int a = 0; a < ndim; a++) DMR_TRY(twiddles(g.G[a], &tw[a]));
    if (batch == 0) return DMR_OK;
    const float kscale = (float)(1.0 / (double)g.gsize);
    DMR_TRY(launch_rows(g.G[0], false, g, tw[0], image, image_real, data, st));
    if (ndim == 2) {
        // the y pass is the fused one: its lines with data in, kept lines out
        ColArgs y = y_pass(g, false);
        y.out_q0 = y.in_q0;
        y.out_n = y.in_n;
        DMR_TRY(launch_toep_z(g.G[1], g, y, nk, kernel, kscale, tw[1], data, st));
    } else {
        DMR_TRY(launch_cols(g.G[1], g, y_pass(g, false), tw[1], data, st));
        ColArgs z = z_pass(g, false);
        z.out_q0 = z.in_q0;
        z.out_n = z.in_n;  // only the kept z leave the fused transform
        DMR_TRY(launch_toep_z(g.G[2], g, z, nk, kernel, kscale, tw[2], data, st));
        DMR_TRY(launch_cols(g.G[1], g, y_pass(g, true), tw[1], data, st));
    }
    return launch_rows(g.G[0], true, g, tw[0], data, 0, out, st);
}

}  // namespace dmr

extern "C" int dmr_fft3_fused(dmr_plan *plan) { return plan && dmr::fft3_applies(plan) ? 1 : 0; }
