// Trajectory gradient of the NUFFT (no counterpart in the reference, whose
// autograd returns no coordinate gradient: src/deepmr/fft/nufft.py:188-209).
//
// For y_b[p] = w_p / scale * sum_taps prod_a KB_a(u_a) K_b[taps], with
// u_a = (x0_a + i_a - k_a) / (W_a/2) and k_a = c_a * s_a + h_a (the plan's
// rescale), the derivative along coordinate axis a is
//   dy_b[p]/dc_a = w_p / scale * (-s_a / (W_a/2)) *
//                  sum_taps KB'_a(u_a) prod_{a' != a} KB_a'(u_a') K_b[taps]
// (taps fixed: the tap set changes only where k_a - W_a/2 crosses an integer).
// The kernel returns g[p, a] = sum_b Re(conj(v_b[p]) dy_b[p]/dc_a) for a
// paired k-space vector v: the forward operator's coordinate gradient with
// v = dL/dy, and (divided by prod(G)) the adjoint operator's with the grid of
// dL/dx and v = the adjoint's input.
#include <algorithm>
#include <cmath>

#include "kb.cuh"
#include "plan.cuh"

namespace dmr {

// KB(u) and dKB/du of the A&S approximation used by the reference
// (src/deepmr/fft/_interp/plan.py:216-248), differentiated term by term.
__device__ __forceinline__ float kb_and_derivative(float u, float beta, float *dkb)
{
    if (fabsf(u) > 1.0f) {
        *dkb = 0.0f;
        return 0.0f;
    }
    const float s = fmaxf(1.0f - u * u, 0.0f);
    const float a = beta * sqrtf(s);
    float i0, di0_over_a;
    if (a < 3.75f) {
        const float t = a / 3.75f;
        const float t2 = t * t;
        i0 = 1.0f + t2 * (3.5156229f + t2 * (3.0899424f + t2 * (1.2067492f
             + t2 * (0.2659732f + t2 * (0.0360768f + t2 * 0.0045813f)))));
        // d/da sum c_k t^(2k) = sum 2k c_k t^(2k-1) / 3.75; divided by a = 3.75 t
        const float p = 2.0f * 3.5156229f + t2 * (4.0f * 3.0899424f + t2 * (6.0f * 1.2067492f
                        + t2 * (8.0f * 0.2659732f + t2 * (10.0f * 0.0360768f + t2 * 12.0f * 0.0045813f))));
        di0_over_a = p / (3.75f * 3.75f);
    } else {
        const float v = 3.75f / a;
        const float P = 0.39894228f + v * (0.01328592f + v * (0.00225319f + v * (-0.00157565f
                        + v * (0.00916281f + v * (-0.02057706f + v * (0.02635537f
                        + v * (-0.01647633f + v * 0.00392377f)))))));
        const float dP = 0.01328592f + v * (2.0f * 0.00225319f + v * (3.0f * -0.00157565f
                         + v * (4.0f * 0.00916281f + v * (5.0f * -0.02057706f + v * (6.0f * 0.02635537f
                         + v * (7.0f * -0.01647633f + v * 8.0f * 0.00392377f))))));
        const float e = expf(a) * rsqrtf(a);
        i0 = P * e;
        const float di0 = e * (P * (1.0f - 0.5f / a) - dP * 3.75f / (a * a));
        di0_over_a = di0 / a;
    }
    // da/du = -beta^2 u / a
    *dkb = -beta * beta * u * di0_over_a;
    return i0;
}

// One warp per sample; lanes loop over coils. Grid in FFT order.
template <int NDIM, int WMAX>
__global__ void traj_grad_kernel(Geom g, const float *__restrict__ sc0, const float *__restrict__ sc1,
                                 const float *__restrict__ sc2, const int32_t *__restrict__ sidx,
                                 const int64_t *__restrict__ foff, const float2 *__restrict__ grid,
                                 const float2 *__restrict__ v, int64_t batch,
                                 const float *__restrict__ weight, int wpb, float inv_scale,
                                 float rs0, float rs1, float rs2, float post, float *__restrict__ out)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const float rs[3] = {rs0, rs1, rs2};
    for (int64_t j = warp; j < g.total; j += nwarps) {
        const int32_t p = sidx[j];
        int lo = 0, hi = g.nframes;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (foff[mid] <= p) lo = mid; else hi = mid;
        }
        const int f = lo;
        const float k[3] = {sc0[j], NDIM > 1 ? sc1[j] : 0.0f, NDIM > 2 ? sc2[j] : 0.0f};
        float w[3][WMAX], dw[3][WMAX];
        int idx[3][WMAX];
#pragma unroll
        for (int a = 0; a < 3; a++) {
#pragma unroll
            for (int i = 0; i < WMAX; i++) {
                w[a][i] = 0.0f;
                dw[a][i] = 0.0f;
                idx[a][i] = 0;
            }
        }
#pragma unroll
        for (int a = 0; a < NDIM; a++) {
            const int W = g.W[a];
            const int x0 = W == 1 ? (int)k[a] : (int)ceil((double)k[a] - 0.5 * (double)W);
#pragma unroll
            for (int i = 0; i < WMAX; i++) {
                if (i >= W) continue;
                idx[a][i] = pmod(x0 + i - g.half[a], g.G[a]);  // FFT-order position
                if (W == 1) {
                    w[a][i] = 1.0f;
                } else {
                    const float u = (float)(((double)(x0 + i) - (double)k[a]) * g.inv_hw[a]);
                    float d;
                    w[a][i] = kb_and_derivative(u, g.beta[a], &d);
                    // du/dc = -(1 / (W/2)) * rescale factor
                    dw[a][i] = d * (float)(-g.inv_hw[a]) * rs[a];
                }
            }
        }
        float acc[3] = {0.0f, 0.0f, 0.0f};
        for (int64_t b = lane; b < batch; b += 32) {
            const float2 *gb = grid + (b * g.nframes + f) * g.gsize;
            float2 D[3] = {make_float2(0, 0), make_float2(0, 0), make_float2(0, 0)};
            for (int iz = 0; iz < (NDIM > 2 ? g.W[2] : 1); iz++) {
                const float wz = NDIM > 2 ? w[2][iz] : 1.0f;
                const float dwz = NDIM > 2 ? dw[2][iz] : 0.0f;
                const int64_t oz = NDIM > 2 ? (int64_t)idx[2][iz] * g.G[1] * g.G[0] : 0;
                for (int iy = 0; iy < (NDIM > 1 ? g.W[1] : 1); iy++) {
                    const float wy = NDIM > 1 ? w[1][iy] : 1.0f;
                    const float dwy = NDIM > 1 ? dw[1][iy] : 0.0f;
                    const int64_t oy = oz + (NDIM > 1 ? (int64_t)idx[1][iy] * g.G[0] : 0);
#pragma unroll
                    for (int ix = 0; ix < WMAX; ix++) {
                        if (ix >= g.W[0]) continue;
                        const float2 K = gb[oy + idx[0][ix]];
                        const float cx = dw[0][ix] * wy * wz;
                        const float cy = w[0][ix] * dwy * wz;
                        const float cz = w[0][ix] * wy * dwz;
                        D[0].x += cx * K.x; D[0].y += cx * K.y;
                        D[1].x += cy * K.x; D[1].y += cy * K.y;
                        D[2].x += cz * K.x; D[2].y += cz * K.y;
                    }
                }
            }
            const int64_t o = b * g.total + p;
            const float2 vb = v[o];
            float s = inv_scale;
            if (weight) s *= weight[wpb ? o : (int64_t)p];
#pragma unroll
            for (int a = 0; a < 3; a++) acc[a] += s * (vb.x * D[a].x + vb.y * D[a].y);  // Re(conj(v) D)
        }
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int m = 16; m > 0; m >>= 1) acc[a] += __shfl_xor_sync(0xffffffffu, acc[a], m);
        if (lane < NDIM) out[(int64_t)p * NDIM + lane] = acc[lane] * post;
    }
}

int forward_grid(dmr_plan *p, const void *image, int image_real, int64_t batch, void *workspace,
                 size_t workspace_bytes, cudaStream_t st, float2 **grid_out);

}  // namespace dmr

using namespace dmr;

extern "C" int dmr_nufft_traj_grad(dmr_plan *p, const void *image, int image_real, const void *v,
                                   int64_t batch, const float *weight, int weight_per_batch,
                                   double post_scale, float *grad, void *workspace,
                                   size_t workspace_bytes, void *stream)
{
    DMR_CHECK(p && image && v && grad && batch >= 1, DMR_ERR_INVALID, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    const Geom &g = p->g;
    int wm = 1;
    for (int a = 0; a < g.ndim; a++) wm = std::max(wm, g.W[a]);
    DMR_CHECK(wm <= 8, DMR_ERR_UNSUPPORTED, "trajectory gradient supports widths up to 8");
    float2 *grid = nullptr;
    DMR_TRY(forward_grid(p, image, image_real, batch, workspace, workspace_bytes, st, &grid));
    if (g.total == 0) return DMR_OK;
    float rs[3] = {1.0f, 1.0f, 1.0f};
    for (int a = 0; a < g.ndim; a++) rs[a] = std::ceil(p->os[a] * (float)g.N[a]) / (float)g.N[a];
    const int64_t *d_foff = p->foff_dev;
    const int threads = 256;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(g.total * 32, threads), (int64_t)sms * 16));
    const float inv = (float)(1.0 / p->scale);
    const float post = (float)post_scale;
#define TG(N, W)                                                                                              \
    traj_grad_kernel<N, W><<<blocks, threads, 0, st>>>(g, p->scoord[0], p->scoord[1], p->scoord[2], p->sidx, \
                                                       d_foff, grid, (const float2 *)v, batch, weight,        \
                                                       weight_per_batch, inv, rs[0], rs[1], rs[2], post, grad)
    const int w4 = wm <= 4 ? 4 : 8;
    if (g.ndim == 1) { if (w4 == 4) TG(1, 4); else TG(1, 8); }
    else if (g.ndim == 2) { if (w4 == 4) TG(2, 4); else TG(2, 8); }
    else { if (w4 == 4) TG(3, 4); else TG(3, 8); }
#undef TG
    DMR_LAUNCHED("traj_grad_kernel");
    return DMR_OK;
}
