// Kaiser-Bessel interpolation kernel of the reference
// (src/deepmr/fft/_interp/plan.py:216-248): I0(beta * sqrt(1 - u^2)) through
// the Abramowitz & Stegun 9.8.1 (argument < 3.75) and 9.8.2 (argument >= 3.75)
// polynomial approximations; zero for |u| > 1. The reference evaluates it in
// float64 and stores float32; the device version evaluates in float32
// (agreement within a few float32 ulps), the host version in float64.
#pragma once

#include <math.h>

namespace dmr {

__device__ __forceinline__ float kb_f32(float u, float beta)
{
    if (fabsf(u) > 1.0f) return 0.0f;
    const float a = beta * sqrtf(fmaxf(1.0f - u * u, 0.0f));
    if (a < 3.75f) {
        const float t = a / 3.75f;
        const float t2 = t * t;
        return 1.0f + t2 * (3.5156229f + t2 * (3.0899424f + t2 * (1.2067492f
               + t2 * (0.2659732f + t2 * (0.0360768f + t2 * 0.0045813f)))));
    }
    const float v = 3.75f / a;
    const float p = 0.39894228f + v * (0.01328592f + v * (0.00225319f + v * (-0.00157565f
                  + v * (0.00916281f + v * (-0.02057706f + v * (0.02635537f
                  + v * (-0.01647633f + v * 0.00392377f)))))));
    return p * expf(a) * rsqrtf(a);
}

// kb_f32 with both branches of I0 evaluated and one selected (the same
// arithmetic, no divergence when the lanes of a warp fall on both sides)
__device__ __forceinline__ float kb_f32_select(float u, float beta)
{
    const float a = beta * sqrtf(fmaxf(1.0f - u * u, 0.0f));
    const float t = a / 3.75f;
    const float t2 = t * t;
    const float small = 1.0f + t2 * (3.5156229f + t2 * (3.0899424f + t2 * (1.2067492f
                        + t2 * (0.2659732f + t2 * (0.0360768f + t2 * 0.0045813f)))));
    const float v = 3.75f / a;
    const float p = 0.39894228f + v * (0.01328592f + v * (0.00225319f + v * (-0.00157565f
                  + v * (0.00916281f + v * (-0.02057706f + v * (0.02635537f
                  + v * (-0.01647633f + v * 0.00392377f)))))));
    const float large = p * expf(a) * rsqrtf(a);
    const float r = a < 3.75f ? small : large;
    return fabsf(u) > 1.0f ? 0.0f : r;
}

inline double kb_f64(double u, double beta)
{
    if (fabs(u) > 1.0) return 0.0;
    const double a = beta * sqrt(1.0 - u * u);
    const double t = a / 3.75;
    if (a < 3.75) {
        const double t2 = t * t;
        return 1.0 + t2 * (3.5156229 + t2 * (3.0899424 + t2 * (1.2067492
               + t2 * (0.2659732 + t2 * (0.0360768 + t2 * 0.0045813)))));
    }
    const double v = 1.0 / t;
    const double p = 0.39894228 + v * (0.01328592 + v * (0.00225319 + v * (-0.00157565
                   + v * (0.00916281 + v * (-0.02057706 + v * (0.02635537
                   + v * (-0.01647633 + v * 0.00392377)))))));
    return p * exp(a) / sqrt(a);
}

// First tap of a sample at rescaled coordinate k: ceil(k - W/2) in float64
// (plan.py:260); truncation on a Cartesian axis (plan.py:117-121).
__device__ __forceinline__ int first_tap_dev(float k, int W)
{
    if (W == 1) return (int)k;
    return (int)ceil((double)k - 0.5 * (double)W);
}

// Kernel weight of tap i for a sample at rescaled coordinate k with first tap x0
// (plan.py:260-268): KB(((x0 + i) - k) / (W/2)); 1 on Cartesian axes.
__device__ __forceinline__ float tap_weight(int x0, int i, float k, int W, double inv_hw, float beta)
{
    if (W == 1) return 1.0f;
    const double u = ((double)(x0 + i) - (double)k) * inv_hw;
    return kb_f32((float)u, beta);
}

}  // namespace dmr
