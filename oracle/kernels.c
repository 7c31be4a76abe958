/*
 * ORACLE — test infrastructure only, never part of the product path.
 *
 * Plain-C restatement of the CPU loops of the reference NUFFT
 * (deepmr, src/deepmr/fft/_interp/*.py), used by tests/, by the smoke check
 * and by bench.py's CPU-baseline leg to check and time the CUDA library.
 *
 * Every function follows one reference routine, cited at its definition.
 * Complex64 arrays are interleaved (re, im) float pairs, exactly like
 * torch.complex64 / numpy.complex64 memory.
 *
 * Differences from the reference that do not change results beyond fp32
 * rounding: Numba compiles with fastmath (it may contract a*b+c into FMA and
 * vectorise reductions); this file is compiled with -ffp-contract=off and
 * sums in the reference's loop order.
 */
#include <math.h>
#include <stdint.h>
#include <stddef.h>

/* Kaiser-Bessel kernel, src/deepmr/fft/_interp/plan.py:216-248.
 * I0(beta*sqrt(1-x^2)) through the Abramowitz & Stegun 9.8.1 (|x|<3.75) and
 * 9.8.2 (x>=3.75) polynomial approximations, evaluated in double precision
 * like the reference's Numba function (float64 arguments). Zero for |x|>1. */
double oracle_kb(double x, double beta)
{
    if (fabs(x) > 1.0) return 0.0;
    double a = beta * sqrt(1.0 - x * x);
    double t = a / 3.75;
    if (a < 3.75) {
        double t2 = t * t;
        return 1.0 + t2 * (3.5156229 + t2 * (3.0899424 + t2 * (1.2067492
                 + t2 * (0.2659732 + t2 * (0.0360768 + t2 * 0.0045813)))));
    }
    double u = 1.0 / t;
    double p = 0.39894228 + u * (0.01328592 + u * (0.00225319 + u * (-0.00157565
             + u * (0.00916281 + u * (-0.02057706 + u * (0.02635537
             + u * (-0.01647633 + u * 0.00392377)))))));
    return p * exp(a) / sqrt(a);
}

/* Per-axis interpolator precompute, src/deepmr/fft/_interp/plan.py:251-269:
 * x0 = ceil(k - W/2); value[i] = KB((x0+i-k)/(W/2), beta);
 * index[i] = (x0+i) mod G (Python float modulo: result in [0, G)). */
void oracle_prepare_interpolator(const float *coord, int64_t npts, int width,
                                 double beta, int gsize, float *value,
                                 int32_t *index)
{
    const double half = width / 2.0;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < npts; i++) {
        const double k = (double)coord[i];
        const double x0 = ceil(k - half);
        for (int xi = 0; xi < width; xi++) {
            value[i * width + xi] = (float)oracle_kb(((x0 + xi) - k) / half, beta);
            double m = fmod(x0 + xi, (double)gsize);
            if (m < 0) m += gsize;
            index[i * width + xi] = (int32_t)m;
        }
    }
}

/* Interpolation grid -> samples, src/deepmr/fft/_interp/interp.py:124-227.
 * cart:    (F, B, Gz, Gy, Gx) complex64 (leading spatial dims absent for ndim<3)
 * noncart: (F, B, M) complex64, accumulated into (caller zeroes it)
 * value/index[a]: per spatial axis a in (z, y, x) order, (F, M, W_a) arrays.
 * One parallel iteration per (frame, batch, point), as the reference's prange. */
void oracle_interpolate(int ndim, int64_t nframes, int64_t batch, int64_t npts,
                        const int32_t *gshape, const int32_t *width,
                        const float *cart, float *noncart,
                        const float *const *value, const int32_t *const *index)
{
    int64_t gsize = 1;
    for (int a = 0; a < ndim; a++) gsize *= gshape[a];
    const int64_t total = nframes * batch * npts;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < total; i++) {
        const int64_t frame = i / (batch * npts);
        const int64_t tmp = i % (batch * npts);
        const int64_t b = tmp / npts;
        const int64_t point = tmp % npts;
        const float *g = cart + 2 * (frame * batch + b) * gsize;
        float *out = noncart + 2 * ((frame * batch + b) * npts + point);
        float re = out[0], im = out[1];
        const int64_t row = frame * npts + point;
        if (ndim == 1) {
            const int wx = width[0];
            for (int ix = 0; ix < wx; ix++) {
                const int32_t idx = index[0][row * wx + ix];
                const float v = value[0][row * wx + ix];
                re += v * g[2 * idx];
                im += v * g[2 * idx + 1];
            }
        } else if (ndim == 2) {
            const int wy = width[0], wx = width[1];
            for (int iy = 0; iy < wy; iy++) {
                const int32_t idy = index[0][row * wy + iy];
                const float vy = value[0][row * wy + iy];
                for (int ix = 0; ix < wx; ix++) {
                    const int32_t idx = index[1][row * wx + ix];
                    const float v = vy * value[1][row * wx + ix];
                    const int64_t o = (int64_t)idy * gshape[1] + idx;
                    re += v * g[2 * o];
                    im += v * g[2 * o + 1];
                }
            }
        } else {
            const int wz = width[0], wy = width[1], wx = width[2];
            for (int iz = 0; iz < wz; iz++) {
                const int32_t idz = index[0][row * wz + iz];
                const float vz = value[0][row * wz + iz];
                for (int iy = 0; iy < wy; iy++) {
                    const int32_t idy = index[1][row * wy + iy];
                    const float vy = vz * value[1][row * wy + iy];
                    for (int ix = 0; ix < wx; ix++) {
                        const int32_t idx = index[2][row * wx + ix];
                        const float v = vy * value[2][row * wx + ix];
                        const int64_t o = ((int64_t)idz * gshape[1] + idy) * gshape[2] + idx;
                        re += v * g[2 * o];
                        im += v * g[2 * o + 1];
                    }
                }
            }
        }
        out[0] = re;
        out[1] = im;
    }
}

/* Gridding samples -> grid, src/deepmr/fft/_interp/grid.py:181-284.
 * One parallel iteration per (frame, batch); points are visited sequentially,
 * so each grid sums its contributions in sample order (deterministic), like
 * the reference's CPU path. cart is accumulated into (caller zeroes it). */
void oracle_gridding(int ndim, int64_t nframes, int64_t batch, int64_t npts,
                     const int32_t *gshape, const int32_t *width,
                     float *cart, const float *noncart,
                     const float *const *value, const int32_t *const *index)
{
    int64_t gsize = 1;
    for (int a = 0; a < ndim; a++) gsize *= gshape[a];
    const int64_t total = nframes * batch;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < total; i++) {
        const int64_t frame = i / batch;
        const int64_t b = i % batch;
        float *g = cart + 2 * (frame * batch + b) * gsize;
        const float *src = noncart + 2 * (frame * batch + b) * npts;
        for (int64_t point = 0; point < npts; point++) {
            const float sre = src[2 * point], sim = src[2 * point + 1];
            const int64_t row = frame * npts + point;
            if (ndim == 1) {
                const int wx = width[0];
                for (int ix = 0; ix < wx; ix++) {
                    const int32_t idx = index[0][row * wx + ix];
                    const float v = value[0][row * wx + ix];
                    g[2 * idx] += v * sre;
                    g[2 * idx + 1] += v * sim;
                }
            } else if (ndim == 2) {
                const int wy = width[0], wx = width[1];
                for (int iy = 0; iy < wy; iy++) {
                    const int32_t idy = index[0][row * wy + iy];
                    const float vy = value[0][row * wy + iy];
                    for (int ix = 0; ix < wx; ix++) {
                        const int32_t idx = index[1][row * wx + ix];
                        const float v = vy * value[1][row * wx + ix];
                        const int64_t o = (int64_t)idy * gshape[1] + idx;
                        g[2 * o] += v * sre;
                        g[2 * o + 1] += v * sim;
                    }
                }
            } else {
                const int wz = width[0], wy = width[1], wx = width[2];
                for (int iz = 0; iz < wz; iz++) {
                    const int32_t idz = index[0][row * wz + iz];
                    const float vz = value[0][row * wz + iz];
                    for (int iy = 0; iy < wy; iy++) {
                        const int32_t idy = index[1][row * wy + iy];
                        const float vy = vz * value[1][row * wy + iy];
                        for (int ix = 0; ix < wx; ix++) {
                            const int32_t idx = index[2][row * wx + ix];
                            const float v = vy * value[2][row * wx + ix];
                            const int64_t o = ((int64_t)idz * gshape[1] + idy) * gshape[2] + idx;
                            g[2 * o] += v * sre;
                            g[2 * o + 1] += v * sim;
                        }
                    }
                }
            }
        }
    }
}

/* Direct non-uniform DFT in double precision (no reference counterpart; it
 * is the exact operator the NUFFT approximates):
 *   y[b, p] = sum_x img[b, x] * exp(-2*pi*i * sum_d k_d[p] * (x_d - N_d//2) / N_d)
 * img: (B, Nz, Ny, Nx) complex128, coord: (M, ndim) float64 in grid units,
 * (x, y, z) order; out: (B, M) complex128. */
void oracle_nudft(int ndim, int64_t batch, int64_t npts, const int32_t *shape,
                  const double *img, const double *coord, double *out)
{
    int64_t isize = 1;
    for (int a = 0; a < ndim; a++) isize *= shape[a];
    const double twopi = 6.283185307179586476925286766559;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t p = 0; p < npts; p++) {
        double kz = 0, ky = 0, kx = 0;
        /* coord order is (x, y, z); shape order is (z, y, x) */
        kx = coord[p * ndim + 0];
        if (ndim >= 2) ky = coord[p * ndim + 1];
        if (ndim >= 3) kz = coord[p * ndim + 2];
        const int nz = ndim >= 3 ? shape[0] : 1;
        const int ny = ndim >= 2 ? shape[ndim - 2] : 1;
        const int nx = shape[ndim - 1];
        for (int64_t b = 0; b < batch; b++) {
            double sre = 0, sim = 0;
            const double *im = img + 2 * b * isize;
            for (int z = 0; z < nz; z++) {
                const double pz = ndim >= 3 ? kz * (z - nz / 2) / nz : 0.0;
                for (int y = 0; y < ny; y++) {
                    const double py = ndim >= 2 ? ky * (y - ny / 2) / ny : 0.0;
                    for (int x = 0; x < nx; x++) {
                        const double ph = -twopi * (pz + py + kx * (x - nx / 2) / nx);
                        const double c = cos(ph), s = sin(ph);
                        const int64_t o = ((int64_t)z * ny + y) * nx + x;
                        const double are = im[2 * o], aim = im[2 * o + 1];
                        sre += are * c - aim * s;
                        sim += are * s + aim * c;
                    }
                }
            }
            out[2 * (b * npts + p)] = sre;
            out[2 * (b * npts + p) + 1] = sim;
        }
    }
}
