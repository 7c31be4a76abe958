// CG-SENSE building blocks: the SENSE + Toeplitz normal operator and a
// conjugate-gradient solver whose scalars never leave the device.
//
// Reference: EncodingOp / NUFFTGramOp / SenseOp (src/deepmr/recon/alg/linop.py:108-148,
// src/deepmr/linops/nufft.py:189-241, src/deepmr/linops/coil.py:11-205) and
// cg_solve / CGStep (src/deepmr/optim/cg.py:16-221). The reference chains
// torch operations (coil multiply, Toeplitz self-adjoint per coil, coil sum)
// and computes CG inner products in complex64; here coil expansion is fused
// into the zero-pad kernel, coil combination (+ lambda x) into the crop
// kernel, and inner products accumulate in float64 with a fixed two-stage
// reduction (bitwise reproducible, independent of what else runs on the GPU).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "plan.cuh"

namespace dmr {

std::shared_ptr<FftPlan> get_fft_plan(int ndim, const int *dims_zyx, int64_t batch, int *err);

struct PadGeom {
    int K[3], N[3];     // Toeplitz grid and image extents (x, y, z)
    int so[3], si[3], cp[3];
    int64_t ksize, isize;
};

static int fft_run(FftPlan &fp, float2 *data, int dir, void *work, cudaStream_t st)
{
    std::lock_guard<std::mutex> lk(fp.mu);
    cufftResult r = cufftSetStream(fp.handle, st);
    if (r == CUFFT_SUCCESS) r = cufftSetWorkArea(fp.handle, work);
    if (r == CUFFT_SUCCESS) r = cufftExecC2C(fp.handle, (cufftComplex *)data, (cufftComplex *)data, dir);
    DMR_CHECK(r == CUFFT_SUCCESS, DMR_ERR_CUFFT, "cufftExecC2C failed (code %d)", (int)r);
    return DMR_OK;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ float2 cmulc(float2 a, float2 b)  // conj(a) * b
{
    return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

// data[c, q] = S_c[i] * x[i] on the centred copy region of the Toeplitz grid, 0 elsewhere
__global__ void sense_pad_kernel(PadGeom g, int64_t ncoils, const float2 *__restrict__ maps,
                                 const float2 *__restrict__ x, float2 *__restrict__ data)
{
    const int64_t n = ncoils * g.ksize;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = e / g.ksize;
        const int64_t q = e - c * g.ksize;
        const int qx = (int)(q % g.K[0]);
        const int64_t t = q / g.K[0];
        const int qy = (int)(t % g.K[1]);
        const int qz = (int)(t / g.K[1]);
        const int qq[3] = {qx, qy, qz};
        bool valid = true;
        int li[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            valid = valid && qq[a] >= g.so[a] && qq[a] < g.so[a] + g.cp[a];
            li[a] = qq[a] - g.so[a] + g.si[a];
        }
        float2 v = make_float2(0.0f, 0.0f);
        if (valid) {
            const int64_t i = ((int64_t)li[2] * g.N[1] + li[1]) * g.N[0] + li[0];
            v = cmul(maps[c * g.isize + i], x[i]);
        }
        data[e] = v;
    }
}

// out[i] = sum_c conj(S_c[i]) * data[c, q(i)] + lamda * x[i], coils summed in order
__global__ void sense_crop_combine_kernel(PadGeom g, int64_t ncoils, const float2 *__restrict__ maps,
                                          const float2 *__restrict__ data, const float2 *__restrict__ x,
                                          float lamda, float2 *__restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < g.isize;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int ix = (int)(i % g.N[0]);
        const int64_t t = i / g.N[0];
        const int iy = (int)(t % g.N[1]);
        const int iz = (int)(t / g.N[1]);
        const int ii[3] = {ix, iy, iz};
        // crop: image index ii lies in the copy region of resize (K -> N)
        bool valid = true;
        int kq[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            // pad offsets so/si map image li -> grid q = li - si + so
            kq[a] = ii[a] - g.si[a] + g.so[a];
            valid = valid && ii[a] >= g.si[a] && ii[a] < g.si[a] + g.cp[a];
        }
        float2 acc = make_float2(0.0f, 0.0f);
        if (valid) {
            const int64_t q = ((int64_t)kq[2] * g.K[1] + kq[1]) * g.K[0] + kq[0];
            for (int64_t c = 0; c < ncoils; c++) {
                const float2 m = maps[c * g.isize + i];
                const float2 d = data[c * g.ksize + q];
                const float2 p = cmulc(m, d);
                acc.x += p.x;
                acc.y += p.y;
            }
        }
        if (lamda != 0.0f) {
            acc.x += lamda * x[i].x;
            acc.y += lamda * x[i].y;
        }
        out[i] = acc;
    }
}

__global__ void toep_mul_kernel(float2 *__restrict__ data, const float2 *__restrict__ kern, int64_t ksize,
                                int64_t n, float s)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x) {
        const float2 o = cmul(kern[e % ksize], data[e]);
        data[e] = make_float2(o.x * s, o.y * s);
    }
}

// ---------------------------------------------------------------------------
// conjugate gradient (cg.py:150-221) with float64 inner products
// ---------------------------------------------------------------------------
constexpr int kCgParts = 512;  // fixed partition of every reduction (deterministic)

struct CgState {
    double rsold[2];  // complex, as the reference's first dot(r, r)
    double rsnew;
    double alpha[2];
    double beta;
    double pad[2];
    double parts[2 * kCgParts];
};

// per-block partial of sum conj(a) b (or |a|^2 when b == a), fixed grid kCgParts
__global__ void cdot_partial_kernel(const float2 *__restrict__ a, const float2 *__restrict__ b, int64_t n,
                                    double *__restrict__ parts)
{
    double re = 0.0, im = 0.0;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x) {
        const float2 u = a[e], v = b[e];
        re += (double)u.x * v.x + (double)u.y * v.y;
        im += (double)u.x * v.y - (double)u.y * v.x;
    }
    __shared__ double sr[256], si[256];
    sr[threadIdx.x] = re;
    si[threadIdx.x] = im;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            sr[threadIdx.x] += sr[threadIdx.x + h];
            si[threadIdx.x] += si[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        parts[2 * blockIdx.x] = sr[0];
        parts[2 * blockIdx.x + 1] = si[0];
    }
}

__device__ __forceinline__ void sum_parts(const double *parts, double &re, double &im)
{
    re = 0.0;
    im = 0.0;
    for (int i = 0; i < kCgParts; i++) {
        re += parts[2 * i];
        im += parts[2 * i + 1];
    }
}

// mode 0: rsold = <r, r> (initialisation); 1: alpha = rsold / <p, AHAp>;
// 2: rsnew = Re<r, r>, beta = rsnew / rsold, rsold = rsnew
__global__ void cg_scalar_kernel(CgState *__restrict__ s, int mode)
{
    double re, im;
    sum_parts(s->parts, re, im);
    if (mode == 0) {
        s->rsold[0] = re;
        s->rsold[1] = im;
        s->rsnew = re;
    } else if (mode == 1) {
        const double den = re * re + im * im;  // rsold / (re + i im)
        s->alpha[0] = (s->rsold[0] * re + s->rsold[1] * im) / den;
        s->alpha[1] = (s->rsold[1] * re - s->rsold[0] * im) / den;
    } else {
        s->rsnew = re;
        // beta = rsnew / rsold with rsold complex (real after the first step)
        const double d = s->rsold[0] * s->rsold[0] + s->rsold[1] * s->rsold[1];
        s->beta = re * s->rsold[0] / d;
        s->pad[0] = -re * s->rsold[1] / d;  // imaginary part of beta (zero in exact arithmetic)
        s->rsold[0] = re;
        s->rsold[1] = 0.0;
    }
}

__global__ void cg_init_kernel(const float2 *__restrict__ ahy, float2 *__restrict__ x, float2 *__restrict__ r,
                               float2 *__restrict__ p, int64_t n)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x) {
        const float2 v = ahy[e];
        x[e] = make_float2(0.0f, 0.0f);
        r[e] = v;
        p[e] = v;
    }
}

// x += alpha p; r -= alpha q  (complex64 arithmetic like the reference)
__global__ void cg_update_xr_kernel(float2 *__restrict__ x, float2 *__restrict__ r, const float2 *__restrict__ p,
                                    const float2 *__restrict__ q, int64_t n, const CgState *__restrict__ s)
{
    const float2 a = make_float2((float)s->alpha[0], (float)s->alpha[1]);
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x) {
        const float2 ap = cmul(p[e], a);
        const float2 aq = cmul(q[e], a);
        x[e] = make_float2(x[e].x + ap.x, x[e].y + ap.y);
        r[e] = make_float2(r[e].x - aq.x, r[e].y - aq.y);
    }
}

// p = r + beta p
__global__ void cg_update_p_kernel(float2 *__restrict__ p, const float2 *__restrict__ r, int64_t n,
                                   const CgState *__restrict__ s)
{
    const float2 bt = make_float2((float)s->beta, (float)s->pad[0]);
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
         e += (int64_t)gridDim.x * blockDim.x) {
        const float2 bp = cmul(p[e], bt);
        p[e] = make_float2(r[e].x + bp.x, r[e].y + bp.y);
    }
}

static int blocks_for(int64_t n)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 256), (int64_t)sms * 8));
}

static void pad_geom(int ndim, const int32_t *kshape, const int32_t *ishape, PadGeom &g)
{
    memset(&g, 0, sizeof(g));
    g.ksize = g.isize = 1;
    for (int a = 0; a < 3; a++) {
        g.K[a] = a < ndim ? kshape[ndim - 1 - a] : 1;
        g.N[a] = a < ndim ? ishape[ndim - 1 - a] : 1;
        g.si[a] = std::max(g.N[a] / 2 - g.K[a] / 2, 0);
        g.so[a] = std::max(g.K[a] / 2 - g.N[a] / 2, 0);
        g.cp[a] = std::min(g.N[a] - g.si[a], g.K[a] - g.so[a]);
        g.ksize *= g.K[a];
        g.isize *= g.N[a];
    }
}

}  // namespace dmr

using namespace dmr;

extern "C" int dmr_sense_normal(int ndim, const int32_t *kshape, const int32_t *ishape, const void *kernel,
                                const void *maps, int64_t ncoils, const void *x, void *out, float lamda,
                                void *workspace, size_t workspace_bytes, void *stream)
{
    DMR_CHECK(ndim >= 1 && ndim <= 3 && kshape && ishape && kernel && maps && x && out && ncoils >= 1,
              DMR_ERR_INVALID, "bad argument");
    DMR_CHECK(x != out, DMR_ERR_INVALID, "x and out must not alias");
    cudaStream_t st = (cudaStream_t)stream;
    PadGeom g;
    pad_geom(ndim, kshape, ishape, g);
    int dims[3];
    for (int i = 0; i < ndim; i++) dims[i] = kshape[i];
    int err = DMR_OK;
    auto fp = get_fft_plan(ndim, dims, ncoils, &err);
    if (!fp) return err;
    const size_t a = align_up((size_t)ncoils * g.ksize * sizeof(float2), 256);
    const size_t b = align_up(fp->work_bytes, 256);
    DMR_CHECK(workspace && workspace_bytes >= a + b, DMR_ERR_WORKSPACE, "workspace too small: %zu < %zu",
              workspace_bytes, a + b);
    float2 *data = (float2 *)workspace;
    void *work = fp->work_bytes ? (char *)workspace + a : nullptr;
    const int64_t n = ncoils * g.ksize;
    sense_pad_kernel<<<blocks_for(n), 256, 0, st>>>(g, ncoils, (const float2 *)maps, (const float2 *)x, data);
    DMR_LAUNCHED("sense_pad_kernel");
    DMR_TRY(fft_run(*fp, data, CUFFT_FORWARD, work, st));
    toep_mul_kernel<<<blocks_for(n), 256, 0, st>>>(data, (const float2 *)kernel, g.ksize, n,
                                                   (float)(1.0 / (double)g.ksize));
    DMR_LAUNCHED("toep_mul_kernel");
    DMR_TRY(fft_run(*fp, data, CUFFT_INVERSE, work, st));
    sense_crop_combine_kernel<<<blocks_for(g.isize), 256, 0, st>>>(g, ncoils, (const float2 *)maps, data,
                                                                  (const float2 *)x, lamda, (float2 *)out);
    DMR_LAUNCHED("sense_crop_combine_kernel");
    return DMR_OK;
}

extern "C" int dmr_cg_state_bytes(size_t *bytes)
{
    DMR_CHECK(bytes, DMR_ERR_INVALID, "NULL argument");
    *bytes = align_up(sizeof(CgState), 256);
    return DMR_OK;
}

extern "C" int dmr_cg_init(const void *ahy, void *x, void *r, void *p, int64_t n, void *state, void *stream)
{
    DMR_CHECK(ahy && x && r && p && state && n >= 1, DMR_ERR_INVALID, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    CgState *s = (CgState *)state;
    cg_init_kernel<<<blocks_for(n), 256, 0, st>>>((const float2 *)ahy, (float2 *)x, (float2 *)r, (float2 *)p, n);
    DMR_LAUNCHED("cg_init_kernel");
    cdot_partial_kernel<<<kCgParts, 256, 0, st>>>((const float2 *)r, (const float2 *)r, n, s->parts);
    DMR_LAUNCHED("cdot_partial_kernel");
    cg_scalar_kernel<<<1, 1, 0, st>>>(s, 0);
    DMR_LAUNCHED("cg_scalar_kernel");
    return DMR_OK;
}

extern "C" int dmr_cg_step(void *x, void *r, void *p, const void *q, int64_t n, void *state, void *stream)
{
    DMR_CHECK(x && r && p && q && state && n >= 1, DMR_ERR_INVALID, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    CgState *s = (CgState *)state;
    cdot_partial_kernel<<<kCgParts, 256, 0, st>>>((const float2 *)p, (const float2 *)q, n, s->parts);
    DMR_LAUNCHED("cdot_partial_kernel");
    cg_scalar_kernel<<<1, 1, 0, st>>>(s, 1);
    DMR_LAUNCHED("cg_scalar_kernel");
    cg_update_xr_kernel<<<blocks_for(n), 256, 0, st>>>((float2 *)x, (float2 *)r, (const float2 *)p,
                                                       (const float2 *)q, n, s);
    DMR_LAUNCHED("cg_update_xr_kernel");
    cdot_partial_kernel<<<kCgParts, 256, 0, st>>>((const float2 *)r, (const float2 *)r, n, s->parts);
    DMR_LAUNCHED("cdot_partial_kernel");
    cg_scalar_kernel<<<1, 1, 0, st>>>(s, 2);
    DMR_LAUNCHED("cg_scalar_kernel");
    cg_update_p_kernel<<<blocks_for(n), 256, 0, st>>>((float2 *)p, (const float2 *)r, n, s);
    DMR_LAUNCHED("cg_update_p_kernel");
    return DMR_OK;
}

extern "C" int dmr_cg_residual(const void *state, double *rs, void *stream)
{
    DMR_CHECK(state && rs, DMR_ERR_INVALID, "bad argument");
    const CgState *s = (const CgState *)state;
    DMR_CUDA(cudaMemcpyAsync(rs, &s->rsnew, sizeof(double), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    DMR_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return DMR_OK;
}
