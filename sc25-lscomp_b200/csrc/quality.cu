// quality.cu -- the lossy quality report on the GPU (include/lscomp.h,
// lscomp_quality_u16 / _u32): PSNR and the 7x7x7 SSIM of an original stack
// and its decoded copy, with the definitions of the reference's host
// utilities (lsCOMP/src/cuLSZ_utility.cu:757-946, computePSNR and
// computeSSIM), which the reference's workflow applies to float copies of
// the data.  Values are converted to float as those copies would be.
//
//   PSNR: one pass; per-block partial sums (double) and min/max, added on
//   the host in block order.
//   SSIM: one thread per window (7x7x7, windows every 2 elements along each
//   axis), the window's statistics computed exactly as the reference does
//   (float min/max, double sums, two passes); per-block partial sums added
//   on the host in block order.  Results equal the host functions' up to the
//   order of the final sums.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <vector>
#include "lscomp.h"

namespace {

constexpr int kQThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kQThreads) psnr_kernel(const T *ori, const T *dec, unsigned long long n,
                                                         double *part, float *part_lo, float *part_hi)
{
    __shared__ double s_se[kQThreads], s_s22[kQThreads];
    __shared__ float s_lo[kQThreads], s_hi[kQThreads];
    double se = 0, s22 = 0;
    float lo = (float)ori[0], hi = lo;
    for (unsigned long long i = blockIdx.x * (unsigned long long)kQThreads + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * kQThreads) {
        const float o = (float)ori[i], d = (float)dec[i];
        lo = o < lo ? o : lo;
        hi = o > hi ? o : hi;
        const float e = fabsf(d - o);
        se += e * e;  // the product in float, the sum in double, as computePSNR does
        s22 += d * d;
    }
    s_se[threadIdx.x] = se;
    s_s22[threadIdx.x] = s22;
    s_lo[threadIdx.x] = lo;
    s_hi[threadIdx.x] = hi;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < kQThreads; k++) {
            se += s_se[k];
            s22 += s_s22[k];
            lo = s_lo[k] < lo ? s_lo[k] : lo;
            hi = s_hi[k] > hi ? s_hi[k] : hi;
        }
        part[2 * blockIdx.x] = se;
        part[2 * blockIdx.x + 1] = s22;
        part_lo[blockIdx.x] = lo;
        part_hi[blockIdx.x] = hi;
    }
}

// SSIM of the window at (o0, o1, o2) (size0 fastest), as SSIM_3d_calcWindow_float.
template <typename T>
__device__ double ssim_window(const T *x, const T *y, unsigned long long s1, unsigned long long s0, uint32_t o0,
                              uint32_t o1, uint32_t o2)
{
    constexpr int w = 7;
    int np = 0;
    const unsigned long long first = o0 + s0 * (o1 + s1 * (unsigned long long)o2);
    float xmin = (float)x[first], xmax = xmin;
    double sx = 0, sy = 0;
    for (uint32_t i2 = o2; i2 < o2 + w; i2++)
        for (uint32_t i1 = o1; i1 < o1 + w; i1++)
            for (uint32_t i0 = o0; i0 < o0 + w; i0++) {
                const unsigned long long k = i0 + s0 * (i1 + s1 * (unsigned long long)i2);
                const float a = (float)x[k], b = (float)y[k];
                xmin = a < xmin ? a : xmin;
                xmax = a > xmax ? a : xmax;
                sx += a;
                sy += b;
                np++;
            }
    const double mx = sx / np, my = sy / np;
    double vx = 0, vy = 0, cxy = 0;
    for (uint32_t i2 = o2; i2 < o2 + w; i2++)
        for (uint32_t i1 = o1; i1 < o1 + w; i1++)
            for (uint32_t i0 = o0; i0 < o0 + w; i0++) {
                const unsigned long long k = i0 + s0 * (i1 + s1 * (unsigned long long)i2);
                const double a = (float)x[k], b = (float)y[k];
                vx += (a - mx) * (a - mx);
                vy += (b - my) * (b - my);
                cxy += (a - mx) * (b - my);
            }
    vx /= np;
    vy /= np;
    cxy /= np;
    const double sdx = sqrt(vx), sdy = sqrt(vy);
    const float range = xmax - xmin;
    const double c1 = range == 0 ? 0.01 * 0.01 : 0.01 * 0.01 * range * range;
    const double c2 = range == 0 ? 0.03 * 0.03 : 0.03 * 0.03 * range * range;
    const double c3 = c2 / 2;
    const double lum = (2 * mx * my + c1) / (mx * mx + my * my + c1);
    const double con = (2 * sdx * sdy + c2) / (sdx * sdx + sdy * sdy + c2);
    const double str = (cxy + c3) / (sdx * sdy + c3);
    return lum * con * str;
}

template <typename T>
__global__ void __launch_bounds__(kQThreads) ssim_kernel(const T *x, const T *y, unsigned long long s1,
                                                         unsigned long long s0, uint32_t n0, uint32_t n1,
                                                         unsigned long long nw, double *part)
{
    __shared__ double s_sum[kQThreads];
    const unsigned long long wid = blockIdx.x * (unsigned long long)kQThreads + threadIdx.x;
    double v = 0;
    if (wid < nw) {
        const uint32_t i0 = (uint32_t)(wid % n0);
        const unsigned long long r = wid / n0;
        const uint32_t i1 = (uint32_t)(r % n1), i2 = (uint32_t)(r / n1);
        v = ssim_window<T>(x, y, s1, s0, 2 * i0, 2 * i1, 2 * i2);
    }
    s_sum[threadIdx.x] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int k = 0; k < kQThreads; k++) s += s_sum[k];  // windows in order
        part[blockIdx.x] = s;
    }
}

int status_of(cudaError_t e)
{
    if (e == cudaSuccess) return LSCOMP_OK;
    if (e == cudaErrorMemoryAllocation) return LSCOMP_ERR_NOMEM;
    return LSCOMP_ERR_CUDA;
}

template <typename T>
int quality_t(const T *ori, const T *dec, uint32_t x, uint32_t y, uint32_t z, double psnr[6], double *ssim,
              cudaStream_t st)
{
    if (!ori || !dec || !x || !y || !z || (!psnr && !ssim)) return LSCOMP_ERR_ARG;
    const unsigned long long n = (unsigned long long)x * y * z;
    if (psnr) {
        const unsigned nblk = (unsigned)((n + kQThreads - 1) / kQThreads < 4096 ? (n + kQThreads - 1) / kQThreads : 4096);
        double *d_part = nullptr;
        float *d_lo = nullptr, *d_hi = nullptr;
        cudaError_t e = cudaMalloc(&d_part, 2ull * nblk * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&d_lo, nblk * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&d_hi, nblk * sizeof(float));
        if (e == cudaSuccess) {
            psnr_kernel<T><<<nblk, kQThreads, 0, st>>>(ori, dec, n, d_part, d_lo, d_hi);
            e = cudaGetLastError();
        }
        std::vector<double> part(2ull * nblk);
        std::vector<float> lo(nblk), hi(nblk);
        if (e == cudaSuccess) e = cudaMemcpyAsync(part.data(), d_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(lo.data(), d_lo, nblk * sizeof(float), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hi.data(), d_hi, nblk * sizeof(float), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaFree(d_part);
        cudaFree(d_lo);
        cudaFree(d_hi);
        if (e != cudaSuccess) return status_of(e);
        double se = 0, s22 = 0, l = lo[0], h = hi[0];
        for (unsigned b = 0; b < nblk; b++) {
            se += part[2 * b];
            s22 += part[2 * b + 1];
            l = lo[b] < l ? lo[b] : l;
            h = hi[b] > h ? hi[b] : h;
        }
        const double mse = se / n, range = h - l;
        psnr[0] = mse;
        psnr[1] = range;
        psnr[2] = 20 * log10(range) - 10 * log10(mse);
        psnr[3] = sqrt(se);
        psnr[4] = sqrt(se) / sqrt(s22);
        psnr[5] = sqrt(mse) / range;
    }
    if (ssim) {
        // windows of 7 every 2 elements; a dimension below 7 leaves none and
        // the mean is undefined (NaN), as in the host function
        const uint32_t n0 = z >= 7 ? (z - 7) / 2 + 1 : 0, n1 = y >= 7 ? (y - 7) / 2 + 1 : 0,
                       n2 = x >= 7 ? (x - 7) / 2 + 1 : 0;
        const unsigned long long nw = (unsigned long long)n0 * n1 * n2;
        if (nw == 0) {
            *ssim = NAN;
            return LSCOMP_OK;
        }
        const unsigned long long nblk = (nw + kQThreads - 1) / kQThreads;
        if (nblk > 0x7fffffffull) return LSCOMP_ERR_TOO_LARGE;
        double *d_part = nullptr;
        cudaError_t e = cudaMalloc(&d_part, nblk * sizeof(double));
        if (e == cudaSuccess) {
            ssim_kernel<T><<<(unsigned)nblk, kQThreads, 0, st>>>(ori, dec, y, z, n0, n1, nw, d_part);
            e = cudaGetLastError();
        }
        std::vector<double> part(nblk);
        if (e == cudaSuccess) e = cudaMemcpyAsync(part.data(), d_part, nblk * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaFree(d_part);
        if (e != cudaSuccess) return status_of(e);
        double s = 0;
        for (unsigned long long b = 0; b < nblk; b++) s += part[b];
        *ssim = s / (double)nw;
    }
    return LSCOMP_OK;
}

}  // namespace

extern "C" {

int lscomp_quality_u16(const uint16_t *d_ori, const uint16_t *d_dec, uint32_t x, uint32_t y, uint32_t z,
                       double psnr[6], double *ssim, void *stream)
{
    return quality_t<uint16_t>(d_ori, d_dec, x, y, z, psnr, ssim, (cudaStream_t)stream);
}

int lscomp_quality_u32(const uint32_t *d_ori, const uint32_t *d_dec, uint32_t x, uint32_t y, uint32_t z,
                       double psnr[6], double *ssim, void *stream)
{
    return quality_t<uint32_t>(d_ori, d_dec, x, y, z, psnr, ssim, (cudaStream_t)stream);
}

}  // extern "C"
