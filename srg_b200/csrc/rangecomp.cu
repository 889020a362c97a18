// rangecomp.cu -- range compression of decoded Sentinel-1 echo lines on the GPU.
//
// Follows sentinel/processsub.f90:86-123 in what it computes: the chirp
// replica of the decoded pulse parameters (processsub.f90:101-107, built on
// the host with the reference's types: t = (j-1)/samplefreq in FP32, the
// phase in FP64, each sample rounded to complex64 and divided by npts),
// its 32,768-point spectrum, and per line: the samples zero-padded to 32,768,
// forward FFT, times the conjugate replica spectrum, inverse FFT
// (unnormalised), the first nvalid = nsamps - npts samples kept.  The lines
// go through in blocks: one kernel pads a block, cuFFT transforms it, one
// kernel multiplies, cuFFT transforms back, one kernel writes the valid
// samples.  FFTs by cuFFT (the reference uses FFTW in single precision).
#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/srg_bp.h"
#include "host_internal.h"

using namespace srg;
using namespace srg::detail;

namespace {

constexpr int kRangeFFT = 32768;  // ranfft (processsub.f90:38)
constexpr int kBlock = 256;       // lines per transform batch

#define CKR(call)                                                                      \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            return fail(SRG_E_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));   \
    } while (0)
#define CKFR(call)                                                                     \
    do {                                                                               \
        cufftResult r_ = (call);                                                       \
        if (r_ != CUFFT_SUCCESS) return fail(SRG_E_CUDA, "%s failed: cufft %d", #call, (int)r_); \
    } while (0)

__global__ void rc_pad_kernel(const float2 *__restrict__ in, long long ld, int l0, int nlines, int nsamps,
                              float2 *__restrict__ buf) {
    const long long total = (long long)kBlock * kRangeFFT;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int l = (int)(i / kRangeFFT), n = (int)(i - (long long)l * kRangeFFT);
        float2 v = make_float2(0.f, 0.f);
        if (l0 + l < nlines && n < nsamps) v = in[(long long)(l0 + l) * ld + n];
        buf[i] = v;
    }
}

// spectrum times the conjugate replica spectrum
__global__ void rc_mul_kernel(float2 *__restrict__ buf, const float2 *__restrict__ ref) {
    const long long total = (long long)kBlock * kRangeFFT;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const float2 a = buf[i], r = ref[i & (kRangeFFT - 1)];
        buf[i] = make_float2(a.x * r.x + a.y * r.y, a.y * r.x - a.x * r.y);
    }
}

__global__ void rc_out_kernel(const float2 *__restrict__ buf, int l0, int nlines, int nvalid,
                              float2 *__restrict__ out, long long ldo) {
    const int nl = min(kBlock, nlines - l0);
    const long long total = (long long)nl * nvalid;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int l = (int)(i / nvalid), n = (int)(i - (long long)l * nvalid);
        out[(long long)(l0 + l) * ldo + n] = buf[(long long)l * kRangeFFT + n];
    }
}

struct RcCtx {
    std::mutex mu;
    cufftHandle plan_blk = 0, plan_one = 0;
    bool have_plans = false;
    DevBuf buf, ref;
    float key[4] = {NAN, NAN, NAN, NAN};  // replica parameters of `ref`
};
RcCtx g_rc[64];

int grid_of(long long n) { return (int)std::min<long long>((n + 255) / 256, 148LL * 32); }

}  // namespace

extern "C" {

int srg_range_replica(float samplefreq, float startfreq, float ramprate, float pulselength,
                      float *replica, int n, int *npts_out) {
    if (!replica || n < 1 || !(samplefreq > 0) || !(pulselength > 0))
        return fail(SRG_E_ARG, "bad replica arguments");
    const double pi = 4.0 * std::atan2(1.0, 1.0);
    const float prod = pulselength * samplefreq;  // real*4 product
    const int npts = (int)prod;                   // truncated, as the Fortran assignment
    if (npts < 1 || npts > n) return fail(SRG_E_ARG, "replica of %d samples does not fit %d", npts, n);
    std::memset(replica, 0, sizeof(float) * 2 * (size_t)n);
    for (int j = 1; j <= npts; ++j) {
        const double t = (double)((float)(j - 1) / samplefreq);
        const double phase = 2.0 * pi * (double)startfreq * t + pi * (double)ramprate * t * t;
        replica[2 * (j - 1)] = (float)std::cos(phase) / (float)npts;
        replica[2 * (j - 1) + 1] = (float)std::sin(phase) / (float)npts;
    }
    if (npts_out) *npts_out = npts;
    return SRG_OK;
}

int srg_range_compress_device(const float *lines, long long ld_in, int nlines, int nsamps,
                              float samplefreq, float startfreq, float ramprate, float pulselength,
                              float *out, long long ld_out, int *nvalid_out, void *stream) {
    if (!lines || !out || nlines < 1 || nsamps < 1 || nsamps > kRangeFFT || ld_in < nsamps)
        return fail(SRG_E_ARG, "bad range-compression sizes: nlines=%d nsamps=%d (<= %d) ld=%lld",
                    nlines, nsamps, kRangeFFT, ld_in);
    std::vector<float> rep(2 * (size_t)kRangeFFT);
    int npts = 0;
    int rc = srg_range_replica(samplefreq, startfreq, ramprate, pulselength, rep.data(), kRangeFFT, &npts);
    if (rc) return rc;
    const int nvalid = nsamps - npts;
    if (nvalid < 1) return fail(SRG_E_ARG, "pulse of %d samples leaves no valid sample of %d", npts, nsamps);
    if (ld_out < nvalid) return fail(SRG_E_ARG, "output row of %lld < %d valid samples", ld_out, nvalid);
    int dev = 0;
    CKR(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(SRG_E_ARG, "device %d out of range", dev);
    RcCtx &x = g_rc[dev];
    std::lock_guard<std::mutex> g(x.mu);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!x.have_plans) {
        CKFR(cufftPlan1d(&x.plan_blk, kRangeFFT, CUFFT_C2C, kBlock));
        CKFR(cufftPlan1d(&x.plan_one, kRangeFFT, CUFFT_C2C, 1));
        x.have_plans = true;
    }
    if ((rc = x.buf.ensure(sizeof(float2) * (size_t)kBlock * kRangeFFT)) ||
        (rc = x.ref.ensure(sizeof(float2) * (size_t)kRangeFFT)))
        return rc;
    float2 *ref = static_cast<float2 *>(x.ref.p), *buf = static_cast<float2 *>(x.buf.p);
    const float key[4] = {samplefreq, startfreq, ramprate, pulselength};
    if (std::memcmp(key, x.key, sizeof key) != 0) {
        // replica spectrum (processsub.f90:101-108)
        CKR(cudaMemcpyAsync(ref, rep.data(), sizeof(float2) * kRangeFFT, cudaMemcpyHostToDevice, st));
        CKFR(cufftSetStream(x.plan_one, st));
        CKFR(cufftExecC2C(x.plan_one, reinterpret_cast<cufftComplex *>(ref),
                          reinterpret_cast<cufftComplex *>(ref), CUFFT_FORWARD));
        CKR(cudaStreamSynchronize(st));  // `rep` is pageable host memory that goes out of scope
        std::memcpy(x.key, key, sizeof key);
    }
    CKFR(cufftSetStream(x.plan_blk, st));
    for (int l0 = 0; l0 < nlines; l0 += kBlock) {
        rc_pad_kernel<<<grid_of((long long)kBlock * kRangeFFT), 256, 0, st>>>(
            reinterpret_cast<const float2 *>(lines), ld_in, l0, nlines, nsamps, buf);
        CKR(cudaGetLastError());
        CKFR(cufftExecC2C(x.plan_blk, reinterpret_cast<cufftComplex *>(buf),
                          reinterpret_cast<cufftComplex *>(buf), CUFFT_FORWARD));
        rc_mul_kernel<<<grid_of((long long)kBlock * kRangeFFT), 256, 0, st>>>(buf, ref);
        CKR(cudaGetLastError());
        CKFR(cufftExecC2C(x.plan_blk, reinterpret_cast<cufftComplex *>(buf),
                          reinterpret_cast<cufftComplex *>(buf), CUFFT_INVERSE));
        rc_out_kernel<<<grid_of((long long)kBlock * nvalid), 256, 0, st>>>(
            buf, l0, nlines, nvalid, reinterpret_cast<float2 *>(out), ld_out);
        CKR(cudaGetLastError());
    }
    if (nvalid_out) *nvalid_out = nvalid;
    return SRG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// 2x oversampling of range lines (a finer line for the linear interpolation of
// the backprojection): even output samples are the input samples, odd ones an
// 8-tap Hann-windowed sinc at the half-sample point (taps normalised to unit
// DC gain, FP32); samples beyond the line read as 0.  2*nsamps - 1 samples
// per line.  No reference counterpart: the reference interpolates the
// original line linearly.
namespace {

__global__ void oversample2_kernel(const float2 *__restrict__ in, long long ld_in, int nlines, int nsamps,
                                   float2 *__restrict__ out, long long ld_out, float h0, float h1,
                                   float h2, float h3) {
    const int nout = 2 * nsamps - 1;
    const long long total = (long long)nlines * nout;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int l = (int)(i / nout), m = (int)(i - (long long)l * nout);
        const float2 *row = in + (long long)l * ld_in;
        float2 v;
        if ((m & 1) == 0) {
            v = row[m >> 1];
        } else {
            const int k = m >> 1;  // between samples k and k+1
            const float h[4] = {h0, h1, h2, h3};
            float re = 0.f, im = 0.f;
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const int a = k - t, b = k + 1 + t;
                const float2 sa = a >= 0 ? row[a] : make_float2(0.f, 0.f);
                const float2 sb = b < nsamps ? row[b] : make_float2(0.f, 0.f);
                re = fmaf(h[t], sa.x + sb.x, re);
                im = fmaf(h[t], sa.y + sb.y, im);
            }
            v = make_float2(re, im);
        }
        out[(long long)l * ld_out + m] = v;
    }
}

}  // namespace

extern "C" {

void srg_oversample_taps(float taps[4]) {
    const double pi = 4.0 * std::atan2(1.0, 1.0);
    double h[4], s = 0.0;
    for (int t = 0; t < 4; ++t) {
        const double x = t + 0.5;
        const double sinc = std::sin(pi * x) / (pi * x);
        const double win = 0.5 * (1.0 + std::cos(pi * x / 4.0));
        h[t] = sinc * win;
        s += 2.0 * h[t];
    }
    for (int t = 0; t < 4; ++t) taps[t] = (float)(h[t] / s);
}

int srg_oversample_range_device(const float *in, long long ld_in, int nlines, int nsamps, float *out,
                                long long ld_out, void *stream) {
    if (!in || !out || nlines < 1 || nsamps < 2 || ld_in < nsamps || ld_out < 2LL * nsamps - 1)
        return fail(SRG_E_ARG, "bad oversampling sizes: nlines=%d nsamps=%d ld_in=%lld ld_out=%lld",
                    nlines, nsamps, ld_in, ld_out);
    float h[4];
    srg_oversample_taps(h);
    const long long total = (long long)nlines * (2LL * nsamps - 1);
    oversample2_kernel<<<grid_of(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const float2 *>(in), ld_in, nlines, nsamps, reinterpret_cast<float2 *>(out),
        ld_out, h[0], h[1], h[2], h[3]);
    CKR(cudaGetLastError());
    return SRG_OK;
}

}  // extern "C"
