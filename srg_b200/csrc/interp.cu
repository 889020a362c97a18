// interp.cu -- expected error of the backprojection's range interpolation,
// estimated from the range lines' own spectrum; the autotuner's choice
// between interpolating the original lines and 2x-oversampled ones.
//
// Every term interpolates its range line linearly between the two bins
// around the term's range (sentinel/azimuth_compress.cu:65-69, the
// reference's only interpolation).  For a line with power spectrum P(nu)
// (nu in cycles per sample) and a fractional offset u uniform in [0, 1), the
// interpolated value differs from the band-limited line at that point by
//   H_u(nu) = (1 - u) + u e^{i 2 pi nu} - e^{i 2 pi nu u}
// per unit of spectrum, so the relative RMS error is
//   sqrt( sum_nu P(nu) <|H_u(nu)|^2>_u / sum_nu P(nu) ).
// On a 2x-oversampled line (srg_oversample_range_device: even samples the
// original, odd ones the 8-tap filter G(nu) at the half-sample point) the
// term interpolates between an original sample and a filtered one, on a grid
// of half a bin:
//   even start: (1 - u) + u G(nu)          against e^{i pi nu u}
//   odd start:  (1 - u) G(nu) + u e^{i 2 pi nu}  against e^{i pi nu (1 + u)}.
// The error a term adds is a random complex vector; its component across
// the signal, the phase error, carries half the power: phase RMS (rad) =
// relative RMS / sqrt(2).  The spectrum is the mean |FFT|^2 of a sample of
// lines zero-padded to a power of two (cuFFT).
#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <complex>
#include <vector>

#include "host_internal.h"

using namespace srg;
using namespace srg::detail;

namespace {

__global__ void ie_pad_kernel(const float2 *__restrict__ in, long long ld, int nlines, int nsample,
                              int nsamps, int nfft, float2 *__restrict__ buf) {
    const long long total = (long long)nsample * nfft;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(i / nfft), n = (int)(i - (long long)q * nfft);
        const long long line = (long long)q * nlines / nsample;  // evenly spread sample
        buf[i] = n < nsamps ? in[line * ld + n] : make_float2(0.f, 0.f);
    }
}

__global__ void ie_power_kernel(const float2 *__restrict__ spec, int nsample, int nfft,
                                float *__restrict__ psd) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nfft; j += gridDim.x * blockDim.x) {
        float acc = 0.f;
        for (int q = 0; q < nsample; ++q) {
            const float2 v = spec[(long long)q * nfft + j];
            acc = fmaf(v.x, v.x, fmaf(v.y, v.y, acc));
        }
        psd[j] = acc;
    }
}

}  // namespace

extern "C" int srg_interp_error(const float *lines, long long ld, int nlines, int nsamps,
                                int sample_lines, double *err_linear, double *err_oversampled,
                                void *stream) {
    if (!lines || nlines < 1 || nsamps < 2 || ld < nsamps || sample_lines < 1)
        return fail(SRG_E_ARG, "bad arguments (nlines %d nsamps %d ld %lld sample %d)", nlines,
                    nsamps, ld, sample_lines);
    const int nsample = std::min(sample_lines, nlines);
    int nfft = 1;
    while (nfft < nsamps) nfft <<= 1;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    float2 *buf = nullptr;
    float *psd = nullptr;
    cufftHandle plan = 0;
    bool have_plan = false;
    int rc = SRG_OK;
    std::vector<float> p(nfft);
    do {
        if (cudaMalloc(&buf, sizeof(float2) * (size_t)nsample * nfft) != cudaSuccess ||
            cudaMalloc(&psd, sizeof(float) * (size_t)nfft) != cudaSuccess) {
            cudaGetLastError();
            rc = fail(SRG_E_NOMEM, "spectrum scratch of %d x %d samples", nsample, nfft);
            break;
        }
        const long long total = (long long)nsample * nfft;
        const int blocks = (int)std::min<long long>((total + 255) / 256, 65535);
        ie_pad_kernel<<<blocks, 256, 0, st>>>(reinterpret_cast<const float2 *>(lines), ld, nlines,
                                             nsample, nsamps, nfft, buf);
        if (cufftPlan1d(&plan, nfft, CUFFT_C2C, nsample) != CUFFT_SUCCESS) {
            rc = fail(SRG_E_CUDA, "cufftPlan1d(%d, batch %d) failed", nfft, nsample);
            break;
        }
        have_plan = true;
        if (cufftSetStream(plan, st) != CUFFT_SUCCESS ||
            cufftExecC2C(plan, reinterpret_cast<cufftComplex *>(buf),
                         reinterpret_cast<cufftComplex *>(buf), CUFFT_FORWARD) != CUFFT_SUCCESS) {
            rc = fail(SRG_E_CUDA, "cufftExecC2C failed");
            break;
        }
        ie_power_kernel<<<(nfft + 255) / 256, 256, 0, st>>>(buf, nsample, nfft, psd);
        cudaError_t e = cudaMemcpyAsync(p.data(), psd, sizeof(float) * nfft, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = fail(SRG_E_CUDA, "spectrum failed: %s", cudaGetErrorString(e));
    } while (false);
    if (have_plan) cufftDestroy(plan);
    cudaFree(buf);
    cudaFree(psd);
    if (rc) return rc;

    float h[4];
    srg_oversample_taps(h);
    const double pi = ref_pi();
    constexpr int kU = 64;  // offsets u = (q + 0.5) / kU
    double tot = 0.0, el = 0.0, eo = 0.0;
    using cd = std::complex<double>;
    auto ex = [](double a) { return cd(std::cos(a), std::sin(a)); };
    for (int j = 0; j < nfft; ++j) {
        const double w = p[j];
        if (!(w > 0.0)) continue;
        const double nu = (j < nfft / 2 ? j : j - nfft) / (double)nfft;
        cd g(0.0, 0.0);
        for (int t = 0; t < 4; ++t) g += (double)h[t] * (ex(-2 * pi * nu * t) + ex(2 * pi * nu * (1 + t)));
        double sl = 0.0, so = 0.0;
        for (int q = 0; q < kU; ++q) {
            const double u = (q + 0.5) / kU;
            sl += std::norm((1 - u) + u * ex(2 * pi * nu) - ex(2 * pi * nu * u));
            so += std::norm((1 - u) + u * g - ex(pi * nu * u));
            so += std::norm((1 - u) * g + u * ex(2 * pi * nu) - ex(pi * nu * (1 + u)));
        }
        tot += w;
        el += w * sl / kU;
        eo += w * so / (2 * kU);
    }
    if (!(tot > 0.0)) {
        if (err_linear) *err_linear = 0.0;
        if (err_oversampled) *err_oversampled = 0.0;
        return SRG_OK;
    }
    if (err_linear) *err_linear = std::sqrt(el / tot) / std::sqrt(2.0);
    if (err_oversampled) *err_oversampled = std::sqrt(eo / tot) / std::sqrt(2.0);
    return SRG_OK;
}
