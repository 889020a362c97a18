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
// Pulses of up to 4,096 samples (Sentinel-1 IW: ~3,370) take the fused
// overlap-save kernel instead (rc_os_kernel below), same samples.
#include <cuda_runtime.h>
#include <cufft.h>

#include <climits>
#include <cmath>
#include <complex>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/srg_bp.h"
#include "host_internal.h"
#include "smem_fft.cuh"

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

// ---------------------------------------------------------------------------
// Fused matched filter by overlap-save.  The samples the reference keeps,
// y[n] = 32768 sum_{j < npts} conj(r[j]) x[n + j] for n < nvalid, are a
// linear correlation (the 32,768-point circular one never wraps into them),
// so 8,192-point transforms give them exactly up to rounding: a segment of
// 8,192 samples from s0 (zeros past the line) yields y[s0 .. s0 + L),
// L = 8192 - npts + 1.  A CTA (one per SM, persistent) takes (line,
// segment) items in turn: it loads the segment's samples once, transforms
// them in shared memory, multiplies by the filter
// H = (32768 / 8192) conj(DFT_8192(r)), transforms back (a forward transform
// of the conjugate, conjugated) and writes its L outputs once: the lines
// cross HBM once each way, where the cuFFT path below takes five passes over
// 32,768-point rows.  Transforms: Stockham autosort passes of radix 16, 16,
// 16 and 2 (16 values per thread per pass), each DFT in registers, the
// padded shared layout i + i / 16 keeping the 16-strided accesses off common
// banks, the twiddles of each pass from its own table in shared memory
// (exactly rounded, laid out so that a warp reads consecutive entries),
// loaded once per CTA.  Pulses of more than 4,096 samples take the cuFFT
// path.
constexpr int kOsM = 8192;                       // segment transform
constexpr int kOsMaxPts = kOsM / 2;              // longest pulse the segments take
constexpr int kOsBuf = smem_fft::kBuf;          // padded segment (float2)
constexpr int kOsThreads = smem_fft::kThreads;   // one radix-16 work item per thread
constexpr int kOsTw16 = smem_fft::kTw16, kOsTw256 = smem_fft::kTw256, kOsTw2 = smem_fft::kTw2;
constexpr int kOsTw = smem_fft::kTw;
constexpr int kOsSmem = (kOsBuf + kOsTw) * (int)sizeof(float2);
using smem_fft::brev;
using smem_fft::cadd;
using smem_fft::cconj;
using smem_fft::cmul;
using smem_fft::csub;
using smem_fft::dft;
__device__ __forceinline__ int os_pad(int i) { return smem_fft::pad(i); }
__device__ __forceinline__ void os_pass(float2 *buf, int Ns, const float2 *tw) {
    smem_fft::pass16<kOsM>(buf, Ns, tw);
}

// Persistent: each CTA takes segments (line, s0) in turn, after loading the
// twiddle tables once.
__global__ void __launch_bounds__(kOsThreads, 1)
rc_os_kernel(const float2 *__restrict__ in, long long ld_in, int nsamps, int nvalid, int L,
             int nseg, int nitems, const float2 *__restrict__ H, const float2 *__restrict__ twg,
             float2 *__restrict__ out, long long ld_out) {
    extern __shared__ float2 os_sm[];
    float2 *buf = os_sm, *tw = os_sm + kOsBuf;
    const int t = threadIdx.x;
    for (int i = t; i < kOsTw; i += kOsThreads) tw[i] = __ldg(twg + i);
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int line = item / nseg, s0 = (item - line * nseg) * L;
        const float2 *x = in + (long long)line * ld_in;
        // forward transform, pass 1 (Ns = 1) straight from the line
        {
            float2 v[16];
#pragma unroll
            for (int r = 0; r < 16; ++r) {
                const int i = s0 + t + r * kOsThreads;
                v[r] = i < nsamps ? __ldg(x + i) : make_float2(0.f, 0.f);
            }
            dft<16>(v);
#pragma unroll
            for (int r = 0; r < 16; ++r) buf[os_pad(t * 16 + r)] = v[brev<16>(r)];
        }
        __syncthreads();  // (the first time also the tables)
        os_pass(buf, 16, tw + kOsTw16);
        os_pass(buf, 256, tw + kOsTw256);
        // last pass (radix 2, Ns = 4096): each item touches only its own pair,
        // so the filter and the conjugation of the inverse go in place
#pragma unroll
        for (int it = 0; it < kOsM / 2 / kOsThreads; ++it) {
            const int j = t + it * kOsThreads;
            const float2 a = buf[os_pad(j)], b = cmul(buf[os_pad(j + kOsM / 2)], tw[kOsTw2 + j]);
            buf[os_pad(j)] = cconj(cmul(cadd(a, b), __ldg(H + j)));
            buf[os_pad(j + kOsM / 2)] = cconj(cmul(csub(a, b), __ldg(H + j + kOsM / 2)));
        }
        __syncthreads();
        // inverse: forward transform of the conjugate
        os_pass(buf, 1, nullptr);
        os_pass(buf, 16, tw + kOsTw16);
        os_pass(buf, 256, tw + kOsTw256);
        float2 *y = out + (long long)line * ld_out + s0;
        const int nout = min(L, nvalid - s0);
#pragma unroll
        for (int it = 0; it < kOsM / 2 / kOsThreads; ++it) {
            const int j = t + it * kOsThreads;
            const float2 a = buf[os_pad(j)], b = cmul(buf[os_pad(j + kOsM / 2)], tw[kOsTw2 + j]);
            if (j < nout) y[j] = cconj(cadd(a, b));
            if (j + kOsM / 2 < nout) y[j + kOsM / 2] = cconj(csub(a, b));
        }
        __syncthreads();  // the segment's reads are done before the next one's writes
    }
}

// Forward DFT (sign -1, unnormalised) of a power-of-two length, in FP64 on
// the host: iterative radix-2 decimation in time.
void host_fft(std::vector<std::complex<double>> &a) {
    const int n = (int)a.size();
    for (int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    const double pi = 4.0 * std::atan2(1.0, 1.0);
    for (int len = 2; len <= n; len <<= 1) {
        for (int k = 0; k < len / 2; ++k) {
            const std::complex<double> w = std::polar(1.0, -2.0 * pi * k / len);
            for (int i = 0; i < n; i += len) {
                const std::complex<double> u = a[i + k], v = a[i + k + len / 2] * w;
                a[i + k] = u + v;
                a[i + k + len / 2] = u - v;
            }
        }
    }
}

struct RcCtx {
    std::mutex mu;
    cufftHandle plan_blk = 0, plan_one = 0;
    bool have_plans = false;
    DevBuf buf, ref;
    float key[4] = {NAN, NAN, NAN, NAN};  // replica parameters of `ref`
    // overlap-save path: filter spectrum, twiddle tables, their parameters
    DevBuf os_h, os_tw;
    bool os_ready = false;
    int sms = 0;
    float os_key[4] = {NAN, NAN, NAN, NAN};
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
    if (npts <= kOsMaxPts) {
        // fused overlap-save kernel (see rc_os_kernel)
        if ((rc = x.os_h.ensure(sizeof(float2) * kOsM)) || (rc = x.os_tw.ensure(sizeof(float2) * kOsTw)))
            return rc;
        const double pi = 4.0 * std::atan2(1.0, 1.0);
        if (!x.os_ready) {
            const std::vector<float2> tw = smem_fft::twiddle_tables();
            CKR(cudaFuncSetAttribute(rc_os_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kOsSmem));
            CKR(cudaDeviceGetAttribute(&x.sms, cudaDevAttrMultiProcessorCount, dev));
            CKR(cudaMemcpyAsync(x.os_tw.p, tw.data(), sizeof(float2) * kOsTw, cudaMemcpyHostToDevice, st));
            CKR(cudaStreamSynchronize(st));  // `tw` is pageable host memory that goes out of scope
            x.os_ready = true;
        }
        const float key[4] = {samplefreq, startfreq, ramprate, pulselength};
        if (std::memcmp(key, x.os_key, sizeof key) != 0) {
            // H = (32768 / 8192) conj(DFT_8192(replica)), in FP64 from the
            // replica's complex64 samples
            std::vector<std::complex<double>> a(kOsM);
            for (int j = 0; j < npts; ++j) a[j] = std::complex<double>(rep[2 * j], rep[2 * j + 1]);
            host_fft(a);
            std::vector<float2> h(kOsM);
            const double scale = (double)kRangeFFT / kOsM;
            for (int k = 0; k < kOsM; ++k)
                h[k] = make_float2((float)(scale * a[k].real()), (float)(-scale * a[k].imag()));
            CKR(cudaMemcpyAsync(x.os_h.p, h.data(), sizeof(float2) * kOsM, cudaMemcpyHostToDevice, st));
            CKR(cudaStreamSynchronize(st));  // `h` is pageable host memory that goes out of scope
            std::memcpy(x.os_key, key, sizeof key);
        }
        const int L = kOsM - npts + 1;
        const int nseg = (nvalid + L - 1) / L;
        if ((long long)nlines * nseg > INT_MAX) return fail(SRG_E_ARG, "too many lines: %d", nlines);
        const int nitems = nlines * nseg;
        rc_os_kernel<<<std::min(nitems, x.sms), kOsThreads, kOsSmem, st>>>(
            reinterpret_cast<const float2 *>(lines), ld_in, nsamps, nvalid, L, nseg, nitems,
            static_cast<const float2 *>(x.os_h.p), static_cast<const float2 *>(x.os_tw.p),
            reinterpret_cast<float2 *>(out), ld_out);
        CKR(cudaGetLastError());
        if (nvalid_out) *nvalid_out = nvalid;
        return SRG_OK;
    }
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
