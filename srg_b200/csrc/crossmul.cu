// crossmul.cu -- interferograms of co-registered complex64 images on the GPU.
//
// Follows int/crossmul.f90:95-185 line for line in what it computes; the
// layout is the GPU's: every output line of every pair is independent, so the
// images are transformed whole (one batched FFT per image and direction,
// cuFFT; for lines of 2,049-4,096 samples one fused shared-memory kernel per
// line instead, upsample4096_kernel) and one fused kernel forms the cross
// products, the two-sample reclaim, the looks down and across, the
// square-rooted amplitudes and the zero-input mask.  Per image:
//   1. in * scale, zero-padded from na to nnn = the first 2^i >= na (i >= 1)
//      (crossmul.f90:69-73, 128-135);
//   2. forward FFT of nnn points (FFTW sign -1, unnormalised);
//   3. spectrum bins [0, nnn/2) to [0, nnn/2) and [nnn/2, nnn) to
//      [2nnn - nnn/2, 2nnn) of a zeroed 2nnn array (crossmul.f90:136-137);
//   4. inverse FFT of 2nnn points (sign +1), / nnn / 2 (crossmul.f90:139-141).
// Per pair and output sample (line L, column j), with u1, u2 the upsampled
// lines: igram = sum_k sum_i (u1 conj(u2))[2c] + (u1 conj(u2))[2c+1],
// c = j looksac + k, i over the looksdn input lines of L (crossmul.f90:155-172);
// amp likewise with (|u1|^2, |u2|^2), then (sqrt re, sqrt im) (:173); both
// zeroed where |sum of the raw input over the look window| <= 1e-6 in either
// image (crossmul.f90:112-125, 176-184).  Sums run in the reference's order
// (reclaim, then down, then across) in FP32 as the reference's complex*8.
#include <cuda_runtime.h>
#include <cufft.h>

#include <mutex>
#include <vector>

#include "../../include/srg_bp.h"
#include "host_internal.h"
#include "smem_fft.cuh"

using namespace srg;
using namespace srg::detail;

namespace {

#define CKC(call)                                                                      \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            return fail(SRG_E_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));   \
    } while (0)
#define CKF(call)                                                                      \
    do {                                                                               \
        cufftResult r_ = (call);                                                       \
        if (r_ != CUFFT_SUCCESS) return fail(SRG_E_CUDA, "%s failed: cufft %d", #call, (int)r_); \
    } while (0)

// in * scale, zero-padded to nnn, for nl lines
__global__ void pad_scale_kernel(const float2 *__restrict__ in, long long ld, int na, int nnn, int nl,
                                 float scale, float2 *__restrict__ out) {
    const long long total = (long long)nl * nnn;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int l = (int)(i / nnn), n = (int)(i - (long long)l * nnn);
        float2 v = make_float2(0.f, 0.f);
        if (n < na) {
            const float2 x = in[(long long)l * ld + n];
            v = make_float2(x.x * scale, x.y * scale);
        }
        out[i] = v;
    }
}

// nnn-point spectrum -> 2nnn array with the upper half of the bins at the top
__global__ void spread_kernel(const float2 *__restrict__ X, int nnn, int nl, float2 *__restrict__ up) {
    const int n2 = 2 * nnn, h = nnn / 2;
    const long long total = (long long)nl * n2;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int l = (int)(i / n2), m = (int)(i - (long long)l * n2);
        float2 v = make_float2(0.f, 0.f);
        if (m < h) v = X[(long long)l * nnn + m];
        else if (m >= n2 - h) v = X[(long long)l * nnn + (m - nnn)];
        up[i] = v;
    }
}

__device__ __forceinline__ float2 cmul_conj(float2 a, float2 b) {  // a * conj(b)
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// one thread per output sample (L, j)
__global__ void crossmul_looks_kernel(const float2 *__restrict__ up1, const float2 *__restrict__ up2,
                                      const float2 *__restrict__ in1, const float2 *__restrict__ in2,
                                      long long ld, int nnn, int nout_lines, int nout_cols,
                                      int looksac, int looksdn, int mask, float2 *__restrict__ igram,
                                      float2 *__restrict__ amp) {
    const long long total = (long long)nout_lines * nout_cols;
    const float inv = 1.f / (float)nnn;  // a power of two: same as the reference's division
    const int n2 = 2 * nnn;
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total;
         o += (long long)gridDim.x * blockDim.x) {
        const int L = (int)(o / nout_cols), j = (int)(o - (long long)L * nout_cols);
        float2 ig = make_float2(0.f, 0.f), am = make_float2(0.f, 0.f);
        float2 m1 = make_float2(0.f, 0.f), m2 = make_float2(0.f, 0.f);
        for (int k = 0; k < looksac; ++k) {
            const int c = j * looksac + k;
            float2 gd = make_float2(0.f, 0.f), ad = make_float2(0.f, 0.f);
            float2 s1 = make_float2(0.f, 0.f), s2 = make_float2(0.f, 0.f);
            for (int i = 0; i < looksdn; ++i) {
                const long long l = (long long)L * looksdn + i;
                const float2 *u1 = up1 + l * n2, *u2 = up2 + l * n2;
                float2 a0 = u1[2 * c], a1 = u1[2 * c + 1], b0 = u2[2 * c], b1 = u2[2 * c + 1];
                a0 = make_float2(a0.x * inv * 0.5f, a0.y * inv * 0.5f);
                a1 = make_float2(a1.x * inv * 0.5f, a1.y * inv * 0.5f);
                b0 = make_float2(b0.x * inv * 0.5f, b0.y * inv * 0.5f);
                b1 = make_float2(b1.x * inv * 0.5f, b1.y * inv * 0.5f);
                const float2 g0 = cmul_conj(a0, b0), g1 = cmul_conj(a1, b1);
                gd.x += g0.x + g1.x;
                gd.y += g0.y + g1.y;
                ad.x += (a0.x * a0.x + a0.y * a0.y) + (a1.x * a1.x + a1.y * a1.y);
                ad.y += (b0.x * b0.x + b0.y * b0.y) + (b1.x * b1.x + b1.y * b1.y);
                if (mask) {
                    const float2 x1 = in1[l * ld + c], x2 = in2[l * ld + c];
                    s1.x += x1.x;
                    s1.y += x1.y;
                    s2.x += x2.x;
                    s2.y += x2.y;
                }
            }
            ig.x += gd.x;
            ig.y += gd.y;
            am.x += ad.x;
            am.y += ad.y;
            m1.x += s1.x;
            m1.y += s1.y;
            m2.x += s2.x;
            m2.y += s2.y;
        }
        am = make_float2(sqrtf(am.x), sqrtf(am.y));
        if (mask && (hypotf(m1.x, m1.y) <= 1.e-6f || hypotf(m2.x, m2.y) <= 1.e-6f)) {
            ig = make_float2(0.f, 0.f);
            am = make_float2(0.f, 0.f);
        }
        igram[o] = ig;
        amp[o] = am;
    }
}

// Steps 1-4 for one image when nnn = 4096 (lines of 2,049-4,096 samples),
// fused per line in shared memory: in * scale padded to 4,096, the forward
// transform, the spread into 8,192 bins and the inverse transform (the
// forward transform of the conjugate, conjugated; unnormalised), written
// once as the line's 8,192 upsampled samples: the image crosses HBM once
// each way where the cuFFT path takes five passes over padded rows.
// Persistent: one CTA of smem_fft::kThreads per SM takes lines in turn,
// after loading the twiddle tables once.
constexpr int kXmSmem = (smem_fft::kBuf + smem_fft::kTw) * (int)sizeof(float2);

// One line of one image, steps 1-4 with nnn = 4096.  With the spectrum X
// spread as step 3 does, the unnormalised 8,192-point inverse u has
// u[2n] = 4096 x_s[n] (x_s = in * scale padded to 4096: the forward and
// inverse 4,096-point transforms cancel) and u[2n + 1] = the 4,096-point
// inverse of X[k] s_k exp(i pi k / 4096), s_k = 1 for k < 2048 and -1 for the
// bins moved to the top.  So the odd samples come from two 4,096-point
// transforms (the inverse as the forward transform of the conjugate) and
// the even ones straight from the input (even_sample): u[2n + 1] is left in
// buf[pad(n)], n < 4096.  All kThreads threads call it; tw holds the
// twiddle tables.
__device__ __forceinline__ float2 even_sample(const float2 *__restrict__ x, int n, int na,
                                              float scale) {
    if (n >= na) return make_float2(0.f, 0.f);
    const float2 a = __ldg(x + n);
    return make_float2(a.x * scale * 4096.f, a.y * scale * 4096.f);
}

__device__ __forceinline__ void upsample_line(const float2 *__restrict__ x, int na, float scale,
                                              float2 *buf, const float2 *tw) {
    using namespace smem_fft;
    constexpr int N = 4096, T = kThreads;
    const int t = threadIdx.x;
    // forward 4,096-point transform, pass 1 (Ns = 1) from the line
    if (t < N / 16) {
        float2 v[16];
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            const int i = t + r * (N / 16);
            float2 a = make_float2(0.f, 0.f);
            if (i < na) {
                a = __ldg(x + i);
                a = make_float2(a.x * scale, a.y * scale);
            }
            v[r] = a;
        }
        dft<16>(v);
#pragma unroll
        for (int r = 0; r < 16; ++r) buf[pad(t * 16 + r)] = v[brev<16>(r)];
    }
    __syncthreads();
    pass16<N>(buf, 16, tw + kTw16);
    pass16<N>(buf, 256, tw + kTw256);
    // conj(X[k] s_k exp(i pi k / 4096)) = s_k conj(X[k]) exp(-2 pi i k / 8192),
    // each item its own entry
#pragma unroll
    for (int q = 0; q < N / T; ++q) {
        const int k = t + q * T;
        const float2 z = cmul(cconj(buf[pad(k)]), tw[kTw2 + k]);
        buf[pad(k)] = k < N / 2 ? z : make_float2(-z.x, -z.y);
    }
    __syncthreads();
    pass16<N>(buf, 1, nullptr);
    pass16<N>(buf, 16, tw + kTw16);
    pass16<N>(buf, 256, tw + kTw256);
#pragma unroll
    for (int q = 0; q < N / T; ++q) buf[pad(t + q * T)] = cconj(buf[pad(t + q * T)]);
    __syncthreads();
}

__global__ void __launch_bounds__(smem_fft::kThreads, 1)
upsample4096_kernel(const float2 *__restrict__ in, long long ld, int na, int nl, float scale,
                    const float2 *__restrict__ twg, float2 *__restrict__ up) {
    using namespace smem_fft;
    extern __shared__ float2 xm_sm[];
    float2 *buf = xm_sm, *tw = xm_sm + kBuf;
    const int t = threadIdx.x;
    for (int i = t; i < kTw; i += kThreads) tw[i] = __ldg(twg + i);
    __syncthreads();
    for (int l = blockIdx.x; l < nl; l += gridDim.x) {
        const float2 *x = in + (long long)l * ld;
        upsample_line(x, na, scale, buf, tw);
        float4 *u = reinterpret_cast<float4 *>(up + (long long)l * 8192);  // (u[2n], u[2n + 1])
        for (int j = t; j < 4096; j += kThreads) {
            const float2 e = even_sample(x, j, na, scale), o = buf[pad(j)];
            u[j] = make_float4(e.x, e.y, o.x, o.y);
        }
        __syncthreads();  // the line's reads are done before the next one's writes
    }
}

// One radix-16 pass of a 4,096-point transform per half-CTA, each half on its
// own buffer (threads t < 256: buf of the first half, t >= 256: of the
// second); otherwise as smem_fft::pass16.  Every thread calls it.
__device__ __forceinline__ void pass16_halves(float2 *buf, int Ns, const float2 *tw) {
    using namespace smem_fft;
    constexpr int J = 256;
    const int j = threadIdx.x & (J - 1), k = j & (Ns - 1);
    float2 v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = buf[pad(j + r * J)];
    __syncthreads();
    if (Ns > 1) {
#pragma unroll
        for (int r = 1; r < 16; ++r) v[r] = cmul(v[r], tw[(r - 1) * Ns + k]);
    }
    dft<16>(v);
    const int base = (j - k) * 16 + k;
#pragma unroll
    for (int r = 0; r < 16; ++r) buf[pad(base + r * Ns)] = v[brev<16>(r)];
    __syncthreads();
}

// upsample_line for two lines at once, one per half-CTA: x0 into b0 (threads
// t < 256), x1 into b1 (t >= 256; x1 null: that half transforms zeros).
__device__ __forceinline__ void upsample_two(const float2 *__restrict__ x0,
                                             const float2 *__restrict__ x1, int na, float scale,
                                             float2 *b0, float2 *b1, const float2 *tw) {
    using namespace smem_fft;
    constexpr int N = 4096, J = 256;
    const int t = threadIdx.x, jt = t & (J - 1);
    const float2 *x = t < J ? x0 : x1;
    float2 *buf = t < J ? b0 : b1;
    {
        float2 v[16];
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            const int i = jt + r * J;
            float2 a = make_float2(0.f, 0.f);
            if (x && i < na) {
                a = __ldg(x + i);
                a = make_float2(a.x * scale, a.y * scale);
            }
            v[r] = a;
        }
        dft<16>(v);
#pragma unroll
        for (int r = 0; r < 16; ++r) buf[pad(jt * 16 + r)] = v[brev<16>(r)];
    }
    __syncthreads();
    pass16_halves(buf, 16, tw + kTw16);
    pass16_halves(buf, 256, tw + kTw256);
#pragma unroll
    for (int q = 0; q < N / J; ++q) {
        const int k = jt + q * J;
        const float2 z = cmul(cconj(buf[pad(k)]), tw[kTw2 + k]);
        buf[pad(k)] = k < N / 2 ? z : make_float2(-z.x, -z.y);
    }
    __syncthreads();
    pass16_halves(buf, 1, nullptr);
    pass16_halves(buf, 16, tw + kTw16);
    pass16_halves(buf, 256, tw + kTw256);
#pragma unroll
    for (int q = 0; q < N / J; ++q) buf[pad(jt + q * J)] = cconj(buf[pad(jt + q * J)]);
    __syncthreads();
}

// One pair's interferogram and amplitude samples of one grid line (looks of
// one line down), from the two images' odd upsampled samples in shared
// memory and their even ones from the input: the sums of
// crossmul_looks_kernel with looksdn = 1, in its order.
__device__ __forceinline__ void form_pair(const float2 *up1, const float2 *up2,
                                          const float2 *__restrict__ in1,
                                          const float2 *__restrict__ in2, int na, float scale,
                                          int nout_cols, int looksac, int mask, float2 *ig_out,
                                          float2 *am_out) {
    const float inv = 1.f / 4096.f;  // a power of two: same as the reference's division
    for (int j = threadIdx.x; j < nout_cols; j += smem_fft::kThreads) {
        float2 ig = make_float2(0.f, 0.f), am = make_float2(0.f, 0.f);
        float2 m1 = make_float2(0.f, 0.f), m2 = make_float2(0.f, 0.f);
        for (int q = 0; q < looksac; ++q) {
            const int c = j * looksac + q;
            float2 gd = make_float2(0.f, 0.f), ad = make_float2(0.f, 0.f);
            float2 s1 = make_float2(0.f, 0.f), s2 = make_float2(0.f, 0.f);
            float2 a0 = even_sample(in1, c, na, scale), a1 = up1[smem_fft::pad(c)];
            float2 b0 = even_sample(in2, c, na, scale), b1 = up2[smem_fft::pad(c)];
            a0 = make_float2(a0.x * inv * 0.5f, a0.y * inv * 0.5f);
            a1 = make_float2(a1.x * inv * 0.5f, a1.y * inv * 0.5f);
            b0 = make_float2(b0.x * inv * 0.5f, b0.y * inv * 0.5f);
            b1 = make_float2(b1.x * inv * 0.5f, b1.y * inv * 0.5f);
            const float2 g0 = cmul_conj(a0, b0), g1 = cmul_conj(a1, b1);
            gd.x += g0.x + g1.x;
            gd.y += g0.y + g1.y;
            ad.x += (a0.x * a0.x + a0.y * a0.y) + (a1.x * a1.x + a1.y * a1.y);
            ad.y += (b0.x * b0.x + b0.y * b0.y) + (b1.x * b1.x + b1.y * b1.y);
            if (mask) {
                const float2 x1 = __ldg(in1 + c), x2 = __ldg(in2 + c);
                s1.x += x1.x;
                s1.y += x1.y;
                s2.x += x2.x;
                s2.y += x2.y;
            }
            ig.x += gd.x;
            ig.y += gd.y;
            am.x += ad.x;
            am.y += ad.y;
            m1.x += s1.x;
            m1.y += s1.y;
            m2.x += s2.x;
            m2.y += s2.y;
        }
        am = make_float2(sqrtf(am.x), sqrtf(am.y));
        if (mask && (hypotf(m1.x, m1.y) <= 1.e-6f || hypotf(m2.x, m2.y) <= 1.e-6f)) {
            ig = make_float2(0.f, 0.f);
            am = make_float2(0.f, 0.f);
        }
        ig_out[j] = ig;
        am_out[j] = am;
    }
}

// The whole stack with looks of one line down and nnn = 4096, fused: per grid
// line, images k and k + 1 are upsampled at once (one per half-CTA) into two
// of three shared buffers while image k - 1's line is still in the third,
// and the pairs (k - 1, k) and (k, k + 1) of that line are formed from them:
// the images are read once and no upsampled image goes through HBM.
// Persistent over lines.
constexpr int kXmLine = 4096 + 4096 / 16;  // padded 4,096-point buffer (float2)
constexpr int kXmStackSmem = (3 * kXmLine + smem_fft::kTw) * (int)sizeof(float2);
// Images of one launch (its pointers travel as a kernel parameter, 1.5 KB):
// longer stacks go in launches of up to kXmChunk images overlapping by one.
constexpr int kXmChunk = 64;
struct StackPtrs {
    const float2 *img[kXmChunk];
    float2 *ig[kXmChunk - 1], *am[kXmChunk - 1];
};

__global__ void __launch_bounds__(smem_fft::kThreads, 1)
crossmul_stack4096_kernel(const __grid_constant__ StackPtrs p, int n, long long ld, int na,
                          int nlines, int nout_cols, int looksac, float scale, int mask,
                          const float2 *__restrict__ twg) {
    const float2 *const *imgs = p.img;
    float2 *const *igrams = p.ig;
    float2 *const *amps = p.am;
    using namespace smem_fft;
    extern __shared__ float2 xm_sm[];
    float2 *tw = xm_sm + 3 * kXmLine;
    const int t = threadIdx.x;
    for (int i = t; i < kTw; i += kThreads) tw[i] = __ldg(twg + i);
    __syncthreads();
    for (int l = blockIdx.x; l < nlines; l += gridDim.x) {
        const long long row = (long long)l * ld, orow = (long long)l * nout_cols;
        int prev = -1;  // buffer holding image k - 1's line
        for (int k = 0; k < n; k += 2) {
            const int a = prev < 0 ? 0 : (prev + 1) % 3, b = prev < 0 ? 1 : (prev + 2) % 3;
            float2 *ua = xm_sm + a * kXmLine, *ub = xm_sm + b * kXmLine;
            const bool two = k + 1 < n;
            upsample_two(imgs[k] + row, two ? imgs[k + 1] + row : nullptr, na, scale, ua, ub, tw);
            if (k > 0)
                form_pair(xm_sm + prev * kXmLine, ua, imgs[k - 1] + row, imgs[k] + row, na, scale,
                          nout_cols, looksac, mask, igrams[k - 1] + orow, amps[k - 1] + orow);
            if (two)
                form_pair(ua, ub, imgs[k] + row, imgs[k + 1] + row, na, scale, nout_cols, looksac,
                          mask, igrams[k] + orow, amps[k] + orow);
            __syncthreads();  // the pairs' reads are done before the buffers are written again
            prev = two ? b : a;
        }
    }
}

struct Plan {
    int n = 0, batch = 0;
    cufftHandle h = 0;
    bool ok = false;
};

struct XmCtx {
    std::mutex mu;
    Plan fwd, inv;
    DevBuf pad, upA, upB;
    DevBuf tw;          // twiddle tables of the fused kernels (smem_fft)
    bool fused_ready = false;
    int sms = 0;
};
XmCtx g_xm[64];

int plan_for(Plan &p, int n, int batch) {
    if (p.ok && p.n == n && p.batch == batch) return SRG_OK;
    if (p.ok) cufftDestroy(p.h);
    p.ok = false;
    CKF(cufftPlan1d(&p.h, n, CUFFT_C2C, batch));
    p.n = n;
    p.batch = batch;
    p.ok = true;
    return SRG_OK;
}

int grid_for(long long n) {
    long long g = (n + 255) / 256;
    return (int)std::min<long long>(g, 148LL * 32);
}

// upsampled lines of one image into `up` (nl x 2nnn)
int upsample(XmCtx &x, const float2 *in, long long ld, int na, int nnn, int nl, float scale,
             float2 *up, cudaStream_t st) {
    if (nnn == 4096) {
        upsample4096_kernel<<<std::min(nl, x.sms), smem_fft::kThreads, kXmSmem, st>>>(
            in, ld, na, nl, scale, static_cast<const float2 *>(x.tw.p), up);
        CKC(cudaGetLastError());
        return SRG_OK;
    }
    float2 *pad = static_cast<float2 *>(x.pad.p);
    pad_scale_kernel<<<grid_for((long long)nl * nnn), 256, 0, st>>>(in, ld, na, nnn, nl, scale, pad);
    CKC(cudaGetLastError());
    CKF(cufftSetStream(x.fwd.h, st));
    CKF(cufftExecC2C(x.fwd.h, reinterpret_cast<cufftComplex *>(pad),
                     reinterpret_cast<cufftComplex *>(pad), CUFFT_FORWARD));
    spread_kernel<<<grid_for((long long)nl * 2 * nnn), 256, 0, st>>>(pad, nnn, nl, up);
    CKC(cudaGetLastError());
    CKF(cufftSetStream(x.inv.h, st));
    CKF(cufftExecC2C(x.inv.h, reinterpret_cast<cufftComplex *>(up),
                     reinterpret_cast<cufftComplex *>(up), CUFFT_INVERSE));
    return SRG_OK;
}

int check_args(long long ld, int na, int nlines, int looksac, int looksdn) {
    if (na < 1 || ld < na || nlines < 1 || looksac < 1 || looksdn < 1)
        return fail(SRG_E_ARG, "bad crossmul sizes: na=%d ld=%lld nlines=%d looks=%d x %d", na, ld,
                    nlines, looksac, looksdn);
    if (na / looksac < 1 || nlines / looksdn < 1)
        return fail(SRG_E_ARG, "looks %d x %d exceed the image %d x %d", looksac, looksdn, na, nlines);
    if (na > (1 << 24)) return fail(SRG_E_ARG, "line of %d samples exceeds 2^24", na);
    return SRG_OK;
}

int fft_length(int na) {  // crossmul.f90:69-73: first 2^i >= na, i = 1..24
    int n = 2;
    while (n < na) n *= 2;
    return n;
}

int run_stack(const float *const *slcs, int n, long long ld, int na, int nlines, int looksac,
              int looksdn, float scale, int mask, float *const *igrams, float *const *amps,
              void *stream) {
    int rc = check_args(ld, na, nlines, looksac, looksdn);
    if (rc) return rc;
    if (n < 2 || !slcs || !igrams || !amps) return fail(SRG_E_ARG, "need >= 2 images and outputs");
    for (int k = 0; k < n; ++k)
        if (!slcs[k]) return fail(SRG_E_ARG, "null image %d", k);
    for (int k = 0; k + 1 < n; ++k)
        if (!igrams[k] || !amps[k]) return fail(SRG_E_ARG, "null output of pair %d", k);
    int dev = 0;
    CKC(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(SRG_E_ARG, "device %d out of range", dev);
    XmCtx &x = g_xm[dev];
    std::lock_guard<std::mutex> g(x.mu);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nnn = fft_length(na);
    const int nout_lines = nlines / looksdn, nout_cols = na / looksac;
    const int nl = nout_lines * looksdn;
    if (nnn == 4096) {  // the fused kernels (upsample4096_kernel, crossmul_stack4096_kernel)
        if (!x.fused_ready) {
            if ((rc = x.tw.ensure(sizeof(float2) * smem_fft::kTw))) return rc;
            const std::vector<float2> tw = smem_fft::twiddle_tables();
            CKC(cudaFuncSetAttribute(upsample4096_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     kXmSmem));
            CKC(cudaFuncSetAttribute(crossmul_stack4096_kernel,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, kXmStackSmem));
            CKC(cudaDeviceGetAttribute(&x.sms, cudaDevAttrMultiProcessorCount, dev));
            CKC(cudaMemcpyAsync(x.tw.p, tw.data(), sizeof(float2) * smem_fft::kTw,
                                cudaMemcpyHostToDevice, st));
            CKC(cudaStreamSynchronize(st));  // `tw` is pageable host memory that goes out of scope
            x.fused_ready = true;
        }
        if (looksdn == 1) {  // the whole stack, in launches of up to kXmChunk images
            for (int k0 = 0; k0 + 1 < n; k0 += kXmChunk - 1) {
                const int m = std::min(kXmChunk, n - k0);
                StackPtrs p{};
                for (int k = 0; k < m; ++k) p.img[k] = reinterpret_cast<const float2 *>(slcs[k0 + k]);
                for (int k = 0; k + 1 < m; ++k) {
                    p.ig[k] = reinterpret_cast<float2 *>(igrams[k0 + k]);
                    p.am[k] = reinterpret_cast<float2 *>(amps[k0 + k]);
                }
                crossmul_stack4096_kernel<<<std::min(nout_lines, x.sms), smem_fft::kThreads,
                                            kXmStackSmem, st>>>(
                    p, m, ld, na, nout_lines, nout_cols, looksac, scale, mask,
                    static_cast<const float2 *>(x.tw.p));
                CKC(cudaGetLastError());
            }
            return SRG_OK;
        }
    } else if ((rc = plan_for(x.fwd, nnn, nl)) || (rc = plan_for(x.inv, 2 * nnn, nl)) ||
               (rc = x.pad.ensure((size_t)nl * nnn * sizeof(float2)))) {
        return rc;
    }
    const size_t up_bytes = (size_t)nl * 2 * nnn * sizeof(float2);
    if ((rc = x.upA.ensure(up_bytes)) || (rc = x.upB.ensure(up_bytes))) return rc;
    float2 *cur = static_cast<float2 *>(x.upA.p), *nxt = static_cast<float2 *>(x.upB.p);
    if ((rc = upsample(x, reinterpret_cast<const float2 *>(slcs[0]), ld, na, nnn, nl, scale, cur, st)))
        return rc;
    for (int k = 0; k + 1 < n; ++k) {
        const float2 *a = reinterpret_cast<const float2 *>(slcs[k]);
        const float2 *b = reinterpret_cast<const float2 *>(slcs[k + 1]);
        if (b == a) {
            CKC(cudaMemcpyAsync(nxt, cur, up_bytes, cudaMemcpyDeviceToDevice, st));
        } else if ((rc = upsample(x, b, ld, na, nnn, nl, scale, nxt, st))) {
            return rc;
        }
        crossmul_looks_kernel<<<grid_for((long long)nout_lines * nout_cols), 256, 0, st>>>(
            cur, nxt, a, b, ld, nnn, nout_lines, nout_cols, looksac, looksdn, mask,
            reinterpret_cast<float2 *>(igrams[k]), reinterpret_cast<float2 *>(amps[k]));
        CKC(cudaGetLastError());
        std::swap(cur, nxt);
    }
    return SRG_OK;
}

}  // namespace

extern "C" {

int srg_crossmul_device(const float *slc1, const float *slc2, long long ld, int na, int nlines,
                        int looksac, int looksdn, float scale, int mask, float *igram, float *amp,
                        void *stream) {
    const float *s[2] = {slc1, slc2};
    float *ig[1] = {igram};
    float *am[1] = {amp};
    return run_stack(s, 2, ld, na, nlines, looksac, looksdn, scale, mask, ig, am, stream);
}

int srg_crossmul_stack_device(const float *const *slcs, int n, long long ld, int na, int nlines,
                              int looksac, int looksdn, float scale, int mask, float *const *igrams,
                              float *const *amps, void *stream) {
    return run_stack(slcs, n, ld, na, nlines, looksac, looksdn, scale, mask, igrams, amps, stream);
}

}  // extern "C"
