// smem_fft.cuh -- complex FP32 FFTs of 4,096 and 8,192 points held in one
// CTA's shared memory, for the fused kernels of range compression
// (rangecomp.cu) and interferogram formation (crossmul.cu).
//
// Stockham autosort passes of radix 16 (and a final radix 2 for 8,192
// points), one work item of 16 values per thread and pass, each DFT in
// registers; the shared layout pads one element every 16 (index i + i / 16)
// so the 16-strided accesses of a pass fall on distinct banks.  Each pass
// takes its twiddles exp(-2 pi i r k / (16 Ns)) from its own exactly rounded
// table, laid out [(r - 1) Ns + k] so that a warp reads consecutive entries:
// the tables depend only on 16 Ns, so one set (Ns = 16 and 256, and the
// radix-2 pass's exp(-2 pi i k / 8192)) serves both sizes.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

namespace srg {
namespace smem_fft {

constexpr int kMaxN = 8192;
constexpr int kBuf = kMaxN + (kMaxN >> 4);  // padded 8,192-point buffer (float2)
constexpr int kThreads = kMaxN / 16;        // one radix-16 work item per thread at 8,192
// twiddle tables: Ns = 16 at [kTw16 + (r - 1) 16 + k], Ns = 256 at
// [kTw256 + (r - 1) 256 + k], the radix-2 pass at [kTw2 + k], k < 4096
constexpr int kTw16 = 0, kTw256 = 15 * 16, kTw2 = kTw256 + 15 * 256;
constexpr int kTw = kTw2 + kMaxN / 2;

// The twiddle tables above (exp(-2 pi i x) rounded from FP64), for upload.
inline std::vector<float2> twiddle_tables() {
    const double pi = 4.0 * std::atan2(1.0, 1.0);
    std::vector<float2> tw(kTw);
    auto w = [&](double num, double den) {
        return make_float2((float)std::cos(2.0 * pi * num / den), (float)-std::sin(2.0 * pi * num / den));
    };
    for (int Ns : {16, 256})
        for (int r = 1; r < 16; ++r)
            for (int k = 0; k < Ns; ++k)
                tw[(Ns == 16 ? kTw16 : kTw256) + (r - 1) * Ns + k] = w((double)r * k, 16.0 * Ns);
    for (int k = 0; k < kMaxN / 2; ++k) tw[kTw2 + k] = w(k, kMaxN);
    return tw;
}

namespace {
// exp(-2 pi i q / 16), q = 0..7
__constant__ float2 kW16[8] = {{1.000000000f, 0.000000000f},   {0.923879533f, -0.382683432f},
                               {0.707106781f, -0.707106781f},  {0.382683432f, -0.923879533f},
                               {0.000000000f, -1.000000000f},  {-0.382683432f, -0.923879533f},
                               {-0.707106781f, -0.707106781f}, {-0.923879533f, -0.382683432f}};
}  // namespace

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ int pad(int i) { return i + (i >> 4); }
template <int R>
__host__ __device__ __forceinline__ constexpr int brev(int i) {
    int o = 0;
    for (int b = 1, t = R >> 1; b < R; b <<= 1, t >>= 1)
        if (i & b) o |= t;
    return o;
}

// R-point DFT in registers (R <= 16), in place: input X in natural order,
// output DFT(X)[r] in v[brev<R>(r)] (radix-2 decimation in time on the
// bit-reversed view a[p] = v[brev<R>(p)], so no permutation moves data; the
// butterflies of half-size h take exp(-2 pi i q / (2h)) = kW16[8 q / h]).
template <int R>
__device__ __forceinline__ void dft(float2 (&v)[R]) {
#pragma unroll
    for (int h = 1; h < R; h <<= 1) {
#pragma unroll
        for (int i = 0; i < R; i += 2 * h) {
#pragma unroll
            for (int q = 0; q < h; ++q) {
                float2 &lo = v[brev<R>(i + q)], &hi = v[brev<R>(i + q + h)];
                const float2 b = q == 0 ? hi : cmul(hi, kW16[q * (8 / h)]);
                hi = csub(lo, b);
                lo = cadd(lo, b);
            }
        }
    }
}

// One radix-16 Stockham pass of an N-point transform (N = 4096 or 8192) in
// shared memory; threads j < N / 16 each take one work item: item j reads
// v[r] = x[j + r N / 16], scales v[r] by exp(-2 pi i r k / (16 Ns)) =
// tw[(r - 1) Ns + k] (tw: that pass's table), k = j mod Ns, takes the
// 16-point DFT and writes y[(j - k) 16 + k + r Ns].  Every thread of the
// CTA must call it (it holds two barriers).
template <int N>
__device__ __forceinline__ void pass16(float2 *buf, int Ns, const float2 *tw) {
    constexpr int J = N / 16;
    static_assert(N == 4096 || N == 8192, "transform size");
    constexpr bool every = J >= kThreads;  // every thread of a kThreads CTA has an item
    const int j = threadIdx.x, k = j & (Ns - 1);
    const bool item = every || j < J;
    float2 v[16];
    // (threads without an item load too, from a valid index, and discard: the
    // register array is then set on every path and stays in registers)
    const int jl = every ? j : (j & (J - 1));
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = buf[pad(jl + r * J)];
    __syncthreads();
    if (item) {
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < 16; ++r) v[r] = cmul(v[r], tw[(r - 1) * Ns + k]);
        }
        dft<16>(v);
        const int base = (j - k) * 16 + k;
#pragma unroll
        for (int r = 0; r < 16; ++r) buf[pad(base + r * Ns)] = v[brev<16>(r)];
    }
    __syncthreads();
}

}  // namespace smem_fft
}  // namespace srg
