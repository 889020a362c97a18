// bp_kernel.cuh -- the tiled time-domain backprojection kernels (sm_100a).
//
// Work decomposition.  A burst's output window [firstpix, lastpix] x
// [0, nlines) is cut into TX x TY pixel tiles; a persistent grid pulls
// (burst, tile) items from a global counter, so one launch covers any number
// of bursts of uneven size.  Each thread owns M = TX*TY/NT pixels of the tile
// and walks the tile's pulse range [kmin, kmax) -- the union of its pixels'
// aperture windows -- in chunks of CK pulses.
//
// Per chunk, warp 0 derives the per-pulse quantities in FP64 (the
// satellite position; for the split form the tile's reference range R_c, its
// unit look vector and the phase of R_c), picks the range-bin window the tile
// needs for those pulses, and one thread issues a single 2D TMA load of
// CK pulse rows x WB bins of complex64 into shared memory.  All threads then
// read the two interpolation taps of each term from shared memory.  Terms
// whose bin falls outside the staged window (never for a tile whose geometry
// matches the window estimate) read global memory instead, so the result
// never depends on the estimate.
//
// The sum for pixel p (sentinel/azimuth_compress.cu:59-79):
//   out[p] = (1/(aze-azs)) * sum_{k in [azs,aze), R in [rngstart, rngend-dmrg]}
//            lerp(burst[k], (R - rngstart)/dmrg) * exp(+j 4 pi R / lambda),
//   R = |xyz[p] - satloc[k]|.
//
// FORM_FP64: R, the bin, the phase, sincos and the accumulation in FP64 with
// the reference's operation order (bit-identical bins and weights); FP32
// interpolation as azimuth_compress.cu:69.
//
// FORM_SPLIT: per tile and pulse one FP64 reference range R_c = |x_c - s_k|
// (x_c: ECEF of the tile-centre pixel) with unit vector u_k.  For pixel
// offset d = xyz[p] - x_c (FP64, rounded to FP32 once per pixel):
//   dR = R - R_c = w + n / (2 (R_c + w)),  w = d.u_k,  n = |d|^2 - w^2
// (exact identity up to terms < 1e-8 m for |d| < 1 km), evaluated in FP32 as
//   dR = w + n * (1/(2R_c)) * (1 - w/R_c).
// The phase needs frac(2 R / lambda) to ~1e-4 cycle, far below the FP32
// resolution of 2 w / lambda (~1e4 cycles).  It is carried as
//   phase = frac(K R_c) [FP64 per pulse] + c_p(k) + K * n-term,   K = 2/lambda,
// where c_p(k) = frac(K d.u_k) is seeded once per pixel and tile with
// compensated (double-float) two-product/two-sum arithmetic and then advanced
// pulse to pulse by the exact increment K d.(u_{k+1} - u_k) (FP64-derived,
// ~0.05 cycle per pulse), re-reduced to [-1/2, 1/2] at every chunk.  The
// accumulated rounding of c stays below 1e-5 cycle over a full aperture.
#pragma once
#include <climits>
#include <cuda.h>
#include "common.cuh"
#include "geom.cuh"
#include "ptx.cuh"

namespace srg {

enum { FORM_FP64 = 0, FORM_SPLIT = 1 };

struct Ctl {
    uint64_t bar;
    int item, kmin, kmax, bmin, bmax, x0, need, abort;
    double xc[3];
    double rc0, rc1;      // R_c at kmin and kmax-1
    float seed_hi[3], seed_lo[3];
};

// Unevaluated-sum (double-float) helpers for the seed.
__device__ __forceinline__ void two_sum(float a, float b, float &s, float &e) {
    s = __fadd_rn(a, b);
    const float bb = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}
__device__ __forceinline__ void two_prod(float a, float b, float &p, float &e) {
    p = __fmul_rn(a, b);
    e = __fmaf_rn(a, b, -p);
}

// frac(K * (d . u)) with d = dh + dl, u = uh + ul, K = Kh + Kl, all float,
// in double-float arithmetic; |result| <= ~0.5.  The dot product d . u is
// returned as the unevaluated sum whi + wlo.
__device__ __forceinline__ float seed_phase(const float dh[3], const float dl[3], const float uh[3],
                                            const float ul[3], float Kh, float Kl, float *whi,
                                            float *wlo) {
    float p0, e0, p1, e1, p2, e2;
    two_prod(dh[0], uh[0], p0, e0);
    two_prod(dh[1], uh[1], p1, e1);
    two_prod(dh[2], uh[2], p2, e2);
    float s1, t1, s2, t2;
    two_sum(p0, p1, s1, t1);
    two_sum(s1, p2, s2, t2);
    float lo = t1 + t2 + e0 + e1 + e2;
    lo = fmaf(dh[0], ul[0], lo);
    lo = fmaf(dh[1], ul[1], lo);
    lo = fmaf(dh[2], ul[2], lo);
    lo = fmaf(dl[0], uh[0], lo);
    lo = fmaf(dl[1], uh[1], lo);
    lo = fmaf(dl[2], uh[2], lo);
    if (whi) {
        *whi = s2;
        *wlo = lo;
    }
    // (s2 + lo) * (Kh + Kl)
    float P, E;
    two_prod(s2, Kh, P, E);
    float lo2 = fmaf(s2, Kl, fmaf(lo, Kh, E));
    const float f = __fsub_rn(P, rintf(P));  // exact: |P| < 2^23
    const float c = f + lo2;
    return c - rintf(c);
}

template <int TX, int TY, int NT>
struct PixelMap {
    static constexpr int NPIX = TX * TY;
    static constexpr int M = NPIX / NT;
    static_assert(NPIX % NT == 0, "tile must be a multiple of the block");
    __device__ static __forceinline__ void at(int tid, int m, int &x, int &y) {
        const int li = tid + m * NT;
        x = li % TX;
        y = li / TX;
    }
};

__device__ __forceinline__ int warp_min(int v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int warp_max(int v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ float2 ld_sample(const BurstDev &B, int k, int gi) {
    const int p = gi - B.bin0;  // column of bin gi in the lines held
    if (gi >= 0 && gi < B.S && (unsigned)p < (unsigned)B.nbins && k < B.P)
        return __ldg(B.burst + (long long)k * B.ldb + p);
    return make_float2(0.f, 0.f);
}

// Bytes of dynamic shared memory for a kernel shape.
template <int FORM, int CK>
__host__ __device__ constexpr int params_bytes() {
    return FORM == FORM_SPLIT ? CK * 48 : CK * 32;
}
// The sample window starts at the first 1024-byte boundary after the
// parameters (TMA destination alignment); the launch reserves the slack.
constexpr int kSampleAlign = 1024;

template <int FORM, int TX, int TY, int NT, int CK>
__global__ void __launch_bounds__(NT)
bp_tiles(const BurstDev *__restrict__ bursts, int nbursts, int total_tiles,
         const CUtensorMap *__restrict__ tmaps, int *__restrict__ work_counter,
         int *__restrict__ err, int WB, const int *__restrict__ tile_list) {
    using PM = PixelMap<TX, TY, NT>;
    constexpr int M = PM::M;
    static_assert(CK <= 32, "one warp prepares a chunk");
    extern __shared__ __align__(128) unsigned char dsm[];
    __shared__ Ctl ctl;
    constexpr int PB = params_bytes<FORM, CK>();
    float4 *prm4 = reinterpret_cast<float4 *>(dsm);          // split: 3 float4 per pulse
    double *prmd = reinterpret_cast<double *>(dsm);          // fp64: 4 doubles per pulse
    float2 *samp;
    {
        const uint32_t off = smem_u32(dsm + PB);
        samp = reinterpret_cast<float2 *>(dsm + PB + ((kSampleAlign - (off & (kSampleAlign - 1))) &
                                                     (kSampleAlign - 1)));
    }
    const int tid = threadIdx.x;
    const int lane = tid & 31;

    if (tid == 0) {
        mbar_init(&ctl.bar, 1);
        fence_barrier_init();
    }
    __syncthreads();
    uint32_t phase = 0;
    // work items index the list of tiles with a formed pixel when there is one
    const int nitems = tile_list ? tile_list[0] : total_tiles;

    for (;;) {
        if (tid == 0) ctl.item = atomicAdd(work_counter, 1);
        __syncthreads();
        const int item = ctl.item;
        if (item >= nitems) break;
        const int tile = tile_list ? tile_list[1 + item] : item;
        int b = 0;
        while (b + 1 < nbursts && bursts[b + 1].tile_base <= tile) ++b;
        const BurstDev &B = bursts[b];
        const int ti = tile - B.tile_base;
        const int px0 = B.firstpix + (ti % B.tiles_x) * TX;
        const int ly0 = (ti / B.tiles_x) * TY;

        // ---- prologue: pixel ECEF, aperture windows, tile pulse range ----
        if (tid == 0) {
            ctl.kmin = INT_MAX;
            ctl.kmax = INT_MIN;
            ctl.bmin = INT_MAX;
            ctl.bmax = INT_MIN;
            ctl.abort = 0;
        }
        __syncthreads();
        double X[M][3];
        int azs[M], aze[M];
        int lk0 = INT_MAX, lk1 = INT_MIN;
#pragma unroll
        for (int m = 0; m < M; ++m) {
            int x, y;
            PM::at(tid, m, x, y);
            const int px = px0 + x, line = ly0 + y;
            X[m][0] = X[m][1] = X[m][2] = 0.0;
            azs[m] = aze[m] = 0;
            if (px <= B.lastpix_eff && line < B.nlines) {
                const double h = (double)B.dem[(long long)line * B.dem_ld + px];
                pixel_ecef(B, line, px, h, X[m][0], X[m][1], X[m][2]);
                const double az = pixel_azoff(B, B.coef + 3 * line, px);
                pixel_window(B, az, azs[m], aze[m]);
                if (aze[m] > azs[m]) {
                    lk0 = min(lk0, azs[m]);
                    lk1 = max(lk1, aze[m]);
                }
            }
        }
        lk0 = warp_min(lk0);
        lk1 = warp_max(lk1);
        if (lane == 0 && lk0 < lk1) {
            atomicMin(&ctl.kmin, lk0);
            atomicMax(&ctl.kmax, lk1);
        }
        __syncthreads();
        const int kmin = ctl.kmin, kmax = ctl.kmax;
        if (kmin >= kmax) {
            // nothing formed in this tile: zeros
#pragma unroll
            for (int m = 0; m < M; ++m) {
                int x, y;
                PM::at(tid, m, x, y);
                const int px = px0 + x, line = ly0 + y;
                if (px <= B.lastpix_eff && line < B.nlines)
                    B.out[(long long)line * B.out_ld + (px - B.out_pix0)] = make_float2(0.f, 0.f);
            }
            __syncthreads();
            continue;
        }

        // ---- tile reference point and range-window bounds ----
        if (tid == 0) {
            const int cx = min(max(px0 + TX / 2, B.firstpix), B.lastpix_eff);
            const int cy = min(ly0 + TY / 2, B.nlines - 1);
            const double h = (double)B.dem[(long long)cy * B.dem_ld + cx];
            double xc[3];
            pixel_ecef(B, cy, cx, h, xc[0], xc[1], xc[2]);
            ctl.xc[0] = xc[0];
            ctl.xc[1] = xc[1];
            ctl.xc[2] = xc[2];
            const double *s0 = B.satloc + 3 * kmin;
            const double *s1 = B.satloc + 3 * (kmax - 1);
            const double u0 = xc[0] - s0[0], u1 = xc[1] - s0[1], u2 = xc[2] - s0[2];
            const double r0 = sqrt(u0 * u0 + u1 * u1 + u2 * u2);
            const double v0 = xc[0] - s1[0], v1 = xc[1] - s1[1], v2 = xc[2] - s1[2];
            ctl.rc0 = r0;
            ctl.rc1 = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
            if (FORM == FORM_SPLIT) {
                const double uu[3] = {u0 / r0, u1 / r0, u2 / r0};
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const float hi = __double2float_rn(uu[c]);
                    ctl.seed_hi[c] = hi;
                    ctl.seed_lo[c] = __double2float_rn(uu[c] - (double)hi);
                }
            }
        }
        __syncthreads();
        {
            int lb0 = INT_MAX, lb1 = INT_MIN;
            const double *s0 = B.satloc + 3 * kmin;
            const double *s1 = B.satloc + 3 * (kmax - 1);
#pragma unroll
            for (int m = 0; m < M; ++m) {
                if (aze[m] > azs[m]) {
                    const double a0 = X[m][0] - s0[0], a1 = X[m][1] - s0[1], a2 = X[m][2] - s0[2];
                    const double c0 = X[m][0] - s1[0], c1 = X[m][1] - s1[1], c2 = X[m][2] - s1[2];
                    const double d0 = (sqrt(a0 * a0 + a1 * a1 + a2 * a2) - ctl.rc0) * B.inv_dmrg;
                    const double d1 = (sqrt(c0 * c0 + c1 * c1 + c2 * c2) - ctl.rc1) * B.inv_dmrg;
                    lb0 = min(lb0, (int)floor(fmin(d0, d1)));
                    lb1 = max(lb1, (int)ceil(fmax(d0, d1)));
                }
            }
            lb0 = warp_min(lb0);
            lb1 = warp_max(lb1);
            if (lane == 0 && lb0 <= lb1) {
                atomicMin(&ctl.bmin, lb0);
                atomicMax(&ctl.bmax, lb1);
            }
        }

        // ---- per-pixel state of the chosen form ----
        float d[M][3], dd[M], c[M];
        float accr[M], acci[M];
        double accr_d[M], acci_d[M];
#pragma unroll
        for (int m = 0; m < M; ++m) {
            accr[m] = acci[m] = 0.f;
            accr_d[m] = acci_d[m] = 0.0;
            d[m][0] = d[m][1] = d[m][2] = 0.f;
            dd[m] = c[m] = 0.f;
            if (FORM == FORM_SPLIT && aze[m] > azs[m]) {
                float dh[3], dl[3];
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    const double dv = X[m][q] - ctl.xc[q];
                    dh[q] = __double2float_rn(dv);
                    dl[q] = __double2float_rn(dv - (double)dh[q]);
                    d[m][q] = dh[q];
                }
                dd[m] = fmaf(dh[0], dh[0], fmaf(dh[1], dh[1], dh[2] * dh[2]));
                c[m] = seed_phase(dh, dl, ctl.seed_hi, ctl.seed_lo, B.K_hi, B.K_lo, nullptr, nullptr);
            }
        }
        __syncthreads();
        const int bmin = ctl.bmin - 1;
        const int bmax = ctl.bmax + 2;
        const double xcx = ctl.xc[0], xcy = ctl.xc[1], xcz = ctl.xc[2];
        const bool use_tma = B.tmap >= 0;

        // ---- pulse chunks ----
        for (int k0 = kmin; k0 < kmax; k0 += CK) {
            const int nk = min(CK, kmax - k0);
            __syncthreads();  // the previous chunk's readers are done
            if (tid < 32) {
                const int k = k0 + lane;
                const bool on = lane < nk;
                double rbabs = 0.0;
                if (on) {
                    const double *s = B.satloc + 3 * k;
                    const double sx = s[0], sy = s[1], sz = s[2];
                    const double ux = xcx - sx, uy = xcy - sy, uz = xcz - sz;
                    const double R = sqrt(ux * ux + uy * uy + uz * uz);
                    rbabs = (R - B.rngstart) * B.inv_dmrg;
                    if (FORM == FORM_SPLIT) {
                        const double iR = 1.0 / R;
                        const double ex = ux * iR, ey = uy * iR, ez = uz * iR;
                        const double *sn = B.satloc + 3 * min(k + 1, B.P - 1);
                        const double nx = xcx - sn[0], ny = xcy - sn[1], nz = xcz - sn[2];
                        const double iRn = 1.0 / sqrt(nx * nx + ny * ny + nz * nz);
                        const double q = R * B.K;
                        const float ref = __double2float_rn(q - rint(q));
                        float4 *p = prm4 + 3 * lane;
                        p[0] = make_float4(__double2float_rn(ex), __double2float_rn(ey),
                                           __double2float_rn(ez), ref);
                        p[1] = make_float4(__double2float_rn(B.K * (nx * iRn - ex)),
                                           __double2float_rn(B.K * (ny * iRn - ey)),
                                           __double2float_rn(B.K * (nz * iRn - ez)), 0.f);
                        p[2] = make_float4(__double2float_rn(0.5 * iR), __double2float_rn(iR), 0.f, 0.f);
                    } else {
                        double *p = prmd + 4 * lane;
                        p[0] = sx;
                        p[1] = sy;
                        p[2] = sz;
                    }
                }
                int lo = on ? (int)floor(rbabs) : INT_MAX;
                int hi = on ? (int)ceil(rbabs) : INT_MIN;
                lo = warp_min(lo);
                hi = warp_max(hi);
                const int x0 = (lo + bmin) & ~1;  // TMA: x * 8 bytes must be 16-byte aligned
                if (FORM == FORM_SPLIT && on) prm4[3 * lane + 1].w = __double2float_rn(rbabs - (double)x0);
                if (lane == 0) {
                    ctl.x0 = x0;
                    ctl.need = hi + bmax - x0 + 1;
                    if (use_tma) {
                        if (k0 == kmin) fence_tensormap_acquire(tmaps + B.tmap);
                        fence_proxy_async_shared();
                        mbar_arrive_expect_tx(&ctl.bar, (uint32_t)(WB * CK * 8));
                        tma_load_2d(samp, tmaps + B.tmap, &ctl.bar, x0 - B.bin0, k0);
                    }
                }
            }
            __syncthreads();
            const int x0 = ctl.x0;
            if (!use_tma) {
                for (int idx = tid; idx < CK * WB; idx += NT) {
                    const int j = idx / WB;
                    samp[idx] = ld_sample(B, k0 + j, x0 + (idx - j * WB));
                }
                __syncthreads();
            } else {
                const bool ok = mbar_wait_bounded(&ctl.bar, phase, B.spin);
                if (__syncthreads_or(!ok)) {
                    // give up on this launch: record, let the copy drain, leave
                    if (tid == 0) atomicOr(err, ERR_TMA_TIMEOUT);
                    mbar_wait_bounded(&ctl.bar, phase);
                    return;
                }
                phase ^= 1;
            }

            if (FORM == FORM_SPLIT) {
                const float tlo = (float)(-(double)x0);
                const float thi = __double2float_rn((B.rmax - B.rngstart) * B.inv_dmrg - (double)x0);
                const float invd = B.inv_dmrg_f, Kf = B.K_f;
                for (int j = 0; j < nk; ++j) {
                    const int k = k0 + j;
                    const float4 pa = prm4[3 * j + 0];
                    const float4 pb = prm4[3 * j + 1];
                    const float4 pc = prm4[3 * j + 2];
                    const float2 *row = samp + j * WB;
#pragma unroll
                    for (int m = 0; m < M; ++m) {
                        const float w = fmaf(d[m][0], pa.x, fmaf(d[m][1], pa.y, d[m][2] * pa.z));
                        const float n = fmaf(-w, w, dd[m]);
                        const float s = fmaf(-w, pc.y, 1.f);
                        const float dr2 = (n * pc.x) * s;
                        const float t = fmaf(w + dr2, invd, pb.w);
                        const float ph = fmaf(dr2, Kf, c[m] + pa.w);
                        c[m] = fmaf(d[m][0], pb.x, fmaf(d[m][1], pb.y, fmaf(d[m][2], pb.z, c[m])));
                        const float fl = floorf(t);
                        const int i = (int)fl;
                        const float fr = t - fl;
                        const bool ok = (k >= azs[m]) & (k < aze[m]) & (t >= tlo) & (t <= thi);
                        const bool inwin = (unsigned)i < (unsigned)(WB - 1);
                        const int is = inwin ? i : 0;
                        float2 s0 = row[is], s1 = row[is + 1];
                        if (ok && !inwin) {
                            s0 = ld_sample(B, k, i + x0);
                            s1 = ld_sample(B, k, i + x0 + 1);
                        }
                        float vr = fmaf(fr, s1.x - s0.x, s0.x);
                        float vi = fmaf(fr, s1.y - s0.y, s0.y);
                        vr = ok ? vr : 0.f;
                        vi = ok ? vi : 0.f;
                        float sn, cs;
                        __sincosf(6.283185307179586f * ph, &sn, &cs);
                        accr[m] = fmaf(vr, cs, fmaf(-vi, sn, accr[m]));
                        acci[m] = fmaf(vr, sn, fmaf(vi, cs, acci[m]));
                    }
                }
#pragma unroll
                for (int m = 0; m < M; ++m) c[m] -= rintf(c[m]);
            } else {
                const double rs = B.rngstart, rmax = B.rmax, dm = B.dmrg, k4 = B.k4pi;
                for (int j = 0; j < nk; ++j) {
                    const int k = k0 + j;
                    const double sx = prmd[4 * j + 0], sy = prmd[4 * j + 1], sz = prmd[4 * j + 2];
                    const float2 *row = samp + j * WB;
#pragma unroll
                    for (int m = 0; m < M; ++m) {
                        if (k < azs[m] || k >= aze[m]) continue;
                        const double vx = dsub(X[m][0], sx), vy = dsub(X[m][1], sy),
                                     vz = dsub(X[m][2], sz);
                        const double R = __dsqrt_rn(dadd(dadd(dmul(vx, vx), dmul(vy, vy)), dmul(vz, vz)));
                        if (!(R >= rs && R <= rmax)) continue;
                        const double r = ddiv(dsub(R, rs), dm);
                        const double fl = floor(r);
                        const int ig = (int)fl;
                        const double fr = dsub(r, fl);
                        const float w0 = __double2float_rn(dsub(1.0, fr));
                        const float w1 = __double2float_rn(fr);
                        const int i = ig - x0;
                        float2 s0, s1;
                        if ((unsigned)i < (unsigned)(WB - 1)) {
                            s0 = row[i];
                            s1 = row[i + 1];
                        } else {
                            s0 = ld_sample(B, k, ig);
                            s1 = ld_sample(B, k, ig + 1);
                        }
                        const float cre = __fadd_rn(__fmul_rn(s0.x, w0), __fmul_rn(s1.x, w1));
                        const float cim = __fadd_rn(__fmul_rn(s0.y, w0), __fmul_rn(s1.y, w1));
                        double sn, cs;
                        sincos(dmul(k4, R), &sn, &cs);
                        const double a = (double)cre, bq = (double)cim;
                        accr_d[m] += a * cs - bq * sn;
                        acci_d[m] += a * sn + bq * cs;
                    }
                }
            }
        }

        // ---- epilogue: scale by 1/(aze-azs) in FP32, as azimuth_compress.cu:78-79 ----
#pragma unroll
        for (int m = 0; m < M; ++m) {
            int x, y;
            PM::at(tid, m, x, y);
            const int px = px0 + x, line = ly0 + y;
            if (px <= B.lastpix_eff && line < B.nlines) {
                float2 o = make_float2(0.f, 0.f);
                const int n = aze[m] - azs[m];
                if (n > 0) {
                    const float sc = __double2float_rn(ddiv(1.0, (double)n));
                    const float re = FORM == FORM_SPLIT ? accr[m] : __double2float_rn(accr_d[m]);
                    const float im = FORM == FORM_SPLIT ? acci[m] : __double2float_rn(acci_d[m]);
                    o = make_float2(__fmul_rn(re, sc), __fmul_rn(im, sc));
                }
                B.out[(long long)line * B.out_ld + (px - B.out_pix0)] = o;
            }
        }
        __syncthreads();
    }
}

}  // namespace srg
