// bp_ws.cuh -- warp-specialised tiled backprojection (sm_100a).
//
// Same sum, work decomposition and arithmetic forms as bp_kernel.cuh (read
// that header first); this variant reorganises the pulse loop:
//
// * One producer warp per CTA prepares chunk c+1.. while NC consumer warps
//   work on chunk c: it derives the per-pulse quantities in FP64, picks the
//   chunk's range-bin window and issues the TMA load of CK pulse rows x WB
//   bins into an NS-deep ring of shared-memory stages.  Full/empty mbarriers
//   (bounded waits) replace CTA-wide barriers inside a tile.
// * Chunks lying inside every formed pixel's aperture window and inside the
//   range window ("interior" chunks, the common case) run without per-term
//   predicates.  The producer proves, per chunk, that no term can leave the
//   staged window: a pixel's bin offset from the tile centre is linear in
//   the look direction u_k, so between the tile's first and last pulse it
//   deviates from the straight line through its end values (which the
//   window covers with a one-bin margin) by at most
//   max|d| * max_k |u_k - u_lin(k)| / dmrg; the chunk is marked interior
//   only when that bound is below half a bin (a smooth orbit gives ~1e-4).
//   The taps' index is still clamped for memory safety.  Edge chunks use the
//   general path (per-term aperture and range tests, global-memory fallback
//   for taps outside the window).
// * Split form: the per-term state is w = d.u_k, held as the unevaluated sum
//   of a per-tile constant whi and a small accumulator dwa (|dwa| < ~1 m, so
//   its rounding stays below 1e-6 m over a whole aperture), and the phase
//   c = 2 pi frac(K d.u_k) in radians; whi + dwa and c are seeded once per
//   pixel and tile in compensated arithmetic and both advance by the same
//   increment dw = d.(u_{k+1} - u_k), exact to FP32 relative precision
//   because |dw| <~ 1e-3 m.  The second-order range term
//   dr2 = (|d|^2 - w^2) (1/(2 R_c) - w/(2 R_c^2)) changes by < 1e-5 m over a
//   chunk and is linear in the pulse index to ~1e-9 m, so it is evaluated
//   exactly once per pixel and chunk, with its slope g = (d dr2 / dw) * dw_mid,
//   and folded into the two accumulators, which then advance by dw + g: per
//   term only the increment, two accumulations, the bin and the phase remain.
// * Closed forms (split form, chunks whose taps all lie in the staged window;
//   at the aperture edges with a per-term azimuth-window test): over one chunk R_c is a
//   quadratic in the pulse index and u_{k+1} - u_k is linear in it (a smooth
//   orbit leaves residuals of ~1e-10 m), so the bin and the phase of every
//   term are quadratics in the pulse index whose coefficients each pixel
//   derives once per chunk; a term then costs two adds for each (forward
//   differences from the chunk's first pulse; their rounding over <= 31
//   pulses raised the image phase error against the FP64 form from 0.018 to
//   0.021 mrad RMS on the IW scene, for 4 % speed).  The producer fits R_c and the
//   increments and checks the fits at every pulse of the chunk; a chunk whose
//   bound exceeds kPolyTolRad of phase (an orbit with a kink, a chunk shorter
//   than three pulses) takes the per-pulse form instead.  The tap index comes
//   from an add rounded toward -inf (floor in the mantissa), which keeps the
//   conversion pipe free for the sine and cosine.
#pragma once
#include <climits>
#include <cuda.h>
#include <type_traits>
#include "bp_kernel.cuh"

namespace srg {

// 16-byte aligned: the consumers read it with vector loads (a quarter of the
// scalar loads per chunk).
struct __align__(16) StageHdr {
    int x0;        // first staged bin
    int fast;      // 1: every tap of the chunk lies in the staged window and the range limits
    int interior;  // 1: the chunk lies inside every formed pixel's azimuth window
    int poly;      // 1: the closed forms below hold to < kPolyTolRad of phase
    float tlo, thi;       // range test in window-relative bins (general path)
    float dmx, dmy, dmz;  // u_{k+1} - u_k at the chunk's middle pulse
    float inv2R, c2;      // 1/(2 R_c) and 1/(2 R_c^2) at the chunk's middle pulse
    // closed forms over the chunk in the centred pulse index f = j - (nk-1)/2:
    // R_c at the chunk's first pulse and its first and second forward differences:
    float r0, r1, r2;     // as window-relative bins
    float p0, p1, p2;     // as phase (rad), p0 in [-pi, pi]
    float u0x, u0y, u0z;  // u_{j+1} - u_j = u0 + j us (j = pulse index within the chunk)
    float usx, usy, usz;
};

struct CtlWS {
    uint64_t full[4], empty[4];
    int item, kmin, kmax, azs_max, aze_min, bmin, bmax, abort;
    int dmax_bits;        // max |d| over formed pixels (non-negative float bits)
    unsigned spin;        // poll limit of the bounded waits
    double xc[3];
    double rc0, rc1;
    double ua[3], ub[3];  // unit look vectors at kmin and kmax-1
    float seed_hi[3], seed_lo[3];
};

constexpr double kTwoPi = 6.283185307179586476925;
constexpr float kTwoPiHi = 6.28318548202514648f;     // float(2 pi)
constexpr float kTwoPiLo = -1.74845553e-7f;          // 2 pi - float(2 pi)
constexpr float kInvTwoPi = 0.159154943091895336f;
// Largest phase error (rad) the producer accepts from the chunk's closed forms
// (quadratic R_c, linear look-vector increments) before it falls back to the
// per-pulse form; the fit residuals of a smooth orbit are ~1e-8 rad.
constexpr double kPolyTolRad = 1e-4;

// 1/n for the pulse counts of a chunk (n <= 32), rounded to nearest: the
// producer's fits multiply by these instead of dividing (an IEEE division is
// a dependent sequence of about ten instructions on the producer's path).
__constant__ float kRecipSmall[33] = {
    0.f,        1.f / 1,  1.f / 2,  1.f / 3,  1.f / 4,  1.f / 5,  1.f / 6,  1.f / 7,  1.f / 8,
    1.f / 9,    1.f / 10, 1.f / 11, 1.f / 12, 1.f / 13, 1.f / 14, 1.f / 15, 1.f / 16, 1.f / 17,
    1.f / 18,   1.f / 19, 1.f / 20, 1.f / 21, 1.f / 22, 1.f / 23, 1.f / 24, 1.f / 25, 1.f / 26,
    1.f / 27,   1.f / 28, 1.f / 29, 1.f / 30, 1.f / 31, 1.f / 32};

// floor(t) for -2^22 <= t < 2^22 without the conversion pipe: adding 1.5 * 2^23
// rounded toward -inf leaves floor(t) in the low mantissa bits.
constexpr float kFloorMagic = 12582912.f;
constexpr int kFloorMagicBits = 0x4B400000;
// Width (pixels across) of the block of 32 pixels a warp owns per slot.  The
// two taps of a lane are 8-byte words of one staged row; lanes of a half-warp
// whose bins differ by a multiple of 16 share shared-memory banks, so narrow
// blocks (fewer range bins per half-warp) conflict less.
#ifndef SRG_PIX_BLOCK_X
#define SRG_PIX_BLOCK_X 4
#endif
constexpr int kPixBlockX = SRG_PIX_BLOCK_X;

// Per-pulse parameters of one chunk (split: 2 x float4; FP64: satloc + pad).
template <int FORM>
struct PulseParams;
template <>
struct PulseParams<FORM_SPLIT> {
    float4 a;  // du (= u_{k+1} - u_k) x, y, z; ref phase (rad)
    float4 b;  // rb (window-relative bin of R_c), unused x3
};
template <>
struct PulseParams<FORM_FP64> {
    double s[4];  // satloc x, y, z, unused
};

template <int FORM, int CK>
__host__ __device__ constexpr int ws_params_bytes() {
    return (int)sizeof(PulseParams<FORM>) * CK;
}

// Dynamic shared memory of a shape: params of every stage, then the sample
// windows from the first 1024-byte boundary, then a 16-byte guard (a tap index
// masked to the row width may address the first sample after the last row).
template <int FORM, int CK, int NS>
__host__ __device__ constexpr int ws_smem_bytes(int WB) {
    return NS * ws_params_bytes<FORM, CK>() + 1024 + NS * CK * WB * 8 + 16;
}

// Tap index of a term from the bits of floor(t) + kFloorMagic.  The fast paths
// have proven t in [0, WB - 1); for memory safety any other t still lands in
// the stage: masked to the row when WB is a power of two (the magic's low bits
// are zero), clamped otherwise.
template <int WB>
__device__ __forceinline__ unsigned tap_index(float tm) {
    if constexpr ((WB & (WB - 1)) == 0) return __float_as_uint(tm) & (unsigned)(WB - 1);
    else return min(__float_as_uint(tm) - (unsigned)kFloorMagicBits, (unsigned)(WB - 2));
}

// Chunk schedule of a tile: the pulse range [kmin, kmax) is cut at ka and kb
// (the interior segment [ka, kb) lies inside every formed pixel's aperture)
// and each of the three segments into chunks of at most CK pulses, so that
// only the edge segments need the general path.
struct ChunkPlan {
    int kmin, ka, kb, kmax, na, nb, nc;
    __device__ __forceinline__ void init(int k0, int k1, int smax, int emin, int CK) {
        kmin = k0;
        kmax = k1;
        ka = max(k0, min(smax, k1));
        kb = max(ka, min(emin, k1));
        na = (ka - k0 + CK - 1) / CK;
        nb = (kb - ka + CK - 1) / CK;
        nc = (k1 - kb + CK - 1) / CK;
    }
    __device__ __forceinline__ int count() const { return na + nb + nc; }
    // first pulse and length of chunk c
    __device__ __forceinline__ void chunk(int c, int CK, int &k0, int &nk) const {
        if (c < na) {
            k0 = kmin + c * CK;
            nk = min(CK, ka - k0);
        } else if (c < na + nb) {
            k0 = ka + (c - na) * CK;
            nk = min(CK, kb - k0);
        } else {
            k0 = kb + (c - na - nb) * CK;
            nk = min(CK, kmax - k0);
        }
    }
};

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// WB: staged bins per pulse (the launch passes the same value as its last
// argument, shared with the first-generation kernels); MINB: blocks per SM
// the register allocation is sized for.
// GATE: the range lines may still be uploading (BurstDev::ready); the
// producer waits for each chunk's rows.  A separate instantiation, because
// the wait's code alone costs the ungated kernel ~4 % (measured).
template <int FORM, int TX, int TY, int NC, int CK, int NS, int WB, int MINB, bool GATE = false>
__global__ void __launch_bounds__((NC + 1) * 32, MINB)
bp_ws(const BurstDev *__restrict__ bursts, int nbursts, int total_tiles,
      const CUtensorMap *__restrict__ tmaps, int *__restrict__ work_counter,
      int *__restrict__ err, int /* window, = WB */, const int *__restrict__ tile_list) {
    constexpr int NCT = NC * 32;
    constexpr int M = TX * TY / NCT;
    // each warp and slot covers a PBX x PBY block of pixels (PBY = 32 / PBX)
    constexpr int PBX = (TY % (32 / kPixBlockX) == 0) ? kPixBlockX : 8, PBY = 32 / PBX;
    constexpr int BX = TX / PBX;
    static_assert(TX % PBX == 0 && TY % PBY == 0 && (TX / PBX) * (TY / PBY) == NC * M, "tile / warp map");
    static_assert(CK < 32, "the producer warp covers CK + 1 pulses");
    static_assert(NS >= 2 && NS <= 4, "stage ring");
    // every stage's TMA destination on a 128-byte boundary (the first stage
    // starts on a 1024-byte one), and the box rows a multiple of 16 bytes
    static_assert((CK * WB * 8) % 128 == 0 && WB % 2 == 0, "stage stride");
    using PP = PulseParams<FORM>;

    extern __shared__ __align__(128) unsigned char dsm[];
    __shared__ CtlWS ctl;
    __shared__ StageHdr hdr[NS];
    // per-tile line / column factors of the ECEF (a sheared tile touches
    // TY + lspan lines, lspan < kMaxShear)
    __shared__ double lat_tab[TY + kMaxShear][4], lon_tab[TX][2];
    PP *prm = reinterpret_cast<PP *>(dsm);
    float2 *samp0;
    {
        const uint32_t off = smem_u32(dsm + NS * ws_params_bytes<FORM, CK>());
        samp0 = reinterpret_cast<float2 *>(dsm + NS * ws_params_bytes<FORM, CK>() +
                                           ((1024 - (off & 1023)) & 1023));
    }
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const bool producer = warp == NC;

    if (tid == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(&ctl.full[s], 32);
            mbar_init(&ctl.empty[s], NC);
        }
        fence_barrier_init();
        ctl.abort = 0;
        ctl.spin = bursts[0].spin;
        // Later items are claimed by the producer once it has issued a tile's
        // last chunk, so the atomic's latency hides behind the consumers' last
        // chunks (claiming a whole tile ahead would unbalance the tail).
        ctl.item = atomicAdd(work_counter, 1);
    }
    __syncthreads();
    // work items index the list of tiles with a formed pixel when there is one
    const int nitems = tile_list ? tile_list[0] : total_tiles;
    // Range lines arriving in pulse order (GATE, one burst): take the tiles in
    // the order their pulses arrive.
    bool reverse = false;
    if constexpr (GATE) {
        if (nbursts == 1) reverse = lines_against_pulses(bursts[0]);
    }
    // GATE with row blocks: a tile's stores are counted once the CTA has
    // passed the barrier after them; the count that completes a row block
    // raises the block's word, releasing its copy back to the host.
    auto tile_stored = [&](const BurstDev &B, int ly0) {
        if constexpr (GATE) {
            if (tid == 0 && B.rb_done) {
                const int k = (ly0 / TY) / B.rb_tile_rows;
                if (atomicAdd(B.rb_count + k, 1) == B.rb_expect[k] - 1) {
                    __threadfence_system();
                    atomicExch(B.rb_done + k, B.rb_seq);
                }
            }
        }
    };
    uint32_t gchunk = 0;  // chunks issued/consumed by this CTA so far (uniform)
    uint32_t issued = 0, issued_par = 0;  // producer lane 0: stages with a TMA issued this tile
    int b = 0;  // burst of the current tile (tiles grow, so the search resumes here)

    for (;;) {
        if (tid == 0) {
            ctl.kmin = INT_MAX;
            ctl.kmax = INT_MIN;
            ctl.azs_max = INT_MIN;
            ctl.aze_min = INT_MAX;
            ctl.bmin = INT_MAX;
            ctl.bmax = INT_MIN;
            ctl.dmax_bits = 0;
        }
        __syncthreads();
        const int item = ctl.item;
        if (item >= nitems) break;
        const int order = reverse ? nitems - 1 - item : item;
        const int tile = tile_list ? tile_list[1 + order] : order;
        while (b + 1 < nbursts && bursts[b + 1].tile_base <= tile) ++b;
        const BurstDev &B = bursts[b];
        const int ti = tile - B.tile_base;
        // pixel (x, y) of the tile: column px0 + x, line
        // ly0 + y + tile_dline(shear, x) - dmax; its line factors are
        // lat_tab[y + tile_dline(shear, x) - dmax + lspan] (the table starts
        // at line ly0 - lspan)
        const int shear = B.shear;
        const int px0 = B.firstpix + (ti % B.tiles_x) * TX;
        const int ly0 = (ti / B.tiles_x) * TY;
        const int dmax = tile_dmax(shear, TX), lspan = tile_span(shear, TX);

        // ---- prologue ----
        // Phase A: consumers solve their pixels' aperture windows; the producer
        // warp, idle until the tile's pulse range is known, builds the tile's
        // line / column ECEF factors and the tile-centre position.
        double X[M][3];
        int azs[M], aze[M];
        short hgt[M];
        if (!producer) {
            int k0 = INT_MAX, k1 = INT_MIN, smax = INT_MIN, emin = INT_MAX;
#pragma unroll
            for (int m = 0; m < M; ++m) {
                const int bi = warp + NC * m;
                const int x = PBX * (bi % BX) + lane % PBX, y = PBY * (bi / BX) + lane / PBX;
                const int px = px0 + x, line = ly0 + y + tile_dline(shear, x) - dmax;
                X[m][0] = X[m][1] = X[m][2] = 0.0;
                azs[m] = aze[m] = 0;
                hgt[m] = 0;
                if (px <= B.lastpix_eff && line >= 0 && line < B.nlines) {
                    hgt[m] = B.dem[(long long)line * B.dem_ld + px];
                    pixel_window(B, pixel_azoff(B, B.coef + 3 * line, px), azs[m], aze[m]);
                    if (aze[m] > azs[m]) {
                        k0 = min(k0, azs[m]);
                        k1 = max(k1, aze[m]);
                        smax = max(smax, azs[m]);
                        emin = min(emin, aze[m]);
                    }
                }
            }
            k0 = warp_min(k0);
            k1 = warp_max(k1);
            smax = warp_max(smax);
            emin = warp_min(emin);
            if (lane == 0 && k0 < k1) {
                atomicMin(&ctl.kmin, k0);
                atomicMax(&ctl.kmax, k1);
                atomicMax(&ctl.azs_max, smax);
                atomicMin(&ctl.aze_min, emin);
            }
        } else {
            for (int r = lane; r < TY + lspan + TX; r += 32) {
                if (r < TY + lspan) {
                    const LineTrig L = line_trig(B, ly0 - lspan + r);
                    lat_tab[r][0] = L.slat;
                    lat_tab[r][1] = L.clat;
                    lat_tab[r][2] = L.re;
                    lat_tab[r][3] = L.rez;
                } else {
                    col_trig(B, px0 + r - TY - lspan, lon_tab[r - TY - lspan][0],
                             lon_tab[r - TY - lspan][1]);
                }
            }
            __syncwarp();
            if (lane == 0) {
                // tile-centre pixel, inside the burst (its factors are in the
                // tables; the clamp only guards the index)
                const int cx = min(max(px0 + TX / 2, B.firstpix), B.lastpix_eff);
                const int tx = cx - px0;
                const int cy = min(max(ly0 + TY / 2 + tile_dline(shear, tx) - dmax, 0), B.nlines - 1);
                const int ty = min(max(cy - ly0 + lspan, 0), TY + lspan - 1);
                pixel_ecef_from(lat_tab[ty][0], lat_tab[ty][1], lat_tab[ty][2], lat_tab[ty][3],
                                lon_tab[tx][0], lon_tab[tx][1],
                                (double)B.dem[(long long)cy * B.dem_ld + cx], ctl.xc[0], ctl.xc[1],
                                ctl.xc[2]);
            }
        }
        __syncthreads();
        const int kmin = ctl.kmin, kmax = ctl.kmax;
        if (kmin >= kmax) {
            if (!producer) {
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    const int bi = warp + NC * m;
                    const int x = PBX * (bi % BX) + lane % PBX, y = PBY * (bi / BX) + lane / PBX;
                    const int px = px0 + x, line = ly0 + y + tile_dline(shear, x) - dmax;
                    if (px <= B.lastpix_eff && line >= 0 && line < B.nlines)
                        B.out[(long long)line * B.out_ld + (px - B.out_pix0)] = make_float2(0.f, 0.f);
                }
            } else if (lane == 0) {
                ctl.item = atomicAdd(work_counter, 1);
            }
            if (GATE && B.rb_done) __threadfence();
            __syncthreads();
            tile_stored(B, ly0);
            continue;
        }
        // Phase B: consumers place their formed pixels; the producer's lane 0
        // derives the ranges and look vectors of the tile centre at the first
        // and last pulse and the compensated seed of the look vector.
        if (!producer) {
#pragma unroll
            for (int m = 0; m < M; ++m) {
                if (aze[m] > azs[m]) {
                    const int bi = warp + NC * m;
                    const int x = PBX * (bi % BX) + lane % PBX, y = PBY * (bi / BX) + lane / PBX;
                    const int ty = y + tile_dline(shear, x) - dmax + lspan;  // the pixel's table line
                    pixel_ecef_from(lat_tab[ty][0], lat_tab[ty][1], lat_tab[ty][2], lat_tab[ty][3],
                                    lon_tab[x][0], lon_tab[x][1], (double)hgt[m], X[m][0], X[m][1],
                                    X[m][2]);
                }
            }
        } else if (lane == 0) {
            const double xc[3] = {ctl.xc[0], ctl.xc[1], ctl.xc[2]};
            const double *s0 = B.satloc + 3 * kmin;
            const double *s1 = B.satloc + 3 * (kmax - 1);
            const double u0 = xc[0] - s0[0], u1 = xc[1] - s0[1], u2 = xc[2] - s0[2];
            const double r0 = sqrt(u0 * u0 + u1 * u1 + u2 * u2);
            const double v0 = xc[0] - s1[0], v1 = xc[1] - s1[1], v2 = xc[2] - s1[2];
            const double r1 = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
            ctl.rc0 = r0;
            ctl.rc1 = r1;
            const double i0 = 1.0 / r0, i1 = 1.0 / r1;
            const double uu[3] = {u0 * i0, u1 * i0, u2 * i0};
            ctl.ua[0] = uu[0];
            ctl.ua[1] = uu[1];
            ctl.ua[2] = uu[2];
            ctl.ub[0] = v0 * i1;
            ctl.ub[1] = v1 * i1;
            ctl.ub[2] = v2 * i1;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float hi = __double2float_rn(uu[c]);
                ctl.seed_hi[c] = hi;
                ctl.seed_lo[c] = __double2float_rn(uu[c] - (double)hi);
            }
        }
        __syncthreads();
        float d[M][3], dd[M], cph[M], whi[M], dwa[M], accr[M], acci[M];
        double accr_d[M], acci_d[M];
        if (!producer) {
            int lb0 = INT_MAX, lb1 = INT_MIN;
            float dmx = 0.f;
            // bin offsets of the pixel from the tile centre at the tile's first and
            // last pulse, to second order in d = x - x_c (error < 1e-4 m at
            // |d| < 1 km; the window keeps a bin of margin on both sides)
            const float ua0 = (float)ctl.ua[0], ua1 = (float)ctl.ua[1], ua2 = (float)ctl.ua[2];
            const float ub0 = (float)ctl.ub[0], ub1 = (float)ctl.ub[1], ub2 = (float)ctl.ub[2];
            const float h0 = (float)(0.5 / ctl.rc0), h1 = (float)(0.5 / ctl.rc1);
            const float invd = B.inv_dmrg_f;
#pragma unroll
            for (int m = 0; m < M; ++m) {
                accr[m] = acci[m] = 0.f;
                accr_d[m] = acci_d[m] = 0.0;
                d[m][0] = d[m][1] = d[m][2] = 0.f;
                dd[m] = cph[m] = whi[m] = dwa[m] = 0.f;
                if (aze[m] > azs[m]) {
                    float dh[3], dl[3];
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        const double dv = X[m][q] - ctl.xc[q];
                        dh[q] = __double2float_rn(dv);
                        dl[q] = __double2float_rn(dv - (double)dh[q]);
                        d[m][q] = dh[q];
                    }
                    dd[m] = fmaf(dh[0], dh[0], fmaf(dh[1], dh[1], dh[2] * dh[2]));
                    const float wa = fmaf(dh[0], ua0, fmaf(dh[1], ua1, dh[2] * ua2));
                    const float wb = fmaf(dh[0], ub0, fmaf(dh[1], ub1, dh[2] * ub2));
                    const float e0 = fmaf(fmaf(-wa, wa, dd[m]), h0, wa) * invd;
                    const float e1 = fmaf(fmaf(-wb, wb, dd[m]), h1, wb) * invd;
                    lb0 = min(lb0, (int)floorf(fminf(e0, e1)));
                    lb1 = max(lb1, (int)ceilf(fmaxf(e0, e1)));
                    dmx = fmaxf(dmx, sqrtf(dd[m]) * 1.0001f);
                    if (FORM == FORM_SPLIT)
                        cph[m] = (float)kTwoPi * seed_phase(dh, dl, ctl.seed_hi, ctl.seed_lo, B.K_hi,
                                                            B.K_lo, &whi[m], &dwa[m]);
                }
            }
            lb0 = warp_min(lb0);
            lb1 = warp_max(lb1);
            const int dbits = __reduce_max_sync(0xffffffffu, __float_as_int(dmx));
            if (lane == 0 && lb0 <= lb1) {
                atomicMin(&ctl.bmin, lb0);
                atomicMax(&ctl.bmax, lb1);
                atomicMax(&ctl.dmax_bits, dbits);
            }
        }
        __syncthreads();
        ChunkPlan plan;
        plan.init(kmin, kmax, ctl.azs_max, ctl.aze_min, CK);
        const int nchunks = plan.count();
        const bool use_tma = B.tmap >= 0;

        issued = 0;
        if (producer) {
            // ---- producer warp ----
            const int bmin = ctl.bmin - 1, bmax = ctl.bmax + 2;
            const double xcx = ctl.xc[0], xcy = ctl.xc[1], xcz = ctl.xc[2];
            const int azs_max = ctl.azs_max, aze_min = ctl.aze_min;
            const double rmaxb = (B.rmax - B.rngstart) * B.inv_dmrg;
            const double uax = ctl.ua[0], uay = ctl.ua[1], uaz = ctl.ua[2];
            const double dux = ctl.ub[0] - uax, duy = ctl.ub[1] - uay, duz = ctl.ub[2] - uaz;
            const double span = kmax - 1 > kmin ? 1.0 / (double)(kmax - 1 - kmin) : 0.0;
            const double dev_scale = (double)__int_as_float(ctl.dmax_bits) * B.inv_dmrg;
            const double *satl = B.satloc;
            const int Pm1 = B.P - 1;
            // burst constants of the chunk loop held in registers: the loop's
            // barrier waits clobber memory, so fields read from the descriptor
            // inside it would be loaded again on every chunk
            const double rng0 = B.rngstart, idmrg = B.inv_dmrg, Kc = B.K;
            const int tmap_i = B.tmap, bin0 = B.bin0;
            const float idmrg_f = (float)idmrg, kpk_f = (float)(kTwoPi * Kc);
            // upload gate (GATE only), held in registers with the last value seen
            const int *const ready = GATE ? B.ready : nullptr;
            const int ready_base = GATE ? B.ready_base : 0, ready_rows = GATE ? B.ready_rows : 1;
            int ready_seen = INT_MIN;
            // satellite position of this lane's pulse, one chunk ahead
            double nsx, nsy, nsz;
            {
                int k0n, nkn;
                plan.chunk(0, CK, k0n, nkn);
                const double *sp = satl + 3 * min(k0n + lane, Pm1);
                nsx = sp[0];
                nsy = sp[1];
                nsz = sp[2];
            }
            for (int c = 0; c < nchunks; ++c) {
                const uint32_t g = gchunk + c;
                const int s = g % NS;
                const uint32_t r = g / NS;
                int k0, nk;
                plan.chunk(c, CK, k0, nk);
                const int k = min(k0 + lane, Pm1);
                const double sx = nsx, sy = nsy, sz = nsz;
                if (c + 1 < nchunks) {  // prefetch the next chunk's orbit
                    int k0n, nkn;
                    plan.chunk(c + 1, CK, k0n, nkn);
                    const double *sp = satl + 3 * min(k0n + lane, Pm1);
                    nsx = sp[0];
                    nsy = sp[1];
                    nsz = sp[2];
                }
                const double ux = xcx - sx, uy = xcy - sy, uz = xcz - sz;
                const double uu = ux * ux + uy * uy + uz * uz;
                const double rs = rsqrt(uu);
                const double R = uu * rs;
                const double ex = ux * rs, ey = uy * rs, ez = uz * rs;
                const double nx = __shfl_down_sync(0xffffffffu, ex, 1);
                const double ny = __shfl_down_sync(0xffffffffu, ey, 1);
                const double nz = __shfl_down_sync(0xffffffffu, ez, 1);
                const double rbabs = (R - rng0) * idmrg;
                const bool act = lane < nk;
                // deviation of the look vector from the tile's straight line
                const double f = (double)(k - kmin) * span;
                const double gx = ex - (uax + f * dux), gy = ey - (uay + f * duy),
                             gz = ez - (uaz + f * duz);
                const float dev =
                    act ? sqrtf((float)(gx * gx + gy * gy + gz * gz)) * (float)dev_scale * 1.0001f : 0.f;
                const int lo = __reduce_min_sync(0xffffffffu, act ? (int)floor(rbabs) : INT_MAX);
                const int hi = __reduce_max_sync(0xffffffffu, act ? (int)ceil(rbabs) : INT_MIN);
                const int devmax = __reduce_max_sync(0xffffffffu, __float_as_int(dev));
                const int x0 = (lo + bmin) & ~1;  // TMA: x * 8 bytes on a 16-byte boundary
                const int need = hi + bmax - x0 + 1;
                // Everything the stage needs is reduced to floats before the stage
                // wait, so that no FP64 value stays live across it.
                StageHdr hv;
                hv.x0 = x0;
                {
                    const bool interior = k0 >= azs_max && k0 + nk <= aze_min;
                    const bool rangeok = x0 >= 1 && (double)(x0 + WB) <= rmaxb - 1.0;
                    const bool bounded = __int_as_float(devmax) < 0.5f;
                    hv.fast = (rangeok && bounded && need <= WB) ? 1 : 0;
                    hv.interior = interior ? 1 : 0;
                }
                hv.tlo = (float)(-(double)x0);
                hv.thi = __double2float_rn(rmaxb - (double)x0);
                {
                    const double Rmid = __shfl_sync(0xffffffffu, R, nk / 2);
                    hv.dmx = __double2float_rn(__shfl_sync(0xffffffffu, nx - ex, nk / 2));
                    hv.dmy = __double2float_rn(__shfl_sync(0xffffffffu, ny - ey, nk / 2));
                    hv.dmz = __double2float_rn(__shfl_sync(0xffffffffu, nz - ez, nk / 2));
                    const float rm = (float)Rmid, irm = __frcp_rn(rm);
                    hv.inv2R = 0.5f * irm;
                    hv.c2 = hv.inv2R * irm;
                }
                hv.poly = 0;
                hv.r0 = hv.r1 = hv.r2 = hv.p0 = hv.p1 = hv.p2 = 0.f;
                hv.u0x = hv.u0y = hv.u0z = hv.usx = hv.usy = hv.usz = 0.f;
                float4 pa = make_float4(0.f, 0.f, 0.f, 0.f);
                float pb = 0.f;
                if constexpr (FORM == FORM_SPLIT) {
                    {
                        const double q = R * Kc;
                        pa = make_float4(__double2float_rn(nx - ex), __double2float_rn(ny - ey),
                                         __double2float_rn(nz - ez), __double2float_rn(kTwoPi * (q - rint(q))));
                        pb = __double2float_rn(rbabs - (double)x0);
                    }
                    // closed forms: R_c - R_c(0) quadratic through pulses 0, jm, jb
                    // (Newton form, recentred on jc); look-vector increments linear
                    // through 0 and jb; each checked against every pulse of the
                    // chunk.  The offsets from pulse 0 are < ~1 m, so FP32 carries
                    // them to ~1e-7 m, well inside the tolerance.
                    const int jm = (nk - 1) >> 1, jb = nk - 1;
                    const float jc = 0.5f * (float)jb;
                    const double Ra = __shfl_sync(0xffffffffu, R, 0);
                    const float dR = (float)(R - Ra);
                    const float dRm = __shfl_sync(0xffffffffu, dR, jm);
                    const float dRb = __shfl_sync(0xffffffffu, dR, jb);
                    float c0 = 0.f, c1 = 0.f, c2 = 0.f;
                    float u0[3], us[3];
                    const float pq[3] = {pa.x, pa.y, pa.z};
                    if (nk >= 3) {
                        const float D1 = dRm * kRecipSmall[jm];
                        const float D2 = ((dRb - dRm) * kRecipSmall[jb - jm] - D1) * kRecipSmall[jb];
                        c2 = D2;
                        c1 = fmaf(D2, 2.f * jc - (float)jm, D1);
                        c0 = fmaf(jc * (jc - (float)jm), D2, jc * D1);
                    }
                    const float fj = (float)lane - jc;
                    float err = fabsf(dR - fmaf(fmaf(c2, fj, c1), fj, c0));
                    const float ij = nk >= 3 ? kRecipSmall[jb] : 0.f;
                    const float dmaxc = (float)nk * __int_as_float(ctl.dmax_bits);
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        u0[c] = __shfl_sync(0xffffffffu, pq[c], 0);
                        us[c] = (__shfl_sync(0xffffffffu, pq[c], jb) - u0[c]) * ij;
                        // w error accumulated over the chunk: nk * step error * max |d|
                        err = fmaf(fabsf(pq[c] - fmaf((float)lane, us[c], u0[c])), dmaxc, err);
                    }
                    // the fitted R_c at the first pulse (f = -jc), its first and
                    // second forward differences.  Only R_c itself needs FP64 (its
                    // phase); the differences (|dR| < ~0.1 m per pulse) and the
                    // fit's offset from Ra (< ~2 m) are FP32 quantities already,
                    // and FP64 steps on them would only lengthen the producer's
                    // path, which the consumers wait on (measured 1.9 %).
                    const double cR = Ra + (double)fmaf(fmaf(c2, jc, -c1), jc, c0);
                    const float fD1 = fmaf(c2, 1.f - 2.f * jc, c1), fD2 = 2.f * c2;
                    const double q = cR * Kc;
                    hv.r0 = __double2float_rn((cR - rng0) * idmrg - (double)x0);
                    hv.r1 = fD1 * idmrg_f;
                    hv.r2 = fD2 * idmrg_f;
                    hv.p0 = __double2float_rn(kTwoPi * (q - rint(q)));
                    hv.p1 = fD1 * kpk_f;
                    hv.p2 = fD2 * kpk_f;
                    hv.u0x = u0[0];
                    hv.u0y = u0[1];
                    hv.u0z = u0[2];
                    hv.usx = us[0];
                    hv.usy = us[1];
                    hv.usz = us[2];
                    const float resmax =
                        __int_as_float(__reduce_max_sync(0xffffffffu, __float_as_int(act ? err : 0.f)));
                    hv.poly = (nk >= 3 && (double)resmax * kTwoPi * Kc < kPolyTolRad) ? 1 : 0;
                }
                if (!mbar_wait_bounded(&ctl.empty[s], (r & 1) ^ 1, ctl.spin)) {
                    ctl.abort = 1;
                    break;
                }
                // Range lines still in transfer: wait (bounded) until the rows
                // of this chunk are in device memory.
                if (GATE && ready) {
                    const int target = ready_base + (min(k0 + CK, Pm1 + 1) + ready_rows - 1) / ready_rows;
                    if (ready_seen < target) {
                        if (!wait_word_at_least(ready, target, ctl.spin)) {
                            if (lane == 0) atomicOr(err, ERR_UPLOAD_TIMEOUT);
                            ctl.abort = 1;
                            break;
                        }
                        // the rows were seen through a generic-proxy acquire;
                        // order the TMA (async-proxy) reads of them after it
                        if (lane == 0) fence_proxy_async_global();
                        ready_seen = target;
                    }
                }
                // The copy first: the stage's header and pulse parameters are
                // written while it is in flight.  expect_tx arms the byte count
                // without arriving; the phase still needs all 32 lane arrivals
                // below, which follow those writes.
                if (lane == 0 && use_tma) {
                    if (c == 0) fence_tensormap_acquire(tmaps + tmap_i);
                    fence_proxy_async_shared();
                    mbar_expect_tx(&ctl.full[s], (uint32_t)(WB * CK * 8));
                    tma_load_2d(samp0 + (size_t)s * CK * WB, tmaps + tmap_i, &ctl.full[s],
                                x0 - bin0, k0);
                    issued |= 1u << s;
                    issued_par = (issued_par & ~(1u << s)) | ((r & 1u) << s);
                }
                if constexpr (FORM == FORM_FP64) {
                    if (lane < CK) {
                        double *q = prm[s * CK + lane].s;
                        q[0] = sx;
                        q[1] = sy;
                        q[2] = sz;
                    }
                }
                if constexpr (FORM == FORM_SPLIT) {
                    if (lane < CK) {
                        PP &p = prm[s * CK + lane];
                        p.a = pa;
                        p.b = make_float4(pb, 0.f, 0.f, 0.f);
                    }
                }
                if (lane == 0) hdr[s] = hv;
                if (!use_tma) {
                    // no TMA descriptor for this burst: stage the window with plain loads
                    float2 *w = samp0 + (size_t)s * CK * WB;
                    for (int idx = lane; idx < CK * WB; idx += 32) {
                        const int j = idx / WB;
                        w[idx] = ld_sample(B, k0 + j, x0 + (idx - j * WB));
                    }
                }
                __syncwarp();
                mbar_arrive(&ctl.full[s]);
            }
            if (lane == 0) ctl.item = atomicAdd(work_counter, 1);
        } else {
            // ---- consumer warps ----
            // burst constants in registers (the loop's waits clobber memory)
            const float invd_c = B.inv_dmrg_f, Kr_c = (float)(kTwoPi * B.K);
            const double rng0_c = B.rngstart, rmax_c = B.rmax, dmrg_c = B.dmrg, k4pi_c = B.k4pi;
            for (int c = 0; c < nchunks; ++c) {
                const uint32_t g = gchunk + c;
                const int s = g % NS;
                const uint32_t r = g / NS;
                if (!mbar_wait_bounded(&ctl.full[s], r & 1, ctl.spin)) {
                    ctl.abort = 1;
                    break;
                }
                const StageHdr h = hdr[s];
                int k0, nk;
                plan.chunk(c, CK, k0, nk);
                const float2 *win = samp0 + (size_t)s * CK * WB;
                const PP *pp = prm + s * CK;
                if constexpr (FORM == FORM_SPLIT) {
                    const float invd = invd_c;
                    const float Kr = Kr_c;
                  if (h.fast && h.poly) {
                    // Closed forms.  Within the chunk the pixel's range offset from
                    // R_c advances by dw_j = d.(u0 + j us) + g (g: slope of the folded
                    // second-order term), so uacc_j = dwa + dr2_0 + sum_{i<j} dw_i is
                    // a quadratic in j: uacc_0 = dwa + dr2_0, first difference
                    // d.u0 + g, second difference d.us.  With R_c's quadratic (from the
                    // producer, in the same form) the bin and the phase are advanced per
                    // term by forward differences from the chunk's first pulse.
                    const float jc = 0.5f * (float)(nk - 1);
                    const float jmid = (float)(nk >> 1);
                    float T0[M], T1[M], T2[M], P0[M], P1[M], P2[M];
#pragma unroll
                    for (int m = 0; m < M; ++m) {
                        const float w0 = whi[m] + dwa[m];
                        const float n0 = fmaf(-w0, w0, dd[m]);
                        const float q0 = fmaf(-w0, h.c2, h.inv2R);
                        const float dr0 = n0 * q0;
                        const float a1 = fmaf(d[m][0], h.u0x, fmaf(d[m][1], h.u0y, d[m][2] * h.u0z));
                        const float bq = fmaf(d[m][0], h.usx, fmaf(d[m][1], h.usy, d[m][2] * h.usz));
                        const float g = fmaf(-2.f * w0, q0, -n0 * h.c2) * fmaf(bq, jmid, a1);
                        const float A = a1 + g;
                        T0[m] = fmaf(whi[m] + (dwa[m] + dr0), invd, h.r0);
                        T1[m] = fmaf(A, invd, h.r1);
                        T2[m] = fmaf(bq, invd, h.r2);
                        const float p0 = fmaf(Kr, dr0, cph[m] + h.p0);
                        const float nr = rintf(p0 * kInvTwoPi);
                        P0[m] = fmaf(-nr, kTwoPiLo, fmaf(-nr, kTwoPiHi, p0));
                        P1[m] = fmaf(Kr, A, h.p1);
                        P2[m] = fmaf(Kr, bq, h.p2);
                        // state at the next chunk: sum of d.(u0 + j us) over the chunk
                        const float S = (float)nk * fmaf(bq, jc, a1);
                        dwa[m] += S;
                        cph[m] = fmaf(Kr, S, cph[m]);
                    }
                    // edge chunks add the exact azimuth-window test of every term;
                    // the differences and the floor run on pixel pairs (f32x2)
                    static_assert(M % 2 == 0, "pixel pairs");
                    auto terms = [&](auto masked) {
                        constexpr bool MASKED = decltype(masked)::value;
                        int ja[M], nj[M];
#pragma unroll
                        for (int m = 0; m < M; ++m) {
                            ja[m] = max(azs[m] - k0, 0);
                            nj[m] = max(min(aze[m] - k0, nk) - ja[m], 0);
                        }
                        // bin (tt) and phase (pv) at the current pulse, their first (dt,
                        // dp) and second (ddt, ddp) differences, per pixel pair
                        uint64_t tt[M / 2], dt[M / 2], ddt[M / 2], pv[M / 2], dp[M / 2], ddp[M / 2];
#pragma unroll
                        for (int e = 0; e < M / 2; ++e) {
                            tt[e] = f2_pack(T0[2 * e], T0[2 * e + 1]);
                            dt[e] = f2_pack(T1[2 * e], T1[2 * e + 1]);
                            ddt[e] = f2_pack(T2[2 * e], T2[2 * e + 1]);
                            pv[e] = f2_pack(P0[2 * e], P0[2 * e + 1]);
                            dp[e] = f2_pack(P1[2 * e], P1[2 * e + 1]);
                            ddp[e] = f2_pack(P2[2 * e], P2[2 * e + 1]);
                        }
                        const uint64_t mag = f2_pack(kFloorMagic, kFloorMagic);
                        // pair accumulators: sum vr cs, sum vi sn, sum (vr sn + vi cs)
                        uint64_t aR[M / 2], aM[M / 2], aI[M / 2];
#pragma unroll
                        for (int e = 0; e < M / 2; ++e) aR[e] = aM[e] = aI[e] = 0ull;
// unroll 5 measured best of 2..8 (31 = 6 x 5 + 1)
#pragma unroll 5
                        for (int j = 0; j < nk; ++j) {
                            const float2 *row = win + j * WB;
#pragma unroll
                            for (int e = 0; e < M / 2; ++e) {
                                const uint64_t t = tt[e];
                                const uint64_t ph = pv[e];
                                tt[e] = f2_add(tt[e], dt[e]);
                                dt[e] = f2_add(dt[e], ddt[e]);
                                pv[e] = f2_add(pv[e], dp[e]);
                                dp[e] = f2_add(dp[e], ddp[e]);
                                const uint64_t tm = f2_add_rm(t, mag);
                                const uint64_t fr = f2_sub(t, f2_sub(tm, mag));
                                float tmv[2], frv[2], phv[2];
                                f2_unpack(tm, tmv[0], tmv[1]);
                                f2_unpack(fr, frv[0], frv[1]);
                                f2_unpack(ph, phv[0], phv[1]);
                                float vr[2], vi[2], sn[2], cs[2];
#pragma unroll
                                for (int h2 = 0; h2 < 2; ++h2) {
                                    const int m = 2 * e + h2;
                                    // proven in the window by the producer; bounded for memory safety
                                    const unsigned ic = tap_index<WB>(tmv[h2]);
                                    const float2 s0 = row[ic], s1 = row[ic + 1];
                                    vr[h2] = fmaf(frv[h2], s1.x - s0.x, s0.x);
                                    vi[h2] = fmaf(frv[h2], s1.y - s0.y, s0.y);
                                    if constexpr (MASKED) {
                                        const bool ok = (unsigned)(j - ja[m]) < (unsigned)nj[m];
                                        vr[h2] = ok ? vr[h2] : 0.f;
                                        vi[h2] = ok ? vi[h2] : 0.f;
                                    }
                                    __sincosf(phv[h2], &sn[h2], &cs[h2]);
                                }
                                const uint64_t VR = f2_pack(vr[0], vr[1]), VI = f2_pack(vi[0], vi[1]);
                                const uint64_t SN = f2_pack(sn[0], sn[1]), CS = f2_pack(cs[0], cs[1]);
                                aR[e] = f2_fma(VR, CS, aR[e]);
                                aM[e] = f2_fma(VI, SN, aM[e]);
                                aI[e] = f2_fma(VI, CS, f2_fma(VR, SN, aI[e]));
                            }
                        }
#pragma unroll
                        for (int e = 0; e < M / 2; ++e) {
                            float r0, r1, m0, m1, i0, i1;
                            f2_unpack(aR[e], r0, r1);
                            f2_unpack(aM[e], m0, m1);
                            f2_unpack(aI[e], i0, i1);
                            accr[2 * e] += r0 - m0;
                            accr[2 * e + 1] += r1 - m1;
                            acci[2 * e] += i0;
                            acci[2 * e + 1] += i1;
                        }
                    };
                    if (h.interior) terms(std::false_type{});
                    else terms(std::true_type{});
                  } else {
                    // per pixel and chunk: second-order term and its slope, folded
                    // into the accumulators (uacc = dwa + dr2, cphp = cph + Kr dr2)
                    float uacc[M], cphp[M], gsl[M], dr0[M];
#pragma unroll
                    for (int m = 0; m < M; ++m) {
                        const float w0 = whi[m] + dwa[m];
                        const float n0 = fmaf(-w0, w0, dd[m]);
                        const float q0 = fmaf(-w0, h.c2, h.inv2R);
                        dr0[m] = n0 * q0;
                        const float dwm = fmaf(d[m][0], h.dmx, fmaf(d[m][1], h.dmy, d[m][2] * h.dmz));
                        gsl[m] = fmaf(-2.f * w0, q0, -n0 * h.c2) * dwm;
                        uacc[m] = dwa[m] + dr0[m];
                        cphp[m] = fmaf(dr0[m], Kr, cph[m]);
                    }
                    if (h.fast && h.interior) {
                        // consecutive pulses share only the two accumulators, so
                        // unrolling gives the scheduler independent terms
#pragma unroll 2
                        for (int j = 0; j < nk; ++j) {
                            const float4 pa = pp[j].a;
                            const float rb = pp[j].b.x;
                            const float2 *row = win + j * WB;
#pragma unroll
                            for (int m = 0; m < M; ++m) {
                                const float dwp = fmaf(d[m][0], pa.x, fmaf(d[m][1], pa.y, fmaf(d[m][2], pa.z, gsl[m])));
                                const float t = fmaf(whi[m] + uacc[m], invd, rb);
                                const float ph = cphp[m] + pa.w;
                                uacc[m] += dwp;
                                cphp[m] = fmaf(dwp, Kr, cphp[m]);
                                const float tm = __fadd_rd(t, kFloorMagic);
                                const float fr = t - (tm - kFloorMagic);
                                // proven in range by the producer; clamped for memory safety
                                const unsigned ic = tap_index<WB>(tm);
                                const float2 s0 = row[ic], s1 = row[ic + 1];
                                const float vr = fmaf(fr, s1.x - s0.x, s0.x);
                                const float vi = fmaf(fr, s1.y - s0.y, s0.y);
                                float sn, cs;
                                __sincosf(ph, &sn, &cs);
                                accr[m] = fmaf(vr, cs, fmaf(-vi, sn, accr[m]));
                                acci[m] = fmaf(vr, sn, fmaf(vi, cs, acci[m]));
                            }
                        }
                    } else {
                        // general path: exact aperture and range tests, taps from
                        // global memory when outside the staged window
                        for (int j = 0; j < nk; ++j) {
                            const int k = k0 + j;
                            const float4 pa = pp[j].a;
                            const float rb = pp[j].b.x;
                            const float2 *row = win + j * WB;
#pragma unroll
                            for (int m = 0; m < M; ++m) {
                                const float dwp = fmaf(d[m][0], pa.x, fmaf(d[m][1], pa.y, fmaf(d[m][2], pa.z, gsl[m])));
                                const float t = fmaf(whi[m] + uacc[m], invd, rb);
                                const float ph = cphp[m] + pa.w;
                                uacc[m] += dwp;
                                cphp[m] = fmaf(dwp, Kr, cphp[m]);
                                const float fl = floorf(t);
                                const int i = (int)fl;
                                const float fr = t - fl;
                                const bool ok = (k >= azs[m]) & (k < aze[m]) & (t >= h.tlo) & (t <= h.thi);
                                const bool inwin = (unsigned)i < (unsigned)(WB - 1);
                                const int is = inwin ? i : 0;
                                float2 s0 = row[is], s1 = row[is + 1];
                                if (ok && !inwin) {
                                    s0 = ld_sample(B, k, i + h.x0);
                                    s1 = ld_sample(B, k, i + h.x0 + 1);
                                }
                                float vr = fmaf(fr, s1.x - s0.x, s0.x);
                                float vi = fmaf(fr, s1.y - s0.y, s0.y);
                                vr = ok ? vr : 0.f;
                                vi = ok ? vi : 0.f;
                                float sn, cs;
                                __sincosf(ph, &sn, &cs);
                                accr[m] = fmaf(vr, cs, fmaf(-vi, sn, accr[m]));
                                acci[m] = fmaf(vr, sn, fmaf(vi, cs, acci[m]));
                            }
                        }
                    }
                    // back to the plain accumulators: remove the folded dr2 terms
#pragma unroll
                    for (int m = 0; m < M; ++m) {
                        const float lin = fmaf((float)nk, gsl[m], dr0[m]);
                        dwa[m] = uacc[m] - lin;
                        cph[m] = fmaf(-lin, Kr, cphp[m]);
                    }
                  }
                    // keep the carried phase in [-pi, pi]
#pragma unroll
                    for (int m = 0; m < M; ++m) {
                        const float nr = rintf(cph[m] * kInvTwoPi);
                        cph[m] = fmaf(-nr, kTwoPiLo, fmaf(-nr, kTwoPiHi, cph[m]));
                    }
                } else {
                    const double rs = rng0_c, rmx = rmax_c, dm = dmrg_c, k4 = k4pi_c;
                    const int x0 = h.x0;
                    const bool fast = h.fast && h.interior;
                    for (int j = 0; j < nk; ++j) {
                        const int k = k0 + j;
                        const double sx = pp[j].s[0], sy = pp[j].s[1], sz = pp[j].s[2];
                        const float2 *row = win + j * WB;
#pragma unroll
                        for (int m = 0; m < M; ++m) {
                            if (!fast && (k < azs[m] || k >= aze[m])) continue;
                            const double vx = dsub(X[m][0], sx), vy = dsub(X[m][1], sy),
                                         vz = dsub(X[m][2], sz);
                            const double R = __dsqrt_rn(dadd(dadd(dmul(vx, vx), dmul(vy, vy)), dmul(vz, vz)));
                            const bool inr = R >= rs && R <= rmx;
                            if (!fast && !inr) continue;
                            const double rr = ddiv(dsub(R, rs), dm);
                            const double fl = floor(rr);
                            const int ig = (int)fl;
                            const double fr = dsub(rr, fl);
                            const float w0 = __double2float_rn(dsub(1.0, fr));
                            const float w1 = __double2float_rn(fr);
                            const int i = ig - x0;
                            float2 s0, s1;
                            if ((unsigned)i < (unsigned)(WB - 1)) {
                                s0 = row[i];
                                s1 = row[i + 1];
                            } else {
                                // outside the staged window (the window estimate missed):
                                // the fast path skipped the range test, apply it here
                                if (!inr) continue;
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
                __syncwarp();
                if (lane == 0) mbar_arrive(&ctl.empty[s]);
            }
            // ---- epilogue ----
            if (!ctl.abort) {
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    const int bi = warp + NC * m;
                    const int x = PBX * (bi % BX) + lane % PBX, y = PBY * (bi / BX) + lane / PBX;
                    const int px = px0 + x,
                              line = ly0 + y + tile_dline(B.shear, x) - tile_dmax(B.shear, TX);
                    if (px <= B.lastpix_eff && line >= 0 && line < B.nlines) {
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
                if (GATE && B.rb_done) __threadfence();
            }
        }
        gchunk += nchunks;
        __syncthreads();
        if (ctl.abort) {
            if (tid == 0) atomicOr(err, ERR_TMA_TIMEOUT);
            // let the copies this CTA issued drain before it leaves (bounded by
            // the default limit whatever the launch's: a copy in flight ends in us)
            if (producer && lane == 0) {
                for (int s = 0; s < NS; ++s)
                    if (issued & (1u << s)) mbar_wait_bounded(&ctl.full[s], (issued_par >> s) & 1u);
            }
            return;
        }
        tile_stored(B, ly0);
    }
}

}  // namespace srg
