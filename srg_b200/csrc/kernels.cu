// kernels.cu -- auxiliary device kernels and the compiled shapes of the
// tiled backprojection.
#include <cstring>

#include "bp_kernel.cuh"
#include "bp_ws.cuh"
#include "kernels.h"

namespace srg {

// ---------------------------------------------------------------------------
// Per-line azimuth-centre parabola (sentinel/azimuth_compress.cu:438-481).
// The reference runs this loop serially on the host; the arithmetic here is
// the same operation for operation.  Lines firstline .. lastline-1 get a
// parabola; the last line keeps zeros (the reference leaves it unset), so it
// is never formed.  The three samples of a line (first, middle and last pixel:
// a Newton zero-Doppler solve each) run on three lanes of a warp, ten lines
// per warp, and lane 3i writes line i's coefficients.
__device__ int centre_sample(const BurstDev &B, const Orbit &o, const CentreParams &cp, int line,
                             int s) {
    const int half = (B.lastpix - B.firstpix) / 2 - 1;
    const int pix = B.firstpix + s * half;
    double g[3] = {0.0, 0.0, 0.0};
    if (pix >= B.firstpix && pix <= B.lastpix && pix >= 0 && pix < B.W) {
        const double h = (double)B.dem[(long long)line * B.dem_ld + pix];
        pixel_ecef(B, line, pix, h, g[0], g[1], g[2]);
    }
    const double rngpix = zero_doppler_range(o, g, cp.tmid, cp.xm, cp.vm);
    double u0 = dsub(g[0], cp.xm[0]), u1 = dsub(g[1], cp.xm[1]), u2 = dsub(g[2], cp.xm[2]);
    const double umag = __dsqrt_rn(dadd(dadd(dmul(u0, u0), dmul(u1, u1)), dmul(u2, u2)));
    u0 = ddiv(u0, umag);
    u1 = ddiv(u1, umag);
    u2 = ddiv(u2, umag);
    const double udotv = dadd(dadd(dmul(cp.vm[0], u0), dmul(cp.vm[1], u1)), dmul(cp.vm[2], u2));
    const double fd = dmul(ddiv(2.0, cp.wvl), udotv);
    const double veff = __dsqrt_rn(
        dadd(dadd(dmul(cp.vm[0], cp.vm[0]), dmul(cp.vm[1], cp.vm[1])), dmul(cp.vm[2], cp.vm[2])));
    const double num = dsub(dmul(ddiv(ddiv(ddiv(dmul(rngpix, cp.wvl), 2.0), veff), veff), fd),
                            ddiv(ddiv(dmul(dmul(rngpix, cp.angc0), cp.pi), 180.0), veff));
    const double den = dadd(1.0, ddiv(ddiv(dmul(dmul(rngpix, cp.angc1), cp.pi), 180.0), veff));
    const double td = ddiv(num, den);
    return (int)dadd(dmul(td, cp.prf), (double)(B.P / 2));
}

// Lanes 3i, 3i+1, 3i+2 hold samples 0, 1, 2 of one line; lane 3i stores.
__device__ __forceinline__ void store_coef(int lane, int y, bool last, double *cl) {
    const int y1 = __shfl_down_sync(0xffffffffu, y, 1);
    const int y2 = __shfl_down_sync(0xffffffffu, y, 2);
    if (cl && lane % 3 == 0) {
        if (last) {
            cl[0] = cl[1] = cl[2] = 0.0;
        } else {
            cl[0] = dmul(0.5, dsub((double)(y + y2), dmul(2.0, (double)y1)));
            cl[1] = dmul(0.5, (double)(y2 - y));
            cl[2] = (double)y1;
        }
    }
}

__global__ void line_centres_kernel(BurstDev B, Orbit o, CentreParams cp, double *coef) {
    const int lane = threadIdx.x & 31;
    const int line = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 10 + lane / 3;
    const bool mine = lane < 30 && line < B.nlines;
    const bool last = line == B.nlines - 1;
    int y = 0;
    if (mine && !last) y = centre_sample(B, o, cp, line, lane % 3);
    store_coef(lane, y, last, mine ? coef + 3 * line : nullptr);
}

// Batched per-line azimuth centres over all bursts of a scene (the same
// arithmetic as line_centres_kernel; lines numbered across the bursts).
__global__ void line_centres_batch_kernel(const BurstDev *__restrict__ bursts,
                                          const CentreJob *__restrict__ jobs, int n, int total) {
    const int lane = threadIdx.x & 31;
    const int gid = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 10 + lane / 3;
    const bool mine = lane < 30 && gid < total;
    int b = 0;
    if (mine)
        while (b + 1 < n && jobs[b + 1].line_base <= gid) ++b;
    const CentreJob &J = jobs[b];
    const BurstDev &B = bursts[b];
    const int line = gid - J.line_base;
    const bool last = line == B.nlines - 1;
    int y = 0;
    if (mine && !last) y = centre_sample(B, J.orbit, J.cp, line, lane % 3);
    store_coef(lane, y, last, mine ? J.coef + 3 * line : nullptr);
}

// ---------------------------------------------------------------------------
// Exact executed-term count with the reference's FP64 predicate
// (azimuth_compress.cu:54-64), one thread per pixel.
__global__ void count_terms_kernel(BurstDev B, unsigned long long *terms) {
    const int nx = B.lastpix_eff - B.firstpix + 1;
    const long long npix = (long long)nx * B.nlines;
    unsigned long long cnt = 0;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < npix;
         idx += (long long)gridDim.x * blockDim.x) {
        const int line = (int)(idx / nx);
        const int px = B.firstpix + (int)(idx - (long long)line * nx);
        double X[3];
        const double h = (double)B.dem[(long long)line * B.dem_ld + px];
        pixel_ecef(B, line, px, h, X[0], X[1], X[2]);
        int azs, aze;
        pixel_window(B, pixel_azoff(B, B.coef + 3 * line, px), azs, aze);
        for (int k = azs; k < aze; ++k) {
            const double *s = B.satloc + 3 * k;
            const double vx = dsub(X[0], s[0]), vy = dsub(X[1], s[1]), vz = dsub(X[2], s[2]);
            const double R = __dsqrt_rn(dadd(dadd(dmul(vx, vx), dmul(vy, vy)), dmul(vz, vz)));
            cnt += (R >= B.rngstart && R <= B.rmax) ? 1 : 0;
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(terms, cnt);
}

// ---------------------------------------------------------------------------
// Range bins a burst's sum can read.  For every formed pixel of the box the
// terms run over its aperture window [azs, aze) (azimuth_compress.cu:54-58)
// and read bins floor((R_k - rngstart) / dmrg) and the next one (:65-69).
// Where R_k^2 is convex in the pulse index k (the host checks the pulses for
// it) R_k is largest at an end of the window and smallest where the forward
// difference of R_k^2 turns non-negative, found by bisection; the pixel's
// bins lie between those of its smallest and largest range (+1 for the
// second tap).  band[0] / band[1] are lowered / raised to the extremes over
// all formed pixels (preset to INT_MAX / INT_MIN by the caller).  A block
// takes a patch of kBandLines x kBandCols pixels and evaluates the latitude
// and longitude sines and cosines once per line and column of it.
constexpr int kBandLines = 8, kBandCols = 64;
__global__ void __launch_bounds__(256) range_band_kernel(BurstDev B, int *band) {
    __shared__ double lt[kBandLines][4], ct[kBandCols][2];
    const int nx = B.lastpix_eff - B.firstpix + 1;
    const int l0 = blockIdx.y * kBandLines, c0 = blockIdx.x * kBandCols;
    const int t = threadIdx.x;
    if (t < kBandLines) {
        if (l0 + t < B.nlines) {
            const LineTrig L = line_trig(B, l0 + t);
            lt[t][0] = L.slat;
            lt[t][1] = L.clat;
            lt[t][2] = L.re;
            lt[t][3] = L.rez;
        }
    } else if (t < kBandLines + kBandCols) {
        const int c = t - kBandLines;
        if (c0 + c < nx) col_trig(B, B.firstpix + c0 + c, ct[c][0], ct[c][1]);
    }
    __syncthreads();
    int lo = INT_MAX, hi = INT_MIN;
    for (int q = t; q < kBandLines * kBandCols; q += blockDim.x) {
        const int yl = q / kBandCols, xc = q - yl * kBandCols;
        const int line = l0 + yl, col = c0 + xc;
        if (line >= B.nlines || col >= nx) continue;
        const int px = B.firstpix + col;
        int azs, aze;
        pixel_window(B, pixel_azoff(B, B.coef + 3 * line, px), azs, aze);
        if (aze <= azs) continue;
        double X[3];
        pixel_ecef_from(lt[yl][0], lt[yl][1], lt[yl][2], lt[yl][3], ct[xc][0], ct[xc][1],
                        (double)B.dem[(long long)line * B.dem_ld + px], X[0], X[1], X[2]);
        auto r2 = [&](int k) {
            const double *s = B.satloc + 3 * k;
            const double vx = X[0] - s[0], vy = X[1] - s[1], vz = X[2] - s[2];
            return vx * vx + vy * vy + vz * vz;
        };
        int a = azs, b = aze - 1;
        while (a < b) {
            const int m = (a + b) >> 1;
            if (r2(m + 1) < r2(m)) a = m + 1;
            else b = m;
        }
        const double rmin = sqrt(r2(a)), rmax = sqrt(fmax(r2(azs), r2(aze - 1)));
        const double blo = fmin(fmax(floor((rmin - B.rngstart) * B.inv_dmrg), -1e9), 1e9);
        const double bhi = fmin(fmax(floor((rmax - B.rngstart) * B.inv_dmrg) + 1.0, -1e9), 1e9);
        lo = min(lo, (int)blo);
        hi = max(hi, (int)bhi);
    }
    lo = warp_min(lo);
    hi = warp_max(hi);
    if ((threadIdx.x & 31) == 0 && lo <= hi) {
        atomicMin(band, lo);
        atomicMax(band + 1, hi);
    }
}

// ---------------------------------------------------------------------------
// Ordered merge (azimuth_compress.cu:527-531): replace where |Re(src)| > 1e-18.
__global__ void merge_kernel(float2 *dst, long long dst_ld, const float2 *src, long long src_ld,
                             int rows, int cols) {
    const long long n = (long long)rows * cols;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / cols);
        const int c = (int)(i - (long long)r * cols);
        const float2 v = src[(long long)r * src_ld + c];
        if (fabs((double)v.x) > 1.e-18) dst[(long long)r * dst_ld + c] = v;
    }
}

// Ordered merge of every burst of a scene into the scene raster: for each
// scene pixel the last burst (in order) whose output there has
// |Re| > 1e-18 wins, which is what merging the bursts one after the other
// with the reference's rule gives.  Each CTA covers a 32 x 32 patch (four
// rows per thread) and first collects (ballot) the bursts whose output window
// meets it.  With the work-list mask of the backprojection that wrote the
// outputs (tiles of 2^tx_log2 x 2^ty_log2 pixels), a burst whose tile at the
// pixel has no formed pixel is passed over without reading its output (that
// output is zero, which the rule never takes).
__global__ void __launch_bounds__(256) merge_scene_kernel(const BurstDev *__restrict__ bursts, int n,
                                                          float2 *dst, long long dst_ld, int lines,
                                                          int cols,
                                                          const unsigned char *__restrict__ tmask,
                                                          int tx_log2, int ty_log2) {
    const int c0 = blockIdx.x * 32, l0 = blockIdx.y * 32;
    __shared__ unsigned mask[8];  // up to 256 bursts
    const int nw = (n + 31) / 32;
    if (threadIdx.y == 0) {
        for (int w = 0; w < nw; ++w) {
            const int b = w * 32 + threadIdx.x;
            bool hit = false;
            if (b < n) {
                const BurstDev &B = bursts[b];
                const int gl0 = B.firstline, gl1 = B.firstline + B.nlines - 1;
                hit = !(gl1 < l0 || gl0 > l0 + 31 || B.lastpix_eff < c0 || B.firstpix > c0 + 31);
            }
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            if (threadIdx.x == 0) mask[w] = m;
        }
    }
    __syncthreads();
    const int c = c0 + threadIdx.x;
    if (c >= cols) return;
#pragma unroll 1
    for (int rr = 0; rr < 4; ++rr) {
        const int l = l0 + threadIdx.y + 8 * rr;
        if (l >= lines) break;
        bool done = false;
        for (int w = nw - 1; w >= 0 && !done; --w) {
            unsigned m = mask[w];
            while (m) {
                const int bit = 31 - __clz(m);
                m &= ~(1u << bit);
                const BurstDev &B = bursts[w * 32 + bit];
                const int ll = l - B.firstline;
                if (ll < 0 || ll >= B.nlines || c < B.firstpix || c > B.lastpix_eff) continue;
                if (tmask) {
                    // the tile of (ll, c): its column block, then the tile
                    // row from the line less the column's line offset
                    const int xc = c - B.firstpix, x = xc & ((1 << tx_log2) - 1);
                    const int lr = ll - tile_dline(B.shear, x) + tile_dmax(B.shear, 1 << tx_log2);
                    const int ti = (lr >> ty_log2) * B.tiles_x + (xc >> tx_log2);
                    if (!tmask[B.tile_base + ti]) continue;
                }
                const float2 v = B.out[(long long)ll * B.out_ld + (c - B.out_pix0)];
                if (fabs((double)v.x) > 1.e-18) {
                    dst[(long long)l * dst_ld + c] = v;
                    done = true;
                    break;
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Per-pulse orbit (sentinel/sentineltimingsub.f90:55-66 with
// orbithermite.f), one thread per pulse.  Window start int((t-t1)/dt) - 1
// (1-based) as the reference; clamped to the vector array, where the
// reference would read outside it.
__global__ void pulse_orbit_kernel(const double *times, int P, Orbit o, double *pos, double *vel) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= P) return;
    const double t = times[k];
    int loc = (int)ddiv(dsub(t, o.t[0]), dsub(o.t[1], o.t[0]));
    int s = min(max(loc - 2, 0), o.n - 4);
    hermite4(o.x + 3 * s, o.v + 3 * s, o.t + s, t, pos + 3 * k, vel + 3 * k);
}

// ---------------------------------------------------------------------------
// Synthetic-scene forward projection: every pixel of the burst window with a
// non-zero reflectivity adds a * sinc^2(L sin(psi)/lambda) * exp(-j 4 pi R / lambda)
// to the two range bins around R of every pulse (the adjoint of linear
// interpolation).  FP64 geometry; atomic accumulation.
__global__ void forward_project_kernel(BurstDev B, const float2 *refl, long long refl_ld,
                                       const double *satvel, double antenna,
                                       const float *range_offset) {
    const int nx = B.lastpix_eff - B.firstpix + 1;
    const long long npix = (long long)nx * B.nlines;
    const double pi = 3.141592653589793;
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= npix) return;
    const int line = (int)(idx / nx);
    const int px = B.firstpix + (int)(idx - (long long)line * nx);
    const float2 a = refl[(long long)line * refl_ld + px];
    if (a.x == 0.f && a.y == 0.f) return;
    double X[3];
    pixel_ecef(B, line, px, (double)B.dem[(long long)line * B.dem_ld + px], X[0], X[1], X[2]);
    // extra two-way path of the scatterer (e.g. surface motion along the line of sight)
    const double dR = range_offset ? (double)range_offset[(long long)line * refl_ld + px] : 0.0;
    const double wvl = 2.0 / B.K;
    float2 *out = const_cast<float2 *>(B.burst);
    for (int k = 0; k < B.P; ++k) {
        const double *s = B.satloc + 3 * k;
        const double dx = X[0] - s[0], dy = X[1] - s[1], dz = X[2] - s[2];
        const double R0 = sqrt(dx * dx + dy * dy + dz * dz);
        const double R = R0 + dR;
        const double r = (R - B.rngstart) * B.inv_dmrg;
        if (!(r >= 0.0 && r < (double)(B.S - 1))) continue;
        const double *v = satvel + 3 * k;
        const double vn = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        const double spsi = (dx * v[0] + dy * v[1] + dz * v[2]) / (vn * R0);
        const double arg = pi * antenna * spsi / wvl;
        const double sc = fabs(arg) < 1e-12 ? 1.0 : sin(arg) / arg;
        const double w = sc * sc;
        if (w < 1e-7) continue;
        double sn, cs;
        sincos(B.k4pi * R, &sn, &cs);
        // a * w * exp(-j phase)
        const double vr = w * ((double)a.x * cs + (double)a.y * sn);
        const double vi = w * ((double)a.y * cs - (double)a.x * sn);
        const int i = (int)floor(r);
        const double fr = r - i;
        float2 *row = out + (long long)k * B.ldb;
        atomicAdd(&row[i].x, (float)(vr * (1.0 - fr)));
        atomicAdd(&row[i].y, (float)(vi * (1.0 - fr)));
        atomicAdd(&row[i + 1].x, (float)(vr * fr));
        atomicAdd(&row[i + 1].y, (float)(vi * fr));
    }
}

// ---------------------------------------------------------------------------
// Calibration: FMA issue-rate peak.  Every thread runs 8 independent FMA
// chains (enough to cover the pipeline latency at full occupancy); the
// result is written so the work cannot be elided.
// ---------------------------------------------------------------------------
// Work list of the backprojection: the tiles that can hold a formed pixel.
// A pixel is formed only where its line's azimuth-centre parabola lies inside
// (ap2, P - ap2) (pixel_azoff, azimuth_compress.cu:169-175); a burst's grid
// limits span more lines than its pulses see, and on the IW scene 72 % of the
// tiles have no formed pixel.  Without the list every persistent CTA claims
// those tiles too and runs their prologue only to write zeros.
//
// The mask is conservative: a tile is dropped only when, on every one of its
// lines, the parabola over the tile's columns stays outside the interval by
// 1e-3 pulse (its extremes over [arg(first column), arg(last column)] are at
// the ends or the vertex; the column arguments are the same rounded quotients
// pixel_azoff forms, monotonic in the column).  A dropped tile's pixels get
// the zeros the backprojection writes for unformed pixels.  One warp per tile.
__device__ __forceinline__ double azoff_fit(const double *c, double arg) {
    return dadd(dadd(dmul(dmul(c[0], arg), arg), dmul(c[1], arg)), c[2]);
}

// floor(a / b) and ceil(a / b) for b > 0 (integer division truncates)
__device__ __forceinline__ int floor_div(int a, int b) { return a >= 0 ? a / b : -((b - 1 - a) / b); }
__device__ __forceinline__ int ceil_div(int a, int b) { return -floor_div(-a, b); }

__global__ void __launch_bounds__(256) tile_mask_kernel(const BurstDev *__restrict__ bursts, int tx,
                                                        int ty, unsigned char *__restrict__ mask,
                                                        int *__restrict__ seg_count,
                                                        int *__restrict__ band) {
    const BurstDev &B = bursts[blockIdx.y];
    const int lane = threadIdx.x & 31;
    const int ti = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (ti >= B.tiles_x * B.tiles_y) return;
    const int col0 = B.firstpix + (ti % B.tiles_x) * tx;
    const int ly0 = (ti / B.tiles_x) * ty;
    const int dmax = tile_dmax(B.shear, tx), span = tile_span(B.shear, tx);
    // lane j < ty + span: the tile's columns [px0, px1] on line ly0 - span + j,
    // clipped to the burst's: the x in [0, tx) whose line offset
    // d(x) = floor(shear x / 32) puts the line among the tile's rows,
    // lo <= d(x) <= hi (one interval: d is monotone in x)
    const int line = ly0 - span + lane;
    const int lo = line - ly0 + dmax - ty + 1, hi = line - ly0 + dmax, sh = B.shear;
    int xa, xb;
    if (sh == 0) {
        xa = lo <= 0 && hi >= 0 ? 0 : tx;
        xb = tx - 1;
    } else if (sh > 0) {  // 32 lo <= sh x < 32 (hi + 1)
        xa = ceil_div(32 * lo, sh);
        xb = ceil_div(32 * (hi + 1), sh) - 1;
    } else {              // 32 lo <= sh x < 32 (hi + 1), sh < 0
        xa = floor_div(-32 * (hi + 1), -sh) + 1;
        xb = floor_div(-32 * lo, -sh);
    }
    xa = max(xa, 0);
    xb = min(xb, tx - 1);
    const int px0 = col0 + xa, px1 = min(col0 + xb, B.lastpix_eff);
    bool keep = false;
    if (lane < ty + span && line >= 0 && line < B.nlines && px0 <= px1) {
        const double *c = B.coef + 3 * line;
        const float den = (float)(B.lastpix - B.firstpix);
        const double a0 = dsub(dmul((double)__fdiv_rn((float)(px0 - B.firstpix), den), 2.0), 1.0);
        const double a1 = dsub(dmul((double)__fdiv_rn((float)(px1 - B.firstpix), den), 2.0), 1.0);
        const double f0 = azoff_fit(c, a0), f1 = azoff_fit(c, a1);
        double lo = fmin(f0, f1), hi = fmax(f0, f1);
        if (c[0] != 0.0) {
            const double v = -c[1] / (2.0 * c[0]);
            if (v > a0 && v < a1) {
                const double fv = azoff_fit(c, v);
                lo = fmin(lo, fv);
                hi = fmax(hi, fv);
            }
        }
        const bool finite = isfinite(f0) && isfinite(f1) && isfinite(lo) && isfinite(hi);
        keep = !finite || !(hi < (double)B.ap2 - 1e-3 || lo > (double)(B.P - B.ap2) + 1e-3);
    }
    keep = __any_sync(0xffffffffu, keep);
    if (B.rb_order && ti == 0 && lane == 0) *B.rb_order = lines_against_pulses(B) ? 1 : 0;
    if (!keep && lane < tx && col0 + lane <= B.lastpix_eff) {
        const int l0 = ly0 + tile_dline(B.shear, lane) - dmax;
        for (int y = max(0, -l0); y < ty && l0 + y < B.nlines; ++y)
            B.out[(long long)(l0 + y) * B.out_ld + (col0 + lane - B.out_pix0)] = make_float2(0.f, 0.f);
    }
    if (lane == 0) {
        const int t = B.tile_base + ti;
        mask[t] = keep ? 1 : 0;
        if (keep) {
            atomicAdd(seg_count + (t >> kTileSegShift), 1);
            if (band) {
                atomicMin(band, max(ly0 - span, 0));
                atomicMax(band + 1, min(ly0 + ty - 1, B.nlines - 1));
            }
            if (B.rb_expect) atomicAdd(B.rb_expect + (ti / B.tiles_x) / B.rb_tile_rows, 1);
        }
    }
}

// Ordered compaction of the mask: block s writes the kept tiles of segment s
// (kTileSeg tiles, 16 per thread) after those of the segments before it.
// list[0] = number of kept tiles, list[1..] = their indices, ascending.
__global__ void __launch_bounds__(256) tile_compact_kernel(const unsigned char *__restrict__ mask,
                                                           const int *__restrict__ seg_count,
                                                           int total, int *__restrict__ list) {
    static_assert(kTileSeg == 256 * 16, "16 tiles per thread");
    __shared__ int wsum[8];
    __shared__ int base;
    const int s = blockIdx.x, tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (w == 0) {
        int acc = 0;
        for (int i = lane; i < s; i += 32) acc += seg_count[i];
#pragma unroll
        for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) base = acc;
    }
    const int t0 = s * kTileSeg + tid * 16;
    unsigned bits = 0;
#pragma unroll
    for (int k = 0; k < 16; ++k)
        if (t0 + k < total && mask[t0 + k]) bits |= 1u << k;
    const int cnt = __popc(bits);
    int inc = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += v;
    }
    if (lane == 31) wsum[w] = inc;
    __syncthreads();
    int wbase = 0, btotal = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int v = wsum[i];
        wbase += i < w ? v : 0;
        btotal += v;
    }
    int pos = base + wbase + inc - cnt;
    while (bits) {
        const int k = __ffs(bits) - 1;
        bits &= bits - 1;
        list[1 + pos++] = t0 + k;
    }
    if (s == (int)gridDim.x - 1 && tid == 0) list[0] = base + btotal;
}

template <typename T>
__global__ void __launch_bounds__(256) fma_peak_kernel(T *sink, int iters, T a, T b) {
    T x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = (T)(threadIdx.x + i);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = fma(x[i], a, b);
    }
    T s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += x[i];
    if (s == (T)12345.678) sink[blockIdx.x] = s;
}

cudaError_t launch_fma_peak(int fp64, int blocks, int iters, void *sink, cudaStream_t st) {
    if (fp64)
        fma_peak_kernel<double><<<blocks, 256, 0, st>>>((double *)sink, iters, 0.999999, 1e-7);
    else
        fma_peak_kernel<float><<<blocks, 256, 0, st>>>((float *)sink, iters, 0.999999f, 1e-7f);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Compiled shapes.  First generation (bp_tiles): {form, tile_x, tile_y,
// threads, chunk, window}.  Warp-specialised (bp_ws): {form, tile_x, tile_y,
// consumer warps, chunk, stages, window, min blocks per SM}; block = consumer
// warps + 1.
#define SRG_SHAPES(X)                  \
    X(FORM_SPLIT, 32, 8, 128, 32, 160)  \
    X(FORM_SPLIT, 32, 16, 128, 16, 192) \
    X(FORM_FP64, 32, 4, 128, 32, 128)   \
    X(FORM_FP64, 32, 8, 128, 32, 160)

#define SRG_WS_SHAPES(X)                    \
    X(FORM_SPLIT, 32, 8, 4, 31, 2, 128, 3)  \
    X(FORM_SPLIT, 32, 8, 4, 16, 3, 128, 3)  \
    X(FORM_SPLIT, 32, 8, 4, 16, 3, 128, 4)  \
    X(FORM_SPLIT, 32, 8, 4, 16, 2, 128, 3)  \
    X(FORM_SPLIT, 32, 8, 4, 24, 3, 128, 3)  \
    X(FORM_SPLIT, 16, 16, 4, 16, 3, 96, 3)  \
    X(FORM_SPLIT, 32, 16, 4, 16, 3, 144, 2)  \
    X(FORM_SPLIT, 16, 16, 4, 31, 2, 128, 3)  \
    X(FORM_SPLIT, 32, 8, 4, 16, 2, 256, 3)

#define SRG_WS_FP64_SHAPES(X)               \
    X(FORM_FP64, 32, 4, 4, 16, 2, 128, 3)   \
    X(FORM_FP64, 32, 8, 4, 16, 2, 128, 2)

#define SRG_ENTRY(F, TXv, TYv, NTv, CKv, WBv)                                                   \
    {F, {TXv, TYv, NTv, CKv, WBv}, params_bytes<F, CKv>() + 1024 + CKv * WBv * 8,               \
     (const void *)bp_tiles<F, TXv, TYv, NTv, CKv>,                                             \
     "bp_tiles<" #F "," #TXv "x" #TYv ",threads " #NTv ",chunk " #CKv ",window " #WBv ">", 0},
#define SRG_WS_ENTRY(F, TXv, TYv, NCv, CKv, NSv, WBv, MBv)                                      \
    {F, {TXv, TYv, (NCv + 1) * 32, CKv, WBv}, ws_smem_bytes<F, CKv, NSv>(WBv),                  \
     (const void *)bp_ws<F, TXv, TYv, NCv, CKv, NSv, WBv, MBv>,                                 \
     "bp_ws<" #F "," #TXv "x" #TYv ",consumer warps " #NCv ",chunk " #CKv ",stages " #NSv       \
     ",window " #WBv ",min blocks " #MBv ">", 1},

// The first shape of a form is its default: the fastest measured on the
// B200 (warp-specialised for the split form, first generation for FP64).
const KernelEntry kKernels[] = {SRG_WS_SHAPES(SRG_WS_ENTRY) SRG_SHAPES(SRG_ENTRY)
                                    SRG_WS_FP64_SHAPES(SRG_WS_ENTRY)};
const int kNumKernels = sizeof(kKernels) / sizeof(kKernels[0]);

// Gated twins (range lines still uploading; the drop-in entry) of the
// default warp-specialised shapes.  Not listed among the tunable shapes.
#define SRG_WS_GATED_ENTRY(F, TXv, TYv, NCv, CKv, NSv, WBv, MBv)                                \
    {F, {TXv, TYv, (NCv + 1) * 32, CKv, WBv}, ws_smem_bytes<F, CKv, NSv>(WBv),                  \
     (const void *)bp_ws<F, TXv, TYv, NCv, CKv, NSv, WBv, MBv, true>,                           \
     "bp_ws<" #F "," #TXv "x" #TYv ",consumer warps " #NCv ",chunk " #CKv ",stages " #NSv       \
     ",window " #WBv ",min blocks " #MBv ",gated>", 1},
const KernelEntry kGatedKernels[] = {SRG_WS_GATED_ENTRY(FORM_SPLIT, 32, 8, 4, 31, 2, 128, 3)};
const int kNumGatedKernels = sizeof(kGatedKernels) / sizeof(kGatedKernels[0]);

const KernelEntry *gated_twin(const KernelEntry &e) {
    for (int i = 0; i < kNumGatedKernels; ++i) {
        const KernelEntry &g = kGatedKernels[i];
        // same template arguments: the names agree up to the closing '>'
        const size_t n = std::strlen(e.name);
        if (g.form == e.form && n > 1 && std::strncmp(g.name, e.name, n - 1) == 0 &&
            g.name[n - 1] == ',')
            return &g;
    }
    return nullptr;
}

cudaError_t launch_tiles(const KernelEntry &e, int grid, size_t smem, cudaStream_t st,
                         const BurstDev *bursts, int nb, int total, const CUtensorMap *tmaps,
                         int *counter, int *err, const int *tile_list) {
    int WB = e.shape.window;
    void *args[] = {(void *)&bursts, (void *)&nb, (void *)&total, (void *)&tmaps,
                    (void *)&counter, (void *)&err, (void *)&WB, (void *)&tile_list};
    return cudaLaunchKernel(e.fn, dim3(grid), dim3(e.shape.threads), args, smem, st);
}

cudaError_t launch_line_centres(const BurstDev &B, const Orbit &o, const CentreParams &cp,
                                double *coef, cudaStream_t st) {
    const int warps = (B.nlines + 9) / 10;  // ten lines per warp
    line_centres_kernel<<<(warps + 3) / 4, 128, 0, st>>>(B, o, cp, coef);
    return cudaGetLastError();
}

cudaError_t launch_count_terms(const BurstDev &B, unsigned long long *terms, int sms,
                               cudaStream_t st) {
    const int nt = 256;
    const long long npix = (long long)(B.lastpix_eff - B.firstpix + 1) * B.nlines;
    if (npix <= 0) return cudaSuccess;
    long long blocks = (npix + nt - 1) / nt;
    if (blocks > 64LL * sms) blocks = 64LL * sms;
    count_terms_kernel<<<(int)blocks, nt, 0, st>>>(B, terms);
    return cudaGetLastError();
}

cudaError_t launch_merge(float2 *dst, long long dst_ld, const float2 *src, long long src_ld,
                         int rows, int cols, int sms, cudaStream_t st) {
    const long long n = (long long)rows * cols;
    if (n <= 0) return cudaSuccess;
    long long blocks = (n + 255) / 256;
    if (blocks > 32LL * sms) blocks = 32LL * sms;
    merge_kernel<<<(int)blocks, 256, 0, st>>>(dst, dst_ld, src, src_ld, rows, cols);
    return cudaGetLastError();
}

cudaError_t launch_line_centres_batch(const BurstDev *bursts, const CentreJob *jobs, int n,
                                      int total, cudaStream_t st) {
    if (total <= 0) return cudaSuccess;
    const int warps = (total + 9) / 10;  // ten lines per warp
    line_centres_batch_kernel<<<(warps + 3) / 4, 128, 0, st>>>(bursts, jobs, n, total);
    return cudaGetLastError();
}

cudaError_t launch_tile_list(const BurstDev *bursts, int nbursts, int max_burst_tiles, int total,
                             int tx, int ty, void *scratch, cudaStream_t st, int *band) {
    if (total <= 0 || nbursts <= 0 || max_burst_tiles <= 0 || tx > 32 || ty > 32)
        return cudaErrorInvalidValue;
    int *list = static_cast<int *>(scratch);
    int *seg = tile_list_segments(scratch, total);
    unsigned char *mask = tile_list_mask(scratch, total);
    const int nseg = (total + kTileSeg - 1) / kTileSeg;
    cudaError_t e = cudaMemsetAsync(seg, 0, sizeof(int) * nseg, st);
    if (e != cudaSuccess) return e;
    tile_mask_kernel<<<dim3((max_burst_tiles + 7) / 8, nbursts), 256, 0, st>>>(bursts, tx, ty, mask,
                                                                                 seg, band);
    tile_compact_kernel<<<nseg, 256, 0, st>>>(mask, seg, total, list);
    return cudaGetLastError();
}

cudaError_t launch_merge_scene(const BurstDev *bursts, int n, float2 *dst, long long dst_ld,
                               int lines, int cols, cudaStream_t st, const unsigned char *tile_mask,
                               int tx, int ty) {
    if (lines <= 0 || cols <= 0 || n <= 0) return cudaSuccess;
    if (n > 256) return cudaErrorInvalidValue;
    int txl = 0, tyl = 0;
    while ((1 << txl) < tx) ++txl;
    while ((1 << tyl) < ty) ++tyl;
    if (tile_mask && ((1 << txl) != tx || (1 << tyl) != ty)) tile_mask = nullptr;  // powers of two only
    dim3 grid((cols + 31) / 32, (lines + 31) / 32);
    merge_scene_kernel<<<grid, dim3(32, 8), 0, st>>>(bursts, n, dst, dst_ld, lines, cols, tile_mask,
                                                     txl, tyl);
    return cudaGetLastError();
}

cudaError_t launch_range_band(const BurstDev &B, int *band, int sms, cudaStream_t st) {
    (void)sms;
    const int nx = B.lastpix_eff - B.firstpix + 1;
    if (nx <= 0 || B.nlines <= 0) return cudaSuccess;
    const dim3 grid((nx + kBandCols - 1) / kBandCols, (B.nlines + kBandLines - 1) / kBandLines);
    range_band_kernel<<<grid, 256, 0, st>>>(B, band);
    return cudaGetLastError();
}

cudaError_t launch_pulse_orbit(const double *times, int P, const Orbit &o, double *pos,
                               double *vel, cudaStream_t st) {
    if (P <= 0) return cudaSuccess;
    pulse_orbit_kernel<<<(P + 127) / 128, 128, 0, st>>>(times, P, o, pos, vel);
    return cudaGetLastError();
}

cudaError_t launch_forward_project(const BurstDev &B, const float2 *refl, long long refl_ld,
                                   const double *satvel, double antenna, const float *range_offset,
                                   cudaStream_t st) {
    const long long npix = (long long)(B.lastpix_eff - B.firstpix + 1) * B.nlines;
    if (npix <= 0) return cudaSuccess;
    forward_project_kernel<<<(int)((npix + 127) / 128), 128, 0, st>>>(B, refl, refl_ld, satvel,
                                                                       antenna, range_offset);
    return cudaGetLastError();
}

}  // namespace srg
