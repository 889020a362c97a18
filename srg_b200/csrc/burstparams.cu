// burstparams.cu -- per-burst scalars of the azimuth_compress_ call, derived
// from the decoded Sentinel-1 line headers and the per-pulse velocities the
// way sentinel/backprojectgpusub.f90 derives them before each call:
//
//   burstparams  (:406-429)  start time, PRF, sampling rate, PRI, near range
//                            and wavelength from the first line's header;
//   fdopcoefs    (:262-309)  the azimuth steering angle of every line from
//                            its beam address, fitted linearly against time
//                            (linfit, :381-403) over all but 20 lines at each
//                            end: angc0, angc1;
//   the loop body (:190-227) aperture (50 % of the TOPS aperture, from the
//                            velocity at mid-burst), azimuth and range limits.
//
// Host code.  The arithmetic keeps the Fortran's precisions, because they
// decide the values bit for bit: the literals the reference writes without a
// d exponent are single precision (fref and 1.e-6 in fdopcoefs and
// burstparams, wvl), the steering angles, per-line PRF and times are REAL
// (float), linfit sums single-precision products in double and returns
// single-precision coefficients.
#include <cmath>
#include <cstdint>
#include <cstring>

#include "host_internal.h"

using namespace srg::detail;

namespace {

constexpr double kFref = 37.53472224;  // MHz, as a REAL*8 literal (burstparams)
constexpr double kSol = 299792458.0;

// Big-endian unsigned fields of a line header (processsub.f90:163-173).
int in2(const unsigned char *b) { return (int)b[1] + 256 * (int)b[0]; }
int in3(const unsigned char *b) { return (int)b[2] + 256 * (int)b[1] + 65536 * (int)b[0]; }
double d8(const unsigned char *b) {
    double d;
    std::memcpy(&d, b, 8);
    return d;
}

// processsub.f90:176-211: sampling rate (MHz) of a range decimation code; the
// fractions are REAL (3./4.*4. in single precision), times fref in double.
bool sample_frequency(int code, double *mhz) {
    float f;
    switch (code) {
        case 0: f = 3.f / 4.f * 4.f; break;
        case 1: f = 2.f / 3.f * 4.f; break;
        case 3: f = 5.f / 9.f * 4.f; break;
        case 4: f = 4.f / 9.f * 4.f; break;
        case 5: f = 3.f / 8.f * 4.f; break;
        case 6: f = 1.f / 3.f * 4.f; break;
        case 7: f = 1.f / 6.f * 4.f; break;
        case 8: f = 3.f / 7.f * 4.f; break;
        case 9: f = 5.f / 16.f * 4.f; break;
        case 10: f = 3.f / 26.f * 4.f; break;
        case 11: f = 4.f / 11.f * 4.f; break;
        default: return false;  // the reference returns an undefined value
    }
    *mhz = (double)f * kFref;
    return true;
}

// Header bytes of line i: the first 10 complex64 samples (80 bytes).
const unsigned char *header(const float *lines, long long ld, int i) {
    return reinterpret_cast<const unsigned char *>(lines + 2 * (size_t)ld * (size_t)i);
}

}  // namespace

extern "C" int srg_burst_params(const float *lines, long long ld, int P, int S,
                                const double *satvel, srg_burst_params_t *out) {
    if (!lines || !satvel || !out) return fail(SRG_E_ARG, "null argument");
    if (P < 41 || S < 11 || ld < S)
        return fail(SRG_E_ARG, "need >= 41 lines of >= 11 samples (P=%d S=%d ld=%lld)", P, S, ld);
    srg_burst_params_t r;
    std::memset(&r, 0, sizeof r);
    // burstparams (:406-429), from the first line's header
    const unsigned char *h0 = header(lines, ld, 0);
    const int pri_code = in3(h0 + 50);
    if (pri_code == 0) return fail(SRG_E_ARG, "PRI code 0 in the first line's header");
    r.starttime = d8(h0 + 68);
    r.prf = kFref / pri_code * (double)1.e6f;
    double fs_mhz;
    const int decimation = (int)h0[40];
    if (!sample_frequency(decimation, &fs_mhz))
        return fail(SRG_E_ARG, "unknown range decimation code %d", decimation);
    r.samplefreq = fs_mhz * (double)1.e6f;
    const double swst = in3(h0 + 53) / kFref * (double)1.e-6f;
    const int irank = (int)(h0[49] & 31);
    r.pri = pri_code / kFref * (double)1.e-6f;
    r.range0 = kSol / 2. * (irank * r.pri + swst) + 60.;
    r.wvl = (double)0.05546576f;
    // fdopcoefs (:262-309): fref is a REAL literal there
    const double fref_s = (double)37.53472224f;
    double sumx = 0., sumx2 = 0., sumxy = 0., sumy = 0.;
    const int npts = P - 40;
    const float half = (float)P / 2.f;
    for (int i = 21; i <= P - 20; ++i) {  // t(21), ang(21), lines - 40 points (1-based i)
        const unsigned char *h = header(lines, ld, i - 1);
        const int word = in2(h + 60);
        const int azimuthbeam = word & 1023;
        const float ang = (float)azimuthbeam / 1024.f * 1.8f - 0.9f;
        const int code = in3(h + 50);
        if (code == 0) return fail(SRG_E_ARG, "PRI code 0 in the header of line %d", i - 1);
        const float prf_i = (float)(fref_s / code * (double)1.e6f);
        const float t = ((float)i - half) / prf_i;
        sumx = sumx + (double)t;
        sumx2 = sumx2 + (double)(t * t);
        sumxy = sumxy + (double)(t * ang);
        sumy = sumy + (double)ang;
    }
    const double den = npts * sumx2 - sumx * sumx;
    if (!(den != 0.)) return fail(SRG_E_ARG, "degenerate line times in the headers");
    const float c1 = (float)((npts * sumxy - sumx * sumy) / den);
    const float c0 = (float)((sumy * sumx2 - sumx * sumxy) / den);
    r.angc0 = (double)c0;
    r.angc1 = (double)c1;
    // aperture (:190-209): velocity at mid-burst, scaled to the ground
    const double re = 6378137.0, ht = 700000.0;
    const double pi = ref_pi();
    const double *v = satvel + 3 * (size_t)(P / 2 - 1);
    double vmag = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    vmag = vmag * (re / (re + ht));
    const double aperturetime = (r.range0 * r.wvl / 2 / vmag / vmag * r.prf) /
                                (1. + r.range0 * r.angc1 * pi / 180. / vmag);
    const double burstpoints = aperturetime * r.prf * 0.5;
    if (!std::isfinite(burstpoints) || burstpoints < 0 || burstpoints > 1e9)
        return fail(SRG_E_ARG, "aperture out of range (%g points)", burstpoints);
    r.aperture = (int)burstpoints;
    // azimuth and range limits (:213-227)
    r.tstart = r.starttime;
    r.dtaz = 1.0 / r.prf;
    r.tend = r.tstart + (P - 1) * r.dtaz;
    r.tmid = 0.5 * (r.tstart + r.tend);
    const double slant_range_time = 2 * r.range0 / kSol;
    r.rngstart = slant_range_time * kSol / 2.0;
    r.dmrg = kSol / 2.0 / r.samplefreq;
    r.rngend = r.rngstart + (S - 1) * r.dmrg;
    *out = r;
    return SRG_OK;
}
