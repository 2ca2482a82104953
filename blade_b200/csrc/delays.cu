// Geometric delays: the astrometric half of Modules::Phasor::ATA
// (src/modules/phasor/ata.cc:9-173), which the reference computes with ERFA
// through radiointerferometryc99 (neither is vendored).  Restated here from
// published formulas, FP64 throughout:
//   * time scales: UT1 = UTC + DUT1; TT = UTC + 69.184 s (TAI - UTC = 37 s);
//   * Greenwich mean sidereal time, IAU 1982 (Aoki et al. 1982; Meeus,
//     Astronomical Algorithms, 2nd ed., eq. 12.4), apparent = mean + dpsi cos(eps);
//   * precession, IAU 1976 (Lieske et al. 1977): P = R3(-z_A) R2(theta_A) R3(-zeta_A);
//   * nutation, the four leading terms of IAU 1980 (Meeus ch. 22):
//     N = R1(-eps) R3(-dpsi) R1(eps0);
//   * annual aberration in the circular-orbit approximation (Meeus ch. 23):
//     p' = p + kappa (sin L, -cos L cos eps, -cos L sin eps), kappa = 20.49552";
//   * the source direction in the terrestrial frame s = R3(GAST) N P p' (polar
//     motion neglected), and per antenna a and beam b
//       delay[b, a] = ((r_a - r_ref) . s_b - (r_a - r_ref) . s_boresight) / c,
//     the reference's TPi = (WPi - WPr) / C - (Wi - Wr) / C (ata.cc:39-47), W
//     being the projection of the antenna's array-centred position on the source
//     direction.  The array reference position cancels from these differences.
// Per block the host computes one direction per beam (the scalar astrometry);
// the A x B projections run on the device.
#include <math.h>

#include <vector>

#include "common.cuh"

namespace bb {
namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kAs2Rad = kPi / (180.0 * 3600.0);
constexpr double kDeg2Rad = kPi / 180.0;
constexpr double kC = 299792458.0;

struct M3 {
    double m[3][3];
};

M3 mul(const M3& a, const M3& b) {
    M3 r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) r.m[i][j] = a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j] + a.m[i][2] * b.m[2][j];
    return r;
}

// Frame rotations about x, y, z by angle t (the Explanatory Supplement's R1, R2, R3).
M3 r1(double t) {
    const double c = cos(t), s = sin(t);
    return M3{{{1, 0, 0}, {0, c, s}, {0, -s, c}}};
}
M3 r2(double t) {
    const double c = cos(t), s = sin(t);
    return M3{{{c, 0, -s}, {0, 1, 0}, {s, 0, c}}};
}
M3 r3(double t) {
    const double c = cos(t), s = sin(t);
    return M3{{{c, s, 0}, {-s, c, 0}, {0, 0, 1}}};
}

void apply(const M3& a, const double (&v)[3], double (&o)[3]) {
    for (int i = 0; i < 3; i++) o[i] = a.m[i][0] * v[0] + a.m[i][1] * v[1] + a.m[i][2] * v[2];
}

}  // namespace

// Unit vector of (ra, dec) (ICRS, radians) in the terrestrial frame at UTC julian
// date jd with UT1 - UTC = dut1 seconds.
void source_itrs(double ra, double dec, double jd, double dut1, double (&s)[3]) {
    const double jd_ut1 = jd + dut1 / 86400.0;
    const double jd_tt = jd + 69.184 / 86400.0;
    const double t = (jd_tt - 2451545.0) / 36525.0;  // Julian centuries of TT from J2000.0
    // nutation (leading IAU 1980 terms) and obliquity
    const double om = (125.04452 - 1934.136261 * t) * kDeg2Rad;
    const double ls = (280.4665 + 36000.7698 * t) * kDeg2Rad;
    const double lm = (218.3165 + 481267.8813 * t) * kDeg2Rad;
    const double dpsi = (-17.20 * sin(om) - 1.32 * sin(2 * ls) - 0.23 * sin(2 * lm) + 0.21 * sin(2 * om)) * kAs2Rad;
    const double deps = (9.20 * cos(om) + 0.57 * cos(2 * ls) + 0.10 * cos(2 * lm) - 0.09 * cos(2 * om)) * kAs2Rad;
    const double eps0 = (84381.448 - 46.8150 * t - 0.00059 * t * t + 0.001813 * t * t * t) * kAs2Rad;
    const double eps = eps0 + deps;
    // annual aberration: Sun's true longitude from its mean longitude and anomaly
    const double l0 = (280.46646 + 36000.76983 * t + 0.0003032 * t * t) * kDeg2Rad;
    const double ma = (357.52911 + 35999.05029 * t - 0.0001537 * t * t) * kDeg2Rad;
    const double cen = ((1.914602 - 0.004817 * t - 0.000014 * t * t) * sin(ma) + (0.019993 - 0.000101 * t) * sin(2 * ma) +
                        0.000289 * sin(3 * ma)) * kDeg2Rad;
    const double lsun = l0 + cen;
    const double kappa = 20.49552 * kAs2Rad;
    double p[3] = {cos(dec) * cos(ra), cos(dec) * sin(ra), sin(dec)};
    p[0] += kappa * sin(lsun);
    p[1] += -kappa * cos(lsun) * cos(eps);
    p[2] += -kappa * cos(lsun) * sin(eps);
    const double n = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    for (double& v : p) v /= n;
    // precession (IAU 1976)
    const double zeta = (2306.2181 * t + 0.30188 * t * t + 0.017998 * t * t * t) * kAs2Rad;
    const double z = (2306.2181 * t + 1.09468 * t * t + 0.018203 * t * t * t) * kAs2Rad;
    const double theta = (2004.3109 * t - 0.42665 * t * t - 0.041833 * t * t * t) * kAs2Rad;
    const M3 P = mul(r3(-z), mul(r2(theta), r3(-zeta)));
    const M3 N = mul(r1(-eps), mul(r3(-dpsi), r1(eps0)));
    // Greenwich apparent sidereal time
    const double du = jd_ut1 - 2451545.0, tu = du / 36525.0;
    double gmst = 280.46061837 + 360.98564736629 * du + 0.000387933 * tu * tu - tu * tu * tu / 38710000.0;
    gmst = fmod(gmst, 360.0) * kDeg2Rad;
    const double gast = gmst + dpsi * cos(eps);
    const M3 W = mul(r3(gast), mul(N, P));
    apply(W, p, s);
}

namespace {

constexpr uint32_t kMaxVec = 1024;  // antennas + beams per call

// Baselines to the reference antenna [A][3] then beam direction differences
// s_b - s_boresight [B][3], passed by value (24 KB of launch parameters).
struct DelayArgs {
    uint32_t A, B;
    double v[3 * kMaxVec];
};

// delays[b, a] = (bl_a . (s_b - s_0)) / c, one thread per (b, a).
__global__ void delays_kernel(const __grid_constant__ DelayArgs g, double* __restrict__ out) {
    const uint64_t n = (uint64_t)g.A * g.B;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t b = (uint32_t)(i / g.A), a = (uint32_t)(i - (uint64_t)b * g.A);
        const double* r = g.v + 3 * a;
        const double* d = g.v + 3 * (g.A + b);
        out[i] = (r[0] * d[0] + r[1] * d[1] + r[2] * d[2]) / kC;
    }
}

}  // namespace
}  // namespace bb

extern "C" int blade_geometric_delays(const double* antenna_positions, uint64_t A, uint64_t reference_antenna,
                                      const double* array_reference_lla, double boresight_ra, double boresight_dec,
                                      const double* beam_coordinates, uint64_t B, double julian_date, double dut1,
                                      double* delays, blade_stream_t stream) {
    using namespace bb;
    const char* who = "blade_geometric_delays";
    if (A == 0 || B == 0) return BLADE_SUCCESS;
    if (!antenna_positions || !beam_coordinates || !delays) return set_error(BLADE_ERROR, "%s: null buffer", who);
    if (reference_antenna >= A)
        return set_error(BLADE_ERROR, "%s: reference antenna %llu out of range (A = %llu)", who,
                         (unsigned long long)reference_antenna, (unsigned long long)A);
    if (A + B > kMaxVec)
        return set_error(BLADE_ERROR, "%s: at most %u antennas + beams per call (A = %llu, B = %llu)", who, kMaxVec,
                         (unsigned long long)A, (unsigned long long)B);
    if (array_reference_lla && !(fabs(array_reference_lla[1]) <= kPi / 2))
        return set_error(BLADE_ERROR, "%s: array reference latitude out of range", who);
    if (!isfinite(julian_date) || !isfinite(dut1)) return set_error(BLADE_ERROR, "%s: invalid date", who);
    // host: baselines to the reference antenna and per-beam direction differences
    DelayArgs g;
    g.A = (uint32_t)A;
    g.B = (uint32_t)B;
    const double* ref = antenna_positions + 3 * reference_antenna;
    for (uint64_t a = 0; a < A; a++)
        for (int k = 0; k < 3; k++) g.v[3 * a + k] = antenna_positions[3 * a + k] - ref[k];
    double s0[3];
    source_itrs(boresight_ra, boresight_dec, julian_date, dut1, s0);
    for (uint64_t b = 0; b < B; b++) {
        double sb[3];
        source_itrs(beam_coordinates[2 * b], beam_coordinates[2 * b + 1], julian_date, dut1, sb);
        for (int k = 0; k < 3; k++) g.v[3 * (A + b) + k] = sb[k] - s0[k];
    }
    delays_kernel<<<grid_for(A * B, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(g, delays);
    return check_launch(who);
}

extern "C" int blade_source_direction(double ra, double dec, double julian_date, double dut1, double* direction) {
    if (!direction) return bb::set_error(BLADE_ERROR, "blade_source_direction: null output");
    double s[3];
    bb::source_itrs(ra, dec, julian_date, dut1, s);
    for (int k = 0; k < 3; k++) direction[k] = s[k];
    return BLADE_SUCCESS;
}
