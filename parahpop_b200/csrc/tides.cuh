// Epoch-only Earth tide coefficient sets (IERS Conventions 2010 ch. 6):
// solid tide degree 2/3 direct + induced degree 4, frequency-dependent
// corrections (Tables 6.5a-c), zero-tide permanent term, solid pole tide;
// FES2004 ocean tide (18 waves, degree/order <= 6) and ocean pole tide.
//
// Restates src/common/engine/paraHPOP/model/accelerations/hpop_compat/
// HpopCorrections.h:94-322 (gmst06 :94, legendreValues :105, bodyGeometry
// :158, tideArguments :175, poleWobble :187, solidFromGeometry :201,
// oceanFromEpoch :298).  The coefficient sets depend only on the epoch and
// the Sun / Moon geometry, so the kernels evaluate them once per stage epoch
// and fold them into the low-degree geopotential; host and device share this
// header.  Units: SI, E = ICRF -> ITRF rotation (row-major).
#pragma once
#include <math.h>

#if defined(__CUDACC__)
#define PHOP_HD __host__ __device__ __forceinline__
#else
#define PHOP_HD inline
#endif

namespace phop {
namespace tides {

struct PhopFreqTerm { signed char multiplier[5]; double inPhase, outPhase; };
struct PhopOceanWave { signed char doodson[6]; unsigned short begin, end; };
struct PhopOceanTerm { unsigned char n, m; double cp, sp, cm, sm; };

#if defined(__CUDACC__)
#define PHOP_TIDE_TABLE(type, name, count) __constant__ type dev_##name[count]
#include "tables/tide_tables.inc"
#undef PHOP_TIDE_TABLE
#endif
#define PHOP_TIDE_TABLE(type, name, count) static const type host_##name[count]
#include "tables/tide_tables.inc"
#undef PHOP_TIDE_TABLE

#if defined(__CUDA_ARCH__)
#define TIDET(name) dev_##name
#else
#define TIDET(name) host_##name
#endif

struct Epoch {
    double E[9];              // ICRF -> ITRF
    double sun[3], moon[3];   // geocentric ICRF, m
    double mjdUtc, ut1Utc, ttUtc, xpArcsec, ypArcsec;
};

struct Coeffs {
    double C[7][7];
    double S[7][7];
};

// Constants of the tide and relativity model (HpopCorrections.h:25-34).
struct Consts {
    static constexpr double muEarth = 398600.4415e9;
    static constexpr double radius = 6378.1363e3;
    static constexpr double muSun = 132712440041.279419e9;
    static constexpr double muMoon = 398600.4415e9 / 81.3005682214972154;
    static constexpr double c = 299792457.999999984;
};

constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kTwoPi = 2.0 * kPi;
constexpr double kArcsec = kPi / (180.0 * 3600.0);

PHOP_HD double positiveMod(double x, double period) {
    const double a = fmod(x, period);
    return a < 0.0 ? a + period : a;
}

PHOP_HD void clear(Coeffs& c) {
    for (int n = 0; n < 7; ++n)
        for (int m = 0; m < 7; ++m) c.C[n][m] = c.S[n][m] = 0.0;
}

PHOP_HD void rotate(const double E[9], const double x[3], double out[3]) {
    for (int i = 0; i < 3; ++i) out[i] = E[3 * i] * x[0] + E[3 * i + 1] * x[1] + E[3 * i + 2] * x[2];
}

// Earth rotation angle + IAU 2006 GMST polynomial (operation order as SOFA)
PHOP_HD double gmst06(double mjdUt1, double mjdTt) {
    const double eraT = mjdUt1 + (2400000.5 - 2451545.0);
    const double f = fmod(mjdUt1, 1.0) + fmod(2400000.5, 1.0);
    const double era = positiveMod(kTwoPi * (f + 0.7790572732640 + 0.00273781191135448 * eraT), kTwoPi);
    const double t = ((2400000.5 - 2451545.0) + mjdTt) / 36525.0;
    return positiveMod(
        era + (0.014506 + (4612.156534 + (1.3915817 + (-0.00000044 + (-0.000029956 - 0.0000000368 * t) * t) * t) * t) * t)
                  * kArcsec,
        kTwoPi);
}

// fully normalised associated Legendre values P[n][m](sin phi), n <= nmax
PHOP_HD void legendreValues(int nmax, double phi, double p[7][7]) {
    for (int n = 0; n < 7; ++n)
        for (int m = 0; m < 7; ++m) p[n][m] = 0.0;
    const double s = sin(phi), c = cos(phi);
    p[0][0] = 1.0;
    if (nmax == 0) return;
    p[1][1] = sqrt(3.0) * c;
    for (int n = 2; n <= nmax; ++n) p[n][n] = sqrt((2.0 * n + 1) / (2.0 * n)) * c * p[n - 1][n - 1];
    for (int n = 1; n <= nmax; ++n) p[n][n - 1] = sqrt(2.0 * n + 1) * s * p[n - 1][n - 1];
    for (int m = 0; m <= nmax; ++m)
        for (int n = m + 2; n <= nmax; ++n)
            p[n][m] = sqrt((2.0 * n + 1) / ((n - m) * double(n + m)))
                * (sqrt(2.0 * n - 1) * s * p[n - 1][m] - sqrt(((n + m - 1) * double(n - m - 1)) / (2.0 * n - 3)) * p[n - 2][m]);
}

// Delaunay arguments (rad) and GMST for the tide epoch
PHOP_HD void arguments(const Epoch& in, double args[5], double& thetaG) {
    const double mjdTt = in.mjdUtc + in.ttUtc / 86400.0;
    const double t = (mjdTt - 51544.5) / 36525.0, t2 = t * t, t3 = t2 * t, t4 = t3 * t;
    args[0] = positiveMod(485868.249036 + 1717915923.2178 * t + 31.8792 * t2 + 0.051635 * t3 - 0.00024470 * t4, 1296000.0) * kArcsec;
    args[1] = positiveMod(1287104.79305 + 129596581.0481 * t - 0.5532 * t2 + 0.000136 * t3 - 0.00001149 * t4, 1296000.0) * kArcsec;
    args[2] = positiveMod(335779.526232 + 1739527262.8478 * t - 12.7512 * t2 - 0.001037 * t3 + 0.00000417 * t4, 1296000.0) * kArcsec;
    args[3] = positiveMod(1072260.70369 + 1602961601.2090 * t - 6.3706 * t2 + 0.006593 * t3 - 0.00003169 * t4, 1296000.0) * kArcsec;
    args[4] = positiveMod(450160.398036 - 6962890.5431 * t + 7.4722 * t2 + 0.007702 * t3 - 0.00005939 * t4, 1296000.0) * kArcsec;
    thetaG = gmst06(in.mjdUtc + in.ut1Utc / 86400.0, mjdTt);
}

// pole coordinates relative to the IERS 2010 mean pole (arcsec)
PHOP_HD void poleWobble(const Epoch& in, double& m1, double& m2) {
    const double t = (in.mjdUtc + in.ttUtc / 86400.0 - 51544.5) / 365.25;
    double x, y;
    if (t < 10.0) {
        x = 55.974 + t * (1.8243 + t * (0.18413 + t * 0.007024));
        y = 346.346 + t * (1.7896 + t * (-0.10729 - t * 0.000908));
    } else {
        x = 23.513 + 7.6141 * t;
        y = 358.891 - 0.6287 * t;
    }
    m1 = in.xpArcsec - 1e-3 * x;
    m2 = -(in.ypArcsec - 1e-3 * y);
}

PHOP_HD PhopFreqTerm freqTerm(int order, int i) {
    if (order == 0) return TIDET(tide_freq0)[i];
    if (order == 1) return TIDET(tide_freq1)[i];
    return TIDET(tide_freq2)[i];
}

// solid Earth tide (zero-tide static field) coefficient corrections
PHOP_HD void solid(const Epoch& in, Coeffs& out, bool zeroTide = true) {
    clear(out);
    double moon[3], sun[3];
    rotate(in.E, in.moon, moon);
    rotate(in.E, in.sun, sun);
    const double moonLon = atan2(moon[1], moon[0]);
    const double sunLon = atan2(sun[1], sun[0]);
    const double moonRatio = Consts::radius / sqrt(moon[0] * moon[0] + moon[1] * moon[1] + moon[2] * moon[2]);
    const double sunRatio = Consts::radius / sqrt(sun[0] * sun[0] + sun[1] * sun[1] + sun[2] * sun[2]);
    double moonP[7][7], sunP[7][7];
    legendreValues(3, atan2(moon[2], hypot(moon[0], moon[1])), moonP);
    legendreValues(3, atan2(sun[2], hypot(sun[0], sun[1])), sunP);
    // degree 2 (and induced degree 4): IERS (6.6), (6.7), Table 6.3
    const double moonF = Consts::muMoon / Consts::muEarth * pow(moonRatio, 3.0);
    const double sunF = Consts::muSun / Consts::muEarth * pow(sunRatio, 3.0);
    double qC[3], qS[3];
    for (int m = 0; m <= 2; ++m) {
        qC[m] = moonF * moonP[2][m] * cos(m * moonLon) + sunF * sunP[2][m] * cos(m * sunLon);
        qS[m] = moonF * moonP[2][m] * sin(m * moonLon) + sunF * sunP[2][m] * sin(m * sunLon);
    }
    out.C[2][0] = 0.30190 / 5.0 * qC[0];
    out.C[2][1] = 0.29830 / 5.0 * qC[1] - 0.00144 / 5.0 * qS[1];
    out.S[2][1] = 0.00144 / 5.0 * qC[1] + 0.29830 / 5.0 * qS[1];
    out.C[2][2] = 0.30102 / 5.0 * qC[2] - 0.00130 / 5.0 * qS[2];
    out.S[2][2] = 0.00130 / 5.0 * qC[2] + 0.30102 / 5.0 * qS[2];
    out.C[4][0] = -0.00089 / 5.0 * qC[0];
    out.C[4][1] = -0.00080 / 5.0 * qC[1];
    out.S[4][1] = -0.00080 / 5.0 * qS[1];
    out.C[4][2] = -0.00057 / 5.0 * qC[2];
    out.S[4][2] = -0.00057 / 5.0 * qS[2];
    // degree 3 direct
    const double moon3 = Consts::muMoon / Consts::muEarth * pow(moonRatio, 4.0);
    const double sun3 = Consts::muSun / Consts::muEarth * pow(sunRatio, 4.0);
    for (int m = 0; m <= 3; ++m) {
        const double k3 = (m == 3 ? 0.094 : 0.093) / 7.0;
        out.C[3][m] = k3 * (moon3 * moonP[3][m] * cos(m * moonLon) + sun3 * sunP[3][m] * cos(m * sunLon));
        if (m) out.S[3][m] = k3 * (moon3 * moonP[3][m] * sin(m * moonLon) + sun3 * sunP[3][m] * sin(m * sunLon));
    }
    // frequency-dependent corrections (Tables 6.5a-c, units 1e-12)
    double args[5], thetaG;
    arguments(in, args, thetaG);
    for (int order = 0; order <= 2; ++order) {
        const int count = order == 0 ? 21 : (order == 1 ? 48 : 2);
        double dC = 0.0, dS = 0.0;
        for (int i = 0; i < count; ++i) {
            const PhopFreqTerm term = freqTerm(order, i);
            double arg = 0.0;
            for (int j = 0; j < 5; ++j) arg += term.multiplier[j] * args[j];
            const double phase = order * (thetaG + kPi) - arg;
            const double c = cos(phase), s = sin(phase);
            if (order == 0) {
                dC += 1e-12 * (term.inPhase * c - term.outPhase * s);
            } else if (order == 1) {
                dC += 1e-12 * (term.inPhase * s + term.outPhase * c);
                dS += 1e-12 * (term.inPhase * c - term.outPhase * s);
            } else {
                dC += 1e-12 * term.inPhase * c;
                dS -= 1e-12 * term.inPhase * s;
            }
        }
        out.C[2][order] += dC;
        out.S[2][order] += dS;
    }
    // permanent deformation (IERS 6.13), removed for a zero-tide field
    const double permanent = 4.4228e-8 * (-0.31460) * 0.30190;
    if (zeroTide) out.C[2][0] -= permanent;
    // solid pole tide (IERS 6.22)
    double m1, m2;
    poleWobble(in, m1, m2);
    out.C[2][1] += -1.333e-9 * (m1 + 0.0115 * m2);
    out.S[2][1] += -1.333e-9 * (m2 - 0.0115 * m1);
}

// FES2004 ocean tide (degree/order <= 6) plus the degree-2 ocean pole tide
PHOP_HD void ocean(const Epoch& in, Coeffs& out) {
    clear(out);
    double f[5], gmst;
    arguments(in, f, gmst);
    const double s = f[2] + f[4], h = s - f[3];
    const double beta[6] = {gmst + kPi - s, s, h, s - f[0], -f[4], h - f[1]};
    for (int w = 0; w < 18; ++w) {
        const PhopOceanWave wave = TIDET(tide_fes_waves)[w];
        double theta = 0.0;
        for (int j = 0; j < 6; ++j) theta += wave.doodson[j] * beta[j];
        const double co = cos(theta), si = sin(theta);
        for (int i = wave.begin; i < wave.end; ++i) {
            const PhopOceanTerm t = TIDET(tide_fes_terms)[i];
            out.C[t.n][t.m] += (t.cp + t.cm) * co + (t.sp + t.sm) * si;
            if (t.m) out.S[t.n][t.m] += (t.sp - t.sm) * co - (t.cp - t.cm) * si;
        }
    }
    double m1, m2;
    poleWobble(in, m1, m2);
    out.C[2][1] += -2.1778e-10 * (m1 - 0.01724 * m2);
    out.S[2][1] += -1.7232e-10 * (m2 - 0.03365 * m1);
}

}  // namespace tides
}  // namespace phop
