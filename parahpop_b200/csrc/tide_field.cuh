// Time-variable geopotential from Earth tides: the corrections dC_nm, dS_nm
// (n <= 6, fully normalised) that the tides add to the static field at one
// epoch.  Written from the IERS Conventions 2010 (Petit & Luzum, IERS TN 36),
// chapter 6:
//
//   solid tide, step 1   eq. (6.6) degrees 2 and 3 with the anelastic Love
//                        numbers of Table 6.3, eq. (6.7) the degree-4
//                        response to the degree-2 tide
//   solid tide, step 2   eqs. (6.8a-c), frequency-dependent corrections,
//                        Tables 6.5a-c (units 1e-12)
//   permanent tide       eq. (6.13), removed from C20 for a zero-tide field
//   ocean tide           eq. (6.15), FES2004: 18 waves, degree/order <= 6
//   pole tides           eqs. (6.22) solid, (6.24) ocean, about the IERS 2010
//                        mean pole (eq. 7.25)
//   arguments            Delaunay arguments eq. (5.43), GMST eq. (5.32) from
//                        the Earth rotation angle eq. (5.15); Doodson
//                        variables from the Delaunay ones (Table 6.4 note)
//
// The numbers of Tables 6.5a-c and of the FES2004 model come from the
// generated tables/tide_tables.inc.  The model constants (GM, radius, the
// Sun and Moon GM, the speed of light) are those of the ParaHPOP tide model
// (src/common/engine/paraHPOP/model/accelerations/hpop_compat/
// HpopCorrections.h:25-31), so the corrections match the reference's.
//
// Structure (this package's own):
//   * The tide-raising potential of the Sun and Moon (6.6) is formed from
//     closed-form complex solid harmonics of their body-fixed unit vectors:
//     with t = z/r and w = (x - iy)/r = cos(phi) e^{-i lambda},
//     P_nm(sin phi) e^{-i m lambda} = N_nm (d^m P_n / dt^m)(t) w^m, so no
//     latitude, longitude or Legendre recursion is evaluated.
//   * Each Table 6.5 term's phasor e^{i theta_f} is a product of integer
//     powers of the five Delaunay phasors e^{i F_j} and of e^{i(theta_g+pi)}
//     (one sine/cosine pair per argument per epoch instead of one per term).
//   * The FES2004 amplitudes are held slot-major ("dense": wave x (n, m)
//     slot, already combined as C+ + C-, S+ + S-, S+ - S-, C+ - C-), so that
//     one lane of a warp owns each output coefficient and sums it over the
//     18 waves without any reduction.
//   * On the device one warp forms one epoch's corrections (tideDeltasWarp):
//     the 71 frequency terms are split across the lanes and folded by xor
//     shuffles, lanes 0-17 each evaluate one wave's Doodson phasor, and lane
//     s < 25 assembles slot s.  The host form (tideDeltasHost) runs the same
//     pieces one after the other; it backs the CPU check of this header
//     against the reference's known answers.
#pragma once
#include <math.h>

#if defined(__CUDACC__)
#define PHOP_TF_HD __host__ __device__ __forceinline__
#else
#define PHOP_TF_HD inline
#endif

namespace phop {
namespace tidefield {

// ---- generated tables (numbers of IERS Tables 6.5a-c and FES2004) -----------------------------
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
#define PHOP_TF_TABLE(name) dev_##name
#else
#define PHOP_TF_TABLE(name) host_##name
#endif

// ---- constants ---------------------------------------------------------------------------------
constexpr double kMuEarth = 398600.4415e9;                        // m^3/s^2
constexpr double kRadius = 6378.1363e3;                           // m
constexpr double kMuSun = 132712440041.279419e9;
constexpr double kMuMoon = 398600.4415e9 / 81.3005682214972154;
constexpr double kLight = 299792457.999999984;                    // m/s
constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kTwoPi = 2.0 * kPi;
constexpr double kArcsecToRad = kPi / 648000.0;

constexpr int kFreqTerms = 71;   // Tables 6.5b (21 zonal), 6.5a (48 diurnal), 6.5c (2 semidiurnal)
constexpr int kWaves = 18;       // FES2004 waves
constexpr int kSlots = 25;       // (n, m) for 2 <= n <= 6, 0 <= m <= n; slot s is triangle index s + 3

// ---- epoch inputs and the slot-major ocean table ------------------------------------------------
struct Epoch {
    double E[9];              // ICRF -> ITRF rotation, row-major
    double sun[3], moon[3];   // geocentric ICRF positions, m
    double mjdUtc, ut1Utc, ttUtc;  // UTC MJD; UT1 - UTC and TT - UTC, s
    double xp, yp;            // pole coordinates, arcsec
};

struct OceanAmp {
    double sumC, sumS;   // C+ + C-, S+ + S-    (dC = sumC cos + sumS sin)
    double difS, difC;   // S+ - S-, C+ - C-    (dS = difS cos - difC sin)
};

PHOP_TF_HD void slotDegreeOrder(int s, int& n, int& m) {
    n = 2;
    while (s > n) {
        s -= n + 1;
        ++n;
    }
    m = s;
}

// Slot-major FES2004 amplitudes: out[w * kSlots + s] (host).
inline void buildOceanTable(OceanAmp out[kWaves * kSlots]) {
    for (int k = 0; k < kWaves * kSlots; ++k) out[k] = OceanAmp{0.0, 0.0, 0.0, 0.0};
    for (int w = 0; w < kWaves; ++w) {
        const PhopOceanWave wave = host_tide_fes_waves[w];
        for (int i = wave.begin; i < wave.end; ++i) {
            const PhopOceanTerm t = host_tide_fes_terms[i];
            const int s = t.n * (t.n + 1) / 2 + t.m - 3;
            OceanAmp& a = out[w * kSlots + s];
            a.sumC += t.cp + t.cm;
            a.sumS += t.sp + t.sm;
            if (t.m) {  // the S coefficient of a zonal term does not exist
                a.difS += t.sp - t.sm;
                a.difC += t.cp - t.cm;
            }
        }
    }
}

// ---- small complex helpers ---------------------------------------------------------------------
struct Cx {
    double re, im;
};
PHOP_TF_HD Cx cmul(Cx a, Cx b) { return Cx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
PHOP_TF_HD Cx cscale(Cx a, double f) { return Cx{a.re * f, a.im * f}; }
PHOP_TF_HD Cx cadd(Cx a, Cx b) { return Cx{a.re + b.re, a.im + b.im}; }
PHOP_TF_HD Cx cexpi(double x) { return Cx{cos(x), sin(x)}; }
// z^k for an integer -2 <= k <= 2 given z and z^2 (unit z: the inverse is the conjugate)
PHOP_TF_HD Cx cpow2(Cx z, Cx z2, int k) {
    const Cx p = (k == 1 || k == -1) ? z : (k == 0 ? Cx{1.0, 0.0} : z2);
    return k < 0 ? Cx{p.re, -p.im} : p;
}

PHOP_TF_HD double wrapPeriod(double x, double period) {
    const double r = fmod(x, period);
    return r < 0.0 ? r + period : r;
}

// ---- astronomical arguments ------------------------------------------------------------------
// Delaunay arguments l, l', F, D, Omega (rad), IERS (5.43): polynomials in
// Julian centuries of TT since J2000, coefficients in arcseconds.
PHOP_TF_HD void delaunay(double mjdTt, double F[5]) {
    const double t = (mjdTt - 51544.5) / 36525.0;
    const double c[5][5] = {{485868.249036, 1717915923.2178, 31.8792, 0.051635, -0.00024470},
                            {1287104.79305, 129596581.0481, -0.5532, 0.000136, -0.00001149},
                            {335779.526232, 1739527262.8478, -12.7512, -0.001037, 0.00000417},
                            {1072260.70369, 1602961601.2090, -6.3706, 0.006593, -0.00003169},
                            {450160.398036, -6962890.5431, 7.4722, 0.007702, -0.00005939}};
    for (int j = 0; j < 5; ++j) {
        const double arcsec = c[j][0] + t * (c[j][1] + t * (c[j][2] + t * (c[j][3] + t * c[j][4])));
        F[j] = wrapPeriod(arcsec, 1296000.0) * kArcsecToRad;
    }
}

// Greenwich mean sidereal time (rad), IERS (5.32): the Earth rotation angle
// (5.15) of UT1 plus the precession polynomial in TT centuries.
PHOP_TF_HD double gmst(double mjdUt1, double mjdTt) {
    const double du = mjdUt1 - 51544.5;  // days of UT1 since J2000
    const double era = kTwoPi * (fmod(du, 1.0) + 0.7790572732640 + 0.00273781191135448 * du);
    const double t = (mjdTt - 51544.5) / 36525.0;
    const double poly =
        0.014506 + t * (4612.156534 + t * (1.3915817 + t * (-0.00000044 + t * (-0.000029956 + t * -0.0000000368))));
    return wrapPeriod(era + poly * kArcsecToRad, kTwoPi);
}

struct Arguments {
    double F[5];    // Delaunay arguments
    double theta;   // GMST
};

PHOP_TF_HD Arguments arguments(const Epoch& ep) {
    Arguments a;
    const double mjdTt = ep.mjdUtc + ep.ttUtc / 86400.0;
    delaunay(mjdTt, a.F);
    a.theta = gmst(ep.mjdUtc + ep.ut1Utc / 86400.0, mjdTt);
    return a;
}

// Doodson argument of FES wave w from the Delaunay arguments: variables
// (tau, s, h, p, N', p_s) with s = F + Omega, h = s - D, p = s - l,
// N' = -Omega, p_s = s - D - l', tau = theta_g + pi - s.
PHOP_TF_HD Cx wavePhasor(int w, const Arguments& a) {
    const double s = a.F[2] + a.F[4];
    const double h = s - a.F[3];
    const double beta[6] = {a.theta + kPi - s, s, h, s - a.F[0], -a.F[4], h - a.F[1]};
    const PhopOceanWave wave = PHOP_TF_TABLE(tide_fes_waves)[w];
    double x = 0.0;
    for (int k = 0; k < 6; ++k) x += wave.doodson[k] * beta[k];
    return cexpi(x);
}

// ---- solid tide: Sun and Moon potential -------------------------------------------------------
// H_nm = sum over Sun, Moon of (GM_j/GM_E) (R/r_j)^(n+1) P_nm(sin phi_j)
// e^{-i m lambda_j}, n = 2 (m = 0..2) and n = 3 (m = 0..3), body-fixed.
struct Raising {
    Cx h2[3], h3[4];
};

PHOP_TF_HD void addBody(const double E[9], const double pos[3], double gmRatio, Raising& out) {
    double b[3];
    for (int i = 0; i < 3; ++i) b[i] = E[3 * i] * pos[0] + E[3 * i + 1] * pos[1] + E[3 * i + 2] * pos[2];
    const double r = sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
    const double inv = 1.0 / r;
    const double t = b[2] * inv;
    const Cx w{b[0] * inv, -b[1] * inv};
    const Cx w2 = cmul(w, w), w3 = cmul(w2, w);
    const double rho = kRadius * inv;
    const double f2 = gmRatio * rho * rho * rho, f3 = f2 * rho;
    // normalised N_nm (d^m P_n/dt^m): n = 2
    const double s5 = 2.23606797749978969640, s15 = 3.87298334620741688518;
    out.h2[0].re += f2 * (0.5 * s5 * (3.0 * t * t - 1.0));
    out.h2[1] = cadd(out.h2[1], cscale(w, f2 * s15 * t));
    out.h2[2] = cadd(out.h2[2], cscale(w2, f2 * 0.5 * s15));
    // n = 3: sqrt(7)/2 (5t^3 - 3t), sqrt(21/8)(5t^2 - 1), sqrt(105/4) t, sqrt(35/8)
    const double s7 = 2.64575131106459059050;
    out.h3[0].re += f3 * (0.5 * s7 * t * (5.0 * t * t - 3.0));
    out.h3[1] = cadd(out.h3[1], cscale(w, f3 * 1.62018517460196461570 * (5.0 * t * t - 1.0)));
    out.h3[2] = cadd(out.h3[2], cscale(w2, f3 * 5.12347538297980212014 * t));
    out.h3[3] = cadd(out.h3[3], cscale(w3, f3 * 2.09165006633518887180));
}

PHOP_TF_HD Raising raising(const Epoch& ep) {
    Raising r;
    for (int m = 0; m < 3; ++m) r.h2[m] = Cx{0.0, 0.0};
    for (int m = 0; m < 4; ++m) r.h3[m] = Cx{0.0, 0.0};
    addBody(ep.E, ep.moon, kMuMoon / kMuEarth, r);
    addBody(ep.E, ep.sun, kMuSun / kMuEarth, r);
    return r;
}

// Step-1 correction of slot (n, m): dC - i dS = k_nm / (2n+1) H_nm (6.6),
// degree 4 from the degree-2 potential with k+_nm (6.7); Table 6.3.
PHOP_TF_HD void step1(const Raising& h, int n, int m, double& dC, double& dS) {
    double kR = 0.0, kI = 0.0;
    Cx H{0.0, 0.0};
    if (n == 2) {
        const double re[3] = {0.30190, 0.29830, 0.30102}, im[3] = {0.0, -0.00144, -0.00130};
        kR = re[m] / 5.0;
        kI = im[m] / 5.0;
        H = h.h2[m];
    } else if (n == 3) {
        kR = (m == 3 ? 0.094 : 0.093) / 7.0;
        H = h.h3[m];
    } else if (n == 4 && m <= 2) {
        const double plus[3] = {-0.00089, -0.00080, -0.00057};
        kR = plus[m] / 5.0;
        H = h.h2[m];
    }
    dC = kR * H.re - kI * H.im;
    dS = -(kR * H.im + kI * H.re);
}

// ---- solid tide step 2: frequency-dependent corrections --------------------------------------
// Phasors shared by the 71 terms of one epoch.
struct FreqPhasors {
    Cx z[5], z2[5];   // e^{i F_j}, e^{2i F_j}
    Cx g1, g2;        // e^{i(theta_g + pi)}, e^{2i(theta_g + pi)}
};

PHOP_TF_HD FreqPhasors freqPhasors(const Arguments& a) {
    FreqPhasors p;
    for (int j = 0; j < 5; ++j) {
        p.z[j] = cexpi(a.F[j]);
        p.z2[j] = cmul(p.z[j], p.z[j]);
    }
    p.g1 = cexpi(a.theta + kPi);
    p.g2 = cmul(p.g1, p.g1);
    return p;
}

// Adds term i (0-20: Table 6.5b, order 0; 21-68: 6.5a, order 1; 69-70:
// 6.5c, order 2) into acc = {dC20, dC21, dS21, dC22, dS22} (units 1e-12):
// theta_f = m (theta_g + pi) - N.F, (6.8a-c).
PHOP_TF_HD void addFreqTerm(int i, const FreqPhasors& p, double acc[5]) {
    const int order = i < 21 ? 0 : (i < 69 ? 1 : 2);
    const PhopFreqTerm term = order == 0 ? PHOP_TF_TABLE(tide_freq0)[i]
                                         : (order == 1 ? PHOP_TF_TABLE(tide_freq1)[i - 21] : PHOP_TF_TABLE(tide_freq2)[i - 69]);
    Cx e = order == 0 ? Cx{1.0, 0.0} : (order == 1 ? p.g1 : p.g2);
    for (int j = 0; j < 5; ++j) e = cmul(e, cpow2(p.z[j], p.z2[j], -term.multiplier[j]));
    const double ip = term.inPhase, op = term.outPhase;
    if (order == 0) {
        acc[0] += ip * e.re - op * e.im;
    } else if (order == 1) {
        acc[1] += ip * e.im + op * e.re;
        acc[2] += ip * e.re - op * e.im;
    } else {
        acc[3] += ip * e.re;
        acc[4] -= ip * e.im;
    }
}

// ---- pole tides ---------------------------------------------------------------------------------
// Wobble (m1, m2) of the pole about the IERS 2010 mean pole (arcsec).
PHOP_TF_HD void wobble(const Epoch& ep, double& m1, double& m2) {
    const double y = (ep.mjdUtc + ep.ttUtc / 86400.0 - 51544.5) / 365.25;  // years since 2000.0
    double xm, ym;                                                         // mas
    if (y < 10.0) {
        xm = 55.974 + y * (1.8243 + y * (0.18413 + y * 0.007024));
        ym = 346.346 + y * (1.7896 + y * (-0.10729 + y * -0.000908));
    } else {
        xm = 23.513 + 7.6141 * y;
        ym = 358.891 - 0.6287 * y;
    }
    m1 = ep.xp - xm * 1e-3;
    m2 = -(ep.yp - ym * 1e-3);
}

// ---- one slot --------------------------------------------------------------------------------
struct SlotInputs {
    Raising h;
    double freq[5];   // step-2 sums, units 1e-12
    double m1, m2;    // pole wobble
    Cx wave[kWaves];  // Doodson phasors (host form; the device passes them by shuffle)
};

// Solid-tide part of slot (n, m): steps 1 and 2, permanent tide, pole tide.
PHOP_TF_HD void solidSlot(const SlotInputs& in, int n, int m, bool zeroTide, double& dC, double& dS) {
    if (n > 4) {
        dC = dS = 0.0;
        return;
    }
    step1(in.h, n, m, dC, dS);
    if (n == 2) {
        if (m == 0) {
            dC += 1e-12 * in.freq[0];
            if (zeroTide) dC -= 4.4228e-8 * (-0.31460) * 0.30190;  // (6.13): A0 H0 k20
        } else if (m == 1) {
            dC += 1e-12 * in.freq[1] - 1.333e-9 * (in.m1 + 0.0115 * in.m2);
            dS += 1e-12 * in.freq[2] - 1.333e-9 * (in.m2 - 0.0115 * in.m1);
        } else {
            dC += 1e-12 * in.freq[3];
            dS += 1e-12 * in.freq[4];
        }
    }
}

// Ocean part of slot s over waves [w0, w1) with the given phasors.
PHOP_TF_HD void oceanWave(const OceanAmp* table, int s, int w, Cx ph, double& dC, double& dS) {
    const OceanAmp a = table[w * kSlots + s];
    dC += a.sumC * ph.re + a.sumS * ph.im;
    dS += a.difS * ph.re - a.difC * ph.im;
}

PHOP_TF_HD void oceanPole(const SlotInputs& in, double& dC21, double& dS21) {
    dC21 += -2.1778e-10 * (in.m1 - 0.01724 * in.m2);
    dS21 += -1.7232e-10 * (in.m2 - 0.03365 * in.m1);
}

// ---- host form -------------------------------------------------------------------------------
// Separate solid and ocean sets, C[n][m], S[n][m] for n <= 6 (zero rows
// below degree 2): the pieces of tideDeltasWarp run one after the other.
inline void tideSetsHost(const Epoch& ep, bool zeroTide, const OceanAmp* table, double solidC[7][7],
                         double solidS[7][7], double oceanC[7][7], double oceanS[7][7]) {
    SlotInputs in;
    in.h = raising(ep);
    const Arguments a = arguments(ep);
    const FreqPhasors fp = freqPhasors(a);
    for (int k = 0; k < 5; ++k) in.freq[k] = 0.0;
    for (int i = 0; i < kFreqTerms; ++i) addFreqTerm(i, fp, in.freq);
    wobble(ep, in.m1, in.m2);
    for (int w = 0; w < kWaves; ++w) in.wave[w] = wavePhasor(w, a);
    for (int n = 0; n < 7; ++n)
        for (int m = 0; m < 7; ++m) solidC[n][m] = solidS[n][m] = oceanC[n][m] = oceanS[n][m] = 0.0;
    for (int s = 0; s < kSlots; ++s) {
        int n, m;
        slotDegreeOrder(s, n, m);
        solidSlot(in, n, m, zeroTide, solidC[n][m], solidS[n][m]);
        double c = 0.0, d = 0.0;
        for (int w = 0; w < kWaves; ++w) oceanWave(table, s, w, in.wave[w], c, d);
        if (n == 2 && m == 1) oceanPole(in, c, d);
        oceanC[n][m] = c;
        oceanS[n][m] = d;
    }
}

#if defined(__CUDACC__)
// ---- device form: one warp per epoch ---------------------------------------------------------
// Every lane passes the same epoch; lane s < kSlots returns slot s's total
// correction (solid and / or ocean, scaled by scale[n]) in dC, dS; other
// lanes return zeros.  All 32 lanes of the warp must call it together.
__device__ __forceinline__ void tideDeltasWarp(const Epoch& ep, bool solid, bool ocean, bool zeroTide,
                                               const OceanAmp* __restrict__ table, const double scale[7], double& dC,
                                               double& dS) {
    const int lane = threadIdx.x & 31;
    const Arguments a = arguments(ep);
    SlotInputs in;
    wobble(ep, in.m1, in.m2);
    for (int k = 0; k < 5; ++k) in.freq[k] = 0.0;
    if (solid) {
        in.h = raising(ep);
        const FreqPhasors fp = freqPhasors(a);
        for (int i = lane; i < kFreqTerms; i += 32) addFreqTerm(i, fp, in.freq);
#pragma unroll
        for (int k = 0; k < 5; ++k)
            for (int off = 16; off > 0; off >>= 1) in.freq[k] += __shfl_xor_sync(0xffffffffu, in.freq[k], off);
    }
    Cx mine{0.0, 0.0};
    if (ocean && lane < kWaves) mine = wavePhasor(lane, a);
    dC = dS = 0.0;
    const int s = lane < kSlots ? lane : 0;
    int n, m;
    slotDegreeOrder(s, n, m);
    double oc = 0.0, os = 0.0;
    if (ocean) {
        for (int w = 0; w < kWaves; ++w) {
            const Cx ph{__shfl_sync(0xffffffffu, mine.re, w), __shfl_sync(0xffffffffu, mine.im, w)};
            oceanWave(table, s, w, ph, oc, os);
        }
        if (n == 2 && m == 1) oceanPole(in, oc, os);
    }
    if (lane >= kSlots) return;
    double sc = 0.0, ss = 0.0;
    if (solid) solidSlot(in, n, m, zeroTide, sc, ss);
    // the reference sums the solid and the ocean set per coefficient
    dC = (sc + oc) * scale[n];
    dS = (ss + os) * scale[n];
}
#endif

}  // namespace tidefield
}  // namespace phop
