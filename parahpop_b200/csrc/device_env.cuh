// Device-resident environment and the per-epoch environment record.
//
// Everything the force model needs that depends on the epoch only (third-body
// positions, the ICRF -> ITRF rotation and its rate, tide coefficient sets,
// the time and space-weather inputs of NRLMSISE-00) is evaluated once per
// stage epoch into an EpochRecord.  Batches whose objects share one time grid
// evaluate the records ahead of the step kernel (one per step and stage);
// mixed batches (per-object time) interpolate them in time from a grid of
// records at 30 s spacing.
//
// Reference behaviour restated (paths relative to the reference tree):
//   Chebyshev ephemeris    third_party/parm/parm/interpolate/chebyshev/Interpolator.h:71-86,
//                          detail/Interpolators.h:65-75, brie/core/Type2BodyUnit.h:47-60
//   IERS2000 rotation      third_party/brie/brie/orientations/detail/IERS2000Model.h:56-215,526-555,
//                          LagrangeInterp.h:88-130, parm/interpolate/lagrange/Interpolator.h:61-104,416-432,812-833
//   EOP time + tides       src/common/engine/paraHPOP/model/environment/earthcorrections/EarthCorrections.h:46-105,
//                          model/accelerations/EarthCorrections.h:8-90
//   NRLMSISE epoch inputs  src/common/engine/paraHPOP/model/environment/atmosphere/Nrlmsise00.cu:83-235
#pragma once
#include <math.h>
#include <stdint.h>
#include <stddef.h>

#include "nrl_fast.cuh"
#include "tide_field.cuh"

namespace phop {

constexpr int kMaxBodies = 12;
constexpr int kMaxChain = 4;
constexpr int kMaxPoles = 1;  // bodies other than the Earth with the J2 model or an atmosphere
constexpr int kTideTri = 28;  // n <= 6 triangle, index n(n+1)/2 + m

constexpr int kMaxExpBands = 16;

enum BodyFlag : int { kGravity = 1, kShape = 2, kRadiation = 4, kAtmosphere = 8, kOcculting = 16, kOblateness = 32 };

struct DevEnv {
    // geopotential (normalised), triangle n(n+1)/2+m, device pointers
    int shDegree, shOrder, shNormalized;
    double shR, shGM;
    double tideScale[7];  // converts tide-model dC/dS (SI constants) to the field's GM and radius
    const double* shC;
    const double* shS;
    const double* shFac;  // interleaved (a_nm | c_m, b_nm)
    // bodies, sorted by NAIF id (Bodies.h:105-120)
    int nbodies;
    int bodyId[kMaxBodies];
    int bodyFlags[kMaxBodies];
    double bodyGm[kMaxBodies];
    double bodyRadius[kMaxBodies];
    int chainPlus[kMaxBodies][kMaxChain];   // ephemeris units summed (-1 = none)
    int chainMinus[kMaxBodies][kMaxChain];  // ephemeris units subtracted
    int sunIndex, moonIndex, earthIndex;    // body slots (-1 when absent)
    int sunUnitsPlus[kMaxChain], sunUnitsMinus[kMaxChain];
    int moonUnitsPlus[kMaxChain], moonUnitsMinus[kMaxChain];
    double flattening, au, earthRadius;
    int anyOcculter;
    // oblateness (J2) model: constants-file J2, GM and sphere of influence
    double bodyJ2[kMaxBodies], bodyGmConst[kMaxBodies], bodySoi[kMaxBodies];
    // exponential atmosphere (when no NRLMSISE-00): bands ascending in h0,
    // each {rho0 (kg/km^3), h0, scaleHeight, hCutoff (km)}
    int nExp;
    double expSeg[kMaxExpBands][4];
    // Type-2 Chebyshev units
    int neph;
    const int* ephNint;
    const int* ephPdeg;
    const int64_t* ephOffset;
    const double* ephData;
    // IERS2000 orientation unit
    int hasRot, rotNnut, rotNerp;
    int rotKind, rotNint, rotPdeg, rotEcliptic;  // 4: IERS2000 model unit; 3: binary Chebyshev Euler angles;
                                                 // 1: IAU body model
    int iauDeg[3], iauNp[3];                     // kind 1: RA, Dec, PM coefficient and amplitude counts
    int iauBaryOffset, iauNpDeg, iauNpAngles;    // kind 1: barycentric angle polynomials in rotData (-1: none)
    const double* rotData;
    // NRLMSISE-00 weather
    int hasNrl, nrlNdays;
    double nrlStartMjd, nrlHcutoff, nrlDensityScale;
    const double* nrlWeather;  // 13 x ndays component-major
    const nrlf::NrlEpochBlock* nrlBlocks;  // per (UTC day record, 3-hour ap slot): index record * 8 + slot
    // Earth corrections
    int solid, ocean, relativity, zeroTide;
    int tidesAlone;  // tides on without a gravity field: the deltas are summed on their own (degree <= 6)
    const tidefield::OceanAmp* tideOcean;  // FES2004 amplitudes, slot-major (tide_field.cuh)
    int eopN;
    double eopFirstMjd;
    const double* eop;  // 4 x n component-major
    // bodies other than the Earth with the J2 model: each body's record
    // slot for its polar axis (-1: none) and its IAU body model (the
    // reference's default orientation target, the body's own NAIF id)
    int poleSlot[kMaxBodies];
    int nPoles;
    int poleDeg[kMaxPoles][3], poleNp[kMaxPoles][3];
    int poleData[kMaxPoles];    // offset of the model's coefficients in poleCoef
    int poleBary[kMaxPoles];    // offset of its barycentric angle polynomials from there (-1: none)
    int poleNpDeg[kMaxPoles];
    const double* poleCoef;
    // a field on a body other than the Earth (shFrame = 1): the IAU body
    // model of its frame (coefficients at poleCoef + shFrameData); shTides:
    // the Earth's tide deltas join the field (the field is the Earth's)
    int shFrame, shTides;
    int shFrameDeg[3], shFrameNp[3];
    int shFrameData, shFrameBary, shFrameNpDeg;
    // the exponential atmosphere on a body other than the Earth: its body
    // index (-1: none; its pole slot gives axis, rate and velocity) and flattening
    int atmBody;
    double atmFlattening;
};

struct EpochRecord {
    double R[9];                 // ICRF -> ITRF
    double w[3];                 // Earth angular velocity, inertial, rad/s
    double body[kMaxBodies][3];  // body positions relative to the Earth, km
    double indirect[3];          // sum over third bodies of -gm rb / |rb|^3 (km/s^2): epoch-only
    double dC[kTideTri];         // tide coefficient deltas, field units
    double dS[kTideTri];
    double pole[kMaxPoles][3];   // polar (body z) axes of the J2 bodies other than the Earth, inertial
    double poleW[kMaxPoles][3];  // their angular velocities, inertial, rad/s
    double poleV[kMaxPoles][3];  // their velocities relative to the Earth, km/s
    double fieldR[9];            // ICRF -> body rotation of a field on a body other than the Earth
    double nrlSec, nrlGast;      // UTC seconds of day, apparent sidereal time (h)
    double et;                   // the record's epoch, TDB seconds past J2000
    int nrlBlock, nrlValid;      // nrlValid: 1 / 0, or -1 = time inputs not evaluated yet (from et)
    int tideValid, pad;
};
// Fields 0 .. kInterpFields - 1 of a record (rotation to tide deltas) are the
// ones the per-object-time force model interpolates in time.
constexpr int kInterpFields = (int)(offsetof(EpochRecord, nrlSec) / sizeof(double));

// NRLMSISE-00 time inputs of one epoch
struct NrlTime {
    double sec, gast;
    int block, valid;
};

#if defined(__CUDACC__)
// ---- time ---------------------------------------------------------------------
static __host__ __device__ __forceinline__ double mjdToEt(double mjd) { return fma(mjd, 86400.0, -43200.0); }
static __host__ __device__ __forceinline__ double etToMjd(double et) { return fma(et, 1.0 / 86400.0, 0.5); }

// ---- Chebyshev ephemeris (Clenshaw) --------------------------------------------------
static __device__ __forceinline__ void chebPosition(const DevEnv& e, int u, double t, double out[3]) {
    const double* d = e.ephData + e.ephOffset[u];
    const int n = e.ephNint[u], deg = e.ephPdeg[u];
    const double r = d[0];
    const double* starts = d + 1;
    const double* cf = d + 1 + n;
    long idx = (long)((t - starts[0]) / (2 * r));
    idx = idx < 0 ? 0 : (idx >= n ? n - 1 : idx);
    const double s = (t - starts[idx]) / r - 1.0;
    const double s2 = 2 * s;
    for (int dim = 0; dim < 3; ++dim) {
        const double* c = cf + (int64_t)dim * (deg + 1) * n;
        double w = 0, x = 0;
        for (int i = 0; i < deg; ++i) {
            w = c[idx + (int64_t)(deg - i) * n] - w;
            const double nx = fma(s2, x, w);
            w = x;
            x = nx;
        }
        out[dim] = fma(s, x, c[idx] - w);
    }
}

// velocity (km/s) of a Chebyshev unit: the derivative of its series
static __device__ __forceinline__ void chebVelocity(const DevEnv& e, int u, double t, double out[3]) {
    const double* d = e.ephData + e.ephOffset[u];
    const int n = e.ephNint[u], deg = e.ephPdeg[u];
    const double r = d[0];
    const double* starts = d + 1;
    const double* cf = d + 1 + n;
    long idx = (long)((t - starts[0]) / (2 * r));
    idx = idx < 0 ? 0 : (idx >= n ? n - 1 : idx);
    const double s = (t - starts[idx]) / r - 1.0;
    const double s2 = 2 * s;
    for (int dim = 0; dim < 3; ++dim) {
        const double* c = cf + (int64_t)dim * (deg + 1) * n;
        double w = 0, x = 0, dw = 0, v = 0;
        for (int i = 0; i < deg; ++i) {
            w = c[idx + (int64_t)(deg - i) * n] - w;
            const double nx = fma(s2, x, w);
            w = x;
            x = nx;
            const double nv = fma(s2, v, fma(2.0, w, -dw));
            dw = v;
            v = nv;
        }
        out[dim] = (1.0 / r) * fma(s, v, x - dw);
    }
}

static __device__ __forceinline__ void chainVelocity(const DevEnv& e, const int* plus, const int* minus, double t,
                                                     double out[3]) {
    out[0] = out[1] = out[2] = 0.0;
    double p[3];
    for (int k = 0; k < kMaxChain && plus[k] >= 0; ++k) {
        chebVelocity(e, plus[k], t, p);
        out[0] += p[0]; out[1] += p[1]; out[2] += p[2];
    }
    for (int k = 0; k < kMaxChain && minus[k] >= 0; ++k) {
        chebVelocity(e, minus[k], t, p);
        out[0] -= p[0]; out[1] -= p[1]; out[2] -= p[2];
    }
}

static __device__ __forceinline__ void chainPosition(const DevEnv& e, const int* plus, const int* minus, double t,
                                              double out[3]) {
    out[0] = out[1] = out[2] = 0.0;
    double p[3];
    for (int k = 0; k < kMaxChain && plus[k] >= 0; ++k) {
        chebPosition(e, plus[k], t, p);
        out[0] += p[0]; out[1] += p[1]; out[2] += p[2];
    }
    for (int k = 0; k < kMaxChain && minus[k] >= 0; ++k) {
        chebPosition(e, minus[k], t, p);
        out[0] -= p[0]; out[1] -= p[1]; out[2] -= p[2];
    }
}

// ---- Lagrange interpolation (product form, centred clamped stencil) ------------------------
template <int NPTS, int NCH>
static __device__ __forceinline__ void lagrangeEval(const double* ys, int stride, const double* keys, double x0, double h,
                                             int n, double t, bool uniform, double* val, double* der) {
    long lo;
    double q;
    constexpr long half = NPTS / 2;
    if (uniform) {
        const long f = (long)floor((t - x0) / h);
        lo = f - half + 1;
        lo = lo < 0 ? 0 : lo;
        lo = lo > n - NPTS ? n - NPTS : lo;
        q = (t - (x0 + (double)lo * h)) / h;
    } else {
        long a = 0, b = n;
        while (a < b) {
            const long mid = a + ((b - a) >> 1);
            if (keys[mid] <= t) a = mid + 1; else b = mid;
        }
        lo = a - 1 - half + 1;
        lo = lo < 0 ? 0 : lo;
        lo = lo > n - NPTS ? n - NPTS : lo;
        q = t;
    }
#pragma unroll
    for (int c = 0; c < NCH; ++c) val[c] = der[c] = 0.0;
#pragma unroll
    for (int j = 0; j < NPTS; ++j) {
        double prod = 1, dprod = 0, denom = 1;
#pragma unroll
        for (int m = 0; m < NPTS; ++m) {
            if (m == j) continue;
            double f, dfac;
            if (uniform) {
                f = q - (double)m;
                dfac = (double)(j - m);
            } else {
                f = q - keys[lo + m];
                dfac = keys[lo + j] - keys[lo + m];
            }
            dprod = fma(dprod, f, prod);
            prod *= f;
            denom *= dfac;
        }
        const double inv = 1.0 / denom;
        const double wv = prod * inv, wd = dprod * inv;
#pragma unroll
        for (int c = 0; c < NCH; ++c) {
            const double y = ys[(int64_t)c * stride + lo + j];
            val[c] = fma(wv, y, val[c]);
            der[c] = fma(wd, y, der[c]);
        }
    }
    if (uniform) {
#pragma unroll
        for (int c = 0; c < NCH; ++c) der[c] *= 1.0 / h;
    }
}

static __device__ __forceinline__ void mat3mul(double C[9], const double A[9], const double B[9]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}

// Rotation ICRF -> body from RA, Dec, PM (rad) and the inertial angular
// velocity from their rates: the passive Z-X-Z rotation with angles
// pi/2 + RA, pi/2 - Dec, PM (frames/Rotation.h:124-133), composed with the
// ICRF -> ECLIPJ2000 bias Rx(obliquity) for ecliptic-based angles, and the
// 3-1-3 Euler kinematics mapped back to ICRF (frames/Frames.h:57-166).
static __device__ void eulerBodyRotation(double ra, double dec, double pm, double raDot, double decDot, double pmDot,
                                         bool ecliptic, double R[9], double w[3]) {
    double s1, c1, sx, cx, s3, c3;
    sincos(M_PI / 2 + ra, &s1, &c1);
    sincos(M_PI / 2 - dec, &sx, &cx);
    sincos(pm, &s3, &c3);
    const double A[9] = {c3 * c1 - s3 * cx * s1, c3 * s1 + s3 * cx * c1, s3 * sx,
                         -s3 * c1 - c3 * cx * s1, -s3 * s1 + c3 * cx * c1, c3 * sx,
                         sx * s1, -sx * c1, cx};
    double sa, ca, sd, cd;
    sincos(ra, &sa, &ca);
    sincos(dec, &sd, &cd);
    double om[3] = {decDot * sa + pmDot * ca * cd, -decDot * ca + pmDot * sa * cd, raDot + pmDot * sd};
    if (ecliptic) {
        const double eps = 84381.448 / 3600.0 * (M_PI / 180.0);
        double se, ce;
        sincos(eps, &se, &ce);
        const double E[9] = {1, 0, 0, 0, ce, se, 0, -se, ce};  // ICRF -> ECLIPJ2000
        mat3mul(R, A, E);
        // omega_icrf = E^T omega_ecl
        const double o1 = ce * om[1] - se * om[2], o2 = se * om[1] + ce * om[2];
        om[1] = o1;
        om[2] = o2;
    } else {
        for (int k = 0; k < 9; ++k) R[k] = A[k];
    }
    w[0] = om[0];
    w[1] = om[1];
    w[2] = om[2];
}

// ICRF -> ITRF93 rotation and inertial angular velocity from a binary
// orientation unit: three Chebyshev angle series (v0, v1, v2) and their rates
// (the Type-2 evaluation of the ephemeris, parm chebyshev Interpolator.h),
// RA = v0 - pi/2, Dec = pi/2 - v1, PM = v2 mod 2 pi
// (orientations/RefEphUnit.h:769-790, rates :890-900 with the Dec sign
// flipped), the rotation Rz(PM) Rx(pi/2 - Dec) Rz(pi/2 + RA)
// (frames/Rotation.h:124-133), composed with the ICRF -> ECLIPJ2000 bias
// Rx(obliquity) for ecliptic-based units, and the body rate from the 3-1-3
// Euler kinematics mapped back to ICRF (frames/Frames.h:57-166).
static __device__ void binaryEarthRotation(const DevEnv& e, double t, double R[9], double w[3]) {
    const double* d = e.rotData;
    const int n = e.rotNint, deg = e.rotPdeg;
    const double r = d[0];
    const double* starts = d + 1;
    const double* cf = d + 1 + n;
    long idx = (long)((t - starts[0]) / (2 * r));
    idx = idx < 0 ? 0 : (idx >= n ? n - 1 : idx);
    const double s = (t - starts[idx]) / r - 1.0;
    const double s2 = 2 * s;
    double val[3], rate[3];
    for (int dim = 0; dim < 3; ++dim) {
        const double* c = cf + (int64_t)dim * (deg + 1) * n;
        double b1 = 0, b0 = 0, db1 = 0, db0 = 0;
        for (int i = 0; i < deg; ++i) {
            b1 = c[idx + (int64_t)(deg - i) * n] - b1;
            const double nb = fma(s2, b0, b1);
            b1 = b0;
            b0 = nb;
            const double nd = fma(s2, db0, fma(2.0, b1, -db1));
            db1 = db0;
            db0 = nd;
        }
        val[dim] = fma(s, b0, c[idx] - b1);
        rate[dim] = (1.0 / r) * fma(s, db0, b0 - db1);
    }
    const double ra = val[0] - M_PI / 2, dec = M_PI / 2 - val[1], pm = fmod(val[2], 2 * M_PI);
    eulerBodyRotation(ra, dec, pm, rate[0], -rate[1], rate[2], e.rotEcliptic != 0, R, w);
}

// IAU body model (orientations/RefEphUnit.h:100-330, 640-770,
// core/Polynomial.h:33-160, frames/Frames.h:224-290): RA, Dec polynomials in
// Julian centuries and PM in days of TDB (degrees, ascending coefficients),
// plus sum_i a_i sin(p_i(T)) (RA, PM) / a_i cos(p_i(T)) (Dec) over the
// body's barycentric angle polynomials p_i (degrees, centuries); the angles
// reduced mod 360, then the rotation and rate as for a binary unit.
static __device__ void iauRotation(const double* d, const int degs[3], const int nps[3], int baryOffset, int npDeg,
                                   double t, double R[9], double w[3]) {
    const double secToCenturies = 3155760000.0, secToDays = 86400.0, deg = M_PI / 180.0;
    const double T = t / secToCenturies, D = t / secToDays;
    auto horner = [](const double* c, int n, double x) {
        double r = 0.0;
        for (int i = 0; i < n; ++i) r = fma(r, x, c[n - 1 - i]);
        return r;
    };
    auto hornerRate = [](const double* c, int n, double x) {
        double r = 0.0;
        for (int i = 0; i + 1 < n; ++i) r = fma(r, x, c[n - 1 - i] * (double)(n - 1 - i));
        return r;
    };
    const int nRa = degs[0], nDec = degs[1], nPm = degs[2];
    double ang[3] = {horner(d, nRa, T), horner(d + nRa, nDec, T), horner(d + nRa + nDec, nPm, D)};
    double rate[3] = {hornerRate(d, nRa, T) / secToCenturies, hornerRate(d + nRa, nDec, T) / secToCenturies,
                      hornerRate(d + nRa + nDec, nPm, D) / secToDays};
    if (baryOffset >= 0) {
        const double* amp = d + nRa + nDec + nPm;
        const double* bary = d + baryOffset;
        for (int comp = 0; comp < 3; ++comp) {
            const bool isSin = comp != 1;
            double sum = 0.0, dsum = 0.0;
            for (int i = 0; i < nps[comp]; ++i) {
                const double* p = bary + (int64_t)i * npDeg;
                double v = 0.0, dv = 0.0, tp = 1.0;
                for (int j = 0; j < npDeg; ++j) {
                    v = fma(p[j], tp, v);
                    if (j + 1 < npDeg) dv = fma(p[j + 1] * (double)(j + 1), tp, dv);
                    tp *= T;
                }
                double sv, cv;
                sincos(v * deg, &sv, &cv);
                sum = fma(amp[i], isSin ? sv : cv, sum);
                dsum = fma(amp[i], (isSin ? cv : -sv) * dv * deg, dsum);
            }
            ang[comp] += sum;
            rate[comp] += dsum / secToCenturies;
            amp += nps[comp];
        }
    }
    eulerBodyRotation(fmod(ang[0], 360.0) * deg, fmod(ang[1], 360.0) * deg, fmod(ang[2], 360.0) * deg,
                      rate[0] * deg, rate[1] * deg, rate[2] * deg, false, R, w);
}


static __device__ void iauEarthRotation(const DevEnv& e, double t, double R[9], double w[3]) {
    iauRotation(e.rotData, e.iauDeg, e.iauNp, e.iauBaryOffset, e.iauNpDeg, t, R, w);
}

// ICRF -> ITRF rotation and inertial angular velocity of the IERS2000 unit
static __device__ void earthRotation(const DevEnv& e, double t, double R[9], double w[3]) {
    if (e.rotKind == 3) {
        binaryEarthRotation(e, t, R, w);
        return;
    }
    if (e.rotKind == 1) {
        iauEarthRotation(e, t, R, w);
        return;
    }
    const double inv = 1.0 / 86400.0;
    const double tdbMjd = t * inv + 0.5;
    const double g = (M_PI / 180.0) * (357.53 + 0.9856003 * (tdbMjd - 0.5));
    const double corr = (0.001658 * sin(g) + 0.000014 * sin(2.0 * g)) * inv;
    double frac = fmod(t, 86400.0) * inv + 0.5;
    frac -= floor(frac);
    const double dayFrac = frac - corr;
    const double ttMjd = tdbMjd - corr;
    const int nn = e.rotNnut, ne = e.rotNerp;
    const double* d = e.rotData;
    const double* cst = d + 3 * nn + 5 * ne;
    double nodes[8], rates[8];
    lagrangeEval<6, 3>(d, nn, nullptr, cst[0], cst[1], nn, ttMjd, true, nodes, rates);
    lagrangeEval<4, 5>(d + 3 * nn, ne, cst + 4, 0, 0, ne, ttMjd, false, nodes + 3, rates + 3);
    const double X = nodes[0] + nodes[6], Y = nodes[1] + nodes[7], s = nodes[2];
    const double Xd = rates[0] * inv + rates[6] * inv, Yd = rates[1] * inv + rates[7] * inv, sd = rates[2] * inv;
    const double r2 = X * X + Y * Y, rr = sqrt(r2), fr = 1.0 / sqrt(1.0 - r2);
    const double E = r2 > 0 ? atan2(Y, X) : 0.0;
    const double D = atan(rr * fr);
    const double Ed = r2 > 0 ? (Yd * X - Xd * Y) / r2 : 0.0;
    const double Dd = (X * Xd + Y * Yd) * fr / rr;
    const double ms = -E - s, msd = -Ed - sd;
    const double dut1 = nodes[5], dut1d = rates[5] * inv;
    const double ut1jd = ttMjd + dut1 - 0.5;
    const double f = fmod(dayFrac + dut1 - 0.5, 1.0);
    double theta = 2 * M_PI * (f + 0.7790572732640 + 0.00273781191135448 * ut1jd);
    theta = theta - 2 * M_PI * floor(theta / (2 * M_PI));
    const double thetad = 2 * M_PI * ((inv + dut1d) + 0.00273781191135448 * inv);
    const double sp = -6.24e-15 * (ttMjd - 0.5), spd = -7.2205e-20;
    const double xp = nodes[3], yp = nodes[4], xpd = rates[3] * inv, ypd = rates[4] * inv;
    double s1, c1, s2, c2, s3, c3;
    sincos(E, &s1, &c1);
    sincos(D, &s2, &c2);
    sincos(ms, &s3, &c3);
    const double PN[9] = {c1 * c2 * c3 - s1 * s3, c1 * s3 + s1 * c2 * c3, -c3 * s2, -s1 * c3 - c1 * c2 * s3,
                          c1 * c3 - s1 * c2 * s3, s2 * s3, s2 * c1, s2 * s1, c2};
    const double c1d = -s1 * Ed, s1d = c1 * Ed, c2d = -s2 * Dd, s2d = c2 * Dd, c3d = -s3 * msd, s3d = c3 * msd;
    const double c2s3 = c2 * s3, c2c3 = c2 * c3, c2s3d = c2d * s3 + c2 * s3d, c2c3d = c2d * c3 + c2 * c3d;
    const double PNd[9] = {-s1d * s3 - s1 * s3d + c1d * c2c3 + c1 * c2c3d, c1d * s3 + c1 * s3d + s1d * c2c3 + s1 * c2c3d,
                           -c3d * s2 - c3 * s2d, -s1d * c3 - s1 * c3d - c1d * c2s3 - c1 * c2s3d,
                           c1d * c3 + c1 * c3d - s1d * c2s3 - s1 * c2s3d, s2d * s3 + s2 * s3d, s2d * c1 + s2 * c1d,
                           s2d * s1 + s2 * s1d, c2d};
    double st, ct;
    sincos(theta, &st, &ct);
    const double ER[9] = {ct, st, 0, -st, ct, 0, 0, 0, 1};
    const double ERd[9] = {-st * thetad, ct * thetad, 0, -ct * thetad, -st * thetad, 0, 0, 0, 0};
    const double PM[9] = {1.0, sp, xp, -sp, 1.0, -yp, -xp, yp, 1.0};
    const double PMd[9] = {0.0, spd, xpd, -spd, 0.0, -ypd, -xpd, ypd, 0.0};
    double ERPN[9], a[9], t1[9], t2[9], t3[9], Rd[9];
    mat3mul(ERPN, ER, PN);
    mat3mul(R, PM, ERPN);
    mat3mul(a, ERd, PN);
    mat3mul(t1, PM, a);
    mat3mul(t2, PMd, ERPN);
    mat3mul(a, ER, PNd);
    mat3mul(t3, PM, a);
#pragma unroll
    for (int i = 0; i < 9; ++i) Rd[i] = t1[i] + t2[i] + t3[i];
    double M[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) M[3 * i + j] = Rd[i] * R[j] + Rd[3 + i] * R[3 + j] + Rd[6 + i] * R[6 + j];
    w[0] = 0.5 * (M[7] - M[5]);
    w[1] = 0.5 * (M[2] - M[6]);
    w[2] = 0.5 * (M[3] - M[1]);
}

// ---- EOP-based time for the tide model -------------------------------------------------------
static __device__ __forceinline__ double tdbMinusTt(double mjdTt) {
    const double t = (mjdTt - 51544.5) / 36525;
    return 0.001657 * sin(628.3076 * t + 6.2401) + 0.000022 * sin(575.3385 * t + 4.2970)
        + 0.000014 * sin(1256.6152 * t + 6.1969) + 0.000005 * sin(606.9777 * t + 4.0212)
        + 0.000005 * sin(52.9691 * t + 0.4444) + 0.000002 * sin(21.3299 * t + 5.5431)
        + 0.000010 * sin(628.3076 * t + 4.2490);
}

static __device__ bool eopTime(const DevEnv& e, double et, tidefield::Epoch& ep) {
    if (e.eopN < 2 || !isfinite(et)) return false;
    const double* xp = e.eop;
    const double* yp = e.eop + e.eopN;
    const double* dut = e.eop + 2 * e.eopN;
    const double* dat = e.eop + 3 * e.eopN;
    double ttEt = et;
    for (int j = 0; j < 2; ++j) ttEt = et - tdbMinusTt(51544.5 + ttEt / 86400);
    double utc = 51544.5 + (ttEt - 69.184) / 86400;
    for (int j = 0; j < 3; ++j) {
        double day = floor(utc - e.eopFirstMjd);
        day = day < 0 ? 0 : day;
        day = day > (double)(e.eopN - 1) ? (double)(e.eopN - 1) : day;
        utc = 51544.5 + (ttEt - 32.184 - dat[(int)day]) / 86400;
    }
    if (!(utc >= e.eopFirstMjd) || !(utc < e.eopFirstMjd + (double)(e.eopN - 1))) return false;
    const int i = (int)floor(utc - e.eopFirstMjd);
    const double f = utc - floor(utc);
    ep.mjdUtc = utc;
    ep.ut1Utc = dut[i] + f * (dut[i + 1] - dut[i]);
    ep.ttUtc = 32.184 + dat[i];
    ep.xp = xp[i] + f * (xp[i + 1] - xp[i]);
    ep.yp = yp[i] + f * (yp[i + 1] - yp[i]);
    return true;
}

// ---- NRLMSISE-00 epoch inputs -----------------------------------------------------------------
static __device__ __forceinline__ double taiMinusUtc(double mjd) {
    const double dates[27] = {41499, 41683, 42048, 42413, 42778, 43144, 43509, 43874, 44239,
                              44786, 45151, 45516, 46247, 47161, 47892, 48257, 48804, 49169,
                              49534, 50083, 50630, 51179, 53736, 54832, 56109, 57204, 57754};
    double dat = 10.0;
#pragma unroll
    for (int i = 0; i < 27; ++i)
        if (mjd >= dates[i]) dat = 11.0 + i;
    return dat;
}

static __device__ __forceinline__ double etToMjdUtc(double et) {
    const double days = et / 86400.0;
    const double g = 6.240075674 + 0.01720197034 * days;
    const double tdbTt = 0.001657 * sin(g) + 0.000022 * sin(2.0 * g);
    const double mjdTt = 51544.5 + (et - tdbTt) / 86400.0;
    const double first = mjdTt - (32.184 + taiMinusUtc(mjdTt)) / 86400.0;
    return mjdTt - (32.184 + taiMinusUtc(first)) / 86400.0;
}

static __device__ __forceinline__ double wrapHours(double h) {
    h = fmod(h, 24.0);
    return h < 0.0 ? h + 24.0 : h;
}

static __device__ double gastHours(double mjdUtc) {
    const double kMjdJ2000 = 51544.5, kDeg = 0.0174532925199432957692, kTwoPi = 6.28318530717958647693;
    const double mjd0 = floor(mjdUtc);
    const double ut1 = 86400.0 * (mjdUtc - mjd0);
    const double t0 = (mjd0 - kMjdJ2000) / 36525.0;
    const double t = (mjdUtc - kMjdJ2000) / 36525.0;
    const double gmstSec = 24110.54841 + 8640184.812866 * t0 + 1.002737909350795 * ut1 + (0.093104 - 6.2e-6 * t) * t * t;
    const double gmst = kTwoPi * (gmstSec / 86400.0 - floor(gmstSec / 86400.0));
    const double mjdTt = mjdUtc + (32.184 + taiMinusUtc(mjdUtc)) / 86400.0;
    const double tt = (mjdTt - kMjdJ2000) / 36525.0;
    const double om = (125.04452 - 1934.136261 * tt) * kDeg;
    const double ls = (280.4665 + 36000.7698 * tt) * kDeg;
    const double lm = (218.3165 + 481267.8813 * tt) * kDeg;
    const double dpsi = -17.20 * sin(om) - 1.32 * sin(2.0 * ls) - 0.23 * sin(2.0 * lm) + 0.21 * sin(2.0 * om);
    const double eps = (23.43929111 - (46.8150 + (0.00059 - 0.001813 * tt) * tt) * tt / 3600.0) * kDeg;
    const double eqeq = dpsi / 3600.0 * kDeg * cos(eps);
    return wrapHours((gmst + eqeq) * 24.0 / kTwoPi);
}

static __device__ __noinline__ NrlTime nrlTime(const DevEnv& e, double et) {
    NrlTime t;
    const double mjdUtc = etToMjdUtc(et);
    // weather record and 3-hour slot (Nrlmsise00.cu:207-214)
    const int rec = (int)floor(mjdUtc - e.nrlStartMjd);
    t.valid = (rec >= 3 && rec < e.nrlNdays);
    int slot = (int)floor((mjdUtc - floor(mjdUtc)) * 8.0);
    slot = slot < 0 ? 0 : (slot > 7 ? 7 : slot);
    t.block = t.valid ? rec * 8 + slot : 0;
    // seconds of day as calendarDate forms them (Nrlmsise00.cu:113-130)
    double sod = (mjdUtc - floor(mjdUtc)) * 86400.0;
    if (sod < 0.0) sod += 86400.0;
    const int hour = (int)(sod / 3600.0);
    const int minute = (int)((sod - hour * 3600.0) / 60.0);
    const double second = sod - hour * 3600.0 - minute * 60.0;
    t.sec = hour * 3600.0 + minute * 60.0 + second;
    t.gast = gastHours(mjdUtc);
    return t;
}

static __device__ void nrlEpoch(const DevEnv& e, double et, EpochRecord& r) {
    const NrlTime t = nrlTime(e, et);
    r.nrlValid = t.valid;
    r.nrlBlock = t.block;
    r.nrlSec = t.sec;
    r.nrlGast = t.gast;
}

// ---- full epoch record ------------------------------------------------------------------------
// Everything of a record but the tide corrections, one thread per record:
// rotation, body positions, the epoch-only indirect third-body term, the
// NRLMSISE-00 time inputs.  The tide deltas are left at zero (NaN with
// tideValid = 0 when the EOP table does not cover the epoch) and `tin` gets
// the tide model's inputs; returns whether the tide corrections are to be
// formed (epochRecordsKernel does that one warp per record).
static __device__ bool evalEpochRecordBase(const DevEnv& e, double et, EpochRecord& r, tidefield::Epoch& tin) {
    r.et = et;
    for (int i = 0; i < 9; ++i) r.R[i] = (i % 4 == 0) ? 1.0 : 0.0;
    r.w[0] = r.w[1] = r.w[2] = 0.0;
    if (e.hasRot) earthRotation(e, et, r.R, r.w);
    for (int k = 0; k < kMaxPoles; ++k)
        for (int i = 0; i < 3; ++i) r.pole[k][i] = r.poleW[k][i] = r.poleV[k][i] = 0.0;
    for (int b = 0; b < e.nbodies; ++b) {
        const int k = e.poleSlot[b];
        if (k < 0) continue;
        // the body's z axis in inertial axes (the third row of its ICRF ->
        // body rotation), its angular velocity and its velocity
        double Rb[9];
        iauRotation(e.poleCoef + e.poleData[k], e.poleDeg[k], e.poleNp[k], e.poleBary[k], e.poleNpDeg[k], et, Rb,
                    r.poleW[k]);
        r.pole[k][0] = Rb[6];
        r.pole[k][1] = Rb[7];
        r.pole[k][2] = Rb[8];
        if (b == e.atmBody) chainVelocity(e, e.chainPlus[b], e.chainMinus[b], et, r.poleV[k]);
    }
    for (int i = 0; i < 9; ++i) r.fieldR[i] = (i % 4 == 0) ? 1.0 : 0.0;
    if (e.shFrame) {
        double wb[3];
        iauRotation(e.poleCoef + e.shFrameData, e.shFrameDeg, e.shFrameNp, e.shFrameBary, e.shFrameNpDeg, et, r.fieldR,
                    wb);
    }
    for (int b = 0; b < e.nbodies; ++b) chainPosition(e, e.chainPlus[b], e.chainMinus[b], et, r.body[b]);
    // the indirect part of the third-body attraction (PointGravity.h:76-105):
    // the Earth's acceleration towards each body, the same for every object
    r.indirect[0] = r.indirect[1] = r.indirect[2] = 0.0;
    for (int b = 0; b < e.nbodies; ++b) {
        if (!(e.bodyFlags[b] & kGravity) || b == e.earthIndex) continue;
        const double* rb = r.body[b];
        const double rbn = sqrt(rb[0] * rb[0] + rb[1] * rb[1] + rb[2] * rb[2]);
        const double f2 = -e.bodyGm[b] * (1.0 / (rbn * rbn * rbn));
        r.indirect[0] += f2 * rb[0];
        r.indirect[1] += f2 * rb[1];
        r.indirect[2] += f2 * rb[2];
    }
    for (int k = 0; k < kTideTri; ++k) r.dC[k] = r.dS[k] = 0.0;
    r.tideValid = 1;
    bool tides = false;
    if (e.solid || e.ocean) {
        if (!eopTime(e, et, tin)) {
            r.tideValid = 0;
            for (int k = 0; k < kTideTri; ++k) r.dC[k] = r.dS[k] = NAN;
        } else {
            double sun[3], moon[3];
            chainPosition(e, e.sunUnitsPlus, e.sunUnitsMinus, et, sun);
            chainPosition(e, e.moonUnitsPlus, e.moonUnitsMinus, et, moon);
            for (int k = 0; k < 3; ++k) {
                tin.sun[k] = 1000.0 * sun[k];
                tin.moon[k] = 1000.0 * moon[k];
            }
            for (int k = 0; k < 9; ++k) tin.E[k] = r.R[k];
            tides = true;
        }
    }
    if (e.hasNrl) nrlEpoch(e, et, r);
    else {
        r.nrlValid = 0;
    }
    return tides;
}

#endif  // __CUDACC__

}  // namespace phop
