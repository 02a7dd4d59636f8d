// CPU oracle: a scalar FP64 restatement of ParaHPOP's host backend for the
// batched fixed-step RKF78 full-force propagation.  TEST INFRASTRUCTURE ONLY:
// the tests, the smoke check and the CPU-baseline leg of the benchmark call it
// as the checker; the product never links it.
//
// Follows, function by function (paths relative to the reference tree):
//   fixed-step control   src/common/engine/paraHPOP/propagators/FixedStep.h:7-47
//   host loop            src/common/engine/paraHPOP/propagators/host/Propagator.h:61-82
//   RKF78 step           third_party/parm/parm/integrate/rk/host/Step.h:33-124,
//                        tableau third_party/parm/parm/integrate/rk/coefs/tableau.h:19-64
//   right-hand side      src/common/engine/paraHPOP/model/accelerations/PrivateAccelerations.h:29-208
//   point gravity        .../accelerations/PointGravity.h:19-105
//   spherical harmonics  .../accelerations/SphericalHarmonics.h:30-41,
//                        sphericalharmonics/Evaluation.h:111-159,282-295,
//                        DegreeLoop.h:51-132, LegendreRecursor.h:170-360,
//                        PseudoPhasor.h:26-110, Coefficients.h:480-535
//   SRP + shadow         .../accelerations/SRP.h:17-70, environment/eclipse/Shadow.h:84-147
//   drag                 .../accelerations/Drag.h:50-73,
//                        environment/atmosphere/Nrlmsise00.cu:83-327
//   Earth corrections    .../accelerations/EarthCorrections.h:8-105,
//                        hpop_compat/HpopCorrections.h:121-145,339-376,
//                        environment/earthcorrections/EarthCorrections.h:46-105
//   ephemeris            third_party/parm/parm/interpolate/chebyshev/Interpolator.h:37-110,226-260,
//                        detail/Interpolators.h:65-75, brie/core/Type2BodyUnit.h:47-60
//   Earth orientation    third_party/brie/brie/orientations/detail/IERS2000Model.h:56-215,
//                        LagrangeInterp.h:88-130, RotationModelUnit.h:96-148,
//                        parm/interpolate/lagrange/Interpolator.h:61-104,416-432,812-833
//
// The empirical NRLMSISE-00 model (gtd7d) and the epoch-only tide
// coefficient sets are the reference's own sources, compiled unchanged into
// oracle/_ref/ref_models.o (oracle/ref_models.cpp) and linked here; nothing
// of the product is included, so every GPU-vs-oracle comparison checks the
// product's drag and tide code against the reference's.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

extern "C" {
double ref_nrl_density(int doy, double sec, double alt, double glat, double glong, double lst, double f107A,
                       double f107, double ap, const double ap_a[7]);
void ref_tide_coefficients(const double E[9], const double sun[3], const double moon[3], double mjdUtc, double ut1Utc,
                           double ttUtc, double xp, double yp, int zeroTide, int solid, double C[49], double S[49]);
}

namespace tide {
// epoch inputs of the tide model (HpopCorrections.h:19-23)
struct Epoch {
    double E[9];             // ICRF -> ITRF, row-major
    double sun[3], moon[3];  // geocentric ICRF, m
    double mjdUtc, ut1Utc, ttUtc, xpArcsec, ypArcsec;
};
struct Coeffs {
    double C[7][7];
    double S[7][7];
};
// constants of the tide and relativity model (HpopCorrections.h:25-31)
constexpr double kMuEarth = 398600.4415e9;
constexpr double kRadius = 6378.1363e3;
constexpr double kLight = 299792457.999999984;

inline void rotate(const double E[9], const double x[3], double out[3]) {
    for (int i = 0; i < 3; ++i) out[i] = E[3 * i] * x[0] + E[3 * i + 1] * x[1] + E[3 * i + 2] * x[2];
}
// solid (zero-tide or tide-free) or ocean coefficient set of the reference
inline void coefficients(const Epoch& ep, bool solid, bool zeroTide, Coeffs& out) {
    double C[49], S[49];
    ref_tide_coefficients(ep.E, ep.sun, ep.moon, ep.mjdUtc, ep.ut1Utc, ep.ttUtc, ep.xpArcsec, ep.ypArcsec,
                          zeroTide ? 1 : 0, solid ? 1 : 0, C, S);
    for (int n = 0; n < 7; ++n)
        for (int m = 0; m < 7; ++m) {
            out.C[n][m] = C[7 * n + m];
            out.S[n][m] = S[7 * n + m];
        }
}
}  // namespace tide

extern "C" {

enum { F_GRAVITY = 1, F_SHAPE = 2, F_RADIATION = 4, F_ATMOSPHERE = 8, F_OCCULTING = 16, F_OBLATENESS = 32 };

typedef struct {
    // geopotential (normalised), triangle index n(n+1)/2+m
    int sh_degree, sh_order, sh_normalized;
    double sh_R, sh_GM;
    const double* sh_C;
    const double* sh_S;
    // bodies, sorted by NAIF id
    int nbodies;
    const int* body_id;
    const double* body_gm;
    const double* body_radius;
    const int* body_flags;
    double flattening;  // Earth
    double au;
    // Type-2 Chebyshev ephemeris units
    int neph;
    const int* eph_target;
    const int* eph_center;
    const int* eph_nint;
    const int* eph_pdeg;
    const int64_t* eph_offset;
    const double* eph_data;
    // IERS2000 orientation unit
    int has_rot, rot_nnut, rot_nerp;
    const double* rot_data;
    // NRLMSISE-00
    int has_nrl, nrl_ndays;
    double nrl_start_mjd, nrl_hcutoff, nrl_density_scale;
    const double* nrl_weather;  // 13 x ndays, component-major
    // Earth corrections
    int solid, ocean, relativity, zero_tide;
    int eop_n;
    double eop_first_mjd;
    const double* eop;  // 4 x n: xp, yp, ut1-utc, tai-utc (component-major)
    // oblateness (J2) model and exponential atmosphere
    const double* body_j2;        // per body, from the constants file (0 when absent)
    const double* body_gm_const;  // per body GM from the constants file (the J2 model's)
    const double* body_soi;       // per body sphere of influence, km (1e20 when absent)
    int n_exp;                    // exponential atmosphere bands (0: none)
    const double* exp_seg;        // 4 x n_exp component-major: rho0, h0, scaleHeight, hCutoff; ascending h0
    // Earth frame: 4 = the IERS2000 unit above; 3 = binary Chebyshev Euler
    // angles in rot_data ([r, starts, 3 angle blocks], ITRF93)
    int rot_kind, rot_nint, rot_pdeg, rot_ecliptic;
    // kind 1, IAU body model: RA, Dec, PM coefficient counts, their
    // nutation-precession amplitude counts, and the barycentric angle
    // polynomials appended to rot_data (offset -1: none)
    int iau_deg[3], iau_np[3];
    int iau_bary_offset, iau_np_deg, iau_np_angles;
    // per body (index as body_id): the IAU body model of a body other than
    // the Earth, for its J2 model (data NULL: none), laid out as rot_data of
    // kind 1 with its barycentric angles at frame_bary_offset (-1: none)
    const double* frame_data[12];
    int frame_deg[12][3], frame_np[12][3], frame_bary_offset[12], frame_np_deg[12];
    double body_flattening[12];  // per body: its "flattening" (geodetic height for drag)
} OracleEnv;

}  // extern "C"

namespace {

const int kEarth = 399, kSun = 10, kMoon = 301;

struct V3 {
    double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double norm(V3 a) { return sqrt(dot(a, a)); }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double rcube(V3 a) {
    const double r = norm(a);
    return 1.0 / (r * r * r);
}
inline V3 mat(const double R[9], V3 v) {
    return {R[0] * v.x + R[1] * v.y + R[2] * v.z, R[3] * v.x + R[4] * v.y + R[5] * v.z,
            R[6] * v.x + R[7] * v.y + R[8] * v.z};
}
inline V3 matT(const double R[9], V3 v) {
    return {R[0] * v.x + R[3] * v.y + R[6] * v.z, R[1] * v.x + R[4] * v.y + R[7] * v.z,
            R[2] * v.x + R[5] * v.y + R[8] * v.z};
}

// ---- time (IF/util/TimeConversion.h:30-40) --------------------------------
inline double mjdToEt(double mjd) { return fma(mjd, 86400.0, -43200.0); }
inline double etToMjd(double et) { return fma(et, 1.0 / 86400.0, 0.5); }

// ---- Chebyshev ephemeris ----------------------------------------------------
V3 chebUnit(const OracleEnv& e, int u, double t, V3* vel) {
    const double* d = e.eph_data + e.eph_offset[u];
    const int n = e.eph_nint[u], deg = e.eph_pdeg[u];
    const double r = d[0];
    const double* starts = d + 1;
    const double* cf = d + 1 + n;
    long idx = (long)((t - starts[0]) / (2 * r));
    if (idx < 0) idx = 0;
    if (idx >= n) idx = n - 1;
    const double s = (t - starts[idx]) / r - 1.0;
    const double s2 = 2 * s;
    double out[3], dout[3];
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
        out[dim] = fma(s, x, c[idx] - w);
        dout[dim] = (1.0 / r) * fma(s, v, x - dw);
    }
    if (vel) *vel = {dout[0], dout[1], dout[2]};
    return {out[0], out[1], out[2]};
}

int unitOf(const OracleEnv& e, int target) {
    for (int u = 0; u < e.neph; ++u)
        if (e.eph_target[u] == target) return u;
    return -1;
}

// position of `body` relative to `center` via the common ancestor of their chains
V3 position(const OracleEnv& e, double t, int body, int center) {
    if (body == center) return {0, 0, 0};
    int pb[16], pc[16], nb = 0, nc = 0;
    for (int b = body; nb < 16; b = e.eph_center[unitOf(e, b)]) {
        pb[nb++] = b;
        if (b == 0 || unitOf(e, b) < 0) break;
    }
    for (int b = center; nc < 16; b = e.eph_center[unitOf(e, b)]) {
        pc[nc++] = b;
        if (b == 0 || unitOf(e, b) < 0) break;
    }
    int common = 0;
    for (int i = 0; i < nb && !common; ++i)
        for (int j = 0; j < nc; ++j)
            if (pb[i] == pc[j]) {
                common = pb[i] == 0 ? -1 : pb[i];
                break;
            }
    if (common == -1) common = 0;
    V3 p = {0, 0, 0};
    for (int i = 0; i < nb && pb[i] != common; ++i) p = p + chebUnit(e, unitOf(e, pb[i]), t, nullptr);
    for (int j = 0; j < nc && pc[j] != common; ++j) p = p - chebUnit(e, unitOf(e, pc[j]), t, nullptr);
    return p;
}

// velocity of `body` relative to `center` (km/s): the chain's Chebyshev derivatives
V3 velocity(const OracleEnv& e, double t, int body, int center) {
    if (body == center) return {0, 0, 0};
    int pb[16], pc[16], nb = 0, nc = 0;
    for (int b = body; nb < 16; b = e.eph_center[unitOf(e, b)]) {
        pb[nb++] = b;
        if (b == 0 || unitOf(e, b) < 0) break;
    }
    for (int b = center; nc < 16; b = e.eph_center[unitOf(e, b)]) {
        pc[nc++] = b;
        if (b == 0 || unitOf(e, b) < 0) break;
    }
    int common = 0;
    for (int i = 0; i < nb && !common; ++i)
        for (int j = 0; j < nc; ++j)
            if (pb[i] == pc[j]) {
                common = pb[i] == 0 ? -1 : pb[i];
                break;
            }
    if (common == -1) common = 0;
    V3 v = {0, 0, 0}, dv;
    for (int i = 0; i < nb && pb[i] != common; ++i) {
        chebUnit(e, unitOf(e, pb[i]), t, &dv);
        v = v + dv;
    }
    for (int j = 0; j < nc && pc[j] != common; ++j) {
        chebUnit(e, unitOf(e, pc[j]), t, &dv);
        v = v - dv;
    }
    return v;
}

// ---- Earth orientation ------------------------------------------------------
void lagrange(const double* ys, int stride, int nch, const double* keys, double x0, double h, int npts, int n,
              double t, bool uniform, double* val, double* der) {
    long lo;
    double q;
    const long half = npts / 2;
    if (uniform) {
        const long f = (long)floor((t - x0) / h);
        lo = f - half + 1;
        if (lo < 0) lo = 0;
        if (lo > n - npts) lo = n - npts;
        q = (t - (x0 + (double)lo * h)) / h;
    } else {
        long a = 0, b = n;
        while (a < b) {
            const long mid = a + ((b - a) >> 1);
            if (keys[mid] <= t) a = mid + 1; else b = mid;
        }
        lo = a - 1 - half + 1;
        if (lo < 0) lo = 0;
        if (lo > n - npts) lo = n - npts;
        q = t;
    }
    for (int c = 0; c < nch; ++c) val[c] = der[c] = 0.0;
    for (int j = 0; j < npts; ++j) {
        double prod = 1, dprod = 0, denom = 1;
        for (int m = 0; m < npts; ++m) {
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
        for (int c = 0; c < nch; ++c) {
            const double y = ys[(int64_t)c * stride + lo + j];
            val[c] = fma(wv, y, val[c]);
            der[c] = fma(wd, y, der[c]);
        }
    }
    if (uniform)
        for (int c = 0; c < nch; ++c) der[c] *= 1.0 / h;
}

void mat3mul(double C[9], const double A[9], const double B[9]) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}

// ICRF -> ITRF rotation R and inertial angular velocity w at ET `t`
// ICRF -> ITRF93 from a binary orientation unit (orientations/RefEphUnit.h
// :769-790 and :890-900, frames/Rotation.h:124-133, frames/Frames.h:57-166):
// angles RA = v0 - pi/2, Dec = pi/2 - v1, PM = v2 mod 2 pi from three
// Chebyshev series, R = Rz(PM) Rx(pi/2 - Dec) Rz(pi/2 + RA) [Rx(obliquity)
// for ECLIPJ2000-based units], omega from the 3-1-3 Euler kinematics.
void eulerRotation(double ra, double dec, double pm, double raDot, double decDot, double pmDot, bool ecliptic,
                   double R[9], V3* w);

void binaryEarthRotation(const OracleEnv& e, double t, double R[9], V3* w) {
    const double* d = e.rot_data;
    const int n = e.rot_nint, deg = e.rot_pdeg;
    const double r = d[0];
    const double* starts = d + 1;
    const double* cf = d + 1 + n;
    long idx = (long)((t - starts[0]) / (2 * r));
    if (idx < 0) idx = 0;
    if (idx >= n) idx = n - 1;
    const double s = (t - starts[idx]) / r - 1.0;
    double v[3], vd[3];
    for (int dim = 0; dim < 3; ++dim) {
        // Chebyshev series and its derivative by the three-term recurrences
        // T_{k+1} = 2 s T_k - T_{k-1}, T'_{k+1} = 2 T_k + 2 s T'_k - T'_{k-1}
        const double* c = cf + (int64_t)dim * (deg + 1) * n;
        double T0 = 1.0, T1 = s, D0 = 0.0, D1 = 1.0;
        double sum = c[idx], dsum = 0.0;
        if (deg >= 1) {
            sum += c[idx + n] * T1;
            dsum += c[idx + n] * D1;
        }
        for (int k = 2; k <= deg; ++k) {
            const double T2 = 2.0 * s * T1 - T0, D2 = 2.0 * T1 + 2.0 * s * D1 - D0;
            sum += c[idx + (int64_t)k * n] * T2;
            dsum += c[idx + (int64_t)k * n] * D2;
            T0 = T1;
            T1 = T2;
            D0 = D1;
            D1 = D2;
        }
        v[dim] = sum;
        vd[dim] = dsum / r;
    }
    const double ra = v[0] - M_PI / 2, dec = M_PI / 2 - v[1], pm = fmod(v[2], 2 * M_PI);
    eulerRotation(ra, dec, pm, vd[0], -vd[1], vd[2], e.rot_ecliptic != 0, R, w);
}

// IAU body model (orientations/RefEphUnit.h:100-330, 640-770): RA and Dec
// polynomials in Julian centuries, PM in days (degrees), with the
// nutation-precession series over the barycentric angle polynomials; angles
// mod 360, then as for a binary unit.
void iauRotation(const double* d, const int* degs, const int* nps, int baryOffset, int npDeg, double t, double R[9],
                 V3* w) {
    const double cy = 3155760000.0, dy = 86400.0, deg = M_PI / 180.0;
    const double T = t / cy, D = t / dy;
    auto poly = [](const double* c, int n, double x, double* der) {
        // ascending coefficients: value and derivative by powers
        double v = 0.0, dv = 0.0, p = 1.0;
        for (int k = 0; k < n; ++k) {
            v += c[k] * p;
            if (k + 1 < n) dv += c[k + 1] * (k + 1) * p;
            p *= x;
        }
        *der = dv;
        return v;
    };
    const int n0 = degs[0], n1 = degs[1], n2 = degs[2];
    double r0, r1, r2;
    double ang[3] = {poly(d, n0, T, &r0), poly(d + n0, n1, T, &r1), poly(d + n0 + n1, n2, D, &r2)};
    double rate[3] = {r0 / cy, r1 / cy, r2 / dy};
    if (baryOffset >= 0) {
        const double* amp = d + n0 + n1 + n2;
        for (int comp = 0; comp < 3; ++comp) {
            for (int i = 0; i < nps[comp]; ++i) {
                double dp;
                const double a = poly(d + baryOffset + (int64_t)i * npDeg, npDeg, T, &dp);
                if (comp == 1) {
                    ang[comp] += amp[i] * cos(a * deg);
                    rate[comp] += -amp[i] * sin(a * deg) * dp * deg / cy;
                } else {
                    ang[comp] += amp[i] * sin(a * deg);
                    rate[comp] += amp[i] * cos(a * deg) * dp * deg / cy;
                }
            }
            amp += nps[comp];
        }
    }
    eulerRotation(fmod(ang[0], 360.0) * deg, fmod(ang[1], 360.0) * deg, fmod(ang[2], 360.0) * deg, rate[0] * deg,
                  rate[1] * deg, rate[2] * deg, false, R, w);
}

void iauEarthRotation(const OracleEnv& e, double t, double R[9], V3* w) {
    iauRotation(e.rot_data, e.iau_deg, e.iau_np, e.iau_bary_offset, e.iau_np_deg, t, R, w);
}

// passive Z-X-Z rotation (pi/2 + RA, pi/2 - Dec, PM) [then the ICRF ->
// ECLIPJ2000 bias], omega from the 3-1-3 Euler kinematics mapped to ICRF
void eulerRotation(double ra, double dec, double pm, double raDot, double decDot, double pmDot, bool ecliptic,
                   double R[9], V3* w) {
    const double a1 = M_PI / 2 + ra, a2 = M_PI / 2 - dec;
    auto rz = [](double a, double M[9]) {
        const double c = cos(a), sn = sin(a);
        const double m[9] = {c, sn, 0, -sn, c, 0, 0, 0, 1};
        for (int k = 0; k < 9; ++k) M[k] = m[k];
    };
    auto rx = [](double a, double M[9]) {
        const double c = cos(a), sn = sin(a);
        const double m[9] = {1, 0, 0, 0, c, sn, 0, -sn, c};
        for (int k = 0; k < 9; ++k) M[k] = m[k];
    };
    auto mul = [](const double A[9], const double B[9], double C[9]) {
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
    };
    double Z1[9], X[9], Z3[9], T[9], A[9];
    rz(a1, Z1);
    rx(a2, X);
    rz(pm, Z3);
    mul(X, Z1, T);
    mul(Z3, T, A);
    V3 om = {decDot * sin(ra) + pmDot * cos(ra) * cos(dec), -decDot * cos(ra) + pmDot * sin(ra) * cos(dec),
             raDot + pmDot * sin(dec)};
    if (ecliptic) {
        double E[9];
        rx(84381.448 / 3600.0 * (M_PI / 180.0), E);
        mul(A, E, R);
        om = {om.x, E[4] * om.y + E[7] * om.z, E[5] * om.y + E[8] * om.z};  // E^T omega
    } else {
        for (int k = 0; k < 9; ++k) R[k] = A[k];
    }
    if (w) *w = om;
}

void earthRotation(const OracleEnv& e, double t, double R[9], V3* w) {
    if (e.rot_kind == 3) {
        binaryEarthRotation(e, t, R, w);
        return;
    }
    if (e.rot_kind == 1) {
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
    const int nn = e.rot_nnut, ne = e.rot_nerp;
    const double* d = e.rot_data;
    const double* cst = d + 3 * nn + 5 * ne;
    double nodes[8], rates[8];
    lagrange(d, nn, 3, nullptr, cst[0], cst[1], 6, nn, ttMjd, true, nodes, rates);
    lagrange(d + 3 * nn, ne, 5, cst + 4, 0, 0, 4, ne, ttMjd, false, nodes + 3, rates + 3);
    // IERS2000Model::computePrelude + composeMatrix
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
    const double c1 = cos(E), s1 = sin(E), c2 = cos(D), s2 = sin(D), c3 = cos(ms), s3 = sin(ms);
    const double PN[9] = {c1 * c2 * c3 - s1 * s3, c1 * s3 + s1 * c2 * c3, -c3 * s2, -s1 * c3 - c1 * c2 * s3,
                          c1 * c3 - s1 * c2 * s3, s2 * s3, s2 * c1, s2 * s1, c2};
    const double c1d = -s1 * Ed, s1d = c1 * Ed, c2d = -s2 * Dd, s2d = c2 * Dd, c3d = -s3 * msd, s3d = c3 * msd;
    const double c2s3 = c2 * s3, c2c3 = c2 * c3, c2s3d = c2d * s3 + c2 * s3d, c2c3d = c2d * c3 + c2 * c3d;
    const double PNd[9] = {-s1d * s3 - s1 * s3d + c1d * c2c3 + c1 * c2c3d, c1d * s3 + c1 * s3d + s1d * c2c3 + s1 * c2c3d,
                           -c3d * s2 - c3 * s2d, -s1d * c3 - s1 * c3d - c1d * c2s3 - c1 * c2s3d,
                           c1d * c3 + c1 * c3d - s1d * c2s3 - s1 * c2s3d, s2d * s3 + s2 * s3d, s2d * c1 + s2 * c1d,
                           s2d * s1 + s2 * s1d, c2d};
    const double ct = cos(theta), st = sin(theta);
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
    for (int i = 0; i < 9; ++i) Rd[i] = t1[i] + t2[i] + t3[i];
    if (w) {
        double M[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) M[3 * i + j] = Rd[i] * R[j] + Rd[3 + i] * R[3 + j] + Rd[6 + i] * R[6 + j];
        *w = {0.5 * (M[7] - M[5]), 0.5 * (M[2] - M[6]), 0.5 * (M[3] - M[1])};
    }
}

// ---- spherical harmonics ----------------------------------------------------
struct ShFactors {
    std::vector<double> f;  // interleaved (a_nm | c_m, b_nm), triangle index
};

void shFactors(const OracleEnv& e, ShFactors& out) {
    const int N = e.sh_degree, M = e.sh_order;
    out.f.assign((size_t)(N + 1) * (N + 2), 0.0);
    for (int m = 0; m <= M; ++m)
        for (int n = m; n <= N; ++n) {
            const size_t i = 2 * ((size_t)n * (n + 1) / 2 + m);
            if (n == m) {
                double cm;
                if (e.sh_normalized) cm = (m == 1) ? sqrt(3.0) : (m == 0 ? 1.0 : sqrt((2.0 * m + 1.0) / (2.0 * m)));
                else cm = (m == 1 || m == 0) ? 1.0 : (2.0 * m - 1.0);
                out.f[i] = cm;
            } else {
                const double nn = n, mm = m;
                if (e.sh_normalized) {
                    out.f[i] = sqrt(((2.0 * nn - 1.0) * (2.0 * nn + 1.0)) / ((nn - mm) * (nn + mm)));
                    out.f[i + 1] = sqrt(((2.0 * nn + 1.0) * (nn + mm - 1.0) * (nn - mm - 1.0))
                                        / ((2.0 * nn - 3.0) * (nn + mm) * (nn - mm)));
                } else {
                    out.f[i] = (2.0 * nn - 1.0) / (nn - mm);
                    out.f[i + 1] = (nn + mm - 1.0) / (nn - mm);
                }
            }
        }
}

V3 shBodyFixed(const OracleEnv& e, const ShFactors& F, V3 p) {
    const int N = e.sh_degree, M = e.sh_order;
    const size_t half = (size_t)(N + 1) * (N + 2) / 2;
    const double rn = norm(p);
    const double rho = sqrt(p.x * p.x + p.y * p.y);
    const double sinPhi = p.z / rn, cosPhi = rho / rn;
    const double sinL = rho > 1e-14 ? p.y / rho : 0.0, cosL = rho > 1e-14 ? p.x / rho : 1.0;
    const double alpha = e.sh_R / rn;
    double sinML = 0.0, cosML = 1.0;
    double Pmm = 1.0, dPmm = 0.0, alpham = 1.0;
    V3 acc = {0, 0, 0};
    for (int m = 0; m <= M; ++m) {
        double Pn = Pmm, dPn = dPmm, Pn1 = 0.0, dPn1 = 0.0, alphan = alpham;
        V3 col = {0, 0, 0};
        for (int n = m; n <= N; ++n) {
            const size_t ti = (size_t)n * (n + 1) / 2 + m;
            const double c = e.sh_C[ti];
            const double s = m > 0 ? e.sh_S[ti] : 0.0;
            const double C = c * cosML + s * sinML;
            const double S = c * sinML - s * cosML;
            double divCos = (m == 0 || cosPhi == 0.0) ? 0.0 : Pn / cosPhi;
            if (m == 1 && cosPhi == 0.0) {
                const double sign = sinPhi > 0.0 ? 1.0 : ((n & 1) ? 1.0 : -1.0);
                double v = 0.5 * (double)n * (n + 1.0);
                if (e.sh_normalized) v *= sqrt(2.0 * (2.0 * n + 1.0) / ((double)n * (n + 1.0)));
                divCos = sign * v;
            }
            col.x -= ((n + 1) * alphan * Pn * C);
            col.y += (alphan * dPn * C);
            col.z -= (m * alphan * divCos * S);
            if (n < N) {
                const double a = F.f[2 * ((size_t)(n + 1) * (n + 2) / 2 + m)];
                const double b = F.f[2 * ((size_t)(n + 1) * (n + 2) / 2 + m) + 1];
                const double P2 = Pn1;
                Pn1 = Pn;
                Pn = a * sinPhi * Pn1 - b * P2;
                const double dP2 = dPn1;
                dPn1 = dPn;
                dPn = a * (sinPhi * dPn1 + cosPhi * Pn1) - b * dP2;
                alphan *= alpha;
            }
        }
        acc = acc + col;
        if (m < M) {
            const double ns = cosL * sinML + sinL * cosML;
            const double nc = cosL * cosML - sinL * sinML;
            sinML = ns;
            cosML = nc;
            const double cm = F.f[2 * ((size_t)(m + 1) * (m + 2) / 2 + (m + 1))];
            const double nP = cm * cosPhi * Pmm;
            const double ndP = cm * (cosPhi * dPmm - sinPhi * Pmm);
            Pmm = nP;
            dPmm = ndP;
            alpham *= alpha;
        }
    }
    (void)half;
    acc = (e.sh_GM / (rn * rn)) * acc;
    return {cosPhi * cosL * acc.x - sinPhi * cosL * acc.y - sinL * acc.z,
            cosPhi * sinL * acc.x - sinPhi * sinL * acc.y + cosL * acc.z, sinPhi * acc.x + cosPhi * acc.y};
}

// ---- eclipse (dual cone) -----------------------------------------------------
double clampd(double x, double lo, double hi) { return fmin(fmax(x, lo), hi); }

double shadowFactor(V3 rS, V3 rB, double RSun, double RBody) {
    const double s2 = dot(rS, rS), b2 = dot(rB, rB), sb = dot(rS, rB);
    const double iS = 1.0 / sqrt(s2), iB = 1.0 / sqrt(b2);
    if (b2 <= RBody * RBody) return 0.0;
    const double a = asin(clampd(RSun * iS, 0, 1));
    const double b = asin(clampd(RBody * iB, 0, 1));
    const double c = acos(clampd(sb * iS * iB, -1, 1));
    if (c >= a + b) return 1.0;
    if (c <= fabs(b - a)) {
        if (b >= a) return 0.0;
        return 1.0 - (b * b) / (a * a);
    }
    const double a2 = a * a, bb = b * b, c2 = c * c;
    const double x = (c2 + a2 - bb) / (2.0 * c);
    const double y = sqrt(fmax(a2 - x * x, 0.0));
    const double al = acos(clampd(x / a, -1, 1));
    const double be = acos(clampd((c - x) / b, -1, 1));
    return 1.0 - (a2 * al + bb * be - c * y) / (a2 * 3.14159265358979323846);
}

// ---- NRLMSISE-00 inputs (Nrlmsise00.cu:83-267) --------------------------------
double taiMinusUtc(double mjd) {
    static const double dates[] = {41499, 41683, 42048, 42413, 42778, 43144, 43509, 43874, 44239,
                                   44786, 45151, 45516, 46247, 47161, 47892, 48257, 48804, 49169,
                                   49534, 50083, 50630, 51179, 53736, 54832, 56109, 57204, 57754};
    double dat = 10.0;
    for (int i = 0; i < 27; ++i)
        if (mjd >= dates[i]) dat = 11.0 + i;
    return dat;
}

double etToMjdUtc(double et) {
    const double days = et / 86400.0;
    const double g = 6.240075674 + 0.01720197034 * days;
    const double tdbTt = 0.001657 * sin(g) + 0.000022 * sin(2.0 * g);
    const double mjdTt = 51544.5 + (et - tdbTt) / 86400.0;
    const double first = mjdTt - (32.184 + taiMinusUtc(mjdTt)) / 86400.0;
    return mjdTt - (32.184 + taiMinusUtc(first)) / 86400.0;
}

void calendarDate(double mjd, int& year, int& month, int& day, int& hour, int& minute, double& second) {
    const long a = (long)floor(mjd + 2400001.0);
    long b = 0, c = 0;
    if (a < 2299161) c = a + 1524;
    else {
        b = (long)((a - 1867216.25) / 36524.25);
        c = a + b - b / 4 + 1525;
    }
    const long d = (long)((c - 122.1) / 365.25);
    const long e = 365 * d + d / 4;
    const long f = (long)((c - e) / 30.6001);
    day = (int)(c - e - (long)(30.6001 * f));
    month = (int)(f - 1 - 12 * (f / 14));
    year = (int)(d - 4715 - (7 + month) / 10);
    double sod = (mjd - floor(mjd)) * 86400.0;
    if (sod < 0.0) sod += 86400.0;
    hour = (int)(sod / 3600.0);
    minute = (int)((sod - hour * 3600.0) / 60.0);
    second = sod - hour * 3600.0 - minute * 60.0;
}

int dayOfYear(int year, int month, int day) {
    int days[12] = {31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31};
    if ((year % 4 == 0 && year % 100 != 0) || year % 400 == 0) days[1] = 29;
    int out = day;
    for (int m = 1; m < month; ++m) out += days[m - 1];
    return out;
}

double wrapHours(double h) {
    h = fmod(h, 24.0);
    return h < 0.0 ? h + 24.0 : h;
}

double gastHours(double mjdUtc) {
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

double weatherAt(const OracleEnv& e, int comp, int rec) { return e.nrl_weather[(int64_t)comp * e.nrl_ndays + rec]; }
double apAtLag(const OracleEnv& e, int rec, int slot, int lag) {
    const int h = 24 + slot - lag;
    return weatherAt(e, 5 + h % 8, rec - 3 + h / 8);
}

bool fillWeather(const OracleEnv& e, double mjdUtc, double& f107, double& f107a, double& avgAp, double ap[7]) {
    const int rec = (int)floor(mjdUtc - e.nrl_start_mjd);
    if (rec < 3 || rec >= e.nrl_ndays) return false;
    int slot = (int)floor((mjdUtc - floor(mjdUtc)) * 8.0);
    if (slot < 0) slot = 0;
    if (slot > 7) slot = 7;
    f107 = weatherAt(e, 2, rec - 1);  // adjusted flux, previous day
    f107a = weatherAt(e, 3, rec);
    avgAp = weatherAt(e, 4, rec);
    ap[0] = avgAp;
    ap[1] = weatherAt(e, 5 + slot, rec);
    ap[2] = apAtLag(e, rec, slot, 1);
    ap[3] = apAtLag(e, rec, slot, 2);
    ap[4] = apAtLag(e, rec, slot, 3);
    ap[5] = ap[6] = 0.0;
    for (int d = 4; d <= 11; ++d) ap[5] += apAtLag(e, rec, slot, d);
    for (int d = 12; d <= 19; ++d) ap[6] += apAtLag(e, rec, slot, d);
    ap[5] /= 8.0;
    ap[6] /= 8.0;
    return true;
}

bool geodetic(V3 f, double radius, double flat, double& lat, double& lon, double& alt) {
    const double rho2 = f.x * f.x + f.y * f.y;
    if (!(rho2 + f.z * f.z > 0.0)) return false;
    const double e2 = flat * (2.0 - flat);
    double dz = e2 * f.z, zdz = f.z + dz, n = radius, nh = 0.0;
    for (int it = 0; it < 20; ++it) {
        zdz = f.z + dz;
        nh = sqrt(rho2 + zdz * zdz);
        const double sp = zdz / nh;
        n = radius / sqrt(1.0 - e2 * sp * sp);
        const double next = n * e2 * sp;
        if (fabs(dz - next) < 1.0e-12 * radius) {
            dz = next;
            break;
        }
        dz = next;
    }
    zdz = f.z + dz;
    nh = sqrt(rho2 + zdz * zdz);
    lon = atan2(f.y, f.x);
    lat = atan2(zdz, sqrt(rho2));
    alt = nh - n;
    return isfinite(lat) && isfinite(lon) && isfinite(alt);
}

double nrlDensity(const OracleEnv& e, V3 fixed, double et, double Req) {
    const double mjdUtc = etToMjdUtc(et);
    double lat, lon, alt;
    if (!geodetic(fixed, Req, e.flattening, lat, lon, alt)) return NAN;
    if (alt > e.nrl_hcutoff) return 0.0;
    double f107, f107a, avgAp, ap[7];
    if (!fillWeather(e, mjdUtc, f107, f107a, avgAp, ap)) return NAN;
    int y, mo, d, h, mi;
    double s;
    calendarDate(mjdUtc, y, mo, d, h, mi, s);
    const double sec = h * 3600.0 + mi * 60.0 + s;
    const double kRad = 57.2957795130823208768;
    const double rho = ref_nrl_density(dayOfYear(y, mo, d), sec, alt, lat * kRad, lon * kRad,
                                       wrapHours(gastHours(mjdUtc) + lon * kRad / 15.0), f107a, f107, avgAp, ap);
    if (!isfinite(rho) || rho < 0.0) return NAN;
    return (rho * 1.0e9) * e.nrl_density_scale;
}

// ---- Earth corrections --------------------------------------------------------
double tdbMinusTt(double mjdTt) {
    const double t = (mjdTt - 51544.5) / 36525;
    return 0.001657 * sin(628.3076 * t + 6.2401) + 0.000022 * sin(575.3385 * t + 4.2970)
        + 0.000014 * sin(1256.6152 * t + 6.1969) + 0.000005 * sin(606.9777 * t + 4.0212)
        + 0.000005 * sin(52.9691 * t + 0.4444) + 0.000002 * sin(21.3299 * t + 5.5431)
        + 0.000010 * sin(628.3076 * t + 4.2490);
}

bool eopTime(const OracleEnv& e, double et, tide::Epoch& ep) {
    if (e.eop_n < 2 || !isfinite(et)) return false;
    const double* xp = e.eop;
    const double* yp = e.eop + e.eop_n;
    const double* dut = e.eop + 2 * e.eop_n;
    const double* dat = e.eop + 3 * e.eop_n;
    double ttEt = et;
    for (int j = 0; j < 2; ++j) ttEt = et - tdbMinusTt(51544.5 + ttEt / 86400);
    double utc = 51544.5 + (ttEt - 69.184) / 86400;
    for (int j = 0; j < 3; ++j) {
        double day = floor(utc - e.eop_first_mjd);
        if (day < 0) day = 0;
        if (day > (double)(e.eop_n - 1)) day = (double)(e.eop_n - 1);
        utc = 51544.5 + (ttEt - 32.184 - dat[(int)day]) / 86400;
    }
    if (!(utc >= e.eop_first_mjd) || !(utc < e.eop_first_mjd + (double)(e.eop_n - 1))) return false;
    const int i = (int)floor(utc - e.eop_first_mjd);
    const double f = utc - floor(utc);
    ep.mjdUtc = utc;
    ep.ut1Utc = dut[i] + f * (dut[i + 1] - dut[i]);
    ep.ttUtc = 32.184 + dat[i];
    ep.xpArcsec = xp[i] + f * (xp[i + 1] - xp[i]);
    ep.ypArcsec = yp[i] + f * (yp[i + 1] - yp[i]);
    return true;
}

// fully normalised Legendre values and latitude derivatives, degree <= 6
void legendreWithDerivative(int nmax, double phi, double p[7][7], double dp[7][7]) {
    for (int n = 0; n < 7; ++n)
        for (int m = 0; m < 7; ++m) p[n][m] = dp[n][m] = 0.0;
    const double s = sin(phi), c = cos(phi);
    p[0][0] = 1.0;
    if (nmax == 0) return;
    p[1][1] = sqrt(3.0) * c;
    dp[1][1] = -sqrt(3.0) * s;
    for (int n = 2; n <= nmax; ++n) {
        const double k = sqrt((2.0 * n + 1) / (2.0 * n));
        p[n][n] = k * c * p[n - 1][n - 1];
        dp[n][n] = k * (c * dp[n - 1][n - 1] - s * p[n - 1][n - 1]);
    }
    for (int n = 1; n <= nmax; ++n) {
        const double k = sqrt(2.0 * n + 1);
        p[n][n - 1] = k * s * p[n - 1][n - 1];
        dp[n][n - 1] = k * (c * p[n - 1][n - 1] + s * dp[n - 1][n - 1]);
    }
    for (int m = 0; m <= nmax; ++m)
        for (int n = m + 2; n <= nmax; ++n) {
            const double k = sqrt((2.0 * n + 1) / ((n - m) * double(n + m)));
            const double a = sqrt(2.0 * n - 1);
            const double b = sqrt(((n + m - 1) * double(n - m - 1)) / (2.0 * n - 3));
            p[n][m] = k * (a * s * p[n - 1][m] - b * p[n - 2][m]);
            dp[n][m] = k * (a * s * dp[n - 1][m] + a * c * p[n - 1][m] - b * dp[n - 2][m]);
        }
}

// gradient of a low-degree coefficient set, SI in / SI out (inertial axes)
void tideGradient(const tide::Epoch& ep, const double rin[3], const tide::Coeffs& cf, int maxDeg,
                  double out[3]) {
    const double mu = tide::kMuEarth, R = tide::kRadius;
    double r[3];
    tide::rotate(ep.E, rin, r);
    const double d = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    const double phi = asin(r[2] / d), lon = atan2(r[1], r[0]);
    double p[7][7], dp[7][7];
    legendreWithDerivative(maxDeg, phi, p, dp);
    double dUdr = 0, dUdlat = 0, dUdlon = 0, cosM[7], sinM[7];
    for (int m = 0; m <= maxDeg; ++m) {
        cosM[m] = cos(m * lon);
        sinM[m] = sin(m * lon);
    }
    for (int n = 0; n <= maxDeg; ++n) {
        const double power = pow(R / d, double(n));
        const double b1 = (-mu / (d * d)) * power * (n + 1);
        const double b2 = (mu / d) * power;
        double q1 = 0, q2 = 0, q3 = 0;
        for (int m = 0; m <= n; ++m) {
            const double v = cf.C[n][m] * cosM[m] + cf.S[n][m] * sinM[m];
            q1 += p[n][m] * v;
            q2 += dp[n][m] * v;
            q3 += m * p[n][m] * (cf.S[n][m] * cosM[m] - cf.C[n][m] * sinM[m]);
        }
        dUdr += q1 * b1;
        dUdlat += q2 * b2;
        dUdlon += q3 * b2;
    }
    const double xy2 = r[0] * r[0] + r[1] * r[1], xy = sqrt(xy2);
    const double q = (1.0 / d * dUdr - r[2] / (d * d * xy) * dUdlat);
    const double bf[3] = {q * r[0] - (1.0 / xy2 * dUdlon) * r[1], q * r[1] + (1.0 / xy2 * dUdlon) * r[0],
                          1.0 / d * dUdr * r[2] + xy / (d * d) * dUdlat};
    for (int i = 0; i < 3; ++i) out[i] = ep.E[i] * bf[0] + ep.E[3 + i] * bf[1] + ep.E[6 + i] * bf[2];
}

V3 earthCorrections(const OracleEnv& e, V3 pos, V3 vel, double et) {
    double r[3] = {1000.0 * pos.x, 1000.0 * pos.y, 1000.0 * pos.z};
    double v[3] = {1000.0 * vel.x, 1000.0 * vel.y, 1000.0 * vel.z};
    double solid[3] = {0, 0, 0}, ocean[3] = {0, 0, 0}, rel[3] = {0, 0, 0};
    if (e.solid || e.ocean) {
        tide::Epoch ep;
        if (!eopTime(e, et, ep)) return {NAN, NAN, NAN};
        const V3 sun = position(e, et, kSun, kEarth), moon = position(e, et, kMoon, kEarth);
        ep.sun[0] = 1000.0 * sun.x; ep.sun[1] = 1000.0 * sun.y; ep.sun[2] = 1000.0 * sun.z;
        ep.moon[0] = 1000.0 * moon.x; ep.moon[1] = 1000.0 * moon.y; ep.moon[2] = 1000.0 * moon.z;
        earthRotation(e, et, ep.E, nullptr);
        tide::Coeffs cf;
        if (e.solid) {
            tide::coefficients(ep, true, e.zero_tide != 0, cf);
            tideGradient(ep, r, cf, 4, solid);
        }
        if (e.ocean) {
            tide::coefficients(ep, false, false, cf);
            tideGradient(ep, r, cf, 6, ocean);
        }
    }
    if (e.relativity) {
        const double mu = tide::kMuEarth, c = tide::kLight;
        const double rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        const double vv = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        const double rv = r[0] * v[0] + r[1] * v[1] + r[2] * v[2];
        const double f = mu / (c * c * pow(rr, 3.0));
        for (int i = 0; i < 3; ++i) rel[i] = f * ((4.0 * mu / rr - vv * vv) * r[i] + 4.0 * rv * v[i]);
    }
    return {1.0e-3 * (solid[0] + ocean[0] + rel[0]), 1.0e-3 * (solid[1] + ocean[1] + rel[1]),
            1.0e-3 * (solid[2] + ocean[2] + rel[2])};
}

// ---- oblateness and exponential drag --------------------------------------------
// J2 acceleration in the body frame (J2.h:17-33)
V3 j2BodyFixed(V3 p, double gm, double j2, double radius) {
    const double invr = 1.0 / norm(p);
    const double invr2 = invr * invr;
    const double invr5 = invr2 * invr2 * invr;
    const double base = 1.0 - 5.0 * (p.z * p.z) * invr2;
    const double c = -1.5 * gm * j2 * invr5 * radius * radius;
    return V3{c * p.x * base, c * p.y * base, c * p.z * (base + 2.0)};
}

// Geodetic altitude about the body's polar axis (atmosphere/Geodetic.h:40-75)
double geodeticAltitude(V3 r, V3 pole, double Req, double flattening) {
    if (flattening == 0.0) return norm(r) - Req;
    const double r2 = dot(r, r);
    const double z = dot(r, pole);
    const double xy = r2 - z * z;
    const double flatsq = (2.0 - flattening) * flattening;
    double d0 = 0.0, d = 1e10, sfq = 0.0, zd = z;
    while (std::fabs(d - d0) > 1e-9) {
        d0 = d;
        const double z2 = zd * zd;
        sfq = z2 / (xy + z2);
        d = Req * flatsq * std::sqrt(sfq / (1.0 - flatsq * sfq));
        zd = z + std::copysign(d, z);
    }
    return std::sqrt(xy + zd * zd) - Req / std::sqrt(1.0 - flatsq * sfq);
}

// Piecewise exponential profile: band = number of bands above the first
// whose base h0 <= h (PiecewiseExponentialAtmosphere.h:40-90)
int expBand(const OracleEnv& e, double h) {
    int band = 0;
    for (int s = 1; s < e.n_exp; ++s) band += e.exp_seg[e.n_exp + s] <= h ? 1 : 0;
    return band;
}

// ---- right-hand side ----------------------------------------------------------
struct Object {
    double mass, area, cd, cr;  // area km^2, cr folded with srp/drag area ratio
};

V3 acceleration(const OracleEnv& e, const ShFactors& F, V3 pos, V3 vel, double et, const Object& o) {
    V3 acc = {0, 0, 0};
    const double AMS = o.cr * o.area / o.mass;
    const double BC = o.cd * o.area / o.mass;
    bool haveRot = false;
    double R[9];
    V3 w = {0, 0, 0};
    for (int bi = 0; bi < e.nbodies; ++bi) {
        const int body = e.body_id[bi];
        const int fl = e.body_flags[bi];
        const V3 bodyPos = position(e, et, body, kEarth);
        if (fl & F_GRAVITY) {
            const double gm = e.body_gm[bi];
            if (body != kEarth) {
                const V3 d = pos - bodyPos;
                acc = acc + ((-gm * rcube(d)) * d + (-gm * rcube(bodyPos)) * bodyPos);
            } else {
                acc = acc + (-gm * rcube(pos)) * pos;
            }
        }
        if (fl & F_SHAPE) {
            // the field in its body's frame: the Earth's, or another body's IAU model
            const V3 dp = (body != kEarth) ? pos - bodyPos : pos;
            if (body != kEarth) {
                double Rb[9];
                V3 wb;
                iauRotation(e.frame_data[bi], e.frame_deg[bi], e.frame_np[bi], e.frame_bary_offset[bi],
                            e.frame_np_deg[bi], et, Rb, &wb);
                acc = acc + matT(Rb, shBodyFixed(e, F, mat(Rb, dp)));
            } else {
                if (!haveRot) {
                    earthRotation(e, et, R, &w);
                    haveRot = true;
                }
                acc = acc + matT(R, shBodyFixed(e, F, mat(R, dp)));
            }
        }
        if ((fl & F_OBLATENESS) && !(fl & F_SHAPE)) {
            // J2 model (PrivateAccelerations.h:88-97, J2.h:63-78), in the
            // body's own frame: the Earth's, or another body's IAU model
            const V3 dp = (body != kEarth) ? pos - bodyPos : pos;
            if (norm(dp) <= e.body_soi[bi]) {
                if (body != kEarth) {
                    double Rb[9];
                    V3 wb;
                    iauRotation(e.frame_data[bi], e.frame_deg[bi], e.frame_np[bi], e.frame_bary_offset[bi],
                                e.frame_np_deg[bi], et, Rb, &wb);
                    acc = acc + matT(Rb, j2BodyFixed(mat(Rb, dp), e.body_gm_const[bi], e.body_j2[bi],
                                                     e.body_radius[bi]));
                } else {
                    if (!haveRot) {
                        earthRotation(e, et, R, &w);
                        haveRot = true;
                    }
                    acc = acc + matT(R, j2BodyFixed(mat(R, dp), e.body_gm_const[bi], e.body_j2[bi],
                                                    e.body_radius[bi]));
                }
            }
        }
        if (fl & F_RADIATION) {
            const V3 dp = pos - bodyPos;
            double occ = 1.0;
            bool anyOcc = false;
            for (int oj = 0; oj < e.nbodies; ++oj)
                if ((e.body_flags[oj] & F_OCCULTING) && e.body_id[oj] != kSun) anyOcc = true;
            const double f = e.au * e.au * 4.56e-3 * AMS;
            const V3 srp = (f * rcube(dp)) * dp;
            if (anyOcc) {
                for (int oj = 0; oj < e.nbodies; ++oj) {
                    const int ob = e.body_id[oj];
                    if (!(e.body_flags[oj] & F_OCCULTING) || ob == kSun) continue;
                    const V3 op = (ob == kEarth) ? V3{0, 0, 0} : position(e, et, ob, kEarth);
                    occ *= shadowFactor(dp, pos - op, e.body_radius[bi], e.body_radius[oj]);
                }
                acc = acc + occ * srp;
            } else {
                acc = acc + srp;
            }
        }
        if ((fl & F_ATMOSPHERE) && body != kEarth && e.n_exp > 0) {
            // exponential drag in another body's atmosphere (PrivateAccelerations.h:137-206):
            // relative to the body, about its polar axis, the air moving with
            // its rotation and its velocity
            double Rb[9];
            V3 wb;
            iauRotation(e.frame_data[bi], e.frame_deg[bi], e.frame_np[bi], e.frame_bary_offset[bi], e.frame_np_deg[bi],
                        et, Rb, &wb);
            const V3 rrel = pos - bodyPos;
            const V3 pole = {Rb[6], Rb[7], Rb[8]};
            const double h = geodeticAltitude(rrel, pole, e.body_radius[bi], e.body_flattening[bi]);
            const int band = expBand(e, h);
            const int n = e.n_exp;
            if (h <= e.exp_seg[3 * n + band]) {
                const V3 vr = vel - velocity(e, et, body, kEarth) - cross(wb, rrel);
                const double rho = e.exp_seg[band] * std::exp(-(h - e.exp_seg[n + band]) / e.exp_seg[2 * n + band]);
                acc = acc + ((-0.5 * rho * BC * norm(vr)) * vr);
            }
        }
        if ((fl & F_ATMOSPHERE) && body == kEarth && !e.has_nrl && e.n_exp > 0) {
            // exponential drag (PrivateAccelerations.h:137-206)
            if (!haveRot) {
                earthRotation(e, et, R, &w);
                haveRot = true;
            }
            const V3 pole = {R[6], R[7], R[8]};  // body z axis in inertial axes
            const double h = geodeticAltitude(pos, pole, e.body_radius[bi], e.flattening);
            const int band = expBand(e, h);
            const int n = e.n_exp;
            if (h <= e.exp_seg[3 * n + band]) {
                const V3 vr = vel - cross(w, pos);
                const double rho = e.exp_seg[band] * std::exp(-(h - e.exp_seg[n + band]) / e.exp_seg[2 * n + band]);
                acc = acc + ((-0.5 * rho * BC * norm(vr)) * vr);
            }
        }
        if ((fl & F_ATMOSPHERE) && body == kEarth && e.has_nrl) {
            if (!haveRot) {
                earthRotation(e, et, R, &w);
                haveRot = true;
            }
            const V3 fixed = mat(R, pos);
            const double rho = nrlDensity(e, fixed, et, e.body_radius[bi]);
            const V3 vr = vel - cross(w, pos);
            const double bc = o.cd * o.area / o.mass;
            acc = acc + ((-0.5 * rho * bc * norm(vr)) * vr);
        }
    }
    if (e.solid || e.ocean || e.relativity) acc = acc + earthCorrections(e, pos, vel, et);
    return acc;
}

// ---- RKF78 (parm/integrate/rk/coefs/tableau.h:24-48) -----------------------------
const double kC[12] = {2. / 27, 1. / 9, 1. / 6, 5. / 12, 1. / 2, 5. / 6, 1. / 6, 2. / 3, 1. / 3, 1.0, 0, 1.0};
const double kA[12][12] = {
    {2. / 27, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {1. / 36, 1. / 12, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {1. / 24, 0, 1. / 8, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {5. / 12, 0, -25. / 16, 25. / 16, 0, 0, 0, 0, 0, 0, 0, 0},
    {1. / 20, 0, 0, 1. / 4, 1. / 5, 0, 0, 0, 0, 0, 0, 0},
    {-25. / 108, 0, 0, 125. / 108, -65. / 27, 125. / 54, 0, 0, 0, 0, 0, 0},
    {31. / 300, 0, 0, 0, 61. / 225, -2. / 9, 13. / 900, 0, 0, 0, 0, 0},
    {2.0, 0, 0, -53. / 6, 704. / 45, -107. / 9, 67. / 90, 3.0, 0, 0, 0, 0},
    {-91. / 108, 0, 0, 23. / 108, -976. / 135, 311. / 54, -19. / 60, 17. / 6, -1. / 12, 0, 0, 0},
    {2383. / 4100, 0, 0, -341. / 164, 4496. / 1025, -301. / 82, 2133. / 4100, 45. / 82, 45. / 164, 18. / 41, 0, 0},
    {3. / 205, 0, 0, 0, 0, -6. / 41, -3. / 205, -3. / 41, 3. / 41, 6. / 41, 0, 0},
    {-1777. / 4100, 0, 0, -341. / 164, 4496. / 1025, -289. / 82, 2193. / 4100, 51. / 82, 33. / 164, 12. / 41, 0, 1.0}};
const double kB[13] = {0, 0, 0, 0, 0, 34. / 105, 9. / 35, 9. / 35, 9. / 280, 9. / 280, 0, 41. / 840, 41. / 840};

void rhs(const OracleEnv& e, const ShFactors& F, const Object& o, const double y[6], double t, double k[6]) {
    const V3 a = acceleration(e, F, {y[0], y[1], y[2]}, {y[3], y[4], y[5]}, t, o);
    k[0] = y[3]; k[1] = y[4]; k[2] = y[5];
    k[3] = a.x; k[4] = a.y; k[5] = a.z;
}

void stepRKF78(const OracleEnv& e, const ShFactors& F, const Object& o, double y[6], double dt, double t0) {
    double k[13][6];
    for (int s = 0; s < 13; ++s) {
        double ys[6];
        for (int d = 0; d < 6; ++d) ys[d] = y[d];
        if (s >= 1)
            for (int j = 0; j < s; ++j)
                if (kA[s - 1][j] != 0) {
                    const double coef = dt * kA[s - 1][j];
                    for (int d = 0; d < 6; ++d) ys[d] += coef * k[j][d];
                }
        double ts = t0;
        if (s >= 1) ts += dt * kC[s - 1];
        rhs(e, F, o, ys, ts, k[s]);
    }
    for (int s = 0; s < 13; ++s)
        if (kB[s] != 0) {
            const double cb = dt * kB[s];
            for (int d = 0; d < 6; ++d) y[d] += cb * k[s][d];
        }
}

}  // namespace

extern "C" {

// Propagates objects [0, n) in place.  Per-object duration / step arrays
// (one value per object) generalise the reference's single run duration and
// step.  Returns 0, or 1 if an object did not reach its end within
// max_steps steps.  out_epoch receives the final MJD2000 TDB epochs.
int oracle_propagate(const OracleEnv* env, int64_t n, const double* epoch_mjd, double* state, const double* mass_kg,
                     const double* drag_area_m2, const double* srp_area_m2, const double* cd, const double* cr,
                     const double* duration_s, const double* step_s, int64_t max_steps, double* out_epoch,
                     int threads) {
    const OracleEnv& e = *env;
    ShFactors F;
    if (e.sh_degree > 0) shFactors(e, F);
    int status = 0;
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(dynamic, 1) reduction(| : status)
    for (int64_t i = 0; i < n; ++i) {
        Object o;
        o.mass = mass_kg[i];
        o.area = drag_area_m2[i] * 1e-6;  // driver.cpp:118
        o.cd = cd[i];
        o.cr = cr[i] * srp_area_m2[i] / drag_area_m2[i];  // driver.cpp:120
        const double step = step_s[i], dur = duration_s[i];
        const double start = mjdToEt(epoch_mjd[i]);
        double cur = start;
        const double end = mjdToEt(epoch_mjd[i] + dur / 86400.0);
        const double span = end - cur;
        double dt = std::min(step, span);
        double* y = state + 6 * i;
        bool done = false;
        for (int64_t k = 0; k < max_steps && !done; ++k) {
            stepRKF78(e, F, o, y, dt, cur);
            cur += dt;
            const double rem = end - cur;
            done = rem <= 0;
            dt = done ? 0 : std::min(step, rem);
        }
        if (!done) status |= 1;
        out_epoch[i] = etToMjd(cur);
    }
    return status;
}

// One right-hand side evaluation (km/s^2) for unit tests.
void oracle_acceleration(const OracleEnv* env, const double pos[3], const double vel[3], double et, double mass_kg,
                         double drag_area_m2, double srp_area_m2, double cd, double cr, double out[3]) {
    ShFactors F;
    if (env->sh_degree > 0) shFactors(*env, F);
    Object o;
    o.mass = mass_kg;
    o.area = drag_area_m2 * 1e-6;
    o.cd = cd;
    o.cr = cr * srp_area_m2 / drag_area_m2;
    const V3 a = acceleration(*env, F, {pos[0], pos[1], pos[2]}, {vel[0], vel[1], vel[2]}, et, o);
    out[0] = a.x; out[1] = a.y; out[2] = a.z;
}

// Pieces exposed for the known-answer tests against the reference's sources.
double oracle_nrl_density(int doy, double sec, double alt, double glat, double glong, double lst, double f107A,
                          double f107, double ap, const double ap_a[7]) {
    return ref_nrl_density(doy, sec, alt, glat, glong, lst, f107A, f107, ap, ap_a);
}

void oracle_tides(const double r[3], const double v[3], const double sun[3], const double moon[3], const double E[9],
                  double mjdUtc, double ut1Utc, double ttUtc, double xp, double yp, double solidC[49],
                  double solidS[49], double oceanC[49], double oceanS[49], double acc_solid[3], double acc_ocean[3],
                  double acc_rel[3]) {
    tide::Epoch ep;
    for (int k = 0; k < 3; ++k) {
        ep.sun[k] = sun[k];
        ep.moon[k] = moon[k];
    }
    for (int k = 0; k < 9; ++k) ep.E[k] = E[k];
    ep.mjdUtc = mjdUtc; ep.ut1Utc = ut1Utc; ep.ttUtc = ttUtc; ep.xpArcsec = xp; ep.ypArcsec = yp;
    tide::Coeffs cs, co;
    tide::coefficients(ep, true, true, cs);
    tide::coefficients(ep, false, false, co);
    for (int n = 0; n < 7; ++n)
        for (int m = 0; m < 7; ++m) {
            solidC[7 * n + m] = cs.C[n][m]; solidS[7 * n + m] = cs.S[n][m];
            oceanC[7 * n + m] = co.C[n][m]; oceanS[7 * n + m] = co.S[n][m];
        }
    tideGradient(ep, r, cs, 4, acc_solid);
    tideGradient(ep, r, co, 6, acc_ocean);
    const double mu = tide::kMuEarth, c = tide::kLight;
    const double rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    const double vv = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const double rv = r[0] * v[0] + r[1] * v[1] + r[2] * v[2];
    const double f = mu / (c * c * pow(rr, 3.0));
    for (int i = 0; i < 3; ++i) acc_rel[i] = f * ((4.0 * mu / rr - vv * vv) * r[i] + 4.0 * rv * v[i]);
}

void oracle_earth_rotation(const OracleEnv* env, double et, double R[9], double w[3]) {
    V3 ww;
    earthRotation(*env, et, R, &ww);
    w[0] = ww.x; w[1] = ww.y; w[2] = ww.z;
}

void oracle_body_position(const OracleEnv* env, double et, int body, int center, double out[3]) {
    const V3 p = position(*env, et, body, center);
    out[0] = p.x; out[1] = p.y; out[2] = p.z;
}

}  // extern "C"
