// The reference's own empirical-model sources as C functions for the CPU
// oracle (test infrastructure; the object goes to oracle/_ref/ only and is
// linked into the oracle library, never into the product).
//
// Compiles, unchanged, the reference's NRLMSISE-00 model
// (src/common/engine/paraHPOP/model/environment/atmosphere/detail/Nrlmsise00Model.inl
// and Nrlmsise00Data.inl, instantiated as Nrlmsise00.cu:53-78 does for the
// CPU backend) and its IERS 2010 / FES2004 tide coefficient code
// (src/common/engine/paraHPOP/model/accelerations/hpop_compat/HpopCorrections.h:
// solidCoefficients :326, oceanCoefficients :331).  With these the oracle's
// drag density and tide coefficient sets are the reference's arithmetic, not
// a second copy of the product's.
//
// Build (oracle/Makefile.ref target models):
//   g++ -O3 -march=x86-64-v3 -fPIC -std=c++17 -I$REF/src/common/engine -c oracle/ref_models.cpp
#include <cmath>
#include <cstdio>

namespace refmodels {
struct nrlmsise_flags { int switches[24]; double sw[24]; double swc[24]; };
struct ap_array { double a[7]; };
struct nrlmsise_input {
    int year, doy;
    double sec, alt, g_lat, g_long, lst, f107A, f107, ap;
    ap_array* ap_a;
};
struct nrlmsise_output { double d[9]; double t[2]; };
#define NRL_COEFFICIENT static
#define NRL_FUNCTION
#include "paraHPOP/model/environment/atmosphere/detail/Nrlmsise00Data.inl"
struct NrlModel {
#include "paraHPOP/model/environment/atmosphere/detail/Nrlmsise00Model.inl"
};
#undef NRL_COEFFICIENT
#undef NRL_FUNCTION
}  // namespace refmodels

#include "paraHPOP/model/accelerations/hpop_compat/HpopCorrections.h"

extern "C" {

// Total mass density (kg/m^3) of gtd7d with every switch on and switch 9 =
// -1 (the 3-hour ap history), the reference CPU backend's setting.
double ref_nrl_density(int doy, double sec, double alt, double glat, double glong, double lst, double f107A,
                       double f107, double ap, const double ap_a[7]) {
    refmodels::ap_array aps{};
    for (int k = 0; k < 7; ++k) aps.a[k] = ap_a[k];
    refmodels::nrlmsise_input in{};
    in.year = 0;
    in.doy = doy;
    in.sec = sec;
    in.alt = alt;
    in.g_lat = glat;
    in.g_long = glong;
    in.lst = lst;
    in.f107A = f107A;
    in.f107 = f107;
    in.ap = ap;
    in.ap_a = &aps;
    refmodels::nrlmsise_flags fl{};
    for (int k = 0; k < 24; ++k) fl.switches[k] = 1;
    fl.switches[9] = -1;
    refmodels::nrlmsise_output out{};
    refmodels::NrlModel model{};
    model.gtd7d(&in, &fl, &out);
    return out.d[5];
}

// Solid (solid != 0; zero-tide or tide-free static field) or ocean tide
// coefficient corrections C[n][m], S[n][m] (7 x 7, row-major) for an epoch:
// E = ICRF -> ITRF rotation (row-major), Sun and Moon geocentric ICRF (m),
// UTC MJD, UT1 - UTC and TT - UTC (s), pole coordinates (arcsec).
void ref_tide_coefficients(const double E[9], const double sun[3], const double moon[3], double mjdUtc, double ut1Utc,
                           double ttUtc, double xp, double yp, int zeroTide, int solid, double C[49], double S[49]) {
    namespace h = paraHPOP::model::accelerations::hpop;
    h::Input in{};
    for (int k = 0; k < 3; ++k) {
        in.sun[k] = sun[k];
        in.moon[k] = moon[k];
    }
    for (int k = 0; k < 9; ++k) in.E[k] = E[k];
    in.mjdUtc = mjdUtc;
    in.ut1Utc = ut1Utc;
    in.ttUtc = ttUtc;
    in.xpArcsec = xp;
    in.ypArcsec = yp;
    h::Constants k;
    k.zeroTide = zeroTide != 0;
    h::Coefficients c;
    if (solid)
        h::solidCoefficients(in, k, c);
    else
        h::oceanCoefficients(in, k, c);
    for (int n = 0; n < 7; ++n)
        for (int m = 0; m < 7; ++m) {
            C[7 * n + m] = c.C[n][m];
            S[7 * n + m] = c.S[n][m];
        }
}

}  // extern "C"
