// Known-answer generator built from the reference's own model sources
// (test infrastructure; output goes to oracle/_ref/ only).
//
// Compiles, unchanged, the reference's NRLMSISE-00 model
// (src/common/engine/paraHPOP/model/environment/atmosphere/detail/Nrlmsise00Model.inl
// and Nrlmsise00Data.inl, instantiated the way Nrlmsise00.cu:53-78 does for
// the CPU backend) and its IERS 2010 / FES2004 tide and relativity code
// (src/common/engine/paraHPOP/model/accelerations/hpop_compat/HpopCorrections.h),
// then evaluates them on a fixed input grid read from stdin and prints one
// JSON object per line.  tests/golden/make_golden.py drives it.
//
// Build (oracle/Makefile.ref target kat):
//   g++ -O2 -std=c++17 -I$REF/src/common/engine oracle/ref_kat.cpp -o oracle/_ref/ref_kat
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

namespace refnrl {
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
}  // namespace refnrl

#include "paraHPOP/model/accelerations/hpop_compat/HpopCorrections.h"

static void nrl_case() {
    // doy sec alt glat glong lst f107A f107 ap a0..a6
    double v[16];
    for (double& x : v)
        if (std::scanf("%lf", &x) != 1) return;
    refnrl::ap_array aps{};
    for (int k = 0; k < 7; ++k) aps.a[k] = v[9 + k];
    refnrl::nrlmsise_input in{};
    in.year = 0;
    in.doy = (int)v[0];
    in.sec = v[1];
    in.alt = v[2];
    in.g_lat = v[3];
    in.g_long = v[4];
    in.lst = v[5];
    in.f107A = v[6];
    in.f107 = v[7];
    in.ap = v[8];
    in.ap_a = &aps;
    refnrl::nrlmsise_flags fl{};
    for (int k = 0; k < 24; ++k) fl.switches[k] = 1;
    fl.switches[9] = -1;
    refnrl::nrlmsise_output out{};
    refnrl::NrlModel model{};
    model.gtd7d(&in, &fl, &out);
    std::printf("{\"kind\":\"nrl\",\"rho\":%.17g}\n", out.d[5]);
}

static void tide_case() {
    namespace h = paraHPOP::model::accelerations::hpop;
    h::Input in{};
    double* f[] = {in.r, in.v, in.sun, in.moon};
    for (double* p : f)
        for (int k = 0; k < 3; ++k)
            if (std::scanf("%lf", &p[k]) != 1) return;
    for (int k = 0; k < 9; ++k) std::scanf("%lf", &in.E[k]);
    std::scanf("%lf %lf %lf %lf %lf", &in.mjdUtc, &in.ut1Utc, &in.ttUtc, &in.xpArcsec, &in.ypArcsec);
    h::Constants k;
    h::Coefficients cs, co;
    h::solidCoefficients(in, k, cs);
    h::oceanCoefficients(in, k, co);
    const h::Outputs o = h::evaluate(in, k, true, true, true);
    std::printf("{\"kind\":\"tide\",\"solidC\":[");
    for (int n = 0; n < 7; ++n)
        for (int m = 0; m < 7; ++m) std::printf("%s%.17g", (n || m) ? "," : "", cs.C[n][m]);
    std::printf("],\"solidS\":[");
    for (int n = 0; n < 7; ++n)
        for (int m = 0; m < 7; ++m) std::printf("%s%.17g", (n || m) ? "," : "", cs.S[n][m]);
    std::printf("],\"oceanC\":[");
    for (int n = 0; n < 7; ++n)
        for (int m = 0; m < 7; ++m) std::printf("%s%.17g", (n || m) ? "," : "", co.C[n][m]);
    std::printf("],\"oceanS\":[");
    for (int n = 0; n < 7; ++n)
        for (int m = 0; m < 7; ++m) std::printf("%s%.17g", (n || m) ? "," : "", co.S[n][m]);
    std::printf("],\"solid\":[%.17g,%.17g,%.17g],\"ocean\":[%.17g,%.17g,%.17g],\"rel\":[%.17g,%.17g,%.17g]}\n",
                o.solid[0], o.solid[1], o.solid[2], o.ocean[0], o.ocean[1], o.ocean[2], o.relativity[0],
                o.relativity[1], o.relativity[2]);
}

int main() {
    char kind[16];
    while (std::scanf("%15s", kind) == 1) {
        if (!std::strcmp(kind, "nrl")) nrl_case();
        else if (!std::strcmp(kind, "tide")) tide_case();
    }
    return 0;
}
