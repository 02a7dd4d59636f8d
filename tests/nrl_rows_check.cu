// Host check of the NRLMSISE-00 globe7 coefficient rows (nrl_fast.cuh,
// nrlGlobeRows): for random inputs, the dot products of the rows with the 71
// monomials (plus the latitude-dependent ap rows of pt and pd[0]) against the
// term-by-term globe7 of the straight restatement (nrlmsise00.cuh).  Prints
// the largest absolute difference over all tables and inputs.
#include <cmath>
#include <cstdio>
#include <random>

#include "nrl_fast.cuh"

using namespace phop;

static double monomial(int i, const nrl::Model<double>& m, double lon, double sec) {
    const double dgtr = 1.74533E-2, sr = 7.2722E-5;
    const double cgl = cos(dgtr * lon), sgl = sin(dgtr * lon);
    const double c2gl = cos(2.0 * dgtr * lon), s2gl = sin(2.0 * dgtr * lon);
    const double cs = cos(sr * sec), ss = sin(sr * sec);
    const double x = m.plg[0][1], x2 = x * x;
    const double U1 = cs * c2gl - ss * s2gl, U2 = ss * c2gl + cs * s2gl;
    const auto& P = m.plg;
    const double mono[9] = {x, P[0][3], P[0][5], x2, x * P[0][3], x * P[0][5], x2 * x, x2 * P[0][3], x2 * P[0][5]};
    if (i == 0) return 1.0;
    if (i == 1) return x;
    if (i <= 6) return P[0][i];
    const int d1[4] = {1, 2, 3, 5}, s1[4] = {2, 3, 4, 5};
    if (i <= 10) return P[1][d1[i - 7]] * m.ctloc;
    if (i <= 14) return P[1][d1[i - 11]] * m.stloc;
    if (i <= 18) return P[2][s1[i - 15]] * m.c2tloc;
    if (i <= 22) return P[2][s1[i - 19]] * m.s2tloc;
    const int t1[3] = {3, 4, 6};
    if (i <= 25) return P[3][t1[i - 23]] * m.s3tloc;
    if (i <= 28) return P[3][t1[i - 26]] * m.c3tloc;
    if (i <= 34) return P[1][i - 28] * cgl;
    if (i <= 40) return P[1][i - 34] * sgl;
    const int l1[3] = {2, 4, 6};
    if (i <= 43) return x * P[1][l1[i - 41]] * cgl;
    if (i <= 46) return x * P[1][l1[i - 44]] * sgl;
    if (i <= 55) return cs * mono[i - 47];
    if (i <= 64) return ss * mono[i - 56];
    const int u1[3] = {3, 5, 7};
    if (i <= 67) return P[2][u1[i - 65]] * U1;
    if (i <= 70) return P[2][u1[i - 68]] * U2;
    return 0.0;
}

int main() {
    std::mt19937_64 rng(11);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    const double apChoices[9] = {0, 3, 7, 15, 27, 48, 80, 132, 207};
    double worst = 0.0;
    int bad = 0;
    for (int trial = 0; trial < 500; ++trial) {
        nrl::Input<double> in{};
        in.doy = 1 + (int)(U(rng) * 365.0);
        in.sec = U(rng) * 86400.0;
        in.alt = 400.0;
        in.g_lat = -89.0 + 178.0 * U(rng);
        in.g_long = -180.0 + 360.0 * U(rng);
        in.lst = 24.0 * U(rng);
        in.f107A = 70.0 + 180.0 * U(rng);
        in.f107 = 70.0 + 230.0 * U(rng);
        for (int k = 0; k < 7; ++k) in.ap_a[k] = apChoices[(int)(U(rng) * 9.0) % 9];
        in.ap = in.ap_a[0];
        nrlf::NrlEpochBlock b;
        nrlf::nrlSlotBlock(in.doy, in.f107, in.f107A, in.ap_a, b);
        if (!b.valid) bad++;
        for (int t = 0; t < nrlf::kGlobeTasks; ++t) {
            const int k = nrlf::globeTaskTable(t);
            const double* p = nrlf::globeTable(k);
            nrl::Model<double> m{};
            m.g0Cached = false;
            m.prepareBasis(in);
            const double ref = m.globe7(p, in);
            double g = 0.0, ap = 0.0;
            for (int i = 0; i < nrlf::kGlobeBasis; ++i) {
                const double mi = monomial(i, m, in.g_long, in.sec);
                g += b.globeRows[i / 2][t][i % 2] * mi;
                if (k == 0) ap += b.globeRows[i / 2][nrlf::kApRowPt][i % 2] * mi;
                if (k == 2) ap += b.globeRows[i / 2][nrlf::kApRowPd0][i % 2] * mi;
            }
            if (k == 0 || k == 2) g += m.apt0 * ap;  // the table's own latitude-dependent ap response
            const double d = fabs(g - ref);
            if (!(d <= worst)) worst = d;
        }
    }
    printf("{\"max_abs_diff\": %.3e, \"invalid_blocks\": %d}\n", worst, bad);
    return 0;
}
