// NRLMSISE-00 total mass density for the step kernel, split into an
// epoch-only part and a per-object part.
//
// Same model and call sequence as nrlmsise00.cuh (gtd7d, switch 9 = -1), but
// every sub-expression that depends only on the UTC day and the 3-hour ap
// slot (day-of-year phases cd32/cd18/cd14/cd39, the F10.7 terms t[0], f1, f2,
// the six 3-hour-ap responses g0 of Eq. A24d) is evaluated once per (day,
// slot) into an NrlEpochBlock when the environment is loaded, and the
// per-object part evaluates only what depends on the seconds of day,
// latitude, longitude, local time and altitude.  Differences of angles are
// expanded with precomputed table constants (cos(x - p) = cos x cos p +
// sin x sin p) and integer powers are products; results agree with the
// straight restatement to rounding (checked against it by the tests).
//
// T is the arithmetic type of the per-object part (double, or float in
// split precision); the epoch block is always double.
#pragma once
#ifndef PHOP_NRL_ROLLED_GLOBE
#define PHOP_NRL_ROLLED_GLOBE 1
#endif
#include <math.h>

#include "nrlmsise00.cuh"

namespace phop {
namespace nrlf {

using namespace ::phop::nrl;  // coefficient tables

constexpr int kGlobeTables = 11;  // pt, ps, pd[0..8]
constexpr int kGlobSTables = 14;  // ptl[0..3], pma[0..9]

struct NrlGlobeEpoch {
    double cd32, cd18, cd14, cd39;
    double t0, f1, f2;            // F10.7 terms of globe7
    double g0[6];                 // Eq. A24d responses to ap[1..6]
    double c131, s131, c97, s97, c136, s136;  // table phase constants
    double c71, s71, c58, s58, c79, s79;      // cos / sin (sr p[k]) for the seconds-of-day phases
    double apt0;                  // sg0 ap response when it does not depend on latitude (p[138] == 0)
    int aptEpochOnly;             // 1: apt0 above holds it
    int pad;
};

struct NrlGlobSEpoch {
    double cd32, cd18, cd14, cd39;
    double lonA;  // p80 cos(dr(doy-p81)) + p85 cos(2dr(doy-p86))  (multiplies plg[0][1])
    double lonB;  // p83 cos(dr(doy-p84)) + p87 cos(2dr(doy-p88))
};

// globe7 as dot products.  Every term of G(L) (globe7) is a coefficient that
// depends only on the table and the (day, ap slot) times a monomial of the
// object's Legendre functions and its local-time, longitude and seconds-of-day
// phases; the 71 monomials of globeMonomial cover every table.  Per block the
// rows hold those coefficients in task order (rows 0..10), with each table's
// ap response folded in where it is epoch-only; the two tables whose ap
// response depends on latitude (pt and pd[0]: p[138] != 0) keep their ap
// terms apart in rows 11 and 12, scaled per object.  Rows 13..15 are zero so
// that every lane split takes the same number of rows.  Stored pair-major:
// globeRows[q][t] = row t's coefficients of monomials 2q and 2q + 1, so the
// L lanes of a group, reading rows rL .. rL + L - 1 of one pair, read one
// contiguous 16L-byte span (one cache line for L <= 8).
constexpr int kGlobeBasis = 72;  // 71 monomials and a zero pad (16-byte rows)
constexpr int kGlobeRows = 16;
constexpr int kApRowPt = 11, kApRowPd0 = 12;

// Per-species parameters of the thermospheric number densities (gts7 of
// Nrlmsise00Model.inl:522-720), one row per species in the lane order of
// Fast::gts7 (N, H, O, O2, Ar, He, N2): every species is
//   d = main(g, pdm0, pd0, xm, alpha)
//   if z <= lim:  d = dnet(d, dm, zhm28, xmm, xm) * ccor2(z, r1, c1h1, c1zh, c1h2) * ccor2(z, r2, c2h, c2zh, c2h)
//   d *= ccor2(z, rc, cah1, cazh, cah2)
// with r1 = log(b28 k1 k2 / b) (rlLog) or k1, ccor(z, r, h, zh) written as
// ccor2 with h2 = h (the same value bit for bit), and a zero r for a factor
// that species does not have (ccor2 with r = 0 is exactly 1).
enum NrlSpeciesParam {
    kSpPdm0, kSpPd0, kSpXm, kSpAlpha, kSpLim, kSpRlLog, kSpK1, kSpK2, kSpC1H1, kSpC1Zh, kSpC1H2,
    kSpR2, kSpC2H, kSpC2Zh, kSpRc, kSpCaH1, kSpCaZh, kSpCaH2, kSpParams
};
constexpr int kNrlSpecies = 7;

struct NrlEpochBlock {
    alignas(16) double globeRows[kGlobeBasis / 2][kGlobeRows][2];
    double species[kNrlSpecies][kSpParams];
    NrlGlobeEpoch ge[kGlobeTables];
    NrlGlobSEpoch gs[kGlobSTables];
    double dfa;
    double f107A;
    int doy;
    int valid;
};

#if defined(__CUDACC__)

// Global-memory copies of the coefficient tables, read through L1 where the
// lanes of a warp evaluate different tables at once (constant-bank reads
// serialise on distinct addresses).
#define PHOP_NRL_TABLE(name, count) static __device__ const double gdev_##name[count]
#include "tables/nrlmsise00_coeffs.inc"
#undef PHOP_NRL_TABLE

// table order of the globe7 calls: pt, ps, pd[0..8]
__host__ __device__ __forceinline__ const double* globeTable(int k) {
    return k == 0 ? NRLT(pt) : k == 1 ? NRLT(ps) : NRLT(pd) + 150 * (k - 2);
}
__device__ __forceinline__ const double* globSTableGlobal(int k) {
    return k < 4 ? gdev_nrl_ptl + 100 * k : gdev_nrl_pma + 100 * (k - 4);
}
__device__ __forceinline__ const double* globeTableGlobal(int k) {
    return k == 0 ? gdev_nrl_pt : k == 1 ? gdev_nrl_ps : gdev_nrl_pd + 150 * (k - 2);
}

// The globe7 evaluations of one gts7 call in task order: tinf (pt), g0 (ps),
// tlb (pd[3]), then N2, He, O, O2, Ar, H, N and anomalous O (pd[2], pd[0],
// pd[1], pd[4] .. pd[8]).
constexpr int kGlobeTasks = 11;
__host__ __device__ __forceinline__ int globeTaskTable(int t) {
    return t == 0 ? 0 : t == 1 ? 1 : t == 2 ? 5 : t == 3 ? 4 : t == 4 ? 2 : t == 5 ? 3 : t;
}
__host__ __device__ __forceinline__ const double* globSTable(int k) {
    return k < 4 ? NRLT(ptl) + 100 * k : NRLT(pma) + 100 * (k - 4);
}

// sg0 (Eq. A24a) from the ap decay factor and the six 3-hour responses g0
template <typename T>
__host__ __device__ __forceinline__ T sg0FromExp(T exp1, const double g0[6]) {
    const T e2 = exp1 * exp1, e3 = e2 * exp1, e4 = e2 * e2, e8 = e4 * e4, e12 = e8 * e4;
    const T e19 = e12 * e4 * e3;
    const T sumex = T(1.0) + (T(1.0) - e19) / (T(1.0) - exp1) * sqrt(exp1);
    return (T(g0[0]) + (T(g0[1]) * exp1 + T(g0[2]) * e2 + T(g0[3]) * e3
                        + (T(g0[4]) * e4 + T(g0[5]) * e12) * (T(1.0) - e8) / (T(1.0) - exp1)))
        / sumex;
}

// Coefficient rows of one (day, ap slot) block (layout above; monomial
// order in globeMonomial).  The expansion is exact algebra of globe7
// (Nrlmsise00Model.inl:686 globe7): products of the table's factors that do
// not depend on the object (f1, f2, 1 + p80 dfa, the UT factor
// (1 + p95 x)(1 + p81 dfa)(1 + p119 cd14 x) multiplied out in powers of
// x = P(1,0), and the phase constants of cos(a - p)) are formed here once.
// Returns false when a table other than pt / pd[0] has a latitude-dependent
// ap response (the coefficient set is fixed, so this never happens).
__host__ __device__ inline bool nrlGlobeRows(NrlEpochBlock& b) {
    bool ok = true;
    double M[kGlobeRows][kGlobeBasis];
    for (int r = 0; r < kGlobeRows; ++r)
        for (int i = 0; i < kGlobeBasis; ++i) M[r][i] = 0.0;
    const double dfa = b.dfa;
    for (int t = 0; t < kGlobeTasks; ++t) {
        const int k = globeTaskTable(t);
        const double* p = globeTable(k);
        const NrlGlobeEpoch& g = b.ge[k];
        double* E = M[t];
        double A[kGlobeBasis];
        for (int i = 0; i < kGlobeBasis; ++i) A[i] = 0.0;
        const double f1 = g.f1, f2 = g.f2, cd14 = g.cd14;
        // time-independent, annual / semiannual
        E[0] = p[30] + g.t0 + p[18] * g.cd32 + p[15] * g.cd18;
        E[1] = p[26] + f1 * p[9] * cd14 + p[37] * g.cd39;
        E[2] = p[1] + p[14] * dfa + p[16] * g.cd18;
        E[3] = f1 * p[10] * cd14;
        E[4] = p[2];
        E[6] = p[22];
        // diurnal (P11, P12, P13, P15) x (cos, sin) of the local time
        E[7] = f2 * p[3];
        E[8] = f2 * p[11] * cd14;
        E[9] = f2 * p[4];
        E[10] = f2 * p[27];
        E[11] = f2 * p[6];
        E[12] = f2 * p[12] * cd14;
        E[13] = f2 * p[7];
        E[14] = f2 * p[28];
        // semidiurnal (P22, P23, P24, P25)
        E[15] = f2 * p[5];
        E[16] = f2 * p[23] * cd14;
        E[17] = f2 * p[41];
        E[18] = f2 * p[35] * cd14;
        E[19] = f2 * p[8];
        E[20] = f2 * p[33] * cd14;
        E[21] = f2 * p[42];
        E[22] = f2 * p[36] * cd14;
        // terdiurnal (P33, P34, P36) x (sin, cos)
        E[23] = f2 * p[39];
        E[24] = f2 * p[93] * cd14;
        E[25] = f2 * p[46] * cd14;
        E[26] = f2 * p[40];
        E[27] = f2 * p[94] * cd14;
        E[28] = f2 * p[48] * cd14;
        // longitudinal (P11 .. P16) x (cos, sin) of the longitude
        const double lf = 1.0 + p[80] * dfa;
        E[29] = lf * (p[103] + p[109] * cd14);
        E[30] = lf * p[64];
        E[31] = lf * (p[104] + p[110] * cd14);
        E[32] = lf * p[65];
        E[33] = lf * (p[105] + p[111] * cd14);
        E[34] = lf * p[66];
        E[35] = lf * (p[106] + p[112] * cd14);
        E[36] = lf * p[90];
        E[37] = lf * (p[107] + p[113] * cd14);
        E[38] = lf * p[91];
        E[39] = lf * (p[108] + p[114] * cd14);
        E[40] = lf * p[92];
        // UT: x^q {x, P30, P50} x (cos, sin) of the seconds-of-day phase
        const double uf = 1.0 + p[81] * dfa;
        const double w[3] = {1.0, p[95] + p[119] * cd14, p[95] * p[119] * cd14};
        const double v[3] = {p[68], p[69], p[70]};
        for (int q = 0; q < 3; ++q)
            for (int m = 0; m < 3; ++m) {
                E[47 + 3 * q + m] = uf * w[q] * v[m] * g.c71;
                E[56 + 3 * q + m] = uf * w[q] * v[m] * g.s71;
            }
        // mixed UT / longitude: (P23, P25, P27) x (cos, sin)(sr sec + 2 lon)
        const double q79 = 1.0 + p[137] * dfa;
        for (int i = 0; i < 3; ++i) {
            const double c = p[76 + i];
            E[65 + i] = q79 * c * g.c79;
            E[68 + i] = q79 * c * g.s79;
        }
        if (p[51] != 0.0) {
            // magnetic activity terms, multiplied by the ap response apt0
            A[0] = p[50];
            A[2] = p[96];
            A[4] = p[54];
            A[1] = p[125] * cd14;
            A[3] = p[126] * cd14;
            A[5] = p[127] * cd14;
            A[7] = p[128] * g.c131;
            A[9] = p[129] * g.c131;
            A[10] = p[130] * g.c131;
            A[11] = p[128] * g.s131;
            A[13] = p[129] * g.s131;
            A[14] = p[130] * g.s131;
            const int k97[3] = {52, 98, 67};
            for (int i = 0; i < 3; ++i) {
                const double c = p[k97[i]];
                A[30 + 2 * i] += c * g.c97;
                A[36 + 2 * i] += c * g.s97;
                A[41 + i] = p[132] * c * g.c97;
                A[44 + i] = p[132] * c * g.s97;
            }
            for (int i = 0; i < 3; ++i) {
                const double c = p[133 + i] * cd14;
                A[29 + 2 * i] += c * g.c136;
                A[35 + 2 * i] += c * g.s136;
            }
            for (int i = 0; i < 3; ++i) {
                A[47 + i] += p[55 + i] * g.c58;
                A[56 + i] += p[55 + i] * g.s58;
            }
            if (g.aptEpochOnly) {
                for (int i = 0; i < kGlobeBasis; ++i) E[i] += g.apt0 * A[i];
            } else if (k == 0 || k == 2) {
                double* R = M[k == 0 ? kApRowPt : kApRowPd0];
                for (int i = 0; i < kGlobeBasis; ++i) R[i] = A[i];
            } else {
                ok = false;
            }
        }
    }
    for (int q = 0; q < kGlobeBasis / 2; ++q)
        for (int r = 0; r < kGlobeRows; ++r) {
            b.globeRows[q][r][0] = M[r][2 * q];
            b.globeRows[q][r][1] = M[r][2 * q + 1];
        }
    return ok;
}

// Species rows (layout above) from the model tables; the F10.7 factor of the
// O and O2 terms is the block's.
__host__ __device__ inline void nrlSpeciesRows(NrlEpochBlock& b) {
    const double f107Term = 1.0 + NRL_PDL(0)[23] * (b.f107A - 150.0);
    auto row = [&](int r, double pdm0, double pd0, double xm, double alpha, double lim) {
        double* q = b.species[r];
        for (int k = 0; k < kSpParams; ++k) q[k] = 0.0;
        q[kSpPdm0] = pdm0;
        q[kSpPd0] = pd0;
        q[kSpXm] = xm;
        q[kSpAlpha] = alpha;
        q[kSpLim] = lim;
        q[kSpK2] = 1.0;
        q[kSpC1H1] = q[kSpC1H2] = q[kSpC2H] = q[kSpCaH1] = q[kSpCaH2] = 1.0;
        return q;
    };
    auto c1 = [](double* q, int rlLog, double k1, double k2, double h1, double zh, double h2) {
        q[kSpRlLog] = rlLog;
        q[kSpK1] = k1;
        q[kSpK2] = k2;
        q[kSpC1H1] = h1;
        q[kSpC1Zh] = zh;
        q[kSpC1H2] = h2;
    };
    auto c2 = [](double* q, double r, double h, double zh) {
        q[kSpR2] = r;
        q[kSpC2H] = h;
        q[kSpC2Zh] = zh;
    };
    double* q;
    // N
    q = row(0, NRL_PDM(6, 0), NRL_PD(7)[0], 14.0, 0.0, 450.0);
    c1(q, 1, NRL_PDM(6, 1), fabs(NRL_PDL(0)[2]), NRL_PDM(6, 5) * NRL_PDL(0)[1], NRL_PDM(6, 4) * NRL_PDL(0)[0],
       NRL_PDM(6, 5) * NRL_PDL(0)[1]);
    c2(q, NRL_PDM(6, 3) * NRL_PDL(0)[5], NRL_PDM(6, 7) * NRL_PDL(0)[4], NRL_PDM(6, 6) * NRL_PDL(0)[3]);
    // H
    q = row(1, NRL_PDM(5, 0), NRL_PD(6)[0], 1.0, -0.38, 320.0);
    c1(q, 1, NRL_PDM(5, 1), fabs(NRL_PDL(1)[17]), NRL_PDM(5, 5) * NRL_PDL(1)[11], NRL_PDM(5, 4) * NRL_PDL(1)[10],
       NRL_PDM(5, 5) * NRL_PDL(1)[11]);
    c2(q, NRL_PDM(5, 3) * NRL_PDL(1)[20], NRL_PDM(5, 7) * NRL_PDL(1)[19], NRL_PDM(5, 6) * NRL_PDL(1)[18]);
    // O: constant r1 with a two-scale-height correction
    q = row(2, NRL_PDM(1, 0), NRL_PD(1)[0], 16.0, 0.0, 300.0);
    c1(q, 0, NRL_PDM(1, 1) * NRL_PDL(1)[16] * f107Term, 1.0, NRL_PDM(1, 5) * NRL_PDL(1)[3],
       NRL_PDM(1, 4) * NRL_PDL(1)[2], NRL_PDM(1, 5) * NRL_PDL(1)[4]);
    c2(q, NRL_PDM(1, 3) * NRL_PDL(1)[14], NRL_PDM(1, 7) * NRL_PDL(1)[13], NRL_PDM(1, 6) * NRL_PDL(1)[12]);
    // O2, with its correction at every altitude
    q = row(3, NRL_PDM(3, 0), NRL_PD(4)[0], 32.0, 0.0, 250.0);
    c1(q, 1, NRL_PDM(3, 1), 1.0, NRL_PDM(3, 5) * NRL_PDL(1)[7], NRL_PDM(3, 4) * NRL_PDL(1)[6],
       NRL_PDM(3, 5) * NRL_PDL(1)[7]);
    q[kSpRc] = NRL_PDM(3, 3) * NRL_PDL(1)[23] * f107Term;
    q[kSpCaH1] = NRL_PDM(3, 7) * NRL_PDL(1)[22];
    q[kSpCaZh] = NRL_PDM(3, 6) * NRL_PDL(1)[21];
    q[kSpCaH2] = NRL_PDM(3, 7) * NRL_PDL(0)[22];
    // Ar
    q = row(4, NRL_PDM(4, 0), NRL_PD(5)[0], 40.0, 0.17, 240.0);
    c1(q, 1, NRL_PDM(4, 1), 1.0, NRL_PDM(4, 5) * NRL_PDL(1)[9], NRL_PDM(4, 4) * NRL_PDL(1)[8],
       NRL_PDM(4, 5) * NRL_PDL(1)[9]);
    // He (z < 200 km: the largest double below 200)
    q = row(5, NRL_PDM(0, 0), NRL_PD(0)[0], 4.0, -0.38, 199.99999999999997);
    c1(q, 1, NRL_PDM(0, 1), 1.0, NRL_PDM(0, 5) * NRL_PDL(1)[1], NRL_PDM(0, 4) * NRL_PDL(1)[0],
       NRL_PDM(0, 5) * NRL_PDL(1)[1]);
    // N2: mixing only (below 160 km)
    row(6, NRL_PDM(2, 0), NRL_PD(2)[0], 28.0, 0.0, 160.0);
}

// (day, ap slot) part: day of year, F10.7 of the previous day, 81-day mean,
// ap history (as Nrlmsise00.cu:207-235 fills them).
__host__ __device__ inline void nrlSlotBlock(int doy, double f107, double f107A, const double apa[7],
                                             NrlEpochBlock& b) {
    const double dr = 1.72142E-2, sr = 7.2722E-5;
    const double df = f107 - f107A;
    const double dfa = f107A - 150.0;
    b.dfa = dfa;
    b.f107A = f107A;
    b.doy = doy;
    b.valid = 1;
    const double dd = (double)doy;
    for (int k = 0; k < kGlobeTables; ++k) {
        const double* p = globeTable(k);
        NrlGlobeEpoch& g = b.ge[k];
        g.cd32 = cos(dr * (dd - p[31]));
        g.cd18 = cos(2.0 * dr * (dd - p[17]));
        g.cd14 = cos(dr * (dd - p[13]));
        g.cd39 = cos(2.0 * dr * (dd - p[38]));
        g.t0 = p[19] * df * (1.0 + p[59] * dfa) + p[20] * df * df + p[21] * dfa + p[29] * (dfa * dfa);
        g.f1 = 1.0 + (p[47] * dfa + p[19] * df + p[20] * df * df);
        g.f2 = 1.0 + (p[49] * dfa + p[19] * df + p[20] * df * df);
        g.c71 = cos(sr * p[71]);
        g.s71 = sin(sr * p[71]);
        g.c58 = cos(sr * p[58]);
        g.s58 = sin(sr * p[58]);
        g.c79 = cos(sr * p[79]);
        g.s79 = sin(sr * p[79]);
        for (int i = 0; i < 6; ++i) g.g0[i] = nrl::Model<double>::g0(apa[i + 1], p);
        g.c131 = cos(0.2618 * p[131]);
        g.s131 = sin(0.2618 * p[131]);
        g.c97 = cos(1.74533E-2 * p[97]);
        g.s97 = sin(1.74533E-2 * p[97]);
        g.c136 = cos(1.74533E-2 * p[136]);
        g.s136 = sin(1.74533E-2 * p[136]);
        // tables whose ap-decay rate has no latitude term: the whole sg0
        // response is epoch-only
        g.aptEpochOnly = (p[51] != 0.0 && p[138] == 0.0) ? 1 : 0;
        g.apt0 = 0.0;
        if (g.aptEpochOnly) {
            double exp1 = exp(-10800.0 * fabs(p[51]));
            if (exp1 > 0.99999) exp1 = 0.99999;
            g.apt0 = sg0FromExp(exp1, g.g0);
        }
    }
    if (!nrlGlobeRows(b)) b.valid = 0;
    nrlSpeciesRows(b);
    for (int k = 0; k < kGlobSTables; ++k) {
        const double* p = globSTable(k);
        NrlGlobSEpoch& g = b.gs[k];
        g.cd32 = cos(dr * (dd - p[31]));
        g.cd18 = cos(2.0 * dr * (dd - p[17]));
        g.cd14 = cos(dr * (dd - p[13]));
        g.cd39 = cos(2.0 * dr * (dd - p[38]));
        g.lonA = p[80] * cos(dr * (dd - p[81])) + p[85] * cos(2.0 * dr * (dd - p[86]));
        g.lonB = p[83] * cos(dr * (dd - p[84])) + p[87] * cos(2.0 * dr * (dd - p[88]));
    }
}

// Mesosphere temperature nodes and the N2 mixing density of one call, kept
// apart from Fast so that only this small block needs an address (the
// out-of-line densu and lower-atmosphere paths write and read it) while the
// rest of the per-object state stays in registers.
template <typename T>
struct NrlMeso {
    T tn1[5], tgn1[2];
    T dm28;
};

// Per-object part.  Returns the gtd7d total mass density in kg/m^3.
template <typename T>
struct Fast {
    const NrlEpochBlock& eb;
    T gsurf, re;
    T plg[4][9];
    T ctloc, stloc, c2tloc, s2tloc, s3tloc, c3tloc;
    T cgl, sgl, c2gl, s2gl;  // cos / sin of (dgtr * g_long) and of twice it
    T glat, absLat, gLong;
    T csec, ssec;  // cos / sin (sr * seconds of day)
    T apt0;

    __device__ __forceinline__ Fast(const NrlEpochBlock& b, double sec) : eb(b) {
        double sc, cc;
        sincos(7.2722E-5 * sec, &sc, &cc);
        csec = T(cc);
        ssec = T(sc);
    }

    __device__ __forceinline__ T zeta(T zz, T zl) const { return (zz - zl) * (re + zl) * rcp(re + zz); }

    __device__ __forceinline__ void basis(T lat, T lst) {
        const T dgtr = T(1.74533E-2), hr = T(0.2618);
        T c, s;
        sincos(lat * dgtr, &c, &s);  // c = sin(lat), s = cos(lat)
        const T c2 = c * c, c4 = c2 * c2, s2 = s * s;
        plg[0][1] = c;
        plg[0][2] = T(0.5) * (T(3.0) * c2 - T(1.0));
        plg[0][3] = T(0.5) * (T(5.0) * c * c2 - T(3.0) * c);
        plg[0][4] = (T(35.0) * c4 - T(30.0) * c2 + T(3.0)) / T(8.0);
        plg[0][5] = (T(63.0) * c2 * c2 * c - T(70.0) * c2 * c + T(15.0) * c) / T(8.0);
        plg[0][6] = (T(11.0) * c * plg[0][5] - T(5.0) * plg[0][4]) / T(6.0);
        plg[1][1] = s;
        plg[1][2] = T(3.0) * c * s;
        plg[1][3] = T(1.5) * (T(5.0) * c2 - T(1.0)) * s;
        plg[1][4] = T(2.5) * (T(7.0) * c2 * c - T(3.0) * c) * s;
        plg[1][5] = T(1.875) * (T(21.0) * c4 - T(14.0) * c2 + T(1.0)) * s;
        plg[1][6] = (T(11.0) * c * plg[1][5] - T(6.0) * plg[1][4]) / T(5.0);
        plg[2][2] = T(3.0) * s2;
        plg[2][3] = T(15.0) * s2 * c;
        plg[2][4] = T(7.5) * (T(7.0) * c2 - T(1.0)) * s2;
        plg[2][5] = T(3.0) * c * plg[2][4] - T(2.0) * plg[2][3];
        plg[2][6] = (T(11.0) * c * plg[2][5] - T(7.0) * plg[2][4]) / T(4.0);
        plg[2][7] = (T(13.0) * c * plg[2][6] - T(8.0) * plg[2][5]) / T(5.0);
        plg[3][3] = T(15.0) * s2 * s;
        plg[3][4] = T(105.0) * s2 * s * c;
        plg[3][5] = (T(9.0) * c * plg[3][4] - T(7.) * plg[3][3]) / T(2.0);
        plg[3][6] = (T(11.0) * c * plg[3][5] - T(8.) * plg[3][4]) / T(3.0);
        // multiples of the local-time and longitude angles by the double- and
        // triple-angle identities (one sincos each)
        sincos(hr * lst, &stloc, &ctloc);
        s2tloc = T(2.0) * stloc * ctloc;
        c2tloc = (ctloc - stloc) * (ctloc + stloc);
        s3tloc = stloc * (T(3.0) - T(4.0) * stloc * stloc);
        c3tloc = ctloc * (T(4.0) * ctloc * ctloc - T(3.0));
        sincos(dgtr * gLong, &sgl, &cgl);
        s2gl = T(2.0) * sgl * cgl;
        c2gl = (cgl - sgl) * (cgl + sgl);
    }

    __device__ __forceinline__ T glob7s(int k) const { return glob7sAt(k, globSTable(k)); }

    __device__ __forceinline__ T glob7sAt(int k, const double* __restrict__ p) const {
        const NrlGlobSEpoch& g = eb.gs[k];
        const T dfa = T(eb.dfa);
        T tt = T(p[21]) * dfa;
        tt += T(p[1]) * plg[0][2] + T(p[2]) * plg[0][4] + T(p[22]) * plg[0][6] + T(p[26]) * plg[0][1]
            + T(p[14]) * plg[0][3] + T(p[59]) * plg[0][5];
        tt += (T(p[18]) + T(p[47]) * plg[0][2] + T(p[29]) * plg[0][4]) * T(g.cd32);
        tt += (T(p[15]) + T(p[16]) * plg[0][2] + T(p[30]) * plg[0][4]) * T(g.cd18);
        tt += (T(p[9]) * plg[0][1] + T(p[10]) * plg[0][3] + T(p[20]) * plg[0][5]) * T(g.cd14);
        tt += (T(p[37]) * plg[0][1]) * T(g.cd39);
        {
            const T t71 = T(p[11]) * plg[1][2] * T(g.cd14);
            const T t72 = T(p[12]) * plg[1][2] * T(g.cd14);
            tt += ((T(p[3]) * plg[1][1] + T(p[4]) * plg[1][3] + t71) * ctloc
                   + (T(p[6]) * plg[1][1] + T(p[7]) * plg[1][3] + t72) * stloc);
        }
        {
            const T t81 = (T(p[23]) * plg[2][3] + T(p[35]) * plg[2][5]) * T(g.cd14);
            const T t82 = (T(p[33]) * plg[2][3] + T(p[36]) * plg[2][5]) * T(g.cd14);
            tt += ((T(p[5]) * plg[2][2] + T(p[41]) * plg[2][4] + t81) * c2tloc
                   + (T(p[8]) * plg[2][2] + T(p[42]) * plg[2][4] + t82) * s2tloc);
        }
        tt += T(p[39]) * plg[3][3] * s3tloc + T(p[40]) * plg[3][3] * c3tloc;
        tt += (T(p[50]) * apt0 + T(p[96]) * plg[0][2] * apt0);
        tt += (T(1.0) + plg[0][1] * T(g.lonA) + T(g.lonB))
            * ((T(p[64]) * plg[1][2] + T(p[65]) * plg[1][4] + T(p[66]) * plg[1][6] + T(p[74]) * plg[1][1]
                + T(p[75]) * plg[1][3] + T(p[76]) * plg[1][5]) * cgl
               + (T(p[90]) * plg[1][2] + T(p[91]) * plg[1][4] + T(p[92]) * plg[1][6] + T(p[77]) * plg[1][1]
                  + T(p[78]) * plg[1][3] + T(p[79]) * plg[1][5]) * sgl);
        return tt;
    }

    // out of line and without `this`: only the rarer paths (below za, the
    // low-altitude species corrections) call it; the main species densities
    // use the direct form
    static __device__ __noinline__ T densu(T alt, T dlb, T tinf, T tlb, T xm, T alpha, T* tz, T zlb, T s2,
                                           const T* zn1, T re, T gsurf, NrlMeso<T>& ms) {
        auto zeta = [re](T zz, T zl) { return ((zz - zl) * (re + zl) / (re + zz)); };
        T* meso_tn1 = ms.tn1;
        T* meso_tgn1 = ms.tgn1;
        const T rgas = T(831.4);
        T xs[5], ys[5], y2out[5];
        T x = T(0), z1 = T(0), t1 = T(0), zgdif = T(0);
        const int mn1 = 5;
        const T za = zn1[0];
        T z = (alt > za) ? alt : za;
        const T zg2 = zeta(z, zlb);
        const T tt = tinf - (tinf - tlb) * exp(-s2 * zg2);
        const T ta = tt;
        *tz = tt;
        T densu_temp = *tz;
        if (alt < za) {
            const T q = (re + zlb) / (re + za);
            meso_tgn1[0] = (tinf - ta) * s2 * (q * q);
            meso_tn1[0] = ta;
            z = (alt > zn1[mn1 - 1]) ? alt : zn1[mn1 - 1];
            z1 = zn1[0];
            const T z2 = zn1[mn1 - 1];
            t1 = meso_tn1[0];
            const T t2 = meso_tn1[mn1 - 1];
            const T zg = zeta(z, z1);
            zgdif = zeta(z2, z1);
            for (int k = 0; k < mn1; k++) {
                xs[k] = zeta(zn1[k], z1) / zgdif;
                ys[k] = T(1.0) / meso_tn1[k];
            }
            const T r2 = (re + z2) / (re + z1);
            const T yd1 = -meso_tgn1[0] / (t1 * t1) * zgdif;
            const T yd2 = -meso_tgn1[1] / (t2 * t2) * zgdif * (r2 * r2);
            nrl::Model<T>::spline(xs, ys, mn1, yd1, yd2, y2out);
            x = zg / zgdif;
            const T y = nrl::Model<T>::splint(xs, ys, y2out, mn1, x);
            *tz = T(1.0) / y;
            densu_temp = *tz;
        }
        if (xm == T(0)) return densu_temp;
        const T g1 = T(1.0) + zlb / re;
        T glb = gsurf / (g1 * g1);
        const T gamma = xm * glb / (s2 * rgas * tinf);
        T expl = exp(-s2 * gamma * zg2);
        if (expl > T(50.0)) expl = T(50.0);
        if (tt <= T(0)) expl = T(50.0);
        densu_temp = dlb * pow((tlb / tt), ((T(1.0) + alpha + gamma))) * expl;
        if (alt >= za) return densu_temp;
        const T g2 = T(1.0) + z1 / re;
        glb = gsurf / (g2 * g2);
        const T gamm = xm * glb * zgdif / rgas;
        const T yi = nrl::Model<T>::splini(xs, ys, y2out, mn1, x);
        expl = gamm * yi;
        if (expl > T(50.0)) expl = T(50.0);
        if (*tz <= T(0)) expl = T(50.0);
        return densu_temp * pow((t1 / *tz), (T(1.0) + alpha)) * exp(-expl);
    }

    // densu below za shares everything but the altitude between calls with
    // the same tinf / tlb: the temperature at za, the mesosphere node
    // profile and its spline.  lowProfile forms that part once (with densu's
    // side effect on the first node); densuBelow evaluates one call from it,
    // in the same operations as densu.
    struct LowProfile {
        T xs[5], ys[5], y2[5];
        T zgdif, rzgdif, t1, zg2, tt;
    };

    // 1 / x for the nonzero, well-scaled denominators of the mesosphere
    // profile and the species corrections (heights, scale heights,
    // temperatures, gravity ratios, mass differences): a single-precision
    // estimate refined by two Newton-Raphson steps r <- r + r (1 - x r)
    // (relative error 2^-21 -> 2^-42 -> below one ulp), without the branches
    // of the IEEE division sequence, so that independent quotients overlap.
    static __device__ __forceinline__ double rcp(double x) {
        double r = (double)__fdividef(1.0f, (float)x);
        r = fma(r, fma(-x, r, 1.0), r);
        return fma(r, fma(-x, r, 1.0), r);
    }
    static __device__ __forceinline__ float rcp(float x) { return 1.0f / x; }

    // Clamped cubic spline through the five mesosphere nodes: the reference's
    // tridiagonal sweep (spline, Nrlmsise00Model.inl:289) with the interval
    // reciprocals and slopes formed once.
    static __device__ __forceinline__ void spline5(const T* x, const T* y, T yp1, T ypn, T* y2) {
        T r[4], d[4], u[4];
        for (int i = 0; i < 4; ++i) {
            r[i] = rcp(x[i + 1] - x[i]);
            d[i] = (y[i + 1] - y[i]) * r[i];
        }
        y2[0] = T(-0.5);
        u[0] = (T(3.0) * r[0]) * (d[0] - yp1);
        for (int i = 1; i < 4; ++i) {
            const T w = rcp(x[i + 1] - x[i - 1]);
            const T sig = (x[i] - x[i - 1]) * w;
            const T rp = rcp(sig * y2[i - 1] + T(2.0));
            y2[i] = (sig - T(1.0)) * rp;
            u[i] = (T(6.0) * (d[i] - d[i - 1]) * w - sig * u[i - 1]) * rp;
        }
        const T un = (T(3.0) * r[3]) * (ypn - d[3]);
        y2[4] = (un - T(0.5) * u[3]) * rcp(T(0.5) * y2[3] + T(1.0));
        for (int k = 3; k >= 0; --k) y2[k] = y2[k] * y2[k + 1] + u[k];
    }

    // spline value and integral from xa[0] (splint :256, splini :218) on the
    // five nodes, with one reciprocal per interval
    static __device__ __forceinline__ T splint5(const T* xa, const T* ya, const T* y2a, T x) {
        int klo = 0, khi = 4;
        while (khi - klo > 1) {
            const int k = (khi + klo) >> 1;
            if (xa[k] > x) khi = k;
            else klo = k;
        }
        const T h = xa[khi] - xa[klo];
        const T rh = rcp(h);
        const T a = (xa[khi] - x) * rh;
        const T b = (x - xa[klo]) * rh;
        return a * ya[klo] + b * ya[khi] + ((a * a * a - a) * y2a[klo] + (b * b * b - b) * y2a[khi]) * h * h / T(6.0);
    }
    static __device__ __forceinline__ T splini5(const T* xa, const T* ya, const T* y2a, T x) {
        T yi = T(0);
        for (int klo = 0, khi = 1; x > xa[klo] && khi < 5; ++klo, ++khi) {
            const T xx = khi < 4 ? (x < xa[khi] ? x : xa[khi]) : x;
            const T h = xa[khi] - xa[klo];
            const T rh = rcp(h);
            const T a = (xa[khi] - xx) * rh;
            const T b = (xx - xa[klo]) * rh;
            const T a2 = a * a;
            const T b2 = b * b;
            yi += ((T(1.0) - a2) * ya[klo] * T(0.5) + b2 * ya[khi] * T(0.5)
                   + ((-(T(1.0) + a2 * a2) * T(0.25) + a2 * T(0.5)) * y2a[klo]
                      + (b2 * b2 * T(0.25) - b2 * T(0.5)) * y2a[khi]) * h * h / T(6.0)) * h;
        }
        return yi;
    }

    // dnet (Nrlmsise00Model.inl:180) and ccor2 (:138) for the species
    // corrections: the same branches and operations, quotients by reciprocal
    // and the power as exp(log(.) / a); ccor(z, r, h, zh) is ccor2 with
    // h2 = h, whose second exponential is then the first.
    static __device__ __forceinline__ T dnetFast(T dd, T dm, T zhm, T xmm, T xm) {
        const T a = zhm * rcp(xmm - xm);
        const T ra = (xmm - xm) * rcp(zhm);  // 1 / a
        if (!((dm > T(0)) && (dd > T(0)))) {
            if ((dd == T(0)) && (dm == T(0))) dd = T(1);
            if (dm == T(0)) return dd;
            if (dd == T(0)) return dm;
        }
        const T ylog = a * log(dm * rcp(dd));
        if (ylog < T(-10)) return dd;
        if (ylog > T(10)) return dm;
        return dd * exp(log(T(1.0) + exp(ylog)) * ra);
    }
    static __device__ __forceinline__ T ccor2Fast(T alt, T r, T h1, T zh, T h2) {
        const T e1 = (alt - zh) * rcp(h1);
        const T e2 = h2 == h1 ? e1 : (alt - zh) * rcp(h2);
        if ((e1 > T(70)) || (e2 > T(70))) return T(1.0);
        if ((e1 < T(-70)) && (e2 < T(-70))) return exp(r);
        const T ex1 = exp(e1);
        const T ex2 = h2 == h1 ? ex1 : exp(e2);
        return exp(r * rcp(T(1.0) + T(0.5) * (ex1 + ex2)));
    }

    static __device__ __noinline__ void lowProfile(LowProfile& lp, T tinf, T tlb, T zlb, T s2, const T* zn1, T re,
                                                   NrlMeso<T>& ms) {
        auto zeta = [re](T zz, T zl) { return (zz - zl) * (re + zl) * rcp(re + zz); };
        const T za = zn1[0];
        lp.zg2 = zeta(za, zlb);
        lp.tt = tinf - (tinf - tlb) * exp(-s2 * lp.zg2);
        const T ta = lp.tt;
        const T q = (re + zlb) * rcp(re + za);
        ms.tgn1[0] = (tinf - ta) * s2 * (q * q);
        ms.tn1[0] = ta;
        const T z1 = zn1[0];
        const T z2 = zn1[4];
        lp.t1 = ms.tn1[0];
        const T t2 = ms.tn1[4];
        lp.zgdif = zeta(z2, z1);
        lp.rzgdif = rcp(lp.zgdif);
        lp.xs[0] = T(0.0);
        lp.xs[4] = T(1.0);
        for (int k = 1; k < 4; k++) lp.xs[k] = zeta(zn1[k], z1) * lp.rzgdif;
        for (int k = 0; k < 5; k++) lp.ys[k] = rcp(ms.tn1[k]);
        const T r2 = (re + z2) * rcp(re + z1);
        const T yd1 = -ms.tgn1[0] * rcp(lp.t1 * lp.t1) * lp.zgdif;
        const T yd2 = -ms.tgn1[1] * rcp(t2 * t2) * lp.zgdif * (r2 * r2);
        spline5(lp.xs, lp.ys, yd1, yd2, lp.y2);
    }
    static __device__ __noinline__ T densuBelow(T alt, T dlb, T tinf, T tlb, T xm, T alpha, T zlb, T s2,
                                                const T* zn1, T re, T gsurf, const LowProfile& lp) {
        const T rgas = T(831.4);
        const T z = (alt > zn1[4]) ? alt : zn1[4];
        const T z1 = zn1[0];
        const T zg = (z - z1) * (re + z1) * rcp(re + z);
        const T x = zg * lp.rzgdif;
        const T y = splint5(lp.xs, lp.ys, lp.y2, x);
        const T tz = rcp(y);
        if (xm == T(0)) return tz;
        const T g1 = T(1.0) + zlb / re;
        const T glb = gsurf * rcp(g1 * g1);
        const T gamma = xm * glb * rcp(s2 * rgas * tinf);
        T expl = exp(-s2 * gamma * lp.zg2);
        if (expl > T(50.0)) expl = T(50.0);
        if (lp.tt <= T(0)) expl = T(50.0);
        const T densuTemp = dlb * exp((T(1.0) + alpha + gamma) * log(tlb * rcp(lp.tt))) * expl;
        const T g2 = T(1.0) + z1 / re;
        const T gamm = xm * (gsurf * rcp(g2 * g2)) * lp.zgdif / rgas;
        const T yi = splini5(lp.xs, lp.ys, lp.y2, x);
        expl = gamm * yi;
        if (expl > T(50.0)) expl = T(50.0);
        if (tz <= T(0)) expl = T(50.0);
        return densuTemp * exp((T(1.0) + alpha) * log(lp.t1 * rcp(tz))) * exp(-expl);
    }

    // Monomial i of the globe7 basis (order of the coefficient rows; i is a
    // compile-time constant after unrolling).  x = P(1,0); U1, U2 = cos, sin of
    // (sr sec + 2 dgtr lon).
    __device__ __forceinline__ T globeMonomial(int i, T x, T x2, T U1, T U2) const {
        switch (i) {
            case 0: return T(1.0);
            case 1: return x;
            case 2: return plg[0][2];
            case 3: return plg[0][3];
            case 4: return plg[0][4];
            case 5: return plg[0][5];
            case 6: return plg[0][6];
            case 7: return plg[1][1] * ctloc;
            case 8: return plg[1][2] * ctloc;
            case 9: return plg[1][3] * ctloc;
            case 10: return plg[1][5] * ctloc;
            case 11: return plg[1][1] * stloc;
            case 12: return plg[1][2] * stloc;
            case 13: return plg[1][3] * stloc;
            case 14: return plg[1][5] * stloc;
            case 15: return plg[2][2] * c2tloc;
            case 16: return plg[2][3] * c2tloc;
            case 17: return plg[2][4] * c2tloc;
            case 18: return plg[2][5] * c2tloc;
            case 19: return plg[2][2] * s2tloc;
            case 20: return plg[2][3] * s2tloc;
            case 21: return plg[2][4] * s2tloc;
            case 22: return plg[2][5] * s2tloc;
            case 23: return plg[3][3] * s3tloc;
            case 24: return plg[3][4] * s3tloc;
            case 25: return plg[3][6] * s3tloc;
            case 26: return plg[3][3] * c3tloc;
            case 27: return plg[3][4] * c3tloc;
            case 28: return plg[3][6] * c3tloc;
            case 29: return plg[1][1] * cgl;
            case 30: return plg[1][2] * cgl;
            case 31: return plg[1][3] * cgl;
            case 32: return plg[1][4] * cgl;
            case 33: return plg[1][5] * cgl;
            case 34: return plg[1][6] * cgl;
            case 35: return plg[1][1] * sgl;
            case 36: return plg[1][2] * sgl;
            case 37: return plg[1][3] * sgl;
            case 38: return plg[1][4] * sgl;
            case 39: return plg[1][5] * sgl;
            case 40: return plg[1][6] * sgl;
            case 41: return x * plg[1][2] * cgl;
            case 42: return x * plg[1][4] * cgl;
            case 43: return x * plg[1][6] * cgl;
            case 44: return x * plg[1][2] * sgl;
            case 45: return x * plg[1][4] * sgl;
            case 46: return x * plg[1][6] * sgl;
            case 47: return csec * x;
            case 48: return csec * plg[0][3];
            case 49: return csec * plg[0][5];
            case 50: return csec * x2;
            case 51: return csec * (x * plg[0][3]);
            case 52: return csec * (x * plg[0][5]);
            case 53: return csec * (x2 * x);
            case 54: return csec * (x2 * plg[0][3]);
            case 55: return csec * (x2 * plg[0][5]);
            case 56: return ssec * x;
            case 57: return ssec * plg[0][3];
            case 58: return ssec * plg[0][5];
            case 59: return ssec * x2;
            case 60: return ssec * (x * plg[0][3]);
            case 61: return ssec * (x * plg[0][5]);
            case 62: return ssec * (x2 * x);
            case 63: return ssec * (x2 * plg[0][3]);
            case 64: return ssec * (x2 * plg[0][5]);
            case 65: return plg[2][3] * U1;
            case 66: return plg[2][5] * U1;
            case 67: return plg[2][7] * U1;
            case 68: return plg[2][3] * U2;
            case 69: return plg[2][5] * U2;
            case 70: return plg[2][7] * U2;
            default: return T(0.0);
        }
    }

    // Latitude-dependent ap response sg0 of table k (pt or pd[0]).
    __device__ __forceinline__ T aptLatitude(const double* __restrict__ p, const double* g0) const {
        T exp1 = exp(T(-10800.0) * fabs(T(p[51])) / (T(1.0) + T(p[138]) * (T(45.0) - absLat)));
        if (exp1 > T(0.99999)) exp1 = T(0.99999);
        return sg0FromExp(exp1, g0);
    }

    // The 11 globe7 values of one gts7 call (task order above), with the ap
    // response apt0 left by the pd[3] table (used by the mesosphere glob7s
    // terms) and by the last table (used below 72.5 km).  Each lane of a
    // group of L takes kGlobeRows / L coefficient rows (rows j, j + L, ...)
    // and forms their dot products with the monomials (two partial sums per
    // row, read two coefficients at a time); the row values are exchanged by
    // shuffles.  The latitude-dependent ap responses of pt and pd[0] are
    // formed on lanes 0 and 1.
    template <int L>
    __device__ __forceinline__ void globeTasks(T (&G)[kGlobeTasks], T& aptTlb, T& aptLast, int j, int groupBase) {
        static_assert(kGlobeRows % L == 0, "lane split of the coefficient rows");
        // rows 13..15 are zero: lane j takes rows j, j + L, ... below 13 only
        // (rows r L + j < 16 stay inside the block for every lane)
        constexpr int R = (kApRowPd0 + 1 + L - 1) / L;
        const T x = plg[0][1], x2 = x * x;
        const T U1 = csec * c2gl - ssec * s2gl, U2 = ssec * c2gl + csec * s2gl;
        const double2* __restrict__ rows = reinterpret_cast<const double2*>(&eb.globeRows[0][0][0]);
        T acc[R], acc2[R];
#pragma unroll
        for (int r = 0; r < R; ++r) acc[r] = acc2[r] = T(0.0);
#if PHOP_NRL_ROLLED_GLOBE
        if constexpr (L <= 4) {
        // the monomials formed once into a small local array, then a rolled
        // dot-product loop: a short instruction stream (the step kernel
        // alternates this model with the geopotential loop, and both compete
        // for the instruction cache; measured 1-2 % faster on the uneven
        // population at two lanes than the fully unrolled form, which the
        // eight- and sixteen-lane kernels keep: they call the model out of line)
        T mono[kGlobeBasis + 1];
#pragma unroll
        for (int i = 0; i <= kGlobeBasis; ++i) mono[i] = globeMonomial(i, x, x2, U1, U2);
#pragma unroll 1
        for (int i = 0; i < kGlobeBasis; i += 2) {
            const T b0 = mono[i], b1 = mono[i + 1];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const double2 c = __ldg(rows + (i / 2) * kGlobeRows + r * L + j);
                acc[r] = fma(T(c.x), b0, acc[r]);
                acc2[r] = fma(T(c.y), b1, acc2[r]);
            }
        }
        } else {
#pragma unroll
        for (int i = 0; i < kGlobeBasis; i += 2) {
            const T b0 = globeMonomial(i, x, x2, U1, U2), b1 = globeMonomial(i + 1, x, x2, U1, U2);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const double2 c = __ldg(rows + (i / 2) * kGlobeRows + r * L + j);
                acc[r] = fma(T(c.x), b0, acc[r]);
                acc2[r] = fma(T(c.y), b1, acc2[r]);
            }
        }
        }
#else
#pragma unroll
        for (int i = 0; i < kGlobeBasis; i += 2) {
            const T b0 = globeMonomial(i, x, x2, U1, U2), b1 = globeMonomial(i + 1, x, x2, U1, U2);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const double2 c = __ldg(rows + (i / 2) * kGlobeRows + r * L + j);
                acc[r] = fma(T(c.x), b0, acc[r]);
                acc2[r] = fma(T(c.y), b1, acc2[r]);
            }
        }
#endif
        const unsigned mask = L >= 32 ? 0xffffffffu : ((1u << L) - 1u) << groupBase;
        // value of row t: accumulator t / L of lane t % L
        auto rowValue = [&](int t) -> T {
            const T v = acc[t / L] + acc2[t / L];
            if (L == 1) return v;
            return __shfl_sync(mask, v, groupBase + t % L);
        };
        T aptPt, aptPd0;
        if (L == 1) {
            aptPt = aptLatitude(globeTable(0), eb.ge[0].g0);
            aptPd0 = aptLatitude(globeTable(2), eb.ge[2].g0);
        } else {
            const int k = (j & 1) ? 2 : 0;
            const T a = aptLatitude(globeTableGlobal(k), eb.ge[k].g0);
            aptPt = __shfl_sync(mask, a, groupBase);
            aptPd0 = __shfl_sync(mask, a, groupBase + 1);
        }
#pragma unroll
        for (int t = 0; t < kGlobeTasks; ++t) G[t] = rowValue(t);
        G[0] = fma(aptPt, rowValue(kApRowPt), G[0]);
        G[4] = fma(aptPd0, rowValue(kApRowPd0), G[4]);
        // apt0 after task t in the sequential order: the value set by the last
        // table up to t whose ap term is present (p[51] != 0)
        T aptSeq = apt0;
#pragma unroll
        for (int t = 0; t < kGlobeTasks; ++t) {
            const int k = globeTaskTable(t);
            if (globeTable(k)[51] != 0.0) aptSeq = k == 0 ? aptPt : k == 2 ? aptPd0 : T(eb.ge[k].apt0);
            if (t == 2) aptTlb = aptSeq;
        }
        aptLast = aptSeq;
        apt0 = aptLast;
    }

    // thermosphere (alt >= 72.5 km): number densities d[0..8] (m^-3), from
    // the globe7 values G (task order).  Above za the main density of each
    // species, densu(z, dlb, tinf, tlb, xm, alpha) with dlb = pdm exp(g) pd,
    // is formed as pdm pd exp(g + (1 + alpha + gamma) ln(tlb/tt) - s gamma zg2):
    // the temperature profile tt and its logarithm are shared by the
    // species, and one exponential replaces exp, pow and exp.
    template <int L>
    __device__ __forceinline__ void gts7(T alt, const T (&G)[kGlobeTasks], T aptTlb, T* d, NrlMeso<T>& ms, int j,
                                         int groupBase) {
        T* meso_tn1 = ms.tn1;
        T* meso_tgn1 = ms.tgn1;
        T& dm28 = ms.dm28;
        T zn1[5] = {T(NRL_PDL(1)[15]), T(110.0), T(100.0), T(90.0), T(72.5)};
        const T za = zn1[0];
        for (int j = 0; j < 9; j++) d[j] = T(0);
        const T z = alt;
        T dummyT;
        const T tinf = (z > za) ? T(NRL_PTM(0)) * T(NRL_PT[0]) * (T(1.0) + G[0]) : T(NRL_PTM(0)) * T(NRL_PT[0]);
        const T g0v = (z > zn1[4]) ? T(NRL_PTM(3)) * T(NRL_PS[0]) * (T(1.0) + G[1]) : T(NRL_PTM(3)) * T(NRL_PS[0]);
        const T tlb = T(NRL_PTM(1)) * (T(1.0) + G[2]) * T(NRL_PD(3)[0]);
        const T s = g0v * rcp(tinf - tlb);
        const T ptl30 = T(NRL_PTM(4)) * T(NRL_PTL(3)[0]);
        // the five glob7s tables of the mesosphere nodes (ptl[0..3], pma[8]),
        // evaluated on all converged lanes when any object is below 300 km;
        // L > 1 lanes share them as for globe7
        T gs[5];
        const bool meso = z < T(300.0);
        if (__any_sync(__activemask(), meso)) {
            apt0 = aptTlb;
            if (L == 1) {
#pragma unroll
                for (int k = 0; k < 5; ++k) gs[k] = glob7s(k < 4 ? k : 12);
            } else {
                const unsigned mask = ((1u << L) - 1u) << groupBase;
#pragma unroll
                for (int r = 0; r < (5 + L - 1) / L; ++r) {
                    const int k = r * L + j;
                    T v = T(0.0);
                    if (k < 5) v = glob7sAt(k < 4 ? k : 12, globSTableGlobal(k < 4 ? k : 12));
#pragma unroll
                    for (int jj = 0; jj < L; ++jj)
                        if (r * L + jj < 5) gs[r * L + jj] = __shfl_sync(mask, v, groupBase + jj);
                }
            }
        }
        if (meso) {
            meso_tn1[1] = T(NRL_PTM(6)) * T(NRL_PTL(0)[0]) / (T(1.0) - gs[0]);
            meso_tn1[2] = T(NRL_PTM(2)) * T(NRL_PTL(1)[0]) / (T(1.0) - gs[1]);
            meso_tn1[3] = T(NRL_PTM(7)) * T(NRL_PTL(2)[0]) / (T(1.0) - gs[2]);
            meso_tn1[4] = ptl30 / (T(1.0) - gs[3]);
            meso_tgn1[1] = T(NRL_PTM(8)) * T(NRL_PMA(8)[0]) * (T(1.0) + gs[4]) * meso_tn1[4] * meso_tn1[4]
                / (ptl30 * ptl30);
        } else {
            meso_tn1[1] = T(NRL_PTM(6)) * T(NRL_PTL(0)[0]);
            meso_tn1[2] = T(NRL_PTM(2)) * T(NRL_PTL(1)[0]);
            meso_tn1[3] = T(NRL_PTM(7)) * T(NRL_PTL(2)[0]);
            meso_tn1[4] = ptl30;
            meso_tgn1[1] = T(NRL_PTM(8)) * T(NRL_PMA(8)[0]) * meso_tn1[4] * meso_tn1[4] / (ptl30 * ptl30);
        }
        const T zlb = T(NRL_PTM(5));
        const T xmm = T(NRL_PDM(2, 4));
        // shared temperature profile of the main species densities (densu, z >= za)
        const T rgas = T(831.4);
        const T zg2 = zeta(z >= za ? z : za, zlb);
        const T tt = tinf - (tinf - tlb) * exp(-s * zg2);
        const bool direct = z >= za && tt > T(0);
        T lnX = T(0), kGamma = T(0);
        if (direct) {
            lnX = log(tlb * rcp(tt));
            const T g1 = T(1.0) + zlb / re;
            kGamma = gsurf * rcp(g1 * g1 * s * rgas * tinf);  // gamma = xm * kGamma
        }
        auto mainDensity = [&](T g, T pdm0, T pd0, T xm, T alpha) -> T {
            if (direct) {
                const T gamma = xm * kGamma;
                return pdm0 * pd0 * exp(g + (T(1.0) + alpha + gamma) * lnX - s * gamma * zg2);
            }
            return densu(z, pdm0 * exp(g) * pd0, tinf, tlb, xm, alpha, &dummyT, zlb, s, zn1, re, gsurf, ms);
        };
        // Low-altitude corrections: for species s below its altitude limit,
        // b_s = densu(zb_s, db_s, tinf, tlb, xm_s - xmm, alpha_s - 1) and the
        // mixing density dm_s = densu(z, b_s, tinf, tlb, xmm, 0).  Task t =
        // N2, He, O, O2, Ar, H, N.  With L > 1 lanes the tasks are spread over
        // the group's lanes (the costly spline path of densu then runs once
        // per lane instead of once per task on every lane) and exchanged by
        // shuffles; the combination below is the same for every L.
        const T zhf = T(NRL_PDL(1)[24]) * (T(1.0) + T(NRL_PDL(0)[24]) * plg[0][1] * T(eb.ge[0].cd14));
        auto needTask = [&](int t) -> bool {
            switch (t) {
                case 0: return !(z > T(450.0) && z >= za);
                case 1: return z < T(200.0);
                case 2: return z <= T(300.0);
                case 3: return z <= T(250.0);
                case 4: return z <= T(240.0);
                case 5: return z <= T(320.0);
                default: return z <= T(450.0);
            }
        };
        // Tasks any object of the converged lanes needs run on all of them
        // (results unused where not needed): objects of one warp differ by a
        // few km in altitude, and running each one's own subset would split
        // the warp into serialised paths.
        unsigned needBits = 0;
#pragma unroll
        for (int t = 0; t < 7; ++t)
            if (needTask(t)) needBits |= 1u << t;
        needBits = __reduce_or_sync(__activemask(), needBits);
        auto taskOn = [&](int t) { return (needBits >> t) & 1u; };
        LowProfile low;
        if (taskOn(0)) lowProfile(low, tinf, tlb, zlb, s, zn1, re, ms);
        auto corrTask = [&](int t, T& bOut, T& dmOut) {
            T zb, xm, al, pdm0, pd0, g;
            switch (t) {
                case 0: zb = T(NRL_PDM(2, 2)) * zhf; xm = T(28.0); al = T(-1.0); pdm0 = T(NRL_PDM(2, 0)); pd0 = T(NRL_PD(2)[0]); g = G[3]; break;
                case 1: zb = T(NRL_PDM(0, 2)); xm = T(4.); al = T(-1.38); pdm0 = T(NRL_PDM(0, 0)); pd0 = T(NRL_PD(0)[0]); g = G[4]; break;
                case 2: zb = T(NRL_PDM(1, 2)); xm = T(16.0); al = T(-1.0); pdm0 = T(NRL_PDM(1, 0)); pd0 = T(NRL_PD(1)[0]); g = G[5]; break;
                case 3: zb = T(NRL_PDM(3, 2)); xm = T(32.); al = T(-1.); pdm0 = T(NRL_PDM(3, 0)); pd0 = T(NRL_PD(4)[0]); g = G[6]; break;
                case 4: zb = T(NRL_PDM(4, 2)); xm = T(40.); al = T(-0.83); pdm0 = T(NRL_PDM(4, 0)); pd0 = T(NRL_PD(5)[0]); g = G[7]; break;
                case 5: zb = T(NRL_PDM(5, 2)); xm = T(1.); al = T(-1.38); pdm0 = T(NRL_PDM(5, 0)); pd0 = T(NRL_PD(6)[0]); g = G[8]; break;
                default: zb = T(NRL_PDM(6, 2)); xm = T(14.); al = T(-1.); pdm0 = T(NRL_PDM(6, 0)); pd0 = T(NRL_PD(7)[0]); g = G[9]; break;
            }
            const T db = pdm0 * exp(g) * pd0;
            bOut = zb < za ? densuBelow(zb, db, tinf, tlb, xm - xmm, al, zlb, s, zn1, re, gsurf, low)
                           : densu(zb, db, tinf, tlb, xm - xmm, al, &dummyT, zlb, s, zn1, re, gsurf, ms);
            dmOut = T(0.0);
            if (t != 0 || z <= T(160.0)) {
                if (direct) {
                    // densu(z, b, tinf, tlb, xmm, 0) above za, from the shared profile
                    const T gamma = xmm * kGamma;
                    dmOut = bOut * exp((T(1.0) + gamma) * lnX - s * gamma * zg2);
                } else {
                    dmOut = densu(z, bOut, tinf, tlb, xmm, T(0.0), &dummyT, zlb, s, zn1, re, gsurf, ms);
                }
            }
        };
        T bv[7], dmv[7];
#pragma unroll
        for (int t = 0; t < 7; ++t) bv[t] = dmv[t] = T(0.0);
        if (L == 1) {
#pragma unroll
            for (int t = 0; t < 7; ++t)
                if (taskOn(t)) corrTask(t, bv[t], dmv[t]);
        } else if (taskOn(0)) {  // every other task's limit is below N2's
            // slots in order of decreasing altitude limit (N2, N, H, O, O2, Ar,
            // He), so the tasks active at an altitude fill the first rounds
            constexpr int kSlot[7] = {0, 6, 5, 2, 3, 4, 1};
            const unsigned mask = ((1u << L) - 1u) << groupBase;
#pragma unroll
            for (int r = 0; r < (7 + L - 1) / L; ++r) {
                const int k = r * L + j;
                T bb = T(0.0), dd = T(0.0);
                if (k < 7) {
                    const int t = k == 0 ? 0 : k == 1 ? 6 : k == 2 ? 5 : k == 3 ? 2 : k == 4 ? 3 : k == 5 ? 4 : 1;
                    if (taskOn(t)) corrTask(t, bb, dd);
                }
#pragma unroll
                for (int jj = 0; jj < L; ++jj) {
                    const int kk = r * L + jj;
                    if (kk < 7) {
                        bv[kSlot[kk]] = __shfl_sync(mask, bb, groupBase + jj);
                        dmv[kSlot[kk]] = __shfl_sync(mask, dd, groupBase + jj);
                    }
                }
            }
        }
        const T zhm28 = T(NRL_PDM(2, 3)) * T(NRL_PDL(1)[5]);
        const T b28 = bv[0];
        if (z <= T(160.0)) dm28 = dmv[0];
        // The seven species densities, lane-parallel: lane j of the group
        // takes species rows j, j + L, ... of eb.species (N, H, O, O2 first:
        // the ones corrected at orbital altitudes) in one data-driven form,
        // so the lanes of a group run the same instructions; the results are
        // exchanged by shuffles.  Row -> d index, G task and correction task:
        constexpr int kDPos[kNrlSpecies] = {7, 6, 1, 3, 4, 0, 2};
        constexpr int kGIdx[kNrlSpecies] = {9, 8, 5, 6, 7, 4, 3};
        constexpr int kTask[kNrlSpecies] = {6, 5, 2, 3, 4, 1, 0};
        auto speciesDensity = [&](int r) -> T {
            const double* __restrict__ q = eb.species[r];
            T g = T(0), b = T(0), dm = T(0);
#pragma unroll
            for (int k = 0; k < kNrlSpecies; ++k)
                if (k == r) {
                    g = G[kGIdx[k]];
                    b = bv[kTask[k]];
                    dm = dmv[kTask[k]];
                }
            const T xm = T(q[kSpXm]);
            T dn = mainDensity(g, T(q[kSpPdm0]), T(q[kSpPd0]), xm, T(q[kSpAlpha]));
            if (z <= T(q[kSpLim])) {
                dn = dnetFast(dn, dm, zhm28, xmm, xm);
                const T r1 = q[kSpRlLog] != 0.0 ? log(b28 * T(q[kSpK1]) * T(q[kSpK2]) * rcp(b)) : T(q[kSpK1]);
                dn = dn * ccor2Fast(z, r1, T(q[kSpC1H1]), T(q[kSpC1Zh]), T(q[kSpC1H2]));
                if (q[kSpR2] != 0.0) dn = dn * ccor2Fast(z, T(q[kSpR2]), T(q[kSpC2H]), T(q[kSpC2Zh]), T(q[kSpC2H]));
            }
            if (q[kSpRc] != 0.0)
                dn = dn * ccor2Fast(z, T(q[kSpRc]), T(q[kSpCaH1]), T(q[kSpCaZh]), T(q[kSpCaH2]));
            return dn;
        };
        {
            const unsigned smask = L >= 32 ? 0xffffffffu : ((1u << L) - 1u) << groupBase;
#pragma unroll
            for (int rr = 0; rr < (kNrlSpecies + L - 1) / L; ++rr) {
                const int r = rr * L + j;
                T v = T(0);
                if (r < kNrlSpecies) v = speciesDensity(r);
#pragma unroll
                for (int jj = 0; jj < L; ++jj) {
                    const int rk = rr * L + jj;
                    if (rk < kNrlSpecies) d[kDPos[rk]] = L == 1 ? v : __shfl_sync(smask, v, groupBase + jj);
                }
            }
        }
        // anomalous O: densu with tinf = tlb = tho, where ln(tlb/tt) = 0
        const T tho = T(NRL_PDM(7, 9)) * T(NRL_PDL(0)[6]);
        T dd;
        if (direct) {
            const T g1 = T(1.0) + zlb / re;
            const T gamma = T(16.0) * gsurf * rcp(g1 * g1 * s * rgas * tho);
            dd = T(NRL_PDM(7, 0)) * T(NRL_PD(8)[0]) * exp(G[10] - s * gamma * zg2);
        } else {
            dd = densu(z, T(NRL_PDM(7, 0)) * exp(G[10]) * T(NRL_PD(8)[0]), tho, tho, T(16.), T(0.0), &dummyT, zlb, s, zn1, re, gsurf, ms);
        }
        const T zsht = T(NRL_PDM(7, 5)), zmho = T(NRL_PDM(7, 4));
        const T gz = T(1.0) + zmho / re;
        const T rzsht = rcp(zsht);
        const T rzsho = gsurf * T(16.0) * rcp(T(831.4) * tho * gz * gz);  // 1 / zsho
        d[8] = dd * exp(-zsht * rzsho * (exp(-(z - zmho) * rzsht) - T(1.)));
        for (int i = 0; i < 9; i++) d[i] = d[i] * T(1.0E6);
    }

    // gtd7 + gtd7d total mass density (kg/m^3); lane j of a group of L
    // lanes starting at groupBase (all lanes of the group get the result)
    template <int L>
    __device__ __forceinline__ T density(T lat, T lon, T alt, T lst, int j, int groupBase) {
        glat = lat;
        absLat = fabs(lat);
        gLong = lon;
        apt0 = T(0);
        NrlMeso<T> ms;
        ms.dm28 = T(0);
        ms.tn1[0] = T(0);
        ms.tgn1[0] = T(0);
        // glatf
        const T c2 = cos(T(2.0) * T(1.74533E-2) * lat);
        gsurf = T(980.616) * (T(1.0) - T(0.0026373) * c2);
        re = T(2.0) * gsurf * rcp(T(3.085462E-6) + T(2.27E-9) * c2) * T(1.0E-5);
        basis(lat, lst);
        T G[kGlobeTasks];
        T aptTlb = T(0), aptLast = T(0);
        globeTasks<L>(G, aptTlb, aptLast, j, groupBase);
        T d[9];
        const T zn2top = T(72.5);
        gts7<L>(alt > zn2top ? alt : zn2top, G, aptTlb, d, ms, j, groupBase);
        if (!(alt >= zn2top)) {
            apt0 = aptLast;
            return lowerAtmosphere(*this, alt, d, ms);
        }
        return (T(1.66E-24) * (T(4.0) * d[0] + T(16.0) * d[1] + T(28.0) * d[2] + T(32.0) * d[3] + T(40.0) * d[4]
                               + d[6] + T(14.0) * d[7] + T(16.0) * d[8]))
            / T(1000);
    }

    // below 72.5 km (not reached in orbit, kept for completeness)
    static __device__ __noinline__ T lowerAtmosphere(Fast f, T alt, const T* d, const NrlMeso<T>& ms) {
        const T gsurf = f.gsurf, re = f.re, dm28 = ms.dm28;
        const T* meso_tn1 = ms.tn1;
        const T* meso_tgn1 = ms.tgn1;
        auto glob7s = [&f](int k) { return f.glob7s(k); };
        nrl::Model<T> m;
        m.gsurf = gsurf;
        m.re = re;
        const T zn3[5] = {T(32.5), T(20.0), T(15.0), T(10.0), T(0.0)};
        const T zn2[4] = {T(72.5), T(55.0), T(45.0), T(32.5)};
        T tn2[4], tgn2[2], tn3[5] = {0, 0, 0, 0, 0}, tgn3[2] = {0, 0};
        tgn2[0] = meso_tgn1[1];
        tn2[0] = meso_tn1[4];
        tn2[1] = T(NRL_PMA(0)[0]) * T(NRL_PAVGM(0)) / (T(1.0) - glob7s(4 + 0));
        tn2[2] = T(NRL_PMA(1)[0]) * T(NRL_PAVGM(1)) / (T(1.0) - glob7s(4 + 1));
        tn2[3] = T(NRL_PMA(2)[0]) * T(NRL_PAVGM(2)) / (T(1.0) - glob7s(4 + 2));
        const T q2 = T(NRL_PMA(2)[0]) * T(NRL_PAVGM(2));
        tgn2[1] = T(NRL_PAVGM(8)) * T(NRL_PMA(9)[0]) * (T(1.0) + glob7s(4 + 9)) * tn2[3] * tn2[3] / (q2 * q2);
        tn3[0] = tn2[3];
        if (alt <= zn3[0]) {
            tgn3[0] = tgn2[1];
            tn3[1] = T(NRL_PMA(3)[0]) * T(NRL_PAVGM(3)) / (T(1.0) - glob7s(4 + 3));
            tn3[2] = T(NRL_PMA(4)[0]) * T(NRL_PAVGM(4)) / (T(1.0) - glob7s(4 + 4));
            tn3[3] = T(NRL_PMA(5)[0]) * T(NRL_PAVGM(5)) / (T(1.0) - glob7s(4 + 5));
            tn3[4] = T(NRL_PMA(6)[0]) * T(NRL_PAVGM(6)) / (T(1.0) - glob7s(4 + 6));
            const T q6 = T(NRL_PMA(6)[0]) * T(NRL_PAVGM(6));
            tgn3[1] = T(NRL_PMA(7)[0]) * T(NRL_PAVGM(7)) * (T(1.0) + glob7s(4 + 7)) * tn3[4] * tn3[4] / (q6 * q6);
        }
        const T zmix = T(62.5);
        T dmc = T(0);
        if (alt > zmix) dmc = T(1.0) - (zn2[0] - alt) / (zn2[0] - zmix);
        const T dm28m = dm28 * T(1.0E6);
        const T xmm = T(NRL_PDM(2, 4));
        T tz = T(0);
        const T dz28 = d[2];
        T o[9];
        T dmr = d[2] / dm28m - T(1.0);
        o[2] = m.densm(alt, dm28m, xmm, &tz, 5, zn3, tn3, tgn3, 4, zn2, tn2, tgn2) * (T(1.0) + dmr * dmc);
        dmr = d[0] / (dz28 * T(NRL_PDM(0, 1))) - T(1.0);
        o[0] = o[2] * T(NRL_PDM(0, 1)) * (T(1.0) + dmr * dmc);
        dmr = d[3] / (dz28 * T(NRL_PDM(3, 1))) - T(1.0);
        o[3] = o[2] * T(NRL_PDM(3, 1)) * (T(1.0) + dmr * dmc);
        dmr = d[4] / (dz28 * T(NRL_PDM(4, 1))) - T(1.0);
        o[4] = o[2] * T(NRL_PDM(4, 1)) * (T(1.0) + dmr * dmc);
        return (T(1.66E-24) * (T(4.0) * o[0] + T(28.0) * o[2] + T(32.0) * o[3] + T(40.0) * o[4])) / T(1000);
    }
};

#endif  // __CUDACC__

}  // namespace nrlf
}  // namespace phop
