// Kernel bodies shared by the per-precision translation units.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <type_traits>

#include "nrlmsise00.cuh"
#include "propagate.cuh"

namespace phop {


// ---- RKF78 tableau (parm/integrate/rk/coefs/tableau.h:24-48) ----------------------------
__host__ __device__ constexpr double rkA(int s, int j) {
    // s = stage - 1 (row), j = column; rows list the nonzero Fehlberg coefficients
    return s == 0 ? (j == 0 ? 2. / 27 : 0)
         : s == 1 ? (j == 0 ? 1. / 36 : j == 1 ? 1. / 12 : 0)
         : s == 2 ? (j == 0 ? 1. / 24 : j == 2 ? 1. / 8 : 0)
         : s == 3 ? (j == 0 ? 5. / 12 : j == 2 ? -25. / 16 : j == 3 ? 25. / 16 : 0)
         : s == 4 ? (j == 0 ? 1. / 20 : j == 3 ? 1. / 4 : j == 4 ? 1. / 5 : 0)
         : s == 5 ? (j == 0 ? -25. / 108 : j == 3 ? 125. / 108 : j == 4 ? -65. / 27 : j == 5 ? 125. / 54 : 0)
         : s == 6 ? (j == 0 ? 31. / 300 : j == 4 ? 61. / 225 : j == 5 ? -2. / 9 : j == 6 ? 13. / 900 : 0)
         : s == 7 ? (j == 0 ? 2.0 : j == 3 ? -53. / 6 : j == 4 ? 704. / 45 : j == 5 ? -107. / 9
                    : j == 6 ? 67. / 90 : j == 7 ? 3.0 : 0)
         : s == 8 ? (j == 0 ? -91. / 108 : j == 3 ? 23. / 108 : j == 4 ? -976. / 135 : j == 5 ? 311. / 54
                    : j == 6 ? -19. / 60 : j == 7 ? 17. / 6 : j == 8 ? -1. / 12 : 0)
         : s == 9 ? (j == 0 ? 2383. / 4100 : j == 3 ? -341. / 164 : j == 4 ? 4496. / 1025 : j == 5 ? -301. / 82
                    : j == 6 ? 2133. / 4100 : j == 7 ? 45. / 82 : j == 8 ? 45. / 164 : j == 9 ? 18. / 41 : 0)
         : s == 10 ? (j == 0 ? 3. / 205 : j == 5 ? -6. / 41 : j == 6 ? -3. / 205 : j == 7 ? -3. / 41
                     : j == 8 ? 3. / 41 : j == 9 ? 6. / 41 : 0)
         : s == 11 ? (j == 0 ? -1777. / 4100 : j == 3 ? -341. / 164 : j == 4 ? 4496. / 1025 : j == 5 ? -289. / 82
                     : j == 6 ? 2193. / 4100 : j == 7 ? 51. / 82 : j == 8 ? 33. / 164 : j == 9 ? 12. / 41
                     : j == 11 ? 1.0 : 0)
         : 0;
}
__host__ __device__ constexpr double rkC(int s) {
    return s == 0 ? 2. / 27 : s == 1 ? 1. / 9 : s == 2 ? 1. / 6 : s == 3 ? 5. / 12 : s == 4 ? 1. / 2
         : s == 5 ? 5. / 6 : s == 6 ? 1. / 6 : s == 7 ? 2. / 3 : s == 8 ? 1. / 3 : s == 9 ? 1.0
         : s == 10 ? 0 : 1.0;
}
__host__ __device__ constexpr double rkB(int s) {
    return s == 5 ? 34. / 105 : s == 6 ? 9. / 35 : s == 7 ? 9. / 35 : s == 8 ? 9. / 280 : s == 9 ? 9. / 280
         : s == 11 ? 41. / 840 : s == 12 ? 41. / 840 : 0;
}

// ---- RK stage storage ------------------------------------------------------------------------
// Lane j of a group owns state components d = j + c*L (c < CPL).  The stage
// derivatives live in shared memory, [stage][component slot][thread], so that
// consecutive threads hit consecutive banks.
static __constant__ double c_rkA[12][12] = {
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

template <int CPL>
struct StageStore {
    double* base;  // shared memory, 13 * CPL * blockDim doubles
    int stride;    // blockDim.x
    __device__ __forceinline__ double& at(int s, int c) const {
        return base[((s * CPL) + c) * stride + threadIdx.x];
    }
};

// y_s = y + sum_j (dt a_sj) k_j in stage order (Step.h:33-84)
template <int CPL>
static __device__ __forceinline__ void combine(int s, const double (&y)[CPL], const StageStore<CPL>& k, double dt,
                                        double (&ys)[CPL]) {
#pragma unroll
    for (int c = 0; c < CPL; ++c) ys[c] = y[c];
    for (int jj = 0; jj < s; ++jj) {
        const double a = c_rkA[s - 1][jj];
        if (a != 0.0) {
            const double coef = dt * a;
#pragma unroll
            for (int c = 0; c < CPL; ++c) ys[c] = fma(coef, k.at(jj, c), ys[c]);
        }
    }
}

// y += sum_s (dt b_s) k_s in stage order (Step.h:86-104)
template <int CPL>
static __device__ __forceinline__ void finalUpdate(double (&y)[CPL], const StageStore<CPL>& k, double dt, bool apply) {
    double yn[CPL];
#pragma unroll
    for (int c = 0; c < CPL; ++c) yn[c] = y[c];
#pragma unroll
    for (int s = 0; s < 13; ++s)
        if (rkB(s) != 0.0) {
            const double cb = dt * rkB(s);
#pragma unroll
            for (int c = 0; c < CPL; ++c) yn[c] = fma(cb, k.at(s, c), yn[c]);
        }
    if (apply) {
#pragma unroll
        for (int c = 0; c < CPL; ++c) y[c] = yn[c];
    }
}

// ---- epoch records as the force model reads them -----------------------------------------
// A shared-grid batch reads the precomputed record of its (step, stage) in
// place.  A per-object-time batch interpolates each field where the force
// model reads it (4-point Lagrange in the batch's record grid, weights
// depending on the epoch alone), so no record is copied into the thread's
// local memory.
struct RecordRef {
    const EpochRecord* r;
    // the record of the object held by lane (lane ^ delta)
    __device__ __forceinline__ RecordRef partner(unsigned mask, int delta) const {
        const unsigned long long q = __shfl_xor_sync(mask, (unsigned long long)r, delta);
        return RecordRef{(const EpochRecord*)q};
    }
    __device__ __forceinline__ double R(int i) const { return r->R[i]; }
    __device__ __forceinline__ double W(int i) const { return r->w[i]; }
    __device__ __forceinline__ double body(int b, int i) const { return r->body[b][i]; }
    __device__ __forceinline__ double indirect(int i) const { return r->indirect[i]; }
    __device__ __forceinline__ double dC(int k) const { return r->dC[k]; }
    __device__ __forceinline__ double dS(int k) const { return r->dS[k]; }
    __device__ __forceinline__ double pole(int k, int i) const { return r->pole[k][i]; }
    __device__ __forceinline__ double poleW(int k, int i) const { return r->poleW[k][i]; }
    __device__ __forceinline__ double poleV(int k, int i) const { return r->poleV[k][i]; }
    __device__ __forceinline__ double SR(int i) const { return r->fieldR[i]; }
    // NRLMSISE-00 time inputs; valid = -1 (evaluate at the epoch in `sec`
    // when an object below the cut-off needs them) when the record has none
    __device__ __forceinline__ NrlTime nrlDeferred() const {
        NrlTime t{r->nrlSec, r->nrlGast, r->nrlBlock, r->nrlValid};
        if (t.valid < 0) t.sec = r->et;
        return t;
    }
};

struct RecordInterp {
    // value pairs of the stencil's records i0, i0 + 1 (field f at g[f]); those
    // of records i0 + 2, i0 + 3 follow 2 kInterpFields pairs later
    const double2* g;
    double w0, w1, w2, w3;
    double et;        // the stage epoch (TDB s past J2000)
    __device__ __forceinline__ RecordInterp partner(unsigned mask, int delta) const {
        RecordInterp o;
        o.g = (const double2*)__shfl_xor_sync(mask, (unsigned long long)g, delta);
        o.w0 = __shfl_xor_sync(mask, w0, delta);
        o.w1 = __shfl_xor_sync(mask, w1, delta);
        o.w2 = __shfl_xor_sync(mask, w2, delta);
        o.w3 = __shfl_xor_sync(mask, w3, delta);
        o.et = __shfl_xor_sync(mask, et, delta);
        return o;
    }
    // explicit roundings: every copy of this code gives the same bits (the
    // geopotential of lane-group pairs evaluates it for both objects)
    __device__ __forceinline__ double at(int off) const {
        const double2 x = g[off], y = g[2 * kInterpFields + off];
        return __fma_rn(w3, y.y, __fma_rn(w2, y.x, __fma_rn(w1, x.y, __dmul_rn(w0, x.x))));
    }
    __device__ __forceinline__ double R(int i) const { return at((int)(offsetof(EpochRecord, R) / 8) + i); }
    __device__ __forceinline__ double W(int i) const { return at((int)(offsetof(EpochRecord, w) / 8) + i); }
    __device__ __forceinline__ double body(int b, int i) const {
        return at((int)(offsetof(EpochRecord, body) / 8) + 3 * b + i);
    }
    __device__ __forceinline__ double indirect(int i) const {
        return at((int)(offsetof(EpochRecord, indirect) / 8) + i);
    }
    __device__ __forceinline__ double dC(int k) const { return at((int)(offsetof(EpochRecord, dC) / 8) + k); }
    __device__ __forceinline__ double dS(int k) const { return at((int)(offsetof(EpochRecord, dS) / 8) + k); }
    __device__ __forceinline__ double pole(int k, int i) const {
        return at((int)(offsetof(EpochRecord, pole) / 8) + 3 * k + i);
    }
    __device__ __forceinline__ double poleW(int k, int i) const {
        return at((int)(offsetof(EpochRecord, poleW) / 8) + 3 * k + i);
    }
    __device__ __forceinline__ double poleV(int k, int i) const {
        return at((int)(offsetof(EpochRecord, poleV) / 8) + 3 * k + i);
    }
    __device__ __forceinline__ double SR(int i) const { return at((int)(offsetof(EpochRecord, fieldR) / 8) + i); }
    // NRLMSISE-00 time inputs: evaluated exactly at the stage epoch by the
    // drag model, only for objects below the density cut-off
    __device__ __forceinline__ NrlTime nrlDeferred() const { return NrlTime{et, 0.0, 0, -1}; }
};

// body-fixed (ITRF) components of an inertial vector, and back
template <class Rec>
static __device__ __forceinline__ void toBody(const Rec& r, const double v[3], double out[3]) {
    out[0] = r.R(0) * v[0] + r.R(1) * v[1] + r.R(2) * v[2];
    out[1] = r.R(3) * v[0] + r.R(4) * v[1] + r.R(5) * v[2];
    out[2] = r.R(6) * v[0] + r.R(7) * v[1] + r.R(8) * v[2];
}
template <class Rec>
static __device__ __forceinline__ void fromBody(const Rec& r, const double a[3], double out[3]) {
    out[0] = r.R(0) * a[0] + r.R(3) * a[1] + r.R(6) * a[2];
    out[1] = r.R(1) * a[0] + r.R(4) * a[1] + r.R(7) * a[2];
    out[2] = r.R(2) * a[0] + r.R(5) * a[1] + r.R(8) * a[2];
}

// ---- spherical harmonics, lane-split over orders --------------------------------------------
template <int L, typename T, class Rec>
static __device__ __forceinline__ void shAccel(const StepParams& p, const typename TileOf<T>::type* __restrict__ tile,
                                        const Rec& rec, double x, double y, double z, double out[3]) {
    using Tile = typename TileOf<T>::type;
    const int j = (int)(threadIdx.x % L);
    const int N = p.env.shDegree, M = p.env.shOrder;
    const int lowDeg = p.lowDeg;
    const bool tides = p.env.shTides != 0;
    const LowTable* __restrict__ low = p.low;
    const double* __restrict__ diagC = p.diagC;
    const double rn = sqrt(x * x + y * y + z * z);
    const double rho = sqrt(x * x + y * y);
    const double sinPhi = z / rn, cosPhi = rho / rn;
    const double sinL = rho > 1e-14 ? y / rho : 0.0;
    const double cosL = rho > 1e-14 ? x / rho : 1.0;
    const double alpha = p.env.shR / rn;
    const double invCos = cosPhi == 0.0 ? 0.0 : 1.0 / cosPhi;
    // diagonal state (reference recurrences) for this lane's first column
    double Pmm = 1.0, dPmm = 0.0, cML = 1.0, sML = 0.0, am = 1.0;
    int m = 0;
    auto advance = [&]() {
        const double ns = cosL * sML + sinL * cML;
        const double nc = cosL * cML - sinL * sML;
        sML = ns;
        cML = nc;
        const double cm = diagC[m + 1];
        const double nP = cm * cosPhi * Pmm;
        const double ndP = cm * (cosPhi * dPmm - sinPhi * Pmm);
        Pmm = nP;
        dPmm = ndP;
        am *= alpha;
        ++m;
    };
    for (int t = 0; t < j; ++t)
        if (m < M) advance();
    // block advance m -> m + L in one step where the per-L factor table is
    // present: P_{m+L} = D_m cos^L P_m and dP_{m+L} = D'_m cos^L dP_m with
    // D_m = c_{m+1} ... c_{m+L}, D'_m = D_m (m+L)/m (closed forms of the
    // diagonal recurrences; m = 0 starts from dP_L = -L sin cos^{L-1} D_0), the
    // phasor rotated by L lambda and alpha^m scaled by alpha^L.
    const double2* __restrict__ diagStep = p.diagStep;
    double cosL1 = 1.0, cLam = 1.0, sLam = 0.0, aL = 1.0;
    if (L > 1 && diagStep) {
#pragma unroll
        for (int t = 0; t < L - 1; ++t) cosL1 *= cosPhi;
#pragma unroll
        for (int t = 0; t < L; ++t) {
            const double ns = cosL * sLam + sinL * cLam;
            const double nc = cosL * cLam - sinL * sLam;
            sLam = ns;
            cLam = nc;
            aL *= alpha;
        }
    }
    const double cosLp = cosL1 * cosPhi;
    const T u = T(alpha * sinPhi), v = T(alpha * cosPhi), a2 = T(alpha * alpha);
    double ar = 0.0, aphi = 0.0, alam = 0.0;
    const int nblocks = p.nblocks;
    for (int b = 0; b < nblocks; ++b) {
        const int mcol = b * L + j;
        const bool act = mcol <= M;
        double SA0 = 0, SA1 = 0, SA2 = 0, SA3 = 0, SA4 = 0, SA5 = 0;
        T P = T(0), P1 = T(0), dP = T(0), dP1 = T(0);
        if (act && mcol <= lowDeg) {
            // n = mcol .. lowDeg in FP64 with the epoch's tide deltas (n <= 6)
            double Pn = Pmm, Pn1 = 0.0, dPn = dPmm, dPn1 = 0.0, an = am, anPrev = am;
            const int nEnd = N < lowDeg ? N : lowDeg;
            for (int n = mcol; n <= nEnd; ++n) {
                const int ti = n * (n + 1) / 2 + mcol;
                // order 0 has no sine term: nothing to read for it
                double c = low->C[ti], s = mcol == 0 ? 0.0 : low->S[ti];
                if (n <= 6 && tides) {
                    c += rec.dC(ti);
                    if (mcol != 0) s += rec.dS(ti);
                }
                const double q = an * Pn, qd = an * dPn, np1 = (double)(n + 1);
                SA0 = fma(np1 * c, q, SA0);
                SA1 = fma(np1 * s, q, SA1);
                SA2 = fma(c, qd, SA2);
                SA3 = fma(s, qd, SA3);
                SA4 = fma(c, q, SA4);
                SA5 = fma(s, q, SA5);
                if (n < N) {
                    const int tn = (n + 1) * (n + 2) / 2 + mcol;
                    const double fa = low->a[tn], fb = low->b[tn];
                    const double P2 = Pn1;
                    Pn1 = Pn;
                    Pn = fa * sinPhi * Pn1 - fb * P2;
                    const double dP2 = dPn1;
                    dPn1 = dPn;
                    dPn = fa * (sinPhi * dPn1 + cosPhi * Pn1) - fb * dP2;
                    anPrev = an;
                    an *= alpha;
                }
            }
            P = T(an * Pn);
            P1 = T(anPrev * Pn1);
            dP = T(an * dPn);
            dP1 = T(anPrev * dPn1);
        } else if (act) {
            P = T(am * Pmm);
            dP = T(am * dPmm);
        }
        // n > 8 part from the lane-interleaved tile
        const int2 blk = p.blocks[b];
        T Scc = T(0), Ssc = T(0), Sdc = T(0), Sds = T(0), Spc = T(0), Sps = T(0);
        const Tile* tp = tile + blk.x + j;
        for (int i = 0; i < blk.y; ++i, tp += L) {
            const Tile e = *tp;
            Scc = fma(T(e.cp), P, Scc);
            Ssc = fma(T(e.sp), P, Ssc);
            Spc = fma(T(e.c), P, Spc);
            Sps = fma(T(e.s), P, Sps);
            Sdc = fma(T(e.c), dP, Sdc);
            Sds = fma(T(e.s), dP, Sds);
            const T Pn = fma(T(e.a), u * P, -T(e.b) * (a2 * P1));
            const T dPn = fma(T(e.a), fma(u, dP, v * P), -T(e.b) * (a2 * dP1));
            P1 = P;
            P = Pn;
            dP1 = dP;
            dP = dPn;
        }
        if (act) {
            const double cc = SA0 + (double)Scc, sc = SA1 + (double)Ssc;
            const double dc = SA2 + (double)Sdc, ds = SA3 + (double)Sds;
            const double pc = SA4 + (double)Spc, ps = SA5 + (double)Sps;
            ar -= cML * cc + sML * sc;
            aphi += cML * dc + sML * ds;
            alam -= ((double)mcol * invCos) * (sML * pc - cML * ps);
        }
        if (L > 1 && diagStep) {
            if (m + L <= M) {
                const double2 f = diagStep[m];
                const double nP = f.x * cosLp * Pmm;
                const double ndP = m == 0 ? -(double)L * sinPhi * cosL1 * f.x : f.y * cosLp * dPmm;
                Pmm = nP;
                dPmm = ndP;
                const double ns = cLam * sML + sLam * cML;
                const double nc = cLam * cML - sLam * sML;
                sML = ns;
                cML = nc;
                am *= aL;
                m += L;
            } else {
                m = M + 1;  // beyond the last order: the lane's later columns are inactive
            }
        } else {
            for (int t = 0; t < L; ++t)
                if (m < M) advance();
        }
    }
    // fold the group's partial sums (the group's lanes only: in split
    // precision groups of one warp may take different precisions)
    const unsigned groupMask = L >= 32 ? 0xffffffffu : (((1u << L) - 1u) << ((threadIdx.x & 31) - j));
#pragma unroll
    for (int off = L / 2; off > 0; off >>= 1) {
        ar += __shfl_xor_sync(groupMask, ar, off);
        aphi += __shfl_xor_sync(groupMask, aphi, off);
        alam += __shfl_xor_sync(groupMask, alam, off);
    }
    if (cosPhi == 0.0 && M >= 1) {
        // exact pole: the m = 1 longitudinal term takes its analytical limit
        // (DegreeLoop.h:98-103, Coefficients.h:123-131)
        double an = alpha;
        for (int n = 1; n <= N; ++n) {
            const int ti = n * (n + 1) / 2 + 1;
            double s = p.env.shS[ti];
            if (n <= 6 && tides) s += rec.dS(ti);
            const double sign = sinPhi > 0.0 ? 1.0 : ((n & 1) ? 1.0 : -1.0);
            double lim = 0.5 * (double)n * (n + 1.0);
            if (p.env.shNormalized) lim *= sqrt(2.0 * (2.0 * n + 1.0) / ((double)n * (n + 1.0)));
            // S~ = c sin(l) - s cos(l) with sin(l) = 0, cos(l) = 1 at the pole
            alam -= an * (sign * lim) * (-s);
            an *= alpha;
        }
    }
    const double g = p.env.shGM / (rn * rn);
    ar *= g;
    aphi *= g;
    alam *= g;
    out[0] = cosPhi * cosL * ar - sinPhi * cosL * aphi - sinL * alam;
    out[1] = cosPhi * sinL * ar - sinPhi * sinL * aphi + cosL * alam;
    out[2] = sinPhi * ar + cosPhi * aphi;
}

// ---- spherical harmonics for a pair of objects, packed FP32 ---------------------------------
// Two FP32 values in one 64-bit register pair, operated on by the packed
// f32x2 instructions of sm_100.
struct F2 {
    unsigned long long v;
};
static __device__ __forceinline__ F2 f2(float lo, float hi) {
    F2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(lo), "f"(hi));
    return r;
}
static __device__ __forceinline__ F2 f2fma(F2 a, F2 b, F2 c) {
    F2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return d;
}
static __device__ __forceinline__ F2 f2mul(F2 a, F2 b) {
    F2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
static __device__ __forceinline__ void f2split(F2 a, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a.v));
}
// The FP64 form of the same pair: two doubles, operated on one by one.
struct D2 {
    double lo, hi;
};
template <typename T> struct PairOf;
template <> struct PairOf<float> {
    using type = F2;
    static __device__ __forceinline__ F2 make(float a, float b) { return f2(a, b); }
    static __device__ __forceinline__ F2 fma(F2 a, F2 b, F2 c) { return f2fma(a, b, c); }
    static __device__ __forceinline__ F2 mul(F2 a, F2 b) { return f2mul(a, b); }
    static __device__ __forceinline__ void split(F2 a, float& lo, float& hi) { f2split(a, lo, hi); }
};
template <> struct PairOf<double> {
    using type = D2;
    static __device__ __forceinline__ D2 make(double a, double b) { return D2{a, b}; }
    static __device__ __forceinline__ D2 fma(D2 a, D2 b, D2 c) { return D2{::fma(a.lo, b.lo, c.lo), ::fma(a.hi, b.hi, c.hi)}; }
    static __device__ __forceinline__ D2 mul(D2 a, D2 b) { return D2{__dmul_rn(a.lo, b.lo), __dmul_rn(a.hi, b.hi)}; }
    static __device__ __forceinline__ void split(D2 a, double& lo, double& hi) {
        lo = a.lo;
        hi = a.hi;
    }
};

// Per-object quantities of the column recursion.
struct ShGeo {
    double sinPhi, cosPhi, sinL, cosL, alpha, invCos;
};
// The per-object parts of the pair geopotential (shGeo, shDiagStart,
// shDiagStep, shLowColumn and the column sums) are written with explicit
// roundings (__fma_rn, __dmul_rn, ...): each lane evaluates them for both
// objects of its pair, in two copies of the code, and an object's result must
// not depend on whether it is the pair's first or second object (that is, on
// which other object shares its warp).  Plain expressions would leave each
// copy's multiply-add contraction to the compiler.
static __device__ __forceinline__ ShGeo shGeo(double x, double y, double z, double R) {
    ShGeo g;
    const double rho2 = __fma_rn(y, y, __dmul_rn(x, x));
    const double rn = __dsqrt_rn(__fma_rn(z, z, rho2));
    const double rho = __dsqrt_rn(rho2);
    g.sinPhi = __ddiv_rn(z, rn);
    g.cosPhi = __ddiv_rn(rho, rn);
    g.sinL = rho > 1e-14 ? __ddiv_rn(y, rho) : 0.0;
    g.cosL = rho > 1e-14 ? __ddiv_rn(x, rho) : 1.0;
    g.alpha = __ddiv_rn(R, rn);
    g.invCos = g.cosPhi == 0.0 ? 0.0 : __drcp_rn(g.cosPhi);
    return g;
}

// Diagonal of one object: P_mm, dP_mm, cos / sin m lambda, alpha^m, and the
// closed-form step by W orders (P_{m+W} = D_m cos^W P_m, the phasor rotated
// by W lambda, alpha^W), as shAccel forms them.
struct ShDiag {
    double Pmm, dPmm, cML, sML, am;
    double cosW1, cLam, sLam, aW;  // cos^(W-1) phi, cos / sin W lambda, alpha^W
};

// FP64 low part of column `mcol` of one object (n = mcol .. lowDeg, tide
// deltas for n <= 6): the six column sums and the FP32 start values of the
// tile rows (degrees lowDeg + 1 and lowDeg).
template <typename T, class Rec>
static __device__ __forceinline__ void shLowColumn(const StepParams& p, const Rec& rec, const ShGeo& g,
                                                   const ShDiag& d, int mcol, double S[6], T& P, T& P1, T& dP,
                                                   T& dP1) {
    const LowTable* __restrict__ low = p.low;
    const int N = p.env.shDegree, lowDeg = p.lowDeg;
    const bool tides = p.env.shTides != 0;
    double Pn = d.Pmm, Pn1 = 0.0, dPn = d.dPmm, dPn1 = 0.0, an = d.am, anPrev = d.am;
    const int nEnd = N < lowDeg ? N : lowDeg;
    for (int k = 0; k < 6; ++k) S[k] = 0.0;
    for (int n = mcol; n <= nEnd; ++n) {
        const int ti = n * (n + 1) / 2 + mcol;
        // order 0 has no sine term: nothing to read for it
        double c = low->C[ti], s = mcol == 0 ? 0.0 : low->S[ti];
        if (n <= 6 && tides) {
            c = __dadd_rn(c, rec.dC(ti));
            if (mcol != 0) s = __dadd_rn(s, rec.dS(ti));
        }
        const double q = __dmul_rn(an, Pn), qd = __dmul_rn(an, dPn), np1 = (double)(n + 1);
        S[0] = __fma_rn(__dmul_rn(np1, c), q, S[0]);
        S[1] = __fma_rn(__dmul_rn(np1, s), q, S[1]);
        S[2] = __fma_rn(c, qd, S[2]);
        S[3] = __fma_rn(s, qd, S[3]);
        S[4] = __fma_rn(c, q, S[4]);
        S[5] = __fma_rn(s, q, S[5]);
        if (n < N) {
            const int tn = (n + 1) * (n + 2) / 2 + mcol;
            const double fa = low->a[tn], fb = low->b[tn];
            const double P2 = Pn1;
            Pn1 = Pn;
            Pn = __fma_rn(__dmul_rn(fa, g.sinPhi), Pn1, -__dmul_rn(fb, P2));
            const double dP2 = dPn1;
            dPn1 = dPn;
            dPn = __fma_rn(fa, __fma_rn(g.sinPhi, dPn1, __dmul_rn(g.cosPhi, Pn1)), -__dmul_rn(fb, dP2));
            anPrev = an;
            an = __dmul_rn(an, g.alpha);
        }
    }
    P = (T)__dmul_rn(an, Pn);
    P1 = (T)__dmul_rn(anPrev, Pn1);
    dP = (T)__dmul_rn(an, dPn);
    dP1 = (T)__dmul_rn(anPrev, dPn1);
}

static __device__ __forceinline__ void shDiagStart(const StepParams& p, const ShGeo& g, int first, int W,
                                                   ShDiag& d) {
    const double* __restrict__ diagC = p.diagC;
    const int M = p.env.shOrder;
    d.Pmm = 1.0;
    d.dPmm = 0.0;
    d.cML = 1.0;
    d.sML = 0.0;
    d.am = 1.0;
    for (int m = 0; m < first && m < M; ++m) {
        const double ns = __fma_rn(g.cosL, d.sML, __dmul_rn(g.sinL, d.cML));
        const double nc = __fma_rn(g.cosL, d.cML, -__dmul_rn(g.sinL, d.sML));
        d.sML = ns;
        d.cML = nc;
        const double cm = diagC[m + 1];
        const double nP = __dmul_rn(__dmul_rn(cm, g.cosPhi), d.Pmm);
        const double ndP = __dmul_rn(cm, __fma_rn(g.cosPhi, d.dPmm, -__dmul_rn(g.sinPhi, d.Pmm)));
        d.Pmm = nP;
        d.dPmm = ndP;
        d.am = __dmul_rn(d.am, g.alpha);
    }
    d.cosW1 = 1.0;
    d.cLam = 1.0;
    d.sLam = 0.0;
    d.aW = 1.0;
    for (int t = 0; t < W - 1; ++t) d.cosW1 = __dmul_rn(d.cosW1, g.cosPhi);
    for (int t = 0; t < W; ++t) {
        const double ns = __fma_rn(g.cosL, d.sLam, __dmul_rn(g.sinL, d.cLam));
        const double nc = __fma_rn(g.cosL, d.cLam, -__dmul_rn(g.sinL, d.sLam));
        d.sLam = ns;
        d.cLam = nc;
        d.aW = __dmul_rn(d.aW, g.alpha);
    }
}

// advance the diagonal from order m to m + W (shAccel's block step)
static __device__ __forceinline__ void shDiagStep(const double2* __restrict__ diagStep, const ShGeo& g, int m, int W,
                                                  ShDiag& d) {
    const double2 f = diagStep[m];
    const double cosWp = __dmul_rn(d.cosW1, g.cosPhi);
    const double nP = __dmul_rn(__dmul_rn(f.x, cosWp), d.Pmm);
    const double ndP = m == 0 ? __dmul_rn(__dmul_rn(__dmul_rn(-(double)W, g.sinPhi), d.cosW1), f.x)
                              : __dmul_rn(__dmul_rn(f.y, cosWp), d.dPmm);
    d.Pmm = nP;
    d.dPmm = ndP;
    const double ns = __fma_rn(d.cLam, d.sML, __dmul_rn(d.sLam, d.cML));
    const double nc = __fma_rn(d.cLam, d.cML, -__dmul_rn(d.sLam, d.sML));
    d.sML = ns;
    d.cML = nc;
    d.am = __dmul_rn(d.am, d.aW);
}

// one column's contribution (FP64 low sums S plus the tile part t) to an
// object's (ar, aphi, alam) partial sums
template <typename T>
static __device__ __forceinline__ void columnSums(int mcol, const ShGeo& g, const ShDiag& d, const double S[6],
                                                  const T t[6], double acc[3]) {
    double c[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) c[k] = __dadd_rn(S[k], (double)t[k]);
    const double mInv = __dmul_rn((double)mcol, g.invCos);
    acc[0] = __dsub_rn(acc[0], __fma_rn(d.cML, c[0], __dmul_rn(d.sML, c[1])));
    acc[1] = __dadd_rn(acc[1], __fma_rn(d.cML, c[2], __dmul_rn(d.sML, c[3])));
    acc[2] = __dsub_rn(acc[2], __dmul_rn(mInv, __fma_rn(d.sML, c[4], -__dmul_rn(d.cML, c[5]))));
}

// Geopotential of the two objects of a pair of lane groups: the 2L lanes of
// groups 2k and 2k+1 split the orders (lane pj of the pair takes
// m = b 2L + pj, from the tile built for 2L lanes) and every lane runs its
// columns for both objects (object of the first group, object of the
// second), so each coefficient loaded from shared memory serves two objects
// -- the column loop is bound by shared-memory bandwidth, not arithmetic.
// Split precision runs the tile part as packed FP32 pairs (f32x2); FP64
// runs it as two interleaved columns.  The low part and the diagonal stay
// FP64 per object.  Returns the calling lane's own object's acceleration
// (body frame, km/s^2), the same on every lane of its group.
template <int L, typename T, class Rec>
static __device__ __forceinline__ void shAccelPair(const StepParams& p, const typename TileOf<T>::type* __restrict__ tile,
                                                   const Rec& rec, double x, double y, double z, double out[3]) {
    using Pr = PairOf<T>;
    using V = typename Pr::type;
    using Tile = typename TileOf<T>::type;
    constexpr int W = 2 * L;
    const int lane = (int)(threadIdx.x & 31);
    const int pj = lane % W;
    const bool second = pj >= L;
    const unsigned pairMask = W >= 32 ? 0xffffffffu : (((1u << W) - 1u) << (lane - pj));
    const int N = p.env.shDegree, M = p.env.shOrder;
    const int lowDeg = p.lowDeg;
    const double ox = __shfl_xor_sync(pairMask, x, L), oy = __shfl_xor_sync(pairMask, y, L),
                 oz = __shfl_xor_sync(pairMask, z, L);
    const Rec orec = rec.partner(pairMask, L);
    const ShGeo g0 = second ? shGeo(ox, oy, oz, p.env.shR) : shGeo(x, y, z, p.env.shR);
    const ShGeo g1 = second ? shGeo(x, y, z, p.env.shR) : shGeo(ox, oy, oz, p.env.shR);
    const Rec& r0 = second ? orec : rec;
    const Rec& r1 = second ? rec : orec;
    ShDiag d0, d1;
    shDiagStart(p, g0, pj, W, d0);
    shDiagStart(p, g1, pj, W, d1);
    const V u = Pr::make((T)(g0.alpha * g0.sinPhi), (T)(g1.alpha * g1.sinPhi));
    const V v = Pr::make((T)(g0.alpha * g0.cosPhi), (T)(g1.alpha * g1.cosPhi));
    const V a2 = Pr::make((T)(g0.alpha * g0.alpha), (T)(g1.alpha * g1.alpha));
    double acc0[3] = {0.0, 0.0, 0.0}, acc1[3] = {0.0, 0.0, 0.0};  // ar, aphi, alam
    const double2* __restrict__ diagStep = p.diagStep;
    const int nblocks = p.nblocks;
    for (int b = 0; b < nblocks; ++b) {
        const int mcol = b * W + pj;
        const bool act = mcol <= M;
        double S0[6] = {0, 0, 0, 0, 0, 0}, S1[6] = {0, 0, 0, 0, 0, 0};
        T P0 = T(0), P10 = T(0), dP0 = T(0), dP10 = T(0), P1_ = T(0), P11 = T(0), dP1_ = T(0), dP11 = T(0);
        if (act && mcol <= lowDeg) {
            shLowColumn<T>(p, r0, g0, d0, mcol, S0, P0, P10, dP0, dP10);
            shLowColumn<T>(p, r1, g1, d1, mcol, S1, P1_, P11, dP1_, dP11);
        } else if (act) {
            P0 = (T)(d0.am * d0.Pmm);
            dP0 = (T)(d0.am * d0.dPmm);
            P1_ = (T)(d1.am * d1.Pmm);
            dP1_ = (T)(d1.am * d1.dPmm);
        }
        V P = Pr::make(P0, P1_), Pm1 = Pr::make(P10, P11), dP = Pr::make(dP0, dP1_), dPm1 = Pr::make(dP10, dP11);
        V Scc = Pr::make(T(0), T(0)), Ssc = Scc, Spc = Scc, Sps = Scc, Sdc = Scc, Sds = Scc;
        const int2 blk = p.blocks[b];
        const Tile* tp = tile + blk.x + pj;
        for (int i = 0; i < blk.y; ++i, tp += W) {
            const Tile e = *tp;
            const V c = Pr::make(T(e.c), T(e.c)), s = Pr::make(T(e.s), T(e.s));
            const V cp = Pr::make(T(e.cp), T(e.cp)), sp = Pr::make(T(e.sp), T(e.sp));
            const V fa = Pr::make(T(e.a), T(e.a)), nb = Pr::make(-T(e.b), -T(e.b));
            Scc = Pr::fma(cp, P, Scc);
            Ssc = Pr::fma(sp, P, Ssc);
            Spc = Pr::fma(c, P, Spc);
            Sps = Pr::fma(s, P, Sps);
            Sdc = Pr::fma(c, dP, Sdc);
            Sds = Pr::fma(s, dP, Sds);
            const V Pn = Pr::fma(fa, Pr::mul(u, P), Pr::mul(nb, Pr::mul(a2, Pm1)));
            const V dPn = Pr::fma(fa, Pr::fma(u, dP, Pr::mul(v, P)), Pr::mul(nb, Pr::mul(a2, dPm1)));
            Pm1 = P;
            P = Pn;
            dPm1 = dP;
            dP = dPn;
        }
        if (act) {
            T t0[6], t1[6];
            Pr::split(Scc, t0[0], t1[0]);
            Pr::split(Ssc, t0[1], t1[1]);
            Pr::split(Sdc, t0[2], t1[2]);
            Pr::split(Sds, t0[3], t1[3]);
            Pr::split(Spc, t0[4], t1[4]);
            Pr::split(Sps, t0[5], t1[5]);
            columnSums<T>(mcol, g0, d0, S0, t0, acc0);
            columnSums<T>(mcol, g1, d1, S1, t1, acc1);
        }
        const int m = b * W + pj;
        if (m + W <= M) {
            shDiagStep(diagStep, g0, m, W, d0);
            shDiagStep(diagStep, g1, m, W, d1);
        }
    }
    // fold the pair's lanes: both objects' partial sums over all 2L lanes
#pragma unroll
    for (int off = W / 2; off > 0; off >>= 1)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            acc0[k] += __shfl_xor_sync(pairMask, acc0[k], off);
            acc1[k] += __shfl_xor_sync(pairMask, acc1[k], off);
        }
    const ShGeo& g = second ? g1 : g0;
    double ar = second ? acc1[0] : acc0[0], aphi = second ? acc1[1] : acc0[1], alam = second ? acc1[2] : acc0[2];
    if (g.cosPhi == 0.0 && M >= 1) {
        // exact pole: the m = 1 longitudinal term's analytical limit (as shAccel)
        const bool tides = p.env.shTides != 0;
        double an = g.alpha;
        for (int n = 1; n <= N; ++n) {
            const int ti = n * (n + 1) / 2 + 1;
            double s = p.env.shS[ti];
            if (n <= 6 && tides) s += rec.dS(ti);
            const double sign = g.sinPhi > 0.0 ? 1.0 : ((n & 1) ? 1.0 : -1.0);
            double lim = 0.5 * (double)n * (n + 1.0);
            if (p.env.shNormalized) lim *= sqrt(2.0 * (2.0 * n + 1.0) / ((double)n * (n + 1.0)));
            alam -= an * (sign * lim) * (-s);
            an *= g.alpha;
        }
    }
    (void)lowDeg;
    const double rn = p.env.shR / g.alpha;
    const double gm = p.env.shGM / (rn * rn);
    ar *= gm;
    aphi *= gm;
    alam *= gm;
    out[0] = g.cosPhi * g.cosL * ar - g.sinPhi * g.cosL * aphi - g.sinL * alam;
    out[1] = g.cosPhi * g.sinL * ar - g.sinPhi * g.sinL * aphi + g.cosL * alam;
    out[2] = g.sinPhi * ar + g.cosPhi * aphi;
}

// ---- the remaining forces ------------------------------------------------------------------
static __device__ __forceinline__ double shadowFactor(const double rS[3], const double rB[3], double RSun, double RBody) {
    const double s2 = rS[0] * rS[0] + rS[1] * rS[1] + rS[2] * rS[2];
    const double b2 = rB[0] * rB[0] + rB[1] * rB[1] + rB[2] * rB[2];
    const double sb = rS[0] * rB[0] + rS[1] * rB[1] + rS[2] * rB[2];
    const double iS = rsqrt(s2), iB = rsqrt(b2);
    if (b2 <= RBody * RBody) return 0.0;
    {
        // clear full sunlight (c > a + b) or full shadow of a body larger
        // than the Sun's disc (c < b - a), decided on cosines without the
        // inverse trigonometric functions; within 1e-9 of either boundary
        // the angles below decide, as the reference's evaluation does
        const double sa = fmin(fmax(RSun * iS, 0.0), 1.0), sbd = fmin(fmax(RBody * iB, 0.0), 1.0);
        const double ca = sqrt(1.0 - sa * sa), cb = sqrt(1.0 - sbd * sbd);
        const double cc = fmin(fmax(sb * iS * iB, -1.0), 1.0);
        if (cc < ca * cb - sa * sbd - 1e-9) return 1.0;
        if (sbd > sa && cc > ca * cb + sa * sbd + 1e-9) return 0.0;
    }
    const double a = asin(fmin(fmax(RSun * iS, 0.0), 1.0));
    const double b = asin(fmin(fmax(RBody * iB, 0.0), 1.0));
    const double c = acos(fmin(fmax(sb * iS * iB, -1.0), 1.0));
    if (c >= a + b) return 1.0;
    if (c <= fabs(b - a)) return b >= a ? 0.0 : 1.0 - (b * b) / (a * a);
    const double a2 = a * a, bb = b * b, c2 = c * c;
    const double x = (c2 + a2 - bb) / (2.0 * c);
    const double yv = sqrt(fmax(a2 - x * x, 0.0));
    const double al = acos(fmin(fmax(x / a, -1.0), 1.0));
    const double be = acos(fmin(fmax((c - x) / b, -1.0), 1.0));
    return 1.0 - (a2 * al + bb * be - c * yv) / (a2 * 3.14159265358979323846);
}

// NRLMSISE-00 density (kg/km^3) at ITRF position f; the L lanes of a group
// share the globe7 tables of the model and all return the same value.
template <int L>
static __device__ __forceinline__ double nrlDensityBody(const DevEnv& e, NrlTime t, const double f[3]);

// Out of line for eight and sixteen lanes, where the caller's live state is
// small enough that the call's register saves cost less than the larger
// inlined kernel; inline for one to four lanes (measured both ways).
template <int L>
static __device__ __noinline__ double nrlDensityCall(const DevEnv& e, NrlTime t, const double f[3]) {
    return nrlDensityBody<L>(e, t, f);
}
// FP64 in both precision forms: an FP32 per-object model (the split form's
// option at one time) was slower and moved 500 km objects by more than 1 cm
// in 24 h.
template <int L>
static __device__ __forceinline__ double nrlDensity(const DevEnv& e, NrlTime t, const double f[3]) {
    if constexpr (L <= 4) return nrlDensityBody<L>(e, t, f);
    else return nrlDensityCall<L>(e, t, f);
}

template <int L>
static __device__ __forceinline__ double nrlDensityBody(const DevEnv& e, NrlTime t, const double f[3]) {
    // geodetic latitude / longitude / altitude (Nrlmsise00.cu:243-266)
    const double rho2 = f[0] * f[0] + f[1] * f[1];
    if (!(rho2 + f[2] * f[2] > 0.0)) return NAN;
    const double radius = e.earthRadius;
    const double e2 = e.flattening * (2.0 - e.flattening);
    double dz = e2 * f[2], zdz = f[2] + dz, nn = radius, nh = 0.0;
    for (int it = 0; it < 20; ++it) {
        zdz = f[2] + dz;
        const double sp = zdz * rsqrt(rho2 + zdz * zdz);
        nn = radius * rsqrt(1.0 - e2 * sp * sp);
        const double next = nn * e2 * sp;
        if (fabs(dz - next) < 1.0e-12 * radius) {
            dz = next;
            break;
        }
        dz = next;
    }
    zdz = f[2] + dz;
    nh = sqrt(rho2 + zdz * zdz);
    const double lon = atan2(f[1], f[0]);
    const double lat = atan2(zdz, sqrt(rho2));
    const double alt = nh - nn;
    if (!(isfinite(lat) && isfinite(lon) && isfinite(alt))) return NAN;
    if (alt > e.nrlHcutoff) return 0.0;
    if (t.valid < 0) t = nrlTime(e, t.sec);  // deferred: `sec` holds the stage epoch (TDB s past J2000)
    if (!t.valid) return NAN;
    const double kRad = 57.2957795130823208768;
    const double lst = wrapHours(t.gast + lon * kRad / 15.0);
    const int lane = (int)(threadIdx.x & 31);
    nrlf::Fast<double> model(e.nrlBlocks[t.block], t.sec);
    const double rhoSi = model.template density<L>(lat * kRad, lon * kRad, alt, lst, lane % L, lane - lane % L);
    if (!isfinite(rhoSi) || rhoSi < 0.0) return NAN;
    return (rhoSi * 1.0e9) * e.nrlDensityScale;
}

// Geodetic altitude about the polar axis `pole` (atmosphere/Geodetic.h:40-75);
// the fixed-point iteration converges quadratically, bounded here.
static __device__ __forceinline__ double geodeticHeight(const double r[3], const double pole[3], double Req,
                                                        double flattening) {
    const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    if (flattening == 0.0) return sqrt(r2) - Req;
    const double z = r[0] * pole[0] + r[1] * pole[1] + r[2] * pole[2];
    const double xy = r2 - z * z;
    const double flatsq = (2.0 - flattening) * flattening;
    double d0 = 0.0, d = 1e10, sfq = 0.0, zd = z;
    for (int it = 0; it < 64 && fabs(d - d0) > 1e-9; ++it) {
        d0 = d;
        const double z2 = zd * zd;
        sfq = z2 / (xy + z2);
        d = Req * flatsq * sqrt(sfq / (1.0 - flatsq * sfq));
        zd = z + copysign(d, z);
    }
    return sqrt(xy + zd * zd) - Req / sqrt(1.0 - flatsq * sfq);
}

// Tide potential alone (solid + ocean coefficient deltas of the epoch, degree
// <= 6, the tide model's GM and radius), for an Earth without a gravity field
// file: the deltas otherwise join the field's low-degree block.  The body-
// frame gradient of sum_nm (mu/r)(R/r)^n P_nm (dC cos m lon + dS sin m lon)
// in geocentric latitude/longitude, as the reference's Earth corrections
// evaluate it (hpop_compat/HpopCorrections.h:336-367); fully normalised
// Legendre functions by the column recurrences and their latitude
// derivatives in closed form (the reference recurses them alongside,
// HpopCorrections.h:121-145).
template <class Rec>
static __device__ __noinline__ void tideAloneAccel(const Rec r, const double pos[3], double acc[3]) {
    double b[3];
    toBody(r, pos, b);
    const double x = b[0], y = b[1], z = b[2];
    const double mu = tidefield::kMuEarth * 1e-9, Re = tidefield::kRadius * 1e-3;  // km^3/s^2, km
    const double xy2 = x * x + y * y, xy = sqrt(xy2);
    const double d = sqrt(xy2 + z * z);
    const double sphi = z / d, cphi = xy / d, tphi = z / xy;
    const double cl = x / xy, sl = y / xy;
    double p[7][7], dp[7][7];
    // column recurrences: P_mm from P_{m-1,m-1}, then upward in n
    p[0][0] = 1.0;
    for (int m = 0; m <= 6; ++m) {
        if (m > 0) p[m][m] = sqrt((2.0 * m + 1.0) / (m == 1 ? 1.0 : 2.0 * m)) * cphi * p[m - 1][m - 1];
        if (m < 6) p[m + 1][m] = sqrt(2.0 * m + 3.0) * sphi * p[m][m];
        for (int n = m + 2; n <= 6; ++n) {
            const double nn = (double)n, mm = (double)m;
            const double a = sqrt((4.0 * nn * nn - 1.0) / (nn * nn - mm * mm));
            const double b = sqrt((2.0 * nn + 1.0) * (nn - 1.0 - mm) * (nn - 1.0 + mm) / ((2.0 * nn - 3.0) * (nn * nn - mm * mm)));
            p[n][m] = a * sphi * p[n - 1][m] - b * p[n - 2][m];
        }
    }
    // d/dphi P_nm = k_nm P_{n,m+1} - m tan(phi) P_nm, k_n0 = sqrt(n(n+1)/2), k_nm = sqrt((n-m)(n+m+1))
    for (int n = 0; n <= 6; ++n)
        for (int m = 0; m <= n; ++m) {
            const double up = m < n ? p[n][m + 1] : 0.0;
            const double k = m == 0 ? sqrt(0.5 * n * (n + 1.0)) : sqrt((double)(n - m) * (n + m + 1.0));
            dp[n][m] = k * up - (double)m * tphi * p[n][m];
        }
    double cm[7], sm[7];
    cm[0] = 1.0;
    sm[0] = 0.0;
    for (int m = 1; m <= 6; ++m) {
        cm[m] = cl * cm[m - 1] - sl * sm[m - 1];
        sm[m] = sl * cm[m - 1] + cl * sm[m - 1];
    }
    double dUdr = 0.0, dUdlat = 0.0, dUdlon = 0.0, power = 1.0;
    const double ratio = Re / d;
    for (int n = 0; n <= 6; ++n) {
        double q1 = 0.0, q2 = 0.0, q3 = 0.0;
        for (int m = 0; m <= n; ++m) {
            const int ti = n * (n + 1) / 2 + m;
            const double c = r.dC(ti), s = r.dS(ti);
            const double v = c * cm[m] + s * sm[m];
            q1 += p[n][m] * v;
            q2 += dp[n][m] * v;
            q3 += (double)m * p[n][m] * (s * cm[m] - c * sm[m]);
        }
        dUdr += q1 * (-mu / (d * d)) * power * (n + 1.0);
        dUdlat += q2 * (mu / d) * power;
        dUdlon += q3 * (mu / d) * power;
        power *= ratio;
    }
    const double q = dUdr / d - z / (d * d * xy) * dUdlat;
    const double bf0 = q * x - (dUdlon / xy2) * y, bf1 = q * y + (dUdlon / xy2) * x;
    const double bf2 = dUdr / d * z + xy / (d * d) * dUdlat;
    const double bf[3] = {bf0, bf1, bf2};
    double a[3];
    fromBody(r, bf, a);
    acc[0] += a[0];
    acc[1] += a[1];
    acc[2] += a[2];
}

// full right-hand side acceleration (km/s^2); every lane of the group calls it.
// PAIR: the geopotential of lane-group pairs (a separate kernel instantiation,
// so the one-object-per-lane kernel keeps its own register allocation).
template <int L, typename T, bool PAIR, class Rec>
static __device__ __forceinline__ void accelerations(const StepParams& p, const typename TileOf<T>::type* tile,
                                              const Rec& r, const double pos[3], const double vel[3],
                                              double bc, double ams, double acc[3]) {
    const DevEnv& e = p.env;
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int bi = 0; bi < e.nbodies; ++bi) {
        const int fl = e.bodyFlags[bi];
        const bool isEarth = (bi == e.earthIndex);
        // the body-fixed position (field, J2 and NRLMSISE-00 terms) and the
        // body's position (direct attraction and radiation pressure), each
        // read from the record once
        double fb[3] = {0.0, 0.0, 0.0}, rb[3] = {0.0, 0.0, 0.0};
        if (isEarth && ((fl & (kShape | kOblateness)) || ((fl & kAtmosphere) && e.hasNrl))) toBody(r, pos, fb);
        if (((fl & (kGravity | kAtmosphere)) && !isEarth) || (fl & kRadiation)) {
            rb[0] = r.body(bi, 0);
            rb[1] = r.body(bi, 1);
            rb[2] = r.body(bi, 2);
        }
        if (fl & kGravity) {
            const double gm = e.bodyGm[bi];
            if (isEarth) {
                const double rr = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
                const double f = -gm * (1.0 / (rr * rr * rr));
                ax += f * pos[0];
                ay += f * pos[1];
                az += f * pos[2];
            } else {
                // direct part per object; the indirect part (epoch-only) is
                // the record's sum, added after the loop
                const double d0 = pos[0] - rb[0], d1 = pos[1] - rb[1], d2 = pos[2] - rb[2];
                const double ird = rsqrt(d0 * d0 + d1 * d1 + d2 * d2);
                const double f1 = -gm * (ird * ird * ird);
                ax += f1 * d0;
                ay += f1 * d1;
                az += f1 * d2;
            }
        }
        if (fl & kShape) {
            // body-fixed position: the Earth's frame, or the field body's
            // own (IAU) frame about its position
            double bx = fb[0], by = fb[1], bz = fb[2];
            if (!isEarth) {
                const double d0 = pos[0] - rb[0], d1 = pos[1] - rb[1], d2 = pos[2] - rb[2];
                bx = r.SR(0) * d0 + r.SR(1) * d1 + r.SR(2) * d2;
                by = r.SR(3) * d0 + r.SR(4) * d1 + r.SR(5) * d2;
                bz = r.SR(6) * d0 + r.SR(7) * d1 + r.SR(8) * d2;
            }
            double a[3];
            if constexpr (!std::is_same<T, double>::value) {
                // split precision: objects below the split radius keep the
                // tile part in FP64 (from the FP64 tile in global memory)
                if constexpr (PAIR)
                    shAccelPair<L, T>(p, tile, r, bx, by, bz, a);
                else if (p.splitRadius > 0.0 && bx * bx + by * by + bz * bz < p.splitRadius * p.splitRadius)
                    shAccel<L, double>(p, (const TileD*)p.tile64, r, bx, by, bz, a);
                else
                    shAccel<L, T>(p, tile, r, bx, by, bz, a);
            } else {
                if constexpr (PAIR)
                    shAccelPair<L, T>(p, tile, r, bx, by, bz, a);
                else
                    shAccel<L, T>(p, tile, r, bx, by, bz, a);
            }
            double ai[3];
            if (isEarth) {
                fromBody(r, a, ai);
            } else {
                ai[0] = r.SR(0) * a[0] + r.SR(3) * a[1] + r.SR(6) * a[2];
                ai[1] = r.SR(1) * a[0] + r.SR(4) * a[1] + r.SR(7) * a[2];
                ai[2] = r.SR(2) * a[0] + r.SR(5) * a[1] + r.SR(8) * a[2];
            }
            ax += ai[0];
            ay += ai[1];
            az += ai[2];
        }
        if ((fl & kOblateness) && !(fl & kShape) && !isEarth) {
            // J2 model of another body (J2.h:17-33,63-78, PrivateAccelerations.h:88-97):
            // position relative to the body, inside its sphere of influence;
            // the model is axisymmetric, so the body frame enters through its
            // polar axis u alone: a = c (d (1 - 5 z^2 / r^2) + 2 z u), z = u . d
            const double d0 = pos[0] - rb[0], d1 = pos[1] - rb[1], d2 = pos[2] - rb[2];
            const double rr2 = d0 * d0 + d1 * d1 + d2 * d2;
            const int slot = e.poleSlot[bi];
            if (slot >= 0 && rr2 <= e.bodySoi[bi] * e.bodySoi[bi]) {
                const double u0 = r.pole(slot, 0), u1 = r.pole(slot, 1), u2 = r.pole(slot, 2);
                const double invr = rsqrt(rr2);
                const double invr2 = invr * invr;
                const double z = u0 * d0 + u1 * d1 + u2 * d2;
                const double base = 1.0 - 5.0 * (z * z) * invr2;
                const double c = -1.5 * e.bodyGmConst[bi] * e.bodyJ2[bi] * (invr2 * invr2 * invr) * e.bodyRadius[bi]
                                 * e.bodyRadius[bi];
                ax += c * (d0 * base + 2.0 * z * u0);
                ay += c * (d1 * base + 2.0 * z * u1);
                az += c * (d2 * base + 2.0 * z * u2);
            }
        }
        if ((fl & kOblateness) && !(fl & kShape) && isEarth) {
            // J2 model in the body frame (J2.h:17-33,63-78), inside the sphere of influence
            const double rr = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
            if (rr <= e.bodySoi[bi]) {
                const double bx = fb[0], by = fb[1], bz = fb[2];
                const double invr = 1.0 / sqrt(bx * bx + by * by + bz * bz);
                const double invr2 = invr * invr;
                const double invr5 = invr2 * invr2 * invr;
                const double base = 1.0 - 5.0 * (bz * bz) * invr2;
                const double c = -1.5 * e.bodyGmConst[bi] * e.bodyJ2[bi] * invr5 * e.bodyRadius[bi] * e.bodyRadius[bi];
                const double aj[3] = {c * bx * base, c * by * base, c * bz * (base + 2.0)};
                double ai[3];
                fromBody(r, aj, ai);
                ax += ai[0];
                ay += ai[1];
                az += ai[2];
            }
        }
        if (fl & kRadiation) {
            const double dp[3] = {pos[0] - rb[0], pos[1] - rb[1], pos[2] - rb[2]};
            const double ird = rsqrt(dp[0] * dp[0] + dp[1] * dp[1] + dp[2] * dp[2]);
            double occ = 1.0;
            if (e.anyOcculter) {
                for (int oj = 0; oj < e.nbodies; ++oj) {
                    if (!(e.bodyFlags[oj] & kOcculting) || oj == e.sunIndex) continue;
                    const double rB[3] = {pos[0] - r.body(oj, 0), pos[1] - r.body(oj, 1), pos[2] - r.body(oj, 2)};
                    occ *= shadowFactor(dp, rB, e.bodyRadius[bi], e.bodyRadius[oj]);
                }
            }
            const double f = occ * ((e.au * e.au * 4.56e-3 * ams) * (ird * ird * ird));
            ax += f * dp[0];
            ay += f * dp[1];
            az += f * dp[2];
        }
        if ((fl & kAtmosphere) && !isEarth && e.nExp > 0 && e.poleSlot[bi] >= 0) {
            // exponential drag in another body's atmosphere (PrivateAccelerations.h:143-204):
            // geodetic height about its polar axis, the air moving with its
            // rotation and its velocity relative to the Earth
            const int k = e.poleSlot[bi];
            const double d[3] = {pos[0] - rb[0], pos[1] - rb[1], pos[2] - rb[2]};
            const double pole[3] = {r.pole(k, 0), r.pole(k, 1), r.pole(k, 2)};
            const double h = geodeticHeight(d, pole, e.bodyRadius[bi], e.atmFlattening);
            int band = 0;
            for (int sgi = 1; sgi < e.nExp; ++sgi) band += e.expSeg[sgi][1] <= h ? 1 : 0;
            if (h <= e.expSeg[band][3]) {
                const double rho = e.expSeg[band][0] * exp(-(h - e.expSeg[band][1]) / e.expSeg[band][2]);
                const double w[3] = {r.poleW(k, 0), r.poleW(k, 1), r.poleW(k, 2)};
                const double vr0 = vel[0] - r.poleV(k, 0) - (w[1] * d[2] - w[2] * d[1]);
                const double vr1 = vel[1] - r.poleV(k, 1) - (w[2] * d[0] - w[0] * d[2]);
                const double vr2 = vel[2] - r.poleV(k, 2) - (w[0] * d[1] - w[1] * d[0]);
                const double f = -0.5 * rho * bc * sqrt(vr0 * vr0 + vr1 * vr1 + vr2 * vr2);
                ax += f * vr0;
                ay += f * vr1;
                az += f * vr2;
            }
        }
        if ((fl & kAtmosphere) && isEarth && !e.hasNrl && e.nExp > 0) {
            // piecewise exponential drag (PrivateAccelerations.h:137-206,
            // PiecewiseExponentialAtmosphere.h:40-90): band = bands above the
            // first whose base h0 <= h; no drag above the band's cut-off
            const double pole[3] = {r.R(6), r.R(7), r.R(8)};  // body z axis in inertial axes
            const double h = geodeticHeight(pos, pole, e.bodyRadius[bi], e.flattening);
            int band = 0;
            for (int sgi = 1; sgi < e.nExp; ++sgi) band += e.expSeg[sgi][1] <= h ? 1 : 0;
            if (h <= e.expSeg[band][3]) {
                const double rho = e.expSeg[band][0] * exp(-(h - e.expSeg[band][1]) / e.expSeg[band][2]);
                const double w[3] = {r.W(0), r.W(1), r.W(2)};
                const double vr0 = vel[0] - (w[1] * pos[2] - w[2] * pos[1]);
                const double vr1 = vel[1] - (w[2] * pos[0] - w[0] * pos[2]);
                const double vr2 = vel[2] - (w[0] * pos[1] - w[1] * pos[0]);
                const double f = -0.5 * rho * bc * sqrt(vr0 * vr0 + vr1 * vr1 + vr2 * vr2);
                ax += f * vr0;
                ay += f * vr1;
                az += f * vr2;
            }
        }
        if ((fl & kAtmosphere) && isEarth && e.hasNrl) {
            const double rho = nrlDensity<L>(e, r.nrlDeferred(), fb);
            const double w[3] = {r.W(0), r.W(1), r.W(2)};
            const double vr0 = vel[0] - (w[1] * pos[2] - w[2] * pos[1]);
            const double vr1 = vel[1] - (w[2] * pos[0] - w[0] * pos[2]);
            const double vr2 = vel[2] - (w[0] * pos[1] - w[1] * pos[0]);
            const double f = -0.5 * rho * bc * sqrt(vr0 * vr0 + vr1 * vr1 + vr2 * vr2);
            ax += f * vr0;
            ay += f * vr1;
            az += f * vr2;
        }
    }
    ax += r.indirect(0);
    ay += r.indirect(1);
    az += r.indirect(2);
    if (e.tidesAlone) {
        double t[3] = {0.0, 0.0, 0.0};
        tideAloneAccel(r, pos, t);
        ax += t[0];
        ay += t[1];
        az += t[2];
    }
    if (e.relativity) {
        const double mu = tidefield::kMuEarth, c = tidefield::kLight;
        const double r0 = 1000.0 * pos[0], r1 = 1000.0 * pos[1], r2 = 1000.0 * pos[2];
        const double v0 = 1000.0 * vel[0], v1 = 1000.0 * vel[1], v2 = 1000.0 * vel[2];
        const double irr = rsqrt(r0 * r0 + r1 * r1 + r2 * r2);
        const double v2n = v0 * v0 + v1 * v1 + v2 * v2;
        const double rv = r0 * v0 + r1 * v1 + r2 * v2;
        const double f = mu * (irr * irr * irr) / (c * c);
        const double g = 4.0 * mu * irr - v2n;
        ax += 1.0e-3 * (f * (g * r0 + 4.0 * rv * v0));
        ay += 1.0e-3 * (f * (g * r1 + 4.0 * rv * v1));
        az += 1.0e-3 * (f * (g * r2 + 4.0 * rv * v2));
    }
    acc[0] = ax;
    acc[1] = ay;
    acc[2] = az;
}

// ---- TMA bulk staging of the coefficient tile --------------------------------------------------
// Stages the tile with bulk copies (32 KB chunks) on one mbarrier and waits
// for them with a bounded poll.  Returns whether the whole CTA saw the copies
// land; on a time-out the CTA reads the tile from global memory instead (the
// copies, should any still be in flight, only write the tile's region of
// shared memory, which the CTA then leaves alone).  `issue` = false arms the
// barrier without any copy (a test of the time-out path: nothing is in
// flight when the wait gives up).
static __device__ __forceinline__ bool stageTile(void* dst, const void* src, int bytes, bool issue, long polls) {
    __shared__ __align__(8) uint64_t bar;
    const uint32_t barAddr = (uint32_t)__cvta_generic_to_shared(&bar);
    const uint32_t dstAddr = (uint32_t)__cvta_generic_to_shared(dst);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(barAddr));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(barAddr), "r"(bytes) : "memory");
        const int chunk = 32768;
        for (int off = 0; issue && off < bytes; off += chunk) {
            const int sz = (bytes - off) < chunk ? (bytes - off) : chunk;
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    dstAddr + off),
                "l"((const char*)src + off), "r"(sz), "r"(barAddr)
                : "memory");
        }
    }
    __syncthreads();
    // bounded wait on phase 0
    uint32_t done = 0;
    for (long it = 0; it < polls && !done; ++it) {
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(barAddr), "r"(0)
            : "memory");
    }
    return __syncthreads_and((int)done) != 0;
}

// ---- the persistent step kernel ----------------------------------------------------------------
// Stage record of a per-object-time batch: 4-point Lagrange weights in the
// batch's record grid (rotation, angular velocity, body positions, tide
// deltas; a 30 s spacing keeps the interpolation error of the rotation below
// 1e-12 relative), read field by field by the force model; the NRLMSISE-00
// time inputs are evaluated exactly at the stage epoch by the drag model
// when it needs them.
static __device__ __forceinline__ RecordInterp recordFromGrid(const StepParams& p, double et) {
    // stencil k0 - 1 .. k0 + 2 around the absolute grid index k0 = floor(et / H);
    // q depends on et alone, so the weights are the same in every batch
    const double u = et / p.gridH;
    const double kf = floor(u);
    int64_t i0 = (int64_t)kf - 1 - p.gridBase;
    i0 = i0 < 0 ? 0 : (i0 > p.gridN - 4 ? p.gridN - 4 : i0);
    const double q = u - kf + 1.0;
    double w[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        double num = 1.0, den = 1.0;
#pragma unroll
        for (int m = 0; m < 4; ++m)
            if (m != j) {
                num *= q - (double)m;
                den *= (double)(j - m);
            }
        w[j] = num / den;
    }
    return RecordInterp{p.gridPairs + i0 * kInterpFields, w[0], w[1], w[2], w[3], et};
}

// MAXT: the thread bound the kernel is compiled for, which sets its register
// budget (the register file is split over the SM's four sub-partitions, so
// 320 or 384 threads leave 168 registers a thread and 256 threads leave 255).
template <int L, typename T, bool SHARED_GRID, bool PAIR, int MAXT>
__global__ void __launch_bounds__(MAXT, 1) propagateKernel(const __grid_constant__ StepParams p) {
    using Tile = typename TileOf<T>::type;
    constexpr int CPL = (6 + L - 1) / L;
    extern __shared__ __align__(128) unsigned char smem[];
    const Tile* tile = (const Tile*)p.tile;
    int kOffset = 0;
    if (!SHARED_GRID && !p.gridPairs) {  // per-object time needs the batch's record grid
        if (threadIdx.x == 0) atomicExch(p.errorFlag, 3);
        return;
    }
    if (p.useSmemTile) {
        const bool test = p.tileWaitTest != 0;
        if (stageTile(smem, p.tile, p.tileBytes, !test, test ? 4096L : (1L << 24)))
            tile = (const Tile*)smem;
        else if (threadIdx.x == 0 && p.tileFallbacks)
            atomicAdd(p.tileFallbacks, 1);  // this CTA reads the tile from global memory
        kOffset = p.tileBytes;
    }
    StageStore<CPL> kst{(double*)(smem + kOffset), (int)blockDim.x};
    const int lane = (int)(threadIdx.x & 31);
    const int j = lane % L;
    const int g = lane / L;
    constexpr int groups = 32 / L;
    const int groupBase = lane - j;
    // Work items are groups of 32/L consecutive objects (in the processing
    // order, i.e. by altitude).  The first wave is assigned statically with
    // consecutive items on different CTAs, so the costly low-altitude groups
    // spread over all SMs instead of landing on the CTAs that start first;
    // later items come from the atomic queue.
    const int64_t nItems = (p.n + groups - 1) / groups;
    const int64_t firstWave = (int64_t)gridDim.x * (blockDim.x / 32);
    auto nextItem = [&]() {
        int64_t next = 0;
        if (lane == 0) next = firstWave + (int64_t)atomicAdd(p.workCounter, 1);
        return __shfl_sync(0xffffffffu, next, 0);
    };
    for (int64_t item = (int64_t)(threadIdx.x / 32) * gridDim.x + blockIdx.x; item < nItems; item = nextItem()) {
        const int64_t base = item * groups;
        const int64_t slot = base + g;
        const bool valid = slot < p.n;
        const int64_t sidx = valid ? slot : p.n - 1;
        const int64_t oi = p.order ? p.order[sidx] : sidx;
        const int64_t stride = p.stride ? p.stride : p.n;
        double y[CPL];
#pragma unroll
        for (int c = 0; c < CPL; ++c) {
            const int d = j + c * L;
            y[c] = d < 6 ? p.state[(int64_t)d * stride + oi] : 0.0;
        }
        const double bc = p.bc[oi], ams = p.ams[oi];
        double cur = 0.0, dtv = 0.0, endv = 0.0, stepv = 0.0;
        bool done = false;
        if (!SHARED_GRID) {
            cur = p.cur[oi];
            dtv = p.dt[oi];
            endv = p.end[oi];
            stepv = p.step[oi];
            done = !valid || !(dtv > 0.0);  // a resident batch keeps objects that have reached their end
        }
        const int64_t nsteps = SHARED_GRID ? (int64_t)p.nsteps : p.maxSteps;
        for (int64_t kstep = 0; kstep < nsteps; ++kstep) {
            if (!SHARED_GRID) {
                if (!__any_sync(0xffffffffu, !done)) break;
            }
            const double t0 = SHARED_GRID ? p.stepT0[kstep] : cur;
            const double dt = SHARED_GRID ? p.stepDt[kstep] : dtv;
            // one copy of the force model: the stage loop is not unrolled
#pragma unroll 1
            for (int s = 0; s < 13; ++s) {
                double ys[CPL];
                combine<CPL>(s, y, kst, dt, ys);
                double st[6];
#pragma unroll
                for (int d = 0; d < 6; ++d) {
                    const double own = ys[(d / L) < CPL ? (d / L) : 0];
                    st[d] = (L == 1) ? ys[d < CPL ? d : 0] : __shfl_sync(0xffffffffu, own, groupBase + d % L);
                }
                double acc[3];
                if (SHARED_GRID) {
                    const RecordRef rec{p.records + kstep * 13 + s};
                    accelerations<L, T, PAIR>(p, tile, rec, st, st + 3, bc, ams, acc);
                } else {
                    const double ts = s == 0 ? t0 : t0 + dt * rkC(s - 1);
                    const RecordInterp rec = recordFromGrid(p, ts);
                    accelerations<L, T, PAIR>(p, tile, rec, st, st + 3, bc, ams, acc);
                }
#pragma unroll
                for (int c = 0; c < CPL; ++c) {
                    const int d = j + c * L;
                    kst.at(s, c) = d < 3 ? st[d + 3] : (d < 6 ? acc[d - 3] : 0.0);
                }
            }
            finalUpdate<CPL>(y, kst, dt, SHARED_GRID || !done);
            if (SHARED_GRID && p.traj && (kstep + 1) % p.trajEvery == 0 && valid
                && (kstep + 1) / p.trajEvery <= p.trajRecords) {
                double* rec = p.traj + (int64_t)((kstep + 1) / p.trajEvery - 1) * 6 * p.n;
#pragma unroll
                for (int c = 0; c < CPL; ++c) {
                    const int d = j + c * L;
                    if (d < 6) rec[(int64_t)d * p.n + oi] = y[c];
                }
            }
            if (!SHARED_GRID && !done) {
                // FixedStep.h:30-37
                cur += dtv;
                const double rem = endv - cur;
                done = rem <= 0;
                dtv = done ? 0.0 : fmin(stepv, rem);
            }
        }
        if (valid) {
#pragma unroll
            for (int c = 0; c < CPL; ++c) {
                const int d = j + c * L;
                if (d < 6) p.state[(int64_t)d * stride + oi] = y[c];
            }
            if (!SHARED_GRID && j == 0) {
                p.cur[oi] = cur;
                p.dt[oi] = dtv;
                p.unfinished[oi] = done ? 0 : 1;
            }
        }
    }
}

}  // namespace phop
