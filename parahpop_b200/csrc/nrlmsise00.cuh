// NRLMSISE-00 empirical atmosphere (Picone, Hedin & Drob 2002), total mass
// density path used for drag.
//
// This is a restatement of the published model in the form the reference
// evaluates it: gtd7d with every switch on except switch 9 = -1 (3-hour ap
// history), fed by ``evaluateNrlmsise00HostDensity``
// (src/common/engine/paraHPOP/model/environment/atmosphere/Nrlmsise00.cu:270-327;
// model equations detail/Nrlmsise00Model.inl: tselec :76, glatf :103, ccor :116,
// ccor2 :138, scalh :165, dnet :180, splini :218, splint :256, spline :289,
// densm :331, densu :452, g0/sumex/sg0 :578-628, globe7 :686, glob7s :879,
// gtd7 :959, gtd7d :1085, gts7 :1185).
//
// Differences in form only (results identical):
//  * the per-evaluation model state (the C release's file-scope globals) is a
//    struct member, so one thread evaluates one object with no shared state;
//  * coefficient tables are never written (the C release clamps p[24] and
//    sets p[99] in place; here those are local values), so they can live in
//    constant memory;
//  * only the switch pattern the propagator uses is compiled (sw[i] = 1 for
//    i != 9, sw[9] = -1), which removes the untaken branches.
//
// The header compiles as host C++ and as CUDA device code; T is the
// arithmetic type (double for the reference-parity path).
#pragma once
#include <math.h>

#if defined(__CUDACC__)
#define PHOP_HD __host__ __device__ __forceinline__
#else
#define PHOP_HD inline
#endif

namespace phop {
namespace nrl {

// -- coefficient storage ------------------------------------------------------
#if defined(__CUDACC__)
#define PHOP_NRL_TABLE(name, count) __constant__ double dev_##name[count]
#include "tables/nrlmsise00_coeffs.inc"
#undef PHOP_NRL_TABLE
#endif
#define PHOP_NRL_TABLE(name, count) static const double host_##name[count]
#include "tables/nrlmsise00_coeffs.inc"
#undef PHOP_NRL_TABLE

#if defined(__CUDA_ARCH__)
#define NRLT(name) dev_nrl_##name
#else
#define NRLT(name) host_nrl_##name
#endif

// Row accessors for the multi-row blocks (row-major, as published).
#define NRL_PT (NRLT(pt))
#define NRL_PS (NRLT(ps))
#define NRL_PD(i) (NRLT(pd) + 150 * (i))
#define NRL_PDL(i) (NRLT(pdl) + 25 * (i))
#define NRL_PTL(i) (NRLT(ptl) + 100 * (i))
#define NRL_PMA(i) (NRLT(pma) + 100 * (i))
#define NRL_PDM(i, j) (NRLT(pdm)[10 * (i) + (j)])
#define NRL_PTM(i) (NRLT(ptm)[(i)])
#define NRL_PAVGM(i) (NRLT(pavgm)[(i)])

// Inputs the drag path supplies (the C release's nrlmsise_input, minus year).
template <typename T>
struct Input {
    int doy;
    T sec, alt, g_lat, g_long, lst, f107A, f107, ap;
    T ap_a[7];
};

template <typename T>
struct Model {
    // model state carried between the sub-models of one evaluation
    T gsurf, re;
    T dm28;
    T meso_tn1[5], meso_tn2[4], meso_tn3[5];
    T meso_tgn1[2], meso_tgn2[2], meso_tgn3[2];
    T dfa;
    T plg[4][9];
    T ctloc, stloc, c2tloc, s2tloc, s3tloc, c3tloc;
    T apt0;
    bool g0Cached;
    T g0p24, g0p25, g0v[6];

    // ---- small helpers --------------------------------------------------
    PHOP_HD void glatf(T lat) {
        const T dgtr = T(1.74533E-2);
        const T c2 = cos(T(2.0) * dgtr * lat);
        gsurf = T(980.616) * (T(1.0) - T(0.0026373) * c2);
        re = T(2.0) * gsurf / (T(3.085462E-6) + T(2.27E-9) * c2) * T(1.0E-5);
    }

    PHOP_HD static T ccor(T alt, T r, T h1, T zh) {
        T e = (alt - zh) / h1;
        if (e > T(70)) return exp(T(0.0));
        if (e < T(-70)) return exp(r);
        const T ex = exp(e);
        e = r / (T(1.0) + ex);
        return exp(e);
    }

    PHOP_HD static T ccor2(T alt, T r, T h1, T zh, T h2) {
        const T e1 = (alt - zh) / h1;
        const T e2 = (alt - zh) / h2;
        if ((e1 > T(70)) || (e2 > T(70))) return exp(T(0.0));
        if ((e1 < T(-70)) && (e2 < T(-70))) return exp(r);
        const T ex1 = exp(e1);
        const T ex2 = exp(e2);
        return exp(r / (T(1.0) + T(0.5) * (ex1 + ex2)));
    }

    PHOP_HD T scalh(T alt, T xm, T temp) const {
        const T rgas = T(831.4);
        T g = gsurf / (pow((T(1.0) + alt / re), T(2.0)));
        return rgas * temp / (g * xm);
    }

    PHOP_HD static T dnet(T dd, T dm, T zhm, T xmm, T xm) {
        T a = zhm / (xmm - xm);
        if (!((dm > T(0)) && (dd > T(0)))) {
            if ((dd == T(0)) && (dm == T(0))) dd = T(1);
            if (dm == T(0)) return dd;
            if (dd == T(0)) return dm;
        }
        const T ylog = a * log(dm / dd);
        if (ylog < T(-10)) return dd;
        if (ylog > T(10)) return dm;
        return dd * pow((T(1.0) + exp(ylog)), (T(1.0) / a));
    }

    // integral of the cubic spline from xa[0] to x
    PHOP_HD static T splini(const T* xa, const T* ya, const T* y2a, int n, T x) {
        T yi = T(0);
        int klo = 0, khi = 1;
        while ((x > xa[klo]) && (khi < n)) {
            T xx = x;
            if (khi < (n - 1)) xx = (x < xa[khi]) ? x : xa[khi];
            const T h = xa[khi] - xa[klo];
            const T a = (xa[khi] - xx) / h;
            const T b = (xx - xa[klo]) / h;
            const T a2 = a * a;
            const T b2 = b * b;
            yi += ((T(1.0) - a2) * ya[klo] / T(2.0) + b2 * ya[khi] / T(2.0)
                   + ((-(T(1.0) + a2 * a2) / T(4.0) + a2 / T(2.0)) * y2a[klo]
                      + (b2 * b2 / T(4.0) - b2 / T(2.0)) * y2a[khi]) * h * h / T(6.0)) * h;
            klo++;
            khi++;
        }
        return yi;
    }

    PHOP_HD static T splint(const T* xa, const T* ya, const T* y2a, int n, T x) {
        int klo = 0, khi = n - 1;
        while ((khi - klo) > 1) {
            const int k = (khi + klo) / 2;
            if (xa[k] > x) khi = k; else klo = k;
        }
        const T h = xa[khi] - xa[klo];
        const T a = (xa[khi] - x) / h;
        const T b = (x - xa[klo]) / h;
        return a * ya[klo] + b * ya[khi]
            + ((a * a * a - a) * y2a[klo] + (b * b * b - b) * y2a[khi]) * h * h / T(6.0);
    }

    // second derivatives of the natural/clamped cubic spline (n <= 5)
    PHOP_HD static void spline(const T* x, const T* y, int n, T yp1, T ypn, T* y2) {
        T u[5];
        if (yp1 > T(0.99E30)) {
            y2[0] = T(0);
            u[0] = T(0);
        } else {
            y2[0] = T(-0.5);
            u[0] = (T(3.0) / (x[1] - x[0])) * ((y[1] - y[0]) / (x[1] - x[0]) - yp1);
        }
        for (int i = 1; i < (n - 1); i++) {
            const T sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1]);
            const T p = sig * y2[i - 1] + T(2.0);
            y2[i] = (sig - T(1.0)) / p;
            u[i] = (T(6.0) * ((y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1]))
                        / (x[i + 1] - x[i - 1]) - sig * u[i - 1]) / p;
        }
        T qn, un;
        if (ypn > T(0.99E30)) {
            qn = T(0);
            un = T(0);
        } else {
            qn = T(0.5);
            un = (T(3.0) / (x[n - 1] - x[n - 2])) * (ypn - (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]));
        }
        y2[n - 1] = (un - qn * u[n - 2]) / (qn * y2[n - 2] + T(1.0));
        for (int k = n - 2; k >= 0; k--) y2[k] = y2[k] * y2[k + 1] + u[k];
    }

    PHOP_HD T zeta(T zz, T zl) const { return ((zz - zl) * (re + zl) / (re + zz)); }

    // temperature / density profile below 72.5 km (two spline segments)
    PHOP_HD T densm(T alt, T d0, T xm, T* tz, int mn3, const T* zn3, const T* tn3, const T* tgn3,
                    int mn2, const T* zn2, const T* tn2, const T* tgn2) const {
        T xs[5], ys[5], y2out[5];
        const T rgas = T(831.4);
        T densm_tmp = d0;
        if (alt > zn2[0]) return (xm == T(0.0)) ? *tz : d0;
        // stratosphere / mesosphere temperature
        T z = (alt > zn2[mn2 - 1]) ? alt : zn2[mn2 - 1];
        int mn = mn2;
        T z1 = zn2[0], z2 = zn2[mn - 1];
        T t1 = tn2[0], t2 = tn2[mn - 1];
        T zg = zeta(z, z1);
        T zgdif = zeta(z2, z1);
        for (int k = 0; k < mn; k++) {
            xs[k] = zeta(zn2[k], z1) / zgdif;
            ys[k] = T(1.0) / tn2[k];
        }
        T yd1 = -tgn2[0] / (t1 * t1) * zgdif;
        T yd2 = -tgn2[1] / (t2 * t2) * zgdif * (pow(((re + z2) / (re + z1)), T(2.0)));
        spline(xs, ys, mn, yd1, yd2, y2out);
        T x = zg / zgdif;
        T y = splint(xs, ys, y2out, mn, x);
        *tz = T(1.0) / y;
        if (xm != T(0.0)) {
            const T glb = gsurf / (pow((T(1.0) + z1 / re), T(2.0)));
            const T gamm = xm * glb * zgdif / rgas;
            const T yi = splini(xs, ys, y2out, mn, x);
            T expl = gamm * yi;
            if (expl > T(50.0)) expl = T(50.0);
            densm_tmp = densm_tmp * (t1 / *tz) * exp(-expl);
        }
        if (alt > zn3[0]) return (xm == T(0.0)) ? *tz : densm_tmp;
        // troposphere / stratosphere temperature
        z = alt;
        mn = mn3;
        z1 = zn3[0];
        z2 = zn3[mn - 1];
        t1 = tn3[0];
        t2 = tn3[mn - 1];
        zg = zeta(z, z1);
        zgdif = zeta(z2, z1);
        for (int k = 0; k < mn; k++) {
            xs[k] = zeta(zn3[k], z1) / zgdif;
            ys[k] = T(1.0) / tn3[k];
        }
        yd1 = -tgn3[0] / (t1 * t1) * zgdif;
        yd2 = -tgn3[1] / (t2 * t2) * zgdif * (pow(((re + z2) / (re + z1)), T(2.0)));
        spline(xs, ys, mn, yd1, yd2, y2out);
        x = zg / zgdif;
        y = splint(xs, ys, y2out, mn, x);
        *tz = T(1.0) / y;
        if (xm != T(0.0)) {
            const T glb = gsurf / (pow((T(1.0) + z1 / re), T(2.0)));
            const T gamm = xm * glb * zgdif / rgas;
            const T yi = splini(xs, ys, y2out, mn, x);
            T expl = gamm * yi;
            if (expl > T(50.0)) expl = T(50.0);
            densm_tmp = densm_tmp * (t1 / *tz) * exp(-expl);
        }
        return (xm == T(0.0)) ? *tz : densm_tmp;
    }

    // Bates temperature profile above ZA and spline below, with the
    // diffusive density.  Writes the ZA node (tn1[0], tgn1[0]) like the C
    // release does.
    PHOP_HD T densu(T alt, T dlb, T tinf, T tlb, T xm, T alpha, T* tz, T zlb, T s2, int mn1, const T* zn1,
                    T* tn1, T* tgn1) const {
        const T rgas = T(831.4);
        T xs[5], ys[5], y2out[5];
        T x = T(0), z1 = T(0), t1 = T(0), zgdif = T(0);
        int mn = 0;
        const T za = zn1[0];
        T z = (alt > za) ? alt : za;
        const T zg2 = zeta(z, zlb);
        const T tt = tinf - (tinf - tlb) * exp(-s2 * zg2);
        const T ta = tt;
        *tz = tt;
        T densu_temp = *tz;
        if (alt < za) {
            const T dta = (tinf - ta) * s2 * pow(((re + zlb) / (re + za)), T(2.0));
            tgn1[0] = dta;
            tn1[0] = ta;
            z = (alt > zn1[mn1 - 1]) ? alt : zn1[mn1 - 1];
            mn = mn1;
            z1 = zn1[0];
            const T z2 = zn1[mn - 1];
            t1 = tn1[0];
            const T t2 = tn1[mn - 1];
            const T zg = zeta(z, z1);
            zgdif = zeta(z2, z1);
            for (int k = 0; k < mn; k++) {
                xs[k] = zeta(zn1[k], z1) / zgdif;
                ys[k] = T(1.0) / tn1[k];
            }
            const T yd1 = -tgn1[0] / (t1 * t1) * zgdif;
            const T yd2 = -tgn1[1] / (t2 * t2) * zgdif * pow(((re + z2) / (re + z1)), T(2.0));
            spline(xs, ys, mn, yd1, yd2, y2out);
            x = zg / zgdif;
            const T y = splint(xs, ys, y2out, mn, x);
            *tz = T(1.0) / y;
            densu_temp = *tz;
        }
        if (xm == T(0)) return densu_temp;
        // density above ZA
        T glb = gsurf / pow((T(1.0) + zlb / re), T(2.0));
        const T gamma = xm * glb / (s2 * rgas * tinf);
        T expl = exp(-s2 * gamma * zg2);
        if (expl > T(50.0)) expl = T(50.0);
        if (tt <= T(0)) expl = T(50.0);
        const T densa = dlb * pow((tlb / tt), ((T(1.0) + alpha + gamma))) * expl;
        densu_temp = densa;
        if (alt >= za) return densu_temp;
        // density below ZA
        glb = gsurf / pow((T(1.0) + z1 / re), T(2.0));
        const T gamm = xm * glb * zgdif / rgas;
        const T yi = splini(xs, ys, y2out, mn, x);
        expl = gamm * yi;
        if (expl > T(50.0)) expl = T(50.0);
        if (*tz <= T(0)) expl = T(50.0);
        return densu_temp * pow((t1 / *tz), (T(1.0) + alpha)) * exp(-expl);
    }

    // 3-hour magnetic activity functions (Eq. A24a-d)
    PHOP_HD static T g0(T a, const double* p) {
        const T p24 = (T(p[24]) < T(1.0E-4)) ? T(1.0E-4) : sqrt(T(p[24]) * T(p[24]));
        return (a - T(4.0) + (T(p[25]) - T(1.0)) * (a - T(4.0) + (exp(-p24 * (a - T(4.0))) - T(1.0)) / p24));
    }
    PHOP_HD static T sumex(T ex) {
        return (T(1.0) + (T(1.0) - pow(ex, T(19.0))) / (T(1.0) - ex) * pow(ex, T(0.5)));
    }
    PHOP_HD T sg0(T ex, const double* p, const T* ap) {
        T g[6];
        if (g0Cached && T(p[24]) == g0p24 && T(p[25]) == g0p25) {
            for (int k = 0; k < 6; ++k) g[k] = g0v[k];
        } else {
            for (int k = 0; k < 6; ++k) g[k] = g0(ap[k + 1], p);
            if (!g0Cached) {
                g0p24 = T(p[24]);
                g0p25 = T(p[25]);
                for (int k = 0; k < 6; ++k) g0v[k] = g[k];
                g0Cached = true;
            }
        }
        return (g[0] + (g[1] * ex + g[2] * ex * ex + g[3] * pow(ex, T(3.0))
                        + (g[4] * pow(ex, T(4.0)) + g[5] * pow(ex, T(12.0))) * (T(1.0) - pow(ex, T(8.0))) / (T(1.0) - ex)))
            / sumex(ex);
    }

    // latitude Legendre basis and local-time harmonics for one evaluation
    PHOP_HD void prepareBasis(const Input<T>& in) {
        const T dgtr = T(1.74533E-2);
        const T hr = T(0.2618);
        const T tloc = in.lst;
        const T c = sin(in.g_lat * dgtr);
        const T s = cos(in.g_lat * dgtr);
        const T c2 = c * c;
        const T c4 = c2 * c2;
        const T s2 = s * s;
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
        stloc = sin(hr * tloc);
        ctloc = cos(hr * tloc);
        s2tloc = sin(T(2.0) * hr * tloc);
        c2tloc = cos(T(2.0) * hr * tloc);
        s3tloc = sin(T(3.0) * hr * tloc);
        c3tloc = cos(T(3.0) * hr * tloc);
    }

    // G(L) of the upper thermosphere (switch 9 = -1 branch)
    PHOP_HD T globe7(const double* p, const Input<T>& in) {
        T t[14];
        const T sr = T(7.2722E-5);
        const T dgtr = T(1.74533E-2);
        const T dr = T(1.72142E-2);
        const T hr = T(0.2618);
        const T tloc = in.lst;
        const T doy = T(in.doy);
        for (int j = 0; j < 14; j++) t[j] = T(0);
        const T cd32 = cos(dr * (doy - T(p[31])));
        const T cd18 = cos(T(2.0) * dr * (doy - T(p[17])));
        const T cd14 = cos(dr * (doy - T(p[13])));
        const T cd39 = cos(T(2.0) * dr * (doy - T(p[38])));
        // F10.7 effect
        const T df = in.f107 - in.f107A;
        dfa = in.f107A - T(150.0);
        t[0] = T(p[19]) * df * (T(1.0) + T(p[59]) * dfa) + T(p[20]) * df * df + T(p[21]) * dfa
            + T(p[29]) * pow(dfa, T(2.0));
        const T f1 = T(1.0) + (T(p[47]) * dfa + T(p[19]) * df + T(p[20]) * df * df);
        const T f2 = T(1.0) + (T(p[49]) * dfa + T(p[19]) * df + T(p[20]) * df * df);
        // time independent
        t[1] = (T(p[1]) * plg[0][2] + T(p[2]) * plg[0][4] + T(p[22]) * plg[0][6])
            + (T(p[14]) * plg[0][2]) * dfa + T(p[26]) * plg[0][1];
        // symmetrical annual / semiannual, asymmetrical annual / semiannual
        t[2] = T(p[18]) * cd32;
        t[3] = (T(p[15]) + T(p[16]) * plg[0][2]) * cd18;
        t[4] = f1 * (T(p[9]) * plg[0][1] + T(p[10]) * plg[0][3]) * cd14;
        t[5] = T(p[37]) * plg[0][1] * cd39;
        // diurnal
        {
            const T t71 = (T(p[11]) * plg[1][2]) * cd14;
            const T t72 = (T(p[12]) * plg[1][2]) * cd14;
            t[6] = f2 * ((T(p[3]) * plg[1][1] + T(p[4]) * plg[1][3] + T(p[27]) * plg[1][5] + t71) * ctloc
                         + (T(p[6]) * plg[1][1] + T(p[7]) * plg[1][3] + T(p[28]) * plg[1][5] + t72) * stloc);
        }
        // semidiurnal
        {
            const T t81 = (T(p[23]) * plg[2][3] + T(p[35]) * plg[2][5]) * cd14;
            const T t82 = (T(p[33]) * plg[2][3] + T(p[36]) * plg[2][5]) * cd14;
            t[7] = f2 * ((T(p[5]) * plg[2][2] + T(p[41]) * plg[2][4] + t81) * c2tloc
                         + (T(p[8]) * plg[2][2] + T(p[42]) * plg[2][4] + t82) * s2tloc);
        }
        // terdiurnal
        t[13] = f2 * ((T(p[39]) * plg[3][3] + (T(p[93]) * plg[3][4] + T(p[46]) * plg[3][6]) * cd14) * s3tloc
                      + (T(p[40]) * plg[3][3] + (T(p[94]) * plg[3][4] + T(p[48]) * plg[3][6]) * cd14) * c3tloc);
        // magnetic activity from the 3-hour ap history (switch 9 = -1)
        if (p[51] != 0) {
            T exp1 = exp(T(-10800.0) * sqrt(T(p[51]) * T(p[51]))
                         / (T(1.0) + T(p[138]) * (T(45.0) - sqrt(in.g_lat * in.g_lat))));
            if (exp1 > T(0.99999)) exp1 = T(0.99999);
            apt0 = sg0(exp1, p, in.ap_a);
            t[8] = apt0 * (T(p[50]) + T(p[96]) * plg[0][2] + T(p[54]) * plg[0][4]
                           + (T(p[125]) * plg[0][1] + T(p[126]) * plg[0][3] + T(p[127]) * plg[0][5]) * cd14
                           + (T(p[128]) * plg[1][1] + T(p[129]) * plg[1][3] + T(p[130]) * plg[1][5])
                               * cos(hr * (tloc - T(p[131]))));
        }
        if (in.g_long > T(-1000.0)) {
            // longitudinal
            t[10] = (T(1.0) + T(p[80]) * dfa)
                * ((T(p[64]) * plg[1][2] + T(p[65]) * plg[1][4] + T(p[66]) * plg[1][6] + T(p[103]) * plg[1][1]
                    + T(p[104]) * plg[1][3] + T(p[105]) * plg[1][5]
                    + (T(p[109]) * plg[1][1] + T(p[110]) * plg[1][3] + T(p[111]) * plg[1][5]) * cd14)
                       * cos(dgtr * in.g_long)
                   + (T(p[90]) * plg[1][2] + T(p[91]) * plg[1][4] + T(p[92]) * plg[1][6] + T(p[106]) * plg[1][1]
                      + T(p[107]) * plg[1][3] + T(p[108]) * plg[1][5]
                      + (T(p[112]) * plg[1][1] + T(p[113]) * plg[1][3] + T(p[114]) * plg[1][5]) * cd14)
                       * sin(dgtr * in.g_long));
            // ut and mixed ut / longitude
            t[11] = (T(1.0) + T(p[95]) * plg[0][1]) * (T(1.0) + T(p[81]) * dfa)
                * (T(1.0) + T(p[119]) * plg[0][1] * cd14)
                * ((T(p[68]) * plg[0][1] + T(p[69]) * plg[0][3] + T(p[70]) * plg[0][5])
                   * cos(sr * (in.sec - T(p[71]))));
            t[11] += (T(p[76]) * plg[2][3] + T(p[77]) * plg[2][5] + T(p[78]) * plg[2][7])
                * cos(sr * (in.sec - T(p[79])) + T(2.0) * dgtr * in.g_long) * (T(1.0) + T(p[137]) * dfa);
            // ut / longitude magnetic activity
            if (p[51] != 0) {
                t[12] = apt0 * (T(1.) + T(p[132]) * plg[0][1])
                        * ((T(p[52]) * plg[1][2] + T(p[98]) * plg[1][4] + T(p[67]) * plg[1][6])
                           * cos(dgtr * (in.g_long - T(p[97]))))
                    + apt0 * (T(p[133]) * plg[1][1] + T(p[134]) * plg[1][3] + T(p[135]) * plg[1][5]) * cd14
                        * cos(dgtr * (in.g_long - T(p[136])))
                    + apt0 * (T(p[55]) * plg[0][1] + T(p[56]) * plg[0][3] + T(p[57]) * plg[0][5])
                        * cos(sr * (in.sec - T(p[58])));
            }
        }
        // switches 1..14 all enter with |sw| = 1
        T tinf = T(p[30]);
        for (int i = 0; i < 14; i++) tinf = tinf + t[i];
        return tinf;
    }

    // G(L) of the lower atmosphere
    PHOP_HD T glob7s(const double* p, const Input<T>& in) const {
        const T pset = T(2.0);
        const T parameterSet = (p[99] == 0.0) ? pset : T(p[99]);
        if (parameterSet != pset) return T(-1);
        T t[14];
        const T dr = T(1.72142E-2);
        const T dgtr = T(1.74533E-2);
        const T doy = T(in.doy);
        for (int j = 0; j < 14; j++) t[j] = T(0.0);
        const T cd32 = cos(dr * (doy - T(p[31])));
        const T cd18 = cos(T(2.0) * dr * (doy - T(p[17])));
        const T cd14 = cos(dr * (doy - T(p[13])));
        const T cd39 = cos(T(2.0) * dr * (doy - T(p[38])));
        t[0] = T(p[21]) * dfa;
        t[1] = T(p[1]) * plg[0][2] + T(p[2]) * plg[0][4] + T(p[22]) * plg[0][6] + T(p[26]) * plg[0][1]
            + T(p[14]) * plg[0][3] + T(p[59]) * plg[0][5];
        t[2] = (T(p[18]) + T(p[47]) * plg[0][2] + T(p[29]) * plg[0][4]) * cd32;
        t[3] = (T(p[15]) + T(p[16]) * plg[0][2] + T(p[30]) * plg[0][4]) * cd18;
        t[4] = (T(p[9]) * plg[0][1] + T(p[10]) * plg[0][3] + T(p[20]) * plg[0][5]) * cd14;
        t[5] = (T(p[37]) * plg[0][1]) * cd39;
        {
            const T t71 = T(p[11]) * plg[1][2] * cd14;
            const T t72 = T(p[12]) * plg[1][2] * cd14;
            t[6] = ((T(p[3]) * plg[1][1] + T(p[4]) * plg[1][3] + t71) * ctloc
                    + (T(p[6]) * plg[1][1] + T(p[7]) * plg[1][3] + t72) * stloc);
        }
        {
            const T t81 = (T(p[23]) * plg[2][3] + T(p[35]) * plg[2][5]) * cd14;
            const T t82 = (T(p[33]) * plg[2][3] + T(p[36]) * plg[2][5]) * cd14;
            t[7] = ((T(p[5]) * plg[2][2] + T(p[41]) * plg[2][4] + t81) * c2tloc
                    + (T(p[8]) * plg[2][2] + T(p[42]) * plg[2][4] + t82) * s2tloc);
        }
        t[13] = T(p[39]) * plg[3][3] * s3tloc + T(p[40]) * plg[3][3] * c3tloc;
        t[8] = (T(p[50]) * apt0 + T(p[96]) * plg[0][2] * apt0);
        if (in.g_long > T(-1000.0)) {
            t[10] = (T(1.0)
                     + plg[0][1] * (T(p[80]) * cos(dr * (doy - T(p[81]))) + T(p[85]) * cos(T(2.0) * dr * (doy - T(p[86]))))
                     + T(p[83]) * cos(dr * (doy - T(p[84]))) + T(p[87]) * cos(T(2.0) * dr * (doy - T(p[88]))))
                * ((T(p[64]) * plg[1][2] + T(p[65]) * plg[1][4] + T(p[66]) * plg[1][6] + T(p[74]) * plg[1][1]
                    + T(p[75]) * plg[1][3] + T(p[76]) * plg[1][5]) * cos(dgtr * in.g_long)
                   + (T(p[90]) * plg[1][2] + T(p[91]) * plg[1][4] + T(p[92]) * plg[1][6] + T(p[77]) * plg[1][1]
                      + T(p[78]) * plg[1][3] + T(p[79]) * plg[1][5]) * sin(dgtr * in.g_long));
        }
        T tt = T(0);
        for (int i = 0; i < 14; i++) tt += t[i];
        return tt;
    }

    // thermospheric part (alt >= 72.5 km); d[0..8] number densities, t[0..1]
    PHOP_HD void gts7(const Input<T>& in, T* d, T* tout) {
        T zn1[5] = {T(120.0), T(110.0), T(100.0), T(90.0), T(72.5)};
        const int mn1 = 5;
        const T dgtr = T(1.74533E-2);
        const T dr = T(1.72142E-2);
        const T alpha[9] = {T(-0.38), T(0.0), T(0.0), T(0.0), T(0.17), T(0.0), T(-0.38), T(0.0), T(0.0)};
        const T altl[8] = {T(200.0), T(300.0), T(160.0), T(250.0), T(240.0), T(450.0), T(320.0), T(450.0)};
        const T za = T(NRL_PDL(1)[15]);
        zn1[0] = za;
        for (int j = 0; j < 9; j++) d[j] = T(0);
        g0Cached = false;
        prepareBasis(in);
        const T z = in.alt;
        T tinf;
        if (z > zn1[0])
            tinf = T(NRL_PTM(0)) * T(NRL_PT[0]) * (T(1.0) + globe7(NRL_PT, in));
        else
            tinf = T(NRL_PTM(0)) * T(NRL_PT[0]);
        tout[0] = tinf;
        T g0v_;
        if (z > zn1[4])
            g0v_ = T(NRL_PTM(3)) * T(NRL_PS[0]) * (T(1.0) + globe7(NRL_PS, in));
        else
            g0v_ = T(NRL_PTM(3)) * T(NRL_PS[0]);
        const T tlb = T(NRL_PTM(1)) * (T(1.0) + globe7(NRL_PD(3), in)) * T(NRL_PD(3)[0]);
        const T s = g0v_ / (tinf - tlb);
        if (z < T(300.0)) {
            meso_tn1[1] = T(NRL_PTM(6)) * T(NRL_PTL(0)[0]) / (T(1.0) - glob7s(NRL_PTL(0), in));
            meso_tn1[2] = T(NRL_PTM(2)) * T(NRL_PTL(1)[0]) / (T(1.0) - glob7s(NRL_PTL(1), in));
            meso_tn1[3] = T(NRL_PTM(7)) * T(NRL_PTL(2)[0]) / (T(1.0) - glob7s(NRL_PTL(2), in));
            meso_tn1[4] = T(NRL_PTM(4)) * T(NRL_PTL(3)[0]) / (T(1.0) - glob7s(NRL_PTL(3), in));
            meso_tgn1[1] = T(NRL_PTM(8)) * T(NRL_PMA(8)[0]) * (T(1.0) + glob7s(NRL_PMA(8), in)) * meso_tn1[4]
                * meso_tn1[4] / (pow((T(NRL_PTM(4)) * T(NRL_PTL(3)[0])), T(2.0)));
        } else {
            meso_tn1[1] = T(NRL_PTM(6)) * T(NRL_PTL(0)[0]);
            meso_tn1[2] = T(NRL_PTM(2)) * T(NRL_PTL(1)[0]);
            meso_tn1[3] = T(NRL_PTM(7)) * T(NRL_PTL(2)[0]);
            meso_tn1[4] = T(NRL_PTM(4)) * T(NRL_PTL(3)[0]);
            meso_tgn1[1] = T(NRL_PTM(8)) * T(NRL_PMA(8)[0]) * meso_tn1[4] * meso_tn1[4]
                / (pow((T(NRL_PTM(4)) * T(NRL_PTL(3)[0])), T(2.0)));
        }
        const T zlb = T(NRL_PTM(5));
        T tz;
        // N2
        const T g28 = globe7(NRL_PD(2), in);
        const T zhf = T(NRL_PDL(1)[24]) * (T(1.0) + T(NRL_PDL(0)[24]) * sin(dgtr * in.g_lat)
                                                        * cos(dr * (T(in.doy) - T(NRL_PT[13]))));
        tout[0] = tinf;
        const T xmm = T(NRL_PDM(2, 4));
        const T db28 = T(NRL_PDM(2, 0)) * exp(g28) * T(NRL_PD(2)[0]);
        d[2] = densu(z, db28, tinf, tlb, T(28.0), alpha[2], &tout[1], zlb, s, mn1, zn1, meso_tn1, meso_tgn1);
        const T zh28 = T(NRL_PDM(2, 2)) * zhf;
        const T zhm28 = T(NRL_PDM(2, 3)) * T(NRL_PDL(1)[5]);
        const T xmd = T(28.0) - xmm;
        T b28 = T(0.0);
        if (!(z > altl[7] && z >= zn1[0]))
            b28 = densu(zh28, db28, tinf, tlb, xmd, (alpha[2] - T(1.0)), &tz, zlb, s, mn1, zn1, meso_tn1, meso_tgn1);
        if (z <= altl[2]) {
            dm28 = densu(z, b28, tinf, tlb, xmm, alpha[2], &tz, zlb, s, mn1, zn1, meso_tn1, meso_tgn1);
            d[2] = dnet(d[2], dm28, zhm28, xmm, T(28.0));
        }
        // He
        const T g4 = globe7(NRL_PD(0), in);
        const T db04 = T(NRL_PDM(0, 0)) * exp(g4) * T(NRL_PD(0)[0]);
        d[0] = densu(z, db04, tinf, tlb, T(4.), alpha[0], &tout[1], zlb, s, mn1, zn1, meso_tn1, meso_tgn1);
        if (z < altl[0]) {
            const T zh04 = T(NRL_PDM(0, 2));
            const T b04 = densu(zh04, db04, tinf, tlb, T(4.) - xmm, alpha[0] - T(1.), &tout[1], zlb, s, mn1, zn1,
                                meso_tn1, meso_tgn1);
            const T dm04 = densu(z, b04, tinf, tlb, xmm, T(0.), &tout[1], zlb, s, mn1, zn1, meso_tn1, meso_tgn1);
            d[0] = dnet(d[0], dm04, zhm28, xmm, T(4.));
            const T rl = log(b28 * T(NRL_PDM(0, 1)) / b04);
            const T zc04 = T(NRL_PDM(0, 4)) * T(NRL_PDL(1)[0]);
            const T hc04 = T(NRL_PDM(0, 5)) * T(NRL_PDL(1)[1]);
            d[0] = d[0] * ccor(z, rl, hc04, zc04);
        }
        // O
        const T g16 = globe7(NRL_PD(1), in);
        const T db16 = T(NRL_PDM(1, 0)) * exp(g16) * T(NRL_PD(1)[0]);
        d[1] = densu(z, db16, tinf, tlb, T(16.), alpha[1], &tout[1], zlb, s, mn1, zn1, meso_tn1, meso_tgn1);
        if (z <= altl[1]) {
            const T zh16 = T(NRL_PDM(1, 2));
            const T b16 = densu(zh16, db16, tinf, tlb, T(16.0) - xmm, (alpha[1] - T(1.0)), &tout[1], zlb, s, mn1,
                                zn1, meso_tn1, meso_tgn1);
            const T dm16 = densu(z, b16, tinf, tlb, xmm, T(0.), &tout[1], zlb, s, mn1, zn1, meso_tn1, meso_tgn1);
            d[1] = dnet(d[1], dm16, zhm28, xmm, T(16.));
            const T rl = T(NRL_PDM(1, 1)) * T(NRL_PDL(1)[16]) * (T(1.0) + T(NRL_PDL(0)[23]) * (in.f107A - T(150.0)));
            const T hc16 = T(NRL_PDM(1, 5)) * T(NRL_PDL(1)[3]);
            const T zc16 = T(NRL_PDM(1, 4)) * T(NRL_PDL(1)[2]);
            const T hc216 = T(NRL_PDM(1, 5)) * T(NRL_PDL(1)[4]);
            d[1] = d[1] * ccor2(z, rl, hc16, zc16, hc216);
            const T hcc16 = T(NRL_PDM(1, 7)) * T(NRL_PDL(1)[13]);
            const T zcc16 = T(NRL_PDM(1, 6)) * T(NRL_PDL(1)[12]);
            const T rc16 = T(NRL_PDM(1, 3)) * T(NRL_PDL(1)[14]);
            d[1] = d[1] * ccor(z, rc16, hcc16, zcc16);
        }
        // O2
        const T g32 = globe7(NRL_PD(4), in);
        const T db32 = T(NRL_PDM(3, 0)) * exp(g32) * T(NRL_PD(4)[0]);
        d[3] = densu(z, db32, tinf, tlb, T(32.), alpha[3], &tout[1], zlb, s, mn1, zn1, meso_tn1, meso_tgn1);
        {
            if (z <= altl[3]) {
                const T zh32 = T(NRL_PDM(3, 2));
                const T b32 = densu(zh32, db32, tinf, tlb, T(32.) - xmm, alpha[3] - T(1.), &tout[1], zlb, s, mn1,
                                    zn1, meso_tn1, meso_tgn1);
                const T dm32 = densu(z, b32, tinf, tlb, xmm, T(0.), &tout[1], zlb, s, mn1, zn1, meso_tn1, meso_tgn1);
                d[3] = dnet(d[3], dm32, zhm28, xmm, T(32.));
                const T rl = log(b28 * T(NRL_PDM(3, 1)) / b32);
                const T hc32 = T(NRL_PDM(3, 5)) * T(NRL_PDL(1)[7]);
                const T zc32 = T(NRL_PDM(3, 4)) * T(NRL_PDL(1)[6]);
                d[3] = d[3] * ccor(z, rl, hc32, zc32);
            }
            const T hcc32 = T(NRL_PDM(3, 7)) * T(NRL_PDL(1)[22]);
            const T hcc232 = T(NRL_PDM(3, 7)) * T(NRL_PDL(0)[22]);
            const T zcc32 = T(NRL_PDM(3, 6)) * T(NRL_PDL(1)[21]);
            const T rc32 = T(NRL_PDM(3, 3)) * T(NRL_PDL(1)[23]) * (T(1.) + T(NRL_PDL(0)[23]) * (in.f107A - T(150.)));
            d[3] = d[3] * ccor2(z, rc32, hcc32, zcc32, hcc232);
        }
        // Ar
        const T g40 = globe7(NRL_PD(5), in);
        const T db40 = T(NRL_PDM(4, 0)) * exp(g40) * T(NRL_PD(5)[0]);
        d[4] = densu(z, db40, tinf, tlb, T(40.), alpha[4], &tout[1], zlb, s, mn1, zn1, meso_tn1, meso_tgn1);
        if (z <= altl[4]) {
            const T zh40 = T(NRL_PDM(4, 2));
            const T b40 = densu(zh40, db40, tinf, tlb, T(40.) - xmm, alpha[4] - T(1.), &tout[1], zlb, s, mn1, zn1,
                                meso_tn1, meso_tgn1);
            const T dm40 = densu(z, b40, tinf, tlb, xmm, T(0.), &tout[1], zlb, s, mn1, zn1, meso_tn1, meso_tgn1);
            d[4] = dnet(d[4], dm40, zhm28, xmm, T(40.));
            const T rl = log(b28 * T(NRL_PDM(4, 1)) / b40);
            const T hc40 = T(NRL_PDM(4, 5)) * T(NRL_PDL(1)[9]);
            const T zc40 = T(NRL_PDM(4, 4)) * T(NRL_PDL(1)[8]);
            d[4] = d[4] * ccor(z, rl, hc40, zc40);
        }
        // H
        const T g1 = globe7(NRL_PD(6), in);
        const T db01 = T(NRL_PDM(5, 0)) * exp(g1) * T(NRL_PD(6)[0]);
        d[6] = densu(z, db01, tinf, tlb, T(1.), alpha[6], &tout[1], zlb, s, mn1, zn1, meso_tn1, meso_tgn1);
        if (z <= altl[6]) {
            const T zh01 = T(NRL_PDM(5, 2));
            const T b01 = densu(zh01, db01, tinf, tlb, T(1.) - xmm, alpha[6] - T(1.), &tout[1], zlb, s, mn1, zn1,
                                meso_tn1, meso_tgn1);
            const T dm01 = densu(z, b01, tinf, tlb, xmm, T(0.), &tout[1], zlb, s, mn1, zn1, meso_tn1, meso_tgn1);
            d[6] = dnet(d[6], dm01, zhm28, xmm, T(1.));
            const T rl = log(b28 * T(NRL_PDM(5, 1)) * sqrt(T(NRL_PDL(1)[17]) * T(NRL_PDL(1)[17])) / b01);
            const T hc01 = T(NRL_PDM(5, 5)) * T(NRL_PDL(1)[11]);
            const T zc01 = T(NRL_PDM(5, 4)) * T(NRL_PDL(1)[10]);
            d[6] = d[6] * ccor(z, rl, hc01, zc01);
            const T hcc01 = T(NRL_PDM(5, 7)) * T(NRL_PDL(1)[19]);
            const T zcc01 = T(NRL_PDM(5, 6)) * T(NRL_PDL(1)[18]);
            const T rc01 = T(NRL_PDM(5, 3)) * T(NRL_PDL(1)[20]);
            d[6] = d[6] * ccor(z, rc01, hcc01, zcc01);
        }
        // N
        const T g14 = globe7(NRL_PD(7), in);
        const T db14 = T(NRL_PDM(6, 0)) * exp(g14) * T(NRL_PD(7)[0]);
        d[7] = densu(z, db14, tinf, tlb, T(14.), alpha[7], &tout[1], zlb, s, mn1, zn1, meso_tn1, meso_tgn1);
        if (z <= altl[7]) {
            const T zh14 = T(NRL_PDM(6, 2));
            const T b14 = densu(zh14, db14, tinf, tlb, T(14.) - xmm, alpha[7] - T(1.), &tout[1], zlb, s, mn1, zn1,
                                meso_tn1, meso_tgn1);
            const T dm14 = densu(z, b14, tinf, tlb, xmm, T(0.), &tout[1], zlb, s, mn1, zn1, meso_tn1, meso_tgn1);
            d[7] = dnet(d[7], dm14, zhm28, xmm, T(14.));
            const T rl = log(b28 * T(NRL_PDM(6, 1)) * sqrt(T(NRL_PDL(0)[2]) * T(NRL_PDL(0)[2])) / b14);
            const T hc14 = T(NRL_PDM(6, 5)) * T(NRL_PDL(0)[1]);
            const T zc14 = T(NRL_PDM(6, 4)) * T(NRL_PDL(0)[0]);
            d[7] = d[7] * ccor(z, rl, hc14, zc14);
            const T hcc14 = T(NRL_PDM(6, 7)) * T(NRL_PDL(0)[4]);
            const T zcc14 = T(NRL_PDM(6, 6)) * T(NRL_PDL(0)[3]);
            const T rc14 = T(NRL_PDM(6, 3)) * T(NRL_PDL(0)[5]);
            d[7] = d[7] * ccor(z, rc14, hcc14, zcc14);
        }
        // anomalous O
        const T g16h = globe7(NRL_PD(8), in);
        const T db16h = T(NRL_PDM(7, 0)) * exp(g16h) * T(NRL_PD(8)[0]);
        const T tho = T(NRL_PDM(7, 9)) * T(NRL_PDL(0)[6]);
        const T dd = densu(z, db16h, tho, tho, T(16.), alpha[8], &tout[1], zlb, s, mn1, zn1, meso_tn1, meso_tgn1);
        const T zsht = T(NRL_PDM(7, 5));
        const T zmho = T(NRL_PDM(7, 4));
        const T zsho = scalh(zmho, T(16.0), tho);
        d[8] = dd * exp(-zsht / zsho * (exp(-(z - zmho) / zsht) - T(1.)));
        // (the C release's closing temperature-only densu call rewrites the
        // ZA spline node with the value every earlier call already wrote;
        // it does not affect any density and is omitted)
        // switch 0 = 1: SI units (m^-3 number densities)
        for (int i = 0; i < 9; i++) d[i] = d[i] * T(1.0E6);
    }

    // gtd7 followed by the gtd7d total mass density including anomalous O;
    // returns kg/m^3
    PHOP_HD T densityGtd7d(Input<T> in) {
        T d[9], tt[2];
        const T zn3[5] = {T(32.5), T(20.0), T(15.0), T(10.0), T(0.0)};
        const T zn2[4] = {T(72.5), T(55.0), T(45.0), T(32.5)};
        const T zmix = T(62.5);
        glatf(in.g_lat);
        const T xmm = T(NRL_PDM(2, 4));
        const T altIn = in.alt;
        in.alt = (altIn > zn2[0]) ? altIn : zn2[0];
        gts7(in, d, tt);
        in.alt = altIn;
        const T dm28m = dm28 * T(1.0E6);
        if (!(in.alt >= zn2[0])) {
            // lower mesosphere / upper stratosphere nodes
            meso_tgn2[0] = meso_tgn1[1];
            meso_tn2[0] = meso_tn1[4];
            meso_tn2[1] = T(NRL_PMA(0)[0]) * T(NRL_PAVGM(0)) / (T(1.0) - glob7s(NRL_PMA(0), in));
            meso_tn2[2] = T(NRL_PMA(1)[0]) * T(NRL_PAVGM(1)) / (T(1.0) - glob7s(NRL_PMA(1), in));
            meso_tn2[3] = T(NRL_PMA(2)[0]) * T(NRL_PAVGM(2)) / (T(1.0) - glob7s(NRL_PMA(2), in));
            meso_tgn2[1] = T(NRL_PAVGM(8)) * T(NRL_PMA(9)[0]) * (T(1.0) + glob7s(NRL_PMA(9), in)) * meso_tn2[3]
                * meso_tn2[3] / (pow((T(NRL_PMA(2)[0]) * T(NRL_PAVGM(2))), T(2.0)));
            meso_tn3[0] = meso_tn2[3];
            if (in.alt <= zn3[0]) {
                meso_tgn3[0] = meso_tgn2[1];
                meso_tn3[1] = T(NRL_PMA(3)[0]) * T(NRL_PAVGM(3)) / (T(1.0) - glob7s(NRL_PMA(3), in));
                meso_tn3[2] = T(NRL_PMA(4)[0]) * T(NRL_PAVGM(4)) / (T(1.0) - glob7s(NRL_PMA(4), in));
                meso_tn3[3] = T(NRL_PMA(5)[0]) * T(NRL_PAVGM(5)) / (T(1.0) - glob7s(NRL_PMA(5), in));
                meso_tn3[4] = T(NRL_PMA(6)[0]) * T(NRL_PAVGM(6)) / (T(1.0) - glob7s(NRL_PMA(6), in));
                meso_tgn3[1] = T(NRL_PMA(7)[0]) * T(NRL_PAVGM(7)) * (T(1.0) + glob7s(NRL_PMA(7), in)) * meso_tn3[4]
                    * meso_tn3[4] / (pow((T(NRL_PMA(6)[0]) * T(NRL_PAVGM(6))), T(2.0)));
            }
            T dmc = T(0);
            if (in.alt > zmix) dmc = T(1.0) - (zn2[0] - in.alt) / (zn2[0] - zmix);
            const T dz28 = d[2];
            T tz = T(0);
            T dmr = d[2] / dm28m - T(1.0);
            T o[9];
            o[2] = densm(in.alt, dm28m, xmm, &tz, 5, zn3, meso_tn3, meso_tgn3, 4, zn2, meso_tn2, meso_tgn2);
            o[2] = o[2] * (T(1.0) + dmr * dmc);
            dmr = d[0] / (dz28 * T(NRL_PDM(0, 1))) - T(1.0);
            o[0] = o[2] * T(NRL_PDM(0, 1)) * (T(1.0) + dmr * dmc);
            o[1] = T(0);
            o[8] = T(0);
            dmr = d[3] / (dz28 * T(NRL_PDM(3, 1))) - T(1.0);
            o[3] = o[2] * T(NRL_PDM(3, 1)) * (T(1.0) + dmr * dmc);
            dmr = d[4] / (dz28 * T(NRL_PDM(4, 1))) - T(1.0);
            o[4] = o[2] * T(NRL_PDM(4, 1)) * (T(1.0) + dmr * dmc);
            o[6] = T(0);
            o[7] = T(0);
            for (int i = 0; i < 9; ++i) d[i] = (i == 5) ? d[i] : o[i];
        }
        // gtd7d: total mass density including anomalous oxygen, kg/m^3
        T rho = T(1.66E-24) * (T(4.0) * d[0] + T(16.0) * d[1] + T(28.0) * d[2] + T(32.0) * d[3] + T(40.0) * d[4]
                               + d[6] + T(14.0) * d[7] + T(16.0) * d[8]);
        return rho / T(1000);
    }
};

template <typename T>
PHOP_HD T density(const Input<T>& in) {
    Model<T> m;
    m.gsurf = m.re = T(0);
    m.dm28 = T(0);
    for (int k = 0; k < 5; ++k) m.meso_tn1[k] = m.meso_tn3[k] = T(0);
    for (int k = 0; k < 4; ++k) m.meso_tn2[k] = T(0);
    for (int k = 0; k < 2; ++k) m.meso_tgn1[k] = m.meso_tgn2[k] = m.meso_tgn3[k] = T(0);
    m.dfa = T(0);
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 9; ++j) m.plg[i][j] = T(0);
    m.ctloc = m.stloc = m.c2tloc = m.s2tloc = m.s3tloc = m.c3tloc = T(0);
    m.apt0 = T(0);
    m.g0Cached = false;
    m.g0p24 = m.g0p25 = T(0);
    for (int k = 0; k < 6; ++k) m.g0v[k] = T(0);
    return m.densityGtd7d(in);
}

}  // namespace nrl
}  // namespace phop
