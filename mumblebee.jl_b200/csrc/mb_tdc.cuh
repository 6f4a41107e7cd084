// Device kernels of the three-dimensional non-symmetric cones (exponential and power), one thread
// per cone: determinant chains in double-double, the analytic pivoted Hessian factor, third
// derivatives, the Halley shadow solves, the Tunçel/BFGS scaling and the certified log-form line
// search.  Restated from Mumblebee.jl src/IPM/src/cone/tdc/{tdc,exp,pow,utils}.jl (file:line on each
// function).  The two-word log₂/exp₂ that the reference takes from DoubleFloats' tables are computed
// here in double-double from published methods (error-free transforms, power-of-two range reduction,
// log m = 2 atanh((m-1)/(m+1)), reduced Taylor series for exp), relative accuracy ~1e-31.
#pragma once
#include <cstdint>
#include "mb_device.cuh"

#define MB_INF __longlong_as_double(0x7ff0000000000000LL)
#define MB_NAN __longlong_as_double(0x7ff8000000000000LL)
#define MB_DMIN 2.2250738585072014e-308
#define MB_EPS 2.220446049250313e-16

namespace mb {


// ------------------------------------------------------------------ double-double
struct DD { double h, l; };
__device__ __forceinline__ DD dd_fast(double a, double b) { double s = a + b; return {s, b - (s - a)}; }
__device__ __forceinline__ DD dd_twosum(double a, double b) {
    double s = a + b, bb = s - a;
    return {s, (a - (s - bb)) + (b - bb)};
}
__device__ __forceinline__ DD dd_add(DD a, DD b) {
    DD s = dd_twosum(a.h, b.h);
    DD t = dd_twosum(a.l, b.l);
    s.l += t.h;
    s = dd_fast(s.h, s.l);
    s.l += t.l;
    return dd_fast(s.h, s.l);
}
__device__ __forceinline__ DD dd_mul(DD a, DD b) {
    double p = a.h * b.h;
    double e = fma(a.h, b.h, -p);
    e += a.h * b.l + a.l * b.h;
    return dd_fast(p, e);
}
__device__ __forceinline__ DD dd_div(DD a, DD b) {
    double q1 = a.h / b.h;
    DD r = dd_add(a, dd_mul({-q1, 0.0}, b));
    double q2 = r.h / b.h;
    r = dd_add(r, dd_mul({-q2, 0.0}, b));
    double q3 = r.h / b.h;
    DD q = dd_fast(q1, q2);
    return dd_add(q, {q3, 0.0});
}
#define DD_LN2 (DD{0.6931471805599453, 2.3190468138462996e-17})
#define DD_INV_LN2 (DD{1.4426950408889634, 2.0355273740931033e-17})

// natural log of a positive double-double: x = 2^k m, m in [1/sqrt2, sqrt2),
// log m = 2 atanh(t), t = (m-1)/(m+1)
__device__ __forceinline__ DD dd_log(DD x) {
    int k;
    double mh = frexp(x.h, &k);           // x.h = mh 2^k, mh in [0.5, 1)
    DD m = {mh, ldexp(x.l, -k)};
    if (m.h < 0.70710678118654752) { m.h *= 2; m.l *= 2; k -= 1; }
    DD num = dd_add(m, {-1.0, 0.0});           // exact leading part (Sterbenz) + low word
    DD den = dd_add(m, {1.0, 0.0});
    DD t = dd_div(num, den);
    DD t2 = dd_mul(t, t);
    DD sum = {0.0, 0.0};
    for (int j = 49; j >= 1; j -= 2) sum = dd_add(dd_div({1.0, 0.0}, {(double)j, 0.0}), dd_mul(sum, t2));
    DD lm = dd_mul(dd_mul({2.0, 0.0}, t), sum);
    return dd_add(dd_mul({(double)k, 0.0}, DD_LN2), lm);
}
// exp of a double-double r, |r| moderate: r = k ln2 + s, exp(s) by Taylor on s/2^8, squared back
__device__ __forceinline__ DD dd_exp(DD r) {
    if (r.h > 709.78) return {MB_INF, 0.0};
    if (r.h < -745.2) return {0.0, 0.0};
    double kf = nearbyint(r.h * DD_INV_LN2.h);
    DD s = dd_add(r, dd_mul({-kf, 0.0}, DD_LN2));
    s = {ldexp(s.h, -8), ldexp(s.l, -8)};
    DD term = {1.0, 0.0}, sum = {1.0, 0.0};
    for (int j = 1; j <= 14; ++j) {
        term = dd_div(dd_mul(term, s), {(double)j, 0.0});
        sum = dd_add(sum, term);
    }
    for (int j = 0; j < 8; ++j) sum = dd_mul(sum, sum);
    int k = (int)kf;
    return {ldexp(sum.h, k), ldexp(sum.l, k)};
}

// two-word log(x1/x2)  (IPM/src/utils.jl:78-117 twolog2rat / twolograt)
__device__ __forceinline__ DD twolograt(double x1, double x2) {
    DD q = dd_div({x1, 0.0}, {x2, 0.0});
    return dd_log(q);
}
__device__ __forceinline__ DD twolog2rat(double x1, double x2) { return dd_mul(twolograt(x1, x2), DD_INV_LN2); }
__device__ __forceinline__ DD twolog2(double x) { return dd_mul(dd_log({x, 0.0}), DD_INV_LN2); }
// two-word 2^(ah + al)  (IPM/src/utils.jl:120-123 twoexp2)
__device__ __forceinline__ DD twoexp2(DD a) { return dd_exp(dd_mul(a, DD_LN2)); }
// twodiv  (IPM/src/utils.jl:125-129)
__device__ __forceinline__ void twodiv(double ah, double al, double bh, double bl, double& qh, double& ql) {
    double q1 = ah / bh;
    double r = fma(-q1, bh, ah) + al - q1 * bl;
    DD s = dd_twosum(q1, r / bh);
    qh = s.h; ql = s.l;
}

// ------------------------------------------------------------------ cache slots (tdc.jl:142-163)
// L[0..8] (3x3 column-major), sd[9..11], seed[12], d1..d4[13..16], h0p[17], h0d[18]
enum { TD_L = 0, TD_SD = 9, TD_SEED = 12, TD_D1 = 13, TD_D2 = 14, TD_D3 = 15, TD_D4 = 16, TD_H0P = 17, TD_H0D = 18 };

__device__ __forceinline__ double tdot3(const double* x, const double* y) {   // dotstatic (cone/utils.jl:21-31)
    double s = 0;
    for (int i = 0; i < 3; ++i) s = fma(x[i], y[i], s);
    return s;
}
__device__ __forceinline__ double tcdot3(const double* p, const double* d) {  // cdotstatic (IPM/src/utils.jl:55-70)
    double s = 0, c = 0;
    for (int i = 0; i < 3; ++i) {
        double pr = p[i] * d[i], e = fma(p[i], d[i], -pr);
        DD t = dd_twosum(s, pr);
        s = t.h; c += e + t.l;
    }
    return s + c;
}

// ------------------------------------------------------------------ exponential cone (exp.jl)
__device__ __forceinline__ void expdet(double x1, double x2, double x3, double& psi, double& ipsi, double& lr, double& lrm1) {
    DD l = twolograt(x1, x2);                                   // exp.jl:44-59
    DD m = dd_twosum(l.h, -1.0);
    lrm1 = m.h + (m.l + l.l);
    double ph = l.h * x2, pe = fma(l.h, x2, -ph);
    pe = fma(l.l, x2, pe);
    DD s = dd_twosum(ph, -x3);
    DD ps = dd_twosum(s.h, s.l + pe);
    double ih, il;
    twodiv(1.0, 0.0, ps.h, ps.l, ih, il);
    psi = ps.h + ps.l; ipsi = ih + il; lr = l.h + l.l;
}

__device__ double exp_dualgrad(double* sp, double seed, const double* d, double& h0) {  // exp.jl:224-370
    const double fmin = MB_DMIN, inf = MB_INF;
    const double eps = MB_EPS;
    double d1 = d[0], d2 = d[1], d3 = d[2];
    if (d3 == 0) {
        double p2 = 1.0 / d2, s = d2 / d1;
        sp[0] = s * p2; sp[1] = p2; sp[2] = -inf;
        h0 = (d1 >= 0 && d2 >= 0) ? inf : -inf;
        return p2;
    }
    double md3 = -d3;
    double rat = md3 / d1;
    double lr = (fmin <= rat && rat < inf) ? log(rat) : log(md3) - log(d1);
    double w = d2 / md3;
    double R = w - (lr - 1.0);
    if (!(R > 0)) R = fmin;
    double lo = R / 2, hi = R;
    double v = 1.0 / (fmax(seed, fmin) * md3);
    if (!(lo < v && v < hi)) {
        v = (R <= 2) ? R / 2 + R * R / 16 : R - log(R);
        if (!(lo < v && v < hi)) v = 0.7 * R;
    }
    for (int it = 0; it < 60; ++it) {
        double fv = v + log1p(v) - R;
        double fp = 1.0 + 1.0 / (1.0 + v);
        if (fv < 0) lo = v;
        else if (fv > 0) hi = v;
        else break;
        double fpp = -(fp - 1.0) * (fp - 1.0);
        double vn = v - 2 * fv * fp / (2 * fp * fp - fv * fpp);
        if (!(lo < vn && vn < hi)) {
            if (vn == lo || vn == hi) { v = vn; break; }
            vn = (lo + hi) / 2;
        }
        bool conv = fabs(vn - v) < 4 * eps * fabs(vn);
        v = vn;
        if (conv) break;
    }
    double q = md3 * v, p2 = 1.0 / q;
    double s = md3 * (v + 1.0) / d1;
    if (!(0 < s && s < inf)) s = exp(lr + log1p(v));
    sp[0] = s * p2; sp[1] = p2; sp[2] = p2 * log(s) + 1.0 / d3;
    h0 = 1.0 - lr + w;
    return p2;
}

__device__ __forceinline__ void exp_jetprim(double tau, const double* p, const double* Dp, double& h, double& hp, double& hpp) {
    const double fmin = MB_DMIN, inf = MB_INF;
    const double nan = MB_NAN;
    double x1 = fma(tau, Dp[0], p[0]), x2 = fma(tau, Dp[1], p[1]), x3 = fma(tau, Dp[2], p[2]);
    if (x1 > 0 && x2 > 0) {                                     // exp.jl:441-471
        double q = x1 / x2;
        double s = (fmin <= q && q < inf) ? log(q) : log(x1) - log(x2);
        double w = x3 / x2;
        h = s - w;
        double wp = (Dp[2] - w * Dp[1]) / x2;
        hp = Dp[0] / x1 - Dp[1] / x2 - wp;
        hpp = -(Dp[0] / x1) * (Dp[0] / x1) + (Dp[1] / x2) * (Dp[1] / x2) + 2 * wp * Dp[1] / x2;
        return;
    } else if (x1 >= 0 && x2 == 0) {
        h = x3 <= 0 ? inf : -inf; hp = nan; hpp = nan; return;
    }
    h = -inf; hp = nan; hpp = nan;
}

__device__ __forceinline__ void exp_jetdual(double tau, const double* d, const double* Dd, double& h, double& hp, double& hpp) {
    const double inf = MB_INF, nan = MB_NAN;
    double z1 = fma(tau, Dd[0], d[0]), z2 = fma(tau, Dd[1], d[1]), z3 = fma(tau, Dd[2], d[2]);
    if (z1 > 0 && z3 < 0) {                                     // exp.jl:481-503
        double r = z2 / z3;
        h = 1.0 + log(z1) - r - log(-z3);
        double rp = (Dd[1] - r * Dd[2]) / z3;
        hp = Dd[0] / z1 - rp - Dd[2] / z3;
        hpp = -(Dd[0] / z1) * (Dd[0] / z1) + 2 * rp * Dd[2] / z3 + (Dd[2] / z3) * (Dd[2] / z3);
        return;
    } else if (z1 >= 0 && z2 >= 0 && z3 == 0) {
        h = inf; hp = nan; hpp = nan; return;
    }
    h = -inf; hp = nan; hpp = nan;
}

// ------------------------------------------------------------------ power cone (pow.jl)
__device__ __forceinline__ void powdet(double x1, double x2, double x3, double al, double& P, double& rho, double& invdet) {
    double a = 2 * al;                                          // pow.jl:53-71
    DD r = twolog2rat(x1, x2);
    DD g = twolog2(x2);
    DD L2 = dd_add(dd_mul({a, 0.0}, r), {2 * g.h, 2 * g.l});
    DD Pd = twoexp2(L2);
    double qh = x3 * x3, ql = fma(x3, x3, -qh);
    DD f = dd_twosum(Pd.h, -qh);
    DD dt = dd_twosum(f.h, f.l + (Pd.l - ql));
    double ih, il;
    twodiv(1.0, 0.0, dt.h, dt.l, ih, il);
    double rh = Pd.h * ih, re = fma(Pd.h, ih, -rh);
    re = fma(Pd.h, il, fma(Pd.l, ih, re));
    DD rr = dd_twosum(rh, re);
    P = Pd.h + Pd.l; rho = rr.h + rr.l; invdet = ih + il;
}

__device__ double pow_dualgrad(double* sp, double seed, const double* d, double al, double& h0) {  // pow.jl:269-448
    const double fmin = MB_DMIN, inf = MB_INF;
    const double eps = MB_EPS;
    double d1 = d[0], d2 = d[1], d3 = d[2];
    double a = 2 * al, b = 2 - 2 * al;
    if (d3 == 0) {
        sp[0] = (a + 1 - al) / d1; sp[1] = (b + al) / d2; sp[2] = 0.0;
        h0 = inf;
        return 1.0;
    }
    double k1 = (1 - al) / a, k2 = al / b, t1 = a / d1, t2 = b / d2;
    double z1 = (d3 / 2) * t2, z1s = z1 * z1, z2 = t1 / t2, z2a = pow(z2, a), W0 = z1s * z2a;
    bool normal = fmin <= z1s && z1s < inf && fmin <= z2 && z2 < inf && fmin <= z2a && z2a < inf && fmin <= W0 && W0 < inf;
    double lW0;
    if (!normal) {
        lW0 = 2 * log(fabs(d3)) - log(4.0) + a * (log(a) - log(d1)) + b * (log(b) - log(d2));
        W0 = exp(lW0);
    } else {
        lW0 = log(W0);
    }
    double f0 = 1 - W0;
    if (!(f0 > 0)) f0 = fmin;
    double lo = f0 / 2, hi = f0;
    double u = 1.0 / fmax(seed, 1.0);
    if (!(lo < u && u < hi)) {
        double Fpp0 = 1.0 - (k1 * k1 * a + k2 * k2 * b);
        u = -4 * lW0 / (8 - lW0 * Fpp0);
        if (!(lo < u && u < hi)) u = 0.7 * f0;
    }
    for (int it = 0; it < 60; ++it) {
        double r1 = 1 + k1 * u, r2 = 1 + k2 * u;
        double Fv = lW0 + a * log1p(k1 * u) + b * log1p(k2 * u) - log1p(-u);
        double sg = k1 * a / r1 + k2 * b / r2;
        double Fp = sg + 1 / (1 - u);
        if (Fv < 0) lo = u;
        else if (Fv > 0) hi = u;
        else break;
        double sgp = -(k1 * k1 * a / (r1 * r1) + k2 * k2 * b / (r2 * r2));
        double Fpp = sgp + 1 / ((1 - u) * (1 - u));
        double un, alt;
        if (1 / (1 - u) > 4 * sg) {
            un = 1 - (1 - u) * exp(Fv);
            alt = u - 2 * Fv * Fp / (2 * Fp * Fp - Fv * Fpp);
        } else {
            un = u - 2 * Fv * Fp / (2 * Fp * Fp - Fv * Fpp);
            alt = 1 - (1 - u) * exp(Fv);
        }
        if (!(lo < un && un < hi)) {
            if (un == lo || un == hi) { u = un; break; }
            un = (lo < alt && alt < hi) ? alt : (lo + hi) / 2;
        }
        bool conv = fabs(un - u) < 4 * eps * (1 + fabs(un));
        u = un;
        if (conv) break;
    }
    double rho = 1.0 / u;
    sp[0] = (a * rho + 1 - al) / d1; sp[1] = (b * rho + al) / d2; sp[2] = -2 * (rho - 1.0) / d3;
    h0 = -lW0 / 2;
    return rho;
}

__device__ __forceinline__ void pow_jetprim(double tau, const double* p, const double* Dp, double al, double& h, double& hp, double& hpp) {
    const double inf = MB_INF, nan = MB_NAN;
    double be = 1.0 - al;                                       // pow.jl:505-531
    double x1 = fma(tau, Dp[0], p[0]), x2 = fma(tau, Dp[1], p[1]), x3 = fma(tau, Dp[2], p[2]);
    if (x1 > 0 && x2 > 0) {
        if (x3 == 0) { h = inf; hp = nan; hpp = nan; return; }
        h = al * log(x1) + be * log(x2) - log(fabs(x3));
        hp = al * Dp[0] / x1 + be * Dp[1] / x2 - Dp[2] / x3;
        hpp = -al * (Dp[0] / x1) * (Dp[0] / x1) - be * (Dp[1] / x2) * (Dp[1] / x2) + (Dp[2] / x3) * (Dp[2] / x3);
        return;
    } else if ((x1 == 0 && x2 >= 0) || (x1 >= 0 && x2 == 0)) {
        h = x3 == 0 ? 0.0 : -inf; hp = nan; hpp = nan; return;
    }
    h = -inf; hp = nan; hpp = nan;
}

__device__ __forceinline__ void pow_jetdual(double tau, const double* d, const double* Dd, double al, double& h, double& hp, double& hpp) {
    const double inf = MB_INF, nan = MB_NAN;
    double be = 1.0 - al;                                       // pow.jl:540-566
    double s1 = fma(tau, Dd[0], d[0]), s2 = fma(tau, Dd[1], d[1]), s3 = fma(tau, Dd[2], d[2]);
    if (s1 > 0 && s2 > 0) {
        if (s3 == 0) { h = inf; hp = nan; hpp = nan; return; }
        h = al * log(s1 / al) + be * log(s2 / be) - log(fabs(s3));
        hp = al * Dd[0] / s1 + be * Dd[1] / s2 - Dd[2] / s3;
        hpp = -al * (Dd[0] / s1) * (Dd[0] / s1) - be * (Dd[1] / s2) * (Dd[1] / s2) + (Dd[2] / s3) * (Dd[2] / s3);
        return;
    } else if ((s1 == 0 && s2 >= 0) || (s1 >= 0 && s2 == 0)) {
        h = s3 == 0 ? 0.0 : -inf; hp = nan; hpp = nan; return;
    }
    h = -inf; hp = nan; hpp = nan;
}

// ------------------------------------------------------------------ shared TDC machinery (tdc.jl)
struct TD {
    int kind;      // CONE_EXP or CONE_POW
    double al;     // α of the power cone
};

__device__ __forceinline__ void tddet(const TD& c, double* C, const double* x) {   // exp.jl:379-392, pow.jl:454-467
    if (c.kind == 4) {
        double psi, ipsi, lr, lrm1;
        expdet(x[0], x[1], x[2], psi, ipsi, lr, lrm1);
        C[TD_D1] = psi; C[TD_D2] = ipsi; C[TD_D3] = lr; C[TD_D4] = lrm1;
        C[TD_H0P] = lr - x[2] / x[1];
    } else {
        double P, rho, inv;
        powdet(x[0], x[1], x[2], c.al, P, rho, inv);
        C[TD_D1] = P; C[TD_D2] = rho; C[TD_D3] = inv;
        C[TD_H0P] = log(P) / 2 - log(fabs(x[2]));
    }
}

__device__ __forceinline__ void tdbarrgrad(const TD& c, double* g, const double* x, const double* C) {
    if (c.kind == 4) {                                           // exp.jl:67-75
        double ipsi = C[TD_D2], lrm1 = C[TD_D4];
        g[0] = -(x[1] * ipsi + 1) / x[0];
        g[1] = -lrm1 * ipsi - 1.0 / x[1];
        g[2] = ipsi;
    } else {                                                     // pow.jl:78-87
        double a = 2 * c.al, b = 2 - 2 * c.al, rho = C[TD_D2], inv = C[TD_D3];
        g[0] = -(a * rho + 1 - c.al) / x[0];
        g[1] = -(b * rho + c.al) / x[1];
        g[2] = 2 * x[2] * inv;
    }
}

__device__ __forceinline__ bool tdfact(const TD& c, double* L, const double* x, const double* C) {
    if (c.kind == 4) {                                           // exp.jl:82-106
        double psi = C[TD_D1], ipsi = C[TD_D2], lrm1 = C[TD_D4];
        double x1 = x[0], x2 = x[1];
        double r1 = 1 + x2 * ipsi, r2 = (psi + 2 * x2) / (psi + x2);
        bool flag = psi > 0 && r1 > 0 && r2 > 0 && isfinite(r1) && isfinite(r2);
        if (flag) {
            double s1 = sqrt(r1);
            L[0] = ipsi; L[1] = -x2 * ipsi / x1; L[2] = -lrm1 * ipsi;
            L[4] = s1 / x1; L[5] = -ipsi / s1; L[8] = sqrt(r2) / x2;
            L[3] = 0; L[6] = 0; L[7] = 0;
        }
        return flag;
    }
    double P = C[TD_D1], rho = C[TD_D2], inv = C[TD_D3];          // pow.jl:100-135
    double x1 = x[0], x2 = x[1], x3 = x[2];
    double a = 2 * c.al, b = 2 - 2 * c.al;
    double w = rho * inv, s = P + x3 * x3;
    double l1 = a / x1, l2 = b / x2;
    double d1 = (2 * rho * a + b) / (2 * x1 * x1), d2 = (2 * rho * b + a) / (2 * x2 * x2);
    double cc = rho * x3 * x3 / s;
    double r1 = d1 - cc * l1 * l1;
    double r2 = (d1 * d2 - cc * (l2 * l2 * d1 + l1 * l1 * d2)) / r1;
    bool flag = r1 > 0 && r2 > 0 && isfinite(r2);
    if (flag) {
        L[0] = sqrt(2 * s) * inv;
        L[1] = -2 * l1 * x3 * w / L[0];
        L[2] = -2 * l2 * x3 * w / L[0];
        L[4] = sqrt(r1);
        L[8] = sqrt(r2);
        L[5] = -cc * l1 * l2 / L[4];
        L[3] = 0; L[6] = 0; L[7] = 0;
    }
    return flag;
}

__device__ __forceinline__ void tdbarrthird(const TD& c, double* D, const double* x, const double* u, const double* C) {
    if (c.kind == 4) {                                           // exp.jl:113-145
        double ipsi = C[TD_D2], lrm1 = C[TD_D4];
        double x1 = x[0], x2 = x[1], u1 = u[0], u2 = u[1], u3 = u[2];
        double g1 = x2 / x1, g2 = lrm1, gu = g1 * u1 + g2 * u2 - u3;
        double H11 = -x2 / (x1 * x1), H21 = 1.0 / x1, H22 = -1.0 / x2;
        double Hu1 = H11 * u1 + H21 * u2, Hu2 = H21 * u1 + H22 * u2;
        double i2 = ipsi * ipsi, i3 = i2 * ipsi;
        double al = -2 * gu * i3;
        double x13 = x1 * x1 * x1, x12 = x1 * x1;
        D[0] = al * g1 * g1 + (2 * g1 * Hu1 + H11 * gu) * i2 - (2 * x2 * u1 / x13 - u2 / x12) * ipsi - 2 * u1 / x13;
        D[1] = al * g1 * g2 + (g1 * Hu2 + g2 * Hu1 + H21 * gu) * i2 + u1 / x12 * ipsi;
        D[2] = -al * g1 - Hu1 * i2;
        D[4] = al * g2 * g2 + (2 * g2 * Hu2 + H22 * gu) * i2 - u2 / (x2 * x2) * ipsi - 2 * u2 / (x2 * x2 * x2);
        D[5] = -al * g2 - Hu2 * i2;
        D[8] = al;
    } else {                                                     // pow.jl:142-188
        double P = C[TD_D1], rho = C[TD_D2], inv = C[TD_D3];
        double x1 = x[0], x2 = x[1], x3 = x[2], u1 = u[0], u2 = u[1], u3 = u[2];
        double a = 2 * c.al, b = 2 - 2 * c.al;
        double l1 = a / x1, l2 = b / x2, m1 = u1 / x1, m2 = u2 / x2;
        double p1 = P * l1, p2 = P * l2, p3 = -2 * x3;
        double dot = p1 * u1 + p2 * u2 + p3 * u3;
        double pp11 = P * l1 * (l1 - 1.0 / x1), pp22 = P * l2 * (l2 - 1.0 / x2), pp12 = P * l1 * l2;
        double dp1 = pp11 * u1 + pp12 * u2, dp2 = pp12 * u1 + pp22 * u2, dp3 = -2 * u3;
        double i2 = inv * inv, i3 = i2 * inv;
        double c2 = dot * i2, c3 = 2 * dot * i3;
        double K = rho * a * b * (a - 1) * (m2 - m1);
        D[0] = 2 * dp1 * p1 * i2 - c3 * p1 * p1 - K / (x1 * x1) + c2 * pp11 - b * m1 / (x1 * x1);
        D[4] = 2 * dp2 * p2 * i2 - c3 * p2 * p2 - K / (x2 * x2) + c2 * pp22 - a * m2 / (x2 * x2);
        D[1] = (dp2 * p1 + p2 * dp1) * i2 - c3 * p2 * p1 + K / (x1 * x2) + c2 * pp12;
        D[8] = 2 * dp3 * p3 * i2 - c3 * p3 * p3 - 2 * c2;
        D[2] = (dp3 * p1 + p3 * dp1) * i2 - c3 * p3 * p1;
        D[5] = (dp3 * p2 + p3 * dp2) * i2 - c3 * p3 * p2;
    }
    D[3] = D[1]; D[6] = D[2]; D[7] = D[5];
}

__device__ __forceinline__ double tddualgrad(const TD& c, double* sp, double seed, const double* d, double* C) {
    double h0;
    double next = c.kind == 4 ? exp_dualgrad(sp, seed, d, h0) : pow_dualgrad(sp, seed, d, c.al, h0);
    C[TD_H0D] = h0;
    return next;
}

// f''(p) x = b with the pivoted factor  (tdc.jl:53-70)
__device__ __forceinline__ void tdhessldiv(const double* L, double* b) {
    double b1 = b[0], b2 = b[1], b3 = b[2];
    double y1 = b3 / L[0];
    double y2 = (b1 - L[1] * y1) / L[4];
    double y3 = (b2 - L[2] * y1 - L[5] * y2) / L[8];
    double z3 = y3 / L[8];
    double z2 = (y2 - L[5] * z3) / L[4];
    double z1 = (y1 - L[1] * z2 - L[2] * z3) / L[0];
    b[0] = z2; b[1] = z3; b[2] = z1;
}
// out = f''(p) v  (tdc.jl:79-95)
__device__ __forceinline__ void tdhessmul(double* out, const double* L, const double* v) {
    double v1 = v[0], v2 = v[1], v3 = v[2];
    double r1 = L[0] * v3 + L[1] * v1 + L[2] * v2;
    double r2 = L[4] * v1 + L[5] * v2;
    double r3 = L[8] * v2;
    double t1 = L[0] * r1;
    double t2 = L[1] * r1 + L[4] * r2;
    double t3 = L[2] * r1 + L[5] * r2 + L[8] * r3;
    out[0] = t2; out[1] = t3; out[2] = t1;
}
// H += μ Pᵀ L Lᵀ P  (tdc.jl:104-118); H is 3x3 column-major
__device__ __forceinline__ void tdgram(double* H, const double* L, double mu) {
    double L11 = L[0], L21 = L[1], L22 = L[4], L31 = L[2], L32 = L[5], L33 = L[8];
    H[8] += mu * (L11 * L11);
    H[0] += mu * (L21 * L21 + L22 * L22);
    H[4] += mu * (L31 * L31 + L32 * L32 + L33 * L33);
    H[2] += mu * L21 * L11; H[6] = H[2];
    H[5] += mu * L31 * L11; H[7] = H[5];
    H[1] += mu * (L31 * L21 + L32 * L22); H[3] = H[1];
}
__device__ __forceinline__ void tdger(double* H, const double* x, const double* y, double al) {  // gerstatic! with β = 1
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) H[i + 3 * j] = fma(1.0, H[i + 3 * j], al * x[i] * y[j]);
}

// t of the Tunçel scaling  (tdc.jl:308-376)
__device__ __forceinline__ double tdbfgs(const double* L, const double* sp, const double* sd, const double* z, const double* p,
                            double muv, double mut) {
    double w[3], Hw[3], Hz[3];
    for (int i = 0; i < 3; ++i) w[i] = fma(-mut, p[i], sp[i]);
    tdhessmul(Hw, L, w);
    double wHw = tdot3(w, Hw);
    double t = 0;
    if (wHw > 0) {
        tdhessmul(Hz, L, z);
        double fppzz = tdot3(z, Hz), sdz = tdot3(sd, z), wHz = tdot3(Hw, z);
        DD s1 = dd_twosum(fppzz, -(sdz * sdz) / 3);
        DD s2 = dd_twosum(s1.h, -(wHz * wHz) / wHw);
        t = muv * (s2.h + (s1.l + s2.l));
    }
    return t;
}

// Tunçel scaling added to H  (tdc.jl:186-294); returns flag, ⟨p*, d*⟩ and the next seed
__device__ bool tdscale(const TD& c, double* H, const double* p, const double* d, double* C, double& spsd) {
    const double eps = MB_EPS;
    double* L = C + TD_L;
    double* sd = C + TD_SD;
    double seed = C[TD_SEED];
    double sp[3], z[3];
    double next = 1.0;
    spsd = 0;
    tddet(c, C, p);
    tdbarrgrad(c, sd, p, C);
    for (int i = 0; i < 3; ++i) sd[i] *= -1;
    bool flag = tdfact(c, L, p, C);
    if (flag) {
        next = tddualgrad(c, sp, seed, d, C);
        double muv = tdot3(p, d) / 3;
        spsd = tcdot3(sp, sd);
        double mut = spsd / 3;
        z[0] = fma(p[1], sp[2], -p[2] * sp[1]);
        z[1] = fma(p[2], sp[0], -p[0] * sp[2]);
        z[2] = fma(p[0], sp[1], -p[1] * sp[0]);
        double nz = sqrt(tdot3(z, z)), np = sqrt(tdot3(p, p)), nsp = sqrt(tdot3(sp, sp));
        if (nz < eps * (np * nsp + eps)) {
            tdgram(H, L, muv);
        } else {
            for (int i = 0; i < 3; ++i) z[i] /= nz;
            double t = tdbfgs(L, sp, sd, z, p, muv, mut);
            if (t <= 0 || !isfinite(t)) {
                tdgram(H, L, muv);
            } else {
                double dp[3], ddv[3];
                for (int i = 0; i < 3; ++i) { dp[i] = fma(-muv, sp[i], p[i]); ddv[i] = fma(-muv, sd[i], d[i]); }
                double pd = 3 * muv, dpd = tcdot3(dp, ddv);
                tdger(H, d, d, 1.0 / pd);
                tdger(H, ddv, ddv, 1.0 / dpd);
                tdger(H, z, z, t);
            }
        }
    }
    C[TD_SEED] = next;
    return flag;
}

// -d - σμ f'(p) - η, η = -½ f'''(p)[Δp, f''(p)⁻¹Δd]  (tdc.jl:394-438)
__device__ __forceinline__ void tdcorr(const TD& c, double* r, const double* p, const double* d, const double* Dp, const double* Dd,
                          double sm, const double* C) {
    double v[3] = {Dd[0], Dd[1], Dd[2]}, D[9], eta[3];
    tdhessldiv(C + TD_L, v);
    tdbarrthird(c, D, p, Dp, C);
    for (int i = 0; i < 3; ++i) {
        double s = 0;
        for (int k = 0; k < 3; ++k) s = fma(D[i + 3 * k], v[k], s);
        eta[i] = -0.5 * s;
    }
    const double* sd = C + TD_SD;
    for (int i = 0; i < 3; ++i) { r[i] = fma(sm, sd[i], -1.0 * d[i]); r[i] = fma(-1.0, eta[i], r[i]); }
}
__device__ __forceinline__ void tdcorr0(double* r, const double* d, double sm, const double* C) {  // tdc.jl:446-450
    const double* sd = C + TD_SD;
    for (int i = 0; i < 3; ++i) r[i] = fma(sm, sd[i], -1.0 * d[i]);
}

// certified log-form line search  (tdc/utils.jl:24-200)
template <class Jet>
__device__ double nflog3(Jet jet, double hi, double glo, double gplo) {
    const double eps = MB_EPS, nan = MB_NAN;
    const double NB = 65536 * eps, K = 8, tol = eps;
    const int maxit = 53;
    double tb = hi, lo = 0, nb = NB;
    if (!(glo >= nb)) return lo;
    double ghi, gphi, gpphi;
    jet(hi, ghi, gphi, gpphi);
    if (ghi >= nb) return hi;
    double whi = (isfinite(gphi) && gphi != 0) ? nb / fabs(gphi) : 0.0;
    auto absorb = [&](double m, double g, double gp, double gpp) {
        if (g >= nb) { lo = m; glo = g; gplo = gp; }
        else {
            hi = m; ghi = g; gphi = gp; gpphi = gpp;
            whi = (isfinite(gp) && gp != 0) ? nb / fabs(gp) : 0.0;
        }
    };
    auto done = [&]() { return hi - lo < fmax(K * whi, tol * (1.0 + hi)); };
    for (int it = 0; it < maxit; ++it) {
        double wid = hi - lo, m;
        if (isfinite(ghi) && ghi >= -nb) {
            m = hi - 3 * fmax(whi, eps * (1.0 + hi)) / 2;
        } else if (isfinite(ghi) && isfinite(glo)) {
            m = lo + glo * wid / (glo - ghi);
            double best = fabs((ghi - glo) / wid - gplo);
            double dlo = tb - lo, dhi = tb - hi;
            if (dhi > 0) {
                double ulo = log(dlo), uhi = log(dhi);
                double cc = (glo - ghi) / (ulo - uhi);
                double e = fabs(-cc / dlo - gplo);
                if (e < best) {
                    best = e;
                    double m2 = tb - exp(ulo - glo * (ulo - uhi) / (glo - ghi));
                    if (lo < m2 && m2 < hi) m = m2;
                }
                double bb = (glo - ghi) / (1.0 / dhi - 1.0 / dlo);
                double aa = glo + bb / dlo;
                e = fabs(-bb / (dlo * dlo) - gplo);
                if (e < best && aa != 0) {
                    double m2 = tb - bb / aa;
                    if (lo < m2 && m2 < hi) m = m2;
                }
            }
        } else {
            m = lo + wid / 2;
        }
        if (!(lo < m && m < hi)) m = lo + wid / 2;
        double g, gp, gpp;
        jet(m, g, gp, gpp);
        absorb(m, g, gp, gpp);
        if (done()) break;
        double dd = tb - hi;
        m = nan;
        if (isfinite(gpphi) && isfinite(gphi) && gphi != 0 && dd > 0) {
            double rho = gpphi * dd / gphi;
            if (0.5 < rho && rho < 1.5) m = tb - dd * exp(ghi / (gphi * dd));
            else if (1.5 <= rho && rho < 3) {
                double den = ghi - gphi * dd;
                if (den != 0) m = tb + gphi * dd * dd / den;
            }
        }
        if (!(lo < m && m < hi)) {
            m = hi - 2 * ghi * gphi / (2 * gphi * gphi - ghi * gpphi);
            if (!(lo < m && m < hi)) m = hi - ghi / gphi;
        }
        if (!(lo < m && m < hi)) m = lo + (hi - lo) / 2;
        jet(m, g, gp, gpp);
        absorb(m, g, gp, gpp);
        if (done()) break;
        if (2 * (hi - lo) > wid) {
            m = lo + (hi - lo) / 2;
            jet(m, g, gp, gpp);
            absorb(m, g, gp, gpp);
            if (done()) break;
        }
    }
    return lo;
}

__device__ void tdmaxsteps(const TD& c, const double* p, const double* Dp, const double* d, const double* Dd,
                              const double* C, double& tp, double& td) {   // tdc.jl:463-483
    double hip = 1.0, hid = 1.0;
    if (Dp[0] < 0) hip = jmin(hip, -p[0] / Dp[0]);
    if (Dp[1] < 0) hip = jmin(hip, -p[1] / Dp[1]);
    if (c.kind == 4) {   // z₁ > 0, z₃ < 0  (exp.jl:169-187)
        if (Dd[0] < 0) hid = jmin(hid, -d[0] / Dd[0]);
        if (Dd[2] > 0) hid = jmin(hid, -d[2] / Dd[2]);
    } else {             // s₁ > 0, s₂ > 0  (pow.jl:216-233)
        if (Dd[0] < 0) hid = jmin(hid, -d[0] / Dd[0]);
        if (Dd[1] < 0) hid = jmin(hid, -d[1] / Dd[1]);
    }
    double hp0p, hp0d;
    if (c.kind == 4) {
        double w = p[2] / p[1];
        hp0p = Dp[0] / p[0] - Dp[1] / p[1] - (Dp[2] - w * Dp[1]) / p[1];
        double r = d[1] / d[2];
        hp0d = Dd[0] / d[0] - (Dd[1] - r * Dd[2]) / d[2] - Dd[2] / d[2];
        tp = nflog3([&](double t, double& h, double& hp, double& hpp) { exp_jetprim(t, p, Dp, h, hp, hpp); }, hip, C[TD_H0P], hp0p);
        td = nflog3([&](double t, double& h, double& hp, double& hpp) { exp_jetdual(t, d, Dd, h, hp, hpp); }, hid, C[TD_H0D], hp0d);
    } else {
        double al = c.al;
        hp0p = al * Dp[0] / p[0] + (1.0 - al) * Dp[1] / p[1] - Dp[2] / p[2];
        hp0d = al * Dd[0] / d[0] + (1.0 - al) * Dd[1] / d[1] - Dd[2] / d[2];
        tp = nflog3([&](double t, double& h, double& hp, double& hpp) { pow_jetprim(t, p, Dp, al, h, hp, hpp); }, hip, C[TD_H0P], hp0p);
        td = nflog3([&](double t, double& h, double& hp, double& hpp) { pow_jetdual(t, d, Dd, al, h, hp, hpp); }, hid, C[TD_H0D], hp0d);
    }
}

__device__ __forceinline__ void tdidentity(const TD& c, double* x) {
    if (c.kind == 4) { x[0] = 1.2909282315382298; x[1] = 0.8051015526498357; x[2] = -0.8278379086082098; }  // exp.jl:15-20
    else { x[0] = sqrt(1 + c.al); x[1] = sqrt(2 - c.al); x[2] = 0.0; }                           // pow.jl:27-33
}
__device__ __forceinline__ void tdinitcache(const TD& c, double* C) { C[TD_SEED] = c.kind == 4 ? 0.8051015526498357 : 1.0; }

// dualshadow! / primalshadow!  (tdc.jl:491-501)
__device__ __forceinline__ bool tddualshadow(const TD& c, double* sd, const double* p, double* C) {
    tddet(c, C, p);
    tdbarrgrad(c, sd, p, C);
    for (int i = 0; i < 3; ++i) sd[i] *= -1;
    return true;
}
__device__ __forceinline__ bool tdprimalshadow(const TD& c, double* sp, const double* d, double* C) {
    tddualgrad(c, sp, 0.0, d, C);
    return true;
}

}  // namespace mb
