// ORACLE — test infrastructure only.  Cone kernels of the CPU FP64 restatement (see
// ipm_oracle.cpp for the parity status).  Each function cites the reference file:line it
// restates; paths are inside the Mumblebee.jl project (src/IPM/src/...).
#pragma once
#include <cmath>
#include <cstdint>
#include <limits>

enum { CONE_FREE = 0, CONE_POS = 1, CONE_SOC = 2, CONE_SDP = 3, CONE_EXP = 4, CONE_POW = 5 };

namespace orc {

// Julia min/max on floats propagate NaN.
static inline double jmin(double a, double b) { return (a != a || b != b) ? std::numeric_limits<double>::quiet_NaN() : (b < a ? b : a); }
static inline double jmax(double a, double b) { return (a != a || b != b) ? std::numeric_limits<double>::quiet_NaN() : (b > a ? b : a); }
static inline double muladd(double a, double b, double c) { return std::fma(a, b, c); }

// error-free transforms  (IPM/src/utils.jl:27-53)
static inline void twosum(double a, double b, double& s, double& e) {
    s = a + b;
    double bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}
static inline void twoprod(double a, double b, double& p, double& e) {
    p = a * b;
    e = std::fma(a, b, -p);
}
static inline double cdot(const double* p, const double* d, int64_t n) {
    double s = 0, c = 0;
    for (int64_t i = 0; i < n; ++i) {
        double pr, e, e2;
        twoprod(p[i], d[i], pr, e);
        twosum(s, pr, s, e2);
        c += e + e2;
    }
    return s + c;
}

// ---------------------------------------------------------------- second-order cone (soc.jl)
// socdot  (soc.jl:48-61)
static inline void socdot(const double* x, const double* y, int64_t n, double& hi, double& lo) {
    double s, c;
    twoprod(x[0], y[0], s, c);
    for (int64_t i = 1; i < n; ++i) {
        double p, e, e2;
        twoprod(x[i], y[i], p, e);
        twosum(s, -p, s, e2);
        c += -e + e2;
    }
    twosum(s, c, hi, lo);
}

// socroot!  (soc.jl:82-110)
static inline void socroot(double* x, const double* w, double beta, bool flag, int64_t n) {
    double sg, al;
    if (!flag) { sg = -1.0; al = 1.0 / beta; } else { sg = 1.0; al = beta; }
    double w1p1 = w[0] + 1;
    double wpdx = w1p1 * x[0];
    for (int64_t i = 1; i < n; ++i) wpdx = muladd(sg * w[i], x[i], wpdx);
    wpdx /= w1p1;
    x[0] = al * muladd(wpdx, w1p1, -x[0]);
    for (int64_t i = 1; i < n; ++i) x[i] = al * muladd(sg * wpdx, w[i], x[i]);
}

// cache layout (soc.jl:146-156): beta, pdet, ddet, pdetlo, ddetlo, w[n]
static inline bool socscale(double* H, double* c, const double* p, const double* d, int64_t n, double* spsd_out) {
    double* w = c + 5;
    double pdet, pdetlo, ddet, ddetlo;
    socdot(p, p, n, pdet, pdetlo);
    socdot(d, d, n, ddet, ddetlo);
    bool flag = pdet > 0 && p[0] > 0 && ddet > 0 && d[0] > 0;
    double beta = 0, spsd = 0;
    if (flag) {  // soc.jl:192-263
        double pdot = cdot(p, d, n);
        double spdet = std::sqrt(pdet), sddet = std::sqrt(ddet);
        double kappa = std::sqrt(2.0 * muladd(spdet, sddet, pdot));
        beta = std::sqrt(spdet / sddet);
        w[0] = muladd(d[0], beta, p[0] / beta) / kappa;
        for (int64_t i = 1; i < n; ++i) w[i] = muladd(-d[i], beta, p[i] / beta) / kappa;
        double eta = 1.0 / (beta * beta), eta2 = 2 * eta;
        double w1 = w[0];
        H[0] = muladd(eta2, w1 * w1, H[0] - eta);
        double nw1 = -eta2 * w1;
        for (int64_t i = 1; i < n; ++i) { double t = muladd(nw1, w[i], H[0 + i * n]); H[i] = t; H[0 + i * n] = t; }
        for (int64_t j = 1; j < n; ++j) {
            double wj = w[j];
            H[j + j * n] = muladd(eta2, wj * wj, H[j + j * n] + eta);
            double ew = eta2 * wj;
            for (int64_t i = j + 1; i < n; ++i) { double t = muladd(ew, w[i], H[j + i * n]); H[i + j * n] = t; H[j + i * n] = t; }
        }
        spsd = 4 * pdot / (pdet * ddet);
    }
    c[0] = beta; c[1] = pdet; c[2] = ddet; c[3] = pdetlo; c[4] = ddetlo;
    *spsd_out = spsd;
    return flag;
}

// soccorr!  (soc.jl:282-351)
static inline void soccorr(double* r, const double* c, const double* p, const double* Dp0, const double* Dd0,
                           double sm, int64_t n, double* work) {
    const double* w = c + 5;
    double beta = c[0], pdet = c[1];
    double* Dp = work;
    double* Dd = work + n;
    for (int64_t i = 0; i < n; ++i) { Dp[i] = Dp0[i]; Dd[i] = Dd0[i]; }
    socroot(Dp, w, beta, false, n);
    socroot(Dd, w, beta, true, n);
    double Dp1 = Dp[0], Dd1 = Dd[0];
    double dt = 0;
    for (int64_t i = 0; i < n; ++i) dt += Dp[i] * Dd[i];
    r[0] = dt;
    for (int64_t i = 1; i < n; ++i) r[i] = muladd(Dd1, Dp[i], Dp1 * Dd[i]);
    for (int64_t i = 0; i < n; ++i) Dp[i] = p[i];
    socroot(Dp, w, beta, false, n);
    double Dpdet, lo;
    socdot(Dp, Dp, n, Dpdet, lo);
    Dp1 = Dp[0];
    double Dpr;
    socdot(Dp, r, n, Dpr, lo);
    double r1 = Dpr / Dpdet;
    r[0] = r1;
    double iDp1 = 1.0 / Dp1;
    for (int64_t i = 1; i < n; ++i) r[i] = muladd(-r1, Dp[i], r[i]) * iDp1;
    for (int64_t i = 0; i < n; ++i) r[i] += Dp[i];
    socroot(r, w, beta, false, n);
    double gamma = 2 * sm / pdet;
    r[0] = muladd(gamma, p[0], -r[0]);
    for (int64_t i = 1; i < n; ++i) r[i] = muladd(-gamma, p[i], -r[i]);
}

// soccorr0!  (soc.jl:362-379)
static inline void soccorr0(double* r, const double* c, const double* p, double sm, int64_t n) {
    const double* w = c + 5;
    double beta = c[0], pdet = c[1];
    double eta = (1.0 / beta) * (1.0 / beta);
    double wp, lo;
    socdot(w, p, n, wp, lo);
    double t = 2 * eta * wp;
    double c1 = 2 * sm / pdet + eta;
    r[0] = muladd(c1, p[0], -t * w[0]);
    for (int64_t i = 1; i < n; ++i) r[i] = muladd(t, w[i], -c1 * p[i]);
}

// socmaxstep  (soc.jl:391-470)
static inline double socmaxstep(const double* x, const double* Dx, double c, double clo, int64_t n) {
    const double eps = std::numeric_limits<double>::epsilon();
    double a, alo, b, blo;
    socdot(Dx, Dx, n, a, alo);
    socdot(x, Dx, n, b, blo);
    b *= 2; blo *= 2;
    double tau = 1.0;
    if (std::fabs(a) > eps * jmax(std::fabs(b), std::fabs(c))) {
        double bb, bblo, ac, aclo, s0, s0lo;
        twoprod(b, b, bb, bblo);
        bblo = muladd(2 * b, blo, bblo);
        twoprod(4 * a, c, ac, aclo);
        aclo = muladd(4 * a, clo, muladd(4 * alo, c, aclo));
        twosum(bb, -ac, s0, s0lo);
        double dd = s0 + ((bblo - aclo) + s0lo);
        if (dd > -(eps * jmax(bb, std::fabs(ac)))) {
            double s = std::sqrt(jmax(dd, 0.0));
            double q = -(b + std::copysign(s, b)) / 2;
            double tau1 = b >= 0 ? q / a : c / q;
            if (tau1 > 0) tau = jmin(tau, tau1);
        }
    } else if (b < 0) {
        tau = jmin(tau, -c / b);
    }
    double Dx1 = Dx[0];
    if (Dx1 < 0) tau = jmin(tau, -x[0] / Dx1);
    return tau;
}

// socshadow!  (soc.jl:488-504)
static inline bool socshadow(double* s, const double* x, int64_t n) {
    double xdet, lo;
    socdot(x, x, n, xdet, lo);
    bool flag = xdet > 0 && x[0] > 0;
    if (flag) {
        double g = 2 / xdet;
        s[0] = g * x[0];
        for (int64_t i = 1; i < n; ++i) s[i] = -g * x[i];
    }
    return flag;
}

// ---------------------------------------------------------------- orthant (pos.jl)
static inline double posmaxstep(const double* x, const double* Dx, int64_t n) {  // pos.jl:155-167
    double tau = 1.0;
    for (int64_t i = 0; i < n; ++i) if (Dx[i] < 0) tau = jmin(tau, -x[i] / Dx[i]);
    return tau;
}

}  // namespace orc

#include "oracle_tdc.hpp"
#include "oracle_sdp.hpp"

namespace orc {

// ---------------------------------------------------------------- dispatch
static inline int64_t cone_degree(int k, int64_t n) {
    switch (k) {
        case CONE_POS: return n;           // pos.jl:21-23
        case CONE_SOC: return 2;           // soc.jl:116-118
        case CONE_FREE: return 0;          // noc.jl:20-22
        case CONE_EXP: case CONE_POW: return 3;   // tdc.jl:131-134
        case CONE_SDP: return triroot(n);  // sdp.jl:41-43
        default: return 0;
    }
}
static inline int64_t cone_cachesize(int k, int64_t n) {
    switch (k) {
        case CONE_SOC: return 5 + n;       // soc.jl:124-126
        case CONE_EXP: case CONE_POW: return 19;  // tdc.jl:140-143
        case CONE_SDP: return sdp_cachesize(n);
        default: return 0;
    }
}
static inline int64_t cone_workspacesize(int k, int64_t n) {
    switch (k) {
        case CONE_SOC: return 2 * n;       // soc.jl:132-134
        case CONE_EXP: case CONE_POW: return 15;  // tdc.jl:122-125
        case CONE_SDP: return sdp_workspacesize(n);
        default: return 0;
    }
}
static inline void cone_identity(int k, double kp, int64_t n, double* x) {
    switch (k) {
        case CONE_EXP: case CONE_POW: tdidentity(TD{k, kp}, x); break;
        case CONE_POS: for (int64_t i = 0; i < n; ++i) x[i] = 1.0; break;      // pos.jl:43-50
        case CONE_SOC: for (int64_t i = 0; i < n; ++i) x[i] = 0.0; if (n > 0) x[0] = std::sqrt(2.0); break;  // soc.jl:163-167
        case CONE_SDP: sdp_identity(x, n); break;
        default: for (int64_t i = 0; i < n; ++i) x[i] = 0.0; break;             // noc.jl:38-41
    }
}
static inline bool cone_scale(int k, double kp, int64_t n, double* H, const double* p, const double* d, double* c,
                              double* work, double* spsd) {
    switch (k) {
        case CONE_SDP: return sdp_scale(H, n, c, p, d, work, *spsd);
        case CONE_EXP: case CONE_POW: return tdscale(TD{k, kp}, H, p, d, c, *spsd);
        case CONE_POS: {  // pos.jl:75-84
            double s = 0;
            for (int64_t i = 0; i < n; ++i) { H[i + i * n] += d[i] / p[i]; s += 1.0 / (p[i] * d[i]); }
            *spsd = s;
            return true;
        }
        case CONE_SOC: return socscale(H, c, p, d, n, spsd);
        default: *spsd = 0; return true;
    }
}
static inline void cone_corr(int k, double kp, int64_t n, double* r, const double* p, const double* d,
                             const double* Dp, const double* Dd, double sm, double* c, double* work) {
    switch (k) {
        case CONE_EXP: case CONE_POW: tdcorr(TD{k, kp}, r, p, d, Dp, Dd, sm, c); break;
        case CONE_POS: for (int64_t i = 0; i < n; ++i) r[i] = (sm - Dp[i] * Dd[i]) / p[i] - d[i]; break;  // pos.jl:107-120
        case CONE_SOC: soccorr(r, c, p, Dp, Dd, sm, n, work); break;
        case CONE_SDP: sdp_corr(r, c, Dp, Dd, sm, n, work); break;
        default: for (int64_t i = 0; i < n; ++i) r[i] = 0.0; break;   // noc.jl:63-77
    }
}
static inline void cone_corr0(int k, double, int64_t n, double* r, const double* p, const double* d, double sm,
                              double* c, double* work) {
    switch (k) {
        case CONE_EXP: case CONE_POW: tdcorr0(r, d, sm, c); break;
        case CONE_SDP: sdp_corr0(r, c, sm, n, work); break;
        case CONE_POS: for (int64_t i = 0; i < n; ++i) r[i] = sm / p[i] - d[i]; break;  // pos.jl:126-137
        case CONE_SOC: soccorr0(r, c, p, sm, n); break;
        default: for (int64_t i = 0; i < n; ++i) r[i] = 0.0; break;
    }
}
static inline void cone_maxsteps(int k, double kp, int64_t n, const double* p, const double* Dp, const double* d,
                                 const double* Dd, double* c, double* work, double* tp, double* td) {
    switch (k) {
        case CONE_SDP: {   // sdp.jl:516-519: τp through R, τd through S scaled by Σ
            int64_t dd = triroot(n);
            *tp = sdp_maxstep(c, Dp, nullptr, n, work);
            *td = sdp_maxstep(c + dd * dd, Dd, c + 2 * dd * dd, n, work);
            break;
        }
        case CONE_EXP: case CONE_POW: tdmaxsteps(TD{k, kp}, p, Dp, d, Dd, c, *tp, *td); break;
        case CONE_POS: *tp = posmaxstep(p, Dp, n); *td = posmaxstep(d, Dd, n); break;
        case CONE_SOC: *tp = socmaxstep(p, Dp, c[1], c[3], n); *td = socmaxstep(d, Dd, c[2], c[4], n); break;
        default: *tp = 1.0; *td = 1.0; break;
    }
}
// dual shadow d* = -f'(p)
static inline bool cone_shadow(int k, double kp, int64_t n, double* s, const double* x, double* c, double* work) {
    switch (k) {
        case CONE_SDP: return sdp_shadow(s, x, n, work);
        case CONE_EXP: case CONE_POW: return tddualshadow(TD{k, kp}, s, x, c);
        case CONE_POS: for (int64_t i = 0; i < n; ++i) s[i] = 1.0 / x[i]; return true;  // pos.jl:198-204
        case CONE_SOC: return socshadow(s, x, n);
        default: for (int64_t i = 0; i < n; ++i) s[i] = 0.0; return true;
    }
}
// primal shadow p*: -f'(p*) = d
static inline bool cone_pshadow(int k, double kp, int64_t n, double* s, const double* x, double* c, double* work) {
    if (k == CONE_EXP || k == CONE_POW) return tdprimalshadow(TD{k, kp}, s, x, c);
    return cone_shadow(k, kp, n, s, x, c, work);
}
static inline void cone_initcache(int k, double kp, int64_t, double* c) {
    if (k == CONE_EXP || k == CONE_POW) tdinitcache(TD{k, kp}, c);
}

}  // namespace orc
