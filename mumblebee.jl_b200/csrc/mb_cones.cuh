// Device cone kernels: one warp per cone (lanes across the cone's coordinates).  Restated from
// Mumblebee.jl src/IPM/src/cone/{pos,soc,noc}.jl; file:line citations on each function.
// Compensated J-products are reduced across lanes with error-free transforms, so they carry the
// same ~2u accuracy as the sequential compensated loops of the reference (the rounding of the
// last bits differs because the summation order does).
#pragma once
#include "mb_device.cuh"

namespace mb {

// J-inner product x₁y₁ − x₂y₂ − … as a (hi, lo) pair  (soc.jl:48-61)
__device__ __forceinline__ void w_socdot(const double* x, const double* y, int n, double& hi, double& lo) {
    const int lane = threadIdx.x & 31;
    double s = 0, c = 0;
    for (int i = lane; i < n; i += 32) {
        double p, e, e2;
        twoprod(x[i], y[i], p, e);
        if (i == 0) { twosum(s, p, s, e2); c += e + e2; }
        else { twosum(s, -p, s, e2); c += -e + e2; }
    }
    warp_csum(s, c);
    twosum(s, c, hi, lo);
}
// compensated plain dot (IPM/src/utils.jl:41-53)
__device__ __forceinline__ double w_cdot(const double* x, const double* y, int n) {
    const int lane = threadIdx.x & 31;
    double s = 0, c = 0;
    for (int i = lane; i < n; i += 32) {
        double p, e, e2;
        twoprod(x[i], y[i], p, e);
        twosum(s, p, s, e2);
        c += e + e2;
    }
    warp_csum(s, c);
    return s + c;
}
__device__ __forceinline__ double w_dot(const double* x, const double* y, int n) {
    const int lane = threadIdx.x & 31;
    double s = 0;
    for (int i = lane; i < n; i += 32) s = fma(x[i], y[i], s);
    return warp_sum(s);
}

// y = √H x (flag=false) or solve √H y = x (flag=true) at the NT point  (soc.jl:82-110)
__device__ __forceinline__ void w_socroot(double* x, const double* w, double beta, bool flag, int n) {
    const int lane = threadIdx.x & 31;
    double sg = flag ? 1.0 : -1.0, al = flag ? beta : 1.0 / beta;
    double w1p1 = w[0] + 1;
    double part = 0;
    for (int i = lane; i < n; i += 32) part = (i == 0) ? fma(w1p1, x[0], part) : fma(sg * w[i], x[i], part);
    double wpdx = warp_sum(part) / w1p1;
    __syncwarp();
    for (int i = lane; i < n; i += 32)
        x[i] = (i == 0) ? al * fma(wpdx, w1p1, -x[0]) : al * fma(sg * wpdx, w[i], x[i]);
    __syncwarp();
}

// NT scaling point in factored form β, w = ω/β  (soc.jl:192-230, 257-262); warp per cone.
// cache: beta, pdet, ddet, pdetlo, ddetlo, w[n]
__device__ bool w_socpoint(double* c, const double* p, const double* d, int n, double& spsd) {
    const int lane = threadIdx.x & 31;
    double* w = c + 5;
    double pdet, pdetlo, ddet, ddetlo;
    w_socdot(p, p, n, pdet, pdetlo);
    w_socdot(d, d, n, ddet, ddetlo);
    bool flag = pdet > 0 && p[0] > 0 && ddet > 0 && d[0] > 0;
    double beta = 0;
    spsd = 0;
    if (flag) {
        double pdot = w_cdot(p, d, n);
        double spdet = sqrt(pdet), sddet = sqrt(ddet);
        double kappa = sqrt(2.0 * fma(spdet, sddet, pdot));
        beta = sqrt(spdet / sddet);
        for (int i = lane; i < n; i += 32)
            w[i] = (i == 0 ? fma(d[0], beta, p[0] / beta) : fma(-d[i], beta, p[i] / beta)) / kappa;
        spsd = 4 * pdot / (pdet * ddet);
    }
    if (lane == 0) { c[0] = beta; c[1] = pdet; c[2] = ddet; c[3] = pdetlo; c[4] = ddetlo; }
    __syncwarp();
    return flag;
}

// H = Q + (2 (Jw)(Jw)ᵀ − J) / β² on an (n x n) block (soc.jl:231-256), all threads of the CTA, in
// one pass over H: each unordered pair takes the upper entry of Q as its addend and is written to
// both halves, as the reference does; `qzero` skips the reads of an all-zero Q block.
__device__ void b_sochess(double* H, const double* Q, bool qzero, const double* c, int n) {
    const double* w = c + 5;
    const double beta = c[0];
    const double eta = 1.0 / (beta * beta), eta2 = 2 * eta;
    const double w1 = w[0];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int cc = warp; cc < n; cc += NW) {
        for (int r = lane; r < n; r += 32) {
            const int a = min(r, cc), b = max(r, cc);
            const double q = qzero ? 0.0 : Q[a + (int64_t)b * n];
            double v;
            if (a == b) v = a == 0 ? fma(eta2, w1 * w1, q - eta) : fma(eta2, w[a] * w[a], q + eta);
            else v = a == 0 ? fma(-eta2 * w1, w[b], q) : fma(eta2 * w[a], w[b], q);
            H[r + (int64_t)cc * n] = v;
        }
    }
}

// (H x)_i for row i of an SOC block with a zero Q block: H = (2 z zᵀ − diag(1, −1, …, −1)) / β² with
// z = Jw = (w₁, −w₂, …), so H x = η (−x₁, x₂, …) + 2η z (zᵀx); `zx` = zᵀx of the cone
__device__ __forceinline__ double socz_row(const double* c, const double* x, int i, double zx) {
    const double* w = c + 5;
    const double eta = 1.0 / (c[0] * c[0]), eta2 = 2 * eta;
    const double zi = i == 0 ? w[0] : -w[i];
    return fma(eta2 * zi, zx, i == 0 ? -eta * x[0] : eta * x[i]);
}

// zᵀx of one cone (warp): z = (w₁, −w₂, …)
__device__ __forceinline__ double w_soczdot(const double* c, const double* x, int n) {
    const double* w = c + 5;
    const int lane = threadIdx.x & 31;
    double s = 0;
    for (int i = lane; i < n; i += 32) s = fma(i == 0 ? w[0] : -w[i], x[i], s);
    return warp_sum(s);
}

// Mehrotra corrector  (soc.jl:282-351); work holds 2n doubles owned by this warp
__device__ void w_soccorr(double* r, const double* c, const double* p, const double* Dp0, const double* Dd0,
                          double sm, int n, double* work) {
    const int lane = threadIdx.x & 31;
    const double* w = c + 5;
    double beta = c[0], pdet = c[1];
    double* Dp = work;
    double* Dd = work + n;
    for (int i = lane; i < n; i += 32) { Dp[i] = Dp0[i]; Dd[i] = Dd0[i]; }
    __syncwarp();
    w_socroot(Dp, w, beta, false, n);
    w_socroot(Dd, w, beta, true, n);
    double Dp1 = Dp[0], Dd1 = Dd[0];
    double r1 = w_dot(Dp, Dd, n);
    for (int i = lane; i < n; i += 32) r[i] = (i == 0) ? r1 : fma(Dd1, Dp[i], Dp1 * Dd[i]);
    __syncwarp();
    for (int i = lane; i < n; i += 32) Dp[i] = p[i];
    __syncwarp();
    w_socroot(Dp, w, beta, false, n);
    double Dpdet, lo, Dpr;
    w_socdot(Dp, Dp, n, Dpdet, lo);
    Dp1 = Dp[0];
    w_socdot(Dp, r, n, Dpr, lo);
    r1 = Dpr / Dpdet;
    double iDp1 = 1.0 / Dp1;
    __syncwarp();
    for (int i = lane; i < n; i += 32) r[i] = ((i == 0) ? r1 : fma(-r1, Dp[i], r[i]) * iDp1) + Dp[i];
    __syncwarp();
    w_socroot(r, w, beta, false, n);
    double gamma = 2 * sm / pdet;
    for (int i = lane; i < n; i += 32) r[i] = (i == 0) ? fma(gamma, p[0], -r[0]) : fma(-gamma, p[i], -r[i]);
    __syncwarp();
}

// corrector with Δp = Δd = 0  (soc.jl:362-379)
__device__ void w_soccorr0(double* r, const double* c, const double* p, double sm, int n) {
    const int lane = threadIdx.x & 31;
    const double* w = c + 5;
    double beta = c[0], pdet = c[1];
    double eta = (1.0 / beta) * (1.0 / beta);
    double wp, lo;
    w_socdot(w, p, n, wp, lo);
    double t = 2 * eta * wp;
    double c1 = 2 * sm / pdet + eta;
    for (int i = lane; i < n; i += 32) r[i] = (i == 0) ? fma(c1, p[0], -t * w[0]) : fma(t, w[i], -c1 * p[i]);
    __syncwarp();
}

// largest τ ≤ 1 with x + τΔx ∈ K  (soc.jl:391-470)
__device__ double w_socmaxstep(const double* x, const double* Dx, double c, double clo, int n) {
    const double eps = 2.220446049250313e-16;
    double a, alo, b, blo;
    w_socdot(Dx, Dx, n, a, alo);
    w_socdot(x, Dx, n, b, blo);
    b *= 2; blo *= 2;
    double tau = 1.0;
    if (fabs(a) > eps * jmax(fabs(b), fabs(c))) {
        double bb, bblo, ac, aclo, s0, s0lo;
        twoprod(b, b, bb, bblo);
        bblo = fma(2 * b, blo, bblo);
        twoprod(4 * a, c, ac, aclo);
        aclo = fma(4 * a, clo, fma(4 * alo, c, aclo));
        twosum(bb, -ac, s0, s0lo);
        double dd = s0 + ((bblo - aclo) + s0lo);
        if (dd > -(eps * jmax(bb, fabs(ac)))) {
            double s = sqrt(jmax(dd, 0.0));
            double q = -(b + copysign(s, b)) / 2;
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

// s = -f'(x) = 2Jx/det(x)  (soc.jl:488-504)
__device__ bool w_socshadow(double* s, const double* x, int n) {
    const int lane = threadIdx.x & 31;
    double xdet, lo;
    w_socdot(x, x, n, xdet, lo);
    bool flag = xdet > 0 && x[0] > 0;
    if (flag) {
        double g = 2 / xdet;
        for (int i = lane; i < n; i += 32) s[i] = (i == 0) ? g * x[0] : -g * x[i];
    }
    __syncwarp();
    return flag;
}

// orthant ratio test  (pos.jl:155-167)
__device__ __forceinline__ double w_posmaxstep(const double* x, const double* Dx, int n) {
    const int lane = threadIdx.x & 31;
    double tau = 1.0;
    for (int i = lane; i < n; i += 32) if (Dx[i] < 0) tau = jmin(tau, -x[i] / Dx[i]);
    return warp_jmin(tau);
}

__device__ __forceinline__ int cone_degree(int k, int n) {
    return k == CONE_POS ? n : (k == CONE_SOC ? 2 : 0);   // pos.jl:21-23, soc.jl:116-118, noc.jl:20-22
}

// identity element e with -f'(e) = e  (pos.jl:43-50, soc.jl:163-167, noc.jl:38-41)
__device__ __forceinline__ void w_identity(int k, int n, double* x) {
    const int lane = threadIdx.x & 31;
    for (int i = lane; i < n; i += 32)
        x[i] = (k == CONE_POS) ? 1.0 : ((k == CONE_SOC && i == 0) ? sqrt(2.0) : 0.0);
    __syncwarp();
}

}  // namespace mb
