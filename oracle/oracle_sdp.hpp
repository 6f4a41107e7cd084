// ORACLE — test infrastructure only (see ipm_oracle.cpp).  Semidefinite cone of Mumblebee.jl,
// restated in FP64 on the CPU: the NT scaling through a Cholesky pair and a one-sided Jacobi SVD,
// the Lyapunov corrector, the eigmin step, and the shadows.
//
//   src/IPM/src/cone/sdp.jl        SemidefiniteCone: degree, cache/workspace layout, sdpscale!,
//                                   sdpcorr!, sdpcorr0!, sdpmaxstep, sdpshadow!
//   src/IPM/src/cone/eig.jl        svdjacobi!, eigminstatic, tridiagonalize!, minorpass,
//                                   laguerremin, eigminsturm!
//   src/IPM/src/cone/utils.jl      smat!/svec!, cholstatic!, l/ldiv/lmul static kernels, mulstatic!,
//                                   syrkstatic!, symmetrize!, skron!
//
// The reference runs unrolled kernels for d ≤ 8 and BLAS/LAPACK above; both compute the same
// mathematics, and this file restates the unrolled kernels' accumulation order for every d (the
// BLAS order for d > 8 is not specified).  Matrices are d×d column-major, 0-based.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <utility>

namespace orc {

static inline int64_t triroot(int64_t n) {   // sdp.jl:29-31
    int64_t t = 1 + 8 * n, r = (int64_t)std::sqrt((double)t);
    while (r * r > t) --r;
    while ((r + 1) * (r + 1) <= t) ++r;
    return (r - 1) / 2;
}

#define SDP_AT(A, i, j) (A)[(size_t)(i) + (size_t)(j) * (size_t)d]

// smat!: lower triangle of M from svec v (utils.jl:630-664)
static inline void sdp_smat(double* M, const double* v, int d) {
    const double a = std::sqrt(2.0);
    int k = 0;
    for (int j = 0; j < d; ++j) {
        SDP_AT(M, j, j) = v[k++];
        for (int i = j + 1; i < d; ++i) SDP_AT(M, i, j) = v[k++] / a;
    }
}
// svec! (utils.jl:594-628)
static inline void sdp_svec(double* v, const double* M, int d) {
    const double a = std::sqrt(2.0);
    int k = 0;
    for (int j = 0; j < d; ++j) {
        v[k++] = SDP_AT(M, j, j);
        for (int i = j + 1; i < d; ++i) v[k++] = a * SDP_AT(M, i, j);
    }
}
// symmetrize!: strict upper from lower (utils.jl:451-470)
static inline void sdp_symm(double* M, int d) {
    for (int j = 0; j < d; ++j)
        for (int i = 0; i < j; ++i) SDP_AT(M, i, j) = SDP_AT(M, j, i);
}
// cholstatic!: lower Cholesky in place, false on a nonpositive pivot (utils.jl:380-412)
static inline bool sdp_chol(double* A, int d) {
    for (int j = 0; j < d; ++j) {
        double djj = SDP_AT(A, j, j);
        for (int p = 0; p < j; ++p) djj = std::fma(-SDP_AT(A, j, p), SDP_AT(A, j, p), djj);
        if (!(djj > 0)) return false;
        double ljj = std::sqrt(djj);
        SDP_AT(A, j, j) = ljj;
        for (int i = j + 1; i < d; ++i) {
            double num = SDP_AT(A, i, j);
            for (int p = 0; p < j; ++p) num = std::fma(-SDP_AT(A, i, p), SDP_AT(A, j, p), num);
            SDP_AT(A, i, j) = num / ljj;
        }
    }
    return true;
}
// mulstatic!: C = op(A) op(B), s accumulated over k = 1..d (utils.jl:225-253)
static inline void sdp_mul(double* C, const double* A, bool tA, const double* B, bool tB, int d) {
    for (int j = 0; j < d; ++j)
        for (int i = 0; i < d; ++i) {
            double s = 0;
            for (int k = 0; k < d; ++k) {
                double a = tA ? SDP_AT(A, k, i) : SDP_AT(A, i, k);
                double b = tB ? SDP_AT(B, j, k) : SDP_AT(B, k, j);
                s = std::fma(a, b, s);
            }
            SDP_AT(C, i, j) = s;
        }
}
// lmulstatic!(LowerTriangular(L)', A): A ← Lᵀ A, rows top-down, p accumulated from d-1 down to i
// (utils.jl:134-172)
static inline void sdp_lmul_lt(double* A, const double* L, int d) {
    for (int c = 0; c < d; ++c)
        for (int i = 0; i < d; ++i) {
            double acc = 0;
            for (int p = d - 1; p >= i; --p) acc = std::fma(SDP_AT(L, p, i), SDP_AT(A, p, c), acc);
            SDP_AT(A, i, c) = acc;
        }
}
// lmulstatic!(LowerTriangular(L), A): A ← L A, rows bottom-up, p accumulated from i down to 0
static inline void sdp_lmul_l(double* A, const double* L, int d) {
    for (int c = 0; c < d; ++c)
        for (int i = d - 1; i >= 0; --i) {
            double acc = 0;
            for (int p = i; p >= 0; --p) acc = std::fma(SDP_AT(L, i, p), SDP_AT(A, p, c), acc);
            SDP_AT(A, i, c) = acc;
        }
}
// ldivstatic!(LowerTriangular(L), M): M ← L⁻¹ M (utils.jl:186-220)
static inline void sdp_ldiv_l(double* M, const double* L, int d) {
    for (int c = 0; c < d; ++c)
        for (int r = 0; r < d; ++r) {
            double num = SDP_AT(M, r, c);
            for (int p = 0; p < r; ++p) num = std::fma(-SDP_AT(L, r, p), SDP_AT(M, p, c), num);
            SDP_AT(M, r, c) = num / SDP_AT(L, r, r);
        }
}
// ldivstatic!(LowerTriangular(L)', M): M ← L⁻ᵀ M
static inline void sdp_ldiv_lt(double* M, const double* L, int d) {
    for (int c = 0; c < d; ++c)
        for (int r = d - 1; r >= 0; --r) {
            double num = SDP_AT(M, r, c);
            for (int p = r + 1; p < d; ++p) num = std::fma(-SDP_AT(L, p, r), SDP_AT(M, p, c), num);
            SDP_AT(M, r, c) = num / SDP_AT(L, r, r);
        }
}
// syrkstatic!: lower C = A Aᵀ, k accumulated from d-1 down to 0 (utils.jl:327-376)
static inline void sdp_syrk(double* C, const double* A, int d) {
    for (int j = 0; j < d; ++j)
        for (int i = j; i < d; ++i) {
            double acc = 0;
            for (int k = d - 1; k >= 0; --k) acc = std::fma(SDP_AT(A, i, k), SDP_AT(A, j, k), acc);
            SDP_AT(C, i, j) = acc;
        }
}
// skron!: H += A ⊗ₛ A over svec coordinates, H is n×n with leading dimension ldh (utils.jl:475-514)
static inline void sdp_skron(double* H, int64_t ldh, const double* A, int d) {
    const double a = std::sqrt(2.0);
    int64_t tll = 0;
    for (int l = 0; l < d; ++l) {
        int64_t tij = 0;
        for (int j = 0; j < d; ++j) {
            double Ajl = SDP_AT(A, j, l);
            H[tij + tll * ldh] += Ajl * Ajl; ++tij;
            for (int i = j + 1; i < d; ++i) { H[tij + tll * ldh] += a * SDP_AT(A, i, l) * Ajl; ++tij; }
        }
        int64_t tkl = tll;
        for (int k = l + 1; k < d; ++k) {
            ++tkl; tij = 0;
            for (int j = 0; j < d; ++j) {
                double Ajk = SDP_AT(A, j, k), Ajl = SDP_AT(A, j, l);
                H[tij + tkl * ldh] += a * Ajk * Ajl; ++tij;
                for (int i = j + 1; i < d; ++i) {
                    H[tij + tkl * ldh] += SDP_AT(A, i, k) * Ajl + SDP_AT(A, i, l) * Ajk; ++tij;
                }
            }
        }
        tll += d - l;
    }
}

// ------------------------------------------------------------------------------------- eig.jl
// one-sided Jacobi SVD in place: U ← left singular vectors, s ← singular values; false when 30
// odd-even sweeps did not orthogonalize the columns (eig.jl:1-175)
static inline bool sdp_svdjacobi(double* U, double* sg, int d) {
    double nA = 0;
    for (int j = 0; j < d; ++j)
        for (int i = 0; i < d; ++i) nA = std::fmax(nA, std::fabs(SDP_AT(U, i, j)));
    bool done = false;
    int eA = std::ilogb(nA), eA1 = eA >> 1;
    double r1 = std::ldexp(1.0, -eA1), r2 = std::ldexp(1.0, -(eA - eA1));
    for (int j = 0; j < d; ++j)
        for (int i = 0; i < d; ++i) { SDP_AT(U, i, j) *= r1; SDP_AT(U, i, j) *= r2; }
    const double eps = std::numeric_limits<double>::epsilon();
    int iter = 0;
    while (!done && iter < 30) {
        ++iter;
        done = true;
        for (int j = 0; j < d; ++j) {
            double s = 0;
            for (int i = 0; i < d; ++i) s = std::fma(SDP_AT(U, i, j), SDP_AT(U, i, j), s);
            sg[j] = s;
        }
        for (int k = 1; k <= d; ++k) {
            int strt = (k & 1) ? 0 : 1;
            for (int p = strt; p < d - 1; p += 2) {
                int q = p + 1;
                double g = 0;
                for (int i = 0; i < d; ++i) g = std::fma(SDP_AT(U, i, p), SDP_AT(U, i, q), g);
                double dp = sg[p], dq = sg[q];
                if (g * g > (double)d * (eps * eps) * dp * dq) {
                    done = false;
                    double z = (dq - dp) / 2;
                    double w = std::sqrt(std::fma(z, z, g * g));
                    double dl = z + std::copysign(w, z);
                    double nu = 1.0 / std::sqrt(2 * w * std::fabs(dl));
                    double c = dl * nu, s = g * nu, t = g / dl;
                    for (int i = 0; i < d; ++i) {
                        double bp = SDP_AT(U, i, p), bq = SDP_AT(U, i, q);
                        SDP_AT(U, i, p) = std::fma(s, bp, c * bq);
                        SDP_AT(U, i, q) = std::fma(c, bp, -s * bq);
                    }
                    sg[p] = std::fma(t, g, dq);
                    sg[q] = std::fma(-t, g, dp);
                } else {
                    for (int i = 0; i < d; ++i) std::swap(SDP_AT(U, i, p), SDP_AT(U, i, q));
                    sg[p] = dq; sg[q] = dp;
                }
            }
        }
    }
    for (int j = 0; j < d; ++j) {
        double nrm = std::sqrt(sg[j]);
        sg[j] = std::ldexp(nrm, eA);
        double r = 1.0 / nrm;
        for (int i = 0; i < d; ++i) SDP_AT(U, i, j) *= r;
    }
    return done;
}

static inline double sdp_nanmin(double a, double b) { return (a != a || b != b) ? NAN : (b < a ? b : a); }
static inline double sdp_nanmax(double a, double b) { return (a != a || b != b) ? NAN : (b > a ? b : a); }

// eigminstatic for d = 1, 2, 3 (eig.jl:180-268)
static inline double sdp_eigmin_small(const double* M, int d) {
    if (d == 1) return M[0];
    if (d == 2) {
        double M11 = SDP_AT(M, 0, 0), M22 = SDP_AT(M, 1, 1), M21 = SDP_AT(M, 1, 0);
        double h = (M11 + M22) / 2, r = std::hypot((M11 - M22) / 2, M21);
        double lmax = h >= 0 ? h + r : h - r;
        if (lmax == 0) return lmax;
        return sdp_nanmin(lmax, std::fma(M11, M22, -M21 * M21) / lmax);
    }
    const double eps = std::numeric_limits<double>::epsilon();
    double M11 = SDP_AT(M, 0, 0), M22 = SDP_AT(M, 1, 1), M33 = SDP_AT(M, 2, 2);
    double M21 = SDP_AT(M, 1, 0), M31 = SDP_AT(M, 2, 0), M32 = SDP_AT(M, 2, 1);
    double m = std::fabs(M11);
    for (double x : {M22, M33, M21, M31, M32}) m = sdp_nanmax(m, std::fabs(x));
    if (m == 0) return 0.0;
    if (!std::isfinite(m)) return NAN;
    int e = std::ilogb(m);
    double s = std::ldexp(1.0, -e);
    double B11 = M11 * s, B22 = M22 * s, B33 = M33 * s, B21 = M21 * s, B31 = M31 * s, B32 = M32 * s;
    double q = (B11 + B22 + B33) / 3;
    double C11 = B11 - q, C22 = B22 - q, C33 = B33 - q;
    double p = std::sqrt((C11 * C11 + C22 * C22 + C33 * C33 + 2 * (B21 * B21 + B31 * B31 + B32 * B32)) / 6);
    double r;
    if (p <= 4 * eps * std::fmax(std::fabs(q), 1.0)) {
        r = 4 * eps * std::fabs(q);
    } else {
        double D11 = C11 / p, D22 = C22 / p, D33 = C33 / p, D21 = B21 / p, D31 = B31 / p, D32 = B32 / p;
        r = (D11 * (D22 * D33 - D32 * D32) - D21 * (D21 * D33 - D32 * D31) + D31 * (D21 * D32 - D22 * D31)) / 2;
        r = std::fmin(std::fmax(r, -1.0), 1.0);
        r = 2 * p * (-std::cos((std::acos(r) + M_PI + M_PI) / 3) + 16 * eps / std::sqrt(std::fmax(1.0 - r * r, 16 * eps)));
    }
    return std::ldexp(q - r, e);
}

// Householder tridiagonalization of the symmetric M (lower triangle used): diagonal → a,
// off-diagonal → b (eig.jl:270-389)
static inline void sdp_tridiagonalize(double* M, double* a, double* b, int d) {
    for (int k = 0; k < d - 2; ++k) {
        double nxr = 0;
        for (int i = k + 2; i < d; ++i) nxr += SDP_AT(M, i, k) * SDP_AT(M, i, k);
        double x1 = SDP_AT(M, k + 1, k);
        if (nxr == 0) {
            b[k] = x1;
            SDP_AT(M, k + 1, k) = 0;
        } else {
            double bk = -std::copysign(std::sqrt(x1 * x1 + nxr), x1);
            b[k] = bk;
            SDP_AT(M, k + 1, k) = 1;
            double r = 1.0 / (x1 - bk);
            for (int i = k + 2; i < d; ++i) SDP_AT(M, i, k) *= r;
            double tau = (bk - x1) / bk;
            double c = 0;
            for (int i = k + 1; i < d; ++i) {
                double wi = 0;
                for (int j = k + 1; j <= i; ++j) wi += SDP_AT(M, i, j) * SDP_AT(M, j, k);
                for (int j = i + 1; j < d; ++j) wi += SDP_AT(M, j, i) * SDP_AT(M, j, k);
                wi *= tau;
                a[i] = wi;
                c += wi * SDP_AT(M, i, k);
            }
            c *= tau / 2;
            for (int i = k + 1; i < d; ++i) a[i] -= c * SDP_AT(M, i, k);
            for (int j = k + 1; j < d; ++j) {
                double vj = SDP_AT(M, j, k), wj = a[j];
                for (int i = j; i < d; ++i) SDP_AT(M, i, j) -= SDP_AT(M, i, k) * wj + a[i] * vj;
            }
        }
    }
    if (d >= 2) b[d - 2] = SDP_AT(M, d - 1, d - 2);
    for (int i = 0; i < d; ++i) a[i] = SDP_AT(M, i, i);
}

// leading principal minors of T − λI (Sturm): positive definiteness and tr((T−λI)⁻¹),
// tr((T−λI)⁻²) (eig.jl:391-462)
static inline bool sdp_minorpass(const double* a, const double* b, double lam, int n, double& s1, double& s2) {
    bool flag = false;
    s1 = s2 = 0;
    const double hi = std::ldexp(1.0, 511), lo = 1.0 / hi;
    double p = 1, pd = 0, pdd = 0;
    double q = a[0] - lam, qd = -1, qdd = 0;
    if (q > 0) {
        flag = true;
        for (int i = 1; i < n; ++i) {
            double av = a[i] - lam, bv = b[i - 1] * b[i - 1];
            double r = std::fma(av, q, -bv * p);
            double rd = std::fma(av, qd, std::fma(-bv, pd, -q));
            double rdd = std::fma(av, qdd, std::fma(-bv, pdd, -2 * qd));
            if (!(r > 0)) { flag = false; break; }
            if (std::fabs(r) > hi) { r *= lo; rd *= lo; rdd *= lo; q *= lo; qd *= lo; qdd *= lo; }
            else if (std::fabs(r) < lo) { r *= hi; rd *= hi; rdd *= hi; q *= hi; qd *= hi; qdd *= hi; }
            p = q; pd = qd; pdd = qdd;
            q = r; qd = rd; qdd = rdd;
        }
        if (flag) {
            s1 = -qd / q;
            s2 = std::fma(s1, s1, -qdd / q);
        }
    }
    return flag;
}

// Laguerre iteration for the smallest eigenvalue of T in [lo, hi] (eig.jl:464-485)
static inline double sdp_laguerremin(const double* a, const double* b, double lo, double hi, int n) {
    const double eps = std::numeric_limits<double>::epsilon();
    double md = lo;
    for (int it = 0; it < 40; ++it) {
        double s1, s2;
        bool flag = sdp_minorpass(a, b, md, n, s1, s2);
        if (!flag) {
            hi = md;
            md = (lo + hi) / 2;
            if (!(md > lo)) break;
        } else {
            lo = md;
            md = std::fmin(lo + n / (s1 + std::sqrt(std::fmax(0.0, (n - 1) * std::fma((double)n, s2, -s1 * s1)))),
                           std::nextafter(hi, -INFINITY));
            if (!(md > lo + 4 * eps * std::fmax(1.0, std::fabs(lo)))) break;
        }
    }
    return lo;
}

// eigmin via tridiagonalization + Laguerre, capped at λmax (eig.jl:487-589); a, b scratch (d each)
static inline double sdp_eigminsturm(double* M, double* a, double* b, int d, double lmax) {
    sdp_tridiagonalize(M, a, b, d);
    double tmax = 0;
    for (int i = 0; i < d; ++i) tmax = sdp_nanmax(tmax, std::fabs(a[i]));
    for (int i = 0; i < d - 1; ++i) tmax = sdp_nanmax(tmax, std::fabs(b[i]));
    if (tmax == 0) return 0.0;
    if (!std::isfinite(tmax)) return NAN;
    if (d == 1) return a[0];
    int texp = std::ilogb(tmax);
    if (texp != 0) {
        double s = std::ldexp(1.0, -texp);
        for (int i = 0; i < d; ++i) a[i] *= s;
        for (int i = 0; i < d - 1; ++i) b[i] *= s;
    }
    double lo = INFINITY, hi = INFINITY, bim1 = 0;
    for (int i = 0; i < d - 1; ++i) {
        double ai = a[i], bi = b[i];
        lo = sdp_nanmin(lo, ai - std::fabs(bim1) - std::fabs(bi));
        hi = sdp_nanmin(hi, ai);
        bim1 = bi;
    }
    double an = a[d - 1];
    hi = sdp_nanmin(sdp_nanmin(hi, an), std::ldexp(lmax, -texp));
    lo = sdp_nanmin(sdp_nanmin(lo, an - std::fabs(bim1)), hi);
    return std::ldexp(sdp_laguerremin(a, b, lo, hi, d), texp);
}

// ------------------------------------------------------------------------------------- sdp.jl
// cache: R (d²) | S (d²) | s (d) (sdp.jl:76-88); workspace max(3d², 2d² + 2d) (sdp.jl:57-70)
static inline int64_t sdp_cachesize(int64_t n) { int64_t d = triroot(n); return 2 * d * d + d; }
static inline int64_t sdp_workspacesize(int64_t n) {
    int64_t d = triroot(n);
    return std::max<int64_t>(3 * d * d, 2 * d * d + 2 * d);
}
static inline void sdp_identity(double* x, int64_t n) {   // sdpid! (sdp.jl:98-110)
    int d = (int)triroot(n);
    for (int64_t i = 0; i < n; ++i) x[i] = 0;
    int64_t k = 0;
    for (int j = 0; j < d; ++j) { x[k] = 1; k += d - j; }
}

// sdpscale!: H += W ⊗ₛ W with W = R Σ Rᵀ the NT point; caches R = LP⁻ᵀU, S = LP U, s = Σ;
// ⟨p*, d*⟩ = Σ 1/sᵢ² (sdp.jl:121-263)
static inline bool sdp_scale(double* H, int64_t n, double* c, const double* p, const double* dv, double* work,
                             double& spsd) {
    int d = (int)triroot(n);
    size_t m = (size_t)d * d;
    double *R = c, *S = c + m, *sg = c + 2 * m;
    double *P = work, *D = work + m;
    sdp_smat(P, p, d);
    sdp_smat(D, dv, d);
    spsd = 0;
    if (!sdp_chol(P, d)) return false;
    if (!sdp_chol(D, d)) return false;
    for (int j = 0; j < d; ++j)
        for (int i = 0; i < d; ++i) SDP_AT(R, i, j) = i >= j ? SDP_AT(D, i, j) : 0.0;
    sdp_lmul_lt(R, P, d);                      // R = LPᵀ LD
    if (!sdp_svdjacobi(R, sg, d)) return false;
    for (size_t k = 0; k < m; ++k) S[k] = R[k];
    sdp_lmul_l(S, P, d);                       // S = LP U
    sdp_ldiv_lt(R, P, d);                      // R = LP⁻ᵀ U
    for (int j = 0; j < d; ++j) {
        double a = std::sqrt(sg[j]);
        for (int i = 0; i < d; ++i) SDP_AT(P, i, j) = SDP_AT(R, i, j) * a;
    }
    sdp_syrk(D, P, d);
    sdp_symm(D, d);
    sdp_skron(H, n, D, d);
    double sp = 0;
    for (int i = 0; i < d; ++i) sp += 1.0 / (sg[i] * sg[i]);
    spsd = sp;
    return true;
}

// the Lyapunov step Ŵ = Σ^½(σμΣ⁻¹ − Σ − 𝓛⁻¹(AB))Σ^½, closed as r = svec(R Ŵ Rᵀ) (sdp.jl:293-431)
static inline void sdp_close(double* r, const double* R, double* W, double* T, int d) {
    sdp_mul(T, W, false, R, true, d);          // T = Ŵ Rᵀ
    sdp_mul(W, R, false, T, false, d);         // W = R Ŵ Rᵀ
    sdp_svec(r, W, d);
}
static inline void sdp_corr(double* r, const double* c, const double* Dp, const double* Dd, double sm, int64_t n,
                            double* work) {
    int d = (int)triroot(n);
    size_t m = (size_t)d * d;
    const double *R = c, *S = c + m, *sg = c + 2 * m;
    double *DP = work, *DD = work + m, *W = work + 2 * m;
    sdp_smat(DP, Dp, d); sdp_smat(DD, Dd, d);
    sdp_symm(DP, d); sdp_symm(DD, d);
    sdp_mul(W, DP, false, R, false, d);  sdp_mul(DP, R, true, W, false, d);    // A = Rᵀ ΔP R
    sdp_mul(W, DD, false, S, false, d);  sdp_mul(DD, S, true, W, false, d);    // B = Sᵀ ΔD S
    sdp_mul(W, DP, false, DD, false, d);                                       // W = A B
    for (int j = 0; j < d; ++j) {
        double sj = sg[j];
        for (int i = 0; i < j; ++i) {
            double v = -((sg[i] * SDP_AT(W, i, j) + sj * SDP_AT(W, j, i)) / (sg[i] + sj));   // weightedmean
            SDP_AT(W, i, j) = v; SDP_AT(W, j, i) = v;
        }
        SDP_AT(W, j, j) = sm - sj * sj - SDP_AT(W, j, j);
    }
    sdp_close(r, R, W, DP, d);
}
static inline void sdp_corr0(double* r, const double* c, double sm, int64_t n, double* work) {   // sdp.jl:437-510
    int d = (int)triroot(n);
    size_t m = (size_t)d * d;
    const double *R = c, *sg = c + 2 * m;
    double *DP = work, *W = work + 2 * m;
    for (size_t k = 0; k < m; ++k) W[k] = 0;
    for (int j = 0; j < d; ++j) SDP_AT(W, j, j) = sm - sg[j] * sg[j];
    sdp_close(r, R, W, DP, d);
}

// largest τ ≤ 1 with X + τΔX PSD through the congruence F: 1/max(1, −λmin(Fᵀ ΔX F ./ (s sᵀ)))
// (sdp.jl:530-630)
static inline double sdp_maxstep(const double* F, const double* Dx, const double* scale, int64_t n, double* work) {
    int d = (int)triroot(n);
    size_t m = (size_t)d * d;
    double *M = work, *C = work + m, *a = work + 2 * m, *b = work + 2 * m + d;
    sdp_smat(M, Dx, d);
    sdp_symm(M, d);
    sdp_mul(C, M, false, F, false, d);         // C = ΔX F
    sdp_mul(M, F, true, C, false, d);          // M = Fᵀ ΔX F
    if (scale)
        for (int j = 0; j < d; ++j)
            for (int i = 0; i < d; ++i) SDP_AT(M, i, j) /= scale[i] * scale[j];
    for (int j = 0; j < d; ++j) {
        for (int i = j; i < d; ++i) SDP_AT(C, i, j) = SDP_AT(M, i, j);
        SDP_AT(C, j, j) += 1.0;
    }
    if (sdp_chol(C, d)) return 1.0;
    double lam = d <= 3 ? sdp_eigmin_small(M, d) : sdp_eigminsturm(M, a, b, d, -1.0);
    return 1.0 / sdp_nanmax(1.0, -lam);
}

// X⁻¹ in svec (the shadow of either side; sdp.jl:640-705); false when X is not positive definite
static inline bool sdp_shadow(double* s, const double* x, int64_t n, double* work) {
    int d = (int)triroot(n);
    size_t m = (size_t)d * d;
    double *M = work, *Z = work + m;
    sdp_smat(M, x, d);
    if (!sdp_chol(M, d)) return false;
    for (int j = 0; j < d; ++j)
        for (int i = 0; i < d; ++i) SDP_AT(Z, i, j) = i == j ? 1.0 : 0.0;
    sdp_ldiv_l(Z, M, d);
    sdp_ldiv_lt(Z, M, d);
    sdp_svec(s, Z, d);
    return true;
}

#undef SDP_AT

}  // namespace orc
