// Semidefinite cone on the device: the whole CTA works on one cone at a time (its matrices are
// d×d dense, so every step is a small dense kernel).  Restates SemidefiniteCone of Mumblebee.jl:
//
//   src/IPM/src/cone/sdp.jl     sdpscale! (NT point through chol(P), chol(D) and the SVD of LPᵀLD),
//                                sdpcorr!, sdpcorr0!, sdpmaxstep, sdpshadow!, cache/workspace layout
//   src/IPM/src/cone/eig.jl     svdjacobi!, eigminstatic, tridiagonalize!, minorpass, laguerremin,
//                                eigminsturm!
//   src/IPM/src/cone/utils.jl   smat!/svec!, cholstatic!, the triangular l/ldiv/lmul kernels,
//                                mulstatic!, syrkstatic!, symmetrize!, skron!
//
// Every b_* function is called by all threads of the block with the same arguments and ends with a
// barrier.  Work is split so that each output element (or each column of a triangular multiply or
// solve) is produced by one thread with the reference's accumulation order; the sequential pieces
// (Cholesky pivots, Jacobi inner products, the tridiagonal Laguerre search) run on one thread.
// Matrices are d×d column-major in the instance's cone workspace; R | S | s live in the cone cache.
#pragma once
#include "mb_device.cuh"

namespace mb {

struct SdpSh {
    double* red;       // ≥ 1 double of block-shared scratch (the reduction buffer)
    int* flag;         // one block-shared int
    double* tile = nullptr;   // optional block-shared scratch for b_skron_sm
    int tilecap = 0;          // its size in doubles
};

#define SAT(A, i, j) (A)[(size_t)(i) + (size_t)(j) * (size_t)d]

__device__ __forceinline__ int sdp_triroot(int n) {   // sdp.jl:29-31
    int t = 1 + 8 * n, r = (int)sqrt((double)t);
    while (r * r > t) --r;
    while ((r + 1) * (r + 1) <= t) ++r;
    return (r - 1) / 2;
}
// svec position of (i, j), i ≥ j, and its inverse
__device__ __forceinline__ int sdp_sidx(int i, int j, int d) { return j * d - j * (j - 1) / 2 + (i - j); }
__device__ __forceinline__ void sdp_ij(int t, int d, int& i, int& j) {
    int jj = 0, s = 0;
    while (t >= s + (d - jj)) { s += d - jj; ++jj; }
    j = jj; i = jj + (t - s);
}

// smat! (utils.jl:630-664): lower triangle, and with `full` the upper too
__device__ void b_smat(double* M, const double* v, int d, bool full) {
    const double a = sqrt(2.0);
    for (int t = threadIdx.x; t < d * d; t += NT) {
        int i = t % d, j = t / d;
        if (i == j) M[t] = v[sdp_sidx(i, j, d)];
        else if (i > j) M[t] = v[sdp_sidx(i, j, d)] / a;
        else if (full) M[t] = v[sdp_sidx(j, i, d)] / a;
    }
    __syncthreads();
}
// svec! (utils.jl:594-628)
__device__ void b_svec(double* v, const double* M, int d) {
    const double a = sqrt(2.0);
    for (int t = threadIdx.x; t < d * d; t += NT) {
        int i = t % d, j = t / d;
        if (i == j) v[sdp_sidx(i, j, d)] = M[t];
        else if (i > j) v[sdp_sidx(i, j, d)] = a * M[t];
    }
    __syncthreads();
}
// cholstatic! (utils.jl:380-412): lower Cholesky in place; false (uniformly) on a nonpositive pivot
__device__ bool b_chol(double* A, int d, SdpSh sh) {
    for (int j = 0; j < d; ++j) {
        if (threadIdx.x == 0) {
            double djj = SAT(A, j, j);
            for (int p = 0; p < j; ++p) djj = fma(-SAT(A, j, p), SAT(A, j, p), djj);
            bool ok = djj > 0;
            double ljj = ok ? sqrt(djj) : 0.0;
            if (ok) SAT(A, j, j) = ljj;
            sh.red[0] = ljj;
            *sh.flag = ok ? 1 : 0;
        }
        __syncthreads();
        if (!*sh.flag) { __syncthreads(); return false; }
        double ljj = sh.red[0];
        for (int i = j + 1 + threadIdx.x; i < d; i += NT) {
            double num = SAT(A, i, j);
            for (int p = 0; p < j; ++p) num = fma(-SAT(A, i, p), SAT(A, j, p), num);
            SAT(A, i, j) = num / ljj;
        }
        __syncthreads();
    }
    return true;
}
// mulstatic! (utils.jl:225-253): C = op(A) op(B), C distinct from A and B
__device__ void b_mul(double* C, const double* A, bool tA, const double* B, bool tB, int d) {
    for (int t = threadIdx.x; t < d * d; t += NT) {
        int i = t % d, j = t / d;
        double s = 0;
        for (int k = 0; k < d; ++k) {
            double a = tA ? SAT(A, k, i) : SAT(A, i, k);
            double b = tB ? SAT(B, j, k) : SAT(B, k, j);
            s = fma(a, b, s);
        }
        C[t] = s;
    }
    __syncthreads();
}
// A ← Lᵀ A (lmulstatic! with LowerTriangular(L)', utils.jl:134-172): one thread per column
__device__ void b_lmul_lt(double* A, const double* L, int d) {
    for (int c = threadIdx.x; c < d; c += NT)
        for (int i = 0; i < d; ++i) {
            double acc = 0;
            for (int p = d - 1; p >= i; --p) acc = fma(SAT(L, p, i), SAT(A, p, c), acc);
            SAT(A, i, c) = acc;
        }
    __syncthreads();
}
// A ← L A
__device__ void b_lmul_l(double* A, const double* L, int d) {
    for (int c = threadIdx.x; c < d; c += NT)
        for (int i = d - 1; i >= 0; --i) {
            double acc = 0;
            for (int p = i; p >= 0; --p) acc = fma(SAT(L, i, p), SAT(A, p, c), acc);
            SAT(A, i, c) = acc;
        }
    __syncthreads();
}
// M ← L⁻¹ M (ldivstatic!, utils.jl:186-220)
__device__ void b_ldiv_l(double* M, const double* L, int d) {
    for (int c = threadIdx.x; c < d; c += NT)
        for (int r = 0; r < d; ++r) {
            double num = SAT(M, r, c);
            for (int p = 0; p < r; ++p) num = fma(-SAT(L, r, p), SAT(M, p, c), num);
            SAT(M, r, c) = num / SAT(L, r, r);
        }
    __syncthreads();
}
// M ← L⁻ᵀ M
__device__ void b_ldiv_lt(double* M, const double* L, int d) {
    for (int c = threadIdx.x; c < d; c += NT)
        for (int r = d - 1; r >= 0; --r) {
            double num = SAT(M, r, c);
            for (int p = r + 1; p < d; ++p) num = fma(-SAT(L, p, r), SAT(M, p, c), num);
            SAT(M, r, c) = num / SAT(L, r, r);
        }
    __syncthreads();
}
// syrkstatic! + symmetrize!: C = A Aᵀ, both triangles (utils.jl:327-376, 451-470)
__device__ void b_syrk_full(double* C, const double* A, int d) {
    for (int t = threadIdx.x; t < d * d; t += NT) {
        int i = t % d, j = t / d;
        if (i < j) continue;
        double acc = 0;
        for (int k = d - 1; k >= 0; --k) acc = fma(SAT(A, i, k), SAT(A, j, k), acc);
        SAT(C, i, j) = acc;
        SAT(C, j, i) = acc;
    }
    __syncthreads();
}
// skron!: H += A ⊗ₛ A in svec coordinates, H n×n with leading dimension ldh (utils.jl:475-514)
__device__ void b_skron(double* H, int64_t ldh, const double* A, int d) {
    const double a = sqrt(2.0);
    const int n = d * (d + 1) / 2;
    for (int64_t t = threadIdx.x; t < (int64_t)n * n; t += NT) {
        int r = (int)(t % n), c = (int)(t / n);
        int i, j, k, l;
        sdp_ij(r, d, i, j);
        sdp_ij(c, d, k, l);
        double v;
        if (k == l) v = i == j ? SAT(A, j, l) * SAT(A, j, l) : a * SAT(A, i, l) * SAT(A, j, l);
        else v = i == j ? a * SAT(A, j, k) * SAT(A, j, l) : SAT(A, i, k) * SAT(A, j, l) + SAT(A, i, l) * SAT(A, j, k);
        H[r + (int64_t)c * ldh] += v;
    }
    __syncthreads();
}

// b_skron with A and the svec index table (r -> (i, j)) staged in shared memory `sm` of at least
// d² + n doubles: a warp per column of H, its lanes down the rows, each entry from the same formula
// and operand order as b_skron.  With `assign` H is overwritten instead of added to.
__device__ void b_skron_sm(double* H, int64_t ldh, const double* A, int d, double* sm, bool assign) {
    const double a = sqrt(2.0);
    const int n = d * (d + 1) / 2;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double* As = sm;
    int* tab = reinterpret_cast<int*>(sm + (size_t)d * d);
    for (int t = threadIdx.x; t < d * d; t += NT) As[t] = A[t];
    for (int r = threadIdx.x; r < n; r += NT) { int i, j; sdp_ij(r, d, i, j); tab[2 * r] = i; tab[2 * r + 1] = j; }
    __syncthreads();
    for (int c = warp; c < n; c += NW) {
        const int k = tab[2 * c], l = tab[2 * c + 1];
        double* Hc = H + (int64_t)c * ldh;
        for (int r = lane; r < n; r += 32) {
            const int i = tab[2 * r], j = tab[2 * r + 1];
            double v;
            if (k == l) v = i == j ? SAT(As, j, l) * SAT(As, j, l) : a * SAT(As, i, l) * SAT(As, j, l);
            else v = i == j ? a * SAT(As, j, k) * SAT(As, j, l) : SAT(As, i, k) * SAT(As, j, l) + SAT(As, i, l) * SAT(As, j, k);
            if (assign) Hc[r] = v; else Hc[r] += v;
        }
    }
    __syncthreads();
}

// H x for an SDP block whose Q block is zero, H = W ⊗ₛ W: (W ⊗ₛ W) svec(X) = svec(W X W), two d×d
// products instead of a pass over the n×n block.  Workspace 2d².
__device__ void b_sdphx(double* y, const double* W, const double* x, int n, double* work) {
    const int d = sdp_triroot(n);
    const size_t m = (size_t)d * d;
    double *X = work, *T = work + m;
    b_smat(X, x, d, true);
    b_mul(T, W, false, X, false, d);   // T = W X
    b_mul(X, T, false, W, false, d);   // X = W X W
    b_svec(y, X, d);
}

// one-sided Jacobi SVD (eig.jl:1-175): U ← left singular vectors, sg ← singular values; the
// disjoint pairs of one odd-even round run on separate warps.  false when 30 sweeps did not
// orthogonalize the columns.
__device__ bool b_svdjacobi(double* U, double* sg, int d, SdpSh sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double nA = 0;
    for (int t = threadIdx.x; t < d * d; t += NT) nA = fmax(nA, fabs(U[t]));
    nA = block_reduce(nA, sh.red, OpMax(), 0.0);
    const int eA = ilogb(nA), eA1 = eA >> 1;
    const double r1 = ldexp(1.0, -eA1), r2 = ldexp(1.0, -(eA - eA1));
    for (int t = threadIdx.x; t < d * d; t += NT) { U[t] *= r1; U[t] *= r2; }
    __syncthreads();
    const double eps = 2.220446049250313e-16;
    bool done = false;
    int iter = 0;
    while (!done && iter < 30) {
        ++iter;
        if (threadIdx.x == 0) *sh.flag = 1;
        for (int j = threadIdx.x; j < d; j += NT) {
            double s = 0;
            for (int i = 0; i < d; ++i) s = fma(SAT(U, i, j), SAT(U, i, j), s);
            sg[j] = s;
        }
        __syncthreads();
        for (int k = 1; k <= d; ++k) {
            const int strt = (k & 1) ? 0 : 1, npair = (d - strt) / 2;
            for (int pi = warp; pi < npair; pi += NW) {
                const int p = strt + 2 * pi, q = p + 1;
                double g = 0;
                if (lane == 0)
                    for (int i = 0; i < d; ++i) g = fma(SAT(U, i, p), SAT(U, i, q), g);
                g = __shfl_sync(0xffffffffu, g, 0);
                const double dp = sg[p], dq = sg[q];
                if (g * g > (double)d * (eps * eps) * dp * dq) {
                    if (lane == 0) *sh.flag = 0;
                    const double z = (dq - dp) / 2;
                    const double w = sqrt(fma(z, z, g * g));
                    const double dl = z + copysign(w, z);
                    const double nu = 1.0 / sqrt(2 * w * fabs(dl));
                    const double c = dl * nu, s = g * nu, t = g / dl;
                    for (int i = lane; i < d; i += 32) {
                        double bp = SAT(U, i, p), bq = SAT(U, i, q);
                        SAT(U, i, p) = fma(s, bp, c * bq);
                        SAT(U, i, q) = fma(c, bp, -s * bq);
                    }
                    __syncwarp();
                    if (lane == 0) { sg[p] = fma(t, g, dq); sg[q] = fma(-t, g, dp); }
                } else {
                    for (int i = lane; i < d; i += 32) {
                        double bp = SAT(U, i, p);
                        SAT(U, i, p) = SAT(U, i, q);
                        SAT(U, i, q) = bp;
                    }
                    __syncwarp();
                    if (lane == 0) { sg[p] = dq; sg[q] = dp; }
                }
                __syncwarp();
            }
            __syncthreads();
        }
        done = *sh.flag != 0;
        __syncthreads();
    }
    for (int j = threadIdx.x; j < d; j += NT) {
        double nrm = sqrt(sg[j]);
        sg[j] = ldexp(nrm, eA);
        double r = 1.0 / nrm;
        for (int i = 0; i < d; ++i) SAT(U, i, j) *= r;
    }
    __syncthreads();
    return done;
}

// ---- eigmin (one thread) --------------------------------------------------------------------
__device__ __forceinline__ double sdp_nanmin(double a, double b) { return (a != a || b != b) ? MB_NAN : (b < a ? b : a); }
__device__ __forceinline__ double sdp_nanmax(double a, double b) { return (a != a || b != b) ? MB_NAN : (b > a ? b : a); }

// eigminstatic, d = 1, 2, 3 (eig.jl:180-268)
__device__ double t_eigmin_small(const double* M, int d) {
    if (d == 1) return M[0];
    if (d == 2) {
        double M11 = SAT(M, 0, 0), M22 = SAT(M, 1, 1), M21 = SAT(M, 1, 0);
        double h = (M11 + M22) / 2, r = hypot((M11 - M22) / 2, M21);
        double lmax = h >= 0 ? h + r : h - r;
        if (lmax == 0) return lmax;
        return sdp_nanmin(lmax, fma(M11, M22, -M21 * M21) / lmax);
    }
    const double eps = 2.220446049250313e-16, pi = 3.141592653589793;
    double M11 = SAT(M, 0, 0), M22 = SAT(M, 1, 1), M33 = SAT(M, 2, 2);
    double M21 = SAT(M, 1, 0), M31 = SAT(M, 2, 0), M32 = SAT(M, 2, 1);
    double m = fabs(M11);
    m = sdp_nanmax(m, fabs(M22)); m = sdp_nanmax(m, fabs(M33));
    m = sdp_nanmax(m, fabs(M21)); m = sdp_nanmax(m, fabs(M31)); m = sdp_nanmax(m, fabs(M32));
    if (m == 0) return 0.0;
    if (!isfinite(m)) return MB_NAN;
    int e = ilogb(m);
    double s = ldexp(1.0, -e);
    double B11 = M11 * s, B22 = M22 * s, B33 = M33 * s, B21 = M21 * s, B31 = M31 * s, B32 = M32 * s;
    double q = (B11 + B22 + B33) / 3;
    double C11 = B11 - q, C22 = B22 - q, C33 = B33 - q;
    double p = sqrt((C11 * C11 + C22 * C22 + C33 * C33 + 2 * (B21 * B21 + B31 * B31 + B32 * B32)) / 6);
    double r;
    if (p <= 4 * eps * fmax(fabs(q), 1.0)) {
        r = 4 * eps * fabs(q);
    } else {
        double D11 = C11 / p, D22 = C22 / p, D33 = C33 / p, D21 = B21 / p, D31 = B31 / p, D32 = B32 / p;
        r = (D11 * (D22 * D33 - D32 * D32) - D21 * (D21 * D33 - D32 * D31) + D31 * (D21 * D32 - D22 * D31)) / 2;
        r = fmin(fmax(r, -1.0), 1.0);
        r = 2 * p * (-cos((acos(r) + pi + pi) / 3) + 16 * eps / sqrt(fmax(1.0 - r * r, 16 * eps)));
    }
    return ldexp(q - r, e);
}

// tridiagonalize! (eig.jl:270-389): diagonal → a, off-diagonal → b
__device__ void t_tridiagonalize(double* M, double* a, double* b, int d) {
    for (int k = 0; k < d - 2; ++k) {
        double nxr = 0;
        for (int i = k + 2; i < d; ++i) nxr += SAT(M, i, k) * SAT(M, i, k);
        double x1 = SAT(M, k + 1, k);
        if (nxr == 0) {
            b[k] = x1;
            SAT(M, k + 1, k) = 0;
        } else {
            double bk = -copysign(sqrt(x1 * x1 + nxr), x1);
            b[k] = bk;
            SAT(M, k + 1, k) = 1;
            double r = 1.0 / (x1 - bk);
            for (int i = k + 2; i < d; ++i) SAT(M, i, k) *= r;
            double tau = (bk - x1) / bk;
            double c = 0;
            for (int i = k + 1; i < d; ++i) {
                double wi = 0;
                for (int j = k + 1; j <= i; ++j) wi += SAT(M, i, j) * SAT(M, j, k);
                for (int j = i + 1; j < d; ++j) wi += SAT(M, j, i) * SAT(M, j, k);
                wi *= tau;
                a[i] = wi;
                c += wi * SAT(M, i, k);
            }
            c *= tau / 2;
            for (int i = k + 1; i < d; ++i) a[i] -= c * SAT(M, i, k);
            for (int j = k + 1; j < d; ++j) {
                double vj = SAT(M, j, k), wj = a[j];
                for (int i = j; i < d; ++i) SAT(M, i, j) -= SAT(M, i, k) * wj + a[i] * vj;
            }
        }
    }
    if (d >= 2) b[d - 2] = SAT(M, d - 1, d - 2);
    for (int i = 0; i < d; ++i) a[i] = SAT(M, i, i);
}

// tridiagonalize! on the whole block: the same Householder steps as t_tridiagonalize, with each
// element's arithmetic unchanged; the O(d²) parts of a step (scaling the reflector, w = τ M v and
// the rank-2 update) run one element or row per thread, the two inner products on thread 0 in
// their sequential order.  M is d×d (lower triangle used) in shared or global memory.
__device__ void b_tridiagonalize(double* M, double* a, double* b, int d, SdpSh sh) {
    double* sc = sh.red;   // sc[0] = r, sc[1] = τ, sc[2] = c, sc[3] = 1 when the reflector is trivial
    for (int k = 0; k < d - 2; ++k) {
        if (threadIdx.x == 0) {
            double nxr = 0;
            for (int i = k + 2; i < d; ++i) nxr += SAT(M, i, k) * SAT(M, i, k);
            double x1 = SAT(M, k + 1, k);
            if (nxr == 0) {
                b[k] = x1;
                SAT(M, k + 1, k) = 0;
                sc[3] = 1;
            } else {
                double bk = -copysign(sqrt(x1 * x1 + nxr), x1);
                b[k] = bk;
                SAT(M, k + 1, k) = 1;
                sc[0] = 1.0 / (x1 - bk);
                sc[1] = (bk - x1) / bk;
                sc[3] = 0;
            }
        }
        __syncthreads();
        if (sc[3] != 0) { __syncthreads(); continue; }
        const double r = sc[0], tau = sc[1];
        for (int i = k + 2 + threadIdx.x; i < d; i += NT) SAT(M, i, k) *= r;
        __syncthreads();
        for (int i = k + 1 + threadIdx.x; i < d; i += NT) {
            double wi = 0;
            for (int j = k + 1; j <= i; ++j) wi += SAT(M, i, j) * SAT(M, j, k);
            for (int j = i + 1; j < d; ++j) wi += SAT(M, j, i) * SAT(M, j, k);
            a[i] = wi * tau;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double c = 0;
            for (int i = k + 1; i < d; ++i) c += a[i] * SAT(M, i, k);
            sc[2] = c * (tau / 2);
        }
        __syncthreads();
        const double c = sc[2];
        for (int i = k + 1 + threadIdx.x; i < d; i += NT) a[i] -= c * SAT(M, i, k);
        __syncthreads();
        const int w = d - k - 1;   // trailing order; element (i, j), i ≥ j ≥ k + 1
        for (int t = threadIdx.x; t < w * w; t += NT) {
            const int i = k + 1 + t % w, j = k + 1 + t / w;
            if (i >= j) SAT(M, i, j) -= SAT(M, i, k) * a[j] + a[i] * SAT(M, j, k);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (d >= 2) b[d - 2] = SAT(M, d - 1, d - 2);
        for (int i = 0; i < d; ++i) a[i] = SAT(M, i, i);
    }
    __syncthreads();
}

// minorpass (eig.jl:391-462)
__device__ bool t_minorpass(const double* a, const double* b, double lam, int n, double& s1, double& s2) {
    bool flag = false;
    s1 = s2 = 0;
    const double hi = ldexp(1.0, 511), lo = 1.0 / hi;
    double p = 1, pd = 0, pdd = 0;
    double q = a[0] - lam, qd = -1, qdd = 0;
    if (q > 0) {
        flag = true;
        for (int i = 1; i < n; ++i) {
            double av = a[i] - lam, bv = b[i - 1] * b[i - 1];
            double r = fma(av, q, -bv * p);
            double rd = fma(av, qd, fma(-bv, pd, -q));
            double rdd = fma(av, qdd, fma(-bv, pdd, -2 * qd));
            if (!(r > 0)) { flag = false; break; }
            if (fabs(r) > hi) { r *= lo; rd *= lo; rdd *= lo; q *= lo; qd *= lo; qdd *= lo; }
            else if (fabs(r) < lo) { r *= hi; rd *= hi; rdd *= hi; q *= hi; qd *= hi; qdd *= hi; }
            p = q; pd = qd; pdd = qdd;
            q = r; qd = rd; qdd = rdd;
        }
        if (flag) {
            s1 = -qd / q;
            s2 = fma(s1, s1, -qdd / q);
        }
    }
    return flag;
}

// laguerremin (eig.jl:464-485)
__device__ double t_laguerremin(const double* a, const double* b, double lo, double hi, int n) {
    const double eps = 2.220446049250313e-16;
    double md = lo;
    for (int it = 0; it < 40; ++it) {
        double s1, s2;
        bool flag = t_minorpass(a, b, md, n, s1, s2);
        if (!flag) {
            hi = md;
            md = (lo + hi) / 2;
            if (!(md > lo)) break;
        } else {
            lo = md;
            md = fmin(lo + n / (s1 + sqrt(fmax(0.0, (n - 1) * fma((double)n, s2, -s1 * s1)))), nextafter(hi, -MB_INF));
            if (!(md > lo + 4 * eps * fmax(1.0, fabs(lo)))) break;
        }
    }
    return lo;
}

// eigminsturm! (eig.jl:487-589)
__device__ double t_eigminsturm_ab(double* a, double* b, int d, double lmax);
__device__ double t_eigminsturm(double* M, double* a, double* b, int d, double lmax) {
    t_tridiagonalize(M, a, b, d);
    return t_eigminsturm_ab(a, b, d, lmax);
}
// the Sturm / Laguerre part of eigminsturm! on the tridiagonal (a, b)
__device__ double t_eigminsturm_ab(double* a, double* b, int d, double lmax) {
    double tmax = 0;
    for (int i = 0; i < d; ++i) tmax = sdp_nanmax(tmax, fabs(a[i]));
    for (int i = 0; i < d - 1; ++i) tmax = sdp_nanmax(tmax, fabs(b[i]));
    if (tmax == 0) return 0.0;
    if (!isfinite(tmax)) return MB_NAN;
    if (d == 1) return a[0];
    int texp = ilogb(tmax);
    if (texp != 0) {
        double s = ldexp(1.0, -texp);
        for (int i = 0; i < d; ++i) a[i] *= s;
        for (int i = 0; i < d - 1; ++i) b[i] *= s;
    }
    double lo = MB_INF, hi = MB_INF, bim1 = 0;
    for (int i = 0; i < d - 1; ++i) {
        double ai = a[i], bi = b[i];
        lo = sdp_nanmin(lo, ai - fabs(bim1) - fabs(bi));
        hi = sdp_nanmin(hi, ai);
        bim1 = bi;
    }
    double an = a[d - 1];
    hi = sdp_nanmin(sdp_nanmin(hi, an), ldexp(lmax, -texp));
    lo = sdp_nanmin(sdp_nanmin(lo, an - fabs(bim1)), hi);
    return ldexp(t_laguerremin(a, b, lo, hi, d), texp);
}

// ---- cone methods (sdp.jl) --------------------------------------------------------------------
// identity (sdpid!, sdp.jl:98-110), one warp
__device__ __forceinline__ void w_sdpidentity(double* x, int n) {
    const int d = sdp_triroot(n);
    for (int t = threadIdx.x & 31; t < n; t += 32) {
        int i, j;
        sdp_ij(t, d, i, j);
        x[t] = i == j ? 1.0 : 0.0;
    }
    __syncwarp();
}

// sdpscale! (sdp.jl:121-263): H += W ⊗ₛ W (H = W ⊗ₛ W with `assign`), W = R Σ Rᵀ; cache
// R = LP⁻ᵀU | S = LP U | s = Σ | W; spsd = Σ 1/sᵢ².  Workspace 2d².  false (uniformly) when p or d
// is not positive definite or the SVD did not converge.
__device__ bool b_sdpscale(double* H, int n, double* c, const double* p, const double* dv, double* work,
                           double& spsd, SdpSh sh, bool assign = false) {
    const int d = sdp_triroot(n);
    const size_t m = (size_t)d * d;
    double *R = c, *S = c + m, *sg = c + 2 * m;
    double *P = work, *D = work + m;
    spsd = 0;
    b_smat(P, p, d, false);
    b_smat(D, dv, d, false);
    if (!b_chol(P, d, sh)) return false;
    if (!b_chol(D, d, sh)) return false;
    for (int t = threadIdx.x; t < d * d; t += NT) R[t] = (t % d) >= (t / d) ? D[t] : 0.0;
    __syncthreads();
    b_lmul_lt(R, P, d);                        // R = LPᵀ LD
    if (!b_svdjacobi(R, sg, d, sh)) return false;
    for (int t = threadIdx.x; t < d * d; t += NT) S[t] = R[t];
    __syncthreads();
    b_lmul_l(S, P, d);                         // S = LP U
    b_ldiv_lt(R, P, d);                        // R = LP⁻ᵀ U
    for (int t = threadIdx.x; t < d * d; t += NT) P[t] = R[t] * sqrt(sg[t / d]);
    __syncthreads();
    b_syrk_full(D, P, d);                      // W = (R Σ^½)(R Σ^½)ᵀ
    double* Wc = c + 2 * m + d;
    for (int t = threadIdx.x; t < d * d; t += NT) Wc[t] = D[t];
    if (sh.tile && (int64_t)d * d + n <= sh.tilecap) b_skron_sm(H, n, D, d, sh.tile, assign);
    else {
        if (assign) { for (int64_t t = threadIdx.x; t < (int64_t)n * n; t += NT) H[t] = 0.0; __syncthreads(); }
        b_skron(H, n, D, d);
    }
    if (threadIdx.x == 0) {
        double sp = 0;
        for (int i = 0; i < d; ++i) sp += 1.0 / (sg[i] * sg[i]);
        sh.red[0] = sp;
    }
    __syncthreads();
    spsd = sh.red[0];
    __syncthreads();
    return true;
}

// r = svec(R Ŵ Rᵀ) (the closing congruence of sdpcorr!/sdpcorr0!); T scratch
__device__ void b_sdpclose(double* r, const double* R, double* W, double* T, int d) {
    b_mul(T, W, false, R, true, d);
    b_mul(W, R, false, T, false, d);
    b_svec(r, W, d);
}

// sdpcorr! (sdp.jl:293-431): Ŵ off-diagonal −(sᵢXᵢⱼ + sⱼXⱼᵢ)/(sᵢ+sⱼ), diagonal σμ − sⱼ² − Xⱼⱼ with
// X = (Rᵀ ΔP R)(Sᵀ ΔD S).  Workspace 3d².
__device__ void b_sdpcorr(double* r, const double* c, const double* Dp, const double* Dd, double sm, int n,
                          double* work) {
    const int d = sdp_triroot(n);
    const size_t m = (size_t)d * d;
    const double *R = c, *S = c + m, *sg = c + 2 * m;
    double *DP = work, *DD = work + m, *W = work + 2 * m;
    b_smat(DP, Dp, d, true);
    b_smat(DD, Dd, d, true);
    b_mul(W, DP, false, R, false, d);  b_mul(DP, R, true, W, false, d);     // A = Rᵀ ΔP R
    b_mul(W, DD, false, S, false, d);  b_mul(DD, S, true, W, false, d);     // B = Sᵀ ΔD S
    b_mul(W, DP, false, DD, false, d);                                      // W = A B
    for (int t = threadIdx.x; t < d * d; t += NT) {
        int i = t % d, j = t / d;
        if (i < j) {
            double v = -((sg[i] * SAT(W, i, j) + sg[j] * SAT(W, j, i)) / (sg[i] + sg[j]));
            SAT(W, i, j) = v;
            SAT(W, j, i) = v;
        } else if (i == j) {
            SAT(W, j, j) = sm - sg[j] * sg[j] - SAT(W, j, j);
        }
    }
    __syncthreads();
    b_sdpclose(r, R, W, DP, d);
}

// sdpcorr0! (sdp.jl:437-510): Ŵ = diag(σμ − sⱼ²)
__device__ void b_sdpcorr0(double* r, const double* c, double sm, int n, double* work) {
    const int d = sdp_triroot(n);
    const size_t m = (size_t)d * d;
    const double *R = c, *sg = c + 2 * m;
    double *DP = work, *W = work + 2 * m;
    for (int t = threadIdx.x; t < d * d; t += NT) {
        int i = t % d, j = t / d;
        W[t] = i == j ? sm - sg[j] * sg[j] : 0.0;
    }
    __syncthreads();
    b_sdpclose(r, R, W, DP, d);
}

// sdpmaxstep (sdp.jl:530-630): 1 when I + M ≻ 0 for M = Fᵀ ΔX F ./ (scale scaleᵀ), else
// 1/max(1, −λmin(M)).  Workspace 2d² + 2d.  Returns the same value on every thread.
__device__ double b_sdpmaxstep(const double* F, const double* Dx, const double* scale, int n, double* work, SdpSh sh) {
    const int d = sdp_triroot(n);
    const size_t m = (size_t)d * d;
    double *M = work, *C = work + m, *a = work + 2 * m, *b = work + 2 * m + d;
    b_smat(M, Dx, d, true);
    b_mul(C, M, false, F, false, d);           // C = ΔX F
    b_mul(M, F, true, C, false, d);            // M = Fᵀ ΔX F
    for (int t = threadIdx.x; t < d * d; t += NT) {
        int i = t % d, j = t / d;
        double v = M[t];
        if (scale) { v /= scale[i] * scale[j]; M[t] = v; }
        if (i >= j) C[t] = i == j ? v + 1.0 : v;
    }
    __syncthreads();
    if (b_chol(C, d, sh)) return 1.0;
    if (d > 3) {   // the tridiagonalization on the whole block, in shared memory when it fits
        double* T = (sh.tile && (int64_t)d * d <= sh.tilecap) ? sh.tile : M;
        if (T != M) { for (int t = threadIdx.x; t < d * d; t += NT) T[t] = M[t]; __syncthreads(); }
        b_tridiagonalize(T, a, b, d, sh);
    }
    if (threadIdx.x == 0) {
        double lam = d <= 3 ? t_eigmin_small(M, d) : t_eigminsturm_ab(a, b, d, -1.0);
        sh.red[0] = 1.0 / sdp_nanmax(1.0, -lam);
    }
    __syncthreads();
    double tau = sh.red[0];
    __syncthreads();
    return tau;
}

// sdpshadow! (sdp.jl:640-705): s = svec(X⁻¹); false (uniformly) when X is not positive definite
__device__ bool b_sdpshadow(double* s, const double* x, int n, double* work, SdpSh sh) {
    const int d = sdp_triroot(n);
    const size_t m = (size_t)d * d;
    double *M = work, *Z = work + m;
    b_smat(M, x, d, false);
    if (!b_chol(M, d, sh)) return false;
    for (int t = threadIdx.x; t < d * d; t += NT) Z[t] = (t % d) == (t / d) ? 1.0 : 0.0;
    __syncthreads();
    b_ldiv_l(Z, M, d);
    b_ldiv_lt(Z, M, d);
    b_svec(s, Z, d);
    return true;
}

#undef SAT

}  // namespace mb
