// ORACLE (test infrastructure only): the compensated block-sparse products extmul! / twomul! of
// BlockSparseArrays, restated loop for loop from src/comp/comp.jl:51-311 and
// src/comp/twogemv.jl:5-121.  Compiled without FP contraction (ISO C++, no -ffast-math), so the
// error-free transformations hold; std::fma is the correctly rounded fused multiply-add.
// Included by ipm_oracle.cpp inside namespace orc (uses BSM).

// twosum, twomul (comp.jl:51-61)
static inline void c_twosum(double x, double y, double& s, double& e) {
    s = x + y;
    const double xp = s - y;
    const double yp = s - xp;
    e = (x - xp) + (y - yp);
}
static inline void c_twomul(double x, double y, double& p, double& e) {
    p = x * y;
    e = std::fma(x, y, -p);
}
// twoacc (comp.jl:68-72)
static inline void c_twoacc(double& D, double& d, double a, double x) {
    double p, ep, es;
    c_twomul(a, x, p, ep);
    c_twosum(D, p, D, es);
    d = d + (ep + es);
}
// twoaxpy! (comp.jl:75-84)
static inline void c_twoaxpy(double* s, double* cs, i64 i, double a, double x) {
    double p, ep, sg, es;
    c_twomul(a, x, p, ep);
    c_twosum(s[i], p, sg, es);
    s[i] = sg;
    cs[i] += ep + es;
}
// twofold! (comp.jl:86-94)
static inline void c_twofold(double* s, double* cs, i64 j, double D, double d) {
    double sg, e;
    c_twosum(s[j], D, sg, e);
    s[j] = sg;
    cs[j] += d + e;
}

// twogemv_impl! (twogemv.jl:87-121) with twogemv_one! / twogemv_blk! (:5-85): (s, cs) ← op(A) b
static void c_twogemv(const BSM& A, bool trans, const double* b, double* s, double* cs) {
    const i64 nout = trans ? A.ncol : A.nrow;
    std::fill(s, s + nout, 0.0);
    std::fill(cs, cs + nout, 0.0);
    for (i64 v = 0; v < A.nvtx; ++v) {
        const i64 jstrt = A.xcol[v], ncol = A.ncols(v);
        for (i64 e = A.xsrc[v]; e < A.xsrc[v + 1]; ++e) {
            const i64 u = A.tgt[e], istrt = A.xrow[u], nrow = A.nrows(u);
            const double* blk = A.val.data() + A.xblk[e];
            if (nrow == 1 && ncol == 1) {   // twogemv_one!
                if (!trans) c_twoaxpy(s, cs, istrt, blk[0], b[jstrt]);
                else c_twoaxpy(s, cs, jstrt, blk[0], b[istrt]);
            } else if (!trans) {            // twogemv_blk! :N
                for (i64 j = 0; j < ncol; ++j) {
                    const double bj = b[jstrt + j];
                    for (i64 i = 0; i < nrow; ++i) c_twoaxpy(s, cs, istrt + i, blk[i + j * nrow], bj);
                }
            } else {                        // twogemv_blk! :T (each SIMD lane is one column)
                for (i64 j = 0; j < ncol; ++j) {
                    double D = 0.0, d = 0.0;
                    for (i64 i = 0; i < nrow; ++i) c_twoacc(D, d, blk[i + j * nrow], b[istrt + i]);
                    c_twofold(s, cs, jstrt + j, D, d);
                }
            }
        }
    }
}

// extaxpby! (pair = false, comp.jl:107-170) and twoaxpby! (pair = true, comp.jl:183-248)
static void c_epilogue(i64 n, double* c, double* cc, double alpha, const double* s, const double* cs, double beta,
                       bool pair) {
    for (i64 i = 0; i < n; ++i) {
        double hi, tail;
        if (beta == 0.0) {
            if (alpha == 1.0) {
                hi = s[i]; tail = cs[i];
            } else {
                double p, ep;
                c_twomul(alpha, s[i], p, ep);
                hi = p; tail = std::fma(alpha, cs[i], ep);
            }
        } else if (beta == 1.0 || beta == -1.0) {
            const double ci = beta == 1.0 ? c[i] : -c[i];
            double sg, es;
            if (alpha == 1.0) {
                c_twosum(ci, s[i], sg, es);
                hi = sg; tail = cs[i] + es;
            } else if (alpha == -1.0) {
                c_twosum(ci, -s[i], sg, es);
                hi = sg; tail = es - cs[i];
            } else {
                double p, ep;
                c_twomul(alpha, s[i], p, ep);
                c_twosum(ci, p, sg, es);
                hi = sg; tail = std::fma(alpha, cs[i], ep) + es;
            }
        } else {
            double p1, e1, p2, e2, sg, e3;
            c_twomul(alpha, s[i], p1, e1);
            c_twomul(beta, c[i], p2, e2);
            c_twosum(p1, p2, sg, e3);
            hi = sg; tail = std::fma(alpha, cs[i], e1) + e2 + e3;
        }
        if (pair) c_twosum(hi, tail, c[i], cc[i]);
        else c[i] = hi + tail;
    }
}
