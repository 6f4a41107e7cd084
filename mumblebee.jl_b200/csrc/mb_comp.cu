// Compensated block-sparse matrix-vector products: extmul! / twomul! of BlockSparseArrays
// (BlockSparseArrays/src/comp/comp.jl:1-311, comp/twogemv.jl:1-121).
//
// One fused launch per call: each thread owns one output entry, runs phase 1 (the pair (s, cs) of
// op(A) b accumulated with error-free transformations) in exactly the order twogemv_impl! visits
// that entry, then the α/β epilogue of extaxpby! or twoaxpby! with the reference's branches.  The
// order makes the results bitwise equal to the reference's:
//   A b  (:N): row i takes its terms in ascending column order (vertices ascending, columns
//              ascending inside a vertex; one arc per vertex reaches a given row), each through
//              twoaxpy!: (s, cs) += a b_j.
//   Aᵀ b (:T): column j takes one register pair (Δ, δ) per block of its vertex, arcs in ascending
//              target order, rows ascending inside the block (twoacc), folded into (s, cs) at the
//              end of the block (twofold!); a 1 x 1 block goes through twoaxpy! directly
//              (twogemv_one!).
// Every stored block entry takes part, explicit zeros included, as in the reference.  All sums
// and products are the non-contracting __dadd_rn / __dsub_rn / __dmul_rn: an error-free
// transformation computes its error term from the rounded result, so a fused multiply-add
// formed by the compiler would change it.
#include <cstdint>

#include "mb_internal.h"

namespace mb {

__device__ __forceinline__ void two_sum(double x, double y, double& s, double& e) {   // comp.jl:51-56
    s = __dadd_rn(x, y);
    const double xp = __dsub_rn(s, y);
    const double yp = __dsub_rn(s, xp);
    e = __dadd_rn(__dsub_rn(x, xp), __dsub_rn(y, yp));
}

__device__ __forceinline__ void two_mul(double x, double y, double& p, double& e) {   // comp.jl:58-61
    p = __dmul_rn(x, y);
    e = fma(x, y, -p);
}

// (s, cs) += a x  (twoaxpy!, comp.jl:75-84)
__device__ __forceinline__ void two_axpy(double& s, double& cs, double a, double x) {
    double p, ep, sg, es;
    two_mul(a, x, p, ep);
    two_sum(s, p, sg, es);
    s = sg;
    cs = __dadd_rn(cs, __dadd_rn(ep, es));
}

// (Δ, δ) += a x  (twoacc, comp.jl:68-72)
__device__ __forceinline__ void two_acc(double& D, double& d, double a, double x) {
    double p, ep, es;
    two_mul(a, x, p, ep);
    two_sum(D, p, D, es);
    d = __dadd_rn(d, __dadd_rn(ep, es));
}

// (s, cs) += (Δ, δ)  (twofold!, comp.jl:86-94)
__device__ __forceinline__ void two_fold(double& s, double& cs, double D, double d) {
    double sg, e;
    two_sum(s, D, sg, e);
    s = sg;
    cs = __dadd_rn(cs, __dadd_rn(d, e));
}

// The epilogue c ← α (s + cs) + β c of extaxpby! (pair = false, comp.jl:107-170) or twoaxpby!
// (pair = true, comp.jl:183-248).  bcls: 0 β = 0, 1 β = 1, 2 β = -1, 3 otherwise; acls: 1 α = 1,
// 2 α = -1, 0 otherwise (β = 0 has no α = -1 branch in the reference).
__device__ __forceinline__ void epilogue(double s, double cs, double alpha, double beta, int acls, int bcls,
                                         bool pair, double* c, double* cc, int64_t i) {
    double hi, tail;   // c = hi + tail (folded) or (c, cc) = two_sum(hi, tail)
    if (bcls == 0) {
        if (acls == 1) {
            hi = s; tail = cs;
        } else {
            double p, ep;
            two_mul(alpha, s, p, ep);
            hi = p; tail = fma(alpha, cs, ep);
        }
    } else if (bcls == 1 || bcls == 2) {
        const double ci = bcls == 1 ? c[i] : -c[i];
        double sg, es;
        if (acls == 1) {
            two_sum(ci, s, sg, es);
            hi = sg; tail = __dadd_rn(cs, es);
        } else if (acls == 2) {
            two_sum(ci, -s, sg, es);
            hi = sg; tail = __dsub_rn(es, cs);
        } else {
            double p, ep;
            two_mul(alpha, s, p, ep);
            two_sum(ci, p, sg, es);
            hi = sg; tail = __dadd_rn(fma(alpha, cs, ep), es);
        }
    } else {
        double p1, e1, p2, e2, sg, e3;
        two_mul(alpha, s, p1, e1);
        two_mul(beta, c[i], p2, e2);
        two_sum(p1, p2, sg, e3);
        hi = sg; tail = __dadd_rn(__dadd_rn(fma(alpha, cs, e1), e2), e3);
    }
    if (pair) {
        double a, b;
        two_sum(hi, tail, a, b);
        c[i] = a; cc[i] = b;
    } else {
        c[i] = __dadd_rn(hi, tail);
    }
}

// One output per thread.  N: ptr/idx/val is the CSR of the stored entries (columns ascending);
// T: the CSC (rows ascending), brk[k] = 1 where entry k opens a block of its column, 2 where that
// block is 1 x 1.
__global__ void __launch_bounds__(256) twomv_kernel(TwoMv a) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nout) return;
    const int64_t k0 = a.ptr[r], k1 = a.ptr[r + 1];
    double s = 0.0, cs = 0.0;
    if (!a.trans) {
        for (int64_t k = k0; k < k1; ++k) two_axpy(s, cs, a.val[k], a.b[a.idx[k]]);
    } else {
        double D = 0.0, d = 0.0;
        bool open = false;
        for (int64_t k = k0; k < k1; ++k) {
            const int f = a.brk[k];
            if (f) {
                if (open) two_fold(s, cs, D, d);
                open = false; D = 0.0; d = 0.0;
            }
            if (f == 2) {
                two_axpy(s, cs, a.val[k], a.b[a.idx[k]]);
            } else {
                two_acc(D, d, a.val[k], a.b[a.idx[k]]);
                open = true;
            }
        }
        if (open) two_fold(s, cs, D, d);
    }
    if (a.s) { a.s[r] = s; a.cs[r] = cs; }
    epilogue(s, cs, a.alpha, a.beta, a.acls, a.bcls, a.cc != nullptr, a.c, a.cc, r);
}

}  // namespace mb

extern "C" int mb_launch_twomv(const mb::TwoMv* a, cudaStream_t st) {
    if (a->nout <= 0) return (int)cudaSuccess;
    const int64_t nb = (a->nout + 255) / 256;
    mb::twomv_kernel<<<(unsigned)nb, 256, 0, st>>>(*a);
    return (int)cudaGetLastError();
}
