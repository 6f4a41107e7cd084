// Block-cooperative device building blocks of the batched IPM solver: reductions, vector
// kernels and block-sparse matrix-vector products.  Every function is called by all NT threads
// of a CTA and ends with a barrier unless stated otherwise; reductions use a fixed tree so the
// result is bit-reproducible and independent of what other CTAs are doing.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "mb_internal.h"

namespace mb {

constexpr int NT = CTA_THREADS;  // threads per CTA
constexpr int NW = NT / 32;      // warps per CTA

struct Shared;                   // defined in mb_solver.cu

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
// NaN-propagating min (Julia semantics for `min`/`minimum` on floats)
__device__ __forceinline__ double jmin(double a, double b) {
    return (a != a || b != b) ? __longlong_as_double(0x7ff8000000000000LL) : (b < a ? b : a);
}
__device__ __forceinline__ double jmax(double a, double b) {
    return (a != a || b != b) ? __longlong_as_double(0x7ff8000000000000LL) : (b > a ? b : a);
}
__device__ __forceinline__ double warp_jmin(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = jmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// error-free transforms (IPM/src/utils.jl:27-38)
__device__ __forceinline__ void twosum(double a, double b, double& s, double& e) {
    s = a + b;
    double bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}
__device__ __forceinline__ void twoprod(double a, double b, double& p, double& e) {
    p = a * b;
    e = fma(a, b, -p);
}
// combine two compensated partial sums
__device__ __forceinline__ void cadd(double& s, double& c, double s2, double c2) {
    double t, e;
    twosum(s, s2, t, e);
    s = t;
    c = c + c2 + e;
}
__device__ __forceinline__ void warp_csum(double& s, double& c) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double s2 = __shfl_xor_sync(0xffffffffu, s, o);
        double c2 = __shfl_xor_sync(0xffffffffu, c, o);
        // combine in a lane-order independent way: the lower lane's value first
        int lane = threadIdx.x & 31;
        if (lane & o) { double ts = s, tc = c; s = s2; c = c2; s2 = ts; c2 = tc; }
        cadd(s, c, s2, c2);
    }
}

// Block reduction scratch lives in Shared::red (NW + 2 doubles).
template <class Op>
__device__ __forceinline__ double block_reduce(double v, double* red, Op op, double init) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double t = lane < NW ? red[lane] : init;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t = op(t, __shfl_xor_sync(0xffffffffu, t, o));
        if (lane == 0) red[NW] = t;
    }
    __syncthreads();
    double r = red[NW];
    __syncthreads();
    return r;
}
struct OpSum { __device__ double operator()(double a, double b) const { return a + b; } };
struct OpMax { __device__ double operator()(double a, double b) const { return fmax(a, b); } };
struct OpJmin { __device__ double operator()(double a, double b) const { return jmin(a, b); } };
struct OpMin { __device__ double operator()(double a, double b) const { return fmin(a, b); } };

__device__ __forceinline__ double bdot(const double* x, const double* y, int n, double* red) {
    double s = 0;
    for (int i = threadIdx.x; i < n; i += NT) s += x[i] * y[i];
    return block_reduce(s, red, OpSum(), 0.0);
}
__device__ __forceinline__ double bnorm(const double* x, int n, double* red) {
    return sqrt(bdot(x, x, n, red));
}
// ‖v ./ s‖  (ipm/solver/utils.jl:11-19 scalenorm)
__device__ __forceinline__ double bscalenorm(const double* v, const double* s, int n, double* red) {
    double a = 0;
    for (int i = threadIdx.x; i < n; i += NT) { double t = v[i] / s[i]; a += t * t; }
    return sqrt(block_reduce(a, red, OpSum(), 0.0));
}

__device__ __forceinline__ void bcopy(double* y, const double* x, int n) {
    for (int i = threadIdx.x; i < n; i += NT) y[i] = x[i];
    __syncthreads();
}
__device__ __forceinline__ void bfill(double* y, double a, int n) {
    for (int i = threadIdx.x; i < n; i += NT) y[i] = a;
    __syncthreads();
}
// y += a x
__device__ __forceinline__ void baxpy(double a, const double* x, double* y, int n) {
    for (int i = threadIdx.x; i < n; i += NT) y[i] = fma(a, x[i], y[i]);
    __syncthreads();
}

// Sparse products over the nonzeros of a block-sparse matrix (BlockSparseArrays/src/blas/gemv.jl:
// 321-343 computes the same sums over the dense blocks; their explicit zeros add nothing).  A thread
// owns a row (CSR) or column (CSC) of at most LONG_ROW entries, a warp a longer one; each sum runs
// in a fixed order.
constexpr int G = 16;

template <class Op>
__device__ __forceinline__ double group_reduce(double v, Op op) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(0xffffffffu, v, o, G));
    return v;
}

// Groups of G lanes (equilibration's row and column maxima).  The loop bound is uniform per warp
// (both groups of a warp enter group_reduce together).
constexpr int GPW = 32 / G;   // groups per warp

// y <- alpha A x + beta y: a thread per row of at most LONG_ROW entries, a warp per longer row
// (A.longr, listed by the host); each row is summed in a fixed order.
__device__ void spmv(const DevSp& A, const double* x, double* y, double alpha, double beta) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < A.nrow; i += NT) {
        const int k0 = A.rptr[i], k1 = A.rptr[i + 1];
        if (k1 - k0 > LONG_ROW) continue;
        double acc = 0;
        for (int k = k0; k < k1; ++k) acc = fma(A.val[k], x[A.cidx[k]], acc);
        y[i] = beta == 0.0 ? alpha * acc : fma(alpha, acc, beta * y[i]);
    }
    for (int t = warp; t < A.nlongr; t += NW) {
        const int i = A.longr[t];
        double acc = 0;
        for (int k = A.rptr[i] + lane; k < A.rptr[i + 1]; k += 32) acc = fma(A.val[k], x[A.cidx[k]], acc);
        acc = warp_sum(acc);
        if (lane == 0) y[i] = beta == 0.0 ? alpha * acc : fma(alpha, acc, beta * y[i]);
    }
    __syncthreads();
}

// y <- alpha Aᵀ x + beta y, by columns of A the same way (A.longc)
__device__ void spmvT(const DevSp& A, const double* x, double* y, double alpha, double beta) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int j = threadIdx.x; j < A.ncol; j += NT) {
        const int k0 = A.cptr[j], k1 = A.cptr[j + 1];
        if (k1 - k0 > LONG_ROW) continue;
        double acc = 0;
        for (int k = k0; k < k1; ++k) acc = fma(A.val[A.cpos[k]], x[A.ridx[k]], acc);
        y[j] = beta == 0.0 ? alpha * acc : fma(alpha, acc, beta * y[j]);
    }
    for (int t = warp; t < A.nlongc; t += NW) {
        const int j = A.longc[t];
        double acc = 0;
        for (int k = A.cptr[j] + lane; k < A.cptr[j + 1]; k += 32) acc = fma(A.val[A.cpos[k]], x[A.ridx[k]], acc);
        acc = warp_sum(acc);
        if (lane == 0) y[j] = beta == 0.0 ? alpha * acc : fma(alpha, acc, beta * y[j]);
    }
    __syncthreads();
}

// dot(x, A, y)  (block_sparse_matrix.jl:1094-1109)
__device__ double spdot(const DevSp& A, const double* x, const double* y, double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double s = 0;
    for (int i = threadIdx.x; i < A.nrow; i += NT) {
        const int k0 = A.rptr[i], k1 = A.rptr[i + 1];
        if (k1 - k0 > LONG_ROW) continue;
        double acc = 0;
        for (int k = k0; k < k1; ++k) acc = fma(A.val[k], y[A.cidx[k]], acc);
        s = fma(x[i], acc, s);
    }
    for (int t = warp; t < A.nlongr; t += NW) {
        const int i = A.longr[t];
        double acc = 0;
        for (int k = A.rptr[i] + lane; k < A.rptr[i + 1]; k += 32) acc = fma(A.val[k], y[A.cidx[k]], acc);
        acc = warp_sum(acc);
        if (lane == 0) s = fma(x[i], acc, s);
    }
    return block_reduce(s, red, OpSum(), 0.0);
}

}  // namespace mb
