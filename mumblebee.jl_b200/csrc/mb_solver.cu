// Batched device-resident interior-point solver for sm_100a.
//
// One CTA runs one complete solve of Mumblebee.jl's predictor–corrector IPM
// (src/IPM/src/ipm/solver/ipm.jl:577-774) on one problem instance that lives in HBM: Ruiz
// equilibration, BᵀB assembly into multifrontal front storage, NT/cone scaling, the Uzawa
// iterative refinement + CG KKT solves over a supernodal Cholesky factor, step to the boundary,
// termination tests and the δ augmentation schedule.  A persistent grid pulls instance indices
// from a device work counter, so instances of any size mix in one launch and a finished CTA
// immediately starts the next instance (continuous batching); nothing a CTA computes depends on
// which other instances share the launch.
//
// Precision: iterates, residuals, refinement, cone algebra and termination checks are FP64.  The
// KKT factor is stored and computed in FT (double, or float for the mixed-precision path).
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include "mb_internal.h"

// MB_TC = 1 builds the tensor-core variant of the solver kernels (mb_solver_tc.cu): the FP32
// factor's update tiles on tcgen05.  A kernel that contains tcgen05 instructions runs one CTA per
// SM (measured on B200: the occupancy calculator and the scheduler both drop from two to one), so
// the default build, whose batched FP64 path needs two resident instances per SM to hide latency,
// carries none; its extern "C" entry points get the suffix _tc in the variant.
#ifndef MB_TC
#define MB_TC 0
#endif
#if MB_TC
#define MB_SFX(name) name##_tc
#else
#define MB_SFX(name) name
#endif
#include "mb_device.cuh"
#include "mb_cones.cuh"
#include "mb_tdc.cuh"
#include "mb_sdp.cuh"

namespace mb {

constexpr int TS = 64;   // trailing-update tile
constexpr double MIXED_MAX_SOLVES = 4;   // KKT solves (IR passes + CG steps) an FP32 iteration may take
constexpr int TLD = 36;  // sizes Shared::tile: four 64 x 36 double tiles (FP64, FP32 and tensor-core stages fit in it)

// Block-shared scratch (dynamic shared memory: it exceeds the 48 KB static limit).  `tile` holds the
// two stages (A and B operand each) of the double-buffered front update.
struct Shared {
    double red[NW + 2];
    double diag[32 * 33];
    double dinv[32];        // 1 / L[c][c] of the diagonal block in sh.diag
    double col[32];         // one column of the diagonal block being factored
    double xs[32];
    double acc[32];
    double tile[4 * TS * TLD];   // stage 0 A, B, stage 1 A, B of the front update; x slices in solves
    int flag;
    int ibuf[8];
    long long wait_ns;      // grid-cooperative mode: longest wait at a grid barrier
    unsigned long long mbar[2];   // tensor-core update: completion of the MMAs that read stage 0 / 1
    unsigned int tmem;      // tensor-core update: base address of the CTA's accumulator columns
    unsigned int tc_ph;     // tensor-core update: parity of the next wait on mbar[b] at bit b
    int tc_on;              // FP32 update tiles on the tensor cores: TMEM held, barriers set up
    int tc_ok;              // tensor-core update: 0 once a completion wait ran out
    int* tc_err;            // set to 2 when a completion wait runs out (instance status word 7, or the
                            // grid-cooperative abort flag on a helper CTA)
};
static_assert(offsetof(Shared, tile) % 16 == 0, "16-byte copies stage into Shared::tile");

// D += A·B on the FP64 tensor path (mma.m8n8k4, fragments: A[g][t], B[t][g], C[g][2t+i] with
// g = lane/4, t = lane%4)
__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1) : "d"(a), "d"(b));
}

// Factor the kb x kb diagonal block at k0 in shared memory (sh.diag, S[r * 33 + c] = L[k0 + r][k0 + c]),
// all warps: per column the pivot's square root and reciprocal (every thread computes the same),
// the column scaled by the reciprocal, then the trailing triangle's rank-1 update, two barriers per
// column.  Each entry takes its updates in increasing column order, as a row held in registers
// would, with the same fused forms.  The factor is left in sh.diag, with 1 / L[c][c] in sh.dinv for
// the panel, and written back to M; its inverse goes to the block's upper triangle for the
// triangular solves.  Returns the failing pivot (1-based in the front) or 0.
template <class FT>
__device__ __noinline__ int diag_factor(FT* M, int nf, int k0, int kb, Shared& sh) {
    const int64_t ld = front_ld(nf);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    FT* S = reinterpret_cast<FT*>(sh.diag);
    FT* dinv = reinterpret_cast<FT*>(sh.dinv);
    for (int t = tid; t < 32 * 32; t += NT) {
        const int r = t & 31, c = t >> 5;
        if (r < kb && c <= r) S[r * 33 + c] = M[(k0 + r) + (int64_t)(k0 + c) * ld];
    }
    __syncthreads();
    int fail = 0;
    for (int c = 0; c < kb; ++c) {
        const FT dd = S[c * 33 + c];
        if (!(dd > FT(0))) { fail = c + 1; break; }
        const FT dc = sqrt(dd);
        const FT r = FT(1) / dc;
        if (tid == c) { S[c * 33 + c] = dc; dinv[c] = r; }
        else if (tid > c && tid < kb) S[tid * 33 + c] = S[tid * 33 + c] * r;   // L[tid][c]
        __syncthreads();
        for (int t = tid; t < 32 * 32; t += NT) {
            const int i = t & 31, j = t >> 5;
            if (j > c && i >= j && i < kb) S[i * 33 + j] -= S[i * 33 + c] * S[j * 33 + c];
        }
        __syncthreads();
    }
    if (!fail) {
        for (int t = tid; t < 32 * 32; t += NT) {
            const int r = t & 31, c = t >> 5;
            if (r < kb && c <= r) M[(k0 + r) + (int64_t)(k0 + c) * ld] = S[r * 33 + c];
        }
    }
    if (tid == 0) sh.flag = fail ? k0 + fail : 0;
    __syncthreads();
    const int flag = sh.flag;
    if (warp == 1 && !flag) {
        // X = L⁻¹ for the triangular solves, on warp 1 while the others go on to the panel rows: lane c
        // forms column c of X by forward substitution in axpy order (X[k][c] = −(Σ_{j<k} L[k][j] X[j][c])
        // / L[k][k], times the reciprocal pivot) and stores X[k][c], k > c, transposed into the block's
        // upper triangle, M[k0 + c, k0 + k], which nothing else reads; X[c][c] = 1 / L[c][c] is not stored.
        // The next barrier (the end of the panel rows) orders it before sh.diag is overwritten.
        const int c = lane;
        FT acc[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) acc[i] = FT(0);
#pragma unroll
        for (int k = 0; k < 32; ++k) {
            if (k >= kb) continue;
            const FT xk = k < c ? FT(0) : (k == c ? dinv[c] : -acc[k] * dinv[k]);
            if (k > c && c < kb) M[(k0 + c) + (int64_t)(k0 + k) * ld] = xk;
#pragma unroll
            for (int i = k + 1; i < 32; ++i) acc[i] = fma(S[i * 33 + k], xk, acc[i]);
        }
    }
    return flag;
}

// The inverses of the 32 x 32 diagonal blocks of a front whose residual columns already hold L
// (the stable factor writes L directly): the layout diag_factor leaves, a warp per block, lane c
// forming column c of X = L⁻¹ in the same axpy order and storing X[k][c], k > c, at M[k0 + c, k0 + k].
__device__ __noinline__ void front_block_inverses(double* M, int nf, int nres) {
    const int64_t ld = front_ld(nf);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int b = warp; b * 32 < nres; b += NW) {
        const int k0 = b * 32, kb = min(32, nres - k0), c = lane;
        double acc[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) acc[i] = 0.0;
#pragma unroll
        for (int k = 0; k < 32; ++k) {
            if (k >= kb) continue;
            const double dk = 1.0 / M[(k0 + k) + (int64_t)(k0 + k) * ld];
            const double xk = k < c ? 0.0 : (k == c ? dk : -acc[k] * dk);
            if (k > c && c < kb) M[(k0 + c) + (int64_t)(k0 + k) * ld] = xk;
#pragma unroll
            for (int i = k + 1; i < 32; ++i)
                if (i < kb) acc[i] = fma(M[(k0 + i) + (int64_t)(k0 + k) * ld], xk, acc[i]);
        }
    }
    __syncthreads();
}

// The stable factor's blocked Householder step: apply the reflectors of panel columns
// [j0, j0 + np) to the trailing columns [j0 + np, nfr) of the column-major W (leading dimension
// ld).  Reflector p lives on row j0 + p and rows [lo, lo + cnt - 1); its values are staged at
// vs[p * cnt + t] (t = 0: the row j0 + p entry) and cf[p] is its scale (0: no reflection).  A warp
// holds one trailing column in registers (rows [lo, ..) across the lanes as the unblocked loop
// indexes them, the panel rows one per lane), applies the np reflectors in order with the same
// per-lane accumulation, butterfly reduction and fused forms as applying them one at a time, and
// stores the column once: the same values, with the trailing block read and written once per
// panel instead of once per column.
constexpr int QR_PANEL = 16;   // reflectors per panel
constexpr int QR_SEG = 16;     // register slots per lane: supports of up to 32 * QR_SEG values
__device__ __noinline__ void qr_apply_panel(double* W, int64_t ld, int nfr, int j0, int np, int lo, int cnt,
                                            const double* vs, const double* cf) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // two columns per warp (k and k + NW): their reflector chains are independent and interleave
    for (int k = j0 + np + warp; k < nfr; k += 2 * NW) {
        const bool two = k + NW < nfr;
        double* wk = W + (int64_t)k * ld;
        double* wl = W + (int64_t)(two ? k + NW : k) * ld;
        double x[QR_SEG], y[QR_SEG];
#pragma unroll
        for (int r = 0; r < QR_SEG; ++r) {
            const int t = lane + 32 * r;
            const bool in = t >= 1 && t < cnt;
            x[r] = in ? wk[lo + t - 1] : 0.0;
            y[r] = in ? wl[lo + t - 1] : 0.0;
        }
        double h = lane < np ? wk[j0 + lane] : 0.0;   // lane p: row j0 + p
        double g = lane < np ? wl[j0 + lane] : 0.0;
        for (int p = 0; p < np; ++p) {
            const double c = cf[p];
            if (c == 0.0) continue;
            const double* v = vs + (int64_t)p * cnt;
            const double h0 = __shfl_sync(0xffffffffu, h, p);
            const double g0 = __shfl_sync(0xffffffffu, g, p);
            if (lane == 0) { x[0] = h0; y[0] = g0; }   // slot t = 0 is row j0 + p
            double dt = 0.0, du = 0.0;
#pragma unroll
            for (int r = 0; r < QR_SEG; ++r) {
                const int t = lane + 32 * r;
                if (t < cnt) { dt += v[t] * x[r]; du += v[t] * y[r]; }
            }
            dt = warp_sum(dt) * c;
            du = warp_sum(du) * c;
#pragma unroll
            for (int r = 0; r < QR_SEG; ++r) {
                const int t = lane + 32 * r;
                if (t < cnt) { x[r] -= dt * v[t]; y[r] -= du * v[t]; }
            }
            const double hn = __shfl_sync(0xffffffffu, x[0], 0);
            const double gn = __shfl_sync(0xffffffffu, y[0], 0);
            if (lane == p) { h = hn; g = gn; }
        }
#pragma unroll
        for (int r = 0; r < QR_SEG; ++r) {
            const int t = lane + 32 * r;
            if (t >= 1 && t < cnt) {
                wk[lo + t - 1] = x[r];
                if (two) wl[lo + t - 1] = y[r];
            }
        }
        if (lane < np) {
            wk[j0 + lane] = h;
            if (two) wl[j0 + lane] = g;
        }
    }
    __syncthreads();
}

// Panel solve L21 = A21 L11^{-T} for the rows [k0 + kb, nf) owned by this rank (row blocks of NT
// rows dealt round-robin over nranks CTAs), multiplying by the reciprocal pivots.  With `load`, the
// factored diagonal block is first read back from M into sh.diag (a helper CTA that did not
// factor it) and its reciprocal pivots recomputed.  Each block of NT rows is first staged into
// shared memory by cp.async, all 32 columns in flight at once; a thread then solves its row in
// column (axpy) order, so the updates after each pivot are independent of one another, while every
// entry still takes its terms in increasing column order, as the row's dot products would.
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc, int bytes) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);   // bytes < 16: the rest zero-filled
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gsrc), "r"(bytes) : "memory");
}

template <class FT>
__device__ __forceinline__ void cp_async_ft(FT* sdst, const FT* gsrc, bool valid) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    if constexpr (sizeof(FT) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gsrc), "r"(valid ? 8 : 0) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(gsrc), "r"(valid ? 4 : 0) : "memory");
}
template <class FT>
__device__ __noinline__ void panel_rows(FT* M, int nf, int k0, int kb, Shared& sh, int rank, int nranks, bool load) {
    const int64_t ld = front_ld(nf);
    const int tid = threadIdx.x;
    FT* S = reinterpret_cast<FT*>(sh.diag);
    FT* dinv = reinterpret_cast<FT*>(sh.dinv);
    if (load) {
        for (int t = tid; t < 32 * 32; t += NT) {
            const int r = t & 31, c = t >> 5;
            if (r < kb && c <= r) S[r * 33 + c] = M[(k0 + r) + (int64_t)(k0 + c) * ld];
        }
        __syncthreads();
        if (tid < kb) dinv[tid] = FT(1) / S[tid * 33 + tid];   // as diag_factor computes it
        __syncthreads();
    }
    // staged rows: T[c * LD + sft + r], r < NT.  FP64 blocks come in 16-byte copies of row pairs
    // (LD even keeps each staged column 16-byte aligned); pairs start at even rows, so a block that
    // starts at an odd row is staged from the row before, sft = 1, with a 129th pair per column
    constexpr int LD = sizeof(FT) == 8 ? NT + 2 : NT + 1, NP = NT / 2;
    static_assert(32 * LD * 8 <= (int)sizeof(double) * 4 * TS * TLD, "a staged row block fits in Shared::tile");
    FT* T = reinterpret_cast<FT*>(sh.tile);
    const int j0 = k0 + kb;
    for (int base = j0 + rank * NT; base < nf; base += NT * nranks) {
        int sft = 0;
        if constexpr (sizeof(FT) == 8) {
            sft = base & 1;
            const int b0 = base - sft;
            for (int idx = tid; idx < 32 * NP + 32 * sft; idx += NT) {
                const bool last = idx >= 32 * NP;
                const int c = last ? idx - 32 * NP : idx / NP, u = last ? NP : idx % NP, gr = b0 + 2 * u;
                const int nv = c < kb ? min(2, max(0, nf - gr)) : 0;
                cp_async16(T + c * LD + 2 * u, nv ? M + gr + (int64_t)(k0 + c) * ld : M, 8 * nv);
            }
        } else {
            for (int idx = tid; idx < 32 * NT; idx += NT) {
                const int c = idx / NT, r = idx - c * NT, row = base + r;
                const bool v = row < nf && c < kb;
                cp_async_ft<FT>(T + c * LD + r, v ? M + row + (int64_t)(k0 + c) * ld : M, v);
            }
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        __syncthreads();
        const int i = base + tid;
        if (i < nf) {
            FT x[32];
#pragma unroll
            for (int c = 0; c < 32; ++c) x[c] = T[c * LD + sft + tid];
#pragma unroll
            for (int cc = 0; cc < 32; ++cc) {
                if (cc < kb) {
                    x[cc] = x[cc] * dinv[cc];
#pragma unroll
                    for (int c = cc + 1; c < 32; ++c) x[c] -= x[cc] * S[c * 33 + cc];
                }
            }
            FT* wp = M + i + (int64_t)k0 * ld;
#pragma unroll
            for (int c = 0; c < 32; ++c) if (c < kb) wp[(int64_t)c * ld] = x[c];
        }
        __syncthreads();                       // the block is read before the next one is staged
    }
}

// ---- FP64 left-looking front factorization ---------------------------------------------------
__device__ __forceinline__ void cp_async8(void* sdst, const void* gsrc, bool valid) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    const int sz = valid ? 8 : 0;   // 0: write zeros, read nothing
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gsrc), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Stage rows [r0, r0 + 64) x columns [k0, k0 + 32) of the column-major front M (16-byte aligned,
// even leading dimension ld) into buf column by column: row r of column c at
// buf[c * CLD + (r0 & 1) + r - r0], zero where the row is >= rmax or the column >= kmax.  16-byte
// copies of row pairs, which start on a 16-byte boundary at even rows: a warp copies one column's
// 64 rows (512 contiguous bytes) per instruction; for an odd r0 the pairs start one row early and
// lane 0 copies a 33rd pair.
constexpr int CLD = 68;   // staged column stride (doubles): fragment loads of 8 rows x 4 columns hit 32 distinct banks
static_assert(4 * 32 * CLD <= 4 * TS * TLD, "four staged tiles fit in Shared::tile");
__device__ __forceinline__ void stage_tile_f64(double* buf, const double* M, int64_t ld, int r0, int rmax, int k0,
                                               int kmax) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int p = r0 & 1, base = r0 - p;
    for (int c = warp; c < 32; c += NW) {
        const int gc = k0 + c;
        for (int u = lane; u < 32 + p; u += 32) {
            const int gr = base + 2 * u;
            const int nv = gc < kmax ? min(2, max(0, rmax - gr)) : 0;
            cp_async16(buf + c * CLD + 2 * u, nv ? M + gr + (int64_t)gc * ld : M, 8 * nv);
        }
    }
}

// One 64 x nb tile of the trailing update: rows [rb, rb + 64) x columns [J, J + nb) (nb <= 64) of
// the column-major front M (order nf), M[r, c] -= Σ_{k in [K0, K1)} M[r, k] M[c, k] for
// r >= c.  The K columns must be final (K1 <= J).
struct UTile { int rb, J, nb; };

// The tiles one CTA updates, in order, and the K range they share.  Every tile takes
// nk = ceil((K1 - K0) / 32) chunks; the (tile, chunk) sequence is one software pipeline: the copy
// of the next chunk (of this tile or the next one) is in flight while the current chunk is on the
// tensor pipe, so a tile costs no prologue of its own.  The accumulators start from the tile's
// current values of M (loaded while the first chunk's copy is in flight) and take the update
// with negated B fragments, so the epilogue is a plain store.
template <class TileAt>
__device__ __noinline__ void tiles_f64(double* M, int nf, int ntile, int K0, int K1, Shared& sh, TileAt at) {
    const int64_t ld = front_ld(nf);
    constexpr int WRN = NW / 4, RW = TS / WRN, MR = RW / 8;
    if (ntile <= 0 || K1 <= K0) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wr = warp >> 2, wc = warp & 3;
    const int nk = (K1 - K0 + 31) / 32;
    const int nstep = ntile * nk;
    double* A[2] = {sh.tile, sh.tile + 2 * 32 * CLD};
    double* B[2] = {sh.tile + 32 * CLD, sh.tile + 3 * 32 * CLD};
    auto stage = [&](int s, int buf) {
        const UTile u = at(s / nk);
        const int k0 = K0 + 32 * (s % nk);
        stage_tile_f64(A[buf], M, ld, u.rb, nf, k0, K1);
        stage_tile_f64(B[buf], M, ld, u.J, min(nf, u.J + u.nb), k0, K1);
        cp_async_commit();
    };
    double acc[MR][2][2];
    UTile u = at(0);
    bool skip = false;
    stage(0, 0);
    for (int s = 0; s < nstep; ++s) {
        const int q = s % nk, cur = s & 1;
        if (q == 0) {
            u = at(s / nk);
            skip = wc * 16 >= u.nb || (u.rb == u.J && wr * RW + RW - 1 < wc * 16);
            const int cmax = min(nf, u.J + u.nb);
#pragma unroll
            for (int a = 0; a < MR; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b)
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const int row = u.rb + wr * RW + a * 8 + g;
                        const int col = u.J + wc * 16 + b * 8 + 2 * t + e;
                        acc[a][b][e] = (!skip && row < nf && col < cmax && row >= col) ? M[row + (int64_t)col * ld] : 0.0;
                    }
        }
        if (s + 1 < nstep) {
            stage(s + 1, cur ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        if (!skip) {
            const double* ta = A[cur] + (u.rb & 1) + wr * RW + g + t * CLD;
            const double* tb = B[cur] + (u.J & 1) + wc * 16 + g + t * CLD;
            const int kb4 = (min(32, K1 - K0 - 32 * q) + 3) & ~3;
            for (int k = 0; k < kb4; k += 4) {
                const double b0 = -tb[k * CLD], b1 = -tb[k * CLD + 8];
#pragma unroll
                for (int a = 0; a < MR; ++a) {
                    const double av = ta[k * CLD + a * 8];
                    dmma(acc[a][0][0], acc[a][0][1], av, b0);
                    dmma(acc[a][1][0], acc[a][1][1], av, b1);
                }
            }
        }
        __syncthreads();
        if (q == nk - 1 && !skip) {
            const int cmax = min(nf, u.J + u.nb);
#pragma unroll
            for (int a = 0; a < MR; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b)
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const int row = u.rb + wr * RW + a * 8 + g;
                        const int col = u.J + wc * 16 + b * 8 + 2 * t + e;
                        if (row < nf && col < cmax && row >= col) M[row + (int64_t)col * ld] = acc[a][b][e];
                    }
        }
    }
    __syncthreads();
}

// M[r, c] -= Σ_{k in [K0, K1)} M[r, k] M[c, k] for c in [J0, J0 + nb) (nb <= 64), r in [J0, nf),
// r >= c: the 64-row tiles from J0 down, dealt round-robin over nranks CTAs.  Requires K1 <= J0.
__device__ void update_cols_f64(double* M, int nf, int J0, int nb, int K0, int K1, Shared& sh, int rank = 0,
                                int nranks = 1) {
    if (K1 <= K0 || nb <= 0) return;
    const int first = J0 + TS * rank, step = TS * nranks;
    const int ntile = first < nf ? (nf - first + step - 1) / step : 0;
    tiles_f64(M, nf, ntile, K0, K1, sh, [=](int i) { return UTile{first + step * i, J0, nb}; });
    __syncthreads();
}

__device__ __forceinline__ void cp_async4(void* sdst, const void* gsrc, bool valid) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    const int sz = valid ? 4 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(gsrc), "r"(sz) : "memory");
}

// FP32 stage: rows [r0, r0 + 64) x columns [k0, k0 + 32) of M as buf[c * 68 + r] (k-major, so a
// thread reads its 4 rows as one float4), zero where the row is >= rmax or the column >= kmax
constexpr int T32LD = 68;
__device__ __forceinline__ void stage_tile_f32(float* buf, const float* M, int64_t ld, int r0, int rmax, int k0, int kmax) {
    for (int i = threadIdx.x; i < 64 * 32; i += NT) {
        const int r = i & 63, c = i >> 6;
        const int gr = r0 + r, gc = k0 + c;
        const bool v = gr < rmax && gc < kmax;
        cp_async4(buf + c * T32LD + r, v ? M + gr + (int64_t)gc * ld : M, v);
    }
}

// FP32 twin of tiles_f64: each thread owns a 4 x 4 block of the 64 x 64 tile (FFMA), same
// cross-tile pipeline, accumulators started from M
template <class TileAt>
__device__ __noinline__ void tiles_f32(float* M, int nf, int ntile, int K0, int K1, Shared& sh, TileAt at) {
    const int64_t ld = front_ld(nf);
    if (ntile <= 0 || K1 <= K0) return;
    const int tr = threadIdx.x & 15, tc = threadIdx.x >> 4;
    const int nk = (K1 - K0 + 31) / 32;
    const int nstep = ntile * nk;
    float* A[2] = {reinterpret_cast<float*>(sh.tile), reinterpret_cast<float*>(sh.tile + 2 * TS * TLD)};
    float* B[2] = {reinterpret_cast<float*>(sh.tile + TS * TLD), reinterpret_cast<float*>(sh.tile + 3 * TS * TLD)};
    auto stage = [&](int s, int buf) {
        const UTile u = at(s / nk);
        const int k0 = K0 + 32 * (s % nk);
        stage_tile_f32(A[buf], M, ld, u.rb, nf, k0, K1);
        stage_tile_f32(B[buf], M, ld, u.J, min(nf, u.J + u.nb), k0, K1);
        cp_async_commit();
    };
    float acc[4][4];
    UTile u = at(0);
    bool skip = false;
    stage(0, 0);
    for (int s = 0; s < nstep; ++s) {
        const int q = s % nk, cur = s & 1;
        if (q == 0) {
            u = at(s / nk);
            skip = tc * 4 >= u.nb || (u.rb == u.J && tr * 4 + 3 < tc * 4);
            const int cmax = min(nf, u.J + u.nb);
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const int row = u.rb + tr * 4 + a, col = u.J + tc * 4 + b;
                    acc[a][b] = (!skip && row < nf && col < cmax && row >= col) ? M[row + (int64_t)col * ld] : 0.f;
                }
        }
        if (s + 1 < nstep) {
            stage(s + 1, cur ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        if (!skip) {
            const float* ta = A[cur];
            const float* tb = B[cur];
            const int kb = min(32, K1 - K0 - 32 * q);
            for (int k = 0; k < kb; ++k) {
                const float4 av = *reinterpret_cast<const float4*>(ta + k * T32LD + tr * 4);
                const float4 bv = *reinterpret_cast<const float4*>(tb + k * T32LD + tc * 4);
                const float ar[4] = {av.x, av.y, av.z, av.w}, br[4] = {-bv.x, -bv.y, -bv.z, -bv.w};
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) acc[a][b] = fmaf(ar[a], br[b], acc[a][b]);
            }
        }
        __syncthreads();
        if (q == nk - 1 && !skip) {
            const int cmax = min(nf, u.J + u.nb);
#pragma unroll
            for (int b = 0; b < 4; ++b)
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    const int row = u.rb + tr * 4 + a, col = u.J + tc * 4 + b;
                    if (row < nf && col < cmax && row >= col) M[row + (int64_t)col * ld] = acc[a][b];
                }
        }
    }
    __syncthreads();
}

#if MB_TC
// ---- FP32 update tiles on the 5th-generation tensor cores (tcgen05.mma kind::tf32) -----------
// 3xTF32: a = ah + al with ah = a rounded to TF32 and al = the rest rounded to TF32; a·b is taken
// as al·bh + ah·bl + ah·bh (al·bl lies below FP32 rounding).  The tensor cores accumulate one
// 16-column K step of these products in FP32 in tensor memory (two 128 x 64 accumulators, 128 TMEM
// columns, lane = tile row, column = tile column, alternating between steps); the CTA's threads
// subtract each step's partial product from the tile in FP32 registers, round to nearest, so the
// update keeps FP32-grade accuracy (the tensor cores' own accumulation truncates).  The threads
// stage A (128 rows) and B (64 rows) of each step from the column-major front into shared memory in
// the canonical K-major, no-swizzle layout (core matrices of 8 rows x 16 bytes), hi and lo parts
// separately, two stages alternating; one thread issues the step's six MMAs and commits them to
// the stage's mbarrier, on which every thread waits before reading the step's accumulator.  The
// operands pass through registers for the hi/lo split, so they are staged by the threads rather
// than by TMA; the next step's loads and the previous step's read-out overlap the MMAs.
constexpr int TC_M = 128, TC_N = 64, TC_KC = 16;
constexpr int TC_A_BYTES = TC_M * TC_KC * 4;                      // one part (hi or lo) of A, one stage
constexpr int TC_B_BYTES = TC_N * TC_KC * 4;
constexpr int TC_STAGE = 2 * TC_A_BYTES + 2 * TC_B_BYTES;        // A hi, A lo, B hi, B lo
constexpr int TC_LBO_A = (TC_M / 8) * 128, TC_LBO_B = (TC_N / 8) * 128;   // between 16-byte K groups
constexpr int TC_MIN_FRONT = 128;                                // smaller fronts stay on FFMA tiles
constexpr long long TC_WAIT_NS = 1000000000LL;                   // bounded completion wait (1 s)
// instruction descriptor: D F32 (bits 4-5 = 1), A and B TF32 (bits 7-9, 10-12 = 2), both K-major,
// N >> 3 at bits 17-22, M >> 4 at bits 24-28
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                              ((uint32_t)(TC_M >> 4) << 24);
static_assert(NT == 256, "the staging maps assume 256 threads");
static_assert(2 * TC_STAGE <= (int)sizeof(double) * 4 * TS * TLD, "two stages fit in Shared::tile");

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start address, leading (K-direction) and stride (8-row group)
// byte offsets, all >> 4; version 1 (bit 46); no swizzle (bits 61-63 = 0)
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
                 ::"r"(d), "l"(a), "l"(b), "r"(TC_IDESC), "r"(acc) : "memory");
}
__device__ __forceinline__ void tc_commit(unsigned long long* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}
// thread-local wait for the completion of the barrier phase of parity `ph`; false when it has not
// completed within TC_WAIT_NS
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, uint32_t ph) {
    const uint32_t a = smem_u32(bar);
    unsigned long long t0 = 0;
    for (unsigned it = 0;; ++it) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}\n" : "=r"(ok) : "r"(a), "r"(ph) : "memory");
        if (ok) return true;
        if ((it & 255) == 0) {
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            if (it == 0) t0 = t;
            else if ((long long)(t - t0) > TC_WAIT_NS) return false;
        }
    }
}
// 32 lanes x 32 columns of FP32 accumulator from tensor memory (the warp's lane quarter), waited
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                 "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
                 "tcgen05.wait::ld.sync.aligned;\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                   "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                   "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr) : "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}
// a = hi + lo + O(2^-22 |a|): hi = a rounded to nearest TF32, lo = the rest (exact in FP32) rounded
// to nearest TF32; the tensor cores take both as they are
__device__ __forceinline__ void tf32_split(float a, float& hi, float& lo) {
    uint32_t h, l;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(a));
    hi = __uint_as_float(h);
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(a - hi));
    lo = __uint_as_float(l);
}

// The trailing-update tiles of tiles_f32, 128 rows each, on the tensor cores: M[r, c] -=
// Σ_{k in [K0, K1)} M[r, k] M[c, k] for r in [rb, rb + 128), c in [J, J + nb), r >= c; every
// (tile, 16-column K step) pair is one pipeline step.  Each step's product goes to its own
// accumulator (two, alternating) and is subtracted from the tile in FP32 registers while the next
// step's MMAs run, so the tensor cores' FP32 accumulation covers 16 products only.
template <class TileAt>
__device__ __noinline__ void tiles_tc32(float* M, int nf, int ntile, int K0, int K1, Shared& sh, TileAt at) {
    const int64_t ld = front_ld(nf);
    if (ntile <= 0 || K1 <= K0) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int quad = warp & 3, half = warp >> 2;
    const int nk = (K1 - K0 + TC_KC - 1) / TC_KC;
    const int nstep = ntile * nk;
    unsigned char* st = reinterpret_cast<unsigned char*>(sh.tile);
    const uint32_t st0 = smem_u32(st);
    // the accumulator columns and the two barriers belong to the CTA from tc_setup to tc_teardown;
    // the barriers' phases carry over from the previous call
    const uint32_t tmem = sh.tmem;
    uint32_t ph[2] = {sh.tc_ph & 1u, (sh.tc_ph >> 1) & 1u};
    // the operand rows this thread stages: A row ra (16-byte K groups ga and ga + 2), B row rb_
    const int ra = tid & 127, ga = tid >> 7;
    const int rb_ = tid & 63, gb = tid >> 6;
    float va0[4], va1[4], vb[4];
    int tile_next = -1;
    UTile unext{0, 0, 0};
    auto load = [&](int s) {
        const int ti = s / nk;
        if (ti != tile_next) { unext = at(ti); tile_next = ti; }
        const int k0 = K0 + TC_KC * (s % nk);
        const int cmax = min(nf, unext.J + unext.nb);
        const int r = unext.rb + ra, c = unext.J + rb_;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int k1 = k0 + 4 * ga + j, k2 = k0 + 4 * (ga + 2) + j, k3 = k0 + 4 * gb + j;
            va0[j] = (r < nf && k1 < K1) ? M[r + (int64_t)k1 * ld] : 0.f;
            va1[j] = (r < nf && k2 < K1) ? M[r + (int64_t)k2 * ld] : 0.f;
            vb[j] = (c < cmax && k3 < K1) ? M[c + (int64_t)k3 * ld] : 0.f;
        }
    };
    // row r, K group g of an operand of R rows: hi part at base + off, lo part at base + part + off
    auto put = [&](unsigned char* base, int r, int g, int R, const float (&v)[4], int part) {
        float4 h, l;
        tf32_split(v[0], h.x, l.x); tf32_split(v[1], h.y, l.y);
        tf32_split(v[2], h.z, l.z); tf32_split(v[3], h.w, l.w);
        const int off = g * (R / 8) * 128 + (r >> 3) * 128 + (r & 7) * 16;
        *reinterpret_cast<float4*>(base + off) = h;
        *reinterpret_cast<float4*>(base + part + off) = l;
    };
    // Read-out of step r: this thread's 32 outputs (tile row 32 quad + lane, columns 32 half + j)
    // of the step's partial product leave tensor memory and are subtracted, in FP32 round-to-nearest,
    // from acc, which holds M's values at the tile's first step and is stored back after its last
    float acc[32];
    UTile ur{0, 0, 0};
    auto readout = [&](int r) {
        const int b = r & 1, q = r % nk;
        if (q == 0) {
            ur = at(r / nk);
            const int row = ur.rb + 32 * quad + lane, cmax = min(nf, ur.J + ur.nb);
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const int col = ur.J + 32 * half + j;
                acc[j] = (row < nf && col < cmax && row >= col) ? M[row + (int64_t)col * ld] : 0.f;
            }
        }
        if (!mbar_wait(&sh.mbar[b], ph[b])) sh.tc_ok = 0;
        ph[b] ^= 1u;
        tc_fence_after();
        __syncwarp();
        float v[32];
        tc_ld32(tmem + (uint32_t)(b * TC_N) + ((uint32_t)(32 * quad) << 16) + 32 * half, v);
#pragma unroll
        for (int j = 0; j < 32; ++j) acc[j] -= v[j];
        tc_fence_before();
        if (q == nk - 1) {
            const int row = ur.rb + 32 * quad + lane, cmax = min(nf, ur.J + ur.nb);
            if (row < nf) {
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int col = ur.J + 32 * half + j;
                    if (col < cmax && row >= col) M[row + (int64_t)col * ld] = acc[j];
                }
            }
        }
    };
    load(0);
    int s = 0;
    for (; s < nstep; ++s) {
        const int b = s & 1, q = s % nk;
        // stage b and accumulator b are free: step s - 2 was read out by every thread (after its wait)
        __syncthreads();
        if (!sh.tc_ok) break;
        unsigned char* sb = st + b * TC_STAGE;
        put(sb, ra, ga, TC_M, va0, TC_A_BYTES);
        put(sb, ra, ga + 2, TC_M, va1, TC_A_BYTES);
        put(sb + 2 * TC_A_BYTES, rb_, gb, TC_N, vb, TC_B_BYTES);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // generic writes -> tensor-core reads
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t d = tmem + (uint32_t)(b * TC_N);
            const uint32_t a_hi = st0 + b * TC_STAGE, a_lo = a_hi + TC_A_BYTES;
            const uint32_t b_hi = a_hi + 2 * TC_A_BYTES, b_lo = b_hi + TC_B_BYTES;
#pragma unroll
            for (int kk = 0; kk < TC_KC / 8; ++kk) {
                const uint32_t oa = kk * 2 * TC_LBO_A, ob = kk * 2 * TC_LBO_B;
                tc_mma(d, tc_desc(a_lo + oa, TC_LBO_A, 128), tc_desc(b_hi + ob, TC_LBO_B, 128), kk > 0 ? 1u : 0u);
                tc_mma(d, tc_desc(a_hi + oa, TC_LBO_A, 128), tc_desc(b_lo + ob, TC_LBO_B, 128), 1u);
                tc_mma(d, tc_desc(a_hi + oa, TC_LBO_A, 128), tc_desc(b_hi + ob, TC_LBO_B, 128), 1u);
            }
            tc_commit(&sh.mbar[b]);
        }
        (void)q;
        if (s + 1 < nstep) load(s + 1);
        if (s >= 1) readout(s - 1);        // overlaps the MMAs of step s
    }
    __syncthreads();
    if (s == nstep && sh.tc_ok) readout(nstep - 1);
    __syncthreads();
    // a wait that ran out: the solve is reported failed, and the barriers' phases are unknown, so
    // this CTA's later updates use the FFMA tiles
    if (tid == 0) {
        if (!sh.tc_ok) {
            if (sh.tc_err) atomicExch(sh.tc_err, 2);
            sh.tc_on = 0;
        }
        sh.tc_ph = ph[0] | (ph[1] << 1);
    }
    __syncthreads();
}

// Set-up of the tensor-core update for the CTA's lifetime, by all its threads: warp 0 allocates
// the accumulator's TMEM columns, thread 0 initialises the two stage barriers.  `on` = 0 leaves
// the FFMA tiles in use and allocates nothing.
__device__ void tc_setup(Shared& sh, bool on) {
    __syncthreads();
    if (threadIdx.x == 0) { sh.tc_on = on ? 1 : 0; sh.tc_ok = 1; sh.tc_ph = 0; sh.tc_err = nullptr; }
    if (!on) { __syncthreads(); return; }
    __syncwarp();                        // the .sync.aligned tcgen05 forms need converged warps
    if ((threadIdx.x >> 5) == 0)
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&sh.tmem)), "r"(2 * TC_N) : "memory");
    if (threadIdx.x == 0) {
        mbar_init(&sh.mbar[0]);
        mbar_init(&sh.mbar[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}

// Release of the accumulator columns before the CTA exits (after tc_setup with on = 1; a CTA must
// free its TMEM before it ends)
__device__ void tc_teardown(Shared& sh, bool on) {
    tc_fence_before();
    __syncthreads();
    if (!on) return;
    tc_fence_after();
    __syncwarp();
    if ((threadIdx.x >> 5) == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(sh.tmem), "r"(2 * TC_N) : "memory");
    __syncthreads();
}

// FP32 trailing update on the tensor cores: 128-row tiles from J0 down, dealt round-robin over
// nranks CTAs
__device__ void update_cols_tc32(float* M, int nf, int J0, int nb, int K0, int K1, Shared& sh, int rank, int nranks) {
    if (K1 <= K0 || nb <= 0) return;
    const int first = J0 + TC_M * rank, step = TC_M * nranks;
    const int ntile = first < nf ? (nf - first + step - 1) / step : 0;
    tiles_tc32(M, nf, ntile, K0, K1, sh, [=](int i) { return UTile{first + step * i, J0, nb}; });
}

// the separator's Schur complement on the tensor cores: the 128-row tiles of every 64-column block
// of [J0, nf), in column-block order, dealt round-robin over nranks CTAs
__device__ void schur_tiles_tc32(float* M, int nf, int J0, int K0, int K1, Shared& sh, int rank, int nranks) {
    if (K1 <= K0 || J0 >= nf) return;
    const int nblk = (nf - J0 + 63) / 64;
    int total = 0;
    for (int b = 0; b < nblk; ++b) total += (nf - J0 - 64 * b + TC_M - 1) / TC_M;
    const int ntile = rank < total ? (total - rank + nranks - 1) / nranks : 0;
    auto at = [=](int i) {
        int gi = rank + nranks * i, b = 0;
        for (;;) {
            const int nt = (nf - J0 - 64 * b + TC_M - 1) / TC_M;
            if (gi < nt) break;
            gi -= nt;
            ++b;
        }
        const int J = J0 + 64 * b;
        return UTile{J + TC_M * gi, J, min(64, nf - J)};
    };
    tiles_tc32(M, nf, ntile, K0, K1, sh, at);
}

#else
// the default build has no tensor-core tiles
__device__ void update_cols_tc32(float*, int, int, int, int, int, Shared&, int, int) {}
__device__ void schur_tiles_tc32(float*, int, int, int, int, Shared&, int, int) {}
__device__ __forceinline__ void tc_setup(Shared& sh, bool) {
    __syncthreads();
    if (threadIdx.x == 0) { sh.tc_on = 0; sh.tc_ok = 1; sh.tc_ph = 0; sh.tc_err = nullptr; }
    __syncthreads();
}
__device__ __forceinline__ void tc_teardown(Shared&, bool) { __syncthreads(); }
#endif

// FP32 update tiles go to the tensor cores for fronts from TC_MIN_FRONT up unless
// settings.fp32_tiles selects the FFMA tiles
__device__ __forceinline__ bool use_tc32(int nf, const Shared& sh) { return MB_TC && sh.tc_on && nf >= 128; }

__device__ void update_cols_f32(float* M, int nf, int J0, int nb, int K0, int K1, Shared& sh, int rank = 0,
                                int nranks = 1) {
    if (K1 <= K0 || nb <= 0) return;
    if (use_tc32(nf, sh)) {
        update_cols_tc32(M, nf, J0, nb, K0, K1, sh, rank, nranks);
        __syncthreads();
        return;
    }
    const int first = J0 + TS * rank, step = TS * nranks;
    const int ntile = first < nf ? (nf - first + step - 1) / step : 0;
    tiles_f32(M, nf, ntile, K0, K1, sh, [=](int i) { return UTile{first + step * i, J0, nb}; });
    __syncthreads();
}

// Schur complement of a front's separator block, M[r, c] -= Σ_{k in [K0, K1)} M[r, k] M[c, k] for
// J0 <= c <= r < nf: every (64-column block, row tile) pair in column-block order, dealt
// round-robin over nranks CTAs, all of one CTA's tiles in one pipeline.  With K0 > 0 it is the
// trailing update of a right-looking step.
template <class FT>
__device__ void schur_tiles(FT* M, int nf, int J0, int K0, int K1, Shared& sh, int rank, int nranks) {
    if (K1 <= K0 || J0 >= nf) return;
    const int nblk = (nf - J0 + 63) / 64;               // column blocks; block b has nblk - b row tiles
    const int total = nblk * (nblk + 1) / 2;
    const int ntile = rank < total ? (total - rank + nranks - 1) / nranks : 0;
    // tile gi of the sequence: the column block b and its first tile `base` are kept from the
    // previous call (the pipelines ask for tiles in increasing order; a smaller one restarts)
    auto at = [=, b = 0, base = 0](int i) mutable {
        const int gi = rank + nranks * i;
        if (gi < base) { b = 0; base = 0; }
        while (gi - base >= nblk - b) { base += nblk - b; ++b; }
        const int J = J0 + 64 * b;
        return UTile{J + TS * (gi - base), J, min(64, nf - J)};
    };
    if constexpr (sizeof(FT) == 8) tiles_f64((double*)M, nf, ntile, K0, K1, sh, at);
    else if (use_tc32(nf, sh)) schur_tiles_tc32((float*)M, nf, J0, K0, K1, sh, rank, nranks);
    else tiles_f32((float*)M, nf, ntile, K0, K1, sh, at);
    __syncthreads();
}



// forward-solve row update for the 32-column block at k0: x[row i] -= L[i, k0:k0+kb] xs for the rows
// i >= k0 + kb of this rank (row blocks of NT dealt over nranks CTAs); xs = sh.xs, or with `load`
// read back from x (a helper CTA)
template <class FT>
__device__ void lsolve_rows(const FT* M, int nf, int nres, int r0, const int* sep, double* x, int k0, int kb,
                            Shared& sh, int rank, int nranks, bool load) {
    const int64_t ld = front_ld(nf);
    const int tid = threadIdx.x;
    if (load) {
        if (tid < kb) sh.xs[tid] = x[r0 + k0 + tid];
        __syncthreads();
    }
    for (int i = k0 + kb + rank * NT + tid; i < nf; i += NT * nranks) {
        const FT* Mi = M + i + (int64_t)k0 * ld;
        double t = 0;
        if (kb == 32) {   // all 32 loads in flight before the FMA chain
            FT v[32];
#pragma unroll
            for (int c = 0; c < 32; ++c) v[c] = Mi[(int64_t)c * ld];
#pragma unroll
            for (int c = 0; c < 32; ++c) t = fma((double)v[c], sh.xs[c], t);
        } else {
            for (int c = 0; c < kb; ++c) t = fma((double)Mi[(int64_t)c * ld], sh.xs[c], t);
        }
        int tg = i < nres ? r0 + i : sep[i - nres];
        x[tg] -= t;
    }
    __syncthreads();
}

// backward-solve column dots for the 32-column block at k0: out[c] = L[k0+kb:, k0+c] · x[rows], one
// warp per column, columns dealt over the gw-th of `gws` warps of the grid
template <class FT>
__device__ void usolve_dots(const FT* M, int nf, int nres, int r0, const int* sep, const double* x, int k0, int kb,
                            double* out, int gw, int gws) {
    const int64_t ld = front_ld(nf);
    const int lane = threadIdx.x & 31;
    for (int c = gw; c < kb; c += gws) {
        const FT* Mc = M + (int64_t)(k0 + c) * ld;
        double t0 = 0, t1 = 0, t2 = 0, t3 = 0;
        int i = k0 + kb + lane;
        for (; i + 96 < nf; i += 128) {   // four rows per lane in flight
            int s0 = i < nres ? r0 + i : sep[i - nres];
            int s1 = i + 32 < nres ? r0 + i + 32 : sep[i + 32 - nres];
            int s2 = i + 64 < nres ? r0 + i + 64 : sep[i + 64 - nres];
            int s3 = i + 96 < nres ? r0 + i + 96 : sep[i + 96 - nres];
            double m0 = (double)Mc[i], m1 = (double)Mc[i + 32], m2 = (double)Mc[i + 64], m3 = (double)Mc[i + 96];
            t0 = fma(m0, x[s0], t0); t1 = fma(m1, x[s1], t1); t2 = fma(m2, x[s2], t2); t3 = fma(m3, x[s3], t3);
        }
        for (; i < nf; i += 32) {
            int src = i < nres ? r0 + i : sep[i - nres];
            t0 = fma((double)Mc[i], x[src], t0);
        }
        double t = warp_sum((t0 + t1) + (t2 + t3));
        if (lane == 0) out[c] = t;
    }
}

// ---- grid-cooperative help for large fronts (CoopCtl) ----------------------------------------
constexpr long long COOP_WAIT_NS = 60000000000LL;   // default longest wait at a grid barrier (60 s)
constexpr int COOP_MIN_FRONT = 192;                 // fronts from this order up use the helpers
constexpr int COOP_MIN_SOLVE = 2048;                // ... and in the triangular solves from this order up

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_volatile_i32(const int* p) { return *(const volatile int*)p; }
__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid barrier over all CTAs of the cooperative launch.  Returns false (on every thread) once any
// wait has run past sh.wait_ns; the barrier then no longer waits.
__device__ bool coop_barrier(CoopCtl* c, const Shared& sh) {
    __syncthreads();
    if (threadIdx.x == 0 && ld_volatile_i32(&c->abort) == 0) {
        const unsigned int g = ld_acquire_u32(&c->gen);
        __threadfence();
        const unsigned int prev = atomicAdd(&c->count, 1u);
        if (prev + 1 == gridDim.x) {
            atomicExch(&c->count, 0u);
            __threadfence();
            atomicAdd(&c->gen, 1u);
        } else {
            const unsigned long long t0 = gtimer();
            unsigned int nap = 100;   // ns; backs off to 1 us so idle helpers poll the hot word rarely
            while (ld_acquire_u32(&c->gen) == g) {
                if (ld_volatile_i32(&c->abort) != 0) break;
                if ((long long)(gtimer() - t0) > sh.wait_ns) { atomicExch(&c->abort, 1); break; }
                __nanosleep(nap);
                if (nap < 1000) nap *= 2;
            }
        }
    }
    __syncthreads();
    asm volatile("fence.acq_rel.gpu;" ::: "memory");
    return ld_volatile_i32(&c->abort) == 0;
}

// one command's share for this rank (every CTA of the grid runs it between two barriers)
__device__ void coop_exec(CoopCtl* c, Shared& sh, int rank, int nranks) {
    if (threadIdx.x == 0) {
        const volatile CoopCtl* vc = c;
        sh.ibuf[0] = vc->cmd;
        for (int k = 0; k < 7; ++k) sh.ibuf[1 + k] = vc->ia[k];
    }
    __syncthreads();
    const int cmd = sh.ibuf[0];
    const int* ia = sh.ibuf + 1;
    const volatile CoopCtl* vc = c;
    void* p0 = vc->pa[0];
    void* p1 = vc->pa[1];
    void* p2 = vc->pa[2];
    const long long l0 = vc->la[0];
    __syncthreads();
    const int tid = threadIdx.x;
    if (cmd == COOP_FILL) {                 // p0[0 .. l0) = 0 (doubles)
        double* x = (double*)p0;
        for (long long i = (long long)rank * NT + tid; i < l0; i += (long long)NT * nranks) x[i] = 0;
    } else if (cmd == COOP_COPY) {          // (FT) p0[i] = p1[i], i < l0; ia[0] = FP32
        const double* src = (const double*)p1;
        if (ia[0]) { float* dst = (float*)p0; for (long long i = (long long)rank * NT + tid; i < l0; i += (long long)NT * nranks) dst[i] = (float)src[i]; }
        else { double* dst = (double*)p0; for (long long i = (long long)rank * NT + tid; i < l0; i += (long long)NT * nranks) dst[i] = src[i]; }
    } else if (cmd == COOP_UPDATE) {        // update_cols(p0, nf=ia1, J0=ia2, nb=ia3, K0=ia4, K1=ia5); ia0 = FP32
        if (ia[0]) update_cols_f32((float*)p0, ia[1], ia[2], ia[3], ia[4], ia[5], sh, rank, nranks);
        else update_cols_f64((double*)p0, ia[1], ia[2], ia[3], ia[4], ia[5], sh, rank, nranks);
    } else if (cmd == COOP_PANEL) {         // panel_rows(p0, nf=ia1, k0=ia2, kb=ia3); ia0 = FP32
        if (ia[0]) panel_rows<float>((float*)p0, ia[1], ia[2], ia[3], sh, rank, nranks, rank != 0);
        else panel_rows<double>((double*)p0, ia[1], ia[2], ia[3], sh, rank, nranks, rank != 0);
    } else if (cmd == COOP_SCHUR) {         // schur_tiles(p0, nf=ia1, J0=ia2, K0=ia4, K1=ia3)
        if (ia[0]) schur_tiles<float>((float*)p0, ia[1], ia[2], ia[4], ia[3], sh, rank, nranks);
        else schur_tiles<double>((double*)p0, ia[1], ia[2], ia[4], ia[3], sh, rank, nranks);
    } else if (cmd == COOP_LROWS) {         // lsolve_rows(p0, nf=ia1, nres=ia2, r0=ia3, sep=p1, x=p2, k0=ia4, kb=ia5)
        if (ia[0]) lsolve_rows<float>((const float*)p0, ia[1], ia[2], ia[3], (const int*)p1, (double*)p2, ia[4], ia[5], sh, rank, nranks, true);
        else lsolve_rows<double>((const double*)p0, ia[1], ia[2], ia[3], (const int*)p1, (double*)p2, ia[4], ia[5], sh, rank, nranks, true);
    } else if (cmd == COOP_UDOTS) {         // usolve_dots(...) into c->acc, columns over all warps of the grid
        const int gw = rank * NW + (threadIdx.x >> 5), gws = nranks * NW;
        if (ia[0]) usolve_dots<float>((const float*)p0, ia[1], ia[2], ia[3], (const int*)p1, (const double*)p2, ia[4], ia[5], c->acc, gw, gws);
        else usolve_dots<double>((const double*)p0, ia[1], ia[2], ia[3], (const int*)p1, (const double*)p2, ia[4], ia[5], c->acc, gw, gws);
    } else if (cmd == COOP_EXTEND) {        // parent p1 += child p0's update block; ia: FP32, nfr, nres, nsep, np; p2 = rel
        const int nfr = ia[1], nres = ia[2], nsep = ia[3], np = ia[4];
        const int* rel = (const int*)p2;
        for (long long t = (long long)rank * NT + tid; t < (long long)nsep * nsep; t += (long long)NT * nranks) {
            const int i = (int)(t % nsep), j = (int)(t / nsep);
            if (i < j) continue;
            const long long dst = rel[i] + (long long)rel[j] * front_ld(np), src = (nres + i) + (long long)(nres + j) * front_ld(nfr);
            if (ia[0]) ((float*)p1)[dst] += ((const float*)p0)[src];
            else ((double*)p1)[dst] += ((const double*)p0)[src];
        }
    }
    __syncthreads();
}

// leader: post a command (fields set by the caller's thread 0 through `post`) and run its share
template <class Post>
__device__ bool coop_call(CoopCtl* c, Shared& sh, Post post) {
    if (threadIdx.x == 0) post(c);
    if (!coop_barrier(c, sh)) return false;
    coop_exec(c, sh, 0, gridDim.x);
    return coop_barrier(c, sh);
}

// helpers: serve commands until COOP_EXIT or an abort
__device__ void coop_helper(CoopCtl* c, Shared& sh) {
    for (;;) {
        if (!coop_barrier(c, sh)) return;
        if (threadIdx.x == 0) sh.ibuf[0] = ((const volatile CoopCtl*)c)->cmd;
        __syncthreads();
        const int cmd = sh.ibuf[0];
        __syncthreads();
        if (cmd == COOP_EXIT) return;
        coop_exec(c, sh, blockIdx.x, gridDim.x);
        if (!coop_barrier(c, sh)) return;
    }
}

template <class FT> struct IsF32 { static constexpr int v = 0; };
template <> struct IsF32<float> { static constexpr int v = 1; };

// forward solve with front f: x[res] <- D⁻¹ x[res]; x[sep] -= L_off x[res]
template <class FT, bool COOP = false>
__device__ void front_lsolve(const FT* M, int nf, int nres, int r0, const int* sep, double* x, Shared& sh,
                             CoopCtl* coop = nullptr) {
    const int64_t ld = front_ld(nf);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double* T = sh.diag;   // the 32x32 diagonal triangle, T[c*33 + r] = L[k0+r, k0+c]
    for (int k0 = 0; k0 < nres; k0 += 32) {
        const int kb = min(32, nres - k0);
        for (int idx = tid; idx < 32 * 32; idx += NT) {
            int r = idx & 31, c = idx >> 5;
            if (r < kb && c < kb && r >= c) T[c * 33 + r] = (double)M[(k0 + r) + (int64_t)(k0 + c) * ld];
        }
        __syncthreads();
        if (warp == 0) {
            double xv = lane < kb ? x[r0 + k0 + lane] : 0.0;
            for (int c = 0; c < kb; ++c) {
                if (lane == c) xv = xv / T[c * 33 + c];
                double xc = __shfl_sync(0xffffffffu, xv, c);
                if (lane > c && lane < kb) xv -= T[c * 33 + lane] * xc;
            }
            if (lane < kb) { x[r0 + k0 + lane] = xv; sh.xs[lane] = xv; }
        }
        __syncthreads();
        if (!COOP || !coop) {
            lsolve_rows<FT>(M, nf, nres, r0, sep, x, k0, kb, sh, 0, 1, false);
        } else if (!coop_call(coop, sh, [&](CoopCtl* c) {
                       c->cmd = COOP_LROWS; c->pa[0] = (void*)M; c->pa[1] = (void*)sep; c->pa[2] = x;
                       c->ia[0] = IsF32<FT>::v; c->ia[1] = nf; c->ia[2] = nres; c->ia[3] = r0; c->ia[4] = k0; c->ia[5] = kb;
                   })) {
            return;
        }
    }
}

// backward solve with front f: x[res] -= L_offᵀ x[sep]; x[res] <- D⁻ᵀ x[res]
template <class FT, bool COOP = false>
__device__ void front_usolve(const FT* M, int nf, int nres, int r0, const int* sep, double* x, Shared& sh,
                             CoopCtl* coop = nullptr) {
    const int64_t ld = front_ld(nf);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nblk = (nres + 31) / 32;
    double* T = sh.diag;   // T[c*33 + r] = L[k0+r, k0+c]
    for (int bk = nblk - 1; bk >= 0; --bk) {
        const int k0 = bk * 32, kb = min(32, nres - k0);
        for (int idx = tid; idx < 32 * 32; idx += NT) {
            int r = idx & 31, c = idx >> 5;
            if (r < kb && c < kb && r >= c) T[c * 33 + r] = (double)M[(k0 + r) + (int64_t)(k0 + c) * ld];
        }
        if (!COOP || !coop) {
            usolve_dots<FT>(M, nf, nres, r0, sep, x, k0, kb, sh.acc, warp, NW);
        } else {
            if (!coop_call(coop, sh, [&](CoopCtl* c) {
                    c->cmd = COOP_UDOTS; c->pa[0] = (void*)M; c->pa[1] = (void*)sep; c->pa[2] = x;
                    c->ia[0] = IsF32<FT>::v; c->ia[1] = nf; c->ia[2] = nres; c->ia[3] = r0; c->ia[4] = k0; c->ia[5] = kb;
                }))
                return;
            if (threadIdx.x < kb) sh.acc[threadIdx.x] = ((const volatile CoopCtl*)coop)->acc[threadIdx.x];
        }
        __syncthreads();
        if (warp == 0) {
            double yv = lane < kb ? x[r0 + k0 + lane] - sh.acc[lane] : 0.0;
            for (int c = kb - 1; c >= 0; --c) {
                if (lane == c) yv = yv / T[c * 33 + c];
                double xc = __shfl_sync(0xffffffffu, yv, c);
                if (lane < c) yv -= T[lane * 33 + c] * xc;
            }
            if (lane < kb) x[r0 + k0 + lane] = yv;
        }
        __syncthreads();
    }
}


// ---- triangular solves of one front with its slice of x in shared memory ----------------------
// Fronts of order [XSM_MIN, COOP_MIN_SOLVE) keep xf[i] = x[front row i] in Shared::tile (idle during a solve)
// for the whole front: the panel loads do not depend on x, so they are issued before each diagonal
// solve and the row updates and dots read x from shared memory.  The diagonal steps apply the
// block inverse diag_factor stored (a lane per row, no serial chain over the block's columns).
constexpr int XSM_CAP = 4 * TS * TLD;   // doubles in Shared::tile
constexpr int XSM_MIN = 64;             // smaller fronts stay on the global-memory sweep (no gather)
static_assert(COOP_MIN_SOLVE + 8 * 32 <= XSM_CAP, "front slice of x and dot partials must fit");

template <class FT>
__device__ __noinline__ void front_lsolve_sm(const FT* M, int nf, int nres, int r0, const int* sep, double* x, Shared& sh) {
    const int64_t ld = front_ld(nf);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double* xf = sh.tile;
    double* T = sh.diag;   // T[c*33 + r] = L[k0+r, k0+c]
    for (int i = tid; i < nf; i += NT) xf[i] = x[i < nres ? r0 + i : sep[i - nres]];
    __syncthreads();
    for (int k0 = 0; k0 < nres; k0 += 32) {
        const int kb = min(32, nres - k0);
        const int i0 = k0 + kb + tid;
        FT v[32];
        if (kb == 32 && i0 < nf) {   // first panel row of this thread, in flight during the diagonal solve
            const FT* Mi = M + i0 + (int64_t)k0 * ld;
#pragma unroll
            for (int c = 0; c < 32; ++c) v[c] = Mi[(int64_t)c * ld];
        }
        for (int idx = tid; idx < 32 * 32; idx += NT) {   // T[r*33 + c] = X[r][c], c < r (L⁻¹ of the block)
            int c = idx & 31, r = idx >> 5;
            if (r < kb && c < r) T[r * 33 + c] = (double)M[(k0 + c) + (int64_t)(k0 + r) * ld];
        }
        if (tid < kb) sh.dinv[tid] = 1.0 / (double)M[(k0 + tid) + (int64_t)(k0 + tid) * ld];
        __syncthreads();
        if (warp == 0 && lane < kb) {   // x = L⁻¹ b for the block, a lane per row
            const int r = lane;
            double s0 = 0, s1 = 0;
            for (int c = 0; c + 1 < r; c += 2) { s0 = fma(T[r * 33 + c], xf[k0 + c], s0); s1 = fma(T[r * 33 + c + 1], xf[k0 + c + 1], s1); }
            if (r & 1) s0 = fma(T[r * 33 + r - 1], xf[k0 + r - 1], s0);
            const double xv = fma(sh.dinv[r], xf[k0 + r], s0 + s1);
            sh.xs[r] = xv;
        }
        __syncthreads();
        if (tid < kb) xf[k0 + tid] = sh.xs[tid];
        for (int i = i0; i < nf; i += NT) {
            const FT* Mi = M + i + (int64_t)k0 * ld;
            double t = 0;
            if (kb == 32) {
                if (i != i0) {
#pragma unroll
                    for (int c = 0; c < 32; ++c) v[c] = Mi[(int64_t)c * ld];
                }
#pragma unroll
                for (int c = 0; c < 32; ++c) t = fma((double)v[c], sh.xs[c], t);
            } else {
                for (int c = 0; c < kb; ++c) t = fma((double)Mi[(int64_t)c * ld], sh.xs[c], t);
            }
            xf[i] -= t;
        }
        __syncthreads();
    }
    for (int i = tid; i < nf; i += NT) x[i < nres ? r0 + i : sep[i - nres]] = xf[i];
    __syncthreads();
}

// backward sweep of one front: for each 32-column block from the last, the dots
// L[k0+kb:, k0+c] · xf[k0+kb:] (16 columns at a time in registers, a warp reduce-scatter, then
// across warps), then the transposed diagonal solve
template <class FT>
__device__ __noinline__ void front_usolve_sm(const FT* M, int nf, int nres, int r0, const int* sep, double* x, Shared& sh) {
    const int64_t ld = front_ld(nf);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nblk = (nres + 31) / 32;
    double* xf = sh.tile;
    double* part = sh.tile + XSM_CAP - NW * 32;   // part[w*32 + c]: warp w's share of column c's dot
    double* T = sh.diag;
    for (int i = tid; i < nf; i += NT) xf[i] = x[i < nres ? r0 + i : sep[i - nres]];
    __syncthreads();
    for (int bk = nblk - 1; bk >= 0; --bk) {
        const int k0 = bk * 32, kb = min(32, nres - k0);
        for (int h = 0; h < kb; h += 16) {
            const int hb = min(16, kb - h);
            double acc[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[j] = 0;
            for (int i = k0 + kb + tid; i < nf; i += NT) {
                const FT* Mi = M + i + (int64_t)(k0 + h) * ld;
                const double xi = xf[i];
                if (hb == 16) {
                    FT v[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j) v[j] = Mi[(int64_t)j * ld];
#pragma unroll
                    for (int j = 0; j < 16; ++j) acc[j] = fma((double)v[j], xi, acc[j]);
                } else {
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        if (j < hb) acc[j] = fma((double)Mi[(int64_t)j * ld], xi, acc[j]);
                }
            }
            // reduce over the warp: afterwards lane l (and l + 16) holds column h + (l & 15)
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], 16);
#pragma unroll
            for (int o = 8; o >= 1; o >>= 1) {
                const bool up = lane & o;
#pragma unroll
                for (int j = 0; j < o; ++j) {
                    const double send = up ? acc[j] : acc[j + o];
                    const double keep = up ? acc[j + o] : acc[j];
                    acc[j] = keep + __shfl_xor_sync(0xffffffffu, send, o);
                }
            }
            if (lane < 16) part[warp * 32 + h + lane] = acc[0];
        }
        for (int idx = tid; idx < 32 * 32; idx += NT) {   // T[r*33 + c] = X[r][c], c < r (L⁻¹ of the block)
            int c = idx & 31, r = idx >> 5;
            if (r < kb && c < r) T[r * 33 + c] = (double)M[(k0 + c) + (int64_t)(k0 + r) * ld];
        }
        if (tid < kb) sh.dinv[tid] = 1.0 / (double)M[(k0 + tid) + (int64_t)(k0 + tid) * ld];
        __syncthreads();
        if (warp == 0) {   // x = L⁻ᵀ y for the block, a lane per row: x_c = Σ_{r ≥ c} X[r][c] y_r
            double dot = 0;
            if (lane < kb) {
#pragma unroll
                for (int w = 0; w < NW; ++w) dot += part[w * 32 + lane];
            }
            const double yv = lane < kb ? xf[k0 + lane] - dot : 0.0;
            sh.xs[lane] = yv;
            __syncwarp();
            if (lane < kb) {
                const int c = lane;
                double s0 = 0, s1 = 0;
                int r = c + 1;
                for (; r + 1 < kb; r += 2) { s0 = fma(T[r * 33 + c], sh.xs[r], s0); s1 = fma(T[(r + 1) * 33 + c], sh.xs[r + 1], s1); }
                if (r < kb) s0 = fma(T[r * 33 + c], sh.xs[r], s0);
                xf[k0 + c] = fma(sh.dinv[c], yv, s0 + s1);
            }
        }
        __syncthreads();
    }
    for (int i = tid; i < nres; i += NT) x[r0 + i] = xf[i];
    __syncthreads();
}


template <class FT>
__device__ __forceinline__ void update_cols(FT* M, int nf, int J0, int nb, int K0, int K1, Shared& sh);
template <>
__device__ __forceinline__ void update_cols<double>(double* M, int nf, int J0, int nb, int K0, int K1, Shared& sh) {
    update_cols_f64(M, nf, J0, nb, K0, K1, sh);
}
template <>
__device__ __forceinline__ void update_cols<float>(float* M, int nf, int J0, int nb, int K0, int K1, Shared& sh) {
    update_cols_f32(M, nf, J0, nb, K0, K1, sh);
}

constexpr int COOP_ABORTED = -1;   // front_chol result when the grid barrier timed out
constexpr int COOP_RL_FRONT = 1024; // grid-cooperative fronts from this order up factor right-looking

// Front factorization: left-looking over 64-column blocks (each column updated once, from final L
// columns), 32-column diagonal/panel steps inside a block, then the separator's Schur complement
// (the update matrix handed to the parent by extend-add).  With `coop` and a front of at least
// COOP_MIN_FRONT, the update tiles and panel rows are shared with the helper CTAs.  A shared front
// of at least COOP_RL_FRONT factors right-looking instead: after each 64-column block its trailing
// matrix, separator included, takes the block's rank-64 update as one command of tiles over the
// whole grid.  A left-looking step has (nf - J) / 64 row tiles of depth J, so near the end of a
// large front a few CTAs carry all the work while the rest wait; the trailing update has
// ((nf - J) / 64)² / 2 tiles of depth 64 at every step.  The factor is the one-CTA factor bit for
// bit: an entry's accumulator starts from the front's value and takes the products in increasing k
// with the same chunk boundaries either way, and storing it between steps is exact.
template <class FT, bool COOP>
__device__ int front_chol_ll(FT* M, int nf, int nres, Shared& sh, CoopCtl* coop, long long* tf) {
    const bool big = COOP && coop != nullptr && nf >= COOP_MIN_FRONT;
    const bool rl = big && nf >= COOP_RL_FRONT;
    // tf[0..2]: SM clocks in the trailing updates, the diagonal blocks and the panel rows
    auto tic = [&]() -> long long { __syncthreads(); return clock64(); };
    auto toc = [&](int k, long long t0) { __syncthreads(); tf[k] += clock64() - t0; };
    auto upd = [&](int J0, int nb, int K0, int K1) -> bool {
        if (K1 <= K0 || nb <= 0) return true;
        const long long t0 = tic();
        bool ok = true;
        if (!big) update_cols<FT>(M, nf, J0, nb, K0, K1, sh);
        else ok = coop_call(coop, sh, [&](CoopCtl* c) {
            c->cmd = COOP_UPDATE; c->pa[0] = M;
            c->ia[0] = IsF32<FT>::v; c->ia[1] = nf; c->ia[2] = J0; c->ia[3] = nb; c->ia[4] = K0; c->ia[5] = K1;
        });
        toc(0, t0);
        return ok;
    };
    auto trail = [&](int J0, int K0, int K1) -> bool {   // right-looking step: columns [J0, nf)
        const long long t0 = tic();
        const bool ok = coop_call(coop, sh, [&](CoopCtl* c) {
            c->cmd = COOP_SCHUR; c->pa[0] = M;
            c->ia[0] = IsF32<FT>::v; c->ia[1] = nf; c->ia[2] = J0; c->ia[3] = K1; c->ia[4] = K0;
        });
        toc(0, t0);
        return ok;
    };
    for (int J = 0; J < nres; J += 64) {
        const int nb = min(64, nres - J);
        if (!rl && !upd(J, nb, 0, J)) return COOP_ABORTED;
        for (int h = 0; h < nb; h += 32) {
            const int k0 = J + h, kb = min(32, nb - h);
            if (h > 0 && !upd(k0, kb, J, J + 32)) return COOP_ABORTED;
            // thread 0's clock without barriers around these two, so warp 1 can work on the diagonal
            // block's inverse while the others start the panel rows
            long long t0 = clock64();
            const int info = diag_factor<FT>(M, nf, k0, kb, sh);
            tf[1] += clock64() - t0;
            if (info) return info;
            t0 = clock64();
            if (!big) panel_rows<FT>(M, nf, k0, kb, sh, 0, 1, false);
            else if (!coop_call(coop, sh, [&](CoopCtl* c) {
                         c->cmd = COOP_PANEL; c->pa[0] = M;
                         c->ia[0] = IsF32<FT>::v; c->ia[1] = nf; c->ia[2] = k0; c->ia[3] = kb;
                     }))
                return COOP_ABORTED;
            tf[2] += clock64() - t0;
        }
        if (rl && J + nb < nf && !trail(J + nb, J, J + nb)) return COOP_ABORTED;
    }
    if (rl) return 0;                    // the trailing updates covered the separator block
    const long long t0 = tic();
    if (!big) {
        schur_tiles<FT>(M, nf, nres, 0, nres, sh, 0, 1);
    } else if (nres > 0 && nf > nres &&
               !coop_call(coop, sh, [&](CoopCtl* c) {   // the whole separator block in one command
                   c->cmd = COOP_SCHUR; c->pa[0] = M;
                   c->ia[0] = IsF32<FT>::v; c->ia[1] = nf; c->ia[2] = nres; c->ia[3] = nres; c->ia[4] = 0;
               })) {
        return COOP_ABORTED;
    }
    toc(0, t0);
    return 0;
}

// ---------------------------------------------------------------------------------------------
// the per-instance solver
// ---------------------------------------------------------------------------------------------
// body(v, nc, t) for every entry t < nc² of every vertex block v (nc = its column count) with
// pred(v): blocks of one or two columns a thread each, blocks below 1024 entries a warp each, larger
// ones over the whole CTA, then a barrier.  A vertex of one scalar column otherwise costs a pass of
// the whole CTA over a dependent load chain; the entries are disjoint and each is written once, so
// the split changes no result.
template <class Pred, class Body>
__device__ void for_vertex_blocks(const int* xcol, int nv, Pred pred, Body body) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int v = tid; v < nv; v += NT) {
        const int nc = xcol[v + 1] - xcol[v];
        if (nc <= 2 && pred(v))
            for (int t = 0; t < nc * nc; ++t) body(v, nc, t);
    }
    for (int v = warp; v < nv; v += NW) {
        const int nc = xcol[v + 1] - xcol[v];
        if (nc > 2 && nc * nc < 1024 && pred(v))
            for (int t = lane; t < nc * nc; t += 32) body(v, nc, t);
    }
    for (int v = 0; v < nv; ++v) {
        const int nc = xcol[v + 1] - xcol[v];
        if (nc * nc >= 1024 && pred(v))
            for (int t = tid; t < nc * nc; t += NT) body(v, nc, t);
    }
    __syncthreads();
}

// row pair q of an FT column that starts on a pair boundary, from two FP64 values
__device__ __forceinline__ void store_pair(double* m, int q, double2 a) { reinterpret_cast<double2*>(m)[q] = a; }
__device__ __forceinline__ void store_pair(float* m, int q, double2 a) {
    reinterpret_cast<float2*>(m)[q] = make_float2((float)a.x, (float)a.y);
}

template <bool COOP>   // COOP: the leader of a grid-cooperative launch (else no cooperative code is built)
struct Ctx {
    const DevInst& I;
    Settings set;
    Shared& sh;
    CoopCtl* coop;          // grid-cooperative mode (one large instance), else null
    double* red;
    double* F64;            // the factor storage viewed as FP64 ...
    float* F32;             // ... or as FP32 (same buffer)
    bool use32;             // this iteration factors in FP32
    bool fellback;          // mixed precision: the FP64 factor is in use for good
    int switched;           // mixed precision: moved to FP64 after a solve-heavy FP32 iteration
    int nfp32, nfallback;   // iterations accepted with the FP32 factor; FP64 redos
    int stall0;             // history rows before the last precision switch (the stall window starts there)
    bool stallhit;          // the last step_ ended on the stall test
    bool kktfail;           // the last iteration's factorization or a KKT solve failed
    int n, m, nv;
    double *Df, *Qp, *wf, *Dpa, *Dda, *Dp, *Dd, *df, *dx, *cgw, *tn;
    double *Dg, *Dya, *Dy, *dg, *dyv, *cgp, *tm1, *tm2;
    double *vstep, *vspsd, *vflag, *vscl, *vnrm, *vswp;
    double *vsocz;          // vertices whose diagonal block of Q is zero and whose H block is applied
                            // in structured form: 1 = SOC (rank one plus diagonal), 2 = SDP (W ⊗ₛ W)
    double *vsocdot;        // zᵀx of such an SOC cone during a product with H
    int nsocz;              // how many such vertices
    double *hx;             // (H x) of the structured SDP blocks during a product with H
    double delta;
    double nf, ng, sf, sg, nB;
    int nrow_hist;
    int nretry;
    int nfact;              // numeric factorizations performed
    long long tsec[NSEC];   // per-section SM clocks (thread 0)
    long long ntrsv, ngemv;
    __device__ long long tic() const { __syncthreads(); return clock64(); }
    __device__ void toc(int sec, long long t0) { __syncthreads(); tsec[sec] += clock64() - t0; }
    __device__ Ctx(const DevInst& I_, const Settings& s_, Shared& sh_, CoopCtl* coop_ = nullptr)
        : I(I_), set(s_), sh(sh_), coop(coop_) {
        red = sh.red;
        F64 = reinterpret_cast<double*>(I.F);
        F32 = reinterpret_cast<float*>(I.F);
        use32 = set.precision == 1 || (set.precision == 2 && I.status[5] == 0 && I.status[6] == 0);
        fellback = I.status[5] != 0 || I.status[6] != 0;
        switched = I.status[6];
        nfp32 = I.status[4]; nfallback = I.status[5];
        n = I.n; m = I.m; nv = I.nvtx;
        double* v = I.vn;
        Df = v; Qp = v + n; wf = v + 2 * (int64_t)n; Dpa = v + 3 * (int64_t)n; Dda = v + 4 * (int64_t)n;
        Dp = v + 5 * (int64_t)n; Dd = v + 6 * (int64_t)n; df = v + 7 * (int64_t)n; dx = v + 8 * (int64_t)n;
        cgw = v + 9 * (int64_t)n; tn = v + 10 * (int64_t)n; hx = v + 12 * (int64_t)n;
        double* w = I.vm;
        Dg = w; Dya = w + m; Dy = w + 2 * (int64_t)m; dg = w + 3 * (int64_t)m; dyv = w + 4 * (int64_t)m;
        cgp = w + 5 * (int64_t)m; tm1 = w + 6 * (int64_t)m; tm2 = w + 7 * (int64_t)m;
        double* z = I.vv;
        vstep = z; vspsd = z + nv; vflag = z + 2 * nv; vscl = z + 3 * nv; vnrm = z + 4 * nv; vswp = z + 5 * nv;
        vsocz = z + 6 * nv; vsocdot = z + 7 * nv;
        nsocz = (int)I.scal[SCAL_NSOCZ];
        stall0 = (int)I.scal[SCAL_STALL0]; stallhit = false;
        delta = 1; nrow_hist = 0; nretry = 0;
        nf = I.scal[5]; ng = I.scal[6]; sf = I.scal[7]; sg = I.scal[8]; nB = I.scal[9];
        nrow_hist = I.status[1]; nretry = I.status[2]; nfact = I.status[3];
        for (int k = 0; k < NSEC; ++k) tsec[k] = (long long)I.scal[SCAL_SEC + k];
        ntrsv = (long long)I.scal[SCAL_NTRSV]; ngemv = (long long)I.scal[SCAL_NGEMV];
    }
    __device__ void save() {
        if (threadIdx.x == 0) {
            I.scal[5] = nf; I.scal[6] = ng; I.scal[7] = sf; I.scal[8] = sg; I.scal[9] = nB;
            I.status[1] = nrow_hist; I.status[2] = nretry; I.status[3] = nfact;
            I.status[4] = nfp32; I.status[5] = nfallback; I.status[6] = switched;
            for (int k = 0; k < NSEC; ++k) I.scal[SCAL_SEC + k] = (double)tsec[k];
            I.scal[SCAL_NTRSV] = (double)ntrsv; I.scal[SCAL_NGEMV] = (double)ngemv;
            I.scal[SCAL_STALL0] = (double)stall0;
        }
        __syncthreads();
    }

    // ---- set-up --------------------------------------------------------------------------
    // Ruiz equilibration  (src/IPM/src/scaling/scaling.jl:52-184).  Q = blockdiag(Qd) + Qo.
    __device__ void equilibrate(int itmax, double tol) {
        const DevSp& B = I.B; const DevSp& Q = I.Q;
        const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
        double* rnrm = tm1; double* rswp = tm2; double* cmax = tn;
        for (int v = tid; v < nv; v += NT) { vscl[v] = 1; vswp[v] = 1; }
        for (int i = tid; i < m; i += NT) { rswp[i] = 1; I.yscl[i] = 1; }
        __syncthreads();
        // column j's largest |entry| over B, Q's off-diagonal blocks and its Qd block column (skipped when the
        // block is zero), over the entries l0, l0 + step, ...
        auto colmax = [&](int j, int l0, int step) {
            double mx = 0;
            for (int k = B.cptr[j] + l0; k < B.cptr[j + 1]; k += step) mx = fmax(mx, fabs(B.val[B.cpos[k]]));
            for (int k = Q.cptr[j] + l0; k < Q.cptr[j + 1]; k += step) mx = fmax(mx, fabs(Q.val[Q.cpos[k]]));
            if (!(I.hflag[j] & 2)) {
                const int v = I.colvtx[j], c0 = I.xcol[v], nc = I.xcol[v + 1] - c0;
                const double* qd = I.Qd + I.hdoff[v] + (int64_t)(j - c0) * nc;
                for (int r = l0; r < nc; r += step) mx = fmax(mx, fabs(qd[r]));
            }
            return mx;
        };
        auto longcol = [&](int j) { return B.cptr[j + 1] - B.cptr[j] > LONG_ROW || (I.hflag[j] & 1); };
        for (int it = 0; it < itmax; ++it) {
            // infnorms!: row maxima of B; column maxima of B, Qo and the Qd blocks.  A thread per short row or
            // column, a warp per long one (maxima do not depend on the order)
            for (int i = tid; i < m; i += NT) {
                const int k0 = B.rptr[i], k1 = B.rptr[i + 1];
                if (k1 - k0 > LONG_ROW) continue;
                double mx = 0;
                for (int k = k0; k < k1; ++k) mx = fmax(mx, fabs(B.val[k]));
                rnrm[i] = mx;
            }
            for (int t = warp; t < B.nlongr; t += NW) {
                const int i = B.longr[t];
                double mx = 0;
                for (int k = B.rptr[i] + lane; k < B.rptr[i + 1]; k += 32) mx = fmax(mx, fabs(B.val[k]));
                mx = warp_max(mx);
                if (lane == 0) rnrm[i] = mx;
            }
            for (int j = tid; j < n; j += NT) if (!longcol(j)) cmax[j] = colmax(j, 0, 1);
            for (int t = warp; t < B.nlongc + I.nhlong; t += NW) {
                const int j = t < B.nlongc ? B.longc[t] : I.hlong[t - B.nlongc];
                if (t >= B.nlongc && B.cptr[j + 1] - B.cptr[j] > LONG_ROW) continue;   // listed twice: done above
                const double mx = warp_max(colmax(j, lane, 32));
                if (lane == 0) cmax[j] = mx;
            }
            __syncthreads();
            double dd = 0;
            for (int v = tid; v < nv; v += NT) {
                double mx = 0;
                for (int j = I.xcol[v]; j < I.xcol[v + 1]; ++j) mx = fmax(mx, cmax[j]);
                double nn = sqrt(mx);
                dd = fmax(dd, fabs(1.0 - nn));
                if (nn != 0) { vswp[v] = 1.0 / nn; vscl[v] *= vswp[v]; }
            }
            for (int i = tid; i < m; i += NT) {
                double nn = sqrt(rnrm[i]);
                dd = fmax(dd, fabs(1.0 - nn));
                if (nn != 0) { rswp[i] = 1.0 / nn; I.yscl[i] *= rswp[i]; }
            }
            dd = block_reduce(dd, red, OpMax(), 0.0);
            // applyscaling!: B ← E B D, Q ← D Q D (each entry once, in any order)
            for (int i = tid; i < m; i += NT) {
                const int k0 = B.rptr[i], k1 = B.rptr[i + 1];
                if (k1 - k0 > LONG_ROW) continue;
                for (int k = k0; k < k1; ++k) B.val[k] *= rswp[i] * vswp[I.colvtx[B.cidx[k]]];
            }
            for (int t = warp; t < B.nlongr; t += NW) {
                const int i = B.longr[t];
                for (int k = B.rptr[i] + lane; k < B.rptr[i + 1]; k += 32) B.val[k] *= rswp[i] * vswp[I.colvtx[B.cidx[k]]];
            }
            for (int i = tid; i < n; i += NT) {
                const double su = vswp[I.colvtx[i]];
                for (int k = Q.rptr[i]; k < Q.rptr[i + 1]; ++k) Q.val[k] *= su * vswp[I.colvtx[Q.cidx[k]]];
            }
            for_vertex_blocks(I.xcol, nv, [&](int v) { return !(I.hflag[I.xcol[v]] & 2); },   // a zero block stays
                              [&](int v, int, int t) { I.Qd[I.hdoff[v] + t] *= vswp[v] * vswp[v]; });
            if (dd < tol) break;
        }
        for (int j = tid; j < n; j += NT) { I.pscl[j] = vscl[I.colvtx[j]]; I.f[j] *= I.pscl[j]; }
        for (int i = tid; i < m; i += NT) I.g[i] *= I.yscl[i];
        __syncthreads();
    }

    // row position of scalar column s in front f's row list
    __device__ int rowpos(int f, int s) const {
        int r0 = I.fres0[f], nres = I.fnres[f];
        if (s >= r0 && s < r0 + nres) return s - r0;
        int lo = I.fsepp[f], hi = I.fsepp[f + 1];
        while (lo < hi) { int md = (lo + hi) >> 1; if (I.fsep[md] < s) lo = md + 1; else hi = md; }
        return nres + (lo - I.fsepp[f]);
    }
    __device__ int64_t fpos(int i, int j) const {   // offset in F of entry (i, j), i >= j
        int f = I.cfront[j];
        const int64_t ld = front_ld(I.fnres[f] + I.fnsep[f]);
        return I.fptr[f] + rowpos(f, i) + (int64_t)(j - I.fres0[f]) * ld;
    }

    // Finit ← lower part of BᵀB in front layout  (uzawa.jl:29 `B' * B`; gemm.jl:48-82; chordal.jl:1-80).
    // Rows of B are accumulated one after another (fixed summation order); within a row every
    // nonzero pair (a >= b) is owned by one thread.
    __device__ void build_finit() {
        const DevSp& B = I.B;
        const int tid = threadIdx.x;
        if (COOP && coop && I.fsize >= ((int64_t)1 << 20)) {
            coop_call(coop, sh, [&](CoopCtl* c) { c->cmd = COOP_FILL; c->pa[0] = I.Finit; c->la[0] = I.fsize; });
        } else {
            for (int64_t i = tid; i < I.fsize; i += NT) I.Finit[i] = 0;
            __syncthreads();
        }
        for (int r = 0; r < m; ++r) {
            const int k0 = B.rptr[r], nz = B.rptr[r + 1] - k0;
            const int np = nz * (nz + 1) / 2;
            for (int t = tid; t < np; t += NT) {
                int a = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
                while ((a + 1) * (a + 2) / 2 <= t) ++a;
                while (a * (a + 1) / 2 > t) --a;
                int b = t - a * (a + 1) / 2;
                int ca = B.cidx[k0 + a], cb = B.cidx[k0 + b];
                I.Finit[fpos(ca, cb)] += B.val[k0 + a] * B.val[k0 + b];
            }
            if (np) __syncthreads();
        }
    }

    // y <- alpha (blockdiag(D) + Qo) x + beta y with D = Qd (the data Q) or Hd (the scaled H)
    __device__ void amul(const double* Dblk, const double* x, double* y, double alpha, double beta) {
        const DevSp& Q = I.Q;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const bool isH = Dblk == I.Hd;
        if (isH && nsocz > 0) {   // zᵀx of the structured SOC cones, (W ⊗ₛ W) x of the structured SDP cones
            for (int v = warp; v < nv; v += NW) {
                if (vsocz[v] != 1.0) continue;
                const int c0 = I.xcol[v];
                const double s = w_soczdot(I.cache + I.cxblk[v], x + c0, I.xcol[v + 1] - c0);
                if (lane == 0) vsocdot[v] = s;
            }
            for (int v = 0; v < nv; ++v) {
                if (vsocz[v] != 2.0) continue;
                const int c0 = I.xcol[v], nc = I.xcol[v + 1] - c0, d = sdp_triroot(nc);
                b_sdphx(hx + c0, I.cache + I.cxblk[v] + 2 * (int64_t)d * d + d, x + c0, nc, I.work);
            }
            __syncthreads();
        }
        auto head = [&](int i, double acc) {   // y[i] from the row's sum
            y[i] = beta == 0.0 ? alpha * acc : fma(alpha, acc, beta * y[i]);
        };
        // rows with at most LONG_ROW terms: a thread each (I.hflag marks the others)
        for (int i = threadIdx.x; i < n; i += NT) {
            if (I.hflag[i] & 1) continue;
            const int v = I.colvtx[i], c0 = I.xcol[v], nc = I.xcol[v + 1] - c0;
            double acc = 0;
            if (nsocz > 0 && vsocz[v] != 0.0) {   // zero Q block: H in structured form, Qd block skipped
                if (isH) acc = vsocz[v] == 1.0 ? socz_row(I.cache + I.cxblk[v], x + c0, i - c0, vsocdot[v]) : hx[i];
            } else {
                const double* row = Dblk + I.hdoff[v] + (int64_t)(i - c0) * nc;   // symmetric: row = column
                for (int j = 0; j < nc; ++j) acc = fma(row[j], x[c0 + j], acc);
            }
            for (int k = Q.rptr[i]; k < Q.rptr[i + 1]; ++k) acc = fma(Q.val[k], x[Q.cidx[k]], acc);
            head(i, acc);
        }
        // longer rows (I.hlong): a warp each
        for (int t = warp; t < I.nhlong; t += NW) {
            const int i = I.hlong[t];
            const int v = I.colvtx[i], c0 = I.xcol[v], nc = I.xcol[v + 1] - c0;
            double acc = 0;
            if (nsocz > 0 && vsocz[v] != 0.0) {
                if (isH && lane == 0) acc = vsocz[v] == 1.0 ? socz_row(I.cache + I.cxblk[v], x + c0, i - c0, vsocdot[v]) : hx[i];
            } else {
                const double* row = Dblk + I.hdoff[v] + (int64_t)(i - c0) * nc;
                for (int j = lane; j < nc; j += 32) acc = fma(row[j], x[c0 + j], acc);
            }
            for (int k = Q.rptr[i] + lane; k < Q.rptr[i + 1]; k += 32) acc = fma(Q.val[k], x[Q.cidx[k]], acc);
            acc = warp_sum(acc);
            if (lane == 0) head(i, acc);
        }
        __syncthreads();
    }

    // d*(p) for every cone, dst ≠ src (dualshadow!, cone.jl:562-608)
    __device__ void dualshadow_all(double* dst, const double* src) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int v = warp; v < nv; v += NW) {
            const int k = I.kind[v], c0 = I.xcol[v], nc = I.xcol[v + 1] - c0;
            if (k == CONE_POS) { for (int i = lane; i < nc; i += 32) dst[c0 + i] = 1.0 / src[c0 + i]; }
            else if (k == CONE_SOC) w_socshadow(dst + c0, src + c0, nc);
            else if (k == CONE_EXP || k == CONE_POW) {
                if (lane == 0) tddualshadow(TD{k, I.kpar[v]}, dst + c0, src + c0, I.cache + I.cxblk[v]);
                __syncwarp();
            } else if (k != CONE_SDP) { for (int i = lane; i < nc; i += 32) dst[c0 + i] = 0; }
        }
        __syncthreads();
        for (int v = 0; v < nv; ++v) {
            if (I.kind[v] != CONE_SDP) continue;
            const int c0 = I.xcol[v], nc = I.xcol[v + 1] - c0;
            b_sdpshadow(dst + c0, src + c0, nc, I.work, SdpSh{red, &sh.flag});
        }
        __syncthreads();
    }

    // r = F2(p) dp, the second derivative of the barrier per cone (primalhess!, cone.jl:579-591):
    // pos.jl:193-203, soc.jl:510-530 (det(p) from the cache), tdc.jl:509-511 (the cached factor L),
    // sdp.jl:696-742 (the cached R); free: 0
    __device__ void primalhess_all(double* r, const double* pv, const double* dp) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int v = warp; v < nv; v += NW) {
            const int k = I.kind[v], c0 = I.xcol[v], nc = I.xcol[v + 1] - c0;
            const double* C = I.cache + I.cxblk[v];
            if (k == CONE_POS) {
                for (int i = lane; i < nc; i += 32) { const double q = pv[c0 + i]; r[c0 + i] = dp[c0 + i] / (q * q); }
            } else if (k == CONE_SOC) {
                double hi, lo;
                w_socdot(pv + c0, dp + c0, nc, hi, lo);
                const double pdet = C[1], t = hi / pdet, gm = 2 / pdet, t2 = 2 * t;
                for (int i = lane; i < nc; i += 32)
                    r[c0 + i] = i == 0 ? gm * fma(t2, pv[c0], -dp[c0]) : gm * fma(-t2, pv[c0 + i], dp[c0 + i]);
            } else if (k == CONE_EXP || k == CONE_POW) {
                if (lane == 0) tdhessmul(r + c0, C + TD_L, dp + c0);
            } else if (k != CONE_SDP) {
                for (int i = lane; i < nc; i += 32) r[c0 + i] = 0;
            }
            __syncwarp();
        }
        __syncthreads();
        for (int v = 0; v < nv; ++v) {
            if (I.kind[v] != CONE_SDP) continue;
            const int c0 = I.xcol[v], nc = I.xcol[v + 1] - c0, d = sdp_triroot(nc);
            const double* R = I.cache + I.cxblk[v];
            double *U = I.work, *A = I.work + (int64_t)d * d;
            b_smat(U, dp + c0, d, true);
            b_mul(A, R, true, U, false, d);  b_mul(U, A, false, R, false, d);    // Ũ = Rᵀ U R
            b_mul(A, R, false, U, false, d); b_mul(U, A, false, R, true, d);     // R Ũ Rᵀ
            b_svec(r + c0, U, d);
        }
        __syncthreads();
    }

    // r = F3(p)[u, w], the third derivative of the barrier per cone (primalthird!, cone.jl:595-607):
    // pos.jl:209-219, soc.jl:535-560, tdc.jl:517-521, sdp.jl:747-790; free: 0
    __device__ void primalthird_all(double* r, const double* pv, const double* u, const double* w) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int v = warp; v < nv; v += NW) {
            const int k = I.kind[v], c0 = I.xcol[v], nc = I.xcol[v + 1] - c0;
            const double* C = I.cache + I.cxblk[v];
            if (k == CONE_POS) {
                for (int i = lane; i < nc; i += 32) {
                    const double q = pv[c0 + i];
                    r[c0 + i] = -2 * u[c0 + i] * w[c0 + i] / (q * q * q);
                }
            } else if (k == CONE_SOC) {
                double a1, a2, a3, lo;
                w_socdot(pv + c0, u + c0, nc, a1, lo);
                w_socdot(pv + c0, w + c0, nc, a2, lo);
                w_socdot(u + c0, w + c0, nc, a3, lo);
                const double pdet = C[1], u1 = a1 / pdet, u2 = a2 / pdet, vv = a3 / pdet, gm = 4 / pdet;
                const double cc = fma(-4 * u1, u2, vv);
                for (int i = lane; i < nc; i += 32) {
                    const double t = fma(u1, w[c0 + i], fma(u2, u[c0 + i], cc * pv[c0 + i]));
                    r[c0 + i] = i == 0 ? gm * t : -gm * t;
                }
            } else if (k == CONE_EXP || k == CONE_POW) {
                if (lane == 0) {
                    double D[9];
                    tdbarrthird(TD{k, I.kpar[v]}, D, pv + c0, u + c0, C);
                    for (int i = 0; i < 3; ++i)
                        r[c0 + i] = D[i] * w[c0] + D[i + 3] * w[c0 + 1] + D[i + 6] * w[c0 + 2];
                }
            } else if (k != CONE_SDP) {
                for (int i = lane; i < nc; i += 32) r[c0 + i] = 0;
            }
            __syncwarp();
        }
        __syncthreads();
        for (int v = 0; v < nv; ++v) {
            if (I.kind[v] != CONE_SDP) continue;
            const int c0 = I.xcol[v], nc = I.xcol[v + 1] - c0, d = sdp_triroot(nc);
            const int64_t q = (int64_t)d * d;
            const double* R = I.cache + I.cxblk[v];
            double *U = I.work, *V = I.work + q, *A = I.work + 2 * q;
            b_smat(U, u + c0, d, true);
            b_smat(V, w + c0, d, true);
            b_mul(A, R, true, U, false, d); b_mul(U, A, false, R, false, d);     // Ũ
            b_mul(A, R, true, V, false, d); b_mul(V, A, false, R, false, d);     // Ṽ
            b_mul(A, U, false, V, false, d);                                     // Ũ Ṽ
            for (int t = threadIdx.x; t < d * d; t += NT) {                      // Ũ Ṽ + Ṽ Ũ, into V
                const int i = t % d, j = t / d;
                V[t] = i == j ? 2 * A[t] : A[t] + A[j + (int64_t)i * d];
            }
            __syncthreads();
            b_mul(U, R, false, V, false, d); b_mul(A, U, false, R, true, d);     // R (Ũ Ṽ + Ṽ Ũ) Rᵀ
            b_svec(r + c0, A, d);
            for (int i = threadIdx.x; i < nc; i += NT) r[c0 + i] = -r[c0 + i];
            __syncthreads();
        }
        __syncthreads();
    }

    // frule2! (ipm/differential.jl:82-260): two first-order solves, then the second-order solve on
    // -(μ′ F3(p)[Δp1, Δp2] + Δμ1 F2(p) Δp2 + Δμ2 F2(p) Δp1); the exchange layout is DevInst::sx's
    __device__ void sensitivity2() {
        double* f1 = I.sx; double* g1 = f1 + n; double* f2 = g1 + m; double* g2 = f2 + n;
        double* o = g2 + m;                                  // p1 y1 d1 p2 y2 d2 p12 y12 d12
        double *op1 = o, *oy1 = op1 + n, *od1 = oy1 + m, *op2 = od1 + n, *oy2 = op2 + n, *od2 = oy2 + m;
        double *op12 = od2 + n, *oy12 = op12 + n, *od12 = oy12 + m, *ss = od12 + n;
        use32 = false;
        const double dl = getaug();
        double rho;
        if (!initkkt(dl, rho)) { if (threadIdx.x == 0) ss[2] = 0; __syncthreads(); return; }
        const double mu0 = nrow_hist > 0 ? hrow(0).mu : 0.0;
        const double tol = mu0 == 0 ? 0.1 * set.gap_tol : 0.1 * hrow(nrow_hist - 1).mu / mu0;
        const double ftol = tol * (1 + nf), gtol = tol * (1 + ng);
        const double dmu1 = ss[0], dmu2 = ss[1];
        double* ds = Dd;           // d*(p), then F2 scratch
        double* fx = wf; double* gx = Dg;
        double* p1 = Dpa; double* y1 = Dya; double* d1 = Dda;
        double* p2 = Dp; double* y2 = Dy; double* d2 = df;
        dualshadow_all(ds, I.p);
        for (int set2 = 0; set2 < 2; ++set2) {
            const double* fs = set2 ? f2 : f1; const double* gs = set2 ? g2 : g1;
            const double dm = set2 ? dmu2 : dmu1;
            double* px = set2 ? p2 : p1; double* yx = set2 ? y2 : y1; double* dx = set2 ? d2 : d1;
            for (int i = threadIdx.x; i < n; i += NT) fx[i] = fma(dm, ds[i], fs[i] * I.pscl[i]);
            for (int i = threadIdx.x; i < m; i += NT) gx[i] = gs[i] * I.yscl[i];
            __syncthreads();
            solvekkt(0, px, yx, I.Hd, fx, gx, false, ftol, gtol, 1);
            amul(I.Hd, px, dx, 1, 0);                      // Δd = Δμ d* - (H - Q) Δp
            amul(I.Qd, px, dx, -1, 1);
            for (int i = threadIdx.x; i < n; i += NT) dx[i] = fma(dm, ds[i], -dx[i]);
            __syncthreads();
        }
        primalthird_all(fx, I.p, p1, p2);
        for (int i = threadIdx.x; i < n; i += NT) fx[i] *= I.mut;
        __syncthreads();
        if (dmu1 != 0) {
            primalhess_all(ds, I.p, p2);
            for (int i = threadIdx.x; i < n; i += NT) fx[i] = fma(dmu1, ds[i], fx[i]);
            __syncthreads();
        }
        if (dmu2 != 0) {
            primalhess_all(ds, I.p, p1);
            for (int i = threadIdx.x; i < n; i += NT) fx[i] = fma(dmu2, ds[i], fx[i]);
            __syncthreads();
        }
        for (int i = threadIdx.x; i < n; i += NT) {
            fx[i] = -fx[i];
            op1[i] = p1[i] * I.pscl[i]; od1[i] = d1[i] / I.pscl[i];
            op2[i] = p2[i] * I.pscl[i]; od2[i] = d2[i] / I.pscl[i];
        }
        for (int i = threadIdx.x; i < m; i += NT) { oy1[i] = y1[i] * I.yscl[i]; oy2[i] = y2[i] * I.yscl[i]; gx[i] = 0; }
        __syncthreads();
        solvekkt(0, p2, y2, I.Hd, fx, gx, false, ftol, gtol, 1);
        amul(I.Hd, p2, fx, -1, 1);                         // Δd12 = rhs - (H - Q) Δp12
        amul(I.Qd, p2, fx, 1, 1);
        for (int i = threadIdx.x; i < n; i += NT) { op12[i] = p2[i] * I.pscl[i]; od12[i] = fx[i] / I.pscl[i]; }
        for (int i = threadIdx.x; i < m; i += NT) oy12[i] = y2[i] * I.yscl[i];
        if (threadIdx.x == 0) ss[2] = 1;
        __syncthreads();
    }

    // frule! / rrule! (ipm/differential.jl:5-79, 263-334) at the current iterate: δ = getaug, an FP64
    // factorization, one KKT solve (cold, at least one refinement pass), the rest H/Q products and the
    // dual shadow.  Seeds and results in I.sx (solver order, unscaled); sx[4n+2m+2] = 1 on success.
    __device__ void sensitivity(bool reverse) {
        double* sa = I.sx; double* sb = sa + n; double* sc = sb + m;
        double* oa = sc + n; double* ob = oa + n; double* oc = ob + m; double* ss = oc + n;
        use32 = false;
        const double dl = getaug();
        double rho;
        if (!initkkt(dl, rho)) { if (threadIdx.x == 0) ss[2] = 0; __syncthreads(); return; }
        const double mu0 = nrow_hist > 0 ? hrow(0).mu : 0.0;
        const double tol = mu0 == 0 ? 0.1 * set.gap_tol : 0.1 * hrow(nrow_hist - 1).mu / mu0;
        const double ftol = tol * (1 + nf), gtol = tol * (1 + ng);
        if (!reverse) {
            const double dmu = ss[0];
            for (int i = threadIdx.x; i < n; i += NT) wf[i] = sa[i] * I.pscl[i];
            for (int i = threadIdx.x; i < m; i += NT) Dg[i] = sb[i] * I.yscl[i];
            __syncthreads();
            dualshadow_all(Dd, I.p);
            for (int i = threadIdx.x; i < n; i += NT) { Dd[i] *= dmu; wf[i] += Dd[i]; }
            __syncthreads();
            solvekkt(0, Dp, Dy, I.Hd, wf, Dg, false, ftol, gtol, 1);
            amul(I.Hd, Dp, Dd, -1, 1);                 // Δd = Δμ d* − (H − Q) Δp
            amul(I.Qd, Dp, Dd, 1, 1);
            for (int i = threadIdx.x; i < n; i += NT) { oa[i] = Dp[i] * I.pscl[i]; oc[i] = Dd[i] / I.pscl[i]; }
            for (int i = threadIdx.x; i < m; i += NT) ob[i] = Dy[i] * I.yscl[i];
        } else {
            for (int i = threadIdx.x; i < n; i += NT) { wf[i] = sa[i] * I.pscl[i]; Dd[i] = sc[i] / I.pscl[i]; }
            for (int i = threadIdx.x; i < m; i += NT) Dg[i] = sb[i] * -I.yscl[i];
            __syncthreads();
            amul(I.Hd, Dd, wf, -1, 1);                 // Δp −= (H − Q) Δd
            amul(I.Qd, Dd, wf, 1, 1);
            solvekkt(0, Dp, Dy, I.Hd, wf, Dg, false, ftol, gtol, 1);
            for (int i = threadIdx.x; i < n; i += NT) { Dd[i] += Dp[i]; oa[i] = Dp[i] * I.pscl[i]; }
            for (int i = threadIdx.x; i < m; i += NT) ob[i] = -Dy[i] * I.yscl[i];
            __syncthreads();
            dualshadow_all(wf, I.p);
            const double dm = bdot(Dd, wf, n, red);
            if (threadIdx.x == 0) ss[1] = dm;
        }
        if (threadIdx.x == 0) ss[2] = 1;
        __syncthreads();
    }

    // vsocz / nsocz: SOC and SDP vertices whose diagonal block of Q is zero (not stored: qd0off < 0)
    __device__ void mark_socz() {
        int cnt = 0;
        for (int v = threadIdx.x; v < nv; v += NT) {
            const int k = I.kind[v];
            const bool st = (k == CONE_SOC || k == CONE_SDP) && I.qd0off[v] < 0;
            vsocz[v] = st ? (k == CONE_SOC ? 1 : 2) : 0;
            cnt += st;
        }
        cnt = (int)block_reduce((double)cnt, red, OpSum(), 0.0);
        nsocz = cnt;
        if (threadIdx.x == 0) I.scal[SCAL_NSOCZ] = (double)cnt;
        __syncthreads();
    }

    __device__ void startingpoint() {  // solver/ipm.jl:331-365
        const int warp = threadIdx.x >> 5;
        for (int v = warp; v < nv; v += NW) {
            int k = I.kind[v];
            int c0 = I.xcol[v], nc = I.xcol[v + 1] - c0;
            if (k == CONE_EXP || k == CONE_POW) {
                if ((threadIdx.x & 31) == 0) { tdidentity(TD{k, I.kpar[v]}, I.p + c0); tdidentity(TD{k, I.kpar[v]}, I.d + c0); }
                __syncwarp();
                continue;
            }
            if (k == CONE_SDP) { w_sdpidentity(I.p + c0, nc); w_sdpidentity(I.d + c0, nc); continue; }
            w_identity(k, nc, I.p + c0);
            w_identity(k, nc, I.d + c0);
        }
        __syncthreads();
        spmv(I.B, I.p, tm1, 1, 0);
        amul(I.Qd, I.p, tn, 1, 0);
        const double eps = 2.220446049250313e-16;
        double np = bnorm(I.p, n, red), nz = bnorm(tm1, m, red), nw = bnorm(tn, n, red);
        double sp = nz > eps * np ? fmax(1.0, bnorm(I.g, m, red) / nz) : 1.0;
        double sd = np > eps ? fmax(1.0, (bnorm(I.f, n, red) + sp * nw) / np) : 1.0;
        for (int i = threadIdx.x; i < n; i += NT) { I.p[i] *= sp; I.d[i] *= sd; }
        __syncthreads();
    }

    // ---- cone fan-outs  (cone/cone.jl:146-553) -------------------------------------------
    __device__ bool scale_all(double& spsd_sum) {
        const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
        // H_vv ← Q_vv for every cone block (cone.jl:146-174); SOC blocks are written below and
        // structured SDP blocks are assigned by b_sdpscale
        for_vertex_blocks(I.xcol, nv,
                          [&](int v) { return !(I.kind[v] == CONE_FREE || I.kind[v] == CONE_SOC || vsocz[v] == 2.0); },
                          [&](int v, int, int t) { I.Hd[I.hdoff[v] + t] = I.Qd[I.hdoff[v] + t]; });
        // per cone: scaling point and ⟨p*, d*⟩
        for (int v = warp; v < nv; v += NW) {
            int k = I.kind[v];
            int c0 = I.xcol[v], nc = I.xcol[v + 1] - c0;
            double sp = 0; bool fl = true;
            const double* p = I.p + c0; const double* d = I.d + c0;
            if (k == CONE_POS) {   // pos.jl:75-84
                double* Hv = I.Hd + I.hdoff[v];
                double s = 0;
                for (int i = lane; i < nc; i += 32) { Hv[i + (int64_t)i * nc] += d[i] / p[i]; s += 1.0 / (p[i] * d[i]); }
                sp = warp_sum(s);
            } else if (k == CONE_SOC) {
                fl = w_socpoint(I.cache + I.cxblk[v], p, d, nc, sp);
            } else if (k == CONE_EXP || k == CONE_POW || k == CONE_SDP) {
                continue;
            }
            if (lane == 0) { vflag[v] = fl ? 1.0 : 0.0; vspsd[v] = sp; }
        }
        // exponential / power cones: one thread per cone (tdc.jl:186-294)
        for (int v = tid; v < nv; v += NT) {
            int k = I.kind[v];
            if (k != CONE_EXP && k != CONE_POW) continue;
            int c0 = I.xcol[v];
            double sp = 0;
            bool fl = tdscale(TD{k, I.kpar[v]}, I.Hd + I.hdoff[v], I.p + c0, I.d + c0, I.cache + I.cxblk[v], sp);
            vflag[v] = fl ? 1.0 : 0.0; vspsd[v] = sp;
        }
        __syncthreads();
        // semidefinite cones: the whole block per cone (sdp.jl:121-263)
        for (int v = 0; v < nv; ++v) {
            if (I.kind[v] != CONE_SDP) continue;
            int c0 = I.xcol[v], nc = I.xcol[v + 1] - c0;
            double sp = 0;
            bool fl = b_sdpscale(I.Hd + I.hdoff[v], nc, I.cache + I.cxblk[v], I.p + c0, I.d + c0, I.work, sp,
                                 SdpSh{red, &sh.flag, sh.tile, XSM_CAP}, vsocz[v] == 2.0);
            if (threadIdx.x == 0) { vflag[v] = fl ? 1.0 : 0.0; vspsd[v] = sp; }
        }
        __syncthreads();
        // SOC Hessian blocks H = Q + (2 (Jw)(Jw)ᵀ − J) / β² (soc.jl:231-256); H = Q where the scaling failed
        for (int v = 0; v < nv; ++v) {
            if (I.kind[v] != CONE_SOC) continue;
            int nc = I.xcol[v + 1] - I.xcol[v];
            const double* q = I.Qd + I.hdoff[v];
            double* h = I.Hd + I.hdoff[v];
            if (vflag[v] == 0.0) { for (int t = tid; t < nc * nc; t += NT) h[t] = q[t]; }
            else b_sochess(h, q, vsocz[v] != 0.0, I.cache + I.cxblk[v], nc);
        }
        __syncthreads();
        double ok = 1, s = 0;
        for (int v = threadIdx.x; v < nv; v += NT) { ok = fmin(ok, vflag[v]); s += vspsd[v]; }
        ok = block_reduce(ok, red, OpMin(), 1.0);
        spsd_sum = block_reduce(s, red, OpSum(), 0.0);
        return ok > 0;
    }

    __device__ void initcorrector(double* fr, const double* Dpv, const double* Ddv, double sm) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        double* work = I.work + (int64_t)warp * I.wsize;
        for (int v = warp; v < nv; v += NW) {
            int k = I.kind[v];
            int c0 = I.xcol[v], nc = I.xcol[v + 1] - c0;
            if (k == CONE_POS) {   // pos.jl:107-120
                for (int i = lane; i < nc; i += 32) fr[c0 + i] = (sm - Dpv[c0 + i] * Ddv[c0 + i]) / I.p[c0 + i] - I.d[c0 + i];
            } else if (k == CONE_SOC) {
                w_soccorr(fr + c0, I.cache + I.cxblk[v], I.p + c0, Dpv + c0, Ddv + c0, sm, nc, work);
            } else if (k == CONE_FREE) {
                for (int i = lane; i < nc; i += 32) fr[c0 + i] = 0;
            }
        }
        for (int v = threadIdx.x; v < nv; v += NT) {   // tdc.jl:394-438
            int k = I.kind[v];
            if (k != CONE_EXP && k != CONE_POW) continue;
            int c0 = I.xcol[v];
            tdcorr(TD{k, I.kpar[v]}, fr + c0, I.p + c0, I.d + c0, Dpv + c0, Ddv + c0, sm, I.cache + I.cxblk[v]);
        }
        __syncthreads();
        for (int v = 0; v < nv; ++v) {   // sdp.jl:293-431, the whole block per cone
            if (I.kind[v] != CONE_SDP) continue;
            int c0 = I.xcol[v], nc = I.xcol[v + 1] - c0;
            b_sdpcorr(fr + c0, I.cache + I.cxblk[v], Dpv + c0, Ddv + c0, sm, nc, I.work);
        }
    }

    __device__ void initpredictor(double* fr, double sm) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int v = warp; v < nv; v += NW) {
            int k = I.kind[v];
            int c0 = I.xcol[v], nc = I.xcol[v + 1] - c0;
            if (k == CONE_POS) {   // pos.jl:126-137
                for (int i = lane; i < nc; i += 32) fr[c0 + i] = sm / I.p[c0 + i] - I.d[c0 + i];
            } else if (k == CONE_SOC) {
                w_soccorr0(fr + c0, I.cache + I.cxblk[v], I.p + c0, sm, nc);
            } else if (k == CONE_FREE) {
                for (int i = lane; i < nc; i += 32) fr[c0 + i] = 0;
            }
        }
        for (int v = threadIdx.x; v < nv; v += NT) {   // tdc.jl:446-450
            int k = I.kind[v];
            if (k != CONE_EXP && k != CONE_POW) continue;
            int c0 = I.xcol[v];
            tdcorr0(fr + c0, I.d + c0, sm, I.cache + I.cxblk[v]);
        }
        __syncthreads();
        for (int v = 0; v < nv; ++v) {   // sdp.jl:437-510
            if (I.kind[v] != CONE_SDP) continue;
            int c0 = I.xcol[v], nc = I.xcol[v + 1] - c0;
            b_sdpcorr0(fr + c0, I.cache + I.cxblk[v], sm, nc, I.work);
        }
    }

    __device__ double maxsteps(const double* Dpv, const double* Ddv, double step_frac) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int v = warp; v < nv; v += NW) {
            int k = I.kind[v];
            int c0 = I.xcol[v], nc = I.xcol[v + 1] - c0;
            double tp = 1, td = 1;
            if (k == CONE_POS) {
                tp = w_posmaxstep(I.p + c0, Dpv + c0, nc);
                td = w_posmaxstep(I.d + c0, Ddv + c0, nc);
            } else if (k == CONE_SOC) {
                const double* c = I.cache + I.cxblk[v];
                tp = w_socmaxstep(I.p + c0, Dpv + c0, c[1], c[3], nc);
                td = w_socmaxstep(I.d + c0, Ddv + c0, c[2], c[4], nc);
            }
            if (k == CONE_EXP || k == CONE_POW || k == CONE_SDP) continue;
            if (k != CONE_FREE) { tp *= step_frac; td *= step_frac; }
            if (lane == 0) vstep[v] = jmin(tp, td);
        }
        for (int v = threadIdx.x; v < nv; v += NT) {   // tdc.jl:463-483 (certified nflog3 steps)
            int k = I.kind[v];
            if (k != CONE_EXP && k != CONE_POW) continue;
            int c0 = I.xcol[v];
            double tp = 1, td = 1;
            tdmaxsteps(TD{k, I.kpar[v]}, I.p + c0, Dpv + c0, I.d + c0, Ddv + c0, I.cache + I.cxblk[v], tp, td);
            vstep[v] = jmin(tp * step_frac, td * step_frac);
        }
        __syncthreads();
        for (int v = 0; v < nv; ++v) {   // sdp.jl:516-519: τp through R, τd through S and Σ
            if (I.kind[v] != CONE_SDP) continue;
            int c0 = I.xcol[v], nc = I.xcol[v + 1] - c0;
            const double* c = I.cache + I.cxblk[v];
            const int64_t dd = sdp_triroot(nc);
            double tp = b_sdpmaxstep(c, Dpv + c0, nullptr, nc, I.work, SdpSh{red, &sh.flag, sh.tile, XSM_CAP});
            double td = b_sdpmaxstep(c + dd * dd, Ddv + c0, c + 2 * dd * dd, nc, I.work, SdpSh{red, &sh.flag, sh.tile, XSM_CAP});
            if (threadIdx.x == 0) vstep[v] = jmin(tp * step_frac, td * step_frac);
        }
        __syncthreads();
        double mn = __longlong_as_double(0x7ff0000000000000LL);
        for (int v = threadIdx.x; v < nv; v += NT) mn = jmin(mn, vstep[v]);
        mn = block_reduce(mn, red, OpJmin(), __longlong_as_double(0x7ff0000000000000LL));
        return nv == 0 ? 1.0 : mn;
    }

    __device__ void zerofree(double* x) {
        for (int v = threadIdx.x >> 5; v < nv; v += NW)
            if (I.kind[v] == CONE_FREE)
                for (int j = I.xcol[v] + (threadIdx.x & 31); j < I.xcol[v + 1]; j += 32) x[j] = 0;
        __syncthreads();
    }

    // ---- factor  (kkt/uzawa.jl:73-115) ----------------------------------------------------
    __device__ void assemble(double dl, double rho) {
        if (use32) assemble_t<float>(F32, dl, rho); else assemble_t<double>(F64, dl, rho);
    }
    template <class FT>
    __device__ void assemble_t(FT* F, double dl, double rho) {
        const int tid = threadIdx.x;
        if (COOP && coop && I.fsize >= ((int64_t)1 << 20)) {   // the copy F <- Finit shared with the helpers
            coop_call(coop, sh, [&](CoopCtl* c) {
                c->cmd = COOP_COPY; c->pa[0] = F; c->pa[1] = I.Finit; c->la[0] = I.fsize; c->ia[0] = IsF32<FT>::v;
            });
        } else {
            // only the lower triangle of each front is ever read (factor, solves, extend-add, norms):
            // large fronts copy it a warp per column in 16-byte row pairs, from the even row at or
            // above the diagonal (columns start on 16-byte boundaries: even leading dimension, Finit
            // and F aligned) to the padding row of an odd order, so at most one upper-triangle entry,
            // which the factor rewrites before anything reads it, and the unread padding row come
            // along; small fronts are copied whole and flat
            const int lane = tid & 31, warp = tid >> 5;
            for (int f = 0; f < I.nfront; ++f) {
                const int nfr = I.fnres[f] + I.fnsep[f];
                const int64_t ld = front_ld(nfr);
                FT* M = F + I.fptr[f];
                const double* M0 = I.Finit + I.fptr[f];
                if (nfr < 64) {
                    for (int t = tid; t < ld * nfr; t += NT) M[t] = (FT)M0[t];
                    continue;
                }
                for (int j = warp; j < nfr; j += NW) {
                    const int i0 = j & ~1, np = (((nfr + 1) & ~1) - i0) >> 1;
                    const double2* A2 = reinterpret_cast<const double2*>(M0 + (int64_t)j * ld + i0);
                    FT* Mj = M + (int64_t)j * ld + i0;
                    int q = lane;
                    for (; q + 96 < np; q += 128) {
                        const double2 a0 = A2[q], a1 = A2[q + 32], a2 = A2[q + 64], a3 = A2[q + 96];
                        store_pair(Mj, q, a0); store_pair(Mj, q + 32, a1); store_pair(Mj, q + 64, a2); store_pair(Mj, q + 96, a3);
                    }
                    for (; q < np; q += 32) store_pair(Mj, q, A2[q]);
                }
            }
        }
        __syncthreads();
        // + δ H: diagonal blocks (lower part) and the off-diagonal nonzeros of Q (chordal.jl:1-80)
        for_vertex_blocks(I.xcol, nv, [](int) { return true; }, [&](int v, int nc, int t) {
            const int r = t % nc, c = t / nc;
            if (r >= c) {
                const int64_t q = I.hdpos[v] + r + (int64_t)c * I.hdld[v];
                F[q] = (FT)(I.Finit[q] + dl * I.Hd[I.hdoff[v] + t]);
            }
        });
        for (int t = tid; t < I.nqoff; t += NT) {
            int64_t q = I.qoffpos[t];
            F[q] = (FT)(I.Finit[q] + dl * I.Q.val[I.qoffk[t]]);
        }
        __syncthreads();
        if (rho != 0) {
            for (int f = 0; f < I.nfront; ++f) {
                const int nres = I.fnres[f];
                const int64_t ld = front_ld(nres + I.fnsep[f]);
                FT* M = F + I.fptr[f];
                for (int j = tid; j < nres; j += NT) M[j + (int64_t)j * ld] = (FT)((double)M[j + (int64_t)j * ld] + rho);
            }
            __syncthreads();
        }
    }

    __device__ double factor_lower_norm() {
        return use32 ? factor_lower_norm_t<float>(F32) : factor_lower_norm_t<double>(F64);
    }
    template <class FT>
    __device__ double factor_lower_norm_t(const FT* F) {
        double s = 0;
        for (int f = 0; f < I.nfront; ++f) {
            int nres = I.fnres[f], nfr = nres + I.fnsep[f];
            const int64_t ld = front_ld(nfr);
            const FT* M = F + I.fptr[f];
            for (int64_t t = threadIdx.x; t < (int64_t)nres * nfr; t += NT) {
                int i = (int)(t % nfr), j = (int)(t / nfr);
                if (i >= j) { double x = (double)M[i + (int64_t)j * ld]; s += x * x; }
            }
        }
        return sqrt(block_reduce(s, red, OpSum(), 0.0));
    }

    __device__ int numeric_factor() {
        return use32 ? numeric_factor_t<float>(F32) : numeric_factor_t<double>(F64);
    }
    template <class FT>
    __device__ int numeric_factor_t(FT* F) {
        for (int f = 0; f < I.nfront; ++f) {
            int nres = I.fnres[f], nsep = I.fnsep[f], nfr = nres + nsep;
            FT* M = F + I.fptr[f];
            int info = front_chol_ll<FT, COOP>(M, nfr, nres, sh, coop, tsec + SEC_FUPD);
            if (info == COOP_ABORTED) return COOP_ABORTED;
            if (info) return I.fres0[f] + info;
            int p = I.fparent[f];
            if (p >= 0 && nsep > 0) {
                const long long te = tic();
                int np = I.fnres[p] + I.fnsep[p];
                FT* P = F + I.fptr[p];
                const int* rel = I.frel + I.fsepp[f];
                if (COOP && coop && nsep >= COOP_MIN_FRONT) {   // extend-add shared with the helpers
                    if (!coop_call(coop, sh, [&](CoopCtl* c) {
                            c->cmd = COOP_EXTEND; c->pa[0] = M; c->pa[1] = P; c->pa[2] = (void*)rel;
                            c->ia[0] = IsF32<FT>::v; c->ia[1] = nfr; c->ia[2] = nres; c->ia[3] = nsep; c->ia[4] = np;
                        }))
                        return COOP_ABORTED;
                    toc(SEC_FEXTEND, te);
                    continue;
                }
                const int64_t ldc = front_ld(nfr), ldp = front_ld(np);
                for (int j = threadIdx.x >> 5; j < nsep; j += NW) {   // column j of the update matrix per warp
                    const FT* Mj = M + nres + (int64_t)(nres + j) * ldc;
                    FT* Pj = P + (int64_t)rel[j] * ldp;
                    for (int i = j + (threadIdx.x & 31); i < nsep; i += 32) Pj[rel[i]] += Mj[i];
                }
                toc(SEC_FEXTEND, te);
            }
        }
        return 0;
    }

    // ---- stable factor  (kkt/uzawa.jl:117-163; utils.jl:186-200) ----------------------------
    // F Fᵀ = δ H + Bᵀ B without forming BᵀB.  Front by front, the stacked system
    //   W = [ √δ U_v  for the front's vertices (U_vᵀ U_v = H_vv, a Cholesky per nonzero diagonal
    //                 block, as cholblockdiag!; a zero block gives no rows) ;
    //         the rows of B whose first column lies in the front ;
    //         each child's R triangle over its separator ]
    // has WᵀW = the front's part of δH + BᵀB plus what its descendants pass up, and its Householder
    // QR gives R with RᵀR = WᵀW: the front's rows of R, signed to a positive diagonal, are the
    // factor's columns (the rank-m update of √δ·chol(H) by the rows of B that the reference's
    // lowrankupdate! makes, in exact arithmetic), and the trailing triangle goes to the parent,
    // kept in the upper triangle of the front's separator block.  Returns 0, the 1-based column
    // of a zero pivot, or -1 when a nonzero diagonal block of H is not positive definite.  FP64.
    __device__ int stable_factor(double dl) {
        double* F = F64;
        const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
        const double sd = sqrt(dl);
        double* W = I.swork;
        for (int f = 0; f < I.nfront; ++f) {
            const int nres = I.fnres[f], nsep = I.fnsep[f], nfr = nres + nsep, r0 = I.fres0[f];
            const int b0 = I.sbrp[f], nb = I.sbrp[f + 1] - b0;
            int rows = nres + nb;
            for (int k = I.fchp[f]; k < I.fchp[f + 1]; ++k) rows += I.fnsep[I.fch[k]];
            const int64_t ld = rows;
            for (int64_t t = tid; t < ld * nfr; t += NT) W[t] = 0.0;
            __syncthreads();
            // √δ U_v in rows and columns [c0, c0 + nc) of W
            const int v1 = nres > 0 ? I.colvtx[r0 + nres - 1] + 1 : 0;
            for (int v = nres > 0 ? I.colvtx[r0] : 0; v < v1; ++v) {
                const int c0 = I.xcol[v] - r0, nc = I.xcol[v + 1] - I.xcol[v];
                const double* h = I.Hd + I.hdoff[v];   // lower triangle read
                int nz = 0;
                for (int t = tid; t < nc * nc; t += NT) nz |= (t % nc >= t / nc && h[t] != 0.0);
                if (!__syncthreads_or(nz)) continue;
                for (int t = tid; t < nc * nc; t += NT) {
                    const int i = t % nc, j = t / nc;
                    if (i <= j) W[(c0 + i) + (int64_t)(c0 + j) * ld] = h[j + i * nc];
                }
                for (int j = 0; j < nc; ++j) {
                    __syncthreads();
                    double* Wjj = W + (c0 + j) + (int64_t)(c0 + j) * ld;
                    const double dd = *Wjj;
                    if (!(dd > 0.0)) return -1;
                    const double u = sqrt(dd), ru = 1.0 / u;
                    __syncthreads();
                    int nzr = 0;
                    for (int k = j + 1 + tid; k < nc; k += NT) {
                        const double x = Wjj[(int64_t)(k - j) * ld] * ru;
                        Wjj[(int64_t)(k - j) * ld] = x;
                        nzr |= x != 0.0;
                    }
                    if (tid == 0) *Wjj = u;
                    if (!__syncthreads_or(nzr)) continue;   // an empty row updates nothing (a diagonal block)
                    const int mt = nc - j - 1;
                    for (int t = tid; t < mt * mt; t += NT) {
                        const int i = j + 1 + t % mt, k = j + 1 + t / mt;
                        if (i <= k)
                            W[(c0 + i) + (int64_t)(c0 + k) * ld] -= W[(c0 + j) + (int64_t)(c0 + i) * ld] * W[(c0 + j) + (int64_t)(c0 + k) * ld];
                    }
                }
                __syncthreads();
                for (int t = tid; t < nc * nc; t += NT) {
                    const int i = t % nc, j = t / nc;
                    if (i <= j) W[(c0 + i) + (int64_t)(c0 + j) * ld] *= sd;
                }
            }
            // the front's rows of B, then the children's triangles
            for (int t = tid; t < nb; t += NT) {
                const int i = I.sbrow[b0 + t];
                for (int k = I.B.rptr[i]; k < I.B.rptr[i + 1]; ++k) W[(nres + t) + (int64_t)I.sbloc[k] * ld] = I.B.val[k];
            }
            int rc = nres + nb;
            for (int q = I.fchp[f]; q < I.fchp[f + 1]; ++q) {
                const int c = I.fch[q], cres = I.fnres[c], cs = I.fnsep[c], cn = cres + cs;
                const double* Mc = F + I.fptr[c];
                const int* rel = I.frel + I.fsepp[c];
                for (int t = tid; t < cs * cs; t += NT) {
                    const int r = t % cs, j = t / cs;
                    if (r <= j) W[(rc + r) + (int64_t)rel[j] * ld] = Mc[(cres + r) + (int64_t)(cres + j) * front_ld(cn)];
                }
                rc += cs;
            }
            __syncthreads();
            if (rows < nres) return r0 + rows + 1;
            // Householder QR: column j's reflector v = (a − β, w[j+1..]), β = −sign(a)‖w[j..]‖,
            // applied as w_k −= (vᵀw_k) / (β(β − a)) v, a warp per column.  The vertex rows form an
            // upper triangle that no reflector fills (each touches row j and the rows from nres
            // on), so v lives on row j and rows [lo, rows), lo = max(j + 1, nres).
            const int jmax = min(rows, nfr);
            // columns j < nres share the support size cntp; they go in panels of np reflectors when
            // the panel's supports fit in shared memory and a column's in registers
            const int cntp = 1 + rows - nres;
            const int pmax = cntp <= 32 * QR_SEG ? min(QR_PANEL, XSM_CAP / cntp) : 1;
            for (int j0 = 0; j0 < jmax;) {
              const int np = (pmax > 1 && j0 < nres) ? min(pmax, min(nres, jmax) - j0) : 1;
              const bool panel = np > 1;
              const int kend = panel ? j0 + np : nfr;   // a panel's reflectors reach later columns in qr_apply_panel
              for (int j = j0; j < j0 + np; ++j) {
                double* wj = W + (int64_t)j * ld;
                const double a = wj[j];
                const int lo = max(j + 1, nres), cnt = 1 + rows - lo;
                double s = 0.0;
                for (int i = lo + tid; i < rows; i += NT) s += wj[i] * wj[i];
                s = block_reduce(s, red, OpSum(), 0.0);
                double beta = a;
                if (s > 0.0) {
                    const double nrm = sqrt(a * a + s);
                    beta = a > 0.0 ? -nrm : nrm;
                    const double cf = 1.0 / (beta * (beta - a));
                    if (tid == 0) wj[j] = a - beta;
                    __syncthreads();
                    // the reflector's support staged in shared memory when it fits, so that only w_k
                    // comes from global memory; the same values in the same order either way
                    double* vs = sh.tile + (panel ? (j - j0) * cnt : 0);
                    const bool vsm = cnt <= XSM_CAP;
                    if (vsm)
                        for (int t = tid; t < cnt; t += NT) vs[t] = wj[t == 0 ? j : lo + t - 1];
                    if (panel && tid == 0) sh.acc[j - j0] = cf;
                    __syncthreads();
                    for (int k = j + 1 + warp; k < kend; k += NW) {
                        double* wk = W + (int64_t)k * ld;
                        double dt = 0.0;
#pragma unroll 4
                        for (int t = lane; t < cnt; t += 32) {
                            const int i = t == 0 ? j : lo + t - 1;
                            dt += (vsm ? vs[t] : wj[i]) * wk[i];
                        }
                        dt = warp_sum(dt) * cf;
#pragma unroll 4
                        for (int t = lane; t < cnt; t += 32) {
                            const int i = t == 0 ? j : lo + t - 1;
                            wk[i] -= dt * (vsm ? vs[t] : wj[i]);
                        }
                    }
                    __syncthreads();
                    if (tid == 0) wj[j] = beta;
                } else if (panel && tid == 0) {
                    sh.acc[j - j0] = 0.0;
                }
                if (j < nres && !(fabs(beta) > 0.0)) return r0 + j + 1;
              }
              if (panel) {
                  __syncthreads();
                  qr_apply_panel(W, ld, nfr, j0, np, nres, cntp, sh.tile, sh.acc);
              }
              j0 += np;
            }
            __syncthreads();
            double* M = F + I.fptr[f];
            const int64_t ldm = front_ld(nfr);
            for (int64_t t = tid; t < (int64_t)nfr * nres; t += NT) {
                const int i = (int)(t % nfr), j = (int)(t / nfr);
                if (i >= j) M[i + (int64_t)j * ldm] = (W[j + (int64_t)j * ld] < 0.0 ? -1.0 : 1.0) * W[j + (int64_t)i * ld];
            }
            for (int t = tid; t < nsep * nsep; t += NT) {
                const int r = t % nsep, c = t / nsep;
                if (r <= c) M[(nres + r) + (int64_t)(nres + c) * ldm] = nres + r < jmax ? W[(nres + r) + (int64_t)(nres + c) * ld] : 0.0;
            }
            __syncthreads();
            front_block_inverses(M, nfr, nres);
        }
        return 0;
    }

    __device__ bool initkkt(double dl, double& rho) {
        delta = dl;
        if (set.stable) {   // StableUzawaSolver: no ρ retry (uzawa.jl:162 returns zero(T))
            long long ta = tic();
            const int info = stable_factor(dl);
            toc(SEC_FUPD, ta);
            nfact++;
            rho = 0;
            return info == 0;
        }
        long long ta = tic();
        assemble(dl, 0.0);
        toc(SEC_ASSEMBLE, ta);
        int info = numeric_factor();
        nfact++;
        rho = 0;
        if (info != 0) {
            assemble(dl, 0.0);
            rho = 2.220446049250313e-16 * factor_lower_norm();
            assemble(dl, rho);
            info = numeric_factor();
            nfact++;
            nretry++;
        }
        return info == 0;
    }

    __device__ void Lsolve(double* x) {
        long long t0 = tic(); ntrsv++;
        Lsolve_(x);
        toc(SEC_TRSV, t0);
    }
    __device__ void Usolve(double* x) {
        long long t0 = tic(); ntrsv++;
        Usolve_(x);
        toc(SEC_TRSV, t0);
    }
    __device__ void Lsolve_(double* x) { if (use32) Lsolve_t<float>(F32, x); else Lsolve_t<double>(F64, x); }
    __device__ void Usolve_(double* x) { if (use32) Usolve_t<float>(F32, x); else Usolve_t<double>(F64, x); }
    template <class FT>
    __device__ void Lsolve_t(const FT* F, double* x) {
        for (int f = 0; f < I.nfront; ++f) {
            int nres = I.fnres[f], nfr = nres + I.fnsep[f];
            if (nfr >= XSM_MIN && nfr < COOP_MIN_SOLVE) front_lsolve_sm<FT>(F + I.fptr[f], nfr, nres, I.fres0[f], I.fsep + I.fsepp[f], x, sh);
            else front_lsolve<FT, COOP>(F + I.fptr[f], nfr, nres, I.fres0[f], I.fsep + I.fsepp[f], x, sh,
                             nfr >= COOP_MIN_SOLVE ? coop : nullptr);
        }
    }
    template <class FT>
    __device__ void Usolve_t(const FT* F, double* x) {
        for (int f = I.nfront - 1; f >= 0; --f) {
            int nres = I.fnres[f], nfr = nres + I.fnsep[f];
            if (nfr >= XSM_MIN && nfr < COOP_MIN_SOLVE) front_usolve_sm<FT>(F + I.fptr[f], nfr, nres, I.fres0[f], I.fsep + I.fsepp[f], x, sh);
            else front_usolve<FT, COOP>(F + I.fptr[f], nfr, nres, I.fres0[f], I.fsep + I.fsepp[f], x, sh,
                             nfr >= COOP_MIN_SOLVE ? coop : nullptr);
        }
    }

    // ---- KKT solve  (kkt/kkt.jl:9-21; kkt/cg.jl:69-167; kkt/uzawa.jl:199-227, 319-507) -------
    __device__ void mulkkt(double* u, double* v, const double* Ablk, const double* x, const double* yv) {
        long long t0 = tic(); ngemv += 3;
        amul(Ablk, x, u, 1, 0);
        spmvT(I.B, yv, u, -1, 1);
        spmv(I.B, x, v, 1, 0);
        toc(SEC_GEMV, t0);
    }

    __device__ int cg(int stopmode, double* x, double* yv, double* u, double atol, int itmax, int& niter) {
        const double eps = 2.220446049250313e-16;
        niter = 0;
        double nu2 = bdot(u, u, m, red), nu = sqrt(nu2);
        if (threadIdx.x == 0) I.cghist[0] = nu;
        double np2 = nu2;
        bfill(yv, 0.0, m);
        int status = CG_SOLVED;
        bool stop0 = false;
        if (stopmode) stop0 = bscalenorm(u, I.yscl, m, red) / (1 + sg) <= set.feas_tol;
        if (nu > atol && !stop0) {
            status = CG_ITMAX;
            if (itmax > 0) {
                bcopy(cgp, u, m);
                status = CG_CONTINUE;
                while (status == CG_CONTINUE) {
                    niter += 1;
                    spmvT(I.B, cgp, cgw, 1, 0);
                    Lsolve(cgw);
                    double ep2 = bdot(cgw, cgw, n, red);
                    if (ep2 <= eps * np2) status = CG_NUMERICAL_FAILURE;
                    else {
                        Usolve(cgw);
                        double a = nu2 / ep2;
                        for (int i = threadIdx.x; i < m; i += NT) yv[i] = fma(a, cgp[i], yv[i]);
                        for (int i = threadIdx.x; i < n; i += NT) x[i] = fma(a, cgw[i], x[i]);
                        __syncthreads();
                        spmv(I.B, cgw, u, -a, 1);
                        double pnu2 = nu2;
                        nu2 = bdot(u, u, m, red); nu = sqrt(nu2);
                        if (threadIdx.x == 0 && niter <= set.newton_max_iter) I.cghist[niter] = nu;
                        bool st = false;
                        if (stopmode) st = bscalenorm(u, I.yscl, m, red) / (1 + sg) <= set.feas_tol;
                        if (nu <= atol || 1.0 + nu <= 1.0 || st) status = CG_SOLVED;
                        else if (niter >= itmax) status = CG_ITMAX;
                        else {
                            double b = nu2 / pnu2;
                            for (int i = threadIdx.x; i < m; i += NT) cgp[i] = fma(b, cgp[i], u[i]);
                            __syncthreads();
                            np2 = nu2 + b * b * np2;
                        }
                    }
                }
            }
        }
        return status;
    }

    struct KKTOut { int ncg, nir, status; double dmin, dmax; };

    __device__ void kktwindow(int nir, int ncg, double ftol, double gtol, double& dmin, double& dmax) {
        const double NaN = __longlong_as_double(0x7ff8000000000000LL);
        dmin = dmax = NaN;
        if (nir >= 1) {
            double logd = log(delta), logfres = log(I.uhist[1]);
            double loggtol = log(gtol), logftol = log(ftol);
            int i = 0;
            double logdmax = -__longlong_as_double(0x7ff0000000000000LL);
            double logdmin = logd + logfres - logftol;
            while (logdmin > logdmax && i < ncg + 1) {
                i += 1;
                double loggres = log(I.cghist[i - 1]);
                logdmax = logd + (loggtol - loggres) / (double)i;
            }
            dmin = exp(logdmin);
            dmax = exp(logdmax);
        }
    }

    // stopmode 1 = solveexact!'s fstop/gstop on the scaled residual norms (solver/ipm.jl:278-315)
    __device__ KKTOut solvekkt(int stopmode, double* x, double* yv, const double* A, const double* fv,
                               const double* gv, bool warm, double ftol, double gtol, int irmin) {
        const double stall = set.refine_stall_tol;
        const int irmax = set.refine_max_iter, cgmax = set.newton_max_iter;
        const double dl = delta, alpha = 1.0 / dl;
        int nir = 0, ncg = 0;
        if (warm) {
            mulkkt(df, dg, A, x, yv);
            for (int i = threadIdx.x; i < n; i += NT) df[i] = fv[i] - df[i];
            for (int i = threadIdx.x; i < m; i += NT) dg[i] = gv[i] - dg[i];
            __syncthreads();
        } else {
            for (int i = threadIdx.x; i < n; i += NT) { df[i] = fv[i]; x[i] = 0; }
            for (int i = threadIdx.x; i < m; i += NT) { dg[i] = gv[i]; yv[i] = 0; }
            __syncthreads();
        }
        double fres = bnorm(df, n, red), fprv = fres;
        if (threadIdx.x == 0) I.uhist[0] = fres;
        auto fstop = [&]() { return stopmode ? bscalenorm(df, I.pscl, n, red) / (1 + sf) <= set.feas_tol : false; };
        int irstat;
        if (nir >= irmin && (fres <= ftol || fstop())) irstat = KKT_SOLVED;
        else if (nir >= irmax) irstat = KKT_IRMAX;
        else irstat = KKT_CONTINUE;
        while (irstat == KKT_CONTINUE) {
            nir += 1;
            for (int i = threadIdx.x; i < n; i += NT) dx[i] = df[i] * dl;
            __syncthreads();
            spmvT(I.B, dg, dx, 1, 1);
            Lsolve(dx);
            Usolve(dx);
            spmv(I.B, dx, dg, -1, 1);
            for (int i = threadIdx.x; i < n; i += NT) x[i] += dx[i];
            for (int i = threadIdx.x; i < m; i += NT) yv[i] = fma(alpha, dg[i], yv[i]);
            __syncthreads();
            mulkkt(df, dg, A, x, yv);
            for (int i = threadIdx.x; i < n; i += NT) df[i] = fv[i] - df[i];
            for (int i = threadIdx.x; i < m; i += NT) dg[i] = gv[i] - dg[i];
            __syncthreads();
            fres = bnorm(df, n, red);
            if (threadIdx.x == 0) I.uhist[nir] = fres;
            if (nir >= irmin && (fres <= ftol || fstop())) irstat = KKT_SOLVED;
            else if (nir > 1 && fres > (1 - stall) * fprv) irstat = KKT_STAGNATED;
            else if (nir >= irmax) irstat = KKT_IRMAX;
            else irstat = KKT_CONTINUE;
            fprv = fres;
        }
        for (int i = threadIdx.x; i < m; i += NT) yv[i] = fma(-alpha, dg[i], yv[i]);
        __syncthreads();
        int cgstat = cg(stopmode, x, dyv, dg, gtol, cgmax, ncg);
        for (int i = threadIdx.x; i < m; i += NT) { yv[i] = fma(alpha, dyv[i], yv[i]); yv[i] = fma(alpha, dg[i], yv[i]); }
        __syncthreads();
        int status;
        if (cgstat == CG_NUMERICAL_FAILURE) status = KKT_NUMERICAL_FAILURE;
        else if (irstat == KKT_STAGNATED) status = KKT_STAGNATED;
        else if (irstat == KKT_IRMAX || cgstat == CG_ITMAX) status = KKT_ITMAX;
        else status = KKT_SOLVED;
        KKTOut o{ncg, nir, status, 0, 0};
        kktwindow(nir, ncg, ftol, gtol, o.dmin, o.dmax);
        return o;
    }

    // ---- the iteration  (solver/ipm.jl:86-99, 502-571, 577-774; solver/solver.jl:20-52) ------
    __device__ void residuals() {
        mulkkt(Df, Dg, I.Qd, I.p, I.y);
        for (int i = threadIdx.x; i < n; i += NT) Df[i] = I.d[i] + I.f[i] - Df[i];
        for (int i = threadIdx.x; i < m; i += NT) Dg[i] = I.g[i] - Dg[i];
        __syncthreads();
    }

    __device__ static bool isopt(double mu, double mus, double mut, double pobj, double dobj, double pres, double dres,
                                 int nu, double gap_tol, double feas_tol) {
        if (!(pres < feas_tol && dres < feas_tol)) return false;
        double tol = gap_tol * fmax(1.0, fmin(fabs(pobj), fabs(dobj)));
        if (mut > 0 && nu > 0) return (double)nu * (mu - mut + mut * log1p(mus * mut - 1.0)) <= tol;
        return pobj - dobj < tol;
    }

    __device__ bool isprimalinfeasible(double rtol, double atol) {
        double gy = bdot(I.g, I.y, m, red), ny = bnorm(I.y, m, red);
        bool fl = gy > atol * ny * (1 + ng);
        if (fl) {
            double nQp = bnorm(Qp, n, red);
            for (int i = threadIdx.x; i < n; i += NT) wf[i] = Qp[i] - I.d[i];
            __syncthreads();
            spmvT(I.B, I.y, wf, -1, 1);
            double nwf = bnorm(wf, n, red), nd = bnorm(I.d, n, red);
            fl = fmax(nQp, nwf) < rtol * gy * (1 + nd / ny);
        }
        return fl;
    }
    __device__ bool isdualinfeasible(double rtol, double atol) {
        double fp = bdot(I.f, I.p, n, red), np = bnorm(I.p, n, red);
        bool fl = fp > atol * np * (1 + nf);
        if (fl) {
            spmv(I.B, I.p, Dya, 1, 0);
            double a = bnorm(Dya, m, red), b = bnorm(Qp, n, red);
            fl = fmax(a, b) < rtol * fabs(fp);
        }
        return fl;
    }
    __device__ int nearstatus(int status, double mu, double mus, double pobj, double dobj, double pres, double dres) {
        double fct = set.near_factor;
        if (isopt(mu, mus, I.mut, pobj, dobj, pres, dres, I.nu, fct * set.gap_tol, fct * set.feas_tol)) status = NEAR_OPTIMAL;
        else if (isprimalinfeasible(fct * set.infeas_rel, set.infeas_abs)) status = NEAR_PRIMAL_INFEASIBLE;
        else if (isdualinfeasible(fct * set.infeas_rel, set.infeas_abs)) status = NEAR_DUAL_INFEASIBLE;
        return status;
    }
    __device__ const Row& hrow(int i) const { return *reinterpret_cast<const Row*>(I.hist + (int64_t)i * ROW_DOUBLES); }
    __device__ bool isstalled() const {
        const int window = 5;
        int nh = nrow_hist;
        double tol = set.stall_tol;
        if (nh - stall0 > window) {
            for (int i = nh - window; i < nh; ++i) {
                bool muok = hrow(i).mu < (1 - tol) * hrow(i - 1).mu;
                bool pok = hrow(i).pres < (1 - tol) * hrow(i - 1).pres;
                bool dok = hrow(i).dres < (1 - tol) * hrow(i - 1).dres;
                if (muok || pok || dok) return false;
            }
            return true;
        }
        return false;
    }
    __device__ double getaug() {
        double s = 0;
        for (int64_t i = threadIdx.x; i < I.hdoff[nv]; i += NT) s += I.Hd[i] * I.Hd[i];
        for (int k = threadIdx.x; k < I.Q.nnz; k += NT) s += I.Q.val[k] * I.Q.val[k];
        double nH = sqrt(block_reduce(s, red, OpSum(), 0.0));
        if (nB == 0 || nH == 0) return 1.0;
        if (nrow_hist == 0) return set.aug_tol * nB * nB / nH;
        const Row& r = hrow(nrow_hist - 1);
        double dl = r.delta, dmin = r.dmin, dmax = r.dmax;
        if (r.ppass > 1) {
            if (isfinite(dmin)) dl = fmax(dl, dmin);
            dl *= 10;
        } else if (isfinite(dmin) && isfinite(dmax) && dmin > 0 && dmax > 0) {
            dl = sqrt(dmin) * sqrt(dmax);
        }
        return dl;
    }

    // One iteration.  Mixed precision (settings.precision == 2): the iteration runs with the FP32
    // factor; if a KKT solve misses its tolerance it is redone from the saved iterate with the FP64
    // factor, which stays in use for the rest of the solve.
    __device__ int step() {
        if (set.precision != 2 || fellback) { use32 = set.precision == 1; return step_(); }
        double* sp = I.vn + (int64_t)NVEC_N * n; double* sd = sp + n; double* sy = I.vm + (int64_t)NVEC_M * m;
        for (int i = threadIdx.x; i < n; i += NT) { sp[i] = I.p[i]; sd[i] = I.d[i]; }
        for (int i = threadIdx.x; i < m; i += NT) sy[i] = I.y[i];
        for (int64_t i = threadIdx.x; i < I.cxblk[nv]; i += NT) I.cache2[i] = I.cache[i];
        __syncthreads();
        use32 = true;
        stallhit = false;
        int st = step_();
        if (!kktfail && !stallhit) {
            nfp32++;
            // an FP32 factor that needed more KKT solves than MIXED_MAX_SOLVES costs more in solves
            // than it saved in the factorization: keep this iteration and factor in FP64 from now on
            const Row& r = hrow(nrow_hist - 1);
            if (r.piter + r.ppass + r.citer + r.cpass > MIXED_MAX_SOLVES) { fellback = true; switched = 1; }
            return st;
        }
        // a KKT solve missed its tolerance, or the FP32 iterates stalled: redo this iteration from the
        // saved iterate with the FP64 factor, kept from now on (after a stall the stall window restarts)
        for (int i = threadIdx.x; i < n; i += NT) { I.p[i] = sp[i]; I.d[i] = sd[i]; }
        for (int i = threadIdx.x; i < m; i += NT) I.y[i] = sy[i];
        for (int64_t i = threadIdx.x; i < I.cxblk[nv]; i += NT) I.cache[i] = I.cache2[i];
        __syncthreads();
        nrow_hist--;
        if (stallhit) { switched = 1; stall0 = nrow_hist; }
        fellback = true; use32 = false; nfallback++;
        return step_();
    }

    __device__ int step_() {
        const double NaN = __longlong_as_double(0x7ff8000000000000LL);
        kktfail = false;
        int status = CONTINUE;
        Row row{NaN, NaN, NaN, NaN, 0.0, 0, 0, (double)KKT_SOLVED, 0, 0, (double)KKT_SOLVED, NaN, NaN, NaN, 0.0, NaN, NaN};
        long long tg = tic();
        double dl = getaug();
        toc(SEC_AUG, tg);
        double pd = bdot(I.p, I.d, n, red);
        double spsd = 0;
        long long t0 = tic();
        bool ok = scale_all(spsd);
        toc(SEC_SCALE, t0);
        if (!ok) {
            status = NUMERICAL_FAILURE;
        } else {
            long long tr = tic();
            residuals();
            double nuf = (double)max(I.nu, 1);
            double mu = pd / nuf, mus = spsd / nuf, chi = mu * mus - 1;
            double pres = bscalenorm(Dg, I.yscl, m, red) / (1 + sg);
            double dres = bscalenorm(Df, I.pscl, n, red) / (1 + sf);
            amul(I.Qd, I.p, Qp, 1, 0);
            double pQp = bdot(I.p, Qp, n, red);
            double pobj = pQp / 2 - bdot(I.f, I.p, n, red);
            double dobj = bdot(I.g, I.y, m, red) - pQp / 2;
            row.mu = mu; row.chi = chi; row.pres = pres; row.dres = dres; row.pobj = pobj; row.dobj = dobj;
            toc(SEC_RESID, tr);
            if (isopt(mu, mus, I.mut, pobj, dobj, pres, dres, I.nu, set.gap_tol, set.feas_tol)) status = OPTIMAL;
            else if (isprimalinfeasible(set.infeas_rel, set.infeas_abs)) status = PRIMAL_INFEASIBLE;
            else if (isdualinfeasible(set.infeas_rel, set.infeas_abs)) status = DUAL_INFEASIBLE;
            else if (nrow_hist >= set.max_iter) status = nearstatus(ITERATION_LIMIT, mu, mus, pobj, dobj, pres, dres);
            else if (isstalled()) { stallhit = true; status = nearstatus(STALLED, mu, mus, pobj, dobj, pres, dres); }
            else if (I.nu == 0) {
                double rho;
                bool iok = initkkt(dl, rho);
                row.rho = rho;
                if (!iok) status = nearstatus(NUMERICAL_FAILURE, mu, mus, pobj, dobj, pres, dres);
                else {
                    const double eps = 2.220446049250313e-16;
                    KKTOut o = solvekkt(1, Dpa, Dya, I.Hd, Df, Dg, false, eps, eps, 0);
                    row.piter = o.ncg; row.ppass = o.nir; row.pstat = o.status; row.dmin = o.dmin; row.dmax = o.dmax;
                    for (int i = threadIdx.x; i < n; i += NT) I.p[i] += Dpa[i];
                    for (int i = threadIdx.x; i < m; i += NT) I.y[i] += Dya[i];
                    __syncthreads();
                }
            } else if (!(mu > 0)) {
                status = nearstatus(NUMERICAL_FAILURE, mu, mus, pobj, dobj, pres, dres);
            } else {
                double rho;
                long long t1 = tic();
                bool iok = initkkt(dl, rho);
                toc(SEC_INITKKT, t1);
                row.rho = rho;
                if (!iok) { kktfail = true; status = nearstatus(NUMERICAL_FAILURE, mu, mus, pobj, dobj, pres, dres); }
                else {
                    double mu1 = nrow_hist == 0 ? mu : hrow(0).mu;
                    double tol;
                    if (I.mut > 0) tol = 0.1 * fmin(fabs(mu - I.mut) / fabs(mu1 - I.mut), 1.0);
                    else tol = 0.1 * mu / mu1;
                    double ftol = tol * (1 + nf), gtol = tol * (1 + ng);
                    // predictor  (solver/ipm.jl:119-163)
                    long long t2 = tic();
                    if (I.mut > 0) initpredictor(wf, I.mut);
                    else { for (int i = threadIdx.x; i < n; i += NT) wf[i] = -I.d[i]; __syncthreads(); }
                    baxpy(1.0, Df, wf, n);
                    KKTOut po = solvekkt(0, Dpa, Dya, I.Hd, wf, Dg, false, ftol, gtol, 1);
                    bcopy(Dda, Df, n);
                    spmvT(I.B, Dya, Dda, -1, -1);
                    amul(I.Qd, Dpa, Dda, 1, 1);
                    row.piter = po.ncg; row.ppass = po.nir; row.pstat = po.status; row.dmin = po.dmin; row.dmax = po.dmax;
                    zerofree(Dda);
                    toc(SEC_PRED, t2);
                    // corrector  (solver/ipm.jl:181-272)
                    long long t3 = tic();
                    double taua = maxsteps(Dpa, Dda, 1.0);
                    toc(SEC_MAXSTEPS, t3);
                    t3 = tic();
                    double sm = 0;
                    for (int j = threadIdx.x; j < n; j += NT) sm += (I.p[j] + taua * Dpa[j]) * (I.d[j] + taua * Dda[j]);
                    sm = block_reduce(sm, red, OpSum(), 0.0);
                    double mua = sm / (double)I.nu;
                    if (I.mut > 0) {
                        double dmu = mu - I.mut;
                        if (dmu > 0) {
                            double dmua = fmin(fmax(mua - I.mut, 0.0), dmu);
                            sm = I.mut + fmin(fmax(dmua * (dmua / dmu) * (dmua / dmu), 0.0), dmu);
                        } else sm = I.mut;
                    } else {
                        double t = mua * (mua / mu) * (mua / mu);
                        sm = t > mu ? mu : (t < 0 ? 0.0 : t);
                    }
                    initcorrector(wf, Dpa, Dda, sm);
                    baxpy(1.0, Df, wf, n);
                    bcopy(Dp, Dpa, n);
                    bcopy(Dy, Dya, m);
                    KKTOut co = solvekkt(0, Dp, Dy, I.Hd, wf, Dg, true, ftol, gtol, 1);
                    bcopy(Dd, Df, n);
                    spmvT(I.B, Dy, Dd, -1, -1);
                    amul(I.Qd, Dp, Dd, 1, 1);
                    row.citer = co.ncg; row.cpass = co.nir; row.cstat = co.status;
                    zerofree(Dd);
                    toc(SEC_CORR, t3);
                    if (po.status != KKT_SOLVED || co.status != KKT_SOLVED) {
                        kktfail = true;
                        status = nearstatus(NUMERICAL_FAILURE, mu, mus, pobj, dobj, pres, dres);
                    } else {
                        long long t4 = tic();
                        double st = maxsteps(Dp, Dd, set.step_frac);
                        toc(SEC_MAXSTEPS, t4);
                        row.step = st;
                        for (int i = threadIdx.x; i < n; i += NT) { I.p[i] = fma(st, Dp[i], I.p[i]); I.d[i] = fma(st, Dd[i], I.d[i]); }
                        for (int i = threadIdx.x; i < m; i += NT) I.y[i] = fma(st, Dy[i], I.y[i]);
                        __syncthreads();
                    }
                }
            }
        }
        row.delta = dl;
        if (threadIdx.x == 0 && nrow_hist <= set.max_iter)
            *reinterpret_cast<Row*>(I.hist + (int64_t)nrow_hist * ROW_DOUBLES) = row;
        nrow_hist++;
        __syncthreads();
        return status;
    }

    // result(s, status)  (solver/ipm.jl:30-74): scalars + unscaled iterates in solver order
    __device__ void result(int status) {
        const double NaN = __longlong_as_double(0x7ff8000000000000LL);
        double mu = NaN, pres = NaN, dres = NaN, pobj = NaN, dobj = NaN;
        bool infeas = status == PRIMAL_INFEASIBLE || status == NEAR_PRIMAL_INFEASIBLE ||
                      status == DUAL_INFEASIBLE || status == NEAR_DUAL_INFEASIBLE;
        if (!(infeas || nrow_hist == 0)) {
            residuals();
            amul(I.Qd, I.p, Qp, 1, 0);
            double pQp = bdot(I.p, Qp, n, red);
            pobj = pQp / 2 - bdot(I.f, I.p, n, red);
            dobj = bdot(I.g, I.y, m, red) - pQp / 2;
            mu = I.nu == 0 ? NaN : bdot(I.p, I.d, n, red) / (double)I.nu;
            pres = bscalenorm(Dg, I.yscl, m, red) / (1 + sg);
            dres = bscalenorm(Df, I.pscl, n, red) / (1 + sf);
        }
        save();
        if (threadIdx.x == 0) {
            I.scal[0] = mu; I.scal[1] = pres; I.scal[2] = dres; I.scal[3] = pobj; I.scal[4] = dobj;
            I.status[0] = status;
        }
        for (int i = threadIdx.x; i < n; i += NT) { I.po[i] = I.p[i] * I.pscl[i]; I.dout[i] = I.d[i] / I.pscl[i]; }
        for (int i = threadIdx.x; i < m; i += NT) I.yo[i] = I.y[i] * I.yscl[i];
        __syncthreads();
    }
};

// init (solver/ipm.jl:431-478 and reinit! :375-429), then the solve_impl! loop
// (solver/solver.jl:119-145) and result, or one of those pieces (mode)
template <bool COOP>
__device__ void solve_instance(const DevInst& I, const Settings& set, Shared& sh, int mode, CoopCtl* coop) {
    const int n = I.n, m = I.m;
    if (mode == MODE_SOLVE || mode == MODE_INIT || mode == MODE_REINIT) {
        if (threadIdx.x == 0) { for (int k = 0; k < NSTAT; ++k) I.status[k] = 0; }
        __syncthreads();
    }
    Ctx<COOP> c(I, set, sh, coop);
    if (mode == MODE_SOLVE || mode == MODE_INIT) {
        // working copies of the inputs: a solve never modifies the uploaded problem
        for (int i = threadIdx.x; i < I.B.nnz; i += NT) I.B.val[i] = I.B.val0[i];
        for (int i = threadIdx.x; i < I.Q.nnz; i += NT) I.Q.val[i] = I.Q.val0[i];
        for (int v = threadIdx.x >> 5; v < I.nvtx; v += NW) {   // Qd ← the stored blocks, zero for the others
            const int64_t o = I.qd0off[v], h0 = I.hdoff[v], nb = I.hdoff[v + 1] - h0;
            for (int64_t t = threadIdx.x & 31; t < nb; t += 32) I.Qd[h0 + t] = o < 0 ? 0.0 : I.Qd0[o + t];
        }
        for (int i = threadIdx.x; i < n; i += NT) { I.f[i] = I.f0[i]; I.p[i] = I.p0[i]; I.d[i] = I.d0[i]; }
        for (int i = threadIdx.x; i < m; i += NT) { I.g[i] = I.g0[i]; I.y[i] = I.y0[i]; }
        __syncthreads();
        // H = copy(Q) happens after equilibration (IPMSolver constructor order)
        for (int k = threadIdx.x; k < NSCAL; k += NT) I.scal[k] = 0;
        for (int k = 0; k < NSEC; ++k) c.tsec[k] = 0;
        c.stall0 = 0;
        c.ntrsv = 0; c.ngemv = 0;
        long long t0 = c.tic();
        if (set.scale_max_iter > 0) c.equilibrate(set.scale_max_iter, 1e-3);
        else {
            for (int j = threadIdx.x; j < n; j += NT) I.pscl[j] = 1;
            for (int i = threadIdx.x; i < m; i += NT) I.yscl[i] = 1;
            __syncthreads();
        }
        c.toc(SEC_EQUIL, t0);
        t0 = c.tic();
        c.build_finit();
        c.toc(SEC_FINIT, t0);
        for (int64_t i = threadIdx.x; i < I.hdoff[I.nvtx]; i += NT) I.Hd[i] = I.Qd[i];   // H = copy(Q)
        c.mark_socz();
        double s = 0;
        for (int i = threadIdx.x; i < I.B.nnz; i += NT) s += I.B.val[i] * I.B.val[i];
        c.nB = sqrt(block_reduce(s, c.red, OpSum(), 0.0));
        c.nf = bnorm(I.f, n, c.red);
        c.ng = bnorm(I.g, m, c.red);
        c.sg = bscalenorm(I.g, I.yscl, m, c.red);
        c.sf = bscalenorm(I.f, I.pscl, n, c.red);
    } else if (mode == MODE_REINIT) {
        // reinit! (solver/ipm.jl:375-429): new f or g in the solver's scaling, a fresh start, an empty
        // history; the equilibration, Q, B and BᵀB of the first init stay
        if (I.reinit_fg & 1) {
            for (int i = threadIdx.x; i < n; i += NT) I.f[i] = I.f0[i] * I.pscl[i];
            __syncthreads();
            c.nf = bnorm(I.f, n, c.red);
            c.sf = bscalenorm(I.f, I.pscl, n, c.red);
        }
        if (I.reinit_fg & 2) {
            for (int i = threadIdx.x; i < m; i += NT) I.g[i] = I.g0[i] * I.yscl[i];
            __syncthreads();
            c.ng = bnorm(I.g, m, c.red);
            c.sg = bscalenorm(I.g, I.yscl, m, c.red);
        }
        for (int i = threadIdx.x; i < n; i += NT) { I.p[i] = I.p0[i]; I.d[i] = I.d0[i]; }
        for (int i = threadIdx.x; i < m; i += NT) I.y[i] = I.y0[i];
        c.stall0 = 0;
        __syncthreads();
    }
    if (mode == MODE_SOLVE || mode == MODE_INIT || mode == MODE_REINIT) {
        if (!I.has_p0 && !I.has_d0) {
            c.startingpoint();
            if (I.has_y0) { for (int i = threadIdx.x; i < m; i += NT) I.y[i] /= I.yscl[i]; }
            else { for (int i = threadIdx.x; i < m; i += NT) I.y[i] = 0; }
            __syncthreads();
        } else {
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            if (!(I.has_p0 && I.has_d0)) {
                for (int v = warp; v < I.nvtx; v += NW) {   // dualshadow! / primalshadow!
                    int k = I.kind[v], c0 = I.xcol[v], nc = I.xcol[v + 1] - c0;
                    double* dst = !I.has_d0 ? I.d + c0 : I.p + c0;
                    const double* src = !I.has_d0 ? I.p + c0 : I.d + c0;
                    if (k == CONE_POS) { for (int i = lane; i < nc; i += 32) dst[i] = 1.0 / src[i]; }
                    else if (k == CONE_SOC) w_socshadow(dst, src, nc);
                    else if (k == CONE_EXP || k == CONE_POW) {
                        if (lane == 0) {
                            double* C = I.cache + I.cxblk[v];
                            if (!I.has_d0) tddualshadow(TD{k, I.kpar[v]}, dst, src, C);
                            else tdprimalshadow(TD{k, I.kpar[v]}, dst, src, C);
                        }
                        __syncwarp();
                    }
                    else if (k == CONE_SDP) {}
                    else { for (int i = lane; i < nc; i += 32) dst[i] = 0; }
                }
                __syncthreads();
                for (int v = 0; v < I.nvtx; ++v) {   // sdpshadow! for either side (sdp.jl:640-705)
                    if (I.kind[v] != CONE_SDP) continue;
                    int c0 = I.xcol[v], nc = I.xcol[v + 1] - c0;
                    double* dst = !I.has_d0 ? I.d + c0 : I.p + c0;
                    const double* src = !I.has_d0 ? I.p + c0 : I.d + c0;
                    b_sdpshadow(dst, src, nc, I.work, SdpSh{c.red, &sh.flag});
                }
            }
            __syncthreads();
            if (!I.has_y0) for (int i = threadIdx.x; i < m; i += NT) I.y[i] = 0;
            for (int i = threadIdx.x; i < n; i += NT) { I.p[i] /= I.pscl[i]; I.d[i] *= I.pscl[i]; }
            for (int i = threadIdx.x; i < m; i += NT) I.y[i] /= I.yscl[i];
            __syncthreads();
        }
        for (int v = threadIdx.x; v < I.nvtx; v += NT)   // initcache! (exp.jl:22-25, pow.jl:35-38)
            if (I.kind[v] == CONE_EXP || I.kind[v] == CONE_POW) tdinitcache(TD{I.kind[v], I.kpar[v]}, I.cache + I.cxblk[v]);
        __syncthreads();
        c.save();
        if (threadIdx.x == 0) I.status[0] = CONTINUE;
        __syncthreads();
    }
    if (mode == MODE_SOLVE) {
        int status = CONTINUE;
        while (status == CONTINUE) status = c.step();
        c.result(status);
    } else if (mode == MODE_STEP) {
        int status = c.step();
        c.save();
        if (threadIdx.x == 0) I.status[0] = status;
        __syncthreads();
    } else if (mode == MODE_RESULT) {
        c.result(I.status[0]);
    } else if (mode == MODE_FRULE || mode == MODE_RRULE) {
        c.sensitivity(mode == MODE_RRULE);
    } else if (mode == MODE_FRULE2) {
        c.sensitivity2();
    }
}

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

struct BatchArgs {
    const DevInst* inst;
    int ninst;
    int mode;
    Settings set;
    int* counter;     // work queue head
    // optional per-instance completion stamps (serving loop): done[(seq0 + k) % cap] = seq0 + k + 1,
    // written to mapped host memory after a system-scope fence
    unsigned long long* done;
    long long seq0;
    int cap;
};

__global__ void __launch_bounds__(NT, CTA_PER_SM) MB_SFX(ipm_batch_kernel)(BatchArgs a) {
    extern __shared__ __align__(16) unsigned char mb_dsmem[];
    Shared& sh = *reinterpret_cast<Shared*>(mb_dsmem);
    __shared__ int next;
    const bool tc = MB_TC && a.set.precision != 0;   // the tensor-core build, and an FP32 factor may run
    tc_setup(sh, tc);
    for (;;) {
        if (threadIdx.x == 0) next = atomicAdd(a.counter, 1);
        __syncthreads();
        int k = next;
        __syncthreads();
        if (k >= a.ninst) break;
        if (threadIdx.x == 0) sh.tc_err = a.inst[k].status + 7;
        __syncthreads();
        unsigned long long t0 = globaltimer();
        solve_instance<false>(a.inst[k], a.set, sh, a.mode, nullptr);
        if (threadIdx.x == 0) {
            a.inst[k].scal[SCAL_T0] = __longlong_as_double((long long)t0);
            a.inst[k].scal[SCAL_T1] = __longlong_as_double((long long)globaltimer());
            if (a.done) {
                __threadfence_system();
                const long long seq = a.seq0 + k;
                *(volatile unsigned long long*)&a.done[seq % a.cap] = (unsigned long long)seq + 1;
            }
        }
    }
    tc_teardown(sh, tc);
}

// One large instance on the whole GPU (cooperative launch): CTA 0 runs the solve and posts the
// dense work of its large fronts to the other CTAs; COOP_EXIT releases them when it is done.
__global__ void __launch_bounds__(NT, CTA_PER_SM) MB_SFX(ipm_coop_kernel)(BatchArgs a, CoopCtl* c) {
    extern __shared__ __align__(16) unsigned char mb_dsmem[];
    Shared& sh = *reinterpret_cast<Shared*>(mb_dsmem);
    const bool tc = MB_TC && a.set.precision != 0;   // the tensor-core build, and an FP32 factor may run
    tc_setup(sh, tc);
    if (threadIdx.x == 0) {
        sh.wait_ns = a.set.coop_wait > 0 ? (long long)(a.set.coop_wait * 1e9) : COOP_WAIT_NS;
        sh.tc_err = blockIdx.x == 0 ? a.inst[0].status + 7 : &c->abort;
    }
    __syncthreads();
    if (blockIdx.x != 0) {
        coop_helper(c, sh);
        tc_teardown(sh, tc);
        return;
    }
    const DevInst& I = a.inst[0];
    const unsigned long long t0 = globaltimer();
    solve_instance<true>(I, a.set, sh, a.mode, c);
    __syncthreads();
    if (threadIdx.x == 0) {
        I.scal[SCAL_T0] = __longlong_as_double((long long)t0);
        I.scal[SCAL_T1] = __longlong_as_double((long long)globaltimer());
        c->cmd = COOP_EXIT;
    }
    coop_barrier(c, sh);
    if (threadIdx.x == 0 && ld_volatile_i32(&c->abort) != 0) I.status[7] = 1;
    tc_teardown(sh, tc);
}

}  // namespace mb

// grid-cooperative launch of one instance: every CTA of the grid co-resident (grid <= 2 per SM)
extern "C" int MB_SFX(mb_launch_coop)(const mb::DevInst* d_inst, int mode, const mb::Settings* set, mb::CoopCtl* d_ctl,
                              int grid, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(d_ctl, 0, sizeof(mb::CoopCtl), stream);
    if (e != cudaSuccess) return -1;
    e = cudaFuncSetAttribute(mb::MB_SFX(ipm_coop_kernel), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(mb::Shared));
    if (e != cudaSuccess) return -1;
    mb::BatchArgs a;
    a.inst = d_inst; a.ninst = 1; a.mode = mode; a.set = *set; a.counter = nullptr;
    a.done = nullptr; a.seq0 = 0; a.cap = 1;
    void* args[] = {(void*)&a, (void*)&d_ctl};
    e = cudaLaunchCooperativeKernel((const void*)mb::MB_SFX(ipm_coop_kernel), dim3(grid), dim3(mb::NT), args,
                                    sizeof(mb::Shared), stream);
    return e == cudaSuccess ? 0 : -2;
}

// ---------------------------------------------------------------------------------------------
// launch entry used by the host runtime
// ---------------------------------------------------------------------------------------------
extern "C" int MB_SFX(mb_launch_batch)(const mb::DevInst* d_inst, int ninst, int mode, const mb::Settings* set,
                               int* d_counter, int grid, int fp32, cudaStream_t stream) {
    mb::BatchArgs a;
    a.inst = d_inst; a.ninst = ninst; a.mode = mode; a.set = *set; a.counter = d_counter;
    a.done = nullptr; a.seq0 = 0; a.cap = 1;
    cudaError_t e = cudaMemsetAsync(d_counter, 0, sizeof(int), stream);
    if (e != cudaSuccess) return -1;
    (void)fp32;
    e = cudaFuncSetAttribute(mb::MB_SFX(ipm_batch_kernel), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(mb::Shared));
    if (e != cudaSuccess) return -1;
    mb::MB_SFX(ipm_batch_kernel)<<<grid, mb::NT, sizeof(mb::Shared), stream>>>(a);
    e = cudaGetLastError();
    return e == cudaSuccess ? 0 : -2;
}

#if !MB_TC
// ---------------------------------------------------------------------------------------------
// Fixed device scratch for mb_batch_solve_static (no counterpart in the reference).
//
// Some callers may not allocate device memory during service: a process that reserved its HBM
// budget up front (a cudaMalloc could fail, or take it past the budget, mid-service), and a
// process whose other streams run latency-critical work (cudaFree, and cudaMalloc when it has to
// grow the heap, synchronise the whole device).  For them the batched solve can run from this
// file-scope array, which the driver places when it loads this module.  It is one per device and
// per process: calls that overlap in time on one device race on it.
// ---------------------------------------------------------------------------------------------
#include "../../include/mumblebee_gpu.h"

static __device__ __align__(256) unsigned char mb_static_scratch_buf[MB_STATIC_SCRATCH_BYTES];

// Device address and size of the scratch on `device`.  The address is looked up on every call,
// with that device current (cudaGetSymbolAddress, which loads the module on the first call and is
// a table lookup after that), so it stays right if the host application resets the device or
// tears down and recreates its primary context between calls; the previously current device is
// restored.  Returns a cudaError_t value (0 on success).
extern "C" int mb_static_scratch(int device, void** ptr, size_t* bytes) {
    if (!ptr || !bytes || device < 0) return (int)cudaErrorInvalidValue;
    int cur = -1;
    cudaError_t e = cudaGetDevice(&cur);
    if (e != cudaSuccess) return (int)e;
    if (cur != device && (e = cudaSetDevice(device)) != cudaSuccess) return (int)e;
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, mb_static_scratch_buf);
    if (cur != device) {
        cudaError_t r = cudaSetDevice(cur);
        if (e == cudaSuccess) e = r;
    }
    if (e != cudaSuccess) return (int)e;
    *ptr = p;
    *bytes = sizeof(mb_static_scratch_buf);
    return (int)cudaSuccess;
}

#endif  // !MB_TC

// the serving loop's launch: one admission wave of ring slots [seq0, seq0 + ninst), each instance
// stamping done[(seq0 + k) % cap] when it finishes
extern "C" int MB_SFX(mb_launch_wave)(const mb::DevInst* d_inst, int ninst, const mb::Settings* set, int* d_counter, int grid,
                              unsigned long long* done, long long seq0, int cap, cudaStream_t stream) {
    mb::BatchArgs a;
    a.inst = d_inst; a.ninst = ninst; a.mode = mb::MODE_SOLVE; a.set = *set; a.counter = d_counter;
    a.done = done; a.seq0 = seq0; a.cap = cap;
    cudaError_t e = cudaMemsetAsync(d_counter, 0, sizeof(int), stream);
    if (e != cudaSuccess) return -1;
    e = cudaFuncSetAttribute(mb::MB_SFX(ipm_batch_kernel), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(mb::Shared));
    if (e != cudaSuccess) return -1;
    mb::MB_SFX(ipm_batch_kernel)<<<grid, mb::NT, sizeof(mb::Shared), stream>>>(a);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// CTAs of ipm_coop_kernel that can be co-resident (the grid of a cooperative launch)
extern "C" int MB_SFX(mb_coop_grid)(int device, int nsm) {
    (void)device;
    int per_sm = 0;
    if (cudaFuncSetAttribute(mb::MB_SFX(ipm_coop_kernel), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(mb::Shared)) != cudaSuccess)
        return nsm;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mb::MB_SFX(ipm_coop_kernel), mb::NT, sizeof(mb::Shared)) != cudaSuccess || per_sm < 1)
        return nsm;
    return nsm * (per_sm < mb::CTA_PER_SM ? per_sm : mb::CTA_PER_SM);
}
