// Internal layout shared by the host runtime (mb_host.cpp) and the device solver
// (mb_solver.cu).  One `DevInst` describes one problem instance resident in HBM; the batched
// solver kernel assigns one CTA to one instance and runs the whole interior-point solve there.
#pragma once
#include <cstdint>

namespace mb {

// launch shape of the batched solver: CTA_THREADS threads per instance, CTA_PER_SM instances
// resident per SM (the kernel is latency-bound; a second resident instance hides latency)
constexpr int CTA_THREADS = 256;
constexpr int CTA_PER_SM = 2;

// Leading dimension of a front of order nf in the factor storage F: nf rounded up to even.  F and
// every front in it start on a 256-byte boundary, so each FP64 column starts on a 16-byte boundary
// and the FP64 update tiles are staged with 16-byte copies of row pairs.  Row nf of a column of
// odd order is padding that nothing reads.  (Measured on B200: rounding up to a multiple of 4, or
// to 2 mod 4, slows the triangular solves more than it gives.)
#ifdef __CUDACC__
__host__ __device__
#endif
inline int64_t front_ld(int64_t nf) { return nf + (nf & 1); }

enum ConeKind { CONE_FREE = 0, CONE_POS = 1, CONE_SOC = 2, CONE_SDP = 3, CONE_EXP = 4, CONE_POW = 5 };

// IPMStatus (src/IPM/src/ipm/ipm.jl:1), KKTStatus (kkt/kkt.jl:1), CGStatus (kkt/cg.jl:1-6)
enum IPMStatus { CONTINUE = 0, OPTIMAL, NEAR_OPTIMAL, STALLED, NUMERICAL_FAILURE, ITERATION_LIMIT,
                 PRIMAL_INFEASIBLE, DUAL_INFEASIBLE, ILL_POSED, NEAR_PRIMAL_INFEASIBLE,
                 NEAR_DUAL_INFEASIBLE, NEAR_ILL_POSED };
enum KKTStatus { KKT_CONTINUE = 0, KKT_SOLVED, KKT_STAGNATED, KKT_ITMAX, KKT_NUMERICAL_FAILURE, KKT_IRMAX };
enum CGStatus { CG_CONTINUE = 0, CG_SOLVED, CG_NUMERICAL_FAILURE, CG_ITMAX };

// Settings, field order shared with mb_settings in include/mumblebee_gpu.h
struct Settings {
    int32_t verbose, max_iter, scale_max_iter, refine_max_iter, newton_max_iter, stable, precision, large;
    double step_frac, feas_tol, gap_tol, near_factor, stall_tol, refine_stall_tol, aug_tol, infeas_abs, infeas_rel;
    double coop_wait;   // seconds at a grid barrier of the grid-cooperative mode (<= 0: 60)
    int32_t fp32_tiles; // FP32 factor update tiles: 0 runtime's choice, 1 FFMA, 2 tensor cores (tcgen05)
    int32_t reserved;
};

// One history row: the 17 fields of IPMHistoryRow (history/ipm.jl:1-4), stored as doubles.
struct Row {
    double pres, dres, pobj, dobj, step;
    double piter, ppass, pstat, citer, cpass, cstat;
    double dmin, dmax, rho, delta, mu, chi;
};
constexpr int ROW_DOUBLES = 17;

// Scalar sparse matrix on the device: the nonzeros of a BlockSparseMatrix (explicit zeros of its
// dense blocks dropped; they contribute nothing to any sum), CSR order, with a CSC index into the
// same value array so that A x and Aᵀ x are both gathers.
struct DevSp {
    int nrow, ncol, nnz;
    const int* rptr;        // nrow+1
    const int* cidx;        // nnz: column of each CSR entry (ascending within a row)
    double* val;            // nnz, CSR order (mutable: equilibration scales in place)
    const double* val0;     // nnz, pristine copy
    const int* cptr;        // ncol+1
    const int* ridx;        // nnz: row of each CSC entry (ascending within a column)
    const int* cpos;        // nnz: CSR position of each CSC entry
    int nlongr, nlongc;     // rows / columns with more than LONG_ROW entries (a warp each; the rest a thread each)
    const int* longr;       // nlongr rows
    const int* longc;       // nlongc columns
};

constexpr int LONG_ROW = 32;   // sparse products: longer rows or columns go to a warp, shorter ones to a thread

struct DevInst {
    int n, m, nvtx, nfront;
    int nu;                 // cone degree ν
    int has_p0, has_d0, has_y0;
    int reinit_fg;          // MODE_REINIT: bit 0 = f0 holds a new f, bit 1 = g0 holds a new g
    double* sx;             // MODE_FRULE / MODE_RRULE exchange, solver order, unscaled: seeds a (n), b (m),
                            // c (n), then results a (n), b (m), c (n), then [Δμ in, dμ out, ok];
                            // MODE_FRULE2: Δf1, Δg1, Δf2, Δg2, then nine results (Δp, Δy, Δd for
                            // sets 1, 2 and the second order), then [Δμ1, Δμ2, ok]
    double mut;             // barrier target μ′ (0 = exact solve)
    const int* xcol;        // nvtx+1: columns of each vertex
    const int* colvtx;      // n: vertex of each column
    const int* cfront;      // n: front owning each column
    DevSp B, Q;
    // rows of the product (blockdiag(Hd or Qd) + Q off-diagonal blocks) x that have more than LONG_ROW
    // terms (a warp each); hflag[i] bit 0 marks them for the thread-per-row pass to skip, bit 1 marks
    // the rows of a vertex whose diagonal Q block is zero
    int nhlong;
    const int* hlong;
    const int* hflag;
    // dense diagonal blocks (nc x nc per vertex, column-major): Q's (working + pristine) and H's
    const int64_t* hdoff;   // nvtx+1
    double* Qd; const double* Qd0; double* Hd;
    const int64_t* qd0off;  // nvtx: offset of a vertex's pristine block in Qd0, -1 when it is zero (not stored)
    const int64_t* hdpos;   // per vertex: offset in F of its diagonal block's (0,0) entry
    const int* hdld;        // per vertex: leading dimension of its front
    // Q nonzeros outside the diagonal blocks, lower triangle: CSR position and F offset
    int nqoff;
    const int* qoffk; const int64_t* qoffpos;
    const int* kind;        // cone kind per vertex
    const double* kpar;     // cone parameter per vertex
    const int64_t* cxblk;   // cache offsets per vertex (nvtx+1)
    double* cache;
    double* cache2;         // saved cache (mixed-precision redo)
    int wsize;              // per-cone workspace length (max over cones)
    // fronts (multifrontal): front f owns scalar columns [fres0[f], fres0[f]+fnres[f]) and the
    // separator rows fsep[fsepp[f] .. fsepp[f+1]); its column-major storage (order nres+nsep,
    // leading dimension front_ld(nres+nsep)) starts at fptr[f]; frel maps separator rows to
    // positions in the parent's row list.
    const int* fres0; const int* fnres; const int* fnsep; const int* fparent;
    const int64_t* fptr; const int* fsepp; const int* fsep; const int* frel;
    int64_t fsize;
    double* Finit;          // fsize doubles: lower part of BᵀB in front layout, built on the device
    void* F;                // fsize FT (double or float)
    // stable factor (settings.stable): rows of B per front (sbrp[f] .. sbrp[f+1] of sbrow), the front
    // position of each CSR entry of B in its row's front, the children of each front (fchp / fch),
    // and the scratch of one front's stacked QR system
    const int* sbrp; const int* sbrow; const int* sbloc; const int* fchp; const int* fch;
    double* swork;
    // pristine vectors and working copies
    const double* f0; const double* g0; const double* p0; const double* d0; const double* y0;
    double* f; double* g;
    double* pscl; double* yscl;
    double* p; double* d; double* y;
    double* vn;             // NVEC_N n-vectors
    double* vm;             // NVEC_M m-vectors
    double* vv;             // NVEC_V nvtx-vectors
    double* work;           // cone workspace (wsize per warp)
    double* po; double* dout; double* yo;   // result iterates (user scaling, solver order)
    double* hist;           // max_iter+1 rows (ROW_DOUBLES each)
    double* uhist;          // refine_max_iter + 2
    double* cghist;         // newton_max_iter + 1
    int* status;            // [0] IPM status, [1] rows written, [2] factor retries, [3] factorizations,
                            // [4] FP32 iterations, [5] FP64 redos (mixed precision)
    double* scal;           // NSCAL: mu pres dres pobj dobj nf ng sf sg nB, timers, counters
};

constexpr int NVEC_N = 13;  // Df Qp wf Dpa Dda Dp Dd df dx cgw  tmp1 tmp2 (tmp2 also: column maxima)  hx
constexpr int NVEC_M = 8;   // Dg Dya Dy dg dy cgp tmp1 tmp2
// two more n-vectors and one m-vector follow the above (saved p, d, y of a mixed-precision redo)
constexpr int NVEC_V = 8;   // step spsd flag vscl vnrm vswp socz socdot
constexpr int NSCAL = 32;   // mu pres dres pobj dobj | nf ng sf sg nB | section clocks (NSEC) | counters
// section timers (SM clock cycles), the TimerOutputs sections of the reference plus set-up; the
// last four split the numeric factorization (inside initkkt)
enum Section { SEC_EQUIL = 0, SEC_FINIT, SEC_SCALE, SEC_INITKKT, SEC_PRED, SEC_CORR, SEC_MAXSTEPS, SEC_TRSV, SEC_GEMV,
               SEC_ASSEMBLE, SEC_RESID, SEC_AUG, SEC_FUPD, SEC_FDIAG, SEC_FPANEL, SEC_FEXTEND, NSEC };
constexpr int SCAL_SEC = 10;        // scal[10 .. 10+NSEC)
constexpr int SCAL_NTRSV = 26;      // triangular solve sweeps
constexpr int SCAL_NGEMV = 27;      // block-sparse matvecs
constexpr int SCAL_T0 = 28;         // %globaltimer (ns, bit pattern) when a CTA took the instance
constexpr int SCAL_T1 = 29;         // %globaltimer (ns, bit pattern) when its solve finished
constexpr int SCAL_NSOCZ = 30;      // second-order cones whose diagonal block of Q is zero
constexpr int SCAL_STALL0 = 31;     // history rows before the mixed-precision switch after an FP32 stall
static_assert(SCAL_SEC + NSEC <= SCAL_NTRSV, "section clocks overlap the counters");
constexpr int NSTAT = 8;    // status, history rows, factor retries, factorizations, FP32 iterations, FP64 redos,
                            // switched-to-FP64 flag, grid-barrier timeout flag

// kernel modes: a full solve, or the pieces used by the step-wise API
enum Mode { MODE_SOLVE = 0, MODE_INIT = 1, MODE_STEP = 2, MODE_RESULT = 3, MODE_REINIT = 4, MODE_FRULE = 5,
            MODE_RRULE = 6, MODE_FRULE2 = 7 };

// Grid-cooperative mode for one large instance: CTA 0 (the leader) runs the iteration; the other
// CTAs of a cooperative launch help with the dense work of large fronts (assembly copy, factor
// update tiles, panel rows, extend-add).  The leader posts a command here and meets the helpers at
// a grid barrier; every wait is bounded (COOP_WAIT_NS), after which `abort` is set and every role
// returns.  The host zeroes this block before each launch.
struct CoopCtl {
    unsigned int count;     // barrier arrivals
    unsigned int gen;       // barrier generation
    int abort;              // a barrier wait timed out
    int cmd;                // command for the helpers
    int ia[8];
    long long la[4];
    void* pa[4];
    double acc[32];         // backward-solve column dots gathered from the helpers
};
enum CoopCmd { COOP_NONE = 0, COOP_EXIT = 1, COOP_FILL = 2, COOP_COPY = 3, COOP_UPDATE = 4, COOP_PANEL = 5,
               COOP_EXTEND = 6, COOP_LROWS = 7, COOP_UDOTS = 8, COOP_SCHUR = 9 };

// One compensated product c ← α op(A) b + β c (extmul! / twomul!), a thread per output: N walks
// the CSR of A's stored entries, T the CSC with block marks (brk: 1 opens a block of the column,
// 2 opens a 1 x 1 block).  cc == nullptr: folded result (extmul!); else the pair (twomul!).
// s, cs (nullable) receive phase 1's pair.  acls / bcls classify α and β as the reference's
// epilogue branches do (acls 1: α = 1, 2: α = -1, 0 else; bcls 0: β = 0, 1: β = 1, 2: β = -1, 3 else).
struct TwoMv {
    int64_t nout;
    int trans, acls, bcls;
    const int64_t* ptr; const int32_t* idx; const double* val; const unsigned char* brk;
    const double* b;
    double alpha, beta;
    double* c; double* cc; double* s; double* cs;
};


}  // namespace mb
