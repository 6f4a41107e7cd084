/*
 * mumblebee_gpu.h — C ABI of libmbgpu.so, the B200 (sm_100a) interior-point solver that stands in
 * for the hot path of Mumblebee.jl's `IPM` module behind its public solver API.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, returns 0 on success or a
 * negative MB_E* code (never aborts), and copies caller-owned host inputs at create time.  Device
 * state lives behind opaque handles.  Index arrays of block-sparse matrices are 1-based, exactly as
 * BlockSparseMatrix stores them.  Numerical outcomes are statuses (IPMStatus), not errors.
 *
 * Reference interfaces replaced (paths inside the Mumblebee.jl project):
 *   mb_problem_create       IPMProblem(Q, B, f, g, μ, K[, P1, P2])        src/IPM/src/ipm/problem.jl:49-71
 *   mb_problem_create_csc   IPMProblem(Q::SparseMatrixCSC, B, f, g, μ, K, s; compress)
 *                                                                          src/IPM/src/ipm/problem.jl:84-127
 *   mb_solver_create        init(prob, settings; p0, d0, y0) → IPMSolver   src/IPM/src/ipm/solver/ipm.jl:431-491
 *   mb_solver_step          step!(solver) → IPMStatus                      src/IPM/src/ipm/solver/ipm.jl:577-774
 *   mb_solver_solve         solve!(solver)                                 src/IPM/src/ipm/solver/solver.jl:119-150
 *   mb_solver_result        result(solver, status) → IPMResult            src/IPM/src/ipm/solver/ipm.jl:30-74
 *   mb_solver_history       IPMHistory rows                                src/IPM/src/ipm/history/ipm.jl:1-71
 *   mb_solver_reinit        reinit!(s; p0, d0, y0, f, g)                   src/IPM/src/ipm/solver/ipm.jl:371-429
 *   mb_solver_timers        print_timers(s) (TimerOutput sections)         src/IPM/src/ipm/solver/ipm.jl:137-755
 *   mb_solver_frule         frule!(Δp, Δy, Δd, s, Δf, Δg, Δμ)              src/IPM/src/ipm/differential.jl:5-79
 *   mb_solver_rrule         rrule!(Δf, Δg, s, Δp, Δy, Δd)                  src/IPM/src/ipm/differential.jl:263-334
 *   mb_solver_frule2        frule2!(…, s, Δf1, Δg1, Δμ1, Δf2, Δg2, Δμ2)    src/IPM/src/ipm/differential.jl:82-260
 *   mb_batch_solve          solve(prob, settings) over many problems      src/IPM/src/ipm/solver/ipm.jl:798-804
 *   mb_settings             IPMSettings                                    src/IPM/src/ipm/settings/ipm.jl:1-18
 *   mb_extmul / mb_twomul   extmul!(c, A, b, α, β), twomul!(c, cc, A, b, α, β)
 *                                                                          src/BlockSparseArrays/src/comp/comp.jl:280-311
 */
#ifndef MUMBLEBEE_GPU_H
#define MUMBLEBEE_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* error codes */
#define MB_OK 0
#define MB_E_ARG (-1)      /* invalid argument or inconsistent shapes (the reference's @assert) */
#define MB_E_CUDA (-2)     /* a CUDA runtime call failed */
#define MB_E_NOMEM (-3)    /* device or host allocation failed */
#define MB_E_STATE (-4)    /* call not valid in the handle's current state */
#define MB_E_UNSUPPORTED (-5)
#define MB_E_TIMEOUT (-6)  /* a bounded device-side wait ran out (a grid barrier of the grid-cooperative
                              mode, settings.coop_wait): the solve was abandoned, the context stays usable */

/* cone kinds (the AbstractCone subtypes of src/IPM/src/cone/) */
#define MB_CONE_FREE 0     /* CofreeCone        cone/noc.jl */
#define MB_CONE_POS 1      /* PositiveCone      cone/pos.jl */
#define MB_CONE_SOC 2      /* SecondOrderCone   cone/soc.jl */
#define MB_CONE_SDP 3      /* SemidefiniteCone  cone/sdp.jl (svec) */
#define MB_CONE_EXP 4      /* ExponentialCone   cone/tdc/exp.jl */
#define MB_CONE_POW 5      /* PowerCone(α)      cone/tdc/pow.jl; α in cone_param */

/* IPMStatus (src/IPM/src/ipm/ipm.jl:1), same order */
enum mb_status {
    MB_CONTINUE = 0, MB_OPTIMAL, MB_NEAR_OPTIMAL, MB_STALLED, MB_NUMERICAL_FAILURE, MB_ITERATION_LIMIT,
    MB_PRIMAL_INFEASIBLE, MB_DUAL_INFEASIBLE, MB_ILL_POSED, MB_NEAR_PRIMAL_INFEASIBLE,
    MB_NEAR_DUAL_INFEASIBLE, MB_NEAR_ILL_POSED
};

/* algorithmic flops of one factorization above which a lone instance runs grid-cooperatively */
#define MB_LARGE_FLOPS 1.0e9

/* factor precision */
#define MB_PREC_FP64 0     /* FP64 factor */
#define MB_PREC_FP32 1     /* FP32 factor, FP64 refinement, residuals and termination tests */
#define MB_PREC_MIXED 2    /* FP32 factor until a KKT solve misses its tolerance; that iteration is
                              redone with the FP64 factor, which is kept for the rest of the solve */

/* IPMSettings (settings/ipm.jl:2-17) + precision.  Integer fields first, then doubles. */
typedef struct mb_settings {
    int32_t verbose;
    int32_t max_iter;          /* 100 */
    int32_t scale_max_iter;    /* 10  equilibration sweeps */
    int32_t refine_max_iter;   /* 10  KKT iterative-refinement passes */
    int32_t newton_max_iter;   /* 100 CG iterations per KKT solve */
    int32_t stable;            /* 0   1: the StableUzawaSolver factor (kkt/uzawa.jl:117-163): per-vertex
                                      Cholesky of H updated by the rows of B, no BᵀB, no ρ retry; a
                                      nonzero diagonal block of H that is not positive definite, or a
                                      zero pivot, ends the solve with NUMERICAL_FAILURE.  Needs
                                      precision MB_PREC_FP64 and Q without off-diagonal blocks
                                      (MB_E_UNSUPPORTED otherwise); never grid-cooperative */
    int32_t precision;         /* MB_PREC_FP64 */
    int32_t large;             /* 0: a single instance whose factorization exceeds MB_LARGE_FLOPS runs
                                  grid-cooperatively (all SMs help with its large fronts); 1: always
                                  for a single instance; -1: never */
    double step_frac;          /* 0.99 */
    double feas_tol;           /* 1e-8 */
    double gap_tol;            /* 1e-8 */
    double near_factor;        /* 1000 */
    double stall_tol;          /* 1e-3 */
    double refine_stall_tol;   /* 0.5 */
    double aug_tol;            /* 1e-7 */
    double infeas_abs;         /* 1e-8 */
    double infeas_rel;         /* 1e-8 */
    double coop_wait;          /* 60  seconds a CTA of the grid-cooperative mode waits at a grid barrier;
                                      when a wait runs out every CTA returns and the call fails with
                                      MB_E_TIMEOUT (<= 0: 60) */
    int32_t fp32_tiles;        /* 0   the FP32 factor's trailing-update tiles (MB_PREC_FP32, and the FP32
                                      iterations of MB_PREC_MIXED) on fronts of order >= 128: 2 on the
                                      tensor cores (tcgen05.mma kind::tf32, 3xTF32 split, per-step FP32
                                      read-out; those kernels run one CTA per SM), 1 on FFMA (two CTAs
                                      per SM), 0 the runtime's choice: the tensor cores for a lone
                                      grid-cooperative instance, FFMA for batches */
    int32_t reserved;          /* 0 */
} mb_settings;

/* BlockSparseMatrix{Float64,Int64} (BlockSparseArrays/src/block_sparse_matrix.jl:10-158), 1-based */
typedef struct mb_bsm {
    int64_t nout, nvtx, narc, ncol, nrow, nbnz;
    const int64_t* xsrc;   /* nvtx+1 */
    const int64_t* xcol;   /* nvtx+1 */
    const int64_t* xrow;   /* nout+1 */
    const int64_t* xblk;   /* narc+1 */
    const int64_t* tgt;    /* narc   */
    const double* val;     /* nbnz   */
} mb_bsm;

/* SparseMatrixCSC{Float64,Int64}, 1-based colptr/rowval */
typedef struct mb_csc {
    int64_t m, n;
    const int64_t* colptr;  /* n+1 */
    const int64_t* rowval;  /* nnz */
    const double* nzval;    /* nnz */
} mb_csc;

/* IPMResult scalars (result/ipm.jl:1-15) */
typedef struct mb_result {
    int32_t status;
    int32_t niter;
    int32_t nsolve;
    int32_t nfactor_retry;   /* ρ-regularized refactorizations (uzawa.jl:97-112) */
    int32_t nfactor;         /* numeric factorizations performed (including retries) */
    int32_t nfp32;           /* iterations accepted with the FP32 factor (MB_PREC_MIXED / _FP32) */
    int32_t nfallback;       /* iterations redone with the FP64 factor (MB_PREC_MIXED) */
    int32_t reserved;
    double mu, pres, dres, pobj, dobj;
    double factor_flops;     /* algorithmic flops of one factorization: Σ_fronts r³/3 + r²s + rs² */
} mb_result;

/* IPMHistoryRow (history/ipm.jl:1-4), integer and status fields stored as doubles */
typedef struct mb_history_row {
    double pres, dres, pobj, dobj, step;
    double piter, ppass, pstat, citer, cpass, cstat;
    double dmin, dmax, rho, delta, mu, chi;
} mb_history_row;

typedef struct mb_ctx mb_ctx;
typedef struct mb_problem mb_problem;
typedef struct mb_solver mb_solver;

/* library */
int mb_version(int32_t* major, int32_t* minor);
void mb_settings_default(mb_settings* s);

/* context: one device, one stream */
int mb_ctx_create(int32_t device, mb_ctx** out);
int mb_ctx_destroy(mb_ctx* ctx);
int mb_last_error(mb_ctx* ctx, char* buf, int64_t size);

/* problems (host-side block form; nothing is uploaded until a solver or batch uses it).  `ctx` may be
 * NULL for a host-only problem (front-end and symbolic analysis need no GPU); a solver needs a
 * problem created with a context, a batch takes its context from mb_batch_prepare. */
int mb_problem_create(mb_ctx* ctx, const mb_bsm* Q, const mb_bsm* B, const double* f, const double* g,
                      double mu, const int32_t* cone_kind, const double* cone_param,
                      const int64_t* P1, const int64_t* P2, mb_problem** out);
int mb_problem_create_csc(mb_ctx* ctx, const mb_csc* Q, const mb_csc* B, const double* f, const double* g,
                          double mu, int64_t ncone, const int32_t* cone_kind, const int64_t* cone_size,
                          const double* cone_param, double compress, mb_problem** out);
/* sizes of the block form: n, m, nvtx, nout, narc(B), nbnz(B), narc(Q), nbnz(Q) */
int mb_problem_info(const mb_problem* prob, int64_t* info8);
/* copy the block form out (arrays sized by mb_problem_info; 1-based) */
int mb_problem_export(const mb_problem* prob, int64_t* Bxsrc, int64_t* Bxcol, int64_t* Bxrow, int64_t* Bxblk,
                      int64_t* Btgt, double* Bval, int64_t* Qxsrc, int64_t* Qxblk, int64_t* Qtgt, double* Qval,
                      double* f, double* g, int32_t* kind, double* param, int64_t* P1, int64_t* P2);
int mb_problem_destroy(mb_problem* prob);

/* symbolic analysis (the host stand-in for CliqueTrees.symbolic, kkt/kkt.jl:23-53):
 * vperm (nvtx, 0-based user vertex per solver vertex, postordered), and the front partition */
int mb_problem_symbolic(const mb_problem* prob, int64_t* vperm, int64_t* nfront, int64_t* res0, int64_t* nres,
                        int64_t* nsep, int64_t* parent, int64_t cap);

/* device bytes one instance of this problem occupies under these settings (host-only query; the
 * serving loop admits requests by this footprint) */
int mb_problem_footprint(mb_problem* prob, const mb_settings* settings, int64_t* bytes);

/* single solver: init / step! / solve! / result */
int mb_solver_create(mb_problem* prob, const mb_settings* settings, const double* p0, const double* d0,
                     const double* y0, mb_solver** out);
int mb_solver_step(mb_solver* s, int32_t* status);
int mb_solver_solve(mb_solver* s, int32_t* status);
int mb_solver_result(mb_solver* s, double* p, double* d, double* y, mb_result* res);
int mb_solver_history(mb_solver* s, mb_history_row* rows, int32_t cap, int32_t* nrows);
/* reinit!(s; p0, d0, y0, f, g)  src/IPM/src/ipm/solver/ipm.jl:371-429: restart from the cone identity
 * (or the given p0/d0/y0, completed by shadows) with an empty history, on a new f (n) and/or g (m)
 * when given (user order); NULL keeps the current one.  The equilibration, Q, B and BᵀB stay. */
int mb_solver_reinit(mb_solver* s, const double* p0, const double* d0, const double* y0, const double* f,
                     const double* g);
/* frule!(Δp, Δy, Δd, s, Δf, Δg, Δμ)  src/IPM/src/ipm/differential.jl:5-79: tangents of the current
 * iterate for seeds on f (n), g (m) and μ; user order, NULL seed = 0, NULL output = skipped.  The
 * factorization at the current iterate is redone (FP64); MB_E_STATE when it fails. */
int mb_solver_frule(mb_solver* s, const double* df, const double* dg, double dmu, double* dp, double* dy, double* dd);
/* frule2!  src/IPM/src/ipm/differential.jl:82-260: tangents for two seed sets (Δf1 Δg1 Δμ1,
 * Δf2 Δg2 Δμ2) and the second-order tangent; out = nine output pointers Δp1 Δy1 Δd1 Δp2 Δy2 Δd2
 * Δp12 Δy12 Δd12 (each NULL to skip); as mb_solver_frule */
int mb_solver_frule2(mb_solver* s, const double* df1, const double* dg1, double dmu1, const double* df2,
                     const double* dg2, double dmu2, double* const* out);
/* rrule!(Δf, Δg, s, Δp, Δy, Δd)  src/IPM/src/ipm/differential.jl:263-334: cotangents of f, g and μ
 * for seeds on p (n), y (m), d (n); as mb_solver_frule */
int mb_solver_rrule(mb_solver* s, const double* dp, const double* dy, const double* dd, double* df, double* dg,
                    double* dmu);
/* the solver's section timers (print_timers, the TimerOutput of IPMSolver): MB_NSECTIONS + 2 doubles,
 * laid out as for mb_batch_timers */
int mb_solver_timers(mb_solver* s, double* out, int64_t cap);
int mb_solver_destroy(mb_solver* s);

/* batched solve: every problem solved by a persistent launch (one CTA per instance at a time).
 * With grid = 0 and 1024 or more problems the call is split into two or four chunks (problems
 * taken largest first by an estimate of their cost), each planned, uploaded and launched on its
 * own stream, so host planning overlaps device work; each instance is solved exactly as alone.  Outputs per problem i:
 * p_out[i] (n_i), d_out[i] (n_i), y_out[i] (m_i), results[i]; any output pointer may be NULL to
 * skip it.  `grid` = CTAs of the persistent launch (0 = two per SM). */
int mb_batch_solve(mb_ctx* ctx, mb_problem* const* probs, int32_t nprob, const mb_settings* settings,
                   int32_t grid, double* const* p_out, double* const* d_out, double* const* y_out,
                   mb_result* results);

/* the same with every input already resident on the device: set up once, then time solves.
 * mb_batch_prepare uploads, mb_batch_run launches and waits (device time in *ms), mb_batch_fetch
 * copies results back. */
typedef struct mb_batch mb_batch;
int mb_batch_prepare(mb_ctx* ctx, mb_problem* const* probs, int32_t nprob, const mb_settings* settings,
                     mb_batch** out);
int mb_batch_run(mb_batch* b, int32_t grid, float* ms);
int mb_batch_fetch(mb_batch* b, double* const* p_out, double* const* d_out, double* const* y_out,
                   mb_result* results);
int mb_batch_stats(mb_batch* b, int64_t* stats8);   /* bytes: input, workspace, factor; kernel launches */
/* per-instance section timers after mb_batch_fetch, MB_NSECTIONS + 2 doubles each: SM clocks spent
 * in equilibrate, BᵀB, scale, initkkt, predictor, corrector, maxsteps, triangular solves, matvecs,
 * KKT assembly, residuals, getaug, and inside initkkt the factor's trailing updates, diagonal
 * blocks, panel rows and extend-add; then the number of triangular-solve sweeps and of matvecs
 * (the TimerOutputs sections of the reference, solver/ipm.jl:137-755, split further) */
#define MB_NSECTIONS 16
int mb_batch_timers(mb_batch* b, double* out, int64_t cap);
/* per-instance device timestamps after mb_batch_fetch, 2 int64 each: the GPU global timer (ns)
 * when a CTA took the instance from the work queue and when its solve finished.  Latency of an
 * instance submitted with the launch = finish − the launch's earliest take. */
int mb_batch_times(mb_batch* b, int64_t* out, int64_t cap);
int mb_batch_destroy(mb_batch* b);

/* mb_batch_solve without any device allocation: every device array of the batch is placed in one
 * fixed, file-scope device scratch of MB_STATIC_SCRATCH_BYTES.  No counterpart in the reference
 * (Mumblebee.jl allocates its solver state per solve).  It is for callers that may not allocate
 * device memory during service: a process that reserved its HBM budget up front (a cudaMalloc
 * could fail or take it past the budget mid-service), and a process whose other streams run
 * latency-critical work (cudaFree, and cudaMalloc when it grows the heap, synchronise the whole
 * device).  It calls no cudaMalloc, cudaMallocHost or cudaFree and no allocating library routine;
 * the host-side symbolic planning still uses ordinary heap memory.
 * Limit: all instances together (their mb_problem_footprint bytes plus a few KB of alignment) must
 * fit in MB_STATIC_SCRATCH_BYTES (32 MiB, e.g. two 400-asset portfolio instances); larger inputs
 * return MB_E_NOMEM before any device work, with the needed size in mb_last_error.
 * The scratch is one per device and per process: calls that overlap in time on one device (two
 * host threads, or two contexts on the same device) race on it and corrupt each other's results.
 * Every call looks up the scratch's device address with that device current (the first call on a
 * device may load the module, so make it before any stream capture begins); the lookup is repeated
 * on each call, so a cudaDeviceReset by the host application between calls is harmless (the
 * scratch then starts over with undefined contents, which every call overwrites before use).
 * Arguments, outputs and the grid-cooperative rule for a lone large instance (settings.large) as
 * mb_batch_solve; the control block of that mode lives in the scratch too. */
#define MB_STATIC_SCRATCH_BYTES (32u << 20)
int mb_batch_solve_static(mb_ctx* ctx, mb_problem* const* probs, int32_t nprob, const mb_settings* settings,
                          int32_t grid, double* const* p_out, double* const* d_out, double* const* y_out,
                          mb_result* results);

/* Serving loop (continuous batching).  No counterpart in the reference, which solves one problem
 * per call: a server owns one device arena of `arena_bytes` and a ring of `capacity` request
 * slots.  Requests are planned on `nplanners` host threads (0 = half the cores), admitted in
 * arrival order while their footprint (mb_problem_footprint plus alignment) fits the arena and a
 * slot is free, and launched in admission waves on a pool of streams, so they start on SMs as
 * earlier requests' CTAs retire while those keep running; each is copied back as it finishes.
 * Results equal those of mb_batch_solve for the same problem.  The problem must stay alive until
 * its ticket has finished.  States: 0 queued, 1 planned, 2 running,
 * 3 done, 4 failed (mb_server_result returns the failure's code and message). */
typedef struct mb_server mb_server;
int mb_server_create(mb_ctx* ctx, const mb_settings* settings, int64_t arena_bytes, int32_t capacity,
                     int32_t nplanners, mb_server** out);
int mb_server_submit(mb_server* s, mb_problem* prob, int64_t* ticket);
int mb_server_poll(mb_server* s, int64_t ticket, int32_t* state);
int mb_server_wait(mb_server* s, int64_t ticket, double timeout_s, int32_t* state);
/* outputs as mb_solver_result; times5 = [submitted, admitted, finished] (host seconds since the
 * server started) and the device global-timer stamps (ns) of the solve's start and end.  Releases
 * the ticket. */
int mb_server_result(mb_server* s, int64_t ticket, double* p, double* d, double* y, mb_result* res,
                     double* times5);
/* queued, planned, running, completed, failed, kernel launches, arena bytes in use, arena bytes */
int mb_server_stats(mb_server* s, int64_t* stats8);
int mb_server_destroy(mb_server* s);

/* ---- compensated block-sparse products --------------------------------------------------------
 * extmul!(c, A, b, α, β[, s, cs]) and twomul!(c, cc, A, b, α, β[, s, cs]) of BlockSparseArrays
 * (src/comp/comp.jl:280-311, src/comp/twogemv.jl:87-121): c ← α op(A) b + β c with op(A) = A
 * (trans = 0) or Aᵀ (trans = 1), phase 1 accumulated with error-free transformations.  extmul
 * leaves c as accurate as if computed in doubled precision and rounded once; twomul leaves the
 * normalized pair (c, cc) whose hi part equals extmul's c bitwise.  Each output entry takes its
 * terms in the reference's order, so results are bitwise those of the reference.  b has ncol
 * (trans = 0) or nrow (trans = 1) entries, c / cc the other count; c is read only when β ≠ 0; s
 * and cs (both or neither) receive the unscaled pair of op(A) b.  Host buffers; the call returns
 * when the outputs are written. */
typedef struct mb_matrix mb_matrix;
/* uploads A (mb_bsm, 1-based) once, as scalar CSR and CSC views of all its stored block entries */
int mb_matrix_create(mb_ctx* ctx, const mb_bsm* A, mb_matrix** out);
int mb_matrix_destroy(mb_matrix* A);
int mb_extmul(mb_matrix* A, int32_t trans, const double* b, double alpha, double beta, double* c,
              double* s, double* cs);
int mb_twomul(mb_matrix* A, int32_t trans, const double* b, double alpha, double beta, double* c,
              double* cc, double* s, double* cs);

#ifdef __cplusplus
}
#endif
#endif
