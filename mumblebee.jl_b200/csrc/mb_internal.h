// Internal layout shared by the host runtime (mb_host.cpp) and the device solver
// (mb_solver.cu).  One `DevInst` describes one problem instance resident in HBM; the batched
// solver kernel assigns one CTA to one instance and runs the whole interior-point solve there.
#pragma once
#include <cstdint>

namespace mb {

enum ConeKind { CONE_FREE = 0, CONE_POS = 1, CONE_SOC = 2, CONE_SDP = 3, CONE_EXP = 4, CONE_POW = 5 };

// IPMStatus (src/IPM/src/ipm/ipm.jl:1), KKTStatus (kkt/kkt.jl:1), CGStatus (kkt/cg.jl:1-6)
enum IPMStatus { CONTINUE = 0, OPTIMAL, NEAR_OPTIMAL, STALLED, NUMERICAL_FAILURE, ITERATION_LIMIT,
                 PRIMAL_INFEASIBLE, DUAL_INFEASIBLE, ILL_POSED, NEAR_PRIMAL_INFEASIBLE,
                 NEAR_DUAL_INFEASIBLE, NEAR_ILL_POSED };
enum KKTStatus { KKT_CONTINUE = 0, KKT_SOLVED, KKT_STAGNATED, KKT_ITMAX, KKT_NUMERICAL_FAILURE, KKT_IRMAX };
enum CGStatus { CG_CONTINUE = 0, CG_SOLVED, CG_NUMERICAL_FAILURE, CG_ITMAX };

// Settings, field order shared with mb_settings in include/mumblebee_gpu.h
struct Settings {
    int32_t verbose, max_iter, scale_max_iter, refine_max_iter, newton_max_iter, stable, precision, reserved;
    double step_frac, feas_tol, gap_tol, near_factor, stall_tol, refine_stall_tol, aug_tol, infeas_abs, infeas_rel;
};

// One history row: the 17 fields of IPMHistoryRow (history/ipm.jl:1-4), stored as doubles.
struct Row {
    double pres, dres, pobj, dobj, step;
    double piter, ppass, pstat, citer, cpass, cstat;
    double dmin, dmax, rho, delta, mu, chi;
};
constexpr int ROW_DOUBLES = 17;

// Block-sparse matrix on the device, 0-based: block-CSC by vertex (column blocks) plus a
// block-CSR arc index by out-vertex (row blocks) so both A x and Aᵀ x are gathers.
struct DevBSM {
    int nout, nvtx, narc, ncol, nrow;
    const int* xsrc;        // nvtx+1
    const int* xcol;        // nvtx+1
    const int* xrow;        // nout+1
    const int* tgt;         // narc
    const int64_t* xblk;    // narc+1
    double* val;            // nbnz (mutable: equilibration scales in place)
    const int* rptr;        // nout+1: arcs of out-vertex u are rarc[rptr[u] .. rptr[u+1])
    const int* rarc;        // arc ids grouped by target
    const int* rvtx;        // the source vertex of each grouped arc
    const int* rowout;      // nrow: out-vertex of each row
    const int* colvtx;      // ncol: vertex of each column
};

struct DevInst {
    int n, m, nvtx, nfront;
    int nu;                 // cone degree ν
    int has_p0, has_d0, has_y0;
    double mut;             // barrier target μ′ (0 = exact solve)
    DevBSM B, Q;            // Q shares B's vertex/column layout; Q.xrow == Q.xcol
    double* H;              // values of H (Q's pattern)
    const int* qdiag;       // per vertex: arc of the diagonal block in Q/H, -1 if none
    const int64_t* hpos;    // per Q/H arc: offset in F of the block's (0,0) entry, -1 if the block is upper
    const int* hld;         // per Q/H arc: leading dimension of its front
    const int* kind;        // cone kind per vertex
    const double* kpar;     // cone parameter per vertex
    const int64_t* cxblk;   // cache offsets per vertex (nvtx+1)
    double* cache;
    int wsize;              // per-cone workspace length (max over cones)
    // fronts (multifrontal): front f owns scalar columns [fres0[f], fres0[f]+fnres[f]) and the
    // separator rows fsep[fsepp[f] .. fsepp[f+1]); its (nres+nsep)^2 column-major storage starts at
    // fptr[f]; frel maps separator rows to positions in the parent's row list.
    const int* fres0; const int* fnres; const int* fnsep; const int* fparent;
    const int64_t* fptr; const int* fsepp; const int* fsep; const int* frel;
    int64_t fsize;
    // L = BᵀB in front layout, built on the device from B at set-up
    double* Finit;          // fsize doubles
    void* F;                // fsize FT (double or float)
    // pristine inputs (never written) and their working copies (equilibrated in place at init)
    const double* Bval0; const double* Qval0; const double* f0; const double* g0;
    const double* p0; const double* d0; const double* y0;
    double* f; double* g;
    double* pscl; double* yscl;
    // iterates and workspace
    double* p; double* d; double* y;
    double* vn;             // NVEC_N n-vectors
    double* vm;             // NVEC_M m-vectors
    double* vv;             // NVEC_V nvtx-vectors
    double* work;           // cone workspace (wsize per warp)
    const int* vfront;      // per vertex: its front
    double* po; double* dout; double* yo;   // result iterates (user scaling, solver order)
    double* hist;           // max_iter+1 rows (ROW_DOUBLES each)
    double* uhist;          // refine_max_iter + 2
    double* cghist;         // newton_max_iter + 1
    // outputs
    int* status;            // [0] IPM status, [1] rows written, [2] factor retries, [3] error code
    double* scal;           // mu, pres, dres, pobj, dobj, nf, ng, sf, sg, nB, plus spares
};

constexpr int NVEC_N = 12;  // Df Qp wf Dpa Dda Dp Dd df dx cgw  tmp1 tmp2
constexpr int NVEC_M = 8;   // Dg Dya Dy dg dy cgp tmp1 tmp2
constexpr int NVEC_V = 6;   // step spsd flag vscl vnrm vswp
constexpr int NSCAL = 16;   // mu pres dres pobj dobj | nf ng sf sg nB
constexpr int NSTAT = 4;    // status, history rows, factor retries, error

// kernel modes: a full solve, or the pieces used by the step-wise API
enum Mode { MODE_SOLVE = 0, MODE_INIT = 1, MODE_STEP = 2, MODE_RESULT = 3 };

}  // namespace mb
