"""Compensated block-sparse products on the device: extmul! and twomul! of BlockSparseArrays
(src/comp/comp.jl:280-311, src/comp/twogemv.jl:87-121), through the C ABI (mb_matrix_create,
mb_extmul, mb_twomul).

    A = BlockSparseMatrix(blocksparse(M, colsizes, rowsizes))
    extmul(c, A, b, alpha, beta)           # c ← α A b + β c, as if in doubled precision
    extmul(c, A.T, b, alpha, beta)         # c ← α Aᵀ b + β c
    twomul(c, cc, A, b, alpha, beta)       # the normalized pair (c, cc); c equals extmul's bitwise

Results are bitwise those of the reference: every output entry takes its terms in the order the
reference's block loops give it.  c is read only when β ≠ 0; s and cs, when given, receive the
unscaled pair of op(A) b (the reference's workspace arguments)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .ipm import Context, _a64, _f64, _p


def blocksparse(M, colsizes, rowsizes, keep_zero_blocks: bool = False) -> dict:
    """The BlockSparseMatrix fields (1-based) of the dense matrix M partitioned into column blocks
    (vertices) of sizes `colsizes` and row blocks of sizes `rowsizes`.  Each block with a nonzero
    entry (every block with `keep_zero_blocks`) is stored dense, column-major; arcs run in
    ascending target order, as block_sparse_matrix.jl:658-716 requires."""
    M = np.asarray(M, dtype=np.float64)
    nrow, ncol = M.shape
    xcol = np.concatenate([[0], np.cumsum(colsizes)]).astype(np.int64)
    xrow = np.concatenate([[0], np.cumsum(rowsizes)]).astype(np.int64)
    if xcol[-1] != ncol or xrow[-1] != nrow:
        raise ValueError("block sizes do not add up to the matrix shape")
    xsrc, tgt, xblk, val = [0], [], [0], []
    for v in range(len(colsizes)):
        for u in range(len(rowsizes)):
            blk = M[xrow[u]:xrow[u + 1], xcol[v]:xcol[v + 1]]
            if blk.size == 0 or (not keep_zero_blocks and not blk.any()):
                continue
            tgt.append(u)
            val.append(blk.ravel(order="F"))
            xblk.append(xblk[-1] + blk.size)
        xsrc.append(len(tgt))
    val = np.concatenate(val) if val else np.zeros(0)
    return dict(nout=len(rowsizes), nvtx=len(colsizes), narc=len(tgt), ncol=ncol, nrow=nrow, nbnz=int(val.size),
                xsrc=np.asarray(xsrc, np.int64) + 1, xcol=xcol + 1, xrow=xrow + 1,
                xblk=np.asarray(xblk, np.int64) + 1, tgt=np.asarray(tgt, np.int64) + 1, val=val)


class BlockSparseMatrix:
    """A BlockSparseMatrix resident on the device (mb_matrix): uploaded once, used by any number
    of products.  `A.T` is its transpose for extmul / twomul."""

    def __init__(self, d: dict, ctx: Context | None = None):
        self.ctx = ctx or Context.default()
        L = self.ctx.L
        a = {k: _a64(d[k]) for k in ("xsrc", "xcol", "xrow", "xblk", "tgt")}
        a["val"] = _f64(d["val"])
        s = _lib.mb_bsm(d["nout"], d["nvtx"], d["narc"], d["ncol"], d["nrow"], d["nbnz"],
                        *[_p(a[k], C.c_int64) for k in ("xsrc", "xcol", "xrow", "xblk", "tgt")],
                        _p(a["val"], C.c_double))
        h = C.c_void_p()
        _lib.check(L.mb_matrix_create(self.ctx.h, C.byref(s), C.byref(h)), self.ctx, "mb_matrix_create")
        self.h = h
        self.shape = (int(d["nrow"]), int(d["ncol"]))

    @property
    def T(self) -> "_Transpose":
        return _Transpose(self)

    def __del__(self):
        if getattr(self, "h", None):
            self.ctx.L.mb_matrix_destroy(self.h)
            self.h = None


class _Transpose:
    def __init__(self, A: BlockSparseMatrix):
        self.A = A
        self.shape = (A.shape[1], A.shape[0])


def _out(x, n, name):
    if not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous and x.flags.writeable):
        raise TypeError(f"{name} must be a writable contiguous float64 array")
    if x.shape != (n,):
        raise ValueError(f"{name} must have length {n}")
    return x


def _run(c, cc, A, b, alpha, beta, s, cs):
    trans = isinstance(A, _Transpose)
    M = A.A if trans else A
    nout, nin = A.shape
    c = _out(c, nout, "c")
    if cc is not None:
        cc = _out(cc, nout, "cc")
    if (s is None) != (cs is None):
        raise ValueError("s and cs go together")
    if s is not None:
        s, cs = _out(s, nout, "s"), _out(cs, nout, "cs")
    b = _f64(b)
    if b.shape != (nin,):
        raise ValueError(f"b must have length {nin}")
    pd = lambda x: _p(x, C.c_double)
    L = M.ctx.L
    if cc is None:
        rc = L.mb_extmul(M.h, int(trans), pd(b), float(alpha), float(beta), pd(c), pd(s), pd(cs))
    else:
        rc = L.mb_twomul(M.h, int(trans), pd(b), float(alpha), float(beta), pd(c), pd(cc), pd(s), pd(cs))
    _lib.check(rc, M.ctx, "mb_extmul" if cc is None else "mb_twomul")
    return c, cc


def extmul(c, A, b, alpha, beta, s=None, cs=None):
    """extmul!(c, A, b, α, β[, s, cs]): c ← α op(A) b + β c in place; returns c."""
    return _run(c, None, A, b, alpha, beta, s, cs)[0]


def twomul(c, cc, A, b, alpha, beta, s=None, cs=None):
    """twomul!(c, cc, A, b, α, β[, s, cs]): the normalized pair (c, cc) in place; returns it."""
    return _run(c, cc, A, b, alpha, beta, s, cs)
