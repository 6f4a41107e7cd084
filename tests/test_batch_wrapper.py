"""Host logic of the batched Python entry points (no GPU): the per-problem output pointers that
batch_solve passes to the C library point at the right slices of its contiguous buffers, and the
results it returns read back every field of the mb_result array in the right place."""
import ctypes as C

import numpy as np

from mumblebee_b200 import ipm as I


class _Prob:
    """the two things _batch_call reads from a problem: its shape and its handle"""

    def __init__(self, n, m, h):
        self._info = {"n": n, "m": m}
        self.h = C.c_void_p(h)

    def _nm(self):
        return self._info["n"], self._info["m"]


class _Ctx:
    h = None


def _fake_solve(calls):
    """a stand-in for mb_batch_solve: writes p[i][j] = 1000 i + j, d = -(1000 i + j), y = 0.5 + 1000 i + j
    through the pointer arrays and per-problem result fields derived from i"""

    def fn(h, arr, k, cs, grid, P, D, Y, res):
        calls.append((k, grid, [arr[i] for i in range(k)]))
        for i in range(k):
            n, m = _SHAPES[i]
            for j in range(n):
                P[i][j] = 1000.0 * i + j
                D[i][j] = -(1000.0 * i + j)
            for j in range(m):
                Y[i][j] = 0.5 + 1000.0 * i + j
            r = res[i]
            r.status, r.niter, r.nsolve = i % 12, 10 + i, 20 + i
            r.nfactor_retry, r.nfactor, r.nfp32, r.nfallback = i % 3, 30 + i, i % 5, i % 2
            r.mu, r.pres, r.dres = 1e-9 * (i + 1), 1e-10 * (i + 1), 2e-10 * (i + 1)
            r.pobj, r.dobj, r.factor_flops = float(i), float(i) - 1e-9, 1e6 * (i + 1)
        return 0

    return fn


_SHAPES = [(3, 2), (1, 0), (5, 4), (0, 1), (7, 3)]


def test_batch_call_maps_outputs_and_results(monkeypatch):
    monkeypatch.setattr(I, "check", lambda rc, h, what: None)
    probs = [_Prob(n, m, 100 + i) for i, (n, m) in enumerate(_SHAPES)]
    calls = []
    out = I._batch_call(_fake_solve(calls), probs, I.IPMSettings(), 7, _Ctx(), "fake")
    assert len(calls) == 1 and calls[0][0] == len(probs) and calls[0][1] == 7
    assert calls[0][2] == [100 + i for i in range(len(probs))]   # problem handles in order
    for i, (r, (n, m)) in enumerate(zip(out, _SHAPES)):
        assert r.p.shape == (n,) and r.d.shape == (n,) and r.y.shape == (m,)
        np.testing.assert_array_equal(r.p, 1000.0 * i + np.arange(n))
        np.testing.assert_array_equal(r.d, -(1000.0 * i + np.arange(n)))
        np.testing.assert_array_equal(r.y, 0.5 + 1000.0 * i + np.arange(m))
        assert r.status == I.IPMStatus(i % 12) and isinstance(r.status, I.IPMStatus)
        assert (r.niter, r.nsolve, r.nfactor_retry, r.nfactor, r.nfp32, r.nfallback) == \
            (10 + i, 20 + i, i % 3, 30 + i, i % 5, i % 2)
        assert (r.mu, r.pres, r.dres) == (1e-9 * (i + 1), 1e-10 * (i + 1), 2e-10 * (i + 1))
        assert (r.pobj, r.dobj, r.factor_flops) == (float(i), float(i) - 1e-9, 1e6 * (i + 1))
        assert len(r.history) == 0


def test_batch_call_views_do_not_overlap(monkeypatch):
    monkeypatch.setattr(I, "check", lambda rc, h, what: None)
    probs = [_Prob(n, m, 1) for n, m in _SHAPES]
    out = I._batch_call(_fake_solve([]), probs, I.IPMSettings(), 0, _Ctx(), "fake")
    out[2].p[:] = -1.0   # writing one problem's view leaves its neighbours alone
    np.testing.assert_array_equal(out[0].p, np.arange(3.0))
    np.testing.assert_array_equal(out[4].p, 4000.0 + np.arange(7))


def test_result_dtype_matches_the_c_struct():
    assert I._RESULT_DTYPE.itemsize == C.sizeof(I.mb_result)
    for name, _ in I.mb_result._fields_:
        assert I._RESULT_DTYPE.fields[name][1] == getattr(I.mb_result, name).offset


def test_empty_batches_return_empty_lists():
    assert I.batch_solve([]) == []
    assert I.batch_solve_static([]) == []


def test_problem_shape_is_read_once(monkeypatch):
    calls = []

    class _L:
        @staticmethod
        def mb_problem_info(h, a):
            calls.append(1)
            a[0], a[1] = 11, 4
            return 0

        @staticmethod
        def mb_problem_destroy(h):
            return 0

    p = I.IPMProblem.__new__(I.IPMProblem)
    p.ctx = type("Ctx", (), {"L": _L})()
    p.h = C.c_void_p(1)
    assert p.info()["n"] == 11 and p._nm() == (11, 4) and p.info()["m"] == 4
    assert len(calls) == 1
