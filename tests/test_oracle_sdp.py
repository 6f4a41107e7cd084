"""Known-answer tests of the oracle's semidefinite cone (src/IPM/src/cone/sdp.jl, eig.jl,
cone/utils.jl restated in oracle/oracle_sdp.hpp) against numpy linear algebra: the NT Hessian
block maps p to d, the shadow is the inverse, the zero corrector is σμ p⁻¹ − d, the steps are the
largest PSD-preserving steps, eigmin and the Jacobi SVD match numpy."""
import numpy as np
import pytest

import oracle

R2 = np.sqrt(2.0)


def svec(M):
    d = M.shape[0]
    return np.concatenate([[M[j, j]] + [R2 * M[i, j] for i in range(j + 1, d)] for j in range(d)])


def smat(v):
    d = int((np.sqrt(1 + 8 * len(v)) - 1) // 2)
    M = np.zeros((d, d)); k = 0
    for j in range(d):
        M[j, j] = v[k]; k += 1
        for i in range(j + 1, d):
            M[i, j] = M[j, i] = v[k] / R2; k += 1
    return M


def spd(rng, d, cond=10.0):
    Q, _ = np.linalg.qr(rng.standard_normal((d, d)))
    return Q @ np.diag(np.exp(rng.uniform(0, np.log(cond), d))) @ Q.T


def sym(rng, d):
    A = rng.standard_normal((d, d))
    return (A + A.T) / 2


@pytest.mark.parametrize("d", [1, 2, 3, 4, 7, 8, 9, 13])
def test_scale_shadow_corr0(d):
    rng = np.random.default_rng(d)
    P, D = spd(rng, d), spd(rng, d)
    n = d * (d + 1) // 2
    z = np.zeros(n)
    r = oracle.sdp_probe(svec(P), svec(D), z, z, 0.3)
    assert r["ok"] and r["shadow_ok"]
    H = r["H"]
    np.testing.assert_allclose(H, H.T, rtol=0, atol=1e-10 * np.abs(H).max())
    np.testing.assert_allclose(H @ svec(P), svec(D), rtol=1e-9, atol=1e-9)      # W P W = D
    np.testing.assert_allclose(r["shadow"], svec(np.linalg.inv(P)), rtol=1e-9, atol=1e-10)
    np.testing.assert_allclose(r["spsd"], np.trace(np.linalg.inv(P) @ np.linalg.inv(D)), rtol=1e-10)
    R, S = r["R"], r["S"]
    np.testing.assert_allclose(R @ R.T, np.linalg.inv(P), rtol=1e-8, atol=1e-10)   # R Rᵀ = P⁻¹
    np.testing.assert_allclose(R.T @ S, np.eye(d), atol=1e-10)                     # Rᵀ S = I
    np.testing.assert_allclose(r["corr0"], svec(0.3 * np.linalg.inv(P) - D), rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(r["corr"], r["corr0"], rtol=0, atol=1e-12)          # Δ = 0
    assert r["tp"] == 1.0 and r["td"] == 1.0


@pytest.mark.parametrize("d", [1, 2, 3, 5, 8, 11])
def test_steps_are_largest_psd_steps(d):
    rng = np.random.default_rng(100 + d)
    P, D = spd(rng, d), spd(rng, d)
    dP, dD = 3 * sym(rng, d), 3 * sym(rng, d)
    r = oracle.sdp_probe(svec(P), svec(D), svec(dP), svec(dD), 0.1)
    assert r["ok"]
    for X, dX, tau in ((P, dP, r["tp"]), (D, dD, r["td"])):
        L = np.linalg.cholesky(X)
        lam = np.linalg.eigvalsh(np.linalg.solve(L, np.linalg.solve(L, dX).T).T).min()
        want = 1.0 / max(1.0, -lam)
        assert tau == pytest.approx(want, rel=1e-9)
        if tau < 1:
            assert np.linalg.eigvalsh(X + tau * dX).min() == pytest.approx(0.0, abs=1e-8 * np.abs(X).max())


@pytest.mark.parametrize("d", [2, 4, 6])
def test_corrector_formula(d):
    # r = svec(R Ŵ Rᵀ), Ŵ off-diagonal −(sᵢXᵢⱼ + sⱼXⱼᵢ)/(sᵢ+sⱼ), diagonal σμ − sⱼ² − Xⱼⱼ, X = (RᵀΔP R)(SᵀΔD S)
    rng = np.random.default_rng(200 + d)
    P, D = spd(rng, d), spd(rng, d)
    dP, dD = sym(rng, d), sym(rng, d)
    r = oracle.sdp_probe(svec(P), svec(D), svec(dP), svec(dD), 0.7)
    R, S, s = r["R"], r["S"], r["s"]
    X = (R.T @ dP @ R) @ (S.T @ dD @ S)
    W = np.zeros((d, d))
    for j in range(d):
        for i in range(j):
            W[i, j] = W[j, i] = -(s[i] * X[i, j] + s[j] * X[j, i]) / (s[i] + s[j])
        W[j, j] = 0.7 - s[j] ** 2 - X[j, j]
    np.testing.assert_allclose(r["corr"], svec(R @ W @ R.T), rtol=1e-9, atol=1e-10)


def test_scale_rejects_non_pd():
    P = np.diag([1.0, -1.0, 2.0])
    r = oracle.sdp_probe(svec(P), svec(np.eye(3)), np.zeros(6), np.zeros(6), 1.0)
    assert not r["ok"] and not r["shadow_ok"]


@pytest.mark.parametrize("d", [1, 2, 3, 4, 6, 10, 17])
def test_eigmin_and_jacobi_svd(d):
    rng = np.random.default_rng(300 + d)
    M = sym(rng, d) * 10.0 ** rng.uniform(-3, 3)
    A = rng.standard_normal((d, d))
    lam_sturm, lam_small, U, sv, ok = oracle.sdp_eig(M, np.inf, A)
    want = np.linalg.eigvalsh(M).min()
    scale = np.abs(M).max()
    assert lam_sturm == pytest.approx(want, abs=1e-12 * scale)
    if d <= 3:
        assert lam_small == pytest.approx(want, abs=1e-12 * scale)
    assert ok
    np.testing.assert_allclose(np.sort(sv), np.sort(np.linalg.svd(A, compute_uv=False)), rtol=1e-12)
    np.testing.assert_allclose(U.T @ U, np.eye(d), atol=1e-12)
    np.testing.assert_allclose(U.T @ A @ A.T @ U, np.diag(sv ** 2), atol=1e-10 * np.abs(A).max() ** 2 * d)


# ----------------------------------------------------------------------------- whole solves
from helpers import block_problem, oracle_solve          # noqa: E402
from mumblebee_b200 import generators as G               # noqa: E402


@pytest.mark.parametrize("d,seed", [(2, 0), (5, 1), (9, 2)])
def test_oracle_sdp_eigmin_known_answer(d, seed):
    pb, lam = G.sdp_eigmin(d, seed)
    _, r = oracle_solve(block_problem(pb))
    assert r["status"] == "OPTIMAL"
    assert abs(r["pobj"] - lam) <= 1e-7 * max(1.0, abs(lam))


@pytest.mark.parametrize("pb", [G.sdp(3, 4, 10, 0.3, 0, 0), G.sdp(2, 6, 15, 0.3, 5, 1), G.maxcut(12, 6, 2, 0)],
                         ids=["sdp3x4", "sdp2x6_pos", "maxcut12"])
def test_oracle_sdp_solves_to_optimal_psd_iterates(pb):
    prob = block_problem(pb)
    s, r = oracle_solve(prob)
    assert r["status"] == "OPTIMAL"
    assert r["pres"] < 1e-8 and r["dres"] < 1e-8
    assert abs(r["pobj"] - r["dobj"]) <= 1e-8 * max(1.0, abs(r["pobj"]))
    off = 0
    for k, n in zip(pb["kinds"], pb["sizes"]):
        if k == G.CONE_SDP:
            for v in (r["p"], r["d"]):
                assert np.linalg.eigvalsh(smat(v[off:off + n])).min() > -1e-8
        off += n
